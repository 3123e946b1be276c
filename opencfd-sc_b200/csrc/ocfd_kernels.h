// ocfd_kernels.h -- launch interface between the instance code (ocfd_api.cu)
// and the kernels (ocfd_face.cu, ocfd_update.cu, ocfd_aux.cu).
#pragma once

#include <cuda_runtime.h>

#include "ocfd_device.cuh"

namespace ocfd {

// Central-difference coefficients per direction (OCFD_dxyz_viscous.f90:9-16).
struct DCoef {
  double h[3];
  double a1[3], a2[3], a3[3];          // CD6
  double c1[3], c2[3], c3[3], c4[3];   // CD8
};

// Arguments of the viscous-gradient kernel (stress and heat flux -> Ev).
template <typename R, typename S>
struct ViscArgs {
  Grid g;
  Phys ph;
  DCoef dc;
  const S* d;
  const S* u;
  const S* v;
  const S* w;
  const S* T;
  const float* q4;   // FP32 instances: u,v,w,T interleaved (haloed, 4 floats a point); u..T unused
  const S* met[22];  // haloed metrics (OCFD_M_* order); S = double or float copies
  R* ev;             // Ev1..Ev3, interior points, (d*n + point)*4 + component
};

// Arguments of the stage-tail kernels (flux difference, viscous divergence,
// RK3, primitive recovery, face refresh, periodic halo).
template <typename R>
struct UpdArgs {
  Grid g;
  Phys ph;
  DCoef dc;
  const R* hf[3];      // face fluxes of x, y, z
  long long fs[3];     // per-variable strides
  int fper[3];         // faces stored 1..n (periodic: face 0 == face n)
  double h_1[3];       // 1/hx, 1/hy, 1/hz
  const R* ev;         // viscous fluxes ((d*n + point)*4 + component) or nullptr
  const double* ajac;  // haloed Ajac
  const double* pd;    // haloed d,u,v,w (mass force)
  const double* pu;
  const double* pv;
  const double* pw;
  double* du;          // 5 interior arrays
  double* f;
  const double* fn;
  double* prim[5];     // haloed d,u,v,w,T (T: the buffer being written)
  const double* told;  // haloed T of the previous stage (negative-T repair)
  float* p32[5];       // FP32 copy of d in p32[0] (mixed precision) or nullptr; p32[1..4] unused
  float* q32;          // FP32 copies of u,v,w,T interleaved, 4 floats a haloed point
  DevStatus* st;
  int krk;
  int fuse_bc;         // BC_None without ghost cells: face refresh + halo in-kernel
  int lean;            // mixed + fuse_bc: stages 1-2 leave the FP64 d,u,v,w unwritten
                       // (nothing reads them before stage 3 rewrites them)
  int visc;
  int chr;
};

// A short list of device arrays passed by value (safe inside captured graphs).
template <typename T>
struct PtrList {
  T* p[16];
  int n;
};

// Table of a batched launch (several instances, one kernel launch): per
// instance its argument block and {first linear block of its part of the grid,
// that part's x extent, its y extent, unused}.  Both arrays live on the device.
template <typename A>
struct BatchTab {
  const A* args;
  const int4* ent;
  int count;
};
// The instance owning linear block lin, and the block's (x, y, z) coordinates
// within that instance's grid (binary search over the first blocks).
template <typename A>
__device__ __forceinline__ int batch_locate(const BatchTab<A>& b, int lin, int& bx, int& by, int& bz) {
  int lo = 0, hi = b.count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&b.ent[mid].x) <= lin)
      lo = mid;
    else
      hi = mid - 1;
  }
  const int4 e = __ldg(&b.ent[lo]);
  int l = lin - e.x;
  bx = l % e.y;
  l /= e.y;
  by = l % e.z;
  bz = l / e.z;
  return lo;
}

// Copies instance q's argument block into shared memory (the block's threads
// share it; reads from shared memory do not alias the kernel's global stores,
// so the compiler need not keep every field in registers).
template <typename A>
__device__ __forceinline__ const A& batch_args(const BatchTab<A>& b, int q, A* sa) {
  static_assert(sizeof(A) % 4 == 0, "argument blocks are copied as 4-byte words");
  const int* src = reinterpret_cast<const int*>(b.args + q);
  int* dst = reinterpret_cast<int*>(sa);
  for (int t = threadIdx.x; t < (int)(sizeof(A) / 4); t += blockDim.x) dst[t] = __ldg(src + t);
  __syncthreads();
  return *sa;
}

// ---- persistent batched stage (ocfd_batch_stage.cuh): one launch per RK stage
// item kinds
enum { BW_FACE_X = 0, BW_FACE_Y = 1, BW_FACE_Z = 2, BW_VISC = 3, BW_TAIL = 4, BW_NEGT = 5 };

// Tables of one stage launch (device memory; S = R in the batched paths).
template <typename R>
struct StageTab {
  const FaceArgs<R>* face[3];   // per member, one stage's face-sweep arguments
  const ViscArgs<R, R>* visc;   // per member
  const UpdArgs<R>* upd;        // per member (tail)
  const UpdArgs<double>* negt;  // per member (repair)
  const int4* seg;              // segments by first item: {first item, member * 8 + kind, x extent, y extent}
  const int2* need;             // per member: {phase-A items, tail items}
  int* ctr;                     // [0] next item, [1 + q] phase-A items done, [1 + n + q] tail items done;
                                // zero at launch
  int nseg, nitems, count;
};

// Whether a persistent stage kernel exists for this combination.
// scheme: OCFD_SCHEME_* (flux-vector WENO7 and characteristic OMP6, viscous).
inline bool batch_stage_supported(bool chr, int scheme, bool visc) {
  return visc && ((!chr && scheme == 2) || (chr && scheme == 3));
}

// One stage launch of nblocks persistent blocks; nblocks == 0 sets the kernel's
// shared-memory limit and returns its resident blocks per SM in *per_sm (call
// outside graph capture).  cudaErrorNotSupported: no persistent kernel for the
// combination.
template <typename R>
cudaError_t launch_batch_stage(bool chr, int scheme, int variant, const StageTab<R>& t, int nblocks, cudaStream_t st,
                               int* per_sm);

template <typename R, typename S>
cudaError_t launch_face(int dir, bool chr, int scheme, const FaceArgs<S>& a, cudaStream_t st);
template <typename R, typename S>
cudaError_t launch_face_batch(int dir, bool chr, int scheme, int variant, const BatchTab<FaceArgs<S>>& b,
                              int nblocks, cudaStream_t st);
template <typename S>
dim3 face_batch_dims(int dir, int variant, const FaceArgs<S>& a);
// raise the dynamic shared-memory limit of every face kernel (call outside graph capture)
cudaError_t setup_face_kernels();
// shared-memory limits of the batched face kernels (once per device, before the first batch launch)
cudaError_t setup_face_batch_kernels_f64();
cudaError_t setup_face_batch_kernels_f32();

template <typename R, typename S>
cudaError_t launch_visc_grad(const ViscArgs<R, S>& a, cudaStream_t st);

// du = inviscous flux divergence (+ mass force)
template <typename R>
cudaError_t launch_div_inv(const UpdArgs<R>& a, cudaStream_t st);
// du(2:5) += viscous divergence
template <typename R>
cudaError_t launch_visc_div(const UpdArgs<R>& a, cudaStream_t st);
// the whole stage tail in one pass
template <typename R>
cudaError_t launch_fused(const UpdArgs<R>& a, cudaStream_t st);

cudaError_t launch_rk3(const Grid& g, double* f, const double* fn, const double* du, double dt, int krk,
                       cudaStream_t st);
// primitive recovery (+ negative-T detection, FP32 copies)
cudaError_t launch_duvwt(const UpdArgs<double>& a, cudaStream_t st);
// serial in-order repair of the points with T <= 0 (handle_NegativeT)
cudaError_t launch_negt_fix(const UpdArgs<double>& a, cudaStream_t st);
// Batched versions (one launch for all instances of a BatchTab; the grid of an
// instance is that of the single launch, see update_dims()).
template <typename R, typename S>
cudaError_t launch_visc_grad_batch(const BatchTab<ViscArgs<R, S>>& b, int nblocks, cudaStream_t st);
template <typename R>
cudaError_t launch_fused_batch(const BatchTab<UpdArgs<R>>& b, int nblocks, bool chr, bool visc, bool fuse_bc,
                               bool i32, cudaStream_t st);
cudaError_t launch_negt_fix_batch(const BatchTab<UpdArgs<double>>& b, cudaStream_t st);
inline dim3 update_dims(const Grid& g) { return dim3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz); }

// periodic face halo of narr haloed arrays (exchange_boundary_xyz)
cudaError_t launch_halo(const Grid& g, const int periodic[3], PtrList<double> arrs, cudaStream_t st);
cudaError_t launch_halo_f32x4(const Grid& g, const int periodic[3], PtrList<float4> arrs, cudaStream_t st);
cudaError_t launch_halo_f32(const Grid& g, const int periodic[3], PtrList<float> arrs, cudaStream_t st);
// BC dispatch on the primitives (blunt2d / user isothermal wall)
cudaError_t launch_bc_wall(const Grid& g, const Phys& ph, double* const prim[5], cudaStream_t st);
// BC_BoundaryLayer / BC_SweptCorner (OCFD_BC_Boundarylayers.f90): boundary data
// on the device and the per-call scalars.
struct BcLayer {
  const double* inlet;   // (ny,nz,5) at i = 1
  const double* upper;   // (nx,nz,5) at j = ny
  const double* pertb;   // (nx,nz) wall perturbation shape
  const int* dirichlet;  // (nx,nz) 1: Dirichlet upper boundary, 0: non-reflecting
  const double* aix;     // haloed metrics read by the wall condition
  const double* aiy;
  const double* aiz;
  const double* ayy;     // haloed coordinates read by the swept-corner wall test
  const double* azz;
  double ht;             // wall perturbation time factor at this step's tt
  double u0, v0;         // cos(AoA), sin(AoA)
};
cudaError_t launch_bc_layer(const Grid& g, const Phys& ph, const BcLayer& bl, double* const prim[5], cudaStream_t st);
// init_bc_nonRef (OCFD_BC_Boundarylayers.f90:273-311): Dirichlet mask of the upper boundary
cudaError_t launch_bc_layer_mask(const Grid& g, const double* axx, const double* ayy, int mode, double sy0, int* mask,
                                 cudaStream_t st);
// f refresh on the six faces from the primitives (OCFD_BC.f90:150-218)
cudaError_t launch_bc_refresh(const Grid& g, const Phys& ph, double* f, double* const prim[5], cudaStream_t st);
// Flow_Ghost_Extent_2nd
cudaError_t launch_ghost(const Grid& g, const Phys& ph, double* const prim[5], cudaStream_t st);
// FP32 copies of the primitives
cudaError_t launch_refresh_shell(const Grid& g, const int periodic[3], double* const prim[5], float* p32, float* q32,
                                 cudaStream_t st);
cudaError_t launch_to_f32x4(const double* u, const double* v, const double* w, const double* T, float* dst, long long n,
                            cudaStream_t st);
cudaError_t launch_to_f32(const double* src, float* dst, long long n, cudaStream_t st);
// init3d: f from primitives
cudaError_t launch_init3d(const Grid& g, const Phys& ph, double* f, double* const prim[5], cudaStream_t st);

// comput_Rhybrid; scratch holds p (haloed) and reduction partials
cudaError_t launch_rhybrid(const Grid& g, const Phys& ph, const DCoef& dc, const double* d, const double* T,
                           const double* const met[22], double* rh, double* scratch, int sensor,
                           const double* hybrid_para, cudaStream_t st);
size_t rhybrid_scratch_doubles(const Grid& g);

// filtering of f for one filter column; scratch >= 2 haloed arrays
cudaError_t launch_filter(const Grid& g, const Phys& ph, double* f, double* scratch, const double* col,
                          cudaStream_t st);

// init_mesh on the device: coords (3 haloed arrays, interior filled) -> metrics
cudaError_t launch_ana_q(const Grid& g, const Phys& ph, const DCoef& dc, double* const prim[5],
                         const double* const met[22], double* q, cudaStream_t st);
cudaError_t launch_ana_average(const Grid& g, double* const prim[5], double* mean, int K, cudaStream_t st);
cudaError_t launch_ana_corner(const Grid& g, const Phys& ph, double* const prim[5], const double* axx,
                              const double* ayy, double* out, cudaStream_t st);
cudaError_t launch_gather_box(const Grid& g, const double* src, int ib, int ie, int jb, int je, int kb, int ke,
                              double* dst, cudaStream_t st);
cudaError_t launch_metric_nonzero(const Grid& g, double* const met[22], unsigned int* nonzero, cudaStream_t st);
cudaError_t launch_mesh(const Grid& g, const Phys& ph, const DCoef& dc, double* const met[22],
                        const double span[3][3], bool jac_given, cudaStream_t st);

// show_flow_msg / ana_box partial sums (deterministic two-level reduction)
cudaError_t launch_flow_msg(const Grid& g, const Phys& ph, const double* f, double* const prim[5],
                            const double* ajac, double* scratch, double* out3, cudaStream_t st);
cudaError_t launch_ana_box(const Grid& g, const Phys& ph, const DCoef& dc, double* const prim[5],
                           const double* const met[22], double* scratch, double* out14, double* out_drms,
                           cudaStream_t st);
size_t reduce_scratch_doubles(const Grid& g);

}  // namespace ocfd
