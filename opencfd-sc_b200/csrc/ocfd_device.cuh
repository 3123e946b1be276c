// ocfd_device.cuh -- device-side layout, argument blocks and the per-point
// flux splitting shared by the kernels.
//
// Layout in HBM (one solver instance):
//   haloed scalars  q[(i+3) + NXH*((j+3) + NYH*(k+3))], i,j,k = -3..n+4 (LAP = 4),
//                   i fastest: the reference's own (1-LAP:n+LAP)^3 order, so that
//                   uploads/downloads are plain copies and every directional
//                   sweep reads rows of consecutive i (coalesced).
//   interior 5-vectors f[(i-1) + nx*((j-1) + ny*((k-1) + nz*m))], SoA by variable.
//   face fluxes     per direction d, faces g = 0..n_d along d, SoA by variable:
//                   x: g + (nx+1)*((j-1) + ny*(k-1));  y: (i-1) + nx*(g + (ny+1)*(k-1));
//                   z: (i-1) + nx*((j-1) + ny*g).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ocfd {

constexpr int LAP = 4;

struct Grid {
  int nx, ny, nz;
  int nxh, nyh, nzh;
  long long n;   // nx*ny*nz
  long long nh;  // nxh*nyh*nzh
  __host__ __device__ __forceinline__ long long ih(int i, int j, int k) const {
    return (long long)(i + LAP - 1) + (long long)nxh * ((long long)(j + LAP - 1) + (long long)nyh * (long long)(k + LAP - 1));
  }
  __host__ __device__ __forceinline__ long long ii(int i, int j, int k) const {
    return (long long)(i - 1) + (long long)nx * ((long long)(j - 1) + (long long)ny * (long long)(k - 1));
  }
  __host__ __device__ __forceinline__ long long hstride(int dir) const {
    return dir == 0 ? 1LL : (dir == 1 ? (long long)nxh : (long long)nxh * nyh);
  }
  __host__ __device__ __forceinline__ int len(int dir) const { return dir == 0 ? nx : (dir == 1 ? ny : nz); }
  // index of face g (0..n_d) of the pencil through interior point (i,j,k)
  __host__ __device__ __forceinline__ long long face(int dir, int g, int i, int j, int k) const {
    if (dir == 0) return (long long)g + (long long)(nx + 1) * ((long long)(j - 1) + (long long)ny * (k - 1));
    if (dir == 1) return (long long)(i - 1) + (long long)nx * ((long long)g + (long long)(ny + 1) * (k - 1));
    return (long long)(i - 1) + (long long)nx * ((long long)(j - 1) + (long long)ny * g);
  }
  __host__ __device__ __forceinline__ long long nfaces(int dir) const { return n / len(dir) * (len(dir) + 1); }
};

// Scalar physics/scheme constants shared by all kernels of one instance.
struct Phys {
  double gamma, ma, re, pr, cv, cp, dt, ref_amu_t0;
  double hx, hy, hz;
  double ud7l[8];
  double hyb1, hyb2;  // Hybrid_para(2), (3)
  double mass_force[3];
  int if_mass_force;
  int scheme_vis;     // 5 = CD6, 6 = CD8
  int periodic[3];
  int bi[6];          // Bound_index: i-, i+, j-, j+, k-, k+
  int sb[6];          // Scheme_boundary
  int ka1, kb1, ka2, kb2;
  int ibc;
  int ghost[6];
  double bc_para0;
  double bc_p[14];  // BC_Para(1:14) of BC_BoundaryLayer / BC_SweptCorner
  // reciprocals precomputed on the host for the production build
  double inv_ma;    // 1/Ma
  double inv_2g;    // 1/(2 gamma)
  double inv_g;     // 1/gamma
  double inv_gm1;   // 1/(gamma-1)
  double sw_tmp3;   // (3-gamma)/(2(gamma-1))
  double inv_cv;    // 1/Cv
  // bit m: metric array m is +0.0 wherever the kernels read it (box grids:
  // the off-diagonal metrics); its loads are skipped
  unsigned int metzero;
};

// The production build replaces divisions by multiplications with a shared or
// precomputed reciprocal (results move by a few ulp; an FP64 division costs
// about ten FP64-pipe instructions).  The strict build keeps every division of
// the reference, in order, for bit-identical parity with the oracle.
#ifdef OCFD_STRICT
#define OCFD_FEWER_DIVS 0
#else
#define OCFD_FEWER_DIVS 1
#endif
// Production build, flux-vector form: a face stores h(F+) + h(F-) (5 arrays)
// instead of both terms (10 arrays), and the update kernel differences the
// sums; the reference's order (h1(i) - h1(i-1) + h2(i) - h2(i-1)) is kept by
// the strict build.
#define OCFD_FV_SUMMED OCFD_FEWER_DIVS
// Production build: the 5 face-flux components of a face are stored as a
// 4-component record (32 bytes FP64, 16 bytes FP32; one 256-/128-bit access)
// followed, after all records, by the 5th component as its own array: element
// (face f, component m < 4) at 4 f + m, component 4 at 4 nfaces + f.  The
// strict build keeps one array per component (f + m nfaces).
#ifndef OCFD_HF_REC
#define OCFD_HF_REC OCFD_FEWER_DIVS
#endif

// 4 consecutive values (32-byte aligned FP64 / 16-byte aligned FP32): one
// 256-bit (sm_100) or 128-bit global access.
__device__ __forceinline__ void rec4_store(double* p, double a, double b, double c, double d) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a), "d"(b), "d"(c), "d"(d) : "memory");
}
__device__ __forceinline__ void rec4_store(float* p, float a, float b, float c, float d) {
  *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
}
// read-only within the launch, or written by other blocks of the same launch
// before a counted wait (the persistent batched stage: no block reads a line of
// these arrays before the wait, so no stale copy can sit in its L1)
__device__ __forceinline__ void rec4_load(const double* p, double* o) {
  asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(o[0]), "=d"(o[1]), "=d"(o[2]), "=d"(o[3]) : "l"(p));
}
__device__ __forceinline__ void rec4_load(const float* p, float* o) {
  const float4 t = __ldg(reinterpret_cast<const float4*>(p));
  o[0] = t.x;
  o[1] = t.y;
  o[2] = t.z;
  o[3] = t.w;
}
// the 5 face-flux components of face f (record layout or one array per component)
template <typename R>
__device__ __forceinline__ void hf_store5(R* out, long long f, long long nf, const R* v) {
#if OCFD_HF_REC
  rec4_store(out + 4 * f, v[0], v[1], v[2], v[3]);
  out[4 * nf + f] = v[4];
#else
#pragma unroll
  for (int m = 0; m < 5; m++) out[f + m * nf] = v[m];
#endif
}
// offset of component m of face f
__host__ __device__ __forceinline__ long long hf_at(long long f, long long nf, int m) {
#if OCFD_HF_REC
  return m < 4 ? 4 * f + m : 4 * nf + f;
#else
  return f + m * nf;
#endif
}

// Metric m at haloed index c, or the constant +0.0 when the array holds only zeros.
template <typename R, typename S>
__device__ __forceinline__ R met_at(const Phys& ph, int m, const S* arr, long long c) {
  return ((ph.metzero >> m) & 1u) ? R(0) : R(__ldg(arr + c));
}

// Steger-Warming splitting of one point: split_Stager_Warming,
// OCFD_flux_split.f90:5-70 (the P2 term is dropped there, :51-60).
template <typename R>
__device__ __forceinline__ void split_sw(const Phys& ph, R g, R c, R d, R u, R v, R w, R A1, R A2, R A3, R* fp,
                                         R* fm) {
  const R tmp1 = R(2) * (g - R(1));
#if OCFD_FEWER_DIVS
  const R tmp3 = R(ph.sw_tmp3);
#else
  const R tmp3 = (R(3) - g) / (R(2) * (g - R(1)));
#endif
#if OCFD_FEWER_DIVS
  const R s2 = A1 * A1 + A2 * A2 + A3 * A3;
  R ss1 = rsqrt(s2);
  R ss = s2 * ss1;
#else
  R ss = sqrt(A1 * A1 + A2 * A2 + A3 * A3);
  R ss1 = R(1) / ss;
#endif
  R ak1 = A1 * ss1, ak2 = A2 * ss1, ak3 = A3 * ss1;
  R vs = A1 * u + A2 * v + A3 * w;
  R E1 = vs, E2 = vs - c * ss, E3 = vs + c * ss;
  R E1P = (E1 + fabs(E1)) * R(0.5), E2P = (E2 + fabs(E2)) * R(0.5), E3P = (E3 + fabs(E3)) * R(0.5);
  R E1M = E1 - E1P, E2M = E2 - E2P, E3M = E3 - E3P;
#if OCFD_FEWER_DIVS
  R tmp0 = d * R(ph.inv_2g);
#else
  R tmp0 = d / (R(2) * g);
#endif
  R uc1 = u - c * ak1, uc2 = u + c * ak1;
  R vc1 = v - c * ak2, vc2 = v + c * ak2;
  R wc1 = w - c * ak3, wc2 = w + c * ak3;
  R vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * R(0.5);
  R vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * R(0.5);
  R vv = (g - R(1)) * (u * u + v * v + w * w);
  R W2 = tmp3 * c * c;
  fp[0] = tmp0 * (tmp1 * E1P + E2P + E3P);
  fp[1] = tmp0 * (tmp1 * E1P * u + E2P * uc1 + E3P * uc2);
  fp[2] = tmp0 * (tmp1 * E1P * v + E2P * vc1 + E3P * vc2);
  fp[3] = tmp0 * (tmp1 * E1P * w + E2P * wc1 + E3P * wc2);
  fp[4] = tmp0 * (E1P * vv + E2P * vvc1 + E3P * vvc2 + W2 * (E2P + E3P));
  fm[0] = tmp0 * (tmp1 * E1M + E2M + E3M);
  fm[1] = tmp0 * (tmp1 * E1M * u + E2M * uc1 + E3M * uc2);
  fm[2] = tmp0 * (tmp1 * E1M * v + E2M * vc1 + E3M * vc2);
  fm[3] = tmp0 * (tmp1 * E1M * w + E2M * wc1 + E3M * wc2);
  fm[4] = tmp0 * (E1M * vv + E2M * vvc1 + E3M * vvc2 + W2 * (E2M + E3M));
}

// Local Lax-Friedrichs splitting of one point (eigenvalue bound per point):
// split_Local_LaxFriedrichs, OCFD_flux_split.f90:73-104.
template <typename R>
__device__ __forceinline__ void split_llf(const Phys& ph, R g, R c, R d, R u, R v, R w, R A1, R A2, R A3, R* fp,
                                          R* fm) {
#if OCFD_FEWER_DIVS
  const R tmp0 = R(ph.inv_g);
  const R tmp1 = R(ph.inv_gm1);
#else
  const R tmp0 = R(1) / g;
  const R tmp1 = R(1) / (g - R(1));
#endif
  R ss = sqrt(A1 * A1 + A2 * A2 + A3 * A3);
  R un = A1 * u + A2 * v + A3 * w;
  R lamda0 = fabs(un) + ss * c;
  R p1 = tmp0 * d * c * c;
  R E0 = tmp1 * p1 + R(0.5) * d * (u * u + v * v + w * w);
  R h0 = E0 + p1;
  fp[0] = R(0.5) * (d * un + lamda0 * d);
  fp[1] = R(0.5) * (d * u * un + A1 * p1 + lamda0 * d * u);
  fp[2] = R(0.5) * (d * v * un + A2 * p1 + lamda0 * d * v);
  fp[3] = R(0.5) * (d * w * un + A3 * p1 + lamda0 * d * w);
  fp[4] = R(0.5) * (h0 * un + lamda0 * E0);
  fm[0] = R(0.5) * (d * un - lamda0 * d);
  fm[1] = R(0.5) * (d * u * un + A1 * p1 - lamda0 * d * u);
  fm[2] = R(0.5) * (d * v * un + A2 * p1 - lamda0 * d * v);
  fm[3] = R(0.5) * (d * w * un + A3 * p1 - lamda0 * d * w);
  fm[4] = R(0.5) * (h0 * un - lamda0 * E0);
}

// The splittings for a sweep whose metric row has a single non-zero component,
// the one along the sweep (box and 1-D grids; production build only): A is
// that component, |grad xi| = |A| and the unit normal is sign(A) along DIR, so
// the square root, the reciprocal and the products with the zero components of
// the general forms above drop out (results move by rounding only).
template <int DIR, typename R>
__device__ __forceinline__ void split_sw_axis(const Phys& ph, R g, R c, R d, R u, R v, R w, R A, R* fp, R* fm) {
  const R tmp1 = R(2) * (g - R(1));
  const R tmp3 = R(ph.sw_tmp3);
  const R ss = fabs(A);
  const R cs = c * copysign(R(1), A);  // c ak_DIR
  const R vs = A * (DIR == 0 ? u : (DIR == 1 ? v : w));
  R E1 = vs, E2 = vs - c * ss, E3 = vs + c * ss;
  R E1P = (E1 + fabs(E1)) * R(0.5), E2P = (E2 + fabs(E2)) * R(0.5), E3P = (E3 + fabs(E3)) * R(0.5);
  R E1M = E1 - E1P, E2M = E2 - E2P, E3M = E3 - E3P;
  R tmp0 = d * R(ph.inv_2g);
  R uc1 = u, uc2 = u, vc1 = v, vc2 = v, wc1 = w, wc2 = w;
  if (DIR == 0) {
    uc1 = u - cs;
    uc2 = u + cs;
  } else if (DIR == 1) {
    vc1 = v - cs;
    vc2 = v + cs;
  } else {
    wc1 = w - cs;
    wc2 = w + cs;
  }
  R vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * R(0.5);
  R vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * R(0.5);
  R vv = (g - R(1)) * (u * u + v * v + w * w);
  R W2 = tmp3 * c * c;
  fp[0] = tmp0 * (tmp1 * E1P + E2P + E3P);
  fp[1] = tmp0 * (tmp1 * E1P * u + E2P * uc1 + E3P * uc2);
  fp[2] = tmp0 * (tmp1 * E1P * v + E2P * vc1 + E3P * vc2);
  fp[3] = tmp0 * (tmp1 * E1P * w + E2P * wc1 + E3P * wc2);
  fp[4] = tmp0 * (E1P * vv + E2P * vvc1 + E3P * vvc2 + W2 * (E2P + E3P));
  fm[0] = tmp0 * (tmp1 * E1M + E2M + E3M);
  fm[1] = tmp0 * (tmp1 * E1M * u + E2M * uc1 + E3M * uc2);
  fm[2] = tmp0 * (tmp1 * E1M * v + E2M * vc1 + E3M * vc2);
  fm[3] = tmp0 * (tmp1 * E1M * w + E2M * wc1 + E3M * wc2);
  fm[4] = tmp0 * (E1M * vv + E2M * vvc1 + E3M * vvc2 + W2 * (E2M + E3M));
}

template <int DIR, typename R>
__device__ __forceinline__ void split_llf_axis(const Phys& ph, R g, R c, R d, R u, R v, R w, R A, R* fp, R* fm) {
  const R tmp0 = R(ph.inv_g);
  const R tmp1 = R(ph.inv_gm1);
  const R un = A * (DIR == 0 ? u : (DIR == 1 ? v : w));
  const R lamda0 = fabs(un) + fabs(A) * c;
  const R p1 = tmp0 * d * c * c;
  const R E0 = tmp1 * p1 + R(0.5) * d * (u * u + v * v + w * w);
  const R h0 = E0 + p1;
  const R Ap = A * p1;
  fp[0] = R(0.5) * (d * un + lamda0 * d);
  fp[1] = R(0.5) * (DIR == 0 ? d * u * un + Ap + lamda0 * d * u : d * u * un + lamda0 * d * u);
  fp[2] = R(0.5) * (DIR == 1 ? d * v * un + Ap + lamda0 * d * v : d * v * un + lamda0 * d * v);
  fp[3] = R(0.5) * (DIR == 2 ? d * w * un + Ap + lamda0 * d * w : d * w * un + lamda0 * d * w);
  fp[4] = R(0.5) * (h0 * un + lamda0 * E0);
  fm[0] = R(0.5) * (d * un - lamda0 * d);
  fm[1] = R(0.5) * (DIR == 0 ? d * u * un + Ap - lamda0 * d * u : d * u * un - lamda0 * d * u);
  fm[2] = R(0.5) * (DIR == 1 ? d * v * un + Ap - lamda0 * d * v : d * v * un - lamda0 * d * v);
  fm[3] = R(0.5) * (DIR == 2 ? d * w * un + Ap - lamda0 * d * w : d * w * un - lamda0 * d * w);
  fm[4] = R(0.5) * (h0 * un - lamda0 * E0);
}

// Metric row of sweep DIR (A?1 arrays 13 + 3 DIR .. 15 + 3 DIR) has its two
// off-diagonal components identically +0.0.
template <int DIR>
__host__ __device__ __forceinline__ bool axis_aligned(unsigned int metzero) {
  const int m0 = 13 + 3 * DIR;
  const unsigned int off = (DIR == 0 ? 6u : (DIR == 1 ? 5u : 3u)) << m0;  // the two components other than DIR
  return (metzero & off) == off;
}

// set_hybrid_scheme: OCFD_SetHybrid.f90:2-15
__device__ __forceinline__ int hybrid_index(double R0, double t1, double t2) {
  if (R0 <= t1) return 1;
  if (R0 <= t2) return 2;
  return 3;
}

// Arguments of the face-flux kernels (one direction).
template <typename S>
struct FaceArgs {
  Grid g;
  const S* d;
  const S* u;
  const S* v;
  const S* w;
  const S* T;
  const float* q4;   // FP32 sweeps: u,v,w,T interleaved (haloed, 4 floats a point); u..T unused
  const S* A1;
  const S* A2;
  const S* A3;
  const double* rh;  // Rhybrid (haloed, FP64) or nullptr
  void* hh;          // face fluxes (R), nvar arrays of g.nfaces(dir)
  long long fs;      // per-variable stride of hh
  int fbeg, fend;    // faces computed: fbeg..fend
  int split;         // 1 SW, 2 LLF
  int* err;          // DevStatus::error of the instance (bounded waits record 4 there)
  int no_tma;        // host side: stage the tile with plain loads (a TMA wait of this instance gave up)
  int test_tx;       // 0; test of the bounded TMA waits: bytes the staging expects beyond its copies
  Phys ph;
};

// Device-side status words of one instance (written by kernels, read by host).
struct DevStatus {
  int negt_count;     // points with T <= 0 found by the current primitive recovery
  int negt_list[16];  // their haloed linear indices (first 16)
  int error;          // sticky error: 3 = negative-T limit exceeded, 4 = a bounded device wait gave up
  int negt_last;      // points repaired in the last stage
  int negt_total;     // points repaired since creation
  int pad[12];
};

}  // namespace ocfd
