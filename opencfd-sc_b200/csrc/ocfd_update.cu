// ocfd_update.cu -- viscous terms, flux divergence, RK3, primitive recovery
// with the negative-temperature repair, boundary conditions and halos.
//
// The step path runs, per RK stage: three face-flux launches (ocfd_face.cu),
// one viscous-gradient launch and ONE fused stage-tail launch that does the
// work of the reference's du_inviscous flux difference, du_viscous divergence,
// OCFD_time_adv_RK3, comput_duvwT and (for BC_None) the face refresh of
// OCFD_bc plus next stage's exchange_boundary_xyz, in a single pass over HBM.
// The stage-by-stage C ABI uses the unfused kernels below; both share the same
// device functions, so they produce the same bits.
#include <algorithm>
#include <utility>

#include "ocfd_update_body.cuh"

namespace ocfd {

// Block order of the single-instance update kernels (32 x 8 tiles per plane):
// y-slabs of sy tile rows, and inside a slab plane after plane in k, so that
// the planes a block's z-stencil reads were touched shortly before and are
// still in L2 on large grids (measured at 512^3: viscous 12% and tail 12%
// faster; at 256^3 whole planes are faster and are kept).
struct SlabOrder {
  int gx, gy, sy;
};
// grid (gx, sy, slabs * nz): blockIdx.z = slab * nz + k, block rows past gy idle
__device__ __forceinline__ bool slab_decode(const SlabOrder& so, int nz, int& bx, int& by, int& bz) {
  const int sl = blockIdx.z / nz;
  bz = blockIdx.z - sl * nz;
  by = sl * so.sy + blockIdx.y;
  bx = blockIdx.x;
  return by < so.gy;
}
static dim3 slab_grid(const SlabOrder& so, int nz) {
  const int slabs = (so.gy + so.sy - 1) / so.sy;
  return dim3(so.gx, so.sy, slabs * nz);
}
static SlabOrder slab_order(const Grid& g) {
  SlabOrder so;
  so.gx = (g.nx + 31) / 32;
  so.gy = (g.ny + 7) / 8;
  so.sy = so.gy;  // whole planes while 3 planes (the z-reuse distance) fit in L2
  const long long plane = 400LL * g.nx * g.ny;  // ~400 bytes per point touched by the tail kernel
  if (3 * plane > 100000000LL) {
    const long long rows = 40000000LL / (3LL * 400 * g.nx);
    so.sy = (int)std::max(1LL, std::min((long long)so.gy, rows / 8));
    if ((long long)((so.gy + so.sy - 1) / so.sy) * g.nz > 65535) so.sy = so.gy;  // gridDim.z limit
  }
  return so;
}

template <typename R, typename S, bool SLAB, bool AXS = false>
__global__ void __launch_bounds__(256, OCFD_VISC_MINB) k_visc_grad(ViscArgs<R, S> a, SlabOrder so) {
  if (!SLAB) {
    visc_grad_body<R, S, AXS>(a, blockIdx.x, blockIdx.y, blockIdx.z);
    return;
  }
  int bx, by, bz;
  if (!slab_decode(so, a.g.nz, bx, by, bz)) return;
  visc_grad_body<R, S, AXS>(a, bx, by, bz);
}
template <typename R, typename S>
__global__ void __launch_bounds__(256, OCFD_VISCB_MINB) k_visc_grad_batch(BatchTab<ViscArgs<R, S>> b) {
  __shared__ __align__(16) ViscArgs<R, S> sa;
  int bx, by, bz;
  const int q = batch_locate(b, blockIdx.x, bx, by, bz);
  const ViscArgs<R, S>& A = batch_args(b, q, &sa);
  // the member's own variant, as its single-instance launch chooses it
  if (OCFD_VISC_AXS && visc_axis_aligned(A.ph.metzero))
    visc_grad_body<R, S, OCFD_VISC_AXS != 0>(A, bx, by, bz);
  else
    visc_grad_body<R, S>(A, bx, by, bz);
}

template <typename R, typename S>
cudaError_t launch_visc_grad(const ViscArgs<R, S>& a, cudaStream_t st) {
  const SlabOrder so = slab_order(a.g);
  constexpr bool kAx = OCFD_VISC_AXS != 0;
  const bool ax = kAx && visc_axis_aligned(a.ph.metzero);
  if (so.sy == so.gy) {
    if (ax)
      k_visc_grad<R, S, false, kAx><<<update_dims(a.g), 256, 0, st>>>(a, so);
    else
      k_visc_grad<R, S, false><<<update_dims(a.g), 256, 0, st>>>(a, so);
  } else {
    if (ax)
      k_visc_grad<R, S, true, kAx><<<slab_grid(so, a.g.nz), 256, 0, st>>>(a, so);
    else
      k_visc_grad<R, S, true><<<slab_grid(so, a.g.nz), 256, 0, st>>>(a, so);
  }
  return cudaGetLastError();
}
template <typename R, typename S>
cudaError_t launch_visc_grad_batch(const BatchTab<ViscArgs<R, S>>& b, int nblocks, cudaStream_t st) {
  k_visc_grad_batch<R, S><<<nblocks, 256, 0, st>>>(b);
  return cudaGetLastError();
}
template cudaError_t launch_visc_grad<double, double>(const ViscArgs<double, double>&, cudaStream_t);
template cudaError_t launch_visc_grad<float, float>(const ViscArgs<float, float>&, cudaStream_t);
template cudaError_t launch_visc_grad_batch<double, double>(const BatchTab<ViscArgs<double, double>>&, int,
                                                           cudaStream_t);
template cudaError_t launch_visc_grad_batch<float, float>(const BatchTab<ViscArgs<float, float>>&, int, cudaStream_t);


// ---------------------------------------------------------------------------
template <bool CHAR, typename R>
__global__ void __launch_bounds__(256) k_div_inv(UpdArgs<R> a) {
  const Grid& G = a.g;
  const int i = blockIdx.x * 32 + (threadIdx.x & 31) + 1;
  const int j = blockIdx.y * 8 + (threadIdx.x >> 5) + 1;
  const int k = blockIdx.z + 1;
  if (i > G.nx || j > G.ny) return;
  R du[5];
  inv_div<CHAR>(a, i, j, k, du);
  const long long o = G.ii(i, j, k);
#pragma unroll
  for (int m = 0; m < 5; m++) a.du[o + m * G.n] = double(du[m]);
}

template <typename R>
__global__ void __launch_bounds__(256) k_visc_div(UpdArgs<R> a) {
  const Grid& G = a.g;
  const int i = blockIdx.x * 32 + (threadIdx.x & 31) + 1;
  const int j = blockIdx.y * 8 + (threadIdx.x >> 5) + 1;
  const int k = blockIdx.z + 1;
  if (i > G.nx || j > G.ny) return;
  const long long o = G.ii(i, j, k);
  R du[5];
#pragma unroll
  for (int m = 0; m < 5; m++) du[m] = R(a.du[o + m * G.n]);
  visc_div(a, i, j, k, du);
#pragma unroll
  for (int m = 1; m < 5; m++) a.du[o + m * G.n] = double(du[m]);
}


template <bool CHAR, bool VISC, bool FUSEBC, typename R, bool SLAB, typename IX>
__global__ void __launch_bounds__(256, OCFD_TAIL_MINB) k_fused(UpdArgs<R> a, SlabOrder so) {
  if (!SLAB) {
    fused_body<CHAR, VISC, FUSEBC, R, IX>(a, blockIdx.x, blockIdx.y, blockIdx.z);
    return;
  }
  int bx, by, bz;
  if (!slab_decode(so, a.g.nz, bx, by, bz)) return;
  fused_body<CHAR, VISC, FUSEBC, R, IX>(a, bx, by, bz);
}
template <bool CHAR, bool VISC, bool FUSEBC, typename R, typename IX = long long>
__global__ void __launch_bounds__(256, OCFD_TAILB_MINB) k_fused_batch(BatchTab<UpdArgs<R>> b) {
  __shared__ __align__(16) UpdArgs<R> sa;
  int bx, by, bz;
  const int q = batch_locate(b, blockIdx.x, bx, by, bz);
  fused_body<CHAR, VISC, FUSEBC, R, IX>(batch_args(b, q, &sa), bx, by, bz);
}

template <typename R>
cudaError_t launch_div_inv(const UpdArgs<R>& a, cudaStream_t st) {
  dim3 grid((a.g.nx + 31) / 32, (a.g.ny + 7) / 8, a.g.nz);
  if (a.chr)
    k_div_inv<true, R><<<grid, 256, 0, st>>>(a);
  else
    k_div_inv<false, R><<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}
template <typename R>
cudaError_t launch_visc_div(const UpdArgs<R>& a, cudaStream_t st) {
  dim3 grid((a.g.nx + 31) / 32, (a.g.ny + 7) / 8, a.g.nz);
  k_visc_div<R><<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}
template <typename R>
cudaError_t launch_fused(const UpdArgs<R>& a, cudaStream_t st) {
  const SlabOrder so = slab_order(a.g);
  const bool slab = so.sy != so.gy;
  const dim3 grid = slab ? slab_grid(so, a.g.nz) : update_dims(a.g);
  // FP32 tails index faces and viscous fluxes in 32 bits when every offset fits
  long long fmax = 0;
  for (int d = 0; d < 3; d++) fmax = std::max(fmax, a.fs[d]);
  const bool i32 = sizeof(R) == 4 && 12LL * a.g.n < 2147483647LL && 10LL * fmax < 2147483647LL;
#define OCFD_FUSED(C, V, B)                                                     \
  if (!!a.chr == C && !!a.visc == V && !!a.fuse_bc == B) {                      \
    if (i32 && slab)                                                            \
      k_fused<C, V, B, R, true, int><<<grid, 256, 0, st>>>(a, so);              \
    else if (i32)                                                               \
      k_fused<C, V, B, R, false, int><<<grid, 256, 0, st>>>(a, so);             \
    else if (slab)                                                              \
      k_fused<C, V, B, R, true, long long><<<grid, 256, 0, st>>>(a, so);        \
    else                                                                        \
      k_fused<C, V, B, R, false, long long><<<grid, 256, 0, st>>>(a, so);       \
  }
  OCFD_FUSED(false, false, false)
  OCFD_FUSED(false, false, true)
  OCFD_FUSED(false, true, false)
  OCFD_FUSED(false, true, true)
  OCFD_FUSED(true, false, false)
  OCFD_FUSED(true, false, true)
  OCFD_FUSED(true, true, false)
  OCFD_FUSED(true, true, true)
#undef OCFD_FUSED
  return cudaGetLastError();
}
template <typename R>
cudaError_t launch_fused_batch(const BatchTab<UpdArgs<R>>& b, int nblocks, bool chr, bool visc, bool fuse_bc,
                               bool i32, cudaStream_t st) {
  // 32-bit face and viscous-flux offsets (FP32, every member's offsets fit),
  // as the single-instance tail
  if (sizeof(R) == 4 && i32 && fuse_bc) {
    if (chr && visc) k_fused_batch<true, true, true, R, int><<<nblocks, 256, 0, st>>>(b);
    if (chr && !visc) k_fused_batch<true, false, true, R, int><<<nblocks, 256, 0, st>>>(b);
    if (!chr && visc) k_fused_batch<false, true, true, R, int><<<nblocks, 256, 0, st>>>(b);
    if (!chr && !visc) k_fused_batch<false, false, true, R, int><<<nblocks, 256, 0, st>>>(b);
    return cudaGetLastError();
  }
#define OCFD_FUSED(C, V, B) \
  if (chr == C && visc == V && fuse_bc == B) k_fused_batch<C, V, B, R><<<nblocks, 256, 0, st>>>(b);
  OCFD_FUSED(false, false, false)
  OCFD_FUSED(false, false, true)
  OCFD_FUSED(false, true, false)
  OCFD_FUSED(false, true, true)
  OCFD_FUSED(true, false, false)
  OCFD_FUSED(true, false, true)
  OCFD_FUSED(true, true, false)
  OCFD_FUSED(true, true, true)
#undef OCFD_FUSED
  return cudaGetLastError();
}
template cudaError_t launch_fused_batch<double>(const BatchTab<UpdArgs<double>>&, int, bool, bool, bool, bool,
                                                cudaStream_t);
template cudaError_t launch_fused_batch<float>(const BatchTab<UpdArgs<float>>&, int, bool, bool, bool, bool,
                                               cudaStream_t);
template cudaError_t launch_div_inv<double>(const UpdArgs<double>&, cudaStream_t);
template cudaError_t launch_div_inv<float>(const UpdArgs<float>&, cudaStream_t);
template cudaError_t launch_visc_div<double>(const UpdArgs<double>&, cudaStream_t);
template cudaError_t launch_visc_div<float>(const UpdArgs<float>&, cudaStream_t);
template cudaError_t launch_fused<double>(const UpdArgs<double>&, cudaStream_t);
template cudaError_t launch_fused<float>(const UpdArgs<float>&, cudaStream_t);

// ---------------------------------------------------------------------------
// OCFD_time_adv_RK3 alone (stage API)
__global__ void k_rk3(Grid G, double* f, const double* fn, const double* du, double dt, int krk) {
  const long long n5 = 5 * G.n;
  const double al = krk == 2 ? 3.0 / 4.0 : 1.0 / 3.0;
  const double be = krk == 2 ? 1.0 / 4.0 : 2.0 / 3.0;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n5; c += (long long)gridDim.x * blockDim.x) {
    if (krk == 1)
      f[c] = fn[c] + dt * du[c];
    else
      f[c] = al * fn[c] + be * (f[c] + dt * du[c]);
  }
}
cudaError_t launch_rk3(const Grid& g, double* f, const double* fn, const double* du, double dt, int krk,
                       cudaStream_t st) {
  k_rk3<<<148 * 8, 256, 0, st>>>(g, f, fn, du, dt, krk);
  return cudaGetLastError();
}

// comput_duvwT alone (stage API): primitives, negative-T detection
__global__ void __launch_bounds__(256) k_duvwt(UpdArgs<double> a) {
  const Grid& G = a.g;
  const int i = blockIdx.x * 32 + (threadIdx.x & 31) + 1;
  const int j = blockIdx.y * 8 + (threadIdx.x >> 5) + 1;
  const int k = blockIdx.z + 1;
  if (i > G.nx || j > G.ny) return;
  const long long o = G.ii(i, j, k), n = G.n;
  double fv[5], q[5];
#pragma unroll
  for (int m = 0; m < 5; m++) fv[m] = a.f[o + m * n];
  prims_of(fv, a.ph.cv, a.ph.inv_cv, q);
  const long long h = G.ih(i, j, k);
  if (q[4] <= 0.0) record_negt(a.st, h);
#pragma unroll
  for (int m = 0; m < 5; m++) a.prim[m][h] = q[m];
  if (a.p32[0]) {
    a.p32[0][h] = float(q[0]);
    reinterpret_cast<float4*>(a.q32)[h] = make_float4(float(q[1]), float(q[2]), float(q[3]), float(q[4]));
  }
}
cudaError_t launch_duvwt(const UpdArgs<double>& a, cudaStream_t st) {
  dim3 grid((a.g.nx + 31) / 32, (a.g.ny + 7) / 8, a.g.nz);
  k_duvwt<<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

__global__ void k_negt_fix(UpdArgs<double> a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  negt_fix_body(a);
}
// one block per instance
__global__ void k_negt_fix_batch(BatchTab<UpdArgs<double>> b) {
  if (threadIdx.x != 0 || (int)blockIdx.x >= b.count) return;
  negt_fix_body(b.args[blockIdx.x]);
}
cudaError_t launch_negt_fix(const UpdArgs<double>& a, cudaStream_t st) {
  k_negt_fix<<<1, 32, 0, st>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_negt_fix_batch(const BatchTab<UpdArgs<double>>& b, cudaStream_t st) {
  k_negt_fix_batch<<<b.count, 32, 0, st>>>(b);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// exchange_boundary_xyz with one rank (OCFD_mpi.f90:183-233): the 4-layer face
// halos of every periodic direction, over the interior of the other two.
template <typename T>
__global__ void k_halo(Grid G, int px, int py, int pz, PtrList<T> arrs) {
  const int narr = arrs.n;
  const long long nxl = px ? 2LL * LAP * G.ny * G.nz : 0;
  const long long nyl = py ? 2LL * LAP * G.nx * G.nz : 0;
  const long long nzl = pz ? 2LL * LAP * G.nx * G.ny : 0;
  const long long tot = nxl + nyl + nzl;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot * narr;
       t += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(t / tot);
    long long e = t % tot;
    T* p = arrs.p[a];
    long long dst, src;
    if (e < nxl) {
      const int side = (int)(e % 2);
      e /= 2;
      const int l = (int)(e % LAP) + 1;
      e /= LAP;
      const int j = (int)(e % G.ny) + 1, k = (int)(e / G.ny) + 1;
      if (side == 0) {
        dst = G.ih(G.nx + l, j, k);
        src = G.ih(l, j, k);
      } else {
        dst = G.ih(1 - l, j, k);
        src = G.ih(G.nx + 1 - l, j, k);
      }
    } else if (e < nxl + nyl) {
      e -= nxl;
      const int side = (int)(e % 2);
      e /= 2;
      const int i = (int)(e % G.nx) + 1;
      e /= G.nx;
      const int l = (int)(e % LAP) + 1, k = (int)(e / LAP) + 1;
      if (side == 0) {
        dst = G.ih(i, G.ny + l, k);
        src = G.ih(i, l, k);
      } else {
        dst = G.ih(i, 1 - l, k);
        src = G.ih(i, G.ny + 1 - l, k);
      }
    } else {
      e -= nxl + nyl;
      const int side = (int)(e % 2);
      e /= 2;
      const int i = (int)(e % G.nx) + 1;
      e /= G.nx;
      const int j = (int)(e % G.ny) + 1, l = (int)(e / G.ny) + 1;
      if (side == 0) {
        dst = G.ih(i, j, G.nz + l);
        src = G.ih(i, j, l);
      } else {
        dst = G.ih(i, j, 1 - l);
        src = G.ih(i, j, G.nz + 1 - l);
      }
    }
    p[dst] = p[src];
  }
}
cudaError_t launch_halo(const Grid& g, const int periodic[3], PtrList<double> arrs, cudaStream_t st) {
  if (!periodic[0] && !periodic[1] && !periodic[2]) return cudaSuccess;
  k_halo<double><<<148 * 4, 256, 0, st>>>(g, periodic[0], periodic[1], periodic[2], arrs);
  return cudaGetLastError();
}
cudaError_t launch_halo_f32x4(const Grid& g, const int periodic[3], PtrList<float4> arrs, cudaStream_t st) {
  if (!periodic[0] && !periodic[1] && !periodic[2]) return cudaSuccess;
  k_halo<float4><<<148 * 4, 256, 0, st>>>(g, periodic[0], periodic[1], periodic[2], arrs);
  return cudaGetLastError();
}
cudaError_t launch_halo_f32(const Grid& g, const int periodic[3], PtrList<float> arrs, cudaStream_t st) {
  if (!periodic[0] && !periodic[1] && !periodic[2]) return cudaSuccess;
  k_halo<float><<<148 * 4, 256, 0, st>>>(g, periodic[0], periodic[1], periodic[2], arrs);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// BC dispatch on the primitives (OCFD_BC.f90:8-23): ocfd_bc_blunt2d
// (OCFD_BC_Def.f90:4-33), or the BC_User_Def slot filled with an isothermal
// wall (T = Tw, density from the 2nd-order pressure extrapolation of
// OCFD_BC_Boundarylayers.f90:129-133) and the same free stream at j = ny.
__global__ void k_bc_wall(Grid G, Phys ph, double* d, double* u, double* v, double* w, double* T) {
  const long long tot = (long long)G.nx * G.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % G.nx) + 1, k = (int)(t / G.nx) + 1;
    const long long h1 = G.ih(i, 1, k), h2 = G.ih(i, 2, k), h3 = G.ih(i, 3, k), hn = G.ih(i, G.ny, k);
    if (ph.ibc == 1) {
      d[h1] = d[h2];
      u[h1] = 0.0;
      v[h1] = 0.0;
      w[h1] = 0.0;
      T[h1] = T[h2];
    } else {
      const double Tw = ph.bc_para0;
      u[h1] = 0.0;
      v[h1] = 0.0;
      w[h1] = 0.0;
      T[h1] = Tw;
      d[h1] = (4.0 * d[h2] * T[h2] - d[h3] * T[h3]) / (3.0 * Tw);
    }
    d[hn] = 1.0;
    u[hn] = 1.0;
    v[hn] = 0.0;
    w[hn] = 0.0;
    T[hn] = 1.0;
  }
}
cudaError_t launch_bc_wall(const Grid& g, const Phys& ph, double* const prim[5], cudaStream_t st) {
  if (ph.ibc != 1 && ph.ibc != 99) return cudaSuccess;
  k_bc_wall<<<148 * 2, 256, 0, st>>>(g, ph, prim[0], prim[1], prim[2], prim[3], prim[4]);
  return cudaGetLastError();
}

// f refresh on the six faces (OCFD_BC.f90:150-218); each boundary point once.
__global__ void k_bc_refresh(Grid G, double cv, double* f, const double* d, const double* u, const double* v,
                             const double* w, const double* T) {
  const long long nxf = 2LL * G.ny * G.nz;
  const long long nyf = 2LL * (G.nx - 2) * G.nz;
  const long long nzf = 2LL * (G.nx - 2) * (G.ny - 2);
  const long long tot = nxf + nyf + nzf;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    long long e = t;
    if (e < nxf) {
      i = (e % 2) ? G.nx : 1;
      e /= 2;
      j = (int)(e % G.ny) + 1;
      k = (int)(e / G.ny) + 1;
    } else if (e < nxf + nyf) {
      e -= nxf;
      j = (e % 2) ? G.ny : 1;
      e /= 2;
      i = (int)(e % (G.nx - 2)) + 2;
      k = (int)(e / (G.nx - 2)) + 1;
    } else {
      e -= nxf + nyf;
      k = (e % 2) ? G.nz : 1;
      e /= 2;
      i = (int)(e % (G.nx - 2)) + 2;
      j = (int)(e / (G.nx - 2)) + 2;
    }
    const long long h = G.ih(i, j, k), o = G.ii(i, j, k);
    double q[5] = {d[h], u[h], v[h], w[h], T[h]}, fv[5];
    refresh_of(q, cv, fv);
    for (int m = 0; m < 5; m++) f[o + m * G.n] = fv[m];
  }
}
cudaError_t launch_bc_refresh(const Grid& g, const Phys& ph, double* f, double* const prim[5], cudaStream_t st) {
  k_bc_refresh<<<148 * 2, 256, 0, st>>>(g, ph.cv, f, prim[0], prim[1], prim[2], prim[3], prim[4]);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// BC_BoundaryLayer (ocfd_bc_BoundaryLayer, OCFD_BC_Boundarylayers.f90:17-169) and
// BC_SweptCorner (ocfd_bc_swept_corner, :443-618).  The reference's loops run in
// this order -- inlet, upper, wall, outlet (, side planes) -- and later loops
// read points earlier ones wrote, so each is one launch.
__global__ void k_bcl_inlet(Grid G, Phys ph, BcLayer bl, double* d, double* u, double* v, double* w, double* T) {
  const long long tot = (long long)G.ny * G.nz, nyz = tot;
  const int data = ph.ibc == 3 ? 1 : (int)llrint(ph.bc_p[0]);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t % G.ny) + 1, k = (int)(t / G.ny) + 1;
    const long long h = G.ih(1, j, k);
    if (data == 0) {
      // the reference's free-stream inlet sets T = 0 (:58-66)
      d[h] = 1.0;
      u[h] = bl.u0;
      v[h] = bl.v0;
      w[h] = 0.0;
      T[h] = 0.0;
    } else {
      d[h] = bl.inlet[t];
      u[h] = bl.inlet[t + nyz];
      v[h] = bl.inlet[t + 2 * nyz];
      w[h] = bl.inlet[t + 3 * nyz];
      T[h] = bl.inlet[t + 4 * nyz];
    }
  }
}
__global__ void k_bcl_upper(Grid G, Phys ph, BcLayer bl, double* d, double* u, double* v, double* w, double* T) {
  const long long tot = (long long)G.nx * G.nz, nxz = tot;
  const int data = ph.ibc == 3 ? 0 : (int)llrint(ph.bc_p[1]);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    if (!bl.dirichlet[t]) continue;
    const int i = (int)(t % G.nx) + 1, k = (int)(t / G.nx) + 1;
    const long long h = G.ih(i, G.ny, k);
    if (data == 0) {
      d[h] = 1.0;
      u[h] = bl.u0;
      v[h] = bl.v0;
      w[h] = 0.0;
      T[h] = 1.0;
    } else {
      d[h] = bl.upper[t];
      u[h] = bl.upper[t + nxz];
      v[h] = bl.upper[t + 2 * nxz];
      w[h] = bl.upper[t + 3 * nxz];
      T[h] = bl.upper[t + 4 * nxz];
    }
  }
}
__global__ void k_bcl_wall(Grid G, Phys ph, BcLayer bl, double* d, double* u, double* v, double* w, double* T) {
  const long long tot = (long long)G.nx * G.nz;
  const bool sc = ph.ibc == 3;
  const double Tw = sc ? ph.bc_p[1] : ph.bc_p[4];
  const double A = sc ? ph.bc_p[4] : ph.bc_p[7];
  const double wall_zl = ph.bc_p[2], epsl = 1.0e-7;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % G.nx) + 1, k = (int)(t / G.nx) + 1;
    const long long h1 = G.ih(i, 1, k), h2 = G.ih(i, 2, k), h3 = G.ih(i, 3, k);
    if (sc) {
      const double zz = bl.azz[h1], yy = bl.ayy[h1];
      if (!((zz >= -epsl && zz <= wall_zl + epsl) || yy <= epsl)) {
        // off the wall: first-order extrapolation (:552-558)
        d[h1] = d[h2];
        T[h1] = T[h2];
        u[h1] = u[h2];
        v[h1] = v[h2];
        w[h1] = w[h2];
        continue;
      }
    }
    const double aix = bl.aix[h1], aiy = bl.aiy[h1], aiz = bl.aiz[h1];
    const double tmp = 1.0 / (sqrt(aix * aix + aiy * aiy + aiz * aiz));
    const double A0 = A * bl.ht * bl.pertb[t];
    u[h1] = A0 * aix * tmp;
    v[h1] = A0 * aiy * tmp;
    w[h1] = A0 * aiz * tmp;
    if (Tw > 0.0) {
      T[h1] = Tw;
      d[h1] = (4.0 * d[h2] * T[h2] - d[h3] * T[h3]) / (3.0 * Tw);
    } else {
      T[h1] = (4.0 * T[h2] - T[h3]) / 3.0;
      d[h1] = (4.0 * d[h2] - d[h3]) / 3.0;
    }
  }
}
__global__ void k_bcl_outlet(Grid G, int mode, double* d, double* u, double* v, double* w, double* T) {
  const long long tot = (long long)G.ny * G.nz;
  double* Q[5] = {d, u, v, w, T};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t % G.ny) + 1, k = (int)(t / G.ny) + 1;
    const long long h = G.ih(G.nx, j, k), h1 = G.ih(G.nx - 1, j, k), h2 = G.ih(G.nx - 2, j, k);
#pragma unroll
    for (int q = 0; q < 5; q++) Q[q][h] = mode == 1 ? Q[q][h1] : 2.0 * Q[q][h1] - Q[q][h2];
  }
}
// swept corner side planes k = 1 (from k = 2) and k = nz (from nz - 1), :573-618
__global__ void k_bcl_zside(Grid G, int kdst, int ksrc, double* d, double* u, double* v, double* w, double* T) {
  const long long tot = (long long)G.nx * G.ny;
  double* Q[5] = {d, u, v, w, T};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % G.nx) + 1, j = (int)(t / G.nx) + 1;
#pragma unroll
    for (int q = 0; q < 5; q++) Q[q][G.ih(i, j, kdst)] = Q[q][G.ih(i, j, ksrc)];
  }
}
cudaError_t launch_bc_layer(const Grid& g, const Phys& ph, const BcLayer& bl, double* const prim[5], cudaStream_t st) {
  double *d = prim[0], *u = prim[1], *v = prim[2], *w = prim[3], *T = prim[4];
  k_bcl_inlet<<<148, 256, 0, st>>>(g, ph, bl, d, u, v, w, T);
  k_bcl_upper<<<148, 256, 0, st>>>(g, ph, bl, d, u, v, w, T);
  k_bcl_wall<<<148, 256, 0, st>>>(g, ph, bl, d, u, v, w, T);
  const int outlet = (int)llrint(ph.ibc == 3 ? ph.bc_p[0] : ph.bc_p[3]);
  if (outlet == 1 || outlet == 2) k_bcl_outlet<<<148, 256, 0, st>>>(g, outlet, d, u, v, w, T);
  if (ph.ibc == 3) {
    if (llrint(ph.bc_p[10]) == 1) k_bcl_zside<<<148, 256, 0, st>>>(g, 1, 2, d, u, v, w, T);
    if (llrint(ph.bc_p[11]) == 1) k_bcl_zside<<<148, 256, 0, st>>>(g, g.nz, g.nz - 1, d, u, v, w, T);
  }
  return cudaGetLastError();
}

// init_bc_nonRef: mode 0 automatic (Dirichlet where the upper boundary's slope
// dy/dx >= tan(AoA) + 1e-6), 1 non-reflecting everywhere, 2 Dirichlet everywhere.
__global__ void k_bcl_mask(Grid G, const double* axx, const double* ayy, int mode, double sy0, int* mask) {
  const long long tot = (long long)G.nx * G.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % G.nx) + 1, k = (int)(t / G.nx) + 1;
    int dir = 0;
    if (mode == 2) {
      dir = 1;
    } else if (mode == 0) {
      const int ia = i == 1 ? i + 1 : i, ib = i == 1 ? i : i - 1;
      const double sy = (ayy[G.ih(ia, G.ny, k)] - ayy[G.ih(ib, G.ny, k)]) / (axx[G.ih(ia, G.ny, k)] - axx[G.ih(ib, G.ny, k)]);
      dir = sy >= sy0 + 1.0e-6;
    }
    mask[t] = dir;
  }
}
cudaError_t launch_bc_layer_mask(const Grid& g, const double* axx, const double* ayy, int mode, double sy0, int* mask,
                                 cudaStream_t st) {
  k_bcl_mask<<<148, 256, 0, st>>>(g, axx, ayy, mode, sy0, mask);
  return cudaGetLastError();
}

// Flow_Ghost_Userdef (OCFD_GhostCell_UserDef.f90:13-20): swept corner k- symmetry
// (Flow_Ghost_Sweptcorner :54-73) and flat-plate j- extrapolation with the
// limiter [0.5, 2] (Flow_Ghost_flatplate :106-136).
__global__ void k_ghost_user(Grid G, Phys ph, double* d, double* u, double* v, double* w, double* T) {
  const bool sc = ph.ibc == 3 && ph.ghost[4] == -1;
  const long long tot = sc ? (long long)G.nx * G.ny * LAP : (long long)G.nx * G.nz * LAP;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    if (sc) {
      const int i = (int)(t % G.nx) + 1, j = (int)((t / G.nx) % G.ny) + 1, k = 1 - LAP + (int)(t / ((long long)G.nx * G.ny));
      const long long h = G.ih(i, j, k), h1 = G.ih(i, j, 1 - k);
      u[h] = u[h1];
      v[h] = v[h1];
      w[h] = -w[h1];
      d[h] = d[h1];
      T[h] = T[h1];
    } else {
      const double s1 = 0.5, s2 = 2.0;
      const int i = (int)(t % G.nx) + 1, k = (int)((t / G.nx) % G.nz) + 1, j = 1 - LAP + (int)(t / ((long long)G.nx * G.nz));
      const long long h = G.ih(i, j, k), hw = G.ih(i, 1, k), h1 = G.ih(i, 2 - j, k);
      u[h] = 2.0 * u[hw] - u[h1];
      v[h] = 2.0 * v[hw] - v[h1];
      w[h] = 2.0 * w[hw] - w[h1];
      double dg = 2.0 * d[hw] - d[h1];
      double Tg = 2.0 * T[hw] - T[h1];
      if (dg < s1 * d[hw]) dg = s1 * d[hw];
      if (dg > s2 * d[hw]) dg = s2 * d[hw];
      if (Tg < s1 * T[hw]) Tg = s1 * T[hw];
      if (Tg > s2 * T[hw]) Tg = s2 * T[hw];
      d[h] = dg;
      T[h] = Tg;
    }
  }
}

// Flow_Ghost_Extent_2nd (OCFD_GhostCell.f90:164-286): mirror extrapolation with
// the density/temperature limiter [0.8, 1.2] of the boundary value.
__global__ void k_ghost(Grid G, Phys ph, double* d, double* u, double* v, double* w, double* T) {
  const double s1 = 0.8, s2 = 1.2;
  long long cnt[6];
  long long tot = 0;
  for (int f = 0; f < 6; f++) {
    const int dir = f / 2;
    const long long tr = dir == 0 ? (long long)G.ny * G.nz : (dir == 1 ? (long long)G.nx * G.nz : (long long)G.nx * G.ny);
    cnt[f] = (ph.ghost[f] == 1 || ph.ghost[f] == 2) ? tr * LAP : 0;
    tot += cnt[f];
  }
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    long long e = t;
    int face = 0;
    while (e >= cnt[face]) e -= cnt[face++];
    const int dir = face / 2, hi = face % 2;
    const int nn = G.len(dir);
    const int l = (int)(e % LAP) + 1;
    e /= LAP;
    const int n1 = dir == 0 ? G.ny : G.nx;
    const int a = (int)(e % n1) + 1, b = (int)(e / n1) + 1;
    const int g = hi ? nn + l : 1 - l;
    const int g1 = hi ? 2 * nn - g : 2 - g;
    const int eb = hi ? nn : 1;
    auto H = [&](int along) -> long long {
      if (dir == 0) return G.ih(along, a, b);
      if (dir == 1) return G.ih(a, along, b);
      return G.ih(a, b, along);
    };
    const long long hg = H(g), he = H(eb), hg1 = H(g1);
    u[hg] = 2.0 * u[he] - u[hg1];
    v[hg] = 2.0 * v[he] - v[hg1];
    w[hg] = 2.0 * w[he] - w[hg1];
    double dg = 2.0 * d[he] - d[hg1];
    double Tg = 2.0 * T[he] - T[hg1];
    if (dg < s1 * d[he]) dg = s1 * d[he];
    if (dg > s2 * d[he]) dg = s2 * d[he];
    if (Tg < s1 * T[he]) Tg = s1 * T[he];
    if (Tg > s2 * T[he]) Tg = s2 * T[he];
    d[hg] = dg;
    T[hg] = Tg;
  }
}
cudaError_t launch_ghost(const Grid& g, const Phys& ph, double* const prim[5], cudaStream_t st) {
  bool any = false;
  for (int f = 0; f < 6; f++) any = any || ph.ghost[f] == 1 || ph.ghost[f] == 2;
  if (any) k_ghost<<<148 * 2, 256, 0, st>>>(g, ph, prim[0], prim[1], prim[2], prim[3], prim[4]);
  if ((ph.ibc == 3 && ph.ghost[4] == -1) || (ph.ibc == 2 && ph.ghost[2] == -1))
    k_ghost_user<<<148 * 2, 256, 0, st>>>(g, ph, prim[0], prim[1], prim[2], prim[3], prim[4]);
  return cudaGetLastError();
}

// FP32 copies of the primitives at the points a boundary condition may have
// changed after the stage tail wrote them: in every non-periodic direction the
// boundary plane and the ghost layers beyond it (all other points keep the
// tail's copies).  Grid: (nxh/32, nyh/8, nzh) threads over the haloed array.
__global__ void k_refresh_shell(Grid G, int px, int py, int pz, const double* d, const double* u, const double* v,
                                const double* w, const double* T, float* p32, float4* q32) {
  const int hi = blockIdx.x * 32 + (threadIdx.x & 31), hj = blockIdx.y * 8 + (threadIdx.x >> 5),
            hk = blockIdx.z;
  if (hi >= G.nxh || hj >= G.nyh) return;
  const int i = hi - LAP + 1, j = hj - LAP + 1, k = hk - LAP + 1;
  const bool shell = (!px && (i <= 1 || i >= G.nx)) || (!py && (j <= 1 || j >= G.ny)) ||
                     (!pz && (k <= 1 || k >= G.nz));
  if (!shell) return;
  const long long c = (long long)hi + (long long)G.nxh * ((long long)hj + (long long)G.nyh * hk);
  p32[c] = float(d[c]);
  q32[c] = make_float4(float(u[c]), float(v[c]), float(w[c]), float(T[c]));
}
cudaError_t launch_refresh_shell(const Grid& g, const int periodic[3], double* const prim[5], float* p32, float* q32,
                                 cudaStream_t st) {
  if (periodic[0] && periodic[1] && periodic[2]) return cudaSuccess;
  k_refresh_shell<<<dim3((g.nxh + 31) / 32, (g.nyh + 7) / 8, g.nzh), 256, 0, st>>>(
      g, periodic[0], periodic[1], periodic[2], prim[0], prim[1], prim[2], prim[3], prim[4], p32,
      reinterpret_cast<float4*>(q32));
  return cudaGetLastError();
}
__global__ void k_to_f32x4(const double* u, const double* v, const double* w, const double* T, float4* dst,
                           long long n) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    dst[c] = make_float4(float(u[c]), float(v[c]), float(w[c]), float(T[c]));
}
cudaError_t launch_to_f32x4(const double* u, const double* v, const double* w, const double* T, float* dst, long long n,
                            cudaStream_t st) {
  k_to_f32x4<<<148 * 8, 256, 0, st>>>(u, v, w, T, reinterpret_cast<float4*>(dst), n);
  return cudaGetLastError();
}
__global__ void k_to_f32(const double* src, float* dst, long long n) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    dst[c] = float(src[c]);
}
cudaError_t launch_to_f32(const double* src, float* dst, long long n, cudaStream_t st) {
  k_to_f32<<<148 * 8, 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}

// init3d (OCFD_init.f90:10-20)
__global__ void k_init3d(Grid G, double cv, double* f, const double* d, const double* u, const double* v,
                         const double* w, const double* T) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G.n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % G.nx) + 1, j = (int)((t / G.nx) % G.ny) + 1, k = (int)(t / ((long long)G.nx * G.ny)) + 1;
    const long long h = G.ih(i, j, k);
    const double dd = d[h], uu = u[h], vv = v[h], ww = w[h], TT = T[h];
    f[t] = dd;
    f[t + G.n] = dd * uu;
    f[t + 2 * G.n] = dd * vv;
    f[t + 3 * G.n] = dd * ww;
    f[t + 4 * G.n] = dd * ((uu * uu + vv * vv + ww * ww) * 0.5 + cv * TT);
  }
}
cudaError_t launch_init3d(const Grid& g, const Phys& ph, double* f, double* const prim[5], cudaStream_t st) {
  k_init3d<<<148 * 8, 256, 0, st>>>(g, ph.cv, f, prim[0], prim[1], prim[2], prim[3], prim[4]);
  return cudaGetLastError();
}

}  // namespace ocfd
