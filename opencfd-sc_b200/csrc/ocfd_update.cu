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

#include "ocfd_kernels.h"
#include "ocfd_schemes.cuh"

// Minimum resident blocks per SM requested for the viscous-gradient and
// stage-tail kernels (both memory-latency bound: more resident warps keep
// more loads in flight, at the price of registers).  Measured best on B200 at
// 256^3: FP64 tail 4, FP32 tail 5 (with the interleaved viscous fluxes; 5 and
// 6 before), FP64 viscous 4, FP32 viscous 6 (against 2-3 blocks with the
// compiler's own register choice).
#ifndef OCFD_VISC64_MINB
#define OCFD_VISC64_MINB 4
#endif
#ifndef OCFD_VISC32_MINB
#define OCFD_VISC32_MINB 6
#endif
#ifndef OCFD_TAIL64_MINB
#define OCFD_TAIL64_MINB 4
#endif
#ifndef OCFD_TAIL32_MINB
#define OCFD_TAIL32_MINB 5
#endif
#define OCFD_VISC_MINB (sizeof(R) == 8 ? OCFD_VISC64_MINB : OCFD_VISC32_MINB)
#define OCFD_TAIL_MINB (sizeof(R) == 8 ? OCFD_TAIL64_MINB : OCFD_TAIL32_MINB)

namespace ocfd {

// ---------------------------------------------------------------------------
// Central derivatives OCFD_dx0/dy0/dz0 (OCFD_dxyz_viscous.f90:3-239) of a
// pencil given by an accessor at(off) = q(l+off).  Interior CD6/CD8 and the
// low-order closures of a non-periodic boundary.
// Coefficients of one direction, by value (no reference into the kernel's
// parameter block, which would force it into local memory).
template <typename R>
struct D0C {
  R h, a1, a2, a3, c1, c2, c3, c4;
};
template <typename R>
__device__ __forceinline__ D0C<R> d0c(const DCoef& c, int dir) {
  return D0C<R>{R(c.h[dir]), R(c.a1[dir]), R(c.a2[dir]), R(c.a3[dir]),
                R(c.c1[dir]), R(c.c2[dir]), R(c.c3[dir]), R(c.c4[dir])};
}

// Four values operated on element by element (the four viscous-flux components
// of one direction, differentiated together); each element sees exactly the
// scalar operations.
template <typename R>
struct V4 {
  R v[4];
};
template <typename R>
__device__ __forceinline__ V4<R> operator+(const V4<R>& a, const V4<R>& b) {
  return V4<R>{{a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2], a.v[3] + b.v[3]}};
}
template <typename R>
__device__ __forceinline__ V4<R> operator-(const V4<R>& a, const V4<R>& b) {
  return V4<R>{{a.v[0] - b.v[0], a.v[1] - b.v[1], a.v[2] - b.v[2], a.v[3] - b.v[3]}};
}
template <typename R>
__device__ __forceinline__ V4<R> operator*(R c, const V4<R>& a) {
  return V4<R>{{c * a.v[0], c * a.v[1], c * a.v[2], c * a.v[3]}};
}
template <typename R>
__device__ __forceinline__ V4<R> operator/(const V4<R>& a, R c) {
  return V4<R>{{a.v[0] / c, a.v[1] / c, a.v[2] / c, a.v[3] / c}};
}
// the four components of one point of an interleaved viscous-flux array
__device__ __forceinline__ V4<double> ldg4(const double* p) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
  return V4<double>{{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ V4<float> ldg4(const float* p) {
  const float4 a = __ldg(reinterpret_cast<const float4*>(p));
  return V4<float>{{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ void st4(double* p, double a, double b, double c, double d) {
  // two 16-byte stores (four scalar stores measured 10% slower in the viscous kernel)
  reinterpret_cast<double2*>(p)[0] = make_double2(a, b);
  reinterpret_cast<double2*>(p)[1] = make_double2(c, d);
}
__device__ __forceinline__ void st4(float* p, float a, float b, float c, float d) {
  *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
}

// Closures only: called for l in {1,2,3,(4)} or {(n-3),n-2,n-1,n}, never reads
// outside 1..n along the direction (the Ev arrays carry no halo).  V: the
// accessor's value type (R, or V4<R> for four components at once).
template <typename R, typename F, typename V = decltype(std::declval<F>()(0))>
__device__ __forceinline__ V d0_bnd(F at, int l, int nn, int cd8, D0C<R> k) {
  V r = V();
  if (l == 1) r = (R(-3) * at(0) + R(4) * at(1) - at(2)) / (R(2) * k.h);
  else if (l == 2) r = (at(1) - at(-1)) / (R(2) * k.h);
  else if (l == 3) r = (R(8) * (at(1) - at(-1)) - (at(2) - at(-2))) / (R(12) * k.h);
  else if (cd8 && l == 4) r = k.a1 * (at(3) - at(-3)) + k.a2 * (at(2) - at(-2)) + k.a3 * (at(1) - at(-1));
  if (l == nn) r = (at(-2) - R(4) * at(-1) + R(3) * at(0)) / (R(2) * k.h);
  else if (l == nn - 1) r = (at(1) - at(-1)) / (R(2) * k.h);
  else if (l == nn - 2) r = (R(8) * (at(1) - at(-1)) - (at(2) - at(-2))) / (R(12) * k.h);
  else if (cd8 && l == nn - 3) r = k.a1 * (at(3) - at(-3)) + k.a2 * (at(2) - at(-2)) + k.a3 * (at(1) - at(-1));
  return r;
}

template <typename R, typename F, typename V = decltype(std::declval<F>()(0))>
__device__ __forceinline__ V d0(F at, int l, int nn, int periodic, int cd8, D0C<R> k) {
  const int lo = cd8 ? 4 : 3, hi = cd8 ? nn - 3 : nn - 2;
  if (periodic || (l > lo && l < hi)) {
    if (!cd8) return k.a1 * (at(3) - at(-3)) + k.a2 * (at(2) - at(-2)) + k.a3 * (at(1) - at(-1));
    return k.c1 * (at(1) - at(-1)) + k.c2 * (at(2) - at(-2)) + k.c3 * (at(3) - at(-3)) + k.c4 * (at(4) - at(-4));
  }
  return d0_bnd<R, F, V>(at, l, nn, cd8, k);
}

// ---------------------------------------------------------------------------
// du_viscous part 1 (OCFD_viscous.f90:193-264): comput_Amu (:135-149), the 12
// gradients, stress and heat flux, and the contravariant viscous fluxes Ev.
template <typename R, typename S>
__device__ __forceinline__ void visc_grad_body(const ViscArgs<R, S>& a, const int bx, const int by, const int bz) {
  const Grid& G = a.g;
  const int i = bx * 32 + (threadIdx.x & 31) + 1;
  const int j = by * 8 + (threadIdx.x >> 5) + 1;
  const int k = bz + 1;
  if (i > G.nx || j > G.ny) return;
  const long long c = G.ih(i, j, k);
  const int cd8 = a.ph.scheme_vis == 6;
  const int lcoord[3] = {i, j, k};
  R gr[4][3];  // [u,v,w,T][k,i,s]
  R uu, vv, ww, T;
  if constexpr (sizeof(S) == 4) {
    // FP32 copies: u,v,w,T interleaved, one 16-byte load per stencil point
    const float4* base = reinterpret_cast<const float4*>(a.q4) + c;
#pragma unroll
    for (int dir = 0; dir < 3; dir++) {
      const long long hs = G.hstride(dir);
      auto at = [&](int off) -> V4<R> {
        const float4 t = __ldg(base + off * hs);
        return V4<R>{{R(t.x), R(t.y), R(t.z), R(t.w)}};
      };
      const V4<R> g4 = d0<R>(at, lcoord[dir], G.len(dir), a.ph.periodic[dir], cd8, d0c<R>(a.dc, dir));
#pragma unroll
      for (int q = 0; q < 4; q++) gr[q][dir] = g4.v[q];
    }
    const float4 t = __ldg(base);
    uu = R(t.x);
    vv = R(t.y);
    ww = R(t.z);
    T = R(t.w);
  } else {
    const S* q4[4] = {a.u, a.v, a.w, a.T};
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int dir = 0; dir < 3; dir++) {
        const long long hs = G.hstride(dir);
        const S* base = q4[q] + c;
        auto at = [&](int off) -> R { return R(__ldg(base + off * hs)); };
        gr[q][dir] = d0<R>(at, lcoord[dir], G.len(dir), a.ph.periodic[dir], cd8, d0c<R>(a.dc, dir));
      }
  }
  R M[22];
#pragma unroll
  for (int m = 3; m < 22; m++) M[m] = met_at<R>(a.ph, m, a.met[m], c);
  const R Akx = M[3], Aky = M[4], Akz = M[5], Aix = M[6], Aiy = M[7], Aiz = M[8], Asx = M[9], Asy = M[10],
          Asz = M[11];
  const R ux = gr[0][0] * Akx + gr[0][1] * Aix + gr[0][2] * Asx;
  const R vx = gr[1][0] * Akx + gr[1][1] * Aix + gr[1][2] * Asx;
  const R wx = gr[2][0] * Akx + gr[2][1] * Aix + gr[2][2] * Asx;
  const R Tx = gr[3][0] * Akx + gr[3][1] * Aix + gr[3][2] * Asx;
  const R uy = gr[0][0] * Aky + gr[0][1] * Aiy + gr[0][2] * Asy;
  const R vy = gr[1][0] * Aky + gr[1][1] * Aiy + gr[1][2] * Asy;
  const R wy = gr[2][0] * Aky + gr[2][1] * Aiy + gr[2][2] * Asy;
  const R Ty = gr[3][0] * Aky + gr[3][1] * Aiy + gr[3][2] * Asy;
  const R uz = gr[0][0] * Akz + gr[0][1] * Aiz + gr[0][2] * Asz;
  const R vz = gr[1][0] * Akz + gr[1][1] * Aiz + gr[1][2] * Asz;
  const R wz = gr[2][0] * Akz + gr[2][1] * Aiz + gr[2][2] * Asz;
  const R Tz = gr[3][0] * Akz + gr[3][1] * Aiz + gr[3][2] * Asz;
  const R div = ux + vy + wz;
  // Sutherland viscosity, comput_Amu
  const R Tsb = R(110.4 / a.ph.ref_amu_t0), TmpR = R(1.0 / a.ph.re);
  if constexpr (sizeof(S) != 4) T = R(__ldg(a.T + c));
  const R Amu = TmpR * (R(1) + Tsb) * sqrt(T * T * T) / (Tsb + T);
  const R Amuk = R(a.ph.cp) * Amu / R(a.ph.pr);
  const R t23 = R(2.0 / 3.0);
  const R s11 = (R(2) * ux - t23 * div) * Amu;
  const R s22 = (R(2) * vy - t23 * div) * Amu;
  const R s33 = (R(2) * wz - t23 * div) * Amu;
  const R s12 = (uy + vx) * Amu;
  const R s13 = (uz + wx) * Amu;
  const R s23 = (vz + wy) * Amu;
  if constexpr (sizeof(S) != 4) {
    uu = R(__ldg(a.u + c));
    vv = R(__ldg(a.v + c));
    ww = R(__ldg(a.w + c));
  }
  const R E1 = uu * s11 + vv * s12 + ww * s13 + Amuk * Tx;
  const R E2 = uu * s12 + vv * s22 + ww * s23 + Amuk * Ty;
  const R E3 = uu * s13 + vv * s23 + ww * s33 + Amuk * Tz;
  const long long o = G.ii(i, j, k);
  const long long n = G.n;
  // Ev stored direction by direction, the four components of a point together:
  // element (d, point o, component m) at (d*n + o)*4 + m
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const R A1 = M[13 + 3 * d], A2 = M[14 + 3 * d], A3 = M[15 + 3 * d];
    st4(a.ev + ((long long)d * n + o) * 4, A1 * s11 + A2 * s12 + A3 * s13, A1 * s12 + A2 * s22 + A3 * s23,
        A1 * s13 + A2 * s23 + A3 * s33, A1 * E1 + A2 * E2 + A3 * E3);
  }
}

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

template <typename R, typename S, bool SLAB>
__global__ void __launch_bounds__(256, OCFD_VISC_MINB) k_visc_grad(ViscArgs<R, S> a, SlabOrder so) {
  if (!SLAB) {
    visc_grad_body(a, blockIdx.x, blockIdx.y, blockIdx.z);
    return;
  }
  int bx, by, bz;
  if (!slab_decode(so, a.g.nz, bx, by, bz)) return;
  visc_grad_body(a, bx, by, bz);
}
template <typename R, typename S>
__global__ void __launch_bounds__(256, OCFD_VISC_MINB) k_visc_grad_batch(BatchTab<ViscArgs<R, S>> b) {
  __shared__ __align__(16) ViscArgs<R, S> sa;
  int bx, by, bz;
  const int q = batch_locate(b, blockIdx.x, bx, by, bz);
  visc_grad_body(batch_args(b, q, &sa), bx, by, bz);
}

template <typename R, typename S>
cudaError_t launch_visc_grad(const ViscArgs<R, S>& a, cudaStream_t st) {
  const SlabOrder so = slab_order(a.g);
  if (so.sy == so.gy)
    k_visc_grad<R, S, false><<<update_dims(a.g), 256, 0, st>>>(a, so);
  else
    k_visc_grad<R, S, true><<<slab_grid(so, a.g.nz), 256, 0, st>>>(a, so);
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
// Flux difference of the three sweeps into du (OCFD_inviscous.f90:106-108,
// :144-146, :182-184; OCFD_inviscous_character.f90:58-62, :98-102, :137-141),
// plus the mass force (:189-201).
// IX: index type of the face / viscous-flux offsets (int when every offset fits,
// measured 6% faster on the FP32 tail; long long otherwise).
template <bool CHAR, typename R, typename IX = long long>
__device__ __forceinline__ void inv_div(const UpdArgs<R>& a, int i, int j, int k, R du[5]) {
  const Grid& G = a.g;
  const int lc[3] = {i, j, k};
  IX f1[3], f0[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const int l = lc[d];
    const int lm = (l == 1 && a.fper[d]) ? G.len(d) : l - 1;
    f1[d] = (IX)G.face(d, l, i, j, k);
    f0[d] = (IX)G.face(d, lm, i, j, k);
  }
  const R ajac = R(a.ajac[G.ih(i, j, k)]);
#pragma unroll
  for (int m = 0; m < 5; m++) {
    R dd[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const R* H = a.hf[d];
      const IX fs = (IX)a.fs[d];
      if (!CHAR && !OCFD_FV_SUMMED)
        dd[d] = (H[f1[d] + m * fs] - H[f0[d] + m * fs] + H[f1[d] + (5 + m) * fs] - H[f0[d] + (5 + m) * fs]) *
                R(a.h_1[d]);
      else
        dd[d] = (H[f1[d] + m * fs] - H[f0[d] + m * fs]) * R(a.h_1[d]);
    }
    R acc = dd[0];
    acc = acc + dd[1];
    du[m] = -(acc + dd[2]) * ajac;
  }
  if (a.ph.if_mass_force == 1) {
    const long long c = G.ih(i, j, k);
    const R d = R(a.pd[c]), u = R(a.pu[c]), v = R(a.pv[c]), w = R(a.pw[c]);
    const R F0 = R(a.ph.mass_force[0]), F1 = R(a.ph.mass_force[1]), F2 = R(a.ph.mass_force[2]);
    du[1] = du[1] + d * F0;
    du[2] = du[2] + d * F1;
    du[3] = du[3] + d * F2;
    du[4] = du[4] + d * (u * F0 + v * F1 + w * F2);
  }
}

// du_viscous part 2 (OCFD_viscous.f90:266-282): du(:,:,:,m+1) +=
// (d/dxi Ev1 + d/deta Ev2 + d/dzeta Ev3) * Ajac, periodic directions read
// the wrapped neighbours (the reference's exchange_boundary_x/y/z of Ev).
template <typename R, typename IX = long long>
__device__ __forceinline__ void visc_div(const UpdArgs<R>& a, int i, int j, int k, R du[5]) {
  const Grid& G = a.g;
  const int cd8 = a.ph.scheme_vis == 6;
  const IX o = (IX)G.ii(i, j, k);
  const IX n = (IX)G.n;
  const int lc[3] = {i, j, k};
  const IX is[3] = {1, (IX)G.nx, (IX)G.nx * (IX)G.ny};
  const R ajac = R(a.ajac[G.ih(i, j, k)]);
  // points within 4 of a periodic end read wrapped neighbours (the Ev arrays
  // carry no halo); the others address their neighbours directly
  bool wz[3];
#pragma unroll
  for (int d = 0; d < 3; d++) wz[d] = a.ph.periodic[d] && (lc[d] <= 4 || lc[d] > G.len(d) - 4);
  V4<R> s[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const R* E = a.ev + ((IX)d * n + o) * 4;
    const int l = lc[d], nn = G.len(d);
    const int per = a.ph.periodic[d];
    const IX st = is[d] * 4;
    if (!wz[d]) {
      auto at = [&](int off) -> V4<R> { return ldg4(E + (IX)off * st); };
      s[d] = d0<R>(at, l, nn, per, cd8, d0c<R>(a.dc, d));
    } else {
      auto at = [&](int off) -> V4<R> {
        int l2 = l + off;
        l2 = l2 < 1 ? l2 + nn : (l2 > nn ? l2 - nn : l2);
        return ldg4(E + (IX)(l2 - l) * st);
      };
      s[d] = d0<R>(at, l, nn, per, cd8, d0c<R>(a.dc, d));
    }
  }
#pragma unroll
  for (int m = 0; m < 4; m++) du[m + 1] = du[m + 1] + (s[0].v[m] + s[1].v[m] + s[2].v[m]) * ajac;
}

// primitive recovery of one point (comput_duvwT, OCFD_Time_Adv.f90:48-52)
// (production build: one reciprocal of the density instead of four divisions)
__device__ __forceinline__ void prims_of(const double* f, double cv, double inv_cv, double* q) {
  const double f1 = f[0], f2 = f[1], f3 = f[2], f4 = f[3], f5 = f[4];
  q[0] = f1;
#if OCFD_FEWER_DIVS
  const double r1 = 1.0 / f1;
  q[1] = f2 * r1;
  q[2] = f3 * r1;
  q[3] = f4 * r1;
  q[4] = (f5 - (f2 * q[1] + f3 * q[2] + f4 * q[3]) * 0.5) * (r1 * inv_cv);
#else
  q[1] = f2 / f1;
  q[2] = f3 / f1;
  q[3] = f4 / f1;
  q[4] = (f5 - (f2 * q[1] + f3 * q[2] + f4 * q[3]) * 0.5) / (f1 * cv);
#endif
}

// f from primitives on a boundary face (OCFD_BC.f90:153-157)
__device__ __forceinline__ void refresh_of(const double* q, double cv, double* f) {
  const double d = q[0], u = q[1], v = q[2], w = q[3], T = q[4];
  f[0] = d;
  f[1] = d * u;
  f[2] = d * v;
  f[3] = d * w;
  f[4] = d * (cv * T + (u * u + v * v + w * w) * 0.5);
}

__device__ __forceinline__ bool on_boundary_face(const Grid& G, int i, int j, int k) {
  return i == 1 || i == G.nx || j == 1 || j == G.ny || k == 1 || k == G.nz;
}

// write value x of haloed array p at (i,j,k) into its periodic face-halo images
__device__ __forceinline__ void mirror(const Grid& G, const int* per, double* p, int i, int j, int k, double x) {
  if (per[0]) {
    if (i <= LAP) p[G.ih(i + G.nx, j, k)] = x;
    if (i > G.nx - LAP) p[G.ih(i - G.nx, j, k)] = x;
  }
  if (per[1]) {
    if (j <= LAP) p[G.ih(i, j + G.ny, k)] = x;
    if (j > G.ny - LAP) p[G.ih(i, j - G.ny, k)] = x;
  }
  if (per[2]) {
    if (k <= LAP) p[G.ih(i, j, k + G.nz)] = x;
    if (k > G.nz - LAP) p[G.ih(i, j, k - G.nz)] = x;
  }
}
__device__ __forceinline__ void mirror32(const Grid& G, const int* per, float* p, int i, int j, int k, float x) {
  if (per[0]) {
    if (i <= LAP) p[G.ih(i + G.nx, j, k)] = x;
    if (i > G.nx - LAP) p[G.ih(i - G.nx, j, k)] = x;
  }
  if (per[1]) {
    if (j <= LAP) p[G.ih(i, j + G.ny, k)] = x;
    if (j > G.ny - LAP) p[G.ih(i, j - G.ny, k)] = x;
  }
  if (per[2]) {
    if (k <= LAP) p[G.ih(i, j, k + G.nz)] = x;
    if (k > G.nz - LAP) p[G.ih(i, j, k - G.nz)] = x;
  }
}

// the same for one component (stride 4, offset c) of an interleaved FP32 array
__device__ __forceinline__ void mirror32c(const Grid& G, const int* per, float* p, int c, int i, int j, int k,
                                          float x) {
  if (per[0]) {
    if (i <= LAP) p[4 * G.ih(i + G.nx, j, k) + c] = x;
    if (i > G.nx - LAP) p[4 * G.ih(i - G.nx, j, k) + c] = x;
  }
  if (per[1]) {
    if (j <= LAP) p[4 * G.ih(i, j + G.ny, k) + c] = x;
    if (j > G.ny - LAP) p[4 * G.ih(i, j - G.ny, k) + c] = x;
  }
  if (per[2]) {
    if (k <= LAP) p[4 * G.ih(i, j, k + G.nz) + c] = x;
    if (k > G.nz - LAP) p[4 * G.ih(i, j, k - G.nz) + c] = x;
  }
}
__device__ __forceinline__ void mirror4(const Grid& G, const int* per, float4* p, int i, int j, int k, float4 x) {
  if (per[0]) {
    if (i <= LAP) p[G.ih(i + G.nx, j, k)] = x;
    if (i > G.nx - LAP) p[G.ih(i - G.nx, j, k)] = x;
  }
  if (per[1]) {
    if (j <= LAP) p[G.ih(i, j + G.ny, k)] = x;
    if (j > G.ny - LAP) p[G.ih(i, j - G.ny, k)] = x;
  }
  if (per[2]) {
    if (k <= LAP) p[G.ih(i, j, k + G.nz)] = x;
    if (k > G.nz - LAP) p[G.ih(i, j, k - G.nz)] = x;
  }
}

__device__ __forceinline__ void record_negt(DevStatus* st, long long h) {
  int slot = atomicAdd(&st->negt_count, 1);
  if (slot < 16) st->negt_list[slot] = (int)h;
}

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

// The fused stage tail.
template <bool CHAR, bool VISC, bool FUSEBC, typename R, typename IX = long long>
__device__ __forceinline__ void fused_body(const UpdArgs<R>& a, const int bx, const int by, const int bz) {
  const Grid& G = a.g;
  const int i = bx * 32 + (threadIdx.x & 31) + 1;
  const int j = by * 8 + (threadIdx.x >> 5) + 1;
  const int k = bz + 1;
  if (i > G.nx || j > G.ny) return;
  R du[5];
  inv_div<CHAR, R, IX>(a, i, j, k, du);
  if (VISC) visc_div<R, IX>(a, i, j, k, du);
  const long long o = G.ii(i, j, k);
  const long long n = G.n;
  double dd[5];
#pragma unroll
  for (int m = 0; m < 5; m++) dd[m] = double(du[m]);
  if (a.du)
#pragma unroll
    for (int m = 0; m < 5; m++) a.du[o + m * n] = dd[m];
  // OCFD_time_adv_RK3 (OCFD_Time_Adv.f90:14-35)
  double fv[5];
  const double dt = a.ph.dt;
  if (a.krk == 1) {
#pragma unroll
    for (int m = 0; m < 5; m++) fv[m] = a.fn[o + m * n] + dt * dd[m];
  } else {
    const double al = a.krk == 2 ? 3.0 / 4.0 : 1.0 / 3.0;
    const double be = a.krk == 2 ? 1.0 / 4.0 : 2.0 / 3.0;
#pragma unroll
    for (int m = 0; m < 5; m++) fv[m] = al * a.fn[o + m * n] + be * (a.f[o + m * n] + dt * dd[m]);
  }
  double q[5];
  prims_of(fv, a.ph.cv, a.ph.inv_cv, q);
  const long long h = G.ih(i, j, k);
  if (q[4] <= 0.0) record_negt(a.st, h);
  if (FUSEBC && on_boundary_face(G, i, j, k)) refresh_of(q, a.ph.cv, fv);
#pragma unroll
  for (int m = 0; m < 5; m++) a.f[o + m * n] = fv[m];
  const int m0 = (a.lean && a.krk < 3) ? 4 : 0;  // lean stages: FP64 T only
#pragma unroll
  for (int m = 0; m < 5; m++) {
    if (m >= m0) {
      a.prim[m][h] = q[m];
      if (FUSEBC) mirror(G, a.ph.periodic, a.prim[m], i, j, k, q[m]);
    }
  }
  if (a.p32[0]) {
    a.p32[0][h] = float(q[0]);
    if (FUSEBC) mirror32(G, a.ph.periodic, a.p32[0], i, j, k, float(q[0]));
    const float4 x = make_float4(float(q[1]), float(q[2]), float(q[3]), float(q[4]));
    float4* q4 = reinterpret_cast<float4*>(a.q32);
    q4[h] = x;
    if (FUSEBC) mirror4(G, a.ph.periodic, q4, i, j, k, x);
  }
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
template <bool CHAR, bool VISC, bool FUSEBC, typename R>
__global__ void __launch_bounds__(256, OCFD_TAIL_MINB) k_fused_batch(BatchTab<UpdArgs<R>> b) {
  __shared__ __align__(16) UpdArgs<R> sa;
  int bx, by, bz;
  const int q = batch_locate(b, blockIdx.x, bx, by, bz);
  fused_body<CHAR, VISC, FUSEBC, R>(batch_args(b, q, &sa), bx, by, bz);
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
                               cudaStream_t st) {
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
template cudaError_t launch_fused_batch<double>(const BatchTab<UpdArgs<double>>&, int, bool, bool, bool, cudaStream_t);
template cudaError_t launch_fused_batch<float>(const BatchTab<UpdArgs<float>>&, int, bool, bool, bool, cudaStream_t);
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

// handle_NegativeT (OCFD_handle_NegativeT.f90:1-17) for the points detected in
// this stage, in the reference's loop order (k, j, i).  The reference repairs
// in place while sweeping, so a neighbour earlier in the sweep contributes its
// new value and a later neighbour (or a halo cell) the value of the previous
// stage, kept in told.  More than 10 points: the reference stops (:13-16).
__device__ __forceinline__ void negt_fix_body(const UpdArgs<double>& a) {
  DevStatus* st = a.st;
  const int cnt = st->negt_count;
  st->negt_last = cnt;
  if (cnt == 0) return;
  st->negt_count = 0;
  st->negt_total += cnt;
  if (cnt > 10) {
    st->error = 3;
    return;
  }
  int idx[16];
  for (int q = 0; q < cnt; q++) idx[q] = st->negt_list[q];
  for (int p = 1; p < cnt; p++)  // insertion sort, cnt <= 10
    for (int q = p; q > 0 && idx[q - 1] > idx[q]; q--) {
      int t = idx[q];
      idx[q] = idx[q - 1];
      idx[q - 1] = t;
    }
  const Grid& G = a.g;
  double* Tn = a.prim[4];
  const long long sx = 1, sy = G.nxh, sz = (long long)G.nxh * G.nyh;
  auto interior = [&](long long h) -> bool {
    long long i = h % G.nxh - (LAP - 1), r = h / G.nxh;
    long long j = r % G.nyh - (LAP - 1), k = r / G.nyh - (LAP - 1);
    return i >= 1 && i <= G.nx && j >= 1 && j <= G.ny && k >= 1 && k <= G.nz;
  };
  for (int q = 0; q < cnt; q++) {
    const long long h = idx[q];
    auto Tv = [&](long long nb) -> double { return (interior(nb) && nb < h) ? Tn[nb] : a.told[nb]; };
    const double T = (Tv(h + sx) + Tv(h - sx) + Tv(h + sy) + Tv(h - sy) + Tv(h + sz) + Tv(h - sz)) / 6.0;
    Tn[h] = T;
    const int i = (int)(h % G.nxh) - (LAP - 1);
    const int j = (int)((h / G.nxh) % G.nyh) - (LAP - 1);
    const int k = (int)(h / ((long long)G.nxh * G.nyh)) - (LAP - 1);
    if (a.p32[0]) a.q32[4 * h + 3] = float(T);
    if (a.fuse_bc) {
      mirror(G, a.ph.periodic, Tn, i, j, k, T);
      if (a.p32[0]) mirror32c(G, a.ph.periodic, a.q32, 3, i, j, k, float(T));
      if (on_boundary_face(G, i, j, k)) {
        const long long o = G.ii(i, j, k);
        double qv[5] = {a.prim[0][h], a.prim[1][h], a.prim[2][h], a.prim[3][h], T}, fv[5];
        if (a.lean && a.krk < 3) {
          // FP64 d,u,v,w were not written this stage: recover them from f
          double fo[5], qo[5];
          for (int m = 0; m < 5; m++) fo[m] = a.f[o + m * G.n];
          prims_of(fo, a.ph.cv, a.ph.inv_cv, qo);
          for (int m = 0; m < 4; m++) qv[m] = qo[m];
        }
        refresh_of(qv, a.ph.cv, fv);
        for (int m = 0; m < 5; m++) a.f[o + m * G.n] = fv[m];
      }
    }
  }
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
