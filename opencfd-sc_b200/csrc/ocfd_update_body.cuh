// ocfd_update_body.cuh -- device bodies of the stage kernels (viscous
// gradients, flux and viscous divergence, the fused stage tail, the
// negative-temperature repair), shared by the single-instance and batched
// launches (ocfd_update.cu) and the persistent batched stage kernel
// (ocfd_batch_stage.cuh), so that all of them compute the same bits.
#pragma once

#include <utility>

#include "ocfd_kernels.h"
#include "ocfd_schemes.cuh"

// Minimum resident blocks per SM requested for the viscous-gradient and
// stage-tail kernels (both memory-latency bound: more resident warps keep
// more loads in flight, at the price of registers).  Measured best on B200 at
// 256^3: FP64 tail 4 with the face-flux records (3.52 against 3.75 ms per step
// at 5 blocks; with one array per face-flux component 5 was best: 3 / 4 / 6
// blocks 3.93 / 3.63 / 4.37 against 3.60 ms), FP32 tail 5 (with the
// interleaved viscous fluxes; 5 and 6 before), FP64 viscous 4 (3 / 5 / 6
// blocks: 3.48 / 4.04 / 5.49 against 2.76 ms per step: fewer warps expose the
// stencil-load latency, more spill), FP32 viscous 6 (against 2-3 blocks with
// the compiler's own register choice).
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
// FP64 viscous fluxes (four components of a point, 32 bytes) moved by single
// 256-bit global loads and stores
#ifndef OCFD_V256
#define OCFD_V256 1
#endif
#define OCFD_TAIL_MINB (sizeof(R) == 8 ? OCFD_TAIL64_MINB : OCFD_TAIL32_MINB)
// the batched launches (arguments from shared memory, the member search):
// the FP32 tail at 4 blocks (5 spilled about 600 bytes; 4 measured 0.5-1.5%
// faster over the served member sets), the viscous kernel as the single one
#ifndef OCFD_VISCB32_MINB
#define OCFD_VISCB32_MINB OCFD_VISC32_MINB
#endif
#ifndef OCFD_TAILB32_MINB
#define OCFD_TAILB32_MINB 4
#endif
#define OCFD_VISCB_MINB (sizeof(R) == 8 ? OCFD_VISC64_MINB : OCFD_VISCB32_MINB)
#define OCFD_TAILB_MINB (sizeof(R) == 8 ? OCFD_TAIL64_MINB : OCFD_TAILB32_MINB)

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
// the four components of one point of an interleaved viscous-flux array (32
// bytes, 32-byte aligned: the arrays start on 256-byte boundaries).
// OCFD_V256: one 256-bit access (sm_100) in place of two 16-byte ones.
__device__ __forceinline__ V4<double> ldg4(const double* p) {
#if OCFD_V256
  double a, b, c, d;
  asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
  return V4<double>{{a, b, c, d}};
#else
  const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
  return V4<double>{{a.x, a.y, b.x, b.y}};
#endif
}
__device__ __forceinline__ V4<float> ldg4(const float* p) {
  const float4 a = __ldg(reinterpret_cast<const float4*>(p));
  return V4<float>{{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ void st4(double* p, double a, double b, double c, double d) {
#if OCFD_V256
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a), "d"(b), "d"(c), "d"(d) : "memory");
#else
  // two 16-byte stores (four scalar stores measured 10% slower in the viscous kernel)
  reinterpret_cast<double2*>(p)[0] = make_double2(a, b);
  reinterpret_cast<double2*>(p)[1] = make_double2(c, d);
#endif
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
// Whether every off-diagonal metric the viscous body reads is identically zero
// (Aky Akz Aix Aiz Asx Asy of the gradients, Aky1 Akz1 Aix1 Aiz1 Asx1 Asy1 of the
// fluxes): a grid whose axes are the coordinate axes (box, stretched box).
#ifndef OCFD_VISC_AXS
#define OCFD_VISC_AXS OCFD_FEWER_DIVS
#endif
__host__ __device__ __forceinline__ bool visc_axis_aligned(unsigned int metzero) {
  const unsigned int off = (1u << 4) | (1u << 5) | (1u << 6) | (1u << 8) | (1u << 9) | (1u << 10) | (1u << 14) |
                           (1u << 15) | (1u << 16) | (1u << 18) | (1u << 19) | (1u << 20);
  return (metzero & off) == off;
}

// AXS (production build, visc_axis_aligned grids): the Cartesian gradients and
// the contravariant fluxes take only the diagonal metrics -- the general form's
// other terms add exact zeros, so the values are the same (up to the sign of a
// zero) with a third of the metric registers and products.
template <typename R, typename S, bool AXS = false>
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
  if constexpr (AXS) {
    // metric indices (flow_data order): Akx 3, Aiy 7, Asz 11, Akx1 13, Aiy1 17, Asz1 21
    const R Akx = R(__ldg(a.met[3] + c)), Aiy = R(__ldg(a.met[7] + c)), Asz = R(__ldg(a.met[11] + c));
    const R ux = gr[0][0] * Akx, vx = gr[1][0] * Akx, wx = gr[2][0] * Akx, Tx = gr[3][0] * Akx;
    const R uy = gr[0][1] * Aiy, vy = gr[1][1] * Aiy, wy = gr[2][1] * Aiy, Ty = gr[3][1] * Aiy;
    const R uz = gr[0][2] * Asz, vz = gr[1][2] * Asz, wz = gr[2][2] * Asz, Tz = gr[3][2] * Asz;
    const R div = ux + vy + wz;
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
    const R A1 = R(__ldg(a.met[13] + c)), A2 = R(__ldg(a.met[17] + c)), A3 = R(__ldg(a.met[21] + c));
    st4(a.ev + o * 4, A1 * s11, A1 * s12, A1 * s13, A1 * E1);
    st4(a.ev + (n + o) * 4, A2 * s12, A2 * s22, A2 * s23, A2 * E2);
    st4(a.ev + (2 * n + o) * 4, A3 * s13, A3 * s23, A3 * s33, A3 * E3);
  } else {
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
}

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
#if OCFD_HF_REC
  // record layout: the four leading components of a face in one 256-bit
  // (FP64) / 128-bit (FP32) load; the same operations, direction by direction
  {
    R acc[5];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const R* H = a.hf[d];
      const IX fs = (IX)a.fs[d];
      R h1[5], h0[5];
      rec4_load(H + 4 * f1[d], h1);
      rec4_load(H + 4 * f0[d], h0);
      h1[4] = H[4 * fs + f1[d]];
      h0[4] = H[4 * fs + f0[d]];
#pragma unroll
      for (int m = 0; m < 5; m++) {
        const R dd = (h1[m] - h0[m]) * R(a.h_1[d]);
        if (d == 0)
          acc[m] = dd;
        else if (d == 1)
          acc[m] = acc[m] + dd;
        else
          du[m] = -(acc[m] + dd) * ajac;
      }
    }
  }
#else
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
#endif
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

// handle_NegativeT (OCFD_handle_NegativeT.f90:1-17) for the points detected in
// this stage, in the reference's loop order (k, j, i).  The reference repairs
// in place while sweeping, so a neighbour earlier in the sweep contributes its
// new value and a later neighbour (or a halo cell) the value of the previous
// stage, kept in told.  More than 10 points: the reference stops (:13-16).
// Values that other blocks of the same launch may have written (the persistent
// batched stage kernel runs this after the member's stage tail) are read
// through L2, past this SM's L1.
__device__ __forceinline__ void negt_fix_body(const UpdArgs<double>& a) {
  DevStatus* st = a.st;
  const int cnt = __ldcg(&st->negt_count);
  st->negt_last = cnt;
  if (cnt == 0) return;
  st->negt_count = 0;
  st->negt_total += cnt;
  if (cnt > 10) {
    // a gave-up wait of this step (4, 5) is the cause to report: it stays
    const int prev = __ldcg(&st->error);
    if (prev != 4 && prev != 5) st->error = 3;
    return;
  }
  int idx[16];
  for (int q = 0; q < cnt; q++) idx[q] = __ldcg(&st->negt_list[q]);
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
    auto Tv = [&](long long nb) -> double { return (interior(nb) && nb < h) ? __ldcg(Tn + nb) : a.told[nb]; };
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
        double qv[5] = {__ldcg(a.prim[0] + h), __ldcg(a.prim[1] + h), __ldcg(a.prim[2] + h),
                        __ldcg(a.prim[3] + h), T},
               fv[5];
        if (a.lean && a.krk < 3) {
          // FP64 d,u,v,w were not written this stage: recover them from f
          double fo[5], qo[5];
          for (int m = 0; m < 5; m++) fo[m] = __ldcg(a.f + o + m * G.n);
          prims_of(fo, a.ph.cv, a.ph.inv_cv, qo);
          for (int m = 0; m < 4; m++) qv[m] = qo[m];
        }
        refresh_of(qv, a.ph.cv, fv);
        for (int m = 0; m < 5; m++) a.f[o + m * G.n] = fv[m];
      }
    }
  }
}

}  // namespace ocfd
