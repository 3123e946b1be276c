// ocfd_schemes.cuh -- point-form upwind reconstructions on a register window.
//
// v points at the window element of the face's left point, so v[-3..4] are the
// stencil values f(i-3..i+4) around face i+1/2.  Each function restates one
// reference routine operation by operation (no reassociation), so that an
// FP64 build without FMA contraction reproduces the reference bit for bit;
// the normal build lets the compiler contract a*b+c into FMAs.
//
// R is the arithmetic type: double for the FP64 path, float for the mixed path.
#pragma once

#include <cuda_runtime.h>

namespace ocfd {

template <typename R>
__device__ __forceinline__ R sq(R x) { return x * x; }

#ifndef OCFD_FEWER_DIVS
#ifdef OCFD_STRICT
#define OCFD_FEWER_DIVS 0
#else
#define OCFD_FEWER_DIVS 1
#endif
#endif

// Normalised WENO sum (a0 q0 + ...) / (a0 + ...) with a_k = C_k / (ep + S_k)^2,
// in the reference's order.  Production FP64 build: every a_k is multiplied by
// the product of all (ep + S_j)^2, a'_k = C_k prod_{j != k} (ep + S_j)^2, which
// leaves the normalised weights unchanged and needs one division instead of
// one per candidate plus one.  (ep + S)^2 >= ep^2, and the indicators of
// physical fluxes keep the products far inside the double range; FP32, whose
// range is too small for the products, keeps the reference form.
template <typename R>
__device__ __forceinline__ R weno_sum3(R ep, R C0, R C1, R C2, R S0, R S1, R S2, R q0, R q1, R q2) {
#if OCFD_FEWER_DIVS
  if (sizeof(R) == 8) {
    const R D0 = sq(ep + S0), D1 = sq(ep + S1), D2 = sq(ep + S2);
    const R w0 = C0 * (D1 * D2), w1 = C1 * (D0 * D2), w2 = C2 * (D0 * D1);
    return (w0 * q0 + w1 * q1 + w2 * q2) / (w0 + w1 + w2);
  }
#endif
  R a0 = C0 / sq(ep + S0);
  R a1 = C1 / sq(ep + S1);
  R a2 = C2 / sq(ep + S2);
  R am = a0 + a1 + a2;
  return (a0 * q0 + a1 * q1 + a2 * q2) / am;
}
template <typename R>
__device__ __forceinline__ R weno_sum4(R ep, R C0, R C1, R C2, R C3, R S0, R S1, R S2, R S3, R q0, R q1, R q2,
                                       R q3) {
#if OCFD_FEWER_DIVS
  if (sizeof(R) == 8) {
    const R D0 = sq(ep + S0), D1 = sq(ep + S1), D2 = sq(ep + S2), D3 = sq(ep + S3);
    const R P01 = D0 * D1, P23 = D2 * D3;
    const R w0 = C0 * (D1 * P23), w1 = C1 * (D0 * P23), w2 = C2 * (P01 * D3), w3 = C3 * (P01 * D2);
    return (w0 * q0 + w1 * q1 + w2 * q2 + w3 * q3) / (w0 + w1 + w2 + w3);
  }
#endif
  R a0 = C0 / sq(ep + S0);
  R a1 = C1 / sq(ep + S1);
  R a2 = C2 / sq(ep + S2);
  R a3 = C3 / sq(ep + S3);
  R am = a0 + a1 + a2 + a3;
  return (a0 * q0 + a1 * q1 + a2 * q2 + a3 * q3) / am;
}

template <typename R>
__device__ __forceinline__ R sign1(R b) { return copysign(R(1), b); }

template <typename R>
__device__ __forceinline__ R rmin(R a, R b) { return a < b ? a : b; }
template <typename R>
__device__ __forceinline__ R rmax(R a, R b) { return a > b ? a : b; }

// hh_weno5P: OCFD_Schemes_1.f90:9-29 (array form OCFD_weno5P, OCFD_Schemes.f90:6-28)
template <typename R>
__device__ __forceinline__ R weno5P(const R* v) {
  const R ep = R(1.0e-6), C03 = R(3.0 / 10.0), C13 = R(3.0 / 5.0), C23 = R(1.0 / 10.0);
  const R k1312 = R(13.0 / 12.0), k14 = R(1.0 / 4.0);
  R S0 = k1312 * sq(v[0] - R(2) * v[1] + v[2]) + k14 * sq(R(3) * v[0] - R(4) * v[1] + v[2]);
  R S1 = k1312 * sq(v[-1] - R(2) * v[0] + v[1]) + k14 * sq(v[-1] - v[1]);
  R S2 = k1312 * sq(v[-2] - R(2) * v[-1] + v[0]) + k14 * sq(v[-2] - R(4) * v[-1] + R(3) * v[0]);
  R q03 = R(1.0 / 3.0) * v[0] + R(5.0 / 6.0) * v[1] - R(1.0 / 6.0) * v[2];
  R q13 = R(-1.0 / 6.0) * v[-1] + R(5.0 / 6.0) * v[0] + R(1.0 / 3.0) * v[1];
  R q23 = R(1.0 / 3.0) * v[-2] - R(7.0 / 6.0) * v[-1] + R(11.0 / 6.0) * v[0];
  return weno_sum3(ep, C03, C13, C23, S0, S1, S2, q03, q13, q23);
}

// hh_weno5M: OCFD_Schemes_1.f90:31-52 (OCFD_weno5M, OCFD_Schemes.f90:30-53)
template <typename R>
__device__ __forceinline__ R weno5M(const R* v) {
  const R ep = R(1.0e-6), C03 = R(3.0 / 10.0), C13 = R(3.0 / 5.0), C23 = R(1.0 / 10.0);
  const R k1312 = R(13.0 / 12.0), k14 = R(1.0 / 4.0);
  R S0 = k1312 * sq(v[1] - R(2) * v[0] + v[-1]) + k14 * sq(R(3) * v[1] - R(4) * v[0] + v[-1]);
  R S1 = k1312 * sq(v[2] - R(2) * v[1] + v[0]) + k14 * sq(v[2] - v[0]);
  R S2 = k1312 * sq(v[3] - R(2) * v[2] + v[1]) + k14 * sq(v[3] - R(4) * v[2] + R(3) * v[1]);
  R q03 = R(1.0 / 3.0) * v[1] + R(5.0 / 6.0) * v[0] - R(1.0 / 6.0) * v[-1];
  R q13 = R(-1.0 / 6.0) * v[2] + R(5.0 / 6.0) * v[1] + R(1.0 / 3.0) * v[0];
  R q23 = R(1.0 / 3.0) * v[3] - R(7.0 / 6.0) * v[2] + R(11.0 / 6.0) * v[1];
  return weno_sum3(ep, C03, C13, C23, S0, S1, S2, q03, q13, q23);
}

// hh_weno5P_boundary / hh_weno5M_boundary: OCFD_Schemes_1.f90:266-325.
// del: 1 = DEL_LIFT, 2 = DEL_RIGHT
template <typename R>
__device__ __forceinline__ R weno5P_bnd(const R* v, int del) {
  const R ep = R(1.0e-6), C03 = R(3.0 / 10.0), C13 = R(3.0 / 5.0), C23 = R(1.0 / 10.0);
  const R k1312 = R(13.0 / 12.0), k14 = R(1.0 / 4.0);
  R a0 = R(0), q03 = R(0), a2 = R(0), q23 = R(0);
  if (del != 2) {
    R S0 = k1312 * sq(v[0] - R(2) * v[1] + v[2]) + k14 * sq(R(3) * v[0] - R(4) * v[1] + v[2]);
    a0 = C03 / sq(ep + S0);
    q03 = R(1.0 / 3.0) * v[0] + R(5.0 / 6.0) * v[1] - R(1.0 / 6.0) * v[2];
  }
  R S1 = k1312 * sq(v[-1] - R(2) * v[0] + v[1]) + k14 * sq(v[-1] - v[1]);
  R a1 = C13 / sq(ep + S1);
  R q13 = R(-1.0 / 6.0) * v[-1] + R(5.0 / 6.0) * v[0] + R(1.0 / 3.0) * v[1];
  if (del != 1) {
    R S2 = k1312 * sq(v[-2] - R(2) * v[-1] + v[0]) + k14 * sq(v[-2] - R(4) * v[-1] + R(3) * v[0]);
    a2 = C23 / sq(ep + S2);
    q23 = R(1.0 / 3.0) * v[-2] - R(7.0 / 6.0) * v[-1] + R(11.0 / 6.0) * v[0];
  }
  R am = a0 + a1 + a2;
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}

template <typename R>
__device__ __forceinline__ R weno5M_bnd(const R* v, int del) {
  const R ep = R(1.0e-6), C03 = R(3.0 / 10.0), C13 = R(3.0 / 5.0), C23 = R(1.0 / 10.0);
  const R k1312 = R(13.0 / 12.0), k14 = R(1.0 / 4.0);
  R a0 = R(0), q03 = R(0), a2 = R(0), q23 = R(0);
  if (del != 1) {
    R S0 = k1312 * sq(v[1] - R(2) * v[0] + v[-1]) + k14 * sq(R(3) * v[1] - R(4) * v[0] + v[-1]);
    a0 = C03 / sq(ep + S0);
    q03 = R(1.0 / 3.0) * v[1] + R(5.0 / 6.0) * v[0] - R(1.0 / 6.0) * v[-1];
  }
  R S1 = k1312 * sq(v[2] - R(2) * v[1] + v[0]) + k14 * sq(v[2] - v[0]);
  R a1 = C13 / sq(ep + S1);
  R q13 = R(-1.0 / 6.0) * v[2] + R(5.0 / 6.0) * v[1] + R(1.0 / 3.0) * v[0];
  if (del != 2) {
    R S2 = k1312 * sq(v[3] - R(2) * v[2] + v[1]) + k14 * sq(v[3] - R(4) * v[2] + R(3) * v[1]);
    a2 = C23 / sq(ep + S2);
    q23 = R(1.0 / 3.0) * v[3] - R(7.0 / 6.0) * v[2] + R(11.0 / 6.0) * v[1];
  }
  R am = a0 + a1 + a2;
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}

// WENO7 (WENO-JS, 4 candidate stencils): hh_weno7P OCFD_Schemes_1.f90:58-121
// (array form OCFD_weno7P, OCFD_Schemes.f90:59-124)
#define OCFD_W7_COEFFS                                                                                 \
  const R C0 = R(1.0 / 35.0), C1 = R(12.0 / 35.0), C2 = R(18.0 / 35.0), C3 = R(4.0 / 35.0);            \
  const R a11 = R(-2.0 / 6.0), a12 = R(9.0 / 6.0), a13 = R(-18.0 / 6.0), a14 = R(11.0 / 6.0);          \
  const R a21 = R(1.0 / 6.0), a23 = R(3.0 / 6.0), a24 = R(2.0 / 6.0);                                  \
  const R a31 = R(-2.0 / 6.0), a32 = R(-3.0 / 6.0), a34 = R(-1.0 / 6.0);                               \
  const R a41 = R(-11.0 / 6.0), a42 = R(18.0 / 6.0), a43 = R(-9.0 / 6.0), a44 = R(2.0 / 6.0);          \
  const R b12 = R(4), b13 = R(-5), b14 = R(2), b22 = R(-2), b41 = R(2), b42 = R(-5), b43 = R(4);        \
  const R c12 = R(3);                                                                                  \
  const R d12 = R(13.0 / 12.0), d13 = R(1043.0 / 960.0), d14 = R(1.0 / 12.0);                          \
  const R e11 = R(-3.0 / 12.0), e12 = R(13.0 / 12.0), e13 = R(-23.0 / 12.0), e14 = R(25.0 / 12.0);     \
  const R e21 = R(1.0 / 12.0), e22 = R(-5.0 / 12.0), e23 = R(13.0 / 12.0), e24 = R(3.0 / 12.0);        \
  const R e31 = R(-1.0 / 12.0), e32 = R(7.0 / 12.0), e33 = R(7.0 / 12.0), e34 = R(-1.0 / 12.0);        \
  const R e41 = R(3.0 / 12.0), e42 = R(13.0 / 12.0), e43 = R(-5.0 / 12.0), e44 = R(1.0 / 12.0);        \
  const R ep = R(1.0e-8)

template <typename R>
__device__ __forceinline__ R weno7P(const R* v) {
  OCFD_W7_COEFFS;
  R S10 = a11 * v[-3] + a12 * v[-2] + a13 * v[-1] + a14 * v[0];
  R S11 = a21 * v[-2] - v[-1] + a23 * v[0] + a24 * v[1];
  R S12 = a31 * v[-1] + a32 * v[0] + v[1] + a34 * v[2];
  R S13 = a41 * v[0] + a42 * v[1] + a43 * v[2] + a44 * v[3];
  R S20 = -v[-3] + b12 * v[-2] + b13 * v[-1] + b14 * v[0];
  R S21 = v[-1] + b22 * v[0] + v[1];
  R S22 = v[0] + b22 * v[1] + v[2];
  R S23 = b41 * v[0] + b42 * v[1] + b43 * v[2] - v[3];
  R S30 = -v[-3] + c12 * (v[-2] - v[-1]) + v[0];
  R S31 = -v[-2] + c12 * (v[-1] - v[0]) + v[1];
  R S32 = -v[-1] + c12 * (v[0] - v[1]) + v[2];
  R S33 = -v[0] + c12 * (v[1] - v[2]) + v[3];
  R S0 = S10 * S10 + d12 * S20 * S20 + d13 * S30 * S30 + d14 * S10 * S30;
  R S1 = S11 * S11 + d12 * S21 * S21 + d13 * S31 * S31 + d14 * S11 * S31;
  R S2 = S12 * S12 + d12 * S22 * S22 + d13 * S32 * S32 + d14 * S12 * S32;
  R S3 = S13 * S13 + d12 * S23 * S23 + d13 * S33 * S33 + d14 * S13 * S33;
  R q0 = e11 * v[-3] + e12 * v[-2] + e13 * v[-1] + e14 * v[0];
  R q1 = e21 * v[-2] + e22 * v[-1] + e23 * v[0] + e24 * v[1];
  R q2 = e31 * v[-1] + e32 * v[0] + e33 * v[1] + e34 * v[2];
  R q3 = e41 * v[0] + e42 * v[1] + e43 * v[2] + e44 * v[3];
  return weno_sum4(ep, C0, C1, C2, C3, S0, S1, S2, S3, q0, q1, q2, q3);
}

// hh_weno7M: OCFD_Schemes_1.f90:124-187 (OCFD_weno7M, OCFD_Schemes.f90:127-193)
template <typename R>
__device__ __forceinline__ R weno7M(const R* v) {
  OCFD_W7_COEFFS;
  R S10 = a11 * v[4] + a12 * v[3] + a13 * v[2] + a14 * v[1];
  R S11 = a21 * v[3] - v[2] + a23 * v[1] + a24 * v[0];
  R S12 = a31 * v[2] + a32 * v[1] + v[0] + a34 * v[-1];
  R S13 = a41 * v[1] + a42 * v[0] + a43 * v[-1] + a44 * v[-2];
  R S20 = -v[4] + b12 * v[3] + b13 * v[2] + b14 * v[1];
  R S21 = v[2] + b22 * v[1] + v[0];
  R S22 = v[1] + b22 * v[0] + v[-1];
  R S23 = b41 * v[1] + b42 * v[0] + b43 * v[-1] - v[-2];
  R S30 = -v[4] + c12 * (v[3] - v[2]) + v[1];
  R S31 = -v[3] + c12 * (v[2] - v[1]) + v[0];
  R S32 = -v[2] + c12 * (v[1] - v[0]) + v[-1];
  R S33 = -v[1] + c12 * (v[0] - v[-1]) + v[-2];
  R S0 = S10 * S10 + d12 * S20 * S20 + d13 * S30 * S30 + d14 * S10 * S30;
  R S1 = S11 * S11 + d12 * S21 * S21 + d13 * S31 * S31 + d14 * S11 * S31;
  R S2 = S12 * S12 + d12 * S22 * S22 + d13 * S32 * S32 + d14 * S12 * S32;
  R S3 = S13 * S13 + d12 * S23 * S23 + d13 * S33 * S33 + d14 * S13 * S33;
  R q0 = e11 * v[4] + e12 * v[3] + e13 * v[2] + e14 * v[1];
  R q1 = e21 * v[3] + e22 * v[2] + e23 * v[1] + e24 * v[0];
  R q2 = e31 * v[2] + e32 * v[1] + e33 * v[0] + e34 * v[-1];
  R q3 = e41 * v[1] + e42 * v[0] + e43 * v[-1] + e44 * v[-2];
  return weno_sum4(ep, C0, C1, C2, C3, S0, S1, S2, S3, q0, q1, q2, q3);
}

// ---- packed FP32 (production mixed path, sm_100): two reconstructions per
// instruction.  FFMA2 / FADD2 / FMUL2 apply one IEEE single-precision operation,
// rounded to nearest, to each of two lanes; the issue-bound FP32 face sweeps
// issue half the arithmetic instructions.  Lanes round as the scalar operations
// would, but the contraction into FMAs is fixed here rather than left to the
// compiler, so results can differ from the scalar form in the last bits; the
// batched and single-instance sweeps share this code and agree bit for bit.
#ifndef OCFD_F32X2
#define OCFD_F32X2 OCFD_FEWER_DIVS
#endif
struct F2 {
  float2 v;
};
__device__ __forceinline__ F2 f2(float a) { return F2{make_float2(a, a)}; }
__device__ __forceinline__ F2 f2(float a, float b) { return F2{make_float2(a, b)}; }
__device__ __forceinline__ F2 add2(F2 a, F2 b) { return F2{__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 mul2(F2 a, F2 b) { return F2{__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return F2{__ffma2_rn(a.v, b.v, c.v)}; }

// WENO7 of two windows at once: w[0..6] are the stencil values at offsets -3..3
// of weno7P.  Lane x: F+ (weno7P of the F+ window); lane y: F- -- weno7M(v) is
// weno7P of the mirrored window v'(k) = v(1 - k), term for term, so the caller
// puts F-(1 - k) in lane y of w[k + 3].  Same terms and order as weno7P; the
// weights' divisions are per lane.
__device__ __forceinline__ float2 weno7_x2(const F2* w) {
  const F2 C0 = f2(float(1.0 / 35.0)), C1 = f2(float(12.0 / 35.0)), C2 = f2(float(18.0 / 35.0)), C3 = f2(float(4.0 / 35.0));
  const F2 m1 = f2(-1.0f), b2 = f2(-2.0f), c3 = f2(3.0f);
  const F2 *v = w + 3;
  // S1k, S2k, S3k: weno7P's smoothness differences
  F2 S10 = fma2(f2(float(11.0 / 6.0)), v[0], fma2(f2(float(-18.0 / 6.0)), v[-1], fma2(f2(float(9.0 / 6.0)), v[-2], mul2(f2(float(-2.0 / 6.0)), v[-3]))));
  F2 S11 = fma2(f2(float(2.0 / 6.0)), v[1], fma2(f2(float(3.0 / 6.0)), v[0], fma2(m1, v[-1], mul2(f2(float(1.0 / 6.0)), v[-2]))));
  F2 S12 = fma2(f2(float(-1.0 / 6.0)), v[2], add2(fma2(f2(float(-3.0 / 6.0)), v[0], mul2(f2(float(-2.0 / 6.0)), v[-1])), v[1]));
  F2 S13 = fma2(f2(float(2.0 / 6.0)), v[3], fma2(f2(float(-9.0 / 6.0)), v[2], fma2(f2(float(18.0 / 6.0)), v[1], mul2(f2(float(-11.0 / 6.0)), v[0]))));
  F2 S20 = fma2(f2(2.0f), v[0], fma2(f2(-5.0f), v[-1], fma2(f2(4.0f), v[-2], mul2(m1, v[-3]))));
  F2 S21 = add2(fma2(b2, v[0], v[-1]), v[1]);
  F2 S22 = add2(fma2(b2, v[1], v[0]), v[2]);
  F2 S23 = fma2(m1, v[3], fma2(f2(4.0f), v[2], fma2(f2(-5.0f), v[1], mul2(f2(2.0f), v[0]))));
  F2 S30 = add2(fma2(c3, fma2(m1, v[-1], v[-2]), mul2(m1, v[-3])), v[0]);
  F2 S31 = add2(fma2(c3, fma2(m1, v[0], v[-1]), mul2(m1, v[-2])), v[1]);
  F2 S32 = add2(fma2(c3, fma2(m1, v[1], v[0]), mul2(m1, v[-1])), v[2]);
  F2 S33 = add2(fma2(c3, fma2(m1, v[2], v[1]), mul2(m1, v[0])), v[3]);
  const F2 d12 = f2(float(13.0 / 12.0)), d13 = f2(float(1043.0 / 960.0)), d14 = f2(float(1.0 / 12.0));
  auto beta = [&](F2 a, F2 b, F2 c) {
    return fma2(mul2(d14, a), c, fma2(mul2(d13, c), c, fma2(mul2(d12, b), b, mul2(a, a))));
  };
  const F2 S0 = beta(S10, S20, S30), S1 = beta(S11, S21, S31), S2 = beta(S12, S22, S32), S3 = beta(S13, S23, S33);
  // candidate values q0..q3
  const F2 q0 = fma2(f2(float(25.0 / 12.0)), v[0], fma2(f2(float(-23.0 / 12.0)), v[-1], fma2(f2(float(13.0 / 12.0)), v[-2], mul2(f2(float(-3.0 / 12.0)), v[-3]))));
  const F2 q1 = fma2(f2(float(3.0 / 12.0)), v[1], fma2(f2(float(13.0 / 12.0)), v[0], fma2(f2(float(-5.0 / 12.0)), v[-1], mul2(f2(float(1.0 / 12.0)), v[-2]))));
  const F2 q2 = fma2(f2(float(-1.0 / 12.0)), v[2], fma2(f2(float(7.0 / 12.0)), v[1], fma2(f2(float(7.0 / 12.0)), v[0], mul2(f2(float(-1.0 / 12.0)), v[-1]))));
  const F2 q3 = fma2(f2(float(1.0 / 12.0)), v[3], fma2(f2(float(-5.0 / 12.0)), v[2], fma2(f2(float(13.0 / 12.0)), v[1], mul2(f2(float(3.0 / 12.0)), v[0]))));
  // weights a_k = C_k / (ep + S_k)^2 (divisions per lane), normalised sum
  const F2 ep = f2(float(1.0e-8));
  F2 D0 = add2(ep, S0), D1 = add2(ep, S1), D2 = add2(ep, S2), D3 = add2(ep, S3);
  D0 = mul2(D0, D0);
  D1 = mul2(D1, D1);
  D2 = mul2(D2, D2);
  D3 = mul2(D3, D3);
  const F2 a0 = f2(C0.v.x / D0.v.x, C0.v.y / D0.v.y), a1 = f2(C1.v.x / D1.v.x, C1.v.y / D1.v.y);
  const F2 a2 = f2(C2.v.x / D2.v.x, C2.v.y / D2.v.y), a3 = f2(C3.v.x / D3.v.x, C3.v.y / D3.v.y);
  const F2 am = add2(add2(add2(a0, a1), a2), a3);
  const F2 num = fma2(a3, q3, fma2(a2, q2, fma2(a1, q1, mul2(a0, q0))));
  return make_float2(num.v.x / am.v.x, num.v.y / am.v.y);
}

// minmod2 / minmod4: OCFD_Schemes.f90:274-289
// minmod2 = 0.5*(sign(1,x1) + sign(1,x2)) * min(|x1|, |x2|): the sign factor is
// +-1 when the sign bits agree and 0 otherwise, so for finite arguments the
// value is min(|x1|,|x2|) with the sign of x1, or +0 -- the same bits, one
// comparison instead of three floating-point operations.
__device__ __forceinline__ bool sign_bits_differ(double a, double b) {
  return (__double_as_longlong(a) ^ __double_as_longlong(b)) < 0;
}
__device__ __forceinline__ bool sign_bits_differ(float a, float b) {
  return (__float_as_int(a) ^ __float_as_int(b)) < 0;
}
template <typename R>
__device__ __forceinline__ R minmod2(R x1, R x2) {
  return sign_bits_differ(x1, x2) ? R(0) : copysign(rmin(fabs(x1), fabs(x2)), x1);
}
// minmod4 = 0.5*(s1+s2) * |0.5*(s1+s3)| * |0.5*(s1+s4)| * min|x| (s = sign(1,x)):
// +0 when the sign bits of x1 and x2 differ; otherwise the product carries the
// sign of x1 and is min|x| when x3 and x4 share that sign bit, else a zero.
template <typename R>
__device__ __forceinline__ R minmod4(R x1, R x2, R x3, R x4) {
  if (sign_bits_differ(x1, x2)) return R(0);
  const R m = rmin(rmin(rmin(fabs(x1), fabs(x2)), fabs(x3)), fabs(x4));
  return copysign((sign_bits_differ(x1, x3) || sign_bits_differ(x1, x4)) ? R(0) : m, x1);
}

// OMP6 (optimized 6th-order monotonicity-preserving) coefficients,
// OCFD_Schemes_1.f90:203-209: m = 0.015, n = 0, kappa = 4, and ep = 1.e-10 as a
// single-precision literal widened to double.
struct Omp6C {
  static constexpr double m = 0.015, n = 0.0;
  static constexpr double a = 0.5 * (m + n), b = 0.5 * (m - n);
  static constexpr double a1 = a;
  static constexpr double a2 = 1.0 / 60.0 - b - 6.0 * a;
  static constexpr double a3 = -2.0 / 15.0 + 6.0 * b + 15.0 * a;
  static constexpr double a4 = 37.0 / 60.0 - 15.0 * b - 20.0 * a;
  static constexpr double a5 = 37.0 / 60.0 + 20.0 * b + 15.0 * a;
  static constexpr double a6 = -2.0 / 15.0 - 6.0 * a - 15.0 * b;
  static constexpr double a7 = 1.0 / 60.0 + a + 6.0 * b;
  static constexpr double a8 = -b;
  static constexpr double kappa = 4.0;
  static constexpr double ep = (double)1.e-10f;
};

// The limiter branch of OMP6 (taken rarely in smooth flow), kept out of line
// so that the common path stays small.  Written for the P orientation
// (vm2..v2 = v(-2)..v(2)); the M form passes the values mirrored about the face.
// vlc is the value subtracted in the lc term: v(-1) in hh_OMP6P
// (OCFD_Schemes_1.f90:219) but v(0) -- not the mirror v(2) -- in hh_OMP6M (:253).
template <typename R>
__device__ __forceinline__ R omp6_limit_inl(R mid_nf, R vm2, R vm1, R v0, R v1, R v2, R vlc) {
  const R kappa = R(Omp6C::kappa);
  R d1 = vm2 + v0 - R(2) * vm1;
  R d2 = vm1 + v1 - R(2) * v0;
  R d3 = v0 + v2 - R(2) * v1;
  R ul = v0 + kappa * (v0 - vm1);
  R md = R(0.5) * (v0 + v1) - R(0.5) * minmod4(R(4) * d2 - d3, R(4) * d3 - d2, d2, d3);
  R lc = v0 + R(0.5) * (v0 - vlc) + kappa * minmod4(R(4) * d1 - d2, R(4) * d2 - d1, d2, d1) / R(3);
  R fmin = rmax(rmin(rmin(v0, v1), md), rmin(rmin(v0, ul), lc));
  R fmax = rmin(rmax(rmax(v0, v1), md), rmax(rmax(v0, ul), lc));
  return mid_nf + minmod2(fmax - mid_nf, fmin - mid_nf);
}
template <typename R>
__device__ __noinline__ R omp6_limit(R mid_nf, R vm2, R vm1, R v0, R v1, R v2, R vlc) {
  return omp6_limit_inl(mid_nf, vm2, vm1, v0, v1, v2, vlc);
}

// hh_OMP6P: OCFD_Schemes_1.f90:195-226 (OCFD_OMP6P, OCFD_Schemes.f90:201-234)
template <typename R>
__device__ __forceinline__ R omp6P(const R* v) {
  R mid_nf = R(Omp6C::a1) * v[4] + R(Omp6C::a2) * v[3] + R(Omp6C::a3) * v[2] + R(Omp6C::a4) * v[1] +
             R(Omp6C::a5) * v[0] + R(Omp6C::a6) * v[-1] + R(Omp6C::a7) * v[-2] + R(Omp6C::a8) * v[-3];
  R mp = v[0] + minmod2((v[1] - v[0]), R(Omp6C::kappa) * (v[0] - v[-1]));
  if ((mid_nf - v[0]) * (mid_nf - mp) >= R(Omp6C::ep)) mid_nf = omp6_limit(mid_nf, v[-2], v[-1], v[0], v[1], v[2], v[-1]);
  return mid_nf;
}

// hh_OMP6M: OCFD_Schemes_1.f90:228-260 (OCFD_OMP6M, OCFD_Schemes.f90:236-271).
template <typename R>
__device__ __forceinline__ R omp6M(const R* v) {
  R mid_nf = R(Omp6C::a1) * v[-3] + R(Omp6C::a2) * v[-2] + R(Omp6C::a3) * v[-1] + R(Omp6C::a4) * v[0] +
             R(Omp6C::a5) * v[1] + R(Omp6C::a6) * v[2] + R(Omp6C::a7) * v[3] + R(Omp6C::a8) * v[4];
  R mp = v[1] + minmod2((v[0] - v[1]), R(Omp6C::kappa) * (v[1] - v[2]));
  if ((mid_nf - v[1]) * (mid_nf - mp) >= R(Omp6C::ep)) mid_nf = omp6_limit(mid_nf, v[3], v[2], v[1], v[0], v[-1], v[0]);
  return mid_nf;
}

// hh_UD7L_P / _M: OCFD_Schemes_1.f90:328-348 (OCFD_UD7L_P/M, OCFD_Schemes.f90:292-316)
template <typename R>
__device__ __forceinline__ R ud7lP(const R* U, const R* v) {
  return U[0] * v[-3] + U[1] * v[-2] + U[2] * v[-1] + U[3] * v[0] + U[4] * v[1] + U[5] * v[2] + U[6] * v[3] +
         U[7] * v[4];
}
template <typename R>
__device__ __forceinline__ R ud7lM(const R* U, const R* v) {
  return U[0] * v[4] + U[1] * v[3] + U[2] * v[2] + U[3] * v[1] + U[4] * v[0] + U[5] * v[-1] + U[6] * v[-2] +
         U[7] * v[-3];
}

// Scheme ids (OCFD_parameters.f90:23-27)
enum : int { SCH_WENO5 = 1, SCH_WENO7 = 2, SCH_OMP6 = 3, SCH_UD7L = 4, SCH_HYBRID = 10 };

// Interior scheme of OCFD2d_flux1 / flux_x1 (and the hybrid selection of
// OCFD_HybridP / hh_HybridP, OCFD_Schemes.f90:319-337, OCFD_Schemes_1.f90:351-365)
template <int SCHEME, typename R>
__device__ __forceinline__ R schemeP(const R* v, const R* U, int ihy) {
  if (SCHEME == SCH_OMP6) return omp6P(v);
  if (SCHEME == SCH_WENO7) return weno7P(v);
  if (SCHEME == SCH_WENO5) return weno5P(v);
  if (SCHEME == SCH_UD7L) return ud7lP(U, v);
  if (ihy == 1) return ud7lP(U, v);
  if (ihy == 2) return weno7P(v);
  return weno5P(v);
}
template <int SCHEME, typename R>
__device__ __forceinline__ R schemeM(const R* v, const R* U, int ihy) {
  if (SCHEME == SCH_OMP6) return omp6M(v);
  if (SCHEME == SCH_WENO7) return weno7M(v);
  if (SCHEME == SCH_WENO5) return weno5M(v);
  if (SCHEME == SCH_UD7L) return ud7lM(U, v);
  if (ihy == 1) return ud7lM(U, v);
  if (ihy == 2) return weno7M(v);
  return weno5M(v);
}

}  // namespace ocfd
