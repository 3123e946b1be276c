// ocfd_face.cuh -- face-flux kernels of the inviscous terms, one launch per
// direction: split -> (characteristic projection) -> reconstruction, written
// as numerical fluxes h(i+1/2) per face.  The flux difference, the Jacobian
// scaling and the rest of the stage happen in the update kernel
// (ocfd_update.cu), which reads these faces.
//
// Reference: du_inviscous (OCFD_inviscous.f90:53-203) with OCFD2d_flux1/2
// (:210-361) for the flux-vector form, du_inviscous_Character
// (OCFD_inviscous_character.f90:3-159) with flux_charteric / flux_x1 / flux_x2
// (:162-416) for the characteristic form.
//
// Tiling: a block owns NP pencils x TF consecutive faces along the sweep
// direction (NP*TF = 256 threads, one face per thread).  Phase 1 loads the
// TF+7 points of its stencil (coalesced along i for x, across i for y/z),
// computes the split fluxes once per point and stages them in shared memory.
// Phase 2 computes one face per thread from a register window of 8 points.
// For a periodic direction face 0 equals face n bit for bit, so only faces
// 1..n are computed: n faces for n points, no tile does extra work.
#pragma once
#include <cstring>

#include "ocfd_device.cuh"
#include "ocfd_kernels.h"
#include "ocfd_schemes.cuh"
#include "ocfd_tma.cuh"

namespace ocfd {

// Tile shapes (NP pencils x TF faces, one face per thread).  Variants 0 and 1
// (256 threads) are the choices of the batch autotuner -- variant 1 (TF = 32)
// wastes fewer threads on short pencils.  Variant 2 (128 threads) is the
// single-instance tile of the characteristic OMP6 sweeps: at 256^3 it measured
// 5-9% faster there than variant 0 (four blocks per SM overlap one another's
// barrier and load phases better than two), but slower on the hybrid and
// WENO7 sweeps, which keep variant 0.  Variants 3 (64 threads) and 4 (128
// threads, TF = 32 along y and z) measured slower.
template <int DIR, int V>
struct FaceTileV;
template <>
struct FaceTileV<0, 0> {
  static constexpr int NP = 4, TF = 64;
};
template <>
struct FaceTileV<0, 1> {
  static constexpr int NP = 8, TF = 32;
};
template <>
struct FaceTileV<1, 0> {
  static constexpr int NP = 16, TF = 16;
};
template <>
struct FaceTileV<1, 1> {
  static constexpr int NP = 8, TF = 32;
};
template <>
struct FaceTileV<2, 0> {
  static constexpr int NP = 16, TF = 16;
};
template <>
struct FaceTileV<2, 1> {
  static constexpr int NP = 8, TF = 32;
};
// 128-thread tiles (more, smaller blocks per SM)
template <>
struct FaceTileV<0, 2> {
  static constexpr int NP = 2, TF = 64;
};
template <>
struct FaceTileV<1, 2> {
  static constexpr int NP = 8, TF = 16;
};
template <>
struct FaceTileV<2, 2> {
  static constexpr int NP = 8, TF = 16;
};
template <>
struct FaceTileV<0, 3> {
  static constexpr int NP = 1, TF = 64;
};
template <>
struct FaceTileV<1, 3> {
  static constexpr int NP = 4, TF = 16;
};
template <>
struct FaceTileV<2, 3> {
  static constexpr int NP = 4, TF = 16;
};
template <>
struct FaceTileV<1, 4> {
  static constexpr int NP = 4, TF = 32;
};
template <>
struct FaceTileV<2, 4> {
  static constexpr int NP = 4, TF = 32;
};
// tile of a single-instance sweep
template <int DIR, bool CHAR, int SCHEME>
struct FaceTile : FaceTileV<DIR, (CHAR && SCHEME == SCH_OMP6) ? 2 : 0> {};

// Grid of one launch: (x, y, z) blocks for a face sweep of instance a.
template <int DIR, int NP, int TF, typename S>
__host__ __forceinline__ dim3 face_grid(const FaceArgs<S>& a) {
  const int nf = a.fend - a.fbeg + 1;
  if (DIR == 0) return dim3((nf + TF - 1) / TF, (a.g.ny + NP - 1) / NP, a.g.nz);
  return dim3((a.g.nx + NP - 1) / NP, (nf + TF - 1) / TF, DIR == 1 ? a.g.nz : a.g.ny);
}

// ---------------------------------------------------------------------------
// Flux-vector form, boundary-aware reconstruction of one face (OCFD2d_flux1).
template <int SCHEME, typename R>
__device__ __forceinline__ R nc_flux1_bnd(const R* v, const R* U, int g, int nn, int ihy, const Phys& ph, int dir) {
  const int bi0 = ph.bi[2 * dir], bi1 = ph.bi[2 * dir + 1], sb0 = ph.sb[2 * dir], sb1 = ph.sb[2 * dir + 1];
  const int Ka = ph.ka1, Kb = ph.kb1;
  const int ib = (bi0 == 0 || sb0 == -1) ? 0 : -Ka + 1;
  const int ie = (bi1 == 0 || sb1 == -1) ? nn : nn - Kb;
  R h = R(0);
  if (g >= ib && g <= ie) h = schemeP<SCHEME>(v, U, ihy);
  if (bi0 == 1 && g <= -Ka) {
    if (sb0 == 0) {
      if (g == 0)
        h = (R(2) * v[1] + R(5) * v[2] - v[3]) / R(6);
      else if (g == 1)
        h = (R(2) * v[0] + R(5) * v[1] - v[2]) / R(6);
      else if (g == 2)
        h = weno5P_bnd(v, 1);
      else
        h = weno5P(v);
    } else if (sb0 == 1) {
      h = weno5P(v);
    }
  }
  if (bi1 == 1 && g >= nn - Kb + 1) {
    if (sb1 == 0) {
      if (g == nn)
        h = (R(2) * v[-2] - R(7) * v[-1] + R(11) * v[0]) / R(6);
      else if (g == nn - 1)
        h = weno5P_bnd(v, 2);
      else
        h = weno5P(v);
    } else if (sb1 == 1) {
      h = weno5P(v);
    }
  }
  return h;
}

// OCFD2d_flux2 (OCFD_inviscous.f90:287-361)
template <int SCHEME, typename R>
__device__ __forceinline__ R nc_flux2_bnd(const R* v, const R* U, int g, int nn, int ihy, const Phys& ph, int dir) {
  const int bi0 = ph.bi[2 * dir], bi1 = ph.bi[2 * dir + 1], sb0 = ph.sb[2 * dir], sb1 = ph.sb[2 * dir + 1];
  const int Ka = ph.ka2, Kb = ph.kb2;
  const int ib = (bi0 == 0 || sb0 == -1) ? 0 : -Ka + 1;
  const int ie = (bi1 == 0 || sb1 == -1) ? nn : nn - Kb;
  R h = R(0);
  if (g >= ib && g <= ie) h = schemeM<SCHEME>(v, U, ihy);
  if (bi0 == 1 && g <= -Ka) {
    if (sb0 == 0) {
      if (g == 0)
        h = (R(2) * v[3] - R(7) * v[2] + R(11) * v[1]) / R(6);
      else if (g == 1)
        h = weno5M_bnd(v, 1);
      else
        h = weno5M(v);
    } else if (sb0 == 1) {
      h = weno5M(v);
    }
  }
  if (bi1 == 1 && g >= nn - Kb + 1) {
    if (sb1 == 0) {
      if (g == nn)
        h = (R(2) * v[0] + R(5) * v[-1] - v[-2]) / R(6);
      else if (g == nn - 1)
        h = (R(2) * v[1] + R(5) * v[0] - v[-1]) / R(6);
      else if (g == nn - 2)
        h = weno5M_bnd(v, 2);
      else
        h = weno5M(v);
    } else if (sb1 == 1) {
      h = weno5M(v);
    }
  }
  return h;
}

// Characteristic form: flux_x1 (OCFD_inviscous_character.f90:313-364) for a
// face that is not an interior face.
template <typename R>
__device__ __forceinline__ R ch_flux1_bnd(const R* ff, int g, int nn, const Phys& ph, int dir) {
  const int bi0 = ph.bi[2 * dir], bi1 = ph.bi[2 * dir + 1], sb0 = ph.sb[2 * dir], sb1 = ph.sb[2 * dir + 1];
  const int Ka = ph.ka1, Kb = ph.kb1;
  if (g <= -Ka && bi0 == 1 && sb0 != -1) {
    if (sb0 == 0) {
      if (g == 1) return (R(2) * ff[0] + R(5) * ff[1] - ff[2]) / R(6);
      if (g == 2) return weno5P_bnd(ff, 1);
      return weno5P(ff);
    } else if (sb0 == 1) {
      return weno5P(ff);
    }
  } else if (g > nn - Kb && bi1 == 1 && sb1 != -1) {
    if (sb1 == 0) {
      if (g == nn - 1) return weno5P_bnd(ff, 2);
      return weno5P(ff);
    } else if (sb1 == 1) {
      return weno5P(ff);
    }
  }
  return R(0);
}

// flux_x2 (OCFD_inviscous_character.f90:367-416), non-interior face
template <typename R>
__device__ __forceinline__ R ch_flux2_bnd(const R* ff, int g, int nn, const Phys& ph, int dir) {
  const int bi0 = ph.bi[2 * dir], bi1 = ph.bi[2 * dir + 1], sb0 = ph.sb[2 * dir], sb1 = ph.sb[2 * dir + 1];
  const int Ka = ph.ka2, Kb = ph.kb2;
  if (g <= -Ka && bi0 == 1 && sb0 != -1) {
    if (sb0 == 0) {
      if (g == 1) return weno5M_bnd(ff, 1);
      return weno5M(ff);
    } else if (sb0 == 1) {
      return weno5M(ff);
    }
  } else if (g > nn - Kb && bi1 == 1 && sb1 != -1) {
    if (sb1 == 0) {
      if (g == nn - 1) return (R(2) * ff[1] + R(5) * ff[0] - ff[-1]) / R(6);
      if (g == nn - 2) return weno5M_bnd(ff, 2);
      return weno5M(ff);
    } else if (sb1 == 1) {
      return weno5M(ff);
    }
  }
  return R(0);
}

// Stencil ranges of the projected values each scheme reads (set_parameters,
// OCFD_readpara.f90:288-315).  The hybrid's WENO5/WENO7 faces read subsets.
template <int SCHEME>
struct Stencil {
  static constexpr int PLO = -3, PHI = 4, MLO = -3, MHI = 4;
};
template <>
struct Stencil<SCH_WENO7> {
  static constexpr int PLO = -3, PHI = 3, MLO = -2, MHI = 4;
};
template <>
struct Stencil<SCH_WENO5> {
  static constexpr int PLO = -2, PHI = 2, MLO = -1, MHI = 3;
};

// Block-wide queue of OMP6 limiter evaluations (characteristic form,
// production build).  The monotonicity test of the ten characteristic
// components of a face is cheap; the limiter that a failed test calls is not,
// and the faces that need it are scattered, so a warp running it for one lane
// would idle the other 31.  Instead each flagged (face, component) is queued
// in shared memory -- its unlimited value and a tag (stencil window, component,
// side) -- and the whole block evaluates the queue, one entry per thread:
// eigenvector row, the five projected stencil values and the limiter.  The
// capacity is ten entries per face, so the queue never overflows.
// Shared-memory layout of a tile's points.  FP32 characteristic form, x and y
// sweeps: one record of 20 floats a point (F+, unused x3, F-, u, v, w, c, A1,
// A2, A3).  Otherwise one array per variable (10 split fluxes, +7 face-state
// arrays for the characteristic form).  Measured at 256^3 against the arrays:
// FP32 x 3% and y 2% faster, z 0.6% slower; FP64 records of 18 doubles (two
// 16-byte halves of F+ and F-) 17% slower on y and z, whose blocks then no
// longer fit four to an SM.
template <int DIR, bool CHAR, typename R>
constexpr int face_ps() {
  return (CHAR && sizeof(R) == 4 && DIR != 2) ? 20 : 1;
}

template <int NF>  // faces (threads) per block
struct LimQueue {
  static constexpr int CAP = 10 * NF;
  template <typename R>
  static constexpr size_t bytes() {
    return ((size_t)CAP * sizeof(R) + (CAP + 1) * sizeof(int) + 15) / 16 * 16;
  }
};

// Arithmetic with explicit rounding: never contracted or reassociated, so an
// expression written with these gives the same bits wherever it is inlined.
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float xfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double xrcp(double a) { return __drcp_rn(a); }
__device__ __forceinline__ float xrcp(float a) { return __frcp_rn(a); }

// Characteristic basis of one face, production build: the rows of L = S and
// R = S^-1 of flux_charteric (OCFD_inviscous_character.f90:216-248) applied
// without forming the matrices.  AXS: the sweep's metric row has a single
// non-zero component (box and 1-D grids), so n = s e_DIR with s its sign, and
// the general construction gives l = s e_y, m = e_z (DIR 0), l = -s e_x, m = e_z
// (DIR 1), l = -s e_x, m = -e_y (DIR 2): exact 0 and +-1 entries, whose terms
// the projections and the back projection skip.  Derived quantities (V2, un,
// ul, um, m) are recomputed where used, so that a face kept for the deferred
// limiter pass holds only u, v, w, c and the basis.
template <int DIR, bool AXS, typename R>
struct CharBasis {
  static constexpr int LI = DIR == 0 ? 1 : 0;  // AXS: the velocity component along l
  static constexpr int MI = DIR == 2 ? 1 : 2;  // and along m
  R u, v, w, c;
  R n1, n2, n3, l1, l2, l3;  // AXS: n1 holds s, the others are unused

  __device__ __forceinline__ void init(R u1, R v1, R w1, R c1, R a1, R a2, R a3) {
    u = u1;
    v = v1;
    w = w1;
    c = c1;
    if constexpr (AXS) {
      n1 = copysign(R(1), DIR == 0 ? a1 : (DIR == 1 ? a2 : a3));
    } else {
      const R rs = rsqrt(xfma(a3, a3, xfma(a2, a2, xmul(a1, a1))));
      n1 = xmul(a1, rs);
      n2 = xmul(a2, rs);
      n3 = xmul(a3, rs);
      if (fabs(n3) <= fabs(n2)) {
        const R rl = rsqrt(xfma(n2, n2, xmul(n1, n1)));
        l1 = -xmul(n2, rl);
        l2 = xmul(n1, rl);
        l3 = R(0);
      } else {
        const R rl = rsqrt(xfma(n3, n3, xmul(n1, n1)));
        l1 = -xmul(n3, rl);
        l3 = xmul(n1, rl);
        l2 = R(0);
      }
    }
  }
  __device__ __forceinline__ R vel(int q) const { return q == 0 ? u : (q == 1 ? v : w); }
  __device__ __forceinline__ R sl() const { return DIR == 0 ? n1 : -n1; }  // AXS: the non-zero entry of l
  // m = n x l
  __device__ __forceinline__ R m1() const { return xfma(n2, l3, -xmul(n3, l2)); }
  __device__ __forceinline__ R m2() const { return xfma(n3, l1, -xmul(n1, l3)); }
  __device__ __forceinline__ R m3() const { return xfma(n1, l2, -xmul(n2, l1)); }
  __device__ __forceinline__ R V2() const { return xmul(xfma(w, w, xfma(v, v, xmul(u, u))), R(0.5)); }
  __device__ __forceinline__ R un() const {
    return AXS ? xmul(n1, vel(DIR)) : xfma(w, n3, xfma(v, n2, xmul(u, n1)));
  }
  __device__ __forceinline__ R ul() const {
    return AXS ? xmul(sl(), vel(LI)) : xfma(w, l3, xfma(v, l2, xmul(u, l1)));
  }
  __device__ __forceinline__ R um() const {
    if constexpr (AXS) return DIR == 2 ? -v : w;
    return xfma(w, m3(), xfma(v, m2(), xmul(u, m1())));
  }
  // c = L f for one point (rows 0, 3, 4 through A = (V2,-u,-v,-w,1).f and
  // B = (un,-n).f: F0 - KK A and KK1 A +- X1 B)
  __device__ __forceinline__ void proj(R f0, R f1, R f2, R f3, R f4, R KK, R KK1, R X1, R V2_, R un_, R ul_,
                                       R um_, R* cc) const {
    const R A = xadd(xfma(-w, f3, xfma(-v, f2, xfma(-u, f1, xmul(V2_, f0)))), f4);
    cc[0] = xfma(-KK, A, f0);
    const R KA = xmul(KK1, A);
    if constexpr (AXS) {
      const R f[3] = {f1, f2, f3};
      const R B = xfma(-n1, f[DIR], xmul(un_, f0));
      cc[1] = xfma(-ul_, f0, xmul(sl(), f[LI]));
      cc[2] = xfma(-um_, f0, DIR == 2 ? -f[MI] : f[MI]);
      cc[3] = xfma(X1, B, KA);
      cc[4] = xfma(-X1, B, KA);
    } else {
      const R m1_ = m1(), m2_ = m2(), m3_ = m3();
      const R B = xfma(-n3, f3, xfma(-n2, f2, xfma(-n1, f1, xmul(un_, f0))));
      cc[1] = xfma(-ul_, f0, xfma(l3, f3, xfma(l2, f2, xmul(l1, f1))));
      cc[2] = xfma(-um_, f0, xfma(m3_, f3, xfma(m2_, f2, xmul(m1_, f1))));
      cc[3] = xfma(X1, B, KA);
      cc[4] = xfma(-X1, B, KA);
    }
  }
  // hh = R h0 (OCFD_inviscous_character.f90:284-288), H = V2 + c^2/(gamma-1)
  __device__ __forceinline__ void back(const R* h0, R* hh, R inv_gm1) const {
    const R V2_ = V2(), un_ = un(), ul_ = ul(), um_ = um();
    const R H = xfma(xmul(c, c), inv_gm1, V2_);
    hh[0] = xadd(xadd(h0[0], h0[3]), h0[4]);
    if constexpr (AXS) {
      const R cs = xmul(c, n1);
      R q[3];
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const R vk = vel(k);
        if (k == DIR)
          q[k] = xfma(xadd(vk, cs), h0[4], xfma(xadd(vk, -cs), h0[3], xmul(vk, h0[0])));
        else if (k == LI)
          q[k] = xfma(vk, h0[4], xfma(vk, h0[3], xfma(sl(), h0[1], xmul(vk, h0[0]))));
        else
          q[k] = xfma(vk, h0[4], xfma(vk, h0[3], xadd(xmul(vk, h0[0]), DIR == 2 ? -h0[2] : h0[2])));
      }
      hh[1] = q[0];
      hh[2] = q[1];
      hh[3] = q[2];
    } else {
      const R m1_ = m1(), m2_ = m2(), m3_ = m3();
      hh[1] = xfma(xfma(c, n1, u), h0[4],
                   xfma(xfma(-c, n1, u), h0[3], xfma(m1_, h0[2], xfma(l1, h0[1], xmul(u, h0[0])))));
      hh[2] = xfma(xfma(c, n2, v), h0[4],
                   xfma(xfma(-c, n2, v), h0[3], xfma(m2_, h0[2], xfma(l2, h0[1], xmul(v, h0[0])))));
      hh[3] = xfma(xfma(c, n3, w), h0[4],
                   xfma(xfma(-c, n3, w), h0[3], xfma(m3_, h0[2], xfma(l3, h0[1], xmul(w, h0[0])))));
    }
    hh[4] = xfma(xfma(c, un_, H), h0[4],
                 xfma(xfma(-c, un_, H), h0[3], xfma(um_, h0[2], xfma(ul_, h0[1], xmul(V2_, h0[0])))));
  }
};

// CharBasis::proj (c = L f) of two points at once, in the two lanes of packed
// FP32 operations; each lane performs proj's own explicitly rounded operations
// (a negation is a product with -1, which is exact), so both lanes give proj's
// bits.
template <int DIR, bool AXS>
__device__ __forceinline__ void char_proj2(const CharBasis<DIR, AXS, float>& b, const F2* f, float KK, float KK1,
                                           float X1, float V2_, float un_, float ul_, float um_, F2* cc) {
  const F2 A = add2(fma2(f2(-b.w), f[3], fma2(f2(-b.v), f[2], fma2(f2(-b.u), f[1], mul2(f2(V2_), f[0])))), f[4]);
  cc[0] = fma2(f2(-KK), A, f[0]);
  const F2 KA = mul2(f2(KK1), A);
  if constexpr (AXS) {
    constexpr int LI = CharBasis<DIR, AXS, float>::LI, MI = CharBasis<DIR, AXS, float>::MI;
    const F2 B = fma2(f2(-b.n1), f[1 + DIR], mul2(f2(un_), f[0]));
    cc[1] = fma2(f2(-ul_), f[0], mul2(f2(b.sl()), f[1 + LI]));
    cc[2] = fma2(f2(-um_), f[0], DIR == 2 ? mul2(f2(-1.0f), f[1 + MI]) : f[1 + MI]);
    cc[3] = fma2(f2(X1), B, KA);
    cc[4] = fma2(f2(-X1), B, KA);
  } else {
    const float m1_ = b.m1(), m2_ = b.m2(), m3_ = b.m3();
    const F2 B = fma2(f2(-b.n3), f[3], fma2(f2(-b.n2), f[2], fma2(f2(-b.n1), f[1], mul2(f2(un_), f[0]))));
    cc[1] = fma2(f2(-ul_), f[0], fma2(f2(b.l3), f[3], fma2(f2(b.l2), f[2], mul2(f2(b.l1), f[1]))));
    cc[2] = fma2(f2(-um_), f[0], fma2(f2(m3_), f[3], fma2(f2(m2_), f[2], mul2(f2(m1_), f[1]))));
    cc[3] = fma2(f2(X1), B, KA);
    cc[4] = fma2(f2(-X1), B, KA);
  }
}

// One queued limiter evaluation (OCFD_inviscous_character.f90:205-248 for the
// face state and row r of the left eigenvector matrix, :256-270 for the
// projection, OCFD_Schemes_1.f90:212-224 for the limiter): the face whose
// stencil window starts at wb, component r, F+ points -2..2 (window 1..5) or
// F- mirrored (window 6..2), unlimited value mid.  Written in explicitly
// rounded operations, so that every kernel that inlines it produces the same
// bits.
// Window element (var, stencil point q) at wb[var * VS + (var >= 5 ? GAP : 0) + q * QS].
// AXS: the axis-aligned basis of CharBasis (n = s e_DIR, l and m of exact 0 and
// +-1 entries).
template <typename R, int VS, int QS, int GAP, int DIR = 0, bool AXS = false>
__device__ __forceinline__ R lim_eval(const R* wb, int r, int minus, R mid, R gm1) {
  auto mean = [&](int var) {
    return xmul(xadd(wb[var * VS + GAP + 3 * QS], wb[var * VS + GAP + 4 * QS]), R(0.5));  // var >= 10
  };
  const R u1 = mean(10), v1 = mean(11), w1 = mean(12), c1 = mean(13);
  R n1, n2, n3, l1, l2, l3;
  if constexpr (AXS) {
    const R s = copysign(R(1), mean(14 + DIR));
    n1 = DIR == 0 ? s : R(0);
    n2 = DIR == 1 ? s : R(0);
    n3 = DIR == 2 ? s : R(0);
    l1 = DIR == 0 ? R(0) : -s;
    l2 = DIR == 0 ? s : R(0);
    l3 = R(0);
  } else {
    const R a1 = mean(14), a2 = mean(15), a3 = mean(16);
    const R rs = rsqrt(xfma(a3, a3, xfma(a2, a2, xmul(a1, a1))));
    n1 = xmul(a1, rs);
    n2 = xmul(a2, rs);
    n3 = xmul(a3, rs);
    if (fabs(n3) <= fabs(n2)) {
      const R rl = rsqrt(xfma(n2, n2, xmul(n1, n1)));
      l1 = -xmul(n2, rl);
      l2 = xmul(n1, rl);
      l3 = R(0);
    } else {
      const R rl = rsqrt(xfma(n3, n3, xmul(n1, n1)));
      l1 = -xmul(n3, rl);
      l3 = xmul(n1, rl);
      l2 = R(0);
    }
  }
  R c[5];
  if (r == 1) {
    c[0] = -xfma(w1, l3, xfma(v1, l2, xmul(u1, l1)));
    c[1] = l1;
    c[2] = l2;
    c[3] = l3;
    c[4] = R(0);
  } else if (r == 2) {
    const R m1 = xfma(n2, l3, -xmul(n3, l2)), m2 = xfma(n3, l1, -xmul(n1, l3)), m3 = xfma(n1, l2, -xmul(n2, l1));
    c[0] = -xfma(w1, m3, xfma(v1, m2, xmul(u1, m1)));
    c[1] = m1;
    c[2] = m2;
    c[3] = m3;
    c[4] = R(0);
  } else {
    const R rc = xrcp(c1);
    const R KK = xmul(gm1, xmul(rc, rc));
    const R V2 = xmul(xfma(w1, w1, xfma(v1, v1, xmul(u1, u1))), R(0.5));
    if (r == 0) {
      c[0] = xfma(-KK, V2, R(1));
      c[1] = xmul(KK, u1);
      c[2] = xmul(KK, v1);
      c[3] = xmul(KK, w1);
      c[4] = -KK;
    } else {
      const R KK1 = xmul(KK, R(0.5)), X1 = xmul(R(0.5), rc);
      const R sX = r == 3 ? X1 : -X1;
      const R un = xfma(w1, n3, xfma(v1, n2, xmul(u1, n1)));
      c[0] = xfma(sX, un, xmul(KK1, V2));
      c[1] = xfma(-sX, n1, -xmul(KK1, u1));
      c[2] = xfma(-sX, n2, -xmul(KK1, v1));
      c[3] = xfma(-sX, n3, -xmul(KK1, w1));
      c[4] = KK1;
    }
  }
  const R* w0 = wb + (minus ? 5 * VS + GAP + 6 * QS : QS);
  const int qs = minus ? -QS : QS;
  R x[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const R* wq = w0 + k * qs;
    x[k] = xfma(c[4], wq[4 * VS], xfma(c[3], wq[3 * VS], xfma(c[2], wq[2 * VS], xfma(c[1], wq[VS], xmul(c[0], wq[0])))));
  }
  const R s0 = x[2], s1 = x[3], vlc = minus ? x[3] : x[1];  // v(0), v(1), the lc reference
  const R kappa = R(Omp6C::kappa);
  const R d1 = xfma(R(-2), x[1], xadd(x[0], s0));
  const R d2 = xfma(R(-2), s0, xadd(x[1], s1));
  const R d3 = xfma(R(-2), s1, xadd(s0, x[4]));
  const R ul = xfma(kappa, xadd(s0, -x[1]), s0);
  const R md = xfma(R(-0.5), minmod4(xfma(R(4), d2, -d3), xfma(R(4), d3, -d2), d2, d3), xmul(R(0.5), xadd(s0, s1)));
  const R lc = xfma(R(Omp6C::kappa / 3.0), minmod4(xfma(R(4), d1, -d2), xfma(R(4), d2, -d1), d2, d1),
                    xfma(R(0.5), xadd(s0, -vlc), s0));
  const R fmin = rmax(rmin(rmin(s0, s1), md), rmin(rmin(s0, ul), lc));
  const R fmax = rmin(rmax(rmax(s0, s1), md), rmax(rmax(s0, ul), lc));
  return xadd(mid, minmod2(xadd(fmax, -mid), xadd(fmin, -mid)));
}

// ---------------------------------------------------------------------------
// ALLIN: every face of the launch is an interior face (periodic direction), so
// the boundary-closure paths are compiled out.
// The body of one block; (bx, by, bz) are its block coordinates within the
// instance's own launch grid.
// TMA: the eight input arrays were staged in shared memory by the caller
// (tile: TmaBox slots of d, u, v, w, T, A1, A2, A3; toff: offset of the first
// stencil point / pencil in the tile's innermost dimension).
// AXS (production build, ALLIN sweeps): the sweep's metric row has a single
// non-zero component (axis_aligned); the splitting and the characteristic
// basis use the axis-aligned forms.
template <int DIR, bool CHAR, int SCHEME, bool ALLIN, int NP, int TF, typename R, typename S, bool TMA = false,
          bool AXS = false>
__device__ __forceinline__ void face_body(const FaceArgs<S>& a, const int bx, const int by, const int bz, R* sm,
                                          const S* tile = nullptr, int toff = 0, R* qbase = nullptr) {
  constexpr int LT = TF + 7;
  // shared memory (face_ps).  Records (PS > 1): F+ and F- each start on a
  // 16-byte boundary (GAP unused values after F+), so that four components of
  // a stencil point come in one 16-byte load; the 80-byte record stride keeps
  // a warp's 16-byte accesses free of bank conflicts.
  constexpr int PS = face_ps<DIR, CHAR, R>();
  constexpr int GAP = PS > 1 ? 3 : 0;
  constexpr int VS = PS > 1 ? 1 : NP * LT;  // stride between variables
  auto PI = [](int l, int p) -> int { return DIR == 0 ? p * LT + l : l * NP + p; };  // point of the tile
  auto SI = [&](int var, int l, int p) -> int { return var * VS + (var >= 5 ? GAP : 0) + PI(l, p) * PS; };

  const Grid& G = a.g;
  const Phys& ph = a.ph;
  const int nn = G.len(DIR);
  int g0, pbase;
  if (DIR == 0) {
    g0 = a.fbeg + bx * TF;
    pbase = by * NP;  // NP consecutive j of plane k = bz + 1
  } else {
    g0 = a.fbeg + by * TF;
    pbase = bx * NP;
  }
  // pencil p -> (i,j,k) with the along-direction index left at 0
  auto pencil = [&](int p, int& i, int& j, int& k) -> bool {
    if (DIR == 0) {
      i = 0;
      j = pbase + p + 1;
      k = bz + 1;
      return j <= G.ny;
    } else if (DIR == 1) {
      i = pbase + p + 1;
      j = 0;
      k = bz + 1;
      return i <= G.nx;
    } else {
      i = pbase + p + 1;
      j = bz + 1;
      k = 0;
      return i <= G.nx;
    }
  };
  const long long hs = G.hstride(DIR);
  const R gam = R(ph.gamma), ma = R(ph.ma);
  // deferred OMP6 limiter (characteristic form, production build): queue after
  // the staged point records -- CAP unlimited values, CAP tags (window offset * 16 +
  // component * 2 + side), the entry count
  constexpr bool DEFER = CHAR && SCHEME == SCH_OMP6 && OCFD_FEWER_DIVS;
  constexpr int JC = LimQueue<NP * TF>::CAP;  // one face per thread: blockDim.x == NP * TF
  // (qbase: the caller's queue, which may share memory with the staged input
  // tile -- dead after phase 1; the entry count lies past that tile)
  R* const jv = qbase ? qbase : sm + (PS > 1 ? PS : 17) * NP * LT;
  int* const jtag = reinterpret_cast<int*>(jv + JC);
  int* const jn = jtag + JC;
  if (DEFER && threadIdx.x == 0) *jn = 0;

  // ---- phase 1: split fluxes of the tile's points into shared memory
  for (int t = threadIdx.x; t < NP * LT; t += blockDim.x) {
    int l, p;
    if (DIR == 0) {
      l = t % LT;
      p = t / LT;
    } else {
      p = t % NP;
      l = t / NP;
    }
    int i, j, k;
    bool ok = pencil(p, i, j, k);
    const int gl = g0 - 3 + l;  // point index along DIR
    ok = ok && gl <= nn + LAP;
    R d = R(1), u = R(1), v = R(1), w = R(1), T = R(1), A1 = R(1), A2 = R(1), A3 = R(1);
    if (ok && TMA) {
      using B = TmaBox<DIR, NP, TF, S>;
      const int e = DIR == 0 ? p * B::BX + l + toff : l * B::BX + p + toff;
      d = R(tile[e]);
      if constexpr (sizeof(S) == 4) {  // slots 1-4: the interleaved u,v,w,T tile
        const float4 t = reinterpret_cast<const float4*>(tile + B::SLOT_ELEMS)[e];
        u = R(t.x);
        v = R(t.y);
        w = R(t.z);
        T = R(t.w);
      } else {
        u = R(tile[B::SLOT_ELEMS + e]);
        v = R(tile[2 * B::SLOT_ELEMS + e]);
        w = R(tile[3 * B::SLOT_ELEMS + e]);
        T = R(tile[4 * B::SLOT_ELEMS + e]);
      }
      const int m0 = 13 + 3 * DIR;
      if constexpr (AXS) {
        A1 = DIR == 0 ? R(tile[5 * B::SLOT_ELEMS + e]) : R(0);
        A2 = DIR == 1 ? R(tile[6 * B::SLOT_ELEMS + e]) : R(0);
        A3 = DIR == 2 ? R(tile[7 * B::SLOT_ELEMS + e]) : R(0);
      } else {
        A1 = ((ph.metzero >> m0) & 1u) ? R(0) : R(tile[5 * B::SLOT_ELEMS + e]);
        A2 = ((ph.metzero >> (m0 + 1)) & 1u) ? R(0) : R(tile[6 * B::SLOT_ELEMS + e]);
        A3 = ((ph.metzero >> (m0 + 2)) & 1u) ? R(0) : R(tile[7 * B::SLOT_ELEMS + e]);
      }
    } else if (ok) {
      long long h = G.ih(i, j, k) + (long long)gl * hs;
      d = R(__ldg(a.d + h));
      if constexpr (sizeof(S) == 4) {  // FP32 copies: u,v,w,T interleaved
        const float4 t = __ldg(reinterpret_cast<const float4*>(a.q4) + h);
        u = R(t.x);
        v = R(t.y);
        w = R(t.z);
        T = R(t.w);
      } else {
        u = R(__ldg(a.u + h));
        v = R(__ldg(a.v + h));
        w = R(__ldg(a.w + h));
        T = R(__ldg(a.T + h));
      }
      if constexpr (AXS) {
        A1 = DIR == 0 ? R(__ldg(a.A1 + h)) : R(0);
        A2 = DIR == 1 ? R(__ldg(a.A2 + h)) : R(0);
        A3 = DIR == 2 ? R(__ldg(a.A3 + h)) : R(0);
      } else {
        A1 = met_at<R>(ph, 13 + 3 * DIR, a.A1, h);
        A2 = met_at<R>(ph, 14 + 3 * DIR, a.A2, h);
        A3 = met_at<R>(ph, 15 + 3 * DIR, a.A3, h);
      }
    }
#if OCFD_FEWER_DIVS
    const R c = sqrt(T) * R(ph.inv_ma);
#else
    const R c = sqrt(T) / ma;  // cc: OCFD_inviscous.f90:67
#endif
    R fp[5], fm[5];
    if constexpr (AXS) {
      const R Ad = DIR == 0 ? A1 : (DIR == 1 ? A2 : A3);
      if (a.split == 1)
        split_sw_axis<DIR>(ph, gam, c, d, u, v, w, Ad, fp, fm);
      else
        split_llf_axis<DIR>(ph, gam, c, d, u, v, w, Ad, fp, fm);
    } else {
      if (a.split == 1)
        split_sw(ph, gam, c, d, u, v, w, A1, A2, A3, fp, fm);
      else
        split_llf(ph, gam, c, d, u, v, w, A1, A2, A3, fp, fm);
    }
    if constexpr (PS > 1) {
      // the point's record in 16-byte stores (the unused slots get zeros)
      float4* r4 = reinterpret_cast<float4*>(sm + PI(l, p) * PS);
      r4[0] = make_float4(fp[0], fp[1], fp[2], fp[3]);
      r4[1] = make_float4(fp[4], 0.f, 0.f, 0.f);
      r4[2] = make_float4(fm[0], fm[1], fm[2], fm[3]);
      r4[3] = make_float4(fm[4], u, v, w);
      r4[4] = make_float4(c, A1, A2, A3);
    } else {
#pragma unroll
      for (int m = 0; m < 5; m++) {
        sm[SI(m, l, p)] = fp[m];
        sm[SI(5 + m, l, p)] = fm[m];
      }
      if (CHAR) {
        sm[SI(10, l, p)] = u;
        sm[SI(11, l, p)] = v;
        sm[SI(12, l, p)] = w;
        sm[SI(13, l, p)] = c;
        // axis-aligned sweeps read only the direction's metric component
        if (!AXS || DIR == 0) sm[SI(14, l, p)] = A1;
        if (!AXS || DIR == 1) sm[SI(15, l, p)] = A2;
        if (!AXS || DIR == 2) sm[SI(16, l, p)] = A3;
      }
    }
  }
  __syncthreads();

  // ---- phase 2: one face per thread
  R U[8];
#pragma unroll
  for (int q = 0; q < 8; q++) U[q] = R(ph.ud7l[q]);
  R* out = reinterpret_cast<R*>(a.hh);
  // window element (var, stencil offset s) of this thread's face at
  // wb[var*VS + (var >= 5 ? GAP : 0) + (s+3)*QS]
  constexpr int QS = (DIR == 0 ? 1 : NP) * PS;
  // state of a face whose limiter evaluations are queued: the F+ / F- parts of
  // the characteristic flux, the flags of the queued components and their first
  // queue entry, the face's output offset and the basis of the back projection
  R dP[5], dM[5];
  unsigned dfl = 0;
  int djb = 0;
  bool dpend = false;
  long long dfo = 0;
  CharBasis<DIR, AXS, R> dcb{};

  for (int t = threadIdx.x; t < NP * TF; t += blockDim.x) {
    int f, p;
    if (DIR == 0) {
      f = t % TF;
      p = t / TF;
    } else {
      p = t % NP;
      f = t / NP;
    }
    int i, j, k;
    if (!pencil(p, i, j, k)) continue;
    const int g = g0 + f;
    if (g > a.fend) continue;
    const R* wb = sm + PI(f, p) * PS;
    auto W = [&](int var, int q) -> R { return wb[var * VS + (var >= 5 ? GAP : 0) + q * QS]; };
    // components vb..vb+3 (vb = 0: F+, 5: F-) of stencil point q
    auto W4 = [&](int vb, int q, R* o) {
      if constexpr (PS > 1) {
        const float4 t = *reinterpret_cast<const float4*>(wb + vb + (vb >= 5 ? GAP : 0) + q * QS);
        o[0] = t.x;
        o[1] = t.y;
        o[2] = t.z;
        o[3] = t.w;
      } else {
#pragma unroll
        for (int v = 0; v < 4; v++) o[v] = W(vb + v, q);
      }
    };
    int ii = DIR == 0 ? g : i, jj = DIR == 1 ? g : j, kk = DIR == 2 ? g : k;
    const long long fo = G.face(DIR, g, ii, jj, kk);
    int ihy = 0;
    if (SCHEME == SCH_HYBRID) {
      // OCFD_inviscous.f90:76-81: Rhb0 = max(Rhybrid(g), Rhybrid(g+1))
      long long h = G.ih(i, j, k) + (long long)g * hs;
      double r0 = __ldg(a.rh + h), r1 = __ldg(a.rh + h + hs);
      ihy = hybrid_index(rmax(r0, r1), ph.hyb1, ph.hyb2);
    }
    const int bi0 = ph.bi[2 * DIR], bi1 = ph.bi[2 * DIR + 1], sb0 = ph.sb[2 * DIR], sb1 = ph.sb[2 * DIR + 1];

    if (!CHAR) {
      // ---- flux-vector form: h1 (F+) and h2 (F-) per variable
      const int ib1 = (bi0 == 0 || sb0 == -1) ? 0 : -ph.ka1 + 1, ie1 = (bi1 == 0 || sb1 == -1) ? nn : nn - ph.kb1;
      const int ib2 = (bi0 == 0 || sb0 == -1) ? 0 : -ph.ka2 + 1, ie2 = (bi1 == 0 || sb1 == -1) ? nn : nn - ph.kb2;
      const bool inner = ALLIN || (g >= ib1 && g <= ie1 && g >= ib2 && g <= ie2);
      if (inner) {
#pragma unroll 1
        for (int m = 0; m < 5; m++) {
          R h1, h2;
          if constexpr (OCFD_F32X2 && sizeof(R) == 4 && SCHEME == SCH_WENO7) {
            // production FP32: F+ and F- by one packed evaluation -- the F+
            // window in lane x, the F- window mirrored (offset k holds F-(1-k))
            // in lane y
            F2 w2[7];
#pragma unroll
            for (int q = 0; q < 7; q++) w2[q] = f2(float(W(m, q)), float(W(5 + m, 7 - q)));
            const float2 h = weno7_x2(w2);
            h1 = h.x;
            h2 = h.y;
          } else {
            R wv[8];
#pragma unroll
            for (int q = 0; q < 8; q++) wv[q] = W(m, q);
            h1 = schemeP<SCHEME>(wv + 3, U, ihy);
#pragma unroll
            for (int q = 0; q < 8; q++) wv[q] = W(5 + m, q);
            h2 = schemeM<SCHEME>(wv + 3, U, ihy);
          }
          if (OCFD_FV_SUMMED) {
            out[hf_at(fo, a.fs, m)] = h1 + h2;
          } else {
            out[fo + (long long)m * a.fs] = h1;
            out[fo + (long long)(5 + m) * a.fs] = h2;
          }
        }
      } else if (!ALLIN) {
#pragma unroll 1
        for (int m = 0; m < 5; m++) {
          R wv[8];
#pragma unroll
          for (int q = 0; q < 8; q++) wv[q] = W(m, q);
          const R h1 = nc_flux1_bnd<SCHEME>(wv + 3, U, g, nn, ihy, ph, DIR);
#pragma unroll
          for (int q = 0; q < 8; q++) wv[q] = W(5 + m, q);
          const R h2 = nc_flux2_bnd<SCHEME>(wv + 3, U, g, nn, ihy, ph, DIR);
          if (OCFD_FV_SUMMED) {
            out[hf_at(fo, a.fs, m)] = h1 + h2;
          } else {
            out[fo + (long long)m * a.fs] = h1;
            out[fo + (long long)(5 + m) * a.fs] = h2;
          }
        }
      }
      continue;
    }

    // ---- characteristic form (flux_charteric)
    const int ia = (bi0 == 0 || sb0 != 0) ? 0 : 1;
    const int ibf = (bi1 == 0 || sb1 != 0) ? nn : nn - 1;
    R hh[5];
    if (!ALLIN && (g < ia || g > ibf)) {
      // non-reflecting boundary faces, OCFD_inviscous_character.f90:295-309
#pragma unroll 1
      for (int m = 0; m < 5; m++) {
        if (g == 0)
          hh[m] = (R(2) * W(m, 4) + R(5) * W(m, 5) - W(m, 6) + R(2) * W(5 + m, 6) - R(7) * W(5 + m, 5) +
                   R(11) * W(5 + m, 4)) / R(6);
        else
          hh[m] = (R(2) * W(m, 1) - R(7) * W(m, 2) + R(11) * W(m, 3) + R(2) * W(5 + m, 3) + R(5) * W(5 + m, 2) -
                   W(5 + m, 1)) / R(6);
      }
    } else {
      const bool inner1 =
          ALLIN || ((bi0 == 0 || g > -ph.ka1 || sb0 == -1) && (bi1 == 0 || g <= nn - ph.kb1 || sb1 == -1));
      const bool inner2 =
          ALLIN || ((bi0 == 0 || g > -ph.ka2 || sb0 == -1) && (bi1 == 0 || g <= nn - ph.kb2 || sb1 == -1));
      const bool inner = inner1 && inner2;
      if (ihy == 1) {
        // linear hybrid face: no characteristic projection (:192-194, :281-282)
#pragma unroll 1
        for (int m = 0; m < 5; m++) {
          R wv[8];
#pragma unroll
          for (int q = 0; q < 8; q++) wv[q] = W(m, q);
          const R h1 = (ALLIN || inner) ? schemeP<SCHEME>(wv + 3, U, ihy) : ch_flux1_bnd(wv + 3, g, nn, ph, DIR);
#pragma unroll
          for (int q = 0; q < 8; q++) wv[q] = W(5 + m, q);
          const R h2 = (ALLIN || inner) ? schemeM<SCHEME>(wv + 3, U, ihy) : ch_flux2_bnd(wv + 3, g, nn, ph, DIR);
          hh[m] = h1 + h2;
        }
      } else {
        // face state: arithmetic means of the two neighbours (:205-211)
        auto mean = [&](int var) -> R { return xmul(xadd(W(var, 3), W(var, 4)), R(0.5)); };
        const R u1 = mean(10);
        const R v1 = mean(11);
        const R w1 = mean(12);
        const R c1 = mean(13);
        const R a1 = (AXS && DIR != 0) ? R(0) : mean(14);
        const R a2 = (AXS && DIR != 1) ? R(0) : mean(15);
        const R a3 = (AXS && DIR != 2) ? R(0) : mean(16);
        // orthonormal basis (n,l,m) and L = S, R = S^-1 (:216-248)
#if OCFD_FEWER_DIVS
        CharBasis<DIR, AXS, R> cb;
        cb.init(u1, v1, w1, c1, a1, a2, a3);
        const R V2 = cb.V2(), un = cb.un(), ul = cb.ul(), um = cb.um();
        const R rc = R(1) / c1;
        const R KK = xmul(xadd(R(ph.gamma), R(-1)), xmul(rc, rc));
        const R KK1 = xmul(KK, R(0.5));
        const R X1 = xmul(R(0.5), rc);
        // rows of L through two shared dot products: with A = (V2,-u,-v,-w,1).F and
        // B = (un,-n1,-n2,-n3,0).F, rows 0, 3, 4 are F0 - KK A and KK1 A +- X1 B
        auto proj5v = [&](R f0, R f1, R f2, R f3, R f4, R* c) {
          cb.proj(f0, f1, f2, f3, f4, KK, KK1, X1, V2, un, ul, um, c);
        };
        auto proj5 = [&](int vb, int q, R* c) {
          R f4[4];
          W4(vb, q, f4);
          proj5v(f4[0], f4[1], f4[2], f4[3], W(vb + 4, q), c);
        };
#else
        R ss = sqrt(a1 * a1 + a2 * a2 + a3 * a3);
        const R n1 = a1 / ss, n2 = a2 / ss, n3 = a3 / ss;
        R l1, l2, l3;
        if (fabs(n3) <= fabs(n2)) {
          ss = sqrt(n1 * n1 + n2 * n2);
          l1 = -n2 / ss;
          l2 = n1 / ss;
          l3 = R(0);
        } else {
          ss = sqrt(n1 * n1 + n3 * n3);
          l1 = -n3 / ss;
          l3 = n1 / ss;
          l2 = R(0);
        }
        const R m1 = n2 * l3 - n3 * l2, m2 = n3 * l1 - n1 * l3, m3 = n1 * l2 - n2 * l1;
        const R un = u1 * n1 + v1 * n2 + w1 * n3;
        const R ul = u1 * l1 + v1 * l2 + w1 * l3;
        const R um = u1 * m1 + v1 * m2 + w1 * m3;
        const R V2 = (u1 * u1 + v1 * v1 + w1 * w1) * R(0.5);
        const R KK = (R(ph.gamma) - R(1)) / (c1 * c1);
        const R KK1 = KK * R(0.5);
        const R X1 = R(1) / (R(2) * c1);
        const R L[5][5] = {{R(1) - KK * V2, KK * u1, KK * v1, KK * w1, -KK},
                           {-ul, l1, l2, l3, R(0)},
                           {-um, m1, m2, m3, R(0)},
                           {KK1 * V2 + X1 * un, -X1 * n1 - KK1 * u1, -X1 * n2 - KK1 * v1, -X1 * n3 - KK1 * w1, KK1},
                           {KK1 * V2 - X1 * un, X1 * n1 - KK1 * u1, X1 * n2 - KK1 * v1, X1 * n3 - KK1 * w1, KK1}};
        // projection of one stencil point (:256-260 / :266-270), row r
        auto proj_row = [&](int r, int vb, int q) -> R {
          const R f0 = W(vb, q), f1 = W(vb + 1, q), f2 = W(vb + 2, q), f3 = W(vb + 3, q);
          if (r == 1 || r == 2) return L[r][0] * f0 + L[r][1] * f1 + L[r][2] * f2 + L[r][3] * f3;
          return L[r][0] * f0 + L[r][1] * f1 + L[r][2] * f2 + L[r][3] * f3 + L[r][4] * W(vb + 4, q);
        };
#endif
        R h0[5];
        if (SCHEME == SCH_OMP6 && inner) {
          // OMP6, interior face: the linear part of hh_OMP6P/M (OCFD_Schemes_1.f90:211,244) is
          // accumulated while the stencil is projected point by point, in the
          // reference's term order; only v(-1..1) (F+) / v(0..2) (F-) are kept for
          // the monotonicity test, the two outer values are recomputed in the
          // (rare) limiter branch.
          const R oa[8] = {R(Omp6C::a1), R(Omp6C::a2), R(Omp6C::a3), R(Omp6C::a4),
                           R(Omp6C::a5), R(Omp6C::a6), R(Omp6C::a7), R(Omp6C::a8)};
          const R kap = R(Omp6C::kappa), ep = R(Omp6C::ep);
#if OCFD_FEWER_DIVS
          // production build: the projection is linear, so the linear part is
          // L (sum_s a_s F(s)) -- the stencil sum taken in physical space and
          // projected once -- and only the three points of the monotonicity test
          // are projected (results move by rounding only).  Components that fail
          // the test are queued for the block-wide limiter pass below.
          if constexpr (OCFD_F32X2 && sizeof(R) == 4 && PS == 1) {
            // production FP32, sweeps without point records (z): the F+ and F-
            // blocks below in the two lanes of packed operations -- step s takes
            // F+(7 - s) and F-(s), both with oa[s]; every lane operation is the
            // blocks' own explicitly rounded operation, so the results are the
            // same bits (z sweep at 256^3: 1.73 -> 1.65 ms per step).  The x and y
            // sweeps (point records) keep the blocks one after the other: with
            // both sides live they spill at 64 registers and measured slower
            // (1.74 -> 1.92 ms), and at 85 registers slower still.
            const F2 m1 = f2(-1.0f), kap2 = f2(float(kap));
            // X4: the middle test point pb of both sides; MP: the test's bound
            // mp = pb + minmod2(t1, kap t2) with t1 = pc - pb, t2 = pb - pa (F+)
            // and t1 = pa - pb, t2 = pb - pc (F-), formed as the points arrive
            F2 G2[5], X4[5], MP[5];
#pragma unroll
            for (int s = 0; s <= 7; s++) {
              R fp[5], fm[5];
              if constexpr (PS > 1) {
                W4(0, 7 - s, fp);
                fp[4] = W(4, 7 - s);
                W4(5, s, fm);
                fm[4] = W(9, s);
              } else {
#pragma unroll
                for (int v = 0; v < 5; v++) {
                  fp[v] = W(v, 7 - s);
                  fm[v] = W(5 + v, s);
                }
              }
              F2 f[5];
#pragma unroll
              for (int v = 0; v < 5; v++) f[v] = f2(float(fp[v]), float(fm[v]));
              const F2 c = f2(float(oa[s]));
#pragma unroll
              for (int v = 0; v < 5; v++) G2[v] = s == 0 ? mul2(c, f[v]) : fma2(c, f[v], G2[v]);
              // the points of the monotonicity test: step 3 holds F+ point 4 (pc)
              // and F- point 3 (pa), step 4 pb of both, step 5 F+ point 2 (pa)
              // and F- point 5 (pc)
              if (s == 3) char_proj2(cb, f, KK, KK1, X1, V2, un, ul, um, MP);  // held in MP until step 4
              if (s == 4) {
                char_proj2(cb, f, KK, KK1, X1, V2, un, ul, um, X4);
#pragma unroll
                for (int r = 0; r < 5; r++) MP[r] = fma2(m1, X4[r], MP[r]);  // t1
              }
              if (s == 5) {
                F2 X5[5];
                char_proj2(cb, f, KK, KK1, X1, V2, un, ul, um, X5);
#pragma unroll
                for (int r = 0; r < 5; r++) {
                  const F2 t2 = mul2(kap2, fma2(m1, X5[r], X4[r]));
                  MP[r] = add2(X4[r], f2(minmod2(MP[r].v.x, t2.v.x), minmod2(MP[r].v.y, t2.v.y)));
                }
              }
            }
            F2 D[5];
            char_proj2(cb, G2, KK, KK1, X1, V2, un, ul, um, D);
#pragma unroll
            for (int r = 0; r < 5; r++) {
              const F2 tt = mul2(fma2(m1, X4[r], D[r]), fma2(m1, MP[r], D[r]));
              dfl |= (tt.v.x >= float(ep) ? 1u : 0u) << r;
              dfl |= (tt.v.y >= float(ep) ? 1u : 0u) << (5 + r);
              dP[r] = D[r].v.x;
              dM[r] = D[r].v.y;
            }
          } else {
          {
            // per component: oa[0] F(7) + oa[1] F(6) + ... + oa[7] F(0), in this order
            R G[5];
            R pa[5], pb[5], pc[5];
            if constexpr (PS > 1) {  // point by point, four components a load
              R f4[4];
              W4(0, 7, f4);
#pragma unroll
              for (int v = 0; v < 4; v++) G[v] = xmul(oa[0], f4[v]);
              G[4] = xmul(oa[0], W(4, 7));
#pragma unroll
              for (int q = 6; q >= 0; q--) {
                W4(0, q, f4);
                const R f5 = W(4, q);
#pragma unroll
                for (int v = 0; v < 4; v++) G[v] = xfma(oa[7 - q], f4[v], G[v]);
                G[4] = xfma(oa[7 - q], f5, G[4]);
                // the points of the monotonicity test, projected from these loads
                if (q == 4) proj5v(f4[0], f4[1], f4[2], f4[3], f5, pc);
                if (q == 3) proj5v(f4[0], f4[1], f4[2], f4[3], f5, pb);
                if (q == 2) proj5v(f4[0], f4[1], f4[2], f4[3], f5, pa);
              }
              proj5v(G[0], G[1], G[2], G[3], G[4], dP);
            } else {
              // point by point: the three points of the monotonicity test are
              // projected from the values the stencil sum loaded (one
              // shared-memory read of each point)
#pragma unroll
              for (int q = 7; q >= 0; q--) {
                R f[5];
#pragma unroll
                for (int v = 0; v < 5; v++) f[v] = W(v, q);
#pragma unroll
                for (int v = 0; v < 5; v++) G[v] = q == 7 ? xmul(oa[0], f[v]) : xfma(oa[7 - q], f[v], G[v]);
                if (q == 4) proj5v(f[0], f[1], f[2], f[3], f[4], pc);
                if (q == 3) proj5v(f[0], f[1], f[2], f[3], f[4], pb);
                if (q == 2) proj5v(f[0], f[1], f[2], f[3], f[4], pa);
              }
              proj5v(G[0], G[1], G[2], G[3], G[4], dP);
            }
#pragma unroll
            for (int r = 0; r < 5; r++) {
              const R mp = xadd(pb[r], minmod2(xadd(pc[r], -pb[r]), xmul(kap, xadd(pb[r], -pa[r]))));
              dfl |= (xmul(xadd(dP[r], -pb[r]), xadd(dP[r], -mp)) >= ep ? 1u : 0u) << r;
            }
          }
          {
            // per component: oa[0] F(0) + oa[1] F(1) + ... + oa[7] F(7), in this order
            R G[5];
            R pa[5], pb[5], pc[5];
            if constexpr (PS > 1) {
              R f4[4];
              W4(5, 0, f4);
#pragma unroll
              for (int v = 0; v < 4; v++) G[v] = xmul(oa[0], f4[v]);
              G[4] = xmul(oa[0], W(9, 0));
#pragma unroll
              for (int q = 1; q <= 7; q++) {
                W4(5, q, f4);
                const R f5 = W(9, q);
#pragma unroll
                for (int v = 0; v < 4; v++) G[v] = xfma(oa[q], f4[v], G[v]);
                G[4] = xfma(oa[q], f5, G[4]);
                if (q == 3) proj5v(f4[0], f4[1], f4[2], f4[3], f5, pa);
                if (q == 4) proj5v(f4[0], f4[1], f4[2], f4[3], f5, pb);
                if (q == 5) proj5v(f4[0], f4[1], f4[2], f4[3], f5, pc);
              }
              proj5v(G[0], G[1], G[2], G[3], G[4], dM);
            } else {
#pragma unroll
              for (int q = 0; q <= 7; q++) {
                R f[5];
#pragma unroll
                for (int v = 0; v < 5; v++) f[v] = W(5 + v, q);
#pragma unroll
                for (int v = 0; v < 5; v++) G[v] = q == 0 ? xmul(oa[0], f[v]) : xfma(oa[q], f[v], G[v]);
                if (q == 3) proj5v(f[0], f[1], f[2], f[3], f[4], pa);
                if (q == 4) proj5v(f[0], f[1], f[2], f[3], f[4], pb);
                if (q == 5) proj5v(f[0], f[1], f[2], f[3], f[4], pc);
              }
              proj5v(G[0], G[1], G[2], G[3], G[4], dM);
            }
#pragma unroll
            for (int r = 0; r < 5; r++) {
              const R mp = xadd(pb[r], minmod2(xadd(pa[r], -pb[r]), xmul(kap, xadd(pb[r], -pc[r]))));
              dfl |= (xmul(xadd(dM[r], -pb[r]), xadd(dM[r], -mp)) >= ep ? 1u : 0u) << (5 + r);
            }
          }
          }
          if (dfl) {
            // queue entries djb, djb+1, ... in the order (r, F+ then F-)
            djb = atomicAdd(jn, __popc(dfl));
            const int woff = (int)(wb - sm);
            int e = djb;
#pragma unroll
            for (int r = 0; r < 5; r++) {
#pragma unroll
              for (int side = 0; side < 2; side++) {
                if ((dfl >> (5 * side + r)) & 1u) {
                  jv[e] = side ? dM[r] : dP[r];
                  jtag[e] = 16 * woff + 2 * r + side;
                  e++;
                }
              }
            }
          }
          dpend = true;
          dfo = fo;
          dcb = cb;
          continue;
#else
          {
            R mid[5], vm1[5], v0[5], vp1[5];
#pragma unroll
            for (int s = 4; s >= -3; s--) {
              const int q = s + 3;
              const R f0 = W(0, q), f1 = W(1, q), f2 = W(2, q), f3 = W(3, q), f4 = W(4, q);
              R c[5];
              c[0] = L[0][0] * f0 + L[0][1] * f1 + L[0][2] * f2 + L[0][3] * f3 + L[0][4] * f4;
              c[1] = L[1][0] * f0 + L[1][1] * f1 + L[1][2] * f2 + L[1][3] * f3;
              c[2] = L[2][0] * f0 + L[2][1] * f1 + L[2][2] * f2 + L[2][3] * f3;
              c[3] = L[3][0] * f0 + L[3][1] * f1 + L[3][2] * f2 + L[3][3] * f3 + L[3][4] * f4;
              c[4] = L[4][0] * f0 + L[4][1] * f1 + L[4][2] * f2 + L[4][3] * f3 + L[4][4] * f4;
#pragma unroll
              for (int r = 0; r < 5; r++) {
                mid[r] = (s == 4) ? oa[0] * c[r] : mid[r] + oa[4 - s] * c[r];
                if (s == -1) vm1[r] = c[r];
                if (s == 0) v0[r] = c[r];
                if (s == 1) vp1[r] = c[r];
              }
            }
#pragma unroll
            for (int r = 0; r < 5; r++) {
              const R mp = v0[r] + minmod2((vp1[r] - v0[r]), kap * (v0[r] - vm1[r]));
              if ((mid[r] - v0[r]) * (mid[r] - mp) >= ep) {
                const R vm2 = proj_row(r, 0, 1), vp2 = proj_row(r, 0, 5);
                mid[r] = omp6_limit(mid[r], vm2, vm1[r], v0[r], vp1[r], vp2, vm1[r]);
              }
              h0[r] = mid[r];
            }
          }
          {
            R mid[5], v0[5], v1[5], v2[5];
#pragma unroll
            for (int s = -3; s <= 4; s++) {
              const int q = s + 3;
              const R f0 = W(5, q), f1 = W(6, q), f2 = W(7, q), f3 = W(8, q), f4 = W(9, q);
              R c[5];
              c[0] = L[0][0] * f0 + L[0][1] * f1 + L[0][2] * f2 + L[0][3] * f3 + L[0][4] * f4;
              c[1] = L[1][0] * f0 + L[1][1] * f1 + L[1][2] * f2 + L[1][3] * f3;
              c[2] = L[2][0] * f0 + L[2][1] * f1 + L[2][2] * f2 + L[2][3] * f3;
              c[3] = L[3][0] * f0 + L[3][1] * f1 + L[3][2] * f2 + L[3][3] * f3 + L[3][4] * f4;
              c[4] = L[4][0] * f0 + L[4][1] * f1 + L[4][2] * f2 + L[4][3] * f3 + L[4][4] * f4;
#pragma unroll
              for (int r = 0; r < 5; r++) {
                mid[r] = (s == -3) ? oa[0] * c[r] : mid[r] + oa[s + 3] * c[r];
                if (s == 0) v0[r] = c[r];
                if (s == 1) v1[r] = c[r];
                if (s == 2) v2[r] = c[r];
              }
            }
#pragma unroll
            for (int r = 0; r < 5; r++) {
              const R mp = v1[r] + minmod2((v0[r] - v1[r]), kap * (v1[r] - v2[r]));
              if ((mid[r] - v1[r]) * (mid[r] - mp) >= ep) {
                const R v3 = proj_row(r, 5, 6), vm1 = proj_row(r, 5, 2);
                mid[r] = omp6_limit(mid[r], v3, v2[r], v1[r], v0[r], vm1, v0[r]);
              }
              h0[r] = h0[r] + mid[r];
            }
          }
#endif
        } else {
          // ---- F+ projected onto the characteristic variables (:254-261), reconstructed
          {
            R q[5][8];
            constexpr int LO = Stencil<SCHEME>::PLO, HI = Stencil<SCHEME>::PHI;
#pragma unroll
            for (int s = -3; s <= 4; s++) {
#if OCFD_FEWER_DIVS
              R c[5] = {R(0), R(0), R(0), R(0), R(0)};
              if (s >= LO && s <= HI) proj5(0, s + 3, c);
#pragma unroll
              for (int r = 0; r < 5; r++) q[r][s + 3] = c[r];
#else
#pragma unroll
              for (int r = 0; r < 5; r++) q[r][s + 3] = (s < LO || s > HI) ? R(0) : proj_row(r, 0, s + 3);
#endif
            }
            if (ALLIN || inner1) {
#pragma unroll
              for (int r = 0; r < 5; r++) h0[r] = schemeP<SCHEME>(q[r] + 3, U, ihy);
            } else {
#pragma unroll
              for (int r = 0; r < 5; r++) h0[r] = ch_flux1_bnd(q[r] + 3, g, nn, ph, DIR);
            }
          }
          // ---- F- (:264-271)
          {
            R q[5][8];
            constexpr int LO = Stencil<SCHEME>::MLO, HI = Stencil<SCHEME>::MHI;
#pragma unroll
            for (int s = -3; s <= 4; s++) {
#if OCFD_FEWER_DIVS
              R c[5] = {R(0), R(0), R(0), R(0), R(0)};
              if (s >= LO && s <= HI) proj5(5, s + 3, c);
#pragma unroll
              for (int r = 0; r < 5; r++) q[r][s + 3] = c[r];
#else
#pragma unroll
              for (int r = 0; r < 5; r++) q[r][s + 3] = (s < LO || s > HI) ? R(0) : proj_row(r, 5, s + 3);
#endif
            }
            if (ALLIN || inner2) {
#pragma unroll
              for (int r = 0; r < 5; r++) h0[r] = h0[r] + schemeM<SCHEME>(q[r] + 3, U, ihy);
            } else {
#pragma unroll
              for (int r = 0; r < 5; r++) h0[r] = h0[r] + ch_flux2_bnd(q[r] + 3, g, nn, ph, DIR);
            }
          }
        }
        // ---- back to physical space, hh = R h0 (:284-288); R = S^-1 (:244-248)
#if OCFD_FEWER_DIVS
        cb.back(h0, hh, R(ph.inv_gm1));
#else
        const R H = V2 + R(1) / KK;
        hh[0] = h0[0] + h0[3] + h0[4];
        hh[1] = u1 * h0[0] + l1 * h0[1] + m1 * h0[2] + (u1 - c1 * n1) * h0[3] + (u1 + c1 * n1) * h0[4];
        hh[2] = v1 * h0[0] + l2 * h0[1] + m2 * h0[2] + (v1 - c1 * n2) * h0[3] + (v1 + c1 * n2) * h0[4];
        hh[3] = w1 * h0[0] + l3 * h0[1] + m3 * h0[2] + (w1 - c1 * n3) * h0[3] + (w1 + c1 * n3) * h0[4];
        hh[4] = V2 * h0[0] + ul * h0[1] + um * h0[2] + (H - c1 * un) * h0[3] + (H + c1 * un) * h0[4];
#endif
      }
    }
    hf_store5(out, fo, a.fs, hh);
  }
  if constexpr (DEFER) {
    __syncthreads();
    const int nj = min(*jn, JC);
    const R gm1 = R(ph.gamma) - R(1);
    for (int e = threadIdx.x; e < nj; e += blockDim.x) {
      const int tag = jtag[e];
      jv[e] = lim_eval<R, VS, QS, GAP, DIR, AXS>(sm + (tag >> 4), (tag >> 1) & 7, tag & 1, jv[e], gm1);
    }
    __syncthreads();
    if (dpend) {
      if (dfl) {
        int e = djb;
#pragma unroll
        for (int r = 0; r < 5; r++) {
          if ((dfl >> r) & 1u) dP[r] = jv[e++];
          if ((dfl >> (5 + r)) & 1u) dM[r] = jv[e++];
        }
      }
      // back to physical space, hh = R h0 (OCFD_inviscous_character.f90:284-288)
      R h0[5];
#pragma unroll
      for (int r = 0; r < 5; r++) h0[r] = xadd(dP[r], dM[r]);
      R hh[5];
      dcb.back(h0, hh, R(ph.inv_gm1));
      hf_store5(out, dfo, a.fs, hh);
    }
  }
}

template <int DIR, bool CHAR, int NP, int TF, typename R>
constexpr size_t face_smem_points() {
  // split fluxes (+ face state)
  return (size_t)(face_ps<DIR, CHAR, R>() > 1 ? face_ps<DIR, CHAR, R>() : (CHAR ? 17 : 10)) * NP * (TF + 7) *
         sizeof(R);
}
template <int DIR, bool CHAR, int NP, int TF, typename R>
constexpr size_t face_smem() {
  // (+ the limiter queue)
  return face_smem_points<DIR, CHAR, NP, TF, R>() + (CHAR ? LimQueue<NP * TF>::template bytes<R>() : 0);
}
// TMA sweeps: the limiter queue shares memory with the eight staged input
// tiles (read only in phase 1, the queue is used after phase 1's barrier) when
// its entry count -- written before phase 1 -- lies past them.
template <int DIR, bool CHAR, int SCHEME, int NP, int TF, typename R, typename S>
struct FaceTmaSmem {
  using B = TmaBox<DIR, NP, TF, S>;
  static constexpr size_t TILE = 8 * (size_t)B::SLOT;
  static constexpr size_t QB = LimQueue<NP * TF>::template bytes<R>();
  static constexpr size_t COUNT_AT = (size_t)LimQueue<NP * TF>::CAP * (sizeof(R) + sizeof(int));
  static constexpr bool ALIAS = CHAR && SCHEME == SCH_OMP6 && OCFD_FEWER_DIVS && COUNT_AT >= TILE;
  static constexpr size_t UNION = ALIAS ? (TILE > QB ? TILE : QB) : TILE;  // before the staged points
  static constexpr size_t BYTES =
      128 + UNION + (ALIAS ? face_smem_points<DIR, CHAR, NP, TF, R>() : face_smem<DIR, CHAR, NP, TF, R>());
};

// Minimum resident blocks per SM.  FP64: two (<= 128 registers) measured
// faster than one.  FP32: four (<= 64 registers) -- 17% faster than two on the
// characteristic OMP6 sweeps at 256^3 despite a few spilled registers, equal on
// the flux-vector sweeps.
#ifndef OCFD_FACE32_MINB
#define OCFD_FACE32_MINB 4
#endif
#define OCFD_FACE_MINB (sizeof(R) == 8 ? 2 : OCFD_FACE32_MINB)
// threads and minimum resident blocks of the single-instance sweeps
#define OCFD_FACE_NT (FaceTile<DIR, CHAR, SCHEME>::NP * FaceTile<DIR, CHAR, SCHEME>::TF)
#ifndef OCFD_FACE64_MINB128
#define OCFD_FACE64_MINB128 4  // FP64, 128-thread tiles: 4 blocks (128 registers); 5 (96
                               // registers) measured 2% faster on x, 8% slower on y and z
#endif
#ifndef OCFD_FACE64_MINB128_AX
#define OCFD_FACE64_MINB128_AX 5  // the axis-aligned variants (about 110 registers at 4 blocks)
#endif
#define OCFD_FACE_BOUNDS                                                                                     \
  __launch_bounds__(OCFD_FACE_NT,                                                                            \
                    (OCFD_FACE_NT == 128 && sizeof(R) == 8) ? (AXS ? OCFD_FACE64_MINB128_AX : OCFD_FACE64_MINB128) \
                                                            : OCFD_FACE_MINB * 256 / OCFD_FACE_NT)
template <int DIR, bool CHAR, int SCHEME, bool ALLIN, typename R, typename S, bool AXS = false>
__global__ void OCFD_FACE_BOUNDS k_face(FaceArgs<S> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  face_body<DIR, CHAR, SCHEME, ALLIN, FaceTile<DIR, CHAR, SCHEME>::NP, FaceTile<DIR, CHAR, SCHEME>::TF, R, S, false,
            AXS>(a, blockIdx.x, blockIdx.y, blockIdx.z, reinterpret_cast<R*>(smem_raw));
}

// Batched launch: the blocks of all instances in one 1-D grid; each block finds
// its instance and its block coordinates from the batch table.  Periodic
// instances only (ALLIN).
template <int DIR, bool CHAR, int SCHEME, int V, typename R, typename S>
__global__ void __launch_bounds__(256, OCFD_FACE_MINB) k_face_batch(BatchTab<FaceArgs<S>> b) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(16) FaceArgs<S> sa;
  int bx, by, bz;
  const int q = batch_locate(b, blockIdx.x, bx, by, bz);
  const FaceArgs<S>& A = batch_args(b, q, &sa);
  // the member's own sweep variant, as its single-instance launch would choose
  // it (batched and single results are the same bits)
  if (OCFD_FEWER_DIVS && axis_aligned<DIR>(A.ph.metzero))
    face_body<DIR, CHAR, SCHEME, true, FaceTileV<DIR, V>::NP, FaceTileV<DIR, V>::TF, R, S, false,
              OCFD_FEWER_DIVS != 0>(A, bx, by, bz, reinterpret_cast<R*>(smem_raw));
  else
    face_body<DIR, CHAR, SCHEME, true, FaceTileV<DIR, V>::NP, FaceTileV<DIR, V>::TF, R, S>(
        A, bx, by, bz, reinterpret_cast<R*>(smem_raw));
}

// Single-instance sweep with the input tiles staged by TMA (the arithmetic is
// that of k_face).  ALLIN: a periodic direction; otherwise the sweep includes
// the boundary closures, and tile points past the haloed array (read as zeros
// by the copy) are not used.
template <int DIR, bool CHAR, int SCHEME, typename R, typename S, bool AXS = false, bool ALLIN = true>
__global__ void OCFD_FACE_BOUNDS k_face_tma(FaceArgs<S> a, const __grid_constant__ FaceTmaMaps tm) {
  constexpr int NP = FaceTile<DIR, CHAR, SCHEME>::NP, TF = FaceTile<DIR, CHAR, SCHEME>::TF;
  using B = TmaBox<DIR, NP, TF, S>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  // TMA destinations start on 128-byte boundaries (128 bytes of the launch's
  // dynamic shared memory are reserved for this rounding)
  unsigned char* base = smem_raw + ((128 - (smem_u32(smem_raw) & 127u)) & 127u);
  using L = FaceTmaSmem<DIR, CHAR, SCHEME, NP, TF, R, S>;
  S* tile = reinterpret_cast<S*>(base);
  R* sm = reinterpret_cast<R*>(base + L::UNION);
  R* qbase = L::ALIAS ? reinterpret_cast<R*>(base) : nullptr;
  const int bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z;
  const int g0 = a.fbeg + (DIR == 0 ? bx : by) * TF;  // first face; its stencil starts at g0 - 3
  const int pbase = (DIR == 0 ? by : bx) * NP;
  // haloed (0-based) coordinates of the tile's first element: index + LAP - 1
  const int x0 = DIR == 0 ? g0 : pbase + 4;
  const int toff = x0 % B::A;
  const int c0 = x0 - toff;
  const int c1 = DIR == 0 ? pbase + 4 : (DIR == 1 ? g0 : bz + 4);
  const int c2 = DIR == 2 ? g0 : bz + 4;
  // once a block of this instance has given up on its tile copies (error 4),
  // the launch's results are invalid: later blocks issue no copies and leave
  if (__syncthreads_or(threadIdx.x == 0 && *reinterpret_cast<volatile const int*>(a.err) == 4)) return;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int m0 = 13 + 3 * DIR;
    bool need[8];
    uint32_t bytes = 0;
    for (int q = 0; q < 8; q++) {
      need[q] = q < 5 || !((a.ph.metzero >> (m0 + q - 5)) & 1u);
      if (need[q]) bytes += B::BYTES;
    }
    mbar_arrive_expect_tx(&bar, bytes + (uint32_t)a.test_tx);
    if constexpr (sizeof(S) == 4) {
      // FP32: d, then u,v,w,T interleaved (one 4-D copy filling slots 1-4)
      tma_load_3d(tile, &tm.m[0], c0, c1, c2, &bar);
      tma_load_4d(tile + B::SLOT_ELEMS, &tm.m[1], 0, c0, c1, c2, &bar);
      for (int q = 5; q < 8; q++)
        if (need[q]) tma_load_3d(tile + q * B::SLOT_ELEMS, &tm.m[q], c0, c1, c2, &bar);
    } else {
      for (int q = 0; q < 8; q++)
        if (need[q]) tma_load_3d(tile + q * B::SLOT_ELEMS, &tm.m[q], c0, c1, c2, &bar);
    }
  }
  // bounded wait (about a second); a block that gives up records the error and
  // waits once more, again bounded, for its copies before leaving
  bool done = mbar_wait_bounded(&bar, 0, 1u << 20);
  if (__syncthreads_or(!done)) {
    if (threadIdx.x == 0) {
      atomicExch(a.err, 4);
      mbar_wait_bounded(&bar, 0, 1u << 20);
    }
    return;
  }
  face_body<DIR, CHAR, SCHEME, ALLIN, NP, TF, R, S, true, AXS>(a, bx, by, bz, sm, tile, toff, qbase);
}


// ---------------------------------------------------------------------------
template <int DIR, bool CHAR, int SCHEME, bool ALLIN, typename R, typename S, bool AXS = false>
static cudaError_t launch_face_t(const FaceArgs<S>& a, cudaStream_t st) {
  constexpr int NP = FaceTile<DIR, CHAR, SCHEME>::NP, TF = FaceTile<DIR, CHAR, SCHEME>::TF;
  constexpr size_t smem = face_smem<DIR, CHAR, NP, TF, R>();
  auto kern = k_face<DIR, CHAR, SCHEME, ALLIN, R, S, AXS>;
  if (a.g.n == 0) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<face_grid<DIR, NP, TF>(a), NP * TF, smem, st>>>(a);
  return cudaGetLastError();
}

// Batched face sweep.  nblocks == 0 asks for the shared-memory attribute to be
// set instead of a launch; the host fills b from face_batch_dims().
template <int DIR, bool CHAR, int SCHEME, int V, typename R, typename S>
static cudaError_t launch_face_batch_t(const BatchTab<FaceArgs<S>>& b, int nblocks, cudaStream_t st) {
  constexpr int NP = FaceTileV<DIR, V>::NP, TF = FaceTileV<DIR, V>::TF;
  constexpr size_t smem = face_smem<DIR, CHAR, NP, TF, R>();
  auto kern = k_face_batch<DIR, CHAR, SCHEME, V, R, S>;
  if (nblocks == 0) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<nblocks, NP * TF, smem, st>>>(b);
  return cudaGetLastError();
}

template <typename R, typename S>
cudaError_t launch_face_batch(int dir, bool chr, int scheme, int variant, const BatchTab<FaceArgs<S>>& b,
                              int nblocks, cudaStream_t st) {
#define OCFD_FB_CASE(D, C, SC)                                                     \
  if (dir == D && chr == C && scheme == SC)                                        \
    return variant ? launch_face_batch_t<D, C, SC, 1, R, S>(b, nblocks, st)        \
                   : launch_face_batch_t<D, C, SC, 0, R, S>(b, nblocks, st);
#define OCFD_FB_SCHEMES(D, C) \
  OCFD_FB_CASE(D, C, SCH_WENO5) \
  OCFD_FB_CASE(D, C, SCH_WENO7) \
  OCFD_FB_CASE(D, C, SCH_OMP6)  \
  OCFD_FB_CASE(D, C, SCH_UD7L)  \
  OCFD_FB_CASE(D, C, SCH_HYBRID)
  OCFD_FB_SCHEMES(0, false)
  OCFD_FB_SCHEMES(1, false)
  OCFD_FB_SCHEMES(2, false)
  OCFD_FB_SCHEMES(0, true)
  OCFD_FB_SCHEMES(1, true)
  OCFD_FB_SCHEMES(2, true)
#undef OCFD_FB_SCHEMES
#undef OCFD_FB_CASE
  return cudaErrorInvalidValue;
}

// Per-instance launch grid of a batched face sweep for tile variant V.
template <typename S>
dim3 face_batch_dims(int dir, int variant, const FaceArgs<S>& a) {
  if (dir == 0) return variant ? face_grid<0, 8, 32>(a) : face_grid<0, 4, 64>(a);
  if (dir == 1) return variant ? face_grid<1, 8, 32>(a) : face_grid<1, 16, 16>(a);
  return variant ? face_grid<2, 8, 32>(a) : face_grid<2, 16, 16>(a);
}

// ---- TMA path: tensor maps of the sweep's eight input arrays
bool face_tma_enabled();
bool face_tma32_enabled();
bool encode_tile_map(CUtensorMap* map, const void* base, bool f64, const Grid& g, int bx, int by, int bz);
// 4-D map of the interleaved FP32 u,v,w,T copy (4 floats a haloed point), box (4, bx, by, bz)
bool encode_tile_map4(CUtensorMap* map, const void* base, const Grid& g, int bx, int by, int bz);

template <typename S>
inline bool tma_strides_ok(const Grid& g) {
  return ((long long)g.nxh * sizeof(S)) % 16 == 0 && ((long long)g.nxh * g.nyh * sizeof(S)) % 16 == 0;
}

template <int DIR, bool CHAR, int SCHEME, typename R, typename S, bool AXS = false, bool ALLIN = true>
static cudaError_t launch_face_tma_t(const FaceArgs<S>& a, cudaStream_t st) {
  constexpr int NP = FaceTile<DIR, CHAR, SCHEME>::NP, TF = FaceTile<DIR, CHAR, SCHEME>::TF;
  using B = TmaBox<DIR, NP, TF, S>;
  constexpr size_t smem = FaceTmaSmem<DIR, CHAR, SCHEME, NP, TF, R, S>::BYTES;
  auto kern = k_face_tma<DIR, CHAR, SCHEME, R, S, AXS, ALLIN>;
  if (a.g.n == 0) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  FaceTmaMaps tm;
  memset(&tm, 0, sizeof(tm));
  const S* arr[8] = {a.d, a.u, a.v, a.w, a.T, a.A1, a.A2, a.A3};
  for (int q = 0; q < 8; q++) {
    bool ok = true;
    if (sizeof(S) == 4 && q == 1)
      ok = encode_tile_map4(&tm.m[1], a.q4, a.g, B::BX, B::BY, B::BZ);
    else if (sizeof(S) == 8 || q == 0 || q >= 5)
      ok = encode_tile_map(&tm.m[q], arr[q], sizeof(S) == 8, a.g, B::BX, B::BY, B::BZ);
    if (!ok) return cudaErrorInvalidValue;
  }
  kern<<<face_grid<DIR, NP, TF>(a), NP * TF, smem, st>>>(a, tm);
  return cudaGetLastError();
}

// One (direction, form, scheme) combination: the TMA-staged sweep (FP64:
// periodic directions measured 1-3% faster at 256^3; FP32 with the four
// interleaved u,v,w,T floats of a point as the innermost dimension of a 4-D
// copy), the axis-aligned variant when the metric row allows it (production
// build).  An empty grid
// asks for the shared-memory attribute of every variant instead.
template <int D, bool C, int SC, typename R, typename S>
static cudaError_t launch_face_dc(const FaceArgs<S>& a, cudaStream_t st) {
  constexpr bool kAx = OCFD_FEWER_DIVS != 0;
  if (a.g.n == 0) {
    cudaError_t e = launch_face_t<D, C, SC, false, R, S>(a, st);
    if (e == cudaSuccess) e = launch_face_t<D, C, SC, true, R, S>(a, st);
    if (kAx && e == cudaSuccess) e = launch_face_t<D, C, SC, true, R, S, kAx>(a, st);
    if (e == cudaSuccess) e = launch_face_tma_t<D, C, SC, R, S>(a, st);
    if (kAx && e == cudaSuccess) e = launch_face_tma_t<D, C, SC, R, S, kAx>(a, st);
    if (e == cudaSuccess) e = launch_face_tma_t<D, C, SC, R, S, false, false>(a, st);
    return e;
  }
  const bool allin = a.ph.periodic[D] != 0;
  const bool tma = !a.no_tma && (sizeof(S) == 8 ? face_tma_enabled() : face_tma32_enabled()) && tma_strides_ok<S>(a.g);
  if (!allin) {
    if (tma) return launch_face_tma_t<D, C, SC, R, S, false, false>(a, st);
    return launch_face_t<D, C, SC, false, R, S>(a, st);
  }
  const bool ax = kAx && axis_aligned<D>(a.ph.metzero);
  if (tma) return ax ? launch_face_tma_t<D, C, SC, R, S, kAx>(a, st) : launch_face_tma_t<D, C, SC, R, S>(a, st);
  return ax ? launch_face_t<D, C, SC, true, R, S, kAx>(a, st) : launch_face_t<D, C, SC, true, R, S>(a, st);
}

template <typename R, typename S>
cudaError_t launch_face(int dir, bool chr, int scheme, const FaceArgs<S>& a, cudaStream_t st) {
#define OCFD_FACE_CASE(D, C, SC) \
  if (dir == D && chr == C && scheme == SC) return launch_face_dc<D, C, SC, R, S>(a, st);
#define OCFD_FACE_SCHEMES(D, C)         \
  OCFD_FACE_CASE(D, C, SCH_WENO5)       \
  OCFD_FACE_CASE(D, C, SCH_WENO7)       \
  OCFD_FACE_CASE(D, C, SCH_OMP6)        \
  OCFD_FACE_CASE(D, C, SCH_UD7L)        \
  OCFD_FACE_CASE(D, C, SCH_HYBRID)
  OCFD_FACE_SCHEMES(0, false)
  OCFD_FACE_SCHEMES(1, false)
  OCFD_FACE_SCHEMES(2, false)
  OCFD_FACE_SCHEMES(0, true)
  OCFD_FACE_SCHEMES(1, true)
  OCFD_FACE_SCHEMES(2, true)
#undef OCFD_FACE_SCHEMES
#undef OCFD_FACE_CASE
  return cudaErrorInvalidValue;
}

}  // namespace ocfd
