"""Second, independent transcription of the reference's array-form hot-path
routines in NumPy (TEST INFRASTRUCTURE ONLY).

Written from the Fortran sources directly -- not from oracle/ocfd_oracle.c --
so that the C oracle, which the GPU parity tests trust, is checked by a second
reading of the same routines.  Every expression keeps the Fortran operand order
(IEEE double, no fused multiply-add: NumPy evaluates each operation rounded,
left to right like gfortran without fast-math), so on the same inputs this
module and the C oracle must agree bit for bit.  Only tests/ import it.

Covered (file:line of the reference, src/):
  OCFD_Schemes.f90:6-358      WENO5/WENO7/OMP6/UD7L/hybrid array forms, minmod2/4
  OCFD_Schemes_1.f90:9-384    the point forms and the WENO5 boundary forms
  OCFD_inviscous.f90:53-361   du_inviscous with OCFD2d_flux1/2 (boundary closures)
  OCFD_flux_split.f90:5-104   Steger-Warming and local Lax-Friedrichs splitting
  OCFD_inviscous_character.f90:3-416  du_inviscous_Character, flux_charteric,
                              flux_x1/x2, the L (S) and R (S1) matrices
  OCFD_dxyz_viscous.f90:3-239 OCFD_dx0/dy0/dz0, CD6/CD8 with boundary closures
  OCFD_viscous.f90:29-149     du_viscous and comput_Amu
  OCFD_SetHybrid.f90:2-15     set_hybrid_scheme

Arrays are NumPy C-order views of the Fortran layout: haloed fields are
(nz+8, ny+8, nx+8) with Fortran index i at position i + 3 (LAP = 4); f and du
are (5, nz, ny, nx).  A sweep moves its direction to the last axis.
"""
from __future__ import annotations

import numpy as np

LAP = 4
SCH_WENO5, SCH_WENO7, SCH_OMP6, SCH_UD7L, SCH_CD6, SCH_CD8, SCH_HYBRID = 1, 2, 3, 4, 5, 6, 10
DEL_LIFT, DEL_RIGHT = 1, 2

# ---------------------------------------------------------------------------
# constants of the schemes (OCFD_Schemes.f90 / OCFD_Schemes_1.f90), folded in
# double precision in the order the parameter statements write them
W5_EP, W5_C03, W5_C13, W5_C23 = 1.0e-6, 3.0 / 10.0, 3.0 / 5.0, 1.0 / 10.0
W7 = dict(C0=1.0 / 35.0, C1=12.0 / 35.0, C2=18.0 / 35.0, C3=4.0 / 35.0,
          a11=-2.0 / 6.0, a12=9.0 / 6.0, a13=-18.0 / 6.0, a14=11.0 / 6.0,
          a21=1.0 / 6.0, a23=3.0 / 6.0, a24=2.0 / 6.0,
          a31=-2.0 / 6.0, a32=-3.0 / 6.0, a34=-1.0 / 6.0,
          a41=-11.0 / 6.0, a42=18.0 / 6.0, a43=-9.0 / 6.0, a44=2.0 / 6.0,
          b12=4.0, b13=-5.0, b14=2.0, b22=-2.0, b41=2.0, b42=-5.0, b43=4.0, c12=3.0,
          d12=13.0 / 12.0, d13=1043.0 / 960.0, d14=1.0 / 12.0,
          e11=-3.0 / 12.0, e12=13.0 / 12.0, e13=-23.0 / 12.0, e14=25.0 / 12.0,
          e21=1.0 / 12.0, e22=-5.0 / 12.0, e23=13.0 / 12.0, e24=3.0 / 12.0,
          e31=-1.0 / 12.0, e32=7.0 / 12.0, e33=7.0 / 12.0, e34=-1.0 / 12.0,
          e41=3.0 / 12.0, e42=13.0 / 12.0, e43=-5.0 / 12.0, e44=1.0 / 12.0, ep=1.0e-8)
OMP_KAPPA = 4.0
OMP_EP = float(np.float32(1.0e-10))  # "ep = 1.e-10": a default-real (single precision) literal
_OMP_m, _OMP_n = 0.015, 0.0
_OMP_a = 0.5 * (_OMP_m + _OMP_n)
_OMP_b = 0.5 * (_OMP_m - _OMP_n)
OMP_A = (_OMP_a,
         1.0 / 60.0 - _OMP_b - 6.0 * _OMP_a,
         -2.0 / 15.0 + 6.0 * _OMP_b + 15.0 * _OMP_a,
         37.0 / 60.0 - 15.0 * _OMP_b - 20.0 * _OMP_a,
         37.0 / 60.0 + 20.0 * _OMP_b + 15.0 * _OMP_a,
         -2.0 / 15.0 - 6.0 * _OMP_a - 15.0 * _OMP_b,
         1.0 / 60.0 + _OMP_a + 6.0 * _OMP_b,
         -_OMP_b)


def sq(x):
    """x**2 with an integer exponent: one multiplication."""
    return x * x


def sign1(x):
    """Fortran sign(1.d0, x)."""
    return np.copysign(1.0, x)


def minmod2(x1, x2):
    return 0.5 * (sign1(x1) + sign1(x2)) * np.minimum(np.abs(x1), np.abs(x2))


def minmod4(x1, x2, x3, x4):
    m = 0.5 * (sign1(x1) + sign1(x2))
    m = m * np.abs(0.5 * (sign1(x1) + sign1(x3)))
    m = m * np.abs(0.5 * (sign1(x1) + sign1(x4)))
    return m * np.minimum(np.minimum(np.minimum(np.abs(x1), np.abs(x2)), np.abs(x3)), np.abs(x4))


def min3(a, b, c):
    return np.minimum(np.minimum(a, b), c)


def max3(a, b, c):
    return np.maximum(np.maximum(a, b), c)


# ---------------------------------------------------------------------------
# point forms: V(s) is the stencil value v(s) of every face at once
def weno5P(V, dele=0):
    """hh_weno5P / hh_weno5P_boundary (OCFD_Schemes_1.f90:9-30, 266-296)."""
    z = 0.0 * V(0)
    a0 = q03 = a2 = q23 = z
    if dele != DEL_RIGHT:
        S0 = 13.0 / 12.0 * sq(V(0) - 2.0 * V(1) + V(2)) + 1.0 / 4.0 * sq(3.0 * V(0) - 4.0 * V(1) + V(2))
        a0 = W5_C03 / sq(W5_EP + S0)
        q03 = 1.0 / 3.0 * V(0) + 5.0 / 6.0 * V(1) - 1.0 / 6.0 * V(2)
    S1 = 13.0 / 12.0 * sq(V(-1) - 2.0 * V(0) + V(1)) + 1.0 / 4.0 * sq(V(-1) - V(1))
    a1 = W5_C13 / sq(W5_EP + S1)
    q13 = -1.0 / 6.0 * V(-1) + 5.0 / 6.0 * V(0) + 1.0 / 3.0 * V(1)
    if dele != DEL_LIFT:
        S2 = 13.0 / 12.0 * sq(V(-2) - 2.0 * V(-1) + V(0)) + 1.0 / 4.0 * sq(V(-2) - 4.0 * V(-1) + 3.0 * V(0))
        a2 = W5_C23 / sq(W5_EP + S2)
        q23 = 1.0 / 3.0 * V(-2) - 7.0 / 6.0 * V(-1) + 11.0 / 6.0 * V(0)
    am = a0 + a1 + a2
    return (a0 * q03 + a1 * q13 + a2 * q23) / am


def weno5M(V, dele=0):
    """hh_weno5M / hh_weno5M_boundary (OCFD_Schemes_1.f90:32-52, 298-325)."""
    z = 0.0 * V(0)
    a0 = q03 = a2 = q23 = z
    if dele != DEL_LIFT:
        S0 = 13.0 / 12.0 * sq(V(1) - 2.0 * V(0) + V(-1)) + 1.0 / 4.0 * sq(3.0 * V(1) - 4.0 * V(0) + V(-1))
        a0 = W5_C03 / sq(W5_EP + S0)
        q03 = 1.0 / 3.0 * V(1) + 5.0 / 6.0 * V(0) - 1.0 / 6.0 * V(-1)
    S1 = 13.0 / 12.0 * sq(V(2) - 2.0 * V(1) + V(0)) + 1.0 / 4.0 * sq(V(2) - V(0))
    a1 = W5_C13 / sq(W5_EP + S1)
    q13 = -1.0 / 6.0 * V(2) + 5.0 / 6.0 * V(1) + 1.0 / 3.0 * V(0)
    if dele != DEL_RIGHT:
        S2 = 13.0 / 12.0 * sq(V(3) - 2.0 * V(2) + V(1)) + 1.0 / 4.0 * sq(V(3) - 4.0 * V(2) + 3.0 * V(1))
        a2 = W5_C23 / sq(W5_EP + S2)
        q23 = 1.0 / 3.0 * V(3) - 7.0 / 6.0 * V(2) + 11.0 / 6.0 * V(1)
    am = a0 + a1 + a2
    return (a0 * q03 + a1 * q13 + a2 * q23) / am


def _weno7(v, m3, m2, m1, c0, p1, p2, p3):
    """WENO-JS7 on the seven values of a stencil ordered towards the face
    (OCFD_Schemes.f90:59-124 for F+: v(i-3..i+3); :129-193 for F-: v(i+4..i-2))."""
    k = W7
    S10 = k["a11"] * m3 + k["a12"] * m2 + k["a13"] * m1 + k["a14"] * c0
    S11 = k["a21"] * m2 - m1 + k["a23"] * c0 + k["a24"] * p1
    S12 = k["a31"] * m1 + k["a32"] * c0 + p1 + k["a34"] * p2
    S13 = k["a41"] * c0 + k["a42"] * p1 + k["a43"] * p2 + k["a44"] * p3
    S20 = -m3 + k["b12"] * m2 + k["b13"] * m1 + k["b14"] * c0
    S21 = m1 + k["b22"] * c0 + p1
    S22 = c0 + k["b22"] * p1 + p2
    S23 = k["b41"] * c0 + k["b42"] * p1 + k["b43"] * p2 - p3
    S30 = -m3 + k["c12"] * (m2 - m1) + c0
    S31 = -m2 + k["c12"] * (m1 - c0) + p1
    S32 = -m1 + k["c12"] * (c0 - p1) + p2
    S33 = -c0 + k["c12"] * (p1 - p2) + p3
    S0 = S10 * S10 + k["d12"] * S20 * S20 + k["d13"] * S30 * S30 + k["d14"] * S10 * S30
    S1 = S11 * S11 + k["d12"] * S21 * S21 + k["d13"] * S31 * S31 + k["d14"] * S11 * S31
    S2 = S12 * S12 + k["d12"] * S22 * S22 + k["d13"] * S32 * S32 + k["d14"] * S12 * S32
    S3 = S13 * S13 + k["d12"] * S23 * S23 + k["d13"] * S33 * S33 + k["d14"] * S13 * S33
    a0 = k["C0"] / sq(k["ep"] + S0)
    a1 = k["C1"] / sq(k["ep"] + S1)
    a2 = k["C2"] / sq(k["ep"] + S2)
    a3 = k["C3"] / sq(k["ep"] + S3)
    am = a0 + a1 + a2 + a3
    q0 = k["e11"] * m3 + k["e12"] * m2 + k["e13"] * m1 + k["e14"] * c0
    q1 = k["e21"] * m2 + k["e22"] * m1 + k["e23"] * c0 + k["e24"] * p1
    q2 = k["e31"] * m1 + k["e32"] * c0 + k["e33"] * p1 + k["e34"] * p2
    q3 = k["e41"] * c0 + k["e42"] * p1 + k["e43"] * p2 + k["e44"] * p3
    return (a0 * q0 + a1 * q1 + a2 * q2 + a3 * q3) / am


def weno7P(V):
    """hh_weno7P (OCFD_Schemes_1.f90:58-121), stencil v(-3..3)."""
    return _weno7(V, V(-3), V(-2), V(-1), V(0), V(1), V(2), V(3))


def weno7M(V):
    """hh_weno7M (OCFD_Schemes_1.f90:124-187), stencil v(-2..4) mirrored."""
    return _weno7(V, V(4), V(3), V(2), V(1), V(0), V(-1), V(-2))


def omp6P(V):
    """hh_OMP6P (OCFD_Schemes_1.f90:195-225) = OCFD_OMP6P (OCFD_Schemes.f90:201-236)."""
    A = OMP_A
    mid = (A[0] * V(4) + A[1] * V(3) + A[2] * V(2) + A[3] * V(1) + A[4] * V(0) + A[5] * V(-1) + A[6] * V(-2)
           + A[7] * V(-3))
    mp = V(0) + minmod2((V(1) - V(0)), OMP_KAPPA * (V(0) - V(-1)))
    test = (mid - V(0)) * (mid - mp) >= OMP_EP
    d1 = V(-2) + V(0) - 2.0 * V(-1)
    d2 = V(-1) + V(1) - 2.0 * V(0)
    d3 = V(0) + V(2) - 2.0 * V(1)
    ul = V(0) + OMP_KAPPA * (V(0) - V(-1))
    md = 0.5 * (V(0) + V(1)) - 0.5 * minmod4(4.0 * d2 - d3, 4.0 * d3 - d2, d2, d3)
    lc = V(0) + 0.5 * (V(0) - V(-1)) + OMP_KAPPA * minmod4(4.0 * d1 - d2, 4.0 * d2 - d1, d2, d1) / 3.0
    fmin = np.maximum(min3(V(0), V(1), md), min3(V(0), ul, lc))
    fmax = np.minimum(max3(V(0), V(1), md), max3(V(0), ul, lc))
    return np.where(test, mid + minmod2(fmax - mid, fmin - mid), mid)


def omp6M(V):
    """hh_OMP6M (OCFD_Schemes_1.f90:227-260) = OCFD_OMP6M (OCFD_Schemes.f90:238-271)."""
    A = OMP_A
    mid = (A[0] * V(-3) + A[1] * V(-2) + A[2] * V(-1) + A[3] * V(0) + A[4] * V(1) + A[5] * V(2) + A[6] * V(3)
           + A[7] * V(4))
    mp = V(1) + minmod2((V(0) - V(1)), OMP_KAPPA * (V(1) - V(2)))
    test = (mid - V(1)) * (mid - mp) >= OMP_EP
    d1 = V(3) + V(1) - 2.0 * V(2)
    d2 = V(2) + V(0) - 2.0 * V(1)
    d3 = V(1) + V(-1) - 2.0 * V(0)
    ul = V(1) + OMP_KAPPA * (V(1) - V(2))
    md = 0.5 * (V(1) + V(0)) - 0.5 * minmod4(4.0 * d2 - d3, 4.0 * d3 - d2, d2, d3)
    lc = V(1) + 0.5 * (V(1) - V(0)) + OMP_KAPPA * minmod4(4.0 * d1 - d2, 4.0 * d2 - d1, d2, d1) / 3.0
    fmin = np.maximum(min3(V(1), V(0), md), min3(V(1), ul, lc))
    fmax = np.minimum(max3(V(1), V(0), md), max3(V(1), ul, lc))
    return np.where(test, mid + minmod2(fmax - mid, fmin - mid), mid)


def ud7lP(V, U):
    """hh_UD7L_P (OCFD_Schemes_1.f90:328-337); U = Scheme%UD7L(1:8)."""
    return (U[0] * V(-3) + U[1] * V(-2) + U[2] * V(-1) + U[3] * V(0) + U[4] * V(1) + U[5] * V(2) + U[6] * V(3)
            + U[7] * V(4))


def ud7lM(V, U):
    """hh_UD7L_M (OCFD_Schemes_1.f90:339-348)."""
    return (U[0] * V(4) + U[1] * V(3) + U[2] * V(2) + U[3] * V(1) + U[4] * V(0) + U[5] * V(-1) + U[6] * V(-2)
            + U[7] * V(-3))


def hybridP(V, U, ihy):
    """hh_HybridP (OCFD_Schemes_1.f90:351-366): 1 UD7L, 2 WENO7, else WENO5."""
    with np.errstate(all="ignore"):
        return np.where(ihy == 1, ud7lP(V, U), np.where(ihy == 2, weno7P(V), weno5P(V)))


def hybridM(V, U, ihy):
    """hh_HybridM (OCFD_Schemes_1.f90:368-384)."""
    with np.errstate(all="ignore"):
        return np.where(ihy == 1, ud7lM(V, U), np.where(ihy == 2, weno7M(V), weno5M(V)))


def scheme_point(scheme, sign, V, U, ihy):
    """The interior scheme of a face, F+ (sign > 0) or F- (sign < 0)."""
    if scheme == SCH_OMP6:
        return omp6P(V) if sign > 0 else omp6M(V)
    if scheme == SCH_WENO7:
        return weno7P(V) if sign > 0 else weno7M(V)
    if scheme == SCH_WENO5:
        return weno5P(V) if sign > 0 else weno5M(V)
    if scheme == SCH_UD7L:
        return ud7lP(V, U) if sign > 0 else ud7lM(V, U)
    if scheme == SCH_HYBRID:
        return hybridP(V, U, ihy) if sign > 0 else hybridM(V, U, ihy)
    raise ValueError(f"scheme {scheme}")


def stencil_range(scheme):
    """(Ka1, Kb1, Ka2, Kb2) of set_parameters (OCFD_readpara.f90:288-315)."""
    if scheme == SCH_WENO5:
        return -2, 2, -1, 3
    if scheme == SCH_WENO7:
        return -3, 3, -2, 4
    return -3, 4, -3, 4


# ---------------------------------------------------------------------------
# flux-vector form: OCFD2d_flux1 / OCFD2d_flux2 over pencils (last axis)
def flux_pencils(f1d, sign, scheme, bound, sbound, U=None, ihy=None):
    """OCFD2d_flux1 (sign > 0) / OCFD2d_flux2 (sign < 0), OCFD_inviscous.f90:210-361.
    f1d: (..., n + 8) values of index 1-LAP..n+LAP; bound = Bound_index(1:2),
    sbound = Scheme_boundary(1:2) of the direction; ihy: (..., n + 1) hybrid
    indices of the faces.  Returns hh(0:n), shape (..., n + 1)."""
    n = f1d.shape[-1] - 2 * LAP
    Ka1, Kb1, Ka2, Kb2 = stencil_range(scheme)
    Ka, Kb = (Ka1, Kb1) if sign > 0 else (Ka2, Kb2)
    ib = 0 if (bound[0] == 0 or sbound[0] == -1) else -Ka + 1
    ie = n if (bound[1] == 0 or sbound[1] == -1) else n - Kb
    hh = np.zeros(f1d.shape[:-1] + (n + 1,))
    F = lambda i: f1d[..., i + LAP - 1]  # noqa: E731  Fortran index -> value

    def V_at(faces):
        idx = np.asarray(faces)
        return lambda s: f1d[..., idx + s + LAP - 1]

    faces = np.arange(ib, ie + 1)
    if len(faces):
        hy = None if ihy is None else ihy[..., faces]
        with np.errstate(all="ignore"):
            hh[..., faces] = scheme_point(scheme, sign, V_at(faces), U, hy)
    w5 = weno5P if sign > 0 else weno5M
    if bound[0] == 1:
        for i in range(0, -Ka + 1):
            if sbound[0] == 0:
                if sign > 0 and i in (0, 1):
                    hh[..., i] = (2.0 * F(1) + 5.0 * F(2) - F(3)) / 6.0
                elif sign < 0 and i == 0:
                    hh[..., i] = (2.0 * F(3) - 7.0 * F(2) + 11.0 * F(1)) / 6.0
                elif (sign > 0 and i == 2) or (sign < 0 and i == 1):
                    hh[..., i] = w5(V_at(i), DEL_LIFT)
                else:
                    hh[..., i] = w5(V_at(i))
            elif sbound[0] == 1:
                hh[..., i] = w5(V_at(i))
    if bound[1] == 1:
        for i in range(n - Kb + 1, n + 1):
            if sbound[1] == 0:
                if sign > 0 and i == n:
                    hh[..., i] = (2.0 * F(n - 2) - 7.0 * F(n - 1) + 11.0 * F(n)) / 6.0
                elif sign < 0 and i in (n, n - 1):
                    hh[..., i] = (2.0 * F(n) + 5.0 * F(n - 1) - F(n - 2)) / 6.0
                elif (sign > 0 and i == n - 1) or (sign < 0 and i == n - 2):
                    hh[..., i] = w5(V_at(i), DEL_RIGHT)
                else:
                    hh[..., i] = w5(V_at(i))
            elif sbound[1] == 1:
                hh[..., i] = w5(V_at(i))
    return hh


# ---------------------------------------------------------------------------
# flux splitting (OCFD_flux_split.f90), all points of the pencils at once
def split_sw(gamma, c1, d1, u1, v1, w1, A1, A2, A3):
    """split_Stager_Warming (OCFD_flux_split.f90:5-70): (fp, fm), each 5 arrays."""
    tmp1 = 2.0 * (gamma - 1.0)
    tmp3 = (3.0 - gamma) / (2.0 * (gamma - 1.0))
    ss = np.sqrt(A1 * A1 + A2 * A2 + A3 * A3)
    ss1 = 1.0 / ss
    ak1, ak2, ak3 = A1 * ss1, A2 * ss1, A3 * ss1
    vs = A1 * u1 + A2 * v1 + A3 * w1
    E1 = vs
    E2 = vs - c1 * ss
    E3 = vs + c1 * ss
    E1P = (E1 + np.abs(E1)) * 0.5
    E2P = (E2 + np.abs(E2)) * 0.5
    E3P = (E3 + np.abs(E3)) * 0.5
    E1M, E2M, E3M = E1 - E1P, E2 - E2P, E3 - E3P
    tmp0 = d1 / (2.0 * gamma)
    uc1, uc2 = u1 - c1 * ak1, u1 + c1 * ak1
    vc1, vc2 = v1 - c1 * ak2, v1 + c1 * ak2
    wc1, wc2 = w1 - c1 * ak3, w1 + c1 * ak3
    vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * 0.5
    vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * 0.5
    vv = (gamma - 1.0) * (u1 * u1 + v1 * v1 + w1 * w1)
    W2 = tmp3 * c1 * c1

    def part(E1x, E2x, E3x):
        return [tmp0 * (tmp1 * E1x + E2x + E3x),
                tmp0 * (tmp1 * E1x * u1 + E2x * uc1 + E3x * uc2),
                tmp0 * (tmp1 * E1x * v1 + E2x * vc1 + E3x * vc2),
                tmp0 * (tmp1 * E1x * w1 + E2x * wc1 + E3x * wc2),
                tmp0 * (E1x * vv + E2x * vvc1 + E3x * vvc2 + W2 * (E2x + E3x))]

    return part(E1P, E2P, E3P), part(E1M, E2M, E3M)


def split_llf(gamma, c1, d1, u1, v1, w1, A1, A2, A3):
    """split_Local_LaxFriedrichs (OCFD_flux_split.f90:73-104)."""
    tmp0 = 1.0 / gamma
    tmp1 = 1.0 / (gamma - 1.0)
    ss = np.sqrt(A1 * A1 + A2 * A2 + A3 * A3)
    un = A1 * u1 + A2 * v1 + A3 * w1
    lam = np.abs(un) + ss * c1
    p1 = tmp0 * d1 * c1 * c1
    E0 = tmp1 * p1 + 0.5 * d1 * (u1 * u1 + v1 * v1 + w1 * w1)
    h0 = E0 + p1
    fp = [0.5 * (d1 * un + lam * d1), 0.5 * (d1 * u1 * un + A1 * p1 + lam * d1 * u1),
          0.5 * (d1 * v1 * un + A2 * p1 + lam * d1 * v1), 0.5 * (d1 * w1 * un + A3 * p1 + lam * d1 * w1),
          0.5 * (h0 * un + lam * E0)]
    fm = [0.5 * (d1 * un - lam * d1), 0.5 * (d1 * u1 * un + A1 * p1 - lam * d1 * u1),
          0.5 * (d1 * v1 * un + A2 * p1 - lam * d1 * v1), 0.5 * (d1 * w1 * un + A3 * p1 - lam * d1 * w1),
          0.5 * (h0 * un - lam * E0)]
    return fp, fm


# ---------------------------------------------------------------------------
# the solver state the routines read (from the module globals of flow_data)
class State:
    """Parameters and haloed fields of one instance.  p: the ocfd_params fields
    used here (attributes of the same names); prims: d, u, v, w, T haloed;
    met: the 22 haloed metric arrays in the OCFD_M_* order; rh: Rhybrid."""

    def __init__(self, p, prims, met, rh=None):
        self.p = p
        self.nx, self.ny, self.nz = p.nx, p.ny, p.nz
        self.d, self.u, self.v, self.w, self.T = [np.asarray(a, dtype=np.float64) for a in prims]
        self.met = [np.asarray(a, dtype=np.float64) for a in met]
        self.rh = rh


# metric ids (OCFD_M_*): Axx..Azz 0-2, Akx..Ajac 3-12, Akx1..Asz1 13-21
M_AKX, M_AJAC, M_AKX1 = 3, 12, 13


def _pencils(a, d, nx, ny, nz):
    """Interior pencils of direction d with the whole halo along d: the
    direction moved to the last axis."""
    if d == 0:
        return a[LAP:LAP + nz, LAP:LAP + ny, :]
    if d == 1:
        return np.moveaxis(a[LAP:LAP + nz, :, LAP:LAP + nx], 1, -1)
    return np.moveaxis(a[:, LAP:LAP + ny, LAP:LAP + nx], 0, -1)


def _unpencil(x, d):
    """(…, n) in the moved layout back to (nz, ny, nx)."""
    if d == 0:
        return x
    if d == 1:
        return np.moveaxis(x, -1, 1)
    return np.moveaxis(x, -1, 0)


def set_hybrid_scheme(R0, th1, th2):
    """OCFD_SetHybrid.f90:2-15 (vectorised)."""
    return np.where(R0 <= th1, 1, np.where(R0 <= th2, 2, 3))


def _sweep_inputs(st, d):
    p = st.p
    nx, ny, nz = st.nx, st.ny, st.nz
    P = lambda a: _pencils(a, d, nx, ny, nz)  # noqa: E731
    cc = np.sqrt(st.T) / p.ma  # OCFD_inviscous.f90:64-70
    args = [P(cc), P(st.d), P(st.u), P(st.v), P(st.w)] + [P(st.met[M_AKX1 + 3 * d + q]) for q in range(3)]
    split = split_sw if p.flux_splitting == 1 else split_llf
    fp, fm = split(p.gamma, *args)
    ihy = None
    if p.scheme_invis == SCH_HYBRID:
        rh = P(st.rh)
        n = rh.shape[-1] - 2 * LAP
        r0 = np.maximum(rh[..., LAP - 1:LAP + n], rh[..., LAP:LAP + n + 1])  # Rhybrid(i), Rhybrid(i+1), i = 0..n
        ihy = set_hybrid_scheme(r0, p.hybrid_para[1], p.hybrid_para[2])
    return args, fp, fm, ihy


def _bounds(p, d):
    bi = (p.bound_index[2 * d], p.bound_index[2 * d + 1])
    sb = (p.scheme_boundary[2 * d], p.scheme_boundary[2 * d + 1])
    return bi, sb


def _hstep(p, d):
    return 1.0 / (p.hx, p.hy, p.hz)[d]


def _ud7l(p):
    return [p.ud7l[q] for q in range(8)]


def du_inviscous(st) -> np.ndarray:
    """du_inviscous (OCFD_inviscous.f90:53-203): du (5, nz, ny, nx)."""
    p = st.p
    du = None
    for d in range(3):
        _, fp, fm, ihy = _sweep_inputs(st, d)
        bi, sb = _bounds(p, d)
        h_1 = _hstep(p, d)
        part = []
        for m in range(5):
            h1 = flux_pencils(fp[m], +1, p.scheme_invis, bi, sb, _ud7l(p), ihy)
            h2 = flux_pencils(fm[m], -1, p.scheme_invis, bi, sb, _ud7l(p), ihy)
            part.append(_unpencil((h1[..., 1:] - h1[..., :-1] + h2[..., 1:] - h2[..., :-1]) * h_1, d))
        if d == 0:
            du = np.array(part)
        elif d == 1:
            du = du + np.array(part)
        else:
            ajac = st.met[M_AJAC][LAP:-LAP, LAP:-LAP, LAP:-LAP]
            du = -(du + np.array(part)) * ajac
    if p.if_mass_force == 1:  # OCFD_inviscous.f90:189-201
        du = _mass_force(st, du)
    return du


def _mass_force(st, du):
    p = st.p
    I = (slice(LAP, -LAP),) * 3
    d, u, v, w = st.d[I], st.u[I], st.v[I], st.w[I]
    F = [p.mass_force[q] for q in range(3)]
    du = du.copy()
    du[1] = du[1] + d * F[0]
    du[2] = du[2] + d * F[1]
    du[3] = du[3] + d * F[2]
    du[4] = du[4] + d * (u * F[0] + v * F[1] + w * F[2])
    return du


# ---------------------------------------------------------------------------
# characteristic form (OCFD_inviscous_character.f90)
def char_basis(gamma, u1, v1, w1, c1, a1, a2, a3):
    """The face state's L = S and R = S1 matrices (OCFD_inviscous_character.f90:
    216-248), each a 5x5 nested list of arrays."""
    ss = np.sqrt(a1 * a1 + a2 * a2 + a3 * a3)
    n1, n2, n3 = a1 / ss, a2 / ss, a3 / ss
    pick = np.abs(n3) <= np.abs(n2)
    ssa = np.sqrt(n1 * n1 + n2 * n2)
    ssb = np.sqrt(n1 * n1 + n3 * n3)
    zero = 0.0 * n1
    with np.errstate(all="ignore"):  # both branches are evaluated; the one not taken may divide by zero
        l1 = np.where(pick, -n2 / ssa, -n3 / ssb)
        l2 = np.where(pick, n1 / ssa, zero)
        l3 = np.where(pick, zero, n1 / ssb)
    m1 = n2 * l3 - n3 * l2
    m2 = n3 * l1 - n1 * l3
    m3 = n1 * l2 - n2 * l1
    un = u1 * n1 + v1 * n2 + w1 * n3
    ul = u1 * l1 + v1 * l2 + w1 * l3
    um = u1 * m1 + v1 * m2 + w1 * m3
    V2 = (u1 * u1 + v1 * v1 + w1 * w1) * 0.5
    KK = (gamma - 1.0) / (c1 * c1)
    KK1 = KK * 0.5
    X1 = 1.0 / (2.0 * c1)
    H = V2 + 1.0 / KK
    one = zero + 1.0
    S = [[1.0 - KK * V2, KK * u1, KK * v1, KK * w1, -KK],
         [-ul, l1, l2, l3, zero],
         [-um, m1, m2, m3, zero],
         [KK1 * V2 + X1 * un, -X1 * n1 - KK1 * u1, -X1 * n2 - KK1 * v1, -X1 * n3 - KK1 * w1, KK1],
         [KK1 * V2 - X1 * un, X1 * n1 - KK1 * u1, X1 * n2 - KK1 * v1, X1 * n3 - KK1 * w1, KK1]]
    S1 = [[one, zero, zero, one, one],
          [u1, l1, m1, u1 - c1 * n1, u1 + c1 * n1],
          [v1, l2, m2, v1 - c1 * n2, v1 + c1 * n2],
          [w1, l3, m3, w1 - c1 * n3, w1 + c1 * n3],
          [V2, ul, um, H - c1 * un, H + c1 * un]]
    return S, S1


def _flux_x(sign, scheme, V, U, ihy, faces, nn, Ka, Kb, bi, sb):
    """flux_x1 (sign > 0, :313-364) / flux_x2 (sign < 0, :367-416) of every face
    in `faces` (the last axis of V's values)."""
    inner = (((bi[0] == 0) | (faces > -Ka) | (sb[0] == -1)) & ((bi[1] == 0) | (faces <= nn - Kb) | (sb[1] == -1)))
    with np.errstate(all="ignore"):
        hh = scheme_point(scheme, sign, V, U, ihy)
    out = np.where(inner, hh, 0.0 * hh)
    w5 = weno5P if sign > 0 else weno5M
    for q, i in enumerate(faces):
        if inner[q]:
            continue
        Vq = lambda s, q=q: V(s)[..., q]  # noqa: E731
        if i <= -Ka and bi[0] == 1 and sb[0] != -1:
            if sb[0] == 0:
                if sign > 0 and i == 1:
                    val = (2.0 * Vq(0) + 5.0 * Vq(1) - Vq(2)) / 6.0
                elif (sign > 0 and i == 2) or (sign < 0 and i == 1):
                    val = w5(Vq, DEL_LIFT)
                else:
                    val = w5(Vq)
            else:
                val = w5(Vq)
        elif i > nn - Kb and bi[1] == 1 and sb[1] != -1:
            if sb[1] == 0:
                if sign < 0 and i == nn - 1:
                    val = (2.0 * Vq(1) + 5.0 * Vq(0) - Vq(-1)) / 6.0
                elif (sign > 0 and i == nn - 1) or (sign < 0 and i == nn - 2):
                    val = w5(Vq, DEL_RIGHT)
                else:
                    val = w5(Vq)
            else:
                val = w5(Vq)
        else:
            continue
        out[..., q] = val
    return out


def flux_charteric(p, d, args, fp, fm, ihy):
    """flux_charteric (OCFD_inviscous_character.f90:162-310) over pencils:
    hh (5, …, nn + 1)."""
    c1, d1, u1, v1, w1, A1, A2, A3 = args
    nn = c1.shape[-1] - 2 * LAP
    bi, sb = _bounds(p, d)
    Ka1, Kb1, Ka2, Kb2 = stencil_range(p.scheme_invis)
    ia = 0 if (bi[0] == 0 or sb[0] != 0) else 1
    ib = nn if (bi[1] == 0 or sb[1] != 0) else nn - 1
    faces = np.arange(ia, ib + 1)
    at = lambda a, s: a[..., faces + s + LAP - 1]  # noqa: E731  value at face index + s
    mean = lambda a: (at(a, 0) + at(a, 1)) * 0.5  # noqa: E731
    S, S1 = char_basis(p.gamma, mean(u1), mean(v1), mean(w1), mean(c1), mean(A1), mean(A2), mean(A3))
    hy = None if ihy is None else ihy[..., faces]
    linear = np.zeros(faces.shape, dtype=bool) if hy is None else (hy == 1)

    def projected(F, r, s):
        f = [at(F[m], s) for m in range(5)]
        return S[r][0] * f[0] + S[r][1] * f[1] + S[r][2] * f[2] + S[r][3] * f[3] + S[r][4] * f[4]

    U = _ud7l(p)
    h0 = []
    for r in range(5):
        Vp = lambda s, r=r: np.where(linear, at(fp[r], s), projected(fp, r, s))  # noqa: E731
        Vm = lambda s, r=r: np.where(linear, at(fm[r], s), projected(fm, r, s))  # noqa: E731
        h1 = _flux_x(+1, p.scheme_invis, Vp, U, hy, faces, nn, Ka1, Kb1, bi, sb)
        h2 = _flux_x(-1, p.scheme_invis, Vm, U, hy, faces, nn, Ka2, Kb2, bi, sb)
        h0.append(h1 + h2)
    hh = np.zeros((5,) + c1.shape[:-1] + (nn + 1,))
    for r in range(5):
        back = S1[r][0] * h0[0] + S1[r][1] * h0[1] + S1[r][2] * h0[2] + S1[r][3] * h0[3] + S1[r][4] * h0[4]
        hh[r][..., faces] = np.where(linear, h0[r], back)
    F = lambda a, i: a[..., i + LAP - 1]  # noqa: E731
    if bi[0] == 1 and sb[0] == 0:  # non-reflecting boundary faces, :295-309
        for m in range(5):
            hh[m][..., 0] = (2.0 * F(fp[m], 1) + 5.0 * F(fp[m], 2) - F(fp[m], 3) + 2.0 * F(fm[m], 3)
                             - 7.0 * F(fm[m], 2) + 11.0 * F(fm[m], 1)) / 6.0
    if bi[1] == 1 and sb[1] == 0:
        for m in range(5):
            hh[m][..., nn] = (2.0 * F(fp[m], nn - 2) - 7.0 * F(fp[m], nn - 1) + 11.0 * F(fp[m], nn)
                              + 2.0 * F(fm[m], nn) + 5.0 * F(fm[m], nn - 1) - F(fm[m], nn - 2)) / 6.0
    return hh


def du_inviscous_character(st) -> np.ndarray:
    """du_inviscous_Character (OCFD_inviscous_character.f90:3-159)."""
    p = st.p
    du = None
    for d in range(3):
        args, fp, fm, ihy = _sweep_inputs(st, d)
        hh = flux_charteric(p, d, args, fp, fm, ihy)
        h_1 = _hstep(p, d)
        part = np.array([_unpencil((hh[m][..., 1:] - hh[m][..., :-1]) * h_1, d) for m in range(5)])
        if d == 0:
            du = part
        elif d == 1:
            du = du + part
        else:
            ajac = st.met[M_AJAC][LAP:-LAP, LAP:-LAP, LAP:-LAP]
            du = -(du + part) * ajac
    if p.if_mass_force == 1:  # OCFD_inviscous_character.f90:145-156
        du = _mass_force(st, du)
    return du


# ---------------------------------------------------------------------------
# central derivatives and the viscous terms
def d0(p, f, d):
    """OCFD_dx0 / OCFD_dy0 / OCFD_dz0 (OCFD_dxyz_viscous.f90:3-239): the
    derivative along direction d of a haloed array, on the interior."""
    nx, ny, nz = p.nx, p.ny, p.nz
    h = (p.hx, p.hy, p.hz)[d]
    a1, a2, a3 = 1.0 / (60.0 * h), -3.0 / (20.0 * h), 3.0 / (4.0 * h)
    c1, c2, c3, c4 = 0.8 / h, -0.2 / h, 3.80952380952380952e-2 / h, -3.571428571428571428e-3 / h
    P = _pencils(f, d, nx, ny, nz)
    n = P.shape[-1] - 2 * LAP
    F = lambda s: P[..., LAP + s:LAP + s + n]  # noqa: E731  f(i + s), i = 1..n
    if p.scheme_vis == SCH_CD6:
        fx = a1 * (F(3) - F(-3)) + a2 * (F(2) - F(-2)) + a3 * (F(1) - F(-1))
    elif p.scheme_vis == SCH_CD8:
        fx = c1 * (F(1) - F(-1)) + c2 * (F(2) - F(-2)) + c3 * (F(3) - F(-3)) + c4 * (F(4) - F(-4))
    else:
        raise ValueError("only CD6 or CD8 in the viscous terms")
    fx = fx.copy()
    if p.iperiodic[d] == 0:
        G = lambda i: P[..., i + LAP - 1]  # noqa: E731
        fx[..., 0] = (-3.0 * G(1) + 4.0 * G(2) - G(3)) / (2.0 * h)
        fx[..., 1] = (G(3) - G(1)) / (2.0 * h)
        fx[..., 2] = (8.0 * (G(4) - G(2)) - (G(5) - G(1))) / (12.0 * h)
        if p.scheme_vis == SCH_CD8:
            fx[..., 3] = a1 * (G(7) - G(1)) + a2 * (G(6) - G(2)) + a3 * (G(5) - G(3))
        fx[..., n - 1] = (G(n - 2) - 4.0 * G(n - 1) + 3.0 * G(n)) / (2.0 * h)
        fx[..., n - 2] = (G(n) - G(n - 2)) / (2.0 * h)
        fx[..., n - 3] = (8.0 * (G(n - 1) - G(n - 3)) - (G(n) - G(n - 4))) / (12.0 * h)
        if p.scheme_vis == SCH_CD8:
            fx[..., n - 4] = a1 * (G(n) - G(n - 6)) + a2 * (G(n - 1) - G(n - 5)) + a3 * (G(n - 2) - G(n - 4))
    return _unpencil(fx, d)


def comput_amu(p, T):
    """comput_Amu (OCFD_viscous.f90:135-149) on the interior; T**3 = T*T*T."""
    Tsb = 110.4 / p.ref_amu_t0
    tmpR = 1.0 / p.re
    Ti = T[LAP:-LAP, LAP:-LAP, LAP:-LAP]
    return tmpR * (1.0 + Tsb) * np.sqrt(Ti * Ti * Ti) / (Tsb + Ti)


def _exchange_periodic(a, d):
    """exchange_boundary_x/y/z (OCFD_mpi.f90:183-233) on one rank, periodic
    direction d: the 4 halo layers each side wrap to the other end."""
    a = a.copy()
    ax = 2 - d
    n = a.shape[ax] - 2 * LAP
    sl = lambda s: tuple(s if q == ax else slice(None) for q in range(3))  # noqa: E731
    a[sl(slice(0, LAP))] = a[sl(slice(n, n + LAP))]
    a[sl(slice(n + LAP, n + 2 * LAP))] = a[sl(slice(LAP, 2 * LAP))]
    return a


def du_viscous(st, du) -> np.ndarray:
    """du_viscous (OCFD_viscous.f90:29-131): du (5, nz, ny, nx) with the viscous
    fluxes' divergence added to components 2..5."""
    p = st.p
    I = (slice(LAP, -LAP),) * 3
    M = [m[I] for m in st.met]
    amu = comput_amu(p, st.T)
    g = {}
    for name, f in (("u", st.u), ("v", st.v), ("w", st.w), ("T", st.T)):
        g[name] = [d0(p, f, d) for d in range(3)]  # ?k, ?i, ?s
    Akx, Aky, Akz, Aix, Aiy, Aiz, Asx, Asy, Asz = M[3:12]

    def cart(q, Ak, Ai, As):
        return g[q][0] * Ak + g[q][1] * Ai + g[q][2] * As

    ux, vx, wx, Tx = (cart(q, Akx, Aix, Asx) for q in "uvwT")
    uy, vy, wy, Ty = (cart(q, Aky, Aiy, Asy) for q in "uvwT")
    uz, vz, wz, Tz = (cart(q, Akz, Aiz, Asz) for q in "uvwT")
    div = ux + vy + wz
    Amu1 = amu
    Amuk = p.cp * amu / p.pr
    t23 = 2.0 / 3.0
    s11 = (2.0 * ux - t23 * div) * Amu1
    s22 = (2.0 * vy - t23 * div) * Amu1
    s33 = (2.0 * wz - t23 * div) * Amu1
    s12 = (uy + vx) * Amu1
    s13 = (uz + wx) * Amu1
    s23 = (vz + wy) * Amu1
    u, v, w = st.u[I], st.v[I], st.w[I]
    E1 = u * s11 + v * s12 + w * s13 + Amuk * Tx
    E2 = u * s12 + v * s22 + w * s23 + Amuk * Ty
    E3 = u * s13 + v * s23 + w * s33 + Amuk * Tz
    out = du.copy()
    nh = st.d.shape
    for m in range(4):
        divE = None
        for d in range(3):
            A1, A2, A3 = M[M_AKX1 + 3 * d], M[M_AKX1 + 3 * d + 1], M[M_AKX1 + 3 * d + 2]
            comp = (A1 * s11 + A2 * s12 + A3 * s13, A1 * s12 + A2 * s22 + A3 * s23,
                    A1 * s13 + A2 * s23 + A3 * s33, A1 * E1 + A2 * E2 + A3 * E3)[m]
            Ev = np.zeros(nh)
            Ev[I] = comp
            if p.iperiodic[d]:
                Ev = _exchange_periodic(Ev, d)
            dd = d0(p, Ev, d)
            divE = dd if divE is None else divE + dd
        out[m + 1] = out[m + 1] + divE * M[M_AJAC]
    return out
