"""ctypes wrapper of the CPU oracle (test infrastructure only).

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg,
always as the checker.  Builds oracle/_build/liboracle.so on first use when a C
compiler is present.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
sys.path.insert(0, os.path.join(_ROOT, "opencfd-sc_b200"))
from ocfd_b200.params import LAP, N_METRICS, OcfdParams  # noqa: E402

LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

ORC_F, ORC_FN, ORC_DU, ORC_AMU, ORC_D, ORC_U, ORC_V, ORC_W, ORC_T, ORC_RHYBRID, ORC_METRIC0 = range(11)

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER(OcfdParams)
        dp = C.POINTER(C.c_double)
        L.orc_default_params.argtypes = [P]
        L.orc_set_parameters.argtypes = [P]
        L.orc_set_parameters.restype = C.c_int
        L.orc_create.argtypes = [P]
        L.orc_create.restype = C.c_void_p
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_array.argtypes = [C.c_void_p, C.c_int]
        L.orc_array.restype = dp
        L.orc_get_time.argtypes = [C.c_void_p, C.POINTER(C.c_int), dp]
        L.orc_set_time.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.orc_init_mesh.argtypes = [C.c_void_p, dp, dp, dp]
        L.orc_init_mesh_jacobian.argtypes = [C.c_void_p, dp, dp, dp, dp * 10]
        L.orc_init3d.argtypes = [C.c_void_p, dp * 5]
        for name in ["orc_halo_prims", "orc_comput_rhybrid", "orc_du_inviscous", "orc_du_inviscous_character",
                     "orc_du_viscous", "orc_bc", "orc_filtering"]:
            getattr(L, name).argtypes = [C.c_void_p]
        L.orc_exchange_xyz.argtypes = [C.c_void_p, dp]
        L.orc_rk3.argtypes = [C.c_void_p, C.c_int]
        L.orc_duvwt.argtypes = [C.c_void_p]
        L.orc_duvwt.restype = C.c_int
        L.orc_step.argtypes = [C.c_void_p]
        L.orc_step.restype = C.c_int
        L.orc_show_flow_msg.argtypes = [C.c_void_p, dp]
        L.orc_ana_box.argtypes = [C.c_void_p, dp]
        L.orc_flux1d.argtypes = [C.c_void_p, C.c_int, C.c_int, dp, C.c_int, C.POINTER(C.c_int), dp]
        L.orc_char_matrices.argtypes = [C.c_double, dp, dp, dp, dp]
        L.orc_d0.argtypes = [C.c_void_p, C.c_int, dp, dp]
        L.orc_ana_q.argtypes = [C.c_void_p, dp]
        L.orc_ana_time_average.argtypes = [C.c_void_p, dp, C.c_int]
        L.orc_ana_corner.argtypes = [C.c_void_p, dp]
        L.orc_set_bc_layer.argtypes = [C.c_void_p, dp, dp, dp, C.c_int, C.c_double, dp, dp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_parameters(p: OcfdParams) -> OcfdParams:
    q = p.copy()
    if lib().orc_set_parameters(C.byref(q)) != 0:
        raise ValueError("unsupported scheme")
    return q


class Oracle:
    """Single-rank restatement of the reference solver state (flow_data etc.)."""

    def __init__(self, p: OcfdParams):
        self.p = set_parameters(p)
        self.h = lib().orc_create(C.byref(self.p))
        self.nx, self.ny, self.nz = self.p.nx, self.p.ny, self.p.nz
        self.shape_h = (self.nz + 2 * LAP, self.ny + 2 * LAP, self.nx + 2 * LAP)  # C view of Fortran order

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # ---- views (numpy arrays in C order = Fortran order reversed: [m][k][j][i])
    def _view(self, id_, shape):
        ptr = lib().orc_array(self.h, id_)
        n = int(np.prod(shape))
        return np.ctypeslib.as_array(ptr, shape=(n,)).reshape(shape)

    @property
    def f(self):
        return self._view(ORC_F, (5, self.nz, self.ny, self.nx))

    @property
    def fn(self):
        return self._view(ORC_FN, (5, self.nz, self.ny, self.nx))

    @property
    def du(self):
        return self._view(ORC_DU, (5, self.nz, self.ny, self.nx))

    def prim(self, q: int):
        return self._view(ORC_D + q, self.shape_h)

    @property
    def rhybrid(self):
        return self._view(ORC_RHYBRID, self.shape_h)

    def metric(self, m: int):
        return self._view(ORC_METRIC0 + m, self.shape_h)

    def metrics(self):
        return [self.metric(m) for m in range(N_METRICS)]

    # ---- operations
    def init_mesh(self, x=None, y=None, z=None, jac=None):
        if x is None:
            lib().orc_init_mesh(self.h, None, None, None)
            return
        xs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z)]
        if jac is None:
            lib().orc_init_mesh(self.h, _dp(xs[0]), _dp(xs[1]), _dp(xs[2]))
        else:
            js = [np.ascontiguousarray(a, dtype=np.float64) for a in jac]
            lib().orc_init_mesh_jacobian(self.h, _dp(xs[0]), _dp(xs[1]), _dp(xs[2]),
                                         (C.POINTER(C.c_double) * 10)(*[_dp(a) for a in js]))

    def init3d(self, prims):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in prims]
        ptrs = (C.POINTER(C.c_double) * 5)(*[_dp(a) for a in arrs])
        lib().orc_init3d(self.h, ptrs)

    def set_time(self, istep, tt):
        lib().orc_set_time(self.h, istep, tt)

    def time(self):
        i = C.c_int()
        t = C.c_double()
        lib().orc_get_time(self.h, C.byref(i), C.byref(t))
        return i.value, t.value

    def halo_prims(self):
        lib().orc_halo_prims(self.h)

    def comput_rhybrid(self):
        lib().orc_comput_rhybrid(self.h)

    def du_inviscous(self):
        lib().orc_du_inviscous(self.h)

    def du_inviscous_character(self):
        lib().orc_du_inviscous_character(self.h)

    def du_viscous(self):
        lib().orc_du_viscous(self.h)

    def rk3(self, krk):
        lib().orc_rk3(self.h, krk)

    def duvwt(self):
        return lib().orc_duvwt(self.h)

    def bc(self):
        lib().orc_bc(self.h)

    def set_bc_layer(self, data):
        """BC_BoundaryLayer / BC_SweptCorner boundary data (ocfd_b200.bclayer.BcLayerData)."""
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                for a in (data.inlet, data.upper, data.pertb)]
        tm = np.ascontiguousarray(data.tm, dtype=np.float64)
        fait = np.ascontiguousarray(data.fait, dtype=np.float64)
        self._bl = (arrs, tm, fait)
        lib().orc_set_bc_layer(self.h, *[None if a is None else _dp(a) for a in arrs], len(tm), data.beta,
                               _dp(tm) if len(tm) else None, _dp(fait) if len(fait) else None)

    def filtering(self):
        lib().orc_filtering(self.h)

    def step(self, n=1):
        for _ in range(n):
            if lib().orc_step(self.h) != 0:
                raise RuntimeError("Number of Negative Temperature Points > Limit, STOP !")

    def show_flow_msg(self):
        e = np.zeros(3)
        lib().orc_show_flow_msg(self.h, _dp(e))
        return e

    def ana_q(self):
        q = np.empty((self.p.nz, self.p.ny, self.p.nx))
        lib().orc_ana_q(self.h, _dp(q))
        return q

    def ana_time_average(self, mean, k_average: int):
        """mean (5, nz, ny, nx) updated in place with the current d,u,v,w,T."""
        lib().orc_ana_time_average(self.h, _dp(mean), k_average)

    def ana_corner(self):
        out = np.empty(3 * self.p.nx)
        lib().orc_ana_corner(self.h, _dp(out))
        return out.reshape(3, self.p.nx)

    def ana_box(self):
        e = np.zeros(20)
        lib().orc_ana_box(self.h, _dp(e))
        return e

    def flux1d(self, f1d, sign, dir_=0, scm=None):
        n = len(f1d) - 2 * LAP
        f1d = np.ascontiguousarray(f1d, dtype=np.float64)
        hh = np.zeros(n + 1)
        sc = np.zeros(n + 1, dtype=np.int32) if scm is None else np.ascontiguousarray(scm, dtype=np.int32)
        lib().orc_flux1d(self.h, dir_, sign, _dp(f1d), n, sc.ctypes.data_as(C.POINTER(C.c_int)), _dp(hh))
        return hh

    def d0(self, dir_, fh):
        fh = np.ascontiguousarray(fh, dtype=np.float64)
        out = np.zeros((self.nz, self.ny, self.nx))
        lib().orc_d0(self.h, dir_, _dp(fh), _dp(out))
        return out


def char_matrices(gamma, uvwc, a123):
    S = np.zeros(25)
    S1 = np.zeros(25)
    u = np.ascontiguousarray(uvwc, dtype=np.float64)
    a = np.ascontiguousarray(a123, dtype=np.float64)
    lib().orc_char_matrices(gamma, _dp(u), _dp(a), _dp(S), _dp(S1))
    return S.reshape(5, 5), S1.reshape(5, 5)
