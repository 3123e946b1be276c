"""Host-side mirror of OpenCFD-SC's solver interface over the C ABI.

``Solver`` exposes the reference's hot-path subroutines under their own names
(exchange_boundary_xyz, comput_Rhybrid, du_inviscous, du_inviscous_Character,
du_viscous, OCFD_time_adv_RK3, comput_duvwT, OCFD_bc, filtering) with the same
argument meaning and call order as NS_solver (OCFD_NS_Solver.f90:21-78), plus
``step`` -- the fused, CUDA-graph-captured equivalent of one pass of the time
loop.  Errors are raised, matching the reference's print-and-stop: more than
10 negative-temperature points raise NegativeTemperatureStop.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .params import LAP, N_METRICS, PRECISION_MIXED, SCHEME_HYBRID, OcfdParams


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_parameters(p: OcfdParams, strict: bool = False) -> OcfdParams:
    """set_parameters (OCFD_readpara.f90:261-341) through the library."""
    q = p.copy()
    r = _lib.lib(strict).ocfd_set_parameters(C.byref(q))
    if r != 0:
        raise _lib.OcfdError(r, "unsupported configuration")
    return q


def footprint(p: OcfdParams) -> int:
    return int(_lib.lib().ocfd_gpu_footprint(C.byref(p)))


class Solver:
    def __init__(self, p: OcfdParams, device: int = 0, strict: bool = False):
        self.L = _lib.lib(strict)
        self.p = set_parameters(p, strict)
        self.nx, self.ny, self.nz = self.p.nx, self.p.ny, self.p.nz
        self.shape_h = (self.nz + 2 * LAP, self.ny + 2 * LAP, self.nx + 2 * LAP)
        self.shape5 = (5, self.nz, self.ny, self.nx)
        h = C.c_void_p()
        r = self.L.ocfd_gpu_create(C.byref(self.p), device, C.byref(h))
        if r != 0:
            raise _lib.OcfdError(r, f"ocfd_gpu_create failed (device {device})")
        self.h = h

    # ------------------------------------------------------------------ plumbing
    def _check(self, r: int, what: str):
        if r == 0:
            return
        msg = self.L.ocfd_gpu_last_error(self.h)
        msg = msg.decode() if msg else ""
        if r == _lib.OCFD_E_NEGT:
            raise _lib.NegativeTemperatureStop(r, msg or what)
        raise _lib.OcfdError(r, f"{what}: {msg}")

    def close(self):
        if getattr(self, "h", None):
            self.L.ocfd_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream(self) -> int:
        return int(self.L.ocfd_gpu_stream(self.h) or 0)

    def sync(self):
        self._check(self.L.ocfd_gpu_sync(self.h), "sync")

    # ------------------------------------------------------------------ init (init3d)
    def init_mesh(self, x=None, y=None, z=None, jac=None):
        """init_mesh (OCFD_mesh.f90:1-58) on the device; None -> mesh_gen('box').
        jac: the ten interior metric arrays Akx..Asz, Ajac of a GRID_AND_JACOBIAN3D
        grid file (comput_Jacobian3d is then skipped)."""
        if x is None:
            self._check(self.L.ocfd_gpu_init_mesh(self.h, None, None, None), "init_mesh")
            return
        xs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z)]
        if jac is None:
            self._check(self.L.ocfd_gpu_init_mesh(self.h, _dp(xs[0]), _dp(xs[1]), _dp(xs[2])), "init_mesh")
        else:
            js = [np.ascontiguousarray(a, dtype=np.float64) for a in jac]
            arr = (C.POINTER(C.c_double) * 10)(*[_dp(a) for a in js])
            self._check(self.L.ocfd_gpu_init_mesh_jacobian(self.h, _dp(xs[0]), _dp(xs[1]), _dp(xs[2]), arr),
                        "init_mesh")

    def upload_metrics(self, metrics):
        ms = [np.ascontiguousarray(m, dtype=np.float64) for m in metrics]
        arr = (C.POINTER(C.c_double) * 22)(*[_dp(m) for m in ms])
        self._check(self.L.ocfd_gpu_upload_metrics(self.h, arr), "upload_metrics")

    def set_bc_layer(self, data):
        """Boundary data of BC_BoundaryLayer / BC_SweptCorner (ocfd_b200.bclayer.BcLayerData)."""
        keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                for a in (data.inlet, data.upper, data.pertb, data.tm, data.fait)]
        ptr = lambda a: None if a is None or a.size == 0 else _dp(a)
        d = _lib.OcfdBcLayer(ptr(keep[0]), ptr(keep[1]), ptr(keep[2]), len(data.tm), data.beta, ptr(keep[3]),
                             ptr(keep[4]))
        self._check(self.L.ocfd_gpu_set_bc_layer(self.h, C.byref(d)), "set_bc_layer")

    def metric_zero_mask(self) -> int:
        """Bit m: metric m is identically +0.0 where the kernels read it (loads skipped)."""
        return int(self.L.ocfd_gpu_metric_zero_mask(self.h))

    def download_metrics(self):
        ms = [np.empty(self.shape_h) for _ in range(N_METRICS)]
        arr = (C.POINTER(C.c_double) * 22)(*[_dp(m) for m in ms])
        self._check(self.L.ocfd_gpu_download_metrics(self.h, arr), "download_metrics")
        return ms

    def init3d(self, prims, istep: int = 0, tt: float = 0.0):
        """init3d (OCFD_init.f90:1-20) from interior primitives + OCFD_bc (OCFD_NS_Solver.f90:15)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in prims]
        ptrs = (C.POINTER(C.c_double) * 5)(*[_dp(a) for a in arrs])
        self._check(self.L.ocfd_gpu_init3d(self.h, ptrs, istep, tt), "init3d")

    def upload_state(self, f=None, prims_haloed=None, istep=0, tt=0.0):
        fa = None if f is None else np.ascontiguousarray(f, dtype=np.float64)
        pp = None
        keep = []
        if prims_haloed is not None:
            keep = [np.ascontiguousarray(a, dtype=np.float64) for a in prims_haloed]
            pp = (C.POINTER(C.c_double) * 5)(*[_dp(a) for a in keep])
        self._check(self.L.ocfd_gpu_upload_state(self.h, None if fa is None else _dp(fa),
                                                 None if pp is None else C.cast(pp, C.c_void_p), istep, tt),
                    "upload_state")

    # ------------------------------------------------------------------ downloads
    def download_state(self):
        f = np.empty(self.shape5)
        prims = [np.empty(self.shape_h) for _ in range(5)]
        pp = (C.POINTER(C.c_double) * 5)(*[_dp(a) for a in prims])
        self._check(self.L.ocfd_gpu_download_state(self.h, _dp(f), C.cast(pp, C.c_void_p)), "download_state")
        return f, prims

    def download_f(self):
        f = np.empty(self.shape5)
        self._check(self.L.ocfd_gpu_download_state(self.h, _dp(f), None), "download_state")
        return f

    def download_du(self):
        du = np.empty(self.shape5)
        self._check(self.L.ocfd_gpu_download_du(self.h, _dp(du)), "download_du")
        return du

    def download_rhybrid(self):
        rh = np.empty(self.shape_h)
        self._check(self.L.ocfd_gpu_download_rhybrid(self.h, _dp(rh)), "download_rhybrid")
        return rh

    def time(self):
        i = C.c_int()
        t = C.c_double()
        self._check(self.L.ocfd_gpu_get_time(self.h, C.byref(i), C.byref(t)), "get_time")
        return i.value, t.value

    # ------------------------------------------------------------------ the reference's subroutines
    def save_fn(self):
        self._check(self.L.ocfd_gpu_save_fn(self.h), "save_fn")

    def exchange_boundary_xyz(self):
        """exchange_boundary_xyz(d,u,v,w,T) (OCFD_NS_Solver.f90:35-39)."""
        self._check(self.L.ocfd_gpu_halo_prims(self.h), "exchange_boundary_xyz")

    def comput_Rhybrid(self):
        self._check(self.L.ocfd_gpu_rhybrid(self.h), "comput_Rhybrid")

    def du_inviscous(self):
        self._check(self.L.ocfd_gpu_du_inviscous(self.h), "du_inviscous")

    def du_inviscous_Character(self):
        self._check(self.L.ocfd_gpu_du_inviscous_character(self.h), "du_inviscous_Character")

    def du_viscous(self):
        self._check(self.L.ocfd_gpu_du_viscous(self.h), "du_viscous")

    def OCFD_time_adv_RK3(self, krk: int):
        self._check(self.L.ocfd_gpu_rk3(self.h, krk), "OCFD_time_adv_RK3")

    def comput_duvwT(self) -> int:
        n = C.c_int()
        self._check(self.L.ocfd_gpu_duvwt(self.h, C.byref(n)), "comput_duvwT")
        return n.value

    def OCFD_bc(self):
        self._check(self.L.ocfd_gpu_bc(self.h), "OCFD_bc")

    def filtering(self):
        self._check(self.L.ocfd_gpu_filter(self.h), "filtering")

    def stage_step(self):
        """One pass of the time loop through the stage operators, in the
        reference's call order (OCFD_NS_Solver.f90:23-67)."""
        self.save_fn()
        for krk in (1, 2, 3):
            self.exchange_boundary_xyz()
            if krk == 1 and self.p.scheme_invis == SCHEME_HYBRID:
                self.comput_Rhybrid()
            if self.p.if_scheme_character == 0:
                self.du_inviscous()
            else:
                self.du_inviscous_Character()
            if self.p.if_viscous == 1:
                self.du_viscous()
            self.OCFD_time_adv_RK3(krk)
            self.comput_duvwT()
            self.OCFD_bc()
        self._check(self.L.ocfd_gpu_advance_clock(self.h), "advance_clock")
        self.filtering()

    def step(self, n: int = 1, sync: bool = True):
        """n time steps on the fused, graph-captured path."""
        self._check(self.L.ocfd_gpu_step(self.h, n, 1 if sync else 0), "step")

    def step_kernels(self) -> int:
        """Kernels one captured time step launches (-1 before the first captured step)."""
        return int(self.L.ocfd_gpu_step_kernels(self.h))

    PROFILE_GROUPS = ["sensor", "face_x", "face_y", "face_z", "visc_grad", "stage_tail", "negt_bc_halo", "step"]

    def profile_steps(self, n: int = 3) -> dict:
        """n eager steps with CUDA events around each kernel group (ms per step)."""
        ms = np.zeros(8)
        self._check(self.L.ocfd_gpu_profile_steps(self.h, n, _dp(ms)), "profile_steps")
        return dict(zip(self.PROFILE_GROUPS, ms.tolist()))

    # ------------------------------------------------------------------ diagnostics
    def show_flow_msg(self) -> np.ndarray:
        e = np.zeros(3)
        self._check(self.L.ocfd_gpu_show_flow_msg(self.h, _dp(e)), "show_flow_msg")
        return e

    def ana_box(self) -> np.ndarray:
        e = np.zeros(20)
        self._check(self.L.ocfd_gpu_ana_box(self.h, _dp(e)), "ana_box")
        return e

    def ana_q(self) -> np.ndarray:
        """ana_getQ: the Q criterion, (nz, ny, nx)."""
        q = np.empty((self.nz, self.ny, self.nx))
        self._check(self.L.ocfd_gpu_ana_q(self.h, _dp(q)), "ana_q")
        return q

    def ana_time_average(self):
        """ana_time_average: add the current d,u,v,w,T to the running means."""
        self._check(self.L.ocfd_gpu_ana_time_average(self.h), "ana_time_average")

    def download_average(self):
        """(means [d,u,v,w,T] each (nz, ny, nx), K_average, t_average)."""
        means = [np.empty((self.nz, self.ny, self.nx)) for _ in range(5)]
        pp = (C.POINTER(C.c_double) * 5)(*[_dp(a) for a in means])
        k = C.c_int()
        t = np.zeros(1)
        self._check(self.L.ocfd_gpu_download_average(self.h, C.cast(pp, C.c_void_p), C.byref(k), _dp(t)),
                    "download_average")
        return means, k.value, float(t[0])

    def upload_average(self, means, k_average: int, t_average: float):
        keep = [np.ascontiguousarray(a, dtype=np.float64) for a in means]
        pp = (C.POINTER(C.c_double) * 5)(*[_dp(a) for a in keep])
        self._check(self.L.ocfd_gpu_upload_average(self.h, C.cast(pp, C.c_void_p), k_average, t_average),
                    "upload_average")

    def ana_corner(self) -> np.ndarray:
        """Ana_corner: (3, nx) span averages u_t(j=2), T(j=2), p_wall."""
        out = np.empty(3 * self.nx)
        self._check(self.L.ocfd_gpu_ana_corner(self.h, _dp(out)), "ana_corner")
        return out.reshape(3, self.nx)

    def download_block(self, ib, ie, jb, je, kb, ke):
        """d,u,v,w,T of the interior box [ib,ie]x[jb,je]x[kb,ke] (1-based, inclusive),
        each (ke-kb+1, je-jb+1, ie-ib+1)."""
        shp = (ke - kb + 1, je - jb + 1, ie - ib + 1)
        out = [np.empty(shp) for _ in range(5)]
        pp = (C.POINTER(C.c_double) * 5)(*[_dp(a) for a in out])
        self._check(self.L.ocfd_gpu_download_block(self.h, ib, ie, jb, je, kb, ke, C.cast(pp, C.c_void_p)),
                    "download_block")
        return out

    @property
    def mixed(self) -> bool:
        return self.p.precision == PRECISION_MIXED


class Batch:
    """Several solver instances advanced together (ocfd_batch_*): one launch per
    kernel and RK stage for all of them when their configuration allows it (one
    persistent launch per stage for the flux-vector WENO7 and characteristic
    OMP6 forms), bit-identical to stepping each alone."""

    def __init__(self, members: list[Solver]):
        if not members:
            raise ValueError("empty batch")
        self.members = list(members)
        self.L = members[0].L
        hs = (C.c_void_p * len(members))(*[m.h for m in members])
        b = C.c_void_p()
        r = self.L.ocfd_batch_create(C.cast(hs, C.POINTER(C.c_void_p)), len(members), C.byref(b))
        if r != 0:
            raise _lib.OcfdError(r, "ocfd_batch_create failed")
        self.b = b

    def _check(self, r: int, what: str):
        if r == 0:
            return
        msg = self.L.ocfd_batch_last_error(self.b)
        msg = msg.decode() if msg else ""
        if r == _lib.OCFD_E_NEGT:
            raise _lib.NegativeTemperatureStop(r, msg or what)
        raise _lib.OcfdError(r, f"{what}: {msg}")

    def step(self, n: int = 1, sync: bool = True):
        self._check(self.L.ocfd_batch_step(self.b, n, 1 if sync else 0), "batch_step")

    def set_tiles(self, variants):
        v = (C.c_int * 3)(*variants)
        self._check(self.L.ocfd_batch_set_tiles(self.b, v), "batch_set_tiles")

    def set_persistent(self, on):
        """Launch mode where the persistent stage kernel exists: None (the
        default) keeps the faster of the two, timed on the first steps; True:
        one persistent launch per RK stage; False: one launch per kernel and
        stage."""
        v = -1 if on is None else (1 if on else 0)
        self._check(self.L.ocfd_batch_set_persistent(self.b, v), "batch_set_persistent")

    def mode_times(self):
        """Device ms of the two steps timed per launch mode (per kernel,
        persistent) by the launch-mode choice, or None before it ran."""
        ms = (C.c_float * 2)()
        if self.L.ocfd_batch_mode_times(self.b, ms) != 0:
            return None
        return float(ms[0]), float(ms[1])

    def mode(self) -> int:
        """0: members on their own graphs, 1: one batched launch per kernel and
        stage, 2: one persistent launch per stage."""
        r = self.L.ocfd_batch_mode(self.b)
        if r < 0:
            self._check(r, "batch_mode")
        return r

    def info(self):
        fused = C.c_int()
        v = (C.c_int * 3)()
        self._check(self.L.ocfd_batch_info(self.b, C.byref(fused), v), "batch_info")
        return bool(fused.value), list(v)

    def close(self):
        if getattr(self, "b", None):
            self.L.ocfd_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
