"""Host side of BC_BoundaryLayer and BC_SweptCorner (OCFD_BC_Boundarylayers.f90):
the boundary data the reference builds at its first BC call, in the layout of
ocfd_gpu_set_bc_layer.

- read_profile_1d / read_plane_2d: the inlet and upper-boundary data files of
  init_bcdata_boundarylayer (:171-270): flow1d-inlet.dat / flow1d-upper.dat
  (formatted: one header line, then "coordinate d u v T" per point, w = 0) and
  flow2d-inlet.dat / flow2d-upper.dat (unformatted: five records d,u,v,w,T).
- wall_perturbation: init_bc_wall_perturbation (:313-400), the wall
  blowing/suction shape (type 1: multi-wavenumber, Rai, AIAA 95-0583; type 2:
  random).
- time_factor: the amplitudes and phases of get_ht_multifrequancy (:404-440).

The reference draws its random phases with Fortran's random_number; here a
seeded numpy generator draws them in the same order (wall phases, then time
phases), so a run is reproducible but not the same draw as a Fortran run.

Arrays are numpy C-order with the Fortran index order reversed: inlet (5, nz, ny),
upper (5, nz, nx), wall shape (nz, nx).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import fileio

PI = 3.14159265358979  # the constant of OCFD_BC_Boundarylayers.f90:319,410


@dataclass
class BcLayerData:
    inlet: np.ndarray | None = None   # (5, nz, ny)
    upper: np.ndarray | None = None   # (5, nz, nx)
    pertb: np.ndarray | None = None   # (nz, nx)
    beta: float = 0.0                 # base frequency of the time factor (<= 0: factor 1)
    tm: np.ndarray = field(default_factory=lambda: np.zeros(0))
    fait: np.ndarray = field(default_factory=lambda: np.zeros(0))


def read_profile_1d(path: str, n: int) -> np.ndarray:
    """flow1d-*.dat: header line, then n lines "coordinate d u v T" -> (n, 5) d,u,v,w=0,T."""
    with open(path) as fh:
        fh.readline()
        rows = [list(map(lambda t: float(t.replace("d", "e").replace("D", "e")), fh.readline().split()))
                for _ in range(n)]
    a = np.asarray(rows)
    out = np.zeros((n, 5))
    out[:, 0:3] = a[:, 1:4]
    out[:, 4] = a[:, 4]
    return out


def write_profile_1d(path: str, coord, prof) -> None:
    """Write a flow1d-*.dat file (prof (n, 5) d,u,v,w,T; w is not stored)."""
    with open(path, "w") as fh:
        fh.write("variables = coordinate, d, u, v, T\n")
        for c, q in zip(coord, prof):
            fh.write(f"{c:.17e} {q[0]:.17e} {q[1]:.17e} {q[2]:.17e} {q[4]:.17e}\n")


def read_plane_2d(path: str, n1: int, n2: int) -> np.ndarray:
    """flow2d-*.dat: five unformatted records of (n1, n2) -> (5, n2, n1)."""
    out = np.empty((5, n2, n1))
    with open(path, "rb") as fh:
        for m in range(5):
            out[m] = np.frombuffer(fileio._read_record(fh, n1 * n2 * 8), dtype="<f8").reshape(n2, n1)
    return out


def write_plane_2d(path: str, plane) -> None:
    with open(path, "wb") as fh:
        for m in range(5):
            fileio._write_record(fh, np.ascontiguousarray(plane[m], dtype="<f8").tobytes())


def inlet_from_profile(prof, nz: int) -> np.ndarray:
    """(ny, 5) profile -> (5, nz, ny), the same for every k (BcData_inlet = 1)."""
    prof = np.asarray(prof, dtype=np.float64)
    return np.ascontiguousarray(np.broadcast_to(prof.T[:, None, :], (5, nz, prof.shape[0])))


def upper_from_profile(prof, nz: int) -> np.ndarray:
    """(nx, 5) profile -> (5, nz, nx) (BcData_upper = 1)."""
    return inlet_from_profile(prof, nz)


def wall_perturbation(kind: int, x_wall, z_wall, xbegin: float, xend: float, mz: int, zl: float,
                      rng: np.random.Generator) -> np.ndarray:
    """init_bc_wall_perturbation (:313-400) on the wall coordinates x_wall, z_wall
    (nz, nx) (Axx, Azz at j = 1)."""
    x_wall = np.asarray(x_wall, dtype=np.float64)
    z_wall = np.asarray(z_wall, dtype=np.float64)
    out = np.zeros_like(x_wall)
    if kind == 1:
        faiz = np.zeros(max(mz, 0))
        zlw = np.zeros(max(mz, 0))
        if mz > 0:
            ztmp = 0.0
            for k in range(mz):
                faiz[k] = rng.random()
                zlw[k] = 1.0 if k == 0 else zlw[k - 1] / 1.25
                ztmp = ztmp + zlw[k]
            zlw = zlw / ztmp
        nz, nx = x_wall.shape
        for k in range(nz):
            for i in range(nx):
                x = x_wall[k, i]
                if xbegin <= x <= xend:
                    seta = 2.0 * PI * (x - xbegin) / (xend - xbegin)
                    fx = 4.0 / math.sqrt(27.0) * math.sin(seta) * (1.0 - math.cos(seta))
                else:
                    fx = 0.0
                seta = z_wall[k, i] / zl
                if mz > 0:
                    gz = 0.0
                    for m in range(1, mz + 1):
                        gz = gz + zlw[m - 1] * math.sin(2.0 * PI * m * (seta + faiz[m - 1]))
                elif mz == 0:
                    gz = 1.0
                else:
                    gz = math.sin(-2.0 * PI * mz * seta)
                out[k, i] = fx * gz
    elif kind == 2:
        nz, nx = x_wall.shape
        for k in range(nz):
            for i in range(nx):
                if xbegin <= x_wall[k, i] <= xend:
                    out[k, i] = 2.0 * (rng.random() - 0.5)
    return out


def time_factor(mt: int, rng: np.random.Generator):
    """Amplitudes TM (1, 1/1.25, ... normalised) and random phases of
    get_ht_multifrequancy (:404-432)."""
    tm = np.zeros(max(mt, 0))
    fait = np.zeros(max(mt, 0))
    t = 0.0
    for k in range(mt):
        fait[k] = rng.random()
        tm[k] = 1.0 if k == 0 else tm[k - 1] / 1.25
        t = t + tm[k]
    if mt > 0:
        tm = tm / t
    return tm, fait


def boundary_layer_bc_para(p, inlet=1, upper=0, nonref=0, outlet=2, tw=-1.0, dis_type=0, amp=0.0, xbegin=0.0,
                           xend=1.0, mt=0, mz=0, zl=1.0, freq=0.0):
    """BC_Para(1:14) of ocfd_bc_BoundaryLayer (:27-44)."""
    vals = [inlet, upper, nonref, outlet, tw, 0.0, dis_type, amp, xbegin, xend, mt, mz, zl, freq]
    for q, v in enumerate(vals):
        p.bc_para[q] = float(v)
    return p


def swept_corner_bc_para(p, outlet=2, tw=-1.0, wall_zl=1.0, dis_type=0, amp=0.0, xbegin=0.0, xend=1.0, mt=0, mz=0,
                         freq=0.0, z1=1, z2=1):
    """BC_Para(1:12) of ocfd_bc_swept_corner (:454-470)."""
    vals = [outlet, tw, wall_zl, dis_type, amp, xbegin, xend, mt, mz, freq, z1, z2]
    for q, v in enumerate(vals):
        p.bc_para[q] = float(v)
    return p
