"""The reference's on-disk formats, as Fortran unformatted sequential records
(each record framed by a 4-byte little-endian length before and after).

- Flow files ``opencfd.dat`` (restart input) and ``OCFD%08d.dat`` (output):
  read_flow_data / save_flow_data (OCFD_IO.f90:5-65) with the record layout of
  read_3d1 / write_3d1 (OCFD_IO_mpi.f90:132-282): record 1 holds
  (Istep: int32, tt: real64); then d, u, v, w, T follow, each as nz records of
  nx*ny real64 (one k-plane per record, i fastest).
- Grid file ``OCFD-grid.dat``: read_mesh1d (x(nx), y(ny), z(nz) as three
  records), read_mesh2d_plane (x(nx,ny), y(nx,ny), z(nz)),
  read_mesh2d_AxialSymm (x(nx,ny), R(nx,ny), seta(nz); y = R cos(seta),
  z = R sin(seta)) and read_mesh3d (x, y, z as nz plane records each, followed
  for Iflag_Gridtype 31 by Akx, Aky, Akz, Aix, Aiy, Aiz, Asx, Asy, Asz, Ajac in
  the same layout) (OCFD_mesh.f90:187-317).

Arrays are numpy (nz, ny, nx) C-order, i.e. the Fortran (nx, ny, nz) layout.
"""
from __future__ import annotations

import numpy as np

from .params import GRID1D, GRID2D_AXIAL_SYMM, GRID2D_PLANE, GRID3D, GRID_AND_JACOBIAN3D

_MARK = np.dtype("<i4")


def _write_record(fh, payload: bytes) -> None:
    n = np.array([len(payload)], dtype=_MARK).tobytes()
    fh.write(n)
    fh.write(payload)
    fh.write(n)


def _read_record(fh, nbytes: int | None = None) -> bytes:
    head = fh.read(4)
    if len(head) != 4:
        raise EOFError("truncated record marker")
    n = int(np.frombuffer(head, dtype=_MARK)[0])
    if nbytes is not None and n != nbytes:
        raise ValueError(f"record of {n} bytes where {nbytes} were expected")
    body = fh.read(n)
    tail = fh.read(4)
    if len(body) != n or len(tail) != 4 or int(np.frombuffer(tail, dtype=_MARK)[0]) != n:
        raise ValueError("corrupt record framing")
    return body


def write_flow(path: str, istep: int, tt: float, prims) -> None:
    """save_flow_data: prims = [d, u, v, w, T], each (nz, ny, nx) float64."""
    with open(path, "wb") as fh:
        _write_record(fh, np.array([istep], dtype="<i4").tobytes() + np.array([tt], dtype="<f8").tobytes())
        for q in prims:
            q = np.ascontiguousarray(q, dtype="<f8")
            for k in range(q.shape[0]):
                _write_record(fh, q[k].tobytes())


def read_flow(path: str, nx: int, ny: int, nz: int):
    """read_flow_data: returns (istep, tt, [d, u, v, w, T]) with (nz, ny, nx) arrays."""
    with open(path, "rb") as fh:
        r1 = _read_record(fh, 12)
        istep = int(np.frombuffer(r1[:4], dtype="<i4")[0])
        tt = float(np.frombuffer(r1[4:], dtype="<f8")[0])
        prims = []
        for _ in range(5):
            q = np.empty((nz, ny, nx))
            for k in range(nz):
                q[k] = np.frombuffer(_read_record(fh, nx * ny * 8), dtype="<f8").reshape(ny, nx)
            prims.append(q)
    return istep, tt, prims


def _write_planes(fh, a) -> None:
    a = np.ascontiguousarray(a, dtype="<f8")
    for k in range(a.shape[0]):
        _write_record(fh, a[k].tobytes())


def _read_planes(fh, nx: int, ny: int, nz: int) -> np.ndarray:
    a = np.empty((nz, ny, nx))
    for k in range(nz):
        a[k] = np.frombuffer(_read_record(fh, nx * ny * 8), dtype="<f8").reshape(ny, nx)
    return a


def write_grid(path: str, gridtype: int, x, y, z, jac=None) -> None:
    """OCFD-grid.dat in the layout read_mesh* expect for this Iflag_Gridtype.
    GRID1D: x(nx), y(ny), z(nz); GRID2D_PLANE: x, y (ny, nx) and z(nz);
    GRID2D_AXIAL_SYMM: x, R (ny, nx) and seta(nz); GRID3D: x, y, z (nz, ny, nx);
    GRID_AND_JACOBIAN3D: the same plus jac, the ten (nz, ny, nx) arrays Akx, Aky,
    Akz, Aix, Aiy, Aiz, Asx, Asy, Asz, Ajac."""
    with open(path, "wb") as fh:
        if gridtype in (GRID1D, GRID2D_PLANE, GRID2D_AXIAL_SYMM):
            for a in (x, y, z):
                _write_record(fh, np.ascontiguousarray(a, dtype="<f8").tobytes())
        elif gridtype in (GRID3D, GRID_AND_JACOBIAN3D):
            for a in (x, y, z):
                _write_planes(fh, a)
            if gridtype == GRID_AND_JACOBIAN3D:
                if jac is None or len(jac) != 10:
                    raise ValueError("Iflag_Gridtype 31 needs the ten metric / Jacobian arrays")
                for a in jac:
                    _write_planes(fh, a)
        else:
            raise ValueError(f"Iflag_Gridtype {gridtype} has no grid file")


def read_grid(path: str, gridtype: int, nx: int, ny: int, nz: int):
    """Read OCFD-grid.dat and expand it to three (nz, ny, nx) coordinate arrays
    (what init_mesh passes on to the Jacobian); for GRID_AND_JACOBIAN3D a fourth
    item, the list of the ten metric / Jacobian arrays, follows."""
    with open(path, "rb") as fh:
        if gridtype == GRID1D:
            x = np.frombuffer(_read_record(fh, nx * 8), dtype="<f8")
            y = np.frombuffer(_read_record(fh, ny * 8), dtype="<f8")
            z = np.frombuffer(_read_record(fh, nz * 8), dtype="<f8")
            Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
            return X.copy(), Y.copy(), Z.copy()
        if gridtype in (GRID2D_PLANE, GRID2D_AXIAL_SYMM):
            x2 = np.frombuffer(_read_record(fh, nx * ny * 8), dtype="<f8").reshape(ny, nx)
            y2 = np.frombuffer(_read_record(fh, nx * ny * 8), dtype="<f8").reshape(ny, nx)
            z1 = np.frombuffer(_read_record(fh, nz * 8), dtype="<f8")
            X = np.broadcast_to(x2, (nz, ny, nx)).copy()
            if gridtype == GRID2D_PLANE:
                Y = np.broadcast_to(y2, (nz, ny, nx)).copy()
                Z = np.broadcast_to(z1[:, None, None], (nz, ny, nx)).copy()
            else:
                # read_mesh2d_AxialSymm (OCFD_mesh.f90:286-317): y horizontal, z up,
                # seta the angle from the y axis
                Y = y2[None, :, :] * np.cos(z1)[:, None, None]
                Z = y2[None, :, :] * np.sin(z1)[:, None, None]
            return X, Y, Z
        if gridtype in (GRID3D, GRID_AND_JACOBIAN3D):
            out = [_read_planes(fh, nx, ny, nz) for _ in range(3)]
            if gridtype == GRID3D:
                return tuple(out)
            jac = [_read_planes(fh, nx, ny, nz) for _ in range(10)]
            return out[0], out[1], out[2], jac
    raise ValueError(f"Iflag_Gridtype {gridtype} has no grid file")
