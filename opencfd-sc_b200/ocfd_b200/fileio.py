"""The reference's on-disk formats, as Fortran unformatted sequential records
(each record framed by a 4-byte little-endian length before and after).

- Flow files ``opencfd.dat`` (restart input) and ``OCFD%08d.dat`` (output):
  read_flow_data / save_flow_data (OCFD_IO.f90:5-65) with the record layout of
  read_3d1 / write_3d1 (OCFD_IO_mpi.f90:132-282): record 1 holds
  (Istep: int32, tt: real64); then d, u, v, w, T follow, each as nz records of
  nx*ny real64 (one k-plane per record, i fastest).
- Grid file ``OCFD-grid.dat``: read_mesh1d (x(nx), y(ny), z(nz) as three
  records), read_mesh2d_plane (x(nx,ny), y(nx,ny), z(nz)) and read_mesh3d (x,
  y, z as nz plane records each) (OCFD_mesh.f90:187-283).

Arrays are numpy (nz, ny, nx) C-order, i.e. the Fortran (nx, ny, nz) layout.
"""
from __future__ import annotations

import numpy as np

from .params import GRID1D, GRID2D_PLANE, GRID3D

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


def write_grid(path: str, gridtype: int, x, y, z) -> None:
    """OCFD-grid.dat in the layout read_mesh* expect for this Iflag_Gridtype."""
    with open(path, "wb") as fh:
        if gridtype == GRID1D:
            for a in (x, y, z):
                _write_record(fh, np.ascontiguousarray(a, dtype="<f8").tobytes())
        elif gridtype == GRID2D_PLANE:
            _write_record(fh, np.ascontiguousarray(x, dtype="<f8").tobytes())
            _write_record(fh, np.ascontiguousarray(y, dtype="<f8").tobytes())
            _write_record(fh, np.ascontiguousarray(z, dtype="<f8").tobytes())
        elif gridtype == GRID3D:
            for a in (x, y, z):
                a = np.ascontiguousarray(a, dtype="<f8")
                for k in range(a.shape[0]):
                    _write_record(fh, a[k].tobytes())
        else:
            raise ValueError(f"Iflag_Gridtype {gridtype} has no grid file")


def read_grid(path: str, gridtype: int, nx: int, ny: int, nz: int):
    """Read OCFD-grid.dat and expand it to three (nz, ny, nx) coordinate arrays
    (what init_mesh passes on to the Jacobian)."""
    with open(path, "rb") as fh:
        if gridtype == GRID1D:
            x = np.frombuffer(_read_record(fh, nx * 8), dtype="<f8")
            y = np.frombuffer(_read_record(fh, ny * 8), dtype="<f8")
            z = np.frombuffer(_read_record(fh, nz * 8), dtype="<f8")
            Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
            return X.copy(), Y.copy(), Z.copy()
        if gridtype == GRID2D_PLANE:
            x2 = np.frombuffer(_read_record(fh, nx * ny * 8), dtype="<f8").reshape(ny, nx)
            y2 = np.frombuffer(_read_record(fh, nx * ny * 8), dtype="<f8").reshape(ny, nx)
            z1 = np.frombuffer(_read_record(fh, nz * 8), dtype="<f8")
            X = np.broadcast_to(x2, (nz, ny, nx)).copy()
            Y = np.broadcast_to(y2, (nz, ny, nx)).copy()
            Z = np.broadcast_to(z1[:, None, None], (nz, ny, nx)).copy()
            return X, Y, Z
        if gridtype == GRID3D:
            out = []
            for _ in range(3):
                a = np.empty((nz, ny, nx))
                for k in range(nz):
                    a[k] = np.frombuffer(_read_record(fh, nx * ny * 8), dtype="<f8").reshape(ny, nx)
                out.append(a)
            return tuple(out)
    raise ValueError(f"Iflag_Gridtype {gridtype} has no grid file")
