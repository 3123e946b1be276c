"""Host side of OCFD_analysis (OCFD_ANA.f90:3-31): the ANA_Para schedule of the
deck and the reference's output files, with the computation on the device.

ANA_Para(1, m) is the analysis code, ANA_Para(2, m) its step interval and
ANA_Para(3:52, m) its data.  Codes (OCFD_parameters.f90:36-37):
  100 ana_time_average  running means of d,u,v,w,T; restart from
                        opencfd.dat.average; every ana_data(1) steps
                        OCFD%08d.dat.average (record (K_average, t_average),
                        then d,u,v,w,T as nz records of nx*ny)
  101 ana_getQ          Q-%07d.dat (nz records of nx*ny)
  102 ana_box            statistics.dat row (appended, formatted)
  103 ana_savedata       planes / points / blocks (OCFD_ANA_savedata.f90),
                        appended records
  104 Ana_corner         WallUtp-log.dat (appended: (Istep, tt), then
                        u_t, T, p_w as one record)
"""
from __future__ import annotations

import os
import re

import numpy as np

from . import fileio
from .params import _num, _values

ANA_TIME_AVERAGE, ANA_Q, ANA_BOX, ANA_SAVEDATA, ANA_CORNER, ANA_USER = 100, 101, 102, 103, 104, 99


def read_analysis(path_or_text: str, is_text: bool = False):
    """ANA_Number and ANA_Para(100, 10) of the namelist /control_opencfd/
    (OCFD_readpara.f90:12,21,58-59) -> list of (code, interval, data[50])."""
    text = path_or_text if is_text else open(path_or_text).read()
    m = re.search(r"[&$]control_opencfd(.*?)(?:[&$]end|/\s*$)", text, re.S | re.I)
    if not m:
        raise ValueError("namelist /control_opencfd/ not found")
    body = "\n".join(line.split("!")[0] for line in m.group(1).splitlines())
    number = 0
    para = np.zeros(1000)  # ANA_Para(100, 10) in Fortran (column-major) order
    parts = re.split(r"([A-Za-z_][A-Za-z0-9_]*(?:\([^)]*\))?)\s*=", body)
    for i in range(1, len(parts) - 1, 2):
        key, vals = parts[i].strip().lower(), _values(parts[i + 1])
        base = re.sub(r"\(.*\)", "", key)
        sub = re.search(r"\(([^)]*)\)", key)
        if base == "ana_number":
            number = int(_num(vals[0]))
        elif base == "ana_para":
            start = 0
            if sub:
                ix = [x.strip() for x in sub.group(1).split(",")]
                r0 = int(ix[0].split(":")[0]) - 1 if ix[0] not in ("", ":") else 0
                c0 = int(ix[1].split(":")[0]) - 1 if len(ix) > 1 and ix[1] not in ("", ":") else 0
                start = r0 + 100 * c0
            for c, v in enumerate(vals):
                para[start + c] = _num(v)
    if number > 10:
        raise ValueError("ANA_Number and NFiltering should <=10")
    cols = para.reshape(10, 100)
    return [(int(round(cols[q, 0])), int(round(cols[q, 1])), cols[q, 2:52].copy()) for q in range(number)]


def fortran_e(x: float, w: int = 20, d: int = 13) -> str:
    """Fortran Ew.dE2 edit descriptor: 0.ddd...E+xx, right-aligned in w columns."""
    if x == 0.0:
        body = "0." + "0" * d + "E+00"
    else:
        mant, ex = f"{abs(x):.{d - 1}E}".split("E")
        digits = mant.replace(".", "")
        e = int(ex) + 1
        body = f"0.{digits}E{'+' if e >= 0 else '-'}{abs(e):02d}"
        if x < 0:
            body = "-" + body
    return body.rjust(w)


class Analysis:
    """OCFD_analysis for one solver instance, writing into `outdir`."""

    def __init__(self, solver, entries, outdir: str = "."):
        self.s = solver
        self.entries = entries
        self.outdir = outdir
        self._avg_started = False

    def _path(self, name):
        return os.path.join(self.outdir, name)

    def run(self):
        """OCFD_analysis after a step: every entry whose interval divides Istep."""
        istep, tt = self.s.time()
        for code, every, data in self.entries:
            if every <= 0 or istep % every != 0:
                continue
            if code == ANA_TIME_AVERAGE:
                self.time_average(istep, data)
            elif code == ANA_Q:
                q = self.s.ana_q()
                with open(self._path(f"Q-{istep:07d}.dat"), "wb") as fh:
                    for k in range(q.shape[0]):
                        fileio._write_record(fh, np.ascontiguousarray(q[k]).tobytes())
            elif code == ANA_BOX:
                row = self.s.ana_box()
                with open(self._path("statistics.dat"), "a") as fh:
                    fh.write("".join(fortran_e(x) for x in row) + "\n")  # '(20(E20.13E2))', :307
            elif code == ANA_SAVEDATA:
                self.savedata(istep, tt, data)
            elif code == ANA_CORNER:
                out = self.s.ana_corner()
                with open(self._path("WallUtp-log.dat"), "ab") as fh:
                    fileio._write_record(fh, np.array([istep], "<i4").tobytes() + np.array([tt], "<f8").tobytes())
                    fileio._write_record(fh, np.ascontiguousarray(out, dtype="<f8").tobytes())
            else:
                raise ValueError(f"analysis code {code} is not supported")

    def time_average(self, istep, data):
        s = self.s
        if not self._avg_started:
            self._avg_started = True
            path = self._path("opencfd.dat.average")
            if os.path.exists(path):
                with open(path, "rb") as fh:
                    r1 = fileio._read_record(fh, 12)
                    k_avg = int(np.frombuffer(r1[:4], "<i4")[0])
                    t_avg = float(np.frombuffer(r1[4:], "<f8")[0])
                    means = []
                    for _ in range(5):
                        a = np.empty((s.nz, s.ny, s.nx))
                        for k in range(s.nz):
                            a[k] = np.frombuffer(fileio._read_record(fh, s.nx * s.ny * 8), "<f8").reshape(s.ny, s.nx)
                        means.append(a)
                s.upload_average(means, k_avg, t_avg)
        s.ana_time_average()
        every_save = int(round(data[0]))
        if every_save > 0 and istep % every_save == 0:
            means, k_avg, t_avg = s.download_average()
            with open(self._path(f"OCFD{istep:08d}.dat.average"), "wb") as fh:
                fileio._write_record(fh, np.array([k_avg], "<i4").tobytes() + np.array([t_avg], "<f8").tobytes())
                for a in means:
                    for k in range(a.shape[0]):
                        fileio._write_record(fh, np.ascontiguousarray(a[k]).tobytes())

    def savedata(self, istep, tt, data):
        """ana_savedata (OCFD_ANA_savedata.f90:3-196): 1 YZ planes, 2 XZ planes,
        3 XY planes, 4 points (save_points_locations.dat), 5 a block."""
        s = self.s
        kind = int(round(data[0]))
        head = np.array([istep], "<i4").tobytes() + np.array([tt], "<f8").tobytes()
        if kind in (1, 2, 3):
            points, band = int(round(data[1])), int(round(data[2]))
            tag = {1: "YZ", 2: "XZ", 3: "XY"}[kind]
            for ka in range(1, points + 1):
                at = int(round(data[2 + ka]))
                with open(self._path(f"savedata-{tag}{ka:03d}.dat"), "ab") as fh:
                    fileio._write_record(fh, head)
                    for a in range(at, at + band):
                        if kind == 1:
                            blk = s.download_block(a, a, 1, s.ny, 1, s.nz)
                        elif kind == 2:
                            blk = s.download_block(1, s.nx, a, a, 1, s.nz)
                        else:
                            blk = s.download_block(1, s.nx, 1, s.ny, a, a)
                        for q in blk:
                            fileio._write_record(fh, np.ascontiguousarray(q, dtype="<f8").tobytes())
        elif kind == 4:
            with open(self._path("save_points_locations.dat")) as fh:
                m = int(fh.readline().split()[0])
                pts = [tuple(int(x) for x in fh.readline().split()[:3]) for _ in range(m)]
            vals = np.empty((5, m))
            for c, (i, j, k) in enumerate(pts):
                blk = s.download_block(i, i, j, j, k, k)
                vals[:, c] = [b.ravel()[0] for b in blk]
            with open(self._path("save_points.dat"), "ab") as fh:
                fileio._write_record(fh, np.array([tt], "<f8").tobytes())
                for q in range(5):
                    fileio._write_record(fh, vals[q].tobytes())
        elif kind == 5:
            ib, ie, jb, je, kb, ke, fk = (int(round(x)) for x in data[1:8])
            blk = s.download_block(ib, ie, jb, je, kb, ke)
            with open(self._path(f"savedata-block{fk:03d}.dat"), "ab") as fh:
                fileio._write_record(fh, head)
                for q in blk:
                    fileio._write_record(fh, np.ascontiguousarray(q, dtype="<f8").tobytes())
