"""ctypes mirror of ``ocfd_params`` (include/ocfd_gpu.h) and the opencfd2.in reader.

The field order is the C struct's; ``read_namelist`` restates read_parameter
(OCFD_readpara.f90:3-200): the namelist /control_opencfd/ with the defaults of
:28-65, names upper-cased (capitalize, :322-332) and mapped by find_scheme /
find_bc (:203-258).  AoA is converted from degrees to radians as at :143.
"""
from __future__ import annotations

import ctypes as C
import math
import re

LAP = 4

SCHEME = {"WENO5": 1, "WENO7": 2, "OMP6": 3, "UD7L": 4, "CD6": 5, "CD8": 6, "HYBRID": 10, "SCHEME_USER": 99}
SCHEME_WENO5, SCHEME_WENO7, SCHEME_OMP6, SCHEME_UD7L, SCHEME_CD6, SCHEME_CD8, SCHEME_HYBRID = 1, 2, 3, 4, 5, 6, 10
SPLIT_SW, SPLIT_LLF = 1, 2
BC = {"BC_NONE": 0, "BC_BLUNT2D": 1, "BC_BOUNDARYLAYER": 2, "BC_SWEPTCORNER": 3, "BC_USER_DEF": 99}
BC_NONE, BC_BLUNT2D, BC_BOUNDARYLAYER, BC_SWEPTCORNER, BC_USER_DEF = 0, 1, 2, 3, 99
GRIDGEN, GRID1D, GRID2D_PLANE, GRID2D_AXIAL_SYMM, GRID3D, GRID_AND_JACOBIAN3D = 0, 10, 20, 21, 30, 31
PRECISION_FP64, PRECISION_MIXED = 0, 1

# metric ids (OCFD_M_* in the header)
METRIC_NAMES = ["Axx", "Ayy", "Azz", "Akx", "Aky", "Akz", "Aix", "Aiy", "Aiz", "Asx", "Asy", "Asz", "Ajac",
                "Akx1", "Aky1", "Akz1", "Aix1", "Aiy1", "Aiz1", "Asx1", "Asy1", "Asz1"]
N_METRICS = 22


class OcfdParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("lap", C.c_int32),
        ("iperiodic", C.c_int32 * 3),
        ("iflag_gridtype", C.c_int32),
        ("periodic_span", (C.c_double * 3) * 3),
        ("scheme_invis", C.c_int32),
        ("scheme_vis", C.c_int32),
        ("if_scheme_character", C.c_int32),
        ("flux_splitting", C.c_int32),
        ("scheme_boundary", C.c_int32 * 6),
        ("if_viscous", C.c_int32),
        ("if_mass_force", C.c_int32),
        ("ibc", C.c_int32),
        ("ghost_cell", C.c_int32 * 6),
        ("nfiltering", C.c_int32),
        ("istep_show", C.c_int32), ("istep_save", C.c_int32),
        ("precision", C.c_int32),
        ("ma", C.c_double), ("re", C.c_double), ("gamma", C.c_double), ("pr", C.c_double),
        ("ref_amu_t0", C.c_double), ("dt", C.c_double), ("end_time", C.c_double), ("aoa", C.c_double),
        ("ud7l_diss", C.c_double),
        ("mass_force", C.c_double * 3),
        ("hybrid_para", C.c_double * 100),
        ("bc_para", C.c_double * 100),
        ("filter_para", (C.c_double * 100) * 10),
        ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double),
        ("cv", C.c_double), ("cp", C.c_double),
        ("ud7l", C.c_double * 8),
        ("bound_index", C.c_int32 * 6),
        ("ka1", C.c_int32), ("kb1", C.c_int32), ("ka2", C.c_int32), ("kb2", C.c_int32),
        ("reserved", C.c_int32 * 8),
    ]

    def copy(self) -> "OcfdParams":
        q = OcfdParams()
        C.memmove(C.byref(q), C.byref(self), C.sizeof(OcfdParams))
        return q


def default_params() -> OcfdParams:
    """Namelist defaults, OCFD_readpara.f90:28-65."""
    p = OcfdParams()
    p.gamma = 1.4
    p.re = 100.0
    p.ma = 1.0
    p.pr = 0.7
    p.lap = LAP
    p.scheme_invis = SCHEME_WENO5
    p.scheme_vis = SCHEME_CD6
    p.ref_amu_t0 = 288.15
    p.dt = 1.0e-4
    p.end_time = 100.0
    p.iflag_gridtype = GRID3D
    p.ibc = BC_NONE
    p.istep_show = 1
    p.istep_save = 1000
    p.if_viscous = 1
    p.ud7l_diss = 1.0
    for i in range(100):
        p.hybrid_para[i] = 1.0
    p.flux_splitting = SPLIT_SW
    return p


def set_parameters_py(p: OcfdParams) -> OcfdParams:
    """Python restatement of set_parameters/set_scheme_para (OCFD_readpara.f90:261-341),
    used where the native library is not loaded (deck parsing, footprint estimates)."""
    p.hx = 1.0 / (p.nx - 1.0)
    p.hy = 1.0 / (p.ny - 1.0)
    p.hz = 1.0 / (p.nz - 1.0)
    p.cv = 1.0 / (p.gamma * (p.gamma - 1.0) * p.ma * p.ma)
    p.cp = p.cv * p.gamma
    for d in range(3):
        b = 1 if p.iperiodic[d] == 0 else 0
        p.bound_index[2 * d] = b
        p.bound_index[2 * d + 1] = b
    ka = {SCHEME_WENO5: (-2, 2, -1, 3), SCHEME_WENO7: (-3, 3, -2, 4)}.get(p.scheme_invis, (-3, 4, -3, 4))
    p.ka1, p.kb1, p.ka2, p.kb2 = ka
    ud7 = [-3.0, 25.0, -101.0, 319.0, 214.0, -38.0, 4.0, 0.0]
    cd8 = [-3.0, 29.0, -139.0, 533.0, 533.0, -139.0, 29.0, -3.0]
    for k in range(8):
        p.ud7l[k] = p.ud7l_diss * ud7[k] / 420.0 + (1.0 - p.ud7l_diss) * cd8[k] / 840.0
    return p


# --------------------------------------------------------------------------------------
# opencfd2.in reader (namelist /control_opencfd/)

_INT_KEYS = {
    "nx_global": "nx", "ny_global": "ny", "nz_global": "nz", "lap": "lap",
    "if_scheme_character": "if_scheme_character", "if_viscous": "if_viscous",
    "istep_show": "istep_show", "istep_save": "istep_save", "iflag_gridtype": "iflag_gridtype",
    "if_mass_force": "if_mass_force", "nfiltering": "nfiltering", "flux_splitting": "flux_splitting",
}
_REAL_KEYS = {"ma": "ma", "re": "re", "gamma": "gamma", "pr": "pr", "ref_amu_t0": "ref_amu_t0", "dt": "dt",
              "end_time": "end_time", "ud7l_diss": "ud7l_diss"}
_IGNORED = {"npx0", "npy0", "npz0", "ana_number", "ana_para"}


def _values(text: str) -> list[str]:
    out = []
    for tok in re.findall(r"\"[^\"]*\"|'[^']*'|[^,\s]+", text):
        m = re.fullmatch(r"(\d+)\*(.+)", tok)
        if m:
            out.extend([m.group(2)] * int(m.group(1)))
        else:
            out.append(tok)
    return out


def _num(tok: str) -> float:
    return float(tok.lower().replace("d", "e"))


def read_namelist(path_or_text: str, is_text: bool = False) -> OcfdParams:
    """Read an opencfd2.in deck (read_parameter, OCFD_readpara.f90:3-200)."""
    text = path_or_text if is_text else open(path_or_text).read()
    m = re.search(r"[&$]control_opencfd(.*?)(?:[&$]end|/\s*$)", text, re.S | re.I)
    if not m:
        raise ValueError("namelist /control_opencfd/ not found")
    body = "\n".join(line.split("!")[0] for line in m.group(1).splitlines())
    p = default_params()
    # split into "key = values" assignments
    parts = re.split(r"([A-Za-z_][A-Za-z0-9_]*(?:\([^)]*\))?)\s*=", body)
    for i in range(1, len(parts) - 1, 2):
        key, vals = parts[i].strip(), _values(parts[i + 1])
        kl = key.lower()
        base = re.sub(r"\(.*\)", "", kl)
        sub = re.search(r"\(([^)]*)\)", kl)
        if base in _INT_KEYS:
            setattr(p, _INT_KEYS[base], int(_num(vals[0])))
        elif base in _REAL_KEYS:
            setattr(p, _REAL_KEYS[base], _num(vals[0]))
        elif base in ("iperiodic_x", "iperiodic_y", "iperiodic_z"):
            p.iperiodic["xyz".index(base[-1])] = int(_num(vals[0]))
        elif base in ("periodic_ispan", "periodic_jspan", "periodic_kspan"):
            d = "ijk".index(base[9])
            for c, v in enumerate(vals[:3]):
                p.periodic_span[d][c] = _num(v)
        elif base == "aoa":
            p.aoa = _num(vals[0]) * 3.1415926535897932 / 180.0
        elif base in ("scheme_invis", "scheme_vis"):
            name = vals[0].strip("\"'").upper()
            if name not in SCHEME:
                raise ValueError(f"This Scheme is not supported !! {name}")
            setattr(p, base, SCHEME[name])
        elif base == "boundarycondition":
            name = vals[0].strip("\"'").upper()
            if name not in BC:
                raise ValueError(f"This Boundary Condition is not supported !! {name}")
            p.ibc = BC[name]
        elif base in ("scheme_boundary", "ghost_cell", "mass_force", "bc_para", "hybrid_para"):
            arr = getattr(p, base)
            start = int(sub.group(1).split(":")[0]) - 1 if sub else 0
            for c, v in enumerate(vals):
                arr[start + c] = type(arr[0])(_num(v))
        elif base == "filter_para":
            # Filter_Para(:, m) = column m
            col = 0
            if sub:
                ix = sub.group(1).split(",")
                col = int(ix[1]) - 1 if len(ix) > 1 else 0
            for c, v in enumerate(vals):
                p.filter_para[col][c] = _num(v)
        elif base in _IGNORED:
            pass
        else:
            raise ValueError(f"unknown namelist key {key}")
    if p.nfiltering > 10:
        raise ValueError("ANA_Number and NFiltering should <=10")
    return p


def ceil_div(a: int, b: int) -> int:
    return -(-a // b)


def dt_cfl(u_max_plus_c: float, h: float, cfl: float) -> float:
    """Fixed dt from a CFL number (the reference has no CFL control; dt is fixed)."""
    return cfl * h / u_max_plus_c if u_max_plus_c > 0 else math.inf
