"""Host-side logic without a GPU: the parameter deck, set_parameters, the C ABI
exports, the device-memory footprint, and the multi-process replica timing."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from ocfd_b200 import _lib, cases
from ocfd_b200.params import (BC_BLUNT2D, SCHEME_HYBRID, SCHEME_OMP6, SCHEME_UD7L, SCHEME_WENO5, SCHEME_WENO7,
                              OcfdParams, default_params, read_namelist, set_parameters_py)
from pyoracle import Oracle
from pyoracle import set_parameters as orc_set_parameters

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def test_deck_tgv_reads_like_read_parameter():
    p = read_namelist(os.path.join(GOLDEN, "deck_tgv.in"))
    assert (p.nx, p.ny, p.nz) == (128, 128, 128)
    assert p.scheme_invis == SCHEME_OMP6 and p.scheme_vis == 5
    assert abs(p.ma - 0.1) < 1e-15 and abs(p.re - 1600.0) < 1e-12
    assert list(p.iperiodic) == [1, 1, 1]
    assert abs(p.periodic_span[0][0] - 6.2831853071795864) < 1e-15 and p.periodic_span[0][1] == 0.0
    assert p.ibc == 0
    # defaults of OCFD_readpara.f90:28-65 for keys the deck omits
    assert p.gamma == 1.4 and p.pr == 0.7 and p.ref_amu_t0 == 288.15 and p.flux_splitting == 1
    assert all(p.hybrid_para[i] == 1.0 for i in range(100))


def test_deck_blunt_reads_like_read_parameter():
    p = read_namelist(os.path.join(GOLDEN, "deck_blunt.in"))
    assert p.ibc == BC_BLUNT2D and p.scheme_invis == SCHEME_WENO5 and p.if_scheme_character == 1
    assert list(p.iperiodic) == [0, 0, 1] and p.periodic_span[2][2] == 1.0
    assert p.iflag_gridtype == 20


def test_deck_rejects_unknown_scheme():
    with pytest.raises(ValueError):
        read_namelist("&control_opencfd\n Scheme_Invis='FOO'\n/", is_text=True)


@pytest.mark.parametrize("scheme,ka", [(SCHEME_WENO5, (-2, 2, -1, 3)), (SCHEME_WENO7, (-3, 3, -2, 4)),
                                       (SCHEME_OMP6, (-3, 4, -3, 4)), (SCHEME_UD7L, (-3, 4, -3, 4)),
                                       (SCHEME_HYBRID, (-3, 4, -3, 4))])
def test_set_parameters_three_ways(scheme, ka):
    """ocfd_set_parameters (library), the oracle and the Python restatement agree."""
    p = default_params()
    p.nx, p.ny, p.nz = 24, 20, 16
    p.iperiodic[0] = 1
    p.scheme_invis = scheme
    p.ud7l_diss = 0.3
    p.ma = 0.7
    lib = _lib.lib()
    q = p.copy()
    assert lib.ocfd_set_parameters(C.byref(q)) == 0
    o = orc_set_parameters(p)
    r = set_parameters_py(p.copy())
    for x in (q, o, r):
        assert (x.ka1, x.kb1, x.ka2, x.kb2) == ka
        assert x.hx == 1.0 / 23.0 and x.hy == 1.0 / 19.0 and x.hz == 1.0 / 15.0
        assert x.cv == 1.0 / (1.4 * (1.4 - 1.0) * 0.7 * 0.7)
        assert list(x.bound_index) == [0, 0, 1, 1, 1, 1]
        assert list(x.ud7l) == list(q.ud7l)


@pytest.mark.parametrize("field,value", [("lap", 3), ("nx", 6), ("scheme_vis", 1), ("ibc", 2), ("ibc", 3),
                                         ("flux_splitting", 3), ("nfiltering", 11), ("precision", 2)])
def test_set_parameters_rejects_unsupported(field, value):
    p = cases.tgv_params(16)
    setattr(p, field, value)
    assert _lib.lib().ocfd_set_parameters(C.byref(p)) == _lib.OCFD_E_PARAM


def test_library_exports_every_header_symbol():
    text = open(os.path.join(ROOT, "include", "ocfd_gpu.h")).read()
    names = set(re.findall(r"\b(ocfd_\w+)\s*\(", text))
    assert len(names) > 30
    for strict in (False, True):
        L = _lib.lib(strict)
        for n in sorted(names):
            assert hasattr(L, n), n
    assert names <= set(_lib.EXPORTED) | {"ocfd_batch_step"}, names - set(_lib.EXPORTED)


def test_params_struct_matches_c_layout():
    """sizeof(ocfd_params) seen by ctypes equals the C compiler's."""
    import subprocess
    import tempfile

    src = '#include <stdio.h>\n#include "ocfd_gpu.h"\nint main(){printf("%zu %zu", sizeof(ocfd_params), ' \
          'offsetof(ocfd_params, ka1));return 0;}\n'
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src.replace("#include <stdio.h>", "#include <stdio.h>\n#include <stddef.h>"))
        exe = os.path.join(d, "t")
        subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert int(out[0]) == C.sizeof(OcfdParams)
    assert int(out[1]) == OcfdParams.ka1.offset


def test_footprint_fits_the_named_configs():
    from ocfd_b200.solver import footprint

    gb = 1 << 30
    tgv = set_parameters_py(cases.tgv_params(256, scheme=SCHEME_OMP6, character=1))
    hit = set_parameters_py(cases.hit_params(512))
    assert footprint(tgv) < 20 * gb
    assert footprint(hit) < 170 * gb  # 512^3 FP64 fits one B200
    mixed = hit.copy()
    mixed.precision = 1
    # FP32 copies of the primitives and metrics are added, the face and viscous fluxes halve
    assert footprint(mixed) < 170 * gb
    assert abs(footprint(mixed) - footprint(hit)) < 0.1 * footprint(hit)


def test_golden_oracle_fixture_reproduces():
    """The committed oracle output (tests/golden/make_golden.py) still reproduces."""
    g = np.load(os.path.join(GOLDEN, "tgv12_oracle.npz"))
    for name in ("weno7", "omp6_char"):
        p = cases.tgv_params(12, scheme=SCHEME_WENO7 if name == "weno7" else SCHEME_OMP6,
                             character=0 if name == "weno7" else 1, dt=0.005)
        o = Oracle(p)
        o.init_mesh()
        o.init3d(cases.tgv_prims(o.p))
        o.step(3)
        np.testing.assert_array_equal(o.f, g[name])
        o.close()
