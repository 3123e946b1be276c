"""FP32 face sweeps with their input tiles staged by TMA (OCFD_FACE_TMA32=1;
the library reads the switch once per process, so each setting runs in a child
process of this test): on a periodic box (TGV, characteristic OMP6 and
flux-vector WENO7) and on the curvilinear cylinder grid with walls (non-periodic
sweeps), the mixed-precision state after a few steps agrees with the plain-load
sweeps to FP32 rounding, and its error against the FP64 run is that of the
plain-load sweeps."""
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _cases():
    from ocfd_b200.params import SCHEME_OMP6, SCHEME_WENO7
    from ocfd_testlib import curvilinear_case, tgv_case

    out = {}
    for name, kw in (("omp6c", dict(scheme=SCHEME_OMP6, character=1, ma=0.3, dt=0.004)),
                     ("weno7fv", dict(scheme=SCHEME_WENO7, character=0, ma=0.3, dt=0.004))):
        p, _, prims = tgv_case(n=(24, 20, 16), **kw)
        out[name] = (p, None, prims)
    out["cylinder"] = curvilinear_case(n=(24, 20, 8))
    return out


def _child(path):
    from ocfd_b200.solver import Solver

    res = {}
    for name, (p, X, prims) in _cases().items():
        for prec in (0, 1):
            q = p.copy()
            q.precision = prec
            s = Solver(q)
            if X is None:
                s.init_mesh()
            else:
                s.init_mesh(*X)
            s.init3d(prims)
            s.step(3)
            res[f"{name}_{prec}"] = s.download_f()
            s.close()
    np.savez(path, **res)


def _run(tmp_path, flag):
    out = os.path.join(str(tmp_path), f"tma32_{flag}.npz")
    env = dict(os.environ, OCFD_FACE_TMA32=flag)
    subprocess.run([sys.executable, os.path.abspath(__file__), out], check=True, env=env, timeout=600)
    return np.load(out)


@pytest.mark.gpu
def test_fp32_tma_staging_matches_plain_loads(tmp_path):
    plain, tma = _run(tmp_path, "0"), _run(tmp_path, "1")
    rel = lambda a, b: float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))
    for name in ("omp6c", "weno7fv", "cylinder"):
        f64 = plain[f"{name}_0"]
        np.testing.assert_array_equal(tma[f"{name}_0"], f64)  # FP64 runs do not use the switch
        a, b = tma[f"{name}_1"], plain[f"{name}_1"]
        assert rel(a, b) < 1e-6, name
        e_tma, e_plain = rel(a, f64), rel(b, f64)
        assert e_tma < 2.0 * e_plain + 1e-9, (name, e_tma, e_plain)


if __name__ == "__main__":
    for p in (os.path.dirname(HERE), os.path.join(os.path.dirname(HERE), "opencfd-sc_b200"), HERE):
        sys.path.insert(0, p)
    _child(sys.argv[1])
