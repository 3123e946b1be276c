"""Regenerates tests/golden/tgv12_oracle.npz: the oracle's conserved state after
3 time steps of a 12^3 Taylor-Green vortex (WENO7 flux-vector form, and OMP6
characteristic form), dt = 0.005.  A regression fixture for the oracle itself:
the reference cannot be built here (no Fortran compiler / MPI) and ships no
stored outputs.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "opencfd-sc_b200")]

from ocfd_b200 import cases  # noqa: E402
from ocfd_b200.params import SCHEME_OMP6, SCHEME_WENO7  # noqa: E402
from pyoracle import Oracle  # noqa: E402


def main():
    out = {}
    for name, scheme, ch in (("weno7", SCHEME_WENO7, 0), ("omp6_char", SCHEME_OMP6, 1)):
        p = cases.tgv_params(12, scheme=scheme, character=ch, dt=0.005)
        o = Oracle(p)
        o.init_mesh()
        o.init3d(cases.tgv_prims(o.p))
        o.step(3)
        out[name] = o.f.copy()
        o.close()
    np.savez_compressed(os.path.join(HERE, "tgv12_oracle.npz"), **out)


if __name__ == "__main__":
    main()
