"""Regenerates tests/golden/tgv256_history.npz: the oracle's kinetic-energy,
enstrophy and show_flow_msg histories of the 256^3 characteristic Taylor-Green
runs (OMP6, and the UD7L(CD8)/WENO7/WENO5 hybrid with sensor 1), 500 time steps
at dt = 0.0005, recorded every 5 steps, plus the conserved state after the last
step sampled on every 16th point in each direction.

The reference cannot be built here (no Fortran compiler / MPI), so the CPU
restatement of the reference (the oracle) is the CPU run these histories come
from.  The GPU test (tests/test_gpu_history.py) runs the same decks through the
C ABI and compares.  About 2 hours on 8 host cores:

    OMP_NUM_THREADS=8 python tests/golden/make_tgv256_history.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "opencfd-sc_b200")]

from ocfd_b200 import cases  # noqa: E402
from pyoracle import Oracle  # noqa: E402

N, STEPS, EVERY, DT, SUB = 256, 500, 5, 0.0005, 16


def run(scheme: str) -> dict:
    p = cases.tgv_char_params(N, scheme, dt=DT, steps=STEPS)
    o = Oracle(p)
    o.init_mesh()
    o.init3d(cases.tgv_prims(o.p))
    steps, msg, box = [0], [o.show_flow_msg()], [o.ana_box()]
    t0 = time.time()
    while steps[-1] < STEPS:
        o.step(EVERY)
        steps.append(steps[-1] + EVERY)
        msg.append(o.show_flow_msg())
        box.append(o.ana_box())
        print(f"{scheme} step {steps[-1]} ke {msg[-1][1]:.15e} {time.time() - t0:.0f} s", flush=True)
    f = o.f[:, ::SUB, ::SUB, ::SUB].copy()
    o.close()
    return {"steps": np.array(steps), "flow_msg": np.array(msg), "ana_box": np.array(box), "f_sub": f}


def main():
    out = {"dt": np.array(DT), "every": np.array(EVERY), "sub": np.array(SUB)}
    for scheme in ("OMP6", "HYBRID"):
        for k, v in run(scheme).items():
            out[f"{scheme.lower()}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "tgv256_history.npz"), **out)


if __name__ == "__main__":
    main()
