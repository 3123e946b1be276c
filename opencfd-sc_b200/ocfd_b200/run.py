"""Command-line runner: a named synthetic case or an opencfd2.in deck on one GPU.

    python -m ocfd_b200.run --case tgv --n 128 --scheme OMP6 --character 1 --steps 2
    python -m ocfd_b200.run --deck opencfd2.in --steps 100 --show 10

It mirrors the reference's program flow (opencfd.f90:26-29 -> NS_solver,
OCFD_NS_Solver.f90:5-88): read parameters, set_parameters, init_mesh, initial
field, then the time loop with show_flow_msg every Istep_show steps.  The
initial field of a deck run is the reference's fallback when opencfd.dat is
absent (read_flow_data -> flowfield_init('TGV'), OCFD_IO.f90:17-20,
OCFD_flowinit.f90:18-28); --tgv-pressure uses the Taylor-Green field with its
pressure term instead.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import cases
from .params import GRID1D, GRIDGEN, SCHEME, read_namelist
from .solver import Solver


def build(args):
    if args.deck:
        p = read_namelist(args.deck)
        if args.precision == "mixed":
            p.precision = 1
        return p, None
    sch = SCHEME[args.scheme.upper()]
    if args.case == "tgv":
        p = cases.tgv_params(args.n, scheme=sch, character=args.character, dt=args.dt, split=args.split)
        if sch == SCHEME["HYBRID"]:
            p.hybrid_para[0] = 1
            p.hybrid_para[1] = 0.004
            p.hybrid_para[2] = 0.01
            p.ud7l_diss = 0.0
    elif args.case == "hit":
        p = cases.hit_params(args.n, re=args.re, dt=args.dt)
    elif args.case == "cylinder":
        p = cases.cylinder_params(dt=args.dt, character=args.character)
    else:
        raise SystemExit(f"unknown case {args.case}")
    p.precision = 1 if args.precision == "mixed" else 0
    return p, args.case


def initial_field(s: Solver, case, args):
    p = s.p
    if case == "tgv" or (case is None and args.tgv_pressure):
        s.init_mesh()
        s.init3d(cases.tgv_prims(p))
    elif case == "hit":
        X, Y, Z = cases.hit_coords(p.nx)
        s.init_mesh(X, Y, Z)
        s.init3d(cases.hit_prims(p.nx, mt=0.6, ma=p.ma))
    elif case == "cylinder":
        X, Y, Z = cases.cylinder_grid(p.nx, p.ny, p.nz)
        s.init_mesh(X, Y, Z)
        s.init3d(cases.cylinder_prims(p.nx, p.ny, p.nz))
    else:
        if p.iflag_gridtype not in (GRIDGEN, GRID1D):
            raise SystemExit("deck runs without coordinates support Iflag_Gridtype 0 (box) here")
        s.init_mesh()
        x, y, z = cases.box_coords(p.nx, p.ny, p.nz)
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        # flowfield_init('TGV'): rho = T = 1, u = sin x cos y cos z, v = -cos x sin y cos z, w = 0
        d = np.ones_like(X)
        s.init3d([d, np.sin(X) * np.cos(Y) * np.cos(Z), -np.cos(X) * np.sin(Y) * np.cos(Z), np.zeros_like(X), d])


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--deck")
    ap.add_argument("--case", default="tgv", choices=["tgv", "hit", "cylinder"])
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--scheme", default="WENO7")
    ap.add_argument("--character", type=int, default=0)
    ap.add_argument("--split", type=int, default=1)
    ap.add_argument("--dt", type=float, default=0.001)
    ap.add_argument("--re", type=float, default=500.0)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--show", type=int, default=0, help="show_flow_msg every N steps (0: at the end)")
    ap.add_argument("--tgv-pressure", action="store_true")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    p, case = build(args)
    s = Solver(p, device=args.device)
    initial_field(s, case, args)
    t0 = time.time()
    done = 0
    show = args.show or args.steps
    while done < args.steps:
        k = min(show, args.steps - done)
        s.step(k)
        done += k
        istep, tt = s.time()
        e = s.show_flow_msg()
        print(json.dumps({"Istep": istep, "tt": tt, "E_total": e[0], "E_kinetic": e[1], "entropy": e[2]}), flush=True)
    wall = time.time() - t0
    n = s.p.nx * s.p.ny * s.p.nz
    print(json.dumps({"steps": done, "wall_s": wall, "GPts/s": n * done / wall / 1e9}), flush=True)
    s.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
