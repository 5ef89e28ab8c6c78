#!/usr/bin/env python
"""Fixtures that pin the absorbing-boundary operator fit (lps_b200.abcfit) to
the reference preprocessor itself, on geometries its stock build cannot make.

The preprocessor (preprocessor/main.cpp) is compiled by oracle/Makefile with
its domain radius, spacing and m-ratio overridden (-DREF_DOMAIN_RADIUS,
-DREF_DX, -DREF_M; arithmetic unchanged) and run with a Poisson ratio on the
command line, one OpenBLAS thread.  For each case the fixture keeps what its
files say about the ring, the clouds and the sweep (dt, StepNo) in full, and
the operator rows of every 10th absorbing node (G_u and G_v rows 2i, 2i+1,
G_theta row i), as the 16-digit text the solver reads:

* fit_r10_nu35  -- R=10 mm, dx=0.5 mm, m=4, nu=0.35
* fit_r10_m3    -- R=10 mm, dx=0.5 mm, m=3, nu=0.25
* fit_r8_dx025  -- R=8 mm, dx=0.25 mm, m=4, nu=0.30

Needs the reference sources (--ref or LPS_REFERENCE).  Run from the
repository root:  python tests/golden/make_fit_golden.py --ref <reference root>
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "peridynamic-lps-absorbing-boundary_b200"))
from lps_b200.files import read_input_set  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
REFBIN = os.path.join(ROOT, "oracle", "_ref")
STRIDE = 10

CASES = {
    # name: (R, dx, m, nu)
    "fit_r10_nu35": (10.0, 0.5, 4, 0.35),
    "fit_r10_m3": (10.0, 0.5, 3, 0.25),
    "fit_r8_dx025": (8.0, 0.25, 4, 0.30),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("LPS_REFERENCE"),
                    help="root of the reference project (default: $LPS_REFERENCE)")
    args = ap.parse_args()
    if not args.ref or not os.path.isdir(os.path.join(args.ref, "src")):
        ap.error("give --ref <reference root> or set LPS_REFERENCE")
    work = tempfile.mkdtemp(prefix="lps_fitgold_")
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
    try:
        for name, (R, dx, m, nu) in CASES.items():
            defs = f"-DREF_DOMAIN_RADIUS={R} -DREF_DX={dx} -DREF_M={m}.0"
            subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "preproc-variant", f"REF={args.ref}",
                            f"DEFS={defs}", f"NAME={name}"], check=True)
            subprocess.run([os.path.join(REFBIN, f"lps_abc_preprocessor_{name}"), name, str(nu)], cwd=work,
                           check=True, capture_output=True, env=env)
            s = read_input_set(os.path.join(work, name))
            rows = np.arange(0, s.n_abc, STRIDE)
            uv_rows = np.stack([2 * rows, 2 * rows + 1], axis=1).ravel()
            np.savez_compressed(os.path.join(OUT, f"{name}.npz"), case=np.array([R, dx, m, nu]),
                                n_nodes=s.n_nodes, n_steps=s.n_steps, dt=s.dt, nodes=s.nodes,
                                inf_nodes=s.inf_nodes, clouds=s.clouds, rows=rows, gu=s.gu[uv_rows],
                                gv=s.gv[uv_rows], gtheta=s.gtheta[rows], data2_extra=s.data2_extra)
            print(f"{name}: {s.n_nodes} nodes, {s.n_abc} ABC nodes, C={s.max_cloud}, dt={s.dt:g}, "
                  f"{os.path.getsize(os.path.join(OUT, name + '.npz')) / 1024:.1f} KB")
    finally:
        shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    main()
