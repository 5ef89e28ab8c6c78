#!/usr/bin/env python
"""Regenerate the golden fixtures in tests/golden/ by running the reference.

Needs the read-only reference sources (--ref, or the LPS_REFERENCE environment
variable) and a C++ compiler; it builds oracle/_ref/ with oracle/Makefile, then:

* ``td``  -- the reference's own test set (tests/generate_test_data.cpp: R=30,
  dx=0.5, no absorbing layer, 300 steps), solved by the reference solver with
  per-step output (SUBSTEP_NO=1) and a binary final-state dump; plus the same
  set with nu=0.35 written into .data2 (lambda != mu exercises the theta
  coupling of the force, src/main.cpp:857-863).
* ``r10`` -- an absorbing-boundary set from the reference preprocessor with
  DOMAIN_RADIUS patched to 10 mm (dx=0.5, m=4, nu=0.25: 1257 nodes, 460 ABC
  nodes, C=49), cut to 600 steps, solved with the default switches
  (G_theta), with THETA_ABC_METHOD=0 (IDW), KINEMATIC_VELOCITY_ABC=1,
  ABCS_STEP=-1, with nu=0.35 in .data2, and with the stock build (30-step
  cadence, VTK on) for file-format parity.  This small set is mildly unstable
  in the reference itself (E grows about 50x in 600 steps; with nu=0.35 and
  the nu=0.25 operators it grows 1e12x), so comparisons are relative.
* ``r20`` -- the same with DOMAIN_RADIUS=20 mm (5025 nodes, 972 ABC nodes),
  which stays bounded: 1000 steps, default switches and IDW.

Outputs: <name>_inputs.npz (the input arrays exactly as the reference read
them from its 16-digit text files) and <name>_<variant>.npz (energy/verify
logs and final u, v, a, theta, m).  Run from the repository root:

    python tests/golden/make_golden.py
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
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from lps_b200.files import read_input_set, read_log, write_input_set  # noqa: E402
import oracle_ctypes  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
REFBIN = os.path.join(ROOT, "oracle", "_ref")

VARIANTS = {
    # name: (-D flags for the patched solver)
    "m1": "-DSUBSTEP_NO=1 -DREF_NO_VTK -DREF_DUMP",
    "m0": "-DSUBSTEP_NO=1 -DREF_NO_VTK -DREF_DUMP -DTHETA_ABC_METHOD=0",
    "kin": "-DSUBSTEP_NO=1 -DREF_NO_VTK -DREF_DUMP -DKINEMATIC_VELOCITY_ABC=1",
    "off": "-DSUBSTEP_NO=1 -DREF_NO_VTK -DREF_DUMP -DABCS_STEP=-1",
    "stock": "-DREF_DUMP",
}


def make(*targets, defs=None, name=None, ref=None):
    cmd = ["make", "-s", "-C", os.path.join(ROOT, "oracle")] + list(targets)
    if ref:
        cmd.append(f"REF={ref}")
    if defs is not None:
        cmd += [f"DEFS={defs}", f"NAME={name}"]
    subprocess.run(cmd, check=True)


def save_inputs(path, s):
    np.savez_compressed(path, n_steps=s.n_steps, n_abc=s.n_abc, max_cloud=s.max_cloud,
                        scal=np.array([s.E, s.nu, s.rho, s.wf, s.t0, s.t1, s.dt, s.delta, s.dx, s.dy, s.s0]),
                        data2_extra=s.data2_extra, nodes=s.nodes, bctypes=s.bctypes, u0=s.u0, v0=s.v0,
                        inf_nodes=s.inf_nodes, clouds=s.clouds, gu=s.gu, gv=s.gv, gtheta=s.gtheta)


def set_steps(job, steps):
    """Cut a generated set to `steps` steps (StepNo is the 2nd entry of .data1)."""
    d1 = open(job + ".data1").read().split()
    d1[1] = str(steps)
    open(job + ".data1", "w").write("\n".join(d1) + "\n")


def run_solver(binary, job, prefix, threads):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([binary, prefix, os.path.basename(job)], cwd=os.path.dirname(job), env=env,
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{binary} failed: {r.stdout[-2000:]} {r.stderr[-2000:]}")
    return r.stdout


def save_outputs(path, job, prefix, meta, keep_vtk=()):
    st = oracle_ctypes.read_state_dump(job + prefix + ".state")
    extra = {}
    for step in keep_vtk:
        for tag in ("", "-vel", "-theta"):
            f = f"{job}{prefix}{tag}-{step}.vtk"
            if os.path.exists(f):
                extra[f"vtk{tag.replace('-', '_')}_{step}"] = np.frombuffer(open(f, "rb").read(), np.uint8)
    en = open(job + prefix + ".energy", "rb").read()
    ve = open(job + prefix + ".verify", "rb").read()
    np.savez_compressed(path, energy=read_log(job + prefix + ".energy"), verify=read_log(job + prefix + ".verify"),
                        energy_text=np.frombuffer(en, np.uint8), verify_text=np.frombuffer(ve, np.uint8),
                        u=st["u"], v=st["v"], a=st["a"], theta=st["theta"], m=st["m"],
                        meta=np.array(meta), **extra)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("LPS_REFERENCE"),
                    help="root of the reference project (default: $LPS_REFERENCE)")
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--r10-steps", type=int, default=600)
    ap.add_argument("--r20-steps", type=int, default=1000)
    args = ap.parse_args()
    if not args.ref or not os.path.isdir(os.path.join(args.ref, "src")):
        ap.error("give --ref <reference root> or set LPS_REFERENCE")
    make("ref", ref=args.ref)
    for v, defs in VARIANTS.items():
        make("ref-variant", defs=defs, name=v, ref=args.ref)
    make("preproc-variant", defs="-DREF_DOMAIN_RADIUS=10.0", name="R10", ref=args.ref)
    make("preproc-variant", defs="-DREF_DOMAIN_RADIUS=20.0", name="R20", ref=args.ref)
    work = tempfile.mkdtemp(prefix="lps_golden_")
    try:
        # ---- td: the reference's own test set -------------------------------
        td = os.path.join(work, "td")
        subprocess.run([os.path.join(REFBIN, "generate_test_data"), "td"], cwd=work, check=True,
                       capture_output=True)
        s = read_input_set(td)
        save_inputs(os.path.join(OUT, "td_inputs.npz"), s)
        run_solver(os.path.join(REFBIN, "PD2_LPS_ABC_m1"), td, "_m1", args.threads)
        save_outputs(os.path.join(OUT, "td_m1.npz"), td, "_m1", ["td", "m1", "nu=0.25"])
        s35 = read_input_set(td)
        s35.nu = 0.35
        td35 = os.path.join(work, "td35")
        write_input_set(td35, s35)
        run_solver(os.path.join(REFBIN, "PD2_LPS_ABC_m1"), td35, "_m1", args.threads)
        save_outputs(os.path.join(OUT, "td_nu35.npz"), td35, "_m1", ["td", "m1", "nu=0.35"])
        # ---- r10: small absorbing-boundary set ------------------------------
        r10 = os.path.join(work, "r10")
        env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
        subprocess.run([os.path.join(REFBIN, "lps_abc_preprocessor_R10"), "r10", "0.25"], cwd=work,
                       check=True, capture_output=True, env=env)
        set_steps(r10, args.r10_steps)
        s = read_input_set(r10)
        save_inputs(os.path.join(OUT, "r10_inputs.npz"), s)
        for v in ("m1", "m0", "kin", "off"):
            run_solver(os.path.join(REFBIN, f"PD2_LPS_ABC_{v}"), r10, f"_{v}", args.threads)
            save_outputs(os.path.join(OUT, f"r10_{v}.npz"), r10, f"_{v}", ["r10", v, "nu=0.25"])
        run_solver(os.path.join(REFBIN, "PD2_LPS_ABC_stock"), r10, "_stock", args.threads)
        save_outputs(os.path.join(OUT, "r10_stock.npz"), r10, "_stock", ["r10", "stock", "nu=0.25"],
                     keep_vtk=(0, args.r10_steps))
        s35 = read_input_set(r10)
        s35.nu = 0.35
        r35 = os.path.join(work, "r35")
        write_input_set(r35, s35)
        run_solver(os.path.join(REFBIN, "PD2_LPS_ABC_m1"), r35, "_m1", args.threads)
        save_outputs(os.path.join(OUT, "r10_nu35.npz"), r35, "_m1", ["r10", "m1", "nu=0.35"])
        # ---- r20: bounded absorbing-boundary set ----------------------------
        r20 = os.path.join(work, "r20")
        subprocess.run([os.path.join(REFBIN, "lps_abc_preprocessor_R20"), "r20", "0.25"], cwd=work,
                       check=True, capture_output=True, env=env)
        set_steps(r20, args.r20_steps)
        s = read_input_set(r20)
        save_inputs(os.path.join(OUT, "r20_inputs.npz"), s)
        for v in ("m1", "m0"):
            run_solver(os.path.join(REFBIN, f"PD2_LPS_ABC_{v}"), r20, f"_{v}", args.threads)
            save_outputs(os.path.join(OUT, f"r20_{v}.npz"), r20, f"_{v}", ["r20", v, "nu=0.25"])
    finally:
        shutil.rmtree(work, ignore_errors=True)
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f"{f:24s} {os.path.getsize(os.path.join(OUT, f)) / 1024:8.1f} KB")


if __name__ == "__main__":
    main()
