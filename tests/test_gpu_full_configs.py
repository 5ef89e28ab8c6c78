"""Benchmark configurations at full size and full step count, against the FP64
oracle (oracle/lps_oracle.c, run on the host cores).

Configuration 1 (Example 1: 196,321 nodes, 4000 steps, diagnostics every 30
steps) runs in the default GPU suite: one oracle run of about 80 s on 16
cores, compared with
* the FP64 plain form on the dense and on the neighbour-list kernels:
  displacement and velocity relative L2 <= 1e-11 after the full run, the
  dE/E0 series within 1e-10 and the energy series within 1e-11 relative;
* the FP32-mixed form on both kernel paths: displacement relative L2 <= 1e-5
  and final dE/E0 within 1e-4 of the oracle.

Configurations 2 (7 x 196,321 nodes) and 5 (785,349 nodes, m=8) at their
full 4000 steps need 10 to 20 minutes of oracle time each, more than the
default suite allows; they run when LPS_FULL_CONFIGS=1 is set, with the same
bars.  LPS_CONFIG5_STEPS cuts configuration 5 to fewer steps (its oracle
run at m=8 costs about 0.2 s per step on 16 cores).  Each test prints the
errors it measured.
"""
import os

import numpy as np
import pytest

import oracle_ctypes as O
from golden_io import rel_l2
from lps_b200 import configs
from lps_b200.api import Solver

pytestmark = pytest.mark.gpu

STATE_TOL = 1e-11
DE_TOL64 = 1e-10
U_TOL32 = 1e-5
DE_TOL32 = 1e-4
DIAG_EVERY = 30

full_only = pytest.mark.skipif(os.environ.get("LPS_FULL_CONFIGS") != "1",
                               reason="full-length oracle runs of 10-20 min: set LPS_FULL_CONFIGS=1")


def gpu_run(sets, precision, path, max_horizon=128):
    with Solver(sets, precision=precision, path=path, max_horizon=max_horizon) as sv:
        sv.step(sets[0].n_steps, diag_every=DIAG_EVERY)
        out = [(sv.read_diag(k), sv.download(k)) for k in range(len(sets))]
        info = sv.info(0)
    assert info["path"] == path
    return out


def check_fp64(name, d, st, r):
    eu, ev = rel_l2(st["u"], r["u"]), rel_l2(st["v"], r["v"])
    dE = np.max(np.abs(d["dE_rel"] - r["diag"]["dE_rel"]))
    dEn = np.max(np.abs(d["E"] - r["diag"]["E"]) / np.abs(r["diag"]["E"]))
    print(f"{name}: u rel L2 {eu:.2e}, v rel L2 {ev:.2e}, dE/E0 series {dE:.1e}, E rel {dEn:.1e}")
    assert len(d) == len(r["diag"])
    assert eu <= STATE_TOL and ev <= STATE_TOL
    assert dE <= DE_TOL64
    assert dEn <= 1e-11


def check_fp32(name, d, st, r):
    eu = rel_l2(st["u"], r["u"])
    dE = abs(d["dE_rel"][-1] - r["diag"]["dE_rel"][-1])
    print(f"{name}: u rel L2 {eu:.2e}, final dE/E0 {d['dE_rel'][-1]:.6f} vs {r['diag']['dE_rel'][-1]:.6f} "
          f"(diff {dE:.1e})")
    assert eu <= U_TOL32
    assert dE <= DE_TOL32


@pytest.fixture(scope="module")
def example1():
    (s,) = configs.example1()
    r = O.run(s, substep=DIAG_EVERY)
    assert r["status"] == 0
    return s, r


@pytest.mark.parametrize("path", ["dense", "csr"])
def test_example1_fp64_vs_oracle(example1, path):
    s, r = example1
    ((d, st),) = gpu_run([s], "fp64", path)
    check_fp64(f"config 1 fp64 {path}", d, st, r)


@pytest.mark.parametrize("path", ["dense", "csr"])
def test_example1_fp32_mixed_vs_oracle(example1, path):
    s, r = example1
    ((d, st),) = gpu_run([s], "fp32_mixed", path)
    check_fp32(f"config 1 fp32_mixed {path}", d, st, r)


@full_only
def test_poisson7_fp32_mixed_vs_oracle():
    """Configuration 2: the seven instances in one batch, FP32-mixed and FP64,
    each held to its own oracle run."""
    sets = configs.poisson7()
    out32 = gpu_run(sets, "fp32_mixed", "dense")
    out64 = gpu_run(sets, "fp64", "dense")
    for k, s in enumerate(sets):
        r = O.run(s, substep=DIAG_EVERY)
        assert r["status"] == 0
        check_fp32(f"config 2 nu={s.nu} fp32_mixed", *out32[k], r)
        check_fp64(f"config 2 nu={s.nu} fp64", *out64[k], r)


@full_only
def test_horizon8_vs_oracle():
    """Configuration 5 (m=8, 224 neighbours): both kernel paths, both forms
    (steps: LPS_CONFIG5_STEPS, default the configuration's 4000)."""
    (s,) = configs.horizon8(int(os.environ.get("LPS_CONFIG5_STEPS", configs.STEPS["horizon8"])))
    r = O.run(s, substep=DIAG_EVERY, max_horizon=256)
    assert r["status"] == 0
    for path in ("dense", "csr"):
        ((d, st),) = gpu_run([s], "fp64", path, max_horizon=256)
        check_fp64(f"config 5 fp64 {path}", d, st, r)
        ((d, st),) = gpu_run([s], "fp32_mixed", path, max_horizon=256)
        check_fp32(f"config 5 fp32_mixed {path}", d, st, r)
