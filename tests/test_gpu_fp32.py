"""The FP32-mixed form (through the C ABI), on the dense-stencil kernels and on
the neighbour-list (CSR) kernels, against the FP64 oracle and the FP64 plain
form.

Its error budget: displacement relative L2 <= 1e-5 after the run and final
dE/E0 within 1e-4 of the FP64 result.  Bond arithmetic runs in FP32, so
nothing here is compared bit for bit except results that do not depend on
the arithmetic precision (the packing of a batch).
"""
import numpy as np
import pytest

import oracle_ctypes as O
from golden_io import VARIANT_OPTS, VERIFY_COL, inputs_for, load_golden, rel_l2
from lps_b200 import gen
from lps_b200.api import Solver

pytestmark = pytest.mark.gpu

U_TOL = 1e-5     # displacement relative L2
DE_TOL = 1e-4    # final dE/E0, absolute difference


def run(s, n_steps, diag_every, precision="fp32_mixed", **opts):
    with Solver(s, precision=precision, **opts) as sv:
        sv.step(n_steps, diag_every=diag_every)
        d = sv.read_diag(0)
        st = sv.download(0)
        info = sv.info(0)
    return d, st, info


@pytest.mark.parametrize("m", [2, 3, 4, 5, 6, 8])
def test_fp32_vs_oracle_generated(m):
    """Generated discs with passive averaging ABC operators vs the FP64 oracle."""
    s = gen.disc_problem(R=24.0, dx=0.5, m=m, nu=0.3, n_steps=400, sigma=4.0)
    r = O.run(s, substep=40, max_horizon=256)
    d, st, info = run(s, 400, 40, max_horizon=256)
    assert r["status"] == 0
    assert info["path"] == "dense" and info["precision"] == 1
    assert rel_l2(st["u"], r["u"]) <= U_TOL
    assert abs(d["dE_rel"][-1] - r["diag"]["dE_rel"][-1]) <= DE_TOL
    np.testing.assert_allclose(d["E"], r["diag"]["E"], rtol=1e-4, atol=0)


def test_fp32_vs_reference_golden():
    """The compiled reference's own outputs (stable R=20 fixture)."""
    s = inputs_for("r20", "m1")
    g = load_golden("r20_m1")
    d, st, _ = run(s, s.n_steps, 1)
    assert rel_l2(st["u"], g["u"]) <= U_TOL
    assert abs(d["dE_rel"][-1] - g["verify"][-1, VERIFY_COL["dE_rel"]]) <= DE_TOL


def test_fp32_poisson_batch_full_size():
    """The seven-instance Poisson-ratio batch (196,321 nodes each), 4000 steps:
    FP32-mixed vs the FP64 plain form, which is itself held to the oracle at
    1e-11 by the FP64 parity tests."""
    sets = gen.poisson_batch()
    res = {}
    for prec in ("fp64", "fp32_mixed"):
        with Solver(sets, precision=prec) as sv:
            sv.step(4000, diag_every=400)
            res[prec] = [(sv.read_diag(k), sv.download(k)["u"]) for k in range(len(sets))]
    for k in range(len(sets)):
        (d64, u64), (d32, u32) = res["fp64"][k], res["fp32_mixed"][k]
        assert rel_l2(u32, u64) <= U_TOL, k
        assert abs(d32["dE_rel"][-1] - d64["dE_rel"][-1]) <= DE_TOL, k


def test_fp32_batch_equals_single():
    """Packing does not change any instance's arithmetic."""
    sets = [gen.disc_problem(R=12.0, m=4, nu=0.2, n_steps=60, sigma=3.0),
            gen.disc_problem(R=20.0, m=3, nu=0.4, n_steps=60, sigma=5.0, centre=(2.0, -1.5)),
            gen.disc_problem(R=9.0, m=5, nu=0.3, n_steps=60, sigma=2.0, abc="none")]
    with Solver(sets, precision="fp32_mixed") as sv:
        sv.step(60, diag_every=6)
        batch = [sv.download(k) for k in range(len(sets))]
    for k, s in enumerate(sets):
        _, st1, _ = run(s, 60, 6)
        for key in ("u", "v", "a", "theta"):
            np.testing.assert_array_equal(batch[k][key], st1[key])


def test_fp32_graphs_match_eager():
    s = gen.disc_problem(R=15.0, m=4, nu=0.35, n_steps=37, sigma=3.0)
    _, st1, _ = run(s, 37, 5)
    _, st2, _ = run(s, 37, 5, use_graphs=False)
    for key in ("u", "v", "a", "theta"):
        np.testing.assert_array_equal(st1[key], st2[key])


# ---------------------------------------------------------------------------
# The FP32-mixed form on the neighbour-list (CSR) kernels


@pytest.mark.parametrize("m", [3, 4, 5, 8])
def test_fp32_csr_vs_oracle_generated(m):
    """The CSR kernels in FP32-mixed form vs the FP64 oracle, m = 3, 4, 5, 8."""
    s = gen.disc_problem(R=24.0, dx=0.5, m=m, nu=0.3, n_steps=400, sigma=4.0)
    r = O.run(s, substep=40, max_horizon=256)
    d, st, info = run(s, 400, 40, path="csr", max_horizon=256)
    assert r["status"] == 0
    assert info["path"] == "csr" and info["precision"] == 1
    assert rel_l2(st["u"], r["u"]) <= U_TOL
    assert abs(d["dE_rel"][-1] - r["diag"]["dE_rel"][-1]) <= DE_TOL
    np.testing.assert_allclose(d["E"], r["diag"]["E"], rtol=1e-4, atol=0)


@pytest.mark.parametrize("variant", ["m1", "m0"])
def test_fp32_csr_vs_reference_golden(variant):
    """The compiled reference's own outputs (the stable R=20 fixtures, G_theta
    and inverse-distance ABC dilatation) through the CSR kernels."""
    s = inputs_for("r20", variant)
    g = load_golden(f"r20_{variant}")
    d, st, _ = run(s, s.n_steps, 1, path="csr", **VARIANT_OPTS[variant])
    assert rel_l2(st["u"], g["u"]) <= U_TOL
    assert abs(d["dE_rel"][-1] - g["verify"][-1, VERIFY_COL["dE_rel"]]) <= DE_TOL


@pytest.mark.parametrize("path", ["csr", "dense"])
def test_fp32_kinematic_velocity_vs_oracle(path):
    """KINEMATIC_VELOCITY_ABC = 1 (src/main.cpp:940-943) in FP32-mixed form."""
    s = gen.disc_problem(R=24.0, dx=0.5, m=4, nu=0.35, n_steps=400, sigma=4.0)
    r = O.run(s, substep=40, kinematic_v=1)
    d, st, info = run(s, 400, 40, path=path, kinematic_v=1)
    assert r["status"] == 0 and info["path"] == path
    assert rel_l2(st["u"], r["u"]) <= U_TOL
    assert abs(d["dE_rel"][-1] - r["diag"]["dE_rel"][-1]) <= DE_TOL


def test_fp32_csr_arbitrary_nodes():
    """A node set that is not a lattice (every node moved by up to 0.1 dx):
    the automatic path is the CSR one, in FP32-mixed form, held to the oracle."""
    s = gen.disc_problem(R=20.0, dx=0.5, m=4, nu=0.25, n_steps=300, sigma=4.0, jitter=0.1, seed=7)
    r = O.run(s, substep=30)
    d, st, info = run(s, 300, 30)
    assert r["status"] == 0
    assert info["path"] == "csr" and info["precision"] == 1
    assert rel_l2(st["u"], r["u"]) <= U_TOL
    assert abs(d["dE_rel"][-1] - r["diag"]["dE_rel"][-1]) <= DE_TOL


def test_fp32_csr_batch_equals_single():
    """Packing does not change any instance's arithmetic on the CSR kernels."""
    sets = [gen.disc_problem(R=12.0, m=4, nu=0.2, n_steps=60, sigma=3.0),
            gen.disc_problem(R=14.0, m=3, nu=0.4, n_steps=60, sigma=4.0, jitter=0.05, seed=3)]
    with Solver(sets, precision="fp32_mixed", path="csr") as sv:
        sv.step(60, diag_every=6)
        batch = [sv.download(k) for k in range(len(sets))]
    for k, s in enumerate(sets):
        _, st1, _ = run(s, 60, 6, path="csr")
        for key in ("u", "v", "a", "theta"):
            np.testing.assert_array_equal(batch[k][key], st1[key])
