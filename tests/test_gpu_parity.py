"""Parity of the CUDA path (through the C ABI) with the reference and the oracle.

Bars (the FP64 plain form): displacement and velocity relative L2 <= 1e-11
after the run, the dE/E0 series within 1e-10 (relative once |dE/E0| > 1,
which only the unstable r10 fixtures reach), weighted volumes bit-identical.
Accelerations and dilatations are differences of nearly equal terms, so they
are held to 1e-9 relative L2.
"""
import numpy as np
import pytest

import oracle_ctypes as O
from golden_io import (ENERGY_COL, GOLDEN_CASES, VARIANT_OPTS, VERIFY_COL, inputs_for, load_golden,
                       rel_l2)
from lps_b200 import gen
from lps_b200.api import LpsError, Solver

pytestmark = pytest.mark.gpu

STATE_TOL = 1e-11
DERIVED_TOL = 1e-9
DE_TOL = 1e-10
PATHS = ["csr", "dense"]


def run_gpu(s, path, n_steps=None, diag_every=1, **opts):
    n = s.n_steps if n_steps is None else n_steps
    with Solver(s, path=path, **opts) as sv:
        sv.step(n, diag_every=diag_every)
        d = sv.read_diag(0, check=False)
        st = sv.download(0)
        info = sv.info(0)
        launches = sv.kernel_launches
    return d, st, info, launches


def check_series(d, en, ve):
    E = en[:, ENERGY_COL["E"]]
    assert np.max(np.abs(d["E"] - E) / np.abs(E)) <= 1e-11
    dE = ve[:, VERIFY_COL["dE_rel"]]
    assert np.max(np.abs(d["dE_rel"] - dE) / np.maximum(1.0, np.abs(dE))) <= DE_TOL
    for name in ("Ek", "Ep"):
        assert np.max(np.abs(d[name] - en[:, ENERGY_COL[name]])) <= 1e-11 * np.max(np.abs(E)), name
    for name in ("max_u", "theta_max", "uB_rms", "vB_rms"):
        ref = en[:, ENERGY_COL[name]]
        assert np.max(np.abs(d[name] - ref)) <= 1e-9 * max(np.max(np.abs(ref)), 1e-300), name
    for name in ("max_v", "max_a"):
        ref = ve[:, VERIFY_COL[name]]
        assert np.max(np.abs(d[name] - ref)) <= 1e-9 * np.max(np.abs(ref)), name


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("case,variant", GOLDEN_CASES, ids=[f"{c}_{v}" for c, v in GOLDEN_CASES])
def test_golden_parity(case, variant, path):
    """CUDA path vs the compiled reference's own outputs."""
    s = inputs_for(case, variant)
    g = load_golden(f"{case}_{variant}")
    d, st, info, launches = run_gpu(s, path, **VARIANT_OPTS[variant])
    assert info["path"] == path
    assert launches >= 3 * s.n_steps
    assert len(d) == s.n_steps
    np.testing.assert_allclose(d["t"], g["energy"][:, 0], rtol=1e-15, atol=0)
    for k in ("u", "v"):
        assert rel_l2(st[k], g[k]) <= STATE_TOL, k
    for k in ("a", "theta"):
        assert rel_l2(st[k], g[k]) <= DERIVED_TOL, k
    np.testing.assert_array_equal(st["m"], g["m"])
    check_series(d, g["energy"], g["verify"])


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("m", [3, 4, 5, 8])
def test_oracle_parity_generated(m, path):
    """Generated discs (nu=0.3, passive averaging ABC) vs the oracle."""
    s = gen.disc_problem(R=24.0, dx=0.5, m=m, nu=0.3, n_steps=240, sigma=4.0)
    r = O.run(s, substep=20, max_horizon=256)
    d, st, info, _ = run_gpu(s, path, diag_every=20, max_horizon=256)
    assert r["status"] == 0
    for k in ("u", "v"):
        assert rel_l2(st[k], r[k]) <= STATE_TOL, k
    for k in ("a", "theta"):
        assert rel_l2(st[k], r[k]) <= DERIVED_TOL, k
    dE = r["diag"]["dE_rel"]
    assert np.max(np.abs(d["dE_rel"] - dE)) <= DE_TOL
    # the argmax node of a radial pulse is a near-tie that round-off may flip;
    # compare the maximum itself
    np.testing.assert_allclose(d["max_u"], r["diag"]["max_u"], rtol=1e-12, atol=0)


@pytest.mark.parametrize("path", PATHS)
def test_batch_equals_single(path):
    """Uneven instances packed in one handle give each instance's own result."""
    sets = [gen.disc_problem(R=12.0, m=4, nu=0.2, n_steps=60, sigma=3.0),
            gen.disc_problem(R=20.0, m=3, nu=0.4, n_steps=60, sigma=5.0, centre=(2.0, -1.5)),
            gen.disc_problem(R=9.0, m=5, nu=0.3, n_steps=60, sigma=2.0, abc="none")]
    with Solver(sets, path=path) as sv:
        sv.step(60, diag_every=6)
        batch = [(sv.read_diag(k), sv.download(k)) for k in range(len(sets))]
    for k, s in enumerate(sets):
        d1, st1, _, _ = run_gpu(s, path, n_steps=60, diag_every=6)
        for key in ("u", "v", "a", "theta"):
            np.testing.assert_array_equal(batch[k][1][key], st1[key])
        # the dense batch shares one row pitch, so the reduction tree groups
        # cells differently than a single instance: equal up to rounding
        np.testing.assert_allclose(batch[k][0]["E"], d1["E"], rtol=1e-13, atol=0)


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("n_steps,diag_every", [(37, 5), (24, 0)])
def test_graphs_match_eager(path, n_steps, diag_every):
    """Captured graphs give the eager steps' bits.  With 24 steps and no
    diagnostics the call ends on the last step of a graph, which must leave v,
    a and theta current at every node (the dense path writes them at interior
    nodes only on such full steps)."""
    s = gen.disc_problem(R=15.0, m=4, nu=0.35, n_steps=n_steps, sigma=3.0)
    d1, st1, _, _ = run_gpu(s, path, diag_every=diag_every)
    d2, st2, _, _ = run_gpu(s, path, diag_every=diag_every, use_graphs=False)
    for key in ("u", "v", "a", "theta"):
        np.testing.assert_array_equal(st1[key], st2[key])
    if diag_every:
        np.testing.assert_array_equal(d1["E"], d2["E"])
    else:
        # against a run with diagnostics every step (all steps full)
        d3, st3, _, _ = run_gpu(s, path, diag_every=1)
        for key in ("u", "v", "a", "theta"):
            np.testing.assert_array_equal(st1[key], st3[key])


def test_reset_and_set_initial_repeat():
    s = gen.disc_problem(R=15.0, m=4, nu=0.3, n_steps=30, sigma=3.0)
    with Solver(s) as sv:
        sv.step(30, diag_every=10)
        a = sv.download(0)
        e1 = sv.read_diag(0)
        sv.set_initial(0, s.u0 * 2.0, s.v0)
        sv.reset()
        sv.step(30, diag_every=10)
        b = sv.download(0)
        sv.read_diag(0)
        sv.set_initial(0, s.u0, s.v0)
        sv.reset()
        sv.step(30, diag_every=10)
        c = sv.download(0)
        e3 = sv.read_diag(0)
    assert rel_l2(b["u"], 2.0 * a["u"]) <= 1e-13   # linear system
    np.testing.assert_array_equal(a["u"], c["u"])
    np.testing.assert_array_equal(e1["E"], e3["E"])


def test_nonfinite_initial_condition_is_fatal():
    """A NaN in the initial displacement ends in the reference's FATAL status."""
    s = gen.disc_problem(R=10.0, m=4, n_steps=10, sigma=3.0)
    s.u0 = s.u0.copy()
    s.u0[10] = np.nan
    with Solver(s) as sv:
        sv.step(10, diag_every=5)
        with pytest.raises(LpsError) as e:
            sv.read_diag(0)
        assert e.value.status == -3


def test_horizon_overflow_is_an_error():
    s = gen.disc_problem(R=10.0, m=8, n_steps=1, abc="none")
    with pytest.raises(LpsError) as e:
        Solver(s, max_horizon=128)   # m=8: 225 entries with self
    assert e.value.status == -2


@pytest.mark.parametrize("precision", ["fp64", "fp32_mixed"])
def test_autotune_changes_no_result(precision):
    """The autotuner only picks rows per thread and resident CTAs per SM for
    the tile kernels: every result is the same bits as with the defaults, and
    so is a run fixed at two rows per dilatation thread or (FP32-mixed) four
    rows per force thread."""
    sets = [gen.disc_problem(R=14.0, m=4, nu=0.3, n_steps=40, sigma=3.0),
            gen.disc_problem(R=11.0, m=3, nu=0.2, n_steps=40, sigma=2.5)]
    out = {}
    for tune in (False, True):
        with Solver(sets, precision=precision, autotune=tune) as sv:
            sv.step(40, diag_every=10)
            out[tune] = [(sv.read_diag(k), sv.download(k)) for k in range(len(sets))]
            info = sv.info(0)
        assert info["path"] == "dense"
        assert 1 <= info["tile_ctas_theta"] <= 8 and 1 <= info["tile_ctas_force"] <= 8
        assert info["tile_rows_theta"] in (2, 4)
    with Solver(sets, precision=precision, theta_rows=2) as sv:
        assert sv.info(0)["tile_rows_theta"] == 2
        sv.step(40, diag_every=10)
        out["rows2"] = [(sv.read_diag(k), sv.download(k)) for k in range(len(sets))]
    others = [True, "rows2"]
    if precision == "fp32_mixed":
        # four rows per force thread (the FP32-mixed form's other force kernel)
        with Solver(sets, precision=precision, force_rows=4) as sv:
            assert sv.info(0)["tile_rows_force"] == 4
            sv.step(40, diag_every=10)
            out["force4"] = [(sv.read_diag(k), sv.download(k)) for k in range(len(sets))]
        others.append("force4")
    for other in others:
        for k in range(len(sets)):
            for key in ("u", "v", "a", "theta"):
                np.testing.assert_array_equal(out[other][k][1][key], out[False][k][1][key])
            np.testing.assert_array_equal(out[other][k][0]["E"], out[False][k][0]["E"])


@pytest.mark.parametrize("kind", ["lattice_m8", "jittered_m4"])
def test_gpu_horizon_search_equals_host(kind):
    """The horizon search on the GPU (lps_horizons.cu) gives the host bucket
    grid's horizons: same weighted volumes bit for bit and the same state,
    bit for bit, after some steps on the neighbour-list kernels."""
    if kind == "lattice_m8":
        s = gen.disc_problem(R=30.0, dx=0.5, m=8, nu=0.3, n_steps=40, sigma=5.0)
        opts = dict(max_horizon=256)
    else:
        s = gen.disc_problem(R=30.0, dx=0.5, m=4, nu=0.3, n_steps=40, sigma=5.0, jitter=0.2, seed=11)
        opts = {}
    out = {}
    for build in ("host", "gpu"):
        with Solver(s, path="csr", horizon_build=build, **opts) as sv:
            info = sv.info(0)
            assert info["horizon_on_gpu"] == (build == "gpu")
            sv.step(40, diag_every=20)
            out[build] = (sv.download(0), info["max_horizon_len"])
    assert out["host"][1] == out["gpu"][1]
    for key in ("m", "u", "v", "a", "theta"):
        np.testing.assert_array_equal(out["host"][0][key], out["gpu"][0][key])
