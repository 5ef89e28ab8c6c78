"""The absorbing-boundary operator fit (lps_b200.abcfit, the host C++ fit in
liblps_b200.so) against the reference preprocessor's own output.

* r10 / r20: the Example-1 preprocessor with DOMAIN_RADIUS 10 and 20 mm
  (tests/golden/*_inputs.npz): the full sweep picks the reference's dt and
  every G_u, G_v, G_theta entry matches its 16-digit text to 1e-15.
* fit_*: geometries and Poisson ratios the stock preprocessor cannot make
  (tests/golden/make_fit_golden.py): nu = 0.35; m = 3; dx = 0.25 mm.  The
  generator's lattice, ring and clouds equal the preprocessor's bit for bit,
  and the sweep's dt and the sampled operator rows match.

No GPU: the fit runs on the host cores (dgelsd from scipy's OpenBLAS).
"""
import os

import numpy as np
import pytest

from lps_b200 import abcfit, gen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-15   # the fixtures hold 16 significant digits of values below 1


def test_fit_matches_reference_r10_with_sweep():
    d = np.load(os.path.join(GOLDEN, "r10_inputs.npz"))
    sc = d["scal"]  # E, nu, rho, wf, t0, t1, dt, delta, dx, dy, s0
    r = abcfit.fit(d["nodes"], d["inf_nodes"], d["clouds"], E=sc[0], nu=sc[1], rho=sc[2], delta=sc[7], dx=sc[8],
                   dy=sc[9])
    assert r["dt"] == sc[6]
    assert r["n_steps"] == 12000 and r["stable_found"] == 1 and r["dgelsd_failures"] == 0
    for k in ("gu", "gv", "gtheta"):
        assert np.max(np.abs(r[k] - d[k])) <= TOL, k


def test_fit_matches_reference_r20_at_its_dt():
    d = np.load(os.path.join(GOLDEN, "r20_inputs.npz"))
    sc = d["scal"]
    r = abcfit.fit(d["nodes"], d["inf_nodes"], d["clouds"], E=sc[0], nu=sc[1], rho=sc[2], delta=sc[7], dx=sc[8],
                   dy=sc[9], sweep=False, dt=sc[6], dk_factor=0.9)
    for k in ("gu", "gv", "gtheta"):
        assert np.max(np.abs(r[k] - d[k])) <= TOL, k


@pytest.mark.parametrize("name", ["fit_r10_nu35", "fit_r10_m3", "fit_r8_dx025"])
def test_generator_and_fit_match_reference(name):
    f = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    R, dx, m, nu = f["case"]
    s = gen.disc_problem(R=R, dx=dx, m=int(m), nu=nu, n_steps=10, abc="lsq")
    np.testing.assert_array_equal(s.nodes, f["nodes"])
    np.testing.assert_array_equal(s.inf_nodes, f["inf_nodes"])
    np.testing.assert_array_equal(s.clouds, f["clouds"])
    assert s.dt == f["dt"]
    assert s.fit["n_steps"] == f["n_steps"]
    rows = f["rows"]
    uv = np.stack([2 * rows, 2 * rows + 1], axis=1).ravel()
    assert np.max(np.abs(s.gu[uv] - f["gu"])) <= TOL
    assert np.max(np.abs(s.gv[uv] - f["gv"])) <= TOL
    assert np.max(np.abs(s.gtheta[rows] - f["gtheta"])) <= TOL


def test_fit_rejects_bad_arguments():
    with pytest.raises(ValueError):
        abcfit.fit(np.zeros((4, 2)), np.array([7], np.int32), np.zeros((1, 3), np.int32), E=0.19, nu=0.25,
                   rho=8e-15, delta=2.0, dx=0.5)


def test_fit_cache_returns_the_fit(tmp_path, monkeypatch):
    """The on-disk operator cache (shared by the processes of one host) gives
    back exactly the operators, time step and fit record that a fresh fit
    gives, for the second caller as for the first."""
    from lps_b200 import configs, gen
    monkeypatch.setenv("LPS_FIT_CACHE", str(tmp_path))
    pick = (1.75e-8, 0.9)
    direct = gen.disc_problem(R=10.0, dx=0.5, m=4, nu=0.3, n_steps=20, abc="lsq", dt=pick[0], dk_factor=pick[1],
                              sigma=3.0)
    first = configs._fitted(10.0, 0.5, 4, 0.3, 20, pick, {"sigma": 3.0})
    second = configs._fitted(10.0, 0.5, 4, 0.3, 20, pick, {"sigma": 3.0})
    assert len(list(tmp_path.glob("*.npz"))) == 1
    for s in (first, second):
        for k in ("gu", "gv", "gtheta", "u0", "nodes", "clouds", "inf_nodes", "bctypes"):
            np.testing.assert_array_equal(getattr(s, k), getattr(direct, k))
        assert (s.dt, s.t1, s.n_steps) == (direct.dt, direct.t1, direct.n_steps)
        assert s.fit == direct.fit
