"""Pins the C oracle (oracle/lps_oracle.c) to outputs of the compiled reference.

The fixtures in tests/golden/ were produced by the reference solver itself
(tests/golden/make_golden.py); the oracle must reproduce them up to the order
of equidistant neighbours, far inside the FP64 parity bar of the GPU path
(displacement relative L2 <= 1e-11, dE/E0 series within 1e-10).
"""
import numpy as np
import pytest

import oracle_ctypes as O
from golden_io import (ENERGY_COL, GOLDEN_CASES, VARIANT_OPTS, VERIFY_COL, inputs_for, load_golden,
                       rel_l2)

PIN_STATE_TOL = 1e-12     # relative L2 of u and v after the run
PIN_DERIVED_TOL = 1e-10   # relative L2 of a and theta (differences of near-equal terms)
PIN_SERIES_TOL = 1e-12    # relative E difference and the other logged columns
PIN_DE_TOL = 1e-10        # |dE/E0| difference, relative once |dE/E0| > 1


@pytest.fixture(scope="module", params=GOLDEN_CASES, ids=lambda c: f"{c[0]}_{c[1]}")
def pinned(request):
    case, variant = request.param
    s = inputs_for(case, variant)
    g = load_golden(f"{case}_{variant}")
    r = O.run(s, substep=1, **VARIANT_OPTS[variant])
    return case, variant, s, g, r


def test_status_and_record_count(pinned):
    case, variant, s, g, r = pinned
    assert r["status"] == 0
    assert len(r["diag"]) == g["energy"].shape[0] == s.n_steps


def test_final_state(pinned):
    case, variant, s, g, r = pinned
    for k in ("u", "v"):
        assert rel_l2(r[k], g[k]) <= PIN_STATE_TOL, k
    for k in ("a", "theta"):
        assert rel_l2(r[k], g[k]) <= PIN_DERIVED_TOL, k
    # weighted volumes follow the same operation order: identical bits
    np.testing.assert_array_equal(r["m"], g["m"])


def test_energy_and_verify_series(pinned):
    case, variant, s, g, r = pinned
    d = r["diag"]
    en, ve = g["energy"], g["verify"]
    # logs hold 16 significant digits (setprecision(16)), not round-trip doubles
    np.testing.assert_allclose(d["t"], en[:, ENERGY_COL["t"]], rtol=1e-15, atol=0)
    E = en[:, ENERGY_COL["E"]]
    assert np.max(np.abs(d["E"] - E) / np.abs(E)) <= PIN_SERIES_TOL
    dE = ve[:, VERIFY_COL["dE_rel"]]
    assert np.max(np.abs(d["dE_rel"] - dE) / np.maximum(1.0, np.abs(dE))) <= PIN_DE_TOL
    for name in ("Ek", "Ep"):
        ref = en[:, ENERGY_COL[name]]
        assert np.max(np.abs(d[name] - ref)) <= PIN_SERIES_TOL * np.max(np.abs(E)), name
    for name in ("max_u", "theta_max", "uB_rms", "vB_rms"):
        ref = en[:, ENERGY_COL[name]]
        scale = max(np.max(np.abs(ref)), 1e-300)
        assert np.max(np.abs(d[name] - ref)) <= PIN_SERIES_TOL * scale, name
    for name in ("max_v", "max_a"):
        ref = ve[:, VERIFY_COL[name]]
        assert np.max(np.abs(d[name] - ref)) <= PIN_SERIES_TOL * np.max(np.abs(ref)), name
    # momentum sums cancel to round-off; compare against the momentum scale
    pscale = s.rho * s.dx * s.dy * np.max(np.abs(d["max_v"])) * np.sqrt(s.n_nodes)
    for name in ("Px", "Py"):
        assert np.max(np.abs(d[name] - en[:, ENERGY_COL[name]])) <= 1e-10 * pscale, name


def test_horizon_counts():
    # m=4 lattice: 68 neighbours + self for an interior node (src/main.cpp:352)
    s = inputs_for("td", "m1")
    r, lengths, hz = O.build_horizons(s.nodes, s.delta + s.dx / 2.0 + 1e-5, 128)
    assert r == 69
    assert np.all(hz[np.arange(s.n_nodes), 0] == np.arange(s.n_nodes))


def test_planted_mistake_is_caught():
    """A wrong oracle (rho perturbed by 1e-9) must fail the pin."""
    s = inputs_for("td", "m1")
    g = load_golden("td_m1")
    s.rho = s.rho * (1 + 1e-9)
    r = O.run(s, n_steps=s.n_steps, substep=1)
    assert rel_l2(r["u"], g["u"]) > PIN_STATE_TOL
