"""CPU-only tests: file formats, generator geometry, and the C ABI surface."""
import os
import re

import numpy as np
import pytest

from golden_io import load_inputs
from lps_b200 import gen
from lps_b200.files import InputSetError, read_input_set, write_input_set

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_input_set_roundtrip(tmp_path):
    s = load_inputs("r10")
    job = str(tmp_path / "r10")
    write_input_set(job, s)
    t = read_input_set(job)
    assert (t.n_nodes, t.n_abc, t.max_cloud, t.n_steps) == (s.n_nodes, s.n_abc, s.max_cloud, s.n_steps)
    for k in ("nodes", "u0", "v0", "gu", "gv", "gtheta"):
        np.testing.assert_array_equal(getattr(t, k), getattr(s, k))
    for k in ("bctypes", "inf_nodes", "clouds"):
        np.testing.assert_array_equal(getattr(t, k), getattr(s, k))
    assert t.dt == s.dt and t.nu == s.nu and t.delta == s.delta


def test_short_file_is_an_error(tmp_path):
    s = load_inputs("td")
    job = str(tmp_path / "td")
    write_input_set(job, s)
    lines = open(job + ".icvalues").read().split("\n")
    open(job + ".icvalues", "w").write("\n".join(lines[: len(lines) // 2]))
    with pytest.raises(InputSetError):
        read_input_set(job)


def test_missing_file_is_an_error(tmp_path):
    with pytest.raises(InputSetError):
        read_input_set(str(tmp_path / "nothing"))


@pytest.mark.parametrize("case,R", [("r10", 10.0), ("r20", 20.0)])
def test_generator_matches_reference_preprocessor_geometry(case, R):
    """Lattice, absorbing ring, clouds and BC types equal the reference
    preprocessor's (preprocessor/main.cpp:851-902) bit for bit."""
    ref = load_inputs(case)
    s = gen.disc_problem(R=R, dx=0.5, m=4, pulse="reference")
    np.testing.assert_array_equal(s.nodes, ref.nodes)
    np.testing.assert_array_equal(s.inf_nodes, ref.inf_nodes)
    np.testing.assert_array_equal(s.clouds, ref.clouds)
    np.testing.assert_array_equal(s.bctypes, ref.bctypes)
    assert s.max_cloud == ref.max_cloud == 49
    # the reference IC was written with 16 digits; ours differs by <= 1 ulp-ish
    assert np.max(np.abs(s.u0 - ref.u0)) < 1e-15


def test_example1_geometry_counts():
    s = gen.disc_problem(R=125.0, dx=0.5, m=4)
    assert (s.n_nodes, s.n_abc, s.max_cloud) == (196321, 6268, 49)


def _declared_symbols():
    txt = "".join(open(os.path.join(ROOT, "include", h)).read() for h in ("lps_cuda.h", "lps_abcfit.h"))
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*|int64_t)\s*\*?\s*(lps_\w+)\(", txt, re.M)))


def test_abi_library_exports_every_declared_symbol():
    from lps_b200 import api
    lib = api.load_library()
    syms = _declared_symbols()
    assert len(syms) >= 14 and "lps_abcfit" in syms
    for name in syms:
        assert hasattr(lib, name), name
    assert set(api.EXPORTED) <= set(syms)


def test_abi_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from lps_b200.api import LpsError, Solver
    with pytest.raises(LpsError) as e:
        Solver(load_inputs("td"))
    assert e.value.status == -9


def test_abi_rejects_bad_theta_rows_before_device():
    """Options are checked before any device call: rows per dilatation
    thread other than 0 (default), 2 or 4 is LPS_ERR_INVALID_ARG."""
    from lps_b200.api import LpsError, Solver
    with pytest.raises(LpsError) as e:
        Solver(load_inputs("td"), theta_rows=3)
    assert e.value.status == -1
    assert "theta_rows" in str(e.value)


def test_abi_rejects_bad_force_rows_before_device():
    """Rows per FP32-mixed force thread other than 0 (default), 2 or 4 is
    LPS_ERR_INVALID_ARG, before any device call."""
    from lps_b200.api import LpsError, Solver
    with pytest.raises(LpsError) as e:
        Solver(load_inputs("td"), force_rows=3)
    assert e.value.status == -1
    assert "force_rows" in str(e.value)


def test_every_least_squares_configuration_has_a_sweep_pick():
    """Each disc of the configurations built with least-squares operators
    (Example 1, the Poisson-ratio batch, the 12.57 M-node domain through its
    R = 20 mm proxy, the m = 8 disc) has a tabulated (dt, delta_kappa) pick,
    so building a configuration never stops for a missing sweep."""
    from lps_b200 import configs
    for disc in configs.LSQ_DISCS:
        pick = configs.sweep_pick(*disc)
        assert pick is not None, disc
        dt, dk = pick
        assert 1e-9 < dt < 1e-7 and 0.0 < dk <= 5.0, (disc, pick)
