"""The allocation-free diagnostics entry point, checked against the handle's own.

lps_state_diag_noalloc is for callers that must not allocate device memory
when they call it (see include/lps_cuda.h).  Here it reduces a state that the
regular entry points produced, and its numbers must equal the diagnostics
record lps_read_diag returned for that same state, on two calls in a row
(the second call reuses the static scratch the first one left behind).
This file is named to run after every other test file.
"""
import ctypes as C

import numpy as np
import pytest

from lps_b200 import gen
from lps_b200.api import Solver, load_library

pytestmark = pytest.mark.gpu

SUM_RTOL = 1e-12   # sums differ from the handle's only by reduction order


def _bind(lib):
    f = lib.lps_state_diag_noalloc
    dp = C.c_void_p
    f.argtypes = [C.c_int, dp, dp, dp, dp, dp, C.c_double, C.c_double, C.c_double, C.c_double, dp, dp]
    f.restype = C.c_int
    return f


@pytest.fixture(scope="module")
def state_and_record():
    s = gen.disc_problem(R=20.0, dx=0.5, m=4, nu=0.3, n_steps=90, sigma=4.0, centre=(1.5, -2.0))
    with Solver(s) as sv:
        sv.step(90, diag_every=90)
        rec = sv.read_diag(0)[-1]
        st = sv.download(0)
        out_r = sv.info(0)["output_exclude_r"]
    return s, st, rec, out_r


def test_noalloc_matches_read_diag_twice(state_and_record):
    import torch
    s, st, rec, out_r = state_and_record
    lib = load_library()
    f = _bind(lib)
    dev = torch.device("cuda", 0)
    xy = torch.from_numpy(np.ascontiguousarray(s.nodes).ravel()).to(dev)
    u = torch.from_numpy(st["u"]).to(dev)
    v = torch.from_numpy(st["v"]).to(dev)
    a = torch.from_numpy(st["a"]).to(dev)
    th = torch.from_numpy(st["theta"]).to(dev)
    results = []
    for _ in range(2):
        out = torch.full((10,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        status = f(s.n_nodes, xy.data_ptr(), u.data_ptr(), v.data_ptr(), a.data_ptr(), th.data_ptr(),
                   s.rho, s.dx, s.dy, out_r, out.data_ptr(), None)
        assert status == 0, lib.lps_last_error(None)
        torch.cuda.synchronize()
        results.append(out.cpu().numpy())
    np.testing.assert_array_equal(results[0], results[1])
    r = results[0]
    np.testing.assert_allclose(r[0], rec["Ek"], rtol=SUM_RTOL, atol=0)
    pscale = s.rho * s.dx * s.dy * np.abs(st["v"]).sum()
    assert abs(r[1] - rec["Px"]) <= SUM_RTOL * pscale
    assert abs(r[2] - rec["Py"]) <= SUM_RTOL * pscale
    for i, key in ((3, "max_u"), (4, "max_v"), (5, "max_a"), (6, "theta_min"), (7, "theta_max")):
        assert r[i] == rec[key], key
    assert int(r[8]) == rec["max_u_node"]
    assert int(r[9]) == rec["max_v_node"]


def test_noalloc_rejects_oversize_input():
    lib = load_library()
    f = _bind(lib)
    big = 1048576 + 1   # LPS_NOALLOC_MAX_NODES + 1; rejected before any launch
    status = f(big, 1, 1, 1, 1, 1, 1.0, 1.0, 1.0, -1.0, 1, None)
    assert status == -1
    assert b"LPS_NOALLOC_MAX_NODES" in lib.lps_last_error(None)


def test_noalloc_rejects_misaligned_views():
    lib = load_library()
    f = _bind(lib)
    # a view that starts on an odd double (8-byte aligned only) is refused
    # before any launch; the addresses are never dereferenced
    ok16, odd8 = 4096, 4096 + 8
    for args in ((odd8, ok16, ok16, ok16), (ok16, odd8, ok16, ok16), (ok16, ok16, odd8, ok16),
                 (ok16, ok16, ok16, odd8)):
        status = f(1000, *args, ok16, 1.0, 1.0, 1.0, -1.0, ok16, None)
        assert status == -1
        assert b"16-byte aligned" in lib.lps_last_error(None)
    status = f(1000, ok16, ok16, ok16, ok16, ok16 + 4, 1.0, 1.0, 1.0, -1.0, ok16, None)
    assert status == -1
