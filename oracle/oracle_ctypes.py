"""ctypes binding of the C oracle (liblps_oracle.so) and readers for the
reference checker outputs.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py -- never by the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblps_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class Problem(C.Structure):
    _fields_ = [("n_nodes", C.c_int), ("n_abc", C.c_int), ("max_cloud", C.c_int),
                ("n_prenotch", C.c_int),
                ("E", C.c_double), ("nu", C.c_double), ("rho", C.c_double), ("dt", C.c_double),
                ("delta", C.c_double), ("dx", C.c_double), ("dy", C.c_double),
                ("nodes", _dp), ("bctypes", _ip), ("u0", _dp), ("v0", _dp), ("prenotch", _dp),
                ("inf_nodes", _ip), ("clouds", _ip), ("gu", _dp), ("gv", _dp), ("gtheta", _dp)]


class Options(C.Structure):
    _fields_ = [("abcs_step", C.c_int), ("theta_method", C.c_int), ("kinematic_v", C.c_int),
                ("max_horizon", C.c_int), ("substep", C.c_int), ("n_threads", C.c_int)]


DIAG_FIELDS = ("t", "E", "Ek", "Ep", "Px", "Py", "max_u", "max_v", "max_a",
               "theta_min", "theta_max", "uB_rms", "vB_rms", "dE_rel")


class Diag(C.Structure):
    _fields_ = [(f, C.c_double) for f in DIAG_FIELDS] + [
        ("step", C.c_int), ("max_u_node", C.c_int), ("max_v_node", C.c_int), ("n_active_abc", C.c_int)]


DIAG_DTYPE = np.dtype([(f, np.float64) for f in DIAG_FIELDS] +
                      [("step", np.int32), ("max_u_node", np.int32), ("max_v_node", np.int32),
                       ("n_active_abc", np.int32)])
assert DIAG_DTYPE.itemsize == C.sizeof(Diag)

_lib = None


def build() -> None:
    """Compile liblps_oracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _lib.lpso_run.restype = C.c_int
        _lib.lpso_run.argtypes = [C.POINTER(Problem), C.POINTER(Options), C.c_int, C.c_void_p, C.c_int,
                                  _ip, _dp, _dp, _dp, _dp, _dp, _dp]
        _lib.lpso_build_horizons.restype = C.c_int
        _lib.lpso_build_horizons.argtypes = [C.c_int, _dp, C.c_double, C.c_int, _ip, _ip]
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None and a.size else None


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None and a.size else None


def run(s, n_steps=None, abcs_step=2, theta_method=1, kinematic_v=0, max_horizon=128,
        substep=30, n_threads=0):
    """Run the oracle on an InputSet; returns dict(status, diag, u, v, a, theta, m, elapsed)."""
    n_steps = s.n_steps if n_steps is None else n_steps
    keep = dict(nodes=np.ascontiguousarray(s.nodes, np.float64).ravel(),
                bct=np.ascontiguousarray(s.bctypes, np.int32), u0=np.ascontiguousarray(s.u0, np.float64),
                v0=np.ascontiguousarray(s.v0, np.float64),
                pre=np.ascontiguousarray(s.prenotch, np.float64).ravel(),
                inf=np.ascontiguousarray(s.inf_nodes, np.int32),
                clouds=np.ascontiguousarray(s.clouds, np.int32).ravel(),
                gu=np.ascontiguousarray(s.gu, np.float64).ravel(),
                gv=np.ascontiguousarray(s.gv, np.float64).ravel(),
                gth=np.ascontiguousarray(s.gtheta, np.float64).ravel())
    p = Problem(n_nodes=s.n_nodes, n_abc=s.n_abc, max_cloud=s.max_cloud, n_prenotch=s.n_prenotch,
                E=s.E, nu=s.nu, rho=s.rho, dt=s.dt, delta=s.delta, dx=s.dx, dy=s.dy,
                nodes=_d(keep["nodes"]), bctypes=_i(keep["bct"]), u0=_d(keep["u0"]), v0=_d(keep["v0"]),
                prenotch=_d(keep["pre"]), inf_nodes=_i(keep["inf"]), clouds=_i(keep["clouds"]),
                gu=_d(keep["gu"]), gv=_d(keep["gv"]), gtheta=_d(keep["gth"]))
    o = Options(abcs_step=abcs_step, theta_method=theta_method, kinematic_v=kinematic_v,
                max_horizon=max_horizon, substep=substep, n_threads=n_threads)
    max_diag = n_steps // max(substep, 1) + 1
    diag = np.zeros(max_diag, DIAG_DTYPE)
    nd = C.c_int(0)
    N = s.n_nodes
    u, v, a = np.zeros(2 * N), np.zeros(2 * N), np.zeros(2 * N)
    th, m = np.zeros(N), np.zeros(N)
    el = C.c_double(0.0)
    st = lib().lpso_run(C.byref(p), C.byref(o), n_steps, diag.ctypes.data_as(C.c_void_p), max_diag,
                        C.byref(nd), _d(u), _d(v), _d(a), _d(th), _d(m), C.byref(el))
    return dict(status=st, diag=diag[:nd.value], u=u, v=v, a=a, theta=th, m=m, elapsed=el.value)


def build_horizons(nodes: np.ndarray, radius: float, max_len: int = 128):
    nodes = np.ascontiguousarray(nodes, np.float64).ravel()
    n = nodes.size // 2
    lengths = np.zeros(n, np.int32)
    hz = np.zeros((n, max_len), np.int32)
    r = lib().lpso_build_horizons(n, _d(nodes), radius, max_len, _i(lengths), _i(hz))
    return r, lengths, hz


def read_state_dump(path: str):
    """Binary final-state dump of the checker build of the reference solver
    (written after the time loop): int32 N, u[2N], v[2N], a[2N], theta[N], m[N]."""
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw[:4], np.int32)[0])
    vals = np.frombuffer(raw[4:], np.float64)
    return dict(u=vals[:2 * n].copy(), v=vals[2 * n:4 * n].copy(), a=vals[4 * n:6 * n].copy(),
                theta=vals[6 * n:7 * n].copy(), m=vals[7 * n:8 * n].copy())
