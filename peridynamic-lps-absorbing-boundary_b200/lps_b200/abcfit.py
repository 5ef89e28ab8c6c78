"""ctypes binding of the absorbing-boundary operator fit (include/lps_abcfit.h).

``fit`` computes the preprocessor's least-squares updating vectors G_u, G_v
and G_theta, and by default its (dt, delta_kappa) stability sweep, for any
disc's ring and clouds (preprocessor/main.cpp:809-1268).  It runs on the host
cores; LAPACK dgelsd comes from scipy's bundled OpenBLAS (the library the
reference preprocessor is linked against in this build), held to one thread
per call while the fit runs its own threads.
"""
from __future__ import annotations

import ctypes as C
import glob
import os

import numpy as np

from .api import LIB_PATH

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class _Params(C.Structure):
    _fields_ = [("E", C.c_double), ("nu", C.c_double), ("rho", C.c_double), ("delta", C.c_double),
                ("dx", C.c_double), ("dy", C.c_double), ("abcs_step", C.c_int32), ("sweep", C.c_int32),
                ("dt", C.c_double), ("dk_factor", C.c_double), ("n_threads", C.c_int32), ("pad", C.c_int32)]


class _Result(C.Structure):
    _fields_ = [("dt", C.c_double), ("delta_kappa", C.c_double), ("dk_factor", C.c_double),
                ("sweep_max_g", C.c_double), ("max_norm_gu", C.c_double), ("max_norm_gv", C.c_double),
                ("max_norm_gtheta", C.c_double), ("m_ref", C.c_double), ("n_steps", C.c_int32),
                ("n_modes", C.c_int32), ("n_failed", C.c_int32), ("stable_found", C.c_int32),
                ("dgelsd_failures", C.c_int32), ("pad", C.c_int32)]


_state = {}


def _library():
    if "lib" not in _state:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} not built")
        lib = C.CDLL(LIB_PATH)
        lib.lps_abcfit.argtypes = [C.POINTER(_Params), _dp, C.c_int32, _ip, C.c_int32, _ip, C.c_int32, C.c_void_p,
                                   _dp, _dp, _dp, C.POINTER(_Result)]
        lib.lps_abcfit.restype = C.c_int
        _state["lib"] = lib
    return _state["lib"]


def lapack_dgelsd():
    """Address of scipy's bundled OpenBLAS dgelsd (Fortran convention)."""
    if "dgelsd" not in _state:
        import scipy
        import scipy.linalg  # noqa: F401  (loads the library so threadpoolctl sees it)
        libdir = os.path.dirname(scipy.__file__) + ".libs"
        libs = sorted(glob.glob(os.path.join(libdir, "libscipy_openblas*.so")))
        if not libs:
            raise OSError(f"no scipy OpenBLAS under {libdir}")
        blas = C.CDLL(libs[0])
        _state["blas"] = blas
        _state["dgelsd"] = C.cast(blas.scipy_dgelsd_, C.c_void_p).value
    return _state["dgelsd"]


def fit(nodes, inf_nodes, clouds, E, nu, rho, delta, dx, dy=None, abcs_step=2, sweep=True, dt=None,
        dk_factor=1.0, n_threads=0):
    """Fit the operators of the ABC nodes inf_nodes with clouds [n_abc, C]
    (node indices, -1 padded).  Returns a dict with gu, gv [2 n_abc, 2 S C],
    gtheta [n_abc, S C] (S = abcs_step) and the chosen dt, delta_kappa,
    dk_factor, n_steps (ceil(210 us / dt)) and the norms of the result."""
    dy = dx if dy is None else dy
    nodes = np.ascontiguousarray(nodes, np.float64).reshape(-1, 2)
    inf_nodes = np.ascontiguousarray(inf_nodes, np.int32)
    clouds = np.ascontiguousarray(clouds, np.int32)
    NA, Cw = clouds.shape
    S = abs(abcs_step)
    gu = np.zeros((2 * NA, 2 * S * Cw))
    gv = np.zeros((2 * NA, 2 * S * Cw))
    gth = np.zeros((NA, S * Cw))
    if not sweep and dt is None:
        raise ValueError("sweep=False needs dt")
    p = _Params(E=E, nu=nu, rho=rho, delta=delta, dx=dx, dy=dy, abcs_step=S, sweep=1 if sweep else 0,
                dt=dt or 0.0, dk_factor=dk_factor, n_threads=n_threads, pad=0)
    r = _Result()
    fn = lapack_dgelsd()
    from threadpoolctl import threadpool_limits
    with threadpool_limits(limits=1, user_api="blas"):
        st = _library().lps_abcfit(C.byref(p), nodes.ctypes.data_as(_dp), nodes.shape[0],
                                   inf_nodes.ctypes.data_as(_ip), NA, clouds.ctypes.data_as(_ip), Cw, fn,
                                   gu.ctypes.data_as(_dp), gv.ctypes.data_as(_dp), gth.ctypes.data_as(_dp),
                                   C.byref(r))
    if st != 0:
        raise ValueError("lps_abcfit: bad argument")
    out = {f: getattr(r, f) for f, _ in _Result._fields_ if f != "pad"}
    out.update(gu=gu, gv=gv, gtheta=gth)
    return out
