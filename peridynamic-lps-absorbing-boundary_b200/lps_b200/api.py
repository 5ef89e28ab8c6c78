"""ctypes binding of the C ABI in include/lps_cuda.h (liblps_b200.so).

The library is built in-tree by ``__graft_entry__.build()`` (or ``make -C
peridynamic-lps-absorbing-boundary_b200/csrc``).  There is no CPU fallback:
if the shared library is missing or no sm_100 device is present, the calls
raise.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

from .files import InputSet

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "liblps_b200.so")

LPS_OK = 0
STATUS = {0: "LPS_OK", -1: "LPS_ERR_INVALID_ARG", -2: "LPS_ERR_HORIZON", -3: "LPS_ERR_NONFINITE",
          -4: "LPS_ERR_LAME", -5: "LPS_ERR_LAMBDA_PD", -6: "LPS_ERR_CUDA", -7: "LPS_ERR_NOMEM",
          -8: "LPS_ERR_UNSUPPORTED", -9: "LPS_ERR_NO_DEVICE"}
PRECISION = {"fp64": 0, "fp32_mixed": 1}
PATH = {"auto": 0, "dense": 1, "csr": 2}
PATH_NAME = {v: k for k, v in PATH.items()}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class LpsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class _Problem(C.Structure):
    _fields_ = [("n_nodes", C.c_int32), ("n_abc", C.c_int32), ("max_cloud", C.c_int32),
                ("n_prenotch", C.c_int32),
                ("E", C.c_double), ("nu", C.c_double), ("rho", C.c_double), ("dt", C.c_double),
                ("delta", C.c_double), ("dx", C.c_double), ("dy", C.c_double),
                ("nodes", _dp), ("bctypes", _ip), ("u0", _dp), ("v0", _dp), ("prenotch", _dp),
                ("inf_nodes", _ip), ("clouds", _ip), ("gu", _dp), ("gv", _dp), ("gtheta", _dp)]


class _Options(C.Structure):
    _fields_ = [("abcs_step", C.c_int32), ("theta_method", C.c_int32), ("kinematic_v", C.c_int32),
                ("max_horizon", C.c_int32), ("precision", C.c_int32), ("path", C.c_int32),
                ("device", C.c_int32), ("use_graphs", C.c_int32), ("stream", C.c_void_p),
                ("autotune", C.c_int32), ("theta_rows", C.c_int32), ("horizon_build", C.c_int32),
                ("force_rows", C.c_int32)]


DIAG_FIELDS = ("t", "E", "Ek", "Ep", "Px", "Py", "max_u", "max_v", "max_a",
               "theta_min", "theta_max", "uB_rms", "vB_rms", "dE_rel")


class _Diag(C.Structure):
    _fields_ = [(f, C.c_double) for f in DIAG_FIELDS] + [
        ("step", C.c_int32), ("max_u_node", C.c_int32), ("max_v_node", C.c_int32),
        ("n_active_abc", C.c_int32)]


DIAG_DTYPE = np.dtype([(f, np.float64) for f in DIAG_FIELDS] +
                      [("step", np.int32), ("max_u_node", np.int32), ("max_v_node", np.int32),
                       ("n_active_abc", np.int32)])


class _Info(C.Structure):
    _fields_ = [("n_instances", C.c_int32), ("path", C.c_int32), ("precision", C.c_int32),
                ("max_horizon_len", C.c_int32), ("total_nodes", C.c_int64), ("total_abc", C.c_int64),
                ("m_ref", C.c_double), ("m_min", C.c_double), ("lam", C.c_double), ("mu", C.c_double),
                ("kappa", C.c_double), ("alpha", C.c_double), ("lambda_pd", C.c_double),
                ("output_exclude_r", C.c_double), ("domain_radius", C.c_double), ("dt_lps", C.c_double),
                ("device_bytes", C.c_int64), ("step", C.c_int64), ("n_abc_m_corrected", C.c_int32),
                ("pad", C.c_int32), ("tile_ctas_theta", C.c_int32), ("tile_ctas_force", C.c_int32),
                ("tile_rows_theta", C.c_int32), ("tile_rows_force", C.c_int32), ("horizon_ms", C.c_double),
                ("horizon_on_gpu", C.c_int32), ("pad3", C.c_int32)]


class _KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_int32), ("pad", C.c_int32),
                ("total_ms", C.c_double)]


EXPORTED = ("lps_default_options", "lps_create", "lps_set_initial", "lps_reset", "lps_step",
            "lps_read_diag", "lps_download", "lps_synchronize", "lps_get_info", "lps_last_error",
            "lps_status_string", "lps_destroy", "lps_kernel_launches", "lps_profile_kernels")

_lib = None


def load_library(path: str = LIB_PATH):
    """Load liblps_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{path} not built; run __graft_entry__.build() or make -C {PKG_DIR}/csrc")
    lib = C.CDLL(path)
    lib.lps_default_options.argtypes = [C.POINTER(_Options)]
    lib.lps_default_options.restype = None
    lib.lps_create.argtypes = [C.POINTER(_Problem), C.c_int, C.POINTER(_Options), C.POINTER(C.c_void_p)]
    lib.lps_set_initial.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
    lib.lps_reset.argtypes = [C.c_void_p]
    lib.lps_step.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.lps_read_diag.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    lib.lps_download.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _dp]
    lib.lps_synchronize.argtypes = [C.c_void_p]
    lib.lps_get_info.argtypes = [C.c_void_p, C.c_int, C.POINTER(_Info)]
    lib.lps_last_error.argtypes = [C.c_void_p]
    lib.lps_last_error.restype = C.c_char_p
    lib.lps_status_string.argtypes = [C.c_int]
    lib.lps_status_string.restype = C.c_char_p
    lib.lps_destroy.argtypes = [C.c_void_p]
    lib.lps_destroy.restype = None
    lib.lps_kernel_launches.argtypes = [C.c_void_p]
    lib.lps_kernel_launches.restype = C.c_int64
    lib.lps_profile_kernels.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(_KernelTime), C.c_int,
                                        C.POINTER(C.c_int)]
    lib.lps_profile_kernels.restype = C.c_int
    for name in ("lps_create", "lps_set_initial", "lps_reset", "lps_step", "lps_read_diag",
                 "lps_download", "lps_synchronize", "lps_get_info"):
        getattr(lib, name).restype = C.c_int
    _lib = lib
    return lib


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None and a.size else None


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None and a.size else None


class Solver:
    """A batch of LPS instances on one GPU (one ``lps_handle``)."""

    def __init__(self, problems: Sequence[InputSet] | InputSet, abcs_step: int = 2,
                 theta_method: int = 1, kinematic_v: int = 0, max_horizon: int = 128,
                 precision: str = "fp64", path: str = "auto", device: int = 0,
                 use_graphs: bool = True, stream: int | None = None, autotune: bool = False,
                 theta_rows: int = 0, horizon_build: str = "auto", force_rows: int = 0):
        lib = load_library()
        if isinstance(problems, InputSet):
            problems = [problems]
        self._lib = lib
        self.sets = list(problems)
        self._keep = []
        arr = (_Problem * len(self.sets))()
        for k, s in enumerate(self.sets):
            keep = dict(nodes=np.ascontiguousarray(s.nodes, np.float64).ravel(),
                        bct=np.ascontiguousarray(s.bctypes, np.int32),
                        u0=np.ascontiguousarray(s.u0, np.float64), v0=np.ascontiguousarray(s.v0, np.float64),
                        pre=np.ascontiguousarray(s.prenotch, np.float64).ravel(),
                        inf=np.ascontiguousarray(s.inf_nodes, np.int32),
                        clouds=np.ascontiguousarray(s.clouds, np.int32).ravel(),
                        gu=np.ascontiguousarray(s.gu, np.float64).ravel(),
                        gv=np.ascontiguousarray(s.gv, np.float64).ravel(),
                        gth=np.ascontiguousarray(s.gtheta, np.float64).ravel())
            self._keep.append(keep)
            arr[k] = _Problem(n_nodes=s.n_nodes, n_abc=s.n_abc, max_cloud=s.max_cloud,
                              n_prenotch=s.n_prenotch, E=s.E, nu=s.nu, rho=s.rho, dt=s.dt,
                              delta=s.delta, dx=s.dx, dy=s.dy, nodes=_d(keep["nodes"]),
                              bctypes=_i(keep["bct"]), u0=_d(keep["u0"]), v0=_d(keep["v0"]),
                              prenotch=_d(keep["pre"]), inf_nodes=_i(keep["inf"]),
                              clouds=_i(keep["clouds"]), gu=_d(keep["gu"]), gv=_d(keep["gv"]),
                              gtheta=_d(keep["gth"]))
        o = _Options()
        lib.lps_default_options(C.byref(o))
        o.abcs_step, o.theta_method, o.kinematic_v = abcs_step, theta_method, kinematic_v
        o.max_horizon, o.precision, o.path = max_horizon, PRECISION[precision], PATH[path]
        o.device, o.use_graphs = device, int(use_graphs)
        o.stream = stream
        o.autotune = int(autotune)
        o.theta_rows = int(theta_rows)
        o.force_rows = int(force_rows)
        o.horizon_build = {"auto": 0, "host": 1, "gpu": 2}[horizon_build]
        h = C.c_void_p()
        st = lib.lps_create(arr, len(self.sets), C.byref(o), C.byref(h))
        if st != LPS_OK:
            raise LpsError(st, lib.lps_last_error(None).decode())
        self._h = h

    # -- helpers -------------------------------------------------------------
    def _check(self, st: int) -> None:
        if st != LPS_OK:
            raise LpsError(st, self._lib.lps_last_error(self._h).decode())

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.lps_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- API -----------------------------------------------------------------
    def set_initial(self, k: int, u0: np.ndarray | None = None, v0: np.ndarray | None = None) -> None:
        u = None if u0 is None else np.ascontiguousarray(u0, np.float64)
        v = None if v0 is None else np.ascontiguousarray(v0, np.float64)
        self._check(self._lib.lps_set_initial(self._h, k, _d(u), _d(v)))

    def reset(self) -> None:
        self._check(self._lib.lps_reset(self._h))

    def step(self, n: int, diag_every: int = 0) -> None:
        self._check(self._lib.lps_step(self._h, int(n), int(diag_every)))

    def synchronize(self) -> None:
        self._check(self._lib.lps_synchronize(self._h))

    def read_diag(self, k: int = 0, max_records: int = 1 << 20, check: bool = True) -> np.ndarray:
        out = np.zeros(max_records, DIAG_DTYPE)
        n = C.c_int(0)
        st = self._lib.lps_read_diag(self._h, k, out.ctypes.data_as(C.c_void_p), max_records, C.byref(n))
        if check or st != -3:
            self._check(st)
        return out[:n.value]

    def download(self, k: int = 0) -> dict:
        s = self.sets[k]
        N = s.n_nodes
        u, v, a = np.zeros(2 * N), np.zeros(2 * N), np.zeros(2 * N)
        th, m = np.zeros(N), np.zeros(N)
        self._check(self._lib.lps_download(self._h, k, _d(u), _d(v), _d(a), _d(th), _d(m)))
        return dict(u=u, v=v, a=a, theta=th, m=m)

    def download_into(self, k: int, u: np.ndarray | None = None, v: np.ndarray | None = None) -> None:
        self._check(self._lib.lps_download(self._h, k, _d(u), _d(v), None, None, None))

    def info(self, k: int = 0) -> dict:
        i = _Info()
        self._check(self._lib.lps_get_info(self._h, k, C.byref(i)))
        d = {f: getattr(i, f) for f, _ in _Info._fields_ if f != "pad"}
        d["path"] = PATH_NAME.get(d["path"], d["path"])
        return d

    def profile_kernels(self, n_steps: int, diag_every: int = 0) -> dict:
        """Run n_steps eager steps with CUDA events between the launches;
        returns {kernel: (launches, total_ms)}."""
        buf = (_KernelTime * 16)()
        n = C.c_int(0)
        self._check(self._lib.lps_profile_kernels(self._h, int(n_steps), int(diag_every), buf, 16,
                                                  C.byref(n)))
        return {buf[i].name.decode(): (buf[i].launches, buf[i].total_ms) for i in range(n.value)}

    def set_initial_ptr(self, k: int, u0_ptr: int, v0_ptr: int) -> None:
        """set_initial from raw host pointers (e.g. pinned torch tensors)."""
        self._check(self._lib.lps_set_initial(self._h, k, C.cast(C.c_void_p(u0_ptr), _dp),
                                              C.cast(C.c_void_p(v0_ptr), _dp)))

    def download_u_ptr(self, k: int, u_ptr: int) -> None:
        self._check(self._lib.lps_download(self._h, k, C.cast(C.c_void_p(u_ptr), _dp), None, None,
                                           None, None))

    @property
    def kernel_launches(self) -> int:
        return int(self._lib.lps_kernel_launches(self._h))
