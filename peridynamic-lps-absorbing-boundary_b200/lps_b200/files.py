"""Reader and writer for the solver's input file set and its log files.

The file set is the contract between the reference preprocessor and the
reference solver (whitespace-separated text):

=================  ==========================================  ======================
file               content                                      reference reader
=================  ==========================================  ======================
``.data1``         NodeNo StepNo PrenotchNo VINodesNo            src/main.cpp:178,195-200
                   constrainsNo maxCloudSize
``.data2``         E nu rho wf t0 t1 dt delta dx dy s0           src/main.cpp:186-212
                   [m_ref kappa alpha lambda_pd]
``.nodes``         N x 2 coordinates                             src/main.cpp:231
``.bctypes``       2N ints (1 = absorbing node)                  src/main.cpp:235
``.bcvalues``      2N doubles (unused by the time loop)          src/main.cpp:239
``.icvalues``      2N initial displacement, x/y interleaved      src/main.cpp:247
``.icdvalues``     2N initial velocity                           src/main.cpp:243
``.prenotch``      P x 4 crack segments                          src/main.cpp:252-254
``.vinodes``       V ints (unused)                               src/main.cpp:255-257
``.infNodesIndex`` NA node indices of absorbing nodes            src/main.cpp:276-280
``.iClouds``       NA x C cloud indices, -1 padded               src/main.cpp:271-275
``.ciNodesU/V``    2NA x 2*ABCS_STEP*C  G_u / G_v                src/main.cpp:261-270
``.ciNodesTheta``  NA x ABCS_STEP*C  G_theta                     src/main.cpp:281-292
=================  ==========================================  ======================

Writers use 16 significant digits, as preprocessor/main.cpp:1308-1453 does.
Unlike the reference readers (src/helpers/utils.h:25-80), a file that holds
fewer values than its header promises is an error here.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np


class InputSetError(ValueError):
    """An input file is missing or shorter than the counts in ``.data1`` say."""


@dataclass
class InputSet:
    n_nodes: int
    n_steps: int
    n_abc: int
    max_cloud: int
    E: float
    nu: float
    rho: float
    dt: float
    delta: float
    dx: float
    dy: float
    nodes: np.ndarray                      # (N, 2) float64
    bctypes: np.ndarray                    # (2N,) int32
    u0: np.ndarray                         # (2N,) float64
    v0: np.ndarray                         # (2N,) float64
    wf: float = 0.0
    t0: float = 0.0
    t1: float = 0.0
    s0: float = 0.0
    data2_extra: np.ndarray = field(default_factory=lambda: np.zeros(0))
    bcvalues: np.ndarray | None = None
    prenotch: np.ndarray = field(default_factory=lambda: np.zeros((0, 4)))
    vinodes: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    inf_nodes: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    clouds: np.ndarray = field(default_factory=lambda: np.zeros((0, 0), np.int32))
    gu: np.ndarray = field(default_factory=lambda: np.zeros((0, 0)))
    gv: np.ndarray = field(default_factory=lambda: np.zeros((0, 0)))
    gtheta: np.ndarray = field(default_factory=lambda: np.zeros((0, 0)))

    @property
    def n_prenotch(self) -> int:
        return int(self.prenotch.shape[0])


def _read_numbers(path: str, count: int, what: str) -> np.ndarray:
    if not os.path.exists(path):
        raise InputSetError(f"Cannot read {path}")
    if count == 0:
        return np.zeros(0)
    vals = np.fromfile(path, sep=" ") if os.path.getsize(path) else np.zeros(0)
    if vals.size < count:
        raise InputSetError(f"{path}: expected {count} values for {what}, found {vals.size}")
    return vals[:count]


def _round_int(a: np.ndarray) -> np.ndarray:
    # Integer index files are read as double and rounded, src/helpers/utils.h:61,76.
    return np.floor(a + 0.5).astype(np.int32)


def read_input_set(job: str, abcs_step: int = 2, theta_method: int = 1) -> InputSet:
    """Read ``<job>.*`` like src/main.cpp:176-293 (strict about short files)."""
    d1 = _read_numbers(job + ".data1", 6, "control data")
    n_nodes, n_steps, n_pre, n_vi, n_abc, max_cloud = (int(round(x)) for x in d1)
    if not os.path.exists(job + ".data2"):
        raise InputSetError(f"Cannot read {job}.data2")
    d2 = np.fromfile(job + ".data2", sep=" ")
    if d2.size < 11:
        raise InputSetError(f"{job}.data2: expected 11 or 15 values, found {d2.size}")
    nodes = _read_numbers(job + ".nodes", 2 * n_nodes, "nodes").reshape(n_nodes, 2)
    bct = _round_int(_read_numbers(job + ".bctypes", 2 * n_nodes, "bctypes"))
    bcv = _read_numbers(job + ".bcvalues", 2 * n_nodes, "bcvalues")
    v0 = _read_numbers(job + ".icdvalues", 2 * n_nodes, "icdvalues")
    u0 = _read_numbers(job + ".icvalues", 2 * n_nodes, "icvalues")
    s = InputSet(n_nodes=n_nodes, n_steps=n_steps, n_abc=n_abc, max_cloud=max_cloud,
                 E=d2[0], nu=d2[1], rho=d2[2], wf=d2[3], t0=d2[4], t1=d2[5], dt=d2[6],
                 delta=d2[7], dx=d2[8], dy=d2[9], s0=d2[10], data2_extra=d2[11:15].copy(),
                 nodes=nodes, bctypes=bct, bcvalues=bcv, u0=u0, v0=v0)
    if n_pre > 0:
        s.prenotch = _read_numbers(job + ".prenotch", 4 * n_pre, "prenotch").reshape(n_pre, 4)
    if n_vi > 0:
        s.vinodes = _round_int(_read_numbers(job + ".vinodes", n_vi, "vinodes"))
    if abcs_step != -1 and n_abc > 0:
        cpc = 2 if abcs_step == 1 else 4
        s.gu = _read_numbers(job + ".ciNodesU", 2 * n_abc * cpc * max_cloud, "G_u").reshape(2 * n_abc, cpc * max_cloud)
        s.gv = _read_numbers(job + ".ciNodesV", 2 * n_abc * cpc * max_cloud, "G_v").reshape(2 * n_abc, cpc * max_cloud)
        s.clouds = _round_int(_read_numbers(job + ".iClouds", n_abc * max_cloud, "iClouds")).reshape(n_abc, max_cloud)
        s.inf_nodes = _round_int(_read_numbers(job + ".infNodesIndex", n_abc, "infNodesIndex"))
        if theta_method == 1:
            s.gtheta = _read_numbers(job + ".ciNodesTheta", n_abc * abs(abcs_step) * max_cloud,
                                     "G_theta").reshape(n_abc, abs(abcs_step) * max_cloud)
    return s


def _write_lines(path: str, arr: np.ndarray, fmt: str) -> None:
    arr = np.asarray(arr)
    with open(path, "w") as f:
        if arr.ndim == 1:
            if arr.size:
                f.write("\n".join(fmt % v for v in arr.tolist()))
                f.write("\n")
        else:
            for row in arr.tolist():
                f.write(" ".join(fmt % v for v in row))
                f.write("\n")


def write_input_set(job: str, s: InputSet) -> None:
    """Write ``<job>.*`` in the layout preprocessor/main.cpp:1294-1453 writes."""
    d = os.path.dirname(job)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(job + ".data1", "w") as f:
        f.write("%d\n%d\n%d\n%d\n%d\n%d\n" % (s.n_nodes, s.n_steps, s.n_prenotch, s.vinodes.size,
                                             s.n_abc, s.max_cloud))
    d2 = [s.E, s.nu, s.rho, s.wf, s.t0, s.t1, s.dt, s.delta, s.dx, s.dy, s.s0] + list(s.data2_extra)
    _write_lines(job + ".data2", np.array(d2), "%.16g")
    _write_lines(job + ".nodes", s.nodes, "%.16g")
    _write_lines(job + ".bctypes", s.bctypes.astype(np.int64), "%d")
    bcv = s.bcvalues if s.bcvalues is not None else np.zeros(2 * s.n_nodes)
    _write_lines(job + ".bcvalues", bcv, "%.16g")
    _write_lines(job + ".icvalues", s.u0, "%.16g")
    _write_lines(job + ".icdvalues", s.v0, "%.16g")
    _write_lines(job + ".prenotch", s.prenotch, "%.16g")
    _write_lines(job + ".vinodes", s.vinodes.astype(np.int64), "%d")
    if s.n_abc > 0:
        _write_lines(job + ".infNodesIndex", s.inf_nodes.astype(np.int64), "%d")
        _write_lines(job + ".iClouds", s.clouds.astype(np.int64), "%d")
        _write_lines(job + ".ciNodesU", s.gu, "%.16g")
        _write_lines(job + ".ciNodesV", s.gv, "%.16g")
        if s.gtheta.size:
            _write_lines(job + ".ciNodesTheta", s.gtheta, "%.16g")


ENERGY_COLUMNS = ("t", "E", "Ek", "Ep", "Px", "Py", "max_u", "theta_max", "uB_rms", "vB_rms")
VERIFY_COLUMNS = ("t", "E", "dE_rel", "Px", "Py", "theta_max", "max_u", "max_v", "max_a")


def read_log(path: str) -> np.ndarray:
    """Read a ``.energy`` or ``.verify`` log (``#`` header line, then rows)."""
    rows = []
    with open(path) as f:
        for line in f:
            if line.startswith("#") or not line.strip():
                continue
            rows.append([float(x) for x in line.split()])
    return np.array(rows, dtype=np.float64).reshape(len(rows), -1)
