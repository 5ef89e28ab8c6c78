"""The command-line drop-in PD2_LPS_ABC_B200 (csrc/pd2_lps_abc_b200.cpp).

CPU tests cover what happens before any device work: usage, the input file
checks and the error exit without a device.  The GPU tests run it on an
input set of the reference preprocessor and compare its .energy, .verify and
VTK files with the ones the compiled reference wrote for the same inputs
(tests/golden/r10_stock.npz): same layout line by line, numbers within the
FP64 parity bars.
"""
import os
import subprocess

import numpy as np
import pytest

from golden_io import load_golden, load_inputs
from lps_b200.files import write_input_set

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "peridynamic-lps-absorbing-boundary_b200", "PD2_LPS_ABC_B200")


def run_exe(cwd, *args):
    if not os.path.exists(EXE):
        pytest.fail("PD2_LPS_ABC_B200 is not built (make -C peridynamic-lps-absorbing-boundary_b200/csrc)")
    return subprocess.run([EXE, *args], cwd=cwd, capture_output=True, text=True, timeout=600)


def test_usage_exits_zero(tmp_path):
    r = run_exe(tmp_path)
    assert r.returncode == 0 and "Usage:" in r.stdout


def test_short_input_file_is_fatal(tmp_path):
    s = load_inputs("r10")
    write_input_set(str(tmp_path / "r10"), s)
    lines = open(tmp_path / "r10.icvalues").read().splitlines()
    open(tmp_path / "r10.icvalues", "w").write("\n".join(lines[: len(lines) // 2]) + "\n")
    r = run_exe(tmp_path, "_x", "r10")
    assert r.returncode == 1
    assert "FATAL: Cannot read r10.icvalues" in r.stderr


def test_missing_input_file_is_fatal(tmp_path):
    r = run_exe(tmp_path, "_x", "nothing")
    assert r.returncode == 1
    assert "FATAL: Cannot read nothing.data1" in r.stderr


def test_without_device_exits_one(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    write_input_set(str(tmp_path / "r10"), load_inputs("r10"))
    r = run_exe(tmp_path, "_x", "r10")
    assert r.returncode == 1
    assert "no CUDA device" in r.stderr


def _numbers(text):
    out = []
    for ln in text.splitlines():
        if ln.startswith("#"):
            continue
        out.append([float(x) for x in ln.split()])
    return np.array(out)


def _split_vtk(raw):
    """Lines of a legacy VTK file: (layout lines, data lines as numbers)."""
    lines = raw.splitlines()
    layout, data = [], []
    section = None
    for ln in lines:
        head = ln.split(" ")[0]
        if head in ("VECTORS", "SCALARS", "LOOKUP_TABLE", "POINT_DATA", "VERTICES", "POINTS", "#", "DATASET",
                    "ASCII", "PD2_LPS_ABC"):
            layout.append(ln)
            section = head
        elif section in ("VECTORS", "LOOKUP_TABLE"):
            data.append([float(x) for x in ln.split()])
        else:
            layout.append(ln)   # coordinates and connectivity: exact
    return layout, data


@pytest.mark.gpu
@pytest.mark.parametrize("path", ["dense", "csr"])
def test_outputs_match_reference_files(tmp_path, path):
    s = load_inputs("r10")
    g = load_golden("r10_stock")
    write_input_set(str(tmp_path / "r10"), s)
    r = run_exe(tmp_path, "_stock", "r10", "--path", path)
    assert r.returncode == 0, r.stderr
    assert "Time marching took" in r.stdout
    for ext, key in ((".energy", "energy_text"), (".verify", "verify_text")):
        ours = open(tmp_path / f"r10_stock{ext}").read()
        ref = bytes(g[key]).decode()
        assert ours.splitlines()[0] == ref.splitlines()[0]
        assert len(ours.splitlines()) == len(ref.splitlines())
        a, b = _numbers(ours), _numbers(ref)
        assert a.shape == b.shape
        np.testing.assert_array_equal(a[:, 0], b[:, 0])          # t
        scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
        assert np.max(np.abs(a - b) / scale) <= 1e-9, ext
    for name, key in (("r10_stock-0.vtk", "vtk_0"), ("r10_stock-600.vtk", "vtk_600"),
                      ("r10_stock-vel-600.vtk", "vtk_vel_600"), ("r10_stock-theta-600.vtk", "vtk_theta_600")):
        lo, do = _split_vtk(open(tmp_path / name).read())
        lr, dr = _split_vtk(bytes(g[key]).decode())
        assert lo == lr, name
        do, dr = np.array(do, dtype=object), np.array(dr, dtype=object)
        assert len(do) == len(dr)
        x = np.concatenate([np.asarray(v, float) for v in do])
        y = np.concatenate([np.asarray(v, float) for v in dr])
        assert np.max(np.abs(x - y)) <= 1e-9 * max(np.max(np.abs(y)), 1e-300), name


@pytest.mark.gpu
def test_nonfinite_state_is_fatal(tmp_path):
    # a displacement whose energy overflows to Inf at the first output step
    # (a NaN cannot be written into the text files the solver reads)
    s = load_inputs("r10")
    s.u0 = s.u0.copy()
    s.u0[5] = 1e300
    write_input_set(str(tmp_path / "r10"), s)
    r = run_exe(tmp_path, "_nan", "r10", "--no-vtk")
    assert r.returncode == 1
    assert "FATAL: Energy is NaN/Inf at step 30!" in r.stderr
    # the record of the failing step is written before the exit, as the reference does
    assert len(open(tmp_path / "r10_nan.energy").read().splitlines()) == 2


@pytest.mark.gpu
def test_async_and_sync_output_write_the_same_bytes(tmp_path):
    """The background VTK writer (default) and --sync-output (each output
    step's files written before the next steps) produce identical files."""
    s = load_inputs("r10")
    for mode in ("async", "sync"):
        d = tmp_path / mode
        d.mkdir()
        write_input_set(str(d / "r10"), s)
        extra = ["--sync-output"] if mode == "sync" else ["--output-threads", "3"]
        r = run_exe(d, "_o", "r10", *extra)
        assert r.returncode == 0, r.stderr
    names = sorted(f for f in os.listdir(tmp_path / "async") if f.startswith("r10_o"))
    assert len(names) == 2 + 1 + 3 * (s.n_steps // 30)
    assert names == sorted(f for f in os.listdir(tmp_path / "sync") if f.startswith("r10_o"))
    for f in names:
        assert open(tmp_path / "async" / f, "rb").read() == open(tmp_path / "sync" / f, "rb").read(), f
