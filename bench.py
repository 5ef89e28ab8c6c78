#!/usr/bin/env python
"""Benchmark of the LPS time marcher: node-steps/s on B200.

Workload (default ``poisson7``): the Poisson-ratio batch -- seven instances of
the Example 1 geometry (R=125 mm, dx=0.5 mm, m=4: 196,321 nodes, 6,268
absorbing nodes, cloud size 49 each) with nu in {0.15,...,0.45}, a radial
Gaussian pulse (A=1e-3 mm, sigma=40/3 mm), run together in one handle for
4000 time steps with diagnostics every 30 steps (the reference's output
cadence, src/main.cpp:34,981).  One bench step = one complete run of the batch
from its initial state.  Inputs are synthetic (lps_b200.gen, lps_b200.configs):
geometry, rings and clouds equal the reference preprocessor's, and each
instance carries its own least-squares absorbing operators, time step and
wavenumber range from the preprocessor's stability sweep (lps_b200.abcfit);
the 64-instance batch alone uses passive averaging operators of the same
shape.

``--impl reference`` times the reference solver itself (compiled from its
sources into oracle/_ref/, output off) on the host cores instead.

Timing: W untimed bench steps, then K timed ones bracketed by a barrier and
cuda synchronize, CUDA events on the solver's stream, max over ranks; L2 is
flushed (256 MiB write) before every timed run, and the per-run working set
(about 540 MB) exceeds L2 anyway.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "peridynamic-lps-absorbing-boundary_b200")
sys.path.insert(0, PKG)

METRIC = "node-steps/s on 1 B200: FP64 plain vs FP32-mixed batched at ≤1e-5 rel L2 err"
NUS = (0.15, 0.20, 0.25, 0.30, 0.35, 0.40, 0.45)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["poisson7", "example1", "large", "uneven64", "horizon8"],
                    default="poisson7",
                    help="poisson7: the 7-instance Poisson-ratio batch (the headline); example1, large "
                         "(12.57 M nodes), uneven64 (64-instance batch), horizon8 (m=8): the other "
                         "benchmark configurations")
    ap.add_argument("--time-steps", type=int, default=None,
                    help="time steps per bench step (default: the configuration's own count)")
    ap.add_argument("--diag-every", type=int, default=30)
    ap.add_argument("--precision", choices=["both", "fp64", "fp32_mixed"], default="both",
                    help="both: the FP32-mixed form is the headline value, the FP64 plain form "
                         "is timed beside it on the same workload")
    ap.add_argument("--path", default="auto")
    ap.add_argument("--cpu-sample-steps", type=int, default=None,
                    help="time steps of the CPU sample (default: about 1.2e8 bond-weighted node-steps, "
                         "10-20 s on 16 host cores)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep full occupancy instead of searching the tile kernels' resident CTAs at "
                         "setup (for launch lists whose first launches should be the time steps)")
    return ap.parse_args()


WORKLOAD_TEXT = {
    "poisson7": "Poisson-ratio batch: 7 x Example-1 disc (R=125 mm, dx=0.5 mm, m=4), nu 0.15..0.45",
    "example1": "Example 1 disc (R=125 mm, dx=0.5 mm, m=4, nu=0.25)",
    "large": "large single domain (R=500 mm, dx=0.25 mm, m=4, nu=0.30, 12.57 M nodes)",
    "uneven64": "uneven batch of 64 discs (R 50..250 mm, dx=0.5 mm, m 3..5, seed 20261203)",
    "horizon8": "large-horizon disc (R=250 mm, dx=0.5 mm, m=8: 224 neighbours, nu=0.40)",
}
NEIGHBOURS = {3: 36, 4: 68, 5: 96, 8: 224}
_LSQ = ("synthetic, seeded (generated geometry, ring and clouds as the reference preprocessor builds them; "
        "least-squares absorbing operators, dt and delta_kappa from its stability sweep, per instance)")
DATA_TEXT = {"poisson7": _LSQ, "example1": _LSQ, "large": _LSQ, "horizon8": _LSQ,
             "uneven64": "synthetic, seeded (generated geometry, ring and clouds; passive averaging absorbing "
                         "operators of the same shape, dt = 17.5 ns)"}


def workload_sets(name, n_steps):
    from lps_b200 import configs
    return configs.build(name, n_steps)


def workload_config(name, sets, args):
    nb = sorted({NEIGHBOURS.get(int(round(s.delta / s.dx)), None) for s in sets}, key=str)
    return {"workload": WORKLOAD_TEXT[name],
            "instances": len(sets), "nodes": sum(s.n_nodes for s in sets),
            "nodes_per_instance": sets[0].n_nodes if len(sets) < 8 else [min(s.n_nodes for s in sets),
                                                                          max(s.n_nodes for s in sets)],
            "abc_nodes": sum(s.n_abc for s in sets), "cloud_size": max(s.max_cloud for s in sets),
            "neighbours": nb[0] if len(nb) == 1 else nb, "time_steps_per_run": args.time_steps,
            "diag_every": args.diag_every,
            "precision": ("fp32_mixed (value), fp64 (beside it)" if args.precision == "both"
                          else args.precision), "path": args.path,
            "l2": "flushed (256 MiB write) before each timed run; working set > L2"}


# ---------------------------------------------------------------------------
# CPU reference timing (the reference's own solver, compiled from its sources)
def reference_cpu(s, n_steps, threads):
    """Run oracle/_ref/PD2_LPS_ABC_timing on set s for n_steps; returns
    (node_steps_per_s, seconds, kind) or None when the binary is missing."""
    from lps_b200.files import write_input_set
    wide = int(round(s.delta / s.dx)) > 5   # m=8: 225 horizon entries need MAX_HORIZON_LENGTH=256
    binary = os.path.join(ROOT, "oracle", "_ref", "PD2_LPS_ABC_timing256" if wide else "PD2_LPS_ABC_timing")
    if not os.path.exists(binary):
        return None
    work = tempfile.mkdtemp(prefix="lps_ref_")
    try:
        s = _copy_steps(s, n_steps)
        job = os.path.join(work, "ex")
        write_input_set(job, s)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        r = subprocess.run([binary, "_t", "ex"], cwd=work, env=env, capture_output=True, text=True)
        m = re.search(r"Time marching took ([0-9.eE+-]+) seconds", r.stdout)
        if r.returncode != 0 or not m:
            raise RuntimeError(f"reference solver failed: {r.stdout[-500:]} {r.stderr[-500:]}")
        sec = float(m.group(1))
        return s.n_nodes * n_steps / sec, sec
    finally:
        shutil.rmtree(work, ignore_errors=True)


def _copy_steps(s, n_steps):
    import copy
    t = copy.copy(s)
    t.n_steps = n_steps
    return t


def oracle_cpu(s, n_steps, threads):
    """Fallback CPU leg: the C restatement (oracle/liblps_oracle.so)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_ctypes
    r = oracle_ctypes.run(s, n_steps=n_steps, substep=10 ** 9, n_threads=threads, max_horizon=256)
    return s.n_nodes * n_steps / r["elapsed"], r["elapsed"]


CPU_MAX_NODES = 2_000_000


def cpu_sample(sets, args):
    """The instance the CPU legs time and their step count: the nu=0.25
    instance where there is one (else the first), for about 1.2e8
    neighbour-weighted node-steps unless --cpu-sample-steps is given.  An
    instance above CPU_MAX_NODES nodes (the 12.57 M-node domain) is timed on a
    proxy: a disc of the same dx, horizon, nu and dt with 196,321 nodes (R = 250 dx),
    because the reference's own setup (reading the text files and its k-d tree
    horizon search) takes longer than the whole bench for 12.57 M nodes; its
    time-marching rate per node-step does not depend on the disc's size.
    Returns (set, steps, note)."""
    s = next((t for t in sets if abs(t.nu - 0.25) < 1e-12), sets[0])
    note = ""
    if s.n_nodes > CPU_MAX_NODES:
        from lps_b200 import gen
        m = int(round(s.delta / s.dx))
        R = 250.0 * s.dx
        s = gen.disc_problem(R=R, dx=s.dx, m=m, nu=s.nu, E=s.E, rho=s.rho, dt=s.dt, n_steps=1, abc="average")
        note = f" (proxy disc R={R:g} mm of the same dx, m, nu and dt: the workload's own instance is too large " \
               f"for the reference's setup within the bench)"
    if args.cpu_sample_steps:
        return s, args.cpu_sample_steps, note
    w = NEIGHBOURS.get(int(round(s.delta / s.dx)), 68) / 68.0
    return s, max(10, int(round(1.2e8 / (s.n_nodes * w)))), note


def cpu_leg(s, n_steps, threads):
    res = reference_cpu(s, n_steps, threads)
    if res is not None:
        return res + ("reference",)
    return oracle_cpu(s, n_steps, threads) + ("port",)


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        uuid = str(uuid)
        self.uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
        self.proc, self.lines = None, []

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        cmd = ["nvidia-smi", f"--id={self.uuid}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
               "-lms", "200"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(sets, kernel, precision="fp64"):
    """Compulsory DRAM bytes of one launch of `kernel` in this build's layout
    (each array read or written once per launch).  Returns (bytes,
    grading_bytes): the second is the per-node figure the roofline is graded
    against (force pass 80 B/node FP64, 56 B/node FP32-mixed; step 168 B/node
    FP64, 140 B/node FP32-mixed; + 148 C B per ABC node), or None where that
    figure does not apply."""
    n = sum(s.n_nodes for s in sets)
    abc = sum(s.n_abc * s.max_cloud for s in sets)
    f32 = precision == "fp32_mixed"
    step_node = 140 if f32 else 168
    table = {
        # an ordinary (not full) step at an interior node -- v, a and theta are
        # written only where later steps read them, and on full steps:
        # FP64: read u_pred 16, theta 8, coef 16, vh 16; write vh 16,
        # u_pred(next) 16.  FP32-mixed: read u_pred32 8, A' 4, vh 16, u_pred 16;
        # write vh 16, u_pred(next) 16, u_pred32(next) 8
        "force_tiles": ((84 if f32 else 88) * n, (56 if f32 else 80) * n),
        # dilatation: FP64 read u_pred 16, m 8, write theta 8; FP32-mixed read
        # u_pred32 8, write A' 4 (full tiles need no m and no B')
        "theta_tiles": ((12 if f32 else 32) * n, None),
        # G_u, G_v of the step and G_theta of the next: 18C doubles + 4C index
        # bytes per ABC node (the gathered state hits L2)
        "abc_sell": (148 * abc, 148 * abc),
        # neighbour-list path
        "predict_csr": (80 * n, None),
        "theta_csr": (32 * n, None),
        "force_csr": (80 * n + 132 * abc, 80 * n),
        # end-of-step ABC merge + prediction: read s 16, v 16, a 16; write
        # u 16, u_pred 16, vh 16 (+ u_pred32 8) per ABC node
        "abc_predict": (sum(s.n_abc for s in sets) * (104 if f32 else 96), None),
        "step": (step_node * n + 148 * abc, step_node * n + 148 * abc),
    }
    return table.get(kernel, (None, None))


def measured_traffic(kernel, precision, workload):
    """DRAM bytes per launch of `kernel` on `workload` from the committed ncu
    summaries (profiles/ncu_traffic.json), if listed."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p)).get(workload, {})
    return d.get(precision, {}).get(kernel, {}).get("dram_bytes_per_launch")


# ---------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank, precision, with_cpu=True):
    import numpy as np
    import torch
    import torch.distributed as dist
    from lps_b200.api import Solver
    from lps_b200.shard import job_time_ms

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    sets = workload_sets(args.workload, args.time_steps)
    stream = torch.cuda.Stream(device=dev)
    wide = max(int(round(s.delta / s.dx)) for s in sets) > 5  # m = 8: 225 horizon entries
    sv = Solver(sets, precision=precision, path=args.path, device=local_rank,
                stream=stream.cuda_stream, autotune=not args.no_autotune, max_horizon=256 if wide else 128)
    info = sv.info(0)
    T, K, W = args.time_steps, args.steps, args.warmup
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def one_run():
        sv.reset()
        sv.step(T, diag_every=args.diag_every)

    for _ in range(W):
        one_run()
        for k in range(len(sets)):
            sv.read_diag(k)
    barrier()
    clocks = ClockSampler(str(torch.cuda.get_device_properties(dev).uuid))
    if rank == 0 or world > 1:
        clocks.start()
    launches0 = sv.kernel_launches
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    barrier()
    for i in range(K):
        with torch.cuda.stream(stream):
            flush.fill_(float(i))
        ev[i][0].record(stream)
        one_run()
        ev[i][1].record(stream)
    barrier()
    launches = sv.kernel_launches - launches0
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    final_dE, final_u = [], []
    for k in range(len(sets)):
        d = sv.read_diag(k)
        final_dE.append(float(d["dE_rel"][-1]) if len(d) else None)
        final_u.append(sv.download(k)["u"])
    ms_max = job_time_ms(ms, device=dev)   # max over ranks
    node_steps = world * sum(s.n_nodes for s in sets) * T * K
    value = node_steps / (ms_max / 1e3)

    # ---- end to end through the C ABI: host inputs in, host results out ----
    pin_u0 = [torch.from_numpy(np.ascontiguousarray(s.u0)).pin_memory() for s in sets]
    pin_v0 = [torch.from_numpy(np.ascontiguousarray(s.v0)).pin_memory() for s in sets]
    pin_out = [torch.empty(2 * s.n_nodes, dtype=torch.float64).pin_memory() for s in sets]
    barrier()
    # CUDA events on the solver's stream; the host-side work of each call
    # (scatter, copies, log reads) lies between them on the device timeline
    e2e_ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    e2e_ev[0].record(stream)
    n_rec = 0
    for _ in range(K):
        for k in range(len(sets)):
            sv.set_initial_ptr(k, pin_u0[k].data_ptr(), pin_v0[k].data_ptr())
        sv.reset()
        sv.step(T, diag_every=args.diag_every)
        for k in range(len(sets)):
            n_rec += len(sv.read_diag(k))
            sv.download_u_ptr(k, pin_out[k].data_ptr())
    e2e_ev[1].record(stream)
    barrier()
    e2e_value = node_steps / (job_time_ms(e2e_ev[0].elapsed_time(e2e_ev[1]), device=dev) / 1e3)
    h2d = sum(2 * 2 * s.n_nodes * 8 for s in sets)
    d2h = sum(2 * s.n_nodes * 8 for s in sets) + (n_rec // K) * 128

    # ---- per-kernel device times (live, CUDA events on the same stream) ----
    sv.reset()
    prof = sv.profile_kernels(120, diag_every=args.diag_every)
    sv.close()
    top = max(prof.items(), key=lambda kv: kv[1][1])
    name, (nl, tot) = top
    per_launch_ms = tot / nl
    ab, ab_grade = algorithmic_bytes(sets, name, precision)
    peak, peak_kind = measured_peak_hbm()
    gbs = lambda b, ms: b / (ms / 1e3) / 1e9 if b else None  # noqa: E731
    achieved = gbs(ab_grade if ab_grade else ab, per_launch_ms)
    step_ms = sum(v[1] for v in prof.values()) / 120.0
    kernels = {}
    for k, v in prof.items():
        b, _ = algorithmic_bytes(sets, k, precision)
        kernels[k] = {"launches": v[0], "ms_per_launch": v[1] / v[0], "algorithmic_bytes": b,
                      "achieved_gbs": gbs(b, v[1] / v[0]),
                      "traffic": measured_traffic(k, precision, args.workload)}
    step_bytes, _ = algorithmic_bytes(sets, "step", precision)
    roofline = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                "traffic": measured_traffic(name, precision, args.workload),
                "algorithmic_bytes_per_launch": ab_grade or ab,
                "actual_layout_bytes_per_launch": ab, "ms_per_launch": per_launch_ms,
                "kernels": kernels, "serialized_step_ms": step_ms,
                "step_algorithmic_bytes": step_bytes,
                "time_step_ms": ms_max / K / T,
                "step_hbm_frac": gbs(step_bytes, ms_max / K / T) / peak}

    out = {"metric": METRIC, "value": value, "unit": "node-steps/s", "n_gpus": world, "steps": K,
           "warmup": W, "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64" if precision == "fp64" else "f32+f64",
           "data": DATA_TEXT[args.workload],
           "config": workload_config(args.workload, sets, args) | {"parallelism": f"replicas{world}"},
           "e2e": {"value": e2e_value, "unit": "node-steps/s", "h2d_bytes_per_step": h2d,
                   "d2h_bytes_per_step": d2h,
                   "excludes": "lps_create (host setup and the one-time upload of geometry and "
                               "absorbing-boundary operators), as the reference's timer excludes its setup"},
           "gpu_launches": launches, "roofline": roofline, "clocks": clk,
           "kernel_path": info["path"], "tile_ctas": [info["tile_ctas_theta"], info["tile_ctas_force"]],
           "tile_rows_theta": info["tile_rows_theta"], "tile_rows_force": info["tile_rows_force"],
           "final_dE_rel": final_dE, "_u": final_u}
    if with_cpu and rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        s_cpu, n_cpu, note = cpu_sample(sets, args)
        v, sec, kind = cpu_leg(s_cpu, n_cpu, threads)
        out["cpu_baseline"] = {"value": v, "unit": "node-steps/s", "cores": threads, "kind": kind,
                               "sample": f"one nu={s_cpu.nu:g} instance ({s_cpu.n_nodes} nodes), "
                                         f"{n_cpu} time steps, output off, {sec:.2f} s{note}"}
    return out


def run_reference(args):
    """The reference's CPU solver on the same workload (bounded sample)."""
    threads = os.cpu_count() or 1
    sets = workload_sets(args.workload, args.time_steps)
    s, per_run, note = cpu_sample(sets, args)
    per_step = max(1, per_run // 4)
    n = per_step * (args.warmup + args.steps)
    v, sec, kind = cpu_leg(s, n, threads)
    return {"metric": METRIC, "value": v, "unit": "node-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sec / (args.warmup + args.steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": DATA_TEXT[args.workload],
            "config": workload_config(args.workload, sets, args) | {"parallelism": "openmp"},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "node-steps/s", "cores": threads, "kind": kind,
                             "sample": f"one nu={s.nu:g} instance ({s.n_nodes} nodes), {n} time steps "
                                       f"({per_step} per bench step), output off, {sec:.2f} s{note}"},
            "e2e": {"value": v, "unit": "node-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    if args.time_steps is None:
        sys.path.insert(0, PKG)
        from lps_b200.configs import STEPS
        args.time_steps = STEPS[args.workload]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    if args.precision == "both":
        out64 = run_ours(args, rank, world, local_rank, "fp64", with_cpu=False)
        out = run_ours(args, rank, world, local_rank, "fp32_mixed")
        out["fp64"] = {"value": out64["value"], "ms_per_step": out64["ms_per_step"],
                       "e2e": out64["e2e"]["value"], "gpu_launches": out64["gpu_launches"],
                       "final_dE_rel": out64["final_dE_rel"], "clocks": out64["clocks"],
                       "kernels_ms": {k: v["ms_per_launch"] for k, v in out64["roofline"]["kernels"].items()},
                       "time_step_ms": out64["roofline"]["time_step_ms"],
                       "step_hbm_frac": out64["roofline"]["step_hbm_frac"]}
        out["fp32_mixed_over_fp64"] = out["value"] / out64["value"]
        import numpy as np
        rel = [float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(out["_u"], out64["_u"])]
        dde = [abs(a - b) for a, b in zip(out["final_dE_rel"], out64["final_dE_rel"])]
        out["fp32_mixed_error_vs_fp64"] = {"u_rel_l2_max": max(rel), "final_dE_rel_absdiff_max": max(dde),
                                           "u_rel_l2": rel}
    else:
        out = run_ours(args, rank, world, local_rank, args.precision)
    out.pop("_u", None)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
