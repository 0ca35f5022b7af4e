#!/usr/bin/env python
"""Benchmark of the TeaLeaf implicit heat-conduction solve on B200.

Metric (the reference's headline): seconds per timestep of the implicit solve at a
relative residual of 1e-10 (sum r^2 < 1e-20 sum b^2, b = rho*e), plain FP64; lower is
better.  Workload (the 2D 4096^2 configuration): 4096 x 4096 cells on a 10 x 10 domain,
dt = 0.004, the seeded 16-state layout (rectangles/circles, density log-uniform in
[0.1, 100], energy uniform in [1, 25], conductivity 1/density), Chebyshev with 30 CG
presteps.  (PPCG, the configuration's other solver, does not reach 1e-10 on this deck in
FP64: its recursive residual stalls near 2e-9 relative, on the reference's own kernels
too.)  A step is one timestep: one call of ext_tea_leaf_solve_ (tea_leaf() of the
reference) on data resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Timing: W untimed timesteps, then K timesteps between CUDA events recorded on the
library's own stream, barrier + synchronize on both sides, max over ranks.  Every field
array is 135 MB (> 126 MB of L2), so no L2 flush is needed between steps.  With N > 1
(torchrun) each rank solves its own replica of the workload (the benchmark does not split
one solve over ranks) and rank 0 prints one JSON line.

Beside the headline the line carries: `e2e` (the same timesteps through the public driver
API), `roofline` (the dominant fused kernel against the measured copy peak, with its ncu
traffic), `step_canonical` (the timestep's rate in canonical bytes), `cpu_baseline` (the
reference's own kernels on the host cores), `per_call` (the per-call ext_* path),
`fp32_refined` and `fp32_refined_learned` (the precision form, and with the learned warm
start), `c5_3d512_ppcg` (3D 512^3 PPCG: plain FP64 against FP32-refined with PPCG and with
Chebyshev corrections, and with the 3D learned warm start) and `c3_3d256` (3D 256^3 CG and
PPCG).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent

# One GPU per process: restrict visibility before any CUDA initialisation.
if "LOCAL_RANK" in os.environ and "CUDA_VISIBLE_DEVICES" not in os.environ:
    os.environ["CUDA_VISIBLE_DEVICES"] = os.environ["LOCAL_RANK"]

sys.path.insert(0, str(ROOT))
import __graft_entry__  # noqa: E402

tea = __graft_entry__.load_package()

CELLS = 4096
STATES = 16
SEED = 4096
EPS_REL = 1e-10
SOLVER = "chebyshev"
METRIC = "s/timestep at rel residual 1e-10 (plain FP64, 2D 4096^2, Chebyshev)"
WORDS = {  # algorithmic FP64 words per interior cell of one launch
    "cg_sweep_a": 8,   # read p, r, u, Kx, Ky; write u, p, w
    "cg_sweep_b": 3,   # read r, w; write r
    "cheby_iterate": 7,  # read u, u0, p, Kx, Ky; write u', p
    "cheby_pair": 7,  # the same words for two iterations (one pass)
    "cheby_quad": 7,  # four iterations per pass: read u, u0, p, Kx, Ky; write u, p
}
KERNEL_IDS = {"cg_sweep_a": 2, "cheby_quad": 11, "cheby_pair": 6, "cg_sweep_b": 5}
ALL_KERNEL_IDS = {"ppcg_inner": 1, "cg_sweep_a": 2, "cheby_iterate": 3, "jacobi": 4, "cg_sweep_b": 5,
                  "cheby_pair": 6, "cg32_sweep_a": 7, "cg32_sweep_b": 8, "cheby32_pair": 9, "ppcg_pair": 10,
                  "cheby_quad": 11, "cheby32_quad": 12, "ppcg32_pair": 13}
PROFILES = ROOT / "profiles"
# The reference's own per-timestep iteration counts on this deck (its Kokkos-OpenMP kernels,
# oracle/_ref, 30 timesteps at 4096^2), recorded by tests/golden/make_golden_large.py.  They
# scale the reference arm's measured per-iteration costs to whole timesteps.
REF_LARGE = ROOT / "tests" / "golden" / "ref_large.json"
REF_CASE = "c2_2d4096_cheby"


def workload_spec(steps=1):
    return tea.DeckSpec(dim=2, cells=CELLS, states=STATES, seed=SEED, solver=SOLVER, end_step=steps, dt=0.004,
                        eps=1e-15, eps_rel=EPS_REL, max_iters=20000, presteps=30, inner_steps=10,
                        check_result=False, summary_frequency=0)


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(kernel: str):
    """dram bytes per launch of `kernel` from the committed ncu summary, or None."""
    p = PROFILES / f"{kernel}_2d4096.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("dram_bytes_per_launch")
    return None


def progress(msg: str) -> None:
    """A progress line on stderr (the JSON result goes to stdout)."""
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


# ----------------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clock/throttle samples taken during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        visible = os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0]
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9 or (visible.isdigit() and f[0] != visible):
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


# ----------------------------------------------------------------------------- distributed

def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=900))
    return rank, world


def dist_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def dist_done(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


# ----------------------------------------------------------------------------- GPU arm

def parse_states(deck: str, dx: float, dy: float):
    """The state tables as read_input builds them (tealeaf_2d/read_input.f90:216-297)."""
    states = {}
    for line in deck.splitlines():
        w = line.replace("=", " ").split()
        if not w or w[0] != "state":
            continue
        sid = int(w[1])
        st = {"density": 0.0, "energy": 0.0, "xmin": 0.0, "xmax": 0.0, "ymin": 0.0, "ymax": 0.0, "radius": 0.0,
              "geometry": 0}
        k = 2
        while k + 1 < len(w):
            key, val = w[k], w[k + 1]
            if key == "geometry":
                st["geometry"] = {"rectangle": 1, "circle": 2, "point": 3}[val]
            else:
                st[key] = float(val)
            k += 2
        if sid >= 2:
            st["xmin"] += dx / 100.0
            st["ymin"] += dy / 100.0
            st["xmax"] -= dx / 100.0
            st["ymax"] -= dy / 100.0
        states[sid] = st
    return [states[k] for k in sorted(states)]


def setup_chunk(lib, spec):
    """start() of the reference (tealeaf_2d/start.f90:24-162) through the C ABI."""
    import numpy as np

    n = spec.cells
    ch = tea.ExtChunk(lib, 2, n, n)
    dx = (spec.domain - 0.0) / float(n)
    ch.initialise(0.0, 0.0, dx, dx)
    states = parse_states(tea.seeded_deck(spec), dx, dx)
    arr = {k: np.array([s[k] for s in states], dtype=np.float64) for k in
           ("density", "energy", "xmin", "xmax", "ymin", "ymax", "radius")}
    geo = np.array([s["geometry"] for s in states], dtype=np.int32)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    I = lambda v: ctypes.byref(ctypes.c_int(v))
    ch.call("ext_generate_chunk_", I(len(states)), P(arr["density"]), P(arr["energy"]), P(arr["xmin"]),
            P(arr["xmax"]), P(arr["ymin"]), P(arr["ymax"]), P(arr["radius"]), P(geo), I(1), I(2), I(3))
    ch.update_halo({1, 2, 3}, 2)
    ch.call("ext_set_field_kernel_")
    return ch


def solve_params(spec, precision=0):
    p = tea.SolveParams()
    p.solver = tea.SOLVERS[spec.solver]
    p.coefficient = 2 if spec.inverse_density else 1
    p.preconditioner = 1 if spec.preconditioner else 0
    p.max_iters = spec.max_iters
    p.ch_cg_presteps = spec.presteps
    p.ch_cg_errswitch = 0
    p.ppcg_inner_steps = spec.inner_steps
    p.check_result = 0
    p.dt = spec.dt
    p.eps = spec.eps
    p.ch_cg_epslim = float(ctypes.c_float(1e-5).value)
    p.eps_rel = spec.eps_rel
    p.precision = precision
    return p


def gpu_arm(args, world, precision=0, kernels=True, ws_net=0):
    import torch

    lib = tea.cuda_library(2)
    spec = workload_spec()
    ch = setup_chunk(lib, spec)
    if ws_net:
        lib.tea_ws_attach_(ch.cid, ctypes.byref(ctypes.c_int(ws_net)))
    stream_ptr = ctypes.c_void_p()
    lib.tea_chunk_stream_(ch.cid, ctypes.byref(stream_ptr))
    stream = torch.cuda.ExternalStream(stream_ptr.value)
    params = solve_params(spec, precision)
    results = []
    for _ in range(args.warmup):
        results.append(ch.solve(params))
    warm = list(results)
    results.clear()
    dist_barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler()
    clocks.start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for _ in range(args.steps):
        results.append(ch.solve(params))
    t_end.record(stream)
    t_end.synchronize()
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    dist_barrier(world)
    ms = t_start.elapsed_time(t_end)
    ms_max = dist_max(ms, world)
    sec_per_step = ms_max / 1000.0 / args.steps
    bad = [r for r in results if r["status"] not in (0, 7)]

    # Kernel-level: the fused kernels of the timestep, launched back to back on the same
    # stream between CUDA events, on the chunk's live fields (steady-state operands).
    cells = CELLS * CELLS
    summaries = []
    for _ in range(1):
        v = [ctypes.c_double() for _ in range(4)]
        lib.ext_field_summary_kernel_(ch.cid, *[ctypes.byref(x) for x in v])
        summaries = [x.value for x in v]
    kernel_ms = {}
    for name, kid in (KERNEL_IDS.items() if kernels else ()):
        kms = ctypes.c_double(0.0)
        lib.tea_kernel_timing_(ch.cid, ctypes.byref(ctypes.c_int(kid)), ctypes.byref(ctypes.c_int(30)),
                               ctypes.byref(kms))
        kernel_ms[name] = kms.value
    lib.ext_finalise_()

    cg = [r["cg_steps"] for r in results]
    cheby = [r["cheby_steps"] for r in results]
    iters = [r["iterations"] for r in results]
    mean_cg = sum(cg) / len(cg)
    mean_ch = sum(cheby) / len(cheby)
    if kernels:
        # Chebyshev iterations run four per pass, with a two-iteration pass ending at each
        # convergence check (4 + 4 + 2 per 10 iterations once the checks start).
        share = {"cg_sweep_a": mean_cg * kernel_ms["cg_sweep_a"], "cg_sweep_b": mean_cg * kernel_ms["cg_sweep_b"],
                 "cheby_quad": mean_ch / 5.0 * kernel_ms["cheby_quad"],
                 "cheby_pair": mean_ch / 10.0 * kernel_ms["cheby_pair"]}
        dominant = max(share, key=share.get)
        alg_bytes = WORDS[dominant] * 8 * cells
    else:
        dominant, alg_bytes = None, None
    # Chebyshev passes: 7 words per pass of four or two iterations (3 passes per 10 iterations).
    step_words = (WORDS["cg_sweep_a"] + WORDS["cg_sweep_b"]) * mean_cg + WORDS["cheby_pair"] * mean_ch * 0.3
    # The same timestep counted in canonical words per iteration (each iteration's arrays
    # once, fusion and temporal blocking not credited): CG 12, Chebyshev 7 (2D).
    canon_words = CANONICAL_WORDS[2]["cg"] * mean_cg + CANONICAL_WORDS[2]["cheby"] * mean_ch
    return {
        "sec_per_step": sec_per_step, "ms_total": ms_max, "clocks": clock_info, "iterations": iters,
        "cg_steps": cg, "cheby_steps": cheby, "kernel_ms": kernel_ms, "dominant": dominant,
        "alg_bytes": alg_bytes, "step_alg_gbs": step_words * 8 * cells / sec_per_step / 1e9,
        "step_canonical_gbs": canon_words * 8 * cells / sec_per_step / 1e9, "canonical_words": canon_words,
        "cells_iters_per_s": cells * (sum(iters) / len(iters)) / sec_per_step,
        "warmup_iterations": [r["iterations"] for r in warm], "bad_status": [r["status"] for r in bad],
        "corrections": [r["corrections"] for r in results], "summary": summaries,
        "exact_errors": [r["exact_error"] for r in results],
        "warm_start_used": [r["warm_start_used"] for r in results],
        "warm_r0_ratio": [r["warm_r0_guess"] / r["warm_r0_plain"] if r["warm_r0_plain"] else None for r in results],
    }


def e2e_arm(args):
    """End to end through the public API: tea_run_deck (the C++ driver) runs the deck
    through the C ABI -- host state tables in, set-up, timesteps, a field summary read back
    after every step -- and the wall clock of the K steps after W warm-up steps is taken
    from the driver's per-step records."""
    spec = workload_spec(steps=args.warmup + args.steps)
    deck = tea.seeded_deck(spec)
    summary, recs = tea.run_deck(deck, 2, fused=True, summary_every_step=True)
    w, k = args.warmup, args.steps
    t0 = recs[w - 1]["wall_end"] if w > 0 else 0.0
    t1 = recs[w + k - 1]["wall_end"]
    h0 = recs[w - 1]["h2d_bytes"] if w > 0 else 0
    d0 = recs[w - 1]["d2h_bytes"] if w > 0 else 0
    return {
        "value": (t1 - t0) / k,
        "h2d_bytes_per_step": (recs[w + k - 1]["h2d_bytes"] - h0) / k,
        "d2h_bytes_per_step": (recs[w + k - 1]["d2h_bytes"] - d0) / k,
        "iterations": [r["iterations"] for r in recs],
        "temp": summary["temp"],
    }


def per_call_arm():
    """The drop-in path as the reference's own driver drives it: tea_run_deck without the
    whole-solve entry point, so every iteration is the reference's per-call ext_* sequence
    (ext_cg_calc_w_, ext_cg_calc_ur_, ext_cg_calc_p_, halo updates, ...) with each reduction
    read back to the host.  One warm-up timestep, then timestep 2 timed by the driver."""
    spec = workload_spec(steps=2)
    summary, recs = tea.run_deck(tea.seeded_deck(spec), 2, fused=False, summary_every_step=True)
    r = recs[1]
    return {"value": r["wall_end"] - recs[0]["wall_end"], "unit": "s", "timestep": 2,
            "iterations": r["iterations"], "temp": summary["temp"]}


# ----------------------------------------------------------------------------- CPU (reference) arm

def reference_costs(threads: int, n_cg=40, n_cheby=40):
    """Per-iteration costs of the reference's own Kokkos-OpenMP kernels (oracle/_ref,
    compiled from the reference sources) on this deck, timed by the driver around
    tea_leaf() on `threads` host cores.  A full 4096^2 timestep takes the CPU minutes, so
    the sample is bounded: the first timestep cut after n_cg CG iterations (no switch),
    and again with the Chebyshev switch forced at iteration 20 (tl_ch_cg_errswitch with
    an unbounded tl_ch_cg_epslim) and cut n_cheby iterations later."""
    ref = ROOT / "oracle" / "_ref" / "libtea_ref2d.so"
    if not ref.exists():
        raise FileNotFoundError(str(ref))
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="true")

    def run(max_iters, force_switch):
        spec = workload_spec()
        spec.max_iters = max_iters
        spec.eps_rel = 0.0
        spec.eps = 1e-300
        if not force_switch:
            spec.presteps = 10 ** 6
        deck = tea.seeded_deck(spec)
        if force_switch:
            deck = deck.replace("*endtea", "tl_ch_cg_errswitch\ntl_ch_cg_epslim=1e300\n*endtea")
        with tempfile.TemporaryDirectory() as td:
            (pathlib.Path(td) / "tea.in").write_text(deck)
            subprocess.run([str(tea.tea_leaf_exe()), "--dim", "2", "--backend", str(ref), "--quiet", "--no-out", "--json",
                            str(pathlib.Path(td) / "o.json"), str(pathlib.Path(td) / "tea.in")],
                           check=True, env=env, capture_output=True, timeout=1200)
            return json.loads((pathlib.Path(td) / "o.json").read_text())["records"][0]

    t0 = time.perf_counter()
    a = run(n_cg, False)
    t_cg = a["solve_seconds"] / n_cg
    b = run(19 + n_cheby, True)
    # 19 CG iterations, the switch iteration (first Chebyshev step: about two iterations of
    # work plus two norms) and n_cheby - 1 further Chebyshev iterations.
    t_cheby = max(b["solve_seconds"] - 19 * t_cg, 0.0) / (n_cheby + 1)
    return {"t_cg": t_cg, "t_cheby": t_cheby, "wall": time.perf_counter() - t0, "threads": threads,
            "cg_iters": a["iterations"], "cheby_run_iters": b["iterations"]}


def reference_counts():
    """{timestep: (CG iterations, Chebyshev loop passes)} of the reference on the benchmark
    deck, and the thread count they were recorded at.  The reference prints n - 1 for a
    solve that exits in loop pass n (tealeaf_2d/tea_solve.f90:543); passes 1 .. switch - 1
    are CG, the rest Chebyshev."""
    d = json.loads(REF_LARGE.read_text())[REF_CASE]
    spec = workload_spec(steps=len(d["ref"]["records"]))
    spec.summary_frequency = 1
    if d["deck"] != tea.seeded_deck(spec):
        raise ValueError(f"{REF_LARGE.name}: {REF_CASE} was recorded on another deck")
    counts = {}
    for r in d["ref"]["records"]:
        cg = r["switch_step"] - 1 if r["switch_step"] > 0 else r["iterations"] + 1
        counts[r["step"]] = (cg, r["iterations"] + 1 - cg)
    return counts, d["threads"]


def counts_for(steps):
    """The reference's counts for `steps`; a timestep beyond the recorded ones takes the last
    recorded timestep's counts.  Returns (list, note)."""
    counts, threads = reference_counts()
    last = max(counts)
    out = [counts[min(s, last)] for s in steps]
    beyond = [s for s in steps if s > last]
    note = (f"the reference's own counts for timesteps {steps[0]}-{steps[-1]} (recorded at {threads} threads)"
            + (f"; timesteps {beyond[0]}-{beyond[-1]} take timestep {last}'s" if beyond else ""))
    return out, note


def cpu_estimate(costs, cg, cheby_passes):
    # The first Chebyshev pass runs about two iterations' work (init, one iterate, two norms).
    return costs["t_cg"] * cg + costs["t_cheby"] * (cheby_passes + 1)


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_arm(args, rank, world):
    """--impl reference: the reference's CPU implementation on this box's host cores.  Each
    step times a bounded sample of the timestep it stands for (reference_costs: CG and
    Chebyshev iterations of the reference's kernels on this deck) and scales the measured
    per-iteration costs by the reference's own iteration counts for that timestep."""
    if rank != 0:
        dist_done(world)
        return
    threads = host_threads()
    steps = list(range(args.warmup + 1, args.warmup + args.steps + 1))
    line = {"impl": "reference", "metric": METRIC, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": False}
    try:
        counts, note = counts_for(steps)
        if not (ROOT / "oracle" / "_ref" / "libtea_ref2d.so").exists():
            raise FileNotFoundError("oracle/_ref (the reference's Kokkos-OpenMP kernels built from its sources) "
                                    "is not built")
    except (OSError, ValueError, KeyError) as exc:
        line["unavailable"] = str(exc)
        print(json.dumps(line))
        dist_done(world)
        return
    for _ in range(args.warmup):
        reference_costs(threads, 10, 10)
    samples, per_iter = [], []
    for cg, ch in counts:
        c = reference_costs(threads, 40, 40)
        samples.append(cpu_estimate(c, cg, ch))
        per_iter.append((c["t_cg"], c["t_cheby"]))
    value = statistics.mean(samples)
    mean_cg = sum(c[0] for c in counts) / len(counts)
    mean_ch = sum(c[1] for c in counts) / len(counts)
    line.update({
        "value": value, "ms_per_step": value * 1000.0, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded 16-state layout)",
        "config": {"workload": "2d_4096x4096_16states_chebyshev_rel1e-10", "cells": CELLS * CELLS,
                   "solver": SOLVER, "timesteps_timed": steps, "per_step_s": samples,
                   "ms_per_iteration_cg_cheby": [statistics.mean(t[0] for t in per_iter) * 1e3,
                                                 statistics.mean(t[1] for t in per_iter) * 1e3]},
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "reference",
                         "sample": "per step: the first timestep of the deck cut after 40 CG iterations, and with "
                                   "the Chebyshev switch forced at iteration 20 cut 40 iterations later; the "
                                   f"per-iteration costs scaled by {note} (mean {mean_cg:.0f} CG + {mean_ch:.0f} "
                                   "Chebyshev iterations per timestep)"},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    })
    print(json.dumps(line))
    dist_done(world)


# The other configurations' 3D workloads (seeded box/sphere layouts): timed through the
# public driver (tea_run_deck: deck in, field summary out), plain FP64 and FP32-refined.
WORKLOADS_3D = {
    "3d128_ppcg": dict(cells=128, solver="ppcg", states=24, seed=512),
    "3d256_cg": dict(cells=256, solver="cg", states=12, seed=256),
    "3d256_ppcg": dict(cells=256, solver="ppcg", states=12, seed=256),
    "3d256_cheby": dict(cells=256, solver="chebyshev", states=12, seed=256),
    "3d512_ppcg": dict(cells=512, solver="ppcg", states=24, seed=512),
}


INNER_SOLVERS = {0: "cg", 1: "chebyshev", 2: "ppcg"}

# Canonical FP64 words per interior cell of one iteration, each array counted once as the
# reference's unfused kernels touch it: CG (w = A p with p.w; u, r update with r.r; p update)
# 12 in 2D and 13 in 3D, a Chebyshev iteration 7 / 8, a PPCG inner step 8 / 9 (its outer
# iteration is a CG iteration plus the inner steps).
CANONICAL_WORDS = {2: {"cg": 12, "cheby": 7, "ppcg_inner": 8}, 3: {"cg": 13, "cheby": 8, "ppcg_inner": 9}}


def canonical_step_words(dim, solver, iterations, cheby_steps, inner_steps=10):
    """Canonical words per cell of one timestep: the reference prints n - 1 for a solve
    that ends in loop pass n, passes 1 .. switch - 1 being CG and the rest Chebyshev or
    PPCG outer iterations (cheby_steps of them)."""
    w = CANONICAL_WORDS[dim]
    n = iterations + 1
    if solver == "cg":
        return w["cg"] * n
    cg = max(n - cheby_steps, 0)
    if solver == "chebyshev":
        return w["cg"] * cg + w["cheby"] * cheby_steps
    return w["cg"] * cg + (w["cg"] + inner_steps * w["ppcg_inner"]) * cheby_steps


def run_3d(workload, warmup, steps, arm_steps=None, ws=None):
    """s/timestep of a 3D configuration, plain FP64 and FP32-refined on the same deck, each
    timestep's solve timed by the driver around the synchronous ext_tea_leaf_solve_ call
    (the reference's wall clock around tea_leaf(), tealeaf_2d/diffuse.f90:74-85); the first
    `warmup` timesteps are run and not timed.  FP32-refined corrects with the deck's own
    method (PPCG decks: FP32 PPCG); on PPCG and Chebyshev decks `fp32_refined_cheby_inner`
    also times it with FP32 Chebyshev corrections (tl_inner_solver chebyshev), and with a
    trained 3D network `ws` (train_3d_network) `fp32_refined_cheby_inner_learned` times that
    form with the learned warm start attached.  `arm_steps` maps an arm's name to a smaller
    number of timed timesteps."""
    w = WORKLOADS_3D[workload]
    spec = tea.DeckSpec(dim=3, cells=w["cells"], states=w["states"], seed=w["seed"], solver=w["solver"],
                        end_step=warmup + steps, dt=0.004, eps=1e-15, eps_rel=EPS_REL, max_iters=20000,
                        presteps=30, inner_steps=10, check_result=True, summary_frequency=0)
    deck = tea.seeded_deck(spec)
    out = {"workload": workload, "cells": w["cells"] ** 3, "states": w["states"], "solver": w["solver"],
           "unit": "s/timestep", "rel_residual": EPS_REL, "timesteps_timed": list(range(warmup + 1, warmup + steps + 1))}
    summaries = {}
    n = lambda name: (arm_steps or {}).get(name, steps)
    arms = [("fp64", tea.PRECISION_FP64, deck, n("fp64")),
            ("fp32_refined", tea.PRECISION_FP32_REFINED, deck, n("fp32_refined"))]
    if w["solver"] in ("ppcg", "chebyshev"):
        cheby_deck = deck.replace("*endtea", "tl_inner_solver chebyshev\n*endtea")
        arms.append(("fp32_refined_cheby_inner", tea.PRECISION_FP32_REFINED, cheby_deck,
                     n("fp32_refined_cheby_inner")))
        if ws:
            arms.append(("fp32_refined_cheby_inner_learned", tea.PRECISION_FP32_REFINED, cheby_deck,
                         n("fp32_refined_cheby_inner_learned")))
    for name, precision, dk, nsteps in arms:
        progress(f"{workload}: {name}, {warmup} + {nsteps} timesteps")
        learned = name.endswith("_learned")
        summary, recs = tea.run_deck(dk, 3, fused=True, precision=precision, summary_every_step=True,
                                     end_step=warmup + nsteps, ws_net=ws["net"].id if learned else 0,
                                     ws_mode=tea.WS_ATTACH if learned else 0)
        timed = recs[warmup:warmup + nsteps]
        summaries[name] = summary
        out[name] = {"s_per_step": sum(r["solve_seconds"] for r in timed) / len(timed),
                     "per_step_s": [r["solve_seconds"] for r in timed],
                     "iterations": [r["iterations"] for r in timed],
                     "switch_step": [r["switch_step"] for r in timed],
                     "cheby_steps": [r["cheby_steps"] for r in timed],
                     "corrections": [r["corrections"] for r in timed],
                     "exact_error_over_eps": [r["exact_error"] / r["eps_used"] for r in timed]}
        if precision == tea.PRECISION_FP32_REFINED:
            out[name]["inner_solver"] = [INNER_SOLVERS.get(r["inner_solver"], "?") for r in timed]
        if precision == tea.PRECISION_FP64:
            words = [canonical_step_words(3, w["solver"], r["iterations"], r["cheby_steps"]) for r in timed]
            gbs = [wd * 8 * w["cells"] ** 3 / r["solve_seconds"] / 1e9 for wd, r in zip(words, timed)]
            out[name]["step_canonical"] = {"gbs": gbs, "frac": [x / load_peaks()[0] for x in gbs],
                                           "words_per_cell": words}
        if learned:
            out[name]["warm_start_used"] = [r["warm_start_used"] for r in timed]
            out[name]["warm_r0_ratio"] = [r["warm_r0_guess"] / r["warm_r0_plain"] if r["warm_r0_plain"] else None
                                          for r in timed]
    for name in [a[0] for a in arms[1:]]:
        out[name]["speedup_vs_fp64"] = out["fp64"]["s_per_step"] / out[name]["s_per_step"]
    out["speedup_fp32_refined"] = out["fp32_refined"]["speedup_vs_fp64"]
    if ws and "fp32_refined_cheby_inner_learned" in out:
        a, b = out["fp32_refined_cheby_inner"], out["fp32_refined_cheby_inner_learned"]
        saved = a["s_per_step"] - b["s_per_step"]
        cost = ws["record_s"] + ws["train_s"]
        b["iterations_saved"] = ([x - y for x, y in zip(a["iterations"], b["iterations"])]
                                 if len(a["iterations"]) == len(b["iterations"]) else None)
        b["seconds_saved_per_step"] = saved
        b["training"] = {k: v for k, v in ws.items() if k != "net"}
        b["amortised_after_steps"] = cost / saved if saved > 0 else None
    # Field summaries after the same timesteps (each arm's last timestep).
    last = {a[0]: a[3] for a in arms}
    out["field_summary_max_rel_diff"] = {
        name: max(tea.rel_diff(summaries["fp64"][k], summaries[name][k]) for k in ("vol", "mass", "ie", "temp"))
        for name in last if name != "fp64" and last[name] == last["fp64"]}
    return out


def train_dt(dt: float, cells: int, target_cells: int) -> float:
    """The timestep that gives a coarser training deck the target deck's face coefficients:
    K = dt w / h^2 with h = domain / cells, so dt scales with (target_cells / cells)^2."""
    return dt * (target_cells / cells) ** 2


def train_3d_network():
    """The 512^3 configuration's learned warm start: a 3D U-Net (3 levels, 24 base channels,
    3x3x3 convolutions, bfloat16) trained by the library's own kernels on pairs the 3D
    solver generates at 128^3 (four seeded 24-state layouts, timesteps 1-6 of each), with dt
    scaled so that the operator's coefficients match those of the 512^3 deck."""
    t0 = time.perf_counter()
    net = tea.WarmStart(3, 24, seed=512, dim=3)
    for k in range(4):
        spec = tea.DeckSpec(dim=3, cells=128, states=24, seed=513 + k, solver="ppcg", end_step=6,
                            dt=train_dt(0.004, 128, 512),
                            eps=1e-15, eps_rel=EPS_REL, max_iters=20000, presteps=30, inner_steps=10,
                            check_result=False, summary_frequency=0)
        tea.run_deck(tea.seeded_deck(spec), 3, fused=True, ws_net=net.id, ws_mode=tea.WS_RECORD)
    t_record = time.perf_counter() - t0
    progress(f"3D network: {net.pairs()} pairs recorded in {t_record:.1f} s; training")
    t1 = time.perf_counter()
    loss_first, loss_last, ms_step = net.train(steps=2000, batch=2, crop=64, lr=1e-3, seed=512)
    progress(f"3D network: loss {loss_first:.3f} -> {loss_last:.3f}, {ms_step:.2f} ms/step")
    return {"net": net, "pairs": net.pairs(),
            "layouts": "4 seeded 128^3 24-state layouts x 6 timesteps, dt 0.064 (the 512^3 deck's K)",
            "record_s": t_record, "train_s": time.perf_counter() - t1, "train_ms_per_step": ms_step, "steps": 2000,
            "batch": "2 crops of 64^3", "lr": 1e-3, "loss_first": loss_first, "loss_last": loss_last,
            "network": "3D U-Net, 3 levels, 24/48/96 channels, 3x3x3 convolutions, bfloat16 weights"}


def workload_3d(args):
    """--workload NAME: run_3d of that configuration with the command line's steps (the
    512^3 PPCG configuration with its trained 3D network when --learned is given)."""
    ws = train_3d_network() if args.learned else None
    out = run_3d(args.workload, args.warmup, args.steps, ws=ws)
    if ws:
        ws["net"].close()
    print(json.dumps(out))


def learned_2d_at_scale(args):
    """--workload 2d4096_learned: the 2D learned configuration at its stated scale.  A 4-level
    U-Net (32/64/64/64 channels, about half a million parameters) is trained by the
    library's kernels on 4032 pairs the solver generates from 64 seeded 1024^2 layouts (63
    timesteps each); then the 4096^2 deck runs with PPCG for --steps timesteps in the
    FP32-refined form (FP32 Chebyshev corrections; FP64 PPCG stalls above 1e-10 on this deck),
    with and without the learned warm start, through the driver (deck in, field summary out)."""
    t0 = time.perf_counter()
    net = tea.WarmStart(4, 32, seed=SEED, max_channels=64)
    for k in range(64):
        spec = tea.DeckSpec(dim=2, cells=1024, states=STATES, seed=SEED + 100 + k, solver="cg", end_step=63,
                            dt=train_dt(0.004, 1024, CELLS), eps=1e-15, eps_rel=1e-8, max_iters=20000,
                            summary_frequency=0,
                            check_result=False)
        tea.run_deck(tea.seeded_deck(spec), 2, fused=True, ws_net=net.id, ws_mode=tea.WS_RECORD)
        progress(f"2D network at scale: layout {k + 1}/64 recorded ({net.pairs()} pairs)")
    t_record = time.perf_counter() - t0
    t1 = time.perf_counter()
    loss_first, loss_last, ms_step = net.train(steps=4000, batch=8, crop=128, lr=3e-4, seed=SEED)
    t_train = time.perf_counter() - t1
    progress(f"2D network at scale: loss {loss_first:.3f} -> {loss_last:.3f} in {t_train:.0f} s")
    spec = tea.DeckSpec(dim=2, cells=CELLS, states=STATES, seed=SEED, solver="ppcg", end_step=args.steps, dt=0.004,
                        eps=1e-15, eps_rel=EPS_REL, max_iters=20000, presteps=30, inner_steps=10,
                        check_result=False, summary_frequency=0)
    deck = tea.seeded_deck(spec).replace("*endtea", "tl_inner_solver chebyshev\n*endtea")
    out = {"workload": "2d_4096x4096_16states_ppcg_rel1e-10_learned", "timesteps": args.steps,
           "form": "FP32-refined, FP32 Chebyshev corrections (tl_inner_solver chebyshev)",
           "network": {"levels": 4, "channels": [32, 64, 64, 64], "params": net.param_count(),
                       "pairs": net.pairs(),
                       "layouts": "64 seeded 1024^2 layouts x 63 timesteps (CG, FP64, targets to rel. residual 1e-8), "
                                  "dt 0.064 (the 4096^2 deck's K)",
                       "record_s": t_record, "train_s": t_train, "train_ms_per_step": ms_step, "train_steps": 4000,
                       "batch": "8 crops of 128^2", "loss_first": loss_first, "loss_last": loss_last}}
    runs = {}
    for name, ws_net in (("fp32_refined", 0), ("fp32_refined_learned", net.id)):
        progress(f"2D network at scale: {name}, {args.steps} timesteps")
        summary, recs = tea.run_deck(deck, 2, fused=True, precision=tea.PRECISION_FP32_REFINED,
                                     summary_every_step=True, ws_net=ws_net, ws_mode=tea.WS_ATTACH if ws_net else 0)
        runs[name] = (summary, recs)
        out[name] = {"s_per_step": sum(r["solve_seconds"] for r in recs) / len(recs),
                     "iterations": sum(r["iterations"] for r in recs),
                     "exact_error_over_eps_max": max(r["exact_error"] / r["eps_used"] for r in recs),
                     "warm_start_used": sum(r["warm_start_used"] for r in recs)}
    a, b = out["fp32_refined"], out["fp32_refined_learned"]
    saved = a["s_per_step"] - b["s_per_step"]
    b["iterations_saved"] = a["iterations"] - b["iterations"]
    b["seconds_saved_per_step"] = saved
    b["amortised_after_steps"] = (t_record + t_train) / saved if saved > 0 else None
    b["field_summary_max_rel_diff"] = max(tea.rel_diff(runs["fp32_refined"][0][k], runs["fp32_refined_learned"][0][k])
                                          for k in ("vol", "mass", "ie", "temp"))
    net.close()
    print(json.dumps(out))


def learned_arm(args, world):
    """FP32-refined + learned warm start on the same workload: a U-Net (3 levels, 32 base
    channels) trained on pairs the solver generates from four other seeded 1024^2 layouts
    (6 timesteps each), then attached to the workload's chunk.  Returns the timing and the
    training cost."""
    t0 = time.perf_counter()
    net = tea.WarmStart(3, 32, seed=SEED)
    for k in range(4):
        spec = tea.DeckSpec(dim=2, cells=1024, states=STATES, seed=SEED + 1 + k, solver=SOLVER, end_step=6,
                            dt=train_dt(0.004, 1024, CELLS),
                            eps=1e-15, eps_rel=EPS_REL, max_iters=20000, presteps=30, summary_frequency=0,
                            check_result=False)
        tea.run_deck(tea.seeded_deck(spec), 2, fused=True, ws_net=net.id, ws_mode=tea.WS_RECORD)
    t_record = time.perf_counter() - t0
    t1 = time.perf_counter()
    loss_first, loss_last, ms_step = net.train(steps=1000, batch=8, crop=128, lr=1e-4, seed=SEED)
    t_train = time.perf_counter() - t1
    r = gpu_arm(args, world, precision=1, kernels=False, ws_net=net.id)
    net.close()
    r.update({"record_s": t_record, "train_s": t_train, "train_ms_per_step": ms_step, "loss_first": loss_first,
              "loss_last": loss_last, "pairs": 24})
    return r


# Algorithmic FP64-equivalent words per cell of each fused kernel in 3D (FP32 words count
# half): the 7-point sweeps read one more coefficient array than their 2D forms.
WORDS_3D = {"ppcg_inner": 9, "cg_sweep_a": 9, "cheby_iterate": 8, "jacobi": 6, "cg_sweep_b": 3, "cheby_pair": 8,
            "cg32_sweep_a": 4.5, "cg32_sweep_b": 1.5, "cheby32_pair": 4, "ppcg_pair": 9, "ppcg32_pair": 4.5}


def ws_predict_3d(args):
    """--workload NAME --kernel ws_predict: the 3D warm-start network's prediction (3 levels,
    24/48/96 channels, seeded weights) on the configuration's chunk after one timestep solved
    to a relative residual of 1e-3 (the prediction's cost does not depend on the state),
    `reps` times; device milliseconds of each."""
    w = WORKLOADS_3D[args.workload]
    spec = tea.DeckSpec(dim=3, cells=w["cells"], states=w["states"], seed=w["seed"], solver=w["solver"], end_step=1,
                        dt=0.004, eps=1e-15, eps_rel=1e-3, max_iters=20000, presteps=30, inner_steps=10,
                        check_result=False, summary_frequency=0)
    tea.run_deck(tea.seeded_deck(spec), 3, fused=True, keep_chunk=True)
    lib = tea.cuda_library(3)
    net = tea.WarmStart(3, 24, seed=512, dim=3)
    ms = ctypes.c_double(0.0)
    times = []
    for _ in range(args.reps):
        rc = lib.tea_ws_predict_(ctypes.byref(ctypes.c_int(net.id)), ctypes.byref(ctypes.c_int(1)), None,
                                 ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError(f"tea_ws_predict_: status {rc}")
        times.append(ms.value)
    print(json.dumps({"workload": args.workload, "kernel": "ws_predict", "cells": w["cells"] ** 3,
                      "predict_ms": times}))
    net.close()
    lib.ext_finalise_()


def kernel_only_3d(args):
    """--workload NAME --kernel K: one timestep of the 3D configuration through the driver
    (the FP32-refined form for the FP32 kernels, so that their arrays exist), then K launched
    1 + reps times back to back on the chunk's live fields."""
    if args.kernel == "ws_predict":
        ws_predict_3d(args)
        return
    w = WORKLOADS_3D[args.workload]
    fp32 = args.kernel.startswith(("cg32", "cheby32", "ppcg32"))
    spec = tea.DeckSpec(dim=3, cells=w["cells"], states=w["states"], seed=w["seed"], solver=w["solver"], end_step=1,
                        dt=0.004, eps=1e-15, eps_rel=EPS_REL, max_iters=20000, presteps=30, inner_steps=10,
                        check_result=False, summary_frequency=0)
    tea.run_deck(tea.seeded_deck(spec), 3, fused=True, keep_chunk=True,
                 precision=tea.PRECISION_FP32_REFINED if fp32 else tea.PRECISION_FP64)
    lib = tea.cuda_library(3)
    ms = ctypes.c_double(0.0)
    lib.tea_kernel_timing_(ctypes.byref(ctypes.c_int(1)), ctypes.byref(ctypes.c_int(ALL_KERNEL_IDS[args.kernel])),
                           ctypes.byref(ctypes.c_int(args.reps)), ctypes.byref(ms))
    cells = w["cells"] ** 3
    gbs = WORDS_3D[args.kernel] * 8 * cells / (ms.value / 1e3) / 1e9 if ms.value > 0 else None
    print(json.dumps({"workload": args.workload, "kernel": args.kernel, "ms_per_launch": ms.value,
                      "algorithmic_gbs": gbs}))
    lib.ext_finalise_()


def kernel_only(args):
    """Set up the 4096^2 workload and launch one fused kernel 1 + reps times (no solve)."""
    if args.workload:
        kernel_only_3d(args)
        return
    lib = tea.cuda_library(2)
    ch = setup_chunk(lib, workload_spec())
    ms = ctypes.c_double(0.0)
    lib.tea_kernel_timing_(ch.cid, ctypes.byref(ctypes.c_int(ALL_KERNEL_IDS[args.kernel])),
                           ctypes.byref(ctypes.c_int(args.reps)), ctypes.byref(ms))
    # FP32 kernels: their FP32 words counted as half FP64 words.
    words = {"ppcg_inner": 8, "cg_sweep_a": 8, "cheby_iterate": 7, "jacobi": 5, "cg_sweep_b": 3,
             "cheby_pair": 7, "cg32_sweep_a": 4, "cg32_sweep_b": 1.5, "cheby32_pair": 3.5,
             "ppcg_pair": 8, "cheby_quad": 7, "cheby32_quad": 3.5, "ppcg32_pair": 4}[args.kernel]
    gbs = words * 8 * CELLS * CELLS / (ms.value / 1e3) / 1e9 if ms.value > 0 else None
    print(json.dumps({"kernel": args.kernel, "ms_per_launch": ms.value, "algorithmic_gbs": gbs}))
    lib.ext_finalise_()


# ----------------------------------------------------------------------------- main

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-refined", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-per-call", action="store_true", help="skip timing the per-call ext_* path")
    ap.add_argument("--no-3d", action="store_true",
                    help="skip the 3D lines (512^3 PPCG and 256^3 CG/PPCG, plain FP64 against FP32-refined)")
    ap.add_argument("--kernel", choices=sorted(ALL_KERNEL_IDS) + ["ws_predict"],
                    help="only launch one fused kernel --reps times on the 4096^2 workload, or after one "
                         "timestep of --workload (for ncu captures)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--workload", choices=sorted(WORKLOADS_3D) + ["2d4096_learned"],
                    help="time a 3D configuration instead (plain FP64 and FP32-refined, through the driver), or "
                         "the 2D learned configuration at its stated scale (2d4096_learned)")
    ap.add_argument("--learned", action="store_true", help="with --workload 3d512_ppcg: also the learned warm start")
    args = ap.parse_args()
    if args.kernel:
        kernel_only(args)
        return
    if args.workload == "2d4096_learned":
        learned_2d_at_scale(args)
        return
    if args.workload:
        workload_3d(args)
        return
    if args.warmup < 1:
        ap.error("--warmup must be >= 1")
    rank, world = dist_init()
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return

    g = gpu_arm(args, world)
    refined = None if args.no_refined else gpu_arm(args, world, precision=1, kernels=False)
    learned = None if args.no_refined or args.no_learned else learned_arm(args, world)
    e2e = None if args.no_e2e else e2e_arm(args)
    if e2e and world > 1:
        e2e["value"] = dist_max(e2e["value"], world)  # the slowest replica, as for value
    per_call = None if args.no_per_call else per_call_arm()
    # The 3D 512^3 PPCG configuration: plain FP64 against FP32-refined with FP32 PPCG
    # corrections (the deck's method; two timed timesteps, it is the slowest arm) and with
    # FP32 Chebyshev corrections, one warm-up timestep and five timed ones otherwise.
    ws3 = None if args.no_3d or args.no_learned else train_3d_network()
    c5 = None if args.no_3d else run_3d("3d512_ppcg", 1, 5, {"fp32_refined": 2}, ws=ws3)
    if ws3:
        ws3["net"].close()
    # The 3D 256^3 configuration: CG and PPCG, plain FP64 against FP32-refined, each with its
    # per-step exact error and field-summary difference (one warm-up and three timed timesteps).
    c3 = None if args.no_3d else {w: run_3d(w, 1, 3) for w in ("3d256_cg", "3d256_ppcg")}
    if rank != 0:
        dist_done(world)
        return
    peak, peak_kind = load_peaks()
    dom = g["dominant"]
    achieved = g["alg_bytes"] / (g["kernel_ms"][dom] / 1000.0) / 1e9
    traffic = load_traffic(dom)
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        try:
            threads = host_threads()
            counts, note = counts_for(list(range(args.warmup + 1, args.warmup + args.steps + 1)))
            costs = reference_costs(threads)
            cpu = {"value": statistics.mean(cpu_estimate(costs, cg, ch) for cg, ch in counts), "unit": "s",
                   "cores": threads, "kind": "reference",
                   "sample": (f"the first timestep cut after 40 CG iterations, and with the Chebyshev switch forced "
                              f"at iteration 20 cut 40 iterations later ({costs['wall']:.1f} s of CPU work); "
                              f"{costs['t_cg'] * 1e3:.2f} ms per CG and {costs['t_cheby'] * 1e3:.2f} ms per Chebyshev "
                              f"iteration scaled by {note}")}
        except Exception as exc:  # noqa: BLE001
            cpu = {"value": None, "unit": "s", "cores": None, "kind": "reference", "sample": f"unavailable: {exc}"}
    line = {
        "metric": METRIC, "value": g["sec_per_step"], "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": g["sec_per_step"] * 1000.0, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded 16-state layout)",
        "config": {"workload": "2d_4096x4096_16states_chebyshev_rel1e-10", "cells": CELLS * CELLS,
                   "solver": SOLVER, "presteps": 30, "dt": 0.004, "l2": "inputs larger than L2 (135 MB per field)",
                   "parallelism": "replicas" if world > 1 else "single",
                   "timesteps_timed": list(range(args.warmup + 1, args.warmup + args.steps + 1)),
                   "iterations": g["iterations"], "cg_steps": g["cg_steps"], "cheby_steps": g["cheby_steps"]},
        "cells_iterations_per_s": g["cells_iters_per_s"],
        "step_algorithmic_gbs": g["step_alg_gbs"],
        # The whole timestep's rate in canonical bytes (every iteration's arrays counted once
        # as an unfused iteration reads and writes them: CG 12 words per cell, Chebyshev 7),
        # against the measured copy peak; fusion and temporal blocking take it above the
        # kernels' own fractions, and past 1.0 where they save more than the kernels lose.
        "step_canonical": {"gbs": g["step_canonical_gbs"], "frac": g["step_canonical_gbs"] / load_peaks()[0],
                           "words_per_cell": g["canonical_words"]},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": traffic, "alg_bytes_per_launch": g["alg_bytes"],
                     "launch_ms": g["kernel_ms"][dom], "kernel_ms": g["kernel_ms"],
                     # every timed kernel's algorithmic GB/s as a fraction of the same peak
                     "kernel_frac": {k: WORDS[k] * 8 * CELLS * CELLS / (ms / 1e3) / 1e9 / peak
                                     for k, ms in g["kernel_ms"].items() if ms > 0}},
        "clocks": g["clocks"],
        # 8 fused launches per four CG iterations (the graph's loop body holds four; the
        # launches after the last iteration return at once), about 3 per 10 Chebyshev
        # iterations (passes of four, and of two ending at each convergence check), and
        # about 27 per-call launches per timestep (set-up, halo updates, the switch, finalise).
        "gpu_launches": int(sum(8 * ((c + 3) // 4) + (3 * h + 9) // 10 + 27
                                for c, h in zip(g["cg_steps"], g["cheby_steps"]))),
        "cpu_baseline": cpu,
    }
    if e2e:
        timed = e2e["iterations"][args.warmup:args.warmup + args.steps]
        line["config"]["e2e_iterations_match"] = timed == g["iterations"]
        line["e2e"] = {"value": e2e["value"], "unit": "s", "h2d_bytes_per_step": e2e["h2d_bytes_per_step"],
                       "d2h_bytes_per_step": e2e["d2h_bytes_per_step"]}
    if refined:
        # The precision form on the same workload: FP32 inner CG inside FP64 defect
        # correction to the same relative residual, and its field-summary difference to
        # the FP64 solve after the same timesteps.
        diff = max(tea.rel_diff(a, b) for a, b in zip(refined["summary"], g["summary"]))
        line["fp32_refined"] = {"value": refined["sec_per_step"], "unit": "s",
                                "speedup_vs_fp64": g["sec_per_step"] / refined["sec_per_step"],
                                "iterations": refined["iterations"], "fp64_cg_steps": refined["cg_steps"],
                                "fp32_chebyshev_steps": refined["cheby_steps"], "corrections": refined["corrections"],
                                "exact_errors": refined["exact_errors"],
                                "field_summary_max_rel_diff_vs_fp64": diff, "clocks": refined["clocks"]}
    if learned:
        # FP32-refined + learned warm start: the same timesteps with the network attached;
        # training cost (pair recording + training) stated beside it.
        diff = max(tea.rel_diff(a, b) for a, b in zip(learned["summary"], g["summary"]))
        saved = refined["sec_per_step"] - learned["sec_per_step"] if refined else None
        cost = learned["record_s"] + learned["train_s"]
        line["fp32_refined_learned"] = {
            "value": learned["sec_per_step"], "unit": "s", "speedup_vs_fp64": g["sec_per_step"] / learned["sec_per_step"],
            "iterations": learned["iterations"], "warm_start_used": learned["warm_start_used"],
            # Iterations saved per timestep against FP32-refined alone (negative: more).
            "iterations_saved": ([a - b for a, b in zip(refined["iterations"], learned["iterations"])]
                                 if refined else None),
            "seconds_saved_per_step": saved,
            "warm_r0_ratio": learned["warm_r0_ratio"], "corrections": learned["corrections"],
            "field_summary_max_rel_diff_vs_fp64": diff,
            "training": {"pairs": learned["pairs"],
                         "layouts": "4 seeded 1024^2 layouts x 6 timesteps, dt 0.064 (the 4096^2 deck's K)",
                         "record_s": learned["record_s"], "train_s": learned["train_s"],
                         "train_ms_per_step": learned["train_ms_per_step"], "steps": 1000,
                         "loss_first": learned["loss_first"], "loss_last": learned["loss_last"]},
            "amortised_after_steps": (cost / saved) if saved and saved > 0 else None,
            "clocks": learned["clocks"]}
    if c5:
        line["c5_3d512_ppcg"] = c5
    if c3:
        line["c3_3d256"] = c3
    if per_call:
        # The same deck through the per-call ext_* entry points (what an unchanged Fortran
        # driver calls), timestep 2; the fused arm's timesteps are later ones.
        line["per_call"] = per_call
    if g["bad_status"]:
        line["status_warnings"] = g["bad_status"]
    print(json.dumps(line))
    dist_done(world)


if __name__ == "__main__":
    main()
