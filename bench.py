#!/usr/bin/env python
"""Throughput of the fused Henon-map tracking path on B200.

Workload (the modulated dynamic-aperture scan): a 1024x1024 grid of initial
conditions x0, y0 in [0, 0.6], px0 = py0 = 0, tunes (0.168, 0.201), SPS
modulation with epsilon in {1, 16, 64} and mu in {0, 0.2}, barrier 10,
10^5 turns.  One step = the six (epsilon, mu) scans, each a full tracking
pass of the 2^20 particles.  Synthetic, deterministic inputs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value      : nominal particle-turns/s over the whole job (particles x turns,
             lost particles counted as tracked -- the reference's own
             convention), inputs resident in HBM, CUDA events on the launch
             stream, max over ranks.
e2e        : the same metric through the public API with host buffers:
             pinned host arrays -> particles -> track -> steps read back.
roofline   : executed FP64 flops (survivor-turns x 26 or 42) / summed device
             time of the tracking kernels, against the FP64 FMA-chain peak
             measured in the same process.
cpu_baseline: the reference's own CPU path (built from its sources by
             oracle/build_ref.sh) on a strided subsample of the grid, all
             host cores; reported, not a target.
Multi-GPU (torchrun): each rank scans its own 2^20-particle interleaved
slice of a 1024 x (1024 N) grid; no collective in the data path ("weak").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "FP64 particle-turns/s (% FP64 peak); batched and adjoint vs plain, same GPU"
UNIT = "particle-turns/s"
TUNES = (0.168, 0.201)
EPSILONS = (1.0, 16.0, 64.0)
MUS = (0.0, 0.2)
BARRIER = 10.0
FLOPS_PER_TURN = {False: 26.0, True: 42.0}  # mu == 0 / mu != 0 (algorithmic)
L2_FLUSH_BYTES = 256 << 20
# DRAM bytes (read + write) per particle of a tracking launch's input list,
# measured by ncu on the staged exact kernel (512x512 DA scan, 1024-turn
# chunk of 262,144 particles: 8.42 MB read, 0.3 KB written).
NCU_BYTES_PER_LIST_PARTICLE = 32.1


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1,
                    help="ranks, one per GPU; without torchrun's environment the script "
                         "re-executes itself under torch.distributed.run with that many")
    ap.add_argument("--launch-check", action="store_true",
                    help="start the ranks, join them in a process group (NCCL with GPUs, "
                         "gloo without) and print who joined; no tracking")
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--turns", type=int, default=100_000)
    ap.add_argument("--side", type=int, default=1024)
    ap.add_argument("--arith", choices=["exact", "fast"], default="exact")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched / adjoint / indicator measurements")
    ap.add_argument("--only", choices=["batched", "adjoint", "indicators", "tunes", "constructs",
                                       "kicks", "ghosts", "long_horizon"], default=None,
                    help="run one supplementary measurement alone and print its JSON")
    ap.add_argument("--extra-side", type=int, default=None,
                    help="grid side of --only indicators / tunes (default 512 / 128)")
    ap.add_argument("--extra-turns", type=int, default=None,
                    help="turns of --only indicators / tunes (default 1e5 / 1e4)")
    ap.add_argument("--stage-turns", type=int, default=None,
                    help="turn records per staged bulk copy (0: direct reads; "
                         "default: the library's setting)")
    return ap.parse_args()


def workload_config(args, n_gpus):
    return {"workload": "modulated DA scan: 1024x1024 grid x0,y0 in [0,0.6], px0=py0=0, "
                        "SPS eps in {1,16,64} x mu in {0,0.2}, 1e5 turns, barrier 10",
            "particles_per_gpu": args.side * args.side, "turns": args.turns,
            "epsilon": list(EPSILONS), "mu": list(MUS), "tunes": list(TUNES),
            "arith": args.arith, "parallelism": f"particle shards x{n_gpus}",
            "l2": "flushed between steps (256 MiB write); state < L2, compute-bound"}


def grid_slice(side: int, rank: int, world: int):
    """Rank's interleaved slice of a side x (side*world) grid on [0, 0.6]^2."""
    xs = np.linspace(0.0, 0.6, side * world)[rank::world]
    ys = np.linspace(0.0, 0.6, side)
    xx, yy = np.meshgrid(xs, ys)
    x = np.ascontiguousarray(xx.ravel())
    y = np.ascontiguousarray(yy.ravel())
    return x, np.zeros_like(x), y, np.zeros_like(y)


# ---- clocks --------------------------------------------------------------------

def smi_id(local: int) -> str:
    """nvidia-smi's name for CUDA device `local`: nvidia-smi numbers all of
    the machine's GPUs, CUDA only those in CUDA_VISIBLE_DEVICES (given as
    indices or UUIDs), so the visible list maps one onto the other."""
    vis = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    if local < len(vis):
        return vis[local]
    return str(local)


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during a region."""

    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = smi_id(device_index)
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            if self.thread:
                self.thread.join(timeout=2)

    def summary(self):
        mhz, maxs, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                mhz.append(float(parts[0]))
                maxs.append(float(parts[1]))
            except ValueError:
                continue
            for name, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(name)
        if not mhz:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(mhz), "sm_min_mhz": min(mhz), "sm_max_mhz": max(maxs),
                "reasons": sorted(reasons), "samples": len(mhz)}


# ---- CPU baseline (the reference's own CPU path) -----------------------------------

# The CPU sample: every CPU_STRIDE-th grid point per axis (43^2 = 1849 of the
# 1024^2 grid), all six scans, the full turn count -- about 1.1e9 nominal
# particle-turns, about 5 s on the 16 host cores of a B200 box.  The same
# sample in the reference arm (one run per step) and in the GPU arm's
# cpu_baseline leg (best of 3).
CPU_STRIDE = 24


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_cpu_sample(turns: int, side: int, repeats: int = 1, stride: int = CPU_STRIDE):
    """Runs the reference's CPU tracker (henon_tracker::track,
    src/henon.cu:2701-2752, all host threads) on the fixed strided sample of
    the grid for all six (eps, mu) scans, `repeats` times on the same
    inputs; the value is the best run's."""
    from oracle import oracle as O

    R = O.reference_module("default") or O.reference_module("fmad_off")
    kind = "reference"
    if R is None:
        kind = "port"
    x, px, y, py = grid_slice(side, 0, 1)
    sel = np.zeros((side, side), bool)
    sel[::stride, ::stride] = True
    sel = sel.ravel()
    sx, spx, sy, spy = (np.ascontiguousarray(a[sel]) for a in (x, px, y, py))
    n = sx.size
    best, runs, results = None, [], {}
    for _ in range(max(1, repeats)):
        results = {}
        t0 = time.perf_counter()
        for eps in EPSILONS:
            if kind == "reference":
                tr = R.henon_tracker(turns, TUNES[0], TUNES[1], "sps", float("nan"), eps, 0)
            else:
                tabs = O.tables(turns, TUNES[0], TUNES[1], "sps", epsilon=eps)
            for mu in MUS:
                if kind == "reference":
                    p = R.particles_4d(sx, spx, sy, spy)
                    tr.track(p, turns, mu, BARRIER)
                    results[(eps, mu)] = p
                else:
                    results[(eps, mu)] = O.track(sx, spx, sy, spy, np.zeros(n, np.uint32), tabs,
                                                 turns, mu, BARRIER)
        dt = time.perf_counter() - t0
        runs.append(dt)
        best = dt if best is None else min(best, dt)
    dt = best
    nominal = n * turns * len(EPSILONS) * len(MUS)
    cores = os.cpu_count() if kind == "reference" else O.max_threads()
    # Final states of the sample (outside the timed region), for the parity
    # check of the GPU's exact arithmetic against this CPU path.
    states = {}
    for key, r in results.items():
        if kind == "reference":
            states[key] = tuple(np.asarray(a) for a in (r.get_x(), r.get_px(), r.get_y(),
                                                        r.get_py(), r.get_steps()))
        else:
            states[key] = tuple(np.asarray(a) for a in r[:5])
    return {"value": nominal / dt, "unit": UNIT, "cores": cores, "kind": kind,
            "cpu_model": cpu_model(),
            "sample": f"every {stride}th grid point per axis ({n} particles) x {turns} turns x "
                      f"6 (eps, mu) scans = {nominal:.3g} nominal particle-turns; best of "
                      f"{len(runs)} runs on the same inputs: {dt:.2f} s (table setup included)",
            "runs_s": runs, "_sel": np.flatnonzero(sel), "_states": states}


# ---- supplementary measurements (one GPU) ---------------------------------------------

def bench_batched(C, arith, both_arith=True):
    """Mixed-size workload: 64 parameter sets, log-uniform 1k-256k particles
    in the 4D ball r < 0.6 and 1e3-1e6 turns, as one batch (graph replay)
    versus one plain tracking call per set at the tracker's tuned shape for
    the same arithmetic.  Survival counts must agree.
    The batch runs the autotuner's shape for this GPU model and arithmetic
    (autotune.batch_shape: the committed cache, or a tuning run); with
    both_arith the other arithmetic is measured too, both arms in it."""
    import torch

    from henon_map_cpp_b200 import autotune, sweep

    sets, coords = sweep.heterogeneous_sets(seed=20261203)
    shape = autotune.batch_shape(sets, coords, arith)
    b = C.Batch(sets)
    autotune.configure_batch(b, shape, arith)
    b.load(*coords)
    b.run(True)  # capture + warm-up
    times = []
    for _ in range(2):
        t0 = time.perf_counter()
        b.run(True)
        times.append(time.perf_counter() - t0)
    t_batch = min(times)
    steps_batch = b.get(C.FIELD_STEPS)
    # the same batch tracked as one group on the whole device (no overlap of
    # chunk ramp-downs)
    b.set_groups(1)
    b.set_grid_share(0.0)
    b.run(True)
    t0 = time.perf_counter()
    b.run(True)
    t_one_group = time.perf_counter() - t0
    autotune.configure_batch(b, shape, arith)
    # plain: one chunked tracking call per set on device arrays, at the
    # tracker's own tuned shape for this arithmetic (restored afterwards)
    saved_config, saved_staging = C.get_track_config(), C.get_track_staging()
    plain_shape = autotune.apply(arith)
    t_plain, equal, o = 0.0, True, 0
    stream = torch.cuda.current_stream().cuda_stream
    for s in sets:
        n = s["n_particles"]
        tr = C.Tracker(s["n_turns"], s["omega_x"], s["omega_y"], "sps", float("nan"),
                       s["epsilon"], 0)
        dev = [torch.from_numpy(np.ascontiguousarray(c[o:o + n])).cuda() for c in coords]
        st = torch.zeros(n, dtype=torch.int32, device="cuda")
        ws = torch.empty(C.load().hm_track_workspace_bytes(n), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        C.call("hm_track_device", *[d.data_ptr() for d in dev], st.data_ptr(), n,
               tr.device_tables(), s["n_turns"], 0, s["n_turns"], s["mu"], s["barrier"], 0,
               arith, ws.data_ptr(), stream)
        torch.cuda.synchronize()
        t_plain += time.perf_counter() - t0
        equal &= bool(np.array_equal(st.cpu().numpy().view(np.uint32), steps_batch[o:o + n]))
        o += n
    C.set_track_config(*saved_config)
    C.set_track_staging(saved_staging)
    nominal = float(sum(s["n_particles"] * s["n_turns"] for s in sets))
    out = {"workload": "64 sets, tunes U[0.15,0.32], eps U[0,64], mu U[-0.5,0.5], "
                       "log-uniform 1e3-2.56e5 particles in the 4D ball r<0.6, "
                       "log-uniform 1e3-1e6 turns (seed 20261203)",
           "arith": "fast" if arith == C.ARITH_FAST else "exact",
           "tuned_shape": shape, "shape_source": "autotune.batch_shape (tuning.json)",
           "plain_track_shape": plain_shape,
           "particles": int(sum(s["n_particles"] for s in sets)),
           "nominal_particle_turns": nominal, "executed_particle_turns": float(steps_batch.sum()),
           "batched_s": t_batch, "one_group_s": t_one_group, "plain_sum_s": t_plain,
           "speedup": t_plain / t_batch,
           "batched_value": nominal / t_batch, "survival_equal_to_plain": equal,
           "n_chunks": b.n_chunks(), "timing": "wall clock around synchronous runs, best of 2"}
    if both_arith:
        other = C.ARITH_FAST if arith == C.ARITH_EXACT else C.ARITH_EXACT
        o = bench_batched(C, other, both_arith=False)
        out["other_arith"] = {k: o[k] for k in ("arith", "tuned_shape", "plain_track_shape",
                                                  "batched_s", "plain_sum_s", "speedup",
                                                  "survival_equal_to_plain")}
    return out


def bench_long_horizon(C, arith, side=1024, turns=1_000_000):
    """The DA scan's second horizon: the same 1024^2 grid and six (eps, mu)
    scans tracked for 1e6 turns, one pass, CUDA events around each scan."""
    import torch

    x0, px0, y0, py0 = grid_slice(side, 0, 1)
    n = x0.size
    dev0 = [torch.from_numpy(a).cuda() for a in (x0, px0, y0, py0)]
    work = [torch.empty_like(d) for d in dev0]
    steps = torch.zeros(n, dtype=torch.int32, device="cuda")
    ws = torch.empty(C.load().hm_track_workspace_bytes(n), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    total_ms, executed, flops, per_scan = 0.0, 0.0, 0.0, {}
    for eps in EPSILONS:
        tr = C.Tracker(turns, TUNES[0], TUNES[1], "sps", float("nan"), eps, 0)
        for mu in MUS:
            for w, d in zip(work, dev0):
                w.copy_(d)
            steps.zero_()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            C.call("hm_track_device", *[w.data_ptr() for w in work], steps.data_ptr(), n,
                   tr.device_tables(), turns, 0, turns, mu, BARRIER, 0, arith, ws.data_ptr(),
                   stream.cuda_stream)
            b.record(stream)
            b.synchronize()
            ms = a.elapsed_time(b)
            e = float(steps.sum(dtype=torch.int64).item())
            total_ms += ms
            executed += e
            flops += e * FLOPS_PER_TURN[mu != 0.0]
            per_scan[f"eps{eps:g}_mu{mu:g}"] = {
                "ms": ms, "survivors": int((steps == turns).sum().item())}
    return {"workload": f"{side}x{side} grid on [0,0.6]^2, SPS eps in {{1,16,64}} x mu in "
                        f"{{0,0.2}}, {turns} turns, barrier 10",
            "seconds": total_ms * 1e-3,
            "nominal_particle_turns_per_s": n * turns * 6 / (total_ms * 1e-3),
            "executed_particle_turns_per_s": executed / (total_ms * 1e-3),
            "achieved_tflops": flops / (total_ms * 1e-3) / 1e12, "scans": per_scan,
            "timing": "CUDA events around each scan's hm_track_device call, one pass"}


def bench_adjoint(C):
    """Adjoint of the Birkhoff-weighted orbit loss: 65,536 particles,
    x0, y0 ~ U[0, 0.3], px0, py0 ~ N(0, 0.01^2), eps 16, mu 0.1, 1e4 turns,
    checkpoints every 100 turns; versus one forward tracking pass."""
    import math

    import torch

    from henon_map_cpp_b200 import autograd as AG

    rng = np.random.default_rng(5)
    n, nt = 65_536, 10_000
    pts = [torch.tensor(a, device="cuda") for a in
           (rng.uniform(0, 0.3, n), rng.normal(0, 0.01, n), rng.uniform(0, 0.3, n),
            rng.normal(0, 0.01, n))]
    theta = torch.tensor([2 * math.pi * 0.168, 2 * math.pi * 0.201, 16.0, 0.1],
                         dtype=torch.float64)

    def timed(fn, reps=3):
        fn()
        best = 1e30
        for _ in range(reps):
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            b.synchronize()
            best = min(best, a.elapsed_time(b) * 1e-3)
        return best

    import ctypes

    per_thread = {}
    saved = ctypes.c_int()
    C.call("hm_get_adjoint_config", ctypes.byref(saved))
    for pt in (1, 2):
        C.call("hm_set_adjoint_config", pt)
        per_thread[pt] = timed(lambda: AG.per_particle(*pts, theta, nt, checkpoint_every=100,
                                                       reverse="inverse"))
    C.call("hm_set_adjoint_config", saved.value)
    t_adj = per_thread[saved.value]
    t_replay = timed(lambda: AG.per_particle(*pts, theta, nt, checkpoint_every=100,
                                             reverse="replay"))
    t_loss = timed(lambda: AG.per_particle(*pts, theta, nt, mode="loss"))
    tr = C.Tracker(nt, 0.168, 0.201, "sps", float("nan"), 16.0, 0)
    work = [torch.empty_like(p) for p in pts]
    st = torch.zeros(n, dtype=torch.int32, device="cuda")
    ws = torch.empty(C.load().hm_track_workspace_bytes(n), dtype=torch.uint8, device="cuda")

    def track():
        for w_, p in zip(work, pts):
            w_.copy_(p)
        st.zero_()
        C.call("hm_track_device", *[w_.data_ptr() for w_ in work], st.data_ptr(), n,
               tr.device_tables(), nt, 0, nt, 0.1, 10.0, 0, C.ARITH_EXACT, ws.data_ptr(),
               torch.cuda.current_stream().cuda_stream)

    t_track = timed(track)
    r = AG.per_particle(*pts, theta, nt, checkpoint_every=100)
    return {"workload": "65,536 particles, 1e4 turns, eps 16, mu 0.1, checkpoints every 100",
            "adjoint_s": t_adj, "adjoint_particles_per_thread": saved.value,
            "adjoint_s_by_particles_per_thread": {str(k): v for k, v in per_thread.items()},
            "adjoint_replay_s": t_replay, "forward_track_s": t_track,
            "forward_loss_s": t_loss, "adjoint_over_forward_track": t_adj / t_track,
            "reverse_sweep": "inverse map from the next checkpoint (replay variant also timed)",
            "survivors": int(r["survived"].sum().item()),
            "timing": "CUDA events, best of 3 after one warm-up"}


def bench_indicators(C, turns=100_000, side=512):
    """Tangent map + indicators fused: 512x512 grid on [0, 0.4]^2, eps 32,
    mu 0, windows at the 13 log-spaced turns 1e2..1e5 (MEGNO, Birkhoff-MEGNO,
    Lyapunov with tangent vectors, Birkhoff tunes)."""
    import torch

    v = np.linspace(0.0, 0.4, side)
    xx, yy = np.meshgrid(v, v)
    x, y = xx.ravel(), yy.ravel()
    z = np.zeros_like(x)
    n = x.size
    T = [int(t) for t in np.unique(np.round(np.logspace(2, 5, 13)))]

    def run(nt):
        tr = C.Tracker(nt + 1, 0.168, 0.201, "sps", float("nan"), 32.0, 0)
        p = C.Particles(x, z, y, z)
        objs = dict(matrix=C.Matrices(n), megno=C.Megno(n), megno_birkhoff=C.MegnoBirkhoff(n, T),
                    vectors=C.Vectors(np.tile([1.0, 0.0, 0.0, 0.0], (n, 1))),
                    lyapunov=C.Lyapunov(n, T), tune=C.TuneBirkhoff(n, T))
        objs["tune"].first_add(p)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        C.track_indicators(tr, p, nt, 0.0, 10.0, **objs)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, p

    run(1000)
    dt, p = run(turns)
    steps = p.get(C.FIELD_STEPS)
    return {"workload": f"{side}x{side} grid on [0,0.4]^2, eps 32, mu 0, {turns} turns, "
                        "MEGNO + Birkhoff-MEGNO + Lyapunov + Birkhoff tunes at 13 windows",
            "seconds": dt, "nominal_particle_turns_per_s": n * turns / dt,
            "executed_particle_turns_per_s": float(steps.sum()) / dt,
            "timing": "wall clock around one synchronous call (4096-turn launches)"}


def bench_constructs(C, turns=1000, side=256):
    """The reference's per-turn construct loop (tests/test_new_standard.ipynb:
    one call per construct and turn, 7 launches a turn) against the fused
    call, on the same 256x256 grid on [0, 0.4]^2 (eps 32, mu 0), MEGNO,
    Birkhoff-MEGNO, Lyapunov with tangent vectors and Birkhoff tunes at the
    windows 100, 300, 1000."""
    import torch

    v = np.linspace(0.0, 0.4, side)
    xx, yy = np.meshgrid(v, v)
    x, y = xx.ravel(), yy.ravel()
    z = np.zeros_like(x)
    n = x.size
    T = [100, 300, 1000]

    def setup():
        tr = C.Tracker(turns + 1, 0.168, 0.201, "sps", float("nan"), 32.0, 0)
        p = C.Particles(x, z, y, z)
        o = dict(matrix=C.Matrices(n), matrix_old=C.Matrices(n), megno=C.Megno(n),
                 megno_birkhoff=C.MegnoBirkhoff(n, T),
                 vectors=C.Vectors(np.tile([1.0, 0.0, 0.0, 0.0], (n, 1))),
                 lyapunov=C.Lyapunov(n, T), tune=C.TuneBirkhoff(n, T))
        o["tune"].first_add(p)
        return tr, p, o

    tr, p, o = setup()
    J = C.Matrices(n)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(turns):
        o["matrix_old"].explicit_copy(o["matrix"])
        tr.track(p, 1, 0.0, 10.0)
        o["matrix"].structured_multiply(tr, p, 0.0)
        o["megno"].add(o["matrix"], o["matrix_old"])
        o["megno_birkhoff"].add(o["matrix"], o["matrix_old"])
        J.set_with_tracker(tr, p, 0.0)
        o["vectors"].multiply(J)
        o["lyapunov"].add(o["vectors"])
        o["vectors"].normalize()
        o["tune"].add(p)
    torch.cuda.synchronize()
    per_call_s = time.perf_counter() - t0
    per_call_megno = o["megno"].get()

    tr, p, o = setup()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    C.track_indicators(tr, p, turns, 0.0, 10.0, **o)
    torch.cuda.synchronize()
    fused_s = time.perf_counter() - t0
    same = bool(np.array_equal(o["megno"].get(), per_call_megno, equal_nan=True))
    return {"workload": f"{side}x{side} grid on [0,0.4]^2, eps 32, mu 0, {turns} turns, MEGNO + "
                        "Birkhoff-MEGNO + Lyapunov + Birkhoff tunes at windows 100/300/1000",
            "per_call_s": per_call_s, "fused_s": fused_s, "speedup": per_call_s / fused_s,
            "fused_particle_turns_per_s": n * turns / fused_s,
            "per_call_particle_turns_per_s": n * turns / per_call_s,
            "megno_bit_equal": same,
            "timing": "wall clock; the per-call loop issues one call per construct and turn"}


def bench_kicks(C, turns=10_000, side=512):
    """Tracking with reproducible random kicks (kick_module 1e-7 every turn,
    Philox keyed by seed, particle and turn) against the same tracking
    without kicks: 512x512 grid on [0, 0.5]^2, eps 16, mu 0.2."""
    import torch

    v = np.linspace(0.0, 0.5, side)
    xx, yy = np.meshgrid(v, v)
    x, y = xx.ravel(), yy.ravel()
    z = np.zeros_like(x)
    n = x.size
    tr = C.Tracker(turns, 0.168, 0.201, "sps", float("nan"), 16.0, 0)

    def run(kick):
        p = C.Particles(x, z, y, z)
        p.kick_seed = 12345
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tr.track(p, turns, 0.2, 10.0, kick)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, p

    run(1e-7)
    plain_s, _ = run(float("nan"))
    kicked_s, p = run(1e-7)
    _, p2 = run(1e-7)
    return {"workload": f"{side}x{side} grid on [0,0.5]^2, eps 16, mu 0.2, {turns} turns, "
                        "kick_module 1e-7",
            "kicked_s": kicked_s, "plain_s": plain_s,
            "kicked_particle_turns_per_s": n * turns / kicked_s,
            "kicked_over_plain_time": kicked_s / plain_s,
            "reproducible": bool(np.array_equal(p.get(C.FIELD_X), p2.get(C.FIELD_X),
                                                equal_nan=True)),
            "timing": "wall clock around one hm_track call"}


def bench_ghosts(C, turns=1000, side=256, every=10, fused_turns=20_000):
    """The displacement (ghost) Lyapunov loop of tests/test_new_standard.ipynb
    on 256x256 base particles on [0, 0.5]^2 with x and y ghosts at 1e-10
    (eps 64, mu 0), renormalised every 10 turns: as the notebook runs it
    through the drop-in facade (track + displacement read + renormalize per
    step, `turns` turns), and fused (track_ghost_lyapunov, `fused_turns`
    turns, the same steps); the fused result is checked against the loop on
    the loop's horizon."""
    import torch

    import henon_map_cpp_b200 as hm

    v = np.linspace(0.0, 0.5, side)
    xx, yy = np.meshgrid(v, v)
    x, y = xx.ravel(), yy.ravel()
    z = np.zeros_like(x)

    def make(n_turns):
        p = hm.particles(x, z, y, z)
        p.add_ghost(1e-10, "x")
        p.add_ghost(1e-10, "y")
        t = hm.henon_tracker(n_turns + every, 0.168, 0.201, "sps", np.nan, 64.0, 0)
        return p, t

    p, t = make(turns)
    lyap = np.zeros((x.size, 2))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(turns // every):
        t.track(p, every, 0.0)
        lyap += np.log(np.asarray(p.get_displacement_module()).reshape(x.size, 2) / 1e-10)
        p.renormalize(1e-10)
    torch.cuda.synchronize()
    loop_s = time.perf_counter() - t0

    q, tq = make(turns)
    fused_lyap = tq.track_ghost_lyapunov(q, turns // every, every, 0.0, 1e-10)
    same_state = all(np.array_equal(np.asarray(getattr(p, g)()), np.asarray(getattr(q, g)()),
                                    equal_nan=True)
                     for g in ("get_x", "get_px", "get_y", "get_py", "get_steps"))
    m = np.isfinite(lyap)
    lyap_rel = float(np.max(np.abs(fused_lyap[m] - lyap[m]) / np.maximum(np.abs(lyap[m]), 1e-300))) \
        if m.any() else 0.0

    q, tq = make(fused_turns)
    tq.track_ghost_lyapunov(q, 10, every, 0.0, 1e-10)  # warm-up
    q, tq = make(fused_turns)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tq.track_ghost_lyapunov(q, fused_turns // every, every, 0.0, 1e-10)
    torch.cuda.synchronize()
    fused_s = time.perf_counter() - t0
    n_all = 3 * x.size
    return {"workload": f"{side}x{side} base particles + x and y ghosts at 1e-10, eps 64, mu 0, "
                        f"renormalised every {every}",
            "loop_turns": turns, "loop_seconds": loop_s,
            "loop_particle_turns_per_s": n_all * turns / loop_s,
            "loop_steps_per_s": (turns // every) / loop_s,
            "fused_turns": fused_turns, "fused_seconds": fused_s,
            "fused_particle_turns_per_s": n_all * fused_turns / fused_s,
            "fused_over_loop": (n_all * fused_turns / fused_s) / (n_all * turns / loop_s),
            "fused_state_bit_equal_to_loop": bool(same_state),
            "fused_lyap_max_rel_diff": lyap_rel,
            "timing": "wall clock; each loop step is track + displacement read + renormalize; "
                      "the fused call is one synchronous call"}


# ---- reference arm ---------------------------------------------------------------

def bench_tunes(C, turns=10_000, side=128):
    """all_tunes of a 128x128 grid on [0, 0.5]^2 (eps 16, mu 0.2): the orbit
    of 1e4 turns is recorded on the device, its mean removed, then Birkhoff
    and FFT tunes of the windows [0, 1000], [1000, 5000], [5000, 1e4] and of
    the full orbit."""
    import torch

    v = np.linspace(0.0, 0.5, side)
    xx, yy = np.meshgrid(v, v)
    x, y = xx.ravel(), yy.ravel()
    z = np.zeros_like(x)
    n = x.size
    frm, to = [0, turns // 10, turns // 2], [turns // 10, turns // 2, turns]

    def run():
        tr = C.Tracker(turns, 0.168, 0.201, "sps", float("nan"), 16.0, 0)
        p = C.Particles(x, z, y, z)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b, f = C.tracker_orbit_tunes(tr, p, turns, 0.2, 10.0, frm, to, True, True)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, b

    run()
    dt, b = min((run() for _ in range(3)), key=lambda r: r[0])
    orbit_bytes = 32.0 * n * (turns + 1)
    return {"workload": f"{side}x{side} grid on [0,0.5]^2, eps 16, mu 0.2, {turns} turns, "
                        "orbit recorded, mean removed, Birkhoff + FFT tunes of 3 windows "
                        "and the full orbit",
            "seconds": dt, "nominal_particle_turns_per_s": n * turns / dt,
            "orbit_bytes": orbit_bytes, "orbit_gb_per_s": orbit_bytes / dt / 1e9,
            "finite_tunes": int(np.isfinite(b).sum()),
            "timing": "wall clock around one synchronous call (record + tunes), best of 3 "
                      "after one warm-up"}


def run_only(args):
    import torch

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    from henon_map_cpp_b200 import _capi as C

    arith = C.ARITH_FAST if args.arith == "fast" else C.ARITH_EXACT
    kw = {}
    if args.extra_side is not None:
        kw["side"] = args.extra_side
    if args.extra_turns is not None:
        kw["turns"] = args.extra_turns
    fn = {"batched": lambda: bench_batched(C, arith), "adjoint": lambda: bench_adjoint(C),
          "indicators": lambda: bench_indicators(C, **kw),
          "tunes": lambda: bench_tunes(C, **kw),
          "constructs": lambda: bench_constructs(C, **kw),
          "kicks": lambda: bench_kicks(C, **kw),
          "ghosts": lambda: bench_ghosts(C, **kw),
          "long_horizon": lambda: bench_long_horizon(C, arith, **kw)}[args.only]
    print(json.dumps({"only": args.only, **fn()}), flush=True)


def run_reference_arm(args):
    """The reference's own CPU tracker on the fixed sample (CPU_STRIDE), one
    sample run per step, on rank 0 only; value = median over the steps."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    for _ in range(args.warmup):
        reference_cpu_sample(args.turns, args.side)
    vals, times = [], []
    res = None
    for _ in range(args.steps):
        t0 = time.perf_counter()
        res = reference_cpu_sample(args.turns, args.side)
        times.append(time.perf_counter() - t0)
        vals.append(res["value"])
    value = statistics.median(vals)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * statistics.median(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args, 1), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": res["cores"],
                             "kind": res["kind"], "cpu_model": res["cpu_model"],
                             "sample": res["sample"].split("; best of")[0] +
                                       f"; one run per step, median of {len(vals)} steps",
                             "step_values": vals},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---- our arm -----------------------------------------------------------------------

def run_ours(args):
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    from henon_map_cpp_b200 import _capi as C  # fails loudly if the library is missing

    arith = C.ARITH_FAST if args.arith == "fast" else C.ARITH_EXACT
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    peak_tflops, _ = C.fp64_peak(0.3)
    # Launch shape chosen by the autotuner for this GPU model and arithmetic
    # (the committed tuning.json, or a tuning run of ~30 s when absent).
    from henon_map_cpp_b200 import autotune

    track_shape = autotune.apply(arith)
    if args.stage_turns is not None:
        C.set_track_staging(args.stage_turns)
    args.stage_turns = C.get_track_staging()

    trackers = {eps: C.Tracker(args.turns, TUNES[0], TUNES[1], "sps", float("nan"), eps, 0)
                for eps in EPSILONS}
    x0, px0, y0, py0 = grid_slice(args.side, rank, world)
    n = x0.size
    dev0 = [torch.from_numpy(a).cuda() for a in (x0, px0, y0, py0)]
    work = [torch.empty_like(d) for d in dev0]
    steps = torch.zeros(n, dtype=torch.int32, device="cuda")
    ws = torch.empty(C.load().hm_track_workspace_bytes(n), dtype=torch.uint8, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def one_step(mode):
        executed = 0.0
        flops = 0.0
        for eps in EPSILONS:
            tab = trackers[eps].device_tables()
            for mu in MUS:
                for w, d in zip(work, dev0):
                    w.copy_(d)
                steps.zero_()
                C.call("hm_track_device", *[w.data_ptr() for w in work], steps.data_ptr(), n,
                       tab, args.turns, 0, args.turns, mu, BARRIER, 0, mode, ws.data_ptr(), sptr)
                s = float(steps.sum(dtype=torch.int64).item())
                executed += s
                flops += s * FLOPS_PER_TURN[mu != 0.0]
        return executed, flops

    def final_states(mode):
        """One untimed step; each scan's final x, px, y, py, steps (host)."""
        out = {}
        for eps in EPSILONS:
            tab = trackers[eps].device_tables()
            for mu in MUS:
                for w, d in zip(work, dev0):
                    w.copy_(d)
                steps.zero_()
                C.call("hm_track_device", *[w.data_ptr() for w in work], steps.data_ptr(), n,
                       tab, args.turns, 0, args.turns, mu, BARRIER, 0, mode, ws.data_ptr(), sptr)
                out[(eps, mu)] = tuple(w.cpu().numpy() for w in work) + (
                    steps.cpu().numpy().view(np.uint32),)
        return out

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    prof_work = {}

    def timed(mode, n_steps, n_warm):
        for _ in range(n_warm):
            one_step(mode)
        barrier()
        C.set_profiling(True)
        total_ms, executed, flops = 0.0, 0.0, 0.0
        for _ in range(n_steps):
            flush.zero_()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            e, f = one_step(mode)
            b.record(stream)
            b.synchronize()
            total_ms += a.elapsed_time(b)
            executed += e
            flops += f
        kernel_ms, launches = C.get_profile()
        prof_work["list_particles"], prof_work["chunk_turns"] = C.get_profile_work()
        C.set_profiling(False)
        barrier()
        return total_ms, executed, flops, kernel_ms, launches

    with ClockSampler(local) as clocks:
        total_ms, executed, flops, kernel_ms, launches = timed(arith, args.steps, args.warmup)
    clock_summary = clocks.summary()
    # Bytes per launch: algorithmic (36 B in + 36 B out per list particle,
    # 32 B of records per turn) and DRAM traffic scaled from an ncu capture
    # of the same kernel (NCU_BYTES_PER_LIST_PARTICLE).
    lp, ct = prof_work["list_particles"], prof_work["chunk_turns"]
    algo_bytes = (72.0 * lp + 32.0 * ct) / launches if launches else None
    traffic = (NCU_BYTES_PER_LIST_PARTICLE * lp + 32.0 * ct) / launches if launches else None

    # Whole-job numbers: max time over ranks, sum of work.
    rank_ms = [total_ms / args.steps]
    if dist is not None:
        every = [torch.zeros(1, dtype=torch.float64, device="cuda") for _ in range(world)]
        dist.all_gather(every, torch.tensor([total_ms], dtype=torch.float64, device="cuda"))
        rank_ms = [float(t_.item()) / args.steps for t_ in every]
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        w = torch.tensor([executed, flops], dtype=torch.float64, device="cuda")
        dist.all_reduce(w, op=dist.ReduceOp.SUM)
        executed, flops = (float(v) for v in w.tolist())
    nominal = float(n) * args.turns * len(EPSILONS) * len(MUS) * args.steps * world
    value = nominal / (total_ms * 1e-3)

    # Roofline of the tracking kernel on this rank (per-launch average).
    local_flops = flops / world if dist is not None else flops
    achieved_tf = local_flops / (kernel_ms * 1e-3) / 1e12 if kernel_ms > 0 else 0.0

    # The other arithmetic, for reference (not the headline), in its own
    # tuned shape.
    other = C.ARITH_EXACT if arith == C.ARITH_FAST else C.ARITH_FAST
    other_shape = autotune.apply(other)
    o_ms, o_exec, o_flops, o_kms, _ = timed(other, 1, 1)
    autotune.apply(arith)
    if args.stage_turns is not None:
        C.set_track_staging(args.stage_turns)
    o_tf = o_flops / (o_kms * 1e-3) / 1e12 if o_kms > 0 else 0.0
    if dist is not None:
        t = torch.tensor([o_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        o_ms = float(t.item())
    o_value = float(n) * args.turns * 6 * world / (o_ms * 1e-3)

    # Turn records read directly vs staged through shared memory by bulk
    # copies (one step each, same workload and arithmetic).
    staging = None
    if world == 1 and not args.no_extras:
        staging = {"workload": "the headline step, one timed step per setting",
                   "unit": "achieved FP64 TFLOP/s of track_chunk_kernel"}
        default_stage = C.get_track_staging()
        for st in (0, 64, 256, 512):
            C.set_track_staging(st)
            _, _, s_flops, s_kms, _ = timed(arith, 1, 1)
            staging[str(st)] = s_flops / (s_kms * 1e-3) / 1e12 if s_kms > 0 else None
        C.set_track_staging(default_stage)

    # End to end through the public API with host buffers.
    e2e = None
    if not args.no_e2e:
        pinned = [torch.from_numpy(a).pin_memory().numpy() for a in (x0, px0, y0, py0)]
        out_steps = torch.empty(n, dtype=torch.int32).pin_memory().numpy().view(np.uint32)

        phase_s = {"create": 0.0, "track": 0.0, "get": 0.0, "destroy": 0.0}

        def e2e_step():
            for eps in EPSILONS:
                for mu in MUS:
                    t0 = time.perf_counter()
                    p = C.Particles(*pinned)
                    t1 = time.perf_counter()
                    p_tr = trackers[eps]
                    p_tr.arith = arith
                    p_tr.track(p, args.turns, mu, BARRIER)
                    t2 = time.perf_counter()
                    C.call("hm_particles_get", p.h, C.FIELD_STEPS,
                           out_steps.ctypes.data_as(C.c_void_p))
                    t3 = time.perf_counter()
                    del p
                    t4 = time.perf_counter()
                    for k, dt in zip(phase_s, (t1 - t0, t2 - t1, t3 - t2, t4 - t3)):
                        phase_s[k] += dt

        e2e_step()
        barrier()
        for k in phase_s:
            phase_s[k] = 0.0
        C.set_profiling(True)
        with ClockSampler(local) as e2e_clocks:
            t0 = time.perf_counter()
            for _ in range(args.steps):
                e2e_step()
            torch.cuda.synchronize()
            e2e_s = time.perf_counter() - t0
        e2e_kernel_ms, _ = C.get_profile()
        C.set_profiling(False)
        if dist is not None:
            t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = {"value": float(n) * args.turns * 6 * world * args.steps / e2e_s, "unit": UNIT,
               "steps": args.steps,
               "h2d_bytes_per_step": 6 * 4 * 8 * n, "d2h_bytes_per_step": 6 * 4 * n,
               "ms_per_step": e2e_s * 1e3 / args.steps,
               "kernel_ms_per_step": e2e_kernel_ms / args.steps,
               "phase_ms_per_step": {k: v * 1e3 / args.steps for k, v in phase_s.items()},
               "clocks": e2e_clocks.summary(),
               "path": "hm_particles_create (pinned host) -> hm_track -> hm_particles_get(steps)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = reference_cpu_sample(args.turns, args.side, repeats=3)

    # Parity of this run's results (one untimed step per arithmetic): the
    # exact arithmetic against the reference's CPU path on the CPU leg's
    # sample, bit for bit; the fast arithmetic against the exact on the
    # whole grid (survival turns).
    parity = None
    if world == 1:
        exact_states = final_states(C.ARITH_EXACT)
        fast_states = final_states(C.ARITH_FAST)
        pts = same_steps = same_survival = 0
        for key, (_, _, _, _, se) in exact_states.items():
            sf = fast_states[key][4]
            pts += se.size
            same_steps += int(np.count_nonzero(se == sf))
            same_survival += int(np.count_nonzero((se == args.turns) == (sf == args.turns)))
        parity = {"fast_vs_exact": {"grid_points": pts,
                                    "survival_turns_equal": same_steps / pts,
                                    "survival_equal": same_survival / pts}}
        del fast_states
        if cpu is not None:
            sel = cpu["_sel"]
            n_cmp = steps_eq = coords_eq = 0
            for key, ref in cpu["_states"].items():
                got = exact_states[key]
                n_cmp += sel.size
                steps_eq += int(np.count_nonzero(got[4][sel] == ref[4].astype(np.uint32)))
                same = np.ones(sel.size, bool)
                for k in range(4):
                    a = got[k][sel].copy()
                    b = np.array(ref[k], dtype=np.float64)
                    a[np.isnan(a)] = np.nan  # one NaN pattern on both sides
                    b[np.isnan(b)] = np.nan
                    same &= a.view(np.uint64) == b.view(np.uint64)
                coords_eq += int(np.count_nonzero(same))
            parity["exact_vs_cpu_baseline"] = {
                "kind": cpu["kind"], "particles": n_cmp,
                "survival_turns_equal": steps_eq / n_cmp, "coordinates_bit_equal": coords_eq / n_cmp}
        del exact_states
    if cpu is not None:
        cpu = {k: v for k, v in cpu.items() if not k.startswith("_")}

    extras = {}
    if world == 1 and not args.no_extras:
        extras["long_horizon"] = bench_long_horizon(C, arith)
        extras["batched"] = bench_batched(C, arith)
        extras["adjoint"] = bench_adjoint(C)
        extras["indicators"] = bench_indicators(C)
        extras["tunes"] = bench_tunes(C)
        extras["constructs"] = bench_constructs(C)
        extras["kicks"] = bench_kicks(C)
        extras["ghosts"] = bench_ghosts(C)

    if rank == 0:
        peak_unit = "TFLOP/s"
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args, world),
            "rank_ms_per_step": rank_ms,
            "track_shape": track_shape,
            "executed_particle_turns_per_s": executed / (total_ms * 1e-3),
            "survivor_fraction": executed / nominal,
            "roofline": {"bound": "fp64", "achieved": achieved_tf, "peak": peak_tflops,
                         "unit": peak_unit, "frac": achieved_tf / peak_tflops if peak_tflops else None,
                         "traffic": traffic,
                         "traffic_source": "bytes per launch: DRAM read+write per list particle "
                                           "from ncu (32.1 B, 512^2 DA scan, staged kernel) x list "
                                           "particles + 32 B of records per turn",
                         "algorithmic_bytes": algo_bytes,
                         "peak_source": "FP64 FMA-chain microbenchmark in this process "
                                        "(hm_fp64_peak; FMA = 2 flops)",
                         "kernel": "track_chunk_kernel", "kernel_ms": kernel_ms,
                         "launches": launches},
            "other_arith": {"arith": "fast" if other == C.ARITH_FAST else "exact",
                            "track_shape": other_shape,
                            "value": o_value, "achieved_tflops": o_tf,
                            "frac": o_tf / peak_tflops if peak_tflops else None},
            "table_staging": staging,
            "gpu_launches": launches,
            "clocks": clock_summary,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "parity": parity,
            **extras,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def launch_ranks(n: int, argv: list[str]) -> int:
    """Re-executes this script as n ranks under torch.distributed.run on this
    node (rendezvous on 127.0.0.1), the command the multi-GPU runs use; NCCL
    logs its communicator set-up (NCCL_DEBUG=INFO, INIT subsystem) unless the
    caller chose otherwise.  Returns torchrun's exit status."""
    import socket

    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    env = dict(os.environ)
    env.setdefault("NCCL_DEBUG", "INFO")
    env.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={n}", "--master-addr", "127.0.0.1", f"--master-port={port}",
           str(Path(__file__).resolve()), *argv]
    return subprocess.call(cmd, env=env)


def check_world(args) -> None:
    """Under torchrun the rank count must be the one --gpus asks for."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}")


def run_launch_check(args) -> None:
    """Joins the ranks in a process group (NCCL when GPUs are visible, gloo
    otherwise), gathers (rank, local rank, device) from each and prints one
    line from rank 0."""
    import datetime

    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    use_gpu = torch.cuda.is_available()
    backend = "nccl" if use_gpu else "gloo"
    me = {"rank": rank, "local_rank": local,
          "device": torch.cuda.get_device_name(local) if use_gpu else "cpu"}
    ranks = [me]
    if world > 1:
        if use_gpu:
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
        ranks = [None] * world
        dist.all_gather_object(ranks, me)
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"launch_check": True, "n_gpus": world, "backend": backend,
                          "ranks": ranks}), flush=True)


def main():
    args = parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        raise SystemExit(launch_ranks(args.gpus, sys.argv[1:]))
    if "WORLD_SIZE" in os.environ:
        check_world(args)
    if args.launch_check:
        run_launch_check(args)
    elif args.impl == "reference":
        run_reference_arm(args)
    elif args.only:
        run_only(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
