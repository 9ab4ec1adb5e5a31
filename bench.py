"""Benchmark of the pressure-Poisson hot path on B200.

Workload (one "step"): one complete solve of the 2-D 1024 x 1024 variable-coefficient
pressure Poisson -- beta = 1/rho with rho = 1000 inside 64 seeded bubbles (radii 8-48
cells) and 1 outside, a seeded Gaussian right-hand side with zero mean -- from a zero
initial guess to ||f - A p||_2 <= 1e-10 ||f||_2 by PCG with a 6-level V(2,2) red-black
multigrid preconditioner, FP64 throughout, set-up (beta coarsening) included.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

The line also carries the RK3 time-step legs ("rk3"): the 1-D boiling column of 512 flow
cells (film 0.1, density ratio 1000, viscosity ratio 20, conductivity ratio 25, 10 K
superheat) and a batch of 4096 independent columns of uneven length (128-2048 cells, 2-20 K,
density ratio 100-1600), whole RK3 steps in one persistent launch, beside the CPU
restatement's time for the same steps; and the 2-D film-boiling step on 512 x 1536 (level
set 1024 x 3072) with FP64 and mixed-precision pressure solves, its fields after one step
compared with the FP64 CPU restatement.  "bubble_tracking" times BUBBLE_TRACKING +
BUBBLE_EIGENV of four level sets on a 256^3 grid (one launch) against the CPU restatement.

Under torchrun each rank solves its own replica (the 2-D multigrid does not shard
here); value = solves of all ranks / the slowest rank's time.  Rank 0 prints one JSON
line.  --impl reference times the CPU restatement of the same solve (the reference has
no GPU path and cannot be compiled here) on all host cores, rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK3 steps/s & MG solves/s at 1e-10 residual: plain FP64 vs mixed+learned"
UNIT = "MG solves/s"
N = 1024
NLEVELS = 6
RTOL = 1e-10
WORKLOAD = ("2-D 1024x1024 variable-coefficient pressure Poisson, beta=1/rho with rho 1000:1 in 64 seeded "
            "bubbles (radii 8-48 cells), Gaussian RHS; PCG with 6-level V(2,2) red-black multigrid "
            "preconditioner to 1e-10 relative residual from p=0, set-up included; coarsest level by one inner V-cycle")


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks sampler
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu=uuid,{self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            if self.uuid and parts[0].lower().replace("gpu-", "") != self.uuid:
                continue
            self.samples.append(parts[1:])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        smax = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for name, v in zip(names, s[4:8]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ------------------------------------------------------------------ CPU legs (oracle)
def cpu_solves(case, max_seconds, max_solves, mixed=False):
    """Time the CPU restatement of the same solve (OpenMP on all host cores)."""
    from oracle import oracle
    oracle.lib(native=True)
    times, its = [], []
    t_all = time.perf_counter()
    while len(times) < max_solves:
        t0 = time.perf_counter()
        _, it, rel, _, st = oracle.mg_solve(case.f, case.bx, case.by, case.hx, case.hy, nlevels=NLEVELS, ncoarse=1,
                                           sym=5, method="pcg", mixed=mixed, rtol=RTOL, max_cycles=200, native=True)
        times.append(time.perf_counter() - t0)
        its.append(it)
        if time.perf_counter() - t_all > max_seconds:
            break
    return times, its


def bench_config(n, nlevels, ncoarse, precision, world):
    """The workload's config dict, the same in both arms."""
    workload = WORKLOAD if n == N else WORKLOAD.replace("1024x1024", f"{n}x{n}").replace(
        "6-level", f"{nlevels}-level")
    return {"workload": workload, "nx": n, "ny": n, "nlevels": nlevels, "nu1": 2, "nu2": 2, "ncoarse": ncoarse,
            "rtol": RTOL, "solver": "MG-PCG", "precision": precision, "l2_flush": "256 MiB write between steps",
            "parallelism": f"replicas x{world}"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from lica_boiling1d_b200.inputs import bubble_poisson_case
    threads = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    case = bubble_poisson_case(N)
    mixed = args.precision == "mixed"
    cpu_solves(case, 1e9, max(1, args.warmup), mixed)  # warm-up (also builds the native oracle)
    times, its = cpu_solves(case, 1e9, args.steps, mixed)
    total = sum(times)
    value = len(times) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": len(times), "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f64+f32", "data": "synthetic",
        "config": bench_config(N, NLEVELS, args.ncoarse, args.precision, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "port",
                         "sample": f"{len(times)} complete solves (one per step), FP64 C++/OpenMP restatement"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "iterations": its[-1],
    }
    line["rk3"] = {"cpu_baseline": rk3_cpu()[0]}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ RK3 column legs
COLUMN512 = dict(n=512, z0=0.1, denr=1000.0, visr=20.0, tcr=25.0, jakob=0.009, cflmax=0.3, steps=2000)
BATCH_NCOL = 4096


def column512_props():
    from lica_boiling1d_b200.column import ColumnProps
    return ColumnProps(denr=COLUMN512["denr"], visr=COLUMN512["visr"], tcr=COLUMN512["tcr"], jakob=COLUMN512["jakob"], cflmax=COLUMN512["cflmax"])


def column512_oracle(steps):
    """The 512-cell column on the CPU restatement, one thread (as the reference's 1-D case runs): the
    final state, the per-step interface history (TIME, place, VOL_TOT_IPHS, DT) and the
    seconds the steps took."""
    from oracle import oracle
    props = column512_props()
    st = oracle.col_init(COLUMN512["n"], 1.0, COLUMN512["z0"], props)
    hist = np.zeros((steps, 4))
    t0 = time.perf_counter()
    for s in range(steps):
        tb = float(st["scal"][1])
        if oracle.col_step(st, COLUMN512["n"], 1.0, props, native=True) != 0:
            raise RuntimeError(f"oracle column step {s + 1} failed")
        hist[s] = oracle.col_history_record(st, tb, native=True)
    return st, hist, time.perf_counter() - t0


def rk3_cpu(col_steps_n=COLUMN512["steps"]):
    """The CPU restatement's time for the same steps: the whole run of the 512-cell
    column (single thread), and a sample of the uneven batch run over all host cores
    (independent columns; the oracle releases the GIL).  Returns the figures and, apart,
    the final state and history."""
    from concurrent.futures import ThreadPoolExecutor

    from lica_boiling1d_b200.column import uneven_batch
    from oracle import oracle
    oracle.lib(native=True)
    col_state, col_hist, col_s = column512_oracle(col_steps_n)
    col_rate = col_steps_n / col_s
    k = col_steps_n
    n, length, z0, bprops = uneven_batch(BATCH_NCOL, seed=0)
    sample = list(range(0, BATCH_NCOL, max(1, BATCH_NCOL // 256)))
    states = {c: oracle.col_init(int(n[c]), float(length[c]), float(z0[c]), bprops[c]) for c in sample}
    cores = os.cpu_count()

    def run(c, steps):
        for _ in range(steps):
            oracle.col_step(states[c], int(n[c]), float(length[c]), bprops[c], native=True)
        return steps
    with ThreadPoolExecutor(cores) as ex:
        list(ex.map(lambda c: run(c, 1), sample))          # warm-up step
        t0 = time.perf_counter()
        done = sum(ex.map(lambda c: run(c, 2), sample))
        dt = time.perf_counter() - t0
    cells = float(np.mean([n[c] for c in sample]))
    col_steps = done / dt
    return {"column_512_steps_per_s": col_rate, "column_512_sample": f"all {k} steps of the 512-cell column (CFL 0.3), one thread",
            "batch_column_steps_per_s": col_steps, "batch_steps_per_s": col_steps / BATCH_NCOL,
            "batch_cell_updates_per_s": col_steps * cells, "cores": cores,
            "batch_sample": f"{len(sample)} of the {BATCH_NCOL} columns x 2 steps on {cores} threads"}, (col_state, col_hist)


def profile_batch(ncol, steps, threads):
    """Only the uneven batch: one warm-up launch of one step, then one launch of `steps`
    steps (for ncu: the second k_column_steps launch is the measured one)."""
    import torch

    from lica_boiling1d_b200.column import ColumnBatch, uneven_batch
    torch.cuda.set_device(0)
    n, length, z0, bprops = uneven_batch(ncol, seed=0)
    batch = ColumnBatch.films(n, length, z0, bprops).to("cuda")
    batch.steps(1, threads=threads)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    st = batch.steps(steps, threads=threads)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    print(json.dumps({"profile_batch": ncol, "steps": steps, "threads": threads, "ms_per_step": ms / steps,
                      "cells": int(n.sum()), "status": int(st.max())}), flush=True)


def column_roofline(state_bytes, ms_per_step, kernel):
    """HBM roofline of the fused column step: its algorithmic traffic is the column state read
    and written once per step (every other array lives in shared memory or in a scratch
    that stays in L2), timed by CUDA events over the persistent launch."""
    alg = 2 * state_bytes
    achieved = alg / (ms_per_step / 1e3) / 1e9
    peak, src = peaks()
    return {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": src, "traffic": None,
            "alg_bytes_per_step": alg,
            "note": "latency-bound, not bandwidth-bound: one CTA per column walks the step's phases in order "
                    "(three Thomas sweeps per substep on one thread, band lists, the TEMP_EXTP iterations); "
                    "the per-phase cycle profile is the lica_gpu_column_profile_device record"}


def rk3_legs(dev, flush, steps_col=COLUMN512["steps"], steps_batch=1000, warmup=3, rank=0, world=1, slowest=lambda x: x,
             film_steps=10, film_compare=False):
    import torch

    from lica_boiling1d_b200 import column as colmod
    from lica_boiling1d_b200 import native, shard
    from lica_boiling1d_b200.column import ColumnBatch, Columns, uneven_batch
    out = {}
    props = column512_props()
    # the 512-cell column: one column from its initial state, one persistent launch of steps_col steps that
    # records the interface history (warm-up on a separate copy)
    col0 = Columns.film(COLUMN512["n"], 1.0, [COLUMN512["z0"]], props)
    warm = col0.to(dev)
    warm.steps(warmup, props, threads=256)
    col = col0.to(dev)
    hist = torch.zeros((1, steps_col, 4), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush.fill_(3)
    l0 = native.launch_count()
    colmod.history(hist)
    e0.record()
    st = col.steps(steps_col, props, threads=256)
    e1.record()
    torch.cuda.synchronize(dev)
    colmod.history(None)
    launches = native.launch_count() - l0
    if int(st.max()) != 0:
        raise RuntimeError(f"column step status {int(st.max())}")
    ms = e0.elapsed_time(e1)
    out["column_512"] = {
        "workload": "1-D boiling column, 512 uniform flow cells (1024 refined), film 0.1 L, density ratio "
                    "1000, viscosity ratio 20, conductivity ratio 25, Jakob 0.009 (10 K), RK3 at CFL 0.3, "
                    f"{steps_col} steps from the initial state in one persistent launch, FP64, 1-D POISSON exact",
        "steps_per_s": steps_col / (ms / 1e3), "ms_per_step": ms / steps_col, "steps": steps_col, "threads": 256,
        "cell_updates_per_s": COLUMN512["n"] * steps_col / (ms / 1e3), "gpu_launches": launches,
        "interface_height": float(col.to(None).stats[0][5])}
    out["_column_gpu"] = (col.to(None), hist[0].cpu().numpy())
    # end to end: the host-array C-ABI entry, one step per call (state copied in and out)
    host = warm.to(None)
    pinned = {k: torch.from_numpy(v).pin_memory().numpy() for k, v in host.arrays.items()}
    hcol = Columns(COLUMN512["n"], 1.0, pinned)
    ke = 20
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(ke):
        hcol.steps(1, props)
    e2e_s = time.perf_counter() - t0
    bytes_state = sum(a.nbytes for a in pinned.values())
    out["column_512"]["roofline"] = column_roofline(bytes_state, ms / steps_col, "k_column_steps<256>")
    out["column_512"]["e2e"] = {"steps_per_s": ke / e2e_s, "h2d_bytes_per_step": bytes_state,
                                "d2h_bytes_per_step": bytes_state,
                                "path": "lica_gpu_column_steps (C ABI), host arrays, one step per call"}
    # the 4096-column batch: the uneven batch (over N ranks: contiguous blocks balanced by cells, no collective
    # per step), CTA width picked by a short trial of each candidate
    n_all, length, z0, bprops = uneven_batch(BATCH_NCOL, seed=0)
    lo, hi = shard.partition(n_all, world)[rank]
    n = n_all[lo:hi]
    batch = ColumnBatch.films(n, length[lo:hi], z0[lo:hi], bprops[lo:hi]).to(dev)
    from lica_boiling1d_b200 import autotune
    (th, cap), trial = autotune.tune(batch, force=True)
    batch.steps(warmup, threads=th, tri_cap=cap)
    torch.cuda.synchronize(dev)
    flush.fill_(5)
    l0 = native.launch_count()
    e0.record()
    st = batch.steps(steps_batch, threads=th, tri_cap=cap)
    e1.record()
    torch.cuda.synchronize(dev)
    launches = native.launch_count() - l0
    if int(st.max()) != 0:
        raise RuntimeError(f"batch status {int(st.max())}")
    ms = slowest(e0.elapsed_time(e1))
    cells = int(n_all.sum())
    # the one gather at the end: interface height and vapour volume of every column
    fin = batch.to(None).arrays
    hist = shard.gather_histories([(lo + c, float(fin["stats"][c][5]), float(fin["scal"][c][4]))
                                   for c in range(len(n))], world)
    batch_bytes = sum(int(a.numel()) * a.element_size() for a in batch.arrays.values())
    out["batch_4096"] = {
        "roofline": column_roofline(batch_bytes, ms / steps_batch, f"k_column_steps<{th}>"),
        "workload": f"{BATCH_NCOL} independent 1-D boiling columns, uneven 128-2048 flow cells (seeded, "
                    f"{cells} in total), superheat 2-20 K, density ratio 100-1600, FP64 (the 1-D pressure solve is "
                    f"the exact Thomas sweep), {steps_batch} RK3 steps in one persistent launch per rank, longest first",
        "steps_per_s": steps_batch / (ms / 1e3), "ms_per_step": ms / steps_batch, "steps": steps_batch,
        "column_steps_per_s": BATCH_NCOL * steps_batch / (ms / 1e3), "cell_updates_per_s": cells * steps_batch / (ms / 1e3),
        "threads": th, "tri_cap": cap, "autotune_ms_per_step": trial,
        "autotune": "lica_boiling1d_b200.autotune: CTA width 64/128/256 x Thomas arrays in shared memory or "
                    "scratch, timed on a copy of the batch, cached per GPU",
        "gpu_launches": launches,
        "ranks": world, "sharding": "contiguous column blocks balanced by cells, strong scaling of the fixed batch",
        "gathered_columns": len(hist)}
    if film_steps > 0:
        out["film_2d"] = film_leg(dev, flush, steps=film_steps, compare=film_compare)
    return out


# ------------------------------------------------------------------ 2-D film boiling
FILM = dict(nx=512, ny=1536, y0=64.0, amp=4.0)


BUB = dict(n=256, nlvs=4, reps=20)


def bubble_fields(dev, n, nlvs):
    """PSI_TMP of nlvs level sets on an n^3 unit-cube grid (two rotated ellipsoids each, edges
    smeared over about a cell; 1 outside) and seeded velocity fields, built on the device."""
    import torch
    from lica_boiling1d_b200.bubbles import BubbleGrid
    grid = BubbleGrid.uniform(n, n, n, 1.0, 1.0, 1.0)
    x = torch.tensor(grid.xp, device=dev).view(1, 1, -1)
    y = torch.tensor(grid.yp, device=dev).view(1, -1, 1)
    z = torch.tensor(grid.zp, device=dev).view(-1, 1, 1)
    rng = np.random.default_rng(11)
    psi = torch.ones((nlvs,) + grid.field_shape, dtype=torch.float64, device=dev)
    for q in range(nlvs):
        for _ in range(2):
            c = rng.uniform(0.25, 0.75, 3)
            ax = rng.uniform(0.06, 0.16, 3)
            rot = np.linalg.qr(rng.standard_normal((3, 3)))[0]
            d = [x - c[0], y - c[1], z - c[2]]
            r2 = sum(((d[0] * rot[0, k] + d[1] * rot[1, k] + d[2] * rot[2, k]) / ax[k]) ** 2 for k in range(3))
            phi = (torch.sqrt(r2) - 1.0) * float(ax.min())
            psi[q] = torch.minimum(psi[q], torch.clamp(0.5 + phi * (n / 1.5), 0.0, 1.0))
    psi[:, [0, -1]] = 1.0
    psi[:, :, [0, -1]] = 1.0
    psi[:, :, :, [0, -1]] = 1.0
    g = torch.Generator(device=dev).manual_seed(12)
    uvw = [torch.randn(grid.field_shape, dtype=torch.float64, device=dev, generator=g) for _ in range(3)]
    return grid, psi.contiguous(), uvw


def bubble_leg(dev, flush, compare=True):
    """BUBBLE_TRACKING + BUBBLE_EIGENV of four level sets on a 256^3 grid (one launch): level
    sets per second, the HBM roofline of the one-pass kernel, and the records against the
    oracle's two-sweep restatement, whose single-thread time is the CPU baseline."""
    import torch

    from lica_boiling1d_b200 import bubbles, native
    n, nlvs, reps = BUB["n"], BUB["nlvs"], BUB["reps"]
    grid, psi, (u, v, w) = bubble_fields(dev, n, nlvs)
    tr = bubbles.BubbleTracker(grid, nlvs)
    st = torch.cuda.current_stream(dev)
    for _ in range(3):
        raw = tr.track(psi, u, v, w, stream=st)
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    l0 = native.launch_count()
    for k in range(reps):
        flush.fill_(k & 0xFF)
        ev[k][0].record(st)
        raw = tr.track(psi, u, v, w, out=raw, stream=st)
        ev[k][1].record(st)
    torch.cuda.synchronize(dev)
    launches = native.launch_count() - l0
    ms = sum(a.elapsed_time(b) for a, b in ev) / reps
    rec = bubbles.records(raw)
    tr.close()
    interior = psi[:, 1:-1, 1:-1, 1:-1]
    gas = int((interior != 1.0).sum().item())
    cells = n ** 3
    alg = 8.0 * nlvs * cells + 24.0 * gas
    peak, src = peaks()
    achieved = alg / (ms / 1e3) / 1e9
    out = {"workload": f"BUBBLE_TRACKING + BUBBLE_EIGENV of {nlvs} level sets (two rotated ellipsoidal bubbles "
                       f"each) on a uniform {n}^3 grid, FP64, one launch; PSI_TMP fields "
                       f"{nlvs * psi[0].numel() * 8 / 1e6:.0f} MB (> L2), 256 MiB flush between launches",
           "level_sets_per_s": nlvs / (ms / 1e3), "ms_per_call": ms, "cells_per_s": nlvs * cells / (ms / 1e3),
           "gas_cells": gas, "gpu_launches": launches,
           "roofline": {"bound": "hbm", "kernel": "k_bubble", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_source": src, "traffic": None,
                        "alg_bytes_per_launch": alg,
                        "note": "8 B of PSI_TMP per cell and level set, plus U, V, W (24 B) at each gas cell"}}
    if compare:
        from oracle import oracle
        h = [a.cpu().numpy() for a in (psi, u, v, w)]
        oracle.lib()
        t0 = time.perf_counter()
        ref = oracle.bubble_tracking(grid.as_dict(), *h)
        cpu_s = time.perf_counter() - t0
        rel = lambda a, b: float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))  # noqa: E731
        out["vs_oracle"] = {"max_rel_diff_volume": rel(rec["vol"], ref["vol"]),
                            "max_rel_diff_centroid_velocity": rel(rec["col"][:, :6], ref["col"][:, :6]),
                            "max_rel_diff_eigenvalues": rel(np.sort(rec["ami"], axis=1), np.sort(ref["ami"], axis=1)),
                            "max_rel_diff_aspect_ratio": rel(rec["col"][:, 6], ref["col"][:, 6]),
                            "max_abs_diff_angles_deg": float(np.max(np.abs(rec["col"][:, 7:] - ref["col"][:, 7:]))),
                            "note": "one-pass Welford/Chan moments on the GPU against the reference's two sweeps; "
                                    "eigenvalues compared sorted (the diagonal position Jacobi leaves each in "
                                    "depends on the rotation path)"}
        out["cpu_baseline"] = {"value": nlvs / cpu_s, "unit": "level sets/s", "cores": 1, "kind": "port",
                               "sample": f"the whole workload once ({nlvs} level sets, {n}^3), oracle C++ "
                                         "restatement, one thread"}
    return out


def film_leg(dev, flush, steps=10, warmup=2, compare=True):
    """One RK3 step of 2-D film boiling on 512 x 1536 (level set 1024 x 3072; interface
    y = 64 h + 4 h cos(2 pi x), superheat 5 K via Ja), FP64 and with mixed-precision pressure
    solves: steps/s, pressure-solve iterations, and (compare) each field after one step against
    the FP64 CPU restatement, whose time is the CPU baseline.  The state starts from the
    hydrostatic pressure of the initial film."""
    import torch

    from lica_boiling1d_b200 import film2d as G
    from lica_boiling1d_b200 import native
    P = G.default_props()
    nx, ny = FILM["nx"], FILM["ny"]
    st0 = G.initial_state(nx, ny, FILM["y0"], FILM["amp"], props=P)
    dt = G.stable_dt(nx, P)
    out = {"workload": f"2-D film boiling, {nx} x {ny} MAC flow grid, level set {2 * nx} x {2 * ny}, interface "
                       f"y = {FILM['y0']:.0f} h + {FILM['amp']:.0f} h cos(2 pi x / Lx), liquid/vapour ratios of the "
                       "film-boiling benchmark (density 40, viscosity 20, conductivity 40, specific heat 2), "
                       "superheat 5 K (Ja 0.1), Re 69.2, Fr 1; one RK3 step = 3 substeps (3 incremental MG-PCG "
                       "pressure solves to 1e-10 relative residual, or to FP64's attainable accuracy where it lies "
                       "above 1e-10: LICA_STALLED) + 2 reinitialisation iterations, FP64 physics",
           "dt": dt, "inputs_vs_l2": "state and scratch (about 220 MB) larger than L2, plus a 256 MiB flush"}
    first = {}
    net = None
    from lica_boiling1d_b200 import train_guess
    arms = ["fp64", "mixed", "fp64_warm", "mixed_warm"]
    if os.path.exists(train_guess.SOLVER_PAIR_WEIGHTS):
        from lica_boiling1d_b200.unet import LearnedGuess
        net = LearnedGuess(1, ny, nx)
        train_guess.load(net, train_guess.SOLVER_PAIR_WEIGHTS)
        arms.append("mixed_learned")
    for arm in arms:
        prec = "fp64" if arm.startswith("fp64") else "mixed"
        gpu = G.Film2D(nx, ny, P, precision=prec)
        if arm == "mixed_learned":
            gpu.set_guess(net)
        if arm.endswith("_warm"):
            gpu.warm_start(True)
        state = G.to_device(st0)
        gpu.step(state, dt)
        torch.cuda.synchronize(dev)
        first[arm] = G.to_host(state)
        for _ in range(warmup):
            gpu.step(state, dt)
        torch.cuda.synchronize(dev)
        flush.fill_(7)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = native.launch_count()
        its, rels, stats, grels = [], [], [], []
        e0.record()
        for _ in range(steps):
            inf = gpu.step(state, dt)
            its.append(inf["iterations"])
            rels.append(inf["rel"])
            stats.append(inf["status"])
            grels.append(inf["guess_rel"])
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
        gpu.close()
        out[arm] = {"steps_per_s": steps / (ms / 1e3), "ms_per_step": ms / steps, "steps": steps,
                    "flow_cell_updates_per_s": nx * ny * steps / (ms / 1e3),
                    "ls_cell_updates_per_s": 4 * nx * ny * steps / (ms / 1e3),
                    "mg_iterations_per_substep": its[-1], "mg_rel_residual_per_substep": rels[-1],
                    "mg_status_per_substep": stats[-1], "gpu_launches": native.launch_count() - l0}
        if arm == "mixed_learned":
            out[arm]["guess_rel_per_substep"] = grels[-1]
            out[arm]["mean_iterations_saved_vs_mixed"] = float(np.mean(out["mixed"]["_its"]) - np.mean(its))
            out[arm]["note"] = ("mixed-precision MG-PCG started from the U-Net guess trained on 20,000 "
                                "1024^2 bubble-Poisson and 512 x 1536 film (this film's own systems) pairs; zero where the guess is "
                                "no better")
        if arm.endswith("_warm"):
            out[arm]["mean_iterations_saved_vs_cold"] = float(np.mean(out[prec]["_its"]) - np.mean(its))
            out[arm]["note"] = ("each substep's solve starts from the increment the same substep solved in the "
                                "previous step (lica_film2d_set_warm_start)")
        out[arm]["_its"] = its
    if net is not None:
        net.close()
    for arm in arms:
        out[arm].pop("_its", None)
    out["ratio_mixed_learned_vs_fp64"] = (out["mixed_learned"]["steps_per_s"] / out["fp64"]["steps_per_s"]
                                          if "mixed_learned" in out else None)
    out["ratio_mixed_vs_fp64"] = out["mixed"]["steps_per_s"] / out["fp64"]["steps_per_s"]
    out["ratio_mixed_warm_vs_fp64"] = out["mixed_warm"]["steps_per_s"] / out["fp64"]["steps_per_s"]
    if compare:
        from oracle import film2d as F
        F.step_native(G.initial_state(64, 192, 8.0, 2.0, props=P), G.stable_dt(64, P), P, 3)  # load the library
        t0 = time.perf_counter()
        ref, info = F.step_native(st0, dt, P, G.levels_for(nx, ny))
        cpu_s = time.perf_counter() - t0
        errs = {}
        for arm in arms:
            errs[arm] = {k: float(np.linalg.norm(first[arm][k] - ref[k]) / max(np.linalg.norm(ref[k]), 1e-300))
                         for k in ref}
        out["rel_l2_error_vs_fp64_oracle"] = errs
        out["oracle_mg_iterations"] = info["iterations"]
        out["cpu_baseline"] = {"steps_per_s": 1.0 / cpu_s, "kind": "port", "cores": os.cpu_count(),
                               "sample": "one step of the same workload: the C++/OpenMP restatement (film2d.cpp, "
                                         "bit-identical to the numpy one away from the multigrid's reductions) on all "
                                         "host threads"}
    return out


def oracle_error(case, nlevels, p_gpu, mixed=False):
    """Relative L2 difference of a GPU solution from the FP64 oracle's solve of the same
    system to the same tolerance (the oracle's C++ multigrid-PCG with the GPU's cycle)."""
    from oracle import oracle
    p_ref, _, _, _, st = oracle.mg_solve(case.f, case.bx, case.by, case.hx, case.hy, nlevels=nlevels, ncoarse=1,
                                         sym=5, method="pcg", mixed=False, rtol=RTOL, max_cycles=200, native=True)
    return float(np.linalg.norm(p_gpu - p_ref) / np.linalg.norm(p_ref))


# ------------------------------------------------------------------ GPU leg
ALG_BYTES_PER_CELL = {  # FP64, level 0: each distinct array read or written once per cell
    "down0": 8 * (3 + 1 + 0.25),       # read f, bx, by; write u, f_coarse
    "up0": 8 * (5 + 0.25),             # read u, u_coarse(1/4), f, bx, by; write u
    "pupdate": 8 * 5,                  # read z, p, bx, by; write p
    "xupdate": 8 * 7,                  # read x, p, f, bx, by; write x, r
}


# DRAM bytes per level-0 launch from one ncu capture at 1024x1024 FP64
# (dram__bytes_read.sum + dram__bytes_write.sum; profiles/mg_k_down_k_up_level0_1024_fp64.md),
# scaled by cells for other sizes.
NCU_DRAM_BYTES_1024 = {"down0": 33.571840e6 + 0.037888e6, "up0": 44.064768e6 + 0.158976e6}


def run_ours(args):
    import torch
    import torch.distributed as dist

    from lica_boiling1d_b200 import native, poisson
    from lica_boiling1d_b200.inputs import bubble_poisson_case

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    n = args.n
    nlevels = NLEVELS + int(round(np.log2(n / N)))
    case = bubble_poisson_case(n)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    f, bx, by = t(case.f), t(case.bx), t(case.by)
    p = torch.zeros((n, n), dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    solver = poisson.MultigridPoisson(n, n, case.hx, case.hy, nlevels=nlevels, ncoarse=args.ncoarse,
                                      precision=args.precision, use_graph=not args.no_graph)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def slowest(x):
        if world == 1:
            return x
        v = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(v, op=dist.ReduceOp.MAX)
        return float(v.item())

    # warm-up (builds and caches the graph)
    for _ in range(args.warmup):
        p.zero_()
        solver.solve(p, f, bx, by, rtol=RTOL)
    torch.cuda.synchronize(dev)

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    props = torch.cuda.get_device_properties(dev)
    uuid = str(props.uuid).lower().replace("gpu-", "") if hasattr(props, "uuid") else None
    clocks = ClockSampler(uuid)
    clocks.start()
    time.sleep(0.4)
    barrier()
    torch.cuda.synchronize(dev)
    l0 = native.launch_count()
    its = []
    for k in range(args.steps):
        flush.fill_(k & 0xFF)            # > L2 between timed solves
        p.zero_()
        ev[k][0].record(stream)
        it, rel, st = solver.solve(p, f, bx, by, rtol=RTOL)
        ev[k][1].record(stream)
        its.append(it)
        if st != 0:
            raise RuntimeError(f"solve did not converge: status {st} rel {rel}")
    torch.cuda.synchronize(dev)
    barrier()
    launches = native.launch_count() - l0
    clk = clocks.stop()
    p_last = p.cpu().numpy()
    total_ms = sum(a.elapsed_time(b) for a, b in ev)
    total_ms = slowest(total_ms)
    value = world * args.steps / (total_ms / 1e3)

    e2e, roofline, variants, cpu = None, None, {}, None
    rk3 = None
    if not args.skip_rk3:
        rk3 = rk3_legs(dev, flush, steps_col=args.column_steps, steps_batch=args.batch_steps, rank=rank, world=world,
                       slowest=slowest, film_steps=args.film_steps,
                       film_compare=(rank == 0 and world == 1 and not args.skip_cpu))
        col_gpu_state, col_gpu_hist = rk3.pop("_column_gpu")
        if rank == 0 and world == 1 and not args.skip_cpu:
            rk3["cpu_baseline"], (col_ref, col_ref_hist) = rk3_cpu(args.column_steps)
            rk3["cpu_baseline"]["kind"] = "port"
            same = {k: bool(np.array_equal(col_gpu_state.arrays[k][0], v)) for k, v in col_ref.items()}
            rk3["column_512"]["vs_oracle"] = {
                "history_steps_compared": int(col_ref_hist.shape[0]),
                "history_bit_identical": bool(np.array_equal(col_gpu_hist, col_ref_hist)),
                "history_max_abs_diff": {name: float(np.abs(col_gpu_hist[:, q] - col_ref_hist[:, q]).max())
                                         for q, name in enumerate(("time", "place", "vapour_volume", "dt"))},
                "final_state_bit_identical": all(same.values()),
                "final_interface_place": float(col_ref_hist[-1, 1]),
                "final_vapour_volume": float(col_ref_hist[-1, 2]),
                "note": "interface history = the reference's 0interface.dat (TIME, place) and VOL_TOT_IPHS per step"}
    if args.no_e2e:
        return finish(args, locals())
    # end-to-end through the host C-ABI entry: H2D of p0, f, bx, by; solve; D2H of p
    hf = torch.from_numpy(case.f.copy()).pin_memory().numpy()
    hbx = torch.from_numpy(case.bx.copy()).pin_memory().numpy()
    hby = torch.from_numpy(case.by.copy()).pin_memory().numpy()
    hp = torch.zeros((n, n), dtype=torch.float64).pin_memory().numpy()
    for _ in range(2):
        hp[...] = 0.0
        solver.solve(hp, hf, hbx, hby, rtol=RTOL, stream=stream)
    ke = max(3, min(args.steps, 10))
    eve = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(ke)]
    barrier()
    torch.cuda.synchronize(dev)
    for k in range(ke):
        flush.fill_(k & 0xFF)
        hp[...] = 0.0
        eve[k][0].record(stream)
        solver.solve(hp, hf, hbx, hby, rtol=RTOL, stream=stream)
        eve[k][1].record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    single_ms = slowest(sum(a.elapsed_time(b) for a, b in eve))
    # a sequence of independent solves through lica_mg_solve_host_batch: each system's p0, f,
    # bx, by uploaded and its p downloaded, the transfers of neighbouring systems overlapping
    # each solve; host clock around the synchronous call (it returns after the last download)
    kb = max(4, min(args.steps, 16))
    hps = [torch.zeros((n, n), dtype=torch.float64).pin_memory().numpy() for _ in range(kb)]
    solver.solve_batch(hps[:2], [hf] * 2, [hbx] * 2, [hby] * 2, rtol=RTOL)
    for a in hps:
        a[...] = 0.0
    barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    bres = solver.solve_batch(hps, [hf] * kb, [hbx] * kb, [hby] * kb, rtol=RTOL)
    batch_ms = slowest((time.perf_counter() - t0) * 1e3)
    barrier()
    if any(r[2] != 0 for r in bres):
        raise RuntimeError(f"batch solve status {[r[2] for r in bres]}")
    e2e = {"value": world * kb / (batch_ms / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": int(hp.nbytes + hf.nbytes + hbx.nbytes + hby.nbytes),
           "d2h_bytes_per_step": int(hp.nbytes), "steps": kb,
           "path": "lica_mg_solve_host_batch (C ABI), pinned host arrays, uploads and downloads overlapping the "
                   "solves; host clock around the call",
           "single_call": {"value": world * ke / (single_ms / 1e3), "steps": ke,
                           "path": "lica_mg_solve_host, one solve per call, CUDA events"}}

    if args.no_profile:
        return finish(args, locals())
    # kernel-class timing: one profiled solve (separate launches bracketed by CUDA events)
    solver.profile(True)
    for _ in range(3):
        flush.fill_(1)
        p.zero_()
        solver.solve(p, f, bx, by, rtol=RTOL)
    prof = solver.profile_read()
    solver.profile(False)
    level0 = {k: prof[k] for k in ALG_BYTES_PER_CELL}
    dom = max(level0, key=lambda k: level0[k][0])
    ms, nl = level0[dom]
    avg_s = ms / 1e3 / max(nl, 1)
    alg = ALG_BYTES_PER_CELL[dom] * n * n
    peak, peak_kind = peaks()
    achieved = alg / avg_s / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": (NCU_DRAM_BYTES_1024[dom] * (n * n) / (1024 * 1024)
                            if dom in NCU_DRAM_BYTES_1024 and args.precision == "fp64" else None),
                "traffic_source": "ncu capture of the same kernel at 1024x1024 (cold cache), scaled by cells",
                "alg_bytes_per_launch": alg, "avg_launch_us": avg_s * 1e6,
                "kernel_classes_ms_per_solve": {k: v[0] / 3 for k, v in prof.items()},
                "note": "one profiled solve as separate launches after the timed region; working set is L2-resident"}

    # secondary: the mixed-precision preconditioner on the same workload
    if args.precision == "fp64" and not args.skip_variants:
        sm = poisson.MultigridPoisson(n, n, case.hx, case.hy, nlevels=nlevels, ncoarse=args.ncoarse,
                                      precision="mixed")
        for _ in range(3):
            p.zero_()
            sm.solve(p, f, bx, by, rtol=RTOL)
        evm = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(ke)]
        itm = []
        for k in range(ke):
            flush.fill_(k & 0xFF)
            p.zero_()
            evm[k][0].record(stream)
            itm.append(sm.solve(p, f, bx, by, rtol=RTOL)[0])
            evm[k][1].record(stream)
        torch.cuda.synchronize(dev)
        mms = sum(a.elapsed_time(b) for a, b in evm)
        err_mixed = oracle_error(case, nlevels, p.cpu().numpy()) if not args.skip_cpu else None
        variants["mixed"] = {"value": ke / (mms / 1e3), "unit": UNIT, "iterations": itm[-1],
                             "rel_l2_error_vs_fp64_oracle": err_mixed,
                             "note": "FP32 smoothing/restriction/prolongation, FP64 residual, CG and coarsest solve"}
        sm.close()
        if not args.skip_2048 and n == N:
            c2 = bubble_poisson_case(2 * N)
            f2, bx2, by2 = t(c2.f), t(c2.bx), t(c2.by)
            p2 = torch.zeros_like(f2)
            for prec in ("fp64", "mixed"):
                s2 = poisson.MultigridPoisson(2 * N, 2 * N, c2.hx, c2.hy, nlevels=nlevels + 1, ncoarse=args.ncoarse,
                                              precision=prec)
                for _ in range(3):
                    p2.zero_()
                    s2.solve(p2, f2, bx2, by2, rtol=RTOL)
                ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                       for _ in range(ke)]
                it2 = []
                for k in range(ke):
                    flush.fill_(k & 0xFF)
                    p2.zero_()
                    ev2[k][0].record(stream)
                    it2.append(s2.solve(p2, f2, bx2, by2, rtol=RTOL)[0])
                    ev2[k][1].record(stream)
                torch.cuda.synchronize(dev)
                ms2 = sum(a.elapsed_time(b) for a, b in ev2)
                err2 = oracle_error(c2, nlevels + 1, p2.cpu().numpy()) if not args.skip_cpu else None
                variants[f"{prec}_2048"] = {"value": ke / (ms2 / 1e3), "unit": UNIT, "iterations": it2[-1],
                                            "rel_l2_error_vs_fp64_oracle": err2,
                                            "note": "the same 64 bubbles in the unit domain at 2048x2048 (radii "
                                                    "16-96 cells), 7 levels"}
                s2.close()
            del f2, bx2, by2, p2
        if not args.skip_learned:
            lg = learned_leg(args, dev, case, n, nlevels, f, bx, by, p, flush, stream, ke)
            if "unavailable" in lg:
                variants["learned"] = lg
            else:
                its0 = its[-1]
                variants["learned"] = {
                    "value": lg["fp64"]["value"], "unit": UNIT, "iterations": lg["fp64"]["iterations"],
                    "vcycles_saved": its0 - lg["fp64"]["iterations"], "guess": lg["guess"],
                    "note": "FP64 MG-PCG from the U-Net guess (guess + check + solve per step)"}
                variants["mixed_learned"] = {
                    "value": lg["mixed"]["value"], "unit": UNIT, "iterations": lg["mixed"]["iterations"],
                    "vcycles_saved": itm[-1] - lg["mixed"]["iterations"],
                    "note": "mixed-precision MG-PCG from the U-Net guess (guess + check + solve per step)"}

    bubbles_leg = None
    if rank == 0 and not args.skip_bubbles:
        bubbles_leg = bubble_leg(dev, flush, compare=(world == 1 and not args.skip_cpu))
    err_headline = oracle_error(case, nlevels, p_last) if (rank == 0 and not args.skip_cpu) else None
    if rank == 0 and world == 1 and not args.skip_cpu and n == N:
        threads = os.cpu_count()
        times, cits = cpu_solves(case, 15.0, 30)
        cpu = {"value": len(times) / sum(times), "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{len(times)} complete solves of the same workload (~15 s), FP64 C++/OpenMP restatement"}

    return finish(args, locals())


UNET_LAYERS = [(16, 0, 32, 0), (32, 0, 32, 0), (32, 0, 64, 1), (64, 0, 64, 1), (64, 0, 128, 2), (128, 0, 128, 2),
               (128, 64, 64, 1), (64, 0, 64, 1), (64, 32, 32, 0), (32, 0, 32, 0)]


def unet_flops(n):
    """Tensor-core FLOPs of one U-Net guess at n x n (the executed 3x3 MMAs, layer 0's 16
    padded input channels included) plus the 1x1 head."""
    tot = sum(2.0 * (n >> lv) ** 2 * 9 * (c0 + c1) * co for c0, c1, co, lv in UNET_LAYERS)
    return tot + 2.0 * n * n * 32


def learned_leg(args, dev, case, n, nlevels, f, bx, by, p, flush, stream, reps):
    """The learned initial guess (shipped weights, trained by the project's own kernels)
    feeding the FP64 and the mixed-precision MG-PCG to the same tolerance; each timed step
    is guess + residual check (zero fallback) + solve."""
    import torch

    from lica_boiling1d_b200 import poisson, train_guess
    from lica_boiling1d_b200.unet import LearnedGuess
    if not os.path.exists(train_guess.SOLVER_PAIR_WEIGHTS):
        return {"unavailable": "no trained weights in the package"}
    net = LearnedGuess(1, n, n)
    train_guess.load(net, train_guess.SOLVER_PAIR_WEIGHTS)
    rho = torch.from_numpy(case.rho[None].copy()).to(dev)
    F, BX, BY = f[None], bx[None], by[None]
    x0 = torch.empty_like(F)
    out = {}
    # the guess alone
    for _ in range(3):
        net.guess(rho, F, case.hx * case.hy, out=x0)
    evg = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for k in range(reps):
        flush.fill_(k & 0xFF)
        evg[k][0].record(stream)
        net.guess(rho, F, case.hx * case.hy, out=x0)
        evg[k][1].record(stream)
    torch.cuda.synchronize(dev)
    gms = sum(a.elapsed_time(b) for a, b in evg) / reps
    fl = unet_flops(n)
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peak = float(json.load(fh)["bf16_tflops"])
        peak_src = "measured (cuBLAS bf16 burst)"
    except Exception:
        peak, peak_src = 1590.0, "fallback"
    ach = fl / (gms / 1e3) / 1e12
    out["guess"] = {"ms": gms, "gflop": fl / 1e9,
                    "roofline": {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                                 "frac": ach / peak, "peak_source": peak_src},
                    "note": "10 tcgen05 convolutions (BF16, FP32 accumulate) + pooling/upsampling/head"}
    _, rel0 = net.guess_checked(rho, F, BX, BY, case.hx, case.hy, out=x0)
    out["guess"]["rel_residual"] = float(rel0[0])
    out["guess"]["weights"] = "20,000 pairs from 1024^2 bubble-Poisson and 512 x 1536 film solves (unet_guess_solver_pairs.npy)"
    if os.path.exists(train_guess.WEIGHTS):
        # the same network trained on 16,000 256^2 bubble problems only, for comparison
        alt = LearnedGuess(1, n, n)
        train_guess.load(alt, train_guess.WEIGHTS)
        _, rel_alt = alt.guess_checked(rho, F, BX, BY, case.hx, case.hy, out=x0)
        alt.close()
        out["guess"]["rel_residual_bubble_only_weights"] = float(rel_alt[0])
    for prec in ("fp64", "mixed"):
        s = poisson.MultigridPoisson(n, n, case.hx, case.hy, nlevels=nlevels, ncoarse=args.ncoarse, precision=prec)
        for _ in range(3):
            net.guess_checked(rho, F, BX, BY, case.hx, case.hy, out=x0)
            p.copy_(x0[0])
            s.solve(p, f, bx, by, rtol=RTOL)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        its = []
        for k in range(reps):
            flush.fill_(k & 0xFF)
            evs[k][0].record(stream)
            net.guess_checked(rho, F, BX, BY, case.hx, case.hy, out=x0)
            p.copy_(x0[0])
            it, rel, st = s.solve(p, f, bx, by, rtol=RTOL)
            evs[k][1].record(stream)
            its.append(it)
            if st != 0:
                raise RuntimeError(f"solve from the learned guess: status {st}")
        torch.cuda.synchronize(dev)
        ms = sum(a.elapsed_time(b) for a, b in evs)
        out[prec] = {"value": reps / (ms / 1e3), "unit": UNIT, "iterations": its[-1], "rel_residual": rel}
        s.close()
    net.close()
    return out


def profile_guess(reps):
    """A few U-Net guesses on the 1024 x 1024 workload (for ncu captures of the tensor-core
    convolutions); prints the mean guess time."""
    import torch

    from lica_boiling1d_b200 import train_guess
    from lica_boiling1d_b200.inputs import bubble_poisson_case
    from lica_boiling1d_b200.unet import LearnedGuess
    case = bubble_poisson_case(N)
    net = LearnedGuess(1, N, N)
    if os.path.exists(train_guess.WEIGHTS):
        train_guess.load(net)
    rho = torch.from_numpy(case.rho[None].copy()).cuda()
    f = torch.from_numpy(case.f[None].copy()).cuda()
    x0 = torch.empty_like(f)
    net.guess(rho, f, case.hx * case.hy, out=x0)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        net.guess(rho, f, case.hx * case.hy, out=x0)
    b.record()
    torch.cuda.synchronize()
    print(f"U-Net guess {N}x{N}: {a.elapsed_time(b) / reps:.3f} ms over {reps} guesses "
          f"({unet_flops(N) / 1e9:.1f} GFLOP each)")
    net.close()


def profile_film(steps):
    """A few 2-D film-boiling steps on 512 x 1536 (for ncu launch lists of the step's kernels);
    prints the mean step time."""
    import torch

    from lica_boiling1d_b200 import film2d as G
    P = G.default_props()
    nx, ny = FILM["nx"], FILM["ny"]
    st0 = G.initial_state(nx, ny, FILM["y0"], FILM["amp"], props=P)
    dt = G.stable_dt(nx, P)
    gpu = G.Film2D(nx, ny, P)
    state = G.to_device(st0)
    gpu.step(state, dt)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        gpu.step(state, dt)
    b.record()
    torch.cuda.synchronize()
    print(f"2-D film step {nx}x{ny}: {a.elapsed_time(b) / steps:.3f} ms over {steps} steps")
    gpu.close()


def profile_bubbles(calls):
    """A few bubble-statistics launches on the 256^3, four-level-set workload (for ncu);
    prints the mean launch time."""
    import torch

    from lica_boiling1d_b200 import bubbles
    dev = torch.device("cuda:0")
    grid, psi, (u, v, w) = bubble_fields(dev, BUB["n"], BUB["nlvs"])
    tr = bubbles.BubbleTracker(grid, BUB["nlvs"])
    raw = tr.track(psi, u, v, w)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(calls):
        raw = tr.track(psi, u, v, w, out=raw)
    b.record()
    torch.cuda.synchronize()
    print(f"bubble statistics {BUB['n']}^3 x {BUB['nlvs']}: {a.elapsed_time(b) / calls:.4f} ms over {calls} calls")
    tr.close()


def finish(args, v):
    import torch.distributed as dist
    if v["rank"] == 0:
        n = v["n"]
        line = {
            "metric": METRIC, "value": v["value"], "unit": UNIT, "n_gpus": v["world"], "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v["total_ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64+f32",
            "data": "synthetic",
            "config": bench_config(n, v["nlevels"], args.ncoarse, args.precision, v["world"]),
            "iterations": v["its"][-1], "rel_residual": v["rel"],
            "rel_l2_error_vs_fp64_oracle": v.get("err_headline"),
            "roofline": v["roofline"], "cpu_baseline": v["cpu"], "e2e": v["e2e"], "gpu_launches": int(v["launches"]),
            "clocks": v["clk"], "variants": v["variants"], "rk3": v.get("rk3"),
            "bubble_tracking": v.get("bubbles_leg"),
        }
        print(json.dumps(line), flush=True)
    v["solver"].close()
    if v["world"] > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-variants", action="store_true")
    ap.add_argument("--n", type=int, default=N, help="grid size (default: the 1024x1024 workload)")
    ap.add_argument("--ncoarse", type=int, default=1, help="inner V-cycles of the coarsest-level solve")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end and later legs (profiling runs)")
    ap.add_argument("--no-profile", action="store_true", help="skip the kernel-class timing and later legs")
    ap.add_argument("--skip-rk3", action="store_true", help="skip the RK3 column legs")
    ap.add_argument("--skip-learned", action="store_true", help="skip the learned-guess legs")
    ap.add_argument("--skip-2048", action="store_true", help="skip the 2048x2048 solves")
    ap.add_argument("--skip-bubbles", action="store_true", help="skip the 3-D bubble-statistics leg")
    ap.add_argument("--profile-guess", type=int, default=0,
                    help="only run this many U-Net guesses at 1024x1024 (profiling) and exit")
    ap.add_argument("--column-steps", type=int, default=COLUMN512["steps"], help="timed steps of the 512-cell column")
    ap.add_argument("--batch-steps", type=int, default=1000, help="timed steps of the 4096-column batch")
    ap.add_argument("--film-steps", type=int, default=10, help="timed steps of the 2-D film (0: skip the leg)")
    ap.add_argument("--profile-film", type=int, default=0, help="run N 2-D film steps only (ncu launch lists)")
    ap.add_argument("--profile-bubbles", type=int, default=0,
                    help="run N bubble-statistics launches only (256^3, four level sets; for ncu)")
    ap.add_argument("--profile-batch", type=int, default=0,
                    help="only run NCOL columns of the uneven batch (profiling runs); see --batch-steps, --threads")
    ap.add_argument("--threads", type=int, default=64, help="column CTA width for --profile-batch")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch kernels one by one instead of one CUDA graph per solve (for ncu, which cannot "
                         "profile kernels of a graph with a conditional node)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.profile_batch:
        profile_batch(args.profile_batch, args.batch_steps, args.threads)
        return
    if args.profile_guess:
        profile_guess(args.profile_guess)
        return
    if args.profile_bubbles:
        profile_bubbles(args.profile_bubbles)
        return
    if args.profile_film:
        profile_film(args.profile_film)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
