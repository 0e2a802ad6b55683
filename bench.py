#!/usr/bin/env python
"""Benchmark: implicit time steps per second of the wall-cilia simulation.

Workload (one array per GPU): 256 prescribed Fulford-Blake cilia x 20
segments (5120 segments) on a 16 x 16 wall lattice of spacing 20a, segment
spacing 2.6a, phases U(0, 2 pi) from a seed, angles N(0, 0.05), dt = T/300,
dynamic phase and shape-rotation rates with the reference's own
generalised-force tables, FP32 pair mobility, FP64 GMRES to a relative
residual of 1e-6.  A step is one implicit time step (kinematics, patch
preconditioner refresh, RHS, GMRES, state update).  The headline runs the
line-patch block-Jacobi preconditioner (16-filament lattice lines along the
beat direction, inverted on the device every step); the same state is also
stepped with the reference's block-diagonal preconditioner ("plain GMRES"),
which stops at its 350-iteration cap on this workload.  Every rank runs its
own array (replicas: the path does not shard a single array), so `value` is
the sum over ranks (weak scaling).

On one GPU the line also carries the batched workload: 64 independent arrays
with U{16..256} cilia each (phases N(0, 0.05)), stepped together in one graph
launch per step, against the same 64 arrays stepped as separate simulations.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`--impl reference` times the reference's own step code on the host cores
(its mobility_solver/filament/swimmer sources compiled unmodified for the host
in FP64 by oracle/ref_build.py: host GMRES with its block-diagonal
preconditioner, beat and time stepping, with an OpenMP RPY sum for the
mobility products since the reference has no CPU mobility of its own) on a
bounded sample of the same workload: whole implicit steps of the same
5120-segment array, as many as fit a fixed time budget.  Its line also
carries the reference's own CUDA code timed on the same GPU (Mss_mult, its
whole GPU step, its cuFCM apply) as context.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

NX = 16            # 16 x 16 = 256 cilia
NSEG = 20
SEG_SEP = 2.6
SPACING = 20.0
GMRES_TOL = 1e-6
TRAJECTORY_BLOCK = 10  # timed steps run in blocks of this many from the seeded initial state, each restarted
F_PAIR = 154       # algorithmic flops of one 3x3 wall RPY pair (cuda_functions.cu:63-150)
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # nominal SIMT FP32 peak at max SM clock
# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum, one ncu capture each):
PAIR_KERNEL_DRAM_BYTES = 182_500            # rpy_wall_sym_batch_kernel, 5120 segments
REFRESH_UPDATE_DRAM_BYTES = 37_500_000      # gj_update_kernel, 16 patches of 992
L2_FLUSH_BYTES = 256 << 20


def workload_inputs(s_table_from="engine"):
    from cufcm_fil_b200 import workloads
    data = np.load(ROOT / "cufcm_fil_b200" / "data" / "fulford_blake_nseg20_sep2.6.npz")
    F = NX * NX
    bases = workloads.lattice_bases(F, NX, SPACING, 0.5 * SEG_SEP)
    rng = np.random.default_rng(2024)
    phase0 = rng.uniform(0.0, 2.0 * math.pi, F)
    angle0 = rng.normal(0.0, 0.05, F)
    # The arclength table over one period is what the reference's WRITE_GENERALISED_FORCES pre-run writes;
    # the engine regenerates it on the device by the same bisection, the reference arm on the host.
    if s_table_from == "engine":
        from cufcm_fil_b200.sim import arclength_table
        s_table = arclength_table(nseg=NSEG, seg_sep=SEG_SEP, steps=300)
    else:  # the reference's own pre-run (its s-value table, written with six significant digits)
        from oracle import ref_step
        _, _, s_table = ref_step.wgf_tables(NSEG, SEG_SEP)
    return dict(bases=bases, nseg=NSEG, seg_sep=SEG_SEP, dt=1.0 / 300, phase0=phase0, angle0=angle0,
                spring_factor=0.01, phase_refs=data["phase"], angle_refs=data["angle"], s_table=s_table)


def config_dict(extra=None):
    c = {"workload": "implicit wall-cilia simulation: 256 cilia x 20 segments, 16x16 lattice spacing 20a, "
                     "Fulford-Blake beat, dt=T/300, GMRES tol 1e-6",
         "preconditioner": "line-patch block-Jacobi (lattice lines of 16 cilia along the beat direction, FP32 "
                           "inverses rebuilt every step); not learned",
         "plain": "block-diagonal preconditioner of the reference (apply_preconditioner_new)",
         "n_cilia": NX * NX, "segments_per_cilium": NSEG, "segments": NX * NX * NSEG, "lattice_spacing": SPACING,
         "segment_spacing": SEG_SEP, "gmres_tol": GMRES_TOL, "l2": "flushed between timed steps (256 MiB write)",
         "trajectory": f"timed steps in blocks of {TRAJECTORY_BLOCK} consecutive steps 0.. from the seeded initial "
                       "state, each block restarted from it outside the timed region (chaotic dynamics)"}
    if extra:
        c.update(extra)
    return c


# --------------------------------------------------------------------- clocks
class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- distributed
def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch
        import torch.distributed as dist
        dist.barrier()
        torch.cuda.synchronize()


def _reduce(world, value, op):
    if world == 1:
        return float(value)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(world, value):
    """Timing of a multi-rank run: the slowest rank's device time."""
    import torch.distributed as dist
    return _reduce(world, value, dist.ReduceOp.MAX if world > 1 else None)


def sum_over_ranks(world, value):
    """Whole-job work: every rank runs its own replica."""
    import torch.distributed as dist
    return _reduce(world, value, dist.ReduceOp.SUM if world > 1 else None)


def replica_throughput(world, steps_per_rank, rank_ms):
    """value = (steps of all ranks) / (slowest rank's time), the weak-scaling aggregate."""
    total_steps = sum_over_ranks(world, steps_per_rank)
    slowest_ms = max_over_ranks(world, rank_ms)
    return total_steps / (slowest_ms / 1e3), slowest_ms


# ----------------------------------------------------------------------- ours
def _events(n):
    import torch
    return [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]


def time_steps(sim, stream, flush, nt, steps, clocks=None, restart=None, block=0):
    """Device time of `steps` graph-launched steps, L2 flushed before each (outside the events).  With `restart`
    (a checkpoint of the state at step nt), the steps run in blocks of `block` steps nt, nt+1, ..., each block
    restarted from the checkpoint (outside the events)."""
    import torch
    ev = _events(steps)
    torch.cuda.synchronize()
    for k in range(steps):
        q = k % block if restart is not None else k
        if restart is not None and k > 0 and q == 0:
            sim.restore(restart)
        with torch.cuda.stream(stream):
            flush.zero_()
            ev[k][0].record(stream)
        sim.step_async(nt + q)
        with torch.cuda.stream(stream):
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev)


def time_refresh(sim, stream, flush, reps=5):
    """Device time of one rebuild of the patch inverses (assembly + Gauss-Jordan), mean of `reps`."""
    import torch
    ev = _events(reps)
    for _ in range(2):
        sim.refresh_preconditioner()
    torch.cuda.synchronize()
    for k in range(reps):
        with torch.cuda.stream(stream):
            flush.zero_()
            ev[k][0].record(stream)
        sim.refresh_preconditioner()
        with torch.cuda.stream(stream):
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev) / reps


def run_batched(local, inp, world=1, rank=0):
    """64 independent arrays with U{16..256} cilia: one batch vs 64 single-array simulations.  With several ranks
    the arrays are binned by cost (cufcm_fil_b200.shard) and every rank steps its own bin as one batch: no
    collective on the data path, the slowest rank's step time for the whole job."""
    import torch
    from cufcm_fil_b200 import shard, workloads
    from cufcm_fil_b200.sim import WallCiliaBatch, WallCiliaSimulation
    B, W, K = 64, 3, 5
    rng = np.random.default_rng(4)
    counts = rng.integers(16, 257, B)
    all_specs = []
    for n in counts:
        nx = int(math.ceil(math.sqrt(n)))
        all_specs.append(dict(bases=workloads.lattice_bases(int(n), nx, SPACING, 0.5 * SEG_SEP),
                              phase0=rng.normal(0.0, 0.05, n), angle0=rng.normal(0.0, 0.05, n)))
    shared = dict(nseg=NSEG, seg_sep=SEG_SEP, dt=inp["dt"], spring_factor=inp["spring_factor"],
                  phase_refs=inp["phase_refs"], angle_refs=inp["angle_refs"], s_table=inp["s_table"],
                  gmres_tol=GMRES_TOL, device=local)
    costs = [shard.array_cost(int(n), NSEG) for n in counts]
    bins = shard.bin_by_cost(costs, world)
    if world > 1:
        return run_batched_sharded(all_specs, shared, bins, costs, world, rank, W, K)
    specs = all_specs
    with WallCiliaBatch(specs, **shared) as bt:
        for nt in range(W):
            bt.step(nt)
        tuning = bt.autotune()
        stream = torch.cuda.ExternalStream(bt.stream_handle())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        for nt in range(W, W + K):
            bt.step_async(nt)
        b.record(stream)
        b.synchronize()
        batch_ms = a.elapsed_time(b) / K
        it, _, _, rc = bt.last_solve()
        loop_iters = [int(bt.iteration_log(q, W + K)[W:W + K].max()) for q in range(B)]
        launches = int(bt.launches_per_step(max(loop_iters)))
    sims = [WallCiliaSimulation(**shared, **sp) for sp in specs]
    for s_ in sims:
        for nt in range(W):
            s_.step(nt)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for nt in range(W, W + K):
        for s_ in sims:
            s_.step_async(nt)
    torch.cuda.synchronize()
    for s_ in sims:
        s_.last_solve()
    conc_ms = (time.perf_counter() - t0) * 1e3 / K
    t0 = time.perf_counter()
    for nt in range(W + K, W + 2 * K):
        for s_ in sims:
            s_.step(nt)
    seq_ms = (time.perf_counter() - t0) * 1e3 / K
    for s_ in sims:
        s_.close()
    return {"workload": f"{B} wall arrays, U{{16..256}} cilia x {NSEG} segments ({int(counts.sum())} cilia, "
                        f"{int(((counts * NSEG) ** 2).sum())} pairs per batched matvec), phases N(0,0.05), "
                        "block-diagonal preconditioner, one graph launch per step",
            "array_timesteps_per_s": B / (batch_ms / 1e3), "ms_per_step": batch_ms,
            "gmres_iters_max_per_step": max(loop_iters), "gpu_launches_per_step": launches, "tuning": tuning,
            "vs_separate_concurrent": conc_ms / batch_ms, "separate_concurrent_ms_per_step": conc_ms,
            "vs_separate_sequential": seq_ms / batch_ms, "separate_sequential_ms_per_step": seq_ms,
            "timing": "batch: CUDA events on its stream; separate runs: host wall clock around 64 graph launches "
                      "per step on 64 streams (concurrent) or with a wait after each (sequential)"}


def run_batched_sharded(all_specs, shared, bins, costs, world, rank, W, K):
    """The batched workload over `world` ranks: rank r steps the arrays of bins[r] as one batch."""
    import torch
    from cufcm_fil_b200 import shard
    from cufcm_fil_b200.sim import WallCiliaBatch
    mine = bins[rank]
    with WallCiliaBatch([all_specs[i] for i in mine], **shared) as bt:
        for nt in range(W):
            bt.step(nt)
        stream = torch.cuda.ExternalStream(bt.stream_handle())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(world)
        a.record(stream)
        for nt in range(W, W + K):
            bt.step_async(nt)
        b.record(stream)
        b.synchronize()
        local_ms = a.elapsed_time(b) / K
        bt.last_solve()
        iters = {i: int(bt.iteration_log(q, W + K)[W:W + K].max()) for q, i in enumerate(mine)}
    slowest = max_over_ranks(world, local_ms)
    per_rank = shard.gather_to_root({"rank": rank, "arrays": len(mine), "ms_per_step": local_ms, "iters": iters},
                                    world)
    if rank != 0:
        return None
    B = len(all_specs)
    return {"workload": f"{B} wall arrays, U{{16..256}} cilia x {NSEG} segments, binned by cost over {world} ranks "
                        "(no collective on the data path), block-diagonal preconditioner, one graph launch per "
                        "step per rank",
            "array_timesteps_per_s": B / (slowest / 1e3), "ms_per_step": slowest, "scaling": "strong",
            "bin_imbalance": shard.imbalance(costs, bins), "ranks": per_rank,
            "timing": "CUDA events on each rank's batch stream; the job's step time is the slowest rank's"}


def _last_solve(sim):
    """(converged, error text) of the last solve; a non-finite solve (the colliding cilia of the 20a lattices can
    reach one) is reported, not raised, so that one leg does not end the benchmark."""
    from cufcm_fil_b200 import _lib
    try:
        return bool(sim.last_solve().status == _lib.CF_OK), None
    except _lib.CufilError as exc:
        return False, str(exc)


def run_large(local, inp, flush, steps=4):
    """1024 cilia (32 x 32 lattice, 20 480 segments): whole-line patches against the block-diagonal preconditioner."""
    import torch
    from cufcm_fil_b200 import _lib
    from cufcm_fil_b200.sim import lattice_simulation
    out = {"workload": "1024 cilia x 20 segments, 32x32 lattice spacing 20a, phases U(0,2pi), GMRES tol 1e-6"}
    for name, code in (("line_patches", _lib.CF_PRECOND_LINE), ("block_diagonal", _lib.CF_PRECOND_BLOCK_DIAG)):
        sim = lattice_simulation(32, spacing=SPACING, nseg=NSEG, seg_sep=SEG_SEP, s_table=inp["s_table"],
                                 gmres_tol=GMRES_TOL, device=local, precond=code)
        stream = torch.cuda.ExternalStream(sim.stream_handle())
        sim.step(0)
        ms = time_steps(sim, stream, flush, 1, steps)
        converged, err = _last_solve(sim)
        its = sim.iteration_log(1 + steps)[1:1 + steps]
        out[name] = {"timesteps_per_s": steps / (ms / 1e3), "ms_per_step": ms / steps,
                     "gmres_iters_per_step": float(np.mean(its)), "converged": converged}
        if err:
            out[name]["error"] = err
        sim.close()
    out["speedup"] = out["line_patches"]["timesteps_per_s"] / out["block_diagonal"]["timesteps_per_s"]
    out["learned"] = run_learned_large(local, inp, flush, steps)
    if out["learned"].get("timesteps_per_s"):
        out["learned_vs_plain"] = out["learned"]["timesteps_per_s"] / out["block_diagonal"]["timesteps_per_s"]
        out["learned_vs_line_patches"] = out["learned"]["timesteps_per_s"] / out["line_patches"]["timesteps_per_s"]
    return out


def run_learned_large(local, inp, flush, steps, seeds=(7, 8, 9), max_pairs=40):
    """The learned preconditioner at the 32 x 32 size: a per-filament network trained by the library's own kernels
    on ~1e5 (features, target) pairs that line-patch runs of three other seeded states produce, applied on top of
    the line patches in flexible GMRES (CF_PRECOND_LEARNED_LINE) on the benchmark state; the correction weight
    is chosen on that first step among 1, 0.5, 0.25, 0 (0: the network switched off)."""
    import torch
    from cufcm_fil_b200 import _lib, learned
    from cufcm_fil_b200.mlp import FilamentMLP
    from cufcm_fil_b200.sim import lattice_simulation

    def make(seed, precond):
        return lattice_simulation(32, spacing=SPACING, nseg=NSEG, seg_sep=SEG_SEP, s_table=inp["s_table"],
                                  gmres_tol=GMRES_TOL, device=local, precond=precond, seed=seed)

    t0 = time.perf_counter()
    x, t = learned.collect(make, seeds=seeds, max_pairs=max_pairs, base=_lib.CF_PRECOND_LINE)
    collect_s = time.perf_counter() - t0
    n_pairs = int(x.shape[0])
    net = FilamentMLP(x.shape[1], 256, t.shape[1], max_batch=4096, seed=0, device=local)
    t0 = time.perf_counter()
    losses = learned.train(net, x, t, steps=1500, batch=2048, lr=3e-4, report_every=500)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    del x, t
    by_weight = {}
    for w in (1.0, 0.5, 0.25, 0.0):
        with make(2024, _lib.CF_PRECOND_LEARNED_LINE) as sim:
            sim.set_network(net)
            sim.set_network_weight(w)
            try:
                r = sim.step(0)
                by_weight[w] = (r.iterations, r.status)
            except _lib.CufilError:
                by_weight[w] = (None, _lib.CF_NONFINITE)
    ok = [w for w in by_weight if by_weight[w][1] == _lib.CF_OK]
    best = min(ok, key=lambda w: (by_weight[w][0], -w)) if ok else 0.0
    out = {"pairs": n_pairs, "collect_s": collect_s, "train_s": train_s, "losses": losses, "weight": best,
           "first_step_iterations_by_weight": {str(k): v[0] for k, v in by_weight.items()},
           "network": f"{net.n_in} -> 256 -> 256 -> {net.n_out}, BF16 tensor-core GEMMs, FP32 accumulation"}
    with make(2024, _lib.CF_PRECOND_LEARNED_LINE) as sim:
        sim.set_network(net)
        sim.set_network_weight(best)
        stream = torch.cuda.ExternalStream(sim.stream_handle())
        sim.step(0)
        ms = time_steps(sim, stream, flush, 1, steps)
        converged, err = _last_solve(sim)
        its = sim.iteration_log(1 + steps)[1:1 + steps]
        out.update({"timesteps_per_s": steps / (ms / 1e3), "ms_per_step": ms / steps,
                    "gmres_iters_per_step": float(np.mean(its)), "converged": converged})
        if err:
            out["error"] = err
    net.close()
    return out


def run_fcm(local, flush, reps=5):
    """Fast FCM at the sphere-with-cilia size: 1000 cilia x 20 segments + 10 000 body blobs, 512^3 grid, box 1024a,
    alpha 1, beta 10, eta 6; CUDA events around whole applies and per stage; spread and gather against HBM."""
    import torch
    from cufcm_fil_b200 import workloads
    from cufcm_fil_b200.fcm import FcmSolver
    segs, blobs = workloads.sphere_with_cilia()
    Y = np.concatenate([segs, blobs])
    n = Y.shape[0]
    F = np.random.default_rng(11).standard_normal((n, 3))
    kw = dict(rh=1.0, alpha=1.0, beta=10.0, eta=6.0, nx=512, ny=512, nz=512, boxsize=1024.0)
    dev = torch.device("cuda", local)
    with FcmSolver(n, device=local, **kw) as s:
        yd = torch.as_tensor(Y.astype(np.float32).ravel(), device=dev)
        fd = torch.as_tensor(F.astype(np.float32).ravel(), device=dev)
        vd = torch.empty(3 * n, device=dev)
        st = torch.cuda.Stream(device=dev)
        for _ in range(2):
            s.apply_device(yd, fd, vd, stream=st)
        ev = _events(reps)
        st.synchronize()
        for k in range(reps):
            with torch.cuda.stream(st):
                flush.zero_()
                ev[k][0].record(st)
            s.apply_device(yd, fd, vd, stream=st)
            with torch.cuda.stream(st):
                ev[k][1].record(st)
        st.synchronize()
        apply_ms = sum(a.elapsed_time(b) for a, b in ev) / reps
        info = s.info()
        s.set_timing(True)  # per-stage events: a separate pass, outside the whole-apply timing
        stages = {k: 0.0 for k in FcmSolver.STAGES}
        for _ in range(reps):
            s.apply_device(yd, fd, vd, stream=st)
            st.synchronize()
            for k, v in s.stage_times().items():
                stages[k] += v / reps
        s.set_timing(False)
    ngd = int(info["ngd"])
    grid = 512 ** 3
    spread_bytes = n * ngd ** 3 * 3 * 8   # atomic read-modify-write per support point and component
    gather_bytes = n * ngd ** 3 * 3 * 4
    hbm = measured_hbm_gbs()
    out = {"workload": f"{n} particles (20 000 segments + 10 000 body blobs on a sphere of radius 100a), box 1024a, "
                       f"512^3 FP32 grid, ngd {ngd}, Gaussian width a/sqrt(pi)",
           "apply_ms": apply_ms, "stages_ms": stages, "hbm_peak_gbs": hbm,
           "note": "algorithmic bytes: spread N ngd^3 3 x 8 B, gather N ngd^3 3 x 4 B; CUDA events per stage"}
    if stages.get("spread"):
        out["spread_gbs"] = spread_bytes / (stages["spread"] * 1e-3) / 1e9
        out["spread_frac"] = out["spread_gbs"] / hbm
    if stages.get("gather"):
        out["gather_gbs"] = gather_bytes / (stages["gather"] * 1e-3) / 1e9
        out["gather_frac"] = out["gather_gbs"] / hbm
    return out


def run_swimmer(steps=20):
    """The free swimmer (cf_swim): 256 Fulford-Blake cilia x 20 segments on a sphere of diameter 6 filament
    lengths (radius 148a) represented by 2562 blobs, 7942 particles; steps from the seeded state.  The step is
    host-driven (one synchronisation per GMRES iteration): host wall clock around synchronous steps."""
    import time
    from cufcm_fil_b200 import swim
    gold = np.load(ROOT / "tests" / "golden" / "reference_forcing_nseg20_sep2.6.npz")
    tips = np.load(ROOT / "tests" / "golden" / "ref_tips_16x16_80a.npz")
    F, B = 256, 2562
    geo = swim.sphere_geometry(swim.fibonacci_normals(F), swim.fibonacci_normals(B, 0.3), ar=6.0)
    rng = np.random.default_rng(12)
    with swim.CiliatedSwimmer(geometry=geo, phase0=rng.uniform(0, 2 * np.pi, F), angle0=rng.normal(0, 0.05, F),
                              phase_refs=gold["fb_phase"], angle_refs=gold["fb_angle"],
                              s_table=tips["s_table"]) as s:
        s.step(0)
        t0 = time.perf_counter()
        its = [s.step(nt).iterations for nt in range(1, 1 + steps)]
        dt = time.perf_counter() - t0
        bv = s.state()["body_v"]
    return {"workload": f"free sphere (radius {geo.radius:.0f}a, {B} blobs) with {F} cilia x 20 segments, "
                        f"{F * 20 + B} particles, GMRES tol 1e-6, the reference's body preconditioner",
            "timesteps_per_s": steps / dt, "ms_per_step": 1e3 * dt / steps,
            "gmres_iters_per_step": float(np.mean(its)), "body_speed": float(np.linalg.norm(bv[:3])),
            "timing": "host wall clock around synchronous steps (steps 1..20)"}


def run_elastic_sim(steps=30):
    """Elastic instability cilia (cf_elastic): 256 filaments x 20 segments on a 16 x 16 wall lattice at 80a,
    Broyden's method at the reference's settings; host wall clock around synchronous steps after step 0."""
    import time
    from cufcm_fil_b200 import workloads
    from cufcm_fil_b200.elastic import ElasticCiliaSimulation
    bases = workloads.lattice_bases(256, 16, 80.0, 1.3)
    with ElasticCiliaSimulation(bases=bases) as sim:
        sim.step(0)
        t0 = time.perf_counter()
        its = [sim.step(nt) for nt in range(1, 1 + steps)]
        dt = time.perf_counter() - t0
    return {"workload": "256 elastic cilia x 20 segments (instability-driven, DIMENSIONLESS_FORCE 220), 16x16 "
                        "wall lattice at 80a, dt = 36.3833/300, Broyden tol 1e-4",
            "timesteps_per_s": steps / dt, "ms_per_step": 1e3 * dt / steps,
            "broyden_iters_per_step": float(np.mean(its)),
            "timing": "host wall clock around synchronous steps (steps 1..30)"}


def measured_bf16_tflops():
    try:
        return float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["bf16_tflops"])
    except (OSError, KeyError, ValueError):
        return 1590.0  # fallback dense BF16 rate of this GPU pool


def measured_hbm_gbs():
    try:
        return float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0  # fallback copy bandwidth of this GPU pool


def run_ours(args):
    import torch
    from cufcm_fil_b200 import RpyMobilitySolver, _lib
    from cufcm_fil_b200.sim import WallCiliaSimulation, lattice_simulation

    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    inp = workload_inputs()
    sim = lattice_simulation(NX, spacing=SPACING, nseg=NSEG, seg_sep=SEG_SEP, s_table=inp["s_table"],
                             gmres_tol=GMRES_TOL, device=local, precond=_lib.CF_PRECOND_LINE, line_patch=NX)
    stream = torch.cuda.ExternalStream(sim.stream_handle(), device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    initial = sim.checkpoint()  # the seeded initial state: every timed block starts here
    nt = 0
    for _ in range(args.warmup):
        sim.step_async(nt)
        nt += 1
    sim.last_solve()
    # No autotuning here: some launch shapes (dot-product chunk, update tile and grid) change the order of the
    # FP64 sums, and at this spacing the dynamics are chaotic, so a timed choice would make the trajectory --
    # and the iteration counts -- differ from run to run.  The default shapes keep every run identical.
    tuning = sim.tuning()
    torch.cuda.synchronize()

    # The timed steps run in blocks of TRAJECTORY_BLOCK steps 0, 1, ... from the seeded initial state, each block
    # restarted from it (outside the events).  At 20a spacing the dynamics are chaotic: any change in the order of a
    # floating-point sum moves a long trajectory, its GMRES iteration counts with it, and near-contact states make
    # the saddle system nearly singular, so some trajectories' rates grow without bound after a few dozen steps (one
    # build's run met a non-finite residual at step 27).  Restarted blocks time the same early stretch every run.
    first_nt = 0
    snapshot = initial
    sim.restore(snapshot)
    block = min(TRAJECTORY_BLOCK, args.steps)
    barrier(world)
    with ClockSampler(local) as clocks:
        total_ms = time_steps(sim, stream, flush, first_nt, args.steps, restart=snapshot, block=block)
    barrier(world)
    res = sim.last_solve()
    block_iters = sim.iteration_log(4096)[[i % 4096 for i in range(first_nt, first_nt + block)]]
    iters = np.array([block_iters[k % block] for k in range(args.steps)])
    launches = int(sum(sim.launches_per_step(int(i)) for i in iters))
    value, max_ms = replica_throughput(world, float(args.steps), total_ms)
    steps_all = sum_over_ranks(world, float(args.steps))

    # ---- end to end through the host API: state up from pinned memory, step, results down; the same steps
    #      as the timed region (the same blocks from the same checkpoint, restored outside the events)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float64)).pin_memory()
    st = snapshot
    F = NX * NX
    N = F * NSEG
    h_x = torch.empty(3 * N, dtype=torch.float32).pin_memory()
    h_f = torch.empty(6 * N, dtype=torch.float32).pin_memory()
    barrier(world)
    e2e_local = 0.0
    e2e_iter_list = []
    done = 0
    while done < args.steps:
        n_blk = min(block, args.steps - done)
        sim.restore(st)  # the warm start too: the block then starts exactly as the timed ones
        h_phase, h_angle, h_pd, h_ad = (pin(st[k]) for k in ("phase", "angle", "phase_dot", "angle_dot"))
        torch.cuda.synchronize()
        e_events = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        e_events[0].record(stream)
        for k in range(n_blk):
            # H2D 4*F doubles of state; D2H 4*F doubles of state, 3N + 6N floats of positions and forces, status
            state = (h_phase, h_angle, h_pd, h_ad)
            r = sim.step_io(first_nt + k, state_in=state, state_out=state, x_segs=h_x, f_segs=h_f)
            e2e_iter_list.append(r.iterations)
        e_events[1].record(stream)
        torch.cuda.synchronize()
        e2e_local += e_events[0].elapsed_time(e_events[1])
        done += n_blk
    e2e_ms = max_over_ranks(world, e2e_local)
    e2e_value = steps_all / (e2e_ms / 1e3)
    e2e_iters = float(np.mean(e2e_iter_list))

    # ---- the patch refresh (Gauss-Jordan inversion of every patch block) alone
    info = sim.precond_info()
    refresh_ms = time_refresh(sim, stream, flush)
    refresh_tflops = info["refresh_flops"] / (refresh_ms * 1e-3) / 1e12

    # ---- the pair mobility product (tile kernel + reduce) on this geometry: RPY pairs/s
    x_segs, _ = sim.segments()
    mob = RpyMobilitySolver(N, 0, wall=True, seg_dof=3, device=local)
    xd = torch.as_tensor(x_segs, device=dev)
    fd = torch.randn(6 * N, device=dev)
    vd = torch.empty(6 * N, device=dev)
    ms = torch.cuda.Stream(device=dev)
    for _ in range(5):
        mob.apply_device(xd, fd, vd, stream=ms)
    ms.synchronize()
    reps = 50
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    mt = 0.0
    for r in range(reps):
        with torch.cuda.stream(ms):
            flush.zero_()
            a.record(ms)
        mob.apply_device(xd, fd, vd, stream=ms)
        with torch.cuda.stream(ms):
            b.record(ms)
        ms.synchronize()
        mt += a.elapsed_time(b)
    apply_us = mt / reps * 1e3
    pairs = float(N) * N
    pair_tflops = pairs * F_PAIR / (apply_us * 1e-6) / 1e12
    mob.finalise()

    # ---- plain GMRES (the reference's block-diagonal preconditioner) from the same state
    plain_steps = min(args.steps, 8)
    psim = WallCiliaSimulation(**inp, gmres_tol=GMRES_TOL, device=local, precond=_lib.CF_PRECOND_BLOCK_DIAG)
    pstream = torch.cuda.ExternalStream(psim.stream_handle(), device=dev)
    for k in range(2):
        psim.step(k)
    plain_ms = time_steps(psim, pstream, flush, 2, plain_steps)
    pres = psim.last_solve()
    piters = psim.iteration_log(2 + plain_steps)[2:2 + plain_steps]
    psim.close()
    plain_value = plain_steps / (plain_ms / 1e3)

    batched = run_batched(local, inp, world, rank) if not args.no_batched else None
    large = run_large(local, inp, flush) if (world == 1 and not args.no_batched) else None
    fcm = run_fcm(local, flush) if (world == 1 and not args.no_batched) else None
    swimmer = run_swimmer() if (world == 1 and not args.no_batched) else None
    elastic = run_elastic_sim() if (world == 1 and not args.no_batched) else None
    cpu = cpu_baseline(inp) if (rank == 0 and world == 1 and not args.no_cpu_baseline) else None

    if rank == 0:
        cs = clocks.summary()
        step_ms = max_ms / args.steps
        refresh_share = refresh_ms / step_ms
        pair_share = float(np.mean(iters) + 1) * apply_us * 1e-3 / step_ms
        tc_peak = measured_bf16_tflops() / 2.0 / 3.0  # TF32 at half the BF16 rate, three products per FP32 product
        roof_refresh = {"bound": "tensor", "achieved": refresh_tflops, "peak": tc_peak, "unit": "TFLOP/s",
                        "frac": refresh_tflops / tc_peak, "traffic": REFRESH_UPDATE_DRAM_BYTES,
                        "kernel": "patch refresh",
                        "share_of_step": refresh_share,
                        "frac_of_nominal_fp32": refresh_tflops / FP32_PEAK_TFLOPS,
                        "note": f"assembly + blocked Gauss-Jordan of {info['patches']} patch blocks of "
                                f"{info['max_n']} unknowns, 2 n^3 flop each per rebuild, CUDA events around one "
                                "rebuild; the rank-64 updates run as three TF32 tcgen05 products per FP32 product: "
                                "peak = measured dense BF16 rate / 2 (TF32) / 3 (products), of measured; the rebuild "
                                "is bound by its chain of 16 pivot-block inverses (FP32 SIMT), not by the tensor "
                                "cores; traffic: one gj_update launch (the refresh's top kernel; 16 per rebuild), ncu"}
        roof_pairs = {"bound": "fp32", "achieved": pair_tflops, "peak": FP32_PEAK_TFLOPS, "unit": "TFLOP/s",
                      "frac": pair_tflops / FP32_PEAK_TFLOPS, "traffic": PAIR_KERNEL_DRAM_BYTES,
                      "kernel": "pair mobility product",
                      "share_of_step": pair_share,
                      "note": f"{F_PAIR} flop/pair x {N}^2 pairs per launch (tile kernel + reduce), CUDA events; "
                              "nominal FP32 SIMT peak; traffic: the tile kernel's DRAM bytes per launch, ncu"}
        dominant, other = (roof_refresh, roof_pairs) if refresh_share >= pair_share else (roof_pairs, roof_refresh)
        line = {
            "metric": "timesteps/s, learned-precond vs plain GMRES at tol 1e-6; RPY pairs/s", "value": value,
            "unit": "timesteps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 pairs and patch inverses / f64 GMRES",
            "data": "synthetic (seeded phases; reference forcing tables)",
            "config": config_dict({"parallelism": f"replicas x{world}"}),
            "gmres_iters_per_step": float(np.mean(iters)), "last_relres": res.relative_residual,
            "plain_gmres": {"value": plain_value, "unit": "timesteps/s", "steps": plain_steps,
                            "gmres_iters_per_step": float(np.mean(piters)), "last_relres": pres.relative_residual,
                            "converged": bool(pres.status == _lib.CF_OK)},
            "speedup_vs_plain": value / plain_value,
            "rpy_pairs_per_s": pairs / (apply_us * 1e-6), "rpy_apply_us": apply_us,
            "patch_refresh_ms": refresh_ms, "tuning": tuning,
            # build-comparable figure: the step time outside the refresh per GMRES iteration (the iteration count
            # itself follows the chaotic trajectory, which any change in a floating-point sum order moves)
            "ms_per_gmres_iteration": (max_ms / args.steps - refresh_ms) / max(1.0, float(np.mean(iters))),
            "roofline": dominant, "roofline_other": other,
            "traffic_note": "ncu: one gj_update launch, the refresh's top kernel, reads 37.4 MB of DRAM under "
                            "ncu's cold cache (one read of the upper block triangle; the 63 MB of patch matrices "
                            "stay L2-resident between rounds); the pair kernel 0.18 MB: both are compute-bound",
            "e2e": {"value": e2e_value, "unit": "timesteps/s", "h2d_bytes_per_step": 4 * F * 8,
                    "d2h_bytes_per_step": 4 * F * 8 + 3 * N * 4 + 6 * N * 4 + 40, "gmres_iters_per_step": e2e_iters,
                    "call": "WallCiliaSimulation.step_io (cf_sim_step_io): state up, step, state + positions + "
                            "forces down, one synchronisation",
                    "steps": "the timed blocks of steps replayed from the seeded initial state (state and warm "
                             "start restored outside the events)"},
            "gpu_launches": launches, "clocks": cs,
            "batched": batched,
            "lattice_32x32": large,
            "fcm": fcm,
            "swimmer": swimmer,
            "elastic": elastic,
            "cpu_baseline": cpu,
            "vs_cpu_same_precond": (plain_value / cpu["value"]) if cpu else None,
        }
        print(json.dumps(line), flush=True)
    sim.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _oracle_sim(inp):
    from oracle import implicit
    return implicit.WallCilia(bases=inp["bases"], nseg=inp["nseg"], seg_sep=inp["seg_sep"], shape_sequence=1,
                              dt=inp["dt"], phase0=inp["phase0"], angle0=inp["angle0"],
                              spring_factor=inp["spring_factor"], phase_refs=inp["phase_refs"],
                              angle_refs=inp["angle_refs"], s_table=inp["s_table"], gmres_tol=GMRES_TOL)


def cpu_pairs_per_s(x, reps=5):
    """The oracle's OpenMP wall RPY sum (all host threads) over every pair of x, FP64 and FP32: median pairs/s
    of `reps` timed products on identical inputs (one untimed product first)."""
    import oracle
    n = x.shape[0]
    f = np.random.default_rng(7).standard_normal((n, 3))
    out = {}
    for name, dt in (("f64", np.float64), ("f32", np.float32)):
        xx, ff = x.astype(dt), f.astype(dt)
        oracle.rpy_apply(xx, xx, ff, wall=1, vdof=3, fdof=3, self_by_index=True, dtype=dt)
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            oracle.rpy_apply(xx, xx, ff, wall=1, vdof=3, fdof=3, self_by_index=True, dtype=dt)
            ts.append(time.perf_counter() - t0)
        out[name] = float(n) * n / statistics.median(ts)
    return out


def cpu_baseline(inp, steps=1):
    """The oracle (FP64 restatement of the reference's step, pinned to the reference's own step code) on all
    host cores: one implicit step; and the OpenMP RPY sum on the same geometry in pairs/s."""
    import oracle
    sim = _oracle_sim(inp)
    t0 = time.perf_counter()
    its = []
    for nt in range(steps):
        it, _ = sim.step(nt)
        its.append(it)
    dt = time.perf_counter() - t0
    pps = cpu_pairs_per_s(sim.x)
    return {"value": steps / dt, "unit": "timesteps/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"{steps} implicit step(s) of the same 5120-segment array from the same initial state "
                      f"({int(np.mean(its))} GMRES iterations, block-diagonal preconditioner)",
            "rpy_pairs_per_s_f64": pps["f64"], "rpy_pairs_per_s_f32": pps["f32"],
            "rpy_sample": f"wall 3x3 RPY sum over all {sim.x.shape[0]}^2 pairs of the step-0 geometry, OpenMP over "
                          "targets on every host thread, median of 5"}


# ------------------------------------------------------------------ reference
REFERENCE_BUDGET_S = 150.0


def reference_gpu_timings(inp, steps=3):
    """The reference's own CUDA code on this GPU (beside the host-core arm; not the line's value):
    Mss_mult (cuda_functions.cu:362-474, FP32, one thread per target) with CUDA events at 5120 and 20 480
    segments; the reference's whole step (host FP32 GMRES + Mss_mult per iteration, rpy_mobility_solver.cu)
    on the benchmark array, host wall time per step as the reference measures it; the reference cuFCM apply
    (FCM_solver::hydrodynamic_solver) at the sphere-with-cilia size."""
    import ctypes
    import torch
    from oracle import ref_step
    from cufcm_fil_b200 import workloads
    out = {}
    lib_rpy = ROOT / "oracle" / "_ref" / "libref_rpy_wall3.so"
    if lib_rpy.exists():
        L = ctypes.CDLL(str(lib_rpy))
        vp, i = ctypes.c_void_p, ctypes.c_int
        L.ref_set_sizes.argtypes = [i, i, i, i]
        L.ref_mss_async.argtypes = [vp, vp, vp, i, i]
        mss = {}
        for nx in (16, 32):
            x = workloads.vertical_lattice(nx, nx, NSEG, spacing=SPACING).astype(np.float32)
            n = x.shape[0]
            xd = torch.as_tensor(x.ravel(), device="cuda")
            fd = torch.randn(6 * n, device="cuda")
            vd = torch.empty(6 * n, device="cuda")
            assert L.ref_set_sizes(1, NSEG, n // NSEG, 0) == 0
            p = lambda t: ctypes.c_void_p(t.data_ptr())
            for _ in range(3):
                L.ref_mss_async(p(vd), p(fd), p(xd), 0, n)
            torch.cuda.synchronize()
            reps = 20
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            cur = torch.cuda.default_stream()  # the reference launches on the legacy default stream
            a.record(cur)
            for _ in range(reps):
                L.ref_mss_async(p(vd), p(fd), p(xd), 0, n)
            b.record(cur)
            torch.cuda.synchronize()
            us = a.elapsed_time(b) / reps * 1e3
            mss[str(n)] = {"us": us, "pairs_per_s": float(n) * n / (us * 1e-6),
                           "tflops": float(n) * n * F_PAIR / (us * 1e-6) / 1e12}
        out["mss_mult"] = mss
    if ref_step.available("step_dyn_gpu"):
        F = NX * NX
        r = ref_step.run(nfil=F, fil_x_dim=NX, spacing=SPACING, phase0=inp["phase0"], angle0=inp["angle0"],
                         steps=1 + steps, phase_refs=inp["phase_refs"], angle_refs=inp["angle_refs"],
                         s_table=inp["s_table"], variant="step_dyn_gpu", timeout=600.0)
        sec = r.seconds[1:] if len(r.seconds) > 1 else r.seconds
        out["step"] = {"value": 1.0 / float(np.mean(sec)), "unit": "timesteps/s", "steps": int(len(sec)),
                       "gmres_iters_per_step": float(np.mean(r.iterations[1:] if len(sec) > 1 else r.iterations)),
                       "note": "the reference's step (FP32 build) with its rpy_mobility_solver back-end on this GPU, "
                               "block-diagonal preconditioner, first step untimed; host wall time per step"}
    lib_fcm = ROOT / "oracle" / "_ref" / "libref_fcm.so"
    if lib_fcm.exists():
        Lf = ctypes.CDLL(str(lib_fcm))
        Lf.ref_fcm_create.restype = ctypes.c_void_p
        Lf.ref_fcm_create.argtypes = [ctypes.c_int] + [ctypes.c_float] * 4 + [ctypes.c_int] * 3 + [ctypes.c_float]
        Lf.ref_fcm_apply.argtypes = [ctypes.c_void_p] * 6
        segs, blobs = workloads.sphere_with_cilia()
        Y = np.concatenate([segs, blobs]).astype(np.float32)
        n = Y.shape[0]
        Fr = np.random.default_rng(11).standard_normal((n, 3)).astype(np.float32)
        h = Lf.ref_fcm_create(n, 1.0, 1.0, 10.0, 6.0, 512, 512, 512, 1024.0)
        yd = torch.as_tensor(Y.ravel(), device="cuda")
        fd = torch.as_tensor(Fr.ravel(), device="cuda")
        td = torch.zeros(3 * n, device="cuda")
        vd = torch.zeros(3 * n, device="cuda")
        wd = torch.zeros(3 * n, device="cuda")
        p = lambda t: ctypes.c_void_p(t.data_ptr())
        for _ in range(2):
            Lf.ref_fcm_apply(h, p(yd), p(fd), p(td), p(vd), p(wd))
        ts = []
        for _ in range(5):
            t0 = time.perf_counter()
            assert Lf.ref_fcm_apply(h, p(yd), p(fd), p(td), p(vd), p(wd)) == 0
            ts.append(time.perf_counter() - t0)
        out["cufcm_apply_ms"] = statistics.median(ts) * 1e3
        out["cufcm_note"] = ("FCM_solver::hydrodynamic_solver at 30 000 particles, 512^3, alpha 1 beta 10 eta 6; "
                             "host wall time of the synchronous call, median of 5")
    return out


def run_reference(args):
    world, rank, _ = dist_init()
    if rank != 0:
        return
    import oracle
    from oracle import ref_step
    inp = workload_inputs(s_table_from="reference")
    F = NX * NX
    # The reference's own prescribed-cilia step code (mobility_solver.cpp, filament.cpp, ...: host GMRES, its
    # block-diagonal preconditioner, beat and time stepping) built for the host in FP64, its mobility products
    # by the oracle's OpenMP RPY sum (the reference has no CPU mobility of its own).  Bounded: the first step
    # is untimed, then as many steps as the budget allows.
    r = ref_step.run(nfil=F, fil_x_dim=NX, spacing=SPACING, phase0=inp["phase0"], angle0=inp["angle0"],
                     steps=1 + args.steps, phase_refs=inp["phase_refs"], angle_refs=inp["angle_refs"],
                     s_table=inp["s_table"], variant="step_dyn_f64", budget=REFERENCE_BUDGET_S)
    timed = r.seconds[1:] if len(r.seconds) > 1 else r.seconds
    its = r.iterations[1:] if len(r.seconds) > 1 else r.iterations
    done = int(len(timed))
    value = done / float(np.sum(timed)) if done else 0.0
    cores = oracle.num_threads()
    sample = (f"{done} full implicit step(s) of the 5120-segment array after 1 untimed, bounded by a "
              f"{REFERENCE_BUDGET_S:.0f} s budget: the reference's own step code (FP64 host build) with an "
              "OpenMP RPY sum for its mobility products")
    line = {
        "impl": "reference", "metric": "timesteps/s, learned-precond vs plain GMRES at tol 1e-6; RPY pairs/s",
        "value": value, "unit": "timesteps/s", "n_gpus": world, "steps": done, "warmup": 1,
        "ms_per_step": float(np.mean(timed)) * 1e3 if done else None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded phases; reference forcing tables)",
        "config": config_dict(), "gmres_iters_per_step": float(np.mean(its)) if done else None,
        "cpu_baseline": {"value": value, "unit": "timesteps/s", "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    try:
        import torch
        if torch.cuda.is_available():
            line["reference_gpu"] = reference_gpu_timings(inp)
    except Exception as exc:  # the GPU timings are extra context; the host-core arm stands without them
        line["reference_gpu"] = {"unavailable": f"{type(exc).__name__}: {exc}"[:200]}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
