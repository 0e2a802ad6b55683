"""Measurement entry points (the command lines of the committed profiles).

  python -m cufcm_fil_b200.perf step --nx 16 --precond line --steps 2 [--warm W] [--block B]
      implicit steps of the benchmark lattice (lattice_simulation), each timed
      with CUDA events, and a fit of step time against GMRES iterations; with
      CUFIL_NO_GRAPH=1 every kernel is an ordinary launch, which is what a
      profiler's launch list needs.
  python -m cufcm_fil_b200.perf fcm --grid 512 --reps 5
      the sphere-with-cilia FCM workload (1000 cilia x 20 segments + 10 000
      body blobs, box 1024a): stage times of one apply and the achieved
      bandwidth of spreading and interpolation against their algorithmic bytes
      (spread: N ngd^3 x 3 read-modify-writes of 4 bytes each way; gather:
      N ngd^3 x 3 reads of 4 bytes).
  python -m cufcm_fil_b200.perf refresh --nx 16 --reps 20
      one rebuild of the line-patch inverses of the benchmark lattice after its
      first step (assembly + the Gauss-Jordan rounds), CUDA events on the
      engine's stream, L2 flushed before each rebuild: mean and minimum.
  python -m cufcm_fil_b200.perf elastic --nx 16 --steps 4
      elastic instability cilia (cf_elastic): nx x nx filaments of 20
      segments on a wall lattice at 80a, Broyden's method at the reference's
      settings; host wall clock per synchronous step after step 0.
  python -m cufcm_fil_b200.perf swimmer --steps 4
      the free swimmer (cf_swim) of the benchmark: 256 cilia x 20 segments on a
      sphere of 2562 blobs; host wall clock per synchronous step after step 0.
  python -m cufcm_fil_b200.perf mlp --batch 1024 --reps 50
      forward passes of the learned preconditioner's network (182 -> 256 -> 256
      -> 62, BF16 GEMMs) at one filament per row, as one GMRES iteration of the
      32 x 32 lattice runs it; CUDA events around each pass.
Each prints one JSON line.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import _lib


def run_steps(nx: int, precond: str, steps: int, line_patch: int = 0, warm: int = 0, block: int = 0):
    """`warm` untimed steps, then `steps` implicit steps, each timed with CUDA events on the engine's stream
    (without warm-up steps the first includes the graph capture).  With `block`, steps 0 .. block - 1 run
    again and again, each block restored from the seeded initial state (outside the events; the 20a lattice
    cannot run long stretches, its colliding cilia reach non-finite states).  With three or more timed
    steps, a least-squares fit step_ms = fixed_ms + ms_per_iteration * iterations splits the step time into
    the per-step part (kinematics, right-hand side, refresh, finish) and the cost of one GMRES iteration."""
    import torch
    from .sim import lattice_simulation
    code = {"line": _lib.CF_PRECOND_LINE, "block": _lib.CF_PRECOND_BLOCK_DIAG, "none": _lib.CF_PRECOND_NONE}[precond]
    its, ms = [], []
    with lattice_simulation(nx, precond=code, line_patch=line_patch) as sim:
        stream = torch.cuda.ExternalStream(sim.stream_handle())
        initial = sim.checkpoint() if block else None

        def nt_of(k):
            if not block:
                return k
            if k > 0 and k % block == 0:
                sim.restore(initial)
            return k % block
        for k in range(warm):
            sim.step(nt_of(k))
        torch.cuda.synchronize()
        for k in range(warm, warm + steps):
            nt = nt_of(k)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            its.append(sim.step(nt).iterations)
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
    out = {"nx": nx, "precond": precond, "warm": warm, "block": block, "steps": steps, "gmres_iterations": its,
           "step_ms": ms}
    if steps >= 3 and len(set(its)) > 1:
        slope, icpt = np.polyfit(np.asarray(its, float), np.asarray(ms, float), 1)
        out.update(fixed_ms=float(icpt), ms_per_iteration=float(slope), mean_step_ms=float(np.mean(ms)))
    return out


def warm_up(fn, seconds: float = 1.0):
    """Repeats `fn` for about `seconds` of device time, so that the GPU has left its idle clocks before the
    timed launches (short runs otherwise start at a fraction of the boost clock)."""
    import time
    import torch
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < seconds or n < 3:
        fn()
        n += 1
        if n % 16 == 0:
            torch.cuda.synchronize()
    torch.cuda.synchronize()


def run_refresh(nx: int, reps: int):
    import torch
    from .sim import lattice_simulation
    with lattice_simulation(nx, precond=_lib.CF_PRECOND_LINE) as sim:
        sim.step(0)
        stream = torch.cuda.ExternalStream(sim.stream_handle())
        flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")  # 256 MiB, twice the L2
        warm_up(lambda: sim.refresh_preconditioner())
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for a, b in ev:
            with torch.cuda.stream(stream):
                flush.zero_()
                a.record(stream)
            sim.refresh_preconditioner()
            with torch.cuda.stream(stream):
                b.record(stream)
        torch.cuda.synchronize()
        ms = [a.elapsed_time(b) for a, b in ev]
    return {"nx": nx, "reps": reps, "refresh_ms_mean": float(np.mean(ms)), "refresh_ms_min": float(np.min(ms))}


def run_elastic(nx: int, steps: int):
    import time
    from . import workloads
    from .elastic import ElasticCiliaSimulation
    with ElasticCiliaSimulation(bases=workloads.lattice_bases(nx * nx, nx, 80.0, 1.3)) as sim:
        sim.step(0)
        ms, its = [], []
        for nt in range(1, 1 + steps):
            t0 = time.perf_counter()
            its.append(sim.step(nt))
            ms.append(1e3 * (time.perf_counter() - t0))
    return {"nx": nx, "steps": steps, "broyden_iterations": its, "step_ms": ms}


def run_swimmer(steps: int):
    import time
    from pathlib import Path
    from . import swim
    golden = Path(__file__).resolve().parents[1] / "tests" / "golden"
    gold = np.load(golden / "reference_forcing_nseg20_sep2.6.npz")
    tips = np.load(golden / "ref_tips_16x16_80a.npz")
    F, B = 256, 2562
    geo = swim.sphere_geometry(swim.fibonacci_normals(F), swim.fibonacci_normals(B, 0.3), ar=6.0)
    rng = np.random.default_rng(12)
    with swim.CiliatedSwimmer(geometry=geo, phase0=rng.uniform(0, 2 * np.pi, F), angle0=rng.normal(0, 0.05, F),
                              phase_refs=gold["fb_phase"], angle_refs=gold["fb_angle"],
                              s_table=tips["s_table"]) as sim:
        sim.step(0)
        ms, its = [], []
        for nt in range(1, 1 + steps):
            t0 = time.perf_counter()
            its.append(sim.step(nt).iterations)
            ms.append(1e3 * (time.perf_counter() - t0))
    return {"steps": steps, "gmres_iterations": its, "step_ms": ms}


def run_fcm(grid: int, reps: int, hbm_gbs: float | None = None):
    import torch
    from . import workloads
    from .fcm import FcmSolver
    segs, blobs = workloads.sphere_with_cilia()
    Y = np.concatenate([segs, blobs])
    n = Y.shape[0]
    F = np.random.default_rng(11).standard_normal((n, 3))
    kw = dict(rh=1.0, alpha=1.0, beta=10.0, eta=6.0, nx=grid, ny=grid, nz=grid, boxsize=1024.0)
    Yd = torch.as_tensor(Y.astype(np.float32).ravel(), device="cuda")
    Fd = torch.as_tensor(F.astype(np.float32).ravel(), device="cuda")
    Vd = torch.empty_like(Fd)
    with FcmSolver(n, **kw) as s:
        info = s.info()
        s.set_timing(True)
        for _ in range(2):
            s.apply_device(Yd, Fd, Vd)
        torch.cuda.synchronize()
        acc = {k: 0.0 for k in FcmSolver.STAGES}
        for _ in range(reps):
            s.apply_device(Yd, Fd, Vd)
            torch.cuda.synchronize()
            for k, v in s.stage_times().items():
                acc[k] += v / reps
    ngd3 = int(info["ngd"]) ** 3
    spread_bytes = n * ngd3 * 3 * 8
    gather_bytes = n * ngd3 * 3 * 4
    out = {"grid": grid, "particles": n, "ngd": int(info["ngd"]), "stage_ms": acc,
           "total_ms": sum(acc.values()),
           "spread_GBps": spread_bytes / (acc["spread"] * 1e-3) / 1e9 if acc["spread"] > 0 else None,
           "gather_GBps": gather_bytes / (acc["gather"] * 1e-3) / 1e9 if acc["gather"] > 0 else None}
    if hbm_gbs:
        out["spread_frac"] = out["spread_GBps"] / hbm_gbs
        out["gather_frac"] = out["gather_GBps"] / hbm_gbs
    return out


def run_mlp(batch: int, reps: int):
    import torch
    from .mlp import FilamentMLP
    with FilamentMLP(182, 256, 62, max_batch=batch, seed=0) as net:
        x = torch.randn(batch, 182, device="cuda")
        y = torch.empty(batch, 62, device="cuda")
        st = torch.cuda.Stream()
        torch.cuda.synchronize()
        warm_up(lambda: net.forward(x, y, stream=st), 0.5)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for a, b in ev:  # events on the stream the network's kernels run on
            a.record(st)
            net.forward(x, y, stream=st)
            b.record(st)
        st.synchronize()
        us = sorted(1e3 * a.elapsed_time(b) for a, b in ev)
    flop = 2 * batch * (182 * 256 + 256 * 256 + 256 * 62)
    return {"batch": batch, "forward_us_median": us[len(us) // 2], "flop_per_forward": flop,
            "tflops": flop / (us[len(us) // 2] * 1e-6) / 1e12}


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m cufcm_fil_b200.perf")
    sub = ap.add_subparsers(dest="what", required=True)
    st = sub.add_parser("step")
    st.add_argument("--nx", type=int, default=16)
    st.add_argument("--precond", choices=["line", "block", "none"], default="line")
    st.add_argument("--steps", type=int, default=2)
    st.add_argument("--line-patch", type=int, default=0)
    st.add_argument("--warm", type=int, default=0)
    st.add_argument("--block", type=int, default=0)
    fc = sub.add_parser("fcm")
    fc.add_argument("--grid", type=int, default=512)
    fc.add_argument("--reps", type=int, default=5)
    fc.add_argument("--hbm-gbs", type=float, default=None)
    rf = sub.add_parser("refresh")
    rf.add_argument("--nx", type=int, default=16)
    rf.add_argument("--reps", type=int, default=20)
    el = sub.add_parser("elastic")
    el.add_argument("--nx", type=int, default=16)
    el.add_argument("--steps", type=int, default=4)
    sw = sub.add_parser("swimmer")
    sw.add_argument("--steps", type=int, default=4)
    ml = sub.add_parser("mlp")
    ml.add_argument("--batch", type=int, default=1024)
    ml.add_argument("--reps", type=int, default=50)
    a = ap.parse_args(argv)
    if a.what == "step":
        print(json.dumps(run_steps(a.nx, a.precond, a.steps, a.line_patch, a.warm, a.block)))
    elif a.what == "refresh":
        print(json.dumps(run_refresh(a.nx, a.reps)))
    elif a.what == "elastic":
        print(json.dumps(run_elastic(a.nx, a.steps)))
    elif a.what == "swimmer":
        print(json.dumps(run_swimmer(a.steps)))
    elif a.what == "mlp":
        print(json.dumps(run_mlp(a.batch, a.reps)))
    else:
        print(json.dumps(run_fcm(a.grid, a.reps, a.hbm_gbs)))


if __name__ == "__main__":
    main()
