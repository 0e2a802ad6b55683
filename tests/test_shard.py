"""Sharding independent wall arrays over ranks: world-size-2 gloo ranks on the CPU.

Each rank takes its bin of arrays (cufcm_fil_b200.shard.bin_by_cost), steps
them through the FP64 oracle (the restatement of the reference's step, pinned
to the reference's own step code by tests/test_ref_step.py) and the results are
gathered on rank 0.  The union must equal a single-process run of every array,
bit for bit: the data path has no collective, so sharding changes nothing but
where each array runs.
"""
import multiprocessing as mp
import os
import socket
from datetime import timedelta
from pathlib import Path

import numpy as np
import pytest

from cufcm_fil_b200 import shard, workloads

GOLD = Path(__file__).resolve().parent / "golden" / "reference_forcing_nseg20_sep2.6.npz"


def _specs():
    rng = np.random.default_rng(42)
    out = []
    for n in (1, 4, 2, 3, 1, 2):
        out.append(dict(n=n, phase0=rng.uniform(0, 2 * np.pi, n), angle0=rng.normal(0, 0.05, n)))
    return out


def _run_array(spec, steps):
    from oracle import implicit
    g = np.load(GOLD)
    n = spec["n"]
    nx = int(np.ceil(np.sqrt(n)))
    sim = implicit.WallCilia(bases=workloads.lattice_bases(n, nx, 40.0, 1.3), shape_sequence=1, nseg=20, seg_sep=2.6,
                             dt=1 / 300, phase0=spec["phase0"], angle0=spec["angle0"], spring_factor=0.01,
                             phase_refs=g["fb_phase"], angle_refs=g["fb_angle"], s_table=None,
                             gmres_tol=1e-6, nthreads=1)
    its = [sim.step(nt)[0] for nt in range(steps)]
    return {"tips": sim.tips(), "phase": sim.phase.copy(), "phase_dot": sim.phase_dot.copy(), "iters": its}


def _worker(rank, world, port, steps, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        specs = _specs()
        bins = shard.bin_by_cost([shard.array_cost(sp["n"], 20) for sp in specs], world)
        mine = {i: _run_array(specs[i], steps) for i in bins[rank]}
        got = shard.gather_to_root(mine, world)
        if rank == 0:
            merged = {}
            for part in got:
                merged.update(part)
            q.put((bins, merged))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_bins_are_deterministic_and_balanced():
    costs = [shard.array_cost(n, 20) for n in np.random.default_rng(4).integers(16, 257, 64)]
    bins = shard.bin_by_cost(costs, 8)
    assert bins == shard.bin_by_cost(costs, 8)
    assert sorted(i for b in bins for i in b) == list(range(64))
    assert shard.imbalance(costs, bins) < 1.1
    assert shard.bin_by_cost(costs, 1) == [list(range(64))]


def test_two_ranks_step_their_arrays_and_the_union_equals_one_process():
    steps, world = 3, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    bins, merged = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(merged) == list(range(len(_specs())))
    assert all(len(b) > 0 for b in bins)
    for i, spec in enumerate(_specs()):
        ref = _run_array(spec, steps)
        for k in ("tips", "phase", "phase_dot"):
            np.testing.assert_array_equal(merged[i][k], ref[k])
        assert merged[i]["iters"] == ref["iters"]
