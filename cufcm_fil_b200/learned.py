"""Training of the learned preconditioner's network (CF_PRECOND_LEARNED, CF_PRECOND_LEARNED_LINE).

The pairs come from the plain solver itself: every Arnoldi product w = A z of
its steps gives, per filament, the features of w and the part (z - P(w)) / s
that its preconditioner P misses (WallCiliaSimulation.collect_pairs), with P
the block-diagonal preconditioner (base CF_PRECOND_BLOCK_DIAG, network mode
CF_PRECOND_LEARNED) or the line patches (base CF_PRECOND_LINE, network mode
CF_PRECOND_LEARNED_LINE).  The network is trained on them by the library's own
kernels (FilamentMLP.train_step: BF16 tensor-core GEMMs, Adam).  `compare`
runs the same state with and without the network, the check that decides
whether a trained network is worth using: the base preconditioner stays the
fallback and the reference point.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from .mlp import FilamentMLP


LEARNED_MODE = {_lib.CF_PRECOND_BLOCK_DIAG: _lib.CF_PRECOND_LEARNED, _lib.CF_PRECOND_LINE: _lib.CF_PRECOND_LEARNED_LINE}


def collect(make_sim, seeds, steps_per_seed=1, max_pairs=120, base=_lib.CF_PRECOND_BLOCK_DIAG):
    """Training pairs from runs of `make_sim(seed, base)` (one simulation per seed)."""
    import torch
    xs, ts = [], []
    for seed in seeds:
        with make_sim(seed, base) as sim:
            for nt in range(steps_per_seed):
                x, t = sim.collect_pairs(nt, max_pairs)
                xs.append(x)
                ts.append(t)
    return torch.cat(xs), torch.cat(ts)


def train(net: FilamentMLP, x, t, steps=2000, batch=2048, lr=1e-3, seed=0, report_every=0):
    """Adam on random batches of the pairs; returns the losses seen at the report points."""
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    losses = []
    n = x.shape[0]
    batch = min(batch, n, net.max_batch)
    for k in range(steps):
        idx = torch.randint(0, n, (batch,), device="cuda", generator=g)
        xb, tb = x[idx].contiguous(), t[idx].contiguous()
        want = report_every and (k % report_every == 0 or k == steps - 1)
        loss = net.train_step(xb, tb, lr=lr, want_loss=bool(want))
        if want:
            losses.append(loss)
    return losses


@dataclass
class Comparison:
    block_diagonal_iterations: int
    block_diagonal_status: int
    learned_iterations: int
    learned_status: int
    weight: float = 1.0
    by_weight: dict = None

    @property
    def gain(self) -> float:
        """Iterations of the base solve over those of the learned one (>1: the network helps)."""
        return self.block_diagonal_iterations / max(self.learned_iterations, 1)

    @property
    def use_learned(self) -> bool:
        return self.learned_status == _lib.CF_OK and self.learned_iterations < self.block_diagonal_iterations


def compare(make_sim, seed, net: FilamentMLP, nt=0, weights=(1.0, 0.5, 0.25),
            base=_lib.CF_PRECOND_BLOCK_DIAG) -> Comparison:
    """Step nt of the same state with the base preconditioner and with the network on top of it at each
    correction weight; the weight with the fewest converged iterations is reported."""
    with make_sim(seed, base) as sim:
        rb = sim.step(nt)
    by_weight = {}
    for w in weights:
        with make_sim(seed, LEARNED_MODE[base]) as sim:
            sim.set_network(net)
            sim.set_network_weight(w)
            r = sim.step(nt)
            by_weight[w] = (r.iterations, r.status)
    ok = [w for w in weights if by_weight[w][1] == _lib.CF_OK]
    best = min(ok, key=lambda w: by_weight[w][0]) if ok else weights[0]
    return Comparison(rb.iterations, rb.status, by_weight[best][0], by_weight[best][1], best, by_weight)
