"""GPU tests of the learned preconditioner's network (cf_mlp) against the numpy oracle.

The oracle (oracle/mlp.py) rounds every GEMM operand to BF16 where the kernel
does and accumulates in FP64; the kernel accumulates in FP32 on the tensor
cores.  Tolerances: outputs 1e-4 relative L2; gradients 2e-3 relative L2 per
parameter block (FP32 accumulation order and rare ReLU-mask flips at 0).
"""
import numpy as np
import pytest
import torch

from oracle import mlp as omlp
from cufcm_fil_b200.mlp import FilamentMLP

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("n_in,hid,n_out,n", [(182, 256, 62, 300), (40, 64, 10, 77)])
def test_forward_and_gradients_match_oracle(n_in, hid, n_out, n):
    rng = np.random.default_rng(0)
    X = rng.standard_normal((n, n_in)).astype(np.float32)
    T = rng.standard_normal((n, n_out)).astype(np.float32)
    with FilamentMLP(n_in, hid, n_out, max_batch=512, seed=3) as net:
        p = net.params()
        p[np.arange(p.size) % 7 == 0] += 0.01  # nonzero biases too
        net.set_params(p)
        xd, td = torch.tensor(X, device="cuda"), torch.tensor(T, device="cuda")
        yd = torch.empty((n, n_out), device="cuda")
        net.forward(xd, yd)
        torch.cuda.synchronize()
        _, _, Yref = omlp.forward(p, X, n_in, hid, n_out)
        assert rel(yd.cpu().numpy(), Yref) < 1e-4
        loss, g = net.gradients(xd, td)
        loss_ref, g_ref = omlp.gradients(p, X, T, n_in, hid, n_out)
        assert abs(loss - loss_ref) <= 1e-5 * loss_ref
        sizes = [n_in * hid, hid, hid * hid, hid, hid * n_out, n_out]
        o = 0
        for name, s in zip(["W1", "b1", "W2", "b2", "W3", "b3"], sizes):
            assert rel(g[o:o + s], g_ref[o:o + s]) < 2e-3, name
            o += s


def test_training_reduces_the_loss_on_a_linear_target():
    rng = np.random.default_rng(1)
    n_in, n_out, n = 32, 8, 2048
    W = rng.standard_normal((n_in, n_out)) / np.sqrt(n_in)
    X = rng.standard_normal((n, n_in)).astype(np.float32)
    T = (X @ W).astype(np.float32)
    with FilamentMLP(n_in, 64, n_out, max_batch=n, seed=5) as net:
        xd, td = torch.tensor(X, device="cuda"), torch.tensor(T, device="cuda")
        first = net.train_step(xd, td, lr=1e-3, want_loss=True)
        for _ in range(300):
            net.train_step(xd, td, lr=1e-3)
        last = net.train_step(xd, td, lr=1e-3, want_loss=True)
    assert last < 0.05 * first, (first, last)
