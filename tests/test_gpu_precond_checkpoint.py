"""Versioned checkpoints of the learned preconditioner's network (cf_precond_save / cf_precond_load)."""
import numpy as np
import pytest

from cufcm_fil_b200 import _lib
from cufcm_fil_b200.mlp import FilamentMLP

pytestmark = pytest.mark.gpu


def test_save_load_round_trip_and_rejects_damaged_files(cuda, tmp_path):
    torch = cuda
    net = FilamentMLP(40, 64, 10, max_batch=128, seed=3)
    p = net.params()
    p += np.random.default_rng(1).standard_normal(p.size).astype(np.float32) * 0.01
    net.set_params(p)
    path = tmp_path / "net.cfp"
    net.save(path, weight=0.25)
    got, w = FilamentMLP.load(path, max_batch=64)
    assert w == 0.25 and (got.n_in, got.hidden, got.n_out) == (40, 64, 10)
    np.testing.assert_array_equal(got.params(), p)
    x = torch.randn(50, 40, device="cuda")
    y1 = torch.empty(50, 10, device="cuda")
    y2 = torch.empty(50, 10, device="cuda")
    net.forward(x, y1)
    got.forward(x, y2)
    torch.cuda.synchronize()
    assert torch.equal(y1, y2)
    raw = path.read_bytes()
    for name, data in {"flipped": raw[:100] + bytes([raw[100] ^ 1]) + raw[101:],
                       "truncated": raw[:-4], "magic": b"X" + raw[1:],
                       "version": raw[:8] + (2).to_bytes(4, "little") + raw[12:]}.items():
        bad = tmp_path / f"{name}.cfp"
        bad.write_bytes(data)
        with pytest.raises(_lib.CufilError) as ei:
            FilamentMLP.load(bad)
        assert ei.value.code == _lib.CF_EINVAL, name
    net.close()
    got.close()
