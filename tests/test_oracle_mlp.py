"""The MLP oracle against finite differences (exact FP64 mode) and its BF16 rounding rule."""
import numpy as np

from oracle import mlp as omlp


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-3], np.float32)
    r = omlp.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # tie: rounds to even (1.0)
    assert r[2] == 1.0 + 2 ** -7            # above the tie: rounds up
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-3) <= 2 ** -8 * 3.0e-3   # half an ulp (8 significant bits)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    n_in, hid, n_out, n = 6, 8, 3, 11
    npar = n_in * hid + hid + hid * hid + hid + hid * n_out + n_out
    p = rng.standard_normal(npar) * 0.5
    X = rng.standard_normal((n, n_in))
    T = rng.standard_normal((n, n_out))
    loss, g = omlp.gradients(p, X, T, n_in, hid, n_out, exact=True)
    h = 1e-6
    for i in rng.choice(npar, 40, replace=False):
        e = np.zeros(npar)
        e[i] = h
        lp, _ = omlp.gradients(p + e, X, T, n_in, hid, n_out, exact=True)
        lm, _ = omlp.gradients(p - e, X, T, n_in, hid, n_out, exact=True)
        assert abs((lp - lm) / (2 * h) - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), i
