"""Bounded device waits that give up are reported, not silently summed.

The staged tile kernel (every product except the symmetric 3x3 wall kernel)
waits for its bulk-copied sources on an mbarrier with an iteration limit.  The
test hook cf_set_wait_limit(0) makes that first wait give up at once; the block
still drains its copies with the full limit before it exits, so the GPU state
stays clean.  The handle path must then return CF_TIMEOUT with NaN velocities,
and the next product with the default limit must be correct again.
"""
import numpy as np
import pytest

import oracle
from cufcm_fil_b200 import RpyMobilitySolver, _lib, workloads

pytestmark = pytest.mark.gpu

DEFAULT_LIMIT = 0xFFFFFFFF  # clamped to the full limit


def _forces(n, seed):
    f = np.zeros((n, 6), np.float32)
    f[:] = workloads.random_forces(n, 6, seed=seed)
    return f


def test_given_up_wait_returns_timeout_then_recovers(cuda):
    x = workloads.vertical_lattice(4, 4, 20).astype(np.float32)
    n = x.shape[0]
    f = _forces(n, 3)
    with RpyMobilitySolver(n, 0, wall=True, seg_dof=6) as mob:
        v_ok, _ = mob.apply(x, f)
        try:
            _lib.call("cf_set_wait_limit", 0)
            with pytest.raises(_lib.CufilError) as ei:
                mob.apply(x, f)
            assert ei.value.code == _lib.CF_TIMEOUT
            assert "bounded device wait" in str(ei.value)
            assert np.all(np.isnan(mob.v_segs_host))
        finally:
            _lib.call("cf_set_wait_limit", DEFAULT_LIMIT)
        v_again, _ = mob.apply(x, f)
    np.testing.assert_array_equal(v_again, v_ok)
    v64, _ = oracle.mobility_full(x, f, wall=True, seg_dof=6)
    assert oracle.rel_l2(v_again, v64) <= 1e-5
