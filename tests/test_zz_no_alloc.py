"""The allocation-free wall product against the allocating one, through the C ABI.

cf_rpy_wall_segments_noalloc is for callers that cannot allocate device memory
at call time -- code running under CUDA stream capture, where cudaMalloc is not
allowed, or a host whose own allocator owns all device memory -- so its
scratch is a fixed array inside libcufil.so.  This test calls it twice in a
row (different forces, same array) and compares each result with
RpyMobilitySolver.apply_device (the handle-based entry point, which allocates
its scratch at creation) at the tolerance of the mobility contract, 1e-5
relative L2.  It lives in its own file, collected last.
"""
import ctypes

import numpy as np
import pytest

import oracle
from cufcm_fil_b200 import RpyMobilitySolver, _lib, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _noalloc(torch, x, f, n):
    v = torch.empty(6 * n, device="cuda")
    stream = torch.cuda.current_stream()
    _lib.call("cf_rpy_wall_segments_noalloc", ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(f.data_ptr()),
              ctypes.c_void_p(v.data_ptr()), n, ctypes.c_void_p(stream.cuda_stream))
    stream.synchronize()
    return v.cpu().numpy()


@pytest.mark.parametrize("nx,ny,nseg", [(16, 16, 20), (7, 3, 13)])
def test_noalloc_matches_allocating_entry_point_twice(cuda, nx, ny, nseg):
    torch = cuda
    x = workloads.vertical_lattice(nx, ny, nseg).astype(np.float32)
    n = x.shape[0]
    xd = torch.as_tensor(x.ravel(), device="cuda")
    with RpyMobilitySolver(n, 0, wall=True, seg_dof=3) as mob:
        for seed in (1, 2):  # two calls in a row share the library's scratch array
            f = np.zeros((n, 6), np.float32)
            f[:, :3] = workloads.random_forces(n, 3, seed=seed)
            fd = torch.as_tensor(f.ravel(), device="cuda")
            got = _noalloc(torch, xd, fd, n)
            ref = torch.empty(6 * n, device="cuda")
            mob.apply_device(xd, fd, ref, stream=torch.cuda.current_stream())
            torch.cuda.synchronize()
            ref = ref.cpu().numpy()
            assert oracle.rel_l2(got, ref) <= TOL
            assert np.all(got.reshape(n, 6)[:, 3:] == 0.0)


def test_noalloc_rejects_sizes_beyond_its_limit(cuda):
    torch = cuda
    n = 8193
    x = torch.zeros(3 * n, device="cuda")
    v = torch.zeros(6 * n, device="cuda")
    rc = _lib.load().cf_rpy_wall_segments_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                                   ctypes.c_void_p(v.data_ptr()), n, None)
    assert rc == _lib.CF_EINVAL
    assert "8192" in _lib.last_error()


def test_noalloc_given_up_wait_gives_nan_then_recovers(cuda):
    # The entry point never synchronises, so a bounded wait that gives up
    # (forced here by the cf_set_wait_limit test hook) shows as NaN outputs,
    # never as stale partial sums of an earlier call; the next call with the
    # default limit is correct again.
    torch = cuda
    x = workloads.vertical_lattice(4, 4, 20).astype(np.float32)
    n = x.shape[0]
    xd = torch.as_tensor(x.ravel(), device="cuda")
    f = np.zeros((n, 6), np.float32)
    f[:, :3] = workloads.random_forces(n, 3, seed=4)
    fd = torch.as_tensor(f.ravel(), device="cuda")
    good = _noalloc(torch, xd, fd, n)
    try:
        _lib.call("cf_set_wait_limit", 0)
        bad = _noalloc(torch, xd, fd, n)
    finally:
        _lib.call("cf_set_wait_limit", 0xFFFFFFFF)
    assert np.all(np.isnan(bad))
    again = _noalloc(torch, xd, fd, n)
    np.testing.assert_array_equal(again, good)

