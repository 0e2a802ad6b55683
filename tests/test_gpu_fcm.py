"""GPU parity of the fast FCM engine (cf_fcm) through the C ABI.

Against the FP64 oracle (oracle/fcm.py, restatement of src/cufcm) on small
grids, and against the reference's own cuFCM solver built from its sources
(oracle/_ref/libref_fcm.so) on the same FP32 inputs.  Tolerances: 1e-4
relative L2 against FP64 (FP32 FFTs of the whole grid), 2e-5 against the
reference's FP32 solver.
"""
import ctypes
from pathlib import Path

import numpy as np
import pytest

import oracle
from oracle import fcm as ofcm
from cufcm_fil_b200 import workloads
from cufcm_fil_b200.fcm import FcmSolver

pytestmark = pytest.mark.gpu

REF_FCM = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libref_fcm.so"


def _random_particles(n, box, seed):
    """n points on a jittered cubic lattice filling the periodic box (spacing > 2.5 a)."""
    rng = np.random.default_rng(seed)
    m = int(np.ceil(n ** (1.0 / 3.0)))
    h = box / m
    idx = rng.permutation(m ** 3)[:n]
    cells = np.stack(np.unravel_index(idx, (m, m, m)), axis=1).astype(float)
    jitter = rng.uniform(-0.5, 0.5, (n, 3)) * max(0.0, h - 2.5)
    return (cells + 0.5) * h + jitter


def _ref_fcm(torch, Y, F, **kw):
    L = ctypes.CDLL(str(REF_FCM))
    L.ref_fcm_create.restype = ctypes.c_void_p
    L.ref_fcm_create.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float]
    L.ref_fcm_apply.argtypes = [ctypes.c_void_p] * 6
    n = Y.shape[0]
    s = L.ref_fcm_create(n, kw["rh"], kw["alpha"], kw["beta"], kw["eta"], kw["nx"], kw["ny"], kw["nz"], kw["boxsize"])
    dev = torch.device("cuda")
    y = torch.as_tensor(np.ascontiguousarray(Y, np.float32).ravel(), device=dev)
    f = torch.as_tensor(np.ascontiguousarray(F, np.float32).ravel(), device=dev)
    t = torch.zeros(3 * n, device=dev)
    v = torch.zeros(3 * n, device=dev)
    w = torch.zeros(3 * n, device=dev)
    p = lambda a: ctypes.c_void_p(a.data_ptr())
    assert L.ref_fcm_apply(s, p(y), p(f), p(t), p(v), p(w)) == 0
    return v.cpu().numpy().reshape(n, 3)


@pytest.mark.parametrize("grid,box,beta,eta,n", [(32, 64.0, 8.0, 5.0, 40), (64, 128.0, 10.0, 6.0, 80)])
def test_fcm_matches_fp64_oracle(cuda, grid, box, beta, eta, n):
    kw = dict(rh=1.0, alpha=1.0, beta=beta, eta=eta, nx=grid, ny=grid, nz=grid, boxsize=box)
    Y = _random_particles(n, box, seed=grid)
    F = np.random.default_rng(grid + 1).standard_normal((n, 3))
    with FcmSolver(n, **kw) as s:
        v = s.hydrodynamic_solver(Y, F)
    v64 = ofcm.fcm_apply(Y.astype(np.float32).astype(np.float64), F.astype(np.float32).astype(np.float64),
                         ofcm.FcmParams(**kw))
    assert oracle.rel_l2(v, v64) <= 1e-4


def test_fcm_matches_reference_cufcm(cuda):
    if not REF_FCM.exists():
        pytest.skip("reference cuFCM not built")
    kw = dict(rh=1.0, alpha=1.0, beta=10.0, eta=6.0, nx=128, ny=128, nz=128, boxsize=256.0)
    n = 3000
    Y = _random_particles(n, 256.0, seed=7)
    F = np.random.default_rng(8).standard_normal((n, 3))
    with FcmSolver(n, **kw) as s:
        v = s.hydrodynamic_solver(Y, F)
    vr = _ref_fcm(cuda, Y, F, **kw)
    assert oracle.rel_l2(v, vr) <= 2e-5


def test_sphere_with_cilia_full_size_vs_reference_and_rpy(cuda):
    # 1000 cilia x 20 segments + 10 000 body blobs on a sphere of radius 100a, box 1024a, 512^3 grid,
    # Gaussian width a/sqrt(pi), alpha = 1, beta = 10, eta = 6 (input/simulation_info_cilia).
    segs, blobs = workloads.sphere_with_cilia()
    Y = np.concatenate([segs, blobs])
    n = Y.shape[0]
    F = np.random.default_rng(11).standard_normal((n, 3))
    F -= F.mean(axis=0)  # a periodic box has no net force; the unbounded comparison is meaningful without one
    kw = dict(rh=1.0, alpha=1.0, beta=10.0, eta=6.0, nx=512, ny=512, nz=512, boxsize=1024.0)
    with FcmSolver(n, **kw) as s:
        v = s.hydrodynamic_solver(Y, F)
    if REF_FCM.exists():
        vr = _ref_fcm(cuda, Y, F, **kw)
        assert oracle.rel_l2(v, vr) <= 2e-5
    # against the FP64 unbounded RPY sum on sampled rows: the engine's error is the reference's error
    rows = np.random.default_rng(12).choice(n, 400, replace=False)
    vrpy = oracle.rpy_apply(Y[rows], Y, F, wall=0, vdof=3, fdof=3, t_ids=rows)
    err_ours = oracle.rel_l2(v[rows], vrpy)
    print(f"FCM vs unbounded FP64 RPY, sampled rows: relative L2 {err_ours:.3e}")
    assert err_ours < 0.25  # periodic images of a dense 30 000-particle body in a 1024a box
    if REF_FCM.exists():
        err_ref = oracle.rel_l2(vr[rows], vrpy)
        print(f"reference cuFCM vs the same: {err_ref:.3e}")
        assert err_ours <= err_ref * 1.01 + 1e-6


def test_segment_blob_adapter_equals_plain_apply(cuda):
    segs, blobs = workloads.sphere_with_cilia(n_cilia=20, nseg=5, n_body=200, radius=15.0, centre=(32, 32, 32))
    ns, nb = segs.shape[0], blobs.shape[0]
    rng = np.random.default_rng(3)
    f6 = np.zeros((ns, 6))
    f6[:, :3] = rng.standard_normal((ns, 3))
    f6[:, 3:] = rng.standard_normal((ns, 3))  # torques are ignored (translation-only FCM)
    fb = rng.standard_normal((nb, 3))
    kw = dict(rh=1.0, alpha=1.0, beta=8.0, eta=5.0, nx=32, ny=32, nz=32, boxsize=64.0)
    with FcmSolver(ns + nb, **kw) as s:
        vs, vb = s.evaluate_full_mobility(segs, f6, blobs, fb)
        v = s.hydrodynamic_solver(np.concatenate([segs, blobs]), np.concatenate([f6[:, :3], fb]))
    np.testing.assert_allclose(vs.reshape(-1, 6)[:, :3], v[:ns], rtol=1e-6, atol=1e-7)
    assert np.all(vs.reshape(-1, 6)[:, 3:] == 0)
    np.testing.assert_allclose(vb.reshape(-1, 3), v[ns:], rtol=1e-6, atol=1e-7)
