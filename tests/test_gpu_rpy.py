"""GPU parity of the RPY block products through the C ABI.

Each case checks libcufil.so against
  * the FP64 oracle (restatement of src/cilia/cuda_functions.cu:9-757):
    relative L2 <= 1e-5, the tolerance of the mobility contract;
  * the reference's own CUDA kernels (oracle/_ref, built from the reference
    sources) on the same FP32 inputs: relative L2 <= 1e-5.
Full-size cases use size-independent properties (linearity, symmetry of the
grand mobility) plus oracle rows sampled at random.
"""
import numpy as np
import pytest

import oracle
from cufcm_fil_b200 import RpyMobilitySolver, workloads
from tests import refkernels

pytestmark = pytest.mark.gpu

TOL = 1e-5


def seg_inputs(n_x, n_y, nseg, dof, seed, spacing=20.0):
    x = workloads.vertical_lattice(n_x, n_y, nseg, spacing=spacing)
    f6 = np.zeros((x.shape[0], 6))
    f6[:, :dof] = workloads.random_forces(x.shape[0], dof, seed)
    return x.astype(np.float32), f6.astype(np.float32)


@pytest.mark.parametrize("wall", [True, False])
@pytest.mark.parametrize("dof", [3, 6])
def test_plain_matvec_320_vs_fp64_oracle_and_reference(cuda, wall, dof):
    # 16 vertical filaments x 20 segments on a 4x4 lattice of spacing 20 above the wall.
    x, f = seg_inputs(4, 4, 20, dof, seed=12345)
    with RpyMobilitySolver(x.shape[0], 0, wall=wall, seg_dof=dof) as mob:
        v, _ = mob.apply(x, f)
    v64, _ = oracle.mobility_full(x.astype(np.float64), f.astype(np.float64), wall=wall, seg_dof=dof)
    assert oracle.rel_l2(v, v64) <= TOL
    var = refkernels.variant_name(wall, dof)
    if refkernels.available(var):
        vref, _ = refkernels.full_mobility(cuda, var, x, f)
        assert oracle.rel_l2(v, vref) <= TOL
        assert oracle.rel_l2(vref, v64) <= 1e-4  # the reference's plain FP32 sum, for the record


@pytest.mark.parametrize("dof", [3, 6])
def test_unbounded_segments_and_blobs_all_blocks(cuda, dof):
    # cilia on a sphere-like shell + body blobs on a Fibonacci sphere, unequal radii
    rng = np.random.default_rng(5)
    xb = workloads.fibonacci_sphere(700, 20.0)
    dirs = workloads.fibonacci_sphere(30, 1.0)
    xs = np.concatenate([dirs * (21.5 + 2.2 * k) for k in range(10)])
    fs = np.zeros((xs.shape[0], 6))
    fs[:, :dof] = rng.standard_normal((xs.shape[0], dof))
    fb = rng.standard_normal((xb.shape[0], 3))
    args = dict(wall=False, seg_dof=dof, seg_radius=1.0, blob_radius=0.8, mu=1.0)
    with RpyMobilitySolver(xs.shape[0], xb.shape[0], wall=False, seg_dof=dof, seg_radius=1.0,
                           blob_radius=0.8) as mob:
        vs, vb = mob.apply(xs, fs, xb, fb)
    vs64, vb64 = oracle.mobility_full(xs, fs, xb, fb, **args)
    assert oracle.rel_l2(vs, vs64) <= TOL
    assert oracle.rel_l2(vb, vb64) <= TOL


def test_unbounded_equal_radii_matches_reference_cross_blocks(cuda):
    # The reference's unbounded build uses RSEG = RBLOB = 1 (config.hpp), so compare with radius 1.
    rng = np.random.default_rng(9)
    xb = workloads.fibonacci_sphere(500, 15.0)
    xs = np.concatenate([workloads.fibonacci_sphere(40, 1.0) * (16.5 + 2.2 * k) for k in range(8)])
    for dof in (3, 6):
        fs = np.zeros((xs.shape[0], 6), np.float32)
        fs[:, :dof] = rng.standard_normal((xs.shape[0], dof))
        fb = rng.standard_normal((xb.shape[0], 3)).astype(np.float32)
        with RpyMobilitySolver(xs.shape[0], xb.shape[0], wall=False, seg_dof=dof) as mob:
            vs, vb = mob.apply(xs, fs, xb, fb)
        var = refkernels.variant_name(False, dof)
        if not refkernels.available(var):
            pytest.skip("reference kernels not built")
        vs_r, vb_r = refkernels.full_mobility(cuda, var, xs.astype(np.float32), fs, xb.astype(np.float32), fb)
        assert oracle.rel_l2(vs, vs_r) <= TOL
        assert oracle.rel_l2(vb, vb_r) <= TOL


@pytest.mark.parametrize("n_fil,nseg", [(1, 1), (1, 20), (3, 7), (17, 13)])
def test_ragged_sizes(cuda, n_fil, nseg):
    x = workloads.vertical_lattice(n_fil, 1, nseg).astype(np.float32)
    f = np.zeros((x.shape[0], 6), np.float32)
    f[:, :3] = workloads.random_forces(x.shape[0], 3, seed=n_fil * 100 + nseg)
    with RpyMobilitySolver(x.shape[0], 0, wall=True, seg_dof=3) as mob:
        v, _ = mob.apply(x, f)
    v64, _ = oracle.mobility_full(x, f, wall=True, seg_dof=3)
    assert oracle.rel_l2(v, v64) <= TOL
    assert np.all(v.reshape(-1, 6)[:, 3:] == 0.0)  # prescribed segments: angular slots written as 0


@pytest.mark.parametrize("n_side,dof", [(16, 3), (32, 3), (16, 6)])
def test_full_size_rows_linearity_symmetry(cuda, n_side, dof):
    # 256 / 1024 cilia x 20 segments (5120 / 20480 segments) on a spacing-20 wall lattice.
    x, f = seg_inputs(n_side, n_side, 20, dof, seed=1)
    _, g = seg_inputs(n_side, n_side, 20, dof, seed=2)
    n = x.shape[0]
    with RpyMobilitySolver(n, 0, wall=True, seg_dof=dof) as mob:
        vf, _ = mob.apply(x, f)
        vg, _ = mob.apply(x, g)
        vfg, _ = mob.apply(x, 2.0 * f - 0.5 * g)
    # sampled rows against the FP64 oracle
    rows = np.random.default_rng(0).choice(n, 96, replace=False)
    vrows, _ = oracle.mobility_full(x, f, wall=True, seg_dof=dof, seg_targets=rows)
    got = vf.reshape(n, 6)[rows]
    assert oracle.rel_l2(got, vrows.reshape(-1, 6)) <= TOL
    # linearity
    assert oracle.rel_l2(vfg, 2.0 * vf.astype(np.float64) - 0.5 * vg) <= 1e-5
    # symmetry of the grand mobility: <g, M f> = <f, M g>
    k = dof
    a = np.dot(g[:, :k].astype(np.float64).ravel(), vf.reshape(n, 6)[:, :k].astype(np.float64).ravel())
    b = np.dot(f[:, :k].astype(np.float64).ravel(), vg.reshape(n, 6)[:, :k].astype(np.float64).ravel())
    assert abs(a - b) <= 1e-5 * max(abs(a), abs(b))


def test_device_path_equals_host_path(cuda):
    torch = cuda
    x, f = seg_inputs(8, 8, 20, 3, seed=4)
    n = x.shape[0]
    with RpyMobilitySolver(n, 0, wall=True, seg_dof=3) as mob:
        vh, _ = mob.apply(x, f)
        xd = torch.as_tensor(x.ravel(), device="cuda")
        fd = torch.as_tensor(f.ravel(), device="cuda")
        vd = torch.empty(6 * n, device="cuda")
        s = torch.cuda.current_stream()
        mob.apply_device(xd, fd, vd, stream=s)
        s.synchronize()
    np.testing.assert_array_equal(vd.cpu().numpy(), vh)


def test_individual_blocks_follow_reference_write_semantics(cuda):
    # evaluate_segment_segment writes, evaluate_segment_blob accumulates (Mss_mult / Msb_mult).
    rng = np.random.default_rng(3)
    xs = workloads.vertical_lattice(3, 3, 10).astype(np.float32)
    xs[:, 2] += 30.0
    xb = workloads.fibonacci_sphere(200, 10.0, centre=(0, 0, 5.0)).astype(np.float32)
    mob = RpyMobilitySolver(xs.shape[0], xb.shape[0], wall=False, seg_dof=3)
    mob.x_segs_host[:] = xs.ravel()
    mob.x_blobs_host[:] = xb.ravel()
    mob.f_segs_host[:] = rng.standard_normal(mob.f_segs_host.size)
    mob.f_blobs_host[:] = rng.standard_normal(mob.f_blobs_host.size)
    for fn in ("copy_segment_positions_to_device", "copy_blob_positions_to_device",
               "copy_segment_forces_to_device", "copy_blob_forces_to_device"):
        getattr(mob, fn)()
    mob.evaluate_segment_segment_mobility()
    mob.copy_segment_velocities_to_host()
    v_ss = mob.v_segs_host.copy()
    mob.evaluate_segment_blob_mobility()
    mob.copy_segment_velocities_to_host()
    v_total = mob.v_segs_host.copy()
    mob.evaluate_segment_segment_mobility()
    mob.copy_segment_velocities_to_host()
    np.testing.assert_array_equal(mob.v_segs_host, v_ss)
    vs64, _ = oracle.mobility_full(xs, mob.f_segs_host, xb, mob.f_blobs_host, wall=False, seg_dof=3)
    assert oracle.rel_l2(v_total, vs64) <= TOL
    mob.finalise()
