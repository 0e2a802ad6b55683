"""CPU checks of the oracle's RPY restatement (no GPU).

The grand mobility matrix of both the Swan-Brady wall blocks and the unbounded
RPY blocks is symmetric and, for non-overlapping spheres, positive definite;
the restatement of src/cilia/cuda_functions.cu:9-358 must show both.  The FP32
and FP64 builds of the same source must agree to FP32 rounding.
"""
import numpy as np
import pytest

import oracle
from cufcm_fil_b200 import workloads


def dense_matrix(x, *, wall, dof, radius=1.0, mu=1.0):
    """Columns of M by applying it to unit vectors (small systems only)."""
    n = x.shape[0]
    m = np.zeros((n * dof, n * dof))
    for col in range(n * dof):
        f = np.zeros((n, dof))
        f.flat[col] = 1.0
        m[:, col] = oracle.rpy_apply(x, x, f, wall=wall, vdof=dof, fdof=dof, self_by_index=True, at=radius,
                                     as_=radius, mu=mu).ravel()
    return m


@pytest.mark.parametrize("wall", [1, 0])
@pytest.mark.parametrize("dof", [3, 6])
def test_mobility_symmetric_positive_definite(wall, dof):
    x = workloads.vertical_lattice(2, 2, 6, spacing=6.0, base_z=2.0, seg_sep=2.2)
    m = dense_matrix(x, wall=wall, dof=dof)
    asym = np.abs(m - m.T).max() / np.abs(m).max()
    assert asym < 1e-12, asym
    eig = np.linalg.eigvalsh(0.5 * (m + m.T))
    assert eig.min() > 0.0


def test_wall_self_mobility_far_from_wall_is_stokes():
    x = np.array([[0.0, 0.0, 1e6]])
    f = np.array([[1.0, 2.0, 3.0]])
    v = oracle.rpy_apply(x, x, f, wall=1, vdof=3, fdof=3, self_by_index=True)
    np.testing.assert_allclose(v[0], f[0] / (6 * np.pi), rtol=1e-5)


def test_wall_pair_far_apart_decays():
    # Two spheres far apart above the wall: the wall image cancels the Stokeslet at large lateral
    # separation, so the pair velocity decays faster than 1/r.
    xt = np.array([[0.0, 0.0, 3.0]])
    f = np.array([[1.0, 0.0, 0.0]])
    v1 = oracle.rpy_apply(xt, np.array([[100.0, 0.0, 3.0]]), f, wall=1, vdof=3, fdof=3)
    v2 = oracle.rpy_apply(xt, np.array([[200.0, 0.0, 3.0]]), f, wall=1, vdof=3, fdof=3)
    assert abs(v2[0, 0]) < abs(v1[0, 0]) / 4


def test_unbounded_coincident_equal_spheres_is_self_mobility():
    # r = 0 enters the containment branch: A = 1/(6 pi mu a), rot-rot 1/(8 pi mu a^3).
    x = np.array([[1.0, 2.0, 3.0]])
    f = np.array([[1.0, -2.0, 0.5, 0.3, 0.2, -0.1]])
    a, mu = 1.5, 2.0
    v = oracle.rpy_apply(x, x, f, wall=0, vdof=6, fdof=6, at=a, as_=a, mu=mu)
    np.testing.assert_allclose(v[0, :3], f[0, :3] / (6 * np.pi * mu * a), rtol=1e-12)
    np.testing.assert_allclose(v[0, 3:], f[0, 3:] / (8 * np.pi * mu * a ** 3), rtol=1e-12)


@pytest.mark.parametrize("wall,dof", [(1, 3), (1, 6), (0, 3), (0, 6)])
def test_f32_build_matches_f64(wall, dof):
    x = workloads.vertical_lattice(4, 4, 20)
    f = workloads.random_forces(x.shape[0], dof, seed=7)
    v64 = oracle.rpy_apply(x, x, f, wall=wall, vdof=dof, fdof=dof, self_by_index=True)
    v32 = oracle.rpy_apply(x, x, f, wall=wall, vdof=dof, fdof=dof, self_by_index=True, dtype=np.float32)
    assert oracle.rel_l2(v32, v64) < 2e-6


def test_target_subset_matches_full_rows():
    x = workloads.vertical_lattice(4, 4, 20)
    f = workloads.random_forces(x.shape[0], 3, seed=3)
    full = oracle.rpy_apply(x, x, f, wall=1, vdof=3, fdof=3, self_by_index=True)
    rows = np.array([0, 5, 77, 319])
    sub = oracle.rpy_apply(x[rows], x, f, wall=1, vdof=3, fdof=3, self_by_index=True, t_ids=rows)
    np.testing.assert_array_equal(sub, full[rows])
