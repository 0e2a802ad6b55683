"""GPU tests of batched uneven arrays (cf_batch) through the C ABI.

A batch must give every array exactly what its own single-array run gives:
the pair work list, the dot-product chunks and the 32-row update blocks are
laid out per array, so every sum is formed in the same order and the results
are bit-identical; masking an array that stopped must not disturb the others.
Failures are injected on the host (a NaN phase), never as a device fault.
"""
import math
from pathlib import Path

import numpy as np
import pytest

from cufcm_fil_b200 import _lib, workloads
from cufcm_fil_b200.sim import WallCiliaBatch, WallCiliaSimulation

pytestmark = pytest.mark.gpu

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "reference_forcing_nseg20_sep2.6.npz")
SHARED = dict(nseg=20, seg_sep=2.6, dt=1 / 300, spring_factor=0.01, phase_refs=GOLD["fb_phase"],
              angle_refs=GOLD["fb_angle"], gmres_tol=1e-6, gmres_max_iter=350)


def array_spec(n_fil, spacing, seed):
    rng = np.random.default_rng(seed)
    nx = max(1, int(math.ceil(math.sqrt(n_fil))))
    return dict(bases=workloads.lattice_bases(n_fil, nx, spacing, 1.3),
                phase0=rng.normal(0.0, 0.05, n_fil) + 0.3 * seed, angle0=rng.normal(0.0, 0.05, n_fil))


SPECS = [(5, 20.0, 1), (12, 12.0, 2), (2, 30.0, 3), (9, 8.0, 4)]  # uneven sizes and conditioning


def run_single(spec, steps, **kw):
    with WallCiliaSimulation(**dict(SHARED, **kw), **spec) as sim:
        its, states = [], []
        for nt in range(steps):
            r = sim.step(nt)
            its.append(r.iterations)
            states.append(sim.state())
        return its, states


def test_batch_is_bit_identical_to_single_runs():
    specs = [array_spec(*s) for s in SPECS]
    steps = 4
    single = [run_single(sp, steps) for sp in specs]
    with WallCiliaBatch(specs, **SHARED) as batch:
        for nt in range(steps):
            it, rel, rc = batch.step(nt)
            assert rc == _lib.CF_OK
            st = batch.state()
            for b in range(len(specs)):
                assert it[b] == single[b][0][nt], (b, nt, it, [s[0][nt] for s in single])
                for key in ("phase", "angle", "phase_dot", "angle_dot"):
                    np.testing.assert_array_equal(st[b][key], single[b][1][nt][key])
        # arrays converge after different iteration counts (the masking path ran)
        assert len(set(int(i) for i in it)) > 1


def test_batch_solution_satisfies_each_system():
    specs = [array_spec(*s) for s in SPECS[:3]]
    with WallCiliaBatch(specs, **SHARED) as batch:
        batch.step(0)
        _, rel, _ = batch.step(1)
        assert np.all(rel <= 1e-6)
        for b, sp in enumerate(specs):
            x = batch.solution(b)
            assert x.shape == (batch.sizes[b],)
            assert np.all(np.isfinite(x))


def test_nonfinite_array_is_reported_and_isolated():
    specs = [array_spec(*s) for s in SPECS[:3]]
    with WallCiliaBatch(specs, **SHARED) as batch:
        st = batch.state()
        phase = np.concatenate([s["phase"] for s in st])
        phase[batch.n_fils[0] + 1] = np.nan  # one filament of array 1
        batch.set_state(phase=phase)
        batch.step_async(0)
        it, rel, status, rc = batch.last_solve()
        assert rc == _lib.CF_NONFINITE
        assert status[1] == 3 and status[0] == 1 and status[2] == 1, status
        st = batch.state()
    # the healthy arrays get exactly their own runs' results
    for b in (0, 2):
        ref_its, ref_states = run_single(specs[b], 1)
        assert it[b] == ref_its[0]
        np.testing.assert_array_equal(st[b]["phase_dot"], ref_states[0]["phase_dot"])


def test_autotune_keeps_state_and_picks_candidates():
    specs = [array_spec(*s) for s in SPECS]
    with WallCiliaBatch(specs, **SHARED) as batch:
        batch.step(0)
        st0 = batch.state()
        choice = batch.autotune()
        assert choice["pair_ctas_per_sm"] in (2, 4, 6, 8)
        assert choice["dots_chunk"] in (1024, 2048, 4096, 8192)
        assert choice["dots_blocks_per_sm"] in (1, 2, 4)
        assert choice["update_blocks_per_sm"] in (2, 4, 8, 16)
        assert choice["update_rows"] in (32, 64, 128, 256)
        assert batch.tuning() == choice
        st1 = batch.state()  # tuning writes scratch only
        for b in range(len(specs)):
            for key in ("phase", "phase_dot", "angle_dot"):
                np.testing.assert_array_equal(st0[b][key], st1[b][key])
        it1, _, _ = batch.step(1)
        st_tuned = batch.state()
    with WallCiliaBatch(specs, **SHARED) as ref:
        ref.step(0)
        it_ref, _, _ = ref.step(1)
        st_ref = ref.state()
    # another dot-product chunk changes the summation order only
    assert np.all(np.abs(it1 - it_ref) <= 1)
    for b in range(len(specs)):
        np.testing.assert_allclose(st_tuned[b]["phase_dot"], st_ref[b]["phase_dot"], rtol=1e-6, atol=1e-9)


def test_batch_graph_and_host_loop_agree(monkeypatch):
    specs = [array_spec(*s) for s in SPECS[:3]]
    with WallCiliaBatch(specs, **SHARED) as g:
        for nt in range(2):
            it_g, _, _ = g.step(nt)
        st_g = g.state()
    monkeypatch.setenv("CUFIL_NO_GRAPH", "1")
    with WallCiliaBatch(specs, **SHARED) as h:
        for nt in range(2):
            it_h, _, _ = h.step(nt)
        st_h = h.state()
    np.testing.assert_array_equal(it_g, it_h)
    for b in range(len(specs)):
        np.testing.assert_array_equal(st_g[b]["phase_dot"], st_h[b]["phase_dot"])


def test_batch_rejects_mismatched_shared_settings():
    specs = [array_spec(*s) for s in SPECS[:2]]
    bad = dict(SHARED, dt=1 / 200)
    with pytest.raises(_lib.CufilError):
        WallCiliaBatch([dict(specs[0], **SHARED), dict(specs[1], **bad)])
