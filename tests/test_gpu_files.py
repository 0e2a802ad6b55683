"""The drop-in executable and the reference's data files, against the reference's own writers.

cufcm_fil_b200.cilia reads input/globals.ini, the forcing tables and the
initial-condition file as the reference's executable does and appends the
reference's data files through cf_sim_write_data.  The reference's own step
code, built for the host in FP64 with its own writers (oracle/_ref/ref_step_*,
"write" mode), runs the same 21 steps; both sets of files must have the same
lines, the same number of fields per line, the same step labels, and values
equal to the stated tolerances (the engine's pair sums are FP32).
"""
import io
from pathlib import Path

import numpy as np
import pytest

from oracle import ref_step
from cufcm_fil_b200 import cilia, workloads

pytestmark = pytest.mark.gpu

HERE = Path(__file__).resolve().parent
GOLD = np.load(HERE / "golden" / "reference_forcing_nseg20_sep2.6.npz")
TIPS = np.load(HERE / "golden" / "ref_tips_16x16_80a.npz")


def _setup(tmp, F, nx, spacing, phase0, angle0, steps):
    f = tmp / "input" / "forcing"
    f.mkdir(parents=True)
    tag = "NSEG=20_SEP=2.600000.dat"
    for k in ("phase", "angle"):
        v = GOLD["fb_" + k]
        (f / f"fulford_and_blake_reference_{k}_generalised_forces_{tag}").write_text(
            f"{v.size} " + " ".join(repr(float(x)) for x in v))
    s = TIPS["s_table"]
    (f / f"fulford_and_blake_reference_s_values_{tag}").write_text(
        f"{s.shape[0]} {s.shape[1]} " + " ".join(repr(float(x)) for x in s.ravel()))
    np.savetxt(tmp / "psi.dat", np.concatenate([[0.01, 1.0], phase0, angle0]), newline=" ")
    (tmp / "input" / "globals.ini").write_text(
        "[Parameters]\nnswim=1.0\nnseg=20.0\nnfil=%d.0\nnblob=0.0\nspring_factor=0.01\nseg_sep=2.6\nperiod=1.0\n"
        "sim_length=%r\nfil_spacing=%r\nfil_x_dim=%d.0\nfene_model=0.0\nforce_noise_mag=0.0\nomega_spread=0.0\n"
        "[Filenames]\nsimulation_dir=out/\nsimulation_file=sim\nsimulation_icstate_name=psi.dat\n"
        % (F, (steps - 1) / 300 + 1e-9, spacing, nx))


def test_drop_in_executable_writes_the_reference_files(tmp_path, monkeypatch):
    F, nx, spacing, steps = 4, 2, 40.0, 21
    rng = np.random.default_rng(21)
    phase0, angle0 = rng.uniform(0, 2 * np.pi, F), rng.normal(0, 0.05, F)
    _setup(tmp_path, F, nx, spacing, phase0, angle0, steps)
    monkeypatch.chdir(tmp_path)
    log = io.StringIO()
    prefix = cilia.run("input/globals.ini", tol=1e-6, precond="block", log=log)
    assert f"Completed step {steps}/{steps}" in log.getvalue()
    ref = ref_step.run(nfil=F, fil_x_dim=nx, spacing=spacing, phase0=phase0, angle0=angle0, steps=steps,
                       phase_refs=GOLD["fb_phase"], angle_refs=GOLD["fb_angle"], s_table=TIPS["s_table"],
                       write=True)
    L = 2.6 * 19
    tol = {"_true_states.dat": 2e-6, "_seg_states.dat": 2e-5 * L, "_body_states.dat": 0.0,
           "_seg_vels.dat": 1e-4, "_seg_forces.dat": 1e-4}
    for suffix, atol in tol.items():
        ours = (tmp_path / (prefix + suffix)).read_text().strip("\n").split("\n")
        theirs = ref.files[suffix].strip("\n").split("\n")
        assert len(ours) == len(theirs) == 3, suffix        # steps 0, 10, 20
        for a, b in zip(ours, theirs):
            ta, tb = a.split(), b.split()
            assert len(ta) == len(tb) and ta[0] == tb[0], suffix
            va, vb = np.array(ta[1:], float), np.array(tb[1:], float)
            scale = max(1.0, np.abs(vb).max()) if suffix in ("_seg_vels.dat", "_seg_forces.dat") else 1.0
            assert np.abs(va - vb).max() <= atol * scale, (suffix, np.abs(va - vb).max())
    # what pyfile/find_periodic reads back (newton_solver.py:73-86)
    state = np.loadtxt(tmp_path / (prefix + "_true_states.dat"))[-1][2:]
    assert state.shape == (2 * F,)
    refs = np.loadtxt(tmp_path / (prefix + "_fil_references.dat"))
    np.testing.assert_allclose(refs.reshape(F, 3), workloads.lattice_bases(F, nx, spacing, 1.3))
    assert "NFIL" in (tmp_path / (prefix + ".par")).read_text()
