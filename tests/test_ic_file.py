"""The initial-condition reader (cf_read_ic) on the reference's psi.dat layout; host only, no GPU."""
import numpy as np
import pytest

from cufcm_fil_b200 import _lib
from cufcm_fil_b200.cilia import read_ic


def test_reads_the_layout_the_sweep_drivers_write(tmp_path):
    # pyfile/find_periodic/newton_solver.py:52-55 writes [k, T, phases, angles] with np.savetxt(newline=" ")
    F = 5
    rng = np.random.default_rng(0)
    x = np.concatenate([[0.01, 1.0], rng.uniform(0, 2 * np.pi, F), rng.normal(0, 0.1, F)])
    p = tmp_path / "psi.dat"
    np.savetxt(p, x, newline=" ")
    h, ph, an = read_ic(p, F)
    np.testing.assert_array_equal(h, x[:2])
    np.testing.assert_array_equal(ph, x[2:2 + F])
    np.testing.assert_array_equal(an, x[2 + F:])


def test_values_beyond_the_filaments_are_ignored(tmp_path):
    # extra values after the 2 + 2F the reader needs are ignored, as filament.cpp:322-333 ignores them
    p = tmp_path / "psi.dat"
    p.write_text("0 0 " + " ".join(str(v) for v in range(10)) + "\n")
    _, ph, an = read_ic(p, 3)
    np.testing.assert_array_equal(ph, [0, 1, 2])
    np.testing.assert_array_equal(an, [3, 4, 5])


def test_short_or_missing_file_is_an_error(tmp_path):
    p = tmp_path / "psi.dat"
    p.write_text("0 0 1 2 3")
    with pytest.raises(_lib.CufilError) as ei:
        read_ic(p, 2)
    assert ei.value.code == _lib.CF_EINVAL and "2 header values" in str(ei.value)
    with pytest.raises(_lib.CufilError):
        read_ic(tmp_path / "absent.dat", 2)
