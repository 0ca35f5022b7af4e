"""The benchmark's byte accounting (bench.py), checked on the host: the canonical words per
cell of a timestep follow the reference's iteration count (n - 1 printed for a solve ending
in loop pass n, tealeaf_2d/tea_solve.f90:543) and its CG / Chebyshev / PPCG split."""
import importlib.util

from conftest import ROOT

_spec = importlib.util.spec_from_file_location("bench", ROOT / "bench.py")
bench = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(bench)


def test_canonical_words_per_timestep():
    # CG: every loop pass is a CG iteration, 12 words per cell in 2D, 13 in 3D.
    assert bench.canonical_step_words(2, "cg", 99, 0) == 12 * 100
    assert bench.canonical_step_words(3, "cg", 647, 0) == 13 * 648
    # Chebyshev (2D): passes 1 .. n - cheby are CG, the rest Chebyshev iterations.
    assert bench.canonical_step_words(2, "chebyshev", 7219, 4085) == 12 * 3135 + 7 * 4085
    # PPCG (3D, 10 inner steps): an outer iteration is a CG iteration plus 10 inner steps of 9.
    assert bench.canonical_step_words(3, "ppcg", 1220, 370) == 13 * 851 + (13 + 90) * 370


def test_training_dt_matches_the_target_coefficients():
    # K = dt w / h^2 with h = domain / cells: a 4x coarser deck needs a 16x larger dt.
    assert abs(bench.train_dt(0.004, 128, 512) - 0.064) < 1e-15
    assert abs(bench.train_dt(0.004, 1024, 4096) - 0.064) < 1e-15
