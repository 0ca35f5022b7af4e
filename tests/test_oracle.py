"""The oracle (oracle/tea_oracle.c, the C restatement of the reference's ext_* kernels)
pinned against the reference's own outputs.

* Bit-for-bit against fixtures produced by the reference's Kokkos-OpenMP kernels
  (tests/golden/ref_runs.json, made by tests/golden/make_golden.py from oracle/_ref),
  with the oracle's sums in the reference's single-thread order.
* Against the reference's known answers (KATs) within its own 0.001 % threshold
  (tealeaf_2d/field_summary.f90:149).
* Live against oracle/_ref when it has been built here.
"""
import math
import os
import pathlib
import subprocess
import json

import pytest

from conftest import (PORT, REFLIB, SUM_COMPENSATED, SUM_SEQUENTIAL, golden_runs, kat_decks, port_lib, rel,
                      same, tea)

FIELDS = ("iterations", "error", "exact_error", "vol", "mass", "ie", "temp")
# The two shipped known-answer decks run ~4000 and ~2200 CG iterations; they are
# covered by test_port_known_answers and excluded from the bitwise sweep.
SWEEP = sorted(k for k in golden_runs() if not k.startswith("kat_"))


@pytest.mark.parametrize("name", SWEEP)
def test_port_bitwise_equals_reference_fixture(name):
    case = golden_runs()[name]
    dim = case["dim"]
    _, recs = tea.run_deck(case["deck"], dim, backend=port_lib(dim, SUM_SEQUENTIAL), summary_every_step=True)
    ref = case["ref"]["records"]
    assert len(recs) == len(ref)
    for a, b in zip(recs, ref):
        for k in FIELDS:
            assert same(a[k], b[k]), f"{name} step {b['step']} {k}: port {a[k]!r} reference {b[k]!r}"


@pytest.mark.parametrize("dim", [2, 3])
def test_port_known_answers(dim):
    kat = kat_decks()[str(dim)]
    summary, recs = tea.run_deck(kat["deck"], dim, backend=port_lib(dim, SUM_SEQUENTIAL))
    qa = abs(100.0 * (summary["temp"] / kat["expected_temp"]) - 100.0)
    assert summary["kat_available"] == 1
    assert qa < kat["threshold_percent"], f"known answer missed by {qa} %"
    ref = golden_runs()[f"kat_{dim}d"]["ref"]
    assert [r["iterations"] for r in recs] == [r["iterations"] for r in ref["records"]]
    assert summary["temp"] == ref["temp"]


@pytest.mark.parametrize("name", ["2d_cg_plain", "2d_chebyshev_plain", "2d_ppcg_plain", "3d_cg_plain",
                                  "3d_ppcg_plain", "2d_ppcg_16states_256"])
def test_compensated_sums_stay_within_tolerance(name):
    """The CUDA library sums in double-double; against the reference's plain sums the
    per-step iteration counts agree to +-1 and the field summary to 1e-10 relative
    (the parity bar of the specification)."""
    case = golden_runs()[name]
    dim = case["dim"]
    _, recs = tea.run_deck(case["deck"], dim, backend=port_lib(dim, SUM_COMPENSATED), summary_every_step=True)
    for a, b in zip(recs, case["ref"]["records"]):
        assert abs(a["iterations"] - b["iterations"]) <= 1
        for k in ("vol", "mass", "ie", "temp"):
            assert rel(a[k], b[k]) <= 1e-10, (name, k, a[k], b[k])


@pytest.mark.skipif(not REFLIB[2].exists(), reason="oracle/_ref not built (needs the reference sources)")
def test_port_bitwise_equals_live_reference(tmp_path):
    """One fresh seeded deck per dimension, run live through the compiled reference."""
    for dim, cells in ((2, 50), (3, 14)):
        spec = tea.DeckSpec(dim=dim, cells=cells, states=6, seed=999 + dim, solver="ppcg", end_step=2,
                            eps=1e-14, presteps=15, inner_steps=5, summary_frequency=1)
        deck = tea.seeded_deck(spec)
        (tmp_path / "tea.in").write_text(deck)
        env = dict(os.environ, OMP_NUM_THREADS="1")
        subprocess.run([str(tea.tea_leaf_exe()), "--dim", str(dim), "--backend", str(REFLIB[dim]), "--quiet", "--no-out",
                        "--summary-every-step", "--json", str(tmp_path / "r.json"), str(tmp_path / "tea.in")],
                       check=True, env=env, capture_output=True)
        ref = json.loads((tmp_path / "r.json").read_text())["records"]
        _, recs = tea.run_deck(deck, dim, backend=port_lib(dim, SUM_SEQUENTIAL), summary_every_step=True)
        for a, b in zip(recs, ref):
            for k in FIELDS:
                assert same(a[k], b[k]), (dim, k, a[k], b[k])


TINY = [(2, (7, 5), "cg"), (2, (1, 9), "cg"), (2, (9, 1), "ppcg"), (2, (2, 2), "chebyshev"), (2, (3, 1), "jacobi"),
        (3, (8, 8, 8), "cg"), (3, (3, 4, 5), "ppcg"), (3, (1, 6, 2), "chebyshev"), (3, (2, 1, 3), "jacobi")]


@pytest.mark.skipif(not REFLIB[2].exists(), reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("dim,shape,solver", TINY)
def test_port_bitwise_equals_live_reference_on_tiny_grids(tmp_path, dim, shape, solver):
    """Grids down to one cell wide in an axis, against the compiled reference."""
    spec = tea.DeckSpec(dim=dim, cells=shape[0], states=4, seed=50, solver=solver, end_step=2, eps=1e-15,
                        max_iters=2000, presteps=5, inner_steps=4, summary_frequency=1)
    deck = tea.seeded_deck(spec)
    for axis, n in zip("yz", shape[1:]):
        deck = deck.replace(f"{axis}_cells={shape[0]}\n", f"{axis}_cells={n}\n")
    (tmp_path / "tea.in").write_text(deck)
    subprocess.run([str(tea.tea_leaf_exe()), "--dim", str(dim), "--backend", str(REFLIB[dim]), "--quiet", "--no-out",
                    "--summary-every-step", "--json", str(tmp_path / "r.json"), str(tmp_path / "tea.in")],
                   check=True, env=dict(os.environ, OMP_NUM_THREADS="1"), capture_output=True)
    ref = json.loads((tmp_path / "r.json").read_text())["records"]
    _, recs = tea.run_deck(deck, dim, backend=port_lib(dim, SUM_SEQUENTIAL), summary_every_step=True)
    assert len(recs) == len(ref) == 2
    for a, b in zip(recs, ref):
        for k in FIELDS:
            assert same(a[k], b[k]), (shape, solver, b["step"], k, a[k], b[k])


def test_port_bitwise_equals_reference_at_c1_size():
    """The 2D 512^2 configuration (6 seeded states, CG, eps 1e-15, 10 timesteps; about 11,000
    iterations) at its stated size: the port, with its sums in the reference's single-thread
    order, reproduces every per-step iteration count, error, exact error and field summary
    of the reference's own kernels (tests/golden/ref_large.json, recorded at one thread)."""
    case = json.loads((pathlib.Path(__file__).parent / "golden" / "ref_large.json").read_text())["c1_2d512_cg"]
    assert case["threads"] == 1
    _, recs = tea.run_deck(case["deck"], 2, backend=port_lib(2, SUM_SEQUENTIAL), summary_every_step=True)
    ref = case["ref"]["records"]
    assert len(recs) == len(ref) == 10
    for a, b in zip(recs, ref):
        for k in FIELDS:
            assert same(a[k], b[k]), f"step {b['step']} {k}: port {a[k]!r} reference {b[k]!r}"
