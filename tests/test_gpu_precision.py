"""The FP32-refined precision form of ext_tea_leaf_solve_ against the FP64 oracle.

FP32 inner solves inside FP64 defect correction -- CG for CG and Jacobi decks; for
Chebyshev and PPCG decks a first inner CG whose scalars give the eigenvalue bounds, then
FP32 Chebyshev (PPCG decks: FP32 PPCG with the deck's inner steps) -- must reach the same convergence target as the FP64 solve (tested on the
true FP64 residual), and the field summary must stay within 1e-9 relative of the FP64
oracle's (the bar the specification sets for the precision form), step by step.
"""
import pytest

from conftest import SUM_COMPENSATED, golden_runs, kat_decks, port_lib, rel, tea

pytestmark = pytest.mark.gpu

FIELD_SUMMARY_TOL = 1e-9


def _spec(dim, solver, seed):
    return tea.DeckSpec(dim=dim, cells=96 if dim == 2 else 24, states=8, seed=seed, solver=solver, end_step=4,
                        eps=1e-15, eps_rel=1e-10, max_iters=20000, summary_frequency=1, check_result=True)


@pytest.mark.parametrize("dim,solver,seed", [(2, "cg", 11), (2, "chebyshev", 12), (2, "ppcg", 13), (2, "jacobi", 14),
                                             (3, "cg", 15), (3, "ppcg", 16)])
def test_fp32_refined_matches_fp64_oracle(dim, solver, seed):
    deck = tea.seeded_deck(_spec(dim, solver, seed))
    # The FP64 reference point: the oracle solving with CG to the same relative target.
    ref_deck = deck.replace(tea.SOLVER_KEYWORDS[tea.SOLVERS[solver]], "tl_use_cg")
    _, ref = tea.run_deck(ref_deck, dim, backend=port_lib(dim, SUM_COMPENSATED), summary_every_step=True)
    _, got = tea.run_deck(deck, dim, fused=True, precision=tea.PRECISION_FP32_REFINED, summary_every_step=True)
    for a, b in zip(got, ref):
        assert a["corrections"] >= 1
        if solver in ("chebyshev", "ppcg"):
            assert a["cheby_steps"] > 0, a  # the FP32 Chebyshev / PPCG corrections ran
        if solver == "ppcg" and a["corrections"] >= 2:
            assert a["inner_solver"] == 2, a  # PPCG decks correct with FP32 PPCG
        assert a["exact_error"] < a["eps_used"], (a["step"], a["exact_error"], a["eps_used"])
        for k in ("vol", "mass", "ie", "temp"):
            assert rel(a[k], b[k]) <= FIELD_SUMMARY_TOL, (a["step"], k, a[k], b[k], rel(a[k], b[k]))


@pytest.mark.parametrize("dim", [2, 3])
def test_fp32_refined_known_answer(dim):
    kat = kat_decks()[str(dim)]
    summary, recs = tea.run_deck(kat["deck"], dim, fused=True, precision=tea.PRECISION_FP32_REFINED)
    qa = abs(100.0 * (summary["temp"] / kat["expected_temp"]) - 100.0)
    assert qa < kat["threshold_percent"], qa
    ref = golden_runs()[f"kat_{dim}d"]["ref"]
    assert rel(summary["temp"], ref["temp"]) <= FIELD_SUMMARY_TOL
