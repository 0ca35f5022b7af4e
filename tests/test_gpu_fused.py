"""The whole-solve entry point ext_tea_leaf_solve_ (fused kernels, CUDA-graph loops with
the convergence test on the device) against the per-call ext_* sequence.

For every golden deck: per-step iteration counts, errors, exact errors and field
summaries bit-identical to the per-call path (and so to the oracle), and the final
fields the next timestep depends on (u, energy1) bit-identical, halos included."""
import numpy as np
import pytest

from conftest import SUM_COMPENSATED, golden_runs, kat_decks, port_lib, same, tea

pytestmark = pytest.mark.gpu

FIELDS = ("iterations", "error", "exact_error", "vol", "mass", "ie", "temp")
CASES = sorted(golden_runs())


@pytest.mark.parametrize("name", CASES)
def test_fused_equals_per_call(name):
    case = golden_runs()[name]
    dim = case["dim"]
    _, fused = tea.run_deck(case["deck"], dim, fused=True, summary_every_step=True)
    _, percall = tea.run_deck(case["deck"], dim, summary_every_step=True)
    assert len(fused) == len(percall)
    for a, b in zip(fused, percall):
        for k in FIELDS:
            assert same(a[k], b[k]), f"{name} step {a['step']} {k}: fused {a[k]!r} per-call {b[k]!r}"


@pytest.mark.parametrize("name", ["2d_cg_plain", "2d_chebyshev_precond", "2d_ppcg_plain", "2d_jacobi_plain",
                                  "3d_cg_precond", "3d_chebyshev_plain", "3d_ppcg_density", "3d_jacobi_plain"])
def test_fused_final_fields_equal_oracle(name):
    case = golden_runs()[name]
    dim = case["dim"]
    gpu = tea.cuda_library(dim)
    port = tea.load_library(port_lib(dim, SUM_COMPENSATED))
    tea.run_deck(case["deck"], dim, fused=True, keep_chunk=True)
    tea.run_deck(case["deck"], dim, backend=port_lib(dim, SUM_COMPENSATED), keep_chunk=True)
    try:
        g = tea.ExtChunk.__new__(tea.ExtChunk)
        c = tea.ExtChunk.__new__(tea.ExtChunk)
        for obj, lib in ((g, gpu), (c, port)):
            obj.lib, obj.dim, obj.id = lib, dim, 1
            import ctypes
            dims = (ctypes.c_int * 3)()
            assert lib.tea_chunk_dims_(ctypes.byref(ctypes.c_int(1)), dims) == 0
            obj.X, obj.Y, obj.Z = dims[0], dims[1], dims[2]
        for f in ("u", "energy1", "density", "energy0", "kx", "ky") + (("kz",) if dim == 3 else ()):
            a, b = g.read(f), c.read(f)
            assert np.array_equal(a, b), f"{name}: {f} differs at {np.argwhere(a != b)[:3].tolist()}"
    finally:
        gpu.ext_finalise_()
        port.ext_finalise_()


@pytest.mark.parametrize("dim", [2, 3])
def test_fused_known_answer(dim):
    kat = kat_decks()[str(dim)]
    s_f, r_f = tea.run_deck(kat["deck"], dim, fused=True)
    s_p, r_p = tea.run_deck(kat["deck"], dim)
    assert [r["iterations"] for r in r_f] == [r["iterations"] for r in r_p]
    assert s_f["temp"] == s_p["temp"] and s_f["kat_passed"] == 1


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("inner", [4, 5, 6, 7])
def test_fused_ppcg_inner_step_splits(dim, inner):
    """The whole-solve path runs PPCG inner steps two per pass: every step in pairs when the
    count is even (the last pair also forms the 2-norm), else an even number of pairs and
    single steps after them; r moves between r and w.  4, 5, 6 and 7 inner steps cover
    each split (even and odd numbers of pairs, with and without single steps), against
    the per-call path bit for bit."""
    spec = tea.DeckSpec(dim=dim, cells=48 if dim == 2 else 20, states=6, seed=60 + inner, solver="ppcg", end_step=2,
                        inner_steps=inner, eps=1e-15, eps_rel=1e-10, max_iters=5000, summary_frequency=1,
                        check_result=True)
    deck = tea.seeded_deck(spec)
    _, fused = tea.run_deck(deck, dim, fused=True, summary_every_step=True)
    _, percall = tea.run_deck(deck, dim, summary_every_step=True)
    assert len(fused) == len(percall) == 2
    assert all(r["cheby_steps"] > 0 for r in fused)  # the PPCG phase ran
    for a, b in zip(fused, percall):
        for k in FIELDS:
            assert same(a[k], b[k]), f"{dim}D {inner} inner steps, step {a['step']} {k}: {a[k]!r} vs {b[k]!r}"


def test_fused_chebyshev_2048_equals_per_call():
    """A 2048^2 Chebyshev timestep, fused against per-call bit for bit.  The small golden
    decks run the multi-iteration passes on few, short segments; at this size every warp
    streams a long segment under full memory load, where an asynchronous copy read before
    it has landed would show (a four-iteration pass with a miscounted copy schedule passed
    every small deck and failed here)."""
    spec = tea.DeckSpec(dim=2, cells=2048, states=16, seed=2048, solver="chebyshev", end_step=1, dt=0.004,
                        eps=1e-15, eps_rel=1e-10, max_iters=20000, presteps=30, summary_frequency=1,
                        check_result=False)
    deck = tea.seeded_deck(spec)
    sf, rf = tea.run_deck(deck, 2, fused=True, summary_every_step=True)
    sp, rp = tea.run_deck(deck, 2, summary_every_step=True)
    assert rf[0]["cheby_steps"] > 100  # the Chebyshev phase ran
    for k in FIELDS:
        assert same(rf[0][k], rp[0][k]), f"{k}: fused {rf[0][k]!r} per-call {rp[0][k]!r}"
