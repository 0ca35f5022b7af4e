"""Generate the golden fixtures under tests/golden/ from the reference itself.

It needs the reference's sources (``TEA_REFERENCE``, default ``/root/reference``) and
oracle/_ref built from them by ``make -C oracle ref REF=$TEA_REFERENCE``:

    python tests/golden/make_golden.py

Writes:
* ``kat_decks.json`` -- the two input decks the reference ships (tealeaf_2d/tea.in,
  tealeaf_3d/tea.in) with their known answers (tealeaf_2d/field_summary.f90:107,
  tealeaf_3d/field_summary.f90:115) and the 0.001 % threshold (:149).
* ``ref_runs.json`` -- per-step iteration counts, errors and field summaries of the
  reference's own Kokkos-OpenMP kernels (oracle/_ref, driven by the C++ driver, one
  thread so the sums are in index order) on the shipped decks and on seeded decks that
  cover every solver and option.  The GPU tests compare against these without needing
  /root/reference at run time.
"""
from __future__ import annotations

import json
import os
import pathlib
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF = pathlib.Path(os.environ.get("TEA_REFERENCE", "/root/reference"))
sys.path.insert(0, str(ROOT))

import __graft_entry__  # noqa: E402

tea = __graft_entry__.load_package()

KATS = {
    2: {"deck": REF / "tealeaf_2d" / "tea.in", "test_problem": 11, "expected": 103.46970921076068,
        "source": "tealeaf_2d/field_summary.f90:107"},
    3: {"deck": REF / "tealeaf_3d" / "tea.in", "test_problem": 11, "expected": 58.442896702081427,
        "source": "tealeaf_3d/field_summary.f90:115"},
}


def seeded_cases():
    """Small seeded decks: every solver x {plain, preconditioned, density coefficient}."""
    cases = []
    for dim, cells, states in ((2, 72, 5), (3, 22, 7)):
        for solver in ("cg", "chebyshev", "ppcg", "jacobi"):
            for variant in ("plain", "precond", "density"):
                spec = tea.DeckSpec(dim=dim, cells=cells, states=states, seed=100 + len(cases), solver=solver,
                                    end_step=3, eps=1e-15, max_iters=20000 if solver == "jacobi" else 1000,
                                    presteps=20 if dim == 3 else 30, inner_steps=8,
                                    inverse_density=(variant != "density"), preconditioner=(variant == "precond"),
                                    summary_frequency=1)
                cases.append({"name": f"{dim}d_{solver}_{variant}", "dim": dim, "deck": tea.seeded_deck(spec)})
    # A larger 2D case with the 16-state generator of the benchmark configuration.
    spec = tea.DeckSpec(dim=2, cells=256, states=16, seed=4096, solver="ppcg", end_step=2, eps=1e-15,
                        summary_frequency=1)
    cases.append({"name": "2d_ppcg_16states_256", "dim": 2, "deck": tea.seeded_deck(spec)})
    spec = tea.DeckSpec(dim=3, cells=48, states=12, seed=256, solver="cg", end_step=2, eps=1e-15,
                        summary_frequency=1)
    cases.append({"name": "3d_cg_12states_48", "dim": 3, "deck": tea.seeded_deck(spec)})
    # Non-square, ragged grids on the square domain, so dx != dy (!= dz): a kernel that
    # mixed up two extents or two cell widths would still pass every square deck above.
    for dim, shape, solver, seed in ((2, (97, 41), "cg", 900), (2, (33, 150), "chebyshev", 901),
                                     (2, (97, 41), "ppcg", 902), (2, (33, 150), "jacobi", 903),
                                     (3, (19, 11, 27), "cg", 904), (3, (29, 23, 9), "chebyshev", 905),
                                     (3, (19, 11, 27), "ppcg", 906), (3, (29, 23, 9), "jacobi", 907)):
        cases.append(_non_square(dim, shape, solver, seed, "plain"))
    # The same grids with the diagonal preconditioner and with the density coefficient.
    for dim, shape, solver, seed, variant in ((2, (97, 41), "chebyshev", 910, "precond"),
                                              (2, (33, 150), "ppcg", 911, "density"),
                                              (3, (19, 11, 27), "cg", 912, "precond"),
                                              (3, (29, 23, 9), "ppcg", 913, "precond")):
        cases.append(_non_square(dim, shape, solver, seed, variant))
    return cases


def _non_square(dim, shape, solver, seed, variant):
    spec = tea.DeckSpec(dim=dim, cells=shape[0], states=6, seed=seed, solver=solver, end_step=3, eps=1e-15,
                        max_iters=20000 if solver == "jacobi" else 1000, presteps=20, inner_steps=6,
                        inverse_density=(variant != "density"), preconditioner=(variant == "precond"),
                        summary_frequency=1)
    deck = tea.seeded_deck(spec)
    for axis, n in zip("yz", shape[1:]):
        deck = deck.replace(f"{axis}_cells={shape[0]}\n", f"{axis}_cells={n}\n")
    name = f"{dim}d_{solver}_" + "x".join(str(n) for n in shape) + ("" if variant == "plain" else f"_{variant}")
    return {"name": name, "dim": dim, "deck": deck}


def run_ref(dim: int, deck: str, threads: int, keep_extra=()) -> dict:
    lib = ROOT / "oracle" / "_ref" / f"libtea_ref{dim}d.so"
    tmp = HERE / f"_tmp_{os.getpid()}"
    tmp.mkdir(exist_ok=True)
    (tmp / "tea.in").write_text(deck)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="false")
    subprocess.run([str(tea.tea_leaf_exe()), "--dim", str(dim), "--backend", str(lib), "--quiet", "--no-out",
                    "--summary-every-step", "--json", str(tmp / "out.json"), str(tmp / "tea.in")],
                   check=True, env=env, capture_output=True)
    out = json.loads((tmp / "out.json").read_text())
    for p in tmp.iterdir():
        p.unlink()
    tmp.rmdir()
    keep = ("step", "iterations", "error", "exact_error", "vol", "mass", "ie", "temp", "switch_step", "est_itc",
            *keep_extra)
    return {"temp": out["temp"], "qa_diff": out["qa_diff"], "kat_passed": out["kat_passed"],
            "records": [{k: r[k] for k in keep} for r in out["records"]]}


def main():
    kat = {}
    for dim, k in KATS.items():
        kat[str(dim)] = {"deck": k["deck"].read_text(), "test_problem": k["test_problem"],
                         "expected_temp": k["expected"], "threshold_percent": 0.001, "source": k["source"]}
    (HERE / "kat_decks.json").write_text(json.dumps(kat, indent=1) + "\n")
    # A case whose deck is unchanged keeps its recorded run (the reference is deterministic
    # at one thread); new or changed decks are run.
    old = json.loads((HERE / "ref_runs.json").read_text()) if (HERE / "ref_runs.json").exists() else {}

    def ref_of(name, dim, deck):
        if name in old and old[name]["deck"] == deck:
            return old[name]["ref"]
        return run_ref(dim, deck, 1)

    runs = {}
    for dim in (2, 3):
        runs[f"kat_{dim}d"] = {"dim": dim, "deck": kat[str(dim)]["deck"],
                               "ref": ref_of(f"kat_{dim}d", dim, kat[str(dim)]["deck"])}
    for case in seeded_cases():
        runs[case["name"]] = {"dim": case["dim"], "deck": case["deck"],
                              "ref": ref_of(case["name"], case["dim"], case["deck"])}
        print(case["name"], [r["iterations"] for r in runs[case["name"]]["ref"]["records"]], flush=True)
    (HERE / "ref_runs.json").write_text(json.dumps(runs, indent=1) + "\n")


if __name__ == "__main__":
    main()
