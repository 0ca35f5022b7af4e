"""Generate tests/golden/ref_large.json: the reference's own runs of the benchmark
configurations at their stated sizes.

The reference's Kokkos-OpenMP kernels (oracle/_ref, built by ``make -C oracle ref``
from the reference's sources) are driven by the C++ driver, as in make_golden.py, on:

* ``c1_2d512_cg``      -- 2D 512^2, 6 seeded states, CG, eps 1e-15, 10 timesteps (one thread);
* ``c2_2d4096_cheby``  -- 2D 4096^2, 16 seeded states, Chebyshev (30 CG presteps), relative
                          residual 1e-10, 30 timesteps: the benchmark deck, so the counts
                          also scale the benchmark's reference arm to whole timesteps;
* ``c2_2d4096_ppcg``   -- the same layout with PPCG (10 inner steps), timestep 1, relative
                          residual 1e-8 (FP64 PPCG stalls near 2e-9 on this deck);
* ``c3_3d256_cg`` / ``c3_3d256_ppcg`` -- 3D 256^3, 12 seeded states, timestep 1, relative
                          residual 1e-10.

Each case records the thread count: the reference's sums run in per-thread order, so
counts at another thread count may differ by the rounding of a few sums.  For the 512^2
case, whose absolute eps 1e-15 sits at the rounding floor of sum r^2, the per-step counts at
2, 4 and 8 threads are recorded too (``iterations_by_threads``).  Cases already
in the file with the same deck and threads are kept.  The larger cases take the CPU from
minutes (512^2, 256^3) to an hour or more (30 timesteps at 4096^2).

    python tests/golden/make_golden_large.py [case ...]
"""
from __future__ import annotations

import json
import pathlib
import sys
import time

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

import make_golden  # noqa: E402

tea = make_golden.tea
OUT = HERE / "ref_large.json"


def cases():
    D = tea.DeckSpec
    return {
        "c1_2d512_cg": (2, 1, D(dim=2, cells=512, states=6, seed=512, solver="cg", end_step=10, eps=1e-15,
                                max_iters=10000, check_result=True, summary_frequency=1)),
        "c3_3d256_cg": (3, 8, D(dim=3, cells=256, states=12, seed=256, solver="cg", end_step=1, eps=1e-15,
                                eps_rel=1e-10, max_iters=20000, check_result=True, summary_frequency=1)),
        "c3_3d256_ppcg": (3, 8, D(dim=3, cells=256, states=12, seed=256, solver="ppcg", end_step=1, eps=1e-15,
                                  eps_rel=1e-10, max_iters=20000, presteps=30, inner_steps=10, check_result=True,
                                  summary_frequency=1)),
        "c2_2d4096_ppcg": (2, 8, D(dim=2, cells=4096, states=16, seed=4096, solver="ppcg", end_step=1, eps=1e-15,
                                   eps_rel=1e-8, max_iters=12000, presteps=30, inner_steps=10, check_result=True,
                                   summary_frequency=1)),
        "c2_2d4096_cheby": (2, 8, D(dim=2, cells=4096, states=16, seed=4096, solver="chebyshev", end_step=30,
                                    eps=1e-15, eps_rel=1e-10, max_iters=20000, presteps=30, check_result=False,
                                    summary_frequency=1)),
    }


VARIANTS = {"c1_2d512_cg": (2, 4, 8)}


def main():
    want = sys.argv[1:]
    old = json.loads(OUT.read_text()) if OUT.exists() else {}
    for name, (dim, threads, spec) in cases().items():
        if want and name not in want:
            continue
        deck = tea.seeded_deck(spec)
        variants = VARIANTS.get(name, ())
        if (name in old and old[name]["deck"] == deck and old[name]["threads"] == threads
                and all(str(v) in old[name].get("iterations_by_threads", {}) for v in variants)):
            continue
        t0 = time.time()
        ref = make_golden.run_ref(dim, deck, threads, keep_extra=("cheby_steps", "solve_seconds"))
        old[name] = {"dim": dim, "threads": threads, "deck": deck, "ref": ref,
                     "wall_seconds": round(time.time() - t0, 1)}
        if variants:
            old[name]["iterations_by_threads"] = {
                str(v): [r["iterations"] for r in make_golden.run_ref(dim, deck, v)["records"]] for v in variants}
        OUT.write_text(json.dumps(old, indent=1) + "\n")
        print(name, f"{time.time() - t0:.0f} s", [r["iterations"] for r in ref["records"]], flush=True)


if __name__ == "__main__":
    main()
