"""Host logic of the C++ driver: tea.in semantics of the reference's parser and
read_input, and the switch-time scalar algorithms (eigenvalues, Chebyshev coefficients).
Runs on the CPU against the oracle backend."""
import ctypes
import os

import numpy as np
import pytest

from conftest import SUM_SEQUENTIAL, port_lib, tea

BASE = """*tea
state 1 density=100.0 energy=0.0001
state 2 density=0.1 energy=25.0 geometry=rectangle xmin=0.0 xmax=1.0 ymin=1.0 ymax=2.0
x_cells=24
y_cells=20
xmin=0.0
ymin=0.0
xmax=10.0
ymax=10.0
tl_use_cg
{extra}
*endtea
"""


def run(extra="", **kw):
    return tea.run_deck(BASE.format(extra=extra), 2, backend=port_lib(2, SUM_SEQUENTIAL), **kw)


def test_defaults_use_single_precision_literals():
    # read_input.f90:49,51: dtinit=0.1 and eps=1.0e-10 are default-real literals.
    summary, recs = run("end_step=2")
    assert recs[0]["dt"] == float(np.float32(0.1))
    assert recs[0]["eps_used"] == float(np.float32(1.0e-10))
    assert summary["steps"] == 2


def test_end_time_stops_the_run():
    # diffuse.f90:89: stop when time + g_small > end_time.  g_small (1e-16) is below half
    # an ulp of 1.0, so time == end_time does not stop the run: 0.25 x 5 steps.
    summary, recs = run("initial_timestep=0.25\nend_time=1.0")
    assert summary["steps"] == 5
    summary, recs = run("initial_timestep=0.3\nend_time=1.0")
    assert summary["steps"] == 4


def test_parser_comments_case_and_separators():
    a, ra = run("end_step=2\ninitial_timestep=0.004")
    b, rb = run("END_STEP 2 ! a comment\nInitial_Timestep,0.004 ; another")
    assert [r["iterations"] for r in ra] == [r["iterations"] for r in rb]
    assert a["temp"] == b["temp"]


def test_value_on_the_next_line_is_read():
    # parse_getword(.TRUE.) wraps to the next line for a missing value.
    a, _ = run("end_step\n2\ninitial_timestep=0.004")
    assert a["steps"] == 2


def test_relative_target_sets_eps_from_b():
    _, recs = run("end_step=1\ninitial_timestep=0.004\ntl_eps_rel=1e-10")
    assert recs[0]["eps_used"] > 0 and recs[0]["eps_used"] != float(np.float32(1e-10))


def test_missing_states_is_an_error():
    with pytest.raises(RuntimeError, match="No states"):
        tea.run_deck("*tea\nx_cells=4\n*endtea\n", 2, backend=port_lib(2, SUM_SEQUENTIAL))


def _drv():
    lib = tea.driver()
    lib.tea_calc_eigenvalues_c.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                           ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                           ctypes.POINTER(ctypes.c_double)]
    lib.tea_tridiag_extremes_c.argtypes = lib.tea_calc_eigenvalues_c.argtypes
    lib.tea_calc_ch_coefs_c.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                        ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                        ctypes.c_int]
    return lib


@pytest.mark.parametrize("n,seed", [(5, 0), (20, 1), (30, 2), (64, 3)])
def test_eigenvalues_match_dense_solver(n, seed):
    """The Lanczos tridiagonal of tea_leaf_cheby.f90:285-332 solved by the restated tqli
    agrees with LAPACK on the same matrix."""
    rng = np.random.default_rng(seed)
    alphas = rng.uniform(0.2, 2.0, n)
    betas = rng.uniform(0.01, 0.9, n)
    lo, hi = ctypes.c_double(), ctypes.c_double()
    P = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    info = _drv().tea_calc_eigenvalues_c(P(alphas), P(betas), n, ctypes.byref(lo), ctypes.byref(hi))
    assert info == 0
    d = np.array([1 / alphas[k] + (betas[k - 1] / alphas[k - 1] if k else 0.0) for k in range(n)])
    e = np.array([np.sqrt(betas[k]) / alphas[k] for k in range(n - 1)])
    ev = np.linalg.eigvalsh(np.diag(d) + np.diag(e, 1) + np.diag(e, -1))
    assert abs(lo.value - ev[0]) <= 1e-12 * abs(ev[-1])
    assert abs(hi.value - ev[-1]) <= 1e-12 * abs(ev[-1])


@pytest.mark.parametrize("n,seed", [(1, 4), (7, 5), (64, 6), (1500, 7)])
def test_tridiagonal_extremes_by_bisection(n, seed):
    """The Sturm-bisection extremes (used while FP64 CG presteps run in the FP32-refined
    form) agree with a dense solver on the same Lanczos tridiagonal."""
    rng = np.random.default_rng(seed)
    alphas = rng.uniform(0.2, 2.0, n)
    betas = rng.uniform(0.01, 0.9, n)
    lo, hi = ctypes.c_double(), ctypes.c_double()
    P = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert _drv().tea_tridiag_extremes_c(P(alphas), P(betas), n, ctypes.byref(lo), ctypes.byref(hi)) == 0
    d = np.array([1 / alphas[k] + (betas[k - 1] / alphas[k - 1] if k else 0.0) for k in range(n)])
    e = np.array([np.sqrt(betas[k]) / alphas[k] for k in range(n - 1)])
    ev = np.linalg.eigvalsh(np.diag(d) + np.diag(e, 1) + np.diag(e, -1))
    assert abs(lo.value - ev[0]) <= 1e-11 * abs(ev[-1])
    assert abs(hi.value - ev[-1]) <= 1e-11 * abs(ev[-1])


def test_chebyshev_coefficients_recurrence():
    n = 40
    al = np.zeros(n)
    be = np.zeros(n)
    th = ctypes.c_double()
    P = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    _drv().tea_calc_ch_coefs_c(P(al), P(be), 0.05, 3.9, ctypes.byref(th), n)
    theta = (3.9 + 0.05) / 2
    delta = (3.9 - 0.05) / 2
    sigma = theta / delta
    rho_old = 1.0 / sigma
    for k in range(n):
        rho_new = 1.0 / (2.0 * sigma - rho_old)
        assert al[k] == rho_new * rho_old
        assert be[k] == 2.0 * rho_new / delta
        rho_old = rho_new
    assert th.value == theta


@pytest.mark.parametrize("dim", [2, 3])
def test_default_deck_when_none_exists(tmp_path, dim):
    """initialise.f90:69-97: with no input deck the reference writes its default one
    (10 x 10 [x 2] cells, five states, Jacobi, test_problem 1) and runs it; the tea_leaf
    executable does the same.  Against the compiled reference (when built) on that deck,
    every per-step record is identical."""
    import json
    import subprocess

    from conftest import PORT, REFLIB

    runs = {}
    for name, lib in (("port", PORT[dim]), ("ref", REFLIB[dim])):
        if name == "ref" and not lib.exists():
            continue
        d = tmp_path / name
        d.mkdir()
        subprocess.run([str(tea.tea_leaf_exe()), "--dim", str(dim), "--backend", str(lib), "--quiet",
                        "--summary-every-step", "--json", "out.json"], cwd=d, check=True, capture_output=True,
                       env=dict(os.environ, OMP_NUM_THREADS="1"))
        deck = (d / "tea.in").read_text().splitlines()
        assert deck[0] == "*tea" and deck[-1] == "*endtea"
        assert " tl_use_jacobi" in deck and " test_problem 1" in deck
        assert (" z_cells=2" in deck) == (dim == 3)
        runs[name] = json.loads((d / "out.json").read_text())
        assert runs[name]["steps"] == 10 and runs[name]["test_problem"] == 1
        log = (d / "tea.out").read_text()  # the reference's default output file
        assert log.count(" Step ") == 10 and "Iteration count" in log
    if "ref" in runs:
        keys = ("iterations", "error", "vol", "mass", "ie", "temp")
        for a, b in zip(runs["port"]["records"], runs["ref"]["records"]):
            assert all(a[k] == b[k] for k in keys), (a, b)


def test_positional_deck_and_output(tmp_path):
    """tea_leaf.f90:68-85: the first argument replaces tea.in and the second tea.out."""
    import subprocess

    from conftest import PORT

    (tmp_path / "my.in").write_text(BASE.format(extra="end_step=2"))
    subprocess.run([str(tea.tea_leaf_exe()), "--dim", "2", "--backend", str(PORT[2]), "--quiet", "my.in", "my.out"],
                   cwd=tmp_path, check=True, capture_output=True)
    assert not (tmp_path / "tea.in").exists() and not (tmp_path / "tea.out").exists()
    assert (tmp_path / "my.out").read_text().count(" Step ") == 2
