import ctypes
import json
import math
import pathlib
import shutil
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import __graft_entry__  # noqa: E402

tea = __graft_entry__.load_package()

GOLDEN = ROOT / "tests" / "golden"
PORT = {2: ROOT / "oracle" / "libtea_port2d.so", 3: ROOT / "oracle" / "libtea_port3d.so"}
REFLIB = {2: ROOT / "oracle" / "_ref" / "libtea_ref2d.so", 3: ROOT / "oracle" / "_ref" / "libtea_ref3d.so"}

SUM_SEQUENTIAL = 0   # the reference's single-thread Kokkos order
SUM_COMPENSATED = 1  # double-double, order independent: what the CUDA library computes


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def _ensure_built():
    if not all(p.exists() for p in PORT.values()):
        subprocess.run([shutil.which("make") or "make", "-C", str(ROOT / "oracle"), "port"], check=True)
    needed = [tea.driver_path(), tea.tea_leaf_exe(), tea.lib_path(2), tea.lib_path(3)]
    if not all(p.exists() for p in needed):
        tea.build()


_ensure_built()


def port_lib(dim: int, mode: int) -> pathlib.Path:
    """The oracle port for `dim`, with its reduction mode set (the driver dlopens the same
    file, so it shares the library instance and the mode)."""
    lib = tea.load_library(PORT[dim])
    lib.oracle_set_sum_mode(ctypes.c_int(mode))
    return PORT[dim]


def golden_runs() -> dict:
    return json.loads((GOLDEN / "ref_runs.json").read_text())


def kat_decks() -> dict:
    return json.loads((GOLDEN / "kat_decks.json").read_text())


def same(a, b) -> bool:
    """Bitwise equality of two doubles, NaN equal to NaN."""
    if isinstance(a, float) and isinstance(b, float) and math.isnan(a) and math.isnan(b):
        return True
    return a == b


def rel(a: float, b: float) -> float:
    return tea.rel_diff(a, b)


@pytest.fixture(scope="session")
def teapkg():
    return tea
