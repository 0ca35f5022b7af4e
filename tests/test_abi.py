"""The C-ABI libraries load on a machine without a GPU and export every entry point the
public headers declare (no compute call is made here)."""
import ctypes
import re

import pytest

from conftest import PORT, ROOT, tea

HEADERS = {2: ["tea_ext_2d.h", "tea_b200.h"], 3: ["tea_ext_3d.h", "tea_b200.h"]}


def declared(header: str):
    text = (ROOT / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text)) - {"if", "sizeof"})


@pytest.mark.parametrize("dim", [2, 3])
def test_cuda_library_exports_declared_symbols(dim):
    lib = ctypes.CDLL(str(tea.lib_path(dim)))
    names = [n for h in HEADERS[dim] for n in declared(h)]
    assert "ext_cg_calc_w_" in names and "ext_tea_leaf_solve_" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_port_exports_reference_abi(dim):
    lib = ctypes.CDLL(str(PORT[dim]))
    names = declared(HEADERS[dim][0])
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_driver_exports():
    lib = ctypes.CDLL(str(tea.driver_path()))
    for n in ("tea_run_deck", "tea_driver_last_error", "tea_calc_eigenvalues_c", "tea_calc_ch_coefs_c"):
        assert hasattr(lib, n), n


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        tea.load_library(tmp_path / "libtea2d_b200.so")


def _cuda_device_present() -> bool:
    import torch

    return torch.cuda.is_available()


@pytest.mark.skipif(_cuda_device_present(), reason="a CUDA device is present")
def test_no_device_is_reported_not_hidden():
    """Without a GPU the CUDA library has no CPU path: ext_init_ records TEA_ERR_NO_DEVICE
    (status 6) with a message, and the driver stops with an error instead of running."""
    lib = tea.cuda_library(2)
    x, y, rank = ctypes.c_int(8), ctypes.c_int(8), ctypes.c_int(0)
    lib.ext_init_(ctypes.byref(x), ctypes.byref(y), ctypes.byref(rank))
    status = ctypes.c_int(-1)
    lib.ext_get_status_(ctypes.byref(status))
    lib.tea_last_error.restype = ctypes.c_char_p
    assert status.value == 6
    assert b"no CPU path" in lib.tea_last_error()
    spec = tea.DeckSpec(dim=2, cells=16, states=3, end_step=1)
    with pytest.raises(RuntimeError, match="status 6"):
        tea.run_deck(tea.seeded_deck(spec), 2)
