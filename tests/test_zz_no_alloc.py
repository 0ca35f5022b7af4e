"""The allocation-free 2-norm entry point, tea_2norm_noalloc_, against ext_calculate_2norm_.

tea_2norm_noalloc_ serves callers whose device memory belongs to their own pool
allocator and who therefore cannot let a library call cudaMalloc; it works on the
caller's own array and keeps its reduction scratch in a static device array.  Here the
caller's buffers come from torch (the caller may allocate; the entry point does not),
hold the same values as a chunk's r field, and the result must equal the chunk-based
entry point's bit for bit -- both sum in double-double and round once, the tolerance
every GPU-vs-oracle reduction test in this suite uses -- on two calls in a row, which
share the static scratch.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from conftest import tea

pytestmark = pytest.mark.gpu

TEA_ERR_BAD_ARGUMENT = 2
MAX_CELLS = 8192 * 2048


def _i(v):
    return ctypes.byref(ctypes.c_int(v))


def _call(lib, field, nx, ny, nz, out, stream):
    lib.tea_2norm_noalloc_.restype = ctypes.c_int
    return lib.tea_2norm_noalloc_(ctypes.c_void_p(field), _i(nx), _i(ny), _i(nz), ctypes.c_void_p(out),
                                  ctypes.c_void_p(stream))


@pytest.mark.parametrize("dim,shape", [(2, (300, 203, 1)), (2, (4096, 4096, 1)), (3, (41, 30, 17))])
def test_noalloc_2norm_matches_ext_calculate_2norm(dim, shape):
    import torch

    lib = tea.cuda_library(dim)
    nx, ny, nz = shape
    ch = tea.ExtChunk(lib, dim, nx, ny, nz)
    try:
        rng = np.random.default_rng(nx + ny + nz)
        stream = torch.cuda.current_stream().cuda_stream
        for call in range(2):
            field = rng.uniform(-3.0, 3.0, (ch.Z, ch.Y, ch.X)) * (10.0 ** (4 * call))
            ch.write("r", field)
            expected = ch.norm2(True)
            assert expected > 0.0
            dev = torch.from_numpy(field.reshape(-1)).to("cuda")
            out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
            rc = _call(lib, dev.data_ptr(), nx, ny, nz, out.data_ptr(), stream)
            torch.cuda.synchronize()
            assert rc == 0
            assert out.item() == expected, (call, out.item(), expected)
    finally:
        lib.ext_finalise_()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = tea.cuda_library(3)
    # 512^3 inner cells exceed the 16,777,216 cells the static scratch serves; no kernel
    # is launched, so the (non-null, never dereferenced) pointers are not touched.
    rc = _call(lib, 16, 512, 512, 512, 16, 0)
    assert rc == TEA_ERR_BAD_ARGUMENT
    st = ctypes.c_int(0)
    lib.ext_get_status_(ctypes.byref(st))
    assert st.value == TEA_ERR_BAD_ARGUMENT
    lib.tea_last_error.restype = ctypes.c_char_p
    assert b"exceed" in lib.tea_last_error()
    assert 512 ** 3 > MAX_CELLS
