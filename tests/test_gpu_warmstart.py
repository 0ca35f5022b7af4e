"""The learned warm start on the GPU: the network's kernels against the CPU oracle, the
tensor-core convolution and weight gradient against the CUDA-core ones, training, and
what the trained network gains in the solve.

There is no reference counterpart (TeaLeaf has no learned component); the numerics are
held to oracle/warmstart_oracle.py (float64, itself pinned by finite differences in
tests/test_warmstart_oracle.py) within bfloat16 tolerances, and the solve is judged by
converging to the same tolerance with fewer iterations.
"""
import importlib.util

import numpy as np
import pytest

from conftest import ROOT, rel, tea

pytestmark = pytest.mark.gpu

_spec = importlib.util.spec_from_file_location("warmstart_oracle", ROOT / "oracle" / "warmstart_oracle.py")
wo = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(wo)

# bfloat16 storage (8 significant bits) through a few layers: relative L2 errors of a few
# per cent against the float64 oracle.
FWD_TOL = 3e-2
GRAD_COS = 0.99


def _flat(p, levels, base, dim=2):
    parts = []
    for name, _, _ in wo.layer_shapes(levels, base, wo.in_channels(dim)):
        parts += [p[name + ".w"].reshape(-1), p[name + ".b"].reshape(-1)]
    parts += [p["head.w"], p["head.b"]]
    return np.concatenate(parts).astype(np.float32)


def _split(flat, levels, base, dim=2):
    out, off = {}, 0
    nt = wo.taps(dim)
    for name, co, ci in wo.layer_shapes(levels, base, wo.in_channels(dim)):
        out[name + ".w"] = flat[off:off + co * nt * ci].reshape(co, nt, ci)
        off += co * nt * ci
        out[name + ".b"] = flat[off:off + co]
        off += co
    c0 = wo.channels(levels, base)[0]
    out["head.w"] = flat[off:off + c0]
    out["head.b"] = flat[off + c0:off + c0 + 1]
    return out


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _case(levels, base, n, hw, seed, dim=2):
    rng = np.random.default_rng(seed)
    p = wo.init_params(levels, base, seed=seed, dim=dim)
    x = rng.normal(size=(n,) + (hw,) * dim + (wo.in_channels(dim),)) * 0.5
    t = rng.normal(size=(n,) + (hw,) * dim) * 0.1
    return p, x, t


def _cos(a, b):
    a, b = np.asarray(a, np.float64).reshape(-1), np.asarray(b, np.float64).reshape(-1)
    return float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))


@pytest.mark.parametrize("reference_conv", [True, False], ids=["cuda_cores", "tensor_cores"])
@pytest.mark.parametrize("levels,base", [(2, 16), (3, 32)])
def test_forward_and_gradients_match_oracle(reference_conv, levels, base):
    p, x, t = _case(levels, base, 2, 32, seed=levels * 7 + base)
    net = tea.WarmStart(levels, base, seed=0)
    try:
        net.set_reference_conv(reference_conv)
        net.set_params(_flat(p, levels, base))
        y, loss, grads = net.eval(x, t)
        ys, gsum, lsum = [], None, 0.0
        for i in range(x.shape[0]):
            yi, cache = wo.forward(p, x[i], levels, base)
            gi = wo.backward(p, cache, yi, t[i], levels, base)
            ys.append(yi)
            lsum += wo.loss(yi, t[i])
            gsum = gi if gsum is None else {k: gsum[k] + gi[k] for k in gi}
        y_ref = np.stack(ys)
        assert _rel_l2(y, y_ref) <= FWD_TOL, _rel_l2(y, y_ref)
        assert rel(loss, lsum / x.shape[0]) <= 0.05
        # The GPU averages the loss over all n images at once: scale the oracle's per-image
        # gradients the same way.
        g = _split(grads, levels, base)
        for k, ref in gsum.items():
            ref = ref / x.shape[0]
            a, b = g[k].reshape(-1).astype(np.float64), ref.reshape(-1)
            cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
            assert cos >= GRAD_COS, (k, cos)
            assert 0.9 <= np.linalg.norm(a) / (np.linalg.norm(b) + 1e-30) <= 1.1, k
    finally:
        net.close()


def test_residual_loss_gradients_match_oracle():
    levels, base = 2, 16
    p, x, t = _case(levels, base, 2, 32, seed=31)
    rng = np.random.default_rng(32)
    kxy = rng.uniform(0.5, 20.0, (2, 32, 32, 2))
    net = tea.WarmStart(levels, base, seed=0)
    try:
        net.set_params(_flat(p, levels, base))
        y, loss, grads = net.eval(x, t, kxy)
        lsum, gsum = 0.0, None
        for i in range(2):
            yi, cache = wo.forward(p, x[i], levels, base)
            kx, ky = kxy[i, :, :, 0], kxy[i, :, :, 1]
            lsum += wo.residual_loss(yi, t[i], kx, ky)
            gy = wo.residual_loss_grad(yi, t[i], kx, ky) / 2  # the GPU averages over both images
            gi = wo.backward(p, cache, yi, t[i], levels, base, gy=gy)
            gsum = gi if gsum is None else {k: gsum[k] + gi[k] for k in gi}
        assert rel(loss, lsum / 2) <= 0.05, (loss, lsum / 2)
        g = _split(grads, levels, base)
        for k, ref in gsum.items():
            a, b = g[k].reshape(-1).astype(np.float64), ref.reshape(-1)
            cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
            assert cos >= GRAD_COS, (k, cos)
    finally:
        net.close()


def test_tensor_core_convolution_equals_cuda_cores():
    levels, base = 3, 32
    p, x, _ = _case(levels, base, 1, 256, seed=5)  # 65536 pixels: many 128-pixel tiles
    net = tea.WarmStart(levels, base, seed=0)
    try:
        net.set_params(_flat(p, levels, base))
        net.set_reference_conv(True)
        y_ref, _, _ = net.eval(x)
        net.set_reference_conv(False)
        y_tc, _, _ = net.eval(x)
        assert _rel_l2(y_tc, y_ref) <= 1e-2, _rel_l2(y_tc, y_ref)
    finally:
        net.close()


def test_tensor_core_weight_gradients_equal_cuda_cores():
    """The weight and bias gradients on the tensor cores (k_wgrad_tc: per tap a GEMM over
    the pixels, MN-major operands straight from the NHWC rows, a ones column for the bias)
    against the CUDA-core kernel, on 32768 pixels per layer (many pixel slices per tap)."""
    levels, base = 3, 32
    p, x, t = _case(levels, base, 2, 128, seed=9)
    net = tea.WarmStart(levels, base, seed=0)
    try:
        net.set_params(_flat(p, levels, base))
        net.set_reference_conv(True)
        _, _, g_ref = net.eval(x, t)
        net.set_reference_conv(False)
        _, _, g_tc = net.eval(x, t)
        gr, gt = _split(g_ref, levels, base), _split(g_tc, levels, base)
        for k in gr:
            a, b = gt[k].reshape(-1).astype(np.float64), gr[k].reshape(-1).astype(np.float64)
            cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
            assert cos >= 0.999 and _rel_l2(a, b) <= 3e-2, (k, cos, _rel_l2(a, b))
    finally:
        net.close()


def _deck(seed, steps=8, cells=128):
    spec = tea.DeckSpec(dim=2, cells=cells, states=8, seed=seed, solver="cg", end_step=steps, dt=0.004, eps=1e-15,
                        eps_rel=1e-10, max_iters=20000, summary_frequency=1, check_result=True)
    return tea.seeded_deck(spec)


def test_training_reduces_loss_and_warm_started_solves_converge(capsys):
    """Training on solver-generated pairs lowers the loss; on an unseen layout the solve
    starts from the network's (smoothed) guess whenever that has the smaller FP64 residual and
    converges to the same tolerance and field summary.  What the network gains is measured
    and printed: on these decks the accepted guesses lower the initial residual, yet CG
    takes a few per cent more iterations than from u0 (the guess's remaining error sits in
    the low modes that CG resolves slowest)."""
    net = tea.WarmStart(3, 32, seed=1)
    try:
        for seed in (101, 102, 103):  # training layouts
            tea.run_deck(_deck(seed), 2, fused=True, ws_net=net.id, ws_mode=tea.WS_RECORD)
        assert net.pairs() == 24
        # The loss is the smoothed guess's error energy relative to the plain start's.
        first, last, ms = net.train(steps=600, batch=8, crop=64, lr=1e-4, seed=7)
        assert last < 0.5 and last < first, (first, last)
        deck = _deck(204)  # unseen
        _, plain = tea.run_deck(deck, 2, fused=True, summary_every_step=True)
        _, warm = tea.run_deck(deck, 2, fused=True, summary_every_step=True, ws_net=net.id, ws_mode=tea.WS_ATTACH)
        assert sum(r["warm_start_used"] for r in warm) >= len(warm) // 2
        for a, b in zip(warm, plain):
            assert a["exact_error"] < a["eps_used"]
            for k in ("vol", "mass", "ie", "temp"):
                assert rel(a[k], b[k]) <= 1e-9, (a["step"], k)
        it_plain = sum(r["iterations"] for r in plain)
        it_warm = sum(r["iterations"] for r in warm)
        with capsys.disabled():
            print(f"\nwarm start: loss {first:.3f} -> {last:.3f}; CG iterations {it_warm} vs {it_plain} from u0 "
                  f"({100.0 * (it_warm - it_plain) / it_plain:+.1f}%)")
        # A rejected guess restores the plain start bit for bit: until the first accepted
        # guess the two runs are the same run.
        for a, b in zip(warm, plain):
            if a["warm_start_used"]:
                break
            assert a["iterations"] == b["iterations"] and a["temp"] == b["temp"], (a["step"], a, b)
        # What the network gains on these decks, as recorded on a B200: a loss of 7.0-7.2 %
        # more CG iterations (1884-1888 against 1761).  The bar holds that recorded loss, so
        # that a worse network fails here rather than passing inside a loose bound.
        assert it_warm <= 1.10 * it_plain, (it_warm, it_plain)
    finally:
        net.close()


# ----------------------------------------------------------------------------- 3D network

@pytest.mark.parametrize("reference_conv", [True, False], ids=["cuda_cores", "tensor_cores"])
@pytest.mark.parametrize("levels,base,hw", [(2, 16, 8), (3, 24, 16)])
def test_3d_forward_and_gradients_match_oracle(reference_conv, levels, base, hw):
    """The 3D network of the 3D library (3x3x3 convolutions, 2x2x2 pooling, five input
    features; base 24 is the 512^3 configuration's, whose channel counts the tensor-core
    kernels pad to multiples of 16) against the float64 oracle: forward, loss and every
    parameter gradient."""
    p, x, t = _case(levels, base, 2, hw, seed=levels * 7 + base, dim=3)
    net = tea.WarmStart(levels, base, seed=0, dim=3)
    try:
        net.set_reference_conv(reference_conv)
        net.set_params(_flat(p, levels, base, dim=3))
        y, loss, grads = net.eval(x, t)
        ys, gsum, lsum = [], None, 0.0
        for i in range(x.shape[0]):
            yi, cache = wo.forward(p, x[i], levels, base)
            gi = wo.backward(p, cache, yi, t[i], levels, base)
            ys.append(yi)
            lsum += wo.loss(yi, t[i])
            gsum = gi if gsum is None else {k: gsum[k] + gi[k] for k in gi}
        y_ref = np.stack(ys)
        assert _rel_l2(y, y_ref) <= FWD_TOL, _rel_l2(y, y_ref)
        assert rel(loss, lsum / x.shape[0]) <= 0.05
        g = _split(grads, levels, base, dim=3)
        for k, ref in gsum.items():
            ref = ref / x.shape[0]
            if k == "head.b":
                # 2 mean(y - t): a sum that cancels, so its error is held to the scale of its
                # terms, 2 mean |y - t|, rather than to its own (small) value.
                scale = 2.0 * float(np.mean(np.abs(y_ref - t)))
                assert abs(float(g[k][0]) - float(ref[0])) <= 0.05 * scale, (k, g[k], ref, scale)
                continue
            assert _cos(g[k], ref) >= GRAD_COS, (k, _cos(g[k], ref))
            assert 0.9 <= np.linalg.norm(g[k]) / (np.linalg.norm(ref) + 1e-30) <= 1.1, k
    finally:
        net.close()


def test_3d_residual_loss_gradients_match_oracle():
    levels, base, hw = 2, 16, 8
    p, x, t = _case(levels, base, 2, hw, seed=41, dim=3)
    rng = np.random.default_rng(42)
    kk = rng.uniform(0.5, 20.0, (2, hw, hw, hw, 3))
    net = tea.WarmStart(levels, base, seed=0, dim=3)
    try:
        net.set_params(_flat(p, levels, base, dim=3))
        y, loss, grads = net.eval(x, t, kk)
        lsum, gsum = 0.0, None
        for i in range(2):
            yi, cache = wo.forward(p, x[i], levels, base)
            kx, ky, kz = kk[i, ..., 0], kk[i, ..., 1], kk[i, ..., 2]
            lsum += wo.residual_loss(yi, t[i], kx, ky, kz)
            gy = wo.residual_loss_grad(yi, t[i], kx, ky, kz) / 2  # the GPU averages over both images
            gi = wo.backward(p, cache, yi, t[i], levels, base, gy=gy)
            gsum = gi if gsum is None else {k: gsum[k] + gi[k] for k in gi}
        assert rel(loss, lsum / 2) <= 0.05, (loss, lsum / 2)
        g = _split(grads, levels, base, dim=3)
        for k, ref in gsum.items():
            assert _cos(g[k], ref) >= GRAD_COS, (k, _cos(g[k], ref))
    finally:
        net.close()


def test_3d_tensor_cores_equal_cuda_cores():
    """3x3x3 convolutions and weight gradients on the tensor cores against the CUDA-core
    kernels over 2 x 32^3 voxels (many 128-voxel tiles and pixel slices per tap)."""
    levels, base = 3, 24
    p, x, t = _case(levels, base, 2, 32, seed=13, dim=3)
    net = tea.WarmStart(levels, base, seed=0, dim=3)
    try:
        net.set_params(_flat(p, levels, base, dim=3))
        net.set_reference_conv(True)
        y_ref, _, g_ref = net.eval(x, t)
        net.set_reference_conv(False)
        y_tc, _, g_tc = net.eval(x, t)
        assert _rel_l2(y_tc, y_ref) <= 1e-2, _rel_l2(y_tc, y_ref)
        gr, gt = _split(g_ref, levels, base, dim=3), _split(g_tc, levels, base, dim=3)
        for k in gr:
            assert _cos(gt[k], gr[k]) >= 0.999 and _rel_l2(gt[k], gr[k]) <= 3e-2, (k, _cos(gt[k], gr[k]))
    finally:
        net.close()


@pytest.mark.parametrize("mode", [0, 2], ids=["tma", "cp_async"])
@pytest.mark.parametrize("dim", [2, 3])
def test_row_segment_convolution_matches_oracle_and_cuda_cores(dim, mode):
    """Images 128 pixels wide take the row-segment kernels at full resolution (one staged row
    segment serves the three x-taps), k_conv_tc below: k_conv_tma (mode 0: segments and
    packed weights moved by TMA) and k_conv_rows (mode 2: per-thread copies).  Forward and
    every gradient against the CUDA-core kernels, and the forward against the oracle."""
    levels, base = 2, 24
    rng = np.random.default_rng(77 + dim)
    p = wo.init_params(levels, base, seed=dim, dim=dim)
    shape = (2, 4, 4, 128) if dim == 3 else (2, 8, 128)
    x = rng.normal(size=shape + (wo.in_channels(dim),)) * 0.5
    t = rng.normal(size=shape) * 0.1
    net = tea.WarmStart(levels, base, seed=0, dim=dim)
    try:
        net.set_params(_flat(p, levels, base, dim=dim))
        net.set_conv_mode(1)
        y_ref, _, g_ref = net.eval(x, t)
        net.set_conv_mode(mode)
        y_tc, _, g_tc = net.eval(x, t)
        assert _rel_l2(y_tc, y_ref) <= 1e-2, _rel_l2(y_tc, y_ref)
        gr, gt = _split(g_ref, levels, base, dim=dim), _split(g_tc, levels, base, dim=dim)
        for k in gr:
            if k == "head.b":
                continue
            assert _cos(gt[k], gr[k]) >= 0.999 and _rel_l2(gt[k], gr[k]) <= 3e-2, (k, _cos(gt[k], gr[k]))
        y_o = np.stack([wo.forward(p, x[i], levels, base)[0] for i in range(x.shape[0])])
        assert _rel_l2(y_tc, y_o) <= FWD_TOL, _rel_l2(y_tc, y_o)
    finally:
        net.close()


def _deck3d(seed, steps=4, cells=32, solver="cg"):
    spec = tea.DeckSpec(dim=3, cells=cells, states=8, seed=seed, solver=solver, end_step=steps, dt=0.004, eps=1e-15,
                        eps_rel=1e-10, max_iters=20000, presteps=30, inner_steps=10, summary_frequency=1,
                        check_result=True)
    return tea.seeded_deck(spec)


def test_3d_training_and_warm_started_solves(capsys):
    """The 3D network trained on the 3D solver's own pairs: the loss falls, and on an unseen
    layout each solve converges to the same tolerance and field summary whether or not the
    guess is used; a rejected guess leaves the run exactly the plain run."""
    net = tea.WarmStart(3, 24, seed=1, dim=3)
    try:
        for seed in (301, 302, 303):
            tea.run_deck(_deck3d(seed), 3, fused=True, ws_net=net.id, ws_mode=tea.WS_RECORD)
        assert net.pairs() == 12
        first, last, ms = net.train(steps=300, batch=4, crop=16, lr=1e-4, seed=7)
        assert last < first, (first, last)
        deck = _deck3d(404)
        _, plain = tea.run_deck(deck, 3, fused=True, summary_every_step=True)
        _, warm = tea.run_deck(deck, 3, fused=True, summary_every_step=True, ws_net=net.id, ws_mode=tea.WS_ATTACH)
        for a, b in zip(warm, plain):
            assert a["exact_error"] < a["eps_used"]
            for k in ("vol", "mass", "ie", "temp"):
                assert rel(a[k], b[k]) <= 1e-9, (a["step"], k)
        for a, b in zip(warm, plain):
            if a["warm_start_used"]:
                break
            assert a["iterations"] == b["iterations"] and a["temp"] == b["temp"], (a["step"], a, b)
        it_plain = sum(r["iterations"] for r in plain)
        it_warm = sum(r["iterations"] for r in warm)
        used = sum(r["warm_start_used"] for r in warm)
        with capsys.disabled():
            print(f"\n3D warm start: loss {first:.3f} -> {last:.3f} ({ms:.2f} ms/step); guesses used {used}/{len(warm)}; "
                  f"CG iterations {it_warm} vs {it_plain} from u0 ({100.0 * (it_warm - it_plain) / it_plain:+.1f}%)")
    finally:
        net.close()
