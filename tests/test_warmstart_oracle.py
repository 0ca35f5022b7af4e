"""The warm-start network oracle (oracle/warmstart_oracle.py) pinned by finite differences.

The learned warm start has no counterpart in the reference, so its CPU oracle is checked
against itself: every parameter gradient of the analytic backward pass must match a
central difference of the float64 loss.
"""
import numpy as np
import pytest

from conftest import ROOT

import importlib.util

_spec = importlib.util.spec_from_file_location("warmstart_oracle", ROOT / "oracle" / "warmstart_oracle.py")
wo = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(wo)


@pytest.mark.parametrize("levels,base,hw,dim", [(2, 4, 8, 2), (3, 4, 8, 2), (2, 4, 4, 3), (3, 2, 4, 3)])
def test_oracle_gradients_match_finite_differences(levels, base, hw, dim):
    rng = np.random.default_rng(levels * 10 + base + dim)
    p = wo.init_params(levels, base, seed=3, dim=dim)
    x = rng.normal(size=(hw,) * dim + (wo.in_channels(dim),))
    target = rng.normal(size=(hw,) * dim)
    y, cache = wo.forward(p, x, levels, base)
    g = wo.backward(p, cache, y, target, levels, base)
    assert set(g) == set(p)
    h = 1e-6
    for name, arr in p.items():
        flat = arr.reshape(-1)
        for idx in rng.choice(flat.size, size=min(4, flat.size), replace=False):
            old = flat[idx]
            flat[idx] = old + h
            lp = wo.loss(wo.forward(p, x, levels, base)[0], target)
            flat[idx] = old - h
            lm = wo.loss(wo.forward(p, x, levels, base)[0], target)
            flat[idx] = old
            fd = (lp - lm) / (2 * h)
            an = g[name].reshape(-1)[idx]
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (name, idx, fd, an)


def test_layer_shapes_follow_the_unet():
    shapes = wo.layer_shapes(3, 32)
    assert [s[0] for s in shapes] == ["enc0a", "enc0b", "enc1a", "enc1b", "enc2a", "enc2b", "dec1a", "dec1b",
                                      "dec0a", "dec0b"]
    assert dict((n, (co, ci)) for n, co, ci in shapes)["dec1a"] == (64, 128 + 64)
    params = sum(co * 9 * ci + co for _, co, ci in shapes) + 32 + 1
    assert 400_000 < params < 600_000  # about half a million parameters


def test_3d_convolution_is_the_direct_sum():
    """The 3x3x3 convolution against a direct loop over output pixels and taps (tap
    t = 9*dz + 3*dy + dx, zero padding)."""
    rng = np.random.default_rng(4)
    x = rng.normal(size=(3, 4, 5, 2))
    w = rng.normal(size=(3, 27, 2))
    b = rng.normal(size=3)
    y = wo.conv3x3(x, w, b)
    D, H, W, _ = x.shape
    for z, yy, xx in [(0, 0, 0), (1, 2, 3), (2, 3, 4), (0, 3, 1)]:
        acc = b.copy()
        for t in range(27):
            dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
            sz, sy, sx = z + dz, yy + dy, xx + dx
            if 0 <= sz < D and 0 <= sy < H and 0 <= sx < W:
                acc += w[:, t, :] @ x[sz, sy, sx]
        assert np.allclose(y[z, yy, xx], acc)
    # pooling and upsampling over 2x2x2 blocks
    v = rng.normal(size=(4, 4, 2, 3))
    assert np.allclose(wo.avgpool2(v)[1, 0, 0], v[2:4, 0:2, 0:2].mean(axis=(0, 1, 2)))
    assert np.allclose(wo.upsample2(wo.avgpool2(v))[3, 1, 1], wo.avgpool2(v)[1, 0, 0])


def test_3d_residual_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(19)
    shape = (3, 4, 5)
    y, t = rng.normal(size=shape), rng.normal(size=shape)
    kx, ky, kz = (rng.uniform(0.1, 5.0, shape) for _ in range(3))
    g = wo.residual_loss_grad(y, t, kx, ky, kz)
    h = 1e-6
    for idx in [(0, 0, 0), (1, 2, 3), (2, 3, 4), (2, 0, 1)]:
        yp, ym = y.copy(), y.copy()
        yp[idx] += h
        ym[idx] -= h
        fd = (wo.residual_loss(yp, t, kx, ky, kz) - wo.residual_loss(ym, t, kx, ky, kz)) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-6 * max(1.0, abs(fd)), (idx, fd, g[idx])
    assert np.allclose(wo.apply_a(np.ones(shape), kx, ky, kz), 1.0)
    # symmetric: u.(A v) = v.(A u)
    u, v = rng.normal(size=shape), rng.normal(size=shape)
    assert np.isclose(np.sum(u * wo.apply_a(v, kx, ky, kz)), np.sum(v * wo.apply_a(u, kx, ky, kz)))


def test_residual_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(9)
    H, W = 6, 7
    y, t = rng.normal(size=(H, W)), rng.normal(size=(H, W))
    kx, ky = rng.uniform(0.1, 5.0, (H, W)), rng.uniform(0.1, 5.0, (H, W))
    g = wo.residual_loss_grad(y, t, kx, ky)
    h = 1e-6
    for idx in [(0, 0), (2, 3), (5, 6), (3, 0)]:
        yp, ym = y.copy(), y.copy()
        yp[idx] += h
        ym[idx] -= h
        fd = (wo.residual_loss(yp, t, kx, ky) - wo.residual_loss(ym, t, kx, ky)) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-6 * max(1.0, abs(fd)), (idx, fd, g[idx])
    # A is the operator with zero-flux edges: constants are its eigenvectors (eigenvalue 1).
    assert np.allclose(wo.apply_a(np.ones((H, W)), kx, ky), 1.0)


def test_capped_four_level_network_has_half_a_million_parameters():
    """The 2D learned configuration's network: 4 levels of 32 base channels whose doubling
    stops at 64 (32/64/64/64), about half a million parameters."""
    assert wo.channels(4, 32, 64) == [32, 64, 64, 64]
    shapes = wo.layer_shapes(4, 32, cap=64)
    params = sum(co * 9 * ci + co for _, co, ci in shapes) + 32 + 1
    assert params == 471_969
    # The 3D configuration's network: 3 levels of 24 channels, 3x3x3 taps, five inputs.
    shapes3 = wo.layer_shapes(3, 24, wo.in_channels(3))
    assert dict((n, (co, ci)) for n, co, ci in shapes3)["dec1a"] == (48, 96 + 48)
    assert wo.taps(3) == 27
