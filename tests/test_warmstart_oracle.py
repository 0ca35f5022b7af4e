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


@pytest.mark.parametrize("levels,base,hw", [(2, 4, 8), (3, 4, 8)])
def test_oracle_gradients_match_finite_differences(levels, base, hw):
    rng = np.random.default_rng(levels * 10 + base)
    p = wo.init_params(levels, base, seed=3)
    x = rng.normal(size=(hw, hw, wo.IN_CHANNELS))
    target = rng.normal(size=(hw, hw))
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
