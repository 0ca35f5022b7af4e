"""ORACLE -- test infrastructure only: a float64 numpy restatement of the learned
warm-start network (forward and backward), used by the tests to check the CUDA kernels.

The reference (TeaLeaf) has no learned component, so nothing here follows a reference
file; this module is pinned by its own finite-difference gradient check
(tests/test_warmstart_oracle.py).  The CUDA library computes the same functions in
bfloat16 storage with float32 accumulation.

Layout: one image at a time, NHWC without the N (arrays shaped (H, W, C)).

Network (a U-Net of `levels` levels, `base` channels at full resolution, channel count
doubling per level):

    encoder level l:  x = relu(conv3x3(x, enc[l].a)); x = relu(conv3x3(x, enc[l].b));
                      skip[l] = x; x = avgpool2(x) unless l is the last level
    decoder level l (from levels-2 down to 0):
                      x = concat(upsample2(x), skip[l]);
                      x = relu(conv3x3(x, dec[l].a)); x = relu(conv3x3(x, dec[l].b))
    head:             y = conv1x1(x) to one channel

conv3x3 weights are shaped (Cout, 9, Cin) -- tap t = 3*dy + dx, zero padding -- with a
bias per output channel; the head is (Cin,) weights and a scalar bias.
"""
from __future__ import annotations

import numpy as np

IN_CHANNELS = 4  # r0 / scale, log10(density) / 2, log10(1 + Kx) / 4, log10(1 + Ky) / 4


def channels(levels: int, base: int):
    return [base * (2 ** l) for l in range(levels)]


def layer_shapes(levels: int, base: int, cin: int = IN_CHANNELS):
    """(name, Cout, Cin) of every 3x3 convolution, in the order the CUDA library stores them."""
    ch = channels(levels, base)
    out = []
    prev = cin
    for l in range(levels):
        out.append((f"enc{l}a", ch[l], prev))
        out.append((f"enc{l}b", ch[l], ch[l]))
        prev = ch[l]
    for l in range(levels - 2, -1, -1):
        out.append((f"dec{l}a", ch[l], ch[l + 1] + ch[l]))
        out.append((f"dec{l}b", ch[l], ch[l]))
    return out


def init_params(levels: int, base: int, seed: int = 0, cin: int = IN_CHANNELS):
    rng = np.random.default_rng(seed)
    p = {}
    for name, co, ci in layer_shapes(levels, base, cin):
        p[name + ".w"] = rng.normal(0.0, np.sqrt(2.0 / (9 * ci)), (co, 9, ci))
        p[name + ".b"] = rng.normal(0.0, 0.01, co)
    c0 = channels(levels, base)[0]
    p["head.w"] = rng.normal(0.0, np.sqrt(1.0 / c0), c0)
    p["head.b"] = np.zeros(1)
    return p


# ----------------------------------------------------------------------------- primitives

def conv3x3(x, w, b):
    H, W, _ = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (0, 0)))
    y = np.broadcast_to(b, (H, W, w.shape[0])).copy()
    for t in range(9):
        dy, dx = divmod(t, 3)
        y += xp[dy:dy + H, dx:dx + W, :] @ w[:, t, :].T
    return y


def conv3x3_backward(x, w, gy):
    """Gradients of conv3x3 with respect to x, w and b, given dL/dy."""
    H, W, _ = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (0, 0)))
    gw = np.zeros_like(w)
    gxp = np.zeros_like(xp)
    for t in range(9):
        dy, dx = divmod(t, 3)
        patch = xp[dy:dy + H, dx:dx + W, :]
        gw[:, t, :] = np.einsum("hwo,hwi->oi", gy, patch)
        gxp[dy:dy + H, dx:dx + W, :] += gy @ w[:, t, :]
    gb = gy.sum(axis=(0, 1))
    return gxp[1:H + 1, 1:W + 1, :], gw, gb


def avgpool2(x):
    H, W, C = x.shape
    return x.reshape(H // 2, 2, W // 2, 2, C).mean(axis=(1, 3))


def avgpool2_backward(gy):
    return np.repeat(np.repeat(gy, 2, axis=0), 2, axis=1) / 4.0


def upsample2(x):
    return np.repeat(np.repeat(x, 2, axis=0), 2, axis=1)


def upsample2_backward(gy):
    H, W, C = gy.shape
    return gy.reshape(H // 2, 2, W // 2, 2, C).sum(axis=(1, 3))


# ----------------------------------------------------------------------------- network

def forward(p, x, levels: int, base: int):
    """Returns (prediction (H, W), cache for backward)."""
    cache = {"x0": x}
    skips = []
    h = x
    for l in range(levels):
        for s in "ab":
            name = f"enc{l}{s}"
            cache[name + ".in"] = h
            h = np.maximum(conv3x3(h, p[name + ".w"], p[name + ".b"]), 0.0)
            cache[name + ".out"] = h
        skips.append(h)
        if l < levels - 1:
            h = avgpool2(h)
    for l in range(levels - 2, -1, -1):
        up = upsample2(h)
        h = np.concatenate([up, skips[l]], axis=2)
        for s in "ab":
            name = f"dec{l}{s}"
            cache[name + ".in"] = h
            h = np.maximum(conv3x3(h, p[name + ".w"], p[name + ".b"]), 0.0)
            cache[name + ".out"] = h
    cache["head.in"] = h
    y = h @ p["head.w"] + p["head.b"][0]
    return y, cache


def loss(y, target):
    return float(np.mean((y - target) ** 2))


def apply_a(v, kx, ky):
    """The solver's operator on one (H, W) image: kx, ky are each cell's face coefficients
    to its left and below; faces through the image's edges carry no flux."""
    kxl = kx.copy()
    kxl[:, 0] = 0.0
    kxr = np.zeros_like(kx)
    kxr[:, :-1] = kx[:, 1:]
    kyd = ky.copy()
    kyd[0, :] = 0.0
    kyu = np.zeros_like(ky)
    kyu[:-1, :] = ky[1:, :]
    a = (1.0 + kxl + kxr + kyd + kyu) * v
    a[:, 1:] -= kxl[:, 1:] * v[:, :-1]
    a[:, :-1] -= kxr[:, :-1] * v[:, 1:]
    a[1:, :] -= kyd[1:, :] * v[:-1, :]
    a[:-1, :] -= kyu[:-1, :] * v[1:, :]
    return a


SMOOTH_SWEEPS, OMEGA = 8, 0.8  # the warm start's damped Jacobi sweeps of the guess


def diag_a(kx, ky):
    H, W = kx.shape
    d = np.ones((H, W))
    d[:, 1:] += kx[:, 1:]
    d[:, :-1] += kx[:, 1:]
    d[1:, :] += ky[1:, :]
    d[:-1, :] += ky[1:, :]
    return d


def smooth(e, kx, ky):
    """The sweeps acting on the guess's error: e <- (I - omega D^-1 A) e."""
    d = diag_a(kx, ky)
    for _ in range(SMOOTH_SWEEPS):
        e = e - OMEGA * apply_a(e, kx, ky) / d
    return e


def smooth_transpose(g, kx, ky):
    d = diag_a(kx, ky)
    for _ in range(SMOOTH_SWEEPS):
        g = g - OMEGA * apply_a(g / d, kx, ky)
    return g


def residual_loss(y, target, kx, ky):
    """The training loss of the warm start: the energy norm of the smoothed guess's error,
    relative to that of the plain start (du = 0), when target is the true du."""
    es = smooth(y - target, kx, ky)
    return float(np.sum(es * apply_a(es, kx, ky)) / np.sum(target * apply_a(target, kx, ky)))


def residual_loss_grad(y, target, kx, ky):
    es = smooth(y - target, kx, ky)
    g = 2.0 * apply_a(es, kx, ky) / np.sum(target * apply_a(target, kx, ky))  # A is symmetric
    return smooth_transpose(g, kx, ky)


def backward(p, cache, y, target, levels: int, base: int, gy=None):
    """Gradients with respect to every parameter of loss(y, target), or, given gy = dL/dy,
    of that loss."""
    ch = channels(levels, base)
    g = {}
    if gy is None:
        gy = 2.0 * (y - target) / y.size
    h = cache["head.in"]
    g["head.w"] = np.einsum("hw,hwc->c", gy, h)
    g["head.b"] = np.array([gy.sum()])
    gh = gy[:, :, None] * p["head.w"][None, None, :]
    gskip = [None] * levels
    for l in range(0, levels - 1):
        for s in "ba":
            name = f"dec{l}{s}"
            gpre = gh * (cache[name + ".out"] > 0)
            gh, g[name + ".w"], g[name + ".b"] = conv3x3_backward(cache[name + ".in"], p[name + ".w"], gpre)
        c_up = ch[l + 1]
        gskip[l] = gh[:, :, c_up:]
        gh = upsample2_backward(gh[:, :, :c_up])
    for l in range(levels - 1, -1, -1):
        if l < levels - 1:
            gh = avgpool2_backward(gh) + gskip[l]
        for s in "ba":
            name = f"enc{l}{s}"
            gpre = gh * (cache[name + ".out"] > 0)
            gh, g[name + ".w"], g[name + ".b"] = conv3x3_backward(cache[name + ".in"], p[name + ".w"], gpre)
    return g


def features(r0, density, kx, ky):
    """Network input of a timestep (inner cells, (H, W) arrays): r0 = u0 - A u0, the residual
    of the plain start, scaled by its largest magnitude (also the scale of the target du),
    and the coefficients."""
    scale = float(np.max(np.abs(r0)))
    scale = scale if scale > 0.0 else 1.0
    x = np.stack([r0 / scale, np.log10(density) / 2.0, np.log10(1.0 + kx) / 4.0, np.log10(1.0 + ky) / 4.0],
                 axis=2)
    return x, scale
