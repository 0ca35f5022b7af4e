"""ORACLE -- test infrastructure only: a float64 numpy restatement of the learned
warm-start network (forward and backward), used by the tests to check the CUDA kernels.

The reference (TeaLeaf) has no learned component, so nothing here follows a reference
file; this module is pinned by its own finite-difference gradient check
(tests/test_warmstart_oracle.py).  The CUDA library computes the same functions in
bfloat16 storage with float32 accumulation.

Layout: one image at a time, channels last without the batch dimension: arrays shaped
(H, W, C) for the 2D network and (D, H, W, C) for the 3D one.  Every function takes its
dimension from the array it is given.

Network (a U-Net of `levels` levels, `base` channels at full resolution, channel count
doubling per level, up to an optional cap):

    encoder level l:  x = relu(conv(x, enc[l].a)); x = relu(conv(x, enc[l].b));
                      skip[l] = x; x = avgpool2(x) unless l is the last level
    decoder level l (from levels-2 down to 0):
                      x = concat(upsample2(x), skip[l]);
                      x = relu(conv(x, dec[l].a)); x = relu(conv(x, dec[l].b))
    head:             y = conv1x1(x) to one channel

conv is 3x3 in 2D and 3x3x3 in 3D with zero padding; its weights are shaped
(Cout, taps, Cin) with tap t = 3*dy + dx (2D) or t = 9*dz + 3*dy + dx (3D), and a bias per
output channel; the head is (Cin,) weights and a scalar bias.  avgpool2 averages 2x2
(2x2x2) blocks and upsample2 copies each coarse pixel to its block.
"""
from __future__ import annotations

import itertools

import numpy as np

IN_CHANNELS = 4  # 2D: r0 / scale, log10(density) / 2, log10(1 + Kx) / 4, log10(1 + Ky) / 4
IN_CHANNELS_3D = 5  # 3D: the same and log10(1 + Kz) / 4


def in_channels(dim: int = 2) -> int:
    return IN_CHANNELS_3D if dim == 3 else IN_CHANNELS


def taps(dim: int = 2) -> int:
    return 3 ** dim


def channels(levels: int, base: int, cap: int = 0):
    """Channels per level: doubling from `base`, stopped at `cap` when it is positive."""
    return [min(base * (2 ** l), max(cap, base)) if cap > 0 else base * (2 ** l) for l in range(levels)]


def layer_shapes(levels: int, base: int, cin: int = IN_CHANNELS, cap: int = 0):
    """(name, Cout, Cin) of every convolution, in the order the CUDA library stores them."""
    ch = channels(levels, base, cap)
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


def init_params(levels: int, base: int, seed: int = 0, cin: int | None = None, dim: int = 2, cap: int = 0):
    rng = np.random.default_rng(seed)
    cin = in_channels(dim) if cin is None else cin
    t = taps(dim)
    p = {}
    for name, co, ci in layer_shapes(levels, base, cin, cap):
        p[name + ".w"] = rng.normal(0.0, np.sqrt(2.0 / (t * ci)), (co, t, ci))
        p[name + ".b"] = rng.normal(0.0, 0.01, co)
    c0 = channels(levels, base)[0]
    p["head.w"] = rng.normal(0.0, np.sqrt(1.0 / c0), c0)
    p["head.b"] = np.zeros(1)
    return p


# ----------------------------------------------------------------------------- primitives

def _tap_offsets(nd: int):
    """Offsets (0..2 per spatial axis, slowest axis first) of taps 0, 1, ...: tap t is
    np.unravel_index(t, (3,) * nd), i.e. t = 3*dy + dx or 9*dz + 3*dy + dx."""
    return list(itertools.product(range(3), repeat=nd))


def _window(xp, off, shape):
    return xp[tuple(slice(o, o + n) for o, n in zip(off, shape))]


def conv3x3(x, w, b):
    """The network's convolution: 3x3 on (H, W, C) images, 3x3x3 on (D, H, W, C) volumes."""
    nd = x.ndim - 1
    shape = x.shape[:nd]
    xp = np.pad(x, [(1, 1)] * nd + [(0, 0)])
    y = np.broadcast_to(b, shape + (w.shape[0],)).copy()
    for t, off in enumerate(_tap_offsets(nd)):
        y += _window(xp, off, shape) @ w[:, t, :].T
    return y


def conv3x3_backward(x, w, gy):
    """Gradients of conv3x3 with respect to x, w and b, given dL/dy."""
    nd = x.ndim - 1
    shape = x.shape[:nd]
    xp = np.pad(x, [(1, 1)] * nd + [(0, 0)])
    gw = np.zeros_like(w)
    gxp = np.zeros_like(xp)
    gflat = gy.reshape(-1, gy.shape[-1])
    for t, off in enumerate(_tap_offsets(nd)):
        patch = _window(xp, off, shape)
        gw[:, t, :] = gflat.T @ patch.reshape(-1, patch.shape[-1])
        _window(gxp, off, shape)[...] += gy @ w[:, t, :]
    gb = gflat.sum(axis=0)
    inner = tuple(slice(1, n + 1) for n in shape)
    return gxp[inner], gw, gb


def _blocks(x):
    """View of x with each spatial axis n split into (n // 2, 2)."""
    nd = x.ndim - 1
    new = []
    for n in x.shape[:nd]:
        new += [n // 2, 2]
    return x.reshape(new + [x.shape[-1]]), tuple(range(1, 2 * nd, 2))


def avgpool2(x):
    v, axes = _blocks(x)
    return v.mean(axis=axes)


def avgpool2_backward(gy):
    nd = gy.ndim - 1
    return upsample2(gy) / float(2 ** nd)


def upsample2(x):
    nd = x.ndim - 1
    for a in range(nd):
        x = np.repeat(x, 2, axis=a)
    return x


def upsample2_backward(gy):
    v, axes = _blocks(gy)
    return v.sum(axis=axes)


# ----------------------------------------------------------------------------- network

def forward(p, x, levels: int, base: int):
    """Returns (prediction (H, W) or (D, H, W), cache for backward)."""
    nd = x.ndim - 1
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
        h = np.concatenate([up, skips[l]], axis=nd)
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


def _coefs(v, kx, ky, kz):
    """(axis of v, face coefficient array) per spatial axis: x is the last axis, then y, z."""
    ks = [(v.ndim - 1, kx), (v.ndim - 2, ky)]
    if kz is not None:
        ks.append((v.ndim - 3, kz))
    return ks


def _sl(nd, axis, s):
    idx = [slice(None)] * nd
    idx[axis] = s
    return tuple(idx)


def _lo_hi(k, axis):
    """A cell's face coefficient on its low side (zero on the image's low edge) and on its
    high side (the next cell's low face; zero on the high edge)."""
    nd = k.ndim
    lo = k.copy()
    lo[_sl(nd, axis, slice(0, 1))] = 0.0
    hi = np.zeros_like(k)
    hi[_sl(nd, axis, slice(0, -1))] = k[_sl(nd, axis, slice(1, None))]
    return lo, hi


def apply_a(v, kx, ky, kz=None):
    """The solver's operator on one image ((H, W), or (D, H, W) with kz): kx, ky (, kz) are
    each cell's face coefficients to its left, below (and behind); faces through the
    image's edges carry no flux."""
    nd = v.ndim
    diag = np.ones_like(v)
    off = np.zeros_like(v)
    for axis, k in _coefs(v, kx, ky, kz):
        lo, hi = _lo_hi(k, axis)
        diag += lo + hi
        off[_sl(nd, axis, slice(1, None))] += lo[_sl(nd, axis, slice(1, None))] * v[_sl(nd, axis, slice(0, -1))]
        off[_sl(nd, axis, slice(0, -1))] += hi[_sl(nd, axis, slice(0, -1))] * v[_sl(nd, axis, slice(1, None))]
    return diag * v - off


SMOOTH_SWEEPS, OMEGA = 8, 0.8  # the warm start's damped Jacobi sweeps of the guess


def diag_a(kx, ky, kz=None):
    d = np.ones_like(kx)
    for axis, k in _coefs(kx, kx, ky, kz):
        lo, hi = _lo_hi(k, axis)
        d += lo + hi
    return d


def smooth(e, kx, ky, kz=None):
    """The sweeps acting on the guess's error: e <- (I - omega D^-1 A) e."""
    d = diag_a(kx, ky, kz)
    for _ in range(SMOOTH_SWEEPS):
        e = e - OMEGA * apply_a(e, kx, ky, kz) / d
    return e


def smooth_transpose(g, kx, ky, kz=None):
    d = diag_a(kx, ky, kz)
    for _ in range(SMOOTH_SWEEPS):
        g = g - OMEGA * apply_a(g / d, kx, ky, kz)
    return g


def residual_loss(y, target, kx, ky, kz=None):
    """The training loss of the warm start: the energy norm of the smoothed guess's error,
    relative to that of the plain start (du = 0), when target is the true du."""
    es = smooth(y - target, kx, ky, kz)
    return float(np.sum(es * apply_a(es, kx, ky, kz)) / np.sum(target * apply_a(target, kx, ky, kz)))


def residual_loss_grad(y, target, kx, ky, kz=None):
    es = smooth(y - target, kx, ky, kz)
    g = 2.0 * apply_a(es, kx, ky, kz) / np.sum(target * apply_a(target, kx, ky, kz))  # A is symmetric
    return smooth_transpose(g, kx, ky, kz)


def backward(p, cache, y, target, levels: int, base: int, gy=None, cap: int = 0):
    """Gradients with respect to every parameter of loss(y, target), or, given gy = dL/dy,
    of that loss."""
    ch = channels(levels, base, cap)
    g = {}
    if gy is None:
        gy = 2.0 * (y - target) / y.size
    h = cache["head.in"]
    g["head.w"] = gy.reshape(-1) @ h.reshape(-1, h.shape[-1])
    g["head.b"] = np.array([gy.sum()])
    gh = gy[..., None] * p["head.w"]
    gskip = [None] * levels
    for l in range(0, levels - 1):
        for s in "ba":
            name = f"dec{l}{s}"
            gpre = gh * (cache[name + ".out"] > 0)
            gh, g[name + ".w"], g[name + ".b"] = conv3x3_backward(cache[name + ".in"], p[name + ".w"], gpre)
        c_up = ch[l + 1]
        gskip[l] = gh[..., c_up:]
        gh = upsample2_backward(gh[..., :c_up])
    for l in range(levels - 1, -1, -1):
        if l < levels - 1:
            gh = avgpool2_backward(gh) + gskip[l]
        for s in "ba":
            name = f"enc{l}{s}"
            gpre = gh * (cache[name + ".out"] > 0)
            gh, g[name + ".w"], g[name + ".b"] = conv3x3_backward(cache[name + ".in"], p[name + ".w"], gpre)
    return g


def features(r0, density, kx, ky, kz=None):
    """Network input of a timestep (inner cells, (H, W) or (D, H, W) arrays): r0 = u0 - A u0,
    the residual of the plain start, scaled by its largest magnitude (also the scale of the
    target du), and the coefficients."""
    scale = float(np.max(np.abs(r0)))
    scale = scale if scale > 0.0 else 1.0
    parts = [r0 / scale, np.log10(density) / 2.0, np.log10(1.0 + kx) / 4.0, np.log10(1.0 + ky) / 4.0]
    if kz is not None:
        parts.append(np.log10(1.0 + kz) / 4.0)
    return np.stack(parts, axis=r0.ndim), scale
