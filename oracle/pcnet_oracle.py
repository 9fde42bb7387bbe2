"""CPU oracle of the learned-preconditioner network (test infrastructure only).

Only tests/ and the benchmark's checks import this module; the product path
never does.  It restates, in numpy float64, the network of
piro_b200/csrc/pcnet.cu:

  input channels (r, r*f); four bias-free 3x3x3 convolutions, channels
  2 -> 16 -> 16 -> 16 -> 1, GELU (tanh form) after the first three, zero padding outside
  the interior of the ghost-inclusive grid; parameters one flat vector, per
  layer W[tap][ci][co], tap = (dz+1)*9 + (dy+1)*3 + (dx+1);

with its loss (masked MSE) and the analytic gradient.  With `emulate=True`
the values the device rounds to BF16 (weights, input, pre-activations,
activations, data gradients) are rounded here at the same points, so the
device gradients are compared against the same function; with
`emulate=False` everything is float64, which is what the finite-difference
check of the analytic gradient uses.  PIRO itself has no learned component:
this oracle is pinned by that finite-difference check, not by reference
fixtures.
"""
from __future__ import annotations

import math

import numpy as np

LAYERS = [(2, 16), (16, 16), (16, 16), (16, 1)]
TAPS = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def layout():
    """Offsets of each layer's weights and the total parameter count."""
    off, w = 0, []
    for ci, co in LAYERS:
        w.append(off)
        off += 27 * ci * co
    return w, off


def num_params() -> int:
    return layout()[1]


def unpack(params):
    wo, _ = layout()
    return [params[wo[l]:wo[l] + 27 * ci * co].reshape(27, ci, co) for l, (ci, co) in enumerate(LAYERS)]


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


_C = math.sqrt(2.0 / math.pi)
_A = 0.044715


def gelu(x):
    """GELU, tanh form (Hendrycks & Gimpel 2016): 0.5 x (1 + tanh(c (x + a x^3)))."""
    return 0.5 * x * (1.0 + np.tanh(_C * (x + _A * x ** 3)))


def gelu_d(x):
    t = np.tanh(_C * (x + _A * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * _C * (1.0 + 3.0 * _A * x * x)


def interior(nx, ny, nz):
    m = np.zeros((nz, ny, nx), bool)
    m[1:-1, 1:-1, 1:-1] = True
    return m


def _conv(x, W):
    """x (B, nz, ny, nx, ci) zero outside the interior -> (B, nz, ny, nx, co), 0 on the boundary."""
    B, nz, ny, nx, _ = x.shape
    out = np.zeros((B, nz, ny, nx, W.shape[2]))
    acc = np.zeros((B, nz - 2, ny - 2, nx - 2, W.shape[2]))
    for t, (dz, dy, dx) in enumerate(TAPS):
        xs = x[:, 1 + dz:nz - 1 + dz, 1 + dy:ny - 1 + dy, 1 + dx:nx - 1 + dx, :]
        acc += xs @ W[t]
    out[:, 1:-1, 1:-1, 1:-1, :] = acc
    return out


def _conv_t(gy, W):
    """Transpose of _conv's linear part: gx[c'] = sum_t W[t] gy[c' - off(t)], interior c'."""
    B, nz, ny, nx, _ = gy.shape
    gx = np.zeros((B, nz, ny, nx, W.shape[1]))
    acc = np.zeros((B, nz - 2, ny - 2, nx - 2, W.shape[1]))
    for t, (dz, dy, dx) in enumerate(TAPS):
        gs = gy[:, 1 - dz:nz - 1 - dz, 1 - dy:ny - 1 - dy, 1 - dx:nx - 1 - dx, :]
        acc += gs @ W[t].T
    gx[:, 1:-1, 1:-1, 1:-1, :] = acc
    return gx


def _conv_w(x, gy):
    """dW[t] = sum_c x[c + off(t)]^T gy[c] over interior c."""
    B, nz, ny, nx, ci = x.shape
    co = gy.shape[-1]
    g = gy[:, 1:-1, 1:-1, 1:-1, :].reshape(-1, co)
    dW = np.zeros((27, ci, co))
    for t, (dz, dy, dx) in enumerate(TAPS):
        xs = x[:, 1 + dz:nz - 1 + dz, 1 + dy:ny - 1 + dy, 1 + dx:nx - 1 + dx, :].reshape(-1, ci)
        dW[t] = xs.T @ g
    return dW


def _grid(a, B, n):
    nx, ny, nz = n
    return np.asarray(a, np.float64).reshape(B, nz, ny, nx)


def forward(params, n, r, feat, emulate=True, keep=False):
    """Network output (B, N) for inputs r, feat (B, N) on grids n = (nx, ny, nz)."""
    nx, ny, nz = n
    r = np.atleast_2d(r)
    B = r.shape[0]
    rnd = bf16 if emulate else (lambda v: np.asarray(v, np.float64))
    P = rnd(params)
    layers = unpack(P)
    m = interior(nx, ny, nz)[None, :, :, :, None]
    rg = _grid(r, B, n)
    rf = rg * _grid(np.atleast_2d(feat), B, n)
    if emulate:
        rf = rf.astype(np.float32)  # the device forms r * f in FP32 before rounding
    x = np.stack([rg, rf], axis=-1)
    x = np.where(m, rnd(x), 0.0)
    acts, pre = [x], []
    for l in range(3):
        y = rnd(_conv(acts[-1], layers[l]))
        pre.append(y)
        acts.append(np.where(m, rnd(gelu(y)), 0.0))
    out = _conv(acts[-1], layers[3])[..., 0]
    if emulate:
        out = out.astype(np.float32).astype(np.float64)
    out = out.reshape(B, -1)
    if keep:
        return out, dict(acts=acts, pre=pre, layers=layers, m=m)
    return out


def loss_grad(params, n, r, feat, target, mask, emulate=True):
    """Masked MSE loss and its gradient with respect to the flat parameters."""
    nx, ny, nz = n
    out, st = forward(params, n, r, feat, emulate, keep=True)
    B = out.shape[0]
    t = np.atleast_2d(target).astype(np.float64)
    mk = np.atleast_2d(mask).astype(np.float64)
    msum = mk.sum()
    d = out - t
    loss = float((mk * d * d).sum() / msum)
    if emulate:
        gout = (np.float32(2.0) * mk.astype(np.float32) * d.astype(np.float32)
                * np.float32(1.0 / msum)).astype(np.float64)
    else:
        gout = 2.0 * mk * d / msum
    # boundary outputs are constant zeros: no gradient flows from them
    gout = gout * interior(nx, ny, nz).reshape(1, -1)
    rnd = bf16 if emulate else (lambda v: v)
    acts, pre, layers, m = st["acts"], st["pre"], st["layers"], st["m"]
    grads = [None] * 4
    gy = gout.reshape(B, nz, ny, nx, 1)
    for l in (3, 2, 1, 0):
        grads[l] = _conv_w(acts[l], gy)
        if l > 0:
            gx = _conv_t(gy, layers[l])
            gy = np.where(m, rnd(gx * gelu_d(pre[l - 1])), 0.0)
    wo, total = layout()
    g = np.zeros(total)
    for l in range(4):
        g[wo[l]:wo[l] + grads[l].size] = grads[l].reshape(-1)
    return loss, g


def init_params(seed: int = 0) -> np.ndarray:
    """Random parameters for tests (not the device's initialiser)."""
    rng = np.random.default_rng(seed)
    wo, total = layout()
    p = np.zeros(total)
    for l, (ci, co) in enumerate(LAYERS):
        sd = math.sqrt(2.0 / (27 * ci)) * (0.1 if l == 3 else 1.0)
        p[wo[l]:wo[l] + 27 * ci * co] = rng.standard_normal(27 * ci * co) * sd
    return p
