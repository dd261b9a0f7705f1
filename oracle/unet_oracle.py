"""CPU oracle of the learned pressure preconditioner's U-Net (test
infrastructure only: the product never imports this module).

The network has no counterpart in the reference solver; this module is its
specification in NumPy, used by the tests to check the library's CUDA forward
pass and its hand-written backward kernels:

* ``forward``: the same layer list as the library (11 3x3x3 convolutions, two
  stride-2, two prolongation-plus-skip joins, leaky ReLU 0.1), with activations
  rounded to BF16 (round-to-nearest-even) at exactly the points where the
  library stores BF16, weights used in their BF16-rounded form and biases in
  FP32.  Arithmetic is FP64, so it differs from the device's FP32
  accumulation only by rounding.
* ``backward``: reverse-mode gradients of the training loss
  (``loss_and_grad``: mean squared error plus an optional squared-difference
  term between grid neighbours) with respect to every parameter, in the
  library's parameter layout (per layer: weights [27][cin][cout] with tap
  k = (dx+1) + 3 (dy+1) + 9 (dz+1), then the bias).
* ``forward_plain`` / ``backward_plain``: the same network in FP64 without
  rounding, smooth enough between the activation kinks for central finite
  differences, which is how the tests pin this oracle.

Arrays are (nz, ny, nx, ch), voxel x fastest, like the device layout.
"""
from __future__ import annotations

import numpy as np

LEAKY = 0.1
# (level, channels) of tensors t0..t13
TENSORS = [(0, 1), (0, 16), (1, 32), (1, 32), (2, 64), (2, 64), (2, 64),
           (2, 32), (1, 32), (1, 32), (1, 16), (0, 16), (0, 16), (0, 1)]
# conv layers: (input tensor, output tensor, stride, act)
CONVS = [(0, 1, 1, 1), (1, 2, 2, 1), (2, 3, 1, 1), (3, 4, 2, 1), (4, 5, 1, 1), (5, 6, 1, 1),
         (6, 7, 1, 1), (8, 9, 1, 1), (9, 10, 1, 1), (11, 12, 1, 1), (12, 13, 1, 0)]
# prolongation joins: (coarse tensor, skip tensor, output tensor)
UPS = [(7, 3, 8), (10, 1, 11)]
# execution order: conv index >= 0, join -1 - index
ORDER = [0, 1, 2, 3, 4, 5, 6, -1, 7, 8, -2, 9, 10]


def layer_shapes():
    out = []
    for (ti, to, _, _) in CONVS:
        cin, cout = TENSORS[ti][1], TENSORS[to][1]
        out.append((27 * cin * cout, cout, cin, cout))
    return out


def param_count() -> int:
    return sum(w + b for (w, b, _, _) in layer_shapes())


def split_params(theta):
    """Per-layer (W[27, cin, cout], b[cout]) views of a flat parameter vector."""
    res, o = [], 0
    for (nw, nb, cin, cout) in layer_shapes():
        res.append((theta[o:o + nw].reshape(27, cin, cout), theta[o + nw:o + nw + nb]))
        o += nw + nb
    return res


def bf16(a):
    """Round to BF16 (nearest, ties to even) and return as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def level_dims(dims):
    """Grid dims (nx, ny, nz) of the three levels."""
    d0 = tuple(int(v) for v in dims)
    for v in d0:
        if v < 5 or (v - 1) % 4:
            raise ValueError("each axis needs (n - 1) % 4 == 0 and n >= 5")
    d1 = tuple((v - 1) // 2 + 1 for v in d0)
    d2 = tuple((v - 1) // 2 + 1 for v in d1)
    return [d0, d1, d2]


def _taps():
    for k in range(27):
        yield k, k % 3 - 1, (k // 3) % 3 - 1, k // 9 - 1


def _window(pad, dx, dy, dz, out_shape, stride):
    Z, Y, X = out_shape
    if stride == 1:
        return pad[1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X]
    return pad[1 + dz:1 + dz + 2 * Z - 1:2, 1 + dy:1 + dy + 2 * Y - 1:2, 1 + dx:1 + dx + 2 * X - 1:2]


def conv(x, W, b, stride, out_shape):
    """3x3x3 convolution with zero padding; x (Z, Y, X, cin)."""
    pad = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.broadcast_to(b, tuple(out_shape) + (W.shape[2],)).astype(np.float64).copy()
    for k, dx, dy, dz in _taps():
        out += _window(pad, dx, dy, dz, out_shape, stride) @ W[k]
    return out


def conv_backward(x, W, g, stride, need_dx=True):
    """(dx, dW, db) for out = conv(x, W, b) and upstream gradient g."""
    out_shape = g.shape[:3]
    pad = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    gpad = np.zeros_like(pad) if need_dx else None
    dW = np.zeros_like(W)
    cin, cout = W.shape[1], W.shape[2]
    g2 = g.reshape(-1, cout)
    for k, dx, dy, dz in _taps():
        win = _window(pad, dx, dy, dz, out_shape, stride)
        dW[k] = win.reshape(-1, cin).T @ g2
        if need_dx:
            _window(gpad, dx, dy, dz, out_shape, stride)[...] += g @ W[k].T
    db = g2.sum(axis=0)
    dx_ = gpad[1:-1, 1:-1, 1:-1] if need_dx else None
    return dx_, dW, db


def _up1(a, axis):
    n = a.shape[axis]
    shape = list(a.shape)
    shape[axis] = 2 * n - 1
    out = np.zeros(shape)
    sl = [slice(None)] * a.ndim
    sl[axis] = slice(0, None, 2)
    out[tuple(sl)] = a
    lo = [slice(None)] * a.ndim
    hi = [slice(None)] * a.ndim
    lo[axis], hi[axis] = slice(0, -1), slice(1, None)
    sl[axis] = slice(1, None, 2)
    out[tuple(sl)] = 0.5 * (a[tuple(lo)] + a[tuple(hi)])
    return out


def _up1_t(g, axis):
    n = (g.shape[axis] + 1) // 2
    sl = [slice(None)] * g.ndim
    sl[axis] = slice(0, None, 2)
    out = g[tuple(sl)].copy()
    odd = [slice(None)] * g.ndim
    odd[axis] = slice(1, None, 2)
    go = 0.5 * g[tuple(odd)]
    lo = [slice(None)] * g.ndim
    hi = [slice(None)] * g.ndim
    lo[axis], hi[axis] = slice(0, n - 1), slice(1, n)
    out[tuple(lo)] += go
    out[tuple(hi)] += go
    return out


def prolong(a):
    """Vertex-centred trilinear prolongation of (Z, Y, X, ch)."""
    return _up1(_up1(_up1(a, 0), 1), 2)


def prolong_t(g):
    return _up1_t(_up1_t(_up1_t(g, 2), 1), 0)


def forward(theta, x, bf16_round=True):
    """Network output (FP64) and the list of stored tensors for ``backward``.
    x: (nz, ny, nx) input grid."""
    rnd = bf16 if bf16_round else (lambda a: np.asarray(a, dtype=np.float64))
    layers = split_params(np.asarray(theta, dtype=np.float32))
    dims = level_dims(x.shape[::-1])
    t = [None] * len(TENSORS)
    t[0] = rnd(x)[..., None]
    for op in ORDER:
        if op >= 0:
            ti, to, stride, act = CONVS[op]
            W, b = layers[op]
            Wr = rnd(W)
            lv = TENSORS[to][0]
            y = conv(t[ti], Wr, b.astype(np.float64), stride, dims[lv][::-1])
            if act:
                y = np.where(y < 0, LEAKY * y, y)
            t[to] = y if to == len(TENSORS) - 1 else rnd(y)
        else:
            ci, si, oi = UPS[-1 - op]
            t[oi] = rnd(prolong(t[ci]) + t[si])
    return t[-1][..., 0], t


def loss_and_grad(out, target, w_l2=1.0, w_h1=0.0):
    """Training loss of one sample and its gradient with respect to out:
    w_l2 mean(d^2) + w_h1 (1/n) sum over axes and neighbour pairs of
    (d[i+e] - d[i])^2, with d = out - target on the (nz, ny, nx) grid."""
    d = np.asarray(out, dtype=np.float64) - target
    n = d.size
    loss = w_l2 * np.sum(d * d) / n
    g = 2.0 * w_l2 * d / n
    for ax in range(3):
        df = np.diff(d, axis=ax)
        loss += w_h1 * np.sum(df * df) / n
        gd = np.zeros_like(d)
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax], hi[ax] = slice(0, -1), slice(1, None)
        gd[tuple(lo)] -= df
        gd[tuple(hi)] += df
        g += 2.0 * w_h1 * gd / n
    return float(loss), g


def backward(theta, t, target, w_l2=1.0, w_h1=0.0):
    """Training loss (``loss_and_grad``) and its gradient with respect to the
    parameters (flat, library layout)."""
    layers = split_params(np.asarray(theta, dtype=np.float32))
    loss, gout = loss_and_grad(t[-1][..., 0], target, w_l2, w_h1)
    g = [None] * len(TENSORS)
    g[-1] = gout[..., None]
    grads = [None] * len(CONVS)
    for op in reversed(ORDER):
        if op >= 0:
            ti, to, stride, act = CONVS[op]
            W, _ = layers[op]
            go = g[to]
            if act:
                go = go * np.where(t[to] > 0, 1.0, LEAKY)
            dx, dW, db = conv_backward(t[ti], bf16(W), go, stride, need_dx=ti != 0)
            grads[op] = (dW, db)
            if ti != 0:
                g[ti] = dx if g[ti] is None else g[ti] + dx
        else:
            ci, si, oi = UPS[-1 - op]
            go = g[oi]
            gc = prolong_t(go)
            g[ci] = gc if g[ci] is None else g[ci] + gc
            g[si] = go if g[si] is None else g[si] + go
    flat = np.concatenate([np.concatenate([dW.ravel(), db.ravel()]) for (dW, db) in grads])
    return loss, flat


def backward_plain(theta, t, target, w_l2=1.0, w_h1=0.0):
    """Gradient of the FP64 network without BF16 rounding (weights used as
    given), for finite-difference checks."""
    layers = split_params(np.asarray(theta, dtype=np.float64))
    loss, gout = loss_and_grad(t[-1][..., 0], target, w_l2, w_h1)
    g = [None] * len(TENSORS)
    g[-1] = gout[..., None]
    grads = [None] * len(CONVS)
    for op in reversed(ORDER):
        if op >= 0:
            ti, to, stride, act = CONVS[op]
            W, _ = layers[op]
            go = g[to]
            if act:
                go = go * np.where(t[to] > 0, 1.0, LEAKY)
            dx, dW, db = conv_backward(t[ti], W, go, stride, need_dx=ti != 0)
            grads[op] = (dW, db)
            if ti != 0:
                g[ti] = dx if g[ti] is None else g[ti] + dx
        else:
            ci, si, oi = UPS[-1 - op]
            go = g[oi]
            gc = prolong_t(go)
            g[ci] = gc if g[ci] is None else g[ci] + gc
            g[si] = go if g[si] is None else g[si] + go
    return loss, np.concatenate([np.concatenate([dW.ravel(), db.ravel()]) for (dW, db) in grads])


def forward_plain(theta, x):
    """FP64 forward without any rounding (theta used in FP64)."""
    layers = split_params(np.asarray(theta, dtype=np.float64))
    dims = level_dims(x.shape[::-1])
    t = [None] * len(TENSORS)
    t[0] = np.asarray(x, dtype=np.float64)[..., None]
    for op in ORDER:
        if op >= 0:
            ti, to, stride, act = CONVS[op]
            W, b = layers[op]
            y = conv(t[ti], W, b, stride, dims[TENSORS[to][0]][::-1])
            if act:
                y = np.where(y < 0, LEAKY * y, y)
            t[to] = y
        else:
            ci, si, oi = UPS[-1 - op]
            t[oi] = prolong(t[ci]) + t[si]
    return t[-1][..., 0], t


def init_params(seed: int) -> np.ndarray:
    """Seeded parameters for tests (numpy Generator; not the library's init)."""
    rng = np.random.default_rng(seed)
    out = []
    for (nw, nb, cin, cout), (_, _, _, act) in zip(layer_shapes(), CONVS):
        sd = np.sqrt(2.0 / (27 * cin)) if act else 0.3 * np.sqrt(1.0 / (27 * cin))
        out.append(rng.normal(0, sd, nw))
        out.append(rng.normal(0, 0.05, nb))
    return np.concatenate(out).astype(np.float32)
