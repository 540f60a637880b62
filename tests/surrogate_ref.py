"""CPU reference of the learned surrogate (test infrastructure): the 3x3x3 convolutions, the
network's forward and backward passes and the loss, in float64 numpy without autograd.

The GPU keeps weights and activations in bf16 with f32 accumulation; `bf16` rounds an array the
same way (round to nearest even), so the reference can reproduce the GPU's rounding points where a
test needs it.  Layouts follow include/bfvm.h: activations [B][Z][Y][X][32], weights
[27][32 out][32 in] with tap t = 9 (dz+1) + 3 (dy+1) + (dx+1).
"""

import numpy as np

C = 32
TAPS = 27
LAYERS = 10
LAYER_PARAMS = TAPS * C * C + C
FEATURE_SCALE = 16.0


def bf16(a):
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def offsets(t):
    return t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1


def _shifted(x, t):
    """x[v + off_t] with zeros outside, for x [B][Z][Y][X][C]."""
    dz, dy, dx = offsets(t)
    B, Z, Y, X, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    return xp[:, 1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X, :]


def conv3d(x, W, b=None):
    """out[v][co] = sum_t sum_ci W[t][co][ci] x[v + off_t][ci] (+ b[co])."""
    x = np.asarray(x, np.float64)
    out = np.zeros(x.shape[:4] + (W.shape[1],))
    for t in range(TAPS):
        out += _shifted(x, t) @ np.asarray(W[t], np.float64).T
    if b is not None:
        out += b
    return out


def conv3d_wgrad(x, g):
    """dW[t][co][ci] = sum_v g[v][co] x[v + off_t][ci]."""
    x = np.asarray(x, np.float64)
    g = np.asarray(g, np.float64)
    dW = np.zeros((TAPS, g.shape[-1], x.shape[-1]))
    for t in range(TAPS):
        dW[t] = np.einsum("bzyxo,bzyxi->oi", g, _shifted(x, t))
    return dW


def conv3d_input_grad(g, W):
    """d/dx of sum(g * conv3d(x, W)): the convolution of g with the flipped, transposed weights."""
    Wt = np.stack([np.asarray(W[TAPS - 1 - t], np.float64).T for t in range(TAPS)])
    return conv3d(g, Wt)


def split_params(params):
    p = np.asarray(params, np.float64).reshape(LAYERS, LAYER_PARAMS)
    return [(p[l, :TAPS * C * C].reshape(TAPS, C, C), p[l, TAPS * C * C:]) for l in range(LAYERS)]


def features(field, src, sink, dtype=np.float32):
    """[B][Z][Y][X][32]: field, 16 x sources, 16 x sinks, zeros (field etc. [B][Z][Y][X][S])."""
    S = field.shape[-1]
    f = np.zeros(field.shape[:4] + (C,), dtype)
    f[..., :S] = field
    f[..., S:2 * S] = np.asarray(src, dtype) * dtype(FEATURE_SCALE)
    f[..., 2 * S:3 * S] = np.asarray(sink, dtype) * dtype(FEATURE_SCALE)
    return f


def forward(params, field, src, sink, round_bf16=True):
    """The network (surrogate_net.cu): returns the prediction and the activations.  With
    round_bf16 the weights, features and stored activations are rounded as the GPU rounds them."""
    if round_bf16:
        def r(a):
            return bf16(np.asarray(a, np.float32)).astype(np.float64)
    else:
        def r(a):
            return np.asarray(a, np.float64)
    layers = split_params(params)
    W = [(r(w), b) for w, b in layers]
    S = field.shape[-1]
    feat = r(features(field, src, sink, np.float32 if round_bf16 else np.float64))
    h = [None] * 5
    t = [None] * 4
    h[0] = r(np.maximum(conv3d(feat, *W[0]), 0))
    for k in range(4):
        t[k] = r(np.maximum(conv3d(h[k], *W[2 * k + 1]), 0))
        h[k + 1] = r(conv3d(t[k], *W[2 * k + 2]) + h[k])
    proj = conv3d(h[4], *W[9])
    pred = np.asarray(field, np.float64) + proj[..., :S]
    return pred, dict(feat=feat, h=h, t=t, W=W)


def gradients(params, field, src, sink, target, round_bf16=False):
    """Mean squared error and its gradient with respect to every parameter, in the parameter
    layout, by the backward pass of the network (no autograd)."""
    pred, a = forward(params, field, src, sink, round_bf16)
    S = field.shape[-1]
    n = pred.size
    diff = pred - target
    loss = float(np.mean(diff ** 2))
    g = np.zeros(pred.shape[:4] + (C,))
    g[..., :S] = 2 * diff / n
    grads = [None] * LAYERS
    W, h, t = a["W"], a["h"], a["t"]

    def layer_grad(x, gy):
        return np.concatenate([conv3d_wgrad(x, gy).reshape(-1), gy.sum(axis=(0, 1, 2, 3))])

    grads[9] = layer_grad(h[4], g)
    gh = conv3d_input_grad(g, W[9][0])
    for k in range(3, -1, -1):
        grads[2 * k + 2] = layer_grad(t[k], gh)
        gt = conv3d_input_grad(gh, W[2 * k + 2][0]) * (t[k] > 0)
        grads[2 * k + 1] = layer_grad(h[k], gt)
        gh = gh + conv3d_input_grad(gt, W[2 * k + 1][0])
        if k == 0:
            gh = gh * (h[0] > 0)
    grads[0] = layer_grad(a["feat"], gh)
    return loss, np.concatenate(grads)


def loss_of(params, field, src, sink, target):
    pred, _ = forward(params, field, src, sink, round_bf16=False)
    return float(np.mean((pred - target) ** 2))
