"""The CPU reference of the learned surrogate (tests/surrogate_ref.py) against itself: its
backward pass against central finite differences in float64, and the convolution identities the
GPU kernels rely on (the input gradient as a convolution with flipped, transposed weights)."""

import numpy as np

import surrogate_ref as ref


def _problem(seed, shape=(1, 3, 3, 4), S=2):
    rng = np.random.default_rng(seed)
    B, Z, Y, X = shape
    field = rng.random((B, Z, Y, X, S))
    src = rng.random((B, Z, Y, X, S)) * 0.05
    sink = rng.random((B, Z, Y, X, S)) * 0.05
    target = field + 0.1 * rng.standard_normal(field.shape)
    params = rng.standard_normal(ref.LAYERS * ref.LAYER_PARAMS) * 0.05
    return params, field, src, sink, target


def test_backward_matches_finite_differences():
    params, field, src, sink, target = _problem(1)
    loss, grads = ref.gradients(params, field, src, sink, target)
    assert np.isclose(loss, ref.loss_of(params, field, src, sink, target))
    rng = np.random.default_rng(2)
    # a few weights and biases of every layer
    picks = []
    for l in range(ref.LAYERS):
        base = l * ref.LAYER_PARAMS
        picks += list(base + rng.integers(0, ref.TAPS * ref.C * ref.C, 3)) + [base + ref.TAPS * ref.C * ref.C + 1]
    h = 1e-6
    for i in picks:
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        fd = (ref.loss_of(p1, field, src, sink, target) - ref.loss_of(p2, field, src, sink, target)) / (2 * h)
        assert abs(fd - grads[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, grads[i])


def test_input_gradient_is_the_flipped_convolution():
    rng = np.random.default_rng(3)
    x = rng.standard_normal((2, 3, 4, 5, ref.C))
    W = rng.standard_normal((ref.TAPS, ref.C, ref.C))
    g = rng.standard_normal((2, 3, 4, 5, ref.C))
    # <g, conv(x)> = <conv_input_grad(g), x> = <wgrad(x, g), W>
    lhs = float(np.sum(g * ref.conv3d(x, W)))
    assert np.isclose(lhs, float(np.sum(ref.conv3d_input_grad(g, W) * x)))
    assert np.isclose(lhs, float(np.sum(ref.conv3d_wgrad(x, g) * W)))


def test_bf16_rounding():
    a = np.array([1.0, 1.00390625, 1.005859375, -2.5e-3, 3.0e38], np.float32)
    r = ref.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == np.float32(1.0078125)
    assert abs(r[3] - a[3]) <= abs(a[3]) * 2 ** -8
