"""The learned surrogate on the GPU: its tensor-core convolutions against the float64 reference
of tests/surrogate_ref.py, then the network's gradients and training.

Inputs and weights are bf16 values, so a convolution's only difference from the reference is the
f32 accumulation of 864 products: agreement to ~1e-6 of the output's scale."""

import ctypes

import numpy as np
import pytest

import surrogate_ref as ref

pytestmark = pytest.mark.gpu


def _t(a, dtype):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dtype).cuda()


def _shape(X, Y, Z, B):
    return (ctypes.c_int32 * 4)(X, Y, Z, B)


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _conv(x, W, b=None, residual=None, relu=0, mask=None, out_ch=0):
    """bfvm_sur_conv3d on bf16 copies of the arrays: (bf16 output, f32 output) as float64."""
    import torch

    from parabiofvm_b200 import _abi

    lib = _abi.load()
    B, Z, Y, X, _ = x.shape
    xt = _t(x, torch.bfloat16)
    wt = _t(W, torch.bfloat16)
    bt = None if b is None else _t(b, torch.float32)
    rt = None if residual is None else _t(residual, torch.bfloat16)
    mt = None if mask is None else _t(mask, torch.bfloat16)
    out = torch.zeros_like(xt)
    of = torch.zeros(x.shape[:4] + (out_ch,), dtype=torch.float32, device="cuda") if out_ch else None
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _abi.check(lib.bfvm_sur_conv3d(_shape(X, Y, Z, B), _ptr(xt), _ptr(wt), _ptr(bt), _ptr(rt), relu, _ptr(mt),
                                   _ptr(out), _ptr(of), None, out_ch, _ptr(err), None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return out.float().cpu().numpy().astype(np.float64), None if of is None else of.cpu().numpy().astype(np.float64)


def _rand_bf16(rng, shape, scale=1.0):
    return ref.bf16((rng.standard_normal(shape) * scale).astype(np.float32)).astype(np.float64)


@pytest.mark.parametrize("shape", [(128, 2, 2, 1), (160, 3, 4, 2), (300, 2, 3, 1)])
def test_conv_matches_reference(shape):
    X, Y, Z, B = shape
    rng = np.random.default_rng(X + Y)
    x = _rand_bf16(rng, (B, Z, Y, X, 32))
    W = _rand_bf16(rng, (27, 32, 32), 0.05)
    b = rng.standard_normal(32).astype(np.float32)
    _, got = _conv(x, W, b, out_ch=32)
    want = ref.conv3d(x, W, b)
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()


def test_conv_epilogue_residual_relu_mask():
    rng = np.random.default_rng(5)
    B, Z, Y, X = 1, 3, 2, 128
    x = _rand_bf16(rng, (B, Z, Y, X, 32))
    W = _rand_bf16(rng, (27, 32, 32), 0.05)
    b = rng.standard_normal(32).astype(np.float32) * 0.1
    res = _rand_bf16(rng, (B, Z, Y, X, 32))
    mask = _rand_bf16(rng, (B, Z, Y, X, 32))
    got, _ = _conv(x, W, b, residual=res, relu=1, mask=mask)
    want = np.maximum(ref.conv3d(x, W, b) + res, 0) * (mask > 0)
    # bf16 output: within half a bf16 unit of the exact value
    assert np.all(np.abs(got - want) <= np.abs(want) * 2.0 ** -8 + 1e-6)


def test_input_gradient_with_flipped_weights():
    rng = np.random.default_rng(6)
    B, Z, Y, X = 2, 3, 3, 128
    g = _rand_bf16(rng, (B, Z, Y, X, 32))
    W = _rand_bf16(rng, (27, 32, 32), 0.05)
    Wt = np.stack([W[26 - t].T for t in range(27)])
    _, got = _conv(g, Wt, out_ch=32)
    want = ref.conv3d_input_grad(g, W)
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()


@pytest.mark.parametrize("shape", [(128, 2, 2, 1), (160, 3, 2, 2)])
def test_weight_gradient_matches_reference(shape):
    import torch

    from parabiofvm_b200 import _abi

    X, Y, Z, B = shape
    rng = np.random.default_rng(7 + X)
    x = _rand_bf16(rng, (B, Z, Y, X, 32))
    g = _rand_bf16(rng, (B, Z, Y, X, 32))
    lib = _abi.load()
    dW = torch.zeros((27, 32, 32), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    xt, gt = _t(x, torch.bfloat16), _t(g, torch.bfloat16)  # held until the kernel has run
    _abi.check(lib.bfvm_sur_conv3d_wgrad(_shape(X, Y, Z, B), _ptr(xt), _ptr(gt), _ptr(dW), _ptr(err), None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    want = ref.conv3d_wgrad(x, g)
    got = dW.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()


# ------------------------------------------------------------------------------------------------
# the network


def _net_problem(seed, grid=(128, 2, 2), S=2, B=1):
    rng = np.random.default_rng(seed)
    X, Y, Z = grid
    field = rng.random((B, Z, Y, X, S)).astype(np.float32)
    src = (rng.random((B, Z, Y, X, S)) * 0.05).astype(np.float32)
    sink = (rng.random((B, Z, Y, X, S)) * 0.05).astype(np.float32)
    target = (field + 0.05 * rng.standard_normal(field.shape)).astype(np.float32)
    return field, src, sink, target


def test_network_gradients_match_reference():
    """bfvm_sur_gradients against the float64 backward pass of the reference on the GPU's own
    bf16-rounded forward activations: the GPU keeps the backward's activations in bf16 as well, so
    the gradients agree to bf16 precision (a few 1e-3 relative), layer by layer."""
    import torch

    from parabiofvm_b200.surrogate import Surrogate

    grid, S = (128, 2, 2), 2
    field, src, sink, target = _net_problem(3, grid, S)
    net = Surrogate(grid, S, max_batch=1, seed=5)
    params = net.save()
    dev = [torch.from_numpy(a.reshape(-1).copy()).cuda() for a in (field, src, sink, target)]
    pred = torch.empty_like(dev[0])
    loss = net.gradients(*dev, pred)
    grads = net.load_gradients().astype(np.float64)
    want_loss, want = ref.gradients(params, field, src, sink, target, round_bf16=True)
    pred_ref, _ = ref.forward(params, field, src, sink, round_bf16=True)
    assert np.abs(pred.cpu().numpy().reshape(pred_ref.shape) - pred_ref).max() <= 1e-3 * np.abs(pred_ref).max()
    assert abs(loss - want_loss) <= 1e-3 * want_loss
    for l in range(ref.LAYERS):
        g = grads[l * ref.LAYER_PARAMS:(l + 1) * ref.LAYER_PARAMS]
        w = want[l * ref.LAYER_PARAMS:(l + 1) * ref.LAYER_PARAMS]
        rel = np.linalg.norm(g - w) / max(np.linalg.norm(w), 1e-30)
        assert rel < 3e-2, (l, rel)
    net.close()


def test_agent_rates_match_numpy():
    import torch

    from parabiofvm_b200.surrogate import Microenvironment, agent_rates, random_agents

    env = Microenvironment((128, 8, 6), 20, [1000.0, 5000.0], [0.1, 0.5], 0.01)
    rng = np.random.default_rng(4)
    a = random_agents(env, rng, 3000)
    dev = {k: torch.from_numpy(np.ascontiguousarray(v, np.float32)).cuda() for k, v in a.items()}
    src = torch.empty(env.voxels * env.S, dtype=torch.float32, device="cuda")
    sink = torch.empty_like(src)
    stream = torch.cuda.current_stream()
    agent_rates((0, 0, 0), (20, 20, 20), env.grid, env.time_step, dev, src, sink, stream)
    torch.cuda.synchronize()
    f = np.float32
    pos = a["pos"].astype(f)
    v = (pos // f(20)).astype(np.int64)
    lin = v[:, 0] + env.grid[0] * (v[:, 1] + env.grid[1] * v[:, 2])
    w = f(env.time_step) * a["vol"].astype(f) / f(8000)
    want_src = np.zeros((env.voxels, env.S))
    want_sink = np.zeros((env.voxels, env.S))
    np.add.at(want_src, lin, a["sec"] * a["sat"] * w[:, None])
    np.add.at(want_sink, lin, (a["upt"] + a["sec"]) * w[:, None])
    np.testing.assert_allclose(src.cpu().numpy().reshape(-1, env.S), want_src, rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(sink.cpu().numpy().reshape(-1, env.S), want_sink, rtol=1e-5, atol=1e-7)


def _env():
    from parabiofvm_b200.surrogate import Microenvironment

    return Microenvironment((128, 16, 16), 20, [2000.0, 20000.0], [0.1, 0.5], 0.01)


def test_training_reduces_the_loss():
    """Adam steps of the project's own kernels on fresh pairs from the plain solver lower the loss
    (a small mesh, so the test stays short; the full training is parabiofvm_b200.surrogate_train)."""
    from parabiofvm_b200.surrogate import PairGenerator, Surrogate, train

    env = _env()
    net = Surrogate(env.grid, env.S, max_batch=2, seed=1)
    gen = PairGenerator(env, seed=2, agents=(500, 3000))
    losses = train(net, gen, steps=300, batch=2, learning_rate=2e-3)
    assert np.mean(losses[-10:]) < 0.5 * np.mean(losses[:3]), losses[:3] + losses[-10:]
    gen.close()
    net.close()


# the trained network's error on pairs outside its training set, as the training run measured it
# (parabiofvm_b200/data/surrogate_128x4.npz: 2,000 pairs, batch 4, Adam lr 1e-3, best of 11 epochs)
TRAINED_HELD_OUT_REL_L2 = 0.0077


def test_trained_network_on_unseen_pairs():
    """The committed network (trained on 2,000 pairs of the standard 128^3 x 4 microenvironment)
    predicts the field 16 plain steps ahead on pairs it has never seen with the relative L2 error
    its training reached, about 13x below the macro-step without a network (the field itself).
    The 1e-3 at which the controller lets it keep control is not reached: the error plateaued near
    8e-3 over the training epochs."""
    import torch

    from parabiofvm_b200 import surrogate as su

    env = su.standard_environment()
    net = su.Surrogate(env.grid, env.S, max_batch=1, seed=0)
    rec = su.load_trained(net, env)
    assert rec["held_out_rel_l2"] < 0.01
    # pairs of the training data set's generator far beyond its 2,000 training pairs
    gen = su.PairGenerator(env, seed=rec["recipe"]["data_seed"])
    err_net, err_none = su.evaluate(net, gen, range(10_000, 10_006))
    print(f"unseen pairs: rel-L2 {err_net:.4e} with the network, {err_none:.4e} without")
    assert err_net < 1.5 * TRAINED_HELD_OUT_REL_L2, err_net
    assert err_net < 0.15 * err_none, (err_net, err_none)
    torch.cuda.synchronize()
    gen.close()
    net.close()


def test_fallback_controller():
    """Tolerance 0: the first check hands control to the plain solver, and the whole run equals
    plain stepping.  An unreachable tolerance: the surrogate keeps control between checks."""
    import torch

    from parabiofvm_b200.surrogate import Surrogate, random_agents, random_field, run_with_fallback

    env = _env()
    net = Surrogate(env.grid, env.S, max_batch=1, seed=3)
    rng = np.random.default_rng(8)
    agents = random_agents(env, rng, 2000)
    field0 = torch.empty(env.voxels * env.S, device="cuda")
    random_field(env.grid, env.S, rng, field0, torch.cuda.current_stream())

    field = field0.clone()
    rep = run_with_fallback(net, env, field, agents, macro_steps=3, check_every=1, tolerance=0.0)
    assert rep.fell_back_at == 0 and rep.surrogate_steps == 0 and len(rep.checks) == 1
    s = env.solver()
    s.store_densities(field0.cpu().numpy())
    a = agents
    s.store_agents(a["sec"], a["sat"], a["upt"], a["nex"], np.zeros_like(a["sec"]), None, a["vol"], a["pos"])
    s.run_steps(48)
    np.testing.assert_array_equal(field.cpu().numpy(), s.load_densities())
    s.close()

    field = field0.clone()
    rep = run_with_fallback(net, env, field, agents, macro_steps=8, check_every=4, tolerance=1e30)
    assert rep.fell_back_at == -1 and rep.surrogate_steps == 6 and [m for m, _ in rep.checks] == [3, 7]
    assert torch.isfinite(field).all()
    net.close()
