"""The learned surrogate (bfvm_sur_*): a 3D convolutional operator that advances a field 16 steps
at once, trained on the GPU on pairs the plain solver generates, and run under a controller that
checks it against the plain solver and hands control back when it drifts.

- ``Surrogate`` wraps the network of csrc/surrogate_net.cu (tensor-core convolutions, Adam).
- ``PairGenerator`` makes training pairs: a random field (sums of Gaussian bumps), random agents,
  their voxelised secretion terms, and the field 16 plain steps later (bfvm_run_steps).
- ``train`` runs Adam steps on freshly generated batches.
- ``run_with_fallback`` advances a microenvironment in macro-steps of 16: the surrogate steps
  it, every ``check_every``-th macro-step the plain solver re-runs the same interval from the same
  state and, if the surrogate's relative L2 error against it exceeds ``tolerance``, plain stepping
  takes over for good.

Device buffers are torch tensors (plumbing); every computation runs in this library's kernels.
"""

from __future__ import annotations

import ctypes
import dataclasses
import json
import os
import time

import numpy as np

from . import Solver, _abi
from ._abi import check

MACRO_STEPS = 16


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _i3(v):
    return (ctypes.c_int32 * 3)(*[int(x) for x in v])


class Surrogate:
    """The network for fields of `substrates` on a mesh of `grid` voxels (x at least 128), in
    batches of up to `max_batch`."""

    def __init__(self, grid, substrates, max_batch=1, seed=0, device=0, stream=None):
        import torch

        self._lib = _abi.load()
        self.grid = tuple(int(g) for g in grid)
        self.S = int(substrates)
        self.max_batch = int(max_batch)
        self.voxels = self.grid[0] * self.grid[1] * self.grid[2]
        h = ctypes.c_void_p()
        check(self._lib.bfvm_sur_create(ctypes.byref(h), int(device), _i3(self.grid), self.S, self.max_batch,
                                        ctypes.c_uint64(int(seed))))
        self._h = h
        self.stream = stream if stream is not None else torch.cuda.Stream(torch.device("cuda", int(device)))
        check(self._lib.bfvm_sur_set_stream(self._h, ctypes.c_void_p(self.stream.cuda_stream)))
        n = ctypes.c_int64()
        check(self._lib.bfvm_sur_parameter_count(self._h, ctypes.byref(n)))
        self.parameter_count = int(n.value)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.bfvm_sur_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def save(self):
        out = np.empty(self.parameter_count, np.float32)
        check(self._lib.bfvm_sur_save(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def load(self, params):
        p = np.ascontiguousarray(params, np.float32).reshape(-1)
        if p.size != self.parameter_count:
            raise ValueError(f"expected {self.parameter_count} parameters")
        check(self._lib.bfvm_sur_load(self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def _batch(self, field):
        b = field.numel() // (self.voxels * self.S)
        if b * self.voxels * self.S != field.numel() or not 1 <= b <= self.max_batch:
            raise ValueError("fields must hold [batch][voxels][substrates] floats, batch 1..max_batch")
        return b

    def infer(self, field, sources, sinks, out):
        check(self._lib.bfvm_sur_infer(self._h, self._batch(field), _p(field), _p(sources), _p(sinks), _p(out)))

    def gradients(self, field, sources, sinks, target, prediction):
        loss = ctypes.c_float()
        check(self._lib.bfvm_sur_gradients(self._h, self._batch(field), _p(field), _p(sources), _p(sinks),
                                           _p(target), _p(prediction), ctypes.byref(loss)))
        return float(loss.value)

    def load_gradients(self):
        out = np.empty(self.parameter_count, np.float32)
        check(self._lib.bfvm_sur_load_gradients(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def train_step(self, field, sources, sinks, target, prediction, learning_rate=1e-3, read_loss=True):
        loss = ctypes.c_float()
        check(self._lib.bfvm_sur_train_step(self._h, self._batch(field), _p(field), _p(sources), _p(sinks),
                                            _p(target), _p(prediction), float(learning_rate),
                                            ctypes.byref(loss) if read_loss else None))
        return float(loss.value) if read_loss else None

    def synchronize(self):
        check(self._lib.bfvm_sur_synchronize(self._h))


def agent_rates(bbox_min, voxel_shape, grid, dt, agents, sources, sinks, stream):
    """One step's secretion terms per voxel (bfvm_sur_agent_rates) into device tensors; `agents`
    holds device tensors sec, sat, upt, nex [A][S], vol [A], pos [A][3]."""
    lib = _abi.load()
    A = int(agents["vol"].numel())
    S = sources.numel() // (grid[0] * grid[1] * grid[2])
    check(lib.bfvm_sur_agent_rates(_i3(bbox_min), _i3(voxel_shape), _i3(grid), S, float(dt), A,
                                   *[_p(agents[k]) for k in ("sec", "sat", "upt", "nex", "vol", "pos")],
                                   _p(sources), _p(sinks), None, ctypes.c_void_p(stream.cuda_stream)))


def random_field(grid, S, rng, out, stream, bumps=8):
    """A sum of `bumps` Gaussian bumps per substrate (widths 4..16 voxels, amplitudes U(0,1))."""
    lib = _abi.load()
    p = np.empty((S, bumps, 5), np.float32)
    for d in range(3):
        p[..., d] = rng.uniform(0, grid[d], (S, bumps))
    p[..., 3] = rng.uniform(4, 16, (S, bumps))
    p[..., 4] = rng.uniform(0, 1, (S, bumps))
    check(lib.bfvm_sur_random_field(_i3(grid), S, bumps, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), _p(out),
                                    ctypes.c_void_p(stream.cuda_stream)))


@dataclasses.dataclass
class Microenvironment:
    """A mesh with per-substrate coefficients (no Dirichlet conditions), as the surrogate sees it."""
    grid: tuple
    dx: int
    diffusion_coefficients: list
    decay_rates: list
    time_step: float

    @property
    def S(self):
        return len(self.diffusion_coefficients)

    @property
    def voxels(self):
        return self.grid[0] * self.grid[1] * self.grid[2]

    def solver(self, device=0):
        return Solver(3, (0, 0, 0), tuple(g * self.dx for g in self.grid), (self.dx,) * 3,
                      self.diffusion_coefficients, self.decay_rates, self.time_step, device=device)


STANDARD_SEED = 20261205
WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "surrogate_128x4.npz")


def standard_environment(seed=STANDARD_SEED):
    """The 128^3 x 4 microenvironment the surrogate is trained and measured on: dx 20 um, dt 0.01
    min, diffusion coefficients log-uniform in [1e3, 1e5] um^2/min and decay rates uniform in
    [0.01, 1] /min, drawn from `seed`."""
    rng = np.random.default_rng(seed)
    S = 4
    return Microenvironment((128, 128, 128), 20, [float(x) for x in np.exp(rng.uniform(np.log(1e3), np.log(1e5), S))],
                            [float(x) for x in rng.uniform(0.01, 1.0, S)], 0.01)


def load_trained(net, env, path=WEIGHTS_PATH):
    """Load the trained parameters of `path` into `net` after checking that they were trained for
    `env` (grid, voxel size, time step and coefficients).  Returns the file's training record."""
    with np.load(path) as f:
        params = f["parameters"]
        record = json.loads(str(f["record"]))
    want = {"grid": list(env.grid), "dx": env.dx, "time_step": env.time_step,
            "diffusion_coefficients": env.diffusion_coefficients, "decay_rates": env.decay_rates}
    got = record["environment"]
    if (got["grid"] != want["grid"] or got["dx"] != want["dx"] or not np.isclose(got["time_step"], want["time_step"])
            or not np.allclose(got["diffusion_coefficients"], want["diffusion_coefficients"], rtol=1e-6)
            or not np.allclose(got["decay_rates"], want["decay_rates"], rtol=1e-6)):
        raise ValueError(f"{path} was trained for another microenvironment: {got}")
    net.load(params)
    return record


def random_agents(env, rng, count, clustered=False):
    """Agents with the plain workloads' distributions: volume 1000, secretion U(0,10), saturation
    U(0,1), uptake U(0,1), net export 0; uniform or in 16 Gaussian clusters."""
    L = np.array(env.grid, np.float64) * env.dx
    if clustered:
        centres = rng.uniform(0, L, (16, 3))
        pos = centres[rng.integers(0, 16, count)] + rng.normal(0, 4 * env.dx, (count, 3))
        pos = np.clip(pos, 0, L * (1 - 1e-6))
    else:
        pos = rng.uniform(0, L, (count, 3))
    S = env.S
    return dict(sec=rng.uniform(0, 10, (count, S)), sat=rng.uniform(0, 1, (count, S)),
                upt=rng.uniform(0, 1, (count, S)), nex=np.zeros((count, S)), vol=np.full(count, 1000.0),
                pos=np.minimum(pos.astype(np.float32), np.nextafter(L.astype(np.float32), 0)))


class PairGenerator:
    """Training pairs from the plain solver: (field, sources, sinks) -> the field 16 steps later.

    ``fill`` draws a fresh pair from the generator's own sequence; ``fill(..., pair=k)`` makes pair
    k of a fixed data set instead: its field and agents come from a generator seeded with
    (seed, k), and the plain solver is deterministic, so the same k gives the same pair every time
    (a data set of any size costs no memory, only the time to regenerate it)."""

    def __init__(self, env, seed=0, agents=(10_000, 100_000), device=0, stream=None):
        import torch

        self.env = env
        self.seed = int(seed)
        self.rng = np.random.default_rng(seed)
        self.agents = agents
        self.stream = stream if stream is not None else torch.cuda.Stream()
        self.solver = env.solver(device)
        self.solver.set_stream(self.stream.cuda_stream)
        self.device = torch.device("cuda", int(device))

    def close(self):
        self.solver.close()

    def fill(self, field, sources, sinks, target, pair=None):
        """One pair into views of [voxels][S] of device tensors: pair `pair` of the fixed data set,
        or the next fresh pair when `pair` is None."""
        import torch

        env = self.env
        rng = self.rng if pair is None else np.random.default_rng((self.seed, int(pair)))
        with torch.cuda.stream(self.stream):
            random_field(env.grid, env.S, rng, field, self.stream)
            count = int(rng.integers(self.agents[0], self.agents[1] + 1))
            a = random_agents(env, rng, count)
            dev = {k: torch.from_numpy(np.ascontiguousarray(v, np.float32)).to(self.device, non_blocking=False)
                   for k, v in a.items()}
            agent_rates((0, 0, 0), (env.dx,) * 3, env.grid, env.time_step, dev, sources, sinks, self.stream)
            self.solver.store_densities_device(field)
            self.solver.store_agents(a["sec"], a["sat"], a["upt"], a["nex"], np.zeros_like(a["sec"]), None, a["vol"],
                                     a["pos"])
            self.solver.run_steps(MACRO_STEPS, 0)
            self.solver.load_densities_device(target)
            self._keep = dev  # the agent tensors stay alive until the stream has used them

    def batch(self, field, sources, sinks, target, pairs=None):
        for b in range(field.shape[0]):
            self.fill(field[b], sources[b], sinks[b], target[b], None if pairs is None else pairs[b])


def train(net, gen, steps, batch=4, learning_rate=1e-3, log_every=0, log=print):
    """`steps` Adam steps, each on `batch` fresh pairs; returns the losses."""
    import torch

    env = gen.env
    shape = (batch, env.voxels * env.S)
    with torch.cuda.stream(net.stream):
        bufs = [torch.empty(shape, dtype=torch.float32, device=gen.device) for _ in range(5)]
    field, src, sink, target, pred = bufs
    losses = []
    for it in range(steps):
        gen.batch(field, src, sink, target)
        net.stream.wait_stream(gen.stream)
        losses.append(net.train_step(field, src, sink, target, pred, learning_rate))
        gen.stream.wait_stream(net.stream)
        if log_every and (it + 1) % log_every == 0:
            log(f"surrogate step {it + 1}: loss {losses[-1]:.3e}")
    return losses


def train_on_pairs(net, gen, pairs, epochs, batch=4, learning_rate=1e-3, held_out=(), seed=0, log=None):
    """Adam on a fixed data set: pairs 0..pairs-1 of `gen`, `epochs` passes in a shuffled order,
    `batch` pairs per step.  After every epoch the network is evaluated on the pairs listed in
    `held_out` (indices outside the training set).  Returns a list of per-epoch dicts: mean loss,
    and on the held-out pairs the network's mean relative L2 error against the plain solver next to
    that of the field itself (the macro-step without a network)."""
    import torch

    env = gen.env
    shape = (batch, env.voxels * env.S)
    with torch.cuda.stream(net.stream):
        field, src, sink, target, pred = [torch.empty(shape, dtype=torch.float32, device=gen.device)
                                          for _ in range(5)]
    order_rng = np.random.default_rng(seed)
    curve = []
    t0 = time.perf_counter()
    for epoch in range(epochs):
        order = order_rng.permutation(pairs)
        losses = []
        for i in range(0, pairs - batch + 1, batch):
            gen.batch(field, src, sink, target, pairs=order[i:i + batch])
            net.stream.wait_stream(gen.stream)
            losses.append(net.train_step(field, src, sink, target, pred, learning_rate))
            gen.stream.wait_stream(net.stream)
        net_err, none_err = evaluate(net, gen, held_out) if len(held_out) else (None, None)
        curve.append({"epoch": epoch + 1, "steps": (epoch + 1) * (pairs // batch), "loss_mean": float(np.mean(losses)),
                      "loss_last": float(losses[-1]), "held_out_rel_l2": net_err, "held_out_rel_l2_without_net": none_err,
                      "seconds": time.perf_counter() - t0})
        if log:
            log(json.dumps(curve[-1]))
    return curve


def evaluate(net, gen, pairs):
    """Mean relative L2 error on the listed pairs of `gen`, of the network's prediction and of the
    field itself, both against the plain solver's field 16 steps later."""
    import torch

    env = gen.env
    with torch.cuda.stream(net.stream):
        field, src, sink, target, pred = [torch.empty((1, env.voxels * env.S), dtype=torch.float32,
                                                      device=gen.device) for _ in range(5)]
    errs_net, errs_none = [], []
    for k in pairs:
        gen.batch(field, src, sink, target, pairs=[k])
        net.stream.wait_stream(gen.stream)
        net.infer(field, src, sink, pred)
        net.synchronize()
        errs_net.append(rel_l2(pred, target))
        errs_none.append(rel_l2(field, target))
        gen.stream.wait_stream(net.stream)
    return float(np.mean(errs_net)), float(np.mean(errs_none))


def rel_l2(a, b):
    import torch

    return float(torch.linalg.vector_norm(a - b) / torch.clamp(torch.linalg.vector_norm(b), min=1e-30))


@dataclasses.dataclass
class FallbackReport:
    macro_steps: int
    surrogate_steps: int
    checks: list            # (macro step, relative L2 error of the surrogate against plain)
    fell_back_at: int       # macro step where plain stepping took over, or -1
    seconds: float


def run_with_fallback(net, env, field, agents, macro_steps, check_every=8, tolerance=1e-3, device=0, stream=None):
    """Advance `field` (device tensor [voxels][S], updated in place) by macro_steps x 16 steps with
    the agents fixed.  The surrogate takes a macro-step at a time; every check_every-th
    macro-step the plain solver re-runs the same 16 steps from the same state, its result is kept,
    and if the surrogate's relative L2 error against it is above `tolerance` the remaining
    macro-steps run plain.  Returns a FallbackReport."""
    import torch

    stream = stream if stream is not None else net.stream
    solver = env.solver(device)
    solver.set_stream(stream.cuda_stream)
    a = agents
    solver.store_agents(a["sec"], a["sat"], a["upt"], a["nex"], np.zeros_like(a["sec"]), None, a["vol"], a["pos"])
    dev = {k: torch.from_numpy(np.ascontiguousarray(v, np.float32)).to(field.device) for k, v in a.items()}
    with torch.cuda.stream(stream):
        src = torch.empty_like(field)
        sink = torch.empty_like(field)
        pred = torch.empty_like(field)
        plain = torch.empty_like(field)
    agent_rates((0, 0, 0), (env.dx,) * 3, env.grid, env.time_step, dev, src, sink, stream)
    checks = []
    fell_back = -1
    surrogate_steps = 0
    step = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        for m in range(macro_steps):
            if fell_back >= 0:
                solver.run_steps(MACRO_STEPS, step)
                step += MACRO_STEPS
                continue
            if m % check_every == check_every - 1:
                solver.store_densities_device(field)
                net.infer(field, src, sink, pred)
                solver.run_steps(MACRO_STEPS, step)
                solver.load_densities_device(plain)
                err = rel_l2(pred, plain)
                checks.append((m, err))
                field.copy_(plain)
                if err > tolerance:
                    fell_back = m
                    solver.store_densities_device(field)
            else:
                net.infer(field, src, sink, pred)
                field.copy_(pred)
                surrogate_steps += 1
            step += MACRO_STEPS
        if fell_back >= 0:
            solver.load_densities_device(field)
    torch.cuda.synchronize()
    seconds = time.perf_counter() - t0
    solver.close()
    return FallbackReport(macro_steps, surrogate_steps, checks, fell_back, seconds)
