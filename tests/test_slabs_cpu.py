"""z-slabs on the CPU: the library's slab coupling coefficients (bfvm_slab_coefficients, host code)
and the exchange protocol of parabiofvm_b200.slabs over gloo, checked against the Thomas solve of
whole z lines (src/solver/host/diffusion_solver.cpp:72-142, 416-480) and the central-difference z
gradient (src/solver/host/gradient_solver.cpp:170-223).

The slab arithmetic here is a float64 restatement of what the GPU passes do: the reduce pass as
weighted sums with the library's weights (bfvm_slab_reduce_weights), the combine recurrences, and
the solve pass with carries.  The GPU passes themselves are checked against the single-solver step
in tests/test_gpu_slabs.py.
"""

import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def thomas_coefficients(n, h, dims, dt, D, lam):
    """float32 b' [n][S] and c [S] in the reference's operation order."""
    f = np.float32
    D = np.asarray(D, f)
    lam = np.asarray(lam, f)
    c = (-f(dt) * D / f(h * h)).astype(f)
    ends = (f(1) + lam * f(dt) / f(dims) + f(dt) * D / f(h * h)).astype(f)
    mid = (f(1) + lam * f(dt) / f(dims) + f(2) * f(dt) * D / f(h * h)).astype(f)
    b = np.stack([ends if i in (0, n - 1) else mid for i in range(n)])
    bp = np.empty_like(b)
    bp[0] = f(1) / b[0]
    for i in range(1, n):
        bp[i] = f(1) / (b[i] - c * c * bp[i - 1])
    return bp, c


def expand(a, lines):
    """Per-substrate values [..., S] to per-line values [..., lines], line l holding substrate l % S."""
    S = a.shape[-1]
    return np.take(a.astype(np.float64), np.arange(lines) % S, axis=-1)


def slab_solve(d, bp, c, i0, i1, C=None, X=None):
    """Thomas solve of elements [i0, i1) of lines d [i1 - i0][L] (float64), entered with the left
    carry C = d'_{i0-1} and the right carry X = x_{i1} (zero when None).  Returns x and the forward
    values d'."""
    L = d.shape[1]
    b = expand(bp, L)
    e = expand((c[None, :] * bp).astype(np.float32), L)  # e_i = c b'_i, the float product
    cc = expand(c[None, :], L)[0]
    f = np.array(d, np.float64)
    if C is not None and i0 > 0:
        f[0] = f[0] - e[i0 - 1] * C
    for i in range(1, i1 - i0):
        f[i] = f[i] - e[i0 + i - 1] * f[i - 1]
    x = np.empty_like(f)
    last = i1 - i0 - 1
    x[last] = (f[last] - (cc * X if X is not None else 0.0)) * b[i1 - 1]
    for i in range(last - 1, -1, -1):
        x[i] = (f[i] - cc * x[i + 1]) * b[i0 + i]
    return x, f


def combine(A, B, coef, me, lines):
    """The carries (C, X) of slab `me` from every slab's (A, B) [count][L] and the coefficients
    [count][3][S]: C_{k+1} = A_k + Gamma_k C_k, X_{k-1} = B_k + beta_k C_k + Lambda_k X_k."""
    count = len(A)
    Ck = [np.zeros(lines)]
    for k in range(count - 1):
        Ck.append(A[k] + expand(coef[k, 0], lines) * Ck[k])
    X = np.zeros(lines)
    for k in range(count - 1, me, -1):
        X = B[k] + expand(coef[k, 1], lines) * Ck[k] + expand(coef[k, 2], lines) * X
    return Ck[me], X


MESH = dict(n=100, h=20, dims=3, dt=0.01, D=[1000.0, 20000.0, 50.0], lam=[0.1, 1.0, 0.01])


def _line_problem(seed, lines=12):
    rng = np.random.default_rng(seed)
    return rng.random((MESH["n"], lines))


def test_plan_slabs():
    from parabiofvm_b200.slabs import plan_slabs

    assert plan_slabs(10, 3) == [0, 4, 7, 10]
    assert plan_slabs(320, 8) == [0, 40, 80, 120, 160, 200, 240, 280, 320]
    with pytest.raises(ValueError):
        plan_slabs(5, 3)


def test_agent_slabs_follow_the_voxel_planes():
    from parabiofvm_b200.slabs import agent_slabs

    bounds = [0, 3, 5, 9]  # planes of 20 voxels each, mesh from z = -40
    z = np.array([-40.0, -40.0 + 59.999, 20.0, 60.0 - 1e-3, 60.0, 139.99, -45.0, 140.0], np.float32)
    pos = np.stack([np.zeros_like(z), np.zeros_like(z), z], axis=1)
    # voxel planes: z = -40 + 20 k; slab 0 holds planes 0..2 ([-40, 20)), slab 1 planes 3..4, slab 2 5..8;
    # (-60, -40) truncates into plane 0 like the solver's lookup, z >= 140 lies outside
    assert agent_slabs(pos, -40, 20, bounds).tolist() == [0, 0, 1, 1, 2, 2, 0, -1]


@pytest.mark.parametrize("bounds", [[0, 100], [0, 50, 100], [0, 7, 40, 41 + 32, 100], [0, 2, 4, 6, 98, 100]])
def test_coefficients_join_slabs_into_the_whole_line_solve(bounds):
    from parabiofvm_b200.slabs import slab_coefficients

    n = MESH["n"]
    bp, c = thomas_coefficients(n, MESH["h"], MESH["dims"], MESH["dt"], MESH["D"], MESH["lam"])
    coef = slab_coefficients(n, MESH["h"], MESH["D"], MESH["lam"], MESH["dt"], bounds)
    d = _line_problem(1)
    L = d.shape[1]
    whole, _ = slab_solve(d, bp, c, 0, n)
    count = len(bounds) - 1
    A, B = [], []
    for k in range(count):
        x, f = slab_solve(d[bounds[k]:bounds[k + 1]], bp, c, bounds[k], bounds[k + 1])
        A.append(f[-1])
        B.append(x[0])
    parts = []
    for k in range(count):
        C, X = combine(A, B, coef, k, L)
        x, _ = slab_solve(d[bounds[k]:bounds[k + 1]], bp, c, bounds[k], bounds[k + 1], C, X)
        parts.append(x)
    joined = np.concatenate(parts)
    # the coefficients are float32: a few units in the last place of the carries
    np.testing.assert_allclose(joined, whole, rtol=2e-6, atol=1e-7 * np.abs(whole).max())


def test_coefficients_reject_bad_bounds():
    from parabiofvm_b200._abi import BfvmError
    from parabiofvm_b200.slabs import slab_coefficients

    with pytest.raises(BfvmError):
        slab_coefficients(10, 20, [1.0], [0.1], 0.01, [0, 5, 5, 10])
    with pytest.raises(BfvmError):
        slab_coefficients(10, 20, [1.0], [0.1], 0.01, [0, 4, 9])


# ------------------------------------------------------------------------------------------------
# the exchange protocol of slabs.step over gloo, with slabs that run the restated arithmetic


class RestatedSlab:
    """A slab of lines [n][L] whose passes are the float64 restatement above, with the buffers and
    methods slabs.step drives (the field is one z line per (y, x, s) column, no x or y extent)."""

    def __init__(self, d, bounds, index):
        import torch

        from parabiofvm_b200.slabs import slab_coefficients, slab_reduce_weights

        self.bounds, self.index, self.count = bounds, index, len(bounds) - 1
        self.i0, self.i1 = bounds[index], bounds[index + 1]
        self.bp, self.c = thomas_coefficients(MESH["n"], MESH["h"], MESH["dims"], MESH["dt"], MESH["D"], MESH["lam"])
        self.coef = slab_coefficients(MESH["n"], MESH["h"], MESH["D"], MESH["lam"], MESH["dt"], bounds)
        # the reduce pass as the GPU runs it: sums over the planes whose weights the library keeps
        self.a_first, self.wa, self.wb = slab_reduce_weights(MESH["n"], MESH["h"], MESH["D"], MESH["lam"], MESH["dt"],
                                                             self.i0, self.i1)
        self.u = np.array(d[self.i0:self.i1], np.float64)
        self.lines = d.shape[1]
        self.exchange = torch.zeros(2 * self.lines, dtype=torch.float32)
        self.edges = torch.zeros((2, self.lines), dtype=torch.float32)
        self.grad = None

    def diffusion_begin(self):
        import torch

        L = self.lines
        A = np.einsum("kl,kl->l", expand(self.wa, L), self.u[self.a_first - self.i0:]) if len(self.wa) else np.zeros(L)
        B = np.einsum("kl,kl->l", expand(self.wb, L), self.u[:len(self.wb)]) if len(self.wb) else np.zeros(L)
        self.exchange.copy_(torch.from_numpy(np.concatenate([A, B]).astype(np.float32)))

    def diffusion_end(self, gathered):
        g = gathered.numpy().astype(np.float64).reshape(self.count, 2, self.lines)
        C, X = combine(g[:, 0], g[:, 1], self.coef, self.index, self.lines)
        self.u, _ = slab_solve(self.u, self.bp, self.c, self.i0, self.i1, C, X)

    def edge_planes(self):
        import torch

        self.edges.copy_(torch.from_numpy(np.stack([self.u[0], self.u[-1]]).astype(np.float32)))

    def gradient_with(self, below, above):
        h = np.float64(MESH["h"])
        ext = [below.numpy().astype(np.float64)[None]] if below is not None else []
        ext.append(self.u)
        if above is not None:
            ext.append(above.numpy().astype(np.float64)[None])
        v = np.concatenate(ext)
        off = 1 if below is not None else 0
        g = np.empty_like(self.u)
        for z in range(self.u.shape[0]):
            k = z + off
            if k == 0:
                g[z] = (v[1] - v[0]) / h
            elif k == len(v) - 1:
                g[z] = (v[k] - v[k - 1]) / h
            else:
                g[z] = (v[k + 1] - v[k - 1]) / (2 * h)
        self.grad = g

    def secretion(self, recompute):
        pass


def _rank_main(rank, world, port, bounds, results):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from parabiofvm_b200 import slabs

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = RestatedSlab(_line_problem(7), bounds, rank)
        ex = slabs.GroupExchange()
        for i in range(2):
            slabs.step([s], ex, i == 0)
        results[rank] = (s.u.copy(), s.grad.copy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.mark.parametrize("bounds", [[0, 45, 100]])
def test_gloo_two_ranks_step_the_whole_line(bounds):
    import torch.multiprocessing as mp

    world = 2
    with mp.get_context("spawn").Manager() as manager:
        results = manager.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), bounds, results), nprocs=world, join=True,
                           start_method="spawn")
        got = dict(results)
    u = np.concatenate([got[r][0] for r in range(world)])
    g = np.concatenate([got[r][1] for r in range(world)])

    n, h = MESH["n"], float(MESH["h"])
    bp, c = thomas_coefficients(n, MESH["h"], MESH["dims"], MESH["dt"], MESH["D"], MESH["lam"])
    whole = _line_problem(7)
    for _ in range(2):
        whole, _ = slab_solve(whole, bp, c, 0, n)
    grad = np.empty_like(whole)
    grad[0] = (whole[1] - whole[0]) / h
    grad[-1] = (whole[-1] - whole[-2]) / h
    grad[1:-1] = (whole[2:] - whole[:-2]) / (2 * h)
    # the exchanged values are float32
    np.testing.assert_allclose(u, whole, rtol=1e-5, atol=1e-6 * np.abs(whole).max())
    np.testing.assert_allclose(g, grad, rtol=1e-4, atol=1e-6 * np.abs(grad).max())


def test_create_slab_checks_its_arguments_before_the_device():
    import ctypes

    from parabiofvm_b200 import _abi

    lib = _abi.load()
    i3 = lambda v: (ctypes.c_int32 * 3)(*v)  # noqa: E731
    D = (ctypes.c_float * 1)(1000.0)
    lam = (ctypes.c_float * 1)(0.1)

    def create(bounds, slab):
        b = (ctypes.c_int32 * len(bounds))(*bounds)
        h = ctypes.c_void_p()
        rc = lib.bfvm_create_slab(ctypes.byref(h), 0, i3((0, 0, 0)), i3((200, 200, 200)), i3((20, 20, 20)), 1, 0.01,
                                  D, lam, 0, len(bounds) - 1, b, slab)
        return rc, lib.bfvm_last_error().decode()

    assert create([0, 5, 9], 0) == (1, "slab_planes must run from 0 to the mesh's 10 z planes")
    assert create([0, 9, 10], 0)[0] == 1  # a slab of one plane
    assert create([0, 5, 10], 2)[0] == 1  # slab index out of range


def _reduce_weights_f64(bp, c, n, i0, i1):
    """float64 alpha and omega of every plane of the slab [i0, i1) (the linear forms of its zero-carry
    A and B), from the recurrences of the Thomas solve."""
    S = c.size
    e = (c[None, :] * bp).astype(np.float32).astype(np.float64)  # e = c b', the float product
    b = bp.astype(np.float64)
    cc = c.astype(np.float64)
    nl = i1 - i0
    alpha = np.ones((nl, S))
    for i in range(nl - 2, -1, -1):
        alpha[i] = alpha[i + 1] * -e[i0 + i]
    phi = np.empty((nl, S))
    pr = np.ones(S)
    for k in range(nl):
        phi[k] = b[i0 + k] * pr
        pr = pr * -cc * b[i0 + k]
    omega = np.empty((nl, S))
    omega[-1] = phi[-1]
    for i in range(nl - 2, -1, -1):
        omega[i] = phi[i] - e[i0 + i] * omega[i + 1]
    return alpha, omega


@pytest.mark.parametrize("D,bounds", [
    ([1000.0, 20000.0, 50.0], [0, 37, 70, 100]),
    ([1e5, 2e5, 1e3, 10.0], [0, 45, 100]),
    ([1e6, 3e6], [0, 20, 60, 100]),  # slow decay: every plane kept
])
def test_reduce_weights_give_the_zero_carry_values(D, bounds):
    """bfvm_slab_reduce_weights (host code of the reduce pass): the weights match the float64 linear
    forms, the planes left out weigh at most 2^-50 together, and the weighted sums give the slab's
    zero-carry A and B."""
    from parabiofvm_b200.slabs import slab_reduce_weights

    n, h, dt = 100, 20, 0.01
    lam = [0.1] * len(D)
    bp, c = thomas_coefficients(n, h, 3, dt, D, lam)
    d = np.random.default_rng(len(D)).uniform(0, 1, (n, 6 * len(D)))
    for k in range(len(bounds) - 1):
        i0, i1 = bounds[k], bounds[k + 1]
        a_first, wa, wb = slab_reduce_weights(n, h, D, lam, dt, i0, i1)
        alpha, omega = _reduce_weights_f64(bp, c, n, i0, i1)
        if i1 == n:
            assert wa.shape[0] == 0
        else:
            assert a_first + wa.shape[0] == i1
            # float weights: relative rounding, and the smallest ones below float's normal range
            np.testing.assert_allclose(wa, alpha[a_first - i0:], rtol=1e-6, atol=1e-30)
            assert np.abs(alpha[:a_first - i0]).max(axis=1, initial=0).sum() <= 2.0 ** -50
        if i0 == 0:
            assert wb.shape[0] == 0
        else:
            nb = wb.shape[0]
            np.testing.assert_allclose(wb, omega[:nb], rtol=1e-6, atol=1e-30)
            assert np.abs(omega[nb:]).max(axis=1, initial=0).sum() <= 2.0 ** -50
        x, f = slab_solve(d[i0:i1], bp, c, i0, i1)
        L = d.shape[1]
        if i1 < n:
            A = np.einsum("kl,kl->l", expand(wa, L), d[a_first:i1])
            np.testing.assert_allclose(A, f[-1], rtol=1e-6)
        if i0 > 0:
            B = np.einsum("kl,kl->l", expand(wb, L), d[i0:i0 + wb.shape[0]])
            np.testing.assert_allclose(B, x[0], rtol=1e-6)
