"""bfvm_store_agent_positions_async / bfvm_load_internalized_async: the per-step agent copies on the
solver's copy stream give the same results as the synchronous calls, bit for bit, with positions
that change every step and recompute steps that read them."""

import numpy as np
import pytest
import torch

from parabiofvm_b200.workloads import make_solver, synthetic

pytestmark = pytest.mark.gpu


def _pinned(shape):
    return torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()


def test_async_agent_copies_match_synchronous_calls():
    w = synthetic(30, 4, 3000, seed=21, clustered=True, sigma=80.0)
    a = w.agents
    steps = 7
    rng = np.random.default_rng(3)
    L = np.float32(30 * 20)
    moves = [np.clip(a.positions + rng.normal(0, 10.0, a.positions.shape), 0, np.nextafter(L, np.float32(0)))
             .astype(np.float32) for _ in range(steps)]

    sync = make_solver(w)
    want = []
    for k in range(steps):
        sync.store_agent_positions(moves[k])
        sync.diffusion()
        sync.gradient()
        sync.secretion(k % 3 == 0)
        want.append(sync.load_internalized().copy())
    want_field = sync.load_densities()
    sync.close()

    asy = make_solver(w)
    pos = [_pinned(m.shape) for m in moves]
    for p, m in zip(pos, moves):
        p[:] = m
    got = [_pinned((a.count * w.S,)) for _ in range(steps)]
    for k in range(steps):
        asy.store_agent_positions_async(pos[k])
        asy.diffusion()
        asy.gradient()
        asy.secretion(k % 3 == 0)
        asy.load_internalized_async(got[k])
    asy.synchronize()
    got_field = asy.load_densities()
    for k in range(steps):
        np.testing.assert_array_equal(got[k], want[k], err_msg=f"internalized after step {k}")
    np.testing.assert_array_equal(got_field, want_field)
    asy.close()


def test_run_steps_orders_after_pending_copies():
    w = synthetic(24, 2, 800, seed=5)
    a = w.agents
    ref = make_solver(w)
    ref.run_steps(3)
    want = ref.load_internalized().copy()
    ref.close()
    s = make_solver(w)
    out = _pinned((a.count * w.S,))
    s.load_internalized_async(out)  # pending while run_steps queues its graphs
    s.run_steps(3)
    np.testing.assert_array_equal(s.load_internalized(), want)
    s.close()
