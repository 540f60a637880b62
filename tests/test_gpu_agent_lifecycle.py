"""Agents added and removed on the GPU (bfvm_add_agents, bfvm_remove_agents) against the same
changes made to host copies of the agent arrays and stored whole with bfvm_store_agents (the
reference's way: src/solver/device/CUDA/cell_solver.cpp:172-178).  Both solvers then take the same
steps, and everything they hold must agree bit for bit.

add is agent_data::add (src/agent_data.cpp:10-25): new rows appended, zero where no value is given.
remove is agent_data::remove (src/agent_data.cpp:27-53): the then-last agent fills the freed slot.
"""

import numpy as np
import pytest

from parabiofvm_b200.workloads import make_solver, synthetic

KEYS = ("sec", "sat", "upt", "nex", "intern", "frac", "vol", "pos")


def _host(w):
    a = w.agents
    n, S = a.count, w.S
    vals = (a.secretion_rates, a.saturation_densities, a.uptake_rates, a.net_export_rates, a.internalized,
            a.fraction_released, a.volumes, a.positions)
    shapes = [(n, S)] * 6 + [(n,), (n, 3)]
    return {k: np.array(v, np.float32).reshape(s) for k, v, s in zip(KEYS, vals, shapes)}


def _store(s, H):
    s.store_agents(*[H[k] for k in KEYS])


def _host_remove(H, indices):
    n = H["vol"].shape[0]
    for i in indices:
        n -= 1
        for k in KEYS:
            H[k][i] = H[k][n]
    for k in KEYS:
        H[k] = H[k][:n].copy()


def _new_rows(rng, n, S, L):
    return {"sec": rng.uniform(0, 10, (n, S)), "sat": rng.uniform(0, 1, (n, S)), "upt": rng.uniform(0, 1, (n, S)),
            "nex": None, "intern": rng.uniform(0, 5, (n, S)), "frac": None,
            "vol": rng.uniform(500, 1500, n),
            "pos": np.minimum(rng.uniform(0, L, (n, 3)).astype(np.float32), np.nextafter(np.float32(L), 0))}


def _removals(rng, count, k):
    out = []
    for _ in range(k):
        out.append(int(rng.integers(0, count)) if rng.random() < 0.7 else count - 1 - int(rng.integers(0, min(count, 4))))
        count -= 1
    return out


def _same(a, b):
    np.testing.assert_array_equal(a.load_densities(), b.load_densities())
    np.testing.assert_array_equal(a.load_gradients(), b.load_gradients())
    np.testing.assert_array_equal(a.load_internalized(), b.load_internalized())
    assert a.agents_count == b.agents_count


def _pair(seed, agents):
    w = synthetic(24, 4, agents, seed=seed, clustered=True, sigma=60.0, interior_fraction=0.01)
    return w, make_solver(w), make_solver(w), _host(w)


@pytest.mark.gpu
def test_added_and_removed_agents_step_like_stored_ones():
    w, a, b, H = _pair(11, 3000)
    rng = np.random.default_rng(12)
    L = w.bbox_max[0]
    for s in (a, b):
        s.run_steps(3, 0)
    # more agents than the storage holds: it grows on the device, keeping the stored rows
    new = _new_rows(rng, 5000, w.S, L)
    a.add_agents(5000, new["sec"], new["sat"], new["upt"], None, new["intern"], None, new["vol"], new["pos"])
    H["intern"] = b.load_internalized().reshape(-1, w.S)
    for k in KEYS:
        rows = new[k] if new[k] is not None else np.zeros((5000,) + H[k].shape[1:])
        H[k] = np.concatenate([H[k], np.asarray(rows, np.float32).reshape((5000,) + H[k].shape[1:])])
    _store(b, H)
    for s in (a, b):
        s.run_steps(4, 3)
    _same(a, b)
    idx = _removals(rng, a.agents_count, 1200)
    a.remove_agents(idx)
    H["intern"] = b.load_internalized().reshape(-1, w.S)
    _host_remove(H, idx)
    _store(b, H)
    for s in (a, b):
        s.run_steps(5, 7)  # through a recompute step (10)
    _same(a, b)
    a.close()
    b.close()


@pytest.mark.gpu
def test_an_agent_dies_releasing_its_substrates():
    w, a, b, H = _pair(21, 800)
    for s in (a, b):
        s.run_steps(2, 0)
    for i in (17, 798, 0):  # 798: the last agent after the first removal
        for s in (a, b):
            s.release(i)
        a.remove_agents([i])
        H["intern"] = b.load_internalized().reshape(-1, w.S)
        _host_remove(H, [i])
        _store(b, H)
        for s in (a, b):
            s.run_steps(1, 2)
    _same(a, b)
    a.close()
    b.close()


@pytest.mark.gpu
def test_a_refused_removal_changes_nothing():
    from parabiofvm_b200._abi import BfvmError

    w, a, b, H = _pair(31, 500)
    for s in (a, b):
        s.run_steps(2, 0)
    with pytest.raises(BfvmError) as e:
        a.remove_agents([3, 498, 498])  # the third sees 498 agents
    assert e.value.status == 1
    assert a.agents_count == 500
    for s in (a, b):
        s.run_steps(3, 2)
    _same(a, b)
    a.close()
    b.close()


@pytest.mark.gpu
def test_all_agents_leave_then_new_ones_arrive():
    w, a, b, H = _pair(41, 300)
    rng = np.random.default_rng(42)
    for s in (a, b):
        s.run_steps(2, 0)
    a.remove_agents(list(range(299, -1, -2)) + [0] * 150)
    _host_remove(H, list(range(299, -1, -2)) + [0] * 150)
    assert H["vol"].shape[0] == 0 and a.agents_count == 0
    b.store_agents(*[H[k] for k in KEYS])
    for s in (a, b):
        s.run_steps(2, 2)
    new = _new_rows(rng, 40, w.S, w.bbox_max[0])
    a.add_agents(40, new["sec"], new["sat"], new["upt"], None, new["intern"], None, new["vol"], new["pos"])
    for k in KEYS:
        rows = new[k] if new[k] is not None else np.zeros((40,) + H[k].shape[1:])
        H[k] = np.asarray(rows, np.float32).reshape((40,) + H[k].shape[1:])
    _store(b, H)
    for s in (a, b):
        s.run_steps(3, 4)
    _same(a, b)
    a.close()
    b.close()


@pytest.mark.gpu
def test_store_with_same_count_keeps_binning_and_takes_new_amounts():
    """Storing agents with an unchanged count keeps the binning until the next recompute step (as
    the reference's store does) and takes the stored internalized amounts, also while the solver
    holds them in the binning's sorted order: the same as a fresh solver given that state."""
    w = synthetic(30, 4, 2500, seed=17, clustered=True, sigma=80.0)
    a = w.agents
    s = make_solver(w)
    s.run_steps(5, 0)
    field = s.load_densities().copy()
    intern = (s.load_internalized().reshape(a.count, w.S) * 0.5).astype(np.float32)
    s.store_agents(a.secretion_rates, a.saturation_densities, a.uptake_rates, a.net_export_rates, intern,
                   a.fraction_released, a.volumes, a.positions)
    s.run_steps(4, 5)
    w2 = synthetic(30, 4, 2500, seed=17, clustered=True, sigma=80.0)
    w2.densities = field
    w2.agents.internalized = intern
    fresh = make_solver(w2)
    fresh.run_steps(4, 5)
    np.testing.assert_array_equal(s.load_densities(), fresh.load_densities())
    np.testing.assert_array_equal(s.load_gradients(), fresh.load_gradients())
    np.testing.assert_array_equal(s.load_internalized(), fresh.load_internalized())
    s.close()
    fresh.close()


@pytest.mark.gpu
def test_population_that_gains_and_loses_agents_against_the_oracle():
    """A stepped population that gains and loses agents, on the GPU (bfvm_add_agents,
    bfvm_remove_agents) and in the FP32 oracle (agent_data::add/remove restated,
    src/agent_data.cpp:10-53), between recompute steps.  Lines of one register block keep the GPU
    bit-identical to the oracle."""
    from scenarios import make_oracle

    w = synthetic(32, 3, 1500, seed=41, clustered=True, sigma=60.0, interior_fraction=0.02)
    g = make_solver(w)
    o = make_oracle(w, np.float32)
    rng = np.random.default_rng(42)
    first = 0
    for change in range(3):
        g.run_steps(10, first)
        o.run_steps(10, first)
        first += 10
        new = _new_rows(rng, 200 + 50 * change, w.S, 32 * 20)
        args = [new[k] for k in KEYS]
        g.add_agents(len(new["vol"]), *args)
        o.add_agents(len(new["vol"]), *args)
        idx = _removals(rng, g.agents_count, 150)
        g.remove_agents(idx)
        for i in idx:
            o.remove_agent(i)
    g.run_steps(10, first)
    o.run_steps(10, first)
    np.testing.assert_array_equal(g.load_densities(), o.densities())
    np.testing.assert_array_equal(g.load_gradients(), o.gradients())
    np.testing.assert_array_equal(g.load_internalized(), o.internalized())
    g.close()
    o.close()
