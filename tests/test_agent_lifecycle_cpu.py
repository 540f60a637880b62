"""Planning of agent removals on the host (bfvm_plan_agent_removal, no device) against sequential
agent_data::remove calls (src/agent_data.cpp:27-53), restated on agent ids: each removal moves the
then-last agent into the freed slot."""

import numpy as np
import pytest

from parabiofvm_b200 import plan_agent_removal
from parabiofvm_b200._abi import BfvmError


def sequential(agents, indices):
    ids = list(range(agents))
    for i in indices:
        ids[i] = ids[-1]
        ids.pop()
    return ids


def _check(agents, indices):
    remaining, dst, src = plan_agent_removal(agents, indices)
    want = sequential(agents, indices)
    assert remaining == len(want)
    got = np.arange(remaining)
    got[dst] = src
    assert got.tolist() == want
    # moves read rows at or above the final count and write rows below it, each row once
    assert np.all(dst < remaining) and np.all(src >= remaining)
    assert len(set(dst.tolist())) == dst.size and len(set(src.tolist())) == src.size
    return dst.size


@pytest.mark.parametrize("seed", range(25))
def test_moves_reproduce_sequential_removal(seed):
    rng = np.random.default_rng(seed)
    agents = int(rng.integers(1, 300))
    k = int(rng.integers(0, agents + 1))
    idx, c = [], agents
    for _ in range(k):
        # often near the tail, where a removal takes an agent that an earlier removal moved
        i = int(rng.integers(0, c)) if rng.random() < 0.6 else c - 1 - int(rng.integers(0, min(c, 3)))
        idx.append(i)
        c -= 1
    _check(agents, idx)


def test_edge_cases():
    assert _check(10, []) == 0
    assert _check(10, [9, 8, 7]) == 0             # the last agent each time: nothing moves
    assert _check(10, list(range(9, -1, -1))) == 0  # all of them from the back
    assert _check(10, [0] * 10) == 0              # all of them from the front: every row is gone
    assert _check(10, [0]) == 1
    assert _check(6, [1, 1, 1]) == 1              # slot 1 takes 5, then 4, then 3
    assert _check(1, [0]) == 0


def test_an_index_beyond_the_count_at_its_turn_is_refused():
    with pytest.raises(BfvmError) as e:
        plan_agent_removal(5, [4, 4])  # the second removal sees 4 agents
    assert e.value.status == 1
    with pytest.raises(BfvmError):
        plan_agent_removal(5, [-1])
    with pytest.raises(BfvmError):
        plan_agent_removal(0, [0])


def test_any_removal_sequence_matches_sequential_removal():
    from hypothesis import given, settings
    from hypothesis import strategies as st

    @st.composite
    def removals(draw):
        agents = draw(st.integers(min_value=0, max_value=400))
        k = draw(st.integers(min_value=0, max_value=agents))
        idx, c = [], agents
        for _ in range(k):
            idx.append(draw(st.integers(min_value=0, max_value=c - 1)))
            c -= 1
        return agents, idx

    @settings(max_examples=300, deadline=None)
    @given(removals())
    def check(case):
        _check(*case)

    check()


def test_oracle_add_and_remove_follow_agent_data():
    """The oracle's agent_data::add/remove (src/agent_data.cpp:10-53): new rows appended with the given
    values (0 where none is given), and a removal moves the then-last agent into the freed slot."""
    import oracle
    from scenarios import make_oracle, synthetic

    oracle.build()
    w = synthetic(12, 2, 30, seed=5, clustered=True, sigma=40.0)
    o = make_oracle(w, np.float32)
    intern = np.asarray(w.agents.internalized, np.float32).reshape(30, 2).copy()
    new_int = np.arange(8, dtype=np.float32).reshape(4, 2) + 1
    o.add_agents(4, internalized=new_int, volumes=np.full(4, 1000.0), positions=np.full((4, 3), 10.0))
    rows = np.concatenate([intern, new_int])
    np.testing.assert_array_equal(o.internalized().reshape(-1, 2), rows)
    ids = list(range(34))
    for i in (3, 33 - 1, 0):
        o.remove_agent(i)
        ids[i] = ids[-1]
        ids.pop()
    np.testing.assert_array_equal(o.internalized().reshape(-1, 2), rows[ids])
    o.close()
