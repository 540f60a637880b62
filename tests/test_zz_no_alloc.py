"""bfvm_secretion_solve_noalloc: secretion and uptake for callers that cannot allocate GPU memory.

Such callers (a host framework that owns every device allocation, a memory budget planned ahead
of time, code running while another library captures a stream) hand over their own device buffers;
the entry point keeps its binning scratch in a static device array instead of allocating.  It runs
the same kernels in the same order as bfvm_secretion_solve with recompute, so the checks below ask
for the same bits as that entry point and as the FP32 oracle, on calls in a row (each call finds
the previous call's leftovers in the shared scratch array); they also check that a call changes
the device's free memory by nothing and that a call can be captured in a CUDA graph in global
capture mode, where an allocation would fail the capture.

This file is named to be collected last: a failure here comes after every other test has run.
"""

import ctypes

import numpy as np
import pytest

from parabiofvm_b200 import _abi
from parabiofvm_b200.workloads import make_solver, synthetic


def _i3(v):
    return (ctypes.c_int32 * 3)(*[int(t) for t in list(v) + [1] * (3 - len(v))])


def _call(lib, dens_ptr, w, grid, agents, dev, err_ptr, stream_ptr):
    a = agents
    S = len(w.diffusion_coefficients)
    return lib.bfvm_secretion_solve_noalloc(
        ctypes.c_void_p(dens_ptr), w.dims, _i3(w.bbox_min), _i3(w.voxel_shape), _i3(grid), S, float(w.time_step),
        a.count, *[ctypes.c_void_p(dev[k].data_ptr()) for k in ("sec", "sat", "upt", "nex")],
        ctypes.c_void_p(dev["intern"].data_ptr()) if w.compute_internalized else None,
        ctypes.c_void_p(dev["vol"].data_ptr()), ctypes.c_void_p(dev["pos"].data_ptr()),
        ctypes.c_void_p(err_ptr), ctypes.c_void_p(stream_ptr))


@pytest.mark.gpu
@pytest.mark.parametrize("edge,S,agents,internalized", [(40, 4, 6000, True), (24, 3, 2000, False)])
def test_noalloc_matches_secretion_solve(edge, S, agents, internalized):
    """Three recompute calls in a row on the caller's buffers, each checked bit for bit against
    bfvm_secretion_solve and the first two against the FP32 oracle too.  The second call must leave
    the device's free memory unchanged, and the third is captured in a CUDA graph in global capture
    mode, where any allocation would end the capture with an error, then replayed."""
    import torch

    from scenarios import make_oracle

    w = synthetic(edge, S, agents, seed=77 + edge, clustered=True, sigma=60.0, internalized=internalized)
    a = w.agents

    # the existing entry point, three recompute calls in a row
    ref = make_solver(w)
    expect = []
    for _ in range(3):
        ref.secretion(True)
        expect.append((ref.load_densities().copy(), ref.load_internalized().copy() if internalized else None))
    ref.close()
    # the oracle, two calls
    o = make_oracle(w, np.float32)
    oracle_expect = []
    for _ in range(2):
        o.secretion(True)
        oracle_expect.append((o.densities().copy(), o.internalized().copy() if internalized else None))
    o.close()

    # the no-alloc entry point on caller-owned buffers: the field of a second solver (no agents
    # stored there) and agent arrays the test allocates
    w_field = synthetic(edge, S, 0, seed=77 + edge, clustered=True, sigma=60.0, internalized=internalized)
    w_field.densities = w.densities
    own = make_solver(w_field)
    stream = torch.cuda.Stream()
    own.set_stream(stream.cuda_stream)
    dens_ptr, n = own.device_densities()
    assert n == w.densities.size
    dev = {
        "sec": torch.from_numpy(np.ascontiguousarray(a.secretion_rates, np.float32)).cuda(),
        "sat": torch.from_numpy(np.ascontiguousarray(a.saturation_densities, np.float32)).cuda(),
        "upt": torch.from_numpy(np.ascontiguousarray(a.uptake_rates, np.float32)).cuda(),
        "nex": torch.from_numpy(np.ascontiguousarray(a.net_export_rates, np.float32)).cuda(),
        "intern": torch.from_numpy(np.ascontiguousarray(a.internalized, np.float32)).cuda(),
        "vol": torch.from_numpy(np.ascontiguousarray(a.volumes, np.float32)).cuda(),
        "pos": torch.from_numpy(np.ascontiguousarray(a.positions, np.float32)).cuda(),
    }
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    lib = _abi.load()

    def check(call):
        d = own.load_densities()
        np.testing.assert_array_equal(d, expect[call][0], err_msg=f"densities after call {call + 1}")
        if call < 2:
            np.testing.assert_array_equal(d, oracle_expect[call][0], err_msg=f"oracle densities, call {call + 1}")
        if internalized:
            got = dev["intern"].cpu().numpy().reshape(-1)
            np.testing.assert_array_equal(got, expect[call][1].reshape(-1), err_msg=f"internalized, call {call + 1}")
            if call < 2:
                np.testing.assert_array_equal(got, oracle_expect[call][1].reshape(-1),
                                              err_msg=f"oracle internalized, call {call + 1}")

    # call 1: eager
    _abi.check(_call(lib, dens_ptr, w, own.grid, a, dev, err.data_ptr(), stream.cuda_stream))
    stream.synchronize()
    check(0)
    # call 2: eager, with the device's free memory read on both sides
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    _abi.check(_call(lib, dens_ptr, w, own.grid, a, dev, err.data_ptr(), stream.cuda_stream))
    stream.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after == free_before, (free_before, free_after)
    check(1)
    # call 3: captured in global mode, then replayed once
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, capture_error_mode="global"):
        _abi.check(_call(lib, dens_ptr, w, own.grid, a, dev, err.data_ptr(), torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    check(1)  # capturing ran nothing
    graph.replay()
    torch.cuda.synchronize()
    check(2)
    assert int(err.item()) == 0
    del graph
    own.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = _abi.load()
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    args = lambda A, S: (dummy, 3, _i3((0, 0, 0)), _i3((20, 20, 20)), _i3((10, 10, 10)), S, 0.01, A,  # noqa: E731
                         *[dummy] * 4, None, dummy, dummy, None, None)
    assert lib.bfvm_secretion_solve_noalloc(*args(65537, 1)) == 1
    assert b"65536" in lib.bfvm_last_error()
    assert lib.bfvm_secretion_solve_noalloc(*args(65536, 5)) == 1
    assert b"262144" in lib.bfvm_last_error()
