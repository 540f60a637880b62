"""100 steps of the headline configuration, the GPU and the CPU oracles stepping in lockstep.

320^3 voxels x 16 substrates, 1,000,000 agents in 32 Gaussian clusters, 1 % of the interior voxels
pinned, Dirichlet 1.0 on substrate 0 at every face, recompute every 10th step -- the step of the
reference driver (src/main.cpp:64-107).  The GPU solver (graph-replayed steps through the C ABI), the
FP32 oracle and the FP64 oracle start from the same state and advance one step at a time.  After
every one of the first 10 steps and then every 10th:

* the GPU field's maximum relative error against the FP32 oracle (floor 1e-6 of max|ref|) stays
  below the per-step bar, 1e-5; after step 100 it is below the 100-step bar, 1e-4;
* the GPU field's relative L2 distance to the FP64 oracle is at most 1.5x the FP32 oracle's own
  (the GPU is as close to the double-precision result as the reference's FP32 algorithm is).

The comparisons run on the GPU in float64 (torch), so each check takes well under a second; the
oracles' steps take most of the test's few minutes.
"""

import os

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

EDGE, S, AGENTS = 320, 16, 1_000_000
PER_STEP_BAR = 1e-5
FINAL_BAR = 1e-4


def _stats(got, ref):
    """(max relative error with floor 1e-6 of max|ref|, relative L2) of two device tensors, in
    float64."""
    import torch

    g = got.double()
    r = ref.double()
    floor = max(float(r.abs().max()) * 1e-6, 1e-30)
    max_rel = float(((g - r).abs() / r.abs().clamp(min=floor)).max())
    l2 = float(torch.linalg.vector_norm(g - r) / torch.linalg.vector_norm(r).clamp(min=1e-300))
    return max_rel, l2


def test_plain_320_lockstep_100_steps():
    import torch

    import oracle
    from parabiofvm_b200.workloads import make_solver, synthetic
    from scenarios import make_oracle

    oracle.build()
    oracle.set_threads(os.cpu_count() or 1)
    w = synthetic(EDGE, S, AGENTS, seed=20261203, clustered=True, sigma=200.0, interior_fraction=0.01)
    g = make_solver(w)
    o32 = make_oracle(w, np.float32)
    o64 = make_oracle(w, np.float64)
    dev = torch.device("cuda", 0)
    got = torch.empty(w.voxel_count * S, dtype=torch.float32, device=dev)
    checks = [k for k in range(1, 101) if k <= 10 or k % 10 == 0]
    rows = []
    for k in range(100):
        g.run_steps(1, k)
        o32.run_steps(1, k)
        o64.run_steps(1, k)
        if k + 1 not in checks:
            continue
        g.load_densities_device(got)
        g.synchronize()
        r32 = torch.from_numpy(o32.densities()).to(dev)
        r64 = torch.from_numpy(o64.densities()).to(dev)
        e32, l2_32 = _stats(got, r32)
        e64, l2_64 = _stats(got, r64)
        _, own = _stats(r32, r64)
        del r32, r64
        rows.append((k + 1, e32, l2_32, e64, l2_64, own))
        print(f"step {k + 1:3d}: max rel vs FP32 {e32:.2e} (rel-L2 {l2_32:.2e}); vs FP64 max rel {e64:.2e}, "
              f"rel-L2 {l2_64:.3e} (FP32 oracle {own:.3e})", flush=True)
        assert e32 < PER_STEP_BAR, f"step {k + 1}: max rel err {e32:.3e} against the FP32 oracle"
        assert l2_64 <= 1.5 * own + 1e-7, f"step {k + 1}: rel-L2 vs FP64 {l2_64:.3e}, FP32 oracle's {own:.3e}"
    g.close()
    o32.close()
    o64.close()
    assert rows[-1][0] == 100 and rows[-1][1] < FINAL_BAR
