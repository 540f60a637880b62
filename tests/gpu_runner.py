"""Adapter that drives the CUDA library through the same interface as the oracle in the tests."""

from __future__ import annotations

import numpy as np

from scenarios import make_gpu


class GpuRunner:
    """Runs a Scenario on the GPU; every accessor copies back through the C ABI."""

    def __init__(self, scn):
        self.scn = scn
        self.s = make_gpu(scn)

    def diffusion(self):
        self.s.diffusion()

    def dirichlet(self):
        self.s.dirichlet()

    def gradient(self):
        self.s.gradient()

    def secretion(self, recompute):
        self.s.secretion(recompute)

    def release(self, index):
        self.s.release(index)

    def run_steps(self, steps, first_step=0):
        self.s.run_steps(steps, first_step)

    def densities(self):
        return self.s.load_densities()

    def gradients(self):
        return self.s.load_gradients()

    def internalized(self):
        return self.s.load_internalized()

    def close(self):
        self.s.close()


def gpu_runner(scn):
    return GpuRunner(scn)


def step_oracle_style(runner, steps, first_step=0):
    """The reference driver's step sequence through the individual solver calls."""
    for i in range(steps):
        runner.diffusion()
        runner.gradient()
        runner.secretion((first_step + i) % 10 == 0)


def as_f32(a):
    return np.asarray(a, np.float32)
