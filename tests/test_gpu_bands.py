"""The band modes of the LOD step (options xy_band_planes, zg_band_rows): the x and y sweeps run
band by band of z planes, the z sweep and the gradient band by band of y rows, so each band is read
back from L2 by the second kernel.  Every tile is swept by the same code as in whole-field launches,
so fields and gradients must be the same bits; shapes the band modes cannot take run the
whole-field launches."""

import numpy as np
import pytest

from gpu_runner import gpu_runner
from scenarios import synthetic
from test_gpu_parity import _box

pytestmark = pytest.mark.gpu


def _pair(scn, xy, zg):
    banded = gpu_runner(scn)
    plain = gpu_runner(scn)
    banded.s.set_option("xy_band_planes", xy)
    banded.s.set_option("zg_band_rows", zg)
    return banded, plain


def _same(a, b):
    np.testing.assert_array_equal(a.densities(), b.densities())
    np.testing.assert_array_equal(a.gradients(), b.gradients())


@pytest.mark.parametrize("edge,S,xy,zg", [(48, 16, 5, 7), (40, 4, 3, 3), (64, 8, 16, 1), (70, 5, 4, 4),
                                          (36, 16, 35, 35)])
def test_bands_identical_to_whole_field(edge, S, xy, zg):
    """Cubes with Dirichlet faces and interior nodes and clustered agents: bands that do not divide
    the mesh, bands of one row, a shape the band modes cannot take (70 x 5: rows of 6-row x tiles
    and 350-float planes), and bands one short of the mesh."""
    scn = synthetic(edge, S, 1500, seed=7 * edge + S, clustered=True, sigma=60.0, interior_fraction=0.03)
    banded, plain = _pair(scn, xy, zg)
    for first, n in ((0, 2), (2, 9)):
        banded.run_steps(n, first)
        plain.run_steps(n, first)
        _same(banded, plain)
    banded.diffusion()
    plain.diffusion()
    np.testing.assert_array_equal(banded.densities(), plain.densities())
    banded.s.diffusion_gradient()
    plain.s.diffusion_gradient()
    _same(banded, plain)
    banded.close()
    plain.close()


@pytest.mark.parametrize("grid,S,xy,zg", [((96, 40, 72), 16, 8, 6), ((128, 24, 50), 4, 7, 5),
                                          ((40, 64, 33), 8, 1, 9)])
def test_bands_identical_on_boxes(grid, S, xy, zg):
    """Rectangular meshes (lines of different lengths per axis, one of them multi-block) with
    Dirichlet 1.0 on substrate 0 at every face and at 1 % of the interior voxels."""
    w = _box(grid, S, seed=sum(grid) * S)
    banded, plain = _pair(w, xy, zg)
    banded.run_steps(3, 0)
    plain.run_steps(3, 0)
    _same(banded, plain)
    banded.close()
    plain.close()


def test_band_options_are_checked():
    scn = synthetic(24, 4, 0, seed=1)
    g = gpu_runner(scn)
    from parabiofvm_b200 import BfvmError

    for name in ("xy_band_planes", "zg_band_rows"):
        with pytest.raises(BfvmError):
            g.s.set_option(name, -1)
        g.s.set_option(name, 0)
    g.close()
