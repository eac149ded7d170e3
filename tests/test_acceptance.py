"""Acceptance scans against the reference's own (``golden/acceptance_large.npz``,
pyat/at/acceptance on the radiating large ring, made by
``golden/make_golden.py``): the grid and the boundary extraction on the CPU
from the reference's survivor sets, the whole scan on the GPU."""
import os

import numpy as np
import pytest

from at_b200 import acceptance as A
from at_b200 import rings
from conftest import GOLDEN

CASES = {
    "radial": dict(planes=["x", "y"], npoints=[9, 7], amplitudes=[6e-3, 3e-3],
                   grid_mode=A.GridMode.RADIAL),
    "cartesian": dict(planes=["x", "y"], npoints=[11, 6], amplitudes=[6e-3, 3e-3],
                      grid_mode=A.GridMode.CARTESIAN),
    "momentum": dict(planes=["dp"], npoints=[21], amplitudes=[0.04],
                     grid_mode=A.GridMode.CARTESIAN),
}


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(os.path.join(GOLDEN, "acceptance_large.npz")))


def _mask(g, s):
    """Which grid points the reference kept (its survivors are grid columns)."""
    return np.array([any(np.array_equal(g[:, i], s[:, j]) for j in range(s.shape[1]))
                     for i in range(g.shape[1])])


@pytest.mark.parametrize("name", list(CASES))
def test_grid_and_boundary_match_reference(gold, name):
    kw = CASES[name]
    cfg = A.grid_configuration(kw["planes"], kw["npoints"], kw["amplitudes"], kw["grid_mode"],
                               shift_zero=1.0e-6)
    orbit = np.array(rings.LARGE_ORBIT)
    parts, grid = A.get_parts(cfg, orbit)
    np.testing.assert_array_equal(grid.grid, gold[name + "_g"])
    assert parts.shape == (6, gold[name + "_g"].shape[1])
    mask = _mask(gold[name + "_g"], gold[name + "_s"])
    assert mask.sum() == gold[name + "_s"].shape[1]
    b = A.get_grid_boundary(mask, grid, cfg)
    np.testing.assert_array_equal(b, gold[name + "_b"])


def test_unsupported_modes_say_so():
    with pytest.raises(NotImplementedError):
        A.grid_configuration(["x", "y"], [3, 3], [1e-3, 1e-3], A.GridMode.RECURSIVE)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_acceptance_matches_reference(gold, name):
    ring = rings.large_ring(seed=1)
    b, s, g = A.get_acceptance(ring, nturns=32, mode="exact", **CASES[name])
    np.testing.assert_array_equal(g, gold[name + "_g"])
    np.testing.assert_array_equal(s, gold[name + "_s"])
    np.testing.assert_array_equal(b, gold[name + "_b"])


@pytest.mark.gpu
def test_acceptance_at_two_points_matches_reference(gold):
    ring = rings.large_ring(seed=1)
    b, s, g = A.get_acceptance(ring, ["x", "y"], [7, 5], [6e-3, 3e-3], nturns=16,
                               refpts=[0, 61], grid_mode=A.GridMode.RADIAL, mode="exact")
    for k in range(2):
        np.testing.assert_allclose(g[k], gold["multi%d_g" % k], rtol=0, atol=1e-15)
        np.testing.assert_allclose(s[k], gold["multi%d_s" % k], rtol=0, atol=1e-15)
        np.testing.assert_allclose(b[k], gold["multi%d_b" % k], rtol=0, atol=1e-15)


@pytest.mark.gpu
def test_momentum_acceptance_wrapper(gold):
    ring = rings.large_ring(seed=1)
    b, s, g = A.get_momentum_acceptance(ring, 0.04 / 21, 0.04, nturns=32, mode="exact")
    assert b.shape == (2,) and b[0] < 0 < b[1]
