"""Acceptance scans against the reference's own results (golden
``acceptance_large.npz`` and ``acceptance_modes.npz``: pyat/at/acceptance run
on the radiating large ring by ``golden/make_golden.py``).

CPU tests run every search mode with the oracle standing in for the engine's
tracking calls (the oracle is pinned bit for bit to the reference's engine), so
the host logic -- grids, boundaries, the flood-fill walk and the recursive
search with its speculative launches -- is checked against the reference's
outputs exactly.  GPU tests run the same scans on the engine."""
import os

import numpy as np
import pytest

from at_b200 import acceptance as A
from at_b200 import rings
from conftest import GOLDEN
from oracle import oracle

CASES = {
    "radial": dict(planes=["x", "y"], npoints=[9, 7], amplitudes=[6e-3, 3e-3],
                   grid_mode=A.GridMode.RADIAL, nturns=32),
    "cartesian": dict(planes=["x", "y"], npoints=[11, 6], amplitudes=[6e-3, 3e-3],
                      grid_mode=A.GridMode.CARTESIAN, nturns=32),
    "momentum": dict(planes=["dp"], npoints=[21], amplitudes=[0.04],
                     grid_mode=A.GridMode.CARTESIAN, nturns=32),
}
MODES = {
    "cart21": dict(planes=["x", "y"], npoints=[21, 11], amplitudes=[8e-3, 4e-3],
                   grid_mode=A.GridMode.CARTESIAN, nturns=24),
    "rec2d": dict(planes=["x", "y"], npoints=[12, 7], amplitudes=[8e-3, 4e-3],
                  grid_mode=A.GridMode.RECURSIVE, nturns=16),
    "rec1d": dict(planes=["dp"], npoints=[16], amplitudes=[0.04],
                  grid_mode=A.GridMode.RECURSIVE, nturns=16),
    "flood": dict(planes=["x", "y"], npoints=[15, 9], amplitudes=[8e-3, 4e-3],
                  grid_mode=A.GridMode.FLOODFILL, nturns=16),
    "flood_obs": dict(planes=["x", "y"], npoints=[11, 7], amplitudes=[8e-3, 4e-3],
                      grid_mode=A.GridMode.FLOODFILL, nturns=12, refpts=61),
    "rec_obs": dict(planes=["x", "y"], npoints=[8, 5], amplitudes=[8e-3, 4e-3],
                    grid_mode=A.GridMode.RECURSIVE, nturns=12, refpts=61),
}


@pytest.fixture(scope="module")
def gold():
    g = dict(np.load(os.path.join(GOLDEN, "acceptance_large.npz")))
    g.update(np.load(os.path.join(GOLDEN, "acceptance_modes.npz")))
    return g


def _mask(g, s):
    """Which grid points the reference kept (its survivors are grid columns)."""
    return np.array([any(np.array_equal(g[:, i], s[:, j]) for j in range(s.shape[1]))
                     for i in range(g.shape[1])])


def _check(res, gold, name):
    b, s, g = res
    if name.startswith("flood"):
        b, s, g = _drop_unflushed(b, s, g, gold, name)
    np.testing.assert_array_equal(g, gold[name + "_g"], err_msg=name + " tracked")
    np.testing.assert_array_equal(s, gold[name + "_s"], err_msg=name + " survived")
    np.testing.assert_array_equal(b, gold[name + "_b"], err_msg=name + " boundary")


def _drop_unflushed(b, s, g, gold, name):
    """The reference's flood fill runs a queue loop that ends when
    ``multiprocessing.Queue.empty()`` is true, which it can be right after
    the last lost point has queued its neighbours and before they are
    flushed (floodfill_acceptance.py:106-134), so it may leave a few
    registered points untracked.  Here every registered point is tracked.
    Each point the reference lacks must be such a dropped point: a
    4-neighbour of a point it tracked and lost.  Those are removed from this
    result before the exact comparison."""
    ref_g = gold[name + "_g"]
    ref_lost = [tuple(p) for p in ref_g.T
                if not any(np.array_equal(p, q) for q in gold[name + "_s"].T)]
    steps = [np.diff(np.unique(ref_g[k])).min() for k in range(2)]
    extra = [i for i, p in enumerate(g.T) if not any(np.array_equal(p, q) for q in ref_g.T)]
    for i in extra:
        near = [q for q in ref_lost
                if np.isclose(abs(q[0] - g[0, i]) / steps[0] + abs(q[1] - g[1, i]) / steps[1],
                              1.0)]
        assert near, "flood fill tracked %s, which the reference never registered" % g[:, i]
    keep = [p for p in range(g.shape[1]) if p not in extra]
    gk = g[:, keep]
    sk = np.array([p for p in s.T if any(np.array_equal(p, q) for q in gk.T)]).T
    sk = sk.reshape(2, -1)
    # the boundary is the survivors in order of angle, as the search gives it
    bk = sk[:, np.argsort(np.arctan2(sk[1, :], sk[0, :]))] if extra else b
    return bk, sk, gk


def _kwargs(gold, name):
    """The case's arguments; flood fills get the centre the fixture used
    (the ring's 6-D closed orbit at the observation point)."""
    kw = dict(CASES.get(name) or MODES[name])
    if kw["grid_mode"] is A.GridMode.FLOODFILL:
        kw["offset"] = gold["orbit61"] if kw.get("refpts") else gold["orbit0"]
    return kw


@pytest.fixture
def oracle_engine(monkeypatch):
    """Route the scans' tracking calls to the oracle (CPU)."""
    ring = rings.large_ring(seed=1)
    en, rest = ring.energy, ring.particle.rest_energy
    calls = []

    def lost(r, parts, nturns, mode):
        p = np.asfortranarray(parts.copy())
        _, ld = oracle.track(list(r), p, int(nturns), energy=en, rest_energy=rest, losses=True)
        calls.append(p.shape[1])
        return ld["islost"].copy(), ld["turn"].copy()

    def to_end(r, parts, start, mode):
        oracle.track(list(r), parts, 1, energy=en, rest_energy=rest, start_elem=int(start))

    def orbit_at(r, obs, orbit, mode):
        if orbit is not None:
            return np.asarray(orbit, dtype=float)
        o = np.asfortranarray(np.array(rings.LARGE_ORBIT, dtype=float).reshape(6, 1))
        if obs:
            oracle.track(list(r), o, 1, energy=en, rest_energy=rest, end_elem=int(obs))
        return o[:, 0].copy()

    monkeypatch.setattr(A, "_lost", lost)
    monkeypatch.setattr(A, "_to_ring_end", to_end)
    monkeypatch.setattr(A, "_orbit_at", orbit_at)
    return ring, calls


@pytest.mark.parametrize("name", list(CASES))
def test_grid_and_boundary_match_reference(gold, name):
    kw = CASES[name]
    scan = A.make_scan(kw["planes"], kw["npoints"], kw["amplitudes"], kw["grid_mode"])
    parts, grid = A.scan_particles(scan, rings.LARGE_ORBIT)
    np.testing.assert_array_equal(grid, gold[name + "_g"])
    assert parts.shape == (6, gold[name + "_g"].shape[1])
    mask = _mask(gold[name + "_g"], gold[name + "_s"])
    assert mask.sum() == gold[name + "_s"].shape[1]
    np.testing.assert_array_equal(A.grid_boundary(mask, grid, scan), gold[name + "_b"])


@pytest.mark.parametrize("name", ["cartesian", "cart21", "rec2d", "rec1d", "flood",
                                  "flood_obs", "rec_obs"])
def test_search_modes_on_oracle_match_reference(gold, oracle_engine, name):
    """Every search mode, tracking by the oracle, against the reference's
    own get_acceptance on the same ring."""
    ring, calls = oracle_engine
    _check(A.get_acceptance(ring, **_kwargs(gold, name)), gold, name)
    if name.startswith("flood"):
        assert len(calls) == 1            # the whole grid in one launch
    if name == "rec2d":
        # the speculative launches: fewer tracking calls than search steps
        steps = gold[name + "_g"].shape[1]
        assert len(calls) < steps / 3, (len(calls), steps)


def test_floodfill_walk_reaches_border_and_lost_region():
    lost = np.zeros((5, 4), dtype=bool)
    lost[0, :] = True            # a lost border column ...
    lost[1, 1] = True            # ... leading into the interior
    reached = A.floodfill_walk(lost.ravel(), 5, 4).reshape(5, 4)
    border = np.zeros((5, 4), dtype=bool)
    border[[0, -1], :] = True
    border[:, [0, -1]] = True
    assert reached[border].all()
    assert reached[1, 1] and reached[2, 1] and reached[1, 2]   # neighbours of a lost point
    assert not reached[2, 2]                                   # behind survivors


def test_cleaning_equals_morphological_opening():
    """The cartesian boundary's cleaning step is a morphological opening by
    two-point segments (scipy's definition)."""
    from scipy.ndimage import binary_opening
    rng = np.random.default_rng(0)
    for _ in range(500):
        m = rng.random((rng.integers(1, 9), rng.integers(1, 9))) < 0.6
        np.testing.assert_array_equal(A._with_partner(m, 0), binary_opening(m, np.ones((2, 1))))
        np.testing.assert_array_equal(A._with_partner(m, 1), binary_opening(m, np.ones((1, 2))))


def test_scan_definition_errors():
    with pytest.raises(ValueError):
        A.make_scan(["x", "y", "dp"], [3, 3, 3], [1e-3] * 3)
    with pytest.raises(ValueError):
        A.make_scan(["x", "y"], [3], [1e-3, 1e-3])
    with pytest.raises(ValueError):
        A.make_scan(["x", "y"], [3, 3], [1e-3, 1e-3], bounds=[[0, 1]])


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES) + list(MODES))
def test_acceptance_matches_reference(gold, name):
    ring = rings.large_ring(seed=1)
    _check(A.get_acceptance(ring, mode="exact", **_kwargs(gold, name)), gold, name)


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
