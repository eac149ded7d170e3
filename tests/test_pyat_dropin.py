"""The engine inside the reference's own pyat, bound as INTEGRATION.md shows.

pyat is the reference's Python package, built from its sources with its C
engine by ``oracle/build_ref.py --full`` into ``oracle/_ref/pyat_full`` (test
infrastructure; these tests skip where it is absent).  The bindings are the two
a pyat maintainer would add to ``pyat/at/tracking/track.py``:

* GPU backend: ``_gpupass`` -> ``at_b200.gpupass`` (with the backend switch
  ``iscuda`` on), reached by ``Lattice.track(..., use_mp=MPMode.GPU)``
  (track.py:49-51, 115-127);
* CPU engine: ``_atpass`` -> ``at_b200.atpass``, reached by every optics
  function built on ``internal_lpass`` (find_orbit6, find_m66,
  get_acceptance; track.py:129).

Lattices are pyat's own ``Lattice`` and ``Element`` objects, built with pyat's
element classes or loaded by pyat from the reference's ``hmba.mat``.  Each call
is compared with the same call on the reference's own C engine.  Tolerances:
one turn 1e-13 of each coordinate's scale (the engine's default arithmetic is
the reference's operation order; sin/tan are CUDA's), tens of turns 1e-9 (the
long-run bound; a bunch of three times the FODO workload's size is in the
chaotic region, where single-ulp differences grow) with the same loss map, closed orbits 1e-14 m, one-turn matrices from the
reference's central differences (step 3e-8) 1e-7.
"""
import importlib
import math
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, scale_rel_diff

PYAT = os.path.join(ROOT, "oracle", "_ref", "pyat_full")


@pytest.fixture(scope="module")
def at():
    if not os.path.isdir(os.path.join(PYAT, "at")):
        pytest.skip("the reference's pyat is not built (oracle/build_ref.py --full)")
    if PYAT not in sys.path:
        sys.path.insert(0, PYAT)
    mod = sys.modules.get("at")
    if mod is not None and not os.path.abspath(mod.__file__).startswith(PYAT):
        pytest.skip("another package named 'at' is already imported")
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return importlib.import_module("at")


def fodo_pyat(at):
    """The 32-cell FODO ring (3 GeV electrons, 3 MV RF at h = 320) written with
    pyat's element classes, as a user of the reference would."""
    cell = []
    for i in range(32):
        cell += [at.Quadrupole("QF", 0.5, 1.0), at.Drift("D1", 0.3),
                 at.Sextupole("SF", 0.2, 15.0), at.Drift("D1", 0.3),
                 at.Dipole("B", 1.0, 2 * math.pi / 64, EntranceAngle=math.pi / 64,
                           ExitAngle=math.pi / 64), at.Drift("D2", 0.7),
                 at.Quadrupole("QD", 0.5, -1.0), at.Drift("D1", 0.3),
                 at.Sextupole("SD", 0.2, -25.0), at.Drift("D1", 0.3),
                 at.Dipole("B", 1.0, 2 * math.pi / 64, EntranceAngle=math.pi / 64,
                           ExitAngle=math.pi / 64), at.Drift("D2", 0.7)]
    frf = 320 * 299792458.0 / 192.0
    ring = at.Lattice(cell + [at.RFCavity("RF", 0.0, 3e6, frf, 320, 3e9)], energy=3e9,
                      particle="electron", periodicity=1)
    return ring


def hmba_pyat(at):
    path = os.path.join(PYAT, "machine_data", "hmba.mat")
    if not os.path.exists(path):
        pytest.skip("hmba.mat not in the reference build")
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return at.load_mat(path, use="RING")


@pytest.fixture
def gpu_backend(at, monkeypatch):
    """Bind the engine as pyat's GPU backend (track.py:49-51)."""
    import at_b200
    T = importlib.import_module("at.tracking.track")
    monkeypatch.setattr(T, "iscuda", lambda: True)
    monkeypatch.setattr(T, "_gpupass", at_b200.gpupass, raising=False)
    return T


@pytest.fixture
def gpu_engine(at, monkeypatch):
    """Bind the engine in place of pyat's CPU engine (track.py:22, 129)."""
    import at_b200
    T = importlib.import_module("at.tracking.track")
    monkeypatch.setattr(T, "_atpass", at_b200.atpass)
    return T


def test_pyat_elements_compile_to_the_stand_in_table(at):
    """CPU: the lattice compiler reads pyat's own Element objects into the
    same table as the package's stand-in elements of the same ring."""
    from at_b200 import rings
    from at_b200.lattice import compile_lattice
    mine = rings.fodo_ring()
    theirs = fodo_pyat(at)
    a = compile_lattice(list(theirs), 3e9, theirs.particle.rest_energy)
    b = compile_lattice(list(mine), 3e9, mine.particle.rest_energy)
    np.testing.assert_array_equal(a.offsets, b.offsets)
    np.testing.assert_array_equal(a.words.view(np.uint64), b.words.view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["fodo", "hmba"])
def test_lattice_track_on_the_gpu_backend(at, gpu_backend, name):
    """Lattice.track(use_mp=MPMode.GPU) through the binding against the same
    call on the reference's C engine: final coordinates and loss map."""
    from at_b200 import rings
    ring = fodo_pyat(at) if name == "fodo" else hmba_pyat(at)
    n, nt = (2000, 50) if name == "fodo" else (500, 10)
    r0 = rings.gaussian(n, seed=4) * (3.0 if name == "fodo" else 1.0)
    for turns, tol in ((1, 1e-13), (nt, 1e-9)):
        rc, rg = r0.copy(order="F"), r0.copy(order="F")
        _, _, dc = ring.track(rc, turns, losses=True, in_place=True)
        _, _, dg = ring.track(rg, turns, losses=True, in_place=True, use_mp=at.MPMode.GPU)
        lc, lg = dc["loss_map"], dg["loss_map"]
        np.testing.assert_array_equal(lg.islost, lc.islost)
        np.testing.assert_array_equal(lg.turn, lc.turn)
        np.testing.assert_array_equal(lg.elem, lc.elem)
        ok = ~lc.islost
        assert scale_rel_diff(rg[:, ok], rc[:, ok]) <= tol, (name, turns)
    if name == "fodo":
        assert lc.islost.any()


@pytest.mark.gpu
def test_refpts_through_the_gpu_backend(at, gpu_backend):
    from at_b200 import rings
    ring = fodo_pyat(at)
    r0 = rings.gaussian(256, seed=9)
    refs = [0, 10, 100, len(ring)]
    rc, rg = r0.copy(order="F"), r0.copy(order="F")
    oc, *_ = ring.track(rc, 3, refpts=refs, in_place=True)
    og, *_ = ring.track(rg, 3, refpts=refs, in_place=True, use_mp=at.MPMode.GPU)
    assert og.shape == oc.shape == (6, 256, 4, 3)
    assert scale_rel_diff(og.reshape(6, -1), oc.reshape(6, -1)) <= 1e-12


@pytest.mark.gpu
def test_optics_through_the_engine(at, gpu_engine):
    """pyat's find_orbit6 and find_m66 (central differences on internal_lpass)
    with every tracking call on the engine, against the same functions on the
    reference's C engine."""
    ring = hmba_pyat(at).enable_6d(copy=True)
    T = gpu_engine
    orbit_g, _ = at.find_orbit6(ring)
    m_g, _ = at.find_m66(ring, orbit=orbit_g)
    with pytest.MonkeyPatch.context() as mp:
        from at.tracking.atpass import atpass as ref_atpass
        mp.setattr(T, "_atpass", ref_atpass)
        orbit_c, _ = at.find_orbit6(ring)
        m_c, _ = at.find_m66(ring, orbit=orbit_c)
    np.testing.assert_allclose(orbit_g, orbit_c, rtol=0, atol=1e-14)
    np.testing.assert_allclose(m_g, m_c, rtol=0, atol=1e-7 * np.abs(m_c).max())


@pytest.mark.gpu
def test_get_acceptance_through_the_engine(at, gpu_engine):
    """pyat's own get_acceptance (radial grid and its recursive search) with
    every tracking call on the engine, against the reference's C engine."""
    ring = hmba_pyat(at).disable_6d(copy=True)
    kw = dict(planes=["x", "y"], npoints=[9, 5], amplitudes=[10e-3, 4e-3], nturns=16,
              use_mp=False, verbose=False)
    T = gpu_engine
    out = {}
    for mode in (at.GridMode.RADIAL, at.GridMode.RECURSIVE):
        out[mode, "gpu"] = at.get_acceptance(ring, grid_mode=mode, **kw)
        with pytest.MonkeyPatch.context() as mp:
            from at.tracking.atpass import atpass as ref_atpass
            mp.setattr(T, "_atpass", ref_atpass)
            out[mode, "cpu"] = at.get_acceptance(ring, grid_mode=mode, **kw)
        for a, b in zip(out[mode, "gpu"], out[mode, "cpu"]):
            np.testing.assert_array_equal(a, b)
