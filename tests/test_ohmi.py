"""The Ohmi diffusion-matrix path and the equilibrium envelope.

Element diffusion matrices and the reference's ``ohmi_envelope`` on the
radiating large ring come from the reference itself
(``golden/make_golden.py``: pyat/at.c:755-831 ``diffusion_matrix``,
pyat/at/physics/radiation.py:76-276).  The oracle's restatement of the bdiff
branch is pinned to them on the CPU; the GPU element maps (transfer and
diffusion matrices of every element in one launch) are checked against the
oracle and the envelope against the reference.
"""
import json
import os

import numpy as np
import pytest

from at_b200 import elements as E
from at_b200 import radiation, rings
from conftest import ELECTRON_REST, GOLDEN
from oracle import oracle


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(os.path.join(GOLDEN, "ohmi_large.npz")))


@pytest.fixture(scope="module")
def bend_specs():
    with open(os.path.join(GOLDEN, "ohmi_bends.json")) as f:
        return json.load(f)


def _bend(d):
    kw = {k: v for k, v in d.items() if k != "FamName"}
    for k in ("PolynomA", "PolynomB"):
        kw[k] = np.asarray(kw[k], dtype=np.float64)
    return E.Element(d["FamName"], **kw)


def _close(got, want, rel):
    scale = max(np.abs(want).max(), 1e-300)
    np.testing.assert_allclose(got, want, rtol=0, atol=rel * scale)


def test_oracle_diffmatrix_matches_reference(gold, bend_specs):
    """Called like the reference's _dmatr calls it (energy only, no
    particle: gamma = 1e-9 E / E0)."""
    ring = rings.large_ring(seed=1)
    for i, orb, b in zip(gold["idx"], gold["orbits"], gold["belem"]):
        _close(oracle.diffmatrix(ring[int(i)], orb, ring.energy, 0.0), b, 1e-14)
    for d, orb, b in zip(bend_specs, gold["bend_orbits"], gold["bend_b"]):
        _close(oracle.diffmatrix(_bend(d), orb, 3e9, 0.0), b, 1e-14)


def test_non_radiating_elements_have_no_diffusion(gold):
    ring = rings.large_ring(seed=1, radiation=False)
    assert not oracle.diffmatrix(ring[0], gold["orbit"], ring.energy, ELECTRON_REST).any()


def test_envelope_algebra_reproduces_reference(gold):
    """The host part of ohmi_envelope (Sylvester solve, projected
    emittances, normal-mode tunes, damping rates and emittances) on the
    reference's own one-turn and cumulative diffusion matrices."""
    env = radiation.envelope_from_matrices(gold["m66"], gold["bcum"])
    _close(env["r66"], gold["r66"], 1e-10)
    np.testing.assert_allclose(env["emitXYZ"], gold["emitXYZ"], rtol=1e-10)
    np.testing.assert_allclose(env["emitXY"], gold["emitXY"], rtol=1e-10)
    np.testing.assert_allclose(env["tunes"], gold["tunes"], rtol=1e-12)
    np.testing.assert_allclose(env["damping_rates"], gold["damping_rates"], rtol=1e-10)
    np.testing.assert_allclose(env["mode_emittances"], gold["mode_emittances"], rtol=1e-10)


@pytest.mark.gpu
def test_element_maps_match_oracle(gold, bend_specs):
    """One launch computes every element's transfer matrix (exact
    derivatives) and diffusion matrix at the orbit: the diffusion matrices
    equal the oracle's (to the ulp-level difference of gamma and of CUDA's
    tan), the transfer matrices agree with central differences of the
    oracle's element tracking."""
    ring = rings.large_ring(seed=1)
    orbs = gold["orbs_all"][:-1]
    m, b = radiation.element_maps(ring, orbs)
    assert m.shape == (len(ring), 6, 6) and b.shape == (len(ring), 6, 6)
    nrad = 0
    for i in range(len(ring)):
        ob = oracle.diffmatrix(ring[i], orbs[i], ring.energy, 0.0)
        _close(b[i], ob, 1e-12)
        nrad += bool(ob.any())
    assert nrad == 800                     # 32 cells x 25 radiating magnets
    h = 1e-7
    for i in range(0, len(ring), 29):
        x = np.tile(orbs[i][:, None], (1, 12))
        for j in range(6):
            x[j, 2 * j] += h
            x[j, 2 * j + 1] -= h
        x = np.asfortranarray(x)
        oracle.track([ring[i]], x, 1, energy=ring.energy, rest_energy=ELECTRON_REST,
                     element=True, t0=0.0)
        fd = (x[:, 0::2] - x[:, 1::2]) / (2 * h)
        np.testing.assert_allclose(m[i], fd, rtol=0, atol=1e-8 * max(1.0, np.abs(fd).max()))
    # bends with fringe integrals and every edge method, against the reference
    bl = E.Lattice([_bend(d) for d in bend_specs], energy=3e9, particle="electron")
    _, bb = radiation.element_maps(bl, gold["bend_orbits"])
    for k in range(len(bend_specs)):
        _close(bb[k], gold["bend_b"][k], 1e-12)


@pytest.mark.gpu
def test_ohmi_envelope_matches_reference(gold):
    """The cumulative diffusion matrix and the envelope against the
    reference's.  The reference takes its one-turn matrix from central
    differences (find_m66, DPStep 3e-6), whose ~1e-10 error in the damping
    of each plane is relative ~1e-5 of the horizontal damping rate (6.9e-6
    per turn) and moves the emittances by as much; with the reference's own
    one-turn matrix the engine's B_cum gives its emittances to 1e-7."""
    ring = rings.large_ring(seed=1)
    orbs, bcum, mcum = radiation.cumulative_diffusion(ring, gold["orbit"])
    np.testing.assert_allclose(orbs, gold["orbs_all"], rtol=0, atol=1e-12)
    _close(bcum[-1], gold["bcum"], 1e-7)
    env = radiation.envelope_from_matrices(gold["m66"], bcum[-1])
    np.testing.assert_allclose(env["emitXYZ"], gold["emitXYZ"], rtol=1e-7)
    np.testing.assert_allclose(env["mode_emittances"], gold["mode_emittances"], rtol=1e-7)

    emit0, beamdata, emit = radiation.ohmi_envelope(ring, refpts=[0, 100, 1000])
    np.testing.assert_allclose(emit0.orbit6, gold["orbit"], rtol=0, atol=1e-12)
    _close(emit0.m66, gold["m66"], 1e-7)
    np.testing.assert_allclose(emit0.emitXYZ, gold["emitXYZ"], rtol=1e-4)
    np.testing.assert_allclose(emit0.emitXY, gold["emitXY"], rtol=1e-4)
    np.testing.assert_allclose(beamdata.tunes, gold["tunes"], rtol=1e-8)
    np.testing.assert_allclose(beamdata.damping_rates, gold["damping_rates"], rtol=1e-4)
    np.testing.assert_allclose(beamdata.mode_emittances, gold["mode_emittances"], rtol=1e-4)
    # the solution is the fixed point R = M R M^T + B_cum
    rr, mm = emit0.r66, emit0.m66
    _close(mm @ rr @ mm.T + bcum[-1], rr, 1e-10)
    assert emit.r66.shape == (3, 6, 6)
    for k in range(3):
        _close(emit.r66[k], gold["emit_r66"][k], 1e-4)
        np.testing.assert_allclose(emit.emitXYZ[k], gold["emit_emitXYZ"][k], rtol=1e-4)
    print("emittances vs reference:", emit0.emitXYZ / gold["emitXYZ"] - 1)
