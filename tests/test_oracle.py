"""The oracle (oracle/oracle.c) pinned against the reference.

Golden fixtures come from the reference's own C engine and integrators
(tests/golden/make_golden.py); the known-answer values are those of the
reference's test suite (pyat/test/test_basic_elements.py, test_atpass.py).
The oracle is compiled with the same compiler and libm as the reference
build, so agreement is required bit for bit.
"""
import json
import os

import numpy as np
import pytest

import cases
from at_b200 import elements as E
from at_b200 import rings
from oracle import oracle

from conftest import ELECTRON_REST, GOLDEN


def _track_elem(el, r, energy=0.0, rest=0.0):
    oracle.track([el], r, 1, energy=energy, rest_energy=rest, element=True, t0=0.0)
    return r


@pytest.mark.parametrize("name,spec", cases.element_cases(), ids=[c[0] for c in cases.element_cases()])
def test_element_golden(golden, name, spec):
    g = golden("elements.npz")
    el = cases.make_element(spec, E.Element)
    r = g[name + "/in"].copy(order="F")
    rad = "Rad" in spec["PassMethod"] or spec["PassMethod"] == "RFCavityPass"
    _track_elem(el, r, 6e9 if rad else 0.0, ELECTRON_REST if rad else 0.0)
    np.testing.assert_array_equal(r, g[name + "/out"])


def test_fodo_200_turns_losses(golden):
    g = golden("fodo_200turns.npz")
    r = g["rin"].copy(order="F")
    _, ld = oracle.track(rings.fodo_ring(), r, 200, energy=3e9, rest_energy=ELECTRON_REST,
                         losses=True)
    np.testing.assert_array_equal(r, g["rout_final"])
    np.testing.assert_array_equal(ld["islost"], g["islost"])
    np.testing.assert_array_equal(ld["turn"], g["lturn"])
    np.testing.assert_array_equal(ld["elem"], g["lelem"])
    np.testing.assert_array_equal(ld["coord"], g["lcoord"])
    assert 0 < g["islost"].sum() < g["islost"].size


def test_fodo_refpts(golden):
    g = golden("fodo_refpts.npz")
    r = g["rin"].copy(order="F")
    rout, _ = oracle.track(rings.fodo_ring(), r, 30, refpts=g["refpts"], energy=3e9,
                           rest_energy=ELECTRON_REST, losses=True)
    np.testing.assert_array_equal(rout, g["rout"])
    np.testing.assert_array_equal(r, g["rout_final"])


def test_fodo_radiating(golden):
    g = golden("fodo_rad_20turns.npz")
    r = g["rin"].copy(order="F")
    oracle.track(rings.radiating(rings.fodo_ring()), r, 20, energy=3e9, rest_energy=ELECTRON_REST)
    np.testing.assert_array_equal(r, g["rout_final"])


def test_kitchen_sink_turn_counter(golden):
    g = golden("sink_3turns.npz")
    line = [cases.make_element(s, E.Element) for s in cases.kitchen_sink()]
    r = g["rin"].copy(order="F")
    rout, ld = oracle.track(line, r, 3, refpts=g["refpts"], turn=5, energy=6e9,
                            rest_energy=ELECTRON_REST, losses=True)
    np.testing.assert_array_equal(r, g["rout_final"])
    np.testing.assert_array_equal(rout, g["rout"])
    for k, gk in (("islost", "islost"), ("turn", "lturn"), ("elem", "lelem"), ("coord", "lcoord")):
        np.testing.assert_array_equal(ld[k], g[gk])


def test_kitchen_sink_partial_turn(golden):
    g = golden("sink_partial.npz")
    line = [cases.make_element(s, E.Element) for s in cases.kitchen_sink()]
    r = g["rin"].copy(order="F")
    _, ld = oracle.track(line, r, 1, refpts=g["refpts"], start_elem=4, end_elem=15, energy=6e9,
                         rest_energy=ELECTRON_REST, losses=True)
    np.testing.assert_array_equal(r, g["rout_final"])
    np.testing.assert_array_equal(ld["islost"], g["islost"])


def _hmba(tag):
    with open(os.path.join(GOLDEN, "hmba.json")) as f:
        data = json.load(f)[tag]
    return [cases.make_element(d, E.Element) for d in data["specs"]], data


@pytest.mark.parametrize("tag", ["off", "6d"])
def test_hmba_one_turn(golden, tag):
    line, data = _hmba(tag)
    g = golden("hmba_%s.npz" % tag)
    r = g["rin"].copy(order="F")
    oracle.track(line, r, 1, energy=data["energy"], rest_energy=0.0)
    np.testing.assert_array_equal(r, g["rout_final"])


def test_hmba_partial_turns_reference_values():
    """pyat/test/test_atpass.py:157-171 (atol 1e-7) and the fixture (exact)."""
    line, data = _hmba("off")
    for (s, e, expected) in ((100, 0, [3.2e-6, -1.1e-6, 0, 0, 0, 8.4e-8]),
                             (100, 110, [2.6e-6, 1.34e-6, 0, 0, 0, 2.4e-8])):
        r = np.array([0, 1e-6, 0, 0, 0, 0], dtype=np.float64)
        oracle.track(line, r, 1, start_elem=s, end_elem=e, energy=data["energy"])
        np.testing.assert_allclose(r, expected, atol=1e-7)
        np.testing.assert_array_equal(r, data["partial_%d_%d" % (s, e)])


# ---- known answers of the reference's own tests ---------------------------

def test_drift_divergence_known_answer(rin):
    rin[1, 0] = 1e-6
    rin[3, 0] = -2e-6
    _track_elem(E.Drift("d", 1.0), rin)
    np.testing.assert_equal(rin, np.array([1e-6, 1e-6, -2e-6, -2e-6, 0, 2.5e-12]).reshape(6, 1))


def test_two_particles_two_turns_known_answer():
    rin = np.asfortranarray(np.zeros((6, 2)))
    rin[1][0] = 1e-6
    rin[3][0] = -2e-6
    rout, _ = oracle.track([E.Drift("d", 1.0)], rin, 2, refpts=[1])
    np.testing.assert_equal(rout[:, 0, :, 0], np.array([1e-6, 1e-6, -2e-6, -2e-6, 0, 2.5e-12]).reshape(6, 1))
    np.testing.assert_equal(rout[:, 0, :, 1], np.array([2e-6, 1e-6, -4e-6, -2e-6, 0, 5e-12]).reshape(6, 1))
    np.testing.assert_equal(rout[:, 1, :, :], np.zeros((6, 1, 2)))


def test_quad_known_answer(rin):
    rin[0, 0] = 1e-6
    _track_elem(E.Quadrupole("q", 0.4, 1.0), rin)
    expected = np.array([0.9210610203854122, -0.3894182419439, 0, 0, 0, 0.0000000103303797478]).reshape(6, 1) * 1e-6
    np.testing.assert_allclose(rin, expected)


def test_dipole_known_answer(rin):
    rin[0, 0] = 1e-6
    _track_elem(E.Dipole("b", 1.0, 0.1, EntranceAngle=0.05, ExitAngle=0.05), rin)
    np.testing.assert_almost_equal(rin, np.array([1e-6, 0, 0, 0, 0, 1e-7]).reshape(6, 1))


def test_rfcavity_known_answer(rin):
    rfc = E.RFCavity("rf", 0.0, 187500, 3.5237e8, 31, 6.0e9)
    rin[4, 0] = 1e-6
    rin[5, 0] = 1e-6
    _track_elem(rfc, rin, 6.0e9, 0.0)
    np.testing.assert_allclose(rin, np.array([0, 0, 0, 0, 9.99769215e-07, 1.0e-6]).reshape(6, 1), atol=1e-12)


def test_corrector_known_answer(rin):
    rin[0, 0] = 1e-6
    expected = rin.copy()
    expected[1] = 0.9
    expected[3] = 0.5
    _track_elem(E.Corrector("c", 0.0, np.array([0.9, 0.5])), rin)
    np.testing.assert_equal(rin, expected)


def test_aperture_outside_limits_known_answer(rin):
    rin[0, 0] = 1e-2
    rin[2, 0] = -1e-2
    oracle.track([E.Aperture("a", [-1e-3, 1e-3, -1e-4, 1e-4])], rin, 1)
    assert np.isnan(rin[0, 0])
    assert rin[2, 0] == 0.0
