"""The drop-in entry points with the reference's own test cases.

These restate pyat/test/test_atpass.py:8-183 and the element tests of
pyat/test/test_basic_elements.py against ``at_b200.gpupass``/``elempass``:
same inputs, same expected values and tolerances, same exception types.
"""
import json
import os

import numpy as np
import pytest

import at_b200
import cases
from at_b200 import elements as E
from at_b200 import rings
from oracle import oracle

from conftest import ELECTRON_REST, GOLDEN, scale_rel_diff

pytestmark = pytest.mark.gpu
atpass = at_b200.atpass
elempass = at_b200.elempass


def uint32_refpts(refs, n):
    return np.asarray(refs, dtype=np.uint32)


def test_incorrect_types_raises_type_error(rin):
    with pytest.raises(TypeError):
        atpass(1, rin, 1)
    with pytest.raises(TypeError):
        atpass([], 1, 1)
    with pytest.raises(TypeError):
        atpass([], rin, "a")


def test_incorrect_dimensions_raises_value_error():
    with pytest.raises(ValueError):
        atpass([], np.array(np.zeros((7, 1))), 1)
    with pytest.raises(ValueError):
        atpass([], np.array(np.zeros((1, 6))), 1)


def test_c_aligned_array_raises_value_error():
    with pytest.raises(ValueError):
        atpass([], np.zeros((2, 6)), 1)


def test_transposed_array_raises_value_error():
    with pytest.raises(ValueError):
        atpass([], np.asfortranarray(np.zeros((2, 6))).T, 1)


def test_transposed_c_array_does_not_raise():
    atpass([], np.zeros((2, 6)).T, 1)


def test_transposed_c_array_gives_same_result_as_fortran_array():
    rin_fortran = np.array(np.arange(12).reshape(6, 2), order="F") * 1e-5
    rin_c = np.copy(rin_fortran.T, order="C")
    lat = [E.Drift("drift", 1.0)]
    rout_fortran = atpass(lat, rin_fortran, 1)
    rout_c = atpass(lat, rin_c.T, 1)
    np.testing.assert_equal(rout_c, rout_fortran)


def test_missing_pass_method_raises_attribute_error(rin):
    lat = [E.Marker("marker")]
    del lat[0].PassMethod
    with pytest.raises(AttributeError):
        atpass(lat, rin, 1)


def test_missing_integrator_raises_runtime_error(rin):
    with pytest.raises(RuntimeError):
        atpass([E.Drift("drift", 1.0, PassMethod="UnknownPass")], rin, 1)


def test_integrator_error(rin):
    lat = [E.Drift("drift", 1.0)]
    del lat[0].Length
    with pytest.raises(AttributeError):
        atpass(lat, rin, 1)


@pytest.mark.parametrize("reuse", (True, False))
def test_reuse_attributes(rin, reuse):
    lat = [E.Drift("drift", 1.0)]
    rin[0, 0] = 1e-6
    rin[1, 0] = 1e-6
    rin_copy = np.copy(rin)
    atpass(lat, rin, 2)
    atpass(lat, rin_copy, 1)
    lat[0].Length = 2
    atpass(lat, rin_copy, 1, reuse=reuse)
    if reuse:
        np.testing.assert_equal(rin, rin_copy)
    else:
        with pytest.raises(AssertionError):
            np.testing.assert_equal(rin, rin_copy)


def test_two_particles_for_two_turns():
    rin = np.asfortranarray(np.zeros((6, 2)))
    lat = [E.Drift("drift", 1.0)]
    rin[1][0] = 1e-6
    rin[3][0] = -2e-6
    rout = atpass(lat, rin, 2, refpts=uint32_refpts([1], 1))
    np.testing.assert_equal(rout[:, 0, :, 0], np.array([1e-6, 1e-6, -2e-6, -2e-6, 0, 2.5e-12]).reshape(6, 1))
    np.testing.assert_equal(rout[:, 1, :, 0], np.zeros((6, 1)))
    np.testing.assert_equal(rout[:, 0, :, 1], np.array([2e-6, 1e-6, -4e-6, -2e-6, 0, 5e-12]).reshape(6, 1))
    np.testing.assert_equal(rout[:, 1, :, 1], np.zeros((6, 1)))


def test_one_particle_for_two_turns_with_no_refpts(rin):
    lat = [E.Drift("drift", 1.0)]
    rin[1][0] = 1e-6
    rin[3][0] = -2e-6
    atpass(lat, rin, 2)
    np.testing.assert_equal(rin, np.array([2e-6, 1e-6, -4e-6, -2e-6, 0, 5e-12]).reshape(6, 1))


def test_1d_particle():
    lat = [E.Drift("drift", 1.0)]
    rin = np.zeros(6)
    rin[1] = 1e-6
    rout = atpass(lat, rin, 1)
    assert rout.shape == (6, 1, 0, 1)
    np.testing.assert_equal(rin, np.array([1e-6, 1e-6, 0, 0, 0, 5e-13]))


def _hmba_off():
    with open(os.path.join(GOLDEN, "hmba.json")) as f:
        data = json.load(f)["off"]
    lat = E.Lattice([cases.make_element(d, E.Element) for d in data["specs"]],
                    energy=data["energy"], particle="relativistic")
    return lat, data


def test_start_elem():
    lat, data = _hmba_off()
    rin = np.array([0, 1e-6, 0, 0, 0, 0])
    rout = atpass(lat, rin, 1, start_elem=100)
    assert rout.shape == (6, 1, 0, 1)
    np.testing.assert_allclose(rin, np.array([3.2e-6, -1.1e-6, 0, 0, 0, 8.4e-8]), atol=1e-7)
    np.testing.assert_allclose(rin, data["partial_100_0"], rtol=0, atol=1e-18)


def test_end_elem():
    lat, data = _hmba_off()
    rin = np.array([0, 1e-6, 0, 0, 0, 0])
    rout = atpass(lat, rin, 1, start_elem=100, end_elem=110)
    assert rout.shape == (6, 1, 0, 1)
    np.testing.assert_allclose(rin, np.array([2.6e-6, 1.34e-6, 0, 0, 0, 2.4e-8]), atol=1e-7)
    np.testing.assert_allclose(rin, data["partial_100_110"], rtol=0, atol=1e-18)


def test_start_end_elem_errors():
    lat, _ = _hmba_off()
    rin = np.array([0, 1e-6, 0, 0, 0, 0])
    with pytest.raises(ValueError):
        atpass(lat, rin, 1, start_elem=200)
    with pytest.raises(ValueError):
        atpass(lat, rin, 1, end_elem=200)
    with pytest.raises(ValueError):
        atpass(lat, rin, 1, start_elem=100, end_elem=10)
    with pytest.raises(ValueError):
        atpass(lat, rin, 2, end_elem=10)


def test_refpts_dtype_error(rin):
    with pytest.raises(ValueError):
        atpass([E.Drift("d", 1.0)], rin, 1, refpts=np.array([0, 1], dtype=np.int64))


def test_rf_needs_energy(rin):
    with pytest.raises(ValueError):
        elempass(E.RFCavity("rf", 0.0, 1e6, 3.5e8, 31, 6e9), rin)
    with pytest.raises(TypeError):
        elempass(E.RFCavity("rf", 0.0, 1e6, 3.5e8, 31, 6e9), rin, energy=6000000000)


def test_unsupported_pass_method_has_no_fallback(rin):
    with pytest.raises(RuntimeError):
        atpass([E.Element("m66", PassMethod="Matrix66Pass")], rin, 1)


# ---- element tests (pyat/test/test_basic_elements.py) ---------------------

def test_drift_divergence(rin):
    rin[1, 0] = 1e-6
    rin[3, 0] = -2e-6
    elempass(E.Drift("drift", 1.0), rin)
    np.testing.assert_equal(rin, np.array([1e-6, 1e-6, -2e-6, -2e-6, 0, 2.5e-12]).reshape(6, 1))


def test_drift_offset(rin):
    rin[0, 0] = 1e-6
    rin[2, 0] = 2e-6
    orig = rin.copy()
    elempass(E.Drift("drift", 1), rin)
    np.testing.assert_equal(rin, orig)


def test_quad(rin):
    rin[0, 0] = 1e-6
    elempass(E.Quadrupole("quad", 0.4, k=1), rin)
    expected = np.array([0.9210610203854122, -0.3894182419439, 0, 0, 0, 0.0000000103303797478]).reshape(6, 1) * 1e-6
    np.testing.assert_allclose(rin, expected)


def test_dipole(rin):
    rin[0, 0] = 1e-6
    elempass(E.Dipole("dipole", 1.0, 0.1, EntranceAngle=0.05, ExitAngle=0.05), rin)
    np.testing.assert_almost_equal(rin, np.array([1e-6, 0, 0, 0, 0, 1e-7]).reshape(6, 1))


def test_rfcavity(rin):
    rfc = E.RFCavity("rfcavity", 0.0, 187500, 3.5237e8, 31, 6.0e9)
    rin[4, 0] = 1e-6
    rin[5, 0] = 1e-6
    elempass(rfc, rin, energy=+6.0e9)
    np.testing.assert_allclose(rin, np.array([0.0, 0.0, 0.0, 0.0, 9.99769215e-07, 1.0e-6]).reshape(6, 1), atol=1e-12)


def test_corrector(rin):
    rin[0, 0] = 1e-6
    orig = rin.copy()
    orig[1] = 0.9
    orig[3] = 0.5
    elempass(E.Corrector("corrector", 0.0, np.array([0.9, 0.5], dtype=np.float64)), rin)
    np.testing.assert_equal(rin, orig)


def test_marker_and_monitor(rin):
    for el in (E.Marker("m"), E.Monitor("mon")):
        r = np.array(np.random.rand(*rin.shape), order="F")
        orig = r.copy()
        elempass(el, r)
        np.testing.assert_equal(r, orig)


def test_aperture_inside_limits(rin):
    rin[0, 0] = 1e-5
    rin[2, 0] = -1e-5
    orig = rin.copy()
    elempass(E.Aperture("aperture", [-1e-3, 1e-3, -1e-4, 1e-4]), rin)
    np.testing.assert_equal(rin, orig)


def test_aperture_outside_limits(rin):
    rin[0, 0] = 1e-2
    rin[2, 0] = -1e-2
    atpass([E.Aperture("aperture", [-1e-3, 1e-3, -1e-4, 1e-4])], rin, 1)
    assert np.isnan(rin[0, 0])
    assert rin[2, 0] == 0.0


def test_patpass_like_multiple_particles_and_turns():
    """pyat/test/test_patpass.py:12-37 through the drop-in."""
    nturns, nparticles = 10, 10
    rin = np.zeros((6, nparticles), order="F")
    rin[1, 0] = 1e-6
    rin[3, 0] = -2e-6
    rout = atpass([E.Drift("drift", 1.0)], rin, nturns, refpts=uint32_refpts([1], 1))
    assert rout.shape == (6, nparticles, 1, nturns)
    np.testing.assert_equal(rout[:, 0, :, 0], np.array([1e-6, 1e-6, -2e-6, -2e-6, 0, 2.5e-12]).reshape(6, 1))
    for j in range(1, nparticles):
        np.testing.assert_equal(rout[:, j, 0, :], np.zeros((6, nturns)))


# ---- engine semantics -------------------------------------------------------

def test_keep_counter_and_turn_through_rf():
    """The RF phase uses the absolute turn number (attrackfunc.c:24): tracking
    2+3 turns with keep_counter (or turn=2) equals 5 turns in one call."""
    ring = rings.fodo_ring()
    r0 = rings.gaussian(512, seed=9)
    a = r0.copy(order="F")
    atpass(ring, a, 5, mode="exact")
    b = r0.copy(order="F")
    atpass(ring, b, 2, mode="exact")
    atpass(ring, b, 3, keep_counter=True, reuse=True, mode="exact")
    np.testing.assert_array_equal(a, b)
    c = r0.copy(order="F")
    atpass(ring, c, 2, mode="exact")
    atpass(ring, c, 3, turn=2, mode="exact")
    np.testing.assert_array_equal(a, c)
    d = r0.copy(order="F")
    ro = r0.copy(order="F")
    atpass(ring, d, 3, turn=7, mode="exact")
    oracle.track(ring, ro, 3, turn=7, energy=3e9, rest_energy=ELECTRON_REST)
    assert scale_rel_diff(d, ro) <= 1e-14


def test_losses_dict_layout():
    ring = rings.fodo_ring()
    r = rings.gaussian(300, seed=2) * 6.0
    r = np.asfortranarray(r)
    rout, ld = atpass(ring, r, 50, losses=True)
    assert set(ld) == {"islost", "turn", "elem", "coord"}
    assert ld["islost"].dtype == np.bool_ and ld["turn"].dtype == np.uint32
    assert ld["elem"].dtype == np.uint32 and ld["coord"].shape == (6, 300)
    assert ld["coord"].flags.f_contiguous
    lost = ld["islost"]
    assert lost.any() and not lost.all()
    assert np.all(np.isnan(r[0, lost])) and np.all(r[1:, lost] == 0)
    assert np.all(ld["turn"][~lost] == 0) and np.all(ld["coord"][:, ~lost] == 0)


def test_per_turn_statistics_match_final_state():
    ring = rings.fodo_ring()
    r = np.asfortranarray(rings.gaussian(2000, seed=2) * 5.0)
    (rout, ld, st) = at_b200.gpupass(ring, r, 20, losses=True, stats=True)
    alive, mom = st
    assert alive[-1] == int((~ld["islost"]).sum())
    ok = ~ld["islost"]
    np.testing.assert_allclose(mom[-1, :6], r[:, ok].sum(axis=1), rtol=1e-10, atol=1e-15)
    assert np.all(np.diff(alive.astype(np.int64)) <= 0)


def test_gpuinfo():
    info = at_b200.gpuinfo()
    assert len(info) >= 1
    name, ver, sms, plat = info[0]
    assert sms > 0 and plat == "CUDA"
