"""Linear optics and batched orbit searches against the reference's own
results (golden ``optics.npz``: the reference's linopt6 with chromaticity on
the radiating large ring and on its hmba.mat in 6-D, and its find_orbit6 of
four error-seeded large-ring variants, made by ``golden/make_golden.py``).

CPU tests run the optics with the oracle standing in for the engine's
tracking calls (the oracle is pinned bit for bit to the reference's engine):
the host algebra -- Newton steps, finite differences, normal form, phase
unwrapping, slip factor and chromaticity -- is then checked against the
reference at tight tolerances.  GPU tests run the same functions on the
engine.  Tolerances: closed orbits 1e-15 m (1e-13 for the batched engine
runs); optics functions (beta, alpha, dispersion, R, A, M) 1e-9 relative to
each array's scale; phases 1e-9 rad; tunes 1e-11; damping times 1e-8
relative; chromaticities 5e-5 absolute (a difference of two tunes divided by
the momentum step of 3e-6, so tune rounding of a few 1e-11 alone moves it by
1e-5).
"""
import json
import os

import numpy as np
import pytest

import cases
from at_b200 import elements as E
from at_b200 import optics, rings
from conftest import GOLDEN
from oracle import oracle


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(os.path.join(GOLDEN, "optics.npz")))


def hmba6d():
    with open(os.path.join(GOLDEN, "hmba.json")) as f:
        data = json.load(f)["6d"]
    line = [cases.make_element(d, E.Element) for d in data["specs"]]
    return E.Lattice(line, energy=data["energy"], particle="relativistic", periodicity=32)


class _OracleRings:
    """Stand-in for the engine's batched launches: each ring's particles on
    the oracle."""

    launches = 0

    def __init__(self, rings_, device=0):
        self.rings = list(rings_)

    def one_turn(self, which, parts):
        _OracleRings.launches += 1
        out = []
        for k, p in zip(which, parts):
            r = np.asfortranarray(np.array(p, dtype=np.float64))
            ring = self.rings[k]
            oracle.track(list(ring), r, 1, energy=ring.energy,
                         rest_energy=ring.particle.rest_energy)
            out.append(r)
        return out

    def close(self):
        pass


def _oracle_gpupass(ring, r, nturns, refpts=None, mode=None, gpu_pool=None, **kw):
    rout, _ = oracle.track(list(ring), r, nturns, refpts=refpts, energy=ring.energy,
                           rest_energy=ring.particle.rest_energy)
    return rout


def _oracle_exits(ring, r_in, device=0):
    out = np.array(r_in, dtype=np.float64, copy=True)
    for i, e in enumerate(ring):
        r = np.asfortranarray(out[i].reshape(6, 1).copy())
        oracle.track([e], r, 1, energy=ring.energy, rest_energy=ring.particle.rest_energy,
                     element=True, t0=0.0)
        out[i] = r[:, 0]
    return out


@pytest.fixture
def on_oracle(monkeypatch):
    monkeypatch.setattr(optics, "_Rings", _OracleRings)
    monkeypatch.setattr(optics, "gpupass", _oracle_gpupass)
    monkeypatch.setattr(optics, "element_exits", _oracle_exits)


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _check_linopt(res, gold, tag, fields, orbit_tol=1e-15):
    e0, bd, el = res
    np.testing.assert_allclose(bd.tune, gold[tag + "_bd_tune"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(bd.damping_time, gold[tag + "_bd_damping_time"], rtol=1e-8)
    np.testing.assert_allclose(bd.chromaticity, gold[tag + "_bd_chromaticity"], rtol=0,
                               atol=5e-5)
    for f in fields:
        for part, rec in (("el", el), ("e0", e0)):
            want = gold["%s_%s_%s" % (tag, part, f)]
            got = rec[f]
            if f == "closed_orbit":
                np.testing.assert_allclose(got, want, rtol=0, atol=orbit_tol, err_msg=f)
            elif f == "mu":
                np.testing.assert_allclose(got, want, rtol=0, atol=1e-9, err_msg=f)
            elif f == "s_pos":
                np.testing.assert_array_equal(got, want, err_msg=f)
            else:
                assert _rel(got, want) <= 1e-9, (tag, part, f, _rel(got, want))


FIELDS6 = ("alpha", "beta", "mu", "R", "A", "dispersion", "closed_orbit", "M", "s_pos")


def test_linopt6_large_ring_on_oracle(gold, on_oracle):
    ring = rings.large_ring()
    res = optics.linopt6(ring, refpts=gold["large_refpts"], get_chrom=True)
    _check_linopt(res, gold, "large", FIELDS6)


def test_linopt6_hmba_on_oracle(gold, on_oracle):
    ring = hmba6d()
    res = optics.linopt6(ring, refpts=gold["hmba_refpts"], get_chrom=True)
    _check_linopt(res, gold, "hmba", ("alpha", "beta", "mu", "dispersion", "closed_orbit",
                                      "M", "s_pos"))


def test_batched_orbits_on_oracle(gold, on_oracle):
    """Four error-seeded variants in one batch: each orbit is the reference's,
    with one launch per Newton step for all of them."""
    _OracleRings.launches = 0
    stats = {}
    vs = [rings.large_ring_variant(s) for s in (2, 3, 4, 5)]
    orbs = optics.find_orbit6_batch(vs, stats=stats)
    for s, o in zip((2, 3, 4, 5), orbs):
        np.testing.assert_allclose(o, gold["variant%d_orbit" % s], rtol=0, atol=1e-15)
    assert _OracleRings.launches <= 8          # Newton steps, not 4 x steps


def test_disable_6d_and_frequency_copies_share_unchanged_elements():
    ring = rings.large_ring()
    r4 = optics.disable_6d(ring)
    assert type(r4) is type(ring) and r4.energy == ring.energy
    pms = {e.PassMethod for e in r4}
    assert not any(p.endswith("RadPass") for p in pms) and "RFCavityPass" not in pms
    assert sum(a is b for a, b in zip(r4, ring)) > 0            # drifts are shared
    assert all(e.PassMethod.endswith("RadPass") for e in ring
               if e.PassMethod.startswith(("StrMPole", "BndMPole")))     # original untouched
    up = optics._with_frequency_scale(ring, 1.0 + 1e-6)
    for i in optics._cavities(ring):
        assert up[i].Frequency == ring[i].Frequency * (1.0 + 1e-6)


@pytest.mark.gpu
def test_linopt6_large_ring_on_engine(gold):
    res = optics.linopt6(rings.large_ring(), refpts=gold["large_refpts"], get_chrom=True)
    _check_linopt(res, gold, "large", FIELDS6, orbit_tol=1e-13)


@pytest.mark.gpu
def test_linopt6_hmba_on_engine(gold):
    res = optics.linopt6(hmba6d(), refpts=gold["hmba_refpts"], get_chrom=True)
    _check_linopt(res, gold, "hmba", ("alpha", "beta", "mu", "dispersion", "closed_orbit",
                                      "M", "s_pos"), orbit_tol=1e-13)


@pytest.mark.gpu
def test_batched_orbits_on_engine_equal_single_searches(gold):
    """The batched search on the engine: each variant's orbit equals its own
    single-ring search bit for bit (same particles, same arithmetic) and the
    reference's to 1e-13."""
    from at_b200 import physics
    vs = [rings.large_ring_variant(s) for s in (2, 3, 4, 5)]
    stats = {}
    orbs = optics.find_orbit6_batch(vs, stats=stats)
    for s, v, o in zip((2, 3, 4, 5), vs, orbs):
        np.testing.assert_allclose(o, gold["variant%d_orbit" % s], rtol=0, atol=1e-13)
        np.testing.assert_array_equal(o, physics.find_orbit6(v, mode="exact"))
    assert stats["launches"] <= 8


@pytest.mark.gpu
def test_energy_loss_in_one_launch_equals_element_calls():
    from at_b200 import physics
    from at_b200.tracking import elempass
    ring = rings.large_ring()

    def et(e, r):
        elempass(e, r, energy=ring.energy, particle=ring.particle, mode="exact")

    assert optics.energy_loss(ring) == physics.energy_loss(ring, et)
