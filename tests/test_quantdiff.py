"""Quantum diffusion: the QuantDiffPass element and its lumped matrix.

The oracle restates the reference's pass with its random stream (PCG32 and
Marsaglia's polar method, reseeded by reset_rng) and is pinned bit for bit to
the reference (``golden/quantdiff.npz``, ``golden/make_golden.py``).  The GPU
draws its kicks from a counter-based generator instead of one sequential
stream, so engine and oracle agree in distribution, not sample by sample:
the tests check the kicks' mean, covariance and normality against L L^T and
against the oracle's sample, their independence across elements and turns,
reproducibility under reset_rng, and, as physics, that a bunch started on
the Ohmi envelope of the radiating large ring keeps its energy spread and
bunch length when the ring carries its generated diffusion element (and
loses them without it).
"""
import os

import numpy as np
import pytest

from at_b200 import elements as E
from at_b200 import radiation, rings
from at_b200.lattice import compile_lattice
from conftest import ELECTRON_REST, GOLDEN
from oracle import oracle


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(os.path.join(GOLDEN, "quantdiff.npz")))


def _line(g):
    return E.Lattice([
        E.Drift("D1", 0.5),
        E.QuantumDiffusion("QD1", g["l0"]),
        E.Quadrupole("Q", 0.4, 1.2),
        E.QuantumDiffusion("QD2", g["l1"]),
        E.Drift("D2", 0.3),
    ], energy=3e9, particle="electron")


def test_oracle_quantdiff_matches_reference_stream(gold):
    line = _line(gold)
    oracle.reset_rng(seed=4242)
    r = gold["rin"].copy(order="F")
    oracle.track(line, r, 3, energy=3e9, rest_energy=ELECTRON_REST)
    np.testing.assert_array_equal(r, gold["r1"])
    rout, _ = oracle.track(line, r, 2, refpts=gold["refpts"], energy=3e9,
                           rest_energy=ELECTRON_REST)
    np.testing.assert_array_equal(r, gold["r2"])
    np.testing.assert_array_equal(rout, gold["rout"])


def test_lmat_of_the_large_ring_matches_reference(gold):
    """gen_quantdiff_elem's factor, from the reference's own cumulative
    diffusion matrix (golden) through the restated symmetrisation and
    Cholesky factorisation."""
    bcum = np.load(os.path.join(GOLDEN, "ohmi_large.npz"))["bcum"]
    lm = radiation.lmat(0.5 * (bcum + bcum.T))
    scale = np.abs(gold["large_lmatp"]).max()
    np.testing.assert_allclose(lm, gold["large_lmatp"], rtol=0, atol=1e-12 * scale)


def test_quantdiff_compiles_to_the_table(gold):
    cl = compile_lattice(_line(gold), 3e9, ELECTRON_REST)
    from at_b200 import table as T
    w = cl.words[int(cl.offsets[1]):int(cl.offsets[2])]
    np.testing.assert_array_equal(w[T.ATB_QD_L:T.ATB_QD_L + 36], gold["l0"].ravel(order="F"))


def test_rng_keys_follow_reset():
    from at_b200 import tracking
    tracking.reset_rng(seed=5)
    a = [tracking._next_rng_key(0)]
    tracking._rng["calls"] += 1
    a.append(tracking._next_rng_key(0))
    tracking.reset_rng(seed=5)
    assert tracking._next_rng_key(0) == a[0] and a[0] != a[1]
    assert tracking._next_rng_key(1) != a[0]
    tracking.reset_rng(seed=6)
    assert tracking._next_rng_key(0) != a[0]


# ---------------------------------------------------------------- GPU tests --

def _kicks(line, n, nturns=1, seed=11):
    from at_b200 import tracking
    tracking.reset_rng(seed=seed)
    r = np.asfortranarray(np.zeros((6, n)))
    tracking.gpupass(line, r, nturns, mode="exact")
    return r


@pytest.mark.gpu
def test_zero_matrix_is_identity(gold):
    from at_b200 import tracking
    line = _line(gold)
    z = E.Lattice([e if e.PassMethod != "QuantDiffPass" else
                   E.QuantumDiffusion(e.FamName, np.zeros((6, 6))) for e in line],
                  energy=3e9, particle="electron")
    plain = E.Lattice([e for e in line if e.PassMethod != "QuantDiffPass"], energy=3e9,
                      particle="electron")
    r0 = gold["rin"][:, 8:].copy(order="F")
    ra, rb = r0.copy(order="F"), r0.copy(order="F")
    tracking.gpupass(z, ra, 3, mode="exact")
    tracking.gpupass(plain, rb, 3, mode="exact")
    np.testing.assert_array_equal(ra, rb)


@pytest.mark.gpu
def test_kick_statistics(gold):
    """2^20 particles through one element: the whitened kicks L^-1 d have
    zero mean, unit covariance (5 standard errors) and Gaussian one-sigma
    and two-sigma fractions."""
    L = gold["l1"]
    n = 1 << 20
    d = _kicks(E.Lattice([E.QuantumDiffusion("Q", L)], energy=3e9, particle="electron"), n)
    z = np.linalg.solve(L, d)
    se = 1.0 / np.sqrt(n)
    assert np.abs(z.mean(axis=1)).max() < 5 * se
    cov = np.cov(z)
    assert np.abs(cov - np.eye(6)).max() < 5 * np.sqrt(2.0) * se
    for k, p in ((1.0, 0.682689492), (2.0, 0.954499736)):
        frac = (np.abs(z) < k).mean(axis=1)
        assert np.abs(frac - p).max() < 5 * np.sqrt(p * (1 - p) / n)


@pytest.mark.gpu
def test_kicks_independent_across_elements_and_turns(gold):
    """Two elements over three turns: the variance of the summed kicks is
    six times L L^T (kicks of different elements and turns uncorrelated)."""
    L = gold["l0"]
    line = E.Lattice([E.QuantumDiffusion("Q1", L), E.QuantumDiffusion("Q2", L)], energy=3e9,
                     particle="electron")
    n = 1 << 19
    d = _kicks(line, n, nturns=3)
    z = np.linalg.solve(L, d) / np.sqrt(6.0)
    cov = np.cov(z)
    assert np.abs(cov - np.eye(6)).max() < 6 * np.sqrt(2.0 / n)


@pytest.mark.gpu
def test_reproducible_under_reset_rng(gold):
    line = _line(gold)
    a = _kicks(line, 4096, nturns=2, seed=99)
    b = _kicks(line, 4096, nturns=2, seed=99)
    c = _kicks(line, 4096, nturns=2, seed=100)
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, c)
    from at_b200 import tracking
    tracking.reset_rng(seed=99)
    r1 = np.asfortranarray(np.zeros((6, 4096)))
    r2 = np.asfortranarray(np.zeros((6, 4096)))
    tracking.gpupass(line, r1, 2, mode="exact")
    tracking.gpupass(line, r2, 2, mode="exact")        # the next call: new kicks
    assert not np.array_equal(r1, r2)


@pytest.mark.gpu
def test_engine_and_oracle_agree_in_distribution(gold):
    """The golden line, 3 turns, 2^18 particles from one start point: the
    engine's and the oracle's (reference stream) final distributions have
    the same mean and covariance within their sampling errors."""
    line = _line(gold)
    n = 1 << 18
    x0 = np.tile(gold["rin"][:, :1], (1, n))
    g = np.asfortranarray(x0.copy())
    from at_b200 import tracking
    tracking.reset_rng(seed=3)
    tracking.gpupass(line, g, 3, mode="exact")
    o = np.asfortranarray(x0.copy())
    oracle.reset_rng(seed=3)
    oracle.track(line, o, 3, energy=3e9, rest_energy=ELECTRON_REST)
    sd = np.sqrt(np.diag(np.cov(o)))
    assert np.all(np.abs(g.mean(axis=1) - o.mean(axis=1)) < 6 * sd * np.sqrt(2.0 / n))
    cg = np.cov(g) / np.outer(sd, sd)
    co = np.cov(o) / np.outer(sd, sd)
    assert np.abs(cg - co).max() < 6 * np.sqrt(2.0 / n) * 2


@pytest.mark.gpu
def test_equilibrium_on_the_ohmi_envelope():
    """The radiating large ring with its generated diffusion element at the
    end: a bunch started on the envelope R66 at the entrance keeps its
    energy spread, bunch length and vertical size over half a longitudinal
    damping time (3,200 turns); without the element they damp."""
    from at_b200 import tracking
    ring = rings.large_ring(seed=1)
    emit0, beamdata, _ = radiation.ohmi_envelope(ring)
    orbit, r66 = emit0.orbit6, emit0.r66
    qd = radiation.gen_quantdiff_elem(ring, orbit)
    with_qd = E.Lattice(list(ring) + [qd], energy=ring.energy, particle=ring.particle)
    n = 148 * 256
    w, v = np.linalg.eigh(r66)
    root = v @ np.diag(np.sqrt(np.maximum(w, 0.0))) @ v.T
    x0 = np.asfortranarray(orbit[:, None] + root @ np.random.default_rng(2).standard_normal(
        (6, n)))
    c0 = np.cov(x0)
    tracking.reset_rng(seed=21)
    a = x0.copy(order="F")
    tracking.gpupass(with_qd, a, 3200)
    ca = np.cov(a[:, ~np.isnan(a[0])])
    for k, tol in ((4, 0.06), (5, 0.06), (2, 0.10)):
        assert abs(ca[k, k] / c0[k, k] - 1.0) < tol, (k, ca[k, k] / c0[k, k])
    b = x0.copy(order="F")
    tracking.gpupass(ring, b, 1600)
    cb = np.cov(b[:, ~np.isnan(b[0])])
    assert cb[4, 4] / c0[4, 4] < 0.8 and cb[5, 5] / c0[5, 5] < 0.8
    print("variance ratios with diffusion: delta %.4f ct %.4f y %.4f; without: delta %.4f"
          % (ca[4, 4] / c0[4, 4], ca[5, 5] / c0[5, 5], ca[2, 2] / c0[2, 2],
             cb[4, 4] / c0[4, 4]))
