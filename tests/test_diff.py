"""Exact derivatives of tracking (the tangent kernel and its autograd bridge).

The Jacobian with respect to the initial coordinates is checked against the
reference's own one-turn matrix (``find_m66``, pyat/at/physics/matrix.py:
105-165, stored in ``golden/fodo_m66.npz`` by ``golden/make_golden.py``) and
against central finite differences; the derivatives with respect to the 64
quadrupole and 64 sextupole strengths of the FODO ring against central finite
differences with h = 1e-7 and, where the second-order sextupole effect is
below what a step of 1e-7 resolves, a fourth-order difference at a larger
amplitude.  The finite differences track with the exact-arithmetic engine
(whose values the oracle pins bit for bit); the tangent kernel's own values
are checked against that engine too.
"""
import numpy as np
import pytest

from at_b200 import diff, rings
from conftest import ELECTRON_REST
from oracle import oracle

XYSTEP = 3e-8      # DConstant.XYStep of the reference
DPSTEP = 3e-6      # DConstant.DPStep of the reference
S6 = np.kron(np.eye(3), np.array([[0.0, 1.0], [-1.0, 0.0]]))


def _perturbed(line, idx, order, delta):
    lat = line.copy()
    el = line[idx].copy()
    pb = np.array(el.PolynomB, dtype=np.float64)
    pb[order] += delta
    el.PolynomB = pb
    lat[idx] = el
    return lat


# ---------------------------------------------------------------- CPU tests --

def test_fodo_strengths_are_64_quads_and_64_sextupoles():
    ring = rings.fodo_ring()
    ps = diff.multipole_strengths(ring)
    assert len(ps) == 128
    quads, sexts = ps[:64], ps[64:]
    assert all(p.order == 1 for p in quads) and all(p.order == 2 for p in sexts)
    assert [p.index for p in quads] == sorted([12 * c for c in range(32)] +
                                              [12 * c + 6 for c in range(32)])
    assert [p.index for p in sexts] == sorted([12 * c + 2 for c in range(32)] +
                                              [12 * c + 8 for c in range(32)])
    assert {ring[p.index].FamName for p in quads} == {"QF", "QD"}
    assert {ring[p.index].FamName for p in sexts} == {"SF", "SD"}


@pytest.mark.parametrize("params,msg", [
    ([(1, 1)], "no differentiable PolynomB"),            # a drift
    ([(0, 2)], "outside \\[1, MaxOrder"),                # quad MaxOrder is 1
    ([(0, 0)], "outside \\[1, MaxOrder"),                # order 0 carries KickAngle
    ([(0, 1), (0, 1)], "two strengths"),
    ([(10_000, 1)], "outside the lattice"),
])
def test_tracker_rejects_bad_strengths(params, msg):
    with pytest.raises(ValueError, match=msg):
        diff.TangentTracker(rings.fodo_ring(), params)


def test_oracle_fd_matrix_matches_reference_find_m66(golden):
    """The oracle, differentiated the way find_m66 does it (12 particles,
    XYStep/DPStep central differences), reproduces the reference's matrix:
    pins the golden one-turn matrix to the restated integrators."""
    g = golden("fodo_m66.npz")
    orbit, m_ref = g["orbit"], g["m66"]
    steps = np.array([XYSTEP] * 4 + [DPSTEP] * 2)
    d = np.diag(0.5 * steps)
    r = np.asfortranarray(np.concatenate((orbit[:, None] + d, orbit[:, None] - d), axis=1))
    oracle.track(rings.fodo_ring(), r, 1, energy=3e9, rest_energy=ELECTRON_REST)
    m = (r[:, :6] - r[:, 6:]) / steps[None, :]
    np.testing.assert_allclose(m, m_ref, rtol=0, atol=1e-12)


def _oracle_one_turn(line):
    def run(r):
        r = np.asfortranarray(r)
        oracle.track(line, r, 1, energy=line.energy, rest_energy=line.particle.rest_energy)
        return r
    return run


def _oracle_element(line):
    def run(el, r):
        oracle.track([el], r, 1, energy=line.energy, rest_energy=line.particle.rest_energy,
                     element=True, t0=0.0)
    return run


def test_orbit6_matches_reference_find_orbit6(golden):
    """The closed-orbit Newton iteration (with the reference's RF slip
    theta), run on the oracle, lands on the reference's orbit; that orbit
    satisfies M(x) = x + theta."""
    from at_b200 import physics
    ring = rings.fodo_ring()
    g = golden("fodo_m66.npz")
    x = physics._orbit6(ring, _oracle_one_turn(ring))
    np.testing.assert_allclose(x, g["orbit"], rtol=0, atol=1e-15)
    theta = physics._rf_theta(ring)
    assert theta[5] < 0 and abs(theta[5] + 2.7853e-6) < 1e-9      # C (beta - 1)
    r = _oracle_one_turn(ring)(g["orbit"].reshape(6, 1).copy())
    np.testing.assert_allclose(r[:, 0], g["orbit"] + theta, rtol=0, atol=1e-13)


def test_large_ring_orbit_constant_on_oracle():
    """LARGE_ORBIT is the large ring's closed orbit on the oracle."""
    from at_b200 import physics
    ring = rings.large_ring(seed=1)
    el = _oracle_element(ring)
    # the search starts at the synchronous ct of the radiation loss
    u0 = physics.energy_loss(ring, el)
    assert 3.3e5 < u0 < 3.4e5
    x = physics._orbit6(ring, _oracle_one_turn(ring), elem_track=el)
    np.testing.assert_allclose(x, rings.LARGE_ORBIT, rtol=0, atol=1e-15)


# ---------------------------------------------------------------- GPU tests --

torch = pytest.importorskip("torch")


def _dev_rows(r_fortran):
    """(6, N) host array -> (N, 6) float64 tensor on cuda:0."""
    return torch.tensor(np.ascontiguousarray(np.asarray(r_fortran).T), dtype=torch.float64,
                        device="cuda:0")


def _engine_track(line, r, nturns):
    """Exact-arithmetic tracking of a (6, N) array through the plain engine."""
    from at_b200 import tracking
    out = np.asfortranarray(r.copy())
    tracking.gpupass(line, out, nturns, mode="exact")
    return out


def _fodo_bunch(n, sigma=1e-6, seed=0, orbit=None):
    return rings.gaussian(n, [sigma] * 6, seed=seed, centre=orbit)


@pytest.fixture(scope="module")
def fodo():
    return rings.fodo_ring()


@pytest.fixture(scope="module")
def ref_orbit():
    import os
    from conftest import GOLDEN
    return np.load(os.path.join(GOLDEN, "fodo_m66.npz"))["orbit"]


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["fodo", "large"])
def test_tangent_values_equal_exact_engine(which):
    """The tangent kernel tracks the same values as the exact tracking kernel,
    bit for bit, with every pass method and losses."""
    if which == "fodo":
        line, nt = rings.fodo_ring(), 30
        r0 = rings.gaussian(2048, seed=4)
        r0[:, :64] *= 30.0          # some lost
    else:
        line, nt = rings.large_ring(seed=1), 2
        r0 = rings.large_ring_bunch(512, seed=2)
    want = np.asfortranarray(r0.copy())
    from at_b200 import tracking
    tracking.gpupass(line, want, nt, mode="exact")
    tr = diff.TangentTracker(line, diff.multipole_strengths(line)[:8])
    try:
        r, jac, grad, lost = tr.track(_dev_rows(r0), None, nt)
        got = r.cpu().numpy().T
        assert np.array_equal(np.isnan(got[0]), np.isnan(want[0]))
        ok = ~np.isnan(want[0])
        assert np.array_equal(got[:, ok], want[:, ok])
        lost = lost.cpu().numpy()
        assert np.array_equal(lost, np.isnan(want[0]))
        if which == "fodo":
            assert lost.sum() > 0 and (~lost).sum() > 0
        j = jac.cpu().numpy()
        assert np.all(np.isnan(j[lost])) and np.all(np.isfinite(j[~lost]))
    finally:
        tr.close()


@pytest.mark.gpu
def test_m66_matches_reference_find_m66(fodo, golden):
    g = golden("fodo_m66.npz")
    m, _ = diff.find_m66(fodo, orbit=g["orbit"])
    # the reference's matrix is a central difference with DPStep 3e-6: its
    # truncation error in the dispersion column (third-order chromatic
    # terms) is ~6e-8; elsewhere it agrees to ~1e-10
    np.testing.assert_allclose(m, g["m66"], rtol=0, atol=1e-7)
    np.testing.assert_allclose(np.delete(m, 4, axis=1), np.delete(g["m66"], 4, axis=1),
                               rtol=0, atol=1e-9)
    # the engine differentiated the reference's way gives the reference's matrix
    from at_b200 import physics
    mfd, _ = physics.find_m66(fodo, orbit=g["orbit"], mode="exact")
    np.testing.assert_allclose(mfd, g["m66"], rtol=0, atol=1e-12)
    # the exact Jacobian of a symplectic map is symplectic to rounding
    assert np.abs(m.T @ S6 @ m - S6).max() < 1e-12
    # and the reference's closed orbit is the engine's too
    o = physics.find_orbit6(fodo, mode="exact")
    np.testing.assert_allclose(o, g["orbit"], rtol=0, atol=1e-14)


EPS = np.finfo(np.float64).eps


def _assert_fd(got, fd, rmag, h, what, coord_axis, rel=1e-7, ulps=64):
    """Blockwise agreement with a finite difference: for every block (all
    axes but the particle axis, which is last), max |got - fd| must be below
    rel * max |fd| plus the difference's own rounding floor,
    ulps * eps * |r_i| / h, |r_i| the size of the tracked output coordinate
    i, which runs along ``coord_axis``."""
    d = np.abs(got - fd).max(axis=-1)
    s = np.abs(fd).max(axis=-1)
    shape = [1] * d.ndim
    shape[coord_axis] = 6
    noise = np.broadcast_to((ulps * EPS / h) * np.asarray(rmag).reshape(shape), d.shape)
    bound = rel * s + noise
    bad = d > bound
    if bad.any():
        k = np.unravel_index(np.argmax(d / np.maximum(bound, 1e-300)), d.shape)
        raise AssertionError("%s: %d blocks off; worst %s: |diff| %.3e, scale %.3e, floor %.3e"
                             % (what, int(bad.sum()), k, d[k], s[k], noise[k]))
    return float((d / np.maximum(s, 1e-300)).max())


def _coord_fd(line, x, nturns, h, order4=False):
    """(6 out, 6 in, N) differences of the final coordinates with respect to
    the initial ones, through the exact engine."""
    n = x.shape[1]
    offs = (h, -h, 2 * h, -2 * h) if order4 else (h, -h)
    cols = []
    for j in range(6):
        for o in offs:
            xx = x.copy()
            xx[j] += o
            cols.append(xx)
    out = _engine_track(line, np.asfortranarray(np.concatenate(cols, axis=1)), nturns)
    out = out.reshape(6, 6, len(offs), n)          # (i, j, offset, particle)
    if order4:
        fd = (8 * (out[:, :, 0] - out[:, :, 1]) - (out[:, :, 2] - out[:, :, 3])) / (12 * h)
    else:
        fd = (out[:, :, 0] - out[:, :, 1]) / (2 * h)
    return fd


def _fd_strengths(line, params, x, nturns, h, order4=False):
    """Central differences (fourth order when ``order4``) of the final
    coordinates with respect to each strength, shape (P, 6, N)."""
    out = np.empty((len(params), 6, x.shape[1]))
    for q, p in enumerate(params):
        def run(delta):
            return _engine_track(_perturbed(line, p.index, p.order, delta), x, nturns)
        if order4:
            out[q] = (8 * (run(h) - run(-h)) - (run(2 * h) - run(-2 * h))) / (12 * h)
        else:
            out[q] = (run(h) - run(-h)) / (2 * h)
    return out


def _rmag(line, x, nturns):
    return np.abs(_engine_track(line, x, nturns)).max(axis=1)


@pytest.mark.gpu
def test_jacobian_vs_double_differences(fodo, ref_orbit):
    """d r_final / d r0 after one turn on 512 of 65,536 particles (sigma 1e-6
    around the closed orbit) against double-precision central differences
    with h = 1e-7 and fourth-order ones with h = 1e-6."""
    r0 = _fodo_bunch(65536, seed=7, orbit=ref_orbit)
    tr = diff.TangentTracker(fodo)
    try:
        _, jac, _, lost = tr.track(_dev_rows(r0), None, 1)
        assert not bool(lost.any())
        jac = jac.cpu().numpy()
    finally:
        tr.close()
    sub = np.arange(0, 65536, 128)
    x = r0[:, sub]
    got = np.transpose(jac[sub], (1, 2, 0))       # (i, j, particle)
    rm = _rmag(fodo, x, 1)
    _assert_fd(got, _coord_fd(fodo, x, 1, 1e-7), rm, 1e-7, "central h=1e-7", 0)
    _assert_fd(got, _coord_fd(fodo, x, 1, 1e-6, order4=True), rm, 1e-6,
               "fourth order h=1e-6", 0)


@pytest.fixture(scope="module")
def fdq():
    """Binary128 finite differences of the oracle (golden/make_golden_diff.py)."""
    import os
    from conftest import GOLDEN
    return dict(np.load(os.path.join(GOLDEN, "diff_fd.npz")))


def _assert_rel(got, ref, what, rel=1e-7, extra=None):
    """Per block (all axes but the last, the particle axis): max |got - ref|
    <= rel * max |ref| (+1e-15 of the whole array's scale, for blocks that
    vanish, + ``extra`` per block: a difference's own measured error);
    returns the largest block-relative error."""
    d = np.abs(got - ref).max(axis=-1)
    s = np.abs(ref).max(axis=-1)
    bound = rel * s + 1e-15 * np.abs(ref).max()
    if extra is not None:
        bound = bound + extra
    bad = d > bound
    if bad.any():
        k = np.unravel_index(np.argmax(d / np.maximum(bound, 1e-300)), d.shape)
        raise AssertionError("%s: %d blocks off; worst %s: |diff| %.3e, scale %.3e"
                             % (what, int(bad.sum()), k, d[k], s[k]))
    return float((d / np.maximum(s, 1e-300)).max())


@pytest.mark.gpu
@pytest.mark.parametrize("case,ring,nturns", [("fodo1", "fodo", 1), ("fodo100", "fodo", 100),
                                              ("large1", "large", 1)])
def test_jacobian_vs_quad_differences(fdq, case, ring, nturns):
    """d r_final / d r0 against differences taken in binary128: five-point
    (h = 1e-8) to 1e-7 of every (i, j) block; central (h = 1e-7) to 1e-7
    plus that difference's own truncation error, measured as its distance
    from the five-point one (up to ~1e-6 of the (ct, px) block after 100
    turns, where the path length is strongly nonlinear in px)."""
    line = rings.fodo_ring() if ring == "fodo" else rings.large_ring(seed=1)
    x = fdq[case + "_x"]
    tr = diff.TangentTracker(line)
    try:
        _, jac, _, lost = tr.track(_dev_rows(x), None, nturns)
        assert not bool(lost.any())
        got = np.transpose(jac.cpu().numpy(), (1, 2, 0))
    finally:
        tr.close()
    c = np.transpose(fdq[case + "_jac"], (1, 2, 0))
    c4 = np.transpose(fdq[case + "_jac4"], (1, 2, 0))
    e4 = _assert_rel(got, c4, case + " five-point h=1e-8")
    e2 = _assert_rel(got, c, case + " central h=1e-7", extra=np.abs(c - c4).max(axis=-1))
    print("jacobian %s: max block-relative error vs five-point %.2e, vs central %.2e"
          % (case, e4, e2))


@pytest.mark.gpu
@pytest.mark.parametrize("case,nturns", [("fodo1", 1), ("fodo100", 100)])
def test_strength_gradients_vs_quad_differences(fodo, fdq, case, nturns):
    """d r_final / d K for quadrupole and sextupole strengths (all 128 for
    one turn, every eighth for 100) against central (h = 1e-7) and
    five-point (h = 1e-5) differences in binary128: 1e-7 of every
    (strength, coordinate) block."""
    params = diff.multipole_strengths(fodo)
    sel = fdq["fodo100_params"] if case == "fodo100" else np.arange(128)
    x = fdq[case + "_x"]
    tr = diff.TangentTracker(fodo, params)
    try:
        _, _, grad, lost = tr.track(_dev_rows(x), None, nturns)
        assert not bool(lost.any())
        grad = grad.cpu().numpy()[sel]
    finally:
        tr.close()
    for key in ("_grad", "_grad4"):
        e = _assert_rel(grad, fdq[case + key], case + key)
        print("strengths %s%s: max block-relative error %.2e" % (case, key, e))


@pytest.mark.gpu
def test_radiating_strength_gradients_vs_quad_differences(fdq):
    """With radiation the map is not symplectic; the general 6x6 solve still
    gives exact strength derivatives: the radiating, misaligned large ring,
    10 turns, against binary128 differences."""
    line = rings.large_ring(seed=1)
    params = [diff.Strength(int(i), int(o)) for i, o in zip(fdq["large10_idx"],
                                                           fdq["large10_order"])]
    assert {p.order for p in params} == {1, 2}
    tr = diff.TangentTracker(line, params)
    try:
        _, jac, grad, lost = tr.track(_dev_rows(fdq["large10_x"]), None, 10)
        assert not bool(lost.any())
        jac, grad = jac.cpu().numpy(), grad.cpu().numpy()
    finally:
        tr.close()
    assert abs(np.linalg.det(jac[0]) - 1.0) > 1e-5       # damping: not symplectic
    for key in ("_grad", "_grad4"):
        e = _assert_rel(grad, fdq["large10" + key], "large10" + key)
        print("strengths large10%s: max block-relative error %.2e" % (key, e))


@pytest.mark.gpu
@pytest.mark.parametrize("nturns", [1, 100])
def test_full_batch_properties(fodo, ref_orbit, nturns):
    """The workload at its full size: 65,536 particles (sigma 1e-6 around
    the orbit) with all 128 strengths.  Every particle's Jacobian is
    symplectic (the map is); a sub-batch tracked alone gives bit-identical
    values and derivatives (particles are independent); and double-precision
    central differences (h = 1e-7) agree within their own rounding floor."""
    params = diff.multipole_strengths(fodo)
    r0 = _fodo_bunch(65536, seed=11, orbit=ref_orbit)
    tr = diff.TangentTracker(fodo, params)
    try:
        r, jac, grad, lost = tr.track(_dev_rows(r0), None, nturns)
        assert not bool(lost.any())
        sub = np.arange(0, 65536, 256)
        r2, jac2, grad2, _ = tr.track(_dev_rows(r0[:, sub]), None, nturns)
        r, jac, grad = r.cpu().numpy(), jac.cpu().numpy(), grad.cpu().numpy()
        assert np.array_equal(r2.cpu().numpy(), r[sub])
        assert np.array_equal(jac2.cpu().numpy(), jac[sub])
        assert np.array_equal(grad2.cpu().numpy(), grad[:, :, sub])
    finally:
        tr.close()
    assert np.all(np.isfinite(grad)) and np.all(np.isfinite(jac))
    symp = np.abs(np.einsum("nki,kl,nlj->nij", jac, S6, jac) - S6).max()
    assert symp < 1e-11, symp
    x = r0[:, sub]
    _assert_fd(grad[:, :, sub], _fd_strengths(fodo, params, x, nturns, 1e-7),
               _rmag(fodo, x, nturns), 1e-7, "double central h=1e-7", 1, rel=1e-7, ulps=4096)


@pytest.mark.gpu
def test_strengths_override_the_table(fodo, ref_orbit):
    """The strengths tensor replaces the compiled values: tracking with
    K + dK equals tracking a lattice compiled with K + dK."""
    params = diff.multipole_strengths(fodo)
    r0 = _fodo_bunch(1024, seed=3, orbit=ref_orbit) * 50
    tr = diff.TangentTracker(fodo, params)
    try:
        k = tr.k0.clone()
        k[5] += 0.01
        k[70] -= 0.5
        r, _, _, _ = tr.track(_dev_rows(r0), k, 5)
        got = r.cpu().numpy().T
    finally:
        tr.close()
    lat = _perturbed(_perturbed(fodo, params[5].index, 1, 0.01), params[70].index, 2, -0.5)
    want = _engine_track(lat, np.asfortranarray(r0), 5)
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_autograd_function(fodo, ref_orbit):
    """TrackFunction: backward gives J^T g and sum_n G^T g, and passes
    torch.autograd.gradcheck on a small case."""
    params = diff.multipole_strengths(fodo)
    tr = diff.TangentTracker(fodo, params)
    try:
        r0 = _dev_rows(_fodo_bunch(512, seed=5, orbit=ref_orbit)).requires_grad_(True)
        k = tr.k0.clone().requires_grad_(True)
        out = diff.track(tr, r0, k, nturns=10)
        w = torch.randn_like(out)
        (out * w).sum().backward()
        _, jac, grad, _ = tr.track(r0.detach(), k.detach(), 10)
        torch.testing.assert_close(r0.grad, torch.einsum("ni,nij->nj", w, jac), rtol=1e-13,
                                   atol=0)
        torch.testing.assert_close(k.grad, torch.einsum("ni,pin->p", w, grad), rtol=1e-13,
                                   atol=1e-30)

        small = diff.TangentTracker(fodo, params[:2] + params[64:66])
        x0 = rings.gaussian(3, [1e-4, 1e-5, 1e-4, 1e-5, 1e-4, 1e-4], seed=6, centre=ref_orbit)
        x = _dev_rows(x0).requires_grad_(True)
        kk = small.k0.clone().requires_grad_(True)
        assert torch.autograd.gradcheck(lambda a, b: diff.track(small, a, b, nturns=3), (x, kk),
                                        eps=1e-7, atol=1e-8, rtol=1e-5)
        small.close()
    finally:
        tr.close()


@pytest.mark.gpu
def test_engine_validates_strengths(fodo):
    """The C entry point checks the strength list itself."""
    from at_b200._lib import EngineError
    tr = diff.TangentTracker(fodo)
    try:
        r = torch.zeros((4, 6), dtype=torch.float64, device="cuda:0")
        jac = torch.empty((4, 6, 6), dtype=torch.float64, device="cuda:0")
        g = torch.empty((1, 6, 4), dtype=torch.float64, device="cuda:0")
        k = torch.ones(1, dtype=torch.float64, device="cuda:0")
        for pe, po in (([1], [1]), ([0], [2]), ([0], [0]), ([99999], [1])):
            with pytest.raises(EngineError):
                tr.eng.tangent_device(tr.lid, r.data_ptr(), 4, 1, 0, np.array(pe), np.array(po),
                                      k.data_ptr(), jac.data_ptr(), g.data_ptr())
    finally:
        tr.close()
