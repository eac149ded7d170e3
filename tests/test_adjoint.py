"""Reverse-mode derivatives (the adjoint kernels and their autograd bridge).

The adjoint's products are checked against the tangent kernel's Jacobians,
which test_diff.py pins to the reference's find_m66 and to finite
differences: for a cotangent g, dL/d r0 = J^T g per particle and
dL/dK_q = sum_n G_q[n] . g[n].  Both are exact derivatives of the same
arithmetic, accumulated in a different order, so they agree to rounding:
relative 1e-10 of each array's scale on the FODO ring (hand-written element
adjoints), on the reference's hmba lattice (quadrupole fringes: the
dual-number element path) and on the radiating large ring.  They are also
checked directly against differences taken in binary128 (1e-7 of the sum of
the terms' magnitudes).  The forward pass's values equal the exact tracking
engine's bit for bit, and the gradients do not depend on the checkpoint
stride.
"""
import json
import os

import numpy as np
import pytest

import cases
from at_b200 import diff, elements as E, rings
from conftest import GOLDEN

torch = pytest.importorskip("torch")

REL = 1e-10


def _rows(r_fortran):
    return torch.tensor(np.ascontiguousarray(np.asarray(r_fortran).T), dtype=torch.float64,
                        device="cuda:0")


def _hmba_off():
    with open(os.path.join(GOLDEN, "hmba.json")) as f:
        data = json.load(f)["off"]
    line = [cases.make_element(d, E.Element) for d in data["specs"]]
    return E.Lattice(line, energy=data["energy"], particle="relativistic", periodicity=32)


def _scale_rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _tangent_vjp(line, params, r0, k, nturns, g):
    tt = diff.TangentTracker(line, params)
    try:
        r, jac, grad, lost = tt.track(r0, k, nturns)
        gr0 = torch.einsum("ni,nij->nj", g, jac)
        gk = torch.einsum("ni,pin->p", torch.where(lost[:, None], 0.0, g),
                          torch.nan_to_num(grad, nan=0.0))
        return r, gr0, gk, lost
    finally:
        tt.close()


def _adjoint(line, params, r0, k, nturns, g, stride=None):
    at = diff.AdjointTracker(line, params)
    try:
        r, lost, st = at.forward(r0, k, nturns, stride=stride)
        gr0, gk = at.backward(st, g)
        return r, gr0, gk, lost
    finally:
        at.close()


def _check_against_tangent(line, params, x0, nturns, seed=0, rel=REL):
    r0 = _rows(x0)
    k = torch.tensor([float(np.ravel(line[p.index].PolynomB)[p.order]) for p in params],
                     dtype=torch.float64, device="cuda:0")
    g = torch.randn((r0.shape[0], 6), dtype=torch.float64, device="cuda:0",
                    generator=torch.Generator("cuda:0").manual_seed(seed))
    rt, gt, kt, lt = _tangent_vjp(line, params, r0, k, nturns, g)
    ra, ga, ka, la = _adjoint(line, params, r0, k, nturns, g)
    assert torch.equal(la, lt)
    ok = ~la
    assert torch.equal(ra[ok], rt[ok])                     # the same tracked values
    assert torch.isnan(ga[la]).all()
    assert _scale_rel(ga[ok].cpu(), gt[ok].cpu()) <= rel
    if params:
        assert _scale_rel(ka.cpu(), kt.cpu()) <= rel
    return ra, la


@pytest.mark.gpu
@pytest.mark.parametrize("nturns", [1, 20])
def test_fodo_adjoint_equals_tangent_products(nturns):
    ring = rings.fodo_ring()
    params = diff.multipole_strengths(ring)
    orbit = np.load(os.path.join(GOLDEN, "fodo_m66.npz"))["orbit"]
    x0 = rings.gaussian(2048, [1e-4, 1e-5, 1e-4, 1e-5, 1e-4, 1e-4], seed=1, centre=orbit)
    _check_against_tangent(ring, params, x0, nturns)


@pytest.mark.gpu
def test_adjoint_forward_values_equal_exact_engine():
    from at_b200 import tracking
    ring = rings.fodo_ring()
    params = diff.multipole_strengths(ring)
    x0 = rings.gaussian(3000, seed=2) * 6.0               # 66 of them are lost
    out = np.asfortranarray(x0.copy())
    _, ld = tracking.gpupass(ring, out, 30, losses=True, mode="exact")
    at = diff.AdjointTracker(ring, params)
    try:
        r, lost, _ = at.forward(_rows(x0), None, 30)
    finally:
        at.close()
    assert ld["islost"].any()
    np.testing.assert_array_equal(lost.cpu().numpy(), ld["islost"])
    np.testing.assert_array_equal(r.cpu().numpy().T, out)


@pytest.mark.gpu
def test_lost_particles_get_nan_and_add_nothing():
    ring = rings.fodo_ring()
    params = diff.multipole_strengths(ring)
    x0 = rings.gaussian(3000, seed=2) * 6.0
    # large amplitudes: near the chaotic edge the two accumulation orders part
    # by more than at small amplitude
    ra, la = _check_against_tangent(ring, params, x0, 30, seed=4, rel=1e-8)
    assert la.any() and not la.all()


@pytest.mark.gpu
def test_stride_does_not_change_the_gradients():
    """Checkpoints every turn or every 4th turn (blocks tracked again from
    their checkpoint): the same kernels on the same states, bit for bit."""
    ring = rings.fodo_ring()
    params = diff.multipole_strengths(ring)
    x0 = rings.gaussian(1024, [1e-4, 1e-5, 1e-4, 1e-5, 1e-4, 1e-4], seed=3)
    r0 = _rows(x0)
    g = torch.randn((1024, 6), dtype=torch.float64, device="cuda:0",
                    generator=torch.Generator("cuda:0").manual_seed(1))
    k = None
    out = [_adjoint(ring, params, r0, k, 11, g, stride=s) for s in (1, 4, 11)]
    for r, gr0, gk, _ in out[1:]:
        assert torch.equal(r, out[0][0])
        assert torch.equal(gr0, out[0][1])
        assert _scale_rel(gk.cpu(), out[0][2].cpu()) <= 1e-13   # sums in atomic order


@pytest.mark.gpu
def test_hmba_quadrupole_fringes_through_the_dual_path():
    ring = _hmba_off()
    params = diff.multipole_strengths(ring)
    assert params
    x0 = rings.gaussian(512, [1e-4, 1e-5, 1e-4, 1e-5, 1e-4, 1e-4], seed=5)
    _check_against_tangent(ring, params, x0, 3)


@pytest.mark.gpu
def test_radiating_large_ring_through_the_dual_path():
    ring = rings.large_ring()
    params = diff.multipole_strengths(ring)[::40]
    x0 = rings.large_ring_bunch(128, seed=6)
    _check_against_tangent(ring, params, x0, 1)


@pytest.mark.gpu
def test_autograd_through_the_adjoint():
    """diff.track with an AdjointTracker: backward equals the tangent
    tracker's backward, and passes gradcheck on a small case."""
    ring = rings.fodo_ring()
    params = diff.multipole_strengths(ring)
    orbit = np.load(os.path.join(GOLDEN, "fodo_m66.npz"))["orbit"]
    x0 = rings.gaussian(512, [1e-4, 1e-5, 1e-4, 1e-5, 1e-4, 1e-4], seed=7, centre=orbit)
    grads = []
    for cls in (diff.TangentTracker, diff.AdjointTracker):
        tr = cls(ring, params)
        try:
            r0 = _rows(x0).requires_grad_(True)
            k = tr.k0.clone().requires_grad_(True)
            out = diff.track(tr, r0, k, nturns=10)
            (out ** 2).sum().backward()
            grads.append((out.detach(), r0.grad, k.grad))
        finally:
            tr.close()
    (ot, gt, kt), (oa, ga, ka) = grads
    assert torch.equal(ot, oa)
    assert _scale_rel(ga.cpu(), gt.cpu()) <= REL
    assert _scale_rel(ka.cpu(), kt.cpu()) <= REL
    small = diff.AdjointTracker(ring, params[:2] + params[64:66])
    try:
        xs = rings.gaussian(3, [1e-4, 1e-5, 1e-4, 1e-5, 1e-4, 1e-4], seed=6, centre=orbit)
        x = _rows(xs).requires_grad_(True)
        kk = small.k0.clone().requires_grad_(True)
        assert torch.autograd.gradcheck(lambda a, b: diff.track(small, a, b, nturns=3), (x, kk),
                                        eps=1e-7, atol=1e-8, rtol=1e-5)
    finally:
        small.close()


@pytest.mark.gpu
def test_adjoint_validates_strengths():
    from at_b200._lib import EngineError
    ring = rings.fodo_ring()
    at = diff.AdjointTracker(ring)
    try:
        r = torch.zeros((4, 6), dtype=torch.float64, device="cuda:0")
        ck = torch.empty((1, 4, 6), dtype=torch.float64, device="cuda:0")
        k = torch.ones(1, dtype=torch.float64, device="cuda:0")
        for pe, po in (([1], [1]), ([0], [2]), ([0], [0]), ([99999], [1])):
            with pytest.raises(EngineError):
                at.eng.adjoint_forward(at.lid, r.data_ptr(), 4, 1, 0, np.array(pe), np.array(po),
                                       k.data_ptr(), ck.data_ptr(), 1)
        with pytest.raises(EngineError):
            at.eng.adjoint_forward(at.lid, r.data_ptr(), 4, 1, 0, np.array([]), np.array([]),
                                   None, ck.data_ptr(), 0)
    finally:
        at.close()


@pytest.mark.gpu
def test_empty_set_and_zero_turns():
    """No particles: empty results and a zero strength gradient.  Zero turns:
    the final coordinates are the initial ones and the backward pass is the
    identity (dL/d r0 = g, dL/dK = 0)."""
    ring = rings.fodo_ring()
    params = diff.multipole_strengths(ring)
    at = diff.AdjointTracker(ring, params)
    try:
        e = torch.zeros((0, 6), dtype=torch.float64, device="cuda:0")
        r, lost, st = at.forward(e, None, 5)
        gx, gk = at.backward(st, e)
        assert r.shape == (0, 6) and lost.shape == (0,) and gx.shape == (0, 6)
        assert torch.equal(gk, torch.zeros_like(gk))
        x0 = _rows(rings.gaussian(300, [1e-4, 1e-5, 1e-4, 1e-5, 1e-4, 1e-4], seed=8))
        g = torch.randn_like(x0)
        r, lost, st = at.forward(x0, None, 0)
        gx, gk = at.backward(st, g)
        assert torch.equal(r, x0) and not lost.any()
        assert torch.equal(gx, g) and torch.equal(gk, torch.zeros_like(gk))
    finally:
        at.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case,nturns", [("fodo1", 1), ("fodo100", 100)])
def test_adjoint_vs_quad_differences(case, nturns):
    """The adjoint's gradients of L = sum_n g_n . r_n(T) against the same
    contractions of differences taken in binary128 (golden diff_fd.npz:
    five-point, h = 1e-8 for coordinates and 1e-5 for strengths): each within
    1e-7 of the sum of the magnitudes of its terms."""
    fdq = dict(np.load(os.path.join(GOLDEN, "diff_fd.npz")))
    ring = rings.fodo_ring()
    params = diff.multipole_strengths(ring)
    sel = fdq["fodo100_params"] if case == "fodo100" else np.arange(128)
    x = fdq[case + "_x"]
    n = x.shape[1]
    g = np.random.default_rng(3).standard_normal((n, 6))
    at = diff.AdjointTracker(ring, params)
    try:
        r, lost, st = at.forward(_rows(x), None, nturns)
        assert not bool(lost.any())
        gx, gk = at.backward(st, torch.tensor(g, device="cuda:0"))
        gx, gk = gx.cpu().numpy(), gk.cpu().numpy()[sel]
    finally:
        at.close()
    jac4 = fdq[case + "_jac4"]                               # (n, 6, 6)
    grad4 = fdq[case + "_grad4"]                             # (P_sel, 6, n)
    want_x = np.einsum("ni,nij->nj", g, jac4)
    scale_x = np.einsum("ni,nij->nj", np.abs(g), np.abs(jac4))
    assert np.all(np.abs(gx - want_x) <= 1e-7 * scale_x + 1e-300)
    want_k = np.einsum("ni,pin->p", g, grad4)
    scale_k = np.einsum("ni,pin->p", np.abs(g), np.abs(grad4))
    assert np.all(np.abs(gk - want_k) <= 1e-7 * scale_k)


@pytest.mark.gpu
def test_stored_element_states_give_the_same_gradients():
    """The forward pass storing every element's entry state (no tracking in
    the backward sweep) gives the gradients of the re-tracking sweep bit for
    bit (strength sums up to atomic order), lost particles included."""
    ring = rings.fodo_ring()
    params = diff.multipole_strengths(ring)
    x0 = _rows(rings.gaussian(3000, seed=2) * 6.0)         # some are lost on the way
    g = torch.randn((3000, 6), dtype=torch.float64, device="cuda:0",
                    generator=torch.Generator("cuda:0").manual_seed(5))
    out = []
    for store in (False, True):
        at = diff.AdjointTracker(ring, params)
        try:
            r, lost, st = at.forward(x0, None, 30, store_elements=store)
            gx, gk = at.backward(st, g)
            out.append((r, lost, gx, gk))
        finally:
            at.close()
    (r1, l1, gx1, gk1), (r2, l2, gx2, gk2) = out
    assert l1.any() and torch.equal(l1, l2)
    assert torch.equal(torch.nan_to_num(r1, nan=7.0), torch.nan_to_num(r2, nan=7.0))
    assert torch.equal(torch.nan_to_num(gx1, nan=7.0), torch.nan_to_num(gx2, nan=7.0))
    assert _scale_rel(gk2.cpu(), gk1.cpu()) <= 1e-13
