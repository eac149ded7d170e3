"""Exact derivatives of multi-turn tracking and their ``torch.autograd`` bridge.

The tangent kernel (``atb_tangent_device`` in ``include/atb200.h``) tracks a
particle set in forward-mode automatic differentiation: every pass method runs
on dual numbers, so the derivatives are those of the integrators themselves,
not finite differences.  It returns, per particle,

* ``jac`` (N, 6, 6): d r_final / d r_initial (at the closed orbit this is the
  one-turn matrix the reference estimates by central differences in
  ``find_m66``, pyat/at/physics/matrix.py:105-165), and
* ``grad`` (P, 6, N): d r_final / d K_q for P multipole strengths
  K_q = PolynomB[order_q] of chosen elements (quadrupole and sextupole
  strengths, typically).

The adjoint kernels (``atb_adjoint_forward`` / ``atb_adjoint_backward``) give
the reverse mode: a forward pass that stores the state entering every
``stride``-th turn, and one backward sweep that maps dL/d r_final to
dL/d r_initial and dL/dK for any scalar L, at a cost that does not grow with
the number of strengths (:class:`AdjointTracker`; with ``store_elements`` the
forward pass also keeps every element's entry state, so the backward sweep
does not track the turns again, at N x elements x turns x 48 bytes).

``track`` wraps one call as a ``torch.autograd.Function``: the forward pass
returns the final coordinates; the backward pass is either the contraction of
the tangent kernel's saved Jacobians with the incoming gradient
(:class:`TangentTracker`) or the adjoint kernels' backward sweep
(:class:`AdjointTracker`), for both the initial coordinates and the
strengths.  The strengths are read by the kernels from a device tensor, so
they can be optimised directly.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .engine import Engine
from .lattice import compile_lattice
from .tracking import _energy_particle

#: PassMethods whose PolynomB strengths can be differentiated
DIFF_PASS_METHODS = (
    "StrMPoleSymplectic4Pass", "StrMPoleSymplectic4RadPass", "BndMPoleSymplectic4Pass",
    "BndMPoleSymplectic4RadPass", "ThinMPolePass",
)


@dataclass(frozen=True)
class Strength:
    """One differentiated strength: PolynomB[order] of element ``index``."""
    index: int
    order: int


def _principal_order(el) -> int:
    """Highest order with a non-zero PolynomB coefficient (-1 if none)."""
    pb = np.asarray(getattr(el, "PolynomB", ()), dtype=np.float64).ravel()
    nz = np.flatnonzero(pb)
    return int(nz[-1]) if nz.size else -1


def multipole_strengths(line, orders=(1, 2), pass_methods=("StrMPoleSymplectic4Pass",
                                                           "StrMPoleSymplectic4RadPass")):
    """The strengths of the quadrupoles (order 1) and sextupoles (order 2) of
    ``line``: every element with one of ``pass_methods`` whose highest
    non-zero PolynomB order is in ``orders``, grouped by order, in lattice
    order within a group.  On the 32-cell FODO ring this gives the 64
    quadrupole and 64 sextupole strengths."""
    out = []
    for order in orders:
        for i, el in enumerate(line):
            if getattr(el, "PassMethod", None) in pass_methods and _principal_order(el) == order:
                out.append(Strength(i, order))
    return out


class TangentTracker:
    """One lattice on one device, set up for tangent tracking with respect to
    the initial coordinates and the strengths ``params`` (a list of
    :class:`Strength` or ``(index, order)`` pairs)."""

    def __init__(self, line, params=(), energy=None, particle=None, device: int = 0):
        import torch

        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.params = [p if isinstance(p, Strength) else Strength(int(p[0]), int(p[1]))
                       for p in params]
        e, rest, charge = _energy_particle(line, energy, particle)
        seen = set()
        k0 = []
        for p in self.params:
            if not 0 <= p.index < len(line):
                raise ValueError("strength element %d outside the lattice" % p.index)
            if p.index in seen:
                raise ValueError("element %d carries two strengths" % p.index)
            seen.add(p.index)
            el = line[p.index]
            if getattr(el, "PassMethod", None) not in DIFF_PASS_METHODS:
                raise ValueError("element %d (%s) has no differentiable PolynomB" %
                                 (p.index, getattr(el, "PassMethod", None)))
            pb = np.asarray(el.PolynomB, dtype=np.float64).ravel()
            mo = int(getattr(el, "MaxOrder", pb.size - 1))
            if not 1 <= p.order <= mo:
                raise ValueError("PolynomB order %d outside [1, MaxOrder=%d] of element %d" %
                                 (p.order, mo, p.index))
            if p.order == 1 and pb[1] == 0.0 and (getattr(el, "FringeQuadEntrance", 0) or
                                                  getattr(el, "FringeQuadExit", 0)):
                # the table enables the quadrupole fringe only for b1 != 0
                raise ValueError("element %d: quadrupole fringe with PolynomB[1] == 0" % p.index)
            k0.append(float(pb[p.order]))
        self.cl = compile_lattice(line, e, rest, charge)
        self.eng = Engine.get(device)
        self.lid = self.eng.upload(self.cl)
        self.stream = torch.cuda.Stream(self.dev)
        self.pelem = np.array([p.index for p in self.params], dtype=np.int32)
        self.porder = np.array([p.order for p in self.params], dtype=np.int32)
        #: the strengths of the lattice as compiled (device tensor)
        self.k0 = torch.tensor(k0, dtype=torch.float64, device=self.dev)

    @property
    def nparam(self) -> int:
        return len(self.params)

    def track(self, r0, strengths=None, nturns: int = 1, turn0: int = 0):
        """Tangent tracking of ``r0`` ((N, 6) float64 tensor on this device,
        not modified) with ``strengths`` ((P,) tensor, default: the lattice's
        own).  Returns ``(r, jac, grad, lost)``: final coordinates (N, 6),
        d r / d r0 (N, 6, 6), d r / d K (P, 6, N) and the loss flags (N,)."""
        torch = self.torch
        if r0.dtype != torch.float64 or r0.dim() != 2 or r0.shape[1] != 6:
            raise ValueError("r0 must be an (N, 6) float64 tensor")
        if r0.device != self.dev:
            raise ValueError("r0 must be on %s" % self.dev)
        k = self.k0 if strengths is None else strengths
        if k.dtype != torch.float64 or k.shape != (self.nparam,) or k.device != self.dev:
            raise ValueError("strengths must be a (%d,) float64 tensor on %s" %
                             (self.nparam, self.dev))
        k = k.detach().contiguous()
        n = int(r0.shape[0])
        r = r0.detach().contiguous().clone()
        jac = torch.empty((n, 6, 6), dtype=torch.float64, device=self.dev)
        grad = torch.empty((self.nparam, 6, n), dtype=torch.float64, device=self.dev)
        lost = torch.empty((n,), dtype=torch.uint8, device=self.dev)
        # the kernel runs on the tracker's own stream, ordered after the
        # caller's stream (which may be the legacy default stream) and before
        # anything the caller enqueues next
        cur = torch.cuda.current_stream(self.dev)
        self.stream.wait_stream(cur)
        self.eng.tangent_device(self.lid, r.data_ptr(), n, int(nturns), int(turn0), self.pelem,
                                self.porder, k.data_ptr() if self.nparam else None,
                                jac.data_ptr(), grad.data_ptr() if self.nparam else None,
                                lost.data_ptr(), self.stream.cuda_stream)
        cur.wait_stream(self.stream)
        return r, jac, grad, lost.bool()

    def close(self):
        if getattr(self, "lid", None) is not None:
            self.eng.free(self.lid)
            self.lid = None


class AdjointTracker(TangentTracker):
    """The same lattice and strengths set up for reverse mode: ``forward``
    tracks and keeps checkpoints, ``backward`` runs the adjoint sweep."""

    #: checkpoint memory above which turns are stored every ``stride`` turns
    #: (each block of turns is then tracked again from its checkpoint)
    CKPT_BUDGET = 8 << 30

    def _stride(self, n: int, nturns: int) -> int:
        per_turn = 48 * max(n, 1)
        if nturns * per_turn <= self.CKPT_BUDGET:
            return 1
        s = max(1, int(np.ceil(np.sqrt(nturns))))
        while ((nturns + s - 1) // s + s) * per_turn > self.CKPT_BUDGET and s < nturns:
            s *= 2
        return s

    def forward(self, r0, strengths=None, nturns: int = 1, turn0: int = 0, stride=None,
                store_elements: bool = False):
        """Track ``r0`` ((N, 6) float64 tensor on this device, not modified)
        with ``strengths`` ((P,) tensor, default: the lattice's own).
        Returns ``(r, lost, state)``: final coordinates (N, 6), loss flags
        (N,) and what :meth:`backward` needs.  ``store_elements`` keeps every
        element's entry state of every turn (N x elements x turns x 48 bytes)
        so that the backward sweep need not track the turns again."""
        torch = self.torch
        if r0.dtype != torch.float64 or r0.dim() != 2 or r0.shape[1] != 6:
            raise ValueError("r0 must be an (N, 6) float64 tensor")
        if r0.device != self.dev:
            raise ValueError("r0 must be on %s" % self.dev)
        k = self.k0 if strengths is None else strengths
        if k.dtype != torch.float64 or k.shape != (self.nparam,) or k.device != self.dev:
            raise ValueError("strengths must be a (%d,) float64 tensor on %s" %
                             (self.nparam, self.dev))
        k = k.detach().contiguous().clone()
        n, nturns = int(r0.shape[0]), int(nturns)
        if store_elements:
            stride = 1
        stride = self._stride(n, nturns) if stride is None else int(stride)
        nck = max(1, (nturns + stride - 1) // stride)
        r = r0.detach().contiguous().clone()
        ckpt = torch.empty((nck, n, 6), dtype=torch.float64, device=self.dev)
        lost = torch.empty((n,), dtype=torch.uint8, device=self.dev)
        estates = None
        if store_elements and n and nturns:
            estates = torch.empty((nturns, self.cl.nelem, n, 6), dtype=torch.float64,
                                  device=self.dev)
        cur = torch.cuda.current_stream(self.dev)
        self.stream.wait_stream(cur)
        self.eng.adjoint_forward(self.lid, r.data_ptr(), n, nturns, int(turn0), self.pelem,
                                 self.porder, k.data_ptr() if self.nparam else None,
                                 ckpt.data_ptr(), stride, lost.data_ptr(),
                                 self.stream.cuda_stream,
                                 estates.data_ptr() if estates is not None else None)
        cur.wait_stream(self.stream)
        # the final states, kept apart from the r handed back to the caller
        rfinal = r.clone() if estates is not None else None
        state = {"ckpt": ckpt, "k": k, "n": n, "nturns": nturns, "turn0": int(turn0),
                 "stride": stride, "estates": estates, "rfinal": rfinal}
        return r, lost.bool(), state

    def backward(self, state, g):
        """dL/d r0 (N, 6) and dL/dK (P,) for the cotangent ``g`` = dL/d r_final
        ((N, 6) float64 on this device).  Lost particles get NaN rows and add
        nothing to dL/dK."""
        torch = self.torch
        n = state["n"]
        if g.dtype != torch.float64 or tuple(g.shape) != (n, 6) or g.device != self.dev:
            raise ValueError("g must be an (%d, 6) float64 tensor on %s" % (n, self.dev))
        lam = g.detach().contiguous().clone()
        gk = torch.zeros((self.nparam,), dtype=torch.float64, device=self.dev)
        k = state["k"]
        cur = torch.cuda.current_stream(self.dev)
        self.stream.wait_stream(cur)
        self.eng.adjoint_backward(self.lid, state["ckpt"].data_ptr(), n, state["nturns"],
                                  state["turn0"], state["stride"], self.pelem, self.porder,
                                  k.data_ptr() if self.nparam else None, lam.data_ptr(),
                                  gk.data_ptr() if self.nparam else None,
                                  self.stream.cuda_stream,
                                  state["estates"].data_ptr() if state["estates"] is not None
                                  else None,
                                  state["rfinal"].data_ptr() if state["rfinal"] is not None
                                  else None)
        cur.wait_stream(self.stream)
        return lam, gk


def _track_function():
    import torch

    class TrackFunction(torch.autograd.Function):
        """r_final = track(r0, K).  Forward: the tangent kernel (final
        coordinates plus both Jacobians).  Backward: the adjoint products
        grad_r0[n] = J[n]^T g[n] and grad_K[q] = sum_n G[q, :, n] . g[n]."""

        @staticmethod
        def forward(ctx, r0, strengths, tracker, nturns, turn0):
            r, jac, grad, _ = tracker.track(r0, strengths, nturns, turn0)
            ctx.save_for_backward(jac, grad)
            return r

        @staticmethod
        def backward(ctx, g):
            jac, grad = ctx.saved_tensors
            g_r0 = g_k = None
            if ctx.needs_input_grad[0]:
                g_r0 = torch.einsum("ni,nij->nj", g, jac)
            if ctx.needs_input_grad[1]:
                g_k = torch.einsum("ni,pin->p", g, grad)
            return g_r0, g_k, None, None, None

    class AdjointFunction(torch.autograd.Function):
        """r_final = track(r0, K).  Forward: the adjoint kernels' forward pass
        (final coordinates and turn checkpoints).  Backward: their reverse
        sweep, grad_r0 and grad_K in one pass."""

        @staticmethod
        def forward(ctx, r0, strengths, tracker, nturns, turn0):
            r, _, state = tracker.forward(r0, strengths, nturns, turn0)
            ctx.tracker, ctx.state = tracker, state
            return r

        @staticmethod
        def backward(ctx, g):
            g_r0, g_k = ctx.tracker.backward(ctx.state, g.contiguous())
            return (g_r0 if ctx.needs_input_grad[0] else None,
                    g_k if ctx.needs_input_grad[1] else None, None, None, None)

    return TrackFunction, AdjointFunction


_TF = None


def track(tracker: TangentTracker, r0, strengths=None, nturns: int = 1, turn0: int = 0):
    """Differentiable multi-turn tracking: returns the final (N, 6)
    coordinates as a tensor that back-propagates to ``r0`` and ``strengths``
    (both float64 tensors on the tracker's device; ``strengths`` defaults to
    a copy of the lattice's own, which then receives no gradient).  An
    :class:`AdjointTracker` back-propagates through the adjoint kernels, a
    :class:`TangentTracker` through its saved Jacobians."""
    global _TF
    if _TF is None:
        _TF = _track_function()
    k = tracker.k0.clone() if strengths is None else strengths
    fn = _TF[1] if isinstance(tracker, AdjointTracker) else _TF[0]
    return fn.apply(r0, k, tracker, int(nturns), int(turn0))


def find_m66(line, orbit=None, energy=None, particle=None, device: int = 0):
    """One-turn 6x6 matrix at ``orbit`` (default: the 6-D closed orbit) from
    the exact derivatives of the integrators: the analogue of the reference's
    ``find_m66`` (pyat/at/physics/matrix.py:105-165), which differentiates
    12 tracked particles numerically.  Returns ``(m66, orbit)``."""
    import torch

    from . import physics

    if orbit is None:
        orbit = physics.find_orbit6(line, mode="exact")
    tr = TangentTracker(line, (), energy=energy, particle=particle, device=device)
    try:
        r0 = torch.tensor(np.asarray(orbit, dtype=np.float64).reshape(1, 6), device=tr.dev)
        _, jac, _, lost = tr.track(r0, None, 1)
        if bool(lost[0]):
            raise RuntimeError("find_m66: the orbit particle was lost")
        return jac[0].cpu().numpy(), np.asarray(orbit, dtype=np.float64)
    finally:
        tr.close()

