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

``TrackFunction`` wraps one call as a ``torch.autograd.Function``: the forward
pass returns the final coordinates, the backward pass contracts the saved
Jacobians with the incoming gradient (the adjoint, or vector-Jacobian product)
for both the initial coordinates and the strengths.  The strengths are read
by the kernel from a device tensor, so they can be optimised directly.
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

    return TrackFunction


_TF = None


def track(tracker: TangentTracker, r0, strengths=None, nturns: int = 1, turn0: int = 0):
    """Differentiable multi-turn tracking: returns the final (N, 6)
    coordinates as a tensor that back-propagates to ``r0`` and ``strengths``
    (both float64 tensors on the tracker's device; ``strengths`` defaults to
    a copy of the lattice's own, which then receives no gradient)."""
    global _TF
    if _TF is None:
        _TF = _track_function()
    k = tracker.k0.clone() if strengths is None else strengths
    return _TF.apply(r0, k, tracker, int(nturns), int(turn0))


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

