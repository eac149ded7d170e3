"""atb_track_noalloc, the tracking entry point that allocates no memory.

It exists for callers that must not call cudaMalloc on their call path (a
real-time feedback loop, where an allocation would synchronise the device;
an application whose device memory belongs to another allocator).  Here it
is called through the C ABI on device buffers that the test owns, twice in a
row, and each result must be identical to the handle-based
``atb_track_device`` run on the same inputs (same kernel and arithmetic, so
the tolerance is exact equality, as for the engine's other same-kernel
comparisons).  The file is collected last so a failure here cannot hide
another test's; it passes alone in a fresh process and after the others.
"""
import ctypes as C

import numpy as np
import pytest

from at_b200 import _lib, rings
from at_b200.engine import Engine
from at_b200.lattice import compile_lattice

pytestmark = pytest.mark.gpu


def _dev_lattice(torch, cl, dev):
    words = torch.from_numpy(np.ascontiguousarray(cl.words)).to(dev)
    off = torch.from_numpy(np.ascontiguousarray(cl.offsets).view(np.int32)).to(dev)
    return words, off


def _noalloc(torch, cl, words, off, rd, nturns, turn0, lp, mode):
    off_host = np.ascontiguousarray(cl.offsets, dtype=np.uint32)
    L = _lib.lib()
    rc = L.atb_track_noalloc(0, words.data_ptr(), int(cl.words.size), off_host.ctypes.data,
                             off.data_ptr(), int(cl.nelem), rd.data_ptr(), rd.shape[0], nturns,
                             turn0, 1, lp[0].data_ptr(), lp[1].data_ptr(), lp[2].data_ptr(),
                             lp[3].data_ptr(), mode, None)
    _lib.check(rc)


def _losses(torch, n, dev):
    return (torch.zeros(n, dtype=torch.uint8, device=dev),
            torch.zeros(n, dtype=torch.int32, device=dev),
            torch.zeros(n, dtype=torch.int32, device=dev),
            torch.zeros((n, 6), dtype=torch.float64, device=dev))


@pytest.mark.parametrize("ring_name,n,mode", [("fodo", 3000, _lib.MODE_FAST),
                                              ("large", 1500, _lib.MODE_EXACT)])
def test_noalloc_matches_handle_entry_point_twice(ring_name, n, mode):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    if ring_name == "fodo":
        ring = rings.fodo_ring()
        r0 = np.asfortranarray(rings.gaussian(n, seed=11) * 4.0)     # some losses
    else:
        ring = rings.large_ring()                                    # segmented table
        r0 = rings.large_ring_bunch(n, seed=11)
    cl = compile_lattice(ring, ring.energy, ring.particle.rest_energy)
    words, off = _dev_lattice(torch, cl, dev)

    # reference: the existing device entry point on the same inputs
    eng = Engine.get(0)
    lid = eng.upload(cl)
    ra = torch.from_numpy(np.ascontiguousarray(r0.T)).to(dev)
    la = _losses(torch, n, dev)
    rb = ra.clone()
    lb = _losses(torch, n, dev)
    s = torch.cuda.Stream(dev)
    try:
        calls = ((60, 0), (40, 60)) if ring_name == "fodo" else ((7, 0), (5, 7))
        for call, (nturns, turn0) in enumerate(calls):                 # two calls in a row
            with torch.cuda.stream(s):
                eng.track_device(lid, ra.data_ptr(), n, nturns, turn0,
                                 losses=tuple(t.data_ptr() for t in la), mode=mode,
                                 stream=s.cuda_stream)
            eng.sync(s.cuda_stream)
            torch.cuda.synchronize()
            _noalloc(torch, cl, words, off, rb, nturns, turn0, lb, mode)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(rb.cpu().numpy(), ra.cpu().numpy(),
                                          err_msg="call %d" % call)
            for x, y in zip(lb, la):
                np.testing.assert_array_equal(x.cpu().numpy(), y.cpu().numpy())
    finally:
        eng.free(lid)
    if ring_name == "fodo":
        assert la[0].sum().item() > 0            # the loss path was exercised


def test_noalloc_rejects_oversize_requests():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    ring = rings.fodo_ring()
    cl = compile_lattice(ring, ring.energy, ring.particle.rest_energy)
    words, off = _dev_lattice(torch, cl, dev)
    rd = torch.zeros((8, 6), dtype=torch.float64, device=dev)
    off_host = np.ascontiguousarray(cl.offsets, dtype=np.uint32)
    L = _lib.lib()
    too_many = 32768 * 256 + 1                   # ATB_NOALLOC_MAX_PARTICLES + 1
    rc = L.atb_track_noalloc(0, words.data_ptr(), int(cl.words.size), off_host.ctypes.data,
                             off.data_ptr(), int(cl.nelem), rd.data_ptr(), too_many, 1, 0, 0,
                             None, None, None, None, _lib.MODE_FAST, None)
    assert rc == _lib.ATB_ERR_ARG
    assert b"exceed the maximum" in L.atb_last_error()


def test_noalloc_rejects_misaligned_buffers_before_device_work():
    """A caller's own sub-allocator may hand out buffers that are only
    8-byte aligned; the entry point refuses them (the kernels move particles
    in 16-byte vectors) instead of launching."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    ring = rings.fodo_ring()
    cl = compile_lattice(ring, ring.energy, ring.particle.rest_energy)
    words, off = _dev_lattice(torch, cl, dev)
    buf = torch.zeros(6 * 9, dtype=torch.float64, device=dev)
    off_host = np.ascontiguousarray(cl.offsets, dtype=np.uint32)
    L = _lib.lib()
    rc = L.atb_track_noalloc(0, words.data_ptr(), int(cl.words.size), off_host.ctypes.data,
                             off.data_ptr(), int(cl.nelem), buf.data_ptr() + 8, 8, 1, 0, 0,
                             None, None, None, None, _lib.MODE_EXACT, None)
    assert rc == _lib.ATB_ERR_ARG
    assert b"16-byte aligned" in L.atb_last_error()
    assert not buf.any()


def test_handle_path_after_noalloc_keeps_its_shared_memory_limit():
    """The no-alloc set-up must not lower the kernels' shared-memory limit
    that a handle relies on: after a no-alloc call, a handle keeps a 136 KB
    table resident in shared memory (more than the no-alloc path itself
    uses) and tracks it exactly as through the segmented pipeline."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    ring = rings.fodo_ring()
    cl = compile_lattice(ring, ring.energy, ring.particle.rest_energy)
    words, off = _dev_lattice(torch, cl, dev)
    rd = torch.from_numpy(np.ascontiguousarray(rings.gaussian(512, seed=5).T)).to(dev)
    _noalloc(torch, cl, words, off, rd, 2, 0, _losses(torch, 512, dev), _lib.MODE_EXACT)
    torch.cuda.synchronize()

    big = type(ring)(list(ring) * 4, energy=ring.energy, particle=ring.particle)
    cbig = compile_lattice(big, big.energy, big.particle.rest_energy)
    assert 14336 < cbig.words.size <= 20000
    eng = Engine.get(0)
    lid = eng.upload(cbig)
    r0 = rings.gaussian(2048, seed=6)
    try:
        ra = r0.copy(order="F")
        eng.track(lid, ra, 3, mode="exact")                   # segmented (default limits)
        eng.set_launch(resident_max_words=20000)
        rb = r0.copy(order="F")
        eng.track(lid, rb, 3, mode="exact")                   # resident 136 KB table
    finally:
        eng.set_launch(resident_max_words=14336)
        eng.free(lid)
    assert not np.array_equal(ra, r0, equal_nan=True)         # tracked
    np.testing.assert_array_equal(rb, ra)
