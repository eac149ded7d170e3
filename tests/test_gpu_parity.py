"""CUDA engine against the oracle and the reference, on the same seeded inputs.

Tolerances (stated per test):
  * exact mode (the default): bit-identical wherever the path has no sin/tan;
    where the RF cavity's sin or a bend's per-particle tan is involved, CUDA's
    libdevice and glibc may differ by an ulp, so a scale-relative 1e-14 is
    allowed per element and 1e-13 after one turn of a ring;
  * fast mode (FMA, reciprocal reuse): scale-relative 1e-13 after one turn of
    the FODO ring, 2e-13 after one turn of the 2,000-element large ring;
  * 1000 turns at the workloads' own sizes (FODO: 10,000 particles; large
    ring: 2048), against the reference's own engine: 1e-9 scale-relative on
    stable particles that survive in both (a survivor beyond 1e-9 must be
    unstable in the reference's own arithmetic: copies of it started one ulp
    apart end more than 1e-9 apart), and the same lost set, loss turns and
    loss elements except for particles whose loss coordinate lies within 1e-9
    (relative) of the amplitude limit or of the loss element's aperture, or
    whose fate is ill-conditioned (changes when its start moves by one ulp
    in any coordinate, or under FMA-contracted arithmetic); the counts are
    reported.
"Scale-relative" divides each coordinate's largest difference by that
coordinate's largest magnitude over the particles (conftest.scale_rel_diff).
"""
import json
import os

import numpy as np
import pytest

import cases
from at_b200 import elements as E
from at_b200 import rings
from at_b200.engine import Engine
from at_b200.lattice import compile_lattice
from oracle import oracle

from conftest import ELECTRON_REST, GOLDEN, scale_rel_diff

pytestmark = pytest.mark.gpu

TRANSCENDENTAL = ("rf_", "bend_fringe", "bend_full", "thin_ba")


def _gpu_track(line, r, nturns, energy, rest, mode, element=False, **kw):
    eng = Engine.get(0)
    cl = compile_lattice(line, energy, rest, t0=0.0 if element else None)
    lid = eng.upload(cl)
    try:
        out = eng.track(lid, r, nturns, kw.pop("turn", 0), kw.pop("start_elem", 0),
                        kw.pop("end_elem", cl.nelem), mode=mode, element=element, **kw)
    finally:
        eng.free(lid)
    return out


@pytest.mark.parametrize("mode", ["exact", "fast"])
@pytest.mark.parametrize("name,spec", cases.element_cases(), ids=[c[0] for c in cases.element_cases()])
def test_element_vs_oracle(name, spec, mode):
    el = cases.make_element(spec, E.Element)
    r0 = cases.element_particles(256, seed=3)
    rad = "Rad" in spec["PassMethod"] or spec["PassMethod"] == "RFCavityPass"
    en, rest = (6e9, ELECTRON_REST) if rad else (0.0, 0.0)
    ro = r0.copy(order="F")
    oracle.track([el], ro, 1, energy=en, rest_energy=rest, element=True, t0=0.0)
    rg = r0.copy(order="F")
    _gpu_track([el], rg, 1, en, rest, mode, element=True)
    np.testing.assert_array_equal(np.isnan(rg), np.isnan(ro))
    if mode == "exact" and not name.startswith(TRANSCENDENTAL):
        np.testing.assert_array_equal(rg, ro)
    else:
        tol = 1e-14 if mode == "exact" else 1e-13
        assert scale_rel_diff(rg, ro) <= tol


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_element_golden_fixture(golden, mode):
    """The engine against the reference's own outputs (tests/golden)."""
    g = golden("elements.npz")
    for name, spec in cases.element_cases():
        el = cases.make_element(spec, E.Element)
        r = g[name + "/in"].copy(order="F")
        rad = "Rad" in spec["PassMethod"] or spec["PassMethod"] == "RFCavityPass"
        _gpu_track([el], r, 1, 6e9 if rad else 0.0, ELECTRON_REST if rad else 0.0, mode,
                   element=True)
        ref = g[name + "/out"]
        np.testing.assert_array_equal(np.isnan(r), np.isnan(ref), err_msg=name)
        assert scale_rel_diff(r, ref) <= (1e-14 if mode == "exact" else 1e-13), name


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_fodo_one_turn(mode):
    ring = rings.fodo_ring()
    r0 = rings.gaussian(4096)
    ro = r0.copy(order="F")
    oracle.track(ring, ro, 1, energy=3e9, rest_energy=ELECTRON_REST)
    rg = r0.copy(order="F")
    _gpu_track(ring, rg, 1, 3e9, ELECTRON_REST, mode)
    assert scale_rel_diff(rg, ro) <= (1e-14 if mode == "exact" else 1e-13)


def _near_boundary(line, ld, tol=1e-9):
    """Per particle: its loss coordinate lies within ``tol`` (relative) of a
    loss boundary -- the amplitude limit |r_n| = 1 (n < 5, pyat/at.c:123) or,
    at an aperture element, one of its rectangular limits (atlalib.c:169-175)."""
    coord = np.asarray(ld["coord"])
    c = np.abs(coord[:5])
    near = np.any(np.abs(c - 1.0) <= tol, axis=0)
    for i in np.flatnonzero(ld["islost"]):
        el = line[int(ld["elem"][i])]
        lim = getattr(el, "Limits", None)
        if lim is None:
            lim = getattr(el, "RApertures", None)
        if lim is not None:
            lim = np.asarray(lim, dtype=float)
            xy = (coord[0, i], coord[0, i], coord[2, i], coord[2, i])
            near[i] |= any(abs(v - l) <= tol * max(abs(l), 1e-300) for v, l in zip(xy, lim))
    return near


def _ill_conditioned(line, r0, idx, nturns, energy, rest):
    """Per particle of ``idx``: is its loss (lost or not, turn, element)
    decided below the rounding level?  The oracle tracks the particle in the
    reference's arithmetic, twelve copies with one coordinate moved by one
    ulp either way, and the particle again in the same source compiled with
    FMA contraction (a rounding-level change of every operation, the kind of
    difference the engine's CUDA sin or fast arithmetic makes).  A particle
    whose loss point these runs do not share sits on a loss boundary in the
    sense of the parity rule, whatever its final distance to a limit."""
    out = []
    for i in idx:
        base = r0[:, i]
        cols = [base]
        for c in range(6):
            for d in (np.inf, -np.inf):
                p = base.copy()
                p[c] = np.nextafter(p[c], d)
                cols.append(p)
        r = np.asfortranarray(np.stack(cols, axis=1))
        _, ld = oracle.track(line, r, nturns, energy=energy, rest_energy=rest, losses=True)
        fates = {(bool(ld["islost"][k]), int(ld["turn"][k]), int(ld["elem"][k]))
                 for k in range(r.shape[1])}
        if oracle.has_fma():
            rf = np.asfortranarray(base.reshape(6, 1).copy())
            _, lf = oracle.track(line, rf, nturns, energy=energy, rest_energy=rest, losses=True,
                                 nthreads=1, arithmetic="fma")
            fates.add((bool(lf["islost"][0]), int(lf["turn"][0]), int(lf["elem"][0])))
        out.append(len(fates) > 1)
    return np.array(out, dtype=bool)


def _unstable(line, r0, idx, nturns, energy, rest, scale, tol):
    """Per particle of ``idx`` (a survivor in both runs): is its final state
    sensitive beyond ``tol`` (of each coordinate's ``scale``) to its start at
    the rounding level?  The oracle tracks it in the reference's arithmetic
    and twelve copies with one coordinate moved by one ulp either way; a
    particle whose copies end more than ``tol`` apart is not a stable particle
    (its orbit is chaotic near the dynamic aperture, where any rounding
    difference grows turn by turn)."""
    out = []
    for i in idx:
        base = r0[:, i]
        cols = [base]
        for c in range(6):
            for d in (np.inf, -np.inf):
                p = base.copy()
                p[c] = np.nextafter(p[c], d)
                cols.append(p)
        r = np.asfortranarray(np.stack(cols, axis=1))
        oracle.track(line, r, nturns, energy=energy, rest_energy=rest)
        ok = np.all(np.isfinite(r), axis=0)
        spread = np.abs(r[:, ok] - r[:, :1]).max(axis=1) / scale if ok[0] else np.inf
        out.append(bool(np.any(spread > tol)) or not ok.all())
    return np.array(out, dtype=bool)


def _compare_long_run(line, r0, rg, lg, g, energy, rest):
    """The engine's 1000-turn result against the reference's (fixture ``g``).
    A particle may be lost in one and not the other, or lost at another turn
    or element, only if its loss coordinate lies within 1e-9 of a limit or
    its fate is ill-conditioned (changes under a one-ulp move of its start,
    _ill_conditioned).  Stable survivors agree within 1e-9 of each
    coordinate's scale; a survivor beyond that must be unstable in the
    reference's own arithmetic (_unstable).  Returns the counts of lost-set
    flips, of loss turn/element differences and of unstable survivors
    beyond 1e-9."""
    lo = {"islost": g["islost"].astype(bool), "turn": g["lturn"], "elem": g["lelem"],
          "coord": g["lcoord"]}
    nb = _near_boundary(line, lo) | _near_boundary(line, lg)
    flip = lo["islost"] != lg["islost"]
    same = lo["islost"] & lg["islost"]
    moved = same & ((lo["turn"] != lg["turn"]) | (lo["elem"] != lg["elem"]))
    suspect = np.flatnonzero((flip | moved) & ~nb)
    ill = _ill_conditioned(line, r0, suspect, int(g["nturns"]), energy, rest)
    assert ill.all(), "loss differs for well-conditioned particles: %s" % suspect[~ill]
    both = np.flatnonzero(~lo["islost"] & ~lg["islost"])
    ref = g["rout_final"][:, both]
    scale = np.maximum(np.abs(ref).max(axis=1), 1e-300)
    dev = (np.abs(rg[:, both] - ref) / scale[:, None]).max(axis=0)
    far = both[dev > 1e-9]
    unst = _unstable(line, r0, far, int(g["nturns"]), energy, rest, scale, 1e-9)
    assert unst.all(), "stable survivors beyond 1e-9: %s" % far[~unst]
    return int(flip.sum()), int(moved.sum()), int(far.size)


def _check_input(r0, g):
    import hashlib
    dig = hashlib.sha256(np.ascontiguousarray(r0).tobytes()).digest()
    assert dig == bytes(g["rin_sha256"]), "the seeded input differs from the fixture's"


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_fodo_1000_turns_full_size(golden, mode):
    """The FODO workload at its stated size: 10,000 particles (seed 0),
    1000 turns, losses on, against the reference's own engine."""
    ring = rings.fodo_ring()
    g = golden("longrun_fodo.npz")
    r0 = rings.gaussian(10000, seed=0)
    _check_input(r0, g)
    rg = r0.copy(order="F")
    _, lg, _ = _gpu_track(ring, rg, int(g["nturns"]), 3e9, ELECTRON_REST, mode, losses=True)
    flips, moved, far = _compare_long_run(ring, r0, rg, lg, g, 3e9, ELECTRON_REST)
    print("FODO 10000 x 1000 (%s): %d lost-set flips, %d loss-turn differences, %d lost, "
          "%d unstable survivors beyond 1e-9" % (mode, flips, moved, int(lg["islost"].sum()),
                                                 far))
    assert 0.2 < lg["islost"].mean() < 0.45          # the workload loses about 30 %


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_large_ring_1000_turns_full_size(golden, mode):
    """The large radiating ring for 1000 turns with 2048 particles around its
    closed orbit (seed 21), losses on, against the reference's own engine."""
    ring = rings.large_ring()
    g = golden("longrun_large.npz")
    r0 = rings.large_ring_bunch(2048, seed=21)
    _check_input(r0, g)
    rg = r0.copy(order="F")
    _, lg, _ = _gpu_track(ring, rg, int(g["nturns"]), ring.energy, ring.particle.rest_energy,
                          mode, losses=True)
    flips, moved, far = _compare_long_run(ring, r0, rg, lg, g, ring.energy,
                                          ring.particle.rest_energy)
    print("large ring 2048 x 1000 (%s): %d lost-set flips, %d loss-turn differences, %d lost, "
          "%d unstable survivors beyond 1e-9" % (mode, flips, moved, int(lg["islost"].sum()),
                                                 far))
    assert far == 0                       # radiation damping: every survivor is stable


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_golden_lattices(golden, mode):
    tol = 1e-14 if mode == "exact" else 1e-13
    ring = rings.fodo_ring()
    g = golden("fodo_refpts.npz")
    r = g["rin"].copy(order="F")
    rout, ld, _ = _gpu_track(ring, r, 30, 3e9, ELECTRON_REST, mode, refpts=g["refpts"],
                             losses=True)
    assert scale_rel_diff(r, g["rout_final"]) <= 1e-11
    assert scale_rel_diff(rout[:, :, :, 0], g["rout"][:, :, :, 0]) <= tol
    np.testing.assert_array_equal(ld["islost"], g["islost"])
    g = golden("fodo_rad_20turns.npz")
    r = g["rin"].copy(order="F")
    _gpu_track(rings.radiating(ring), r, 20, 3e9, ELECTRON_REST, mode)
    assert scale_rel_diff(r, g["rout_final"]) <= 1e-11


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_kitchen_sink_losses_refpts(golden, mode):
    g = golden("sink_3turns.npz")
    line = [cases.make_element(s, E.Element) for s in cases.kitchen_sink()]
    r = g["rin"].copy(order="F")
    rout, ld, _ = _gpu_track(line, r, 3, 6e9, ELECTRON_REST, mode, refpts=g["refpts"],
                             losses=True, turn=5)
    np.testing.assert_array_equal(ld["islost"], g["islost"])
    np.testing.assert_array_equal(ld["turn"], g["lturn"])
    np.testing.assert_array_equal(ld["elem"], g["lelem"])
    np.testing.assert_array_equal(np.isnan(r), np.isnan(g["rout_final"]))
    assert scale_rel_diff(ld["coord"], g["lcoord"]) <= 1e-12
    assert scale_rel_diff(rout[..., 0], g["rout"][..., 0]) <= 1e-12


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_partial_turn(golden, mode):
    g = golden("sink_partial.npz")
    line = [cases.make_element(s, E.Element) for s in cases.kitchen_sink()]
    r = g["rin"].copy(order="F")
    _, ld, _ = _gpu_track(line, r, 1, 6e9, ELECTRON_REST, mode, refpts=g["refpts"], losses=True,
                          start_elem=4, end_elem=15)
    np.testing.assert_array_equal(ld["islost"], g["islost"])
    assert scale_rel_diff(r, g["rout_final"]) <= 1e-12


@pytest.mark.parametrize("tag", ["off", "6d"])
@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_hmba(golden, tag, mode):
    with open(os.path.join(GOLDEN, "hmba.json")) as f:
        data = json.load(f)[tag]
    line = [cases.make_element(d, E.Element) for d in data["specs"]]
    g = golden("hmba_%s.npz" % tag)
    r = g["rin"].copy(order="F")
    _gpu_track(line, r, 1, data["energy"], 0.0, mode)
    assert scale_rel_diff(r, g["rout_final"]) <= (1e-14 if mode == "exact" else 1e-13)


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_pipelined_segments_match_resident(mode):
    """A table too large for one shared-memory buffer streams through the
    double-buffered bulk-copy pipeline; the result must not depend on it."""
    ring = rings.radiating(rings.fodo_ring())
    r0 = rings.gaussian(1000, seed=4)
    eng = Engine.get(0)
    cl = compile_lattice(ring, 3e9, ELECTRON_REST)
    lid = eng.upload(cl)
    ra = r0.copy(order="F")
    eng.track(lid, ra, 5, mode=mode)
    eng.set_launch(seg_cap_words=1024, resident_max_words=512)
    try:
        rb = r0.copy(order="F")
        eng.track(lid, rb, 5, mode=mode)
    finally:
        eng.set_launch(seg_cap_words=6144, resident_max_words=14336)
        eng.free(lid)
    assert not np.array_equal(ra, r0, equal_nan=True)             # tracked
    np.testing.assert_array_equal(ra, rb)



@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_snapshots_beyond_the_budget_track_in_particle_groups(mode):
    """When one turn of refpts snapshots of all particles exceeds the device
    budget, the runtime tracks the particles in groups and copies each
    group's snapshots into its columns of rout: the snapshots, final
    coordinates, loss map (quantum-diffusion kicks included, keyed by the
    particle's index in the whole set) and survivors per turn equal one
    launch's; the per-turn moments are float sums in another order."""
    qd = E.QuantumDiffusion("QD", np.diag([2e-5, 2e-6, 2e-5, 2e-6, 1e-4, 1e-5]))
    fodo = rings.radiating(rings.fodo_ring())
    ring = E.Lattice(list(fodo) + [qd], energy=fodo.energy, particle=fodo.particle)
    eng = Engine.get(0)
    cl = compile_lattice(ring, ring.energy, ELECTRON_REST)
    lid = eng.upload(cl)
    n, nt = 1000, 3
    refs = np.arange(cl.nelem + 1, dtype=np.uint32)      # every element and the turn's end
    r0 = rings.gaussian(n, seed=4) * 40.0                # about a quarter lost in 3 turns
    # budgets in particle-turns of snapshots: groups of 150 one turn at a time;
    # all particles one turn at a time (turn chunks only); groups of 800 (and
    # the remaining 200) two turns at a time
    runs = []
    try:
        ra = r0.copy(order="F")
        oa = eng.track(lid, ra, nt, refpts=refs, losses=True, stats=True, mode=mode)
        for pt in (150, 1000, 1600):
            eng.set_launch(rout_budget_bytes=refs.size * 48 * pt)
            rb = r0.copy(order="F")
            runs.append((rb, eng.track(lid, rb, nt, refpts=refs, losses=True, stats=True,
                                       mode=mode)))
    finally:
        eng.set_launch(rout_budget_bytes=4 << 30)
        eng.free(lid)
    assert oa[1]["islost"].any() and not oa[1]["islost"].all()
    scale = np.abs(oa[2][1]).max(axis=0)                 # per moment, over the turns
    for rb, ob in runs:
        np.testing.assert_array_equal(rb, ra)
        np.testing.assert_array_equal(ob[0], oa[0])
        for k in oa[1]:
            np.testing.assert_array_equal(ob[1][k], oa[1][k], err_msg=k)
        np.testing.assert_array_equal(ob[2][0], oa[2][0])
        assert (np.abs(ob[2][1] - oa[2][1]) <= 1e-12 * scale).all()


def test_large_snapshot_copies_through_staging_match_direct():
    """Snapshots above 8 MB a chunk come back through two pinned staging
    buffers of 64 MB placed by host threads (pieces that end inside a slot's
    row); below it, by direct copies.  593 MB of snapshots in nine pieces must
    equal the same run returned in direct copies of 150-particle groups."""
    ring = rings.fodo_ring()
    eng = Engine.get(0)
    cl = compile_lattice(ring, ring.energy, ELECTRON_REST)
    lid = eng.upload(cl)
    n, nt = 4000, 8
    refs = np.arange(cl.nelem + 1, dtype=np.uint32)
    r0 = rings.gaussian(n, seed=3) * 20.0
    try:
        ra = r0.copy(order="F")
        oa, la, _ = eng.track(lid, ra, nt, refpts=refs, losses=True)
        eng.set_launch(rout_budget_bytes=refs.size * 48 * 150)
        rb = r0.copy(order="F")
        ob, lb, _ = eng.track(lid, rb, nt, refpts=refs, losses=True)
    finally:
        eng.set_launch(rout_budget_bytes=4 << 30)
        eng.free(lid)
    assert oa.nbytes > 8 * (64 << 20) and la["islost"].any()
    np.testing.assert_array_equal(rb, ra)
    np.testing.assert_array_equal(ob, oa)
    for k in la:
        np.testing.assert_array_equal(lb[k], la[k], err_msg=k)

def test_large_ring_one_turn():
    """The radiating large ring (misaligned, 1954 elements) against the oracle.

    exact: 1e-13, the one-turn bound; the exact kernel differs from the
    oracle only through CUDA's sin/tan against the C library's (a few 1e-14
    after one turn of this ring).  fast: 2e-13 -- FMA contraction alone sets
    the floor here: the oracle's own C source compiled with
    -ffp-contract=fast -mfma differs from the reference order by 1.08e-13 (y)
    after one turn of this ring."""
    ring = rings.large_ring()
    r0 = rings.large_ring_bunch(2048)
    ro = r0.copy(order="F")
    oracle.track(ring, ro, 1, energy=ring.energy, rest_energy=ring.particle.rest_energy)
    for mode, tol in (("exact", 1e-13), ("fast", 2e-13)):
        rg = r0.copy(order="F")
        _gpu_track(ring, rg, 1, ring.energy, ring.particle.rest_energy, mode)
        assert scale_rel_diff(rg, ro) <= tol, mode


def test_find_orbit6_matches_constant():
    from at_b200 import physics
    ring = rings.large_ring()
    orb = physics.find_orbit6(ring)
    np.testing.assert_allclose(orb, rings.LARGE_ORBIT, rtol=0, atol=1e-12)


@pytest.mark.parametrize("pattern", ["tiles", "alternate", "sparse"])
@pytest.mark.parametrize("ring_name", ["fodo", "large"])
def test_all_lost_tiles_stop_early(ring_name, pattern):
    """Tiles whose particles are all lost leave the turn loop early (after
    draining their in-flight table copies when the table streams in
    segments), and tiles whose survivors fit in fewer warps than hold them
    move the survivors to the lowest threads (every other particle lost, or
    one in six, which frees one warp of eight); the results equal a run that
    does neither (with a refpts snapshot) and the oracle's loss map."""
    if ring_name == "fodo":
        ring, en, rest = rings.fodo_ring(), 3e9, ELECTRON_REST
        r0 = rings.gaussian(2048, seed=8)
        nt = 40
    else:
        ring = rings.large_ring()
        en, rest = ring.energy, ring.particle.rest_energy
        r0 = rings.large_ring_bunch(2048, seed=8)
        nt = 6
    if pattern == "tiles":
        r0[:, 256:768] *= 1e3        # two whole tiles lost in the first turn
    elif pattern == "alternate":
        r0[:, 1::2] = 2.0            # every other particle lost at the first element
        r0[:, 600:700] = 2.0         # and a run of them
    else:
        r0[:, 5::6] = 2.0            # one particle in six lost at the first element
    ra = r0.copy(order="F")
    _, la, _ = _gpu_track(ring, ra, nt, en, rest, "exact", losses=True)
    rb = r0.copy(order="F")
    _gpu_track(ring, rb, nt, en, rest, "exact", losses=True,
               refpts=np.array([0], dtype=np.uint32))
    np.testing.assert_array_equal(ra, rb)
    if pattern == "tiles":
        assert la["islost"][256:768].all() and not la["islost"].all()
    elif pattern == "alternate":
        assert la["islost"][1::2].all() and not la["islost"].all()
    else:
        assert la["islost"][5::6].all() and not la["islost"].all()
    ro = r0.copy(order="F")
    _, lo = oracle.track(ring, ro, nt, energy=en, rest_energy=rest, losses=True)
    np.testing.assert_array_equal(la["islost"], lo["islost"])
    np.testing.assert_array_equal(la["turn"], lo["turn"])
    np.testing.assert_array_equal(la["elem"], lo["elem"])


@pytest.mark.parametrize("mode", ["exact", "fast"])
@pytest.mark.parametrize("ring_name", ["fodo", "large"])
def test_two_particles_per_thread_match_one(ring_name, mode):
    """Two particles per thread (particle k of thread t at
    tile.first + k*blockDim + t) against one.  exact: every particle runs the
    same correctly rounded operations, so coordinates, refpts snapshots, loss
    maps and per-turn survivor counts are bit-identical.  fast: the compiler
    may contract a product shared by the two particles differently; the
    single-ulp steps (below 1e-16 absolute on these cases) stay within the
    fast mode's one-turn bound of 2e-13 of each coordinate's scale, with the
    same loss map.  The set (ragged, ~10 % lost) fills every
    SM with full two-particle tiles, the size at which the engine uses them."""
    from at_b200.engine import device_info
    eng = Engine.get(0)
    n = device_info(0)[3] * 128 * 2 + 77
    if ring_name == "fodo":
        ring, en, rest = rings.radiating(rings.fodo_ring()), 3e9, ELECTRON_REST
        r0 = rings.gaussian(n, seed=12)
        nt, refs = 20, np.array([0, 3, 7], dtype=np.uint32)
    else:
        ring = rings.large_ring()
        en, rest = ring.energy, ring.particle.rest_energy
        r0 = rings.large_ring_bunch(n, seed=12)
        nt, refs = 3, np.array([0, 500], dtype=np.uint32)
    r0[:, 5::10] *= 1e3
    cl = compile_lattice(ring, en, rest)
    lid = eng.upload(cl)
    out = []
    try:
        for ppt in (1, 2):
            eng.set_launch(threads=128, particles_per_thread=ppt)
            r = r0.copy(order="F")
            rout, ld, st = eng.track(lid, r, nt, 0, 0, cl.nelem, refpts=refs, losses=True,
                                     stats=True, mode=mode)
            out.append((r, rout, ld, st))
    finally:
        eng.set_launch(threads=256, particles_per_thread=1)
        eng.free(lid)
    (ra, oa, la, sa), (rb, ob, lb, sb) = out
    if mode == "exact":
        np.testing.assert_array_equal(ra, rb)
        np.testing.assert_array_equal(oa, ob)
        np.testing.assert_array_equal(la["coord"], lb["coord"])
    else:
        ok = ~la["islost"]
        assert scale_rel_diff(rb[:, ok], ra[:, ok]) <= 2e-13
        assert scale_rel_diff(ob[:, ok], oa[:, ok]) <= 2e-13
    for k in ("islost", "turn", "elem"):
        np.testing.assert_array_equal(la[k], lb[k])
    assert la["islost"].any() and not la["islost"].all()
    np.testing.assert_array_equal(sa[0], sb[0])
    np.testing.assert_allclose(sa[1], sb[1], rtol=1e-12, atol=1e-300)


def _clear_flag(cl, bit):
    """A copy of ``cl`` whose element headers have flag ``bit`` cleared."""
    import copy
    from at_b200 import table as T
    c = copy.copy(cl)
    c.words = cl.words.copy()
    hdr = c.words.view(np.uint64)
    for off in cl.offsets[:-1]:
        hdr[int(off)] &= ~np.uint64(bit << T.ATB_H_FL_SHIFT)
    return c


@pytest.mark.parametrize("ring_name", ["fodo", "fodo_rad", "large"])
def test_upright_field_evaluation_matches_general(ring_name):
    """The fast kernel evaluates upright magnets (every PolynomA zero) from
    Im = 0 without the skew terms, the same values as the general recursion
    up to the sign of a zero.  The two instances of the magnet code around it
    are compiled apart, so the compiler's FMA contraction may differ between
    them: on the same table with the upright flag cleared the results agree
    within the fast mode's one-turn bound (measured: identical on the
    radiating rings, one coordinate one ulp apart on the plain FODO ring),
    with the same loss map."""
    from at_b200 import table as T
    if ring_name.startswith("fodo"):
        ring, en, rest = rings.fodo_ring(), 3e9, ELECTRON_REST
        if ring_name == "fodo_rad":
            ring = rings.radiating(ring)
        r0, nt = rings.gaussian(4096, seed=13), 20
    else:
        ring = rings.large_ring()
        en, rest = ring.energy, ring.particle.rest_energy
        r0, nt = rings.large_ring_bunch(4096, seed=13), 3
    eng = Engine.get(0)
    cl = compile_lattice(ring, en, rest)
    general = _clear_flag(cl, T.ATB_F_NOSKEW)
    out = []
    for c in (cl, general):
        lid = eng.upload(c)
        try:
            r = r0.copy(order="F")
            _, ld, _ = eng.track(lid, r, nt, 0, 0, c.nelem, losses=True, mode="fast")
        finally:
            eng.free(lid)
        out.append((r, ld))
    np.testing.assert_array_equal(out[0][1]["islost"], out[1][1]["islost"])
    ok = ~out[0][1]["islost"]
    assert scale_rel_diff(out[0][0][:, ok], out[1][0][:, ok]) <= 2e-13
