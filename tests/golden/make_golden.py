"""Generate the golden fixtures under tests/golden/ from the reference itself.

Runs the reference pyat (atcollab/at: its C engine ``pyat/at.c`` and its
``atintegrators``), built from the reference sources by
``oracle/build_ref.py --full`` into ``oracle/_ref/pyat_full``, on the seeded
cases of ``tests/golden/cases.py`` and on the reference's own machine file
``hmba.mat``, and stores inputs and outputs as small ``.npz`` files.  Only
this script touches the reference; the tests read the fixtures.

    python oracle/build_ref.py --full && python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle", "_ref", "pyat_full"))
sys.path.insert(0, HERE)

import at  # noqa: E402  (the reference, built from its sources)
from at.tracking.atpass import atpass, elempass  # noqa: E402

import cases  # noqa: E402

ARRAY_ATTRS = {"PolynomA", "PolynomB", "KickAngle", "T1", "T2", "R1", "R2", "RApertures",
               "EApertures", "Limits", "fringeIntM0", "fringeIntP0", "BendingAngle", "Lmatp"}


def ref_element(d):
    kw = {}
    late = {}
    for k, v in d.items():
        if k in ("FamName",):
            continue
        if k in ARRAY_ATTRS and not (k == "BendingAngle" and np.isscalar(v)):
            a = np.asfortranarray(np.asarray(v, dtype=np.float64))
            if k == "BendingAngle":
                late[k] = a            # a thin multipole's (bax, bay) array
            else:
                kw[k] = a
        else:
            kw[k] = v
    el = at.Element(d.get("FamName", "E"), **kw)
    for k, v in late.items():
        object.__setattr__(el, k, v)
    # pyat's base Element keeps the values as given; make sure the integer
    # attributes are Python ints as the integrators read them with PyLong
    for k in ("MaxOrder", "NumIntSteps", "FringeBendEntrance", "FringeBendExit",
              "FringeQuadEntrance", "FringeQuadExit"):
        if hasattr(el, k):
            setattr(el, k, int(getattr(el, k)))
    return el


def spec_json(d):
    out = {}
    for k, v in d.items():
        if isinstance(v, np.ndarray):
            out[k] = {"shape": list(v.shape), "data": v.ravel(order="F").tolist()}
        else:
            out[k] = v
    return out


def element_fixtures():
    electron = at.Particle("electron")
    res = {}
    meta = {}
    for name, d in cases.element_cases():
        r0 = cases.element_particles()
        if d["PassMethod"] == "AperturePass":
            r0[0, 5] = 5e-3
        r = r0.copy(order="F")
        el = ref_element(d)
        rad = "Rad" in d["PassMethod"] or d["PassMethod"] == "RFCavityPass"
        kw = dict(energy=6e9, particle=electron) if rad else {}
        elempass(el, r, **kw)
        res[name + "/in"] = r0
        res[name + "/out"] = r
        meta[name] = spec_json(d)
    np.savez_compressed(os.path.join(HERE, "elements.npz"), **res)
    with open(os.path.join(HERE, "elements.json"), "w") as f:
        json.dump(meta, f, indent=0, sort_keys=True)


def fodo_fixture():
    sys.path.insert(0, REPO)
    from at_b200 import rings
    ring = rings.fodo_ring()
    line = [ref_element(vars_of(e)) for e in ring]
    r0 = rings.gaussian(10000)[:, ::40].copy(order="F")       # 250 particles
    r0[:, :50] *= 4.0                                         # some to be lost
    r = r0.copy(order="F")
    rout, ld = atpass(line, r, 200, energy=3e9, particle=at.Particle("electron"), losses=True)
    np.savez_compressed(os.path.join(HERE, "fodo_200turns.npz"), rin=r0, rout_final=r,
                        islost=ld["islost"], lturn=ld["turn"], lelem=ld["elem"],
                        lcoord=ld["coord"])
    # refpts snapshots: 64 particles, 30 turns
    r0 = r0[:, 20:84].copy(order="F")
    r = r0.copy(order="F")
    refs = np.array([0, 100, 385], dtype=np.uint32)
    rout, ld = atpass(line, r, 30, refpts=refs, energy=3e9, particle=at.Particle("electron"),
                      losses=True)
    np.savez_compressed(os.path.join(HERE, "fodo_refpts.npz"), rin=r0, rout_final=r,
                        rout=rout, refpts=refs, islost=ld["islost"], lturn=ld["turn"],
                        lelem=ld["elem"], lcoord=ld["coord"])
    # radiating copy, 20 turns
    rr = rings.radiating(ring)
    line = [ref_element(vars_of(e)) for e in rr]
    r0 = rings.gaussian(64, seed=3)
    r = r0.copy(order="F")
    atpass(line, r, 20, energy=3e9, particle=at.Particle("electron"))
    np.savez_compressed(os.path.join(HERE, "fodo_rad_20turns.npz"), rin=r0, rout_final=r)


def ref_lattice(ring):
    """A reference Lattice of one of our rings (cavities as at.RFCavity, which
    the reference finds by class)."""
    line = []
    for e in ring:
        d = vars_of(e)
        if d["PassMethod"] == "RFCavityPass":
            line.append(at.RFCavity(d["FamName"], d["Length"], d["Voltage"], d["Frequency"],
                                    d["HarmNumber"], d["Energy"], TimeLag=d["TimeLag"]))
        else:
            line.append(ref_element(d))
    return at.Lattice(line, energy=ring.energy, particle=at.Particle("electron"), periodicity=1)


def ohmi_fixture():
    """The reference's Ohmi-envelope path on the radiating large ring:
    per-element diffusion matrices (pyat/at.c:755-831 ``diffusion_matrix``)
    at the closed orbit for the first cell's magnets and for bends with fringe
    integrals, the cumulative diffusion matrix (``_dmatr``), and
    ``ohmi_envelope`` (pyat/at/physics/radiation.py:151-276)."""
    sys.path.insert(0, REPO)
    from at_b200 import rings
    from at.physics import radiation as rad
    from at.tracking import diffusion_matrix
    lat = ref_lattice(rings.large_ring(seed=1))
    orbit, _ = at.find_orbit6(lat)
    bbcum, orbs = rad._dmatr(lat, orbit=orbit)
    emit0, beamdata, emit = at.ohmi_envelope(lat, refpts=[0, 100, 1000], orbit=orbit)
    idx = np.array([i for i, e in enumerate(lat[:70]) if e.PassMethod.endswith("RadPass")])
    bel = np.stack([diffusion_matrix(lat[i], np.asfortranarray(orbs[i].copy()), energy=lat.energy)
                    for i in idx])
    # bends with fringe integrals and the four edge methods
    specs, borb, bfr = [], [], []
    rng = np.random.default_rng(17)
    for method in (0, 1, 2, 3):
        d = {"FamName": "BF", "PassMethod": "BndMPoleSymplectic4RadPass", "Length": 0.8,
             "BendingAngle": 0.05, "EntranceAngle": 0.02, "ExitAngle": 0.03,
             "PolynomA": [0.0, 0.0, 0.0], "PolynomB": [0.0, -0.3, 2.0], "MaxOrder": 2,
             "NumIntSteps": 10, "FullGap": 0.04, "FringeInt1": 0.5, "FringeInt2": 0.4,
             "FringeBendEntrance": method, "FringeBendExit": method}
        o = rng.standard_normal(6) * np.array([1e-3, 1e-4, 1e-3, 1e-4, 1e-3, 1e-3])
        specs.append(d)
        borb.append(o)
        bfr.append(diffusion_matrix(ref_element(d), np.asfortranarray(o.copy()), energy=3e9))
    np.savez_compressed(os.path.join(HERE, "ohmi_large.npz"), orbit=orbit, idx=idx,
                        orbits=orbs[idx], belem=bel, bcum=bbcum[-1], orbs_all=orbs,
                        r66=emit0.r66, emitXY=emit0.emitXY, emitXYZ=emit0.emitXYZ,
                        m66=emit0.m66, tunes=beamdata.tunes, damping_rates=beamdata.damping_rates,
                        mode_emittances=beamdata.mode_emittances, bend_orbits=np.array(borb),
                        bend_b=np.array(bfr), refpts=np.array([0, 100, 1000]),
                        emit_r66=emit.r66, emit_emitXYZ=emit.emitXYZ)
    with open(os.path.join(HERE, "ohmi_bends.json"), "w") as f:
        json.dump(specs, f)


def quantdiff_fixture():
    """QuantDiffPass with the reference's random stream: after
    reset_rng(seed=...), two consecutive calls (the stream continues), with
    a refpts snapshot, through a line mixing diffusion kicks and magnets; and
    the reference's gen_quantdiff_elem matrix for the large ring."""
    from at.tracking.atpass import reset_rng
    rng = np.random.default_rng(31)
    mats = []
    for scale in (3e-5, 1e-4):
        m = np.tril(rng.standard_normal((6, 6))) * scale
        mats.append(np.asfortranarray(m))
    specs = [
        {"FamName": "D1", "PassMethod": "DriftPass", "Length": 0.5},
        {"FamName": "QD1", "PassMethod": "QuantDiffPass", "Lmatp": mats[0]},
        {"FamName": "Q", "PassMethod": "StrMPoleSymplectic4Pass", "Length": 0.4,
         "PolynomA": [0.0, 0.0], "PolynomB": [0.0, 1.2], "MaxOrder": 1, "NumIntSteps": 10},
        {"FamName": "QD2", "PassMethod": "QuantDiffPass", "Lmatp": mats[1]},
        {"FamName": "D2", "PassMethod": "DriftPass", "Length": 0.3},
    ]
    line = [ref_element(d) for d in specs]
    r0 = np.asfortranarray(rng.standard_normal((6, 40)) * 1e-4)
    r0[0, 7] = np.nan                       # a lost particle still draws its normals
    r0[1:, 7] = 0.0
    reset_rng(seed=4242)
    r1 = r0.copy(order="F")
    atpass(line, r1, 3, energy=3e9, particle=at.Particle("electron"))
    r2 = r1.copy(order="F")
    refs = np.array([0, 2, 5], dtype=np.uint32)
    rout = atpass(line, r2, 2, refpts=refs, energy=3e9, particle=at.Particle("electron"))
    sys.path.insert(0, REPO)
    from at_b200 import rings
    lat = ref_lattice(rings.large_ring(seed=1))
    lmatp = at.gen_quantdiff_elem(lat).Lmatp
    np.savez_compressed(os.path.join(HERE, "quantdiff.npz"), l0=mats[0], l1=mats[1], rin=r0,
                        r1=r1, r2=r2, rout=rout, refpts=refs, large_lmatp=lmatp)


def acceptance_fixture():
    """The reference's grid-mode acceptance scans (pyat/at/acceptance) on the
    radiating large ring: radial and cartesian 2-D grids, two observation
    points, and a 1-D momentum scan; arrays stored by case name."""
    sys.path.insert(0, REPO)
    from at_b200 import rings
    from at.acceptance import GridMode
    lat = ref_lattice(rings.large_ring(seed=1))
    out = {}
    cases = {
        "radial": dict(planes=["x", "y"], npoints=[9, 7], amplitudes=[6e-3, 3e-3],
                       grid_mode=GridMode.RADIAL),
        "cartesian": dict(planes=["x", "y"], npoints=[11, 6], amplitudes=[6e-3, 3e-3],
                          grid_mode=GridMode.CARTESIAN),
        "momentum": dict(planes=["dp"], npoints=[21], amplitudes=[0.04],
                         grid_mode=GridMode.CARTESIAN),
    }
    for name, kw in cases.items():
        b, sv, g = at.get_acceptance(lat, nturns=32, use_mp=False, **kw)
        out[name + "_b"], out[name + "_s"], out[name + "_g"] = b, sv, g
    b, sv, g = at.get_acceptance(lat, ["x", "y"], [7, 5], [6e-3, 3e-3], nturns=16,
                                 refpts=[0, 61], grid_mode=GridMode.RADIAL, use_mp=False)
    for k in range(2):
        out["multi%d_b" % k], out["multi%d_s" % k], out["multi%d_g" % k] = b[k], sv[k], g[k]
    np.savez_compressed(os.path.join(HERE, "acceptance_large.npz"), **out)


def acceptance_modes_fixture():
    """The reference's other acceptance searches on the radiating large ring
    (pyat/at/acceptance/boundary.py:409-500 recursive, floodfill_acceptance.py
    flood fill) and a larger cartesian grid, at few turns; arrays stored by
    case name (boundary, survived, tracked)."""
    sys.path.insert(0, REPO)
    from at_b200 import rings
    from at.acceptance import GridMode
    lat = ref_lattice(rings.large_ring(seed=1))
    out = {}
    cases_ = {
        "cart21": dict(planes=["x", "y"], npoints=[21, 11], amplitudes=[8e-3, 4e-3],
                       grid_mode=GridMode.CARTESIAN, nturns=24),
        "rec2d": dict(planes=["x", "y"], npoints=[12, 7], amplitudes=[8e-3, 4e-3],
                      grid_mode=GridMode.RECURSIVE, nturns=16),
        "rec1d": dict(planes=["dp"], npoints=[16], amplitudes=[0.04],
                      grid_mode=GridMode.RECURSIVE, nturns=16),
        "flood": dict(planes=["x", "y"], npoints=[15, 9], amplitudes=[8e-3, 4e-3],
                      grid_mode=GridMode.FLOODFILL, nturns=16),
        "flood_obs": dict(planes=["x", "y"], npoints=[11, 7], amplitudes=[8e-3, 4e-3],
                          grid_mode=GridMode.FLOODFILL, nturns=12, refpts=61),
        "rec_obs": dict(planes=["x", "y"], npoints=[8, 5], amplitudes=[8e-3, 4e-3],
                        grid_mode=GridMode.RECURSIVE, nturns=12, refpts=61),
    }
    # the flood fill centres its grid on the orbit of a ring copy whose RF
    # frequency is reset for dp = 0 (boundary.py:303-309 with
    # frequency_control); the fixtures give both searches the ring's own 6-D
    # closed orbit at the observation point instead, through ``offset``
    orbit0 = np.array(rings.LARGE_ORBIT, dtype=np.float64)
    _, orbit61 = lat.find_orbit(refpts=61, orbit=orbit0)
    out["orbit0"], out["orbit61"] = orbit0, np.squeeze(orbit61)
    for name, kw in cases_.items():
        if kw["grid_mode"] is GridMode.FLOODFILL:
            kw = dict(kw, offset=out["orbit61"] if kw.get("refpts") else orbit0)
        b, sv, g = at.get_acceptance(lat, use_mp=False, **kw)
        out[name + "_b"], out[name + "_s"], out[name + "_g"] = b, sv, g
    np.savez_compressed(os.path.join(HERE, "acceptance_modes.npz"), **out)


def longrun_fixture():
    """The two tracking workloads at their stated sizes, run by the reference's
    own engine (OpenMP over every core of this machine): the FODO ring with
    10,000 particles (Gaussian from seed 0) for 1000 turns, and the radiating
    large ring with 2048 particles around its closed orbit (seed 21) for 1000
    turns, losses on.  The inputs are regenerated from their seeds by the
    tests (a digest of each input is stored to catch a generator change)."""
    import hashlib
    sys.path.insert(0, REPO)
    from at_b200 import rings
    nthreads = os.cpu_count() or 1
    for tag, ring, r0, nturns in (
            ("fodo", rings.fodo_ring(), rings.gaussian(10000, seed=0), 1000),
            ("large", rings.large_ring(), rings.large_ring_bunch(2048, seed=21), 1000)):
        lat = ref_lattice(ring)
        r = r0.copy(order="F")
        _, ld = atpass(list(lat), r, nturns, energy=float(ring.energy),
                       particle=at.Particle("electron"), losses=True,
                       omp_num_threads=nthreads)
        np.savez_compressed(os.path.join(HERE, "longrun_%s.npz" % tag),
                            rin_sha256=np.frombuffer(hashlib.sha256(
                                np.ascontiguousarray(r0).tobytes()).digest(), dtype=np.uint8),
                            nturns=nturns, rout_final=r, islost=ld["islost"], lturn=ld["turn"],
                            lelem=ld["elem"], lcoord=ld["coord"])


def optics_fixture():
    """The reference's linopt6 (pyat/at/physics/linear.py:846-971) with
    chromaticity at a few observation points of the radiating large ring and
    of its own hmba.mat in 6-D, and its find_orbit6 of four error-seeded
    large-ring variants (seeds 2-5)."""
    import warnings
    sys.path.insert(0, REPO)
    from at_b200 import rings
    out = {}
    lat = ref_lattice(rings.large_ring(seed=1))
    # pyat switches radiation on and off by element class (Lattice._set_6d):
    # give the generic elements the classes a user's lattice would have
    for i, e in enumerate(lat):
        cls = (at.Dipole if e.PassMethod.startswith("BndMPole") else
               at.Multipole if e.PassMethod.startswith("StrMPole") else None)
        if cls is not None:
            new = cls.__new__(cls)
            for k, v in vars(e).items():
                object.__setattr__(new, k, v)
            lat[i] = new
    refs = np.array([0, 1, 61, 500, 977, 1500, len(lat) - 1], dtype=np.uint32)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        e0, bd, el = at.linopt6(lat, refpts=refs, get_chrom=True)
    out["large_refpts"] = refs
    for k in ("alpha", "beta", "mu", "R", "A", "dispersion", "closed_orbit", "M", "s_pos"):
        out["large_e0_" + k] = e0[k]
        out["large_el_" + k] = el[k]
    for k in ("tune", "chromaticity", "damping_time"):
        out["large_bd_" + k] = bd[k]
    for seed in (2, 3, 4, 5):
        v = ref_lattice(rings.large_ring_variant(seed))
        o, _ = at.find_orbit6(v)
        out["variant%d_orbit" % seed] = o
    hmba = at.load_mat(os.path.join(REPO, "oracle", "_ref", "pyat_full", "machine_data",
                                    "hmba.mat"), use="RING").enable_6d(copy=True)
    hrefs = np.array([0, 5, 40, len(hmba) - 1], dtype=np.uint32)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        e0, bd, el = at.linopt6(hmba, refpts=hrefs, get_chrom=True)
    out["hmba_refpts"] = hrefs
    for k in ("alpha", "beta", "mu", "dispersion", "closed_orbit", "M", "s_pos"):
        out["hmba_el_" + k] = el[k]
        out["hmba_e0_" + k] = e0[k]
    for k in ("tune", "chromaticity", "damping_time"):
        out["hmba_bd_" + k] = bd[k]
    np.savez_compressed(os.path.join(HERE, "optics.npz"), **out)


def m66_fixture():
    """The reference's closed orbit (find_orbit6) and one-turn matrix
    (find_m66, pyat/at/physics/matrix.py:105-165: central differences with
    XYStep/DPStep) of the FODO ring, for the exact-derivative Jacobian."""
    sys.path.insert(0, REPO)
    from at_b200 import rings
    line = []
    for e in rings.fodo_ring():
        d = vars_of(e)
        if d["PassMethod"] == "RFCavityPass":
            # the reference finds its cavities by class
            line.append(at.RFCavity(d["FamName"], d["Length"], d["Voltage"], d["Frequency"],
                                    d["HarmNumber"], d["Energy"], TimeLag=d["TimeLag"]))
        else:
            line.append(ref_element(d))
    lat = at.Lattice(line, energy=3e9, particle=at.Particle("electron"), periodicity=1)
    orbit, _ = at.find_orbit6(lat)
    m66, _ = at.find_m66(lat, orbit=orbit)
    np.savez_compressed(os.path.join(HERE, "fodo_m66.npz"), orbit=orbit, m66=m66)


def vars_of(e):
    d = {}
    for k, v in vars(e).items():
        d[k] = v
    return d


def sink_fixture():
    line = [ref_element(d) for d in cases.kitchen_sink()]
    r0 = cases.element_particles(96, seed=21, scale=0.4)
    r = r0.copy(order="F")
    refs = np.array([0, 3, 7, 12, len(line)], dtype=np.uint32)
    rout, ld = atpass(line, r, 3, refpts=refs, turn=5, energy=6e9,
                      particle=at.Particle("electron"), losses=True)
    np.savez_compressed(os.path.join(HERE, "sink_3turns.npz"), rin=r0, rout_final=r, rout=rout,
                        refpts=refs, islost=ld["islost"], lturn=ld["turn"], lelem=ld["elem"],
                        lcoord=ld["coord"])
    # partial turn: start at element 4, refpts before the start are skipped
    r = r0.copy(order="F")
    rout, ld = atpass(line, r, 1, refpts=refs, start_elem=4, end_elem=15, energy=6e9,
                      particle=at.Particle("electron"), losses=True)
    np.savez_compressed(os.path.join(HERE, "sink_partial.npz"), rin=r0, rout_final=r,
                        rout=rout, refpts=refs, islost=ld["islost"], lturn=ld["turn"],
                        lelem=ld["elem"], lcoord=ld["coord"])


def hmba_fixture():
    path = os.path.join(REPO, "oracle", "_ref", "pyat_full", "machine_data", "hmba.mat")
    ring = at.load_lattice(path)
    out = {}
    for tag, lat in (("off", ring.radiation_off(copy=True)), ("6d", ring.enable_6d(copy=True))):
        specs = []
        for e in lat:
            d = {"FamName": e.FamName, "PassMethod": e.PassMethod}
            for k in ("Length", "PolynomA", "PolynomB", "MaxOrder", "NumIntSteps", "BendingAngle",
                      "EntranceAngle", "ExitAngle", "FringeQuadEntrance", "FringeQuadExit",
                      "Voltage", "Frequency", "HarmNumber", "TimeLag", "Energy",
                      "FringeBendEntrance", "FringeBendExit", "FullGap", "FringeInt1",
                      "FringeInt2"):
                if hasattr(e, k):
                    v = getattr(e, k)
                    d[k] = np.asarray(v).tolist() if isinstance(v, np.ndarray) else v
            specs.append(d)
        line = [ref_element(d) for d in specs]
        r0 = np.asfortranarray(np.random.default_rng(5).standard_normal((6, 32)) *
                               np.array([1e-4, 1e-5, 1e-5, 1e-6, 1e-3, 1e-3])[:, None])
        r = r0.copy(order="F")
        atpass(line, r, 1, energy=float(ring.energy), particle=ring.particle)
        out[tag] = dict(specs=specs, energy=float(ring.energy))
        np.savez_compressed(os.path.join(HERE, "hmba_%s.npz" % tag), rin=r0, rout_final=r)
        if tag == "off":
            # the reference test's partial-turn cases (test_atpass.py:157-171)
            for s, e in ((100, 0), (100, 110)):
                r1 = np.array([0, 1e-6, 0, 0, 0, 0], dtype=np.float64)
                atpass(line, r1, 1, start_elem=s, end_elem=e, energy=float(ring.energy))
                out[tag]["partial_%d_%d" % (s, e)] = r1.tolist()
    with open(os.path.join(HERE, "hmba.json"), "w") as f:
        json.dump(out, f)


FIXTURES = ["element_fixtures", "fodo_fixture", "sink_fixture", "hmba_fixture", "m66_fixture",
            "ohmi_fixture", "quantdiff_fixture", "acceptance_fixture",
            "acceptance_modes_fixture", "longrun_fixture", "optics_fixture"]

if __name__ == "__main__":
    # no argument: every fixture; otherwise the named ones (e.g. acceptance_modes)
    names = sys.argv[1:] or FIXTURES
    for nm in names:
        fn = nm if nm.endswith("_fixture") or nm.endswith("_fixtures") else nm + "_fixture"
        globals()[fn]()
    print("golden fixtures written to", HERE)
