"""The oracle against the known-answer vectors of tests/golden/kat.json
(an independent pure-Python restatement, see make_golden.py) and the
reference's own LandscapeExtent iteration tests (extent.rs:110-160)."""
import numpy as np


def test_seed_from_u64(oracle, kat):
    for s, v in kat["seed_from_u64"].items():
        assert oracle.seed_from_u64(int(s)) == v


def test_seahash_and_wymum(oracle, kat):
    L = oracle.lib()
    for x, v in kat["seahash_diffuse"].items():
        assert L.oracle_seahash_diffuse(int(x)) == v
    for a, b, v in kat["wymum"]:
        assert L.oracle_wymum(a, b) == v


def test_wyhash_sequences(oracle, kat):
    for case in kat["wyhash_sequences"]:
        got = oracle.wyhash_sequence(case["seed"], case["location"], case["time_index"],
                                     len(case["u64"]))
        assert [int(v) for v in got] == case["u64"]


def test_poisson_next_event_time(oracle, kat):
    for case in kat["poisson_next_event_time"]:
        t, rp = oracle.poisson_next_event_time(case["seed"], case["injection"], case["time"])
        assert np.float64(t).view(np.uint64) == case["event_time_bits"]
        assert rp == case["reprime"]
        assert t > case["time"]


def test_poisson_next_event_time_at_other_rates(oracle, kat):
    """Turnover rates 0.05..10 and other intervals (per-cell rates of a
    turnover map use the same function); lambda * delta_t = 20 counts past
    the eight tabulated Devroye ranks."""
    for case in kat["poisson_next_event_time_rates"]:
        t, rp = oracle.poisson_next_event_time(case["seed"], case["injection"], case["time"], case["lambda"],
                                               case["delta_t"])
        assert np.float64(t).view(np.uint64) == case["event_time_bits"]
        assert rp == case["reprime"]


def test_exp_next_event_time(oracle, kat):
    """exp.rs against a restatement whose logarithm is the correctly rounded
    one from 60-digit decimal arithmetic (independent of ln_dd.h)."""
    for case in kat["exp_next_event_time"]:
        t, rp = oracle.exp_next_event_time(case["seed"], case["injection"], case["time"], case["lambda"],
                                           case["delta_t"])
        assert np.float64(t).view(np.uint64) == case["event_time_bits"]
        assert rp == case["reprime"]


def test_normal_dispersal(oracle, kat):
    for d0, d1, sigma, x, y, tx, ty in kat["normal_dispersal"]:
        assert oracle.normal_dispersal(d0, d1, sigma, x, y) == (tx, ty)


def test_circle_origin_order(oracle, kat):
    # the circle sampler walks a (possibly wrapping) LandscapeExtent
    for case in kat["circle_origins"]:
        desc = dict(kind=oracle.ALMOST_INFINITE_NORMAL, speciation_probability=0.1, sigma=1.0,
                    centre_x=case["centre"][0], centre_y=case["centre"][1],
                    radius=case["radius"])
        o = oracle.enumerate_origins(desc)
        assert [[int(a), int(b)] for a, b in zip(o["x"], o["y"])] == case["locations"]
        assert list(o["gref"]) == [(y << 32) | x for x, y in case["locations"]]


def test_extent_iteration_cases_present(kat):
    # restated expectations of the reference's extent tests, incl. wrapping
    m1, m2 = 0xFFFFFFFF, 0xFFFFFFFE
    cases = kat["extent_iter"]
    assert cases[0]["locations"] == [[0, 0]]
    assert cases[1]["locations"][:5] == [[42, 24], [43, 24], [44, 24], [45, 24], [42, 25]]
    assert cases[2]["locations"] == [[m2, m1], [m1, m1], [0, m1], [1, m1],
                                     [m2, 0], [m1, 0], [0, 0], [1, 0]]


def test_nonspatial_reference_runs(oracle, kat):
    """Full reference-schedule runs of tiny NonSpatial scenarios: steps,
    time, species and the delivered speciation stream."""
    for case in kat["nonspatial_runs"]:
        desc = dict(kind=oracle.NON_SPATIAL, speciation_probability=case["speciation"],
                    width=case["width"], height=case["height"], deme=case["deme"])
        r = oracle.simulate(desc, case["seed"], mode=oracle.MODE_REFERENCE)
        assert r.steps == case["steps"]
        assert r.time == case["time"]
        assert r.biodiversity == case["biodiversity"]
        got = [[int(e["gref"]), float(e["prior_time"]), float(e["event_time"]), int(e["x"]),
                int(e["y"]), int(e["index"])] for e in r.speciation]
        assert got == case["events"]


def test_nonspatial_reference_runs_with_exponential_event_times(oracle, kat):
    for case in kat["nonspatial_runs_exp"]:
        desc = dict(kind=oracle.NON_SPATIAL, speciation_probability=case["speciation"],
                    width=case["width"], height=case["height"], deme=case["deme"])
        r = oracle.simulate(desc, case["seed"], mode=oracle.MODE_REFERENCE, event_time_sampler=oracle.SAMPLER_EXP)
        assert (r.steps, r.time, r.biodiversity) == (case["steps"], case["time"], case["biodiversity"])
        got = [[int(e["gref"]), float(e["prior_time"]), float(e["event_time"]), int(e["x"]),
                int(e["y"]), int(e["index"])] for e in r.speciation]
        assert got == case["events"]


def test_nonspatial_origin_order(oracle):
    o = oracle.enumerate_origins(dict(kind=0, speciation_probability=0.1, width=3, height=2,
                                      deme=2))
    assert list(o["gref"]) == list(range(12))
    assert list(zip(o["x"], o["y"], o["index"]))[:5] == [(0, 0, 0), (0, 0, 1), (1, 0, 0),
                                                         (1, 0, 1), (2, 0, 0)]


def _clark2dt_restated(d0, d1, shape_u, tail_p, x, y):
    """almost_infinite_clark2dt.rs:96-107, clark2dt::cdf_inverse / pow_fast_one
    (:167-189) and almost_infinite.rs:100-114, restated in Python."""
    import math
    u01 = (d0 >> 11) * 2.0 ** -53
    u2 = ((d1 >> 11) + 1) * 2.0 ** -53
    expo = 1.0 / tail_p
    base = 1.0 / (1.0 - u01)
    jump = math.sqrt(shape_u * ((base if expo == 1.0 else math.pow(base, expo)) - 1.0))
    theta = u2 * 2.0 * math.pi
    dx, dy = math.cos(theta) * jump, math.sin(theta) * jump

    def rnd(v):  # f64::round: half away from zero
        return int(math.floor(abs(v) + 0.5)) * (1 if v >= 0 else -1)
    return (x + rnd(dx)) % (1 << 32), (y + rnd(dy)) % (1 << 32)


def test_clark2dt_dispersal_matches_restatement(oracle):
    import random
    rng = random.Random(5)
    for shape_u, tail_p in [(4.0, 0.5), (1.0, 1.0), (0.3, 2.5), (25.0, 0.2)]:
        for _ in range(2000):
            d0, d1 = rng.getrandbits(64), rng.getrandbits(64)
            x, y = rng.getrandbits(32), rng.getrandbits(32)
            assert oracle.clark2dt_dispersal(d0, d1, shape_u, tail_p, x, y) == \
                _clark2dt_restated(d0, d1, shape_u, tail_p, x, y)


def se_desc(oracle, case):
    return dict(kind=oracle.SPATIALLY_EXPLICIT, speciation_probability=case["speciation"],
                width=case["width"], height=case["height"],
                habitat=np.array(case["habitat"], dtype=np.uint32),
                dispersal=np.array(case["dispersal"], dtype=np.float64))


def flat_tables(case):
    """The golden per-row tables as the flat layout both implementations use."""
    start, end, sd, ns, au, ae, ak = [], [], [], [], [], [], []
    for row in case["tables"]:
        start.append(len(au))
        for u, e, k in row["atoms"]:
            au.append(u)
            ae.append(e)
            ak.append(k)
        end.append(len(au))
        sd.append(row["self_dispersal"])
        ns.append(row["non_self_event"])
    return (np.array(start, np.uint64), np.array(end, np.uint64), np.array(sd), np.array(ns, np.uint64),
            np.array(au), np.array(ae, np.uint32), np.array(ak, np.uint32))


def test_spatially_explicit_tables_match_restatement(oracle, nb, syn, kat):
    """InMemoryPackedSeparableAliasDispersalSampler::new restated in Python
    (alias/packed.rs:59-121, packed_separable_alias/mod.rs:64-203) against
    the oracle's tables and the backend's host build."""
    for case in kat["spatially_explicit_runs"]:
        start, end, sd, ns, au, ae, ak = flat_tables(case)
        ref = oracle.build_alias(se_desc(oracle, case))
        assert np.array_equal(ref["range_start"], start) and np.array_equal(ref["range_end"], end)
        assert np.array_equal(ref["self_dispersal"].view(np.uint64), sd.view(np.uint64))
        assert np.array_equal(ref["non_self_event"], ns)
        assert np.array_equal(ref["atom_u"].view(np.uint64), au.view(np.uint64))
        assert np.array_equal(ref["atom_e"], ae) and np.array_equal(ref["atom_k"], ak)
        cells, atoms = nb.build_tables(syn.to_scenario(se_desc(oracle, case)))
        assert np.array_equal(cells["atom_start"].astype(np.uint64), start)
        assert np.array_equal(cells["self_dispersal"].view(np.uint64), sd.view(np.uint64))
        assert np.array_equal(atoms["u"].view(np.uint64), au.view(np.uint64))
        assert np.array_equal(atoms["e"], ae) and np.array_equal(atoms["k"], ak)


def test_spatially_explicit_reference_runs(oracle, kat):
    """Full reference-schedule runs of tiny SpatiallyExplicit landscapes (zero
    cells, self-dispersal-only rows, full self-dispersal buckets)."""
    for case in kat["spatially_explicit_runs"]:
        r = oracle.simulate(se_desc(oracle, case), case["seed"], mode=oracle.MODE_REFERENCE)
        assert (r.steps, r.time, r.biodiversity) == (case["steps"], case["time"], case["biodiversity"])
        got = [[int(e["gref"]), float(e["prior_time"]), float(e["event_time"]), int(e["x"]),
                int(e["y"]), int(e["index"])] for e in r.speciation]
        assert got == case["events"]


def check_run(oracle, desc, case):
    r = oracle.simulate(desc, case["seed"], mode=oracle.MODE_REFERENCE)
    assert (r.steps, r.time, r.biodiversity) == (case["steps"], case["time"], case["biodiversity"])
    got = [[int(e["gref"]), float(e["prior_time"]), float(e["event_time"]), int(e["x"]),
            int(e["y"]), int(e["index"])] for e in r.speciation]
    assert got == case["events"]


def test_spatially_implicit_reference_runs(oracle, kat):
    """Local community with migration into a metacommunity at the far corner
    of the plane; no speciation locally, so the water level can be infinite."""
    for case in kat["spatially_implicit_runs"]:
        desc = dict(kind=oracle.SPATIALLY_IMPLICIT, speciation_probability=case["speciation"],
                    width=case["width"], height=case["height"], deme=case["deme"],
                    meta_width=case["meta_width"], meta_height=case["meta_height"],
                    meta_deme=case["meta_deme"], migration_probability=case["migration"])
        check_run(oracle, desc, case)


def test_almost_infinite_reference_runs(oracle, kat):
    """Circle origins (one wrapping across the plane's edge), Normal dispersal
    with clamp-and-round, singleton demes."""
    for case in kat["almost_infinite_runs"]:
        desc = dict(kind=oracle.ALMOST_INFINITE_NORMAL, speciation_probability=case["speciation"],
                    sigma=case["sigma"], radius=case["radius"], centre_x=case["centre"][0],
                    centre_y=case["centre"][1])
        check_run(oracle, desc, case)


def test_turnover_map_reference_runs(oracle, kat):
    """SpatiallyExplicit with a turnover map: each lineage's event times and
    its share of the water level follow its cell's rate (0.1 to 7.5)."""
    for case in kat["turnover_map_runs"]:
        desc = se_desc(oracle, case)
        desc["turnover_map"] = np.array(case["turnover"], dtype=np.float64)
        check_run(oracle, desc, case)


def test_clark2dt_reference_runs(oracle, kat):
    """AlmostInfinite with Clark2Dt dispersal, a fat tail (p = 0.5) and the
    pow-free case (p = 1), one circle wrapping across the plane's edge."""
    for case in kat["clark2dt_runs"]:
        desc = dict(kind=oracle.ALMOST_INFINITE_CLARK2DT, speciation_probability=case["speciation"],
                    shape_u=case["shape_u"], tail_p=case["tail_p"], radius=case["radius"],
                    centre_x=case["centre"][0], centre_y=case["centre"][1])
        check_run(oracle, desc, case)


def canonical_desc(oracle, case):
    """The scenario a canonical-schedule vector was generated on."""
    nu = case["speciation"]
    if case["case"] == "ns":
        return dict(kind=oracle.NON_SPATIAL, speciation_probability=nu, width=case["width"],
                    height=case["height"], deme=case["deme"])
    if case["case"] == "si":
        return dict(kind=oracle.SPATIALLY_IMPLICIT, speciation_probability=nu, width=case["width"],
                    height=case["height"], deme=case["deme"], meta_width=case["meta_width"],
                    meta_height=case["meta_height"], meta_deme=case["meta_deme"],
                    migration_probability=case["migration"])
    if case["case"] == "ai":
        return dict(kind=oracle.ALMOST_INFINITE_NORMAL, speciation_probability=nu, sigma=case["sigma"],
                    radius=case["radius"], centre_x=case["centre"][0], centre_y=case["centre"][1])
    if case["case"] == "wn":
        return wn_desc(oracle, case)
    desc = se_desc(oracle, case)
    if "turnover" in case:
        desc["turnover_map"] = np.array(case["turnover"], dtype=np.float64)
    return desc


def test_canonical_schedule_runs(oracle, kat):
    """The horizon-synchronised schedule the CUDA backend runs: per-round
    horizons from the live lineage count, each lineage advanced to the
    horizon, identical states merged keeping the smallest reference. Pins the
    step, round and merge counts as well as the speciation stream, with long
    rounds (step_slice_max 1024: one round) and short ones (10)."""
    for case in kat["canonical_runs"]:
        sampler = oracle.SAMPLER_EXP if case["sampler"] == "exp" else oracle.SAMPLER_POISSON
        r = oracle.simulate(canonical_desc(oracle, case), case["seed"], mode=oracle.MODE_CANONICAL,
                            step_slice=case["step_slice"], min_round_events=case["min_round_events"],
                            step_slice_max=case["step_slice_max"], event_time_sampler=sampler)
        assert (r.steps, r.n_rounds, r.n_dedup, r.time, r.biodiversity) == (
            case["steps"], case["rounds"], case["dedups"], case["time"], case["biodiversity"]), case["case"]
        got = [[int(e["gref"]), float(e["prior_time"]), float(e["event_time"]), int(e["x"]),
                int(e["y"]), int(e["index"])] for e in r.speciation]
        assert got == case["events"], case["case"]


def wn_desc(oracle, case, speciation=None):
    """A WrappingNoise scenario from a golden case."""
    return dict(kind=oracle.WRAPPING_NOISE, speciation_probability=case.get("speciation", speciation or 0.5),
                noise_seed=case["noise_seed"] if "noise_seed" in case else case["seed"], coverage=case["coverage"],
                scale=case["scale"], persistence=case["persistence"], octaves=case["octaves"],
                sample=tuple(case["sample"]), sigma=case.get("sigma", 1.0))


def test_wrapping_noise_values(oracle, kat):
    """OpenSimplex 2D with wrapping summed over octaves, at lattice corners,
    the plane's far edge and random points, for seeds including i64::MIN."""
    for case in kat["wrapping_noise"]:
        for x, y, v in case["points"]:
            got = oracle.wrapping_noise(case["seed"], case["scale"], case["persistence"], case["octaves"], x, y)
            assert got == v, (case["seed"], x, y)


def test_wrapping_noise_thresholds(oracle, kat):
    """The coverage quantile of 2^16 WyHash-drawn locations' noise, including
    coverage 0 and 1 (the ends of the sorted sample)."""
    for case in kat["wrapping_noise_thresholds"]:
        got = oracle.wrapping_noise_threshold(case["seed"], case["coverage"], case["scale"], case["persistence"],
                                              case["octaves"])
        assert got == case["threshold"], case


def test_wrapping_noise_self_dispersal(oracle, kat):
    for sigma, coverage, p in kat["wrapping_noise_self_dispersal"]:
        assert oracle.wrapping_noise_self_dispersal(sigma, coverage) == p


def test_wrapping_noise_origins(oracle, kat):
    """The rectangle origin sampler keeps the habitable cells in row-major
    order, here over a sample that wraps across the plane's edge."""
    for case in kat["wrapping_noise_origins"]:
        o = oracle.enumerate_origins(wn_desc(oracle, case))
        assert [[int(a), int(b)] for a, b in zip(o["x"], o["y"])] == case["origins"]
        assert list(o["gref"]) == [(y << 32) | x for x, y in case["origins"]]
        assert not o["index"].any()


def test_wrapping_noise_reference_runs(oracle, kat):
    """Full tiny WrappingNoise runs: approximate Normal dispersal with its
    rejection loop (the generator asserts that targets were rejected)."""
    for case in kat["wrapping_noise_runs"]:
        assert case["rejections"] > 0
        check_run(oracle, wn_desc(oracle, case), case)


def test_almost_infinite_rectangle_reference_runs(oracle, kat):
    """AlmostInfinite with the Rectangle sample (every location of the
    extent, one wrapping across the plane's edge; sigma 0 keeps every
    lineage in place)."""
    for case in kat["almost_infinite_rectangle_runs"]:
        desc = dict(kind=oracle.ALMOST_INFINITE_NORMAL, speciation_probability=case["speciation"],
                    sigma=case["sigma"], sample=tuple(case["sample"]))
        check_run(oracle, desc, case)


def _clark2dt_reference_cases():
    import json
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "clark2dt_cdf_inverse.json")) as f:
        return json.load(f)["cases"]


def test_clark2dt_cdf_inverse_matches_the_reference_test(oracle):
    """The reference's own golden bits for clark2dt::cdf_inverse
    (almost_infinite_clark2dt.rs test_cdf_inverse, extracted by
    golden/make_clark2dt_kat.py): the oracle's jump distance equals every one,
    and so does its dispersal displacement for draws that give the same u01
    and an angle of 2 pi (cos = 1, so dx is the jump itself)."""
    import struct
    cases = _clark2dt_reference_cases()
    assert len(cases) == 27
    for c in cases:
        want = int(c["expected_bits"], 16)
        got = oracle.clark2dt_cdf_inverse(c["u01"], c["shape_u"], c["tail_p"])
        assert struct.unpack("<Q", struct.pack("<d", got))[0] == want, c
        # u01 = (d0 >> 11) * 2^-53 exactly (every case's u01 is a multiple of 2^-53)
        d0 = int(c["u01"] * 2.0 ** 53) << 11
        draws = np.array([[d0, (1 << 64) - 1]], dtype=np.uint64)
        dx, dy = oracle.displacements(oracle.ALMOST_INFINITE_CLARK2DT, draws, c["shape_u"], c["tail_p"])
        assert dx.view(np.uint64)[0] == want, c
        assert abs(dy[0]) <= 1e-15 * max(1.0, got)
