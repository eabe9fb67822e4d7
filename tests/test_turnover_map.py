"""SpatiallyExplicit with a turnover map (rustcoalescence/scenarios/src/
spatially_explicit/turnover/map.rs, InMemoryTurnoverRate): every cell's
turnover rate drives its lineages' event times (Poisson and exponential
samplers) and the reference schedule's water level.

CPU: the oracle with a map of one rate equals the uniform-rate run; its
canonical and reference schedules agree on species and distinct events; bad
maps are rejected.  GPU (marked): the backend equals the canonical oracle
bit for bit.
"""
import re
import subprocess

import numpy as np
import pytest

FIELDS = ("gref", "prior_time", "event_time", "x", "y", "index")


def same_stream(a, b):
    if len(a) != len(b):
        return False
    for f in FIELDS:
        x, y = a[f], b[f]
        if x.dtype.kind == "f":
            x, y = x.view(np.uint64), y.view(np.uint64)
        if not np.array_equal(x, y):
            return False
    return True


def map_desc(syn, w, h, nu, seed, uniform=None):
    hab = syn.habitat_map(w, h, 0.15, 12, seed)
    rng = np.random.default_rng(seed + 100)
    if uniform is None:
        turnover = rng.uniform(0.05, 3.0, size=(h, w))
        turnover[hab == 0] = rng.choice([0.0, 1.0], size=int((hab == 0).sum()))
    else:
        turnover = np.full((h, w), uniform)
    return dict(kind=3, speciation_probability=nu, width=w, height=h, habitat=hab,
                dispersal=syn.dispersal_map(hab, 2.0), turnover_map=turnover)


@pytest.mark.parametrize("mode", ["canonical", "reference"])
def test_oracle_map_of_one_rate_equals_uniform_rate(oracle, syn, mode):
    d = map_desc(syn, 12, 10, 5e-3, 4, uniform=0.5)
    u = dict(d)
    del u["turnover_map"]
    kw = dict(mode=oracle.MODE_CANONICAL, step_slice=10, min_round_events=1 << 20, step_slice_max=1024) \
        if mode == "canonical" else dict(mode=oracle.MODE_REFERENCE)
    a = oracle.simulate(d, 4, **kw)
    b = oracle.simulate(u, 4, **kw)
    assert same_stream(a.speciation, b.speciation) and a.steps == b.steps and a.biodiversity == b.biodiversity


@pytest.mark.parametrize("sampler", ["poisson", "exp"])
def test_oracle_schedules_agree_with_a_map(oracle, syn, sampler):
    code = oracle.SAMPLER_EXP if sampler == "exp" else oracle.SAMPLER_POISSON
    d = map_desc(syn, 12, 10, 5e-3, 5)
    c = oracle.simulate(d, 5, mode=oracle.MODE_CANONICAL, step_slice=10, min_round_events=1 << 20,
                        step_slice_max=1024, event_time_sampler=code)
    r = oracle.simulate(d, 5, mode=oracle.MODE_REFERENCE, event_time_sampler=code)
    assert c.biodiversity == r.biodiversity > 0
    assert np.array_equal(oracle.distinct_speciation_set(c.speciation), oracle.distinct_speciation_set(r.speciation))
    u = dict(d)
    del u["turnover_map"]
    p = oracle.simulate(u, 5, mode=oracle.MODE_REFERENCE, event_time_sampler=code)
    assert not np.array_equal(oracle.distinct_speciation_set(p.speciation), oracle.distinct_speciation_set(r.speciation))


def test_oracle_rejects_bad_maps(oracle, syn):
    d = map_desc(syn, 8, 6, 5e-3, 6)
    cell = tuple(np.argwhere(d["habitat"] > 0)[0])
    for value in (0.0, -1.0, np.nan, np.inf):
        bad = dict(d)
        bad["turnover_map"] = d["turnover_map"].copy()
        bad["turnover_map"][cell] = value
        with pytest.raises((RuntimeError, ValueError)):
            oracle.simulate(bad, 6)
    ns = dict(kind=0, speciation_probability=0.01, width=4, height=4, deme=1, turnover_map=np.ones((4, 4)))
    with pytest.raises((RuntimeError, ValueError)):
        oracle.simulate(ns, 1)


def test_driver_reads_a_turnover_map(nb, syn, tmp_path):
    import tiff_util
    d = map_desc(syn, 12, 10, 1e-3, 7)
    paths = {}
    for name, arr in (("habitat", d["habitat"].astype(np.uint32)), ("dispersal", d["dispersal"]),
                      ("turnover", d["turnover_map"])):
        paths[name] = tmp_path / (name + ".tif")
        tiff_util.write_tiff(str(paths[name]), arr, compression=5)
    cfg = """(
        speciation: 0.001, sample: Sample(percentage: 1.0, origin: Habitat, mode: Genesis), rng: Seed(7),
        algorithm: Independent(),
        scenario: SpatiallyExplicit(habitat: "%s", dispersal: "%s", turnover: Map("%s"), mode: Strict),
        reporters: [],
    )""" % (paths["habitat"], paths["dispersal"], paths["turnover"])
    (tmp_path / "c.ron").write_text(cfg)
    r = subprocess.run([nb.DRIVER, "check", str(tmp_path / "c.ron")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "turnover map" in r.stdout
    assert int(re.search(r"(\d+) lineages", r.stdout).group(1)) == int(d["habitat"].sum())
    tiff_util.write_tiff(str(paths["turnover"]), d["turnover_map"][:, :5])
    r = subprocess.run([nb.DRIVER, "check", str(tmp_path / "c.ron")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "dimensions" in r.stderr


def test_loading_with_a_turnover_map_path(nb, syn, tmp_path):
    import tiff_util
    d = map_desc(syn, 12, 10, 1e-3, 8)
    hab = d["habitat"].astype(np.uint32)
    turnover = d["turnover_map"].copy()
    cell = tuple(np.argwhere(hab > 0)[0])
    turnover[cell] = 0.0  # FixMe removes habitat where there is no turnover
    for name, arr in (("h", hab), ("d", d["dispersal"]), ("t", turnover)):
        tiff_util.write_tiff(str(tmp_path / (name + ".tif")), arr)
    sc = nb.spatially_explicit_from_maps(str(tmp_path / "h.tif"), str(tmp_path / "d.tif"),
                                         str(tmp_path / "t.tif"), mode="FixMe")
    assert sc.habitat[cell] == 0 and np.array_equal(sc.turnover, turnover)
    assert not sc.dispersal[cell[0] * 12 + cell[1]].any()


# ---- GPU ----
def check_map(nb, syn, oracle, desc, seed, sampler="poisson"):
    algo = nb.CUDA(event_time_sampler=sampler)
    code = oracle.SAMPLER_EXP if sampler == "exp" else oracle.SAMPLER_POISSON
    with nb.Simulation(syn.to_scenario(desc), desc["speciation_probability"], algo) as sim:
        g = sim.simulate(seed)
    c = oracle.simulate(desc, seed, mode=oracle.MODE_CANONICAL, step_slice=algo.step_slice,
                        min_round_events=algo.min_round_events, step_slice_max=algo.step_slice_max,
                        event_time_sampler=code)
    assert same_stream(g.speciation, c.speciation)
    assert (g.steps, g.n_rounds, g.n_dedup, g.biodiversity) == (c.steps, c.n_rounds, c.n_dedup, c.biodiversity)
    assert np.float64(g.time).view(np.uint64) == np.float64(c.time).view(np.uint64)
    r = oracle.simulate(desc, seed, mode=oracle.MODE_REFERENCE, event_time_sampler=code)
    assert g.biodiversity == r.biodiversity
    assert np.array_equal(nb.distinct_speciation_set(g.speciation), oracle.distinct_speciation_set(r.speciation))
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("sampler", ["poisson", "exp"])
@pytest.mark.parametrize("w,h,nu,seed", [(12, 10, 5e-3, 5), (24, 20, 1e-3, 9)])
def test_gpu_turnover_map_matches_oracle(nb, syn, oracle, sampler, w, h, nu, seed):
    check_map(nb, syn, oracle, map_desc(syn, w, h, nu, seed), seed, sampler)


@pytest.mark.gpu
def test_gpu_map_of_one_rate_equals_uniform_rate(nb, syn):
    d = map_desc(syn, 16, 12, 2e-3, 3, uniform=0.5)
    hab, disp = d["habitat"], d["dispersal"]
    a = nb.simulate(2e-3, nb.SpatiallyExplicit(hab, disp, d["turnover_map"]), 3)
    b = nb.simulate(2e-3, nb.SpatiallyExplicit(hab, disp, 0.5), 3)
    assert same_stream(a.speciation, b.speciation) and (a.steps, a.n_rounds) == (b.steps, b.n_rounds)


@pytest.mark.gpu
def test_gpu_batch_with_maps_equals_single_runs(nb, syn):
    descs = [map_desc(syn, 12, 10, 5e-3, s) for s in (11, 12, 13)]
    scen = [syn.to_scenario(d) for d in descs]
    nus = [d["speciation_probability"] for d in descs]
    batch = nb.simulate_batch(scen, nus, [11, 12, 13], collect=True)
    for j, sc in enumerate(scen):
        single = nb.simulate(nus[j], sc, 11 + j)
        assert same_stream(batch[j].speciation, single.speciation) and batch[j].steps == single.steps


@pytest.mark.gpu
def test_gpu_rejects_zero_turnover_on_habitat(nb, syn):
    d = map_desc(syn, 8, 6, 5e-3, 6)
    t = d["turnover_map"].copy()
    t[tuple(np.argwhere(d["habitat"] > 0)[0])] = 0.0
    with pytest.raises(nb.NecsimError) as e:
        nb.simulate(5e-3, nb.SpatiallyExplicit(d["habitat"], d["dispersal"], t), 6)
    assert e.value.code == -1 and "ZeroTurnoverHabitat" in str(e.value)
