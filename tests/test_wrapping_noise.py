"""WrappingNoise (rustcoalescence/scenarios/src/wrapping_noise.rs) and the
Rectangle sample it shares with AlmostInfinite (almost_infinite/mod.rs:92-122).

CPU: the backend's host noise habitat (threshold, rectangle origins,
argument checks) against the golden vectors and the oracle.
GPU (marked): the whole simulation against the oracle's canonical schedule
bit for bit, and its species set against the reference schedule's.
"""
import numpy as np
import pytest

from test_gpu_parity import check, same_stream

M32 = 0xFFFFFFFF


def wn_desc(oracle, nu, noise_seed, coverage, scale, persistence, octaves, sample, sigma):
    return dict(kind=oracle.WRAPPING_NOISE, speciation_probability=nu, noise_seed=noise_seed, coverage=coverage,
                scale=scale, persistence=persistence, octaves=octaves, sample=tuple(sample), sigma=sigma)


def test_host_origins_match_golden_vectors(nb, syn, oracle, kat):
    """The rectangle sample's habitable cells, row-major, wrapping across
    the plane's edge: the backend's host noise and threshold against the
    independent restatement's."""
    for case in kat["wrapping_noise_origins"]:
        desc = wn_desc(oracle, 0.5, case["seed"], case["coverage"], case["scale"], case["persistence"],
                       case["octaves"], case["sample"], 1.0)
        o = nb.enumerate_origins(syn.to_scenario(desc))
        assert [[int(a), int(b)] for a, b in zip(o["x"], o["y"])] == case["origins"]
        assert list(o["gref"]) == [(y << 32) | x for x, y in case["origins"]]


@pytest.mark.parametrize("coverage", [0.0, 0.3, 0.999, 1.0])
def test_host_origins_match_oracle(nb, syn, oracle, coverage):
    """The default noise (16 octaves, scale 0.07) over a 40 x 25 sample at
    several coverages, including none and all of the plane."""
    desc = wn_desc(oracle, 0.5, 0, coverage, 0.07, 0.5, 16, (M32 - 9, 100, 40, 25), 2.0)
    o = nb.enumerate_origins(syn.to_scenario(desc))
    c = oracle.enumerate_origins(desc)
    assert np.array_equal(o["x"], c["x"]) and np.array_equal(o["y"], c["y"])
    assert np.array_equal(o["gref"], c["gref"])
    assert len(o) == {0.0: 0, 1.0: 1000}.get(coverage, len(c))


def test_host_origins_of_a_large_sample_match_oracle(nb, syn, oracle):
    """A sample large enough for the host's threaded habitat scan."""
    desc = wn_desc(oracle, 0.5, -3, 0.45, 0.3, 0.6, 3, (5, M32 - 100, 300, 250), 2.0)
    o = nb.enumerate_origins(syn.to_scenario(desc))
    c = oracle.enumerate_origins(desc)
    assert len(o) > 10000
    assert np.array_equal(o["x"], c["x"]) and np.array_equal(o["y"], c["y"])


@pytest.mark.parametrize("field,value", [("coverage", -0.1), ("coverage", 1.5), ("scale", 0.0), ("scale", 1.5),
                                         ("persistence", 0.0), ("octaves", 0), ("sigma", -1.0),
                                         ("sigma", float("inf"))])
def test_invalid_arguments_are_rejected(nb, syn, oracle, field, value):
    desc = wn_desc(oracle, 0.5, 0, 0.5, 0.07, 0.5, 2, (0, 0, 4, 4), 2.0)
    desc[field] = value
    with pytest.raises(nb.NecsimError) as e:
        nb.enumerate_origins(syn.to_scenario(desc))
    assert e.value.code == -1


def test_empty_sample_extent_is_rejected(nb):
    sc = nb.WrappingNoise(0, 0.5, 0.07, 0.5, 2, nb.Rectangle((0, 0), 0, 4), 2.0)
    with pytest.raises(nb.NecsimError):
        nb.enumerate_origins(sc)


GPU_CASES = {
    # name: (nu, noise_seed, coverage, scale, persistence, octaves, sample, sigma, seed)
    "default_noise": (0.02, 0, 0.5, 0.07, 0.5, 16, (1000, 2000, 24, 20), 3.0, 7),
    "sparse_habitat": (0.05, 3, 0.2, 0.1, 0.5, 4, (0, 0, 30, 30), 2.0, 11),
    "wrapping_sample": (0.05, -2, 0.7, 0.2, 0.7, 3, (M32 - 5, M32 - 4, 12, 10), 1.5, 12),
    "near_self_dispersal": (0.05, 9, 0.6, 0.05, 0.5, 2, (0, 0, 16, 16), 0.2, 13),
    "full_coverage": (0.03, 1, 1.0, 0.07, 0.5, 3, (7, 7, 20, 20), 4.0, 14),
    # ~38k lineages: the many-lineages-per-lane passes, then the sparse regimes
    "throughput": (0.1, 5, 0.5, 0.05, 0.5, 3, (0, 0, 300, 250), 2.0, 15),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(GPU_CASES))
def test_gpu_matches_oracle(nb, syn, oracle, name):
    nu, ns, cov, scale, pers, octv, sample, sigma, seed = GPU_CASES[name]
    desc = wn_desc(oracle, nu, ns, cov, scale, pers, octv, sample, sigma)
    g = check(nb, syn, oracle, desc, seed)
    assert g.steps > 0


@pytest.mark.gpu
def test_gpu_short_rounds_merge_duplicates_like_oracle(nb, syn, oracle):
    """Rounds of at most 10 events per lineage: lineages that met on a cell
    share their next event time there and merge (85 merges in the oracle)."""
    nu, ns, cov, scale, pers, octv, sample, sigma, seed = GPU_CASES["sparse_habitat"]
    desc = wn_desc(oracle, nu, ns, cov, scale, pers, octv, sample, sigma)
    g = check(nb, syn, oracle, desc, seed, algo=nb.CUDA(step_slice_max=10))
    assert g.n_dedup > 0 and g.n_rounds > 1


@pytest.mark.gpu
def test_gpu_matches_oracle_with_exponential_event_times(nb, syn, oracle):
    nu, ns, cov, scale, pers, octv, sample, sigma, seed = GPU_CASES["sparse_habitat"]
    desc = wn_desc(oracle, nu, ns, cov, scale, pers, octv, sample, sigma)
    algo = nb.CUDA(event_time_sampler="exp")
    g = nb.simulate(nu, syn.to_scenario(desc), seed, algo)
    c = oracle.simulate(desc, seed, mode=oracle.MODE_CANONICAL, step_slice=algo.step_slice,
                        min_round_events=algo.min_round_events, step_slice_max=algo.step_slice_max,
                        event_time_sampler=oracle.SAMPLER_EXP)
    assert (g.steps, g.n_rounds, g.n_dedup, g.biodiversity) == (c.steps, c.n_rounds, c.n_dedup, c.biodiversity)
    assert np.array_equal(nb.distinct_speciation_set(g.speciation), oracle.distinct_speciation_set(c.speciation))


@pytest.mark.gpu
def test_gpu_pause_and_resume_match_oracle(nb, syn, oracle):
    """Paused lineages resume where they stopped; resumed lineages on
    uninhabitable cells fail like the reference's ResumeError::Sample."""
    nu, ns, cov, scale, pers, octv, sample, sigma, seed = GPU_CASES["sparse_habitat"]
    desc = wn_desc(oracle, nu, ns, cov, scale, pers, octv, sample, sigma)
    g = check(nb, syn, oracle, desc, seed, pause=5.0)
    assert g.paused
    with nb.Simulation(syn.to_scenario(desc), nu, nb.CUDA()) as sim:
        rest = sim.resume(g.remaining, 5.0, seed)
    c = oracle.simulate(desc, seed, mode=oracle.MODE_CANONICAL, lineages=g.remaining, resume_time=5.0,
                        step_slice=10, min_round_events=1 << 20, step_slice_max=1024)
    assert same_stream(rest.speciation, c.speciation)
    assert rest.steps == c.steps and rest.biodiversity == c.biodiversity
    bad = g.remaining.copy()
    # a location the noise marks uninhabitable
    o = oracle.enumerate_origins(dict(desc, sample=(0, 0, 30, 30)))
    habitable = {(int(x), int(y)) for x, y in zip(o["x"], o["y"])}
    hole = next((x, y) for y in range(30) for x in range(30) if (x, y) not in habitable)
    bad["x"][0], bad["y"][0] = hole
    with nb.Simulation(syn.to_scenario(desc), nu, nb.CUDA()) as sim:
        with pytest.raises(nb.NecsimError) as e:
            sim.resume(bad, 5.0, seed)
    assert e.value.code == -1


def test_almost_infinite_rectangle_origins(nb, syn, oracle, kat):
    """Every location of the extent, row-major, wrapping at 2^32."""
    for case in kat["almost_infinite_rectangle_runs"]:
        desc = dict(kind=oracle.ALMOST_INFINITE_NORMAL, speciation_probability=case["speciation"],
                    sigma=case["sigma"], sample=tuple(case["sample"]))
        o = nb.enumerate_origins(syn.to_scenario(desc))
        c = oracle.enumerate_origins(desc)
        x, y, w, h = case["sample"]
        assert len(o) == w * h
        assert np.array_equal(o["x"], c["x"]) and np.array_equal(o["y"], c["y"])
        assert np.array_equal(o["gref"], c["gref"])
        assert (int(o["x"][-1]), int(o["y"][-1])) == ((x + w - 1) & M32, (y + h - 1) & M32)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [2, 4])
def test_gpu_almost_infinite_rectangle_matches_oracle(nb, syn, oracle, kind):
    desc = dict(kind=kind, speciation_probability=0.02, sample=(M32 - 10, 3, 30, 20))
    desc.update(dict(sigma=3.0) if kind == 2 else dict(shape_u=4.0, tail_p=0.5))
    check(nb, syn, oracle, desc, 21)
