"""Properties of the oracle's two schedules (CPU): the reference's
Monolithic schedule and the GPU's canonical schedule differ only in which
duplicate lineages are simulated, never in the species or the distinct
speciation events."""
import numpy as np
import pytest


def small_scenarios(syn):
    hab = syn.habitat_map(8, 8, 0.15, 6, 21)
    se = dict(kind=3, speciation_probability=2e-3, width=8, height=8, habitat=hab,
              dispersal=syn.dispersal_map(hab, 1.5))
    return {
        "non_spatial": (dict(kind=0, speciation_probability=2e-3, width=20, height=20, deme=5), 42),
        "spatially_implicit": (dict(kind=1, speciation_probability=1e-3, width=300, height=1,
                                    deme=2, meta_width=5000, meta_height=1, meta_deme=1,
                                    migration_probability=0.1), 5),
        "almost_infinite": (dict(kind=2, speciation_probability=2e-3, sigma=4.0, radius=12,
                                 centre_x=0xFFFFFFFF // 2, centre_y=0xFFFFFFFF // 2), 7),
        "spatially_explicit": (se, 1),
    }


@pytest.mark.parametrize("name", ["non_spatial", "spatially_implicit", "almost_infinite",
                                  "spatially_explicit"])
def test_schedules_agree_on_species(oracle, syn, name):
    desc, seed = small_scenarios(syn)[name]
    ref = oracle.simulate(desc, seed, mode=oracle.MODE_REFERENCE)
    for min_round in (0, 1 << 12):
        can = oracle.simulate(desc, seed, mode=oracle.MODE_CANONICAL, min_round_events=min_round)
        assert can.biodiversity == ref.biodiversity
        assert np.array_equal(oracle.distinct_speciation_set(can.speciation),
                              oracle.distinct_speciation_set(ref.speciation))
        assert can.time == ref.time
    assert ref.biodiversity == len(oracle.distinct_speciation_set(ref.speciation))


def test_dedup_none_keeps_species(oracle, syn):
    desc, seed = small_scenarios(syn)["non_spatial"]
    a = oracle.simulate(desc, seed, dedup_factor=1.0)
    b = oracle.simulate(desc, seed, dedup_factor=0.0)  # DedupCache::None
    assert b.steps >= a.steps
    assert a.biodiversity == b.biodiversity


def test_isolated_individuals_partitions_union(oracle, syn):
    """IsolatedIndividuals partitions (pre_sampler.rs:103-112) simulate
    disjoint origin subsets; their events together give the full set."""
    desc, seed = small_scenarios(syn)["non_spatial"]
    full = oracle.simulate(desc, seed)
    parts = [oracle.simulate(desc, seed, partition=(r, 3)) for r in range(3)]
    assert sum(p.n_initial for p in parts) == full.n_initial
    union = np.unique(np.concatenate([oracle.distinct_speciation_set(p.speciation)
                                      for p in parts]), axis=0)
    assert np.array_equal(union, oracle.distinct_speciation_set(full.speciation))


@pytest.mark.parametrize("mode", [0, 1])
def test_pause_resume_equals_straight_run(oracle, syn, mode):
    desc, seed = small_scenarios(syn)["non_spatial"]
    full = oracle.simulate(desc, seed, mode=mode)
    first = oracle.simulate(desc, seed, mode=mode, pause_before=300.0)
    assert first.status == 1 and first.n_remaining > 0
    rest = oracle.simulate(desc, seed, mode=mode, lineages=first.remaining, resume_time=300.0)
    both = np.unique(np.concatenate([oracle.distinct_speciation_set(first.speciation),
                                     oracle.distinct_speciation_set(rest.speciation)]), axis=0)
    assert np.array_equal(both, oracle.distinct_speciation_set(full.speciation))
    assert all(first.speciation["event_time"] < 300.0)


def test_speciation_probability_one(oracle):
    """nu = 1: every lineage speciates at its first event."""
    desc = dict(kind=0, speciation_probability=1.0, width=5, height=4, deme=3)
    r = oracle.simulate(desc, 9)
    assert r.steps == 60 and r.biodiversity == 60 and r.n_speciation == 60


def test_single_individual(oracle):
    desc = dict(kind=0, speciation_probability=0.05, width=1, height=1, deme=1)
    r = oracle.simulate(desc, 1)
    assert r.biodiversity == 1 and r.n_speciation == 1
