"""Edge cases of the path against the oracle (GPU, marked): empty and
ragged inputs, a pause before any event, resumed lineages outside the
habitat or with an index beyond the deme (the resume fails, as the
reference's ResumeError::Sample), identical resumed lineages (merged by the
first dedup), a single-lineage simulation inside a batch of large ones, and
the documented size limit of the dispersal buffer."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("gref", "prior_time", "event_time", "x", "y", "index")
NS = dict(kind=0, speciation_probability=0.01, width=8, height=6, deme=3)


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


def canonical(oracle, algo, desc, seed, **kw):
    return oracle.simulate(desc, seed, mode=oracle.MODE_CANONICAL, step_slice=algo.step_slice,
                           min_round_events=algo.min_round_events, step_slice_max=algo.step_slice_max, **kw)


def test_empty_resume(nb, syn):
    with nb.Simulation(syn.to_scenario(NS), NS["speciation_probability"]) as sim:
        o = sim.resume(np.zeros(0, dtype=nb.LINEAGE_DTYPE), 5.0, 3)
    assert not o.paused and o.steps == 0 and o.biodiversity == 0 and o.n_remaining == 0
    assert len(o.speciation) == 0


def test_pause_before_any_event(nb, syn, oracle):
    algo = nb.CUDA()
    with nb.Simulation(syn.to_scenario(NS), NS["speciation_probability"], algo) as sim:
        g = sim.simulate(3, pause_before=0.0)
    c = canonical(oracle, algo, NS, 3, pause_before=0.0)
    assert g.paused and g.steps == 0 == c.steps and g.n_remaining == c.n_remaining == 8 * 6 * 3
    assert len(g.speciation) == 0


def test_resume_rejects_exceptional_lineages_and_merges_duplicates(nb, syn, oracle):
    algo = nb.CUDA(step_slice_max=10)  # short rounds: duplicates meet a dedup before they speciate
    origins = oracle.enumerate_origins(NS)
    lins = np.concatenate([origins[:20], origins[:5]]).copy()  # 5 identical pairs (new references)
    lins["gref"][20:] += 1000
    lins["last_event_time"] = 1.5
    with nb.Simulation(syn.to_scenario(NS), NS["speciation_probability"], algo) as sim:
        g = sim.resume(lins, 1.5, 9)
        # a lineage off the landscape or beyond its deme fails the resume
        # (initialiser/resume.rs:79-85, ResumeError::Sample)
        for x, y, i in ((8, 0, 0), (0, 6, 0), (3, 2, 3)):
            bad = lins.copy()
            bad[0]["x"], bad[0]["y"], bad[0]["index"] = x, y, i
            with pytest.raises(nb.NecsimError) as e:
                sim.resume(bad, 1.5, 9)
            assert e.value.code == -1 and "ResumeError::Sample" in str(e.value)
            with pytest.raises(RuntimeError):
                canonical(oracle, algo, NS, 9, lineages=bad, resume_time=1.5)
    c = canonical(oracle, algo, NS, 9, lineages=lins, resume_time=1.5)
    assert g.n_initial == c.n_initial == 25
    assert same_stream(g.speciation, c.speciation) and g.steps == c.steps and g.n_dedup == c.n_dedup >= 5


def test_single_lineage_simulation_in_a_ragged_batch(nb, syn):
    sims = syn.config4(n_sims=3, max_local=3000)
    # a batch shares one scenario kind: a SpatiallyImplicit local community of one individual
    one = dict(kind=1, speciation_probability=0.05, width=1, height=1, deme=1, meta_width=1000, meta_height=1,
               meta_deme=1, migration_probability=0.1)
    descs = [d for d, _ in sims] + [one]
    seeds = [s for _, s in sims] + [77]
    nus = [d["speciation_probability"] * 100 for d, _ in sims] + [0.05]
    scen = [syn.to_scenario(d) for d in descs]
    batch = nb.simulate_batch(scen, nus, seeds, collect=True)
    for j in range(len(descs)):
        single = nb.simulate(nus[j], scen[j], seeds[j])
        assert same_stream(batch[j].speciation, single.speciation) and batch[j].steps == single.steps
    assert batch[-1].n_initial == 1 and batch[-1].biodiversity == 1


def test_dispersal_buffer_limit(nb, syn):
    algo = nb.CUDA(report_dispersal=True, min_round_events=1 << 40)
    with pytest.raises(nb.NecsimError) as e:
        with nb.Simulation(syn.to_scenario(NS), NS["speciation_probability"], algo) as sim:
            sim.simulate(3)
    assert e.value.code == -10 and "16 GiB" in str(e.value)
