"""GPU parity: the sm_100a backend against the oracle (marked gpu).

Bit-exact contract:
  * against the oracle's canonical schedule (the GPU's own schedule):
    the full delivered speciation stream (global reference, prior time,
    event time, origin), steps, time, rounds and dedup counts;
  * against the oracle's reference schedule (the reference's Monolithic
    Independent run): the species count and the sorted set of distinct
    speciation events (event-time bits, x, y, index).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

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


def run_gpu(nb, syn, desc, seed, algo=None, pause=None):
    algo = algo or nb.CUDA()
    with nb.Simulation(syn.to_scenario(desc), desc["speciation_probability"], algo) as sim:
        return sim.simulate(seed, pause_before=pause)


def check(nb, syn, oracle, desc, seed, algo=None, pause=None, reference=True):
    algo = algo or nb.CUDA()
    g = run_gpu(nb, syn, desc, seed, algo, pause)
    c = oracle.simulate(desc, seed, mode=oracle.MODE_CANONICAL, step_slice=algo.step_slice,
                        min_round_events=algo.min_round_events, pause_before=pause,
                        step_slice_max=algo.step_slice_max)
    assert same_stream(g.speciation, c.speciation)
    assert (g.steps, g.n_rounds, g.n_dedup, g.biodiversity) == (c.steps, c.n_rounds, c.n_dedup,
                                                                 c.biodiversity)
    assert np.float64(g.time).view(np.uint64) == np.float64(c.time).view(np.uint64)
    assert g.paused == (c.status == 1) and g.n_remaining == c.n_remaining
    if g.paused:
        rem = np.sort(g.remaining, order="gref")
        crem = np.sort(c.remaining, order="gref")
        for f in ("gref", "x", "y", "index"):
            assert np.array_equal(rem[f], crem[f])
        assert np.array_equal(rem["last_event_time"].view(np.uint64),
                              crem["last_event_time"].view(np.uint64))
    if reference:
        r = oracle.simulate(desc, seed, mode=oracle.MODE_REFERENCE, pause_before=pause)
        assert g.biodiversity == r.biodiversity
        assert np.array_equal(nb.distinct_speciation_set(g.speciation),
                              oracle.distinct_speciation_set(r.speciation))
    return g


def se_desc(syn, w, h, nu, seed, maxv=20, sigma=2.0):
    hab = syn.habitat_map(w, h, 0.15, maxv, seed)
    return dict(kind=3, speciation_probability=nu, width=w, height=h, habitat=hab,
                dispersal=syn.dispersal_map(hab, sigma))


CASES = {
    "ns_tiny": (dict(kind=0, speciation_probability=0.01, width=4, height=4, deme=2), 3),
    "ns_deme1": (dict(kind=0, speciation_probability=0.005, width=30, height=20, deme=1), 11),
    "ns_single": (dict(kind=0, speciation_probability=0.05, width=1, height=1, deme=1), 1),
    "ns_nu_one": (dict(kind=0, speciation_probability=1.0, width=10, height=10, deme=3), 2),
    "si": (dict(kind=1, speciation_probability=1e-3, width=1000, height=1, deme=1,
                meta_width=100000, meta_height=1, meta_deme=1, migration_probability=0.1), 5),
    "si_demes": (dict(kind=1, speciation_probability=5e-3, width=20, height=10, deme=3,
                      meta_width=300, meta_height=7, meta_deme=2, migration_probability=0.3), 6),
    "ai": (dict(kind=2, speciation_probability=1e-3, sigma=10.0, radius=30,
                centre_x=0xFFFFFFFF // 2, centre_y=0xFFFFFFFF // 2), 7),
    "ai_wrap": (dict(kind=2, speciation_probability=2e-3, sigma=3.0, radius=15, centre_x=2,
                     centre_y=0xFFFFFFFF - 1), 8),
    "ai_sigma0": (dict(kind=2, speciation_probability=0.01, sigma=0.0, radius=5, centre_x=100,
                       centre_y=100), 9),
    "ai_clark": (dict(kind=4, speciation_probability=1e-3, shape_u=4.0, tail_p=0.5, radius=25,
                      centre_x=0xFFFFFFFF // 2, centre_y=0xFFFFFFFF // 2), 10),
    "ai_clark_p1": (dict(kind=4, speciation_probability=2e-3, shape_u=1.0, tail_p=1.0, radius=12, centre_x=3,
                         centre_y=0xFFFFFFFF - 2), 11),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_small_scenarios(nb, syn, oracle, name):
    desc, seed = CASES[name]
    check(nb, syn, oracle, desc, seed)


@pytest.mark.parametrize("w,h,nu,seed", [(8, 8, 2e-3, 1), (16, 16, 1e-3, 2), (16, 8, 5e-3, 3)])
def test_spatially_explicit_small(nb, syn, oracle, w, h, nu, seed):
    check(nb, syn, oracle, se_desc(syn, w, h, nu, seed), seed)


def test_config1_nonspatial_full(nb, syn, oracle):
    desc, seed = syn.config1()
    g = check(nb, syn, oracle, desc, seed)
    assert g.n_initial == 100_000


def test_config3_spatially_explicit_full(nb, syn, oracle):
    desc, seed = syn.config3()
    check(nb, syn, oracle, desc, seed)


@pytest.mark.parametrize("algo_kw", [dict(min_round_events=1 << 12), dict(step_slice=3),
                                     dict(block_size=64, grid_size=7), dict(rounds_per_graph=2),
                                     dict(dedup_factor_pct=120)])
def test_launch_and_schedule_parameters(nb, syn, oracle, algo_kw):
    desc, seed = syn.config1()
    check(nb, syn, oracle, desc, seed, algo=nb.CUDA(**algo_kw), reference=False)


def test_launch_shape_does_not_change_output(nb, syn):
    """Block/grid size and graph length only reorder work: identical streams."""
    desc, seed = se_desc(syn, 16, 16, 1e-3, 4), 4
    outs = [run_gpu(nb, syn, desc, seed, nb.CUDA(block_size=b, grid_size=g, rounds_per_graph=r))
            for b, g, r in [(32, 1, 2), (128, 0, 16), (256, 3, 4)]]
    for o in outs[1:]:
        assert same_stream(o.speciation, outs[0].speciation)
        assert o.steps == outs[0].steps


@pytest.mark.parametrize("pause", [50.0, 500.0])
def test_pause(nb, syn, oracle, pause):
    desc, seed = syn.config1()
    g = check(nb, syn, oracle, desc, seed, pause=pause)
    assert g.paused and np.all(g.speciation["event_time"] < pause)


def test_pause_resume_equals_straight_run(nb, syn):
    desc, seed = CASES["ai"]
    with nb.Simulation(syn.to_scenario(desc), desc["speciation_probability"]) as sim:
        full = sim.simulate(seed)
        first = sim.simulate(seed, pause_before=400.0)
        rest = sim.resume(first.remaining, 400.0, seed)
    both = np.unique(np.concatenate([nb.distinct_speciation_set(first.speciation),
                                     nb.distinct_speciation_set(rest.speciation)]), axis=0)
    assert np.array_equal(both, nb.distinct_speciation_set(full.speciation))


def test_resume_matches_oracle(nb, syn, oracle):
    desc, seed = CASES["si_demes"]
    first = oracle.simulate(desc, seed, mode=oracle.MODE_CANONICAL, pause_before=100.0,
                            min_round_events=1 << 20, step_slice_max=1024)
    with nb.Simulation(syn.to_scenario(desc), desc["speciation_probability"]) as sim:
        g = sim.resume(first.remaining, 100.0, seed)
    c = oracle.simulate(desc, seed, mode=oracle.MODE_CANONICAL, lineages=first.remaining,
                        resume_time=100.0, min_round_events=1 << 20)
    assert same_stream(g.speciation, c.speciation)
    assert g.steps == c.steps and g.time == c.time


def test_batch_equals_single_runs(nb, syn):
    sims = syn.config4(n_sims=6, max_local=3000)
    scen = [syn.to_scenario(d) for d, _ in sims]
    nus = [d["speciation_probability"] * 100 for d, _ in sims]  # keep lifetimes short
    seeds = [s for _, s in sims]
    batch = nb.simulate_batch(scen, nus, seeds, collect=True)
    for j in range(len(sims)):
        single = nb.simulate(nus[j], scen[j], seeds[j])
        assert same_stream(batch[j].speciation, single.speciation)
        assert (batch[j].steps, batch[j].biodiversity, batch[j].n_rounds) == (
            single.steps, single.biodiversity, single.n_rounds)


def test_resident_kernel_matches_global_rounds(nb, syn):
    """Small simulations run in the per-simulation resident kernel; with it
    switched off they stay in the global rounds: identical output."""
    sims = syn.config4(n_sims=5, max_local=2000)
    scen = [syn.to_scenario(d) for d, _ in sims]
    nus = [d["speciation_probability"] * 50 for d, _ in sims]
    seeds = [s for _, s in sims]
    a = nb.simulate_batch(scen, nus, seeds, nb.CUDA(resident=True), collect=True)
    b = nb.simulate_batch(scen, nus, seeds, nb.CUDA(resident=False), collect=True)
    for x, y in zip(a, b):
        assert same_stream(x.speciation, y.speciation)
        assert (x.steps, x.n_rounds, x.n_dedup, x.time) == (y.steps, y.n_rounds, y.n_dedup, y.time)


# ---- dispersal events (ReportDispersal) ----
DISP_FIELDS = ("gref", "prior_time", "event_time", "x", "y", "index", "tx", "ty", "tindex")


def same_disp_stream(a, b):
    if len(a) != len(b):
        return False
    for f in DISP_FIELDS:
        x, y = a[f], b[f]
        if x.dtype.kind == "f":
            x, y = x.view(np.uint64), y.view(np.uint64)
        if not np.array_equal(x, y):
            return False
    return True


def packed_key(e, speciation):
    """PackedEvent::cmp key (event.rs:256-280); a speciation's target is its origin."""
    t = (int(e["tx"]), int(e["ty"]), int(e["tindex"])) if not speciation else (int(e["x"]), int(e["y"]),
                                                                               int(e["index"]))
    return (int(np.float64(e["event_time"]).view(np.uint64)), int(e["x"]), int(e["y"]), int(e["index"])) + t + \
        (int(np.float64(e["prior_time"]).view(np.uint64)), int(e["gref"]))


def interleaved(g):
    """The GPU's delivered stream, speciation and dispersal calls in order."""
    out, i, j = [], 0, 0
    for kind, n in g.delivery or []:
        for _ in range(n):
            if kind == "s":
                out.append(packed_key(g.speciation[i], True))
                i += 1
            else:
                out.append(packed_key(g.dispersal[j], False))
                j += 1
    return out


DISP_CASES = {
    "ns": (dict(kind=0, speciation_probability=0.01, width=12, height=10, deme=2), 3),
    "si": (dict(kind=1, speciation_probability=5e-3, width=20, height=10, deme=3,
                meta_width=300, meta_height=7, meta_deme=2, migration_probability=0.3), 6),
    "ai": (dict(kind=2, speciation_probability=2e-3, sigma=3.0, radius=15, centre_x=2,
                centre_y=0xFFFFFFFF - 1), 8),
}


@pytest.mark.parametrize("name", sorted(DISP_CASES) + ["se"])
def test_dispersal_events_match_canonical_oracle(nb, syn, oracle, name):
    desc, seed = DISP_CASES[name] if name != "se" else (se_desc(syn, 8, 8, 2e-3, 4), 4)
    algo = nb.CUDA(report_dispersal=True)
    g = run_gpu(nb, syn, desc, seed, algo)
    c = oracle.simulate(desc, seed, mode=oracle.MODE_CANONICAL, step_slice=algo.step_slice,
                        min_round_events=algo.min_round_events, step_slice_max=algo.step_slice_max,
                        report_dispersal=True, dispersal_cap=g.n_dispersal + 16)
    assert g.n_dispersal == c.n_dispersal > 0
    assert same_disp_stream(g.dispersal, c.dispersal)
    assert same_stream(g.speciation, c.speciation)
    assert (g.steps, g.n_rounds, g.n_dedup, g.biodiversity) == (c.steps, c.n_rounds, c.n_dedup, c.biodiversity)
    # the two kinds reach the reporter as one stream in PackedEvent order
    keys = interleaved(g)
    assert len(keys) == len(g.speciation) + len(g.dispersal)
    assert keys == sorted(keys)
    # and the run without dispersal reporting has the same outcome
    p = run_gpu(nb, syn, desc, seed)
    assert (p.steps, p.biodiversity, p.n_dedup) == (g.steps, g.biodiversity, g.n_dedup)
    assert same_stream(p.speciation, g.speciation)


def test_dispersal_events_batch_and_pause(nb, syn, oracle):
    sims = syn.config4(n_sims=3, max_local=400)
    scen = [syn.to_scenario(d) for d, _ in sims]
    nus = [d["speciation_probability"] for d, _ in sims]
    seeds = [s for _, s in sims]
    outs = nb.simulate_batch(scen, nus, seeds, nb.CUDA(report_dispersal=True), pause_before=3000.0, collect=True)
    for (d, s), g in zip(sims, outs):
        c = oracle.simulate(d, s, mode=oracle.MODE_CANONICAL, min_round_events=1 << 20, step_slice_max=1024,
                            report_dispersal=True, dispersal_cap=g.n_dispersal + 16, pause_before=3000.0)
        assert g.n_dispersal == c.n_dispersal
        assert same_disp_stream(g.dispersal, c.dispersal)
        assert same_stream(g.speciation, c.speciation)
        assert g.biodiversity == c.biodiversity and g.n_remaining == c.n_remaining


def test_priority_split_is_bit_identical(nb, syn):
    """Simulations in a priority engine of their own (priority_list), and
    the others in priority groups, give the same per-simulation results as
    the unsplit batch: every simulation's canonical schedule depends on that
    simulation only."""
    sims = syn.config4(n_sims=6, max_local=3000)
    scen = [syn.to_scenario(d) for d, _ in sims]
    nus = [d["speciation_probability"] * 50 for d, _ in sims]
    seeds = [s for _, s in sims]
    whole = nb.simulate_batch(scen, nus, seeds, collect=True)
    split = nb.simulate_batch(scen, nus, seeds, nb.CUDA(priority_list=[4, 1]), collect=True)
    with nb.Batch(scen, nus, seeds, nb.CUDA(priority_list=[0, 5, 2])) as b:
        assert b.priority == [0, 5, 2]
        b.run()
        again = b.run(collect=True)
    grouped = nb.simulate_batch(scen, nus, seeds, nb.CUDA(priority_list=[3], priority_groups=2, resident=True),
                                collect=True)
    for x, y, z, w in zip(whole, split, again, grouped):
        for o in (y, z, w):
            assert same_stream(x.speciation, o.speciation)
            assert (x.steps, x.n_rounds, x.n_dedup, x.biodiversity, x.time) == (
                o.steps, o.n_rounds, o.n_dedup, o.biodiversity, o.time)
    # the batch's device time spans its engines
    assert split[0].total_ms > 0 and split[0].n_launches > whole[0].n_launches


@pytest.mark.gpu
def test_batch_timeline_on_the_device_clock(nb, syn):
    """Every simulation of a batch reports when it ended (and when the
    resident kernel took it over) on the device clock, from the batch's first
    round: within the batch's span, hand-over before the end, the last end
    at the batch's end."""
    sims = syn.config4()[::16]
    scen = [syn.to_scenario(d) for d, _ in sims]
    nus = [d["speciation_probability"] * 10 for d, _ in sims]
    seeds = [s for _, s in sims]
    algo = nb.CUDA(resident=True, priority_list=[0, 1])
    with nb.Batch(scen, nus, seeds, algo) as b:
        b.run()
        outs = b.run()
    total = outs[0].total_ms
    for o in outs:
        assert 0.0 < o.end_ms <= total + 0.5
        assert o.routed_ms == -1.0 or 0.0 <= o.routed_ms <= o.end_ms
    assert any(o.routed_ms >= 0.0 for o in outs)
    assert max(o.end_ms for o in outs) >= 0.8 * total
    with nb.Simulation(scen[0], nus[0], nb.CUDA()) as sim:
        one = sim.simulate(seeds[0])
    assert 0.0 < one.end_ms <= one.total_ms + 0.5 and one.routed_ms == -1.0
