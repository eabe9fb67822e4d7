"""The exponential event-time sampler (event_time_sampler/exp.rs, the
reference CUDA algorithm's) and its logarithm.

CPU: the shared ln (ln_dd.h) is the correctly rounded logarithm, checked
against 60-digit decimal arithmetic; the oracle's sampler equals a direct
restatement of exp.rs over the oracle's WyHash stream; its canonical and
reference schedules agree on species and distinct events.
GPU (marked): the device's three step regimes (warp-cooperative, per-lane
latency, per-lane throughput) and the resident kernel give the canonical
oracle's stream bit for bit.
"""
import math
from decimal import Decimal, getcontext

import numpy as np
import pytest

INV_PHI = 0x9E3779B97F4A7C15
MASK64 = (1 << 64) - 1


def correctly_rounded_ln(x):
    getcontext().prec = 60
    return float(Decimal(x).ln())  # Decimal(float) is exact; float(Decimal) rounds to nearest


def open_closed(draws):
    """rng.rs:86-93 sample_uniform_open_closed."""
    return ((draws >> np.uint64(11)) + np.uint64(1)).astype(np.float64) * 2.0 ** -53


def test_ln_is_correctly_rounded(oracle):
    rng = np.random.default_rng(5)
    x = open_closed(rng.integers(0, 2 ** 64, size=4000, dtype=np.uint64))
    edges = np.array([2.0 ** -53, 2.0 ** -52, 3 * 2.0 ** -53, 0.5, 0.5 - 2.0 ** -54, 0.5 + 2.0 ** -53,
                      math.sqrt(0.5), np.nextafter(math.sqrt(0.5), 0), np.nextafter(math.sqrt(0.5), 1),
                      1.0 - 2.0 ** -53, 1.0 - 2.0 ** -52, 1.0, 0.25, 0.1, 0.9248807839366053])
    x = np.concatenate([x, edges])
    got = oracle.ln(x)
    want = np.array([correctly_rounded_ln(float(v)) for v in x])
    bad = np.flatnonzero(got.view(np.uint64) != want.view(np.uint64))
    assert bad.size == 0, [(x[i].hex(), got[i], want[i]) for i in bad[:5]]
    assert got[-4] == 0.0  # ln(1) is +0.0, so -ln(1) / lambda is -0.0 and adds nothing


def test_ln_vs_system_log_rate(oracle):
    """The system libm's log is not correctly rounded everywhere: the rate of
    one-ulp differences on the sampler's input distribution is the only gap
    between this backend's Exp stream and a glibc-based run's."""
    rng = np.random.default_rng(9)
    x = open_closed(rng.integers(0, 2 ** 64, size=200_000, dtype=np.uint64))
    got = oracle.ln(x)
    sys_log = np.array([math.log(v) for v in x])
    diff = np.abs(got.view(np.int64) - sys_log.view(np.int64))
    assert diff.max() <= 1
    assert (diff != 0).mean() < 0.005


def restated_exp_next_event_time(oracle, seed, inj, time, lam, delta_t):
    """exp.rs:37-83 line by line over the oracle's WyHash stream."""
    time_step = int(math.floor(time / delta_t))
    event_time = float(time_step) * delta_t
    slice_end = float(time_step + 1) * delta_t
    stream = iter(oracle.wyhash_sequence(seed, inj, time_step, 4096))
    sub_index = 0
    while True:
        u = float(open_closed(np.uint64(next(stream))))
        event_time += -float(oracle.ln(np.array([u]))[0]) / lam
        sub_index = (sub_index + INV_PHI) & MASK64
        if event_time >= slice_end:
            time_step += 1
            sub_index = 0
            event_time = slice_end
            slice_end = float(time_step + 1) * delta_t
            stream = iter(oracle.wyhash_sequence(seed, inj, time_step, 4096))
        elif event_time > time:
            break
    return event_time, (time_step + sub_index) & MASK64


@pytest.mark.parametrize("lam,delta_t", [(0.5, 2.0), (0.5, 0.1), (0.5, 20.0), (3.0, 1.0)])
def test_oracle_sampler_matches_restatement(oracle, lam, delta_t):
    rng = np.random.default_rng(int(lam * 10 + delta_t * 100))
    for _ in range(40):
        seed = oracle.seed_from_u64(int(rng.integers(0, 2 ** 63)))
        inj = int(rng.integers(0, 2 ** 40))
        t = float(rng.choice([0.0, rng.uniform(0, 50), float(rng.integers(0, 25)) * delta_t]))
        got = oracle.exp_next_event_time(seed, inj, t, lam, delta_t)
        want = restated_exp_next_event_time(oracle, seed, inj, t, lam, delta_t)
        assert np.float64(got[0]).view(np.uint64) == np.float64(want[0]).view(np.uint64)
        assert got[1] == want[1]
        assert got[0] > t


def test_exp_differs_from_poisson(oracle):
    seed = oracle.seed_from_u64(3)
    assert oracle.exp_next_event_time(seed, 5, 1.0) != oracle.poisson_next_event_time(seed, 5, 1.0)


CPU_CASES = {
    "ns": (dict(kind=0, speciation_probability=0.02, width=6, height=5, deme=2), 3),
    "si": (dict(kind=1, speciation_probability=5e-3, width=20, height=10, deme=3, meta_width=300,
                meta_height=7, meta_deme=2, migration_probability=0.3), 6),
    "ai": (dict(kind=2, speciation_probability=5e-3, sigma=3.0, radius=6, centre_x=2,
                centre_y=0xFFFFFFFF - 1), 8),
}


@pytest.mark.parametrize("name", sorted(CPU_CASES))
def test_oracle_schedules_agree_with_exp(oracle, name):
    desc, seed = CPU_CASES[name]
    exp = oracle.SAMPLER_EXP
    c = oracle.simulate(desc, seed, mode=oracle.MODE_CANONICAL, step_slice=10, min_round_events=1 << 20,
                        step_slice_max=1024, event_time_sampler=exp)
    r = oracle.simulate(desc, seed, mode=oracle.MODE_REFERENCE, event_time_sampler=exp)
    assert c.biodiversity == r.biodiversity > 0
    assert np.array_equal(oracle.distinct_speciation_set(c.speciation),
                          oracle.distinct_speciation_set(r.speciation))
    p = oracle.simulate(desc, seed, mode=oracle.MODE_REFERENCE)
    assert not np.array_equal(oracle.distinct_speciation_set(p.speciation),
                              oracle.distinct_speciation_set(r.speciation))


def test_oracle_rejects_unknown_sampler(oracle):
    desc, seed = CPU_CASES["ns"]
    with pytest.raises(RuntimeError):
        oracle.simulate(desc, seed, event_time_sampler=2)


# ---- GPU parity ----
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


def se_desc(syn, w, h, nu, seed):
    hab = syn.habitat_map(w, h, 0.15, 20, seed)
    return dict(kind=3, speciation_probability=nu, width=w, height=h, habitat=hab,
                dispersal=syn.dispersal_map(hab, 2.0))


def check_exp(nb, syn, oracle, desc, seed, pause=None, reference=True, **kw):
    algo = nb.CUDA(event_time_sampler="exp", **kw)
    with nb.Simulation(syn.to_scenario(desc), desc["speciation_probability"], algo) as sim:
        g = sim.simulate(seed, pause_before=pause)
    c = oracle.simulate(desc, seed, mode=oracle.MODE_CANONICAL, step_slice=algo.step_slice,
                        min_round_events=algo.min_round_events, pause_before=pause,
                        step_slice_max=algo.step_slice_max, delta_t=algo.delta_t,
                        event_time_sampler=oracle.SAMPLER_EXP)
    assert same_stream(g.speciation, c.speciation)
    assert (g.steps, g.n_rounds, g.n_dedup, g.biodiversity) == (c.steps, c.n_rounds, c.n_dedup,
                                                                 c.biodiversity)
    assert np.float64(g.time).view(np.uint64) == np.float64(c.time).view(np.uint64)
    assert g.paused == (c.status == 1) and g.n_remaining == c.n_remaining
    if reference:
        r = oracle.simulate(desc, seed, mode=oracle.MODE_REFERENCE, pause_before=pause,
                            delta_t=algo.delta_t, event_time_sampler=oracle.SAMPLER_EXP)
        assert g.biodiversity == r.biodiversity
        assert np.array_equal(nb.distinct_speciation_set(g.speciation),
                              oracle.distinct_speciation_set(r.speciation))
    return g


GPU_CASES = {
    "ns_tiny": (dict(kind=0, speciation_probability=0.01, width=4, height=4, deme=2), 3),
    "ns_single": (dict(kind=0, speciation_probability=0.05, width=1, height=1, deme=1), 1),
    "ns_mid": (dict(kind=0, speciation_probability=0.002, width=60, height=50, deme=2), 12),
    "si": (dict(kind=1, speciation_probability=5e-3, width=20, height=10, deme=3, meta_width=300,
                meta_height=7, meta_deme=2, migration_probability=0.3), 6),
    "ai": (dict(kind=2, speciation_probability=1e-3, sigma=10.0, radius=30, centre_x=0xFFFFFFFF // 2,
                centre_y=0xFFFFFFFF // 2), 7),
    "ai_clark": (dict(kind=4, speciation_probability=2e-3, shape_u=1.0, tail_p=1.0, radius=12, centre_x=3,
                      centre_y=0xFFFFFFFF - 2), 11),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(GPU_CASES))
def test_gpu_exp_matches_oracle(nb, syn, oracle, name):
    desc, seed = GPU_CASES[name]
    check_exp(nb, syn, oracle, desc, seed)


@pytest.mark.gpu
def test_gpu_exp_spatially_explicit(nb, syn, oracle):
    check_exp(nb, syn, oracle, se_desc(syn, 16, 16, 1e-3, 2), 2)


@pytest.mark.gpu
@pytest.mark.parametrize("delta_t", [20.0, 0.25, 3.0])
def test_gpu_exp_bucket_widths(nb, syn, oracle, delta_t):
    """lambda * delta_t = 10 puts ~11 samples in a bucket: the warp search
    overflows its 8 samples per bucket and continues sequentially; 0.25
    leaves most buckets empty; 3.0 is not a power of two (t / delta_t is
    divided, not multiplied)."""
    desc, seed = GPU_CASES["ns_mid"]
    check_exp(nb, syn, oracle, desc, seed, delta_t=delta_t)


@pytest.mark.gpu
def test_gpu_exp_config1_full(nb, syn, oracle):
    """100k lineages: the throughput and latency regimes before the tail."""
    desc, seed = syn.config1()
    g = check_exp(nb, syn, oracle, desc, seed, reference=False)
    assert g.n_initial == 100_000


@pytest.mark.gpu
@pytest.mark.parametrize("pause", [5.0, 40.0])
def test_gpu_exp_pause(nb, syn, oracle, pause):
    desc, seed = GPU_CASES["ns_mid"]
    check_exp(nb, syn, oracle, desc, seed, pause=pause, reference=False)


@pytest.mark.gpu
def test_gpu_exp_resident_batch(nb, syn):
    sims = syn.config4(n_sims=5, max_local=2000)
    scen = [syn.to_scenario(d) for d, _ in sims]
    nus = [d["speciation_probability"] * 50 for d, _ in sims]
    seeds = [s for _, s in sims]
    a = nb.simulate_batch(scen, nus, seeds, nb.CUDA(resident=True, event_time_sampler="exp"), collect=True)
    b = nb.simulate_batch(scen, nus, seeds, nb.CUDA(resident=False, event_time_sampler="exp"), collect=True)
    p = nb.simulate_batch(scen, nus, seeds, nb.CUDA(), collect=True)
    for x, y, z in zip(a, b, p):
        assert same_stream(x.speciation, y.speciation)
        assert (x.steps, x.n_rounds, x.n_dedup, x.time) == (y.steps, y.n_rounds, y.n_dedup, y.time)
        assert not same_stream(x.speciation, z.speciation)


@pytest.mark.gpu
def test_gpu_exp_dispersal_events(nb, syn, oracle):
    desc, seed = (dict(kind=2, speciation_probability=2e-3, sigma=3.0, radius=15, centre_x=2,
                       centre_y=0xFFFFFFFF - 1), 8)
    algo = nb.CUDA(report_dispersal=True, event_time_sampler="exp")
    with nb.Simulation(syn.to_scenario(desc), desc["speciation_probability"], algo) as sim:
        g = sim.simulate(seed)
    c = oracle.simulate(desc, seed, mode=oracle.MODE_CANONICAL, step_slice=algo.step_slice,
                        min_round_events=algo.min_round_events, step_slice_max=algo.step_slice_max,
                        report_dispersal=True, dispersal_cap=g.n_dispersal + 16,
                        event_time_sampler=oracle.SAMPLER_EXP)
    assert g.n_dispersal == c.n_dispersal > 0
    for f in ("gref", "prior_time", "event_time", "x", "y", "index", "tx", "ty", "tindex"):
        x, y = g.dispersal[f], c.dispersal[f]
        if x.dtype.kind == "f":
            x, y = x.view(np.uint64), y.view(np.uint64)
        assert np.array_equal(x, y), f
    assert same_stream(g.speciation, c.speciation)


def test_python_rejects_unknown_sampler(nb):
    with pytest.raises(ValueError):
        nb._args_struct(nb.CUDA(event_time_sampler="geometric"))
    assert nb._args_struct(nb.CUDA(event_time_sampler="exp")).event_time_sampler == 1
    assert nb._args_struct(nb.CUDA()).event_time_sampler == 0


@pytest.mark.gpu
def test_gpu_rejects_unknown_sampler(nb, syn, monkeypatch):
    desc, seed = GPU_CASES["ns_tiny"]
    real = nb._args_struct

    def bad(algo):
        a = real(algo)
        a.event_time_sampler = 2
        return a

    monkeypatch.setattr(nb, "_args_struct", bad)
    with pytest.raises(nb.NecsimError) as e:
        nb.simulate_batch([syn.to_scenario(desc)], [0.01], [seed])
    assert e.value.code == -1
