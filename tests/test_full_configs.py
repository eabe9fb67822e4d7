"""Parity at the benchmark configurations' full sizes (marked gpu).

  C2  AlmostInfinite circle r = 100, Normal sigma = 10, nu = 1e-5, seed 7, to
      completion: the GPU equals the canonical oracle on the whole speciation
      stream, steps, rounds, duplicates and time, and the reference-schedule
      oracle on the distinct speciation set and the species count.  The
      Normal displacements pass the device's f64 log/sin/cos where the oracle
      (like the reference) calls the C library; `test_box_muller_device_vs_libm`
      measures how often the two disagree before rounding and checks that no
      disagreement changes a rounded target.
  C4  the 256-simulation SpatiallyImplicit sweep paused at t = 400, every
      simulation against the canonical oracle; the 24 simulations with the
      largest speciation probability run to completion against both oracle
      modes.
  C5  SpatiallyExplicit 128x128 with the dense 16384^2 map, paused at
      t = 400 and to completion, against both oracle modes (the survey's
      fixed-horizon comparison and the full run).

The oracle runs are spread over the host's cores (ctypes releases the GIL).
"""
import concurrent.futures
import os

import numpy as np
import pytest

from test_gpu_parity import same_stream

pytestmark = pytest.mark.gpu

THREADS = max(1, min(32, os.cpu_count() or 1))
CANON = dict(min_round_events=1 << 20, step_slice_max=1024)


def same_time(a, b):
    return np.float64(a).view(np.uint64) == np.float64(b).view(np.uint64)


def same_remaining(g, c):
    rem = np.sort(g.remaining, order="gref")
    crem = np.sort(c.remaining, order="gref")
    for f in ("gref", "x", "y", "index"):
        if not np.array_equal(rem[f], crem[f]):
            return False
    return np.array_equal(rem["last_event_time"].view(np.uint64), crem["last_event_time"].view(np.uint64))


def parallel(fn, items):
    with concurrent.futures.ThreadPoolExecutor(max_workers=THREADS) as ex:
        return list(ex.map(fn, items))


def assert_canonical(g, c):
    assert same_stream(g.speciation, c.speciation)
    assert (g.steps, g.n_rounds, g.n_dedup, g.biodiversity) == (c.steps, c.n_rounds, c.n_dedup, c.biodiversity)
    assert same_time(g.time, c.time)
    assert g.paused == (c.status == 1) and g.n_remaining == c.n_remaining


def assert_reference(nb, oracle, g, r):
    assert g.biodiversity == r.biodiversity
    assert np.array_equal(nb.distinct_speciation_set(g.speciation), oracle.distinct_speciation_set(r.speciation))


# ---- C2 ----

def test_config2_almost_infinite_full(nb, syn, oracle):
    desc, seed = syn.config2()
    with nb.Simulation(syn.to_scenario(desc), desc["speciation_probability"], nb.CUDA()) as sim:
        g = sim.simulate(seed)
    assert g.n_initial == 31_417
    c, r = parallel(lambda mode: oracle.simulate(desc, seed, mode=mode, **CANON),
                    [oracle.MODE_CANONICAL, oracle.MODE_REFERENCE])
    assert_canonical(g, c)
    assert_reference(nb, oracle, g, r)


@pytest.mark.parametrize("dispersal", ["normal", "clark2dt"])
def test_box_muller_device_vs_libm(nb, syn, oracle, dispersal):
    """C2's dispersal draws (2.66e7 events, uniform u64 sample pairs from a
    seeded stream) through the device's displacement arithmetic and the
    C library's: the raw f64 values may differ in the last bits (CUDA's and
    glibc's log/sin/cos/pow round differently), but no difference may cross
    a rounding boundary of clamp_round_dispersal (almost_infinite.rs:100-114),
    so every rounded target agrees."""
    n = 26_600_000
    draws = np.stack([syn.splitmix64(7, n, 0), syn.splitmix64(7, n, 1)], axis=1)
    if dispersal == "normal":
        disp, kind, a, b = nb.Normal(10.0), oracle.ALMOST_INFINITE_NORMAL, 10.0, 0.0
    else:
        disp, kind, a, b = nb.Clark2Dt(4.0, 0.5), oracle.ALMOST_INFINITE_CLARK2DT, 4.0, 0.5
    gx, gy = nb.displacements(draws, disp)
    cx, cy = oracle.displacements(kind, draws, a, b)
    differ = (gx.view(np.uint64) != cx.view(np.uint64)) | (gy.view(np.uint64) != cy.view(np.uint64))
    ulps = np.maximum(np.abs(gx - cx) / np.spacing(np.abs(cx)), np.abs(gy - cy) / np.spacing(np.abs(cy)))
    print("%s: %d of %d displacement pairs differ in their bits (%.3g%%), by at most %.0f ulp" % (
        dispersal, int(differ.sum()), n, 100 * float(differ.mean()), float(ulps.max())))
    flips = int(np.count_nonzero((rust_round(gx) != rust_round(cx)) | (rust_round(gy) != rust_round(cy))))
    assert flips == 0, "%d rounded targets differ" % flips
    # the differences are rounding differences of the last bits
    assert np.all(np.abs(gx - cx) <= 1e-12 * np.abs(cx)) and np.all(np.abs(gy - cy) <= 1e-12 * np.abs(cy))


def test_clark2dt_device_jump_against_the_reference_test(nb):
    """The reference's golden bits for clark2dt::cdf_inverse
    (almost_infinite_clark2dt.rs test_cdf_inverse; tests/golden) through the
    device's displacement arithmetic: draws giving each case's u01 and an
    angle of 2 pi, so dx is the jump.  CUDA's pow and cos may round the last
    bit differently from the C library the reference calls; the number of
    bit-exact cases is printed and every value is within 1e-12 relative."""
    import json
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "clark2dt_cdf_inverse.json")) as f:
        cases = json.load(f)["cases"]
    exact = 0
    for c in cases:
        d0 = int(c["u01"] * 2.0 ** 53) << 11
        draws = np.array([[d0, (1 << 64) - 1]], dtype=np.uint64)
        dx, dy = nb.displacements(draws, nb.Clark2Dt(c["shape_u"], c["tail_p"]))
        want = c["expected"]
        exact += int(dx.view(np.uint64)[0] == int(c["expected_bits"], 16))
        assert abs(dx[0] - want) <= 1e-12 * abs(want), c
        assert abs(dy[0]) <= 1e-12 * max(1.0, abs(want)), c
    print("device jump bit-exact with the reference's test in %d of %d cases" % (exact, len(cases)))


def rust_round(v):
    """f64::round: to the nearest integer, halves away from zero (exact:
    the fraction v - trunc(v) is computed without rounding)."""
    t = np.trunc(v)
    return t + np.where(np.abs(v - t) >= 0.5, np.sign(v), 0.0)


# ---- C4 ----

@pytest.fixture(scope="module")
def sweep(nb, syn):
    sims = syn.config4()
    scen = [syn.to_scenario(d) for d, _ in sims]
    nus = [d["speciation_probability"] for d, _ in sims]
    seeds = [s for _, s in sims]
    return sims, scen, nus, seeds


def test_config4_sweep_paused_every_simulation(nb, oracle, sweep):
    sims, scen, nus, seeds = sweep
    pause = 400.0
    outs = nb.simulate_batch(scen, nus, seeds, nb.CUDA(), pause_before=pause, collect=True)
    assert len(outs) == 256

    def one(j):
        d, s = sims[j]
        c = oracle.simulate(d, s, mode=oracle.MODE_CANONICAL, pause_before=pause, **CANON)
        g = outs[j]
        ok = (same_stream(g.speciation, c.speciation) and
              (g.steps, g.n_rounds, g.n_dedup, g.biodiversity, g.n_remaining) ==
              (c.steps, c.n_rounds, c.n_dedup, c.biodiversity, c.n_remaining) and
              same_time(g.time, c.time) and g.paused and c.status == 1)
        return j, ok, c.steps

    res = parallel(one, range(len(sims)))
    bad = [j for j, ok, _ in res if not ok]
    assert not bad, "simulations differing from the canonical oracle: %s" % bad
    assert sum(st for _, _, st in res) == sum(o.steps for o in outs)


def test_config4_largest_speciation_to_completion(nb, oracle, sweep):
    sims, scen, nus, seeds = sweep
    pick = sorted(range(len(sims)), key=lambda j: -nus[j])[:24]
    outs = nb.simulate_batch([scen[j] for j in pick], [nus[j] for j in pick], [seeds[j] for j in pick],
                             nb.CUDA(), collect=True)

    def one(k):
        d, s = sims[pick[k]]
        c = oracle.simulate(d, s, mode=oracle.MODE_CANONICAL, **CANON)
        r = oracle.simulate(d, s, mode=oracle.MODE_REFERENCE)
        return c, r

    for g, (c, r) in zip(outs, parallel(one, range(len(pick)))):
        assert_canonical(g, c)
        assert_reference(nb, oracle, g, r)


# ---- C5 ----

@pytest.fixture(scope="module")
def config5(syn):
    return syn.config5()


@pytest.mark.parametrize("pause", [400.0, None])
def test_config5_spatially_explicit(nb, syn, oracle, config5, pause):
    desc, seed = config5
    with nb.Simulation(syn.to_scenario(desc), desc["speciation_probability"], nb.CUDA()) as sim:
        g = sim.simulate(seed, pause_before=pause)
    c, r = parallel(lambda mode: oracle.simulate(desc, seed, mode=mode, pause_before=pause, **CANON),
                    [oracle.MODE_CANONICAL, oracle.MODE_REFERENCE])
    assert_canonical(g, c)
    assert_reference(nb, oracle, g, r)
    if pause is not None:
        assert g.paused and same_remaining(g, c)
        assert np.all(g.speciation["event_time"] < pause)
