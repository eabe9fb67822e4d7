"""The learned lifetime scheduler: the MLP's gradients and predictions
against the fp64 oracle (oracle/mlp_oracle.py), training on traces the
backend generates itself, and outcomes that do not change when the trained
model reorders the step queue."""
import os

import numpy as np
import pytest

from oracle import mlp_oracle as mo

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    w = rng.normal(0.0, 0.3, mo.N_PARAMS)
    X = rng.random((40, mo.N_FEATURES))
    T = rng.random(40) * 5.0
    _, g = mo.loss_and_gradients(w, X, T)
    for i in [0, 7, 515, 600, 2000, 4671, 4700, 4740, 4800]:
        e = np.zeros_like(w)
        e[i] = 1e-6
        fd = (mo.loss_and_gradients(w + e, X, T)[0] - mo.loss_and_gradients(w - e, X, T)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i]))


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, -2.5, 3.14159], dtype=np.float32)
    assert mo.to_bf16(x).tolist() == [1.0, 1.0, 1.0078125, -2.5, 3.140625]


def test_model_layout_matches_header(nb):
    assert nb.MODEL_PARAMS == mo.N_PARAMS
    assert nb.MODEL_LAYOUT == mo.LAYOUT
    header = open(os.path.join(ROOT, "include", "necsim_b200.h")).read()
    assert "#define NECSIM_MODEL_PARAMS 4801" in header
    assert "#define NECSIM_MODEL_FEATURES 8" in header


@pytest.mark.gpu
def test_gradients_and_predictions_match_oracle(nb):
    rng = np.random.default_rng(1)
    with nb.LifetimeModel(seed=3) as m:
        # bf16-representable weights: the device computes with exactly these
        w = mo.to_bf16(rng.normal(0.0, 0.25, mo.N_PARAMS).astype(np.float32))
        m.weights = w
        assert np.array_equal(m.weights, w)
        X = rng.random((300, mo.N_FEATURES)).astype(np.float32)
        T = (rng.random(300) * 6.0).astype(np.float32)
        g, L = m.gradients(X, T)
        Lo, go = mo.loss_and_gradients(w.astype(np.float64), X.astype(np.float64), T.astype(np.float64))
        # fp32 accumulation against fp64: relative to the gradient's scale
        assert abs(L - Lo) <= 1e-5 * max(1.0, Lo)
        assert np.max(np.abs(g - go)) <= 2e-5 * np.max(np.abs(go))
        y = m.predict(X)
        yo = mo.forward(w.astype(np.float64), X.astype(np.float64))
        assert np.max(np.abs(y - yo)) <= 1e-4 * max(1.0, np.max(np.abs(yo)))


@pytest.mark.gpu
def test_training_fits_a_known_function(nb):
    rng = np.random.default_rng(2)
    X = rng.random((20000, mo.N_FEATURES)).astype(np.float32)
    T = (3.0 + 2.0 * X[:, 0] - 1.5 * X[:, 3] * X[:, 5] + np.sin(3.0 * X[:, 6])).astype(np.float32)
    with nb.LifetimeModel(seed=4) as m:
        losses = m.train(X, T, epochs=15, batch=512, lr=2e-3, seed=5)
        assert losses[-1] < 0.05 * losses[0]
        pred = m.predict(X[:2000])
        assert np.mean((pred - T[:2000]) ** 2) < 0.02


def _trace_workloads(syn):
    """Small versions of the trace sources: AlmostInfinite (radius 20) and a
    SpatiallyExplicit map (16 x 16)."""
    ai, _ = syn.config2(radius=20)
    ai = dict(ai, speciation_probability=1e-3)
    se, _ = syn.config3(width=16, height=16, map_seed=7)
    se = dict(se, speciation_probability=1e-3)
    return ai, se


@pytest.mark.gpu
def test_traces_train_a_model_that_beats_the_mean(nb, syn):
    # a sweep over the speciation probability (as in the batched sweeps),
    # each run to completion: a row's label is the remaining life of its
    # simulation, set mostly by the speciation probability and the time
    ai, se = _trace_workloads(syn)
    nus = [1e-2, 1e-3, 1e-4] * 2
    X, y = nb.collect_traces([syn.to_scenario(se)] * len(nus), nus, list(range(1, len(nus) + 1)),
                             snapshot_rounds=2, max_rows=60000)
    assert X.shape[0] > 1000 and X.shape[1] == mo.N_FEATURES
    assert np.all(np.isfinite(X)) and np.all(np.isfinite(y)) and np.all(y >= 0.0)
    rng = np.random.default_rng(0)
    idx = rng.permutation(X.shape[0])
    cut = int(0.8 * len(idx))
    tr, te = idx[:cut], idx[cut:]
    with nb.LifetimeModel(seed=7) as m:
        m.train(X[tr], y[tr], epochs=60, batch=256, lr=2e-3, seed=1)
        mse = float(np.mean((m.predict(X[te]) - y[te]) ** 2))
    # the gain over predicting every row's label by the mean
    var = float(np.var(y[te]))
    print(f"held-out MSE {mse:.4f} vs constant predictor {var:.4f} ({var / mse:.2f}x)")
    assert mse < 0.7 * var


@pytest.mark.gpu
@pytest.mark.parametrize("resident", [False, True])
def test_learned_schedule_is_bit_identical(nb, syn, resident):
    ai, se = _trace_workloads(syn)
    X, y = nb.collect_traces([syn.to_scenario(ai)], [ai["speciation_probability"]], [7],
                             snapshot_rounds=8, max_rows=20000)
    with nb.LifetimeModel(seed=9) as m:
        m.train(X, y, epochs=5, batch=1024, lr=2e-3, seed=2)
        sims = syn.config4(n_sims=6, max_local=3000)
        cases = [
            ([syn.to_scenario(d) for d, _ in sims], [d["speciation_probability"] for d, _ in sims],
             [s for _, s in sims]),
            ([syn.to_scenario(se)] * 2, [se["speciation_probability"]] * 2, [11, 12]),
            ([syn.to_scenario(ai)], [ai["speciation_probability"]], [7]),
        ]
        for scen, nus, seeds in cases:
            plain = nb.simulate_batch(scen, nus, seeds, nb.CUDA(resident=resident), collect=True)
            learned = nb.simulate_batch(scen, nus, seeds, nb.CUDA(resident=resident, schedule="learned", model=m),
                                        collect=True)
            for a, b in zip(plain, learned):
                assert (a.steps, a.biodiversity, a.n_speciation, a.n_dedup, a.time, a.n_rounds) == \
                       (b.steps, b.biodiversity, b.n_speciation, b.n_dedup, b.time, b.n_rounds)
                assert np.array_equal(a.speciation, b.speciation)


def test_learned_schedule_requires_a_model(nb):
    with pytest.raises(ValueError):
        nb._args_struct(nb.CUDA(schedule="learned"))
    with pytest.raises(ValueError):
        nb._args_struct(nb.CUDA(schedule="sorted"))


@pytest.mark.gpu
def test_priority_engine_model_against_unsorted_and_heuristics(nb, syn):
    """The benchmark's 256-simulation sweep ends when its longest-lived
    simulation does.  The learned schedule puts the model's 8 longest-lived
    simulations in a priority engine whose rounds wait for no other
    simulation; the arms compared are no priority engine (unsorted) and
    priority engines chosen by two closed-form estimates: nu * J and nu / ln J
    (the expected longest tail of ln J lineages that each speciate at rate
    nu).  Outcomes are identical in every arm.  A priority engine costs little
    when it misses the longest-lived simulation and shortens the sweep when
    it holds it."""
    import math

    import bench
    sims = syn.config4()
    n = len(sims)
    scen = [syn.to_scenario(d) for d, _ in sims]
    nus = [d["speciation_probability"] for d, _ in sims]
    seeds = [s for _, s in sims]
    J = [d["width"] * d["height"] for d, _ in sims]
    k = 8
    model, _ = bench.train_lifetime_model(nb, syn, 0, None)
    try:
        arms = {
            "unsorted": nb.CUDA(resident=True),
            "model": nb.CUDA(resident=True, schedule="learned", model=model, priority_sims=k),
            "nu*J": nb.CUDA(resident=True, priority_list=sorted(range(n), key=lambda j: nus[j] * J[j])[:k]),
            "nu/lnJ": nb.CUDA(resident=True, priority_list=sorted(range(n), key=lambda j: nus[j] / math.log(J[j]))[:k]),
            # the model's priority engine with its tails on 8 SMs of their own
            "model+sms": nb.CUDA(resident=True, schedule="learned", model=model, priority_sims=k, reserve_sms=8),
        }
        res = {}
        for name, algo in arms.items():
            with nb.Batch(scen, nus, seeds, algo) as b:
                b.run()
                ms = b.run()[0].total_ms
                res[name] = (ms, b.priority, b.run(collect=True))
    finally:
        model.close()
    base = res["unsorted"][2]
    for name, (_, _, outs) in res.items():
        for a, b in zip(base, outs):
            assert (a.steps, a.biodiversity, a.n_speciation, a.n_dedup, a.time, a.n_rounds) == \
                   (b.steps, b.biodiversity, b.n_speciation, b.n_dedup, b.time, b.n_rounds), name
            assert np.array_equal(np.sort(a.speciation), np.sort(b.speciation)), name
    longest = max(range(n), key=lambda j: base[j].time)
    t0 = res["unsorted"][0]
    for name, (ms, prio, _) in res.items():
        print("%-9s %8.1f ms (%.3f of unsorted)  priority engine %s  holds the longest-lived (#%d): %s" % (
            name, ms, ms / t0, prio, longest, longest in prio))
    for name, (ms, prio, _) in res.items():
        assert ms <= 1.05 * t0, name  # a priority engine that misses costs little
        if longest in prio:
            assert ms < 0.97 * t0, name  # one that holds the longest-lived simulation gains
    # the model ranks the simulations by predicted remaining life, not by nu * J
    assert longest in res["model"][1]
    if longest not in res["nu*J"][1]:
        assert res["model"][0] < res["nu*J"][0]



@pytest.mark.gpu
@pytest.mark.parametrize("reserve", [4, 16])
def test_reserved_sms_change_no_result(nb, syn, reserve):
    """A priority engine whose tails run on SMs of their own (the other
    engine's kernels leave those SMs, its own leave the rest, and the last
    block of a launch to leave takes the unclaimed work) gives the outcomes
    and speciation events of the run without the reservation, for both
    event-time samplers."""
    sims = syn.config4()[::16]
    scen = [syn.to_scenario(d) for d, _ in sims]
    nus = [d["speciation_probability"] * 10 for d, _ in sims]
    seeds = [s for _, s in sims]
    longest = sorted(range(len(sims)), key=lambda j: nus[j])[:3]
    for sampler in ("poisson", "exp"):
        outs = {}
        for r in (0, reserve):
            algo = nb.CUDA(resident=True, priority_list=longest, reserve_sms=r, event_time_sampler=sampler)
            with nb.Batch(scen, nus, seeds, algo) as b:
                assert sorted(b.priority) == sorted(longest)
                outs[r] = b.run(collect=True)
        for a, b in zip(outs[0], outs[reserve]):
            assert (a.steps, a.biodiversity, a.n_speciation, a.n_dedup, a.time, a.n_rounds) == \
                   (b.steps, b.biodiversity, b.n_speciation, b.n_dedup, b.time, b.n_rounds), sampler
            assert np.array_equal(np.sort(a.speciation), np.sort(b.speciation)), sampler
