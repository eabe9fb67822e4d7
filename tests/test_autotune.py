"""The launch autotuner: it times every candidate on a bounded sample and
its choice leaves the simulation results unchanged."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_picks_the_fastest_candidate_and_keeps_results(nb, syn):
    sims = syn.config4(n_sims=8, max_local=3000)
    scen = [syn.to_scenario(d) for d, _ in sims]
    nus = [d["speciation_probability"] for d, _ in sims]
    seeds = [s for _, s in sims]
    tuned, res = nb.autotune(scen, nus, seeds, sample_pause=300.0, max_sample_lineages=20000)
    assert len(res) == 18
    assert set(res["block_size"]) == {64, 128, 256} and set(res["dedup_factor_pct"]) == {200, 400}
    assert set(res["step_slice"]) == {10, 20, 40}
    assert np.all(res["ms"] > 0)
    i = int(np.argmin(res["ms"]))
    assert (tuned.block_size, tuned.step_slice, tuned.dedup_factor_pct) == \
        (int(res["block_size"][i]), int(res["step_slice"][i]), int(res["dedup_factor_pct"][i]))
    plain = nb.simulate_batch(scen, nus, seeds, nb.CUDA(), collect=True)
    tuned_out = nb.simulate_batch(scen, nus, seeds, tuned, collect=True)
    for a, b in zip(plain, tuned_out):
        assert a.biodiversity == b.biodiversity
        assert np.array_equal(nb.distinct_speciation_set(a.speciation), nb.distinct_speciation_set(b.speciation))
