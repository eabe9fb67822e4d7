"""The benchmark's integer-issue roofline: the round kernels' algorithmic
WyHash mixing work (wymum per event, from the oracle's prime and draw counts
on the canonical schedule the kernels run) against the measured rate of
independent wymum chains."""
import types

import pytest


def test_counts_per_event_from_the_reference_sample():
    import bench
    _, sims = bench.workload("c1")
    counts = {}
    ev, _ = bench.cpu_sample(sims, 30.0, 2, "poisson", counts)
    assert counts["steps"] == ev > 0
    primes, draws = counts["primes"] / ev, counts["draws"] / ev
    # a Poisson event re-primes once and searches 1-3 buckets; it draws the
    # Devroye sample, the event times and the event's own samples
    assert 2.0 < primes < 5.0 and 4.0 < draws < 10.0


def test_canonical_work_counts(nb):
    import bench
    _, sims = bench.workload("c1")
    w = bench.canonical_work(sims, nb.CUDA(), 30.0, 2, "poisson")
    assert w["steps"] > 0 and 2.0 < w["primes"] / w["steps"] < 5.0 and 4.0 < w["draws"] / w["steps"] < 10.0
    assert "1 of 1 simulation(s) to t=30" in w["sample"]


def test_roofline_entry_is_never_fatal(nb):
    import bench
    _, sims = bench.workload("c1")
    broken = types.SimpleNamespace(hash_peak=lambda device: (_ for _ in ()).throw(RuntimeError("no GPU")))
    out = bench.roofline_entry(broken, 0, sims, nb.CUDA(), 20.0, 2, "poisson", 1000, 1.0, 10, "c1")
    assert set(out) == {"error"} and "no GPU" in out["error"]


@pytest.mark.gpu
def test_hash_peak_and_roofline(nb):
    import bench
    peak = nb.hash_peak(0)
    assert 1e10 < peak < 1e14
    _, sims = bench.workload("c1")
    out = bench.roofline_entry(nb, 0, sims, nb.CUDA(), 30.0, 2, "poisson", 2_500_000, 10.0, 100, "c1")
    assert out["bound"] == "integer-issue" and 0.0 < out["frac"] < 1.5
    assert 10.0 < out["wymum_per_event"] < 20.0


def test_cpu_baseline_partitions_single_simulations():
    """The CPU leg spreads a simulation over threads with IsolatedIndividuals
    partitions when the workload has fewer simulations than threads."""
    import bench
    assert bench.cpu_partitions(256, 16) == 1 and bench.cpu_partitions(1, 8) == 8
    assert bench.cpu_partitions(3, 8) == 2 and bench.cpu_partitions(1, 1) == 1
    assert "8 IsolatedIndividuals partitions" in bench.cpu_sample_desc("c1", 400.0, 1, 8)
    assert "partitions" not in bench.cpu_sample_desc("c4", 400.0, 256, 16)
    _, sims = bench.workload("c1")
    one, _ = bench.cpu_sample(sims, 20.0, 1)
    split, _ = bench.cpu_sample(sims, 20.0, 4)
    assert split >= one > 0  # partitions re-simulate duplicates a monolithic run merges
