"""The rustcoalescence-style front end (`necsim-b200`, RON configuration)
and the origin pre-sampler it shares with the package."""
import math
import os
import re
import subprocess

import numpy as np
import pytest

INV_PHI = 6.180339887498949e-1


def presample_restated(n, p, rank=0, size=1):
    """OriginPreSampler::all().percentage(p).partition(rank, size)
    (origin_sampler/pre_sampler.rs:48-112), restated in Python."""
    sel = []
    if p >= 1.0:
        sel = list(range(n))
    elif p > 0.0:
        inv = 1.0 / math.log(1.0 - p)
        q, pos = 0.5, 0
        while pos < n:
            q += INV_PHI
            q -= math.floor(q)
            lq = math.log(q) if q > 0.0 else -math.inf
            skip = math.floor(lq * inv) if lq != -math.inf else math.inf
            if not skip < n - pos:
                break
            pos += int(skip)
            sel.append(pos)
            pos += 1
    return sel[rank::size]


@pytest.mark.parametrize("p", [0.0, 0.01, 0.1, 0.5, 0.9, 0.999, 1.0])
@pytest.mark.parametrize("rank,size", [(0, 1), (1, 3)])
def test_presample_matches_restatement(nb, p, rank, size):
    got = nb.presample_origins(5000, p, rank, size)
    assert got.tolist() == presample_restated(5000, p, rank, size)
    if p == 0.5 and size == 1:
        assert 2300 < len(got) < 2700


def run_driver(nb, mode, text, tmp_path, name="c.ron"):
    path = tmp_path / name
    path.write_text(text)
    return subprocess.run([nb.DRIVER, mode, str(path)], capture_output=True, text=True, timeout=600)


CONFIG = """(
    // a NonSpatial run with the reference's defaults spelled out
    speciation: 0.01,
    sample: Sample(percentage: 1.0, origin: Habitat, mode: Genesis),
    rng: Seed(42),
    pause: None,
    algorithm: Independent(
        delta_t: 2.0, step_slice: 10, dedup_cache: Relative(factor: 1.0),
        parallelism_mode: Monolithic(event_slice: Relative(factor: 2.0)),
    ),
    scenario: NonSpatial(area: (30, 20), deme: 2),
    reporters: [Plugin(library: "x.so", reporters: [Biodiversity(), Execution(), Counter()])],
)
"""


def test_check_parses_a_configuration(nb, tmp_path):
    r = run_driver(nb, "check", CONFIG, tmp_path)
    assert r.returncode == 0, r.stderr
    assert "NonSpatial(area: (30, 20), deme: 2)" in r.stdout and "1200 lineages" in r.stdout


@pytest.mark.parametrize("bad,msg", [
    ("speciation: 0.01,", "missing field `scenario`"),
    ("speciation: 0.01, scenario: NonSpatial(area: (3, 3), deme: 1), algorithm: Gillespie(),", "not the Independent"),
    ("speciation: 0.01, scenario: WrappingNoise(seed: 1),", "not supported"),
    ("speciation: 0.01 scenario: NonSpatial(area: (3, 3), deme: 1),", "expected ')'"),
    ("/* unterminated", "unterminated block comment"),
])
def test_check_rejects_bad_configurations(nb, tmp_path, bad, msg):
    r = run_driver(nb, "check", "(" + bad + ")", tmp_path)
    assert r.returncode == 1
    assert msg in r.stderr


def test_check_partition_and_sample(nb, tmp_path):
    cfg = CONFIG.replace("percentage: 1.0", "percentage: 0.5").replace(
        "Monolithic(event_slice: Relative(factor: 2.0))",
        "IsolatedIndividuals(partition: Partition(rank: 1, size: 2), event_slice: Relative(factor: 2.0))")
    r = run_driver(nb, "check", cfg, tmp_path)
    assert r.returncode == 0, r.stderr
    n = int(re.search(r"(\d+) lineages", r.stdout).group(1))
    assert n == len(presample_restated(1200, 0.5, 1, 2))


def species(out):
    m = re.search(r"biodiversity of (\d+) unique species", out)
    return int(m.group(1)) if m else 0


@pytest.mark.gpu
def test_driver_matches_the_package(nb, syn, oracle, tmp_path):
    r = run_driver(nb, "simulate", CONFIG, tmp_path)
    assert r.returncode == 0, r.stderr
    o = nb.simulate(0.01, nb.NonSpatial((30, 20), 2), 42)
    assert species(r.stdout) == o.biodiversity > 0
    assert "Event Summary" in r.stdout and "The simulation took" in r.stdout


@pytest.mark.gpu
def test_driver_sample_percentage_matches_oracle(nb, syn, oracle, tmp_path):
    cfg = CONFIG.replace("percentage: 1.0", "percentage: 0.3")
    r = run_driver(nb, "simulate", cfg, tmp_path)
    assert r.returncode == 0, r.stderr
    desc = dict(kind=0, speciation_probability=0.01, width=30, height=20, deme=2)
    lins = oracle.enumerate_origins(desc)[nb.presample_origins(1200, 0.3)]
    ref = oracle.simulate(desc, 42, mode=oracle.MODE_REFERENCE, lineages=lins)
    assert species(r.stdout) == ref.biodiversity > 0


@pytest.mark.gpu
def test_driver_pause_writes_a_resumable_config(nb, tmp_path):
    resume = tmp_path / "resume.ron"
    cfg = CONFIG.replace("pause: None", 'pause: Pause(before: 150.0, config: "%s", destiny: List)' % resume)
    r = run_driver(nb, "simulate", cfg, tmp_path, "p.ron")
    assert r.returncode == 0, r.stderr
    assert "paused" in r.stdout and resume.exists()
    first = species(r.stdout)
    r2 = subprocess.run([nb.DRIVER, "simulate", str(resume)], capture_output=True, text=True, timeout=600)
    assert r2.returncode == 0, r2.stderr
    assert "(resumed)" in r2.stdout and "done" in r2.stdout
    straight = nb.simulate(0.01, nb.NonSpatial((30, 20), 2), 42)
    assert first + species(r2.stdout) == straight.biodiversity


@pytest.mark.gpu
def test_driver_writes_an_event_log(nb, tmp_path):
    logdir = tmp_path / "events"
    cfg = CONFIG.replace("pause: None,", 'pause: None,\n    log: EventLog(directory: "%s", capacity: 5000),' % logdir)
    r = run_driver(nb, "simulate", cfg, tmp_path, "l.ron")
    assert r.returncode == 0, r.stderr
    headers, ev = nb.read_event_log(str(logdir))
    n_spec = int((ev["kind"] == 0).sum())
    assert n_spec > 0 and int((ev["kind"] == 2).sum()) > 0  # Counter() turns on dispersal events
    assert len({(int(e["x"]), int(e["y"]), int(e["index"]), float(e["event_time"]))
                for e in ev[ev["kind"] == 0]}) == species(r.stdout)
