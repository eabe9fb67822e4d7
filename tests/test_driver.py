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
    ("speciation: 0.01, scenario: WrappingNoise(seed: 1),", "missing field `coverage`"),
    ("speciation: 0.01, scenario: Torus(size: 1),", "not supported"),
    ("speciation: 0.01, scenario: WrappingNoise(seed: 99999999999999999999, coverage: 0.5, scale: 0.1, "
     "persistence: 0.5, octaves: 1, sample: Rectangle(origin: (x: 0, y: 0), width: 2, height: 2), sigma: 1.0),",
     "malformed i64"),
    ("speciation: 0.01, scenario: AlmostInfinite(sample: Rectangle(origin: (x: 0, y: 0), width: 0, height: 2), "
     "dispersal: Normal(sigma: 1.0)),", "width and height must be in 1..=2^32"),
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


CUDA_CONFIG = CONFIG.replace("""    algorithm: Independent(
        delta_t: 2.0, step_slice: 10, dedup_cache: Relative(factor: 1.0),
        parallelism_mode: Monolithic(event_slice: Relative(factor: 2.0)),
    ),""", """    algorithm: CUDA(ptx_jit: true, block_size: 64, grid_size: 64),""")


def test_check_reports_the_event_time_sampler(nb, tmp_path):
    r = run_driver(nb, "check", CONFIG, tmp_path)
    assert "algorithm Independent, Poisson event times, delta_t 2, step_slice 10" in r.stdout
    assert CUDA_CONFIG != CONFIG
    r = run_driver(nb, "check", CUDA_CONFIG, tmp_path)
    assert r.returncode == 0, r.stderr
    # the reference CUDA algorithm: ExpEventTimeSampler, delta_t 3.0, step_slice 150
    assert "algorithm CUDA, exponential event times, delta_t 3, step_slice 150" in r.stdout


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
    # `replay` of the log through the same reporters reports the same species
    rep = tmp_path / "replay.ron"
    rep.write_text('(log: EventLog(segments: ["%s/*"]), reporters: [Plugin(library: "x.so", '
                   'reporters: [Biodiversity(), Counter()])])' % logdir)
    r2 = subprocess.run([nb.DRIVER, "replay", str(rep)], capture_output=True, text=True, timeout=600)
    assert r2.returncode == 0, r2.stderr
    assert species(r2.stdout) == species(r.stdout) > 0


@pytest.mark.gpu
def test_driver_cuda_algorithm_runs_exponential_event_times(nb, oracle, tmp_path):
    r = run_driver(nb, "simulate", CUDA_CONFIG, tmp_path, "cuda.ron")
    assert r.returncode == 0, r.stderr
    desc = dict(kind=0, speciation_probability=0.01, width=30, height=20, deme=2)
    ref = oracle.simulate(desc, 42, mode=oracle.MODE_REFERENCE, delta_t=3.0, step_slice=150,
                          event_time_sampler=oracle.SAMPLER_EXP)
    assert species(r.stdout) == ref.biodiversity > 0
    o = nb.simulate(0.01, nb.NonSpatial((30, 20), 2), 42,
                    nb.CUDA(event_time_sampler="exp", delta_t=3.0, step_slice=150))
    assert o.biodiversity == ref.biodiversity


# ---- SpatiallyExplicit maps from (Geo)TIFF files ----
def se_tiffs(tmp_path, syn, w=12, h=10, seed=5):
    import tiff_util
    hab = syn.habitat_map(w, h, 0.15, 20, seed)
    disp = syn.dispersal_map(hab, 2.0)
    # a habitable cell stored as 0 (an off-by-one rounding in the map):
    # OffByOne restores it to 1 because dispersal leaves it
    stored = hab.astype(np.uint32).copy()
    c = np.flatnonzero(hab.reshape(-1) > 1)[0]
    stored.reshape(-1)[c] = 0
    hp, dp = tmp_path / "habitat.tif", tmp_path / "dispersal.tif"
    tiff_util.write_tiff(str(hp), stored, compression=5)
    tiff_util.write_tiff(str(dp), disp.astype(np.float64), compression=8, predictor=2)
    return hp, dp, stored, disp


SE_CONFIG = """(
    speciation: 0.001,
    sample: Sample(percentage: 1.0, origin: Habitat, mode: Genesis),
    rng: Seed(7),
    algorithm: Independent(),
    scenario: SpatiallyExplicit(habitat: "%s", dispersal: "%s", turnover: Uniform(0.5)%s),
    reporters: [Plugin(library: "x.so", reporters: [Biodiversity()])],
)
"""


def test_check_reads_tiff_maps(nb, syn, tmp_path):
    hp, dp, hab, disp = se_tiffs(tmp_path, syn)
    fixed, _ = nb.fix_maps(hab, disp, None, "OffByOne")
    changed = np.flatnonzero(fixed != hab)
    assert len(changed) == 1 and fixed.reshape(-1)[changed[0]] == 1 and hab.reshape(-1)[changed[0]] == 0
    r = run_driver(nb, "check", SE_CONFIG % (hp, dp, ""), tmp_path)
    assert r.returncode == 0, r.stderr
    assert "SpatiallyExplicit(12x10 map" in r.stdout
    assert "%d lineages" % int(fixed.sum()) in r.stdout
    r = run_driver(nb, "check", SE_CONFIG % (hp, dp, ", mode: Strict"), tmp_path)
    assert "%d lineages" % int(hab.sum()) in r.stdout
    for extra, msg in ((", mode: Lenient", "FixMe, OffByOne or Strict"),):
        r = run_driver(nb, "check", SE_CONFIG % (hp, dp, extra), tmp_path)
        assert r.returncode == 1 and msg in r.stderr
    r = run_driver(nb, "check", (SE_CONFIG % (hp, dp, "")).replace("Uniform(0.5)", 'Map("t.tif")'), tmp_path)
    assert r.returncode == 1 and "could not read file t.tif" in r.stderr  # a missing turnover map
    r = run_driver(nb, "check", SE_CONFIG % (dp, hp, ""), tmp_path)  # maps swapped: wrong bit widths
    assert r.returncode == 1 and "bitwidth" in r.stderr


REF_MAPS = os.environ.get("NECSIM_REFERENCE_MAPS", "")


@pytest.mark.skipif(not REF_MAPS or not os.path.isdir(os.path.join(REF_MAPS, "test")),
                    reason="set NECSIM_REFERENCE_MAPS to the reference's maps/ folder")
def test_check_reads_the_reference_fixture(nb, tmp_path):
    cfg = (SE_CONFIG % (os.path.join(REF_MAPS, "test", "habitat.tif"), os.path.join(REF_MAPS, "test", "dispersal.tif"), "")
           ).replace("percentage: 1.0", "percentage: 0.01")
    r = run_driver(nb, "check", cfg, tmp_path)
    assert r.returncode == 0, r.stderr
    assert "SpatiallyExplicit(35x41 map" in r.stdout
    n = int(re.search(r"(\d+) lineages", r.stdout).group(1))
    assert n == len(presample_restated(287933, 0.01))


@pytest.mark.gpu
def test_driver_tiff_maps_match_the_package(nb, syn, oracle, tmp_path):
    hp, dp, hab, disp = se_tiffs(tmp_path, syn)
    r = run_driver(nb, "simulate", SE_CONFIG % (hp, dp, ""), tmp_path, "se.ron")
    assert r.returncode == 0, r.stderr
    sc = nb.spatially_explicit_from_maps(str(hp), str(dp))
    o = nb.simulate(0.001, sc, 7)
    assert species(r.stdout) == o.biodiversity > 0
    desc = dict(kind=3, speciation_probability=0.001, width=12, height=10, habitat=sc.habitat,
                dispersal=sc.dispersal)
    ref = oracle.simulate(desc, 7, mode=oracle.MODE_REFERENCE)
    assert ref.biodiversity == o.biodiversity


WN_SCENARIO = ("WrappingNoise(seed: -7, coverage: 0.25, scale: 1.0, persistence: 1.0, octaves: 3, "
               "sample: Rectangle(origin: (x: 4294967276, y: 5), width: 40, height: 30), sigma: 1.0)")


def test_check_wrapping_noise(nb, tmp_path, kat):
    """WrappingNoise in the reference's RON spelling (docs/simulate.ron):
    the lineages are the habitable cells of the Rectangle sample."""
    case = kat["wrapping_noise_origins"][0]
    assert (case["seed"], case["sample"]) == (-7, [4294967276, 5, 40, 30])
    r = run_driver(nb, "check", CONFIG.replace("NonSpatial(area: (30, 20), deme: 2)", WN_SCENARIO), tmp_path)
    assert r.returncode == 0, r.stderr
    assert "WrappingNoise(seed: -7, coverage: 0.25" in r.stdout
    assert int(re.search(r"(\d+) lineages", r.stdout).group(1)) == len(case["origins"])


@pytest.mark.parametrize("sample", ["Rectangle(origin: (x: 4294967294, y: 7), width: 4, height: 3)",
                                    "Rectangle((origin: (x: 1, y: 2), width: 3, height: 4))",
                                    "Extent(origin: (x: 0, y: 0), width: 6, height: 2)"])
def test_check_almost_infinite_rectangle_sample(nb, tmp_path, sample):
    """AlmostInfinite's Rectangle sample (almost_infinite/mod.rs:92-122),
    also as a wrapped LandscapeExtent and by its Extent alias."""
    scen = "AlmostInfinite(sample: %s, dispersal: Normal(sigma: 2.0))" % sample
    r = run_driver(nb, "check", CONFIG.replace("NonSpatial(area: (30, 20), deme: 2)", scen), tmp_path)
    assert r.returncode == 0, r.stderr
    assert "AlmostInfinite(Rectangle(origin:" in r.stdout and "12 lineages" in r.stdout


@pytest.mark.parametrize("scenario", ["NonSpatial(area: (30, 20), deme: 2)", WN_SCENARIO,
                                      "AlmostInfinite(sample: Circle(radius: 12), dispersal: Normal(sigma: 2.0))"])
def test_check_isolated_landscape_partitions(nb, tmp_path, scenario):
    """IsolatedLandscape (independent/src/launch.rs:101-110): each rank keeps
    the sampled origins of its subdomain; the ranks split the sample."""
    base = CONFIG.replace("NonSpatial(area: (30, 20), deme: 2)", scenario).replace("percentage: 1.0", "percentage: 0.7")
    counts = []
    for rank in range(3):
        cfg = base.replace("Monolithic(event_slice: Relative(factor: 2.0))",
                           "IsolatedLandscape(partition: Partition(rank: %d, size: 3), "
                           "event_slice: Relative(factor: 2.0))" % rank)
        r = run_driver(nb, "check", cfg, tmp_path)
        assert r.returncode == 0, r.stderr
        counts.append(int(re.search(r"(\d+) lineages", r.stdout).group(1)))
    r = run_driver(nb, "check", base, tmp_path)
    total = int(re.search(r"(\d+) lineages", r.stdout).group(1))
    # a real split (the wrapping WrappingNoise sample lies at two angles of
    # the radial decomposition, so one of its ranks is empty)
    assert sum(counts) == total and max(counts) < total
    bad = base.replace("Monolithic(event_slice: Relative(factor: 2.0))",
                       "IsolatedLandscape(partition: Partition(rank: 3, size: 3))")
    r = run_driver(nb, "check", bad, tmp_path)
    assert r.returncode == 1 and "rank must be below" in r.stderr


RESTART_SAMPLE = ("sample: Sample(percentage: 1.0, origin: List([(ref: 7, time: 1.5, loc: (x: 3, y: 4, i: 1)), "
                  "(ref: 9, time: 0.25, loc: (x: 0, y: 0, i: 0))]), mode: Restart(after: 150.0)),")


def test_check_restart_sample_mode(nb, tmp_path):
    """Sample mode Restart(after) (dispatch/valid/launch.rs:82-92): the listed
    lineages restart with `after` as the minimum event time."""
    cfg = CONFIG.replace("sample: Sample(percentage: 1.0, origin: Habitat, mode: Genesis),", RESTART_SAMPLE)
    r = run_driver(nb, "check", cfg, tmp_path)
    assert r.returncode == 0, r.stderr
    assert "2 lineages (restarted)" in r.stdout and "restart after t = 150" in r.stdout
    r = run_driver(nb, "check", cfg.replace("after: 150.0", "after: -1.0"), tmp_path)
    assert r.returncode == 1 and "Restart(after)" in r.stderr
    r = run_driver(nb, "check", cfg.replace("mode: Restart(after: 150.0)", "mode: FixUp()"), tmp_path)
    assert r.returncode == 1 and "not supported (Genesis, Resume, Restart)" in r.stderr
    # every listed lineage must lie before the resume point max_after(after, after),
    # the next double above `after` (args/config/sample/mod.rs:118-137): a
    # lineage at `after` itself restarts, one a double later does not
    r = run_driver(nb, "check", cfg.replace("after: 150.0", "after: 1.5"), tmp_path)
    assert r.returncode == 0, r.stderr
    r = run_driver(nb, "check", cfg.replace("after: 150.0", "after: 1.4999999999999998"), tmp_path)
    assert r.returncode == 1 and "Lineage #7 at time 1.5 is not before the resume point" in r.stderr


def test_check_rejects_negative_lineage_times(nb, tmp_path):
    """Lineage::last_event_time is a NonNegativeF64: a negative or NaN time
    does not load, from a List or from a lineage file."""
    cfg = CONFIG.replace("sample: Sample(percentage: 1.0, origin: Habitat, mode: Genesis),",
                         RESTART_SAMPLE.replace("time: 0.25", "time: -0.25"))
    r = run_driver(nb, "check", cfg, tmp_path)
    assert r.returncode == 1 and "negative or NaN" in r.stderr
    f = tmp_path / "neg.bin"
    sample = 'sample: Sample(percentage: 1.0, origin: Bincode(file: "%s"), mode: Resume),' % f
    cfg = CONFIG.replace("sample: Sample(percentage: 1.0, origin: Habitat, mode: Genesis),", sample)
    for bad in (-1.0, float("nan")):
        f.write_bytes(lineage_file([(7, 1.5, 3, 4, 1), (8, bad, 3, 4, 0)]))
        r = run_driver(nb, "check", cfg, tmp_path)
        assert r.returncode == 1 and "negative or NaN" in r.stderr


def test_check_bincode_destiny_must_not_exist(nb, tmp_path):
    """LineageFileSaver::try_new opens the destiny with create_new when the
    configuration is read: an existing file fails before anything runs, and a
    file the run created but never wrote is removed again."""
    lins = tmp_path / "rest.bin"
    cfg = CONFIG.replace("pause: None", 'pause: Pause(before: 150.0, config: "%s", destiny: Bincode(file: "%s"))'
                         % (tmp_path / "resume.ron", lins))
    r = run_driver(nb, "check", cfg, tmp_path)
    assert r.returncode == 0, r.stderr
    assert not lins.exists()
    lins.write_bytes(b"keep")
    r = run_driver(nb, "check", cfg, tmp_path)
    assert r.returncode == 1 and "cannot create the lineage file" in r.stderr
    assert lins.read_bytes() == b"keep"


@pytest.mark.gpu
def test_driver_restart_pause_mode(nb, tmp_path):
    """Pause mode Restart (pause.rs:41-53) writes `mode: Restart(after: <before>)`;
    no lineage has an event between its last one and the pause, so the
    restart completes the straight run's species."""
    resume = tmp_path / "restart.ron"
    cfg = CONFIG.replace("pause: None",
                         'pause: Pause(before: 150.0, config: "%s", destiny: List, mode: Restart)' % resume)
    r = run_driver(nb, "simulate", cfg, tmp_path, "p.ron")
    assert r.returncode == 0, r.stderr
    assert re.search(r"mode:\s*Restart\(\s*after:\s*150\.0,?\s*\)", resume.read_text())
    r2 = subprocess.run([nb.DRIVER, "simulate", str(resume)], capture_output=True, text=True, timeout=600)
    assert r2.returncode == 0, r2.stderr
    assert "(restarted)" in r2.stdout
    straight = nb.simulate(0.01, nb.NonSpatial((30, 20), 2), 42)
    assert species(r.stdout) + species(r2.stdout) == straight.biodiversity


def lineage_file(lineages):
    """Vec<Lineage> in bincode 1.3.3's DefaultOptions (varint integers, f64 as
    8 little-endian bytes), as lineage_file/saver.rs writes it."""
    import struct

    def varint(v):
        if v < 251:
            return bytes([v])
        if v < 1 << 16:
            return b"\xfb" + struct.pack("<H", v)
        if v < 1 << 32:
            return b"\xfc" + struct.pack("<I", v)
        return b"\xfd" + struct.pack("<Q", v)
    out = varint(len(lineages))
    for ref, time, x, y, i in lineages:
        out += varint(ref) + struct.pack("<d", time) + varint(x) + varint(y) + varint(i)
    return out


def test_check_bincode_lineage_file(nb, tmp_path):
    """Sample origin Bincode(file) (lineage_file/loader.rs) with values in
    every varint width."""
    f = tmp_path / "lineages.bin"
    f.write_bytes(lineage_file([(7, 1.5, 3, 4, 1), (1 << 40, 0.25, 70000, 250, 0), (300, 2.0, 1 << 31, 0, 1)]))
    sample = 'sample: Sample(percentage: 1.0, origin: Bincode(file: "%s"), mode: Resume),' % f
    cfg = CONFIG.replace("sample: Sample(percentage: 1.0, origin: Habitat, mode: Genesis),", sample)
    r = run_driver(nb, "check", cfg, tmp_path)
    assert r.returncode == 0, r.stderr
    assert "3 lineages (resumed)" in r.stdout
    f.write_bytes(lineage_file([(7, 1.5, 3, 4, 1)])[:-2])
    r = run_driver(nb, "check", cfg, tmp_path)
    assert r.returncode == 1 and "truncated lineage file" in r.stderr
    # bytes after the list are not read (bincode::Deserializer::with_reader)
    f.write_bytes(lineage_file([(7, 1.5, 3, 4, 1)]) + b"\0")
    r = run_driver(nb, "check", cfg, tmp_path)
    assert r.returncode == 0 and "1 lineages (resumed)" in r.stdout, r.stderr


@pytest.mark.gpu
def test_driver_pause_to_a_bincode_file(nb, tmp_path):
    """Pause destiny Bincode(file) (pause.rs:29-39): the remaining lineages go
    to the file, and the written configuration resumes from it."""
    resume, lins = tmp_path / "resume.ron", tmp_path / "rest.bin"
    cfg = CONFIG.replace("pause: None", 'pause: Pause(before: 150.0, config: "%s", destiny: Bincode(file: "%s"))'
                         % (resume, lins))
    r = run_driver(nb, "simulate", cfg, tmp_path, "p.ron")
    assert r.returncode == 0, r.stderr
    assert lins.exists() and "Bincode" in resume.read_text()
    r2 = subprocess.run([nb.DRIVER, "simulate", str(resume)], capture_output=True, text=True, timeout=600)
    assert r2.returncode == 0, r2.stderr
    straight = nb.simulate(0.01, nb.NonSpatial((30, 20), 2), 42)
    assert species(r.stdout) + species(r2.stdout) == straight.biodiversity
