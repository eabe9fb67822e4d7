"""The reference-format event log (necsim/impls/std/src/event_log/recorder.rs,
bincode 1.3 fixed-width little-endian encoding of EventLogHeader and
PackedEvent): byte layout against an independent struct-level restatement,
segmenting, sorting and kind decoding; and a GPU run logged end to end."""
import ctypes
import os
import struct

import numpy as np
import pytest


def write(nb, directory, spec, disp, capacity):
    log = nb.EventLog(directory, capacity=capacity, speciation=True, dispersal=True)
    r = log.reporter
    if len(spec):
        a = np.ascontiguousarray(spec, dtype=nb.SPECIATION_DTYPE)
        assert r.report_speciation(r.user, a.ctypes.data, len(a)) == 0
    if len(disp):
        a = np.ascontiguousarray(disp, dtype=nb.DISPERSAL_DTYPE)
        assert r.report_dispersal(r.user, a.ctypes.data, len(a)) == 0
    log.close()


def neg(v):
    return -abs(v) if v != 0.0 else -0.0


def test_segment_bytes_match_the_reference_layout(nb, tmp_path):
    spec = np.zeros(1, dtype=nb.SPECIATION_DTYPE)
    spec[0] = (7, 1.5, 2.25, 3, 4, 5, 0)
    disp = np.zeros(1, dtype=nb.DISPERSAL_DTYPE)
    disp[0] = (9, 0.5, 2.0, 1, 2, 0, 6, 7, 0, 0, 0)
    d = str(tmp_path / "log")
    write(nb, d, spec, disp, capacity=10)
    raw = open(os.path.join(d, "0"), "rb").read()
    # EventLogHeader (event_log/mod.rs:9-18): min_time, max_time, length, with_speciation, with_dispersal
    expect = struct.pack("<ddQ??", 2.0, 2.25, 2, True, True)
    # PackedEvent (event.rs:18-28), sorted by event time: the dispersal (t = 2.0) first.
    # Dispersal with LineageInteraction::Maybe: prior +, event -, coalescence = lineage
    expect += struct.pack("<QddIIIIIIQ", 9, 0.5, neg(2.0), 1, 2, 0, 6, 7, 0, 9)
    # Speciation: prior -, event +, target = origin, coalescence = lineage
    expect += struct.pack("<QddIIIIIIQ", 7, neg(1.5), 2.25, 3, 4, 5, 3, 4, 5, 7)
    assert raw == expect


def test_segments_sorted_and_decoded(nb, tmp_path):
    rng = np.random.default_rng(3)
    n = 2500
    spec = np.zeros(n, dtype=nb.SPECIATION_DTYPE)
    spec["gref"] = rng.integers(0, 1 << 40, n)
    spec["prior_time"] = rng.random(n) * 10
    spec["event_time"] = spec["prior_time"] + rng.random(n) + 1e-9
    spec["x"], spec["y"], spec["index"] = rng.integers(0, 50, (3, n))
    disp = np.zeros(n, dtype=nb.DISPERSAL_DTYPE)
    disp["gref"] = rng.integers(0, 1 << 40, n)
    disp["prior_time"] = rng.random(n) * 10
    disp["event_time"] = disp["prior_time"] + rng.random(n) + 1e-9
    for f in ("x", "y", "index", "tx", "ty", "tindex"):
        disp[f] = rng.integers(0, 50, n)
    d = str(tmp_path / "log")
    write(nb, d, spec, disp, capacity=1000)
    names = sorted(os.listdir(d), key=int)
    assert names == [str(i) for i in range(5)]
    headers, ev = nb.read_event_log(d)
    assert [int(h["length"]) for h in headers] == [1000, 1000, 1000, 1000, 1000]
    for name, h in zip(names, headers):
        seg = np.frombuffer(open(os.path.join(d, name), "rb").read()[26:], dtype=nb.PACKED_EVENT_DTYPE)
        t = np.abs(seg["event_time"])
        assert np.all(np.diff(t) >= 0) and t[0] == h["min_time"] and t[-1] == h["max_time"]
    assert len(ev) == 2 * n and np.all(np.diff(ev["event_time"]) >= 0)
    assert set(ev["kind"]) == {0, 2}
    s = ev[ev["kind"] == 0]
    assert sorted(zip(s["gref"], s["event_time"])) == sorted(zip(spec["gref"], spec["event_time"]))
    assert np.array_equal(s["x"], s["tx"]) and np.array_equal(s["gref"], s["coalescence"])
    g = ev[ev["kind"] == 2]
    assert sorted(zip(g["gref"], g["tx"], g["ty"])) == sorted(zip(disp["gref"], disp["tx"], disp["ty"]))


def test_existing_directory_is_refused(nb, tmp_path):
    d = tmp_path / "taken"
    d.mkdir()
    with pytest.raises(nb.NecsimError):
        nb.EventLog(str(d))


def test_no_events_leave_no_directory(nb, tmp_path):
    d = str(tmp_path / "empty")
    nb.EventLog(d).close()
    assert not os.path.exists(d)


@pytest.mark.gpu
def test_simulation_logged_to_disk(nb, syn, tmp_path):
    sc = nb.NonSpatial((20, 20), 2)
    with nb.Simulation(sc, 0.01, nb.CUDA(report_dispersal=True)) as sim:
        ref = sim.simulate(5)
        log = nb.EventLog(str(tmp_path / "run"), capacity=4096, dispersal=True)
        o = sim.simulate(5, event_log=log)
        log.close()
    headers, ev = nb.read_event_log(str(tmp_path / "run"))
    assert sum(int(h["length"]) for h in headers) == len(ev) == o.n_speciation + o.n_dispersal
    s = ev[ev["kind"] == 0]
    assert np.array_equal(np.sort(s["event_time"]), np.sort(ref.speciation["event_time"]))
    assert len(ev[ev["kind"] == 2]) == ref.n_dispersal
    assert o.biodiversity == ref.biodiversity


# ---- replay (event_log/replay/*.rs) ----
def random_events(nb, n, seed):
    rng = np.random.default_rng(seed)
    spec = np.zeros(n, dtype=nb.SPECIATION_DTYPE)
    spec["gref"] = rng.integers(0, 1 << 40, n)
    spec["prior_time"] = rng.random(n) * 10
    spec["event_time"] = spec["prior_time"] + rng.random(n) + 1e-9
    spec["x"], spec["y"], spec["index"] = rng.integers(0, 30, (3, n))
    disp = np.zeros(n, dtype=nb.DISPERSAL_DTYPE)
    disp["gref"] = rng.integers(0, 1 << 40, n)
    disp["prior_time"] = rng.random(n) * 10
    disp["event_time"] = disp["prior_time"] + rng.random(n) + 1e-9
    for f in ("x", "y", "index", "tx", "ty", "tindex"):
        disp[f] = rng.integers(0, 30, n)
    return spec, disp


def packed_key(e, speciation):
    t = (int(e["x"]), int(e["y"]), int(e["index"])) if speciation else (int(e["tx"]), int(e["ty"]), int(e["tindex"]))
    return (float(e["event_time"]), int(e["x"]), int(e["y"]), int(e["index"])) + t + \
        (float(e["prior_time"]), int(e["gref"]))


def test_replay_merges_overlapping_segments_in_packed_order(nb, tmp_path):
    # several logs whose segments overlap in time, written in delivery batches
    logs, keys = [], []
    for j in range(3):
        spec, disp = random_events(nb, 700, 10 + j)
        d = str(tmp_path / ("log%d" % j))
        log = nb.EventLog(d, capacity=97, speciation=True, dispersal=True)
        r = log.reporter
        for k in range(0, 700, 150):  # several batches per log: segments overlap
            a = np.ascontiguousarray(spec[k:k + 150])
            assert r.report_speciation(r.user, a.ctypes.data, len(a)) == 0
            b = np.ascontiguousarray(disp[k:k + 150])
            assert r.report_dispersal(r.user, b.ctypes.data, len(b)) == 0
        log.close()
        logs.append(os.path.join(d, "*"))
        keys += [(packed_key(e, True), "s") for e in spec] + [(packed_key(e, False), "d") for e in disp]
    out = nb.replay_event_log(logs, capacity=13)
    assert out.n_events == len(keys) == len(out.speciation) + len(out.dispersal)
    got = []
    i = j = 0
    for kind, n in out.delivery:
        for _ in range(n):
            if kind == "s":
                got.append((packed_key(out.speciation[i], True), "s"))
                i += 1
            else:
                got.append((packed_key(out.dispersal[j], False), "d"))
                j += 1
    assert got == sorted(keys)
    # delivery batches alternate kinds only where the stream does
    assert all(a[0] != b[0] for a, b in zip(out.delivery, out.delivery[1:]) if a[1] < 4096)


def raw_segment(path, events, with_speciation=True, with_dispersal=True):
    times = [abs(e[2]) for e in events]
    data = struct.pack("<ddQ??", min(times), max(times), len(events), with_speciation, with_dispersal)
    for e in events:
        data += struct.pack("<QddIIIIIIQ", *e)
    open(path, "wb").write(data)


def test_replay_decodes_every_sign_pair(nb, tmp_path):
    # (prior, event) signs: (-, +) speciation; (+, -) Maybe, (+, +) None and
    # (-, -) Coalescence dispersal (event.rs:186-240)
    ev = [(1, -0.5, 1.0, 1, 1, 0, 1, 1, 0, 1), (2, 0.5, -2.0, 1, 1, 0, 2, 2, 0, 2),
          (3, 0.5, 3.0, 1, 1, 0, 3, 3, 0, 3), (4, -0.5, -4.0, 1, 1, 0, 4, 4, 0, 9)]
    raw_segment(str(tmp_path / "0"), ev)
    out = nb.replay_event_log(str(tmp_path / "0"))
    assert out.delivery == [("s", 1), ("d", 3)]
    assert out.speciation[0]["prior_time"] == 0.5 and out.speciation[0]["event_time"] == 1.0
    assert out.dispersal["event_time"].tolist() == [2.0, 3.0, 4.0]
    assert out.dispersal["prior_time"].tolist() == [0.5, 0.5, 0.5]
    assert out.dispersal["tx"].tolist() == [2, 3, 4]


def test_replay_checks_segments_and_needs(nb, tmp_path):
    a = [(1, -0.5, 1.0, 1, 1, 0, 1, 1, 0, 1)]
    raw_segment(str(tmp_path / "a"), a, True, False)
    raw_segment(str(tmp_path / "b"), [(2, -0.5, 2.0, 1, 1, 0, 1, 1, 0, 2)], True, True)
    with pytest.raises(nb.NecsimError, match="mismatch in reporting dispersal"):
        nb.replay_event_log([str(tmp_path / "a"), str(tmp_path / "b")])
    with pytest.raises(nb.NecsimError, match="require dispersal events"):
        nb.replay_event_log(str(tmp_path / "a"), need_dispersal=True)
    out = nb.replay_event_log(str(tmp_path / "a"), need_dispersal=True, strict=False)
    assert "require dispersal events" in out.warning and out.n_events == 1
    with pytest.raises(nb.NecsimError, match="at least one"):
        nb.replay_event_log([])
    with pytest.raises(nb.NecsimError, match="cannot read"):
        nb.replay_event_log(str(tmp_path / "missing"))
    (tmp_path / "short").write_bytes(b"\0" * 10)
    with pytest.raises(nb.NecsimError, match="not an event log segment"):
        nb.replay_event_log(str(tmp_path / "short"))


def test_driver_replays_a_log(nb, tmp_path):
    import subprocess
    spec, disp = random_events(nb, 400, 21)
    spec[1::3]["x"] = spec[0::3][: len(spec[1::3])]["x"]  # some equal neighbours for the species count
    # repeats of events (a duplicate lineage's copy), some with another prior time: late coalescences
    spec[5::40] = spec[4::40][: len(spec[5::40])]
    spec["prior_time"][5::80] -= 1e-3
    disp[7::30] = disp[6::30][: len(disp[7::30])]
    disp["prior_time"][7::60] -= 1e-3
    write(nb, str(tmp_path / "log"), spec, disp, capacity=64)
    cfg = """(
        log: EventLog(segments: ["%s/*"], capacity: 7),
        mode: Strict,
        reporters: [Plugin(library: "x.so", reporters: [Biodiversity(), Counter(), Execution()])],
    )""" % (tmp_path / "log")
    (tmp_path / "r.ron").write_text(cfg)
    r = subprocess.run([nb.DRIVER, "replay", str(tmp_path / "r.ron")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    out = nb.replay_event_log(str(tmp_path / "log/*"))
    species, last = 0, None
    for e in out.speciation:  # biodiversity.rs:33-41 on the replayed stream
        key = (int(e["x"]), int(e["y"]), int(e["index"]), float(e["event_time"]))
        if key != last:
            species += 1
        last = key
    assert "biodiversity of %d unique species" % species in r.stdout
    assert "replayed %d events" % (2 * 400) in r.stdout
    assert counter_summary(out) in r.stdout
    import re
    # Rust's Debug for Duration, as the Execution reporter prints it
    assert re.search(r"The replay took \d+(\.\d*[1-9])?(s|ms|\u00b5s|ns)\n", r.stdout), r.stdout


def counter_summary(out):
    """EventCounterReporter (necsim/plugins/common/src/event_counter.rs) on a
    replayed stream whose dispersal events carry LineageInteraction::Maybe."""
    raw = spec = late_disp = late = 0
    last_s = last_d = last_prior = None
    i = j = 0
    for kind, n in out.delivery:
        for _ in range(n):
            if kind == "s":
                e = out.speciation[i]
                i += 1
                key = (int(e["x"]), int(e["y"]), int(e["index"]), float(e["event_time"]))
                raw += 1
                if key == last_s:
                    late += float(e["prior_time"]) != last_prior
                else:
                    last_s = key
                    spec += 1
            else:
                e = out.dispersal[j]
                j += 1
                key = (int(e["x"]), int(e["y"]), int(e["index"]), float(e["event_time"]), int(e["tx"]),
                       int(e["ty"]), int(e["tindex"]))
                raw += 1
                if key == last_d:
                    late += float(e["prior_time"]) != last_prior
                else:
                    last_d = key
                    late_disp += 1
            last_prior = float(e["prior_time"])
    return ("Event Summary:\n - Total #individuals:\n   %d\n - Total #events:\n   - raw:\n     %d\n"
            "   - deduplicated:\n     %d\n - Speciation:\n    %d\n - Dispersal:\n"
            "   - same location, no coalescence:\n     0\n   - same location, with coalescence:\n     0\n"
            "   - new location, no coalescence:\n     0\n   - new location, with coalescence:\n     0\n"
            "   - detected late, no coalescence:\n     %d\n   - detected late, with coalescence:\n     %d\n"
            % (spec + late, raw, spec + late_disp, spec, (late_disp - late) % (1 << 64), late))


def rust_display(v):
    """Rust's Display for a finite f64: the shortest round-trip digits in
    fixed notation (no exponent, no trailing `.0`)."""
    from decimal import Decimal
    t = format(Decimal(repr(float(v))), "f")
    if "." in t:
        t = t.rstrip("0").rstrip(".")
    return t


def test_driver_csv_reporter(nb, tmp_path):
    """The Csv reporter (necsim/plugins/csv/src/lib.rs) during a replay: a
    header, then `reference,time,x,y,index,type` per event in delivery order,
    with the origin of dispersal events and Rust's f64 Display."""
    import subprocess
    spec, disp = random_events(nb, 120, 5)
    spec["event_time"][:4] = [3.0, 1e-7, 0.30000000000000004, 123456789.125]
    disp["event_time"][:2] = [2.0 ** 60, 5e-324]
    write(nb, str(tmp_path / "log"), spec, disp, capacity=50)
    csv = tmp_path / "events.csv"
    cfg = """(
        log: EventLog(segments: ["%s/*"]),
        reporters: [Plugin(library: "libnecsim_plugins_csv.so", reporters: [Csv(output: "%s")])],
    )""" % (tmp_path / "log", csv)
    (tmp_path / "r.ron").write_text(cfg)
    r = subprocess.run([nb.DRIVER, "replay", str(tmp_path / "r.ron")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    out = nb.replay_event_log(str(tmp_path / "log/*"), need_speciation=True, need_dispersal=True)
    rows, s, d = ["reference,time,x,y,index,type"], 0, 0
    for kind, n in out.delivery:
        src = out.speciation[s:s + n] if kind == "s" else out.dispersal[d:d + n]
        for e in src:
            rows.append("%d,%s,%d,%d,%d,%s" % (e["gref"], rust_display(e["event_time"]), e["x"], e["y"], e["index"],
                                               kind))
        if kind == "s":
            s += n
        else:
            d += n
    assert s == 120 and d == 120
    assert csv.read_text() == "\n".join(rows) + "\n"
    assert {"3", "0.0000001", "0.30000000000000004", "123456789.125", "1152921504606847000"} <= \
        {row.split(",")[1] for row in rows[1:]}


def test_driver_statistics_reporters(nb, tmp_path):
    """GlobalSpeciation, GlobalTurnover and GlobalCoverage (necsim/plugins/
    statistics/src/*.rs) during a replay: each skips an event equal to the
    previous one of its kind (same origin and event time, and target)."""
    import subprocess
    spec, disp = random_events(nb, 150, 9)
    spec[3::25] = spec[2::25][: len(spec[3::25])]  # repeats: skipped
    spec["prior_time"][3::50] -= 1e-3              # equal all the same (prior time is ignored)
    disp[5::20] = disp[4::20][: len(disp[5::20])]
    write(nb, str(tmp_path / "log"), spec, disp, capacity=40)
    outs = {k: tmp_path / ("%s.csv" % k) for k in ("GlobalSpeciation", "GlobalTurnover", "GlobalCoverage")}
    reps = ", ".join('%s(output: "%s")' % (k, v) for k, v in outs.items())
    cfg = """(
        log: EventLog(segments: ["%s/*"]),
        reporters: [Plugin(library: "libnecsim_plugins_statistics.so", reporters: [%s])],
    )""" % (tmp_path / "log", reps)
    (tmp_path / "r.ron").write_text(cfg)
    r = subprocess.run([nb.DRIVER, "replay", str(tmp_path / "r.ron")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    out = nb.replay_event_log(str(tmp_path / "log/*"), need_speciation=True, need_dispersal=True)
    sp, tu, co = ["speciation"], ["turnover"], ["x-from,y-from,index-from,x-to,y-to,index-to"]
    s = d = 0
    last_s = last_d = None
    for kind, n in out.delivery:
        if kind == "s":
            for e in out.speciation[s:s + n]:
                key = (int(e["x"]), int(e["y"]), int(e["index"]), float(e["event_time"]))
                if key != last_s:
                    last_s = key
                    sp.append(rust_display(e["event_time"]))
                    tu.append(rust_display(float(e["event_time"]) - float(e["prior_time"])))
            s += n
        else:
            for e in out.dispersal[d:d + n]:
                key = tuple(int(e[f]) for f in ("x", "y", "index", "tx", "ty", "tindex")) + (float(e["event_time"]),)
                if key != last_d:
                    last_d = key
                    tu.append(rust_display(float(e["event_time"]) - float(e["prior_time"])))
                    co.append("%d,%d,%d,%d,%d,%d" % key[:6])
            d += n
    assert 1 < len(sp) - 1 < 150 and 1 < len(co) - 1 < 150
    assert outs["GlobalSpeciation"].read_text() == "\n".join(sp) + "\n"
    assert outs["GlobalTurnover"].read_text() == "\n".join(tu) + "\n"
    assert outs["GlobalCoverage"].read_text() == "\n".join(co) + "\n"


def test_sign_encoding_follows_the_reference_kats(nb, tmp_path):
    """The event kind lives in the time sign bits (event.rs:105-160), set and
    cleared bit-wise like the reference's make_negative / make_positive,
    whose own tests (event.rs:337-353) pin -0.0 <-> 0.0, 42.0 <-> -42.0 and
    24.0 / -24.0: a speciation event at prior time 0.0 is stored with the
    sign bit alone, and replay gives back +0.0."""
    spec = np.zeros(1, dtype=nb.SPECIATION_DTYPE)
    spec[0] = (3, 0.0, 42.0, 1, 1, 0, 0)
    disp = np.zeros(1, dtype=nb.DISPERSAL_DTYPE)
    disp[0] = (4, 24.0, 42.0, 1, 1, 0, 2, 2, 0, 0, 0)
    d = str(tmp_path / "log")
    write(nb, d, spec, disp, capacity=10)
    seg = np.frombuffer(open(os.path.join(d, "0"), "rb").read()[26:], dtype=nb.PACKED_EVENT_DTYPE)
    bits = {int(g): (int(p), int(e)) for g, p, e in zip(seg["gref"], seg["prior_time"].view(np.uint64),
                                                           seg["event_time"].view(np.uint64))}
    f64 = lambda v: struct.unpack("<Q", struct.pack("<d", v))[0]  # noqa: E731
    assert bits[3] == (0x8000000000000000, f64(42.0))      # make_negative(0.0), make_positive(42.0)
    assert bits[4] == (f64(24.0), f64(-42.0))              # make_positive(24.0), make_negative(42.0)
    _, ev = nb.read_event_log(d)
    s = ev[ev["kind"] == 0][0]
    assert s["prior_time"] == 0.0 and not np.signbit(s["prior_time"]) and s["event_time"] == 42.0
    g = ev[ev["kind"] == 2][0]
    assert (g["prior_time"], g["event_time"]) == (24.0, 42.0)
