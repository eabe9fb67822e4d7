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
