"""The allocation-free round (necsim_gpu_round_noalloc) against the existing
entry point (marked gpu).

The allocation-free round serves callers that cannot allocate device memory
(their host owns the allocator, they run in a fixed arena, or they must not
incur cudaMalloc's synchronisation).  It advances lineages to a horizon in
one round and merges duplicates, using a working area that lives in the
library.  The existing necsim_gpu_simulate_lineages reaches the same horizon
in several rounds; both must leave the same surviving lineages (state and
smallest global reference) and the same distinct speciation events, bit for
bit.  The oracle's canonical schedule run to the same horizon in one round
pins the round itself: the same surviving lineages, the same speciation
events and exactly the same number of executed events.  Two calls in a row
check that the shared working area is reset between calls.  This file sorts
last so a failure here does not hide other results.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_bytes(torch, arr):
    t = torch.from_numpy(np.frombuffer(arr.tobytes(), dtype=np.uint8).copy()).cuda()
    return t


def _bind(nb):
    L = nb.lib()
    L.necsim_gpu_round_noalloc.argtypes = [
        ctypes.POINTER(nb.CScenario), ctypes.POINTER(nb.CArgs), ctypes.c_uint64, ctypes.c_void_p,
        ctypes.c_uint64, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
        ctypes.POINTER(ctypes.c_uint64), ctypes.c_void_p, ctypes.c_uint64,
        ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64), ctypes.c_void_p]
    L.necsim_gpu_round_noalloc.restype = ctypes.c_int
    return L


def _round(nb, torch, scenario_struct, seed_word, lineages, resume_time, horizon, sampler="poisson"):
    L = _bind(nb)
    n = len(lineages)
    d_in = _device_bytes(torch, np.ascontiguousarray(lineages, dtype=nb.LINEAGE_DTYPE))
    d_out = torch.zeros(n * nb.LINEAGE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    d_ev = torch.zeros(n * nb.SPECIATION_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    n_out = ctypes.c_uint64(0)
    n_ev = ctypes.c_uint64(0)
    steps = ctypes.c_uint64(0)
    args = nb._args_struct(nb.CUDA(event_time_sampler=sampler))
    torch.cuda.synchronize()
    rc = L.necsim_gpu_round_noalloc(ctypes.byref(scenario_struct), ctypes.byref(args), seed_word,
                                    d_in.data_ptr(), n, resume_time, horizon, d_out.data_ptr(),
                                    ctypes.byref(n_out), d_ev.data_ptr(), n,
                                    ctypes.byref(n_ev), ctypes.byref(steps), None)
    assert rc == 0, rc
    out = np.frombuffer(d_out.cpu().numpy().tobytes(), dtype=nb.LINEAGE_DTYPE)[:n_out.value]
    ev = np.frombuffer(d_ev.cpu().numpy().tobytes(), dtype=nb.SPECIATION_DTYPE)[:n_ev.value]
    return out.copy(), ev.copy(), steps.value


def _same_lineages(a, b):
    a = np.sort(a, order="gref")
    b = np.sort(b, order="gref")
    if len(a) != len(b):
        return False
    return (np.array_equal(a["gref"], b["gref"]) and np.array_equal(a["x"], b["x"])
            and np.array_equal(a["y"], b["y"]) and np.array_equal(a["index"], b["index"])
            and np.array_equal(a["last_event_time"].view(np.uint64),
                               b["last_event_time"].view(np.uint64)))


SCENARIOS = {
    "non_spatial": (dict(kind=0, speciation_probability=2e-3, width=40, height=40, deme=4), 11),
    "spatially_implicit": (dict(kind=1, speciation_probability=1e-3, width=3000, height=1, deme=1,
                                meta_width=100000, meta_height=1, meta_deme=1, migration_probability=0.1), 5),
    "almost_infinite": (dict(kind=2, speciation_probability=2e-3, sigma=5.0, radius=30, centre_x=1 << 31,
                             centre_y=1 << 31), 11),
}


def _one_round_oracle(oracle, desc, seed, sampler, lineages, resume_time, horizon):
    """The canonical schedule with a round that reaches `horizon` at once."""
    code = oracle.SAMPLER_EXP if sampler == "exp" else oracle.SAMPLER_POISSON
    return oracle.simulate(desc, seed, mode=oracle.MODE_CANONICAL, lineages=lineages, resume_time=resume_time,
                           pause_before=horizon, step_slice=1000, step_slice_max=1000, min_round_events=1,
                           event_time_sampler=code)


def _same_events(a, b):
    key = ["gref", "x", "y", "index"]
    a = np.sort(a, order=key)
    b = np.sort(b, order=key)
    return len(a) == len(b) and all(np.array_equal(a[f], b[f]) for f in key) and all(
        np.array_equal(a[f].view(np.uint64), b[f].view(np.uint64)) for f in ("prior_time", "event_time"))


@pytest.mark.parametrize("sampler", ["poisson", "exp"])
@pytest.mark.parametrize("scenario", sorted(SCENARIOS))
def test_round_noalloc_matches_existing_entry_point(nb, syn, oracle, scenario, sampler):
    torch = pytest.importorskip("torch")
    desc, seed = SCENARIOS[scenario]
    sc, nu = syn.to_scenario(desc), desc["speciation_probability"]
    word = nb.seed_from_u64(seed)
    struct = nb._scenario_struct(sc, nu)
    origins = nb.enumerate_origins(sc, nu)
    assert 0 < len(origins) <= 65536
    algo = nb.CUDA(event_time_sampler=sampler)

    # first call: origins -> horizon 60
    out1, ev1, steps1 = _round(nb, torch, struct, word, origins, 0.0, 60.0, sampler)
    with nb.Simulation(sc, nu, algo) as sim:
        ref1 = sim.resume(origins, 0.0, seed, pause_before=60.0)
    assert _same_lineages(out1, ref1.remaining)
    assert np.array_equal(nb.distinct_speciation_set(ev1),
                          nb.distinct_speciation_set(ref1.speciation))
    c1 = _one_round_oracle(oracle, desc, seed, sampler, origins, 0.0, 60.0)
    assert c1.n_rounds == 1 and steps1 == c1.steps > 0
    assert _same_lineages(out1, c1.remaining) and _same_events(ev1, c1.speciation)

    # second call in a row reuses the working area: survivors -> horizon 150
    out2, ev2, steps2 = _round(nb, torch, struct, word, out1, 60.0, 150.0, sampler)
    with nb.Simulation(sc, nu, algo) as sim:
        ref2 = sim.resume(ref1.remaining, 60.0, seed, pause_before=150.0)
    assert _same_lineages(out2, ref2.remaining)
    assert np.array_equal(nb.distinct_speciation_set(ev2),
                          nb.distinct_speciation_set(ref2.speciation))
    c2 = _one_round_oracle(oracle, desc, seed, sampler, out1, 60.0, 150.0)
    assert c2.n_rounds == 1 and steps2 == c2.steps > 0
    assert _same_lineages(out2, c2.remaining) and _same_events(ev2, c2.speciation)


def test_round_noalloc_rejects_an_unknown_sampler(nb):
    torch = pytest.importorskip("torch")
    L = _bind(nb)
    struct = nb._scenario_struct(nb.NonSpatial((10, 10), 1), 0.01)
    args = nb.CArgs()
    args.event_time_sampler = 7
    n_out, n_ev, steps = ctypes.c_uint64(0), ctypes.c_uint64(0), ctypes.c_uint64(0)
    buf = torch.zeros(64 * 40, dtype=torch.uint8, device="cuda")
    p = buf.data_ptr()
    rc = L.necsim_gpu_round_noalloc(ctypes.byref(struct), ctypes.byref(args), 1, p, 1, 0.0, 10.0, p,
                                    ctypes.byref(n_out), p, 1, ctypes.byref(n_ev), ctypes.byref(steps), None)
    assert rc == -1  # NECSIM_E_INVALID_ARGUMENT


def test_round_noalloc_rejects_too_many_lineages(nb):
    torch = pytest.importorskip("torch")
    L = _bind(nb)
    struct = nb._scenario_struct(nb.NonSpatial((300, 300), 1), 0.01)
    n_out = ctypes.c_uint64(0)
    n_ev = ctypes.c_uint64(0)
    steps = ctypes.c_uint64(0)
    # a real (small) device buffer; the size check rejects the call before use
    buf = torch.zeros(64, dtype=torch.uint8, device="cuda")
    p = buf.data_ptr()
    rc = L.necsim_gpu_round_noalloc(ctypes.byref(struct), None, 1, p, 65537, 0.0, 10.0, p,
                                    ctypes.byref(n_out), p, 65537, ctypes.byref(n_ev),
                                    ctypes.byref(steps), None)
    assert rc == -10  # NECSIM_E_TOO_LARGE
    assert n_out.value == 0 and n_ev.value == 0
