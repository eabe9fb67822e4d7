"""ctypes binding of ``libnecsim_oracle.so`` (test infrastructure only).

The C library restates necsim-rust's CPU Independent algorithm; see
``necsim_oracle.c`` for the reference file:line each function follows.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libnecsim_oracle.so")

NON_SPATIAL = 0
SPATIALLY_IMPLICIT = 1
ALMOST_INFINITE_NORMAL = 2
ALMOST_INFINITE_CLARK2DT = 4
SPATIALLY_EXPLICIT = 3
WRAPPING_NOISE = 5

MODE_REFERENCE = 0
MODE_CANONICAL = 1

SAMPLER_POISSON = 0  # event_time_sampler/poisson.rs
SAMPLER_EXP = 1  # event_time_sampler/exp.rs


class OracleScenario(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("reserved0", ctypes.c_uint32),
        ("speciation_probability", ctypes.c_double),
        ("turnover_rate", ctypes.c_double),
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("deme", ctypes.c_uint32),
        ("meta_width", ctypes.c_uint32),
        ("meta_height", ctypes.c_uint32),
        ("meta_deme", ctypes.c_uint32),
        ("migration_probability", ctypes.c_double),
        ("sigma", ctypes.c_double),
        ("centre_x", ctypes.c_uint32),
        ("centre_y", ctypes.c_uint32),
        ("radius", ctypes.c_uint32),
        ("reserved1", ctypes.c_uint32),
        ("habitat", ctypes.POINTER(ctypes.c_uint32)),
        ("dispersal", ctypes.POINTER(ctypes.c_double)),
        ("shape_u", ctypes.c_double),
        ("tail_p", ctypes.c_double),
        ("turnover", ctypes.POINTER(ctypes.c_double)),
        ("noise_seed", ctypes.c_int64),
        ("coverage", ctypes.c_double),
        ("scale", ctypes.c_double),
        ("persistence", ctypes.c_double),
        ("octaves", ctypes.c_uint64),
        ("sample_x", ctypes.c_uint32),
        ("sample_y", ctypes.c_uint32),
        ("sample_width", ctypes.c_uint64),
        ("sample_height", ctypes.c_uint64),
    ]


class OracleArgs(ctypes.Structure):
    _fields_ = [
        ("delta_t", ctypes.c_double),
        ("step_slice", ctypes.c_uint64),
        ("dedup_factor", ctypes.c_double),
        ("event_slice_factor", ctypes.c_double),
        ("min_round_events", ctypes.c_uint64),
        ("report_dispersal", ctypes.c_int32),
        ("mode", ctypes.c_int32),
        ("partition_rank", ctypes.c_uint32),
        ("partition_size", ctypes.c_uint32),
        ("step_slice_max", ctypes.c_uint64),
        ("event_time_sampler", ctypes.c_int32),
        ("pad", ctypes.c_int32),
    ]


class OracleResult(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32),
        ("pad", ctypes.c_int32),
        ("time", ctypes.c_double),
        ("steps", ctypes.c_uint64),
        ("n_initial", ctypes.c_uint64),
        ("n_remaining", ctypes.c_uint64),
        ("n_speciation", ctypes.c_uint64),
        ("biodiversity", ctypes.c_uint64),
        ("n_dispersal", ctypes.c_uint64),
        ("n_primes", ctypes.c_uint64),
        ("n_draws", ctypes.c_uint64),
        ("n_rounds", ctypes.c_uint64),
        ("n_dedup", ctypes.c_uint64),
    ]


SPECIATION_DTYPE = np.dtype(
    [("gref", "<u8"), ("prior_time", "<f8"), ("event_time", "<f8"),
     ("x", "<u4"), ("y", "<u4"), ("index", "<u4"), ("pad", "<u4")])
DISPERSAL_DTYPE = np.dtype(
    [("gref", "<u8"), ("prior_time", "<f8"), ("event_time", "<f8"),
     ("x", "<u4"), ("y", "<u4"), ("index", "<u4"),
     ("tx", "<u4"), ("ty", "<u4"), ("tindex", "<u4"), ("pad", "<u4"), ("pad2", "<u4")])
LINEAGE_DTYPE = np.dtype(
    [("gref", "<u8"), ("last_event_time", "<f8"),
     ("x", "<u4"), ("y", "<u4"), ("index", "<u4"), ("pad", "<u4")])

assert SPECIATION_DTYPE.itemsize == 40
assert DISPERSAL_DTYPE.itemsize == 56
assert LINEAGE_DTYPE.itemsize == 32


class OracleAliasTables(ctypes.Structure):
    _fields_ = [
        ("n_cells", ctypes.c_uint64),
        ("n_atoms", ctypes.c_uint64),
        ("range_start", ctypes.POINTER(ctypes.c_uint64)),
        ("range_end", ctypes.POINTER(ctypes.c_uint64)),
        ("self_dispersal", ctypes.POINTER(ctypes.c_double)),
        ("non_self_event", ctypes.POINTER(ctypes.c_uint64)),
        ("atom_u", ctypes.POINTER(ctypes.c_double)),
        ("atom_e", ctypes.POINTER(ctypes.c_uint32)),
        ("atom_k", ctypes.POINTER(ctypes.c_uint32)),
    ]


_lib = None


def build():
    """Compile the oracle library in place (gcc, see oracle/Makefile)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp = ctypes.c_void_p
        u64 = ctypes.c_uint64
        L.oracle_simulate.argtypes = [ctypes.POINTER(OracleScenario), ctypes.POINTER(OracleArgs),
                                      u64, ctypes.c_double, ctypes.POINTER(OracleResult),
                                      vp, u64, vp, u64, vp, u64]
        L.oracle_simulate.restype = ctypes.c_int
        L.oracle_simulate_lineages.argtypes = [
            ctypes.POINTER(OracleScenario), ctypes.POINTER(OracleArgs), u64, vp, u64,
            ctypes.c_double, ctypes.c_double, ctypes.POINTER(OracleResult), vp, u64, vp, u64,
            vp, u64]
        L.oracle_simulate_lineages.restype = ctypes.c_int
        L.oracle_seed_from_u64.argtypes = [u64]
        L.oracle_seed_from_u64.restype = u64
        L.oracle_wyhash_sequence.argtypes = [u64, u64, u64, vp, u64]
        L.oracle_wyhash_sequence.restype = None
        L.oracle_seahash_diffuse.argtypes = [u64]
        L.oracle_seahash_diffuse.restype = u64
        L.oracle_wymum.argtypes = [u64, u64]
        L.oracle_wymum.restype = u64
        L.oracle_poisson_next_event_time.argtypes = [u64, u64, ctypes.c_double, ctypes.c_double,
                                                     ctypes.c_double, ctypes.POINTER(u64)]
        L.oracle_poisson_next_event_time.restype = ctypes.c_double
        L.oracle_exp_next_event_time.argtypes = [u64, u64, ctypes.c_double, ctypes.c_double,
                                                 ctypes.c_double, ctypes.POINTER(u64)]
        L.oracle_exp_next_event_time.restype = ctypes.c_double
        L.oracle_ln.argtypes = [vp, vp, u64]
        L.oracle_ln.restype = None
        L.oracle_count_origins.argtypes = [ctypes.POINTER(OracleScenario)]
        L.oracle_count_origins.restype = ctypes.c_int64
        L.oracle_enumerate_origins.argtypes = [ctypes.POINTER(OracleScenario), vp, u64]
        L.oracle_enumerate_origins.restype = ctypes.c_int64
        L.oracle_build_alias.argtypes = [ctypes.POINTER(OracleScenario),
                                         ctypes.POINTER(OracleAliasTables)]
        L.oracle_build_alias.restype = ctypes.c_int
        L.oracle_free_alias.argtypes = [ctypes.POINTER(OracleAliasTables)]
        L.oracle_free_alias.restype = None
        L.oracle_check_dispersal_contract.argtypes = [ctypes.POINTER(OracleScenario)]
        L.oracle_check_dispersal_contract.restype = ctypes.c_int
        L.oracle_normal_dispersal.argtypes = [u64, u64, ctypes.c_double, ctypes.c_uint32,
                                              ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32),
                                              ctypes.POINTER(ctypes.c_uint32)]
        L.oracle_normal_dispersal.restype = None
        L.oracle_displacements.argtypes = [ctypes.c_int32, vp, u64, ctypes.c_double, ctypes.c_double, vp, vp]
        L.oracle_displacements.restype = None
        L.oracle_clark2dt_dispersal.argtypes = [u64, u64, ctypes.c_double, ctypes.c_double, ctypes.c_uint32,
                                                ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32),
                                                ctypes.POINTER(ctypes.c_uint32)]
        L.oracle_clark2dt_dispersal.restype = None
        L.oracle_clark2dt_cdf_inverse.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.oracle_clark2dt_cdf_inverse.restype = ctypes.c_double
        f64 = ctypes.c_double
        L.oracle_wrapping_noise.argtypes = [ctypes.c_int64, f64, f64, u64, ctypes.c_uint32, ctypes.c_uint32]
        L.oracle_wrapping_noise.restype = f64
        L.oracle_wrapping_noise_threshold.argtypes = [ctypes.c_int64, f64, f64, f64, u64]
        L.oracle_wrapping_noise_threshold.restype = f64
        L.oracle_wrapping_noise_self_dispersal.argtypes = [f64, f64]
        L.oracle_wrapping_noise_self_dispersal.restype = f64
        _lib = L
    return _lib


def make_scenario(desc):
    """Build an OracleScenario from a plain dict scenario description.

    Keeps references to numpy arrays alive on the returned object."""
    sc = OracleScenario()
    sc.kind = desc["kind"]
    sc.speciation_probability = desc["speciation_probability"]
    sc.turnover_rate = desc.get("turnover_rate", 0.5)
    sc.width = desc.get("width", 0)
    sc.height = desc.get("height", 0)
    sc.deme = desc.get("deme", 0)
    sc.meta_width = desc.get("meta_width", 0)
    sc.meta_height = desc.get("meta_height", 0)
    sc.meta_deme = desc.get("meta_deme", 0)
    sc.migration_probability = desc.get("migration_probability", 0.0)
    sc.sigma = desc.get("sigma", 0.0)
    sc.centre_x = desc.get("centre_x", 0)
    sc.centre_y = desc.get("centre_y", 0)
    sc.radius = desc.get("radius", 0)
    sc.shape_u = desc.get("shape_u", 0.0)
    sc.tail_p = desc.get("tail_p", 0.0)
    sc.noise_seed = desc.get("noise_seed", 0)
    sc.coverage = desc.get("coverage", 0.0)
    sc.scale = desc.get("scale", 0.0)
    sc.persistence = desc.get("persistence", 0.0)
    sc.octaves = desc.get("octaves", 0)
    sample = desc.get("sample", (0, 0, 0, 0))  # Rectangle: (x, y, width, height)
    sc.sample_x, sc.sample_y, sc.sample_width, sc.sample_height = sample
    keep = []
    if desc.get("habitat") is not None:
        h = np.ascontiguousarray(desc["habitat"], dtype=np.uint32)
        keep.append(h)
        sc.habitat = h.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
    if desc.get("turnover_map") is not None:
        t = np.ascontiguousarray(desc["turnover_map"], dtype=np.float64)
        keep.append(t)
        sc.turnover = t.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    if desc.get("dispersal") is not None:
        d = np.ascontiguousarray(desc["dispersal"], dtype=np.float64)
        keep.append(d)
        sc.dispersal = d.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    sc._keep = keep
    return sc


def make_args(mode=MODE_REFERENCE, delta_t=2.0, step_slice=10, dedup_factor=1.0,
              event_slice_factor=2.0, min_round_events=0, report_dispersal=False,
              partition=(0, 1), step_slice_max=0, event_time_sampler=SAMPLER_POISSON):
    a = OracleArgs()
    a.delta_t = delta_t
    a.step_slice = step_slice
    a.dedup_factor = dedup_factor
    a.event_slice_factor = event_slice_factor
    a.min_round_events = min_round_events
    a.report_dispersal = 1 if report_dispersal else 0
    a.mode = mode
    a.partition_rank = partition[0]
    a.partition_size = partition[1]
    a.step_slice_max = step_slice_max
    a.event_time_sampler = event_time_sampler
    return a


class OracleOutcome:
    def __init__(self, result, speciation, dispersal, remaining):
        self.status = result.status
        self.time = result.time
        self.steps = result.steps
        self.n_initial = result.n_initial
        self.n_remaining = result.n_remaining
        self.n_speciation = result.n_speciation
        self.biodiversity = result.biodiversity
        self.n_dispersal = result.n_dispersal
        self.n_primes = result.n_primes
        self.n_draws = result.n_draws
        self.n_rounds = result.n_rounds
        self.n_dedup = result.n_dedup
        self.speciation = speciation
        self.dispersal = dispersal
        self.remaining = remaining


def simulate(desc, seed, mode=MODE_REFERENCE, pause_before=None, report_dispersal=False,
             lineages=None, resume_time=0.0, speciation_cap=None, dispersal_cap=None, **kw):
    """Run the oracle on a scenario dict; returns an OracleOutcome."""
    L = lib()
    sc = make_scenario(desc)
    args = make_args(mode=mode, report_dispersal=report_dispersal, **kw)
    if lineages is not None:
        n0 = len(lineages)
    else:
        n0 = L.oracle_count_origins(ctypes.byref(sc))
        if n0 < 0:
            raise ValueError("invalid scenario (%d)" % n0)
    cap = speciation_cap if speciation_cap is not None else max(n0, 1)
    spec = np.zeros(cap, dtype=SPECIATION_DTYPE)
    dcap = (dispersal_cap or 0) if report_dispersal else 0
    disp = np.zeros(max(dcap, 1), dtype=DISPERSAL_DTYPE)
    lin = np.zeros(max(n0, 1), dtype=LINEAGE_DTYPE)
    res = OracleResult()
    pb = -1.0 if pause_before is None else float(pause_before)
    if lineages is not None:
        lins = np.ascontiguousarray(lineages, dtype=LINEAGE_DTYPE)
        rc = L.oracle_simulate_lineages(ctypes.byref(sc), ctypes.byref(args), seed,
                                        lins.ctypes.data, len(lins), resume_time, pb,
                                        ctypes.byref(res), spec.ctypes.data, cap,
                                        disp.ctypes.data, dcap, lin.ctypes.data, len(lin))
    else:
        rc = L.oracle_simulate(ctypes.byref(sc), ctypes.byref(args), seed, pb, ctypes.byref(res),
                               spec.ctypes.data, cap, disp.ctypes.data, dcap,
                               lin.ctypes.data, len(lin))
    if rc != 0:
        raise RuntimeError("oracle_simulate failed with status %d" % rc)
    nspec = min(res.n_speciation, cap)
    return OracleOutcome(res, spec[:nspec].copy(), disp[:min(res.n_dispersal, dcap)].copy(),
                         lin[:res.n_remaining].copy())


def seed_from_u64(seed):
    return lib().oracle_seed_from_u64(seed)


def wyhash_sequence(seed, location, time_index, n):
    out = np.zeros(n, dtype=np.uint64)
    lib().oracle_wyhash_sequence(seed, location, time_index, out.ctypes.data, n)
    return out


def poisson_next_event_time(seed, injection, t, lam=0.5, delta_t=2.0):
    rp = ctypes.c_uint64(0)
    v = lib().oracle_poisson_next_event_time(seed, injection, t, lam, delta_t, ctypes.byref(rp))
    return v, rp.value


def exp_next_event_time(seed, injection, t, lam=0.5, delta_t=2.0):
    rp = ctypes.c_uint64(0)
    v = lib().oracle_exp_next_event_time(seed, injection, t, lam, delta_t, ctypes.byref(rp))
    return v, rp.value


def ln(x):
    """The shared correctly rounded logarithm (ln_dd.h) of values in (0, 1]."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    lib().oracle_ln(x.ctypes.data, out.ctypes.data, x.size)
    return out


def enumerate_origins(desc):
    L = lib()
    sc = make_scenario(desc)
    n = L.oracle_count_origins(ctypes.byref(sc))
    out = np.zeros(max(n, 1), dtype=LINEAGE_DTYPE)
    L.oracle_enumerate_origins(ctypes.byref(sc), out.ctypes.data, n)
    return out[:n]


def build_alias(desc):
    """Reference packed separable alias tables as numpy arrays."""
    L = lib()
    sc = make_scenario(desc)
    t = OracleAliasTables()
    rc = L.oracle_build_alias(ctypes.byref(sc), ctypes.byref(t))
    if rc:
        raise RuntimeError("alias build failed")
    nc, na = t.n_cells, t.n_atoms
    out = {
        "range_start": np.ctypeslib.as_array(t.range_start, (nc,)).copy(),
        "range_end": np.ctypeslib.as_array(t.range_end, (nc,)).copy(),
        "self_dispersal": np.ctypeslib.as_array(t.self_dispersal, (nc,)).copy(),
        "non_self_event": np.ctypeslib.as_array(t.non_self_event, (nc,)).copy(),
        "atom_u": np.ctypeslib.as_array(t.atom_u, (max(na, 1),))[:na].copy(),
        "atom_e": np.ctypeslib.as_array(t.atom_e, (max(na, 1),))[:na].copy(),
        "atom_k": np.ctypeslib.as_array(t.atom_k, (max(na, 1),))[:na].copy(),
    }
    L.oracle_free_alias(ctypes.byref(t))
    return out


def check_dispersal_contract(desc):
    return lib().oracle_check_dispersal_contract(ctypes.byref(make_scenario(desc)))


def normal_dispersal(d0, d1, sigma, x, y):
    tx = ctypes.c_uint32(0)
    ty = ctypes.c_uint32(0)
    lib().oracle_normal_dispersal(d0, d1, sigma, x, y, ctypes.byref(tx), ctypes.byref(ty))
    return tx.value, ty.value


def displacements(kind, draws, a, b=0.0):
    """Raw AlmostInfinite displacements (dx, dy) with the C library's
    log/sin/cos/pow: kind ALMOST_INFINITE_NORMAL (a = sigma) or
    ALMOST_INFINITE_CLARK2DT (a = shape u, b = tail p); draws is [n, 2] u64."""
    d = np.ascontiguousarray(draws, dtype=np.uint64)
    n = d.shape[0]
    dx = np.empty(n, dtype=np.float64)
    dy = np.empty(n, dtype=np.float64)
    lib().oracle_displacements(kind, d.ctypes.data, n, a, b, dx.ctypes.data, dy.ctypes.data)
    return dx, dy


def distinct_speciation_set(events):
    """Sorted unique (event_time bits, x, y, index) keys -- the parity set."""
    if len(events) == 0:
        return np.zeros((0, 4), dtype=np.uint64)
    k = np.stack([events["event_time"].view(np.uint64), events["x"].astype(np.uint64),
                  events["y"].astype(np.uint64), events["index"].astype(np.uint64)], axis=1)
    return np.unique(k, axis=0)


def clark2dt_cdf_inverse(u01, shape_u, tail_p):
    """clark2dt::cdf_inverse: the Clark2Dt jump distance for a uniform u01."""
    return lib().oracle_clark2dt_cdf_inverse(u01, shape_u, tail_p)


def clark2dt_dispersal(d0, d1, shape_u, tail_p, x, y):
    tx, ty = ctypes.c_uint32(), ctypes.c_uint32()
    lib().oracle_clark2dt_dispersal(d0, d1, shape_u, tail_p, x, y, ctypes.byref(tx), ctypes.byref(ty))
    return tx.value, ty.value


def wrapping_noise(seed, scale, persistence, octaves, x, y):
    """sum_noise_octaves at (x, y) for the noise seeded with `seed`."""
    return lib().oracle_wrapping_noise(seed, scale, persistence, octaves, x, y)


def wrapping_noise_threshold(seed, coverage, scale, persistence, octaves):
    """WrappingNoiseHabitat's habitable-noise threshold."""
    return lib().oracle_wrapping_noise_threshold(seed, coverage, scale, persistence, octaves)


def wrapping_noise_self_dispersal(sigma, coverage):
    """The approximate Normal dispersal's self-dispersal probability."""
    return lib().oracle_wrapping_noise_self_dispersal(sigma, coverage)
