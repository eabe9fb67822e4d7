"""necsim-rust B200 backend: the Independent coalescence algorithm on sm_100a.

Python mirror of the reference's `rustcoalescence simulate` interface for
this path (RON arguments ``speciation``, ``sample``, ``rng``, ``scenario``,
``algorithm``, ``pause``, ``reporters``; docs/simulate.ron), calling the
C ABI in ``include/necsim_b200.h`` through ctypes.  The CUDA library must be
built (``build.py``); there is no CPU fallback: importing this package on a
machine without the library raises, and simulating without a GPU fails with
the CUDA error the library reports.
"""
import ctypes
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

from . import build as _build

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = _build.LIB

NON_SPATIAL = 0
SPATIALLY_IMPLICIT = 1
ALMOST_INFINITE_NORMAL = 2
ALMOST_INFINITE_CLARK2DT = 4
SPATIALLY_EXPLICIT = 3
WRAPPING_NOISE = 5

ERRORS = {
    -1: "invalid argument", -2: "CUDA error", -3: "out of memory", -4: "device bound check",
    -5: "device wait timeout", -6: "dispersal map contract violated", -7: "empty habitat map",
    -8: "unsupported", -9: "reporter stopped delivery", -10: "too large",
    -11: "dispersal target rejected too often",
}


class NecsimError(RuntimeError):
    def __init__(self, code, message):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "error"), code, message))
        self.code = code


# ---------------------------------------------------------------------------
# ctypes mirror of include/necsim_b200.h
# ---------------------------------------------------------------------------
class CScenario(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32), ("reserved0", ctypes.c_uint32),
        ("speciation_probability", ctypes.c_double), ("turnover_rate", ctypes.c_double),
        ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("deme", ctypes.c_uint32),
        ("meta_width", ctypes.c_uint32), ("meta_height", ctypes.c_uint32),
        ("meta_deme", ctypes.c_uint32),
        ("migration_probability", ctypes.c_double), ("sigma", ctypes.c_double),
        ("centre_x", ctypes.c_uint32), ("centre_y", ctypes.c_uint32),
        ("radius", ctypes.c_uint32), ("reserved1", ctypes.c_uint32),
        ("habitat", ctypes.POINTER(ctypes.c_uint32)),
        ("dispersal", ctypes.POINTER(ctypes.c_double)),
        ("shape_u", ctypes.c_double), ("tail_p", ctypes.c_double),
        ("turnover_map", ctypes.POINTER(ctypes.c_double)),
        ("noise_seed", ctypes.c_int64), ("coverage", ctypes.c_double),
        ("scale", ctypes.c_double), ("persistence", ctypes.c_double),
        ("octaves", ctypes.c_uint64),
        ("sample_x", ctypes.c_uint32), ("sample_y", ctypes.c_uint32),
        ("sample_width", ctypes.c_uint64), ("sample_height", ctypes.c_uint64),
        ("cells", ctypes.c_void_p), ("atoms", ctypes.c_void_p), ("n_atoms", ctypes.c_uint64),
    ]


class CArgs(ctypes.Structure):
    _fields_ = [
        ("delta_t", ctypes.c_double), ("step_slice", ctypes.c_uint64),
        ("min_round_events", ctypes.c_uint64), ("step_slice_max", ctypes.c_uint64),
        ("block_size", ctypes.c_uint32),
        ("grid_size", ctypes.c_uint32), ("dedup_factor_pct", ctypes.c_uint32),
        ("schedule", ctypes.c_uint32), ("report_dispersal", ctypes.c_int32),
        ("device", ctypes.c_int32), ("rounds_per_graph", ctypes.c_uint32),
        ("resident", ctypes.c_uint32), ("event_time_sampler", ctypes.c_uint32),
        ("model", ctypes.c_void_p), ("max_rounds", ctypes.c_uint64),
        ("priority_sims", ctypes.c_uint32), ("priority_groups", ctypes.c_uint32),
        ("priority_list", ctypes.c_void_p),
        ("reserve_sms", ctypes.c_uint32), ("priority_engines", ctypes.c_uint32),
    ]


class COutcome(ctypes.Structure):
    _fields_ = [
        ("paused", ctypes.c_int32), ("pad", ctypes.c_int32), ("time", ctypes.c_double),
        ("steps", ctypes.c_uint64), ("n_initial", ctypes.c_uint64),
        ("n_remaining", ctypes.c_uint64), ("n_speciation", ctypes.c_uint64),
        ("biodiversity", ctypes.c_uint64), ("n_dispersal", ctypes.c_uint64),
        ("n_rounds", ctypes.c_uint64), ("n_dedup", ctypes.c_uint64),
        ("n_launches", ctypes.c_uint64), ("kernel_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double), ("h2d_bytes", ctypes.c_uint64),
        ("d2h_bytes", ctypes.c_uint64), ("n_step_launches", ctypes.c_uint64),
        ("lineage_visits", ctypes.c_uint64), ("resident_ms", ctypes.c_double),
        ("end_ms", ctypes.c_double), ("routed_ms", ctypes.c_double),
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
CELL_DTYPE = np.dtype(
    [("injection", "<u8"), ("self_dispersal", "<f8"), ("atom_start", "<u4"),
     ("atom_count", "<u4"), ("habitat", "<u4"), ("non_self_event", "<u4")])
ATOM_DTYPE = np.dtype([("u", "<f8"), ("e", "<u4"), ("k", "<u4")])

_SPEC_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64)
_DISP_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64)


class CReporter(ctypes.Structure):
    _fields_ = [("user", ctypes.c_void_p), ("report_speciation", _SPEC_CB),
                ("report_dispersal", _DISP_CB)]


SYMBOLS = [
    "necsim_abi_version", "necsim_seed_from_u64", "necsim_gpu_create", "necsim_gpu_simulate",
    "necsim_gpu_simulate_lineages", "necsim_gpu_remaining_lineages",
    "necsim_gpu_simulate_batch", "necsim_gpu_last_error", "necsim_gpu_destroy",
    "necsim_build_tables", "necsim_enumerate_origins", "necsim_subdomain_ranks", "necsim_gpu_batch_create",
    "necsim_gpu_batch_run", "necsim_gpu_batch_last_error", "necsim_gpu_batch_destroy",
    "necsim_model_create", "necsim_model_destroy", "necsim_model_last_error",
    "necsim_model_get_weights", "necsim_model_set_weights", "necsim_model_predict",
    "necsim_model_gradients", "necsim_model_train", "necsim_gpu_trace_batch",
    "necsim_presample_origins", "necsim_gpu_autotune", "necsim_event_log_create",
    "necsim_event_log_reporter", "necsim_event_log_close", "necsim_event_log_replay", "necsim_map_load",
    "necsim_map_free", "necsim_maps_fix", "necsim_gpu_hash_peak", "necsim_gpu_displacements",
    "necsim_gpu_batch_priority",
]

_lib = None


def lib():
    """Loads the CUDA backend library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libnecsim_b200.so is not built: run `python necsim-rust_b200/build.py` "
                          "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    u64 = ctypes.c_uint64
    L.necsim_abi_version.restype = ctypes.c_int
    L.necsim_seed_from_u64.argtypes = [u64]
    L.necsim_seed_from_u64.restype = u64
    L.necsim_gpu_create.argtypes = [P(CScenario), P(CArgs), P(vp)]
    L.necsim_gpu_create.restype = ctypes.c_int
    L.necsim_gpu_simulate.argtypes = [vp, u64, ctypes.c_double, P(CReporter), P(COutcome)]
    L.necsim_gpu_simulate.restype = ctypes.c_int
    L.necsim_gpu_simulate_lineages.argtypes = [vp, vp, u64, ctypes.c_double, u64,
                                               ctypes.c_double, P(CReporter), P(COutcome)]
    L.necsim_gpu_simulate_lineages.restype = ctypes.c_int
    L.necsim_gpu_remaining_lineages.argtypes = [vp, vp, u64, P(u64)]
    L.necsim_gpu_remaining_lineages.restype = ctypes.c_int
    L.necsim_gpu_simulate_batch.argtypes = [P(CScenario), P(u64), ctypes.c_uint32, P(CArgs),
                                            ctypes.c_double, vp, P(COutcome), ctypes.c_char_p,
                                            ctypes.c_size_t]
    L.necsim_gpu_simulate_batch.restype = ctypes.c_int
    L.necsim_gpu_last_error.argtypes = [vp]
    L.necsim_gpu_last_error.restype = ctypes.c_char_p
    L.necsim_gpu_destroy.argtypes = [vp]
    L.necsim_gpu_destroy.restype = None
    L.necsim_build_tables.argtypes = [P(CScenario), vp, vp, u64, P(u64)]
    L.necsim_build_tables.restype = ctypes.c_int
    L.necsim_enumerate_origins.argtypes = [P(CScenario), vp, u64, P(u64)]
    L.necsim_enumerate_origins.restype = ctypes.c_int
    L.necsim_subdomain_ranks.argtypes = [P(CScenario), ctypes.c_uint32, vp, u64, vp, P(ctypes.c_int32)]
    L.necsim_subdomain_ranks.restype = ctypes.c_int
    L.necsim_gpu_batch_create.argtypes = [P(CScenario), P(u64), ctypes.c_uint32, P(CArgs),
                                          ctypes.c_double, P(vp)]
    L.necsim_gpu_batch_create.restype = ctypes.c_int
    L.necsim_gpu_batch_run.argtypes = [vp, vp, P(COutcome)]
    L.necsim_gpu_batch_run.restype = ctypes.c_int
    L.necsim_gpu_batch_last_error.argtypes = [vp]
    L.necsim_gpu_batch_last_error.restype = ctypes.c_char_p
    L.necsim_gpu_batch_destroy.argtypes = [vp]
    L.necsim_gpu_batch_destroy.restype = None
    fp = P(ctypes.c_float)
    L.necsim_gpu_autotune.argtypes = [P(CScenario), P(u64), ctypes.c_uint32, P(CArgs), ctypes.c_double, u64,
                                      P(CArgs), vp, ctypes.c_uint32, P(ctypes.c_uint32), ctypes.c_char_p,
                                      ctypes.c_size_t]
    L.necsim_gpu_autotune.restype = ctypes.c_int
    L.necsim_event_log_create.argtypes = [ctypes.c_char_p, u64, ctypes.c_int32, ctypes.c_int32, P(vp)]
    L.necsim_event_log_create.restype = ctypes.c_int
    L.necsim_event_log_reporter.argtypes = [vp]
    L.necsim_event_log_reporter.restype = CReporter
    L.necsim_event_log_close.argtypes = [vp]
    L.necsim_event_log_close.restype = ctypes.c_int
    L.necsim_presample_origins.argtypes = [u64, ctypes.c_double, ctypes.c_uint32, ctypes.c_uint32, vp, u64, P(u64)]
    L.necsim_presample_origins.restype = ctypes.c_int
    L.necsim_map_load.argtypes = [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, P(vp), P(ctypes.c_uint32),
                                  P(ctypes.c_uint32), ctypes.c_char_p, ctypes.c_size_t]
    L.necsim_map_load.restype = ctypes.c_int
    L.necsim_map_free.argtypes = [vp]
    L.necsim_map_free.restype = None
    L.necsim_maps_fix.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, vp, u64, u64, vp, ctypes.c_int32,
                                  ctypes.c_char_p, ctypes.c_size_t]
    L.necsim_maps_fix.restype = ctypes.c_int
    L.necsim_event_log_replay.argtypes = [vp, u64, u64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                          P(CReporter), P(u64), ctypes.c_char_p, ctypes.c_size_t]
    L.necsim_event_log_replay.restype = ctypes.c_int
    L.necsim_gpu_hash_peak.argtypes = [ctypes.c_int32, P(ctypes.c_double)]
    L.necsim_gpu_hash_peak.restype = ctypes.c_int
    L.necsim_gpu_displacements.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_uint64,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    L.necsim_gpu_displacements.restype = ctypes.c_int
    L.necsim_gpu_batch_priority.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                            ctypes.POINTER(ctypes.c_uint32)]
    L.necsim_gpu_batch_priority.restype = ctypes.c_int
    L.necsim_model_create.argtypes = [ctypes.c_int32, u64, P(vp)]
    L.necsim_model_create.restype = ctypes.c_int
    L.necsim_model_destroy.argtypes = [vp]
    L.necsim_model_destroy.restype = None
    L.necsim_model_last_error.argtypes = [vp]
    L.necsim_model_last_error.restype = ctypes.c_char_p
    L.necsim_model_get_weights.argtypes = [vp, fp]
    L.necsim_model_get_weights.restype = ctypes.c_int
    L.necsim_model_set_weights.argtypes = [vp, fp]
    L.necsim_model_set_weights.restype = ctypes.c_int
    L.necsim_model_predict.argtypes = [vp, fp, u64, fp]
    L.necsim_model_predict.restype = ctypes.c_int
    L.necsim_model_gradients.argtypes = [vp, fp, fp, u64, fp, P(ctypes.c_double)]
    L.necsim_model_gradients.restype = ctypes.c_int
    L.necsim_model_train.argtypes = [vp, fp, fp, u64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float,
                                     u64, P(ctypes.c_double)]
    L.necsim_model_train.restype = ctypes.c_int
    L.necsim_gpu_trace_batch.argtypes = [P(CScenario), P(u64), ctypes.c_uint32, P(CArgs), ctypes.c_double,
                                         ctypes.c_uint32, u64, fp, fp, P(u64), ctypes.c_char_p,
                                         ctypes.c_size_t]
    L.necsim_gpu_trace_batch.restype = ctypes.c_int
    if L.necsim_abi_version() != 3:
        raise ImportError("libnecsim_b200.so ABI version mismatch")
    _lib = L
    return L


# ---------------------------------------------------------------------------
# Reference-shaped configuration (docs/simulate.ron)
# ---------------------------------------------------------------------------
@dataclass
class NonSpatial:
    """`NonSpatial(area: (w, h), deme: d)` (scenarios/src/non_spatial.rs)."""
    area: Tuple[int, int]
    deme: int


@dataclass
class SpatiallyImplicit:
    """`SpatiallyImplicit(local_area, local_deme, meta_area, meta_deme, migration)`
    (scenarios/src/spatially_implicit.rs)."""
    local_area: Tuple[int, int]
    local_deme: int
    meta_area: Tuple[int, int]
    meta_deme: int
    migration: float


@dataclass
class Circle:
    """`Circle(centre: (x, y), radius: r)` sample (almost_infinite/mod.rs:92-107)."""
    radius: int
    centre: Tuple[int, int] = (0xFFFFFFFF // 2, 0xFFFFFFFF // 2)


@dataclass
class Normal:
    """`Normal(sigma: s)` dispersal (almost_infinite/normal.rs)."""
    sigma: float


@dataclass
class Clark2Dt:
    """`Clark2Dt(shape_u: u, tail_p: p)` dispersal (almost_infinite/clark2dt.rs;
    dispersal_sampler/almost_infinite_clark2dt.rs)."""
    shape_u: float
    tail_p: float


@dataclass
class AlmostInfinite:
    """`AlmostInfinite(sample: Circle(..) | Rectangle(..), dispersal: Normal(..) | Clark2Dt(..))`
    (almost_infinite/mod.rs:92-122)."""
    sample: object
    dispersal: object


@dataclass
class SpatiallyExplicit:
    """`SpatiallyExplicit(habitat, dispersal, turnover)` with in-memory maps:
    habitat u32 [h, w], dispersal f64 [h*w, h*w]; turnover a uniform rate
    (spatially_explicit/turnover/uniform.rs) or an f64 [h, w] turnover map
    (turnover/map.rs: every habitable cell's rate > 0)."""
    habitat: np.ndarray
    dispersal: Optional[np.ndarray]
    turnover: Union[float, np.ndarray] = 0.5
    # device tables built before (build_tables: CELL_DTYPE records, ATOM_DTYPE
    # atoms), used instead of building them from `dispersal` (then optional)
    tables: Optional[Tuple[np.ndarray, np.ndarray]] = None


@dataclass
class Rectangle:
    """`Rectangle(origin: (x, y), width: w, height: h)` sample
    (LandscapeExtent, necsim/core/src/landscape/extent.rs; wrapping_noise.rs:51-55)."""
    origin: Tuple[int, int]
    width: int
    height: int


@dataclass
class WrappingNoise:
    """`WrappingNoise(seed, coverage, scale, persistence, octaves, sample, sigma)`
    (rustcoalescence/scenarios/src/wrapping_noise.rs): the almost-infinite
    plane, habitable where OpenSimplex octave noise is at most its coverage
    quantile, approximate Normal dispersal of width sigma, origins the
    habitable locations of the Rectangle sample."""
    seed: int
    coverage: float
    scale: float
    persistence: float
    octaves: int
    sample: Rectangle
    sigma: float


MAP_LOADING_MODES = {"OffByOne": 0, "FixMe": 1, "Strict": 2}


def load_map(path: str, dtype: str = "u32", strict: bool = False) -> np.ndarray:
    """A one-band (Geo)TIFF map as a [height, width] array: "u32" for habitat
    maps, "f64" for dispersal and turnover maps (maps/tiff/mod.rs
    load_map_from_tiff; GDAL no-data samples become 0 unless `strict`)."""
    if dtype not in ("u32", "f64"):
        raise ValueError("dtype must be 'u32' or 'f64'")
    L = lib()
    data = ctypes.c_void_p()
    w, h = ctypes.c_uint32(), ctypes.c_uint32()
    err = ctypes.create_string_buffer(512)
    rc = L.necsim_map_load(os.fsencode(path), 0 if dtype == "u32" else 1, int(bool(strict)), ctypes.byref(data),
                           ctypes.byref(w), ctypes.byref(h), err, 512)
    if rc != 0:
        raise NecsimError(rc, err.value.decode())
    try:
        n = w.value * h.value
        ct = ctypes.c_uint32 if dtype == "u32" else ctypes.c_double
        arr = np.ctypeslib.as_array(ctypes.cast(data, ctypes.POINTER(ct)), shape=(n,)).copy()
    finally:
        L.necsim_map_free(data)
    return arr.reshape(h.value, w.value)


def fix_maps(habitat: np.ndarray, dispersal: np.ndarray, turnover: Optional[np.ndarray] = None,
             mode: str = "OffByOne"):
    """The reference's map fix-ups for a loading mode (maps/mod.rs:56-215) on
    copies of the maps: returns (habitat, dispersal)."""
    if mode not in MAP_LOADING_MODES:
        raise ValueError("mode must be one of %s" % sorted(MAP_LOADING_MODES))
    hab = np.ascontiguousarray(habitat, dtype=np.uint32).copy()
    disp = np.ascontiguousarray(dispersal, dtype=np.float64).copy()
    if hab.ndim != 2 or disp.ndim != 2:
        raise ValueError("habitat and dispersal must be 2-D")
    tv = None
    if turnover is not None:
        tv = np.ascontiguousarray(turnover, dtype=np.float64)
        if tv.shape != hab.shape:
            raise ValueError("the turnover map must have the habitat map's shape")
    err = ctypes.create_string_buffer(512)
    rc = lib().necsim_maps_fix(hab.ctypes.data, hab.shape[1], hab.shape[0], disp.ctypes.data, disp.shape[0],
                               disp.shape[1], tv.ctypes.data if tv is not None else None,
                               MAP_LOADING_MODES[mode], err, 512)
    if rc != 0:
        raise NecsimError(rc, err.value.decode())
    return hab, disp


def spatially_explicit_from_maps(habitat_path: str, dispersal_path: str, turnover: Union[float, str] = 0.5,
                                 mode: str = "OffByOne") -> "SpatiallyExplicit":
    """`SpatiallyExplicit(habitat: "...", dispersal: "...", turnover:
    Uniform(rate) | Map("..."), mode: ...)` (spatially_explicit/turnover/
    uniform.rs and map.rs try_load): the dispersal map, then the turnover map
    when given as a path, then the habitat map, loaded and fixed up as the
    loading mode says."""
    strict = mode == "Strict"
    disp = load_map(dispersal_path, "f64", strict)
    tmap = load_map(turnover, "f64", strict) if isinstance(turnover, (str, bytes, os.PathLike)) else None
    hab = load_map(habitat_path, "u32", strict)
    hab, disp = fix_maps(hab, disp, tmap, mode)
    return SpatiallyExplicit(hab, disp, tmap if tmap is not None else turnover)


@dataclass
class CUDA:
    """`CUDA(...)` algorithm arguments (algorithms/cuda/src/arguments.rs) for
    this backend; defaults follow the Independent algorithm's where results
    depend on them (delta_t 2.0)."""
    delta_t: float = 2.0
    step_slice: int = 10
    block_size: int = 0
    grid_size: int = 0
    min_round_events: int = 1 << 20
    step_slice_max: int = 1024
    dedup_factor_pct: int = 200
    schedule: str = "plain"   # or "learned" (needs `model`)
    device: int = 0
    rounds_per_graph: int = 16
    # batches: simulations with few live lineages move to the per-simulation
    # resident kernel (True: at 8 lineages; an int 2..256: at that many)
    resident: Union[bool, int] = False
    model: Optional["LifetimeModel"] = None
    # reporters consume dispersal events (ReportDispersal): the events leave
    # the device after every round (global rounds only, no CUDA graphs)
    report_dispersal: bool = False
    # "poisson": PoissonEventTimeSampler, the Independent algorithm's
    # (event_time_sampler/poisson.rs); "exp": ExpEventTimeSampler, the CUDA
    # algorithm's (event_time_sampler/exp.rs), -ln(U(0,1]) / lambda per event
    event_time_sampler: str = "poisson"
    # watchdog: a run still active after this many rounds fails with
    # NECSIM_E_TIMEOUT (checked between graph launches); 0: 2^26
    max_rounds: int = 0
    # batches: simulations run in one priority engine beside the others
    # (their own rounds); `priority_list` names them (batch indices), else the
    # learned schedule's model picks `priority_sims` of them (default 8)
    priority_sims: int = 0
    priority_list: Optional[Sequence[int]] = None
    # batches: the other simulations in this many engines of decreasing CUDA
    # stream priority (the learned model's longest-lived first, else batch order)
    priority_groups: int = 0
    # batches with a priority engine: this many SMs run the priority engine's
    # tails alone once its live lineages fit them (0: off)
    reserve_sms: int = 0
    # batches: the priority simulations split into this many engines (0: one
    # engine), so a long tail waits for fewer other ones' bulk
    priority_engines: int = 0


Independent = CUDA

EVENT_TIME_SAMPLERS = {"poisson": 0, "exp": 1}


@dataclass
class Outcome:
    paused: bool
    time: float
    steps: int
    n_initial: int
    n_remaining: int
    n_speciation: int
    biodiversity: int
    n_rounds: int
    n_dedup: int
    n_launches: int
    kernel_ms: float
    total_ms: float
    h2d_bytes: int = 0
    d2h_bytes: int = 0
    n_step_launches: int = 0
    lineage_visits: int = 0
    resident_ms: float = 0.0
    speciation: Optional[np.ndarray] = None
    remaining: Optional[np.ndarray] = None
    n_dispersal: int = 0
    dispersal: Optional[np.ndarray] = None   # with CUDA(report_dispersal=True), collect=True
    delivery: Optional[list] = None          # reporter calls in order: ("s" | "d", count)
    # device-clock ms after the run's (a batch's) first round began: when the
    # simulation ended or paused, and when the resident kernel took it over
    # (-1: never)
    end_ms: float = 0.0
    routed_ms: float = -1.0


def presample_origins(n: int, percentage: float = 1.0, rank: int = 0, size: int = 1) -> np.ndarray:
    """Positions (in enumerate_origins order) of the origins that
    `Sample(percentage: p)` and an IsolatedIndividuals partition (rank, size)
    select among the first n (origin_sampler/pre_sampler.rs:48-112)."""
    L = lib()
    k = ctypes.c_uint64()
    rc = L.necsim_presample_origins(n, percentage, rank, size, None, 0, ctypes.byref(k))
    if rc != 0:
        raise NecsimError(rc, "invalid percentage or partition")
    out = np.zeros(max(k.value, 1), dtype=np.uint64)
    rc = L.necsim_presample_origins(n, percentage, rank, size, out.ctypes.data, k.value, ctypes.byref(k))
    if rc != 0:
        raise NecsimError(rc, "invalid percentage or partition")
    return out[:k.value]


DRIVER = os.path.join(os.path.dirname(LIB_PATH), "necsim-b200")


def seed_from_u64(seed: int) -> int:
    """WyHash seed word of `rng: Seed(seed)` (core/src/cogs/rng.rs:33-63)."""
    return int(lib().necsim_seed_from_u64(seed))


def _scenario_struct(scenario, speciation: float):
    c = CScenario()
    c.speciation_probability = speciation
    c.turnover_rate = 0.5
    keep = []
    if isinstance(scenario, NonSpatial):
        c.kind = NON_SPATIAL
        c.width, c.height = scenario.area
        c.deme = scenario.deme
    elif isinstance(scenario, SpatiallyImplicit):
        c.kind = SPATIALLY_IMPLICIT
        c.width, c.height = scenario.local_area
        c.deme = scenario.local_deme
        c.meta_width, c.meta_height = scenario.meta_area
        c.meta_deme = scenario.meta_deme
        c.migration_probability = scenario.migration
    elif isinstance(scenario, AlmostInfinite):
        if isinstance(scenario.dispersal, Clark2Dt):
            c.kind = ALMOST_INFINITE_CLARK2DT
            c.shape_u = scenario.dispersal.shape_u
            c.tail_p = scenario.dispersal.tail_p
        else:
            c.kind = ALMOST_INFINITE_NORMAL
            c.sigma = scenario.dispersal.sigma
        if isinstance(scenario.sample, Rectangle):
            c.sample_x, c.sample_y = scenario.sample.origin
            c.sample_width, c.sample_height = scenario.sample.width, scenario.sample.height
        else:
            c.centre_x, c.centre_y = scenario.sample.centre
            c.radius = scenario.sample.radius
    elif isinstance(scenario, WrappingNoise):
        c.kind = WRAPPING_NOISE
        c.noise_seed = scenario.seed
        c.coverage = scenario.coverage
        c.scale = scenario.scale
        c.persistence = scenario.persistence
        c.octaves = scenario.octaves
        c.sigma = scenario.sigma
        c.sample_x, c.sample_y = scenario.sample.origin
        c.sample_width, c.sample_height = scenario.sample.width, scenario.sample.height
    elif isinstance(scenario, SpatiallyExplicit):
        c.kind = SPATIALLY_EXPLICIT
        h = np.ascontiguousarray(scenario.habitat, dtype=np.uint32)
        if h.ndim != 2:
            raise ValueError("habitat must be [h, w]")
        c.height, c.width = h.shape
        c.habitat = h.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        keep.append(h)
        if scenario.dispersal is not None:
            d = np.ascontiguousarray(scenario.dispersal, dtype=np.float64)
            if d.shape != (h.size, h.size):
                raise ValueError("dispersal must be [h*w, h*w]")
            c.dispersal = d.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            keep.append(d)
        if scenario.tables is not None:
            cells = np.ascontiguousarray(scenario.tables[0], dtype=CELL_DTYPE)
            atoms = np.ascontiguousarray(scenario.tables[1], dtype=ATOM_DTYPE)
            if cells.shape != (h.size,):
                raise ValueError("tables need one cell record per habitat cell")
            c.cells = cells.ctypes.data
            c.atoms = atoms.ctypes.data if atoms.size else None
            c.n_atoms = atoms.size
            keep += [cells, atoms]
        elif scenario.dispersal is None:
            raise ValueError("SpatiallyExplicit needs a dispersal map or tables")
        if np.ndim(scenario.turnover) == 0:
            c.turnover_rate = float(scenario.turnover)
        else:  # a turnover map (spatially_explicit/turnover/map.rs)
            t = np.ascontiguousarray(scenario.turnover, dtype=np.float64)
            if t.shape != h.shape:
                raise ValueError("the turnover map must have the habitat map's shape")
            c.turnover_map = t.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            keep.append(t)
    else:
        raise TypeError("unknown scenario %r" % (scenario,))
    c._keep = keep
    return c


def _args_struct(algorithm: CUDA):
    a = CArgs()
    a.delta_t = algorithm.delta_t
    a.step_slice = algorithm.step_slice
    a.min_round_events = algorithm.min_round_events
    a.step_slice_max = algorithm.step_slice_max
    a.block_size = algorithm.block_size
    a.grid_size = algorithm.grid_size
    a.dedup_factor_pct = algorithm.dedup_factor_pct
    if algorithm.schedule not in ("plain", "learned"):
        raise ValueError("schedule must be 'plain' or 'learned'")
    a.schedule = 1 if algorithm.schedule == "learned" else 0
    if a.schedule == 1:
        if algorithm.model is None:
            raise ValueError("the learned schedule needs a LifetimeModel")
        a.model = algorithm.model.handle
    a.report_dispersal = 1 if algorithm.report_dispersal else 0
    a.device = algorithm.device
    a.rounds_per_graph = algorithm.rounds_per_graph
    a.resident = int(algorithm.resident) if algorithm.resident is not True else 1
    if algorithm.event_time_sampler not in EVENT_TIME_SAMPLERS:
        raise ValueError("event_time_sampler must be 'poisson' or 'exp'")
    a.event_time_sampler = EVENT_TIME_SAMPLERS[algorithm.event_time_sampler]
    a.max_rounds = algorithm.max_rounds
    a.priority_sims = algorithm.priority_sims
    a.priority_groups = algorithm.priority_groups
    a.reserve_sms = algorithm.reserve_sms
    a.priority_engines = algorithm.priority_engines
    if algorithm.priority_list is not None:
        lst = (ctypes.c_uint32 * max(1, len(algorithm.priority_list)))(*algorithm.priority_list)
        a._priority_keep = lst
        a.priority_list = ctypes.cast(lst, ctypes.c_void_p)
        if not a.priority_sims:
            a.priority_sims = len(algorithm.priority_list)
    return a


class _Collector:
    """Reporter sink gathering speciation and dispersal events (in delivery
    order; `kinds` records the sequence of calls as ("s" | "d", count))."""

    def __init__(self):
        self.chunks = []
        self.disp_chunks = []
        self.kinds = []

        def on_spec(user, ptr, n):
            buf = (ctypes.c_char * (n * SPECIATION_DTYPE.itemsize)).from_address(ptr)
            self.chunks.append(np.frombuffer(bytes(buf), dtype=SPECIATION_DTYPE))
            self.kinds.append(("s", n))
            return 0

        def on_disp(user, ptr, n):
            buf = (ctypes.c_char * (n * DISPERSAL_DTYPE.itemsize)).from_address(ptr)
            self.disp_chunks.append(np.frombuffer(bytes(buf), dtype=DISPERSAL_DTYPE))
            self.kinds.append(("d", n))
            return 0

        self._spec = _SPEC_CB(on_spec)
        self._disp = _DISP_CB(on_disp)
        self.struct = CReporter(None, self._spec, self._disp)

    def events(self):
        if not self.chunks:
            return np.zeros(0, dtype=SPECIATION_DTYPE)
        return np.concatenate(self.chunks)

    def dispersal_events(self):
        if not self.disp_chunks:
            return np.zeros(0, dtype=DISPERSAL_DTYPE)
        return np.concatenate(self.disp_chunks)


def _outcome(o: COutcome, spec=None, remaining=None, col=None) -> Outcome:
    out = Outcome(bool(o.paused), o.time, o.steps, o.n_initial, o.n_remaining, o.n_speciation,
                  o.biodiversity, o.n_rounds, o.n_dedup, o.n_launches, o.kernel_ms, o.total_ms,
                  o.h2d_bytes, o.d2h_bytes, o.n_step_launches, o.lineage_visits, o.resident_ms,
                  spec, remaining)
    out.n_dispersal = o.n_dispersal
    out.end_ms, out.routed_ms = o.end_ms, o.routed_ms
    if col is not None and col.disp_chunks:
        out.dispersal = col.dispersal_events()
        out.delivery = list(col.kinds)
    return out


class Simulation:
    """A scenario bound to the GPU (tables uploaded once), simulated per seed.

    Mirrors `Algorithm::initialise_and_simulate` / `resume_and_simulate`
    (rustcoalescence/algorithms/src/lib.rs:81-107)."""

    def __init__(self, scenario, speciation: float, algorithm: Optional[CUDA] = None):
        self.algorithm = algorithm or CUDA()
        L = lib()
        self._scenario = _scenario_struct(scenario, speciation)
        self._args = _args_struct(self.algorithm)
        ctx = ctypes.c_void_p()
        rc = L.necsim_gpu_create(ctypes.byref(self._scenario), ctypes.byref(self._args),
                                 ctypes.byref(ctx))
        self._ctx = ctx
        if rc != 0:
            msg = L.necsim_gpu_last_error(ctx).decode() if ctx.value else ""
            self.close()
            raise NecsimError(rc, msg)

    def close(self):
        if getattr(self, "_ctx", None) is not None and self._ctx.value:
            lib().necsim_gpu_destroy(self._ctx)
        self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc != 0:
            raise NecsimError(rc, lib().necsim_gpu_last_error(self._ctx).decode())

    def _remaining(self):
        L = lib()
        n = ctypes.c_uint64(0)
        self._check(L.necsim_gpu_remaining_lineages(self._ctx, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), dtype=LINEAGE_DTYPE)
        self._check(L.necsim_gpu_remaining_lineages(self._ctx, out.ctypes.data, n.value,
                                                    ctypes.byref(n)))
        return out[:n.value]

    def simulate(self, seed: int, pause_before: Optional[float] = None, collect: bool = True,
                 wyhash_seed: Optional[int] = None, event_log: Optional["EventLog"] = None) -> Outcome:
        """Simulates every origin lineage; `seed` is the RON `rng: Seed(seed)`."""
        L = lib()
        ws = seed_from_u64(seed) if wyhash_seed is None else wyhash_seed
        col = _Collector() if collect and event_log is None else None
        out = COutcome()
        pb = -1.0 if pause_before is None else float(pause_before)
        rep = event_log.reporter if event_log is not None else (col.struct if col else None)
        rc = L.necsim_gpu_simulate(self._ctx, ws, pb, ctypes.byref(rep) if rep is not None else None,
                                   ctypes.byref(out))
        self._check(rc)
        return _outcome(out, col.events() if col else None,
                        self._remaining() if out.paused else None, col)

    def resume(self, lineages: np.ndarray, resume_time: float, seed: int,
               pause_before: Optional[float] = None, collect: bool = True,
               wyhash_seed: Optional[int] = None) -> Outcome:
        """Simulates the given lineages from `resume_time` (resume_and_simulate)."""
        L = lib()
        ws = seed_from_u64(seed) if wyhash_seed is None else wyhash_seed
        lins = np.ascontiguousarray(lineages, dtype=LINEAGE_DTYPE)
        col = _Collector() if collect else None
        out = COutcome()
        pb = -1.0 if pause_before is None else float(pause_before)
        rc = L.necsim_gpu_simulate_lineages(self._ctx, lins.ctypes.data, len(lins), resume_time,
                                            ws, pb, ctypes.byref(col.struct) if col else None,
                                            ctypes.byref(out))
        self._check(rc)
        return _outcome(out, col.events() if col else None,
                        self._remaining() if out.paused else None, col)


def simulate(speciation: float, scenario, seed: int, algorithm: Optional[CUDA] = None,
             pause_before: Optional[float] = None, collect: bool = True) -> Outcome:
    """One-shot `rustcoalescence simulate` equivalent for this backend."""
    with Simulation(scenario, speciation, algorithm) as sim:
        return sim.simulate(seed, pause_before=pause_before, collect=collect)


def simulate_batch(scenarios: Sequence, speciations: Sequence[float], seeds: Sequence[int],
                   algorithm: Optional[CUDA] = None, pause_before: Optional[float] = None,
                   collect: bool = False) -> List[Outcome]:
    """Runs many independent simulations (one scenario kind) in one batched
    launch per round; returns one Outcome per simulation."""
    L = lib()
    n = len(scenarios)
    structs = (CScenario * n)()
    keep = []
    for j, (sc, nu) in enumerate(zip(scenarios, speciations)):
        c = _scenario_struct(sc, nu)
        keep.append(c)
        structs[j] = c
    seeds_arr = (ctypes.c_uint64 * n)(*[seed_from_u64(s) for s in seeds])
    outs = (COutcome * n)()
    cols = [_Collector() for _ in range(n)] if collect else None
    reps = None
    if collect:
        reps = (CReporter * n)(*[c.struct for c in cols])
    args = _args_struct(algorithm or CUDA())
    err = ctypes.create_string_buffer(512)
    pb = -1.0 if pause_before is None else float(pause_before)
    rc = L.necsim_gpu_simulate_batch(structs, seeds_arr, n, ctypes.byref(args), pb,
                                     ctypes.cast(reps, ctypes.c_void_p) if reps else None,
                                     outs, err, 512)
    if rc != 0:
        raise NecsimError(rc, err.value.decode())
    return [_outcome(outs[j], cols[j].events() if cols else None, None, cols[j] if cols else None)
            for j in range(n)]


class Batch:
    """A resident batch of independent simulations (one scenario kind): the
    set-up (tables, origins, CUDA graph) happens once, `run()` re-simulates
    all of them from their origins on the device."""

    def __init__(self, scenarios: Sequence, speciations: Sequence[float], seeds: Sequence[int],
                 algorithm: Optional[CUDA] = None, pause_before: Optional[float] = None):
        L = lib()
        n = len(scenarios)
        self.n = n
        self._structs = (CScenario * n)()
        self._keep = []
        for j, (sc, nu) in enumerate(zip(scenarios, speciations)):
            c = _scenario_struct(sc, nu)
            self._keep.append(c)
            self._structs[j] = c
        self._seeds = (ctypes.c_uint64 * n)(*[seed_from_u64(s) for s in seeds])
        self._args = _args_struct(algorithm or CUDA())
        pb = -1.0 if pause_before is None else float(pause_before)
        b = ctypes.c_void_p()
        rc = L.necsim_gpu_batch_create(self._structs, self._seeds, n, ctypes.byref(self._args), pb,
                                       ctypes.byref(b))
        self._b = b
        if rc != 0:
            msg = L.necsim_gpu_batch_last_error(b).decode() if b.value else ""
            self.close()
            raise NecsimError(rc, msg)

    def run(self, collect: bool = False) -> List[Outcome]:
        L = lib()
        outs = (COutcome * self.n)()
        cols = [_Collector() for _ in range(self.n)] if collect else None
        reps = (CReporter * self.n)(*[c.struct for c in cols]) if collect else None
        rc = L.necsim_gpu_batch_run(self._b, ctypes.cast(reps, ctypes.c_void_p) if reps else None,
                                    outs)
        if rc != 0:
            raise NecsimError(rc, L.necsim_gpu_batch_last_error(self._b).decode())
        return [_outcome(outs[j], cols[j].events() if cols else None, None, cols[j] if cols else None)
                for j in range(self.n)]

    @property
    def priority(self) -> List[int]:
        """Batch indices of the simulations in the priority engine, in priority order."""
        n = ctypes.c_uint32(0)
        ids = (ctypes.c_uint32 * max(1, self.n))()
        rc = lib().necsim_gpu_batch_priority(self._b, ids, self.n, ctypes.byref(n))
        if rc != 0:
            raise NecsimError(rc, "priority query failed")
        return [int(ids[k]) for k in range(n.value)]

    def close(self):
        if getattr(self, "_b", None) is not None and self._b.value:
            lib().necsim_gpu_batch_destroy(self._b)
        self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def build_tables(scenario: SpatiallyExplicit):
    """Host-side SpatiallyExplicit tables (cells, atoms) as numpy arrays."""
    L = lib()
    c = _scenario_struct(scenario, 0.5)
    n_atoms = ctypes.c_uint64(0)
    rc = L.necsim_build_tables(ctypes.byref(c), None, None, 0, ctypes.byref(n_atoms))
    if rc != 0:
        raise NecsimError(rc, "table build failed")
    cells = np.zeros(c.width * c.height, dtype=CELL_DTYPE)
    atoms = np.zeros(max(n_atoms.value, 1), dtype=ATOM_DTYPE)
    rc = L.necsim_build_tables(ctypes.byref(c), cells.ctypes.data, atoms.ctypes.data,
                               n_atoms.value, ctypes.byref(n_atoms))
    if rc != 0:
        raise NecsimError(rc, "table build failed")
    return cells, atoms[:n_atoms.value]


def enumerate_origins(scenario, speciation: float = 0.5) -> np.ndarray:
    """The scenario's origin lineages in the reference's order (host only)."""
    L = lib()
    c = _scenario_struct(scenario, speciation)
    n = ctypes.c_uint64(0)
    rc = L.necsim_enumerate_origins(ctypes.byref(c), None, 0, ctypes.byref(n))
    if rc != 0:
        raise NecsimError(rc, "origin enumeration failed")
    out = np.zeros(max(n.value, 1), dtype=LINEAGE_DTYPE)
    rc = L.necsim_enumerate_origins(ctypes.byref(c), out.ctypes.data, n.value, ctypes.byref(n))
    if rc != 0:
        raise NecsimError(rc, "origin enumeration failed")
    return out[:n.value]


def subdomain_ranks(scenario, size: int, lineages: np.ndarray, speciation: float = 0.5):
    """IsolatedLandscape: each lineage's subdomain rank under the scenario's
    decomposition into `size` parts (decomposition/{modulo,radial,equal}.rs);
    returns (ranks, exact), exact False when SpatiallyExplicit's weight
    decomposition found fewer parts."""
    c = _scenario_struct(scenario, speciation)
    lins = np.ascontiguousarray(lineages, dtype=LINEAGE_DTYPE)
    ranks = np.zeros(max(len(lins), 1), dtype=np.uint32)
    exact = ctypes.c_int32(1)
    rc = lib().necsim_subdomain_ranks(ctypes.byref(c), size, lins.ctypes.data, len(lins), ranks.ctypes.data,
                                      ctypes.byref(exact))
    if rc != 0:
        raise NecsimError(rc, "subdomain ranks failed")
    return ranks[:len(lins)], bool(exact.value)


def distinct_speciation_set(events: np.ndarray) -> np.ndarray:
    """Sorted unique (event_time bits, x, y, index) rows: the species identities
    (SpeciesIdentity::from_speciation, plugins/species/src/identity.rs:41)."""
    if len(events) == 0:
        return np.zeros((0, 4), dtype=np.uint64)
    k = np.stack([events["event_time"].view(np.uint64), events["x"].astype(np.uint64),
                  events["y"].astype(np.uint64), events["index"].astype(np.uint64)], axis=1)
    return np.unique(k, axis=0)


# ---------------------------------------------------------------------------
# Learned lifetime scheduler
# ---------------------------------------------------------------------------
MODEL_FEATURES = 8
MODEL_PARAMS = 4801
# offsets of the flat parameter array: W1[64][8], b1[64], W2[64][64], b2[64], W3[64], b3
MODEL_LAYOUT = {"W1": (0, (64, 8)), "b1": (512, (64,)), "W2": (576, (64, 64)),
                "b2": (4672, (64,)), "W3": (4736, (64,)), "b3": (4800, (1,))}


def _f32(a, shape_tail=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class LifetimeModel:
    """The MLP (8 -> 64 -> 64 -> 1, bf16 weights, fp32 accumulation) that
    predicts, from a lineage's features, log(1 + remaining events) of its
    simulation's longest-lived lineage; trained and evaluated by the
    backend's own CUDA kernels on `device`."""

    def __init__(self, seed: int = 0, device: int = 0):
        L = lib()
        h = ctypes.c_void_p()
        rc = L.necsim_model_create(device, seed, ctypes.byref(h))
        self._h = h
        if rc != 0:
            msg = L.necsim_model_last_error(h).decode() if h.value else ""
            self.close()
            raise NecsimError(rc, msg)

    @property
    def handle(self):
        return self._h.value

    def _check(self, rc):
        if rc != 0:
            raise NecsimError(rc, lib().necsim_model_last_error(self._h).decode())

    @property
    def weights(self) -> np.ndarray:
        out = np.zeros(MODEL_PARAMS, dtype=np.float32)
        self._check(lib().necsim_model_get_weights(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    @weights.setter
    def weights(self, w):
        w, wp = _f32(w)
        if w.size != MODEL_PARAMS:
            raise ValueError("expected %d parameters" % MODEL_PARAMS)
        self._check(lib().necsim_model_set_weights(self._h, wp))

    def predict(self, X) -> np.ndarray:
        X, xp = _f32(X)
        n = X.shape[0] if X.ndim == 2 else X.size // MODEL_FEATURES
        y = np.zeros(n, dtype=np.float32)
        self._check(lib().necsim_model_predict(self._h, xp, n, y.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return y

    def gradients(self, X, T):
        """(gradient of sum 0.5 (MLP(x) - t)^2 / n, loss)."""
        X, xp = _f32(X)
        T, tp = _f32(T)
        g = np.zeros(MODEL_PARAMS, dtype=np.float32)
        loss = ctypes.c_double()
        self._check(lib().necsim_model_gradients(self._h, xp, tp, T.size,
                                                 g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                 ctypes.byref(loss)))
        return g, loss.value

    def train(self, X, T, epochs: int = 20, batch: int = 1024, lr: float = 2e-3, seed: int = 0) -> np.ndarray:
        """Adam on the device; returns the mean loss of each epoch."""
        X, xp = _f32(X)
        T, tp = _f32(T)
        losses = np.zeros(epochs, dtype=np.float64)
        self._check(lib().necsim_model_train(self._h, xp, tp, T.size, epochs, batch, lr, seed,
                                             losses.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return losses

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().necsim_model_destroy(self._h)
        self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def collect_traces(scenarios: Sequence, speciations: Sequence[float], seeds: Sequence[int],
                   algorithm: Optional[CUDA] = None, pause_before: Optional[float] = None,
                   snapshot_rounds: int = 32, max_rows: int = 1 << 18):
    """Training traces generated by the backend itself: (features [n, 8],
    labels [n] = log(1 + remaining events of the simulation's longest-lived
    lineage at that snapshot)) of lineages snapshotted every
    `snapshot_rounds` rounds of a batch run."""
    L = lib()
    n = len(scenarios)
    structs = (CScenario * n)()
    keep = []
    for j, (sc, nu) in enumerate(zip(scenarios, speciations)):
        c = _scenario_struct(sc, nu)
        keep.append(c)
        structs[j] = c
    seeds_arr = (ctypes.c_uint64 * n)(*[seed_from_u64(s) for s in seeds])
    alg = algorithm or CUDA()
    if alg.schedule != "plain":
        alg = CUDA(**{**alg.__dict__, "schedule": "plain", "model": None})
    args = _args_struct(alg)
    X = np.zeros((max_rows, MODEL_FEATURES), dtype=np.float32)
    y = np.zeros(max_rows, dtype=np.float32)
    got = ctypes.c_uint64()
    err = ctypes.create_string_buffer(512)
    pb = -1.0 if pause_before is None else float(pause_before)
    rc = L.necsim_gpu_trace_batch(structs, seeds_arr, n, ctypes.byref(args), pb, snapshot_rounds, max_rows,
                                  X.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                  y.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.byref(got), err, 512)
    if rc != 0:
        raise NecsimError(rc, err.value.decode())
    return X[:got.value].copy(), y[:got.value].copy()


# ---------------------------------------------------------------------------
# Launch autotuner
# ---------------------------------------------------------------------------
AUTOTUNE_DTYPE = np.dtype([("block_size", "<u4"), ("dedup_factor_pct", "<u4"), ("step_slice", "<u8"),
                           ("ms", "<f8"), ("steps", "<u8")])


def autotune(scenarios: Sequence, speciations: Sequence[float], seeds: Sequence[int],
             algorithm: Optional[CUDA] = None, sample_pause: float = 400.0,
             max_sample_lineages: int = 1 << 22):
    """Picks block size, step_slice and the dedup table factor for a batch
    by timing a bounded sample of it (necsim_gpu_autotune).  Returns
    (CUDA arguments with the winner filled in, per-candidate results)."""
    L = lib()
    base = algorithm or CUDA()
    n = len(scenarios)
    structs = (CScenario * n)()
    keep = []
    for j, (sc, nu) in enumerate(zip(scenarios, speciations)):
        c = _scenario_struct(sc, nu)
        keep.append(c)
        structs[j] = c
    seeds_arr = (ctypes.c_uint64 * n)(*[seed_from_u64(s) for s in seeds])
    args = _args_struct(CUDA(**{**base.__dict__, "schedule": "plain", "model": None}))
    best = CArgs()
    res = np.zeros(32, dtype=AUTOTUNE_DTYPE)
    got = ctypes.c_uint32()
    err = ctypes.create_string_buffer(512)
    rc = L.necsim_gpu_autotune(structs, seeds_arr, n, ctypes.byref(args), sample_pause, max_sample_lineages,
                               ctypes.byref(best), res.ctypes.data, len(res), ctypes.byref(got), err, 512)
    if rc != 0:
        raise NecsimError(rc, err.value.decode())
    tuned = CUDA(**{**base.__dict__, "block_size": best.block_size, "step_slice": best.step_slice,
                    "dedup_factor_pct": best.dedup_factor_pct})
    return tuned, res[:got.value].copy()


# ---------------------------------------------------------------------------
# Event log (event_log/recorder.rs format)
# ---------------------------------------------------------------------------
EVENT_LOG_HEADER_DTYPE = np.dtype([("min_time", "<f8"), ("max_time", "<f8"), ("length", "<u8"),
                                   ("with_speciation", "u1"), ("with_dispersal", "u1")])
PACKED_EVENT_DTYPE = np.dtype([("gref", "<u8"), ("prior_time", "<f8"), ("event_time", "<f8"),
                               ("x", "<u4"), ("y", "<u4"), ("index", "<u4"),
                               ("tx", "<u4"), ("ty", "<u4"), ("tindex", "<u4"), ("coalescence", "<u8")])


def hash_peak(device: int = 0) -> float:
    """wymum (64x64 -> 128-bit multiply-fold) per second over independent
    chains on every SM of `device`: the hash work's integer-issue ceiling."""
    v = ctypes.c_double(0.0)
    rc = lib().necsim_gpu_hash_peak(device, ctypes.byref(v))
    if rc != 0:
        raise NecsimError(rc, "hash peak measurement failed")
    return v.value


def displacements(draws: np.ndarray, dispersal, device: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """The AlmostInfinite displacements (dx, dy) before rounding that the
    kernels compute from sample pairs draws[:, 0], draws[:, 1] (u64) for a
    Normal or Clark2Dt dispersal."""
    d = np.ascontiguousarray(draws, dtype=np.uint64)
    if d.ndim != 2 or d.shape[1] != 2:
        raise ValueError("draws must be [n, 2]")
    n = d.shape[0]
    dx = np.empty(n, dtype=np.float64)
    dy = np.empty(n, dtype=np.float64)
    if isinstance(dispersal, Clark2Dt):
        kind, a, b = ALMOST_INFINITE_CLARK2DT, dispersal.shape_u, dispersal.tail_p
    else:
        kind, a, b = ALMOST_INFINITE_NORMAL, dispersal.sigma, 0.0
    rc = lib().necsim_gpu_displacements(device, kind, d.ctypes.data, n, a, b, dx.ctypes.data, dy.ctypes.data)
    if rc != 0:
        raise NecsimError(rc, "displacement evaluation failed")
    return dx, dy


@dataclass
class Replay:
    """Events of a replayed event log, in PackedEvent order: speciation and
    dispersal arrays, `delivery` the sequence of reporter calls
    (("s" | "d", count)), `warning` the unmet-reporter-needs message of a
    non-strict replay (empty otherwise)."""
    speciation: np.ndarray
    dispersal: np.ndarray
    delivery: list
    n_events: int
    warning: str


def replay_event_log(segments, capacity: int = 100_000, need_speciation: bool = False,
                     need_dispersal: bool = False, strict: bool = True) -> Replay:
    """Reads event-log segments back as one stream (EventLogReplay,
    necsim/impls/std/src/event_log/replay/mod.rs).  `segments` are paths or
    glob patterns (a pattern's matches in order, files only when several
    match, the pattern itself when nothing matches, as replay/globbed.rs)."""
    import glob as _glob
    if isinstance(segments, (str, bytes, os.PathLike)):
        segments = [segments]
    paths = []
    for pat in segments:
        pat = os.fspath(pat)
        found = sorted(_glob.glob(pat))
        if len(found) > 1:
            found = [f for f in found if os.path.isfile(f) or not os.path.exists(f)]
        paths += found if found else [pat]
    arr = (ctypes.c_char_p * len(paths))(*[os.fsencode(p) for p in paths])
    col = _Collector()
    n = ctypes.c_uint64(0)
    err = ctypes.create_string_buffer(512)
    rc = lib().necsim_event_log_replay(ctypes.cast(arr, ctypes.c_void_p), len(paths), capacity,
                                       int(need_speciation), int(need_dispersal), int(strict),
                                       ctypes.byref(col.struct), ctypes.byref(n), err, 512)
    if rc != 0:
        raise NecsimError(rc, err.value.decode())
    return Replay(col.events(), col.dispersal_events(), list(col.kinds), n.value, err.value.decode())


class EventLog:
    """An on-disk event log in the reference's format (EventLogRecorder,
    necsim/impls/std/src/event_log/recorder.rs): pass it to
    `Simulation.simulate(..., event_log=log)`; close() writes the last
    segment.  `directory` must not exist yet."""

    def __init__(self, directory: str, capacity: int = 1_000_000, speciation: bool = True,
                 dispersal: bool = False):
        L = lib()
        h = ctypes.c_void_p()
        rc = L.necsim_event_log_create(os.fsencode(directory), capacity, int(speciation), int(dispersal),
                                       ctypes.byref(h))
        if rc != 0:
            raise NecsimError(rc, "cannot create the event log %s (it must not exist yet)" % directory)
        self._h = h
        self.directory = directory
        self.reporter = L.necsim_event_log_reporter(h)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            rc = lib().necsim_event_log_close(self._h)
            self._h = ctypes.c_void_p()
            if rc != 0:
                raise NecsimError(rc, "could not write the last event log segment")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def read_event_log(directory: str):
    """Reads an event log directory like the reference's replay
    (event_log/replay/segment.rs, sorted_segments.rs): (headers, events) with
    the events of all segments merged in PackedEvent order and decoded:
    `kind` 0 speciation (prior time negative, event time positive), 1
    dispersal without coalescence, 2 dispersal maybe coalescing, 3 dispersal
    with coalescence (event.rs:105-160); times are returned positive."""
    headers, parts = [], []
    names = sorted((n for n in os.listdir(directory) if n.isdigit()), key=int)
    for n in names:
        raw = open(os.path.join(directory, n), "rb").read()
        h = np.frombuffer(raw[:26], dtype=EVENT_LOG_HEADER_DTYPE)[0]
        ev = np.frombuffer(raw[26:], dtype=PACKED_EVENT_DTYPE)
        if len(ev) != int(h["length"]):
            raise ValueError("segment %s: header length %d, %d events" % (n, h["length"], len(ev)))
        headers.append(h)
        parts.append(ev)
    ev = np.concatenate(parts) if parts else np.zeros(0, dtype=PACKED_EVENT_DTYPE)
    prior_neg = (ev["prior_time"].view(np.uint64) >> np.uint64(63)).astype(bool)
    event_neg = (ev["event_time"].view(np.uint64) >> np.uint64(63)).astype(bool)
    kind = np.where(prior_neg & ~event_neg, 0, np.where(prior_neg & event_neg, 1,
                    np.where(~prior_neg & event_neg, 2, 3))).astype(np.uint8)
    out = np.zeros(len(ev), dtype=PACKED_EVENT_DTYPE.descr + [("kind", "u1")])
    for f in PACKED_EVENT_DTYPE.names:
        out[f] = ev[f]
    out["prior_time"] = np.abs(ev["prior_time"])
    out["event_time"] = np.abs(ev["event_time"])
    out["kind"] = kind
    order = np.lexsort((out["gref"], out["prior_time"].view(np.uint64), out["tindex"], out["ty"], out["tx"],
                        out["index"], out["y"], out["x"], out["event_time"].view(np.uint64)))
    return headers, out[order]
