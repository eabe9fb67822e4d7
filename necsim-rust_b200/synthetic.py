"""Seeded synthetic landscapes and sweeps for the benchmark configurations.

No public dataset is involved: the habitat and dispersal maps, and the
batched sweep's parameters, are generated here from a splitmix64 stream so
that every run (tests, benchmark, CPU baseline) sees the same inputs.

Configurations (sizes as in the benchmark definition):
  C1  NonSpatial 100x100, deme 10, speciation 1e-3, seed 42
  C2  AlmostInfinite, Circle radius 100, Normal sigma 10, speciation 1e-5, seed 7
  C3  SpatiallyExplicit 64x64 habitat (0 w.p. 0.15 else U{1..50}), dense
      4096x4096 dispersal (Gaussian sigma 3 cells + 1% uniform, zero into
      non-habitat, rows normalised), speciation 1e-4, seed 1
  C4  256 SpatiallyImplicit simulations: local J = floor(10^U(3,6)) cells of
      deme 1, metacommunity 1e7 cells of deme 1, migration U(0.01, 0.2),
      speciation 10^U(-6,-3), seeds 0..255
  C5  SpatiallyExplicit 128x128 habitat (0 w.p. 0.2 else U{1..500}), dense
      16384x16384 Gaussian (sigma 4) dispersal, speciation 1e-6
"""
import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def splitmix64(seed: int, n: int, stream: int = 0) -> np.ndarray:
    """n outputs of splitmix64 started at `seed` (stream offsets the start)."""
    with np.errstate(over="ignore"):
        k = np.arange(1, n + 1, dtype=np.uint64) + np.uint64(stream) * np.uint64(1 << 40)
        z = np.uint64(seed) + k * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def unit(seed: int, n: int, stream: int = 0) -> np.ndarray:
    """n uniforms in [0, 1) from the splitmix64 stream."""
    return (splitmix64(seed, n, stream) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def habitat_map(width: int, height: int, p_zero: float, max_value: int, seed: int) -> np.ndarray:
    """u32 habitat: 0 with probability p_zero, else uniform in 1..max_value."""
    n = width * height
    z = unit(seed, n, 0)
    v = unit(seed, n, 1)
    h = 1 + np.minimum((v * max_value).astype(np.uint64), max_value - 1)
    h[z < p_zero] = 0
    return h.astype(np.uint32).reshape(height, width)


def dispersal_map(habitat: np.ndarray, sigma: float, uniform_mass: float = 0.01,
                  rows_per_block: int = 256) -> np.ndarray:
    """Dense (h*w) x (h*w) f64 dispersal map: per habitable origin row a
    Gaussian kernel over Euclidean cell distance, mixed with `uniform_mass`
    spread evenly over all cells, zeroed into non-habitat, normalised;
    rows of non-habitat cells are all zero (the in-memory contract,
    dispersal_sampler/in_memory/contract.rs:13-69)."""
    height, width = habitat.shape
    n = width * height
    hab = habitat.reshape(-1) > 0
    xs = np.tile(np.arange(width, dtype=np.float64), height)
    ys = np.repeat(np.arange(height, dtype=np.float64), width)
    out = np.zeros((n, n), dtype=np.float64)
    inv2s2 = 1.0 / (2.0 * sigma * sigma)
    for r0 in range(0, n, rows_per_block):
        r1 = min(n, r0 + rows_per_block)
        dx = xs[None, :] - xs[r0:r1, None]
        dy = ys[None, :] - ys[r0:r1, None]
        g = np.exp(-(dx * dx + dy * dy) * inv2s2)
        g /= g.sum(axis=1, keepdims=True)
        g = (1.0 - uniform_mass) * g + uniform_mass / n
        g[:, ~hab] = 0.0
        g /= g.sum(axis=1, keepdims=True)
        g[~hab[r0:r1], :] = 0.0
        out[r0:r1] = g
    return out


def config1():
    return dict(kind=0, speciation_probability=1e-3, width=100, height=100, deme=10), 42


def config2(radius=100):
    return dict(kind=2, speciation_probability=1e-5, sigma=10.0, radius=radius,
                centre_x=0xFFFFFFFF // 2, centre_y=0xFFFFFFFF // 2), 7


def config3(width=64, height=64, map_seed=3):
    hab = habitat_map(width, height, 0.15, 50, map_seed)
    disp = dispersal_map(hab, 3.0)
    return dict(kind=3, speciation_probability=1e-4, width=width, height=height,
                habitat=hab, dispersal=disp), 1


def config4(n_sims=256, sweep_seed=4, max_local=None):
    """The batched SpatiallyImplicit sweep: list of (scenario dict, seed)."""
    u_j = unit(sweep_seed, n_sims, 0)
    u_m = unit(sweep_seed, n_sims, 1)
    u_n = unit(sweep_seed, n_sims, 2)
    sims = []
    for s in range(n_sims):
        j = int(np.floor(10.0 ** (3.0 + 3.0 * u_j[s])))
        if max_local is not None:
            j = min(j, max_local)
        sims.append((dict(kind=1, speciation_probability=float(10.0 ** (-6.0 + 3.0 * u_n[s])),
                          width=j, height=1, deme=1, meta_width=10_000_000, meta_height=1,
                          meta_deme=1, migration_probability=float(0.01 + 0.19 * u_m[s])), s))
    return sims


def config5(width=128, height=128, map_seed=5):
    hab = habitat_map(width, height, 0.2, 500, map_seed)
    disp = dispersal_map(hab, 4.0)
    return dict(kind=3, speciation_probability=1e-6, width=width, height=height,
                habitat=hab, dispersal=disp), 5


def to_scenario(desc):
    """Scenario dict -> the package's reference-shaped scenario object."""
    import importlib
    nb = importlib.import_module("necsim-rust_b200")
    k = desc["kind"]
    if k == 0:
        return nb.NonSpatial((desc["width"], desc["height"]), desc["deme"])
    if k == 1:
        return nb.SpatiallyImplicit((desc["width"], desc["height"]), desc["deme"],
                                    (desc["meta_width"], desc["meta_height"]), desc["meta_deme"],
                                    desc["migration_probability"])
    if k in (2, 4):
        if "sample" in desc:  # the Rectangle sample (x, y, width, height)
            x, y, w, h = desc["sample"]
            sample = nb.Rectangle((x, y), w, h)
        else:
            sample = nb.Circle(desc["radius"], (desc["centre_x"], desc["centre_y"]))
        if k == 2:
            return nb.AlmostInfinite(sample, nb.Normal(desc["sigma"]))
        return nb.AlmostInfinite(sample, nb.Clark2Dt(desc["shape_u"], desc["tail_p"]))
    if k == 5:
        x, y, w, h = desc["sample"]
        return nb.WrappingNoise(desc["noise_seed"], desc["coverage"], desc["scale"], desc["persistence"],
                                desc["octaves"], nb.Rectangle((x, y), w, h), desc["sigma"])
    turnover = desc.get("turnover_map")
    return nb.SpatiallyExplicit(desc["habitat"], desc["dispersal"],
                                turnover if turnover is not None else desc.get("turnover_rate", 0.5))
