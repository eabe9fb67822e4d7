"""Generates tests/golden/kat.json: known-answer vectors for the hot path.

The values come from a pure-Python restatement of the reference's
arithmetic, written independently of the C oracle, so that the oracle (and
through it the GPU backend) is pinned by a second implementation:

  * SeedableRng::seed_from_u64        necsim/core/src/cogs/rng.rs:33-63
  * WyHash prime_with / sample_u64    necsim/impls/no-std/src/cogs/rng/wyhash.rs:53-119
  * sample_uniform_closed_open        rng.rs:75-82
  * PoissonEventTimeSampler           .../event_time_sampler/poisson.rs:30-109, at several
    turnover rates (lambda * delta_t up to 20: Devroye counts beyond eight ranks)
  * ExpEventTimeSampler               .../event_time_sampler/exp.rs:37-83 with rng.rs:163-167
    sample_exponential, its logarithm the correctly rounded one (60-digit decimal)
  * Box-Muller + clamp_round_dispersal  rng.rs:180-197, habitat/almost_infinite.rs:100-114
  * LandscapeExtent iteration order   necsim/core/src/landscape/extent.rs:80-100, with the
    reference's own test cases (extent.rs:110-160)
  * InMemoryPackedSeparableAliasDispersalSampler tables and draws
    (alias/packed.rs:59-163, packed_separable_alias/{mod,dispersal}.rs)
  * full reference-schedule runs of tiny NonSpatial, SpatiallyImplicit,
    AlmostInfinite and SpatiallyExplicit scenarios (monolithic/mod.rs:43-270)
  * WrappingNoise: OpenSimplex 2D noise with wrapping and its octave sum
    (habitat/wrapping_noise/**), the coverage threshold, the rectangle origin
    sampler and the rejection-sampled Normal dispersal
    (dispersal_sampler/wrapping_noise.rs), with full tiny runs

Run:  python tests/golden/make_golden.py
"""
import json
import math
import os
import struct
from decimal import Decimal, getcontext

M64 = (1 << 64) - 1
P0, P1, P2, P5 = 0xA0761D6478BD642F, 0xE7037ED1A0B428DB, 0x8EBC6AF09C88C6E3, 0xEB44ACCAB455D165
K = 0x6EED0E9DA4D94A4F
INV_PHI = 0x9E3779B97F4A7C15


def seed_from_u64(state):
    seed = b""
    for _ in range(2):
        state = (state * 6364136223846793005 + 11634580027462260723) & M64
        xorshifted = (((state >> 18) ^ state) >> 27) & 0xFFFFFFFF
        rot = state >> 59
        x = ((xorshifted >> rot) | (xorshifted << ((32 - rot) % 32))) & 0xFFFFFFFF
        seed += struct.pack("<I", x)
    return struct.unpack("<Q", seed)[0]


def diffuse(x):
    x = (x * K) & M64
    a, b = x >> 32, x >> 60
    x ^= a >> b
    return (x * K) & M64


def wymum(a, b):
    r = a * b
    return (a ^ (r & M64)) ^ (b ^ (r >> 64))


def rot32(v):
    return ((v << 32) | (v >> 32)) & M64


class Wy:
    def __init__(self, seed):
        self.seed = seed
        self.state = seed

    def prime(self, loc, t):
        h = wymum(rot32(diffuse(loc)) ^ (self.seed ^ P0), rot32(diffuse(t)) ^ P2)
        self.state = wymum(h, 16 ^ P5)

    def u64(self):
        self.state = (self.state + P0) & M64
        return diffuse(wymum(self.state ^ P1, self.state))

    def co(self):
        return float(self.u64() >> 11) * 2.0 ** -53

    def oc(self):
        return float((self.u64() >> 11) + 1) * 2.0 ** -53


def poisson_next(g, inj, t, lam, dt):
    lam_dt = lam * dt
    p0 = math.exp(-lam_dt)
    ts = int(math.floor(t / dt))
    while True:
        g.prime(inj, ts)
        n, prod, acc = 0, p0, p0
        u = g.co()
        while u > acc and prod > 0.0:
            n += 1
            prod *= lam_dt / float(n)
            acc += prod
        best = None
        for k in range(n):
            et = (float(ts) + g.co()) * dt
            if et > t and (best is None or best[0] > et):
                best = (et, k)
        if best is not None:
            break
        ts += 1
    reprime = (ts + INV_PHI * (best[1] + 1)) & M64
    g.prime(inj, reprime)
    return best[0], reprime


def ln_correctly_rounded(u):
    getcontext().prec = 60
    return float(Decimal(u).ln())  # Decimal(float) is exact; float() rounds to nearest


def exp_next(g, inj, t, lam, dt):
    """exp.rs:37-83: exponential inter-event times inside delta_t buckets."""
    ts = int(math.floor(t / dt))
    event_time = float(ts) * dt
    slice_end = float(ts + 1) * dt
    g.prime(inj, ts)
    sub = 0
    while True:
        event_time += -ln_correctly_rounded(g.oc()) / lam
        sub = (sub + INV_PHI) & M64
        if event_time >= slice_end:
            ts += 1
            sub = 0
            event_time = slice_end
            slice_end = float(ts + 1) * dt
            g.prime(inj, ts)
        elif event_time > t:
            break
    reprime = (ts + sub) & M64
    g.prime(inj, reprime)
    return event_time, reprime


def normal_dispersal(d0, d1, sigma, x, y):
    u0 = float((d0 >> 11) + 1) * 2.0 ** -53
    u1 = float(d1 >> 11) * 2.0 ** -53
    r = math.sqrt(-2.0 * math.log(u0))
    theta = -6.283185307179586 * u1
    dx = (r * math.sin(theta)) * sigma + 0.0
    dy = (r * math.cos(theta)) * sigma + 0.0

    def rnd(v):  # f64::round: half away from zero (the subtraction below is exact)
        a = abs(v)
        f = math.floor(a)
        r = int(f) + (1 if a - f >= 0.5 else 0)
        return r if v >= 0 else -r

    W = 1 << 32
    return (x + rnd(dx)) % W, (y + rnd(dy)) % W


def extent_iter(ox, oy, w, h):
    """LandscapeExtent::iter (extent.rs:80-100) for width w and height h."""
    out = []
    for yy in range(h):
        for xx in range(w):
            out.append(((ox + xx) & 0xFFFFFFFF, (oy + yy) & 0xFFFFFFFF))
    return out


def circle_origins(cx, cy, r):
    out = []
    for (x, y) in extent_iter((cx - r) & 0xFFFFFFFF, (cy - r) & 0xFFFFFFFF, 2 * r + 1, 2 * r + 1):
        dx = min((x - cx) & 0xFFFFFFFF, (cx - x) & 0xFFFFFFFF)
        dy = min((y - cy) & 0xFFFFFFFF, (cy - y) & 0xFFFFFFFF)
        if dx * dx + dy * dy <= r * r:
            out.append((x, y))
    return out


# ---------------------------------------------------------------------------
# Tiny end-to-end runs with the reference's Monolithic schedule (NonSpatial)
# ---------------------------------------------------------------------------
def fnv_sample(x, y, i, t, u):
    h = 0xCBF29CE484222325
    data = struct.pack("<IIIdd", x, y, i, t, u)
    for b in data:
        h ^= b
        h = (h * 0x100000001B3) & M64
    return h


class NonSpatialLandscape:
    """habitat/non_spatial.rs, dispersal_sampler/non_spatial.rs:42-66."""

    def __init__(self, w, h, deme):
        self.w, self.h, self.deme = w, h, deme

    def origins(self):
        return [[((yy * self.w + xx) * self.deme + ii), 0.0, xx, yy, ii]
                for yy in range(self.h) for xx in range(self.w) for ii in range(self.deme)]

    def injection(self, x, y, i):
        return (y * self.w + x) * self.deme + i

    def habitat(self, x, y):
        return self.deme

    def nu(self, x, y, nu):
        return nu

    def disperse(self, g, x, y):
        idx = min(int(math.floor(g.co() * float(self.w * self.h))), self.w * self.h - 1)
        return idx % self.w, idx // self.w


class SpatiallyImplicitLandscape:
    """habitat/spatially_implicit.rs (the metacommunity at origin
    (2^32 - mw, 2^32 - mh)), dispersal_sampler/spatially_implicit.rs:58-86,
    speciation_probability/spatially_implicit.rs:31-44 (0 in the local
    community); origins are the local community's."""

    def __init__(self, w, h, deme, mw, mh, mdeme, m):
        self.w, self.h, self.deme, self.mw, self.mh, self.mdeme, self.m = w, h, deme, mw, mh, mdeme, m
        self.mox, self.moy = (1 << 32) - mw, (1 << 32) - mh

    def local(self, x, y):
        return x < self.w and y < self.h

    def origins(self):
        return NonSpatialLandscape(self.w, self.h, self.deme).origins()

    def injection(self, x, y, i):
        if self.local(x, y):
            return (y * self.w + x) * self.deme + i
        return ((((y - self.moy) & 0xFFFFFFFF) * self.mw + ((x - self.mox) & 0xFFFFFFFF)) * self.mdeme + i) & M64

    def habitat(self, x, y):
        return self.deme if self.local(x, y) else self.mdeme

    def nu(self, x, y, nu):
        return 0.0 if self.local(x, y) else nu

    def disperse(self, g, x, y):
        if self.local(x, y) and not (g.co() < self.m):
            idx = min(int(math.floor(g.co() * float(self.w * self.h))), self.w * self.h - 1)
            return idx % self.w, idx // self.w
        n = self.mw * self.mh
        idx = min(int(math.floor(g.co() * float(n))), n - 1)
        return (self.mox + idx % self.mw) & 0xFFFFFFFF, (self.moy + idx // self.mw) & 0xFFFFFFFF


def clark2dt_dispersal(u01, u2, shape_u, tail_p, x, y):
    """almost_infinite_clark2dt.rs:96-107 with clark2dt::cdf_inverse and
    pow_fast_one (x^1 is x itself); the angle is (u2 * 2) * pi."""
    e = 1.0 / tail_p
    base = 1.0 / (1.0 - u01)
    jump = math.sqrt(shape_u * ((base if e == 1.0 else math.pow(base, e)) - 1.0))
    theta = u2 * 2.0 * math.pi
    dx, dy = math.cos(theta) * jump, math.sin(theta) * jump

    def rnd(v):  # f64::round, half away from zero
        a = abs(v)
        f = math.floor(a)
        r = int(f) + (1 if a - f >= 0.5 else 0)
        return r if v >= 0 else -r

    W = 1 << 32
    return (x + rnd(dx)) % W, (y + rnd(dy)) % W


class AlmostInfiniteClarkLandscape:
    """AlmostInfinite habitat with Clark2Dt dispersal (a closed-open then an
    open-closed sample per dispersal)."""

    def __init__(self, cx, cy, r, shape_u, tail_p):
        self.cx, self.cy, self.r, self.shape_u, self.tail_p = cx, cy, r, shape_u, tail_p

    def origins(self):
        return AlmostInfiniteLandscape(self.cx, self.cy, self.r, 0.0).origins()

    def injection(self, x, y, i):
        return (y << 32) | x

    def habitat(self, x, y):
        return 1

    def nu(self, x, y, nu):
        return nu

    def disperse(self, g, x, y):
        u01 = g.co()
        u2 = g.oc()
        return clark2dt_dispersal(u01, u2, self.shape_u, self.tail_p, x, y)


class AlmostInfiniteLandscape:
    """habitat/almost_infinite.rs (one individual per location, injection
    y << 32 | x), the circle origin sampler, Normal dispersal (rng.rs:180-197
    + clamp_round_dispersal); the singleton demes still draw the coalescence
    sample (index 0)."""

    def __init__(self, cx, cy, r, sigma, rectangle=None):
        self.cx, self.cy, self.r, self.sigma, self.rectangle = cx, cy, r, sigma, rectangle

    def origins(self):
        if self.rectangle:  # almost_infinite/mod.rs:98: every location of the extent
            return [[(y << 32) | x, 0.0, x, y, 0] for (x, y) in extent_iter(*self.rectangle)]
        return [[(y << 32) | x, 0.0, x, y, 0] for (x, y) in circle_origins(self.cx, self.cy, self.r)]

    def injection(self, x, y, i):
        return (y << 32) | x

    def habitat(self, x, y):
        return 1

    def nu(self, x, y, nu):
        return nu

    def disperse(self, g, x, y):
        return normal_dispersal(g.u64(), g.u64(), self.sigma, x, y)


FRAC_1_PI = float("0.318309886183790671537767526745028724")  # core::f64::consts::FRAC_1_PI
SQRT_2 = float("1.41421356237309504880168872420969808")     # core::f64::consts::SQRT_2
OS_STRETCH = float("-0.211324865405187")  # open_simplex_noise_2d.rs:9, as written there
OS_SQUISH = float("0.366025403784439")    # open_simplex_noise_2d.rs:10
F64_2_32 = 4294967296.0


def f64_floor(v):
    return v if not math.isfinite(v) else float(math.floor(v))


def f64_round(v):
    """f64::round: half away from zero (v - trunc(v) is exact)."""
    if not math.isfinite(v):
        return v
    t = float(math.trunc(v))
    if abs(v - t) >= 0.5:
        t += math.copysign(1.0, v)
    return t


def f64_div(a, b):
    """IEEE division, also by zero."""
    if b != 0.0:
        return a / b
    if a != a or a == 0.0:
        return math.nan
    return math.copysign(math.inf, a) * math.copysign(1.0, b)


def as_i64(v):
    """Rust's `v as i64`: truncation, saturating, NaN -> 0."""
    if v != v:
        return 0
    if v >= 9223372036854775808.0:
        return (1 << 63) - 1
    if v <= -9223372036854775808.0:
        return -(1 << 63)
    return int(v)


def opensimplex_perm(seed):
    """generate_perm_array (opensimplex_noise/mod.rs:76-96): a Fisher-Yates
    style shuffle of 0..2048 whose i128 seed is never advanced, so the swap
    index at i is (seed * 6364136223846793005 + 1442695040888963407 + 31)
    mod (i + 1) (a truncated remainder made non-negative)."""
    a = seed * 6364136223846793005 + 1442695040888963407 + 31
    source = list(range(2048))
    perm = [0] * 2048
    for i in range(2047, -1, -1):
        r = abs(a) % (i + 1)
        if a < 0:
            r = -r
        if r < 0:
            r += i + 1
        perm[i] = source[r]
        source[r] = source[i]
    return perm


def os_extrapolate(perm, gx, gy, dx, dy, wrap):
    """OpenSimplexNoise2D::extrapolate (open_simplex_noise_2d.rs:21-59): the
    grid point wrapped into [0, wrap), its gradient from two perm lookups."""
    gx = f64_floor(gx - f64_floor(f64_div(gx, wrap)) * wrap)
    gy = f64_floor(gy - f64_floor(f64_div(gy, wrap)) * wrap)
    i0 = (perm[as_i64(gx) & 0xFF] + as_i64(gy)) & 0xFF
    idx = (perm[i0] & 0x0E) >> 1
    px, py = (5.0, 2.0) if idx & 1 == 0 else (2.0, 5.0)
    if idx & 2:
        px *= -1.0
    if idx & 4:
        py *= -1.0
    return px * dx + py * dy


def os_contribute(perm, dx, dy, ox, oy, gx, gy, wrap):
    """utils.rs:5-23 contribute for the 2D evaluator."""
    ds = dx + dy
    sx = (ox - dx) - OS_SQUISH * ds
    sy = (oy - dy) - OS_SQUISH * ds
    attn = 2.0 - (sx * sx + sy * sy)
    if attn <= 0.0:
        return 0.0
    a2 = attn * attn
    a4 = a2 * a2
    return a4 * os_extrapolate(perm, gx + dx, gy + dy, sx, sy, wrap)


def os_eval(perm, x, y, wrap):
    """OpenSimplexNoise2D::eval + get_value + evaluate_inside_triangle
    (open_simplex_noise_2d.rs:61-128): the input pre-squished so that the
    wrap applies in lattice space."""
    s = x + y
    ix, iy = x + OS_SQUISH * s, y + OS_SQUISH * s
    s = ix + iy
    stx, sty = ix + OS_STRETCH * s, iy + OS_STRETCH * s
    gx, gy = f64_floor(stx), f64_floor(sty)
    gs = gx + gy
    sqx, sqy = gx + OS_SQUISH * gs, gy + OS_SQUISH * gs
    insx, insy = stx - gx, sty - gy
    ox, oy = ix - sqx, iy - sqy

    def c(dx, dy):
        return os_contribute(perm, dx, dy, ox, oy, gx, gy, wrap)

    value = c(1.0, 0.0) + c(0.0, 1.0)
    in_sum = insx + insy
    f = 0.0 if in_sum <= 1.0 else 1.0
    z = 1.0 + f - in_sum
    if z > insx or z > insy:
        px, py = (1.0 + f, -1.0 + f) if insx > insy else (-1.0 + f, 1.0 + f)
    else:
        px, py = 1.0 - f, 1.0 - f
    value = value + (c(0.0 + f, 0.0 + f) + c(px, py))
    return value / 47.0


def noise_octaves(perm, x, y, persistence, scale, octaves):
    """sum_noise_octaves (habitat/wrapping_noise/mod.rs:216-249): each octave
    wraps at round(2^32 * frequency), an integer lattice period."""
    max_amp, amp = 0.0, 1.0
    freq = scale * FRAC_1_PI * 3.0
    result = 0.0
    for _ in range(octaves):
        wrap = f64_round(F64_2_32 * freq)
        fixed = wrap / F64_2_32
        result += os_eval(perm, float(x) * fixed, float(y) * fixed, wrap) * amp
        max_amp += amp
        amp *= persistence
        freq *= 2.0
    return result / max_amp


def total_order_key(v):
    """f64::total_cmp as a signed integer key."""
    b = struct.unpack("<q", struct.pack("<d", v))[0]
    return b ^ 0x7FFFFFFFFFFFFFFF if b < 0 else b


def noise_threshold(perm, seed, coverage, scale, persistence, octaves):
    """WrappingNoiseHabitat::new (habitat/wrapping_noise/mod.rs:47-99): the
    noise at 2^16 locations drawn by WyHash::from_seed(seed.to_le_bytes())
    (seed and state the i64's bits), sorted by total order, taken at
    min(floor(2^16 * coverage), 2^16 - 1)."""
    g = Wy(seed & M64)
    samples = []
    for _ in range(1 << 16):
        loc = g.u64()
        samples.append(noise_octaves(perm, loc & 0xFFFFFFFF, loc >> 32, persistence, scale, octaves))
    samples.sort(key=total_order_key)
    return samples[min(int(f64_floor(65536.0 * coverage)), 65535)]


class WrappingNoiseLandscape:
    """WrappingNoise (rustcoalescence/scenarios/src/wrapping_noise.rs): the
    almost-infinite plane, habitable where the octave noise is at most the
    coverage threshold (habitat/wrapping_noise/mod.rs:148-168), the rectangle
    origin sampler over habitable cells (singleton_demes/rectangle.rs:93-120),
    and approximate Normal dispersal (dispersal_sampler/wrapping_noise.rs):
    self-dispersal with probability ps / (ps + (1 - ps) * coverage), ps the
    Normal kernel's own (almost_infinite_normal.rs:22-37, erf from the C
    library), else Normal draws rejected until the target is habitable and
    not the origin."""

    def __init__(self, seed, coverage, scale, persistence, octaves, sample, sigma):
        self.seed, self.coverage, self.scale = seed, coverage, scale
        self.persistence, self.octaves, self.sample, self.sigma = persistence, octaves, sample, sigma
        self.perm = opensimplex_perm(seed)
        self.threshold = noise_threshold(self.perm, seed, coverage, scale, persistence, octaves)
        p1 = math.erf(0.5 / (sigma * SQRT_2)) if sigma > 0.0 else 1.0
        ps = p1 * p1
        self.p_self = ps / (ps + (1.0 - ps) * coverage)
        self.rejections = 0

    def noise(self, x, y):
        return noise_octaves(self.perm, x, y, self.persistence, self.scale, self.octaves)

    def habitat(self, x, y):
        if self.coverage <= 0.0:
            return 0
        if self.coverage >= 1.0:
            return 1
        return 1 if self.noise(x, y) <= self.threshold else 0

    def origins(self):
        ox, oy, w, h = self.sample
        return [[(y << 32) | x, 0.0, x, y, 0] for (x, y) in extent_iter(ox, oy, w, h) if self.habitat(x, y)]

    def injection(self, x, y, i):
        return (y << 32) | x

    def nu(self, x, y, nu):
        return nu

    def disperse(self, g, x, y):
        if g.co() < self.p_self:
            return x, y
        while True:
            tx, ty = normal_dispersal(g.u64(), g.u64(), self.sigma, x, y)
            if self.habitat(tx, ty) != 0 and (tx, ty) != (x, y):
                return tx, ty
            self.rejections += 1


def alias_atoms(events):
    """AliasMethodSamplerAtom::create (alias/packed.rs:59-121): Vose's
    construction with stack-ordered pairing; events = [(event, weight)]."""
    total = 0.0
    for _, wt in events:
        total = total + wt
    n = float(len(events))
    atoms = [[wt * n / total, e, e] for e, wt in events]
    over = [i for i, a in enumerate(atoms) if a[0] > 1.0]
    under = [i for i, a in enumerate(atoms) if a[0] < 1.0]
    while over and under:
        o, u = over.pop(), under.pop()
        atoms[o][0] = atoms[o][0] + atoms[u][0] - 1.0
        atoms[u][2] = atoms[o][1]
        if atoms[o][0] < 1.0:
            under.append(o)
        elif atoms[o][0] > 1.0:
            over.append(o)
    for i in over + under:  # rounding leftovers are full buckets (Vose 1991)
        atoms[i][0] = 1.0
    return atoms


class SpatiallyExplicitLandscape:
    """habitat/in_memory.rs, packed_separable_alias/mod.rs:64-203 (tables) and
    dispersal.rs:16-77 (a draw), coalescence index floor(u * habitat)."""

    def __init__(self, habitat, dispersal, turnover=None):
        self.hab = habitat  # [h][w]
        self.turnover = turnover  # [h][w] rates of a turnover map, or None
        self.h, self.w = len(habitat), len(habitat[0])
        cells = self.w * self.h
        self.prefix, acc = [], 0
        for c in range(cells):
            self.prefix.append(acc)
            acc += habitat[c // self.w][c % self.w]
        self.rows = []
        for row in range(cells):
            events, self_w = [], 0.0
            for col in range(cells):
                wt = dispersal[row][col] * float(habitat[col // self.w][col % self.w])
                if wt > 0.0:
                    events.append((col, wt))
                    if col == row:
                        self_w = wt
            if not events:
                self.rows.append((0.0, row, []))
                continue
            total = 0.0
            for _, wt in events:
                total = total + wt
            self_p = self_w / total
            self_u = self_w * float(len(events)) / total
            non_self = row
            if self_u < 1.0:
                atoms = alias_atoms(events)
                for j, a in enumerate(atoms):
                    if a[1] == row or a[2] == row:
                        if a[1] == row:  # flip: swap the events, u -> 1 - u
                            a[0], a[1], a[2] = 1.0 - a[0], a[2], a[1]
                        non_self = a[1]
                        atoms[j], atoms[-1] = atoms[-1], atoms[j]
                        break
            else:
                atoms = alias_atoms([(e, wt) for e, wt in events if e != row])
            self.rows.append((self_p, non_self, atoms))

    def origins(self):
        out = []
        for y in range(self.h):
            for x in range(self.w):
                for i in range(self.hab[y][x]):
                    out.append([self.injection(x, y, i), 0.0, x, y, i])
        return out

    def injection(self, x, y, i):
        return self.prefix[y * self.w + x] + i

    def habitat(self, x, y):
        return self.hab[y][x]

    def nu(self, x, y, nu):
        return nu

    def disperse(self, g, x, y):
        cell = y * self.w + x
        self_p, non_self, atoms = self.rows[cell]
        if self_p == 1.0:
            target = cell
        elif self_p == 0.0 or non_self != cell or g.co() >= self_p:
            f = g.co() * 1.0 * float(len(atoms))
            i = int(math.floor(f))
            a = atoms[i]
            target = a[1] if (f - float(i)) < a[0] else a[2]
        else:
            target = cell
        return target % self.w, target // self.w


def f64_bits(v):
    return struct.unpack("<Q", struct.pack("<d", v))[0]


def max_after(before, t):
    """PositiveF64::max_after (positive_f64.rs:103-113) for finite times."""
    if t > before:
        return t
    return struct.unpack("<d", struct.pack("<Q", f64_bits(before) + 1))[0]


def canonical_run(land, nu, seed, step_slice=10, min_round_events=1 << 20, step_slice_max=1024, lam=0.5,
                  dt=2.0, sampler=None):
    """The GPU backend's own schedule: every round advances each live
    lineage to a common horizon H' = H + clamp(ceil(min_round_events / n),
    step_slice, step_slice_max) / lambda (lambda the largest habitable rate
    of a turnover map), then merges lineages in identical state (location,
    index, last event time) keeping the smallest global reference."""
    sampler = sampler or poisson_next
    g = Wy(seed_from_u64(seed))
    turnover = getattr(land, "turnover", None)
    lam_rounds = lam
    if turnover:
        lam_rounds = max(turnover[y][x] for y in range(land.h) for x in range(land.w) if land.habitat(x, y) > 0)
    lins = land.origins()
    horizon = min(l[1] for l in lins)
    max_time = max(l[1] for l in lins)
    steps = rounds = dedups = 0
    events = []
    while lins:
        n = len(lins)
        per = -(-min_round_events // n)
        if step_slice_max and per > step_slice_max:
            per = step_slice_max
        per = max(per, step_slice)
        nh = horizon + float(per) / lam_rounds
        rounds += 1
        alive = []
        for lin in lins:
            dead = False
            while True:
                before = lin[1]
                rate = turnover[lin[3]][lin[2]] if turnover else lam
                t, _ = sampler(g, land.injection(lin[2], lin[3], lin[4]), before, rate, dt)
                nxt = max_after(before, t)
                if nxt >= nh:
                    break
                us = g.co()
                steps += 1
                max_time = max(max_time, nxt)
                if us < land.nu(lin[2], lin[3], nu):
                    events.append((nxt, lin[2], lin[3], lin[4], lin[1], lin[0]))
                    dead = True
                    break
                tx, ty = land.disperse(g, lin[2], lin[3])
                ti = int(math.floor(g.co() * float(land.habitat(tx, ty))))
                lin = [lin[0], nxt, tx, ty, ti]
            if not dead:
                alive.append(lin)
        alive.sort(key=lambda l: (l[2], l[3], l[4], f64_bits(l[1]), l[0]))
        lins = []
        for l in alive:
            if lins and lins[-1][2:5] == l[2:5] and f64_bits(lins[-1][1]) == f64_bits(l[1]):
                dedups += 1
                continue
            lins.append(l)
        horizon = nh
    events.sort(key=lambda e: (f64_bits(e[0]), e[1], e[2], e[3], e[1], e[2], e[3], f64_bits(e[4]), e[5]))
    species, last = 0, None
    for e in events:
        key = (e[0], e[1], e[2], e[3])
        species += key != last
        last = key
    return {"steps": steps, "rounds": rounds, "dedups": dedups, "time": max_time, "biodiversity": species,
            "events": [[e[5], e[4], e[0], e[1], e[2], e[3]] for e in events]}


def nonspatial_reference_run(w, h, deme, nu, seed, step_slice=10, dedup=1.0, event_slice=2.0,
                             lam=0.5, dt=2.0, sampler=None):
    return reference_run(NonSpatialLandscape(w, h, deme), nu, seed, step_slice, dedup, event_slice, lam,
                         dt, sampler)


def reference_run(land, nu, seed, step_slice=10, dedup=1.0, event_slice=2.0, lam=0.5, dt=2.0, sampler=None):
    """A full reference-schedule run (parallelisation/independent/monolithic/
    mod.rs:43-270 with the water-level reporter) on a landscape."""
    sampler = sampler or poisson_next
    g = Wy(seed_from_u64(seed))
    lineages = land.origins()
    n = len(lineages)
    slow = [(lin, lin[1]) for lin in lineages]
    fast = []
    es = max(int(n * event_slice), 1)
    cap = int(n * dedup)
    cache = [None] * cap
    level = 0.0
    steps = 0
    max_time = 0.0
    delivered = []
    slow_ev = []

    def inj(lin):
        return land.injection(lin[2], lin[3], lin[4])

    def rate_at(lin):  # turnover_rate/{uniform,in_memory}.rs
        return land.turnover[lin[3]][lin[2]] if getattr(land, "turnover", None) else lam

    while slow:
        rate = 0.0
        for (lin, _) in slow:
            rate = rate + rate_at(lin) * land.nu(lin[2], lin[3], nu)
        level = level + (float(es) / rate if rate > 0.0 else math.inf)  # f64 division
        slow_ev.sort()
        delivered += slow_ev
        slow_ev = []
        active = None
        prev_next = None
        prev_sample = None
        while slow or active is not None:
            nxt = None
            while slow:
                item = slow.pop(0)
                if item[1] < level:
                    nxt = item[0]
                    break
                fast.append(item)
            prev_task, active = active, nxt
            sample, prev_sample = prev_sample, None
            if prev_task is not None and prev_next is not None:
                dup = False
                if sample is not None and cap > 0:
                    idx = fnv_sample(*sample) % cap
                    dup = cache[idx] == sample
                    cache[idx] = sample
                if not dup:
                    (slow if prev_next < level else fast).append((prev_task, prev_next))
            prev_next = None
            if active is None:
                continue
            lin = active
            k = 0
            new_time = lin[1]
            while True:
                before = lin[1]
                t, _ = sampler(g, inj(lin), before, rate_at(lin), dt)
                nt = t if t > before else struct.unpack("<d", struct.pack("<Q", struct.unpack("<Q", struct.pack("<d", before))[0] + 1))[0]
                prev_next = nt
                if k >= step_slice or nt >= level:
                    break
                new_time = nt
                us = g.co()
                if prev_sample is None or not (prev_sample[4] <= us):
                    prev_sample = (lin[2], lin[3], lin[4], nt, us)
                k += 1
                if us < land.nu(lin[2], lin[3], nu):
                    slow_ev.append((nt, lin[2], lin[3], lin[4], lin[1], lin[0]))
                    active = None
                    break
                tx, ty = land.disperse(g, lin[2], lin[3])
                ti = int(math.floor(g.co() * float(land.habitat(tx, ty))))
                lin = [lin[0], nt, tx, ty, ti]
                active = lin
            steps += k
            max_time = max(max_time, new_time)
        slow, fast = fast, []
    slow_ev.sort()
    delivered += slow_ev
    species = 0
    last = None
    for e in delivered:
        key = (e[0], e[1], e[2], e[3])
        if key != last:
            species += 1
        last = key
    return {"steps": steps, "time": max_time, "biodiversity": species,
            "events": [[e[5], e[4], e[0], e[1], e[2], e[3]] for e in delivered]}


def se_case(w, h, case):
    """Small habitat and dispersal maps with zero cells, self-dispersal only
    rows, rows without self-dispersal and a full self-dispersal bucket."""
    import random
    rnd = random.Random(100 + case)
    hab = [[rnd.choice([0, 1, 2, 3]) for _ in range(w)] for _ in range(h)]
    hab[0][0] = 2
    cells = w * h
    disp = []
    for row in range(cells):
        if hab[row // w][row % w] == 0:
            disp.append([0.0] * cells)
            continue
        r = [0.0] * cells
        for col in range(cells):
            if hab[col // w][col % w] > 0 and rnd.random() < 0.6:
                r[col] = float(rnd.randint(1, 9))
        if case == 1 and row % 3 == 0:
            r = [0.0] * cells
            r[row] = 1.0  # self-dispersal only
        if case == 2 and row % 2 == 0:
            r[row] = 50.0  # self-dispersal fills its bucket: removed from the atoms
        if not any(r):
            r[row] = 1.0
        disp.append(r)
    return hab, disp


def main():
    kat = {}
    kat["seed_from_u64"] = {str(s): seed_from_u64(s) for s in [0, 1, 7, 42, 2 ** 63 + 5, M64]}
    kat["seahash_diffuse"] = {str(x): diffuse(x) for x in [0, 1, 12345, 2 ** 40 + 3, M64]}
    kat["wymum"] = [[a, b, wymum(a, b)] for a, b in [(1, 2), (P0, P1), (M64, M64), (12345, 2 ** 63)]]
    seqs = []
    for seed, loc, t in [(seed_from_u64(42), 0, 0), (seed_from_u64(7), 123456, 17),
                         (seed_from_u64(1), (5 << 32) | 9, 2 ** 63)]:
        g = Wy(seed)
        g.prime(loc, t)
        seqs.append({"seed": seed, "location": loc, "time_index": t,
                     "u64": [g.u64() for _ in range(8)]})
    kat["wyhash_sequences"] = seqs
    pois = []
    for seed, inj, t in [(seed_from_u64(42), 0, 0.0), (seed_from_u64(42), 99, 3.5),
                         (seed_from_u64(7), 2 ** 40, 1234.25), (seed_from_u64(1), 17, 1e6 + 0.5)]:
        g = Wy(seed)
        et, rp = poisson_next(g, inj, t, 0.5, 2.0)
        pois.append({"seed": seed, "injection": inj, "time": t, "event_time": et,
                     "event_time_bits": struct.unpack("<Q", struct.pack("<d", et))[0],
                     "reprime": rp})
    kat["poisson_next_event_time"] = pois
    # other turnover rates and intervals; lambda * delta_t = 20 draws Devroye
    # counts past the eight tabulated ranks
    pois_l = []
    for seed, inj, t, lam, dt in [(seed_from_u64(5), 3, 0.0, 0.05, 2.0), (seed_from_u64(5), 3, 10.25, 3.0, 1.0),
                                  (seed_from_u64(11), 2 ** 33 + 1, 7.0, 10.0, 2.0),
                                  (seed_from_u64(12), 77, 123.5, 1.0, 3.0),
                                  (seed_from_u64(13), 0, 0.0, 0.5, 0.25)]:
        for j in range(4):
            g = Wy(seed)
            et, rp = poisson_next(g, inj + j, t, lam, dt)
            pois_l.append({"seed": seed, "injection": inj + j, "time": t, "lambda": lam, "delta_t": dt,
                           "event_time_bits": struct.unpack("<Q", struct.pack("<d", et))[0], "reprime": rp})
    kat["poisson_next_event_time_rates"] = pois_l
    expv = []
    for seed, inj, t, lam, dt in [(seed_from_u64(42), 0, 0.0, 0.5, 2.0), (seed_from_u64(42), 99, 3.5, 0.5, 2.0),
                                  (seed_from_u64(7), 2 ** 40, 1234.25, 0.5, 3.0),
                                  (seed_from_u64(9), 5, 0.0, 5.0, 2.0), (seed_from_u64(9), 6, 40.0, 0.1, 0.5)]:
        for j in range(4):
            g = Wy(seed)
            et, rp = exp_next(g, inj + j, t, lam, dt)
            expv.append({"seed": seed, "injection": inj + j, "time": t, "lambda": lam, "delta_t": dt,
                         "event_time_bits": struct.unpack("<Q", struct.pack("<d", et))[0], "reprime": rp})
    kat["exp_next_event_time"] = expv
    nd = []
    g = Wy(seed_from_u64(3))
    g.prime(1, 1)
    for _ in range(64):
        d0, d1 = g.u64(), g.u64()
        for (x, y, sigma) in [(2 ** 31, 2 ** 31, 10.0), (0, 0, 3.5), (2 ** 32 - 1, 5, 100.0)]:
            tx, ty = normal_dispersal(d0, d1, sigma, x, y)
            nd.append([d0, d1, sigma, x, y, tx, ty])
    kat["normal_dispersal"] = nd
    m1, m2 = 0xFFFFFFFF, 0xFFFFFFFE
    # the reference's own LandscapeExtent iteration tests (extent.rs:110-160)
    kat["extent_iter"] = [
        {"origin": [0, 0], "w": 1, "h": 1, "locations": extent_iter(0, 0, 1, 1)},
        {"origin": [42, 24], "w": 4, "h": 2, "locations": extent_iter(42, 24, 4, 2)},
        {"origin": [m2, m1], "w": 4, "h": 2, "locations": extent_iter(m2, m1, 4, 2)},
    ]
    kat["circle_origins"] = [
        {"centre": [0, 0], "radius": 1, "locations": circle_origins(0, 0, 1)},
        {"centre": [2 ** 31 - 1, 2 ** 31 - 1], "radius": 3,
         "locations": circle_origins(2 ** 31 - 1, 2 ** 31 - 1, 3)},
    ]
    kat["nonspatial_runs"] = []
    for (w, h, deme, nu, seed) in [(2, 2, 2, 0.05, 3), (4, 3, 2, 0.02, 42), (5, 5, 1, 0.1, 9)]:
        r = nonspatial_reference_run(w, h, deme, nu, seed)
        r.update({"width": w, "height": h, "deme": deme, "speciation": nu, "seed": seed})
        kat["nonspatial_runs"].append(r)
    kat["spatially_explicit_runs"] = []
    for (w, h, nu, seed, case) in [(3, 3, 0.05, 4, 0), (4, 3, 0.02, 8, 1), (3, 2, 0.1, 2, 2)]:
        hab, disp = se_case(w, h, case)
        r = reference_run(SpatiallyExplicitLandscape(hab, disp), nu, seed)
        land = SpatiallyExplicitLandscape(hab, disp)
        r.update({"width": w, "height": h, "habitat": hab, "dispersal": disp, "speciation": nu, "seed": seed,
                  "tables": [{"self_dispersal": p, "non_self_event": ns, "atoms": atoms}
                             for p, ns, atoms in land.rows]})
        kat["spatially_explicit_runs"].append(r)
    kat["turnover_map_runs"] = []
    for (w, h, nu, seed, case) in [(3, 3, 0.05, 14, 0), (4, 3, 0.02, 18, 1)]:
        hab, disp = se_case(w, h, case)
        import random
        rnd = random.Random(200 + case)
        turnover = [[(rnd.choice([0.1, 0.5, 2.0, 7.5]) if hab[y][x] else 0.0) for x in range(w)] for y in range(h)]
        r = reference_run(SpatiallyExplicitLandscape(hab, disp, turnover), nu, seed)
        r.update({"width": w, "height": h, "habitat": hab, "dispersal": disp, "turnover": turnover,
                  "speciation": nu, "seed": seed})
        kat["turnover_map_runs"].append(r)
    kat["spatially_implicit_runs"] = []
    for (w, h, deme, mw, mh, mdeme, m, nu, seed) in [(3, 2, 2, 40, 1, 1, 0.2, 0.05, 5),
                                                     (2, 2, 1, 7, 3, 2, 0.5, 0.1, 6)]:
        r = reference_run(SpatiallyImplicitLandscape(w, h, deme, mw, mh, mdeme, m), nu, seed)
        r.update({"width": w, "height": h, "deme": deme, "meta_width": mw, "meta_height": mh, "meta_deme": mdeme,
                  "migration": m, "speciation": nu, "seed": seed})
        kat["spatially_implicit_runs"].append(r)
    kat["almost_infinite_runs"] = []
    for (cx, cy, rad, sigma, nu, seed) in [(2 ** 31 - 1, 2 ** 31 - 1, 2, 3.0, 0.05, 7), (1, 0xFFFFFFFF, 3, 1.5, 0.02, 8)]:
        r = reference_run(AlmostInfiniteLandscape(cx, cy, rad, sigma), nu, seed)
        r.update({"centre": [cx, cy], "radius": rad, "sigma": sigma, "speciation": nu, "seed": seed})
        kat["almost_infinite_runs"].append(r)
    kat["almost_infinite_rectangle_runs"] = []
    for (rect, sigma, nu, seed) in [((0xFFFFFFFF - 1, 7, 4, 3), 2.0, 0.05, 31), ((100, 0xFFFFFFFF, 3, 2), 0.0, 0.1, 32)]:
        r = reference_run(AlmostInfiniteLandscape(0, 0, 0, sigma, rect), nu, seed)
        r.update({"sample": list(rect), "sigma": sigma, "speciation": nu, "seed": seed})
        kat["almost_infinite_rectangle_runs"].append(r)
    kat["clark2dt_runs"] = []
    for (cx, cy, rad, shape_u, tail_p, nu, seed) in [(2 ** 31, 2 ** 31, 2, 4.0, 0.5, 0.05, 21),
                                                     (0, 3, 2, 1.0, 1.0, 0.05, 22)]:
        r = reference_run(AlmostInfiniteClarkLandscape(cx, cy, rad, shape_u, tail_p), nu, seed)
        r.update({"centre": [cx, cy], "radius": rad, "shape_u": shape_u, "tail_p": tail_p, "speciation": nu,
                  "seed": seed})
        kat["clark2dt_runs"].append(r)
    M32 = 0xFFFFFFFF
    noise = []
    for (seed, scale, persistence, octaves) in [(0, 0.07, 0.5, 16), (-7, 1.0, 1.0, 3), (123456789, 0.003, 0.8, 5),
                                                (-(1 << 63), 0.5, 0.25, 2)]:
        perm = opensimplex_perm(seed)
        pts = [(0, 0), (1, 0), (0, 1), (M32, M32), (M32, 0), (12345, 67890), (1 << 31, (1 << 31) - 1)]
        import random
        rnd = random.Random(seed & 0xFFFF)
        pts += [(rnd.randrange(1 << 32), rnd.randrange(1 << 32)) for _ in range(20)]
        pts += [(rnd.randrange(64), rnd.randrange(64)) for _ in range(20)]
        noise.append({"seed": seed, "scale": scale, "persistence": persistence, "octaves": octaves,
                      "points": [[x, y, noise_octaves(perm, x, y, persistence, scale, octaves)] for x, y in pts]})
    kat["wrapping_noise"] = noise
    thresholds = []
    for (seed, coverage, scale, persistence, octaves) in [(0, 0.5, 0.07, 0.5, 16), (-7, 0.25, 1.0, 1.0, 3),
                                                          (123456789, 0.9, 0.003, 0.8, 5), (5, 0.0, 0.1, 0.5, 2),
                                                          (5, 1.0, 0.1, 0.5, 2), (5, 0.99999, 0.1, 0.5, 2)]:
        perm = opensimplex_perm(seed)
        thresholds.append({"seed": seed, "coverage": coverage, "scale": scale, "persistence": persistence,
                           "octaves": octaves,
                           "threshold": noise_threshold(perm, seed, coverage, scale, persistence, octaves)})
    kat["wrapping_noise_thresholds"] = thresholds
    kat["wrapping_noise_self_dispersal"] = []
    for sigma, coverage in [(0.0, 0.5), (0.05, 0.5), (1.0, 0.5), (3.0, 0.4), (3.0, 0.0), (100.0, 1.0)]:
        p1 = math.erf(0.5 / (sigma * SQRT_2)) if sigma > 0.0 else 1.0
        ps = p1 * p1
        kat["wrapping_noise_self_dispersal"].append([sigma, coverage, ps / (ps + (1.0 - ps) * coverage)])
    origins = []
    for (seed, coverage, scale, persistence, octaves, sample) in [
            (-7, 0.25, 1.0, 1.0, 3, (M32 - 19, 5, 40, 30)), (3, 0.4, 0.07, 0.5, 4, (0, 0, 24, 16))]:
        land = WrappingNoiseLandscape(seed, coverage, scale, persistence, octaves, sample, 1.0)
        origins.append({"seed": seed, "coverage": coverage, "scale": scale, "persistence": persistence,
                        "octaves": octaves, "sample": list(sample),
                        "origins": [[o[2], o[3]] for o in land.origins()]})
    kat["wrapping_noise_origins"] = origins
    kat["wrapping_noise_runs"] = []
    wn_cases = [(3, 0.4, 0.07, 0.5, 4, (0, 0, 6, 5), 3.0, 0.05, 11),
                (-2, 0.7, 0.2, 0.7, 3, (M32 - 2, M32 - 1, 5, 4), 1.5, 0.08, 12)]
    for (seed, coverage, scale, persistence, octaves, sample, sigma, nu, rng_seed) in wn_cases:
        land = WrappingNoiseLandscape(seed, coverage, scale, persistence, octaves, sample, sigma)
        r = reference_run(land, nu, rng_seed)
        assert land.rejections > 0
        r.update({"noise_seed": seed, "coverage": coverage, "scale": scale, "persistence": persistence,
                  "octaves": octaves, "sample": list(sample), "sigma": sigma, "speciation": nu, "seed": rng_seed,
                  "rejections": land.rejections})
        kat["wrapping_noise_runs"].append(r)
    canon = []
    hab, disp = se_case(3, 3, 0)
    turnover = kat["turnover_map_runs"][0]["turnover"]
    for name, params, land, nu, seed, sampler in [
            ("ns", {"width": 4, "height": 3, "deme": 2}, NonSpatialLandscape(4, 3, 2), 0.02, 42, None),
            ("ns", {"width": 3, "height": 3, "deme": 2}, NonSpatialLandscape(3, 3, 2), 0.03, 5, exp_next),
            ("si", {"width": 3, "height": 2, "deme": 2, "meta_width": 40, "meta_height": 1, "meta_deme": 1,
                    "migration": 0.2}, SpatiallyImplicitLandscape(3, 2, 2, 40, 1, 1, 0.2), 0.05, 5, None),
            ("ai", {"centre": [2 ** 31 - 1, 2 ** 31 - 1], "radius": 2, "sigma": 3.0},
             AlmostInfiniteLandscape(2 ** 31 - 1, 2 ** 31 - 1, 2, 3.0), 0.05, 7, None),
            ("se", {"width": 3, "height": 3, "habitat": hab, "dispersal": disp},
             SpatiallyExplicitLandscape(hab, disp), 0.05, 4, None),
            ("se", {"width": 3, "height": 3, "habitat": hab, "dispersal": disp, "turnover": turnover},
             SpatiallyExplicitLandscape(hab, disp, turnover), 0.05, 14, None),
            ("wn", {"noise_seed": 3, "coverage": 0.4, "scale": 0.07, "persistence": 0.5, "octaves": 4,
                    "sample": [0, 0, 6, 5], "sigma": 3.0},
             WrappingNoiseLandscape(3, 0.4, 0.07, 0.5, 4, (0, 0, 6, 5), 3.0), 0.05, 11, None)]:
        for step_slice_max in (1024, 10):
            r = canonical_run(land, nu, seed, step_slice_max=step_slice_max, sampler=sampler)
            r.update(params)
            r.update({"case": name, "speciation": nu, "seed": seed, "step_slice": 10,
                      "min_round_events": 1 << 20, "step_slice_max": step_slice_max,
                      "sampler": "exp" if sampler else "poisson"})
            canon.append(r)
    kat["canonical_runs"] = canon
    kat["nonspatial_runs_exp"] = []
    for (w, h, deme, nu, seed) in [(2, 2, 2, 0.05, 3), (4, 3, 2, 0.02, 42)]:
        r = nonspatial_reference_run(w, h, deme, nu, seed, sampler=exp_next)
        r.update({"width": w, "height": h, "deme": deme, "speciation": nu, "seed": seed})
        kat["nonspatial_runs_exp"].append(r)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kat.json")
    with open(path, "w") as f:
        json.dump(kat, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
