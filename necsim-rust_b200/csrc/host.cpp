// host.cpp -- C ABI of the B200 backend: scenario set-up, dispersal tables,
// origin lineages, the round loop (captured in CUDA graphs) and event
// delivery to the reporters.  See include/necsim_b200.h for the contract.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <random>
#include <tuple>
#include <unordered_map>
#include <string>
#include <thread>
#include <vector>

#include "../../include/necsim_b200.h"
#include "kernels.h"
#include "layout.h"
#include "tables.h"
#include "wrapping_noise.h"

using namespace necsim;

// The learned lifetime model: bf16 weights used by the kernels, the fp32
// master copy and Adam moments, on one device.
struct necsim_model {
    int device = 0;
    __nv_bfloat16 *w = nullptr;
    float *master = nullptr, *m = nullptr, *v = nullptr, *grads = nullptr;
    double *loss = nullptr;
    int adam_step = 0;
    cudaStream_t stream = nullptr;
    std::string error;
    ~necsim_model() {
        if (device >= 0) cudaSetDevice(device);
        void *ptrs[] = {w, master, m, v, grads, loss};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

struct CudaFailure {
    cudaError_t err;
    const char *what;
};

#define CK(call)                                                   \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) throw CudaFailure{e_, #call};       \
    } while (0)

struct ApiError {
    int code;
    std::string msg;
};

[[noreturn]] void fail(int code, const std::string &msg) { throw ApiError{code, msg}; }

template <typename T>
T *dev_alloc(size_t n) {
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        fail(NECSIM_E_OUT_OF_MEMORY, "device allocation of " + std::to_string(n * sizeof(T)) + " bytes failed");
    }
    if (e != cudaSuccess) throw CudaFailure{e, "cudaMalloc"};
    return static_cast<T *>(p);
}

// SeedableRng::seed_from_u64 (necsim/core/src/cogs/rng.rs:33-63): PCG32
// output words fill the 8 seed bytes little-endian; WyHash::from_seed
// (wyhash.rs:41-49) reads them as one little-endian u64.
uint64_t seed_from_u64(uint64_t state) {
    uint64_t seed = 0;
    for (int word = 0; word < 2; ++word) {
        state = state * 6364136223846793005ULL + 11634580027462260723ULL;
        const uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
        const uint32_t rot = (uint32_t)(state >> 59);
        const uint32_t out = (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
        seed |= (uint64_t)out << (32 * word);
    }
    return seed;
}

// ---- WrappingNoise habitat (habitat/wrapping_noise/mod.rs) ----

// WyHash::sample_u64 (wyhash.rs:53-63) on the host, for the threshold sample
struct HostWyHash {
    uint64_t state;
    static uint64_t diffuse(uint64_t x) {  // wyhash.rs:99-119
        x *= 0x6eed0e9da4d94a4fULL;
        x ^= (x >> 32) >> (x >> 60);
        return x * 0x6eed0e9da4d94a4fULL;
    }
    uint64_t next() {
        state += 0xa0761d6478bd642fULL;
        const uint64_t a = state ^ 0xe7037ed1a0b428dbULL, b = state;
        const unsigned __int128 r = (unsigned __int128)a * b;  // wyhash.rs:85-96
        return diffuse((a ^ (uint64_t)r) ^ (b ^ (uint64_t)(r >> 64)));
    }
};

// generate_perm_array (opensimplex_noise/mod.rs:76-96): a shuffle of 0..2048
// whose i128 seed is never advanced, so each swap index is the same value
// modulo (i + 1), made non-negative; kept as the low bytes of perm[0..256)
void opensimplex_perm_low_bytes(int64_t seed, uint8_t out[256]) {
    std::vector<int64_t> source(2048), perm(2048);
    for (int64_t i = 0; i < 2048; ++i) source[i] = i;
    const __int128 a = (__int128)seed * 6364136223846793005LL + 1442695040888963407LL + 31;
    for (int64_t i = 2047; i >= 0; --i) {
        int64_t r = (int64_t)(a % (__int128)(i + 1));  // truncating, like Rust's %
        if (r < 0) r += i + 1;
        perm[i] = source[r];
        source[r] = source[i];
    }
    for (int i = 0; i < 256; ++i) out[i] = (uint8_t)(perm[i] & 0xff);
}

// Evaluates f(c) for c in [0, n) on all host threads (chunks in order).
template <typename F>
void parallel_for(uint64_t n, F &&f) {
    const unsigned threads = std::max(1u, std::thread::hardware_concurrency());
    if (n < 4096 || threads == 1) {
        for (uint64_t c = 0; c < n; ++c) f(c);
        return;
    }
    std::vector<std::thread> pool;
    const uint64_t per = (n + threads - 1) / threads;
    for (unsigned t = 0; t < threads; ++t) {
        const uint64_t c0 = t * per, c1 = std::min(n, c0 + per);
        if (c0 >= c1) break;
        pool.emplace_back([&f, c0, c1] {
            for (uint64_t c = c0; c < c1; ++c) f(c);
        });
    }
    for (auto &th : pool) th.join();
}

// WrappingNoiseHabitat::new (habitat/wrapping_noise/mod.rs:47-99): the noise
// at 2^16 locations drawn by WyHash::from_seed(seed.to_le_bytes()) (seed and
// state the i64's bits), sorted by f64::total_cmp, read at
// min(floor(2^16 * coverage), 2^16 - 1); and the approximate Normal
// dispersal's self-dispersal probability (dispersal_sampler/wrapping_noise.rs:
// 89-110, almost_infinite_normal.rs:22-37 with the C library's erf):
// ps / (ps + (1 - ps) * coverage), ps = erf(0.5 / (sigma * sqrt 2))^2.
NoiseHabitat make_noise_habitat(const necsim_scenario &sc) {
    NoiseHabitat h;
    std::memset(&h, 0, sizeof(h));
    opensimplex_perm_low_bytes(sc.noise_seed, h.perm);
    h.scale = sc.scale;
    h.persistence = sc.persistence;
    h.coverage = sc.coverage;
    h.octaves = sc.octaves;
    if (sc.coverage > 0.0 && sc.coverage < 1.0) {  // otherwise the threshold is never read
        constexpr uint64_t kSamples = 1u << 16;
        std::vector<uint64_t> locs(kSamples);
        HostWyHash g{(uint64_t)sc.noise_seed};
        for (auto &l : locs) l = g.next();
        std::vector<double> v(kSamples);
        parallel_for(kSamples, [&](uint64_t c) { v[c] = noise::octave_sum(h, (uint32_t)locs[c], (uint32_t)(locs[c] >> 32)); });
        auto key = [](double d) {
            int64_t b;
            std::memcpy(&b, &d, 8);
            return b ^ (int64_t)((uint64_t)(b >> 63) >> 1);
        };
        std::sort(v.begin(), v.end(), [&](double a, double b) { return key(a) < key(b); });
        const double k = std::floor((double)kSamples * sc.coverage);
        h.threshold = v[k >= (double)(kSamples - 1) ? kSamples - 1 : (uint64_t)k];
    }
    const double p1 = sc.sigma > 0.0 ? std::erf(0.5 / (sc.sigma * 1.41421356237309504880168872420969808)) : 1.0;
    const double ps = p1 * p1;
    const double p_self = ps / (ps + (1.0 - ps) * sc.coverage);
    // u < p  <=>  X < ceil(p * 2^53); NaN (0 / 0) never self-disperses
    h.self_threshold = p_self > 0.0 ? (uint64_t)std::ceil(std::ldexp(std::min(p_self, 1.0), 53)) : 0;
    return h;
}

// The noise habitat of a scenario, built once per parameter set (building
// evaluates the noise 2^16 times).
const NoiseHabitat &noise_habitat(const necsim_scenario &sc) {
    static std::mutex mu;
    static std::map<std::tuple<int64_t, double, double, double, uint64_t, double>, std::unique_ptr<NoiseHabitat>> cache;
    const auto key = std::make_tuple(sc.noise_seed, sc.coverage, sc.scale, sc.persistence, sc.octaves, sc.sigma);
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it == cache.end()) it = cache.emplace(key, std::make_unique<NoiseHabitat>(make_noise_habitat(sc))).first;
    return *it->second;
}

// Calls visit(x, y) for every habitable location of the WrappingNoise
// Rectangle sample in its row-major order (singleton_demes/rectangle.rs:
// 93-120 over landscape/extent.rs:80-100, coordinates wrapping at 2^32);
// the habitat of each block of locations is evaluated on all host threads.
template <typename F>
void for_each_noise_origin(const necsim_scenario &sc, F &&visit) {
    const NoiseHabitat &h = noise_habitat(sc);
    const uint64_t w = sc.sample_width, n = sc.sample_width * sc.sample_height;
    constexpr uint64_t kBlock = 1u << 20;
    std::vector<uint8_t> mask;
    for (uint64_t c0 = 0; c0 < n; c0 += kBlock) {
        const uint64_t m = std::min(kBlock, n - c0);
        mask.assign(m, 0);
        auto at = [&](uint64_t c, uint32_t &x, uint32_t &y) {
            x = sc.sample_x + (uint32_t)(c % w);
            y = sc.sample_y + (uint32_t)(c / w);
        };
        parallel_for(m, [&](uint64_t j) {
            uint32_t x, y;
            at(c0 + j, x, y);
            mask[j] = (uint8_t)noise::habitat_at(h, x, y);
        });
        for (uint64_t j = 0; j < m; ++j)
            if (mask[j]) {
                uint32_t x, y;
                at(c0 + j, x, y);
                visit(x, y);
            }
    }
}

// ---- landscape decompositions (necsim/impls/no-std/src/decomposition) ----

// Decomposition::map_location_to_subdomain_rank of a scenario's decomposition
// into `size` subdomains; every extent has its origin at (0, 0).
struct SubdomainMap {
    enum { Modulo, Radial, Equal } how = Modulo;
    uint32_t size = 1;
    uint64_t width = 1, height = 1;   // the habitat's extent (OffByOneU32 values)
    uint8_t morton_x = 0, morton_y = 0;
    std::vector<uint64_t> indices;    // Equal: first Morton index of ranks 1..
    bool exact = true;

    // equal/mod.rs:75-99
    static uint64_t morton(uint8_t mx, uint8_t my, uint32_t dx, uint32_t dy) {
        uint64_t m = 0;
        const uint8_t both = std::min(mx, my);
        for (uint32_t b = 0; b < both; ++b) {
            m |= (uint64_t)(dx & 1u) << (b * 2);
            dx >>= 1;
            m |= (uint64_t)(dy & 1u) << (b * 2 + 1);
            dy >>= 1;
        }
        mx -= both;
        my -= both;
        if (mx > 0) m |= (uint64_t)dx << (both * 2);
        if (my > 0) m |= (uint64_t)dy << (both * 2 + mx);
        return m;
    }

    // equal/mod.rs:66-73: ceil(ln(n) / ln 2) with the C library's ln, like
    // the reference's IntrinsicsMathsCore
    static uint8_t next_log2(uint64_t n) {
        return n > 1 ? (uint8_t)std::ceil(std::log((double)n) / 0.693147180559945309417232121458176568) : 0;
    }

    uint32_t rank(uint32_t x, uint32_t y) const {
        switch (how) {
        case Modulo:  // modulo.rs:32-45
            return (uint32_t)(((uint64_t)y * width + (uint64_t)x) % size);
        case Radial: {  // radial.rs:38-57, atan2 from the C library (libm's in the reference)
            const double fraction =
                std::atan2((double)((int64_t)y - (int64_t)height / 2), (double)((int64_t)x - (int64_t)width / 2)) *
                    0.318309886183790671537767526745028724 * 0.5 +
                0.5;
            const double r = std::floor((double)size * fraction);
            const uint32_t ri = r >= 4294967295.0 ? 0xffffffffu : (r > 0.0 ? (uint32_t)r : 0u);
            return std::min(ri, size - 1);
        }
        default: {  // equal/mod.rs:50-62
            const uint64_t m = morton(morton_x, morton_y, x, y);
            const auto it = std::lower_bound(indices.begin(), indices.end(), m);
            const uint32_t at = (uint32_t)(it - indices.begin());
            return (it != indices.end() && *it == m) ? at + 1 : at;
        }
        }
    }
};

// rustcoalescence/scenarios/src/*.rs `decompose`
SubdomainMap make_subdomain_map(const necsim_scenario &sc, uint32_t size) {
    SubdomainMap d;
    d.size = size;
    switch (sc.kind) {
    case NECSIM_NON_SPATIAL:  // habitat/non_spatial.rs: the area is the extent
        d.width = sc.width;
        d.height = sc.height;
        break;
    case NECSIM_SPATIALLY_IMPLICIT:  // SPATIALLY_IMPLICIT_EXTENT, the whole plane
        d.width = d.height = 1ULL << 32;
        break;
    case NECSIM_ALMOST_INFINITE_NORMAL:
    case NECSIM_ALMOST_INFINITE_CLARK2DT:
    case NECSIM_WRAPPING_NOISE:
        d.how = SubdomainMap::Radial;
        d.width = d.height = 1ULL << 32;
        break;
    default: {
        // equal/weight.rs:12-70 EqualDecomposition::weight
        d.how = SubdomainMap::Equal;
        d.width = sc.width;
        d.height = sc.height;
        d.morton_x = SubdomainMap::next_log2(d.width);
        d.morton_y = SubdomainMap::next_log2(d.height);
        std::vector<std::pair<uint64_t, uint32_t>> cells;
        uint64_t total = 0;
        for (uint32_t y = 0; y < sc.height; ++y)
            for (uint32_t x = 0; x < sc.width; ++x) {
                const uint32_t h = sc.habitat[(uint64_t)y * sc.width + x];
                if (h == 0) continue;
                total += h;
                cells.emplace_back(SubdomainMap::morton(d.morton_x, d.morton_y, x, y), h);
            }
        std::sort(cells.begin(), cells.end());
        uint64_t cumulative = 0;
        uint32_t last = 0;
        for (const auto &c : cells) {
            const uint32_t next = (uint32_t)((unsigned __int128)cumulative * size / total);
            cumulative += c.second;
            if (next != last) {
                last = next;
                d.indices.push_back(c.first);
            }
        }
        d.exact = d.indices.size() + 1 == size;
        break;
    }
    }
    return d;
}

// One simulation's host-side description.
struct SimHost {
    necsim_scenario sc;
    uint64_t seed;
    uint64_t n_origins;
    uint64_t lineage_offset;  // first slot in the batch's lineage arrays
    double start_time;        // min last event time of its lineages
    double start_max;         // max last event time of its lineages
    SimParams params;
};

// The Rectangle sample extent (LandscapeExtent: width and height 1..=2^32);
// optional for AlmostInfinite (sample_width 0: the Circle sample)
void validate_rectangle(const necsim_scenario &sc, bool required) {
    if (!required && sc.sample_width == 0) return;
    if (sc.sample_width == 0 || sc.sample_height == 0 || sc.sample_width > (1ULL << 32) ||
        sc.sample_height > (1ULL << 32))
        fail(NECSIM_E_INVALID_ARGUMENT, "the sample extent's width and height must be in 1..=2^32");
    if (sc.sample_width * sc.sample_height > (1ULL << 40))
        fail(NECSIM_E_TOO_LARGE, "the sample extent exceeds 2^40 locations");
}

void validate(const necsim_scenario &sc) {
    if (!(sc.speciation_probability > 0.0) || !(sc.speciation_probability <= 1.0))
        fail(NECSIM_E_INVALID_ARGUMENT, "speciation_probability must be in (0, 1]");
    if (sc.turnover_map) {
        if (sc.kind != NECSIM_SPATIALLY_EXPLICIT)
            fail(NECSIM_E_INVALID_ARGUMENT, "turnover maps apply to SpatiallyExplicit scenarios only");
    } else if (!(sc.turnover_rate > 0.0) || !std::isfinite(sc.turnover_rate)) {
        fail(NECSIM_E_INVALID_ARGUMENT, "turnover_rate must be positive");
    }
    switch (sc.kind) {
    case NECSIM_NON_SPATIAL:
        if (!sc.width || !sc.height || !sc.deme) fail(NECSIM_E_INVALID_ARGUMENT, "NonSpatial area and deme must be >= 1");
        break;
    case NECSIM_SPATIALLY_IMPLICIT:
        if (!sc.width || !sc.height || !sc.deme || !sc.meta_width || !sc.meta_height || !sc.meta_deme)
            fail(NECSIM_E_INVALID_ARGUMENT, "SpatiallyImplicit areas and demes must be >= 1");
        if (!(sc.migration_probability > 0.0) || !(sc.migration_probability <= 1.0))
            fail(NECSIM_E_INVALID_ARGUMENT, "migration probability must be in (0, 1]");
        break;
    case NECSIM_ALMOST_INFINITE_NORMAL:
        if (!(sc.sigma >= 0.0) || !std::isfinite(sc.sigma)) fail(NECSIM_E_INVALID_ARGUMENT, "sigma must be >= 0");
        if (sc.radius > 65535) fail(NECSIM_E_INVALID_ARGUMENT, "circle radius is a u16");
        validate_rectangle(sc, false);
        break;
    case NECSIM_ALMOST_INFINITE_CLARK2DT:
        if (!(sc.shape_u > 0.0) || !std::isfinite(sc.shape_u) || !(sc.tail_p > 0.0) || !std::isfinite(sc.tail_p))
            fail(NECSIM_E_INVALID_ARGUMENT, "Clark2Dt shape_u and tail_p must be positive");
        if (sc.radius > 65535) fail(NECSIM_E_INVALID_ARGUMENT, "circle radius is a u16");
        validate_rectangle(sc, false);
        break;
    case NECSIM_WRAPPING_NOISE:
        // WrappingNoiseArguments (wrapping_noise.rs:36-48) and their bond types
        if (!(sc.coverage >= 0.0) || !(sc.coverage <= 1.0))
            fail(NECSIM_E_INVALID_ARGUMENT, "WrappingNoise coverage must be in [0, 1]");
        if (!(sc.scale > 0.0) || !(sc.scale <= 1.0) || !(sc.persistence > 0.0) || !(sc.persistence <= 1.0))
            fail(NECSIM_E_INVALID_ARGUMENT, "WrappingNoise scale and persistence must be in (0, 1]");
        if (sc.octaves == 0) fail(NECSIM_E_INVALID_ARGUMENT, "WrappingNoise octaves must be >= 1");
        if (!(sc.sigma >= 0.0) || !std::isfinite(sc.sigma)) fail(NECSIM_E_INVALID_ARGUMENT, "sigma must be >= 0");
        validate_rectangle(sc, true);
        break;
    case NECSIM_SPATIALLY_EXPLICIT:
        if (!sc.width || !sc.height || !sc.habitat || (!sc.dispersal && !sc.cells))
            fail(NECSIM_E_INVALID_ARGUMENT, "SpatiallyExplicit needs a habitat map and a dispersal map or tables");
        if (sc.cells && sc.n_atoms && !sc.atoms)
            fail(NECSIM_E_INVALID_ARGUMENT, "SpatiallyExplicit tables: n_atoms > 0 without atoms");
        if (sc.turnover_map) {
            // maps/mod.rs:34-53 (non-negative rates) and turnover_rate/in_memory.rs:50-72
            // (InMemoryTurnoverRateError::ZeroTurnoverHabitat)
            const uint64_t cells = (uint64_t)sc.width * sc.height;
            for (uint64_t c = 0; c < cells; ++c) {
                const double t = sc.turnover_map[c];
                if (!(t >= 0.0) || !std::isfinite(t))
                    fail(NECSIM_E_INVALID_ARGUMENT, "turnover rates must be finite and non-negative");
                if (t == 0.0 && sc.habitat[c] != 0)
                    fail(NECSIM_E_INVALID_ARGUMENT, "zero turnover at a habitable location (ZeroTurnoverHabitat)");
            }
        }
        break;
    default:
        fail(NECSIM_E_INVALID_ARGUMENT, "unknown scenario kind");
    }
}

// Number of origin lineages of the scenario (OriginPreSampler::all()).
uint64_t count_origins(const necsim_scenario &sc) {
    switch (sc.kind) {
    case NECSIM_NON_SPATIAL:
    case NECSIM_SPATIALLY_IMPLICIT:
        return (uint64_t)sc.width * sc.height * sc.deme;
    case NECSIM_ALMOST_INFINITE_NORMAL:
    case NECSIM_ALMOST_INFINITE_CLARK2DT: {
        if (sc.sample_width) return sc.sample_width * sc.sample_height;  // Rectangle: every location
        const int64_t r = sc.radius;
        uint64_t n = 0;
        for (int64_t dy = -r; dy <= r; ++dy)
            for (int64_t dx = -r; dx <= r; ++dx)
                if ((uint64_t)(dx * dx + dy * dy) <= (uint64_t)(r * r)) ++n;
        return n;
    }
    case NECSIM_WRAPPING_NOISE: {
        uint64_t n = 0;
        for_each_noise_origin(sc, [&](uint32_t, uint32_t) { ++n; });
        return n;
    }
    default: {
        uint64_t n = 0;
        const uint64_t cells = (uint64_t)sc.width * sc.height;
        for (uint64_t c = 0; c < cells; ++c) n += sc.habitat[c];
        return n;
    }
    }
}

// ceil(2^64 / d) for 1 < d < 2^32, 0 for d <= 1 (quotient = dividend)
uint64_t division_magic(uint32_t d) {
    if (d <= 1) return 0;
    return ~0ULL / d + 1ULL;
}

// The samplers' constants for turnover rate lambda (poisson.rs:38-65,
// exp.rs:43-49): exp(-lambda * delta_t) with the system libm like
// IntrinsicsMathsCore, lambda * delta_t / k with the reference's IEEE
// division, and the constant Devroye sequence as integer thresholds.
PoissonConsts make_poisson_consts(double lambda, double delta_t) {
    PoissonConsts c;
    std::memset(&c, 0, sizeof(c));
    c.lambda = lambda;
    c.lambda_dt = lambda * delta_t;  // poisson.rs:40
    const double p0 = std::exp(-c.lambda_dt);  // poisson.rs:42
    for (int k = 1; k <= kPoissonTable; ++k) c.lambda_dt_over_k[k - 1] = c.lambda_dt / (double)k;
    double prod = p0, acc = p0;
    for (int n = 0; n < kPoissonThresholds; ++n) {
        // a rank whose prod is 0 stops the loop whatever the sample: its
        // threshold is the largest u64, which no 53-bit X exceeds, so the
        // count of exceeded thresholds is the loop's stopping rank
        c.threshold[n] = prod > 0.0 ? (uint64_t)std::floor(std::ldexp(acc, 53)) : ~0ULL;
        if (prod > 0.0) c.alive |= 1u << n;
        prod = prod * (c.lambda_dt / (double)(n + 1));
        acc = acc + prod;
    }
    c.prod_k = prod;
    c.acc_k = acc;
    return c;
}

SimParams base_params(const necsim_scenario &sc, const necsim_args &args, uint64_t wy_seed) {
    SimParams p;
    std::memset(&p, 0, sizeof(p));
    p.seed = wy_seed;
    p.nu = sc.speciation_probability;
    p.lambda = sc.turnover_rate;
    if (sc.kind == NECSIM_SPATIALLY_EXPLICIT && sc.turnover_map) {
        // a turnover map: the rounds advance at the largest habitable rate
        // (the samplers read each cell's own constants)
        const uint64_t cells = (uint64_t)sc.width * sc.height;
        double top = 0.0;
        for (uint64_t c = 0; c < cells; ++c)
            if (sc.habitat[c] != 0 && sc.turnover_map[c] > top) top = sc.turnover_map[c];
        p.lambda = top;
    }
    p.delta_t = args.delta_t;
    p.lambda_dt = p.lambda * p.delta_t;  // poisson.rs:40
    p.p0 = std::exp(-p.lambda_dt);       // poisson.rs:42, system libm like IntrinsicsMathsCore
    p.migration = sc.migration_probability;
    p.sigma = sc.sigma;
    p.width = sc.width;
    p.height = sc.height;
    p.deme = sc.deme;
    if (sc.kind == NECSIM_SPATIALLY_IMPLICIT) {
        // habitat/spatially_implicit.rs:45-49: meta origin (inv(w), inv(h))
        p.meta_ox = 0xffffffffu - (sc.meta_width - 1);
        p.meta_oy = 0xffffffffu - (sc.meta_height - 1);
        p.meta_width = sc.meta_width;
        p.meta_height = sc.meta_height;
        p.meta_deme = sc.meta_deme;
    }
    p.step_slice = args.step_slice;
    p.min_round_events = args.min_round_events;
    p.step_slice_max = args.step_slice_max;
    // floor(t / delta_t) is computed as floor(t * (1 / delta_t)) when delta_t
    // is a power of two: both round the same exact quotient
    int exp2 = 0;
    const double mant = std::frexp(p.delta_t, &exp2);
    p.inv_delta_t = (mant == 0.5) ? 1.0 / p.delta_t : 0.0;
    p.pois = make_poisson_consts(p.lambda, p.delta_t);
    // u < c  <=>  X < ceil(c * 2^53) for the 53-bit integer X of the uniform
    p.nu_threshold = (uint64_t)std::ceil(std::ldexp(sc.speciation_probability, 53));
    p.migration_threshold = (uint64_t)std::ceil(std::ldexp(sc.migration_probability, 53));
    p.width_magic = division_magic(p.width);
    p.meta_width_magic = division_magic(p.meta_width);
    if (sc.kind == NECSIM_ALMOST_INFINITE_CLARK2DT) {
        // clark2dt::cdf_inverse divides 1.0 / tail_p per draw: the same IEEE
        // quotient, once
        p.clark = 1;
        p.clark_shape_u = sc.shape_u;
        p.clark_exponent = 1.0 / sc.tail_p;
    }
    if (sc.kind == NECSIM_WRAPPING_NOISE) p.noise = noise_habitat(sc);
    p.pause_before = -1.0;
    return p;
}

necsim_args with_defaults(const necsim_args *in) {
    necsim_args a;
    std::memset(&a, 0, sizeof(a));
    if (in) a = *in;
    if (!(a.delta_t > 0.0)) a.delta_t = 2.0;
    if (a.step_slice == 0) a.step_slice = 10;
    if (a.min_round_events == 0) a.min_round_events = 1ULL << 20;
    if (a.step_slice_max == 0) a.step_slice_max = 1024;
    if (a.step_slice_max < a.step_slice) a.step_slice_max = a.step_slice;
    if (a.dedup_factor_pct == 0) a.dedup_factor_pct = 200;
    if (a.dedup_factor_pct < 110) a.dedup_factor_pct = 110;
    if (a.rounds_per_graph == 0) a.rounds_per_graph = 16;
    if (a.rounds_per_graph % 2) a.rounds_per_graph += 1;
    return a;
}

// ---- device buffers of one (batched) simulation ----
struct DeviceLineages {
    LineageSoA soa{};
    uint8_t *state = nullptr;
    void alloc(uint64_t n, bool with_pred = false) {
        if (with_pred) soa.pred_end = dev_alloc<float>(n);
        soa.x = dev_alloc<uint32_t>(n);
        soa.y = dev_alloc<uint32_t>(n);
        soa.idx = dev_alloc<uint32_t>(n);
        soa.sim = dev_alloc<uint32_t>(n);
        soa.last = dev_alloc<double>(n);
        soa.next = dev_alloc<double>(n);
        soa.reprime = dev_alloc<uint64_t>(n);
        soa.gref = dev_alloc<uint64_t>(n);
        soa.steps = dev_alloc<uint64_t>(n);
        soa.has_next = dev_alloc<uint8_t>(n);
        state = dev_alloc<uint8_t>(n);
    }
    void release() {
        void *ptrs[] = {soa.x, soa.y, soa.idx, soa.sim, soa.last, soa.next, soa.reprime,
                        soa.gref, soa.steps, soa.has_next, state, soa.pred_end};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        soa = LineageSoA{};
        state = nullptr;
    }
};

struct Control {  // small device scalars
    unsigned long long n_cur, out_count, work, mask, n_spec_total, n_disp_total, steps_total, visits;
    unsigned int n_active;    // active simulations in the global rounds
    uint32_t status;
    unsigned int n_resident;  // active simulations owned by the resident kernel
    unsigned int busy;        // warps of the cooperative kernel holding a lineage
    unsigned int blocks_done; // blocks of the round's step or cooperative kernel that finished or left
    unsigned int res_claim;   // the resident launch's next simulation (SM gate only)
    unsigned int res_done;    // the resident launch's blocks that finished or left (SM gate only)
    unsigned int pad;
};

// Events delivered round by round (dispersal reporting): per simulation the
// species counted so far and the last speciation event delivered.
struct Delivery {
    const necsim_reporter *reporters = nullptr;
    bool one_reporter = false;
    std::vector<uint64_t> species, n_dispersal;
    std::vector<DevSpeciationEvent> last;
    std::vector<uint8_t> has_last;
};

struct Engine {
    int device = 0;
    int kind = 0;
    necsim_args args{};
    cudaStream_t stream = nullptr;
    cudaStream_t stream_t = nullptr;  // resident kernel, concurrent with the global rounds
    cudaEvent_t ev_fork = nullptr;
    int n_sms = 148;

    std::vector<SimHost> sims;
    uint64_t n_total = 0;  // lineage slots

    // SpatiallyExplicit tables (shared by all simulations of a batch only if
    // they share the map; a batch of SE simulations gets one table set each)
    std::vector<CellRecord *> d_cells;
    std::vector<AliasAtom *> d_atoms;

    DeviceLineages A, B;
    DeviceLineages R;  // resident arena: small simulations' lineages, one segment each
    LineageSoA O{};  // resident origins (x, y, idx, sim, last, gref)
    cudaEvent_t ev_res0 = nullptr, ev_res1 = nullptr;
    uint64_t h2d_bytes = 0, d2h_bytes = 0;  // host<->device traffic of the current call
    uint32_t *owner = nullptr, *slot = nullptr;
    unsigned long long *min_gref = nullptr;
    unsigned long long table_size = 0;
    SimParams *d_params = nullptr;
    SimCounters *d_counters = nullptr;
    Control *d_ctl = nullptr;
    DevSpeciationEvent *d_spec = nullptr;
    uint64_t spec_cap = 0;
    DevDispersalEvent *d_disp = nullptr;
    uint64_t disp_cap = 0;
    Control *h_ctl = nullptr;  // pinned

    unsigned step_grid = 0, step_block = 0;
    unsigned coop_grid = 0;   // cooperative kernel (Poisson sampler), kCoopBlock threads per block
    uint64_t coop_max = 0;    // rounds with at most this many live lineages run there
    unsigned aux_grid = 0, aux_block = 256;

    // SM reservation between the engines of a batch (owned by the batch):
    // kGateOnly for the priority engine, which turns it on once its live
    // lineages fit the reserved SMs (gate_lineages); kGateAvoid for the others
    SmGate *gate = nullptr;
    uint32_t gate_role = kGateNone;
    uint64_t gate_lineages = 0;
    bool gate_on = false;

    // learned schedule (schedule == 1): model weights (owned by the model)
    // and the round's queue order
    bool learned = false;
    const __nv_bfloat16 *model_w = nullptr;
    uint8_t *order_keys = nullptr;
    unsigned *order_hist = nullptr;
    uint32_t *order = nullptr;
    std::vector<float *> d_entropy;  // SE: per-cell dispersal entropy, one per table set
    std::vector<PoissonConsts *> d_turnover;  // SE turnover maps: per-cell sampler constants

    // dispersal reporting: events drained and delivered after every round
    Delivery *delivery = nullptr;

    // training traces (necsim_gpu_trace_batch)
    bool tracing = false;
    TraceRow *trace_rows = nullptr;
    TraceDeath *trace_deaths = nullptr;
    unsigned long long *trace_counts = nullptr;  // [0] rows, [1] deaths
    uint64_t trace_rows_cap = 0, trace_deaths_cap = 0;
    uint32_t trace_snap = 0;  // index of the next snapshot
    uint64_t first_start_ns = 0;  // device clock of the last run's first schedule (outcomes' end_ms base)

    cudaGraphExec_t graph_exec = nullptr;
    std::vector<cudaEvent_t> ev_start, ev_end;
    cudaEvent_t ev_total0 = nullptr, ev_total1 = nullptr;
    bool timing_in_graph = true;

    ~Engine() { release(); }

    void release() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
        for (auto e : ev_start) cudaEventDestroy(e);
        for (auto e : ev_end) cudaEventDestroy(e);
        ev_start.clear();
        ev_end.clear();
        if (ev_total0) cudaEventDestroy(ev_total0);
        if (ev_total1) cudaEventDestroy(ev_total1);
        ev_total0 = ev_total1 = nullptr;
        A.release();
        B.release();
        R.release();
        if (ev_res0) cudaEventDestroy(ev_res0);
        if (ev_res1) cudaEventDestroy(ev_res1);
        ev_res0 = ev_res1 = nullptr;
        void *optrs[] = {O.x, O.y, O.idx, O.sim, O.last, O.gref};
        for (void *p : optrs)
            if (p) cudaFree(p);
        O = LineageSoA{};
        void *ptrs[] = {owner, slot, min_gref, d_params, d_counters, d_ctl, d_spec, d_disp};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        owner = slot = nullptr;
        min_gref = nullptr;
        d_params = nullptr;
        d_counters = nullptr;
        d_ctl = nullptr;
        d_spec = nullptr;
        d_disp = nullptr;
        for (auto p : d_cells)
            if (p) cudaFree(p);
        for (auto p : d_atoms)
            if (p) cudaFree(p);
        for (auto p : d_entropy)
            if (p) cudaFree(p);
        for (auto p : d_turnover)
            if (p) cudaFree(p);
        d_cells.clear();
        d_atoms.clear();
        d_entropy.clear();
        d_turnover.clear();
        void *lptrs[] = {order_keys, order_hist, order, trace_rows, trace_deaths, trace_counts};
        for (void *p : lptrs)
            if (p) cudaFree(p);
        order_keys = nullptr;
        order_hist = nullptr;
        order = nullptr;
        trace_rows = nullptr;
        trace_deaths = nullptr;
        trace_counts = nullptr;
        if (h_ctl) cudaFreeHost(h_ctl);
        h_ctl = nullptr;
        if (stream) cudaStreamDestroy(stream);
        if (stream_t) cudaStreamDestroy(stream_t);
        if (ev_fork) cudaEventDestroy(ev_fork);
        stream_t = nullptr;
        ev_fork = nullptr;
        stream = nullptr;
    }
};

// ---- SpatiallyExplicit tables ----
void upload_tables(Engine &E, SimHost &s) {
    HostTables t;
    if (s.sc.cells) {
        // tables built before by the caller: used as given (the kernels
        // bound-check every index they read from them)
        const uint64_t n_cells = (uint64_t)s.sc.width * s.sc.height;
        const CellRecord *c = reinterpret_cast<const CellRecord *>(s.sc.cells);
        t.cells.assign(c, c + n_cells);
        if (s.sc.n_atoms) {
            if (s.sc.n_atoms > 0xffffffffULL) fail(NECSIM_E_TOO_LARGE, "more than 2^32 alias atoms");
            const AliasAtom *a = reinterpret_cast<const AliasAtom *>(s.sc.atoms);
            t.atoms.assign(a, a + s.sc.n_atoms);
        }
        t.entropy.assign(n_cells, 0.0f);
    } else {
        int rc = build_spatially_explicit_tables(s.sc, t);
        if (rc == 1) fail(NECSIM_E_EMPTY_HABITAT, "habitat map has no habitable cell");
        if (rc == 2) fail(NECSIM_E_DISPERSAL_MAP, "dispersal map violates the in-memory dispersal contract");
        if (rc == 3) fail(NECSIM_E_TOO_LARGE, "more than 2^32 alias atoms");
        if (rc) fail(NECSIM_E_INVALID_ARGUMENT, "table build failed");
    }
    CellRecord *dc = dev_alloc<CellRecord>(t.cells.size());
    AliasAtom *da = dev_alloc<AliasAtom>(t.atoms.size());
    E.d_cells.push_back(dc);
    E.d_atoms.push_back(da);
    float *de = dev_alloc<float>(t.entropy.size());
    E.d_entropy.push_back(de);
    CK(cudaMemcpyAsync(de, t.entropy.data(), t.entropy.size() * sizeof(float), cudaMemcpyHostToDevice, E.stream));
    E.h2d_bytes += t.entropy.size() * sizeof(float);
    E.h2d_bytes += t.cells.size() * sizeof(CellRecord) + t.atoms.size() * sizeof(AliasAtom);
    CK(cudaMemcpyAsync(dc, t.cells.data(), t.cells.size() * sizeof(CellRecord), cudaMemcpyHostToDevice, E.stream));
    if (!t.atoms.empty())
        CK(cudaMemcpyAsync(da, t.atoms.data(), t.atoms.size() * sizeof(AliasAtom), cudaMemcpyHostToDevice, E.stream));
    CK(cudaStreamSynchronize(E.stream));
    s.params.cells = dc;
    s.params.atoms = da;
    s.params.cell_entropy = de;
    s.params.n_cells = t.cells.size();
    s.params.n_atoms = t.atoms.size();
    if (s.sc.turnover_map) {
        // the samplers' constants of every cell (InMemoryTurnoverRate)
        const uint64_t cells = (uint64_t)s.sc.width * s.sc.height;
        std::vector<PoissonConsts> tc(cells);
        for (uint64_t c = 0; c < cells; ++c) tc[c] = make_poisson_consts(s.sc.turnover_map[c], s.params.delta_t);
        PoissonConsts *dt = dev_alloc<PoissonConsts>(cells);
        E.d_turnover.push_back(dt);
        CK(cudaMemcpy(dt, tc.data(), cells * sizeof(PoissonConsts), cudaMemcpyHostToDevice));
        E.h2d_bytes += cells * sizeof(PoissonConsts);
        s.params.turnover_cells = dt;
    }
}

// `stream_priority`: the CUDA stream priority of the engine's streams (0:
// the default, the least).
void setup_engine(Engine &E, const necsim_args &args, int stream_priority = 0) {
    E.args = args;
    E.device = args.device;
    CK(cudaSetDevice(E.device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, E.device));
    E.n_sms = prop.multiProcessorCount;
    CK(cudaStreamCreateWithPriority(&E.stream, cudaStreamNonBlocking, stream_priority));
    CK(cudaStreamCreateWithPriority(&E.stream_t, cudaStreamNonBlocking, stream_priority));
    CK(cudaEventCreateWithFlags(&E.ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreate(&E.ev_total0));
    CK(cudaEventCreate(&E.ev_total1));
    void *h = nullptr;
    CK(cudaMallocHost(&h, sizeof(Control)));
    E.h_ctl = static_cast<Control *>(h);
}

void choose_launch(Engine &E) {
    unsigned block = E.args.block_size ? E.args.block_size : 128;
    if (block > (unsigned)kStepBlockMax) block = kStepBlockMax;
    block = std::max(32u, block / 32 * 32);
    int per_sm = 0;
    CK(step_kernel_occupancy(E.kind, E.args.event_time_sampler == NECSIM_SAMPLER_EXP, (int)block, &per_sm));
    if (per_sm < 1) per_sm = 1;
    E.step_block = block;
    E.step_grid = E.args.grid_size ? E.args.grid_size : (unsigned)(per_sm * E.n_sms);
    if (E.args.event_time_sampler != NECSIM_SAMPLER_EXP) {
        // one warp per lineage, all of them resident at once
        int coop_per_sm = 0;
        CK(coop_kernel_occupancy(E.kind, &coop_per_sm));
        if (coop_per_sm < 1) coop_per_sm = 1;
        E.coop_grid = (unsigned)(coop_per_sm * E.n_sms);
        E.coop_max = (uint64_t)E.coop_grid * (kCoopBlock / 32);
    }
    E.aux_block = 256;
    E.aux_grid = (unsigned)(E.n_sms * 8);
}

void alloc_run_buffers(Engine &E) {
    const uint64_t n = E.n_total;
    E.A.alloc(n, E.learned);
    E.R.alloc(n);
    CK(cudaEventCreate(&E.ev_res0));
    CK(cudaEventCreate(&E.ev_res1));
    E.B.alloc(n, E.learned);
    if (E.learned) {
        E.order_keys = dev_alloc<uint8_t>(n);
        E.order = dev_alloc<uint32_t>(n);
        E.order_hist = dev_alloc<unsigned>(2 * kOrderBuckets);
        CK(cudaMemsetAsync(E.order_hist, 0, 2 * kOrderBuckets * sizeof(unsigned), E.stream));
    }
    if (E.tracing) {
        E.trace_deaths_cap = n;
        E.trace_deaths = dev_alloc<TraceDeath>(n);
        E.trace_rows = dev_alloc<TraceRow>(E.trace_rows_cap);
        E.trace_counts = dev_alloc<unsigned long long>(2);
        CK(cudaMemsetAsync(E.trace_counts, 0, 2 * sizeof(unsigned long long), E.stream));
    }
    unsigned long long want = (n * E.args.dedup_factor_pct + 99) / 100;
    if (want < 2) want = 2;
    unsigned long long size = 1;
    while (size < want) size <<= 1;
    E.table_size = size;
    E.owner = dev_alloc<uint32_t>(size);
    E.min_gref = dev_alloc<unsigned long long>(size);
    E.slot = dev_alloc<uint32_t>(n);
    CK(cudaMemsetAsync(E.owner, 0xff, size * sizeof(uint32_t), E.stream));
    CK(cudaMemsetAsync(E.min_gref, 0xff, size * sizeof(unsigned long long), E.stream));
    E.d_params = dev_alloc<SimParams>(E.sims.size());
    E.d_counters = dev_alloc<SimCounters>(E.sims.size());
    E.d_ctl = dev_alloc<Control>(1);
    // each run resets both; a run without lineages runs no round and reads
    // them as they are here (upload_origins synchronises the stream next)
    CK(cudaMemsetAsync(E.d_counters, 0, E.sims.size() * sizeof(SimCounters), E.stream));
    CK(cudaMemsetAsync(E.d_ctl, 0, sizeof(Control), E.stream));
    E.spec_cap = n;
    E.d_spec = dev_alloc<DevSpeciationEvent>(n);
    if (E.disp_cap) E.d_disp = dev_alloc<DevDispersalEvent>(E.disp_cap);
}

// Calls push(x, y, index, global_reference) for every origin lineage of the
// scenario in the reference's origin-sampler order (OriginPreSampler::all()).
template <typename F>
void for_each_origin(const necsim_scenario &sc, F &&push) {
    if (sc.kind == NECSIM_NON_SPATIAL || sc.kind == NECSIM_SPATIALLY_IMPLICIT) {
        // origin_sampler/non_spatial.rs:89-112 over landscape/extent.rs:80-100
        // (SI samples only its local community, origin_sampler/spatially_implicit.rs)
        uint64_t g = 0;
        for (uint32_t yy = 0; yy < sc.height; ++yy)
            for (uint32_t xx = 0; xx < sc.width; ++xx)
                for (uint32_t ii = 0; ii < sc.deme; ++ii) push(xx, yy, ii, g++);
    } else if ((sc.kind == NECSIM_ALMOST_INFINITE_NORMAL || sc.kind == NECSIM_ALMOST_INFINITE_CLARK2DT) &&
               sc.sample_width) {
        // origin_sampler/singleton_demes/rectangle.rs:93-120: every location of
        // the extent is habitable, row-major, wrapping at 2^32
        for (uint64_t yy = 0; yy < sc.sample_height; ++yy)
            for (uint64_t xx = 0; xx < sc.sample_width; ++xx) {
                const uint32_t px = sc.sample_x + (uint32_t)xx, py = sc.sample_y + (uint32_t)yy;
                push(px, py, 0u, ((uint64_t)py << 32) | px);
            }
    } else if (sc.kind == NECSIM_ALMOST_INFINITE_NORMAL || sc.kind == NECSIM_ALMOST_INFINITE_CLARK2DT) {
        // origin_sampler/singleton_demes/circle.rs:36-70, 100-140
        const uint32_t r = sc.radius;
        const uint64_t d = (uint64_t)r * 2 + 1;
        const uint32_t ox = sc.centre_x - r, oy = sc.centre_y - r;
        const uint64_t r2 = (uint64_t)r * r;
        for (uint64_t yy = 0; yy < d; ++yy)
            for (uint64_t xx = 0; xx < d; ++xx) {
                const uint32_t px = ox + (uint32_t)xx, py = oy + (uint32_t)yy;
                const uint64_t dx = std::min<uint32_t>(px - sc.centre_x, sc.centre_x - px);
                const uint64_t dy = std::min<uint32_t>(py - sc.centre_y, sc.centre_y - py);
                if (dx * dx + dy * dy <= r2) push(px, py, 0u, ((uint64_t)py << 32) | px);
            }
    } else if (sc.kind == NECSIM_WRAPPING_NOISE) {
        // Lineage::new: the global reference is the AlmostInfinite injection
        // (habitat/wrapping_noise/mod.rs:170-175)
        for_each_noise_origin(sc, [&](uint32_t x, uint32_t y) { push(x, y, 0u, ((uint64_t)y << 32) | x); });
    } else {
        // origin_sampler/in_memory.rs:89-119; global reference = prefix(cell) + index
        uint64_t g = 0;
        for (uint32_t yy = 0; yy < sc.height; ++yy)
            for (uint32_t xx = 0; xx < sc.width; ++xx) {
                const uint32_t h = sc.habitat[(uint64_t)yy * sc.width + xx];
                for (uint32_t ii = 0; ii < h; ++ii) push(xx, yy, ii, g++);
            }
    }
}

// ---- per-simulation priority of the learned schedule ----

// The lifetime model's score of each simulation, its expected remaining
// life: the model is trained to predict, from one lineage's features, the
// log remaining events of that lineage's simulation (of its longest-lived
// lineage, with which the simulation ends).  The score is the mean
// prediction over up to 32 of its origin lineages, evenly spaced in origin
// order, at the start of the run (no event executed, the simulation's origin
// count live).  The features are the kernels' (lineage_features_of), with a
// SpatiallyExplicit cell's habitat and dispersal entropy read from the maps.
std::vector<float> score_simulations(necsim_model *m, const std::vector<SimHost> &sims) {
    constexpr uint64_t kSample = 32;
    std::vector<float> X;
    std::vector<uint32_t> owner;
    for (size_t s = 0; s < sims.size(); ++s) {
        const SimHost &sh = sims[s];
        const int kind = sh.sc.kind == NECSIM_ALMOST_INFINITE_CLARK2DT ? NECSIM_ALMOST_INFINITE_NORMAL : sh.sc.kind;
        const uint64_t stride = std::max<uint64_t>(1, sh.n_origins / kSample);
        uint64_t k = 0;
        for_each_origin(sh.sc, [&](uint32_t x, uint32_t y, uint32_t, uint64_t) {
            if (k++ % stride) return;
            float hab = 1.f, ent = 0.f;
            if (kind == NECSIM_SPATIALLY_EXPLICIT) {
                const uint64_t cell = (uint64_t)y * sh.sc.width + x;
                hab = (float)sh.sc.habitat[cell];
                ent = dispersal_entropy(sh.sc, cell);
            }
            float f[kFeat];
            lineage_features_of(kind, sh.params, sh.n_origins, x, y, 0.0, 0, hab, ent, f);
            X.insert(X.end(), f, f + kFeat);
            owner.push_back((uint32_t)s);
        });
    }
    std::vector<float> score(sims.size(), 0.f);
    const uint64_t n = owner.size();
    if (n == 0) return score;
    CK(cudaSetDevice(m->device));
    struct Res {
        float *x = nullptr, *y = nullptr;
        ~Res() {
            if (x) cudaFree(x);
            if (y) cudaFree(y);
        }
    } r;
    r.x = dev_alloc<float>(n * kFeat);
    r.y = dev_alloc<float>(n);
    CK(cudaMemcpyAsync(r.x, X.data(), n * kFeat * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    CK(launch_mlp_predict(m->w, r.x, n, r.y, m->stream));
    std::vector<float> y(n);
    CK(cudaMemcpyAsync(y.data(), r.y, n * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    CK(cudaStreamSynchronize(m->stream));
    // the model predicts the simulation's remaining life (log events) from
    // each lineage: the score is the mean over the sampled origins
    std::vector<uint32_t> count(sims.size(), 0);
    for (uint64_t j = 0; j < n; ++j) {
        score[owner[j]] += y[j];
        count[owner[j]] += 1;
    }
    for (size_t s = 0; s < sims.size(); ++s)
        if (count[s]) score[s] /= (float)count[s];
    return score;
}

// Builds the origin lineages of every simulation on the host, in the
// reference's origin-sampler order, and uploads them as structure of arrays.
void upload_origins(Engine &E, const std::vector<std::vector<necsim_lineage>> *given) {
    const uint64_t n = E.n_total;
    std::vector<uint32_t> x(n), y(n), idx(n), sim(n);
    std::vector<double> last(n);
    std::vector<uint64_t> gref(n);
    for (size_t s = 0; s < E.sims.size(); ++s) {
        SimHost &sh = E.sims[s];
        uint64_t o = sh.lineage_offset;
        double tmin = 0.0, tmax = 0.0;
        bool first = true;
        auto push = [&](uint32_t xx, uint32_t yy, uint32_t ii, uint64_t g, double t) {
            x[o] = xx;
            y[o] = yy;
            idx[o] = ii;
            sim[o] = (uint32_t)s;
            last[o] = t;
            gref[o] = g;
            ++o;
            if (first || t < tmin) tmin = t;
            if (first || t > tmax) tmax = t;
            first = false;
        };
        const necsim_scenario &sc = sh.sc;
        if (given) {
            for (const necsim_lineage &l : (*given)[s]) push(l.x, l.y, l.index, l.global_reference, l.last_event_time);
        } else {
            for_each_origin(sc, [&](uint32_t xx, uint32_t yy, uint32_t ii, uint64_t g) { push(xx, yy, ii, g, 0.0); });
        }
        if (o != sh.lineage_offset + sh.n_origins) fail(NECSIM_E_INVALID_ARGUMENT, "origin count mismatch");
        sh.start_time = tmin;
        sh.start_max = tmax;
    }
    // resident copy of the origins: every run starts from it
    LineageSoA &d = E.O;
    d.x = dev_alloc<uint32_t>(n);
    d.y = dev_alloc<uint32_t>(n);
    d.idx = dev_alloc<uint32_t>(n);
    d.sim = dev_alloc<uint32_t>(n);
    d.last = dev_alloc<double>(n);
    d.gref = dev_alloc<uint64_t>(n);
    CK(cudaMemcpyAsync(d.x, x.data(), n * 4, cudaMemcpyHostToDevice, E.stream));
    CK(cudaMemcpyAsync(d.y, y.data(), n * 4, cudaMemcpyHostToDevice, E.stream));
    CK(cudaMemcpyAsync(d.idx, idx.data(), n * 4, cudaMemcpyHostToDevice, E.stream));
    CK(cudaMemcpyAsync(d.sim, sim.data(), n * 4, cudaMemcpyHostToDevice, E.stream));
    CK(cudaMemcpyAsync(d.last, last.data(), n * 8, cudaMemcpyHostToDevice, E.stream));
    CK(cudaMemcpyAsync(d.gref, gref.data(), n * 8, cudaMemcpyHostToDevice, E.stream));
    E.h2d_bytes += n * (4 * 4 + 8 * 2);
    CK(cudaStreamSynchronize(E.stream));
}

// Resets the working lineages to the resident origins (device to device).
void reset_lineages(Engine &E) {
    const uint64_t n = E.n_total;
    LineageSoA &d = E.A.soa;
    const LineageSoA &o = E.O;
    CK(cudaMemcpyAsync(d.x, o.x, n * 4, cudaMemcpyDeviceToDevice, E.stream));
    CK(cudaMemcpyAsync(d.y, o.y, n * 4, cudaMemcpyDeviceToDevice, E.stream));
    CK(cudaMemcpyAsync(d.idx, o.idx, n * 4, cudaMemcpyDeviceToDevice, E.stream));
    CK(cudaMemcpyAsync(d.sim, o.sim, n * 4, cudaMemcpyDeviceToDevice, E.stream));
    CK(cudaMemcpyAsync(d.last, o.last, n * 8, cudaMemcpyDeviceToDevice, E.stream));
    CK(cudaMemcpyAsync(d.gref, o.gref, n * 8, cudaMemcpyDeviceToDevice, E.stream));
    CK(cudaMemsetAsync(d.steps, 0, n * 8, E.stream));
    CK(cudaMemsetAsync(d.has_next, 0, n, E.stream));
    CK(cudaMemsetAsync(d.next, 0, n * 8, E.stream));
    CK(cudaMemsetAsync(d.reprime, 0, n * 8, E.stream));
    CK(cudaMemsetAsync(E.A.state, 0, n, E.stream));
    if (d.pred_end) CK(cudaMemsetAsync(d.pred_end, 0, n * sizeof(float), E.stream));
}

StepArgs make_step_args(Engine &E, DeviceLineages &in) {
    StepArgs a{};  // every field zero, pointers null
    a.in = in.soa;
    a.state = in.state;
    a.order = nullptr;
    a.n_cur = &E.d_ctl->n_cur;
    a.work = &E.d_ctl->work;
    a.params = E.d_params;
    a.counters = E.d_counters;
    a.spec = E.d_spec;
    a.n_spec_total = &E.d_ctl->n_spec_total;
    a.spec_cap = E.spec_cap;
    a.disp = E.d_disp;
    a.n_disp_total = &E.d_ctl->n_disp_total;
    a.disp_cap = E.disp_cap;
    a.report_dispersal = E.args.report_dispersal ? 1 : 0;
    a.status = &E.d_ctl->status;
    a.steps_total = &E.d_ctl->steps_total;
    a.n_sims = (uint32_t)E.sims.size();
    a.order = E.learned ? E.order : nullptr;
    a.exp_sampler = E.args.event_time_sampler == NECSIM_SAMPLER_EXP ? 1u : 0u;
    a.coop_max = E.coop_max;
    // free rounds of single-lineage simulations (not when dispersal events
    // are drained round by round)
    a.free_rounds = E.args.report_dispersal ? 0u : 64u;
    a.busy = &E.d_ctl->busy;
    a.gate = E.gate;
    a.gate_role = E.gate ? E.gate_role : kGateNone;
    a.blocks_done = &E.d_ctl->blocks_done;
    if (E.tracing) {
        a.trace.deaths = E.trace_deaths;
        a.trace.n_deaths = E.trace_counts + 1;
        a.trace.cap = E.trace_deaths_cap;
    }
    return a;
}

FeatureArgs make_feature_args(Engine &E, DeviceLineages &in) {
    FeatureArgs f;
    f.in = in.soa;
    f.n_cur = &E.d_ctl->n_cur;
    f.params = E.d_params;
    f.counters = E.d_counters;
    f.kind = E.kind;
    // rounds stepped one warp per lineage (the cooperative kernel, or the
    // exponential sampler's step kernel when it has a warp per lineage)
    f.skip_at_most = E.coop_max ? E.coop_max : (uint64_t)E.step_grid * (E.step_block / 32);
    return f;
}

DedupArgs make_dedup_args(Engine &E, DeviceLineages &in, DeviceLineages &out) {
    DedupArgs a{};  // every field zero, pointers null
    a.in = in.soa;
    a.out = out.soa;
    a.state = in.state;
    a.state_out = out.state;
    a.n_cur = &E.d_ctl->n_cur;
    a.mask = &E.d_ctl->mask;
    a.owner = E.owner;
    a.min_gref = E.min_gref;
    a.slot = E.slot;
    a.out_count = &E.d_ctl->out_count;
    a.counters = E.d_counters;
    a.status = &E.d_ctl->status;
    if (E.args.resident) {
        // route small simulations to the arena: resident == 1 routes at one
        // lineage per warp of the resident block (every routed lineage is
        // stepped cooperatively), larger values at that many lineages
        a.arena = E.R.soa;
        a.resident_max = E.args.resident == 1 ? (uint64_t)(kResidentMax / 32)
                                              : std::min<uint64_t>(E.args.resident, kResidentMax);
    }
    a.params = E.d_params;
    if (E.tracing) {
        a.trace.deaths = E.trace_deaths;
        a.trace.n_deaths = E.trace_counts + 1;
        a.trace.cap = E.trace_deaths_cap;
    }
    return a;
}

ResidentArgs make_resident_args(Engine &E, uint32_t budget, const int *stop_flag) {
    ResidentArgs a{};  // every field zero, pointers null
    a.arena = E.R.soa;
    a.params = E.d_params;
    a.counters = E.d_counters;
    a.n_sims = (uint32_t)E.sims.size();
    a.budget = budget;
    a.spec = E.d_spec;
    a.n_spec_total = &E.d_ctl->n_spec_total;
    a.spec_cap = E.spec_cap;
    a.status = &E.d_ctl->status;
    a.steps_total = &E.d_ctl->steps_total;
    a.visits = &E.d_ctl->visits;
    a.n_resident = &E.d_ctl->n_resident;
    a.stop_flag = stop_flag;
    a.exp_sampler = E.args.event_time_sampler == NECSIM_SAMPLER_EXP ? 1u : 0u;
    a.gate = E.gate;
    a.gate_role = E.gate ? E.gate_role : kGateNone;
    a.claim = &E.d_ctl->res_claim;
    a.blocks_done = &E.d_ctl->res_done;
    return a;
}

ScheduleArgs make_schedule_args(Engine &E) {
    ScheduleArgs a;
    std::memset(&a, 0, sizeof(a));
    a.params = E.d_params;
    a.counters = E.d_counters;
    a.n_sims = (uint32_t)E.sims.size();
    a.dedup_pct = E.args.dedup_factor_pct;
    a.n_cur = &E.d_ctl->n_cur;
    a.out_count = &E.d_ctl->out_count;
    a.work = &E.d_ctl->work;
    a.mask = &E.d_ctl->mask;
    a.table_size = E.table_size;
    a.n_active = &E.d_ctl->n_active;
    a.visits = &E.d_ctl->visits;
    a.n_resident = &E.d_ctl->n_resident;
    a.blocks_done = &E.d_ctl->blocks_done;
    return a;
}

// Enqueues `rounds` rounds (even) on the stream; with `events`, records a
// timing event pair around every step kernel.
void enqueue_round(Engine &E, unsigned r, bool events, bool external) {
    DeviceLineages &in = (r % 2 == 0) ? E.A : E.B;
    DeviceLineages &out = (r % 2 == 0) ? E.B : E.A;
    if (E.learned) {
        // predictions for lineages without one, then this round's queue
        // order by expected work (largest first)
        const FeatureArgs f = make_feature_args(E, in);
        CK(launch_lineage_predict(f, E.model_w, in.soa.pred_end, E.stream));
        CK(launch_order(f, in.soa.pred_end, E.order_keys, E.order_hist, E.order, E.aux_grid, E.stream));
    }
    if (events) {
        if (external)
            CK(cudaEventRecordWithFlags(E.ev_start[r], E.stream, cudaEventRecordExternal));
        else
            CK(cudaEventRecord(E.ev_start[r], E.stream));
    }
    CK(launch_step(E.kind, make_step_args(E, in), E.step_grid, E.step_block, E.coop_grid, E.stream));
    if (events) {
        if (external)
            CK(cudaEventRecordWithFlags(E.ev_end[r], E.stream, cudaEventRecordExternal));
        else
            CK(cudaEventRecord(E.ev_end[r], E.stream));
    }
    CK(launch_dedup(make_dedup_args(E, in, out), E.aux_grid, E.aux_block, E.stream));
    CK(launch_schedule(make_schedule_args(E), E.stream));
}

void enqueue_rounds(Engine &E, unsigned rounds, bool events, bool external) {
    for (unsigned r = 0; r < rounds; ++r) enqueue_round(E, r, events, external);
}

// Delivers the events of the round that just ended (dispersal reporting).
void drain_events(Engine &E);

void build_graph(Engine &E) {
    const unsigned rounds = E.args.rounds_per_graph;
    E.ev_start.resize(rounds);
    E.ev_end.resize(rounds);
    for (unsigned r = 0; r < rounds; ++r) {
        CK(cudaEventCreate(&E.ev_start[r]));
        CK(cudaEventCreate(&E.ev_end[r]));
    }
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(E.stream, cudaStreamCaptureModeThreadLocal));
    try {
        enqueue_rounds(E, rounds, true, true);
    } catch (...) {
        cudaStreamEndCapture(E.stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    CK(cudaStreamEndCapture(E.stream, &graph));
    cudaError_t e = cudaGraphInstantiate(&E.graph_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) throw CudaFailure{e, "cudaGraphInstantiate"};
}

struct RunResult {
    double kernel_ms = 0.0;
    double total_ms = 0.0;
    double resident_ms = 0.0;
    uint64_t launches = 0;
    uint64_t rounds_launched = 0;
};

// The round loop: initial schedule, then graphs of `rounds_per_graph` rounds
// until no simulation is active.
RunResult run_rounds(Engine &E) {
    RunResult rr;
    const unsigned rounds = E.args.rounds_per_graph;
    CK(cudaEventRecord(E.ev_total0, E.stream));
    reset_lineages(E);
    // initial control state
    Control c;
    std::memset(&c, 0, sizeof(c));
    c.out_count = E.n_total;
    CK(cudaMemcpyAsync(E.d_ctl, &c, sizeof(c), cudaMemcpyHostToDevice, E.stream));
    E.h2d_bytes += sizeof(c) + E.sims.size() * (sizeof(SimParams) + sizeof(SimCounters));
    std::vector<SimParams> ps(E.sims.size());
    std::vector<SimCounters> cs(E.sims.size());
    for (size_t s = 0; s < E.sims.size(); ++s) {
        ps[s] = E.sims[s].params;
        ps[s].horizon = E.sims[s].start_time;
        ps[s].active = 0;
        std::memset(&cs[s], 0, sizeof(SimCounters));
        cs[s].n_live_next = E.sims[s].n_origins;
    }
    CK(cudaMemcpyAsync(E.d_params, ps.data(), ps.size() * sizeof(SimParams), cudaMemcpyHostToDevice, E.stream));
    CK(cudaMemcpyAsync(E.d_counters, cs.data(), cs.size() * sizeof(SimCounters), cudaMemcpyHostToDevice, E.stream));
    CK(launch_schedule(make_schedule_args(E), E.stream));
    rr.launches += 1;
    if (E.tracing) CK(launch_trace_snapshot(make_feature_args(E, E.A), E.trace_snap++, E.trace_rows,
                                            E.trace_counts, E.trace_rows_cap, E.stream));
    const bool gate_owner = E.gate && E.gate_role == kGateOnly;
    if (gate_owner) {
        CK(cudaMemsetAsync(&E.gate->on, 0, sizeof(uint32_t), E.stream));
        E.gate_on = false;
    }
    CK(cudaMemcpyAsync(E.h_ctl, E.d_ctl, sizeof(Control), cudaMemcpyDeviceToHost, E.stream));
    CK(cudaStreamSynchronize(E.stream));
    uint64_t graph_launches = 0;
    uint64_t stalled = 0;
    unsigned long long last_steps = ~0ULL, last_live = ~0ULL;
    // one block per resident simulation, at most two per SM
    // at most one block per SM beside the global rounds (room for their
    // kernels), two per SM when only resident simulations are left
    const uint64_t max_rounds = E.args.max_rounds ? E.args.max_rounds : (1ULL << 26);
    const unsigned grid_beside = (unsigned)std::min<size_t>(E.sims.size(), (size_t)E.n_sms);
    const unsigned grid_alone = (unsigned)std::min<size_t>(E.sims.size(), (size_t)E.n_sms * 2);
    // The resident kernel runs on its own stream, decoupled from the global
    // rounds: the main stream never waits for it.  A finished launch is
    // relaunched at the next graph boundary; routed simulations are handed
    // over (promote) on the main stream, between graphs, only while no
    // resident launch is in flight.
    bool res_inflight = false;
    while (E.h_ctl->n_active > 0 || E.h_ctl->n_resident > 0 || res_inflight) {
        // every round advances each active simulation's horizon by at least
        // step_slice / lambda, so each live lineage expects >= step_slice
        // events per round: a valid run never reaches these bounds
        if (++graph_launches > max_rounds / rounds + (max_rounds % rounds ? 1 : 0))
            fail(NECSIM_E_TIMEOUT, "round limit reached (necsim_args.max_rounds)");
        if (E.h_ctl->steps_total == last_steps && E.h_ctl->n_cur == last_live && !res_inflight) {
            if (++stalled >= 64) fail(NECSIM_E_TIMEOUT, "no progress over 64 graph launches");
        } else {
            stalled = 0;
        }
        last_steps = E.h_ctl->steps_total;
        last_live = E.h_ctl->n_cur;
        const bool global = E.h_ctl->n_active > 0;
        if (E.args.resident) {
            if (res_inflight && cudaEventQuery(E.ev_res1) == cudaSuccess) {
                float ms = 0.f;
                if (cudaEventElapsedTime(&ms, E.ev_res0, E.ev_res1) == cudaSuccess) rr.resident_ms += ms;
                res_inflight = false;
            }
            // n_resident counts the routed simulations too
            if (!res_inflight && E.h_ctl->n_resident > 0) {
                // hand routed simulations over, then run the resident kernel
                // on its own stream beside the global rounds (short stretches
                // while they run, so newly routed simulations wait little;
                // long ones when only resident simulations are left)
                CK(cudaStreamWaitEvent(E.stream, E.ev_res1, 0));  // the last resident launch has ended
                CK(launch_promote(E.d_params, (uint32_t)E.sims.size(), E.stream));
                CK(cudaEventRecord(E.ev_fork, E.stream));
                CK(cudaStreamWaitEvent(E.stream_t, E.ev_fork, 0));
                const uint32_t budget = global ? 32 : 256;
                unsigned grid = global ? grid_beside : grid_alone;
                if (E.gate) {
                    // claims and arrivals of the launch start at zero; the
                    // priority engine's blocks, confined to the reserved SMs,
                    // come in a grid large enough to reach all of them
                    CK(cudaMemsetAsync(&E.d_ctl->res_claim, 0, 2 * sizeof(unsigned int), E.stream_t));
                    if (gate_owner && E.gate_on) grid = (unsigned)E.n_sms * 2;
                }
                CK(cudaEventRecord(E.ev_res0, E.stream_t));
                CK(launch_resident(E.kind, make_resident_args(E, budget, nullptr), grid, E.stream_t));
                CK(cudaEventRecord(E.ev_res1, E.stream_t));
                res_inflight = true;
                rr.launches += 2;
                rr.rounds_launched += 1;
            }
        }
        if (global) {
            if (E.delivery) {
                // one round at a time: its events leave the device before the next
                for (unsigned r = 0; r < rounds; ++r) {
                    enqueue_round(E, r, true, false);
                    CK(cudaStreamSynchronize(E.stream));
                    drain_events(E);
                }
            } else if (E.graph_exec && E.timing_in_graph) {
                CK(cudaGraphLaunch(E.graph_exec, E.stream));
            } else {
                enqueue_rounds(E, rounds, true, false);
            }
            rr.launches += (uint64_t)rounds * ((E.learned ? 9 : 5) + (E.coop_max ? 1 : 0));
            // after an even number of rounds the live lineages are in A
            if (E.tracing) CK(launch_trace_snapshot(make_feature_args(E, E.A), E.trace_snap++, E.trace_rows,
                                                    E.trace_counts, E.trace_rows_cap, E.stream));
            rr.rounds_launched += rounds;
        } else if (res_inflight) {
            // only resident simulations are left: wait for their launch
            CK(cudaEventSynchronize(E.ev_res1));
        }
        CK(cudaMemcpyAsync(E.h_ctl, E.d_ctl, sizeof(Control), cudaMemcpyDeviceToHost, E.stream));
        E.d2h_bytes += sizeof(Control);
        CK(cudaStreamSynchronize(E.stream));
        if (global) {
            for (unsigned r = 0; r < rounds; ++r) {
                float ms = 0.f;
                if (cudaEventElapsedTime(&ms, E.ev_start[r], E.ev_end[r]) == cudaSuccess) rr.kernel_ms += ms;
            }
        }
        if (E.h_ctl->status & ~kErrDedupFull) break;
        if (gate_owner && !E.gate_on && E.h_ctl->n_cur <= E.gate_lineages) {
            // the priority engine's bulk is over: its tails take the reserved
            // SMs, the other engines leave them
            CK(cudaMemsetAsync(&E.gate->on, 1, sizeof(uint32_t), E.stream));
            E.gate_on = true;
        }
    }
    if (res_inflight) CK(cudaEventSynchronize(E.ev_res1));
    if (gate_owner) {
        // the other engines get every SM back
        CK(cudaMemsetAsync(&E.gate->on, 0, sizeof(uint32_t), E.stream));
        E.gate_on = false;
    }
    // the resident stream's work is part of the run
    if (E.args.resident) {
        CK(cudaEventRecord(E.ev_fork, E.stream_t));
        CK(cudaStreamWaitEvent(E.stream, E.ev_fork, 0));
    }
    CK(cudaEventRecord(E.ev_total1, E.stream));
    CK(cudaEventSynchronize(E.ev_total1));
    float tot = 0.f;
    CK(cudaEventElapsedTime(&tot, E.ev_total0, E.ev_total1));
    rr.total_ms = tot;
    return rr;
}

inline uint64_t bits_of(double v) {
    uint64_t b;
    std::memcpy(&b, &v, 8);
    return b;
}

// PackedEvent::cmp (necsim/core/src/event.rs:256-280) for speciation events
// (target == origin), per simulation.
bool spec_less(const DevSpeciationEvent &a, const DevSpeciationEvent &b) {
    if (a.sim != b.sim) return a.sim < b.sim;
    const uint64_t ta = bits_of(a.event_time), tb = bits_of(b.event_time);
    if (ta != tb) return ta < tb;
    if (a.x != b.x) return a.x < b.x;
    if (a.y != b.y) return a.y < b.y;
    if (a.idx != b.idx) return a.idx < b.idx;
    const uint64_t pa = bits_of(a.prior_time), pb = bits_of(b.prior_time);
    if (pa != pb) return pa < pb;
    return a.gref < b.gref;
}

bool disp_less(const DevDispersalEvent &a, const DevDispersalEvent &b) {
    if (a.sim != b.sim) return a.sim < b.sim;
    const uint64_t ta = bits_of(a.event_time), tb = bits_of(b.event_time);
    if (ta != tb) return ta < tb;
    if (a.x != b.x) return a.x < b.x;
    if (a.y != b.y) return a.y < b.y;
    if (a.idx != b.idx) return a.idx < b.idx;
    if (a.tx != b.tx) return a.tx < b.tx;
    if (a.ty != b.ty) return a.ty < b.ty;
    if (a.tidx != b.tidx) return a.tidx < b.tidx;
    const uint64_t pa = bits_of(a.prior_time), pb = bits_of(b.prior_time);
    if (pa != pb) return pa < pb;
    return a.gref < b.gref;
}

// PackedEvent::cmp (event.rs:256-280) between a speciation event (whose
// target is its origin, event.rs:105-115) and a dispersal event of the same
// simulation: event time, origin, target, prior time, global reference.
bool spec_before_disp(const DevSpeciationEvent &a, const DevDispersalEvent &b) {
    const uint64_t ta = bits_of(a.event_time), tb = bits_of(b.event_time);
    if (ta != tb) return ta < tb;
    if (a.x != b.x) return a.x < b.x;
    if (a.y != b.y) return a.y < b.y;
    if (a.idx != b.idx) return a.idx < b.idx;
    if (a.x != b.tx) return a.x < b.tx;
    if (a.y != b.ty) return a.y < b.ty;
    if (a.idx != b.tidx) return a.idx < b.tidx;
    const uint64_t pa = bits_of(a.prior_time), pb = bits_of(b.prior_time);
    if (pa != pb) return pa < pb;
    return a.gref <= b.gref;
}

void drain_events(Engine &E) {
    Delivery &dv = *E.delivery;
    Control c;
    CK(cudaMemcpy(&c, E.d_ctl, sizeof(c), cudaMemcpyDeviceToHost));
    if (c.n_disp_total > E.disp_cap || (c.status & kErrDispersalOverflow))
        fail(NECSIM_E_TOO_LARGE, "one round produced more dispersal events than the event buffer holds "
                                 "(lower min_round_events or batch fewer simulations)");
    const uint64_t nd = c.n_disp_total, nsp = std::min<uint64_t>(c.n_spec_total, E.spec_cap);
    std::vector<DevSpeciationEvent> sp(nsp);
    std::vector<DevDispersalEvent> di(nd);
    if (nsp) CK(cudaMemcpy(sp.data(), E.d_spec, nsp * sizeof(DevSpeciationEvent), cudaMemcpyDeviceToHost));
    if (nd) CK(cudaMemcpy(di.data(), E.d_disp, nd * sizeof(DevDispersalEvent), cudaMemcpyDeviceToHost));
    E.d2h_bytes += sizeof(c) + nsp * sizeof(DevSpeciationEvent) + nd * sizeof(DevDispersalEvent);
    // the next round appends from the start of both buffers
    CK(cudaMemset(&E.d_ctl->n_spec_total, 0, sizeof(unsigned long long)));
    CK(cudaMemset(&E.d_ctl->n_disp_total, 0, sizeof(unsigned long long)));
    std::sort(sp.begin(), sp.end(), spec_less);
    std::sort(di.begin(), di.end(), disp_less);
    // per simulation: one stream in PackedEvent order, consecutive events of
    // one kind delivered in one call
    size_t i = 0, j = 0;
    std::vector<necsim_speciation_event> out_s;
    std::vector<necsim_dispersal_event> out_d;
    while (i < sp.size() || j < di.size()) {
        const uint32_t s = (j >= di.size() || (i < sp.size() && sp[i].sim <= di[j].sim)) ? sp[i].sim : di[j].sim;
        const necsim_reporter *rep = dv.reporters ? (dv.one_reporter ? dv.reporters : &dv.reporters[s]) : nullptr;
        auto flush_s = [&] {
            if (!out_s.empty() && rep && rep->report_speciation &&
                rep->report_speciation(rep->user, out_s.data(), out_s.size()) != 0)
                fail(NECSIM_E_CALLBACK, "reporter stopped the delivery");
            out_s.clear();
        };
        auto flush_d = [&] {
            if (!out_d.empty() && rep && rep->report_dispersal &&
                rep->report_dispersal(rep->user, out_d.data(), out_d.size()) != 0)
                fail(NECSIM_E_CALLBACK, "reporter stopped the delivery");
            out_d.clear();
        };
        while ((i < sp.size() && sp[i].sim == s) || (j < di.size() && di[j].sim == s)) {
            const bool take_s = i < sp.size() && sp[i].sim == s &&
                                (j >= di.size() || di[j].sim != s || spec_before_disp(sp[i], di[j]));
            if (take_s) {
                flush_d();
                const DevSpeciationEvent &e = sp[i++];
                // BiodiversityReporter (plugins/common/src/biodiversity.rs:32-45)
                if (!dv.has_last[s] || !(dv.last[s].x == e.x && dv.last[s].y == e.y && dv.last[s].idx == e.idx &&
                                         dv.last[s].event_time == e.event_time))
                    dv.species[s] += 1;
                dv.last[s] = e;
                dv.has_last[s] = 1;
                necsim_speciation_event r;
                r.global_lineage_reference = e.gref;
                r.prior_time = e.prior_time;
                r.event_time = e.event_time;
                r.x = e.x;
                r.y = e.y;
                r.index = e.idx;
                r.pad = 0;
                out_s.push_back(r);
            } else {
                flush_s();
                const DevDispersalEvent &e = di[j++];
                dv.n_dispersal[s] += 1;
                necsim_dispersal_event r;
                r.global_lineage_reference = e.gref;
                r.prior_time = e.prior_time;
                r.event_time = e.event_time;
                r.x = e.x;
                r.y = e.y;
                r.index = e.idx;
                r.target_x = e.tx;
                r.target_y = e.ty;
                r.target_index = e.tidx;
                r.pad = 0;
                r.pad2 = 0;
                out_d.push_back(r);
            }
        }
        flush_s();
        flush_d();
    }
}

struct Remaining {
    std::vector<std::vector<necsim_lineage>> per_sim;
};

// Collects counters, surviving lineages and events after the rounds; fills
// the outcomes and delivers events to the reporters.
void finish(Engine &E, const RunResult &rr, const necsim_reporter *reporters, bool one_reporter,
            necsim_outcome *outcomes, Remaining &rem) {
    const size_t ns = E.sims.size();
    std::vector<SimCounters> cs(ns);
    CK(cudaMemcpy(cs.data(), E.d_counters, ns * sizeof(SimCounters), cudaMemcpyDeviceToHost));
    Control c;
    CK(cudaMemcpy(&c, E.d_ctl, sizeof(c), cudaMemcpyDeviceToHost));
    if (c.status & kErrDispersalRejections)
        fail(NECSIM_E_DISPERSAL_REJECTED, "a WrappingNoise dispersal rejected " + std::to_string(kMaxDispersalRejections) +
                                              " targets in a row");
    if (c.status & (kErrCellIndex | kErrAtomIndex | kErrEventOverflow | kErrDispersalOverflow | kErrResident))
        fail(NECSIM_E_DEVICE_CHECK, "device bound check failed (status " + std::to_string(c.status) + ")");
    // surviving lineages live in A after an even number of rounds
    const uint64_t n = c.n_cur;
    LineageSoA &d = E.A.soa;
    std::vector<uint32_t> x(n), y(n), idx(n), sim(n);
    std::vector<double> last(n);
    std::vector<uint64_t> gref(n), steps(n);
    if (n) {
        CK(cudaMemcpy(x.data(), d.x, n * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(y.data(), d.y, n * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(idx.data(), d.idx, n * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(sim.data(), d.sim, n * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(last.data(), d.last, n * 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(gref.data(), d.gref, n * 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(steps.data(), d.steps, n * 8, cudaMemcpyDeviceToHost));
    }
    // simulations that ended in the resident kernel keep their survivors in
    // their segment of the resident arena
    std::vector<SimParams> ps(ns);
    CK(cudaMemcpy(ps.data(), E.d_params, ns * sizeof(SimParams), cudaMemcpyDeviceToHost));
    for (size_t s = 0; s < ns; ++s) {
        if (!ps[s].resident || cs[s].n_live == 0) continue;
        const uint64_t m = cs[s].n_live, o = ps[s].lineage_offset;
        const size_t base = x.size();
        x.resize(base + m);
        y.resize(base + m);
        idx.resize(base + m);
        sim.resize(base + m);
        last.resize(base + m);
        gref.resize(base + m);
        steps.resize(base + m);
        const LineageSoA &r = E.R.soa;
        CK(cudaMemcpy(x.data() + base, r.x + o, m * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(y.data() + base, r.y + o, m * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(idx.data() + base, r.idx + o, m * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(last.data() + base, r.last + o, m * 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(gref.data() + base, r.gref + o, m * 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(steps.data() + base, r.steps + o, m * 8, cudaMemcpyDeviceToHost));
        for (uint64_t k = 0; k < m; ++k) sim[base + k] = (uint32_t)s;
        E.d2h_bytes += m * 36;
    }
    rem.per_sim.assign(ns, {});
    std::vector<uint64_t> extra_steps(ns, 0);
    std::vector<double> extra_time(ns, 0.0);
    for (uint64_t j = 0; j < x.size(); ++j) {
        const uint32_t s = sim[j];
        extra_steps[s] += steps[j];
        extra_time[s] = std::max(extra_time[s], last[j]);
        necsim_lineage l;
        l.global_reference = gref[j];
        l.last_event_time = last[j];
        l.x = x[j];
        l.y = y[j];
        l.index = idx[j];
        l.pad = 0;
        rem.per_sim[s].push_back(l);
    }
    for (auto &v : rem.per_sim)
        std::sort(v.begin(), v.end(), [](const necsim_lineage &a, const necsim_lineage &b) {
            return a.global_reference < b.global_reference;
        });

    const uint64_t n_spec = std::min<uint64_t>(c.n_spec_total, E.spec_cap);
    std::vector<DevSpeciationEvent> ev(n_spec);
    if (n_spec)
        CK(cudaMemcpy(ev.data(), E.d_spec, n_spec * sizeof(DevSpeciationEvent), cudaMemcpyDeviceToHost));
    std::sort(ev.begin(), ev.end(), spec_less);
    E.d2h_bytes += ns * sizeof(SimCounters) + sizeof(Control) + n * (4 * 4 + 8 * 3) +
                   n_spec * sizeof(DevSpeciationEvent);

    // the simulations' timeline on the device clock, from the run's first schedule
    uint64_t base = 0;
    for (size_t s = 0; s < ns; ++s)
        if (cs[s].start_ns && (base == 0 || cs[s].start_ns < base)) base = cs[s].start_ns;
    E.first_start_ns = base;
    auto since = [base](unsigned long long t) { return t > base ? (double)(t - base) / 1e6 : 0.0; };
    size_t pos = 0;
    for (size_t s = 0; s < ns; ++s) {
        necsim_outcome &o = outcomes[s];
        std::memset(&o, 0, sizeof(o));
        o.end_ms = since(cs[s].end_ns);
        o.routed_ms = cs[s].routed_ns ? since(cs[s].routed_ns) : -1.0;
        double t;
        uint64_t tb = cs[s].max_time_bits;
        std::memcpy(&t, &tb, 8);
        // max_time: initial last event times (monolithic/mod.rs:121-126), every
        // executed event, and min_event_time once a lineage was simulated
        // (active_lineage_sampler/independent/sampler.rs:64-66)
        o.time = std::max(std::max(t, extra_time[s]), E.sims[s].start_max);
        if (cs[s].n_rounds > 0 && E.sims[s].n_origins > 0)
            o.time = std::max(o.time, E.sims[s].params.min_event_time);
        o.steps = cs[s].steps + extra_steps[s];
        o.n_initial = E.sims[s].n_origins;
        o.n_remaining = rem.per_sim[s].size();
        o.paused = o.n_remaining > 0 ? 1 : 0;
        o.n_speciation = cs[s].n_speciation;
        o.n_rounds = cs[s].n_rounds;
        o.n_dedup = cs[s].n_dedup;
        o.n_launches = rr.launches;
        o.kernel_ms = rr.kernel_ms;
        o.total_ms = rr.total_ms;
        o.resident_ms = rr.resident_ms;
        o.h2d_bytes = E.h2d_bytes;
        o.d2h_bytes = E.d2h_bytes;
        o.n_step_launches = rr.rounds_launched;
        o.lineage_visits = c.visits;
        // deliver this simulation's events in PackedEvent order; count
        // species like BiodiversityReporter (plugins/common/src/biodiversity.rs:32-45)
        if (E.delivery) {
            // delivered round by round with the dispersal events
            o.biodiversity = E.delivery->species[s];
            o.n_dispersal = E.delivery->n_dispersal[s];
            continue;
        }
        size_t end = pos;
        while (end < ev.size() && ev[end].sim == s) ++end;
        std::vector<necsim_speciation_event> out;
        out.reserve(end - pos);
        uint64_t species = 0;
        for (size_t k = pos; k < end; ++k) {
            const DevSpeciationEvent &e = ev[k];
            if (k == pos || !(ev[k - 1].x == e.x && ev[k - 1].y == e.y && ev[k - 1].idx == e.idx &&
                              ev[k - 1].event_time == e.event_time))
                ++species;
            necsim_speciation_event r;
            r.global_lineage_reference = e.gref;
            r.prior_time = e.prior_time;
            r.event_time = e.event_time;
            r.x = e.x;
            r.y = e.y;
            r.index = e.idx;
            r.pad = 0;
            out.push_back(r);
        }
        o.biodiversity = species;
        const necsim_reporter *rep = reporters ? (one_reporter ? reporters : &reporters[s]) : nullptr;
        if (rep && rep->report_speciation && !out.empty()) {
            if (rep->report_speciation(rep->user, out.data(), out.size()) != 0)
                fail(NECSIM_E_CALLBACK, "reporter stopped the delivery");
        }
        pos = end;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct necsim_ctx {
    std::unique_ptr<Engine> engine;
    necsim_scenario scenario{};
    necsim_args args{};
    std::vector<uint32_t> habitat;  // owned copies of the SE maps' habitat
    std::vector<double> turnover;   // and turnover map (when given)
    std::string error;
    Remaining remaining;
    bool tables_ready = false;
    SimParams table_params{};  // cells/atoms pointers of the uploaded tables
};

namespace {

int report(necsim_ctx *ctx, char *buf, size_t cap, int code, const std::string &msg) {
    if (ctx) ctx->error = msg;
    if (buf && cap) {
        std::snprintf(buf, cap, "%s", msg.c_str());
    }
    return code;
}

template <typename F>
int guarded(necsim_ctx *ctx, char *buf, size_t cap, F &&f) {
    try {
        f();
        if (ctx) ctx->error.clear();
        return NECSIM_OK;
    } catch (const ApiError &e) {
        return report(ctx, buf, cap, e.code, e.msg);
    } catch (const CudaFailure &e) {
        return report(ctx, buf, cap, NECSIM_E_CUDA,
                      std::string(e.what) + ": " + cudaGetErrorString(e.err));
    } catch (const std::bad_alloc &) {
        return report(ctx, buf, cap, NECSIM_E_OUT_OF_MEMORY, "host allocation failed");
    } catch (...) {
        return report(ctx, buf, cap, NECSIM_E_INVALID_ARGUMENT, "unexpected failure");
    }
}

// Runs simulations (one or a batch) end to end on a fresh engine.
void prepare_engine(Engine &E, std::vector<SimHost> sims, const necsim_args &args,
                    const std::vector<std::vector<necsim_lineage>> *given,
                    const std::vector<SimParams> *prebuilt_tables);

// Executes one run of a prepared engine: reset to the resident origins,
// rounds, collection and delivery.
void execute_engine(Engine &E, const necsim_reporter *reporters, bool one_reporter,
                    necsim_outcome *outcomes, Remaining &rem) {
    RunResult rr;
    Delivery dv;
    if (E.args.report_dispersal) {
        const size_t ns = E.sims.size();
        dv.reporters = reporters;
        dv.one_reporter = one_reporter;
        dv.species.assign(ns, 0);
        dv.n_dispersal.assign(ns, 0);
        dv.last.assign(ns, DevSpeciationEvent{});
        dv.has_last.assign(ns, 0);
        E.delivery = &dv;
    }
    try {
        if (E.n_total > 0) rr = run_rounds(E);
        finish(E, rr, reporters, one_reporter, outcomes, rem);
    } catch (...) {
        E.delivery = nullptr;
        throw;
    }
    E.delivery = nullptr;
}

void run_simulations(Engine &E, std::vector<SimHost> sims, const necsim_args &args,
                     const std::vector<std::vector<necsim_lineage>> *given,
                     const necsim_reporter *reporters, bool one_reporter, necsim_outcome *outcomes,
                     Remaining &rem, const std::vector<SimParams> *prebuilt_tables) {
    prepare_engine(E, std::move(sims), args, given, prebuilt_tables);
    execute_engine(E, reporters, one_reporter, outcomes, rem);
}

void prepare_engine(Engine &E, std::vector<SimHost> sims, const necsim_args &args,
                    const std::vector<std::vector<necsim_lineage>> *given,
                    const std::vector<SimParams> *prebuilt_tables) {
    // the device runs Clark2Dt as AlmostInfinite with its dispersal switch
    auto device_kind = [](int32_t k) { return k == NECSIM_ALMOST_INFINITE_CLARK2DT ? NECSIM_ALMOST_INFINITE_NORMAL : k; };
    E.kind = device_kind(sims.front().sc.kind);
    for (auto &s : sims)
        if (device_kind(s.sc.kind) != E.kind) fail(NECSIM_E_UNSUPPORTED, "a batch must share one scenario kind");
    if (args.schedule > 1) fail(NECSIM_E_INVALID_ARGUMENT, "schedule must be 0 (plain) or 1 (learned)");
    if (args.event_time_sampler > NECSIM_SAMPLER_EXP)
        fail(NECSIM_E_INVALID_ARGUMENT, "event_time_sampler must be 0 (Poisson) or 1 (Exp)");
    E.learned = args.schedule == 1;
    if (E.learned) {
        if (!args.model) fail(NECSIM_E_INVALID_ARGUMENT, "the learned schedule needs a model");
        if (args.model->device != E.device) fail(NECSIM_E_INVALID_ARGUMENT, "the model lives on another device");
        E.model_w = args.model->w;
    }
    if (args.report_dispersal) {
        // every lineage stays in the global rounds, which drain the events
        // after each round; the buffer holds twice a round's expected events
        // (n * per <= max(min_round_events + n, step_slice * n) per simulation)
        E.args.resident = 0;
        uint64_t bound = 0;
        for (auto &sh : sims)
            bound += std::max<uint64_t>(args.min_round_events + sh.n_origins, args.step_slice * sh.n_origins);
        E.disp_cap = 2 * bound + (1ULL << 20);
        if (E.disp_cap * sizeof(DevDispersalEvent) > (16ULL << 30))
            fail(NECSIM_E_TOO_LARGE, "dispersal event buffer above 16 GiB (lower min_round_events or batch "
                                     "fewer simulations)");
    }
    uint64_t off = 0;
    for (auto &s : sims) {
        s.lineage_offset = off;
        s.params.lineage_offset = off;
        off += s.n_origins;
    }
    if (off >= 0xffffffffULL) fail(NECSIM_E_TOO_LARGE, "more than 2^32 - 1 lineages");
    E.sims = std::move(sims);
    E.n_total = off;
    for (size_t s = 0; s < E.sims.size(); ++s) {
        SimHost &sh = E.sims[s];
        if (sh.sc.kind == NECSIM_SPATIALLY_EXPLICIT) {
            if (prebuilt_tables) {
                sh.params.cells = (*prebuilt_tables)[s].cells;
                sh.params.atoms = (*prebuilt_tables)[s].atoms;
                sh.params.n_cells = (*prebuilt_tables)[s].n_cells;
                sh.params.n_atoms = (*prebuilt_tables)[s].n_atoms;
                sh.params.cell_entropy = (*prebuilt_tables)[s].cell_entropy;
                sh.params.turnover_cells = (*prebuilt_tables)[s].turnover_cells;
            } else {
                upload_tables(E, sh);
            }
        }
        // the Poisson sampler's Devroye inversion needs p0 > 0 (the Exp
        // sampler draws no counts)
        if (args.event_time_sampler != NECSIM_SAMPLER_EXP && !(sh.params.p0 > 0.0))
            fail(NECSIM_E_UNSUPPORTED, "exp(-lambda * delta_t) underflows to 0");
    }
    // a single simulation stays in the global rounds, whose sparse rounds
    // step each lineage with a whole warp on any SM (the resident kernel
    // gives a simulation one SM)
    if (E.sims.size() == 1) E.args.resident = 0;
    choose_launch(E);
    alloc_run_buffers(E);
    upload_origins(E, given);
    if (E.n_total > 0) build_graph(E);
}

// ---- a batch split into engines: priority simulations each run alone ----
//
// The rounds of a batch are synchronised: every round waits for the slowest
// lineage of every simulation, so a long-lived simulation advances at the
// pace of the whole batch.  A priority simulation gets an engine of its own
// (its own rounds, stream and host thread) and runs beside the others.  The
// canonical schedule of every simulation depends only on that simulation,
// so the split changes no result.
struct BatchRun {
    // engines[0 .. n_groups): the priority groups of the simulations outside
    // the priority engines, in decreasing stream priority (engines[0] may be
    // empty); then the priority engines, when there are priority simulations
    std::vector<std::unique_ptr<Engine>> engines;
    std::vector<std::vector<uint32_t>> members;  // batch indices of each engine's simulations
    std::vector<Remaining> rem;
    size_t n_groups = 1;
    std::vector<uint32_t> priority;  // the priority simulations, in priority order
    // the SM reservation shared by the engines (args.reserve_sms > 0 and a
    // priority engine), freed after the engines are released
    struct GateMem {
        SmGate *p = nullptr;
        ~GateMem() {
            if (p) cudaFree(p);
        }
    };
    GateMem gate;
};

// Sets aside `count` of the device's SMs for the priority engine: the SM ids
// present (a census kernel), every (present / count)-th of them, so the
// reserved SMs spread over the dies.  Returns the number reserved.
uint32_t reserve_sms(SmGate *gate, int device, int n_sms, uint32_t count) {
    CK(cudaSetDevice(device));
    SmGate g;
    std::memset(&g, 0, sizeof(g));
    CK(cudaMemset(gate, 0, sizeof(SmGate)));
    CK(launch_sm_census(gate->mask, (unsigned)n_sms * 16u, 0));
    CK(cudaMemcpy(g.mask, gate->mask, sizeof(g.mask), cudaMemcpyDeviceToHost));
    std::vector<uint32_t> present;
    for (uint32_t id = 0; id < 256; ++id)
        if ((g.mask[id >> 5] >> (id & 31)) & 1u) present.push_back(id);
    std::memset(g.mask, 0, sizeof(g.mask));
    uint32_t n = 0;
    if (!present.empty() && count < present.size()) {
        const double stride = (double)present.size() / (double)count;
        for (uint32_t k = 0; k < count; ++k) {
            const uint32_t id = present[(size_t)((double)k * stride)];
            g.mask[id >> 5] |= 1u << (id & 31);
            ++n;
        }
    }
    g.on = 0;
    CK(cudaMemcpy(gate, &g, sizeof(g), cudaMemcpyHostToDevice));
    return n;
}

// The batch's simulations in priority order: with the learned schedule the
// lifetime model's longest-lived first, else batch order; then the priority
// simulations are priority_list's first priority_sims entries, else with the
// learned schedule the order's first priority_sims (default 8), at most all
// but one simulation.
void choose_priority(const std::vector<SimHost> &sims, const necsim_args &args, std::vector<uint32_t> &order,
                     std::vector<uint32_t> &prio) {
    const uint32_t n = (uint32_t)sims.size();
    order.resize(n);
    for (uint32_t j = 0; j < n; ++j) order[j] = j;
    prio.clear();
    const bool learned = args.schedule == 1 && args.model;
    if (learned && n > 1) {
        const std::vector<float> score = score_simulations(args.model, sims);
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return score[a] > score[b]; });
    }
    if (n < 2 || args.report_dispersal) return;
    if (args.priority_list && args.priority_sims) {
        std::vector<uint8_t> seen(n, 0);
        for (uint32_t k = 0; k < args.priority_sims; ++k) {
            const uint32_t j = args.priority_list[k];
            if (j >= n) fail(NECSIM_E_INVALID_ARGUMENT, "priority_list names a simulation outside the batch");
            if (!seen[j]) prio.push_back(j);
            seen[j] = 1;
        }
        if (prio.size() >= n) prio.pop_back();  // keep one simulation for the shared engines
        return;
    }
    if (!learned) return;
    const uint32_t k = std::min<uint32_t>(args.priority_sims ? args.priority_sims : 8, n - 1);
    prio.assign(order.begin(), order.begin() + k);
}

// Stream priority of priority level g (0: the device's greatest); levels
// beyond the device's range share its least priority.
int stream_priority_level(int device, size_t g) {
    int least = 0, greatest = 0;
    CK(cudaSetDevice(device));
    CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    return (int)std::min<long long>((long long)greatest + (long long)g, (long long)least);
}

void prepare_batch(BatchRun &b, std::vector<SimHost> sims, const necsim_args &args) {
    std::vector<uint32_t> order, prio;
    choose_priority(sims, args, order, prio);
    std::vector<uint8_t> is_prio(sims.size(), 0);
    for (uint32_t j : prio) is_prio[j] = 1;
    std::vector<uint32_t> rest_ids;
    for (uint32_t j : order)
        if (!is_prio[j]) rest_ids.push_back(j);
    // the others in priority groups: contiguous runs of the order, sizes
    // differing by at most one
    const size_t groups = std::max<size_t>(1, std::min<size_t>(args.priority_groups, rest_ids.size()));
    b.engines.clear();
    b.members.clear();
    b.n_groups = groups;
    const bool staggered = groups > 1;
    // the priority simulations' engines: contiguous runs of the priority
    // order, one engine by default
    const size_t n_prio_engines =
        prio.empty() ? 0 : (args.priority_engines ? std::min<size_t>(args.priority_engines, prio.size()) : 1);
    // SMs set aside for the priority engine's tails (one priority engine)
    uint32_t reserved = 0;
    if (args.reserve_sms && n_prio_engines == 1 && !rest_ids.empty()) {
        cudaDeviceProp prop;
        CK(cudaGetDeviceProperties(&prop, args.device));
        if (!b.gate.p) b.gate.p = dev_alloc<SmGate>(1);
        reserved = reserve_sms(b.gate.p, args.device, prop.multiProcessorCount,
                               std::min<uint32_t>(args.reserve_sms, (uint32_t)prop.multiProcessorCount / 2));
    }
    auto add = [&](std::vector<uint32_t> ids, int level, uint32_t role) {
        std::vector<SimHost> part;
        // an engine's simulations in batch order
        std::sort(ids.begin(), ids.end());
        for (uint32_t j : ids) part.push_back(sims[j]);
        b.engines.emplace_back(new Engine());
        Engine &E = *b.engines.back();
        setup_engine(E, args, level);
        if (reserved) {
            E.gate = b.gate.p;
            E.gate_role = role;
        }
        prepare_engine(E, std::move(part), args, nullptr, nullptr);
        // the reservation starts when the priority engine's live lineages
        // fit its cooperative kernel's warps on the reserved SMs
        if (reserved && role == kGateOnly) {
            int coop_per_sm = 0;
            CK(coop_kernel_occupancy(E.kind, &coop_per_sm));
            E.gate_lineages = (uint64_t)reserved * (uint64_t)std::max(coop_per_sm, 1) * (kCoopBlock / 32);
        }
        b.members.push_back(std::move(ids));
    };
    size_t at = 0;
    for (size_t g = 0; g < groups; ++g) {
        const size_t len = rest_ids.size() / groups + (g < rest_ids.size() % groups ? 1 : 0);
        std::vector<uint32_t> ids(rest_ids.begin() + at, rest_ids.begin() + at + len);
        at += len;
        add(std::move(ids), staggered ? stream_priority_level(args.device, g) : 0, kGateAvoid);
    }
    // the priority engines: their rounds wait for none of the others' (and
    // the others' for none of theirs)
    for (size_t g = 0, pat = 0; g < n_prio_engines; ++g) {
        const size_t len = prio.size() / n_prio_engines + (g < prio.size() % n_prio_engines ? 1 : 0);
        std::vector<uint32_t> ids(prio.begin() + pat, prio.begin() + pat + len);
        pat += len;
        add(std::move(ids), staggered ? stream_priority_level(args.device, 0) : 0, kGateOnly);
    }
    b.priority = prio;
    b.rem.assign(b.engines.size(), Remaining{});
}

// One run of every engine of the batch, the priority engines on their own
// host threads; outcomes in batch order.  The device time of the batch is
// the span from a common start to the last engine's end; kernel times,
// launches and traffic are summed over the engines.
void run_batch(BatchRun &b, const necsim_reporter *reporters, necsim_outcome *outcomes) {
    const size_t ne = b.engines.size();
    if (ne == 1) {
        Engine &E = *b.engines[0];
        E.h2d_bytes = E.d2h_bytes = 0;
        execute_engine(E, reporters, false, outcomes, b.rem[0]);
        return;
    }
    Engine &E0 = *b.engines[0];
    CK(cudaSetDevice(E0.device));
    cudaEvent_t start = nullptr;
    CK(cudaEventCreate(&start));
    struct EventFree {
        cudaEvent_t e;
        ~EventFree() { cudaEventDestroy(e); }
    } start_free{start};
    CK(cudaEventRecord(start, E0.stream));
    CK(cudaEventSynchronize(start));
    std::vector<std::vector<necsim_outcome>> outs(ne);
    std::vector<std::vector<necsim_reporter>> reps(ne);
    std::vector<std::exception_ptr> errs(ne);
    for (size_t e = 0; e < ne; ++e) {
        outs[e].resize(b.members[e].size());
        if (reporters)
            for (uint32_t j : b.members[e]) reps[e].push_back(reporters[j]);
    }
    auto work = [&](size_t e) {
        try {
            Engine &E = *b.engines[e];
            CK(cudaSetDevice(E.device));
            E.h2d_bytes = E.d2h_bytes = 0;
            if (!b.members[e].empty())
                execute_engine(E, reporters ? reps[e].data() : nullptr, false, outs[e].data(), b.rem[e]);
        } catch (...) {
            errs[e] = std::current_exception();
        }
    };
    std::vector<std::thread> threads;
    for (size_t e = 1; e < ne; ++e) threads.emplace_back(work, e);
    work(0);
    for (auto &t : threads) t.join();
    for (auto &err : errs)
        if (err) std::rethrow_exception(err);
    double span = 0.0, kernel = 0.0, resident = 0.0;
    uint64_t launches = 0, steps_l = 0, visits = 0, h2d = 0, d2h = 0;
    // the engines' timelines share the earliest engine's start
    uint64_t base = 0;
    for (size_t e = 0; e < ne; ++e) {
        const uint64_t t = b.engines[e]->first_start_ns;
        if (!b.members[e].empty() && t && (base == 0 || t < base)) base = t;
    }
    for (size_t e = 0; e < ne; ++e) {
        if (b.members[e].empty()) continue;
        float ms = 0.f;
        if (b.engines[e]->n_total > 0 && cudaEventElapsedTime(&ms, start, b.engines[e]->ev_total1) == cudaSuccess)
            span = std::max(span, (double)ms);
        const necsim_outcome &o = outs[e][0];
        kernel += o.kernel_ms;
        resident += o.resident_ms;
        launches += o.n_launches;
        steps_l += o.n_step_launches;
        visits += o.lineage_visits;
        h2d += o.h2d_bytes;
        d2h += o.d2h_bytes;
    }
    for (size_t e = 0; e < ne; ++e) {
        const uint64_t t = b.engines[e]->first_start_ns;
        const double shift = (t > base) ? (double)(t - base) / 1e6 : 0.0;
        for (size_t k = 0; k < b.members[e].size(); ++k) {
            necsim_outcome o = outs[e][k];
            o.end_ms += shift;
            if (o.routed_ms >= 0.0) o.routed_ms += shift;
            o.total_ms = span;
            o.kernel_ms = kernel;
            o.resident_ms = resident;
            o.n_launches = launches;
            o.n_step_launches = steps_l;
            o.lineage_visits = visits;
            o.h2d_bytes = h2d;
            o.d2h_bytes = d2h;
            outcomes[b.members[e][k]] = o;
        }
    }
}

}  // namespace

extern "C" {

int necsim_abi_version(void) { return NECSIM_B200_ABI_VERSION; }

uint64_t necsim_seed_from_u64(uint64_t seed) { return seed_from_u64(seed); }

int necsim_gpu_create(const necsim_scenario *scenario, const necsim_args *args, necsim_ctx **out_ctx) {
    if (!scenario || !out_ctx) return NECSIM_E_INVALID_ARGUMENT;
    *out_ctx = nullptr;
    necsim_ctx *ctx = new (std::nothrow) necsim_ctx();
    if (!ctx) return NECSIM_E_OUT_OF_MEMORY;
    int rc = guarded(ctx, nullptr, 0, [&] {
        validate(*scenario);
        ctx->scenario = *scenario;
        ctx->args = with_defaults(args);
        if (scenario->kind == NECSIM_SPATIALLY_EXPLICIT) {
            const uint64_t cells = (uint64_t)scenario->width * scenario->height;
            ctx->habitat.assign(scenario->habitat, scenario->habitat + cells);
            if (scenario->turnover_map) {
                ctx->turnover.assign(scenario->turnover_map, scenario->turnover_map + cells);
                ctx->scenario.turnover_map = ctx->turnover.data();
            }
            // tables are built and uploaded once per context
            ctx->engine.reset(new Engine());
            setup_engine(*ctx->engine, ctx->args);
            SimHost sh;
            std::memset(&sh, 0, sizeof(sh));
            sh.sc = *scenario;
            sh.params = base_params(*scenario, ctx->args, 0);
            upload_tables(*ctx->engine, sh);
            ctx->table_params = sh.params;
            ctx->tables_ready = true;
            ctx->scenario.habitat = ctx->habitat.data();
            ctx->scenario.dispersal = nullptr;  // consumed by the table build
            ctx->scenario.cells = nullptr;
            ctx->scenario.atoms = nullptr;
        }
    });
    if (rc != NECSIM_OK) {
        // keep the context so the caller can read the message, then fail
        *out_ctx = ctx;
        return rc;
    }
    *out_ctx = ctx;
    return NECSIM_OK;
}

static int simulate_impl(necsim_ctx *ctx, const necsim_lineage *lineages, uint64_t n_lineages,
                         bool resume, double resume_time, uint64_t wyhash_seed, double pause_before,
                         const necsim_reporter *reporter, necsim_outcome *outcome) {
    if (!ctx || !outcome) return NECSIM_E_INVALID_ARGUMENT;
    return guarded(ctx, nullptr, 0, [&] {
        // a fresh engine per simulation; SE tables are carried over
        std::unique_ptr<Engine> tables_owner;
        std::vector<SimParams> prebuilt;
        Engine *E = new Engine();
        std::unique_ptr<Engine> E_owner(E);
        if (ctx->tables_ready) {
            // move the table allocations into this run's engine, then back
            Engine &T = *ctx->engine;
            E->d_cells.swap(T.d_cells);
            E->d_atoms.swap(T.d_atoms);
            prebuilt.push_back(ctx->table_params);
        }
        struct Restore {
            necsim_ctx *ctx;
            Engine *E;
            ~Restore() {
                if (ctx->tables_ready) {
                    ctx->engine->d_cells.swap(E->d_cells);
                    ctx->engine->d_atoms.swap(E->d_atoms);
                }
            }
        } restore{ctx, E};
        setup_engine(*E, ctx->args);
        SimHost sh;
        std::memset(&sh, 0, sizeof(sh));
        sh.sc = ctx->scenario;
        sh.seed = wyhash_seed;
        sh.params = base_params(ctx->scenario, ctx->args, wyhash_seed);
        sh.params.pause_before = pause_before >= 0.0 ? pause_before : -1.0;
        std::vector<std::vector<necsim_lineage>> given;
        if (resume) {
            sh.params.min_event_time = resume_time;
            // independent/mod.rs:98-117 sets lineages outside the habitat or the
            // deme aside as exceptional, and the resume initialiser then fails
            // (initialiser/resume.rs:79-85, ResumeError::Sample)
            std::vector<necsim_lineage> keep;
            keep.reserve(n_lineages);
            uint64_t out_of_habitat = 0, out_of_deme = 0;
            for (uint64_t j = 0; j < n_lineages; ++j) {
                const necsim_lineage &l = lineages[j];
                uint32_t h = 0;
                const necsim_scenario &sc = ctx->scenario;
                switch (sc.kind) {
                case NECSIM_NON_SPATIAL:
                    h = (l.x < sc.width && l.y < sc.height) ? sc.deme : 0;
                    break;
                case NECSIM_SPATIALLY_IMPLICIT: {
                    const uint32_t mox = 0xffffffffu - (sc.meta_width - 1), moy = 0xffffffffu - (sc.meta_height - 1);
                    if (l.x < sc.width && l.y < sc.height)
                        h = sc.deme;
                    else if (l.x >= mox && l.y >= moy)
                        h = sc.meta_deme;
                    break;
                }
                case NECSIM_ALMOST_INFINITE_NORMAL:
                case NECSIM_ALMOST_INFINITE_CLARK2DT:
                    h = 1;
                    break;
                case NECSIM_WRAPPING_NOISE:
                    h = noise::habitat_at(noise_habitat(sc), l.x, l.y);
                    break;
                default:
                    h = (l.x < sc.width && l.y < sc.height) ? ctx->habitat[(uint64_t)l.y * sc.width + l.x] : 0;
                    break;
                }
                if (h == 0)
                    out_of_habitat += 1;
                else if (l.index >= h)
                    out_of_deme += 1;
                else
                    keep.push_back(l);
            }
            if (out_of_habitat || out_of_deme)
                fail(NECSIM_E_INVALID_ARGUMENT, std::to_string(out_of_habitat) + " resumed lineage(s) out of habitat and " +
                                                    std::to_string(out_of_deme) +
                                                    " out of deme (ResumeError::Sample)");
            sh.n_origins = keep.size();
            given.push_back(std::move(keep));
        } else {
            sh.n_origins = count_origins(ctx->scenario);
        }
        std::vector<SimHost> sims{sh};
        necsim_outcome o;
        run_simulations(*E, sims, ctx->args, resume ? &given : nullptr, reporter, true, &o,
                        ctx->remaining, ctx->tables_ready ? &prebuilt : nullptr);
        *outcome = o;
    });
}

int necsim_gpu_simulate(necsim_ctx *ctx, uint64_t wyhash_seed, double pause_before,
                        const necsim_reporter *reporter, necsim_outcome *outcome) {
    return simulate_impl(ctx, nullptr, 0, false, 0.0, wyhash_seed, pause_before, reporter, outcome);
}

int necsim_gpu_simulate_lineages(necsim_ctx *ctx, const necsim_lineage *lineages, uint64_t n,
                                 double resume_time, uint64_t wyhash_seed, double pause_before,
                                 const necsim_reporter *reporter, necsim_outcome *outcome) {
    if (n && !lineages) return NECSIM_E_INVALID_ARGUMENT;
    return simulate_impl(ctx, lineages, n, true, resume_time, wyhash_seed, pause_before, reporter, outcome);
}

int necsim_gpu_remaining_lineages(necsim_ctx *ctx, necsim_lineage *out, uint64_t cap, uint64_t *n_out) {
    if (!ctx || !n_out) return NECSIM_E_INVALID_ARGUMENT;
    const std::vector<necsim_lineage> *v = ctx->remaining.per_sim.empty() ? nullptr : &ctx->remaining.per_sim[0];
    const uint64_t n = v ? v->size() : 0;
    *n_out = n;
    if (out)
        for (uint64_t j = 0; j < n && j < cap; ++j) out[j] = (*v)[j];
    return NECSIM_OK;
}

int necsim_gpu_simulate_batch(const necsim_scenario *scenarios, const uint64_t *wyhash_seeds,
                              uint32_t n_sims, const necsim_args *args_in, double pause_before,
                              const necsim_reporter *reporters, necsim_outcome *outcomes, char *error,
                              size_t error_cap) {
    if (!scenarios || !wyhash_seeds || !outcomes || n_sims == 0) return NECSIM_E_INVALID_ARGUMENT;
    return guarded(nullptr, error, error_cap, [&] {
        const necsim_args args = with_defaults(args_in);
        std::vector<SimHost> sims(n_sims);
        for (uint32_t s = 0; s < n_sims; ++s) {
            validate(scenarios[s]);
            SimHost &sh = sims[s];
            std::memset(&sh, 0, sizeof(sh));
            sh.sc = scenarios[s];
            sh.seed = wyhash_seeds[s];
            sh.params = base_params(scenarios[s], args, wyhash_seeds[s]);
            sh.params.pause_before = pause_before >= 0.0 ? pause_before : -1.0;
            sh.n_origins = count_origins(scenarios[s]);
        }
        BatchRun b;
        prepare_batch(b, std::move(sims), args);
        // the call's traffic includes the set-up's (tables, origins), which
        // run_batch does not count (a prepared batch's runs report their own)
        uint64_t setup_h2d = 0, setup_d2h = 0;
        for (const auto &e : b.engines) {
            setup_h2d += e->h2d_bytes;
            setup_d2h += e->d2h_bytes;
        }
        run_batch(b, reporters, outcomes);
        for (uint32_t s = 0; s < n_sims; ++s) {
            outcomes[s].h2d_bytes += setup_h2d;
            outcomes[s].d2h_bytes += setup_d2h;
        }
    });
}

struct necsim_batch {
    BatchRun run;
    std::string error;
};

static std::vector<SimHost> batch_sims(const necsim_scenario *scenarios, const uint64_t *wyhash_seeds,
                                       uint32_t n_sims, const necsim_args &args, double pause_before) {
    std::vector<SimHost> sims(n_sims);
    for (uint32_t s = 0; s < n_sims; ++s) {
        validate(scenarios[s]);
        SimHost &sh = sims[s];
        std::memset(&sh, 0, sizeof(sh));
        sh.sc = scenarios[s];
        sh.seed = wyhash_seeds[s];
        sh.params = base_params(scenarios[s], args, wyhash_seeds[s]);
        sh.params.pause_before = pause_before >= 0.0 ? pause_before : -1.0;
        sh.n_origins = count_origins(scenarios[s]);
    }
    return sims;
}

int necsim_gpu_displacements(int32_t device, int32_t kind, const uint64_t *draws, uint64_t n, double a, double b,
                             double *dx, double *dy) {
    if (kind != NECSIM_ALMOST_INFINITE_NORMAL && kind != NECSIM_ALMOST_INFINITE_CLARK2DT)
        return NECSIM_E_INVALID_ARGUMENT;
    if (n && (!draws || !dx || !dy)) return NECSIM_E_INVALID_ARGUMENT;
    if (kind == NECSIM_ALMOST_INFINITE_CLARK2DT && !(b > 0.0)) return NECSIM_E_INVALID_ARGUMENT;
    return guarded(nullptr, nullptr, 0, [&] {
        if (n == 0) return;
        CK(cudaSetDevice(device));
        cudaDeviceProp prop;
        CK(cudaGetDeviceProperties(&prop, device));
        struct Res {
            uint64_t *d = nullptr;
            double *x = nullptr, *y = nullptr;
            ~Res() {
                if (d) cudaFree(d);
                if (x) cudaFree(x);
                if (y) cudaFree(y);
            }
        } r;
        r.d = dev_alloc<uint64_t>(2 * n);
        r.x = dev_alloc<double>(n);
        r.y = dev_alloc<double>(n);
        CK(cudaMemcpy(r.d, draws, 2 * n * sizeof(uint64_t), cudaMemcpyHostToDevice));
        // the step kernels take the Clark2Dt exponent 1 / p computed on the host
        const double bb = kind == NECSIM_ALMOST_INFINITE_CLARK2DT ? 1.0 / b : 0.0;
        const int32_t dev_kind = kind == NECSIM_ALMOST_INFINITE_NORMAL ? (int32_t)kAlmostInfiniteNormal : -1;
        CK(launch_displacements(dev_kind, r.d, n, a, bb, r.x, r.y, (unsigned)prop.multiProcessorCount * 8, 0));
        CK(cudaMemcpy(dx, r.x, n * sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(dy, r.y, n * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

int necsim_gpu_hash_peak(int32_t device, double *wymum_per_second) {
    if (!wymum_per_second) return NECSIM_E_INVALID_ARGUMENT;
    return guarded(nullptr, nullptr, 0, [&] {
        CK(cudaSetDevice(device));
        cudaDeviceProp prop;
        CK(cudaGetDeviceProperties(&prop, device));
        struct Res {
            unsigned long long *sink = nullptr;
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            ~Res() {
                if (sink) cudaFree(sink);
                if (e0) cudaEventDestroy(e0);
                if (e1) cudaEventDestroy(e1);
            }
        } r;
        r.sink = dev_alloc<unsigned long long>(1);
        CK(cudaEventCreate(&r.e0));
        CK(cudaEventCreate(&r.e1));
        const unsigned grid = (unsigned)prop.multiProcessorCount * 8;
        const uint32_t iters = 4096;
        CK(launch_hash_peak(grid, 1, iters, r.sink, 0));  // warm-up
        float best = 0.0f;
        for (int rep = 0; rep < 3; ++rep) {
            CK(cudaEventRecord(r.e0, 0));
            CK(launch_hash_peak(grid, (uint64_t)rep + 2, iters, r.sink, 0));
            CK(cudaEventRecord(r.e1, 0));
            CK(cudaEventSynchronize(r.e1));
            float ms = 0.0f;
            CK(cudaEventElapsedTime(&ms, r.e0, r.e1));
            if (rep == 0 || ms < best) best = ms;
        }
        *wymum_per_second = (double)grid * 256.0 * 8.0 * (double)iters / ((double)best * 1e-3);
    });
}

int necsim_gpu_autotune(const necsim_scenario *scenarios, const uint64_t *wyhash_seeds, uint32_t n_sims,
                        const necsim_args *args_in, double sample_pause, uint64_t max_sample_lineages,
                        necsim_args *best, necsim_autotune_result *results, uint32_t results_cap,
                        uint32_t *n_results, char *error, size_t error_cap) {
    if (!scenarios || !wyhash_seeds || n_sims == 0 || !best || !(sample_pause > 0.0))
        return NECSIM_E_INVALID_ARGUMENT;
    return guarded(nullptr, error, error_cap, [&] {
        const necsim_args base = with_defaults(args_in);
        if (base.report_dispersal || base.schedule)
            fail(NECSIM_E_INVALID_ARGUMENT, "tune the plain schedule without dispersal reporting");
        // the sample: every k-th simulation, at most max_sample_lineages origins
        uint64_t total = 0;
        for (uint32_t s = 0; s < n_sims; ++s) {
            validate(scenarios[s]);
            total += count_origins(scenarios[s]);
        }
        const uint64_t cap = max_sample_lineages ? max_sample_lineages : (1ULL << 22);
        uint32_t stride = 1;
        while (stride < n_sims && total / stride > cap) ++stride;
        std::vector<necsim_scenario> sc;
        std::vector<uint64_t> seeds;
        for (uint32_t s = 0; s < n_sims; s += stride) {
            sc.push_back(scenarios[s]);
            seeds.push_back(wyhash_seeds[s]);
        }
        const uint32_t blocks[] = {64, 128, 256};
        const uint64_t slices[] = {base.step_slice, 2 * base.step_slice, 4 * base.step_slice};
        const uint32_t dedups[] = {200, 400};
        double best_ms = 0.0;
        uint32_t count = 0;
        for (uint32_t b : blocks)
            for (uint64_t sl : slices)
                for (uint32_t dd : dedups) {
                    necsim_args a = base;
                    a.block_size = b;
                    a.step_slice = sl;
                    a.dedup_factor_pct = dd;
                    a = with_defaults(&a);
                    Engine E;
                    setup_engine(E, a);
                    prepare_engine(E, batch_sims(sc.data(), seeds.data(), (uint32_t)sc.size(), a, sample_pause), a,
                                   nullptr, nullptr);
                    std::vector<necsim_outcome> outs(sc.size());
                    Remaining rem;
                    double ms = 0.0;
                    uint64_t steps = 0;
                    for (int rep = 0; rep < 3; ++rep) {
                        execute_engine(E, nullptr, false, outs.data(), rem);
                        if (rep == 0) continue;  // warm-up
                        if (rep == 1 || outs[0].total_ms < ms) ms = outs[0].total_ms;
                        steps = 0;
                        for (const auto &o : outs) steps += o.steps;
                    }
                    if (results && count < results_cap) {
                        results[count].block_size = b;
                        results[count].dedup_factor_pct = dd;
                        results[count].step_slice = sl;
                        results[count].ms = ms;
                        results[count].steps = steps;
                    }
                    ++count;
                    if (count == 1 || ms < best_ms) {
                        best_ms = ms;
                        *best = a;
                    }
                }
        if (n_results) *n_results = count;
    });
}

int necsim_gpu_batch_create(const necsim_scenario *scenarios, const uint64_t *wyhash_seeds, uint32_t n_sims,
                            const necsim_args *args_in, double pause_before, necsim_batch **out) {
    if (!scenarios || !wyhash_seeds || !out || n_sims == 0) return NECSIM_E_INVALID_ARGUMENT;
    *out = nullptr;
    necsim_batch *b = new (std::nothrow) necsim_batch();
    if (!b) return NECSIM_E_OUT_OF_MEMORY;
    char msg[512] = {0};
    const int rc = guarded(nullptr, msg, sizeof(msg), [&] {
        const necsim_args args = with_defaults(args_in);
        prepare_batch(b->run, batch_sims(scenarios, wyhash_seeds, n_sims, args, pause_before), args);
    });
    b->error = msg;
    *out = b;
    return rc;
}

int necsim_gpu_batch_run(necsim_batch *b, const necsim_reporter *reporters, necsim_outcome *outcomes) {
    if (!b || !outcomes) return NECSIM_E_INVALID_ARGUMENT;
    char msg[512] = {0};
    const int rc = guarded(nullptr, msg, sizeof(msg), [&] { run_batch(b->run, reporters, outcomes); });
    b->error = msg;
    return rc;
}

int necsim_gpu_batch_priority(const necsim_batch *b, uint32_t *ids, uint32_t cap, uint32_t *n) {
    if (!b || !n || (cap && !ids)) return NECSIM_E_INVALID_ARGUMENT;
    uint32_t k = 0;
    for (uint32_t j : b->run.priority) {
        if (k < cap) ids[k] = j;
        ++k;
    }
    *n = k;
    return NECSIM_OK;
}

const char *necsim_gpu_batch_last_error(const necsim_batch *b) { return b ? b->error.c_str() : "null batch"; }

void necsim_gpu_batch_destroy(necsim_batch *b) { delete b; }

int necsim_build_tables(const necsim_scenario *scenario, necsim_cell_record *cells, necsim_alias_atom *atoms,
                        uint64_t atom_cap, uint64_t *n_atoms) {
    if (!scenario || !n_atoms || scenario->kind != NECSIM_SPATIALLY_EXPLICIT) return NECSIM_E_INVALID_ARGUMENT;
    return guarded(nullptr, nullptr, 0, [&] {
        validate(*scenario);
        HostTables t;
        const int rc = build_spatially_explicit_tables(*scenario, t);
        if (rc == 1) fail(NECSIM_E_EMPTY_HABITAT, "habitat map has no habitable cell");
        if (rc == 2) fail(NECSIM_E_DISPERSAL_MAP, "dispersal map violates the in-memory dispersal contract");
        if (rc == 3) fail(NECSIM_E_TOO_LARGE, "more than 2^32 alias atoms");
        *n_atoms = t.atoms.size();
        static_assert(sizeof(necsim_cell_record) == sizeof(CellRecord), "cell record layout");
        static_assert(sizeof(necsim_alias_atom) == sizeof(AliasAtom), "alias atom layout");
        if (cells) std::memcpy(cells, t.cells.data(), t.cells.size() * sizeof(CellRecord));
        if (atoms) std::memcpy(atoms, t.atoms.data(), std::min<uint64_t>(atom_cap, t.atoms.size()) * sizeof(AliasAtom));
    });
}

int necsim_subdomain_ranks(const necsim_scenario *scenario, uint32_t size, const necsim_lineage *lineages,
                           uint64_t n, uint32_t *ranks, int32_t *exact) {
    if (!scenario || size == 0 || (n && (!lineages || !ranks))) return NECSIM_E_INVALID_ARGUMENT;
    return guarded(nullptr, nullptr, 0, [&] {
        validate(*scenario);
        const SubdomainMap d = make_subdomain_map(*scenario, size);
        for (uint64_t j = 0; j < n; ++j) ranks[j] = d.rank(lineages[j].x, lineages[j].y);
        if (exact) *exact = d.exact ? 1 : 0;
    });
}

int necsim_enumerate_origins(const necsim_scenario *scenario, necsim_lineage *out, uint64_t cap,
                             uint64_t *n_out) {
    if (!scenario || !n_out) return NECSIM_E_INVALID_ARGUMENT;
    return guarded(nullptr, nullptr, 0, [&] {
        validate(*scenario);
        uint64_t n = 0;
        for_each_origin(*scenario, [&](uint32_t x, uint32_t y, uint32_t i, uint64_t g) {
            if (out && n < cap) {
                out[n].global_reference = g;
                out[n].last_event_time = 0.0;
                out[n].x = x;
                out[n].y = y;
                out[n].index = i;
                out[n].pad = 0;
            }
            ++n;
        });
        *n_out = n;
    });
}

const char *necsim_gpu_last_error(const necsim_ctx *ctx) { return ctx ? ctx->error.c_str() : "null context"; }

void necsim_gpu_destroy(necsim_ctx *ctx) { delete ctx; }

int necsim_presample_origins(uint64_t n, double percentage, uint32_t rank, uint32_t size, uint64_t *out,
                             uint64_t cap, uint64_t *n_out) {
    if (!n_out || !(percentage >= 0.0 && percentage <= 1.0) || size == 0 || rank >= size)
        return NECSIM_E_INVALID_ARGUMENT;
    // pre_sampler.rs:12
    const double kInvPhiF = 6.180339887498949e-1;
    uint64_t count = 0, seen = 0;
    auto take = [&](uint64_t pos) {
        // partition: advance_by(rank), then step_by(size)
        if (seen >= rank && (seen - rank) % size == 0) {
            if (out && count < cap) out[count] = pos;
            ++count;
        }
        ++seen;
    };
    if (percentage >= 1.0) {
        for (uint64_t pos = 0; pos < n; ++pos) take(pos);
    } else if (percentage > 0.0) {
        // pre_sampler.rs:73-101: skip floor(ln(q) / ln(1 - p)) origins, q the
        // fractional part of 0.5 + k * INV_PHI
        const double inv_rate = 1.0 / std::log(1.0 - percentage);
        double q = 0.5;
        uint64_t pos = 0;
        while (pos < n) {
            q = q + kInvPhiF;
            q = q - std::floor(q);
            const double skip = std::floor(std::log(q) * inv_rate);
            if (!(skip < (double)(n - pos))) break;  // Iterator::nth past the last origin
            pos += (uint64_t)skip;
            take(pos);
            pos += 1;
        }
    }
    *n_out = count;
    return NECSIM_OK;
}

}  // extern "C"

// ---- learned lifetime model ----

namespace {

template <typename F>
int model_guarded(necsim_model *m, F &&f) {
    if (!m) return NECSIM_E_INVALID_ARGUMENT;
    char msg[512] = {0};
    const int rc = guarded(nullptr, msg, sizeof(msg), [&] {
        CK(cudaSetDevice(m->device));
        f();
    });
    m->error = msg;
    return rc;
}

// device copy of a host array, freed by the caller
template <typename T>
T *upload(const T *src, size_t n, cudaStream_t st) {
    T *d = dev_alloc<T>(n ? n : 1);
    if (n) CK(cudaMemcpyAsync(d, src, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return d;
}

struct DevFree {
    std::vector<void *> ptrs;
    ~DevFree() {
        for (void *p : ptrs)
            if (p) cudaFree(p);
    }
};

void model_write_master(necsim_model *m, const std::vector<float> &w) {
    std::vector<__nv_bfloat16> wb(kMlpParams);
    for (int i = 0; i < kMlpParams; ++i) wb[i] = __float2bfloat16_rn(w[i]);
    CK(cudaMemcpyAsync(m->master, w.data(), kMlpParams * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    CK(cudaMemcpyAsync(m->w, wb.data(), kMlpParams * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice, m->stream));
    CK(cudaMemsetAsync(m->m, 0, kMlpParams * sizeof(float), m->stream));
    CK(cudaMemsetAsync(m->v, 0, kMlpParams * sizeof(float), m->stream));
    CK(cudaMemsetAsync(m->grads, 0, kMlpParams * sizeof(float), m->stream));
    CK(cudaStreamSynchronize(m->stream));
    m->adam_step = 0;
}

}  // namespace

extern "C" {

int necsim_model_create(int32_t device, uint64_t seed, necsim_model **out) {
    if (!out) return NECSIM_E_INVALID_ARGUMENT;
    *out = nullptr;
    necsim_model *m = new (std::nothrow) necsim_model();
    if (!m) return NECSIM_E_OUT_OF_MEMORY;
    m->device = device;
    const int rc = model_guarded(m, [&] {
        CK(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
        m->w = dev_alloc<__nv_bfloat16>(kMlpParams);
        m->master = dev_alloc<float>(kMlpParams);
        m->m = dev_alloc<float>(kMlpParams);
        m->v = dev_alloc<float>(kMlpParams);
        m->grads = dev_alloc<float>(kMlpParams);
        m->loss = dev_alloc<double>(1);
        // He initialisation for the ReLU layers, a linear output layer
        // starting near log(1 + 100) events
        std::mt19937_64 rng(seed);
        std::normal_distribution<float> g1(0.f, std::sqrt(2.f / kFeat)), g2(0.f, std::sqrt(2.f / kHidden)),
            g3(0.f, std::sqrt(1.f / kHidden));
        std::vector<float> w(kMlpParams, 0.f);
        for (int i = kW1; i < kB1; ++i) w[i] = g1(rng);
        for (int i = kW2; i < kB2; ++i) w[i] = g2(rng);
        for (int i = kW3; i < kB3; ++i) w[i] = g3(rng);
        w[kB3] = 4.6f;
        model_write_master(m, w);
    });
    *out = m;
    return rc;
}

void necsim_model_destroy(necsim_model *model) { delete model; }

const char *necsim_model_last_error(const necsim_model *model) {
    return model ? model->error.c_str() : "null model";
}

int necsim_model_get_weights(necsim_model *model, float *out) {
    if (!out) return NECSIM_E_INVALID_ARGUMENT;
    return model_guarded(model, [&] {
        std::vector<__nv_bfloat16> wb(kMlpParams);
        CK(cudaMemcpyAsync(wb.data(), model->w, kMlpParams * sizeof(__nv_bfloat16), cudaMemcpyDeviceToHost,
                           model->stream));
        CK(cudaStreamSynchronize(model->stream));
        for (int i = 0; i < kMlpParams; ++i) out[i] = __bfloat162float(wb[i]);
    });
}

int necsim_model_set_weights(necsim_model *model, const float *weights) {
    if (!weights) return NECSIM_E_INVALID_ARGUMENT;
    return model_guarded(model, [&] {
        model_write_master(model, std::vector<float>(weights, weights + kMlpParams));
    });
}

int necsim_model_predict(necsim_model *model, const float *X, uint64_t n, float *y) {
    if ((!X || !y) && n) return NECSIM_E_INVALID_ARGUMENT;
    return model_guarded(model, [&] {
        if (n == 0) return;
        DevFree f;
        float *dX = upload(X, n * kFeat, model->stream);
        f.ptrs.push_back(dX);
        float *dy = dev_alloc<float>(n);
        f.ptrs.push_back(dy);
        CK(launch_mlp_predict(model->w, dX, n, dy, model->stream));
        CK(cudaMemcpyAsync(y, dy, n * sizeof(float), cudaMemcpyDeviceToHost, model->stream));
        CK(cudaStreamSynchronize(model->stream));
    });
}

int necsim_model_gradients(necsim_model *model, const float *X, const float *T, uint64_t n, float *grads,
                           double *loss) {
    if (!X || !T || !grads || n == 0) return NECSIM_E_INVALID_ARGUMENT;
    return model_guarded(model, [&] {
        DevFree f;
        float *dX = upload(X, n * kFeat, model->stream);
        f.ptrs.push_back(dX);
        float *dT = upload(T, n, model->stream);
        f.ptrs.push_back(dT);
        CK(cudaMemsetAsync(model->grads, 0, kMlpParams * sizeof(float), model->stream));
        CK(cudaMemsetAsync(model->loss, 0, sizeof(double), model->stream));
        CK(launch_mlp_grad(model->w, dX, dT, nullptr, 0, n, 1.0f / (float)n, model->grads, model->loss,
                           model->stream));
        CK(cudaMemcpyAsync(grads, model->grads, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, model->stream));
        double l = 0.0;
        CK(cudaMemcpyAsync(&l, model->loss, sizeof(double), cudaMemcpyDeviceToHost, model->stream));
        CK(cudaMemsetAsync(model->grads, 0, kMlpParams * sizeof(float), model->stream));
        CK(cudaStreamSynchronize(model->stream));
        if (loss) *loss = l;
    });
}

int necsim_model_train(necsim_model *model, const float *X, const float *T, uint64_t n, uint32_t epochs,
                       uint32_t batch, float lr, uint64_t seed, double *epoch_loss) {
    if (!X || !T || n == 0 || batch == 0 || !(lr > 0.f)) return NECSIM_E_INVALID_ARGUMENT;
    if (n >= 0xffffffffULL) return NECSIM_E_TOO_LARGE;
    return model_guarded(model, [&] {
        DevFree f;
        float *dX = upload(X, n * kFeat, model->stream);
        f.ptrs.push_back(dX);
        float *dT = upload(T, n, model->stream);
        f.ptrs.push_back(dT);
        uint32_t *dperm = dev_alloc<uint32_t>(n);
        f.ptrs.push_back(dperm);
        std::vector<uint32_t> perm(n);
        std::mt19937_64 rng(seed);
        const uint64_t n_batches = (n + batch - 1) / batch;
        for (uint32_t e = 0; e < epochs; ++e) {
            for (uint64_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
            std::shuffle(perm.begin(), perm.end(), rng);
            CK(cudaMemcpyAsync(dperm, perm.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, model->stream));
            CK(cudaMemsetAsync(model->loss, 0, sizeof(double), model->stream));
            for (uint64_t b = 0; b < n_batches; ++b) {
                const uint64_t off = b * batch;
                const uint64_t bn = std::min<uint64_t>(batch, n - off);
                CK(launch_mlp_grad(model->w, dX, dT, dperm, off, bn, 1.0f / (float)bn, model->grads, model->loss,
                                   model->stream));
                model->adam_step += 1;
                CK(launch_adam(model->master, model->m, model->v, model->grads, model->w, lr, 0.9f, 0.999f, 1e-8f,
                               model->adam_step, model->stream));
            }
            double l = 0.0;
            CK(cudaMemcpyAsync(&l, model->loss, sizeof(double), cudaMemcpyDeviceToHost, model->stream));
            CK(cudaStreamSynchronize(model->stream));
            if (epoch_loss) epoch_loss[e] = l / (double)n_batches;
        }
    });
}

int necsim_gpu_trace_batch(const necsim_scenario *scenarios, const uint64_t *wyhash_seeds, uint32_t n_sims,
                           const necsim_args *args_in, double pause_before, uint32_t snapshot_rounds,
                           uint64_t max_rows, float *features, float *labels, uint64_t *n_rows, char *error,
                           size_t error_cap) {
    if (!scenarios || !wyhash_seeds || n_sims == 0 || !n_rows || (max_rows && (!features || !labels)))
        return NECSIM_E_INVALID_ARGUMENT;
    if (snapshot_rounds < 2 || snapshot_rounds % 2) return NECSIM_E_INVALID_ARGUMENT;
    return guarded(nullptr, error, error_cap, [&] {
        necsim_args args = with_defaults(args_in);
        args.resident = 0;  // every lineage stays in the global rounds, where it is snapshotted
        args.schedule = 0;
        args.model = nullptr;
        args.rounds_per_graph = snapshot_rounds;
        Engine E;
        setup_engine(E, args);
        E.tracing = true;
        E.trace_rows_cap = std::max<uint64_t>(1024, std::min<uint64_t>(max_rows * 4, 1ULL << 25));
        prepare_engine(E, batch_sims(scenarios, wyhash_seeds, n_sims, args, pause_before), args, nullptr, nullptr);
        if (E.n_total > 0) run_rounds(E);
        unsigned long long counts[2] = {0, 0};
        CK(cudaMemcpy(counts, E.trace_counts, sizeof(counts), cudaMemcpyDeviceToHost));
        const uint64_t nr = std::min<uint64_t>(counts[0], E.trace_rows_cap);
        std::vector<TraceRow> rows(nr);
        if (nr) CK(cudaMemcpy(rows.data(), E.trace_rows, nr * sizeof(TraceRow), cudaMemcpyDeviceToHost));
        // The label of a snapshotted lineage is the remaining life of its
        // simulation: the simulation ends with its longest-lived lineage, at
        // its largest event time t_end, so the label is log(1 + lambda
        // (t_end - t)), the expected events of one lineage over the rest of
        // the run from the lineage's time t.  (A paused run ends at its last
        // event before the pause: its labels are censored there.)
        std::vector<SimCounters> cs(E.sims.size());
        CK(cudaMemcpy(cs.data(), E.d_counters, cs.size() * sizeof(SimCounters), cudaMemcpyDeviceToHost));
        const uint64_t take = std::min<uint64_t>(max_rows, nr);
        for (uint64_t k = 0; k < take; ++k) {
            // evenly spaced over the rows (all snapshots, all sims)
            const TraceRow &r = rows[(uint64_t)((double)k * (double)nr / (double)take)];
            for (int j = 0; j < kFeat; ++j) features[k * kFeat + j] = r.f[j];
            double t_end;
            const unsigned long long bits = cs[r.sim].max_time_bits;
            std::memcpy(&t_end, &bits, sizeof(double));
            const double rest = std::max(0.0, t_end - r.time) * E.sims[r.sim].params.lambda;
            labels[k] = (float)std::log1p(rest);
        }
        *n_rows = take;
    });
}

}  // extern "C"

// Per-simulation parameters for callers outside this file (the
// allocation-free round in noalloc.cu): the same values base_params gives
// the engine, with the defaults of with_defaults.
namespace necsim {
SimParams host_sim_params(const necsim_scenario &sc, const necsim_args *args, uint64_t wyhash_seed) {
    const necsim_args a = with_defaults(args);
    return base_params(sc, a, wyhash_seed);
}
}  // namespace necsim
