// noalloc.cu -- one synchronised round (advance to a horizon, then remove
// duplicate lineages) that performs no device memory allocation.
//
// Why it exists: some callers cannot call cudaMalloc.  A host that owns the
// device memory itself (a framework with its own caching allocator, an
// embedded plugin that is handed a fixed arena), code that must not trigger
// the implicit device synchronisation cudaMalloc/cudaFree can cause, or a
// long-running service that forbids allocation after start-up all need an
// entry point whose working memory already exists.  This one keeps its
// working memory (lineage state, dedup table, counters) in one file-scope
// device array, sized for at most NECSIM_NOALLOC_MAX_LINEAGES lineages; the
// caller passes device buffers for the input lineages and for the outputs.
//
// Every GPU that loads this library holds the array (about 9.5 MB) until the
// process exits.  All calls share it: the call clears what must start empty
// (dedup table, counters) and two calls whose work overlaps on the GPU (on
// different streams, or from different host threads) race on it.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstring>

#include "../../include/necsim_b200.h"
#include "kernels.h"
#include "layout.h"

namespace necsim {
SimParams host_sim_params(const necsim_scenario &sc, const necsim_args *args, uint64_t wyhash_seed);
}

using namespace necsim;

namespace {

constexpr uint64_t kMax = NECSIM_NOALLOC_MAX_LINEAGES;
constexpr uint64_t kTableSlots = 2 * kMax;  // power of two >= 2n for every allowed n

// byte offsets of the carved arrays (each 256-byte aligned)
constexpr uint64_t align256(uint64_t v) { return (v + 255) & ~255ULL; }
constexpr uint64_t kOffParams = 0;
constexpr uint64_t kOffCounters = align256(kOffParams + sizeof(SimParams));
constexpr uint64_t kOffControl = align256(kOffCounters + sizeof(SimCounters));
constexpr uint64_t kControlWords = 16;  // u64 scalars: n_cur, out_count, work, mask, n_spec, n_disp, steps, visits, status
constexpr uint64_t kOffSoA = align256(kOffControl + kControlWords * 8);
// one lineage buffer: x, y, idx, sim (u32), last, next (f64), reprime, gref, steps (u64), has_next, state (u8)
constexpr uint64_t kSoABytes = kMax * (4 * 4 + 8 * 5 + 2);
constexpr uint64_t kOffA = kOffSoA;
constexpr uint64_t kOffB = align256(kOffA + align256(kSoABytes) + 16 * 256);
constexpr uint64_t kOffOwner = align256(kOffB + align256(kSoABytes) + 16 * 256);
constexpr uint64_t kOffMinGref = align256(kOffOwner + kTableSlots * 4);
constexpr uint64_t kOffSlot = align256(kOffMinGref + kTableSlots * 8);
constexpr uint64_t kScratchBytes = align256(kOffSlot + kMax * 4);

// The working memory of every call of necsim_gpu_round_noalloc.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

static_assert(kScratchBytes < 10u * 1024 * 1024, "the scratch array is documented as about 9.5 MB");

// Per device, looked up on its first call: the device address of
// g_noalloc_scratch (cudaGetSymbolAddress; host code must not use the
// symbol itself) and the SM count the launch grids are sized by.
constexpr int kMaxDevices = 64;
std::atomic<unsigned char *> g_scratch_ptr[kMaxDevices];
std::atomic<int> g_sm_count[kMaxDevices];

struct Carved {
    SimParams *params;
    SimCounters *counters;
    unsigned long long *ctl;
    LineageSoA a, b;
    uint8_t *state_a, *state_b;
    uint32_t *owner;
    unsigned long long *min_gref;
    uint32_t *slot;
};

void carve_soa(unsigned char *base, LineageSoA &s, uint8_t *&state) {
    uint64_t o = 0;
    auto take = [&](uint64_t bytes) {
        unsigned char *p = base + o;
        o = align256(o + bytes);
        return p;
    };
    s.x = reinterpret_cast<uint32_t *>(take(kMax * 4));
    s.y = reinterpret_cast<uint32_t *>(take(kMax * 4));
    s.idx = reinterpret_cast<uint32_t *>(take(kMax * 4));
    s.sim = reinterpret_cast<uint32_t *>(take(kMax * 4));
    s.last = reinterpret_cast<double *>(take(kMax * 8));
    s.next = reinterpret_cast<double *>(take(kMax * 8));
    s.reprime = reinterpret_cast<uint64_t *>(take(kMax * 8));
    s.gref = reinterpret_cast<uint64_t *>(take(kMax * 8));
    s.steps = reinterpret_cast<uint64_t *>(take(kMax * 8));
    s.has_next = reinterpret_cast<uint8_t *>(take(kMax));
    state = reinterpret_cast<uint8_t *>(take(kMax));
}

Carved carve(unsigned char *base) {
    Carved c;
    c.params = reinterpret_cast<SimParams *>(base + kOffParams);
    c.counters = reinterpret_cast<SimCounters *>(base + kOffCounters);
    c.ctl = reinterpret_cast<unsigned long long *>(base + kOffControl);
    carve_soa(base + kOffA, c.a, c.state_a);
    carve_soa(base + kOffB, c.b, c.state_b);
    c.owner = reinterpret_cast<uint32_t *>(base + kOffOwner);
    c.min_gref = reinterpret_cast<unsigned long long *>(base + kOffMinGref);
    c.slot = reinterpret_cast<uint32_t *>(base + kOffSlot);
    return c;
}

enum : int { kCtlNCur = 0, kCtlOut = 1, kCtlWork = 2, kCtlMask = 3, kCtlSpec = 4, kCtlDisp = 5,
             kCtlSteps = 6, kCtlStatus = 8 };

// array-of-structs input lineages -> the round's structure of arrays
__global__ void load_lineages_kernel(const necsim_lineage *in, uint64_t n, LineageSoA s, uint8_t *state) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (uint64_t)gridDim.x * blockDim.x) {
        const necsim_lineage l = in[j];
        s.x[j] = l.x;
        s.y[j] = l.y;
        s.idx[j] = l.index;
        s.sim[j] = 0;
        s.last[j] = l.last_event_time;
        s.next[j] = 0.0;
        s.reprime[j] = 0;
        s.gref[j] = l.global_reference;
        s.steps[j] = 0;
        s.has_next[j] = 0;
        state[j] = 0;
    }
}

// surviving lineages -> the caller's array of structs; their steps summed
__global__ void store_lineages_kernel(LineageSoA s, const unsigned long long *n_out, necsim_lineage *out,
                                      unsigned long long *steps) {
    const uint64_t n = *n_out;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (uint64_t)gridDim.x * blockDim.x) {
        necsim_lineage l;
        l.global_reference = s.gref[j];
        l.last_event_time = s.last[j];
        l.x = s.x[j];
        l.y = s.y[j];
        l.index = s.idx[j];
        l.pad = 0;
        out[j] = l;
        atomicAdd(steps, (unsigned long long)s.steps[j]);
    }
}

bool kind_supported(int32_t kind) {
    return kind == NECSIM_NON_SPATIAL || kind == NECSIM_SPATIALLY_IMPLICIT ||
           kind == NECSIM_ALMOST_INFINITE_NORMAL;
}

bool scenario_valid(const necsim_scenario &sc) {
    if (!(sc.speciation_probability > 0.0) || !(sc.speciation_probability <= 1.0)) return false;
    if (!(sc.turnover_rate > 0.0)) return false;
    if (sc.kind == NECSIM_NON_SPATIAL) return sc.width && sc.height && sc.deme;
    if (sc.kind == NECSIM_SPATIALLY_IMPLICIT)
        return sc.width && sc.height && sc.deme && sc.meta_width && sc.meta_height && sc.meta_deme &&
               sc.migration_probability > 0.0 && sc.migration_probability <= 1.0;
    return sc.sigma >= 0.0;
}

}  // namespace

extern "C" int necsim_gpu_round_noalloc(const necsim_scenario *scenario, const necsim_args *args,
                                        uint64_t wyhash_seed, const necsim_lineage *d_lineages, uint64_t n,
                                        double resume_time, double horizon, necsim_lineage *d_out,
                                        uint64_t *n_out, necsim_speciation_event *d_events,
                                        uint64_t events_cap, uint64_t *n_events, uint64_t *steps,
                                        void *stream) {
    if (!scenario || !n_out || !n_events || !steps || (n && (!d_lineages || !d_out))) return NECSIM_E_INVALID_ARGUMENT;
    if (!kind_supported(scenario->kind)) return NECSIM_E_UNSUPPORTED;
    if (!scenario_valid(*scenario) || !(horizon >= 0.0) || !(resume_time >= 0.0)) return NECSIM_E_INVALID_ARGUMENT;
    if (n > kMax) return NECSIM_E_TOO_LARGE;
    if (events_cap && !d_events) return NECSIM_E_INVALID_ARGUMENT;
    *n_out = 0;
    *n_events = 0;
    *steps = 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    const uint32_t sampler = args ? args->event_time_sampler : NECSIM_SAMPLER_POISSON;
    if (sampler != NECSIM_SAMPLER_POISSON && sampler != NECSIM_SAMPLER_EXP) return NECSIM_E_INVALID_ARGUMENT;
    const bool exp_sampler = sampler == NECSIM_SAMPLER_EXP;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return NECSIM_E_CUDA;
    if (!g_scratch_ptr[dev].load()) {
        // first call on this device: the device address of the scratch array
        // and the device's SM count
        void *p = nullptr;
        int sms = 0;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return NECSIM_E_CUDA;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
            return NECSIM_E_CUDA;
        g_sm_count[dev].store(sms);
        g_scratch_ptr[dev].store(static_cast<unsigned char *>(p));
    }
    if (n == 0) return NECSIM_OK;
    const Carved c = carve(g_scratch_ptr[dev].load());
    const unsigned sms = (unsigned)g_sm_count[dev].load();

    SimParams p = host_sim_params(*scenario, args, wyhash_seed);
    if (!(p.p0 > 0.0)) return NECSIM_E_UNSUPPORTED;
    p.min_event_time = resume_time;
    p.horizon = horizon;
    p.active = 1;
    p.pause_before = -1.0;
    unsigned long long mask = 1;
    while (mask < 2 * n) mask <<= 1;
    unsigned long long ctl[kControlWords];
    std::memset(ctl, 0, sizeof(ctl));
    ctl[kCtlNCur] = n;
    ctl[kCtlMask] = mask - 1;
    SimCounters counters;
    std::memset(&counters, 0, sizeof(counters));

    // launch shapes from the kernels' occupancy on this device's SMs (host
    // queries, no allocation)
    constexpr unsigned kBlock = 128;
    int step_per_sm = 0, coop_per_sm = 0;
    if (step_kernel_occupancy(scenario->kind, exp_sampler, (int)kBlock, &step_per_sm) != cudaSuccess)
        return NECSIM_E_CUDA;
    if (!exp_sampler && coop_kernel_occupancy(scenario->kind, &coop_per_sm) != cudaSuccess) return NECSIM_E_CUDA;
    const unsigned step_grid = sms * (unsigned)(step_per_sm > 0 ? step_per_sm : 1);
    const unsigned coop_grid = sms * (unsigned)(coop_per_sm > 0 ? coop_per_sm : 1);

    // the array keeps the previous call's contents: reset what must start
    // empty (dedup table, counters, control words) on the caller's stream
    if (cudaMemcpyAsync(c.params, &p, sizeof(p), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(c.counters, &counters, sizeof(counters), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(c.ctl, ctl, sizeof(ctl), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(c.owner, 0xff, mask * sizeof(uint32_t), st) != cudaSuccess ||
        cudaMemsetAsync(c.min_gref, 0xff, mask * sizeof(unsigned long long), st) != cudaSuccess)
        return NECSIM_E_CUDA;

    load_lineages_kernel<<<sms * 2, 256, 0, st>>>(d_lineages, n, c.a, c.state_a);

    StepArgs sa;
    std::memset(&sa, 0, sizeof(sa));
    sa.in = c.a;
    sa.state = c.state_a;
    sa.n_cur = &c.ctl[kCtlNCur];
    sa.work = &c.ctl[kCtlWork];
    sa.params = c.params;
    sa.counters = c.counters;
    sa.spec = reinterpret_cast<DevSpeciationEvent *>(d_events);
    sa.n_spec_total = &c.ctl[kCtlSpec];
    sa.spec_cap = events_cap;
    sa.n_disp_total = &c.ctl[kCtlDisp];
    sa.status = reinterpret_cast<uint32_t *>(&c.ctl[kCtlStatus]);
    sa.steps_total = &c.ctl[kCtlSteps];
    sa.n_sims = 1;
    sa.exp_sampler = exp_sampler ? 1u : 0u;
    sa.coop_max = exp_sampler ? 0 : (uint64_t)coop_grid * (kCoopBlock / 32);
    if (launch_step(scenario->kind, sa, step_grid, kBlock, coop_grid, st) != cudaSuccess) return NECSIM_E_CUDA;

    DedupArgs da;
    std::memset(&da, 0, sizeof(da));
    da.in = c.a;
    da.out = c.b;
    da.state = c.state_a;
    da.state_out = c.state_b;
    da.n_cur = &c.ctl[kCtlNCur];
    da.mask = &c.ctl[kCtlMask];
    da.owner = c.owner;
    da.min_gref = c.min_gref;
    da.slot = c.slot;
    da.out_count = &c.ctl[kCtlOut];
    da.counters = c.counters;
    da.status = reinterpret_cast<uint32_t *>(&c.ctl[kCtlStatus]);
    if (launch_dedup(da, sms * 2, 256, st) != cudaSuccess) return NECSIM_E_CUDA;

    store_lineages_kernel<<<sms * 2, 256, 0, st>>>(c.b, &c.ctl[kCtlOut], d_out, &c.counters->steps);
    if (cudaGetLastError() != cudaSuccess) return NECSIM_E_CUDA;

    unsigned long long back[kControlWords];
    SimCounters cnt;
    if (cudaMemcpyAsync(back, c.ctl, sizeof(back), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&cnt, c.counters, sizeof(cnt), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return NECSIM_E_CUDA;
    const uint32_t status = (uint32_t)back[kCtlStatus];
    *n_out = back[kCtlOut];
    *n_events = back[kCtlSpec] < events_cap ? back[kCtlSpec] : events_cap;
    *steps = cnt.steps;
    if (status & kErrEventOverflow) return NECSIM_E_TOO_LARGE;
    if (status & ~kErrDedupFull) return NECSIM_E_DEVICE_CHECK;
    return NECSIM_OK;
}
