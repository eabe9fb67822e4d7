// learned.cu -- kernels of the learned lifetime scheduler (see learned.h):
// lineage features, MLP inference, MLP training (forward + backward + Adam)
// and the bucket sort of the step kernel's queue.
//
// Weights are stored as bf16 and widened to fp32 in shared memory; every
// dot product accumulates in fp32 (fmaf).  Nothing here feeds back into a
// lineage's trajectory: predictions only decide which lineage a lane takes
// next.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>

#include <cstdint>

#include "device_core.cuh"
#include "learned.h"

namespace necsim {

namespace {

constexpr unsigned kFullMask = 0xffffffffu;

// The features of a lineage (lineage_features_of, learned.h), reading the
// SpatiallyExplicit cell's habitat and dispersal entropy from the tables.
__device__ void lineage_features(int kind, const SimParams &p, const SimCounters &c, uint32_t x, uint32_t y,
                                 double last, uint64_t steps, float f[kFeat]) {
    float hab = 1.f, ent = 0.f;
    if (kind == kSpatiallyExplicit) {
        const uint64_t cell = (uint64_t)y * p.width + x;
        if (cell < p.n_cells) {
            hab = (float)p.cells[cell].habitat;
            ent = p.cell_entropy ? p.cell_entropy[cell] : 0.f;
        }
    }
    lineage_features_of(kind, p, c.n_live, x, y, last, steps, hab, ent, f);
}

__device__ __forceinline__ void stage_weights(const __nv_bfloat16 *w, float *Ws) {
    for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) Ws[i] = __bfloat162float(w[i]);
}

// MLP(f) from fp32 weights in shared memory, fp32 accumulation.  Every
// lane reads the same weight at the same time (broadcast); the 64 hidden
// values of layer 1 are the only array held in registers.
__device__ __forceinline__ float mlp_eval(const float *W, const float f[kFeat]) {
    // keep the weight loads inside the caller's loop over rows (hoisting
    // 576 loop-invariant shared loads out of it only spills registers)
    asm volatile("" ::: "memory");
    float h1[kHidden];
#pragma unroll
    for (int j = 0; j < kHidden; ++j) {
        const float4 *w1 = reinterpret_cast<const float4 *>(W + kW1 + j * kFeat);
        const float4 a = w1[0], b = w1[1];
        float z = W[kB1 + j];
        z = fmaf(a.x, f[0], z);
        z = fmaf(a.y, f[1], z);
        z = fmaf(a.z, f[2], z);
        z = fmaf(a.w, f[3], z);
        z = fmaf(b.x, f[4], z);
        z = fmaf(b.y, f[5], z);
        z = fmaf(b.z, f[6], z);
        z = fmaf(b.w, f[7], z);
        h1[j] = fmaxf(z, 0.f);
    }
    float y = W[kB3];
#pragma unroll 1
    for (int j = 0; j < kHidden; ++j) {
        float z = W[kB2 + j];
        const float4 *row = reinterpret_cast<const float4 *>(W + kW2 + j * kHidden);
#pragma unroll
        for (int q = 0; q < kHidden / 4; ++q) {
            const float4 w4 = row[q];
            z = fmaf(w4.x, h1[4 * q], z);
            z = fmaf(w4.y, h1[4 * q + 1], z);
            z = fmaf(w4.z, h1[4 * q + 2], z);
            z = fmaf(w4.w, h1[4 * q + 3], z);
        }
        y = fmaf(W[kW3 + j], fmaxf(z, 0.f), y);
    }
    return y;
}

__global__ void __launch_bounds__(256) mlp_predict_kernel(const __nv_bfloat16 *w, const float *X, uint64_t n, float *y) {
    __shared__ __align__(16) float Ws[kMlpParams];
    stage_weights(w, Ws);
    __syncthreads();
#pragma unroll 1
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
        float f[kFeat];
#pragma unroll
        for (int k = 0; k < kFeat; ++k) f[k] = X[r * kFeat + k];
        y[r] = mlp_eval(Ws, f);
    }
}

__global__ void __launch_bounds__(256) lineage_predict_kernel(FeatureArgs a, const __nv_bfloat16 *w, float *pred_end) {
    const uint64_t n = *a.n_cur;
    if (n <= a.skip_at_most) return;  // the step kernel gives every lineage a warp
    __shared__ __align__(16) float Ws[kMlpParams];
    stage_weights(w, Ws);
    __syncthreads();
#pragma unroll 1
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t steps = a.in.steps[j];
        const float pe = pred_end[j];
        if (pe > 0.f && pe >= (float)steps + 1.0f) continue;  // prediction still ahead
        const uint32_t s = a.in.sim[j];
        float f[kFeat];
        lineage_features(a.kind, a.params[s], a.counters[s], a.in.x[j], a.in.y[j], a.in.last[j], steps, f);
        const float rem = expm1f(fminf(fmaxf(mlp_eval(Ws, f), 0.f), 40.f));
        pred_end[j] = (float)steps + fmaxf(rem, 1.0f);
    }
}

__global__ void trace_snapshot_kernel(FeatureArgs a, uint32_t snap, TraceRow *rows, unsigned long long *n_rows,
                                      uint64_t cap) {
    const uint64_t n = *a.n_cur;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = a.in.sim[j];
        if (!a.params[s].active) continue;
        // about kTraceRowsPerSim rows per simulation and snapshot, so that
        // large simulations do not crowd out the others
        const uint64_t live = a.counters[s].n_live;
        const uint64_t stride = live > kTraceRowsPerSim ? live / kTraceRowsPerSim : 1;
        const uint64_t gref = a.in.gref[j];
        if (stride > 1 && seahash_diffuse(gref ^ ((uint64_t)snap << 40)) % stride != 0) continue;
        TraceRow r;
        lineage_features(a.kind, a.params[s], a.counters[s], a.in.x[j], a.in.y[j], a.in.last[j], a.in.steps[j], r.f);
        r.gref = gref;
        r.steps = a.in.steps[j];
        r.sim = s;
        r.snap = snap;
        r.time = a.in.last[j];
        const unsigned long long i = atomicAdd(n_rows, 1ULL);
        if (i < cap) rows[i] = r;
    }
}

// ---- training: one tile of 64 samples per pass, 256 threads ----
constexpr int kTile = 64;
constexpr int kRow = kHidden + 1;  // padded activation row (bank-conflict free)
constexpr int kGradThreads = 256;

struct GradSmem {
    float W[kMlpParams];
    float W1T[kFeat * kHidden];    // [k][j]
    float W2T[kHidden * kHidden];  // [i][j]
    float X[kTile * kFeat];
    float T[kTile];
    float dy[kTile];
    float H1[kTile * kRow];
    float H2[kTile * kRow];
    float D2[kTile * kRow];
    float D1[kTile * kRow];
};

__global__ void __launch_bounds__(kGradThreads) mlp_grad_kernel(const __nv_bfloat16 *w, const float *X,
                                                                const float *T, const uint32_t *perm,
                                                                uint64_t offset, uint64_t n, float inv_n,
                                                                float *grads, double *loss) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GradSmem &S = *reinterpret_cast<GradSmem *>(smem_raw);
    const int t = threadIdx.x;
    for (int i = t; i < kMlpParams; i += kGradThreads) {
        const float v = __bfloat162float(w[i]);
        S.W[i] = v;
        if (i >= kW1 && i < kB1) {
            const int j = (i - kW1) / kFeat, k = (i - kW1) % kFeat;
            S.W1T[k * kHidden + j] = v;
        } else if (i >= kW2 && i < kB2) {
            const int j = (i - kW2) / kHidden, ii = (i - kW2) % kHidden;
            S.W2T[ii * kHidden + j] = v;
        }
    }
    // per-thread gradient accumulators for the entries this thread owns
    float gW2[16], gW1[2];
#pragma unroll
    for (int m = 0; m < 16; ++m) gW2[m] = 0.f;
    gW1[0] = gW1[1] = 0.f;
    float gb1 = 0.f, gb2 = 0.f, gW3 = 0.f, gb3 = 0.f;
    double lsum = 0.0;
    __syncthreads();

    const uint64_t tiles = (n + kTile - 1) / kTile;
    for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint64_t r0 = tile * kTile;
        // inputs
        for (int e = t; e < kTile * kFeat; e += kGradThreads) {
            const int s = e / kFeat, k = e % kFeat;
            const uint64_t i = r0 + s;
            float v = 0.f;
            if (i < n) {
                const uint64_t row = perm ? perm[offset + i] : offset + i;
                v = X[row * kFeat + k];
            }
            S.X[e] = v;
        }
        if (t < kTile) {
            const uint64_t i = r0 + t;
            S.T[t] = (i < n) ? T[perm ? perm[offset + i] : offset + i] : 0.f;
        }
        __syncthreads();
        // H1 = relu(W1 x + b1)
        for (int e = t; e < kTile * kHidden; e += kGradThreads) {
            const int s = e / kHidden, j = e % kHidden;
            float z = S.W[kB1 + j];
#pragma unroll
            for (int k = 0; k < kFeat; ++k) z = fmaf(S.W1T[k * kHidden + j], S.X[s * kFeat + k], z);
            S.H1[s * kRow + j] = fmaxf(z, 0.f);
        }
        __syncthreads();
        // H2 = relu(W2 h1 + b2)
        for (int e = t; e < kTile * kHidden; e += kGradThreads) {
            const int s = e / kHidden, j = e % kHidden;
            float z = S.W[kB2 + j];
            for (int i = 0; i < kHidden; ++i) z = fmaf(S.W2T[i * kHidden + j], S.H1[s * kRow + i], z);
            S.H2[s * kRow + j] = fmaxf(z, 0.f);
        }
        __syncthreads();
        // output, loss and d loss / d y
        if (t < kTile) {
            float y = S.W[kB3];
            for (int j = 0; j < kHidden; ++j) y = fmaf(S.W[kW3 + j], S.H2[t * kRow + j], y);
            const bool valid = r0 + t < n;
            const float err = valid ? (y - S.T[t]) : 0.f;
            S.dy[t] = err * inv_n;
            lsum += 0.5 * (double)err * (double)err * (double)inv_n;
        }
        __syncthreads();
        // D2 = dy * W3 * relu'(z2); output-layer gradients
        for (int e = t; e < kTile * kHidden; e += kGradThreads) {
            const int s = e / kHidden, j = e % kHidden;
            S.D2[s * kRow + j] = S.H2[s * kRow + j] > 0.f ? S.dy[s] * S.W[kW3 + j] : 0.f;
        }
        if (t < kHidden) {
            float g = 0.f;
            for (int s = 0; s < kTile; ++s) g = fmaf(S.dy[s], S.H2[s * kRow + t], g);
            gW3 += g;
        }
        if (t == 0) {
            float g = 0.f;
            for (int s = 0; s < kTile; ++s) g += S.dy[s];
            gb3 += g;
        }
        __syncthreads();
        // layer 2 gradients and D1 = (W2^T D2) * relu'(z1)
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int e = t + kGradThreads * m;
            const int j = e / kHidden, i = e % kHidden;
            float g = 0.f;
            for (int s = 0; s < kTile; ++s) g = fmaf(S.D2[s * kRow + j], S.H1[s * kRow + i], g);
            gW2[m] += g;
        }
        if (t < kHidden) {
            float g = 0.f;
            for (int s = 0; s < kTile; ++s) g += S.D2[s * kRow + t];
            gb2 += g;
        }
        for (int e = t; e < kTile * kHidden; e += kGradThreads) {
            const int s = e / kHidden, i = e % kHidden;
            float g = 0.f;
            for (int j = 0; j < kHidden; ++j) g = fmaf(S.D2[s * kRow + j], S.W[kW2 + j * kHidden + i], g);
            S.D1[s * kRow + i] = S.H1[s * kRow + i] > 0.f ? g : 0.f;
        }
        __syncthreads();
        // layer 1 gradients
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            const int e = t + kGradThreads * m;
            const int j = e / kFeat, k = e % kFeat;
            float g = 0.f;
            for (int s = 0; s < kTile; ++s) g = fmaf(S.D1[s * kRow + j], S.X[s * kFeat + k], g);
            gW1[m] += g;
        }
        if (t < kHidden) {
            float g = 0.f;
            for (int s = 0; s < kTile; ++s) g += S.D1[s * kRow + t];
            gb1 += g;
        }
        __syncthreads();
    }
#pragma unroll
    for (int m = 0; m < 16; ++m) atomicAdd(&grads[kW2 + t + kGradThreads * m], gW2[m]);
#pragma unroll
    for (int m = 0; m < 2; ++m) atomicAdd(&grads[kW1 + t + kGradThreads * m], gW1[m]);
    if (t < kHidden) {
        atomicAdd(&grads[kB1 + t], gb1);
        atomicAdd(&grads[kB2 + t], gb2);
        atomicAdd(&grads[kW3 + t], gW3);
    }
    if (t == 0) atomicAdd(&grads[kB3], gb3);
    if (t < kTile && lsum != 0.0) atomicAdd(loss, lsum);
}

__global__ void adam_kernel(float *master, float *m, float *v, float *grads, __nv_bfloat16 *w, float lr,
                            float beta1, float beta2, float eps, float corr1, float corr2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    const float g = grads[i];
    const float mi = beta1 * m[i] + (1.f - beta1) * g;
    const float vi = beta2 * v[i] + (1.f - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float upd = lr * (mi / corr1) / (sqrtf(vi / corr2) + eps);
    const float nw = master[i] - upd;
    master[i] = nw;
    w[i] = __float2bfloat16_rn(nw);
    grads[i] = 0.f;
}

// ---- queue order: bucket sort by expected work in the round ----

// events per lineage this round under the canonical schedule
// (clamp(ceil(min_round_events / n_live), step_slice, step_slice_max))
__device__ __forceinline__ float round_events(const SimParams &p, const SimCounters &c) {
    const unsigned long long live = c.n_live ? c.n_live : 1ULL;
    unsigned long long per = (p.min_round_events + live - 1) / live;
    if (p.step_slice_max && per > p.step_slice_max) per = p.step_slice_max;
    const unsigned long long lo = p.step_slice ? p.step_slice : 1ULL;
    if (per < lo) per = lo;
    return (float)per;
}

__global__ void order_key_kernel(FeatureArgs a, const float *pred_end, uint8_t *keys, unsigned *hist) {
    const uint64_t n = *a.n_cur;
    if (n <= a.skip_at_most) return;
    __shared__ unsigned h[kOrderBuckets];
    if (threadIdx.x < kOrderBuckets) h[threadIdx.x] = 0;
    __syncthreads();
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = a.in.sim[j];
        const float rem = pred_end[j] - (float)a.in.steps[j];
        const float work = fmaxf(fminf(round_events(a.params[s], a.counters[s]), rem), 1.0f);
        // bucket 0 holds the most work: 31 - floor(log2(work))
        const int e = ilogbf(work);
        const int b = kOrderBuckets - 1 - (e < 0 ? 0 : (e > kOrderBuckets - 1 ? kOrderBuckets - 1 : e));
        keys[j] = (uint8_t)b;
        atomicAdd(&h[b], 1u);
    }
    __syncthreads();
    if (threadIdx.x < kOrderBuckets && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// exclusive scan of the bucket counts into cursors; clears the counts
__global__ void order_scan_kernel(unsigned *hist) {
    const unsigned lane = threadIdx.x;
    const unsigned c = hist[lane];
    unsigned x = c;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const unsigned y = __shfl_up_sync(kFullMask, x, off);
        if ((int)lane >= off) x += y;
    }
    hist[kOrderBuckets + lane] = x - c;
    hist[lane] = 0;
}

__global__ void order_scatter_kernel(const unsigned long long *n_cur, uint64_t skip_at_most, const uint8_t *keys,
                                     unsigned *hist, uint32_t *order) {
    const uint64_t n = *n_cur;
    if (n <= skip_at_most) return;
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint64_t j = base + threadIdx.x;
        const bool ok = j < n;
        const unsigned b = ok ? keys[j] : 0xffffffffu;
        const unsigned same = __match_any_sync(kFullMask, b);
        const int leader = __ffs(same) - 1;
        unsigned pos = 0;
        if (ok && (int)lane == leader) pos = atomicAdd(&hist[kOrderBuckets + b], (unsigned)__popc(same));
        pos = __shfl_sync(kFullMask, pos, leader);
        if (ok) order[pos + __popc(same & ((1u << lane) - 1u))] = (uint32_t)j;
    }
}

// The current device's SM count, queried once per device; launch grids are
// multiples of it.
unsigned current_sm_count() {
    constexpr int kMaxDevices = 64;
    static std::atomic<int> cache[kMaxDevices];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 1;
    int v = cache[dev].load();
    if (v == 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v < 1) v = 1;
        cache[dev].store(v);
    }
    return (unsigned)v;
}

}  // namespace

cudaError_t launch_trace_snapshot(const FeatureArgs &f, uint32_t snap, TraceRow *rows, unsigned long long *n_rows,
                                  uint64_t cap, cudaStream_t st) {
    trace_snapshot_kernel<<<current_sm_count() * 4, 256, 0, st>>>(f, snap, rows, n_rows, cap);
    return cudaGetLastError();
}

cudaError_t launch_lineage_predict(const FeatureArgs &f, const __nv_bfloat16 *w, float *pred_end, cudaStream_t st) {
    lineage_predict_kernel<<<current_sm_count() * 4, 256, 0, st>>>(f, w, pred_end);
    return cudaGetLastError();
}

cudaError_t launch_order(const FeatureArgs &f, const float *pred_end, uint8_t *keys, unsigned *hist, uint32_t *order,
                         unsigned grid, cudaStream_t st) {
    order_key_kernel<<<grid, 256, 0, st>>>(f, pred_end, keys, hist);
    order_scan_kernel<<<1, 32, 0, st>>>(hist);
    order_scatter_kernel<<<grid, 256, 0, st>>>(f.n_cur, f.skip_at_most, keys, hist, order);
    return cudaGetLastError();
}

cudaError_t launch_mlp_predict(const __nv_bfloat16 *w, const float *X, uint64_t n, float *y, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    uint64_t blocks = (n + 255) / 256;
    if (blocks > current_sm_count() * 8ULL) blocks = current_sm_count() * 8ULL;
    mlp_predict_kernel<<<(unsigned)blocks, 256, 0, st>>>(w, X, n, y);
    return cudaGetLastError();
}

cudaError_t launch_mlp_grad(const __nv_bfloat16 *w, const float *X, const float *T, const uint32_t *perm,
                            uint64_t offset, uint64_t n, float inv_n, float *grads, double *loss, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const size_t smem = sizeof(GradSmem);
    cudaError_t e = cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    uint64_t tiles = (n + kTile - 1) / kTile;
    if (tiles > current_sm_count()) tiles = current_sm_count();
    mlp_grad_kernel<<<(unsigned)tiles, kGradThreads, smem, st>>>(w, X, T, perm, offset, n, inv_n, grads, loss);
    return cudaGetLastError();
}

cudaError_t launch_adam(float *master, float *m, float *v, float *grads, __nv_bfloat16 *w, float lr, float beta1,
                        float beta2, float eps, int step, cudaStream_t st) {
    const float corr1 = 1.f - powf(beta1, (float)step);
    const float corr2 = 1.f - powf(beta2, (float)step);
    adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, st>>>(master, m, v, grads, w, lr, beta1, beta2, eps, corr1,
                                                          corr2);
    return cudaGetLastError();
}

}  // namespace necsim
