// Node graph construction and growth, skinning, forward warp and the solver-map splat.
//
// Integer outputs (node candidates, node and surfel k-NN ids) follow the
// reference bit for bit: the same float expressions with the fused
// multiply-adds spelled out, the same strict-inequality heap, and the same
// Lomuto quicksort.  Weights use __expf as the reference does.
#include <cuda_runtime.h>
#include <cuda_fp16.h>

#include <mutex>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/warpsolve.h"
#include "ws_common.cuh"
#include "ws_obs_point.cuh"
#include "ws_prims.cuh"

namespace ws {

// Squared length as nvcc contracts `x*x + y*y + z*z` under its default -fmad=true.
__device__ __forceinline__ float sq3_fused(float x, float y, float z) {
    return __fmaf_rn(z, z, __fmaf_rn(y, y, __fmul_rn(x, x)));
}

// KnnHeapExpandDevice (libs/star/geometry/node_graph/brute_force_knn.cuh:52-135).
template <int CAP>
struct Heap {
    float d[CAP];
    uint16_t id[CAP];
    int max_id;
    float max_d;
    __device__ __forceinline__ void init(float v) {
#pragma unroll
        for (int i = 0; i < CAP; ++i) { d[i] = v; id[i] = 0; }
        refresh();
    }
    __device__ __forceinline__ void refresh() {
        max_id = 0;
        max_d = d[0];
#pragma unroll
        for (int i = 1; i < CAP; ++i)
            if (d[i] > max_d) { max_d = d[i]; max_id = i; }
    }
    __device__ __forceinline__ void update(uint16_t idx, float dist) {
        if (dist < max_d) {
#pragma unroll
            for (int i = 0; i < CAP; ++i)
                if (i == max_id) { d[i] = dist; id[i] = idx; }
        }
        refresh();
    }
    // Lomuto quicksort on strict <, iterative form of the reference's recursion
    // (same partitions in the same order).
    __device__ void sort() {
        int lo_stack[2 * CAP + 2], hi_stack[2 * CAP + 2];
        int top = 0;
        lo_stack[0] = 0;
        hi_stack[0] = CAP - 1;
        top = 1;
        while (top > 0) {
            --top;
            const int low = lo_stack[top], high = hi_stack[top];
            if (low >= high) continue;
            const float pivot = d[high];
            int i = low - 1;
            for (int j = low; j <= high - 1; ++j) {
                if (d[j] < pivot) {
                    ++i;
                    const float td = d[i]; d[i] = d[j]; d[j] = td;
                    const uint16_t ti = id[i]; id[i] = id[j]; id[j] = ti;
                }
            }
            { const float td = d[i + 1]; d[i + 1] = d[high]; d[high] = td; }
            { const uint16_t ti = id[i + 1]; id[i + 1] = id[high]; id[high] = ti; }
            const int pi = i + 1;
            // recursion order: left part first, then right part
            lo_stack[top] = pi + 1; hi_stack[top] = high; ++top;
            lo_stack[top] = low; hi_stack[top] = pi - 1; ++top;
        }
    }
};

// createVoxelKeyKernel (libs/star/geometry/sampling/VoxelSubsamplerSorting.cu:8-21) with
// encodeVoxel (libs/star/common/encode_utils.h:138-141).  The reference sorts the encoded keys
// as signed ints; a voxel below -512 in z gives a negative key, which sorts first.  The keys here
// go through an unsigned radix sort, so they carry the sign bit flipped (kVoxelKeyBias), which
// orders them as signed ints; the sampler flips it back before decoding.
constexpr uint32_t kVoxelKeyBias = 0x80000000u;
__global__ void k_voxel_key(const float4 *pts, uint32_t n, float voxel, uint32_t *keys, uint32_t *vals) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = pts[i];
        const int vx = __float2int_rd(p.x / voxel), vy = __float2int_rd(p.y / voxel), vz = __float2int_rd(p.z / voxel);
        const int enc = (int)((unsigned)(vx + 512) + (unsigned)(vy + 512) * 1024u + (unsigned)(vz + 512) * 1048576u);
        keys[i] = (uint32_t)enc ^ kVoxelKeyBias;
        vals[i] = i;
    }
}

__global__ void k_voxel_marks(const uint32_t *keys, uint32_t n, uint32_t *marks) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        marks[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// samplingPointsKernel (VoxelSubsamplerSorting.cu:60-96): per voxel the point nearest the
// voxel centre, first wins on ties.  The centre is a rounded float3 computed before the loop
// over the voxel's points, as the source writes it; the intrinsics keep nvcc from fusing its
// product into the subtraction, which moves squared distances by about 1e-10 m^2 and flips
// near-ties between points (about 2 voxels in 89k on a 1M-point torus).
__global__ void k_voxel_sample(const uint32_t *keys, const uint32_t *perm, const uint32_t *head_off, uint32_t n,
                               const float4 *pts, float voxel, float4 *out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (i != 0 && keys[i] == keys[i - 1]) continue;   // not the first point of its voxel
        uint32_t e = i + 1;
        while (e < n && keys[e] == keys[i]) ++e;
        const int enc = (int)(keys[i] ^ kVoxelKeyBias);
        int z = enc / (1024 * 1024);
        int x = enc % 1024;
        int y = (enc - z * 1024 * 1024) / 1024;
        x -= 512; y -= 512; z -= 512;
        const float cx = __fmul_rn(float(x + 0.5), voxel), cy = __fmul_rn(float(y + 0.5), voxel),
                    cz = __fmul_rn(float(z + 0.5), voxel);
        float best = 1e5f;
        uint32_t bi = i;
        for (uint32_t k = i; k < e; ++k) {
            const float4 p = pts[perm[k]];
            const float dd = sq3_fused(__fsub_rn(p.x, cx), __fsub_rn(p.y, cy), __fsub_rn(p.z, cz));
            if (dd < best) { best = dd; bi = k; }
        }
        out[head_off[i]] = pts[perm[bi]];
    }
}

// ---- Overlap check of the node candidates on the device ----
//
// AppendNodeFromVertexHost (libs/star/geometry/node_graph/NodeGraph.cu:652-704) walks the
// candidates in order and keeps one when no candidate kept before it lies within 0.85 R
// (squared distance <= (0.85 R)^2, summed as ((dx*dx + dy*dy) + dz*dz) + dw*dw with dw = 0).
// That is the lexicographically first maximal independent set of the graph that joins
// candidates within 0.85 R, and it comes out of rounds: a candidate is rejected once one of
// its earlier neighbours is kept, and kept once all of them are rejected.  Every decision is
// final and equals the sequential loop's (by induction on the index), and each round decides
// at least the lowest undecided candidate, so at most nv rounds run.

// Dedup grid: cells of 1.125 x the overlap radius.  Two candidates that pass the distance test
// differ by at most r (1 + 2^-22) per axis, i.e. 0.889 cells; the scaled coordinates are
// clamped to +-2^18 cells, where a float resolves 1/32 of a cell, so their rounding adds at most
// 1/32 and such candidates lie in the same or adjacent cells.  Cell coordinates wrap at 1024
// per axis, which only adds far candidates that the distance test turns away.
constexpr float kDedupCellScale = 1.125f;

__device__ __forceinline__ int dedup_cell(float v, float inv_cell) {
    return __float2int_rd(fminf(fmaxf(__fmul_rn(v, inv_cell), -262144.f), 262144.f));
}

__device__ __forceinline__ uint32_t dedup_key(int x, int y, int z) {
    return (uint32_t)(x & 1023) | ((uint32_t)(y & 1023) << 10) | ((uint32_t)(z & 1023) << 20);
}

__global__ void k_dedup_keys(const float4 *cand, uint32_t nv, float inv_cell, uint32_t *keys, uint32_t *ids, int *err) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
        const float4 p = cand[i];
        if (isnan(p.x) || isnan(p.y) || isnan(p.z)) atomicOr(err, 1);
        keys[i] = dedup_key(dedup_cell(p.x, inv_cell), dedup_cell(p.y, inv_cell), dedup_cell(p.z, inv_cell));
        ids[i] = i;
    }
}

__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *a, uint32_t n, uint32_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(a + mid) < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Earlier candidates that overlap candidate i, found in the 3 x 3 rows of three cells around
// it (a row is one key range unless its x wraps).  kFill = false counts them into `cnt`;
// kFill = true writes their indices from offset `cnt[i]` of `nbr`.
template <bool kFill>
__global__ void k_dedup_neighbours(const float4 *cand, const uint32_t *cell_keys, const uint32_t *cell_ids, uint32_t nv,
                                   float inv_cell, float thr, uint32_t *cnt, uint32_t *nbr) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
        const float4 p = cand[i];
        const int cx = dedup_cell(p.x, inv_cell), cy = dedup_cell(p.y, inv_cell), cz = dedup_cell(p.z, inv_cell);
        const int x0 = (cx - 1) & 1023, x1 = (cx + 1) & 1023;
        uint32_t c = 0, out = kFill ? cnt[i] : 0u;
        for (int dz = -1; dz <= 1; ++dz) {
            for (int dy = -1; dy <= 1; ++dy) {
                uint32_t lo_key[2], hi_key[2];
                int ranges = 1;
                if (x0 < x1) {
                    lo_key[0] = dedup_key(x0, cy + dy, cz + dz);
                    hi_key[0] = dedup_key(x1, cy + dy, cz + dz);
                } else {
                    lo_key[0] = dedup_key(x0, cy + dy, cz + dz);
                    hi_key[0] = dedup_key(1023, cy + dy, cz + dz);
                    lo_key[1] = dedup_key(0, cy + dy, cz + dz);
                    hi_key[1] = dedup_key(x1, cy + dy, cz + dz);
                    ranges = 2;
                }
                for (int q = 0; q < ranges; ++q) {
                    for (uint32_t b = lower_bound_u32(cell_keys, nv, lo_key[q]); b < nv && __ldg(cell_keys + b) <= hi_key[q];
                         ++b) {
                        const uint32_t j = __ldg(cell_ids + b);
                        if (j >= i) continue;
                        const float4 o = cand[j];
                        const float ex = o.x - p.x, ey = o.y - p.y, ez = o.z - p.z;
                        const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)), __fmul_rn(ez, ez));
                        if (d2 <= thr) {
                            if (kFill) nbr[out++] = j; else ++c;
                        }
                    }
                }
            }
        }
        if (!kFill) cnt[i] = c;
    }
}

// The rounds for small candidate sets (at most kDedupOneBlockMax), in one block of 1024
// threads.  Decisions (0 open, 1 kept, 2 rejected) live in shared memory, one byte per
// candidate, and are read volatile, so a decision taken earlier in the same round is used at
// once.  Thread t walks candidates t, t + 1024, ... from the first one it has not yet settled.
// On return `decision` holds every decision; `err` is set only if nv + 1 rounds left a
// candidate open, which the argument above excludes.
constexpr int kDedupThreads = 1024;
constexpr uint32_t kDedupOneBlockMax = 16384;

__global__ void __launch_bounds__(kDedupThreads) k_dedup_greedy(const uint32_t *nbr_ptr, const uint32_t *nbr, uint32_t nv,
                                                                uint8_t *decision, int *err) {
    extern __shared__ uint8_t s_decision[];
    volatile uint8_t *dec = s_decision;
    for (uint32_t i = threadIdx.x; i < nv; i += kDedupThreads) dec[i] = 0;
    __syncthreads();
    uint32_t first = threadIdx.x;
    bool done = false;
    for (uint32_t round = 0; round <= nv && !done; ++round) {   // uniform: `done` comes from a block vote
        int open = 0;
        bool settled_prefix = true;
        for (uint32_t i = first; i < nv; i += kDedupThreads) {
            uint8_t d = dec[i];
            if (d == 0) {
                d = 1;
                for (uint32_t k = __ldg(nbr_ptr + i), e = __ldg(nbr_ptr + i + 1); k < e; ++k) {
                    const uint8_t t = dec[__ldg(nbr + k)];
                    if (t == 1) { d = 2; break; }
                    if (t == 0) d = 0;
                }
                if (d != 0) dec[i] = d;
            }
            if (d == 0) {
                open = 1;
                settled_prefix = false;
            } else if (settled_prefix) {
                first = i + kDedupThreads;
            }
        }
        done = !__syncthreads_or(open);
    }
    if (!done && threadIdx.x == 0) atomicOr(err, 2);
    for (uint32_t i = threadIdx.x; i < nv; i += kDedupThreads) decision[i] = s_decision[i];
}

// The same rounds over the whole GPU, for large candidate sets.  One launch whose blocks are
// all resident (a cooperative launch); thread t takes candidates t, t + T, ... (T threads in
// all); decisions in global memory (zeroed before the launch), read volatile; a barrier of our
// own between rounds.  sync[0] counts a barrier's arrivals, sync[1] is its generation, and
// sync[2 + r % 2] says whether round r left a candidate open: every write to it comes before
// round r's barrier, so all threads read the same value after it, and the barrier's last
// arrival clears the other word for round r + 1 (its readers, in round r - 1, have all arrived).
// A barrier wait sleeps with backoff and gives up after about two seconds of requested sleep,
// or at once when another block has: `err` gets 4 and the blocks leave.
constexpr int kDedupGridThreads = 512;
constexpr unsigned long long kDedupBarrierTimeoutNs = 2000000000ull;

__device__ bool dedup_grid_barrier(unsigned *sync, unsigned clear_word, int *err) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile unsigned *gen = sync + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(sync, 1u) == gridDim.x - 1) {
            atomicExch(sync + clear_word, 0u);
            atomicExch(sync, 0u);
            __threadfence();
            atomicAdd(sync + 1, 1u);
        } else {
            unsigned long long waited_ns = 0;
            unsigned sleep_ns = 32;
            while (*gen == g) {
                if (waited_ns > kDedupBarrierTimeoutNs || (*reinterpret_cast<volatile int *>(err) & 4) != 0) {
                    atomicOr(err, 4);
                    ok = 0;
                    break;
                }
                __nanosleep(sleep_ns);
                waited_ns += sleep_ns;
                sleep_ns = min(sleep_ns * 2u, 256u);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

__global__ void __launch_bounds__(kDedupGridThreads) k_dedup_greedy_grid(const uint32_t *nbr_ptr, const uint32_t *nbr,
                                                                        uint32_t nv, uint8_t *decision, unsigned *sync,
                                                                        int *err) {
    volatile uint8_t *dec = decision;
    const uint32_t threads = gridDim.x * blockDim.x;
    uint32_t first = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t round = 0; round <= nv; ++round) {   // uniform: the exit reads a word written before the barrier
        int open = 0;
        bool settled_prefix = true;
        for (uint32_t i = first; i < nv; i += threads) {
            uint8_t d = dec[i];
            if (d == 0) {
                d = 1;
                for (uint32_t k = __ldg(nbr_ptr + i), e = __ldg(nbr_ptr + i + 1); k < e; ++k) {
                    const uint8_t t = dec[__ldg(nbr + k)];
                    if (t == 1) { d = 2; break; }
                    if (t == 0) d = 0;
                }
                if (d != 0) dec[i] = d;
            }
            if (d == 0) {
                open = 1;
                settled_prefix = false;
            } else if (settled_prefix) {
                first = i + threads;
            }
        }
        volatile unsigned *flag = sync + 2 + (round & 1);
        if (open) *flag = 1u;
        if (!dedup_grid_barrier(sync, 2 + ((round + 1) & 1), err)) return;
        if (*flag == 0u) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(err, 2);
}

// Failure-detection self-test of the barrier above: two blocks launched, only block 0 arrives,
// so the generation never advances and block 0 must give up after about two seconds of
// requested sleep with bit 2 of err set, and return.
__global__ void k_barrier_selftest(unsigned *sync, int *err) {
    if (blockIdx.x == 0) dedup_grid_barrier(sync, 2, err);
}

cudaError_t grid_barrier_selftest(int *flags, cudaStream_t st) {
    unsigned *words = nullptr;   // sync[0..3], err
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&words), 5 * sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(words, 0, 5 * sizeof(unsigned), st);
    int *err = reinterpret_cast<int *>(words + 4);
    int flag = 0;
    if (e == cudaSuccess) {
        k_barrier_selftest<<<2, 32, 0, st>>>(words, err);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    const cudaError_t f = cudaFreeAsync(words, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = f;
    *flags = flag;
    return e;
}

__global__ void k_dedup_flags(const uint8_t *decision, uint32_t nv, uint32_t *flags) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x)
        flags[i] = decision[i] == 1 ? 1u : 0u;
}

// Kept candidates in candidate order, w = 1 (the host loop appends make_float4(x, y, z, 1)).
__global__ void k_dedup_emit(const float4 *cand, const uint8_t *decision, const uint32_t *pos, uint32_t nv, float4 *out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x)
        if (decision[i] == 1) {
            const float4 c = cand[i];
            out[pos[i]] = make_float4(c.x, c.y, c.z, 1.0f);
        }
}

__global__ void k_fill_u32(uint32_t *a, uint32_t n, uint32_t v) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = v;
}

// Bounding boxes of runs of kGraphRun consecutive nodes (lo in boxes[0, runs), hi after).
// NaN coordinates stay out of a box: fminf/fmaxf return the other operand.
constexpr int kGraphRun = 32;

__global__ void k_node_boxes(const float4 *nodes, int n, float4 *lo, float4 *hi) {
    const int runs = (n + kGraphRun - 1) / kGraphRun;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < runs; r += gridDim.x * blockDim.x) {
        float4 a = make_float4(INFINITY, INFINITY, INFINITY, 0.f), b = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
        for (int k = r * kGraphRun, e = min(n, (r + 1) * kGraphRun); k < e; ++k) {
            const float4 p = nodes[k];
            a.x = fminf(a.x, p.x); a.y = fminf(a.y, p.y); a.z = fminf(a.z, p.z);
            b.x = fmaxf(b.x, p.x); b.y = fmaxf(b.y, p.y); b.z = fmaxf(b.z, p.z);
        }
        lo[r] = a;
        hi[r] = b;
    }
}

// UpdateNodeDistanceKernel + BuildNodeGraphKernel (libs/star/geometry/node_graph/NodeGraph.cu:10-101):
// half-precision squared distances, k nearest including the node itself, __expf weights normalized.
//
// The reference fills an n x n table of half distances and scans a row of it in column order.
// Here each node scans the other nodes in the same order but skips a run of kGraphRun whose
// box is no nearer than the heap's current maximum.  Such a run cannot change the heap: the
// per-axis gap to the box is at most each member's |dx| (a difference rounded to nearest is
// monotone in its operands), the squared sum and the rounding to half are monotone too, so
// the same expression on the gaps bounds every member's half distance from below, and the
// heap only takes a distance strictly below its maximum.  Every heap update of the full scan
// happens in the same order, so ids, weights and their ties come out the same.
//
// With node_status, a pair with a deleted node (status .y == kDeletedNodeStatus, NodeGraph.h:18)
// gets the half of 1e6, which is infinite (NodeGraph.cu:20-35), so it never enters a heap; a
// deleted node's own row keeps the heap's initial entries.  The boxes may still hold deleted
// nodes: that only makes them larger, and the skip stays exact.  `normalize` divides the weights
// by their sum (USE_INTERPOLATE_WEIGHT_NORMALIZATION, NodeGraph.cu:87-99); without it they are the
// raw __expf values, as the reference's geometry library compiles them.
constexpr uint32_t kDeletedNodeStatus = 0xffffffffu;
__device__ __forceinline__ bool node_deleted(const uint2 *status, int i) {
    return status != nullptr && status[i].y == kDeletedNodeStatus;
}

template <int K>
__global__ void k_node_graph(const float4 *nodes, const uint2 *status, int n, float r2, int normalize,
                             const float4 *box_lo, const float4 *box_hi, uint16_t *knn, float *w, uint16_t *edges) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
        const float4 va = nodes[a];
        Heap<K> h;
        h.init(1e3f);
        const bool a_deleted = node_deleted(status, a);
        for (int r0 = 0, run = 0; r0 < n && !a_deleted; r0 += kGraphRun, ++run) {
            const float4 lo = box_lo[run], hi = box_hi[run];
            const float gx = fmaxf(fmaxf(lo.x - va.x, va.x - hi.x), 0.f);
            const float gy = fmaxf(fmaxf(lo.y - va.y, va.y - hi.y), 0.f);
            const float gz = fmaxf(fmaxf(lo.z - va.z, va.z - hi.z), 0.f);
            const float bound = __fmaf_rn(gz, gz, __fmaf_rn(gy, gy, __fmul_rn(gx, gx)));
            if (__half2float(__float2half_rn(bound)) >= h.max_d) continue;
            for (int b = r0, e = min(n, r0 + kGraphRun); b < e; ++b) {
                const float4 vb = nodes[b];
                const float4 hi_v = (a >= b) ? va : vb, lo_v = (a >= b) ? vb : va;
                const float dx = hi_v.x - lo_v.x, dy = hi_v.y - lo_v.y, dz = hi_v.z - lo_v.z;
                const float dist = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
                h.update((uint16_t)b, node_deleted(status, b) ? __half2float(__float2half_rn(1e6f))
                                                               : __half2float(__float2half_rn(dist)));
            }
        }
        h.sort();
        float wv[K], sum = 0.f;
#pragma unroll
        for (int q = 0; q < K; ++q) wv[q] = __expf(-h.d[q] / (2 * r2));
#pragma unroll
        for (int q = 0; q < K; ++q) sum += wv[q];
        const float inv = 1.0f / sum;
#pragma unroll
        for (int q = 0; q < K; ++q) {
            knn[(size_t)a * K + q] = h.id[q];
            w[(size_t)a * K + q] = normalize ? wv[q] * inv : wv[q];
            // BuildNodeGraphPairKernel (NodeGraph.cu:103-118)
            edges[3 * ((size_t)a * K + q)] = (uint16_t)a;
            edges[3 * ((size_t)a * K + q) + 1] = h.id[q];
            edges[3 * ((size_t)a * K + q) + 2] = (uint16_t)q;
        }
    }
}

// SkinnerKernel (libs/star/geometry/node_graph/Skinner.cu:10-94) and IncSkinnerKernel (:211-302);
// nodes staged in shared memory.  A deleted node (status .y == kDeletedNodeStatus) enters the
// heap at distance 1e6 (Skinner.cu:39-48).  Full skinning (first_vert = 0, prev_nodes = 0) starts
// every heap at 1e6; the incremental form re-skins surfels first_vert .. n_verts - 1: the heap
// starts from the surfel's current neighbours at their distances and takes the nodes
// prev_nodes .. n_nodes - 1.  `normalize` divides the weights by their sum
// (USE_INTERPOLATE_WEIGHT_NORMALIZATION, Skinner.cu:70-74, 278-282).
__global__ void __launch_bounds__(256) k_skinning(const float4 *nodes, const uint2 *status, int n_nodes,
                                                   int prev_nodes, const float4 *verts, int first_vert, int n_verts,
                                                   float r2, int normalize, ushort4 *knn, float4 *sw, float4 *cw) {
    __shared__ float4 tile[1024];
    __shared__ unsigned char gone[1024];
    const int v = first_vert + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const bool live = v < n_verts;
    const float4 p = live ? verts[v] : make_float4(0.f, 0.f, 0.f, 0.f);
    Heap<4> h;
    if (prev_nodes > 0 && live) {
        const ushort4 k4 = knn[v];
        const uint16_t ids[4] = {k4.x, k4.y, k4.z, k4.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float4 q = nodes[min((int)ids[i], n_nodes - 1)];
            h.d[i] = sq3_fused(p.x - q.x, p.y - q.y, p.z - q.z);
            h.id[i] = ids[i];
        }
        h.refresh();
    } else {
        h.init(1e6f);
    }
    for (int base = prev_nodes; base < n_nodes; base += 1024) {
        const int cnt = min(1024, n_nodes - base);
        __syncthreads();
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
            tile[i] = nodes[base + i];
            gone[i] = node_deleted(status, base + i) ? 1 : 0;
        }
        __syncthreads();
        for (int i = 0; i < cnt; ++i) {
            const float4 q = tile[i];
            h.update((uint16_t)(base + i), gone[i] ? 1e6f : sq3_fused(p.x - q.x, p.y - q.y, p.z - q.z));
        }
    }
    if (!live) return;
    h.sort();
    float wv[4], sum = 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float4 q = nodes[min((int)h.id[i], n_nodes - 1)];
        const float dd = sq3_fused(p.x - q.x, p.y - q.y, p.z - q.z);
        wv[i] = __expf(-dd / (2.f * r2));
        sum += wv[i];
    }
    const float inv = 1.f / sum;
    knn[v] = make_ushort4(h.id[0], h.id[1], h.id[2], h.id[3]);
    sw[v] = normalize ? make_float4(inv * wv[0], inv * wv[1], inv * wv[2], inv * wv[3])
                      : make_float4(wv[0], wv[1], wv[2], wv[3]);
    cw[v] = make_float4(1.f, 1.f, 1.f, 1.f);
}

// ForwardWarpVertexAndNodeKernel (libs/star/geometry/surfel/SurfelNodeDeformer.cu:13-79) with
// averageDualQuaternion<4> (libs/star/math/DualQuaternion.hpp:288-306).
__global__ void k_forward_warp(const float *se3, int num_nodes, const float4 *verts, const float4 *normals, int n,
                               const ushort4 *knn, const float4 *sw, const float4 *cw, float4 *out_v, float4 *out_n) {
    const uint16_t last = (uint16_t)(num_nodes - 1);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const ushort4 k4 = knn[i];
        const float4 s4 = sw[i], c4 = cw[i];
        const uint16_t ids[4] = {(uint16_t)min(k4.x, last), (uint16_t)min(k4.y, last), (uint16_t)min(k4.z, last),
                                 (uint16_t)min(k4.w, last)};
        const float wv[4] = {s4.x * c4.x, s4.y * c4.y, s4.z * c4.z, s4.w * c4.w};
        DQf avg;
        avg.q0 = make_float4(0.f, 0.f, 0.f, 0.f);
        avg.q1 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            DQf d = load_dq(se3 + 8ull * ids[k]);
            dq_normalize(d);
            avg.q0 = make_float4(avg.q0.x + wv[k] * d.q0.x, avg.q0.y + wv[k] * d.q0.y, avg.q0.z + wv[k] * d.q0.z,
                                 avg.q0.w + wv[k] * d.q0.w);
            avg.q1 = make_float4(avg.q1.x + wv[k] * d.q1.x, avg.q1.y + wv[k] * d.q1.y, avg.q1.z + wv[k] * d.q1.z,
                                 avg.q1.w + wv[k] * d.q1.w);
        }
        const SE3f T = dq_se3(avg);
        const float4 v = verts[i];
        const float3 o = mul(T.rot, f3(v.x, v.y, v.z)) + T.t;
        out_v[i] = make_float4(o.x, o.y, o.z, v.w);
        if (normals && out_n) {
            const float4 nn = normals[i];
            const float3 on = mul(T.rot, f3(nn.x, nn.y, nn.z));
            out_n[i] = make_float4(on.x, on.y, on.z, nn.w);
        }
    }
}

// Solver-map splat: projection as shaders/solver_map.vert:21-27 (pixel = floor(f x / z + c + 0.5)),
// nearest depth wins, ties to the lower surfel id.
__global__ void k_splat(const float4 *verts, int n, int W, int H, float fx, float fy, float cx, float cy, int fp,
                        unsigned long long *zbuf) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 v = verts[i];
        if (!(v.z > 0.f)) continue;
        const int px = (int)floorf(fx * v.x / v.z + cx + 0.5f);
        const int py = (int)floorf(fy * v.y / v.z + cy + 0.5f);
        const unsigned long long key = ((unsigned long long)__float_as_uint(v.z) << 32) | (unsigned)i;
        for (int dy = -fp; dy <= fp; ++dy)
            for (int dx = -fp; dx <= fp; ++dx) {
                const int x = px + dx, y = py + dy;
                if (x < 0 || y < 0 || x >= W || y >= H) continue;
                atomicMin(zbuf + (size_t)y * W + x, key);
            }
    }
}

__global__ void k_splat_resolve(const unsigned long long *zbuf, int npix, const float4 *av, const float4 *an,
                                uint32_t *index, float4 *vmap, float4 *nmap) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        const unsigned long long k = zbuf[p];
        if (k == ~0ull) {
            index[p] = kInvalidIndex;
            if (vmap) vmap[p] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (nmap) nmap[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
            const uint32_t id = (uint32_t)(k & 0xffffffffu);
            index[p] = id;
            if (vmap) { const float4 v = av[id]; vmap[p] = make_float4(v.x, v.y, v.z, 1.f); }
            if (nmap) { const float4 nn = an[id]; nmap[p] = make_float4(nn.x, nn.y, nn.z, 0.f); }
        }
    }
}

// ---- Solver maps as the reference's solver-map pass draws them --------------------------------
// Renderer::DrawSolverMaps (libs/star/geometry/render/RendererDraw.cu:105-160) draws every surfel as
// a point with shaders/solver_map.vert:21-53 and solver_map.frag:10-17.  Restated per surfel:
//   * v_cam = world2camera (v, 1), summed ((m0 x + m1 y) + m2 z) + m3 per row;
//   * culled when v_cam.z > max depth, v_cam.z <= 0, or the surfel is unstable and not recent:
//     confidence (vertex_confid.w) < threshold.x and |time (color_time.z) - current time| >= threshold.y
//     (threshold.y = -1 culls every unstable surfel, DrawSolverMaps without recent observation);
//   * pixel floor(fx x / z + cx + 0.5), floor(fy y / z + cy + 0.5) (the shader's 0.5 shift: the point
//     lands in the pixel that holds its window position), and `footprint` pixels around it;
//   * the depth test keeps the nearest z (the depth buffer clears to the far plane, so z = max depth
//     never passes it); equal depths keep the lower surfel id (the first one drawn);
//   * outputs: reference vertex (xyz, 1), reference normal (xyz, 0), surfel id, and the normalized
//     rgbd (colour bytes of color_time.x / 127.5 - 1, 1 / z); untouched pixels keep the clear values
//     (zeros, id 0xFFFFFFFF), GLClearValues.h:21-34.
// The depth compare runs on the float camera z, where the GL depth buffer holds a quantised window
// depth; two surfels closer than that quantum can resolve differently there.
struct RenderArgs {
    int W, H, fp;
    float fx, fy, cx, cy, max_depth, current_time, conf_threshold, time_threshold;
    float m[12];   // world2camera rows 0..2, row-major
};

__device__ __forceinline__ float row_dot(const float *m, float4 v) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], v.x), __fmul_rn(m[1], v.y)), __fmul_rn(m[2], v.z)), m[3]);
}

__global__ void k_render_keys(const float4 *vc, const float4 *ct, int n, RenderArgs a, unsigned long long *zbuf) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 v = vc[i];
        const float z = row_dot(a.m + 8, v);
        if (!(z > 0.f) || !(z < a.max_depth)) continue;
        const float t = ct ? ct[i].z : a.current_time;
        if (v.w < a.conf_threshold && fabsf(__fsub_rn(t, a.current_time)) >= a.time_threshold) continue;
        const float x = row_dot(a.m, v), y = row_dot(a.m + 4, v);
        const float fpx = floorf(__fadd_rn(__fadd_rn(__fdiv_rn(__fmul_rn(a.fx, x), z), a.cx), 0.5f));
        const float fpy = floorf(__fadd_rn(__fadd_rn(__fdiv_rn(__fmul_rn(a.fy, y), z), a.cy), 0.5f));
        // a point more than the footprint outside the image covers no pixel (this also keeps the
        // conversion to int in range)
        if (!(fpx >= (float)(-a.fp) && fpx < (float)(a.W + a.fp) && fpy >= (float)(-a.fp) && fpy < (float)(a.H + a.fp)))
            continue;
        const int px = (int)fpx, py = (int)fpy;
        const unsigned long long key = ((unsigned long long)__float_as_uint(z) << 32) | (unsigned)i;
        for (int dy = -a.fp; dy <= a.fp; ++dy)
            for (int dx = -a.fp; dx <= a.fp; ++dx) {
                const int qx = px + dx, qy = py + dy;
                if (qx < 0 || qy < 0 || qx >= a.W || qy >= a.H) continue;
                atomicMin(zbuf + (size_t)qy * a.W + qx, key);
            }
    }
}

__global__ void k_render_resolve(const unsigned long long *zbuf, int npix, const float4 *vc, const float4 *nr,
                                 const float4 *ct, uint32_t *index, float4 *vmap, float4 *nmap, float4 *rgbd) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        const unsigned long long k = zbuf[p];
        const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
        if (k == ~0ull) {
            index[p] = kInvalidIndex;
            if (vmap) vmap[p] = zero;
            if (nmap) nmap[p] = zero;
            if (rgbd) rgbd[p] = zero;
            continue;
        }
        const uint32_t id = (uint32_t)(k & 0xffffffffu);
        index[p] = id;
        if (vmap) { const float4 v = vc[id]; vmap[p] = make_float4(v.x, v.y, v.z, 1.f); }
        if (nmap) { const float4 nn = nr[id]; nmap[p] = make_float4(nn.x, nn.y, nn.z, 0.f); }
        if (rgbd) {
            const int enc = ct ? __float_as_int(ct[id].x) : 0;
            const float z = __uint_as_float((uint32_t)(k >> 32));
            rgbd[p] = make_float4(__fsub_rn(__fdiv_rn((float)((enc & 0x00FF0000) >> 16), 127.5f), 1.f),
                                  __fsub_rn(__fdiv_rn((float)((enc & 0x0000FF00) >> 8), 127.5f), 1.f),
                                  __fsub_rn(__fdiv_rn((float)(enc & 0x000000FF), 127.5f), 1.f), __fdiv_rn(1.f, z));
        }
    }
}

// ---- Observation maps as the reference's observation-map pass draws them ----------------------
// Renderer::DrawObservationMaps (libs/star/geometry/render/RendererDraw.cu:353-394) with
// shaders/geometry.vert:40-86 and observation_map.frag:13-17: the same transform, culls and depth
// rule as the solver-map pass, but each surfel is a GL point as wide as its disk's image
// (obs_point in ws_obs_point.cuh, shared with the host check of the tests).  One thread per
// surfel offers its (z bits, id) key to every pixel of its clipped rectangle; the smallest key
// wins, so the nearest z wins and equal depths keep the lower id (GL_LESS in draw order).
__global__ void k_obs_keys(const float4 *vc, const float4 *nr, const float4 *ct, int n, RenderArgs a,
                           unsigned long long *zbuf) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 v4 = vc[i], n4 = nr[i];
        const float v[4] = {v4.x, v4.y, v4.z, v4.w}, nw[4] = {n4.x, n4.y, n4.z, n4.w};
        const float t = ct ? ct[i].z : a.current_time;
        const ObsCover c = obs_point(v, nw, t, a.m, a.fx, a.fy, a.cx, a.cy, a.W, a.H, a.max_depth, a.current_time,
                                     a.conf_threshold, a.time_threshold);
        if (!c.drawn) continue;
        // z > 0 here, so its bits order like its value
        const unsigned long long key = ((unsigned long long)__float_as_uint(c.z) << 32) | (unsigned)i;
        for (int qy = c.y0; qy <= c.y1; ++qy)   // inside the image: obs_point clips the rectangle
            for (int qx = c.x0; qx <= c.x1; ++qx) atomicMin(zbuf + (size_t)qy * a.W + qx, key);
    }
}

__global__ void k_obs_resolve(const unsigned long long *zbuf, int npix, const float4 *ct, uint32_t *index,
                              float4 *rgbd) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        const unsigned long long k = zbuf[p];
        if (k == ~0ull) {   // the clear values (GLClearValues.h:26-33)
            index[p] = kInvalidIndex;
            if (rgbd) rgbd[p] = make_float4(0.f, 0.f, 0.f, 0.f);
            continue;
        }
        const uint32_t id = (uint32_t)(k & 0xffffffffu);
        index[p] = id;
        if (rgbd) {
            float o[4];
            obs_rgbd(ct ? __float_as_int(ct[id].x) : 0, __uint_as_float((uint32_t)(k >> 32)), o);
            rgbd[p] = make_float4(o[0], o[1], o[2], o[3]);
        }
    }
}

// Scratch of ws_splat_maps_noalloc: one depth/id key per pixel of the largest supported
// image, in the module's static device memory (no allocation at call time).
static __device__ __align__(256) unsigned long long g_noalloc_zbuf[WS_NOALLOC_MAX_PIXELS];

static int grid_of(long long n, int threads) {
    long long g = (n + threads - 1) / threads;
    return (int)std::max(1LL, std::min(g, 148LL * 32));
}

}  // namespace ws

namespace {

// Device address of g_noalloc_zbuf per device, looked up once with that device current.
// Fixed-size table: the lookup path allocates nothing.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned long long *g_noalloc_ptr[kMaxDevices] = {};

int noalloc_scratch(unsigned long long **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return WS_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return WS_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, ws::g_noalloc_zbuf) != cudaSuccess || !p) {
            cudaGetLastError();
            return WS_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = static_cast<unsigned long long *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return WS_OK;
}

// Device temporaries of a node-growth call, from the stream-ordered pool of `st`: taken and
// given back in stream order, so later calls reuse the pool's memory without a device-wide
// synchronisation.
struct DeviceBlocks {
    explicit DeviceBlocks(cudaStream_t s) : st(s) {}
    DeviceBlocks(const DeviceBlocks &) = delete;
    DeviceBlocks &operator=(const DeviceBlocks &) = delete;
    cudaStream_t st;
    std::vector<void *> ptrs;
    cudaError_t err = cudaSuccess;
    template <class T>
    T *get(size_t bytes) {
        void *p = nullptr;
        if (err == cudaSuccess) err = cudaMallocAsync(&p, std::max<size_t>(bytes, 16), st);
        if (err != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return static_cast<T *>(p);
    }
    ~DeviceBlocks() {
        for (void *p : ptrs) cudaFreeAsync(p, st);
    }
};

// Node candidates of a point set and the overlap check, all on the device:
// VoxelSubsamplerSorting::PerformSubsample (libs/star/geometry/sampling/VoxelSubsamplerSorting.cu:8-96)
// on a 0.7 R grid, then the greedy check of AppendNodeFromVertexHost (NodeGraph.cu:652-704).
// On WS_OK, (*nodes)[0 .. *kept) holds the kept candidates in candidate order (w = 1).
// Synchronises `st` (the counts return to the host).
int grow_nodes(const float4 *pts, uint32_t n, float node_radius, DeviceBlocks &mem, cudaStream_t st, float4 **nodes,
               uint32_t *kept) {
    const float voxel = 0.7f * node_radius;
    // n + 1 entries: a spare value buffer later takes the scan of the kept flags and its total.
    uint32_t *keys = mem.get<uint32_t>(4ull * (n + 1)), *vals = mem.get<uint32_t>(4ull * (n + 1));
    uint32_t *keys2 = mem.get<uint32_t>(4ull * (n + 1)), *vals2 = mem.get<uint32_t>(4ull * (n + 1));
    uint32_t *heads = mem.get<uint32_t>(4ull * (n + 1));
    uint32_t *tmp = mem.get<uint32_t>(4ull * (n / ws::kScanTile + 4));
    uint32_t *hist = mem.get<uint32_t>(4ull * 256 * ws::sort_max_tiles(n));
    uint32_t *digit = mem.get<uint32_t>(4ull * 256);
    float4 *cand = mem.get<float4>(16ull * n);
    int *err = mem.get<int>(4);
    if (mem.err != cudaSuccess) return WS_ERR_CUDA;
    uint32_t nv = 0;
    {
        ws::k_voxel_key<<<ws::grid_of(n, 256), 256, 0, st>>>(pts, n, voxel, keys, vals);
        const bool alt = ws::radix_sort<uint32_t>(keys, vals, keys2, vals2, nullptr, n, n, 30, hist, digit, st);
        const uint32_t *sk = alt ? keys2 : keys, *sv = alt ? vals2 : vals;
        ws::k_voxel_marks<<<ws::grid_of(n, 256), 256, 0, st>>>(sk, n, heads);
        ws::exclusive_scan(heads, heads, nullptr, n, n, tmp, st);
        ws::k_voxel_sample<<<ws::grid_of(n, 256), 256, 0, st>>>(sk, sv, heads, n, pts, voxel, cand);
        if (cudaMemcpyAsync(&nv, heads + n, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) return WS_ERR_CUDA;
        if (cudaStreamSynchronize(st) != cudaSuccess) return WS_ERR_CUDA;
    }
    *nodes = mem.get<float4>(16ull * nv);
    if (mem.err != cudaSuccess) return WS_ERR_CUDA;
    *kept = 0;
    if (nv == 0) return WS_OK;
    // The host loop's constants, in the same float arithmetic.
    const float r = 0.85f * node_radius;
    const float thr = r * r;
    const float inv_cell = 1.0f / (ws::kDedupCellScale * r);
    uint32_t *cnt = heads;   // free again: the candidates are written
    uint32_t total = 0;
    int flag = 0;
    const uint32_t *ck = nullptr, *ci = nullptr;
    uint32_t *spare_keys = nullptr, *spare_vals = nullptr;
    {
        if (cudaMemsetAsync(err, 0, 4, st) != cudaSuccess) return WS_ERR_CUDA;
        ws::k_dedup_keys<<<ws::grid_of(nv, 256), 256, 0, st>>>(cand, nv, inv_cell, keys, vals, err);
        const bool alt = ws::radix_sort<uint32_t>(keys, vals, keys2, vals2, nullptr, nv, nv, 30, hist, digit, st);
        ck = alt ? keys2 : keys;
        ci = alt ? vals2 : vals;
        spare_keys = alt ? keys : keys2;
        spare_vals = alt ? vals : vals2;
        ws::k_dedup_neighbours<false><<<ws::grid_of(nv, 128), 128, 0, st>>>(cand, ck, ci, nv, inv_cell, thr, cnt, nullptr);
        ws::exclusive_scan(cnt, cnt, nullptr, nv, nv, tmp, st);
        if (cudaMemcpyAsync(&total, cnt + nv, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(&flag, err, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return WS_ERR_CUDA;
        // AppendNodeFromVertexHost stops on a NaN candidate (LOG(FATAL)).
        if (flag & 1) return WS_ERR_INVALID_ARGUMENT;
    }
    uint32_t *nbr = mem.get<uint32_t>(4ull * total);
    if (mem.err != cudaSuccess) return WS_ERR_CUDA;
    ws::k_dedup_neighbours<true><<<ws::grid_of(nv, 128), 128, 0, st>>>(cand, ck, ci, nv, inv_cell, thr, cnt, nbr);
    uint8_t *decision = reinterpret_cast<uint8_t *>(spare_keys);
    if (nv <= ws::kDedupOneBlockMax) {   // 16 KB of shared memory at most
        ws::k_dedup_greedy<<<1, ws::kDedupThreads, nv, st>>>(cnt, nbr, nv, decision, err);
    } else {
        unsigned *sync = mem.get<unsigned>(16);
        int dev = 0, sms = 0, per_sm = 0, coop = 0;
        if (mem.err != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ws::k_dedup_greedy_grid, ws::kDedupGridThreads, 0) !=
                cudaSuccess ||
            per_sm < 1)
            return WS_ERR_CUDA;
        const long long want = ((long long)nv + ws::kDedupGridThreads - 1) / ws::kDedupGridThreads;
        const int grid = (int)std::min<long long>(want, (long long)per_sm * sms);
        if (cudaMemsetAsync(decision, 0, nv, st) != cudaSuccess || cudaMemsetAsync(sync, 0, 16, st) != cudaSuccess)
            return WS_ERR_CUDA;
        const uint32_t *nbr_ptr = cnt;
        uint32_t nv_arg = nv;
        void *args[] = {(void *)&nbr_ptr, (void *)&nbr, (void *)&nv_arg, (void *)&decision, (void *)&sync, (void *)&err};
        if (cudaLaunchCooperativeKernel((const void *)ws::k_dedup_greedy_grid, dim3(grid), dim3(ws::kDedupGridThreads),
                                        args, 0, st) != cudaSuccess) {
            cudaGetLastError();   // a refused launch leaves no sticky error for later checks
            return WS_ERR_CUDA;
        }
    }
    uint32_t *pos = spare_vals;
    ws::k_dedup_flags<<<ws::grid_of(nv, 256), 256, 0, st>>>(decision, nv, pos);
    ws::exclusive_scan(pos, pos, nullptr, nv, nv, tmp, st);
    ws::k_dedup_emit<<<ws::grid_of(nv, 256), 256, 0, st>>>(cand, decision, pos, nv, *nodes);
    if (cudaGetLastError() != cudaSuccess) return WS_ERR_CUDA;
    uint32_t count = 0;
    if (cudaMemcpyAsync(&count, pos + nv, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&flag, err, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return WS_ERR_CUDA;
    if (flag & 4) return WS_ERR_TIMEOUT;
    if (flag & 2) return WS_ERR_CUDA;
    *kept = count;
    return WS_OK;
}

}  // namespace


extern "C" {

int ws_init_nodes(const float *surfels, int n, float node_radius, float *nodes_host, int cap, int *num_nodes,
                  void *stream) {
    if (!surfels || n <= 0 || !nodes_host || !num_nodes || cap < 2 || !(node_radius > 0.f))
        return WS_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DeviceBlocks mem(st);
    float4 *nodes = nullptr;
    uint32_t kept = 0;
    const int rc = grow_nodes(reinterpret_cast<const float4 *>(surfels), (uint32_t)n, node_radius, mem, st, &nodes, &kept);
    if (rc != WS_OK) return rc;
    // InitializeNodeGraphFromVertex (NodeGraph.cu:479-486): two anchors at the origin come first.
    const float anchors[8] = {0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f};
    const long long total = (long long)kept + 2;
    *num_nodes = (int)std::min<long long>(total, INT_MAX);
    if (total > cap) return WS_ERR_CAPACITY;
    std::memcpy(nodes_host, anchors, sizeof(anchors));
    if (kept && cudaMemcpyAsync(nodes_host + 8, nodes, 16ull * kept, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return WS_ERR_CUDA;
    return cudaStreamSynchronize(st) == cudaSuccess ? WS_OK : WS_ERR_CUDA;
}

int ws_expand_nodes(const float *vertices, int num_vertices, float node_radius, float *reference_nodes,
                    float *live_nodes, unsigned *node_time, unsigned current_time, int cap, int *num_nodes,
                    void *stream) {
    if (!num_nodes || !reference_nodes || num_vertices < 0 || !(node_radius > 0.f) || *num_nodes < 0 ||
        cap < *num_nodes)
        return WS_ERR_INVALID_ARGUMENT;
    // NaiveExpandNodeGraphFromVertexUnsupported (NodeGraph.cu:500-510): nothing to add.
    if (num_vertices == 0) return WS_OK;
    if (!vertices) return WS_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DeviceBlocks mem(st);
    float4 *nodes = nullptr;
    uint32_t kept = 0;
    const int rc =
        grow_nodes(reinterpret_cast<const float4 *>(vertices), (uint32_t)num_vertices, node_radius, mem, st, &nodes, &kept);
    if (rc != WS_OK) return rc;
    const long long before = *num_nodes, total = before + kept;
    if (total > cap) {
        *num_nodes = (int)std::min<long long>(total, INT_MAX);
        return WS_ERR_CAPACITY;
    }
    if (kept) {
        const size_t bytes = 16ull * kept;
        if (cudaMemcpyAsync(reference_nodes + 4 * before, nodes, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return WS_ERR_CUDA;
        if (live_nodes && live_nodes != reference_nodes &&
            cudaMemcpyAsync(live_nodes + 4 * before, nodes, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return WS_ERR_CUDA;
        // updateAppendNodeInitialTime (NodeGraph.cu:316-337)
        if (node_time) {
            ws::k_fill_u32<<<ws::grid_of(kept, 256), 256, 0, st>>>(node_time + before, kept, current_time);
            if (cudaGetLastError() != cudaSuccess) return WS_ERR_CUDA;
        }
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return WS_ERR_CUDA;
    *num_nodes = (int)total;
    return WS_OK;
}

int ws_build_node_graph_ex(const float *nodes, const uint32_t *node_status, int n, int k, float node_radius,
                           int normalize_weights, uint16_t *knn, float *w, uint16_t *edges, void *stream) {
    if (!nodes || n <= 0 || n > 65535 || !knn || !w || !edges || (k != 4 && k != 8)) return WS_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float r2 = node_radius * node_radius;
    const int runs = (n + ws::kGraphRun - 1) / ws::kGraphRun;
    // Run boxes from the stream-ordered pool: the call stays asynchronous.
    float4 *boxes = nullptr;
    if (cudaMallocAsync(reinterpret_cast<void **>(&boxes), 32ull * runs, st) != cudaSuccess) return WS_ERR_CUDA;
    const float4 *nd = reinterpret_cast<const float4 *>(nodes);
    const uint2 *status = reinterpret_cast<const uint2 *>(node_status);
    const int norm = normalize_weights ? 1 : 0;
    ws::k_node_boxes<<<ws::grid_of(runs, 128), 128, 0, st>>>(nd, n, boxes, boxes + runs);
    const int threads = 64;
    const int grid = (n + threads - 1) / threads;
    if (k == 4)
        ws::k_node_graph<4><<<grid, threads, 0, st>>>(nd, status, n, r2, norm, boxes, boxes + runs, knn, w, edges);
    else
        ws::k_node_graph<8><<<grid, threads, 0, st>>>(nd, status, n, r2, norm, boxes, boxes + runs, knn, w, edges);
    const cudaError_t launched = cudaGetLastError();
    const cudaError_t freed = cudaFreeAsync(boxes, st);
    return launched == cudaSuccess && freed == cudaSuccess ? WS_OK : WS_ERR_CUDA;
}

int ws_build_node_graph(const float *nodes, int n, int k, float node_radius, uint16_t *knn, float *w, uint16_t *edges,
                        void *stream) {
    return ws_build_node_graph_ex(nodes, nullptr, n, k, node_radius, 1, knn, w, edges, stream);
}

int ws_skinning_incremental(const float *nodes, const uint32_t *node_status, int num_nodes, int num_prev_nodes,
                            const float *verts, int num_verts, int num_remaining_surfels, float node_radius,
                            int normalize_weights, uint16_t *knn, float *sw, float *cw, void *stream) {
    if (!nodes || num_nodes <= 0 || num_nodes > 65535 || !verts || num_verts < 0 || !knn || !sw || !cw ||
        num_prev_nodes < 0 || num_prev_nodes > num_nodes || num_remaining_surfels < 0 ||
        num_remaining_surfels > num_verts)
        return WS_ERR_INVALID_ARGUMENT;
    const int count = num_verts - num_remaining_surfels;
    if (count == 0) return WS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float r2 = node_radius * node_radius;
    ws::k_skinning<<<(count + 255) / 256, 256, 0, st>>>(
        reinterpret_cast<const float4 *>(nodes), reinterpret_cast<const uint2 *>(node_status), num_nodes,
        num_prev_nodes, reinterpret_cast<const float4 *>(verts), num_remaining_surfels, num_verts, r2,
        normalize_weights ? 1 : 0, reinterpret_cast<ushort4 *>(knn), reinterpret_cast<float4 *>(sw),
        reinterpret_cast<float4 *>(cw));
    return cudaGetLastError() == cudaSuccess ? WS_OK : WS_ERR_CUDA;
}

int ws_skinning_ex(const float *nodes, const uint32_t *node_status, int num_nodes, const float *verts, int num_verts,
                   float node_radius, int normalize_weights, uint16_t *knn, float *sw, float *cw, void *stream) {
    return ws_skinning_incremental(nodes, node_status, num_nodes, 0, verts, num_verts, 0, node_radius,
                                   normalize_weights, knn, sw, cw, stream);
}

int ws_skinning(const float *nodes, int n_nodes, const float *verts, int n_verts, float node_radius, uint16_t *knn,
                float *sw, float *cw, void *stream) {
    return ws_skinning_ex(nodes, nullptr, n_nodes, verts, n_verts, node_radius, 1, knn, sw, cw, stream);
}

int ws_forward_warp(const float *se3, int num_nodes, const float *verts, const float *normals, int n,
                    const uint16_t *knn, const float *sw, const float *cw, float *out_v, float *out_n, void *stream) {
    if (!se3 || num_nodes <= 0 || num_nodes > 65535 || !verts || n < 0 || !knn || !sw || !cw || !out_v)
        return WS_ERR_INVALID_ARGUMENT;
    if (n == 0) return WS_OK;
    ws::k_forward_warp<<<ws::grid_of(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        se3, num_nodes, reinterpret_cast<const float4 *>(verts), reinterpret_cast<const float4 *>(normals), n,
        reinterpret_cast<const ushort4 *>(knn), reinterpret_cast<const float4 *>(sw),
        reinterpret_cast<const float4 *>(cw), reinterpret_cast<float4 *>(out_v), reinterpret_cast<float4 *>(out_n));
    return cudaGetLastError() == cudaSuccess ? WS_OK : WS_ERR_CUDA;
}

int ws_splat_maps(const float *verts, const float *attr_verts, const float *attr_normals, int n, int W, int H, float fx,
                  float fy, float cx, float cy, int footprint, uint32_t *index_map, float *vertex_map,
                  float *normal_map, void *stream) {
    if (!verts || n < 0 || W <= 0 || H <= 0 || !index_map || footprint < 0 || footprint > 8)
        return WS_ERR_INVALID_ARGUMENT;
    if ((vertex_map && !attr_verts) || (normal_map && !attr_normals)) return WS_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned long long *zbuf = nullptr;
    const size_t npix = (size_t)W * H;
    if (cudaMallocAsync(&zbuf, 8 * npix, st) != cudaSuccess) return WS_ERR_CUDA;
    if (cudaMemsetAsync(zbuf, 0xff, 8 * npix, st) != cudaSuccess) {
        cudaFreeAsync(zbuf, st);
        return WS_ERR_CUDA;
    }
    if (n > 0)
        ws::k_splat<<<ws::grid_of(n, 256), 256, 0, st>>>(reinterpret_cast<const float4 *>(verts), n, W, H, fx, fy, cx,
                                                         cy, footprint, zbuf);
    ws::k_splat_resolve<<<ws::grid_of((long long)npix, 256), 256, 0, st>>>(
        zbuf, (int)npix, reinterpret_cast<const float4 *>(attr_verts), reinterpret_cast<const float4 *>(attr_normals),
        index_map, reinterpret_cast<float4 *>(vertex_map), reinterpret_cast<float4 *>(normal_map));
    cudaFreeAsync(zbuf, st);
    return cudaGetLastError() == cudaSuccess ? WS_OK : WS_ERR_CUDA;
}

int ws_splat_maps_noalloc(const float *verts, const float *attr_verts, const float *attr_normals, int n, int W,
                          int H, float fx, float fy, float cx, float cy, int footprint, uint32_t *index_map,
                          float *vertex_map, float *normal_map, void *stream) {
    if (!verts || n < 0 || W <= 0 || H <= 0 || !index_map || footprint < 0 || footprint > 8)
        return WS_ERR_INVALID_ARGUMENT;
    if ((vertex_map && !attr_verts) || (normal_map && !attr_normals)) return WS_ERR_INVALID_ARGUMENT;
    if ((long long)W * H > WS_NOALLOC_MAX_PIXELS) return WS_ERR_CAPACITY;
    unsigned long long *zbuf = nullptr;
    const int st_scratch = noalloc_scratch(&zbuf);
    if (st_scratch != WS_OK) return st_scratch;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t npix = (size_t)W * H;
    // the array keeps the previous call's keys: clear the part this call uses
    if (cudaMemsetAsync(zbuf, 0xff, 8 * npix, st) != cudaSuccess) return WS_ERR_CUDA;
    if (n > 0)
        ws::k_splat<<<ws::grid_of(n, 256), 256, 0, st>>>(reinterpret_cast<const float4 *>(verts), n, W, H, fx, fy, cx,
                                                         cy, footprint, zbuf);
    ws::k_splat_resolve<<<ws::grid_of((long long)npix, 256), 256, 0, st>>>(
        zbuf, (int)npix, reinterpret_cast<const float4 *>(attr_verts), reinterpret_cast<const float4 *>(attr_normals),
        index_map, reinterpret_cast<float4 *>(vertex_map), reinterpret_cast<float4 *>(normal_map));
    return cudaGetLastError() == cudaSuccess ? WS_OK : WS_ERR_CUDA;
}

int ws_render_solver_maps(const float *vertex_confid, const float *normal_radius, const float *color_time,
                          int num_surfels, const ws_render_params *params, uint32_t *index_map, float *vertex_map,
                          float *normal_map, float *rgbd_map, void *stream) {
    if (!params || !vertex_confid || num_surfels < 0 || !index_map) return WS_ERR_INVALID_ARGUMENT;
    const ws_render_params &p = *params;
    if (p.width <= 0 || p.height <= 0 || p.footprint < 0 || p.footprint > 8 || !(p.max_depth > 0.f))
        return WS_ERR_INVALID_ARGUMENT;
    if (normal_map && !normal_radius) return WS_ERR_INVALID_ARGUMENT;
    ws::RenderArgs a;
    a.W = p.width; a.H = p.height; a.fp = p.footprint;
    a.fx = p.fx; a.fy = p.fy; a.cx = p.cx; a.cy = p.cy;
    a.max_depth = p.max_depth; a.current_time = p.current_time;
    a.conf_threshold = p.confidence_threshold; a.time_threshold = p.time_threshold;
    for (int q = 0; q < 12; ++q) a.m[q] = p.world2camera[q];
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t npix = (size_t)p.width * p.height;
    unsigned long long *zbuf = nullptr;
    if (cudaMallocAsync(&zbuf, 8 * npix, st) != cudaSuccess) return WS_ERR_CUDA;
    if (cudaMemsetAsync(zbuf, 0xff, 8 * npix, st) != cudaSuccess) {
        cudaFreeAsync(zbuf, st);
        return WS_ERR_CUDA;
    }
    const float4 *vc = reinterpret_cast<const float4 *>(vertex_confid);
    const float4 *ct = reinterpret_cast<const float4 *>(color_time);
    if (num_surfels > 0) ws::k_render_keys<<<ws::grid_of(num_surfels, 256), 256, 0, st>>>(vc, ct, num_surfels, a, zbuf);
    ws::k_render_resolve<<<ws::grid_of((long long)npix, 256), 256, 0, st>>>(
        zbuf, (int)npix, vc, reinterpret_cast<const float4 *>(normal_radius), ct, index_map,
        reinterpret_cast<float4 *>(vertex_map), reinterpret_cast<float4 *>(normal_map), reinterpret_cast<float4 *>(rgbd_map));
    cudaFreeAsync(zbuf, st);
    return cudaGetLastError() == cudaSuccess ? WS_OK : WS_ERR_CUDA;
}


int ws_render_observation_maps(const float *vertex_confid, const float *normal_radius, const float *color_time,
                               int num_surfels, const ws_render_params *params, uint32_t *index_map, float *rgbd_map,
                               void *stream) {
    if (!params || !vertex_confid || !normal_radius || num_surfels < 0 || !index_map) return WS_ERR_INVALID_ARGUMENT;
    const ws_render_params &p = *params;
    if (p.width <= 0 || p.height <= 0 || !(p.max_depth > 0.f)) return WS_ERR_INVALID_ARGUMENT;
    ws::RenderArgs a;
    a.W = p.width; a.H = p.height; a.fp = 0;
    a.fx = p.fx; a.fy = p.fy; a.cx = p.cx; a.cy = p.cy;
    a.max_depth = p.max_depth; a.current_time = p.current_time;
    a.conf_threshold = p.confidence_threshold; a.time_threshold = p.time_threshold;
    for (int q = 0; q < 12; ++q) a.m[q] = p.world2camera[q];
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t npix = (size_t)p.width * p.height;
    unsigned long long *zbuf = nullptr;
    if (cudaMallocAsync(&zbuf, 8 * npix, st) != cudaSuccess) return WS_ERR_CUDA;
    if (cudaMemsetAsync(zbuf, 0xff, 8 * npix, st) != cudaSuccess) {
        cudaFreeAsync(zbuf, st);
        return WS_ERR_CUDA;
    }
    const float4 *ct = reinterpret_cast<const float4 *>(color_time);
    if (num_surfels > 0)
        ws::k_obs_keys<<<ws::grid_of(num_surfels, 256), 256, 0, st>>>(
            reinterpret_cast<const float4 *>(vertex_confid), reinterpret_cast<const float4 *>(normal_radius), ct,
            num_surfels, a, zbuf);
    ws::k_obs_resolve<<<ws::grid_of((long long)npix, 256), 256, 0, st>>>(zbuf, (int)npix, ct, index_map,
                                                                          reinterpret_cast<float4 *>(rgbd_map));
    cudaFreeAsync(zbuf, st);
    return cudaGetLastError() == cudaSuccess ? WS_OK : WS_ERR_CUDA;
}

}  // extern "C"
