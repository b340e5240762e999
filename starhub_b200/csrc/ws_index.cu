// Index build of the B200 warp-field solver: pixel-term compaction,
// node->term and node-pair->term maps, and the block-CSR sparsity pattern.
//
// All scenes of a batch are processed by the same launches; per-scene counts
// live in device memory (Plan), so nothing here waits on the host.
#include <cuda_runtime.h>

#include <algorithm>

#include "ws_common.cuh"
#include "ws_prims.cuh"
#include "ws_workspace.h"

namespace ws {

constexpr int kPixTileThreads = 256;
constexpr int kPixPerThread = 4;
constexpr int kPixTile = kPixTileThreads * kPixPerThread;   // 1024 pixels per tile

__device__ __forceinline__ void set_error(int *flag, int code) { atomicCAS(flag, 0, code); }

// markPotentialValidImageTermPixelKernel (examples/mono_star/opt/ImageTermKNNFetcher.cu:9-29):
// a pixel is a potential term iff its index map holds a surfel id.
// A pixel counts only when its surfel id is in range (out-of-range ids are treated as empty,
// which keeps every later gather inside the caller's arrays).
__device__ __forceinline__ bool valid_surfel(uint32_t id, const Scene &sc) {
    return id != kInvalidIndex && id < (uint32_t)sc.num_surfels;
}

__global__ void k_pixel_count(const Scene *scenes, const uint32_t *tile_scene, int num_tiles, uint32_t *tile_count) {
    __shared__ uint32_t sm[32];
    const int t = blockIdx.x;
    if (t >= num_tiles) return;
    const Scene &sc = scenes[tile_scene[t]];
    const uint32_t npix = (uint32_t)sc.width * (uint32_t)sc.height;
    const uint32_t p0 = (uint32_t)(t - sc.tile_base) * kPixTile + threadIdx.x * kPixPerThread;
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < kPixPerThread; ++i) {
        const uint32_t p = p0 + i;
        if (p < npix) {
            const uint32_t y = p / (uint32_t)sc.width, x = p - y * (uint32_t)sc.width;
            c += valid_surfel(sc.index_map[(size_t)y * sc.pitch + x], sc) ? 1u : 0u;
        }
    }
    uint32_t total;
    block_excl_scan_u32(c, &total, sm);
    if (threadIdx.x == 0) tile_count[t] = total;
}

// compactPontentialImageTermPixelsKernel (ImageTermKNNFetcher.cu:56-88) fused with
// queryPixelKNNKernel (WarpSolver.cu:7-47): raster-order compaction of
// (x, y, x + flow_x, y + flow_y) and the surfel's 4-NN and weights.
__global__ void k_pixel_compact(const Scene *scenes, const uint32_t *tile_scene, int num_tiles,
                                const uint32_t *tile_offset, ushort4 *pixels, ushort4 *knn,
                                float4 *sw, float4 *cw, uint32_t *term_scene, uint32_t cap, int *err) {
    __shared__ uint32_t sm[32];
    const int t = blockIdx.x;
    if (t >= num_tiles) return;
    const uint32_t s = tile_scene[t];
    const Scene &sc = scenes[s];
    const uint32_t npix = (uint32_t)sc.width * (uint32_t)sc.height;
    const uint32_t p0 = (uint32_t)(t - sc.tile_base) * kPixTile + threadIdx.x * kPixPerThread;
    uint32_t ids[kPixPerThread];
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < kPixPerThread; ++i) {
        const uint32_t p = p0 + i;
        ids[i] = kInvalidIndex;
        if (p < npix) {
            const uint32_t y = p / (uint32_t)sc.width, x = p - y * (uint32_t)sc.width;
            ids[i] = sc.index_map[(size_t)y * sc.pitch + x];
            if (!valid_surfel(ids[i], sc)) ids[i] = kInvalidIndex;
            c += (ids[i] != kInvalidIndex) ? 1u : 0u;
        }
    }
    uint32_t pos = tile_offset[t] + block_excl_scan_u32(c, nullptr, sm);
#pragma unroll
    for (int i = 0; i < kPixPerThread; ++i) {
        if (ids[i] == kInvalidIndex) continue;
        const uint32_t p = p0 + i;
        const uint32_t y = p / (uint32_t)sc.width, x = p - y * (uint32_t)sc.width;
        float2 fl = make_float2(0.f, 0.f);
        if (sc.flow) fl = sc.flow[(size_t)y * sc.pitch + x];
        const unsigned tx = __float2uint_rn(fl.x + float(x));
        const unsigned ty = __float2uint_rn(fl.y + float(y));
        if (pos < cap) {
            pixels[pos] = make_ushort4((unsigned short)x, (unsigned short)y, (unsigned short)tx, (unsigned short)ty);
            ushort4 k4 = sc.surfel_knn[ids[i]];
            const unsigned nn = (unsigned)sc.num_nodes;
            if (k4.x >= nn || k4.y >= nn || k4.z >= nn || k4.w >= nn) {   // node id out of range
                set_error(err, WS_ERR_INVALID_ARGUMENT);
                k4 = make_ushort4(0, 0, 0, 0);
            }
            knn[pos] = k4;
            sw[pos] = sc.surfel_sw[ids[i]];
            cw[pos] = sc.surfel_cw[ids[i]];
            term_scene[pos] = s;
        }
        ++pos;
    }
}

// Per-scene counts and key/value ranges (term_offset_types.h:62-82 size2offset),
// computed after the compaction scan.
__global__ void k_plan(const Scene *scenes, int num_scenes, const uint32_t *tile_offset, int total_tiles,
                       Plan *plan, uint32_t *counts, uint32_t cap_n2t, uint32_t cap_pair, int *err) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t n2t = 0, pair = 0;
    for (int s = 0; s < num_scenes; ++s) {
        const Scene &sc = scenes[s];
        Plan p;
        p.dense_begin = tile_offset[sc.tile_base];
        p.dense_count = tile_offset[sc.tile_base + sc.num_tiles] - p.dense_begin;
        p.n2t_base = n2t;
        p.n2t_count = 4u * p.dense_count + 2u * sc.num_edges + sc.num_nodes + 4u * sc.num_features;
        p.pair_base = pair;
        p.pair_count = 6u * p.dense_count + sc.num_edges + 6u * sc.num_features;
        p.pad[0] = p.pad[1] = 0;
        n2t += p.n2t_count;
        pair += p.pair_count;
        plan[s] = p;
    }
    if (n2t > cap_n2t || pair > cap_pair) {
        set_error(err, WS_ERR_CAPACITY);
        n2t = min(n2t, cap_n2t);
        pair = min(pair, cap_pair);
    }
    counts[kCntDense] = tile_offset[total_tiles];
    counts[kCntN2T] = n2t;
    counts[kCntPairKV] = pair;
}

// Node-graph edge endpoints clamped into the scene (an out-of-range id flags WS_ERR_INVALID_ARGUMENT).
__device__ __forceinline__ void edge_ends(const Scene &sc, uint32_t e, uint16_t &x, uint16_t &y, int *err) {
    x = sc.edges[3 * e];
    y = sc.edges[3 * e + 1];
    const uint16_t last = (uint16_t)(sc.num_nodes - 1);
    if (x > last || y > last) {
        set_error(err, WS_ERR_INVALID_ARGUMENT);
        x = min(x, last);
        y = min(y, last);
    }
}

__device__ __forceinline__ ushort4 clamp_knn(ushort4 k, const Scene &sc, int *err) {
    const uint16_t last = (uint16_t)(sc.num_nodes - 1);
    if (k.x > last || k.y > last || k.z > last || k.w > last) {
        set_error(err, WS_ERR_INVALID_ARGUMENT);
        k = make_ushort4(min(k.x, last), min(k.y, last), min(k.z, last), min(k.w, last));
    }
    return k;
}


// Node->term keys and values (buildTermKeyValueKernel, examples/mono_star/opt/Node2TermsIndex.cu:6-76):
// keys are global node ids, values are the scene-local term ids of the reference's term space
// [dense | reg | node-motion | feature]; self edges get the invalid key.  Per scene the entries
// sit at plan.n2t_base as [4 per dense term | 2 per edge | 1 per node | 4 per feature].  One
// thread per dense term writes that term's 4 entries (its scene from the compaction), and
// one block row per scene writes the scene's other entries, so no entry searches for its scene.
__global__ void k_n2t_kv_dense(const Scene *scenes, const Plan *plan, const uint32_t *counts,
                               const uint32_t *term_scene, const ushort4 *dense_knn, uint32_t *keys, uint32_t *vals) {
    const uint32_t n = counts[kCntDense];
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t s = term_scene[t];
        const Plan &p = plan[s];
        const uint32_t lt = t - p.dense_begin, base = p.n2t_base + 4u * lt, nb = scenes[s].node_base;
        const ushort4 k4 = dense_knn[t];
        keys[base] = nb + k4.x;
        keys[base + 1] = nb + k4.y;
        keys[base + 2] = nb + k4.z;
        keys[base + 3] = nb + k4.w;
        vals[base] = vals[base + 1] = vals[base + 2] = vals[base + 3] = lt;
    }
}

__global__ void k_n2t_kv_tail(const Scene *scenes, const Plan *plan, uint32_t *keys, uint32_t *vals,
                              uint32_t invalid_key, int *err) {
    const Scene &sc = scenes[blockIdx.y];
    const Plan &p = plan[blockIdx.y];
    const uint32_t nd = p.dense_count, ne = sc.num_edges, nn = sc.num_nodes, nf = sc.num_features;
    const uint32_t len = 2u * ne + nn + 4u * nf, base = p.n2t_base + 4u * nd;
    for (uint32_t j0 = blockIdx.x * blockDim.x + threadIdx.x; j0 < len; j0 += gridDim.x * blockDim.x) {
        uint32_t j = j0, key, val;
        if (j < 2u * ne) {
            const uint32_t e = j >> 1;
            uint16_t x, y;
            edge_ends(sc, e, x, y, err);
            key = (x != y) ? sc.node_base + ((j & 1u) ? y : x) : invalid_key;
            val = nd + e;
        } else if ((j -= 2u * ne) < nn) {
            key = sc.node_base + j;
            val = nd + ne + j;
        } else {
            j -= nn;
            const uint32_t f = j >> 2;
            const ushort4 k4 = clamp_knn(sc.feature_knn[f], sc, err);
            const uint32_t slot = j & 3u;
            const uint16_t id = slot == 0 ? k4.x : slot == 1 ? k4.y : slot == 2 ? k4.z : k4.w;
            key = sc.node_base + id;
            val = nd + ne + nn + f;
        }
        keys[base + j0] = key;
        vals[base + j0] = val;
    }
}

// computeTermOffsetKernel (Node2TermsIndex.cu:78-121) as a lower bound per node.
__global__ void k_n2t_offsets(const uint32_t *sorted_keys, const uint32_t *counts, uint32_t total_nodes,
                              uint32_t *offsets) {
    const uint32_t n = counts[kCntN2T];
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g <= total_nodes; g += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = n;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sorted_keys[mid] < g) lo = mid + 1; else hi = mid;
        }
        offsets[g] = lo;
    }
}

// ---------------------------------------------------------------------------
// Node pair -> term map (computeKVNodePairKNN + sort + segmentNodePairKernel +
// compactNodePairKeyKernel, NodePair2TermsIndex.cu:11-169), built row by row from the sorted
// node -> term map instead of by sorting one key per (pair, term).
// The reference's sorted list holds, for a pair i < j, one entry of term t for every way t
// touches both nodes: for a dense or feature term, each knn slot holding i times each slot holding
// j (slot pairs with id_a < id_b); for a non-self edge (i, j) or (j, i), one entry; in term order.
// Row i's node -> term list holds t once per slot of i, in term order, so emitting, for each entry
// of the list, the term's nodes above i (every knn slot above i; the other end of an edge) yields
// exactly row i's entries, each pair's in term order.  The pairs are sorted by (row, column), so
// row i's pairs and entries are one contiguous range after those of the rows before it.
// Pass 1 (one warp per row) counts each column's entries in a small hash table in shared memory
// and keeps the row's columns sorted; two scans give every row its first pair and first entry;
// pass 2 writes the pairs and places every entry at its pair's next free position.
// ---------------------------------------------------------------------------
constexpr int kRowHash = 128;        // hash slots per warp (twice kRowPairsMax)
constexpr int kRowWarps = 4;         // warps per block of the two row passes
constexpr int kRowLanesEntries = 4;  // list entries per lane and pass (loads in flight)
constexpr int kRowChunk = 32 * kRowLanesEntries;   // list entries per pass
constexpr int kRowStage = 3 * kRowChunk;           // their candidates (at most 3 each)

constexpr uint32_t kNoCol = 0xFFFFFFFFu;

// The columns above `row` that list entry `t` (scene-local term id) adds to row `row`'s pairs, in
// c[0..2] (kNoCol where none); returns their number (at most 3).
__device__ __forceinline__ int row_pair_columns(const Scene &sc, const Plan &p, const ushort4 *dense_knn,
                                                uint32_t row, uint32_t t, uint32_t (&c)[3], int *err) {
    const uint32_t nb = (uint32_t)sc.node_base, nd = p.dense_count, ne = (uint32_t)sc.num_edges,
                   nn = (uint32_t)sc.num_nodes;
    c[0] = c[1] = c[2] = kNoCol;
    int n = 0;
    auto push = [&](uint32_t v) {
        c[0] = n == 0 ? v : c[0];
        c[1] = n == 1 ? v : c[1];
        c[2] = n == 2 ? v : c[2];
        n = min(n + 1, 3);
    };
    if (t < nd || t >= nd + ne + nn) {   // dense or feature term: its knn slots above the row
        const ushort4 k4 = t < nd ? dense_knn[p.dense_begin + t] : clamp_knn(sc.feature_knn[t - nd - ne - nn], sc, err);
        if (nb + k4.x > row) push(nb + k4.x);
        if (nb + k4.y > row) push(nb + k4.y);
        if (nb + k4.z > row) push(nb + k4.z);
        if (nb + k4.w > row) push(nb + k4.w);
    } else if (t < nd + ne) {            // edge: its other end
        uint16_t x, y;
        edge_ends(sc, t - nd, x, y, err);
        const uint32_t other = (nb + x == row) ? nb + y : nb + x;
        if (x != y && other > row) push(other);
    }
    return n;
}

// Row `row`'s candidate columns of list entries base .. base + kRowChunk - 1 (below end), staged
// in list order as (column, term); returns their number.  Lane l reads entries base + 32 q + l, so
// every load instruction is coalesced and a lane has kRowLanesEntries gathers in flight.
__device__ __forceinline__ uint32_t stage_row_candidates(const Scene &sc, const Plan &p, const ushort4 *dense_knn,
                                                         const uint32_t *n2t_val, uint32_t row, uint32_t base,
                                                         uint32_t end, uint32_t *st_col, uint32_t *st_term, int lane,
                                                         int *err) {
    uint32_t t[kRowLanesEntries];
#pragma unroll
    for (int q = 0; q < kRowLanesEntries; ++q) {
        const uint32_t e = base + 32u * q + (uint32_t)lane;
        t[q] = e < end ? n2t_val[e] : kNoCol;
    }
    uint32_t carry = 0;
#pragma unroll
    for (int q = 0; q < kRowLanesEntries; ++q) {
        uint32_t col[3] = {kNoCol, kNoCol, kNoCol};
        const int n = t[q] != kNoCol ? row_pair_columns(sc, p, dense_knn, row, t[q], col, err) : 0;
        const uint32_t incl = warp_incl_scan_u32((uint32_t)n);
        const uint32_t off = carry + incl - (uint32_t)n;
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (k < n) {
                st_col[off + k] = col[k];
                st_term[off + k] = t[q];
            }
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    __syncwarp();
    return carry;
}

__device__ __forceinline__ uint32_t col_hash(uint32_t c) { return (c * 2654435761u) >> (32 - 7); }

__global__ void __launch_bounds__(32 * kRowWarps) k_pair_rows_count(
    const Scene *scenes, const Plan *plan, const uint32_t *node_scene, uint32_t total_nodes,
    const uint32_t *n2t_offset, const uint32_t *n2t_val, uint32_t cap_n2t, const ushort4 *dense_knn, uint32_t *row_cols,
    uint32_t *row_cnts, uint32_t *row_pairs, uint32_t *row_entries, int *err) {
    static_assert(kRowHash == 128, "col_hash gives 7 bits");
    __shared__ uint32_t hkey[kRowWarps][kRowHash], hcnt[kRowWarps][kRowHash];
    __shared__ uint32_t lcol[kRowWarps][kRowHash], lcnt[kRowWarps][kRowHash];
    __shared__ uint32_t st_col[kRowWarps][kRowStage], st_term[kRowWarps][kRowStage];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    uint32_t *keys = hkey[wib], *cnts = hcnt[wib];
    const unsigned lower = (1u << lane) - 1u;
    const uint32_t warps = gridDim.x * kRowWarps;
    for (uint32_t row = blockIdx.x * kRowWarps + wib; row < total_nodes; row += warps) {
        for (int k = lane; k < kRowHash; k += 32) {
            keys[k] = kNoCol;
            cnts[k] = 0;
        }
        __syncwarp();
        const uint32_t s = node_scene[row];
        const Scene &sc = scenes[s];
        const Plan &p = plan[s];
        const uint32_t beg = n2t_offset[row], end = n2t_offset[row + 1];
        if (lane == 0 && end > beg + kRowChunk) l2_prefetch_list(n2t_val, beg + kRowChunk, end, cap_n2t);
        bool full = false;
        for (uint32_t base = beg; base < end; base += kRowChunk) {
            const uint32_t total =
                stage_row_candidates(sc, p, dense_knn, n2t_val, row, base, end, st_col[wib], st_term[wib], lane, err);
            for (uint32_t v0 = 0; v0 < total; v0 += 32) {
                const uint32_t v = v0 + (uint32_t)lane;
                const uint32_t c = v < total ? st_col[wib][v] : kNoCol;
                const unsigned peers = __match_any_sync(0xffffffffu, c);
                if (c != kNoCol && (peers & lower) == 0) {   // one insertion per column and pass
                    uint32_t slot = col_hash(c);
                    bool placed = false;
                    for (int probe = 0; probe < kRowHash && !placed; ++probe) {
                        const uint32_t prev = atomicCAS(&keys[slot], kNoCol, c);
                        if (prev == kNoCol || prev == c) {
                            atomicAdd(&cnts[slot], (uint32_t)__popc(peers));
                            placed = true;
                        }
                        slot = (slot + 1) & (kRowHash - 1);
                    }
                    if (!placed) full = true;
                }
            }
            __syncwarp();
        }
        // the table's columns, compacted in slot order, then ranked by column
        uint32_t n_cols = 0;
        for (int q = 0; q < kRowHash / 32; ++q) {
            const uint32_t c = keys[32 * q + lane];
            const unsigned occ = __ballot_sync(0xffffffffu, c != kNoCol);
            if (c != kNoCol) {
                const uint32_t idx = n_cols + (uint32_t)__popc(occ & lower);
                lcol[wib][idx] = c;
                lcnt[wib][idx] = cnts[32 * q + lane];
            }
            n_cols += (uint32_t)__popc(occ);
        }
        __syncwarp();
        full = __any_sync(0xffffffffu, full) || n_cols > (uint32_t)kRowPairsMax;
        if (full) {
            if (lane == 0) set_error(err, WS_ERR_CAPACITY);
            n_cols = 0;
        }
        uint32_t entries = 0;
        for (uint32_t x = (uint32_t)lane; x < n_cols; x += 32) {
            const uint32_t c = lcol[wib][x];
            uint32_t rank = 0;
            for (uint32_t y = 0; y < n_cols; ++y) rank += lcol[wib][y] < c ? 1u : 0u;
            row_cols[(size_t)kRowPairsMax * row + rank] = c;
            row_cnts[(size_t)kRowPairsMax * row + rank] = lcnt[wib][x];
            entries += lcnt[wib][x];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) entries += __shfl_xor_sync(0xffffffffu, entries, o);
        if (lane == 0) {
            row_pairs[row] = n_cols;
            row_entries[row] = full ? 0u : entries;
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(32 * kRowWarps) k_pair_rows_fill(
    const Scene *scenes, const Plan *plan, const uint32_t *node_scene, uint32_t total_nodes,
    const uint32_t *n2t_offset, const uint32_t *n2t_val, uint32_t cap_n2t, const ushort4 *dense_knn, const uint32_t *row_cols,
    const uint32_t *row_cnts, const uint32_t *pair_first, const uint32_t *entry_first, uint32_t cap_half,
    uint32_t cap_kv, uint32_t *half_row, uint32_t *half_col, uint32_t *half_begin, uint32_t *half_end,
    uint32_t *half_scene, uint32_t *row_cnt_lo, uint32_t *pair_val, uint32_t *counts, int *err) {
    __shared__ uint32_t s_col[kRowWarps][kRowPairsMax], s_next[kRowWarps][kRowPairsMax];
    __shared__ uint32_t st_col[kRowWarps][kRowStage], st_term[kRowWarps][kRowStage];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const unsigned lower = (1u << lane) - 1u;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        counts[kCntHalf] = min(pair_first[total_nodes], cap_half);
        if (pair_first[total_nodes] > cap_half) set_error(err, WS_ERR_CAPACITY);
    }
    const uint32_t warps = gridDim.x * kRowWarps;
    for (uint32_t row = blockIdx.x * kRowWarps + wib; row < total_nodes; row += warps) {
        const uint32_t h0 = pair_first[row], n_cols = pair_first[row + 1] - h0;
        const uint32_t s = node_scene[row];
        // the row's pairs: columns ascending, entry ranges one after another from the row's first
        uint32_t carry = entry_first[row];
        for (uint32_t k0 = 0; k0 < n_cols; k0 += 32) {
            const uint32_t k = k0 + (uint32_t)lane;
            const uint32_t c = k < n_cols ? row_cols[(size_t)kRowPairsMax * row + k] : kNoCol;
            const uint32_t n = k < n_cols ? row_cnts[(size_t)kRowPairsMax * row + k] : 0u;
            const uint32_t incl = warp_incl_scan_u32(n);
            const uint32_t begin = carry + incl - n;
            carry += __shfl_sync(0xffffffffu, incl, 31);
            if (k < n_cols) {
                s_col[wib][k] = c;
                s_next[wib][k] = begin;
                const uint32_t h = h0 + k;
                if (h < cap_half) {
                    half_row[h] = row;
                    half_col[h] = c;
                    half_begin[h] = begin;
                    half_end[h] = begin + n;
                    half_scene[h] = s;
                    atomicAdd(&row_cnt_lo[c], 1u);
                }
            }
        }
        __syncwarp();
        if (n_cols == 0) continue;
        const Scene &sc = scenes[s];
        const Plan &p = plan[s];
        const uint32_t beg = n2t_offset[row], end = n2t_offset[row + 1];
        if (lane == 0 && end > beg + kRowChunk) l2_prefetch_list(n2t_val, beg + kRowChunk, end, cap_n2t);
        for (uint32_t base = beg; base < end; base += kRowChunk) {
            const uint32_t total =
                stage_row_candidates(sc, p, dense_knn, n2t_val, row, base, end, st_col[wib], st_term[wib], lane, err);
            for (uint32_t v0 = 0; v0 < total; v0 += 32) {
                const uint32_t v = v0 + (uint32_t)lane;
                const uint32_t c = v < total ? st_col[wib][v] : kNoCol;
                const unsigned peers = __match_any_sync(0xffffffffu, c);
                uint32_t k = 0;
                if (c != kNoCol) {   // the column's place among the row's (binary search)
                    uint32_t lo = 0, hi = n_cols;
                    while (lo < hi) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (s_col[wib][mid] < c) lo = mid + 1; else hi = mid;
                    }
                    k = lo;
                    const uint32_t pos = s_next[wib][min(k, n_cols - 1)] + (uint32_t)__popc(peers & lower);
                    if (k < n_cols && s_col[wib][k] == c && pos < cap_kv) pair_val[pos] = st_term[wib][v];
                }
                __syncwarp();
                if (c != kNoCol && (peers & lower) == 0 && k < n_cols) s_next[wib][k] += (uint32_t)__popc(peers);
                __syncwarp();
            }
        }
    }
}

__global__ void k_row_first(const uint32_t *half_row, const uint32_t *counts, uint32_t *row_first) {
    const uint32_t n = counts[kCntHalf];
    for (uint32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < n; h += gridDim.x * blockDim.x)
        if (h == 0 || half_row[h - 1] != half_row[h]) row_first[half_row[h]] = h;
}

__global__ void k_row_len(const uint32_t *up, const uint32_t *lo, uint32_t total_nodes, uint32_t *len,
                          uint32_t *items) {
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total_nodes; g += gridDim.x * blockDim.x) {
        len[g] = 1u + up[g] + lo[g];
        items[g] = 1u + up[g];   // stored blocks of the row: the diagonal and the upper pairs
    }
}

__global__ void k_col_kv(const uint32_t *half_col, const uint32_t *counts, uint32_t *keys, uint32_t *vals) {
    const uint32_t n = counts[kCntHalf];
    for (uint32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < n; h += gridDim.x * blockDim.x) {
        keys[h] = half_col[h];
        vals[h] = h;
    }
}

// Block-CSR slots: every row is [diagonal, columns < row ascending, columns > row ascending],
// which is the sorted symmetric pair order of computeSymmetricNodePairKernel + sort
// (NodePair2TermsIndex.cu:171-192, 656-675) with the diagonal block placed first as in the
// Bin-Blocked CSR (NodePairRowColumnIndex.cu:110-124).  Also the item record of every pair
// h = (row, col) of the symmetric store (item h + row + 1): its lower entry is its position
// k among the pairs sorted by column (then row).
__global__ void k_slots(const uint32_t *sorted_col, const uint32_t *sorted_h, const uint32_t *counts,
                        const uint32_t *half_row, const uint32_t *half_col, const uint32_t *row_first,
                        const uint32_t *row_cnt_lo, const uint32_t *rowptr, uint32_t cap_blocks,
                        uint32_t *slot_up, uint32_t *slot_lo, uint32_t *colidx, uint2 *item_info,
                        uint32_t *item_col, int *err) {
    const uint32_t n = counts[kCntHalf];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t col = sorted_col[k];
        uint32_t lo = 0, hi = k;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sorted_col[mid] < col) lo = mid + 1; else hi = mid;
        }
        const uint32_t rank_lo = k - lo;
        const uint32_t h = sorted_h[k];
        const uint32_t row = half_row[h];
        const uint32_t s_lo = rowptr[col] + 1u + rank_lo;
        const uint32_t s_up = rowptr[row] + 1u + row_cnt_lo[row] + (h - row_first[row]);
        if (s_lo >= cap_blocks || s_up >= cap_blocks) {
            set_error(err, WS_ERR_CAPACITY);
            slot_lo[h] = slot_up[h] = kInvalidIndex;
            continue;
        }
        slot_lo[h] = s_lo;
        slot_up[h] = s_up;
        colidx[s_lo] = row;
        colidx[s_up] = half_col[h];
        item_info[h + row + 1u] = make_uint2(half_col[h], k);
        item_col[h + row + 1u] = half_col[h];
    }
}

// Diagonal slot of every row, and the item records of the row's diagonal item (the row, marked
// as a row start, and its scene).
__global__ void k_diag_cols(const uint32_t *rowptr, const uint32_t *item_ptr, const uint32_t *node_scene,
                            uint32_t total_nodes, uint32_t cap_blocks, uint32_t *colidx, uint2 *item_info,
                            uint32_t *item_col, int *err) {
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total_nodes; g += gridDim.x * blockDim.x) {
        const uint32_t s = rowptr[g];
        if (s < cap_blocks) colidx[s] = g;
        // the row's first item is its diagonal block
        item_info[item_ptr[g]] = make_uint2(g | kItemRowStart, node_scene[g]);
        item_col[item_ptr[g]] = g | kItemRowStart;
        if (g + 1 == total_nodes && rowptr[total_nodes] > cap_blocks) set_error(err, WS_ERR_CAPACITY);
    }
}

// First row group of every PCG phase-A work unit (kPcgUnitsPerWarp per warp), chosen so that the
// units' stored blocks (items) are about equal.  The groups before `split` (the first half of the
// scenes) and the groups from `split` on get separate units, their numbers in proportion to
// their items (at least one each when both halves have groups): unit w of a half starts at the
// first group of the half whose first item is at or past w / units of the half's items.
// warp_groups[units] is the group count and warp_groups[units + 1] the first half's units.
// unit_info[2w], [2w + 1] describe unit w for the PCG: its groups, rows and items (first, end)
// and the scenes of its first and last group, so that a unit starts from one load.
struct UnitSplit {
    uint32_t split, mid, total, ux, units, groups;
};
__device__ uint32_t unit_first_group(const UnitSplit &U, uint32_t w, const uint32_t *item_ptr,
                                     const uint32_t *group_row, uint32_t total_nodes) {
    if (w >= U.units) return U.groups;
    uint32_t lo, hi, target;
    if (w < U.ux) {
        lo = 0;
        hi = U.split;
        target = (uint32_t)(((unsigned long long)U.mid * w) / U.ux);
    } else {
        lo = U.split;
        hi = U.groups;
        target = U.mid + (uint32_t)(((unsigned long long)(U.total - U.mid) * (w - U.ux)) / (U.units - U.ux));
    }
    while (lo < hi) {
        const uint32_t m = (lo + hi) >> 1;
        if (item_ptr[min(group_row[m], total_nodes)] < target) lo = m + 1;
        else hi = m;
    }
    return lo;
}

__global__ void k_pcg_ranges(const uint32_t *item_ptr, const uint32_t *group_row, const uint32_t *group_scene,
                             uint32_t groups, uint32_t split, uint32_t total_nodes, uint32_t cap_items, uint32_t units,
                             uint32_t *warp_groups, uint4 *unit_info) {
    UnitSplit U;
    U.units = units;
    U.groups = groups;
    U.total = min(item_ptr[total_nodes], cap_items);
    U.split = min(split, groups);
    U.mid = U.split < groups ? min(item_ptr[min(group_row[U.split], total_nodes)], U.total) : U.total;
    U.ux = units;
    if (U.split > 0 && U.split < groups && units > 1) {
        U.ux = (uint32_t)(((unsigned long long)units * U.mid + U.total / 2) / max(U.total, 1u));
        U.ux = min(max(U.ux, 1u), units - 1);
    }
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w <= units + 1; w += gridDim.x * blockDim.x) {
        if (w >= units) {
            warp_groups[w] = (w == units) ? groups : U.ux;
            continue;
        }
        const uint32_t g0 = unit_first_group(U, w, item_ptr, group_row, total_nodes);
        const uint32_t g1 = max(g0, unit_first_group(U, w + 1, item_ptr, group_row, total_nodes));
        warp_groups[w] = g0;
        const uint32_t r0 = g0 < groups ? min(group_row[g0], total_nodes) : total_nodes;
        const uint32_t r1 = g1 < groups ? min(group_row[g1], total_nodes) : total_nodes;
        const uint32_t s0 = g0 < g1 ? group_scene[g0] : 0u, s1 = g0 < g1 ? group_scene[g1 - 1] : 0u;
        unit_info[2 * w] = make_uint4(g0, g1, r0, r1);
        unit_info[2 * w + 1] = make_uint4(min(item_ptr[r0], cap_items), min(item_ptr[r1], cap_items), s0, s1);
    }
}

static inline int grid_for(uint32_t n, int threads, int num_sms) {
    const uint32_t want = (n + threads - 1) / threads;
    const uint32_t cap = (uint32_t)num_sms * 8u;
    return (int)std::max<uint32_t>(1u, std::min<uint32_t>(want, cap));
}

// Node pair -> term map, row by row from the node -> term map (see k_pair_rows_count).
static void pair_index(Workspace &w, cudaStream_t st) {
    const uint32_t N = w.total_nodes;
    const int grid = grid_for(N * 32u, 32 * kRowWarps, w.num_sms);
    k_pair_rows_count<<<grid, 32 * kRowWarps, 0, st>>>(w.scenes, w.plan, w.node_scene, N, w.n2t_offset,
                                                      w.n2t_sorted_val, w.cap_n2t, w.d_knn, w.row_pair_cols, w.row_pair_cnts,
                                                      w.row_cnt_up, w.row_entry_first, w.error_flag);
    exclusive_scan(w.row_cnt_up, w.row_pair_first, nullptr, N, w.cap_nodes, w.scan_tmp, st);
    exclusive_scan(w.row_entry_first, w.row_entry_first, nullptr, N, w.cap_nodes, w.scan_tmp, st);
    cudaMemsetAsync(w.row_cnt_lo, 0, sizeof(uint32_t) * w.cap_nodes, st);
    k_pair_rows_fill<<<grid, 32 * kRowWarps, 0, st>>>(w.scenes, w.plan, w.node_scene, N, w.n2t_offset,
                                                     w.n2t_sorted_val, w.cap_n2t, w.d_knn, w.row_pair_cols, w.row_pair_cnts,
                                                     w.row_pair_first, w.row_entry_first, w.cap_half, w.cap_pair_kv,
                                                     w.half_row, w.half_col, w.half_begin, w.half_end, w.half_scene,
                                                     w.row_cnt_lo,
                                                     w.pair_val, w.counts, w.error_flag);
    w.pair_sorted_val = w.pair_val;
    count_launch(w, 1 + 3 + 3 + 1);
}

void index_build(Workspace &w, cudaStream_t st) {
    const int S = w.num_scenes;
    const int T = (int)w.total_tiles;
    const uint32_t N = w.total_nodes;
    // 1. compaction of potential pixels
    k_pixel_count<<<T, kPixTileThreads, 0, st>>>(w.scenes, w.tile_scene, T, w.tile_count);
    exclusive_scan(w.tile_count, w.tile_count, nullptr, (uint32_t)T, w.cap_tiles, w.scan_tmp, st);
    count_launch(w, 1 + 3);
    k_plan<<<1, 32, 0, st>>>(w.scenes, S, w.tile_count, T, w.plan, w.counts, w.cap_n2t, w.cap_pair_kv, w.error_flag);
    k_pixel_compact<<<T, kPixTileThreads, 0, st>>>(w.scenes, w.tile_scene, T, w.tile_count, w.d_pixels, w.d_knn,
                                                   w.d_sw, w.d_cw, w.d_scene, w.cap_pixels, w.error_flag);
    count_launch(w, 2);
    // 2. node -> term
    const uint32_t n2t_invalid = (1u << w.node_bits) - 1u;
    k_n2t_kv_dense<<<grid_for(w.cap_pixels, 256, w.num_sms), 256, 0, st>>>(w.scenes, w.plan, w.counts, w.d_scene,
                                                                            w.d_knn, w.n2t_key, w.n2t_val);
    k_n2t_kv_tail<<<dim3(16, S), 256, 0, st>>>(w.scenes, w.plan, w.n2t_key, w.n2t_val, n2t_invalid, w.error_flag);
    count_launch(w);
    const bool n2t_alt = radix_sort<uint32_t>(w.n2t_key, w.n2t_val, w.n2t_key_alt, w.n2t_val_alt, w.counts + kCntN2T, 0,
                                              w.cap_n2t, w.node_bits, w.sort_hist, w.sort_digit, st);
    count_launch(w, 1 + 3 * radix_passes(w.node_bits));
    w.n2t_sorted_key = n2t_alt ? w.n2t_key_alt : w.n2t_key;
    w.n2t_sorted_val = n2t_alt ? w.n2t_val_alt : w.n2t_val;
    k_n2t_offsets<<<grid_for(N + 1, 256, w.num_sms), 256, 0, st>>>(w.n2t_sorted_key, w.counts, N, w.n2t_offset);
    count_launch(w);
    // 3. node pair -> term
    pair_index(w, st);
    // 4. block CSR
    k_row_first<<<grid_for(w.cap_half, 256, w.num_sms), 256, 0, st>>>(w.half_row, w.counts, w.row_first);
    k_row_len<<<grid_for(N, 256, w.num_sms), 256, 0, st>>>(w.row_cnt_up, w.row_cnt_lo, N, w.rowptr, w.item_ptr);
    exclusive_scan(w.rowptr, w.rowptr, nullptr, N, w.cap_nodes, w.scan_tmp, st);
    exclusive_scan(w.item_ptr, w.item_ptr, nullptr, N, w.cap_nodes, w.scan_tmp, st);
    k_col_kv<<<grid_for(w.cap_half, 256, w.num_sms), 256, 0, st>>>(w.half_col, w.counts, w.col_key, w.col_val);
    const bool col_alt = radix_sort<uint32_t>(w.col_key, w.col_val, w.col_key_alt, w.col_val_alt, w.counts + kCntHalf,
                                              0, w.cap_half, w.node_bits, w.sort_hist, w.sort_digit, st);
    count_launch(w, 1 + 1 + 3 + 3 + 1 + 3 * radix_passes(w.node_bits));
    const uint32_t *scol = col_alt ? w.col_key_alt : w.col_key;
    const uint32_t *sh = col_alt ? w.col_val_alt : w.col_val;
    k_slots<<<grid_for(w.cap_half, 256, w.num_sms), 256, 0, st>>>(scol, sh, w.counts, w.half_row, w.half_col,
                                                                    w.row_first, w.row_cnt_lo, w.rowptr,
                                                                    w.cap_blocks, w.half_slot_up, w.half_slot_lo, w.colidx,
                                                                    w.item_info, w.item_col, w.error_flag);
    k_diag_cols<<<grid_for(N, 256, w.num_sms), 256, 0, st>>>(w.rowptr, w.item_ptr, w.node_scene, N, w.cap_blocks,
                                                             w.colidx, w.item_info, w.item_col, w.error_flag);
    count_launch(w, 2);
    pcg_ranges(w, st);
}

void pcg_ranges(Workspace &w, cudaStream_t st) {
    const uint32_t units = (uint32_t)(kPcgUnitsPerWarp * pcg_launch_blocks(w) * pcg_warps_per_block());
    k_pcg_ranges<<<grid_for(units + 2, 256, w.num_sms), 256, 0, st>>>(
        w.item_ptr, w.chunk_row, w.chunk_scene, w.total_chunks, pcg_split_group(w), w.total_nodes, w.cap_items, units,
        w.pcg_warp_groups, w.pcg_unit_info);
    count_launch(w);
}

}  // namespace ws
