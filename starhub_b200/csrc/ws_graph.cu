// Node graph construction, skinning, forward warp and the solver-map splat.
//
// Integer outputs (node candidates, node and surfel k-NN ids) follow the
// reference bit for bit: the same float expressions with the fused
// multiply-adds spelled out, the same strict-inequality heap, and the same
// Lomuto quicksort.  Weights use __expf as the reference does.
#include <cuda_runtime.h>
#include <cuda_fp16.h>

#include <mutex>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/warpsolve.h"
#include "ws_common.cuh"
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
// encodeVoxel (libs/star/common/encode_utils.h:138-141).
__global__ void k_voxel_key(const float4 *pts, uint32_t n, float voxel, uint32_t *keys, uint32_t *vals) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = pts[i];
        const int vx = __float2int_rd(p.x / voxel), vy = __float2int_rd(p.y / voxel), vz = __float2int_rd(p.z / voxel);
        keys[i] = (uint32_t)((vx + 512) + (vy + 512) * 1024 + (vz + 512) * 1024 * 1024);
        vals[i] = i;
    }
}

__global__ void k_voxel_marks(const uint32_t *keys, uint32_t n, uint32_t *marks) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        marks[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// samplingPointsKernel (VoxelSubsamplerSorting.cu:60-96): per voxel the point nearest the
// voxel centre, first wins on ties.
__global__ void k_voxel_sample(const uint32_t *keys, const uint32_t *perm, const uint32_t *head_off, uint32_t n,
                               const float4 *pts, float voxel, float4 *out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (i != 0 && keys[i] == keys[i - 1]) continue;   // not the first point of its voxel
        uint32_t e = i + 1;
        while (e < n && keys[e] == keys[i]) ++e;
        const int enc = (int)keys[i];
        int z = enc / (1024 * 1024);
        int x = enc % 1024;
        int y = (enc - z * 1024 * 1024) / 1024;
        x -= 512; y -= 512; z -= 512;
        const float cx = float(x + 0.5) * voxel, cy = float(y + 0.5) * voxel, cz = float(z + 0.5) * voxel;
        float best = 1e5f;
        uint32_t bi = i;
        for (uint32_t k = i; k < e; ++k) {
            const float4 p = pts[perm[k]];
            const float dd = sq3_fused(p.x - cx, p.y - cy, p.z - cz);
            if (dd < best) { best = dd; bi = k; }
        }
        out[head_off[i]] = pts[perm[bi]];
    }
}

// UpdateNodeDistanceKernel + BuildNodeGraphKernel (libs/star/geometry/node_graph/NodeGraph.cu:10-101):
// half-precision squared distances, k nearest including the node itself, __expf weights normalized.
template <int K>
__global__ void k_node_graph(const float4 *nodes, int n, float r2, uint16_t *knn, float *w, uint16_t *edges) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
        const float4 va = nodes[a];
        Heap<K> h;
        h.init(1e3f);
        for (int b = 0; b < n; ++b) {
            const float4 vb = nodes[b];
            const float4 hi = (a >= b) ? va : vb, lo = (a >= b) ? vb : va;
            const float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
            const float dist = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
            h.update((uint16_t)b, __half2float(__float2half_rn(dist)));
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
            w[(size_t)a * K + q] = wv[q] * inv;
            // BuildNodeGraphPairKernel (NodeGraph.cu:103-118)
            edges[3 * ((size_t)a * K + q)] = (uint16_t)a;
            edges[3 * ((size_t)a * K + q) + 1] = h.id[q];
            edges[3 * ((size_t)a * K + q) + 2] = (uint16_t)q;
        }
    }
}

// SkinnerKernel (libs/star/geometry/node_graph/Skinner.cu:10-94); nodes staged in shared memory.
__global__ void __launch_bounds__(256) k_skinning(const float4 *nodes, int n_nodes, const float4 *verts, int n_verts,
                                                   float r2, ushort4 *knn, float4 *sw, float4 *cw) {
    __shared__ float4 tile[1024];
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    const float4 p = v < n_verts ? verts[v] : make_float4(0.f, 0.f, 0.f, 0.f);
    Heap<4> h;
    h.init(1e6f);
    for (int base = 0; base < n_nodes; base += 1024) {
        const int cnt = min(1024, n_nodes - base);
        __syncthreads();
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) tile[i] = nodes[base + i];
        __syncthreads();
        for (int i = 0; i < cnt; ++i) {
            const float4 q = tile[i];
            h.update((uint16_t)(base + i), sq3_fused(p.x - q.x, p.y - q.y, p.z - q.z));
        }
    }
    if (v >= n_verts) return;
    h.sort();
    float wv[4], sum = 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float4 q = nodes[h.id[i]];
        const float dd = sq3_fused(p.x - q.x, p.y - q.y, p.z - q.z);
        wv[i] = __expf(-dd / (2.f * r2));
        sum += wv[i];
    }
    const float inv = 1.f / sum;
    knn[v] = make_ushort4(h.id[0], h.id[1], h.id[2], h.id[3]);
    sw[v] = make_float4(inv * wv[0], inv * wv[1], inv * wv[2], inv * wv[3]);
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

}  // namespace

extern "C" {

int ws_init_nodes(const float *surfels, int n, float node_radius, float *nodes_host, int cap, int *num_nodes,
                  void *stream) {
    if (!surfels || n <= 0 || !nodes_host || !num_nodes || cap < 2 || !(node_radius > 0.f))
        return WS_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float voxel = 0.7f * node_radius;
    uint32_t *keys = nullptr, *vals = nullptr, *keys2 = nullptr, *vals2 = nullptr, *heads = nullptr, *tmp = nullptr,
             *hist = nullptr, *digit = nullptr;
    float4 *cand = nullptr;
    const uint32_t un = (uint32_t)n;
    cudaError_t e = cudaSuccess;
    auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    A(cudaMalloc(&keys, 4ull * un));
    A(cudaMalloc(&vals, 4ull * un));
    A(cudaMalloc(&keys2, 4ull * un));
    A(cudaMalloc(&vals2, 4ull * un));
    A(cudaMalloc(&heads, 4ull * (un + 1)));
    A(cudaMalloc(&tmp, 4ull * (un / ws::kScanTile + 4)));
    A(cudaMalloc(&hist, 4ull * 256 * ws::sort_max_tiles(un)));
    A(cudaMalloc(&digit, 4ull * 256));
    A(cudaMalloc(&cand, 16ull * un));
    std::vector<float4> hc;
    uint32_t nv = 0;
    if (e == cudaSuccess) {
        const float4 *pts = reinterpret_cast<const float4 *>(surfels);
        ws::k_voxel_key<<<ws::grid_of(n, 256), 256, 0, st>>>(pts, un, voxel, keys, vals);
        const bool alt = ws::radix_sort<uint32_t>(keys, vals, keys2, vals2, nullptr, un, un, 30, hist, digit, st);
        const uint32_t *sk = alt ? keys2 : keys, *sv = alt ? vals2 : vals;
        ws::k_voxel_marks<<<ws::grid_of(n, 256), 256, 0, st>>>(sk, un, heads);
        ws::exclusive_scan(heads, heads, nullptr, un, un, tmp, st);
        ws::k_voxel_sample<<<ws::grid_of(n, 256), 256, 0, st>>>(sk, sv, heads, un, pts, voxel, cand);
        A(cudaMemcpyAsync(&nv, heads + un, 4, cudaMemcpyDeviceToHost, st));
        A(cudaStreamSynchronize(st));
        hc.resize(nv);
        if (nv) A(cudaMemcpy(hc.data(), cand, 16ull * nv, cudaMemcpyDeviceToHost));
    }
    for (void *p : {(void *)keys, (void *)vals, (void *)keys2, (void *)vals2, (void *)heads, (void *)tmp, (void *)hist,
                    (void *)digit, (void *)cand})
        if (p) cudaFree(p);
    if (e != cudaSuccess) return WS_ERR_CUDA;
    // NodeGraph::AppendNodeFromVertexHost (NodeGraph.cu:652-704): greedy in candidate order.
    const float r = 0.85f * node_radius;
    const float thr = r * r;
    std::vector<float4> acc;
    for (uint32_t i = 0; i < nv; ++i) {
        const float4 p = make_float4(hc[i].x, hc[i].y, hc[i].z, 1.0f);
        if (std::isnan(p.x) || std::isnan(p.y) || std::isnan(p.z)) return WS_ERR_INVALID_ARGUMENT;
        bool is_node = true;
        for (const float4 &q : acc) {
            const float dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z, dw = q.w - p.w;
            const float d2 = ((dx * dx + dy * dy) + dz * dz) + dw * dw;
            if (d2 <= thr) { is_node = false; break; }
        }
        if (is_node) acc.push_back(p);
    }
    const int total = (int)acc.size() + 2;
    *num_nodes = total;
    if (total > cap) return WS_ERR_CAPACITY;
    for (int a = 0; a < 2; ++a) {
        nodes_host[4 * a] = 0.f; nodes_host[4 * a + 1] = 0.f; nodes_host[4 * a + 2] = 0.f; nodes_host[4 * a + 3] = 1.f;
    }
    std::memcpy(nodes_host + 8, acc.data(), acc.size() * sizeof(float4));
    return WS_OK;
}

int ws_build_node_graph(const float *nodes, int n, int k, float node_radius, uint16_t *knn, float *w, uint16_t *edges,
                        void *stream) {
    if (!nodes || n <= 0 || n > 65535 || !knn || !w || !edges || (k != 4 && k != 8)) return WS_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float r2 = node_radius * node_radius;
    const int threads = 64;
    const int grid = (n + threads - 1) / threads;
    if (k == 4)
        ws::k_node_graph<4><<<grid, threads, 0, st>>>(reinterpret_cast<const float4 *>(nodes), n, r2, knn, w, edges);
    else
        ws::k_node_graph<8><<<grid, threads, 0, st>>>(reinterpret_cast<const float4 *>(nodes), n, r2, knn, w, edges);
    return cudaGetLastError() == cudaSuccess ? WS_OK : WS_ERR_CUDA;
}

int ws_skinning(const float *nodes, int n_nodes, const float *verts, int n_verts, float node_radius, uint16_t *knn,
                float *sw, float *cw, void *stream) {
    if (!nodes || n_nodes <= 0 || n_nodes > 65535 || !verts || n_verts < 0 || !knn || !sw || !cw)
        return WS_ERR_INVALID_ARGUMENT;
    if (n_verts == 0) return WS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float r2 = node_radius * node_radius;
    ws::k_skinning<<<(n_verts + 255) / 256, 256, 0, st>>>(
        reinterpret_cast<const float4 *>(nodes), n_nodes, reinterpret_cast<const float4 *>(verts), n_verts, r2,
        reinterpret_cast<ushort4 *>(knn), reinterpret_cast<float4 *>(sw), reinterpret_cast<float4 *>(cw));
    return cudaGetLastError() == cudaSuccess ? WS_OK : WS_ERR_CUDA;
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
    cudaMemsetAsync(zbuf, 0xff, 8 * npix, st);
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

}  // extern "C"
