// Shared device types and math for the B200 warp-field solver.
//
// Layout conventions (see include/warpsolve.h for the public view):
//   * node ids inside a scene are 16-bit (the reference's ushort knn / ushort3
//     edges); across a batch every node has a 32-bit global id
//     node_base[scene] + local id.
//   * a DualQuaternion is 8 floats: q0.xyzw, q1.xyzw (libs/star/math/DualQuaternion.hpp:206).
//   * per-node vectors use a stride of 8 floats (32 B) so that a 6-vector is
//     two aligned float4 loads.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/warpsolve.h"

namespace ws {

constexpr int kVecStride = 8;        // floats per node in PCG vectors
constexpr int kSdStride = 12;        // floats per node in the PCG's s/d records
constexpr int kRowPairsMax = 64;     // upper node pairs of one row in the pair map (WS_ERR_CAPACITY beyond)
constexpr int kDenseRecord = 32;     // floats per dense-term record, largest layout (128 B)
constexpr int kRegRecord = 16;       // floats per reg-term record (64 B)
constexpr uint32_t kInvalidIndex = 0xFFFFFFFFu;
constexpr uint32_t kItemRowStart = 0x80000000u;   // item_col: the row's first (diagonal) item
constexpr int kRowsPerGroup = 16;   // PCG rows (nodes) per scene-aligned reduction group (divides 32)
// PCG phase-A work units per warp: the units are balanced by stored blocks and taken by ticket.
constexpr int kPcgUnitsPerWarp = 2;

// Dense-term record layouts, chosen per batch.  With the optical-flow term (some scene of the
// batch has lambda_of != 0) a record holds C = 3 channels in 128 B: gradients 0..17 (three
// channels of [rotation | translation]), residuals 18..20, skinning weights 22..25, global
// node ids 26..29.  Without it only the depth channel is kept, C = 1, in 64 B: gradient 0..5,
// residual 6, weights 8..11, node ids 12..15.  A scene with lambda_of = 0 gets bit-identical
// sums either way: its flow rows are scaled by zero and add exact zeros.
template <int C>
struct DenseLayout {
    static_assert(C == 1 || C == 3, "one or three channels");
    static constexpr int kFloats = C == 3 ? 32 : 16;
    static constexpr int kRes = 6 * C;
    static constexpr int kW = C == 3 ? 22 : 8;
    static constexpr int kIds = kW + 4;
};

// ---------------------------------------------------------------------------
// Per-scene descriptor, device resident.  Filled on the host from ws_inputs.
// ---------------------------------------------------------------------------
struct Scene {
    int width, height, pitch;
    float fx, fy, cx, cy;
    float w2c[12];                     // row-major [R | t], world -> camera
    const float4 *mvert, *mnorm;       // measurement maps, camera frame
    const float4 *rvert, *rnorm;       // reference (render) maps, world frame
    const uint32_t *index_map;
    const float2 *flow;                // may be null
    const ushort4 *surfel_knn;
    const float4 *surfel_sw, *surfel_cw;
    int num_surfels;
    int num_nodes, node_base;
    int num_edges, edge_base;
    const uint16_t *edges;             // (i, j, k) triples
    const float *node_cw;              // graph_k per node
    int graph_k;
    float node_r2;
    const float4 *node_coords;
    const float4 *node_motion;         // may be null
    int num_features, feature_base;
    const ushort4 *feature_knn;        // may be null
    float lam_depth, lam_of, lam_reg, lam_node, lam_feat;
    int tile_base, num_tiles;          // pixel tiles of this scene
    int chunk_base, num_chunks;        // PCG row groups (kRowsPerGroup nodes) of this scene
};

// Per-scene counts derived on the device during the index build.
struct Plan {
    uint32_t dense_begin, dense_count;     // compacted dense terms
    uint32_t n2t_base, n2t_count;          // node->term key/value range
    uint32_t pair_base, pair_count;        // pair->term key/value range
    uint32_t pad[2];
};

// One lane asks L2 for entries [from, to) of a list of `cap` 4-byte words (a term list): one bulk
// prefetch from the 16-byte boundary at or below `from`, kept inside the list's allocation.
__device__ __forceinline__ void l2_prefetch_list(const uint32_t *list, uint32_t from, uint32_t to, uint32_t cap) {
    const uint32_t a = from & ~3u, stop = min(to, cap);
    const uint32_t words = stop > a ? ((stop - a + 3u) & ~3u) : 0u;
    if (words > 0 && a + words <= cap)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(list + a), "r"(4u * words) : "memory");
}

// ---------------------------------------------------------------------------
// Small math (FP32 as in the reference; libs/star/math/*).
// ---------------------------------------------------------------------------
struct M33 { float m[3][3]; };
struct SE3f { M33 rot; float3 t; };

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 mul(const M33 &R, float3 v) {
    return f3(R.m[0][0] * v.x + R.m[0][1] * v.y + R.m[0][2] * v.z,
              R.m[1][0] * v.x + R.m[1][1] * v.y + R.m[1][2] * v.z,
              R.m[2][0] * v.x + R.m[2][1] * v.y + R.m[2][2] * v.z);
}
__device__ __forceinline__ float3 tmul(const M33 &R, float3 v) {
    return f3(R.m[0][0] * v.x + R.m[1][0] * v.y + R.m[2][0] * v.z,
              R.m[0][1] * v.x + R.m[1][1] * v.y + R.m[2][1] * v.z,
              R.m[0][2] * v.x + R.m[1][2] * v.y + R.m[2][2] * v.z);
}

struct DQf { float4 q0, q1; };

__device__ __forceinline__ DQf load_dq(const float *p) {
    DQf d;
    d.q0 = *reinterpret_cast<const float4 *>(p);
    d.q1 = *reinterpret_cast<const float4 *>(p + 4);
    return d;
}
__device__ __forceinline__ void store_dq(float *p, const DQf &d) {
    *reinterpret_cast<float4 *>(p) = d.q0;
    *reinterpret_cast<float4 *>(p + 4) = d.q1;
}

// Hamilton product (libs/star/math/Quaternion.hpp:139-148), float4 = (x, y, z, w).
__device__ __forceinline__ float4 qmul(float4 a, float4 b) {
    float4 q;
    q.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
    q.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
    q.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
    q.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
    return q;
}
__device__ __forceinline__ float4 qconj(float4 a) { return make_float4(-a.x, -a.y, -a.z, a.w); }

// DualQuaternion::normalize (DualQuaternion.hpp:150-156; device rsqrt).
__device__ __forceinline__ void dq_normalize(DQf &d) {
    const float inv = rsqrtf(d.q0.x * d.q0.x + d.q0.y * d.q0.y + d.q0.z * d.q0.z + d.q0.w * d.q0.w);
    d.q0 = make_float4(inv * d.q0.x, inv * d.q0.y, inv * d.q0.z, inv * d.q0.w);
    d.q1 = make_float4(inv * d.q1.x, inv * d.q1.y, inv * d.q1.z, inv * d.q1.w);
    const float s = d.q0.x * d.q1.x + d.q0.y * d.q1.y + d.q0.z * d.q1.z + d.q0.w * d.q1.w;
    d.q1 = make_float4(d.q1.x - s * d.q0.x, d.q1.y - s * d.q0.y, d.q1.z - s * d.q0.z, d.q1.w - s * d.q0.w);
}

__device__ __forceinline__ M33 quat_rot(float4 q) {
    M33 r;
    r.m[0][0] = 1 - 2 * q.y * q.y - 2 * q.z * q.z;
    r.m[0][1] = 2 * q.x * q.y - 2 * q.z * q.w;
    r.m[0][2] = 2 * q.x * q.z + 2 * q.y * q.w;
    r.m[1][0] = 2 * q.x * q.y + 2 * q.z * q.w;
    r.m[1][1] = 1 - 2 * q.x * q.x - 2 * q.z * q.z;
    r.m[1][2] = 2 * q.y * q.z - 2 * q.x * q.w;
    r.m[2][0] = 2 * q.x * q.z - 2 * q.y * q.w;
    r.m[2][1] = 2 * q.y * q.z + 2 * q.x * q.w;
    r.m[2][2] = 1 - 2 * q.x * q.x - 2 * q.y * q.y;
    return r;
}

// R - I of a unit quaternion, formed without subtracting 1 from near-1 diagonal terms.
__device__ __forceinline__ M33 quat_rot_minus_identity(float4 q) {
    M33 r;
    r.m[0][0] = -2 * q.y * q.y - 2 * q.z * q.z;
    r.m[0][1] = 2 * q.x * q.y - 2 * q.z * q.w;
    r.m[0][2] = 2 * q.x * q.z + 2 * q.y * q.w;
    r.m[1][0] = 2 * q.x * q.y + 2 * q.z * q.w;
    r.m[1][1] = -2 * q.x * q.x - 2 * q.z * q.z;
    r.m[1][2] = 2 * q.y * q.z - 2 * q.x * q.w;
    r.m[2][0] = 2 * q.x * q.z - 2 * q.y * q.w;
    r.m[2][1] = 2 * q.y * q.z + 2 * q.x * q.w;
    r.m[2][2] = -2 * q.x * q.x - 2 * q.y * q.y;
    return r;
}

// SE(3) with R - I kept beside R, so that differences of warped points of
// about a metre can be formed from quantities of millimetres.
struct SE3d { M33 rot, rot_mi; float3 t; };

__device__ __forceinline__ SE3d dq_se3_split(DQf d) {
    dq_normalize(d);
    SE3d T;
    T.rot = quat_rot(d.q0);
    T.rot_mi = quat_rot_minus_identity(d.q0);
    const float4 two_q1 = make_float4(2.f * d.q1.x, 2.f * d.q1.y, 2.f * d.q1.z, 2.f * d.q1.w);
    const float4 tp = qmul(two_q1, qconj(d.q0));
    T.t = make_float3(tp.x, tp.y, tp.z);
    return T;
}

// DualQuaternion::se3_matrix (DualQuaternion.hpp:182-189).
__device__ __forceinline__ SE3f dq_se3(DQf d) {
    dq_normalize(d);
    SE3f T;
    T.rot = quat_rot(d.q0);
    const float4 two_q1 = make_float4(2.f * d.q1.x, 2.f * d.q1.y, 2.f * d.q1.z, 2.f * d.q1.w);
    const float4 tp = qmul(two_q1, qconj(d.q0));
    T.t = f3(tp.x, tp.y, tp.z);
    return T;
}

// DualQuaternion -> mat34 (DualQuaternion.hpp:169-179).
__device__ __forceinline__ SE3f dq_to_mat34(DQf d) {
    dq_normalize(d);
    float4 q = d.q0;
    const float inv = rsqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    q = make_float4(q.x * inv, q.y * inv, q.z * inv, q.w * inv);
    SE3f T;
    T.rot = quat_rot(q);
    const float4 two_q1 = make_float4(2.f * d.q1.x, 2.f * d.q1.y, 2.f * d.q1.z, 2.f * d.q1.w);
    const float4 tp = qmul(two_q1, qconj(d.q0));
    T.t = f3(tp.x, tp.y, tp.z);
    return T;
}

// Quaternion(const mat33&) (Quaternion.hpp:17-52).
__device__ __forceinline__ float4 quat_from_rot(const M33 &m) {
    float4 q;
    const float tr = m.m[0][0] + m.m[1][1] + m.m[2][2];
    if (tr > 0) {
        const float s = sqrtf(tr + 1.0f) * 2;
        q.w = s * 0.25f;
        q.x = (m.m[2][1] - m.m[1][2]) / s;
        q.y = (m.m[0][2] - m.m[2][0]) / s;
        q.z = (m.m[1][0] - m.m[0][1]) / s;
    } else if ((m.m[0][0] > m.m[1][1]) && (m.m[0][0] > m.m[2][2])) {
        const float s = sqrtf(1.0f + m.m[0][0] - m.m[1][1] - m.m[2][2]) * 2;
        q.w = (m.m[2][1] - m.m[1][2]) / s;
        q.x = 0.25f * s;
        q.y = (m.m[0][1] + m.m[1][0]) / s;
        q.z = (m.m[0][2] + m.m[2][0]) / s;
    } else if (m.m[1][1] > m.m[2][2]) {
        const float s = sqrtf(1.0f + m.m[1][1] - m.m[0][0] - m.m[2][2]) * 2;
        q.w = (m.m[0][2] - m.m[2][0]) / s;
        q.x = (m.m[0][1] + m.m[1][0]) / s;
        q.y = 0.25f * s;
        q.z = (m.m[1][2] + m.m[2][1]) / s;
    } else {
        const float s = sqrtf(1.0f + m.m[2][2] - m.m[0][0] - m.m[1][1]) * 2;
        q.w = (m.m[1][0] - m.m[0][1]) / s;
        q.x = (m.m[0][2] + m.m[2][0]) / s;
        q.y = (m.m[1][2] + m.m[2][1]) / s;
        q.z = 0.25f * s;
    }
    return q;
}

// DualQuaternion(const mat34&) (DualQuaternion.hpp:59-66).
__device__ __forceinline__ DQf dq_from_mat34(const SE3f &T) {
    DQf d;
    d.q0 = quat_from_rot(T.rot);
    const float4 qt = make_float4(0.5f * T.t.x, 0.5f * T.t.y, 0.5f * T.t.z, 0.f);
    d.q1 = qmul(qt, d.q0);
    return d;
}

// ---------------------------------------------------------------------------
// Warp helpers.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Bounded spin limit for every wait in this library (about a second at the
// nanosleep granularity used).
constexpr unsigned long long kSpinLimit = 1ull << 24;

}  // namespace ws
