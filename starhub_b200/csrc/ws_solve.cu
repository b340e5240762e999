// Gauss-Newton iteration of the B200 warp-field solver: term evaluation,
// J^T J / J^T r assembly as warp-segmented reductions over the term lists, and a
// persistent cooperative block-PCG with fused SpMV + dot + axpy.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "ws_common.cuh"
#include "ws_workspace.h"

namespace ws {

__device__ __forceinline__ void set_err(int *flag, int code) { atomicCAS(flag, 0, code); }

// ---------------------------------------------------------------------------
// Warp-field initialisation (SolverIterationData::SetWarpFieldInitialValue,
// examples/mono_star/opt/SolverIterationData.cu:8-17, 112-125).
// ---------------------------------------------------------------------------
__global__ void k_init_warp(const Scene *scenes, const uint32_t *node_scene, uint32_t total_nodes, float *se3) {
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total_nodes; g += gridDim.x * blockDim.x) {
        const Scene &sc = scenes[node_scene[g]];
        (void)sc;
        float4 q0 = make_float4(0.f, 0.f, 0.f, 1.f), q1 = make_float4(0.f, 0.f, 0.f, 0.f);
        reinterpret_cast<float4 *>(se3 + 8ull * g)[0] = q0;
        reinterpret_cast<float4 *>(se3 + 8ull * g)[1] = q1;
    }
}

__global__ void k_copy_init_warp(const float *init, uint32_t node_base, uint32_t num_nodes, float *se3) {
    for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < num_nodes; n += gridDim.x * blockDim.x) {
        const float4 *src = reinterpret_cast<const float4 *>(init + 8ull * n);
        float4 *dst = reinterpret_cast<float4 *>(se3 + 8ull * (node_base + n));
        dst[0] = src[0];
        dst[1] = src[1];
    }
}

// ---------------------------------------------------------------------------
// Dense depth + optical-flow term (computeDenseImageJacobianKernel,
// examples/mono_star/opt/DenseImageJacobianResidual.cu:164-308, with :12-25 and :77-115).
// One thread per compacted term; writes one record in the batch's layout (DenseLayout<C>):
// the gradients and residuals of the depth channel (and of the two flow channels when C = 3),
// the knn weights (spatial * connect) and the global knn node ids.
// ---------------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(256) k_eval_dense(const Scene *scenes, const uint32_t *counts,
                                                     const ushort4 *pixels, const ushort4 *knn, const float4 *sw,
                                                     const float4 *cw, const uint32_t *term_scene, const float *se3,
                                                     float *record) {
    const uint32_t n = counts[kCntDense];
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const Scene &sc = scenes[term_scene[t]];
        const ushort4 k4 = knn[t];
        const float4 s4 = sw[t], c4 = cw[t];
        const uint32_t nb = (uint32_t)sc.node_base;
        const uint32_t g[4] = {nb + k4.x, nb + k4.y, nb + k4.z, nb + k4.w};
        const float w[4] = {s4.x * c4.x, s4.y * c4.y, s4.z * c4.z, s4.w * c4.w};
        // averageDualQuaternion, pointer overload (libs/star/math/DualQuaternion.hpp:244-261)
        DQf avg;
        avg.q0 = make_float4(0.f, 0.f, 0.f, 0.f);
        avg.q1 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const DQf d = load_dq(se3 + 8ull * g[k]);
            avg.q0 = make_float4(avg.q0.x + w[k] * d.q0.x, avg.q0.y + w[k] * d.q0.y, avg.q0.z + w[k] * d.q0.z,
                                 avg.q0.w + w[k] * d.q0.w);
            avg.q1 = make_float4(avg.q1.x + w[k] * d.q1.x, avg.q1.y + w[k] * d.q1.y, avg.q1.z + w[k] * d.q1.z,
                                 avg.q1.w + w[k] * d.q1.w);
        }
        const SE3d T = dq_se3_split(avg);
        const ushort4 px = pixels[t];
        const size_t spix = (size_t)px.y * sc.pitch + px.x;
        const float4 cv4 = sc.rvert[spix], cn4 = sc.rnorm[spix];
        const float3 vw = mul(T.rot, f3(cv4.x, cv4.y, cv4.z)) + T.t;
        const float3 nw = mul(T.rot, f3(cn4.x, cn4.y, cn4.z));
        M33 W;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) W.m[i][j] = sc.w2c[4 * i + j];
        const float3 wt = f3(sc.w2c[3], sc.w2c[7], sc.w2c[11]);
        const float3 vc = mul(W, vw) + wt;
        const float3 nc = mul(W, nw);
        float gr[18];
        float res[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int i = 0; i < 18; ++i) gr[i] = 0.f;
        if (px.z < (unsigned)sc.width && px.w < (unsigned)sc.height) {
            const size_t tpix = (size_t)px.w * sc.pitch + px.z;
            const float4 tv4 = sc.mvert[tpix], tn4 = sc.mnorm[tpix];
            const float3 tv = f3(tv4.x, tv4.y, tv4.z), tn = f3(tn4.x, tn4.y, tn4.z);
            bool ok = true;
            if (fabsf(tv4.x) < 1e-3 && fabsf(tv4.y) < 1e-3 && fabsf(tv4.z) < 1e-3) ok = false;   // is_zero_vertex
            if (dot3(tn, nc) < 0.7f) ok = false;                                                  // global_configs.h:57
            if (fabsf(tv.z - vc.z) > 0.03f) ok = false;                                           // global_configs.h:58
            if (ok) {
                const float3 tvw = tmul(W, tv - wt);   // apply_inversed_se3
                const float3 tnw = tmul(W, tn);        // rot.transpose_dot
                // v_w - v_t = (R - I) v_ref + t + (v_ref - v_t): the same quantity as the
                // reference's dot(n, v_w - v_t), without cancelling two ~1 m vectors in FP32
                const float3 cv = f3(cv4.x, cv4.y, cv4.z);
                const float3 diff = (mul(T.rot_mi, cv) + T.t) + (cv - tvw);
                res[0] = dot3(tnw, diff);
                const float3 rr = cross3(vw, tnw);
                gr[0] = rr.x; gr[1] = rr.y; gr[2] = rr.z;
                gr[3] = tnw.x; gr[4] = tnw.y; gr[5] = tnw.z;
                const float3 row0 = f3(W.m[0][0], W.m[0][1], W.m[0][2]);
                const float3 row1 = f3(W.m[1][0], W.m[1][1], W.m[1][2]);
                const float ex = dot3(row0, diff), ey = dot3(row1, diff);
                if (C == 3 && !(sqrtf(ex * ex + ey * ey) < 1e-6f)) {
                    res[1] = ex;
                    res[2] = ey;
                    const float3 mv = f3(-vw.x, -vw.y, -vw.z);
                    gr[6] = row0.y * mv.z - row0.z * mv.y;
                    gr[7] = -row0.x * mv.z + row0.z * mv.x;
                    gr[8] = row0.x * mv.y - row0.y * mv.x;
                    gr[9] = row0.x; gr[10] = row0.y; gr[11] = row0.z;
                    gr[12] = row1.y * mv.z - row1.z * mv.y;
                    gr[13] = -row1.x * mv.z + row1.z * mv.x;
                    gr[14] = row1.x * mv.y - row1.y * mv.x;
                    gr[15] = row1.x; gr[16] = row1.y; gr[17] = row1.z;
                }
            }
        }
        float4 *out = reinterpret_cast<float4 *>(record + (size_t)DenseLayout<C>::kFloats * t);
        if constexpr (C == 3) {
            out[0] = make_float4(gr[0], gr[1], gr[2], gr[3]);
            out[1] = make_float4(gr[4], gr[5], gr[6], gr[7]);
            out[2] = make_float4(gr[8], gr[9], gr[10], gr[11]);
            out[3] = make_float4(gr[12], gr[13], gr[14], gr[15]);
            out[4] = make_float4(gr[16], gr[17], res[0], res[1]);
            out[5] = make_float4(res[2], 0.f, w[0], w[1]);
            out[6] = make_float4(w[2], w[3], __uint_as_float(g[0]), __uint_as_float(g[1]));
            out[7] = make_float4(__uint_as_float(g[2]), __uint_as_float(g[3]), 0.f, 0.f);
        } else {
            out[0] = make_float4(gr[0], gr[1], gr[2], gr[3]);
            out[1] = make_float4(gr[4], gr[5], res[0], 0.f);
            out[2] = make_float4(w[0], w[1], w[2], w[3]);
            out[3] = make_float4(__uint_as_float(g[0]), __uint_as_float(g[1]), __uint_as_float(g[2]),
                                 __uint_as_float(g[3]));
        }
    }
}

// ---------------------------------------------------------------------------
// ARAP smoothness term (forwardWarpSmootherNodeKernel,
// examples/mono_star/opt/NodeGraphHandler.cu:7-45).  Record (64 B):
//   [0,3) Ti xj, [3,6) Tj xj, [6] connect weight, [7] validity, [8] i, [9] j (global ids),
//   [10,13) Ti xj - Tj xj evaluated without cancellation.
// ---------------------------------------------------------------------------
__global__ void k_eval_reg(const Scene *scenes, const uint32_t *edge_scene, uint32_t total_edges, const float *se3,
                           float *record) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total_edges; e += gridDim.x * blockDim.x) {
        const Scene &sc = scenes[edge_scene[e]];
        const uint32_t el = e - sc.edge_base;
        // out-of-range ids were flagged by the index build; clamp so every read stays in bounds
        const uint16_t last = (uint16_t)(sc.num_nodes - 1);
        const uint16_t i = min(sc.edges[3 * el], last), j = min(sc.edges[3 * el + 1], last);
        const uint16_t k = min(sc.edges[3 * el + 2], (uint16_t)(sc.graph_k - 1));
        const float4 xi = sc.node_coords[i], xj = sc.node_coords[j];
        const SE3d Ti = dq_se3_split(load_dq(se3 + 8ull * (sc.node_base + i)));
        const SE3d Tj = dq_se3_split(load_dq(se3 + 8ull * (sc.node_base + j)));
        const float3 vj = f3(xj.x, xj.y, xj.z);
        const float3 a = mul(Ti.rot, vj) + Ti.t;
        const float3 b = mul(Tj.rot, vj) + Tj.t;
        // Ti xj - Tj xj = ((Ri - I) - (Rj - I)) xj + (ti - tj), free of cancellation
        M33 dR;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int q = 0; q < 3; ++q) dR.m[r][q] = Ti.rot_mi.m[r][q] - Tj.rot_mi.m[r][q];
        const float3 rij = mul(dR, vj) + (Ti.t - Tj.t);
        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const float d2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
        const float valid = (d2 > 64 * sc.node_r2) ? 0.f : 1.f;   // CLIP_FARAWAY_NODEGRAPH_PAIR
        const float c = sc.node_cw[(size_t)i * sc.graph_k + k];
        float4 *out = reinterpret_cast<float4 *>(record + (size_t)kRegRecord * e);
        out[0] = make_float4(a.x, a.y, a.z, b.x);
        out[1] = make_float4(b.y, b.z, c, valid);
        out[2] = make_float4(__uint_as_float(sc.node_base + i), __uint_as_float(sc.node_base + j), rij.x, rij.y);
        out[3] = make_float4(rij.z, 0.f, 0.f, 0.f);
    }
}

// Twist centre of every node for this Gauss-Newton iteration: the node's current warped
// position.  The mixed-precision path solves for each node's twist about this centre
// instead of the world origin (block-Jacobi PCG iterates are invariant under this
// block-diagonal change of variables); the lever arm drops from ~1 m to a few cm,
// which keeps the 6x6 blocks well conditioned in FP32.
__global__ void k_node_centers(const Scene *scenes, const uint32_t *node_scene, uint32_t total_nodes,
                               const float *se3, float4 *centers) {
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total_nodes; g += gridDim.x * blockDim.x) {
        const Scene &sc = scenes[node_scene[g]];
        const float4 x = sc.node_coords[g - sc.node_base];
        const SE3f T = dq_se3(load_dq(se3 + 8ull * g));
        const float3 c = mul(T.rot, f3(x.x, x.y, x.z)) + T.t;
        centers[g] = make_float4(c.x, c.y, c.z, 0.f);
    }
}

// Rotation part of a Jacobian row for a twist about `c`: rho - c x tau.
__device__ __forceinline__ void recentre(float *row, float3 c) {
    const float3 ct = cross3(c, f3(row[3], row[4], row[5]));
    row[0] -= ct.x;
    row[1] -= ct.y;
    row[2] -= ct.z;
}

// Reg Jacobian rows without the connect weight (libs/star/opt/node_graph_reg_jacobian.cuh:85-106).
__device__ __forceinline__ void reg_unit_jacobian(float3 a, float3 b, bool is_i, float J[3][6]) {
    if (is_i) {
        J[0][0] = 0.f;  J[0][1] = a.z;  J[0][2] = -a.y; J[0][3] = 1.f; J[0][4] = 0.f; J[0][5] = 0.f;
        J[1][0] = -a.z; J[1][1] = 0.f;  J[1][2] = a.x;  J[1][3] = 0.f; J[1][4] = 1.f; J[1][5] = 0.f;
        J[2][0] = a.y;  J[2][1] = -a.x; J[2][2] = 0.f;  J[2][3] = 0.f; J[2][4] = 0.f; J[2][5] = 1.f;
    } else {
        J[0][0] = 0.f;  J[0][1] = -b.z; J[0][2] = b.y;  J[0][3] = -1.f; J[0][4] = 0.f;  J[0][5] = 0.f;
        J[1][0] = b.z;  J[1][1] = 0.f;  J[1][2] = -b.x; J[1][3] = 0.f;  J[1][4] = -1.f; J[1][5] = 0.f;
        J[2][0] = -b.y; J[2][1] = b.x;  J[2][2] = 0.f;  J[2][3] = 0.f;  J[2][4] = 0.f;  J[2][5] = -1.f;
    }
}

__device__ __forceinline__ int tri_index(int a, int c) {   // upper triangle (a <= c), row-major
    return a * 6 - (a * (a - 1)) / 2 + (c - a);
}

// ---------------------------------------------------------------------------
// 6x6 block inverses.
// ---------------------------------------------------------------------------
// DenseGaussian<6>::Inverse with partial pivoting (libs/star/math/DenseGaussian.hpp:33-112), FP32.
__device__ void gauss_jordan6(const float *in, float *out) {
    float m[36];
    for (int i = 0; i < 36; ++i) m[i] = in[i];
    int perm[6], reloc[6];
    for (int i = 0; i < 6; ++i) perm[i] = i;
    for (int i = 0; i < 6; ++i) {
        int piv = i;
        float pv = fabsf(m[6 * i + i]);
        for (int j = i + 1; j < 6; ++j)
            if (pv < fabsf(m[6 * j + i])) { pv = fabsf(m[6 * j + i]); piv = j; }
        for (int k = 0; k < 6; ++k) { const float t = m[6 * i + k]; m[6 * i + k] = m[6 * piv + k]; m[6 * piv + k] = t; }
        { const int t = perm[i]; perm[i] = perm[piv]; perm[piv] = t; }
        reloc[i] = perm[i];
        const float inv = 1.0f / m[6 * i + i];
        for (int k = 0; k < 6; ++k) m[6 * i + k] *= inv;
        m[6 * i + i] = inv;
        for (int r = 0; r < 6; ++r) {
            if (r == i) continue;
            const float a = m[6 * r + i];
            for (int k = 0; k < 6; ++k) m[6 * r + k] -= a * m[6 * i + k];
            m[6 * r + i] = -a * m[6 * i + i];
        }
    }
    for (int j = 0; j < 6; ++j)
        for (int i = 0; i < 6; ++i) out[6 * reloc[j] + i] = m[6 * i + j];
}

// Symmetric positive definite 6x6 inverse by Cholesky in FP64.
__device__ void cholesky6_fp64(const double *in, float *out) {
    double L[21];   // packed lower triangle, row i holds i+1 entries
#define LI(i, j) L[(i) * ((i) + 1) / 2 + (j)]
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = in[6 * i + j];
            for (int k = 0; k < j; ++k) s -= LI(i, k) * LI(j, k);
            if (i == j) LI(i, i) = sqrt(s > 0.0 ? s : 1e-300);
            else LI(i, j) = s / LI(j, j);
        }
    double Linv[21];
#define LV(i, j) Linv[(i) * ((i) + 1) / 2 + (j)]
    for (int i = 0; i < 6; ++i) {
        LV(i, i) = 1.0 / LI(i, i);
        for (int j = 0; j < i; ++j) {
            double s = 0.0;
            for (int k = j; k < i; ++k) s -= LI(i, k) * LV(k, j);
            LV(i, j) = s / LI(i, i);
        }
    }
    for (int i = 0; i < 6; ++i)
        for (int j = i; j < 6; ++j) {
            double s = 0.0;
            for (int k = j; k < 6; ++k) s += LV(k, i) * LV(k, j);
            out[6 * i + j] = (float)s;
            out[6 * j + i] = (float)s;
        }
#undef LI
#undef LV
}

// ---------------------------------------------------------------------------
// Diagonal blocks and right-hand side: one warp per node over its node->term list
// (computeBlockDiagonalPreconditionerKernel, examples/mono_star/opt/PreconditionerRhsBuilder.cu:110-261,
// and computeJtResidualWithIndexKernel, JtDotResidualIndexed.cu:40-149).
//
// Every term contributes three scaled Jacobian rows u (lambda * J, 6 values) and a scaled
// residual v, so that D += u u^T and b += v u.  The warp takes 32 list entries at a time,
// copies their records into shared memory with coalesced loads, and each lane sums its own
// term's products in registers; at the end of the list the 27 entries are summed over the
// lanes in lane order through shared memory.  The order is fixed by the list, so results do
// not depend on what else is in the batch.
// Each lane sums its own terms (a few per node) in FP32.  DAcc is the type of the sum over the
// lanes: float for WS_PREC_FP32 (the reference's FP32 sums), double for WS_PREC_MIXED, where D
// feeds the FP64 Cholesky directly.  The FP32 lane sums cost about as much accuracy as storing
// the block in FP32, which the SpMV does anyway, and free the registers that 27 FP64 sums
// would hold, which lets more warps hide the gathers' latency.
// ---------------------------------------------------------------------------

// After a list, the lanes' partial sums go through the staging area, one 36-float slot per
// lane (27 sums for a node, 21 or 36 for a pair); the stride keeps 16-byte accesses by
// consecutive lanes on distinct banks.
constexpr int kSlotWordsF32 = 36;

// Staging of term records for the assembly kernels.  A batch holds kTPL records per lane:
// record r = 32 t + l is lane l's t-th term, at stage + r * kRec (kRec words: a record plus
// padding that keeps 16-byte accesses by consecutive lanes on distinct banks).  Lane l
// names its t-th record through locate(t, src, parts): src in 16-byte units and parts at
// most kParts, 0 for none; kParts is 8 for 128-byte and 4 for 64-byte dense records.  Only
// the first `groups` groups of 32 are fetched.  In pass j of group t
// the kParts lanes of q = l / kParts move record 32 t + j + q kParts, one 16-byte part each
// (cp.async, no registers), so every pass reads 32 / kParts whole records.  Lane l then
// sums its terms in the order l, 32 + l, 64 + l, ..., the same order for every kTPL.
template <int C>
__host__ __device__ constexpr int record_stride() { return C == 3 ? 36 : 20; }
// Records per lane and batch: as many as fit in 40 KB of staging per block, at most 4.
__host__ __device__ constexpr int terms_per_lane(int nt, int rec_words) {
    return (10240 / (nt / 32)) / (32 * rec_words) >= 4 ? 4 : (10240 / (nt / 32)) / (32 * rec_words) >= 2 ? 2 : 1;
}
__host__ __device__ constexpr int max_int(int a, int b) { return a > b ? a : b; }

template <int kRec, int kParts, int kTPL, class Locate>
__device__ __forceinline__ void fetch_records(float *stage, int lane, int groups, Locate locate) {
    static_assert(kParts == 4 || kParts == 8, "64- or 128-byte records");
    const int part = lane & (kParts - 1);
#pragma unroll
    for (int t = 0; t < kTPL; ++t) {
        if (t >= groups) break;   // warp-uniform: the batch's last groups may be past the list
        const float4 *src;
        int parts;
        locate(t, src, parts);
#pragma unroll
        for (int j = 0; j < kParts; ++j) {
            const int r = j + (lane / kParts) * kParts;
            const float4 *p = reinterpret_cast<const float4 *>(
                __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(src), r));
            const int np = __shfl_sync(0xffffffffu, parts, r);
            if (part < np) {
                const unsigned dst =
                    static_cast<unsigned>(__cvta_generic_to_shared(stage + (32 * t + r) * kRec + 4 * part));
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(p + part) : "memory");
            }
        }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Dense record fields in the layout DenseLayout<C> (k_eval_dense).
template <int C>
__device__ __forceinline__ void read_weights(const float *slot, float *wk, uint32_t *ids) {
    if constexpr (C == 3) {
        const float4 a = *reinterpret_cast<const float4 *>(slot + 20);
        const float4 b = *reinterpret_cast<const float4 *>(slot + 24);
        const float2 c = *reinterpret_cast<const float2 *>(slot + 28);
        wk[0] = a.z;
        wk[1] = a.w;
        wk[2] = b.x;
        wk[3] = b.y;
        ids[0] = __float_as_uint(b.z);
        ids[1] = __float_as_uint(b.w);
        ids[2] = __float_as_uint(c.x);
        ids[3] = __float_as_uint(c.y);
    } else {
        const float4 a = *reinterpret_cast<const float4 *>(slot + 8);
        const float4 b = *reinterpret_cast<const float4 *>(slot + 12);
        wk[0] = a.x;
        wk[1] = a.y;
        wk[2] = a.z;
        wk[3] = a.w;
        ids[0] = __float_as_uint(b.x);
        ids[1] = __float_as_uint(b.y);
        ids[2] = __float_as_uint(b.z);
        ids[3] = __float_as_uint(b.w);
    }
}
template <int C>
__device__ __forceinline__ float read_channel(const float *slot, int ch, float *g) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const float2 v = *reinterpret_cast<const float2 *>(slot + 6 * ch + 2 * q);
        g[2 * q] = v.x;
        g[2 * q + 1] = v.y;
    }
    return slot[DenseLayout<C>::kRes + ch];
}

// Reads one record of `n4` 16-byte parts back from a slot.
template <int n4>
__device__ __forceinline__ void read_slot(const float *slot, float *out) {
#pragma unroll
    for (int i = 0; i < n4; ++i) {
        const float4 v = *reinterpret_cast<const float4 *>(slot + 4 * i);
        out[4 * i] = v.x;
        out[4 * i + 1] = v.y;
        out[4 * i + 2] = v.z;
        out[4 * i + 3] = v.w;
    }
}

// Upper-triangle entry e (0..20) of a symmetric 6x6 block -> (a, c), a <= c, row-major order.
__device__ __forceinline__ void tri_decode(int e, int &a, int &c) {
    a = 0;
    c = 0;
#pragma unroll
    for (int r = 0, start = 0; r < 6; start += 6 - r, ++r)
        if (e >= start && e < start + 6 - r) {
            a = r;
            c = r + (e - start);
        }
}

// Regulariser entry (a, c) of the diagonal block: +1e-3 on the diagonal of the origin-twist
// block (PreconditionerRhsBuilder.cu:249-252); for node-centred twists the same term is
// 1e-3 S^T S with S = [[I, 0], [[c]x, I]].
template <class DAcc>
__device__ __forceinline__ DAcc regulariser_entry(int a, int c, float3 cen, bool centred) {
    const DAcc eps = DAcc(1e-3f);
    if (!centred || a >= 3) return a == c ? eps : DAcc(0);
    const DAcc x = cen.x, y = cen.y, z = cen.z;
    const DAcc ca = a == 0 ? x : (a == 1 ? y : z);
    if (c < 3) {
        const DAcc cc = c == 0 ? x : (c == 1 ? y : z);
        return eps * ((a == c ? DAcc(1) + (x * x + y * y + z * z) : DAcc(0)) - ca * cc);
    }
    // -eps [c]x with [c]x = [[0, -z, y], [z, 0, -x], [-y, x, 0]]
    const int k = c - 3;
    DAcc v = DAcc(0);
    if (a == 0) v = k == 1 ? -z : (k == 2 ? y : DAcc(0));
    if (a == 1) v = k == 0 ? z : (k == 2 ? -x : DAcc(0));
    if (a == 2) v = k == 0 ? -y : (k == 1 ? x : DAcc(0));
    return -eps * v;
}

// D += u u^T (upper triangle) and b += v u for one scaled row.
template <class DAcc>
__device__ __forceinline__ void accumulate_row(DAcc *D, DAcc *B, const float *row, float scale, float v) {
    DAcc u[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) u[q] = DAcc(scale * row[q]);
    const DAcc dv = DAcc(v);
#pragma unroll
    for (int a = 0; a < 6; ++a) {
#pragma unroll
        for (int c = a; c < 6; ++c) D[tri_index(a, c)] += u[a] * u[c];
        B[a] += dv * u[a];
    }
}

// NT (threads per block) is chosen by the autotuner among 64, 128 and 256; the work of a
// warp, and so every sum, is the same for all three.
template <class DAcc, int NT, int C>
__global__ void __launch_bounds__(NT, 1024 / NT) k_assemble_node(const Scene *scenes, const Plan *plan,
                                                                     const uint32_t *node_scene, uint32_t total_nodes,
                                                                     const uint32_t *n2t_offset, const uint32_t *n2t_val,
                                                                     uint32_t cap_n2t, const float *drec, const float *rrec,
                                                                     const float *se3, const float4 *centers,
                                                                     const uint32_t *item_ptr, uint32_t cap_items,
                                                                     float *sym_blocks, double *diag64, float *jtr,
                                                                     int *err) {
    constexpr bool kCentred = sizeof(DAcc) == 8;   // mixed precision also uses node-centred twists
    constexpr int kSlot = kSlotWordsF32;             // per-lane partial sums at the end (27 floats)
    constexpr int kRec = record_stride<C>();
    // at most 2 records per lane and 64 registers: 32 warps per SM, which this latency-bound
    // kernel needs more than deeper batches
    constexpr int kTPL = terms_per_lane(NT, kRec) < 2 ? terms_per_lane(NT, kRec) : 2;
    __shared__ __align__(16) float stage[NT / 32][max_int(kTPL * 32 * kRec, 32 * kSlot)];
    const int lane = threadIdx.x & 31;
    float *slots = stage[threadIdx.x >> 5];
    float *mine = slots + lane * kSlot;
    int ea = 0, ec = 0;   // lanes 0..20 finish D(ea, ec), lanes 21..26 finish b
    tri_decode(lane, ea, ec);
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < total_nodes; g += warps) {
        const uint32_t s = node_scene[g];
        const uint32_t beg = n2t_offset[g], end = n2t_offset[g + 1];
        const float4 c4 = centers[g];
        // the list past the first batch, into L2 ahead of the later batches' reads
        if (lane == 0 && end > beg + 32u * kTPL) l2_prefetch_list(n2t_val, beg + 32u * kTPL, end, cap_n2t);
        const Scene &sc = scenes[s];
        const Plan &p = plan[s];
        const uint32_t nd = p.dense_count, ne = sc.num_edges, nn = sc.num_nodes;
        const float lam_d = sc.lam_depth, lam_of = sc.lam_of, lam_r = sc.lam_reg, lam_n = sc.lam_node;
        const bool motion = lam_n != 0.f && sc.node_motion != nullptr;
        const float4 *dbase = reinterpret_cast<const float4 *>(drec + (size_t)DenseLayout<C>::kFloats * p.dense_begin);
        const float4 *rbase = reinterpret_cast<const float4 *>(rrec + (size_t)kRegRecord * sc.edge_base);
        const float3 cen = f3(c4.x, c4.y, c4.z);
        float D[21], B[6];
#pragma unroll
        for (int i = 0; i < 21; ++i) D[i] = 0.f;
#pragma unroll
        for (int i = 0; i < 6; ++i) B[i] = 0.f;
        for (uint32_t base = beg; base < end; base += 32 * kTPL) {
            // 1 dense, 2 regularisation edge, 3 node motion; feature terms have a zero Jacobian
            // (PreconditionerRhsBuilder.cu:214-219)
            auto classify = [&](uint32_t term, const float4 *&src, int &parts) -> int {
                src = nullptr;
                parts = 0;
                if (term < nd) {
                    src = dbase + (size_t)(DenseLayout<C>::kFloats / 4) * term;
                    parts = DenseLayout<C>::kFloats / 4;
                    return 1;
                }
                if (term < nd + ne) {
                    src = rbase + (size_t)(kRegRecord / 4) * (term - nd);
                    parts = kRegRecord / 4;
                    return 2;
                }
                return (term < nd + ne + nn && motion) ? 3 : 0;
            };
            const int groups = (int)min((uint32_t)kTPL, (end - base + 31) / 32);
            fetch_records<kRec, C == 3 ? 8 : 4, kTPL>(slots, lane, groups, [&](int t, const float4 *&src, int &parts) {
                const uint32_t it = base + 32 * t + lane;
                classify(it < end ? n2t_val[it] : kInvalidIndex, src, parts);
            });
            __syncwarp();
#pragma unroll 1
            for (int t = 0; t < groups; ++t) {
                const uint32_t it = base + 32 * t + lane;
                const uint32_t term = it < end ? n2t_val[it] : kInvalidIndex;
                const float4 *src_unused;
                int parts_unused;
                const int kind = classify(term, src_unused, parts_unused);
                const float *rec_t = slots + (32 * t + lane) * kRec;
                if (kind == 1) {
                    // point-to-plane + optical-flow rows (libs/star/opt/dense_image_jacobian.cuh:9-20)
                    float wk[4];
                    uint32_t ids[4];
                    read_weights<C>(rec_t, wk, ids);
                    float w = wk[0];   // weight of the last slot whose node is g
#pragma unroll
                    for (int k = 1; k < 4; ++k) if (ids[k] == g) w = wk[k];
#pragma unroll
                    for (int ch = 0; ch < C; ++ch) {
                        float gl[6];
                        const float res = read_channel<C>(rec_t, ch, gl);
                        if (kCentred) recentre(gl, cen);
                        const float scale = (ch == 0 ? lam_d : lam_of) * w;
                        accumulate_row(D, B, gl, scale, -(scale * res));
                    }
                } else if (kind == 2) {
                    // regularisation rows (node_graph_reg_jacobian.cuh:85-106, 193-233)
                    float rec[kRegRecord];
                    read_slot<kRegRecord / 4>(rec_t, rec);
                    if (rec[7] != 0.f) {
                        const float3 a3 = f3(rec[0], rec[1], rec[2]), b3 = f3(rec[3], rec[4], rec[5]);
                        float J[3][6];
                        reg_unit_jacobian(a3, b3, __float_as_uint(rec[8]) == g, J);
                        const float scale = lam_r * rec[6];
#pragma unroll
                        for (int ch = 0; ch < 3; ++ch) {
                            if (kCentred) recentre(J[ch], cen);
                            accumulate_row(D, B, J[ch], scale, -(scale * rec[10 + ch]));
                        }
                    }
                } else if (kind == 3) {
                    // node-motion rows (node_motion_jacobian.cuh:7-36), lambda_node = 0 by default
                    const uint32_t nl = term - nd - ne;
                    const float4 pred = sc.node_motion[nl];
                    const SE3f T = dq_se3(load_dq(se3 + 8ull * (sc.node_base + nl)));
                    const float res3[3] = {T.t.x - pred.x, T.t.y - pred.y, T.t.z - pred.z};
                    const float scale = lam_n * pred.w;
#pragma unroll
                    for (int ch = 0; ch < 3; ++ch) {
                        float J[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                        J[3 + ch] = 1.f;
                        if (kCentred) recentre(J, cen);
                        accumulate_row(D, B, J, scale, -(scale * res3[ch]));
                    }
                }
            }
            __syncwarp();
        }
        // lane partial sums -> slots; lane e sums entry e over the lanes in lane order
#pragma unroll
        for (int i = 0; i < 21; ++i) mine[i] = D[i];
#pragma unroll
        for (int i = 0; i < 6; ++i) mine[21 + i] = B[i];
        __syncwarp();
        DAcc acc = DAcc(0);
        if (lane < 27) {
#pragma unroll 8
            for (int l = 0; l < 32; ++l) acc += DAcc(slots[l * kSlot + lane]);
        }
        __syncwarp();
        if (lane < 21) {
            acc += regulariser_entry<DAcc>(ea, ec, cen, kCentred);
            float *blk = sym_blocks + 36ull * min(item_ptr[g], cap_items - 1);   // the row's first item
            blk[6 * ea + ec] = (float)acc;
            blk[6 * ec + ea] = (float)acc;
            if (kCentred) diag64[21ull * g + lane] = (double)acc;
        } else if (lane < 29) {
            const float bq = lane < 27 ? (float)acc : 0.f;
            jtr[8ull * g + (lane - 21)] = bq;
            if (isnan(bq)) set_err(err, WS_ERR_NAN);
        }
    }
}

// ---------------------------------------------------------------------------
// Block-diagonal preconditioner, one thread per node: FP64 Cholesky of the FP64
// accumulated block (mixed precision) or the reference's FP32 Gauss-Jordan with
// partial pivoting of the stored block (BlockDiagonalPreconditionerInverse.cuh:14-73).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_block_inverse(const double *diag64, const float *sym_blocks,
                                                       const uint32_t *item_ptr, uint32_t cap_items,
                                                       uint32_t total_nodes, int fp64, float *inv_diag) {
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total_nodes; g += gridDim.x * blockDim.x) {
        float inv[36];
        if (fp64) {
            double Dd[36];
            const double *src = diag64 + 21ull * g;
#pragma unroll
            for (int a = 0; a < 6; ++a)
#pragma unroll
                for (int c = a; c < 6; ++c) {
                    const double v = src[tri_index(a, c)];
                    Dd[6 * a + c] = v;
                    Dd[6 * c + a] = v;
                }
            cholesky6_fp64(Dd, inv);
        } else {
            float full[36];
#pragma unroll
            for (int i = 0; i < 36; ++i) full[i] = sym_blocks[36ull * min(item_ptr[g], cap_items - 1) + i];
            gauss_jordan6(full, inv);
        }
        float4 *o = reinterpret_cast<float4 *>(inv_diag + 36ull * g);
#pragma unroll
        for (int i = 0; i < 9; ++i) o[i] = make_float4(inv[4 * i], inv[4 * i + 1], inv[4 * i + 2], inv[4 * i + 3]);
    }
}

// ---------------------------------------------------------------------------
// Off-diagonal blocks, once per unordered node pair (i < j) over the pair's term list
// (computeDenseImageJtJBlockJacobian, dense_image_jacobian.cuh:82-126; computeRegJtJLocalBlock,
// node_graph_reg_jacobian.cuh:273-358), stored once per pair; the lower-triangle CSR entry reads
// it transposed.
// A dense term's Jacobian rows for the two nodes are the same gradient g scaled by the
// nodes' skinning weights, so the dense part of the block is  sum s g_i g_j^T  with
// s = lambda^2 w_i w_j.  With node-centred twists g_j = S g_i, S = [[I, -[c_j - c_i]x], [0, I]]
// (g_i, g_j: g centred at the row and column nodes), hence the block is  M S^T  with the
// symmetric  M = sum s g_i g_i^T.  Lanes take terms and sum the 21 entries of M in registers;
// the lanes' sums are added in lane order through shared memory, M S^T is formed once per
// pair, and the pair's smoothness terms (at most one per edge direction) are added last, in
// list order, by the whole warp.
// ---------------------------------------------------------------------------
// v[i] for a run-time i < 6, by selects (no local-memory array).
__device__ __forceinline__ float pick6(const float *v, int i) {
    float r = v[0];
#pragma unroll
    for (int k = 1; k < 6; ++k) r = i == k ? v[k] : r;
    return r;
}

template <int NT, int C>
__global__ void __launch_bounds__(NT, 1024 / NT) k_assemble_pair(
    const Scene *scenes, const Plan *plan, const uint32_t *counts,
    const uint32_t *half_row, const uint32_t *half_col, const uint32_t *half_begin, const uint32_t *half_end,
    const uint32_t *half_scene, const uint32_t *pair_val, uint32_t cap_kv, const uint32_t *slot_up, const float *drec, const float *rrec,
    const float4 *centers, int centred, float *sym_blocks, int *err) {
    constexpr int kSlot = kSlotWordsF32;   // per-lane partial sums at the end
    static_assert(kSlot >= 36, "a slot holds one lane's 36 partial sums");
    constexpr int kRec = record_stride<C>();
    // at most 2 records per lane: the staging then leaves room for 32 warps per SM, which
    // this latency-bound kernel needs more than deeper batches (pair lists are short)
    constexpr int kTPL = terms_per_lane(NT, kRec) < 2 ? terms_per_lane(NT, kRec) : 2;
    constexpr int kStageWords = max_int(kTPL * 32 * kRec, 32 * kSlot);
    constexpr int kStash = 4;   // smoothness terms per pair: one per edge direction, so at most 2
    __shared__ __align__(16) float stage[NT / 32][kStageWords + kStash * kRegRecord];
    const int lane = threadIdx.x & 31;
    float *slots = stage[threadIdx.x >> 5];
    float *stash = slots + kStageWords;   // the pair's smoothness records, in list order
    float *mine = slots + lane * kSlot;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t nhalf = counts[kCntHalf];
    // grid-stride: at any time the warps work on neighbouring pairs, whose term records overlap,
    // so the records are read from DRAM about once and then from L2
    for (uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; h < nhalf; h += warps) {
        // the pair's words in one round of loads (its scene among them), then its slot check
        const uint32_t slot = slot_up[h], row = half_row[h], col = half_col[h], beg = half_begin[h],
                       end = half_end[h], s = half_scene[h];
        // the term list of this warp's next pair, into L2 a pair ahead (its bounds come with this
        // pair's words)
        uint32_t next_beg = 0, next_end = 0;
        if (lane == 0 && h + warps < nhalf) {
            next_beg = half_begin[h + warps];
            next_end = half_end[h + warps];
        }
        if (lane == 0 && next_end > next_beg) l2_prefetch_list(pair_val, next_beg, next_end, cap_kv);
        if (slot == kInvalidIndex) continue;   // capacity overflow, already flagged
        const Scene &sc = scenes[s];
        const Plan &p = plan[s];
        const uint32_t nd = p.dense_count, ne = sc.num_edges;
        const float lam_d = sc.lam_depth, lam_of = sc.lam_of, lam_r = sc.lam_reg;
        const float4 *dbase = reinterpret_cast<const float4 *>(drec + (size_t)DenseLayout<C>::kFloats * p.dense_begin);
        const float4 *rbase = reinterpret_cast<const float4 *>(rrec + (size_t)kRegRecord * sc.edge_base);
        const float4 cr4 = centers[row], cc4 = centers[col];
        const float3 c_row = f3(cr4.x, cr4.y, cr4.z), c_col = f3(cc4.x, cc4.y, cc4.z);
        float M[21];
#pragma unroll
        for (int i = 0; i < 21; ++i) M[i] = 0.f;
        int nreg = 0;   // warp-uniform: smoothness records stashed so far
        for (uint32_t base = beg; base < end; base += 32 * kTPL) {
            // 1 dense, 2 regularisation edge (stashed, added after the dense sums); node-motion
            // terms own no pairs
            auto classify = [&](uint32_t term, const float4 *&src, int &parts) -> int {
                src = nullptr;
                parts = 0;
                if (term < nd) {
                    src = dbase + (size_t)(DenseLayout<C>::kFloats / 4) * term;
                    parts = DenseLayout<C>::kFloats / 4;
                    return 1;
                }
                if (term < nd + ne) {
                    src = rbase + (size_t)(kRegRecord / 4) * (term - nd);
                    parts = kRegRecord / 4;
                    return 2;
                }
                return 0;
            };
            const int groups = (int)min((uint32_t)kTPL, (end - base + 31) / 32);
            fetch_records<kRec, C == 3 ? 8 : 4, kTPL>(slots, lane, groups, [&](int t, const float4 *&src, int &parts) {
                const uint32_t it = base + 32 * t + lane;
                classify(it < end ? pair_val[it] : kInvalidIndex, src, parts);
            });
            __syncwarp();
#pragma unroll 1
            for (int t = 0; t < groups; ++t) {
                const uint32_t it = base + 32 * t + lane;
                const float4 *src_unused;
                int parts_unused;
                const int kind = classify(it < end ? pair_val[it] : kInvalidIndex, src_unused, parts_unused);
                const float *rec_t = slots + (32 * t + lane) * kRec;
                const unsigned regs = __ballot_sync(0xffffffffu, kind == 2);
                if (kind == 2) {
                    const int k = nreg + __popc(regs & ((1u << lane) - 1u));
                    if (k < kStash) {
#pragma unroll
                        for (int q = 0; q < kRegRecord / 4; ++q)
                            reinterpret_cast<float4 *>(stash + kRegRecord * k)[q] =
                                reinterpret_cast<const float4 *>(rec_t)[q];
                    } else {
                        set_err(err, WS_ERR_CAPACITY);
                    }
                }
                nreg += __popc(regs);
                if (kind != 1) continue;
                float wk[4];
                uint32_t ids[4];
                read_weights<C>(rec_t, wk, ids);
                float wi = wk[0], wj = wk[0];   // last matching slots
#pragma unroll
                for (int k = 1; k < 4; ++k) {
                    if (ids[k] == row) wi = wk[k];
                    if (ids[k] == col) wj = wk[k];
                }
#pragma unroll
                for (int ch = 0; ch < C; ++ch) {
                    float g[6], u[6];
                    read_channel<C>(rec_t, ch, g);
                    if (centred) recentre(g, c_row);
                    const float lam = ch == 0 ? lam_d : lam_of;
                    const float sc2 = (lam * wi) * (lam * wj);
#pragma unroll
                    for (int q = 0; q < 6; ++q) u[q] = sc2 * g[q];
#pragma unroll
                    for (int i = 0; i < 6; ++i)
#pragma unroll
                        for (int j = i; j < 6; ++j) M[tri_index(i, j)] += u[i] * g[j];
                }
            }
            __syncwarp();
        }
        // lane sums of M -> slots; lane e < 21 sums entry e over the lanes in lane order
#pragma unroll
        for (int i = 0; i < 21; ++i) mine[i] = M[i];
        __syncwarp();
        float m = 0.f;
        if (lane < 21) {
#pragma unroll 8
            for (int l = 0; l < 32; ++l) m += slots[l * kSlot + lane];
        }
        __syncwarp();
        if (lane < 21) {   // the full symmetric M, row-major, in slots[0, 36)
            int ea = 0, ec = 0;
            tri_decode(lane, ea, ec);
            slots[6 * ea + ec] = m;
            slots[6 * ec + ea] = m;
        }
        __syncwarp();
        // A = M S^T: A[:, 0:3] = M[:, 0:3] + M[:, 3:6] [c_col - c_row]x, A[:, 3:6] = M[:, 3:6]
        const float3 dc = f3(c_col.x - c_row.x, c_col.y - c_row.y, c_col.z - c_row.z);
        auto entry = [&](int e) -> float {
            const int r = e / 6, c = e % 6;
            float v = slots[e];
            if (centred && c < 3) {
                const float *mr = slots + 6 * r + 3;
                // column c of [d]x = [[0, -dz, dy], [dz, 0, -dx], [-dy, dx, 0]]
                const float k0 = c == 0 ? 0.f : (c == 1 ? -dc.z : dc.y);
                const float k1 = c == 0 ? dc.z : (c == 1 ? 0.f : -dc.x);
                const float k2 = c == 0 ? -dc.y : (c == 1 ? dc.x : 0.f);
                v += mr[0] * k0 + mr[1] * k1 + mr[2] * k2;
            }
            return v;
        };
        float acc0 = entry(lane), acc1 = lane < 4 ? entry(32 + lane) : 0.f;   // entries lane, 32 + lane
        // smoothness rows (node_graph_reg_jacobian.cuh:85-106, 193-233), in list order
        const int r0 = lane / 6, c0 = lane % 6, r1 = (32 + lane) / 6, c1 = (32 + lane) % 6;
        for (int k = 0; k < min(nreg, kStash); ++k) {
            const float *rec = stash + kRegRecord * k;
            if (rec[7] == 0.f) continue;   // validity
            const float3 a3 = f3(rec[0], rec[1], rec[2]), b3 = f3(rec[3], rec[4], rec[5]);
            const uint32_t ei = __float_as_uint(rec[8]);
            float Jr[3][6], Jc[3][6];
            reg_unit_jacobian(a3, b3, row == ei, Jr);
            reg_unit_jacobian(a3, b3, col == ei, Jc);
            const float scale = lam_r * rec[6];
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) {
                if (centred) {
                    recentre(Jr[ch], c_row);
                    recentre(Jc[ch], c_col);
                }
                acc0 += (scale * pick6(Jr[ch], r0)) * (scale * pick6(Jc[ch], c0));
                if (lane < 4) acc1 += (scale * pick6(Jr[ch], r1)) * (scale * pick6(Jc[ch], c1));
            }
        }
        __syncwarp();
        // item h + row + 1 of the symmetric store: the row's diagonal item and its earlier pairs
        // precede it; row-major, rows of node `row`, columns of node `col`
        float *blk = sym_blocks + 36ull * (h + row + 1);
        blk[lane] = acc0;
        if (lane < 4) blk[32 + lane] = acc1;
    }
}

// ---------------------------------------------------------------------------
// Persistent block PCG (BlockPCG<6>::SolveNoConvergeCheck,
// libs/star/pcg_solver/BlockPCG.cuh:67-190, 325-484) for every scene of the batch.
//
// Rows (nodes) are grouped in scene-aligned groups of kRowsPerGroup.  Phase A (the SpMV) works on
// units, contiguous ranges of groups balanced by stored blocks (kPcgUnitsPerWarp per warp);
// phase B on units of bunit_groups row groups (about kPcgBUnitsPerWarp per warp on small problems,
// whole steps of at least 64 rows on large batches).  The scenes are
// split at a scene boundary into two halves, X and Y, that run half a phase apart: step k of the
// schedule holds X's phase A of iteration k/2 with Y's phase B of iteration k/2 - 1 (k even), or
// X's phase B with Y's phase A of iteration (k-1)/2 (k odd), the two parts' units interleaved in
// proportion.  So at any time some warps stream blocks from DRAM while others do the
// latency-bound per-row work.  The warps take the units by ticket from one counter that grows
// through the launch (the schedule's units in order), so the warps that finish early take the
// remaining units instead of waiting for the slowest.  A unit depends only on units of its
// scenes in the step before, which have smaller tickets, and a warp finishes its unit before it
// takes the next ticket, so the smallest unfinished ticket can always proceed.  Init and the
// twist update take equal numbers of groups per warp.  No block-level synchronisation.
// Per iteration: phase A  d = s + beta d (recomputed for neighbours from s and the
// previous d), q = A d from each stored block read once (the transposed products go
// to the lower rows through a contribution buffer), <d, A d>;  phase B  alpha,
// q += the row's contributions, x += alpha d, r -= alpha q, s = M^-1 r, <r, s>.
// A warp keeps its group's partial in FP64 registers, stores it, and the last group
// of a scene to finish (a fenced atomic ticket) sums that scene's group partials in
// group order, publishes alpha or beta and bumps the scene's generation counter; the
// sums therefore never depend on the rest of the batch.  Before a unit a warp waits only for
// the scenes of the unit's rows; a wait is bounded, and a timed-out wait sets WS_ERR_TIMEOUT and
// the warp leaves.
// ---------------------------------------------------------------------------

struct PcgArgs {
    const Scene *scenes;
    const uint32_t *group_scene, *group_row;
    uint32_t total_groups;
    const uint32_t *rowptr;        // block-CSR row pointers (lower slots follow the diagonal)
    const uint32_t *item_ptr;      // [nodes + 1] first item of every row in the symmetric store
    const uint2 *item_info;        // per item: column | kItemRowStart, lower entry (upper) or scene (diagonal)
    const uint32_t *item_col;      // per item: column | kItemRowStart on a row's diagonal item
    // [units + 2]: first row group of each phase-A work unit, then the group count, then the
    // number of units of the first half (X) of the scenes
    const uint32_t *warp_groups;
    // [2 * units]: per phase-A unit {first group, end group, first row, end row}, {first item,
    // end item, scene of the first group, scene of the last group}
    const uint4 *unit_info;
    uint32_t total_units;          // kPcgUnitsPerWarp x the launch's warps
    uint32_t split_group;          // first group of the second half (Y) of the scenes
    uint32_t *tickets;             // work-unit tickets, growing through a launch (zeroed before it)
    uint32_t bunit_groups;         // row groups of a phase-B unit
    const float *sym_blocks;       // per item: the 6x6 block, row-major
    const float *inv_diag, *jtr;
    float *contrib;                // per lower entry (row j, column i < j): B^T v_i left for row j (6 floats)
    float *x, *r, *q;
    float *sd0, *sd1;         // [node][kSdStride]: s (6) then d (6); swapped every iteration
    double *group_partial;
    double *scalars;          // per scene: [0] delta, [1] alpha, [2] beta, [3] last reduced value
    // per scene, kSceneSync words: [0] phase-A tickets, [1] phase-B / init tickets (arrivals of
    // row groups, growing during a launch), [32] alpha generation, [33] delta/beta generation
    // (bumped when published)
    uint32_t *scene_counter;
    uint32_t cap_blocks, cap_half, cap_items, total_nodes, num_scenes;
    int *err;
    float *se3;
    const float4 *centers;
    int pcg_iters;
    int fp64;                 // FP64 reductions and node-centred twists
};

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;   // requested sleep, about two seconds
constexpr int kSceneSync = 64;        // words per scene in scene_counter (tickets and generations on separate lines)


__device__ __forceinline__ float ldcg(const float *p) { return __ldcg(p); }
__device__ __forceinline__ double ldcg(const double *p) { return __ldcg(p); }

// ---------------------------------------------------------------------------
// Scene reductions.  Every row group writes its partial to group_partial[g]; a warp then
// publishes all groups of its range at once: one fence, and per scene one atomicAdd of the
// number of its groups in that scene.  The arrival that completes the scene's count sums
// the scene's partials in group order (so the value does not depend on who arrives last)
// and updates the scene scalars.
// mode 0: alpha = delta / sum;  mode 1: beta = sum / delta, delta = sum;  mode 2 (init): delta = sum, beta = 0.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void reduce_scene(const PcgArgs &A, uint32_t scene, int mode, int lane) {
    const Scene &sc = A.scenes[scene];
    double v = 0.0;
#pragma unroll 8
    for (int c = lane; c < sc.num_chunks; c += 32) v += __ldcg(A.group_partial + sc.chunk_base + c);
    v = warp_sum(v);
    if (lane == 0) {
        double *S = A.scalars + 8ull * scene;
        if (!A.fp64) v = (double)(float)v;
        if (mode == 0) {
            const double delta = __ldcg(S + 0);
            double alpha = (v != 0.0) ? delta / v : 0.0;
            if (!A.fp64 && v != 0.0) alpha = (double)((float)delta / (float)v);
            S[1] = alpha;
        } else {
            const double delta_old = __ldcg(S + 0);
            double beta = (delta_old != 0.0) ? v / delta_old : 0.0;
            if (!A.fp64 && delta_old != 0.0) beta = (double)((float)v / (float)delta_old);
            S[2] = (mode == 2) ? 0.0 : beta;
            S[0] = v;
        }
        S[3] = v;
        __threadfence();
        // every group of the scene has finished the phase and its scalar is written
        atomicAdd(&A.scene_counter[kSceneSync * scene + 32 + (mode == 0 ? 0 : 1)], 1u);
    }
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Waits until every scene that owns one of the warp's groups has published generation
// `target` of `which` (0: alpha, 1: delta and beta).  Lanes that start a run of a new
// scene wait for that scene; the wait sleeps with backoff and gives up after about two
// seconds of requested sleep (or at once when another warp has already timed out).
__device__ bool wait_scenes(const PcgArgs &A, uint32_t g_begin, uint32_t g_end, int which, uint32_t target,
                            int lane) {
    bool ok = true;
    for (uint32_t base = g_begin; base < g_end; base += 32) {
        const uint32_t g = base + lane;
        const uint32_t sc = g < g_end ? A.group_scene[g] : kInvalidIndex;
        const uint32_t prev = __shfl_up_sync(0xffffffffu, sc, 1);
        if (g < g_end && (lane == 0 || prev != sc)) {
            const uint32_t *gen = A.scene_counter + (size_t)kSceneSync * sc + 32 + which;
            unsigned long long waited_ns = 0;
            unsigned sleep_ns = 32;
            while (ld_acquire(gen) < target) {
                if (waited_ns > kBarrierTimeoutNs || *reinterpret_cast<volatile int *>(A.err) == WS_ERR_TIMEOUT) {
                    set_err(A.err, WS_ERR_TIMEOUT);
                    ok = false;
                    break;
                }
                __nanosleep(sleep_ns);
                waited_ns += sleep_ns;
                sleep_ns = min(sleep_ns * 2u, 256u);
            }
        }
        __syncwarp();
    }
    // the polling lanes' acquire loads, then this barrier, order the whole warp's later reads of
    // the scenes' vectors and scalars after the publications they saw
    ok = __all_sync(0xffffffffu, ok);
    return ok;
}

// wait_scenes for a unit whose groups all lie in one scene: lane 0 polls that scene's generation.
__device__ bool wait_one_scene(const PcgArgs &A, uint32_t scene, int which, uint32_t target, int lane) {
    bool ok = true;
    if (lane == 0) {
        const uint32_t *gen = A.scene_counter + (size_t)kSceneSync * min(scene, A.num_scenes - 1) + 32 + which;
        unsigned long long waited_ns = 0;
        unsigned sleep_ns = 32;
        while (ld_acquire(gen) < target) {
            if (waited_ns > kBarrierTimeoutNs || *reinterpret_cast<volatile int *>(A.err) == WS_ERR_TIMEOUT) {
                set_err(A.err, WS_ERR_TIMEOUT);
                ok = false;
                break;
            }
            __nanosleep(sleep_ns);
            waited_ns += sleep_ns;
            sleep_ns = min(sleep_ns * 2u, 256u);
        }
    }
    // lane 0's acquire load, then this barrier, order the warp's later reads
    return __all_sync(0xffffffffu, __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0);
}

// Failure-detection self-test: one warp runs wait_scenes on one scene whose generation
// nothing advances.  With the bound in place it gives up after about two seconds of requested
// sleep and leaves WS_ERR_TIMEOUT in `err`; the launch then ends like any other.
__global__ void k_wait_selftest(PcgArgs A) {
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < 32) wait_scenes(A, 0u, 1u, 0, 1u, lane);
}

cudaError_t pcg_wait_selftest(int *status, cudaStream_t st) {
    // scene_counter: one scene's kSceneSync words, all zero; group_scene: group 0 -> scene 0; err
    uint32_t *words = nullptr;
    const size_t n_words = kSceneSync + 1 + 1;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&words), 4 * n_words, st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(words, 0, 4 * n_words, st);
    PcgArgs a{};
    a.scene_counter = words;
    a.group_scene = words + kSceneSync;
    a.err = reinterpret_cast<int *>(words + kSceneSync + 1);
    int flag = 0;
    if (e == cudaSuccess) {
        k_wait_selftest<<<1, 32, 0, st>>>(a);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, a.err, 4, cudaMemcpyDeviceToHost, st);
    const cudaError_t f = cudaFreeAsync(words, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = f;
    *status = flag;
    return e;
}

// `phase` counts the publications of the counter: phase A(it) is phase it of counter 0; init
// is phase 0 and phase B(it) phase it + 1 of counter 1.  The tickets only grow during a
// launch, so the arrival that brings them to (phase + 1) times the scene's group count is
// the last one, and no reset sits between the publications.
__device__ void publish_range(const PcgArgs &A, uint32_t g_begin, uint32_t g_end, int mode, int phase, int lane) {
    if (g_begin >= g_end) return;
    __threadfence();   // every lane's vector and partial writes of the phase before the tickets
    __syncwarp();
    const uint32_t ctr = (mode == 0) ? 0u : 1u;
    for (uint32_t base = g_begin; base < g_end; base += 32) {
        const uint32_t g = base + lane;
        const uint32_t sc = g < g_end ? A.group_scene[g] : kInvalidIndex;
        const uint32_t prev = __shfl_up_sync(0xffffffffu, sc, 1);
        const unsigned starts = __ballot_sync(0xffffffffu, g < g_end && (lane == 0 || prev != sc));
        const unsigned inside = __ballot_sync(0xffffffffu, g < g_end);
        for (unsigned m = starts; m; m &= m - 1) {
            const int s0 = __ffs(m) - 1;
            const unsigned later = m & (m - 1);
            const int s1 = later ? __ffs(later) - 1 : 32 - __clz(inside);
            const uint32_t scene = __shfl_sync(0xffffffffu, sc, s0);
            int last = 0;
            if (lane == 0) {
                const uint32_t n = (uint32_t)(s1 - s0);
                const uint32_t ticket = atomicAdd(&A.scene_counter[kSceneSync * scene + ctr], n);
                last = (ticket + n == (uint32_t)A.scenes[scene].num_chunks * (uint32_t)(phase + 1)) ? 1 : 0;
            }
            if (__shfl_sync(0xffffffffu, last, 0)) reduce_scene(A, scene, mode, lane);
        }
    }
}

// Sum over the kRowsPerGroup lanes of one group (fixed butterfly inside the group).
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
    for (int o = kRowsPerGroup / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
    for (int o = kRowsPerGroup / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// <u, v> over 6 entries in the precision of the mode, summed over the group's nodes.
__device__ __forceinline__ double node_dot_group(const PcgArgs &A, const float *u, const float *v, bool valid) {
    if (A.fp64) {
        double p = 0.0;
        if (valid)
#pragma unroll
            for (int i = 0; i < 6; ++i) p += (double)u[i] * (double)v[i];
        return group_sum(p);
    }
    float p = 0.f;
    if (valid)
#pragma unroll
        for (int i = 0; i < 6; ++i) p += u[i] * v[i];
    return (double)group_sum(p);
}

__device__ __forceinline__ void load6(const float *p, float *v) {
    const float4 a = __ldcg(reinterpret_cast<const float4 *>(p));
    const float2 b = __ldcg(reinterpret_cast<const float2 *>(p + 4));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y;
}
__device__ __forceinline__ void load6_f2(const float *p, float *v) {   // 8-byte aligned source
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float2 a = __ldcg(reinterpret_cast<const float2 *>(p) + k);
        v[2 * k] = a.x;
        v[2 * k + 1] = a.y;
    }
}
__device__ __forceinline__ void store6(float *p, const float *v) {
    reinterpret_cast<float4 *>(p)[0] = make_float4(v[0], v[1], v[2], v[3]);
    reinterpret_cast<float2 *>(p + 4)[0] = make_float2(v[4], v[5]);
}
// y = M x for one node's 6x6 block (row-major), consumed a float4 at a time.
__device__ __forceinline__ void matvec6(const float *M, const float *x, float *y) {
#pragma unroll
    for (int i = 0; i < 6; ++i) y[i] = 0.f;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const float4 v = __ldg(reinterpret_cast<const float4 *>(M) + q);
        const float e4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int e = 4 * q + k;
            y[e / 6] += e4[k] * x[e % 6];
        }
    }
}

// ---------------------------------------------------------------------------
// Symmetric block SpMV over one warp's rows, each stored block read once.
// The block store holds, row by row, the diagonal block and then the blocks of the row's
// upper pairs (column > row) in column order; these are the row's items
// u = item_ptr[row] .. item_ptr[row + 1).  For item (i, j) with block B (rows of node i,
// columns of node j) the lane forms a = B v_j, which is added to row i, and, off the
// diagonal, t = B^T v_i, which it stores as lower entry (row j, column i); lower entries
// are numbered by row, then column, so the owner of row j adds its contributions
// afterwards from one contiguous range, in column order (the CSR slot order).
// A warp's items are contiguous, so its blocks stream in as whole lines:
//   * the 32 blocks of a chunk (4608 contiguous bytes) arrive as one 1-D bulk copy
//     (cp.async.bulk, issued by lane 0, its bytes counted on the buffer's mbarrier) into one of
//     two buffers; a buffer takes the copy of the chunk two ahead as soon as the lanes hold its
//     blocks in registers, and the blocks of the chunk three ahead are requested into L2 by a
//     bulk prefetch; both carry an evict-first L2 policy, so that the blocks, read once per
//     iteration, leave L2 before the vectors and contributions the iteration reads back;
//   * the item records (8 bytes) of chunk j + 2 are loaded while chunk j is computed, and the
//     column s/d records (48 bytes, cp.async) of chunk j + 1;
//   * a row's diagonal item (always its first) publishes v_i and its scene's beta through a
//     ring in shared memory, where the row's later items, in this chunk or a later one, read
//     them; rows follow from counting the items that start a row;
//   * the lane that ends a row sums the row's products in item order, continuing a row
//     that began in an earlier chunk from a carried partial sum.
// This is phase A of a PCG iteration: v = d = s + beta d_old (recomputed for every column
// from the s/d record of the previous iteration), q without its lower part, and per row
// <d_i, (A d)_i> summed over the row's items as d_i . a, twice for an off-diagonal item
// (it stands for both orientations).
// Each row's sums run over its items in a fixed order whatever the chunk alignment, so
// results do not depend on which warp handled the row or on the batch.
// ---------------------------------------------------------------------------
constexpr int kPcgThreads = 128;                              // 4 warps per block
constexpr int kPcgBlockFloats = 32 * 36;                      // one chunk's blocks
constexpr int kPcgRecFloats = 32 * kSdStride;                 // one chunk's column records
constexpr int kPcgRing = 64;                                  // rows kept in the per-warp rings
// per warp: two block buffers, two record buffers, the v/beta ring (8 floats a row), the
// <d, A d> ring (a double a row) and two mbarriers; a multiple of 4 floats, so that every
// warp's block buffers start on the 16-byte boundary a bulk copy needs
constexpr int kPcgWarpFloats = 2 * kPcgBlockFloats + 2 * kPcgRecFloats + kPcgRing * 8 + 2 * kPcgRing + 4;
static_assert(kPcgWarpFloats % 4 == 0, "warp areas on 16-byte boundaries");
constexpr size_t kPcgSmemBytes = sizeof(float) * kPcgWarpFloats * (kPcgThreads / 32);
// polls of an mbarrier phase before a wait gives up (each poll may suspend the thread a while)
constexpr int kBulkMaxPolls = 1 << 22;

__device__ __forceinline__ unsigned smem_addr(const void *p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
// L2 policy of the block streams: each stored block is read once per product, so its lines are
// the first to leave L2, and the vectors, item records and contributions that the same product
// reads back stay there.
__device__ __forceinline__ uint64_t evict_first_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(pol));
    return pol;
}
// Lane 0: the blocks of items u .. u + 31 (below u_end) into `buf` by one bulk copy whose bytes
// complete the current phase of `bar`, with L2 policy `pol`; past the range, a plain arrival
// completes it.  The proxy fence orders the lanes' earlier reads of `buf` (ordered before it by a
// __syncwarp) before the bulk copy's writes.  Block addresses are multiples of 144 bytes from a
// 256-byte aligned base, so every copy starts on a 16-byte boundary and moves a multiple of 16 bytes.
__device__ __forceinline__ void bulk_blocks(const float *blocks, uint32_t u, uint32_t u_end, float *buf,
                                            unsigned long long *bar, uint64_t pol) {
    if (u >= u_end) {
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(bar)) : "memory");
        return;
    }
    const unsigned bytes = 144u * min(32u, u_end - u);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;\n"
        ::"r"(smem_addr(buf)), "l"(blocks + 36ull * u), "r"(bytes), "r"(smem_addr(bar)), "l"(pol)
        : "memory");
}
// Lane 0: `n` mbarriers, each completed by one arrival (with its copy's bytes).
__device__ __forceinline__ void bulk_init(unsigned long long *bars, int n) {
    for (int k = 0; k < n; ++k)
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bars + k)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// Waits for phase `parity` of `bar` to complete; false when kBulkMaxPolls polls ran out.  The
// warp agrees on the outcome, so a timeout leaves it converged.
__device__ __forceinline__ bool bulk_wait(unsigned long long *bar, unsigned parity) {
    bool ok = false;
    for (int i = 0; i < kBulkMaxPolls && !ok; ++i) {
        unsigned done;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(done)
                     : "r"(smem_addr(bar)), "r"(parity)
                     : "memory");
        ok = done != 0;
    }
    return __all_sync(0xffffffffu, ok);
}


// Item record: column | kItemRowStart on a row's diagonal item, then the lower entry of the
// transposed use (upper item) or the row's scene (diagonal item); column kInvalidIndex past
// the end of the range.  Loaded raw and only read one chunk later, so the load never stalls
// the warp.
__device__ __forceinline__ uint2 load_item(const uint2 *info, uint32_t u, uint32_t end) {
    uint2 v = make_uint2(kInvalidIndex, kInvalidIndex);
    if (u < end) v = __ldg(info + u);
    return v;
}

// Asks L2 for the blocks of items u .. u + 31 (below u_end) ahead of their bulk copies: one
// bulk prefetch of up to 32 contiguous 144-byte blocks, issued by one lane, with L2 policy `pol`.
__device__ __forceinline__ void l2_prefetch_blocks(const float *blocks, uint32_t u, uint32_t u_end, uint64_t pol) {
    if (u < u_end) {
        const uint32_t bytes = 144u * min(32u, u_end - u);
        asm volatile("cp.async.bulk.prefetch.L2.global.L2::cache_hint [%0], %1, %2;\n" ::"l"(blocks + 36ull * u),
                     "r"(bytes), "l"(pol)
                     : "memory");
    }
}

__device__ __forceinline__ void cp_async16(float *dst, const float *src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prior() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Starts the column side of a chunk: each lane copies its item's s/d record (3 x 16 B) into
// its slot of `recs` and, on a diagonal item, loads its scene's beta into `beta`.
__device__ __forceinline__ void issue_records(const PcgArgs &A, const float *vec_in, uint2 it, float *recs, int lane,
                                             float &beta) {
    beta = 0.f;
    if (it.x != kInvalidIndex) {
        const float *src = vec_in + (size_t)kSdStride * min(it.x & ~kItemRowStart, A.total_nodes - 1);
        float *dst = recs + kSdStride * lane;
#pragma unroll
        for (int p = 0; p < kSdStride / 4; ++p) cp_async16(dst + 4 * p, src + 4 * p);
        if (it.x & kItemRowStart) beta = (float)__ldcg(A.scalars + 8ull * min(it.y, A.num_scenes - 1) + 2);
    }
    cp_async_commit();
}

__device__ __forceinline__ void store6_f2(float *p, const float *v) {   // 8-byte aligned destination
#pragma unroll
    for (int k = 0; k < 3; ++k) reinterpret_cast<float2 *>(p)[k] = make_float2(v[2 * k], v[2 * k + 1]);
}

// Phase A over items u0 .. u1 (rows from r0 on, groups g0 .. g1 - 1); false after a timed-out
// wait for a bulk copy (WS_ERR_TIMEOUT is set).
__device__ bool stream_items(const PcgArgs &A, uint32_t g0, uint32_t g1, uint32_t r0, uint32_t u0, uint32_t u1,
                             const float *vec_in, float *out, float *wsm, int lane) {
    if (g0 >= g1) return true;
    float *blocks = wsm;                                                // [2][32][36]
    float *recs = wsm + 2 * kPcgBlockFloats;                            // [2][32][kSdStride]
    float *vring = recs + 2 * kPcgRecFloats;                            // [kPcgRing][8]: v of the row, beta
    double *gring = reinterpret_cast<double *>(vring + kPcgRing * 8);   // [kPcgRing] <d, A d> by row
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(gring + kPcgRing);
    const uint32_t nchunks = u1 > u0 ? (u1 - u0 + 31) / 32 : 0;
    const uint64_t pol = evict_first_policy();
    if (lane == 0) {
        bulk_init(bars, 2);
        bulk_blocks(A.sym_blocks, u0, u1, blocks, bars, pol);
        bulk_blocks(A.sym_blocks, u0 + 32, u1, blocks + kPcgBlockFloats, bars + 1, pol);
        l2_prefetch_blocks(A.sym_blocks, u0 + 64, u1, pol);
    }
    __syncwarp();
    unsigned phases = 0;   // bit k: parity of the next completion of buffer k's mbarrier
    bool ok = true;
    uint2 cur = load_item(A.item_info, u0 + lane, u1);
    uint2 nxt = load_item(A.item_info, u0 + 32 + lane, u1);
    // first rows of groups win .. win + 31 (lane i holds group win + i), reloaded as groups
    // complete; requested with the item records, before the column records need those
    uint32_t win = g0;
    uint32_t win_row = g0 + lane < A.total_groups ? A.group_row[g0 + lane] : A.total_nodes;
    float beta_cur;
    issue_records(A, vec_in, cur, recs, lane, beta_cur);
    float carry[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    double carry_dot = 0.0;
    uint32_t carry_row = kInvalidIndex;
    // the row of the item before the chunk; the range starts with row r0's diagonal item, so
    // an item's row is this plus the row starts up to and including it (unsigned wrap at r0 = 0)
    uint32_t row_before = r0 - 1u;
    auto group_first = [&](uint32_t g) -> uint32_t {   // first row of group g (g >= win)
        if (g >= A.total_groups) return A.total_nodes;
        if (g - win < 32) return __shfl_sync(0xffffffffu, win_row, (int)(g - win));
        return A.group_row[g];
    };
    uint32_t group = g0, group_end = group_first(g0 + 1);
    for (uint32_t j = 0; j < nchunks; ++j) {
        const int bk = (int)(j & 1u);
        // column records of chunk j + 1 in flight, item records of chunk j + 2 requested
        float beta_next;
        issue_records(A, vec_in, nxt, recs + (bk ^ 1) * kPcgRecFloats, lane, beta_next);
        if (lane == 0) l2_prefetch_blocks(A.sym_blocks, u0 + 32 * (j + 3), u1, pol);
        const uint2 after = load_item(A.item_info, u0 + 32 * (j + 2) + lane, u1);
        if (!bulk_wait(bars + bk, (phases >> bk) & 1u)) {
            if (lane == 0) set_err(A.err, WS_ERR_TIMEOUT);
            ok = false;
            break;
        }
        phases ^= 1u << bk;
        cp_async_wait_prior();
        __syncwarp();
        const bool valid = cur.x != kInvalidIndex;
        const bool diag = valid && (cur.x & kItemRowStart) != 0;
        const unsigned row_starts = __ballot_sync(0xffffffffu, diag);
        const uint32_t row = row_before + (uint32_t)__popc(row_starts & (0xffffffffu >> (31 - lane)));
        row_before += (uint32_t)__popc(row_starts);
        const uint32_t xrow = valid ? min(row, A.total_nodes - 1) : kInvalidIndex;
        float *mine = recs + bk * kPcgRecFloats + kSdStride * lane;
        float *vslot = vring + 8 * (xrow & (kPcgRing - 1));
        float sv[6], dv[6];
        if (valid) {
            const float4 a = reinterpret_cast<const float4 *>(mine)[0];
            const float4 b = reinterpret_cast<const float4 *>(mine)[1];
            const float4 c = reinterpret_cast<const float4 *>(mine)[2];
            sv[0] = a.x; sv[1] = a.y; sv[2] = a.z; sv[3] = a.w; sv[4] = b.x; sv[5] = b.y;
            dv[0] = b.z; dv[1] = b.w; dv[2] = c.x; dv[3] = c.y; dv[4] = c.z; dv[5] = c.w;
            if (diag) {   // the row's v and beta for its later items
                reinterpret_cast<float4 *>(vslot)[0] = make_float4(sv[0] + beta_cur * dv[0], sv[1] + beta_cur * dv[1],
                                                                   sv[2] + beta_cur * dv[2], sv[3] + beta_cur * dv[3]);
                reinterpret_cast<float4 *>(vslot)[1] =
                    make_float4(sv[4] + beta_cur * dv[4], sv[5] + beta_cur * dv[5], beta_cur, 0.f);
            }
        }
        __syncwarp();
        float vr[6], vc[6];   // v of the item's row and column
        float4 blk[9];
        if (valid) {
            const float4 v0 = reinterpret_cast<const float4 *>(vslot)[0];
            const float4 v1 = reinterpret_cast<const float4 *>(vslot)[1];
            vr[0] = v0.x; vr[1] = v0.y; vr[2] = v0.z; vr[3] = v0.w; vr[4] = v1.x; vr[5] = v1.y;
            const float beta = v1.z;   // the item's column lies in its row's scene
#pragma unroll
            for (int i = 0; i < 6; ++i) vc[i] = sv[i] + beta * dv[i];
            const float4 *src = reinterpret_cast<const float4 *>(blocks + bk * kPcgBlockFloats + 36 * lane);
#pragma unroll
            for (int q = 0; q < 9; ++q) blk[q] = src[q];
        }
        __syncwarp();
        // the buffer is free: it takes the blocks of the chunk two ahead
        if (lane == 0) bulk_blocks(A.sym_blocks, u0 + 32 * (j + 2), u1, blocks + bk * kPcgBlockFloats, bars + bk, pol);
        if (valid) {
            // B v_col and B^T v_row from one pass over the block
            float a[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, t[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                const float e4[4] = {blk[q].x, blk[q].y, blk[q].z, blk[q].w};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int e = 4 * q + k, r = e / 6, c = e % 6;
                    a[r] += e4[k] * vc[c];
                    t[c] += e4[k] * vr[r];
                }
            }
            if (!diag) store6_f2(A.contrib + 6ull * min(cur.y, A.cap_half - 1), t);
            double dot = 0.0;
            if (A.fp64) {
#pragma unroll
                for (int i = 0; i < 6; ++i) dot += (double)vr[i] * (double)a[i];
                if (!diag) dot *= 2.0;
            } else {
                float f = 0.f;
#pragma unroll
                for (int i = 0; i < 6; ++i) f += vr[i] * a[i];
                dot = (double)(diag ? f : 2.f * f);
            }
            // the record is in registers now: its slot takes the products
            reinterpret_cast<float4 *>(mine)[0] = make_float4(a[0], a[1], a[2], a[3]);
            reinterpret_cast<float2 *>(mine + 4)[0] = make_float2(a[4], a[5]);
            reinterpret_cast<double *>(mine + 6)[0] = dot;
        }
        __syncwarp();
        // row segments of this chunk: an item ends its row when the next item starts another
        // row or the range ends
        const uint32_t next_first = __shfl_sync(0xffffffffu, nxt.x, 0);
        const uint32_t word_dn = __shfl_down_sync(0xffffffffu, cur.x, 1);
        const uint32_t following = (lane == 31) ? next_first : word_dn;
        const uint32_t row_up = __shfl_up_sync(0xffffffffu, xrow, 1);
        const bool starts = valid && (lane == 0 || row_up != xrow);
        const unsigned start_mask = __ballot_sync(0xffffffffu, starts);
        const unsigned valid_mask = __ballot_sync(0xffffffffu, valid);
        const int last = 31 - __clz(valid_mask);
        const bool ends_row = valid && (following == kInvalidIndex || (following & kItemRowStart) != 0);
        const bool owner = valid && (ends_row || lane == last);
        float sum[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        double dsum = 0.0;
        if (owner) {
            const int first = 31 - __clz(start_mask & (0xffffffffu >> (31 - lane)));
            if (first == 0 && xrow == carry_row) {
#pragma unroll
                for (int i = 0; i < 6; ++i) sum[i] = carry[i];
                dsum = carry_dot;
            }
            const float *chunk = recs + bk * kPcgRecFloats;
            // sequential in item order; unrolled so that the loads of later items overlap
#pragma unroll 4
            for (int l = first; l <= lane; ++l) {
                const float4 a = reinterpret_cast<const float4 *>(chunk + kSdStride * l)[0];
                const float2 b = reinterpret_cast<const float2 *>(chunk + kSdStride * l + 4)[0];
                sum[0] += a.x;
                sum[1] += a.y;
                sum[2] += a.z;
                sum[3] += a.w;
                sum[4] += b.x;
                sum[5] += b.y;
                dsum += reinterpret_cast<const double *>(chunk + kSdStride * l + 6)[0];
            }
            if (ends_row) {
                float4 *qo = reinterpret_cast<float4 *>(A.q + 8ull * xrow);
                qo[0] = make_float4(sum[0], sum[1], sum[2], sum[3]);
                qo[1] = make_float4(sum[4], sum[5], 0.f, 0.f);
                store6_f2(out + (size_t)kSdStride * xrow + 6, vslot);   // d of the row
                gring[xrow & (kPcgRing - 1)] = A.fp64 ? dsum : (double)(float)dsum;
            }
        }
        // partial sums of a row that continues into the next chunk
        const bool cont = __shfl_sync(0xffffffffu, owner && !ends_row ? 1 : 0, last) != 0;
#pragma unroll
        for (int i = 0; i < 6; ++i) carry[i] = __shfl_sync(0xffffffffu, sum[i], last);
        carry_dot = __shfl_sync(0xffffffffu, dsum, last);
        const uint32_t last_row = __shfl_sync(0xffffffffu, xrow, last);
        carry_row = cont ? last_row : kInvalidIndex;
        __syncwarp();
        // groups whose rows are all done: their <d, A d> partial, summed in row order
        const uint32_t done_below = cont ? last_row : last_row + 1;
        while (group < g1 && group_end <= done_below) {
            const uint32_t grow = group_first(group);
            double v = 0.0;
            if (grow + lane < group_end) v = gring[(grow + lane) & (kPcgRing - 1)];
            double part;
            if (A.fp64) {
                part = warp_sum(v);
            } else {
                float f = (float)v;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) f += __shfl_xor_sync(0xffffffffu, f, o);
                part = (double)f;
            }
            if (lane == 0) A.group_partial[group] = part;
            ++group;
            if (group + 1 - win >= 32) {   // slide the window
                win = group;
                win_row = group + lane < A.total_groups ? A.group_row[group + lane] : A.total_nodes;
            }
            group_end = group_first(group + 1);
        }
        cur = nxt;
        nxt = after;
        beta_cur = beta_next;
    }
    // drain the last (empty) copy group, and the phase still outstanding on each block buffer
    // (a copy or an arrival past the range), before the buffers are reused
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    for (int k = 0; k < 2; ++k)
        if (!bulk_wait(bars + k, (phases >> k) & 1u)) {
            if (lane == 0) set_err(A.err, WS_ERR_TIMEOUT);
            ok = false;
        }
    // the next range initialises the mbarriers afresh (after a timeout the launch ends instead)
    if (ok && lane == 0)
        for (int k = 0; k < 2; ++k)
            asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_addr(bars + k)) : "memory");
    __syncwarp();
    return ok;
}

// Adds to v the contributions B^T v_i that the upper items of the rows i < row left as the
// row's lower entries, in column order.  The rows before `row` hold rowptr[row] blocks, of
// which item_ptr[row] are stored items, so the row's lower entries start at the difference.
__device__ __forceinline__ void add_lower(const PcgArgs &A, uint32_t row, float *v) {
    const uint32_t s0 = A.rowptr[row] - A.item_ptr[row];
    uint32_t n = (A.rowptr[row + 1] - A.rowptr[row]) - (A.item_ptr[row + 1] - A.item_ptr[row]);
    n = s0 < A.cap_half ? min(n, A.cap_half - s0) : 0u;
#pragma unroll 4
    for (uint32_t k = 0; k < n; ++k) {
        const float2 *c = reinterpret_cast<const float2 *>(A.contrib + 6ull * (s0 + k));
        const float2 a = __ldcg(c), b = __ldcg(c + 1), d = __ldcg(c + 2);
        v[0] += a.x;
        v[1] += a.y;
        v[2] += b.x;
        v[3] += b.y;
        v[4] += d.x;
        v[5] += d.y;
    }
}

// One step of the per-node phases: lane l takes row l % kRowsPerGroup of group
// g + l / kRowsPerGroup (a scene's last group may have fewer rows).
constexpr int kGroupsPerStep = 32 / kRowsPerGroup;
constexpr int kPcgBUnitsPerWarp = 3;   // phase-B work units per warp (each a run of row groups)
struct NodeStep {
    uint32_t gg, node, scene;
    bool group_ok, valid;
};
__device__ __forceinline__ NodeStep node_step(const PcgArgs &A, uint32_t g, uint32_t g_end, int lane) {
    NodeStep n;
    n.gg = g + (uint32_t)(lane / kRowsPerGroup);
    n.group_ok = n.gg < g_end;
    const uint32_t first = n.group_ok ? A.group_row[n.gg] : 0u;
    const uint32_t stop = !n.group_ok ? 0u : (n.gg + 1 < A.total_groups ? A.group_row[n.gg + 1] : A.total_nodes);
    n.scene = n.group_ok ? min(A.group_scene[n.gg], A.num_scenes - 1) : 0u;
    n.node = first + (uint32_t)(lane % kRowsPerGroup);
    n.valid = n.group_ok && n.node < stop;
    return n;
}

// Twist update of one node from its PCG step x (ApplyWarpFieldUpdateKernel,
// examples/mono_star/opt/SolverIterationData.cu:19-74).
__device__ __forceinline__ void twist_update_row(const PcgArgs &A, uint32_t row, const float *x) {
    float xv[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) xv[c] = x[c];
    if (A.fp64) {
        // node-centred twist -> origin twist: t = t' + c x w
        const float4 c4 = A.centers[row];
        const float3 cw = cross3(f3(c4.x, c4.y, c4.z), f3(xv[0], xv[1], xv[2]));
        xv[3] += cw.x;
        xv[4] += cw.y;
        xv[5] += cw.z;
    }
    const float3 w = f3(xv[0], xv[1], xv[2]);
    SE3f inc;
    if (fabsf(w.x) + fabsf(w.y) + fabsf(w.z) < 1e-4f) {
        inc.rot = M33{{{1.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, {0.f, 0.f, 1.f}}};
    } else {
        const float angle = sqrtf(w.x * w.x + w.y * w.y + w.z * w.z);
        const float3 ax = (1.0f / angle) * w;
        const float c = cosf(angle), sn = sinf(angle), t = 1.0f - c;
        inc.rot.m[0][0] = t * ax.x * ax.x + c;
        inc.rot.m[0][1] = t * ax.x * ax.y - ax.z * sn;
        inc.rot.m[0][2] = t * ax.x * ax.z + ax.y * sn;
        inc.rot.m[1][0] = t * ax.x * ax.y + ax.z * sn;
        inc.rot.m[1][1] = t * ax.y * ax.y + c;
        inc.rot.m[1][2] = t * ax.y * ax.z - ax.x * sn;
        inc.rot.m[2][0] = t * ax.x * ax.z - ax.y * sn;
        inc.rot.m[2][1] = t * ax.y * ax.z + ax.x * sn;
        inc.rot.m[2][2] = t * ax.z * ax.z + c;
    }
    inc.t = f3(xv[3], xv[4], xv[5]);
    const SE3f prev = dq_to_mat34(load_dq(A.se3 + 8ull * row));
    SE3f nw;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            nw.rot.m[i][j] = inc.rot.m[i][0] * prev.rot.m[0][j] + inc.rot.m[i][1] * prev.rot.m[1][j] +
                             inc.rot.m[i][2] * prev.rot.m[2][j];
    nw.t = mul(inc.rot, prev.t) + inc.t;
    store_dq(A.se3 + 8ull * row, dq_from_mat34(nw));
}

__global__ void __launch_bounds__(kPcgThreads, 3) k_pcg(PcgArgs A) {
    extern __shared__ __align__(16) float pcg_smem[];
    const int lane = threadIdx.x & 31;
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    float *wsm = pcg_smem + (threadIdx.x >> 5) * kPcgWarpFloats;
    // init and the twist update work per row, so they take an equal number of groups per warp;
    // every phase reads what others wrote only after a wait for all the groups of the scene, so
    // the partitions of the phases need not agree
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t b_begin = (uint32_t)((unsigned long long)A.total_groups * gwarp / nwarps);
    const uint32_t b_end = (uint32_t)((unsigned long long)A.total_groups * (gwarp + 1) / nwarps);
    const uint32_t br_begin = b_begin < A.total_groups ? A.group_row[b_begin] : A.total_nodes;
    const uint32_t br_end = b_end < A.total_groups ? A.group_row[b_end] : A.total_nodes;

    // ---- init: r = b, s = M^-1 b, x = 0, d = 0, delta = <r, s> ----
    for (uint32_t g = b_begin; g < b_end; g += kGroupsPerStep) {
        const NodeStep n = node_step(A, g, b_end, lane);
        float rv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, sv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (n.valid) {
            const float zero[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            load6(A.jtr + 8ull * n.node, rv);
            matvec6(A.inv_diag + 36ull * n.node, rv, sv);
            store6(A.r + 8ull * n.node, rv);
            store6(A.sd0 + (size_t)kSdStride * n.node, sv);
            store6_f2(A.sd0 + (size_t)kSdStride * n.node + 6, zero);
            store6(A.x + 8ull * n.node, zero);
        }
        const double part = node_dot_group(A, rv, sv, n.valid);
        if (lane % kRowsPerGroup == 0 && n.group_ok) A.group_partial[n.gg] = part;
    }
    publish_range(A, b_begin, b_end, 2, 0, lane);

    // the schedule (see the header comment): X's and Y's phase-A and phase-B unit counts
    const uint32_t G = A.total_groups, gm = min(A.split_group, G), bug = A.bunit_groups;
    const uint32_t ux = min(A.warp_groups[A.total_units + 1], A.total_units), uy = A.total_units - ux;
    const uint32_t bx = (gm + bug - 1) / bug, by = (G - gm + bug - 1) / bug;
    const uint32_t step_even = ux + by, step_odd = bx + uy;   // units of the steps 2, 4, .. and 1, 3, ..
    const uint32_t I = (uint32_t)max(A.pcg_iters, 0);
    // steps 0 .. 2I: step 0 holds X's first phase A only, step 2I Y's last phase B only
    const uint32_t total = I == 0 ? 0u : ux + I * step_odd + (I - 1) * step_even + by;
    uint32_t ticket = 0;
    if (lane == 0) ticket = atomicAdd(A.tickets, 1u);
    ticket = __shfl_sync(0xffffffffu, ticket, 0);
    while (ticket < total) {
        // the ticket's step k and its index i there
        uint32_t k, i;
        if (ticket < ux) {
            k = 0;
            i = ticket;
        } else {
            const uint32_t t = ticket - ux, pair = t / (step_odd + step_even), rem = t % (step_odd + step_even);
            k = 1 + 2 * pair + (rem < step_odd ? 0u : 1u);
            i = rem < step_odd ? rem : rem - step_odd;
        }
        // the step's X and Y units, interleaved in proportion; X's come first in a tie
        const bool odd = (k & 1u) != 0;
        const uint32_t nx = odd ? bx : (k < 2 * I ? ux : 0u);
        const uint32_t ny = odd ? uy : (k > 0 ? by : 0u);
        const uint32_t x_before = (uint32_t)((unsigned long long)i * nx / (nx + ny));
        const bool in_x = (uint32_t)((unsigned long long)(i + 1) * nx / (nx + ny)) > x_before;
        const uint32_t j = in_x ? x_before : i - x_before;
        // X runs phase k % 2 of iteration k / 2, Y half a phase later
        const bool phase_a = in_x ? !odd : odd;
        const int it = (int)(in_x ? k / 2 : (k - 1) / 2);
        const float *sd_old = (it & 1) ? A.sd1 : A.sd0;
        float *sd_new = (it & 1) ? A.sd0 : A.sd1;
        if (phase_a) {
            // ---- phase A: d = s + beta d, q = A d, <d, q> ----
            const uint32_t u = in_x ? j : ux + j;
            const uint4 ua = A.unit_info[2 * u], ub = A.unit_info[2 * u + 1];
            const uint32_t g_begin = min(ua.x, G), g_end = max(g_begin, min(ua.y, G));
            if (g_begin < g_end) {
                // the unit's scenes have finished the last iteration's phase B (init for the first)
                const bool waited = ub.z == ub.w ? wait_one_scene(A, ub.z, 1, (uint32_t)it + 1u, lane)
                                                 : wait_scenes(A, g_begin, g_end, 1, (uint32_t)it + 1u, lane);
                if (!waited) return;
                const uint32_t u_begin = min(ub.x, A.cap_items), u_end = max(u_begin, min(ub.y, A.cap_items));
                if (!stream_items(A, g_begin, g_end, ua.z, u_begin, u_end, sd_old, sd_new, wsm, lane)) return;
                publish_range(A, g_begin, g_end, 0, it, lane);
            }
        } else {
            // ---- phase B: alpha; x += alpha d; r -= alpha q; s = M^-1 r; <r, s> ----
            const uint32_t g_begin = in_x ? j * bug : gm + j * bug;
            const uint32_t g_end = min(g_begin + bug, in_x ? gm : G);
            // the unit's scenes have finished phase A and published alpha; the first step's rows
            // and scenes (fixed for the launch) are read first and tell which scenes to wait for
            NodeStep n = node_step(A, g_begin, g_end, lane);
            bool waited;
            if (g_end - g_begin <= (uint32_t)kGroupsPerStep) {
                const uint32_t s_lo = __reduce_min_sync(0xffffffffu, n.group_ok ? n.scene : 0xffffffffu);
                const uint32_t s_hi = __reduce_max_sync(0xffffffffu, n.group_ok ? n.scene : 0u);
                waited = s_lo == s_hi ? wait_one_scene(A, s_lo, 0, (uint32_t)it + 1u, lane)
                                      : wait_scenes(A, g_begin, g_end, 0, (uint32_t)it + 1u, lane);
            } else {
                waited = wait_scenes(A, g_begin, g_end, 0, (uint32_t)it + 1u, lane);
            }
            if (!waited) return;
            for (uint32_t g = g_begin; g < g_end; g += kGroupsPerStep) {
                if (g != g_begin) n = node_step(A, g, g_end, lane);
                float rv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, sv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (n.valid) {
                    const float alpha = (float)__ldcg(A.scalars + 8ull * n.scene + 1);
                    float xv[6], dv[6], qv[6];
                    load6(A.x + 8ull * n.node, xv);
                    load6_f2(sd_new + (size_t)kSdStride * n.node + 6, dv);
                    load6(A.r + 8ull * n.node, rv);
                    load6(A.q + 8ull * n.node, qv);
                    add_lower(A, n.node, qv);
#pragma unroll
                    for (int c = 0; c < 6; ++c) {
                        xv[c] += alpha * dv[c];
                        rv[c] -= alpha * qv[c];
                    }
                    matvec6(A.inv_diag + 36ull * n.node, rv, sv);
                    store6(A.x + 8ull * n.node, xv);
                    store6(A.r + 8ull * n.node, rv);
                    store6(sd_new + (size_t)kSdStride * n.node, sv);
                    // x is final after the last iteration: the node's twist update
                    // (ApplyWarpFieldUpdateKernel, SolverIterationData.cu:19-74) follows at once
                    if (it + 1 == A.pcg_iters) twist_update_row(A, n.node, xv);
                }
                const double part = node_dot_group(A, rv, sv, n.valid);
                if (lane % kRowsPerGroup == 0 && n.group_ok) A.group_partial[n.gg] = part;
            }
            publish_range(A, g_begin, g_end, 1, it + 1, lane);
        }
        if (lane == 0) ticket = atomicAdd(A.tickets, 1u);
        ticket = __shfl_sync(0xffffffffu, ticket, 0);
    }
    // the twist update runs in the last iteration's phase-B units (below, as x is final); with
    // no PCG iteration it follows init here
    if (A.pcg_iters > 0) return;
    if (!wait_scenes(A, b_begin, b_end, 1, 1u, lane)) return;
    for (uint32_t row = br_begin + lane; row < br_end; row += 32) {
        float xv[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) xv[c] = ldcg(A.x + 8ull * row + c);
        twist_update_row(A, row, xv);
    }
}

// Standalone y = A x over the assembled symmetric store of the last Gauss-Newton iteration
// (x, y: 8 floats per node).  y starts at zero; every row's diagonal-and-upper sum and every
// transposed product B^T x_row of an upper item are added into y with vector atomics, which
// resolve in L2 (y of the whole batch fits there), so DRAM sees the blocks, the item records,
// x and y once each: no contribution buffer and no second pass.  Sums meet in no fixed order.
// The kernel streams a warp's contiguous blocks through kSpmvBuffers shared-memory buffers of
// 4.6 KB: a chunk's 32 blocks (4608 contiguous bytes) arrive as one 1-D bulk copy
// (cp.async.bulk, issued by lane 0, its bytes counted on the buffer's mbarrier, with an
// evict-first L2 policy that keeps x and y in L2), each lane moves
// its item's block into registers, and the buffer at once takes the bulk copy of the chunk
// kSpmvBuffers ahead, which overlaps the arithmetic of the chunks between.  x of the items'
// columns is loaded a chunk ahead into registers, the items' 4-byte column words (item_col: the
// column, with the row's start marked) two chunks ahead.  Warp v takes part v % kSpmvSplit of the
// PCG's work units kPcgUnitsPerWarp (v / kSpmvSplit) .. + kPcgUnitsPerWarp - 1 (by row groups), so
// the ranges are the PCG's, at kSpmvSplit times the warps.
constexpr int kSpmvRing = 64;
constexpr int kSpmvBuffers = 2;
constexpr int kSpmvSplit = 1;
constexpr int kSpmvBlocksPerSm = 3;   // kSpmvSplit x the PCG's 3 blocks per SM: one wave of 12 warps per SM
// per warp: the buffers, the row ring, the lanes' products and one 16-byte slot per mbarrier, a
// multiple of 4 floats, so that every warp's buffers start on the 16-byte boundary a bulk copy needs
constexpr int kSpmvWarpFloats = kSpmvBuffers * 32 * 36 + kSpmvRing * 8 + 32 * 8 + 4 * kSpmvBuffers;
static_assert(kSpmvWarpFloats % 4 == 0, "warp areas on 16-byte boundaries");
constexpr size_t kSpmvSmemBytes = sizeof(float) * (kPcgThreads / 32) * kSpmvWarpFloats;
// Item word of the standalone SpMV: column | kItemRowStart on a row's first (diagonal) item,
// kInvalidIndex past the end of the range.
__device__ __forceinline__ uint32_t load_col(const uint32_t *cols, uint32_t u, uint32_t end) {
    return u < end ? __ldg(cols + u) : kInvalidIndex;
}
__device__ __forceinline__ void spmv_load_x(const PcgArgs &A, const float *x, uint32_t word, float4 &x0, float2 &x1) {
    x0 = make_float4(0.f, 0.f, 0.f, 0.f);
    x1 = make_float2(0.f, 0.f);
    if (word != kInvalidIndex) {
        const uint32_t col = min(word & ~kItemRowStart, A.total_nodes - 1);
        x0 = __ldg(reinterpret_cast<const float4 *>(x + 8ull * col));
        x1 = __ldg(reinterpret_cast<const float2 *>(x + 8ull * col + 4));
    }
}

__global__ void __launch_bounds__(kPcgThreads, kSpmvBlocksPerSm) k_spmv(PcgArgs A, const float *x, float *y) {
    // per warp: the chunk buffers, x of recent rows (by row), each lane's B x_col
    extern __shared__ __align__(16) float spmv_smem[];
    const int lane = threadIdx.x & 31;
    float *bufs = spmv_smem + (threadIdx.x >> 5) * kSpmvWarpFloats;
    float *ring = bufs + kSpmvBuffers * 32 * 36;
    float *prod = ring + kSpmvRing * 8;
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(prod + 32 * 8);   // 16-byte aligned
    unsigned phases = 0;   // bit k: parity of the next completion of buffer k
    const uint64_t pol = evict_first_policy();
    const uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t pv = v / kSpmvSplit, part = v % kSpmvSplit;
    const uint32_t pg0 = min(A.warp_groups[kPcgUnitsPerWarp * pv], A.total_groups);
    const uint32_t pg1 = max(pg0, min(A.warp_groups[kPcgUnitsPerWarp * (pv + 1)], A.total_groups));
    const uint32_t g0 = pg0 + ((pg1 - pg0) * part + kSpmvSplit - 1) / kSpmvSplit;
    const uint32_t g1 = pg0 + ((pg1 - pg0) * (part + 1) + kSpmvSplit - 1) / kSpmvSplit;
    if (g0 >= g1) return;
    const uint32_t r0 = A.group_row[g0], r1 = g1 < A.total_groups ? A.group_row[g1] : A.total_nodes;
    const uint32_t u0 = min(A.item_ptr[r0], A.cap_items), u1 = min(A.item_ptr[r1], A.cap_items);
    uint32_t cur = load_col(A.item_col, u0 + lane, u1);
    uint32_t nxt = load_col(A.item_col, u0 + 32 + lane, u1);
    float4 xa;
    float2 xb;
    spmv_load_x(A, x, cur, xa, xb);
    if (lane == 0) {
        bulk_init(bars, kSpmvBuffers);
        for (int k = 0; k < kSpmvBuffers; ++k) bulk_blocks(A.sym_blocks, u0 + 32u * k, u1, bufs + k * 32 * 36, bars + k, pol);
    }
    __syncwarp();
    float carry[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    uint32_t carry_row = kInvalidIndex;
    // the row of the item before the chunk; the range starts with row r0's diagonal item, so
    // an item's row is this plus the row starts up to and including it (unsigned wrap at r0 = 0)
    uint32_t row_before = r0 - 1u;
    uint32_t chunk = 0;
    for (uint32_t u = u0; u < u1; u += 32, ++chunk) {
        float *buf = bufs + (chunk % kSpmvBuffers) * 32 * 36;
        const uint32_t after = load_col(A.item_col, u + 64 + lane, u1);
        const bool valid = cur != kInvalidIndex;
        const bool diag = valid && (cur & kItemRowStart) != 0;
        const unsigned row_starts = __ballot_sync(0xffffffffu, diag);
        const uint32_t row = row_before + (uint32_t)__popc(row_starts & (0xffffffffu >> (31 - lane)));
        row_before += (uint32_t)__popc(row_starts);
        const uint32_t xrow = valid ? min(row, A.total_nodes - 1) : kInvalidIndex;
        const float xc[6] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y};
        if (valid && diag) {   // a row's first item: publish x of the row for its later items
            float4 *rr = reinterpret_cast<float4 *>(ring + 8 * (xrow & (kSpmvRing - 1)));
            rr[0] = xa;
            rr[1] = make_float4(xb.x, xb.y, 0.f, 0.f);
        }
        // every copy group commits in order: this chunk's is done when at most the
        // kSpmvBuffers - 1 later ones are pending
        const int bk = chunk % kSpmvBuffers;
        if (!bulk_wait(bars + bk, (phases >> bk) & 1u)) {
            if (lane == 0) set_err(A.err, WS_ERR_TIMEOUT);
            break;
        }
        phases ^= 1u << bk;
        float4 b[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) b[q] = reinterpret_cast<const float4 *>(buf + 36 * lane)[q];
        __syncwarp();
        // the buffer is free: the blocks kSpmvBuffers chunks ahead and the next x arrive while
        // this chunk is computed
        if (lane == 0) bulk_blocks(A.sym_blocks, u + 32u * kSpmvBuffers, u1, buf, bars + bk, pol);
        spmv_load_x(A, x, nxt, xa, xb);
        float a[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (valid) {
            const float4 v0 = reinterpret_cast<const float4 *>(ring + 8 * (xrow & (kSpmvRing - 1)))[0];
            const float2 v1 = reinterpret_cast<const float2 *>(ring + 8 * (xrow & (kSpmvRing - 1)) + 4)[0];
            const float vr[6] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y};
            float t[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                const float e4[4] = {b[q].x, b[q].y, b[q].z, b[q].w};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int e = 4 * q + k, r = e / 6, c = e % 6;
                    a[r] += e4[k] * xc[c];
                    t[c] += e4[k] * vr[r];
                }
            }
            if (!diag) {
                float *yc = y + 8ull * min(cur & ~kItemRowStart, A.total_nodes - 1);
                atomicAdd(reinterpret_cast<float4 *>(yc), make_float4(t[0], t[1], t[2], t[3]));
                atomicAdd(reinterpret_cast<float2 *>(yc + 4), make_float2(t[4], t[5]));
            }
            reinterpret_cast<float4 *>(prod + 8 * lane)[0] = make_float4(a[0], a[1], a[2], a[3]);
            reinterpret_cast<float2 *>(prod + 8 * lane + 4)[0] = make_float2(a[4], a[5]);
        }
        __syncwarp();
        // row segments of this chunk, summed in item order by the lane that ends them
        // an item ends its row when the next item starts another row or the range ends
        const uint32_t next_first = __shfl_sync(0xffffffffu, nxt, 0);
        const uint32_t word_dn = __shfl_down_sync(0xffffffffu, cur, 1);
        const uint32_t following = (lane == 31) ? next_first : word_dn;
        const bool starts = valid && (lane == 0 || diag);
        const unsigned start_mask = __ballot_sync(0xffffffffu, starts);
        const unsigned valid_mask = __ballot_sync(0xffffffffu, valid);
        const int last = 31 - __clz(valid_mask);
        const bool ends_row = valid && (following == kInvalidIndex || (following & kItemRowStart) != 0);
        const bool owner = valid && (ends_row || lane == last);
        float sum[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (owner) {
            const int first = 31 - __clz(start_mask & (0xffffffffu >> (31 - lane)));
            if (first == 0 && xrow == carry_row) {
#pragma unroll
                for (int i = 0; i < 6; ++i) sum[i] = carry[i];
            }
#pragma unroll 4
            for (int l = first; l <= lane; ++l) {
                const float4 p0 = reinterpret_cast<const float4 *>(prod + 8 * l)[0];
                const float2 p1 = reinterpret_cast<const float2 *>(prod + 8 * l + 4)[0];
                sum[0] += p0.x;
                sum[1] += p0.y;
                sum[2] += p0.z;
                sum[3] += p0.w;
                sum[4] += p1.x;
                sum[5] += p1.y;
            }
            if (ends_row) {
                atomicAdd(reinterpret_cast<float4 *>(y + 8ull * xrow), make_float4(sum[0], sum[1], sum[2], sum[3]));
                atomicAdd(reinterpret_cast<float2 *>(y + 8ull * xrow + 4), make_float2(sum[4], sum[5]));
            }
        }
        const bool cont = __shfl_sync(0xffffffffu, owner && !ends_row ? 1 : 0, last) != 0;
#pragma unroll
        for (int i = 0; i < 6; ++i) carry[i] = __shfl_sync(0xffffffffu, sum[i], last);
        carry_row = cont ? __shfl_sync(0xffffffffu, xrow, last) : kInvalidIndex;
        __syncwarp();
        cur = nxt;
        nxt = after;
    }
    // every buffer has one phase outstanding (a copy, or an arrival past the range): wait for it,
    // so that no bulk copy still writes when the block's shared memory is released
    for (int k = 0; k < kSpmvBuffers; ++k)
        if (!bulk_wait(bars + k, (phases >> k) & 1u) && lane == 0) set_err(A.err, WS_ERR_TIMEOUT);
}

// ---------------------------------------------------------------------------
// Matrix-free y = A x: the operator of the last Gauss-Newton iteration applied from the
// term records, without the assembled blocks.  A = sum over terms and channels of u u^T,
// with u the scaled Jacobian rows the assembly kernels use (lambda w J for dense terms,
// lambda c J for smoothness edges), plus the diagonal regulariser.  Pass 1 forms per term
// and channel  J x = sum over the term's nodes of u_node . x_node ; pass 2 gathers, per node,
// y = sum over its terms of u_node (J x) in list order (one warp per node, fixed butterfly).
// A term's four node ids are distinct (skinning picks distinct nodes).
// ---------------------------------------------------------------------------
template <int C>
__global__ void k_mf_dense(const Scene *scenes, const uint32_t *counts, const uint32_t *term_scene,
                           const float *drec, const float4 *centers, int centred, const float *x, float *ux) {
    using L = DenseLayout<C>;
    const uint32_t n = counts[kCntDense];
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const Scene &sc = scenes[term_scene[t]];
        const float *rec = drec + (size_t)L::kFloats * t;
        float u[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t node = __float_as_uint(rec[L::kIds + k]);
            const float w = rec[L::kW + k];
            const float4 x0 = *reinterpret_cast<const float4 *>(x + 8ull * node);
            const float2 x1 = *reinterpret_cast<const float2 *>(x + 8ull * node + 4);
            const float xv[6] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y};
            const float4 c4 = centers[node];
#pragma unroll
            for (int ch = 0; ch < C; ++ch) {
                float gl[6];
#pragma unroll
                for (int q = 0; q < 6; ++q) gl[q] = rec[6 * ch + q];
                if (centred) recentre(gl, f3(c4.x, c4.y, c4.z));
                float d = 0.f;
#pragma unroll
                for (int q = 0; q < 6; ++q) d += gl[q] * xv[q];
                u[ch] += w * d;
            }
        }
        const float lam[3] = {sc.lam_depth, sc.lam_of, sc.lam_of};
        reinterpret_cast<float4 *>(ux)[t] = make_float4(lam[0] * u[0], lam[1] * u[1], lam[2] * u[2], 0.f);
    }
}

__global__ void k_mf_reg(const Scene *scenes, const uint32_t *edge_scene, uint32_t total_edges, const float *rrec,
                         const float4 *centers, int centred, const float *x, float *ux) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total_edges; e += gridDim.x * blockDim.x) {
        const Scene &sc = scenes[edge_scene[e]];
        const float *rec = rrec + (size_t)kRegRecord * e;
        const uint32_t ni = __float_as_uint(rec[8]), nj = __float_as_uint(rec[9]);
        float u[3] = {0.f, 0.f, 0.f};
        if (rec[7] != 0.f && ni != nj) {
            const float3 a3 = f3(rec[0], rec[1], rec[2]), b3 = f3(rec[3], rec[4], rec[5]);
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const uint32_t node = side == 0 ? ni : nj;
                float J[3][6];
                reg_unit_jacobian(a3, b3, side == 0, J);
                const float4 c4 = centers[node];
                const float4 x0 = *reinterpret_cast<const float4 *>(x + 8ull * node);
                const float2 x1 = *reinterpret_cast<const float2 *>(x + 8ull * node + 4);
                const float xv[6] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y};
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) {
                    if (centred) recentre(J[ch], f3(c4.x, c4.y, c4.z));
                    float d = 0.f;
#pragma unroll
                    for (int q = 0; q < 6; ++q) d += J[ch][q] * xv[q];
                    u[ch] += d;
                }
            }
            const float s = sc.lam_reg * rec[6];
            u[0] *= s;
            u[1] *= s;
            u[2] *= s;
        }
        reinterpret_cast<float4 *>(ux)[e] = make_float4(u[0], u[1], u[2], 0.f);
    }
}

template <int C>
__global__ void __launch_bounds__(128) k_mf_gather(const Scene *scenes, const Plan *plan, const uint32_t *node_scene,
                                                   uint32_t total_nodes, const uint32_t *n2t_offset,
                                                   const uint32_t *n2t_val, const float *drec, const float *rrec,
                                                   const float *se3, const float4 *centers, int centred,
                                                   const float *ux_dense, const float *ux_reg, const float *x,
                                                   float *y) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < total_nodes; g += warps) {
        const Scene &sc = scenes[node_scene[g]];
        const Plan &p = plan[node_scene[g]];
        const uint32_t nd = p.dense_count, ne = sc.num_edges, nn = sc.num_nodes;
        const float4 c4 = centers[g];
        const float3 cen = f3(c4.x, c4.y, c4.z);
        float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (uint32_t it = n2t_offset[g] + lane; it < n2t_offset[g + 1]; it += 32) {
            const uint32_t term = n2t_val[it];
            if (term < nd) {
                using L = DenseLayout<C>;
                const float *rec = drec + (size_t)L::kFloats * (p.dense_begin + term);
                float w = rec[L::kW];   // weight of the last slot whose node is g
#pragma unroll
                for (int k = 1; k < 4; ++k) if (__float_as_uint(rec[L::kIds + k]) == g) w = rec[L::kW + k];
                const float4 u = reinterpret_cast<const float4 *>(ux_dense)[p.dense_begin + term];
                const float uu[3] = {u.x, u.y, u.z};
                const float lam[3] = {sc.lam_depth, sc.lam_of, sc.lam_of};
#pragma unroll
                for (int ch = 0; ch < C; ++ch) {
                    float gl[6];
#pragma unroll
                    for (int q = 0; q < 6; ++q) gl[q] = rec[6 * ch + q];
                    if (centred) recentre(gl, cen);
                    const float f = lam[ch] * w * uu[ch];
#pragma unroll
                    for (int q = 0; q < 6; ++q) acc[q] += f * gl[q];
                }
            } else if (term < nd + ne) {
                const uint32_t e = sc.edge_base + term - nd;
                const float *rec = rrec + (size_t)kRegRecord * e;
                if (rec[7] == 0.f) continue;
                float J[3][6];
                reg_unit_jacobian(f3(rec[0], rec[1], rec[2]), f3(rec[3], rec[4], rec[5]), __float_as_uint(rec[8]) == g,
                                  J);
                const float4 u = reinterpret_cast<const float4 *>(ux_reg)[e];
                const float uu[3] = {u.x, u.y, u.z};
                const float s = sc.lam_reg * rec[6];
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) {
                    if (centred) recentre(J[ch], cen);
#pragma unroll
                    for (int q = 0; q < 6; ++q) acc[q] += s * uu[ch] * J[ch][q];
                }
            } else if (term < nd + ne + nn && sc.lam_node != 0.f && sc.node_motion) {
                const uint32_t nl = term - nd - ne;
                const float scale = sc.lam_node * sc.node_motion[nl].w;
                const float4 x0 = *reinterpret_cast<const float4 *>(x + 8ull * g);
                const float2 x1 = *reinterpret_cast<const float2 *>(x + 8ull * g + 4);
                const float xv[6] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y};
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) {
                    float J[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                    J[3 + ch] = scale;
                    if (centred) recentre(J, cen);
                    float d = 0.f;
#pragma unroll
                    for (int q = 0; q < 6; ++q) d += J[q] * xv[q];
#pragma unroll
                    for (int q = 0; q < 6; ++q) acc[q] += d * J[q];
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 6; ++q) acc[q] = warp_sum(acc[q]);
        if (lane == 0) {
            // + 1e-3 S^T S x (node-centred twists) or 1e-3 x (origin twists)
            const float4 x0 = *reinterpret_cast<const float4 *>(x + 8ull * g);
            const float2 x1 = *reinterpret_cast<const float2 *>(x + 8ull * g + 4);
            const float3 om = f3(x0.x, x0.y, x0.z), tr = f3(x0.w, x1.x, x1.y);
            float r[6] = {om.x, om.y, om.z, tr.x, tr.y, tr.z};
            if (centred) {
                const float3 v = cross3(cen, om) + tr;   // translation part of S x
                const float3 cv = cross3(cen, v);
                r[0] = om.x - cv.x; r[1] = om.y - cv.y; r[2] = om.z - cv.z;
                r[3] = v.x; r[4] = v.y; r[5] = v.z;
            }
            float4 *yo = reinterpret_cast<float4 *>(y + 8ull * g);
            yo[0] = make_float4(acc[0] + 1e-3f * r[0], acc[1] + 1e-3f * r[1], acc[2] + 1e-3f * r[2], acc[3] + 1e-3f * r[3]);
            yo[1] = make_float4(acc[4] + 1e-3f * r[4], acc[5] + 1e-3f * r[5], 0.f, 0.f);
        }
    }
}

// One warp per row group when that fits, else every co-resident block.
int pcg_launch_blocks(const Workspace &w) {
    const uint32_t want = (w.total_chunks + (kPcgThreads / 32) - 1) / (kPcgThreads / 32);
    const uint32_t cap = (uint32_t)std::min(w.pcg_grid, std::max(1, w.tune.pcg_blocks_per_sm) * w.num_sms);
    return (int)std::max<uint32_t>(1u, std::min<uint32_t>(want, cap));
}
int pcg_warps_per_block() { return kPcgThreads / 32; }

int pcg_max_blocks(int device) {
    int per_sm = 0, sms = 0;
    cudaFuncSetAttribute(k_pcg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPcgSmemBytes);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg, kPcgThreads, kPcgSmemBytes);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return std::max(1, per_sm) * std::max(1, sms);
}

static inline int grid_for(uint32_t n, int threads, int num_sms, int per_sm = 8) {
    const uint32_t want = (n + threads - 1) / threads;
    const uint32_t cap = (uint32_t)num_sms * (uint32_t)per_sm;
    return (int)std::max<uint32_t>(1u, std::min<uint32_t>(want, cap));
}

void init_warp(Workspace &w, cudaStream_t st) {
    k_init_warp<<<grid_for(w.total_nodes, 256, w.num_sms), 256, 0, st>>>(w.scenes, w.node_scene, w.total_nodes, w.se3);
    count_launch(w);
}

void gn_eval(Workspace &w, cudaStream_t st) {
    k_node_centers<<<grid_for(w.total_nodes, 256, w.num_sms), 256, 0, st>>>(w.scenes, w.node_scene, w.total_nodes,
                                                                           w.se3, w.centers);
    count_launch(w);
    if (w.dense_channels == 3)
        k_eval_dense<3><<<grid_for(w.cap_pixels, 256, w.num_sms, 16), 256, 0, st>>>(
            w.scenes, w.counts, w.d_pixels, w.d_knn, w.d_sw, w.d_cw, w.d_scene, w.se3, w.d_record);
    else
        k_eval_dense<1><<<grid_for(w.cap_pixels, 256, w.num_sms, 16), 256, 0, st>>>(
            w.scenes, w.counts, w.d_pixels, w.d_knn, w.d_sw, w.d_cw, w.d_scene, w.se3, w.d_record);
    count_launch(w);
    if (w.total_edges > 0) {
        k_eval_reg<<<grid_for(w.total_edges, 256, w.num_sms), 256, 0, st>>>(w.scenes, w.edge_scene, w.total_edges,
                                                                            w.se3, w.r_record);
        count_launch(w);
    }
}

template <class DAcc, int NT, int C>
static void launch_assemble_node_c(Workspace &w, cudaStream_t st) {
    k_assemble_node<DAcc, NT, C><<<grid_for(w.total_nodes * 32u, NT, w.num_sms, 32 * 128 / NT), NT, 0, st>>>(
        w.scenes, w.plan, w.node_scene, w.total_nodes, w.n2t_offset, w.n2t_sorted_val, w.cap_n2t, w.d_record, w.r_record, w.se3,
        w.centers, w.item_ptr, w.cap_items, w.sym_blocks, w.diag64, w.jtr, w.error_flag);
}

template <class DAcc, int NT>
static void launch_assemble_node(Workspace &w, cudaStream_t st) {
    if (w.dense_channels == 3) launch_assemble_node_c<DAcc, NT, 3>(w, st);
    else launch_assemble_node_c<DAcc, NT, 1>(w, st);
}

template <class DAcc>
static void launch_assemble_node_nt(Workspace &w, int nt, cudaStream_t st) {
    if (nt == 64) {
        launch_assemble_node<DAcc, 64>(w, st);
    } else if (nt == 256) {
        launch_assemble_node<DAcc, 256>(w, st);
    } else {
        launch_assemble_node<DAcc, 128>(w, st);
    }
}

void gn_assemble_node(Workspace &w, cudaStream_t st) {
    if (w.precision == WS_PREC_FP32) launch_assemble_node_nt<float>(w, w.tune.node_threads, st);
    else launch_assemble_node_nt<double>(w, w.tune.node_threads, st);
    count_launch(w);
    k_block_inverse<<<grid_for(w.total_nodes, 128, w.num_sms, 16), 128, 0, st>>>(
        w.diag64, w.sym_blocks, w.item_ptr, w.cap_items, w.total_nodes, w.precision == WS_PREC_MIXED ? 1 : 0,
        w.inv_diag);
    count_launch(w);
}

template <int NT, int C>
static void launch_assemble_pair_c(Workspace &w, cudaStream_t st) {
    k_assemble_pair<NT, C><<<grid_for(w.cap_half * 32u, NT, w.num_sms, 32 * 128 / NT), NT, 0, st>>>(
        w.scenes, w.plan, w.counts, w.half_row, w.half_col, w.half_begin, w.half_end, w.half_scene,
        w.pair_sorted_val, w.cap_pair_kv,
        w.half_slot_up, w.d_record, w.r_record, w.centers, w.precision == WS_PREC_MIXED ? 1 : 0, w.sym_blocks,
        w.error_flag);
}

template <int NT>
static void launch_assemble_pair(Workspace &w, cudaStream_t st) {
    if (w.dense_channels == 3) launch_assemble_pair_c<NT, 3>(w, st);
    else launch_assemble_pair_c<NT, 1>(w, st);
}

void gn_assemble_pair(Workspace &w, cudaStream_t st) {
    if (w.tune.pair_threads == 64) launch_assemble_pair<64>(w, st);
    else if (w.tune.pair_threads == 256) launch_assemble_pair<256>(w, st);
    else launch_assemble_pair<128>(w, st);
    count_launch(w);
}

uint32_t pcg_split_group(const Workspace &w) {
    // the scene boundary nearest to half of the row groups (after the first scene at least)
    const uint32_t half = w.total_chunks / 2;
    uint32_t best = w.total_chunks, end = 0;
    for (int s = 0; s < w.num_scenes && s < (int)w.h_scenes.size(); ++s) {
        end += (uint32_t)w.h_scenes[s].num_chunks;
        if (end >= w.total_chunks) break;
        const uint32_t d = end > half ? end - half : half - end;
        const uint32_t db = best > half ? best - half : half - best;
        if (d < db) best = end;
    }
    return best;
}

static PcgArgs pcg_args(Workspace &w, int pcg_iters) {
    PcgArgs a;
    a.scenes = w.scenes;
    a.group_scene = w.chunk_scene;
    a.group_row = w.chunk_row;
    a.total_groups = w.total_chunks;
    a.rowptr = w.rowptr;
    a.item_ptr = w.item_ptr;
    a.item_info = w.item_info;
    a.item_col = w.item_col;
    a.contrib = w.contrib;
    a.warp_groups = w.pcg_warp_groups;
    a.unit_info = w.pcg_unit_info;
    a.total_units = (uint32_t)(kPcgUnitsPerWarp * pcg_launch_blocks(w) * pcg_warps_per_block());
    a.split_group = pcg_split_group(w);
    a.tickets = w.pcg_tickets;
    {
        // about kPcgBUnitsPerWarp units per warp on problems with a warp per group or so (one row
        // group each); on the large batches units of whole steps, at least two (64 rows): a unit's
        // wait, publication and ticket then serve twice the rows
        const uint64_t slots = (uint64_t)kPcgBUnitsPerWarp * pcg_launch_blocks(w) * pcg_warps_per_block();
        a.bunit_groups = (uint32_t)std::max<uint64_t>(1, (w.total_chunks + slots - 1) / slots);
        const uint32_t step = (uint32_t)kGroupsPerStep;
        if (a.bunit_groups >= step) a.bunit_groups = std::max(2 * step, (a.bunit_groups + step - 1) / step * step);
    }
    a.sym_blocks = w.sym_blocks;
    a.inv_diag = w.inv_diag;
    a.jtr = w.jtr;
    a.x = w.x; a.r = w.r; a.q = w.q; a.sd0 = w.sd0; a.sd1 = w.sd1;
    a.group_partial = w.chunk_partial;
    a.scalars = w.scene_scalars;
    a.scene_counter = w.scene_counter;
    a.cap_blocks = w.cap_blocks;
    a.cap_items = w.cap_items;
    a.cap_half = std::max<uint32_t>(1u, w.cap_half);
    a.num_scenes = (uint32_t)std::max(1, w.num_scenes);
    a.total_nodes = w.total_nodes;
    a.err = w.error_flag;
    a.se3 = w.se3;
    a.centers = w.centers;
    a.pcg_iters = pcg_iters;
    a.fp64 = (w.precision == WS_PREC_MIXED) ? 1 : 0;
    return a;
}

cudaError_t gn_pcg(Workspace &w, int pcg_iters, cudaStream_t st) {
    PcgArgs a = pcg_args(w, pcg_iters);
    const int grid = pcg_launch_blocks(w);
    // tickets and generations start at zero every launch, so a launch that timed out half-way
    // cannot leak into the next
    cudaMemsetAsync(w.scene_counter, 0, sizeof(uint32_t) * kSceneSync * (size_t)w.num_scenes, st);
    cudaMemsetAsync(w.pcg_tickets, 0, sizeof(uint32_t), st);
    void *args[] = {&a};
    count_launch(w);
    return cudaLaunchCooperativeKernel((const void *)k_pcg, dim3(grid), dim3(kPcgThreads), args, kPcgSmemBytes, st);
}

cudaError_t gn_spmv_matrix_free(Workspace &w, const float *x, float *y, float *ux_dense, float *ux_reg,
                                cudaStream_t st) {
    const int centred = w.precision == WS_PREC_MIXED ? 1 : 0;
    if (w.dense_channels == 3)
        k_mf_dense<3><<<grid_for(w.cap_pixels, 256, w.num_sms, 16), 256, 0, st>>>(
            w.scenes, w.counts, w.d_scene, w.d_record, w.centers, centred, x, ux_dense);
    else
        k_mf_dense<1><<<grid_for(w.cap_pixels, 256, w.num_sms, 16), 256, 0, st>>>(
            w.scenes, w.counts, w.d_scene, w.d_record, w.centers, centred, x, ux_dense);
    if (w.total_edges > 0)
        k_mf_reg<<<grid_for(w.total_edges, 256, w.num_sms), 256, 0, st>>>(w.scenes, w.edge_scene, w.total_edges,
                                                                          w.r_record, w.centers, centred, x, ux_reg);
    auto gather = w.dense_channels == 3 ? k_mf_gather<3> : k_mf_gather<1>;
    gather<<<grid_for(w.total_nodes * 32u, 128, w.num_sms, 32), 128, 0, st>>>(
        w.scenes, w.plan, w.node_scene, w.total_nodes, w.n2t_offset, w.n2t_sorted_val, w.d_record, w.r_record, w.se3,
        w.centers, centred, ux_dense, ux_reg, x, y);
    return cudaGetLastError();
}

cudaError_t gn_spmv(Workspace &w, const float *x, float *y, cudaStream_t st) {
    const PcgArgs a = pcg_args(w, 0);
    const cudaError_t attr =
        cudaFuncSetAttribute(k_spmv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSpmvSmemBytes);
    if (attr != cudaSuccess) return attr;
    const cudaError_t e = cudaMemsetAsync(y, 0, 32ull * w.total_nodes, st);
    if (e != cudaSuccess) return e;
    k_spmv<<<kSpmvSplit * pcg_launch_blocks(w), kPcgThreads, kSpmvSmemBytes, st>>>(a, x, y);
    return cudaGetLastError();
}

cudaError_t gn_iteration(Workspace &w, int pcg_iters, cudaStream_t st) {
    gn_eval(w, st);
    gn_assemble_node(w, st);
    gn_assemble_pair(w, st);
    return gn_pcg(w, pcg_iters, st);
}

}  // namespace ws
