// CPU oracle for StarHub's per-frame warp-field solve -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++ restatement of the reference algorithm (changhaonan/StarHub) used
// as the checker for the CUDA library and as the timed CPU baseline.  Each
// function cites the reference file:line it restates.  Parity status: parity
// unpinned (the reference ships no tests or golden vectors and cannot be built
// here: its headers need Eigen/OpenCV/PCL/Boost/nlohmann-json).
//
// Build: see oracle/Makefile.  Compiled with -ffp-contract=off so that every
// multiply-add below happens exactly as written; where the reference relies on
// nvcc's default contraction the fused form is spelled out with fmaf().
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <type_traits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// IEEE binary16 conversion (round to nearest even), written from the format
// definition.  The node graph stores squared node distances as half
// (libs/star/geometry/node_graph/NodeGraph.cu:35).
// ---------------------------------------------------------------------------
uint16_t float_to_half_rn(float f) {
    uint32_t x;
    std::memcpy(&x, &f, 4);
    const uint32_t sign = (x >> 16) & 0x8000u;
    const uint32_t absx = x & 0x7fffffffu;
    if (absx >= 0x7f800000u) {                       // inf / nan
        return (uint16_t)(sign | 0x7c00u | (absx > 0x7f800000u ? 0x200u : 0u));
    }
    const int exp = (int)(absx >> 23) - 127;
    if (exp > 15) return (uint16_t)(sign | 0x7c00u);  // overflow -> inf
    uint32_t mant = absx & 0x7fffffu;
    if (exp >= -14) {                                 // normal half
        uint32_t h = ((uint32_t)(exp + 15) << 10) | (mant >> 13);
        const uint32_t rem = mant & 0x1fffu;
        if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1;   // may carry into exponent / inf
        return (uint16_t)(sign | h);
    }
    if (exp < -25) return (uint16_t)sign;             // rounds to zero
    // subnormal half: value = mant_full * 2^(exp-23), half unit = 2^-24
    mant |= 0x800000u;
    // half subnormal unit is 2^-24: value / 2^-24 = mant * 2^(exp + 1), a right shift by -exp - 1
    const int shift = -exp - 1;
    uint32_t h = mant >> shift;
    const uint32_t rem = mant & ((1u << shift) - 1u);
    const uint32_t halfway = 1u << (shift - 1);
    if (rem > halfway || (rem == halfway && (h & 1u))) h += 1;
    return (uint16_t)(sign | h);
}

float half_to_float(uint16_t h) {
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    const uint32_t exp = (h >> 10) & 0x1fu;
    uint32_t mant = h & 0x3ffu;
    uint32_t bits;
    if (exp == 0) {
        if (mant == 0) {
            bits = sign;
        } else {
            int e = -1;
            do { mant <<= 1; ++e; } while ((mant & 0x400u) == 0);
            bits = sign | ((uint32_t)(127 - 15 - e) << 23) | ((mant & 0x3ffu) << 13);
        }
    } else if (exp == 0x1f) {
        bits = sign | 0x7f800000u | (mant << 13);
    } else {
        bits = sign | ((exp - 15 + 127) << 23) | (mant << 13);
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

// Squared length in the fused order nvcc emits for `x*x + y*y + z*z` under its
// default -fmad=true: fma(z, z, fma(y, y, x*x)).
inline float sq3_fused(float x, float y, float z) {
    return std::fmaf(z, z, std::fmaf(y, y, x * x));
}

int set_threads(int threads) {
#ifdef _OPENMP
    int t = threads > 0 ? threads : omp_get_max_threads();
    return t;
#else
    (void)threads;
    return 1;
#endif
}

// ---------------------------------------------------------------------------
// KNN heap + quicksort (libs/star/geometry/node_graph/brute_force_knn.cuh:52-135).
// Replace-the-maximum on strict `<`, maximum found with strict `>` (first wins),
// then Lomuto quicksort on strict `<`.
// ---------------------------------------------------------------------------
template <int CAP>
struct KnnHeap {
    float distance[CAP];
    uint16_t index[CAP];
    int max_id;
    float max_distance;
    KnnHeap(float init_d) {
        for (int i = 0; i < CAP; ++i) { distance[i] = init_d; index[i] = 0; }
        update_heap();
    }
    // the reference's constructor from given distances and ids (brute_force_knn.cuh:62-70)
    KnnHeap(const float *d, const uint16_t *ids) {
        for (int i = 0; i < CAP; ++i) { distance[i] = d[i]; index[i] = ids[i]; }
        update_heap();
    }
    void update_heap() {
        max_id = 0;
        max_distance = distance[0];
        for (int i = 1; i < CAP; ++i)
            if (distance[i] > max_distance) { max_distance = distance[i]; max_id = i; }
    }
    void update(uint16_t idx, float d) {
        if (d < max_distance) { distance[max_id] = d; index[max_id] = idx; }
        update_heap();
    }
    int partition(int low, int high) {
        const float pivot = distance[high];
        int i = low - 1;
        for (int j = low; j <= high - 1; ++j) {
            if (distance[j] < pivot) {
                ++i;
                std::swap(distance[i], distance[j]);
                std::swap(index[i], index[j]);
            }
        }
        std::swap(distance[i + 1], distance[high]);
        std::swap(index[i + 1], index[high]);
        return i + 1;
    }
    void quick_sort(int low, int high) {
        if (low < high) {
            const int pi = partition(low, high);
            quick_sort(low, pi - 1);
            quick_sort(pi + 1, high);
        }
    }
    void sort() { quick_sort(0, CAP - 1); }
};

// ---------------------------------------------------------------------------
// Small fixed-size math templated on the working precision.
// ---------------------------------------------------------------------------
template <class R> struct V3 { R x, y, z; };
template <class R> inline V3<R> v3(R x, R y, R z) { return {x, y, z}; }
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Row-major 3x3 (the reference stores column-major; only the values matter).
template <class R> struct M33 {
    R m[3][3];
    V3<R> mul(V3<R> v) const {
        return {m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z,
                m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
                m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
    }
    V3<R> tmul(V3<R> v) const {   // transpose(M) * v
        return {m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z,
                m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
                m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z};
    }
};
template <class R> inline M33<R> matmul(const M33<R> &a, const M33<R> &b) {
    M33<R> c;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) c.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
    return c;
}
template <class R> struct SE3 { M33<R> rot; V3<R> trans; };

template <class R> struct Quat { R x, y, z, w; };
template <class R> inline Quat<R> qmul(Quat<R> a, Quat<R> b) {
    // libs/star/math/Quaternion.hpp:139-148
    Quat<R> q;
    q.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
    q.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
    q.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
    q.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
    return q;
}
template <class R> inline Quat<R> qconj(Quat<R> a) { return {-a.x, -a.y, -a.z, a.w}; }

template <class R> struct DQ { Quat<R> q0, q1; };

template <class R> inline R rsqrt_r(R v) { return R(1) / std::sqrt(v); }

// DualQuaternion::normalize (libs/star/math/DualQuaternion.hpp:150-156).
template <class R> inline void dq_normalize(DQ<R> &d) {
    const R inv = rsqrt_r(d.q0.w * d.q0.w + d.q0.x * d.q0.x + d.q0.y * d.q0.y + d.q0.z * d.q0.z);
    d.q0 = {inv * d.q0.x, inv * d.q0.y, inv * d.q0.z, inv * d.q0.w};
    d.q1 = {inv * d.q1.x, inv * d.q1.y, inv * d.q1.z, inv * d.q1.w};
    const R dq = d.q0.x * d.q1.x + d.q0.y * d.q1.y + d.q0.z * d.q1.z + d.q0.w * d.q1.w;
    d.q1 = {d.q1.x - dq * d.q0.x, d.q1.y - dq * d.q0.y, d.q1.z - dq * d.q0.z, d.q1.w - dq * d.q0.w};
}

// Quaternion::rotation_matrix(false) (Quaternion.hpp:96-111).
template <class R> inline M33<R> quat_rot(Quat<R> q) {
    M33<R> r;
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

// DualQuaternion::se3_matrix (DualQuaternion.hpp:182-189): normalize, rotation
// from q0, translation = vec(2 q1 conj(q0)).
template <class R> inline SE3<R> dq_se3(DQ<R> d) {
    dq_normalize(d);
    SE3<R> T;
    T.rot = quat_rot(d.q0);
    Quat<R> two_q1 = {R(2) * d.q1.x, R(2) * d.q1.y, R(2) * d.q1.z, R(2) * d.q1.w};
    const Quat<R> tp = qmul(two_q1, qconj(d.q0));
    T.trans = {tp.x, tp.y, tp.z};
    return T;
}

// DualQuaternion -> mat34 conversion operator (DualQuaternion.hpp:169-179):
// normalized copy, q0.matrix() (which normalizes q0 again), t = vec(2 q1 q0*).
template <class R> inline SE3<R> dq_to_mat34(DQ<R> d) {
    dq_normalize(d);
    Quat<R> q = d.q0;
    const R inv = rsqrt_r(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    q = {q.x * inv, q.y * inv, q.z * inv, q.w * inv};
    SE3<R> T;
    T.rot = quat_rot(q);
    Quat<R> two_q1 = {R(2) * d.q1.x, R(2) * d.q1.y, R(2) * d.q1.z, R(2) * d.q1.w};
    const Quat<R> tp = qmul(two_q1, qconj(d.q0));
    T.trans = {tp.x, tp.y, tp.z};
    return T;
}

// Quaternion(const mat33&) (Quaternion.hpp:17-52).
template <class R> inline Quat<R> quat_from_rot(const M33<R> &m) {
    Quat<R> q;
    const R tr = m.m[0][0] + m.m[1][1] + m.m[2][2];
    if (tr > 0) {
        const R s = std::sqrt(tr + R(1)) * 2;
        q.w = s * R(0.25);
        q.x = (m.m[2][1] - m.m[1][2]) / s;
        q.y = (m.m[0][2] - m.m[2][0]) / s;
        q.z = (m.m[1][0] - m.m[0][1]) / s;
    } else if (m.m[0][0] > m.m[1][1] && m.m[0][0] > m.m[2][2]) {
        const R s = std::sqrt(R(1) + m.m[0][0] - m.m[1][1] - m.m[2][2]) * 2;
        q.w = (m.m[2][1] - m.m[1][2]) / s;
        q.x = R(0.25) * s;
        q.y = (m.m[0][1] + m.m[1][0]) / s;
        q.z = (m.m[0][2] + m.m[2][0]) / s;
    } else if (m.m[1][1] > m.m[2][2]) {
        const R s = std::sqrt(R(1) + m.m[1][1] - m.m[0][0] - m.m[2][2]) * 2;
        q.w = (m.m[0][2] - m.m[2][0]) / s;
        q.x = (m.m[0][1] + m.m[1][0]) / s;
        q.y = R(0.25) * s;
        q.z = (m.m[1][2] + m.m[2][1]) / s;
    } else {
        const R s = std::sqrt(R(1) + m.m[2][2] - m.m[0][0] - m.m[1][1]) * 2;
        q.w = (m.m[1][0] - m.m[0][1]) / s;
        q.x = (m.m[0][2] + m.m[2][0]) / s;
        q.y = (m.m[1][2] + m.m[2][1]) / s;
        q.z = R(0.25) * s;
    }
    return q;
}

// DualQuaternion(const mat34&) (DualQuaternion.hpp:59-66): vec_part * rot_part.
template <class R> inline DQ<R> dq_from_mat34(const SE3<R> &T) {
    const Quat<R> qr = quat_from_rot(T.rot);
    const Quat<R> qt = {R(0.5) * T.trans.x, R(0.5) * T.trans.y, R(0.5) * T.trans.z, R(0)};
    // (1, qt) * (qr, 0) = (qr, qt * qr)
    DQ<R> d;
    d.q0 = qr;
    d.q1 = qmul(qt, qr);
    return d;
}

// Rodrigues as in ApplyWarpFieldUpdateKernel
// (examples/mono_star/opt/SolverIterationData.cu:41-68); the translation is the
// raw twist translation.
template <class R> inline SE3<R> twist_to_se3(const R *x) {
    SE3<R> T;
    const V3<R> w = {x[0], x[1], x[2]};
    const R l1 = std::fabs(w.x) + std::fabs(w.y) + std::fabs(w.z);
    if (l1 < R(1e-4f)) {
        T.rot = {{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}};
    } else {
        const R angle = std::sqrt(w.x * w.x + w.y * w.y + w.z * w.z);
        const V3<R> a = (R(1) / angle) * w;
        const R c = std::cos(angle), s = std::sin(angle), t = R(1) - c;
        T.rot.m[0][0] = t * a.x * a.x + c;
        T.rot.m[0][1] = t * a.x * a.y - a.z * s;
        T.rot.m[0][2] = t * a.x * a.z + a.y * s;
        T.rot.m[1][0] = t * a.x * a.y + a.z * s;
        T.rot.m[1][1] = t * a.y * a.y + c;
        T.rot.m[1][2] = t * a.y * a.z - a.x * s;
        T.rot.m[2][0] = t * a.x * a.z - a.y * s;
        T.rot.m[2][1] = t * a.y * a.z + a.x * s;
        T.rot.m[2][2] = t * a.z * a.z + c;
    }
    T.trans = {x[3], x[4], x[5]};
    return T;
}

template <class R> inline DQ<R> load_dq(const float *p) {
    DQ<R> d;
    d.q0 = {R(p[0]), R(p[1]), R(p[2]), R(p[3])};
    d.q1 = {R(p[4]), R(p[5]), R(p[6]), R(p[7])};
    return d;
}

// ---------------------------------------------------------------------------
// Term id space (examples/mono_star/common/term_offset_types.h:62-118):
// [dense N_d | reg E | node-motion N | feature F].
// ---------------------------------------------------------------------------
struct TermOffsets {
    uint32_t dense, reg, node, feat;   // cumulative ends
};
inline TermOffsets make_offsets(uint32_t nd, uint32_t ne, uint32_t nn, uint32_t nf) {
    TermOffsets o;
    o.dense = nd;
    o.reg = nd + ne;
    o.node = nd + ne + nn;
    o.feat = nd + ne + nn + nf;
    return o;
}

// Stable key/value sort by key (the reference sorts with cub::DeviceRadixSort,
// which is stable): returns the permutation.
template <class K>
std::vector<uint32_t> stable_order(const std::vector<K> &keys) {
    std::vector<uint32_t> perm(keys.size());
    std::iota(perm.begin(), perm.end(), 0u);
    std::stable_sort(perm.begin(), perm.end(), [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
    return perm;
}

// ---------------------------------------------------------------------------
// Index structures shared by the solve.
// ---------------------------------------------------------------------------
struct Node2Term {
    std::vector<uint32_t> offset;       // N + 1
    std::vector<uint32_t> term_index;   // all sorted values (invalid-key entries at the end)
};

// Node2TermsIndex::buildTermKeyValue / sortCompactTermIndex
// (examples/mono_star/opt/Node2TermsIndex.cu:6-121, 312-361).
Node2Term build_node2term(uint32_t nd, const uint16_t *dense_knn, uint32_t ne, const uint16_t *edges,
                          uint32_t nn, uint32_t nf, const uint16_t *feat_knn) {
    const size_t nkv = 4ull * nd + 2ull * ne + nn + 4ull * nf;
    std::vector<uint16_t> keys(nkv);
    std::vector<uint32_t> vals(nkv);
    size_t kv = 0;
    uint32_t term = 0;
    for (uint32_t t = 0; t < nd; ++t, ++term)
        for (int i = 0; i < 4; ++i) { keys[kv] = dense_knn[4ull * t + i]; vals[kv++] = term; }
    for (uint32_t e = 0; e < ne; ++e, ++term) {
        const uint16_t x = edges[3ull * e], y = edges[3ull * e + 1];
        keys[kv] = (x != y) ? x : 0xffff; vals[kv++] = term;
        keys[kv] = (x != y) ? y : 0xffff; vals[kv++] = term;
    }
    for (uint32_t n = 0; n < nn; ++n, ++term) { keys[kv] = (uint16_t)n; vals[kv++] = term; }
    for (uint32_t f = 0; f < nf; ++f, ++term)
        for (int i = 0; i < 4; ++i) { keys[kv] = feat_knn[4ull * f + i]; vals[kv++] = term; }
    const auto perm = stable_order(keys);
    Node2Term m;
    m.term_index.resize(nkv);
    std::vector<uint16_t> sk(nkv);
    for (size_t i = 0; i < nkv; ++i) { m.term_index[i] = vals[perm[i]]; sk[i] = keys[perm[i]]; }
    // CSR offsets of every node id; equals computeTermOffsetKernel wherever that
    // kernel writes (it leaves ids below the first present key unwritten).
    m.offset.assign(nn + 1, 0);
    for (uint32_t node = 0; node <= nn; ++node)
        m.offset[node] = (uint32_t)(std::lower_bound(sk.begin(), sk.end(), (uint16_t)std::min<uint32_t>(node, 0xffffu)) - sk.begin());
    // keys >= nn other than 0xffff cannot occur; offset[nn] is the first invalid key.
    return m;
}

struct Pair2Term {
    std::vector<uint32_t> half_row, half_col, half_begin, half_end;   // unique (i<j) pairs + term ranges
    std::vector<uint32_t> term_index;                                  // sorted term values (all kv)
    std::vector<uint32_t> sym_row, sym_col, sym_begin, sym_end;        // symmetric, sorted by (row, col)
    std::vector<uint32_t> blkrow_offset;                               // N + 1
};

// NodePair2TermsIndex (examples/mono_star/opt/NodePair2TermsIndex.cu:11-193, 591-691)
// and computeRowOffsetKernel (NodePairRowColumnIndex.cu:12-36).  Pairs are kept
// as (row, col) 64-bit keys; for ids < 4096 the order equals the reference's
// `row * 4096 + col` encoding (libs/star/opt/solver_encode.h:8-25).
Pair2Term build_pair2term(uint32_t nd, const uint16_t *dense_knn, uint32_t ne, const uint16_t *edges,
                          uint32_t nn, uint32_t nf, const uint16_t *feat_knn) {
    const uint64_t UNINIT = ~0ull;
    const size_t nkv = 6ull * nd + ne + 6ull * nf;
    std::vector<uint64_t> keys(nkv, UNINIT);
    std::vector<uint32_t> vals(nkv);
    auto knn_pairs = [&](const uint16_t *knn, size_t kv0, uint32_t term) {
        size_t off = 0;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j)
                if (knn[i] < knn[j]) { keys[kv0 + off] = ((uint64_t)knn[i] << 32) | knn[j]; ++off; }
        for (size_t k = 0; k < 6; ++k) vals[kv0 + k] = term;
    };
    uint32_t term = 0;
    for (uint32_t t = 0; t < nd; ++t, ++term) knn_pairs(dense_knn + 4ull * t, 6ull * t, term);
    for (uint32_t e = 0; e < ne; ++e, ++term) {
        const uint16_t x = edges[3ull * e], y = edges[3ull * e + 1];
        const size_t kv = 6ull * nd + e;
        if (x < y) keys[kv] = ((uint64_t)x << 32) | y;
        else if (y < x) keys[kv] = ((uint64_t)y << 32) | x;
        vals[kv] = term;
    }
    term += nn;   // node-motion terms own no pairs
    for (uint32_t f = 0; f < nf; ++f, ++term) knn_pairs(feat_knn + 4ull * f, 6ull * nd + ne + 6ull * f, term);

    const auto perm = stable_order(keys);
    Pair2Term m;
    m.term_index.resize(nkv);
    std::vector<uint64_t> sk(nkv);
    for (size_t i = 0; i < nkv; ++i) { m.term_index[i] = vals[perm[i]]; sk[i] = keys[perm[i]]; }
    for (size_t i = 0; i < nkv; ++i) {
        if (sk[i] == UNINIT) break;
        if (i == 0 || sk[i] != sk[i - 1]) {
            if (!m.half_row.empty()) m.half_end.push_back((uint32_t)i);
            m.half_row.push_back((uint32_t)(sk[i] >> 32));
            m.half_col.push_back((uint32_t)(sk[i] & 0xffffffffu));
            m.half_begin.push_back((uint32_t)i);
        }
    }
    if (!m.half_row.empty()) {
        size_t end = nkv;
        for (size_t i = 0; i < nkv; ++i) if (sk[i] == UNINIT) { end = i; break; }
        m.half_end.push_back((uint32_t)end);
    }
    // Symmetric expansion + sort by (row, col).
    const size_t nh = m.half_row.size();
    std::vector<uint64_t> skeys(2 * nh);
    std::vector<uint32_t> sb(2 * nh), se(2 * nh);
    for (size_t k = 0; k < nh; ++k) {
        skeys[2 * k] = ((uint64_t)m.half_row[k] << 32) | m.half_col[k];
        skeys[2 * k + 1] = ((uint64_t)m.half_col[k] << 32) | m.half_row[k];
        sb[2 * k] = sb[2 * k + 1] = m.half_begin[k];
        se[2 * k] = se[2 * k + 1] = m.half_end[k];
    }
    const auto sp = stable_order(skeys);
    m.sym_row.resize(2 * nh); m.sym_col.resize(2 * nh); m.sym_begin.resize(2 * nh); m.sym_end.resize(2 * nh);
    for (size_t i = 0; i < 2 * nh; ++i) {
        m.sym_row[i] = (uint32_t)(skeys[sp[i]] >> 32);
        m.sym_col[i] = (uint32_t)(skeys[sp[i]] & 0xffffffffu);
        m.sym_begin[i] = sb[sp[i]];
        m.sym_end[i] = se[sp[i]];
    }
    m.blkrow_offset.assign(nn + 1, 0);
    for (uint32_t r = 0; r <= nn; ++r)
        m.blkrow_offset[r] = (uint32_t)(std::lower_bound(m.sym_row.begin(), m.sym_row.end(), r) - m.sym_row.begin());
    return m;
}

// ---------------------------------------------------------------------------
// The Gauss-Newton solve, templated on the working precision R.
// ---------------------------------------------------------------------------
struct DenseTerms {
    std::vector<uint16_t> pixels;   // 4 per term: x, y, x + flow_x, y + flow_y
    std::vector<uint16_t> knn;      // 4 per term
    std::vector<float> sw, cw;      // 4 per term
};

// queryPixelKNNKernel + mark + compaction (examples/mono_star/opt/WarpSolver.cu:7-47,
// ImageTermKNNFetcher.cu:9-29, 56-88): raster order, flow target rounded to
// nearest even with unsigned saturation, truncated to 16 bits by make_ushort4.
DenseTerms compact_pixels(int W, int H, const uint32_t *index_map, const float *flow,
                          const uint16_t *surfel_knn, const float *surfel_sw, const float *surfel_cw) {
    DenseTerms d;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const size_t pix = (size_t)y * W + x;
            const uint32_t s = index_map[pix];
            if (s == 0xFFFFFFFFu) continue;
            const float fx = flow ? flow[2 * pix] : 0.f, fy = flow ? flow[2 * pix + 1] : 0.f;
            auto to_u = [](float v) -> uint32_t {
                if (!(v > 0.f)) return 0u;                       // negative / nan saturate to 0
                if (v >= 4294967296.f) return 0xFFFFFFFFu;
                return (uint32_t)std::nearbyint((double)v);      // default rounding: nearest even
            };
            const uint32_t tx = to_u(fx + (float)x), ty = to_u(fy + (float)y);
            d.pixels.push_back((uint16_t)x); d.pixels.push_back((uint16_t)y);
            d.pixels.push_back((uint16_t)tx); d.pixels.push_back((uint16_t)ty);
            for (int k = 0; k < 4; ++k) {
                d.knn.push_back(surfel_knn[4ull * s + k]);
                d.sw.push_back(surfel_sw[4ull * s + k]);
                d.cw.push_back(surfel_cw[4ull * s + k]);
            }
        }
    return d;
}

// R: bulk arithmetic (terms, assembly, SpMV, vectors); RD: PCG dot products, alpha/beta,
// diagonal-block accumulation and the block inverse (Cholesky when RD is double,
// the reference's Gauss-Jordan when RD is float).
template <class R, class RD = R>
struct Solver {
    static constexpr bool kMixed = !std::is_same<R, RD>::value;
    const orc_problem &p;
    const orc_settings &s;
    int threads;
    DenseTerms dense;
    Node2Term n2t;
    Pair2Term p2t;
    TermOffsets off{};
    uint32_t nd = 0, ne = 0, nn = 0, nf = 0;
    std::vector<DQ<R>> se3;
    // per-iteration term data
    std::vector<R> d_res, d_grad;       // 3, 18 per dense term
    std::vector<V3<R>> ti_xj, tj_xj, reg_res;
    std::vector<uint8_t> valid;
    std::vector<R> cweight;
    std::vector<V3<R>> node_t;
    std::vector<V3<R>> center;      // twist centre per node (origin unless node-centred)

    // eps * S^T S for the centre c: [[(1 + |c|^2) I - c c^T, -[c]x], [[c]x, I]] * eps, eps = 1e-3.
    static void centred_regulariser(const V3<R> &cc, RD *out) {
        const RD eps = RD(1e-3f);
        const RD c[3] = {RD(cc.x), RD(cc.y), RD(cc.z)};
        const RD c2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
        const RD X[3][3] = {{0, -c[2], c[1]}, {c[2], 0, -c[0]}, {-c[1], c[0], 0}};   // [c]x
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                out[6 * a + b] = eps * ((a == b ? RD(1) + c2 : RD(0)) - c[a] * c[b]);
                out[6 * a + 3 + b] = -eps * X[a][b];
                out[6 * (3 + a) + b] = eps * X[a][b];
                out[6 * (3 + a) + 3 + b] = (a == b) ? eps : RD(0);
            }
    }

    // Rotation part of a Jacobian row for a twist taken about `c` instead of the origin:
    // rho - c x tau (the translation part tau is unchanged).
    static void recentre(R *row6, const V3<R> &c) {
        const V3<R> tau = {row6[3], row6[4], row6[5]};
        const V3<R> ct = cross(c, tau);
        row6[0] -= ct.x; row6[1] -= ct.y; row6[2] -= ct.z;
    }
    // system
    std::vector<R> diag, inv_diag, b, offdiag, x;
    std::vector<RD> diag_acc;

    Solver(const orc_problem &p_, const orc_settings &s_) : p(p_), s(s_) { threads = set_threads(s.threads); }

    void build_index() {
        dense = compact_pixels(p.width, p.height, p.index_map, p.flow, p.surfel_knn, p.surfel_sw, p.surfel_cw);
        nd = (uint32_t)(dense.knn.size() / 4);
        ne = (uint32_t)p.num_edges;
        nn = (uint32_t)p.num_nodes;
        nf = (uint32_t)p.num_features;
        off = make_offsets(nd, ne, nn, nf);
        n2t = build_node2term(nd, dense.knn.data(), ne, p.edges, nn, nf, p.feature_knn);
        p2t = build_pair2term(nd, dense.knn.data(), ne, p.edges, nn, nf, p.feature_knn);
    }

    SE3<R> world2cam() const {
        SE3<R> T;
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) T.rot.m[i][j] = R(p.world2cam[4 * i + j]);
        }
        T.trans = {R(p.world2cam[3]), R(p.world2cam[7]), R(p.world2cam[11])};
        return T;
    }

    // computeDenseImageJacobianKernel (examples/mono_star/opt/DenseImageJacobianResidual.cu:164-308)
    // with computePointToPlanceICPTermJacobianResidual (:12-25) and
    // computeModifiedOpticalFlow2DTermJacobianResidual (:77-115).
    void eval_dense() {
        d_res.assign(3ull * nd, R(0));
        d_grad.assign(18ull * nd, R(0));
        const SE3<R> w2c = world2cam();
        const int W = p.width, H = p.height;
#pragma omp parallel for num_threads(threads) schedule(static)
        for (long long t = 0; t < (long long)nd; ++t) {
            // averageDualQuaternion, pointer overload: plain weighted sum, no per-node normalize
            // (libs/star/math/DualQuaternion.hpp:244-261)
            DQ<R> avg{{0, 0, 0, 0}, {0, 0, 0, 0}};
            for (int k = 0; k < 4; ++k) {
                const R w = R(dense.sw[4 * t + k]) * R(dense.cw[4 * t + k]);
                const DQ<R> d = se3[dense.knn[4 * t + k]];
                avg.q0 = {avg.q0.x + w * d.q0.x, avg.q0.y + w * d.q0.y, avg.q0.z + w * d.q0.z, avg.q0.w + w * d.q0.w};
                avg.q1 = {avg.q1.x + w * d.q1.x, avg.q1.y + w * d.q1.y, avg.q1.z + w * d.q1.z, avg.q1.w + w * d.q1.w};
            }
            const SE3<R> T = dq_se3(avg);
            const uint16_t sx = dense.pixels[4 * t], sy = dense.pixels[4 * t + 1];
            const uint16_t tx = dense.pixels[4 * t + 2], ty = dense.pixels[4 * t + 3];
            const size_t spix = (size_t)sy * W + sx;
            const V3<R> cv = {R(p.ref_vertex[4 * spix]), R(p.ref_vertex[4 * spix + 1]), R(p.ref_vertex[4 * spix + 2])};
            const V3<R> cn = {R(p.ref_normal[4 * spix]), R(p.ref_normal[4 * spix + 1]), R(p.ref_normal[4 * spix + 2])};
            const V3<R> vw = T.rot.mul(cv) + T.trans;
            const V3<R> nw = T.rot.mul(cn);
            const V3<R> vc = w2c.rot.mul(vw) + w2c.trans;
            const V3<R> nc = w2c.rot.mul(nw);
            if (!(tx < W && ty < H)) continue;
            const size_t tpix = (size_t)ty * W + tx;
            const float *tv4 = p.measure_vertex + 4 * tpix;
            const float *tn4 = p.measure_normal + 4 * tpix;
            const V3<R> tv = {R(tv4[0]), R(tv4[1]), R(tv4[2])};
            const V3<R> tn = {R(tn4[0]), R(tn4[1]), R(tn4[2])};
            bool ok = true;
            // is_zero_vertex (libs/star/math/vector_ops.hpp:152-156), float compares
            if (std::fabs(tv4[0]) < 1e-3 && std::fabs(tv4[1]) < 1e-3 && std::fabs(tv4[2]) < 1e-3) ok = false;
            if (dot(tn, nc) < R(0.7f)) ok = false;                    // global_configs.h:57
            if (std::fabs(tv.z - vc.z) > R(0.03f)) ok = false;         // global_configs.h:58
            if (!ok) continue;
            // target to world: apply_inversed_se3 / transpose_dot
            const V3<R> tvw = w2c.rot.tmul(tv - w2c.trans);
            const V3<R> tnw = w2c.rot.tmul(tn);
            R *res = &d_res[3 * t];
            R *g = &d_grad[18 * t];
            V3<R> diff = vw - tvw;
            if (kMixed) {
                // (R - I) v_ref + t + (v_ref - v_t): the device kernel's cancellation-free form
                M33<R> Rmi = T.rot;
                for (int a = 0; a < 3; ++a) Rmi.m[a][a] = T.rot.m[a][a] - R(1);
                diff = (Rmi.mul(cv) + T.trans) + (cv - tvw);
            }
            res[0] = dot(tnw, diff);
            const V3<R> gr = cross(vw, tnw);
            g[0] = gr.x; g[1] = gr.y; g[2] = gr.z; g[3] = tnw.x; g[4] = tnw.y; g[5] = tnw.z;
            // modified optical flow: e = (P R_w2c)(v_w - v_t), P = first two rows
            const V3<R> row0 = {w2c.rot.m[0][0], w2c.rot.m[0][1], w2c.rot.m[0][2]};
            const V3<R> row1 = {w2c.rot.m[1][0], w2c.rot.m[1][1], w2c.rot.m[1][2]};
            const R ex = dot(row0, diff), ey = dot(row1, diff);
            if (std::sqrt(ex * ex + ey * ey) < R(1e-6f)) continue;
            res[1] = ex; res[2] = ey;
            // gradient rotation rows = rows of (P R) * skew(-v_w)
            const V3<R> mv = {-vw.x, -vw.y, -vw.z};
            auto rot_row = [&](V3<R> r) {
                // r^T * so3(mv), so3(xi) = [[0,-z,y],[z,0,-x],[-y,x,0]] (libs/star/math/twist.hpp:13-26)
                return V3<R>{r.y * mv.z - r.z * mv.y, -r.x * mv.z + r.z * mv.x, r.x * mv.y - r.y * mv.x};
            };
            const V3<R> g1r = rot_row(row0), g2r = rot_row(row1);
            g[6] = g1r.x; g[7] = g1r.y; g[8] = g1r.z; g[9] = row0.x; g[10] = row0.y; g[11] = row0.z;
            g[12] = g2r.x; g[13] = g2r.y; g[14] = g2r.z; g[15] = row1.x; g[16] = row1.y; g[17] = row1.z;
        }
    }

    // forwardWarpSmootherNodeKernel (examples/mono_star/opt/NodeGraphHandler.cu:7-45).
    void eval_reg() {
        ti_xj.resize(ne); tj_xj.resize(ne); reg_res.resize(ne); valid.resize(ne); cweight.resize(ne);
        for (uint32_t e = 0; e < ne; ++e) {
            const uint16_t i = p.edges[3 * e], j = p.edges[3 * e + 1], k = p.edges[3 * e + 2];
            const float *xi = p.node_coords + 4 * i, *xj = p.node_coords + 4 * j;
            const SE3<R> Ti = dq_se3(se3[i]), Tj = dq_se3(se3[j]);
            const V3<R> vj = {R(xj[0]), R(xj[1]), R(xj[2])};
            ti_xj[e] = Ti.rot.mul(vj) + Ti.trans;
            tj_xj[e] = Tj.rot.mul(vj) + Tj.trans;
            {
                M33<R> dR;
                for (int a = 0; a < 3; ++a)
                    for (int c = 0; c < 3; ++c)
                        dR.m[a][c] = (Ti.rot.m[a][c] - (a == c ? R(1) : R(0))) - (Tj.rot.m[a][c] - (a == c ? R(1) : R(0)));
                reg_res[e] = dR.mul(vj) + (Ti.trans - Tj.trans);
            }
            const float dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
            // squared_norm_xyz(xi - xj) > 64 * r^2, float (CLIP_FARAWAY_NODEGRAPH_PAIR)
            const float d2 = sq3_fused(dx, dy, dz);
            valid[e] = (d2 > 64 * p.node_radius_square) ? 0 : 1;
            cweight[e] = R(p.node_cw[(size_t)i * p.graph_k + k]);
        }
        // ComputeNodeMotionKernel (NodeMotionHandler.cu:9-19)
        node_t.resize(nn);
        center.assign(nn, V3<R>{0, 0, 0});
        for (uint32_t n = 0; n < nn; ++n) {
            const SE3<R> T = dq_se3(se3[n]);
            node_t[n] = T.trans;
            // node-centred twist coordinates (mixed mode): centre = current warped node position
            if (kMixed) {
                const float *x = p.node_coords + 4ull * n;
                center[n] = T.rot.mul(V3<R>{R(x[0]), R(x[1]), R(x[2])}) + T.trans;
            }
        }
    }

    // Weight of node `node` in dense term t: the last matching knn slot
    // (libs/star/opt/dense_image_jacobian.cuh:9-42).
    R dense_weight(uint32_t t, uint32_t node) const {
        int slot = 0;
        for (int k = 0; k < 4; ++k) if (dense.knn[4 * t + k] == node) slot = k;
        return R(dense.sw[4 * t + slot]) * R(dense.cw[4 * t + slot]);
    }

    // Reg Jacobian of node `node` in edge e, 3 channel rows of 6
    // (libs/star/opt/node_graph_reg_jacobian.cuh:123-148).
    void reg_jacobian(uint32_t e, bool is_i, R J[3][6]) const {
        const V3<R> a = ti_xj[e], c = tj_xj[e];
        const R w = cweight[e];
        if (is_i) {
            const R rows[3][6] = {{0, a.z, -a.y, 1, 0, 0}, {-a.z, 0, a.x, 0, 1, 0}, {a.y, -a.x, 0, 0, 0, 1}};
            for (int r = 0; r < 3; ++r) for (int q = 0; q < 6; ++q) J[r][q] = rows[r][q] * w;
        } else {
            const R rows[3][6] = {{0, -c.z, c.y, -1, 0, 0}, {c.z, 0, -c.x, 0, -1, 0}, {-c.y, c.x, 0, 0, 0, -1}};
            for (int r = 0; r < 3; ++r) for (int q = 0; q < 6; ++q) J[r][q] = rows[r][q] * w;
        }
    }

    void reg_jacobian_unit(uint32_t e, bool is_i, R J[3][6]) const {
        const V3<R> a = ti_xj[e], c = tj_xj[e];
        const R ri[3][6] = {{0, a.z, -a.y, 1, 0, 0}, {-a.z, 0, a.x, 0, 1, 0}, {a.y, -a.x, 0, 0, 0, 1}};
        const R rj[3][6] = {{0, -c.z, c.y, -1, 0, 0}, {c.z, 0, -c.x, 0, -1, 0}, {-c.y, c.x, 0, 0, 0, -1}};
        for (int r = 0; r < 3; ++r) for (int q = 0; q < 6; ++q) J[r][q] = is_i ? ri[r][q] : rj[r][q];
    }

    void lambdas(R lam2[3], R &reg2, R &node2) const {
        lam2[0] = R(s.lambda_depth) * R(s.lambda_depth);
        lam2[1] = lam2[2] = R(s.lambda_of) * R(s.lambda_of);
        reg2 = R(s.lambda_reg) * R(s.lambda_reg);
        node2 = R(s.lambda_node) * R(s.lambda_node);
    }

    // computeBlockDiagonalPreconditionerKernel (PreconditionerRhsBuilder.cu:110-261) and
    // computeJtResidualWithIndexKernel (JtDotResidualIndexed.cu:40-149).
    void assemble_node() {
        diag.assign(36ull * nn, R(0));
        diag_acc.assign(36ull * nn, RD(0));
        b.assign(6ull * nn, R(0));
        R lam2[3], reg2, node2;
        lambdas(lam2, reg2, node2);
#pragma omp parallel for num_threads(threads) schedule(dynamic, 16)
        for (long long node = 0; node < (long long)nn; ++node) {
            RD D[36] = {0};
            R bb[6] = {0};
            for (uint32_t it = n2t.offset[node]; it < n2t.offset[node + 1]; ++it) {
                const uint32_t term = n2t.term_index[it];
                if (term < off.dense) {
                    const uint32_t t = term;
                    const R w = dense_weight(t, (uint32_t)node);
                    const R *g = &d_grad[18ull * t];
                    const R *r = &d_res[3ull * t];
                    for (int ch = 0; ch < 3; ++ch) {
                        R gl[6];
                        for (int q = 0; q < 6; ++q) gl[q] = g[6 * ch + q];
                        if (kMixed) recentre(gl, center[node]);
                        R J[6];
                        for (int q = 0; q < 6; ++q) J[q] = gl[q] * w;
                        for (int a = 0; a < 6; ++a) for (int c = 0; c < 6; ++c) D[6 * a + c] += RD(lam2[ch] * J[a]) * RD(J[c]);
                        // quirk kept: the right-hand side weights the dense term by w^2
                        const R ow = lam2[ch] * (w * w);
                        for (int q = 0; q < 6; ++q) bb[q] -= ow * r[ch] * gl[q];
                    }
                } else if (term < off.reg) {
                    const uint32_t e = term - off.dense;
                    if (!valid[e]) continue;
                    const bool is_i = ((uint32_t)node == p.edges[3 * e]);
                    R J[3][6];
                    reg_jacobian(e, is_i, J);
                    if (kMixed) for (int ch = 0; ch < 3; ++ch) recentre(J[ch], center[node]);
                    for (int ch = 0; ch < 3; ++ch)
                        for (int a = 0; a < 6; ++a) for (int c = 0; c < 6; ++c) D[6 * a + c] += RD(reg2 * J[ch][a]) * RD(J[ch][c]);
                    // computeRegTermJtResidual (node_graph_reg_jacobian.cuh:193-233)
                    const V3<R> rr = kMixed ? reg_res[e] : ti_xj[e] - tj_xj[e];
                    const R c2 = cweight[e] * cweight[e];
                    R Ju[3][6];
                    reg_jacobian_unit(e, is_i, Ju);
                    if (kMixed) for (int ch = 0; ch < 3; ++ch) recentre(Ju[ch], center[node]);
                    const R res3[3] = {rr.x * c2, rr.y * c2, rr.z * c2};
                    for (int q = 0; q < 6; ++q) bb[q] -= reg2 * (res3[0] * Ju[0][q] + res3[1] * Ju[1][q] + res3[2] * Ju[2][q]);
                } else if (term < off.node) {
                    const uint32_t n = term - off.reg;
                    const float *pred = p.node_motion_pred ? p.node_motion_pred + 4ull * n : nullptr;
                    const R conf = pred ? R(pred[3]) : R(0);
                    if (kMixed && node2 != R(0) && pred) {
                        for (int ch = 0; ch < 3; ++ch) {
                            R J[6] = {0, 0, 0, 0, 0, 0};
                            J[3 + ch] = conf;
                            recentre(J, center[node]);
                            for (int a = 0; a < 6; ++a) for (int c = 0; c < 6; ++c) D[6 * a + c] += RD(node2 * J[a]) * RD(J[c]);
                            const R res = (ch == 0 ? node_t[n].x - R(pred[0]) : ch == 1 ? node_t[n].y - R(pred[1]) : node_t[n].z - R(pred[2]));
                            for (int q = 0; q < 6; ++q) bb[q] -= node2 * res * conf * J[q];
                        }
                        continue;
                    }
                    for (int a = 0; a < 3; ++a) D[6 * (3 + a) + 3 + a] += RD(node2 * conf * conf);
                    if (pred) {
                        const R c2 = conf * conf;
                        bb[3] -= node2 * (node_t[n].x - R(pred[0])) * c2;
                        bb[4] -= node2 * (node_t[n].y - R(pred[1])) * c2;
                        bb[5] -= node2 * (node_t[n].z - R(pred[2])) * c2;
                    }
                } else {
                    // feature term: zero Jacobian (PreconditionerRhsBuilder.cu:214-219)
                }
            }
            if (kMixed) {
                // the reference's +1e-3 I on the origin twist, seen in node-centred coordinates:
                // 1e-3 S^T S with S = [[I, 0], [[c]x, I]]
                RD reg[36];
                centred_regulariser(center[node], reg);
                for (int q = 0; q < 36; ++q) D[q] += reg[q];
            } else {
                for (int a = 0; a < 6; ++a) D[7 * a] += RD(1e-3f);
            }
            for (int q = 0; q < 36; ++q) { diag[36 * node + q] = R(D[q]); diag_acc[36 * node + q] = D[q]; }
            for (int q = 0; q < 6; ++q) b[6 * node + q] = bb[q];
        }
    }

    // computeJtJNonDiagonalBlockKernel (examples/mono_star/opt/JtJMaterializer.cu:66-174) +
    // assembleBinBlockCSRKernel (JtJMaterializerBinBlockCSR.cu:8-41): the assembled
    // entry A[6*row + r][6*col + c] = sum lambda^2 (J_row^T J_col)[r][c].
    void assemble_pairs() {
        const size_t ns = p2t.sym_row.size();
        offdiag.assign(36 * ns, R(0));
        R lam2[3], reg2, node2;
        lambdas(lam2, reg2, node2);
#pragma omp parallel for num_threads(threads) schedule(dynamic, 64)
        for (long long k = 0; k < (long long)ns; ++k) {
            const uint32_t row = p2t.sym_row[k], col = p2t.sym_col[k];
            R A[36] = {0};
            for (uint32_t it = p2t.sym_begin[k]; it < p2t.sym_end[k]; ++it) {
                const uint32_t term = p2t.term_index[it];
                if (term < off.dense) {
                    const R wr = dense_weight(term, row), wc = dense_weight(term, col);
                    const R *g = &d_grad[18ull * term];
                    for (int ch = 0; ch < 3; ++ch) {
                        const R f = lam2[ch] * (wr * wc);
                        R gr[6], gc[6];
                        for (int q = 0; q < 6; ++q) gr[q] = gc[q] = g[6 * ch + q];
                        if (kMixed) { recentre(gr, center[row]); recentre(gc, center[col]); }
                        for (int a = 0; a < 6; ++a) for (int c = 0; c < 6; ++c) A[6 * a + c] += f * gr[a] * gc[c];
                    }
                } else if (term < off.reg) {
                    const uint32_t e = term - off.dense;
                    if (!valid[e]) continue;
                    // computeRegJtJLocalBlock (libs/star/opt/node_graph_reg_jacobian.cuh:273-358):
                    // unweighted Jacobians scaled once by lambda^2 c^2
                    R Jr[3][6], Jc[3][6];
                    reg_jacobian_unit(e, row == p.edges[3 * e], Jr);
                    reg_jacobian_unit(e, col == p.edges[3 * e], Jc);
                    if (kMixed) for (int ch = 0; ch < 3; ++ch) { recentre(Jr[ch], center[row]); recentre(Jc[ch], center[col]); }
                    const R ws = reg2 * (cweight[e] * cweight[e]);
                    for (int ch = 0; ch < 3; ++ch)
                        for (int a = 0; a < 6; ++a) for (int c = 0; c < 6; ++c) A[6 * a + c] += (ws * Jr[ch][a]) * Jc[ch][c];
                }
                // node-motion terms own no pairs; feature terms have zero Jacobian
            }
            for (int q = 0; q < 36; ++q) offdiag[36 * k + q] = A[q];
        }
    }

    // DenseGaussian<6>::Inverse with partial pivoting (libs/star/math/DenseGaussian.hpp:33-112).
    static void gauss_jordan_inverse(const R *in, R *out) {
        R m[36];
        for (int i = 0; i < 36; ++i) m[i] = in[i];
        int perm[6], reloc[6];
        for (int i = 0; i < 6; ++i) perm[i] = i;
        for (int i = 0; i < 6; ++i) {
            int piv = i;
            R pv = std::fabs(m[6 * i + i]);
            for (int j = i + 1; j < 6; ++j)
                if (pv < std::fabs(m[6 * j + i])) { pv = std::fabs(m[6 * j + i]); piv = j; }
            for (int k = 0; k < 6; ++k) std::swap(m[6 * i + k], m[6 * piv + k]);
            std::swap(perm[i], perm[piv]);
            reloc[i] = perm[i];
            const R inv = R(1) / m[6 * i + i];
            for (int k = 0; k < 6; ++k) m[6 * i + k] *= inv;
            m[6 * i + i] = inv;
            for (int r = 0; r < 6; ++r) {
                if (r == i) continue;
                const R a = m[6 * r + i];
                for (int k = 0; k < 6; ++k) m[6 * r + k] -= a * m[6 * i + k];
                m[6 * r + i] = -a * m[6 * i + i];
            }
        }
        for (int j = 0; j < 6; ++j)
            for (int i = 0; i < 6; ++i) out[6 * reloc[j] + i] = m[6 * i + j];
    }

    // Symmetric 6x6 inverse by Cholesky in double (the FP64 block inversion).
    template <class T>
    static void cholesky_inverse(const T *in, R *out) {
        double L[36] = {0};
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j <= i; ++j) {
                double sum = (double)in[6 * i + j];
                for (int k = 0; k < j; ++k) sum -= L[6 * i + k] * L[6 * j + k];
                if (i == j) L[6 * i + i] = std::sqrt(sum > 0 ? sum : 1e-300);
                else L[6 * i + j] = sum / L[6 * j + j];
            }
        double Linv[36] = {0};
        for (int i = 0; i < 6; ++i) {
            Linv[6 * i + i] = 1.0 / L[6 * i + i];
            for (int j = 0; j < i; ++j) {
                double sum = 0;
                for (int k = j; k < i; ++k) sum -= L[6 * i + k] * Linv[6 * k + j];
                Linv[6 * i + j] = sum / L[6 * i + i];
            }
        }
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) {
                double sum = 0;
                for (int k = std::max(i, j); k < 6; ++k) sum += Linv[6 * k + i] * Linv[6 * k + j];
                out[6 * i + j] = (R)sum;
            }
    }

    void invert_diag() {
        inv_diag.assign(36ull * nn, R(0));
#pragma omp parallel for num_threads(threads) schedule(static)
        for (long long n = 0; n < (long long)nn; ++n) {
            if (std::is_same<RD, double>::value) cholesky_inverse(&diag_acc[36 * n], &inv_diag[36 * n]);
            else gauss_jordan_inverse(&diag[36 * n], &inv_diag[36 * n]);
        }
    }

    void spmv(const std::vector<R> &d, std::vector<R> &q) const {
#pragma omp parallel for num_threads(threads) schedule(static)
        for (long long row = 0; row < (long long)nn; ++row) {
            R acc[6] = {0};
            const R *D = &diag[36 * row];
            for (int a = 0; a < 6; ++a)
                for (int c = 0; c < 6; ++c) acc[a] += D[6 * a + c] * d[6 * row + c];
            for (uint32_t k = p2t.blkrow_offset[row]; k < p2t.blkrow_offset[row + 1]; ++k) {
                const R *A = &offdiag[36ull * k];
                const uint32_t col = p2t.sym_col[k];
                for (int a = 0; a < 6; ++a)
                    for (int c = 0; c < 6; ++c) acc[a] += A[6 * a + c] * d[6ull * col + c];
            }
            for (int a = 0; a < 6; ++a) q[6 * row + a] = acc[a];
        }
    }

    void precond(const std::vector<R> &in, std::vector<R> &out) const {
#pragma omp parallel for num_threads(threads) schedule(static)
        for (long long n = 0; n < (long long)nn; ++n) {
            const R *M = &inv_diag[36 * n];
            for (int a = 0; a < 6; ++a) {
                R acc = 0;
                for (int c = 0; c < 6; ++c) acc += M[6 * a + c] * in[6 * n + c];
                out[6 * n + a] = acc;
            }
        }
    }

    RD vdot(const std::vector<R> &a, const std::vector<R> &bv) const {
        RD acc = 0;
#pragma omp parallel for num_threads(threads) reduction(+ : acc) schedule(static)
        for (long long i = 0; i < (long long)a.size(); ++i) acc += RD(a[i]) * RD(bv[i]);
        return acc;
    }

    // BlockPCG<6>::SolveNoConvergeCheck (libs/star/pcg_solver/BlockPCG.cuh:67-190, 325-484).
    // A zero curvature or zero residual yields a zero step instead of 0/0.
    void pcg() {
        const size_t n6 = 6ull * nn;
        x.assign(n6, R(0));
        std::vector<R> r = b, d(n6), q(n6), t(n6), sv(n6);
        precond(r, d);
        RD delta = vdot(r, d);
        for (int it = 0; it < s.pcg_iters; ++it) {
            spmv(d, q);
            const RD dq = vdot(d, q);
            const R alpha = R((dq != RD(0)) ? delta / dq : RD(0));
            for (size_t i = 0; i < n6; ++i) { x[i] += alpha * d[i]; t[i] = r[i] - alpha * q[i]; }
            precond(t, sv);
            const RD delta_old = delta;
            delta = vdot(t, sv);
            const R beta = R((delta_old != RD(0)) ? delta / delta_old : RD(0));
            for (size_t i = 0; i < n6; ++i) d[i] = sv[i] + beta * d[i];
            r.swap(t);
        }
    }

    // ApplyWarpFieldUpdateKernel (SolverIterationData.cu:19-74).
    void update() {
        for (uint32_t n = 0; n < nn; ++n) {
            R xo[6];
            for (int q = 0; q < 6; ++q) xo[q] = x[6ull * n + q];
            if (kMixed) {
                // local twist about c -> origin twist: t = t' + c x w
                const V3<R> cw = cross(center[n], V3<R>{xo[0], xo[1], xo[2]});
                xo[3] += cw.x; xo[4] += cw.y; xo[5] += cw.z;
            }
            const SE3<R> inc = twist_to_se3(xo);
            const SE3<R> prev = dq_to_mat34(se3[n]);
            SE3<R> nw;
            nw.rot = matmul(inc.rot, prev.rot);
            nw.trans = inc.rot.mul(prev.trans) + inc.trans;
            se3[n] = dq_from_mat34(nw);
        }
    }

    void run(float *out_dq, orc_debug *dbg) {
        build_index();
        se3.resize(nn);
        for (uint32_t n = 0; n < nn; ++n) {
            if (p.init_dq) se3[n] = load_dq<R>(p.init_dq + 8ull * n);
            else se3[n] = DQ<R>{{0, 0, 0, 1}, {0, 0, 0, 0}};
        }
        for (int it = 0; it < s.gn_iters; ++it) {
            eval_dense();
            eval_reg();
            assemble_node();
            invert_diag();
            assemble_pairs();
            pcg();
            if (it == 0 && dbg) dump(dbg);
            update();
        }
        for (uint32_t n = 0; n < nn; ++n) {
            const DQ<R> &d = se3[n];
            const float v[8] = {(float)d.q0.x, (float)d.q0.y, (float)d.q0.z, (float)d.q0.w,
                                (float)d.q1.x, (float)d.q1.y, (float)d.q1.z, (float)d.q1.w};
            std::memcpy(out_dq + 8ull * n, v, sizeof(v));
        }
    }

    void dump(orc_debug *dbg) {
        dbg->num_dense_terms = (int)nd;
        dbg->num_sym_pairs = (int)p2t.sym_row.size();
        if (dbg->dense_residual && (int)nd <= dbg->capacity_terms)
            for (size_t i = 0; i < 3ull * nd; ++i) dbg->dense_residual[i] = (float)d_res[i];
        if (dbg->dense_gradient && (int)nd <= dbg->capacity_terms)
            for (size_t i = 0; i < 18ull * nd; ++i) dbg->dense_gradient[i] = (float)d_grad[i];
        if (dbg->diag_blocks) for (size_t i = 0; i < diag.size(); ++i) dbg->diag_blocks[i] = (float)diag[i];
        if (dbg->inv_diag_blocks) for (size_t i = 0; i < inv_diag.size(); ++i) dbg->inv_diag_blocks[i] = (float)inv_diag[i];
        if (dbg->jtr) for (size_t i = 0; i < b.size(); ++i) dbg->jtr[i] = (float)b[i];
        const size_t ns = p2t.sym_row.size();
        if ((int)ns <= dbg->capacity_pairs) {
            if (dbg->sym_rows) for (size_t i = 0; i < ns; ++i) dbg->sym_rows[i] = p2t.sym_row[i];
            if (dbg->sym_cols) for (size_t i = 0; i < ns; ++i) dbg->sym_cols[i] = p2t.sym_col[i];
            if (dbg->offdiag_blocks) for (size_t i = 0; i < 36 * ns; ++i) dbg->offdiag_blocks[i] = (float)offdiag[i];
        }
        if (dbg->pcg_x) for (size_t i = 0; i < x.size(); ++i) dbg->pcg_x[i] = (float)x[i];
    }
};

}  // namespace

extern "C" {

int orc_version(void) { return 1; }

// VoxelSubsamplerSorting (libs/star/geometry/sampling/VoxelSubsamplerSorting.cu:8-96, 171-272)
// with encodeVoxel/decodeVoxel (libs/star/common/encode_utils.h:138-150).
int orc_voxel_subsample(const float *pts4, int n, float voxel, float *out4, int cap, int *n_out) {
    if (n <= 0) { *n_out = 0; return 0; }
    std::vector<int> keys(n);
    for (int i = 0; i < n; ++i) {
        const int vx = (int)std::floor(pts4[4 * i] / voxel);
        const int vy = (int)std::floor(pts4[4 * i + 1] / voxel);
        const int vz = (int)std::floor(pts4[4 * i + 2] / voxel);
        // encodeVoxel in 32-bit two's complement (the reference's int arithmetic wraps the same way)
        keys[i] = (int)((unsigned)(vx + 512) + (unsigned)(vy + 512) * 1024u + (unsigned)(vz + 512) * 1048576u);
    }
    const auto perm = stable_order(keys);
    int count = 0;
    for (int b = 0; b < n;) {
        int e = b + 1;
        while (e < n && keys[perm[e]] == keys[perm[b]]) ++e;
        const int enc = keys[perm[b]];
        int z = enc / (1024 * 1024);
        int x = enc % 1024;
        int y = (enc - z * 1024 * 1024) / 1024;
        x -= 512; y -= 512; z -= 512;
        const float cx = (float)(x + 0.5) * voxel, cy = (float)(y + 0.5) * voxel, cz = (float)(z + 0.5) * voxel;
        float best = 1e5f;
        int best_i = b;
        for (int i = b; i < e; ++i) {
            const float *q = pts4 + 4 * perm[i];
            const float dd = sq3_fused(q[0] - cx, q[1] - cy, q[2] - cz);
            if (dd < best) { best = dd; best_i = i; }
        }
        if (count >= cap) return -1;
        std::memcpy(out4 + 4 * count, pts4 + 4 * perm[best_i], 16);
        ++count;
        b = e;
    }
    *n_out = count;
    return 0;
}

// NodeGraph::InitializeNodeGraphFromVertex + AppendNodeFromVertexHost
// (libs/star/geometry/node_graph/NodeGraph.cu:460-498, 652-704).
int orc_init_nodes(const float *pts4, int n, float node_radius, float *out4, int cap, int *n_nodes) {
    std::vector<float> cand(4ull * std::max(n, 1));
    int nc = 0;
    if (n > 0 && orc_voxel_subsample(pts4, n, 0.7f * node_radius, cand.data(), n, &nc) != 0) return -1;
    const float r = 0.85f * node_radius;
    const float sample_distance_square = r * r;
    std::vector<float> acc;
    for (int i = 0; i < nc; ++i) {
        const float px = cand[4 * i], py = cand[4 * i + 1], pz = cand[4 * i + 2];
        if (std::isnan(px) || std::isnan(py) || std::isnan(pz)) return -2;
        bool is_node = true;
        for (size_t j = 0; j < acc.size(); j += 4) {
            const float dx = acc[j] - px, dy = acc[j + 1] - py, dz = acc[j + 2] - pz, dw = 1.0f - 1.0f;
            const float d2 = ((dx * dx + dy * dy) + dz * dz) + dw * dw;
            if (d2 <= sample_distance_square) { is_node = false; break; }
        }
        if (is_node) { acc.push_back(px); acc.push_back(py); acc.push_back(pz); acc.push_back(1.0f); }
    }
    const int total = (int)(acc.size() / 4) + 2;
    if (total > cap) return -1;
    for (int a = 0; a < 2; ++a) { out4[4 * a] = 0.f; out4[4 * a + 1] = 0.f; out4[4 * a + 2] = 0.f; out4[4 * a + 3] = 1.f; }
    std::memcpy(out4 + 8, acc.data(), acc.size() * sizeof(float));
    *n_nodes = total;
    return 0;
}

// UpdateNodeDistanceKernel + BuildNodeGraphKernel (NodeGraph.cu:10-101): half squared
// distances, K nearest including self, exp weights, divided by their sum when `normalize`
// (USE_INTERPOLATE_WEIGHT_NORMALIZATION, NodeGraph.cu:87-99).  A pair with a deleted node
// (status[2 i + 1] == 0xFFFFFFFF, NodeGraph.h:18) has the half of 1e6 (infinite) as distance
// (NodeGraph.cu:20-35).  The weights use expf here; the device code uses __expf, so weights
// agree to a few ulps only.
int orc_node_graph_ex(const float *nodes4, const uint32_t *status, int n, int k, float node_radius, int normalize,
                      uint16_t *knn, float *spatial_w) {
    if (k != 4 && k != 8) return -3;
    const float r2 = node_radius * node_radius;
    auto deleted = [&](int i) { return status != nullptr && status[2 * i + 1] == 0xFFFFFFFFu; };
#pragma omp parallel for schedule(dynamic, 16)
    for (int a = 0; a < n; ++a) {
        auto dist = [&](int b) {
            if (deleted(a) || deleted(b)) return half_to_float(float_to_half_rn(1e6f));
            const int hi = std::max(a, b), lo = std::min(a, b);
            const float dx = nodes4[4 * hi] - nodes4[4 * lo];
            const float dy = nodes4[4 * hi + 1] - nodes4[4 * lo + 1];
            const float dz = nodes4[4 * hi + 2] - nodes4[4 * lo + 2];
            const float d = std::fmaf(dz, dz, std::fmaf(dy, dy, dx * dx));
            return half_to_float(float_to_half_rn(d));
        };
        auto finish = [&](const float *dd, const uint16_t *ii) {
            float w[8], sum = 0.f;
            for (int q = 0; q < k; ++q) { w[q] = std::exp(-dd[q] / (2 * r2)); }
            for (int q = 0; q < k; ++q) sum += w[q];
            const float inv = 1.0f / sum;
            for (int q = 0; q < k; ++q) {
                knn[(size_t)a * k + q] = ii[q];
                spatial_w[(size_t)a * k + q] = normalize ? w[q] * inv : w[q];
            }
        };
        if (k == 4) {
            KnnHeap<4> h(1e3f);
            for (int b = 0; b < n; ++b) h.update((uint16_t)b, dist(b));
            h.sort();
            finish(h.distance, h.index);
        } else {
            KnnHeap<8> h(1e3f);
            for (int b = 0; b < n; ++b) h.update((uint16_t)b, dist(b));
            h.sort();
            finish(h.distance, h.index);
        }
    }
    return 0;
}

int orc_node_graph(const float *nodes4, int n, int k, float node_radius, uint16_t *knn, float *spatial_w) {
    return orc_node_graph_ex(nodes4, nullptr, n, k, node_radius, 1, knn, spatial_w);
}

// SkinnerKernel (libs/star/geometry/node_graph/Skinner.cu:10-94) and IncSkinnerKernel (:211-302).
// A deleted node enters at distance 1e6 (Skinner.cu:39-48).  With prev_nodes > 0 the surfels
// first_vert .. n_verts - 1 start their heap from their current neighbours (knn on input) at their
// distances and take the nodes prev_nodes .. n_nodes - 1; otherwise every surfel starts at 1e6
// and takes all nodes.  Weights exp(-d / (2 r^2)), divided by their sum when `normalize`.
int orc_skinning_ex(const float *nodes4, const uint32_t *status, int n_nodes, int prev_nodes, const float *verts4,
                    int first_vert, int n_verts, float node_radius, int normalize, uint16_t *knn, float *spatial_w,
                    float *connect_w, int threads) {
    if (prev_nodes < 0 || prev_nodes > n_nodes || first_vert < 0 || first_vert > n_verts) return -1;
    const float r2 = node_radius * node_radius;
    const int th = set_threads(threads);
    auto deleted = [&](int i) { return status != nullptr && status[2 * i + 1] == 0xFFFFFFFFu; };
#pragma omp parallel for num_threads(th) schedule(static)
    for (int v = first_vert; v < n_verts; ++v) {
        const float *p = verts4 + 4ull * v;
        KnnHeap<4> h(1e6f);
        if (prev_nodes > 0) {
            float d0[4];
            uint16_t i0[4];
            for (int i = 0; i < 4; ++i) {
                i0[i] = knn[4ull * v + i];
                const float *q = nodes4 + 4ull * std::min<int>(i0[i], n_nodes - 1);
                d0[i] = sq3_fused(p[0] - q[0], p[1] - q[1], p[2] - q[2]);
            }
            h = KnnHeap<4>(d0, i0);
        }
        for (int i = prev_nodes; i < n_nodes; ++i) {
            const float *q = nodes4 + 4ull * i;
            h.update((uint16_t)i, deleted(i) ? 1e6f : sq3_fused(p[0] - q[0], p[1] - q[1], p[2] - q[2]));
        }
        h.sort();
        float w[4], sum = 0.f;
        for (int i = 0; i < 4; ++i) {
            const float *q = nodes4 + 4ull * std::min<int>(h.index[i], n_nodes - 1);
            const float d = sq3_fused(p[0] - q[0], p[1] - q[1], p[2] - q[2]);
            w[i] = std::exp(-d / (2.f * r2));
            sum += w[i];
        }
        const float inv = 1.f / sum;
        for (int i = 0; i < 4; ++i) {
            knn[4ull * v + i] = h.index[i];
            spatial_w[4ull * v + i] = normalize ? inv * w[i] : w[i];
            connect_w[4ull * v + i] = 1.f;
        }
    }
    return 0;
}

int orc_skinning(const float *nodes4, int n_nodes, const float *verts4, int n_verts, float node_radius,
                 uint16_t *knn, float *spatial_w, float *connect_w, int threads) {
    return orc_skinning_ex(nodes4, nullptr, n_nodes, 0, verts4, 0, n_verts, node_radius, 1, knn, spatial_w, connect_w,
                           threads);
}

int orc_compact_pixels(int width, int height, const uint32_t *index_map, const float *flow,
                       const uint16_t *surfel_knn, const float *surfel_sw, const float *surfel_cw,
                       uint16_t *pixels, uint16_t *knn, float *sw, float *cw, int cap, int *n_terms) {
    const DenseTerms d = compact_pixels(width, height, index_map, flow, surfel_knn, surfel_sw, surfel_cw);
    const int nt = (int)(d.knn.size() / 4);
    *n_terms = nt;
    if (nt > cap) return -1;
    std::memcpy(pixels, d.pixels.data(), d.pixels.size() * 2);
    std::memcpy(knn, d.knn.data(), d.knn.size() * 2);
    std::memcpy(sw, d.sw.data(), d.sw.size() * 4);
    std::memcpy(cw, d.cw.data(), d.cw.size() * 4);
    return 0;
}

int orc_node2term(int n_dense, const uint16_t *dense_knn, int n_edges, const uint16_t *edges,
                  int n_nodes, int n_feat, const uint16_t *feat_knn,
                  uint32_t *offsets, uint32_t *term_index, int cap_kv, int *n_kv) {
    const Node2Term m = build_node2term(n_dense, dense_knn, n_edges, edges, n_nodes, n_feat, feat_knn);
    *n_kv = (int)m.term_index.size();
    if ((int)m.term_index.size() > cap_kv) return -1;
    std::memcpy(offsets, m.offset.data(), m.offset.size() * 4);
    std::memcpy(term_index, m.term_index.data(), m.term_index.size() * 4);
    return 0;
}

int orc_nodepair2term(int n_dense, const uint16_t *dense_knn, int n_edges, const uint16_t *edges,
                      int n_nodes, int n_feat, const uint16_t *feat_knn,
                      uint32_t *half_rows, uint32_t *half_cols, uint32_t *half_begin,
                      uint32_t *half_end, int cap_half, int *n_half,
                      uint32_t *term_index, int cap_kv, int *n_kv,
                      uint32_t *sym_rows, uint32_t *sym_cols, uint32_t *sym_begin,
                      uint32_t *sym_end, uint32_t *blkrow_offset) {
    const Pair2Term m = build_pair2term(n_dense, dense_knn, n_edges, edges, n_nodes, n_feat, feat_knn);
    const int nh = (int)m.half_row.size();
    *n_half = nh;
    *n_kv = (int)m.term_index.size();
    if (nh > cap_half || (int)m.term_index.size() > cap_kv) return -1;
    std::memcpy(half_rows, m.half_row.data(), 4ull * nh);
    std::memcpy(half_cols, m.half_col.data(), 4ull * nh);
    std::memcpy(half_begin, m.half_begin.data(), 4ull * nh);
    std::memcpy(half_end, m.half_end.data(), 4ull * nh);
    std::memcpy(term_index, m.term_index.data(), 4 * m.term_index.size());
    std::memcpy(sym_rows, m.sym_row.data(), 8ull * nh);
    std::memcpy(sym_cols, m.sym_col.data(), 8ull * nh);
    std::memcpy(sym_begin, m.sym_begin.data(), 8ull * nh);
    std::memcpy(sym_end, m.sym_end.data(), 8ull * nh);
    std::memcpy(blkrow_offset, m.blkrow_offset.data(), 4ull * (n_nodes + 1));
    return 0;
}

// Bin-Blocked CSR structure (NodePairRowColumnIndex.cu:38-125, 383-474;
// libs/star/pcg_solver/note.md): 32 scalar rows per bin, column-major inside a
// bin, bin length = 6 * the longest block row, padding column = -1.
int orc_binblock_csr(int n_nodes, int n_sym, const uint32_t *sym_rows, const uint32_t *sym_cols,
                     int *rowptr, int cap_rowptr, int *n_rowptr, int *colptr, int cap_colptr) {
    const int bin = 32, dim = 6;
    std::vector<uint32_t> off(n_nodes + 1);
    for (int r = 0; r <= n_nodes; ++r)
        off[r] = (uint32_t)(std::lower_bound(sym_rows, sym_rows + n_sym, (uint32_t)r) - sym_rows);
    std::vector<uint32_t> len(n_nodes);
    for (int r = 0; r < n_nodes; ++r) len[r] = 1 + off[r + 1] - off[r];
    const int matrix = n_nodes * dim;
    const int nbins = (matrix + bin - 1) / bin;
    std::vector<uint32_t> nnz(nbins + 1, 0), scan(nbins + 1, 0);
    for (int b = 0; b < nbins; ++b) {
        const uint32_t rb = (uint32_t)(bin * b / dim);
        uint32_t re = (uint32_t)((bin * b + bin - 1) / dim);
        re = std::min<uint32_t>(re, (uint32_t)n_nodes - 1);
        uint32_t mx = 0;
        for (uint32_t r = rb; r <= re; ++r) mx = std::max(mx, len[r]);
        nnz[b] = bin * (dim * mx);
    }
    for (int b = 1; b <= nbins; ++b) scan[b] = scan[b - 1] + nnz[b - 1];
    const int nrp = bin * (nbins + 1);
    *n_rowptr = nrp;
    if (nrp > cap_rowptr) return -1;
    for (int i = 0; i < nrp; ++i) rowptr[i] = (int)(i % bin + scan[i / bin]);
    const int ncol = (int)(scan[nbins] / dim);
    if (ncol > cap_colptr) return -1;
    for (int i = 0; i < cap_colptr; ++i) colptr[i] = -1;
    for (int row = 0; row < matrix; ++row) {
        const int br = row / dim;
        const int data_offset = rowptr[row];
        const int lane = row & 31;
        int c = (data_offset - lane) / dim + lane;
        colptr[c] = dim * br;
        c += bin;
        for (uint32_t k = off[br]; k < off[br + 1]; ++k, c += bin) colptr[c] = (int)(dim * sym_cols[k]);
    }
    return 0;
}

int orc_solve(const orc_problem *p, const orc_settings *s, float *out_dq, orc_debug *dbg) {
    if (!p || !s || !out_dq) return -1;
    if (p->num_nodes <= 0) return -2;
    if (s->precision == ORC_PREC_FP64) {
        Solver<double> sv(*p, *s);
        sv.run(out_dq, dbg);
    } else if (s->precision == ORC_PREC_MIXED) {
        Solver<float, double> sv(*p, *s);
        sv.run(out_dq, dbg);
    } else {
        Solver<float> sv(*p, *s);
        sv.run(out_dq, dbg);
    }
    return 0;
}

// ForwardWarpVertexAndNodeKernel (libs/star/geometry/surfel/SurfelNodeDeformer.cu:13-79) with
// averageDualQuaternion<4> (DualQuaternion.hpp:288-306), which normalizes every node DQ.
int orc_forward_warp(const float *node_dq, int n_nodes, const float *verts4, int n_verts,
                     const uint16_t *knn, const float *sw, const float *cw, float *out4, int threads) {
    (void)n_nodes;
    const int th = set_threads(threads);
#pragma omp parallel for num_threads(th) schedule(static)
    for (int v = 0; v < n_verts; ++v) {
        DQ<double> avg{{0, 0, 0, 0}, {0, 0, 0, 0}};
        for (int k = 0; k < 4; ++k) {
            DQ<double> d = load_dq<double>(node_dq + 8ull * knn[4ull * v + k]);
            dq_normalize(d);
            const double w = (double)sw[4ull * v + k] * (double)cw[4ull * v + k];
            avg.q0 = {avg.q0.x + w * d.q0.x, avg.q0.y + w * d.q0.y, avg.q0.z + w * d.q0.z, avg.q0.w + w * d.q0.w};
            avg.q1 = {avg.q1.x + w * d.q1.x, avg.q1.y + w * d.q1.y, avg.q1.z + w * d.q1.z, avg.q1.w + w * d.q1.w};
        }
        const SE3<double> T = dq_se3(avg);
        const V3<double> pv = {verts4[4ull * v], verts4[4ull * v + 1], verts4[4ull * v + 2]};
        const V3<double> o = T.rot.mul(pv) + T.trans;
        out4[4ull * v] = (float)o.x; out4[4ull * v + 1] = (float)o.y; out4[4ull * v + 2] = (float)o.z;
        out4[4ull * v + 3] = verts4[4ull * v + 3];
    }
    return 0;
}

/* ---- measurement maps (img_proc/vertex_map.cu, img_proc/normal_map.cu, math/eigen33.hpp) ---- */
namespace meas {
struct P3 {
    float x, y, z;
};
static inline P3 p3(float x, float y, float z) { return P3{x, y, z}; }
static inline P3 pcross(P3 a, P3 b) { return p3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline float pdot(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline P3 pmul(P3 a, float s) { return p3(a.x * s, a.y * s, a.z * s); }
static inline float inv_sqrt(float v) { return 1.0f / sqrtf(v); }   // eigen33.h host branch
static const float kEps = 1.192092896e-07f;                          // numeric_limits.hpp:30-32
static const float kMinPos = 1.175494351e-38f;                       // numeric_limits.hpp:35-37

static inline bool is_zero(P3 v) {   // vector_ops.hpp:123-126
    return fabsf(v.x) < 1e-3f && fabsf(v.y) < 1e-3f && fabsf(v.z) < 1e-3f;
}
// eigen33::compute_root2 (eigen33.hpp:6-17)
static void root2(float b, float c, P3 &r) {
    r.x = 0.0f;
    float d = b * b - 4.f * c;
    if (d < 0.f) d = 0.f;
    const float sd = sqrtf(d);
    r.z = 0.5f * (b + sd);
    r.y = 0.5f * (b - sd);
}
// eigen33::compute_root3 (eigen33.hpp:50-98)
static void root3(float c0, float c1, float c2, P3 &r) {
    if (fabsf(c0) < kEps) {
        root2(c2, c1, r);
        return;
    }
    const float inv3 = 1.f / 3.f, sq3 = sqrtf(3.f);
    const float c2o3 = c2 * inv3;
    float ao3 = (c1 - c2 * c2o3) * inv3;
    if (ao3 > 0.f) ao3 = 0.f;
    const float hb = 0.5f * (c0 + c2o3 * (2.f * c2o3 * c2o3 - c1));
    float q = hb * hb + ao3 * ao3 * ao3;
    if (q > 0.f) q = 0.f;
    const float rho = sqrtf(-ao3);
    const float th = atan2f(sqrtf(-q), hb) * inv3;
    const float ct = cosf(th), st = sinf(th);
    r.x = c2o3 + 2.f * rho * ct;
    r.y = c2o3 - rho * (ct + sq3 * st);
    r.z = c2o3 - rho * (ct - sq3 * st);
    if (r.x >= r.y) std::swap(r.x, r.y);
    if (r.y >= r.z) {
        std::swap(r.y, r.z);
        if (r.x >= r.y) std::swap(r.x, r.y);
    }
    if (r.x <= 0.0f) root2(c2, c1, r);
}
// eigen33::unit_orthogonal (eigen33.hpp:19-48)
static P3 unit_orth(P3 s) {
    const float pe = kEps * kEps;
    const bool xs = s.x * s.x <= pe * s.z * s.z, ys = s.y * s.y <= pe * s.z * s.z;
    if (!xs || !ys) {
        const float inv = inv_sqrt(s.x * s.x + s.y * s.y);
        return p3(-s.y * inv, s.x * inv, 0.0f);
    }
    const float inv = inv_sqrt(s.z * s.z + s.y * s.y);
    return p3(0.0f, -s.z * inv, s.y * inv);
}
// the longest of the cross products of the rows of (M - lambda I), normalised
static P3 best_cross(const P3 rows[3], float lambda, float &len) {
    P3 a = rows[0], b = rows[1], c = rows[2];
    a.x -= lambda;
    b.y -= lambda;
    c.z -= lambda;
    const P3 v0 = pcross(a, b), v1 = pcross(a, c), v2 = pcross(b, c);
    const float l0 = pdot(v0, v0), l1 = pdot(v1, v1), l2 = pdot(v2, v2);
    if (l0 >= l1 && l0 >= l2) { len = l0; return pmul(v0, inv_sqrt(l0)); }
    if (l1 >= l0 && l1 >= l2) { len = l1; return pmul(v1, inv_sqrt(l1)); }
    len = l2;
    return pmul(v2, inv_sqrt(l2));
}
// eigen33::compute (eigen33.hpp:100-320), returning evecs[0]
static P3 min_eigenvector(float m[6]) {
    const float scale1 = std::max(std::max(std::max(fabsf(m[0]), fabsf(m[1])), std::max(fabsf(m[2]), fabsf(m[3]))),
                                  std::max(fabsf(m[4]), fabsf(m[5])));
    const float scale = scale1 <= kMinPos ? 1.f : scale1;
    for (int i = 0; i < 6; ++i) m[i] /= scale;
    const float a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5];   // [a b c; b d e; c e f]
    const float c0 = a * d * f + 2.f * b * c * e - a * e * e - d * c * c - f * b * b;
    const float c1 = a * d - b * b + a * f - c * c + d * f - e * e;
    const float c2 = a + d + f;
    P3 ev;
    root3(c0, c1, c2, ev);
    const P3 rows[3] = {p3(a, b, c), p3(b, d, e), p3(c, e, f)};
    float len;
    if (ev.z - ev.x <= kEps) return p3(1.f, 0.f, 0.f);
    if (ev.y - ev.x <= kEps) {
        const P3 e2 = best_cross(rows, ev.z, len);
        const P3 e1 = unit_orth(e2);
        return pcross(e1, e2);
    }
    if (ev.z - ev.y <= kEps) return best_cross(rows, ev.x, len);
    P3 vec[3];
    float mmax[3];
    vec[2] = best_cross(rows, ev.z, mmax[2]);
    int lo = 2, hi = 2;
    vec[1] = best_cross(rows, ev.y, mmax[1]);
    if (mmax[1] <= mmax[lo]) lo = 1;
    if (mmax[1] > mmax[hi]) hi = 1;
    vec[0] = best_cross(rows, ev.x, mmax[0]);
    {   // the reference tests the length of the third cross product here, whichever was longest
        P3 rb = rows[1], rc = rows[2];
        rb.y -= ev.x;
        rc.z -= ev.x;
        const P3 w = pcross(rb, rc);
        const float l3 = pdot(w, w);
        if (l3 <= mmax[lo]) lo = 0;
        if (l3 > mmax[hi]) hi = 0;
    }
    const int mid = 3 - lo - hi;
    P3 t = pcross(vec[(lo + 1) % 3], vec[(lo + 2) % 3]);
    vec[lo] = pmul(t, inv_sqrt(pdot(t, t)));
    t = pcross(vec[(mid + 1) % 3], vec[(mid + 2) % 3]);
    vec[mid] = pmul(t, inv_sqrt(pdot(t, t)));
    return vec[0];
}
}  // namespace meas

int orc_measure_maps(const uint16_t *depth_mm, int width, int height, float fx, float fy, float cx, float cy,
                     float clip_near, float clip_far, float radius_scale, float *vertex4, float *normal4) {
    using namespace meas;
    if (!depth_mm || !vertex4 || !normal4 || width <= 0 || height <= 0) return -1;
    const float ifx = 1.0f / fx, ify = 1.0f / fy;
    std::vector<P3> vert((size_t)width * height);
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            const size_t i = (size_t)y * width + x;
            const float z = float(depth_mm[i]) / (1000.f);
            const bool kept = !(z > clip_far || z < clip_near);
            vert[i] = kept ? p3((float(x) - cx) * ifx * z, (float(y) - cy) * ify * z, z) : p3(0.f, 0.f, 0.f);
            vertex4[4 * i] = vert[i].x;
            vertex4[4 * i + 1] = vert[i].y;
            vertex4[4 * i + 2] = vert[i].z;
            vertex4[4 * i + 3] = kept ? 1.f : 0.f;
        }
    auto at = [&](int x, int y) -> P3 {   // border texels read as zero
        if (x < 0 || y < 0 || x >= width || y >= height) return p3(0.f, 0.f, 0.f);
        return vert[(size_t)y * width + x];
    };
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            float *out = normal4 + 4 * ((size_t)y * width + x);
            out[0] = out[1] = out[2] = out[3] = 0.f;
            const P3 c = at(x, y);
            if (is_zero(c)) continue;
            P3 cen = p3(0.f, 0.f, 0.f);
            int count = 0;
            for (int cy2 = y - 3; cy2 <= y + 3; ++cy2)
                for (int cx2 = x - 3; cx2 <= x + 3; ++cx2) {
                    const P3 p = at(cx2, cy2);
                    if (!is_zero(p)) {
                        cen.x += p.x;
                        cen.y += p.y;
                        cen.z += p.z;
                        ++count;
                    }
                }
            if (count <= 24) continue;
            cen = pmul(cen, 1.0f / count);
            float cov[6] = {0, 0, 0, 0, 0, 0};
            for (int cy2 = y - 3; cy2 < y + 3; ++cy2)      // the reference's loops end one short
                for (int cx2 = x - 3; cx2 < x + 3; ++cx2) {
                    const P3 p = at(cx2, cy2);
                    if (!is_zero(p)) {
                        const P3 dd = p3(p.x - cen.x, p.y - cen.y, p.z - cen.z);
                        cov[0] += dd.x * dd.x;
                        cov[1] += dd.x * dd.y;
                        cov[2] += dd.x * dd.z;
                        cov[3] += dd.y * dd.y;
                        cov[4] += dd.y * dd.z;
                        cov[5] += dd.z * dd.z;
                    }
                }
            P3 n = min_eigenvector(cov);
            if (pdot(n, c) >= 0.0f) n = pmul(n, -1.f);
            const float radius = c.z * (1000 * 1.414f / 570.0f) * radius_scale;   // compute_radius, normal_map.cu:10-23
            const float nz = fabsf(n.z);
            out[0] = n.x;
            out[1] = n.y;
            out[2] = n.z;
            out[3] = nz > 0.5f ? radius / nz : 2.0f * radius;
        }
    return 0;
}

}  // extern "C"

// Renderer::DrawSolverMaps with shaders/solver_map.vert:21-53 and solver_map.frag:10-17
// (libs/star/geometry/render/RendererDraw.cu:105-175); the clear values of GLClearValues.h:21-34.
int orc_render_solver_maps(const float *vc4, const float *nr4, const float *ct4, int n, int W, int H, float fx,
                           float fy, float cx, float cy, const float *m, float max_depth, float current_time,
                           float conf_threshold, float time_threshold, int fp, uint32_t *index_map, float *vertex4,
                           float *normal4, float *rgbd4) {
    if (n < 0 || W <= 0 || H <= 0 || fp < 0) return -1;
    const size_t npix = (size_t)W * H;
    std::vector<float> best_z(npix, 0.f);
    std::vector<int64_t> best_id(npix, -1);
    std::vector<float> surfel_z((size_t)std::max(n, 1), 0.f);
    for (int i = 0; i < n; ++i) {
        const float *v = vc4 + 4ull * i;
        // vec4 world2camera * vec4(v.xyz, 1.0), one row at a time
        const float x = ((m[0] * v[0] + m[1] * v[1]) + m[2] * v[2]) + m[3];
        const float y = ((m[4] * v[0] + m[5] * v[1]) + m[6] * v[2]) + m[7];
        const float z = ((m[8] * v[0] + m[9] * v[1]) + m[10] * v[2]) + m[11];
        surfel_z[i] = z;
        if (!(z > 0.f) || !(z < max_depth)) continue;   // z > max depth or z <= 0; z = max depth fails the depth test
        const float t = ct4 ? ct4[4ull * i + 2] : current_time;
        if (v[3] < conf_threshold && std::fabs(t - current_time) >= time_threshold) continue;
        const float fpx = std::floor((fx * x) / z + cx + 0.5f);
        const float fpy = std::floor((fy * y) / z + cy + 0.5f);
        if (!(fpx >= (float)(-fp) && fpx < (float)(W + fp) && fpy >= (float)(-fp) && fpy < (float)(H + fp))) continue;
        const int px = (int)fpx, py = (int)fpy;
        for (int dy = -fp; dy <= fp; ++dy)
            for (int dx = -fp; dx <= fp; ++dx) {
                const int qx = px + dx, qy = py + dy;
                if (qx < 0 || qy < 0 || qx >= W || qy >= H) continue;
                const size_t q = (size_t)qy * W + qx;
                // depth test: nearer wins; at equal depth the surfel drawn first (lower id) stays
                if (best_id[q] < 0 || z < best_z[q]) { best_z[q] = z; best_id[q] = i; }
            }
    }
    for (size_t q = 0; q < npix; ++q) {
        float *vo = vertex4 ? vertex4 + 4 * q : nullptr;
        float *no = normal4 ? normal4 + 4 * q : nullptr;
        float *ro = rgbd4 ? rgbd4 + 4 * q : nullptr;
        if (best_id[q] < 0) {
            index_map[q] = 0xFFFFFFFFu;
            for (int c = 0; c < 4; ++c) {
                if (vo) vo[c] = 0.f;
                if (no) no[c] = 0.f;
                if (ro) ro[c] = 0.f;
            }
            continue;
        }
        const size_t id = (size_t)best_id[q];
        index_map[q] = (uint32_t)id;
        if (vo) { vo[0] = vc4[4 * id]; vo[1] = vc4[4 * id + 1]; vo[2] = vc4[4 * id + 2]; vo[3] = 1.f; }
        if (no) { no[0] = nr4[4 * id]; no[1] = nr4[4 * id + 1]; no[2] = nr4[4 * id + 2]; no[3] = 0.f; }
        if (ro) {
            int32_t enc = 0;
            if (ct4) std::memcpy(&enc, ct4 + 4 * id, 4);   // floatBitsToInt(color_time.x)
            ro[0] = (float)((enc & 0x00FF0000) >> 16) / 127.5f - 1.0f;
            ro[1] = (float)((enc & 0x0000FF00) >> 8) / 127.5f - 1.0f;
            ro[2] = (float)(enc & 0x000000FF) / 127.5f - 1.0f;
            ro[3] = 1.0f / surfel_z[id];
        }
    }
    return 0;
}

// Renderer::DrawObservationMaps (libs/star/geometry/render/RendererDraw.cu:353-394): every surfel
// drawn as a GL point with shaders/geometry.vert:40-86 and observation_map.frag:13-17, with
// GL_PROGRAM_POINT_SIZE on (Renderer.cu:87-90), so each surfel's point size comes from its disk.
// Restated per surfel, every operation rounded as written:
//   * v_cam = world2camera (v, 1) as in the solver-map pass; culled when z > max depth or z < 0
//     (geometry.vert:42-44) or unstable and not recent; z = 0 projects to infinity and z = max
//     depth fails the depth test against the far plane, so a surfel is drawn iff 0 < z < max depth;
//   * n_c = normalize(R n) with R the rotation rows of world2camera (mat3(world2camera)), where
//     normalize(a) = a / sqrt((a.x a.x + a.y a.y) + a.z a.z);
//   * x1 = ((normalize(n_c.y - n_c.z, -n_c.x, n_c.x) * radius) * 1.41421356) * 0.001, y1 = n_c x x1;
//     the four points v_cam + x1, v_cam + y1, v_cam - y1, v_cam - x1 in image coordinates
//     ((f p.x) / p.z + c); the point size is min(x extent, y extent), at least 0 (a non-finite
//     extent counts as 0), clamped to GL's aliased point-size range [1, 2047];
//   * window position u = (f x) / z + c plus the shader's 0.5 shift; a pixel is covered when its
//     centre lies in the point's square, taken half-open so that a unit point covers exactly the
//     solver-map pixel floor(u + 0.5): columns i with u - S/2 < i <= u + S/2, rows likewise;
//   * nearest z wins, equal z keeps the lower id (GL_LESS, drawn in id order);
//   * outputs: index (surfel id, clear 0xFFFFFFFF) and rgbd = ((colour byte / 255) * 2 - 1 for
//     r, g, b; 1 / z), clear zeros (GLClearValues.h:14-33).
static inline void obs_normalize(const float a[3], float out[3]) {
    const float len = std::sqrt((a[0] * a[0] + a[1] * a[1]) + a[2] * a[2]);
    out[0] = a[0] / len;
    out[1] = a[1] / len;
    out[2] = a[2] / len;
}

int orc_render_observation_maps(const float *vc4, const float *nr4, const float *ct4, int n, int W, int H, float fx,
                                float fy, float cx, float cy, const float *m, float max_depth, float current_time,
                                float conf_threshold, float time_threshold, uint32_t *index_map, float *rgbd4) {
    if (n < 0 || W <= 0 || H <= 0) return -1;
    const size_t npix = (size_t)W * H;
    std::vector<float> best_z(npix, 0.f);
    std::vector<int64_t> best_id(npix, -1);
    std::vector<float> surfel_z((size_t)std::max(n, 1), 0.f);
    for (int i = 0; i < n; ++i) {
        const float *v = vc4 + 4ull * i;
        const float x = ((m[0] * v[0] + m[1] * v[1]) + m[2] * v[2]) + m[3];
        const float y = ((m[4] * v[0] + m[5] * v[1]) + m[6] * v[2]) + m[7];
        const float z = ((m[8] * v[0] + m[9] * v[1]) + m[10] * v[2]) + m[11];
        surfel_z[i] = z;
        if (!(z > 0.f) || !(z < max_depth)) continue;
        const float t = ct4 ? ct4[4ull * i + 2] : current_time;
        if (v[3] < conf_threshold && std::fabs(t - current_time) >= time_threshold) continue;
        // the point size from the surfel's disk (geometry.vert:64-78)
        const float *nw = nr4 + 4ull * i;
        const float rn[3] = {(m[0] * nw[0] + m[1] * nw[1]) + m[2] * nw[2], (m[4] * nw[0] + m[5] * nw[1]) + m[6] * nw[2],
                             (m[8] * nw[0] + m[9] * nw[1]) + m[10] * nw[2]};
        float nc[3], dir[3];
        obs_normalize(rn, nc);
        const float d0[3] = {nc[1] - nc[2], -nc[0], nc[0]};
        obs_normalize(d0, dir);
        float x1[3], y1[3];
        for (int k = 0; k < 3; ++k) x1[k] = ((dir[k] * nw[3]) * 1.41421356f) * 0.001f;
        y1[0] = nc[1] * x1[2] - nc[2] * x1[1];
        y1[1] = nc[2] * x1[0] - nc[0] * x1[2];
        y1[2] = nc[0] * x1[1] - nc[1] * x1[0];
        const float vcam[3] = {x, y, z};
        float px[4], py[4];
        for (int k = 0; k < 4; ++k) {
            const float *off = (k == 0 || k == 3) ? x1 : y1;
            const float sgn = (k == 0 || k == 1) ? 1.f : -1.f;
            const float p0 = sgn > 0.f ? vcam[0] + off[0] : vcam[0] - off[0];
            const float p1 = sgn > 0.f ? vcam[1] + off[1] : vcam[1] - off[1];
            const float p2 = sgn > 0.f ? vcam[2] + off[2] : vcam[2] - off[2];
            px[k] = (fx * p0) / p2 + cx;
            py[k] = (fy * p1) / p2 + cy;
        }
        float xmin = px[0], xmax = px[0], ymin = py[0], ymax = py[0];
        for (int k = 1; k < 4; ++k) {
            xmin = std::min(xmin, px[k]);
            xmax = std::max(xmax, px[k]);
            ymin = std::min(ymin, py[k]);
            ymax = std::max(ymax, py[k]);
        }
        const float xd = std::fabs(xmax - xmin), yd = std::fabs(ymax - ymin);
        float size = xd < yd ? xd : yd;
        if (!(size > 0.f)) size = 0.f;   // a non-finite or negative extent
        size = std::min(std::max(size, 1.f), 2047.f);
        const float half = 0.5f * size;
        const float u = (fx * x) / z + cx, w = (fy * y) / z + cy;
        const float lo_x = std::floor(u - half) + 1.f, hi_x = std::floor(u + half);
        const float lo_y = std::floor(w - half) + 1.f, hi_y = std::floor(w + half);
        if (!(hi_x >= 0.f && lo_x <= (float)(W - 1) && hi_y >= 0.f && lo_y <= (float)(H - 1))) continue;
        const int x0 = (int)std::max(lo_x, 0.f), x1i = (int)std::min(hi_x, (float)(W - 1));
        const int y0 = (int)std::max(lo_y, 0.f), y1i = (int)std::min(hi_y, (float)(H - 1));
        for (int qy = y0; qy <= y1i; ++qy)
            for (int qx = x0; qx <= x1i; ++qx) {
                const size_t q = (size_t)qy * W + qx;
                if (best_id[q] < 0 || z < best_z[q]) { best_z[q] = z; best_id[q] = i; }
            }
    }
    for (size_t q = 0; q < npix; ++q) {
        float *ro = rgbd4 ? rgbd4 + 4 * q : nullptr;
        if (best_id[q] < 0) {
            index_map[q] = 0xFFFFFFFFu;
            if (ro) ro[0] = ro[1] = ro[2] = ro[3] = 0.f;
            continue;
        }
        const size_t id = (size_t)best_id[q];
        index_map[q] = (uint32_t)id;
        if (ro) {
            int32_t enc = 0;
            if (ct4) std::memcpy(&enc, ct4 + 4 * id, 4);   // floatBitsToInt(color_time.x)
            ro[0] = ((float)((enc & 0x00FF0000) >> 16) / 255.f) * 2.0f - 1.0f;
            ro[1] = ((float)((enc & 0x0000FF00) >> 8) / 255.f) * 2.0f - 1.0f;
            ro[2] = ((float)(enc & 0x000000FF) / 255.f) * 2.0f - 1.0f;
            ro[3] = 1.0f / surfel_z[id];
        }
    }
    return 0;
}
