// Measurement maps from a raw depth image: the vertex map and the normal/radius map that the
// solver reads as its measurement (Measure4Solver).  Restates, in one tiled kernel:
//   * createVertexConfidMapKernel (libs/star/img_proc/vertex_map.cu:13-33): back-projection of
//     a depth image in millimetres with the inverse intrinsics, confidence 1;
//   * the clip of filterAndScaleVertexKernel (libs/star/geometry/geometry_map/
//     SurfelMapInitializer.cu:107-137): pixels whose depth lies outside [clip_near, clip_far]
//     become zero vertices (here on the depth in metres, at the full resolution);
//   * createNormalRadiusMapKernel (libs/star/img_proc/normal_map.cu:32-118): the centroid of the
//     non-zero vertices of the 7x7 window, used when more than half of it is valid; their
//     covariance over the window's first 6 rows and columns (the reference's loops stop one short
//     on the high side); the eigenvector of the smallest eigenvalue, turned towards the camera;
//     the surfel radius from the depth and the normal's z;
//   * the closed-form 3x3 symmetric eigen-decomposition of libs/star/math/eigen33.hpp
//     (characteristic cubic solved in trigonometric form, eigenvectors from cross products of
//     the rows of A - lambda I), with the reference's branch order and its tie handling.
// Pixels outside the image read as zero vertices, as the reference's border-mode textures do.
// The eigen solver's branches compare quantities with the FP32 epsilon, so the file is built
// without multiply-add contraction and takes inverse square roots as 1 / sqrtf: the arithmetic
// of the reference's host path (eigen33.h, vector_ops.hpp), which the CPU checker restates.
// (The reference's device build contracts and uses rsqrtf; on windows whose eigenvalues nearly
// tie, that moves the normal by up to a few 1e-2.)
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/warpsolve.h"

namespace ws {
namespace {

constexpr int kTileW = 32, kTileH = 8;   // one thread per output pixel
constexpr int kHalo = 3;                 // half of the 7x7 window
constexpr int kSharedW = kTileW + 2 * kHalo, kSharedH = kTileH + 2 * kHalo;
constexpr float kFltEpsilon = 1.192092896e-07f;
constexpr float kFltMinPositive = 1.175494351e-38f;

__device__ __forceinline__ float3 v3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 scaled(float3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float inv_sqrt(float v) { return 1.0f / sqrtf(v); }
__device__ __forceinline__ float3 unit(float3 a) { return scaled(a, inv_sqrt(dot(a, a))); }
__device__ __forceinline__ bool zero_vertex(float3 p) {   // vector_ops.hpp:123-126
    return fabsf(p.x) < 1e-3f && fabsf(p.y) < 1e-3f && fabsf(p.z) < 1e-3f;
}
__device__ __forceinline__ bool much_smaller(float x, float y) {
    return x * x <= kFltEpsilon * kFltEpsilon * y * y;
}

// Roots of x^2 - b x + c = 0 as (0, smaller, larger); a negative discriminant counts as 0.
__device__ void quadratic_roots(float b, float c, float3 &r) {
    r.x = 0.f;
    float d = b * b - 4.f * c;
    if (d < 0.f) d = 0.f;
    const float sd = sqrtf(d);
    r.z = 0.5f * (b + sd);
    r.y = 0.5f * (b - sd);
}

// Roots of x^3 - c2 x^2 + c1 x - c0 = 0 in ascending order (all real for a symmetric matrix).
__device__ void cubic_roots(float c0, float c1, float c2, float3 &r) {
    if (fabsf(c0) < kFltEpsilon) {   // a zero eigenvalue: the quadratic factor holds the others
        quadratic_roots(c2, c1, r);
        return;
    }
    const float third = 1.f / 3.f;
    const float root3 = sqrtf(3.f);
    const float c2_3 = c2 * third;
    float a_3 = (c1 - c2 * c2_3) * third;
    if (a_3 > 0.f) a_3 = 0.f;
    const float half_b = 0.5f * (c0 + c2_3 * (2.f * c2_3 * c2_3 - c1));
    float q = half_b * half_b + a_3 * a_3 * a_3;
    if (q > 0.f) q = 0.f;
    const float rho = sqrtf(-a_3);
    const float theta = atan2f(sqrtf(-q), half_b) * third;
    const float ct = cosf(theta), st = sinf(theta);
    r.x = c2_3 + 2.f * rho * ct;
    r.y = c2_3 - rho * (ct + root3 * st);
    r.z = c2_3 - rho * (ct - root3 * st);
    float t;
    if (r.x >= r.y) { t = r.x; r.x = r.y; r.y = t; }
    if (r.y >= r.z) {
        t = r.y; r.y = r.z; r.z = t;
        if (r.x >= r.y) { t = r.x; r.x = r.y; r.y = t; }
    }
    if (r.x <= 0.f) quadratic_roots(c2, c1, r);   // clamp a rounding-negative smallest root
}

// A unit vector orthogonal to v.
__device__ float3 orthogonal_unit(float3 v) {
    if (!much_smaller(v.x, v.z) || !much_smaller(v.y, v.z)) {
        const float inv = inv_sqrt(v.x * v.x + v.y * v.y);
        return v3(-v.y * inv, v.x * inv, 0.f);
    }
    const float inv = inv_sqrt(v.z * v.z + v.y * v.y);
    return v3(0.f, -v.z * inv, v.y * inv);
}

// Of the three cross products of the rows of M - lambda I, the longest one, normalised; its
// squared length in len.
__device__ float3 null_direction(const float3 row[3], float lambda, float &len) {
    float3 t0 = row[0], t1 = row[1], t2 = row[2];
    t0.x -= lambda;
    t1.y -= lambda;
    t2.z -= lambda;
    const float3 a = cross(t0, t1), b = cross(t0, t2), c = cross(t1, t2);
    const float la = dot(a, a), lb = dot(b, b), lc = dot(c, c);
    if (la >= lb && la >= lc) {
        len = la;
        return scaled(a, inv_sqrt(la));
    }
    if (lb >= la && lb >= lc) {
        len = lb;
        return scaled(b, inv_sqrt(lb));
    }
    len = lc;
    return scaled(c, inv_sqrt(lc));
}

// Eigenvector of the smallest eigenvalue of the symmetric matrix
// m = [m0 m1 m2; m1 m3 m4; m2 m4 m5] (modified: scaled into [-1, 1]).
__device__ float3 smallest_eigenvector(float m[6]) {
    const float scale0 = fmaxf(fmaxf(fmaxf(fabsf(m[0]), fabsf(m[1])), fmaxf(fabsf(m[2]), fabsf(m[3]))),
                               fmaxf(fabsf(m[4]), fabsf(m[5])));
    const float scale = scale0 <= kFltMinPositive ? 1.f : scale0;
#pragma unroll
    for (int i = 0; i < 6; ++i) m[i] /= scale;
    const float m00 = m[0], m01 = m[1], m02 = m[2], m11 = m[3], m12 = m[4], m22 = m[5];
    const float c0 = m00 * m11 * m22 + 2.f * m01 * m02 * m12 - m00 * m12 * m12 - m11 * m02 * m02 - m22 * m01 * m01;
    const float c1 = m00 * m11 - m01 * m01 + m00 * m22 - m02 * m02 + m11 * m22 - m12 * m12;
    const float c2 = m00 + m11 + m22;
    float3 ev;
    cubic_roots(c0, c1, c2, ev);
    const float3 row[3] = {v3(m00, m01, m02), v3(m01, m11, m12), v3(m02, m12, m22)};
    float len;
    if (ev.z - ev.x <= kFltEpsilon) return v3(1.f, 0.f, 0.f);   // a multiple of I
    if (ev.y - ev.x <= kFltEpsilon) {
        // the two smallest coincide: any unit vector orthogonal to the largest one's
        const float3 e2 = null_direction(row, ev.z, len);
        const float3 e1 = orthogonal_unit(e2);
        return cross(e1, e2);
    }
    if (ev.z - ev.y <= kFltEpsilon) return null_direction(row, ev.x, len);   // the two largest coincide
    // distinct eigenvalues: the directions for the largest, middle and smallest; the least
    // reliable two (shortest cross products) are rebuilt as cross products of the others
    float3 e[3];
    float lens[3];
    e[2] = null_direction(row, ev.z, lens[2]);
    int min_el = 2, max_el = 2;
    e[1] = null_direction(row, ev.y, lens[1]);
    if (lens[1] <= lens[min_el]) min_el = 1;
    if (lens[1] > lens[max_el]) max_el = 1;
    e[0] = null_direction(row, ev.x, lens[0]);
    // the reference compares the third candidate's length here whichever candidate won
    const float3 r1 = v3(row[1].x, row[1].y - ev.x, row[1].z), r2 = v3(row[2].x, row[2].y, row[2].z - ev.x);
    const float3 c = cross(r1, r2);
    const float len3 = dot(c, c);
    if (len3 <= lens[min_el]) min_el = 0;
    if (len3 > lens[max_el]) max_el = 0;
    const int mid_el = 3 - min_el - max_el;
    e[min_el] = unit(cross(e[(min_el + 1) % 3], e[(min_el + 2) % 3]));
    e[mid_el] = unit(cross(e[(mid_el + 1) % 3], e[(mid_el + 2) % 3]));
    return e[0];
}

// compute_radius (normal_map.cu:10-23): the surfel radius in millimetres.
__device__ __forceinline__ float surfel_radius(float depth_m, float normal_z, float radius_scale) {
    const float radius = depth_m * (1000 * 1.414f / 570.0f) * radius_scale;
    const float nz = fabsf(normal_z);
    return nz > 0.5f ? radius / nz : 2.0f * radius;
}

__global__ void __launch_bounds__(kTileW * kTileH) k_measure_maps(const uint16_t *depth, int width, int height,
                                                                  int pitch, float cx, float cy, float inv_fx,
                                                                  float inv_fy, float clip_near, float clip_far,
                                                                  float radius_scale, float4 *vertex_out,
                                                                  float4 *normal_out) {
    __shared__ float3 tile[kSharedH][kSharedW];
    const int x0 = blockIdx.x * kTileW - kHalo, y0 = blockIdx.y * kTileH - kHalo;
    for (int i = threadIdx.y * kTileW + threadIdx.x; i < kSharedW * kSharedH; i += kTileW * kTileH) {
        const int sy = i / kSharedW, sx = i - sy * kSharedW;
        const int gx = x0 + sx, gy = y0 + sy;
        float3 p = v3(0.f, 0.f, 0.f);
        if (gx >= 0 && gy >= 0 && gx < width && gy < height) {
            const float z = float(depth[(size_t)gy * pitch + gx]) / (1000.f);
            if (!(z > clip_far || z < clip_near)) p = v3((gx - cx) * inv_fx * z, (gy - cy) * inv_fy * z, z);
        }
        tile[sy][sx] = p;
    }
    __syncthreads();
    const int x = blockIdx.x * kTileW + threadIdx.x, y = blockIdx.y * kTileH + threadIdx.y;
    if (x >= width || y >= height) return;
    const int tx = threadIdx.x + kHalo, ty = threadIdx.y + kHalo;
    const float3 c = tile[ty][tx];
    float4 normal_radius = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!zero_vertex(c)) {
        float3 centroid = v3(0.f, 0.f, 0.f);
        int count = 0;
        for (int dy = -kHalo; dy <= kHalo; ++dy)
            for (int dx = -kHalo; dx <= kHalo; ++dx) {
                const float3 p = tile[ty + dy][tx + dx];
                if (!zero_vertex(p)) {
                    centroid.x += p.x;
                    centroid.y += p.y;
                    centroid.z += p.z;
                    ++count;
                }
            }
        if (count > (7 * 7) / 2) {
            centroid = scaled(centroid, 1.0f / count);
            float cov[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            for (int dy = -kHalo; dy < kHalo; ++dy)
                for (int dx = -kHalo; dx < kHalo; ++dx) {
                    const float3 p = tile[ty + dy][tx + dx];
                    if (!zero_vertex(p)) {
                        const float3 d = v3(p.x - centroid.x, p.y - centroid.y, p.z - centroid.z);
                        cov[0] += d.x * d.x;
                        cov[1] += d.x * d.y;
                        cov[2] += d.x * d.z;
                        cov[3] += d.y * d.y;
                        cov[4] += d.y * d.z;
                        cov[5] += d.z * d.z;
                    }
                }
            float3 n = smallest_eigenvector(cov);
            if (dot(n, c) >= 0.0f) n = scaled(n, -1.f);   // face the camera
            normal_radius = make_float4(n.x, n.y, n.z, surfel_radius(c.z, n.z, radius_scale));
        }
    }
    // the vertex map keeps confidence 1 for every pixel that passes the clip, zero depth included
    const float z = float(depth[(size_t)y * pitch + x]) / (1000.f);
    const bool kept = !(z > clip_far || z < clip_near);
    const size_t o = (size_t)y * width + x;
    vertex_out[o] = kept ? make_float4(c.x, c.y, c.z, 1.f) : make_float4(0.f, 0.f, 0.f, 0.f);
    normal_out[o] = normal_radius;
}

}  // namespace
}  // namespace ws

extern "C" int ws_measure_maps(const uint16_t *depth_mm, int width, int height, int pitch, float fx, float fy,
                               float cx, float cy, float clip_near, float clip_far, float radius_scale,
                               float *vertex_confid, float *normal_radius, void *stream) {
    if (!depth_mm || !vertex_confid || !normal_radius || width <= 0 || height <= 0 || pitch < width || !(fx > 0.f) ||
        !(fy > 0.f))
        return WS_ERR_INVALID_ARGUMENT;
    const dim3 block(ws::kTileW, ws::kTileH);
    const dim3 grid((width + ws::kTileW - 1) / ws::kTileW, (height + ws::kTileH - 1) / ws::kTileH);
    ws::k_measure_maps<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
        depth_mm, width, height, pitch, cx, cy, 1.0f / fx, 1.0f / fy, clip_near, clip_far, radius_scale,
        reinterpret_cast<float4 *>(vertex_confid), reinterpret_cast<float4 *>(normal_radius));
    return cudaGetLastError() == cudaSuccess ? WS_OK : WS_ERR_CUDA;
}
