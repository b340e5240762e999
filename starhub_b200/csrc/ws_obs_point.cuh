// One surfel of the observation-map pass: whether it is drawn, its camera-frame depth and the
// pixel rectangle its GL point covers.  Renderer::DrawObservationMaps
// (libs/star/geometry/render/RendererDraw.cu:353-394) draws every surfel as a point with
// shaders/geometry.vert:40-86, GL_PROGRAM_POINT_SIZE on (Renderer.cu:87-90), so the point's
// size is the smaller image extent of the surfel's disk:
//   * v_cam = world2camera (v, 1), one row at a time ((m0 x + m1 y) + m2 z) + m3; drawn iff
//     0 < z < max depth (geometry.vert:42-44 culls z > max depth and z < 0; z = 0 projects to
//     infinity and z = max depth fails the depth test against the far plane) and not (confidence
//     < conf_threshold and |time - current_time| >= time_threshold);
//   * n_c = normalize(R n), R the rotation rows of world2camera, normalize(a) = a / sqrt((a.x a.x
//     + a.y a.y) + a.z a.z); x1 = ((normalize(n_c.y - n_c.z, -n_c.x, n_c.x) * radius) *
//     1.41421356) * 0.001 (radius in mm); y1 = n_c x x1;
//   * the image points (f p.x) / p.z + c of v_cam + x1, v_cam + y1, v_cam - y1, v_cam - x1; the
//     size is min(x extent, y extent), 0 when that is not positive or not finite, clamped to
//     GL's aliased point-size range [1, 2047];
//   * the point covers the pixels whose centres lie in its square, taken half-open so that a unit
//     point covers exactly the solver-map pixel floor(u + 0.5): columns i with
//     u - S/2 < i <= u + S/2 around u = (f x) / z + c, rows likewise; the rectangle is clipped to
//     the image.
// Every operation is rounded as written: on the device through the round-to-nearest intrinsics
// (no contraction into FMAs), on the host through plain operators (built without contraction).
// The same source is compiled for both, which lets the host build be compared with the
// oracle's independent restatement on the CPU.
#pragma once
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define WS_OBS_FN __host__ __device__ __forceinline__
#else
#define WS_OBS_FN inline
#endif

#if defined(__CUDA_ARCH__)
#define WS_OBS_ADD(a, b) __fadd_rn((a), (b))
#define WS_OBS_SUB(a, b) __fsub_rn((a), (b))
#define WS_OBS_MUL(a, b) __fmul_rn((a), (b))
#define WS_OBS_DIV(a, b) __fdiv_rn((a), (b))
#define WS_OBS_SQRT(a) __fsqrt_rn(a)
#else
#define WS_OBS_ADD(a, b) ((a) + (b))
#define WS_OBS_SUB(a, b) ((a) - (b))
#define WS_OBS_MUL(a, b) ((a) * (b))
#define WS_OBS_DIV(a, b) ((a) / (b))
#define WS_OBS_SQRT(a) sqrtf(a)
#endif

namespace ws {

struct ObsCover {
    int drawn;            // 0: culled or off the image
    float z;              // camera-frame depth
    int x0, x1, y0, y1;   // covered pixels, inclusive, inside the image
};

WS_OBS_FN void obs_normalize(const float a[3], float out[3]) {
    const float len = WS_OBS_SQRT(WS_OBS_ADD(WS_OBS_ADD(WS_OBS_MUL(a[0], a[0]), WS_OBS_MUL(a[1], a[1])),
                                             WS_OBS_MUL(a[2], a[2])));
    out[0] = WS_OBS_DIV(a[0], len);
    out[1] = WS_OBS_DIV(a[1], len);
    out[2] = WS_OBS_DIV(a[2], len);
}

WS_OBS_FN float obs_row(const float *m, float x, float y, float z) {
    return WS_OBS_ADD(WS_OBS_ADD(WS_OBS_MUL(m[0], x), WS_OBS_MUL(m[1], y)), WS_OBS_MUL(m[2], z));
}

// v: (x, y, z, confidence); nw: (normal, radius in mm); t: last observed time; m: world2camera
// rows 0..2, row-major (12 floats).
WS_OBS_FN ObsCover obs_point(const float v[4], const float nw[4], float t, const float *m, float fx, float fy,
                             float cx, float cy, int W, int H, float max_depth, float current_time,
                             float conf_threshold, float time_threshold) {
    ObsCover c;
    c.drawn = 0;
    c.x0 = c.x1 = c.y0 = c.y1 = 0;
    const float x = WS_OBS_ADD(obs_row(m, v[0], v[1], v[2]), m[3]);
    const float y = WS_OBS_ADD(obs_row(m + 4, v[0], v[1], v[2]), m[7]);
    const float z = WS_OBS_ADD(obs_row(m + 8, v[0], v[1], v[2]), m[11]);
    c.z = z;
    if (!(z > 0.f) || !(z < max_depth)) return c;
    if (v[3] < conf_threshold && fabsf(WS_OBS_SUB(t, current_time)) >= time_threshold) return c;
    // the disk's image extent (geometry.vert:64-78)
    const float rn[3] = {obs_row(m, nw[0], nw[1], nw[2]), obs_row(m + 4, nw[0], nw[1], nw[2]),
                         obs_row(m + 8, nw[0], nw[1], nw[2])};
    float nc[3], dir[3];
    obs_normalize(rn, nc);
    const float d0[3] = {WS_OBS_SUB(nc[1], nc[2]), -nc[0], nc[0]};
    obs_normalize(d0, dir);
    float x1[3], y1[3];
    for (int k = 0; k < 3; ++k) x1[k] = WS_OBS_MUL(WS_OBS_MUL(WS_OBS_MUL(dir[k], nw[3]), 1.41421356f), 0.001f);
    y1[0] = WS_OBS_SUB(WS_OBS_MUL(nc[1], x1[2]), WS_OBS_MUL(nc[2], x1[1]));
    y1[1] = WS_OBS_SUB(WS_OBS_MUL(nc[2], x1[0]), WS_OBS_MUL(nc[0], x1[2]));
    y1[2] = WS_OBS_SUB(WS_OBS_MUL(nc[0], x1[1]), WS_OBS_MUL(nc[1], x1[0]));
    const float vcam[3] = {x, y, z};
    float xmin = 0.f, xmax = 0.f, ymin = 0.f, ymax = 0.f;
    for (int k = 0; k < 4; ++k) {
        const float *off = (k == 0 || k == 3) ? x1 : y1;
        const bool plus = k < 2;
        const float p0 = plus ? WS_OBS_ADD(vcam[0], off[0]) : WS_OBS_SUB(vcam[0], off[0]);
        const float p1 = plus ? WS_OBS_ADD(vcam[1], off[1]) : WS_OBS_SUB(vcam[1], off[1]);
        const float p2 = plus ? WS_OBS_ADD(vcam[2], off[2]) : WS_OBS_SUB(vcam[2], off[2]);
        const float px = WS_OBS_ADD(WS_OBS_DIV(WS_OBS_MUL(fx, p0), p2), cx);
        const float py = WS_OBS_ADD(WS_OBS_DIV(WS_OBS_MUL(fy, p1), p2), cy);
        if (k == 0) {
            xmin = xmax = px;
            ymin = ymax = py;
        } else {   // the comparisons of std::min / std::max, in that argument order
            xmin = (px < xmin) ? px : xmin;
            xmax = (xmax < px) ? px : xmax;
            ymin = (py < ymin) ? py : ymin;
            ymax = (ymax < py) ? py : ymax;
        }
    }
    const float xd = fabsf(WS_OBS_SUB(xmax, xmin)), yd = fabsf(WS_OBS_SUB(ymax, ymin));
    float size = xd < yd ? xd : yd;
    if (!(size > 0.f)) size = 0.f;
    size = (size < 1.f) ? 1.f : size;
    size = (2047.f < size) ? 2047.f : size;
    const float half = WS_OBS_MUL(0.5f, size);
    const float u = WS_OBS_ADD(WS_OBS_DIV(WS_OBS_MUL(fx, x), z), cx);
    const float w = WS_OBS_ADD(WS_OBS_DIV(WS_OBS_MUL(fy, y), z), cy);
    const float lo_x = WS_OBS_ADD(floorf(WS_OBS_SUB(u, half)), 1.f), hi_x = floorf(WS_OBS_ADD(u, half));
    const float lo_y = WS_OBS_ADD(floorf(WS_OBS_SUB(w, half)), 1.f), hi_y = floorf(WS_OBS_ADD(w, half));
    if (!(hi_x >= 0.f && lo_x <= (float)(W - 1) && hi_y >= 0.f && lo_y <= (float)(H - 1))) return c;
    c.x0 = (int)((lo_x < 0.f) ? 0.f : lo_x);
    c.x1 = (int)(((float)(W - 1) < hi_x) ? (float)(W - 1) : hi_x);
    c.y0 = (int)((lo_y < 0.f) ? 0.f : lo_y);
    c.y1 = (int)(((float)(H - 1) < hi_y) ? (float)(H - 1) : hi_y);
    c.drawn = 1;
    return c;
}

// The observation rgbd texel of a surfel (geometry.vert:56-60,83 and observation_map.frag:15): the
// colour bytes of color_time.x (as int bits) as (byte / 255) * 2 - 1, and 1 / z.
WS_OBS_FN void obs_rgbd(int32_t enc, float z, float out[4]) {
    out[0] = WS_OBS_SUB(WS_OBS_MUL(WS_OBS_DIV((float)((enc & 0x00FF0000) >> 16), 255.f), 2.f), 1.f);
    out[1] = WS_OBS_SUB(WS_OBS_MUL(WS_OBS_DIV((float)((enc & 0x0000FF00) >> 8), 255.f), 2.f), 1.f);
    out[2] = WS_OBS_SUB(WS_OBS_MUL(WS_OBS_DIV((float)(enc & 0x000000FF), 255.f), 2.f), 1.f);
    out[3] = WS_OBS_DIV(1.f, z);
}

}  // namespace ws
