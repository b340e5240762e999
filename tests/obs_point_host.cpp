// Host build of the observation-map pass for the CPU check in tests/test_observation_maps.py:
// the per-surfel arithmetic of the library's kernel (starhub_b200/csrc/ws_obs_point.cuh, the same
// source the device kernel compiles), with the kernel's depth rule (the smallest (z bits, surfel
// id) key wins a pixel) run serially.  Built with g++ -ffp-contract=off, so every operation rounds
// as the device intrinsics do.
#include <cstring>
#include <vector>

#include "ws_obs_point.cuh"

extern "C" int obs_maps_host(const float *vc4, const float *nr4, const float *ct4, int n, int W, int H, float fx,
                             float fy, float cx, float cy, const float *m12, float max_depth, float current_time,
                             float conf_threshold, float time_threshold, uint32_t *index, float *rgbd4) {
    if (n < 0 || W <= 0 || H <= 0) return -1;
    const size_t npix = (size_t)W * H;
    std::vector<unsigned long long> keys(npix, ~0ull);
    for (int i = 0; i < n; ++i) {
        const float t = ct4 ? ct4[4ull * i + 2] : current_time;
        const ws::ObsCover c = ws::obs_point(vc4 + 4ull * i, nr4 + 4ull * i, t, m12, fx, fy, cx, cy, W, H, max_depth,
                                             current_time, conf_threshold, time_threshold);
        if (!c.drawn) continue;
        uint32_t zbits;
        std::memcpy(&zbits, &c.z, 4);
        const unsigned long long key = ((unsigned long long)zbits << 32) | (unsigned)i;
        for (int qy = c.y0; qy <= c.y1; ++qy)
            for (int qx = c.x0; qx <= c.x1; ++qx) {
                unsigned long long &k = keys[(size_t)qy * W + qx];
                if (key < k) k = key;
            }
    }
    for (size_t p = 0; p < npix; ++p) {
        float *o = rgbd4 + 4 * p;
        if (keys[p] == ~0ull) {
            index[p] = 0xFFFFFFFFu;
            o[0] = o[1] = o[2] = o[3] = 0.f;
            continue;
        }
        const uint32_t id = (uint32_t)(keys[p] & 0xffffffffu);
        const uint32_t zbits = (uint32_t)(keys[p] >> 32);
        float z;
        std::memcpy(&z, &zbits, 4);
        int32_t enc = 0;
        if (ct4) std::memcpy(&enc, ct4 + 4ull * id, 4);
        index[p] = id;
        ws::obs_rgbd(enc, z, o);
    }
    return 0;
}
