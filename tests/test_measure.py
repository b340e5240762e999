"""Measurement maps from raw depth (vertex map, PCA normal/radius map; the reference's
img_proc/vertex_map.cu:13-33, img_proc/normal_map.cu:32-118 and math/eigen33.hpp).

CPU: the oracle's restatement against known answers (planes seen head-on and tilted,
holes, the depth clip, image borders).  GPU: ws_measure_maps against the oracle on a depth
image of a torus: the vertex map bit for bit (same operations in the same order), the set of
pixels with a normal exactly, normals within 1e-4 and radii within 1e-5 relative on at least
99.9% of them (the device contracts multiply-adds, uses rsqrtf and its own atan2f/cosf/sinf;
a pixel whose eigenvalues tie at the FP32 epsilon can take another branch), and nowhere
further than 2e-2.
"""
import numpy as np
import pytest

FX = FY = 50.0
W, H = 64, 48
CX, CY = (W - 1) / 2, (H - 1) / 2


def plane_depth(n, d, w=W, h=H):
    """Depth in mm of the plane n . X = d seen by the pinhole camera."""
    xs, ys = np.meshgrid(np.arange(w, dtype=np.float64), np.arange(h, dtype=np.float64))
    rays = np.stack([(xs - CX) / FX, (ys - CY) / FY, np.ones_like(xs)], -1)
    z = d / (rays @ np.asarray(n, np.float64))
    return np.round(z * 1000).astype(np.uint16)


def test_vertex_map_back_projects(orc):
    depth = plane_depth([0, 0, 1], 1.0)
    vert, _ = orc.measure_maps(depth, FX, FY, CX, CY)
    y, x = 10, 20
    z = np.float32(depth[y, x]) / np.float32(1000)
    assert vert[y, x, 2] == z and vert[y, x, 3] == 1
    assert vert[y, x, 0] == (np.float32(x) - np.float32(CX)) * (np.float32(1) / np.float32(FX)) * z


def test_plane_seen_head_on(orc):
    depth = plane_depth([0, 0, 1], 1.0)
    _, nrm = orc.measure_maps(depth, FX, FY, CX, CY, radius_scale=1.5)
    inner = nrm[3:-3, 3:-3]
    np.testing.assert_allclose(inner[..., :3], np.broadcast_to([0, 0, -1], inner[..., :3].shape), atol=1e-5)
    np.testing.assert_allclose(inner[..., 3], 1.0 * (1000 * 1.414 / 570.0) * 1.5, rtol=1e-5)
    # a corner pixel sees 16 of 49 window texels: no normal; an edge pixel sees 28: a normal
    assert not nrm[0, 0].any()
    assert nrm[H // 2, 0, 2] < -0.99


def test_tilted_plane_normal_faces_the_camera(orc):
    n = np.array([0.3, -0.2, 1.0])
    n /= np.linalg.norm(n)
    depth = plane_depth(n, 1.0)
    _, nrm = orc.measure_maps(depth, FX, FY, CX, CY)
    inner = nrm[4:-4, 4:-4, :3].reshape(-1, 3)
    # the normal faces the camera (negative z); millimetre depth steps tilt it by about 1e-2
    assert np.abs(inner + n).max() < 2e-2


def test_holes_and_clip(orc):
    depth = plane_depth([0, 0, 1], 1.0)
    depth[10:30, 10:30] = 0          # a hole
    depth[0:5, 40:60] = 4000         # beyond the far clip
    vert, nrm = orc.measure_maps(depth, FX, FY, CX, CY, clip_near=0.1, clip_far=3.0)
    assert not vert[20, 20].any() and not vert[2, 50].any()
    assert not nrm[20, 20].any()     # inside the hole
    assert nrm[20, 7, 2] < -0.99     # beside it: more than half of the window still valid


@pytest.mark.gpu
def test_gpu_measure_maps_match_the_oracle(ws, orc, small_scene):
    from starhub_b200.solver import GpuGeometry
    cam = small_scene.camera
    z = small_scene.meas_vertex[..., 2].astype(np.float64)
    depth = np.round(np.clip(z, 0, 60) * 1000).astype(np.uint16)
    geo = GpuGeometry()
    for _ in range(2):   # twice: the second call must not depend on the first
        vert, nrm = geo.measure_maps(depth, cam, clip_near=0.3, clip_far=2.5, radius_scale=1.0)
    over, onrm = orc.measure_maps(depth, cam.fx, cam.fy, cam.cx, cam.cy, clip_near=0.3, clip_far=2.5)
    np.testing.assert_array_equal(vert, over)
    has = onrm[..., 3] != 0
    np.testing.assert_array_equal(nrm[..., 3] != 0, has)
    assert has.sum() > 1000
    dn = np.abs(nrm[has, :3] - onrm[has, :3]).max(axis=1)
    dr = np.abs(nrm[has, 3] - onrm[has, 3]) / onrm[has, 3]
    within = (dn <= 1e-4) & (dr <= 1e-5)
    assert np.mean(within) >= 0.999, (np.mean(within), np.percentile(dn, [50, 99, 99.9]), dr.max())
    assert dn.max() <= 2e-2, dn.max()
