"""The observation-map pass (Renderer::DrawObservationMaps, RendererDraw.cu:353-394, with
shaders/geometry.vert:40-86 and observation_map.frag:13-17): per-surfel point sizes from the
projected disk, index and rgbd maps.

The CPU test builds the per-surfel arithmetic of the library's kernel (the header
starhub_b200/csrc/ws_obs_point.cuh, which the device kernel compiles too) for the host and
compares it, bit for bit, with the oracle's independent restatement; the GPU test compares
ws_render_observation_maps itself with the oracle."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _inputs(kind, small_scene):
    """(vertex_confid, normal_radius (radius in mm), color_time, camera, world2camera, max_depth,
    current_time, conf_threshold, time_threshold)."""
    from starhub_b200.scenes import Camera, rot_x
    rng = np.random.default_rng(7)
    if kind == "torus":
        sc = small_scene
        n = sc.surfel_vertex.shape[0]
        vc = sc.surfel_vertex.copy()
        vc[:, 3] = rng.uniform(0.0, 3.0, n).astype(np.float32)
        nr = sc.surfel_normal.copy()
        nr[:, 3] = rng.uniform(0.5, 9.0, n).astype(np.float32)   # disk radius in mm
        cam = sc.camera
        w2c = np.eye(4, dtype=np.float32)
        w2c[:3, :3] = rot_x(4.0).astype(np.float32)
        w2c[:3, 3] = [0.01, -0.02, 0.03]
        max_depth = 1.02
    else:
        # a random cloud: surfels in front of, behind and beyond the camera's range, normals of
        # every direction (some whose disk axis is degenerate), radii up to several cm
        n = 4000
        cam = Camera(96, 72, 80.0, 80.0, 47.5, 35.5)
        xyz = np.stack([rng.uniform(-0.6, 0.6, n), rng.uniform(-0.45, 0.45, n), rng.uniform(0.25, 1.95, n)], 1)
        xyz[::50, 2] = -0.3    # behind the camera
        xyz[7::53, 2] = 2.5    # beyond the maximum depth
        vc = np.concatenate([xyz, rng.uniform(0.0, 3.0, (n, 1))], 1).astype(np.float32)
        nrm = rng.normal(size=(n, 3))
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        nrm[::37] = [0.0, np.sqrt(0.5), np.sqrt(0.5)]   # (n.y - n.z, -n.x, n.x) = 0: no disk axis
        rad = rng.uniform(0.2, 40.0, (n, 1))
        nr = np.concatenate([nrm, rad], 1).astype(np.float32)
        w2c = np.eye(4, dtype=np.float32)
        max_depth = 2.0
    ct = np.zeros((n, 4), np.float32)
    ct[:, 0] = rng.integers(0, 1 << 24, n).astype(np.uint32).view(np.float32)
    ct[:, 2] = rng.integers(0, 12, n).astype(np.float32)
    return vc, nr, ct, cam, w2c, max_depth, 10.0, 1.0, 3.0


def _host_build(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ not found")
    so = tmp_path / "libobs_host.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared",
                    "-I", str(ROOT / "starhub_b200" / "csrc"), str(ROOT / "tests" / "obs_point_host.cpp"),
                    "-o", str(so)], check=True)
    return C.CDLL(str(so))


def _run_host(lib, vc, nr, ct, cam, w2c, max_depth, now, conf, tthr):
    h, w = cam.height, cam.width
    idx = np.zeros((h, w), np.uint32)
    rgbd = np.zeros((h, w, 4), np.float32)
    m = np.ascontiguousarray(np.asarray(w2c, np.float32).reshape(16))
    p = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    rc = lib.obs_maps_host(p(vc), p(nr), p(ct), C.c_int(len(vc)), C.c_int(w), C.c_int(h), C.c_float(cam.fx),
                           C.c_float(cam.fy), C.c_float(cam.cx), C.c_float(cam.cy), p(m), C.c_float(max_depth),
                           C.c_float(now), C.c_float(conf), C.c_float(tthr), p(idx), p(rgbd))
    assert rc == 0
    return idx, rgbd


@pytest.mark.parametrize("kind", ["torus", "cloud"])
def test_kernel_arithmetic_matches_the_oracle_on_the_host(orc, small_scene, tmp_path, kind):
    """The kernel's per-surfel arithmetic, built for the host, equals the oracle's restatement of
    the shader bit for bit (index and rgbd maps), with and without the recent-observation pass and
    without colour and time."""
    lib = _host_build(tmp_path)
    args = _inputs(kind, small_scene)
    for tthr in (3.0, -1.0):
        a = args[:-1] + (tthr,)
        hi, hr = _run_host(lib, *[np.ascontiguousarray(x) if isinstance(x, np.ndarray) else x for x in a])
        oi, orgbd = orc.render_observation_maps(*a)
        np.testing.assert_array_equal(hi, oi)
        np.testing.assert_array_equal(hr.view(np.uint32), orgbd.view(np.uint32))
        assert 100 < (oi != 0xFFFFFFFF).sum() < oi.size
    # without colour and time: every surfel observed now, colour bytes zero
    a = (args[0], args[1], None) + args[3:]
    hi, hr = _run_host(lib, np.ascontiguousarray(a[0]), np.ascontiguousarray(a[1]), None, *a[3:])
    oi, orgbd = orc.render_observation_maps(*a)
    np.testing.assert_array_equal(hi, oi)
    np.testing.assert_array_equal(hr.view(np.uint32), orgbd.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["torus", "cloud"])
def test_observation_maps_match_the_oracle(ws, orc, small_scene, kind):
    """ws_render_observation_maps against the oracle's restatement, bit for bit, with and without
    the recent-observation pass, twice in a row on the same inputs, and without colour and time."""
    from starhub_b200.solver import GpuGeometry
    geo = GpuGeometry()
    args = _inputs(kind, small_scene)
    for tthr in (3.0, -1.0, 3.0):
        a = args[:-1] + (tthr,)
        gi, gr = geo.render_observation_maps(*a)
        oi, orgbd = orc.render_observation_maps(*a)
        np.testing.assert_array_equal(gi, oi)
        np.testing.assert_array_equal(gr.view(np.uint32), orgbd.view(np.uint32))
    a = (args[0], args[1], None) + args[3:]   # without colour and time
    gi, gr = geo.render_observation_maps(*a)
    oi, orgbd = orc.render_observation_maps(*a)
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gr.view(np.uint32), orgbd.view(np.uint32))
