"""Node construction, node graph and skinning on the GPU: integer outputs bit-exact
to the oracle, weights within a few ulps (the device uses __expf)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def surfels(orc):
    from starhub_b200 import scenes
    rng = np.random.default_rng(21)
    p, n = scenes.sample_torus(rng, 80_000, 0.3, 0.1)
    p = p @ scenes.rot_x(30.0).T + np.array([0, 0, 1.0])
    return scenes.pack4(p, 1.0)


def test_init_nodes_bit_exact(ws, orc, surfels):
    from starhub_b200.solver import GpuGeometry
    g = GpuGeometry().init_nodes(surfels, 0.025)
    o = orc.OracleGeometry().init_nodes(surfels, 0.025)
    np.testing.assert_array_equal(g, o)


@pytest.mark.parametrize("k", [4, 8])
def test_node_graph_bit_exact(ws, orc, surfels, k):
    from starhub_b200.solver import GpuGeometry
    nodes = orc.OracleGeometry().init_nodes(surfels, 0.025)
    gk, gw, ge = GpuGeometry().node_graph(nodes, k, 0.025)
    ok, ow, oe = orc.OracleGeometry().node_graph(nodes, k, 0.025)
    np.testing.assert_array_equal(gk, ok)
    np.testing.assert_array_equal(ge, oe)
    np.testing.assert_allclose(gw, ow, rtol=2e-5, atol=1e-7)


def test_skinning_bit_exact(ws, orc, surfels):
    from starhub_b200.solver import GpuGeometry
    nodes = orc.OracleGeometry().init_nodes(surfels, 0.025)
    gk, gs, gc = GpuGeometry().skinning(nodes, surfels, 0.025)
    ok, os_, oc = orc.OracleGeometry().skinning(nodes, surfels, 0.025)
    np.testing.assert_array_equal(gk, ok)
    np.testing.assert_array_equal(gc, oc)
    np.testing.assert_allclose(gs, os_, rtol=2e-5, atol=1e-7)


def test_forward_warp_matches_oracle(ws, orc, small_scene):
    from starhub_b200.solver import GpuGeometry
    sc = small_scene
    gv, _ = GpuGeometry().forward_warp(sc.gt_dq, sc.surfel_vertex, sc.surfel_normal, sc.surfel_knn, sc.surfel_sw,
                                       sc.surfel_cw)
    ov = orc.forward_warp(sc.gt_dq, sc.surfel_vertex, sc.surfel_knn, sc.surfel_sw, sc.surfel_cw)
    np.testing.assert_allclose(gv[:, :3], ov[:, :3], atol=2e-6)


def test_splat_matches_numpy(ws, small_scene):
    from starhub_b200 import scenes
    from starhub_b200.solver import GpuGeometry
    sc = small_scene
    gi = GpuGeometry().splat(sc.surfel_vertex, sc.camera, 1)
    ni = scenes.splat_np(sc.surfel_vertex, sc.camera, 1)
    np.testing.assert_array_equal(gi, ni)


@pytest.mark.parametrize("footprint,time_threshold", [(0, 3.0), (1, -1.0)])
def test_render_solver_maps_match_the_oracle(ws, orc, small_scene, footprint, time_threshold):
    """ws_render_solver_maps (the solver-map pass of RendererDraw.cu:105-175 with
    shaders/solver_map.vert:21-53) against the oracle's restatement of the same shader, bit for
    bit: a rigid world-to-camera transform, a depth cut through the torus, confidences and
    observation times that cull part of the unstable surfels, and encoded colours."""
    from starhub_b200.scenes import rot_x
    from starhub_b200.solver import GpuGeometry
    sc = small_scene
    rng = np.random.default_rng(4)
    n = sc.surfel_vertex.shape[0]
    vc = sc.surfel_vertex.copy()
    vc[:, 3] = rng.uniform(0.0, 3.0, n).astype(np.float32)
    ct = np.zeros((n, 4), np.float32)
    ct[:, 0] = rng.integers(0, 1 << 24, n).astype(np.uint32).view(np.float32)
    ct[:, 2] = rng.integers(0, 12, n).astype(np.float32)
    w2c = np.eye(4, dtype=np.float32)
    w2c[:3, :3] = rot_x(4.0).astype(np.float32)
    w2c[:3, 3] = [0.01, -0.02, 0.03]
    args = (vc, sc.surfel_normal, ct, sc.camera, w2c, 1.02, 10.0, 1.0, time_threshold, footprint)
    gi, gv, gn, gr = GpuGeometry().render_solver_maps(*args)
    oi, ov, on, orgbd = orc.render_solver_maps(*args)
    assert 1000 < (oi != 0xFFFFFFFF).sum() < oi.size
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gv, ov)
    np.testing.assert_array_equal(gn, on)
    np.testing.assert_array_equal(gr.view(np.uint32), orgbd.view(np.uint32))
