"""Node-graph growth on the GPU, bit-exact to the oracle.

* ws_init_nodes: voxel subsample plus the greedy overlap check of
  AppendNodeFromVertexHost (NodeGraph.cu:652-704), run on the device in rounds; scenes with
  up to 200k candidates, so that the decisions live in shared memory in one case and in
  global memory in the other.
* ws_expand_nodes: NaiveExpandNodeGraphFromVertexUnsupported (NodeGraph.cu:500-532) appends
  the greedy nodes of the unsupported vertices, sets their initial time, and leaves the
  arrays alone when they are full.
* ws_build_node_graph: the culled scan gives the same ids and weights as the full scan
  (BuildNodeGraphKernel, NodeGraph.cu:10-101), ties in the half distances included."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEDUP_SHARED_MAX = 160 * 1024


def torus_surfels(n, seed):
    from starhub_b200 import scenes
    rng = np.random.default_rng(seed)
    p, _ = scenes.sample_torus(rng, n, 0.3, 0.1)
    p = p @ scenes.rot_x(30.0).T + np.array([0, 0, 1.0])
    return scenes.pack4(p, 1.0)


@pytest.mark.parametrize("n,radius,decisions", [(1_000_000, 0.006, "shared"), (2_500_000, 0.004, "global")])
def test_init_nodes_many_candidates_bit_exact(ws, orc, n, radius, decisions):
    from starhub_b200.solver import GpuGeometry
    s = torus_surfels(n, 31)
    og = orc.OracleGeometry()
    candidates = og.voxel_subsample(s, np.float32(0.7) * np.float32(radius)).shape[0]
    assert (candidates > DEDUP_SHARED_MAX) == (decisions == "global")
    g = GpuGeometry().init_nodes(s, radius)
    o = og.init_nodes(s, radius)
    assert g.shape == o.shape
    np.testing.assert_array_equal(g, o)


def test_init_nodes_nan_surfel_is_rejected(ws):
    from starhub_b200._lib import WarpSolveError
    from starhub_b200.solver import GpuGeometry
    s = torus_surfels(20_000, 3)
    s[123, 1] = np.nan
    with pytest.raises(WarpSolveError):
        GpuGeometry().init_nodes(s, 0.025)


def test_expand_nodes_appends_the_greedy_nodes(ws, orc):
    from starhub_b200._lib import WarpSolveError
    from starhub_b200.solver import GpuGeometry
    s = torus_surfels(200_000, 41)
    radius = 0.01
    og = orc.OracleGeometry()
    base = og.init_nodes(s[:100_000], radius)
    unsupported = s[100_000:]
    grown = og.init_nodes(unsupported, radius)[2:]       # the same greedy pass without the anchors
    want = np.concatenate([base, grown])
    cap = len(want) + 16
    dev = torch.device("cuda")
    ref = torch.zeros((cap, 4), dtype=torch.float32, device=dev)
    ref[: len(base)] = torch.from_numpy(base).to(dev)
    live = ref.clone()
    times = torch.full((cap,), 7, dtype=torch.int32, device=dev)
    geo = GpuGeometry()
    n = geo.expand_nodes(ref, live, len(base), unsupported, radius, node_time=times, current_time=42)
    assert n == len(want)
    np.testing.assert_array_equal(ref[:n].cpu().numpy(), want)
    np.testing.assert_array_equal(live[:n].cpu().numpy(), want)
    t = times.cpu().numpy()
    assert (t[: len(base)] == 7).all() and (t[len(base):n] == 42).all() and (t[n:] == 7).all()

    # No vertices: nothing changes.
    assert geo.expand_nodes(ref, None, n, np.zeros((0, 4), np.float32), radius) == n
    np.testing.assert_array_equal(ref[:n].cpu().numpy(), want)

    # Full arrays: an error, and the arrays stay as they were.
    small = torch.zeros((len(want) - 1, 4), dtype=torch.float32, device=dev)
    small[: len(base)] = torch.from_numpy(base).to(dev)
    before = small.clone()
    with pytest.raises(WarpSolveError):
        geo.expand_nodes(small, None, len(base), unsupported, radius)
    assert torch.equal(small, before)


@pytest.mark.parametrize("k", [4, 8])
def test_node_graph_culled_scan_large_scene(ws, orc, k):
    from starhub_b200.solver import GpuGeometry
    nodes = orc.OracleGeometry().init_nodes(torus_surfels(1_000_000, 31), 0.006)
    gk, gw, ge = GpuGeometry().node_graph(nodes, k, 0.006)
    ok, ow, oe = orc.OracleGeometry().node_graph(nodes, k, 0.006)
    np.testing.assert_array_equal(gk, ok)
    np.testing.assert_array_equal(ge, oe)
    np.testing.assert_allclose(gw, ow, rtol=2e-5, atol=1e-7)


@pytest.mark.parametrize("order", ["lattice", "shuffled"])
@pytest.mark.parametrize("k", [4, 8])
def test_node_graph_ties(ws, orc, order, k):
    """Nodes on a lattice (many equal half distances) plus repeated points, in lattice order
    (runs with tight boxes) or shuffled (wide boxes): the heap's tie-breaking is kept."""
    from starhub_b200.solver import GpuGeometry
    g = np.stack(np.meshgrid(np.arange(16), np.arange(16), np.arange(12), indexing="ij"), -1).reshape(-1, 3)
    p = g.astype(np.float32) * np.float32(0.0125)
    p = np.concatenate([p, p[::37]])                       # exact duplicates
    if order == "shuffled":
        p = p[np.random.default_rng(5).permutation(len(p))]
    nodes = np.concatenate([p, np.ones((len(p), 1), np.float32)], 1)
    gk, gw, ge = GpuGeometry().node_graph(nodes, k, 0.025)
    ok, ow, oe = orc.OracleGeometry().node_graph(nodes, k, 0.025)
    np.testing.assert_array_equal(gk, ok)
    np.testing.assert_array_equal(ge, oe)
    np.testing.assert_allclose(gw, ow, rtol=2e-5, atol=1e-7)
