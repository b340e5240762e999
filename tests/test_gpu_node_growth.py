"""Node-graph growth on the GPU, bit-exact to the oracle.

* ws_init_nodes: voxel subsample plus the greedy overlap check of
  AppendNodeFromVertexHost (NodeGraph.cu:652-704), run on the device in rounds; scenes from
  a few thousand candidates (one block, decisions in shared memory) to 200k (a cooperative
  launch over all SMs with a grid barrier between rounds).
* ws_expand_nodes: NaiveExpandNodeGraphFromVertexUnsupported (NodeGraph.cu:500-532) appends
  the greedy nodes of the unsupported vertices, sets their initial time, and leaves the
  arrays alone when they are full.
* ws_build_node_graph: the culled scan gives the same ids and weights as the full scan
  (BuildNodeGraphKernel, NodeGraph.cu:10-101), ties in the half distances included."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEDUP_ONE_BLOCK_MAX = 16384


def torus_surfels(n, seed):
    from starhub_b200 import scenes
    rng = np.random.default_rng(seed)
    p, _ = scenes.sample_torus(rng, n, 0.3, 0.1)
    p = p @ scenes.rot_x(30.0).T + np.array([0, 0, 1.0])
    return scenes.pack4(p, 1.0)


@pytest.mark.parametrize("n,radius,rounds_on", [(100_000, 0.025, "one block"), (1_000_000, 0.006, "grid"),
                                                (2_500_000, 0.004, "grid")])
def test_init_nodes_many_candidates_bit_exact(ws, orc, n, radius, rounds_on):
    from starhub_b200.solver import GpuGeometry
    s = torus_surfels(n, 31)
    og = orc.OracleGeometry()
    candidates = og.voxel_subsample(s, np.float32(0.7) * np.float32(radius)).shape[0]
    assert (candidates > DEDUP_ONE_BLOCK_MAX) == (rounds_on == "grid")
    g = GpuGeometry().init_nodes(s, radius)
    o = og.init_nodes(s, radius)
    assert g.shape == o.shape
    np.testing.assert_array_equal(g, o)


def test_init_nodes_keys_below_the_encoded_range_sort_as_signed(ws, orc):
    """encodeVoxel (libs/star/common/encode_utils.h:138-141) assumes voxel coordinates in
    (-512, 512); below -512 in z the key is negative, and the reference's sort of int keys puts
    those voxels first.  A torus straddling z = -512 voxels (R = 6 mm: voxel 4.2 mm, z about
    -2.2 m) gives keys of both signs; the device order must be the oracle's signed order."""
    from starhub_b200.solver import GpuGeometry
    s = torus_surfels(60_000, 17)
    s[:, 2] -= np.float32(3.2)                        # z in about [-2.33, -2.07] m
    radius = 0.006
    voxel = np.float32(0.7) * np.float32(radius)
    vz = np.floor(s[:, 2] / voxel).astype(np.int64)
    assert (vz < -512).any() and (vz >= -512).any()
    g = GpuGeometry().init_nodes(s, radius)
    o = orc.OracleGeometry().init_nodes(s, radius)
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


FACADE_PROGRAM = r"""
#include <cstdio>
#include <vector>
#include "starhub_b200/warp_solver.hpp"

static std::vector<float4> read_points(const char *path) {
    std::vector<float4> v;
    FILE *f = std::fopen(path, "rb");
    if (!f) return v;
    float4 p;
    while (std::fread(&p, sizeof(p), 1, f) == 1) v.push_back(p);
    std::fclose(f);
    return v;
}

int main(int argc, char **argv) {
    if (argc != 4) return 2;
    const std::vector<float4> first = read_points(argv[1]), more = read_points(argv[2]);
    float4 *d_first = nullptr, *d_more = nullptr;
    cudaMalloc(&d_first, 16 * first.size());
    cudaMalloc(&d_more, 16 * more.size());
    cudaMemcpy(d_first, first.data(), 16 * first.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(d_more, more.data(), 16 * more.size(), cudaMemcpyHostToDevice);
    star::b200::NodeGraph graph(0.01f, 32768, 4);   // 8,936 + 8,947 nodes
    graph.InitializeNodeGraphFromVertex(d_first, (unsigned)first.size(), 3, true, 0);
    const unsigned n0 = graph.GetNodeSize();
    graph.NaiveExpandNodeGraphFromVertexUnsupported(d_more, (unsigned)more.size(), 5, 0);
    graph.BuildNodeGraphFromScratch(true, 0);
    const unsigned n = graph.GetNodeSize();
    std::vector<float4> nodes(n);
    std::vector<uint16_t> knn(4ull * n);
    std::vector<unsigned> times(n);
    cudaMemcpy(nodes.data(), graph.GetReferenceNodeCoordinate(), 16ull * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(knn.data(), graph.GetNodeKnn(), 8ull * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(times.data(), graph.GetNodeInitialTime(), 4ull * n, cudaMemcpyDeviceToHost);
    FILE *f = std::fopen(argv[3], "wb");
    std::fwrite(&n0, 4, 1, f);
    std::fwrite(&n, 4, 1, f);
    std::fwrite(nodes.data(), 16, n, f);
    std::fwrite(knn.data(), 2, 4ull * n, f);
    std::fwrite(times.data(), 4, n, f);
    std::fclose(f);
    cudaFree(d_first);
    cudaFree(d_more);
    return graph.GetPrevNodeSize() == n0 ? 0 : 3;
}
"""


def test_cpp_facade_node_graph_matches_the_c_abi(ws, orc, tmp_path):
    """star::b200::NodeGraph (the C++ facade) gives the nodes, graph and initial times of the
    C ABI calls it wraps, which the oracle checks above."""
    import shutil
    import subprocess
    from pathlib import Path
    from starhub_b200.solver import GpuGeometry
    root = Path(__file__).resolve().parents[1]
    cuda = Path("/usr/local/cuda")
    if shutil.which("g++") is None:
        pytest.skip("g++ missing")
    s = torus_surfels(200_000, 41)
    first, more = s[:100_000], s[100_000:]
    (tmp_path / "first.bin").write_bytes(first.tobytes())
    (tmp_path / "more.bin").write_bytes(more.tobytes())
    (tmp_path / "prog.cpp").write_text(FACADE_PROGRAM)
    lib_dir = root / "starhub_b200"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(root / "include"), "-I", str(cuda / "include"),
                        str(tmp_path / "prog.cpp"), "-o", str(tmp_path / "prog"), "-L", str(lib_dir), "-lwarpsolve",
                        f"-Wl,-rpath,{lib_dir}", "-L", str(cuda / "lib64"), "-lcudart"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(tmp_path / "prog"), str(tmp_path / "first.bin"), str(tmp_path / "more.bin"),
                        str(tmp_path / "out.bin")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    raw = (tmp_path / "out.bin").read_bytes()
    n0, n = np.frombuffer(raw[:8], np.uint32)
    off = 8
    nodes = np.frombuffer(raw[off:off + 16 * n], np.float32).reshape(n, 4); off += 16 * n
    knn = np.frombuffer(raw[off:off + 8 * n], np.uint16).reshape(n, 4); off += 8 * n
    times = np.frombuffer(raw[off:off + 4 * n], np.uint32)

    geo = GpuGeometry()
    base = geo.init_nodes(first, 0.01)
    assert n0 == len(base)
    dev = torch.device("cuda")
    ref = torch.zeros((32768, 4), dtype=torch.float32, device=dev)
    ref[: len(base)] = torch.from_numpy(base).to(dev)
    total = geo.expand_nodes(ref, None, len(base), more, 0.01)
    assert n == total
    want = ref[:total].cpu().numpy()
    np.testing.assert_array_equal(nodes, want)
    wk, _, _ = geo.node_graph(want, 4, 0.01)
    np.testing.assert_array_equal(knn, wk)
    assert (times[:n0] == 3).all() and (times[n0:] == 5).all()
