"""Re-skinning after node growth, deleted nodes and the reference's unnormalised weights, on the
GPU against the oracle.

* Skinner::PerformIncSkinnningFromLive / IncSkinnerKernel (libs/star/geometry/node_graph/
  Skinner.cu:211-302, 395-415): after nodes were appended, the surfels from num_remaining_surfels on
  are re-skinned from their current neighbours and the appended nodes only.
* Deleted nodes (node status .y == 0xFFFFFFFF, NodeGraph.h:18) are skipped by skinning
  (Skinner.cu:39-48) and by the node graph (NodeGraph.cu:20-35).
* Weights with and without division by their sum: the reference's geometry library is compiled
  without USE_INTERPOLATE_WEIGHT_NORMALIZATION (defined only in
  examples/mono_star/common/global_configs.h:31-32), so its skinning and node-graph weights are the
  raw exponentials (Skinner.cu:70-76, NodeGraph.cu:87-99).

Ids bit-exact; weights within 2e-5 relative (__expf on the device, expf in the oracle).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
R = 0.02


def torus(n, seed):
    from starhub_b200 import scenes
    rng = np.random.default_rng(seed)
    p, _ = scenes.sample_torus(rng, n, 0.3, 0.1)
    p = p @ scenes.rot_x(30.0).T + np.array([0, 0, 1.0])
    return scenes.pack4(p, 1.0)


@pytest.fixture(scope="module")
def grown(orc):
    """Nodes of a first half of a torus, and the nodes grown from the second half appended."""
    s = torus(120_000, 7)
    og = orc.OracleGeometry()
    base = og.init_nodes(s[:60_000], R)
    grown_nodes = og.init_nodes(s[60_000:], R)[2:]
    return s, base, np.concatenate([base, grown_nodes])


def status_with_deleted(n, frac, seed):
    rng = np.random.default_rng(seed)
    st = np.zeros((n, 2), np.uint32)
    st[:, 0] = rng.integers(0, 5, n)
    st[rng.uniform(size=n) < frac, 1] = 0xFFFFFFFF
    return st


@pytest.mark.parametrize("normalize", [True, False])
def test_skinning_with_deleted_nodes(ws, orc, grown, normalize):
    from starhub_b200.solver import GpuGeometry
    s, _, nodes = grown
    st = status_with_deleted(len(nodes), 0.05, 1)
    gk, gs, gc = GpuGeometry().skinning_ex(nodes, s, R, status=st, normalize=normalize)
    ok, osw, oc = orc.OracleGeometry().skinning_ex(nodes, s, R, status=st, normalize=normalize)
    np.testing.assert_array_equal(gk, ok)
    assert not np.isin(gk, np.nonzero(st[:, 1] == 0xFFFFFFFF)[0]).any()
    np.testing.assert_allclose(gs, osw, rtol=2e-5, atol=1e-7)
    np.testing.assert_array_equal(gc, oc)
    if not normalize:
        assert (gs.sum(1) > 1.05).mean() > 0.5          # the raw weights do not sum to one


@pytest.mark.parametrize("normalize", [True, False])
def test_incremental_skinning(ws, orc, grown, normalize):
    """Surfels 0 .. 59,999 stay as they are; 60,000 on start from their skinning over the first
    nodes and take the appended nodes.  The result equals the oracle's incremental form, and, for
    the re-skinned surfels, the full skinning over all nodes."""
    from starhub_b200.solver import GpuGeometry
    s, base, nodes = grown
    geo, og = GpuGeometry(), orc.OracleGeometry()
    k0, w0, c0 = geo.skinning_ex(base, s, R, normalize=normalize)
    first, prev = 60_000, len(base)
    gk, gs, _ = geo.skinning_ex(nodes, s, R, normalize=normalize, prev_nodes=prev, first_vert=first, knn=k0)
    ok, osw, _ = og.skinning_ex(nodes, s, R, normalize=normalize, prev_nodes=prev, first_vert=first, knn=k0)
    np.testing.assert_array_equal(gk, ok)
    np.testing.assert_array_equal(gk[:first], k0[:first])
    np.testing.assert_allclose(gs[first:], osw[first:], rtol=2e-5, atol=1e-7)
    fk, _, _ = og.skinning_ex(nodes, s, R, normalize=normalize)
    assert (gk[first:] == fk[first:]).all(axis=1).mean() > 0.999
    assert (gk[first:] >= prev).any()                    # appended nodes were taken


@pytest.mark.parametrize("k", [4, 8])
@pytest.mark.parametrize("normalize", [True, False])
def test_node_graph_with_deleted_nodes(ws, orc, grown, k, normalize):
    from starhub_b200.solver import GpuGeometry
    _, _, nodes = grown
    st = status_with_deleted(len(nodes), 0.1, 2)
    gk, gw, ge = GpuGeometry().node_graph_ex(nodes, k, R, status=st, normalize=normalize)
    ok, ow, oe = orc.OracleGeometry().node_graph_ex(nodes, k, R, status=st, normalize=normalize)
    np.testing.assert_array_equal(gk, ok)
    np.testing.assert_array_equal(ge, oe)
    live = st[:, 1] != 0xFFFFFFFF
    np.testing.assert_allclose(gw[live], ow[live], rtol=2e-5, atol=1e-7)
    if normalize:
        assert np.isnan(gw[~live]).all() and np.isnan(ow[~live]).all()   # 0 / 0, as the reference
    else:
        assert (gw[~live] == 0).all()
    assert not np.isin(gk[live], np.nonzero(~live)[0]).any()


def test_facade_reanchor_and_skinner(ws, orc, tmp_path):
    """star::b200::NodeGraph::ReAnchor (NodeGraph.cu:574-650) and star::b200::Skinner through the C++
    facade: B's reference nodes are A's live nodes, B keeps A's graph and status (node 7 deleted),
    and skinning against B skips the deleted node, with the reference library's raw weights."""
    import shutil
    import subprocess
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    cuda = Path("/usr/local/cuda")
    if shutil.which("g++") is None:
        pytest.skip("g++ missing")
    s = torus(80_000, 13)
    (tmp_path / "s.bin").write_bytes(s.tobytes())
    lib_dir = root / "starhub_b200"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(root / "include"), "-I", str(cuda / "include"),
                        str(root / "tests" / "facade_reanchor.cpp"), "-o", str(tmp_path / "prog"), "-L", str(lib_dir),
                        "-lwarpsolve", f"-Wl,-rpath,{lib_dir}", "-L", str(cuda / "lib64"), "-lcudart"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(tmp_path / "prog"), str(tmp_path / "s.bin"), str(tmp_path / "out.bin")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    raw = (tmp_path / "out.bin").read_bytes()
    off = 0

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(raw[off:off + np.dtype(dtype).itemsize * count], dtype)
        off += np.dtype(dtype).itemsize * count
        return a

    n = int(take(np.uint32, 1)[0])
    live = take(np.float32, 4 * n).reshape(n, 4)
    nb = int(take(np.uint32, 1)[0])
    bref = take(np.float32, 4 * nb).reshape(nb, 4)
    aknn = take(np.uint16, 4 * n).reshape(n, 4)
    bknn = take(np.uint16, 4 * nb).reshape(nb, 4)
    bst = take(np.uint32, 2 * nb).reshape(nb, 2)
    sknn = take(np.uint16, 4 * len(s)).reshape(-1, 4)
    ssw = take(np.float32, 4 * len(s)).reshape(-1, 4)
    og = orc.OracleGeometry()
    nodes = og.init_nodes(s, 0.02)
    assert nb == n == len(nodes)
    np.testing.assert_array_equal(bref, live)
    np.testing.assert_array_equal(bknn, aknn)
    assert bst[7, 1] == 0xFFFFFFFF and (bst[np.arange(nb) != 7, 1] == 0).all()
    st = np.zeros((n, 2), np.uint32)
    st[7, 1] = 0xFFFFFFFF
    gk, _, _ = og.node_graph_ex(live, 4, 0.02, status=st, normalize=False)
    np.testing.assert_array_equal(aknn, gk)
    ok, osw, _ = og.skinning_ex(bref, s, 0.02, status=st, normalize=False)
    np.testing.assert_array_equal(sknn, ok)
    np.testing.assert_allclose(ssw, osw, rtol=2e-5, atol=1e-7)
    assert not (sknn == 7).any()
