"""Batched uneven solves: every scene's result in a batch equals its solo solve
bit for bit (per-scene reductions never depend on the rest of the batch)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch_scenes(orc):
    from starhub_b200 import scenes
    geo = orc.OracleGeometry()
    out = []
    for i, (scale, w) in enumerate([(0.5, 160), (0.7, 200), (0.45, 120)]):
        spec = scenes.config_spec(0, n_surfels=int(15000 * scale * scale / 0.25), width=w, height=int(w * 0.75),
                                  focal=w * 0.89, scale=scale)
        out.append(scenes.make_scene(spec, geo, seed=100 + i))
    return out


def test_batch_equals_solo(ws, batch_scenes):
    import torch
    from starhub_b200.solver import DeviceScene, WarpSolver
    ds = [DeviceScene.from_scene(s) for s in batch_scenes]
    tot_n = sum(d.num_nodes for d in ds)
    tot_p = sum(d.num_pixels for d in ds)
    tot_e = sum(d.num_edges for d in ds)
    st = torch.cuda.Stream()
    solo = []
    for d in ds:
        s = WarpSolver(max_nodes=d.num_nodes, max_pixels=d.num_pixels, max_edges=d.num_edges)
        s.SetSolverInputs(d)
        s.SolveStreamed(3, 15, stream=st)
        s.Sync()
        solo.append(s.SolvedNodeSE3(0).cpu().numpy().copy())
    b = WarpSolver(max_nodes=tot_n, max_pixels=tot_p, max_edges=tot_e, max_scenes=len(ds))
    b.SetBatchInputs(ds)
    b.SolveStreamed(3, 15, stream=st)
    b.Sync()
    for i in range(len(ds)):
        np.testing.assert_array_equal(b.SolvedNodeSE3(i).cpu().numpy(), solo[i])
    # the mix in another order gives the same per-scene results
    b.SetBatchInputs(ds[::-1])
    b.SolveStreamed(3, 15, stream=st)
    b.Sync()
    for i in range(len(ds)):
        np.testing.assert_array_equal(b.SolvedNodeSE3(len(ds) - 1 - i).cpu().numpy(), solo[i])


def test_batch_index_matches_solo(ws, orc, batch_scenes):
    import torch
    from starhub_b200.solver import DeviceScene, WarpSolver
    ds = [DeviceScene.from_scene(s) for s in batch_scenes]
    b = WarpSolver(max_nodes=sum(d.num_nodes for d in ds), max_pixels=sum(d.num_pixels for d in ds),
                   max_edges=sum(d.num_edges for d in ds), max_scenes=len(ds))
    b.SetBatchInputs(ds)
    b.SolveStreamed(1, 1, stream=torch.cuda.Stream())
    b.Sync()
    for i, sc in enumerate(batch_scenes):
        pix, knn, _, _ = b.dense_terms(i)
        opix, oknn, _, _ = orc.compact_pixels(sc)
        np.testing.assert_array_equal(pix, opix)
        off, ti = b.node2term(i)
        ooff, oti = orc.node2term(oknn, sc.edges, sc.num_nodes)
        np.testing.assert_array_equal(off, ooff)
        np.testing.assert_array_equal(ti, oti[: ooff[-1]])
        p = b.node_pairs(i)
        m = orc.nodepair2term(oknn, sc.edges, sc.num_nodes)
        np.testing.assert_array_equal(p["rows"], m["half_rows"])
        np.testing.assert_array_equal(p["term_index"], m["term_index"][: m["half_end"][-1]])


def test_benchmark_batch_meets_the_bar(ws, orc):
    """The benchmarked configuration: scenes of the 64-scene batch family (8-NN graph, 640x480,
    130 surfels per node, 5 Gauss-Newton x 20 PCG) at its smallest, median and largest node
    counts, solved together through the CUDA-graph replay of the batched solver, each within
    1e-4 relative twist error and 1e-5 m warped-position error of the FP64 oracle."""
    import torch
    from starhub_b200 import scenes
    from starhub_b200.scenes import position_error, twist_error
    from starhub_b200.solver import DeviceScene, GpuGeometry, WarpSolver
    targets = scenes.batch_node_targets(64, 2)
    order = np.argsort(targets, kind="stable")
    picks = [int(order[0]), int(order[32]), int(order[-1])]
    geo = GpuGeometry()
    host = [scenes.batch_scene(int(targets[i]), geo, i) for i in picks]
    assert all(sc.graph_k == 8 for sc in host)
    assert host[-1].num_nodes > 6000
    ds = [DeviceScene.from_scene(sc) for sc in host]
    b = WarpSolver(max_nodes=sum(d.num_nodes for d in ds), max_pixels=sum(d.num_pixels for d in ds),
                   max_edges=sum(d.num_edges for d in ds), max_scenes=len(ds))
    b.SetBatchInputs(ds)
    st = torch.cuda.Stream()
    for _ in range(2):                      # capture, then a replay
        b.SolveStreamed(5, 20, stream=st, graph=True)
    b.Sync()
    for i, sc in enumerate(host):
        dq = b.SolvedNodeSE3(i).cpu().numpy().copy()
        ref = orc.solve(sc, gn_iters=5, pcg_iters=20)
        te, pe = twist_error(dq, ref, sc.nodes), position_error(sc, dq, ref)
        assert te <= 1e-4, f"scene {picks[i]} ({sc.num_nodes} nodes): twist error {te}"
        assert pe <= 1e-5, f"scene {picks[i]} ({sc.num_nodes} nodes): position error {pe}"
