"""Autotuner (ws_autotune): it times the launch-shape candidates on the caller's inputs and
keeps the fastest; no shape may change a result, so a tuned solve equals the default one
bit for bit, and so does every explicit shape."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(small_scene, tiny_scene, precision):
    from starhub_b200.solver import DeviceScene, WarpSolver
    ds = [DeviceScene.from_scene(s) for s in (small_scene, tiny_scene)]
    s = WarpSolver(max_nodes=sum(d.num_nodes for d in ds), max_pixels=sum(d.num_pixels for d in ds),
                   max_edges=sum(d.num_edges for d in ds), max_scenes=2, precision=precision)
    s.SetBatchInputs(ds)
    return s


def _solve(s):
    import torch
    st = torch.cuda.Stream()
    s.SolveStreamed(3, 10, stream=st, graph=True)
    s.Sync()
    return [s.SolvedNodeSE3(i).cpu().numpy().copy() for i in range(2)]


@pytest.mark.parametrize("precision", [0, 1])
def test_autotune_picks_offered_shapes_and_keeps_results(ws, small_scene, tiny_scene, precision):
    import torch
    s = _batch(small_scene, tiny_scene, precision)
    ref = _solve(s)
    t = s.autotune(pcg_iters=10, stream=torch.cuda.Stream())
    assert t["node_threads"] in (64, 128, 256) and t["pair_threads"] in (64, 128, 256)
    assert t["pcg_blocks_per_sm"] >= 1
    assert t["node_ms"][(64, 128, 256).index(t["node_threads"])] > 0
    assert t["pair_ms"][(64, 128, 256).index(t["pair_threads"])] == min(m for m in t["pair_ms"] if m >= 0)
    offered = [m for m in t["pcg_ms"] if m >= 0]
    assert offered and min(offered) == t["pcg_ms"][t["pcg_blocks_per_sm"] - 1]
    tuned = _solve(s)
    for a, b in zip(ref, tuned):
        np.testing.assert_array_equal(a, b)
    for shape in ((64, 64, 1), (128, 256, 2)):
        s.set_tuning(*shape)
        for a, b in zip(ref, _solve(s)):
            np.testing.assert_array_equal(a, b)
