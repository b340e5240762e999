"""Edge cases of the solve on the GPU, through the C ABI.

* A scene with no visible surfel (empty index map) has no dense term: its solve succeeds
  and leaves the warp at the identity (zero right-hand side, zero step).
* A ragged batch (an empty scene between two ordinary ones of very different sizes) gives
  every scene its solo result bit for bit.
* Zero Gauss-Newton iterations return the initial warp.
* Surfel node ids past the scene's node count are reported as WS_ERR_INVALID_ARGUMENT
  (the reference reads them unchecked); the solve still runs inside its buffers.
* A NaN in the inputs that reaches the right-hand side is reported as WS_ERR_NAN
  (the reference calls exit(-1), WarpSolverPCG.cu:21-31).
* Counts beyond the 16-bit node ids and beyond the solver's capacities are refused up front.
* A depth-only scene gets the same result bit for bit with the 64-byte dense records of a
  depth-only batch and with the 128-byte records of a batch that holds a flow scene.
* A batch that needs 64-bit node-pair sort keys gives each scene its result with 32-bit keys.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solver(scenes, precision=0):
    from starhub_b200.solver import WarpSolver
    return WarpSolver(max_nodes=sum(d.num_nodes for d in scenes), max_pixels=sum(d.num_pixels for d in scenes),
                      max_edges=sum(d.num_edges for d in scenes), max_scenes=len(scenes), precision=precision)


def _solve(scenes, gn=3, pcg=10, precision=0):
    import torch
    s = _solver(scenes, precision)
    s.SetBatchInputs(scenes)
    s.SolveStreamed(gn, pcg, stream=torch.cuda.Stream())
    s.Sync()
    return [s.SolvedNodeSE3(i).cpu().numpy().copy() for i in range(len(scenes))]


def _identity(n):
    out = np.zeros((n, 8), np.float32)
    out[:, 3] = 1.0
    return out


def _empty(ds):
    import torch
    return dataclasses.replace(ds, index_map=torch.full_like(ds.index_map, -1))


@pytest.mark.parametrize("precision", [0, 1])
def test_empty_scene_keeps_identity(ws, tiny_scene, precision):
    from starhub_b200.solver import DeviceScene
    ds = _empty(DeviceScene.from_scene(tiny_scene))
    (dq,) = _solve([ds], precision=precision)
    np.testing.assert_allclose(dq, _identity(ds.num_nodes), atol=1e-7, rtol=0)


def test_ragged_batch_equals_solo(ws, small_scene, tiny_scene):
    from starhub_b200.solver import DeviceScene
    a = DeviceScene.from_scene(small_scene)
    b = _empty(DeviceScene.from_scene(tiny_scene))
    c = DeviceScene.from_scene(tiny_scene)
    batch = _solve([a, b, c])
    for got, ds in zip(batch, (a, b, c)):
        (solo,) = _solve([ds])
        np.testing.assert_array_equal(got, solo)


def test_zero_gauss_newton_iterations_return_the_initial_warp(ws, tiny_scene):
    import torch
    from starhub_b200.solver import DeviceScene
    ds = DeviceScene.from_scene(tiny_scene)
    init = torch.from_numpy(tiny_scene.gt_dq.astype(np.float32)).cuda()
    (dq,) = _solve([dataclasses.replace(ds, init_se3=init)], gn=0)
    np.testing.assert_array_equal(dq, tiny_scene.gt_dq.astype(np.float32))


def test_out_of_range_node_ids_are_reported(ws, tiny_scene):
    import torch
    from starhub_b200._lib import WS_ERR_INVALID_ARGUMENT, WarpSolveError
    from starhub_b200.solver import DeviceScene
    ds = DeviceScene.from_scene(tiny_scene)
    visible = np.unique(tiny_scene.index_map[tiny_scene.index_map != 0xFFFFFFFF])[:50].astype(np.int64)
    knn = ds.surfel_knn.clone()
    knn[torch.from_numpy(visible).cuda(), 1] = ds.num_nodes + 3
    bad = dataclasses.replace(ds, surfel_knn=knn)
    s = _solver([bad])
    s.SetBatchInputs([bad])
    s.SolveStreamed(2, 5, stream=torch.cuda.Stream())
    with pytest.raises(WarpSolveError) as e:
        s.Sync()
    assert e.value.status == WS_ERR_INVALID_ARGUMENT
    # the flag is cleared by the read: a clean solve on the same solver reports WS_OK
    s.SetBatchInputs([ds])
    s.SolveStreamed(2, 5, stream=torch.cuda.Stream())
    s.Sync()


def test_nan_right_hand_side_is_reported(ws, tiny_scene):
    import torch
    from starhub_b200._lib import WS_ERR_NAN, WarpSolveError
    from starhub_b200.solver import DeviceScene
    ds = DeviceScene.from_scene(tiny_scene)
    nodes = ds.nodes.clone()
    nodes[5, :3] = float("nan")          # reaches the smoothness residuals of node 5's edges
    bad = dataclasses.replace(ds, nodes=nodes)
    s = _solver([bad])
    s.SetBatchInputs([bad])
    s.SolveStreamed(1, 5, stream=torch.cuda.Stream())
    with pytest.raises(WarpSolveError) as e:
        s.Sync()
    assert e.value.status == WS_ERR_NAN


def test_counts_beyond_limits_are_refused(ws, tiny_scene, small_scene):
    from starhub_b200 import _lib
    from starhub_b200._lib import WS_ERR_CAPACITY, WS_ERR_INVALID_ARGUMENT, WsInputs
    from starhub_b200.solver import DeviceScene
    lib = _lib.load()
    ds = DeviceScene.from_scene(tiny_scene)
    s = _solver([ds])
    inp = ds.to_inputs()
    inp.num_nodes = 70000                # node ids are 16-bit, as in the reference
    arr = (WsInputs * 1)(inp)
    assert lib.ws_set_batch(s._h, arr, 1) == WS_ERR_INVALID_ARGUMENT
    big = DeviceScene.from_scene(small_scene)   # more nodes and pixels than the solver holds
    arr = (WsInputs * 1)(big.to_inputs())
    assert lib.ws_set_batch(s._h, arr, 1) == WS_ERR_CAPACITY
    arr = (WsInputs * 2)(ds.to_inputs(), ds.to_inputs())   # more scenes than max_scenes
    assert lib.ws_set_batch(s._h, arr, 2) == WS_ERR_CAPACITY


@pytest.mark.parametrize("precision", [0, 1])
def test_depth_only_scene_same_in_a_batch_with_flow(ws, tiny_scene, precision):
    import sys
    from pathlib import Path
    from starhub_b200.solver import DeviceScene
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    import make_golden
    d = dict(np.load(Path(__file__).resolve().parent / "golden" / "torus_small_flow.npz"))
    flow = DeviceScene.from_scene(make_golden.scene_from_arrays(d))
    assert flow.lambda_of > 0
    depth = DeviceScene.from_scene(tiny_scene)
    assert depth.lambda_of == 0
    (alone,) = _solve([depth], precision=precision)
    mixed = _solve([flow, depth], precision=precision)
    np.testing.assert_array_equal(mixed[1], alone)


def test_many_scenes_and_a_large_one_give_the_solo_results(ws, tiny_scene):
    """65 scenes, one of them with 5k nodes (global node ids above 2^16 in the batch, 13-bit
    local ids): the node-pair map built row by row and every solve in the batch must equal the
    scenes' solo results bit for bit."""
    from starhub_b200 import scenes
    from starhub_b200.solver import DeviceScene, GpuGeometry
    big = scenes.make_scene(scenes.spec_for_nodes(5000, scenes.config_spec(2)), GpuGeometry(), seed=77)
    assert big.num_nodes > 4096
    b = DeviceScene.from_scene(big)
    t = DeviceScene.from_scene(tiny_scene)
    batch = _solve([t] * 64 + [b], gn=2, pcg=5)
    (solo_b,) = _solve([b], gn=2, pcg=5)
    (solo_t,) = _solve([t], gn=2, pcg=5)
    np.testing.assert_array_equal(batch[-1], solo_b)
    np.testing.assert_array_equal(batch[0], solo_t)
    np.testing.assert_array_equal(batch[63], solo_t)


def test_pcg_wait_gives_up_and_the_device_stays_usable(ws, tiny_scene):
    """The PCG's scene wait is bounded: on a generation counter that nothing advances it
    returns WS_ERR_TIMEOUT (about two seconds of requested sleep), no GPU fault, and a solve
    on the same device afterwards succeeds and equals one before it."""
    import time
    from starhub_b200 import _lib
    from starhub_b200.solver import DeviceScene
    ds = DeviceScene.from_scene(tiny_scene)
    (before,) = _solve([ds])
    t0 = time.perf_counter()
    status = _lib.load().ws_selftest_wait_timeout(None)
    elapsed = time.perf_counter() - t0
    assert status == _lib.WS_ERR_TIMEOUT
    assert 0.05 < elapsed < 60.0
    (after,) = _solve([ds])
    np.testing.assert_array_equal(after, before)


def test_node_growth_barrier_gives_up_and_the_device_stays_usable(ws):
    """The grid barrier between the rounds of the device overlap check is bounded: with one of
    two blocks arriving it returns WS_ERR_TIMEOUT (about two seconds of requested sleep), no
    GPU fault, and node construction afterwards still equals the oracle's."""
    import time
    from starhub_b200 import _lib
    from starhub_b200.solver import GpuGeometry
    t0 = time.perf_counter()
    status = _lib.load().ws_selftest_grid_barrier_timeout(None)
    elapsed = time.perf_counter() - t0
    assert status == _lib.WS_ERR_TIMEOUT
    assert 0.05 < elapsed < 60.0
    rng = np.random.default_rng(9)
    from starhub_b200 import scenes
    p, _ = scenes.sample_torus(rng, 50_000, 0.3, 0.1)
    s = scenes.pack4(p + np.array([0, 0, 1.0]), 1.0)
    sys_path_oracle()
    import oracle as orc
    np.testing.assert_array_equal(GpuGeometry().init_nodes(s, 0.025), orc.OracleGeometry().init_nodes(s, 0.025))


def sys_path_oracle():
    import sys
    from pathlib import Path
    p = str(Path(__file__).resolve().parents[1] / "oracle")
    if p not in sys.path:
        sys.path.insert(0, p)
