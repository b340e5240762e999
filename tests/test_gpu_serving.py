"""The continuous-batching server (ws_server_* / ws_submit / ws_poll) on the GPU.

* A frame's result is bit-identical whether it is solved alone or batched with other
  streams' frames that arrived while the GPU was busy.
* The served result equals the drop-in solver's result on the same inputs, and a
  stream's frames are solved in order, each from the warp the previous frame produced.
* Memory admission: executors that do not fit the budget fail creation, and scenes are
  refused once their resident bytes would exceed it.
* Accuracy: a served frame is within 1e-4 relative twist error of the FP64 oracle.
"""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TWIST_TOL = 1e-4


@pytest.fixture(scope="module")
def streams(ws):
    from starhub_b200 import serving
    return serving.build_streams([600, 900, 750, 500], frames=3, seed=7)


def _server(streams, executors=1, budget=16e9):
    from starhub_b200.serving import Server
    return Server(memory_budget=int(budget), executors=executors, max_batch_scenes=len(streams),
                  max_batch_nodes=sum(s.ds.num_nodes for s in streams),
                  max_batch_pixels=sum(s.ds.num_pixels for s in streams),
                  max_batch_edges=sum(s.ds.num_edges for s in streams))


def _submit(srv, sid, stream, k, out=None):
    fr = stream.frame(k)
    return srv.submit(sid, fr.measure_vertex, fr.measure_normal, stream.ds.reference_vertex,
                      stream.ds.reference_normal, stream.ds.index_map, solution_out=out)


def _direct(stream, k, init=None):
    """The drop-in solver (one scene, stream launch) on frame k of the stream."""
    import torch
    from starhub_b200.solver import WarpSolver
    fr = stream.frame(k)
    ds = dataclasses.replace(stream.ds, measure_vertex=fr.measure_vertex, measure_normal=fr.measure_normal,
                             init_se3=init)
    s = WarpSolver(max_nodes=ds.num_nodes, max_pixels=ds.num_pixels, max_edges=ds.num_edges)
    s.SetSolverInputs(ds)
    st = torch.cuda.Stream()
    s.SolveStreamed(5, 20, stream=st)
    s.Sync()
    return s.SolvedNodeSE3(0).clone()


def test_result_is_the_same_alone_and_in_a_mix(streams):
    import torch
    with _server(streams) as srv:
        ids = [srv.add_scene(s.ds) for s in streams]
        start = srv.warp(ids[0]).clone()
        alone = torch.zeros_like(start)
        info = srv.wait(_submit(srv, ids[0], streams[0], 0, alone))
        assert info["status"] == 0 and info["batch_scenes"] == 1
        srv.set_warp(ids[0], start)
        mixed = torch.zeros_like(start)
        # the first frame occupies the single executor; the next three arrive while it runs
        # and are solved together as the following batch
        r = [_submit(srv, ids[1], streams[1], 0), _submit(srv, ids[0], streams[0], 0, mixed),
             _submit(srv, ids[2], streams[2], 0), _submit(srv, ids[3], streams[3], 0)]
        infos = [srv.wait(x) for x in r]
        assert all(i["status"] == 0 for i in infos)
        assert infos[1]["batch_scenes"] >= 2
        torch.cuda.synchronize()
        assert torch.equal(alone, mixed)
        assert not torch.equal(alone, start)


def test_served_frames_match_the_drop_in_solver_in_order(streams):
    import torch
    s = streams[1]
    with _server(streams, executors=2) as srv:
        sid = srv.add_scene(s.ds)
        out0 = torch.zeros((s.ds.num_nodes, 8), device="cuda")
        out1 = torch.zeros_like(out0)
        r0 = _submit(srv, sid, s, 0, out0)
        r1 = _submit(srv, sid, s, 1, out1)       # queued behind frame 0 of the same stream
        i0, i1 = srv.wait(r0), srv.wait(r1)
        assert i0["status"] == 0 and i1["status"] == 0
        torch.cuda.synchronize()
        x0 = _direct(s, 0)
        x1 = _direct(s, 1, init=x0)
        assert torch.equal(out0, x0)
        assert torch.equal(out1, x1)
        assert torch.equal(srv.warp(sid), x1)


def test_memory_admission(streams):
    from starhub_b200._lib import WS_ERR_CAPACITY, WS_ERR_INVALID_ARGUMENT, WarpSolveError
    with pytest.raises(WarpSolveError) as e:
        _server(streams, budget=1 << 20)
    assert e.value.status == WS_ERR_CAPACITY
    with _server(streams) as srv:
        exec_bytes = srv.stats()["executor_bytes"]
    assert exec_bytes > 0
    with _server(streams, budget=exec_bytes + (128 << 20)) as srv:
        stats = srv.stats()
        assert stats["executor_bytes"] <= stats["memory_budget"]
        admitted = []
        with pytest.raises(WarpSolveError) as e:
            for s in streams * 200:          # a few MB each: the budget runs out well before
                admitted.append(srv.add_scene(s.ds))
        assert e.value.status == WS_ERR_CAPACITY
        assert len(admitted) > 0
        stats = srv.stats()
        assert stats["executor_bytes"] + stats["resident_bytes"] <= stats["memory_budget"]
        assert srv.remove_scene(admitted[0]) == 0
        with pytest.raises(WarpSolveError) as e:
            _submit(srv, 12345, streams[0], 0)
        assert e.value.status == WS_ERR_INVALID_ARGUMENT


def test_served_frame_within_tolerance_of_the_fp64_oracle(streams, orc):
    import torch
    from starhub_b200.scenes import twist_error
    s = streams[3]
    with _server(streams) as srv:
        sid = srv.add_scene(s.ds)
        out = torch.zeros((s.ds.num_nodes, 8), device="cuda")
        assert srv.wait(_submit(srv, sid, s, 0, out))["status"] == 0
    fr = s.frame(0)
    host = dataclasses.replace(s.scene, meas_vertex=fr.measure_vertex.cpu().numpy(),
                               meas_normal=fr.measure_normal.cpu().numpy())
    ref = orc.solve(host, gn_iters=5, pcg_iters=20)
    err = twist_error(out.cpu().numpy(), ref, host.nodes)
    assert err <= TWIST_TOL, err


def test_chained_frames_of_a_large_stream_match_the_fp64_oracle(ws, orc):
    """Serving's own configuration at its upper size: one stream of about 9k nodes (the scene
    family of the serving workload, 8-NN graph, 130 surfels per node), frames 0-3 submitted back
    to back; the server solves each from the warp its previous frame produced.  Each frame's
    solution is checked against the FP64 oracle started from the oracle's solution of the
    previous frame, within 1e-4 relative twist error and 1e-5 m."""
    import torch
    from starhub_b200 import serving
    from starhub_b200.scenes import position_error, twist_error
    (s,) = serving.build_streams([9000], frames=4, seed=11)
    assert s.ds.num_nodes > 8000 and s.scene.graph_k == 8
    outs = [torch.zeros((s.ds.num_nodes, 8), device="cuda") for _ in range(4)]
    with _server([s], executors=2) as srv:
        sid = srv.add_scene(s.ds)
        rids = [_submit(srv, sid, s, k, outs[k]) for k in range(4)]
        assert all(srv.wait(r)["status"] == 0 for r in rids)
    torch.cuda.synchronize()
    prev = None
    for k in range(4):
        fr = s.frame(k)
        host = dataclasses.replace(s.scene, meas_vertex=fr.measure_vertex.cpu().numpy(),
                                   meas_normal=fr.measure_normal.cpu().numpy())
        ref = orc.solve(host, gn_iters=5, pcg_iters=20, init_dq=prev)
        got = outs[k].cpu().numpy()
        assert twist_error(got, ref, host.nodes) <= TWIST_TOL, (k, twist_error(got, ref, host.nodes))
        assert position_error(host, got, ref) <= 1e-5, k
        prev = ref
