"""Serving front end: the continuous-batching request loop of libwarpsolve.so.

`Server` wraps the native server (ws_server_* / ws_submit / ws_poll in include/warpsolve.h):
executors with their own streams solve the waiting frames as batches, each stream's node
graph, surfel skinning and warp stay resident on the device, and scenes and executors are
admitted against a device-memory budget.

`FrameStream` is a synthetic frame source for one stream: a scene built like the benchmark
scenes and a smooth ground-truth motion that advances every frame.  Its measurement maps
are rendered on the GPU (ws_forward_warp + ws_splat_maps) ahead of the timed run, for a
ping-pong cycle of frames, so the load generator only submits.

`run_streams` drives many streams with frames arriving every `period_ms` plus exponential
jitter, and reports solves/s and p50/p99 latency (submit -> solved, host clock).

Nothing here falls back to a CPU path: every solve goes through the CUDA library.
"""
from __future__ import annotations

import ctypes as C
import heapq
import time
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np

from . import _lib
from ._lib import (WS_ERR_NOT_READY, WS_OK, WS_PREC_MIXED, WsFrame, WsRequestInfo, WsServerConfig, WsServerStats,
                   check)


def _ptr(t) -> Optional[int]:
    return None if t is None else int(t.data_ptr())


def _info_dict(info: WsRequestInfo) -> dict:
    return {"status": info.status, "scene": info.scene, "num_nodes": info.num_nodes,
            "batch_scenes": info.batch_scenes, "queue_ms": info.queue_ms, "solve_ms": info.solve_ms,
            "latency_ms": info.latency_ms}


class Server:
    """Persistent request loop on one GPU (see include/warpsolve.h, "Serving")."""

    def __init__(self, memory_budget: int, executors: int = 2, max_batch_scenes: int = 32,
                 max_batch_nodes: int = 200_000, max_batch_pixels: int = 32 * 640 * 480,
                 max_batch_edges: int = 800_000, gn_iters: int = 5, pcg_iters: int = 20,
                 precision: int = WS_PREC_MIXED, device: int = 0):
        self._lib = _lib.load()
        cfg = WsServerConfig()
        cfg.device = device
        cfg.memory_budget = int(memory_budget)
        cfg.executors = executors
        cfg.max_batch_scenes = max_batch_scenes
        cfg.max_batch_nodes = max_batch_nodes
        cfg.max_batch_pixels = max_batch_pixels
        cfg.max_batch_edges = max_batch_edges
        cfg.gn_iters = gn_iters
        cfg.pcg_iters = pcg_iters
        cfg.precision = precision
        h = C.c_void_p()
        check(self._lib.ws_server_create(C.byref(cfg), C.byref(h)), "ws_server_create")
        self._h = h
        self._frames: Dict[int, tuple] = {}   # request id -> tensors kept alive until done

    def close(self) -> None:
        if self._h:
            self._lib.ws_server_destroy(self._h)
            self._h = None
            self._frames.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- scenes ----
    def add_scene(self, device_scene) -> int:
        """Copies a DeviceScene's static state (skinning, graph, camera, penalties, init warp) into
        the server's resident memory.  Raises WarpSolveError(WS_ERR_CAPACITY) past the budget."""
        sid = C.c_int()
        inputs = device_scene.to_inputs()
        check(self._lib.ws_server_add_scene(self._h, C.byref(inputs), C.byref(sid)), "ws_server_add_scene")
        return sid.value

    def remove_scene(self, scene_id: int) -> int:
        return self._lib.ws_server_remove_scene(self._h, scene_id)

    def warp(self, scene_id: int):
        """Copy of the stream's resident warp as a (num_nodes, 8) float32 CUDA tensor."""
        import torch
        p = C.c_void_p()
        n = C.c_int()
        check(self._lib.ws_server_get_warp(self._h, scene_id, C.byref(p), C.byref(n)), "ws_server_get_warp")
        out = torch.empty((n.value, 8), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        check(self._lib.ws_server_copy_warp(self._h, scene_id, C.c_void_p(out.data_ptr())), "ws_server_copy_warp")
        return out

    def set_warp(self, scene_id: int, dq) -> None:
        import torch
        torch.cuda.synchronize()
        check(self._lib.ws_server_set_warp(self._h, scene_id, C.c_void_p(dq.data_ptr())), "ws_server_set_warp")

    # ---- requests ----
    def submit(self, scene_id: int, measure_vertex, measure_normal, reference_vertex, reference_normal, index_map,
               flow=None, cam2world=None, solution_out=None) -> int:
        """Queues one frame; the tensors are kept alive until the request is forgotten."""
        f = WsFrame()
        f.measure_vertex_confid = _ptr(measure_vertex)
        f.measure_normal_radius = _ptr(measure_normal)
        f.reference_vertex = _ptr(reference_vertex)
        f.reference_normal = _ptr(reference_normal)
        f.index_map = _ptr(index_map)
        f.opticalflow = _ptr(flow)
        f.pitch = 0
        m = np.eye(4, dtype=np.float32) if cam2world is None else np.asarray(cam2world, np.float32)
        f.cam2world[:] = [float(v) for v in m.reshape(-1)]
        f.node_motion_pred = None
        f.solution_out = _ptr(solution_out)
        rid = C.c_ulonglong()
        check(self._lib.ws_submit(self._h, scene_id, C.byref(f), C.byref(rid)), "ws_submit")
        self._frames[rid.value] = (measure_vertex, measure_normal, reference_vertex, reference_normal, index_map,
                                   flow, solution_out)
        return rid.value

    def poll(self, request_id: int) -> Optional[dict]:
        info = WsRequestInfo()
        st = self._lib.ws_poll(self._h, C.c_ulonglong(request_id), C.byref(info))
        if st == WS_ERR_NOT_READY:
            return None
        return _info_dict(info)

    def wait(self, request_id: int) -> dict:
        info = WsRequestInfo()
        self._lib.ws_wait(self._h, C.c_ulonglong(request_id), C.byref(info))
        return _info_dict(info)

    def forget(self, request_id: int) -> None:
        self._lib.ws_server_forget(self._h, C.c_ulonglong(request_id))
        self._frames.pop(request_id, None)

    def stats(self) -> dict:
        s = WsServerStats()
        check(self._lib.ws_server_get_stats(self._h, C.byref(s)), "ws_server_get_stats")
        return {k: getattr(s, k) for k, _ in WsServerStats._fields_}


# ---------------------------------------------------------------------------
# synthetic frame streams
# ---------------------------------------------------------------------------
def _motion_path(nodes, surfels, frames: int, max_rot_deg: float, max_trans: float, seed: int, device):
    """`frames` per-node dual quaternions (frames, N, 8) of a smooth motion: frame f is the
    composition of f increments, each a rotation about the warped node plus a translation
    from RBF fields (sigma 0.15 m) bounded by max_rot_deg / max_trans."""
    import torch
    from . import scenes
    rng = np.random.default_rng(seed)
    x = torch.as_tensor(nodes[:, :3], dtype=torch.float64, device=device)
    R = torch.eye(3, dtype=torch.float64, device=device).expand(x.shape[0], 3, 3).clone()
    t = torch.zeros_like(x)
    out = []
    for _ in range(frames):
        cur = torch.einsum("nij,nj->ni", R, x) + t
        inc = scenes.smooth_warp(rng, cur.cpu().numpy().astype(np.float32), surfels, max_rot_deg, max_trans)
        Ri, ti = scenes.dq_to_se3(inc)
        Ri = torch.as_tensor(Ri, dtype=torch.float64, device=device)
        ti = torch.as_tensor(ti, dtype=torch.float64, device=device)
        R = Ri @ R
        t = torch.einsum("nij,nj->ni", Ri, t) + ti
        dq = scenes.se3_to_dq(R.cpu().numpy(), t.cpu().numpy())
        out.append(torch.as_tensor(dq, dtype=torch.float32, device=device))
    return torch.stack(out)


@dataclass
class Frame:
    measure_vertex: object
    measure_normal: object
    gt_dq: object


class FrameStream:
    """One stream: a resident scene plus a cycle of pre-rendered frames (ping-pong order)."""

    def __init__(self, scene, device_scene, frames: int = 8, max_rot_deg: float = 3.0, max_trans: float = 0.005,
                 depth_noise: float = 0.001, seed: int = 0, device: str = "cuda"):
        import torch
        self.scene = scene
        self.ds = device_scene
        lib = _lib.load()
        dev = torch.device(device)
        verts = torch.as_tensor(scene.surfel_vertex, device=dev)
        normals = torch.as_tensor(scene.surfel_normal, device=dev)
        knn = torch.as_tensor(scene.surfel_knn.view(np.int16), device=dev)
        sw = torch.as_tensor(scene.surfel_sw, device=dev)
        cw = torch.as_tensor(scene.surfel_cw, device=dev)
        cam = scene.camera
        path = _motion_path(scene.nodes, scene.surfel_vertex, frames, max_rot_deg, max_trans, seed, dev)
        gen = torch.Generator(device=dev)
        gen.manual_seed(seed)
        st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        self.frames: List[Frame] = []
        for f in range(frames):
            dq = path[f].contiguous()
            wv = torch.empty_like(verts)
            wn = torch.empty_like(normals)
            check(lib.ws_forward_warp(_ptr(dq), int(dq.shape[0]), _ptr(verts), _ptr(normals), int(verts.shape[0]),
                                      _ptr(knn), _ptr(sw), _ptr(cw), _ptr(wv), _ptr(wn), st), "ws_forward_warp")
            idx = torch.empty((cam.height, cam.width), dtype=torch.int32, device=dev)
            vm = torch.empty((cam.height, cam.width, 4), dtype=torch.float32, device=dev)
            nm = torch.empty((cam.height, cam.width, 4), dtype=torch.float32, device=dev)
            check(lib.ws_splat_maps(_ptr(wv), _ptr(wv), _ptr(wn), int(wv.shape[0]), cam.width, cam.height, cam.fx,
                                    cam.fy, cam.cx, cam.cy, 1, _ptr(idx), _ptr(vm), _ptr(nm), st), "ws_splat_maps")
            z = vm[..., 2]
            valid = z > 0
            noise = torch.randn(z.shape, generator=gen, device=dev) * depth_noise
            scale = torch.where(valid, (z + noise) / torch.where(valid, z, torch.ones_like(z)), torch.zeros_like(z))
            vm[..., :3] *= scale[..., None]
            self.frames.append(Frame(vm, nm, dq))
        torch.cuda.synchronize()

    def frame(self, k: int) -> Frame:
        """Ping-pong order over the cycle: 0, 1, ..., F-1, F-2, ..., 1, 0, 1, ..."""
        n = len(self.frames)
        if n == 1:
            return self.frames[0]
        p = k % (2 * n - 2)
        return self.frames[p if p < n else 2 * n - 2 - p]


def build_streams(node_counts, frames: int = 8, seed: int = 4, device: str = "cuda", geometry=None,
                  max_rot_deg: float = 3.0, max_trans: float = 0.005):
    """Frame streams of torus scenes scaled to the given node counts (surfels = 130 x nodes)."""
    from . import scenes
    from .solver import DeviceScene, GpuGeometry
    geo = geometry or GpuGeometry(device=device)
    out = []
    for i, n in enumerate(node_counts):
        spec = scenes.spec_for_nodes(int(n), scenes.config_spec(4))
        sc = scenes.make_scene(spec, geo, seed=1_000_003 * 4 + i + 1000 * seed)
        ds = DeviceScene.from_scene(sc, device=device)
        out.append(FrameStream(sc, ds, frames=frames, max_rot_deg=max_rot_deg, max_trans=max_trans, seed=seed + i,
                               device=device))
    return out


def run_streams(server: Server, streams: List[FrameStream], requests: int, period_ms: float = 33.0,
                jitter_ms: float = 5.0, seed: int = 0, lone: bool = True) -> dict:
    """Frames arrive per stream every period_ms + Exp(jitter_ms); each is submitted at its
    arrival time and solved by the server.  Returns solves/s over the run and latency
    percentiles (submit -> solved).  With `lone`, each stream's frame 0 is first solved alone
    on the idle server (twice; the second latency counts) and its warp restored, which gives
    every request a lone-solve latency of its own scene to be compared with."""
    rng = np.random.default_rng(seed)
    ids = [server.add_scene(s.ds) for s in streams]
    lone_ms = None
    if lone:
        lone_ms = []
        for sid, s in zip(ids, streams):
            start = server.warp(sid).clone()
            fr = s.frame(0)
            t = 0.0
            for _ in range(2):
                server.set_warp(sid, start)
                rid = server.submit(sid, fr.measure_vertex, fr.measure_normal, s.ds.reference_vertex,
                                    s.ds.reference_normal, s.ds.index_map)
                t = server.wait(rid)["latency_ms"]
                server.forget(rid)
            server.set_warp(sid, start)
            lone_ms.append(t)
    heap = [(float(rng.exponential(jitter_ms)) + i * period_ms / len(streams), i, 0) for i in range(len(streams))]
    heapq.heapify(heap)
    submitted = []
    t0 = time.perf_counter()
    while len(submitted) < requests:
        t_arr, i, k = heapq.heappop(heap)
        now = (time.perf_counter() - t0) * 1e3
        if t_arr > now:
            time.sleep((t_arr - now) / 1e3)
        s = streams[i]
        fr = s.frame(k)
        rid = server.submit(ids[i], fr.measure_vertex, fr.measure_normal, s.ds.reference_vertex,
                            s.ds.reference_normal, s.ds.index_map)
        submitted.append((rid, i))
        heapq.heappush(heap, (t_arr + period_ms + float(rng.exponential(jitter_ms)), i, k + 1))
    infos = [server.wait(r) for r, _ in submitted]
    t1 = time.perf_counter()
    for r, _ in submitted:
        server.forget(r)
    lat = np.array([x["latency_ms"] for x in infos])
    ok = sum(1 for x in infos if x["status"] == WS_OK)
    st = server.stats()
    for sid in ids:
        server.remove_scene(sid)
    out = {"requests": len(infos), "solved": ok, "wall_s": t1 - t0, "solves_per_s": ok / (t1 - t0),
           "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
           "mean_ms": float(lat.mean()), "mean_batch_scenes": st["mean_batch_scenes"], "batches": st["batches"],
           "executor_bytes": st["executor_bytes"], "resident_bytes": st["resident_bytes"]}
    if lone_ms is not None:
        ratio = lat / np.array([lone_ms[i] for _, i in submitted])
        out.update({"lone_p50_ms": float(np.percentile(lone_ms, 50)), "lone_p99_ms": float(np.percentile(lone_ms, 99)),
                    "latency_over_lone_p50": float(np.percentile(ratio, 50)),
                    "latency_over_lone_p99": float(np.percentile(ratio, 99))})
    return out


def main():
    import argparse
    import json
    p = argparse.ArgumentParser(description="Serving load: frame streams against the continuous-batching server")
    p.add_argument("--streams", type=int, default=32)
    p.add_argument("--requests", type=int, default=10_000)
    p.add_argument("--min-nodes", type=int, default=1000)
    p.add_argument("--max-nodes", type=int, default=16000)
    p.add_argument("--budget-gb", type=float, default=40.0)
    p.add_argument("--executors", type=int, default=3)
    p.add_argument("--frames", type=int, default=8)
    p.add_argument("--seed", type=int, default=4)
    a = p.parse_args()
    rng = np.random.default_rng(a.seed)
    counts = np.exp(rng.uniform(np.log(a.min_nodes), np.log(a.max_nodes), a.streams)).astype(int)
    streams = build_streams(counts, frames=a.frames, seed=a.seed)
    with Server(memory_budget=int(a.budget_gb * 1e9), executors=a.executors,
                max_batch_scenes=a.streams, max_batch_nodes=int(counts.sum()) + 1024,
                max_batch_pixels=a.streams * 640 * 480,
                max_batch_edges=int(sum(s.ds.num_edges for s in streams)) + 1024) as srv:
        out = run_streams(srv, streams, a.requests, seed=a.seed)
    out["streams"] = a.streams
    out["node_counts"] = [int(c) for c in counts]
    print(json.dumps(out))


if __name__ == "__main__":
    main()
