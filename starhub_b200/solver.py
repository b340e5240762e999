"""Host-side mirror of StarHub's warp-solver interface over the C ABI.

`WarpSolver` keeps the reference's method names and meaning
(examples/mono_star/opt/WarpSolver.h:34-52): `SetSolverInputs` takes one
frame's inputs, `SolveStreamed` runs the Gauss-Newton solve on a CUDA stream,
`SolvedNodeSE3` returns the node dual quaternions.  Device memory, streams and
the upload of numpy inputs use PyTorch (plumbing only); every computation runs
in libwarpsolve.so.  Errors raise `WarpSolveError` with the C status instead of
aborting the process (the reference's STAR_CHECK / exit(-1)).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import WS_PREC_FP32, WS_PREC_MIXED, WsConfig, WsInputs, check


def _dev(a, device, dtype=None):
    if a is None:
        return None
    if isinstance(a, torch.Tensor):
        t = a.to(device=device)
    else:
        t = torch.from_numpy(np.ascontiguousarray(a)).to(device=device)
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    return t.contiguous()


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


@dataclass
class DeviceScene:
    """One scene's solver inputs resident on the GPU (torch tensors).

    Field meaning follows Measure4Solver / Render4Solver / OpticalFlow4Solver
    (libs/star/opt/solver_types.h:21-89), Geometry4Solver and NodeGraph4Solver.
    """
    width: int
    height: int
    fx: float
    fy: float
    cx: float
    cy: float
    cam2world: np.ndarray
    measure_vertex: torch.Tensor
    measure_normal: torch.Tensor
    reference_vertex: torch.Tensor
    reference_normal: torch.Tensor
    index_map: torch.Tensor
    flow: Optional[torch.Tensor]
    surfel_knn: torch.Tensor
    surfel_sw: torch.Tensor
    surfel_cw: torch.Tensor
    nodes: torch.Tensor
    edges: torch.Tensor
    graph_k: int
    node_cw: torch.Tensor
    node_radius_square: float
    node_motion_pred: Optional[torch.Tensor] = None
    feature_knn: Optional[torch.Tensor] = None
    init_se3: Optional[torch.Tensor] = None
    lambda_depth: float = 0.1
    lambda_of: float = 0.0
    lambda_reg: float = 1.0
    lambda_node: float = 0.0
    lambda_feature: float = 1.0

    @property
    def num_nodes(self) -> int:
        return int(self.nodes.shape[0])

    @property
    def num_pixels(self) -> int:
        return int(self.width * self.height)

    @property
    def num_edges(self) -> int:
        return int(self.edges.shape[0])

    @staticmethod
    def from_scene(scene, device="cuda", lambda_reg=None) -> "DeviceScene":
        cam = scene.camera
        return DeviceScene(
            width=cam.width, height=cam.height, fx=cam.fx, fy=cam.fy, cx=cam.cx, cy=cam.cy,
            cam2world=np.asarray(cam.cam2world, np.float32),
            measure_vertex=_dev(scene.meas_vertex, device, torch.float32),
            measure_normal=_dev(scene.meas_normal, device, torch.float32),
            reference_vertex=_dev(scene.ref_vertex, device, torch.float32),
            reference_normal=_dev(scene.ref_normal, device, torch.float32),
            index_map=_dev(scene.index_map.view(np.int32), device, torch.int32),
            flow=_dev(scene.flow, device, torch.float32),
            surfel_knn=_dev(scene.surfel_knn.view(np.int16), device, torch.int16),
            surfel_sw=_dev(scene.surfel_sw, device, torch.float32),
            surfel_cw=_dev(scene.surfel_cw, device, torch.float32),
            nodes=_dev(scene.nodes, device, torch.float32),
            edges=_dev(scene.edges.view(np.int16), device, torch.int16),
            graph_k=int(scene.graph_k),
            node_cw=_dev(scene.node_cw, device, torch.float32),
            node_radius_square=float(np.float32(scene.node_radius) * np.float32(scene.node_radius)),
            lambda_depth=scene.lambda_depth, lambda_of=scene.lambda_of,
            lambda_reg=scene.lambda_reg if lambda_reg is None else lambda_reg,
            lambda_node=scene.lambda_node, lambda_feature=scene.lambda_feature,
            node_motion_pred=_dev(getattr(scene, "node_motion_pred", None), device, torch.float32),
            feature_knn=(None if getattr(scene, "feature_knn", None) is None
                         else _dev(np.ascontiguousarray(scene.feature_knn).view(np.int16), device, torch.int16)),
        )

    def to_inputs(self) -> WsInputs:
        s = WsInputs()
        s.width, s.height, s.pitch = self.width, self.height, 0
        s.fx, s.fy, s.cx, s.cy = self.fx, self.fy, self.cx, self.cy
        s.cam2world[:] = [float(v) for v in np.asarray(self.cam2world, np.float32).reshape(-1)]
        s.measure_vertex_confid = _ptr(self.measure_vertex)
        s.measure_normal_radius = _ptr(self.measure_normal)
        s.reference_vertex = _ptr(self.reference_vertex)
        s.reference_normal = _ptr(self.reference_normal)
        s.index_map = _ptr(self.index_map)
        s.opticalflow = _ptr(self.flow)
        s.num_surfels = int(self.surfel_knn.shape[0])
        s.surfel_knn = _ptr(self.surfel_knn)
        s.surfel_knn_spatial_weight = _ptr(self.surfel_sw)
        s.surfel_knn_connect_weight = _ptr(self.surfel_cw)
        s.num_nodes = self.num_nodes
        s.reference_node_coords = _ptr(self.nodes)
        s.num_edges = self.num_edges
        s.node_graph = _ptr(self.edges)
        s.graph_k = self.graph_k
        s.node_knn_connect_weight = _ptr(self.node_cw)
        s.node_radius_square = self.node_radius_square
        s.node_motion_pred = _ptr(self.node_motion_pred)
        s.num_features = 0 if self.feature_knn is None else int(self.feature_knn.shape[0])
        s.feature_knn = _ptr(self.feature_knn)
        s.lambda_depth, s.lambda_optical_flow = self.lambda_depth, self.lambda_of
        s.lambda_reg, s.lambda_node_translation, s.lambda_feature = self.lambda_reg, self.lambda_node, self.lambda_feature
        s.init_node_se3 = _ptr(self.init_se3)
        return s


def _stream_ptr(stream) -> Optional[C.c_void_p]:
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class WarpSolver:
    """One solver object: capacity fixed at construction, like the reference's
    preallocated WarpSolver (examples/mono_star/opt/WarpSolver.cu:50-103)."""

    def __init__(self, max_nodes: int, max_pixels: int, max_edges: int = None, max_scenes: int = 1,
                 max_features: int = 0, precision: int = WS_PREC_MIXED, device: int = 0):
        lib = _lib.load()
        cfg = WsConfig()
        cfg.max_scenes = max_scenes
        cfg.max_total_nodes = max_nodes
        cfg.max_total_pixels = max_pixels
        cfg.max_total_edges = 8 * max_nodes if max_edges is None else max_edges
        cfg.max_total_features = max_features
        cfg.precision = precision
        cfg.device = device
        h = C.c_void_p()
        check(lib.ws_create(C.byref(cfg), C.byref(h)), "ws_create")
        self._lib = lib
        self._h = h
        self._scenes: List[DeviceScene] = []
        self._inputs = None
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ws_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference interface -------------------------------------------------
    def SetSolverInputs(self, scene: DeviceScene) -> None:
        """WarpSolver::SetSolverInputs (WarpSolver.cu:125-155) for one scene."""
        self.SetBatchInputs([scene])

    def SetBatchInputs(self, scenes: Sequence[DeviceScene]) -> None:
        arr = (WsInputs * len(scenes))(*[s.to_inputs() for s in scenes])
        check(self._lib.ws_set_batch(self._h, arr, len(scenes)), "ws_set_batch")
        self._scenes = list(scenes)
        self._inputs = arr

    def SolveStreamed(self, gn_iters: int = 6, pcg_iters: int = 10, stream=None, graph: bool = False) -> None:
        """WarpSolver::SolveStreamed (WarpSolver.cu:260-279); asynchronous on `stream`."""
        fn = self._lib.ws_solve_graph if graph else self._lib.ws_solve
        check(fn(self._h, gn_iters, pcg_iters, _stream_ptr(stream)), "ws_solve")

    def Sync(self) -> None:
        check(self._lib.ws_sync_status(self._h), "device status")

    def SolvedNodeSE3(self, scene: int = 0) -> torch.Tensor:
        """Device view (N, 8) of the solved node dual quaternions of `scene`."""
        p = C.c_void_p()
        n = C.c_int()
        check(self._lib.ws_get_solution(self._h, scene, C.byref(p), C.byref(n)), "ws_get_solution")
        return _wrap_device_floats(p.value, n.value * 8, self.device).view(n.value, 8)

    def spmv(self, x: torch.Tensor, y: torch.Tensor, stream=None) -> None:
        """y = A x with the last assembled block matrix (x, y: (total_nodes, 8) float32 CUDA)."""
        check(self._lib.ws_spmv(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), _stream_ptr(stream)),
              "ws_spmv")

    def spmv_matrix_free(self, x: torch.Tensor, y: torch.Tensor, stream=None) -> None:
        """y = A x applied from the term records (no assembled blocks)."""
        check(self._lib.ws_spmv_matrix_free(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                            _stream_ptr(stream)), "ws_spmv_matrix_free")

    def autotune(self, pcg_iters: int = 20, stream=None) -> dict:
        """Times the launch-shape candidates on the inputs set and keeps the fastest (ws_autotune)."""
        from ._lib import WsTuning
        t = WsTuning()
        check(self._lib.ws_autotune(self._h, pcg_iters, _stream_ptr(stream), C.byref(t)), "ws_autotune")
        return {"node_threads": t.node_threads, "pair_threads": t.pair_threads,
                "pcg_blocks_per_sm": t.pcg_blocks_per_sm, "node_ms": list(t.node_ms), "pair_ms": list(t.pair_ms),
                "pcg_ms": list(t.pcg_ms)}

    def set_tuning(self, node_threads: int, pair_threads: int, pcg_blocks_per_sm: int) -> None:
        from ._lib import WsTuning
        t = WsTuning()
        t.node_threads, t.pair_threads, t.pcg_blocks_per_sm = node_threads, pair_threads, pcg_blocks_per_sm
        check(self._lib.ws_set_tuning(self._h, C.byref(t)), "ws_set_tuning")

    # -- measurement ---------------------------------------------------------
    def set_profiling(self, enable: bool) -> None:
        check(self._lib.ws_set_profiling(self._h, 1 if enable else 0), "ws_set_profiling")

    PHASES = ("index", "eval", "assemble_node", "assemble_pair", "pcg")

    def phase_times(self):
        """(ms, launches) per phase of the last profiled solve (CUDA events on the solve stream)."""
        ms = (C.c_float * 5)()
        ln = (C.c_int * 5)()
        n = C.c_int()
        check(self._lib.ws_get_phase_times(self._h, ms, ln, 5, C.byref(n)), "ws_get_phase_times")
        return dict(zip(self.PHASES, list(ms))), dict(zip(self.PHASES, list(ln)))

    def graph_kernels(self) -> int:
        n = C.c_int()
        check(self._lib.ws_graph_kernel_count(self._h, C.byref(n)), "ws_graph_kernel_count")
        return n.value

    def counts(self, scene=0):
        nd, nh, nkv = C.c_int(), C.c_int(), C.c_int()
        check(self._lib.ws_get_counts(self._h, scene, C.byref(nd), C.byref(nh), C.byref(nkv)), "ws_get_counts")
        return dict(dense_terms=nd.value, half_pairs=nh.value, n2t_kv=nkv.value)

    # -- index / system copies for parity tests ------------------------------
    def dense_terms(self, scene=0):
        cap = self._scenes[scene].num_pixels
        pix = np.zeros((cap, 4), np.uint16); knn = np.zeros((cap, 4), np.uint16)
        sw = np.zeros((cap, 4), np.float32); cw = np.zeros((cap, 4), np.float32)
        n = C.c_int()
        check(self._lib.ws_get_dense_terms(self._h, scene, pix.ctypes.data, knn.ctypes.data, sw.ctypes.data,
                                           cw.ctypes.data, cap, C.byref(n)), "ws_get_dense_terms")
        k = n.value
        return pix[:k], knn[:k], sw[:k], cw[:k]

    def dense_jacobian(self, scene=0):
        cap = self._scenes[scene].num_pixels
        res = np.zeros((cap, 3), np.float32); grad = np.zeros((cap, 18), np.float32)
        n = C.c_int()
        check(self._lib.ws_get_dense_jacobian(self._h, scene, res.ctypes.data, grad.ctypes.data, cap, C.byref(n)),
              "ws_get_dense_jacobian")
        return res[: n.value], grad[: n.value]

    def node2term(self, scene=0):
        sc = self._scenes[scene]
        nf = 0 if sc.feature_knn is None else int(sc.feature_knn.shape[0])
        cap = 4 * sc.num_pixels + 2 * sc.num_edges + sc.num_nodes + 4 * nf + 64
        off = np.zeros(sc.num_nodes + 1, np.uint32); ti = np.zeros(cap, np.uint32)
        n = C.c_int()
        check(self._lib.ws_get_node2term(self._h, scene, off.ctypes.data, ti.ctypes.data, cap, C.byref(n)),
              "ws_get_node2term")
        return off, ti[: n.value]

    def node_pairs(self, scene=0):
        sc = self._scenes[scene]
        nf = 0 if sc.feature_knn is None else int(sc.feature_knn.shape[0])
        cap = 6 * sc.num_pixels + sc.num_edges + 6 * nf + 64
        rows, cols, b, e = (np.zeros(cap, np.uint32) for _ in range(4))
        ti = np.zeros(cap, np.uint32)
        n, nt = C.c_int(), C.c_int()
        check(self._lib.ws_get_node_pairs(self._h, scene, rows.ctypes.data, cols.ctypes.data, b.ctypes.data,
                                          e.ctypes.data, cap, C.byref(n), ti.ctypes.data, cap, C.byref(nt)),
              "ws_get_node_pairs")
        k = n.value
        return dict(rows=rows[:k], cols=cols[:k], begin=b[:k], end=e[:k], term_index=ti[: nt.value])

    def system(self, scene=0):
        sc = self._scenes[scene]
        n = sc.num_nodes
        cap = n + 2 * 64 * n
        rp = np.zeros(n + 1, np.uint32); cols = np.zeros(cap, np.uint32); blocks = np.zeros((cap, 36), np.float32)
        inv = np.zeros((n, 36), np.float32); jtr = np.zeros((n, 6), np.float32); x = np.zeros((n, 6), np.float32)
        nb = C.c_int()
        check(self._lib.ws_get_system(self._h, scene, rp.ctypes.data, cols.ctypes.data, blocks.ctypes.data, cap,
                                      C.byref(nb), inv.ctypes.data, jtr.ctypes.data, x.ctypes.data), "ws_get_system")
        k = nb.value
        return dict(rowptr=rp, cols=cols[:k], blocks=blocks[:k], inv_diag=inv, jtr=jtr, step=x)


def _wrap_device_floats(ptr: int, count: int, device: int) -> torch.Tensor:
    """Zero-copy torch view of `count` float32 at device address `ptr` (owned by the solver)."""
    class _Holder:
        pass
    h = _Holder()
    h.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f4", "data": (ptr, False), "version": 3,
                                  "strides": None}
    return torch.as_tensor(h, device=f"cuda:{device}")


class GpuGeometry:
    """Node construction, node graph, skinning, forward warp and map splat on the GPU
    (ws_init_nodes, ws_expand_nodes, ws_build_node_graph, ws_skinning, ws_forward_warp, ws_splat_maps)."""

    def __init__(self, device="cuda"):
        self.lib = _lib.load()
        self.device = device

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def init_nodes(self, surfels, node_radius):
        s = _dev(surfels, self.device, torch.float32)
        cap = int(s.shape[0]) + 2
        out = np.zeros((cap, 4), np.float32)
        n = C.c_int()
        check(self.lib.ws_init_nodes(_ptr(s), int(s.shape[0]), float(node_radius), out.ctypes.data, cap, C.byref(n),
                                     self._stream()), "ws_init_nodes")
        return out[: n.value].copy()

    def expand_nodes(self, reference_nodes, live_nodes, num_nodes, vertices, node_radius, node_time=None,
                     current_time=0):
        """Appends nodes grown from `vertices` (NodeGraph::NaiveExpandNodeGraphFromVertexUnsupported,
        NodeGraph.cu:500-532) to device arrays of capacity rows; returns the new node count."""
        v = _dev(vertices, self.device, torch.float32)
        n = C.c_int(int(num_nodes))
        cap = int(reference_nodes.shape[0])
        live = _ptr(live_nodes) if live_nodes is not None else None
        times = _ptr(node_time) if node_time is not None else None
        check(self.lib.ws_expand_nodes(_ptr(v), int(v.shape[0]), float(node_radius), _ptr(reference_nodes), live, times,
                                       int(current_time), cap, C.byref(n), self._stream()), "ws_expand_nodes")
        return n.value

    def node_graph(self, nodes, k, node_radius):
        nd = _dev(nodes, self.device, torch.float32)
        n = int(nd.shape[0])
        knn = torch.empty((n, k), dtype=torch.int16, device=self.device)
        w = torch.empty((n, k), dtype=torch.float32, device=self.device)
        edges = torch.empty((n * k, 3), dtype=torch.int16, device=self.device)
        check(self.lib.ws_build_node_graph(_ptr(nd), n, k, float(node_radius), _ptr(knn), _ptr(w), _ptr(edges),
                                           self._stream()), "ws_build_node_graph")
        return (knn.cpu().numpy().view(np.uint16), w.cpu().numpy(), edges.cpu().numpy().view(np.uint16))

    def node_graph_ex(self, nodes, k, node_radius, status=None, normalize=True):
        """ws_build_node_graph_ex: knn, weights and edges with a node status and the choice of weights."""
        nd = _dev(nodes, self.device, torch.float32)
        stt = None if status is None else _dev(np.ascontiguousarray(status, np.uint32).view(np.int32), self.device)
        n = int(nd.shape[0])
        knn = torch.empty((n, k), dtype=torch.int16, device=self.device)
        w = torch.empty((n, k), dtype=torch.float32, device=self.device)
        edges = torch.empty((n * k, 3), dtype=torch.int16, device=self.device)
        check(self.lib.ws_build_node_graph_ex(_ptr(nd), _ptr(stt), n, k, float(node_radius), 1 if normalize else 0,
                                              _ptr(knn), _ptr(w), _ptr(edges), self._stream()), "ws_build_node_graph_ex")
        return (knn.cpu().numpy().view(np.uint16), w.cpu().numpy(), edges.cpu().numpy().view(np.uint16))

    def skinning_ex(self, nodes, verts, node_radius, status=None, normalize=True, prev_nodes=0, first_vert=0,
                    knn=None):
        """ws_skinning_ex, or with prev_nodes > 0 ws_skinning_incremental starting surfels first_vert.. from
        `knn`; returns (knn, spatial weights, connect weights) of all surfels (rows before first_vert as given)."""
        nd = _dev(nodes, self.device, torch.float32)
        v = _dev(verts, self.device, torch.float32)
        stt = None if status is None else _dev(np.ascontiguousarray(status, np.uint32).view(np.int32), self.device)
        s = int(v.shape[0])
        if knn is None:
            kt = torch.zeros((s, 4), dtype=torch.int16, device=self.device)
        else:
            kt = _dev(np.ascontiguousarray(knn, np.uint16).view(np.int16), self.device)
        sw = torch.zeros((s, 4), dtype=torch.float32, device=self.device)
        cw = torch.zeros((s, 4), dtype=torch.float32, device=self.device)
        if prev_nodes > 0 or first_vert > 0:
            check(self.lib.ws_skinning_incremental(_ptr(nd), _ptr(stt), int(nd.shape[0]), int(prev_nodes), _ptr(v), s,
                                                   int(first_vert), float(node_radius), 1 if normalize else 0,
                                                   _ptr(kt), _ptr(sw), _ptr(cw), self._stream()),
                  "ws_skinning_incremental")
        else:
            check(self.lib.ws_skinning_ex(_ptr(nd), _ptr(stt), int(nd.shape[0]), _ptr(v), s, float(node_radius),
                                          1 if normalize else 0, _ptr(kt), _ptr(sw), _ptr(cw), self._stream()),
                  "ws_skinning_ex")
        return kt.cpu().numpy().view(np.uint16), sw.cpu().numpy(), cw.cpu().numpy()

    def skinning(self, nodes, verts, node_radius):
        nd = _dev(nodes, self.device, torch.float32)
        v = _dev(verts, self.device, torch.float32)
        s = int(v.shape[0])
        knn = torch.empty((s, 4), dtype=torch.int16, device=self.device)
        sw = torch.empty((s, 4), dtype=torch.float32, device=self.device)
        cw = torch.empty((s, 4), dtype=torch.float32, device=self.device)
        check(self.lib.ws_skinning(_ptr(nd), int(nd.shape[0]), _ptr(v), s, float(node_radius), _ptr(knn), _ptr(sw),
                                   _ptr(cw), self._stream()), "ws_skinning")
        return knn.cpu().numpy().view(np.uint16), sw.cpu().numpy(), cw.cpu().numpy()

    def forward_warp(self, dq, verts, normals, knn, sw, cw):
        d = _dev(dq, self.device, torch.float32)
        v = _dev(verts, self.device, torch.float32)
        nrm = _dev(normals, self.device, torch.float32)
        k = _dev(np.ascontiguousarray(knn).view(np.int16), self.device)
        s = _dev(sw, self.device, torch.float32)
        c = _dev(cw, self.device, torch.float32)
        ov = torch.empty_like(v)
        on = torch.empty_like(nrm) if nrm is not None else None
        check(self.lib.ws_forward_warp(_ptr(d), int(d.shape[0]), _ptr(v), _ptr(nrm), int(v.shape[0]), _ptr(k),
                                       _ptr(s), _ptr(c),
                                       _ptr(ov), _ptr(on), self._stream()), "ws_forward_warp")
        return ov.cpu().numpy(), (on.cpu().numpy() if on is not None else None)

    def measure_maps(self, depth_mm, cam, clip_near=0.1, clip_far=3.0, radius_scale=1.0):
        """Vertex and normal/radius maps of a depth image in millimetres (ws_measure_maps);
        returns two (height, width, 4) float32 arrays."""
        d = _dev(np.ascontiguousarray(depth_mm).view(np.int16), self.device)
        vert = torch.empty((cam.height, cam.width, 4), dtype=torch.float32, device=self.device)
        nrm = torch.empty_like(vert)
        check(self.lib.ws_measure_maps(_ptr(d), cam.width, cam.height, cam.width, cam.fx, cam.fy, cam.cx, cam.cy,
                                       clip_near, clip_far, radius_scale, _ptr(vert), _ptr(nrm), self._stream()),
              "ws_measure_maps")
        return vert.cpu().numpy(), nrm.cpu().numpy()

    def render_solver_maps(self, vertex_confid, normal_radius, color_time, cam, world2camera, max_depth,
                           current_time, conf_threshold=1.0, time_threshold=3.0, footprint=0):
        """ws_render_solver_maps: (index (H, W) uint32, vertex, normal, rgbd (H, W, 4) float32)."""
        from ._lib import WsRenderParams
        vc = _dev(vertex_confid, self.device, torch.float32)
        nr = _dev(normal_radius, self.device, torch.float32)
        ct = _dev(color_time, self.device, torch.float32)
        p = WsRenderParams()
        p.width, p.height = cam.width, cam.height
        p.fx, p.fy, p.cx, p.cy = cam.fx, cam.fy, cam.cx, cam.cy
        p.world2camera[:] = [float(v) for v in np.asarray(world2camera, np.float32).reshape(-1)]
        p.max_depth, p.current_time = max_depth, current_time
        p.confidence_threshold, p.time_threshold, p.footprint = conf_threshold, time_threshold, footprint
        idx = torch.empty((cam.height, cam.width), dtype=torch.int32, device=self.device)
        maps = [torch.empty((cam.height, cam.width, 4), dtype=torch.float32, device=self.device) for _ in range(3)]
        check(self.lib.ws_render_solver_maps(_ptr(vc), _ptr(nr), _ptr(ct), int(vc.shape[0]), C.byref(p), _ptr(idx),
                                             _ptr(maps[0]), _ptr(maps[1]), _ptr(maps[2]), self._stream()),
              "ws_render_solver_maps")
        return (idx.cpu().numpy().view(np.uint32),) + tuple(m.cpu().numpy() for m in maps)

    def render_observation_maps(self, vertex_confid, normal_radius, color_time, cam, world2camera, max_depth,
                                current_time, conf_threshold=1.0, time_threshold=3.0):
        """ws_render_observation_maps: (index (H, W) uint32, rgbd (H, W, 4) float32)."""
        from ._lib import WsRenderParams
        vc = _dev(vertex_confid, self.device, torch.float32)
        nr = _dev(normal_radius, self.device, torch.float32)
        ct = _dev(color_time, self.device, torch.float32)
        p = WsRenderParams()
        p.width, p.height = cam.width, cam.height
        p.fx, p.fy, p.cx, p.cy = cam.fx, cam.fy, cam.cx, cam.cy
        p.world2camera[:] = [float(v) for v in np.asarray(world2camera, np.float32).reshape(-1)]
        p.max_depth, p.current_time = max_depth, current_time
        p.confidence_threshold, p.time_threshold, p.footprint = conf_threshold, time_threshold, 0
        idx = torch.empty((cam.height, cam.width), dtype=torch.int32, device=self.device)
        rgbd = torch.empty((cam.height, cam.width, 4), dtype=torch.float32, device=self.device)
        check(self.lib.ws_render_observation_maps(_ptr(vc), _ptr(nr), _ptr(ct), int(vc.shape[0]), C.byref(p),
                                                  _ptr(idx), _ptr(rgbd), self._stream()),
              "ws_render_observation_maps")
        return idx.cpu().numpy().view(np.uint32), rgbd.cpu().numpy()

    def splat(self, verts, cam, footprint):
        v = _dev(verts, self.device, torch.float32)
        idx = torch.empty((cam.height, cam.width), dtype=torch.int32, device=self.device)
        check(self.lib.ws_splat_maps(_ptr(v), None, None, int(v.shape[0]), cam.width, cam.height, cam.fx, cam.fy,
                                     cam.cx, cam.cy, footprint, _ptr(idx), None, None, self._stream()),
              "ws_splat_maps")
        return idx.cpu().numpy().view(np.uint32)
