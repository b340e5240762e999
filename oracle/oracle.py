"""ctypes wrapper of the CPU oracle (oracle/warp_oracle.cpp) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker / the timed CPU restatement of the reference.
Parity status: parity unpinned (see oracle.h).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

ORC_PREC_FP64 = 0
ORC_PREC_FP32_REFERENCE = 1
ORC_PREC_MIXED = 2


def build() -> Path:
    """Compiles the oracle with its Makefile (g++ -O3 -fopenmp)."""
    r = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


class OrcProblem(C.Structure):
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int),
        ("fx", C.c_float), ("fy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
        ("world2cam", C.c_float * 12),
        ("measure_vertex", C.c_void_p), ("measure_normal", C.c_void_p),
        ("ref_vertex", C.c_void_p), ("ref_normal", C.c_void_p),
        ("index_map", C.c_void_p), ("flow", C.c_void_p),
        ("num_surfels", C.c_int), ("surfel_knn", C.c_void_p), ("surfel_sw", C.c_void_p),
        ("surfel_cw", C.c_void_p),
        ("num_nodes", C.c_int), ("node_coords", C.c_void_p), ("graph_k", C.c_int),
        ("num_edges", C.c_int), ("edges", C.c_void_p), ("node_cw", C.c_void_p),
        ("node_radius_square", C.c_float), ("node_motion_pred", C.c_void_p),
        ("num_features", C.c_int), ("feature_knn", C.c_void_p), ("init_dq", C.c_void_p),
    ]


class OrcSettings(C.Structure):
    _fields_ = [
        ("gn_iters", C.c_int), ("pcg_iters", C.c_int),
        ("lambda_depth", C.c_float), ("lambda_of", C.c_float), ("lambda_reg", C.c_float),
        ("lambda_node", C.c_float), ("lambda_feature", C.c_float),
        ("precision", C.c_int), ("threads", C.c_int),
    ]


class OrcDebug(C.Structure):
    _fields_ = [
        ("capacity_terms", C.c_int), ("capacity_pairs", C.c_int),
        ("num_dense_terms", C.c_int), ("num_sym_pairs", C.c_int),
        ("dense_residual", C.c_void_p), ("dense_gradient", C.c_void_p),
        ("diag_blocks", C.c_void_p), ("inv_diag_blocks", C.c_void_p), ("jtr", C.c_void_p),
        ("sym_rows", C.c_void_p), ("sym_cols", C.c_void_p), ("offdiag_blocks", C.c_void_p),
        ("pcg_x", C.c_void_p),
    ]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _c(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


def _i():
    return C.c_int(0)


class OracleGeometry:
    """Node construction, node graph and skinning restated on the CPU."""

    def __init__(self, threads: int = 0):
        self.threads = threads

    def init_nodes(self, surfels, node_radius):
        s = _c(surfels, np.float32)
        cap = s.shape[0] + 2
        out = np.zeros((cap, 4), np.float32)
        n = _i()
        st = lib().orc_init_nodes(_p(s), C.c_int(s.shape[0]), C.c_float(node_radius), _p(out), C.c_int(cap),
                                  C.byref(n))
        if st != 0:
            raise RuntimeError(f"orc_init_nodes failed: {st}")
        return out[: n.value].copy()

    def voxel_subsample(self, pts, voxel):
        p = _c(pts, np.float32)
        out = np.zeros((p.shape[0], 4), np.float32)
        n = _i()
        st = lib().orc_voxel_subsample(_p(p), C.c_int(p.shape[0]), C.c_float(voxel), _p(out), C.c_int(p.shape[0]),
                                       C.byref(n))
        if st != 0:
            raise RuntimeError(f"orc_voxel_subsample failed: {st}")
        return out[: n.value].copy()

    def node_graph(self, nodes, k, node_radius):
        nd = _c(nodes, np.float32)
        n = nd.shape[0]
        knn = np.zeros((n, k), np.uint16)
        w = np.zeros((n, k), np.float32)
        st = lib().orc_node_graph(_p(nd), C.c_int(n), C.c_int(k), C.c_float(node_radius), _p(knn), _p(w))
        if st != 0:
            raise RuntimeError(f"orc_node_graph failed: {st}")
        edges = np.zeros((n * k, 3), np.uint16)
        edges[:, 0] = np.repeat(np.arange(n, dtype=np.uint16), k)
        edges[:, 1] = knn.reshape(-1)
        edges[:, 2] = np.tile(np.arange(k, dtype=np.uint16), n)
        return knn, w, edges

    def node_graph_ex(self, nodes, k, node_radius, status=None, normalize=True):
        """orc_node_graph_ex: knn, weights and edges with node status and optional normalisation."""
        nd = _c(nodes, np.float32)
        n = nd.shape[0]
        stt = _c(status, np.uint32) if status is not None else None
        knn = np.zeros((n, k), np.uint16)
        w = np.zeros((n, k), np.float32)
        st = lib().orc_node_graph_ex(_p(nd), _p(stt), C.c_int(n), C.c_int(k), C.c_float(node_radius),
                                     C.c_int(1 if normalize else 0), _p(knn), _p(w))
        if st != 0:
            raise RuntimeError(f"orc_node_graph_ex failed: {st}")
        edges = np.zeros((n * k, 3), np.uint16)
        edges[:, 0] = np.repeat(np.arange(n, dtype=np.uint16), k)
        edges[:, 1] = knn.reshape(-1)
        edges[:, 2] = np.tile(np.arange(k, dtype=np.uint16), n)
        return knn, w, edges

    def skinning_ex(self, nodes, verts, node_radius, status=None, normalize=True, prev_nodes=0, first_vert=0,
                    knn=None):
        """orc_skinning_ex: full skinning, or with prev_nodes > 0 the incremental form that starts surfels
        first_vert.. from `knn` (their current neighbours) and takes the nodes prev_nodes.."""
        nd = _c(nodes, np.float32)
        v = _c(verts, np.float32)
        stt = _c(status, np.uint32) if status is not None else None
        out_knn = np.zeros((v.shape[0], 4), np.uint16) if knn is None else np.array(knn, np.uint16, copy=True)
        sw = np.zeros((v.shape[0], 4), np.float32)
        cw = np.zeros((v.shape[0], 4), np.float32)
        st = lib().orc_skinning_ex(_p(nd), _p(stt), C.c_int(nd.shape[0]), C.c_int(prev_nodes), _p(v),
                                   C.c_int(first_vert), C.c_int(v.shape[0]), C.c_float(node_radius),
                                   C.c_int(1 if normalize else 0), _p(out_knn), _p(sw), _p(cw), C.c_int(self.threads))
        if st != 0:
            raise RuntimeError(f"orc_skinning_ex failed: {st}")
        return out_knn, sw, cw

    def skinning(self, nodes, verts, node_radius):
        nd = _c(nodes, np.float32)
        v = _c(verts, np.float32)
        knn = np.zeros((v.shape[0], 4), np.uint16)
        sw = np.zeros((v.shape[0], 4), np.float32)
        cw = np.zeros((v.shape[0], 4), np.float32)
        lib().orc_skinning(_p(nd), C.c_int(nd.shape[0]), _p(v), C.c_int(v.shape[0]), C.c_float(node_radius),
                           _p(knn), _p(sw), _p(cw), C.c_int(self.threads))
        return knn, sw, cw


def problem_from_scene(scene, keep):
    """Builds an OrcProblem; `keep` collects the arrays that must outlive the call."""
    cam = scene.camera
    c2w = np.asarray(cam.cam2world, np.float64)
    R = c2w[:3, :3].T
    t = -R @ c2w[:3, 3]
    w2c = np.concatenate([R, t[:, None]], 1).astype(np.float32).reshape(-1)
    arrs = dict(
        mv=_c(scene.meas_vertex, np.float32), mn=_c(scene.meas_normal, np.float32),
        rv=_c(scene.ref_vertex, np.float32), rn=_c(scene.ref_normal, np.float32),
        idx=_c(scene.index_map, np.uint32), flow=_c(scene.flow, np.float32),
        sknn=_c(scene.surfel_knn, np.uint16), ssw=_c(scene.surfel_sw, np.float32),
        scw=_c(scene.surfel_cw, np.float32), nodes=_c(scene.nodes, np.float32),
        edges=_c(scene.edges, np.uint16), ncw=_c(scene.node_cw, np.float32),
    )
    keep.update(arrs)
    p = OrcProblem()
    p.width, p.height = cam.width, cam.height
    p.fx, p.fy, p.cx, p.cy = cam.fx, cam.fy, cam.cx, cam.cy
    p.world2cam[:] = list(w2c)
    p.measure_vertex, p.measure_normal = _p(arrs["mv"]), _p(arrs["mn"])
    p.ref_vertex, p.ref_normal = _p(arrs["rv"]), _p(arrs["rn"])
    p.index_map, p.flow = _p(arrs["idx"]), _p(arrs["flow"])
    p.num_surfels = scene.surfel_vertex.shape[0]
    p.surfel_knn, p.surfel_sw, p.surfel_cw = _p(arrs["sknn"]), _p(arrs["ssw"]), _p(arrs["scw"])
    p.num_nodes = scene.nodes.shape[0]
    p.node_coords = _p(arrs["nodes"])
    p.graph_k = scene.graph_k
    p.num_edges = scene.edges.shape[0]
    p.edges = _p(arrs["edges"])
    p.node_cw = _p(arrs["ncw"])
    p.node_radius_square = float(np.float32(scene.node_radius) * np.float32(scene.node_radius))
    pred = getattr(scene, "node_motion_pred", None)
    feat = getattr(scene, "feature_knn", None)
    if pred is not None:
        keep["pred"] = _c(pred, np.float32)
    if feat is not None:
        keep["feat"] = _c(feat, np.uint16)
    p.node_motion_pred = _p(keep["pred"]) if pred is not None else None
    p.num_features = 0 if feat is None else int(feat.shape[0])
    p.feature_knn = _p(keep["feat"]) if feat is not None else None
    p.init_dq = None
    return p


def solve(scene, precision=ORC_PREC_FP64, gn_iters=None, pcg_iters=None, threads=0, debug=False,
          lambda_reg=None, init_dq=None):
    """Runs the CPU restatement of the full solve (index build + GN loop)."""
    keep = {}
    p = problem_from_scene(scene, keep)
    if init_dq is not None:
        keep["init"] = _c(init_dq, np.float32)
        p.init_dq = _p(keep["init"])
    s = OrcSettings()
    s.gn_iters = scene.gn_iters if gn_iters is None else gn_iters
    s.pcg_iters = scene.pcg_iters if pcg_iters is None else pcg_iters
    s.lambda_depth, s.lambda_of = scene.lambda_depth, scene.lambda_of
    s.lambda_reg = scene.lambda_reg if lambda_reg is None else lambda_reg
    s.lambda_node, s.lambda_feature = scene.lambda_node, scene.lambda_feature
    s.precision, s.threads = precision, threads
    out = np.zeros((scene.nodes.shape[0], 8), np.float32)
    dbg_ptr = None
    dbg = None
    if debug:
        n = scene.nodes.shape[0]
        cap_t = scene.camera.width * scene.camera.height
        cap_p = 64 * n
        bufs = dict(res=np.zeros((cap_t, 3), np.float32), grad=np.zeros((cap_t, 18), np.float32),
                    diag=np.zeros((n, 36), np.float32), inv=np.zeros((n, 36), np.float32),
                    jtr=np.zeros((n, 6), np.float32), rows=np.zeros(cap_p, np.uint32),
                    cols=np.zeros(cap_p, np.uint32), off=np.zeros((cap_p, 36), np.float32),
                    x=np.zeros((n, 6), np.float32))
        keep.update(bufs)
        dbg = OrcDebug()
        dbg.capacity_terms, dbg.capacity_pairs = cap_t, cap_p
        dbg.dense_residual, dbg.dense_gradient = _p(bufs["res"]), _p(bufs["grad"])
        dbg.diag_blocks, dbg.inv_diag_blocks, dbg.jtr = _p(bufs["diag"]), _p(bufs["inv"]), _p(bufs["jtr"])
        dbg.sym_rows, dbg.sym_cols, dbg.offdiag_blocks = _p(bufs["rows"]), _p(bufs["cols"]), _p(bufs["off"])
        dbg.pcg_x = _p(bufs["x"])
        dbg_ptr = C.byref(dbg)
    st = lib().orc_solve(C.byref(p), C.byref(s), _p(out), dbg_ptr)
    if st != 0:
        raise RuntimeError(f"orc_solve failed: {st}")
    if not debug:
        return out
    nd, ns = dbg.num_dense_terms, dbg.num_sym_pairs
    b = keep
    info = dict(num_dense=nd, residual=b["res"][:nd].copy(), gradient=b["grad"][:nd].copy(),
                diag=b["diag"].copy(), inv_diag=b["inv"].copy(), jtr=b["jtr"].copy(),
                sym_rows=b["rows"][:ns].copy(), sym_cols=b["cols"][:ns].copy(),
                offdiag=b["off"][:ns].copy(), step=b["x"].copy())
    return out, info


def compact_pixels(scene):
    cam = scene.camera
    cap = cam.width * cam.height
    pix = np.zeros((cap, 4), np.uint16)
    knn = np.zeros((cap, 4), np.uint16)
    sw = np.zeros((cap, 4), np.float32)
    cw = np.zeros((cap, 4), np.float32)
    n = _i()
    idx = _c(scene.index_map, np.uint32)
    flow = _c(scene.flow, np.float32)
    st = lib().orc_compact_pixels(C.c_int(cam.width), C.c_int(cam.height), _p(idx), _p(flow),
                                  _p(_c(scene.surfel_knn, np.uint16)), _p(_c(scene.surfel_sw, np.float32)),
                                  _p(_c(scene.surfel_cw, np.float32)), _p(pix), _p(knn), _p(sw), _p(cw),
                                  C.c_int(cap), C.byref(n))
    if st != 0:
        raise RuntimeError(f"orc_compact_pixels failed: {st}")
    k = n.value
    return pix[:k], knn[:k], sw[:k], cw[:k]


def node2term(dense_knn, edges, n_nodes, feat_knn=None):
    dk = _c(dense_knn, np.uint16)
    ed = _c(edges, np.uint16)
    fk = _c(feat_knn, np.uint16) if feat_knn is not None else None
    nd, ne = dk.shape[0], ed.shape[0]
    nf = 0 if fk is None else fk.shape[0]
    cap = 4 * nd + 2 * ne + n_nodes + 4 * nf
    off = np.zeros(n_nodes + 1, np.uint32)
    ti = np.zeros(max(cap, 1), np.uint32)
    n = _i()
    st = lib().orc_node2term(C.c_int(nd), _p(dk), C.c_int(ne), _p(ed), C.c_int(n_nodes), C.c_int(nf), _p(fk),
                             _p(off), _p(ti), C.c_int(cap), C.byref(n))
    if st != 0:
        raise RuntimeError(f"orc_node2term failed: {st}")
    return off, ti[: n.value]


def nodepair2term(dense_knn, edges, n_nodes, feat_knn=None):
    dk = _c(dense_knn, np.uint16)
    ed = _c(edges, np.uint16)
    fk = _c(feat_knn, np.uint16) if feat_knn is not None else None
    nd, ne = dk.shape[0], ed.shape[0]
    nf = 0 if fk is None else fk.shape[0]
    cap_kv = max(6 * nd + ne + 6 * nf, 1)
    cap_h = cap_kv
    hr, hc, hb, he = (np.zeros(cap_h, np.uint32) for _ in range(4))
    sr, sc, sb, se = (np.zeros(2 * cap_h, np.uint32) for _ in range(4))
    ti = np.zeros(cap_kv, np.uint32)
    bo = np.zeros(n_nodes + 1, np.uint32)
    nh, nk = _i(), _i()
    st = lib().orc_nodepair2term(C.c_int(nd), _p(dk), C.c_int(ne), _p(ed), C.c_int(n_nodes), C.c_int(nf), _p(fk),
                                 _p(hr), _p(hc), _p(hb), _p(he), C.c_int(cap_h), C.byref(nh), _p(ti), C.c_int(cap_kv),
                                 C.byref(nk), _p(sr), _p(sc), _p(sb), _p(se), _p(bo))
    if st != 0:
        raise RuntimeError(f"orc_nodepair2term failed: {st}")
    h = nh.value
    return dict(half_rows=hr[:h], half_cols=hc[:h], half_begin=hb[:h], half_end=he[:h], term_index=ti[: nk.value],
                sym_rows=sr[: 2 * h], sym_cols=sc[: 2 * h], sym_begin=sb[: 2 * h], sym_end=se[: 2 * h],
                blkrow_offset=bo)


def binblock_csr(n_nodes, sym_rows, sym_cols):
    sr = _c(sym_rows, np.uint32)
    scc = _c(sym_cols, np.uint32)
    nbins = (6 * n_nodes + 31) // 32
    cap_rp = 32 * (nbins + 1)
    rp = np.zeros(cap_rp, np.int32)
    n_rp = _i()
    cap_col = 32 * nbins * (1 + len(sr)) + 64
    col = np.zeros(cap_col, np.int32)
    st = lib().orc_binblock_csr(C.c_int(n_nodes), C.c_int(len(sr)), _p(sr), _p(scc), _p(rp), C.c_int(cap_rp),
                                C.byref(n_rp), _p(col), C.c_int(cap_col))
    if st != 0:
        raise RuntimeError(f"orc_binblock_csr failed: {st}")
    return rp[: n_rp.value], col


def render_solver_maps(vertex_confid, normal_radius, color_time, cam, world2camera, max_depth, current_time,
                       conf_threshold=1.0, time_threshold=3.0, footprint=0):
    """orc_render_solver_maps: (index (H, W) uint32, vertex, normal, rgbd (H, W, 4) float32)."""
    vc = _c(vertex_confid, np.float32)
    nr = _c(normal_radius, np.float32)
    ct = _c(color_time, np.float32) if color_time is not None else None
    m = _c(np.asarray(world2camera, np.float32).reshape(16), np.float32)
    h, w = cam.height, cam.width
    idx = np.zeros((h, w), np.uint32)
    vert = np.zeros((h, w, 4), np.float32)
    nrm = np.zeros((h, w, 4), np.float32)
    rgbd = np.zeros((h, w, 4), np.float32)
    rc = lib().orc_render_solver_maps(_p(vc), _p(nr), _p(ct), C.c_int(vc.shape[0]), C.c_int(w), C.c_int(h),
                                      C.c_float(cam.fx), C.c_float(cam.fy), C.c_float(cam.cx), C.c_float(cam.cy),
                                      _p(m), C.c_float(max_depth), C.c_float(current_time),
                                      C.c_float(conf_threshold), C.c_float(time_threshold), C.c_int(footprint),
                                      _p(idx), _p(vert), _p(nrm), _p(rgbd))
    assert rc == 0
    return idx, vert, nrm, rgbd


def render_observation_maps(vertex_confid, normal_radius, color_time, cam, world2camera, max_depth, current_time,
                            conf_threshold=1.0, time_threshold=3.0):
    """orc_render_observation_maps: (index (H, W) uint32, rgbd (H, W, 4) float32)."""
    vc = _c(vertex_confid, np.float32)
    nr = _c(normal_radius, np.float32)
    ct = _c(color_time, np.float32) if color_time is not None else None
    m = _c(np.asarray(world2camera, np.float32).reshape(16), np.float32)
    h, w = cam.height, cam.width
    idx = np.zeros((h, w), np.uint32)
    rgbd = np.zeros((h, w, 4), np.float32)
    rc = lib().orc_render_observation_maps(_p(vc), _p(nr), _p(ct), C.c_int(vc.shape[0]), C.c_int(w), C.c_int(h),
                                           C.c_float(cam.fx), C.c_float(cam.fy), C.c_float(cam.cx),
                                           C.c_float(cam.cy), _p(m), C.c_float(max_depth), C.c_float(current_time),
                                           C.c_float(conf_threshold), C.c_float(time_threshold), _p(idx), _p(rgbd))
    assert rc == 0
    return idx, rgbd


def measure_maps(depth_mm, fx, fy, cx, cy, clip_near=0.1, clip_far=3.0, radius_scale=1.0):
    """orc_measure_maps: vertex and normal/radius maps, two (H, W, 4) float32 arrays."""
    d = _c(depth_mm, np.uint16)
    h, w = d.shape
    vert = np.zeros((h, w, 4), np.float32)
    nrm = np.zeros((h, w, 4), np.float32)
    rc = lib().orc_measure_maps(_p(d), C.c_int(w), C.c_int(h), C.c_float(fx), C.c_float(fy), C.c_float(cx),
                                C.c_float(cy), C.c_float(clip_near), C.c_float(clip_far), C.c_float(radius_scale),
                                _p(vert), _p(nrm))
    assert rc == 0
    return vert, nrm


def forward_warp(dq, verts, knn, sw, cw, threads=0):
    d = _c(dq, np.float32)
    v = _c(verts, np.float32)
    out = np.zeros_like(v)
    lib().orc_forward_warp(_p(d), C.c_int(d.shape[0]), _p(v), C.c_int(v.shape[0]), _p(_c(knn, np.uint16)),
                           _p(_c(sw, np.float32)), _p(_c(cw, np.float32)), _p(out), C.c_int(threads))
    return out
