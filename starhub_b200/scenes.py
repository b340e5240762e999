"""Seeded synthetic scenes for the warp-field solve (test and benchmark inputs).

A scene is what StarHub's solver consumes for one frame: surfels with their
4-NN skinning, the node graph, the rendered solver maps (index / reference
vertex / reference normal) of the un-warped surfels, and the measurement maps
(vertex / normal) of the surfels warped by a smooth ground-truth node SE(3)
field, with depth noise.  Shapes follow the benchmark configurations:

* torus (R = 0.30 m, r = 0.10 m) 1.0 m in front of a 640x480 pinhole camera
  (fx = fy = 570), tilted 30 degrees about x; nodes voxel-subsampled with node
  radius 2.5 cm; rotation <= 5 deg, translation <= 1 cm; depth noise 1 mm;
* the same torus scaled to a target node count (batched / serving configs);
* a 1280x720 union of torus, sphere (r = 0.2 m) and a bumpy 0.6 x 0.6 m plane
  with optical-flow correspondences on a 4-pixel grid (10 % outliers).

Node construction, node graph and skinning are delegated to a `geometry`
backend (the GPU kernels of libwarpsolve.so via `GpuGeometry`, or any object
with the same four methods); forward warping and the map splat have numpy
implementations here and GPU versions in `GpuGeometry`.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

NODE_RADIUS = 0.025
# Node-graph neighbours per node, self included.  The benchmark configurations build an
# 8-NN graph; the reference ties the graph's K to the skinning K of 4
# (libs/star/geometry/constants.h:6-7), which is the mode its own node graph produces.
BASELINE_GRAPH_K = 8
REFERENCE_GRAPH_K = 4


@dataclass
class Camera:
    width: int
    height: int
    fx: float
    fy: float
    cx: float
    cy: float
    cam2world: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=np.float32))


@dataclass
class Scene:
    camera: Camera
    surfel_vertex: np.ndarray        # (S, 4) float32, w = 1
    surfel_normal: np.ndarray        # (S, 4) float32, w = radius
    nodes: np.ndarray                # (N, 4) float32, w = 1 (two anchors first)
    graph_k: int
    node_knn: np.ndarray             # (N, K) uint16
    node_sw: np.ndarray              # (N, K) float32
    edges: np.ndarray                # (N*K, 3) uint16
    node_cw: np.ndarray              # (N, K) float32
    surfel_knn: np.ndarray           # (S, 4) uint16
    surfel_sw: np.ndarray            # (S, 4) float32
    surfel_cw: np.ndarray            # (S, 4) float32
    gt_dq: np.ndarray                # (N, 8) float32 ground-truth node warp
    index_map: np.ndarray            # (H, W) uint32
    ref_vertex: np.ndarray           # (H, W, 4) float32, world frame
    ref_normal: np.ndarray           # (H, W, 4) float32
    meas_vertex: np.ndarray          # (H, W, 4) float32, camera frame
    meas_normal: np.ndarray          # (H, W, 4) float32
    flow: Optional[np.ndarray]       # (H, W, 2) float32 or None
    node_radius: float = NODE_RADIUS
    lambda_depth: float = 0.1
    lambda_of: float = 0.0
    lambda_reg: float = 1.0
    lambda_node: float = 0.0
    lambda_feature: float = 1.0
    gn_iters: int = 5
    pcg_iters: int = 20
    node_motion_pred: Optional[np.ndarray] = None   # (N, 4) float32: predicted translation, confidence
    feature_knn: Optional[np.ndarray] = None        # (F, 4) uint16: node ids of each feature term

    @property
    def num_nodes(self) -> int:
        return int(self.nodes.shape[0])

    @property
    def num_pixels(self) -> int:
        return int(self.camera.width * self.camera.height)


# ---------------------------------------------------------------------------
# surface sampling
# ---------------------------------------------------------------------------
def rot_x(deg: float) -> np.ndarray:
    a = np.deg2rad(deg)
    c, s = np.cos(a), np.sin(a)
    return np.array([[1, 0, 0], [0, c, -s], [0, s, c]], dtype=np.float64)


def sample_torus(rng, n, R, r):
    """Area-uniform samples on a torus about the z axis: points and outward normals."""
    out_u, out_v = [], []
    need = n
    while need > 0:
        m = int(need * 1.6) + 16
        u = rng.uniform(0, 2 * np.pi, m)
        v = rng.uniform(0, 2 * np.pi, m)
        keep = rng.uniform(0, 1, m) < (R + r * np.cos(v)) / (R + r)
        out_u.append(u[keep]); out_v.append(v[keep])
        need -= int(keep.sum())
    u = np.concatenate(out_u)[:n]; v = np.concatenate(out_v)[:n]
    p = np.stack([(R + r * np.cos(v)) * np.cos(u), (R + r * np.cos(v)) * np.sin(u), r * np.sin(v)], 1)
    nrm = np.stack([np.cos(v) * np.cos(u), np.cos(v) * np.sin(u), np.sin(v)], 1)
    return p, nrm


def sample_sphere(rng, n, radius):
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return radius * d, d


def sample_bumpy_plane(rng, n, size, height_rms, corr):
    """Plane z = h(x, y) over [-size/2, size/2]^2 facing -z; h is a random smooth field."""
    k = 48
    kx = rng.normal(scale=1.0 / corr, size=k)
    ky = rng.normal(scale=1.0 / corr, size=k)
    ph = rng.uniform(0, 2 * np.pi, k)
    amp = np.ones(k) / np.sqrt(k / 2.0) * height_rms
    x = rng.uniform(-size / 2, size / 2, n)
    y = rng.uniform(-size / 2, size / 2, n)
    arg = np.outer(x, kx) + np.outer(y, ky) + ph
    h = (np.sin(arg) * amp).sum(1)
    dhx = (np.cos(arg) * amp * kx).sum(1)
    dhy = (np.cos(arg) * amp * ky).sum(1)
    p = np.stack([x, y, h], 1)
    nrm = np.stack([dhx, dhy, -np.ones(n)], 1)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    return p, nrm


def pack4(p, w):
    out = np.empty((p.shape[0], 4), np.float32)
    out[:, :3] = p
    out[:, 3] = w
    return out


# ---------------------------------------------------------------------------
# ground-truth warp
# ---------------------------------------------------------------------------
def axis_angle_to_R(w):
    th = np.linalg.norm(w, axis=1)
    k = np.where(th[:, None] > 1e-12, w / np.maximum(th, 1e-12)[:, None], 0.0)
    K = np.zeros((w.shape[0], 3, 3))
    K[:, 0, 1], K[:, 0, 2], K[:, 1, 0] = -k[:, 2], k[:, 1], k[:, 2]
    K[:, 1, 2], K[:, 2, 0], K[:, 2, 1] = -k[:, 0], -k[:, 1], k[:, 0]
    s, c = np.sin(th)[:, None, None], np.cos(th)[:, None, None]
    return np.eye(3)[None] + s * K + (1 - c) * (K @ K)


def R_to_quat(R):
    """Rotation matrices to unit quaternions (x, y, z, w) with w >= 0."""
    m = R
    tr = m[:, 0, 0] + m[:, 1, 1] + m[:, 2, 2]
    w = np.sqrt(np.maximum(0.0, 1.0 + tr)) / 2
    x = np.sqrt(np.maximum(0.0, 1.0 + m[:, 0, 0] - m[:, 1, 1] - m[:, 2, 2])) / 2
    y = np.sqrt(np.maximum(0.0, 1.0 - m[:, 0, 0] + m[:, 1, 1] - m[:, 2, 2])) / 2
    z = np.sqrt(np.maximum(0.0, 1.0 - m[:, 0, 0] - m[:, 1, 1] + m[:, 2, 2])) / 2
    x = np.copysign(x, m[:, 2, 1] - m[:, 1, 2])
    y = np.copysign(y, m[:, 0, 2] - m[:, 2, 0])
    z = np.copysign(z, m[:, 1, 0] - m[:, 0, 1])
    q = np.stack([x, y, z, w], 1)
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def qmul(a, b):
    ax, ay, az, aw = a[..., 0], a[..., 1], a[..., 2], a[..., 3]
    bx, by, bz, bw = b[..., 0], b[..., 1], b[..., 2], b[..., 3]
    return np.stack([aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw,
                     aw * bw - ax * bx - ay * by - az * bz], -1)


def se3_to_dq(R, t):
    q0 = R_to_quat(R)
    qt = np.concatenate([0.5 * t, np.zeros((t.shape[0], 1))], 1)
    q1 = qmul(qt, q0)
    return np.concatenate([q0, q1], 1).astype(np.float32)


def dq_to_se3(dq):
    """(N, 8) dual quaternions (normalized here) to rotations (N, 3, 3) and translations (N, 3)."""
    q0 = dq[:, :4].astype(np.float64)
    q1 = dq[:, 4:].astype(np.float64)
    n = np.linalg.norm(q0, axis=1, keepdims=True)
    q0 = q0 / n
    q1 = q1 / n
    q1 = q1 - (q0 * q1).sum(1, keepdims=True) * q0
    x, y, z, w = q0[:, 0], q0[:, 1], q0[:, 2], q0[:, 3]
    R = np.stack([np.stack([1 - 2 * y * y - 2 * z * z, 2 * x * y - 2 * z * w, 2 * x * z + 2 * y * w], 1),
                  np.stack([2 * x * y + 2 * z * w, 1 - 2 * x * x - 2 * z * z, 2 * y * z - 2 * x * w], 1),
                  np.stack([2 * x * z - 2 * y * w, 2 * y * z + 2 * x * w, 1 - 2 * x * x - 2 * y * y], 1)], 1)
    conj = q0 * np.array([-1, -1, -1, 1.0])
    t = qmul(2 * q1, conj)[:, :3]
    return R, t


def rotation_log(R):
    """Rotation vectors of (N, 3, 3) rotations."""
    c = np.clip((R[:, 0, 0] + R[:, 1, 1] + R[:, 2, 2] - 1) / 2, -1.0, 1.0)
    th = np.arccos(c)
    v = np.stack([R[:, 2, 1] - R[:, 1, 2], R[:, 0, 2] - R[:, 2, 0], R[:, 1, 0] - R[:, 0, 1]], 1)
    s = np.sin(th)
    f = np.where(s > 1e-9, th / np.maximum(2 * s, 1e-300), 0.5)
    return v * f[:, None]


def smooth_warp(rng, nodes, surfels, max_rot_deg, max_trans, sigma=0.15, n_rbf=3):
    """Per-node SE(3): rotation about the node plus translation, from RBF fields."""
    x = nodes[:, :3].astype(np.float64)
    centres = surfels[rng.integers(0, surfels.shape[0], n_rbf), :3].astype(np.float64)
    a = rng.normal(size=(n_rbf, 3))
    b = rng.normal(size=(n_rbf, 3))
    g = np.exp(-((x[:, None, :] - centres[None]) ** 2).sum(-1) / (2 * sigma ** 2))
    om = g @ a
    ta = g @ b
    om *= np.deg2rad(max_rot_deg) / max(np.linalg.norm(om, axis=1).max(), 1e-12)
    ta *= max_trans / max(np.linalg.norm(ta, axis=1).max(), 1e-12)
    R = axis_angle_to_R(om)
    t = x - np.einsum("nij,nj->ni", R, x) + ta
    return se3_to_dq(R, t)


# ---------------------------------------------------------------------------
# numpy forward warp and splat
# ---------------------------------------------------------------------------
def forward_warp_np(dq, verts, normals, knn, sw, cw):
    """SurfelNodeDeformer-style warp: blend of normalized node DQs with skinning weights."""
    d = dq[knn.astype(np.int64)].astype(np.float64)              # (S, 4, 8)
    q0, q1 = d[..., :4], d[..., 4:]
    n = np.linalg.norm(q0, axis=-1, keepdims=True)
    q0 = q0 / n
    q1 = q1 / n
    q1 = q1 - (q0 * q1).sum(-1, keepdims=True) * q0
    w = (sw.astype(np.float64) * cw.astype(np.float64))[..., None]
    avg = np.concatenate([(w * q0).sum(1), (w * q1).sum(1)], 1)
    R, t = dq_to_se3(avg)
    v = np.einsum("sij,sj->si", R, verts[:, :3].astype(np.float64)) + t
    out_v = np.concatenate([v, verts[:, 3:4]], 1).astype(np.float32)
    out_n = None
    if normals is not None:
        nn = np.einsum("sij,sj->si", R, normals[:, :3].astype(np.float64))
        out_n = np.concatenate([nn, normals[:, 3:4]], 1).astype(np.float32)
    return out_v, out_n


def splat_np(verts_cam, cam: Camera, footprint=1):
    """Z-buffered splat: per pixel the nearest surfel id (ties to the lower id), 0xFFFFFFFF if none."""
    W, H = cam.width, cam.height
    v = verts_cam.astype(np.float32)
    z = v[:, 2]
    ok = z > 0
    ids = np.nonzero(ok)[0].astype(np.uint64)
    v = v[ok]
    z = v[:, 2]
    px = np.floor(np.float32(cam.fx) * v[:, 0] / z + np.float32(cam.cx) + np.float32(0.5)).astype(np.int64)
    py = np.floor(np.float32(cam.fy) * v[:, 1] / z + np.float32(cam.cy) + np.float32(0.5)).astype(np.int64)
    key = (z.view(np.uint32).astype(np.uint64) << np.uint64(32)) | ids
    pix_all, key_all = [], []
    for dy in range(-footprint, footprint + 1):
        for dx in range(-footprint, footprint + 1):
            x, y = px + dx, py + dy
            m = (x >= 0) & (y >= 0) & (x < W) & (y < H)
            pix_all.append(y[m] * W + x[m])
            key_all.append(key[m])
    pix = np.concatenate(pix_all)
    key = np.concatenate(key_all)
    order = np.argsort(key, kind="stable")
    pix_s = pix[order]
    uniq, first = np.unique(pix_s, return_index=True)
    index = np.full(H * W, 0xFFFFFFFF, np.uint32)
    index[uniq] = (key[order][first] & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    return index.reshape(H, W)


def maps_from_index(index, attr_v, attr_n, w_vertex=1.0, w_normal=0.0):
    H, W = index.shape
    vm = np.zeros((H, W, 4), np.float32)
    nm = np.zeros((H, W, 4), np.float32)
    m = index != 0xFFFFFFFF
    ids = index[m].astype(np.int64)
    vm[m, :3] = attr_v[ids, :3]
    vm[m, 3] = w_vertex
    nm[m, :3] = attr_n[ids, :3]
    nm[m, 3] = w_normal
    return vm, nm


# ---------------------------------------------------------------------------
# scene assembly
# ---------------------------------------------------------------------------
@dataclass
class SceneSpec:
    kind: str = "torus"              # "torus" or "union"
    scale: float = 1.0               # torus size multiplier (node count ~ scale^2)
    n_surfels: int = 200_000
    width: int = 640
    height: int = 480
    focal: float = 570.0
    graph_k: int = BASELINE_GRAPH_K
    max_rot_deg: float = 5.0
    max_trans: float = 0.01
    depth_noise: float = 0.001
    flow: bool = False
    flow_noise_px: float = 0.5
    flow_outliers: float = 0.1
    lambda_reg: float = 1.0
    lambda_of: float = 0.0
    gn_iters: int = 5
    pcg_iters: int = 20
    footprint: int = 1


def config_spec(config: int, **overrides) -> SceneSpec:
    """The benchmark configurations (0: plain torus, 1: large union with flow,
    2: batched torus family, 3: precision stress, 4: serving).  Configurations 0, 2, 3 and 4
    use the 8-NN node graph; configuration 1 names no graph size and keeps the reference's
    K = 4.  `graph_k=REFERENCE_GRAPH_K` gives the reference's own graph for any of them."""
    if config == 0:
        s = SceneSpec()
    elif config == 1:
        s = SceneSpec(kind="union", n_surfels=1_200_000, width=1280, height=720, focal=920.0, flow=True,
                      lambda_of=0.1, gn_iters=10, pcg_iters=30, graph_k=REFERENCE_GRAPH_K)
    elif config == 2:
        s = SceneSpec()
    elif config == 3:
        s = SceneSpec(scale=np.sqrt(4000 / 1800.0), n_surfels=520_000, max_rot_deg=15.0, depth_noise=0.0005,
                      gn_iters=10, pcg_iters=50)
    elif config == 4:
        s = SceneSpec(max_rot_deg=3.0, max_trans=0.005)
    else:
        raise ValueError(f"unknown config {config}")
    for k, v in overrides.items():
        setattr(s, k, v)
    return s


def spec_for_nodes(target_nodes: int, base: SceneSpec = None, surfels_per_node: int = 130) -> SceneSpec:
    """A torus scene scaled so that node construction yields about `target_nodes` nodes."""
    base = base or SceneSpec()
    scale = float(np.sqrt(target_nodes / 1800.0))
    out = SceneSpec(**{k: getattr(base, k) for k in base.__dataclass_fields__})
    out.scale = scale
    out.n_surfels = int(surfels_per_node * target_nodes)
    return out


def batch_node_targets(n: int, seed: int) -> np.ndarray:
    """Node counts of the batched configuration's scenes: log-uniform in [500, 8000]."""
    rng = np.random.default_rng(1_000_003 * 2 + seed)
    return np.exp(rng.uniform(np.log(500), np.log(8000), n)).astype(int)


def batch_scene(target_nodes: int, geometry, index: int, replica: int = 0) -> Scene:
    """Scene `index` of the batched configuration (config 2): the config-0 torus scaled to
    about `target_nodes` nodes, 130 surfels per node, 640x480 maps, 8-NN node graph."""
    spec = spec_for_nodes(int(target_nodes), config_spec(2))
    return make_scene(spec, geometry, seed=1_000_003 * 2 + 1000 * replica + index)


def sample_surface(spec: SceneSpec, rng):
    if spec.kind == "torus":
        p, n = sample_torus(rng, spec.n_surfels, 0.30 * spec.scale, 0.10 * spec.scale)
        Rt = rot_x(30.0)
        p = p @ Rt.T + np.array([0.0, 0.0, 1.0 * spec.scale])
        n = n @ Rt.T
        return p, n
    if spec.kind == "union":
        a = int(spec.n_surfels * 0.45)
        b = int(spec.n_surfels * 0.30)
        c = spec.n_surfels - a - b
        pt, nt = sample_torus(rng, a, 0.30, 0.10)
        Rt = rot_x(30.0)
        pt = pt @ Rt.T + np.array([-0.32, -0.05, 1.1])
        nt = nt @ Rt.T
        ps, ns = sample_sphere(rng, b, 0.2)
        ps = ps + np.array([0.35, 0.05, 0.95])
        pp, npl = sample_bumpy_plane(rng, c, 0.6, 0.005, 0.05)
        pp = pp @ rot_x(-20.0).T + np.array([0.0, 0.1, 1.45])
        npl = npl @ rot_x(-20.0).T
        return np.concatenate([pt, ps, pp]), np.concatenate([nt, ns, npl])
    raise ValueError(spec.kind)


def make_scene(spec: SceneSpec, geometry, seed: int) -> Scene:
    """Builds one scene.  `geometry` provides init_nodes, node_graph, skinning and
    optionally forward_warp / splat (else the numpy versions here are used)."""
    rng = np.random.default_rng(seed)
    cam = Camera(spec.width, spec.height, spec.focal, spec.focal, spec.width / 2.0, spec.height / 2.0)
    p, n = sample_surface(spec, rng)
    sv = pack4(p, 1.0)
    sn = pack4(n, 0.002)
    nodes = geometry.init_nodes(sv, NODE_RADIUS)
    knn, nsw, edges = geometry.node_graph(nodes, spec.graph_k, NODE_RADIUS)
    node_cw = np.ones_like(nsw, dtype=np.float32)
    sknn, ssw, scw = geometry.skinning(nodes, sv, NODE_RADIUS)
    gt = smooth_warp(rng, nodes, sv, spec.max_rot_deg, spec.max_trans)
    fw = getattr(geometry, "forward_warp", None) or forward_warp_np
    sp = getattr(geometry, "splat", None) or (lambda v, c, fp: splat_np(v, c, fp))
    # solver maps of the un-warped surfels (camera = world frame)
    ref_index = sp(sv, cam, spec.footprint)
    ref_v, ref_n = maps_from_index(ref_index, sv, sn, 1.0, 0.0)
    # measurement maps of the warped surfels with depth noise
    wv, wn = fw(gt, sv, sn, sknn, ssw, scw)
    meas_index = sp(wv, cam, spec.footprint)
    mv, mn = maps_from_index(meas_index, wv, wn, 1.0, 0.002)
    m = meas_index != 0xFFFFFFFF
    z = mv[..., 2]
    zn = z + rng.normal(scale=spec.depth_noise, size=z.shape).astype(np.float32)
    scale = np.where(m, zn / np.where(m, z, 1.0), 0.0).astype(np.float32)
    mv[..., :3] *= scale[..., None]
    flow = None
    if spec.flow:
        flow = np.zeros((cam.height, cam.width, 2), np.float32)
        ys, xs = np.mgrid[0:cam.height:4, 0:cam.width:4]
        ids = ref_index[ys, xs]
        ok = ids != 0xFFFFFFFF
        ys, xs, ids = ys[ok], xs[ok], ids[ok].astype(np.int64)
        wp = wv[ids]
        u = cam.fx * wp[:, 0] / wp[:, 2] + cam.cx
        v = cam.fy * wp[:, 1] / wp[:, 2] + cam.cy
        fl = np.stack([u - xs, v - ys], 1) + rng.normal(scale=spec.flow_noise_px, size=(len(xs), 2))
        out = rng.uniform(0, 1, len(xs)) < spec.flow_outliers
        fl[out, 0] = rng.uniform(0, cam.width, out.sum()) - xs[out]
        fl[out, 1] = rng.uniform(0, cam.height, out.sum()) - ys[out]
        flow[ys, xs] = fl.astype(np.float32)
    return Scene(camera=cam, surfel_vertex=sv, surfel_normal=sn, nodes=nodes, graph_k=spec.graph_k,
                 node_knn=knn, node_sw=nsw, edges=edges, node_cw=node_cw, surfel_knn=sknn, surfel_sw=ssw,
                 surfel_cw=scw, gt_dq=gt, index_map=ref_index, ref_vertex=ref_v, ref_normal=ref_n,
                 meas_vertex=mv, meas_normal=mn, flow=flow, lambda_reg=spec.lambda_reg,
                 lambda_of=spec.lambda_of, gn_iters=spec.gn_iters, pcg_iters=spec.pcg_iters)


def node_twists(dq, nodes):
    """Per-node twist of a solved warp: the rotation vector of the node's rotation and
    the displacement of the node centre, (N, 6)."""
    R, t = dq_to_se3(np.asarray(dq))
    x = np.asarray(nodes)[:, :3].astype(np.float64)
    disp = np.einsum("nij,nj->ni", R, x) + t - x
    return np.concatenate([rotation_log(R), disp], 1)


def twist_error(dq_a, dq_b, nodes):
    """Relative twist error of solved warp a against reference b:
    ||twist_a - twist_b|| / ||twist_b||, stacked over all nodes, with each node's
    twist taken about the node itself (`node_twists`)."""
    va = node_twists(dq_a, nodes)
    vb = node_twists(dq_b, nodes)
    return float(np.linalg.norm(va - vb) / max(np.linalg.norm(vb), 1e-30))


def position_error(scene: Scene, dq_a, dq_b):
    """Max distance (m) between surfels warped by a and by b."""
    va, _ = forward_warp_np(np.asarray(dq_a), scene.surfel_vertex, None, scene.surfel_knn, scene.surfel_sw,
                            scene.surfel_cw)
    vb, _ = forward_warp_np(np.asarray(dq_b), scene.surfel_vertex, None, scene.surfel_knn, scene.surfel_sw,
                            scene.surfel_cw)
    return float(np.abs(va[:, :3].astype(np.float64) - vb[:, :3]).max())
