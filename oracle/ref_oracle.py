"""Runs the reference's own CUDA warp solver on a scene (test infrastructure).

oracle/ref/Makefile compiles the reference's solver translation units in place from the
reference tree into oracle/_ref/starref_run; this module writes a scene's solver inputs for it,
runs it in a child process on the GPU, and reads back what the reference built and solved:

* the compacted dense terms (ImageTermKNNFetcher::GetImageTermPixelAndKNN,
  examples/mono_star/opt/ImageTermKNNFetcher.h:55-83);
* the node->term map (Node2TermsIndex::GetNode2TermMap, Node2TermsIndex.h:79-94);
* the node-pair->term map (NodePair2TermsIndex::GetNodePair2TermMap, NodePair2TermsIndex.h:44-55):
  symmetric encoded pairs, their term ranges, the term list and the block-row offsets;
* with counts other than the reference's 6 x 10, the first Gauss-Newton iteration's diagonal
  blocks (with the +1e-3), J^T r, inverse blocks and PCG step;
* the solved node warps (WarpSolver::SolvedNodeSE3).

The reference exits the process on any CUDA error (pcl::gpu::___cudaSafeCall), which is why it
runs as a child process.  It is limited to its own capacities: at most 2048 nodes, 800k surfels,
4-NN node graphs and 32 key-point matches (Constants.cpp:7-18, geometry/constants.h:6-14); a
scene outside them is refused before anything runs.  The reference always has key-point
matches in its pipeline; `num_keypoints` of them are made from surfels of the scene (their
feature terms only enter the index: PreconditionerRhsBuilder.cu:214-219, JtJMaterializer.cu:127-133).
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BINARY = HERE / "_ref" / "starref_run"
MAX_NODES = 2048
MAX_SURFELS = 800_000
MAX_KEYPOINTS = 32


def available() -> bool:
    return BINARY.exists()


def keypoints(scene, count, seed=3):
    """`count` key-point matches made from the scene's surfels: (knn, spatial and connect weights,
    vertices, normals, matches (i, i))."""
    rng = np.random.default_rng(seed)
    pick = np.sort(rng.choice(scene.surfel_knn.shape[0], count, replace=False))
    match = np.stack([np.arange(count), np.arange(count)], 1).astype(np.int32)
    return (scene.surfel_knn[pick].copy(), scene.surfel_sw[pick].copy(), scene.surfel_cw[pick].copy(),
            scene.surfel_vertex[pick].copy(), scene.surfel_normal[pick].copy(), match)


def run(scene, work_dir, gn_iters=6, pcg_iters=10, num_keypoints=16, timeout=600):
    """Solves `scene` with the reference's CUDA solver; returns a dict of its outputs."""
    if scene.graph_k != 4:
        raise ValueError("the reference's node graph has 4 neighbours per node")
    if scene.num_nodes > MAX_NODES or scene.surfel_vertex.shape[0] > MAX_SURFELS:
        raise ValueError("scene outside the reference's capacities")
    if not 1 <= num_keypoints <= MAX_KEYPOINTS:
        raise ValueError("the reference takes 1..32 key-point matches")
    d = Path(work_dir)
    d.mkdir(parents=True, exist_ok=True)
    cam = scene.camera
    nrs = float(np.float32(scene.node_radius) * np.float32(scene.node_radius))
    (d / "params.txt").write_text(
        f"{cam.width} {cam.height} {cam.fx!r} {cam.fy!r} {cam.cx!r} {cam.cy!r} {scene.num_nodes} "
        f"{scene.surfel_vertex.shape[0]} {scene.edges.shape[0]} {nrs!r} {num_keypoints} {gn_iters} {pcg_iters}\n")
    kp_knn, kp_sw, kp_cw, kp_v, kp_n, kp_match = keypoints(scene, num_keypoints)
    arrays = {"meas_vertex": scene.meas_vertex, "meas_normal": scene.meas_normal, "ref_vertex": scene.ref_vertex,
              "ref_normal": scene.ref_normal, "index": scene.index_map, "surfel_knn": scene.surfel_knn,
              "surfel_sw": scene.surfel_sw, "surfel_cw": scene.surfel_cw, "nodes": scene.nodes,
              "edges": scene.edges, "node_cw": scene.node_cw, "node_knn": scene.node_knn, "node_sw": scene.node_sw,
              "kp_knn": kp_knn, "kp_sw": kp_sw, "kp_cw": kp_cw, "kp_vertex": kp_v, "kp_normal": kp_n,
              "kp_match": kp_match}
    if scene.flow is not None:
        arrays["flow"] = scene.flow
    for name, a in arrays.items():
        (d / f"{name}.bin").write_bytes(np.ascontiguousarray(a).tobytes())
    r = subprocess.run([str(BINARY), str(d)], capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"starref_run failed ({r.returncode}): {r.stderr[-2000:]} {r.stdout[-2000:]}")

    def load(name, dtype, shape=None):
        p = d / f"out_{name}.bin"
        if not p.exists():
            raise RuntimeError(f"starref_run wrote no {p.name} (it exits on CUDA errors): {r.stdout[-2000:]}")
        a = np.frombuffer(p.read_bytes(), dtype)
        return a.reshape(shape) if shape is not None else a

    out = {
        "pixels": load("pixels", np.uint16, (-1, 4)),
        "knn": load("term_knn", np.uint16, (-1, 4)),
        "spatial_w": load("term_sw", np.float32, (-1, 4)),
        "connect_w": load("term_cw", np.float32, (-1, 4)),
        "n2t_offset": load("n2t_offset", np.uint32),
        "n2t_terms": load("n2t_terms", np.uint32),
        "pair_keys": load("pair_keys", np.uint32),
        "pair_range": load("pair_range", np.uint32, (-1, 2)),
        "pair_terms": load("pair_terms", np.uint32),
        "blkrow_offset": load("blkrow_offset", np.uint32),
        "se3": load("se3", np.float32, (-1, 8)),
        "feature_knn": kp_knn,
    }
    if (gn_iters, pcg_iters) != (6, 10):
        n = scene.num_nodes
        out.update(diag=load("diag", np.float32, (n, 36)), jtr=load("jtr", np.float32, (n, 6)),
                   inv_diag=load("inv_diag", np.float32, (n, 36)), step=load("step", np.float32, (n, 6)))
    return out


def decode_pairs(keys):
    """encode_nodepair (libs/star/opt/solver_encode.h:8-25): (row, column) of each encoded pair."""
    keys = np.asarray(keys, np.uint32)
    return (keys // 4096).astype(np.uint32), (keys % 4096).astype(np.uint32)
