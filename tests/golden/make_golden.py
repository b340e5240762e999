"""Generates the golden fixtures in this folder.

The reference ships no golden vectors or test data for the solve (its only PCG data files
are referenced at an author's absolute path and not shipped), so these fixtures are
produced by the CPU oracle (the C++ restatement in oracle/) on small seeded scenes and
committed, with this script, as the regression pin of both the oracle and the CUDA path:

* torus_small.npz: a tilted torus, 128x96 pixels, 6000 surfels; the solver inputs
  (maps, skinning, node graph), the bit-exact index structures (compacted dense terms,
  node->term and node-pair->term maps) and the FP64 solve (3 Gauss-Newton x 10 PCG);
* torus_small_flow.npz: the same scene with a flow map on a 4-px grid and lambda_of = 0.1.

The oracle runs single-threaded here, so its FP64 sums have a fixed order and a rerun
reproduces the stored solution exactly.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

GN, PCG = 3, 10


def small_spec(flow: bool):
    from starhub_b200 import scenes
    return scenes.config_spec(0, n_surfels=6000, width=128, height=96, focal=114.0, scale=0.45,
                              flow=flow, lambda_of=0.1 if flow else 0.0, gn_iters=GN, pcg_iters=PCG)


def scene_arrays(sc) -> dict:
    cam = sc.camera
    out = dict(
        camera=np.array([cam.width, cam.height, cam.fx, cam.fy, cam.cx, cam.cy], np.float64),
        surfel_vertex=sc.surfel_vertex, surfel_normal=sc.surfel_normal, nodes=sc.nodes,
        graph_k=np.array(sc.graph_k), node_knn=sc.node_knn, node_sw=sc.node_sw, edges=sc.edges, node_cw=sc.node_cw,
        surfel_knn=sc.surfel_knn, surfel_sw=sc.surfel_sw, surfel_cw=sc.surfel_cw, gt_dq=sc.gt_dq,
        index_map=sc.index_map, ref_vertex=sc.ref_vertex, ref_normal=sc.ref_normal, meas_vertex=sc.meas_vertex,
        meas_normal=sc.meas_normal,
        lambdas=np.array([sc.lambda_depth, sc.lambda_of, sc.lambda_reg, sc.lambda_node, sc.lambda_feature]),
        iters=np.array([sc.gn_iters, sc.pcg_iters]),
    )
    if sc.flow is not None:
        out["flow"] = sc.flow
    return out


def scene_from_arrays(d):
    """Inverse of scene_arrays (used by the tests)."""
    from starhub_b200 import scenes
    w, h, fx, fy, cx, cy = d["camera"]
    cam = scenes.Camera(int(w), int(h), float(fx), float(fy), float(cx), float(cy))
    lam = d["lambdas"]
    return scenes.Scene(
        camera=cam, surfel_vertex=d["surfel_vertex"], surfel_normal=d["surfel_normal"], nodes=d["nodes"],
        graph_k=int(d["graph_k"]), node_knn=d["node_knn"], node_sw=d["node_sw"], edges=d["edges"],
        node_cw=d["node_cw"], surfel_knn=d["surfel_knn"], surfel_sw=d["surfel_sw"], surfel_cw=d["surfel_cw"],
        gt_dq=d["gt_dq"], index_map=d["index_map"], ref_vertex=d["ref_vertex"], ref_normal=d["ref_normal"],
        meas_vertex=d["meas_vertex"], meas_normal=d["meas_normal"], flow=d["flow"] if "flow" in d else None,
        lambda_depth=float(lam[0]), lambda_of=float(lam[1]), lambda_reg=float(lam[2]), lambda_node=float(lam[3]),
        lambda_feature=float(lam[4]), gn_iters=int(d["iters"][0]), pcg_iters=int(d["iters"][1]))


def oracle_outputs(orc, sc) -> dict:
    pix, knn, sw, cw = orc.compact_pixels(sc)
    off, ti = orc.node2term(knn, sc.edges, sc.num_nodes)
    m = orc.nodepair2term(knn, sc.edges, sc.num_nodes)
    sol = orc.solve(sc, gn_iters=GN, pcg_iters=PCG, threads=1)
    return dict(out_pixels=pix, out_knn=knn, out_sw=sw, out_cw=cw, out_n2t_offset=off,
                out_n2t_terms=ti[: off[-1]], out_half_rows=m["half_rows"], out_half_cols=m["half_cols"],
                out_half_begin=m["half_begin"], out_half_end=m["half_end"],
                out_pair_terms=m["term_index"][: m["half_end"][-1]], out_solution_fp64=sol)


def main():
    import oracle as orc
    from starhub_b200 import scenes
    orc.build()
    geo = orc.OracleGeometry()
    for name, flow, seed in (("torus_small", False, 21), ("torus_small_flow", True, 22)):
        sc = scenes.make_scene(small_spec(flow), geo, seed=seed)
        arrays = scene_arrays(sc)
        arrays.update(oracle_outputs(orc, sc))
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        print(name, "nodes", sc.num_nodes, "dense terms", int(arrays["out_n2t_offset"][-1]),
              "bytes", (HERE / f"{name}.npz").stat().st_size)


if __name__ == "__main__":
    main()
