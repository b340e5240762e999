"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py).

CPU: the oracle reproduces the stored index structures bit for bit and the stored FP64
solution exactly (single-threaded, fixed summation order).
GPU: the CUDA path reproduces the stored index structures bit for bit and is within
1e-4 relative twist error and 1e-5 m warped-position error of the stored FP64 solution,
without the oracle at run time.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
FIXTURES = ["torus_small", "torus_small_flow"]


def load(name):
    import make_golden
    d = dict(np.load(GOLDEN / f"{name}.npz"))
    return make_golden.scene_from_arrays(d), d


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_reproduces_golden(orc, name):
    import make_golden
    sc, d = load(name)
    out = make_golden.oracle_outputs(orc, sc)
    for k, v in out.items():
        np.testing.assert_array_equal(v, d[k], err_msg=k)


@pytest.mark.gpu
@pytest.mark.parametrize("name", FIXTURES)
def test_cuda_path_matches_golden(ws, name):
    import torch
    from starhub_b200.scenes import position_error, twist_error
    from starhub_b200.solver import DeviceScene, WarpSolver
    sc, d = load(name)
    ds = DeviceScene.from_scene(sc)
    s = WarpSolver(max_nodes=ds.num_nodes, max_pixels=ds.num_pixels, max_edges=ds.num_edges)
    s.SetSolverInputs(ds)
    s.SolveStreamed(sc.gn_iters, sc.pcg_iters, stream=torch.cuda.Stream())
    s.Sync()
    pix, knn, sw, cw = s.dense_terms()
    n = len(pix)
    np.testing.assert_array_equal(pix, d["out_pixels"][:n])
    np.testing.assert_array_equal(knn, d["out_knn"][:n])
    np.testing.assert_array_equal(sw, d["out_sw"][:n])
    np.testing.assert_array_equal(cw, d["out_cw"][:n])
    off, ti = s.node2term()
    np.testing.assert_array_equal(off, d["out_n2t_offset"])
    np.testing.assert_array_equal(ti, d["out_n2t_terms"])
    p = s.node_pairs()
    np.testing.assert_array_equal(p["rows"], d["out_half_rows"])
    np.testing.assert_array_equal(p["cols"], d["out_half_cols"])
    np.testing.assert_array_equal(p["begin"], d["out_half_begin"])
    np.testing.assert_array_equal(p["end"], d["out_half_end"])
    np.testing.assert_array_equal(p["term_index"], d["out_pair_terms"])
    dq = s.SolvedNodeSE3(0).cpu().numpy().copy()
    ref = d["out_solution_fp64"]
    assert twist_error(dq, ref, sc.nodes) <= 1e-4
    assert position_error(sc, dq, ref) <= 1e-5
