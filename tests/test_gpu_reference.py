"""Parity with the reference itself: its own CUDA warp solver, compiled in place from the
reference tree (oracle/ref/Makefile -> oracle/_ref/starref_run), run on the same inputs.

Scenes: the full-size plain single-solve configuration (200k surfels, 640x480, about 1.6k nodes)
and a reduced one with an optical-flow map, both with the reference's 4-NN node graph and 16
key-point matches (the reference's pipeline always has some; their feature terms only enter the
index).  Within the reference's capacities (2048 nodes, 800k surfels).

* Index structures, bit for bit, three ways (reference, B200 device, oracle): the compacted dense
  terms with their skinning and flow-target pixels, the node->term map including the feature
  block of the term ids, the node-pair->term map and the block-row offsets.
* First Gauss-Newton iteration in the reference's own arithmetic (WS_PREC_FP32: FP32, twists
  about the world origin, Gauss-Jordan inverse): diagonal blocks, J^T r, inverse blocks and the
  PCG step against the reference's.
* Full solve at the reference's 6 x 10 iterations: the reference's FP32 solve, the B200 FP32 and
  mixed solves and the FP64 oracle compared pairwise.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import ref_oracle  # noqa: E402

if not ref_oracle.available():
    pytest.skip("oracle/_ref/starref_run is not built (it needs the reference tree at build time)",
                allow_module_level=True)


@pytest.fixture(scope="module")
def config0_k4(ws):
    from starhub_b200 import scenes
    from starhub_b200.solver import GpuGeometry
    spec = scenes.config_spec(0, graph_k=scenes.REFERENCE_GRAPH_K)
    return scenes.make_scene(spec, GpuGeometry(), seed=1_000_003 * 0)


@pytest.fixture(scope="module")
def flow_scene(ws):
    """A reduced torus with a flow map on a 4-pixel grid (flow targets of the compaction)."""
    from starhub_b200 import scenes
    from starhub_b200.solver import GpuGeometry
    spec = scenes.config_spec(0, n_surfels=60_000, width=320, height=240, focal=285.0, flow=True,
                              graph_k=scenes.REFERENCE_GRAPH_K)
    return scenes.make_scene(spec, GpuGeometry(), seed=12)


def _with_features(sc, feature_knn):
    import dataclasses
    return dataclasses.replace(sc, feature_knn=feature_knn)


def _device_solver(sc, precision, gn, pcg):
    import torch
    from starhub_b200.solver import DeviceScene, WarpSolver
    ds = DeviceScene.from_scene(sc)
    nf = 0 if sc.feature_knn is None else sc.feature_knn.shape[0]
    s = WarpSolver(max_nodes=ds.num_nodes, max_pixels=ds.num_pixels, max_edges=ds.num_edges, max_features=nf,
                   precision=precision)
    s.SetSolverInputs(ds)
    s.SolveStreamed(gn, pcg, stream=torch.cuda.Stream())
    s.Sync()
    return s, s.SolvedNodeSE3(0).cpu().numpy().copy()


def _check_index(ref, s, orc, sc):
    # compacted dense terms: reference == device == oracle
    pix, knn, sw, cw = s.dense_terms()
    opix, oknn, osw, ocw = orc.compact_pixels(sc)
    assert len(ref["pixels"]) > 1000
    for a, b in ((ref["pixels"], pix), (ref["knn"], knn), (ref["spatial_w"], sw), (ref["connect_w"], cw)):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(ref["pixels"], opix)
    np.testing.assert_array_equal(ref["knn"], oknn)
    # node -> term, feature block included
    off, ti = s.node2term()
    ooff, oti = orc.node2term(oknn, sc.edges, sc.num_nodes, feat_knn=sc.feature_knn)
    np.testing.assert_array_equal(ref["n2t_offset"], off)
    np.testing.assert_array_equal(ref["n2t_terms"][: off[-1]], ti)
    np.testing.assert_array_equal(ref["n2t_offset"], ooff)
    # node pair -> term: the reference's symmetric map, its upper half against the half pairs
    rows, cols = ref_oracle.decode_pairs(ref["pair_keys"])
    upper = rows < cols
    p = s.node_pairs()
    np.testing.assert_array_equal(rows[upper], p["rows"])
    np.testing.assert_array_equal(cols[upper], p["cols"])
    np.testing.assert_array_equal(ref["pair_range"][upper, 0], p["begin"])
    np.testing.assert_array_equal(ref["pair_range"][upper, 1], p["end"])
    np.testing.assert_array_equal(ref["pair_terms"][: p["end"][-1]], p["term_index"])
    m = orc.nodepair2term(oknn, sc.edges, sc.num_nodes, feat_knn=sc.feature_knn)
    np.testing.assert_array_equal(ref["pair_terms"][: m["half_end"][-1]], m["term_index"][: m["half_end"][-1]])
    np.testing.assert_array_equal(ref["blkrow_offset"][: sc.num_nodes + 1], m["blkrow_offset"][: sc.num_nodes + 1])
    # every lower entry mirrors an upper one with the same range
    lo = ~upper & (rows != cols)
    mirror = {(int(c), int(r)): tuple(rg) for r, c, rg in zip(rows[lo], cols[lo], ref["pair_range"][lo])}
    assert len(mirror) == int(upper.sum())
    for r, c, rg in zip(rows[upper], cols[upper], ref["pair_range"][upper]):
        assert mirror[(int(r), int(c))] == tuple(rg)


def test_index_bit_exact_to_the_reference(config0_k4, orc, tmp_path):
    ref = ref_oracle.run(config0_k4, tmp_path, gn_iters=1, pcg_iters=1)
    sc = _with_features(config0_k4, ref["feature_knn"])
    s, _ = _device_solver(sc, 0, 1, 1)
    _check_index(ref, s, orc, sc)


def test_flow_targets_bit_exact_to_the_reference(flow_scene, orc, tmp_path):
    assert np.abs(flow_scene.flow).max() > 0
    ref = ref_oracle.run(flow_scene, tmp_path, gn_iters=1, pcg_iters=1)
    sc = _with_features(flow_scene, ref["feature_knn"])
    s, _ = _device_solver(sc, 0, 1, 1)
    _check_index(ref, s, orc, sc)


def test_first_iteration_in_the_reference_arithmetic(config0_k4, orc, tmp_path):
    """WS_PREC_FP32 against the reference's own FP32 kernels, stage by stage.  The blocks and
    J^T r are sums of the same FP32 products in another order (the reference: warp scans over
    32-term batches); the tolerances are FP32 rounding over sums of a few thousand terms.  The
    6x6 blocks are ill-conditioned (twists about the world origin, about 1 m away), so the inverse
    is compared at 1e-3 of its scale, and the step after 10 FP32 PCG iterations, which amplify the
    rounding differences by the condition number, at 2e-3 of its scale; both FP32 steps must also
    be about as far from the FP64 oracle's step as each other."""
    ref = ref_oracle.run(config0_k4, tmp_path, gn_iters=1, pcg_iters=10)
    sc = _with_features(config0_k4, ref["feature_knn"])
    s, _ = _device_solver(sc, 1, 1, 10)
    sysm = s.system()
    diag = sysm["blocks"][sysm["rowptr"][:-1]]
    scale = np.abs(ref["diag"]).max()
    np.testing.assert_allclose(diag, ref["diag"], atol=2e-5 * scale, rtol=0)
    np.testing.assert_allclose(sysm["jtr"], ref["jtr"], atol=2e-5 * np.abs(ref["jtr"]).max(), rtol=0)
    np.testing.assert_allclose(sysm["inv_diag"], ref["inv_diag"], atol=1e-3 * np.abs(ref["inv_diag"]).max(), rtol=0)
    np.testing.assert_allclose(sysm["step"], ref["step"], atol=2e-3 * np.abs(ref["step"]).max(), rtol=0)
    # the FP64 oracle's first step, against which both FP32 solves are measured
    _, info64 = orc.solve(sc, gn_iters=1, pcg_iters=10, debug=True)
    e_ref = np.abs(ref["step"] - info64["step"]).max() / np.abs(info64["step"]).max()
    e_dev = np.abs(sysm["step"] - info64["step"]).max() / np.abs(info64["step"]).max()
    assert e_dev <= max(2 * e_ref, 1e-4), (e_dev, e_ref)


def test_full_solve_against_the_reference(config0_k4, orc, tmp_path):
    """The reference's solve at its own 6 x 10 iterations.  The reference computes in FP32 with
    twists about the world origin; its distance to the FP64 oracle is the FP32 error of those
    ill-conditioned blocks.  The B200 FP32 mode (the same arithmetic, other summation orders) must
    be as close to FP64 as the reference is, the B200 mixed mode within 1e-4 of FP64, and the two
    FP32 solves within the reference's own FP32 error of each other."""
    from starhub_b200.scenes import position_error, twist_error
    ref = ref_oracle.run(config0_k4, tmp_path, gn_iters=6, pcg_iters=10)
    sc = _with_features(config0_k4, ref["feature_knn"])
    fp64 = orc.solve(sc, gn_iters=6, pcg_iters=10)
    _, dev32 = _device_solver(sc, 1, 6, 10)
    _, mixed = _device_solver(sc, 0, 6, 10)
    e_ref = twist_error(ref["se3"], fp64, sc.nodes)
    e_dev32 = twist_error(dev32, fp64, sc.nodes)
    e_mixed = twist_error(mixed, fp64, sc.nodes)
    e_32_32 = twist_error(dev32, ref["se3"], sc.nodes)
    print(f"twist error vs FP64: reference {e_ref:.2e}, B200 fp32 {e_dev32:.2e}, B200 mixed {e_mixed:.2e}; "
          f"B200 fp32 vs reference {e_32_32:.2e}; mixed vs reference {twist_error(mixed, ref['se3'], sc.nodes):.2e}")
    assert np.isfinite(ref["se3"]).all()
    assert e_mixed <= 1e-4
    assert position_error(sc, mixed, fp64) <= 1e-5
    assert e_dev32 <= 2 * e_ref + 1e-5
    assert e_32_32 <= 2 * e_ref + 1e-5
