"""The terms the default penalties leave out, on the GPU against the oracle.

* Node-motion term (ComputeNodeMotionKernel, examples/mono_star/opt/NodeMotionHandler.cu:9-19;
  node_motion_jacobian.cuh:7-36): r = t_i - pred.xyz on each node's translation, weighted by the
  prediction's confidence pred.w, with lambda_node > 0.  First-iteration diagonal blocks and
  J^T r against the oracle's node-centred mixed mode, full solve against the FP64 oracle.
* Feature terms (KeyPoint4Solver::kp_knn): they take part in the term-id space
  [dense | reg | node-motion | feature] (examples/mono_star/common/term_offset_types.h:38-118)
  and in the node->term and node-pair->term maps (Node2TermsIndex.cu:6-76,
  NodePair2TermsIndex.cu:11-193) with a zero Jacobian (PreconditionerRhsBuilder.cu:214-219):
  the maps bit-exact, the solve unchanged by them.
"""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solve(sc, gn, pcg, max_features=0):
    import torch
    from starhub_b200.solver import DeviceScene, WarpSolver
    ds = DeviceScene.from_scene(sc)
    s = WarpSolver(max_nodes=ds.num_nodes, max_pixels=ds.num_pixels, max_edges=ds.num_edges,
                   max_features=max_features)
    s.SetSolverInputs(ds)
    s.SolveStreamed(gn, pcg, stream=torch.cuda.Stream())
    s.Sync()
    return s, s.SolvedNodeSE3(0).cpu().numpy().copy()


@pytest.fixture(scope="module")
def motion_scene(small_scene):
    """The reduced config-0 torus with a node-motion prediction: the ground-truth translation of
    every node's dual quaternion plus 2 mm noise, confidence 0.5-1, lambda_node = 0.3."""
    from starhub_b200.scenes import dq_to_se3
    rng = np.random.default_rng(21)
    _, t = dq_to_se3(small_scene.gt_dq)
    pred = np.zeros((small_scene.num_nodes, 4), np.float32)
    pred[:, :3] = t + rng.normal(scale=0.002, size=t.shape)
    pred[:, 3] = rng.uniform(0.5, 1.0, small_scene.num_nodes)
    return dataclasses.replace(small_scene, node_motion_pred=pred, lambda_node=0.3)


def test_node_motion_first_iteration(ws, orc, motion_scene):
    sc = motion_scene
    s, _ = _solve(sc, 1, 20)
    _, info = orc.solve(sc, gn_iters=1, pcg_iters=20, debug=True, precision=orc.ORC_PREC_MIXED)
    _, plain = orc.solve(dataclasses.replace(sc, node_motion_pred=None, lambda_node=0.0), gn_iters=1,
                         pcg_iters=20, debug=True, precision=orc.ORC_PREC_MIXED)
    # the term is live: it moves J^T r by far more than the tolerance below
    assert np.abs(info["jtr"] - plain["jtr"]).max() > 1e-2 * np.abs(info["jtr"]).max()
    sysm = s.system()
    diag = sysm["blocks"][sysm["rowptr"][:-1]]
    scale = np.abs(info["diag"]).max()
    np.testing.assert_allclose(diag, info["diag"], atol=2e-5 * scale, rtol=0)
    np.testing.assert_allclose(sysm["jtr"], info["jtr"], atol=2e-5 * np.abs(info["jtr"]).max(), rtol=0)


def test_node_motion_full_solve(ws, orc, motion_scene):
    from starhub_b200.scenes import position_error, twist_error
    sc = motion_scene
    _, dq = _solve(sc, sc.gn_iters, sc.pcg_iters)
    ref = orc.solve(sc)
    without = orc.solve(dataclasses.replace(sc, node_motion_pred=None, lambda_node=0.0))
    assert twist_error(without, ref, sc.nodes) > 1e-3          # the term changes the solution
    assert twist_error(dq, ref, sc.nodes) <= 1e-4
    assert position_error(sc, dq, ref) <= 1e-5


@pytest.fixture(scope="module")
def feature_scene(small_scene):
    """The reduced config-0 torus with 700 feature terms: the skinning neighbours of random
    surfels, as KeyPoint4Solver::kp_knn carries them."""
    rng = np.random.default_rng(8)
    pick = rng.choice(small_scene.surfel_knn.shape[0], 700, replace=False)
    return dataclasses.replace(small_scene, feature_knn=small_scene.surfel_knn[pick].copy())


def test_feature_terms_in_the_index_bit_exact(ws, orc, feature_scene):
    sc = feature_scene
    nf = sc.feature_knn.shape[0]
    s, _ = _solve(sc, 1, 1, max_features=nf)
    _, oknn, _, _ = orc.compact_pixels(sc)
    off, ti = s.node2term()
    ooff, oti = orc.node2term(oknn, sc.edges, sc.num_nodes, feat_knn=sc.feature_knn)
    feature_base = len(oknn) + len(sc.edges) + sc.num_nodes
    assert (oti[: ooff[-1]] >= feature_base).sum() == 4 * nf   # every feature term is listed 4 times
    np.testing.assert_array_equal(off, ooff)
    np.testing.assert_array_equal(ti, oti[: ooff[-1]])
    p = s.node_pairs()
    m = orc.nodepair2term(oknn, sc.edges, sc.num_nodes, feat_knn=sc.feature_knn)
    np.testing.assert_array_equal(p["rows"], m["half_rows"])
    np.testing.assert_array_equal(p["cols"], m["half_cols"])
    np.testing.assert_array_equal(p["begin"], m["half_begin"])
    np.testing.assert_array_equal(p["end"], m["half_end"])
    np.testing.assert_array_equal(p["term_index"], m["term_index"][: m["half_end"][-1]])


def test_feature_terms_leave_the_solve_unchanged(ws, orc, feature_scene, small_scene):
    from starhub_b200.scenes import position_error, twist_error
    sc = feature_scene
    _, dq = _solve(sc, sc.gn_iters, sc.pcg_iters, max_features=sc.feature_knn.shape[0])
    _, plain = _solve(small_scene, sc.gn_iters, sc.pcg_iters)
    ref = orc.solve(sc)
    assert twist_error(dq, ref, sc.nodes) <= 1e-4
    assert position_error(sc, dq, ref) <= 1e-5
    assert twist_error(dq, plain, sc.nodes) <= 1e-6
