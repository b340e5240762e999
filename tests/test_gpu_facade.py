"""The C++ facade at the pipeline's call site, on the GPU.

tests/facade_app_callsite.cpp runs the solver calls of examples/mono_star/app.cu:45-150 as
written there (texture-object maps in Measure4Solver / Render4Solver, GArrayViews in
Geometry4Solver / NodeGraph4Solver, the camera from the process-wide configuration, frame 1,
stream 0) and writes SolvedSE3().  Its result must equal, bit for bit, the C ABI solve of the
same inputs at the reference's iteration counts (6 Gauss-Newton x 10 PCG), for the
reference's 4-NN node graph and for the 8-NN graph.
"""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def app_binary(ws, tmp_path_factory):
    cuda = Path("/usr/local/cuda")
    if shutil.which("g++") is None:
        pytest.skip("g++ missing")
    out = tmp_path_factory.mktemp("facade") / "app"
    lib_dir = ROOT / "starhub_b200"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(ROOT / "include"), "-I", str(cuda / "include"),
                        str(ROOT / "tests" / "facade_app_callsite.cpp"), "-o", str(out), "-L", str(lib_dir),
                        "-lwarpsolve", f"-Wl,-rpath,{lib_dir}", "-L", str(cuda / "lib64"), "-lcudart"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def write_inputs(sc, d: Path, frame_idx=1):
    cam = sc.camera
    (d / "params.txt").write_text(f"{cam.width} {cam.height} {sc.graph_k} {frame_idx} {cam.fx} {cam.fy} {cam.cx} "
                                  f"{cam.cy} {float(np.float32(sc.node_radius) * np.float32(sc.node_radius))!r}\n")
    arrays = {"meas_vertex": sc.meas_vertex, "meas_normal": sc.meas_normal, "ref_vertex": sc.ref_vertex,
              "ref_normal": sc.ref_normal, "index": sc.index_map, "surfel_knn": sc.surfel_knn,
              "surfel_sw": sc.surfel_sw, "surfel_cw": sc.surfel_cw, "nodes": sc.nodes, "edges": sc.edges,
              "node_cw": sc.node_cw}
    for name, a in arrays.items():
        (d / f"{name}.bin").write_bytes(np.ascontiguousarray(a).tobytes())


@pytest.mark.parametrize("k", [4, 8])
def test_app_call_site_equals_the_c_abi(app_binary, small_scene, small_scene_k8, tmp_path, k):
    import torch
    from starhub_b200.solver import DeviceScene, WarpSolver
    sc = small_scene if k == 4 else small_scene_k8
    write_inputs(sc, tmp_path)
    r = subprocess.run([str(app_binary), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = np.frombuffer((tmp_path / "se3.bin").read_bytes(), np.float32).reshape(-1, 8)

    ds = DeviceScene.from_scene(sc)
    s = WarpSolver(max_nodes=ds.num_nodes, max_pixels=ds.num_pixels, max_edges=ds.num_edges)
    s.SetSolverInputs(ds)
    s.SolveStreamed(6, 10, stream=torch.cuda.Stream())
    s.Sync()
    want = s.SolvedNodeSE3(0).cpu().numpy()
    assert got.shape == want.shape
    np.testing.assert_array_equal(got, want)


def test_frame_zero_is_a_no_op(app_binary, small_scene, tmp_path):
    """OptimizationProcessorWarpSolver.cu:35-36: frame 0 only initialises the model, so
    SolvedSE3() is empty."""
    write_inputs(small_scene, tmp_path, frame_idx=0)
    r = subprocess.run([str(app_binary), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "se3.bin").read_bytes() == b""
