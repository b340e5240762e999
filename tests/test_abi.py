"""CPU checks of the C ABI library: it loads without a GPU and exports every
entry point include/warpsolve.h declares; host-side argument checks."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def lib():
    from starhub_b200 import build as b
    b.build()
    from starhub_b200 import _lib
    return _lib.load()


def declared_functions():
    text = (ROOT / "include" / "warpsolve.h").read_text()
    return sorted(set(re.findall(r"\b(ws_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "ws_solve" in names and "ws_create" in names and len(names) >= 20


def test_library_exports_every_declared_symbol(lib):
    from starhub_b200 import _lib
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert sorted(_lib.EXPORTED) == declared_functions()


def test_error_strings(lib):
    from starhub_b200 import _lib
    assert _lib.error_string(0) == "ok"
    assert "capacity" in _lib.error_string(_lib.WS_ERR_CAPACITY)


def test_create_rejects_bad_config(lib):
    from starhub_b200._lib import WsConfig
    h = C.c_void_p()
    cfg = WsConfig()
    cfg.max_scenes = 0
    assert lib.ws_create(C.byref(cfg), C.byref(h)) == -1
    assert lib.ws_create(None, C.byref(h)) == -1
    assert lib.ws_destroy(None) == -1
    assert lib.ws_solve(None, 1, 1, None) == -1


def test_default_penalties_match_reference(lib):
    from starhub_b200._lib import WsInputs
    s = WsInputs()
    lib.ws_default_penalties(C.byref(s))
    # PenaltyConstants::setDefaultValue (examples/mono_star/opt/PenaltyConstants.cu:8-15)
    assert (round(s.lambda_depth, 6), s.lambda_optical_flow, s.lambda_reg, s.lambda_node_translation,
            s.lambda_feature) == (0.1, 0.0, 1.0, 0.0, 1.0)


def test_cpp_facade_builds_and_links(lib, tmp_path):
    """The header-only C++ facade (include/starhub_b200/warp_solver.hpp) compiles and links
    against the library: every entry point its classes call is exported."""
    import shutil
    import subprocess
    cuda = Path("/usr/local/cuda")
    if shutil.which("g++") is None or not (cuda / "include" / "cuda_runtime.h").exists():
        pytest.skip("g++ or the CUDA headers are missing")
    src = tmp_path / "facade.cpp"
    src.write_text(
        '#include "starhub_b200/warp_solver.hpp"\n'
        "using namespace star::b200;\n"
        "int use(const float4 *v, unsigned n, cudaStream_t st) {\n"
        "  NodeGraph g(0.025f, 4096, 8);\n"
        "  g.InitializeNodeGraphFromVertex(v, n, 0, true, st);\n"
        "  g.NaiveExpandNodeGraphFromVertexUnsupported(v, n, 1, st);\n"
        "  g.BuildNodeGraphFromScratch(false, st);\n"
        "  OptimizationProcessorWarpSolver p(4096, 640 * 480, 4096 * 8);\n"
        "  return (int)g.GetNodeSize() + (int)p.SolvedSE3().Size();\n"
        "}\n"
        "int main(int argc, char **) { return argc > 100 ? use(nullptr, 0, 0) : 0; }\n")
    lib_dir = ROOT / "starhub_b200"
    cmd = ["g++", "-std=c++17", "-Wall", "-Wextra", "-I", str(ROOT / "include"), "-I", str(cuda / "include"),
           str(src), "-o", str(tmp_path / "facade"), "-L", str(lib_dir), "-lwarpsolve", "-L", str(cuda / "lib64"),
           "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_app_call_site_compiles_against_the_facade(lib, tmp_path):
    """tests/facade_app_callsite.cpp holds the pipeline's solver call site as
    examples/mono_star/app.cu:45-150 writes it (processor constructed from the process-wide
    configuration, ProcessFrame with the seven input structs, the frame index and the stream,
    SolvedSE3() taken as GArrayView<DualQuaternion>), with `star::b200` for `star`.  It compiles
    and links against the facade and the library."""
    import shutil
    import subprocess
    cuda = Path("/usr/local/cuda")
    if shutil.which("g++") is None or not (cuda / "include" / "cuda_runtime.h").exists():
        pytest.skip("g++ or the CUDA headers are missing")
    lib_dir = ROOT / "starhub_b200"
    cmd = ["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"), "-I",
           str(cuda / "include"), str(ROOT / "tests" / "facade_app_callsite.cpp"), "-o", str(tmp_path / "app"),
           "-L", str(lib_dir), "-lwarpsolve", "-L", str(cuda / "lib64"), "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
