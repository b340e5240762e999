"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libwarpsolve.so")


@pytest.fixture(scope="session")
def orc():
    import oracle as orc_mod
    orc_mod.build()
    return orc_mod


@pytest.fixture(scope="session")
def small_scene(orc):
    """Config-0 torus at reduced resolution: 320x240, 60k surfels, about 1.5k nodes, with the
    reference's own 4-NN node graph."""
    from starhub_b200 import scenes
    spec = scenes.config_spec(0, n_surfels=60_000, width=320, height=240, focal=285.0,
                              graph_k=scenes.REFERENCE_GRAPH_K)
    return scenes.make_scene(spec, orc.OracleGeometry(), seed=11)


@pytest.fixture(scope="session")
def small_scene_k8(orc):
    """The same reduced config-0 torus with the 8-NN node graph of the benchmark configurations."""
    from starhub_b200 import scenes
    spec = scenes.config_spec(0, n_surfels=60_000, width=320, height=240, focal=285.0,
                              graph_k=scenes.BASELINE_GRAPH_K)
    return scenes.make_scene(spec, orc.OracleGeometry(), seed=11)


@pytest.fixture(scope="session")
def tiny_scene(orc):
    """Small torus for fast CPU checks: 160x120, 12k surfels, scaled torus."""
    from starhub_b200 import scenes
    spec = scenes.config_spec(0, n_surfels=12_000, width=160, height=120, focal=142.5, scale=0.5,
                              graph_k=scenes.REFERENCE_GRAPH_K)
    return scenes.make_scene(spec, orc.OracleGeometry(), seed=5)


@pytest.fixture(scope="session")
def gpu_available():
    import torch
    return torch.cuda.is_available()


@pytest.fixture(scope="session")
def ws(gpu_available):
    if not gpu_available:
        pytest.skip("no CUDA device")
    from starhub_b200 import build as b
    b.build()
    import starhub_b200 as pkg
    return pkg
