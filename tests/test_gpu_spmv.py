"""Standalone block-SpMV (ws_spmv) against the host product with the assembled system.

y = A x over the symmetric block store (diagonal per node, one block per pair read
transposed for the lower-triangle slot) must equal the block-CSR product of the expanded
system that ws_get_system returns, for every scene of a batch at once.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _host_spmv(system, x):
    rp, cols, blocks = system["rowptr"], system["cols"], system["blocks"]
    y = np.zeros((len(rp) - 1, 6), np.float64)
    for r in range(len(rp) - 1):
        for k in range(rp[r], rp[r + 1]):
            y[r] += blocks[k].reshape(6, 6).astype(np.float64) @ x[cols[k], :6].astype(np.float64)
    return y


@pytest.mark.parametrize("precision", [0, 1])
def test_spmv_matches_host_product(ws, small_scene, tiny_scene, precision):
    import torch
    from starhub_b200.solver import DeviceScene, WarpSolver
    scenes = [small_scene, tiny_scene]
    ds = [DeviceScene.from_scene(s) for s in scenes]
    s = WarpSolver(max_nodes=sum(d.num_nodes for d in ds), max_pixels=sum(d.num_pixels for d in ds),
                   max_edges=sum(d.num_edges for d in ds), max_scenes=2, precision=precision)
    s.SetBatchInputs(ds)
    st = torch.cuda.Stream()
    s.SolveStreamed(2, 5, stream=st)
    s.Sync()
    n_tot = sum(d.num_nodes for d in ds)
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn((n_tot, 8), device="cuda", generator=g)
    y = torch.full((n_tot, 8), float("nan"), device="cuda")
    s.spmv(x, y, stream=st)
    st.synchronize()
    xh, yh = x.cpu().numpy(), y.cpu().numpy()
    base = 0
    for i, d in enumerate(ds):
        ref = _host_spmv(s.system(i), xh[base:base + d.num_nodes])
        got = yh[base:base + d.num_nodes, :6]
        scale = np.abs(ref).max()
        np.testing.assert_allclose(got, ref, atol=1e-5 * scale, rtol=0)
        base += d.num_nodes


@pytest.mark.parametrize("precision", [0, 1])
def test_matrix_free_equals_materialised(ws, small_scene, tiny_scene, precision):
    """The operator applied from the term records equals the assembled matrix's product:
    an independent path through the same Jacobians checks the whole assembly."""
    import torch
    from starhub_b200.solver import DeviceScene, WarpSolver
    ds = [DeviceScene.from_scene(s) for s in (small_scene, tiny_scene)]
    s = WarpSolver(max_nodes=sum(d.num_nodes for d in ds), max_pixels=sum(d.num_pixels for d in ds),
                   max_edges=sum(d.num_edges for d in ds), max_scenes=2, precision=precision)
    s.SetBatchInputs(ds)
    st = torch.cuda.Stream()
    s.SolveStreamed(2, 5, stream=st)
    s.Sync()
    n_tot = sum(d.num_nodes for d in ds)
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn((n_tot, 8), device="cuda", generator=g)
    ya = torch.zeros_like(x)
    yb = torch.zeros_like(x)
    s.spmv(x, ya, stream=st)
    s.spmv_matrix_free(x, yb, stream=st)
    st.synchronize()
    a, b = ya[:, :6].cpu().numpy(), yb[:, :6].cpu().numpy()
    np.testing.assert_allclose(b, a, atol=2e-5 * np.abs(a).max(), rtol=0)
