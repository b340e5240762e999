"""The allocation-free solver-map splat (ws_splat_maps_noalloc) against ws_splat_maps.

Some callers cannot allocate device memory once running: a frame loop or serving
process that reserves its device budget at start-up and admits work by footprint, or
a host whose own memory pool owns the device.  ws_splat_maps_noalloc serves them from
a fixed scratch array in the library's static device memory.  Its outputs must equal
the allocating entry point's exactly (the maps are integer ids and copied vectors),
on two calls in a row with different inputs, so a stale scratch would show.
This file is collected last; it runs the same alone or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _splat(lib, fn, verts, attr_v, attr_n, cam, footprint, stream):
    import torch
    idx = torch.empty((cam.height, cam.width), dtype=torch.int32, device="cuda")
    vm = torch.empty((cam.height, cam.width, 4), dtype=torch.float32, device="cuda")
    nm = torch.empty((cam.height, cam.width, 4), dtype=torch.float32, device="cuda")
    st = fn(C.c_void_p(verts.data_ptr()), C.c_void_p(attr_v.data_ptr()), C.c_void_p(attr_n.data_ptr()),
            int(verts.shape[0]), cam.width, cam.height, cam.fx, cam.fy, cam.cx, cam.cy, footprint,
            C.c_void_p(idx.data_ptr()), C.c_void_p(vm.data_ptr()), C.c_void_p(nm.data_ptr()),
            C.c_void_p(stream.cuda_stream))
    assert st == 0, st
    stream.synchronize()
    return idx.cpu().numpy().view(np.uint32), vm.cpu().numpy(), nm.cpu().numpy()


def test_noalloc_splat_equals_allocating_splat(ws):
    import torch
    from starhub_b200 import _lib, scenes
    lib = _lib.load()
    rng = np.random.default_rng(17)
    p, n = scenes.sample_torus(rng, 120_000, 0.3, 0.1)
    p = p @ scenes.rot_x(30.0).T + np.array([0.0, 0.0, 1.0])
    verts = torch.from_numpy(scenes.pack4(p, 1.0)).cuda()
    normals = torch.from_numpy(scenes.pack4(n, 0.002)).cuda()
    cam = scenes.Camera(640, 480, 570.0, 570.0, 320.0, 240.0)
    stream = torch.cuda.Stream()
    # two calls in a row; the second one sees a shifted, smaller surface, so keys left in the
    # scratch by the first call would change its result if they were not cleared
    inputs = [(verts, 1), (verts * torch.tensor([0.6, 0.6, 1.3, 1.0], device="cuda"), 2)]
    for v, fp in inputs:
        a = _splat(lib, lib.ws_splat_maps, v, v, normals, cam, fp, stream)
        b = _splat(lib, lib.ws_splat_maps_noalloc, v, v, normals, cam, fp, stream)
        assert (a[0] != 0xFFFFFFFF).sum() > 1000
        np.testing.assert_array_equal(b[0], a[0])
        np.testing.assert_array_equal(b[1], a[1])
        np.testing.assert_array_equal(b[2], a[2])


def test_noalloc_splat_rejects_images_above_the_limit(ws):
    from starhub_b200 import _lib
    lib = _lib.load()
    side = int(np.sqrt(_lib.WS_NOALLOC_MAX_PIXELS)) + 2
    dummy = C.c_void_p(1)   # never dereferenced: the size check comes first
    st = lib.ws_splat_maps_noalloc(dummy, None, None, 1, side, side, 1.0, 1.0, 0.0, 0.0, 1, dummy, None, None, None)
    assert st == _lib.WS_ERR_CAPACITY
