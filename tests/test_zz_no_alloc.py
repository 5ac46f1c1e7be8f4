"""The allocation-free entry point (cc_ogc_radii_noalloc) against the regular
detection entry point (cc_world_detect), through the C ABI on the GPU.

The entry point exists for callers that cannot call cudaMalloc (a fixed-budget
frame worker that cannot absorb an allocation's device-wide synchronisation, or
a host that pre-reserves all device memory): it keeps its per-vertex scratch in
a static device array. This test plays such a caller: it owns every input and
output buffer (allocated here with torch), calls the entry point twice in a
row - the second call reuses the scratch the first one left behind - and
checks both results against cc_world_detect's radii and minimum distance.
The tolerance is the one the OGC parity tests use: bit-identical FP64.

This file is collected last so that a run that stops at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from clothcraft_b200 import abi, native, scenes
from clothcraft_b200.vbd import OgcWorld

pytestmark = pytest.mark.gpu

MAX_VERTICES = 262144


def contact_positions():
    sc = scenes.small_sheet(24, seed=7, height=0.104, side=0.2, pins=(), radius=0.002)
    rng = np.random.default_rng(3)
    x = sc.x0.copy()
    x[:, 1] -= 0.0036
    x += rng.uniform(-2e-4, 2e-4, x.shape)
    obs = sc.obstacle
    x_all = np.ascontiguousarray(np.concatenate([x, obs.vertices]))
    tris = np.ascontiguousarray(np.concatenate([sc.mesh.triangles, obs.triangles + sc.n]).astype(np.uint32))
    return x_all, tris, sc.n


def test_noalloc_radii_match_world_detect_on_two_calls_in_a_row():
    import torch

    L = native.load()
    x_all, tris, moving = contact_positions()
    rq, r, relaxation = 0.008, 0.002, 0.45
    world = OgcWorld(x_all, tris, moving)
    ref = world.detect(x_all, rq, abi.cc_ogc_settings(r, 1e4, relaxation, 0.01))
    assert ref["vertex_face_candidates"] + ref["edge_edge_candidates"] > 0
    vf, ee = world.candidates(x_all, rq)
    edges = world.edges()

    dev = torch.device("cuda", 0)

    def dev_u32(a):  # uint32 bits in an int32 tensor owned by this caller
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).to(dev)

    x_d = torch.from_numpy(x_all).to(dev)
    tri_d, edge_d, vf_d, ee_d = dev_u32(tris), dev_u32(edges), dev_u32(vf), dev_u32(ee)
    stream = torch.cuda.current_stream(dev)
    # every output buffer exists before the calls, so the device's free memory
    # can only change if the entry point itself allocates
    bufs = [(torch.full((moving,), -1.0, dtype=torch.float64, device=dev),
             torch.full((1,), -1.0, dtype=torch.float64, device=dev)) for _ in range(2)]
    torch.cuda.synchronize()
    outs, free = [], []
    for radii_d, min_d in bufs:
        free.append(torch.cuda.mem_get_info(dev)[0])
        rc = L.cc_ogc_radii_noalloc(
            x_d.data_ptr(), len(x_all), moving, tri_d.data_ptr(), len(tris), edge_d.data_ptr(), len(edges),
            vf_d.data_ptr(), len(vf), ee_d.data_ptr(), len(ee), rq, relaxation, radii_d.data_ptr(),
            min_d.data_ptr(), C.c_void_p(stream.cuda_stream))
        assert rc == abi.CC_OK
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info(dev)[0])
    # the second call (its kernels already loaded by the first) leaves the
    # device's free memory as it found it: no allocation on this path
    assert free[3] == free[2], free
    for radii_d, min_d in bufs:
        outs.append((radii_d.cpu().numpy(), float(min_d.item())))
    for radii, md in outs:
        assert np.array_equal(radii.view(np.uint64), ref["radii"].view(np.uint64))
        assert np.float64(md).view(np.uint64) == np.float64(ref["minimum_distance"]).view(np.uint64)


def test_noalloc_rejects_more_vertices_than_its_scratch_holds():
    L = native.load()
    rc = L.cc_ogc_radii_noalloc(None, MAX_VERTICES + 1, 1, None, 0, None, 0, None, 0, None, 0, 0.01, 0.45, None,
                                None, None)
    assert rc == abi.CC_ERR_INVALID_ARGUMENT
    buf = C.create_string_buffer(512)
    L.cc_global_last_error(buf, 512)
    assert b"exceed the static scratch limit" in buf.value
