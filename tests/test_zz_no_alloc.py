"""vsg_integrate_noalloc -- integration for callers that cannot allocate
device memory (real-time loops that must not stall on cudaMalloc, hosts with
a fixed memory budget, plug-in hosts whose allocator owns device memory).  Its per-pixel work
buffers live in a fixed device array inside the library instead of buffers
the scene grows with cudaMalloc.

The same frames go through vsg_integrate into one scene and through
vsg_integrate_noalloc into another; after each of two calls in a row the two
volumes must agree (identical block sets, weights and colours, SDF within
1e-5 m -- in fact bit for bit).  The file sorts last so that a run stopping
at the first failure has already run every other test; it also passes alone
in a fresh process.
"""
import numpy as np
import pytest

from parity_util import compare_volumes

pytestmark = pytest.mark.gpu

VSG_ERR_TOO_LARGE = 5


def test_noalloc_integration_matches_integrate(cuda, synth_mod):
    import vsg

    W, H = 320, 240
    fr, K = synth_mod.tabletop_stream(5, 2, W, H)
    kw = dict(voxel_size=0.004, truncation=0.02, hash_num_slots=50021, num_sdf_blocks=60000)
    with_alloc = vsg.Scene(**kw)
    no_alloc = vsg.Scene(**kw)
    maps = [(cuda.from_numpy(f.pointmap).cuda(), cuda.from_numpy(f.rgb).cuda(), cuda.from_numpy(f.normals).cuda())
            for f in fr]
    cuda.cuda.synchronize()
    for i, (pm, rgb, nm) in enumerate(maps):
        f = fr[i]
        with_alloc.integrate(pm, rgb, nm, W, H, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
        cuda.cuda.synchronize()
        free_before = cuda.cuda.mem_get_info()[0]
        no_alloc.integrate_noalloc(pm, rgb, nm, W, H, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
        cuda.cuda.synchronize()
        if i > 0:
            # the first call on the device may load the library's module that
            # holds the work array; later calls must take no device memory
            assert cuda.cuda.mem_get_info()[0] >= free_before
        rc, rv = with_alloc.export()
        nc, nv = no_alloc.export()
        v = compare_volumes(nc, nv, rc, rv)
        assert v["same_blocks"], v
        assert v["weight_mismatch"] == 0 and v["rgb_mismatch"] == 0, v
        assert v["sdf_max_err"] <= 1e-5, v
        assert v["bit_exact"], v
        sa, sn = with_alloc.stats(), no_alloc.stats()
        for key in ("allocated_blocks", "frame_new_blocks", "frame_visible_blocks", "frame_updated_blocks",
                    "frame_updated_voxels", "frame_valid_pixels", "integrated_frames", "flags"):
            assert sa[key] == sn[key], (key, sa[key], sn[key])
        assert sn["frame_updated_voxels"] > 0
        # the scene's own per-pixel buffers were never grown
        assert sn["pixel_buffer_capacity"] == 0 and sa["pixel_buffer_capacity"] >= W * H


def test_noalloc_rejects_frames_beyond_its_array(cuda):
    import vsg

    sc = vsg.Scene(voxel_size=0.004, hash_num_slots=1021, num_sdf_blocks=2000)
    buf = cuda.zeros(16, device="cuda")
    pose = np.eye(4, dtype=np.float32)
    L = vsg.lib()
    # 1025 x 1024 pixels is one row more than the 1,048,576-pixel array;
    # the call must refuse before touching the (too small) buffers
    rc = L.vsg_integrate_noalloc(sc.h, buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 1024, 1025, 0.02,
                                 pose.ctypes.data, 525.0, 525.0, 319.5, 239.5, 0)
    assert rc == VSG_ERR_TOO_LARGE
    assert sc.stats()["integrated_frames"] == 0
