"""CUDA path vs the CPU oracle on seeded synthetic streams (needs a GPU).

Bar: allocated block sets and voxel weights/colours equal, SDF within 1e-5 m
(the kernels are in fact compared bit for bit), raycast depth within 1e-4 m
on >= 99.9 % of pixels with max and RMS error reported.
"""
import numpy as np
import pytest

from parity_util import compare_renders, compare_volumes

pytestmark = pytest.mark.gpu

SDF_TOL = 1e-5
DEPTH_TOL = 1e-4
DEPTH_FRAC = 0.999


def _upload(torch, f):
    pm = torch.from_numpy(np.ascontiguousarray(f.pointmap)).cuda()
    rgb = torch.from_numpy(np.ascontiguousarray(f.rgb)).cuda()
    nm = torch.from_numpy(np.ascontiguousarray(f.normals)).cuda()
    return pm, rgb, nm


def _run_stream(torch, oracle_mod, frames, K, trunc=0.02, voxel=0.004, slots=200000, blocks=200000,
                render_every=1, check_every=1, min_d=0.2, max_d=3.0, alloc_method=1, **scene_kw):
    import vsg

    sc = vsg.Scene(voxel_size=voxel, hash_num_slots=slots, num_sdf_blocks=blocks, truncation=trunc, **scene_kw)
    rr = vsg.Renderer(K.width, K.height)
    orc = oracle_mod.OracleScene(voxel)
    if alloc_method != 1:
        sc.set_alloc_method(alloc_method)
        orc.set_alloc_method(alloc_method)
    reports = []
    for i, f in enumerate(frames):
        pm, rgb, nm = _upload(torch, f)
        sc.integrate(pm, rgb, nm, K.width, K.height, trunc, f.pose, K.fx, K.fy, K.cx, K.cy)
        ost = orc.integrate(f.pointmap, f.rgb, trunc, f.pose, K.fx, K.fy, K.cx, K.cy, normals=f.normals)
        rep = {"frame": i, "oracle": ost}
        if i % check_every == 0 or i == len(frames) - 1:
            gc, gv = sc.export()
            oc, ov = orc.export()
            rep["volume"] = compare_volumes(gc, gv, oc, ov["raw"])
            rep["stats"] = sc.stats()
        if i % render_every == 0 or i == len(frames) - 1:
            rr.render(sc, f.pose, K.fx, K.fy, K.cx, K.cy, min_d, max_d)
            g = rr.download()
            o = orc.render(K.width, K.height, f.pose, K.fx, K.fy, K.cx, K.cy, min_d, max_d)
            rep["render"] = compare_renders(g, o, DEPTH_TOL)
        reports.append(rep)
    sc.close()
    rr.close()
    return reports


def _triangle_digests(verts, norms):
    """Sorted 64-bit digest per triangle of its 18 floats' bit patterns."""
    m = verts.shape[0]
    words = np.concatenate([verts.reshape(m, 9).view(np.uint32), norms.reshape(m, 9).view(np.uint32)], 1)
    h = np.full(m, 0x9E3779B97F4A7C15, np.uint64)
    with np.errstate(over="ignore"):
        for k in range(18):
            h ^= words[:, k].astype(np.uint64) + np.uint64(0x632BE59BD9B4E019) + (h << np.uint64(6)) + (h >> np.uint64(2))
            h *= np.uint64(0xBF58476D1CE4E5B9)
    h.sort()
    return h


def _assert_reports(reports):
    for rep in reports:
        if "volume" in rep:
            v = rep["volume"]
            assert v["same_blocks"], rep
            assert v["weight_mismatch"] == 0, rep
            assert v["rgb_mismatch"] == 0, rep
            assert v["sdf_max_err"] <= SDF_TOL, rep
            assert rep["stats"]["flags"] == 0, rep
            assert rep["stats"]["frame_new_blocks"] == rep["oracle"]["new_blocks"], rep
            assert rep["stats"]["frame_updated_blocks"] == rep["oracle"]["updated_blocks"], rep
            assert rep["stats"]["frame_updated_voxels"] == rep["oracle"]["updated_voxels"], rep
        if "render" in rep:
            r = rep["render"]
            assert r["frac_within_tol"] >= DEPTH_FRAC, rep


@pytest.mark.parametrize("wh,frames", [((160, 120), 6), ((320, 240), 3)])
def test_tabletop_small(cuda, oracle_mod, synth_mod, wh, frames):
    fr, K = synth_mod.tabletop_stream(0, frames, wh[0], wh[1])
    reports = _run_stream(cuda, oracle_mod, fr, K)
    for r in reports:
        print(r)
    _assert_reports(reports)
    # the kernels restate the reference bit for bit
    assert all(r["volume"]["bit_exact"] for r in reports if "volume" in r)
    assert all(r["render"]["bit_exact_all"] for r in reports if "render" in r)
    # the fixed-divisor division passed its exhaustive check for 4 mm, and
    # every running-average divisor its check
    assert reports[-1]["stats"]["fast_division"] == 1
    assert reports[-1]["stats"]["fast_avg_divisors"] == 256


def test_tabletop_full_size(cuda, oracle_mod, synth_mod):
    """640x480, 4 mm, trunc 0.02, 200000 slots: first frames of the stream."""
    fr, K = synth_mod.tabletop_stream(0, 3)
    reports = _run_stream(cuda, oracle_mod, fr, K, render_every=2)
    for r in reports:
        print(r)
    _assert_reports(reports)


def test_tabletop_full_stream_30_frames(cuda, oracle_mod, synth_mod):
    """The whole timed workload: 30 frames 640x480, 4 mm, trunc 0.02, 200000
    slots and blocks, min/max depth 0.2/3.0 m.  The volume is compared with
    the oracle after every frame (the later frames grow the volume, the
    overflow chains and the skip grids) and the full-frame ray cast every
    5th frame and at the last, all bit for bit."""
    fr, K = synth_mod.tabletop_stream(0, 30)
    reports = _run_stream(cuda, oracle_mod, fr, K, render_every=5)
    _assert_reports(reports)
    assert all(r["volume"]["bit_exact"] for r in reports)
    renders = [r["render"] for r in reports if "render" in r]
    assert len(renders) == 7
    for r in renders:
        assert r["bit_exact_all"] and r["hits_gpu"] > 0.5 * r["pixels"], r
    print({"blocks": reports[-1]["volume"]["gpu_blocks"],
           "depth_max_err": max(r["depth_max_err"] for r in renders),
           "depth_rms_err": max(r["depth_rms_err"] for r in renders)})


def test_other_seed_and_truncation(cuda, oracle_mod, synth_mod):
    fr, K = synth_mod.tabletop_stream(7, 4, 200, 150)
    reports = _run_stream(cuda, oracle_mod, fr, K, trunc=0.012, voxel=0.003, slots=50021, blocks=120000)
    _assert_reports(reports)


def test_tiny_hash_forces_overflow_chains(cuda, oracle_mod, synth_mod):
    """Few buckets: most inserts go to the linked-list overflow; the
    allocated set must still be exactly the oracle's."""
    fr, K = synth_mod.tabletop_stream(3, 3, 160, 120)
    reports = _run_stream(cuda, oracle_mod, fr, K, slots=257, blocks=60000, max_chain_nodes=60000)
    _assert_reports(reports)
    assert reports[-1]["stats"]["chain_nodes_used"] > 0


def test_render_empty_scene_leaves_outputs(cuda, synth_mod):
    """With no allocated block the reference returns before launching and
    the output buffers keep their contents (RayCastRender.cu:552-555)."""
    import vsg

    fr, K = synth_mod.tabletop_stream(0, 1, 64, 48)
    sc = vsg.Scene(hash_num_slots=5000, num_sdf_blocks=20000)
    rr = vsg.Renderer(K.width, K.height)
    pm, rgb, nm = _upload(cuda, fr[0])
    sc.integrate(pm, rgb, nm, K.width, K.height, 0.02, fr[0].pose, K.fx, K.fy, K.cx, K.cy)
    rr.render(sc, fr[0].pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    first = rr.download()
    assert (first["depth"] < 1e9).any()
    sc.reset()
    assert sc.stats()["allocated_blocks"] == 0
    rr.render(sc, np.eye(4), K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    second = rr.download()
    for k in first:
        assert np.array_equal(first[k].view(np.uint32), second[k].view(np.uint32)), k


def test_room_1280x720_2mm(cuda, oracle_mod, synth_mod, hosttest_lib):
    """The room workload: 1280x720 frames of a seeded 4x3x2.5 m room with 40
    boxes and 20 spheres on a random walk, 2 mm voxels, truncation 0.01 m,
    2^20 buckets and pool blocks.  Volumes bit-exact after every frame; the
    last frame's full ray cast (depth, position, colour, normal) bit-exact;
    marching cubes over the room volume equal to the oracle's extraction
    from its own volume, triangle for triangle."""
    import ctypes

    import vsg

    fr, K = synth_mod.room_stream(1, 8, 1280, 720)
    voxel, trunc = 0.002, 0.01
    sc = vsg.Scene(voxel_size=voxel, truncation=trunc, hash_num_slots=1 << 20, num_sdf_blocks=1 << 20)
    rr = vsg.Renderer(K.width, K.height)
    orc = oracle_mod.OracleScene(voxel)
    for i, f in enumerate(fr):
        pm, rgb, nm = _upload(cuda, f)
        sc.integrate(pm, rgb, nm, K.width, K.height, trunc, f.pose, K.fx, K.fy, K.cx, K.cy)
        ost = orc.integrate(f.pointmap, f.rgb, trunc, f.pose, K.fx, K.fy, K.cx, K.cy)
        gc, gv = sc.export()
        oc, ov = orc.export()
        v = compare_volumes(gc, gv, oc, ov["raw"])
        assert v["same_blocks"] and v["bit_exact"], (i, v)
        st = sc.stats()
        assert st["flags"] == 0 and st["frame_new_blocks"] == ost["new_blocks"]
        assert st["frame_updated_voxels"] == ost["updated_voxels"]
    f = fr[-1]
    rr.render(sc, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 4.0)
    g = rr.download()
    o = orc.render(K.width, K.height, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 4.0)
    r = compare_renders(g, o, DEPTH_TOL)
    print(r)
    assert r["bit_exact_all"] and r["hits_gpu"] > 0.5 * r["pixels"], r
    # marching cubes (MarchingCubes.cu:352-571) over the room volume
    tab = np.zeros((256, 16), np.uint8)
    hosttest_lib.vsg_test_mc_table.argtypes = [ctypes.c_void_p]
    hosttest_lib.vsg_test_mc_table(tab.ctypes.data)
    probe = vsg.MarchingCubes(1)
    probe.run(sc)
    need = probe.count()
    probe.close()
    mc = vsg.MarchingCubes(need)
    mc.run(sc)
    n, verts, norms = mc.download()
    on, ov_, onrm = orc.marching_cubes(tab, 0.0, voxel, need)
    assert n == on == need > 100000
    # ~10^7 triangles: compared as sorted multisets of 64-bit digests of
    # their 18 floats' bit patterns (both sides append in an unspecified order)
    assert np.array_equal(_triangle_digests(verts, norms), _triangle_digests(ov_, onrm))
    mc.close()
    sc.close()
    rr.close()


@pytest.mark.parametrize("wh,frames,slots", [((160, 120), 6, 200000), ((320, 240), 3, 200000),
                                             ((160, 120), 4, 257)])
def test_normal_direction_allocation(cuda, oracle_mod, synth_mod, wh, frames, slots):
    """Method 2 (allocBlocksFromDepthMapMethod2Kernel, VoxelScene.cu:768-912,
    and the parent-pixel integration branch, :1015-1035): volumes bit-exact
    against the oracle frame by frame, renders within tolerance (257 buckets:
    most blocks in overflow chains)."""
    fr, K = synth_mod.tabletop_stream(2, frames, wh[0], wh[1])
    kw = dict(slots=slots, blocks=200000, max_chain_nodes=200000)
    reports = _run_stream(cuda, oracle_mod, fr, K, alloc_method=2, **kw)
    _assert_reports(reports)
    assert all(r["volume"]["bit_exact"] for r in reports if "volume" in r)
    # the mode allocates a different block set than the camera-z band
    one = _run_stream(cuda, oracle_mod, fr[:1], K, **kw)
    assert one[0]["oracle"]["blocks"] != reports[0]["oracle"]["blocks"]


def test_normal_direction_allocation_mixed_resolutions(cuda, oracle_mod, synth_mod):
    """Parents recorded at one resolution and checked against the next
    frame's image bounds (VoxelScene.cu:1019-1021): alternating 320x240 and
    160x120 frames of one scene, volumes bit-exact against the oracle."""
    import vsg

    big, Kb = synth_mod.tabletop_stream(4, 4, 320, 240)
    small, Ks = synth_mod.tabletop_stream(4, 4, 160, 120)
    sc = vsg.Scene(voxel_size=0.004, hash_num_slots=200000, num_sdf_blocks=200000, truncation=0.02)
    sc.set_alloc_method(2)
    orc = oracle_mod.OracleScene(0.004)
    orc.set_alloc_method(2)
    for i in range(4):
        f, K = (big[i], Kb) if i % 2 == 0 else (small[i], Ks)
        pm, rgb, nm = _upload(cuda, f)
        sc.integrate(pm, rgb, nm, K.width, K.height, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
        orc.integrate(f.pointmap, f.rgb, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy, normals=f.normals)
        gc, gv = sc.export()
        oc, ov = orc.export()
        v = compare_volumes(gc, gv, oc, ov["raw"])
        assert v["same_blocks"] and v["bit_exact"], (i, v)
        assert sc.stats()["flags"] == 0
    sc.close()


def test_normal_direction_allocation_refused_where_unsupported(cuda, synth_mod):
    import vsg

    fr, K = synth_mod.tabletop_stream(0, 1, 64, 48)
    sc = vsg.Scene(voxel_size=0.004, hash_num_slots=20011, num_sdf_blocks=20000, truncation=0.02)
    sc.set_alloc_method(2)
    pm, rgb, nm = _upload(cuda, fr[0])
    with pytest.raises(vsg.VsgError):
        sc.integrate_noalloc(pm, rgb, nm, K.width, K.height, 0.02, fr[0].pose, K.fx, K.fy, K.cx, K.cy)
    with pytest.raises(vsg.VsgError):
        sc.set_alloc_method(3)
    sc.close()


def test_ragged_and_invalid_inputs(cuda, oracle_mod, synth_mod):
    """An image size that fills no tile evenly (157x113), then the same frames
    with NaN, infinite, behind-camera and zero points mixed in, then an
    all-zero frame: volumes bit-exact against the oracle after every frame,
    renders within tolerance, and the coordinate-range flag raised exactly
    when the oracle drops out-of-range blocks (VoxelScene.cu:547-633 lets NaN
    depths through its z test, as the oracle does)."""
    import vsg

    fr, K = synth_mod.tabletop_stream(6, 4, 157, 113)
    rng = np.random.default_rng(9)
    frames = [fr[0], fr[1]]
    for f in fr[2:]:
        pm = f.pointmap.copy()
        u = rng.random(pm.shape[:2])
        pm[u < 0.05] = np.nan
        pm[(u >= 0.05) & (u < 0.07)] = np.inf
        neg = (u >= 0.07) & (u < 0.10)
        pm[neg, 2] = -pm[neg, 2]
        pm[(u >= 0.10) & (u < 0.20)] = 0.0
        frames.append(type(f)(pointmap=pm, rgb=f.rgb, normals=f.normals, depth=f.depth, pose=f.pose))
    z = fr[0]
    frames.append(type(z)(pointmap=np.zeros_like(z.pointmap), rgb=z.rgb, normals=z.normals, depth=z.depth,
                          pose=fr[3].pose))
    sc = vsg.Scene(voxel_size=0.004, hash_num_slots=20011, num_sdf_blocks=60000, truncation=0.02)
    rr = vsg.Renderer(K.width, K.height)
    orc = oracle_mod.OracleScene(0.004)
    for i, f in enumerate(frames):
        pm, rgb, nm = _upload(cuda, f)
        sc.integrate(pm, rgb, nm, K.width, K.height, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
        orc.integrate(f.pointmap, f.rgb, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
        gc, gv = sc.export()
        oc, ov = orc.export()
        v = compare_volumes(gc, gv, oc, ov["raw"])
        assert v["same_blocks"] and v["bit_exact"], (i, v)
        drops = orc.L.orc_coord_range_drops(orc.h)
        assert bool(sc.stats()["flags"] & vsg.FLAG_COORD_RANGE) == (drops > 0), (i, drops)
        assert sc.stats()["flags"] & ~vsg.FLAG_COORD_RANGE == 0
        rr.render(sc, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
        o = orc.render(K.width, K.height, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
        assert compare_renders(rr.download(), o, DEPTH_TOL)["frac_within_tol"] >= DEPTH_FRAC, i
    sc.close()
    rr.close()


def test_render_call_forms(cuda, oracle_mod, synth_mod):
    """RayCastRender::render's argument forms (RayCastRender.cpp:123-183,
    RayCastRender.cu:500-505): a device pose gives the host-pose result bit
    for bit; a camera position apart from the pose's translation is honoured
    as the reference honours it (the oracle with the same camera); a minimum
    or maximum depth of 0 or MINF leaves every output at MINF."""
    import vsg

    fr, K = synth_mod.tabletop_stream(8, 3, 160, 120)
    sc = vsg.Scene(voxel_size=0.004, hash_num_slots=20011, num_sdf_blocks=60000, truncation=0.02)
    orc = oracle_mod.OracleScene(0.004)
    for f in fr:
        pm, rgb, nm = _upload(cuda, f)
        sc.integrate(pm, rgb, nm, K.width, K.height, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
        orc.integrate(f.pointmap, f.rgb, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
    rr = vsg.Renderer(K.width, K.height)
    T = np.asarray(fr[-1].pose, np.float32)
    rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    host = rr.download()
    Td = cuda.from_numpy(np.ascontiguousarray(T.reshape(16))).cuda()
    rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0, pose_dev=Td.data_ptr())
    dev = rr.download()
    for k in ("depth", "position", "color", "normal"):
        assert np.array_equal(host[k].view(np.uint32), dev[k].view(np.uint32)), k
    cam = (T[:3, 3] + np.array([0.01, -0.02, 0.015], np.float32)).astype(np.float32)
    rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0, cam_pos=cam)
    want = orc.render(K.width, K.height, T, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0, cam=cam)
    r = compare_renders(rr.download(), want, DEPTH_TOL)
    assert r["bit_exact_all"], r
    for lo, hi in ((0.0, 3.0), (1e10, 3.0), (0.2, 0.0), (0.2, 1e10)):
        rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, lo, hi)
        out = rr.download()
        for k in ("depth", "position", "color", "normal"):
            assert np.all(out[k] == np.float32(1e10)), (lo, hi, k)
    sc.close()
    rr.close()
