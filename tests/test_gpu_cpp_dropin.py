"""The C++ drop-in classes (include/voxelsg_b200.hpp) driven like the
reference's main loop give the same depths as the Python binding of the C
ABI, the same marching-cubes triangle count and the same stream-out set, and
a stream-out / stream-in round trip leaves the rendered depth unchanged
(needs a GPU; compiles the harness with g++)."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "real-time-depth-fusion-directional-tsdf_b200")
CUDA = "/usr/local/cuda"


@pytest.mark.parametrize("method", [1, 2])
def test_cpp_dropin_matches_binding(cuda, synth_mod, tmp_path, method):
    import vsg

    W, H, N = 160, 120, 3
    fr, K = synth_mod.tabletop_stream(2, N, W, H)
    d = str(tmp_path)
    for i, f in enumerate(fr):
        f.pointmap.astype(np.float32).tofile(os.path.join(d, f"pm_{i}.bin"))
        f.rgb.astype(np.uint8).tofile(os.path.join(d, f"rgb_{i}.bin"))
        f.normals.astype(np.float32).tofile(os.path.join(d, f"nm_{i}.bin"))
        f.pose.astype(np.float32).tofile(os.path.join(d, f"pose_{i}.bin"))
    exe = os.path.join(d, "dropin_frames")
    defs = ["-DUSE_NORMAL_DIR_ALLOC"] if method == 2 else []
    subprocess.run(["g++", "-O2", "-std=c++17", *defs, "-o", exe, os.path.join(ROOT, "tests", "cpp", "dropin_frames.cpp"),
                    "-I", os.path.join(ROOT, "include"), "-I", f"{CUDA}/include", "-L", PKG, "-lvsg",
                    f"-Wl,-rpath,{PKG}", "-L", f"{CUDA}/lib64", "-lcudart"], check=True)
    r = subprocess.run([exe, d, str(N), str(W), str(H), str(K.fx), str(K.fy), str(K.cx), str(K.cy), "0.004", "0.02",
                        "20011", "40000", "0.2", "3.0"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert f"frames={N}" in r.stdout
    sc = vsg.Scene(voxel_size=0.004, truncation=0.02, hash_num_slots=20011, num_sdf_blocks=40000)
    sc.set_alloc_method(method)
    rr = vsg.Renderer(W, H)
    for i, f in enumerate(fr):
        pm = cuda.from_numpy(f.pointmap).cuda()
        rgb = cuda.from_numpy(f.rgb).cuda()
        nm = cuda.from_numpy(f.normals).cuda()
        sc.integrate(pm, rgb, nm, W, H, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
        rr.render(sc, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
        ref = rr.download()["depth"]
        got = np.fromfile(os.path.join(d, f"depth_{i}.bin"), np.float32).reshape(H, W)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), i
        # Method 2 allocates only where its 2 cm rays cross a block boundary, so
        # its early frames hit fewer pixels
        assert (got < 1e9).sum() > (0.5 if method == 1 else 0.1) * W * H
    # the exporters of the last frame
    ply = tmp_path / "cloud_binding.ply"
    rr.save_ply(str(ply))
    assert (tmp_path / "cloud.ply").read_text() == ply.read_text()
    pts = vsg.SurfacePoints(1_000_000)
    pts.extract(sc, -0.1, 0.1, 1)
    assert f"surface_points={pts.count()}" in r.stdout
    assert (tmp_path / "surface.ply").read_text().count("\n") == pts.count() + 14
    mc = vsg.MarchingCubes(250000)
    mc.run(sc, voxel_size=0.004)
    assert f"triangles={min(mc.count(), 2**31 - 1)}" in r.stdout
    assert f"Integrated Frames: {N}" in r.stdout
    head = (tmp_path / "mesh.ply").read_text().splitlines()[:10]
    assert f"element vertex {3 * mc.count()}" in head and f"element face {mc.count()}" in head
    n_out = sc.stream_out(vsg.Store((0.1, 0.1, 0.1)), (0.0, 0.1, 0.0), 0.25)
    assert n_out > 0 and f"streamed_out={n_out} " in r.stdout
    assert f"found={n_out}" in r.stdout and f"streamed_in={n_out} " in r.stdout
    after = np.fromfile(os.path.join(d, "depth_after_stream.bin"), np.float32).reshape(H, W)
    assert np.array_equal(after.view(np.uint32), ref.view(np.uint32))


def test_cpp_depth_map_generator_matches_binding(cuda, synth_mod, tmp_path):
    """CustomDepthMapGenerator from the C++ header (generateFromPointCloud's
    call shape, CustomDepthMapGenerator.cpp:81-222) gives the maps of
    vsg.splat_points in the reference's last-point-wins order, bit for bit,
    with a shorter normal list and no colours."""
    import vsg

    fr, K = synth_mod.tabletop_stream(5, 2, 320, 240)
    T0 = np.asarray(fr[0].pose, np.float64)
    pts, nrm, col = [], [], []
    for f in fr:
        m = np.any(f.pointmap != 0, -1)
        M = np.linalg.inv(T0) @ np.asarray(f.pose, np.float64)
        pts.append((f.pointmap[m].astype(np.float64) @ M[:3, :3].T + M[:3, 3]).astype(np.float32))
        nrm.append((f.normals[m].astype(np.float64) @ M[:3, :3].T).astype(np.float32))
        col.append(f.rgb[m])
    P = np.concatenate(pts)
    N = np.concatenate(nrm)[: len(P) * 2 // 3]
    d = str(tmp_path)
    P.tofile(os.path.join(d, "points.bin"))
    N.tofile(os.path.join(d, "normals.bin"))
    open(os.path.join(d, "colors.bin"), "wb").close()
    exe = os.path.join(d, "splat_cloud")
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", exe, os.path.join(ROOT, "tests", "cpp", "splat_cloud.cpp"),
                    "-I", os.path.join(ROOT, "include"), "-I", f"{CUDA}/include", "-L", PKG, "-lvsg",
                    f"-Wl,-rpath,{PKG}", "-L", f"{CUDA}/lib64", "-lcudart"], check=True)
    r = subprocess.run([exe, d, str(len(P)), str(len(N)), "0", str(K.width), str(K.height), str(K.fx), str(K.fy),
                        str(K.cx), str(K.cy)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    want = vsg.splat_points(cuda.from_numpy(P).cuda(), K.width, K.height, K.fx, K.fy, K.cx, K.cy,
                            normals=cuda.from_numpy(N).cuda())
    H, W = K.height, K.width
    got = {"depth": np.fromfile(os.path.join(d, "depth.bin"), np.float32).reshape(H, W),
           "pointmap": np.fromfile(os.path.join(d, "pointmap.bin"), np.float32).reshape(H, W, 3),
           "normalmap": np.fromfile(os.path.join(d, "normalmap.bin"), np.float32).reshape(H, W, 3),
           "colormap": np.fromfile(os.path.join(d, "colormap.bin"), np.uint8).reshape(H, W, 3)}
    for k, g in got.items():
        assert np.array_equal(g.view(np.uint8), want[k].cpu().numpy().view(np.uint8)), k
    assert want["n_valid"] > 0.5 * W * H and not got["colormap"].any()


def test_wrong_device_is_refused_before_any_launch(cuda, tmp_path):
    """vsg_integrate / vsg_scene_reset / vsg_render / vsg_render_hostpose /
    vsg_scene_stats / vsg_scene_export / vsg_scene_lookup_blocks /
    vsg_renderer_record / vsg_renderer_download / vsg_batch_create with a
    handle recorded on another device return VSG_ERR_INVALID_ARG and touch
    nothing (tests/cpp/device_guard.cu)."""
    from test_cpp_dropin_build import build_device_guard

    exe = build_device_guard(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "device_guard ok" in r.stdout, r.stdout + r.stderr
