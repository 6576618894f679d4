"""Voxel-wise surface-point extraction (vsg_points_*, vsg_extract_points)
against the oracle's restatement of kernelExtractSurfacePoints
(RayCastRender.cu:683-868) on the same volume, bit for bit: positions,
colours and SDF-gradient normals.  The GPU volume is read back into the
oracle; both sides append points in an unspecified order, so points are
compared as sorted multisets of their 12 floats (needs a GPU)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rows(P, C, N):
    a = np.concatenate([P.view(np.uint32), C.view(np.uint32), N.view(np.uint32)], 1)
    return a[np.lexsort(a.T[::-1])]


def _scene(vsg, cuda, synth_mod, seed, W, H, frames, **kw):
    fr, K = synth_mod.tabletop_stream(seed, frames, W, H)
    sc = vsg.Scene(voxel_size=0.004, truncation=0.02, hash_num_slots=kw.get("slots", 20011),
                   num_sdf_blocks=60000)
    for f in fr:
        pm, rgb, nm = (cuda.from_numpy(x).cuda() for x in (f.pointmap, f.rgb, f.normals))
        sc.integrate(pm, rgb, nm, K.width, K.height, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
    return sc


def _oracle_of(oracle_mod, sc):
    coords, vox = sc.export()
    o = oracle_mod.OracleScene(0.004)
    o.load(coords, vox)
    return o


# (-0.1, 0.1, 5) is what the reference's main loop asks for (voxelSG.cpp:661);
# (-0.01, 0.01, 1) are the method's defaults (RayCastRender.h:99-102)
@pytest.mark.parametrize("min_sdf,max_sdf,min_w,slots", [(-0.1, 0.1, 5, 20011), (-0.01, 0.01, 1, 20011),
                                                          (-0.004, 0.02, 2, 257)])
def test_points_match_oracle(cuda, synth_mod, oracle_mod, min_sdf, max_sdf, min_w, slots):
    import vsg

    sc = _scene(vsg, cuda, synth_mod, 31, 160, 120, 5, slots=slots)
    probe = vsg.SurfacePoints(1)
    probe.extract(sc, min_sdf, max_sdf, min_w)
    need = probe.count()
    probe.close()
    pts = vsg.SurfacePoints(need)
    pts.extract(sc, min_sdf, max_sdf, min_w)
    n, P, C, N = pts.download()
    o = _oracle_of(oracle_mod, sc)
    on, oP, oC, oN = o.extract_points(min_sdf, max_sdf, min_w, need)
    assert n == on == need > 500
    assert np.array_equal(_rows(P, C, N), _rows(oP, oC, oN))
    ln = np.linalg.norm(N[:, :3].astype(np.float64), axis=1)
    assert np.all((np.abs(ln - 1) < 1e-5) | (ln == 0)) and (ln > 0).mean() > 0.9
    assert np.all(P[:, 3] == 1.0) and np.all(C[:, 3] == 1.0) and np.all(N[:, 3] == 0.0)


def test_points_capacity_empty_and_ply(cuda, synth_mod, oracle_mod, tmp_path):
    import vsg

    pts = vsg.SurfacePoints(100)
    empty = vsg.Scene(voxel_size=0.004, hash_num_slots=5003, num_sdf_blocks=8000)
    pts.extract(empty)
    assert pts.count() == 0
    sc = _scene(vsg, cuda, synth_mod, 32, 96, 72, 2)
    pts.extract(sc, -0.1, 0.1, 1)
    n, P, C, N = pts.download()
    o = _oracle_of(oracle_mod, sc)
    on, oP, oC, oN = o.extract_points(-0.1, 0.1, 1, n)
    assert n == on > 100 and P.shape[0] == 100
    full = {r.tobytes() for r in _rows(oP, oC, oN)}
    assert all(r.tobytes() in full for r in _rows(P, C, N))
    path = str(tmp_path / "pts.ply")
    pts.save_ply(path)
    lines = open(path).read().splitlines()
    assert lines[0] == "ply" and "element vertex 100" in lines and lines.index("end_header") == 13
    body = np.array([[float(x) for x in ln.split()] for ln in lines[14:]])
    assert body.shape == (100, 9) and np.all((body[:, 6:] >= 0) & (body[:, 6:] <= 255))


def test_raycast_point_cloud_ply(cuda, synth_mod, tmp_path):
    """vsg_renderer_save_ply (RayCastRender::savePointCloudPLY,
    RayCastRender.cpp:221-302) writes exactly the reference's text for the
    render's outputs: hits with depth in (0, 1e9) and finite positions, "%g"
    coordinates, colour clamped and rounded to 0..255; no file when nothing
    was hit."""
    import vsg

    fr, K = synth_mod.tabletop_stream(1, 3, 160, 120)
    sc = _scene(vsg, cuda, synth_mod, 1, 160, 120, 3)
    rr = vsg.Renderer(160, 120)
    rr.render(sc, fr[-1].pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    out = rr.download()
    path = tmp_path / "sub" / "cloud.ply"
    n = rr.save_ply(str(path))
    D, P, C = out["depth"].ravel(), out["position"].reshape(-1, 4), out["color"].reshape(-1, 4)
    ok = np.isfinite(D) & (D > 0) & (np.abs(D) < 1e9) & np.isfinite(P[:, :3]).all(1)
    assert n == int(ok.sum()) > 1000

    def ch(v):
        if not np.isfinite(v):
            return 255
        return int(np.float32(min(max(v, np.float32(0)), np.float32(1))) * np.float32(255) + np.float32(0.5))

    lines = ["ply", "format ascii 1.0", "comment Generated by RayCastRender", f"element vertex {n}",
             "property float x", "property float y", "property float z", "property uchar red",
             "property uchar green", "property uchar blue", "end_header"]
    for i in np.nonzero(ok)[0]:
        p, c = P[i], C[i]
        lines.append("%g %g %g %d %d %d" % (p[0], p[1], p[2], ch(c[0]), ch(c[1]), ch(c[2])))
    assert path.read_text() == "\n".join(lines) + "\n"
    # a view that hits nothing writes no file
    away = np.array(fr[-1].pose, np.float32)
    away[:3, 3] += 100.0
    rr.render(sc, away, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    empty = tmp_path / "none.ply"
    with pytest.raises(vsg.VsgError):
        rr.save_ply(str(empty))
    assert not empty.exists()
    rr.close()
    sc.close()
