"""The ray caster's per-tile distance bounds leave every output bit for bit
as the full march gives it (needs a GPU).

The bounds pre-pass clips the weighted blocks' boxes at half the minimum
depth, projects them onto 8x4 and 64x32 pixel tiles, and is disabled for
poses whose rotation is not orthonormal and for non-positive minimum depths.
These renders exercise each of those paths against the oracle, which always
marches every sample (RayCastRender.cu:276-398): a camera inside the volume
(blocks straddling the camera plane, both minimum depths), a camera far back,
a camera facing away from the scene, very wide and very narrow fields of
view, a scaled rotation and a negative minimum depth.
"""
import numpy as np
import pytest

from parity_util import compare_renders

pytestmark = pytest.mark.gpu

W, H, VOX, TRUNC = 160, 120, 0.004, 0.02


def _rot_y(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, 0.0, s], [0.0, 1.0, 0.0], [-s, 0.0, c]])


@pytest.fixture(scope="module")
def scene(cuda, oracle_mod, synth_mod):
    import vsg

    fr, K = synth_mod.tabletop_stream(5, 4, W, H)
    sc = vsg.Scene(voxel_size=VOX, hash_num_slots=20011, num_sdf_blocks=60000, truncation=TRUNC)
    orc = oracle_mod.OracleScene(VOX)
    for f in fr:
        pm, rgb, nm = (cuda.from_numpy(np.ascontiguousarray(x)).cuda() for x in (f.pointmap, f.rgb, f.normals))
        sc.integrate(pm, rgb, nm, W, H, TRUNC, f.pose, K.fx, K.fy, K.cx, K.cy)
        orc.integrate(f.pointmap, f.rgb, TRUNC, f.pose, K.fx, K.fy, K.cx, K.cy)
    coords, _ = sc.export()
    centre = (np.asarray(coords, np.float64).mean(axis=0) + 0.5) * 8 * VOX
    rr = vsg.Renderer(W, H)
    yield sc, orc, rr, fr, K, centre
    rr.close()
    sc.close()


def _check(scene, T, fx, fy, min_d, max_d, want_hits):
    sc, orc, rr, fr, K, _ = scene
    T = np.ascontiguousarray(np.asarray(T, np.float32))
    rr.render(sc, T, fx, fy, K.cx, K.cy, min_d, max_d)
    got = rr.download()
    want = orc.render(W, H, T, fx, fy, K.cx, K.cy, min_d, max_d)
    r = compare_renders(got, want, 1e-4)
    assert r["bit_exact_all"], r
    hits = int(np.count_nonzero(want["depth"] != np.float32(1e10)))
    if want_hits is True:
        assert hits > 0, "the pose should see the surface"
    elif want_hits is False:
        assert hits == 0, hits
    return hits


@pytest.mark.parametrize("yaw_deg", [0, 90, 180, 270])
@pytest.mark.parametrize("min_d", [0.2, 0.01])
def test_camera_inside_volume(scene, yaw_deg, min_d):
    sc, orc, rr, fr, K, centre = scene
    T = np.asarray(fr[-1].pose, np.float64).copy()
    T[:3, :3] = T[:3, :3] @ _rot_y(np.radians(yaw_deg))
    T[:3, 3] = centre
    _check(scene, T, K.fx, K.fy, min_d, 3.0, want_hits=None)


def test_camera_far_back(scene):
    sc, orc, rr, fr, K, _ = scene
    T = np.asarray(fr[0].pose, np.float64).copy()
    T[:3, 3] -= 4.0 * T[:3, 2]  # 4 m further back along the view axis
    _check(scene, T, K.fx, K.fy, 0.2, 10.0, want_hits=True)


def test_camera_facing_away(scene):
    sc, orc, rr, fr, K, _ = scene
    T = np.asarray(fr[0].pose, np.float64).copy()
    T[:3, :3] = T[:3, :3] @ _rot_y(np.pi)
    T[:3, 3] -= 1.5 * np.asarray(fr[0].pose)[:3, 2]  # step back so nothing is behind the new view
    _check(scene, T, K.fx, K.fy, 0.2, 3.0, want_hits=False)


@pytest.mark.parametrize("f", [30.0, 5000.0])
def test_wide_and_narrow_fields_of_view(scene, f):
    sc, orc, rr, fr, K, _ = scene
    _check(scene, fr[1].pose, f, f, 0.2, 3.0, want_hits=True)


def test_scaled_rotation_disables_bounds(scene):
    sc, orc, rr, fr, K, _ = scene
    T = np.asarray(fr[2].pose, np.float64).copy()
    T[:3, :3] *= 1.02
    _check(scene, T, K.fx, K.fy, 0.2, 3.0, want_hits=True)


def test_negative_minimum_depth(scene):
    sc, orc, rr, fr, K, _ = scene
    _check(scene, fr[3].pose, K.fx, K.fy, -0.3, 3.0, want_hits=True)
