"""March statistics (vsg_scene_march_stats) (needs a GPU).

With the statistics on, renders run the counting ray caster: the samples
skipped as empty, the samples at a skip-cell boundary and the distinct
blocks read are counted; off (the default), they read 0.  Both casters
march the same samples, so every output and the counters both keep (hits,
misses, full samples, jumps, iterations) are equal bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COMMON = ("render_hits", "render_misses", "render_samples_full", "render_jumps", "render_lane_iters",
          "render_warp_iters")
COUNTED = ("render_samples_skipped", "render_singles", "render_blocks_read")


def test_counting_caster_gives_the_same_outputs(cuda, synth_mod):
    import vsg

    fr, K = synth_mod.tabletop_stream(0, 6, 320, 240)
    sc = vsg.Scene(voxel_size=0.004, truncation=0.02, hash_num_slots=50021, num_sdf_blocks=80000)
    rr = vsg.Renderer(K.width, K.height)
    for f in fr:
        pm, rgb, nm = (cuda.from_numpy(x).cuda() for x in (f.pointmap, f.rgb, f.normals))
        sc.integrate(pm, rgb, nm, K.width, K.height, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
    T = fr[-1].pose

    rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    plain, st_plain = rr.download(), sc.stats()
    sc.march_stats(True)
    rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    counted, st_counted = rr.download(), sc.stats()
    sc.march_stats(False)
    rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    again = rr.download()

    for k in plain:
        assert np.array_equal(plain[k].view(np.uint32), counted[k].view(np.uint32)), k
        assert np.array_equal(plain[k].view(np.uint32), again[k].view(np.uint32)), k
    for k in COMMON:
        assert st_plain[k] == st_counted[k], k
    assert st_plain["render_hits"] > 0
    for k in COUNTED:
        assert st_plain[k] == 0, k
        assert st_counted[k] > 0, k
    # every skipped sample was skipped by a jump
    assert st_counted["render_samples_skipped"] >= st_counted["render_jumps"]
    rr.close()
    sc.close()
