"""Opt-in march step (vsg_renderer_set_step) and its autotuner (needs a GPU).

Step 0 is the reference's half-voxel march: a renderer set back to 0 after
another step gives the default depths bit for bit.  A longer step is an
approximation, not the drop-in: it takes fewer march iterations, and its
depths move (and the reference's crossing acceptance, |lastSdf - dist| and
|dist| under 3 voxels, rejects more crossings as the step grows);
vsg.tune_ray_step measures each candidate against the exact march and
returns the fastest step within the caller's depth tolerance, or 0."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scene(vsg, cuda, synth_mod):
    fr, K = synth_mod.tabletop_stream(0, 6, 320, 240)
    sc = vsg.Scene(voxel_size=0.004, truncation=0.02, hash_num_slots=50021, num_sdf_blocks=80000)
    for f in fr:
        pm, rgb, nm = (cuda.from_numpy(x).cuda() for x in (f.pointmap, f.rgb, f.normals))
        sc.integrate(pm, rgb, nm, K.width, K.height, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
    return sc, fr, K


def test_step_zero_is_the_reference_march_and_longer_steps_approximate(cuda, synth_mod):
    import vsg

    sc, fr, K = _scene(vsg, cuda, synth_mod)
    rr = vsg.Renderer(K.width, K.height)
    T = fr[-1].pose
    rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    exact = rr.download()
    it_exact = sc.stats()["render_lane_iters"]
    rr.set_step(0.003)  # 0.75 voxel
    rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    approx = rr.download()
    it_approx = sc.stats()["render_lane_iters"]
    rr.set_step(0.0)
    rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    again = rr.download()
    for k in exact:
        assert np.array_equal(exact[k].view(np.uint32), again[k].view(np.uint32)), k
    he, ha = exact["depth"] < 1e9, approx["depth"] < 1e9
    both = he & ha
    err = np.abs(exact["depth"][both].astype(np.float64) - approx["depth"][both])
    print({"iters": (it_exact, it_approx), "hits": (int(he.sum()), int(ha.sum())),
           "max": float(err.max()) if err.size else 0.0, "within_5mm": float((err <= 5e-3).mean()) if err.size else 0.0})
    assert it_approx < it_exact
    assert not np.array_equal(exact["depth"].view(np.uint32), approx["depth"].view(np.uint32))
    with pytest.raises(vsg.VsgError):
        rr.set_step(-1.0)
    rr.close()
    sc.close()


def test_tune_ray_step_returns_a_step_within_tolerance(cuda, synth_mod):
    import vsg

    sc, fr, K = _scene(vsg, cuda, synth_mod)
    rr = vsg.Renderer(K.width, K.height)
    poses = [fr[i].pose for i in (1, 3, 5)]
    factors = (0.1, 0.15, 0.25, 0.5, 1.0)
    step, table = vsg.tune_ray_step(sc, rr, poses, (K.fx, K.fy, K.cx, K.cy), 0.2, 3.0, 0.02, factors=factors,
                                    tol=2e-3, frac=0.95)
    print(table)
    assert table[0]["step"] == 0.0 and table[0]["frac_within_tol"] == 1.0 and len(table) == 1 + len(factors)
    chosen = [r for r in table if r["step"] == step]
    assert len(chosen) == 1 and (step == 0.0 or chosen[0]["frac_within_tol"] >= 0.95)
    assert all(r["ms"] > 0 for r in table)
    rr.close()
    sc.close()
