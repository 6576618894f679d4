"""Batched form (vsg_batch_*): independent scans of uneven resolution and
frame count advanced together must give, scene by scene and step by step,
exactly the results of vsg_integrate + vsg_render run one scene at a time,
and of the CPU oracle restating the reference.  Covers the eager first step
of each shape, graph replays, and shapes that change as scans finish (needs
a GPU)."""
import numpy as np
import pytest

from parity_util import compare_renders, compare_volumes

pytestmark = pytest.mark.gpu

SCANS = [  # seed, width, height, frames
    (31, 64, 48, 3),
    (32, 160, 120, 5),
    (33, 128, 96, 2),
    (34, 200, 150, 4),
    (35, 96, 72, 5),
]


def _streams(synth_mod):
    out = []
    for seed, w, h, n in SCANS:
        fr, K = synth_mod.tabletop_stream(seed, n, w, h)
        out.append((fr, K))
    return out


def _dev(torch, f):
    return (torch.from_numpy(f.pointmap).cuda(), torch.from_numpy(f.rgb).cuda(), torch.from_numpy(f.normals).cuda())


@pytest.mark.parametrize("autotune", [True, False])
def test_batch_matches_per_scene_path(cuda, synth_mod, autotune):
    import vsg

    streams = _streams(synth_mod)
    kw = dict(voxel_size=0.004, truncation=0.02, hash_num_slots=30011, num_sdf_blocks=40000)
    # per-scene reference runs
    expected = []
    for fr, K in streams:
        sc = vsg.Scene(**kw)
        rr = vsg.Renderer(K.width, K.height)
        per = []
        for f in fr:
            pm, rgb, nm = _dev(cuda, f)
            sc.integrate(pm, rgb, nm, K.width, K.height, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
            rr.render(sc, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
            per.append((sc.export(), rr.download(), sc.stats()))
        expected.append(per)
        sc.close()
        rr.close()
    # the same scans through one batch
    scenes = [vsg.Scene(**kw) for _ in streams]
    rends = [vsg.Renderer(K.width, K.height) for _, K in streams]
    batch = vsg.Batch(scenes, rends)
    batch.autotune(autotune)
    maps = [[_dev(cuda, f) for f in fr] for fr, _ in streams]
    steps = max(len(fr) for fr, _ in streams)
    for t in range(steps):
        frames = []
        for i, (fr, K) in enumerate(streams):
            if t < len(fr):
                pm, rgb, nm = maps[i][t]
                frames.append(batch.frame(i, pm, rgb, nm, K.width, K.height, 0.02, fr[t].pose, K.fx, K.fy,
                                          K.cx, K.cy, 0.2, 3.0, render=True))
        batch.step(frames)
        cuda.cuda.synchronize()
        for i, (fr, K) in enumerate(streams):
            if t >= len(fr):
                continue
            (ec, ev), er, es = expected[i][t]
            gc, gv = scenes[i].export()
            v = compare_volumes(gc, gv, ec, ev)
            assert v["same_blocks"] and v["bit_exact"], (t, i, v)
            r = compare_renders(rends[i].download(), er)
            assert r["bit_exact_all"], (t, i, r)
            st = scenes[i].stats()
            assert st["integrated_frames"] == es["integrated_frames"] == t + 1
            assert st["flags"] == 0
            for key in ("frame_new_blocks", "frame_visible_blocks", "frame_updated_blocks",
                        "frame_updated_voxels"):
                assert st[key] == es[key], (t, i, key)
    batch.close()


def test_batch_rejects_bad_frames(cuda, synth_mod):
    import vsg

    fr, K = synth_mod.tabletop_stream(40, 1, 64, 48)
    sc = vsg.Scene(voxel_size=0.004, hash_num_slots=5003, num_sdf_blocks=8000)
    rr = vsg.Renderer(32, 24)  # wrong size for a 64x48 frame
    b = vsg.Batch([sc], [rr])
    pm, rgb, nm = _dev(cuda, fr[0])
    f = b.frame(0, pm, rgb, nm, 64, 48, 0.02, fr[0].pose, K.fx, K.fy, K.cx, K.cy, render=True)
    with pytest.raises(vsg.VsgError):
        b.step([f])
    f2 = b.frame(1, pm, rgb, nm, 64, 48, 0.02, fr[0].pose, K.fx, K.fy, K.cx, K.cy, render=False)
    with pytest.raises(vsg.VsgError):  # scene index out of range
        b.step([f2])
    f3 = b.frame(0, pm, rgb, nm, 64, 48, 0.02, fr[0].pose, K.fx, K.fy, K.cx, K.cy, render=False)
    with pytest.raises(vsg.VsgError):  # the same scene twice in one step
        b.step([f3, f3])
    b.step([f3])  # integrate only
    cuda.cuda.synchronize()
    assert sc.stats()["integrated_frames"] == 1
    b.close()


def test_batch_matches_oracle(cuda, synth_mod, oracle_mod):
    """Every batched scene against the CPU oracle restating the reference,
    step by step: block sets and voxels bit for bit after each step, the
    full ray cast bit for bit (depth, position, colour, normal), and the
    per-frame counters."""
    import vsg

    streams = _streams(synth_mod)
    kw = dict(voxel_size=0.004, truncation=0.02, hash_num_slots=30011, num_sdf_blocks=40000)
    scenes = [vsg.Scene(**kw) for _ in streams]
    rends = [vsg.Renderer(K.width, K.height) for _, K in streams]
    oracles = [oracle_mod.OracleScene(0.004) for _ in streams]
    batch = vsg.Batch(scenes, rends)
    maps = [[_dev(cuda, f) for f in fr] for fr, _ in streams]
    steps = max(len(fr) for fr, _ in streams)
    for t in range(steps):
        frames, ost = [], {}
        for i, (fr, K) in enumerate(streams):
            if t < len(fr):
                pm, rgb, nm = maps[i][t]
                frames.append(batch.frame(i, pm, rgb, nm, K.width, K.height, 0.02, fr[t].pose, K.fx, K.fy,
                                          K.cx, K.cy, 0.2, 3.0, render=True))
                ost[i] = oracles[i].integrate(fr[t].pointmap, fr[t].rgb, 0.02, fr[t].pose, K.fx, K.fy, K.cx, K.cy)
        batch.step(frames)
        cuda.cuda.synchronize()
        for i, (fr, K) in enumerate(streams):
            if t >= len(fr):
                continue
            gc, gv = scenes[i].export()
            oc, ov = oracles[i].export()
            v = compare_volumes(gc, gv, oc, ov["raw"])
            assert v["same_blocks"] and v["bit_exact"], (t, i, v)
            o = oracles[i].render(K.width, K.height, fr[t].pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
            r = compare_renders(rends[i].download(), o)
            assert r["bit_exact_all"] and r["hits_gpu"] > 0, (t, i, r)
            st = scenes[i].stats()
            assert st["flags"] == 0
            assert st["frame_new_blocks"] == ost[i]["new_blocks"], (t, i)
            assert st["frame_updated_blocks"] == ost[i]["updated_blocks"], (t, i)
            assert st["frame_updated_voxels"] == ost[i]["updated_voxels"], (t, i)
    batch.close()
