"""Streaming blocks between the scene and host memory (vsg_stream_*,
vsg_store_*, vsg_scene_save/load) against the oracle's restatement of
VoxelStreamingManager (oracle.ChunkStore + orc_stream_out / orc_stream_in):
which blocks leave, what the host store holds, which chunks come back, and
that integration and ray casting after out/in cycles stay bit-exact (needs a
GPU)."""
import numpy as np
import pytest

from parity_util import compare_renders, compare_volumes

pytestmark = pytest.mark.gpu

VOXEL, TRUNC = 0.004, 0.02
EXT = (0.1, 0.1, 0.1)  # small chunks: the tabletop spans many of them


def _setup(cuda, synth_mod, oracle_mod, n_frames=10, W=160, H=120, blocks=60000):
    import vsg

    fr, K = synth_mod.tabletop_stream(71, n_frames, W, H)
    sc = vsg.Scene(voxel_size=VOXEL, truncation=TRUNC, hash_num_slots=20011, num_sdf_blocks=blocks)
    rr = vsg.Renderer(W, H)
    o = oracle_mod.OracleScene(VOXEL)
    dev = [tuple(cuda.from_numpy(x).cuda() for x in (f.pointmap, f.rgb, f.normals)) for f in fr]
    return vsg, fr, K, sc, rr, o, dev


def _frame(i, fr, K, sc, rr, o, dev):
    f = fr[i]
    pm, rgb, nm = dev[i]
    sc.integrate(pm, rgb, nm, K.width, K.height, TRUNC, f.pose, K.fx, K.fy, K.cx, K.cy)
    o.integrate(f.pointmap, f.rgb, TRUNC, f.pose, K.fx, K.fy, K.cx, K.cy)
    rr.render(sc, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    want = o.render(K.width, K.height, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    r = compare_renders(rr.download(), want)
    assert r["bit_exact_all"], (i, r)


def _same_volume(sc, o):
    gc, gv = sc.export()
    oc, ov = o.export()
    v = compare_volumes(gc, gv, oc, ov["raw"])
    assert v["same_blocks"] and v["bit_exact"], v


def _same_blocks(a, b):
    (ac, av), (bc, bv) = a, b
    assert ac.shape == bc.shape and np.array_equal(ac, bc)
    assert np.array_equal(av, bv)


def test_stream_out_in_cycles_match_oracle(cuda, synth_mod, oracle_mod):
    vsg, fr, K, sc, rr, o, dev = _setup(cuda, synth_mod, oracle_mod)
    store = vsg.Store(EXT)
    ostore = oracle_mod.ChunkStore(VOXEL, EXT)
    for i in range(4):
        _frame(i, fr, K, sc, rr, o, dev)
    before = sc.stats()["allocated_blocks"]
    # out: everything farther than 0.25 m from a point above the table
    c1, r1 = (0.0, 0.1, 0.0), 0.25
    n = sc.stream_out(store, c1, r1)
    oc, ov = o.stream_out(c1, r1)
    assert n == len(oc) > 100 and n < before
    ostore.add(oc, ov)
    _same_blocks(store.export(), ostore.export())
    _same_volume(sc, o)
    st = sc.stats()
    assert st["allocated_blocks"] == before - n and st["allocated_blocks"] + st["free_blocks"] == 60000
    # integration re-allocates some of the streamed-out positions
    for i in range(4, 6):
        _frame(i, fr, K, sc, rr, o, dev)
    # a second stream-out around another centre: blocks stored twice merge
    c2, r2 = (0.15, 0.05, -0.1), 0.3
    n2 = sc.stream_out(store, c2, r2)
    oc2, ov2 = o.stream_out(c2, r2)
    assert n2 == len(oc2) > 0
    ostore.add(oc2, ov2)
    _same_blocks(store.export(), ostore.export())
    # in: the chunks around a third centre come back (merging into resident blocks)
    c3, r3 = (-0.1, 0.0, 0.05), 0.2
    n_in, n_merged = sc.stream_in(store, c3, r3)
    ic, iv = ostore.take(c3, r3)
    o.stream_in(ic, iv)
    assert n_in == len(ic) > 0
    _same_blocks(store.export(), ostore.export())
    _same_volume(sc, o)
    for i in range(6, 8):
        _frame(i, fr, K, sc, rr, o, dev)
    _same_volume(sc, o)
    # everything back
    n_in, _ = sc.stream_in(store)
    ic, iv = ostore.take(None, -1.0)
    o.stream_in(ic, iv)
    assert n_in == len(ic) and store.info()[0] == 0
    for i in range(8, 10):
        _frame(i, fr, K, sc, rr, o, dev)
    _same_volume(sc, o)
    assert sc.stats()["flags"] == 0


def test_stream_out_all_then_in_all_restores_scene(cuda, synth_mod, oracle_mod):
    vsg, fr, K, sc, rr, o, dev = _setup(cuda, synth_mod, oracle_mod, n_frames=3)
    for i in range(3):
        _frame(i, fr, K, sc, rr, o, dev)
    ref_c, ref_v = sc.export()
    want = rr.download()
    store = vsg.Store()
    n = sc.stream_out(store, (0, 0, 0), 0.0)  # every distance is >= 0
    assert n == len(ref_c) and sc.stats()["allocated_blocks"] == 0
    # empty scene: the renderer leaves its outputs untouched, as in the reference
    f = fr[2]
    rr.render(sc, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    assert compare_renders(rr.download(), want)["bit_exact_all"]
    _same_blocks(store.export(), (ref_c, ref_v))
    n_in, n_merged = sc.stream_in(store)
    assert n_in == n and n_merged == 0
    _same_blocks(sc.export(), (ref_c, ref_v))
    rr.render(sc, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    assert compare_renders(rr.download(), want)["bit_exact_all"]


def test_checkpoint_files_round_trip(cuda, synth_mod, oracle_mod, tmp_path):
    vsg, fr, K, sc, rr, o, dev = _setup(cuda, synth_mod, oracle_mod, n_frames=3)
    for i in range(3):
        _frame(i, fr, K, sc, rr, o, dev)
    path = str(tmp_path / "scene.vsgb")
    sc.save(path)
    sc2 = vsg.Scene(voxel_size=VOXEL, truncation=TRUNC, hash_num_slots=20011, num_sdf_blocks=60000)
    sc2.load(path)
    _same_blocks(sc2.export(), sc.export())
    rr2 = vsg.Renderer(K.width, K.height)
    f = fr[2]
    rr.render(sc, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    rr2.render(sc2, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
    assert compare_renders(rr2.download(), rr.download())["bit_exact_all"]
    # the resumed scene keeps integrating exactly like the original
    pm, rgb, nm = dev[0]
    for s in (sc, sc2):
        s.integrate(pm, rgb, nm, K.width, K.height, TRUNC, fr[0].pose, K.fx, K.fy, K.cx, K.cy)
    _same_blocks(sc2.export(), sc.export())
    # store files
    store = vsg.Store(EXT)
    sc.stream_out(store, (0.0, 0.1, 0.0), 0.2)
    spath = str(tmp_path / "store.vsgb")
    store.save(spath)
    store2 = vsg.Store(EXT)
    store2.load(spath)
    _same_blocks(store2.export(), store.export())
    assert store2.info() == store.info()


def test_stream_in_refuses_when_pool_is_short(cuda, synth_mod, oracle_mod):
    vsg, fr, K, sc, rr, o, dev = _setup(cuda, synth_mod, oracle_mod, n_frames=2)
    for i in range(2):
        _frame(i, fr, K, sc, rr, o, dev)
    store = vsg.Store()
    n = sc.stream_out(store, (0, 0, 0), 0.0)
    small = vsg.Scene(voxel_size=VOXEL, truncation=TRUNC, hash_num_slots=1009, num_sdf_blocks=max(16, n // 2))
    with pytest.raises(vsg.VsgError):
        small.stream_in(store)
    assert store.info()[0] == n  # nothing moved
    assert small.stats()["allocated_blocks"] == 0
