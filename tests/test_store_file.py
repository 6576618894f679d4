"""Host side of streaming, no GPU: the block store (vsg_store_*) reads and
writes checkpoint files in the reference's streaming record layout
(SDFBlockInfo {int3 pos, int ptr} + SDFBlock of 512 12-byte VoxelData
{uchar3 color, uchar weight, float sdf, 2 flag bytes, 2 pad},
VoxelStreamingManager.h:30-76, CUDAHashRef.h:22-45) and merges blocks stored
twice with the oracle's rule."""
import struct

import numpy as np
import pytest


def _file(path, coords, vox8, voxel):
    n = len(coords)
    with open(path, "wb") as f:
        f.write(b"VSGBLK01" + struct.pack("<IIQfI", 16, 12, n, voxel, 0))
        for c in coords:
            f.write(struct.pack("<4i", int(c[0]), int(c[1]), int(c[2]), -1))
        for b in vox8:
            v = b.reshape(512, 8)
            rec = np.zeros((512, 12), np.uint8)
            rec[:, 0:3] = v[:, 4:7]   # colour
            rec[:, 3] = v[:, 7]       # weight
            rec[:, 4:8] = v[:, 0:4]   # sdf
            f.write(rec.tobytes())


def _blocks(rng, n):
    coords = rng.integers(-300, 300, size=(n, 3)).astype(np.int32)
    coords = np.unique(coords, axis=0)
    vox = np.zeros((len(coords), 512, 8), np.uint8)
    sdf = rng.uniform(-0.02, 0.02, (len(coords), 512)).astype(np.float32)
    vox[:, :, 0:4] = sdf.view(np.uint8).reshape(len(coords), 512, 4)
    vox[:, :, 4:7] = rng.integers(0, 256, (len(coords), 512, 3))
    w = rng.integers(0, 30, (len(coords), 512))
    w[rng.random((len(coords), 512)) < 0.3] = 0
    vox[:, :, 7] = w
    vox[w == 0, 0:4] = 0  # unobserved voxels hold sdf 0, as in a scene
    return coords, vox.reshape(len(coords), 4096)


def test_store_reads_reference_records_and_writes_them_back(tmp_path, oracle_mod):
    import vsg

    rng = np.random.default_rng(5)
    coords, vox = _blocks(rng, 200)
    p = str(tmp_path / "a.vsgb")
    _file(p, coords, vox, 0.004)
    st = vsg.Store((0.5, 0.5, 0.5))
    st.load(p)
    gc, gv = st.export()
    order = np.lexsort((coords[:, 2], coords[:, 1], coords[:, 0]))
    assert np.array_equal(gc, coords[order]) and np.array_equal(gv, vox[order])
    # and the library writes the same record layout
    q = str(tmp_path / "b.vsgb")
    st.save(q)
    st2 = vsg.Store((0.5, 0.5, 0.5))
    st2.load(q)
    c2, v2 = st2.export()
    assert np.array_equal(c2, gc) and np.array_equal(v2, gv)
    raw = open(q, "rb").read()
    assert raw[:8] == b"VSGBLK01" and len(raw) == 32 + len(coords) * (16 + 512 * 12)


def test_store_merges_blocks_stored_twice(tmp_path, oracle_mod):
    import vsg

    rng = np.random.default_rng(6)
    coords, vox_a = _blocks(rng, 50)
    _, vox_b = _blocks(np.random.default_rng(7), 50)
    vox_b = vox_b[:len(coords)]
    pa, pb = str(tmp_path / "a.vsgb"), str(tmp_path / "b.vsgb")
    _file(pa, coords, vox_a, 0.004)
    _file(pb, coords, vox_b, 0.004)
    st = vsg.Store()
    st.load(pa)
    st.load(pb)
    assert st.info()[0] == len(coords)
    gc, gv = st.export()
    order = np.lexsort((coords[:, 2], coords[:, 1], coords[:, 0]))
    want = np.stack([oracle_mod.merge_voxels(vox_a[i], vox_b[i]) for i in order])
    assert np.array_equal(gv, want)


def test_chunk_assignment_matches_oracle_store(tmp_path, oracle_mod):
    import vsg

    rng = np.random.default_rng(8)
    coords, vox = _blocks(rng, 300)
    p = str(tmp_path / "c.vsgb")
    _file(p, coords, vox, 0.004)
    st = vsg.Store((0.3, 0.2, 0.5))
    st.load(p)
    o = oracle_mod.ChunkStore(0.004, (0.3, 0.2, 0.5))
    o.add(coords, vox)
    assert st.info() == (len(coords), len(o.chunks))


def test_store_rejects_bad_files(tmp_path):
    import vsg

    p = str(tmp_path / "bad.vsgb")
    open(p, "wb").write(b"NOTVSG00" + bytes(24))
    st = vsg.Store()
    with pytest.raises(vsg.VsgError):
        st.load(p)
    with pytest.raises(vsg.VsgError):
        st.load(str(tmp_path / "missing.vsgb"))
    with pytest.raises(vsg.VsgError):
        vsg.Store((0.0, 1.0, 1.0))


def test_store_refuses_files_whose_size_disagrees_with_their_header(tmp_path):
    """A checkpoint whose header counts more (or fewer) blocks than the file
    holds is refused before any buffer is sized from the count, and the store
    is left as it was: a truncated file, a header claiming 2^31 blocks over a
    one-block body, and trailing bytes."""
    import vsg

    rng = np.random.default_rng(9)
    coords, vox = _blocks(rng, 20)
    good = str(tmp_path / "good.vsgb")
    _file(good, coords, vox, 0.004)
    raw = open(good, "rb").read()
    cases = {
        "truncated": raw[:-1],
        "huge_count": raw[:16] + struct.pack("<Q", 1 << 31) + raw[24:32] + raw[32:32 + 16] +
        raw[32 + 16 * len(coords):32 + 16 * len(coords) + 512 * 12],
        "trailing": raw + b"\0" * 7,
    }
    for name, data in cases.items():
        p = str(tmp_path / f"{name}.vsgb")
        open(p, "wb").write(data)
        st = vsg.Store()
        with pytest.raises(vsg.VsgError):
            st.load(p)
        assert st.info()[0] == 0, name
    st = vsg.Store()
    st.load(good)
    assert st.info()[0] == len(coords)


def test_store_records_and_counts(oracle_mod):
    """vsg_store_add_records files the reference's streaming records like a
    checkpoint file does (merging repeats), and vsg_store_count reports the
    blocks and chunks a stream-in would take, as the oracle's chunk grid
    (ChunkStore.take) chooses them."""
    import vsg

    rng = np.random.default_rng(8)
    coords, vox = _blocks(rng, 300)
    rec = np.zeros((len(coords), 512, 12), np.uint8)
    v = vox.reshape(len(coords), 512, 8)
    rec[:, :, 0:3] = v[:, :, 4:7]
    rec[:, :, 3] = v[:, :, 7]
    rec[:, :, 4:8] = v[:, :, 0:4]
    infos = np.concatenate([coords, -np.ones((len(coords), 1), np.int32)], 1)
    ext = (0.5, 0.5, 0.5)
    st = vsg.Store(ext)
    st.add_records(0.004, infos, rec.reshape(len(coords), -1))
    gc, gv = st.export()
    order = np.lexsort((coords[:, 2], coords[:, 1], coords[:, 0]))
    assert np.array_equal(gc, coords[order]) and np.array_equal(gv, vox[order])
    # the same records again merge voxel by voxel
    st.add_records(0.004, infos, rec.reshape(len(coords), -1))
    oc = oracle_mod.ChunkStore(0.004, ext)
    oc.add(coords, vox)
    oc.add(coords, vox)
    _, gv2 = st.export()
    _, ov2 = oc.export()
    assert np.array_equal(gv2, ov2)
    for center, radius in (((0.0, 0.0, 0.0), 1.0), ((0.5, -0.3, 0.2), 2.5), ((5.0, 5.0, 5.0), 0.5)):
        nb, nc = st.count(center, radius)
        fresh = oracle_mod.ChunkStore(0.004, ext)  # take() removes what it returns
        fresh.add(coords, vox)
        tc, _ = fresh.take(center, radius)
        assert nb == len(tc), (center, radius)
    assert st.count(None, -1.0)[0] == len(coords)
    with pytest.raises(vsg.VsgError):
        st.add_records(0.008, infos[:1], rec[:1].reshape(1, -1))


def test_store_records_parallel_filing_merges_repeats_in_order(oracle_mod):
    """More than 512 records in one call take the chunk-parallel filing
    (groups by chunk, one host thread per chunk); repeats of a block within the
    call merge in input order, exactly as the oracle's sequential filing."""
    import vsg

    rng = np.random.default_rng(11)
    coords, vox = _blocks(rng, 1500)
    rep = rng.choice(len(coords), 600)  # repeated blocks, new voxel contents
    _, vox2 = _blocks(np.random.default_rng(12), 1500)
    all_c = np.concatenate([coords, coords[rep]])
    all_v = np.concatenate([vox, vox2[: len(rep)]])
    perm = rng.permutation(len(all_c))
    all_c, all_v = all_c[perm], all_v[perm]
    v = all_v.reshape(len(all_c), 512, 8)
    rec = np.zeros((len(all_c), 512, 12), np.uint8)
    rec[:, :, 0:3] = v[:, :, 4:7]
    rec[:, :, 3] = v[:, :, 7]
    rec[:, :, 4:8] = v[:, :, 0:4]
    infos = np.concatenate([all_c, -np.ones((len(all_c), 1), np.int32)], 1)
    ext = (0.25, 0.25, 0.25)
    st = vsg.Store(ext)
    st.add_records(0.004, infos, rec.reshape(len(all_c), -1))
    oc = oracle_mod.ChunkStore(0.004, ext)
    oc.add(all_c, all_v)
    gc, gv = st.export()
    ocs, ov = oc.export()
    assert len(gc) == len(coords)
    assert np.array_equal(gc, ocs) and np.array_equal(gv, ov)
    assert st.count(None, -1.0)[0] == len(coords)
