"""The reference's own CUDA kernels (compiled for sm_100a from the reference
sources by oracle/ref_build.py, built per operation without FMA
contraction) against the oracle and the CUDA path on race-free seeded
cases; and the reference as its own build would compile it (nvcc default,
FMA contraction) against the oracle within tolerance."""
import numpy as np
import pytest

from parity_util import compare_renders, compare_volumes

pytestmark = pytest.mark.gpu


def _ref():
    import ref

    if not (ref.available(True) and ref.available(False)):
        pytest.skip("reference kernels not built (oracle/ref_build.py needs the reference sources)")
    return ref


@pytest.mark.parametrize("case", [("tabletop_64x48_4mm", 13, 3, 64, 48, 0.004, 0.02, 1 << 24, 20000),
                                  ("tabletop_80x60_6mm", 13, 2, 80, 60, 0.006, 0.03, 1 << 24, 20000),
                                  ("tabletop_64x48_5mm", 54, 2, 64, 48, 0.005, 0.02, 1 << 24, 20000)])
def test_reference_kernels_match_oracle_and_cuda_path(cuda, oracle_mod, synth_mod, case):
    ref = _ref()
    import sys
    import os

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_golden
    import vsg

    name, seed, n, W, H, voxel, trunc, buckets, blocks = case
    for s in range(seed, seed + 50):
        frames, K = synth_mod.tabletop_stream(s, n, W, H)
        if not make_golden.bucket_collision(oracle_mod, frames, K, voxel, trunc, buckets):
            break
    else:
        pytest.skip("no race-free seed")
    rnf = ref.RefScene(buckets, blocks, voxel, trunc, nofma=True)
    rfm = ref.RefScene(buckets, blocks, voxel, trunc, nofma=False)
    orc = oracle_mod.OracleScene(voxel)
    sc = vsg.Scene(voxel_size=voxel, truncation=trunc, hash_num_slots=50021, num_sdf_blocks=blocks)
    rr = vsg.Renderer(W, H)
    for f in frames:
        pm = cuda.from_numpy(f.pointmap).cuda()
        rgb = cuda.from_numpy(f.rgb).cuda()
        nm = cuda.from_numpy(f.normals).cuda()
        for r in (rnf, rfm):
            r.integrate(pm.data_ptr(), rgb.data_ptr(), nm.data_ptr(), W, H, trunc, f.pose, K.fx, K.fy, K.cx, K.cy)
        orc.integrate(f.pointmap, f.rgb, trunc, f.pose, K.fx, K.fy, K.cx, K.cy)
        sc.integrate(pm, rgb, nm, W, H, trunc, f.pose, K.fx, K.fy, K.cx, K.cy)
        oc, ov = orc.export()
        # reference without contraction == oracle, bit for bit
        c1, v1 = rnf.export()
        res = compare_volumes(c1, v1, oc, ov["raw"])
        assert res["same_blocks"] and res["bit_exact"], res
        # CUDA path == reference
        gc, gv = sc.export()
        res = compare_volumes(gc, gv, c1, v1)
        assert res["same_blocks"] and res["bit_exact"], res
        # reference as shipped (FMA contraction): within the stated tolerances
        c2, v2 = rfm.export()
        res = compare_volumes(c2, v2, oc, ov["raw"])
        print("fma build vs oracle", res)
        assert res["same_blocks"], res
        # contraction can flip an integer decision (pixel rounding, truncation
        # reject) on a handful of voxels; everything else agrees within 1e-5 m
        assert res["weight_mismatch"] <= 1e-3 * max(res["updated_voxels"], 1), res
        r1 = rnf.render(W, H, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
        ro = orc.render(W, H, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
        cmp = compare_renders(r1, ro)
        assert cmp["bit_exact_all"], cmp
        rr.render(sc, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
        cmp = compare_renders(rr.download(), r1)
        assert cmp["bit_exact_all"], cmp
        r2 = rfm.render(W, H, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
        cmp = compare_renders(r2, ro)
        print("fma build render vs oracle", cmp)
        # measured spread of the reference's own contraction choice: >= 99.7 %
        # of depths within 1e-4 m on every checked frame
        assert cmp["frac_within_tol"] >= 0.995, cmp
    rnf.close()
    rfm.close()
