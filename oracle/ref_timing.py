"""Time the reference's own CUDA launchers (built for sm_100a by ref_build.py
into oracle/_ref/, nvcc defaults) on the bench's workload -- the tabletop
stream, 30 frames of 640x480, 4 mm voxels, truncation 0.02 m, 200000
buckets and pool blocks, each frame integrated then ray cast at its pose --
next to this library on the same GPU.  TEST INFRASTRUCTURE / measurement
script: the product never loads the reference build.

    python oracle/ref_timing.py            # prints one JSON line

Reports device time per frame (CUDA events around the launcher calls, host
work inside them included) for the reference's allocate + compact +
integrate and its ray cast, and the same for this library.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "real-time-depth-fusion-directional-tsdf_b200"))


def main():
    import torch

    import ref
    import synth
    import vsg

    fr, K = synth.tabletop_stream(0, 30, 640, 480)
    W, H = K.width, K.height
    dev = [tuple(torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (f.pointmap, f.rgb, f.normals))
           for f in fr]
    poses = [np.ascontiguousarray(np.asarray(f.pose, np.float32).reshape(16)) for f in fr]
    Td = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = {k: torch.zeros(n, dtype=torch.float32, device="cuda")
           for k, n in (("depth", W * H), ("pos", 4 * W * H), ("col", 4 * W * H), ("nrm", 4 * W * H))}
    L = ref.lib(nofma=False)
    res = {}
    for rep in range(2):  # the first pass warms up
        h = L.ref_create(200000, 200000, 0.004, 0.02, 0.01)
        ti = tr = 0.0
        for i, f in enumerate(fr):
            Td.copy_(torch.from_numpy(poses[i]))
            pm, rgb, nm = dev[i]
            a = L.ref_integrate_dev(h, pm.data_ptr(), rgb.data_ptr(), nm.data_ptr(), W, H, 0.02,
                                    poses[i].ctypes.data, Td.data_ptr(), K.fx, K.fy, K.cx, K.cy)
            b = L.ref_render_dev(h, W, H, poses[i].ctypes.data, Td.data_ptr(), K.fx, K.fy, K.cx, K.cy, 0.2, 3.0,
                                 out["depth"].data_ptr(), out["pos"].data_ptr(), out["col"].data_ptr(),
                                 out["nrm"].data_ptr())
            assert a >= 0 and b >= 0
            ti += a
            tr += b
        L.ref_destroy(h)
        res["reference"] = {"integrate_ms_per_frame": ti / len(fr), "render_ms_per_frame": tr / len(fr),
                            "frames_per_s": len(fr) / ((ti + tr) * 1e-3)}
    # this library on the same frames (stream-ordered calls, events around each)
    sc = vsg.Scene(voxel_size=0.004, truncation=0.02, hash_num_slots=200000, num_sdf_blocks=200000)
    rr = vsg.Renderer(W, H)
    for rep in range(2):
        sc.reset()
        ti = tr = 0.0
        for i, f in enumerate(fr):
            pm, rgb, nm = dev[i]
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record()
            sc.integrate(pm, rgb, nm, W, H, 0.02, f.pose, K.fx, K.fy, K.cx, K.cy)
            e[1].record()
            rr.render(sc, f.pose, K.fx, K.fy, K.cx, K.cy, 0.2, 3.0)
            e[2].record()
            torch.cuda.synchronize()
            ti += e[0].elapsed_time(e[1])
            tr += e[1].elapsed_time(e[2])
        res["this_library"] = {"integrate_ms_per_frame": ti / len(fr), "render_ms_per_frame": tr / len(fr),
                               "frames_per_s": len(fr) / ((ti + tr) * 1e-3)}
    res["speedup"] = res["this_library"]["frames_per_s"] / res["reference"]["frames_per_s"]
    res["workload"] = "tabletop 30x640x480, voxel 4mm, trunc 0.02m, 200000 buckets/blocks"
    print(json.dumps(res))


if __name__ == "__main__":
    main()
