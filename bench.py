"""Throughput of the fusion hot path: frames/s of integrate + raycast.

Workload (tabletop stream): 30 float32 point-map frames 640x480
(fx=fy=525, cx=319.5, cy=239.5) ray traced from a seeded scene (plane y=0 +
3 spheres), camera orbiting 1.0 m over 60 degrees, structured-light depth
noise; voxel 4 mm, truncation 0.02 m, 200000 hash buckets, 200000 pool
blocks; every frame is integrated, then ray cast at the same pose with
min/max depth 0.2/3.0 m.  One step = reset + the whole 30-frame stream.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  --impl reference times the CPU restatement
of the reference path (the reference has no CPU implementation of its own)
on the host cores over a bounded sample.

After the timed region the line gains side measurements, each on its own
key: marching cubes and surface points over the headline volume, streaming,
the ray-cast adjoint and the 256-pose x 20-step refinement, the point splat,
the reference's own CUDA kernels on the headline frames (`ref_gpu`), the
room stream (300 frames 1280x720, marching cubes after frames 100/200/300),
the end-to-end C-ABI leg with host buffers (`e2e`), the corridor with
streaming and tracking, its 8-corridor batched form, the 64-scan batched
form, and the CPU baseline.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "real-time-depth-fusion-directional-tsdf_b200")
ORACLE = os.path.join(ROOT, "oracle")
sys.path.insert(0, PKG)

import numpy as np  # noqa: E402

METRIC = "frames/s integrate+raycast 640x480@4mm; batched & adjoint vs plain, same B200"
WORKLOAD = "tabletop 30x640x480 point-map frames, voxel 4mm, trunc 0.02m, 200000 slots"
VOXEL, TRUNC, SLOTS, BLOCKS = 0.004, 0.02, 200000, 200000
MIN_D, MAX_D = 0.2, 3.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=30)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batched-scans", type=int, default=64)
    ap.add_argument("--no-corridor", action="store_true")
    ap.add_argument("--no-room", action="store_true")
    ap.add_argument("--corridor-frames", type=int, default=400)
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--room-frames", type=int, default=300)
    ap.add_argument("--room-only", action="store_true",
                    help="run only the room leg and print its object (profiling runs)")
    ap.add_argument("--headline-only", action="store_true",
                    help="time the headline step and skip every side measurement (profiling runs)")
    ap.add_argument("--corridor-scale", type=float, default=0.1,
                    help="batched corridors: fraction of the U[500,2000] frame counts to run")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        cmd = ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
               "--format=csv,noheader,nounits", "-lms", "100"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thr = threading.Thread(target=self._read, daemon=True)
            self.thr.start()
        except OSError:
            self.proc = None
        # nvidia-smi takes longer to start than a short timed region lasts:
        # wait (at most 5 s) until it prints its first row, taken before the
        # region with the GPU idle, and keep only the rows after it
        t0 = time.monotonic()
        while self.proc and not self.rows and self.proc.poll() is None and time.monotonic() - t0 < 5.0:
            time.sleep(0.01)
        self.first = len(self.rows)
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            # a region shorter than the 100 ms sampling interval may end
            # before its first row: wait (at most 0.3 s) for one
            t0 = time.monotonic()
            while len(self.rows) <= self.first and self.proc.poll() is None and time.monotonic() - t0 < 0.3:
                time.sleep(0.005)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = self.rows[getattr(self, "first", 0):]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peak_hbm() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_stream(args):
    import synth

    frames, K = synth.tabletop_stream(args.seed, args.frames)
    return frames, K


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(frames, K, budget_s: float = 20.0) -> dict:
    """Oracle (CPU restatement, OpenMP) on a bounded sample of the stream:
    all frames integrated, a band of rows ray cast per frame."""
    sys.path.insert(0, ORACLE)
    import oracle

    oracle.build()
    threads = oracle.max_threads()
    orc = oracle.OracleScene(VOXEL)
    rows = 24
    t_int = t_ren = 0.0
    n = 0
    for f in frames:
        t0 = time.perf_counter()
        orc.integrate(f.pointmap, f.rgb, TRUNC, f.pose, K.fx, K.fy, K.cx, K.cy)
        t1 = time.perf_counter()
        y0 = K.height // 2 - rows // 2
        orc.render(K.width, K.height, f.pose, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D, rows=(y0, y0 + rows))
        t2 = time.perf_counter()
        t_int += t1 - t0
        t_ren += (t2 - t1) * (K.height / rows)
        n += 1
        if t_int + t_ren > budget_s:
            break
    fps = n / (t_int + t_ren)
    return {"value": fps, "unit": "frames/s", "cores": threads, "kind": "port", "cpu": cpu_model(),
            "sample": f"{n} frames integrated in full; ray cast on {rows} central rows per frame, "
                      f"scaled to {K.height} rows"}


def ref_gpu_measure(frames, K) -> dict:
    """The reference's own CUDA launchers as the GPU comparator, on the
    headline's frames and GPU, after the timed region.  They are built for
    sm_100a from the reference sources by oracle/ref_build.py (nvcc
    defaults, as the reference's own build compiles them) into oracle/_ref,
    the checker's side of the repository; this leg alone loads them.  Per
    frame: allocBlocksFromDepthMapCUDA + compactifyHashCUDA +
    integrateDepthMapIntoBlocksCUDA, then rayCastRenderCUDA at the frame's
    pose (device pose matrix, 0.2-3.0 m), CUDA events around the launcher
    calls (their host-side work included, as a caller sees it).  This
    library is timed the same way (events around vsg_integrate and
    vsg_render) on the same frames.  Two passes; the second is reported."""
    import torch

    import vsg

    sys.path.insert(0, ORACLE)
    import ref

    if not ref.available(nofma=False):
        return {"unavailable": "reference kernels not built (oracle/_ref/libvsgref.so missing)"}
    W, H = K.width, K.height
    dev = [tuple(torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (f.pointmap, f.rgb, f.normals))
           for f in frames]
    poses = [np.ascontiguousarray(np.asarray(f.pose, np.float32).reshape(16)) for f in frames]
    Td = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = {k: torch.zeros(n, dtype=torch.float32, device="cuda")
           for k, n in (("depth", W * H), ("pos", 4 * W * H), ("col", 4 * W * H), ("nrm", 4 * W * H))}
    L = ref.lib(nofma=False)
    res = {}
    for _ in range(2):
        h = L.ref_create(SLOTS, BLOCKS, VOXEL, TRUNC, 0.01)
        ti = tr = 0.0
        for i in range(len(frames)):
            Td.copy_(torch.from_numpy(poses[i]))
            pm, rgb, nm = dev[i]
            a = L.ref_integrate_dev(h, pm.data_ptr(), rgb.data_ptr(), nm.data_ptr(), W, H, TRUNC,
                                    poses[i].ctypes.data, Td.data_ptr(), K.fx, K.fy, K.cx, K.cy)
            b = L.ref_render_dev(h, W, H, poses[i].ctypes.data, Td.data_ptr(), K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D,
                                 out["depth"].data_ptr(), out["pos"].data_ptr(), out["col"].data_ptr(),
                                 out["nrm"].data_ptr())
            if a < 0 or b < 0:
                L.ref_destroy(h)
                return {"error": "a reference launcher failed"}
            ti += a
            tr += b
        L.ref_destroy(h)
        res["reference"] = {"integrate_ms_per_frame": ti / len(frames), "render_ms_per_frame": tr / len(frames),
                            "frames_per_s": len(frames) / ((ti + tr) * 1e-3)}
    sc = vsg.Scene(voxel_size=VOXEL, truncation=TRUNC, hash_num_slots=SLOTS, num_sdf_blocks=BLOCKS)
    rr = vsg.Renderer(W, H)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    for _ in range(2):
        sc.reset()
        ti = tr = 0.0
        for i, f in enumerate(frames):
            pm, rgb, nm = dev[i]
            e[0].record()
            sc.integrate(pm, rgb, nm, W, H, TRUNC, f.pose, K.fx, K.fy, K.cx, K.cy)
            e[1].record()
            rr.render(sc, f.pose, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D)
            e[2].record()
            torch.cuda.synchronize()
            ti += e[0].elapsed_time(e[1])
            tr += e[1].elapsed_time(e[2])
        res["this_library"] = {"integrate_ms_per_frame": ti / len(frames), "render_ms_per_frame": tr / len(frames),
                               "frames_per_s": len(frames) / ((ti + tr) * 1e-3)}
    sc.close()
    rr.close()
    r, o = res["reference"], res["this_library"]
    res["speedup"] = {"frames_per_s": o["frames_per_s"] / r["frames_per_s"],
                      "integrate": r["integrate_ms_per_frame"] / o["integrate_ms_per_frame"],
                      "render": r["render_ms_per_frame"] / o["render_ms_per_frame"]}
    res["workload"] = WORKLOAD + f", {len(frames)} frames, one frame per call pair"
    res["build"] = "reference VoxelScene.cu, RayCastRender.cu, CUDAHashRef.cu for sm_100a, nvcc defaults"
    return res


def headline_config(args, world: int) -> dict:
    """The headline workload's `config`, the same dict on both arms."""
    return {"workload": WORKLOAD, "frames_per_step": args.frames,
            "l2": "inputs larger than L2 (30 resident frames, 250 MB per step)",
            "parallelism": f"replicas{world}"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    frames, K = make_stream(args)
    res, wall = [], []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        r = cpu_baseline(frames[: max(2, min(len(frames), 4))], K, budget_s=15.0)
        if i >= args.warmup:
            res.append(r["value"])
            wall.append(time.perf_counter() - t0)
    v = statistics.median(res)
    # ms_per_step: the wall time of one sampled step as run (4 frames
    # integrated, a band of rows ray cast); `value` scales the sample to full
    # frames, so 1000 / value is the time one full frame would take
    line = {"metric": METRIC, "value": v, "unit": "frames/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.median(wall), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": headline_config(args, world),
            "sampling": {"sample": r["sample"],
                         "extrapolated": "frames/s of the sample scaled from its ray-cast rows to full frames",
                         "ms_per_full_frame": 1000.0 / v},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "frames/s", "cores": r["cores"], "kind": "port",
                             "cpu": r["cpu"], "sample": r["sample"]},
            "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch

    import vsg

    if args.room_only:
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps({"room": room_measure(measured_peak_hbm()[0], args.room_frames)}), flush=True)
        return

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    frames, K = make_stream(args)
    W, H = K.width, K.height
    dev = [(torch.from_numpy(f.pointmap).cuda(), torch.from_numpy(f.rgb).cuda(),
            torch.from_numpy(f.normals).cuda(), f.pose) for f in frames]
    sc = vsg.Scene(voxel_size=VOXEL, truncation=TRUNC, hash_num_slots=SLOTS, num_sdf_blocks=BLOCKS)
    rr = vsg.Renderer(W, H)

    def step():
        sc.reset()
        for pm, rgb, nm, T in dev:
            sc.integrate(pm, rgb, nm, W, H, TRUNC, T, K.fx, K.fy, K.cx, K.cy)
            rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D)

    # per-frame statistics (algorithmic bytes), outside the timed region; with
    # march statistics on, renders also count the distinct blocks they read
    sc.march_stats(True)
    sc.reset()
    per_frame = []
    for pm, rgb, nm, T in dev:
        sc.integrate(pm, rgb, nm, W, H, TRUNC, T, K.fx, K.fy, K.cx, K.cy)
        rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D)
        per_frame.append(sc.stats())
    sc.march_stats(False)
    sc.timing_reset()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record()
        for _ in range(args.steps):
            step()
        ev1.record()
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if dist:
        import shard

        ms = shard.max_over_ranks(ms, dist)
    # per step: reset (k_init_heap, k_init_counters, k_frame_begin) + per frame: k_frame_begin,
    # k_alloc, k_select, k_integrate, k_render_begin, k_tile_bounds, k_tile_order, k_render
    launches_per_step = 3 + len(dev) * 8
    # per-kernel times (separate pass with events around each launch)
    sc.timing(True)
    sc.timing_reset()
    step()
    kms, kcnt = sc.timing_read()
    sc.timing(False)
    names = {0: "alloc", 1: "integrate", 2: "render", 3: "select"}
    kern = {nm: {"ms_per_launch": float(kms[i] / max(kcnt[i], 1)), "launches": int(kcnt[i])}
            for i, nm in names.items()}
    # algorithmic bytes per launch (canonical 8-B voxel)
    npx = W * H
    upd = np.mean([p["frame_updated_blocks"] for p in per_frame])
    new = np.mean([p["frame_new_blocks"] for p in per_frame])
    vis = np.mean([p["frame_visible_blocks"] for p in per_frame])
    bytes_integ = upd * 512 * 16 + npx * 15
    bytes_alloc = npx * 12 + new * 20 + vis * 16
    n_ray = float(np.mean([p["render_blocks_read"] for p in per_frame]))  # distinct blocks the rays read
    bytes_render = n_ray * 512 * 5 + npx * (4 + 16 + 16 + 16)
    kern["alloc"]["alg_bytes"] = bytes_alloc
    kern["integrate"]["alg_bytes"] = bytes_integ
    kern["render"]["alg_bytes"] = bytes_render
    kern["render"]["blocks_read_per_frame"] = n_ray
    kern["select"]["alg_bytes"] = float(np.mean([p["high_water"] for p in per_frame])) * 9 + vis * 4
    kern["render"]["samples_full_per_frame"] = float(np.mean([p["render_samples_full"] for p in per_frame]))
    for k in ("samples_skipped", "jumps", "singles", "lane_iters", "warp_iters"):
        kern["render"][k + "_per_frame"] = float(np.mean([p["render_" + k] for p in per_frame]))
    dom = max(kern, key=lambda k: kern[k]["ms_per_launch"])
    traffic = issue = None
    try:  # DRAM bytes per launch of the same kernel from one committed ncu capture
        tr = json.load(open(os.path.join(ROOT, "profiles", "roofline_traffic.json")))
        traffic = tr.get("k_" + dom, {}).get("dram_bytes_per_launch")
        # and, for the issue-bound ray caster, that capture's warp-issue figures
        issue = tr.get("k_" + dom, {}).get("issue")
    except (OSError, ValueError):
        pass
    peak, peak_kind = measured_peak_hbm()
    ach = kern[dom]["alg_bytes"] / (kern[dom]["ms_per_launch"] * 1e-3) / 1e9
    total_bytes = bytes_integ + bytes_alloc + bytes_render
    fps = args.frames * args.steps * world / (ms * 1e-3)
    line = {"metric": METRIC, "value": fps, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": headline_config(args, world), "mpix_per_s": fps * npx / 1e6,
            "gpu_launches": launches_per_step * args.steps,
            "kernels": kern,
            "frame_bytes": total_bytes, "frame_gbps": total_bytes * fps / world / 1e9,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "traffic": traffic, "peak_kind": peak_kind,
                         **({"issue_from_ncu": issue} if issue else {})},
            "clocks": clk.summary()}
    # side measurements after the timed step; a failure is recorded in the
    # line instead of losing it
    def side(name, fn, *a):
        try:
            line[name] = fn(*a)
        except Exception as exc:  # noqa: BLE001
            line[name] = {"error": f"{type(exc).__name__}: {exc}"}

    if args.headline_only:
        if rank == 0:
            print(json.dumps(line), flush=True)
        sc.close()
        rr.close()
        if dist:
            dist.destroy_process_group()
        return
    side("marching_cubes", mc_measure, sc, peak)
    side("surface_points", points_measure, sc, peak)
    side("ray_step", ray_step_measure, sc, frames, K)
    side("streaming", stream_measure, sc)
    side("adjoint", adjoint_measure, sc, frames, K)
    side("splat", splat_measure, frames, K, peak)
    if not args.no_ref_gpu and rank == 0:
        side("ref_gpu", ref_gpu_measure, frames, K)
    if not args.no_room:
        side("room", room_measure, peak, args.room_frames)
    if not args.no_e2e:
        line["e2e"] = e2e(args, frames, K, sc, rr)
    if not args.no_corridor:
        side("corridor", corridor_measure, args.corridor_frames)
        side("corridor_batched", corridor_batched_measure, 8, args.corridor_scale)
    if not args.no_batched:
        line["batched"] = run_batched(args, dist)
    if not args.no_cpu and rank == 0:
        line["cpu_baseline"] = cpu_baseline(frames, K)
    if rank == 0:
        print(json.dumps(line), flush=True)
    sc.close()
    rr.close()
    if dist:
        dist.destroy_process_group()


def mc_measure(sc, peak: float, reps: int = 10) -> dict:
    """Marching cubes over the scene as the timed step left it (the 30-frame
    volume): device time per launch from the library's event ring, triangle
    count, and algorithmic bytes = SDF of every block holding a weighted voxel
    (4 B x 512) + 72 B per triangle written (3 vertices + 3 normals, float3)."""
    import vsg

    mc = vsg.MarchingCubes(4_000_000)
    mc.run(sc)
    sc.timing(True)
    sc.timing_reset()
    for _ in range(reps):
        mc.run(sc)
    kms, kcnt = sc.timing_read()
    sc.timing(False)
    sc.timing_reset()
    n = mc.count()
    _, vox = sc.export()
    weighted = int((vox.reshape(-1, 512, 8)[:, :, 7] > 0).any(1).sum())
    mc.close()
    ms = float(kms[4] / max(kcnt[4], 1))
    alg = weighted * 512 * 4 + min(n, 4_000_000) * 72
    gbs = alg / (ms * 1e-3) / 1e9
    return {"triangles": n, "blocks_with_weight": weighted, "ms_per_launch": ms, "alg_bytes": alg,
            "achieved_gbs": gbs, "frac_of_peak": gbs / peak, "launches_timed": int(kcnt[4])}


def corridor_measure(n_frames: int, track_steps: int = 10, r_out: float = 4.0, r_in: float = 3.0,
                     track_frames: int = 100) -> dict:
    """Corridor workload (10 x 2.5 x 2.5 m, 300 primitives, 640x480, 4 mm,
    500 000 buckets, 2 000 000 pool blocks): a there-and-back walk of n_frames, frames
    generated on the device.  Pass 1, at the true poses, per frame: stream
    out every block farther than r_out from a point 1.5 m ahead of the
    camera, stream in the stored chunks (0.5 m) within r_in of it, integrate,
    ray cast -- wall clock per frame (the streaming calls synchronise).
    Pass 2 tracks instead over the first track_frames frames (the outbound
    walk): each frame's pose is estimated by track_steps Gauss-Newton steps
    (vsg.refine_pose) of its depth against the model from a
    constant-velocity prediction (residuals within 2 m and at incidence
    |cos| >= 0.5), then streamed and integrated at the estimate; reported
    with the trajectory error against the true poses (frame-to-model drift
    under the synthetic sensor's range-dependent noise)."""
    import torch

    import synth
    import vsg

    scene = synth.corridor_scene(3)
    K = synth.TABLETOP_K
    W, H = K.width, K.height
    poses = synth.corridor_poses(n_frames)
    frames = [synth.render_frame_torch(scene, K, P, seed=i, zmax=4.0, color_top=2.5) for i, P in enumerate(poses)]
    torch.cuda.synchronize()

    def run(track: bool):
        nf = min(track_frames, n_frames) if track else n_frames
        sc = vsg.Scene(voxel_size=VOXEL, truncation=TRUNC, hash_num_slots=500000, num_sdf_blocks=2000000,
                       max_chain_nodes=2000000)
        rr = vsg.Renderer(W, H)
        store = vsg.Store((0.5, 0.5, 0.5))
        est = []
        n_out = n_in = peak_res = refused = 0
        t_out = t_in = t_fuse = 0.0
        track_ms = 0.0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i, (pm, rgb, nm) in enumerate(frames[:nf]):
            T = poses[i].astype(np.float64)
            if track and i >= 1:
                pred = est[-1] @ (np.linalg.inv(est[-2]) @ est[-1]) if i >= 2 else est[-1]
                target = torch.where(pm[..., 2] > 0, pm[..., 2], torch.full_like(pm[..., 2], 1e10))
                t1 = time.perf_counter()
                T, _ = vsg.refine_pose(sc, rr, target, pred, K.fx, K.fy, K.cx, K.cy, MIN_D, 2.0,
                                       steps=track_steps, min_incidence=0.5)
                track_ms += (time.perf_counter() - t1) * 1e3
            est.append(T)
            T32 = T.astype(np.float32)
            c = (T32[:3, 3] + np.float32(1.5) * T32[:3, 2]).astype(np.float32)
            ta = time.perf_counter()
            n_out += sc.stream_out(store, c, r_out)
            tb = time.perf_counter()
            try:
                n_in += sc.stream_in(store, c, r_in)[0]
            except vsg.VsgError as exc:
                if exc.code != 5:  # VSG_ERR_TOO_LARGE: the pool cannot take them; nothing moved
                    raise
                refused += 1
            tc = time.perf_counter()
            sc.integrate(pm, rgb, nm, W, H, TRUNC, T32, K.fx, K.fy, K.cx, K.cy)
            rr.render(sc, T32, K.fx, K.fy, K.cx, K.cy, MIN_D, 4.0)
            torch.cuda.synchronize()
            t_out += tb - ta
            t_in += tc - tb
            t_fuse += time.perf_counter() - tc
            if i % 20 == 0:
                peak_res = max(peak_res, sc.stats()["allocated_blocks"])
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        st = sc.stats()
        out = {"frames": nf, "frames_per_s_wall": nf / wall, "ms_per_frame_wall": wall * 1e3 / nf,
               "blocks_streamed_out": n_out, "blocks_streamed_in": n_in,
               "resident_blocks_peak": max(peak_res, st["allocated_blocks"]),
               "stored_blocks_end": int(store.info()[0]), "stream_in_refused": refused, "flags": st["flags"],
               "ms_per_frame_stream_out": t_out * 1e3 / nf, "ms_per_frame_stream_in": t_in * 1e3 / nf,
               "ms_per_frame_integrate_render": t_fuse * 1e3 / nf}
        if track:
            terr = [float(np.linalg.norm(e[:3, 3] - p[:3, 3])) for e, p in zip(est, poses)]
            rerr = [float(np.degrees(np.arccos(np.clip((np.trace(e[:3, :3].T @ p[:3, :3]) - 1) / 2, -1, 1))))
                    for e, p in zip(est, poses)]
            out.update({"gn_steps_per_frame": track_steps, "track_ms_per_frame": track_ms / max(nf - 1, 1),
                        "trans_err_mean_m": float(np.mean(terr)), "trans_err_max_m": float(np.max(terr)),
                        "rot_err_mean_deg": float(np.mean(rerr)), "rot_err_max_deg": float(np.max(rerr))})
        sc.close()
        rr.close()
        return out

    res = {"frames": n_frames, "size": "640x480", "slots": 500000, "pool_blocks": 2000000, "r_out_m": r_out,
           "r_in_m": r_in,
           "chunk_m": 0.5, "fusion": run(False), "tracking": run(True)}
    del frames
    torch.cuda.empty_cache()
    return res


def corridor_batched_measure(n_corridors: int = 8, scale: float = 0.1, track_steps: int = 10,
                             r_out: float = 4.0, r_in: float = 3.0, pool_blocks: int = 600000) -> dict:
    """Config 4's batched form: n_corridors corridors (10 x 2.5 x 2.5 m, 300
    primitives, own seeds) of uneven length -- U[500, 2000] frames; the
    default run takes the first `scale` of each walk -- each frame tracked by track_steps
    Gauss-Newton steps from a constant-velocity guess, streamed (out beyond
    r_out, in within r_in of a point 1.5 m ahead of the estimate, 0.5 m
    chunks) and integrated + ray cast at the estimate; 640x480, 4 mm, 500 000
    buckets.  Sequential: the corridors one after the other through the
    per-scene calls (vsg.refine_pose, vsg_stream_out/in, vsg_integrate,
    vsg_render).  Batched: all live corridors advanced together -- tracking
    by vsg.refine_poses (one host synchronisation per Gauss-Newton step, one
    CUDA stream per corridor), streaming by vsg.stream_scenes (host threads,
    one stream each), integration and ray cast by one vsg_batch_step.  The
    two runs compute the same poses and volumes; frames/s by wall clock."""
    import torch

    import synth
    import vsg

    rng = np.random.default_rng(11)
    full = rng.integers(500, 2001, n_corridors)
    lengths = [max(8, int(round(n * scale))) for n in full]
    K = synth.TABLETOP_K
    W, H = K.width, K.height
    data = []
    for c, n in enumerate(lengths):
        scene = synth.corridor_scene(20 + c)
        # the first frames of the full-length walk: the per-frame motion of
        # the full workload (0.5-4 cm) whatever the scale
        poses = synth.corridor_poses(int(full[c]))[:n]
        fr = [synth.render_frame_torch(scene, K, P, seed=1000 * c + i, zmax=4.0, color_top=2.5)
              for i, P in enumerate(poses)]
        tg = [torch.where(pm[..., 2] > 0, pm[..., 2], torch.full_like(pm[..., 2], 1e10)) for pm, _, _ in fr]
        data.append((poses, fr, tg))
    torch.cuda.synchronize()

    def make():
        scs = [vsg.Scene(voxel_size=VOXEL, truncation=TRUNC, hash_num_slots=500000, num_sdf_blocks=pool_blocks,
                         max_chain_nodes=pool_blocks) for _ in lengths]
        rrs = [vsg.Renderer(W, H) for _ in lengths]
        sts = [vsg.Store((0.5, 0.5, 0.5)) for _ in lengths]
        return scs, rrs, sts

    def center(T):
        T32 = T.astype(np.float32)
        return (T32[:3, 3] + np.float32(1.5) * T32[:3, 2]).astype(np.float32)

    def predict(est):
        return est[-1] @ (np.linalg.inv(est[-2]) @ est[-1]) if len(est) >= 2 else est[-1]

    track_kw = dict(steps=track_steps, min_incidence=0.5)

    def sequential():
        scs, rrs, sts = make()
        ests = []
        t0 = time.perf_counter()
        for c, (poses, fr, tg) in enumerate(data):
            est = []
            for i, (pm, rgb, nm) in enumerate(fr):
                T = poses[i].astype(np.float64)
                if i >= 1:
                    T, _ = vsg.refine_pose(scs[c], rrs[c], tg[i], predict(est), K.fx, K.fy, K.cx, K.cy, MIN_D, 2.0,
                                           **track_kw)
                est.append(T)
                cc = center(T)
                scs[c].stream_out(sts[c], cc, r_out)
                try:
                    scs[c].stream_in(sts[c], cc, r_in)
                except vsg.VsgError as exc:
                    if exc.code != 5:  # VSG_ERR_TOO_LARGE: the pool cannot take them; nothing moved
                        raise
                T32 = T.astype(np.float32)
                scs[c].integrate(pm, rgb, nm, W, H, TRUNC, T32, K.fx, K.fy, K.cx, K.cy)
                rrs[c].render(scs[c], T32, K.fx, K.fy, K.cx, K.cy, MIN_D, 4.0)
            ests.append(est)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        for x in scs + rrs + sts:
            x.close()
        return wall, ests

    def batched():
        scs, rrs, sts = make()
        batch = vsg.Batch(scs, rrs)
        cstreams = [torch.cuda.Stream() for _ in lengths]
        ests = [[] for _ in lengths]
        t0 = time.perf_counter()
        for t in range(max(lengths)):
            live = [c for c in range(len(lengths)) if t < lengths[c]]
            track = [c for c in live if t >= 1]
            if track:
                Ts, _ = vsg.refine_poses([scs[c] for c in track], [rrs[c] for c in track],
                                         [data[c][2][t] for c in track], [predict(ests[c]) for c in track],
                                         (K.fx, K.fy, K.cx, K.cy), MIN_D, 2.0,
                                         streams=[cstreams[c] for c in track], **track_kw)
                for c, T in zip(track, Ts):
                    ests[c].append(T)
            for c in live:
                if t == 0:
                    ests[c].append(data[c][0][0].astype(np.float64))
            vsg.stream_scenes([scs[c] for c in live], [sts[c] for c in live], [center(ests[c][t]) for c in live],
                              r_out, r_in, streams=[cstreams[c] for c in live])
            frames = []
            for c in live:
                pm, rgb, nm = data[c][1][t]
                frames.append(batch.frame(c, pm, rgb, nm, W, H, TRUNC, ests[c][t].astype(np.float32), K.fx, K.fy,
                                          K.cx, K.cy, MIN_D, 4.0, render=True))
            batch.step(frames)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        batch.close()
        for x in scs + rrs + sts:
            x.close()
        return wall, ests

    t_seq, e_seq = sequential()
    t_bat, e_bat = batched()
    total = int(sum(lengths))
    same = all(np.array_equal(a, b) for ea, eb in zip(e_seq, e_bat) for a, b in zip(ea, eb))
    terr = [float(np.linalg.norm(e[:3, 3] - p[:3, 3])) for (poses, _, _), est in zip(data, e_bat)
            for e, p in zip(est, poses)]
    terr_seq = [float(np.linalg.norm(e[:3, 3] - p[:3, 3])) for (poses, _, _), est in zip(data, e_seq)
                for e, p in zip(est, poses)]
    del data
    torch.cuda.empty_cache()
    return {"workload": f"{n_corridors} corridors 640x480, the first {scale} of U[500,2000]-frame walks, 300 primitives each, "
                        f"{track_steps} Gauss-Newton steps per frame, streaming r_out {r_out} m / r_in {r_in} m",
            "corridor_frames": lengths, "frames": total,
            "frames_per_s": total / t_bat, "sequential_frames_per_s": total / t_seq,
            "speedup_vs_sequential": t_seq / t_bat, "same_poses_as_sequential": bool(same),
            "trans_err_mean_m": float(np.mean(terr)), "trans_err_max_m": float(np.max(terr)),
            "sequential_trans_err_mean_m": float(np.mean(terr_seq))}


def room_measure(peak: float, n_frames: int = 300, reps: int = 2, mc_every: int = 100,
                 mc_capacity: int = 16_000_000) -> dict:
    """Room workload (1280x720, fx=fy=910, 2 mm voxels, truncation 0.01 m,
    2^20 buckets and pool blocks; 4 x 3 x 2.5 m room with 40 boxes and 20
    spheres, random-walk camera; frames generated on the device): one step =
    reset + n_frames frames, each integrated then ray cast at its pose
    (0.2-4.0 m), with a marching-cubes extraction after every mc_every-th
    frame (frames 100/200/300), the volume far beyond L2.  Frames/s over
    `reps` steps (CUDA events), per-kernel device times and algorithmic bytes
    as for the headline, triangle counts and device times of the
    extractions."""
    import torch

    import synth
    import vsg

    K = synth.ROOM_K
    W, H = K.width, K.height
    scene = synth.room_scene(1)
    poses = synth.random_walk_poses(n_frames, 1)
    frames = [synth.render_frame_torch(scene, K, P, seed=i, zmax=4.0, color_top=2.5) + (P.astype(np.float32),)
              for i, P in enumerate(poses)]
    sc = vsg.Scene(voxel_size=0.002, truncation=0.01, hash_num_slots=1 << 20, num_sdf_blocks=1 << 20)
    rr = vsg.Renderer(W, H)
    mc = vsg.MarchingCubes(mc_capacity)

    def step(mc_counts=None):
        sc.reset()
        for i, (pm, rgb, nm, T) in enumerate(frames):
            sc.integrate(pm, rgb, nm, W, H, 0.01, T, K.fx, K.fy, K.cx, K.cy)
            rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, MIN_D, 4.0)
            if (i + 1) % mc_every == 0:
                mc.run(sc)
                if mc_counts is not None:
                    mc_counts.append(mc.count())

    sc.march_stats(True)
    sc.reset()
    per = []
    for pm, rgb, nm, T in frames:
        sc.integrate(pm, rgb, nm, W, H, 0.01, T, K.fx, K.fy, K.cx, K.cy)
        rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, MIN_D, 4.0)
        per.append(sc.stats())
    sc.march_stats(False)
    step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    sc.timing(True)
    sc.timing_reset()
    tri = []
    step(tri)
    kms, kcnt = sc.timing_read()
    sc.timing(False)
    npx = W * H
    upd = float(np.mean([p["frame_updated_blocks"] for p in per]))
    new = float(np.mean([p["frame_new_blocks"] for p in per]))
    vis = float(np.mean([p["frame_visible_blocks"] for p in per]))
    n_ray = float(np.mean([p["render_blocks_read"] for p in per]))
    alg = {"alloc": npx * 12 + new * 20 + vis * 16, "integrate": upd * 512 * 16 + npx * 15,
           "render": n_ray * 512 * 5 + npx * (4 + 16 + 16 + 16)}
    kern = {}
    for i, nm in {0: "alloc", 1: "integrate", 2: "render"}.items():
        kt = float(kms[i] / max(kcnt[i], 1))
        gbs = alg[nm] / (kt * 1e-3) / 1e9
        kern[nm] = {"ms_per_launch": kt, "alg_bytes": alg[nm], "achieved_gbs": gbs, "frac_of_peak": gbs / peak}
    mc_ms = [float(kms[4] / max(kcnt[4], 1))]
    fps = n_frames * reps / (ms * 1e-3)
    st = sc.stats()
    mc.close()
    sc.close()
    rr.close()
    del frames
    torch.cuda.empty_cache()
    return {"workload": f"room {n_frames}x1280x720, voxel 2mm, trunc 0.01m, 2^20 buckets/blocks, "
                        f"marching cubes after frames {', '.join(str(k) for k in range(mc_every, n_frames + 1, mc_every))}",
            "frames_per_s": fps, "mpix_per_s": fps * npx / 1e6, "ms_per_step": ms / reps, "steps": reps,
            "blocks_end": st["allocated_blocks"], "updated_blocks_per_frame": upd, "kernels": kern,
            "marching_cubes": {"after_frames": list(range(mc_every, n_frames + 1, mc_every)), "triangles": tri,
                               "ms_per_launch": mc_ms[0], "launches_timed": int(kcnt[4]),
                               "capacity": mc_capacity},
            "flags": st["flags"]}


def splat_measure(frames, K, peak: float, reps: int = 10) -> dict:
    """Point-cloud splat (vsg_splat_points, last-wins as the reference's
    generator): the valid points of four stream frames seen from the first
    frame's camera, with normals and colours, onto 640x480.  Device time per
    call from CUDA events (the call's work buffer comes from the stream-
    ordered pool).  Bytes = 27 per point read (point, normal, colour) + 31
    per pixel written (depth, point, normal, colour) + the 16-byte per-pixel
    winner words written and read once.  Device time: the timed calls are
    queued behind a device fill, so the host's issue latency is not timed."""
    import torch

    import vsg

    T0 = np.asarray(frames[0].pose, np.float64)
    pts, nrm, col = [], [], []
    for f in frames[:4]:
        m = np.any(f.pointmap != 0, -1)
        M = np.linalg.inv(T0) @ np.asarray(f.pose, np.float64)
        pts.append((f.pointmap[m].astype(np.float64) @ M[:3, :3].T + M[:3, 3]).astype(np.float32))
        nrm.append((f.normals[m].astype(np.float64) @ M[:3, :3].T).astype(np.float32))
        col.append(f.rgb[m])
    P, N, C = (torch.from_numpy(np.concatenate(x)).cuda() for x in (pts, nrm, col))
    W, H = K.width, K.height
    out = None
    for _ in range(3):
        out = vsg.splat_points(P, W, H, K.fx, K.fy, K.cx, K.cy, normals=N, colors=C)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    bufs = {k: out[k] for k in ("depth", "pointmap", "normalmap", "colormap")}
    L = vsg.lib()
    # a call's host work (argument checks, the stream-ordered work-buffer
    # allocation, five launches) takes about as long as its device work, so
    # the calls are queued behind a device fill of several milliseconds: the
    # events then time the device running them back to back, not host issue
    fill = torch.empty(1 << 28, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    for _ in range(8):
        fill.mul_(1.0)
    e0.record()
    for _ in range(reps):
        vsg.check("vsg_splat_points", L.vsg_splat_points(
            P.data_ptr(), P.shape[0], N.data_ptr(), N.shape[0], C.data_ptr(), C.shape[0], W, H, K.fx, K.fy, K.cx,
            K.cy, 0.0, float("inf"), vsg.SPLAT_LAST, bufs["depth"].data_ptr(), bufs["pointmap"].data_ptr(),
            bufs["normalmap"].data_ptr(), bufs["colormap"].data_ptr(), None, None))
    e1.record()
    torch.cuda.synchronize()
    del fill
    ms = e0.elapsed_time(e1) / reps
    n = int(P.shape[0])
    alg = n * 27 + W * H * (31 + 16 * 2)
    gbs = alg / (ms * 1e-3) / 1e9
    return {"points": n, "pixels_hit": out["n_valid"], "ms_per_call": ms, "mpoints_per_s": n / ms / 1e3,
            "alg_bytes": alg, "achieved_gbs": gbs, "frac_of_peak": gbs / peak}


def points_measure(sc, peak: float, reps: int = 10) -> dict:
    """Surface-point extraction over the scene as the timed step left it, with
    the reference main loop's arguments (-0.1, 0.1, weight >= 5,
    voxelSG.cpp:661): device time per launch from the event ring.  Bytes =
    voxels of every block holding a weighted voxel (8 B x 512) + 48 B per
    point written (three float4)."""
    import vsg

    pts = vsg.SurfacePoints(4_000_000)
    pts.extract(sc, -0.1, 0.1, 5)
    sc.timing(True)
    sc.timing_reset()
    for _ in range(reps):
        pts.extract(sc, -0.1, 0.1, 5)
    kms, kcnt = sc.timing_read()
    sc.timing(False)
    sc.timing_reset()
    n = pts.count()
    pts.close()
    _, vox = sc.export()
    weighted = int((vox.reshape(-1, 512, 8)[:, :, 7] > 0).any(1).sum())
    ms = float(kms[5] / max(kcnt[5], 1))
    alg = weighted * 512 * 8 + min(n, 4_000_000) * 48
    gbs = alg / (ms * 1e-3) / 1e9
    return {"points": n, "ms_per_launch": ms, "alg_bytes": alg, "achieved_gbs": gbs, "frac_of_peak": gbs / peak,
            "launches_timed": int(kcnt[5])}


def adjoint_measure(sc, frames, K, reps: int = 10, n_poses: int = 256, gn_steps: int = 20) -> dict:
    """Ray-cast adjoint at the last frame's pose of the final volume: device
    time of a recording render plus vsg_render_backward (dL/ddepth = 1 on
    every hit pixel, pose and voxel-SDF gradients), and the differentiable
    pose refinement workload: n_poses target poses (the stream's frames in
    turn) perturbed by seeded SE(3) noise (translation N(0, 1 cm), rotation
    N(0, 1 deg) per axis), each refined by gn_steps Gauss-Newton steps
    (vsg.refine_pose: Huber-weighted residuals of the rendered depth against
    the frame's noisy observed depth, 640x480)."""
    import torch

    import vsg

    W, H = K.width, K.height
    rr = vsg.Renderer(W, H)
    rr.record(True)
    T = np.asarray(frames[-1].pose, np.float32)
    gsdf = torch.zeros(sc.params.num_sdf_blocks * 512, dtype=torch.float32, device="cuda")
    rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D)
    gd = (rr.depth_tensor() < 1e9).float()
    hits = int(gd.sum().item())
    for _ in range(3):
        rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D)
        rr.backward(sc, T, K.fx, K.fy, K.cx, K.cy, grad_depth=gd, grad_sdf=gsdf)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    fwd = bwd = 0.0
    skipped = 0
    for _ in range(reps):
        e[0].record()
        rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D)
        e[1].record()
        _, skipped = rr.backward(sc, T, K.fx, K.fy, K.cx, K.cy, grad_depth=gd, grad_sdf=gsdf)
        e[2].record()
        torch.cuda.synchronize()
        fwd += e[0].elapsed_time(e[1])
        bwd += e[1].elapsed_time(e[2])
    # Gauss-Newton normal equations (residual 1 on every hit pixel)
    ne = 0.0
    for _ in range(reps):
        e[0].record()
        rr.pose_normal_equations(sc, T, K.fx, K.fy, K.cx, K.cy, gd)
        e[1].record()
        torch.cuda.synchronize()
        ne += e[0].elapsed_time(e[1])
    # pose refinement against each frame's noisy observed depth (invalid
    # pixels: no residual)
    observed = []
    for f in frames:
        z = torch.from_numpy(np.ascontiguousarray(f.pointmap[..., 2])).cuda()
        observed.append(torch.where(z > 0, z, torch.full_like(z, 1e10)))
    rng = np.random.default_rng(7)
    ratios = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    n_steps = 0
    for k in range(n_poses):
        fi = (k * 7) % len(frames)
        T_true = np.asarray(frames[fi].pose, np.float32)
        target = observed[fi]
        d0 = np.concatenate([rng.normal(size=3) * np.deg2rad(1.0), rng.normal(size=3) * 0.01])
        T_fin, _ = vsg.refine_pose(sc, rr, target, T_true.astype(np.float64) @ vsg.se3_exp(d0), K.fx, K.fy,
                                   K.cx, K.cy, MIN_D, MAX_D, steps=gn_steps)
        n_steps += gn_steps
        D = np.linalg.inv(T_true.astype(np.float64)) @ T_fin
        ang = np.arccos(np.clip((np.trace(D[:3, :3]) - 1) / 2, -1, 1))
        ratios.append(float(np.hypot(ang, np.linalg.norm(D[:3, 3])) /
                            np.hypot(np.linalg.norm(d0[:3]), np.linalg.norm(d0[3:]))))
    torch.cuda.synchronize()
    step_ms = (time.perf_counter() - t0) * 1e3 / n_steps
    rr.close()
    return {"hit_pixels": hits, "render_record_ms": fwd / reps, "backward_ms": bwd / reps,
            "normal_equations_ms": ne / reps, "skipped_pixels": skipped,
            "refine": {"method": "gauss-newton", "poses": n_poses, "steps_per_pose": gn_steps,
                       "target": "the frame's noisy observed depth", "ms_per_step_wall": step_ms,
                       "median_final_over_initial_err": float(np.median(ratios)),
                       "frac_poses_improved": float(np.mean(np.array(ratios) < 1.0))}}


def ray_step_measure(sc, frames, K) -> dict:
    """The opt-in march step (vsg_renderer_set_step, not the drop-in): the
    autotuner vsg.tune_ray_step over 0.1-1.0 x truncation on five of the
    stream's poses of the final volume -- ms per 640x480 ray cast and depth
    error against the reference's half-voxel march, per candidate, and the
    step it picks for a 1 mm tolerance on 99 % of the exact hits."""
    import vsg

    rr = vsg.Renderer(K.width, K.height)
    poses = [frames[i].pose for i in range(0, len(frames), max(1, len(frames) // 5))][:5]
    step, table = vsg.tune_ray_step(sc, rr, poses, (K.fx, K.fy, K.cx, K.cy), MIN_D, MAX_D, TRUNC,
                                    factors=(0.1, 0.15, 0.2, 0.25, 0.5, 0.75, 1.0), tol=1e-3, frac=0.99)
    rr.close()
    return {"chosen_step_m": step, "tolerance_m": 1e-3, "frac": 0.99, "candidates": table}


def stream_measure(sc) -> dict:
    """Streaming over the scene as the timed step left it: every block out to
    host memory and back (wall clock around each synchronous call; the calls
    copy through pinned staging, so PCIe bounds them).  Bytes = 4096 + 16 per
    block each way."""
    import time

    import vsg

    n0 = sc.stats()["allocated_blocks"]
    store = vsg.Store()
    sc.stream_out(store, (0.0, 0.0, 0.0), 3.0e38)  # selects nothing; sets up the staging buffers
    t0 = time.perf_counter()
    n_out = sc.stream_out(store, (0.0, 0.0, 0.0), 0.0)
    t1 = time.perf_counter()
    n_in, _ = sc.stream_in(store)
    t2 = time.perf_counter()
    store.close()
    nb = 4096 + 16
    return {"blocks": n0, "out_blocks": n_out, "in_blocks": n_in, "out_ms": (t1 - t0) * 1e3,
            "in_ms": (t2 - t1) * 1e3, "out_gbs": n_out * nb / max(t1 - t0, 1e-9) / 1e9,
            "in_gbs": n_in * nb / max(t2 - t1, 1e-9) / 1e9}


def run_batched(args, dist=None) -> dict:
    """Batched plain method: independent tabletop scans (own seeds; 160x120 /
    320x240 / 640x480; U[10,200] frames; 50000-400000 buckets) integrated and
    ray cast frame by frame.  Times the same frames one scan after the other
    through vsg_integrate + vsg_render ("plain per-scene") and all scans
    together through vsg_batch_step (graph-replayed steps, autotuned ray
    cast).  Frames are generated on the GPU and resident before timing.
    On N GPUs the scans are partitioned by frames x pixels (no exchange on
    the data path); times are the maximum over ranks."""
    import torch

    import shard
    import synth
    import vsg

    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    all_scans = synth.batched_scans(args.batched_scans)
    work = [len(s["poses"]) * s["K"].width * s["K"].height for s in all_scans]
    scans = [all_scans[i] for i in shard.partition(work, world)[rank]]
    scenes, rends, frames = [], [], []
    for i, sc in enumerate(scans):
        K = sc["K"]
        scenes.append(vsg.Scene(voxel_size=VOXEL, truncation=TRUNC, hash_num_slots=sc["buckets"],
                                num_sdf_blocks=sc["buckets"]))
        rends.append(vsg.Renderer(K.width, K.height))
        geo = synth.tabletop_scene(sc["seed"])
        frames.append([synth.render_frame_torch(geo, K, T, seed=sc["seed"] * 1000 + j) + (T,)
                       for j, T in enumerate(sc["poses"])])
    torch.cuda.synchronize()
    n_frames = sum(len(f) for f in frames)
    n_pix = sum(len(f) * sc["K"].width * sc["K"].height for f, sc in zip(frames, scans))

    def plain_pass():
        for i, sc in enumerate(scans):
            K = sc["K"]
            for pm, rgb, nm, T in frames[i]:
                scenes[i].integrate(pm, rgb, nm, K.width, K.height, TRUNC, T, K.fx, K.fy, K.cx, K.cy)
                rends[i].render(scenes[i], T, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D)

    batch = vsg.Batch(scenes, rends)
    steps = max(len(f) for f in frames)
    step_frames = []
    for t in range(steps):
        fl = []
        for i, sc in enumerate(scans):
            if t < len(frames[i]):
                K = sc["K"]
                pm, rgb, nm, T = frames[i][t]
                fl.append(batch.frame(i, pm, rgb, nm, K.width, K.height, TRUNC, T, K.fx, K.fy, K.cx, K.cy,
                                      MIN_D, MAX_D, render=True))
        step_frames.append(fl)

    def batched_pass():
        for fl in step_frames:
            batch.step(fl)

    def timed(fn):
        for s in scenes:
            s.reset()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return shard.max_over_ranks(e0.elapsed_time(e1) * 1e-3, dist)

    timed(batched_pass)  # first pass: eager steps, autotuning, graph captures
    t_batched = timed(batched_pass)
    timed(plain_pass)  # warm
    t_plain = timed(plain_pass)
    batch.close()
    n_frames = int(shard.sum_over_ranks(n_frames, dist))
    n_pix = shard.sum_over_ranks(n_pix, dist)
    res = {"workload": f"{len(all_scans)} tabletop scans (160x120/320x240/640x480, U[10,200] frames), "
                       f"{n_frames} frames, voxel 4mm, trunc 0.02m",
           "frames": n_frames, "steps": steps,
           "frames_per_s": n_frames / t_batched, "mpix_per_s": n_pix / t_batched / 1e6,
           "plain_per_scene_frames_per_s": n_frames / t_plain,
           "speedup_vs_plain": t_plain / t_batched,
           "sharding": f"{world} rank(s), scans partitioned by frames x pixels, no data-path collective"}
    for s in scenes:
        s.close()
    for r in rends:
        r.close()
    del frames
    torch.cuda.empty_cache()
    return res


def _cudart():
    """The CUDA runtime the library is linked against, for the e2e leg's
    asynchronous copies: $VSG_CUDART if set, else the already loaded
    libcudart.so.12 (libvsg.so depends on it), else the toolkit's copy.
    Raises when none loads: the e2e number must not be silently absent."""
    import ctypes
    import ctypes.util

    names = [os.environ.get("VSG_CUDART"), "libcudart.so.12", ctypes.util.find_library("cudart"),
             os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "lib64", "libcudart.so.12")]
    errors = []
    for n in names:
        if not n:
            continue
        try:
            return ctypes.CDLL(n)
        except OSError as e:
            errors.append(f"{n}: {e}")
    raise RuntimeError("e2e leg: no CUDA runtime library could be loaded (" + "; ".join(errors) + ")")


def e2e(args, frames, K, sc, rr) -> dict:
    """Same stream through the C ABI with pinned host inputs: per frame H2D of
    the point/colour/normal maps, integrate, ray cast, D2H of depth,
    position and colour -- all inside the timed region.  Pipelined over
    three CUDA streams: the H2D of frame i+1 and the D2H of frame i-1 run
    while frame i integrates and renders (two input buffer sets, two
    renderers, two pinned output sets, event dependencies); the scene's own
    updates stay in order on the compute stream.  `serial_value`: the same
    work with every copy and kernel on one stream."""
    import ctypes

    import torch

    import vsg

    W, H = K.width, K.height
    host = [(torch.from_numpy(f.pointmap).pin_memory(), torch.from_numpy(f.rgb).pin_memory(),
             torch.from_numpy(f.normals).pin_memory(), f.pose) for f in frames]
    cudart = _cudart()
    dev_in = [(torch.empty((H, W, 3), dtype=torch.float32, device="cuda"),
               torch.empty((H, W, 3), dtype=torch.uint8, device="cuda"),
               torch.empty((H, W, 3), dtype=torch.float32, device="cuda")) for _ in range(2)]
    rrs = [rr, vsg.Renderer(W, H)]
    outs = [r.outputs() for r in rrs]
    host_out = [(torch.empty((H, W), dtype=torch.float32).pin_memory(),
                 torch.empty((H, W, 4), dtype=torch.float32).pin_memory(),
                 torch.empty((H, W, 4), dtype=torch.float32).pin_memory()) for _ in range(2)]

    def d2h(dst, src_ptr, nbytes, stream):
        cudart.cudaMemcpyAsync(ctypes.c_void_p(dst.data_ptr()), ctypes.c_void_p(src_ptr), ctypes.c_size_t(nbytes),
                               2, ctypes.c_void_p(stream))

    s_in, s_comp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    nf = len(host)

    def step_pipelined():
        ev_in = [torch.cuda.Event() for _ in range(nf)]
        ev_used = [torch.cuda.Event() for _ in range(nf)]   # frame's inputs consumed (integrate done)
        ev_rend = [torch.cuda.Event() for _ in range(nf)]   # frame rendered
        ev_out = [torch.cuda.Event() for _ in range(nf)]    # frame's outputs copied out
        with torch.cuda.stream(s_comp):
            sc.reset(stream=s_comp.cuda_stream)
        for i, (pm, rgb, nm, T) in enumerate(host):
            k = i & 1
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(ev_used[i - 2])
                for dst, src in zip(dev_in[k], (pm, rgb, nm)):
                    dst.copy_(src, non_blocking=True)
                ev_in[i].record(s_in)
            s_comp.wait_event(ev_in[i])
            dpm, drgb, dnm = dev_in[k]
            sc.integrate(dpm, drgb, dnm, W, H, TRUNC, T, K.fx, K.fy, K.cx, K.cy, stream=s_comp.cuda_stream)
            ev_used[i].record(s_comp)
            if i >= 2:
                s_comp.wait_event(ev_out[i - 2])
            rrs[k].render(sc, T, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D, stream=s_comp.cuda_stream)
            ev_rend[i].record(s_comp)
            s_out.wait_event(ev_rend[i])
            od, op, oc = host_out[k]
            d2h(od, outs[k]["depth"], W * H * 4, s_out.cuda_stream)
            d2h(op, outs[k]["position"], W * H * 16, s_out.cuda_stream)
            d2h(oc, outs[k]["color"], W * H * 16, s_out.cuda_stream)
            ev_out[i].record(s_out)
        torch.cuda.synchronize()

    def step_serial():
        sc.reset()
        od, op, oc = host_out[0]
        dpm, drgb, dnm = dev_in[0]
        for pm, rgb, nm, T in host:
            dpm.copy_(pm, non_blocking=True)
            drgb.copy_(rgb, non_blocking=True)
            dnm.copy_(nm, non_blocking=True)
            sc.integrate(dpm, drgb, dnm, W, H, TRUNC, T, K.fx, K.fy, K.cx, K.cy)
            rr.render(sc, T, K.fx, K.fy, K.cx, K.cy, MIN_D, MAX_D)
            d2h(od, outs[0]["depth"], W * H * 4, 0)
            d2h(op, outs[0]["position"], W * H * 16, 0)
            d2h(oc, outs[0]["color"], W * H * 16, 0)
        torch.cuda.synchronize()

    steps = max(3, args.steps // 2)
    res = {}
    for name, fn in (("serial", step_serial), ("pipelined", step_pipelined)):
        for _ in range(2):
            fn()
        t0 = time.perf_counter()
        for _ in range(steps):
            fn()
        res[name] = nf * steps / (time.perf_counter() - t0)
    rrs[1].close()
    return {"value": res["pipelined"], "unit": "frames/s", "h2d_bytes_per_step": nf * W * H * (12 + 3 + 12),
            "d2h_bytes_per_step": nf * W * H * (4 + 16 + 16), "serial_value": res["serial"],
            "streams": "H2D / compute / D2H streams, double-buffered"}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
