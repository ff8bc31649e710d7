"""Benchmark of the transport loop on B200 (one JSON line on rank 0).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload cornell]

A step renders the whole workload once (every pixel x every sample) from the
device-resident scene.  The Cornell workload is the configuration of the plain Cornell
box: 256x256, 64 spp, max depth 8, roulette from depth 3, MIS, RGB binary32.

* value: samples/s of the whole job (all ranks' samples / max-over-ranks device time of
  K steps, CUDA events on the library's stream; the L2 is flushed between steps by
  writing a 256 MiB buffer on that stream, untimed).
* e2e: the same metric through the public API per step (CudaEngine.render_frame with the
  frame uniforms uploaded from host memory + read_export of the radiance to host memory),
  wall clock around each step, max over ranks.
* roofline: the dominant kernel class of an instrumented render of the same workload
  (CUDA events around each kernel class's launches), algorithmic bytes per launch / its
  mean duration, against the measured HBM copy bandwidth.
* cpu_baseline: the oracle (the CPU restatement) on the host cores, bounded sample.

Multi-GPU: replicas (each rank renders its own sample range of the same image; no data
path collective; the barrier and the max-over-ranks timing use torch.distributed).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "samples/s on 1 B200: batched wavefront and adjoint vs plain, at matched RMSE"


def workload(name):
    """(scene, strategy, width, height, spp_per_step, config) of a named workload."""
    from pathtracerglsl_b200 import scenes
    if name == "cornell":
        sc, st = scenes.cornell()
        w, h, spp = scenes.CORNELL_SIZE
        cfg = {"workload": "cornell-c1: 5 Lambert quads + Lambert sphere + dielectric sphere (IOR 1.5), "
                           "0.5x0.5 quad light Le=15, pinhole fov 40deg, MIS, RR from depth 3",
               "width": w, "height": h, "spp": spp, "spp_per_step": spp, "max_depth": 8, "color": "rgb"}
        return sc, st, w, h, spp, cfg
    if name in ("mesh", "mesh-bvh"):
        accel = "bvh" if name == "mesh-bvh" else "cwbvh"
        sc, st, (w, h, spp_total) = scenes.mesh_scene(accel=accel)
        spp = 16
        cfg = {"workload": "mesh-c2: level-8 icosphere (1,310,720 tris) with seeded value-noise displacement "
                           "(amplitude 0.05), 16 seeded similarity instances (TLAS), GGX F0 (0.9,0.6,0.3) with "
                           "per-triangle alpha ~ U(0.05,0.5), Lambert ground 0.5, procedural 1024x512 equirect "
                           "sky + 5e3 sun lobe over 0.5deg, MIS, RR from depth 3",
               "mesh_accel": accel, "width": w, "height": h, "spp": spp_total, "spp_per_step": spp,
               "max_depth": 12, "color": "rgb",
               "step": f"one {spp}-spp frame of the {spp_total}-spp configuration (samples/s is per sample)"}
        return sc, st, w, h, spp, cfg
    if name == "media":
        sc, st, (w, h, spp_total) = scenes.media_scene()
        spp = 16
        cfg = {"workload": "media-c3: dielectric sphere (IOR 1.33) holding a chromatic medium (sigma_t (0.5,1,2), "
                           "albedo 0.9, HG g 0.6) + null-interface sphere with a grey medium (sigma_t 2), Lambert "
                           "ground; sphere light r=0.05 emitting a 3000 K blackbody + 1x1 quad light of radiance 20; "
                           "NEE with equiangular placement (area-light extension), RR from depth 3",
               "width": w, "height": h, "spp": spp_total, "spp_per_step": spp, "max_depth": 64,
               "color": "spectral: 4 hero wavelengths, visible (sech^2) density over 380-780 nm",
               "step": f"one {spp}-spp frame of the {spp_total}-spp configuration (samples/s is per sample)"}
        return sc, st, w, h, spp, cfg
    raise SystemExit(f"unknown workload {name}")


# ---------------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.window = (0.0, float("inf"))

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append((time.time(), ln.strip()))

    def mark(self, t0, t1):
        """Keep only the samples read during [t0, t1] (the timed region)."""
        self.window = (t0, t1)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0, t1 = self.window
        for ts, ln in self.lines:
            if not (t0 <= ts <= t1 + 0.15):
                continue
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if parts[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------------- helpers
def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def cpu_baseline(sc, st, w, h, spp, seconds=10.0):
    """Oracle (CPU restatement) on all host threads over a bounded sample of the workload:
    1 spp over successive 1/16-height bands of the full image (the camera sees the whole
    frame) until about `seconds` of host time."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from pathtracerglsl_b200.compiler import Compiler
    oracle.build()
    r, pk = Compiler().compile(sc, st)
    threads = os.cpu_count() or 1
    band = max(1, h // 16)
    sess = oracle.Session(pk, r)          # scene set-up (the oracle's own BVH) is not timed
    done = 0
    k = 0
    t0 = time.perf_counter()
    while True:
        y0 = (k * band) % h
        th = min(band, h - y0)
        sess.render_tile(w, h, (0, y0, w, th), 1, first_sample=k // 16, salt=1, threads=threads)
        done += w * th
        k += 1
        el = time.perf_counter() - t0
        if el >= seconds or k >= 16 * spp:
            break
    return {"value": done / el, "unit": "samples/s", "cores": threads, "kind": "port",
            "sample": f"{done} samples: 1 spp over {k} bands of {w}x{band} pixels of the {w}x{h} image "
                      f"({el:.1f} s of host time)"}


def dist_setup(gpus):
    """One process per GPU (torchrun's environment): replicas, NCCL for the barrier and the
    max over ranks (pathtracerglsl_b200.replicas)."""
    from pathtracerglsl_b200.replicas import Replicas
    r = Replicas.from_env("nccl")
    return r.rank, r.local, r.world, (r if r.world > 1 else None)


def reduce_max(dist, x):
    return x if dist is None else dist.max(x)


def barrier(dist):
    if dist is not None:
        dist.barrier()


# ---------------------------------------------------------------------------------- arms
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from pathtracerglsl_b200.compiler import Compiler
    if args.workload in ("batch", "metric"):
        return run_reference_batch(args)
    if args.workload == "adjoint":
        from pathtracerglsl_b200 import scenes
        sc, st, (w, h, _spp_p, spp) = scenes.adjoint_scene(0)
        cfg = {"workload": "adjoint-c5 scene, forward walk only (the CPU restatement has no adjoint)",
               "width": w, "height": h, "spp": spp}
    else:
        sc, st, w, h, spp, cfg = workload(args.workload)
    oracle.build()
    r, pk = Compiler().compile(sc, st)
    threads = os.cpu_count() or 1
    # a bounded sample per step: 1 spp over one 1/16-height band of the full image (bands
    # cycle through the image), so --steps K --warmup W stays within a few minutes
    band = max(1, h // 16)
    sess = oracle.Session(pk, r)          # scene set-up (the oracle's own BVH) is not timed

    def step(k):
        y0 = (k * band) % h
        th = min(band, h - y0)
        sess.render_tile(w, h, (0, y0, w, th), 1, first_sample=k // 16, salt=1, threads=threads)
        return w * th

    for i in range(args.warmup):
        step(i)
    t0 = time.perf_counter()
    done = 0
    for i in range(args.steps):
        done += step(args.warmup + i)
    el = time.perf_counter() - t0
    value = done / el
    sspp = 1
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": "samples/s", "cores": threads, "kind": "port",
                             "sample": f"per step 1 spp over a {w}x{band} band of the {w}x{h} image, OpenMP over pixels"},
            "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference_batch(args):
    """The reference arm on the batched mix: the oracle (CPU restatement) on all host threads,
    each step 1 spp over one 1/16-height band of every job of the 64-job mix."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from pathtracerglsl_b200.compiler import Compiler
    jobs, cfg = batch_workload()
    if args.workload == "metric":
        cfg = dict(cfg, workload="metric: " + cfg["workload"])
    oracle.build()
    threads = os.cpu_count() or 1
    sessions = []
    for sc, st, (w, h, spp) in jobs:
        r, pk = Compiler().compile(sc, st)
        sessions.append((oracle.Session(pk, r), w, h, pk, r))   # set-up (the oracle's BVH) untimed

    def step(k):   # one band of every job of the mix
        n = 0
        for sess, w, h, _pk, _r in sessions:
            band = max(1, h // 16)
            y0 = (k * band) % h
            th = min(band, h - y0)
            sess.render_tile(w, h, (0, y0, w, th), 1, first_sample=0, salt=1, threads=threads)
            n += w * th
        return n

    for i in range(args.warmup):
        step(i)
    t0 = time.perf_counter()
    done = 0
    for i in range(args.steps):
        done += step(args.warmup + i)
    el = time.perf_counter() - t0
    value = done / el
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": "samples/s", "cores": threads, "kind": "port",
                             "sample": "per step 1 spp over a 1/16-height band of every job of the 64-job mix, "
                                       "OpenMP over pixels"},
            "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# DRAM bytes of the roofline kernel per closest-hit query (a shaded path, for k_shade), from
# one ncu capture of one whole wave of the workload at 1 spp with the autotuner's pick
# (dram__bytes_read.sum + dram__bytes_write.sum over the wave's launches / the wave's
# queries).  Scaled to a launch of the timed configuration by its queries per launch; the
# line labels it "ncu capture, scaled" (it is not measured in the timed run).
NCU_TRAFFIC_PER_QUERY = {("mesh", "closest"): 216.18, ("cornell", "shade"): 311.37}
# the kernel each workload's roofline is reported for (its dominant traversal / shading kernel)
ROOFLINE_KERNEL = {"mesh": "closest", "mesh-bvh": "closest", "cornell": "shade", "media": "shade"}


def algorithmic_bytes(kernel, c, cw=True):
    """Bytes the algorithm must move per render for one kernel class.  Path state: the
    SoA records each kernel reads and writes.  Traversal: every node popped (80 B wide /
    32 B binary BLAS node, 32 B TLAS node), every triangle tested (48 B: v0, e1, e2) and
    every instance entered (32 B placement).  The few-KB scene tables (regions,
    materials, lights) are cache-resident by design and not counted."""
    paths, closest, shadow = c["paths"], c["closest_queries"], c["shadow_queries"]
    alive = max(closest - paths, 0)
    node_b = 80 if cw else 32

    def trav(prefix):
        return (c.get(prefix + "blas_nodes", 0) * node_b + c.get(prefix + "triangles", 0) * 48
                + c.get(prefix + "tlas_nodes", 0) * 32 + c.get(prefix + "instances", 0) * 32)
    if kernel == "closest":
        return closest * (4 + 32 + 32) + trav("")
    if kernel == "shade":
        return closest * (4 + 136 + 16) + alive * (104 + 4) + shadow * (64 + 4)
    if kernel == "shadow":
        return shadow * (4 + 64 + 32) + trav("shadow_")
    if kernel == "generate":
        return paths * (104 + 4 + 16)
    if kernel == "film":
        return paths * 16
    return 0


def error_tiles(w, h, tile=64, n=4):
    """Crops of the image for the matched-RMSE reference: the whole frame when it is at most
    n tiles in area, else n tile x tile crops spread over it (engine coordinates)."""
    if w * h <= n * tile * tile:
        return [(0, 0, w, h)]
    fr = [(0.2, 0.3), (0.4, 0.65), (0.6, 0.35), (0.8, 0.7)]
    out = []
    for fx, fy in fr[:n]:
        x = min(max(0, int(fx * w) - tile // 2), w - tile)
        y = min(max(0, int(fy * h) - tile // 2), h - tile)
        out.append((x, y, min(tile, w), min(tile, h)))
    return out


def image_error(eng, w, h, spp, salt, ref_spp=65536, chunk=4096):
    """RMSE of one step's image against an FP64-accumulated 65,536-spp reference of the
    same frame rendered by this build with independent random numbers (the whole frame for
    small images, else four 64 x 64 crops rendered as tiles of the full image: each pixel
    computes exactly what the full render computes there).  sigma^2 per pixel channel =
    v / spp + v_ref / ref_spp.  'within_3sigma' takes v from the step's own samples (the
    literal gate, heavy-tailed at 16 spp); 'within_3sigma_ref_var' takes v from the
    reference's 65,536 samples (the per-sample variance, well estimated).  Matched RMSE:
    the measured RMSE equals the predicted one (ratio ~1) and ~99.7 % of channels lie
    within 3 sigma."""
    import numpy as np
    eng.pin_reset_salt(salt)
    eng.reset()
    eng.render_frame(w, h, spp)
    img = eng.read_export("radiance").astype(np.float64)
    var = eng.read_export("variance").astype(np.float64)
    d_all, s_lit, s_ref = [], [], []
    tiles = error_tiles(w, h)
    for (x, y, tw, th) in tiles:
        eng.pin_reset_salt(0x5EED0000 + salt)
        done = 0
        while done < ref_spp:
            k = min(chunk, ref_spp - done)
            eng.render_tile(x, y, tw, th, w, h, k, accumulate=done > 0)
            done += k
        ref = eng.read_export("radiance").astype(np.float64)
        ref_var = eng.read_export("variance").astype(np.float64)
        d_all.append((img[y:y + th, x:x + tw] - ref).ravel())
        s_lit.append((var[y:y + th, x:x + tw] / spp + ref_var / ref_spp).ravel())
        s_ref.append((ref_var / spp + ref_var / ref_spp).ravel())
    eng.width, eng.height = w, h
    eng.pin_reset_salt(salt)
    eng.reset()
    d, sl, sr = np.concatenate(d_all), np.concatenate(s_lit), np.concatenate(s_ref)
    rmse = float(np.sqrt(np.mean(d * d)))
    expected = float(np.sqrt(np.mean(sr)))

    def within(sig2):
        live = sig2 > 0
        return float(np.mean(np.abs(d[live]) <= 3.0 * np.sqrt(sig2[live]))) if live.any() else 1.0
    return {"value": rmse, "expected": expected, "ratio": rmse / expected if expected > 0 else None,
            "within_3sigma": within(sl), "within_3sigma_ref_var": within(sr), "reference_spp": ref_spp,
            "step_spp": spp, "crops": [list(t) for t in tiles],
            "reference": "FP64-accumulated film of this build, independent random numbers"}


def parse_tuning(text):
    """'sort_buckets=16,ray_sort=1' -> {'sort_buckets': 16, 'ray_sort': 1}."""
    out = {}
    for item in text.split(","):
        k, v = item.split("=")
        out[k.strip()] = int(v)
    return out


def run_ours(args):
    import torch
    rank, local, world, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    line = measure_ours(args, args.workload, rank, local, world, dist)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.close()


# the autotuner's pick for the mesh workload on this pool's B200s (recorded from its search
# over pool capacity x sort buckets x ray order), used where the mesh line rides along the
# composite metric run
MESH_PICK = "capacity=33554432,sort_buckets=8,ray_sort=1"


def measure_ours(args, name, rank, local, world, dist, tuning=None, cpu_leg=True, accel_build=None, rmse_leg=True):
    """One plain workload (one ptr_render per step): the JSON line (rank 0; None elsewhere).
    accel_build: where mesh BVHs are built at upload ('host' or 'device'; the upload's wall
    time is reported)."""
    import torch
    from pathtracerglsl_b200.compiler import Compiler
    from pathtracerglsl_b200.engine import CudaEngine

    sc, st, w, h, spp, cfg = workload(name)
    if args.spp:      # a smaller step of the same scene (profiler captures)
        spp = args.spp
        cfg = dict(cfg, spp_per_step=spp)
    renderer, packed = Compiler().compile(sc, st)
    eng = CudaEngine(local)
    accel_build = accel_build or args.accel_build
    eng.set_accel_build(accel_build)
    t_up = time.perf_counter()
    eng.register_scene(packed)
    eng.sync()
    cfg = dict(cfg, accel_build=accel_build, upload_s=time.perf_counter() - t_up)
    eng.load_renderer(renderer)
    eng.pin_reset_salt(1 + rank)      # each replica renders its own sample stream
    stream = torch.cuda.ExternalStream(eng.stream_handle(), device=torch.device("cuda", local))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def step():
        eng.reset()
        eng.render_frame(w, h, spp)

    # per-scene kernels (ptr_specialize: NVRTC, this scene x strategy), compiled before the
    # tuning search and the timed region
    if args.generic:
        cfg = dict(cfg, kernels="generic (precompiled, table-driven)")
    else:
        from pathtracerglsl_b200.engine import EngineError
        try:
            secs = eng.specialize()
            cfg = dict(cfg, kernels=f"specialised for this scene x strategy (NVRTC, {secs:.1f} s compile, untimed)")
        except EngineError as e:
            cfg = dict(cfg, kernels=f"generic: specialisation unavailable ({e})")

    # the project's autotuner picks the pool capacity (2^24 or 2^25 paths), the
    # occupant-sorted shading queue and the ray-coherence queue order for this workload
    # (at least two steps and 0.25 s per candidate, before the warm-up and the timed region)
    from pathtracerglsl_b200 import autotune
    tuning = tuning or args.tuning
    if tuning:   # a recorded pick (e.g. for a profiler run of the same configuration)
        pick = dict(autotune.DEFAULTS, **parse_tuning(tuning))
        eng.set_tuning(**pick)
        cfg = dict(cfg, tuning=pick, tuning_search="a recorded pick of the autotuner")
    else:
        cands = [dict(capacity=c, block=256, sort_buckets=k, ray_sort=r)
                 for c in (0, 1 << 25) for k in (1, 8, 16) for r in (0, 1)]
        tuned = autotune.tune(eng, step, cands, repeats=2, budget_s=60.0, min_time_s=0.25)
        cfg = dict(cfg, tuning={k: tuned["best"][k] for k in autotune.KNOBS},
                   tuning_search=[{k: r[k] for k in autotune.KNOBS + ("ms",)} for r in tuned["results"]])

    for _ in range(args.warmup):
        step()
    eng.sync()
    torch.cuda.synchronize()

    # ---- timed region: K steps, device time with events on the library's stream
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.5)                               # nvidia-smi start-up, outside the window
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier(dist)
    torch.cuda.synchronize()
    t_window = time.time()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(float(k))                 # untimed L2 flush (256 MiB > 126 MB L2)
            starts[k].record(stream)
            step()
            ends[k].record(stream)
    eng.sync()
    torch.cuda.synchronize()
    clocks.mark(t_window, time.time())
    barrier(dist)
    clk = clocks.stop()
    dev_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    dev_ms = reduce_max(dist, dev_ms)
    samples_total = w * h * spp * args.steps * world
    value = samples_total / (dev_ms / 1000.0)

    # ---- end to end through the public API (host uniforms in, host image out)
    img = None
    barrier(dist)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.reset()
        eng.render_frame(w, h, spp)
        img = eng.read_export("radiance", out=img)
    el = reduce_max(dist, time.perf_counter() - t0)
    e2e = {"value": samples_total / el, "unit": "samples/s",
           "h2d_bytes_per_step": 160, "d2h_bytes_per_step": int(img.nbytes)}

    # ---- image error of a step against a high-spp reference of the same frame (untimed)
    rmse = image_error(eng, w, h, spp, 1 + rank) if (rmse_leg and not args.no_rmse) else None

    # ---- instrumented passes (not part of the timed region): per-kernel-class device
    # time with CUDA events, then the traversal tallies of the counting kernels
    from pathtracerglsl_b200 import abi as _abi
    eng.reset()
    prof = eng.profile_render(w, h, spp, _abi.PROFILE_TIMING)
    eng.reset()
    eng.profile_render(w, h, spp, _abi.PROFILE_WORK)
    cnt = eng.counters()
    kernel = ROOFLINE_KERNEL.get(name) or max(prof.items(), key=lambda kv: kv[1][0])[0]
    kms, klaunch = prof[kernel]
    peak, peak_kind = measured_peaks()
    launch_ms = kms / max(klaunch, 1)
    bytes_per_launch = algorithmic_bytes(kernel, cnt, cfg.get("mesh_accel", "cwbvh") == "cwbvh") / max(klaunch, 1)
    achieved = bytes_per_launch / (launch_ms / 1000.0) / 1e9
    total_prof_ms = sum(v[0] for v in prof.values())
    roofline = {"bound": "hbm", "kernel": "k_" + kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": (NCU_TRAFFIC_PER_QUERY[(name, kernel)] * cnt["closest_queries"] / max(klaunch, 1)
                            if (name, kernel) in NCU_TRAFFIC_PER_QUERY else None),
                "traffic_source": ("ncu capture of one wave at 1 spp, scaled by queries per launch"
                                   if (name, kernel) in NCU_TRAFFIC_PER_QUERY else None),
                "bytes_per_launch": bytes_per_launch, "launch_ms": launch_ms,
                "share": {k: v[0] / total_prof_ms for k, v in prof.items()}}
    launches = sum(v[1] for v in prof.values()) + 1   # + the frame-parameter kernel

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(cfg, l2="flushed between steps (256 MiB write, untimed)",
                               parallelism=f"replicas x{world}"),
                "e2e": e2e, "roofline": roofline, "gpu_launches": launches * args.steps,
                "clocks": clk, "rmse": rmse,
                "error_flags": cnt["error_flags"],   # walk stack / guard errors of the counting pass (0 = none)
                "traversal": {k: cnt[k] for k in ("blas_nodes", "triangles", "tlas_nodes", "instances",
                                                   "shadow_blas_nodes", "shadow_triangles", "shadow_tlas_nodes",
                                                   "shadow_instances")},
                "rays": {"closest_per_sample": cnt["closest_queries"] / cnt["paths"],
                         "shadow_per_sample": cnt["shadow_queries"] / cnt["paths"],
                         "mrays_per_s": value * (cnt["closest_queries"] + cnt["shadow_queries"]) / cnt["paths"] / 1e6}}
        if cpu_leg and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(sc, st, w, h, spp)
    eng.close()
    return line if rank == 0 else None


# ---------------------------------------------------------------------------------- batch
def batch_workload():
    from pathtracerglsl_b200 import scenes
    jobs = scenes.batch_scenes(scenes.BATCH_SIZE, seed=0)
    cfg = {"workload": "batch-c4: 64 seeded Cornell-style scenes (Cornell walls + ceiling quad light, 1-200 "
                       "non-overlapping spheres r~U(0.05,0.3), material uniform over Lambert albedo U(0.2,0.9) / "
                       "dielectric IOR U(1.3,1.8) / GGX alpha U(0.05,0.6)), square resolutions 128..1024, "
                       "spp 16..256, max depth 4..32, MIS, RR from depth 3",
           "jobs": len(jobs), "samples_per_step": sum(w * h * spp for _, _, (w, h, spp) in jobs),
           "spheres": [len(sc["objects"]) - 5 for sc, _, _ in jobs], "color": "rgb",
           "step": "every job's full frame (all pixels x all spp) once"}
    return jobs, cfg


def run_batch(args):
    import torch
    rank, local, world, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    line = measure_batch(args, rank, local, world, dist)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.close()


PROGRESSIVE_SPP = 8   # samples per job of the progressive plain (the reference's frame loop)


def measure_batch(args, rank, local, world, dist, cpu_leg=True):
    """Batched wavefront (one ptr_render_batch over the 64 jobs, CUDA graph per wave, the
    mix's union-census kernels) against three plain forms on the same frames: one
    ptr_render per job at its full spp with each job's own per-scene kernels (the
    strongest plain), the same with the generic kernels, and the reference's own frame
    loop (one scene per launch, one sample per pixel per launch: Engine.renderFrame).  All
    forms draw identical per-sample estimators and random streams, so the RMSE is matched
    by construction (the GPU tests check batched = plain per job)."""
    import torch
    from pathtracerglsl_b200.compiler import Compiler
    from pathtracerglsl_b200.engine import CudaEngine, EngineError

    jobs, cfg = batch_workload()
    items = [Compiler().compile(sc, st) for sc, st, _ in jobs]
    frames = [(w, h, spp, 0, 1 + 1000 * rank + j) for j, (_, _, (w, h, spp)) in enumerate(jobs)]
    samples_step = cfg["samples_per_step"]
    eng = CudaEngine(local)
    b = eng.batch(items)
    # batched kernels for the mix's union census and each job's per-scene kernels (NVRTC,
    # untimed), before the tuning search
    specialised = not args.generic
    if specialised:
        try:
            secs = b.specialize(plain=True)
            cfg = dict(cfg, kernels=f"batched: specialised for the mix's union occupant census; plain: each job's "
                                    f"per-scene kernels (NVRTC, {secs:.1f} s of compiles, untimed)")
        except EngineError as e:
            specialised = False
            cfg = dict(cfg, kernels=f"generic: specialisation unavailable ({e})")
    if not specialised:
        cfg = dict(cfg, kernels="generic (precompiled, table-driven)")
    # the project's autotuner picks pool capacity, block size and sort-bucket count on a
    # reduced copy of the mix (every job at 1/16 of its spp), then every arm uses the pick
    from pathtracerglsl_b200 import autotune
    if args.tuning:   # a recorded pick (e.g. for a profiler run of the same configuration)
        pick = dict(autotune.DEFAULTS, **parse_tuning(args.tuning))
        eng.set_tuning(**pick)
        cfg = dict(cfg, tuning=pick, tuning_search="a recorded pick of the autotuner")
    else:
        small = [(w, h, max(1, spp // 16), 0, 7) for (w, h, spp, _f, _s) in frames]
        tuned = autotune.tune(eng, lambda: b.render(small), budget_s=40.0)
        cfg = dict(cfg, tuning={k: tuned["best"][k] for k in autotune.KNOBS},
                   tuning_search=[{k: r[k] for k in autotune.KNOBS + ("ms",)} for r in tuned["results"]])
    stream = torch.cuda.ExternalStream(eng.stream_handle(), device=torch.device("cuda", local))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    for _ in range(args.warmup):
        b.render(frames)
    b.render_plain(frames)
    torch.cuda.synchronize()

    def timed(fn, steps):
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        barrier(dist)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for k in range(steps):
                flush.fill_(float(k))
                starts[k].record(stream)
                fn()
                ends[k].record(stream)
        eng.sync()
        torch.cuda.synchronize()
        return reduce_max(dist, sum(s_.elapsed_time(e_) for s_, e_ in zip(starts, ends)))

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.5)
    t_window = time.time()
    dev_ms = timed(lambda: b.render(frames), args.steps)
    clocks.mark(t_window, time.time())
    clk = clocks.stop()
    value = samples_step * args.steps * world / (dev_ms / 1000.0)
    # the plain forms, a few steps each (the same frames, after the headline's timed region)
    k_plain = min(args.steps, 3)
    plain_ms = timed(lambda: b.render_plain(frames, sync=False), k_plain)
    plain = samples_step * k_plain * world / (plain_ms / 1000.0)
    plain_generic = None
    if specialised:
        b.specialize_off()
        gen_ms = timed(lambda: b.render_plain(frames, sync=False), k_plain)
        plain_generic = samples_step * k_plain * world / (gen_ms / 1000.0)
        b.specialize(plain=True)
    prog_frames = [(w, h, min(spp, PROGRESSIVE_SPP), 0, salt) for (w, h, spp, _f, salt) in frames]
    prog_samples = sum(w * h * spp for (w, h, spp, _f, _s) in prog_frames)
    b.render_progressive([(w, h, 2, 0, salt) for (w, h, _s, _f, salt) in prog_frames])   # untimed warm-up
    prog_ms = timed(lambda: b.render_progressive(prog_frames, sync=False), 2) / 2.0
    progressive = prog_samples * world / (prog_ms / 1000.0)

    # end to end: tables from host memory in, every job's radiance out to host memory
    barrier(dist)
    torch.cuda.synchronize()
    k_e2e = min(args.steps, 5)   # the whole mix is ~2.4 s a step: a few steps bound the run
    t0 = time.perf_counter()
    d2h = 0
    for _ in range(k_e2e):
        b.render(frames)
        d2h = 0
        for j in range(len(b)):
            d2h += b.read_export(j).nbytes
    el = reduce_max(dist, time.perf_counter() - t0)
    e2e = {"value": samples_step * k_e2e * world / el, "unit": "samples/s", "steps": k_e2e,
           "h2d_bytes_per_step": len(b) * (1024 + 32 + 160 + 8), "d2h_bytes_per_step": d2h}

    prof = b.profile(frames)
    cnt = b.counters()
    kernel, (kms, klaunch) = max(prof.items(), key=lambda kv: kv[1][0])
    peak, peak_kind = measured_peaks()
    launch_ms = kms / max(klaunch, 1)
    bytes_per_launch = algorithmic_bytes(kernel, cnt) / max(klaunch, 1)
    achieved = bytes_per_launch / (launch_ms / 1000.0) / 1e9
    total_prof_ms = sum(v[0] for v in prof.values())
    roofline = {"bound": "hbm", "kernel": "k_" + kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
                "bytes_per_launch": bytes_per_launch, "launch_ms": launch_ms,
                "share": {k: v[0] / total_prof_ms for k, v in prof.items()}}
    launches = sum(v[1] for v in prof.values())
    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(cfg, l2="flushed between steps (256 MiB write, untimed)",
                               parallelism=f"replicas x{world}"),
                "plain": {"value": plain, "unit": "samples/s", "ms_per_step": plain_ms / k_plain, "steps": k_plain,
                          "form": "one ptr_render per job at its full spp" +
                                  (", each job's per-scene kernels" if specialised else ", generic kernels"),
                          "batched_over_plain": value / plain,
                          "rmse": "matched: identical per-sample estimators and random streams"},
                "plain_generic": (None if plain_generic is None else
                                  {"value": plain_generic, "unit": "samples/s", "steps": k_plain,
                                   "form": "one ptr_render per job at its full spp, generic kernels",
                                   "batched_over_plain": value / plain_generic}),
                "plain_progressive": {"value": progressive, "unit": "samples/s", "ms": prog_ms,
                                      "samples": prog_samples,
                                      "form": f"the reference's frame loop: one scene and one sample per pixel per "
                                              f"ptr_render (Engine.renderFrame), the first {PROGRESSIVE_SPP} samples "
                                              f"of every job",
                                      "batched_over_plain": value / progressive},
                "e2e": e2e, "roofline": roofline, "gpu_launches": launches * args.steps, "clocks": clk,
                "rays": {"closest_per_sample": cnt["closest_queries"] / cnt["paths"],
                         "shadow_per_sample": cnt["shadow_queries"] / cnt["paths"],
                         "mrays_per_s": value * (cnt["closest_queries"] + cnt["shadow_queries"]) / cnt["paths"] / 1e6}}
        if cpu_leg and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_batch(jobs)
    b.close()
    eng.close()
    return line


def cpu_baseline_batch(jobs, seconds=10.0):
    """The oracle on all host threads over a bounded sample of the mix: 1 spp over one
    1/16-height band of each job in turn until about `seconds` of host time."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from pathtracerglsl_b200.compiler import Compiler
    oracle.build()
    threads = os.cpu_count() or 1
    sessions = []
    for sc, st, (w, h, spp) in jobs:
        r, pk = Compiler().compile(sc, st)
        sessions.append((oracle.Session(pk, r), w, h, pk, r))   # set-up (the oracle's BVH) untimed
    done = 0
    k = 0
    t0 = time.perf_counter()
    while True:
        sess, w, h, _pk, _r = sessions[k % len(sessions)]
        band = max(1, h // 16)
        y0 = ((k // len(sessions)) * band) % h
        th = min(band, h - y0)
        sess.render_tile(w, h, (0, y0, w, th), 1, first_sample=0, salt=1, threads=threads)
        done += w * th
        k += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return {"value": done / el, "unit": "samples/s", "cores": threads, "kind": "port",
            "sample": f"{done} samples: 1 spp over {k} bands (1/16 of a job's height each, the jobs in turn) "
                      f"of the 64-job mix ({el:.1f} s of host time)"}


# ---------------------------------------------------------------------------------- adjoint
def run_adjoint(args):
    import torch
    rank, local, world, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    line = measure_adjoint(args, rank, local, world, dist)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.close()


def measure_adjoint(args, rank, local, world, dist, cpu_leg=True):
    """The inverse-rendering workload: loss = L2 between the image at the current
    parameters (64 spp primal) and a target rendered at seeded +-10 % perturbed parameters;
    one step = one path-replay adjoint pass at 16 spp (forward walk + replay, gradients of
    every material parameter in float64).  Reported beside it: the forward render at the
    same 16 spp (the adjoint's cost ratio) and the 64-spp primal."""
    import torch
    import numpy as np
    from pathtracerglsl_b200 import adjoint, scenes
    from pathtracerglsl_b200.compiler import Compiler
    from pathtracerglsl_b200.engine import CudaEngine

    sc, st, (w, h, spp_p, spp_a) = scenes.adjoint_scene(0)
    renderer, packed = Compiler().compile(sc, st)
    eng = CudaEngine(local)
    eng.register_scene(packed)
    eng.load_renderer(renderer)
    # per-scene kernels for the forward walk and (compiled at the first backward pass, in
    # the warm-up) the replay, untimed
    kernels = "generic (precompiled, table-driven)"
    if not args.generic:
        from pathtracerglsl_b200.engine import EngineError
        try:
            kernels = f"specialised for this scene x strategy (NVRTC, {eng.specialize():.1f} s compile, untimed)"
        except EngineError as e:
            kernels = f"generic: specialisation unavailable ({e})"
    theta = adjoint.param_table(packed)
    mask = adjoint.live_mask(packed)
    rng = np.random.RandomState(11)
    pert = theta * (1 + 0.1 * rng.uniform(-1, 1, theta.shape))
    eng.update_params(adjoint.with_params(packed, pert))
    eng.pin_reset_salt(1000 + rank)
    eng.render_frame(w, h, spp_p)
    target = eng.read_export("radiance").copy()
    eng.update_params(adjoint.with_params(packed, theta))
    eng.pin_reset_salt(2000 + rank)
    eng.reset()
    eng.render_frame(w, h, spp_p)
    primal = eng.read_export("radiance").copy()
    loss, dl = adjoint.l2_loss(primal, target)
    dl = dl.astype(np.float32)
    stream = torch.cuda.ExternalStream(eng.stream_handle(), device=torch.device("cuda", local))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def timed(fn, k_steps):
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(k_steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(k_steps)]
        barrier(dist)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for k in range(k_steps):
                flush.fill_(float(k))
                starts[k].record(stream)
                fn(k)
                ends[k].record(stream)
        eng.sync()
        torch.cuda.synchronize()
        return reduce_max(dist, sum(a.elapsed_time(b) for a, b in zip(starts, ends)))

    def adj_step(k):
        torch.cuda.nvtx.range_push("adjoint_step")   # names the step's launches for a profiler
        g = eng.backward(dl, w, h, spp_a, salt=3000 + 17 * k + rank)
        torch.cuda.nvtx.range_pop()
        return g

    def fwd_step(k):
        eng.pin_reset_salt(3000 + 17 * k + rank)
        eng.reset()
        eng.render_frame(w, h, spp_a)

    for k in range(args.warmup):
        adj_step(k)
        fwd_step(k)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.5)
    t_window = time.time()
    adj_ms = timed(adj_step, args.steps)
    clocks.mark(t_window, time.time())
    clk = clocks.stop()
    fwd_ms = timed(fwd_step, args.steps)
    samples = w * h * spp_a * args.steps * world
    value = samples / (adj_ms / 1000.0)
    # end to end: adjoint image from host memory in, gradient vector out to host memory
    barrier(dist)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g = None
    for k in range(args.steps):
        g = adj_step(k)
    el = reduce_max(dist, time.perf_counter() - t0)
    e2e = {"value": samples / el, "unit": "samples/s", "h2d_bytes_per_step": int(dl.nbytes) + 160,
           "d2h_bytes_per_step": int(g.nbytes)}
    # the forward pass of the same frame, instrumented: per-kernel-class device time
    eng.pin_reset_salt(77)
    eng.reset()
    from pathtracerglsl_b200 import abi as _abi
    prof = eng.profile_render(w, h, spp_a, _abi.PROFILE_TIMING)
    eng.reset()
    eng.profile_render(w, h, spp_a, _abi.PROFILE_WORK)
    cnt = eng.counters()
    if rank == 0:
        kernel, (kms, klaunch) = max(prof.items(), key=lambda kv: kv[1][0])
        peak, peak_kind = measured_peaks()
        launch_ms = kms / max(klaunch, 1)
        bytes_per_launch = algorithmic_bytes(kernel, cnt) / max(klaunch, 1)
        achieved = bytes_per_launch / (launch_ms / 1000.0) / 1e9
        total_prof_ms = sum(v[0] for v in prof.values())
        line = {"metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": adj_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "adjoint-c5: Cornell walls + ceiling light, 64 seeded spheres (Lambert RGB albedo / "
                                       "GGX alpha / dielectric IOR) + one grey-medium sphere (sigma_t 2, albedo 0.9, g 0.6); "
                                       "loss = L2 to a target at seeded +-10 % parameters; path-replay adjoint",
                           "width": w, "height": h, "spp_primal": spp_p, "spp_adjoint": spp_a, "max_depth": 8,
                           "parameters": int(mask.sum()), "color": "rgb", "kernels": kernels,
                           "l2": "flushed between steps (256 MiB write, untimed)", "parallelism": f"replicas x{world}",
                           "step": "one adjoint pass (forward walk + replay + float64 gradient scatter) at 16 spp"},
                "forward": {"value": samples / (fwd_ms / 1000.0), "unit": "samples/s", "ms_per_step": fwd_ms / args.steps,
                            "adjoint_over_forward_cost": adj_ms / fwd_ms},
                "loss": loss, "gradient_l2": float(np.linalg.norm(g[mask])),
                "e2e": e2e, "clocks": clk,
                "roofline": {"bound": "hbm", "kernel": "k_" + kernel + " (forward pass of the step)", "achieved": achieved,
                             "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                             "traffic": None, "bytes_per_launch": bytes_per_launch, "launch_ms": launch_ms,
                             "share": {k: v[0] / total_prof_ms for k, v in prof.items()}},
                "gpu_launches": args.steps * 2 * sum(v[1] for v in prof.values())}
        if cpu_leg and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(sc, st, w, h, spp_a)
            line["cpu_baseline"]["sample"] = "forward only (the oracle has no adjoint): " + line["cpu_baseline"]["sample"]
    eng.close()
    return line if rank == 0 else None


def rails_upload_seconds(local):
    """The mesh workload's scene uploaded from the reference's packed channels
    (ptr_upload_scene_rails): the channels are packed first, untimed (the App's work, whose
    BVH builds the reference already does on the host); timed is the upload call, which
    copies the channels, checks them, gathers the triangles and builds the wide BLAS on the
    device."""
    from pathtracerglsl_b200 import _native, rails
    from pathtracerglsl_b200.compiler import Compiler
    from pathtracerglsl_b200.engine import CudaEngine
    sc, st, *_ = workload("mesh")
    _, packed = Compiler().compile(sc, st)
    pr = rails.pack(packed, _native.load())
    eng = CudaEngine(local)
    try:
        t0 = time.perf_counter()
        eng.register_scene_rails(packed, pr)
        eng.sync()
        return time.perf_counter() - t0
    finally:
        eng.close()


# ---------------------------------------------------------------------------------- the metric
def run_metric(args):
    """The metric's own comparisons in one line: the headline is the batched wavefront on the
    64-job uneven mix (against its plain forms); beside it the path-replay adjoint against the
    forward pass on the adjoint scene, and the plain mesh workload (1080p, 1.31 M-triangle
    instanced CWBVH) with its matched RMSE against a 65,536-spp reference."""
    import torch
    rank, local, world, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    line = measure_batch(args, rank, local, world, dist)
    adj = measure_adjoint(args, rank, local, world, dist, cpu_leg=False)
    mesh = measure_ours(args, "mesh", rank, local, world, dist, tuning=MESH_PICK, cpu_leg=False)
    mesh_dev = measure_ours(args, "mesh", rank, local, world, dist, tuning=MESH_PICK, cpu_leg=False,
                            accel_build="device", rmse_leg=False)
    rails_s = rails_upload_seconds(local)
    if rank == 0:
        line["adjoint"] = {"value": adj["value"], "unit": "samples/s", "ms_per_step": adj["ms_per_step"],
                           "steps": adj["steps"], "config": adj["config"],
                           "forward": adj["forward"], "adjoint_over_forward_cost": adj["forward"]["adjoint_over_forward_cost"],
                           "loss": adj["loss"], "gradient_l2": adj["gradient_l2"], "e2e": adj["e2e"],
                           "roofline": adj["roofline"], "clocks": adj["clocks"]}
        line["mesh"] = {k: mesh[k] for k in ("value", "unit", "ms_per_step", "steps", "config", "e2e", "roofline",
                                             "clocks", "rmse", "rays", "traversal")}
        line["mesh"]["device_built"] = {
            "value": mesh_dev["value"], "unit": "samples/s", "ms_per_step": mesh_dev["ms_per_step"],
            "upload_s": mesh_dev["config"]["upload_s"], "host_built_upload_s": mesh["config"]["upload_s"],
            "over_host_built": mesh_dev["value"] / mesh["value"], "traversal": mesh_dev["traversal"],
            "clocks": mesh_dev["clocks"],
            "form": "the same workload with its 1.31 M-triangle BLAS built on the device (linear BVH + greedy "
                    "eight-wide collapse) instead of the host's SAH builders"}
        line["mesh"]["rails_upload_s"] = rails_s   # the scene from the reference's packed channels
        line["gpu_launches"] = line["gpu_launches"] + adj["gpu_launches"] + mesh["gpu_launches"] + mesh_dev["gpu_launches"]
        line["config"] = dict(line["config"], workload="metric: " + line["config"]["workload"],
                              also="adjoint-c5 (adjoint vs forward) and mesh-c2 (plain, matched RMSE) in the "
                                   "'adjoint' and 'mesh' keys")
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="metric",
                    help="metric (default: batch mix + adjoint + mesh), batch, adjoint, mesh, mesh-bvh, cornell, media")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tuning", default="", help="skip the autotuner: e.g. sort_buckets=16,ray_sort=1")
    ap.add_argument("--spp", type=int, default=0, help="samples per pixel per step (0: the workload's own)")
    ap.add_argument("--no-rmse", action="store_true", help="skip the high-spp image-error reference")
    ap.add_argument("--generic", action="store_true", help="keep the generic kernels (no ptr_specialize)")
    ap.add_argument("--accel-build", default="host", choices=["host", "device"],
                    help="where mesh BVHs are built at upload (plain workloads)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "metric":
        run_metric(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "adjoint":
        run_adjoint(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
