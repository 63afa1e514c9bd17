"""Benchmark of the B200 RVS synthesis path.

Default workload (N=1): 4 perspective inputs 1920x1080 (10-bit YUV420, 16-bit
depth) -> 1 perspective 1920x1080 view, seeded synthetic scene.  A step is
one synthesis of the virtual view from raw input planes resident in HBM:
loading the four views into the scene (copy + colour decode, the
reference's per-frame InputView::load) and synthesising.

  value  views/s with the input planes resident in HBM (device-timed with
         CUDA events around each synthesis; L2 flushed between steps).
  e2e    the same metric through the reference-facing C-ABI calls with host
         buffers (rvsb_host_stream_submit, the frame loop with its
         asynchronous loader and writer): pinned host -> device upload of
         the raw planes, synthesis and download of the YUV420 result every
         step, consecutive frames overlapped; the blocking one-frame call
         rvsb_synthesize_host is reported beside it.
  roofline  of the dominant kernel, with its algorithmic bytes per launch.
  batched / batched_configs  rvsb_synthesize_batch on the plain scene and on
         the two batched configurations (CUDA graphs, autotuned raster).
  served  the serving configuration: Poisson arrivals at 500 req/s for 60 s
         over three resident scene sets (arrival-limited); served_load the
         same mix closed-loop with a fixed number of requests in flight
         (capacity, latency and mean batch at that load).
  parity  every timed output (plain, a batch slot, two targets of each
         batched configuration, one served request per output class)
         against the reference's own CPU synthesis of the same target.
  cpu_baseline  the reference's own CPU synthesis (oracle/_ref, its
         sources compiled unmodified against an OpenCV stand-in; the
         oracle's restatement when that library is not built) on a bounded
         sample, 1 thread (the reference's loops are serial).

Multi-GPU: pose-parallel replicas (each rank synthesises its own views;
no collective on the data path), value = all ranks' views / max time.  The
serving and batched-configuration lines are per-GPU figures and are then
skipped unless asked for (--serve-seconds, --load-seconds).

--impl reference times the same reference CPU synthesis on the host cores,
one view per thread per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rvs-cuda_b200"))

METRIC = "synth views/s + p50/p99 ms, batched-served vs plain on B200, ≥50 dB vs CPU"
UNIT = "views/s"
CACHE = os.path.join(ROOT, ".scene_cache")


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,utilization.gpu,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 10:
                continue
            rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [r for r in rows if r[3].isdigit() and int(r[3]) > 0] or rows
        sm = [float(r[1]) for r in load if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in load for k in range(4) if r[6 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows), "samples_under_load": len(load)}


def percentile(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = (len(xs) - 1) * q / 100.0
    f = int(k)
    c = min(f + 1, len(xs) - 1)
    return xs[f] + (xs[c] - xs[f]) * (k - f)


def workload_plain():
    from rvsb import scenes
    wl = scenes.plain_1080p()
    scenes.cache_planes(wl, CACHE)
    return wl


def reference_cpu():
    """The reference's own CPU synthesis (oracle/_ref/libref.so, its sources
    compiled unmodified against an OpenCV stand-in) when it is built, else
    the oracle's restatement.  Returns (kind, synthesize(wl, target) -> YUV
    planes, description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    try:
        import ref
        ref.lib()
    except Exception:
        ref = None
    if ref is None:
        def synth(inputs, planes, target, exponent):
            return O.synthesize(inputs, planes, target, exponent)
        return "port", synth, "the oracle's restatement of the reference's CPU path"

    def synth(inputs, planes, target, exponent):
        # The reference's CPU mode decodes its inputs with CUDA loader kernels
        # (process_input_frame.cu); here their CPU restatement, which the GPU
        # tests check bit for bit against those kernels.
        cols = [O.decode_color(y, u, v, c.bit_depth_color) for c, (y, u, v, d) in zip(inputs, planes)]
        deps = [O.decode_depth(d, c) for c, (y, u, v, d) in zip(inputs, planes)]
        color, quality = ref.synthesize(inputs, cols, deps, target, exponent)
        return ref.write_color(color, target), quality
    return "reference", synth, ("the reference's own CPU synthesis (rvs/src transform, blending, inpainting, "
                                "writer and camera code compiled unmodified), inputs decoded by the CPU "
                                "restatement of its loader kernels")


def cpu_baseline(wl, n_views=4):
    """The reference's CPU path on `n_views` syntheses of the workload, 1
    thread (its loops are serial)."""
    kind, synth, desc = reference_cpu()
    t0 = time.perf_counter()
    for _ in range(n_views):
        synth(wl.inputs, wl.planes, wl.targets[0], wl.blending_factor)
    dt = time.perf_counter() - t0
    return {"value": n_views / dt, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{n_views} syntheses of the 4x1920x1080 -> 1920x1080 view, 1 thread, "
                      f"{dt:.1f} s; {desc}; host has {os.cpu_count()} cores"}


# With an equirectangular camera the reference's hole mask depends on the
# last bit of its C runtime's float trigonometry (std::cos/sin/atan2/asin);
# the CUDA path evaluates those correctly rounded.  There the mask must equal
# the oracle's (correctly rounded) exactly and the reference's to within this
# fraction of the pixels.
ERP_MASK_TOLERANCE = 1e-5


def parity_of(gpu_yuv, gpu_hole, ref_yuv, ref_quality, debug_matches=None, oracle_quality=None):
    """The parity bar of one output: PSNR per plane against the reference's
    output (10-bit peak), the fraction of samples more than 2 codes off, and
    whether the hole mask (!(quality > 0) before inpainting) is identical."""
    import numpy as np
    out = {}
    big = total = 0
    for name, g, c in zip("YUV", gpu_yuv, ref_yuv):
        d = g.astype(np.float64) - c.astype(np.float64)
        mse = float(np.mean(d * d))
        out["psnr_" + name] = float("inf") if mse == 0 else float(10 * np.log10(1023.0 ** 2 / mse))
        big += int((np.abs(d) > 2).sum())
        total += d.size
    out["frac_gt2"] = big / total
    ref_hole = ~(ref_quality > 0)
    out["mask_identical"] = bool(np.array_equal(gpu_hole, ref_hole))
    out["mask_pixels_differing"] = int((gpu_hole != ref_hole).sum())
    mask_ok = out["mask_identical"]
    if oracle_quality is not None:
        out["mask_identical_to_correctly_rounded_trig"] = bool(np.array_equal(gpu_hole, ~(oracle_quality > 0)))
        mask_ok = (out["mask_identical_to_correctly_rounded_trig"] and
                   out["mask_pixels_differing"] <= ERP_MASK_TOLERANCE * gpu_hole.size)
    if debug_matches is not None:
        out["debug_call_matches_timed_output"] = bool(debug_matches)
    out["ok"] = bool(min(out["psnr_Y"], out["psnr_U"], out["psnr_V"]) >= 50.0 and out["frac_gt2"] <= 0.005
                     and mask_ok and debug_matches is not False)
    return out


class ParityJobs:
    """Outputs of the timed calls kept for the parity check, with the hole
    mask of the same target from rvsb_synthesize_debug on the same scene
    (whose YUV must equal the timed output's)."""

    def __init__(self):
        self.jobs = []

    def add(self, name, scene, inputs, planes, target, p, gpu_planes):
        import numpy as np
        import torch
        wo, ho = target.width, target.height
        timed = tuple(t.cpu().numpy().view(np.uint16).copy() for t in gpu_planes)
        dout = [torch.empty(n, dtype=torch.int16, device="cuda")
                for n in (wo * ho, (wo // 2) * (ho // 2), (wo // 2) * (ho // 2))]
        dbg = {"blend_quality": torch.full((ho, wo), float("nan"), device="cuda")}
        scene.synthesize_debug(target, p, dout, dbg)
        torch.cuda.synchronize()
        dyuv = tuple(t.cpu().numpy().view(np.uint16) for t in dout)
        same = all(np.array_equal(a, b) for a, b in zip(dyuv, timed))
        hole = ~(dbg["blend_quality"].cpu().numpy() > 0)
        shape = ((ho, wo), (ho // 2, wo // 2), (ho // 2, wo // 2))
        self.jobs.append((name, list(inputs), list(planes), target, p.blending_factor,
                          tuple(a.reshape(s) for a, s in zip(timed, shape)), hole, same))

    def run(self):
        """Computes the reference's output of every job (in parallel over the
        host cores) and returns {name: parity}."""
        from concurrent.futures import ThreadPoolExecutor
        kind, synth, _ = reference_cpu()

        def one(job):
            name, inputs, planes, target, exponent, yuv, hole, same = job
            import oracle as O
            from rvsb import abi
            t0 = time.perf_counter()
            oq = None
            if kind == "reference":
                ryuv, rq = synth(inputs, planes, target, exponent)
                if any(c.projection == abi.EQUIRECTANGULAR for c in inputs + [target]):
                    _, oq, _ = O.synthesize(inputs, planes, target, exponent, want_intermediate=True)
            else:
                ryuv, rq, _ = O.synthesize(inputs, planes, target, exponent, want_intermediate=True)
            r = parity_of(yuv, hole, ryuv, rq, same, oq)
            r["against"] = kind
            r["target"] = f"{'ERP' if target.projection else 'perspective'} {target.width}x{target.height}"
            r["cpu_s"] = round(time.perf_counter() - t0, 2)
            return name, r

        with ThreadPoolExecutor(max(1, min(len(self.jobs), os.cpu_count() or 1))) as ex:
            return dict(ex.map(one, self.jobs))


def run_reference(args):
    """--impl reference: the reference's CPU synthesis on the host cores,
    one view per thread per step."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from concurrent.futures import ThreadPoolExecutor
    kind, synth, desc = reference_cpu()
    wl = workload_plain()
    threads = max(1, min(32, os.cpu_count() or 1))

    def one(_):
        synth(wl.inputs, wl.planes, wl.targets[0], wl.blending_factor)

    with ThreadPoolExecutor(threads) as ex:
        for _ in range(args.warmup):
            list(ex.map(one, range(threads)))
        step_times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            list(ex.map(one, range(threads)))
            step_times.append(time.perf_counter() - t0)
    total = sum(step_times)
    value = threads * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene, RVS file formats)",
        "config": {"workload": "plain_1080p: 4 perspective 1920x1080 inputs -> 1 perspective 1920x1080 view",
                   "step": f"{threads} views synthesised in parallel, one per host thread"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{args.steps} steps x {threads} views of the 4x1080p workload; {desc}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def measure_batched(ctx, scene, wl, slots, steps, flush, stream, world, jobs=None):
    """Views/s of rvsb_synthesize_batch on the resident scene: `slots` seeded
    poses of the same distribution per batch (one CUDA graph replay), inputs
    resident, L2 flushed between batches outside the timed events."""
    import torch
    import rvsb
    from rvsb import scenes
    targets = scenes.plain_1080p(n_targets=slots + 1).targets[1:]
    p = rvsb.params(wl.blending_factor)
    batch = rvsb.Batch(scene, slots, graphs=True)
    batch.set_autotune(True)
    batch.reserve(targets[0].width, targets[0].height)
    outs = [[torch.empty(n, dtype=torch.int16, device="cuda")
             for n in (c.width * c.height, (c.width // 2) * (c.height // 2), (c.width // 2) * (c.height // 2))]
            for c in targets]
    for _ in range(3):
        batch.synthesize(targets, p, outs, stream=stream)
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        batch.synthesize(targets, p, outs, stream=stream)
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    launches = batch.last_launch_count()
    variant = batch.last_raster_variant()
    batch.close()
    if jobs is not None:
        jobs.add("batched", scene, wl.inputs, wl.planes, targets[0], p, outs[0])
    from rvsb import replicas
    total = replicas.max_over_ranks(sum(ms) / 1000.0, world)
    return {"value": world * slots * steps / total, "unit": UNIT, "slots": slots, "batches": steps,
            "ms_per_batch": statistics.mean(ms), "ms_per_view": statistics.mean(ms) / slots,
            "launches_per_batch": launches, "graphs": True, "raster_variant": variant,
            "workload": f"plain_1080p scene, {slots} seeded poses per batch"}


def measure_batched_workload(ctx, name, slots, flush, stream, reps=2, jobs=None):
    """Views/s of a batched configuration: every target of the workload
    synthesised with rvsb_synthesize_batch in groups of `slots` (one graph
    replay per group), inputs resident; `reps` timed passes over all targets,
    L2 flushed before each pass."""
    import numpy as np
    import torch
    import rvsb
    from rvsb import scenes
    wl = scenes.WORKLOADS[name]()
    scenes.cache_planes(wl, CACHE)
    sc = rvsb.Scene(ctx, wl.inputs)
    for i, planes in enumerate(wl.planes):
        sc.upload(i, [np.ascontiguousarray(a, np.uint16) for a in planes], on_device=False)
    p = rvsb.params(wl.blending_factor)
    batch = rvsb.Batch(sc, slots, graphs=True)
    batch.set_autotune(True)
    batch.reserve(max(c.width for c in wl.targets), max(c.height for c in wl.targets))
    outs = [[torch.empty(n, dtype=torch.int16, device="cuda")
             for n in (c.width * c.height, (c.width // 2) * (c.height // 2), (c.width // 2) * (c.height // 2))]
            for c in wl.targets]
    batch.synthesize(wl.targets, p, outs, stream=stream)
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        batch.synthesize(wl.targets, p, outs, stream=stream)
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    n = len(wl.targets)
    variant = batch.last_raster_variant()
    batch.close()
    if jobs is not None:
        # the first target and one from the middle of the list (another batch)
        for k in sorted({0, n // 2}):
            jobs.add(f"{name}[{k}]", sc, wl.inputs, wl.planes, wl.targets[k], p, outs[k])
    sc.close()
    del outs
    torch.cuda.empty_cache()
    return {"value": n * reps / (sum(ms) / 1000.0), "unit": UNIT, "targets": n, "slots": slots,
            "raster_variant": variant,
            "ms_per_view": statistics.mean(ms) / n,
            "inputs": f"{len(wl.inputs)} x {wl.inputs[0].width}x{wl.inputs[0].height}"
                      f" {'ERP' if wl.inputs[0].projection else 'perspective'}",
            "outputs": sorted({f"{c.width}x{c.height}" for c in wl.targets})}


def serving_targets(workloads, n, seed=0x5E7E):
    """n requests of the serving mix: scene set chosen uniformly, output
    960x540 / 1920x1080 perspective / 4096x2048 equirectangular in ratio
    5:4:1, pose drawn around the scene set's own target poses."""
    import copy
    import random
    from rvsb import abi
    rng = random.Random(seed)
    out = []
    for _ in range(n):
        s = rng.randrange(len(workloads))
        base = copy.deepcopy(rng.choice(workloads[s].targets))
        r = rng.random()
        pos = [base.position[k] + rng.uniform(-0.02, 0.02) for k in range(3)]
        if r < 0.1:
            near_far = tuple(base.depth_range)
            cam = abi.make_camera(abi.EQUIRECTANGULAR, 4096, 2048, pos, (rng.uniform(-180, 180), 0, 0), near_far)
            cls = "erp4096x2048"
        else:
            w, h = (960, 540) if r < 0.6 else (1920, 1080)
            if base.projection == abi.EQUIRECTANGULAR:
                f = w / 2.0
            else:
                f = base.focal[0] * w / base.width
            rot = (base.rotation[0] + rng.uniform(-2, 2), base.rotation[1], base.rotation[2])
            cam = abi.make_camera(abi.PERSPECTIVE, w, h, pos, rot, tuple(base.depth_range), (f, f))
            cls = f"{w}x{h}"
        out.append((s, cam, cls))
    return out


def measure_served(ctx, seconds, rate, lanes, max_batch, p, jobs=None):
    """Open-loop serving: Poisson arrivals at `rate` requests/s for `seconds`
    on the three resident scene sets (2 x 960x540, 4 x 1920x1080, 4 x ERP
    4096x2048 inputs).  Returns views/s and latency percentiles."""
    import random
    import numpy as np
    import torch
    import rvsb
    from rvsb import scenes
    wls = [scenes.plain_small(), scenes.plain_1080p(n_targets=8), scenes.batched_erp(n_targets=64)]
    scs = []
    for wl in wls:
        scenes.cache_planes(wl, CACHE)
        sc = rvsb.Scene(ctx, wl.inputs)
        for i, planes in enumerate(wl.planes):
            sc.upload(i, [np.ascontiguousarray(a, np.uint16) for a in planes], on_device=False)
        scs.append(sc)
    srv = rvsb.Server(ctx, lanes=lanes, max_batch=max_batch)
    ids = [srv.add_scene(sc) for sc in scs]
    for sid in ids:
        srv.reserve(sid, 1920, 1080)
        srv.reserve(sid, 4096, 2048)
    n = int(seconds * rate)
    reqs = serving_targets(wls, n)
    ring = {}
    for cls, (w, h) in (("960x540", (960, 540)), ("1920x1080", (1920, 1080)), ("erp4096x2048", (4096, 2048))):
        ring[cls] = [[torch.empty(k, dtype=torch.int16, device="cuda") for k in (w * h, w * h // 4, w * h // 4)]
                     for _ in range(16)]
    # warm-up: a few requests of each class on each scene set
    for k, (s, cam, cls) in enumerate(reqs[:24]):
        srv.submit(ids[s], cam, p, ring[cls][k % 16])
    srv.drain(600000)
    srv.poll(100000)
    torch.cuda.synchronize()
    rng = random.Random(0xA221)
    t_next = time.perf_counter()
    submitted = 0
    for k, (s, cam, cls) in enumerate(reqs):
        t_next += rng.expovariate(rate)
        while True:
            d = t_next - time.perf_counter()
            if d <= 0:
                break
            if d > 2e-4:
                time.sleep(d - 1e-4)
        srv.submit(ids[s], cam, p, ring[cls][k % 16])
        submitted += 1
    srv.drain(600000)
    res = srv.poll(n + 16)
    srv.close()
    if jobs is not None:
        # the last request of each output class still holds its ring slot
        last = {}
        for k, (s, cam, cls) in enumerate(reqs):
            last[cls] = k
        for cls, k in sorted(last.items()):
            s, cam, _ = reqs[k]
            jobs.add(f"served_{cls}", scs[s], wls[s].inputs, wls[s].planes, cam, p, ring[cls][k % 16])
    for sc in scs:
        sc.close()
    lat = sorted((r[5] - r[3]) * 1000.0 for r in res if r[1] == 0)
    t0 = min(r[3] for r in res)
    t1 = max(r[5] for r in res)
    per_class = {}
    by_id = {r[0]: r for r in res}
    return {"value": len(lat) / (t1 - t0), "unit": UNIT, "requests": len(res), "failed": sum(r[1] != 0 for r in res),
            "offered_rate": rate, "seconds": seconds, "lanes": lanes, "max_batch": max_batch,
            "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99), "max_ms": lat[-1] if lat else None,
            "mean_batch": statistics.mean(r[2] for r in res),
            "mix": "scene sets 2x960x540 / 4x1920x1080 / 4xERP4096x2048 uniform; outputs 960x540 : 1920x1080 : "
                   "ERP 4096x2048 = 5:4:1; Poisson arrivals; 60 GB budget",
            "duration_note": f"{seconds:g} s of arrivals (the serving configuration names 60 s)",
            "note": "open loop at the configured rate: arrival-limited, not a capacity figure (served_load is)"}


def measure_served_load(ctx, seconds, inflight, lanes, max_batch, p):
    """Closed-loop serving at a fixed load: `inflight` requests of the
    serving mix are kept outstanding (a new one is submitted as each
    completes) for `seconds`; views/s is the capacity at that load, with its
    latency percentiles and the mean batch the server formed."""
    import numpy as np
    import torch
    import rvsb
    from rvsb import scenes
    wls = [scenes.plain_small(), scenes.plain_1080p(n_targets=8), scenes.batched_erp(n_targets=64)]
    scs = []
    for wl in wls:
        scenes.cache_planes(wl, CACHE)
        sc = rvsb.Scene(ctx, wl.inputs)
        for i, planes in enumerate(wl.planes):
            sc.upload(i, [np.ascontiguousarray(a, np.uint16) for a in planes], on_device=False)
        scs.append(sc)
    srv = rvsb.Server(ctx, lanes=lanes, max_batch=max_batch)
    ids = [srv.add_scene(sc) for sc in scs]
    for sid in ids:
        srv.reserve(sid, 1920, 1080)
        srv.reserve(sid, 4096, 2048)
    reqs = serving_targets(wls, 200000, seed=0x10AD)
    # one output buffer per request in flight (a request's buffer is reused
    # only after it completed)
    sizes = {"960x540": (960, 540), "1920x1080": (1920, 1080), "erp4096x2048": (4096, 2048)}
    free = {cls: [[torch.empty(k, dtype=torch.int16, device="cuda") for k in (w * h, w * h // 4, w * h // 4)]
                  for _ in range(inflight)] for cls, (w, h) in sizes.items()}
    held = {}
    nxt = 0

    def submit():
        nonlocal nxt
        s, cam, cls = reqs[nxt % len(reqs)]
        nxt += 1
        buf = free[cls].pop()
        rid = srv.submit(ids[s], cam, p, buf)
        held[rid] = (cls, buf)

    def retire(results):
        for r in results:
            cls, buf = held.pop(r[0])
            free[cls].append(buf)

    # warm-up at the same load
    for _ in range(inflight):
        submit()
    t_end = time.perf_counter() + 1.0
    while time.perf_counter() < t_end:
        res = srv.poll(4096)
        retire(res)
        for _ in res:
            submit()
        if not res:
            time.sleep(2e-5)
    srv.drain(600000)
    retire(srv.poll(1 << 16))
    torch.cuda.synchronize()
    for _ in range(inflight):
        submit()
    done = []
    t_end = time.perf_counter() + seconds
    while time.perf_counter() < t_end:
        res = srv.poll(4096)
        retire(res)
        done.extend(res)
        for _ in res:
            submit()
        if not res:
            time.sleep(2e-5)
    srv.drain(600000)
    tail = srv.poll(1 << 16)
    retire(tail)
    done.extend(tail)
    srv.close()
    for sc in scs:
        sc.close()
    ok = [r for r in done if r[1] == 0]
    lat = sorted((r[5] - r[3]) * 1000.0 for r in ok)
    t0 = min(r[3] for r in done)
    t1 = max(r[5] for r in done)
    return {"value": len(ok) / (t1 - t0), "unit": UNIT, "requests": len(done),
            "failed": len(done) - len(ok), "in_flight": inflight, "lanes": lanes, "max_batch": max_batch,
            "seconds": seconds, "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99),
            "max_ms": lat[-1] if lat else None, "mean_batch": statistics.mean(r[2] for r in done),
            "mix": "the serving mix (scene sets and output classes as in 'served'), closed loop"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--e2e-steps", type=int, default=40)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-slots", type=int, default=16)
    ap.add_argument("--batch-steps", type=int, default=8)
    # the serving and batched-configuration lines are per-GPU figures: by
    # default measured on one GPU only (under torchrun each rank would hold
    # its GPU for them without adding to the job's aggregate)
    ap.add_argument("--serve-seconds", type=float, default=None)
    ap.add_argument("--serve-rate", type=float, default=500.0)
    ap.add_argument("--serve-lanes", type=int, default=4)
    ap.add_argument("--serve-batch", type=int, default=2)
    # closed-loop capacity of the serving path at a fixed number of requests in flight
    ap.add_argument("--load-seconds", type=float, default=None)
    ap.add_argument("--load-in-flight", type=int, default=6)
    ap.add_argument("--load-lanes", type=int, default=2)
    ap.add_argument("--load-batch", type=int, default=4)
    ap.add_argument("--no-batched-configs", action="store_true", default=None)
    # skip the parity check of the timed outputs against the reference's CPU path
    ap.add_argument("--no-parity", action="store_true")
    # only the per-view lines (value, e2e): for launch lists of the per-view path
    ap.add_argument("--plain-only", action="store_true")
    args = ap.parse_args()
    single = int(os.environ.get("WORLD_SIZE", "1")) == 1
    if args.serve_seconds is None:
        args.serve_seconds = 60.0 if single else 0.0
    if args.load_seconds is None:
        args.load_seconds = 10.0 if single else 0.0
    if args.no_batched_configs is None:
        args.no_batched_configs = not single
    if args.plain_only:
        args.no_batched_configs = True
        args.serve_seconds = 0.0
        args.load_seconds = 0.0
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        run_reference(args)
        return

    import numpy as np
    import torch
    import rvsb

    from rvsb import replicas
    world, rank, local = replicas.init()
    barrier = replicas.barrier
    allreduce_max = replicas.max_over_ranks
    torch.cuda.set_device(local)
    wl = workload_plain()
    target = wl.targets[0]
    p = rvsb.params(wl.blending_factor)
    ctx = rvsb.Context(local)
    stream = torch.cuda.current_stream()

    # Resident scene: raw planes uploaded once.
    scene = rvsb.Scene(ctx, wl.inputs)
    dev_planes = []
    for i, planes in enumerate(wl.planes):
        dp = [torch.from_numpy(np.ascontiguousarray(a).view(np.int16)).reshape(-1).cuda() for a in planes]
        dev_planes.append(dp)
        scene.upload(i, dp, on_device=True, stream=stream)
    wo, ho = target.width, target.height
    out = [torch.empty(n, dtype=torch.int16, device="cuda")
           for n in (wo * ho, (wo // 2) * (ho // 2), (wo // 2) * (ho // 2))]
    scene.set_profiling(True)
    scene.set_autotune(True)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def plain_step():
        scene.synthesize_frame(dev_planes, target, p, out, stream=stream)

    sampler = ClockSampler(local)
    sampler.start()
    for _ in range(args.warmup):
        plain_step()
    torch.cuda.synchronize()
    launches_per_step = scene.last_launch_count()

    step_ms, stage_acc = [], {k: 0.0 for k in rvsb.STAGES}
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.zero_()  # L2 flush (256 MiB > 126 MB L2), outside the timed events
        ev[k][0].record(stream)
        plain_step()
        ev[k][1].record(stream)
        ev[k][1].synchronize()
        for name, ms in scene.stage_times().items():
            stage_acc[name] += ms
    torch.cuda.synchronize()
    barrier(world)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    # Parity of the timed outputs: one GPU (every rank runs the same code;
    # with several, rank 0 alone would spend seconds of CPU after the others
    # finished).
    jobs = ParityJobs() if rank == 0 and world == 1 and not args.no_parity else None
    if jobs is not None:
        jobs.add("plain", scene, wl.inputs, wl.planes, target, p, out)
    total_s = sum(step_ms) / 1000.0
    max_total = allreduce_max(total_s, world)
    value = world * args.steps / max_total

    # e2e: reference-facing call with pinned host buffers.  A frame's input
    # planes lie in one pinned buffer in file order (per view: colour Y, U,
    # V, then depth), as a loader that reads a frame's files into one buffer
    # holds them; each output frame is one YUV420 buffer (Y, U, V).
    frame_in = torch.empty(sum(np.asarray(a).size for planes in wl.planes for a in planes),
                           dtype=torch.int16).pin_memory()
    host_planes, off = [], 0
    for planes in wl.planes:
        views = []
        for a in planes:
            t = frame_in[off:off + np.asarray(a).size]
            t.copy_(torch.from_numpy(np.ascontiguousarray(a).view(np.int16).reshape(-1)))
            views.append(t)
            off += t.numel()
        host_planes.append(views)

    def frame_out():
        buf = torch.empty(sum(t.numel() for t in out), dtype=torch.int16).pin_memory()
        parts, o = [], 0
        for t in out:
            parts.append(buf[o:o + t.numel()])
            o += t.numel()
        return parts

    host_out = frame_out()
    h2d = sum(t.numel() * 2 for planes in host_planes for t in planes)
    d2h = sum(t.numel() * 2 for t in host_out)
    for _ in range(3):
        ctx.synthesize_host(wl.inputs, host_planes, target, p, host_out, stream=stream)
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = []
    for _ in range(args.e2e_steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx.synthesize_host(wl.inputs, host_planes, target, p, host_out, stream=stream)
        b.record(stream)
        b.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    barrier(world)
    e2e_total = allreduce_max(sum(e2e_ms) / 1000.0, world)
    e2e_sync_value = world * args.e2e_steps / e2e_total
    # Pipelined frames through the same host buffers (rvsb_host_stream): each
    # step still uploads its 4 views from pinned memory and downloads its
    # YUV420 result; consecutive steps overlap on three streams.  Timed with
    # events on the caller's stream around all steps (join = every download
    # finished).
    hs = rvsb.HostStream(ctx, wl.inputs)
    host_outs = [host_out] + [frame_out() for _ in range(2)]
    for k in range(3):
        hs.submit(host_planes, target, p, host_outs[k % 3], stream=stream)
    hs.join(stream)
    torch.cuda.synchronize()
    barrier(world)
    ev_a, ev_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev_a.record(stream)
    for k in range(args.e2e_steps):
        hs.submit(host_planes, target, p, host_outs[k % 3], stream=stream)
    hs.join(stream)
    ev_b.record(stream)
    ev_b.synchronize()
    pipe_s = allreduce_max(ev_a.elapsed_time(ev_b) / 1000.0, world)
    hs.close()
    barrier(world)
    e2e_value = world * args.e2e_steps / pipe_s
    batched = None
    if not args.plain_only:
        batched = measure_batched(ctx, scene, wl, args.batch_slots, args.batch_steps, flush, stream, world, jobs)
    batched_configs = None
    if not args.no_batched_configs:
        batched_configs = {
            "batched_erp": measure_batched_workload(ctx, "batched_erp", 32, flush, stream, jobs=jobs),
            "batched_mixed": measure_batched_workload(ctx, "batched_mixed", 64, flush, stream, jobs=jobs),
        }
    served = None
    if args.serve_seconds > 0:
        served = measure_served(ctx, args.serve_seconds, args.serve_rate, args.serve_lanes, args.serve_batch, p,
                                jobs)
    served_load = None
    if args.load_seconds > 0:
        served_load = measure_served_load(ctx, args.load_seconds, args.load_in_flight, args.load_lanes,
                                          args.load_batch, p)
    clocks = sampler.stop()

    # Roofline of the dominant kernel (per launch, averaged over the timed steps).
    n_views = len(wl.inputs)
    n_in = sum(c.width * c.height for c in wl.inputs)
    n_out = wo * ho
    stage_avg = {k: v / args.steps for k, v in stage_acc.items()}
    stage_avg["upload_decode"] = statistics.mean(step_ms) - stage_avg["total"]
    # Algorithmic bytes per launch: warp 14 B per input pixel (depth read +
    # warped u, v, z write); the raster kernel reads the warped mesh (12 B
    # per input pixel) and, with the blend fused into it, (10N + 4) B per
    # output pixel (per view colour 3 x u16 + weight fp32, output YUV420 +
    # mask); the inpainting passes are charged the output write (4 B per
    # output pixel).
    blend_bytes = (10 * n_views + 4) * n_out
    algorithmic = {
        "warp": 14 * n_in,
        "raster": 12 * n_in + blend_bytes,
        "inpaint": 4 * n_out,
    }
    kernel_names = {"warp": "warp_kernel", "raster": "raster_kernel", "inpaint": "inpaint_*_kernel"}
    dominant = max(("warp", "bin", "raster", "inpaint"), key=lambda k: stage_avg[k])
    peak, peak_kind = measured_peaks()
    rk = dominant if dominant in algorithmic else "raster"
    achieved = algorithmic[rk] / (stage_avg[rk] / 1000.0) / 1e9
    traffic = None
    prof_path = os.path.join(ROOT, "profiles", "kernel_dram_traffic.json")
    if os.path.exists(prof_path):
        try:
            traffic = json.load(open(prof_path)).get(rk)
        except Exception:
            traffic = None
    roofline = {"kernel": kernel_names[rk], "bound": "hbm",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_launch": algorithmic[rk], "ms_per_launch": stage_avg[rk],
                "dominant_stage": dominant}
    stage_roof = {k: {"ms": stage_avg[k], "GBs": algorithmic[k] / (stage_avg[k] / 1000.0) / 1e9,
                      "frac": algorithmic[k] / (stage_avg[k] / 1000.0) / 1e9 / peak}
                  for k in algorithmic}
    triangles = 2 * sum((c.width - 1) * (c.height - 1) for c in wl.inputs)
    stage_roof["raster"]["triangles_per_s"] = triangles / (stage_avg["raster"] / 1000.0)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(wl)
    parity = None
    if jobs is not None:
        parity = jobs.run()
        parity = {"all_ok": all(v["ok"] for v in parity.values()), "outputs": parity,
                  "bar": "Y/U/V PSNR >= 50 dB and <= 0.5% of samples more than 2 codes off against the "
                         "reference's CPU output, identical hole mask (with an equirectangular camera: identical "
                         "to the correctly rounded trigonometry's and within 1e-5 of the pixels of the "
                         "reference's libm result); the mask from rvsb_synthesize_debug of the same target, "
                         "whose YUV must equal the timed output's"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": statistics.mean(step_ms), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene, RVS file formats: 10-bit YUV420, 16-bit depth)",
            "config": {"workload": "plain_1080p: 4 perspective 1920x1080 inputs -> 1 perspective 1920x1080 view "
                                   "(2x2 grid 0.15 m, f=1500, target +-10 cm / +-5 deg)",
                       "global_batch": world, "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "flushed between steps (256 MiB write outside the timed events)",
                       "blending_factor": wl.blending_factor},
            "p50_ms": percentile(step_ms, 50), "p99_ms": percentile(step_ms, 99),
            "stage_ms": stage_avg, "stage_roofline": stage_roof,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "call": "rvsb_host_stream_submit (pinned host buffers; uploads, synthesis and downloads of "
                            "consecutive frames overlapped, three frames in flight)",
                    "blocking_call": {"value": e2e_sync_value, "unit": UNIT, "p50_ms": percentile(e2e_ms, 50),
                                      "p99_ms": percentile(e2e_ms, 99),
                                      "call": "rvsb_synthesize_host (one frame at a time)"}},
            "batched": batched,
            "served": served,
            "served_load": served_load,
            "batched_configs": batched_configs,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "parity": parity,
            "clocks": clocks,
            "gpu_launches": launches_per_step * args.steps,
        }
        print(json.dumps(line))
    scene.close()
    ctx.close()
    replicas.finish(world)


if __name__ == "__main__":
    main()
