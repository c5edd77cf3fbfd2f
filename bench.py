"""Benchmark: Mrays/s of the path tracer on the 1M-sphere 1080p scene.

Workload (one step = one full frame): 1,000,000 spheres (r = 0.5, positions uniform in a cube
of side 140, per-particle colours), lightbox lighting, perspective camera fit to the scene,
1920x1080, 256 samples per pixel, 1 light sample -- ``Tracer.Path.sample(scene, 256)``.
Synthetic, seeded inputs stand in for the scene (the reference publishes no benchmark data).
``--workload`` selects the other measured configurations (the 1k-sphere 580x580 scene at 64 spp
x 32 light samples, the mixed-geometry 720p scene, Preview of the 1M-sphere scene).

Prints one JSON line:
  value      trace-only throughput: closest-hit queries per second over the K timed frames,
             scene and BVH resident in HBM, device time from CUDA events on the engine's stream
             (max over ranks); every rank renders its own frame (weak scaling, no collective)
  e2e        the same metric through the public API with host buffers: each step writes the
             geometry arrays from host memory, rebuilds the BVH, renders the frame and reads the
             sRGB image back
  roofline   the traversal kernel with the most device time: algorithmic bytes per ray (box and
             primitive test counts of the oracle's BVH on this scene, frozen below) x rays / its
             device time
  cpu_baseline  the CPU oracle on this host's cores on a bounded sample of the same frame
``--impl reference`` times the reference's CPU path (the oracle compiled from the reference's
own fresnel/common headers) on the same workload and prints the same line with impl=reference.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "Mrays/s on 1M-sphere 1080p path trace"


class Workload:
    """One measured configuration.

    box_tests / prim_tests: mean AABB and primitive tests per closest-hit query of the oracle's
    BVH (binned SAH, BVH2, leaves <= 4) on this scene and camera, measured by
    oracle/measure_ray_costs.py and frozen here; prim_bytes: bytes read per primitive test.
    Algorithmic bytes per ray = 24 (ray) + 16 (hit) + 32 A + prim_bytes P + 12 (colour).
    grid_cells / grid_spheres: mean cells visited and spheres tested per closest-hit query of the
    uniform sphere grid (1.5 cells per sphere), measured by the oracle's restatement of the grid
    walk on the rays of an oracle render of the frame (oracle/measure_ray_costs.py --grid) and
    frozen here.  Algorithmic bytes per ray through the grid = 52 + 8 C + 16 S.
    grid_cells / grid_refs for a scene traced through its grid over parts: cells visited and
    references listed in them per query (oracle/measure_ray_costs.py --parts-grid); bytes per ray
    = 52 + 8 C + 36 R (a 32 B record and a 4 B geometry index per reference).
    """

    def __init__(self, key, desc, scene, w, h, spp=1, light_samples=1, preview=False, aa_n=1,
                 box_tests=0.0, prim_tests=0.0, prim_bytes=16, grid_cells=None,
                 grid_spheres=None, grid_refs=None):
        self.key, self.desc, self.scene = key, desc, scene
        self.w, self.h, self.spp, self.light_samples = w, h, spp, light_samples
        self.full_size = (w, h)  # the frozen per-ray costs were measured on this frame
        self.preview, self.aa_n = preview, aa_n
        self.box_tests, self.prim_tests, self.prim_bytes = box_tests, prim_tests, prim_bytes
        self.grid_cells, self.grid_spheres, self.grid_refs = grid_cells, grid_spheres, grid_refs

    @property
    def bytes_per_ray(self):
        return 24 + 16 + 32 * self.box_tests + self.prim_bytes * self.prim_tests + 12

    @property
    def grid_bytes_per_ray(self):
        if self.grid_cells is None or self.grid_spheres is None:
            return None
        return 52 + 8 * self.grid_cells + 16 * self.grid_spheres

    @property
    def parts_grid_bytes_per_ray(self):
        if self.grid_cells is None or self.grid_refs is None:
            return None
        return 52 + 8 * self.grid_cells + 36 * self.grid_refs

    def build(self, device):
        from fresnel_b200 import workloads
        return getattr(workloads, self.scene)(device)


WORKLOADS = {
    "c2": Workload("c2", "config2: 1M spheres r=0.5, box 140, {w}x{h}, {spp} spp, 1 light sample, "
                   "lightbox", "config2", 1920, 1080, spp=256, box_tests=37.74, prim_tests=1.42,
                   grid_cells=2.997, grid_spheres=8.005),
    "c2-preview": Workload("c2-preview", "config2 Preview: 1M spheres, {w}x{h}, anti_alias "
                           "(64 samples per pixel)", "config2", 1920, 1080, preview=True, aa_n=8,
                           box_tests=29.41, prim_tests=0.95),
    "c1": Workload("c1", "config1: 1000 spheres r=0.5, box 20, outline 0.1, cloudy, {w}x{h}, "
                   "{spp} spp x 32 light samples", "config1", 580, 580, spp=64, light_samples=32,
                   box_tests=37.41, prim_tests=1.81, grid_cells=5.038, grid_spheres=10.793),
    "c4": Workload("c4", "config4", "config4", 1024, 1024, spp=16),
    "c5": Workload("c5", "config5", "serving_scene_first", 1280, 720, spp=16),
    "c3": Workload("c3", "config3: 200k spheres + 50k bonds + 20k cubes + 10k icosahedra, "
                   "{w}x{h}, {spp} spp, 1 light sample", "config3", 1280, 720, spp=128,
                   box_tests=43.51, prim_tests=1.86, prim_bytes=28, grid_cells=4.469,
                   grid_refs=10.886),
    "tour": Workload("tour", "kernel tour", "config2", 1920, 1080),
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    # 10 frames of the default workload take about 0.8 s: enough for a few clock samples at
    # nvidia-smi's 200 ms period inside the timed region
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="engine", choices=["engine", "reference"])
    p.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    p.add_argument("--spp", type=int, default=None, help="samples per pixel of one frame")
    p.add_argument("--width", type=int, default=None,
                   help="image width (smaller frames only for profiler captures)")
    p.add_argument("--height", type=int, default=None)
    p.add_argument("--cpu-seconds", type=float, default=15.0,
                   help="target duration of the CPU baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--trace-only", action="store_true",
                   help="skip the end-to-end leg, the CPU baseline and the further "
                        "configurations (profiler captures)")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the further configurations the default run reports under 'also'")
    a = p.parse_args()
    wl = WORKLOADS[a.workload]
    wl.w = a.width or wl.w
    wl.h = a.height or wl.h
    wl.spp = a.spp or wl.spp
    return a, wl


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi takes a moment to start: the timed region begins after its first sample
            t_end = time.monotonic() + 5.0
            while not self.samples and self.proc.poll() is None and time.monotonic() < t_end:
                time.sleep(0.02)
            self.samples.clear()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc is not None:
            # a timed region shorter than the sampling period still gets the sample after it
            t_end = time.monotonic() + 1.0
            while not self.samples and self.proc.poll() is None and time.monotonic() < t_end:
                time.sleep(0.02)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(s[0]) for s in self.samples if num(s[0]) is not None]
        mx = [num(s[1]) for s in self.samples if num(s[1]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if s[3 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


class Replicas:
    """Cross-rank bookkeeping of a replicas run (one process per GPU, each rendering its own
    frames; no data moves between ranks): a barrier, and the max (time) or sum (rays) of one
    number over the ranks.  With no process group every call is the identity."""

    def __init__(self, dist=None, device="cuda"):
        self.dist = dist
        self.device = device

    def _reduce(self, x, op):
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        return x if self.dist is None else self._reduce(x, self.dist.ReduceOp.MAX)

    def sum(self, x):
        return x if self.dist is None else self._reduce(x, self.dist.ReduceOp.SUM)

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def pin_gpu(local):
    """One process per GPU: expose only this rank's GPU to the engine and to torch."""
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x for x in vis.split(",") if x != ""]
        if local < len(ids):
            os.environ["CUDA_VISIBLE_DEVICES"] = ids[local]
    else:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    return local


def load_workloads():
    """The scene generators (fresnel_b200/workloads.py).  When fresnel_b200 is not imported
    (the reference arm), the file is loaded on its own by path, so that no module of the engine
    package, and none of its compiled libraries, is loaded."""
    if "fresnel_b200" in sys.modules:
        from fresnel_b200 import workloads
        return workloads
    import importlib.util
    name = "fresnel_b200_workloads_standalone"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(
            name, os.path.join(REPO, "fresnel_b200", "workloads.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        sys.modules[name] = mod
    return sys.modules[name]


_REFERENCE_API = {}


def reference_device(kind):
    """A CPU device of fresnel's own Python package (the reference's fresnel/*.py, staged
    beside the reference-built oracle) whose compiled backend is the CPU oracle of ``kind``
    and whose value types are the oracle's plain-Python ones: no library of the engine is
    loaded."""
    if kind not in _REFERENCE_API:
        import tempfile

        from oracle import reference_package
        root = tempfile.mkdtemp(prefix="fresnel_reference_")
        _REFERENCE_API[kind] = reference_package.import_fresnel(root, "oracle-values", kind)
    fresnel = _REFERENCE_API[kind]
    return fresnel.Device(mode="cpu")


def cpu_baseline(wl, dev, seconds, kind):
    """Time the CPU oracle on a bounded sample of the frame; ``dev`` is a fresnel-API device
    whose backend is the oracle.

    Path: rounds of random pixels of the frame, one pixel sample (x light samples) each.
    Preview: the frame at 1/8 of the resolution in each direction, same camera and AA level.
    """
    import numpy

    from oracle import cpu_module
    built = getattr(load_workloads(), wl.scene)(dev)
    if isinstance(built, list):  # a frame set: time its first frame
        scene, fw, fh = built[0]
    else:
        scene, fw, fh = built, wl.w, wl.h
    t0 = time.perf_counter()
    scene._scene.handle()  # BVH build, not timed
    build_s = time.perf_counter() - t0
    total_rays = 0
    elapsed = 0.0
    rounds = 0
    if wl.preview:
        w, h = max(1, wl.w // 8), max(1, wl.h // 8)
        tracer = dev.module.TracerDirect(dev._device, w, h)
        tracer.setAntialiasingN(wl.aa_n)
        while elapsed < seconds and rounds < 1000:
            tracer.stats = cpu_module.OrStats()
            t0 = time.perf_counter()
            tracer.render(scene._scene)
            elapsed += time.perf_counter() - t0
            total_rays += tracer.stats.rays
            rounds += 1
        sample = (f"{rounds} Preview renders of the frame at {w}x{h} (AA {wl.aa_n}x{wl.aa_n}), "
                  f"{total_rays} closest-hit queries in {elapsed:.1f} s "
                  f"(BVH build {build_s:.1f} s, not timed)")
    else:
        tracer = dev.module.TracerPath(dev._device, fw, fh, wl.light_samples)
        tracer.setSeed(2)
        rng = numpy.random.default_rng(0)
        n_pix = 1024
        while elapsed < seconds and rounds < 1000:
            pixels = numpy.sort(rng.choice(fw * fh, min(n_pix, fw * fh),
                                           replace=False)).astype(numpy.uint32)
            tracer.stats = cpu_module.OrStats()
            t0 = time.perf_counter()
            tracer.render_pixels(scene._scene, pixels, 1 + rounds, 1, want_m2=False)
            elapsed += time.perf_counter() - t0
            total_rays += tracer.stats.rays
            rounds += 1
            if rounds == 1:
                # scale the batch so that one round takes about a second
                per_pix = elapsed / len(pixels)
                n_pix = int(min(fw * fh, max(256, 1.0 / max(per_pix, 1e-9))))
        sample = (f"{rounds} rounds of random pixels of the {fw}x{fh} frame, 1 sample each "
                  f"x {wl.light_samples} light samples, {total_rays} closest-hit queries in "
                  f"{elapsed:.1f} s (BVH build {build_s:.1f} s, not timed)")
    return {"value": total_rays / elapsed / 1e6, "unit": "Mrays/s", "cores": os.cpu_count(),
            "kind": "reference" if kind == "reference" else "port", "sample": sample,
            "implementation": CPU_PATH_NOTE}


# What the CPU figures are: the reference's CPU renderer uses Embree 4 for its BVH and
# traversal (fresnel/cpu/Scene.cc:15-28), which is not installed; both CPU legs run the oracle's
# scalar binned-SAH BVH2 with the same shading arithmetic instead.
CPU_PATH_NOTE = ("CPU restatement of fresnel's Embree path: fresnel's TracerPath/TracerDirect "
                 "loops and shading over a scalar binned-SAH BVH2 (Embree 4 is not installed), "
                 "all host threads")


def config_of(wl, world):
    """The workload description both arms print."""
    if wl.preview:
        l2 = "scene arrays and BVH larger than L2 at this size; the image is written once per frame"
    else:
        l2 = ("inputs larger than L2 (path state of every sample in flight, plus the scene "
              "arrays and acceleration structure)")
    return {"workload": wl.desc.format(w=wl.w, h=wl.h, spp=wl.spp), "width": wl.w,
            "height": wl.h, "spp": wl.spp if not wl.preview else wl.aa_n * wl.aa_n,
            "light_samples": wl.light_samples, "parallelism": f"replicas{world}", "l2": l2}


def run_reference(args, wl):
    """The reference arm: fresnel's own Python package over the oracle compiled from fresnel's
    own fresnel/common headers (oracle/_ref), timed on this host's cores on bounded samples of
    the same frame.  Under torchrun only rank 0 works."""
    world, rank, _ = dist_init()
    if rank != 0:
        return 0
    from oracle import cpu_module
    kind = "reference" if os.path.exists(cpu_module.LIB_PATHS["reference"]) else "restated"
    dev = reference_device(kind)
    per_step = max(2.0, min(20.0, 60.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_baseline(wl, dev, per_step / 4, kind)
    vals = [cpu_baseline(wl, dev, per_step, kind) for _ in range(args.steps)]
    v = statistics.median(x["value"] for x in vals)
    base = dict(vals[0])
    base["value"] = v
    line = {
        "metric": METRIC if wl.key == "c2" else f"Mrays/s ({wl.key})",
        "value": v, "unit": "Mrays/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)", "config": config_of(wl, world), "cpu_baseline": base,
        "api": f"fresnel's own Python package ({dev.__class__.__module__}) on the "
               f"{'reference-header' if kind == 'reference' else 'restated'} CPU oracle",
        "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def host_arrays(scene):
    """(array, host copy) for every geometry array of the scene (written again each e2e step)."""
    import numpy
    out = []
    for g in scene.geometry:
        for name in ("position", "points", "radius", "orientation", "color"):
            try:
                a = getattr(g, name)
            except (AttributeError, RuntimeError):
                continue
            out.append((a, numpy.array(a[:], copy=True)))
    return out


def run_batch_bench(args, world, rank, barrier_max, barrier_sum, clock_index, emit=True):
    """Trajectory frame set (64 scenes of 1e4-5e5 spheres, 512^2-1024^2, 16 spp): the frames
    traced as one PathBatch (one CUDA graph launch) against 64 sequential plain Path.sample
    calls, and against fresnel's own form of Path.sample, one render call per sample
    (fresnel/tracer.py:250-260).  All three produce identical images (checked), so the
    comparison is at equal error.  Returns the JSON line (printed by rank 0 when ``emit``)."""
    import numpy

    import fresnel_b200 as fresnel
    from fresnel_b200 import workloads
    spp = args.spp or 16
    device = fresnel.Device(mode="gpu", n=1)
    dd = device._device
    frames = workloads.config4(device)
    for s, _, _ in frames:
        s._scene.build()
    # leaf size, primary tile shape and queue depth from the autotuner, on 2-spp probes of
    # the frame set itself; every form below runs with the chosen options
    from fresnel_b200 import autotune
    t0 = time.perf_counter()
    tuner = autotune.Tuner(device, probe_spp=2, repeats=2)
    tuned, probe_ms = tuner.tune([(s, w, h, 1) for s, w, h in frames])
    tune_s = time.perf_counter() - t0
    for s, _, _ in frames:
        s._scene.build()
    plain = [fresnel.tracer.Path(device, w=w, h=h) for _, w, h in frames]
    batched = [fresnel.tracer.Path(device, w=w, h=h) for _, w, h in frames]
    per_sample = [fresnel.tracer.Path(device, w=w, h=h) for _, w, h in frames]
    batch = fresnel.tracer.PathBatch(device)
    # every step renders each frame from the same seed in all three forms, so their images
    # must be identical
    seeds = [1000 * rank + f for f in range(len(frames))]

    def run_plain():
        for (s, _, _), t, seed in zip(frames, plain, seeds):
            t.seed = seed
            t.sample(s, samples=spp)

    def run_per_sample():
        # fresnel's Path.sample: reset, then one render (returning the output) per sample
        for (s, _, _), t, seed in zip(frames, per_sample, seeds):
            t.seed = seed
            t.reset()
            for _ in range(spp):
                t.render(s)

    def run_batch():
        for (s, _, _), t, seed in zip(frames, batched, seeds):
            t.seed = seed
            batch.add(t, s, samples=spp)
        batch.render()

    def timed(fn, tracers, steps):
        for t in tracers:
            t._tracer.resetStats()
        dd.synchronize()
        dd.timerStart()
        for _ in range(steps):
            fn()
        ms = dd.timerStop()
        sts = [t._tracer.getStats() for t in tracers]
        return ms, float(sum(x["rays"] for x in sts)), sts

    for _ in range(args.warmup):
        run_plain()
        run_batch()
    run_per_sample()
    ms_plain, rays_plain, _ = timed(run_plain, plain, args.steps)
    ms_per_sample, rays_per_sample, _ = timed(run_per_sample, per_sample, max(1, args.steps // 2))
    launches0 = batch.stats["kernel_launches"]
    box0, prim0 = batch.stats["box_tests"], batch.stats["prim_tests"]
    with ClockSampler(clock_index) as clk:
        ms_batch, rays_batch, bst = timed(run_batch, batched, args.steps)
    launches = batch.stats["kernel_launches"] - launches0
    # a batch counts its traversal work itself (the tracers count only their rays)
    box = float(batch.stats["box_tests"] - box0)
    prim = float(batch.stats["prim_tests"] - prim0)

    def maxdiff(xs, ys):
        return max(float(numpy.abs(numpy.asarray(a.linear_output[:]) -
                                   numpy.asarray(b.linear_output[:])).max())
                   for a, b in zip(xs, ys))
    diff = maxdiff(plain, batched)
    diff_per_sample = maxdiff(per_sample, batched)

    # end to end: every frame's arrays written from host memory (BVH rebuilt), traced, and its
    # sRGB image read back
    arrays = [host_arrays(s) for s, _, _ in frames]

    def e2e(fn, tracers):
        out_bytes = 0
        t0 = time.perf_counter()
        for arr in arrays:
            for a, host in arr:
                a[:] = host
        fn()
        for t in tracers:
            out_bytes += t.output[:].nbytes
        return (time.perf_counter() - t0) * 1e3, out_bytes

    e2e_plain = [e2e(run_plain, plain)[0] for _ in range(args.steps)]
    e2e_batch = []
    out_bytes = 0
    for _ in range(args.steps):
        ms, out_bytes = e2e(run_batch, batched)
        e2e_batch.append(ms)
    in_bytes = sum(h.nbytes for arr in arrays for _, h in arr)

    ms_plain = barrier_max(ms_plain)
    ms_batch = barrier_max(ms_batch)
    ms_per_sample = barrier_max(ms_per_sample)
    value = barrier_sum(rays_batch) / (ms_batch / 1e3) / 1e6
    value_plain = barrier_sum(rays_plain) / (ms_plain / 1e3) / 1e6
    value_per_sample = barrier_sum(rays_per_sample) / (ms_per_sample / 1e3) / 1e6
    e2e_b = barrier_max(statistics.mean(e2e_batch))
    e2e_p = barrier_max(statistics.mean(e2e_plain))
    rays_frame_set = rays_batch / args.steps
    hbm, peak_kind = peaks()
    # bytes of the structures walked (sphere grids: 52 + 8 per cell + 16 per sphere tested)
    grid = all(int(x.get("grid", 0)) for x in bst)
    bpr = (52.0 + (8.0 if grid else 32.0) * box / rays_batch + 16.0 * prim / rays_batch
           if rays_batch else None)
    achieved = rays_batch * bpr / (ms_batch / 1e3) / 1e9 if bpr else None
    line = {
        "metric": "Mrays/s (c4: 64-frame set, batched)", "value": value, "unit": "Mrays/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_batch / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": f"config4: 64 frames, 1e4-5e5 spheres at the 1M-sphere "
                               f"scene's density, 512^2/768^2/1024^2, {spp} spp, 1 light "
                               "sample; one PathBatch vs 64 sequential Path.sample calls",
                   "frames": len(frames), "spp": spp,
                   "autotune": {"options": tuned, "probe_ms": probe_ms,
                                "settings_measured": len(tuner.log), "seconds": tune_s},
                   "spheres": int(sum(len(s.geometry[0].position[:]) for s, _, _ in frames)),
                   "pixels": int(sum(w * h for _, w, h in frames)),
                   "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (64 scenes, 2.4 GB path state)"},
        "plain": {"value": value_plain, "ms_per_step": ms_plain / args.steps,
                  "e2e_ms_per_step": e2e_p},
        "plain_per_sample": {"value": value_per_sample,
                             "ms_per_step": ms_per_sample / max(1, args.steps // 2),
                             "form": "fresnel's Path.sample: one render call per sample"},
        "batched_over_plain": value / value_plain,
        "batched_over_plain_per_sample": value / value_per_sample,
        "e2e_batched_over_plain": e2e_p / e2e_b,
        "max_abs_image_difference": diff,
        "max_abs_image_difference_per_sample": diff_per_sample,
        "rays_per_frame_set": rays_frame_set,
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm if achieved else None, "traffic": None,
                     "peak_source": peak_kind, "kernel": "whole batch graph (all kernels)",
                     "bytes_per_ray": bpr,
                     "bytes_per_ray_basis": "sphere grids walked, engine counters"
                     if grid else "structures walked, engine counters"},
        "clocks": clk.summary(),
        "e2e": {"value": barrier_sum(rays_frame_set) / (e2e_b / 1e3) / 1e6,
                "unit": "Mrays/s", "h2d_bytes_per_step": int(in_bytes),
                "d2h_bytes_per_step": int(out_bytes), "ms_per_step": e2e_b},
        "batch_stats": batch.stats,
        "cpu_baseline": None,
    }
    if rank == 0 and emit:
        print(json.dumps(line))
    return line


def run_serving_bench(args, world, rank, barrier_max, barrier_sum, clock_index, emit=True,
                      rates=(10.0, 50.0, 100.0, 250.0, 500.0), window=4.0, per_sample=True):
    """Serving trace (config5): Poisson arrivals at 10-500 requests/s over 32 resident scenes of
    1e3-2e6 primitives (spheres and bonds), 256^2-1080p, 1-64 spp.  The continuous-batching
    server against the same requests served one at a time by plain Path.sample calls, and (with
    ``per_sample``) by fresnel's own form of Path.sample, one render call per sample
    (fresnel/tracer.py:250-260); all are real-time (a request exists only from its arrival on)
    and read each image back.  Every request's image is compared between the server and the
    plain run (identical by construction).  Returns the JSON line (printed by rank 0 when
    ``emit``); the headline figures are those of the highest rate."""
    import numpy

    import fresnel_b200 as fresnel
    from fresnel_b200 import serving, workloads
    device = fresnel.Device(mode="gpu", n=1)
    rates = list(rates)
    _, sizes = workloads.config5(rates[0], 1)
    t0 = time.perf_counter()
    scenes = {k: workloads.serving_scene(device, n, seed=4000 + k) for k, n in sizes.items()}
    for sc in scenes.values():
        sc._scene.build()
    device._device.synchronize()
    setup_s = time.perf_counter() - t0
    engine = serving.Engine(device)

    def factory(k):
        return scenes[k], workloads.serving_scene_bytes(sizes[k])

    # warm-up: kernels, graph capture, tracer pools
    warm, _ = workloads.config5(1000.0, 24)
    serving.serve_trace(serving.RenderServer(engine, factory), warm, realtime=False)
    serving.plain_trace(engine, lambda k: scenes[k], workloads.config5(1000.0, 24)[0],
                        realtime=False)

    results = []
    launches = 0
    top = None
    with ClockSampler(clock_index) as clk:
        for rate in rates:
            n = int(min(400, max(40, round(rate * window))))
            reqs, _ = workloads.config5(rate, n)
            srv = serving.RenderServer(engine, factory, hbm_budget=120e9)
            srv.reserve_tracers({res: 12 for res in workloads.SERVING_RESOLUTIONS})
            serving.serve_trace(srv, reqs)
            launches += int(srv.batch.stats["kernel_launches"])
            alone, _ = workloads.config5(rate, n)
            serving.plain_trace(engine, lambda k: scenes[k], alone)
            same = sum(int(numpy.array_equal(a.image, b.image)) for a, b in zip(reqs, alone))
            row = {"rate_per_s": rate, "requests": n, "served": serving.latency_summary(reqs),
                   "plain": serving.latency_summary(alone), "identical_images": same,
                   "steps": srv.steps,
                   "image_bytes": int(sum(r.image.nbytes for r in reqs))}
            row["served_over_plain_throughput"] = (row["served"]["mrays_per_s"] /
                                                   max(row["plain"]["mrays_per_s"], 1e-9))
            row["plain_over_served_p99"] = row["plain"]["p99_ms"] / row["served"]["p99_ms"]
            if per_sample:
                each, _ = workloads.config5(rate, n)
                serving.plain_trace(engine, lambda k: scenes[k], each, per_sample=True)
                row["plain_per_sample"] = serving.latency_summary(each)
                row["plain_per_sample"]["identical_images"] = sum(
                    int(numpy.array_equal(a.image, b.image)) for a, b in zip(reqs, each))
                row["served_over_plain_per_sample_throughput"] = (
                    row["served"]["mrays_per_s"] /
                    max(row["plain_per_sample"]["mrays_per_s"], 1e-9))
                row["plain_per_sample_over_served_p99"] = (
                    row["plain_per_sample"]["p99_ms"] / row["served"]["p99_ms"])
            results.append(row)
            top = row
    sv, pl = top["served"], top["plain"]
    line = {
        "metric": "serving (c5): Mrays/s and p50/p99 time-to-image, continuous batching vs "
                  "plain", "value": sv["mrays_per_s"], "unit": "Mrays/s",
        "n_gpus": world, "steps": len(rates), "warmup": 1,
        "ms_per_step": sv["span_s"] * 1e3 / sv["requests"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": "config5: Poisson arrivals, 32 resident scenes of 1e3-2e6 "
                               "primitives (80% spheres, 20% bonds), "
                               "256^2/640x480/1280x720/1920x1080, 1-64 spp, HBM budget "
                               "120 GB", "rates": rates, "window_s": window,
                   "scene_primitives": int(sum(sizes.values())),
                   "scene_setup_s": setup_s, "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (32 resident scenes)"},
        "p50_ms": sv["p50_ms"], "p99_ms": sv["p99_ms"],
        "plain": {"mrays_per_s": pl["mrays_per_s"], "p50_ms": pl["p50_ms"],
                  "p99_ms": pl["p99_ms"]},
        "rates": results,
        "gpu_launches": launches,
        "roofline": None,
        "clocks": clk.summary(),
        "e2e": {"value": sv["mrays_per_s"], "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(top["image_bytes"] / top["requests"]),
                "note": "the served path is end to end: requests in, sRGB images read back"},
        "cpu_baseline": None,
    }
    if "plain_per_sample" in top:
        pp = top["plain_per_sample"]
        line["plain_per_sample"] = {"mrays_per_s": pp["mrays_per_s"], "p50_ms": pp["p50_ms"],
                                    "p99_ms": pp["p99_ms"]}
    if rank == 0 and emit:
        print(json.dumps(line))
    return line


def main():
    args, wl = parse()
    world, rank, local = dist_init()
    if args.impl == "reference":
        return run_reference(args, wl)
    if world > 1:
        pin_gpu(local)
    import torch

    import fresnel_b200 as fresnel

    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(0)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    reps = Replicas(pg, "cuda")
    barrier_max, barrier_sum = reps.max, reps.sum

    clock_index = int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0] or 0)
    if wl.key in ("c4", "c5"):
        run = run_batch_bench if wl.key == "c4" else run_serving_bench
        run(args, world, rank, barrier_max, barrier_sum, clock_index)
        reps.close()
        return 0
    if wl.key == "tour":
        line = run_tour(fresnel)
        if rank == 0:
            print(json.dumps(line))
        reps.close()
        return 0

    device = fresnel.Device(mode="gpu", n=1)
    scene = wl.build(device)
    dd = device._device
    if wl.preview:
        tracer = fresnel.tracer.Preview(device, w=wl.w, h=wl.h, anti_alias=wl.aa_n > 1)

        def frame():
            tracer.render(scene)
    else:
        tracer = fresnel.tracer.Path(device, w=wl.w, h=wl.h)

        def frame():
            tracer.sample(scene, samples=wl.spp, light_samples=wl.light_samples)
    tracer.seed = 1000 * rank

    # ---- trace-only: BVH built and resident, K full frames ---------------------------------
    scene._scene.build()
    for _ in range(args.warmup):
        frame()
    tracer._tracer.resetStats()
    reps.barrier()
    torch.cuda.synchronize()
    dd.synchronize()
    with ClockSampler(int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0] or 0)) as clk:
        dd.timerStart()
        for _ in range(args.steps):
            frame()
        ms = dd.timerStop()
    torch.cuda.synchronize()
    reps.barrier()
    st = tracer._tracer.getStats()
    # Per-kernel device times from the same K frames rendered again with CUDA events around
    # every launch (the events cost about 2% of a frame, so the timed frames above run without).
    dd.setProfiling(True)
    tracer._tracer.resetStats()
    for _ in range(args.steps):
        frame()
    dd.synchronize()
    pst = tracer._tracer.getStats()
    dd.setProfiling(False)
    for key in ("primary_ms", "shade_ms", "extend_ms", "primary_launches", "shade_launches",
                "extend_launches"):
        st[key] = pst[key]
    rays = float(st["rays"])
    ms_max = barrier_max(ms)
    rays_all = barrier_sum(rays)
    value = rays_all / (ms_max / 1e3) / 1e6

    # roofline of the traversal kernel with the most device time
    hbm, peak_kind = peaks()
    if wl.preview:
        pv = ("k_preview_warp" if dd.getOption("preview_warp") and (wl.aa_n * wl.aa_n) % 32 == 0
              else "k_preview")
        kern = {pv: (rays, ms, args.steps)}
    else:
        primary_rays = float(wl.w * wl.h * wl.spp * args.steps)
        ext_rays = max(0.0, rays - primary_rays)
        # with fused shading (device option fuse_shade) the primary kernel also shades, and
        # without shade launches each bounce traces and shades in one kernel
        primary_name = "k_path_primary_shade" if dd.getOption("fuse_shade") else "k_path_primary"
        ext_name = "k_path_bounce" if st["shade_launches"] == 0 else "k_path_extend"
        if ext_name == "k_path_bounce" and dd.getOption("tail") >= 0:
            # the fused bounces of a wavefront: bounce launches, then one tail launch that
            # follows every remaining path (timed together as the extension kernels)
            ext_name = "k_path_bounce+k_path_tail"
        kern = {primary_name: (primary_rays, st["primary_ms"], st["primary_launches"]),
                ext_name: (ext_rays, st["extend_ms"], st["extend_launches"])}
    dom = max(kern, key=lambda k: kern[k][1])
    dom_rays, dom_ms, launches = kern[dom]
    # Algorithmic bytes per ray of the structure this run traversed, from the engine's own
    # counters over the frame: 24 B of ray in, 16 B of hit out, 12 B of colour at the hit, then
    # per BVH box test 32 B or per grid cell 8 B of reference range, and 16 B per sphere tested
    # (a grid over parts: 36 B per reference, its 32 B record and 4 B geometry index).
    grid_kind = int(st.get("grid", 0))
    grid = grid_kind != 0
    per_box = 8.0 if grid else 32.0
    per_prim = 36.0 if grid_kind == 2 else 16.0
    run_bytes = (52.0 + per_box * st["box_tests"] / rays + per_prim * st["prim_tests"] / rays
                 if rays > 0 else None)
    # The roofline's bytes: for a grid, those of the grid walked (the oracle's frozen cells and
    # spheres per ray when the workload has them, else this run's counters); for a BVH, the
    # reference BVH's fixed box and primitive tests per ray (wl.bytes_per_ray).  The
    # reference-BVH figure of a grid run is kept beside it: it counts the work a BVH would do,
    # not what the kernel read.
    frozen = wl.grid_bytes_per_ray if grid_kind == 1 else wl.parts_grid_bytes_per_ray
    if grid:
        bpr = frozen if frozen and (wl.w, wl.h) == wl.full_size else run_bytes
    else:
        bpr = wl.bytes_per_ray
    achieved = (dom_rays * bpr) / (dom_ms / 1e3) / 1e9 if dom_ms > 0 and bpr else None
    achieved_ref = (dom_rays * wl.bytes_per_ray) / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else None
    achieved_run = ((dom_rays * run_bytes) / (dom_ms / 1e3) / 1e9
                    if dom_ms > 0 and run_bytes else None)
    # DRAM bytes per launch: this kernel's DRAM bytes per ray from an ncu capture
    # (dram__bytes_read.sum + dram__bytes_write.sum over every launch of one frame, divided by
    # that frame's rays) times the mean rays per launch here.
    traffic = None
    prof = os.path.join(REPO, "profiles", "traversal_traffic.json")
    if wl.key == "c2" and os.path.exists(prof) and launches:
        try:
            with open(prof) as f:
                per_ray = json.load(f).get(dom, {}).get("dram_bytes_per_ray")
            if per_ray is not None:
                traffic = per_ray * dom_rays / launches
        except Exception:
            traffic = None

    # Step-level cross-check: every ray of the timed frames at the bytes of the structure walked,
    # plus 36 B per pixel sample (accumulate read + write, sRGB write), over the frames' time.
    pix_samples = float(wl.w * wl.h * (wl.aa_n * wl.aa_n if wl.preview else wl.spp * wl.light_samples)
                        * args.steps)
    step_bps = ((rays * run_bytes + 36.0 * pix_samples) / (ms / 1e3)
                if run_bytes and ms > 0 else None)

    # ---- end to end through the public API with host buffers ----------------------------------
    e2e_ms = []
    out = None
    rays_per_frame = rays / args.steps
    arrays = host_arrays(scene)
    builds = 0
    for step in range(0 if args.trace_only else args.warmup + args.steps):
        if step == args.warmup:
            tracer._tracer.resetStats()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for a, host in arrays:
            a[:] = host
        frame()
        out = tracer.output[:]
        dt = (time.perf_counter() - t0) * 1e3
        if step >= args.warmup:
            e2e_ms.append(dt)
    e2e = None
    if e2e_ms:
        est = tracer._tracer.getStats()
        builds = int(est["bvh_builds"]) + int(est.get("grid_builds", 0))
        e2e_step = barrier_max(statistics.mean(e2e_ms))
        e2e_value = barrier_sum(rays_per_frame) / (e2e_step / 1e3) / 1e6
        assert out is not None and out.shape == (wl.h, wl.w, 4)
        e2e = {"value": e2e_value, "unit": "Mrays/s",
               "h2d_bytes_per_step": int(sum(h.nbytes for _, h in arrays)),
               "d2h_bytes_per_step": int(out.nbytes), "ms_per_step": e2e_step,
               "builds": builds}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline and not args.trace_only:
        try:
            from oracle import cpu_module
            cpu = cpu_baseline(wl, cpu_module.make_device("restated"), args.cpu_seconds,
                               "restated")
        except Exception as e:  # the baseline must not hide the GPU result
            cpu = {"value": None, "unit": "Mrays/s", "error": str(e)[:200]}

    if rank == 0:
        cfg = config_of(wl, world)
        line = {
            "metric": METRIC if wl.key == "c2" else f"Mrays/s ({wl.key})",
            "value": value, "unit": "Mrays/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": cfg,
            "accel": {0: "bvh", 1: "sphere grid", 2: "grid over parts"}[grid_kind],
            "rays_per_frame": rays_per_frame,
            "gpu_launches": int(st["kernel_launches"]),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                         "peak_source": peak_kind, "kernel": dom,
                         "rays": dom_rays, "kernel_ms": dom_ms, "launches": launches,
                         "bytes_per_ray": bpr,
                         "bytes_per_ray_basis": (("sphere grid walked: 52 + 8 per cell + 16 "
                                                  "per sphere tested, oracle counts" if
                                                  bpr != run_bytes else
                                                  "sphere grid walked: 52 + 8 per cell + 16 "
                                                  "per sphere tested, engine counters")
                                                 if grid_kind == 1 else
                                                 ("grid over parts walked: 52 + 8 per cell + 36 "
                                                  "per reference, oracle counts" if
                                                  bpr != run_bytes else
                                                  "grid over parts walked: 52 + 8 per cell + 36 "
                                                  "per reference, engine counters")
                                                 if grid else
                                                 "reference BVH: 52 + 32 A + S P, oracle counts"),
                         "accel": "grid" if grid else "bvh",
                         "bytes_per_ray_run": run_bytes, "achieved_run": achieved_run,
                         "frac_run": (achieved_run / hbm) if achieved_run else None,
                         "bytes_per_ray_ref_bvh": wl.bytes_per_ray,
                         "frac_ref_bvh_bytes": (achieved_ref / hbm) if achieved_ref else None,
                         "step_bytes_per_s": step_bps,
                         "step_frac": step_bps / 1e9 / hbm if step_bps else None},
            "clocks": clk.summary(),
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        if not wl.preview:
            line["mpaths_per_s"] = (wl.w * wl.h * wl.spp * wl.light_samples * args.steps * world
                                    / (ms_max / 1e3) / 1e6)
            line["kernels"] = {"primary_ms": st["primary_ms"], "shade_ms": st["shade_ms"],
                               "extend_ms": st["extend_ms"],
                               "primary_launches": st["primary_launches"],
                               "shade_launches": st["shade_launches"],
                               "extend_launches": st["extend_launches"],
                               "primary_rays": primary_rays, "extension_rays": ext_rays,
                               "primary_kernel": primary_name, "extension_kernel": ext_name}
    extras = None
    if wl.key == "c2" and not args.trace_only and not args.no_extras:
        extras = run_extras(args, wl, fresnel, device, world, rank, barrier_max, barrier_sum,
                            clock_index)
    if rank == 0:
        if extras:
            line["also"] = extras
        print(json.dumps(line))
    reps.close()
    return 0


def run_tour(fresnel):
    """One pass over every kernel family on cases of a few GB at most (the input of a
    per-kernel profiler capture): the LBVH build of the 1M-sphere scene, its sphere-grid build,
    Preview of it at 1920x1080 with 8x8 anti-aliasing through the grid, a 480x270 16-spp path
    render (the fold), the histogram of a 1080p image, a batch of 4 sphere-grid frames and a
    batch of a mixed scene.  Prints the device time of each stage."""
    from fresnel_b200 import workloads
    dev = fresnel.Device(mode="gpu", n=1)
    dd = dev._device
    dd.setOption("path_slots", 4 << 20)
    out = {}

    def stage(name, fn):
        dd.synchronize()
        dd.timerStart()
        fn()
        out[name + "_ms"] = dd.timerStop()
    dd.setOption("accel", 0)
    s_bvh = workloads.config2(dev)
    stage("lbvh_build_1m", s_bvh._scene.build)
    dd.setOption("accel", 1)
    s_grid = workloads.config2(dev)
    stage("grid_build_1m", s_grid._scene.build)
    p = fresnel.tracer.Preview(dev, w=1920, h=1080, anti_alias=True)
    stage("preview_1080p_aa8", lambda: p.render(s_grid))
    t = fresnel.tracer.Path(dev, w=480, h=270)
    stage("path_480x270_16spp", lambda: t.sample(s_grid, samples=16))
    t2 = fresnel.tracer.Path(dev, w=1920, h=1080)
    t2.sample(s_grid, samples=1)
    stage("histogram_1080p", t2.histogram)
    dd.setOption("accel", 2)
    frames = workloads.config4(dev, n_frames=4, seed=3)
    b = fresnel.tracer.PathBatch(dev)
    tracers = [fresnel.tracer.Path(dev, w=w // 2, h=h // 2) for _, w, h in frames]

    def batch_frames():
        for (s, _, _), tr in zip(frames, tracers):
            b.add(tr, s, samples=4)
        b.render()
    stage("batch_4_frames", batch_frames)
    mix = workloads.config3(dev, scale=0.05)
    b2 = fresnel.tracer.PathBatch(dev)
    tr = fresnel.tracer.Path(dev, w=320, h=180)

    def batch_mixed():
        b2.add(tr, mix, samples=4)
        b2.render()
    stage("batch_mixed", batch_mixed)
    return {"metric": "kernel tour: device ms per stage", "stages": out}


def bvh_frames(args, wl, fresnel, device, rank, barrier_max, barrier_sum, steps=4, warmup=2):
    """The headline frame traced through the LBVH (device option accel = 0) instead of the
    sphere grid: Mrays/s over ``steps`` frames, the per-kernel device times of the same frames
    rendered again, and the dominant kernel's fraction on the reference BVH's algorithmic bytes
    per ray (the structure this run walks is a BVH too)."""
    dd = device._device
    old = dd.getOption("accel")
    dd.setOption("accel", 0)
    try:
        scene = wl.build(device)
        tracer = fresnel.tracer.Path(device, w=wl.w, h=wl.h)
        tracer.seed = 1000 * rank + 500
        scene._scene.build()

        def frame():
            tracer.sample(scene, samples=wl.spp, light_samples=wl.light_samples)
        for _ in range(warmup):
            frame()
        tracer._tracer.resetStats()
        dd.synchronize()
        dd.timerStart()
        for _ in range(steps):
            frame()
        ms = dd.timerStop()
        st = tracer._tracer.getStats()
        dd.setProfiling(True)
        tracer._tracer.resetStats()
        for _ in range(steps):
            frame()
        dd.synchronize()
        pst = tracer._tracer.getStats()
        dd.setProfiling(False)
        assert not st.get("grid", 0), "the LBVH frame was traced through a grid"
    finally:
        dd.setOption("accel", old)
    rays = float(st["rays"])
    ms_max = barrier_max(ms)
    value = barrier_sum(rays) / (ms_max / 1e3) / 1e6
    primary_rays = float(wl.w * wl.h * wl.spp * steps)
    kern = {"primary": (primary_rays, pst["primary_ms"], pst["primary_launches"]),
            "extension": (max(0.0, rays - primary_rays), pst["extend_ms"],
                          pst["extend_launches"]),
            "shade": (0.0, pst["shade_ms"], pst["shade_launches"])}
    dom = max(("primary", "extension"), key=lambda k: kern[k][1])
    dom_rays, dom_ms, _ = kern[dom]
    hbm, peak_kind = peaks()
    achieved = dom_rays * wl.bytes_per_ray / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else None
    names = {"primary": "k_path_primary_shade" if dd.getOption("fuse_shade") else
             "k_path_primary", "extension": "k_path_extend" if pst["shade_launches"] else
             "k_path_bounce", "shade": "k_path_shade"}
    return {"workload": wl.desc.format(w=wl.w, h=wl.h, spp=wl.spp) + ", traced through the "
                        "LBVH (accel = 0)",
            "value": value, "unit": "Mrays/s", "ms_per_step": ms_max / steps, "steps": steps,
            "warmup": warmup, "rays_per_frame": rays / steps,
            "kernels_ms_per_frame": {names[k]: v[1] / steps for k, v in kern.items()},
            "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved,
                         "peak": hbm, "peak_source": peak_kind, "unit": "GB/s",
                         "frac": achieved / hbm if achieved else None,
                         "bytes_per_ray": wl.bytes_per_ray,
                         "bytes_per_ray_basis": "reference BVH: 52 + 32 A + S P, oracle counts",
                         "box_tests_per_ray_run": float(st["box_tests"]) / rays,
                         "prim_tests_per_ray_run": float(st["prim_tests"]) / rays}}


def run_extras(args, wl, fresnel, device, world, rank, barrier_max, barrier_sum, clock_index):
    """Further measured configurations reported under "also" by the default run, so that one
    timed run covers them: the headline frame through the LBVH, the 64-frame batched set
    (config4) against plain and per-sample calls, and serving (config5) at 100 requests/s with
    p50/p99 against plain and per-sample serving.  A failure is reported, not raised."""
    out = {}
    small = argparse.Namespace(**vars(args))
    small.steps, small.warmup, small.spp = 2, 1, None
    for key, fn in (
            ("c2_bvh", lambda: bvh_frames(args, wl, fresnel, device, rank, barrier_max,
                                          barrier_sum)),
            ("c4_batched", lambda: run_batch_bench(small, world, rank, barrier_max, barrier_sum,
                                                   clock_index, emit=False)),
            ("c5_serving", lambda: run_serving_bench(small, world, rank, barrier_max,
                                                     barrier_sum, clock_index, emit=False,
                                                     rates=(100.0,), window=3.0))):
        t0 = time.perf_counter()
        try:
            out[key] = fn()
        except Exception as e:  # an extra must not hide the headline result
            out[key] = {"error": f"{type(e).__name__}: {str(e)[:300]}"}
        out[key]["wall_s"] = time.perf_counter() - t0
    return out


if __name__ == "__main__":
    sys.exit(main())
