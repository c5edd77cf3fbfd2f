"""Benchmark: Mrays/s of the path tracer on the 1M-sphere 1080p scene.

Workload (one step = one full frame): 1,000,000 spheres (r = 0.5, positions uniform in a cube
of side 140, per-particle colours), lightbox lighting, perspective camera fit to the scene,
1920x1080, 256 samples per pixel, 1 light sample -- ``Tracer.Path.sample(scene, 256)``.
Synthetic, seeded inputs stand in for the scene (the reference publishes no benchmark data).

Prints one JSON line:
  value      trace-only throughput: closest-hit queries per second over the K timed frames,
             scene and BVH resident in HBM, device time from CUDA events on the engine's stream
             (max over ranks); every rank renders its own frame (weak scaling, no collective)
  e2e        the same metric through the public API with host buffers: each step uploads the
             sphere arrays from host memory, rebuilds the BVH, renders 256 spp and reads the
             sRGB image back
  roofline   the dominant kernel (BVH traversal of extension rays): algorithmic bytes per ray
             (measured A/P costs of the oracle BVH) x rays / its device time
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

# Per-ray algorithmic bytes of the traversal kernel: ray in (24) + hit out (16) + 32 B per
# box test (A per ray) + 16 B per sphere test (P per ray) + 12 B colour at the closest hit.
# A and P are the oracle BVH's (binned SAH, leaves <= 4) mean costs per extension ray on this
# scene and camera, measured by oracle/measure_ray_costs.py and frozen here.
RAY_BOX_TESTS = 37.74
RAY_PRIM_TESTS = 1.42
BYTES_PER_RAY = 24 + 16 + 32 * RAY_BOX_TESTS + 16 * RAY_PRIM_TESTS + 12

WIDTH, HEIGHT, SPP, LIGHT_SAMPLES = 1920, 1080, 256, 1
N_SPHERES, BOX = 1_000_000, 140.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="engine", choices=["engine", "reference"])
    p.add_argument("--spp", type=int, default=SPP, help="samples per pixel of one frame")
    p.add_argument("--width", type=int, default=WIDTH,
                   help="image width (smaller frames only for profiler captures)")
    p.add_argument("--height", type=int, default=HEIGHT)
    p.add_argument("--cpu-seconds", type=float, default=15.0,
                   help="target duration of the CPU baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--trace-only", action="store_true",
                   help="skip the end-to-end leg and the CPU baseline (profiler captures)")
    p.add_argument("--profile-kernels", action="store_true", default=True)
    return p.parse_args()


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


def build_scene(fresnel, device):
    from fresnel_b200 import workloads
    return workloads.config2(device, n=N_SPHERES, box=BOX)


def cpu_baseline(kind, seconds, world_rank=0):
    """Time the CPU oracle on a bounded sample of the frame: random pixels, 1 sample each."""
    import numpy

    import fresnel_b200 as fresnel  # noqa: F401
    from oracle import cpu_module
    dev = cpu_module.make_device(kind)
    scene = build_scene(None, dev)
    t0 = time.perf_counter()
    scene._scene.handle()  # BVH build, not timed
    build_s = time.perf_counter() - t0
    tracer = dev.module.TracerPath(dev._device, WIDTH, HEIGHT, LIGHT_SAMPLES)
    tracer.setSeed(2)
    rng = numpy.random.default_rng(0)
    n_pix = 4096
    total_rays = 0
    elapsed = 0.0
    rounds = 0
    while elapsed < seconds and rounds < 1000:
        pixels = numpy.sort(rng.choice(WIDTH * HEIGHT, n_pix, replace=False)).astype(numpy.uint32)
        tracer.stats = cpu_module.OrStats()
        t0 = time.perf_counter()
        tracer.render_pixels(scene._scene, pixels, 1 + rounds, 1, want_m2=False)
        elapsed += time.perf_counter() - t0
        total_rays += tracer.stats.rays
        rounds += 1
        if rounds == 1:
            # scale the batch so that one round takes about a second
            per_pix = elapsed / n_pix
            n_pix = int(min(WIDTH * HEIGHT, max(1024, 1.0 / max(per_pix, 1e-9))))
    return {"value": total_rays / elapsed / 1e6, "unit": "Mrays/s", "cores": os.cpu_count(),
            "kind": "reference" if kind == "reference" else "port",
            "sample": f"{rounds} rounds of random pixels of the 1920x1080 frame, 1 sample each, "
                      f"{total_rays} closest-hit queries in {elapsed:.1f} s "
                      f"(BVH build {build_s:.1f} s, not timed)"}


def run_reference(args):
    world, rank, _ = dist_init()
    if rank != 0:
        return 0
    from oracle import cpu_module
    kind = "reference" if os.path.exists(cpu_module.LIB_PATHS["reference"]) else "restated"
    per_step = max(2.0, min(20.0, 60.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_baseline(kind, per_step / 4)
    vals = [cpu_baseline(kind, per_step) for _ in range(args.steps)]
    v = statistics.median(x["value"] for x in vals)
    base = dict(vals[0])
    base["value"] = v
    line = {
        "metric": "Mrays/s on 1M-sphere 1080p path trace", "value": v, "unit": "Mrays/s",
        "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded uniform spheres)",
        "config": {"workload": "config2: 1M spheres r=0.5, box 140, 1920x1080, 256 spp, "
                               "1 light sample, lightbox", "inputs": "host memory"},
        "cpu_baseline": base,
        "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    world, rank, local = dist_init()
    if args.impl == "reference":
        return run_reference(args)
    if world > 1:
        pin_gpu(local)
    import numpy
    import torch

    import fresnel_b200 as fresnel
    from fresnel_b200 import workloads  # noqa: F401

    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(0)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist

    def barrier_max(x):
        if pg is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    def barrier_sum(x):
        if pg is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.SUM)
        return float(t.item())

    device = fresnel.Device(mode="gpu", n=1)
    scene = build_scene(fresnel, device)
    tracer = fresnel.tracer.Path(device, w=args.width, h=args.height)
    tracer.seed = 1000 * rank
    dd = device._device

    # ---- trace-only: BVH built and resident, K full frames ---------------------------------
    scene._scene.build()
    for _ in range(args.warmup):
        tracer.sample(scene, samples=args.spp, light_samples=LIGHT_SAMPLES)
    dd.setProfiling(bool(args.profile_kernels))
    tracer._tracer.resetStats()
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    dd.synchronize()
    with ClockSampler(int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0] or 0)) as clk:
        dd.timerStart()
        for _ in range(args.steps):
            tracer.sample(scene, samples=args.spp, light_samples=LIGHT_SAMPLES)
        ms = dd.timerStop()
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    st = tracer._tracer.getStats()
    dd.setProfiling(False)
    rays = float(st["rays"])
    ms_max = barrier_max(ms)
    rays_all = barrier_sum(rays)
    value = rays_all / (ms_max / 1e3) / 1e6

    # roofline of the dominant traversal kernel (primary rays or extension rays)
    hbm, peak_kind = peaks()
    primary_rays = float(args.width * args.height * args.spp * args.steps)
    ext_rays = max(0.0, rays - primary_rays)
    kern = {"k_path_primary": (primary_rays, st["primary_ms"]),
            "k_path_extend": (ext_rays, st["extend_ms"])}
    dom = max(kern, key=lambda k: kern[k][1])
    dom_rays, dom_ms = kern[dom]
    achieved = (dom_rays * BYTES_PER_RAY) / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else None
    # DRAM bytes per launch: the per-ray DRAM traffic of this kernel from an ncu capture
    # (dram__bytes_read.sum + dram__bytes_write.sum over every launch of one frame, divided by
    # that frame's rays) times the mean rays per launch here.
    traffic = None
    prof = os.path.join(REPO, "profiles", "traversal_traffic.json")
    launches = st["primary_launches"] if dom == "k_path_primary" else st["extend_launches"]
    if os.path.exists(prof) and launches:
        try:
            with open(prof) as f:
                per_ray = json.load(f).get(dom, {}).get("dram_bytes_per_ray")
            if per_ray is not None:
                traffic = per_ray * dom_rays / launches
        except Exception:
            traffic = None

    # ---- end to end through the public API with host buffers ----------------------------------
    e2e_ms = []
    out = None
    rays_per_frame = rays / args.steps
    rng = numpy.random.default_rng(1)
    h_pos = rng.uniform(-BOX / 2, BOX / 2, (N_SPHERES, 3)).astype(numpy.float32)
    h_col = rng.uniform(0, 1, (N_SPHERES, 3)).astype(numpy.float32)
    h_rad = numpy.full(N_SPHERES, 0.5, numpy.float32)
    geom = scene.geometry[0]
    builds = 0
    for step in range(0 if args.trace_only else args.warmup + args.steps):
        if step == args.warmup:
            tracer._tracer.resetStats()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        geom.position[:] = h_pos
        geom.radius[:] = h_rad
        geom.color[:] = h_col
        tracer.sample(scene, samples=args.spp, light_samples=LIGHT_SAMPLES)
        out = tracer.output[:]
        dt = (time.perf_counter() - t0) * 1e3
        if step >= args.warmup:
            e2e_ms.append(dt)
    e2e = None
    if e2e_ms:
        builds = int(tracer._tracer.getStats()["bvh_builds"])
        e2e_step = barrier_max(statistics.mean(e2e_ms))
        e2e_value = barrier_sum(rays_per_frame) / (e2e_step / 1e3) / 1e6
        assert out is not None and out.shape == (args.height, args.width, 4)
        e2e = {"value": e2e_value, "unit": "Mrays/s",
               "h2d_bytes_per_step": int(h_pos.nbytes + h_col.nbytes + h_rad.nbytes),
               "d2h_bytes_per_step": int(out.nbytes), "ms_per_step": e2e_step,
               "bvh_builds": builds}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline and not args.trace_only:
        try:
            cpu = cpu_baseline("restated", args.cpu_seconds)
        except Exception as e:  # the baseline must not hide the GPU result
            cpu = {"value": None, "unit": "Mrays/s", "error": str(e)[:200]}

    if rank == 0:
        line = {
            "metric": "Mrays/s on 1M-sphere 1080p path trace", "value": value, "unit": "Mrays/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uniform spheres)",
            "config": {"workload": f"config2: 1M spheres r=0.5, box 140, {args.width}x{args.height}, "
                                   f"{args.spp} spp, 1 light sample, lightbox",
                       "spheres": N_SPHERES, "width": args.width, "height": args.height, "spp": args.spp,
                       "light_samples": LIGHT_SAMPLES,
                       "l2": "inputs larger than L2 (200 MB path state + 115 MB scene)",
                       "parallelism": f"replicas{world}"},
            "rays_per_frame": rays_per_frame,
            "mpaths_per_s": args.width * args.height * args.spp * args.steps * world / (ms_max / 1e3) / 1e6,
            "gpu_launches": int(st["kernel_launches"]),
            "kernels": {"primary_ms": st["primary_ms"], "shade_ms": st["shade_ms"],
                        "extend_ms": st["extend_ms"], "primary_launches": st["primary_launches"],
                        "shade_launches": st["shade_launches"],
                        "extend_launches": st["extend_launches"],
                        "primary_rays": primary_rays, "extension_rays": ext_rays},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                         "peak_source": peak_kind, "kernel": dom,
                         "rays": dom_rays, "kernel_ms": dom_ms, "launches": launches,
                         "bytes_per_ray": BYTES_PER_RAY},
            "clocks": clk.summary(),
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
