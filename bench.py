"""Benchmark of bulbit-b200 on one node.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl bulbit_b200|reference]

Workload (one "step"): the ray-throughput microbenchmark — a 1,048,576-triangle
soup (centroids U[-1,1]^3, vertices centroid + N(0, 0.01^2)), 16,777,216
closest-hit rays and 16,777,216 any-hit rays (t_max = 0.5 x distance to the
target) from the sphere of radius 3 toward U[-1,1]^3; seeded synthetic data.
value = (closest + any-hit rays traced by all ranks) / max-over-ranks device
time, in Mrays/s. The path-tracing workload (Cornell box with a displaced
gold icosphere, 1024x1024, 64 spp) is reported beside it as paths/s and
Mrays/s, and neural-guided against plain path tracing as the ratio of their
relMSE at equal device time (the same scene at 256x256 against a 16384-spp
plain render), and the batch of 16 uneven Cornell-box scenes (per-scene
Mrays/s, the batch against the scenes rendered one by one, guided against
plain relMSE inside the batch).

Each rank is an independent replica (the path does not shard across GPUs);
ranks only meet at barriers and the max-reduction of their timings.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_TRIS = 1 << 20
N_RAYS = 1 << 24
WORKLOAD = ("ray-throughput microbenchmark: 1,048,576-triangle soup (SAH BVH), "
            "16,777,216 closest-hit + 16,777,216 any-hit rays per step")
METRIC = "Mrays/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """SM clock and clock-event (throttle) reason samples while a timed
    region runs: an NVML thread every 10 ms, or nvidia-smi where NVML cannot
    be loaded. The GPU is found by its PCI bus id, so a remapping
    CUDA_VISIBLE_DEVICES cannot point the samples at another GPU. start()
    returns once the first sample is in, so even a short region is covered."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, cuda_index, period_s=0.01):
        self.period = period_s
        self.bus_id = None
        try:
            import torch
            p = torch.cuda.get_device_properties(cuda_index)
            self.bus_id = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        except Exception:  # no CUDA device visible: sample by index
            pass
        self.cuda_index = cuda_index
        self.thread = self.proc = self.path = None
        self.samples = []  # (sm_mhz, sm_max_mhz, set of active reason names)

    def _start_nvml(self):
        import threading
        import pynvml as nv
        nv.nvmlInit()
        h = (nv.nvmlDeviceGetHandleByPciBusId(self.bus_id) if self.bus_id
             else nv.nvmlDeviceGetHandleByIndex(self.cuda_index))
        max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        self.done, first = threading.Event(), threading.Event()

        def run():
            try:
                while True:
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((float(sm), float(max_mhz), {n for n, b in bits.items() if r & b}))
                    first.set()
                    if self.done.wait(self.period):
                        break
            finally:
                first.set()
                nv.nvmlShutdown()

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()
        first.wait(5.0)

    def _start_smi(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        target = self.bus_id if self.bus_id else str(self.cuda_index)
        self.proc = subprocess.Popen(
            ["nvidia-smi", "-i", target, f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
             "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 5.0 and self.proc.poll() is None and os.path.getsize(self.path) == 0:
            time.sleep(0.01)

    def start(self):
        self.samples = []
        try:
            self._start_nvml()
            return
        except Exception:  # no NVML library or no such device: fall back
            self.thread = None
        try:
            self._start_smi()
        except OSError:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.done.set()
            self.thread.join(5.0)
            source = "nvml"
        elif self.proc is not None:
            self.proc.terminate()
            self.proc.wait()
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) < 9:
                        continue
                    try:
                        sm, mx = float(parts[1]), float(parts[2])
                    except ValueError:
                        continue
                    self.samples.append((sm, mx, {n for n, v in zip(self.NAMES, parts[5:9])
                                                  if v.lower().startswith("active")}))
            os.unlink(self.path)
            source = "nvidia-smi"
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"], "samples": 0}
        sm = [s[0] for s in self.samples]
        reasons = set().union(*(s[2] for s in self.samples)) if self.samples else set()
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(s[1] for s in self.samples) if sm else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": source}


# ------------------------------------------------------------------ profiles

def profile_values(name):
    """Machine-readable figures of a committed ncu summary (profiles/<name>):
    every line 'key: <number> ...' (the first word after the colon)."""
    p = os.path.join(ROOT, "profiles", name)
    out = {}
    if not os.path.exists(p):
        return out
    with open(p) as f:
        for line in f:
            line = line.strip()
            if ":" not in line or line.startswith(("|", "#", "`", "(")):
                continue
            key, rest = line.split(":", 1)
            key = key.strip()
            if not key or not all(c.islower() or c.isdigit() or c == "_" for c in key) or not rest.split():
                continue
            try:
                out[key] = float(rest.split()[0])
            except ValueError:
                pass
    return out


def profile_traffic(name):
    """DRAM bytes per launch from a committed ncu summary (profiles/<name>),
    the line 'dram_bytes_per_launch: <int>'."""
    return profile_values(name).get("dram_bytes_per_launch")


# ------------------------------------------------------------------ reference arm

def max_over_ranks(values, device="cpu"):
    """Element-wise maximum of each rank's values (timings) over all ranks;
    every rank calls it, in the same order. Without a process group, the
    values themselves."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def whole_job_rate(units_per_rank, world, max_ms):
    """Units per second of the whole job: every rank's units over the slowest
    rank's time."""
    return world * units_per_rank / (max_ms / 1e3)


REF_WINDOW = 1 << 20


def reference_ray_rate(rs, closest, anyq, warmup, steps, window=REF_WINDOW):
    """The reference's BVH::Intersect + IntersectAny (oracle/_ref, ParallelFor
    over all host threads) on windows of the ray set: each step traces the
    next `window` closest-hit and `window` any-hit rays, sliding through the
    whole set; warm-up steps first (thread pool and first-touch costs).
    Returns (Mrays/s, seconds per step). Both CPU legs use this."""
    n = closest.shape[0]

    def step(k):
        off = (k * window) % n
        return rs.intersect(closest[off:off + window])[2] + rs.intersect_any(anyq[off:off + window])[1]

    for w in range(warmup):
        step(w)
    secs = sum(step(warmup + k) for k in range(steps))
    return 2 * window * steps / secs / 1e6, secs / steps


def run_reference(args, rank):
    """The reference's own CPU BVH (oracle/_ref, compiled from its sources)
    on the same workload: each step traces a bounded sample of the rays on all
    host threads."""
    if rank != 0:
        return
    from bulbit_b200 import scenes
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libbulbit_ref.so not built"}))
        return
    cores = ref.init(0)
    scene = scenes.triangle_soup(N_TRIS, seed=1)
    closest, anyq = scenes.soup_rays(N_RAYS, seed=2)
    rs = ref.RefScene(scene)
    value, step_s = reference_ray_rate(rs, closest, anyq, args.warmup, args.steps)
    desc = (f"{REF_WINDOW} closest-hit + {REF_WINDOW} any-hit rays of the 16,777,216-ray set per step (windows "
            f"sliding through the set), {cores} threads, BVH build {rs.build_seconds:.2f} s excluded")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * step_s,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample_rays_per_step": 2 * REF_WINDOW},
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": cores, "kind": "reference", "sample": desc},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def cpu_baseline(scene, closest, anyq):
    from oracle import ref
    if not ref.available():
        return None
    cores = ref.init(0)
    rs = ref.RefScene(scene)
    # As many steps as the reference arm's default run, so that both legs
    # measure the host at its sustained all-core clock (a short burst runs
    # faster on turbo).
    warmup, steps = 5, 20
    value, _ = reference_ray_rate(rs, closest, anyq, warmup, steps)
    return {"value": value, "unit": "Mrays/s", "cores": cores, "kind": "reference",
            "sample": f"{steps} steps of {REF_WINDOW} closest-hit + {REF_WINDOW} any-hit rays of the workload's ray "
                      f"set after {warmup} warm-up step, {cores} threads (reference BVH::Intersect/IntersectAny "
                      f"via ParallelFor, the same method as --impl reference; BVH build {rs.build_seconds:.2f} s "
                      f"excluded)"}


# ------------------------------------------------------------------ GPU arm

def run_e2e(args, acc, closest, anyq, barrier):
    """Closest + any-hit through the C ABI with pinned host buffers: the
    host->device copy of the rays and the device->host copy of the results
    happen inside each step. Each step submits the closest-hit batch and the
    any-hit batch (bbg_intersect_submit / bbg_intersect_any_submit with
    BBG_MEM_HOST) and waits for both (bbg_accel_synchronize), so the any-hit
    rays' upload overlaps the closest-hit traversal; the same steps through
    the synchronous calls (bbg_intersect, bbg_intersect_any) are timed
    beside it. Returns (steps, submitted seconds, synchronous seconds)."""
    import torch
    n = closest.shape[0]
    pin_c = torch.from_numpy(closest).pin_memory()
    pin_a = torch.from_numpy(anyq).pin_memory()
    pin_h = torch.empty((n, 4), dtype=torch.float32).pin_memory()
    pin_o = torch.empty(n, dtype=torch.uint8).pin_memory()
    steps = max(1, min(args.steps, 5))

    def submitted():
        acc.submit_host_ptr(pin_c.data_ptr(), n, pin_h.data_ptr())
        acc.submit_any_host_ptr(pin_a.data_ptr(), n, pin_o.data_ptr())
        acc.synchronize()

    def synchronous():
        acc.intersect_host_ptr(pin_c.data_ptr(), n, pin_h.data_ptr())
        acc.intersect_any_host_ptr(pin_a.data_ptr(), n, pin_o.data_ptr())

    secs = [measure_copy_rates()]
    for step in (submitted, synchronous):
        step()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            step()
        torch.cuda.synchronize()
        secs.append(time.perf_counter() - t0)
        barrier()
    return steps, secs[1], secs[2], secs[0]


def e2e_line(value, sync_value, steps, secs, rates, bytes_in, bytes_out):
    """The e2e object: the rate, the bytes a step moves, and the step time
    against the least time those copies take at the measured rates."""
    line = {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": bytes_in, "d2h_bytes_per_step": bytes_out,
            "calls": "bbg_intersect_submit + bbg_intersect_any_submit + bbg_accel_synchronize per step",
            "synchronous_calls_value": sync_value}
    if steps and rates:
        bound = copy_bound_ms(rates, bytes_in, bytes_out)
        step_ms = secs * 1e3 / steps
        line["copy_bound"] = {**{k: round(v, 1) for k, v in rates.items()}, "bound_ms": bound, "step_ms": step_ms,
                              "frac": bound / step_ms}
    return line


def measure_copy_rates(nbytes=256 << 20, reps=4):
    """Pinned host<->device copy rates (GB/s) on this box: host to device
    alone, device to host alone, and each direction while both run (two
    streams), timed with CUDA events (cudaMemcpyAsync through torch)."""
    import torch
    h_in = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    h_out = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    d_in = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    d_out = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()

    def timed(ops):
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        start.record()
        ends = []
        for st, fn in ops:
            st.wait_event(start)
            with torch.cuda.stream(st):
                for _ in range(reps):
                    fn()
                e = torch.cuda.Event(enable_timing=True)
                e.record(st)
                ends.append(e)
        torch.cuda.synchronize()
        return max(start.elapsed_time(e) for e in ends) / 1e3

    h2d = (s_in, lambda: d_in.copy_(h_in, non_blocking=True))
    d2h = (s_out, lambda: h_out.copy_(d_out, non_blocking=True))
    timed([h2d, d2h])  # warm-up
    rates = {"h2d_gbs": nbytes * reps / timed([h2d]) / 1e9, "d2h_gbs": nbytes * reps / timed([d2h]) / 1e9,
             "both_each_gbs": nbytes * reps / timed([h2d, d2h]) / 1e9}
    del h_in, h_out, d_in, d_out
    return rates


def copy_bound_ms(rates, bytes_in, bytes_out):
    """Least time to move a step's bytes: both directions at their shared
    rate while the smaller transfer lasts, the rest at the one-way rate."""
    both = min(bytes_in, bytes_out)
    rest_in, rest_out = bytes_in - both, bytes_out - both
    return 1e3 * (both / (rates["both_each_gbs"] * 1e9) + rest_in / (rates["h2d_gbs"] * 1e9)
                  + rest_out / (rates["d2h_gbs"] * 1e9))


PT_WORKLOAD = ("path tracing: closed Cornell box + displaced gold icosphere (8 subdivisions, 1,310,734 "
               "triangles), 1024x1024, 64 spp, 16 bounces, IndependentSampler, power light sampler")


def run_pt(args, barrier, world):
    """The path-tracing workload: one step = one full frame (bbg_render)."""
    import torch
    from bulbit_b200 import abi, lib, scenes
    res = args.pt_res
    scene = scenes.cornell_icosphere(levels=8, width=res, height=res, spp=64, max_bounces=16)
    t0 = time.perf_counter()
    if args.pt_device_split is not None:
        acc = lib.GpuAccel(scene, device_sah=True, split=args.pt_device_split)
    else:
        acc = lib.GpuAccel(scene, split=args.pt_split)
    build_s = time.perf_counter() - t0
    if args.traversal != "default":
        acc.set_traversal(abi.BBG_TRAVERSAL_WIDE if args.traversal == "wide" else abi.BBG_TRAVERSAL_ORDERED)
    integ = lib.GpuPathIntegrator(acc, scene)
    cam = lib.camera(scene.camera)
    params = abi.RenderParams()
    params.spp, params.seed, params.wave_paths, params.use_graph = 64, 0, args.pt_wave, 1
    params.shade_order = abi.BBG_SHADE_QUEUE if args.shade_order == "queue" else abi.BBG_SHADE_SORTED
    n_pix = res * res
    rgb = torch.empty((n_pix, 3), dtype=torch.float32, device="cuda")
    cnt = torch.empty(n_pix, dtype=torch.int32, device="cuda")
    mom = torch.empty((n_pix, 2), dtype=torch.float32, device="cuda")
    fs = abi.Film()
    fs.rgb_sum, fs.count, fs.moments, fs.path_L = rgb.data_ptr(), cnt.data_ptr(), mom.data_ptr(), None
    stats = abi.RenderStats()
    steps = max(1, args.pt_steps)

    def timed(clocks=None):
        for _ in range(max(1, args.warmup)):
            integ.render_device(cam, params, fs, stats)
        barrier()
        if clocks is not None:
            clocks.start()
        ms, r = 0.0, 0
        for _ in range(steps):
            integ.render_device(cam, params, fs, stats)
            ms += stats.device_ms
            r += stats.closest_rays + stats.shadow_rays
        if clocks is not None:
            clocks.info = clocks.stop()
        barrier()
        return ms, r

    clocks = ClockSampler(torch.cuda.current_device())
    clocks.info = None

    # Default launch configuration, then the autotuned one (which the
    # reported value uses; params.wave_paths = 0 lets the tuned wave apply).
    # Device times are the maximum over ranks.
    default_ms, default_rays = timed()
    default_ms = max_over_ranks([default_ms], device="cuda")[0]
    if args.no_autotune:
        tuning = abi.Tuning(128, 16, args.pt_wave, 0.0, 0)
        tune_s = 0.0
        dev_ms, rays = timed(clocks)
        dev_ms = max_over_ranks([dev_ms], device="cuda")[0]
    else:
        t0 = time.perf_counter()
        tuning = integ.autotune(spp=64, seed=0)
        tune_s = time.perf_counter() - t0
        params.wave_paths = 0
        dev_ms, rays = timed(clocks)
        dev_ms = max_over_ranks([dev_ms], device="cuda")[0]
    # End to end through the C ABI with a host film (copied back in the call).
    t0 = time.perf_counter()
    film = integ.render(spp=64)
    e2e_s = max_over_ranks([time.perf_counter() - t0], device="cuda")[0]
    paths = stats.paths
    out = {
        "value": whole_job_rate(paths * steps, world, dev_ms), "unit": "paths/s",
        "mrays_per_s": world * rays / (dev_ms / 1e3) / 1e6, "ms_per_frame": dev_ms / steps,
        "steps": steps, "closest_rays_per_frame": stats.closest_rays, "shadow_rays_per_frame": stats.shadow_rays,
        "default_config_ms_per_frame": default_ms / steps,
        "config": {"workload": PT_WORKLOAD if res == 1024 else f"{PT_WORKLOAD} (reduced to {res}x{res})",
                   "tree": ("split references built on the device, budget %g" % args.pt_device_split
                            if args.pt_device_split is not None else
                            "split references, budget %g" % args.pt_split if args.pt_split is not None else
                            "the reference's SAH tree"),
                   "bvh_build_s": round(build_s, 3), "default_wave_paths": args.pt_wave,
                   "tuned": {"block": tuning.block, "short_stack": tuning.short_stack,
                             "wave_paths": tuning.wave_paths, "autotune_s": round(tune_s, 2)},
                   "cuda_graph": True},
        "clocks": clocks.info,
        "image_mean": float(np.nanmean(film.image())),
        "e2e": {"value": whole_job_rate(paths, world, e2e_s * 1e3), "unit": "paths/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": n_pix * (12 + 4 + 8)},
        "gpu_launches_per_frame": -(-paths // (tuning.wave_paths - tuning.wave_paths % 64)) * (2 + 4 * 17),
    }
    # The same SAH tree built on the device (bbg_accel_create_device_sah): its
    # build time (geometry upload included, as in bvh_build_s), whether it is
    # byte for byte the host build's tree, and a frame over it.
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lib.GpuAccel(scene, device_sah=True).close()  # the first build in a process also loads its kernels
    first_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    dacc = lib.GpuAccel(scene, device_sah=True)
    dev_build_s = time.perf_counter() - t0
    hn, hs = acc.export()
    dn, ds = dacc.export()
    same_tree = bool(hn.shape == dn.shape and np.array_equal(hn.view(np.uint8), dn.view(np.uint8))
                     and np.array_equal(hs, ds))
    dinteg = lib.GpuPathIntegrator(dacc, scene)
    dinteg.set_tuning(tuning.block, tuning.short_stack, tuning.wave_paths)
    dinteg.render_device(cam, params, fs, stats)  # graph capture
    dinteg.render_device(cam, params, fs, stats)
    out["device_sah_tree"] = {"build_s": round(dev_build_s, 4), "first_build_in_process_s": round(first_s, 4),
                              "host_build_s": round(build_s, 3), "identical_to_host_tree": same_tree,
                              "ms_per_frame": stats.device_ms, "paths_per_s": stats.paths / (stats.device_ms / 1e3)}
    dinteg.close()
    dacc.close()
    integ.close()
    acc.close()
    # The same frame over a tree built on split references (a different tree
    # from the reference's SAH tree: hits agree except exact ties); its host
    # build time beside the plain SAH build's.
    if args.pt_split is None and args.pt_split_report > 0:
        t0 = time.perf_counter()
        acc = lib.GpuAccel(scene, split=args.pt_split_report)
        split_build_s = time.perf_counter() - t0
        integ = lib.GpuPathIntegrator(acc, scene)
        # The launch configuration tuned for the reference tree (a different
        # tree, the same frame).
        integ.set_tuning(tuning.block, tuning.short_stack, tuning.wave_paths)
        params.wave_paths = 0
        split_ms, split_rays = timed()
        split_ms = max_over_ranks([split_ms], device="cuda")[0]
        out["split_reference_tree"] = {
            "budget": args.pt_split_report, "value": whole_job_rate(paths * steps, world, split_ms), "unit": "paths/s",
            "mrays_per_s": world * split_rays / (split_ms / 1e3) / 1e6, "ms_per_frame": split_ms / steps,
            "bvh_build_s": round(split_build_s, 3), "launch_configuration": "the reference tree's tuned one"}
        integ.close()
        acc.close()
        # The same budget with the references split and the tree built on the
        # device (bbg_accel_create_device_split): build time (geometry upload
        # included; a first build in the process loads the kernels) and frame.
        torch.cuda.synchronize()
        lib.GpuAccel(scene, device_sah=True, split=args.pt_split_report).close()
        t0 = time.perf_counter()
        acc = lib.GpuAccel(scene, device_sah=True, split=args.pt_split_report)
        dsplit_build_s = time.perf_counter() - t0
        _, dslots = acc.export()
        integ = lib.GpuPathIntegrator(acc, scene)
        integ.set_tuning(tuning.block, tuning.short_stack, tuning.wave_paths)
        params.wave_paths = 0
        ds_ms, ds_rays = timed()
        ds_ms = max_over_ranks([ds_ms], device="cuda")[0]
        out["device_split_tree"] = {
            "budget": args.pt_split_report, "value": whole_job_rate(paths * steps, world, ds_ms), "unit": "paths/s",
            "mrays_per_s": world * ds_rays / (ds_ms / 1e3) / 1e6, "ms_per_frame": ds_ms / steps,
            "bvh_build_s": round(dsplit_build_s, 4), "references": int(len(dslots)),
            "launch_configuration": "the reference tree's tuned one"}
        integ.close()
        acc.close()
    return out, scene


def rel_mse(img, ref):
    """mean over pixels and channels of (x - ref)^2 / (ref^2 + 1e-2)."""
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))


def run_guided(args):
    """Neural path guiding against the plain tracer at equal device time.

    Scene: the path-tracing workload's Cornell box at a reduced resolution
    (args.guided_res). Reference: a 16384-spp plain render. Plain arm: 64 spp.
    Guided arm: a fresh guide trained online while it renders (train on every
    wave, guide_steps Adam steps of 2^16 samples each, lr 1e-2, guide/BSDF
    selection 1/2); its spp is chosen from a probe render so its device time
    matches the plain arm's; every sample, the training ones included, counts
    toward its image."""
    from bulbit_b200 import abi, lib, scenes
    res, wave, steps = args.guided_res, 1 << 21, 8
    scene = scenes.cornell_icosphere(levels=8, width=res, height=res, spp=64, max_bounces=16)
    acc = lib.GpuAccel(scene)
    if args.traversal != "default":
        acc.set_traversal(abi.BBG_TRAVERSAL_WIDE if args.traversal == "wide" else abi.BBG_TRAVERSAL_ORDERED)
    integ = lib.GpuPathIntegrator(acc, scene)
    ref_film = integ.render(spp=16384, seed=7)
    ref = ref_film.image()
    integ.render(spp=64, seed=1)  # graph capture for this shape
    plain = integ.render(spp=64, seed=2)
    t_plain = plain.stats.device_ms
    e_plain = rel_mse(plain.image(), ref)

    def guided(spp, seed, gseed):
        g = lib.GpuGuide(acc.bounds(), seed=gseed)
        f = integ.render(spp=spp, seed=seed, guide=g, train=True, wave_paths=wave, steps=steps, lr=1e-2)
        return f, g

    # Per-spp cost from the faster of two probes (a one-off stall of one
    # probe would otherwise skew the match), then one correction either way
    # if the matched render misses the plain arm's time by more than 5 %
    # (time is not linear in spp: whole waves).
    t_probe = min(guided(64, 3, 5)[0].stats.device_ms, guided(64, 9, 10)[0].stats.device_ms)
    spp_eq = max(1, int(64 * t_plain / t_probe))
    gf, g = guided(spp_eq, 4, 6)
    if abs(gf.stats.device_ms - t_plain) > 0.05 * t_plain:
        spp_eq = max(1, int(spp_eq * t_plain / gf.stats.device_ms))
        gf, g = guided(spp_eq, 4, 6)
    t_guided = gf.stats.device_ms
    e_guided = rel_mse(gf.image(), ref)
    same_spp = integ.render(spp=64, seed=8, guide=g)  # the trained guide, no more training
    e_same = rel_mse(same_spp.image(), ref)
    # Optional: a guide trained far longer than one frame allows (args.guided_pretrain
    # frames of 64 spp, 8 Adam steps per 2^21-path wave), then compared at equal spp.
    pretrained = None
    if args.guided_pretrain > 0:
        gp = lib.GpuGuide(acc.bounds(), seed=11)
        for k in range(args.guided_pretrain):
            integ.render(spp=64, seed=1000 + k, guide=gp, train=True, wave_paths=wave, steps=steps, lr=1e-2)
        pre = [rel_mse(integ.render(spp=64, seed=2000 + k, guide=gp).image(), ref) for k in range(2)]
        pl = [rel_mse(integ.render(spp=64, seed=3000 + k).image(), ref) for k in range(2)]
        pretrained = {"frames": args.guided_pretrain, "adam_steps": args.guided_pretrain * steps * -(-res * res * 64 // wave),
                      "guided_64spp_relMSE": pre, "plain_64spp_relMSE": pl}
    # Monte Carlo error falls as 1/time, so relMSE x time compares the two at
    # exactly equal time; the raw ratio at the matched spp is reported too.
    mlp = profile_values("guide_mlp_cornell128.md")
    out = {
        "metric": "relMSE at equal time, guided / plain", "value": (e_guided * t_guided) / (e_plain * t_plain),
        "mlp": {"kernels": "GuideForwardKernel and GuideWeightGradTcKernel (tcgen05, BF16 in, FP32 accumulators "
                           "in tensor memory); bulbit_b200/csrc/guide.cu",
                "forward_tensor_pipe_active": mlp.get("forward_tensor_pipe_active"),
                "wgrad_tensor_pipe_active": mlp.get("wgrad_tensor_pipe_active"),
                "wgrad_us_per_adam_step": mlp.get("wgrad_us"),
                "profile": "profiles/guide_mlp_cornell128.md"},
        "higher_is_better": False, "raw_relmse_ratio": e_guided / e_plain,
        "plain": {"spp": 64, "device_ms": t_plain, "relMSE": e_plain},
        "guided": {"spp": spp_eq, "device_ms": t_guided, "relMSE": e_guided, "probe_64spp_device_ms": t_probe,
                   "trained_guide_64spp_relMSE": e_same, "trained_guide_64spp_device_ms": same_spp.stats.device_ms},
        "reference": {"spp": 16384, "device_ms": ref_film.stats.device_ms},
        "pretrained_guide": pretrained,
        "config": {"workload": f"Cornell box + displaced gold icosphere (1,310,720 triangles) at {res}x{res}, "
                               "16 bounces; relMSE against a 16384-spp plain render",
                   "wave_paths": wave, "guide_steps_per_wave": steps, "guide_batch": 1 << 16, "guide_lr": 1e-2,
                   "guide_select": 0.5, "time": "device time of each render call (CUDA events)"},
    }
    integ.close()
    acc.close()
    return out


def run_guided_sweep(args):
    """Where the guided estimator bottoms out on the path-tracing scene (the
    Cornell box with the displaced gold icosphere at args.guided_res): guided
    against plain relMSE, at equal spp and at equal device time, over the
    guide/BSDF selection probability, the training budget (frames of online
    training before the measured renders, which keep training), and at one
    point the learning rate and the Adam steps per wave. Each row: three
    64-spp renders; relMSE against a 16384-spp plain render."""
    from bulbit_b200 import lib, scenes
    res, wave = args.guided_res, 1 << 21
    scene = scenes.cornell_icosphere(levels=8, width=res, height=res, spp=64, max_bounces=16)
    acc = lib.GpuAccel(scene)
    integ = lib.GpuPathIntegrator(acc, scene)
    ref = integ.render(spp=16384, seed=7).image()
    # Plain renders in waves of 2^24 paths (one wave per frame at 512^2 and
    # 64 spp: the fewest bounce-level ramp-downs).
    big = 1 << 24
    integ.render(spp=64, seed=1, wave_paths=big)  # graph capture
    plain = [integ.render(spp=64, seed=2 + k, wave_paths=big) for k in range(3)]
    e_plain = float(np.mean([rel_mse(f.image(), ref) for f in plain]))
    t_plain = float(np.mean([f.stats.device_ms for f in plain]))
    rows = []
    grid = [(sel, pre, 1e-2, 8, wave) for sel in (0.1, 0.25, 0.5) for pre in (0, 10, 40)]
    grid += [(0.25, 10, 3e-3, 8, wave), (0.25, 10, 1e-2, 32, wave)]
    # A pretrained guide needs no small waves to learn within the frame: the
    # same renders in waves of 2^24 paths (as the plain renders use), so the
    # guided frame has as many bounce levels, and ramp-downs, as the plain one.
    grid += [(0.1, 10, 1e-2, 8, big), (0.1, 40, 1e-2, 8, big), (0.1, 40, 1e-2, 32, big), (0.25, 40, 1e-2, 8, big)]
    for sel, pre, lr, steps, wave_paths in grid:
        g = lib.GpuGuide(acc.bounds(), seed=11)
        kw = dict(guide=g, train=True, wave_paths=wave_paths, steps=steps, lr=lr, select=sel)
        for k in range(pre):
            integ.render(spp=64, seed=1000 + k, **kw)
        films = [integ.render(spp=64, seed=2000 + k, **kw) for k in range(3)]
        e = float(np.mean([rel_mse(f.image(), ref) for f in films]))
        t = float(np.mean([f.stats.device_ms for f in films]))
        rows.append({"select": sel, "pretrain_frames": pre, "lr": lr, "adam_steps_per_wave": steps,
                     "wave_paths": wave_paths, "relMSE": e,
                     "device_ms": t, "relMSE_ratio": e / e_plain, "time_ratio": t / t_plain,
                     "equal_time_ratio": e * t / (e_plain * t_plain)})
        g.close()
    integ.close()
    acc.close()
    best = min(rows, key=lambda r: r["equal_time_ratio"])
    return {"metric": "relMSE at equal time, guided / plain (sweep)", "best": best, "rows": rows,
            "plain": {"spp": 64, "relMSE": e_plain, "device_ms": t_plain, "wave_paths": big},
            "config": {"workload": f"Cornell box + displaced gold icosphere (1,310,720 triangles) at {res}x{res}, "
                                   "16 bounces, 64 spp per render, relMSE against a 16384-spp plain render",
                       "wave_paths": wave, "guide_batch": 1 << 16}}


def run_batch(args):
    """The batched uneven multi-scene workload: 16 Cornell-box variants
    (seeds 0-15: displaced geodesic sphere of 10^4-2x10^6 triangles drawn
    log-uniform, Lambertian / dielectric / conductor, 256^2-1024^2), 32 spp,
    12 bounces. Each scene is rendered alone and then all 16 as one batch
    (every wavefront stage launched once per level for all scenes); paths/s
    and Mrays/s of both (each autotuned: the batch as a whole, every scene
    alone for itself), per-scene Mrays/s, and a bit-exact check of the
    batch's film of one scene against its own render. Guided vs plain: the
    batch at 96x96 per scene, plain and with one guide per scene (trained
    while rendering), 32 spp; relMSE per scene against a 4096-spp plain
    render, and relMSE x time."""
    from bulbit_b200 import lib, scenes
    t0 = time.perf_counter()
    sc = [scenes.cornell_batch_variant(seed) for seed in range(16)]
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    accs = [lib.GpuAccel(s) for s in sc]
    build_s = time.perf_counter() - t0
    integs = [lib.GpuPathIntegrator(a, s) for a, s in zip(accs, sc)]
    per_scene, alone_ms, alone_rays = [], 0.0, 0
    t0 = time.perf_counter()
    for it in integs:
        it.autotune(spp=32, seed=0)
    tune_alone_s = time.perf_counter() - t0
    for s, it in zip(sc, integs):
        it.render(spp=32, seed=0)  # capture
        f = it.render(spp=32, seed=0)
        rays = f.stats.closest_rays + f.stats.shadow_rays
        alone_ms += f.stats.device_ms
        alone_rays += rays
        per_scene.append({"scene": s.name, "triangles": s.n_prims, "paths": f.stats.paths, "rays": rays,
                          "alone_ms": f.stats.device_ms, "alone_mrays_per_s": rays / f.stats.device_ms / 1e3})
    b = lib.GpuBatch()
    b.render(integs, spp=32, seeds=[0] * 16)  # capture
    _, st_default = b.render(integs, spp=32, seeds=[0] * 16)
    t0 = time.perf_counter()
    bt = b.autotune(integs, spp=32, seeds=[0] * 16)
    tune_batch_s = time.perf_counter() - t0
    b.render(integs, spp=32, seeds=[0] * 16)  # capture
    films, st = b.render(integs, spp=32, seeds=[0] * 16)
    batch_rays = st.closest_rays + st.shadow_rays
    k = int(np.argmin([s.n_prims for s in sc]))
    alone = integs[k].render(spp=32, seed=0)
    exact = bool(np.array_equal(alone.rgb_sum, films[k].rgb_sum) and np.array_equal(alone.count, films[k].count))
    # The same batch over split-reference trees built on the device (budget
    # 3; hits equal the reference trees' except exact ties): the 16 builds'
    # time (after one warm-up build that loads the kernels) and the batch.
    lib.GpuAccel(sc[k], device_sah=True, split=3.0).close()
    t0 = time.perf_counter()
    saccs = [lib.GpuAccel(s, device_sah=True, split=3.0) for s in sc]
    split_build_s = time.perf_counter() - t0
    sintegs = [lib.GpuPathIntegrator(a, s) for a, s in zip(saccs, sc)]
    sb = lib.GpuBatch()
    sbt = sb.autotune(sintegs, spp=32, seeds=[0] * 16)
    sb.render(sintegs, spp=32, seeds=[0] * 16)  # capture
    _, sst = sb.render(sintegs, spp=32, seeds=[0] * 16)
    split_batch = {"budget": 3.0, "value": sst.paths / (sst.device_ms / 1e3), "unit": "paths/s",
                   "batch_ms": sst.device_ms, "mrays_per_s": (sst.closest_rays + sst.shadow_rays) / sst.device_ms / 1e3,
                   "bvh_build_s": round(split_build_s, 2),
                   "tuning": {"block": sbt.block, "short_stack": sbt.short_stack, "wave_paths": sbt.wave_paths}}
    sb.close()
    for it, a in zip(sintegs, saccs):
        it.close()
        a.close()
    # Guided vs plain in the batch, every scene at 96x96 (so that the 4096-spp
    # plain references stay cheap): the plain batch, then the batch with one
    # guide per scene (grouped forward per level, each guide trained online
    # on its scene's records), both at 32 spp; relMSE per scene against its
    # reference, and relMSE x time with the two batches' device times.
    for s in sc:
        s.camera.width = s.camera.height = 96
    refs = [it.render(spp=4096, seed=7).image() for it in integs]
    b.render(integs, spp=32, seeds=[1] * 16)  # capture
    pfilms, pst = b.render(integs, spp=32, seeds=[2] * 16)
    # At this size a scene alone (294,912 paths) leaves the GPU part-idle, so
    # the batch is timed against the scenes rendered one after another too
    # (same launch configuration).
    alone96_ms = 0.0
    for it in integs:
        it.render(spp=32, seed=2)  # capture
        alone96_ms += it.render(spp=32, seed=2).stats.device_ms
    small_scenes = {"config": "the 16 scenes at 96x96, 32 spp, 12 bounces", "paths": pst.paths,
                    "batch_ms": pst.device_ms, "sequential_ms": alone96_ms,
                    "speedup_vs_sequential": alone96_ms / pst.device_ms}
    guides = [lib.GpuGuide(a.bounds(), seed=5) for a in accs]
    gfilms, gst = b.render(integs, spp=32, seeds=[3] * 16, guides=guides, train=True, wave_paths=1 << 22, steps=4)
    time_ratio = gst.device_ms / pst.device_ms
    ratios = []
    for row, ref, pf, gf in zip(per_scene, refs, pfilms, gfilms):
        ep, eg = rel_mse(pf.image(), ref), rel_mse(gf.image(), ref)
        ratios.append(eg / ep)
        row["guided_vs_plain_in_batch_96px_32spp"] = {"plain_relMSE": ep, "guided_relMSE": eg,
                                                      "relMSE_ratio": eg / ep,
                                                      "equal_time_ratio": eg / ep * time_ratio}
    guided_batch = {"plain_batch_ms": pst.device_ms, "guided_batch_ms": gst.device_ms, "time_ratio": time_ratio,
                    "relMSE_ratio_geomean": float(np.exp(np.mean(np.log(ratios)))),
                    "equal_time_ratio_geomean": float(np.exp(np.mean(np.log(ratios)))) * time_ratio,
                    "config": "16 scenes at 96x96, 32 spp, one guide per scene trained online (after each "
                              "4,194,304-path wave, 4 Adam steps of up to 65,536 records per scene the wave covers), "
                              "relMSE against 4096-spp plain renders"}
    for g in guides:
        g.close()
    out = {
        "metric": "paths/s", "value": st.paths / (st.device_ms / 1e3), "unit": "paths/s",
        "mrays_per_s": batch_rays / st.device_ms / 1e3, "batch_ms": st.device_ms,
        "sequential": {"ms": alone_ms, "paths_per_s": st.paths / (alone_ms / 1e3),
                       "mrays_per_s": alone_rays / alone_ms / 1e3},
        "speedup_vs_sequential": alone_ms / st.device_ms,
        "batch_default_config_ms": st_default.device_ms,
        "tuning": {"batch": {"block": bt.block, "short_stack": bt.short_stack, "wave_paths": bt.wave_paths},
                   "batch_autotune_s": round(tune_batch_s, 2), "per_scene_autotune_s": round(tune_alone_s, 2)},
        "batch_film_equals_alone": exact, "device_split_trees": split_batch, "small_scenes": small_scenes,
        "per_scene": per_scene,
        "guided_batch": guided_batch,
        "config": {"workload": "16 uneven Cornell-box variants (seeds 0-15), 32 spp, 12 bounces, one batch",
                   "total_triangles": int(sum(s.n_prims for s in sc)), "paths": st.paths,
                   "scene_generation_s": round(gen_s, 2), "bvh_build_s": round(build_s, 2)},
    }
    b.close()
    for it, a in zip(integs, accs):
        it.close()
        a.close()
    return out


def pt_cpu_baseline(scene, stride=8):
    """The reference PathIntegrator (oracle/_ref) on a bounded sample of the
    path-tracing frame itself: every `stride`-th pixel in x and y of the
    1024x1024 frame (the frame's own mix of sphere, walls and light), all 64
    samples of each, traced by the reference's Li (the body of
    UniDirectionalRayIntegrator::Render's per-sample loop: sampler seed,
    camera ray, Li) over ParallelFor on all host threads."""
    from oracle import ref
    if not ref.available():
        return None
    cores = ref.init(0)
    rs = ref.RefScene(scene)
    rs.make_integrator(spp=scene.spp)
    W, H, spp = scene.camera.width, scene.camera.height, scene.spp
    ys, xs = np.mgrid[stride // 2:H:stride, stride // 2:W:stride]
    pix = (ys * W + xs).reshape(-1).astype(np.int64)
    ids = (pix[:, None] * spp + np.arange(spp, dtype=np.int64)[None, :]).reshape(-1)
    rs.trace_paths(path_ids=ids[: len(ids) // 16])  # warm-up
    _, secs = rs.trace_paths(path_ids=ids)
    return {"value": len(ids) / secs, "unit": "paths/s", "cores": cores, "kind": "reference",
            "sample": f"every {stride}th pixel in x and y of the {W}x{H} frame ({len(pix)} pixels), all {spp} "
                      f"samples each ({len(ids)} paths), traced by the reference PathIntegrator::Li on {cores} "
                      f"threads in {secs:.2f} s; BVH build {rs.build_seconds:.2f} s and integrator set-up "
                      f"{rs.integrator_seconds:.2f} s excluded"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bulbit_b200", choices=["bulbit_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--rays", type=int, default=N_RAYS, help="rays per query set (smaller cases for profiling)")
    ap.add_argument("--workload", default="all",
                    choices=["all", "rays", "pt", "guided", "batch", "guided-frame", "guided-sweep"])
    ap.add_argument("--no-autotune", action="store_true", help="path tracing: default launch configuration only")
    ap.add_argument("--no-batch", action="store_true", help="default workload: leave out the 16-scene batch")
    ap.add_argument("--guided-res", type=int, default=256)
    ap.add_argument("--guided-pretrain", type=int, default=0,
                    help="guided workload: also evaluate a guide trained for this many frames at equal spp")
    ap.add_argument("--traversal", default="default", choices=["default", "ordered", "wide"],
                    help="rays and pt workloads: node layout of the timed traversal")
    ap.add_argument("--pt-res", type=int, default=1024)
    ap.add_argument("--pt-split", type=float, default=None,
                    help="path tracing: build the tree over split references with this budget per primitive")
    ap.add_argument("--pt-device-split", type=float, default=None,
                    help="path tracing: the same, with the references split and the tree built on the device")
    ap.add_argument("--shade-order", default="sorted", choices=["sorted", "queue"],
                    help="path tracing: shade each level grouped by material kind, or in queue order")
    ap.add_argument("--pt-split-report", type=float, default=3.0,
                    help="path tracing: also time the frame over a split-reference tree of this budget (0: skip)")
    ap.add_argument("--pt-steps", type=int, default=3)
    ap.add_argument("--pt-wave", type=int, default=1 << 24)
    args = ap.parse_args()
    rank, world, local = dist_env()

    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import torch.distributed as dist
    from bulbit_b200 import abi, lib, scenes

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    if args.workload == "pt":
        pt, pt_scene = run_pt(args, barrier, world)
        if rank == 0:
            print(json.dumps({"path_tracing": pt}))
        return
    if args.workload == "guided":
        if rank == 0:
            print(json.dumps({"guided_path_tracing": run_guided(args)}))
        return
    if args.workload == "guided-frame":
        # One guided frame with online training (a profiling case): the
        # path-tracing scene at --guided-res, 64 spp, waves of 2^20 paths.
        from bulbit_b200 import lib, scenes
        sc = scenes.cornell_icosphere(levels=8, width=args.guided_res, height=args.guided_res, spp=64,
                                      max_bounces=16)
        acc = lib.GpuAccel(sc)
        integ = lib.GpuPathIntegrator(acc, sc)
        f = integ.render(spp=64, seed=3, guide=lib.GpuGuide(acc.bounds(), seed=5), train=True, wave_paths=1 << 20,
                         steps=8)
        if rank == 0:
            print(json.dumps({"guided_frame": {"device_ms": f.stats.device_ms, "paths": f.stats.paths,
                                               "closest_rays": f.stats.closest_rays,
                                               "shadow_rays": f.stats.shadow_rays}}))
        return
    if args.workload == "guided-sweep":
        if rank == 0:
            print(json.dumps({"guided_sweep": run_guided_sweep(args)}))
        return
    if args.workload == "batch":
        if rank == 0:
            print(json.dumps({"batched_scenes": run_batch(args)}))
        return

    n_rays = args.rays
    scene = scenes.triangle_soup(N_TRIS, seed=1)
    closest, anyq = scenes.soup_rays(n_rays, seed=2)
    t0 = time.perf_counter()
    acc = lib.GpuAccel(scene)
    build_s = time.perf_counter() - t0

    dev_c = torch.from_numpy(closest).cuda()
    dev_a = torch.from_numpy(anyq).cuda()
    hits = torch.empty((n_rays, 4), dtype=torch.float32, device="cuda")
    occ = torch.empty(n_rays, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream

    # Traversal statistics for the algorithmic-bytes roofline (untimed).
    acc.set_counting(True)
    acc.intersect_device(dev_c, hits, sptr)
    nodes_c, prims_c = acc.last_counts()
    acc.intersect_any_device(dev_a, occ, sptr)
    nodes_a, prims_a = acc.last_counts()
    acc.set_counting(False)
    if args.traversal != "default":
        acc.set_traversal(abi.BBG_TRAVERSAL_WIDE if args.traversal == "wide" else abi.BBG_TRAVERSAL_ORDERED)

    def step(events=None):
        with torch.cuda.stream(stream):
            if events is not None:
                events[0].record(stream)
            acc.intersect_device(dev_c, hits, sptr)
            if events is not None:
                events[1].record(stream)
            acc.intersect_any_device(dev_a, occ, sptr)
            if events is not None:
                events[2].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for k in range(args.steps):
        step(ev[k])
    end.record(stream)
    torch.cuda.synchronize()
    barrier()
    clock_info = clocks.stop()
    ms = start.elapsed_time(end)
    closest_ms = [e[0].elapsed_time(e[1]) for e in ev]
    any_ms = [e[1].elapsed_time(e[2]) for e in ev]

    # End to end through the C ABI with host (pinned) buffers: copies inside.
    e2e_steps, e2e_s, e2e_sync_s, copy_rates = 0, float("nan"), float("nan"), None
    if not args.no_e2e:
        e2e_steps, e2e_s, e2e_sync_s, copy_rates = run_e2e(args, acc, closest, anyq, barrier)
    ms, e2e_s, e2e_sync_s = max_over_ranks([ms, e2e_s, e2e_sync_s], device="cuda")

    rays_per_step = 2 * n_rays
    value = whole_job_rate(rays_per_step * args.steps, world, ms) / 1e6
    e2e_value = whole_job_rate(rays_per_step * e2e_steps, world, e2e_s * 1e3) / 1e6 if e2e_steps else None
    e2e_sync = whole_job_rate(rays_per_step * e2e_steps, world, e2e_sync_s * 1e3) / 1e6 if e2e_steps else None

    peaks, peak_kind = load_peaks()
    avg_closest_ms = statistics.mean(closest_ms)
    bytes_closest = n_rays * (32 + 16) + 32 * nodes_c + 48 * prims_c
    achieved = bytes_closest / (avg_closest_ms / 1e3) / 1e9
    prof = profile_values("trace_closest_soup1m.md")
    traffic = prof.get("dram_bytes_per_launch")

    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD if n_rays == N_RAYS else f"{WORKLOAD} (reduced to {n_rays} rays)",
                   "triangles": N_TRIS, "rays_per_step": rays_per_step,
                   "l2": "inputs larger than L2 (512 MiB of rays per query set)",
                   "parallelism": f"replicas x{world}", "bvh_build_s": round(build_s, 3)},
        # The tree and triangles stay in L2 (DRAM traffic is ~2 % of the
        # algorithmic bytes), so the kernel is bound by instruction issue:
        # achieved / frac are the algorithmic bytes per launch over its time
        # against the HBM copy peak (the byte-equivalent rate the reference's
        # traversal work would need), issue_active / alu_pipe_active the
        # measured issue and ALU utilisation (ncu, profiles/).
        "roofline": {"bound": "issue", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                     "issue_active": prof.get("issue_active"), "alu_pipe_active": prof.get("alu_pipe_active"),
                     "threads_per_instruction": prof.get("threads_per_instruction"),
                     "profile": "profiles/trace_closest_soup1m.md",
                     "kernel": "PersistentTraceKernel<closest, 8-wide> (bulbit_b200/csrc/accel.cu)",
                     "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": bytes_closest,
                     "per_ray": {"nodes": nodes_c / n_rays, "prims": prims_c / n_rays,
                                 "any_nodes": nodes_a / n_rays, "any_prims": prims_a / n_rays},
                     "avg_launch_ms": {"closest": avg_closest_ms, "any": statistics.mean(any_ms)}},
        "e2e": e2e_line(e2e_value, e2e_sync, e2e_steps, e2e_s, copy_rates, 2 * n_rays * 32, n_rays * 16 + n_rays * 1),
        "gpu_launches": 2 * args.steps,
        "clocks": clock_info,
    }
    acc.close()
    # The same soup and rays over the tree built on the device (linear BVH):
    # its build time beside the host SAH build, and its closest + any-hit
    # throughput (untimed in the headline; same event method).
    # The first build in a process also loads the build kernels; the second
    # is the build itself.
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lib.GpuAccel(scene, device_build=True).close()
    first_device_build_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    acc = lib.GpuAccel(scene, device_build=True)
    device_build_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev_d = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(max(1, args.steps))]
    for k in range(len(ev_d)):
        step(ev_d[k])
    torch.cuda.synchronize()
    dev_ms = sum(e[0].elapsed_time(e[2]) for e in ev_d)
    # The reference's SAH tree built on the device: build time beside the
    # host build (a second build; the first in a process loads the kernels).
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sah = lib.GpuAccel(scene, device_sah=True)
    first_sah_s = time.perf_counter() - t0
    sah.close()
    sah_ms = []
    for _ in range(3):
        t0 = time.perf_counter()
        sah = lib.GpuAccel(scene, device_sah=True)
        sah_ms.append((time.perf_counter() - t0) * 1e3)
        sah.close()
    line["device_sah_tree"] = {"build_ms": statistics.median(sah_ms), "builds_ms": sah_ms,
                               "first_build_in_process_ms": first_sah_s * 1e3, "host_sah_build_ms": build_s * 1e3,
                               "tree": "the host SAH build's tree, node for node (tests/test_device_sah_gpu.py)",
                               "timing": "wall clock of bbg_accel_create_device_sah (geometry upload included), "
                                         "median of 3 after a first, kernel-loading build"}
    line["device_built_tree"] = {
        "build_ms": device_build_s * 1e3, "first_build_in_process_ms": first_device_build_s * 1e3,
        "host_sah_build_ms": build_s * 1e3,
        "mrays_per_s": rays_per_step * len(ev_d) / (dev_ms / 1e3) / 1e6,
        "closest_ms": statistics.mean(e[0].elapsed_time(e[1]) for e in ev_d),
        "any_ms": statistics.mean(e[1].elapsed_time(e[2]) for e in ev_d)}
    acc.close()
    del dev_c, dev_a, hits, occ
    if args.workload == "all":
        pt, pt_scene = run_pt(args, barrier, world)
        line["path_tracing"] = pt
    # Every collective of the run is behind us: the other ranks leave, and
    # rank 0 alone runs the single-GPU extras (guided rendering, the batch of
    # scenes, the CPU baselines) without anyone waiting on a barrier.
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    if args.workload == "all":
        line["guided_path_tracing"] = run_guided(args)
        if not args.no_batch:
            line["batched_scenes"] = run_batch(args)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(scene, closest, anyq)
        if args.workload == "all":
            line["path_tracing"]["cpu_baseline"] = pt_cpu_baseline(pt_scene)
            cpu = line["path_tracing"]["cpu_baseline"]
            if cpu:
                line["path_tracing"]["vs_cpu_baseline"] = line["path_tracing"]["value"] / cpu["value"]
    print(json.dumps(line))


if __name__ == "__main__":
    main()
