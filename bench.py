"""Benchmark of the wavefront path-tracing hot path (one JSON line on rank 0).

Workload (one step = one full frame): the BVH-stress scene -- 985,090 unique float32 triangles
(three seeded displaced subdivision-7 icospheres instanced 40 times by seeded affine transforms in
a 20^3 volume over a ground plane; 50 % Lambert, 30 % anisotropic GGX conductor, 20 % GGX
dielectric), a 2,048-triangle emissive mesh light and a constant environment of radiance 0.5 --
at 1920 x 1080, 64 samples per pixel, depth 16, power MIS, Russian roulette from depth 3:
132,710,400 path samples per frame and GPU. The scene, camera rays, transport and film
accumulation all run on the device (inputs resident in HBM); `e2e` times the public C-ABI call
with host film buffers (bf200_render_film), copies included. `--workload cornell_spheres_256`
selects the 256 x 256 x 256 spp Cornell box with its GGX conductor and dielectric spheres.

Metric: path samples per second (whole job; weak scaling: every rank renders its own disjoint
sample range of the same frame and the per-GPU films are summed with one NCCL all-reduce).

`--impl reference` times the reference's own CPU implementation of the path (oracle/_ref: the
reference sources compiled as-is, trace_scene_mis + analytic accel + caller-side film, primary
rays from the reference's PinholeCamera) on the host cores over a bounded sample of the same
workload. `--impl reference-cuda` times the reference's own CUDA backend (oracle/_ref/
libbfrefcuda.so: trace_cuda_wavefront_transport with a reused workspace, as its benchmark calls
it) on one-sample-per-pixel batches of the same frame (2,073,600 paths per call at 1080p), and
bf200_trace_paths_with_cones on the same inputs in the same process.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "blackframe-renderer_b200"))
sys.path.insert(0, os.path.join(REPO, "tests"))
sys.path.insert(0, REPO)

import numpy as np  # noqa: E402

from bf200 import abi, multigpu, runtime, scenes  # noqa: E402

WORKLOAD = "bvh_stress_1080p"
METRIC = "path samples/s"
# every workload resolves its materials at the same wavelength packet (sample 0.1), whose CIE
# sensor constants the reference computed into this Cornell fixture
SENSOR_FIXTURE = "cornell_spheres_256"
# algorithmic bytes (the per-unit model of the path: rays, hits, path state, queue slots, film)
CAMERA_RAY_BYTES = 28
EXTENSION_SEGMENT_BYTES = 240
SHADOW_SEGMENT_BYTES = 96
FILM_SAMPLE_BYTES = 24
# algorithmic bytes per unit of each stage (unit: extension segment for trace and shade, shadow
# segment for occlude): trace reads the ray (28) and writes the hit (20); shade owns the rest of the
# extension segment's 240 B; occlude the whole shadow segment
STAGE_BYTES_PER_UNIT = {"trace": 48, "shade": EXTENSION_SEGMENT_BYTES - 48, "occlude": SHADOW_SEGMENT_BYTES}
STAGE_KERNELS = {"trace": "k_trace", "shade": "k_shade<kind> x4 + route/shadow compaction",
                 "occlude": "k_occlude"}
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per processed unit, per workload, from
# one ncu capture of a full-wavefront launch of each stage's kernels in this build (the stage
# kernels' launches at 2,097,152 slots)
MEASURED_TRAFFIC_PER_UNIT = {
    "cornell_spheres_256": {"trace": 56.5, "shade": 372.0, "occlude": None},
    "bvh_stress_1080p": {"trace": 203.0, "shade": None, "occlude": None},
}


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
        return float(data.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        query = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={query}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([v.strip() for v in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if len(s) > 3 + k and s[3 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons}


def workload_setup(workload):
    builder, options, (width, height, spp) = scenes.build_workload(workload)
    g = np.load(os.path.join(REPO, "tests", "golden", f"{SENSOR_FIXTURE}.npz"))
    from helpers import sensor_from_golden
    sensor = sensor_from_golden(g)
    origin, normal, tangent, vfov = scenes.workload_camera(workload)
    camera = runtime.camera_create(origin, normal, tangent, width, height, vfov, scenes.PATH_TIME)
    return builder, options, camera, sensor, (width, height, spp)


def frame_samples(width, height, sample_index, seed=0, pixels=None):
    """SampleIndex records of a frame's pixels (row-major, or the given (x, y) pairs) at one sample
    index, built in bulk."""
    if pixels is None:
        ys, xs = np.divmod(np.arange(width * height, dtype=np.uint64), np.uint64(width))
    else:
        xs, ys = pixels[:, 0], pixels[:, 1]
    n = len(xs)
    table = np.zeros(n, dtype=[("x", "<u4"), ("y", "<u4"), ("s", "<u8"), ("seed", "<u8")])
    table["x"], table["y"] = xs, ys
    table["s"], table["seed"] = sample_index, seed
    return (abi.SampleIndex * n).from_buffer_copy(table.tobytes())


def path_inputs(rays, samples):
    """PathInput records (primary ray, sample index) built in bulk."""
    n = len(samples)
    table = np.zeros(n, dtype=[("ray", "V48"), ("sample", "V24"), ("reserved", "<u8")])
    table["ray"] = np.frombuffer(bytes(rays), dtype="V48")
    table["sample"] = np.frombuffer(bytes(samples), dtype="V24")
    return (abi.PathInput * n).from_buffer_copy(table.tobytes())


def reference_camera_inputs(workload, samples, cones=False):
    """Primary rays (and, with cones, primary ray cones) of the reference's own PinholeCamera for
    the workload's camera (oracle/_ref): no bf200 library is loaded on this path."""
    from oracle.bindings import Reference
    _, _, (width, height, _) = scenes.build_workload(workload)
    origin, normal, tangent, vfov = scenes.workload_camera(workload)
    ref = Reference()
    rays = ref.camera_rays(origin, normal, tangent, width, height, vfov, scenes.PATH_TIME, samples)
    inputs = path_inputs(rays, samples)
    if not cones:
        return inputs
    return inputs, ref.camera_cones(origin, normal, tangent, width, height, vfov, scenes.PATH_TIME, samples)


# Workloads whose CPU baseline is the oracle restatement instead of the compiled reference: the
# reference's only CPU accel here is its analytic one (Embree is absent), which tests every triangle
# of every instance for every ray -- on the 985k-triangle, 40-instance scene more than five minutes
# per path on one core -- so a bounded sample of it cannot finish in a bench step. The restatement
# computes the same paths (pinned bit-exact against the reference by the CPU tests) and rejects
# triangles with a conservative double prefilter first, about 1.4 s per path on one core.
PORT_BASELINE_WORKLOADS = {"bvh_stress_1080p"}


class CpuReference:
    """The reference CPU path on all host threads over bounded random samples of a workload's paths:
    oracle/_ref (trace_scene_mis with the analytic accel), or the oracle restatement for the
    workloads above; primary rays of the reference's own PinholeCamera either way. No bf200 library
    is loaded on this path."""

    def __init__(self, workload):
        from oracle.bindings import CheckerError, Oracle, Reference, reference_available
        if not reference_available():
            raise CheckerError("the CPU reference arm needs oracle/_ref/libbfref.so (oracle/Makefile, target ref)")
        self.workload = workload
        self.builder, self.options, (self.width, self.height, self.spp) = scenes.build_workload(workload)
        self.kind = "port" if workload in PORT_BASELINE_WORKLOADS else "reference"
        self.checker = Oracle() if self.kind == "port" else Reference()
        self.threads = os.cpu_count() or 1
        self.handle = self.checker.scene(self.builder)
        self.rng = np.random.default_rng(5)
        self.per_path = None

    def batch(self, n):
        pixels = np.stack([self.rng.integers(self.width, size=n), self.rng.integers(self.height, size=n)],
                          axis=1).astype(np.uint64)
        samples = frame_samples(self.width, self.height, 0, pixels=pixels)
        sample_index = self.rng.integers(self.spp, size=n)
        for k in range(n):
            samples[k].sample_index = int(sample_index[k])
        return reference_camera_inputs(self.workload, samples)

    def run(self, n):
        """Traces n random paths; returns the seconds taken."""
        inputs = self.batch(n)
        t0 = time.perf_counter()
        self.checker.trace(self.handle, inputs, self.options, self.threads)
        elapsed = time.perf_counter() - t0
        if self.per_path is None:
            self.per_path = max(1e-6, elapsed / n)
        return elapsed

    def sized(self, target_seconds):
        """Paths for about target_seconds of work (at least one per thread)."""
        if self.per_path is None:
            self.run(self.threads)
        return int(max(self.threads, min(200000, target_seconds / self.per_path)))

    def close(self):
        self.checker.destroy(self.handle)

    def describe(self, n):
        what = ("the oracle restatement (pinned bit-exact on the reference; triangles rejected by a conservative "
                "double prefilter before the exact test)" if self.kind == "port" else
                "oracle/_ref: the reference's trace_scene_mis with its analytic accel")
        return (f"{n} random (pixel, sample) paths of {self.workload} per step, primary rays of the reference's "
                f"PinholeCamera, traced by {what} on {self.threads} threads")


def cpu_sample_rate(workload, target_seconds=15.0):
    """One bounded sample of the reference CPU path: (paths/s, threads, kind, sample text, paths,
    seconds)."""
    ref = CpuReference(workload)
    n = ref.sized(target_seconds)
    elapsed = ref.run(n)
    ref.close()
    return n / elapsed, ref.threads, ref.kind, ref.describe(n), n, elapsed


BATCH_WORKLOAD = "batch64"


def run_batch(args, torch, rank, world, local_rank):
    """The 64-scene batch: one bf200_render_films_device call over 64 uneven jobs against the same
    64 jobs rendered one after another with bf200_render_film_device. Each step renders every job
    once; both arms are timed with CUDA events around the whole step (films zeroed before). With N
    GPUs the jobs are sharded whole (multigpu.batch_shard, no exchange) and each step's time is the
    maximum over ranks."""
    import torch.distributed as dist
    from datetime import timedelta
    distributed = world > 1
    if distributed:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    g = np.load(os.path.join(REPO, "tests", "golden", f"{SENSOR_FIXTURE}.npz"))
    from helpers import sensor_from_golden
    sensor = sensor_from_golden(g)
    ctx = runtime.Context(local_rank, path_capacity=args.capacity)
    all_paths = []
    for seed in range(64):
        _, _, (w, h, spp) = scenes.batch_job(seed)
        all_paths.append(w * h * spp)
    mine = multigpu.batch_shard(all_paths, rank, world)
    jobs, films, paths, triangles = [], [], 0, 0
    for seed in mine:
        builder, options, (w, h, spp) = scenes.batch_job(seed)
        scene = ctx.create_scene(builder)
        cam = runtime.camera_create(*scenes.camera_frame_inputs(), w, h, scenes.CAMERA_VFOV, scenes.PATH_TIME)
        sums = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
        counts = torch.zeros((h, w), dtype=torch.int64, device="cuda")
        jobs.append([scene, cam, sensor, options, spp, 0, 0, 0, sums.data_ptr(), counts.data_ptr(), builder])
        films.append((sums, counts))
        paths += w * h * spp
        triangles += builder.triangle_count
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def batched():
        return ctx.render_films_device([j[:10] for j in jobs], lanes=args.lanes)

    def serial():
        return [ctx.render_film_device(*j[:10]) for j in jobs]

    def timed(fn, step):
        for sums, counts in films:
            sums.zero_()
            counts.zero_()
        flush.fill_(step & 0xFF)
        torch.cuda.synchronize()
        if distributed:
            dist.barrier()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        reports = fn()
        stop.record()
        torch.cuda.synchronize()
        ms = start.elapsed_time(stop)
        if distributed:
            t = torch.tensor([ms], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, reports

    for step in range(args.warmup):
        timed(batched, step)
        timed(serial, step)
    batch_ms, serial_ms, failed = [], [], 0
    with ClockSampler(local_rank) as clocks:
        for step in range(args.steps):
            ms, reports = timed(batched, step)
            batch_ms.append(ms)
            failed += sum(r.failed_lanes for r in reports)
            ms, _ = timed(serial, step)
            serial_ms.append(ms)
    batch_total, serial_total = sum(batch_ms), sum(serial_ms)
    total_paths = sum(all_paths)
    value = total_paths * args.steps / (batch_total / 1000.0)
    serial_value = total_paths * args.steps / (serial_total / 1000.0)
    if distributed:
        f = torch.tensor([failed], dtype=torch.int64, device="cuda")
        dist.all_reduce(f)
        failed = int(f.item())
    line = {
        "metric": "batched path samples/s", "value": value, "unit": "path samples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": batch_total / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": BATCH_WORKLOAD, "jobs": 64, "jobs_per_gpu": len(mine), "paths_per_step": total_paths,
                   "unique_triangles_rank0": triangles,
                   "parallelism": f"whole scenes sharded x{world}" if distributed else "single GPU",
                   "lanes": args.lanes or "measured (2, 4 or 8)", "path_capacity": args.capacity,
                   "l2": "flushed between steps (256 MiB write)"},
        "serial": {"value": serial_value, "ms_per_step": serial_total / args.steps},
        "batched_vs_serial": value / serial_value, "lanes_used": ctx.batch_lanes(), "failed_lanes": failed,
        "clocks": clocks.summary(),
    }
    for j in jobs:
        j[0].close()
    ctx.close()
    if distributed:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


ADJOINT_WORKLOAD = "adjoint_icosphere_256"


def run_adjoint_distributed(args, torch, rank, world, local_rank):
    """The adjoint on N GPUs (weak in nothing: the 64 spp of the frame are split across ranks). One
    step: each rank renders its samples (bf200_render_film_device), the films are summed (NCCL
    all-reduce), every rank forms dLoss/d(image) = 2 (image - target), runs
    bf200_render_backward_device on its samples, and the gradients are summed (all-reduce). The
    target is uploaded from pinned host memory and the gradients read back every step (so the
    step is also the end-to-end figure); time = max over ranks of CUDA events around the step."""
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local_rank))
    builder, options, camera, sensor, (width, height, spp) = workload_setup(ADJOINT_WORKLOAD)
    if args.spp > 0:
        spp = args.spp
    share = spp // world
    if share * world != spp:
        raise SystemExit("the adjoint bench splits the samples evenly: spp must be a multiple of the GPU count")
    ctx = runtime.Context(local_rank, path_capacity=args.capacity)
    target_builder = scenes.adjoint_icosphere(scenes.SceneBuilder(), scenes.perturbed_parameters(scenes.adjoint_parameters()))
    target_scene = ctx.create_scene(target_builder)
    sums = torch.zeros((height, width, 8), dtype=torch.float64, device="cuda")
    counts = torch.zeros((height, width), dtype=torch.int64, device="cuda")
    ctx.render_film_device(target_scene, camera, sensor, options, spp, 7, 0, 1, sums.data_ptr(), counts.data_ptr())
    target_host = ((sums[..., :3] + sums[..., 4:7]) / (sums[..., 3:4] + sums[..., 7:8])).float().cpu().pin_memory()
    target_scene.close()
    scene = ctx.create_scene(builder)
    target = torch.empty_like(target_host, device="cuda")
    grads = torch.zeros((len(builder.materials), 8), dtype=torch.float64, device="cuda")
    emission = torch.zeros(1, dtype=torch.float64, device="cuda")
    host_grads = torch.empty((len(builder.materials) * 8 + 1,), dtype=torch.float64).pin_memory()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def step_once():
        target.copy_(target_host, non_blocking=True)
        sums.zero_()
        counts.zero_()
        forward = ctx.render_film_device(scene, camera, sensor, options, share, 0, rank * share, 1, sums.data_ptr(),
                                         counts.data_ptr())
        multigpu.reduce_film(sums, counts)
        image = (sums[..., :3] + sums[..., 4:7]) / (sums[..., 3:4] + sums[..., 7:8])
        image_adjoint = (2.0 * (image - target.double())).float().contiguous()
        retrace = ctx.render_backward_device(scene, camera, sensor, options, share, 0, rank * share, 1,
                                             sums.data_ptr(), counts.data_ptr(), image_adjoint.data_ptr(),
                                             grads.data_ptr(), emission.data_ptr())
        packed = torch.cat([grads.flatten(), emission])
        dist.all_reduce(packed)
        host_grads.copy_(packed, non_blocking=True)
        # forward, loss image, re-trace, and a replay with as many launches as the re-trace
        launches[0] += forward.kernel_launches + 1 + 2 * retrace.kernel_launches
        return float(((image - target.double()) ** 2).sum().item())

    launches = [0]
    for w in range(args.warmup):
        step_once()
    launches[0] = 0
    step_ms = []
    with ClockSampler(local_rank) as clocks:
        for k in range(args.steps):
            flush.fill_(k & 0xFF)
            torch.cuda.synchronize()
            dist.barrier()
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            loss = step_once()
            stop.record()
            torch.cuda.synchronize()
            t = torch.tensor([start.elapsed_time(stop)], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            step_ms.append(float(t.item()))
    total = sum(step_ms)
    paths = width * height * spp
    value = paths * args.steps / (total / 1000.0)
    scene.close()
    ctx.close()
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({
            "metric": "adjoint path samples/s", "value": value, "unit": "path samples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": ADJOINT_WORKLOAD, "width": width, "height": height, "spp": spp,
                       "parallelism": f"samples split x{world}; film and gradient all-reduce",
                       "l2": "flushed between steps (256 MiB write); path state > L2"},
            "loss": loss, "clocks": clocks.summary(),
            "e2e": {"value": value, "unit": "path samples/s", "h2d_bytes_per_step": target_host.numel() * 4,
                    "d2h_bytes_per_step": host_grads.numel() * 8},
            "gpu_launches": launches[0]}), flush=True)


def run_adjoint(args, torch, rank):
    """The path-replay adjoint: one step = one bf200_render_adjoint_device call (forward render of
    256 x 256 x 64 spp, L2 loss against a target rendered at perturbed parameters, replay of every
    path). Timed with CUDA events around the call; the forward render alone is timed beside it."""
    if rank != 0:
        return
    builder, options, camera, sensor, (width, height, spp) = workload_setup(ADJOINT_WORKLOAD)
    if args.spp > 0:
        spp = args.spp
    target_params = scenes.perturbed_parameters(scenes.adjoint_parameters())
    target_builder = scenes.adjoint_icosphere(scenes.SceneBuilder(), target_params)
    ctx = runtime.Context(0, path_capacity=args.capacity)
    scene, target_scene = ctx.create_scene(builder), ctx.create_scene(target_builder)
    sums = torch.zeros((height, width, 8), dtype=torch.float64, device="cuda")
    counts = torch.zeros((height, width), dtype=torch.int64, device="cuda")
    ctx.render_film_device(target_scene, camera, sensor, options, spp, 7, 0, 1, sums.data_ptr(), counts.data_ptr())
    torch.cuda.synchronize()
    target = ((sums[..., :3] + sums[..., 4:7]) / (sums[..., 3:4] + sums[..., 7:8])).float().contiguous()
    target_scene.close()
    materials = len(builder.materials)
    grads = torch.zeros((materials, 8), dtype=torch.float64, device="cuda")
    emission = torch.zeros(1, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    paths = width * height * spp

    def adjoint():
        return ctx.render_adjoint_device(scene, camera, sensor, options, spp, 0, 0, 1, sums.data_ptr(),
                                         counts.data_ptr(), target.data_ptr(), grads.data_ptr(), emission.data_ptr())

    def forward():
        sums.zero_()
        counts.zero_()
        return ctx.render_film_device(scene, camera, sensor, options, spp, 0, 0, 1, sums.data_ptr(),
                                      counts.data_ptr())

    def timed(fn, step):
        flush.fill_(step & 0xFF)
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        out = fn()
        stop.record()
        torch.cuda.synchronize()
        return start.elapsed_time(stop), out

    for step in range(args.warmup):
        timed(adjoint, step)
        timed(forward, step)
    adjoint_ms, forward_ms, results = [], [], []
    with ClockSampler(0) as clocks:
        for step in range(args.steps):
            ms, out = timed(adjoint, step)
            adjoint_ms.append(ms)
            results.append(out)
            ms, _ = timed(forward, step)
            forward_ms.append(ms)
    total = sum(adjoint_ms)
    value = paths * args.steps / (total / 1000.0)
    forward_value = paths * args.steps / (sum(forward_ms) / 1000.0)
    loss, report = results[-1]

    # e2e: target uploaded from pinned host memory and gradients read back every step
    host_target = target.cpu().pin_memory()
    host_grads = torch.empty((materials, 8), dtype=torch.float64).pin_memory()
    host_emission = torch.empty(1, dtype=torch.float64).pin_memory()
    e2e_ms = []
    for step in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        target.copy_(host_target, non_blocking=True)
        adjoint()
        host_grads.copy_(grads, non_blocking=True)
        host_emission.copy_(emission, non_blocking=True)
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t0) * 1000.0)
    e2e_value = paths * len(e2e_ms) / (sum(e2e_ms) / 1000.0)
    # one more call, untimed, with the host-driven loop: profilers see the replay kernels of this
    # call (the device-side loop graph of the timed calls hides its kernels from them)
    options.instrumentation = 1
    adjoint()
    options.instrumentation = 0
    torch.cuda.synchronize()
    g = host_grads.numpy()
    basis = scenes.basis_gradients(g, builder.nanometers)
    ext, shadow = report.extension_segments, report.shadow_segments
    # both passes move the path's algorithmic bytes (camera ray, segments, film once)
    alg = 2 * (CAMERA_RAY_BYTES * paths + EXTENSION_SEGMENT_BYTES * ext + SHADOW_SEGMENT_BYTES * shadow) + \
        FILM_SAMPLE_BYTES * paths
    peak, peak_kind = measured_peaks()
    achieved = alg / (total / args.steps / 1000.0) / 1e9
    line = {
        "metric": "adjoint path samples/s", "value": value, "unit": "path samples/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": ADJOINT_WORKLOAD, "width": width, "height": height, "spp": spp, "max_depth": 8,
                   "mis": "power", "russian_roulette": False, "triangles": builder.triangle_count,
                   "parameters": "albedo 4 materials x 8 basis coefficients, 2 GGX alphas, light scale",
                   "target": "render at parameters + N(0, 0.1), seed 7", "path_capacity": args.capacity,
                   "l2": "flushed between steps (256 MiB write); path state > L2"},
        "forward_only": {"value": forward_value, "ms_per_step": sum(forward_ms) / args.steps},
        "adjoint_over_forward_time": (total / args.steps) / (sum(forward_ms) / args.steps),
        "loss": loss, "gradients": {"albedo_basis_norm": float(np.linalg.norm(basis)),
                                     "alpha": [float(g[scenes.ADJOINT_CONDUCTOR, 4] + g[scenes.ADJOINT_CONDUCTOR, 5]),
                                               float(g[scenes.ADJOINT_DIELECTRIC, 4] +
                                                     g[scenes.ADJOINT_DIELECTRIC, 5])],
                                     "light_scale": float(host_emission[0])},
        "failed_lanes": report.failed_lanes, "clocks": clocks.summary(),
        "e2e": {"value": e2e_value, "unit": "path samples/s", "h2d_bytes_per_step": host_target.numel() * 4,
                "d2h_bytes_per_step": host_grads.numel() * 8 + 8},
        # the forward render's launches, the loss kernel and the replay (as many launches as the forward)
        "gpu_launches": (2 * report.kernel_launches + 1) * args.steps,
        "roofline": {"bound": "hbm", "kernel": "whole adjoint call (forward + replay)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                     "peak_source": peak_kind},
    }
    scene.close()
    ctx.close()
    print(json.dumps(line), flush=True)


IMPORT_WORKLOAD = "mesh_import_obj"
SCENE_JSON_WORKLOAD = "scene_json"
REFIT_WORKLOAD = "refit_bvh_stress"


def run_refit(args, torch):
    """Transform-only refit of the BVH-stress scene (985k triangles, 42 instances, TLAS): each step
    moves every instance (new seeded transforms) with bf200_scene_refit, beside bf200_scene_create
    of the same description (BLAS builds included). Host wall time around each C call (the
    descriptions are made before); the refit's device work (uploads, world normals) is inside it,
    since the call returns after its stream."""
    import copy
    builder, _, _, _, _ = workload_setup("bvh_stress_1080p")
    ctx = runtime.Context(0, path_capacity=args.capacity)
    ctx.set_build_mode(abi.BUILD_DEVICE_LBVH if args.build_mode == "lbvh" else abi.BUILD_HOST_SAH)
    scene = ctx.create_scene(builder)
    rng = np.random.default_rng(2)
    targets = []
    for step in range(args.warmup + args.steps):
        b = copy.copy(builder)
        b.instances = []
        for mesh, material, matrix, mask in builder.instances:
            m = np.array(matrix, np.float32)
            m[:3, 3] = (m[:3, 3] + rng.uniform(-0.5, 0.5, 3)).astype(np.float32)
            b.instances.append((mesh, material, m, mask))
        targets.append(b)
    refit_s = []
    for step, b in enumerate(targets):
        desc = b.desc()  # the caller's description, made before the timed call
        t0 = time.perf_counter()
        scene.refit(b, desc)
        torch.cuda.synchronize()
        if step >= args.warmup:
            refit_s.append(time.perf_counter() - t0)
    create_s = []
    create_stats = None
    for step in range(max(1, min(args.steps, 2))):
        desc = targets[-1].desc()
        t0 = time.perf_counter()
        fresh = ctx.create_scene(targets[-1], desc)
        torch.cuda.synchronize()
        create_s.append(time.perf_counter() - t0)
        st = fresh.stats()
        create_stats = {k: getattr(st, k) for k, _ in st._fields_ if k != "struct_size"}
        fresh.close()
    scene.close()
    ctx.close()
    refit_ms = statistics.median(refit_s) * 1000.0
    create_ms = statistics.median(create_s) * 1000.0
    line = {"metric": "refit ms", "value": refit_ms, "unit": "ms", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": refit_ms, "higher_is_better": False, "scaling": "none",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": REFIT_WORKLOAD, "instances": len(builder.instances),
                       "triangles": builder.triangle_count, "build_mode": args.build_mode},
            "scene_create_ms": create_ms, "create_over_refit": create_ms / refit_ms,
            "scene_create_phases": create_stats, "gpu_launches": 1}
    print(json.dumps(line), flush=True)


def run_mesh_import(args):
    """Scene ingestion: bf200_mesh_load on a seeded 327,680-triangle OBJ (a displaced subdivision-7
    icosphere written with 9 significant digits, about 37 MB), beside the reference's own loader
    (oracle/_ref) on the same file. Host code on both sides; the arrays must be identical."""
    import tempfile
    v, f = scenes.icosphere(7)
    rng = np.random.default_rng(1)
    p = v * (1.0 + 0.02 * rng.uniform(-1.0, 1.0, len(v)))[:, None]
    n = (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)
    uv = rng.uniform(0.0, 1.0, (len(v), 2))
    lines = ["v %.9g %.9g %.9g" % tuple(r) for r in p] + ["vt %.9g %.9g" % tuple(r) for r in uv]
    lines += ["vn %.9g %.9g %.9g" % tuple(map(float, r)) for r in n]
    lines += ["f %d/%d/%d %d/%d/%d %d/%d/%d" % (a + 1, a + 1, a + 1, b + 1, b + 1, b + 1, c + 1, c + 1, c + 1)
              for a, b, c in f]
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "icosphere7.obj")
        with open(path, "w") as handle:
            handle.write("\n".join(lines) + "\n")
        size = os.path.getsize(path)
        for _ in range(args.warmup):
            runtime.load_mesh(path)
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            mesh = runtime.load_mesh(path)
            times.append(time.perf_counter() - t0)
        reference = None
        from oracle.bindings import Reference, reference_available
        if reference_available():
            ref = Reference()
            ref_times = []
            for _ in range(max(1, args.steps)):
                t0 = time.perf_counter()
                want, _, _ = ref.load_mesh(path)
                ref_times.append(time.perf_counter() - t0)
            same = all(np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))
                       for a, b in zip(mesh, want))
            reference = {"value": len(f) / statistics.median(ref_times), "seconds": statistics.median(ref_times),
                         "identical_arrays": same, "kind": "reference"}
    seconds = statistics.median(times)
    line = {"metric": "imported triangles/s", "value": len(f) / seconds, "unit": "triangles/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": seconds * 1000.0, "higher_is_better": True,
            "scaling": "none", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": IMPORT_WORKLOAD, "triangles": len(f), "vertices": len(v), "bytes": size,
                       "host": "one thread"},
            "mb_per_s": size / seconds / 1e6, "reference_loader": reference, "gpu_launches": 0}
    print(json.dumps(line), flush=True)


def scene_json_document():
    """A native scene JSON document of 655,360 triangles: two displaced subdivision-7 icospheres
    (327,680 triangles each), 16 instances in a two-level hierarchy, three materials, a point light
    and the environment; about 50 MB of text written with 9 significant digits, inside every
    default budget of the reference's reader."""
    rng = np.random.default_rng(3)
    geometries = []
    for gid, level in ((10, 7), (11, 7)):
        v, f = scenes.icosphere(level)
        p = (v * (1.0 + 0.02 * rng.uniform(-1.0, 1.0, len(v)))[:, None]).astype(np.float32)
        n = (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)
        uv = rng.uniform(0.0, 1.0, (len(v), 2)).astype(np.float32)
        rows = lambda a: ",".join("[" + ",".join("%.9g" % x for x in r) + "]" for r in a)
        tris = ",".join("[%d,%d,%d]" % tuple(t) for t in f)
        geometries.append((gid, len(f), '{"id":%d,"mesh":{"positions":[%s],"normals":[%s],"texture_coordinates":[%s],'
                           '"triangles":[%s]}}' % (gid, rows(p), rows(n), rows(uv), tris)))
    packet = '{"nanometers":[471.2129,588.7129,706.2129,823.7129],"pdf":[0.0021276595,0.0021276595,0.0021276595,0.0021276595]}'
    lambert = ('{"id":%d,"spectral":{"wavelengths":' + packet + ',"closures":{"frame_mode":"shading_normal",'
               '"tangent_rotation_radians":0,"components":[{"probability":1,"type":"lambertian_reflection",'
               '"weight":[0.5,0.5,0.5,0.5]}]},"emission":[%s],"normal_map":null,"bump_map":null}}')
    materials = [lambert % (20, "0,0,0,0"), lambert % (21, "0,0,0,0"), lambert % (22, "4,3,2,1")]
    instances = []
    for k in range(16):
        m = np.eye(4)
        m[:3, 3] = rng.uniform(-10, 10, 3)
        parent = "null" if k < 4 else str(300 + k % 4)
        instances.append('{"id":%d,"parent":%s,"object":1,"geometry":%d,"material":%d,"local_to_parent":[%s],'
                         '"visibility_mask":4294967295}' % (300 + k, parent, 10 + k % 2, 20 + k % 3,
                                                            ",".join("%.9g" % x for x in m.ravel())))
    text = ('{"schema":"blackframe.scene","schema_version":1,"active":{"film":1,"camera":1,"render_options":1},'
            '"films":[{"id":1,"extent":[1920,1080],"crop":[0,0,1920,1080],"accumulation":"float32"}],'
            '"cameras":[{"id":1,"film":1,"model":{"type":"pinhole","origin":[0,0,30],"normal":[0,0,1],'
            '"tangent":[1,0,0],"bitangent":[0,1,0],"vertical_fov_radians":0.8,"t_min":0,"t_max":1e30,'
            '"visibility_mask":4294967295,"current_medium":0}}],'
            '"render_options":[{"id":1,"film":1,"samples_per_pixel":64,"maximum_path_depth":8,"tile_edge_length":16,'
            '"seed":0,"pixel_jitter":"uniform","mis_heuristic":"power","light_sampling_strategy":"uniform",'
            '"depth_limits":{"diffuse":8,"glossy":8,"specular":8,"transmission":8,"volume":0},'
            '"russian_roulette":{"mode":"disabled"}}],"constant_textures":[],"host_image_textures":[],'
            '"objects":[{"id":1}],"geometries":[' + ",".join(g[2] for g in geometries) + '],"materials":['
            + ",".join(materials) + '],"instances":[' + ",".join(instances) + '],"lights":[{"id":1,'
            '"type":"environment","wavelengths":' + packet + ',"radiance":[0.1,0.1,0.1,0.1]},{"id":2,"type":"point",'
            '"position":[0,20,0],"absolute_position_error":[0,0,0],"spectral_radiant_intensity":[50,50,50,50]}]}')
    return text.encode(), sum(g[1] for g in geometries)


def run_scene_json(args):
    """Native scene JSON ingestion: bf200_scene_json_parse (strict reading, every SceneDescription
    check, hierarchy resolution) plus bf200_scene_json_frame (the committed arrays a render takes)
    on one large document, beside the reference's deserialize_scene_description_json (oracle/_ref)
    on the same bytes. Host code on both sides, one thread; both must accept, and the canonical
    bytes of the product are checked against the reference's once, outside the timing."""
    from bf200 import scene_json
    text, triangles = scene_json_document()
    lim = None  # the reference's default limits, as the reference arm below uses
    for _ in range(args.warmup):
        scene_json.SceneJson(text, lim).close()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        doc = scene_json.SceneJson(text, lim)
        doc.frame()
        times.append(time.perf_counter() - t0)
        doc.close()
    reference = None
    ref_path = os.path.join(REPO, "oracle", "_ref", "libbfref.so")
    if os.path.exists(ref_path):
        import ctypes as C
        lib = C.CDLL(ref_path)
        lib.bfref_scene_json_parse_only.argtypes = [C.c_char_p, C.c_uint64]
        lib.bfref_scene_json_parse_only.restype = C.c_int
        ref_times, codes = [], []
        for _ in range(max(1, args.steps)):
            t0 = time.perf_counter()
            codes.append(lib.bfref_scene_json_parse_only(text, len(text)))
            ref_times.append(time.perf_counter() - t0)
        ref_seconds = statistics.median(ref_times)
        lib.bfref_scene_json_canonical.argtypes = [C.c_char_p, C.c_uint64, C.c_void_p, C.c_char_p, C.c_uint64,
                                                   C.POINTER(C.c_uint64), C.c_char_p, C.c_uint64]
        lib.bfref_scene_json_canonical.restype = C.c_int
        out, size, message = C.create_string_buffer(2 * len(text)), C.c_uint64(), C.create_string_buffer(512)
        rc = lib.bfref_scene_json_canonical(text, len(text), None, out, 2 * len(text), C.byref(size), message, 512)
        with scene_json.SceneJson(text, lim) as doc:
            identical = rc == 0 and doc.canonical() == out.raw[:size.value]
        reference = {"mb_per_s": len(text) / ref_seconds / 1e6, "seconds": ref_seconds, "codes": sorted(set(codes)),
                     "identical_canonical_bytes": identical, "kind": "reference"}
    seconds = statistics.median(times)
    line = {"metric": "scene JSON MB/s", "value": len(text) / seconds / 1e6, "unit": "MB/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": seconds * 1000.0, "higher_is_better": True,
            "scaling": "none", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": SCENE_JSON_WORKLOAD, "bytes": len(text), "triangles": triangles, "instances": 16,
                       "host": "one thread"},
            "reference_reader": reference, "gpu_launches": 0}
    if reference is not None:
        line["speedup_vs_reference"] = reference["seconds"] / seconds
    print(json.dumps(line), flush=True)


def run_reference_arm(args, rank, world):
    """The reference's own CPU implementation of the path, on the host cores of rank 0: each step
    traces a bounded random sample of the workload's paths (about --reference-seconds of work; a
    warm-up step traces one path per thread)."""
    if rank != 0:
        return
    ref = CpuReference(args.workload)
    for _ in range(args.warmup):
        ref.run(ref.threads)
    n = ref.sized(args.reference_seconds)
    seconds = [ref.run(n) for _ in range(args.steps)]
    ref.close()
    total = sum(seconds)
    value = n * args.steps / total
    width, height, spp, depth, mis, _ = scenes.WORKLOADS[args.workload]
    sample = ref.describe(n)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "path samples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "width": width, "height": height, "spp": spp, "max_depth": depth,
                   "mis": mis, "sample_per_step": sample},
        "cpu_baseline": {"value": value, "unit": "path samples/s", "cores": ref.threads, "kind": ref.kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "path samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_cuda_arm(args, rank, world):
    """The reference's own CUDA backend on the workload: each step is one
    trace_cuda_wavefront_transport call on a reused workspace over one sample per pixel of the frame
    (2,073,600 paths at 1080p; the reference benchmark's call shape, Benchmarks/Renderer/
    CudaWavefrontTransportBenchmark.cpp:163-393), inputs from the reference's own camera (rays and
    cones) and results back in host memory. bf200_trace_paths_with_cones runs the same inputs the
    same way (host inputs, host results) beside it, and the per-path results of the two are
    compared. Host wall time around each call (each returns after its device work)."""
    if rank != 0:
        return
    import torch
    from oracle.bindings import ReferenceCuda
    builder, options, (width, height, spp) = scenes.build_workload(args.workload)
    ref = ReferenceCuda()
    t0 = time.perf_counter()
    handle = ref.scene(builder)
    ref_setup_s = time.perf_counter() - t0
    stats = ref.stats(handle)
    ctx = runtime.Context(0, path_capacity=args.capacity)
    t0 = time.perf_counter()
    scene = ctx.create_scene(builder)
    bf_setup_s = time.perf_counter() - t0

    def inputs_for(step):
        samples = frame_samples(width, height, step % spp, seed=0)
        return reference_camera_inputs(args.workload, samples, cones=True)

    def reference_call(inputs, cones, results):
        """One reference call. The reference fails a whole batch when any lane fails (its audits,
        WavefrontTransport.cpp:1984-2835); the failing path is then left out and the call repeated,
        so the timed call is the frame's batch without the paths the reference cannot trace."""
        import re
        from oracle.bindings import CheckerError
        dropped = []
        keep = np.arange(len(inputs))
        for _ in range(16):
            try:
                return _attempt(inputs, cones, keep, results, dropped)
            except CheckerError as error:
                found = re.search(r"path slot (\d+)", str(error))
                if found is None or int(found.group(1)) >= len(keep):
                    raise
                dropped.append(int(keep[int(found.group(1))]))
                keep = np.delete(keep, int(found.group(1)))
        raise RuntimeError("the reference CUDA backend failed 16 batches in a row")

    def _attempt(inputs, cones, keep, results, dropped):
        if len(keep) == len(inputs):
            batch_in, batch_cones = inputs, cones
        else:
            batch_in = (abi.PathInput * len(keep))(*[inputs[int(k)] for k in keep])
            batch_cones = cones[keep]
        out, report, ms = ref.trace(handle, batch_in, options, cones=batch_cones, results=results)
        return out, report, ms, keep, list(dropped)

    ref_ms, bf_ms, ref_paths, dropped_total = [], [], 0, 0
    agreement = None
    for step in range(args.warmup + args.steps):
        inputs, cones = inputs_for(step)
        want, ref_report, ms, keep, dropped = reference_call(inputs, cones, results=step == args.warmup)
        if step >= args.warmup:
            dropped_total += len(dropped)
            ref_paths += len(keep)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        got, _, report = ctx.trace_paths_with_cones(scene, inputs, cones, options)
        torch.cuda.synchronize()
        bf = (time.perf_counter() - t0) * 1000.0
        if step >= args.warmup:
            ref_ms.append(ms)
            bf_ms.append(bf)
        if want is not None:
            from helpers import arrays, relative_error
            a, b = arrays(got), arrays(want)
            a = {k: v[keep] for k, v in a.items()}
            ok = a["lane_status"] == 0
            close = (relative_error(a["radiance"], b["radiance"]) <= 1e-5).all(axis=1) & ok
            same = (a["radiance"].view(np.uint32) == b["radiance"].view(np.uint32)).all(axis=1) & ok
            agreement = {"paths": len(inputs), "bit_exact": float(same.mean()), "within_1e-5": float(close.mean()),
                         "same_termination": float(((a["termination"] == b["termination"]) & ok).mean()),
                         "segments_bf200": [int(report.extension_segments), int(report.shadow_segments)],
                         "segments_reference": [int(ref_report.extension_segments), int(ref_report.shadow_segments)]}
    paths = width * height
    value = ref_paths / (sum(ref_ms) / 1000.0)
    bf_value = paths * len(bf_ms) / (sum(bf_ms) / 1000.0)
    scene.close()
    ctx.close()
    ref.destroy(handle)
    line = {
        "impl": "reference-cuda", "metric": METRIC, "value": value, "unit": "path samples/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sum(ref_ms) / len(ref_ms),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "width": width, "height": height, "paths_per_call": paths,
                   "call": "trace_cuda_wavefront_transport, reused workspace, synchronous transfer, host inputs "
                           "and results (one sample per pixel per call, sample index = step)",
                   "mis": scenes.WORKLOADS[args.workload][4], "max_depth": scenes.WORKLOADS[args.workload][3]},
        "reference_setup": {"seconds": ref_setup_s, **stats},
        "bf200_same_inputs": {"value": bf_value, "ms_per_step": sum(bf_ms) / len(bf_ms),
                              "call": "bf200_trace_paths_with_cones, host inputs and results",
                              "scene_create_seconds": bf_setup_s},
        "bf200_over_reference_cuda": bf_value / value,
        "agreement": agreement,
        "reference_failed_paths_left_out": dropped_total,
        "e2e": {"value": value, "unit": "path samples/s", "h2d_bytes_per_step": paths * 80 + paths * 8,
                "d2h_bytes_per_step": paths * C.sizeof(abi.PathResult)},
    }
    print(json.dumps(line), flush=True)


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", default="bf200", choices=["bf200", "reference", "reference-cuda"])
    parser.add_argument("--capacity", type=int, default=1 << 21)
    parser.add_argument("--reference-seconds", type=float, default=4.0)
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--build-mode", choices=["sah", "lbvh"], default="sah",
                        help="BLAS build of the scene: host binned SAH (default) or the device linear BVH")
    parser.add_argument("--spp", type=int, default=0, help="samples per pixel per step (default: the workload's)")
    parser.add_argument("--workload", default=WORKLOAD,
                        choices=sorted(scenes.WORKLOADS) + [BATCH_WORKLOAD, IMPORT_WORKLOAD, REFIT_WORKLOAD,
                                                         SCENE_JSON_WORKLOAD],
                        help="scene and frame (default: the headline Cornell + spheres frame); "
                             f"{BATCH_WORKLOAD}: the 64-scene batch against 64 serial renders; "
                             f"{ADJOINT_WORKLOAD}: the path-replay adjoint; {IMPORT_WORKLOAD}: OBJ ingestion")
    parser.add_argument("--lanes", type=int, default=0, help="batch lanes (0: autotuned)")
    parser.add_argument("--adjoint-pair", action="store_true",
                        help="run the adjoint workload as the forward/backward pair with NCCL reductions "
                             "(always so on more than one GPU)")
    args = parser.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.impl == "reference-cuda":
        run_reference_cuda_arm(args, rank, world)
        return
    if args.workload == IMPORT_WORKLOAD:
        if rank == 0:
            run_mesh_import(args)
        return
    if args.workload == SCENE_JSON_WORKLOAD:
        if rank == 0:
            run_scene_json(args)
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local_rank)
    if args.workload == BATCH_WORKLOAD:
        run_batch(args, torch, rank, world, local_rank)
        return
    if args.workload == ADJOINT_WORKLOAD:
        if world > 1 or args.adjoint_pair:
            run_adjoint_distributed(args, torch, rank, world, local_rank)
        else:
            run_adjoint(args, torch, rank)
        return
    if args.workload == REFIT_WORKLOAD:
        if rank == 0:
            run_refit(args, torch)
        return
    distributed = world > 1
    if distributed:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    builder, options, camera, sensor, (width, height, spp) = workload_setup(args.workload)
    if args.spp > 0:
        spp = args.spp
    pixels = width * height
    paths_per_step = pixels * spp
    ctx = runtime.Context(local_rank, path_capacity=args.capacity)
    ctx.set_build_mode(abi.BUILD_DEVICE_LBVH if args.build_mode == "lbvh" else abi.BUILD_HOST_SAH)
    scene = ctx.create_scene(builder)
    lib = runtime.library()
    film = torch.zeros((height, width, 4), dtype=torch.float32, device="cuda")
    counts = torch.zeros((height, width), dtype=torch.int64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def render_device(step, instrument=False):
        options.instrumentation = 1 if instrument else 0
        f = abi.Film(width, height, 0, 0, film.data_ptr(), C.cast(counts.data_ptr(), C.POINTER(abi.u64)))
        first, _ = multigpu.rank_sample_range(step, rank, world, spp)  # disjoint per rank and step
        request = abi.FilmRequest(C.sizeof(abi.FilmRequest), spp, first, 0, 0)
        report = abi.Report()
        report.struct_size = C.sizeof(abi.Report)
        status = lib.bf200_render_film_device(ctx.handle, scene.handle, C.byref(camera), C.byref(sensor),
                                              C.byref(request), C.byref(options), C.byref(f), C.byref(report))
        if status != 0:
            raise runtime.Bf200Error(status, lib.bf200_context_last_error(ctx.handle).decode())
        if distributed:
            multigpu.reduce_film(film, counts)  # per-GPU films summed (the only exchange of the path)
        return report

    for step in range(args.warmup):
        film.zero_()
        counts.zero_()
        render_device(step)
    torch.cuda.synchronize()

    # timed region: device-resident inputs, K full frames; L2 flushed between frames. Each frame is
    # timed with CUDA events bracketing the whole library call (which returns after its stream has
    # finished), so launch gaps and per-iteration host round trips are inside the measurement.
    reports = []
    step_ms = []
    with ClockSampler(local_rank) as clocks:
        if distributed:
            dist.barrier()
        torch.cuda.synchronize()
        for step in range(args.steps):
            film.zero_()
            counts.zero_()
            flush.fill_(step & 0xFF)
            torch.cuda.synchronize()
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            report = render_device(args.warmup + step)
            stop.record()
            torch.cuda.synchronize()
            reports.append(report)
            step_ms.append(start.elapsed_time(stop))
        torch.cuda.synchronize()
        if distributed:
            dist.barrier()
    total_ms = sum(step_ms)
    # one more frame, untimed, with per-stage CUDA events inside the library (the stage breakdown
    # and the roofline's per-launch times come from it)
    film.zero_()
    counts.zero_()
    flush.fill_(0x5A)
    torch.cuda.synchronize()
    staged = render_device(args.warmup + args.steps, instrument=True)
    if distributed:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = paths_per_step * world * args.steps / (total_ms / 1000.0)
    failed = sum(r.failed_lanes for r in reports)
    launches = sum(r.kernel_launches for r in reports)
    ext = sum(r.extension_segments for r in reports)
    shadow = sum(r.shadow_segments for r in reports)
    iterations = sum(r.iterations for r in reports)
    stage = {"regenerate": staged.regenerate_milliseconds, "trace": staged.intersect_milliseconds,
             "shade": staged.shade_milliseconds, "occlude": staged.occlude_milliseconds,
             "film": staged.film_milliseconds}

    # e2e: the public C-ABI call with host film buffers (copies in the timed region)
    options.instrumentation = 0
    host_film = np.zeros((height, width, 4), np.float32)
    host_counts = np.zeros((height, width), np.uint64)
    h2d = host_film.nbytes + host_counts.nbytes
    e2e_ms = []
    # one untimed call first: it grows the context's host-film staging buffers once
    ctx.render_film(scene, camera, sensor, options, spp, seed=0, first_sample=(999 * world + rank) * spp,
                    film=(host_film, host_counts))
    for step in range(max(1, min(args.steps, 3))):
        host_film[:] = 0
        host_counts[:] = 0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.render_film(scene, camera, sensor, options, spp, seed=0,
                        first_sample=(1000 + step * world + rank) * spp, film=(host_film, host_counts))
        e2e_ms.append((time.perf_counter() - t0) * 1000.0)
    e2e_total = sum(e2e_ms)
    if distributed:
        t = torch.tensor([e2e_total], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = paths_per_step * world * len(e2e_ms) / (e2e_total / 1000.0)

    # roofline of the dominant stage: algorithmic bytes per launch / average launch time (CUDA events
    # around the stage's launches on the wavefront stream, summed by the library per iteration)
    peak, peak_kind = measured_peaks()
    dominant = max(("trace", "shade", "occlude"), key=lambda k: stage[k])
    per_launch_ms = stage[dominant] / max(1, staged.iterations)
    units = staged.shadow_segments if dominant == "occlude" else staged.extension_segments
    bytes_per_launch = STAGE_BYTES_PER_UNIT[dominant] * units / max(1, staged.iterations)
    achieved = bytes_per_launch / (per_launch_ms / 1000.0) / 1e9
    units_per_launch = units / max(1, staged.iterations)
    traffic_per_unit = MEASURED_TRAFFIC_PER_UNIT.get(args.workload, {}).get(dominant)
    traffic = traffic_per_unit * units_per_launch if traffic_per_unit is not None else None
    whole_bytes = (CAMERA_RAY_BYTES * paths_per_step * args.steps + EXTENSION_SEGMENT_BYTES * ext +
                   SHADOW_SEGMENT_BYTES * shadow + FILM_SAMPLE_BYTES * paths_per_step * args.steps)

    line = {
        "metric": METRIC, "value": value, "unit": "path samples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "width": width, "height": height, "spp": spp, "max_depth": 16,
                   "mis": "power", "paths_per_step_per_gpu": paths_per_step, "path_capacity": args.capacity,
                   "l2": "flushed between steps (256 MiB write); path state > L2",
                   "parallelism": f"sample-partitioned x{world}" if world > 1 else "single GPU",
                   "blas_build": "device linear BVH" if args.build_mode == "lbvh" else "host binned SAH"},
        "rays_per_s": (ext + shadow) / (total_ms / 1000.0) * (world if distributed else 1),
        "segments": {"extension": ext, "shadow": shadow, "iterations": iterations},
        "stage_ms_one_frame": stage, "failed_lanes": failed,
        "first_failure": next(({"status": r.first_failure_status, "path": r.first_failure_path}
                               for r in reports if r.failed_lanes), None),
        "clocks": clocks.summary(),
        "e2e": {"value": e2e_value, "unit": "path samples/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": h2d},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": STAGE_KERNELS[dominant], "achieved": achieved, "peak": peak,
                     "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per unit, scaled to a launch"
                     if traffic is not None else None,
                     "algorithmic_bytes_per_launch": bytes_per_launch, "peak_source": peak_kind,
                     "whole_path_algorithmic_gbs": whole_bytes / (total_ms / 1000.0) / 1e9},
    }
    scene.close()
    ctx.close()
    if rank == 0 and not args.no_cpu_baseline and args.workload in scenes.WORKLOADS:
        rate, threads, kind, sample, _, _ = cpu_sample_rate(args.workload, target_seconds=args.reference_seconds)
        line["cpu_baseline"] = {"value": rate, "unit": "path samples/s", "cores": threads, "kind": kind,
                                "sample": sample}
    if distributed:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
