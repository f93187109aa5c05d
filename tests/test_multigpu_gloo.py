"""The multi-GPU frame logic with two gloo ranks on CPU: each rank renders its sample range
(bf200.multigpu.rank_sample_range) with the oracle, the films are summed with
bf200.multigpu.reduce_film, and the result must equal the film of the whole range rendered in one
process (counts exactly; compensated-double sums to summation-order rounding)."""
import os
import socket

import numpy as np
import pytest

from bf200 import abi, multigpu, runtime, scenes

WIDTH, HEIGHT, SPP = 8, 8, 2


def _film(first, count):
    from helpers import arrays, sensor_from_golden
    from oracle.bindings import Oracle

    oracle = Oracle()
    builder, options, _ = scenes.build_workload("cornell_plain_64")
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cornell_plain_64.npz"))
    sensor = sensor_from_golden(g)
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), WIDTH, HEIGHT, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    n = WIDTH * HEIGHT * count
    samples = (abi.SampleIndex * n)()
    k = 0
    for s in range(first, first + count):
        for y in range(HEIGHT):
            for x in range(WIDTH):
                samples[k].pixel_x, samples[k].pixel_y, samples[k].sample_index = x, y, s
                k += 1
    rays = oracle.camera_rays(cam, samples)
    inputs = (abi.PathInput * n)()
    for i in range(n):
        inputs[i].primary_ray, inputs[i].sample = rays[i], samples[i]
    handle = oracle.scene(builder)
    results, failures = oracle.trace(handle, inputs, options, threads=2)
    oracle.destroy(handle)
    assert failures == 0
    return oracle.film(arrays(results)["radiance"], samples, sensor, WIDTH, HEIGHT, 1)


def _rank(rank, world, port, step, queue):
    import sys

    import torch
    import torch.distributed as dist

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        first, end = multigpu.rank_sample_range(step, rank, world, SPP)
        sums, counts = _film(first, end - first)
        sums_t = torch.from_numpy(sums)
        counts_t = torch.from_numpy(counts.astype(np.int64))
        multigpu.reduce_film(sums_t, counts_t)
        if rank == 0:
            queue.put((sums_t.numpy(), counts_t.numpy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_batch_shards_are_disjoint_complete_and_balanced():
    from bf200 import multigpu, scenes
    paths = []
    for seed in range(64):
        _, _, (w, h, spp) = scenes.batch_job(seed)
        paths.append(w * h * spp)
    for world in (1, 2, 4, 8):
        shards = [multigpu.batch_shard(paths, r, world) for r in range(world)]
        every = sorted(j for shard in shards for j in shard)
        assert every == list(range(64))
        loads = [sum(paths[j] for j in shard) for shard in shards]
        assert max(loads) - min(loads) <= max(paths)  # greedy largest-first: within one job


def test_sample_ranges_are_disjoint_and_complete():
    world, spp = 4, 3
    covered = []
    for step in range(2):
        for rank in range(world):
            first, end = multigpu.rank_sample_range(step, rank, world, spp)
            covered.extend(range(first, end))
    assert sorted(covered) == list(range(2 * world * spp))


def test_two_rank_film_reduce_equals_single_process_film():
    import torch.multiprocessing as mp

    world, step = 2, 1
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, step, queue)) for r in range(world)]
    for p in procs:
        p.start()
    import queue as queue_module

    result = None
    try:
        for _ in range(600):
            try:
                result = queue.get(timeout=0.5)
                break
            except queue_module.Empty:
                if any(p.exitcode not in (None, 0) for p in procs):
                    break
    finally:
        for p in procs:
            p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs) and result is not None
    reduced_sums, reduced_counts = result
    first, _ = multigpu.rank_sample_range(step, 0, world, SPP)
    sums, counts = _film(first, world * SPP)
    expected = sums
    assert (reduced_counts == counts.astype(np.int64)).all()
    assert (reduced_counts == world * SPP).all()
    np.testing.assert_allclose(reduced_sums, expected, rtol=1e-12, atol=1e-300)
