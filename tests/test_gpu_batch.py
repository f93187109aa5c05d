"""Film batches (bf200_render_films_device): every job's film must equal, bit for bit, the film of
the same job rendered alone with bf200_render_film_device, for any lane count."""
import os

import numpy as np
import pytest

from bf200 import abi, runtime, scenes
from helpers import sensor_from_golden

pytestmark = pytest.mark.gpu


def _jobs():
    # (workload, width, height, spp, seed, first sample, precision, max depth, sampler)
    return [
        ("cornell_plain_64", 64, 64, 4, 0, 0, 0, 8, 0),
        ("cornell_spheres_256", 48, 40, 3, 7, 5, 1, 16, 0),
        ("cornell_plain_64", 96, 64, 2, 3, 100, 1, 4, 1),
        ("cornell_spheres_256", 32, 32, 9, 11, 0, 0, 6, 1),
        ("cornell_plain_64", 16, 24, 1, 0, 9, 0, 12, 0),
        ("cornell_spheres_256", 80, 56, 2, 5, 2, 0, 16, 0),
        ("cornell_plain_64", 40, 40, 0, 0, 0, 0, 8, 0),  # no samples: the film stays untouched
    ]


@pytest.fixture(scope="module")
def setup():
    import torch

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cornell_spheres_256.npz"))
    sensor = sensor_from_golden(g)
    with runtime.Context(0, path_capacity=1 << 16) as ctx:
        built = {}
        for name in ("cornell_plain_64", "cornell_spheres_256"):
            builder, _, _ = scenes.build_workload(name)
            built[name] = (builder, ctx.create_scene(builder))
        yield torch, ctx, built, sensor
        for _, scene in built.values():
            scene.close()


def _films(torch, spec):
    _, w, h, _, _, _, precision, _, _ = spec
    sums = torch.zeros((h, w, 4 if precision == 0 else 8), dtype=torch.float32 if precision == 0 else torch.float64,
                       device="cuda")
    counts = torch.zeros((h, w), dtype=torch.int64, device="cuda")
    return sums, counts


@pytest.mark.parametrize("lanes", [0, 1, 3, 16])
def test_batch_films_equal_single_renders(setup, lanes):
    torch, ctx, built, sensor = setup
    specs = _jobs()
    jobs, batch_films, single_films = [], [], []
    for spec in specs:
        name, w, h, spp, seed, first, precision, depth, sampler = spec
        options = abi.default_options(mis="power" if "spheres" in name else "balance", max_depth=depth)
        options.sampler = sampler
        cam = runtime.camera_create(*scenes.camera_frame_inputs(), w, h, scenes.CAMERA_VFOV, scenes.PATH_TIME)
        scene = built[name][1]
        sums, counts = _films(torch, spec)
        single_sums, single_counts = _films(torch, spec)
        ctx.render_film_device(scene, cam, sensor, options, spp, seed, first, precision, single_sums.data_ptr(),
                               single_counts.data_ptr())
        jobs.append((scene, cam, sensor, options, spp, seed, first, precision, sums.data_ptr(), counts.data_ptr()))
        batch_films.append((sums, counts))
        single_films.append((single_sums, single_counts))
    reports = ctx.render_films_device(jobs, lanes=lanes)
    torch.cuda.synchronize()
    for k, spec in enumerate(specs):
        (bs, bc), (ss, sc) = batch_films[k], single_films[k]
        assert torch.equal(bc, sc), f"job {k}: sample counts differ"
        assert (bc == spec[3]).all()
        assert np.array_equal(bs.cpu().numpy().view(np.uint8), ss.cpu().numpy().view(np.uint8)), f"job {k} differs"
        w, h, spp = spec[1], spec[2], spec[3]
        assert reports[k].path_count == w * h * spp and reports[k].failed_lanes == 0


def test_measured_lane_count_keeps_every_film(setup):
    """A batch of 40 jobs with lanes = 0 measures 2, 4 and 8 lanes on its first 24 jobs, keeps the
    fastest for the other 16 and for the next batch of the same job size; every film still equals
    its single render."""
    torch, ctx, built, sensor = setup
    name = "cornell_plain_64"
    scene = built[name][1]
    options = abi.default_options(mis="balance", max_depth=6)
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), 40, 32, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    spec = (name, 40, 32, 2, 0, 0, 0, 6, 0)
    for batch in range(2):
        jobs, films = [], []
        for k in range(40):
            sums, counts = _films(torch, spec)
            jobs.append((scene, cam, sensor, options, 2, 100 * batch + k, 0, 0, sums.data_ptr(), counts.data_ptr()))
            films.append((sums, counts, 100 * batch + k))
        ctx.render_films_device(jobs, lanes=0)
        torch.cuda.synchronize()
        assert ctx.batch_lanes() in (2, 4, 8)
        for sums, counts, seed in films[::7]:
            single_sums, single_counts = _films(torch, spec)
            ctx.render_film_device(scene, cam, sensor, options, 2, seed, 0, 0, single_sums.data_ptr(),
                                   single_counts.data_ptr())
            assert torch.equal(counts, single_counts)
            assert np.array_equal(sums.cpu().numpy().view(np.uint8), single_sums.cpu().numpy().view(np.uint8))


def test_batch_rejects_a_foreign_scene(setup):
    torch, ctx, built, sensor = setup
    builder = built["cornell_plain_64"][0]
    with runtime.Context(0, path_capacity=1 << 12) as other:
        foreign = other.create_scene(builder)
        cam = runtime.camera_create(*scenes.camera_frame_inputs(), 8, 8, scenes.CAMERA_VFOV, scenes.PATH_TIME)
        sums, counts = _films(torch, ("", 8, 8, 1, 0, 0, 0, 8, 0))
        options = abi.default_options(mis="balance", max_depth=8)
        with pytest.raises(runtime.Bf200Error) as info:
            ctx.render_films_device([(foreign, cam, sensor, options, 1, 0, 0, 0, sums.data_ptr(), counts.data_ptr())])
        assert info.value.status == 4
        foreign.close()
