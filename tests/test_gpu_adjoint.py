"""Path-replay adjoint of the film render (bf200_render_adjoint_device).

With the sampled directions held fixed and Russian roulette off, every contribution of a path is
linear in each closure weight and in the emitted radiance, so those gradients are the exact
derivatives of the rendered loss. They are compared with central finite differences of the same
render (same sample indices), with a relative step of 1e-3 on the float32 parameter:
tolerance 2e-3 of the finite difference, plus 1e-4 of the largest gradient tested. They are also
compared with a float64 differentiation of the same paths on the CPU (within 1 %) and with finite
differences of the oracle's films (the CPU restatement of the reference
transport). There the tolerance is 3 %, because up to 1 % of paths may take a different route on
the device (the sine/cosine rounding note of the parity tests).

The roughness gradient is the detached estimator: sampling densities and MIS weights are held
fixed. It is unbiased for the derivative of the expected loss but differs from a finite difference
sample by sample. It is compared with finite differences over several seeds: the mean difference
must lie within four standard errors, plus 3 % of the finite difference.
"""
import copy
import os

import numpy as np
import pytest

from bf200 import abi, runtime, scenes
from helpers import arrays, sensor_from_golden
from oracle.bindings import Oracle

pytestmark = pytest.mark.gpu

WIDTH, HEIGHT, SPP, DEPTH, SEED = 24, 20, 4, 6, 11
WHITE, RED, GREEN, LIGHT, CONDUCTOR, DIELECTRIC = range(6)


def transport_options():
    return abi.default_options(mis="power", max_depth=DEPTH, roulette=False)


def changed(builder, material, lane=None, weight=None, alpha=None, emission=None):
    """Copy of a scene builder with one material's closure weight lane, GGX roughness (both axes)
    or emission (all lanes) replaced by a float32 value."""
    b = copy.copy(builder)
    b.materials = list(builder.materials)
    closures, emitted, frame = b.materials[material]
    kind, lobes, w, params = closures[0]
    w, params, emitted = list(w), list(params), list(emitted)
    if weight is not None:
        w[lane] = np.float32(weight)
    if alpha is not None:
        axes = (8, 9) if kind == abi.CLOSURE_ROUGH_CONDUCTOR else (2, 3)
        for a in axes:
            params[a] = np.float32(alpha)
    if emission is not None:
        emitted = [np.float32(emission)] * 4
    b.materials[material] = ([(kind, lobes, w, params)] + closures[1:], emitted, frame)
    return b


def film_loss(sums, target):
    image = (sums[..., :3] + sums[..., 4:7]) / (sums[..., 3:4] + sums[..., 7:8])
    return float(((image - target) ** 2).sum())


@pytest.fixture(scope="module")
def setup():
    import torch

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cornell_spheres_256.npz"))
    sensor = sensor_from_golden(g)
    builder = scenes.cornell_box(scenes.SceneBuilder(), with_spheres=True)
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), WIDTH, HEIGHT, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    target = np.random.default_rng(7).uniform(0.0, 0.3, (HEIGHT, WIDTH, 3)).astype(np.float32)
    with runtime.Context(0, path_capacity=1 << 16) as ctx:
        yield torch, ctx, builder, cam, sensor, target


def gpu_loss(setup, builder, spp=SPP, seed=SEED):
    torch, ctx, _, cam, sensor, target = setup
    scene = ctx.create_scene(builder)
    sums = torch.zeros((HEIGHT, WIDTH, 8), dtype=torch.float64, device="cuda")
    counts = torch.zeros((HEIGHT, WIDTH), dtype=torch.int64, device="cuda")
    ctx.render_film_device(scene, cam, sensor, transport_options(), spp, seed, 0, 1, sums.data_ptr(),
                           counts.data_ptr())
    scene.close()
    return film_loss(sums.cpu().numpy(), target)


def gpu_adjoint(setup, builder, spp=SPP, seed=SEED):
    torch, ctx, _, cam, sensor, target = setup
    scene = ctx.create_scene(builder)
    sums = torch.full((HEIGHT, WIDTH, 8), 3.0, dtype=torch.float64, device="cuda")  # cleared by the call
    counts = torch.zeros((HEIGHT, WIDTH), dtype=torch.int64, device="cuda")
    grads = torch.zeros((len(builder.materials), 8), dtype=torch.float64, device="cuda")
    emission = torch.zeros(1, dtype=torch.float64, device="cuda")
    tgt = torch.tensor(target, device="cuda")
    loss, report = ctx.render_adjoint_device(scene, cam, sensor, transport_options(), spp, seed, 0, 1,
                                             sums.data_ptr(), counts.data_ptr(), tgt.data_ptr(), grads.data_ptr(),
                                             emission.data_ptr())
    scene.close()
    # a failed path (a reference-inherent numerical failure, about 1 in 10^5 here) is left out of
    # the film and of the gradients
    paths = WIDTH * HEIGHT * spp
    assert report.path_count == paths and report.failed_lanes <= max(1, paths // 10000)
    assert int(counts.sum()) == paths - report.failed_lanes
    return loss, grads.cpu().numpy(), float(emission.cpu()[0]), sums.cpu().numpy()


def steps(value, h):
    """Central difference points value (1 -+ h) as float32, and their spacing."""
    lo, hi = np.float32(value * (1.0 - h)), np.float32(value * (1.0 + h))
    return lo, hi, float(hi) - float(lo)


def derivative(f, value, h):
    """d f / d value by finite differences with relative step h. A closure weight is a reflectance,
    refused above 1 as ClosureSet refuses it, so where value (1 + h) would pass 1 the derivative is
    the second-order one-sided stencil through value, value (1 - h) and value (1 - 2h): the
    derivative at value of the quadratic through the three float32 points (a first-order one-sided
    difference would carry an O(h) error of about 1 % on the multi-bounce dielectric)."""
    lo, hi, d = steps(value, h)
    if float(hi) <= 1.0 or value > 1.0:
        return (f(hi) - f(lo)) / d
    x = [float(np.float32(value * (1.0 - k * h))) for k in range(3)]
    y = [f(np.float32(v)) for v in x]
    return (y[0] * (2.0 * x[0] - x[1] - x[2]) / ((x[0] - x[1]) * (x[0] - x[2])) +
            y[1] * (x[0] - x[2]) / ((x[1] - x[0]) * (x[1] - x[2])) +
            y[2] * (x[0] - x[1]) / ((x[2] - x[0]) * (x[2] - x[1])))


# (material, lane). Lane 3 of the packet (759.5 nm) barely reaches the CIE sensor: a 1e-3 change
# of its weight moves the film by about as much as float32 rounding does, so it is not tested.
WEIGHTS = [(WHITE, 0), (WHITE, 2), (RED, 1), (GREEN, 2), (CONDUCTOR, 0), (DIELECTRIC, 1)]


def test_weight_and_emission_gradients_match_finite_differences(setup):
    _, _, builder, _, _, target = setup
    loss, grads, emission, sums = gpu_adjoint(setup, builder)
    assert abs(loss - film_loss(sums, target)) <= 1e-9 * loss
    # the image is linear in the emitted radiance (no environment): dLoss/dk = sum 2 (I - T) I
    image = (sums[..., :3] + sums[..., 4:7]) / (sums[..., 3:4] + sums[..., 7:8])
    assert abs(emission - float((2.0 * (image - target) * image).sum())) <= 1e-4 * abs(emission)
    scale = max(abs(grads[m, l]) for m, l in WEIGHTS)
    checks = []
    for m, l in WEIGHTS:
        w = float(builder.materials[m][0][0][2][l])
        fd = derivative(lambda v: gpu_loss(setup, changed(builder, m, l, weight=v)), w, 1e-3)
        print(f"weight ({m}, {l}): adjoint {grads[m, l]:.6g}, finite difference {fd:.6g}")
        checks.append((m, l, grads[m, l], fd))
    for m, l, g, fd in checks:
        assert abs(g - fd) <= 2e-3 * abs(fd) + 1e-4 * scale, (m, l, g, fd)
    e = float(builder.materials[LIGHT][1][0])
    fd = e * derivative(lambda v: gpu_loss(setup, changed(builder, LIGHT, emission=v)), e, 1e-3)
    assert abs(emission - fd) <= 2e-3 * abs(fd), (emission, fd)


def oracle_loss(oracle, builder, cam, sensor, target):
    px, py, s = np.meshgrid(np.arange(WIDTH), np.arange(HEIGHT), np.arange(SPP), indexing="ij")
    order = np.lexsort((px.ravel(), py.ravel(), s.ravel()))
    px, py, s = px.ravel()[order], py.ravel()[order], s.ravel()[order]
    samples = (abi.SampleIndex * len(px))()
    for k in range(len(px)):
        samples[k].pixel_x, samples[k].pixel_y = int(px[k]), int(py[k])
        samples[k].sample_index, samples[k].seed = int(s[k]), SEED
    rays = oracle.camera_rays(cam, samples)
    inputs = (abi.PathInput * len(px))()
    for k in range(len(px)):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    handle = oracle.scene(builder)
    results, failures = oracle.trace(handle, inputs, transport_options())
    oracle.destroy(handle)
    assert failures == 0
    film, _ = oracle.film(arrays(results)["radiance"], samples, sensor, WIDTH, HEIGHT, 1)  # compensated sums
    image = film[..., :3] / film[..., 3:4]
    return float(((image - target) ** 2).sum())


def test_gradients_match_the_float64_path_replay(setup):
    """The adjoint's weight and emission gradients against a float64 computation on the CPU along
    the same paths (the oracle's float transport with the device's sine/cosine rounding): every
    radiance contribution of every path is recorded and differentiated with respect to the closure
    weights and the emitter scale in double precision (bfo_weight_gradients), with dLoss/dL per
    path from the device film's image and the film's linear spectrum-to-rgb map. Within 1 %."""
    torch, ctx, builder, cam, sensor, target = setup
    loss, grads, emission, sums = gpu_adjoint(setup, builder)
    image = (sums[..., :3] + sums[..., 4:7]) / (sums[..., 3:4] + sums[..., 7:8])
    weight = sums[..., 3] + sums[..., 7]
    oracle = Oracle(device_trig=True)
    # the film's map from a sample's 4 radiance lanes to its rgb (linear: one film per unit lane)
    one = (abi.SampleIndex * 1)()
    basis = np.zeros((4, 3))
    for lane in range(4):
        radiance = np.zeros((1, 4), np.float32)
        radiance[0, lane] = 1.0
        film, _ = oracle.film(radiance, one, sensor, 1, 1, 1)
        basis[lane] = film[0, 0, :3]
    probe = np.array([[0.3, 1.7, 0.2, 2.5]], np.float32)
    film, _ = oracle.film(probe, one, sensor, 1, 1, 1)
    assert np.allclose(film[0, 0, :3], probe[0].astype(np.float64) @ basis, rtol=1e-6)
    px, py, s = np.meshgrid(np.arange(WIDTH), np.arange(HEIGHT), np.arange(SPP), indexing="ij")
    px, py, s = px.ravel(), py.ravel(), s.ravel()
    samples = (abi.SampleIndex * len(px))()
    for k in range(len(px)):
        samples[k].pixel_x, samples[k].pixel_y = int(px[k]), int(py[k])
        samples[k].sample_index, samples[k].seed = int(s[k]), SEED
    rays = oracle.camera_rays(cam, samples)
    inputs = (abi.PathInput * len(px))()
    for k in range(len(px)):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    d_image = 2.0 * (image - target) / weight[..., None]  # dLoss / d(sample rgb), weight-1 samples
    path_adjoint = d_image[py, px] @ basis.T
    handle = oracle.scene(builder)
    g64, e64, failures = oracle.weight_gradients(handle, inputs, transport_options(), path_adjoint,
                                                 len(builder.materials))
    oracle.destroy(handle)
    assert failures <= max(1, len(px) // 10000)
    scale = max(abs(g64[m, l]) for m, l in WEIGHTS)
    for m, l in WEIGHTS:
        print(f"weight ({m}, {l}): adjoint {grads[m, l]:.8g}, float64 replay {g64[m, l]:.8g}")
        assert abs(grads[m, l] - g64[m, l]) <= 1e-2 * abs(g64[m, l]) + 1e-5 * scale, (m, l, grads[m, l], g64[m, l])
    print(f"emission: adjoint {emission:.8g}, float64 replay {e64:.8g}")
    assert abs(emission - e64) <= 1e-2 * abs(e64)


def test_gradients_match_oracle_finite_differences(setup):
    _, _, builder, cam, sensor, target = setup
    oracle = Oracle(device_trig=True)
    _, grads, emission, _ = gpu_adjoint(setup, builder)
    for m, l in [(WHITE, 1), (RED, 0)]:
        w = float(builder.materials[m][0][0][2][l])
        fd = derivative(lambda v: oracle_loss(oracle, changed(builder, m, l, weight=v), cam, sensor, target), w, 1e-3)
        assert abs(grads[m, l] - fd) <= 0.03 * abs(fd), (m, l, grads[m, l], fd)
    e = float(builder.materials[LIGHT][1][0])
    fd = e * derivative(lambda v: oracle_loss(oracle, changed(builder, LIGHT, emission=v), cam, sensor, target), e,
                        1e-3)
    assert abs(emission - fd) <= 0.03 * abs(fd), (emission, fd)


def test_roughness_gradient_agrees_with_finite_differences_on_average(setup):
    """Conductor at alpha 0.2 and, with alpha raised from 0.05 to 0.3, the dielectric (at 0.05 a
    finite difference is dominated by reflect/transmit choices that flip under the step). Relative
    step 5e-2: the finite difference's flip noise shrinks with the step, its bias grows as its
    square (about 3e-3 here)."""
    _, _, builder, _, _, _ = setup
    spp, seeds = 128, range(100, 116)
    rough_glass = changed(builder, DIELECTRIC, alpha=0.3)
    for m, base, axis, required in [(CONDUCTOR, builder, 8, True), (DIELECTRIC, rough_glass, 2, False)]:
        alpha = float(base.materials[m][0][0][3][axis])
        lo, hi, da = steps(alpha, 5e-2)
        up, down = changed(base, m, alpha=hi), changed(base, m, alpha=lo)
        diffs, fds = [], []
        for seed in seeds:
            _, grads, _, _ = gpu_adjoint(setup, base, spp, seed)
            fd = (gpu_loss(setup, up, spp, seed) - gpu_loss(setup, down, spp, seed)) / da
            diffs.append(grads[m, 4] + grads[m, 5] - fd)
            fds.append(fd)
        mean_fd = float(np.mean(fds))
        stderr = float(np.std(diffs, ddof=1) / np.sqrt(len(diffs)))
        fd_stderr = float(np.std(fds, ddof=1) / np.sqrt(len(fds)))
        print(f"material {m}: adjoint - fd = {np.mean(diffs):.4g} +- {stderr:.3g}, fd {mean_fd:.4g} +- {fd_stderr:.3g}")
        assert abs(np.mean(diffs)) <= 4.0 * stderr + 0.03 * abs(mean_fd)
        if required:  # the comparison has a gradient well above its noise
            assert abs(mean_fd) > 8.0 * stderr


def test_basis_coefficient_gradients_of_the_adjoint_workload(setup):
    """The adjoint workload's parameters (albedo = 8 spectral basis coefficients per material,
    light radiance scale) at 32 x 32 x 4 spp: the per-lane gradients projected on the basis match
    central finite differences of the coefficients (relative step 1e-3, same samples)."""
    torch, ctx, _, _, sensor, _ = setup
    width = height = 32
    params = scenes.adjoint_parameters()
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    options = abi.default_options(mis="power", max_depth=8, roulette=False)
    target = torch.rand((height, width, 3), generator=torch.Generator().manual_seed(3)).mul_(0.3).cuda()

    def render(p, adjoint):
        builder = scenes.adjoint_icosphere(scenes.SceneBuilder(), p, subdivisions=4)
        scene = ctx.create_scene(builder)
        sums = torch.zeros((height, width, 8), dtype=torch.float64, device="cuda")
        counts = torch.zeros((height, width), dtype=torch.int64, device="cuda")
        grads = torch.zeros((len(builder.materials), 8), dtype=torch.float64, device="cuda")
        emission = torch.zeros(1, dtype=torch.float64, device="cuda")
        if adjoint:
            ctx.render_adjoint_device(scene, cam, sensor, options, 4, 5, 0, 1, sums.data_ptr(), counts.data_ptr(),
                                      target.data_ptr(), grads.data_ptr(), emission.data_ptr())
        else:
            ctx.render_film_device(scene, cam, sensor, options, 4, 5, 0, 1, sums.data_ptr(), counts.data_ptr())
        scene.close()
        loss = film_loss(sums.cpu().numpy(), target.cpu().numpy())
        return loss, scenes.basis_gradients(grads.cpu().numpy(), builder.nanometers), float(emission.cpu()[0])

    _, basis, light = render(params, True)
    for row, k in [(0, 1), (3, 4), (1, 4)]:  # (white, 427 nm), (icosphere, 629 nm), (red, 629 nm)
        h = 1e-3 * params["albedo"][row, k]
        up, down = copy.deepcopy(params), copy.deepcopy(params)
        up["albedo"][row, k] += h
        down["albedo"][row, k] -= h
        fd = (render(up, False)[0] - render(down, False)[0]) / (2.0 * h)
        print(f"albedo ({row}, {k}): adjoint {basis[row, k]:.6g}, finite difference {fd:.6g}")
        assert abs(basis[row, k] - fd) <= 5e-3 * abs(fd) + 1e-4 * np.abs(basis).max()
    up, down = dict(params, light_scale=1.001), dict(params, light_scale=0.999)
    fd = (render(up, False)[0] - render(down, False)[0]) / 0.002
    assert abs(light - fd) <= 5e-3 * abs(fd), (light, fd)


def test_forward_backward_pair_matches_the_loss_call(setup):
    """Forward (bf200_render_film_device), dLoss/d(image) computed by the caller, backward
    (bf200_render_backward_device): the same gradients as the one-call loss mode, also for a film
    of several chunks (512 x 512 x 300 spp is 78.6 M paths, more than one 64 M-path chunk)."""
    torch, ctx, builder, cam, sensor, target = setup
    scene = ctx.create_scene(builder)
    for width, height, spp in [(WIDTH, HEIGHT, SPP), (512, 512, 300)]:
        camera = runtime.camera_create(*scenes.camera_frame_inputs(), width, height, scenes.CAMERA_VFOV,
                                       scenes.PATH_TIME)
        tgt = torch.rand((height, width, 3), generator=torch.Generator().manual_seed(5)).mul_(0.3).cuda()
        sums = torch.zeros((height, width, 8), dtype=torch.float64, device="cuda")
        counts = torch.zeros((height, width), dtype=torch.int64, device="cuda")
        one = torch.zeros((len(builder.materials), 8), dtype=torch.float64, device="cuda")
        one_e = torch.zeros(1, dtype=torch.float64, device="cuda")
        loss, _ = ctx.render_adjoint_device(scene, camera, sensor, transport_options(), spp, SEED, 0, 1,
                                            sums.data_ptr(), counts.data_ptr(), tgt.data_ptr(), one.data_ptr(),
                                            one_e.data_ptr())
        sums.zero_()
        counts.zero_()
        ctx.render_film_device(scene, camera, sensor, transport_options(), spp, SEED, 0, 1, sums.data_ptr(),
                               counts.data_ptr())
        image = (sums[..., :3] + sums[..., 4:7]) / (sums[..., 3:4] + sums[..., 7:8])
        assert abs(float(((image - tgt.double()) ** 2).sum()) - loss) <= 1e-9 * loss
        image_adjoint = (2.0 * (image - tgt.double())).float().contiguous()
        two = torch.zeros_like(one)
        two_e = torch.zeros_like(one_e)
        report = ctx.render_backward_device(scene, camera, sensor, transport_options(), spp, SEED, 0, 1,
                                            sums.data_ptr(), counts.data_ptr(), image_adjoint.data_ptr(),
                                            two.data_ptr(), two_e.data_ptr())
        assert report.path_count == width * height * spp
        a, b = one.cpu().numpy(), two.cpu().numpy()
        assert np.allclose(a, b, rtol=1e-5, atol=1e-7 * np.abs(a).max()), (a, b)
        assert abs(float(one_e.cpu()[0]) - float(two_e.cpu()[0])) <= 1e-5 * abs(float(one_e.cpu()[0]))
    scene.close()


def test_film_is_the_calls_render(setup):
    _, _, builder, _, _, _ = setup
    first = gpu_adjoint(setup, builder)
    second = gpu_adjoint(setup, builder)
    # the film is bit-identical; the loss and the gradients are float64 sums by atomics in no
    # fixed order
    assert np.array_equal(first[3], second[3]) and abs(first[0] - second[0]) <= 1e-12 * abs(first[0])
    assert np.allclose(first[1], second[1], rtol=1e-9, atol=0.0)


def test_too_many_materials_is_rejected(setup):
    torch, ctx, builder, cam, sensor, target = setup
    b = copy.copy(builder)
    b.materials = list(builder.materials) + [builder.materials[WHITE]] * 60
    scene = ctx.create_scene(b)
    sums = torch.zeros((HEIGHT, WIDTH, 8), dtype=torch.float64, device="cuda")
    counts = torch.zeros((HEIGHT, WIDTH), dtype=torch.int64, device="cuda")
    grads = torch.zeros((len(b.materials), 8), dtype=torch.float64, device="cuda")
    tgt = torch.tensor(target, device="cuda")
    with pytest.raises(runtime.Bf200Error) as info:
        ctx.render_adjoint_device(scene, cam, sensor, transport_options(), 1, 0, 0, 1, sums.data_ptr(),
                                  counts.data_ptr(), tgt.data_ptr(), grads.data_ptr(), grads.data_ptr())
    scene.close()
    assert info.value.status == 5  # OUT_OF_RANGE
