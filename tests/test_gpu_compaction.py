"""The wavefront's route compaction on the device (bf200_compact_routes_device) against the stable
order that the reference's queue compaction keeps (WavefrontQueueCompaction.hpp: the slots of a
route appended in increasing slot order): every route's queue equals a stable sort of the slots by
key, keys without a route are left out, and the offsets are the routes' prefix counts. Sizes cross
the 4,096-slot tile and 32-slot warp boundaries; key mixes run from all-none to one route only."""
import numpy as np
import pytest
import torch

from bf200 import runtime

pytestmark = pytest.mark.gpu

SIZES = [0, 1, 31, 32, 33, 4095, 4096, 4097, 100003, (1 << 21) + 3]


def keys_for(n, routes, mix, rng):
    if mix == "uniform":
        k = rng.integers(0, routes + 1, n)
        k[k == routes] = 0xFF
    elif mix == "none":
        k = np.full(n, 0xFF)
    elif mix == "one":
        k = np.full(n, routes - 1)
    else:  # runs: long stretches of one key, as a sorted wavefront would have
        k = np.repeat(rng.integers(0, routes + 1, n // 97 + 1), 97)[:n]
        k[k == routes] = 0xFF
    return k.astype(np.uint8)


@pytest.mark.parametrize("routes", [1, 2, 4])
@pytest.mark.parametrize("mix", ["uniform", "none", "one", "runs"])
def test_route_queues_are_stable_compactions(routes, mix):
    rng = np.random.default_rng(routes * 7 + len(mix))
    with runtime.Context(0, path_capacity=1 << 12) as ctx:
        for n in SIZES:
            keys = keys_for(n, routes, mix, rng)
            d_keys = torch.from_numpy(keys).cuda() if n else torch.zeros(1, dtype=torch.uint8, device="cuda")
            d_queue = torch.full((max(n, 1),), 0xFFFFFFFF, dtype=torch.int64, device="cuda").to(torch.int32)
            d_offsets = torch.zeros(routes + 1, dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            ctx.compact_routes_device(d_keys.data_ptr(), n, routes, d_queue.data_ptr(), d_offsets.data_ptr())
            queue = d_queue.cpu().numpy().view(np.uint32)[:n]
            offsets = d_offsets.cpu().numpy().view(np.uint32)
            counts = np.array([(keys == r).sum() for r in range(routes)], np.int64)
            assert (offsets == np.concatenate([[0], np.cumsum(counts)])).all(), (n, offsets, counts)
            for r in range(routes):
                expected = np.nonzero(keys == r)[0].astype(np.uint32)  # increasing slot order
                got = queue[offsets[r]:offsets[r + 1]]
                assert (got == expected).all(), f"n={n} route {r}"
