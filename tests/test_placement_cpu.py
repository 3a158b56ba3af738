"""Placement of independent matrices on several GPUs (rr_place_by_footprint,
rr_footprint): host-only logic, tested against a fake device list."""
import numpy as np
import pytest

import rust_rank_b200 as rr
from rust_rank_b200 import synth


def greedy(footprints, free):
    """The rule restated: largest first (stable), onto the device with the most room left (lowest index on ties)."""
    load = [0] * len(free)
    where = [0] * len(footprints)
    for i in sorted(range(len(footprints)), key=lambda i: -footprints[i]):
        room = [max(f - l, 0) for f, l in zip(free, load)]
        d = max(range(len(free)), key=lambda d: (room[d], -d))
        assert footprints[i] <= room[d]
        where[i] = d
        load[d] += footprints[i]
    return where, load


@pytest.mark.parametrize("seed", range(6))
def test_matches_the_greedy_rule(seed):
    rng = np.random.default_rng(seed)
    fps = rng.integers(1, 1 << 30, size=int(rng.integers(1, 60))).tolist()
    free = [int(sum(fps) // 3 + rng.integers(0, 1 << 30)) for _ in range(int(rng.integers(1, 8)))]
    free[0] = max(free[0], max(fps) * len(fps))  # room for everything somewhere
    where, load = rr.place_by_footprint(fps, free)
    w2, l2 = greedy(fps, free)
    assert where.tolist() == w2 and load.tolist() == l2


def test_balances_equal_devices():
    fps = [100] * 64
    where, load = rr.place_by_footprint(fps, [10_000] * 8)
    assert sorted(np.bincount(where, minlength=8).tolist()) == [8] * 8
    assert load.tolist() == [800] * 8


def test_large_first_then_fill():
    where, load = rr.place_by_footprint([10, 90, 50, 40], [100, 100])
    # 90 -> dev 0, 50 -> dev 1, 40 -> dev 1 (room 50 vs 10), 10 -> dev 0 (room 10 vs 10: lowest index)
    assert where.tolist() == [0, 0, 1, 1] and load.tolist() == [100, 90]


def test_refuses_an_item_that_fits_nowhere():
    with pytest.raises(rr.RRError) as e:
        rr.place_by_footprint([50, 300], [200, 250])
    assert e.value.status == 3  # RR_ENOMEM


def test_fake_fleet_of_graph_complex_matrices():
    """The batched workload's footprints on a fake 4-GPU list with one smaller device."""
    mats = synth.graph_complex_batch(nmat=40, rmin=1000, rmax=20000)
    fps = [rr.footprint(m, n, int(rp[-1]), 16) for rp, _, _, m, n in mats]
    free = [3 * sum(fps) // 8, 3 * sum(fps) // 8, 3 * sum(fps) // 8, sum(fps) // 8]
    where, load = rr.place_by_footprint(fps, free)
    assert all(int(load[d]) <= free[d] for d in range(4))
    assert sum(int(x) for x in load) == sum(fps)
    # the three large devices end within one largest matrix of each other
    big = sorted(int(x) for x in load[:3])
    assert big[-1] - big[0] <= max(fps)


def test_footprint_grows_with_the_matrix():
    a = rr.footprint(10_000, 8_000, 80_000, 16)
    b = rr.footprint(20_000, 16_000, 160_000, 16)
    c = rr.footprint(20_000, 16_000, 160_000, 32)
    assert 0 < a < b < c
    with pytest.raises(rr.RRError):
        rr.footprint(0, 5, 0, 16)
