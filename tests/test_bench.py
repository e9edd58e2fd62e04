"""The benchmark's launch count: the formula over the level structure reproduces the ncu launch lists of the
9,241-bus / 500-outage batch, so the claimed gpu_launches is a count, not a guess."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench_mod(engine_lib):
    sys.path.insert(0, ROOT)
    import bench
    return bench


def test_launch_count_matches_the_launch_lists(bench_mod):
    from olfgpu import native
    _, p, _ = bench_mod.workload(0, 500)
    dense = native.Structure(p, native.PLAN_DENSE_FRONT)
    scaled = native.Structure(p)
    # FP64, four factorizing Newton rounds per solve (the launch lists: 3,990 launches over five solves under
    # schedule 3 with 2-lane solve tiles, 3,910 under the level schedule on the scaled plan; schedule 4 adds the
    # forward tail's prefix launch to the 798 of its list)
    assert bench_mod.launches_per_solve(dense, (3, 2, 256), 4, True, False, False, 0) == 798
    assert bench_mod.launches_per_solve(scaled, (0, 2, 256), 4, False, False, False, 0) == 782
    assert bench_mod.launches_per_solve(dense, (4, 0, 256), 4, True, False, False, 0) == 802
