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


def test_reference_arm_prints_the_contract_line(tmp_path):
    """`bench.py --impl reference` (the oracle on the host cores, a bounded sample of the same outages) prints one JSON
    line with the engine arm's metric and unit, its own cpu_baseline and an e2e object with no device copies."""
    import json
    import subprocess
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--cpu-sample", "4"], capture_output=True, text=True, timeout=900,
                         cwd=str(tmp_path))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == "solves/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
