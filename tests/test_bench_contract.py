"""CPU tests of bench.py: the air launch count it claims, and the reference
arm, the line the driver compares the GPU line against: under two ranks (RANK / WORLD_SIZE as torchrun sets them)
rank 0 prints exactly one JSON line with the contract's keys and rank 1 exits
0 without output. The arm times the oracle's port of the reference kernels
on host cores on a bounded sample of the C5 workload."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(rank, world):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "3", "--ref-step-seconds", "0.3"], cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=600)


def test_reference_arm_other_rank_exits_quietly():
    p = _run(1, 2)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""


def test_reference_arm_rank0_prints_one_contract_line():
    p = _run(0, 2)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "cell-ticks/s" and d["unit"] == "cell-ticks/s"
    assert d["n_gpus"] == 2 and d["steps"] == 1 and d["warmup"] >= 3 and d["higher_is_better"] is True
    assert d["value"] > 0 and d["config"]["workload"].startswith("C5")
    # the same config keys and values the GPU arm prints for the workload
    assert d["config"]["instances"] == 128 and d["config"]["cells"] == 6121601
    assert d["config"]["ticks_per_step"] == 1000
    # the sample covers both strata of C5: the 400x225 group and the heavy tail
    assert "of 64 instances" in d["cpu_baseline"]["sample"] and d["cpu_baseline"]["sample"].count("instances (") == 2
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_air_launch_count_with_temporal_blocking():
    """bench.py's gpu_launches claim for the air chain: 2 (or 3 with a NoUpdate
    + heat instance) launches per tick unblocked; blocks of n <= k ticks make
    n + 1 launches (+ n settles), cut at the end of each captured graph."""
    import types

    sys.path.insert(0, ROOT)
    import bench
    import tpt_field as tf

    def tuning(form, depth):
        return types.SimpleNamespace(air_form=form, temporal_depth=depth)

    tiles, sweep = tf.AIR_FORM_TILES, tf.AIR_FORM_SWEEP
    assert bench.air_launches(1000, tuning(tiles, 1), 2) == 2000
    assert bench.air_launches(1000, tuning(tiles, 1), 3) == 3000
    assert bench.air_launches(1000, tuning(sweep, 5), 2) == 2000
    # 1000 ticks at depth 2: 500 blocks of 3 launches
    assert bench.air_launches(1000, tuning(tiles, 2), 2) == 1500
    # depth 3 over graphs of 50 ticks: 16 blocks of 3 ticks (4 launches) + one of 2 (3) per graph
    assert bench.air_launches(100, tuning(tiles, 3), 2, chunk=50) == 2 * (16 * 4 + 3)
    # with the NoUpdate settle: n + 1 + n per block
    assert bench.air_launches(6, tuning(tiles, 3), 3) == 2 * (3 + 1 + 3)
