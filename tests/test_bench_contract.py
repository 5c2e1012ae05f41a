"""Host-side pieces of bench.py: the replicas-only multi-rank timing (two gloo ranks on CPU) and
the reference arm's JSON line on the smallest workload."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _rank(rank, world, port, times, out):
    import torch
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = bench.max_over_ranks(times[rank], dist, torch, "cpu")
    out.put((rank, ms, bench.replicas_value(world, 10, ms)))
    dist.destroy_process_group()


def test_two_gloo_ranks_time_the_job_by_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    times = [120.0, 150.0]
    ps = [ctx.Process(target=_rank, args=(r, 2, 29517, times, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert [r[1] for r in res] == [150.0, 150.0]
    assert res[0][2] == pytest.approx(2 * 10 / 0.150)


def test_single_process_is_the_identity():
    import bench
    assert bench.max_over_ranks(42.0, None, None, "cpu") == 42.0


def test_reference_arm_prints_one_json_line():
    # whole OC iterations of the oracle are timed; `steps` is the number actually timed
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "cuboid25", "--steps", "2",
                        "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "OC iterations/s"
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["steps"] == 2 and line["steps_requested"] == 2
    assert line["ms_per_step"] == pytest.approx(1000.0 * line["steps"] / line["value"] / line["steps"])
    assert "whole OC iterations" in line["cpu_baseline"]["sample"]


def test_clock_median_uses_samples_under_load():
    # nvidia-smi lines: index, clocks.sm, clocks.max.sm, power, reasons mask, hw_slowdown,
    # hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap, utilization.gpu
    import bench
    c = bench.Clocks(0)
    c.lines = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active, 98",
               "0, 345, 1965, 150.0, 0x0, Not Active, Not Active, Not Active, Not Active, 0",
               "0, 1950, 1965, 900.0, 0x4, Not Active, Not Active, Not Active, Active, 100"]
    s = c.summary()
    assert s["sm_mhz"] == 1957.5 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] == 3 and s["samples_under_load"] == 2
    c.lines = [c.lines[1]]  # nothing under load: the median of what was sampled
    assert bench.Clocks.summary(c)["sm_mhz"] == 345.0
