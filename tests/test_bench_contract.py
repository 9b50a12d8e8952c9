"""bench.py's reference arm (`--impl reference`): the reference's own CPU code
for the disk Poisson workload, one JSON line from rank 0 with the keys the
benchmark contract needs, and silent exit 0 on the other ranks under torchrun.
CPU only: the reference arm does not touch the GPU."""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _run(extra_env: dict) -> subprocess.CompletedProcess:
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    env.update(extra_env)
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                           "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                          cwd=ROOT, env=env, timeout=300)


def test_reference_arm_prints_one_contract_line():
    r = _run({})
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "walks/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and d["steps"] == 1
    assert d["config"]["workload"] and d["config"]["N_walks"] == 4096
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "walks/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_times_each_step_and_reports_the_gpu_arms_config():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps",
                        "2", "--warmup", "1"], capture_output=True, text=True, cwd=ROOT,
                       timeout=300, env={k: v for k, v in os.environ.items()
                                         if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")})
    assert r.returncode == 0, r.stderr
    d = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][0])
    sys.path.insert(0, str(ROOT))
    import bench
    # the measured wall time of a step, not a budget
    assert 0.0 < d["ms_per_step"] < 120000.0
    # the same workload keys as the GPU arm's line
    assert d["config"] == bench.CONFIG
    assert "2 timed steps" in d["cpu_baseline"]["sample"]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, str(ROOT))
    import bench
    secs, counts = bench.reduce_over_ranks(dist, "cpu", 1.0 + rank, [10.0 * (rank + 1), 1.0])
    q.put((rank, secs, counts))
    dist.destroy_process_group()


def test_bench_reduces_time_by_max_and_counts_by_sum_over_two_gloo_ranks():
    import multiprocessing as mp
    sys.path.insert(0, str(ROOT))
    import bench
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = bench.free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, secs, counts in got:
        assert secs == 2.0            # the slowest rank's time
        assert counts == [30.0, 2.0]  # walks and the like summed over ranks


def test_bench_gpus_flag_relaunches_one_process_per_gpu():
    sys.path.insert(0, str(ROOT))
    import bench
    cmd = bench.launch_command(["--gpus", "4", "--steps", "3"], 4, 29512)
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and "--master-addr=127.0.0.1" in cmd
    assert cmd[-4:] == ["--gpus", "4", "--steps", "3"]
    assert bench.parse(["--gpus", "2", "--scaling", "strong"]).scaling == "strong"
