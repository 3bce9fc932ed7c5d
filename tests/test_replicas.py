"""The multi-GPU replica bookkeeping on the CPU: two gloo ranks reduce their timed regions to the
maximum and count both ranks' units (the collective bench.py uses over NCCL), and the reference arm
runs on rank 0 only."""
import json
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    from supra_b200.replicas import job_rate, max_over_ranks, world_size
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        rate, ms = job_rate(100.0, 2, local_ms)
        res = {"world": world_size(), "ms": ms, "rate": rate, "max3": max_over_ranks(3.0 * (rank + 1))}
        dist.barrier()
    finally:
        dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


def test_two_gloo_ranks_take_the_max_and_count_all_units(tmp_path):
    world, port = 2, _free_port()
    mp.spawn(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        res = json.load(open(tmp_path / f"rank{r}.json"))
        assert res["world"] == 2
        assert res["ms"] == 15.0  # the slower rank's time
        assert res["rate"] == pytest.approx(100.0 * 2 * 2 / 0.015)
        assert res["max3"] == 6.0


def test_single_process_is_its_own_job():
    from supra_b200.replicas import job_rate, max_over_ranks
    assert max_over_ranks(7.5) == 7.5
    rate, ms = job_rate(10.0, 4, 20.0)
    assert ms == 20.0 and rate == pytest.approx(10.0 * 4 / 0.02)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    import argparse

    import bench
    args = argparse.Namespace(steps=1, warmup=0, gpus=2)
    assert bench.run_reference(args, rank=1) is None
    assert capsys.readouterr().out == ""


def test_reference_arm_json_line(capsys):
    """One bounded step of the reference arm on the host cores (rank 0): its JSON line carries the
    headline metric, a cpu_baseline describing the run and an e2e entry without device copies."""
    import argparse
    import json

    import bench
    args = argparse.Namespace(steps=1, warmup=0, gpus=1)
    bench.run_reference(args, rank=0)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["value"] > 0 and line["higher_is_better"] is True and line["steps"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
