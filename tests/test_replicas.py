"""Host logic of the multi-GPU replicas (cansfz/replicas.py) with two gloo
ranks on the CPU: the whole-job rate is the work of all ranks over the
slowest rank's time, and the ensemble's cases are split between the ranks
without overlap and with balanced cost."""
import json
import os
import socket

import pytest
import torch.multiprocessing as mp

from cansfz import replicas as R


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, outdir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    r, w, _ = R.setup(backend="gloo", timeout_s=60)
    R.barrier(w)
    rate = R.whole_job_rate(units_local=100.0 * (r + 1), seconds_local=1.0 + r, world=w)
    costs = [float(c) for c in (5, 1, 9, 3, 7, 2, 8, 4)]
    mine = R.assign_cases(costs, w)[r]
    total = R.sum_over_ranks(sum(costs[q] for q in mine), w)
    R.barrier(w)
    R.teardown(w)
    with open(os.path.join(outdir, f"rank{r}.json"), "w") as f:
        json.dump({"rate": rate, "mine": mine, "total": total}, f)


def test_two_gloo_ranks(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    # (100 + 200) units over the slowest rank's 2 s, on both ranks
    assert all(x["rate"] == pytest.approx(150.0) for x in res)
    got = sorted(res[0]["mine"] + res[1]["mine"])
    assert got == list(range(8)) and not set(res[0]["mine"]) & set(res[1]["mine"])
    assert res[0]["total"] == pytest.approx(39.0)


def test_assignment_balance():
    costs = [96 ** 3, 32 ** 3, 64 ** 3, 48 ** 3] * 4 + [256 * 512, 64 * 128] * 8
    for world in (1, 2, 4, 8):
        parts = R.assign_cases(costs, world)
        assert sorted(q for p in parts for q in p) == list(range(len(costs)))
        loads = [sum(costs[q] for q in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
