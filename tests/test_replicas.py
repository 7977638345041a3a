"""The multi-GPU replica plumbing on CPU: two gloo ranks in child processes."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from gpumetropolis_b200 import replicas as R


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=30))
    try:
        r, w, local = R.rank_env()
        seconds = 1.0 + 0.5 * r            # rank 1 is the slow one
        slowest = R.max_over_ranks(seconds)
        rate = R.whole_job_rate(1000, w, slowest)
        out.put((r, w, local, R.replica_seed(7, r), slowest, rate))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 for r in res)
    assert [r[2] for r in res] == [0, 1]
    assert res[0][3] != res[1][3]                 # independent streams per replica
    assert res[0][4] == res[1][4] == 1.5          # MAX over ranks on every rank
    assert res[0][5] == pytest.approx(2 * 1000 / 1.5)


def test_single_process_needs_no_group():
    assert R.max_over_ranks(2.5) == 2.5
    assert R.whole_job_rate(10, 1, 2.0) == 5.0
    with pytest.raises(ValueError):
        R.whole_job_rate(10, 1, 0.0)
