"""The multi-GPU (replica) host logic on CPU: two gloo ranks run the barrier, the maximum of the ranks'
times, the whole-job rate, the round-robin dealing of serving requests and the gathering of their
records on rank 0, as bench.py does with NCCL on GPUs (one process per GPU, independent cases, no
data-path collective)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from compas_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        replicas.barrier(dist)
        own_ms = [12.5, 20.0][rank]  # the slower rank sets the job's time
        t = replicas.max_over_ranks(own_ms, dist)
        rate = replicas.whole_job_rate(256 ** 3, 3, 10, t / 1e3, world)

        class R:
            def __init__(self, rid):
                self.rid = rid

        mine = [r.rid for r in replicas.deal_requests([R(i) for i in range(7)], rank, world)]
        recs = replicas.gather({"rank": rank, "rids": mine}, dist)
        assert [x["rank"] for x in recs] == list(range(world))
        assert sorted(sum((x["rids"] for x in recs), [])) == list(range(7))
        out.put((rank, t, rate, mine))
        replicas.barrier(dist)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, v0, m0), (r1, t1, v1, m1) = res
    assert t0 == t1 == 20.0
    assert v0 == v1 == pytest.approx(2 * 256 ** 3 * 3 * 10 / 0.020)
    assert sorted(m0 + m1) == list(range(7)) and not set(m0) & set(m1)
    assert abs(len(m0) - len(m1)) <= 1


def test_single_process_defaults():
    assert replicas.max_over_ranks(3.5, None) == 3.5
    assert replicas.gather({"a": 1}, None) == [{"a": 1}]
    assert replicas.whole_job_rate(100, 3, 2, 0.5, 1) == 1200.0
    with pytest.raises(ValueError):
        replicas.whole_job_rate(100, 3, 2, 0.0, 1)
