"""The N > 1 path of bench.py on CPU: two gloo ranks agree on the slowest
rank's time and on the whole-job throughput."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from monalisa_b200 import replicas

    assert replicas.init("gloo", timeout_s=60)
    replicas.barrier()
    t = replicas.max_over_ranks(1.5 + rank)  # rank 1 is the slower one
    out[rank] = (t, replicas.throughput(world, 10, t))
    replicas.shutdown()


def test_two_gloo_ranks_take_the_max():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1] == (2.5, 2 * 10 / 2.5)


def test_single_process_is_a_no_op():
    from monalisa_b200 import replicas

    os.environ.pop("WORLD_SIZE", None)
    assert replicas.init("gloo") is False
    assert replicas.max_over_ranks(3.0) == 3.0
    assert replicas.throughput(1, 4, 2.0) == 2.0
