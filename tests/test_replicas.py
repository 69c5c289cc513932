"""The multi-GPU path is replicas only (every rank solves its own right-hand
sides on its own operator copy); its coordination -- barrier, max-over-ranks
time, sum of solves -- runs here as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank))
    from asgard_b200 import replicas
    ws, r, _ = replicas.init("gloo", timeout_s=60)
    replicas.barrier()
    seconds = 1.0 + r            # rank 1 is the slowest
    solves = 3
    res = {
        "world": ws,
        "max": replicas.max_over_ranks(seconds),
        "sum": replicas.sum_over_ranks(solves),
        "rate": replicas.throughput(solves, seconds),
        "seed": replicas.rhs_seed(r),
    }
    replicas.barrier()
    replicas.shutdown()
    out[rank] = res


def test_replica_timing_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        codes = [p.exitcode for p in procs]
        for p in procs:
            if p.is_alive():
                p.kill()
        assert codes == [0, 0], codes
        res = dict(out)
    for r in range(world):
        assert res[r]["world"] == world
        assert res[r]["max"] == 2.0            # slowest rank's time
        assert res[r]["sum"] == 6.0            # all ranks' solves
        assert res[r]["rate"] == pytest.approx(3.0)   # 6 solves / 2 s
    assert res[0]["seed"] != res[1]["seed"]   # independent right-hand sides


def test_single_process_needs_no_process_group():
    from asgard_b200 import replicas
    assert replicas.max_over_ranks(2.5) == 2.5
    assert replicas.throughput(4, 2.0) == 2.0
