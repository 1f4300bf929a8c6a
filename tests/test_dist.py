"""The multi-rank path on CPU: two gloo ranks agree on the slowest rank's
time and report whole-job throughput (weak scaling), as bench.py does under
torchrun with one process per GPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from padeops_b200 import dist as pdist

    r, w, local = pdist.world()
    assert (r, w, local) == (rank, world, rank)
    d = pdist.init("gloo", timeout_s=30)
    try:
        ms = 10.0 + 5.0 * rank          # rank 1 is the slow one
        slowest = pdist.max_over_ranks(ms, d)
        rate = pdist.weak_scaling_rate(1e9, w, slowest / 1e3)
        out.put((rank, slowest, rate))
        d.barrier()
    finally:
        d.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, slowest, rate in res:
        assert slowest == pytest.approx(15.0)
        assert rate == pytest.approx(2e9 / 15e-3)


def test_single_process_needs_no_group(monkeypatch):
    from padeops_b200 import dist as pdist

    monkeypatch.delenv("WORLD_SIZE", raising=False)
    assert pdist.init("gloo") is None
    assert pdist.max_over_ranks(3.5, None) == 3.5


def test_partition_fields_lpt():
    """Uneven fields split over ranks by LPT: every field once, loads within the
    largest field of each other (the LPT bound), deterministic."""
    import numpy as np

    from padeops_b200 import dist as pdist

    rng = np.random.default_rng(96)
    dims = (32, 48, 64, 96, 128, 192, 256, 384)
    costs = [float(np.prod(rng.choice(dims, 3))) * (1.0 if rng.integers(2) else 1.4) for _ in range(96)]
    for world in (1, 2, 4, 8):
        parts = pdist.partition_fields(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(96))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
        assert parts == pdist.partition_fields(costs, world)
