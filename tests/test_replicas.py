"""The multi-GPU mode is replicas only: each rank runs its own copy of the
deck and the ranks meet only in the bench's barrier and MAX reduction of the
timed region.  These CPU tests run that logic on two gloo ranks."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from datetime import timedelta
    import bench
    from ferrox_b200 import api, decks
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        # a replica: its own context from the same deck, nothing shared
        f = api.FerroX(decks.mfim(16, 16, 12))
        cells = f.N
        f.close()
        dist.barrier()
        ms = 10.0 + 5.0 * rank          # the ranks' own timed regions
        ms_max = bench.max_over_ranks(ms, world, device="cpu")
        out.put((rank, cells, ms_max, bench.whole_job_rate(cells, 4, world, ms_max)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_time_by_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    cells = res[0][1]
    assert cells == 16 * 16 * 12 and res[1][1] == cells
    # both ranks see the slowest rank's time, and the rate counts both replicas' cells
    assert [r[2] for r in res] == [15.0, 15.0]
    assert res[0][3] == pytest.approx(cells * 4 * 2 / 0.015)


def test_one_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(7.5, 1, device="cpu") == 7.5
    assert bench.whole_job_rate(1000, 10, 1, 2.0) == pytest.approx(5.0e6)
