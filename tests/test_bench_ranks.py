"""The multi-rank path of bench.py (replicas: one mesh per rank, no data-path
collective) on two gloo ranks on the CPU: the barrier, the max over ranks of
the timed region and the whole-job rate, and the reference arm, which only
rank 0 runs."""
import contextlib
import io
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        r = bench.Ranks(dist, world, "cpu")
        r.barrier()
        seconds = 1.0 + rank  # the slower rank sets the time
        m = r.max(seconds)
        out[rank] = (m, bench.whole_job_rate(100.0, world, m))
        # the reference arm prints on rank 0 only; other ranks return at once
        if rank != 0:
            buf = io.StringIO()
            with contextlib.redirect_stdout(buf):
                bench.main_reference(None, rank, world)
            out[10 + rank] = buf.getvalue()
        r.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_time_and_rate():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world,
                           start_method="spawn", join=True)
        res = dict(out)
    for rank in range(world):
        m, rate = res[rank]
        assert m == 2.0
        assert rate == 100.0 * world / 2.0
    assert res[11] == ""
