"""The multi-process (replica) path of bench.py on CPU: two gloo ranks, the job time is the maximum
over ranks and the throughput counts every rank's DoFs (weak scaling)."""
import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local = [1.0 + rank, 10.0 - rank]  # per-rank apply / end-to-end times (ms)
        ms, ms_e2e = bench.max_over_ranks(local, world, device="cpu")
        out[rank] = (ms, ms_e2e, bench.replica_throughput(1_000_000, world, ms))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_rank():
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
        res = dict(out)
    for rank in (0, 1):
        ms, ms_e2e, tput = res[rank]
        assert ms == 2.0 and ms_e2e == 10.0  # maxima over the two ranks
        assert abs(tput - 2 * 1_000_000 / 2e-3 / 1e9) < 1e-12
