"""SNP sharding across processes (the reference's MPI split) on CPU: the
range arithmetic against the reference's formula, and a world_size-2 gloo
group that partitions a SNP range with no overlap and reduces step times
as the benchmark does (max over ranks)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from omicabelnomm_b200 import shards as SH


def ref_split(m, k, N):
    """src/AIOwrapper.cpp:95-111."""
    if N > 1 and m >= N:
        m_mpi = m // N
        first = m_mpi * k
        cnt = m_mpi + (m - N * m_mpi) if k == N - 1 else m_mpi
        return first, cnt
    return 0, m


@pytest.mark.parametrize("m", [0, 1, 3, 7, 500, 1001, 500000])
@pytest.mark.parametrize("N", [1, 2, 3, 4, 8])
def test_shard_range_is_the_reference_split(m, N):
    covered = []
    for k in range(N):
        first, cnt = SH.shard_range(m, k, N)
        assert (first, cnt) == ref_split(m, k, N)
        covered.extend(range(first, first + cnt))
    if m >= N:
        assert covered == list(range(m))


def test_out_prefix():
    assert SH.out_prefix("res", 100, 0, 2) == "res_mpi1_"
    assert SH.out_prefix("res", 100, 1, 2) == "res_mpi2_"
    assert SH.out_prefix("res", 1, 0, 2) == "res"
    assert SH.out_prefix("res", 100, 0, 1) == "res"


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, m, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    first, cnt = SH.shard_range(m, rank, world)
    got = [None] * world
    dist.all_gather_object(got, (first, cnt))
    step = 0.25 * (rank + 1)                       # this rank's step time
    worst = SH.max_over_ranks(step, dist)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got, worst))


def test_two_ranks_partition_snps_and_take_the_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    m = 1001
    procs = [ctx.Process(target=_worker, args=(r, 2, port, m, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, worst in out:
        assert worst == 0.5
        (f0, c0), (f1, c1) = got
        assert f0 == 0 and f0 + c0 == f1 and f1 + c1 == m
