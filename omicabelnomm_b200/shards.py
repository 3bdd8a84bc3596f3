"""SNP shards across processes (one process per GPU), the analogue of the
reference's MPI mode (src/AIOwrapper.cpp:95-117): every shard scans a
contiguous SNP range with XL and Y replicated; the data path has no
collective.  The only cross-process steps are the host-side timing
reduction (max over ranks) and barriers."""
from __future__ import annotations

from typing import Optional

from . import engine as E


def shard_range(m: int, shard: int, shards: int) -> tuple[int, int]:
    """(first SNP, count) of a shard (oa_shard_range)."""
    return E.shard_range(m, shard, shards)


def out_prefix(out: str, m: int, shard: int, shards: int) -> str:
    """Output prefix of a shard: <out>_mpi<k+1>_ when the SNPs are split."""
    return f"{out}_mpi{shard + 1}_" if shards > 1 and m >= shards else out


def max_over_ranks(x: float, dist=None, device: Optional[object] = None) -> float:
    """Largest value of x over the process group (x itself without one)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
