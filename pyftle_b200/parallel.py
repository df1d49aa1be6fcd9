"""Multi-GPU plumbing: one process per GPU, groups or windows sharded across ranks.

The FTLE hot path has no exchange step: neighbour groups are independent and so
are windows.  A window's N groups are split into contiguous ranges, one per rank
(all K neighbours of a group stay on its rank; the snapshot series is
replicated), every rank advects its range with no communication, and the only
collective is one gather of the per-rank FTLE slices (variable length) at the
end.  Several windows are instead dealt out whole, round-robin by rank.

This replaces the reference's process-level parallelism over windows
(``ParallelExecutor``, parallel.py:171-271), which pickles every window's data
to a worker process.

Everything here is backend-agnostic ``torch.distributed`` (NCCL on GPUs, gloo
in the CPU tests).
"""

from __future__ import annotations

import os
from dataclasses import dataclass
from datetime import timedelta
from typing import List, Sequence, Tuple

import torch
import torch.distributed as dist


@dataclass(frozen=True)
class RankInfo:
    rank: int = 0
    world: int = 1
    local_rank: int = 0

    @classmethod
    def from_env(cls) -> "RankInfo":
        return cls(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                   int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 600.0) -> RankInfo:
    """Initialise the process group when WORLD_SIZE > 1 (env:// rendezvous)."""
    info = RankInfo.from_env()
    if info.world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return info


def group_range(num_groups: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous [g0, g1) share of num_groups for rank (sizes differ by at most one)."""
    base, extra = divmod(num_groups, world)
    g0 = rank * base + min(rank, extra)
    return g0, g0 + base + (1 if rank < extra else 0)


def shard_positions(positions: torch.Tensor, dim: int, rank: int, world: int) -> torch.Tensor:
    """This rank's groups of a role-blocked (K*N, dim) array, still role-blocked."""
    K = 2 * dim
    N = positions.shape[0] // K
    g0, g1 = group_range(N, rank, world)
    return torch.cat([positions[r * N + g0:r * N + g1] for r in range(K)]).contiguous()


def unshard_positions(parts: Sequence[torch.Tensor], dim: int) -> torch.Tensor:
    """Inverse of shard_positions over all ranks' parts (in rank order)."""
    K = 2 * dim
    roles = []
    for r in range(K):
        for p in parts:
            n = p.shape[0] // K
            roles.append(p[r * n:(r + 1) * n])
    return torch.cat(roles)


def windows_of_rank(num_windows: int, rank: int, world: int) -> List[int]:
    """Round-robin assignment of whole windows to ranks."""
    return list(range(rank, num_windows, world))


def max_over_ranks(x: float, device=None) -> float:
    """Max of a scalar over all ranks (the timing rule for multi-GPU runs)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_field(local: torch.Tensor, num_groups: int) -> torch.Tensor:
    """All-gather per-rank FTLE slices (contiguous group ranges) into the full field."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return local
    world = dist.get_world_size()
    sizes = [group_range(num_groups, r, world) for r in range(world)]
    longest = max(g1 - g0 for g0, g1 in sizes)
    buf = torch.zeros(longest, dtype=local.dtype, device=local.device)
    buf[:local.numel()] = local
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    return torch.cat([p[:g1 - g0] for p, (g0, g1) in zip(parts, sizes)])
