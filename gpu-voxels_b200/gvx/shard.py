"""Rank sharding of the path's independent units: maps of a batch (each map's
voxelise + EDT + queries touches only that map) and swept-volume lists (each
list's collision count touches only its own entries and the shared map).

The units are split over the ranks of a torch.distributed process group by a
cost-balanced partition (longest processing time first: units in decreasing
cost go to the least-loaded rank; ties to the lower rank), every rank runs its
own units with the single-GPU kernels, and the per-unit results meet on rank 0
in one reduction: each rank writes its units' rows into a zero tensor of the
full result's shape and the tensors are summed (NCCL over NVLink on GPUs, gloo
in the CPU tests).  No unit's data crosses ranks, so the data path has no
collective; the one reduction moves only results (counts, query outputs).

The reference has no multi-GPU code; this module adds the data-parallel form
the path admits.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence

import numpy as np
import torch


def partition(costs: Sequence[float], world: int) -> List[List[int]]:
    """Unit indices per rank, cost-balanced (LPT).  Deterministic: the same
    costs and world give the same plan on every rank.  Each rank's list is in
    increasing unit order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(costs.shape[0]), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    plan: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        plan[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in plan]


def imbalance(costs: Sequence[float], plan: Sequence[Sequence[int]]) -> float:
    """Largest rank load over the mean load (1.0 = perfect balance)."""
    costs = np.asarray(costs, dtype=np.float64)
    loads = [float(costs[list(p)].sum()) if len(p) else 0.0 for p in plan]
    mean = sum(loads) / max(len(loads), 1)
    return max(loads) / mean if mean > 0 else 1.0


def gather_rows(local: torch.Tensor, rows: Sequence[int], n_rows: int, dist=None, group=None,
                dst: int = 0) -> Optional[torch.Tensor]:
    """Assemble per-unit results on rank `dst`: `local` holds this rank's rows
    (in the order of `rows`), the result has n_rows rows.  Rows no rank owns
    stay zero.  Returns the full tensor on `dst`, None elsewhere (the full
    tensor on every rank when dist is None: a single process)."""
    full = torch.zeros((n_rows,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    if len(rows):
        idx = torch.as_tensor(list(rows), dtype=torch.int64, device=local.device)
        full.index_copy_(0, idx, local)
    if dist is None:
        return full
    dist.reduce(full, dst=dst, op=dist.ReduceOp.SUM, group=group)
    return full if dist.get_rank(group) == dst else None


def run_sharded(costs: Sequence[float], compute: Callable[[List[int]], torch.Tensor], n_rows_of: Callable[[int], int],
                dist=None, group=None, dst: int = 0):
    """Partition the units, run `compute(my_units)` -> a tensor whose rows are
    the units' result rows (unit k owns n_rows_of(k) consecutive rows, in unit
    order), and gather the rows on `dst`.  Returns (full result on dst or
    None, my_units, plan)."""
    world = 1 if dist is None else dist.get_world_size(group)
    rank = 0 if dist is None else dist.get_rank(group)
    plan = partition(costs, world)
    mine = plan[rank]
    starts = np.concatenate([[0], np.cumsum([n_rows_of(k) for k in range(len(costs))])]).astype(np.int64)
    rows = [r for k in mine for r in range(int(starts[k]), int(starts[k + 1]))]
    local = compute(mine)
    if local.shape[0] != len(rows):
        raise ValueError(f"compute returned {local.shape[0]} rows for {len(rows)} expected")
    return gather_rows(local, rows, int(starts[-1]), dist, group, dst), mine, plan


# ---------------------------------------------------------------------------
# the two sharded workloads on GPUs
# ---------------------------------------------------------------------------

class ShardedLists:
    """Per-list collision counts of CSR lists against one BitVectorVoxelMap,
    the lists split over the ranks by length (the kernel's work).  Every rank
    holds the map (a replica of the environment) and builds the CSR of its
    own lists once; `step` runs one batched launch over them and `gather`
    assembles all lists' counts on rank 0."""

    def __init__(self, ids: torch.Tensor, voxels: torch.Tensor, offsets_host: np.ndarray, bvm, dist=None, group=None):
        self.dist, self.group, self.bvm = dist, group, bvm
        offsets_host = np.asarray(offsets_host, dtype=np.int64)
        self.n_lists = offsets_host.shape[0] - 1
        self.lengths = offsets_host[1:] - offsets_host[:-1]
        world = 1 if dist is None else dist.get_world_size(group)
        rank = 0 if dist is None else dist.get_rank(group)
        self.plan = partition(self.lengths.astype(np.float64), world)
        self.mine = self.plan[rank]
        sel = np.asarray(self.mine, dtype=np.int64)
        take = torch.as_tensor(np.concatenate([np.arange(offsets_host[k], offsets_host[k + 1]) for k in sel])
                               if len(sel) else np.zeros(0, np.int64), device=ids.device)
        self.ids = ids.index_select(0, take).contiguous()
        self.vox = voxels.view(-1, 32).index_select(0, take).reshape(-1).contiguous()
        offs = np.zeros(len(self.mine) + 1, dtype=np.int64)
        offs[1:] = np.cumsum(self.lengths[sel]) if len(sel) else []
        self.offs = torch.as_tensor(offs, device=ids.device)
        self.counts = torch.zeros(len(self.mine), dtype=torch.int64, device=ids.device)

    def step(self, mark: bool = False) -> None:
        from .maps import lists_collide_map
        if self.mine:
            lists_collide_map(self.ids, self.vox, self.offs, self.bvm, mark=mark, counts=self.counts)

    def gather(self) -> Optional[torch.Tensor]:
        """All lists' counts (int64 [n_lists]) on rank 0, None elsewhere."""
        return gather_rows(self.counts, self.mine, self.n_lists, self.dist, self.group)


class ShardedBatch:
    """A batch of DistanceVoxelMaps split over ranks: rank r creates and
    processes only its own maps (cost = voxels, the EDT's work), all in one
    gvx Batch.  `step` runs voxelise + EDT + trilinear queries for the local
    maps; `gather` assembles every map's query results on rank 0."""

    def __init__(self, scenes, queries_per_map: Sequence[np.ndarray], dist=None, group=None):
        from .batch import Batch
        from .maps import DistanceVoxelMap

        self.dist, self.group = dist, group
        self.n_maps = len(scenes)
        self.costs = [float(np.prod(s.dims)) for s in scenes]
        world = 1 if dist is None else dist.get_world_size(group)
        rank = 0 if dist is None else dist.get_rank(group)
        self.plan = partition(self.costs, world)
        self.mine = self.plan[rank]
        self.q_counts = [int(q.shape[0]) for q in queries_per_map]
        self.maps = [DistanceVoxelMap(scenes[k].dims, scenes[k].side) for k in self.mine]
        pts = [scenes[k].points for k in self.mine]
        self.pts = torch.as_tensor(np.concatenate(pts).astype(np.float32) if pts else np.zeros((0, 3), np.float32)).cuda()
        offs = np.zeros(len(self.mine) + 1, dtype=np.int64)
        offs[1:] = np.cumsum([p.shape[0] for p in pts])
        self.offs = torch.as_tensor(offs).cuda()
        q = [queries_per_map[k] for k in self.mine]
        self.q = torch.as_tensor(np.concatenate(q).astype(np.float32) if q else np.zeros((0, 3), np.float32)).cuda()
        self.qm = torch.as_tensor(np.concatenate([np.full(queries_per_map[k].shape[0], i, np.int32)
                                                  for i, k in enumerate(self.mine)]) if q else
                                  np.zeros(0, np.int32)).cuda()
        self.batch = Batch(self.maps) if self.maps else None
        self.dist_out = self.grad_out = None

    def step(self) -> None:
        """Voxelise + EDT + queries of this rank's maps (stream-ordered)."""
        if self.batch is None:
            return
        self.batch.voxelize_edt(self.pts, self.offs)
        self.dist_out, self.grad_out = self.batch.query(self.q, self.qm)

    def gather(self) -> Optional[torch.Tensor]:
        """Every map's query results [sum of queries, 4] = (distance, gradient)
        on rank 0 (None on the other ranks), in map order."""
        starts = np.concatenate([[0], np.cumsum(self.q_counts)]).astype(np.int64)
        rows = [r for k in self.mine for r in range(int(starts[k]), int(starts[k + 1]))]
        if self.batch is None:
            local = torch.zeros((0, 4), dtype=torch.float32, device="cuda")
        else:
            local = torch.cat([self.dist_out[:, None], self.grad_out], 1)
        return gather_rows(local, rows, int(starts[-1]), self.dist, self.group)
