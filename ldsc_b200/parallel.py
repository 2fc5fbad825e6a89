"""Sharding an l2 run over the ranks of a process group (one GPU per rank).

The path shards without a data-path collective:

* default per-chromosome mode: chromosomes are independent
  (src/l2/mod.rs:477-553), so each rank takes whole chromosomes, balanced by
  their pair counts;
* --snp-level-masking: every SNP's window is its own, independent of the
  chunk grid (src/l2/compute.rs:1855-1867), so a chromosome may also be cut
  inside; a rank computes its core records plus a halo -- the records its
  core pairs with on either side -- and keeps the core rows;
* --global-pass without masking: the chunk grid runs across chromosomes from
  the first record, so the run is not split (rank 0 computes it).

The only exchange is the final gather of the l2 rows (`gather_l2`), the step
the reference's single process does not need.
"""
from __future__ import annotations

import dataclasses
from typing import Callable, List, Optional, Sequence

import numpy as np

from .api import WindowMode, left_limits
from .plink import BimTable


@dataclasses.dataclass
class Shard:
    rank: int
    core_lo: int     # records [core_lo, core_hi) are this rank's output
    core_hi: int
    call_lo: int     # records [call_lo, call_hi) go into its l2 call
    call_hi: int
    pairs: int       # in-band pairs of the core records (the load)


def _balanced_cuts(load: np.ndarray, units: Sequence[int], world: int) -> List[int]:
    """Cut positions (indices into `units` boundaries) splitting the units into
    `world` contiguous groups with about equal load."""
    cum = np.concatenate([[0], np.cumsum(load)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        i = int(np.searchsorted(cum, target))
        # nearest boundary, never before the previous cut
        if i > 0 and abs(cum[i - 1] - target) <= abs(cum[min(i, len(cum) - 1)] - target):
            i -= 1
        cuts.append(max(cuts[-1], min(i, len(units) - 1)))
    cuts.append(len(units) - 1)
    return cuts


def plan_shards(snps: BimTable, mode: WindowMode, world: int, chunk_c: int = 200,
                snp_level_masking: bool = False, global_pass: bool = False) -> List[Shard]:
    """Split the records over `world` ranks (see the module note)."""
    m = len(snps)
    left = left_limits(snps, mode, chunk_c, snp_level_masking=snp_level_masking, global_pass=global_pass)
    pairs = np.arange(m, dtype=np.int64) - left          # pairs (k, j), k < j, credited to j
    if m == 0 or world == 1 or (global_pass and not snp_level_masking):
        return [Shard(0, 0, m, 0, m, int(pairs.sum()))] + [Shard(r, m, m, m, m, 0) for r in range(1, world)]
    if not snp_level_masking:
        # whole chromosomes: boundaries where the chromosome code changes
        bounds = [0] + [i for i in range(1, m) if snps.chr[i] != snps.chr[i - 1]] + [m]
        load = np.array([pairs[a:b].sum() for a, b in zip(bounds[:-1], bounds[1:])], dtype=np.float64)
        cuts = _balanced_cuts(load, bounds, world)
        out = []
        for r in range(world):
            lo, hi = bounds[cuts[r]], bounds[cuts[r + 1]]
            out.append(Shard(r, lo, hi, lo, hi, int(pairs[lo:hi].sum())))
        return out
    # per-SNP windows: cut anywhere, by pair count; halo from the left limits
    bounds = list(range(m + 1))
    cuts = _balanced_cuts(pairs.astype(np.float64), bounds, world)
    out = []
    for r in range(world):
        lo, hi = cuts[r], cuts[r + 1]
        if lo >= hi:
            out.append(Shard(r, lo, lo, lo, lo, 0))
            continue
        call_lo = int(left[lo:hi].min())
        # right partners k >= hi of the core: left[k] < hi (left is non-decreasing within a chromosome)
        call_hi = hi
        while call_hi < m and left[call_hi] < hi and snps.chr[call_hi] == snps.chr[hi - 1]:
            call_hi += 1
        out.append(Shard(r, lo, hi, call_lo, call_hi, int(pairs[lo:hi].sum())))
    return out


def shard_records(snps: BimTable, sh: Shard) -> BimTable:
    """The records of a shard's l2 call."""
    return snps.subset(np.arange(sh.call_lo, sh.call_hi))


def core_rows(l2_call: np.ndarray, sh: Shard) -> np.ndarray:
    """The core rows of a shard's call output."""
    return l2_call[sh.core_lo - sh.call_lo: sh.core_hi - sh.call_lo]


def run_sharded(compute: Callable[[BimTable], np.ndarray], snps: BimTable, plan: Sequence[Shard], rank: int,
                group=None, dst: Optional[int] = 0) -> Optional[np.ndarray]:
    """Compute this rank's shard with `compute(records) -> l2 rows` and gather
    the full M x K l2 on rank `dst` (every rank when dst is None)."""
    sh = plan[rank]
    part = None
    if sh.call_hi > sh.call_lo:
        part = core_rows(np.asarray(compute(shard_records(snps, sh))), sh)
    return gather_l2(part, plan, rank, group, dst)


def gather_l2(part: Optional[np.ndarray], plan: Sequence[Shard], rank: int, group=None,
              dst: Optional[int] = 0) -> Optional[np.ndarray]:
    """Assemble the core rows of every rank (torch.distributed object
    collectives: any backend)."""
    import torch.distributed as dist
    world = len(plan)
    payload = (plan[rank].core_lo, part)
    if dst is None:
        parts = [None] * world
        dist.all_gather_object(parts, payload, group=group)
    else:
        parts = [None] * world if rank == dst else None
        dist.gather_object(payload, parts, dst=dst, group=group)
        if rank != dst:
            return None
    m = max(s.core_hi for s in plan)
    k = next((p.shape[1] for _, p in parts if p is not None), 1)
    out = np.zeros((m, k), dtype=np.float64)
    for lo, p in parts:
        if p is not None:
            out[lo: lo + p.shape[0]] = p
    return out
