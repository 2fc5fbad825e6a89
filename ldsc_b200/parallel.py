"""Splitting an l2 run into record ranges: over the ranks of a process group
(one GPU per rank), or into slices that run one after another on one GPU
when the panel is larger than device memory.

Every pair (k, j), k < j, that a run accumulates satisfies left[j] <= k,
and left is non-decreasing.  A core of records [lo, hi) therefore gets its
exact l2 from one call over [call_lo, call_hi):

* call_lo = left[lo], the core's smallest limit, moved down to the chunk
  grid (the first record of its chromosome in the default per-chromosome
  mode, record 0 with --global-pass; src/l2/compute.rs:1164-1184).  A call
  that starts on the grid at or below every core limit chunks the core and
  everything after it exactly as the whole run does, and its block_left
  values are not clipped there.  With --snp-level-masking every window is
  the SNP's own (src/l2/compute.rs:1855-1867) and no alignment is needed;
* call_hi = the first record j >= hi with left[j] >= hi: the records after
  the core that pair with one of its records.

The call's own rows outside the core (the halos) are discarded.  Chromosomes
are independent (src/l2/mod.rs:477-553), so a core that holds whole
chromosomes needs no halo.  The only exchange between ranks is the final
gather of the l2 rows (`gather_l2`), the step the reference's single process
does not need: one tensor all-gather of the padded core rows.
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


def _balanced_cuts(load: np.ndarray, world: int) -> List[int]:
    """Cut positions 0 = c_0 <= ... <= c_world = len(load) splitting the
    records into `world` contiguous groups with about equal load."""
    cum = np.concatenate([[0.0], np.cumsum(load, dtype=np.float64)])
    total = cum[-1]
    n = len(load)
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        i = int(np.searchsorted(cum, target))
        # nearest boundary, never before the previous cut
        if i > 0 and abs(cum[i - 1] - target) <= abs(cum[min(i, n)] - target):
            i -= 1
        cuts.append(max(cuts[-1], min(i, n)))
    cuts.append(n)
    return cuts


def chunk_origin(snps: BimTable, global_pass: bool) -> np.ndarray:
    """First record of each record's chunking group: its chromosome's first
    record, or 0 with --global-pass."""
    m = len(snps)
    if global_pass or m == 0:
        return np.zeros(m, dtype=np.int64)
    chr_ = np.asarray(snps.chr)
    starts = np.flatnonzero(np.concatenate([[True], chr_[1:] != chr_[:-1]]))
    return starts[np.searchsorted(starts, np.arange(m), side="right") - 1].astype(np.int64)


def call_range(left: np.ndarray, origin: np.ndarray, chunk_c: int, snp_level_masking: bool,
               lo: int, hi: int) -> tuple:
    """Records [call_lo, call_hi) of the call that gives the core [lo, hi)
    its exact l2 (see the module note)."""
    m = len(left)
    if lo >= hi:
        return lo, lo
    a = int(left[lo])
    if not snp_level_masking:
        g = int(origin[a])
        a = g + (a - g) // chunk_c * chunk_c
    b = max(hi, int(np.searchsorted(left, hi, side="left")))
    return a, min(b, m)


def _shard(rank: int, lo: int, hi: int, left, origin, chunk_c, masking, pairs) -> Shard:
    a, b = call_range(left, origin, chunk_c, masking, lo, hi)
    return Shard(rank, lo, hi, a, b, int(pairs[lo:hi].sum()))


def plan_shards(snps: BimTable, mode: WindowMode, world: int, chunk_c: int = 200,
                snp_level_masking: bool = False, global_pass: bool = False) -> List[Shard]:
    """Split the records over `world` ranks with about equal pair counts."""
    m = len(snps)
    left = left_limits(snps, mode, chunk_c, snp_level_masking=snp_level_masking, global_pass=global_pass)
    pairs = np.arange(m, dtype=np.int64) - left          # pairs (k, j), k < j, credited to j
    origin = chunk_origin(snps, global_pass)
    cuts = _balanced_cuts(pairs.astype(np.float64), world) if m else [0] * (world + 1)
    return [_shard(r, cuts[r], cuts[r + 1], left, origin, chunk_c, snp_level_masking, pairs) for r in range(world)]


def plan_slices(snps: BimTable, mode: WindowMode, max_call_records: int, chunk_c: int = 200,
                snp_level_masking: bool = False, global_pass: bool = False) -> List[Shard]:
    """Consecutive slices for one device, each call at most max_call_records
    records (core plus halos), cores as large as the budget allows."""
    m = len(snps)
    left = left_limits(snps, mode, chunk_c, snp_level_masking=snp_level_masking, global_pass=global_pass)
    pairs = np.arange(m, dtype=np.int64) - left
    origin = chunk_origin(snps, global_pass)
    out: List[Shard] = []
    lo = 0
    while lo < m:
        def fits(hi):
            a, b = call_range(left, origin, chunk_c, snp_level_masking, lo, hi)
            return b - a <= max_call_records
        if not fits(lo + 1):
            a, b = call_range(left, origin, chunk_c, snp_level_masking, lo, lo + 1)
            raise ValueError(f"record {lo} needs a call of {b - a} records (window plus halo), more than "
                             f"the budget of {max_call_records}")
        # largest hi that fits (the call grows with hi)
        good, bad = lo + 1, m + 1
        while bad - good > 1:
            mid = (good + bad) // 2
            if fits(mid):
                good = mid
            else:
                bad = mid
        out.append(_shard(len(out), lo, good, left, origin, chunk_c, snp_level_masking, pairs))
        lo = good
    return out


def shard_records(snps: BimTable, sh: Shard) -> BimTable:
    """The records of a shard's l2 call."""
    return snps.subset(np.arange(sh.call_lo, sh.call_hi))


def core_rows(l2_call: np.ndarray, sh: Shard) -> np.ndarray:
    """The core rows of a shard's call output."""
    return l2_call[sh.core_lo - sh.call_lo: sh.core_hi - sh.call_lo]


def run_sharded(compute: Callable[[BimTable], np.ndarray], snps: BimTable, plan: Sequence[Shard], rank: int,
                group=None, dst: Optional[int] = 0, n_annot: int = 1) -> Optional[np.ndarray]:
    """Compute this rank's shard with `compute(records) -> l2 rows` (numpy,
    or a torch tensor of shape (call records, K)) and gather the full M x K
    l2 on rank `dst` (every rank when dst is None)."""
    sh = plan[rank]
    part = None
    if sh.call_hi > sh.call_lo:
        out = compute(shard_records(snps, sh))
        if not hasattr(out, "is_cuda"):
            out = np.asarray(out)
        part = core_rows(out, sh)
    return gather_l2(part, plan, rank, group, dst, n_annot)


def gather_l2(part, plan: Sequence[Shard], rank: int, group=None, dst: Optional[int] = 0, n_annot: int = 1):
    """Assemble the core rows of every rank with one tensor all-gather.

    ``part`` is this rank's core rows (core_hi - core_lo) x K, as a numpy
    array or a torch tensor (a CUDA tensor stays on the device).  Every rank
    pads its rows to the plan's largest core, so the collective moves equal
    f64 blocks; with the NCCL backend the blocks are CUDA tensors and the
    exchange runs over NVLink, with gloo they are CPU tensors.  Returns the
    M x K l2 as numpy on rank ``dst`` (every rank when dst is None), else
    None; ranks whose core is empty pass part=None."""
    import torch
    import torch.distributed as dist
    world = len(plan)
    nccl = dist.get_backend(group) == "nccl"
    dev = torch.device("cuda", torch.cuda.current_device()) if nccl else torch.device("cpu")
    rows = max(s.core_hi - s.core_lo for s in plan)
    if part is not None:
        t = part if isinstance(part, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(part))
        t = t.to(device=dev, dtype=torch.float64).reshape(t.shape[0], -1)
        n_annot = t.shape[1]
    block = torch.zeros((max(rows, 1), n_annot), dtype=torch.float64, device=dev)
    if part is not None and t.shape[0]:
        block[: t.shape[0]] = t
    blocks = [torch.empty_like(block) for _ in range(world)]
    dist.all_gather(blocks, block, group=group)
    if dst is not None and rank != dst:
        return None
    m = max(s.core_hi for s in plan)
    out = np.zeros((m, n_annot), dtype=np.float64)
    for sh, b in zip(plan, blocks):
        n = sh.core_hi - sh.core_lo
        if n:
            out[sh.core_lo: sh.core_hi] = b[:n].cpu().numpy()
    return out
