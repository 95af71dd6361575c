"""Person sharding of one scoring job across ranks (one process per GPU).

A person's score reads only that person's genotype column and the per-variant
weights that every rank holds, so the scoring pass itself has no exchange
step.  The .fam order is cut into contiguous person ranges of whole .bed bytes
(multiples of 4 people, so a shard's columns are a byte slice of every
SNP-major row), rank r scores its range with the single-GPU engine, and the
only collective is one gather of the finished per-person rows to the rank that
writes the results after the pass.  The reference computes and writes one
cohort from one process (score/pipeline.rs:1739-1775 for the final sums,
score/main.rs:1389 ``write_scores_to_file`` for the .sscore); sharding changes
neither the per-person arithmetic nor the output order.

Work is fixed per rank as ranks are added when every rank keeps its shard size
(weak scaling); a fixed cohort split over more ranks is strong scaling.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Optional, Sequence

import numpy as np

from .prepare import PreparationResult


def person_ranges(total_people: int, world: int) -> list[tuple[int, int]]:
    """Contiguous .fam ranges [start, stop), one per rank, starting on whole
    .bed bytes (start % 4 == 0) and balanced to within one byte (4 people).
    Trailing ranks get empty ranges when there are fewer bytes than ranks."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if total_people < 0:
        raise ValueError("total_people must be >= 0")
    nbytes = (total_people + 3) // 4
    base, extra = divmod(nbytes, world)
    out, b = [], 0
    for r in range(world):
        nb = base + (1 if r < extra else 0)
        start, stop = min(4 * b, total_people), min(4 * (b + nb), total_people)
        out.append((start, stop))
        b += nb
    return out


@dataclass
class PersonShard:
    """One rank's slice of a scoring job."""

    rank: int
    start: int                  # first .fam index of the shard
    stop: int                   # one past the last .fam index
    prep: PreparationResult     # the job restricted to the shard's people
    output_rows: np.ndarray     # i64 [n]: the shard's people as rows of the full output

    @property
    def num_people(self) -> int:
        return self.prep.num_people_to_score


def shard_prep(prep: PreparationResult, start: int, stop: int, rank: int = 0) -> PersonShard:
    """Restrict ``prep`` to .fam people [start, stop).

    The weights, corrections, CSR and baseline are shared unchanged; the
    shard's .fam is the column slice, so fam index f becomes f - start, and the
    output people are those of the full job whose fam index falls in the range
    (in the full job's output order)."""
    if start % 4 != 0 or not 0 <= start <= stop <= prep.total_people_in_fam:
        raise ValueError(f"bad person range [{start}, {stop})")
    o2f = prep.output_idx_to_fam_idx
    if o2f is None:
        out_rows = np.arange(start, stop, dtype=np.int64)
        local_map = None
    else:
        f = o2f.astype(np.int64)
        out_rows = np.nonzero((f >= start) & (f < stop))[0].astype(np.int64)
        local_map = (f[out_rows] - start).astype(np.uint32)
    iids = None
    if prep.final_person_iids is not None:
        iids = [prep.final_person_iids[i] for i in out_rows.tolist()]
    sub = PreparationResult(
        sparse_weights=prep.sparse_weights,
        sparse_missing_corrections=prep.sparse_missing_corrections,
        sparse_score_columns=prep.sparse_score_columns,
        sparse_row_offsets=prep.sparse_row_offsets,
        score_names=list(prep.score_names),
        total_people_in_fam=stop - start,
        required_bim_indices=prep.required_bim_indices,
        output_idx_to_fam_idx=local_map,
        num_people_to_score=len(out_rows),
        baseline=prep.baseline,
        score_variant_counts=prep.score_variant_counts,
        final_person_iids=iids,
    )
    return PersonShard(rank, start, stop, sub, out_rows)


def make_shard(prep: PreparationResult, rank: int, world: int) -> PersonShard:
    start, stop = person_ranges(prep.total_people_in_fam, world)[rank]
    return shard_prep(prep, start, stop, rank)


def slice_rows(rows: np.ndarray, start: int, stop: int) -> np.ndarray:
    """Columns of packed SNP-major rows [V, pitch] holding people [start, stop)."""
    if start % 4 != 0:
        raise ValueError("a shard starts on a whole .bed byte")
    return np.ascontiguousarray(rows[:, start // 4:(stop + 3) // 4])


def gather_rows(sums, counts, output_rows: np.ndarray, num_output: int, num_scores: int,
                group=None, dst: int = 0, device=None):
    """Collect every rank's finished rows into the full [num_output, K] arrays.

    sums (f64) and counts (u32) are [n, K] (or flat n*K) numpy arrays of this
    rank's people; output_rows [n] their rows in the full output.  Every rank
    takes the same two all_gathers (sizes, then padded payload); ``dst``
    returns (sums, counts) as numpy arrays, the other ranks return None.
    ``device`` is where the collective's buffers live (CPU for gloo, the
    rank's GPU for NCCL)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = torch.device("cpu") if device is None else torch.device(device)
    K = num_scores
    n = len(output_rows)
    s = np.asarray(sums, dtype=np.float64).reshape(n, K)
    c = np.asarray(counts, dtype=np.uint32).reshape(n, K)

    size = torch.tensor([n], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(size) for _ in range(world)]
    dist.all_gather(sizes, size, group=group)
    sizes = [int(x.item()) for x in sizes]
    nmax = max(max(sizes), 1)

    # one f64 payload per rank: [row index, K sums, K counts] per person
    pay = torch.zeros((nmax, 1 + 2 * K), dtype=torch.float64)
    if n:
        pay[:n, 0] = torch.from_numpy(output_rows.astype(np.float64))
        pay[:n, 1:1 + K] = torch.from_numpy(s)
        pay[:n, 1 + K:] = torch.from_numpy(c.astype(np.float64))  # exact below 2^53
    pay = pay.to(dev)
    bufs = [torch.empty_like(pay) for _ in range(world)]
    dist.all_gather(bufs, pay, group=group)
    if rank != dst:
        return None
    full_s = np.zeros((num_output, K), dtype=np.float64)
    full_c = np.zeros((num_output, K), dtype=np.uint32)
    seen = np.zeros(num_output, dtype=bool)
    for b, m in zip(bufs, sizes):
        if m == 0:
            continue
        a = b[:m].cpu().numpy()
        rows = a[:, 0].astype(np.int64)
        if seen[rows].any():
            raise RuntimeError("two shards returned the same output row")
        seen[rows] = True
        full_s[rows] = a[:, 1:1 + K]
        full_c[rows] = a[:, 1 + K:].astype(np.uint32)
    if not seen.all():
        raise RuntimeError("the shards do not cover every output row")
    return full_s, full_c


ScoreFn = Callable[[PreparationResult, np.ndarray], tuple]


def score_sharded(prep: PreparationResult, rows: np.ndarray, rank: int, world: int,
                  score_fn: ScoreFn, group=None, dst: int = 0, device=None):
    """Score this rank's person shard of ``rows`` (full packed rows [V, pitch])
    with ``score_fn(shard_prep, shard_rows) -> (sums, counts)`` and gather the
    cohort on ``dst``.  Returns (full sums, full counts) on dst, else None."""
    shard = make_shard(prep, rank, world)
    K = prep.num_scores
    if shard.num_people:
        s, c = score_fn(shard.prep, slice_rows(rows, shard.start, shard.stop))
    else:
        s = np.zeros((0, K), dtype=np.float64)
        c = np.zeros((0, K), dtype=np.uint32)
    return gather_rows(s, c, shard.output_rows, prep.num_people_to_score, K,
                       group=group, dst=dst, device=device)
