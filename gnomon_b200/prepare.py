"""Host-side preparation: the data contract handed to the GPU engine.

Mirrors the parts of gnomon's ``score/prepare.rs`` / ``score/types.rs`` that
the scoring hot path consumes:

* ``apply_simple_score_assignment`` (prepare.rs:197-208): every matched
  (variant, score) record folds into ``dosage_weight`` (+w when the effect
  allele is BIM allele2, -w when it is allele1 — "flipped") and
  ``missing_correction`` (+2w when flipped), summed over duplicates in record
  order with float32 arithmetic;
* ``allele_pair_matches`` / flip test (prepare.rs:211-219, 557-558);
* the CSR emission (prepare.rs:630-650): rows in BIM order, columns strictly
  ascending, ``baseline[k] = sum(missing_correction)`` in float64 and
  ``score_variant_counts[k]`` = number of cells of score k;
* ``bytes_per_variant = ceil(total_people_in_fam / 4)`` (prepare.rs:811).

Text parsing, PGS-catalog normalisation and the multiallelic ("complex")
resolver are outside this path.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Iterable, Optional, Sequence

import numpy as np


@dataclass
class PreparationResult:
    """The subset of gnomon's PreparationResult (types.rs:167-327) the engine reads."""

    sparse_weights: np.ndarray               # f32 [nnz] dosage_weight
    sparse_missing_corrections: np.ndarray   # f32 [nnz]
    sparse_score_columns: np.ndarray         # u32 [nnz]
    sparse_row_offsets: np.ndarray           # u64 [V+1]
    score_names: list
    total_people_in_fam: int
    required_bim_indices: Optional[np.ndarray] = None   # u64 [V] (None = identity)
    output_idx_to_fam_idx: Optional[np.ndarray] = None  # u32 [P] (None = identity)
    num_people_to_score: Optional[int] = None
    baseline: Optional[np.ndarray] = None               # f64 [K]
    score_variant_counts: Optional[np.ndarray] = None   # u32 [K]
    final_person_iids: Optional[list] = None
    # read only by the checkpoint fingerprint (checkpoint.rs:83-121)
    total_variants_in_bim: Optional[int] = None
    required_is_complex: Optional[np.ndarray] = None        # u8 [V]
    pipeline_kind: Optional[object] = None                  # .bed path or fileset boundaries
    # multi-row loci resolved on the CPU after the GPU pass (gnomon_b200.complex)
    complex_rules: list = field(default_factory=list)

    def __post_init__(self):
        self.sparse_weights = np.ascontiguousarray(self.sparse_weights, dtype=np.float32)
        self.sparse_missing_corrections = np.ascontiguousarray(self.sparse_missing_corrections,
                                                               dtype=np.float32)
        self.sparse_score_columns = np.ascontiguousarray(self.sparse_score_columns, dtype=np.uint32)
        self.sparse_row_offsets = np.ascontiguousarray(self.sparse_row_offsets, dtype=np.uint64)
        if self.required_bim_indices is not None:
            self.required_bim_indices = np.ascontiguousarray(self.required_bim_indices, np.uint64)
        if self.output_idx_to_fam_idx is not None:
            self.output_idx_to_fam_idx = np.ascontiguousarray(self.output_idx_to_fam_idx, np.uint32)
        if self.num_people_to_score is None:
            self.num_people_to_score = (len(self.output_idx_to_fam_idx)
                                        if self.output_idx_to_fam_idx is not None
                                        else self.total_people_in_fam)
        K = len(self.score_names)
        if self.baseline is None:
            self.baseline = compute_baseline(self.sparse_score_columns,
                                             self.sparse_missing_corrections, K)
        if self.score_variant_counts is None:
            self.score_variant_counts = np.bincount(self.sparse_score_columns.astype(np.int64),
                                                    minlength=K).astype(np.uint32)

    @property
    def num_scores(self) -> int:
        return len(self.score_names)

    @property
    def num_reconciled_variants(self) -> int:
        return len(self.sparse_row_offsets) - 1

    @property
    def bytes_per_variant(self) -> int:
        return (self.total_people_in_fam + 3) // 4

    @property
    def stride(self) -> int:
        """Score stride padded to 8 lanes (prepare.rs:427-433)."""
        return (self.num_scores + 7) // 8 * 8


def compute_baseline(cols: np.ndarray, corr: np.ndarray, K: int) -> np.ndarray:
    """baseline[k] = sum of missing_correction over score k's cells, float64, CSR order."""
    base = np.zeros(K, dtype=np.float64)
    np.add.at(base, cols.astype(np.int64), corr.astype(np.float64))
    return base


def apply_simple_score_assignment(entry: list, weight: float, is_flipped: bool) -> None:
    """Fold one matched record into ``[dosage_weight, missing_correction]`` (float32)."""
    w = np.float32(weight)
    if is_flipped:
        entry[0] = np.float32(entry[0] - w)
        entry[1] = np.float32(entry[1] + np.float32(2.0) * w)
    else:
        entry[0] = np.float32(entry[0] + w)


def allele_pair_matches(effect: str, other: str, bim_a1: str, bim_a2: str) -> bool:
    return (effect == bim_a1 and other == bim_a2) or (effect == bim_a2 and other == bim_a1)


def fold_cells(rows: np.ndarray, cols: np.ndarray, weights: np.ndarray, flipped: np.ndarray,
               num_rows: int):
    """Fold (row, col, weight, flipped) records into the CSR.

    Duplicated (row, col) records fold in record order with float32 arithmetic,
    as ``apply_simple_score_assignment`` does.  Returns
    (dosage_weight f32, missing_correction f32, cols u32, row_offsets u64).
    """
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    weights = np.asarray(weights, dtype=np.float32)
    flipped = np.asarray(flipped, dtype=bool)
    order = np.lexsort((np.arange(len(rows)), cols, rows))  # stable by record order
    r, c, w, f = rows[order], cols[order], weights[order], flipped[order]
    key_change = np.ones(len(r), dtype=bool)
    key_change[1:] = (r[1:] != r[:-1]) | (c[1:] != c[:-1])
    starts = np.nonzero(key_change)[0]
    dw = np.zeros(len(starts), dtype=np.float32)
    mc = np.zeros(len(starts), dtype=np.float32)
    # vectorised for the common single-record cell, sequential for duplicates
    ends = np.append(starts[1:], len(r))
    single = (ends - starts) == 1
    s1 = starts[single]
    dw[single] = np.where(f[s1], -w[s1], w[s1])
    mc[single] = np.where(f[s1], np.float32(2.0) * w[s1], np.float32(0.0))
    for j in np.nonzero(~single)[0]:
        entry = [np.float32(0.0), np.float32(0.0)]
        for t in range(starts[j], ends[j]):
            apply_simple_score_assignment(entry, float(w[t]), bool(f[t]))
        dw[j], mc[j] = entry
    out_rows = r[starts]
    counts = np.bincount(out_rows, minlength=num_rows)
    offs = np.zeros(num_rows + 1, dtype=np.uint64)
    np.cumsum(counts, out=offs[1:])
    return dw, mc, c[starts].astype(np.uint32), offs


@dataclass
class BimRecord:
    chrom: str
    pos: int
    allele1: str
    allele2: str


@dataclass
class ScoreRecord:
    chrom: str
    pos: int
    effect_allele: str
    other_allele: str
    weights: Sequence[float]   # one per score column (NaN = absent)


def reconcile_simple(bim: Sequence[BimRecord], records: Iterable[ScoreRecord],
                     score_names: Sequence[str], total_people_in_fam: int,
                     keep_fam_indices: Optional[Sequence[int]] = None) -> PreparationResult:
    """Simple-variant merge join of score records against BIM rows.

    A record matches a BIM row at the same (chrom, pos) when its allele pair
    equals the row's (either order); it is flipped when its effect allele is
    BIM allele1 (prepare.rs:557-558).  Rows without any match are not
    required.  Records that match several rows (multiallelic sites) are
    rejected: that resolver is not part of this path.
    """
    by_pos: dict = {}
    for idx, b in enumerate(bim):
        by_pos.setdefault((b.chrom, b.pos), []).append(idx)
    rr, cc, ww, ff = [], [], [], []
    for rec in records:
        matches = [i for i in by_pos.get((rec.chrom, rec.pos), [])
                   if allele_pair_matches(rec.effect_allele, rec.other_allele,
                                          bim[i].allele1, bim[i].allele2)]
        if not matches:
            continue
        if len(matches) > 1:
            raise ValueError(f"ambiguous multiallelic match at {rec.chrom}:{rec.pos}")
        i = matches[0]
        flipped = rec.effect_allele == bim[i].allele1
        for k, w in enumerate(rec.weights):
            if w is None or (isinstance(w, float) and np.isnan(w)):
                continue
            rr.append(i); cc.append(k); ww.append(w); ff.append(flipped)
    required = np.array(sorted(set(rr)), dtype=np.uint64)
    remap = {int(b): j for j, b in enumerate(required)}
    rows = np.array([remap[i] for i in rr], dtype=np.int64)
    dw, mc, cols, offs = fold_cells(rows, np.array(cc, dtype=np.int64),
                                    np.array(ww, dtype=np.float32), np.array(ff, dtype=bool),
                                    len(required))
    keep = None if keep_fam_indices is None else np.asarray(keep_fam_indices, dtype=np.uint32)
    return PreparationResult(dw, mc, cols, offs, list(score_names), total_people_in_fam,
                             required_bim_indices=required, output_idx_to_fam_idx=keep)


def from_workload(w) -> PreparationResult:
    """PreparationResult of a named synthetic workload (gnomon_b200.synth)."""
    from .synth import score_cells
    offs, cols, weight, flipped = score_cells(w)
    dw = np.where(flipped, -weight, weight).astype(np.float32)
    mc = np.where(flipped, np.float32(2.0) * weight, np.float32(0.0)).astype(np.float32)
    names = [f"S{k:03d}" for k in range(w.scores)]
    return PreparationResult(dw, mc, cols, offs, names, w.people)
