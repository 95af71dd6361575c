"""Complex (multiallelic / multi-row) variant resolution after the GPU pass.

The reference scores ordinary variants in its engines and leaves "complex"
loci -- one score variant that several .bim rows could describe -- to a CPU
pass over the finished accumulators (score/complex.rs:994-1307, called from
score/cuda_backend.rs:1465-1535).  For every person, rule (locus) and score
applied to it:

* the person's genotype is read from every candidate .bim row; rows whose
  call is missing (01) are dropped;
* rows whose allele pair equals the score's (either orientation) remain;
  none -> the score counts the locus as missing for that person; one -> its
  effect-allele dosage times the weight is added; several -> the heuristic
  chain below picks a dosage, or the run stops with a fatal ambiguity.

Heuristics, in order (complex.rs:946-973): exact allele-pair match,
unambiguous genotype (both row alleles are score alleles), matching allele
structure (the person's allele lengths equal the score's), consistent dosage,
indel anchor base (conflicting homozygous calls of a short and a long allele
sharing a prefix -> heterozygous), prefer the single heterozygous call,
opposing homozygous calls as heterozygous, and the average dosage of all
remaining interpretations.

Vectorised over people: per rule the candidate rows' codes form one pattern
per person; every distinct pattern is resolved once and applied to all the
people that share it.  Each person's additions happen in rule order and, per
rule, in score-application order -- the reference's order -- so the f64 sums
round identically.  Which samples of each heuristic are reported (up to 5)
and which person a fatal error names are the first ones in output order (the
reference's parallel loop reports whichever thread got there first).
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

# ---- rule data (types.rs:118-146) ---------------------------------------------


@dataclass(frozen=True)
class ScoreInfo:
    effect_allele: str
    other_allele: str
    weight: float            # f32 in the reference
    score_column_index: int


@dataclass
class GroupedComplexRule:
    locus_chr_pos: Tuple[str, int]
    possible_contexts: List[Tuple[int, str, str]]   # (bim row, allele1, allele2)
    score_applications: List[ScoreInfo]


class Heuristic(enum.Enum):
    ExactScoreAlleleMatch = 0
    PrioritizeUnambiguousGenotype = 1
    PreferMatchingAlleleStructure = 2
    ConsistentDosage = 3
    PreferHeterozygous = 4
    IndelAnchorBase = 5
    FallbackOpposingHomozygousAsHet = 6
    FallbackAverageDosageAcrossConflicts = 7


PIPELINE_ORDER = (Heuristic.ExactScoreAlleleMatch, Heuristic.PrioritizeUnambiguousGenotype,
                  Heuristic.PreferMatchingAlleleStructure, Heuristic.ConsistentDosage,
                  Heuristic.IndelAnchorBase, Heuristic.PreferHeterozygous,
                  Heuristic.FallbackOpposingHomozygousAsHet,
                  Heuristic.FallbackAverageDosageAcrossConflicts)

Interpretation = Tuple[int, Tuple[int, str, str]]   # (genotype bits, context)


def _blen(s: str) -> int:
    return len(s.encode())


def pair_matches(si: ScoreInfo, a1: str, a2: str) -> bool:
    return (si.effect_allele == a1 and si.other_allele == a2) or \
        (si.effect_allele == a2 and si.other_allele == a1)


def score_dosage(bits: int, a1: str, a2: str, si: ScoreInfo) -> Optional[float]:
    """Effect-allele dosage of a call w.r.t. a row's (A1, A2); None when the
    row's alleles are not the score's pair (complex.rs:881-910)."""
    if not pair_matches(si, a1, a2):
        return None
    d1 = {0b00: 2.0, 0b10: 1.0, 0b11: 0.0}.get(bits, 0.0)
    if a1 == si.effect_allele:
        return d1
    if a2 == si.effect_allele:
        return 2.0 - d1
    return None


def person_alleles(bits: int, a1: str, a2: str) -> Tuple[str, str]:
    return {0b00: (a1, a1), 0b10: (a1, a2), 0b11: (a2, a2)}.get(bits, ("", ""))


def _single(h: Heuristic, cands: Sequence[Interpretation], si: ScoreInfo):
    if len(cands) != 1:
        return None
    bits, (_, a1, a2) = cands[0]
    d = score_dosage(bits, a1, a2, si)
    return None if d is None else (d, h)


def try_heuristic(h: Heuristic, si: ScoreInfo, inter: Sequence[Interpretation]):
    """(dosage, heuristic) or None (complex.rs:544-877)."""
    ea, oa = si.effect_allele, si.other_allele
    if h is Heuristic.ExactScoreAlleleMatch:
        return _single(h, [x for x in inter if (x[1][1] == ea and x[1][2] == oa)
                           or (x[1][1] == oa and x[1][2] == ea)], si)
    if h is Heuristic.PrioritizeUnambiguousGenotype:
        return _single(h, [x for x in inter if x[1][1] in (ea, oa) and x[1][2] in (ea, oa)], si)
    if h is Heuristic.PreferMatchingAlleleStructure:
        l1, l2 = _blen(ea), _blen(oa)
        keep = []
        for x in inter:
            p1, p2 = person_alleles(x[0], x[1][1], x[1][2])
            n1, n2 = _blen(p1), _blen(p2)
            if n1 == 0:
                continue
            if (n1 == l1 and n2 == l2) or (n1 == l2 and n2 == l1):
                keep.append(x)
        return _single(h, keep, si)
    if h is Heuristic.ConsistentDosage:
        ds = [score_dosage(b, c[1], c[2], si) for b, c in inter]
        if any(d is None for d in ds):
            return None
        return (ds[0], h) if all(abs(d - ds[0]) < 1e-9 for d in ds) else None
    if h is Heuristic.PreferHeterozygous:
        het = [x for x in inter if x[0] == 0b10]
        if len(het) == 1 and any(x[0] != 0b10 for x in inter):
            return _single(h, het, si)
        return None
    if h is Heuristic.IndelAnchorBase:
        hom = [c[1] if b == 0b00 else c[2] for b, c in inter if b in (0b00, 0b11)]
        if len(hom) < 2 or all(a == hom[0] for a in hom):
            return None
        shortest = hom[0]
        for a in hom:                         # first of the minimal byte length
            if _blen(a) < _blen(shortest):
                shortest = a
        longest = hom[0]
        for a in hom:                         # last of the maximal byte length
            if _blen(a) >= _blen(longest):
                longest = a
        if not longest.startswith(shortest) or not all(a in (shortest, longest) for a in hom):
            return None
        if not ((ea == shortest and oa == longest) or (ea == longest and oa == shortest)):
            return None
        return (float(ea == shortest) + float(ea == longest), h)
    if h is Heuristic.FallbackOpposingHomozygousAsHet:
        from00 = {c[1] for b, c in inter if b == 0b00}
        from11 = {c[2] for b, c in inter if b == 0b11}
        if len(from00) != 1 or len(from11) != 1:
            return None
        x00, x11 = next(iter(from00)), next(iter(from11))
        if x00 == x11 or not ((ea == x00 and oa == x11) or (ea == x11 and oa == x00)):
            return None
        return (float(ea == x00) + float(ea == x11), h)
    if h is Heuristic.FallbackAverageDosageAcrossConflicts:
        if not inter:
            return None
        ds = [score_dosage(b, c[1], c[2], si) for b, c in inter]
        if any(d is None for d in ds):
            return None
        total = 0.0
        for d in ds:
            total += d
        return (total / len(inter), h)
    raise ValueError(h)


def resolve_conflict(si: ScoreInfo, inter: Sequence[Interpretation]):
    """First heuristic of the chain that resolves; None when none does."""
    for h in PIPELINE_ORDER:
        r = try_heuristic(h, si, inter)
        if r is not None:
            return r
    return None


# ---- genotype source (complex.rs:17-156) --------------------------------------

class GenotypeSource:
    """2-bit calls of .bim rows for .fam people: one .bed (rows after the
    magic) or several filesets, each holding the global rows from its
    starting index (the multi-file resolver)."""

    def __init__(self, beds: Sequence[np.ndarray], starts: Sequence[int], bytes_per_variant: int):
        if len(beds) != len(starts):
            raise ValueError("Mismatched number of byte sources and fileset boundaries")
        self.beds = [np.asarray(b, dtype=np.uint8).reshape(-1) for b in beds]
        self.starts = np.asarray(starts, dtype=np.int64)
        self.bpv = int(bytes_per_variant)

    @classmethod
    def single(cls, rows: np.ndarray, bytes_per_variant: int) -> "GenotypeSource":
        return cls([rows], [0], bytes_per_variant)

    def codes(self, bim_row: int, fam: np.ndarray) -> np.ndarray:
        i = int(np.searchsorted(self.starts, bim_row, side="right")) - 1
        local = bim_row - int(self.starts[i])
        byte = local * self.bpv + (fam // 4).astype(np.int64)
        bed = self.beds[i]
        if local < 0 or (byte.size and int(byte.max()) >= bed.size):
            raise IOError(f"Genotype bytes of .bim row {bim_row} lie past the end of its .bed")
        return ((bed[byte] >> (2 * (fam % 4)).astype(np.uint8)) & 3).astype(np.uint8)


# ---- the pass -----------------------------------------------------------------

class ComplexResolutionError(RuntimeError):
    def __init__(self, kind: str, message: str):
        super().__init__(message)
        self.kind = kind        # "Compute" (fatal ambiguity) or "Io"


@dataclass
class ComplexReport:
    """Per-heuristic counts and up to 5 sample (person, locus, score) triples."""

    counts: Dict[Heuristic, int] = field(default_factory=dict)
    samples: Dict[Heuristic, list] = field(default_factory=dict)


def _genotype_text(bits: int, a1: str, a2: str) -> str:
    return {0b00: f"{a1}/{a1}", 0b01: "Missing", 0b10: f"{a1}/{a2}",
            0b11: f"{a2}/{a2}"}.get(bits, "Invalid Bits")


def _fatal_report(iid: str, rule: GroupedComplexRule, score_name: str,
                  inter: Sequence[Interpretation]) -> str:
    lines = [f"Fatal: no heuristic resolves the genotype of individual '{iid}' at locus "
             f"{rule.locus_chr_pos[0]}:{rule.locus_chr_pos[1]} for score {score_name}.",
             "Conflicting .bim rows:"]
    for bits, (row, a1, a2) in inter:
        lines.append(f"  row {row}: alleles ({a1}, {a2}), genotype bits {bits:02b} "
                     f"({_genotype_text(bits, a1, a2)})")
    return "\n".join(lines)


def resolve_complex_variants(rules: Sequence[GroupedComplexRule], source: GenotypeSource,
                             output_idx_to_fam: Optional[np.ndarray], num_people: int,
                             score_names: Sequence[str], final_scores: np.ndarray,
                             final_counts: np.ndarray,
                             person_iids: Optional[Sequence[str]] = None) -> ComplexReport:
    """Apply every rule to the [P][K] accumulators in place."""
    report = ComplexReport()
    K = len(score_names)
    S = final_scores.reshape(num_people, K)
    C = final_counts.reshape(num_people, K)
    fam = (np.arange(num_people, dtype=np.int64) if output_idx_to_fam is None
           else np.asarray(output_idx_to_fam, dtype=np.int64))
    iid = (lambda p: person_iids[p]) if person_iids is not None else (lambda p: str(p))
    for rule in rules:
        ctxs = rule.possible_contexts
        try:
            codes = np.stack([source.codes(int(r), fam) for r, _, _ in ctxs]) if ctxs else \
                np.zeros((0, num_people), np.uint8)
        except (IOError, OSError) as e:
            raise ComplexResolutionError("Io", str(e)) from e
        if ctxs:
            pats, inv = np.unique(codes.T, axis=0, return_inverse=True)
            inv = inv.reshape(-1)
        else:
            pats, inv = np.zeros((1, 0), np.uint8), np.zeros(num_people, np.int64)
        for si in rule.score_applications:
            col = si.score_column_index
            w = float(np.float32(si.weight))
            n = len(pats)
            add = np.zeros(n)                       # dosage * weight to add
            kind = np.zeros(n, np.int8)             # 0 add, 1 missing, 2 fatal
            used: List[Optional[Heuristic]] = [None] * n
            inters: List[list] = []
            for j in range(n):
                inter = [(int(b), c) for b, c in zip(pats[j], ctxs)
                         if int(b) != 0b01 and pair_matches(si, c[1], c[2])]
                inters.append(inter)
                if not inter:
                    kind[j] = 1
                elif len(inter) == 1:
                    d = score_dosage(inter[0][0], inter[0][1][1], inter[0][1][2], si)
                    if d is None:
                        kind[j] = 1
                    else:
                        add[j] = d * w
                else:
                    r = resolve_conflict(si, inter)
                    if r is None:
                        kind[j] = 2
                    else:
                        add[j] = r[0] * w
                        used[j] = r[1]
            if (kind == 2).any():
                p = int(np.flatnonzero(kind[inv] == 2)[0])
                raise ComplexResolutionError(
                    "Compute", _fatal_report(iid(p), rule, score_names[col], inters[inv[p]]))
            per = kind[inv]
            sel = per == 0
            S[sel, col] += add[inv[sel]]
            C[per == 1, col] += 1
            hcode = np.array([-1 if u is None else u.value for u in used], np.int64)[inv]
            for h in Heuristic:
                people = np.flatnonzero(hcode == h.value)
                if not people.size:
                    continue
                report.counts[h] = report.counts.get(h, 0) + int(people.size)
                smp = report.samples.setdefault(h, [])
                for p in people[: max(0, 5 - len(smp))]:
                    smp.append((iid(int(p)), rule.locus_chr_pos, score_names[col]))
    return report
