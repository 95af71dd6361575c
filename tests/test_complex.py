"""Complex-variant resolution (score/complex.rs): the reference's own
known-answer cases for the heuristic chain, and the vectorised pass against a
literal per-person restatement of the reference loop."""
from __future__ import annotations

import numpy as np
import pytest

from gnomon_b200.complex import (GenotypeSource, GroupedComplexRule, Heuristic, ScoreInfo,
                                 resolve_complex_variants, resolve_conflict, score_dosage,
                                 try_heuristic, pair_matches)


def si(ea, oa, col=0, w=1.0):
    return ScoreInfo(ea, oa, w, col)


# ---- complex.rs:287-492 known answers -------------------------------------------

def test_heterozygous_fallback_last():
    res = resolve_conflict(si("T", "A"), [(0b00, (10, "A", "T")), (0b11, (11, "A", "T"))])
    assert res[1] is Heuristic.FallbackOpposingHomozygousAsHet
    assert abs(res[0] - 1.0) < 1e-9


def test_existing_priority_over_fallback():
    res = resolve_conflict(si("A", "G"), [(0b10, (20, "A", "G")), (0b11, (21, "A", "T"))])
    assert res[1] is Heuristic.ExactScoreAlleleMatch


def test_fallback_het_requires_both_homozygous_states():
    assert try_heuristic(Heuristic.FallbackOpposingHomozygousAsHet, si("A", "G"),
                         [(0b00, (30, "A", "C")), (0b10, (31, "A", "T"))]) is None


def test_fallback_het_dosage_matches_inferred_pair():
    inter = [(0b00, (40, "C", "T")), (0b11, (41, "C", "T"))]
    h = Heuristic.FallbackOpposingHomozygousAsHet
    assert try_heuristic(h, si("G", "A"), inter) is None
    assert abs(try_heuristic(h, si("C", "T"), inter)[0] - 1.0) < 1e-9
    assert abs(try_heuristic(h, si("T", "C"), inter)[0] - 1.0) < 1e-9


def test_average_dosage_three_conflicts():
    inter = [(0b00, (50, "A", "T")), (0b10, (51, "A", "T")), (0b11, (52, "A", "T"))]
    res = try_heuristic(Heuristic.FallbackAverageDosageAcrossConflicts, si("T", "A"), inter)
    assert abs(res[0] - 1.0) < 1e-9


def test_average_only_as_last_resort():
    res = resolve_conflict(si("T", "A"), [(0b00, (60, "A", "T")), (0b11, (61, "A", "T"))])
    assert res[1] is Heuristic.FallbackOpposingHomozygousAsHet


def test_average_dosage_two_conflicts():
    res = resolve_conflict(si("T", "A"), [(0b00, (70, "A", "T")), (0b00, (71, "T", "A"))])
    assert res[1] is Heuristic.FallbackAverageDosageAcrossConflicts
    assert abs(res[0] - 1.0) < 1e-9


# ---- further cases of the chain ------------------------------------------------

def test_indel_anchor_base_infers_het():
    # C/C from one row and CAGA/CAGA from another: short/long prefix pair -> het
    inter = [(0b00, (1, "C", "CAGA")), (0b11, (2, "C", "CAGA"))]
    assert try_heuristic(Heuristic.IndelAnchorBase, si("CAGA", "C"), inter) == \
        (1.0, Heuristic.IndelAnchorBase)
    # a third unrelated homozygous allele spoils the evidence
    inter3 = inter + [(0b00, (3, "G", "CAGA"))]
    assert try_heuristic(Heuristic.IndelAnchorBase, si("CAGA", "C"), inter3) is None


def test_matching_structure_and_unambiguous():
    s = si("A", "AT")
    inter = [(0b00, (1, "A", "AT")), (0b00, (2, "AT", "A"))]
    # both rows are exact matches: exact and unambiguous do not decide
    assert try_heuristic(Heuristic.ExactScoreAlleleMatch, s, inter) is None
    assert try_heuristic(Heuristic.PrioritizeUnambiguousGenotype, s, inter) is None
    # A/A (lengths 1,1) vs AT/AT (2,2): neither matches the score's (1,2)
    assert try_heuristic(Heuristic.PreferMatchingAlleleStructure, s, inter) is None
    het = [(0b10, (1, "A", "AT")), (0b00, (2, "AT", "A"))]
    assert try_heuristic(Heuristic.PreferMatchingAlleleStructure, s, het) == \
        (1.0, Heuristic.PreferMatchingAlleleStructure)


def test_score_dosage_orientation():
    s = si("G", "A")
    assert score_dosage(0b00, "G", "A", s) == 2.0
    assert score_dosage(0b00, "A", "G", s) == 0.0
    assert score_dosage(0b10, "A", "G", s) == 1.0
    assert score_dosage(0b11, "A", "G", s) == 2.0
    assert score_dosage(0b11, "A", "T", s) is None


# ---- the vectorised pass against a per-person loop ---------------------------------

def _per_person_loop(rules, codes_of, fam, K, S, C):
    """complex.rs:1060-1248, one person at a time."""
    for p in range(len(fam)):
        for rule in rules:
            valid = []
            for ctx in rule.possible_contexts:
                bits = codes_of(ctx[0], fam[p])
                if bits != 0b01:
                    valid.append((bits, ctx))
            for s in rule.score_applications:
                match = [v for v in valid if pair_matches(s, v[1][1], v[1][2])]
                col = s.score_column_index
                w = float(np.float32(s.weight))
                if not match:
                    C[p, col] += 1
                elif len(match) == 1:
                    d = score_dosage(match[0][0], match[0][1][1], match[0][1][2], s)
                    if d is None:
                        C[p, col] += 1
                    else:
                        S[p, col] += d * w
                else:
                    r = resolve_conflict(s, match)
                    assert r is not None
                    S[p, col] += r[0] * w


def _random_case(seed, P=257, V=40, K=3, n_rules=18):
    rng = np.random.default_rng(seed)
    bpv = (P + 3) // 4
    codes = rng.choice(4, size=(V, P), p=[0.45, 0.05, 0.35, 0.15]).astype(np.uint8)
    padded = np.zeros((V, bpv * 4), np.uint8)
    padded[:, :P] = codes
    q = padded.reshape(V, bpv, 4)
    rows = (q[:, :, 0] | (q[:, :, 1] << 2) | (q[:, :, 2] << 4) | (q[:, :, 3] << 6)).astype(np.uint8)
    alleles = ["A", "C", "G", "T", "AT", "CAGA", "C"]
    rules = []
    for r in range(n_rules):
        n_ctx = int(rng.integers(1, 5))
        ctxs = []
        for i, c in enumerate(rng.choice(V, n_ctx, replace=False)):
            if i > 0 and rng.random() < 0.6:     # same locus described twice: conflicts
                a1, a2 = ctxs[0][1:] if rng.random() < 0.5 else ctxs[0][:0:-1]
            else:
                a1, a2 = rng.choice(alleles, 2, replace=False)
            ctxs.append((int(c), str(a1), str(a2)))
        apps = []
        for k in range(K):
            if rng.random() < 0.7:
                base = ctxs[int(rng.integers(len(ctxs)))]
                ea, oa = (base[1], base[2]) if rng.random() < 0.5 else (base[2], base[1])
            else:
                ea, oa = (str(x) for x in rng.choice(alleles, 2, replace=False))
            apps.append(ScoreInfo(ea, oa, float(np.float32(rng.normal())), k))
        rules.append(GroupedComplexRule(("1", 1000 + r), ctxs, apps))
    return rows.reshape(-1), codes, rules, bpv


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("subset", [False, True])
def test_vectorised_pass_matches_per_person_loop(seed, subset):
    rows, codes, rules, bpv = _random_case(seed)
    P, K = codes.shape[1], 3
    fam = np.arange(P) if not subset else \
        np.random.default_rng(seed).permutation(P)[:180]
    n = len(fam)
    rng = np.random.default_rng(seed + 100)
    S0 = rng.normal(size=(n, K))
    C0 = rng.integers(0, 5, size=(n, K)).astype(np.uint32)
    S, C = S0.copy().reshape(-1), C0.copy().reshape(-1)
    rep = resolve_complex_variants(rules, GenotypeSource.single(rows, bpv),
                                   None if not subset else fam.astype(np.uint32), n,
                                   ["S0", "S1", "S2"], S, C)
    S1, C1 = S0.copy(), C0.copy()
    _per_person_loop(rules, lambda r, f: int(codes[r, f]), fam, K, S1, C1)
    np.testing.assert_array_equal(S.reshape(n, K), S1)          # bit exact
    np.testing.assert_array_equal(C.reshape(n, K), C1)
    assert sum(rep.counts.values()) > 0
    for h, smp in rep.samples.items():
        assert 0 < len(smp) <= 5


def test_multi_fileset_source():
    rows, codes, rules, bpv = _random_case(9, V=40)
    split = 17
    r2 = rows.reshape(40, bpv)
    src = GenotypeSource([r2[:split].reshape(-1), r2[split:].reshape(-1)], [0, split], bpv)
    fam = np.arange(codes.shape[1])
    for v in (0, 16, 17, 39):
        np.testing.assert_array_equal(src.codes(v, fam), codes[v])
    with pytest.raises(IOError):
        GenotypeSource.single(rows[:-bpv], bpv).codes(39, fam)
