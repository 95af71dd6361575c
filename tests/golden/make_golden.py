"""Generate the golden fixtures under tests/golden/.

Sources (SauersML/gnomon, read as text; the Rust code cannot run here):

* known_answers.json — the reference's own known-answer unit tests, restated
  as full engine inputs with their asserted outputs:
    - score/batch.rs:1013-1036  one byte 0b01_11_10_00, w=1.5, corr=2.0
      -> partial sums [0, 1.5, 3.0, -2.0], missing [0, 0, 0, 1]
    - score/batch.rs:1039-1066  101 people, calls at people 3/32/99/100
    - score/batch.rs:1069-1114  577 scores, dosages 1/2/0
    - score/prepare.rs:1041-1097 flip aggregation
  The engine returns baseline + partial (pipeline.rs:1739-1775); the
  baseline of these fixtures is the sum of their missing corrections
  (prepare.rs:644-646), so expected finals are baseline + the asserted
  partials.
* gpu_tests_cohort.npz — the deterministic cohort of
  score/tests/gpu_tests.rs:523-628 (genotype key (p*131 + v*17 + 23) % 31,
  weights ((v*31 + s*17 + 7) % 29 - 14)/10 printed with 8 decimals, every
  5th variant's effect allele = BIM allele1), 512 people x 256 variants x
  16 scores, used by the reference's GPU-vs-CPU parity test.
* ld_fixture.npz — the packed rows of data/testdata/ld.bed (200 samples x
  1500 variants, real PLINK bytes), for decode parity.  Copied only when the
  reference tree is present at generation time.
* ld_pgen_fixture.npz — the bytes of data/testdata/ld_p.pgen, the same
  genotypes as a PLINK 2 variable-width .pgen (LD-compressed and 1-bit
  records), for PGEN decode parity against ld_fixture.npz.
* ld_projection_fixture.npz — one HWE-PCA projection block over the real
  ld.bed rows (all 1,500 variants, 200 samples, 6 axes): coefficients from
  the rows' own allele frequencies ((g - 2p) / sqrt(2p(1-p)), map/project.rs
  :2960-2975; every 7th variant allele-swapped), seeded loadings, and the
  expected scores from the float64 restatement of the reference's block
  projection (map/project.rs:322-370, 547-667), frozen here so that the
  kernel and the restatement are both held to the same numbers.

Run: python tests/golden/make_golden.py --reference <path of the reference checkout>
"""
from __future__ import annotations

import argparse
import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def pack(codes_by_person):
    """codes_by_person: list of 2-bit codes (person order) -> packed row bytes."""
    n = len(codes_by_person)
    row = [0] * ((n + 3) // 4)
    for p, c in enumerate(codes_by_person):
        row[p // 4] |= c << (2 * (p % 4))
    return row


def known_answers():
    cases = []
    # batch.rs:1013-1036 -- p0=00, p1=10, p2=11, p3=01
    cases.append(dict(
        name="batch_rs_1013_single_byte",
        cite="score/batch.rs:1013-1036",
        num_people=4, num_scores=1,
        rows=[[0b01_11_10_00]],
        cells=[[0, 0, 1.5, 2.0]],          # (variant, score, dosage_weight, missing_correction)
        partial_sums=[0.0, 1.5, 3.0, -2.0],
        counts=[0, 0, 0, 1],
    ))
    # batch.rs:1039-1066 -- 101 people, (3,code2),(32,code3),(99,code1),(100,code2)
    codes = [0] * 101
    for p, g in [(3, 2), (32, 3), (99, 1), (100, 2)]:
        codes[p] = g
    partial = [0.0] * 101
    partial[3], partial[32], partial[99], partial[100] = 1.5, 3.0, -2.0, 1.5
    cnt = [0] * 101
    cnt[99] = 1
    cases.append(dict(
        name="batch_rs_1039_tail_byte",
        cite="score/batch.rs:1039-1066",
        num_people=101, num_scores=1, rows=[pack(codes)],
        cells=[[0, 0, 1.5, 2.0]], partial_sums=partial, counts=cnt))
    # batch.rs:1069-1114 -- 3 people x 577 scores, weights 1.0, corrections 0;
    # person dosages 1, 2, 0 -> PLINK codes 10, 11, 00
    K = 577
    cases.append(dict(
        name="batch_rs_1069_577_scores",
        cite="score/batch.rs:1069-1114",
        num_people=3, num_scores=K, rows=[pack([2, 3, 0])],
        cells=[[0, k, 1.0, 0.0] for k in range(K)],
        partial_sums=[1.0] * K + [2.0] * K + [0.0] * K,
        counts=[0] * (3 * K)))
    return cases


def flip_cases():
    """prepare.rs:1041-1097 folding cases: records -> (dosage_weight, missing_correction)."""
    return [
        dict(cite="score/prepare.rs:1041-1052", records=[[0.25, False], [-0.10, False]],
             dosage_weight=0.15, missing_correction=0.0, tol=1e-6),
        dict(cite="score/prepare.rs:1055-1065", records=[[0.40, True]],
             dosage_weight=-0.40, missing_correction=0.80, tol=1e-6),
        dict(cite="score/prepare.rs:1068-1097",
             records=[[0.35, False], [0.10, True], [-0.05, False]],
             row_by_row=True, tol=1e-6),
    ]


def gpu_tests_cohort(n_people=512, n_variants=256, n_scores=16):
    """score/tests/gpu_tests.rs:523-628 generator."""
    code_of = {"missing": 1, 0: 0, 1: 2, 2: 3}
    codes = np.zeros((n_variants, n_people), dtype=np.uint8)
    for v in range(n_variants):
        for p in range(n_people):
            key = (p * 131 + v * 17 + 23) % 31
            if key in (0, 1):
                g = "missing"
            elif key <= 9:
                g = 0
            elif key <= 20:
                g = 1
            else:
                g = 2
            codes[v, p] = code_of[g]
    bpv = (n_people + 3) // 4
    packed = np.zeros((n_variants, bpv), dtype=np.uint8)
    for q in range(4):
        packed |= (codes[:, q::4] << (2 * q)).astype(np.uint8)
    # weights printed with "{weight:.8}" then parsed as f32
    w = np.zeros((n_variants, n_scores), dtype=np.float32)
    for v in range(n_variants):
        for s in range(n_scores):
            base = float((v * 31 + s * 17 + 7) % 29)
            w[v, s] = np.float32(float(f"{(base - 14.0) / 10.0:.8f}"))
    flipped = np.array([v % 5 == 0 for v in range(n_variants)])  # effect A == BIM allele1 A
    return packed, w, flipped


def ld_projection(rows: np.ndarray, n_people: int, axes: int = 6, seed: int = 2027):
    import sys
    sys.path.insert(0, str(HERE.parents[1]))
    from oracle import project_oracle
    bpv = (n_people + 3) // 4
    codes = np.stack([(rows >> (2 * s)) & 3 for s in range(4)], axis=-1).reshape(rows.shape[0], -1)
    codes = codes[:, :n_people]
    g = np.choose(codes, [0.0, np.nan, 1.0, 2.0])           # A2 copies; code 01 missing
    p = np.nanmean(g, axis=1) / 2.0
    scale = np.sqrt(2.0 * p * (1.0 - p))
    inv = np.where(scale > 0, 1.0 / np.where(scale > 0, scale, 1.0), 0.0)
    c = (np.arange(3.0)[None, :] - 2.0 * p[:, None]) * inv[:, None]
    c[::7] = c[::7, ::-1]
    coeffs = c.astype(np.float32)
    rng = np.random.default_rng(seed)
    loadings = (rng.standard_normal((rows.shape[0], axes)) / np.sqrt(rows.shape[0])).astype(np.float32)
    scores = project_oracle.project_block(rows.reshape(-1, bpv), n_people, coeffs, loadings)
    return coeffs, loadings, scores


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="root of the reference source tree (read-only)")
    a = ap.parse_args()
    (HERE / "known_answers.json").write_text(json.dumps(
        {"engine_cases": known_answers(), "flip_cases": flip_cases()}, indent=1))
    packed, w, flipped = gpu_tests_cohort()
    np.savez_compressed(HERE / "gpu_tests_cohort.npz", packed=packed, weights=w, flipped=flipped)
    ld = Path(a.reference) / "data" / "testdata" / "ld.bed"
    if ld.exists():
        raw = np.frombuffer(ld.read_bytes(), dtype=np.uint8)
        assert bytes(raw[:3]) == bytes([0x6C, 0x1B, 0x01]), "ld.bed magic"
        n_people, n_var = 200, 1500
        bpv = (n_people + 3) // 4
        rows = raw[3:].reshape(n_var, bpv)
        np.savez_compressed(HERE / "ld_fixture.npz", rows=rows, num_people=n_people)
    if (HERE / "ld_fixture.npz").exists():
        f = np.load(HERE / "ld_fixture.npz")
        coeffs, loadings, scores = ld_projection(f["rows"], int(f["num_people"]))
        np.savez_compressed(HERE / "ld_projection_fixture.npz", coeffs=coeffs, loadings=loadings,
                            scores=scores)
    pg = Path(a.reference) / "data" / "testdata" / "ld_p.pgen"
    if pg.exists():
        np.savez_compressed(HERE / "ld_pgen_fixture.npz",
                            pgen=np.frombuffer(pg.read_bytes(), dtype=np.uint8))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
