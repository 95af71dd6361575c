"""Shared test helpers: fixtures -> PreparationResult, synthetic cases."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from gnomon_b200.prepare import PreparationResult, fold_cells
from gnomon_b200 import synth

GOLDEN = Path(__file__).resolve().parent / "golden"


def known_answer_cases():
    return json.loads((GOLDEN / "known_answers.json").read_text())


def case_prep(case) -> tuple[PreparationResult, np.ndarray]:
    """Engine case (known_answers.json) -> (prep, rows [V, pitch])."""
    P, K = case["num_people"], case["num_scores"]
    rows = np.array(case["rows"], dtype=np.uint8)
    cells = np.array(case["cells"], dtype=np.float64)
    V = rows.shape[0]
    order = np.lexsort((cells[:, 1], cells[:, 0]))
    cells = cells[order]
    counts = np.bincount(cells[:, 0].astype(np.int64), minlength=V)
    offs = np.zeros(V + 1, np.uint64)
    np.cumsum(counts, out=offs[1:])
    prep = PreparationResult(cells[:, 2].astype(np.float32), cells[:, 3].astype(np.float32),
                             cells[:, 1].astype(np.uint32), offs,
                             [f"S{k:03d}" for k in range(K)], P)
    return prep, rows


def expected_final(case, prep):
    partial = np.array(case["partial_sums"], dtype=np.float64)
    K = case["num_scores"]
    return partial + np.tile(prep.baseline, len(partial) // K), np.array(case["counts"], np.uint32)


def cohort_prep(n_scores=16):
    """score/tests/gpu_tests.rs cohort: prep + rows."""
    z = np.load(GOLDEN / "gpu_tests_cohort.npz")
    packed, w, flipped = z["packed"], z["weights"][:, :n_scores], z["flipped"]
    V, K = w.shape
    rows = np.repeat(np.arange(V), K)
    cols = np.tile(np.arange(K), V)
    dw, mc, c, offs = fold_cells(rows, cols, w.reshape(-1), np.repeat(flipped, K), V)
    prep = PreparationResult(dw, mc, c, offs, [f"S{k:03d}" for k in range(K)], 512)
    return prep, packed


def synth_case(people, variants, scores=1, config="plain_2k_x_50k", pitch=None, seed_offset=0):
    """Scaled synthetic workload: (workload, prep, rows [V, pitch])."""
    from gnomon_b200.prepare import from_workload
    base = synth.WORKLOADS[config]
    w = synth.scaled(base, people, variants, scores)
    if seed_offset:
        w = synth.Workload(w.name, w.people, w.variants, w.scores, w.p_lo, w.p_hi,
                           w.missing_rate, w.sigma, w.flip_frac, w.size_lo, w.size_hi,
                           w.config_id + 1000 * seed_offset)
    prep = from_workload(w)
    thr = synth.variant_thresholds(w.seed, 0, variants, w.p_lo, w.p_hi, w.missing_rate)
    bpv = (people + 3) // 4
    rows = synth.synth_rows(w.seed, 0, variants, people, thr, pitch or bpv)
    return w, prep, rows, thr
