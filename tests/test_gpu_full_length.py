"""Every named workload at its full variant length and with all of its scores,
on a subset of its people, through the drop-in host call (``gnm_score_run``)
with both engines, against the CPU oracle.

The engines round inside blocks (the plain kernel's int32 stage grid, the
split-BF16 and 8-bit limb residuals) and sum in FP64 across them, so the
error of a sum depends on how many blocks it crosses: only full-length runs
give the per-workload error figures.  ``tensor`` is the engine's default
(8-bit limbs; the narrow kernel up to 64 scores, else the wide kernel);
``tensor_i8``, ``tensor_i8_pair`` and ``tensor_bf16`` pin the wide kernel on
8-bit limbs (one SM per tile, SM pairs) and on BF16 limbs, and
``tensor_narrow_bf16`` the narrow kernel on BF16 limbs, through a device
plan.  People are the first ``people`` of each cohort
(the generator keys every call by (variant, person), so these are exactly the
full workload's genotypes for those people); weights and score subsets are
the full workload's.

Checks, per workload and engine:
* missing counts bit-exact against the extended-precision oracle;
* plain-engine sums within the reference's tolerance (|d| <= 1e-6 or
  |d| / max(|a|, |b|, 1) <= 1e-6, score/tests/gpu_tests.rs:11-13, 135-147)
  against the restated reference engine and against the extended oracle;
* split-BF16 sums within 1e-6 relative (the same metric) of the extended
  oracle.

Each case prints one ``ERROR_REPORT`` JSON line (pytest -s) with the maximum
relative errors and, for the split-BF16 engine, the error over the sum of the
terms' magnitudes.
"""
import json
import os

import numpy as np
import pytest

from gnomon_b200 import _lib, synth
from gnomon_b200.pipeline import PipelineContext, run
from gnomon_b200.prepare import from_workload
from oracle import oracle

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 1

# workload -> people kept (all variants, all scores)
FULL_LENGTH = {
    "bandwidth_50k_x_1m": 2_048,
    "batched_100k_x_500k_k512": 256,
    "diff_20k_x_200k_k16": 1_024,
    "biobank_500k_x_1p2m_k64": 256,
}

_cache = {}


def full_length_case(name):
    """(workload, prep, rows [V, bpv], extended (sums, counts)) for the first
    FULL_LENGTH[name] people of the named workload; built once per session."""
    if name not in _cache:
        base = synth.WORKLOADS[name]
        w = synth.scaled(base, FULL_LENGTH[name], base.variants)
        assert (w.size_lo, w.size_hi, w.scores) == (base.size_lo, base.size_hi, base.scores)
        prep = from_workload(w)
        thr = synth.variant_thresholds(w.seed, 0, w.variants, w.p_lo, w.p_hi, w.missing_rate)
        rows = oracle.synth_rows(w.seed, 0, w.variants, w.people, thr, w.bytes_per_variant,
                                 threads=THREADS)
        ext = oracle.score_extended(rows, prep, threads=THREADS)
        _cache.clear()   # one workload resident at a time (the batched CSR is 1.6 GB)
        _cache[name] = (w, prep, rows, ext)
    return _cache[name]


def sum_abs_terms(prep, rows, people):
    """sum_v |w'_vk| d_pv + |corr_vk| m_pv for every (p, k): the scale of each
    sum's terms, accumulated in blocks of variants."""
    P, K, V = people, prep.num_scores, prep.num_reconciled_variants
    out = np.zeros((P, K))
    offs = prep.sparse_row_offsets.astype(np.int64)
    for v0 in range(0, V, 16_384):
        v1 = min(V, v0 + 16_384)
        codes = synth.unpack_codes(rows[v0:v1], P).astype(np.int64)
        d = np.where(codes == 2, 1.0, np.where(codes == 3, 2.0, 0.0))
        m = (codes == 1).astype(np.float64)
        e0, e1 = offs[v0], offs[v1]
        vrow = np.repeat(np.arange(v1 - v0), np.diff(offs[v0:v1 + 1]))
        W = np.zeros((v1 - v0, K))
        C = np.zeros((v1 - v0, K))
        W[vrow, prep.sparse_score_columns[e0:e1]] = np.abs(prep.sparse_weights[e0:e1])
        C[vrow, prep.sparse_score_columns[e0:e1]] = np.abs(prep.sparse_missing_corrections[e0:e1])
        out += d.T @ W + m.T @ C
    return out.reshape(-1)


def score_shape(prep, rows, shape):
    """The tensor engine pinned to a shape (gnm_plan_set_shape bits), through
    a device plan."""
    import torch
    from gnomon_b200.device import DevicePlan, row_pitch
    bpv = prep.bytes_per_variant
    pitch = row_pitch(bpv)
    d = torch.zeros((rows.shape[0], pitch), dtype=torch.uint8, device="cuda")
    d[:, :bpv] = torch.from_numpy(np.ascontiguousarray(rows[:, :bpv])).cuda()
    plan = DevicePlan(prep, engine=_lib.ENGINE_TENSOR)
    plan.set_shape(shape)
    s, c = plan.score(d, pitch)
    plan.sync()
    out = s.cpu().numpy(), c.cpu().numpy().astype(np.uint32)
    plan.close()
    return out


SHAPES = {"tensor_i8": 4, "tensor_i8_pair": 12, "tensor_bf16": 0, "tensor_narrow_bf16": 2}


@pytest.mark.parametrize("engine", ["plain", "tensor", "tensor_i8", "tensor_i8_pair",
                                    "tensor_bf16", "tensor_narrow_bf16"])
@pytest.mark.parametrize("name", list(FULL_LENGTH))
def test_full_length_parity(cuda, name, engine):
    if engine == "tensor_narrow_bf16" and synth.WORKLOADS[name].scores > 64:
        pytest.skip("the narrow kernel serves at most 64 scores")
    w, prep, rows, (es, ec) = full_length_case(name)
    if engine in SHAPES:
        s, c = score_shape(prep, rows, SHAPES[engine])
    else:
        eng = _lib.ENGINE_PLAIN if engine == "plain" else _lib.ENGINE_TENSOR
        s, c = run(PipelineContext(prep), np.ascontiguousarray(rows).reshape(-1), engine=eng)
    np.testing.assert_array_equal(c, ec)
    rel = oracle.rel_err(s, es)
    report = {"workload": name, "engine": engine, "people": w.people, "variants": w.variants,
              "scores": w.scores, "cells": int(prep.sparse_row_offsets[-1]),
              "max_rel_err_vs_extended": float(rel.max()),
              "mean_rel_err_vs_extended": float(rel.mean())}
    if engine == "plain":
        rs, rc = oracle.score_reference(rows, prep, threads=THREADS)
        np.testing.assert_array_equal(rc, ec)
        report["max_rel_err_vs_restatement"] = float(oracle.rel_err(s, rs).max())
        assert oracle.within_reference_tolerance(s, rs).all()
        assert oracle.within_reference_tolerance(s, es).all()
    else:
        scale = sum_abs_terms(prep, rows, w.people)
        report["max_err_over_sum_abs_terms"] = float((np.abs(s - es) / np.maximum(scale, 1e-300)).max())
        assert rel.max() <= 1e-6
    print("ERROR_REPORT " + json.dumps(report))
