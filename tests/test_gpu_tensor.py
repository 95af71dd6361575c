"""Split-BF16 tcgen05 engine on the GPU versus the CPU oracle (through the C ABI)."""
import numpy as np
import pytest

from gnomon_b200 import _lib
from gnomon_b200.pipeline import PipelineContext, ScoreCheckpoint, run
from gnomon_b200.prepare import PreparationResult
from helpers import case_prep, expected_final, known_answer_cases, synth_case
from oracle import oracle

pytestmark = pytest.mark.gpu
TENSOR = _lib.ENGINE_TENSOR
CASES = known_answer_cases()["engine_cases"]
# Limb quantisation leaves each weight within 2^-25 of its score's largest
# weight; every FP32 block sum is exact and the cross-block sum is FP64.
TOL = 1e-7


def host_run(prep, rows, **kw):
    return run(PipelineContext(prep), np.ascontiguousarray(rows).reshape(-1), engine=TENSOR, **kw)


def check(prep, rows, got):
    s, c = got
    es, ec = oracle.score_extended(rows, prep)
    np.testing.assert_array_equal(c, ec)
    err = oracle.rel_err(s, es).max()
    assert err < TOL, f"max rel err vs extended oracle {err:.3e}"
    rs, rc = oracle.score_reference(rows, prep, threads=4)
    assert oracle.within_reference_tolerance(s, rs).all()
    return err


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_known_answers(cuda, case):
    prep, rows = case_prep(case)
    s, c = host_run(prep, rows)
    ws, wc = expected_final(case, prep)
    np.testing.assert_allclose(s, ws, rtol=0, atol=1e-9)
    np.testing.assert_array_equal(c, wc)


def test_single_tile(cuda):
    _, prep, rows, _ = synth_case(256, 128, scores=128, config="batched_100k_x_500k_k512")
    check(prep, rows, host_run(prep, rows))


@pytest.mark.parametrize("people,variants,scores", [(1000, 1000, 300), (129, 65, 129),
                                                    (4099, 700, 40)])
def test_ragged_tiles(cuda, people, variants, scores):
    _, prep, rows, _ = synth_case(people, variants, scores=scores,
                                  config="batched_100k_x_500k_k512")
    check(prep, rows, host_run(prep, rows))


@pytest.mark.parametrize("scores", [130, 20])   # wide (score rows as M) and narrow engines
def test_block_flush_past_16k_variants(cuda, scores):
    _, prep, rows, _ = synth_case(300, 40_000, scores=scores, config="batched_100k_x_500k_k512")
    check(prep, rows, host_run(prep, rows))


def test_large_weights_exactness(cuda):
    """Weights of magnitude ~1 with 6.5% missing and 20% flipped variants (the
    reference cohort, score/tests/gpu_tests.rs:523-628): the three-limb
    missing-correction residual (2^-25 of the largest weight per missing
    flipped call) stays inside the reference's 1e-6 tolerance."""
    from helpers import cohort_prep
    prep, rows = cohort_prep(16)
    s, c = host_run(prep, rows)
    es, ec = oracle.score_extended(rows, prep)
    np.testing.assert_array_equal(c, ec)
    assert oracle.rel_err(s, es).max() < 1e-6


def test_streaming_and_unaligned_resume(cuda):
    _, prep, rows, _ = synth_case(700, 3000, scores=20, config="batched_100k_x_500k_k512")
    full = host_run(prep, rows)
    streamed = host_run(prep, rows, block_variants=1000)   # rounded up to 1024
    np.testing.assert_array_equal(streamed[1], full[1])
    assert oracle.rel_err(streamed[0], full[0]).max() < 1e-12
    cut = 1000  # not a multiple of 64
    offs = prep.sparse_row_offsets
    head = PreparationResult(prep.sparse_weights[:offs[cut]],
                             prep.sparse_missing_corrections[:offs[cut]],
                             prep.sparse_score_columns[:offs[cut]], offs[:cut + 1],
                             prep.score_names, 700, baseline=prep.baseline)
    hs, hc = oracle.score_extended(rows[:cut], head)
    got = run(PipelineContext(prep, ScoreCheckpoint(cut, hs, hc)), rows.reshape(-1),
              engine=TENSOR)
    np.testing.assert_array_equal(got[1], full[1])
    assert oracle.rel_err(got[0], full[0]).max() < 1e-7


def test_keep_subset(cuda):
    rng = np.random.default_rng(3)
    _, prep, rows, _ = synth_case(2000, 500, scores=64, config="batched_100k_x_500k_k512")
    keep = rng.choice(2000, 700, replace=False).astype(np.uint32)
    p2 = PreparationResult(prep.sparse_weights, prep.sparse_missing_corrections,
                           prep.sparse_score_columns, prep.sparse_row_offsets, prep.score_names,
                           2000, output_idx_to_fam_idx=keep)
    check(p2, rows, host_run(p2, rows))


def test_tensor_matches_plain(cuda):
    _, prep, rows, _ = synth_case(1500, 800, scores=24, config="batched_100k_x_500k_k512")
    t = host_run(prep, rows)
    p = run(PipelineContext(prep), rows.reshape(-1), engine=_lib.ENGINE_PLAIN)
    np.testing.assert_array_equal(t[1], p[1])
    assert oracle.rel_err(t[0], p[0]).max() < 1e-6


def _condition(prep, rows):
    """sum_v |w'_vk d_pv| + |corr_vk| m_pv per (p, k): the scale of each sum's terms."""
    from gnomon_b200 import synth
    P, K, V = prep.total_people_in_fam, prep.num_scores, prep.num_reconciled_variants
    codes = synth.unpack_codes(rows, P).astype(np.int64)       # [V, P]
    d = np.where(codes == 2, 1.0, np.where(codes == 3, 2.0, 0.0))
    m = (codes == 1).astype(np.float64)
    W = np.zeros((V, K))
    C = np.zeros((V, K))
    offs = prep.sparse_row_offsets.astype(np.int64)
    vrow = np.repeat(np.arange(V), np.diff(offs))
    W[vrow, prep.sparse_score_columns] = np.abs(prep.sparse_weights)
    C[vrow, prep.sparse_score_columns] = np.abs(prep.sparse_missing_corrections)
    return (d.T @ W + m.T @ C).reshape(-1)


@pytest.mark.parametrize("config,people,variants", [("plain_2k_x_50k", 2000, 50_000),
                                                    ("bandwidth_50k_x_1m", 4096, 100_000),
                                                    ("batched_100k_x_500k_k512", 256, 40_000),
                                                    ("diff_20k_x_200k_k16", 1024, 50_000),
                                                    ("biobank_500k_x_1p2m_k64", 512, 60_000)])
def test_error_report_workload_subsets(cuda, config, people, variants):
    """Error report of both engines on the named workloads (the 2,000 x 50,000
    one at full size, the others as subsets with all of their scores): max
    relative error (the reference's metric) and, for the split-BF16 engine,
    the error relative to the sum of |terms|, against the extended-precision
    oracle.  Printed as one ERROR_REPORT line per workload (pytest -s)."""
    import json
    _, prep, rows, _ = synth_case(people, variants, scores=None, config=config)
    s, c = host_run(prep, rows)
    es, ec = oracle.score_extended(rows, prep)
    np.testing.assert_array_equal(c, ec)
    rel = oracle.rel_err(s, es)
    cond = np.abs(s - es) / np.maximum(_condition(prep, rows), 1e-300)
    ps, pc = run(PipelineContext(prep), np.ascontiguousarray(rows).reshape(-1),
                 engine=_lib.ENGINE_PLAIN)
    print("ERROR_REPORT " + json.dumps({
        "workload": config, "people": people, "variants": variants,
        "scores": prep.num_scores, "tensor_max_rel_err": float(rel.max()),
        "tensor_max_err_over_sum_abs_terms": float(cond.max()),
        "plain_max_rel_err": float(oracle.rel_err(ps, es).max())}))
    assert rel.max() < TOL
    np.testing.assert_array_equal(pc, ec)
    assert oracle.within_reference_tolerance(ps, es).all()


@pytest.mark.parametrize("scores,engine", [(7, _lib.ENGINE_PLAIN), (8, _lib.ENGINE_TENSOR)])
def test_auto_engine_rule(cuda, scores, engine):
    """Default options: plain kernel below 8 score columns, tensor engine from
    8.  Either way the drop-in call's counts are exact and its sums are within
    the reference's tolerance of the restated reference engine."""
    from gnomon_b200.device import DevicePlan
    _, prep, rows, _ = synth_case(1500, 900, scores=scores, config="batched_100k_x_500k_k512")
    plan = DevicePlan(prep)   # AUTO
    try:
        assert plan.engine == engine
    finally:
        plan.close()
    s, c = run(PipelineContext(prep), np.ascontiguousarray(rows).reshape(-1))
    rs, rc = oracle.score_reference(rows, prep, threads=4)
    np.testing.assert_array_equal(c, rc)
    assert oracle.within_reference_tolerance(s, rs).all()


def test_large_csr_and_results_through_pinned_ring(cuda):
    """The end-to-end call uploads a CSR above 128 MB per array, and copies
    results above 128 MB back, through its pinned host ring (host threads
    fill or drain one 64 MB chunk while the DMA moves the other). Both
    directions are checked against the restated reference engine."""
    # 256 people x 131,072 variants x 256 dense scores: 33.5 M cells, 134 MB per CSR array
    _, prep, rows, _ = synth_case(256, 131_072, scores=256, config="diff_20k_x_200k_k16")
    assert prep.sparse_weights.nbytes >= (128 << 20)   # the ring is used from 128 MiB
    s, c = host_run(prep, rows)
    rs, rc = oracle.score_reference(rows, prep, threads=8)
    np.testing.assert_array_equal(c, rc)
    assert oracle.within_reference_tolerance(s, rs).all()
    # 131,072 people x 256 variants x 128 scores: 134 MB of FP64 sums
    _, prep, rows, _ = synth_case(131_072, 256, scores=128, config="diff_20k_x_200k_k16")
    s, c = host_run(prep, rows)
    assert s.nbytes >= (128 << 20)
    rs, rc = oracle.score_reference(rows, prep, threads=8)
    np.testing.assert_array_equal(c, rc)
    assert oracle.within_reference_tolerance(s, rs).all()
