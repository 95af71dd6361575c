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


def test_block_flush_past_16k_variants(cuda):
    _, prep, rows, _ = synth_case(300, 40_000, scores=130, config="batched_100k_x_500k_k512")
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
