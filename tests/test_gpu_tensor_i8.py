"""The tensor engine on 8-bit integer limbs (tcgen05 kind::i8) against the CPU
oracle, through a device plan pinned to it with gnm_plan_set_shape: the wide
kernel on one SM per tile (gnm_t8_accumulate, shape bit 2) and on SM pairs
(gnm_t8_pair, cta_group::2, shape bits 2 and 3), and the narrow kernel
(gnm_t8_narrow, shape bits 1 and 2)."""
import numpy as np
import pytest
import torch

from gnomon_b200 import _lib
from gnomon_b200.device import DevicePlan, row_pitch
from helpers import case_prep, cohort_prep, expected_final, known_answer_cases, synth_case
from oracle import oracle

pytestmark = pytest.mark.gpu
I8, I8_SCORE_TILES_FIRST, BF16 = 4, 5, 0
PAIR, PAIR_SCORE_TILES_FIRST = 12, 13
NARROW8, NARROW_BF16 = 6, 2
I8_SHAPES = [I8, PAIR]
CASES = known_answer_cases()["engine_cases"]
# Four 8-bit limbs leave each weight and missing correction within 2^-31.9
# of its score's largest value; block sums are exact integers, the
# cross-block sum is FP64.
TOL = 1e-7


def device_rows(rows, bpv):
    pitch = row_pitch(bpv)
    V = rows.shape[0]
    d = torch.zeros((max(V, 1), pitch), dtype=torch.uint8, device="cuda")
    if V:
        d[:V, :bpv] = torch.from_numpy(np.ascontiguousarray(rows[:, :bpv])).cuda()
    return d, pitch


def plan_run(prep, rows, shape=I8, blocks=None):
    d, pitch = device_rows(rows, prep.bytes_per_variant)
    plan = DevicePlan(prep, engine=_lib.ENGINE_TENSOR)
    plan.set_shape(shape)
    assert plan.shape == shape
    if blocks is None:
        s, c = plan.score(d, pitch)
    else:
        plan.reset()
        for v0, n in blocks:
            plan.accumulate(d[v0:], pitch, v0, n)
        s, c = plan.outputs()
        plan.finalize(s, c)
    plan.sync()
    out = s.cpu().numpy(), c.cpu().numpy().astype(np.uint32)
    plan.close()
    return out


def check(prep, rows, got, tol=TOL):
    s, c = got
    es, ec = oracle.score_extended(rows, prep)
    np.testing.assert_array_equal(c, ec)
    err = oracle.rel_err(s, es).max()
    assert err < tol, f"max rel err vs extended oracle {err:.3e}"
    return err


@pytest.mark.parametrize("shape", I8_SHAPES + [NARROW8])
@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_known_answers(cuda, case, shape):
    prep, rows = case_prep(case)
    if shape & 2 and prep.num_scores > 64:
        pytest.skip("the narrow kernel serves at most 64 scores")
    s, c = plan_run(prep, rows, shape)
    ws, wc = expected_final(case, prep)
    np.testing.assert_allclose(s, ws, rtol=0, atol=1e-9)
    np.testing.assert_array_equal(c, wc)


@pytest.mark.parametrize("people,variants,scores,shape", [
    (256, 128, 128, I8), (1000, 1000, 300, I8), (129, 65, 129, I8_SCORE_TILES_FIRST),
    (4099, 700, 40, I8), (300, 40_000, 130, I8),
    (256, 128, 256, PAIR), (1000, 1000, 300, PAIR), (129, 65, 129, PAIR_SCORE_TILES_FIRST),
    (100, 700, 40, PAIR), (4099, 700, 520, PAIR_SCORE_TILES_FIRST), (300, 40_000, 130, PAIR),
    (256, 128, 16, NARROW8), (1000, 1000, 64, NARROW8), (129, 65, 17, NARROW8),
    (4099, 700, 40, NARROW8), (300, 40_000, 30, NARROW8)])
def test_against_the_oracle(cuda, people, variants, scores, shape):
    """Ragged people / score tiles and a partial last stage.  On SM pairs:
    an odd number of 128-score tiles (the last pair's second CTA holds no
    scores), a last people tile whose second half is partly filled or
    empty (129 and 100 people)."""
    _, prep, rows, _ = synth_case(people, variants, scores=scores,
                                  config="batched_100k_x_500k_k512")
    check(prep, rows, plan_run(prep, rows, shape))


@pytest.mark.parametrize("shape", I8_SHAPES + [NARROW8])
def test_blocks_past_the_flush(cuda, shape):
    """One call over more than 2^23 variants: the kernel drains its S32 sums
    into the FP64 partials at the 2^23-variant block end, restarts them, and
    drains again at the ragged end of the call."""
    import os
    from gnomon_b200 import synth
    from gnomon_b200.prepare import from_workload
    people, variants = 128, (1 << 23) + 3 * 128 + 77
    w = synth.scaled(synth.WORKLOADS["batched_100k_x_500k_k512"], people, variants, 3)
    prep = from_workload(w)
    thr = synth.variant_thresholds(w.seed, 0, variants, w.p_lo, w.p_hi, w.missing_rate)
    threads = os.cpu_count() or 1
    rows = oracle.synth_rows(w.seed, 0, variants, people, thr, w.bytes_per_variant,
                             threads=threads)
    s, c = plan_run(prep, rows, shape)
    es, ec = oracle.score_extended(rows, prep, threads=threads)
    np.testing.assert_array_equal(c, ec)
    err = oracle.rel_err(s, es).max()
    assert err < 1e-6, f"max rel err vs extended oracle {err:.3e}"


@pytest.mark.parametrize("shape", I8_SHAPES + [NARROW8])
def test_large_weights_exactness(cuda, shape):
    """The reference cohort (weights ~1, 6.5% missing, 20% flipped)."""
    prep, rows = cohort_prep(16)
    check(prep, rows, plan_run(prep, rows, shape), tol=1e-6)


@pytest.mark.parametrize("shape", I8_SHAPES + [NARROW8])
def test_blocks_aligned_and_not(cuda, shape):
    """Blocks starting at multiples of 128 run on 8-bit limbs; a block that does
    not falls back to the BF16 kernel into the same partials."""
    _, prep, rows, _ = synth_case(700, 3000, scores=20, config="batched_100k_x_500k_k512")
    whole = plan_run(prep, rows, shape)
    aligned = plan_run(prep, rows, shape, blocks=[(0, 1024), (1024, 1024), (2048, 952)])
    mixed = plan_run(prep, rows, shape, blocks=[(0, 1024), (1024, 960), (1984, 1016)])
    for got in (aligned, mixed):
        np.testing.assert_array_equal(got[1], whole[1])
        assert oracle.rel_err(got[0], whole[0]).max() < 1e-7


def test_matches_bf16_limbs(cuda):
    _, prep, rows, _ = synth_case(1500, 2000, scores=200, config="batched_100k_x_500k_k512")
    a = plan_run(prep, rows, I8)
    b = plan_run(prep, rows, BF16)
    np.testing.assert_array_equal(a[1], b[1])
    assert oracle.rel_err(a[0], b[0]).max() < 2e-7
    # one SM or SM pairs: the same integer sums in the same order
    c = plan_run(prep, rows, PAIR)
    np.testing.assert_array_equal(c[1], a[1])
    np.testing.assert_array_equal(c[0], a[0])


def test_narrow_matches_bf16_limbs(cuda):
    _, prep, rows, _ = synth_case(1500, 2000, scores=40, config="batched_100k_x_500k_k512")
    a = plan_run(prep, rows, NARROW8)
    b = plan_run(prep, rows, NARROW_BF16)
    np.testing.assert_array_equal(a[1], b[1])
    assert oracle.rel_err(a[0], b[0]).max() < 2e-7


@pytest.mark.parametrize("bad", [8, 9, 10, 14, 16])
def test_shape_rejects_invalid(cuda, bad):
    """SM pairs without 8-bit limbs or with the narrow kernel, unknown bits."""
    _, prep, rows, _ = synth_case(300, 256, scores=20, config="batched_100k_x_500k_k512")
    plan = DevicePlan(prep, engine=_lib.ENGINE_TENSOR)
    with pytest.raises(_lib.GnomonGpuError) as ei:
        plan.set_shape(bad)
    assert ei.value.status == _lib.GNM_ERR_INVALID
    plan.close()
