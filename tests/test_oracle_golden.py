"""The CPU oracle against the reference's own known-answer tests (no GPU)."""
import numpy as np
import pytest

from helpers import GOLDEN, case_prep, cohort_prep, expected_final, known_answer_cases
from oracle import oracle
from gnomon_b200.prepare import apply_simple_score_assignment, fold_cells
from gnomon_b200 import synth

CASES = known_answer_cases()["engine_cases"]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
@pytest.mark.parametrize("path", [-1, 0, 1], ids=["routed", "person_major", "variant_major"])
def test_reference_restatement_known_answers(case, path):
    prep, rows = case_prep(case)
    want_s, want_c = expected_final(case, prep)
    s, c = oracle.score_reference(rows, prep, threads=2, force_path=path)
    np.testing.assert_allclose(s, want_s, rtol=0, atol=1e-9)
    np.testing.assert_array_equal(c, want_c)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_extended_and_numpy_known_answers(case):
    prep, rows = case_prep(case)
    want_s, want_c = expected_final(case, prep)
    for fn in (oracle.score_extended, oracle.score_numpy):
        s, c = fn(rows, prep)
        np.testing.assert_allclose(s, want_s, rtol=0, atol=1e-9)
        np.testing.assert_array_equal(c, want_c)


def test_flip_folding_known_answers():
    for case in known_answer_cases()["flip_cases"]:
        entry = [np.float32(0), np.float32(0)]
        for w, f in case["records"]:
            apply_simple_score_assignment(entry, w, f)
        if case.get("row_by_row"):
            for d in (0.0, 1.0, 2.0):
                row = sum(np.float32(w) * (2.0 - d) if f else np.float32(w) * d
                          for w, f in case["records"])
                assert abs(float(entry[1] + entry[0] * np.float32(d)) - row) < case["tol"]
        else:
            assert abs(float(entry[0]) - case["dosage_weight"]) < case["tol"]
            assert abs(float(entry[1]) - case["missing_correction"]) < case["tol"]
        # the vectorised CSR folding agrees with the sequential rule
        recs = case["records"]
        dw, mc, cols, offs = fold_cells(np.zeros(len(recs)), np.zeros(len(recs)),
                                        np.array([r[0] for r in recs], np.float32),
                                        np.array([r[1] for r in recs]), 1)
        assert dw[0] == entry[0] and mc[0] == entry[1]
        assert list(offs) == [0, 1] and list(cols) == [0]


def test_gpu_tests_cohort_all_scorers_agree():
    prep, rows = cohort_prep(16)
    ref_s, ref_c = oracle.score_reference(rows, prep, threads=3)
    ext_s, ext_c = oracle.score_extended(rows, prep)
    np_s, np_c = oracle.score_numpy(rows, prep)
    assert oracle.within_reference_tolerance(ref_s, ext_s).all()
    assert np.abs(ext_s - np_s).max() < 1e-9
    np.testing.assert_array_equal(ref_c, ext_c)
    np.testing.assert_array_equal(ref_c, np_c)
    # the cohort has missing calls in every person (keys 0,1 of 31)
    assert (ref_c.reshape(512, 16) > 0).all()


def test_routing_paths_agree_on_synthetic():
    from helpers import synth_case
    _, prep, rows, _ = synth_case(3000, 2000, scores=1)
    a = oracle.score_reference(rows, prep, force_path=0)
    b = oracle.score_reference(rows, prep, force_path=1)
    e = oracle.score_extended(rows, prep)
    assert oracle.within_reference_tolerance(a[0], e[0]).all()
    assert oracle.within_reference_tolerance(b[0], e[0]).all()
    np.testing.assert_array_equal(a[1], e[1])
    np.testing.assert_array_equal(b[1], e[1])


def test_ld_fixture_decode():
    z = np.load(GOLDEN / "ld_fixture.npz")
    rows, P = z["rows"], int(z["num_people"])
    d = oracle.decode(rows, P)
    codes = synth.unpack_codes(rows, P)
    want = np.select([codes == 0, codes == 1, codes == 2, codes == 3], [0, -1, 1, 2]).astype(np.int8)
    np.testing.assert_array_equal(d, want)
    assert d.shape == (1500, 200)
    # real PLINK data: every class occurs
    assert set(np.unique(d)) <= {-1, 0, 1, 2} and (d == 2).any() and (d == 1).any()
