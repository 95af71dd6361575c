"""Host-side preparation (prepare.rs semantics)."""
import numpy as np
import pytest

from gnomon_b200.prepare import BimRecord, ScoreRecord, fold_cells, reconcile_simple


def test_reconcile_flip_and_orientation():
    bim = [BimRecord("1", 100, "A", "G"), BimRecord("1", 200, "C", "T"),
           BimRecord("1", 300, "A", "C")]
    recs = [ScoreRecord("1", 100, "A", "G", [0.5, float("nan")]),   # effect == allele1 -> flipped
            ScoreRecord("1", 200, "T", "C", [0.25, -1.0]),          # effect == allele2
            ScoreRecord("1", 250, "A", "G", [9.0, 9.0]),            # no BIM row
            ScoreRecord("1", 100, "G", "A", [0.125, 0.0])]          # duplicate, not flipped
    prep = reconcile_simple(bim, recs, ["S0", "S1"], 8)
    assert list(prep.required_bim_indices) == [0, 1]
    assert list(prep.sparse_row_offsets) == [0, 2, 4]
    assert list(prep.sparse_score_columns) == [0, 1, 0, 1]
    # variant 0 score 0: -0.5 (flipped) + 0.125 ; correction 1.0
    assert prep.sparse_weights[0] == np.float32(-0.5) + np.float32(0.125)
    assert prep.sparse_missing_corrections[0] == np.float32(1.0)
    assert prep.sparse_weights[1] == np.float32(0.0)
    assert list(prep.sparse_weights[2:]) == [np.float32(0.25), np.float32(-1.0)]
    assert prep.baseline[0] == 1.0 and prep.baseline[1] == 0.0
    assert list(prep.score_variant_counts) == [2, 2]
    assert prep.bytes_per_variant == 2 and prep.stride == 8


def test_multiallelic_is_rejected():
    bim = [BimRecord("1", 100, "A", "G"), BimRecord("1", 100, "G", "A")]
    with pytest.raises(ValueError):
        reconcile_simple(bim, [ScoreRecord("1", 100, "A", "G", [1.0])], ["S"], 4)


def test_fold_cells_rows_without_cells():
    dw, mc, cols, offs = fold_cells(np.array([2, 0]), np.array([1, 0]),
                                    np.array([1.0, 2.0], np.float32), np.array([True, False]), 4)
    assert list(offs) == [0, 1, 1, 2, 2]
    assert list(dw) == [2.0, -1.0] and list(mc) == [0.0, 2.0]
