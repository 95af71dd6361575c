"""The C-ABI library: loads, exports every declared symbol, validates inputs (no GPU work)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from gnomon_b200 import _lib
from gnomon_b200.pipeline import prep_view
from helpers import case_prep, known_answer_cases

HEADER = Path(__file__).resolve().parent.parent / "include" / "gnomon_gpu.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(gnm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)
    assert lib.gnm_abi_version() == 1


def _run(prep, rows):
    lib = _lib.load()
    pv = prep_view(prep)
    bv = _lib.gnm_bed_view()
    bv.data = rows.ctypes.data
    bv.data_len = rows.size
    P, K = prep.num_people_to_score, prep.num_scores
    s = np.zeros(P * K)
    c = np.zeros(P * K, np.uint32)
    err = _lib.gnm_error()
    st = lib.gnm_score_run(C.byref(pv), C.byref(bv), None, s.ctypes.data, c.ctypes.data,
                           C.byref(err))
    return st, err.message.decode()


def test_invalid_prep_is_rejected_before_any_device_work():
    prep, rows = case_prep(known_answer_cases()["engine_cases"][0])
    prep.sparse_row_offsets = np.array([0, 5], np.uint64)  # nnz 5 > 1 cell
    prep.sparse_score_columns = np.array([0, 0, 0, 0, 0], np.uint32)  # not ascending
    prep.sparse_weights = np.zeros(5, np.float32)
    prep.sparse_missing_corrections = np.zeros(5, np.float32)
    st, msg = _run(prep, rows)
    assert st == _lib.GNM_ERR_INVALID and "ascending" in msg


def test_declines_without_cuda_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    prep, rows = case_prep(known_answer_cases()["engine_cases"][0])
    st, msg = _run(prep, rows)
    assert st == _lib.GNM_DECLINED, msg


def test_watchdog_selftest_declines_without_cuda_device():
    import ctypes as C
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    e = _lib.gnm_error()
    st = _lib.load().gnm_watchdog_selftest(-1, 1000, None, C.byref(e))
    assert st == _lib.GNM_DECLINED


def test_release_cached_memory_declines_without_cuda_device():
    import ctypes as C
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    e = _lib.gnm_error()
    assert _lib.load().gnm_release_cached_memory(-1, C.byref(e)) == _lib.GNM_DECLINED


def test_parallel_validation_reports_the_first_bad_row():
    """The CSR is checked on several host threads; the error reported is the
    one a serial scan would meet first (lowest variant), not whichever thread
    finishes first."""
    from gnomon_b200.prepare import PreparationResult
    V = 200_000
    offs = np.arange(V + 1, dtype=np.uint64)              # one cell per variant
    w = np.zeros(V, np.float32)
    prep = PreparationResult(w, w.copy(), np.zeros(V, np.uint32), offs, ["S0", "S1"], 8)
    rows = np.zeros((V, 2), np.uint8)
    # variant 100,000 gets a second cell with the same column (not ascending);
    # variant 150,000 a column past the last score
    offs2 = offs.copy()
    offs2[100_001:] += 1
    cols = np.zeros(V + 1, np.uint32)
    cols[150_001] = 7
    prep.sparse_row_offsets = offs2
    prep.sparse_score_columns = cols
    prep.sparse_weights = np.zeros(V + 1, np.float32)
    prep.sparse_missing_corrections = np.zeros(V + 1, np.float32)
    st, msg = _run(prep, rows)
    assert st == _lib.GNM_ERR_INVALID and "ascending" in msg, msg
    # with the early error fixed, the later one is reported
    cols = cols.copy()
    cols[100_001] = 1
    prep.sparse_score_columns = cols
    st, msg = _run(prep, rows)
    assert st == _lib.GNM_ERR_INVALID and "out of range" in msg, msg
