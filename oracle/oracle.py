"""CPU oracle for the scoring hot path — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, and only as the checker / timed CPU baseline.  The
product (``gnomon_b200``) never imports it.

Three independent restatements of gnomon's scoring arithmetic:

* ``score_reference``  — C restatement of the reference CPU engine
  (score/batch.rs, score/kernel.rs, score/decide.rs, score/pipeline.rs; see
  gnm_oracle.c for line citations), the parity target for the plain path;
* ``score_extended``   — C per-genotype scorer in x87 long double, the
  "FP64 oracle" for error reports;
* ``score_numpy``      — a vectorised float64 numpy scorer written from the
  semantics in score/prepare.rs:197-208 and score/batch.rs:489-503, used to
  cross-check the two C scorers on small cases.

Parity of the restatement is pinned by the reference's own known-answer tests
(tests/golden/).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libgnm_oracle.so"
_lib = None


def build() -> Path:
    """Compile gnm_oracle.c (make) when the shared object is missing or stale."""
    src = HERE / "gnm_oracle.c"
    if LIB.exists() and LIB.stat().st_mtime >= src.stat().st_mtime:
        return LIB
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    vp, u64, i32 = C.c_void_p, C.c_uint64, C.c_int
    lib.oracle_synth_rows.argtypes = [vp, u64, u64, u64, u64, vp, u64]
    lib.oracle_synth_rows.restype = None
    lib.oracle_decode.argtypes = [vp, u64, u64, u64, vp, u64]
    lib.oracle_decode.restype = None
    lib.oracle_score_reference.argtypes = [vp, u64, u64, u64, u64, vp, u64, u64, vp, vp, vp, vp,
                                           vp, i32, i32, vp, vp]
    lib.oracle_score_reference.restype = i32
    lib.oracle_score_extended.argtypes = [vp, u64, u64, vp, u64, u64, vp, vp, vp, vp, vp, vp, vp]
    lib.oracle_score_extended.restype = i32
    lib.oracle_score_extended_mt.argtypes = [vp, u64, u64, vp, u64, u64, vp, vp, vp, vp, vp, vp,
                                             vp, i32]
    lib.oracle_score_extended_mt.restype = i32
    lib.oracle_backward_extended.argtypes = [vp, u64, u64, vp, u64, u64, vp, vp, vp, vp, vp]
    lib.oracle_backward_extended.restype = i32
    _lib = lib
    return lib


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


def _prep_arrays(prep):
    w = np.ascontiguousarray(prep.sparse_weights, np.float32)
    c = np.ascontiguousarray(prep.sparse_missing_corrections, np.float32)
    cols = np.ascontiguousarray(prep.sparse_score_columns, np.uint32)
    offs = np.ascontiguousarray(prep.sparse_row_offsets, np.uint64)
    o2f = None if prep.output_idx_to_fam_idx is None else np.ascontiguousarray(
        prep.output_idx_to_fam_idx, np.uint32)
    base = np.ascontiguousarray(prep.baseline, np.float64)
    return w, c, cols, offs, o2f, base


def synth_rows(seed: int, v0: int, n: int, num_people: int, thr: np.ndarray, pitch: int,
               threads: int = 1):
    """Synthetic rows [n, pitch] of variants v0..v0+n-1, people 0..num_people-1.

    ``threads`` > 1 fills disjoint variant ranges from that many host threads
    (ctypes releases the GIL during each call); the bytes do not depend on it."""
    rows = np.zeros((n, pitch), dtype=np.uint8)
    t = np.ascontiguousarray(thr, dtype=np.uint32)
    lib = load()
    if threads <= 1 or n < 2 * threads:
        lib.oracle_synth_rows(rows.ctypes.data, pitch, v0, n, num_people, t.ctypes.data, seed)
        return rows
    from concurrent.futures import ThreadPoolExecutor
    per = -(-n // threads)

    def fill(j0):
        j1 = min(n, j0 + per)
        lib.oracle_synth_rows(rows.ctypes.data + j0 * pitch, pitch, v0 + j0, j1 - j0, num_people,
                              t.ctypes.data + j0 * 12, seed)

    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(fill, range(0, n, per)))
    return rows


def decode(rows: np.ndarray, num_people: int) -> np.ndarray:
    rows = np.ascontiguousarray(rows, dtype=np.uint8)
    n, pitch = rows.shape
    out = np.zeros((n, num_people), dtype=np.int8)
    load().oracle_decode(rows.ctypes.data, pitch, n, num_people, out.ctypes.data, num_people)
    return out


def score_reference(rows: np.ndarray, prep, threads: int = 1, force_path: int = -1):
    """Restated reference CPU engine: (sums f64 [P*K], counts u32 [P*K]).

    rows: [V, pitch] packed rows in reconciled order.
    force_path: -1 route like decide.rs, 0 = all person-major, 1 = all variant-major.
    """
    rows = np.ascontiguousarray(rows, dtype=np.uint8)
    V, pitch = rows.shape
    w, c, cols, offs, o2f, base = _prep_arrays(prep)
    P, K = prep.num_people_to_score, prep.num_scores
    sums = np.zeros(P * K, dtype=np.float64)
    counts = np.zeros(P * K, dtype=np.uint32)
    r = load().oracle_score_reference(rows.ctypes.data, pitch, prep.bytes_per_variant,
                                      prep.total_people_in_fam, P, _p(o2f), K, V, w.ctypes.data,
                                      c.ctypes.data, cols.ctypes.data, offs.ctypes.data,
                                      base.ctypes.data, threads, force_path, sums.ctypes.data,
                                      counts.ctypes.data)
    if r != 0:
        raise MemoryError("oracle_score_reference failed")
    return sums, counts


def score_extended(rows: np.ndarray, prep, threads: Optional[int] = None):
    """Extended-precision (x87 long double) scorer: (sums f64 [P*K], counts u32 [P*K]).

    People are split over ``threads`` host threads (default: all cores); each
    cell is still summed in variant order, so the result is thread-count
    independent."""
    import os
    threads = threads or os.cpu_count() or 1
    rows = np.ascontiguousarray(rows, dtype=np.uint8)
    V, pitch = rows.shape
    w, c, cols, offs, o2f, base = _prep_arrays(prep)
    P, K = prep.num_people_to_score, prep.num_scores
    sums = np.zeros(P * K, dtype=np.float64)
    counts = np.zeros(P * K, dtype=np.uint32)
    r = load().oracle_score_extended_mt(rows.ctypes.data, pitch, P, _p(o2f), K, V, w.ctypes.data,
                                        c.ctypes.data, cols.ctypes.data, offs.ctypes.data,
                                        base.ctypes.data, sums.ctypes.data, counts.ctypes.data,
                                        int(threads))
    if r != 0:
        raise MemoryError("oracle_score_extended failed")
    return sums, counts


def backward_extended(rows: np.ndarray, prep, grad_s: np.ndarray):
    rows = np.ascontiguousarray(rows, dtype=np.uint8)
    V, pitch = rows.shape
    _, _, cols, offs, o2f, _ = _prep_arrays(prep)
    P, K = prep.num_people_to_score, prep.num_scores
    gs = np.ascontiguousarray(grad_s, dtype=np.float32).reshape(-1)
    gw = np.zeros(V * K, dtype=np.float64)
    gc = np.zeros(V * K, dtype=np.float64)
    r = load().oracle_backward_extended(rows.ctypes.data, pitch, P, _p(o2f), K, V,
                                        cols.ctypes.data, offs.ctypes.data, gs.ctypes.data,
                                        gw.ctypes.data, gc.ctypes.data)
    if r != 0:
        raise MemoryError("oracle_backward_extended failed")
    return gw.reshape(V, K), gc.reshape(V, K)


def score_numpy(rows: np.ndarray, prep):
    """Vectorised float64 scorer (independent of the C code; small cases)."""
    P, K = prep.num_people_to_score, prep.num_scores
    V = prep.num_reconciled_variants
    fam = prep.total_people_in_fam
    bpv = (fam + 3) // 4
    r = np.asarray(rows)[:, :bpv]
    codes = np.stack([(r >> (2 * q)) & 3 for q in range(4)], axis=-1).reshape(V, bpv * 4)[:, :fam]
    if prep.output_idx_to_fam_idx is not None:
        codes = codes[:, prep.output_idx_to_fam_idx.astype(np.int64)]
    dos = np.where(codes == 2, 1.0, np.where(codes == 3, 2.0, 0.0))   # [V, P]
    miss = (codes == 1).astype(np.float64)
    W = np.zeros((V, K)); Cm = np.zeros((V, K)); M = np.zeros((V, K))
    offs = prep.sparse_row_offsets.astype(np.int64)
    rows_of = np.repeat(np.arange(V), np.diff(offs))
    cols = prep.sparse_score_columns.astype(np.int64)
    W[rows_of, cols] = prep.sparse_weights.astype(np.float64)
    Cm[rows_of, cols] = prep.sparse_missing_corrections.astype(np.float64)
    M[rows_of, cols] = 1.0
    sums = prep.baseline[None, :] + dos.T @ W - miss.T @ Cm
    counts = np.rint(miss.T @ M).astype(np.uint32)
    return sums.reshape(-1), counts.reshape(-1)


def rel_err(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """The reference's tolerance metric: |a-b| / max(|a|, |b|, 1) (gpu_tests.rs:135-147)."""
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), 1.0)


def within_reference_tolerance(a, b, abs_eps=1e-6, rel_eps=1e-6) -> np.ndarray:
    """gpu_tests.rs:11-13, 135-147: |d| <= 1e-6 OR d/max(|a|,|b|,1) <= 1e-6."""
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    d = np.abs(a - b)
    return (d <= abs_eps) | (rel_err(a, b) <= rel_eps)
