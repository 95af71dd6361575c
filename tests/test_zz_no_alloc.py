"""gnm_score_noalloc: the allocation-free entry point against the existing one.

For callers that cannot allocate device memory while scoring (a host whose
caching allocator owns the whole device, or a callback in which an allocation
would synchronise the device), gnm_score_noalloc keeps its scratch in a static
device array.  This test calls it through the C ABI twice in a row (the second
call reuses the array left over by the first) and checks each result against
gnm_score_device on the same inputs, with the tolerance the other tests use:
missing counts bit-exact, sums within the reference's 1e-6 metric.  It runs
last (file name) and also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from gnomon_b200 import _lib
from gnomon_b200.prepare import PreparationResult
from helpers import synth_case
from oracle import oracle

pytestmark = pytest.mark.gpu


def _noalloc(lib, d_rows, pitch, V, P, d_w, d_c, d_m, baseline, d_s, d_n):
    err = _lib.gnm_error()
    st = lib.gnm_score_noalloc(d_rows, pitch, V, P, d_w, d_c, d_m, baseline, d_s, d_n, None,
                               C.byref(err))
    return st, err.message.decode()


def test_noalloc_matches_existing_entry_point(cuda):
    import torch
    from gnomon_b200.device import DevicePlan, row_pitch
    lib = _lib.load()
    rng = np.random.default_rng(11)
    for people, variants in [(7001, 3001), (5003, 1234)]:
        _, full, rows, _ = synth_case(people, variants, scores=1, seed_offset=variants)
        member = rng.random(variants) < 0.9
        w = np.where(member, full.sparse_weights, 0).astype(np.float32)
        c = np.where(member, full.sparse_missing_corrections, 0).astype(np.float32)
        offs = np.zeros(variants + 1, np.uint64)
        np.cumsum(member, out=offs[1:])
        prep = PreparationResult(w[member], c[member], np.zeros(member.sum(), np.uint32), offs,
                                 ["S000"], people)
        pitch = row_pitch(prep.bytes_per_variant)
        host = np.zeros((variants, pitch), np.uint8)
        host[:, :rows.shape[1]] = rows
        d_rows = torch.from_numpy(host).cuda()

        plan = DevicePlan(prep, engine=_lib.ENGINE_PLAIN)
        ref_s, ref_c = plan.score(d_rows, pitch)
        plan.sync()
        ref_s, ref_c = ref_s.cpu().numpy(), ref_c.cpu().numpy().astype(np.uint32)

        d_w = torch.from_numpy(w).cuda()
        d_c = torch.from_numpy(c).cuda()
        d_m = torch.from_numpy(member.astype(np.uint8)).cuda()
        for call in range(2):
            d_s = torch.full((people,), float("nan"), dtype=torch.float64, device="cuda")
            d_n = torch.full((people,), -1, dtype=torch.int32, device="cuda")
            st, msg = _noalloc(lib, d_rows.data_ptr(), pitch, variants, people, d_w.data_ptr(),
                               d_c.data_ptr(), d_m.data_ptr(), float(prep.baseline[0]),
                               d_s.data_ptr(), d_n.data_ptr())
            assert st == _lib.GNM_OK, msg
            s, n = d_s.cpu().numpy(), d_n.cpu().numpy().astype(np.uint32)
            np.testing.assert_array_equal(n, ref_c, err_msg=f"call {call}")
            assert oracle.within_reference_tolerance(s, ref_s).all(), f"call {call}"
            assert oracle.rel_err(s, ref_s).max() < 1e-6
        plan.close()


def _case_rows(people, variants, seed_offset):
    """Workload weights from helpers.synth_case's generator, rows from the C
    generator (threaded: the 65,536-person case has 1e8 calls)."""
    import os
    from gnomon_b200 import synth
    from gnomon_b200.prepare import from_workload
    base = synth.WORKLOADS["plain_2k_x_50k"]
    w = synth.scaled(base, people, variants, 1)
    w = synth.Workload(w.name, w.people, w.variants, w.scores, w.p_lo, w.p_hi, w.missing_rate,
                       w.sigma, w.flip_frac, w.size_lo, w.size_hi,
                       w.config_id + 1000 * seed_offset)
    thr = synth.variant_thresholds(w.seed, 0, variants, w.p_lo, w.p_hi, w.missing_rate)
    rows = oracle.synth_rows(w.seed, 0, variants, people, thr, w.bytes_per_variant,
                             threads=os.cpu_count() or 1)
    return from_workload(w), rows


@pytest.mark.parametrize("people,variants,with_member", [
    (2_000, 120_001, True),     # three scratch chunks of 48,840 rows, ragged last stage
    (65_536, 3_000, False),     # the people limit, every variant a member (d_member NULL)
    (65_535, 3_001, True),      # one person below the limit, ragged last byte
])
def test_noalloc_chunks_and_limits(cuda, people, variants, with_member):
    """Inputs that cross the scratch's stage-table chunks (the chunks add into
    the same partial slots), a NULL membership array, and people at the
    limit, against gnm_score_device on two calls in a row."""
    import torch
    from gnomon_b200.device import DevicePlan, row_pitch
    lib = _lib.load()
    full, rows = _case_rows(people, variants, seed_offset=people + variants)
    rng = np.random.default_rng(people)
    member = rng.random(variants) < 0.9 if with_member else np.ones(variants, bool)
    w = np.where(member, full.sparse_weights, 0).astype(np.float32)
    c = np.where(member, full.sparse_missing_corrections, 0).astype(np.float32)
    offs = np.zeros(variants + 1, np.uint64)
    np.cumsum(member, out=offs[1:])
    prep = PreparationResult(w[member], c[member], np.zeros(member.sum(), np.uint32), offs,
                             ["S000"], people)
    pitch = row_pitch(prep.bytes_per_variant)
    host = np.zeros((variants, pitch), np.uint8)
    host[:, :rows.shape[1]] = rows
    d_rows = torch.from_numpy(host).cuda()
    plan = DevicePlan(prep, engine=_lib.ENGINE_PLAIN)
    ref_s, ref_c = plan.score(d_rows, pitch)
    plan.sync()
    ref_s, ref_c = ref_s.cpu().numpy(), ref_c.cpu().numpy().astype(np.uint32)
    plan.close()
    d_w = torch.from_numpy(w).cuda()
    d_c = torch.from_numpy(c).cuda()
    d_m = torch.from_numpy(member.astype(np.uint8)).cuda() if with_member else None
    for call in range(2):
        d_s = torch.full((people,), float("nan"), dtype=torch.float64, device="cuda")
        d_n = torch.full((people,), -1, dtype=torch.int32, device="cuda")
        st, msg = _noalloc(lib, d_rows.data_ptr(), pitch, variants, people, d_w.data_ptr(),
                           d_c.data_ptr(), None if d_m is None else d_m.data_ptr(),
                           float(prep.baseline[0]), d_s.data_ptr(), d_n.data_ptr())
        assert st == _lib.GNM_OK, msg
        s, n = d_s.cpu().numpy(), d_n.cpu().numpy().astype(np.uint32)
        np.testing.assert_array_equal(n, ref_c, err_msg=f"call {call}")
        assert oracle.within_reference_tolerance(s, ref_s).all(), f"call {call}"
        assert oracle.rel_err(s, ref_s).max() < 1e-6


def test_noalloc_rejects_bad_row_layout_before_device_work(cuda):
    lib = _lib.load()
    st, msg = _noalloc(lib, 8, 16, 10, 8, 16, 16, None, 0.0, 16, 16)
    assert st == _lib.GNM_ERR_INVALID and "16-byte boundary" in msg
    st, msg = _noalloc(lib, 16, 24, 10, 8, 16, 16, None, 0.0, 16, 16)
    assert st == _lib.GNM_ERR_INVALID and "multiple of 16" in msg
    st, msg = _noalloc(lib, 16, 16, 10, 100, 16, 16, None, 0.0, 16, 16)
    assert st == _lib.GNM_ERR_INVALID and "smaller" in msg


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    lib = _lib.load()
    st, msg = _noalloc(lib, 16, 16, _lib_max_variants() + 1, 8, 16, 16, None, 0.0, 16, 16)
    assert st == _lib.GNM_ERR_INVALID and "GNM_NOALLOC_MAX_VARIANTS" in msg
    st, msg = _noalloc(lib, 16, 16, 8, 65536 + 1, 16, 16, None, 0.0, 16, 16)
    assert st == _lib.GNM_ERR_INVALID and "GNM_NOALLOC_MAX_PEOPLE" in msg


def _lib_max_variants():
    return 262144
