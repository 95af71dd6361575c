"""Device watchdog on the GPU, without a fault: a bounded wait on an mbarrier
that nothing signals expires, the kernel records it and returns, the host
reports GNM_ERR_TIMEOUT, and the same context keeps scoring correctly."""
import ctypes as C
import time

import numpy as np
import pytest

from gnomon_b200 import _lib
from gnomon_b200.pipeline import PipelineContext, run
from helpers import synth_case
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("wait_ns", [50_000_000, 250_000_000])
def test_bounded_wait_expires_and_context_survives(cuda, wait_ns):
    import torch
    from gnomon_b200.device import DevicePlan, row_pitch
    _, prep, rows, _ = synth_case(3000, 500, scores=2, config="diff_20k_x_200k_k16")
    pitch = row_pitch(prep.bytes_per_variant)
    dev = np.zeros((500, pitch), np.uint8)
    dev[:, :rows.shape[1]] = rows
    d_rows = torch.from_numpy(dev).cuda()
    plan = DevicePlan(prep, engine=_lib.ENGINE_PLAIN)       # created before the expiry
    before = [t.cpu().numpy() for t in plan.score(d_rows, pitch)]
    plan.sync()

    e = _lib.gnm_error()
    waited = C.c_uint64(0)
    t0 = time.perf_counter()
    st = _lib.load().gnm_watchdog_selftest(0, wait_ns, C.byref(waited), C.byref(e))
    wall = time.perf_counter() - t0
    assert st == _lib.GNM_ERR_TIMEOUT, e.message
    assert b"bounded wait expired" in e.message
    assert wait_ns <= waited.value < wait_ns + 50_000_000
    assert wall < wait_ns / 1e9 + 5.0

    # the context is still usable: the old plan and a fresh run both score
    after = [t.cpu().numpy() for t in plan.score(d_rows, pitch)]
    plan.sync()
    np.testing.assert_array_equal(after[0], before[0])
    np.testing.assert_array_equal(after[1], before[1])
    s, c = run(PipelineContext(prep), rows.reshape(-1), engine=_lib.ENGINE_PLAIN)
    rs, rc = oracle.score_reference(rows, prep, threads=4)
    np.testing.assert_array_equal(c, rc)
    assert oracle.within_reference_tolerance(s, rs).all()
    plan.close()
