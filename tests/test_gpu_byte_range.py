"""Row bytes served by a read callback (gnm_bed_view.read_at) instead of a
mapped file: the reference's ``ByteRangeSource::read_at`` (shared/files.rs:
187-245) for remote / non-local filesets.

The engine reads every required row through the callback (from several host
threads), in the order ``required_bim_indices`` lists them, so out-of-order
and sparse row maps are served exactly; a callback that fails ends the call
with GNM_ERR_PRODUCER (``PipelineError("Producer")``, the reference's
producer-thread failure).
"""
import threading

import numpy as np
import pytest

from gnomon_b200 import _lib
from gnomon_b200.pipeline import ByteRangeSource, PipelineContext, PipelineError, run
from gnomon_b200.prepare import PreparationResult
from helpers import synth_case
from oracle import oracle

pytestmark = pytest.mark.gpu


def _permuted_case(people, file_rows, used, scores, seed):
    """A .bed of `file_rows` rows; the preparation scores `used` of them in a
    shuffled order (required_bim_indices), with the workload's weights."""
    _, full, rows, _ = synth_case(people, file_rows, scores=scores,
                                  config="batched_100k_x_500k_k512", seed_offset=seed)
    rng = np.random.default_rng(seed)
    required = rng.choice(file_rows, used, replace=False).astype(np.uint64)
    offs = full.sparse_row_offsets.astype(np.int64)
    sel_w, sel_c, sel_k, counts = [], [], [], []
    for r in required.astype(np.int64):   # the cells of .bim row r become variant v
        sel_w.append(full.sparse_weights[offs[r]:offs[r + 1]])
        sel_c.append(full.sparse_missing_corrections[offs[r]:offs[r + 1]])
        sel_k.append(full.sparse_score_columns[offs[r]:offs[r + 1]])
        counts.append(offs[r + 1] - offs[r])
    new_offs = np.zeros(used + 1, np.uint64)
    np.cumsum(counts, out=new_offs[1:])
    prep = PreparationResult(np.concatenate(sel_w), np.concatenate(sel_c),
                             np.concatenate(sel_k), new_offs, full.score_names, people,
                             required_bim_indices=required)
    return prep, rows, required


@pytest.mark.parametrize("engine", [_lib.ENGINE_PLAIN, _lib.ENGINE_TENSOR])
def test_read_at_out_of_order_rows(cuda, engine):
    prep, rows, required = _permuted_case(1_500, 3_000, 2_000, scores=12, seed=5)
    data = rows.tobytes()          # the row data after the magic, bpv bytes per row
    bpv = prep.bytes_per_variant
    seen = []
    lock = threading.Lock()

    def read_at(offset, length):
        with lock:
            seen.append(offset // bpv)
        assert offset % bpv == 0 and length == bpv
        return data[offset:offset + length]

    s, c = run(PipelineContext(prep), ByteRangeSource(read_at), engine=engine)
    assert sorted(seen) == sorted(required.tolist())   # each required row read once
    scored = rows[required.astype(np.int64)]
    rs, rc = oracle.score_reference(scored, prep, threads=4)
    np.testing.assert_array_equal(c, rc)
    assert oracle.within_reference_tolerance(s, rs).all()
    # the same call from the bytes themselves gives the same result
    s2, c2 = run(PipelineContext(prep), np.frombuffer(data, np.uint8), engine=engine)
    np.testing.assert_array_equal(c2, c)
    np.testing.assert_array_equal(s2, s)


@pytest.mark.parametrize("fail", ["short", "raise"])
def test_read_at_failure_is_a_producer_error(cuda, fail):
    prep, rows, _ = _permuted_case(700, 1_200, 1_000, scores=3, seed=9)
    data = rows.tobytes()
    calls = [0]
    lock = threading.Lock()

    def read_at(offset, length):
        with lock:
            calls[0] += 1
            n = calls[0]
        if n > 400:   # fails part-way through the rows
            if fail == "raise":
                raise OSError("connection reset")
            return data[offset:offset + length - 1]
        return data[offset:offset + length]

    with pytest.raises(PipelineError) as e:
        run(PipelineContext(prep), ByteRangeSource(read_at), engine=_lib.ENGINE_PLAIN)
    assert e.value.kind == "Producer" and e.value.status == _lib.GNM_ERR_PRODUCER
    assert "read_at" in str(e.value)
    if fail == "raise":
        assert "connection reset" in str(e.value)
    # the context stays usable: the next call scores correctly
    s, c = run(PipelineContext(prep), ByteRangeSource(lambda o, n: data[o:o + n]),
               engine=_lib.ENGINE_PLAIN)
    rs, rc = oracle.score_reference(rows[prep.required_bim_indices.astype(np.int64)], prep,
                                    threads=4)
    np.testing.assert_array_equal(c, rc)
    assert oracle.within_reference_tolerance(s, rs).all()
