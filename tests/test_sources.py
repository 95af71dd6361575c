"""Genotype byte sources on the host (no GPU): a mapped / in-memory .bed and a
read callback (shared/files.rs:187-245), as views for the C ABI and as the
genotype reader of the complex-variant resolver."""
import ctypes as C

import numpy as np

from gnomon_b200 import synth
from gnomon_b200.pipeline import BedSource, ByteRangeSource


def _rows(people=37, variants=50):
    thr = synth.variant_thresholds(99, 0, variants, 0.01, 0.5, 0.05)
    return synth.synth_rows(99, 0, variants, people, thr)


def test_views():
    rows = _rows()
    b = BedSource(rows).view()
    assert b.data == rows.ctypes.data and b.data_len == rows.size and not b.read_at
    r = ByteRangeSource(lambda o, n: rows.reshape(-1)[o:o + n].tobytes()).view()
    assert r.data is None and r.data_len == 0 and r.read_at
    # the C callback copies the requested bytes and reports success with 0
    buf = (C.c_uint8 * 10)()
    assert r.read_at(None, 20, C.cast(buf, C.c_void_p), 10) == 0
    assert bytes(buf) == rows.reshape(-1)[20:30].tobytes()


def test_failing_callback_reports_nonzero_and_keeps_the_error():
    def read_at(offset, length):
        raise OSError("unreachable")
    src = ByteRangeSource(read_at)
    buf = (C.c_uint8 * 4)()
    assert src.view().read_at(None, 0, C.cast(buf, C.c_void_p), 4) != 0
    assert isinstance(src.errors[0], OSError)
    short = ByteRangeSource(lambda o, n: b"\0" * (n - 1)).view()
    assert short.read_at(None, 0, C.cast(buf, C.c_void_p), 4) != 0


def test_genotype_sources_agree():
    people = 37
    rows = _rows(people)
    bpv = rows.shape[1]
    flat = rows.reshape(-1)
    a = BedSource(flat).genotype_source(bpv)
    b = ByteRangeSource(lambda o, n: flat[o:o + n].tobytes()).genotype_source(bpv)
    fam = np.array([0, 3, 4, 17, 36], np.int64)
    for row in (0, 7, 49):
        np.testing.assert_array_equal(a.codes(row, fam), b.codes(row, fam))
        np.testing.assert_array_equal(a.codes(row, fam), synth.unpack_codes(rows[row:row + 1], people)[0, fam])
