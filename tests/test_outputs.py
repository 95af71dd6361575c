"""Score checkpoints (score/checkpoint.rs) and the .sscore writer
(score/main.rs:1389-1548): file formats, validation and text layout."""
from __future__ import annotations

import hashlib
import struct

import numpy as np
import pytest

from gnomon_b200 import checkpoint as ck
from gnomon_b200.prepare import PreparationResult
from gnomon_b200.sscore import format_f32, format_f64, read_sscore, write_sscore


# ---- checkpoint file ----------------------------------------------------------

def test_roundtrip_and_wrong_fingerprint(tmp_path):
    """checkpoint.rs:391-413: write, load, reject a foreign fingerprint."""
    path = tmp_path / "cohort_scores.sscore.gnomon-checkpoint.bin"
    fp = bytes([7] * 32)
    scores, counts = [1.25, -2.5, 3.75], [0, 4, 9]
    ck.write_checkpoint(path, fp, 42, scores, counts)
    got = ck.load_checkpoint(path, fp, 3, 100)
    assert got.completed_variants == 42
    assert got.sum_scores.tolist() == scores
    assert got.missing_counts.tolist() == counts
    with pytest.raises(ck.CheckpointError, match="does not match the prepared"):
        ck.load_checkpoint(path, bytes([8] * 32), 3, 100)


def test_byte_layout(tmp_path):
    path = tmp_path / "x.bin"
    fp = bytes(range(32))
    ck.write_checkpoint(path, fp, 5, np.array([0.5, -1.0]), np.array([3, 1], np.uint32))
    want = (b"GNOMON_SCORE_CHECKPOINT_V1\n" + fp + struct.pack("<QQ", 5, 2)
            + struct.pack("<2d", 0.5, -1.0) + struct.pack("<2I", 3, 1))
    assert path.read_bytes() == want
    assert [p.name for p in tmp_path.iterdir()] == ["x.bin"]   # no temp file left


def test_load_rejections(tmp_path):
    path = tmp_path / "c.bin"
    fp = bytes(32)
    assert ck.load_checkpoint(path, fp, 2, 10) is None            # no file: no checkpoint
    ck.write_checkpoint(path, fp, 11, [1.0, 2.0], [0, 0])
    with pytest.raises(ck.CheckpointError, match="result length 2 does not match"):
        ck.load_checkpoint(path, fp, 3, 20)
    with pytest.raises(ck.CheckpointError, match="completed 11 variants but this run has only 10"):
        ck.load_checkpoint(path, fp, 2, 10)
    path.write_bytes(b"NOT_A_CHECKPOINT_HEADER_XX\n" + bytes(60))
    with pytest.raises(ck.CheckpointError, match="invalid header"):
        ck.load_checkpoint(path, fp, 2, 10)
    with pytest.raises(ck.CheckpointError, match="length mismatch"):
        ck.write_checkpoint(path, fp, 1, [1.0], [0, 0])
    ck.remove_checkpoint(path)
    ck.remove_checkpoint(path)           # removing a missing checkpoint is fine
    assert not path.exists()


def test_checkpoint_path_for_output(tmp_path):
    assert ck.checkpoint_path_for_output("out/cohort_scores.sscore").as_posix() == \
        "out/cohort_scores.sscore.gnomon-checkpoint.bin"
    assert ck.checkpoint_path_for_output("cohort.sscore").as_posix() == \
        "cohort.sscore.gnomon-checkpoint.bin"


def test_writer_rate_limit(tmp_path, monkeypatch):
    """checkpoint.rs:37-65: first block saves, later ones every 30 s, the last
    block and forced saves always; no save without progress."""
    clock = [1000.0]
    monkeypatch.setattr(ck.time, "monotonic", lambda: clock[0])
    w = ck.ScoreCheckpointWriter(tmp_path / "w.bin", bytes(32), total_variants=100)
    s, c = np.zeros(2), np.zeros(2, np.uint32)
    assert w.maybe_save(10, s, c)
    assert not w.maybe_save(10, s, c, force=True)      # no progress
    clock[0] += 29.0
    assert not w.maybe_save(20, s, c)
    assert w.maybe_save(30, s, c, force=True)
    clock[0] += 5.0
    assert w.maybe_save(100, s, c)                     # all variants done
    clock[0] += 31.0
    assert not w.maybe_save(100, s, c)
    assert ck.load_checkpoint(tmp_path / "w.bin", bytes(32), 2, 100).completed_variants == 100


# ---- fingerprint --------------------------------------------------------------

def _small_prep():
    return PreparationResult(
        np.array([0.5, -1.25, 2.0], np.float32), np.array([0.0, 2.5, 0.0], np.float32),
        np.array([0, 1, 1], np.uint32), np.array([0, 1, 3, 3], np.uint64), ["A", "Bee"], 9,
        required_bim_indices=np.array([2, 5, 7], np.uint64),
        output_idx_to_fam_idx=np.array([0, 3, 8], np.uint32),
        final_person_iids=["i0", "i3", "i8"], total_variants_in_bim=12,
        required_is_complex=np.array([0, 1, 0], np.uint8))


def _restated_fingerprint(prep, bed=None):
    """checkpoint.rs:83-121 written out field by field with struct."""
    h = hashlib.sha256()
    q = lambda v: h.update(struct.pack("<Q", v))                 # noqa: E731
    b = lambda x: (q(len(x)), h.update(x))                       # noqa: E731
    q(3); q(9); q(12); q(3); q(3); q(2)
    b(b"A"); b(b"Bee")
    for iid in ("i0", "i3", "i8"):
        b(iid.encode())
    h.update(struct.pack("<2I", 1, 2))                           # score_variant_counts
    h.update(struct.pack("<2d", 0.0, 2.5))                       # baseline
    h.update(struct.pack("<3Q", 2, 5, 7))
    h.update(bytes([0, 1, 0]))
    h.update(struct.pack("<4Q", 0, 1, 3, 3))
    h.update(struct.pack("<3I", 0, 1, 1))
    h.update(struct.pack("<3f", 0.5, -1.25, 2.0))
    h.update(struct.pack("<3f", 0.0, 2.5, 0.0))
    if bed is not None:
        h.update(b"\x00")
        for path, header in ((bed, True), (bed[:-4] + ".bim", False), (bed[:-4] + ".fam", False)):
            b(path.encode())
            import os
            try:
                st = os.stat(path)
                h.update(b"\x01"); q(st.st_size)
                h.update(b"\x01"); q(st.st_mtime_ns // 10**9)
                h.update(struct.pack("<I", st.st_mtime_ns % 10**9))
            except OSError:
                h.update(b"\x00")
            if header:
                with open(path, "rb") as f:
                    h.update(b"\x01" + f.read(3))
    return h.digest()


def test_fingerprint_matches_restatement(tmp_path):
    prep = _small_prep()
    assert ck.fingerprint_preparation(prep) == _restated_fingerprint(prep)
    bed = str(tmp_path / "cohort.chr22.bed")
    (tmp_path / "cohort.chr22.bed").write_bytes(bytes([0x6C, 0x1B, 0x01, 0xFF]))
    (tmp_path / "cohort.chr22.bim").write_text("1\trs1\t0\t1\tA\tG\n")
    # no .fam: hashed as missing
    assert ck.fingerprint_preparation(prep, pipeline=bed) == _restated_fingerprint(prep, bed)


def test_fingerprint_sensitivity():
    prep = _small_prep()
    base = ck.fingerprint_preparation(prep)
    other = _small_prep()
    other.sparse_weights = other.sparse_weights.copy()
    other.sparse_weights[1] = np.float32(-1.2500001)
    assert ck.fingerprint_preparation(other) != base
    assert ck.fingerprint_preparation(prep, total_variants_in_bim=13) != base


def test_strip_fileset_extension():
    assert ck._strip_fileset_extension("acaf_threshold.chr22.bed") == "acaf_threshold.chr22"
    assert ck._strip_fileset_extension("x.pgen") == "x"
    assert ck._strip_fileset_extension("dir/.bed") == "dir/.bed"
    assert ck._strip_fileset_extension("plain") == "plain"
    assert ck._strip_fileset_extension("data.vcf") == "data.vcf"


# ---- .sscore ------------------------------------------------------------------

@pytest.mark.parametrize("x,text", [
    (1.0, "1.0"), (0.3, "0.3"), (123.0, "123.0"), (12.34, "12.34"), (-0.5, "-0.5"),
    (1e-7, "1e-7"), (1.234e-5, "0.00001234"), (1e-5, "0.00001"), (9.999e-6, "9.999e-6"),
    (1e16, "1e16"), (1234567890123456.0, "1234567890123456.0"), (1.5e300, "1.5e300"),
    (0.0, "0.0"), (-0.0, "-0.0"), (0.1 + 0.2, "0.30000000000000004"), (5e-324, "5e-324"),
    (float("nan"), "NaN"), (float("inf"), "inf")])
def test_format_f64_layout(x, text):
    assert format_f64(x) == text


@pytest.mark.parametrize("x,text", [
    (100.0, "100.0"), (0.5, "0.5"), (1e-6, "0.000001"), (1e-7, "1e-7"),
    (1.0 / 3.0 * 100.0, "33.333332"), (1.5e-6, "0.0000015"), (1e13, "1e13"),
    (12345678.0, "12345678.0"), (0.0, "0.0")])
def test_format_f32_layout(x, text):
    assert format_f32(np.float32(x)) == text


def test_write_sscore_layout(tmp_path):
    path = tmp_path / "cohort.sscore"
    sums = np.array([1.5, -3.0, 0.0, 7.25])          # [P=2][K=2]
    missing = np.array([0, 1, 4, 0], np.uint32)
    write_sscore(path, ["p1", "p2"], ["S1", "S2"], np.array([4, 3], np.uint32), sums, missing,
                 score_regions={"S2": "chr1:1-100"})
    want = ("#REGION\tSCORE\tINTERVAL\n#REGION\tS2\tchr1:1-100\n"
            "#IID\tS1_AVG\tS1_MISSING_PCT\tS2_AVG\tS2_MISSING_PCT\n"
            "p1\t0.375\t0.0\t-1.5\t33.333336\n"   # f32: (1/3) * 100
            "p2\t0.0\t100.0\t2.4166666666666665\t0.0\n")
    assert path.read_text() == want
    iids, names, avg, pct = read_sscore(path)
    assert iids == ["p1", "p2"] and names == ["S1", "S2"]
    assert [p.name for p in tmp_path.iterdir()] == ["cohort.sscore"]
