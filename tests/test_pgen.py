"""PLINK 2 .pgen input, CPU side: the oracle against the reference's fixture
pair, the synthetic encoder, and the C ABI's header parse (no GPU work)."""
import collections
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from gnomon_b200 import _lib, synth
from gnomon_b200.pgen import pgen_dims
from oracle import pgen_oracle

GOLDEN = Path(__file__).resolve().parent / "golden"


def ld_pgen():
    return np.load(GOLDEN / "ld_pgen_fixture.npz")["pgen"].tobytes()


def expected_rows(cats, repeats=1):
    """.bed rows of A1 = ALT dosage codes, padding fields 01."""
    V, n = cats.shape
    codes = np.full((V, (n + 3) // 4 * 4), 0b01, np.uint8)
    codes[:, :n] = synth.PGEN_CAT_TO_BED[cats]
    q = codes.reshape(V, -1, 4)
    rows = (q[..., 0] | (q[..., 1] << 2) | (q[..., 2] << 4) | (q[..., 3] << 6)).astype(np.uint8)
    return np.tile(rows, (repeats, 1))


def test_oracle_matches_reference_bed_twin():
    """ld_p.pgen and ld.bed hold the same genotypes (the reference's fixture pair)."""
    z = np.load(GOLDEN / "ld_fixture.npz")
    got = pgen_oracle.decode_to_bed(ld_pgen())
    np.testing.assert_array_equal(got, z["rows"])


def test_reference_fixture_uses_ld_records():
    h = pgen_oracle.parse_header(ld_pgen())
    assert (h["variants"], h["samples"]) == (1500, 200)
    kinds = collections.Counter((h["types"] & 7).tolist())
    assert kinds[2] + kinds[3] > 0 and kinds[0] + kinds[1] > 0


@pytest.mark.parametrize("n", [1, 5, 203, 257, 300, 70001])
def test_encoder_round_trip_through_oracle(n):
    V = 96 if n < 1000 else 24
    cats = synth.pgen_ld_categories(11, V, n)
    data = synth.encode_pgen(cats)
    np.testing.assert_array_equal(pgen_oracle.decode_to_bed(data), expected_rows(cats))


def test_encoder_covers_every_record_type():
    seen = collections.Counter()
    for n in (203, 300, 5000):
        cats = synth.pgen_ld_categories(3, 64, n)
        # constant variants with a few exceptions -> fill types 4 / 6 / 7
        for j, fill in enumerate((0, 2, 3)):
            cats[60 + j] = fill
            cats[60 + j, ::97] = (fill + 1) % 4
        seen.update(pgen_oracle.parse_header(synth.encode_pgen(cats))["types"].tolist())
    assert {0, 1, 2, 3, 4, 6, 7} <= set(seen), seen


def test_repeated_records_keep_their_anchors():
    cats = synth.pgen_ld_categories(7, 256, 9)
    data = synth.encode_pgen(cats, repeats=300)     # 76,800 variants over two blocks
    h = pgen_oracle.parse_header(data)
    assert h["variants"] == 76_800
    rows = pgen_oracle.decode_to_bed(data)
    np.testing.assert_array_equal(rows, expected_rows(cats, 300))


def test_abi_dims():
    assert pgen_dims(ld_pgen()) == (1500, 200)
    data = synth.encode_pgen(synth.pgen_ld_categories(1, 32, 70001))
    assert pgen_dims(data) == (32, 70001)


def corrupt(data: bytes, at: int, value: int) -> bytes:
    b = bytearray(data)
    b[at] = value
    return bytes(b)


def _status(data):
    with pytest.raises(_lib.GnomonGpuError) as ei:
        pgen_dims(data)
    return ei.value.status


def test_abi_rejects_bad_files():
    cats = synth.pgen_ld_categories(2, 40, 300)
    data = synth.encode_pgen(cats)
    types_at = 12 + 8                    # one block: 8-byte offset, then the 8-bit types
    assert _status(data[:5]) == _lib.GNM_ERR_IO                        # no header
    assert _status(b"\x6c\x1c" + data[2:]) == _lib.GNM_ERR_IO          # bad magic
    assert _status(data[:-1]) == _lib.GNM_ERR_IO                       # last record cut
    assert _status(corrupt(data, 2, 0x03)) == _lib.GNM_ERR_INVALID     # unsupported mode
    kind = data[types_at]
    # a multiallelic record: dims reads the header only (opening the file
    # without ALT counts rejects it, tests/test_gpu_pgen.py)
    assert pgen_dims(corrupt(data, types_at, kind | 0x08)) == (40, 300)
    assert _status(corrupt(data, types_at, kind | 0x80)) == _lib.GNM_ERR_IO  # phased dosage alone
    assert _status(corrupt(data, types_at, 5)) == _lib.GNM_ERR_INVALID           # type 5
    # the oracle rejects the same files
    with pytest.raises(pgen_oracle.PgenError):
        pgen_oracle.decode_to_bed(corrupt(data, types_at, kind | 0x08))


def test_abi_phase_bit_is_accepted():
    cats = synth.pgen_ld_categories(2, 40, 300)
    data = synth.encode_pgen(cats)
    types_at = 12 + 8
    assert pgen_dims(corrupt(data, types_at, data[types_at] | 0x10)) == (40, 300)


def test_decode_declines_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    lib = _lib.load()
    data = np.frombuffer(ld_pgen(), np.uint8)
    e = _lib.gnm_error()
    st = lib.gnm_pgen_decode_device(data.ctypes.data, data.nbytes, 0, None, 64, None,
                                    C.byref(e))
    assert st == _lib.GNM_DECLINED


def encode_fixed_width(cats, ref_flags: bool = False):
    """A storage-mode 0x02 .pgen: 2-bit category arrays, no index, laid out
    where the reference's reader looks for them: the body after 12 header
    bytes and one more (shared/adapt_plink2.rs:2048-2057), and after one
    reference-flag bit per variant when the format byte's bits 6-7 are 3."""
    V, n = cats.shape
    q = np.zeros((V, (n + 3) // 4 * 4), np.uint8)
    q[:, :n] = cats
    q = q.reshape(V, -1, 4)
    body = (q[..., 0] | (q[..., 1] << 2) | (q[..., 2] << 4) | (q[..., 3] << 6)).astype(np.uint8)
    fmt = b"\xc0" if ref_flags else b"\x00"
    flags = bytes((V + 7) // 8) if ref_flags else b""
    return (b"\x6c\x1b\x02" + np.array([V, n], "<u4").tobytes() + fmt + b"\x00" + flags +
            body.tobytes())


def test_fixed_width_mode_oracle_and_dims():
    cats = synth.pgen_categories(4, 50, 301)
    data = encode_fixed_width(cats)
    np.testing.assert_array_equal(pgen_oracle.decode_to_bed(data), expected_rows(cats))
    np.testing.assert_array_equal(pgen_oracle.decode_to_bed(encode_fixed_width(cats, True)),
                                  expected_rows(cats))
    assert pgen_dims(data) == (50, 301)
    assert _status(data[:-1]) == _lib.GNM_ERR_IO


def test_long_difflist_oracle():
    n = 400_000
    ids = np.arange(0, n, 2, dtype=np.int64)
    vals = np.random.default_rng(1).integers(1, 4, len(ids)).astype(np.uint8)
    data = synth._pgen_file(n, [4], [synth._difflist_bytes(ids, vals, n)])
    cats = np.zeros((1, n), np.uint8)
    cats[0, ids] = vals
    np.testing.assert_array_equal(pgen_oracle.decode_to_bed(data), expected_rows(cats))


def non_rising_pgens(n=1000):
    """A valid fill record with a two-group difflist, and copies whose ids
    repeat inside a group or fall back across the group boundary."""
    ids = np.arange(0, 200, 2, dtype=np.int64)
    vals = np.ones(len(ids), np.uint8)
    rec = bytes(synth._difflist_bytes(ids, vals, n))
    # length (1 byte), two 2-byte first ids, one group-length byte, 25 value bytes
    deltas_at = 1 + 4 + 1 + 25
    dup = bytearray(rec)
    dup[deltas_at] = 0                       # a zero delta inside group 0
    back = bytearray(rec)
    back[3:5] = (100).to_bytes(2, "little")  # group 1 starts below group 0's last id
    return [synth._pgen_file(n, [4], [r]) for r in (rec, bytes(dup), bytes(back))]


def test_non_rising_difflist_ids_are_malformed():
    ok, dup, back = non_rising_pgens()
    pgen_oracle.decode_to_bed(ok)
    for bad in (dup, back):
        with pytest.raises(pgen_oracle.PgenError, match="rise"):
            pgen_oracle.decode_to_bed(bad)


def test_score_pgen_declines_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from helpers import synth_case
    from gnomon_b200.pgen import score_pgen
    w, prep, rows, _ = synth_case(101, 20, 1)
    cats = synth.BED_TO_PGEN_CAT[synth.unpack_codes(rows, 101)].astype(np.uint8)
    with pytest.raises(_lib.GnomonGpuError) as ei:
        score_pgen(prep, synth.encode_pgen(cats))
    assert ei.value.status == _lib.GNM_DECLINED


def test_zero_variant_file():
    data = synth._pgen_file(7, [], [])
    assert pgen_dims(data) == (0, 7)
    assert pgen_oracle.decode_to_bed(data).shape == (0, 2)


def test_ld_record_without_anchor_is_rejected_by_the_oracle():
    cats = synth.pgen_ld_categories(3, 8, 100)
    types, recs = synth._pgen_records(cats)
    first_ld = next(i for i, k in enumerate(types) if k in (2, 3))
    # drop the records before the first LD one: it now opens the block
    data = synth._pgen_file(100, types[first_ld:], recs[first_ld:])
    with pytest.raises(pgen_oracle.PgenError, match="anchor"):
        pgen_oracle.decode_to_bed(data)


@pytest.mark.parametrize("n", [1, 5, 203, 300, 70001])
def test_c_restatement_matches(n):
    """oracle/pgen_oracle.c (the timed CPU decoder) against the Python oracle."""
    cats = synth.pgen_ld_categories(n, 96 if n < 1000 else 24, n)
    for j, fill in enumerate((0, 2, 3)):
        cats[-3 + j] = fill
        cats[-3 + j, ::37] = (fill + 1) % 4
    data = synth.encode_pgen(cats)
    np.testing.assert_array_equal(pgen_oracle.decode_to_bed_c(data, threads=3),
                                  pgen_oracle.decode_to_bed(data))


def test_c_restatement_fixture_and_errors():
    z = np.load(GOLDEN / "ld_fixture.npz")
    np.testing.assert_array_equal(pgen_oracle.decode_to_bed_c(ld_pgen(), threads=4), z["rows"])
    cats = synth.pgen_ld_categories(7, 256, 9)
    data = synth.encode_pgen(cats, repeats=300)      # two blocks
    np.testing.assert_array_equal(pgen_oracle.decode_to_bed_c(data), expected_rows(cats, 300))
    for bad in non_rising_pgens()[1:]:
        with pytest.raises(pgen_oracle.PgenError):
            pgen_oracle.decode_to_bed_c(bad)
    types, recs = synth._pgen_records(synth.pgen_ld_categories(3, 8, 100))
    first_ld = next(i for i, k in enumerate(types) if k in (2, 3))
    with pytest.raises(pgen_oracle.PgenError):
        pgen_oracle.decode_to_bed_c(synth._pgen_file(100, types[first_ld:], recs[first_ld:]))


def test_abi_dosage_bits_are_accepted():
    cats = synth.pgen_ld_categories(2, 40, 300)
    dos = np.full(cats.shape, 65535, np.uint16)
    dos[cats == 3] = 16384
    for kind in ("list", "dense", "bits"):
        assert pgen_dims(synth.encode_pgen_tracks(cats, dos, kind)) == (40, 300)


def test_dosage_hardcall_rule_matches_the_reference_boundaries():
    """shared/adapt_plink2.rs:3413-3470 (diploid): one allele copy is 16384;
    1638/16384 lies inside the 0.10 tolerance, 1639/16384 outside; 1.5 has
    no hard call; 65535 is missing."""
    f = pgen_oracle.dosage_to_hardcall
    for v, want in [(int(0.05 / 2.0 * 32768.0), 0), (int(1.00 / 2.0 * 32768.0), 1),
                    (int(1.09 / 2.0 * 32768.0), 1), (int(2.00 / 2.0 * 32768.0), 2),
                    (0, 0), (16384, 1), (32768, 2), (16384 + 1638, 1), (16384 + 1639, 255),
                    (16384 - 1638, 1), (16384 - 1639, 255), (24576, 255), (65535, 255)]:
        assert f(v) == want, v


def _one_record_pgen(n, rtype, body):
    return synth._pgen_file(n, [rtype], [bytes(body)])


def test_reference_dense_dosage_record():
    """shared/adapt_plink2.rs:3516-3570: a 2-bit main track of categories
    {0, 1, 3, 3} and a dense dosage track {0, 18022, 18022, 18023} (type bit
    6): the hard calls stand, sample 2's dosage 1.09997 becomes a het, sample
    3's 1.10004 stays missing -> ALT counts {0, 1, 1, missing}."""
    cats = np.array([0, 1, 3, 3], np.uint8)
    body = bytes([int(cats[0] | (cats[1] << 2) | (cats[2] << 4) | (cats[3] << 6))])
    body += np.array([0, 18022, 18022, 18023], "<u2").tobytes()
    rows = pgen_oracle.decode_to_bed(_one_record_pgen(4, 0b0100_0000, body))
    assert rows.shape == (1, 1)
    assert rows[0, 0] == expected_rows(np.array([[0, 1, 1, 3]], np.uint8))[0, 0]


@pytest.mark.parametrize("kind", ["list", "dense", "bits"])
@pytest.mark.parametrize("phase", [None, "all", "partial"])
def test_oracle_dosage_tracks_fill_missing_calls(kind, phase):
    """Every dosage-track layout, behind either phase-track layout, on LD
    records too: missing calls take the dosage's allele count when it is
    within 0.10, hard calls never change, phased dosages change nothing."""
    rng = np.random.default_rng(5)
    cats = synth.pgen_ld_categories(9, 90, 517)
    dos = rng.integers(0, 32769, cats.shape).astype(np.uint16)
    dos[rng.random(cats.shape) < 0.3] = 65535
    near = rng.random(cats.shape) < 0.5       # half of them snapped near a whole count
    dos[near] = (rng.integers(0, 3, near.sum()) * 16384 +
                 rng.integers(-1700, 1700, near.sum())).clip(0, 32768).astype(np.uint16)
    data = synth.encode_pgen_tracks(cats, dos, kind, phase, phased_dosage=kind != "list",
                                    seed=11)
    want = cats.copy()
    for v, i in zip(*np.nonzero(cats == 3)):
        hc = pgen_oracle.dosage_to_hardcall(int(dos[v, i]))
        if hc != 255:
            want[v, i] = hc
    assert (want != cats).any()
    np.testing.assert_array_equal(pgen_oracle.decode_to_bed(data), expected_rows(want))


# ---- multiallelic records (vrtype bit 3) ---------------------------------------

def alt_copy_rows(alleles, rows):
    """.bed rows holding the copies of ALT j per (variant, j), padding 01."""
    out = []
    n = alleles.shape[1]
    for v, j in rows:
        cnt = (alleles[v] == j).sum(axis=1)
        cat = np.where((alleles[v] < 0).any(axis=1), 3, cnt).astype(np.uint8)
        codes = np.full((n + 3) // 4 * 4, 0b01, np.uint8)
        codes[:n] = pgen_oracle.CAT_TO_BED[cat]
        q = codes.reshape(-1, 4)
        out.append(q[:, 0] | (q[:, 1] << 2) | (q[:, 2] << 4) | (q[:, 3] << 6))
    return np.array(out, np.uint8)


MA_COUNTS = [1, 2, 3, 5, 2, 18, 4, 300]


def ma_case(n, seed=7):
    alleles = synth.multiallelic_alleles(seed, MA_COUNTS, n)
    alleles[0] = np.minimum(alleles[0], 1)          # a biallelic variant among them
    rows = [(v, j) for v, a in enumerate(MA_COUNTS) for j in range(1, a + 1)]
    return alleles, rows


def test_reference_multiallelic_known_answer():
    """shared/adapt_plink2.rs:3806-3815: a het patched to ALT 3 and a hom-ALT
    pair patched to ALT 3 / ALT 3, projected onto ALT 1 of a 3-ALT variant."""
    rec = bytes([0x00, 0x01, 0x01, 0x01, 0x0A])
    out, cur = pgen_oracle._project_multiallelic(rec, 0, 3, np.array([1, 2, 2], np.uint8), 3, 1)
    assert list(out) == [0, 0, 2] and cur == len(rec)


@pytest.mark.parametrize("het_fmt,hom_fmt", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_oracle_projects_multiallelic_records(het_fmt, hom_fmt):
    alleles, rows = ma_case(301)
    data = synth.encode_pgen_multiallelic(alleles, MA_COUNTS, het_fmt, hom_fmt, phase="partial")
    got = pgen_oracle.decode_to_bed(data, alt_counts=MA_COUNTS, rows=rows)
    np.testing.assert_array_equal(got, alt_copy_rows(alleles, rows))


def test_oracle_keeps_the_references_multiallelic_edges():
    alleles, rows = ma_case(200, seed=3)
    cats = synth.multiallelic_categories(alleles)
    # no patch: every ALT row reads the plain categories (ALT 1's copies where
    # the record is right, as :2348-2362 reads it)
    plain = synth.encode_pgen_multiallelic(alleles, MA_COUNTS, patch=np.zeros(len(MA_COUNTS), bool))
    got = pgen_oracle.decode_to_bed(plain, alt_counts=MA_COUNTS, rows=rows)
    want = expected_rows(cats)[[v for v, _ in rows]]
    np.testing.assert_array_equal(got, want)
    # a patched record of a variant given one ALT reads as biallelic
    data = synth.encode_pgen_multiallelic(alleles, MA_COUNTS)
    ones = [1] * len(MA_COUNTS)
    got = pgen_oracle.decode_to_bed(data, alt_counts=ones)
    np.testing.assert_array_equal(got, expected_rows(cats))
    with pytest.raises(pgen_oracle.PgenError):
        pgen_oracle.decode_to_bed(data)               # ALT counts needed
    with pytest.raises(pgen_oracle.PgenError):
        pgen_oracle.decode_to_bed(data, alt_counts=MA_COUNTS, rows=[(1, 3)])   # only 2 ALTs


def test_oracle_multiallelic_dosage_only_on_alt1():
    alleles, rows = ma_case(150, seed=5)
    cats = synth.multiallelic_categories(alleles)
    dos = np.full(cats.shape, 65535, np.uint16)
    dos[cats == 3] = 16384                             # one copy for every missing call
    data = synth.encode_pgen_multiallelic(alleles, MA_COUNTS, dosage=dos)
    got = pgen_oracle.decode_to_bed(data, alt_counts=MA_COUNTS, rows=rows)
    want = alt_copy_rows(alleles, rows)
    for r, (v, j) in enumerate(rows):
        if j == 1 or MA_COUNTS[v] <= 1:
            filled = alleles.copy()
            filled[v][(alleles[v] < 0).any(axis=1)] = [0, j]
            want[r] = alt_copy_rows(filled, [(v, j)])[0]
    np.testing.assert_array_equal(got, want)
