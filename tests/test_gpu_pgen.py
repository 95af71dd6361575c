"""PLINK 2 .pgen decode on the GPU (gnm_pgen_decode_device) against the oracle,
and scoring from decoded rows against scoring the same genotypes as a .bed."""
import dataclasses

import numpy as np
import pytest
import torch

from gnomon_b200 import _lib, synth
from gnomon_b200.pgen import decode_to_device, score_pgen
from gnomon_b200.pipeline import PipelineContext, run
from helpers import synth_case
from oracle import oracle, pgen_oracle
from test_pgen import (GOLDEN, corrupt, encode_fixed_width, expected_rows, ld_pgen,
                       non_rising_pgens)

pytestmark = pytest.mark.gpu
SENTINEL = 0xA7


def device_rows(data, n):
    """Decode into sentinel-filled rows; the bytes past each row must survive."""
    m = pgen_oracle.parse_header(data)["variants"]
    bpv = (n + 3) // 4
    pitch = (bpv + 127) // 128 * 128
    rows = torch.full((max(m, 1) * pitch,), SENTINEL, dtype=torch.uint8, device="cuda")
    rows, pitch = decode_to_device(data, rows=rows, pitch=pitch)
    host = rows[:m * pitch].view(m, pitch).cpu().numpy()
    assert (host[:, bpv:] == SENTINEL).all(), "bytes past the row were changed"
    return host[:, :bpv]


def test_reference_fixture(cuda):
    z = np.load(GOLDEN / "ld_fixture.npz")
    np.testing.assert_array_equal(device_rows(ld_pgen(), 200), z["rows"])


@pytest.mark.parametrize("n", [1, 3, 4, 5, 64, 203, 256, 257, 300, 4097, 65537, 70001])
def test_synthetic_every_record_type(cuda, n):
    V = 120 if n < 10_000 else 40
    cats = synth.pgen_ld_categories(n, V, n)
    for j, fill in enumerate((0, 2, 3)):          # near-constant variants: fill types 4 / 6 / 7
        cats[V - 3 + j] = fill
        cats[V - 3 + j, ::37] = (fill + 1) % 4
    data = synth.encode_pgen(cats)
    got = device_rows(data, n)
    np.testing.assert_array_equal(got, pgen_oracle.decode_to_bed(data))
    np.testing.assert_array_equal(got, expected_rows(cats))


def test_long_difflists(cuda):
    """A difflist longer than one shared-memory chunk of 2048 groups (131,072
    entries) is laid out in rounds: a fill record (type 4) with 200,000
    exceptions, then an LD record against it and a shorter fill record."""
    n = 400_000
    ids = np.arange(0, n, 2, dtype=np.int64)
    rng = np.random.default_rng(1)
    vals = rng.integers(1, 4, len(ids)).astype(np.uint8)
    cats = np.zeros((3, n), np.uint8)
    cats[0, ids] = vals
    cats[1] = cats[0]
    flip = ids[::3] + 1
    cats[1, flip] = 1
    cats[2] = 0
    cats[2, 1::5] = 2
    recs = [synth._difflist_bytes(ids, vals, n),
            synth._difflist_bytes(flip, cats[1, flip], n),
            synth._difflist_bytes(np.arange(1, n, 5), cats[2, 1::5], n)]
    data = synth._pgen_file(n, [4, 2, 4], recs)
    np.testing.assert_array_equal(pgen_oracle.decode_to_bed(data), expected_rows(cats))
    np.testing.assert_array_equal(device_rows(data, n), expected_rows(cats))


def test_two_blocks_of_repeated_records(cuda):
    cats = synth.pgen_ld_categories(7, 256, 203)
    data = synth.encode_pgen(cats, repeats=300)   # 76,800 variants: LD anchors per block
    np.testing.assert_array_equal(device_rows(data, 203), expected_rows(cats, 300))


def test_fixed_width_mode(cuda):
    cats = synth.pgen_categories(4, 50, 301)
    data = encode_fixed_width(cats)
    np.testing.assert_array_equal(device_rows(data, 301), expected_rows(cats))


def _find(data, kinds):
    h = pgen_oracle.parse_header(data)
    v = next(i for i, t in enumerate(h["types"].tolist()) if t in kinds)
    return int(h["offsets"][v])


def test_malformed_records_are_reported(cuda):
    cats = synth.pgen_ld_categories(2, 64, 100)
    data = synth.encode_pgen(cats)
    # an LD difflist claiming more entries than samples
    bad = corrupt(data, _find(data, (2, 3)), 0x7F)
    with pytest.raises(_lib.GnomonGpuError) as ei:
        device_rows(bad, 100)
    assert ei.value.status == _lib.GNM_ERR_IO and "overruns" in str(ei.value)
    # a 1-bit record with an invalid pair code
    cats[5] = 0
    cats[5, ::3] = 1
    data = synth.encode_pgen(cats)
    bad = corrupt(data, _find(data, (1,)), 4)
    with pytest.raises(_lib.GnomonGpuError) as ei:
        device_rows(bad, 100)
    assert ei.value.status == _lib.GNM_ERR_IO and "pair code" in str(ei.value)
    # sample ids that repeat or fall back
    ok, dup, back = non_rising_pgens()
    np.testing.assert_array_equal(device_rows(ok, 1000), pgen_oracle.decode_to_bed(ok))
    for bad in (dup, back):
        with pytest.raises(_lib.GnomonGpuError) as ei:
            device_rows(bad, 1000)
        assert ei.value.status == _lib.GNM_ERR_IO
    # the device is still usable
    np.testing.assert_array_equal(device_rows(ld_pgen(), 200),
                                  np.load(GOLDEN / "ld_fixture.npz")["rows"])


def _as_pgen(rows, people):
    codes = synth.unpack_codes(rows, people)
    return synth.BED_TO_PGEN_CAT[codes].astype(np.uint8)


@pytest.mark.parametrize("people,variants,scores,block", [(1001, 300, 1, 0), (2003, 257, 16, 0),
                                                          (1001, 300, 1, 37)])
def test_score_from_pgen_equals_bed(cuda, people, variants, scores, block):
    w, prep, rows, _ = synth_case(people, variants, scores)
    data = synth.encode_pgen(_as_pgen(rows, people))
    s, c = score_pgen(prep, data, block_variants=block)
    bs, bc = run(PipelineContext(prep), rows.reshape(-1))
    np.testing.assert_array_equal(c, bc)
    if block == 0:   # same blocks as the .bed run: same sums
        np.testing.assert_allclose(s, bs, rtol=1e-12, atol=1e-12)
    else:            # other FP32 block sums: the reference's 1e-6 metric
        assert oracle.within_reference_tolerance(s, bs).all()
    es, ec = oracle.score_extended(rows, prep)
    np.testing.assert_array_equal(c, ec)
    rs, _ = oracle.score_reference(rows, prep, threads=4)
    assert oracle.within_reference_tolerance(s, rs).all()


def test_score_from_pgen_gathers_required_variants(cuda):
    people, V = 777, 200
    w, prep, rows, _ = synth_case(people, V, 4)
    other = synth.pgen_ld_categories(5, V, people)
    cats = np.empty((2 * V, people), np.uint8)
    cats[1::2] = _as_pgen(rows, people)          # the scored variants at odd rows
    cats[0::2] = other
    data = synth.encode_pgen(cats)
    prep2 = dataclasses.replace(prep, required_bim_indices=np.arange(1, 2 * V, 2, dtype=np.uint64))
    s, c = score_pgen(prep2, data, block_variants=23)
    bs, bc = run(PipelineContext(prep), rows.reshape(-1))
    np.testing.assert_array_equal(c, bc)
    assert oracle.within_reference_tolerance(s, bs).all()   # 23-variant FP32 blocks


@pytest.mark.parametrize("block", [1, 7, 17, 100, 4096])
def test_range_decode_matches_whole_file(cuda, block):
    """Blocks that start inside a run of LD records decode their anchor into
    the scratch row; every block equals the same rows of a whole-file decode."""
    from gnomon_b200.pgen import PgenFile
    cats = synth.pgen_ld_categories(21, 128, 203)
    data = synth.encode_pgen(cats, repeats=2)
    want = expected_rows(cats, 2)
    V, bpv = want.shape
    pitch = 64
    buf = torch.full((block * pitch,), SENTINEL, dtype=torch.uint8, device="cuda")
    with PgenFile(data) as pg:
        assert (pg.variants, pg.samples) == (V, 203)
        assert pg.device_bytes >= len(data)
        for b0 in range(0, V, block):
            n = min(block, V - b0)
            pg.decode(buf, pitch, b0, n)
            pg.check()
            got = buf[:n * pitch].view(n, pitch).cpu().numpy()
            np.testing.assert_array_equal(got[:, :bpv], want[b0:b0 + n], err_msg=f"block {b0}")
            assert (got[:, bpv:] == SENTINEL).all()


def test_range_errors(cuda):
    from gnomon_b200.pgen import PgenFile
    with PgenFile(ld_pgen()) as pg:
        buf = torch.zeros(64 * 10, dtype=torch.uint8, device="cuda")
        with pytest.raises(_lib.GnomonGpuError) as ei:
            pg.decode(buf, 64, 1495, 10)              # past the last variant
        assert ei.value.status == _lib.GNM_ERR_INVALID
        with pytest.raises(_lib.GnomonGpuError) as ei:
            pg.decode(buf, 56, 0, 10)                 # pitch not a multiple of 16
        assert ei.value.status == _lib.GNM_ERR_INVALID
        pg.decode(buf, 64, 0, 0)                      # empty range: nothing to do
        pg.check()


def test_list_decode(cuda):
    """Any order; LD records whose anchors are not listed read them from
    scratch rows (decoded once each); listed anchors are read from the output."""
    from gnomon_b200.pgen import PgenFile
    cats = synth.pgen_ld_categories(31, 256, 203)
    data = synth.encode_pgen(cats, repeats=2)
    want = expected_rows(cats, 2)
    kinds = pgen_oracle.parse_header(data)["types"] & 7
    ld = np.nonzero((kinds == 2) | (kinds == 3))[0]
    rng = np.random.default_rng(0)
    lists = [rng.permutation(len(want))[:100], ld[::3], np.array([ld[-1]]),
             np.arange(len(want))[::-1]]
    pitch = 64
    with PgenFile(data) as pg:
        for lst in lists:
            buf = torch.full((len(lst) * pitch,), SENTINEL, dtype=torch.uint8, device="cuda")
            pg.decode_list(buf, pitch, lst)
            pg.check()
            got = buf.view(len(lst), pitch).cpu().numpy()
            np.testing.assert_array_equal(got[:, :want.shape[1]], want[lst])
            assert (got[:, want.shape[1]:] == SENTINEL).all()
        with pytest.raises(_lib.GnomonGpuError) as ei:
            pg.decode_list(buf, pitch, [len(want)])          # past the last variant
        assert ei.value.status == _lib.GNM_ERR_INVALID


def test_zero_variants_and_missing_anchor(cuda):
    from gnomon_b200.pgen import PgenFile
    data = synth._pgen_file(7, [], [])
    rows, pitch = decode_to_device(data)
    with PgenFile(data) as pg:
        assert (pg.variants, pg.samples) == (0, 7)
        pg.decode(rows, pitch, 0, 0)
        pg.check()
    cats = synth.pgen_ld_categories(3, 8, 100)
    types, recs = synth._pgen_records(cats)
    first_ld = next(i for i, k in enumerate(types) if k in (2, 3))
    bad = synth._pgen_file(100, types[first_ld:], recs[first_ld:])
    with pytest.raises(_lib.GnomonGpuError) as ei:
        PgenFile(bad)
    assert ei.value.status == _lib.GNM_ERR_IO and "anchor" in str(ei.value)


def _dosage_case(n, V, seed, near_frac=0.6):
    """LD-linked categories and u16 ALT dosages: every missing call gets a
    value, most of them near a whole allele count; some calls get none."""
    rng = np.random.default_rng(seed)
    cats = synth.pgen_ld_categories(seed, V, n)
    cats[rng.random(cats.shape) < 0.05] = 3      # enough missing calls at any n
    dos = rng.integers(0, 32769, cats.shape).astype(np.uint16)
    near = rng.random(cats.shape) < near_frac
    dos[near] = (rng.integers(0, 3, near.sum()) * 16384 +
                 rng.integers(-1700, 1700, near.sum())).clip(0, 32768).astype(np.uint16)
    dos[rng.random(cats.shape) < 0.2] = 65535
    return cats, dos


@pytest.mark.parametrize("kind", ["list", "dense", "bits"])
@pytest.mark.parametrize("phase", [None, "all", "partial"])
@pytest.mark.parametrize("n", [5, 203, 4097, 70001])
def test_dosage_tracks_fill_missing_calls(cuda, kind, phase, n):
    """Dosage tracks of every layout (sample list, dense, presence bits),
    after either phase-track layout and followed by a phased-dosage track, on
    2-bit, 1-bit, fill and LD records: the device rows equal the oracle's
    (missing calls take the dosage's allele count within 0.10, hard calls
    stand), byte for byte, and the bytes past each row are untouched."""
    V = 60 if n < 10_000 else 12
    cats, dos = _dosage_case(n, V, seed=n)
    data = synth.encode_pgen_tracks(cats, dos, kind, phase, phased_dosage=kind != "list",
                                    seed=n + 1)
    want = pgen_oracle.decode_to_bed(data)
    assert not np.array_equal(want, expected_rows(cats))   # some calls were filled
    np.testing.assert_array_equal(device_rows(data, n), want)


def test_reference_dense_dosage_record_on_the_device(cuda):
    """shared/adapt_plink2.rs:3516-3570: categories {0, 1, 3, 3} with dense
    dosages {0, 18022, 18022, 18023} decode to ALT counts {0, 1, 1, missing}."""
    from test_pgen import _one_record_pgen
    cats = np.array([0, 1, 3, 3], np.uint8)
    body = bytes([int(cats[0] | (cats[1] << 2) | (cats[2] << 4) | (cats[3] << 6))])
    body += np.array([0, 18022, 18022, 18023], "<u2").tobytes()
    got = device_rows(_one_record_pgen(4, 0b0100_0000, body), 4)
    np.testing.assert_array_equal(got, expected_rows(np.array([[0, 1, 1, 3]], np.uint8)))


def test_truncated_dosage_track_is_an_io_error(cuda):
    """A dosage track cut short is reported (GNM_ERR_IO) and the context
    decodes the next file correctly."""
    from test_pgen import _one_record_pgen
    cats = np.array([3, 3, 3, 3, 0, 1], np.uint8)
    packed = synth.pack_codes(cats[None, :])[0]
    body = packed.tobytes() + np.array([16384, 0, 32768, 100, 0], "<u2").tobytes()  # one short
    with pytest.raises(_lib.GnomonGpuError) as ei:
        device_rows(_one_record_pgen(6, 0b0100_0000, body), 6)
    assert ei.value.status == _lib.GNM_ERR_IO
    test_reference_dense_dosage_record_on_the_device(cuda)


def test_score_from_dosage_pgen_equals_bed_of_the_filled_calls(cuda):
    """Scoring a .pgen whose missing calls carry dosages equals scoring the
    .bed rows the oracle fills them into (engine plain and tensor)."""
    people, V = 1501, 400
    w, prep, rows, _ = synth_case(people, V, 3)
    cats = _as_pgen(rows, people)
    rng = np.random.default_rng(4)
    dos = np.full(cats.shape, 65535, np.uint16)
    miss = cats == 3
    dos[miss] = (rng.integers(0, 3, miss.sum()) * 16384 +
                 rng.integers(-2000, 2000, miss.sum())).clip(0, 32768).astype(np.uint16)
    data = synth.encode_pgen_tracks(cats, dos, "list", "all", seed=2)
    filled = pgen_oracle.decode_to_bed(data)
    for engine in (_lib.ENGINE_PLAIN, _lib.ENGINE_TENSOR):
        s, c = score_pgen(prep, data, engine=engine)
        bs, bc = run(PipelineContext(prep), np.ascontiguousarray(filled).reshape(-1),
                     engine=engine)
        np.testing.assert_array_equal(c, bc)
        np.testing.assert_allclose(s, bs, rtol=1e-12, atol=1e-12)


# ---- multiallelic records ---------------------------------------------------------

from gnomon_b200.pgen import PgenFile                       # noqa: E402
from test_pgen import MA_COUNTS, alt_copy_rows, ma_case     # noqa: E402


def allele_rows(data, n, alt_counts, rows):
    """Decode (variant, ALT) rows into sentinel-filled device rows."""
    bpv = (n + 3) // 4
    pitch = (bpv + 127) // 128 * 128
    out = torch.full((max(len(rows), 1) * pitch,), SENTINEL, dtype=torch.uint8, device="cuda")
    with PgenFile(data, alt_counts=alt_counts) as pg:
        pg.decode_alleles(out, pitch, [v for v, _ in rows], [j for _, j in rows])
        pg.check()
    host = out[:len(rows) * pitch].view(len(rows), pitch).cpu().numpy()
    assert (host[:, bpv:] == SENTINEL).all(), "bytes past the row were changed"
    return host[:, :bpv]


@pytest.mark.parametrize("n", [3, 300, 4097, 70001])
@pytest.mark.parametrize("het_fmt,hom_fmt", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_multiallelic_rows(cuda, n, het_fmt, hom_fmt):
    """Every (variant, ALT) row of variants with 1-300 ALTs, patches as bit
    arrays or sample lists, with a phase track behind them."""
    alleles, rows = ma_case(n, seed=n + het_fmt * 2 + hom_fmt)
    rows = rows if n < 10_000 else [r for r in rows if r[1] <= 6]
    data = synth.encode_pgen_multiallelic(alleles, MA_COUNTS, het_fmt, hom_fmt, phase="partial")
    got = allele_rows(data, n, MA_COUNTS, rows)
    np.testing.assert_array_equal(got, pgen_oracle.decode_to_bed(data, MA_COUNTS, rows))
    np.testing.assert_array_equal(got, alt_copy_rows(alleles, rows))


def test_multiallelic_edges_and_dosages(cuda):
    """The reference's edges: an unpatched record gives every ALT row the plain
    categories, a patched record of a one-ALT variant reads as biallelic, and
    only ALT 1 rows take dosages; rows listed in any order, ALTs repeated."""
    n = 515
    alleles, rows = ma_case(n, seed=11)
    cats = synth.multiallelic_categories(alleles)
    dos = np.full(cats.shape, 65535, np.uint16)
    dos[cats == 3] = 32768
    patch = np.arange(len(MA_COUNTS)) % 3 != 2
    data = synth.encode_pgen_multiallelic(alleles, MA_COUNTS, 1, 0, patch=patch, dosage=dos,
                                          dosage_kind="bits", phase="all")
    rng = np.random.default_rng(2)
    rows = [rows[i] for i in rng.permutation(len(rows))] + rows[:5]
    np.testing.assert_array_equal(allele_rows(data, n, MA_COUNTS, rows),
                                  pgen_oracle.decode_to_bed(data, MA_COUNTS, rows))
    # given one ALT, a patched record reads as biallelic and its tracks are
    # then read from the patch bytes: the oracle and the decoder agree on the
    # rows, or both find the record malformed
    ones = [1] * len(MA_COUNTS)
    for v in range(len(MA_COUNTS)):
        try:
            want = pgen_oracle.decode_to_bed(data, ones, [(v, 1)])
        except pgen_oracle.PgenError:
            want = None
        if want is not None:
            np.testing.assert_array_equal(allele_rows(data, n, ones, [(v, 1)]), want)
        else:
            with pytest.raises(_lib.GnomonGpuError) as ei:
                allele_rows(data, n, ones, [(v, 1)])
            assert ei.value.status == _lib.GNM_ERR_IO


def test_multiallelic_argument_and_record_errors(cuda):
    n = 200
    alleles, rows = ma_case(n, seed=4)
    data = synth.encode_pgen_multiallelic(alleles, MA_COUNTS, 0, 0)
    pitch = 128
    out = torch.zeros(4 * pitch, dtype=torch.uint8, device="cuda")
    with pytest.raises(_lib.GnomonGpuError) as ei:
        PgenFile(data)                                     # ALT counts needed
    assert ei.value.status == _lib.GNM_ERR_INVALID
    with pytest.raises(_lib.GnomonGpuError) as ei:
        PgenFile(data, alt_counts=[0] + MA_COUNTS[1:])     # a variant with no ALT
    assert ei.value.status == _lib.GNM_ERR_INVALID
    with PgenFile(data, alt_counts=MA_COUNTS) as pg:
        for bad in ([1], [0], [3]):                        # variant 1 has two ALTs
            with pytest.raises(_lib.GnomonGpuError) as ei:
                pg.decode_alleles(out, pitch, [1], bad if bad != [1] else [9])
            assert ei.value.status == _lib.GNM_ERR_INVALID
    # one 3-ALT record (2-bit main track) whose patch is cut short or has an
    # unknown format: malformed, as the oracle finds too
    types, recs = synth._pgen_records(np.tile(np.arange(4, dtype=np.uint8), n // 4)[None, :n])
    main = recs[0]
    assert types[0] & 7 == 0
    for patch in (b"\x00", b"\x02", b"\xf1\x05"):       # no bit array; format 2; list cut
        bad = synth._pgen_file(n, [types[0] | 0x08], [main + patch])
        with pytest.raises(pgen_oracle.PgenError):
            pgen_oracle.decode_to_bed(bad, [3], [(0, 2)])
        with PgenFile(bad, alt_counts=[3]) as pg:
            pg.decode_alleles(out, pitch, [0], [2])
            with pytest.raises(_lib.GnomonGpuError) as ei:
                pg.check()
            assert ei.value.status == _lib.GNM_ERR_IO


def test_score_pgen_over_a_split_bim(cuda):
    """Scoring through a virtual .bim of (variant, ALT) rows equals scoring the
    oracle's decoded rows as a .bed."""
    n = 777
    alleles, rows = ma_case(n, seed=21)
    rows = [r for r in rows if r[1] <= 40]             # 75 virtual .bim rows
    data = synth.encode_pgen_multiallelic(alleles, MA_COUNTS, 1, 1)
    bed_rows = pgen_oracle.decode_to_bed(data, MA_COUNTS, rows)
    w, prep, _, _ = synth_case(n, len(rows), 4)
    for engine in (_lib.ENGINE_PLAIN, _lib.ENGINE_TENSOR):
        s, c = score_pgen(prep, data, engine=engine, alt_counts=MA_COUNTS,
                          bim_variant=[v for v, _ in rows], bim_alt=[j for _, j in rows])
        bs, bc = run(PipelineContext(prep), np.ascontiguousarray(bed_rows).reshape(-1),
                     engine=engine)
        np.testing.assert_array_equal(c, bc)
        np.testing.assert_allclose(s, bs, rtol=1e-12, atol=1e-12)
