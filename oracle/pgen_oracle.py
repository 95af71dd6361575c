"""CPU oracle for PGEN hard-call decoding — TEST INFRASTRUCTURE ONLY.

Only ``tests/`` and ``bench.py``'s CPU-baseline leg import this module, and
only as the checker. The product (``gnomon_b200``) never imports it.

It restates, in plain Python/numpy, how gnomon turns a PLINK 2 ``.pgen``
into the PLINK 1 ``.bed`` rows its scoring engine reads (the "virtual .bed"
of shared/adapt_plink2.rs). The restated steps are:

* the header (shared/adapt_plink2.rs:1512-1716): modes 0x02 (fixed-width
  hard calls) and 0x10 / 0x11 (variable-width). Record types are 4- or 8-bit
  per variant and record lengths 1-4 bytes, in 2^16-variant blocks, skipping
  the allele-count and reference-flag arrays;
* base-128 varints (:1721-1741), bit arrays (:1753-1777), sample-id widths
  (:1812-1822) and difflists (:1920-2040);
* the LD anchor, i.e. the most recent record in the same 2^16 block whose
  main track is not LD-compressed (:2237-2257);
* main-track types 0, 1, 2, 3, 4, 6 and 7, and the REF/ALT swap of type 3
  after its patch (:2574-2666);
* categories to A1 (= ALT, :927-935) dosage (:2682-2692);
* packing into .bed codes, with padding fields set to the missing code
  (:1136-1158).

* the dosage tracks of biallelic records (bits 5-7, :2416-2520): where the
  hard call is missing, the record's ALT dosage (u16, 16384 per allele copy)
  becomes the nearest whole allele count when it lies within 0.10 of it
  (f32 arithmetic, :3211-3255), else the call stays missing; hard calls are
  never overridden.  Samples are treated as diploid (the reference takes
  ploidy from the .pvar/.psam, which this decoder does not read).

* multiallelic records (vrtype bit 3, :2704-2881) when the input variants'
  ALT counts are given (the reference reads them from the .pvar): an output
  row is one (variant, ALT ordinal j) pair of the virtual .bim, and holds the
  number of copies of ALT j. Hets default to ALT 1 and hom-ALTs to ALT 1 / ALT
  1; the record's patch (one format nibble per category: 0 = bit array over
  the category's samples, 1 = id-only difflist, 15 = none; then fixed-width
  ALT values, or for two ALTs a hom-ALT2 flag array) overrides them. The
  reference's own edges are kept: a record without bit 3 gives every ALT row
  the plain categories, a bit-3 record of a variant with one ALT is read as
  biallelic without consuming its patch, and only the rows of ALT 1 read the
  dosage track (:2420). Without ALT counts, bit-3 records are rejected.
Difflists whose sample ids do not rise strictly are rejected as malformed
(PLINK 2 writes strictly rising ids; the reference would apply such a list in
order, later entries winning).
Phase tracks (bit 4) follow the main track and do not change hard calls.
Parity is pinned by the reference's own fixture pair data/testdata/ld.bed
and ld_p.pgen, which hold the same genotypes.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess
from pathlib import Path

import numpy as np

# genotype category (0 hom REF, 1 het, 2 hom ALT, 3 missing) -> .bed code of
# the A1 = ALT dosage (2 -> 00, 1 -> 10, 0 -> 11, missing -> 01)
CAT_TO_BED = np.array([0b11, 0b10, 0b00, 0b01], np.uint8)


class PgenError(ValueError):
    pass


def _varint(buf, cur):
    out, shift = 0, 0
    while True:
        if cur >= len(buf):
            raise PgenError("EOF in varint")
        b = buf[cur]
        cur += 1
        out |= (b & 0x7F) << shift
        if not b & 0x80:
            return out, cur
        shift += 7
        if shift > 63:
            raise PgenError("varint too large")


def _sid_bytes(n):
    return 1 if n <= 1 << 8 else 2 if n <= 1 << 16 else 3 if n <= 1 << 24 else 4


def _difflist(buf, cur, n):
    """-> (ids, cats, cursor after the list)."""
    length, cur = _varint(buf, cur)
    if length == 0:
        return [], [], cur
    groups = (length + 63) // 64
    w = _sid_bytes(n)
    first = []
    for _ in range(groups):
        first.append(int.from_bytes(buf[cur:cur + w], "little"))
        cur += w
    glen = [b + 63 for b in buf[cur:cur + groups - 1]]
    cur += groups - 1
    nvb = (length + 3) // 4
    vals = [(buf[cur + i // 4] >> (2 * (i % 4))) & 3 for i in range(length)]
    cur += nvb
    ids = []
    for g in range(groups):
        count = 64 if g < groups - 1 else length - 64 * (groups - 1)
        start = cur
        ids.append(first[g])
        for _ in range(count - 1):
            d, cur = _varint(buf, cur)
            if d == 0:
                raise PgenError("difflist sample ids do not rise")
            ids.append(ids[-1] + d)
        if g < groups - 1 and cur - start != glen[g]:
            raise PgenError("difflist group byte-length mismatch")
        if g < groups - 1 and ids[-1] >= first[g + 1]:
            raise PgenError("difflist sample ids do not rise")
    return ids, vals, cur


def _difflist_ids(buf, cur, n):
    """An id-only difflist (the dosage track's sample list, :1824-1918):
    -> (ids, cursor after the list)."""
    length, cur = _varint(buf, cur)
    if length == 0:
        return [], cur
    groups = (length + 63) // 64
    w = _sid_bytes(n)
    first = []
    for _ in range(groups):
        if cur + w > len(buf):
            raise PgenError("EOF in difflist first ids")
        first.append(int.from_bytes(buf[cur:cur + w], "little"))
        cur += w
    glen = [b + 63 for b in buf[cur:cur + groups - 1]]
    cur += groups - 1
    ids = []
    for g in range(groups):
        count = 64 if g < groups - 1 else length - 64 * (groups - 1)
        start = cur
        ids.append(first[g])
        for _ in range(count - 1):
            d, cur = _varint(buf, cur)
            ids.append(ids[-1] + d)
        if g < groups - 1 and cur - start != glen[g]:
            raise PgenError("difflist group byte-length mismatch")
    return ids, cur


DOSAGE_TOLERANCE = np.float32(0.10)


def dosage_to_hardcall(v: int) -> int:
    """u16 ALT dosage of a diploid sample -> allele count 0/1/2, or 255 when
    missing (65535) or farther than 0.10 from every whole count
    (shared/adapt_plink2.rs:3211-3255, f32 arithmetic)."""
    if v == 65535:
        return 255
    ds = np.float32(v) * np.float32(1.0 / 32768.0) * np.float32(2.0)
    best, best_d = 255, np.float32(np.inf)
    for c in range(3):
        d = np.float32(abs(ds - np.float32(c)))
        if d < best_d:
            best, best_d = c, d
    return best if best_d <= DOSAGE_TOLERANCE else 255


def _skip_phase(rec, cur, cats):
    """Cursor after a phase track (:2362-2413): one flag bit, then (flag set)
    one presence bit per het padded to a byte, then one bit per phased het."""
    if cur >= len(rec):
        raise PgenError("EOF in phase header")
    h = int(np.count_nonzero(cats == 1))
    bit = 1
    phased = h
    if rec[cur] & 1:
        pres = np.unpackbits(np.frombuffer(rec, np.uint8, (1 + h + 7) // 8, cur),
                             bitorder="little")[1:1 + h] if h else np.zeros(0, np.uint8)
        if len(pres) < h:
            raise PgenError("EOF in phase presence")
        phased = int(pres.sum())
        bit = 1 + h
        bit += (-bit) % 8
    bit += phased
    nbytes = (bit + 7) // 8
    if cur + nbytes > len(rec):
        raise PgenError("EOF in phase track")
    return cur + nbytes


def _dosage_overlay(rec, cur, t, n, cats):
    """Missing hard calls take their dosage's nearest allele count (:2416-2520)."""
    b5, b6 = bool(t & 0b0010_0000), bool(t & 0b0100_0000)
    if b5 and not b6:
        ids, cur = _difflist_ids(rec, cur, n)
    elif b6 and not b5:
        ids = list(range(n))
    else:
        if cur + (n + 7) // 8 > len(rec):
            raise PgenError("EOF in dosage presence bits")
        bits = np.unpackbits(np.frombuffer(rec, np.uint8, (n + 7) // 8, cur),
                             bitorder="little")[:n]
        ids = list(np.nonzero(bits)[0])
        cur += (n + 7) // 8
    if cur + 2 * len(ids) > len(rec):
        raise PgenError("EOF in dosage values")
    vals = np.frombuffer(rec, "<u2", len(ids), cur)
    out = cats.copy()
    for sid, v in zip(ids, vals):
        if sid < n and out[sid] == 3:
            hc = dosage_to_hardcall(int(v))
            if hc != 255:
                out[sid] = hc
    return out


def _bitarray_indices(rec, cur, nbits):
    """Set bits of an nbits-long bit array (:1753-1777) -> (indices, cursor)."""
    nbytes = (nbits + 7) // 8
    if cur + nbytes > len(rec):
        raise PgenError("EOF in bitarray")
    if nbits == 0:
        return [], cur
    bits = np.unpackbits(np.frombuffer(rec, np.uint8, nbytes, cur), bitorder="little")[:nbits]
    return [int(x) for x in np.nonzero(bits)[0]], cur + nbytes


def _packed(rec, cur, width, count):
    """``count`` fixed-width little-endian bit fields (:1779-1810) -> (values, cursor)."""
    if width == 0:
        return [0] * count, cur
    nbytes = (width * count + 7) // 8
    if cur + nbytes > len(rec):
        raise PgenError("EOF in packed values")
    bits = np.unpackbits(np.frombuffer(rec, np.uint8, nbytes, cur), bitorder="little")
    vals = [int(sum(int(bits[i * width + k]) << k for k in range(width))) for i in range(count)]
    return vals, cur + nbytes


def _het_width(ac):
    """Bits of one het's ALT value (value + 2 = its ALT) for ``ac`` ALTs."""
    return 0 if ac == 2 else 1 if ac == 3 else 2 if ac <= 5 else 4 if ac <= 17 else \
        8 if ac <= 257 else 16


def _homalt_width(ac):
    """Bits of one allele of a non-(1,1) hom-ALT-category pair (ac >= 3)."""
    return 2 if ac <= 4 else 4 if ac <= 16 else 8 if ac <= 256 else 16


def _patch_ids(rec, cur, n, fmt, members, what):
    if fmt == 0:
        idx, cur = _bitarray_indices(rec, cur, len(members))
        return [int(members[i]) for i in idx], cur
    if fmt == 1:
        ids, cur = _difflist_ids(rec, cur, n)
        if any(b <= a for a, b in zip(ids, ids[1:])):
            raise PgenError("multiallelic patch sample ids do not rise")
        return ids, cur
    raise PgenError(f"unsupported multiallelic {what} patch format")


def _project_multiallelic(rec, cur, n, cats, alt_count, alt_ord):
    """Copies of ALT ``alt_ord`` per sample (as categories 0/1/2, 3 missing)
    and the cursor after the patch (:2704-2881)."""
    if alt_count <= 1:
        return cats.copy(), cur            # read as biallelic; the patch is not consumed
    if cur >= len(rec):
        raise PgenError("EOF before multiallelic patch header")
    fmt = rec[cur]
    cur += 1
    f1, f2 = fmt & 15, fmt >> 4
    het_alt, pair = {}, {}
    if f1 != 15:
        sids, cur = _patch_ids(rec, cur, n, f1, np.nonzero(cats == 1)[0], "het")
        w = _het_width(alt_count)
        vals, cur = _packed(rec, cur, w, len(sids))
        for sid, v in zip(sids, vals):
            het_alt[sid] = 2 if w == 0 else v + 2
    if f2 != 15:
        sids, cur = _patch_ids(rec, cur, n, f2, np.nonzero(cats == 2)[0], "hom-ALT")
        k = len(sids)
        if alt_count == 2:
            flags, cur = _bitarray_indices(rec, cur, k)
            two = set(flags)
            for i, sid in enumerate(sids):
                pair[sid] = (2, 2) if i in two else (1, 2)
        else:
            vals, cur = _packed(rec, cur, _homalt_width(alt_count), 2 * k)
            for i, sid in enumerate(sids):
                lo, hi = vals[2 * i] + 1, vals[2 * i + 1] + 1
                pair[sid] = (min(lo, hi), max(lo, hi))
    out = cats.copy()
    for i in np.nonzero(cats == 1)[0]:
        out[i] = 1 if het_alt.get(int(i), 1) == alt_ord else 0
    for i in np.nonzero(cats == 2)[0]:
        p = pair.get(int(i), (1, 1))
        out[i] = int(p[0] == alt_ord) + int(p[1] == alt_ord)
    return out, cur


def parse_header(data: bytes):
    """-> dict(mode, variants, samples, offsets[V], types[V], lens[V])."""
    if len(data) < 12 or data[0] != 0x6C or data[1] != 0x1B:
        raise PgenError("not a PGEN (bad magic)")
    mode = data[2]
    m, n = struct.unpack_from("<II", data, 3)
    if mode == 0x02:
        # the reference's reader puts the body after 13 bytes, plus the
        # reference-flag bit array in flag mode 3 (:2048-2057; its test at
        # :3826-3866 asserts 12 + 1)
        rec = (n + 3) // 4
        base = 13 + ((m + 7) // 8 if ((data[11] >> 6) & 3) == 3 else 0)
        offs = base + rec * np.arange(m, dtype=np.uint64)
        return dict(mode=mode, variants=m, samples=n, offsets=offs,
                    types=np.zeros(m, np.uint8), lens=np.full(m, rec, np.uint32))
    if mode not in (0x10, 0x11):
        raise PgenError(f"unsupported PGEN mode 0x{mode:02x}")
    fmt = data[11]
    type_bits = 4 if (fmt & 0x0F) <= 3 else 8
    len_bytes = (fmt & 0x07) % 4 + 1
    ac_bytes = {0: 0, 1: 1, 2: 2, 3: 4}[(fmt >> 4) & 3]
    ref_flag_mode = (fmt >> 6) & 3
    blocks = (m + 0xFFFF) >> 16
    off = 12
    block_offs = list(struct.unpack_from(f"<{blocks}Q", data, off))
    off += 8 * blocks
    types = np.zeros(m, np.uint8)
    lens = np.zeros(m, np.uint32)
    idx = 0
    for _ in range(blocks):
        cnt = min(m - idx, 1 << 16)
        if type_bits == 4:
            raw = np.frombuffer(data, np.uint8, (cnt + 1) // 2, off)
            t = np.empty(2 * len(raw), np.uint8)
            t[0::2], t[1::2] = raw & 15, raw >> 4
            types[idx:idx + cnt] = t[:cnt]
            off += (cnt + 1) // 2
        else:
            types[idx:idx + cnt] = np.frombuffer(data, np.uint8, cnt, off)
            off += cnt
        raw = np.frombuffer(data, np.uint8, cnt * len_bytes, off).reshape(cnt, len_bytes)
        lens[idx:idx + cnt] = sum(raw[:, j].astype(np.uint32) << (8 * j) for j in range(len_bytes))
        off += cnt * len_bytes + cnt * ac_bytes
        if ref_flag_mode == 3:
            off += (cnt + 7) // 8
        idx += cnt
    offsets = np.zeros(m, np.uint64)
    for b in range(blocks):
        lo, hi = b << 16, min(m, (b + 1) << 16)
        offsets[lo] = block_offs[b]
        offsets[lo + 1:hi] = block_offs[b] + np.cumsum(lens[lo:hi - 1].astype(np.uint64))
    return dict(mode=mode, variants=m, samples=n, offsets=offsets, types=types, lens=lens)


def _main_track(rec, kind, n, anchor):
    """-> (categories [n], cursor after the main track)."""
    cats = np.full(n, 3, np.uint8)
    cur = 0
    if kind == 0:
        if len(rec) < (n + 3) // 4:
            raise PgenError("EOF in 2-bit array")
        raw = np.frombuffer(rec, np.uint8, (n + 3) // 4)
        c = np.stack([(raw >> (2 * s)) & 3 for s in range(4)], 1).reshape(-1)[:n]
        return c.astype(np.uint8), (n + 3) // 4
    if kind == 1:
        pairs = {1: (0, 1), 2: (0, 2), 3: (0, 3), 5: (1, 2), 6: (1, 3), 9: (2, 3)}
        if rec[0] not in pairs:
            raise PgenError("invalid 1-bit pair code")
        low, high = pairs[rec[0]]
        bits = np.unpackbits(np.frombuffer(rec, np.uint8, (n + 7) // 8, 1),
                             bitorder="little")[:n]
        cats = np.where(bits == 1, high, low).astype(np.uint8)
        cur = 1 + (n + 7) // 8
    elif kind in (2, 3):
        cats = anchor.copy()
    elif kind in (4, 6, 7):
        cats[:] = {4: 0, 6: 2, 7: 3}[kind]
    else:
        raise PgenError(f"unsupported main-track type {kind}")
    ids, vals, cur = _difflist(rec, cur, n)
    for i, v in zip(ids, vals):
        if i < n:
            cats[i] = v
    if kind == 3:
        cats = np.where(cats == 0, 2, np.where(cats == 2, 0, cats)).astype(np.uint8)
    return cats, cur


def decode_to_bed(data: bytes, alt_counts=None, rows=None) -> np.ndarray:
    """Decode -> [R][ceil(N/4)] .bed rows (padding fields = 01).

    Without ``rows``: one row per variant (ALT 1). ``rows`` = [(variant, ALT
    ordinal)] pairs of a virtual .bim; ``alt_counts`` = each input variant's
    ALT count, needed when a record carries a multiallelic patch."""
    h = parse_header(data)
    m, n = h["variants"], h["samples"]
    bpv = (n + 3) // 4
    ac = None if alt_counts is None else [int(x) for x in alt_counts]
    if ac is not None and len(ac) != m:
        raise PgenError("one ALT count per variant")
    # every record's main track, in file order (LD records read their anchors')
    main, anchor, anchor_idx = [], None, -1
    for v in range(m):
        t = int(h["types"][v])
        if (t & 0b0000_1000) and ac is None:
            raise PgenError(f"variant {v}: multiallelic tracks need the ALT counts")
        if (t & 0b1000_0000) and not (t & 0b0110_0000):
            raise PgenError(f"variant {v}: phased dosage track without a dosage track")
        kind = t & 7
        rec = data[int(h["offsets"][v]):int(h["offsets"][v]) + int(h["lens"][v])]
        if kind in (2, 3):
            if anchor is None or (anchor_idx >> 16) != (v >> 16):
                raise PgenError(f"variant {v}: LD-compressed record without an anchor in its block")
            cats, cur = _main_track(rec, kind, n, anchor)
        else:
            cats, cur = _main_track(rec, kind, n, None)
            anchor, anchor_idx = cats, v   # anchors are the raw main-track categories
        main.append((rec, t, cats, cur))
    plan = [(v, 1) for v in range(m)] if rows is None else list(rows)
    out = np.zeros((len(plan), bpv), np.uint8)
    for r, (v, j) in enumerate(plan):
        rec, t, cats, cur = main[v]
        a = 1 if ac is None else ac[v]
        if ac is not None and not 1 <= j <= max(a, 1):
            raise PgenError(f"row {r}: ALT ordinal {j} of a variant with {a} ALT alleles")
        got = cats
        if t & 0b0000_1000:
            got, cur = _project_multiallelic(rec, cur, n, cats, a, j)
        if t & 0b0001_0000:
            cur = _skip_phase(rec, cur, cats)       # het count of the main track
        if t & 0b0110_0000:
            filled = _dosage_overlay(rec, cur, t, n, got)
            if a <= 1 or j == 1:
                got = filled
        codes = np.full(bpv * 4, 0b01, np.uint8)
        codes[:n] = CAT_TO_BED[got]
        q = codes.reshape(bpv, 4)
        out[r] = q[:, 0] | (q[:, 1] << 2) | (q[:, 2] << 4) | (q[:, 3] << 6)
    return out


# ---- the C restatement (pgen_oracle.c), for timing a compiled CPU decoder ----

_HERE = Path(__file__).resolve().parent
_CLIB = _HERE / "_build" / "libpgen_oracle.so"
_clib = None


def _load_c():
    global _clib
    if _clib is None:
        src = _HERE / "pgen_oracle.c"
        if not _CLIB.exists() or _CLIB.stat().st_mtime < src.stat().st_mtime:
            subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
        lib = C.CDLL(str(_CLIB))
        lib.pgen_oracle_dims.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64),
                                         C.POINTER(C.c_uint64)]
        lib.pgen_oracle_dims.restype = C.c_int
        lib.pgen_oracle_decode.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_int]
        lib.pgen_oracle_decode.restype = C.c_int
        _clib = lib
    return _clib


def decode_to_bed_c(data, threads: int = 0) -> np.ndarray:
    """decode_to_bed through the C restatement on `threads` host threads
    (0 = all); raises PgenError where decode_to_bed does."""
    lib = _load_c()
    buf = np.frombuffer(bytes(data), np.uint8) if not isinstance(data, np.ndarray) else \
        np.ascontiguousarray(data, np.uint8)
    m, n = C.c_uint64(), C.c_uint64()
    if lib.pgen_oracle_dims(buf.ctypes.data, buf.nbytes, C.byref(m), C.byref(n)):
        raise PgenError("not a supported .pgen")
    bpv = (n.value + 3) // 4
    out = np.zeros((m.value, bpv), np.uint8)
    rc = lib.pgen_oracle_decode(buf.ctypes.data, buf.nbytes, out.ctypes.data, bpv,
                                threads or (os.cpu_count() or 1))
    if rc:
        raise PgenError("malformed or unsupported .pgen")
    return out
