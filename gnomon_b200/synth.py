"""Deterministic synthetic workloads for the scoring hot path.

Genotypes follow Hardy-Weinberg: per variant an allele frequency
``p ~ U(p_lo, p_hi)``, per call ``missing`` with probability ``r`` (PLINK code
01) else ``Binomial(2, p)`` allele-2 copies (00 / 10 / 11).  Every call is a
pure function of ``(seed, variant, person)`` through a SplitMix64 counter hash,
so the CUDA generator (``gnm_synth_fill_device``), the C oracle and the numpy
reference below produce byte-identical ``.bed`` rows.

Per-variant thresholds are computed here in float64 (IEEE, no fused ops) and
handed to every generator as uint32 triples ``{t_missing, T0, T1}``:
``code = 01 if u_m < t_missing else 00 if u_g < T0 else 10 if u_g < T1 else 11``
with ``(u_m, u_g)`` the low / high halves of ``mix64(key(seed, v, i))``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

SEED_BASE = 0x676E6F6D6F6E  # "gnomon"
M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def mix64(z: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser on uint64 arrays (wrapping arithmetic)."""
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def allele_freqs(seed: int, v0: int, n: int, p_lo: float, p_hi: float) -> np.ndarray:
    v = np.arange(v0, v0 + n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        h = mix64(np.uint64(seed ^ 0x5DEECE66D) ^ (v * np.uint64(0x9E3779B97F4A7C15)))
    u = (h >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    return p_lo + (p_hi - p_lo) * u


def variant_thresholds(seed: int, v0: int, n: int, p_lo: float, p_hi: float,
                       missing_rate: float) -> np.ndarray:
    """uint32 [n, 3] thresholds {t_missing, T0, T1} for variants v0..v0+n."""
    p = allele_freqs(seed, v0, n, p_lo, p_hi)
    two32 = 4294967296.0
    t = np.empty((n, 3), dtype=np.uint32)
    t[:, 0] = np.uint32(min(np.floor(missing_rate * two32), two32 - 1))
    q = 1.0 - p
    t[:, 1] = np.minimum(np.floor(q * q * two32), two32 - 1).astype(np.uint32)
    t[:, 2] = np.minimum(np.floor((1.0 - p * p) * two32), two32 - 1).astype(np.uint32)
    return t


def genotype_codes(seed: int, v0: int, n: int, num_people: int, thr: np.ndarray,
                   person_begin: int = 0) -> np.ndarray:
    """Reference numpy generator: uint8 codes [n, num_people] (0..3) of cohort
    people person_begin .. person_begin + num_people - 1."""
    v = np.arange(v0, v0 + n, dtype=np.uint64)[:, None]
    i = np.arange(person_begin, person_begin + num_people, dtype=np.uint64)[None, :]
    with np.errstate(over="ignore"):
        key = mix64(np.uint64(seed)) ^ (v * np.uint64(0xD1B54A32D192ED03)) \
            ^ (i * np.uint64(0x8CB92BA72F3D8DD7))
    x = mix64(key)
    um = (x & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    ug = (x >> np.uint64(32)).astype(np.uint32)
    tm, t0, t1 = thr[:, 0:1], thr[:, 1:2], thr[:, 2:3]
    code = np.where(ug < t0, 0, np.where(ug < t1, 2, 3)).astype(np.uint8)
    code[um < tm] = 1
    return code


def pack_codes(codes: np.ndarray, pitch: int | None = None) -> np.ndarray:
    """Pack [n, P] 2-bit codes into SNP-major .bed rows [n, pitch] (person i at bits 2*(i%4))."""
    n, P = codes.shape
    bpv = (P + 3) // 4
    pitch = pitch or bpv
    padded = np.zeros((n, bpv * 4), dtype=np.uint8)
    padded[:, :P] = codes
    q = padded.reshape(n, bpv, 4).astype(np.uint8)
    packed = q[:, :, 0] | (q[:, :, 1] << 2) | (q[:, :, 2] << 4) | (q[:, :, 3] << 6)
    out = np.zeros((n, pitch), dtype=np.uint8)
    out[:, :bpv] = packed
    return out


def unpack_codes(rows: np.ndarray, num_people: int) -> np.ndarray:
    """Inverse of pack_codes: uint8 codes [n, num_people]."""
    n = rows.shape[0]
    bpv = (num_people + 3) // 4
    r = rows[:, :bpv]
    c = np.stack([(r >> (2 * q)) & 3 for q in range(4)], axis=-1).reshape(n, bpv * 4)
    return c[:, :num_people].astype(np.uint8)


def synth_rows(seed: int, v0: int, n: int, num_people: int, thr: np.ndarray,
               pitch: int | None = None, person_begin: int = 0) -> np.ndarray:
    return pack_codes(genotype_codes(seed, v0, n, num_people, thr, person_begin), pitch)


# ---------------------------------------------------------------------------
# Named workloads (the reference's benchmark shapes, synthetic data)
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class Workload:
    name: str
    people: int
    variants: int
    scores: int
    p_lo: float
    p_hi: float
    missing_rate: float
    sigma: float
    flip_frac: float = 0.10
    size_lo: int = 0          # uneven score sizes (0 = every score covers every variant)
    size_hi: int = 0
    config_id: int = 0

    @property
    def seed(self) -> int:
        return SEED_BASE + self.config_id

    @property
    def bytes_per_variant(self) -> int:
        return (self.people + 3) // 4


WORKLOADS = {
    "plain_2k_x_50k": Workload("plain_2k_x_50k", 2_000, 50_000, 1, 0.01, 0.5, 0.01, 0.01,
                               config_id=1),
    "bandwidth_50k_x_1m": Workload("bandwidth_50k_x_1m", 50_000, 1_000_000, 1, 0.01, 0.5,
                                   0.005, 0.005, config_id=2),
    "batched_100k_x_500k_k512": Workload("batched_100k_x_500k_k512", 100_000, 500_000, 512,
                                         0.01, 0.5, 0.01, 0.01, size_lo=10_000,
                                         size_hi=500_000, config_id=3),
    "diff_20k_x_200k_k16": Workload("diff_20k_x_200k_k16", 20_000, 200_000, 16, 0.01, 0.5,
                                    0.01, 0.01, config_id=4),
    "biobank_500k_x_1p2m_k64": Workload("biobank_500k_x_1p2m_k64", 500_000, 1_200_000, 64,
                                        0.005, 0.5, 0.02, 0.01, size_lo=50_000,
                                        size_hi=1_200_000, config_id=5),
}


def scaled(w: Workload, people: int, variants: int, scores: int | None = None) -> Workload:
    """Same generator and distributions at a smaller shape (parity-test sizes)."""
    k = w.scores if scores is None else scores
    # uneven score sizes keep their fraction of the variant count
    lo = max(1, w.size_lo * variants // w.variants) if w.size_lo else 0
    hi = max(lo, w.size_hi * variants // w.variants) if w.size_hi else 0
    return Workload(w.name + f"_scaled_{people}x{variants}x{k}", people, variants, k, w.p_lo,
                    w.p_hi, w.missing_rate, w.sigma, w.flip_frac, lo, hi, w.config_id)


def score_cells(w: Workload, chunk: int = 1 << 16):
    """(row_offsets u64[V+1], cols u32[nnz], weight f32[nnz], flipped bool[nnz]).

    Every score covers every variant when ``size_lo == 0``; otherwise score k
    keeps each variant with probability n_k / V, n_k ~ U(size_lo, size_hi)
    (a hashed Bernoulli subset, so the expected size is n_k).
    """
    V, K = w.variants, w.scores
    rng = np.random.default_rng(w.seed)
    if not w.size_lo:
        offs = np.arange(0, (V + 1) * K, K, dtype=np.uint64)
        cols = np.tile(np.arange(K, dtype=np.uint32), V)
        nnz = V * K
    else:
        sizes = rng.integers(w.size_lo, w.size_hi + 1, size=K)
        thr = np.minimum(np.floor(sizes / V * 2.0 ** 32), 2.0 ** 32 - 1).astype(np.uint64)
        counts = np.zeros(V, dtype=np.uint64)
        col_parts = []
        ks = np.arange(K, dtype=np.uint64)[None, :]
        for v0 in range(0, V, chunk):
            v = np.arange(v0, min(V, v0 + chunk), dtype=np.uint64)[:, None]
            with np.errstate(over="ignore"):
                h = mix64(np.uint64(w.seed ^ 0xC3A5C85C97CB3127) ^ (v * np.uint64(0xFF51AFD7ED558CCD))
                          ^ (ks * np.uint64(0xC4CEB9FE1A85EC53)))
            member = (h >> np.uint64(32)) < thr[None, :]
            counts[v0:v0 + member.shape[0]] = member.sum(axis=1)
            col_parts.append(np.nonzero(member)[1].astype(np.uint32))
        cols = np.concatenate(col_parts) if col_parts else np.zeros(0, np.uint32)
        offs = np.zeros(V + 1, dtype=np.uint64)
        np.cumsum(counts, out=offs[1:])
        nnz = int(offs[-1])
    weight = (rng.standard_normal(nnz) * w.sigma).astype(np.float32)
    flipped = rng.random(nnz) < w.flip_frac
    return offs, cols, weight, flipped


# ---- synthetic PLINK 2 .pgen files ------------------------------------------------

# PGEN genotype category (0 hom REF, 1 het, 2 hom ALT, 3 missing) <-> .bed
# code.  gnomon's virtual .bed writes category c as the .bed code of the
# A1 = ALT dosage: 2 -> 00, 1 -> 10, 0 -> 11, missing -> 01.
PGEN_CAT_TO_BED = np.array([0b11, 0b10, 0b00, 0b01], np.uint8)
BED_TO_PGEN_CAT = np.array([2, 3, 1, 0], np.uint8)   # inverse of PGEN_CAT_TO_BED


def _varint_bytes(x: int) -> bytes:
    out = bytearray()
    while True:
        b = x & 0x7F
        x >>= 7
        if x:
            out.append(b | 0x80)
        else:
            out.append(b)
            return bytes(out)


def _varints(d: np.ndarray):
    """Base-128 varints of an array -> (bytes as uint8 array, bytes per value)."""
    d = np.asarray(d, np.uint64)
    nb = np.ones(len(d), np.int64)
    for k in range(1, 10):
        nb += d >= np.uint64(1) << np.uint64(7 * k)
    out = np.empty(int(nb.sum()), np.uint8)
    starts = np.concatenate([[0], np.cumsum(nb)[:-1]]).astype(np.int64)
    for k in range(int(nb.max()) if len(d) else 0):
        sel = nb > k
        byte = ((d[sel] >> np.uint64(7 * k)) & np.uint64(0x7F)).astype(np.uint8)
        out[starts[sel] + k] = byte | ((nb[sel] > k + 1).astype(np.uint8) << 7)
    return out, nb


def _difflist_bytes(ids: np.ndarray, cats: np.ndarray, n: int) -> bytes:
    """A PLINK 2 difflist of (sample id, category) pairs, ids ascending."""
    ids = np.asarray(ids, np.int64)
    length = len(ids)
    out = bytearray(_varint_bytes(length))
    if length == 0:
        return bytes(out)
    wid = 1 if n <= 1 << 8 else 2 if n <= 1 << 16 else 3 if n <= 1 << 24 else 4
    groups = (length + 63) // 64
    first = ids[::64]
    out += b"".join(int(f).to_bytes(wid, "little") for f in first)
    # deltas inside each group (the first id of a group carries no delta)
    in_group = np.arange(length) % 64 != 0
    deltas = np.diff(ids, prepend=0)[in_group]
    vbytes, nb = _varints(deltas)
    group_of = (np.arange(length) // 64)[in_group]
    gbytes = np.bincount(group_of, weights=nb, minlength=groups).astype(np.int64)
    out += (gbytes[:groups - 1] - 63).astype(np.uint8).tobytes()
    vals = np.zeros((length + 3) // 4 * 4, np.uint8)
    vals[:length] = cats
    q = vals.reshape(-1, 4)
    out += (q[:, 0] | (q[:, 1] << 2) | (q[:, 2] << 4) | (q[:, 3] << 6)).astype(np.uint8).tobytes()
    out += vbytes.tobytes()
    return bytes(out)


def _pgen_records(cats: np.ndarray):
    """Genotype categories [V][N] -> (record types, record bodies), each variant
    in the smallest of the encodings ``encode_pgen`` lists."""
    cats = np.asarray(cats, np.uint8)
    V, n = cats.shape
    pair_code = {(0, 1): 1, (0, 2): 2, (0, 3): 3, (1, 2): 5, (1, 3): 6, (2, 3): 9}
    recs, types = [], []
    anchor = None
    for v in range(V):
        c = cats[v]
        if v % (1 << 16) == 0:
            anchor = None
        options = []
        q = np.zeros((n + 3) // 4 * 4, np.uint8)
        q[:n] = c
        q = q.reshape(-1, 4)
        options.append((0, (q[:, 0] | (q[:, 1] << 2) | (q[:, 2] << 4) | (q[:, 3] << 6))
                        .astype(np.uint8).tobytes()))
        counts = np.bincount(c, minlength=4)
        top = np.argsort(-counts, kind="stable")[:2]
        low, high = int(min(top)), int(max(top))
        if counts[low] > 0 and counts[high] > 0:
            bits = np.zeros((n + 7) // 8 * 8, np.uint8)
            bits[:n] = c == high
            rest = np.nonzero((c != low) & (c != high))[0]
            body = bytes([pair_code[(low, high)]]) + np.packbits(bits, bitorder="little").tobytes()
            options.append((1, body + _difflist_bytes(rest, c[rest], n)))
        for kind, fill in ((4, 0), (6, 2), (7, 3)):
            diff = np.nonzero(c != fill)[0]
            if len(diff) < n // 8:
                options.append((kind, _difflist_bytes(diff, c[diff], n)))
        if anchor is not None:
            diff = np.nonzero(c != anchor)[0]
            options.append((2, _difflist_bytes(diff, c[diff], n)))
            swapped = np.where(c == 0, 2, np.where(c == 2, 0, c)).astype(np.uint8)
            diff = np.nonzero(swapped != anchor)[0]
            options.append((3, _difflist_bytes(diff, swapped[diff], n)))
        kind, body = min(options, key=lambda o: len(o[1]))
        recs.append(body)
        types.append(kind)
        if kind not in (2, 3):
            anchor = c
    return types, recs


def _pgen_file(n: int, types, recs) -> bytes:
    V = len(recs)
    blocks = (V + 0xFFFF) >> 16
    head = bytearray(b"\x6c\x1b\x10")
    head += np.array([V, n], "<u4").tobytes()
    head.append(0x07)                       # 8-bit types, 4-byte lengths, no allele counts
    index_len = 8 * blocks + sum(min(V - (b << 16), 1 << 16) * 5 for b in range(blocks))
    off = len(head) + index_len
    block_offs, pos = [], off
    for b in range(blocks):
        block_offs.append(pos)
        pos += sum(len(r) for r in recs[b << 16:(b + 1) << 16])
    head += np.array(block_offs, "<u8").tobytes()
    for b in range(blocks):
        lo, hi = b << 16, min(V, (b + 1) << 16)
        head += np.array(types[lo:hi], np.uint8).tobytes()
        head += np.array([len(r) for r in recs[lo:hi]], "<u4").tobytes()
    assert len(head) == off
    return bytes(head) + b"".join(recs)


def _difflist_id_bytes(ids: np.ndarray, n: int) -> bytes:
    """An id-only difflist (a dosage track's sample list): varint length,
    first ids, group byte lengths minus 63, base-128 deltas."""
    ids = np.asarray(ids, np.int64)
    length = len(ids)
    out = bytearray(_varint_bytes(length))
    if length == 0:
        return bytes(out)
    wid = 1 if n <= 1 << 8 else 2 if n <= 1 << 16 else 3 if n <= 1 << 24 else 4
    groups = (length + 63) // 64
    out += b"".join(int(f).to_bytes(wid, "little") for f in ids[::64])
    in_group = np.arange(length) % 64 != 0
    deltas = np.diff(ids, prepend=0)[in_group]
    vbytes, nb = _varints(deltas)
    group_of = (np.arange(length) // 64)[in_group]
    gbytes = np.bincount(group_of, weights=nb, minlength=groups).astype(np.int64)
    out += (gbytes[:groups - 1] - 63).astype(np.uint8).tobytes()
    out += vbytes.tobytes()
    return bytes(out)


def _phase_track(cats_v: np.ndarray, rng, partial: bool) -> bytes:
    """A phase track for the hets of one variant: all hets phased (flag 0),
    or (partial) a presence bit per het, padded to a byte, then one phase bit
    per present het."""
    h = int(np.count_nonzero(cats_v == 1))
    if not partial:
        bits = np.concatenate([[0], rng.integers(0, 2, h)]).astype(np.uint8)
    else:
        pres = rng.integers(0, 2, h).astype(np.uint8)
        head = np.concatenate([[1], pres]).astype(np.uint8)
        head = np.concatenate([head, np.zeros((-len(head)) % 8, np.uint8)])
        bits = np.concatenate([head, rng.integers(0, 2, int(pres.sum()))]).astype(np.uint8)
    return np.packbits(bits, bitorder="little").tobytes()


def _dosage_track(dos_v: np.ndarray, kind: str, phased: bool, rng) -> tuple[int, bytes]:
    """(type bits, track bytes) of one variant's u16 ALT dosages; 65535 marks
    samples without a value.  kind: "list" (id difflist, bit 5), "dense"
    (every sample, bit 6) or "bits" (presence bit array, bits 5+6); phased
    adds a phased-dosage track (bit 7)."""
    n = len(dos_v)
    present = np.nonzero(dos_v != 65535)[0]
    if kind == "dense":
        bits, body, d = 0b0100_0000, dos_v.astype("<u2").tobytes(), n
    elif kind == "list":
        bits = 0b0010_0000
        body = _difflist_id_bytes(present, n) + dos_v[present].astype("<u2").tobytes()
        d = len(present)
    elif kind == "bits":
        bits = 0b0110_0000
        mask = np.zeros(n, np.uint8)
        mask[present] = 1
        body = np.packbits(mask, bitorder="little").tobytes() + dos_v[present].astype("<u2").tobytes()
        d = len(present)
    else:
        raise ValueError(kind)
    if phased:
        bits |= 0b1000_0000
        if kind == "dense":
            body += rng.integers(0, 65535, n).astype("<u2").tobytes()
        else:
            pres = rng.integers(0, 2, d).astype(np.uint8)
            body += np.packbits(pres, bitorder="little").tobytes()
            body += rng.integers(0, 65535, int(pres.sum())).astype("<u2").tobytes()
    return bits, body


def encode_pgen_tracks(cats: np.ndarray, dosage: np.ndarray | None = None,
                       dosage_kind: str | list = "list", phase: str | None = None,
                       phased_dosage: bool = False, seed: int = 0) -> bytes:
    """encode_pgen plus the tracks that follow a record's main track: a phase
    track (phase = "all" or "partial") and a dosage track holding
    ``dosage[v]`` (u16 ALT dosages, 16384 per allele copy, 65535 = no value)
    of each variant that has a value, as a sample list, dense array or
    presence bit array (``dosage_kind``, one for all variants or one per
    variant)."""
    cats = np.asarray(cats, np.uint8)
    V, n = cats.shape
    rng = np.random.default_rng(seed)
    types, recs = _pgen_records(cats)
    types, recs = list(types), list(recs)
    for v in range(V):
        body = recs[v]
        if phase is not None:
            body = body + _phase_track(cats[v], rng, phase == "partial")
            types[v] |= 0b0001_0000
        if dosage is not None and np.any(dosage[v] != 65535):
            kind = dosage_kind if isinstance(dosage_kind, str) else dosage_kind[v]
            bits, track = _dosage_track(np.asarray(dosage[v], np.uint16), kind, phased_dosage, rng)
            body = body + track
            types[v] |= bits
        recs[v] = body
    return _pgen_file(n, types, recs)


def _bitarray_bytes(bits) -> bytes:
    bits = np.asarray(bits, np.uint8)
    return np.packbits(bits, bitorder="little").tobytes() if len(bits) else b""


def _packed_bytes(vals, width: int) -> bytes:
    if width == 0 or len(vals) == 0:
        return b""
    vals = np.asarray(vals, np.uint64)
    bits = ((vals[:, None] >> np.arange(width, dtype=np.uint64)) & 1).astype(np.uint8).ravel()
    return np.packbits(bits, bitorder="little").tobytes()


def _het_alt_width(ac: int) -> int:
    return 0 if ac == 2 else 1 if ac == 3 else 2 if ac <= 5 else 4 if ac <= 17 else \
        8 if ac <= 257 else 16


def _homalt_pair_width(ac: int) -> int:
    return 2 if ac <= 4 else 4 if ac <= 16 else 8 if ac <= 256 else 16


def multiallelic_categories(alleles: np.ndarray) -> np.ndarray:
    """Per-sample allele pairs [V][N][2] (0 REF, 1.. ALT ordinal, -1 missing)
    -> PGEN categories [V][N]: 3 missing, else the number of non-REF alleles."""
    a = np.asarray(alleles)
    miss = (a < 0).any(axis=2)
    c = (a > 0).sum(axis=2).astype(np.uint8)
    c[miss] = 3
    return c


def _multiallelic_patch(cats_v, alleles_v, ac: int, het_fmt: int, hom_fmt: int,
                        swap_pairs: bool) -> bytes:
    """The multiallelic patch of one record: hets whose ALT is not ALT 1, and
    hom-ALT-category samples whose allele pair is not (1, 1).  het_fmt /
    hom_fmt: 0 = bit array over the category's samples, 1 = id difflist; a
    category with nothing to patch is written as 15 (absent)."""
    n = len(cats_v)
    het = np.nonzero(cats_v == 1)[0]
    hom = np.nonzero(cats_v == 2)[0]
    het_alt = alleles_v[het].max(axis=1)
    het_mask = het_alt != 1
    pairs = np.sort(alleles_v[hom], axis=1)
    hom_mask = ~((pairs[:, 0] == 1) & (pairs[:, 1] == 1))
    f1 = het_fmt if het_mask.any() else 15
    f2 = hom_fmt if hom_mask.any() else 15
    out = bytearray([f1 | (f2 << 4)])
    if f1 != 15:
        out += _bitarray_bytes(het_mask) if f1 == 0 else _difflist_id_bytes(het[het_mask], n)
        out += _packed_bytes(het_alt[het_mask] - 2, _het_alt_width(ac))
    if f2 != 15:
        out += _bitarray_bytes(hom_mask) if f2 == 0 else _difflist_id_bytes(hom[hom_mask], n)
        sel = pairs[hom_mask]
        if ac == 2:
            out += _bitarray_bytes((sel[:, 0] == 2) & (sel[:, 1] == 2))
        else:
            if swap_pairs:                   # the reader sorts each pair
                sel = sel[:, ::-1]
            out += _packed_bytes((sel - 1).ravel(), _homalt_pair_width(ac))
    return bytes(out)


def encode_pgen_multiallelic(alleles: np.ndarray, alt_counts, het_fmt: int = 0,
                             hom_fmt: int = 0, patch: np.ndarray | None = None,
                             phase: str | None = None, dosage: np.ndarray | None = None,
                             dosage_kind: str = "list", seed: int = 0) -> bytes:
    """A .pgen of variants with ``alt_counts[v]`` ALT alleles from per-sample
    allele pairs [V][N][2] (0 REF, j = ALT j, -1 missing).  Every variant with
    two or more ALTs and ``patch[v]`` (default: all of them) carries a
    multiallelic patch (vrtype bit 3) after its main track; phase and dosage
    tracks follow as in ``encode_pgen_tracks``."""
    alleles = np.asarray(alleles, np.int64)
    V, n, _ = alleles.shape
    cats = multiallelic_categories(alleles)
    rng = np.random.default_rng(seed)
    types, recs = _pgen_records(cats)
    types, recs = list(types), list(recs)
    for v in range(V):
        body = recs[v]
        if int(alt_counts[v]) >= 2 and (patch is None or patch[v]):
            body = body + _multiallelic_patch(cats[v], alleles[v], int(alt_counts[v]), het_fmt,
                                              hom_fmt, bool(v % 2))
            types[v] |= 0b0000_1000
        if phase is not None:
            body = body + _phase_track(cats[v], rng, phase == "partial")
            types[v] |= 0b0001_0000
        if dosage is not None and np.any(dosage[v] != 65535):
            bits, track = _dosage_track(np.asarray(dosage[v], np.uint16), dosage_kind, False, rng)
            body = body + track
            types[v] |= bits
        recs[v] = body
    return _pgen_file(n, types, recs)


def multiallelic_alleles(seed: int, alt_counts, num_people: int, missing_rate: float = 0.02,
                         het_rate: float = 0.3, hom_rate: float = 0.15) -> np.ndarray:
    """Seeded allele pairs [V][N][2] for variants with ``alt_counts[v]`` ALTs:
    REF/REF, het REF/ALT j, ALT pairs (hom or two different ALTs) and missing."""
    rng = np.random.default_rng(seed)
    V = len(alt_counts)
    out = np.zeros((V, num_people, 2), np.int64)
    for v in range(V):
        ac = int(alt_counts[v])
        u = rng.random(num_people)
        alt = rng.integers(1, ac + 1, size=(num_people, 2))
        het = (u >= missing_rate) & (u < missing_rate + het_rate)
        hom = (u >= missing_rate + het_rate) & (u < missing_rate + het_rate + hom_rate)
        out[v, het, 1] = alt[het, 0]
        out[v, hom] = alt[hom]
        out[v, u < missing_rate] = -1
    return out


def encode_pgen(cats: np.ndarray, repeats: int = 1) -> bytes:
    """Genotype categories [V][N] (0 hom REF, 1 het, 2 hom ALT, 3 missing) ->
    a variable-width (mode 0x10) .pgen, 8-bit record types, 4-byte lengths.

    Each variant takes the smallest of these encodings: a 2-bit array (type 0);
    two categories as a bit array plus a difflist (type 1); all hom REF / hom
    ALT / missing plus a difflist (types 4 / 6 / 7); a difflist against the
    most recent non-LD record of its 2^16-variant block (type 2), or against
    that record with REF and ALT homozygotes swapped (type 3).

    ``repeats`` > 1 writes the V records that many times over (variant
    ``r * V + v`` holds the genotypes of variant ``v``); V must then divide
    2^16 so that no repeat straddles a block and every LD record keeps its
    anchor.  Large files are built that way in seconds.
    """
    cats = np.asarray(cats, np.uint8)
    V, n = cats.shape
    if repeats > 1 and (1 << 16) % V:
        raise ValueError("a repeated .pgen needs a variant count that divides 2^16")
    types, recs = _pgen_records(cats)
    return _pgen_file(n, types * repeats, recs * repeats)


def pgen_ld_categories(seed: int, num_variants: int, num_people: int, run: int = 17,
                       change: float = 0.02, swap_every: int = 5) -> np.ndarray:
    """Seeded categories with linkage: within runs of ``run`` variants each one
    copies its predecessor (REF/ALT homozygotes swapped every ``swap_every``-th
    variant) and redraws a ``change`` fraction of people, so the encoder picks
    LD-compressed records (types 2 and 3) as real cohorts do."""
    base = pgen_categories(seed, num_variants, num_people)
    rng = np.random.default_rng(seed ^ 0x5EED)
    c = base.copy()
    for v in range(1, num_variants):
        if v % run == 0:
            continue
        prev = c[v - 1]
        if v % swap_every == 0:
            prev = np.where(prev == 0, 2, np.where(prev == 2, 0, prev))
        redraw = rng.random(num_people) < change
        c[v] = np.where(redraw, base[v], prev)
    return c.astype(np.uint8)


def pgen_categories(seed: int, num_variants: int, num_people: int, p_lo: float = 0.01,
                    p_hi: float = 0.5, missing_rate: float = 0.01) -> np.ndarray:
    """Seeded HWE genotype categories [V][N] for synthetic .pgen files (the same
    generator as synth_rows, read back as PGEN categories)."""
    thr = variant_thresholds(seed, 0, num_variants, p_lo, p_hi, missing_rate)
    codes = genotype_codes(seed, 0, num_variants, num_people, thr)
    return BED_TO_PGEN_CAT[codes]
