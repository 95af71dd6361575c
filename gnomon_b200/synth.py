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
