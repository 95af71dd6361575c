"""The byte-level genotype expansions of the 8-bit tcgen05 kernels
(gnomon_b200/csrc/gnm_tensor.cu), restated with the hardware's byte-permute
rule and checked on the CPU against a direct decode of the .bed codes.

* gnm_t8_backward: one packed word (16 people of one variant) becomes 16
  operand bytes in person order, through code_fields, four shifts and a
  4 x 4 byte transpose of byte permutes;
* gnm_t8_accumulate / gnm_t8_pairs / gnm_t8_narrow: bytes of 16 variant rows
  (one byte column: 4 people) become, per person, 16 operand bytes in
  variant order.
"""
import numpy as np

M32 = 0xFFFFFFFF


def byte_perm(x, y, s):
    """__byte_perm(x, y, s): byte i of the result is byte (s >> 4i) & 7 of
    the eight bytes y:x (x = bytes 0-3)."""
    pool = [(x >> (8 * i)) & 0xFF for i in range(4)] + [(y >> (8 * i)) & 0xFF for i in range(4)]
    return sum(pool[(s >> (4 * i)) & 7] << (8 * i) for i in range(4))


def code_fields(x, missing):
    hi = (x >> 1) & 0x55555555
    lo = x & 0x55555555
    if missing:
        return lo & ~hi & M32
    return ((hi & ~lo) | ((hi & lo) << 1)) & M32


def direct(code, missing):
    """.bed code -> allele-2 dosage (00 -> 0, 01 missing -> 0, 10 -> 1, 11 -> 2)
    or the missing indicator."""
    if missing:
        return 1 if code == 1 else 0
    return {0: 0, 1: 0, 2: 1, 3: 2}[code]


def backward_word(x):
    d = code_fields(x, False)
    s0, s1 = d & 0x03030303, (d >> 2) & 0x03030303
    s2, s3 = (d >> 4) & 0x03030303, (d >> 6) & 0x03030303
    lo01, hi01 = byte_perm(s0, s1, 0x5140), byte_perm(s0, s1, 0x7362)
    lo23, hi23 = byte_perm(s2, s3, 0x5140), byte_perm(s2, s3, 0x7362)
    words = [byte_perm(lo01, lo23, 0x5410), byte_perm(lo01, lo23, 0x7632),
             byte_perm(hi01, hi23, 0x5410), byte_perm(hi01, hi23, 0x7632)]
    return [(w >> (8 * i)) & 0xFF for w in words for i in range(4)]


def test_backward_word_expansion_is_person_order():
    rng = np.random.default_rng(11)
    for x in list(rng.integers(0, 2**32, 2000, dtype=np.uint64)) + [0, M32, 0x55555555, 0xAAAAAAAA]:
        x = int(x)
        got = backward_word(x)
        want = [direct((x >> (2 * p)) & 3, False) for p in range(16)]
        assert got == want


def test_forward_chunk_expansion_is_variant_order():
    """16 rows' bytes of one byte column -> per person q, 16 bytes in row order."""
    rng = np.random.default_rng(12)
    for missing in (False, True):
        for _ in range(500):
            rows = [int(b) for b in rng.integers(0, 256, 16)]
            x = [0, 0, 0, 0]
            for i, b in enumerate(rows):
                x[i >> 2] |= b << (8 * (i & 3))
            x = [code_fields(w, missing) for w in x]
            for q in range(4):
                v = [(w >> (2 * q)) & 0x03030303 for w in x]
                got = [(v[i >> 2] >> (8 * (i & 3))) & 0xFF for i in range(16)]
                want = [direct((rows[i] >> (2 * q)) & 3, missing) for i in range(16)]
                assert got == want
