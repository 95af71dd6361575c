"""PLINK 2 ``.pgen`` hard calls decoded on the GPU into ``.bed`` rows.

gnomon scores a ``.pgen`` fileset by presenting it to the scoring engine as a
virtual ``.bed`` (shared/adapt_plink2.rs:1093-1158): each variant's hard
calls are decoded (:2108-2666) and packed as the ``.bed`` codes of the
A1 = ALT dosage.  Here that decode runs on the device
(``gnm_pgen_decode_device``), writing rows straight into HBM where
``DevicePlan`` reads them; the file's bytes cross PCIe once, compressed.

Supported: storage modes 0x02 and 0x10 / 0x11 (main-track types 0-4, 6, 7;
phase tracks are skipped; a dosage track fills missing hard calls with the
nearest allele count within 0.10, as the reference's virtual .bed does,
samples taken as diploid).  Given each variant's ALT count (the ``.pvar``'s
ALT column), multiallelic records decode one row per (variant, ALT): the
copies of that ALT, as the reference splits them (:2704-2881).  Without ALT
counts they are rejected with ``GNM_ERR_INVALID``; truncated or malformed
files give ``GNM_ERR_IO``.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Tuple, Union

import numpy as np
import torch

from . import _lib
from .device import _stream_ptr, row_pitch
from .prepare import PreparationResult

PgenSource = Union[str, os.PathLike, bytes, bytearray, np.ndarray]


def _bytes(data: PgenSource) -> np.ndarray:
    if isinstance(data, (str, os.PathLike)):
        return np.fromfile(data, dtype=np.uint8)
    if isinstance(data, (bytes, bytearray)):
        return np.frombuffer(bytes(data), dtype=np.uint8)
    return np.ascontiguousarray(data, dtype=np.uint8).reshape(-1)


def pgen_dims(data: PgenSource) -> Tuple[int, int]:
    """(variants, samples) from a ``.pgen`` header."""
    buf = _bytes(data)
    lib = _lib.load()
    m, n = C.c_uint64(), C.c_uint64()
    e = _lib.gnm_error()
    _lib.check(lib.gnm_pgen_dims(buf.ctypes.data, buf.nbytes, C.byref(m), C.byref(n),
                                 C.byref(e)), e)
    return int(m.value), int(n.value)


def decode_to_device(data: PgenSource, device: Optional[int] = None,
                     rows: Optional[torch.Tensor] = None, pitch: Optional[int] = None,
                     stream: Optional[torch.cuda.Stream] = None) -> Tuple[torch.Tensor, int]:
    """Decode every variant into device ``.bed`` rows; returns (rows, pitch).

    ``rows`` (uint8, 16-byte aligned, at least variants x pitch bytes) may be
    supplied; otherwise it is allocated with a 128-byte pitch.  Row ``v`` holds
    ``.pgen`` variant ``v``; bytes past ``ceil(samples / 4)`` are left as
    they were.  Returns after the decode has finished on ``stream``."""
    buf = _bytes(data)
    m, n = pgen_dims(buf)
    bpv = (n + 3) // 4
    dev = torch.cuda.current_device() if device is None else device
    if pitch is None:
        pitch = row_pitch(bpv)
    if rows is None:
        rows = torch.zeros(max(m, 1) * pitch, dtype=torch.uint8, device=torch.device("cuda", dev))
    if not (rows.is_cuda and rows.dtype == torch.uint8 and rows.numel() >= m * pitch):
        raise ValueError("rows must be a CUDA uint8 tensor of at least variants x pitch bytes")
    lib = _lib.load()
    e = _lib.gnm_error()
    _lib.check(lib.gnm_pgen_decode_device(buf.ctypes.data, buf.nbytes, dev, rows.data_ptr(),
                                          pitch, _stream_ptr(stream), C.byref(e)), e)
    return rows, pitch


class PgenFile:
    """A ``.pgen`` resident on one device (``gnm_pgen_open``): decode any
    variant range on demand, asynchronously, e.g. block by block into a
    streaming buffer.  Use from one stream at a time.  ``alt_counts`` (one
    per variant) enables multiallelic records (``gnm_pgen_open_alleles``)."""

    def __init__(self, data: PgenSource, device: Optional[int] = None, alt_counts=None):
        self.lib = _lib.load()
        buf = _bytes(data)
        self.variants, self.samples = pgen_dims(buf)
        self.bytes_per_variant = (self.samples + 3) // 4
        self.device = torch.cuda.current_device() if device is None else device
        handle = C.c_void_p()
        e = _lib.gnm_error()
        if alt_counts is None:
            _lib.check(self.lib.gnm_pgen_open(buf.ctypes.data, buf.nbytes, self.device,
                                              C.byref(handle), C.byref(e)), e)
        else:
            ac = np.ascontiguousarray(alt_counts, dtype=np.uint32).reshape(-1)
            if len(ac) != self.variants:
                raise ValueError("one ALT count per variant")
            _lib.check(self.lib.gnm_pgen_open_alleles(buf.ctypes.data, buf.nbytes, ac.ctypes.data,
                                                      self.device, C.byref(handle), C.byref(e)), e)
        self.handle = handle

    def close(self):
        if getattr(self, "handle", None):
            self.lib.gnm_pgen_close(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def device_bytes(self) -> int:
        return int(self.lib.gnm_pgen_device_bytes(self.handle))

    def decode(self, rows: torch.Tensor, pitch: int, variant_begin: int = 0,
               variant_count: Optional[int] = None, stream=None):
        """Enqueue the decode of a variant range into ``rows`` (row 0 = ``variant_begin``)."""
        n = self.variants - variant_begin if variant_count is None else variant_count
        if not (rows.is_cuda and rows.dtype == torch.uint8 and rows.numel() >= n * pitch):
            raise ValueError("rows must be a CUDA uint8 tensor of at least count x pitch bytes")
        e = _lib.gnm_error()
        _lib.check(self.lib.gnm_pgen_decode(self.handle, variant_begin, n, rows.data_ptr(), pitch,
                                            _stream_ptr(stream), C.byref(e)), e)

    def decode_list(self, rows: torch.Tensor, pitch: int, variants, stream=None):
        """Enqueue the decode of the listed variants (any order) into consecutive rows."""
        lst = np.ascontiguousarray(variants, dtype=np.uint64).reshape(-1)
        if not (rows.is_cuda and rows.dtype == torch.uint8 and rows.numel() >= len(lst) * pitch):
            raise ValueError("rows must be a CUDA uint8 tensor of at least count x pitch bytes")
        e = _lib.gnm_error()
        _lib.check(self.lib.gnm_pgen_decode_list(self.handle, lst.ctypes.data, len(lst),
                                                 rows.data_ptr(), pitch, _stream_ptr(stream),
                                                 C.byref(e)), e)

    def decode_alleles(self, rows: torch.Tensor, pitch: int, variants, alt_ords, stream=None):
        """Enqueue the decode of (variant, ALT) pairs: row i = the copies of ALT
        ``alt_ords[i]`` (1-based) of variant ``variants[i]``."""
        lst = np.ascontiguousarray(variants, dtype=np.uint64).reshape(-1)
        ords = np.ascontiguousarray(alt_ords, dtype=np.uint32).reshape(-1)
        if len(ords) != len(lst):
            raise ValueError("one ALT ordinal per listed variant")
        if not (rows.is_cuda and rows.dtype == torch.uint8 and rows.numel() >= len(lst) * pitch):
            raise ValueError("rows must be a CUDA uint8 tensor of at least count x pitch bytes")
        e = _lib.gnm_error()
        _lib.check(self.lib.gnm_pgen_decode_alleles(self.handle, lst.ctypes.data, ords.ctypes.data,
                                                    len(lst), rows.data_ptr(), pitch,
                                                    _stream_ptr(stream), C.byref(e)), e)

    def check(self, stream=None):
        """Wait for ``stream``; raise if any record decoded so far was malformed."""
        e = _lib.gnm_error()
        _lib.check(self.lib.gnm_pgen_check(self.handle, _stream_ptr(stream), C.byref(e)), e)


def score_pgen(prep: PreparationResult, data: PgenSource, engine: int = _lib.ENGINE_AUTO,
               device: Optional[int] = None, block_variants: int = 0, alt_counts=None,
               bim_variant=None, bim_alt=None) -> Tuple[np.ndarray, np.ndarray]:
    """Score a ``.pgen`` whose variants are the ``.bim``-order rows ``prep`` indexes
    (``gnm_score_pgen``): the reconciled variants (``required_bim_indices``)
    are decoded on the device block by block and scored as they land.
    Returns host (sums f64, missing counts u32), person-major like
    ``gnm_score_run``.  Multi-row loci (``prep.complex_rules``) are resolved on
    the CPU afterwards from the decoded rows, as ``try_run_cuda`` does for a
    ``.bed``.  With ``alt_counts`` the ``.bim`` is virtual
    (``gnm_score_pgen_alleles``): row r holds ALT ``bim_alt[r]`` of variant
    ``bim_variant[r]``."""
    from .pipeline import prep_view
    buf = _bytes(data)
    lib = _lib.load()
    P, K = prep.num_people_to_score, prep.num_scores
    sums = np.empty(P * K, dtype=np.float64)
    counts = np.empty(P * K, dtype=np.uint32)
    pv = prep_view(prep)
    opts = _lib.gnm_run_options()
    opts.engine = engine
    opts.device = -1 if device is None else device
    opts.block_variants = block_variants
    e = _lib.gnm_error()
    if alt_counts is None:
        _lib.check(lib.gnm_score_pgen(C.byref(pv), buf.ctypes.data, buf.nbytes, C.byref(opts),
                                      sums.ctypes.data, counts.ctypes.data, C.byref(e)), e)
    else:
        ac = np.ascontiguousarray(alt_counts, dtype=np.uint32).reshape(-1)
        bv = np.ascontiguousarray(bim_variant, dtype=np.uint64).reshape(-1)
        ba = np.ascontiguousarray(bim_alt, dtype=np.uint32).reshape(-1)
        if len(bv) != len(ba):
            raise ValueError("bim_variant and bim_alt differ in length")
        _lib.check(lib.gnm_score_pgen_alleles(C.byref(pv), buf.ctypes.data, buf.nbytes,
                                              ac.ctypes.data, bv.ctypes.data, ba.ctypes.data,
                                              len(bv), C.byref(opts), sums.ctypes.data,
                                              counts.ctypes.data, C.byref(e)), e)
    if prep.complex_rules:
        from .complex import GenotypeSource, resolve_complex_variants
        m, n = pgen_dims(buf)
        bpv = (n + 3) // 4
        if alt_counts is None:
            rows, pitch = decode_to_device(buf, device=device)
        else:                               # every row of the virtual .bim
            m, pitch = len(bv), row_pitch(bpv)
            dev = torch.cuda.current_device() if device is None else device
            rows = torch.zeros(max(m, 1) * pitch, dtype=torch.uint8,
                               device=torch.device("cuda", dev))
            with PgenFile(buf, device=dev, alt_counts=ac) as pg:
                pg.decode_alleles(rows, pitch, bv, ba)
                pg.check()
        host = rows[:m * pitch].view(m, pitch)[:, :bpv].cpu().numpy().reshape(-1)
        resolve_complex_variants(prep.complex_rules, GenotypeSource.single(host, bpv),
                                 prep.output_idx_to_fam_idx, P, prep.score_names, sums,
                                 counts, prep.final_person_iids)
    return sums, counts
