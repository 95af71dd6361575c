"""Host entry points mirroring gnomon's ``score::pipeline`` API.

``run(context, bed)`` is the counterpart of ``pipeline::run``
(score/pipeline.rs:468) for the GPU slot: it calls ``gnm_score_run`` (the
drop-in for ``cuda_backend::try_run_cuda``, score/cuda_backend.rs:604) and
returns gnomon's per-person result, row-major ``[P][K]`` float64 final sums
(baseline included) and uint32 missing counts.

There is no CPU fallback in this package: when the library declines (no CUDA
device) ``try_run_cuda`` returns ``None`` exactly like the reference, and
``run`` raises, leaving the CPU pipeline to the caller.
"""
from __future__ import annotations

import ctypes as C
import mmap
import os
from dataclasses import dataclass
from pathlib import Path
from typing import Callable, Optional, Union

import numpy as np

from . import _lib
from .checkpoint import ScoreCheckpoint, ScoreCheckpointWriter
from .prepare import PreparationResult

PLINK_MAGIC = bytes([0x6C, 0x1B, 0x01])


@dataclass
class PipelineContext:
    """pipeline.rs:408-446: the prepared inputs, an optional checkpoint to
    resume from, and where / under which fingerprint to write checkpoints
    while scoring (``with_checkpoint``)."""

    prep_result: PreparationResult
    checkpoint: Optional[ScoreCheckpoint] = None
    checkpoint_path: Optional[Path] = None
    checkpoint_fingerprint: Optional[bytes] = None

    @classmethod
    def with_checkpoint(cls, prep_result: PreparationResult,
                        checkpoint: Optional[ScoreCheckpoint], checkpoint_path,
                        checkpoint_fingerprint: bytes) -> "PipelineContext":
        return cls(prep_result, checkpoint, Path(checkpoint_path), checkpoint_fingerprint)

    def checkpoint_completed_variants(self) -> int:
        return self.checkpoint.completed_variants if self.checkpoint is not None else 0


class PipelineError(RuntimeError):
    """PipelineError::{Compute, Io, Producer} (shared/pipeline_error.rs:5-9)."""

    def __init__(self, kind: str, message: str, status: int):
        super().__init__(f"{kind}: {message}")
        self.kind = kind
        self.status = status


_KIND = {_lib.GNM_ERR_IO: "Io", _lib.GNM_ERR_PRODUCER: "Producer"}


def _ptr(a: Optional[np.ndarray]) -> Optional[int]:
    return None if a is None else a.ctypes.data


def prep_view(prep: PreparationResult) -> _lib.gnm_prep_view:
    """Build the C view.  The arrays stay owned by ``prep``."""
    v = _lib.gnm_prep_view()
    v.num_people = prep.num_people_to_score
    v.total_people_in_fam = prep.total_people_in_fam
    v.bytes_per_variant = prep.bytes_per_variant
    v.num_scores = prep.num_scores
    v.num_variants = prep.num_reconciled_variants
    v.sparse_weights = _ptr(prep.sparse_weights)
    v.sparse_missing_corrections = _ptr(prep.sparse_missing_corrections)
    v.sparse_score_columns = _ptr(prep.sparse_score_columns)
    v.sparse_row_offsets = _ptr(prep.sparse_row_offsets)
    v.required_bim_indices = _ptr(prep.required_bim_indices)
    v.output_idx_to_fam_idx = _ptr(prep.output_idx_to_fam_idx)
    base = np.ascontiguousarray(prep.baseline, dtype=np.float64)
    v.baseline = base.ctypes.data
    v._keep = base  # the view must not outlive the baseline array
    return v


class BedSource:
    """Packed rows after the 3-byte magic (shared/files.rs:200-292, :373)."""

    def __init__(self, data: Union[str, os.PathLike, bytes, np.ndarray]):
        self._mm = None
        if isinstance(data, (str, os.PathLike)):
            f = open(data, "rb")
            try:
                self._mm = mmap.mmap(f.fileno(), 0, access=mmap.ACCESS_READ)
            finally:
                f.close()
            buf = np.frombuffer(self._mm, dtype=np.uint8)
            validate_plink_bed_header(buf[:3].tobytes())
            self.rows = buf[3:]
        elif isinstance(data, (bytes, bytearray)):
            buf = np.frombuffer(data, dtype=np.uint8)
            self.rows = buf
        else:
            self.rows = np.ascontiguousarray(data, dtype=np.uint8).reshape(-1)

    def view(self) -> _lib.gnm_bed_view:
        v = _lib.gnm_bed_view()
        v.data = self.rows.ctypes.data if self.rows.size else None
        v.data_len = self.rows.size
        return v

    def genotype_source(self, bytes_per_variant: int):
        from .complex import GenotypeSource
        return GenotypeSource.single(self.rows, bytes_per_variant)


class ByteRangeSource:
    """Row bytes behind a read callback, for sources that are not a local
    file: ``ByteRangeSource::read_at`` (shared/files.rs:187-245) reads
    ``length`` bytes at an offset of the row data (the bytes after the 3-byte
    magic).

    ``read_at(offset, length)`` returns exactly ``length`` bytes; a shorter
    result or an exception makes the engine stop with
    ``PipelineError("Producer")`` (GNM_ERR_PRODUCER), as a failing reader does
    in the reference's producer thread.  The engine may call it from several
    host threads at once."""

    def __init__(self, read_at: Callable[[int, int], bytes]):
        self._read_at = read_at
        self.errors: list = []

        def _cb(_ctx, offset, dst, length):
            try:
                b = read_at(int(offset), int(length))
                if b is None or len(b) != length:
                    return 1
                C.memmove(dst, bytes(b), int(length))
                return 0
            except Exception as e:  # noqa: BLE001 - reported as a producer failure
                self.errors.append(e)
                return 1
        self._cfn = _lib.READ_AT(_cb)   # kept alive as long as the source

    def view(self) -> _lib.gnm_bed_view:
        v = _lib.gnm_bed_view()
        v.data = None
        v.data_len = 0
        v.read_at = self._cfn
        v.user_ctx = None
        return v

    def genotype_source(self, bytes_per_variant: int):
        from .complex import GenotypeSource

        src = self

        class _Rows(GenotypeSource):
            def __init__(self):
                super().__init__([np.zeros(0, np.uint8)], [0], bytes_per_variant)

            def codes(self, bim_row, fam):
                row = np.frombuffer(src._read_at(int(bim_row) * self.bpv, self.bpv), np.uint8)
                if row.size != self.bpv:
                    raise IOError(f"Genotype bytes of .bim row {bim_row} could not be read")
                fam = np.asarray(fam)
                return ((row[(fam // 4).astype(np.int64)] >> (2 * (fam % 4)).astype(np.uint8))
                        & 3).astype(np.uint8)
        return _Rows()


def validate_plink_bed_header(head: bytes) -> None:
    if len(head) < 3 or head[:3] != PLINK_MAGIC:
        raise PipelineError("Io", "not a SNP-major PLINK .bed file (bad magic bytes)",
                            _lib.GNM_ERR_IO)


def try_run_cuda(context: PipelineContext, bed, engine: int = _lib.ENGINE_AUTO,
                 device: int = -1, block_variants: int = 0,
                 on_block: Optional[Callable[[int, np.ndarray, np.ndarray], bool]] = None):
    """``Some((sums, counts))`` -> tuple; ``Ok(None)`` (declined) -> ``None``; errors raise."""
    lib = _lib.load()
    prep = context.prep_result
    src = bed if isinstance(bed, (BedSource, ByteRangeSource)) else BedSource(bed)
    P, K = prep.num_people_to_score, prep.num_scores
    sums = np.empty(P * K, dtype=np.float64)
    counts = np.empty(P * K, dtype=np.uint32)
    pv = prep_view(prep)
    bv = src.view()
    resume = None
    if context.checkpoint is not None:
        cp = context.checkpoint
        rs = np.ascontiguousarray(cp.sum_scores, dtype=np.float64)
        rc = np.ascontiguousarray(cp.missing_counts, dtype=np.uint32)
        if rs.size != P * K or rc.size != P * K:
            raise PipelineError("Compute", "checkpoint accumulator shape mismatch",
                                _lib.GNM_ERR_INVALID)
        resume = _lib.gnm_resume(cp.completed_variants, rs.ctypes.data, rc.ctypes.data)
    opts = _lib.gnm_run_options()
    opts.engine = engine
    opts.device = device
    opts.block_variants = block_variants
    # checkpoints after each variant block, forced when the last one completes
    # (cuda_backend.rs:1638-1648, 1969-2011, 2335-2352)
    writer = None
    if context.checkpoint_path is not None and context.checkpoint_fingerprint is not None:
        writer = ScoreCheckpointWriter(context.checkpoint_path, context.checkpoint_fingerprint,
                                       prep.num_reconciled_variants)
    cb_errors = []
    if on_block is not None or writer is not None:
        V = prep.num_reconciled_variants

        def _cb(_ctx, done, s_ptr, c_ptr):
            s = np.ctypeslib.as_array(C.cast(s_ptr, C.POINTER(C.c_double)), shape=(P * K,))
            c = np.ctypeslib.as_array(C.cast(c_ptr, C.POINTER(C.c_uint32)), shape=(P * K,))
            try:
                if writer is not None:
                    writer.maybe_save(int(done), s, c, force=int(done) >= V)
                if on_block is not None and on_block(int(done), s, c) is False:
                    return 1
                return 0
            except Exception as e:  # noqa: BLE001 - reported after the call returns
                cb_errors.append(e)
                return 1
        opts.on_block = _lib.BLOCK_CB(_cb)
    err = _lib.gnm_error()
    st = lib.gnm_score_run_ex(C.byref(pv), C.byref(bv), C.byref(resume) if resume else None,
                              C.byref(opts), sums.ctypes.data, counts.ctypes.data, C.byref(err))
    if st == _lib.GNM_DECLINED:
        return None
    if cb_errors and isinstance(cb_errors[0], OSError):
        raise PipelineError("Io", f"Failed to write score checkpoint: {cb_errors[0]}",
                            _lib.GNM_ERR_IO) from cb_errors[0]
    if st != _lib.GNM_OK:
        msg = err.message.decode(errors="replace")
        if isinstance(src, ByteRangeSource) and src.errors:
            msg += f" ({src.errors[0]!r})"
        raise PipelineError(_KIND.get(st, "Compute"), msg, st)
    if prep.complex_rules:
        # multi-row loci, on the CPU after the engine (cuda_backend.rs:1465-1535)
        from .complex import ComplexResolutionError, resolve_complex_variants
        try:
            resolve_complex_variants(prep.complex_rules,
                                     src.genotype_source(prep.bytes_per_variant),
                                     prep.output_idx_to_fam_idx, P, prep.score_names, sums,
                                     counts, prep.final_person_iids)
        except ComplexResolutionError as e:
            raise PipelineError(e.kind, str(e), _lib.GNM_ERR_IO if e.kind == "Io"
                                else _lib.GNM_ERR_COMPUTE) from e
    return sums, counts


def run(context: PipelineContext, bed, **kw):
    """pipeline::run for the GPU slot.  Raises when no CUDA device is usable."""
    out = try_run_cuda(context, bed, **kw)
    if out is None:
        raise PipelineError("Compute", "CUDA backend declined (no usable device); this package "
                            "has no CPU pipeline", _lib.GNM_DECLINED)
    return out
