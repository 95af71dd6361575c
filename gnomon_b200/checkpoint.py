"""Score checkpoints in gnomon's on-disk format (score/checkpoint.rs).

A checkpoint holds the running per-person state after a prefix of the
reconciled variants, so an interrupted run resumes instead of starting over:

    MAGIC "GNOMON_SCORE_CHECKPOINT_V1\\n"          (checkpoint.rs:8)
    fingerprint   32 bytes, SHA-256 of the prepared inputs (checkpoint.rs:83-121)
    completed_variants  u64 LE
    result_len          u64 LE  (= P*K)
    sum_scores    result_len x f64 LE   (final sums so far, baseline included)
    missing_counts result_len x u32 LE

Writes go to a unique temporary file in the same directory, are fsynced and
renamed over the target (checkpoint.rs:283-321), so a crash leaves either the
old or the new checkpoint.  ``ScoreCheckpointWriter`` saves at most every 30
seconds and always when the last variant completes (checkpoint.rs:37-65).
The GPU pipeline calls it after every variant block (``pipeline.run`` with a
checkpoint path), the way the reference's CUDA engine does after every
mega-batch (cuda_backend.rs:1638-1648, 1969-2011).
"""
from __future__ import annotations

import hashlib
import os
import struct
import time
from dataclasses import dataclass
from pathlib import Path
from typing import Optional, Sequence, Union

import numpy as np

MAGIC = b"GNOMON_SCORE_CHECKPOINT_V1\n"
CHECKPOINT_INTERVAL_S = 30.0


class CheckpointError(OSError):
    """io::Error of kind InvalidData / InvalidInput from the reference loader."""


@dataclass
class ScoreCheckpoint:
    """Resume state (checkpoint.rs:11-16)."""

    completed_variants: int
    sum_scores: np.ndarray      # f64 [P*K]
    missing_counts: np.ndarray  # u32 [P*K]


# ---- fingerprint (checkpoint.rs:83-235) ---------------------------------------

@dataclass
class FilesetBoundary:
    """One fileset of a multi-file run (types.rs FilesetBoundary)."""

    bed_path: Path
    bim_path: Path
    fam_path: Path
    starting_global_index: int


PipelineIdentity = Union[None, str, os.PathLike, Sequence[FilesetBoundary]]


def _u64(h, v: int) -> None:
    h.update(struct.pack("<Q", v & 0xFFFFFFFFFFFFFFFF))


def _bytes(h, b: bytes) -> None:
    _u64(h, len(b))
    h.update(b)


def _system_time(h, t_ns: int) -> None:
    if t_ns < 0:
        h.update(b"\x00")
        return
    h.update(b"\x01")
    _u64(h, t_ns // 1_000_000_000)
    h.update(struct.pack("<I", t_ns % 1_000_000_000))


def _path_identity(h, path, include_bed_header: bool) -> None:
    text = os.fspath(path)            # hashed as given, not normalised
    path = Path(text)
    _bytes(h, text.encode())
    try:
        st = path.stat()
        h.update(b"\x01")
        _u64(h, st.st_size)
        _system_time(h, st.st_mtime_ns)
    except OSError:
        h.update(b"\x00")
    if include_bed_header:
        try:
            with open(path, "rb") as f:
                head = f.read(3)
            if len(head) != 3:
                raise OSError("short header")
            h.update(b"\x01")
            h.update(head)
        except OSError:
            h.update(b"\x00")


_FILESET_EXTS = ("bed", "bim", "fam", "pgen", "pvar", "psam")


def _strip_fileset_extension(s: str) -> str:
    """The shared prefix of a fileset path (prepare.rs:1110-1118)."""
    base, dot, ext = s.rpartition(".")
    if dot and ext in _FILESET_EXTS and not base.endswith("/"):
        return base
    return s


def _is_pgen(path: str) -> bool:
    return Path(path).suffix == ".pgen"


def _pipeline_identity(h, identity: PipelineIdentity) -> None:
    if identity is None:
        return
    if isinstance(identity, (str, os.PathLike)):
        bed = str(identity)
        h.update(b"\x00")
        _path_identity(h, bed, True)
        meta = ("pvar", "psam") if _is_pgen(bed) else ("bim", "fam")
        stem = _strip_fileset_extension(bed)
        for ext in meta:
            _path_identity(h, f"{stem}.{ext}", False)
        return
    boundaries = list(identity)
    h.update(b"\x01")
    _u64(h, len(boundaries))
    for b in boundaries:
        _path_identity(h, b.bed_path, True)
        _path_identity(h, b.bim_path, False)
        _path_identity(h, b.fam_path, False)
        _u64(h, b.starting_global_index)


def fingerprint_preparation(prep, pipeline: PipelineIdentity = None,
                            total_variants_in_bim: Optional[int] = None,
                            required_is_complex: Optional[np.ndarray] = None) -> bytes:
    """SHA-256 over the prepared inputs in checkpoint.rs:83-121 order.

    Fields the engine does not otherwise need are taken from the arguments or
    from the PreparationResult's optional attributes: the .bim variant count
    (default: the reconciled count), the per-variant complex flags (default:
    none complex) and the fileset identity (a .bed/.pgen path or a list of
    FilesetBoundary; omitted when None)."""
    h = hashlib.sha256()
    V = prep.num_reconciled_variants
    tvb = total_variants_in_bim
    if tvb is None:
        tvb = getattr(prep, "total_variants_in_bim", None)
    if tvb is None:
        tvb = V
    cplx = required_is_complex
    if cplx is None:
        cplx = getattr(prep, "required_is_complex", None)
    if cplx is None:
        cplx = np.zeros(V, dtype=np.uint8)
    _u64(h, prep.num_people_to_score)
    _u64(h, prep.total_people_in_fam)
    _u64(h, tvb)
    _u64(h, V)
    _u64(h, prep.bytes_per_variant)
    _u64(h, len(prep.score_names))
    for name in prep.score_names:
        _bytes(h, str(name).encode())
    for iid in (prep.final_person_iids or []):
        _bytes(h, str(iid).encode())
    h.update(np.asarray(prep.score_variant_counts, "<u4").tobytes())
    h.update(np.asarray(prep.baseline, "<f8").tobytes())
    rbi = prep.required_bim_indices
    h.update((np.arange(V, dtype="<u8") if rbi is None else np.asarray(rbi, "<u8")).tobytes())
    h.update(np.asarray(cplx, dtype=np.uint8).tobytes())
    h.update(np.asarray(prep.sparse_row_offsets, "<u8").tobytes())
    h.update(np.asarray(prep.sparse_score_columns, "<u4").tobytes())
    h.update(np.asarray(prep.sparse_weights, "<f4").tobytes())
    h.update(np.asarray(prep.sparse_missing_corrections, "<f4").tobytes())
    _pipeline_identity(h, pipeline if pipeline is not None else getattr(prep, "pipeline_kind", None))
    return h.digest()


# ---- file format ------------------------------------------------------------

def checkpoint_path_for_output(output_path) -> Path:
    """`<dir>/<output name>.gnomon-checkpoint.bin` (checkpoint.rs:70-81)."""
    p = Path(output_path)
    name = f"{p.name}.gnomon-checkpoint.bin" if p.name else \
        "gnomon_results.sscore.gnomon-checkpoint.bin"
    parent = p.parent if str(p.parent) not in ("", ".") or p.is_absolute() else Path(".")
    return parent / name


def _unique_temp_path(directory: Path, name: str) -> Path:
    return directory / f".{name}.{os.getpid()}.{time.time_ns()}.tmp"


def write_checkpoint(path, fingerprint: bytes, completed_variants: int, sum_scores,
                     missing_counts) -> None:
    s = np.ascontiguousarray(sum_scores, dtype="<f8").reshape(-1)
    c = np.ascontiguousarray(missing_counts, dtype="<u4").reshape(-1)
    if s.size != c.size:
        raise CheckpointError("Checkpoint score/count length mismatch.")
    if len(fingerprint) != 32:
        raise CheckpointError("A checkpoint fingerprint is 32 bytes.")
    path = Path(path)
    if not path.name:
        raise CheckpointError(f"Checkpoint path '{path}' has no file name.")
    directory = path.parent
    directory.mkdir(parents=True, exist_ok=True)
    tmp = _unique_temp_path(directory, path.name)
    fd = os.open(tmp, os.O_WRONLY | os.O_CREAT | os.O_EXCL, 0o644)
    try:
        with os.fdopen(fd, "wb") as f:
            f.write(MAGIC)
            f.write(fingerprint)
            f.write(struct.pack("<QQ", completed_variants, s.size))
            f.write(s.tobytes())
            f.write(c.tobytes())
            f.flush()
            os.fsync(f.fileno())
        os.replace(tmp, path)
    except BaseException:
        try:
            os.unlink(tmp)
        except OSError:
            pass
        raise


def load_checkpoint(path, expected_fingerprint: bytes, expected_result_len: int,
                    total_variants: int) -> Optional[ScoreCheckpoint]:
    """None when the file does not exist; CheckpointError when it does not
    belong to this run (checkpoint.rs:237-300)."""
    path = Path(path)
    try:
        f = open(path, "rb")
    except FileNotFoundError:
        return None
    with f:
        def read(n):
            b = f.read(n)
            if len(b) != n:
                raise CheckpointError(f"Checkpoint '{path}' is truncated.")
            return b
        if read(len(MAGIC)) != MAGIC:
            raise CheckpointError(f"Checkpoint '{path}' has an invalid header.")
        if read(32) != expected_fingerprint:
            raise CheckpointError(
                f"Checkpoint '{path}' does not match the prepared scoring inputs.")
        completed, result_len = struct.unpack("<QQ", read(16))
        if result_len != expected_result_len:
            raise CheckpointError(
                f"Checkpoint '{path}' result length {result_len} does not match current "
                f"result length {expected_result_len}.")
        if completed > total_variants:
            raise CheckpointError(
                f"Checkpoint '{path}' completed {completed} variants but this run has only "
                f"{total_variants}.")
        sums = np.frombuffer(read(8 * result_len), dtype="<f8").astype(np.float64)
        counts = np.frombuffer(read(4 * result_len), dtype="<u4").astype(np.uint32)
    return ScoreCheckpoint(int(completed), sums, counts)


def remove_checkpoint(path) -> None:
    try:
        os.unlink(path)
    except FileNotFoundError:
        pass


class ScoreCheckpointWriter:
    """Rate-limited checkpoint saving (checkpoint.rs:18-65)."""

    def __init__(self, path, fingerprint: bytes, total_variants: int,
                 interval_s: float = CHECKPOINT_INTERVAL_S):
        self.path = Path(path)
        self.fingerprint = fingerprint
        self.total_variants = total_variants
        self.interval_s = interval_s
        self.last_save_at: Optional[float] = None
        self.last_completed_variants = 0

    def maybe_save(self, completed_variants: int, sum_scores, missing_counts,
                   force: bool = False) -> bool:
        if completed_variants <= self.last_completed_variants:
            return False
        due = (force or completed_variants >= self.total_variants or self.last_save_at is None
               or time.monotonic() - self.last_save_at >= self.interval_s)
        if not due:
            return False
        write_checkpoint(self.path, self.fingerprint, completed_variants, sum_scores,
                         missing_counts)
        self.last_save_at = time.monotonic()
        self.last_completed_variants = completed_variants
        return True
