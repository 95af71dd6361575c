"""Per-person output semantics of gnomon's ``.sscore`` writer.

``write_scores_to_file`` (score/main.rs:1389-1548): for each person and score
``AVG = sum / (count_k - missing)`` in float64 (0 when no variant was used) and
``MISSING_PCT = missing / count_k * 100`` in float32 (0 when the score has no
variants); header ``#IID`` then ``<name>_AVG`` / ``<name>_MISSING_PCT`` pairs,
tab separated.  Values are printed with the shortest round-trip decimal
representation (the reference uses ryu); ``#REGION`` metadata lines precede
the header when score regions are given.
"""
from __future__ import annotations

import os
import time
from pathlib import Path
from typing import Optional, Sequence

import numpy as np


def averages(sums: np.ndarray, missing: np.ndarray, score_variant_counts: np.ndarray):
    """(AVG float64 [P,K], MISSING_PCT float32 [P,K]) from [P*K] sums/counts."""
    K = len(score_variant_counts)
    s = np.asarray(sums, np.float64).reshape(-1, K)
    m = np.asarray(missing, np.uint32).reshape(-1, K)
    total = np.asarray(score_variant_counts, np.uint32)[None, :]
    used = np.where(total >= m, total - m, 0).astype(np.float64)   # saturating_sub
    with np.errstate(divide="ignore", invalid="ignore"):
        avg = np.where(used > 0, s / np.where(used > 0, used, 1), 0.0)
        pct = np.where(total > 0, (m.astype(np.float32) / np.maximum(total, 1).astype(np.float32))
                       * np.float32(100.0), np.float32(0.0)).astype(np.float32)
    return avg, pct


def _shortest(x, single: bool) -> tuple[str, int]:
    """(digits, k) with |x| = int(digits) * 10**k and the fewest digits that
    read back to the same float64 (float32 when ``single``)."""
    t = np.float32(x) if single else np.float64(x)
    m, e = np.format_float_scientific(abs(t), unique=True, exp_digits=1).split("e")
    digits = m.replace(".", "").rstrip("0") or "0"
    return digits, int(e) - (len(digits) - 1)


def _ryu(x, single: bool) -> str:
    """Text of one value as the ryu crate (1.0.x) prints it: shortest
    round-trip digits, laid out as ``d.0`` / ``dd.dd`` / ``0.000dd`` when the
    decimal exponent is small (float64: point position -5 < kk <= 16; float32:
    -6 < kk <= 13) and ``d.ddde<exp>`` otherwise."""
    v = float(np.float32(x)) if single else float(x)
    if v != v:
        return "NaN"
    if v in (float("inf"), float("-inf")):
        return "inf" if v > 0 else "-inf"
    sign = "-" if np.signbit(v) else ""
    if v == 0.0:
        return sign + "0.0"
    digits, k = _shortest(v, single)
    hi, lo = (13, -6) if single else (16, -5)
    n = len(digits)
    kk = n + k          # 10^(kk-1) <= |v| < 10^kk
    if 0 <= k and kk <= hi:
        body = digits + "0" * k + ".0"
    elif 0 < kk <= hi:
        body = digits[:kk] + "." + digits[kk:]
    elif lo < kk <= 0:
        body = "0." + "0" * (-kk) + digits
    elif n == 1:
        body = f"{digits}e{kk - 1}"
    else:
        body = f"{digits[0]}.{digits[1:]}e{kk - 1}"
    return sign + body


def format_f64(x: float) -> str:
    return _ryu(x, single=False)


def format_f32(x) -> str:
    return _ryu(x, single=True)


def write_sscore(path, person_iids: Sequence[str], score_names: Sequence[str],
                 score_variant_counts, sums, missing,
                 score_regions: Optional[dict] = None) -> None:
    """Write the .sscore table atomically: a unique temporary file in the same
    directory, fsynced, renamed over the target (main.rs:1398-1548)."""
    avg, pct = averages(sums, missing, score_variant_counts)
    path = Path(path)
    tmp = path.with_name(f".{path.name}.{os.getpid()}.{time.time_ns()}.tmp")
    fd = os.open(tmp, os.O_WRONLY | os.O_CREAT | os.O_EXCL, 0o644)
    try:
        with os.fdopen(fd, "w") as f:
            if score_regions:
                wrote = False
                for name in score_names:
                    if name in score_regions:
                        if not wrote:
                            f.write("#REGION\tSCORE\tINTERVAL\n")
                            wrote = True
                        f.write(f"#REGION\t{name}\t{score_regions[name]}\n")
            f.write("#IID" + "".join(f"\t{n}_AVG\t{n}_MISSING_PCT" for n in score_names) + "\n")
            for p, iid in enumerate(person_iids):
                cells = "".join(f"\t{format_f64(avg[p, k])}\t{format_f32(pct[p, k])}"
                                for k in range(len(score_names)))
                f.write(f"{iid}{cells}\n")
            f.flush()
            os.fsync(f.fileno())
        os.replace(tmp, path)
    except BaseException:
        try:
            os.unlink(tmp)
        except OSError:
            pass
        raise


def read_sscore(path):
    """Parse a .sscore file -> (iids, names, AVG [P,K], MISSING_PCT [P,K])."""
    lines = [ln for ln in Path(path).read_text().splitlines() if not ln.startswith("#REGION")]
    header = lines[0].split("\t")
    assert header[0] == "#IID"
    names = [h[:-4] for h in header[1::2]]
    iids, avg, pct = [], [], []
    for ln in lines[1:]:
        if not ln.strip() or ln.startswith("#"):
            continue
        c = ln.split("\t")
        iids.append(c[0])
        avg.append([float(x) for x in c[1::2]])
        pct.append([float(x) for x in c[2::2]])
    return iids, names, np.array(avg), np.array(pct)
