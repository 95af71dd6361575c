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


def _fmt64(x: float) -> str:
    r = repr(float(x))
    return r.replace("e-0", "e-").replace("e+0", "e").replace("e+", "e")


def _fmt32(x: np.float32) -> str:
    return _fmt64(float(np.format_float_positional(np.float32(x), unique=True, trim="0")
                        if np.isfinite(x) else x))


def write_sscore(path, person_iids: Sequence[str], score_names: Sequence[str],
                 score_variant_counts, sums, missing,
                 score_regions: Optional[dict] = None) -> None:
    """Write the .sscore table atomically (temp file + rename, like the reference)."""
    avg, pct = averages(sums, missing, score_variant_counts)
    path = Path(path)
    tmp = path.with_name(f".{path.name}.{os.getpid()}.tmp")
    with open(tmp, "w") as f:
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
            cells = "".join(f"\t{_fmt64(avg[p, k])}\t{_fmt32(pct[p, k])}"
                            for k in range(len(score_names)))
            f.write(f"{iid}{cells}\n")
    os.replace(tmp, path)


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
