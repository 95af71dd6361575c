"""CPU oracle for HWE-PCA projection blocks — TEST INFRASTRUCTURE ONLY.

Only ``tests/`` and ``bench.py``'s CPU-baseline leg import this module, and
only as the checker; the product (``gnomon_b200``) never imports it.

It restates the reference's GPU projection of a variant block
(map/project.rs) in float64 numpy:
* ``unpack_weighted_plink`` (:322-370): code 00 -> coeffs[v][0], 10 ->
  coeffs[v][1], 11 -> coeffs[v][2], missing (01) -> 0, for every sample;
* ``compute_scores_block`` (:547-667): that matrix times the block's loadings;
* ``accumulate_col_major_scores_into_row_major`` (:721-733): a column-major
  block result added into row-major scores.

Parity is pinned by the reference's own known-answer test of the last step
(map/project.rs:3927-3944) and by the kernel's formula. The reference holds
no golden vectors for the first two steps, so their parity is unpinned beyond
that formula. ``tests/golden/ld_projection_fixture.npz`` freezes this
module's scores for one block over the reference's real ``ld.bed`` rows
(data/testdata), so the restatement and the kernel are held to the same
numbers on real genotypes.
"""
from __future__ import annotations

import numpy as np


def unpack_weighted(packed: np.ndarray, n_samples: int, coeffs: np.ndarray) -> np.ndarray:
    """[filled][n_samples] float64: each sample's code through its variant's coefficients."""
    rows = np.asarray(packed, np.uint8).reshape(-1, (n_samples + 3) // 4)
    codes = np.stack([(rows >> (2 * s)) & 3 for s in range(4)], axis=-1).reshape(rows.shape[0], -1)
    codes = codes[:, :n_samples]
    c = np.asarray(coeffs, np.float32).astype(np.float64).reshape(-1, 3)
    table = np.zeros((c.shape[0], 4), np.float64)   # by code: 00, 01 (missing), 10, 11
    table[:, 0], table[:, 2], table[:, 3] = c[:, 0], c[:, 1], c[:, 2]
    return np.take_along_axis(table, codes.astype(np.int64), axis=1)


def project_block(packed, n_samples, coeffs, loadings) -> np.ndarray:
    """[n_samples][components] float64 sums of one block."""
    a = unpack_weighted(packed, n_samples, coeffs)
    ld = np.asarray(loadings, np.float32).astype(np.float64).reshape(a.shape[0], -1)
    return a.T @ ld


def abs_terms(packed, n_samples, coeffs, loadings) -> np.ndarray:
    """[n_samples][components] sum of |term| (the scale of a sum's rounding)."""
    a = np.abs(unpack_weighted(packed, n_samples, coeffs))
    ld = np.abs(np.asarray(loadings, np.float32).astype(np.float64).reshape(a.shape[0], -1))
    return a.T @ ld


def accumulate_col_major_into_row_major(dst: np.ndarray, src_col_major: np.ndarray,
                                        n_samples: int, components: int) -> None:
    """dst[sample * components + k] += src[k * n_samples + sample]."""
    src = np.asarray(src_col_major, np.float64).reshape(components, n_samples)
    dst.reshape(n_samples, components)[:] += src.T
