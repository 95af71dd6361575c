"""HWE-PCA projection blocks on the GPU (``gnm_project_*``).

gnomon projects samples onto a fitted HWE-PCA model variant block by variant
block (map/project.rs). Its GPU path does three things per block:
* unpacks the packed ``.bed`` codes through per-variant coefficients (code 00
  -> c0, 10 -> c1, 11 -> c2, missing -> 0; ``unpack_weighted_plink``,
  map/project.rs:322-370);
* multiplies the dense result by the block's loadings (``compute_scores_block``,
  :547-667);
* adds the sums into row-major f64 scores (:669-733).

``Projector`` does the same without a dense matrix or a GEMM:
* with 8 or more axes and linear coefficients (the reference's HWE ones), on
  the split-BF16 tensor engine in one pass;
* otherwise on exact FP32 lookup tables, one pass per axis.

The missing-data scan and the per-sample solves that follow stay with the
caller, as in the reference.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib


def hwe_coefficients(freqs, scales, weights=None, swapped=None) -> np.ndarray:
    """Per-variant coefficients [V][3] (f32) of genotypes 0, 1, 2 copies, as the
    reference builds them for a block (map/project.rs:2960-2975):
    ``(g - 2p) / scale * weight`` (0 when the scale is not positive), reversed
    for variants whose alleles are swapped against the model."""
    p = np.asarray(freqs, np.float64)
    s = np.asarray(scales, np.float64)
    w = np.ones_like(p) if weights is None else np.asarray(weights, np.float64)
    inv = np.where(s > 0, 1.0 / np.where(s > 0, s, 1.0), 0.0)
    g = np.arange(3, dtype=np.float64)[None, :]
    c = (g - 2.0 * p[:, None]) * inv[:, None] * w[:, None]
    if swapped is not None:
        sw = np.asarray(swapped, bool)
        c[sw] = c[sw, ::-1]
    return c.astype(np.float32)


class Projector:
    """Scores of ``n_samples`` samples on ``components`` axes, summed over the
    variant blocks passed to ``block``."""

    def __init__(self, n_samples: int, components: int, device: Optional[int] = None):
        self.lib = _lib.load()
        self.n, self.k = int(n_samples), int(components)
        self.bytes_per_variant = (self.n + 3) // 4
        h = C.c_void_p()
        e = _lib.gnm_error()
        _lib.check(self.lib.gnm_project_create(self.n, self.k, -1 if device is None else device,
                                               C.byref(h), C.byref(e)), e)
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            self.lib.gnm_project_destroy(self.handle)
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

    def block(self, packed, coeffs, loadings):
        """One block: packed rows [filled][ceil(n/4)] (u8), coeffs [filled][3]
        and loadings [filled][components]; staged as the reference stages
        them (f32, loadings column-major)."""
        rows = np.ascontiguousarray(packed, dtype=np.uint8).reshape(-1, self.bytes_per_variant)
        filled = rows.shape[0]
        cf = np.ascontiguousarray(coeffs, dtype=np.float32).reshape(filled, 3)
        ld = np.asarray(loadings).reshape(filled, self.k)
        cm = np.ascontiguousarray(ld.T, dtype=np.float32)       # [components][filled]
        e = _lib.gnm_error()
        _lib.check(self.lib.gnm_project_block(self.handle, rows.ctypes.data, filled,
                                              cf.ctypes.data, cm.ctypes.data, C.byref(e)), e)

    def scores(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Add the sums over every block so far into ``out`` [n][components]
        (zeros when not given) and return it."""
        if out is None:
            out = np.zeros((self.n, self.k), np.float64)
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != self.n * self.k:
            raise ValueError("out must be a C-contiguous float64 [n_samples][components] array")
        e = _lib.gnm_error()
        _lib.check(self.lib.gnm_project_scores(self.handle, out.ctypes.data, C.byref(e)), e)
        return out
