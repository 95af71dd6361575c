"""Differentiable polygenic score: ``torch.autograd.Function`` over the sm_100a kernels.

Forward: the plain engine scores all people (FP64 sums).  Backward: the
``gnm_backward_dw_device`` kernel re-unpacks the packed genotype rows (no dense
dosage matrix is ever stored) and returns, per (variant, score),
``G = sum_p d(p,v) dS[p,k]`` and ``C = -sum_{p missing} dS[p,k]``.

The trainable parameter is the score file's effect-allele weight ``w``.  The
prepared cell is ``dosage_weight = +w`` or ``-w`` (flipped) with
``missing_correction = 2w`` when flipped (score/prepare.rs:197-208), and the
baseline is the sum of corrections, so

    dS/dw = d                      (effect allele = BIM allele2)
    dS/dw = 2 * (1 - m) - d        (flipped: the cell contributes w * (2 - d))

which gives dL/dw = G for plain cells and 2 * (colsum(dS) + C) - G for
flipped cells (cells outside a score's variant set get no gradient).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .device import DevicePlan
from .prepare import PreparationResult


def prep_from_dense(weights: np.ndarray, flipped: np.ndarray, member: np.ndarray,
                    total_people_in_fam: int, output_idx_to_fam_idx=None) -> PreparationResult:
    """Dense [V, K] effect weights + flip / membership masks -> CSR PreparationResult."""
    w = np.asarray(weights, np.float32)
    V, K = w.shape
    m = np.asarray(member, bool)
    f = np.asarray(flipped, bool) & m
    rows, cols = np.nonzero(m)
    ww, ff = w[rows, cols], f[rows, cols]
    dw = np.where(ff, -ww, ww).astype(np.float32)
    mc = np.where(ff, np.float32(2.0) * ww, np.float32(0.0)).astype(np.float32)
    offs = np.zeros(V + 1, np.uint64)
    np.cumsum(m.sum(axis=1), out=offs[1:])
    return PreparationResult(dw, mc, cols.astype(np.uint32), offs,
                             [f"S{k:03d}" for k in range(K)], total_people_in_fam,
                             output_idx_to_fam_idx=output_idx_to_fam_idx)


class PolygenicScore(torch.autograd.Function):
    """S[p, k] (float64) = baseline + sum over cells, differentiable in ``weights``."""

    @staticmethod
    def forward(ctx, weights, rows, pitch, flipped, member, total_people_in_fam,
                output_idx_to_fam_idx=None):
        prep = prep_from_dense(weights.detach().cpu().numpy(), flipped.cpu().numpy(),
                               member.cpu().numpy(), total_people_in_fam,
                               output_idx_to_fam_idx)
        plan = DevicePlan(prep, engine=_lib.ENGINE_PLAIN, device=rows.device.index)
        sums, counts = plan.score(rows, pitch)
        plan.sync()
        ctx.plan, ctx.rows, ctx.pitch = plan, rows, pitch
        ctx.save_for_backward(flipped.to(rows.device), member.to(rows.device))
        P, K = prep.num_people_to_score, prep.num_scores
        ctx.mark_non_differentiable(counts)
        return sums.view(P, K), counts.view(P, K)

    @staticmethod
    def backward(ctx, grad_s, grad_counts=None):
        flipped, member = ctx.saved_tensors
        gs = grad_s.detach().to(torch.float32).contiguous()
        G, Cm = ctx.plan.backward(ctx.rows, ctx.pitch, gs, grad_corr=True)
        ctx.plan.sync()
        colsum = gs.to(torch.float64).sum(dim=0, keepdim=True)
        Gd, Cd = G.to(torch.float64), Cm.to(torch.float64)
        dw = torch.where(flipped, 2.0 * (colsum + Cd) - Gd, Gd)
        dw = torch.where(member, dw, torch.zeros_like(dw))
        ctx.plan.close()
        return dw.to(torch.float32), None, None, None, None, None, None


def polygenic_score(weights, rows, pitch, flipped, member, total_people_in_fam,
                    output_idx_to_fam_idx=None):
    """Functional form: returns (sums [P, K] float64 (differentiable), counts [P, K])."""
    return PolygenicScore.apply(weights, rows, pitch, flipped, member, total_people_in_fam,
                                output_idx_to_fam_idx)
