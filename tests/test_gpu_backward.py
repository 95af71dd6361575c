"""Backward kernel dW = G^T dS (re-unpacking genotypes) and the autograd Function.
The kernel tests run both dS limb widths: 8-bit limbs (gnm_t8_backward, the
default) and BF16 limbs (gnm_tc_backward)."""
import numpy as np
import pytest

from gnomon_b200 import _lib
from gnomon_b200.prepare import PreparationResult
from helpers import synth_case
from oracle import oracle

pytestmark = pytest.mark.gpu


def _device_rows(rows, pitch):
    import torch
    dev = np.zeros((rows.shape[0], pitch), np.uint8)
    dev[:, :rows.shape[1]] = rows
    return torch.from_numpy(dev).cuda()


@pytest.mark.parametrize("bits", [8, 16])
@pytest.mark.parametrize("keep", [False, True])
def test_backward_kernel_vs_extended(cuda, keep, bits):
    import torch
    from gnomon_b200.device import DevicePlan, row_pitch
    _, prep, rows, _ = synth_case(3001, 517, scores=19, config="diff_20k_x_200k_k16")
    if keep:
        sel = np.random.default_rng(1).choice(3001, 1111, replace=False).astype(np.uint32)
        prep = PreparationResult(prep.sparse_weights, prep.sparse_missing_corrections,
                                 prep.sparse_score_columns, prep.sparse_row_offsets,
                                 prep.score_names, 3001, output_idx_to_fam_idx=sel)
    P, K = prep.num_people_to_score, prep.num_scores
    gs = np.random.default_rng(2).standard_normal((P, K)).astype(np.float32)
    pitch = row_pitch(prep.bytes_per_variant)
    plan = DevicePlan(prep, engine=_lib.ENGINE_PLAIN)
    plan.set_backward_limbs(bits)
    gw, gc = plan.backward(_device_rows(rows, pitch), pitch, torch.from_numpy(gs).cuda(),
                           grad_corr=True)
    plan.sync()
    ew, ec = oracle.backward_extended(rows, prep, gs)
    scale = np.abs(gs).sum(axis=0).max()
    assert np.abs(gw.cpu().numpy() - ew).max() / scale < 1e-6
    assert np.abs(gc.cpu().numpy() - ec).max() / scale < 1e-6


def test_autograd_finite_differences_and_fp64_gradient(cuda):
    """Refit weights against a phenotype: MSE loss, central differences h=1e-3,
    and the FP64 gradient of the same loss."""
    import torch
    from gnomon_b200 import synth
    from gnomon_b200.autograd import polygenic_score
    from gnomon_b200.device import row_pitch
    w0 = synth.scaled(synth.WORKLOADS["diff_20k_x_200k_k16"], 2000, 600, 4)
    thr = synth.variant_thresholds(w0.seed, 0, 600, w0.p_lo, w0.p_hi, w0.missing_rate)
    rows = synth.synth_rows(w0.seed, 0, 600, 2000, thr)
    rng = np.random.default_rng(5)
    V, K, P = 600, 4, 2000
    member = rng.random((V, K)) < 0.8
    flipped = rng.random((V, K)) < 0.1
    wt = (rng.standard_normal((V, K)) * 0.05).astype(np.float32)
    y = torch.from_numpy(rng.standard_normal(P)).cuda()
    pitch = row_pitch((P + 3) // 4)
    d_rows = _device_rows(rows, pitch)
    fl_t, mb_t = torch.from_numpy(flipped), torch.from_numpy(member)

    def loss_of(wnp):
        wv = torch.from_numpy(wnp).cuda().requires_grad_(True)
        S, _ = polygenic_score(wv, d_rows, pitch, fl_t, mb_t, P)
        L = ((S - y[:, None]) ** 2).mean()
        return L, wv

    L, wv = loss_of(wt)
    L.backward()
    g = wv.grad.cpu().numpy().astype(np.float64)

    # FP64 reference gradient through the extended oracle
    from gnomon_b200.autograd import prep_from_dense
    prep = prep_from_dense(wt, flipped, member, P)
    S64, _ = oracle.score_extended(rows, prep)
    dS = 2.0 * (S64.reshape(P, K) - y.cpu().numpy()[:, None]) / (P * K)
    G, C = oracle.backward_extended(rows, prep, dS.astype(np.float32))
    colsum = dS.sum(axis=0)[None, :]
    g64 = np.where(flipped & member, 2 * (colsum + C) - G, np.where(member, G, 0.0))
    denom = np.abs(g64).max()
    assert np.abs(g - g64).max() / denom < 1e-5

    # central finite differences on a handful of member cells
    h = 1e-3
    cells = [tuple(c) for c in np.argwhere(member)[rng.choice(member.sum(), 12, replace=False)]]
    for (v, k) in cells:
        wp, wm = wt.copy(), wt.copy()
        wp[v, k] += h
        wm[v, k] -= h
        fd = (loss_of(wp)[0].item() - loss_of(wm)[0].item()) / (2 * h)
        assert abs(fd - g[v, k]) <= 1e-4 * max(1.0, abs(g[v, k])) + 1e-7, (v, k, fd, g[v, k])


@pytest.mark.parametrize("bits", [8, 16])
def test_backward_many_people_and_score_scales(cuda, bits):
    """More than 32768 people (two exact FP32 blocks of the BF16 backward), a
    ragged last variant tile, and scores whose dS magnitudes differ by 60
    orders (the per-score limb quantum), one all-zero."""
    import torch
    from gnomon_b200.device import DevicePlan, row_pitch
    _, prep, rows, _ = synth_case(40001, 260, scores=5, config="diff_20k_x_200k_k16")
    P, K = prep.num_people_to_score, prep.num_scores
    rng = np.random.default_rng(7)
    gs = rng.standard_normal((P, K)).astype(np.float32)
    gs[:, 0] *= np.float32(1e-3)
    gs[:, 1] *= np.float32(1e3)
    gs[:, 2] = 0.0
    gs[:, 3] *= np.float32(1e-30)
    gs[::7, 4] = np.float32(0.0)
    pitch = row_pitch(prep.bytes_per_variant)
    plan = DevicePlan(prep, engine=_lib.ENGINE_PLAIN)
    plan.set_backward_limbs(bits)
    gw, gc = plan.backward(_device_rows(rows, pitch), pitch, torch.from_numpy(gs).cuda(),
                           grad_corr=True)
    plan.sync()
    ew, ec = oracle.backward_extended(rows, prep, gs)
    gw, gc = gw.cpu().numpy().astype(np.float64), gc.cpu().numpy().astype(np.float64)
    for k in range(K):
        scale = np.abs(gs[:, k].astype(np.float64)).sum()
        if scale == 0:
            assert not gw[:, k].any() and not gc[:, k].any()
            continue
        assert np.abs(gw[:, k] - ew[:, k]).max() / scale < 1e-6, k
        assert np.abs(gc[:, k] - ec[:, k]).max() / scale < 1e-6, k


def test_backward_limbs_rejects_other_widths(cuda):
    _, prep, _, _ = synth_case(100, 64, scores=2, config="diff_20k_x_200k_k16")
    from gnomon_b200.device import DevicePlan
    plan = DevicePlan(prep, engine=_lib.ENGINE_PLAIN)
    for bad in (0, 4, 32):
        with pytest.raises(_lib.GnomonGpuError) as ei:
            plan.set_backward_limbs(bad)
        assert ei.value.status == _lib.GNM_ERR_INVALID
    plan.close()
