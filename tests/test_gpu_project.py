"""HWE-PCA projection blocks on the GPU (gnm_project_*) against the oracle."""
import numpy as np
import pytest

from gnomon_b200 import synth
from gnomon_b200.project import Projector, hwe_coefficients
from oracle import project_oracle

pytestmark = pytest.mark.gpu
# FP32 stage-table entries and FP32 sums over 120 variants, FP64 beyond:
# every sum within 1e-6 of the sum of its terms' magnitudes
TOL = 1e-6


def block_case(seed, n, filled, k, missing=0.01):
    rng = np.random.default_rng(seed)
    thr = synth.variant_thresholds(seed, 0, filled, 0.01, 0.5, missing)
    rows = synth.synth_rows(seed, 0, filled, n, thr)
    freqs = rng.uniform(0.01, 0.5, filled)
    scales = np.sqrt(2 * freqs * (1 - freqs)) * rng.uniform(0.8, 1.2, filled)
    scales[::97] = 0.0                                   # zero scale -> coefficients 0
    coeffs = hwe_coefficients(freqs, scales, rng.uniform(0.5, 1.5, filled),
                              rng.random(filled) < 0.1)
    loadings = (rng.standard_normal((filled, k)) / np.sqrt(filled)).astype(np.float32)
    return rows, coeffs, loadings


def check(got, rows, n, coeffs, loadings):
    want = project_oracle.project_block(rows, n, coeffs, loadings)
    # the terms' magnitudes, plus the baseline terms c0*L that a missing call
    # cancels (its FP32 record against the FP64 baseline)
    scale = project_oracle.abs_terms(rows, n, coeffs, loadings) + \
        (np.abs(coeffs[:, 0].astype(np.float64)) @ np.abs(loadings.astype(np.float64)))[None, :]
    err = np.abs(got - want)
    assert (err <= TOL * scale + 1e-30).all(), f"max err / scale {np.max(err / (scale + 1e-30)):.2e}"


@pytest.mark.parametrize("n,filled,k", [(1, 29, 1), (5, 30, 3), (203, 31, 2), (4097, 1000, 20),
                                        (50001, 4096, 10)])
def test_block_against_oracle(cuda, n, filled, k):
    rows, coeffs, loadings = block_case(n + filled, n, filled, k)
    with Projector(n, k) as pj:
        pj.block(rows, coeffs, loadings)
        check(pj.scores(), rows, n, coeffs, loadings)


def test_blocks_accumulate_and_scores_add(cuda):
    n, k = 3001, 4
    parts = [block_case(s, n, f, k) for s, f in ((1, 500), (2, 77), (3, 1200))]
    rows = np.concatenate([p[0] for p in parts])
    coeffs = np.concatenate([p[1] for p in parts])
    loadings = np.concatenate([p[2] for p in parts])
    with Projector(n, k) as pj:
        for r, c, l in parts:
            pj.block(r, c, l)
        base = np.full((n, k), 0.5)
        out = pj.scores(base.copy())
        check(out - base, rows, n, coeffs, loadings)   # added into the given scores


def test_missing_calls_contribute_nothing(cuda):
    n, k, filled = 257, 3, 64
    rows, coeffs, loadings = block_case(9, n, filled, k, missing=0.5)
    codes = synth.unpack_codes(rows, n)
    codes[:, ::2] = 1                                     # every other sample all missing
    rows = synth.pack_codes(codes)
    with Projector(n, k) as pj:
        pj.block(rows, coeffs, loadings)
        got = pj.scores()
    check(got, rows, n, coeffs, loadings)
    scale = np.abs(coeffs[:, [0]]).T @ np.abs(loadings)   # per component
    assert (np.abs(got[::2]) <= 1e-6 * scale + 1e-12).all()


@pytest.mark.parametrize("k", [3, 10, 70])
def test_nonlinear_coefficients(cuda, k):
    """Coefficients that are not linear in the dosage take the exact lookup
    tables at any axis count; linear ones with 8 or more axes take the
    tensor engine (the other tests), within the same bar."""
    n, filled = 1501, 700
    rows, coeffs, loadings = block_case(5, n, filled, k)
    coeffs = coeffs.copy()
    coeffs[::3, 2] += 0.25                              # c2 off the line through c0, c1
    with Projector(n, k) as pj:
        pj.block(rows, coeffs, loadings)
        check(pj.scores(), rows, n, coeffs, loadings)


def test_wide_tensor_block(cuda):
    """More than 64 linear axes: the wide tensor kernel."""
    n, filled, k = 2049, 900, 72
    rows, coeffs, loadings = block_case(6, n, filled, k)
    with Projector(n, k) as pj:
        pj.block(rows, coeffs, loadings)
        check(pj.scores(), rows, n, coeffs, loadings)


def test_real_ld_block_against_fixture(cuda):
    """All 1,500 variants of the reference's ld.bed (200 samples) as one block,
    coefficients from the rows' own allele frequencies, against the frozen
    float64 scores of the same block."""
    from pathlib import Path
    g = Path(__file__).resolve().parent / "golden"
    f, d = np.load(g / "ld_fixture.npz"), np.load(g / "ld_projection_fixture.npz")
    rows, n = f["rows"], int(f["num_people"])
    coeffs, loadings = d["coeffs"], d["loadings"]
    with Projector(n, loadings.shape[1]) as pj:
        pj.block(rows, coeffs, loadings)
        got = pj.scores()
    scale = project_oracle.abs_terms(rows, n, coeffs, loadings) + \
        (np.abs(coeffs[:, 0].astype(np.float64)) @ np.abs(loadings.astype(np.float64)))[None, :]
    err = np.abs(got - d["scores"])
    assert (err <= TOL * scale + 1e-30).all(), f"max err / scale {np.max(err / (scale + 1e-30)):.2e}"
