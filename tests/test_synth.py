"""The synthetic generator: numpy reference == C oracle generator; HWE sanity."""
import numpy as np
import pytest

from gnomon_b200 import synth
from oracle import oracle


@pytest.mark.parametrize("people,variants", [(1, 3), (7, 5), (101, 17), (4096 + 3, 9)])
def test_numpy_and_c_generators_match(people, variants):
    thr = synth.variant_thresholds(1234, 10, variants, 0.01, 0.5, 0.02)
    pitch = ((people + 3) // 4 + 15) // 16 * 16
    a = synth.synth_rows(1234, 10, variants, people, thr, pitch)
    b = oracle.synth_rows(1234, 10, variants, people, thr, pitch)
    np.testing.assert_array_equal(a, b)
    # padding people and pitch bytes are zero
    assert (a[:, (people + 3) // 4:] == 0).all()
    if people % 4:
        last = a[:, people // 4]
        assert (last >> (2 * (people % 4)) == 0).all()


def test_hwe_statistics():
    thr = synth.variant_thresholds(99, 0, 400, 0.01, 0.5, 0.01)
    codes = synth.genotype_codes(99, 0, 400, 5000, thr)
    miss = (codes == 1).mean()
    assert abs(miss - 0.01) < 0.002
    p = synth.allele_freqs(99, 0, 400, 0.01, 0.5)
    nm = codes != 1
    d = np.where(codes == 2, 1, np.where(codes == 3, 2, 0))
    est = (d * nm).sum(1) / (2 * nm.sum(1))
    assert np.abs(est - p).max() < 0.03
    assert p.min() >= 0.01 and p.max() <= 0.5


def test_uneven_scores_membership():
    w = synth.scaled(synth.WORKLOADS["batched_100k_x_500k_k512"], 100, 20_000, 8)
    offs, cols, weight, flipped = synth.score_cells(w)
    assert offs[-1] == len(cols) == len(weight)
    sizes = np.bincount(cols, minlength=8)
    assert (sizes > 0).all() and (sizes <= 20_000).all()
    assert 0.07 < flipped.mean() < 0.13
    for v in (0, 5, 19_999):
        r = cols[offs[v]:offs[v + 1]]
        assert (np.diff(r.astype(np.int64)) > 0).all()
