"""The 8-bit limb split the tcgen05 kind::i8 kernels rely on, checked on the CPU.

Every value x of a score (a dosage weight, a missing correction, or a dS entry
of the backward) is written as l0 q0 + l1 q1 + l2 q2 + l3 q3 with
q0 = max |x| over the score / 127 and q(i+1) = q(i) / 254, each limb the
nearest integer to the remainder (gnm_t8_quanta + gnm_t8_build_planes and
gnm_bw_build8 in gnomon_b200/csrc/gnm_tensor.cu).  The kernels' exactness
rests on three facts tested here, for FP32 values of very different scales:

* no limb leaves [-127, 127], so the kernels' clamp never changes a limb;
* the residual is below q3 / 2 = max |x| / (2 * 127 * 254^3), i.e. 2^-31.9
  of the score's largest value;
* |limb x dosage| <= 254 per variant, so S32 sums of up to 2^23 variants (the
  kernels' flush interval) cannot overflow.
"""
import numpy as np
import pytest

STEP = 254.0
LIMBS = 4


def split(x: np.ndarray):
    """Limbs [LIMBS, n] (int, unclamped) and quanta [LIMBS] of one score's values,
    in the kernels' FP64 arithmetic."""
    x = np.asarray(x, np.float32).astype(np.float64)
    am = float(np.abs(x).max()) if x.size else 0.0
    q = am / 127.0 if am > 0 else 1.0
    limbs, quanta = [], []
    r = x.copy()
    for _ in range(LIMBS):
        li = np.rint(r / q)
        limbs.append(li)
        quanta.append(q)
        r = r - li * q
        q = q / STEP
    return np.array(limbs), np.array(quanta), r, am


@pytest.mark.parametrize("scale", [1e-30, 1e-6, 0.01, 1.0, 3e4, 1e30])
@pytest.mark.parametrize("dist", ["normal", "uniform", "sparse_extremes"])
def test_limbs_in_range_and_residual_bound(scale, dist):
    rng = np.random.default_rng([int(np.log10(scale) + 40), len(dist)])
    n = 20_000
    if dist == "normal":
        x = rng.standard_normal(n)
    elif dist == "uniform":
        x = rng.uniform(-1, 1, n)
    else:   # a few large values among tiny ones: most limbs of most values are 0
        x = rng.standard_normal(n) * 1e-6
        x[rng.integers(0, n, 7)] = rng.choice([-1.0, 1.0], 7)
    x = (x * scale).astype(np.float32)
    limbs, quanta, resid, am = split(x)
    assert np.abs(limbs).max() <= 127, "a limb would need the clamp"
    # remainder of the last limb: at most half its quantum (plus FP64 rounding
    # of the subtractions, far below it)
    bound = quanta[-1] / 2 * (1 + 1e-9)
    assert np.abs(resid).max() <= bound
    assert quanta[-1] / 2 <= am * 2.0 ** -31.9
    # the reconstruction the epilogue forms (int x quantum, summed in FP64)
    rec = (limbs * quanta[:, None]).sum(axis=0)
    assert np.abs(rec - x.astype(np.float64)).max() <= am * 2.0 ** -31.9 * (1 + 1e-6)


def test_s32_block_bound():
    """254 per variant over the 2^23-variant flush interval fits S32."""
    per_variant = 127 * 2          # |limb| x dosage 2 (missing indicator: 1)
    flush = 1 << 23
    assert per_variant * flush < 2 ** 31


def test_all_zero_score_has_zero_limbs():
    limbs, quanta, resid, am = split(np.zeros(100, np.float32))
    assert am == 0.0 and not limbs.any() and not resid.any() and quanta[0] == 1.0


def test_one_twenty_eighth_step_wastes_a_bit():
    """The first form stepped by 1/128: its limbs after the first stay within
    +-64, so the same four limbs left 2^-29 instead of 2^-31.9."""
    rng = np.random.default_rng(3)
    x = rng.standard_normal(50_000).astype(np.float32)
    x64 = x.astype(np.float64)
    am = float(np.abs(x64).max())
    q, r = am / 127.0, x64.copy()
    top = 0.0
    for i in range(LIMBS):
        li = np.rint(r / q)
        if i > 0:
            top = max(top, float(np.abs(li).max()))
        r -= li * q
        q /= 128.0
    assert top <= 64
    assert np.abs(r).max() > am * 2.0 ** -31.9   # coarser than the 1/254 step
