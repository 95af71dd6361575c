"""HWE-PCA projection blocks, CPU side: the oracle against the reference's
known-answer test, the coefficient rule, and the C ABI without a device."""
import numpy as np
import pytest

from gnomon_b200 import _lib, synth
from gnomon_b200.project import Projector, hwe_coefficients
from oracle import project_oracle


def test_col_major_accumulation_known_answer():
    """map/project.rs:3927-3944: 3 samples x 2 components, added twice."""
    src = np.array([10.0, 20.0, 30.0, 40.0, 50.0, 60.0], np.float32)
    dst = np.zeros(6)
    project_oracle.accumulate_col_major_into_row_major(dst, src, 3, 2)
    assert dst.tolist() == [10.0, 40.0, 20.0, 50.0, 30.0, 60.0]
    project_oracle.accumulate_col_major_into_row_major(dst, src, 3, 2)
    assert dst.tolist() == [20.0, 80.0, 40.0, 100.0, 60.0, 120.0]


def test_unpack_by_hand():
    # 5 samples: codes 00, 01, 10, 11, 00 for variant 0; 11, 11, 01, 10, 00 for variant 1
    codes = np.array([[0, 1, 2, 3, 0], [3, 3, 1, 2, 0]], np.uint8)
    packed = synth.pack_codes(codes)
    coeffs = np.array([[1.0, 2.0, 4.0], [-1.0, 0.5, 8.0]], np.float32)
    a = project_oracle.unpack_weighted(packed, 5, coeffs)
    np.testing.assert_array_equal(a, [[1, 0, 2, 4, 1], [8, 8, 0, 0.5, -1]])
    loadings = np.array([[1.0, 10.0], [100.0, 1000.0]], np.float32)
    s = project_oracle.project_block(packed, 5, coeffs, loadings)
    np.testing.assert_array_equal(s[:, 0], a[0] * 1 + a[1] * 100)
    np.testing.assert_array_equal(s[:, 1], a[0] * 10 + a[1] * 1000)


def test_hwe_coefficients():
    c = hwe_coefficients([0.1, 0.25, 0.3], [0.5, 2.0, 0.0], [1.0, 3.0, 1.0],
                         swapped=[False, True, False])
    np.testing.assert_allclose(c[0], [-0.4, 1.6, 3.6], rtol=1e-6)
    np.testing.assert_allclose(c[1], [2.25, 0.75, -0.75], rtol=1e-6)   # swapped: reversed
    np.testing.assert_array_equal(c[2], [0, 0, 0])        # zero scale -> 0
    assert c.dtype == np.float32


def test_create_declines_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(_lib.GnomonGpuError) as ei:
        Projector(10, 2)
    assert ei.value.status == _lib.GNM_DECLINED


def test_ld_projection_fixture_reproduces():
    """The restatement still gives the frozen scores of the real ld.bed block."""
    from pathlib import Path
    g = Path(__file__).resolve().parent / "golden"
    f, d = np.load(g / "ld_fixture.npz"), np.load(g / "ld_projection_fixture.npz")
    got = project_oracle.project_block(f["rows"], int(f["num_people"]), d["coeffs"], d["loadings"])
    np.testing.assert_allclose(got, d["scores"], rtol=1e-12, atol=1e-12)
