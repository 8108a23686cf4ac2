"""EmSartRefine's shift measurement (Reconstructor::GetDisplacement,
Reconstructor.cpp:1746-1960).

CPU: the oracle's kernels (conjMul, maxShift, maxShiftWeighted, findPeak)
bit for bit against the reference's own kernel sources compiled for the
host, and the oracle's displacement on images with known shifts. GPU:
esb_rec_cc_displacement against the oracle: the same integer shift, the
correlation maximum and both correlation maps within FP32 FFT rounding.
"""
import numpy as np
import pytest

from oracle import cc as OC
from oracle import ref as R

N_REF = 48


def _ref_or_skip():
    if R.lib() is None:
        pytest.skip("reference kernels not built (no reference tree)")


def _spectra(seed):
    rng = np.random.default_rng(seed)
    shape = (N_REF, N_REF // 2 + 1)
    a = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64) * 1e3
    b = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    return a, b


def test_conj_mul_pinned_to_reference():
    _ref_or_skip()
    a, b = _spectra(1)
    np.testing.assert_array_equal(OC.conj_mul(a, b), R.conj_mul(a, b))


@pytest.mark.parametrize("s", [1, 5, 17, 24])
def test_max_shift_pinned_to_reference(s):
    _ref_or_skip()
    img = np.random.default_rng(s).normal(size=(N_REF, N_REF)).astype(np.float32)
    np.testing.assert_array_equal(OC.max_shift(img, s), R.max_shift(img, s))
    np.testing.assert_array_equal(OC.max_shift_weighted(img, s), R.max_shift(img, s, weighted=True))


def test_find_peak_pinned_to_reference():
    _ref_or_skip()
    rng = np.random.default_rng(3)
    # quantised values: plateaus and equal neighbours exercise the < / <= tests
    img = np.round(rng.normal(size=(N_REF, N_REF)) * 2.0).astype(np.float32)
    img[0, 0], img[N_REF - 1, 5] = 9.0, 9.0  # peaks on the wrapped border
    for thr in (-10.0, 0.0, 1.5, 9.0):
        np.testing.assert_array_equal(OC.find_peak(img, thr), R.find_peak(img, thr))


def _blob(H, W, cx, cy, sigma=2.5):
    y, x = np.mgrid[0:H, 0:W].astype(np.float64)
    return np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2.0 * sigma * sigma))


def _pair(H=40, W=48, d=(3, -2), seed=0, noise=0.01):
    """model: a blob with some texture; residual: the model moved by d
    (x, y) plus noise. GetDisplacement's shift is then -d."""
    rng = np.random.default_rng(seed)
    m = _blob(H, W, W / 2 - 0.3, H / 2 + 0.4) + 0.5 * _blob(H, W, W / 2 + 4, H / 2 - 3, 1.5)
    r = np.roll(m, (d[1], d[0]), axis=(0, 1)) + noise * rng.normal(size=(H, W))
    return r.astype(np.float32), m.astype(np.float32)


@pytest.mark.parametrize("d", [(3, -2), (-4, 0), (0, 5), (0, 0)])
def test_oracle_finds_known_shift(d):
    r, m = _pair(d=d)
    N = 48
    o = OC.cc_displacement(r, m, N, 0, (N - 40) // 2, 6)
    assert o["shift"] == (-float(d[0]), -float(d[1]))
    assert 0.9 < o["cc_value"] <= 1.0 + 1e-6
    assert o["cc_map"].shape == (24, 24)
    # the map is the centre of the correlation, origin at (2s, 2s)
    assert np.unravel_index(np.argmax(o["cc_map"]), (24, 24)) == (12 - d[1], 12 - d[0])


def test_oracle_multi_peak_takes_nearest():
    """Two copies of the model: the stronger at distance 5, the weaker (still
    above 0.9 of the maximum) at distance 2. Single-peak detection takes the
    stronger, multi-peak detection the nearer."""
    H = W = 48
    m = _blob(H, W, 24.0, 24.0, 1.5).astype(np.float32)
    r = (1.0 * np.roll(m, (0, 5), axis=(0, 1)) + 0.95 * np.roll(m, (2, 0), axis=(0, 1))).astype(np.float32)
    single = OC.cc_displacement(r, m, 48, 0, 0, 8)
    multi = OC.cc_displacement(r, m, 48, 0, 0, 8, multi_peak=True)
    assert single["shift"] == (-5.0, 0.0)
    assert multi["shift"] == (0.0, -2.0)
    assert multi["cc_value"] == single["cc_value"]
    assert np.count_nonzero(multi["cc_map_multi"]) == 2


# --------------------------------------------------------------------- GPU


def _rec(W, H):
    import artiatomi_b200 as E

    tilt = np.zeros(1, np.float32)
    return E.Reconstructor(E.ReconConfig(W, H, 1), E.projection_geometry(E.Markers(tilt), W, H), tilt)


GPU_CASES = {
    "rect_single": dict(W=48, H=40, d=(3, -2), s=6, multi=False),
    "rect_multi": dict(W=48, H=40, d=(-4, 1), s=6, multi=True),
    "tall_single": dict(W=40, H=56, d=(0, 5), s=9, multi=False),
    "square_zero_shift": dict(W=64, H=64, d=(0, 0), s=3, multi=True),
    "max_shift_half": dict(W=32, H=32, d=(2, 2), s=16, multi=True),
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(GPU_CASES))
def test_cc_displacement_matches_oracle(case):
    import torch

    from tests.helpers import cuda, host

    p = GPU_CASES[case]
    W, H, s = p["W"], p["H"], p["s"]
    r, m = _pair(H, W, p["d"], seed=len(case))
    N = max(W, H)
    o = OC.cc_displacement(r, m, N, (N - W) // 2, (N - H) // 2, s, multi_peak=p["multi"])
    rec = _rec(W, H)
    cmap = torch.zeros((4 * s, 4 * s), device="cuda")
    cmulti = torch.zeros((4 * s, 4 * s), device="cuda") if p["multi"] else None
    shift, val = rec.cc_displacement(cuda(r), cuda(m), s, p["multi"], cmap, cmulti)
    assert shift == o["shift"], (shift, o["shift"])
    assert shift == (-float(p["d"][0]), -float(p["d"][1]))
    assert abs(val - o["cc_value"]) <= 1e-5 * abs(o["cc_value"])
    np.testing.assert_allclose(host(cmap), o["cc_map"], rtol=0, atol=1e-5)
    if p["multi"]:
        np.testing.assert_array_equal(host(cmulti), o["cc_map_multi"])


@pytest.mark.gpu
def test_cc_displacement_multi_peak_and_no_correlation():
    """The multi-peak case of the oracle test, and an anti-correlated pair
    whose maximum inside max_shift is not positive: (-1000, -1000)."""
    from tests.helpers import cuda

    H = W = 48
    m = _blob(H, W, 24.0, 24.0, 1.5).astype(np.float32)
    r = (1.0 * np.roll(m, (0, 5), axis=(0, 1)) + 0.95 * np.roll(m, (2, 0), axis=(0, 1))).astype(np.float32)
    rec = _rec(W, H)
    assert rec.cc_displacement(cuda(r), cuda(m), 8, False)[0] == (-5.0, 0.0)
    assert rec.cc_displacement(cuda(r), cuda(m), 8, True)[0] == (0.0, -2.0)
    # a flat model correlates with nothing: every value is 0 (or NaN)
    flat = np.ones((H, W), np.float32)
    o = OC.cc_displacement(r, flat, 48, 0, 0, 8)
    got = rec.cc_displacement(cuda(r), cuda(flat), 8, False)
    assert o["shift"] == (-1000.0, -1000.0) and got[0] == (-1000.0, -1000.0)


@pytest.mark.gpu
def test_cc_displacement_rejects_bad_max_shift():
    from artiatomi_b200._lib import EsbError
    from tests.helpers import cuda

    r, m = _pair(32, 32, (1, 1))
    rec = _rec(32, 32)
    for s in (0, 17):
        with pytest.raises(EsbError):
            rec.cc_displacement(cuda(r), cuda(m), s)


def test_oracle_correlation_is_the_normalised_circular_correlation():
    """The FFT route of GetDisplacement (conj(A) B, unnormalised C2R, division
    by N^2 sqrt(SumA SumB)) against the direct sum
    cc(s) = sum_x a(x) b(x + s) / sqrt(sum a^2 sum b^2) of the mean-free
    squares, on a 12 x 12 case without padding."""
    rng = np.random.default_rng(5)
    n = 12
    a = rng.normal(size=(n, n)).astype(np.float32)
    b = rng.normal(size=(n, n)).astype(np.float32)
    o = OC.cc_displacement(a, b, n, 0, 0, 3)
    a0 = a.astype(np.float64) - a.mean(dtype=np.float64)
    b0 = b.astype(np.float64) - b.mean(dtype=np.float64)
    direct = np.zeros((n, n))
    for sy in range(n):
        for sx in range(n):
            direct[sy, sx] = (a0 * np.roll(b0, (-sy, -sx), axis=(0, 1))).sum()
    direct /= np.sqrt((a0 * a0).sum() * (b0 * b0).sum())
    np.testing.assert_allclose(o["cc"], direct, rtol=0, atol=2e-6)
