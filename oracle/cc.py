"""CPU restatement of EmSartRefine's shift measurement (TEST INFRASTRUCTURE).

Reconstructor::GetDisplacement (Reconstructor.cpp:1746-1960) with its kernels
conjMul, maxShift, maxShiftWeighted and findPeak (wbpWeighting.cu:244-386),
in numpy. The FFTs are numpy's (double precision, unnormalised inverse as
cuFFT's C2R); the kernels' single-precision arithmetic is kept operation by
operation. Pinned against the reference's kernels compiled for the host
(oracle/ref.py) by tests/test_cc.py.
"""
from __future__ import annotations

import numpy as np

from .driver import make_square

F32 = np.float32


def conj_mul(a, b):
    """conjMul (wbpWeighting.cu:244-262): conj(a) * b in float32."""
    a = np.asarray(a, np.complex64)
    b = np.asarray(b, np.complex64)
    ax, ay = a.real.astype(F32), a.imag.astype(F32)
    bx, by = b.real.astype(F32), b.imag.astype(F32)
    out = np.empty(a.shape, np.complex64)
    out.real = ax * bx + ay * by
    out.imag = ax * by - ay * bx
    return out


def origin_dist(n):
    """Folded distance of every pixel to the origin (wbpWeighting.cu:276-286):
    [y][x] float32."""
    m = np.arange(n, dtype=F32)
    m = np.where(m > F32(n // 2), F32(n) - m, m).astype(F32)
    return np.sqrt(m[None, :] * m[None, :] + m[:, None] * m[:, None]).astype(F32)


def max_shift(img, s):
    """maxShift (:266-293): zero beyond s."""
    img = np.asarray(img, F32)
    return np.where(origin_dist(img.shape[0]) > F32(s), F32(0.0), img).astype(F32)


def max_shift_weighted(img, s):
    """maxShiftWeighted (:296-327): zero beyond s, else / (distance + 1e-4)."""
    img = np.asarray(img, F32)
    d = origin_dist(img.shape[0])
    return np.where(d > F32(s), F32(0.0), img / (d + F32(0.0001))).astype(F32)


def find_peak(img, threshold):
    """findPeak (:331-386): uint8 mask, 0 at local maxima >= threshold
    (neighbours taken cyclically), 1 elsewhere."""
    v = np.asarray(img, F32)
    xm, xp = np.roll(v, 1, axis=1), np.roll(v, -1, axis=1)  # value at x-1, x+1
    M, P = np.roll(v, 1, axis=0), np.roll(v, -1, axis=0)    # rows y-1, y+1
    Mxm, Mxp = np.roll(M, 1, axis=1), np.roll(M, -1, axis=1)
    Pxm, Pxp = np.roll(P, 1, axis=1), np.roll(P, -1, axis=1)
    peak = ((xm < v) & (xp < v) & (M < v) & (P < v) & (Mxm <= v) & (Pxm < v) & (Mxp <= v) & (Pxp < v)
            & (v >= F32(threshold)))
    return np.where(peak, 0, 1).astype(np.uint8)


def _argmax(v):
    """nppiMaxIndx_32f_C1R: (value, x, y) of the maximum, the first in raster
    order; NaN takes no part (value NaN when nothing else is left)."""
    flat = v.ravel()
    ok = ~np.isnan(flat)
    if not ok.any():
        return float("nan"), 0, 0
    i = int(np.argmax(np.where(ok, flat, -np.inf)))
    n = v.shape[1]
    return float(flat[i]), i % n, i // n


def cc_map(cc, s):
    """The reference's ccMap: the (4s)^2 fft-shifted centre of cc
    (Reconstructor.cpp:275-313, 1833-1860)."""
    n = cc.shape[0]
    idx = (np.arange(4 * s) - 2 * s) % n
    return np.ascontiguousarray(cc[np.ix_(idx, idx)])


def cc_displacement(residual, model, N, bx, by, s, multi_peak=False):
    """GetDisplacement on two H x W float32 images. Returns a dict with
    shift (x, y), cc_value, cc (the normalised correlation before the
    maxShift mask), cc_map and, with multi_peak, cc_map_multi."""
    sq = []
    sums = []
    for img in (residual, model):
        q = make_square(np.ascontiguousarray(img, F32), N, bx, by, 0, 0)  # cts(..., false, false)
        mean = q.astype(np.float64).sum() / float(N * N)                     # nppiMean_32f_C1R
        q = (q - F32(mean)).astype(F32)                                       # nppiSubC_32f_C1IR
        sums.append(((q * q).astype(F32)).astype(np.float64).sum())         # nppiSqr + nppiSum
        sq.append(q)
    fa = np.fft.rfft2(sq[0].astype(np.float64)).astype(np.complex64)
    fb = np.fft.rfft2(sq[1].astype(np.float64)).astype(np.complex64)
    prod = conj_mul(fa, fb)
    cc = (np.fft.irfft2(prod.astype(np.complex128), s=(N, N)) * float(N * N)).astype(F32)  # unnormalised C2R
    div = F32(float(N * N) * np.sqrt(sums[0] * sums[1]))                  # nppiDivC_32f_C1IR
    with np.errstate(divide="ignore", invalid="ignore"):  # a flat image: 0 / 0
        cc = (cc / div).astype(F32)
    out = {"cc": cc, "cc_map": cc_map(cc, s)}
    masked = max_shift(cc, s)
    max_val, x, y = _argmax(masked)
    if multi_peak:
        mask = find_peak(masked, F32(max_val) * F32(0.9))
        w = np.where(mask == 0, F32(1.0), F32(0.0)).astype(F32)   # nppiSet_32f_C1R(1) + nppiSet_32f_C1MR(0)
        w = max_shift_weighted(w, s)
        out["cc_map_multi"] = cc_map(w, s)
        _, x, y = _argmax(w)
    sx, sy = float(x), float(y)
    if sx > N // 2:
        sx -= N
    if sy > N // 2:
        sy -= N
    if not (max_val > 0.0):
        sx = sy = -1000.0
    out["shift"] = (sx, sy)
    out["cc_value"] = max_val
    return out
