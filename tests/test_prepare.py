"""Projection preparation (Reconstructor::PrepareProjection,
Reconstructor.cpp:1158-1383) on the GPU against the oracle's restatement.

Covers the input types, mirror padding (DM4 stacks flipped in y), bad-pixel
replacement, the SART branch with each normalisation (standard deviation,
mean, none: centre-half statistics), the band-pass filter or SkipFilter,
dose weighting, and the WBP branch with its weighting filters and
down-weighted tilts. Rectangular W x H images exercise the centred padding.
The statistics are FP64 sums on both sides (the reference's NPP reductions
are not pinned).
"""
import numpy as np
import pytest

from tests.helpers import cuda, host, rel_l2

W, H = 80, 64

CASES = {
    "sart_std_f32": dict(dtype="f32"),
    "sart_mean_u16": dict(dtype="u16", normalization=0),
    "sart_none_s16": dict(dtype="s16", normalization=2),
    "sart_skip_s32_dm4": dict(dtype="s32", skip_filter=1, mirror_y=1),
    "sart_dose_u32": dict(dtype="u32", dose_weighting=1, accumulated_dose=12.0, pixel_size_nm=0.27),
    "wbp_ramp_downweight": dict(dtype="f32", wbp=1, wbp_filter=0, down_weight_tilts=1, tilt_deg=-48.0, psi_deg=0.7),
    "wbp_contrast10_none": dict(dtype="u16", wbp=1, wbp_filter=3, normalization=2, psi_deg=-1.2, skip_filter=1),
    "sart_no_badpixel_fix": dict(dtype="f32", correct_bad_pixels=0),
}

NP = {"f32": np.float32, "s16": np.int16, "u16": np.uint16, "s32": np.int32, "u32": np.uint32}


def _raw(dtype, seed):
    rng = np.random.default_rng(seed)
    img = rng.poisson(200.0, size=(H, W)).astype(np.float64)
    img += 40.0 * np.sin(np.arange(W) / 7.0)[None, :] + 30.0 * np.cos(np.arange(H) / 5.0)[:, None]
    img[rng.integers(0, H, 6), rng.integers(0, W, 6)] = 5000.0  # hot pixels
    if dtype == "f32":
        return img.astype(np.float32) * 0.37
    return np.clip(np.round(img), 0, None).astype(NP[dtype])


def _config(c):
    pc = dict(normalization=1, correct_bad_pixels=1, bad_pixel_value=10.0, lp=30.0, hp=2.0, lps=6.0, hps=1.0)
    pc.update({k: v for k, v in c.items() if k != "dtype"})
    return pc


def test_oracle_prepare_normalises_sart_images():
    from oracle.driver import prepare_projection

    raw = _raw("f32", 1)
    out, mean, std, bad = prepare_projection(raw, max(W, H), _config(dict(dtype="f32")))
    # counted on the padded square, as the reference does: mirror padding
    # repeats hot pixels that sit near the border
    assert bad >= 6
    assert abs(float(out.astype(np.float64).mean())) < 1e-4  # mean-free after (x - mean) / (-std)
    assert abs(float(out.astype(np.float64).std()) - 1.0) < 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_prepare_projection_matches_oracle(name):
    import torch

    import artiatomi_b200 as E
    from oracle.driver import prepare_projection

    c = CASES[name]
    raw = _raw(c["dtype"], hash(name) % 1000)
    pc = _config(c)
    ref, mean, std, bad = prepare_projection(raw, max(W, H), pc)
    tilt = np.array([0.0], np.float32)
    rec = E.Reconstructor(E.ReconConfig(W, H, 1), E.projection_geometry(E.Markers(tilt), W, H), tilt)
    raw_d = torch.from_numpy(raw.view(np.int16) if c["dtype"] == "u16" else raw).cuda()
    if c["dtype"] == "u16":
        raw_d = raw_d.view(torch.uint16)
    out = torch.zeros((H, W), device="cuda")
    m, s, b = rec.prepare_projection(raw_d, out, **pc)
    got = host(out)
    assert b == bad
    assert abs(m - mean) <= 1e-5 * max(1.0, abs(mean)), (m, mean)
    assert abs(s - std) <= 1e-5 * max(1.0, abs(std)), (s, std)
    assert rel_l2(got, ref) <= 1e-5, rel_l2(got, ref)
    rec.close()
