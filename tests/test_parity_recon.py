"""Driver-level parity: the Reconstructor sequences (FP -> compare -> BP, the
CTF slab chains with cuFFT), the SART loop and the sub-volume WBP on the GPU
against the oracle's restatement of the same reference code paths.

The FFT differs (cuFFT vs the oracle's double radix-2 FFT) in the CTF cases,
so those use rel-L2 <= 1e-4 per projection/volume; the no-CTF SART is held to
rel-L2 <= 1e-5 against the FP32 oracle and 1e-3 against the FP64 oracle.
"""
import numpy as np
import pytest

from tests.helpers import cuda, host, rel_l2, small_case

pytestmark = pytest.mark.gpu


def _projections(case, ctf=False):
    """Measured projections: FP of the phantom by the oracle + noise."""
    from oracle import driver as D
    from oracle import geometry as G

    W, H = case["W"], case["H"]
    out = []
    rng = np.random.default_rng(21)
    for i in range(len(case["tilt"])):
        p = np.zeros((H, W), np.float32)
        d = np.zeros((H, W), np.float32)
        D.fp_march(G.orc_geom(case["og"][i], case["vo"]), case["vol"], 0, W, H, p, d, precision=1)
        p += rng.normal(0, 0.1 * p.std(), p.shape).astype(np.float32)
        out.append(p)
    return np.stack(out)


def _ctf_cfg(W):
    return dict(ctf_mode=True, pixel_size_nm=0.27, ctf_slice_thickness_nm=2.5, amp_contrast=0.0,
                ctf_beta_fac=(10.0, 0.0, 0.008, 0.0), cut_length=(2.0, 2.0), dim_length=(4.0, 4.0))


@pytest.mark.parametrize("sirt,os_", [(1, 1), (3, 2)])
def test_sart_no_ctf(sirt, os_):
    import artiatomi_b200 as E
    from oracle.driver import OracleReconstructor

    case = small_case(n_proj=9, shift=1.0, psi=0.2)
    W, H = case["W"], case["H"]
    projs = _projections(case)
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
    cfgd = dict(lambda_=0.5, oversampling=os_, cut_length=(1.0, 1.0), dim_length=(3.0, 3.0),
                crop=(1.0, 2.0, 1.0, 2.0), crop_dim=(3.0, 3.0, 3.0, 3.0))
    rec = E.Reconstructor(E.ReconConfig(W, H, len(case["tilt"]), **cfgd), case["pg"], case["tilt"])
    vol_d = cuda(np.zeros(case["vol"].shape, np.float32))
    empty = rec.sart(case["vg"], vol_d, cuda(projs), il, iterations=2, sirt_count=sirt)
    assert not empty
    got = host(vol_d)
    for prec, tol in ((0, 1e-5), (1, 1e-3)):
        orc = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], precision=prec)
        vo = np.zeros(case["vol"].shape, np.float32)
        orc.sart(case["vo"], vo, 0, projs, il, 2, sirt)
        assert rel_l2(got, vo) <= tol, (prec, rel_l2(got, vo))


def test_forward_and_back_projection_ctf():
    import torch

    import artiatomi_b200 as E
    from oracle.driver import OracleReconstructor

    case = small_case(dims=(64, 64, 24), n_proj=5, shift=1.0)
    W, H = case["W"], case["H"]
    n = len(case["tilt"])
    rng = np.random.default_rng(5)
    defocus = np.stack([rng.uniform(2900, 3100, n), rng.uniform(3100, 3200, n), rng.uniform(0, 180, n)], 1)
    defocus = defocus.astype(np.float32).ravel()
    cfgd = _ctf_cfg(W)
    rec = E.Reconstructor(E.ReconConfig(W, H, n, **cfgd), case["pg"], case["tilt"], defocus)
    orc = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], defocus, precision=0)
    vol_d = cuda(case["vol"])
    proj_v, dist_v, _ = rec.views()
    for i in range(n):
        rec.reset_projections()
        rec.forward_projection(case["vg"], vol_d, i, False)
        orc.reset()
        orc.forward_projection(case["vo"], case["vol"], 0, i, False)
        e = rel_l2(host(proj_v), orc.proj)
        assert e <= 1e-4, (i, e)
        e = rel_l2(host(dist_v), orc.dist)
        assert e <= 1e-6, (i, e)
    # CTF back projection of a random residual
    vol_b = cuda(np.zeros(case["vol"].shape, np.float32))
    vo = np.zeros(case["vol"].shape, np.float32)
    for i in range(n):
        res = rng.normal(size=(H, W)).astype(np.float32)
        proj_v.copy_(cuda(res))
        rec.back_projection(case["vg"], vol_b, i, 2.0)
        orc.back_projection(case["vo"], vo, 0, i, 2.0, img=res.copy())
    e = rel_l2(host(vol_b), vo)
    assert e <= 1e-4, e


def test_sart_ctf():
    import artiatomi_b200 as E
    from oracle.driver import OracleReconstructor

    case = small_case(dims=(64, 64, 24), n_proj=5, shift=0.5)
    W, H = case["W"], case["H"]
    n = len(case["tilt"])
    rng = np.random.default_rng(15)
    defocus = np.stack([rng.uniform(2900, 3100, n), rng.uniform(3100, 3200, n), rng.uniform(0, 180, n)], 1)
    defocus = defocus.astype(np.float32).ravel()
    projs = _projections(case)
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
    cfgd = dict(_ctf_cfg(W), lambda_=0.5, oversampling=2)
    rec = E.Reconstructor(E.ReconConfig(W, H, n, **cfgd), case["pg"], case["tilt"], defocus)
    vol_d = cuda(np.zeros(case["vol"].shape, np.float32))
    rec.sart(case["vg"], vol_d, cuda(projs), il, iterations=2, sirt_count=2)
    orc = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], defocus, precision=0)
    vo = np.zeros(case["vol"].shape, np.float32)
    orc.sart(case["vo"], vo, 0, projs, il, 2, 2)
    e = rel_l2(host(vol_d), vo)
    assert e <= 1e-4, e


@pytest.mark.parametrize("ctf,batched", [(False, False), (False, True), (True, True)])
def test_subvolume_wbp(ctf, batched):
    import artiatomi_b200 as E
    from oracle import geometry as G
    from oracle.driver import OracleReconstructor

    W = H = 96
    n = 7
    tilt = np.linspace(-60, 60, n).astype(np.float32)
    rng = np.random.default_rng(31)
    projs = rng.normal(size=(n, H, W)).astype(np.float32)
    full, fo = E.volume_geometry((96, 96, 40)), G.volume_geometry((96, 96, 40))
    sizes = [16, 24, 16, 32]
    pos = rng.uniform(20, 76, size=(len(sizes), 3))
    pos[:, 2] = rng.uniform(10, 30, len(sizes))
    shifts = rng.uniform(-1.5, 1.5, size=(len(sizes), n, 2)).astype(np.float32)
    sub = [E.subvolume_geometry(s, 1.0, full, p) for s, p in zip(sizes, pos)]
    subo = [G.subvolume_geometry(s, 1.0, fo, p) for s, p in zip(sizes, pos)]
    from artiatomi_b200 import _lib as L

    pair = (L.ProjGeom * (len(sizes) * n))()
    pair_o = []
    for p in range(len(sizes)):
        g = E.projection_geometry(E.Markers(tilt), W, H, extra_shift=shifts[p])
        for i in range(n):
            pair[p * n + i] = g[i]
        pair_o.append(G.projection_geometry(tilt, width=W, height=H, extra_shift=shifts[p]))
    active = (np.linalg.norm(shifts, axis=2) < 2.0 - 0.5).astype(np.uint8)
    defocus = np.stack([np.full(n, 3000.0), np.full(n, 3100.0), np.full(n, 20.0)], 1).astype(np.float32).ravel()
    cfgd = dict(oversampling=2, ctf_mode=ctf, pixel_size_nm=0.27, ctf_slice_thickness_nm=4.0,
                ctf_beta_fac=(10.0, 0.0, 0.008, 0.0))
    pg = E.projection_geometry(E.Markers(tilt), W, H)
    rec = E.Reconstructor(E.ReconConfig(W, H, n, **cfgd), pg, tilt, defocus if ctf else None)
    boxes = [cuda(np.zeros((s, s, s), np.float32)) for s in sizes]
    il = np.arange(n, dtype=np.int32)
    rec.subvolume_wbp(full, sub, pair, boxes, cuda(projs), il, active=active, batched=batched)
    orc = OracleReconstructor(cfgd, W, H, G.projection_geometry(tilt, width=W, height=H), tilt,
                              defocus if ctf else None)
    bo = [np.zeros((s, s, s), np.float32) for s in sizes]
    orc.subvolume_wbp(fo, subo, pair_o, bo, projs, il, active=active)
    for b, o in zip(boxes, bo):
        e = rel_l2(host(b), o)
        assert e <= (1e-4 if ctf else 1e-5), e
        assert np.abs(o).sum() > 0
