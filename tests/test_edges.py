"""Edge cases of the reconstruction path: rectangular detectors with CTF
padding, volume widths that are not a multiple of the 4-voxel quads, empty
work lists, the 256-slab limit and invalid counts."""
import numpy as np
import pytest

from tests.helpers import cuda, host, rel_l2, small_case


@pytest.mark.gpu
def test_fast_sart_ragged_sizes_with_ctf():
    """W != H (the CTF square is padded on one axis only), a volume width of
    50 (the last two voxels of each row lie beyond the last quad and are never
    updated, as in the reference) and an odd depth."""
    import artiatomi_b200 as E
    from oracle.driver import OracleReconstructor
    from tests.test_parity_recon import _ctf_cfg, _projections

    case = small_case(dims=(50, 44, 17), n_proj=5, W=72, H=56, shift=1.0, psi=0.2)
    W, H, n = case["W"], case["H"], len(case["tilt"])
    rng = np.random.default_rng(3)
    dmid = rng.uniform(2800.0, 3200.0, n)
    defocus = np.stack([dmid - 40.0, dmid + 40.0, rng.uniform(0, 180, n)], 1).astype(np.float32).ravel()
    projs = _projections(case)
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
    cfgd = dict(_ctf_cfg(max(W, H)), lambda_=0.5, oversampling=2)
    rec = E.Reconstructor(E.ReconConfig(W, H, n, variant=E.VARIANT_FAST, **cfgd), case["pg"], case["tilt"], defocus)
    v = cuda(np.zeros(case["vol"].shape, np.float32))
    rec.sart(case["vg"], v, cuda(projs), il, iterations=2, sirt_count=2)
    got = host(v)
    orc = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], defocus, precision=1)
    ref = np.zeros(case["vol"].shape, np.float32)
    orc.sart(case["vo"], ref, 0, projs, il, 2, 2)
    assert np.abs(ref).max() > 0
    assert np.all(got[:, :, 48:] == 0) and np.all(ref[:, :, 48:] == 0)
    assert rel_l2(got, ref) <= 1e-3, rel_l2(got, ref)


@pytest.mark.gpu
def test_empty_work_lists():
    import torch

    import artiatomi_b200 as E
    from artiatomi_b200 import _lib as L

    case = small_case(dims=(32, 32, 16), n_proj=3, W=32, H=32)
    rec = E.Reconstructor(E.ReconConfig(32, 32, 3, variant=E.VARIANT_FAST), case["pg"], case["tilt"])
    projs = torch.zeros((3, 32, 32), device="cuda")
    # no particles, and particles with no projection
    rec.subvolume_wbp(case["vg"], [], (L.ProjGeom * 0)(), [], projs, np.array([0, 1, 2], np.int32))
    box = torch.ones((16, 16, 16), device="cuda")
    sub = [E.subvolume_geometry(16, 1.0, case["vg"], (16, 16, 8))]
    pair = (L.ProjGeom * 3)(*[case["pg"][i] for i in range(3)])
    for batched in (False, True):
        rec.subvolume_wbp(case["vg"], sub, pair, [box], projs, np.zeros(0, np.int32), batched=batched)
        rec.subvolume_wbp(case["vg"], sub, pair, [box], projs, np.array([0, 1, 2], np.int32),
                          active=np.zeros((1, 3), np.uint8), batched=batched)
    assert float(box.min()) == 1.0 and float(box.max()) == 1.0
    # a SART run needs at least one projection
    v = torch.zeros((16, 32, 32), device="cuda")
    with pytest.raises(L.EsbError):
        rec.sart(case["vg"], v, projs, np.zeros(0, np.int32), iterations=1, sirt_count=1)
    with pytest.raises(L.EsbError):
        rec.sart(case["vg"], v, projs, np.array([0, 5], np.int32), iterations=1, sirt_count=1)


@pytest.mark.gpu
def test_more_than_256_ctf_slabs_is_reported():
    import torch

    import artiatomi_b200 as E
    from artiatomi_b200 import _lib as L
    from tests.test_parity_recon import _ctf_cfg

    case = small_case(dims=(64, 64, 64), n_proj=3, W=64, H=64)
    cfgd = dict(_ctf_cfg(64), ctf_slice_thickness_nm=0.05)  # ~0.2 voxel slabs: > 256 per projection
    defocus = np.tile(np.array([3000.0, 3100.0, 10.0], np.float32), 3)
    rec = E.Reconstructor(E.ReconConfig(64, 64, 3, variant=E.VARIANT_FAST, **cfgd), case["pg"], case["tilt"], defocus)
    rec.reset_projections()
    with pytest.raises(L.EsbError, match="256 CTF slabs"):
        rec.forward_projection(case["vg"], torch.zeros((64, 64, 64), device="cuda"), 1, False)
