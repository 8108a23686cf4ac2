"""The SART projection update that allocates no device memory
(esb_sart_projection_update_noalloc) against the reconstructor path that
owns cudaMalloc'd buffers, and against the CPU oracle.

The no-allocation entry point exists for callers that cannot call
cudaMalloc: an application whose device memory is owned and budgeted by its
own allocator, a process that must not allocate after start-up, or a loop
that must not pay cudaMalloc's implicit synchronisation. Its scratch lives in
a fixed array inside the library, shared by every call and keeping the last
call's contents. Two calls in a row must therefore give the same volumes as
two reconstructor steps. The first call uses volume_is_empty (traversal
length only), the second the full forward projection. Both paths run the same
kernels of the variant the configuration names, so the tolerance is the
kernel bar of the other tests (rel-L2 <= 1e-5, in practice bit-exact).
Against the oracle: the FAITHFUL kernels match its FP32 arithmetic (1e-5),
the FAST kernels its FP64 arithmetic (1e-4; the reference's float chords
are ~1 % noisy per update, the FAST chords exact).

This file is collected last so that a failure here comes after every other
test has run.
"""
import numpy as np
import pytest

from tests.helpers import cuda, host, rel_l2, small_case

pytestmark = pytest.mark.gpu

TOL = 1e-5
ORACLE_TOL = {0: 1e-5, 1: 1e-4}  # FAITHFUL vs FP32 oracle, FAST vs FP64 oracle


def _cfgd(os_):
    return dict(lambda_=0.5, oversampling=os_, cut_length=(1.0, 1.0), dim_length=(3.0, 3.0), crop=(1.0, 2.0, 1.0, 2.0),
                crop_dim=(3.0, 3.0, 3.0, 3.0))


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("os_", [1, 2])
def test_noalloc_update_matches_reconstructor_twice(os_, variant):
    import artiatomi_b200 as E

    case = small_case(n_proj=5, shift=1.0, psi=0.2)
    W, H = case["W"], case["H"]
    rng = np.random.default_rng(40 + os_)
    real = rng.normal(size=(len(case["tilt"]), H, W)).astype(np.float32) * 10
    real_d = cuda(real)
    cfg = E.ReconConfig(W, H, len(case["tilt"]), variant=variant, **_cfgd(os_))
    rec = E.Reconstructor(cfg, case["pg"], case["tilt"])
    vol0 = case["vol"].copy()
    vol_ref = cuda(vol0)
    vol_new = cuda(vol0)
    for call, (index, empty) in enumerate(((2, True), (4, False))):
        rec.reset_projections()
        rec.forward_projection(case["vg"], vol_ref, index, empty)
        rec.compare(case["vg"], real_d[index], index)
        rec.back_projection(case["vg"], vol_ref, index, 2.0)
        E.sart_projection_update_noalloc(cfg, case["pg"][index], case["vg"], vol_new, real_d[index], 2.0, empty)
        a, b = host(vol_new), host(vol_ref)
        assert np.abs(b - vol0).max() > 0, "the reference step changed nothing"
        err = rel_l2(a - vol0, b - vol0)
        assert err <= TOL, (call, err)
    rec.close()


@pytest.mark.parametrize("variant", [0, 1])
def test_noalloc_update_matches_oracle(variant):
    """Two calls in a row against the oracle's Reconstructor sequence
    (Reconstructor.cpp:429-490, 1386-1405, 871-887)."""
    import artiatomi_b200 as E
    from oracle.driver import OracleReconstructor

    case = small_case(n_proj=5, shift=1.0, psi=0.2)
    W, H = case["W"], case["H"]
    rng = np.random.default_rng(7)
    real = rng.normal(size=(len(case["tilt"]), H, W)).astype(np.float32) * 10
    real_d = cuda(real)
    cfgd = _cfgd(2)
    cfg = E.ReconConfig(W, H, len(case["tilt"]), variant=variant, **cfgd)
    orc = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], precision=variant)
    vol0 = case["vol"].copy()
    vol_d = cuda(vol0)
    vol_o = vol0.copy()
    for index, empty in ((2, True), (4, False)):
        E.sart_projection_update_noalloc(cfg, case["pg"][index], case["vg"], vol_d, real_d[index], 2.0, empty)
        orc.reset()
        orc.forward_projection(case["vo"], vol_o, 0, index, empty)
        orc.compare(case["vo"], real[index], index)
        orc.back_projection(case["vo"], vol_o, 0, index, 2.0, img=orc.proj.copy())
        err = rel_l2(host(vol_d) - vol0, vol_o - vol0)
        assert err <= ORACLE_TOL[variant], (index, err)


def test_noalloc_allocates_no_device_memory():
    """After a first call (which may load the kernels), further calls leave
    the device's free memory unchanged."""
    import torch

    import artiatomi_b200 as E

    case = small_case(n_proj=3)
    W, H = case["W"], case["H"]
    real = cuda(np.random.default_rng(1).normal(size=(H, W)).astype(np.float32))
    vol = cuda(case["vol"])
    stream = torch.cuda.Stream()
    for variant in (0, 1):
        cfg = E.ReconConfig(W, H, 3, variant=variant, **_cfgd(2))
        E.sart_projection_update_noalloc(cfg, case["pg"][1], case["vg"], vol, real, 1.0, False, stream=stream)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for variant in (0, 1):
        cfg = E.ReconConfig(W, H, 3, variant=variant, **_cfgd(2))
        for _ in range(3):
            E.sart_projection_update_noalloc(cfg, case["pg"][1], case["vg"], vol, real, 1.0, False, stream=stream)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_oversized_and_ctf():
    import artiatomi_b200 as E
    from artiatomi_b200._lib import EsbError, NOALLOC_MAX_PIXELS

    case = small_case(n_proj=2)
    vol = cuda(case["vol"])
    real = cuda(np.zeros((64, 64), np.float32))
    big = E.ReconConfig(4096, 2048, 2)
    assert 4096 * 2048 > NOALLOC_MAX_PIXELS
    with pytest.raises(EsbError, match="exceeds the scratch limit"):
        E.sart_projection_update_noalloc(big, case["pg"][0], case["vg"], vol, real)
    ctf = E.ReconConfig(64, 64, 2, ctf_mode=True)
    with pytest.raises(EsbError, match="CTF"):
        E.sart_projection_update_noalloc(ctf, case["pg"][0], case["vg"], vol, real)
    bad = E.ReconConfig(64, 64, 2, variant=7)
    with pytest.raises(EsbError, match="variant"):
        E.sart_projection_update_noalloc(bad, case["pg"][0], case["vg"], vol, real)
