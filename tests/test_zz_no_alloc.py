"""The SART projection update that allocates no device memory
(esb_sart_projection_update_noalloc) against the reconstructor path that
owns cudaMalloc'd buffers.

The no-allocation entry point exists for callers that cannot call
cudaMalloc: an application whose device memory is owned and budgeted by its
own allocator, a process that must not allocate after start-up, or a loop
that must not pay cudaMalloc's implicit synchronisation. Its scratch lives in
a fixed array inside the library, shared by every call and keeping the last
call's contents. Two calls in a row must therefore give the same volumes as
two reconstructor steps. The first call uses volume_is_empty (traversal
length only), the second the full forward projection. Both paths run the same
kernels, so the tolerance is the faithful-kernel bar of the other tests
(rel-L2 <= 1e-5, in practice bit-exact).

This file is collected last so that a failure here comes after every other
test has run.
"""
import numpy as np
import pytest

from tests.helpers import cuda, host, rel_l2, small_case

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.mark.parametrize("os_", [1, 2])
def test_noalloc_update_matches_reconstructor_twice(os_):
    import torch

    import artiatomi_b200 as E

    case = small_case(n_proj=5, shift=1.0, psi=0.2)
    W, H = case["W"], case["H"]
    rng = np.random.default_rng(40 + os_)
    real = rng.normal(size=(len(case["tilt"]), H, W)).astype(np.float32) * 10
    real_d = cuda(real)
    cfg = E.ReconConfig(W, H, len(case["tilt"]), lambda_=0.5, oversampling=os_, cut_length=(1.0, 1.0),
                        dim_length=(3.0, 3.0), crop=(1.0, 2.0, 1.0, 2.0), crop_dim=(3.0, 3.0, 3.0, 3.0))
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
