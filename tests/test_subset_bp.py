"""The back-projection of an ordered subset in one volume pass
(esb_reconstructor_fuse_subsets, k_bp_axis_set) against one pass per
projection (EmSart.cpp:649-673: SIRTCount back-projections, each adding its
update to the volume).

FP32 volumes: bit for bit equal, with CTF slabs and without, for full and
partial last subsets, and fewer kernel launches. FP16 volumes: the subset's
updates are summed in float and rounded once, so the volume is at least as
close to the FP64 oracle as with a rounding per projection.
"""
import numpy as np
import pytest

from tests.helpers import cuda, host, rel_l2, small_case

pytestmark = pytest.mark.gpu


def _run(ctf, os_, sirt, fuse, n_proj=7, dtype=np.float32, iterations=2):
    import torch

    import artiatomi_b200 as E
    from tests.test_parity_fast import _defocus
    from tests.test_parity_recon import _ctf_cfg, _projections

    case = small_case(dims=(64, 64, 24), n_proj=n_proj, shift=0.5, psi=0.2)
    W, H = case["W"], case["H"]
    n = len(case["tilt"])
    defocus = _defocus(n, 15) if ctf else None
    projs = _projections(case)
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
    cfgd = dict(_ctf_cfg(W), lambda_=0.5, oversampling=os_) if ctf else dict(lambda_=0.5, oversampling=os_)
    rec = E.Reconstructor(E.ReconConfig(W, H, n, variant=E.VARIANT_FAST, **cfgd), case["pg"], case["tilt"], defocus)
    rec.fuse_subsets(fuse)
    v = torch.zeros(case["vol"].shape, dtype=torch.float16 if dtype == np.float16 else torch.float32, device="cuda")
    l0 = E.kernel_launches()
    rec.sart(case["vg"], v, cuda(projs), il, iterations=iterations, sirt_count=sirt)
    torch.cuda.synchronize()
    launches = E.kernel_launches() - l0
    rec.close()
    return host(v.float()), launches, (case, cfgd, projs, il, defocus)


@pytest.mark.parametrize("ctf,os_,sirt,n_proj", [(False, 1, 3, 7), (False, 2, 4, 7), (True, 2, 2, 5), (True, 2, 3, 5)])
def test_subset_pass_equals_per_projection(ctf, os_, sirt, n_proj):
    _run(ctf, os_, sirt, True, n_proj, iterations=1)  # launch shapes tuned and cached before counting
    fused, lf, _ = _run(ctf, os_, sirt, True, n_proj)
    sep, ls, _ = _run(ctf, os_, sirt, False, n_proj)
    assert np.abs(sep).max() > 0
    np.testing.assert_array_equal(fused, sep)
    # one back-projection launch per subset instead of one per projection
    subsets = (n_proj + sirt - 1) // sirt
    assert ls - lf == 2 * (n_proj - subsets), (ls, lf)


def test_subset_pass_fp16_rounds_once():
    from oracle.driver import OracleReconstructor

    fused, _, (case, cfgd, projs, il, defocus) = _run(True, 2, 5, True, n_proj=5, dtype=np.float16, iterations=3)
    sep, _, _ = _run(True, 2, 5, False, n_proj=5, dtype=np.float16, iterations=3)
    orc = OracleReconstructor(cfgd, case["W"], case["H"], case["og"], case["tilt"], defocus, precision=1)
    vo = np.zeros(case["vol"].shape, np.float32)
    orc.sart(case["vo"], vo, 0, projs, il, 3, 5)
    e_fused, e_sep = rel_l2(fused, vo), rel_l2(sep, vo)
    print(f"FP16 volume vs FP64 oracle: one rounding per subset {e_fused:.3e}, per projection {e_sep:.3e}")
    assert e_fused <= e_sep
