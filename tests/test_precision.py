"""Reduced-precision volume storage (FP16, BF16) with FP32 arithmetic.

SART (fast kernels, 3 iterations) with the volume stored as FP32, FP16 or
BF16, against the FP64 oracle on the same inputs. Every back-projection
store rounds to nearest; the error grows with the storage format's unit in
the last place (FP16 2^-11, BF16 2^-8 relative), because updates smaller
than half of it are dropped.
"""
import numpy as np
import pytest

from tests.helpers import cuda, rel_l2, small_case


@pytest.mark.gpu
def test_storage_precision_against_fp64():
    import torch

    import artiatomi_b200 as E
    from oracle.driver import OracleReconstructor
    from tests.test_parity_recon import _projections

    case = small_case(dims=(64, 64, 32), n_proj=9, shift=1.0, psi=0.2)
    W, H = case["W"], case["H"]
    projs = _projections(case)
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
    cfgd = dict(lambda_=0.5, oversampling=2)
    orc = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], precision=1)
    ref = np.zeros(case["vol"].shape, np.float32)
    orc.sart(case["vo"], ref, 0, projs, il, 3, 2)
    p_d = cuda(projs)
    errs = {}
    for name, dt in (("f32", torch.float32), ("f16", torch.float16), ("bf16", torch.bfloat16)):
        rec = E.Reconstructor(E.ReconConfig(W, H, len(case["tilt"]), variant=E.VARIANT_FAST, **cfgd), case["pg"],
                              case["tilt"])
        v = torch.zeros(case["vol"].shape, dtype=dt, device="cuda")
        rec.sart(case["vg"], v, p_d, il, iterations=3, sirt_count=2)
        torch.cuda.synchronize()
        errs[name] = rel_l2(v.float().cpu().numpy(), ref)
        rec.close()
    # measured on B200: f32 1.6e-4, f16 8.0e-4, bf16 6.2e-3
    assert errs["f32"] <= 2e-4, errs
    assert errs["f16"] <= 1.5e-3, errs
    assert errs["bf16"] <= 1.2e-2, errs
