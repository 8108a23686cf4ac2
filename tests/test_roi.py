"""ForwardProjectionROI (Reconstructor.cpp:1519-1529, 649-859) through
esb_rec_forward_projection_roi.

Without CTF the region's rays are exactly the whole-detector projection's
(same kernel, same rays) and nothing else is written. With CTF every slab
image is filtered over the whole detector, so a region's projection spreads
beyond it; the chain is linear in the slab images, so the projections of the
two halves of the detector add up to the whole-detector projection, and a
region covering the detector gives it bit for bit. Traversal lengths are
written for the region's rays only.
"""
import numpy as np
import pytest

from tests.helpers import cuda, host, rel_l2, small_case


def _setup(ctf):
    import artiatomi_b200 as E
    from tests.test_parity_recon import _ctf_cfg

    case = small_case(dims=(48, 40, 20), n_proj=3, W=64, H=56, shift=1.0, psi=0.2)
    W, H, n = case["W"], case["H"], len(case["tilt"])
    cfgd = dict(_ctf_cfg(max(W, H))) if ctf else {}
    defocus = np.tile(np.array([2900.0, 3100.0, 20.0], np.float32), n) if ctf else None
    rec = E.Reconstructor(E.ReconConfig(W, H, n, variant=E.VARIANT_FAST, **cfgd), case["pg"], case["tilt"], defocus)
    vol = cuda(np.ascontiguousarray(case["vol"], np.float32))
    return rec, case, vol, W, H


def _project(rec, case, vol, roi=None, empty=False):
    rec.reset_projections()
    if roi is None:
        rec.forward_projection(case["vg"], vol, 1, empty)
    else:
        rec.forward_projection_roi(case["vg"], vol, 1, roi, empty)
    p, d, _ = rec.views()
    return host(p).copy(), host(d).copy()


@pytest.mark.gpu
@pytest.mark.parametrize("empty", [False, True])
def test_roi_projection_without_ctf_is_the_region_of_the_full_one(empty):
    rec, case, vol, W, H = _setup(False)
    fp, fd = _project(rec, case, vol, empty=empty)
    roi = (9, 5, 41, 30)
    rp, rd = _project(rec, case, vol, roi, empty)
    inside = np.zeros((H, W), bool)
    inside[5:30, 9:41] = True
    np.testing.assert_array_equal(rp[inside], fp[inside])
    np.testing.assert_array_equal(rd[inside], fd[inside])
    assert not rp[~inside].any() and not rd[~inside].any()
    assert np.abs(fd[inside]).max() > 0
    # a region reaching past the detector is clipped; an empty one writes nothing
    cp, cd = _project(rec, case, vol, (-20, 30, W + 50, H + 9), empty)
    np.testing.assert_array_equal(cp[30:], fp[30:])
    np.testing.assert_array_equal(cd[30:], fd[30:])
    ep, ed = _project(rec, case, vol, (20, 20, 20, 40), empty)
    assert not ep.any() and not ed.any()


@pytest.mark.gpu
def test_roi_projection_with_ctf_adds_up_to_the_full_one():
    rec, case, vol, W, H = _setup(True)
    fp, fd = _project(rec, case, vol)
    wp, wd = _project(rec, case, vol, (0, 0, W, H))
    np.testing.assert_array_equal(wp, fp)
    np.testing.assert_array_equal(wd, fd)
    top, tdist = _project(rec, case, vol, (0, 0, W, 23))
    bottom, bdist = _project(rec, case, vol, (0, 23, W, H))
    assert np.abs(top[23:]).max() > 0  # the CTF spreads the region's signal
    assert rel_l2(top + bottom, fp) <= 1e-5, rel_l2(top + bottom, fp)
    np.testing.assert_array_equal(tdist[:23], fd[:23])
    assert not tdist[23:].any()
    np.testing.assert_array_equal(tdist + bdist, fd)
