"""Host geometry of libesb (C++) against the oracle's numpy restatement of
Projection.cpp / Volume.cpp / Reconstructor.cpp helpers: bit-exact."""
import numpy as np
import pytest

import artiatomi_b200 as E
from oracle import geometry as G


def _markers(n, seed=0):
    rng = np.random.default_rng(seed)
    tilt = np.linspace(-60, 60, n).astype(np.float32)
    xs = rng.uniform(-3, 3, n).astype(np.float32)
    ys = rng.uniform(-3, 3, n).astype(np.float32)
    mag = rng.uniform(0.95, 1.05, n).astype(np.float32)
    psi = rng.uniform(-1, 1, n).astype(np.float32)
    return tilt, xs, ys, mag, psi


@pytest.mark.parametrize("cfg", [dict(), dict(add_tilt_angle=1.5, phi_angle=2.0, add_tilt_x_angle=0.7),
                                 dict(use_fix_psi_angle=True, psi_angle=10.0)])
def test_projection_geometry_bit_exact(cfg):
    tilt, xs, ys, mag, psi = _markers(13)
    es = np.random.default_rng(5).uniform(-2, 2, (13, 2)).astype(np.float32)
    tc = E.TiltConfig(**cfg)
    pg = E.projection_geometry(E.Markers(tilt, xs, ys, mag, psi), 200, 160, tc, extra_shift=es)
    og = G.projection_geometry(tilt, xs, ys, mag, psi, 200, 160, cfg, extra_shift=es)
    for a, b in zip(og, pg):
        for k, kk in (("det", "detektor"), ("u", "u_pitch"), ("v", "v_pitch"), ("n", "proj_norm"),
                      ("detMat", "detector_matrix")):
            np.testing.assert_array_equal(np.asarray(a[k], np.float32), np.array(list(getattr(b, kk)), np.float32))


def test_detector_matrix_inverts_frame():
    tilt, xs, ys, mag, psi = _markers(7)
    for g in G.projection_geometry(tilt, xs, ys, mag, psi, 128, 96):
        M = np.asarray(g["detMat"], np.float64).reshape(4, 4)
        for px, py in ((0.0, 0.0), (10.5, 3.25), (127.0, 95.0)):
            p = g["det"].astype(np.float64) + px * g["u"] + py * g["v"] + 7.0 * g["n"]
            q = M[:3, :3] @ p + M[:3, 3]
            np.testing.assert_allclose(q, [px, py, 7.0], atol=2e-3)


@pytest.mark.parametrize("count,part", [(1, 0), (3, 0), (3, 2), (4, 1)])
def test_volume_geometry_bit_exact(count, part):
    dims = (96, 80, 50)
    vs, sh = (1.5, 1.5, 1.5), (2.0, -3.0, 4.5)
    a = E.volume_geometry(dims, vs, sh, count, part)
    b = G.volume_geometry(dims, vs, sh, count, part)
    np.testing.assert_array_equal(np.array(a.bbox_min[:]), b.bbMin)
    np.testing.assert_array_equal(np.array(a.bbox_max[:]), b.bbMax)
    np.testing.assert_array_equal(np.array(a.bbox_rcp[:]), b.bbRcp)
    np.testing.assert_array_equal(np.array(a.dim[:]), b.dim)
    assert a.z_shift == b.zShift
    np.testing.assert_array_equal(np.array(a.full_bbox_min[:]), b.full_min)


def test_subvolume_geometry_bit_exact():
    full = E.volume_geometry((400, 400, 100), (2, 2, 2))
    fo = G.volume_geometry((400, 400, 100), (2, 2, 2))
    for pos, sh in (((100, 120, 50), (0.5, -1.0, 2.0)), ((1, 1, 1), (0, 0, 0))):
        a = E.subvolume_geometry(48, 1.0, full, pos, sh)
        b = G.subvolume_geometry(48, 1.0, fo, pos, sh)
        np.testing.assert_array_equal(np.array(a.bbox_min[:]), b.bbMin)
        np.testing.assert_array_equal(np.array(a.bbox_max[:]), b.bbMax)


def test_hit_points_and_defocus_distances():
    tilt, xs, ys, mag, psi = _markers(9)
    pg = E.projection_geometry(E.Markers(tilt, xs, ys, mag, psi), 256, 256)
    og = G.projection_geometry(tilt, xs, ys, mag, psi, 256, 256)
    vg, vo = E.volume_geometry((256, 256, 64)), G.volume_geometry((256, 256, 64))
    for a, b in zip(pg, og):
        assert list(E.compute_hit_points(a, vg)) == G.compute_hit_points(b, vo)
        assert E.defocus_distances(a, vg, 256, 256) == pytest.approx(G.defocus_distances(b, vo), abs=0)


def test_defocus_min_max():
    import ctypes as C
    from artiatomi_b200._lib import lib

    for ray, ign, sw in ((9850.3, 0, 0), (10123.7, 1, 0), (10003.0, 0, 1)):
        a, b = C.c_float(), C.c_float()
        lib.esb_defocus_min_max(ray, 3000.0, 3100.0, 30.0, 0.5, 0.27, 30.0, 2.0, ign, sw, C.byref(a), C.byref(b))
        ea, eb = G.defocus_min_max(ray, 3000.0, 3100.0, 30.0, 0.5, 0.27, 30.0, 2.0, bool(ign), bool(sw))
        assert (a.value, b.value) == pytest.approx((ea, eb), rel=1e-6)


def test_mag_aniso_matrix():
    a = E.mag_aniso_matrix(1.02, 35.0, 512, 400)
    b = G.mag_aniso(1.02, 35.0, 512, 400)
    np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-4)
    np.testing.assert_array_equal(E.mag_aniso_matrix(1.0, 0.0, 64, 64), np.eye(3, dtype=np.float32).ravel())


def test_projection_index_list_matches_reference_order():
    tilt = np.linspace(-60, 60, 41).astype(np.float32)
    a = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, tilt)
    b = G.index_list_random_start_zero(tilt)
    np.testing.assert_array_equal(a, b)
    assert a[0] == 20 and sorted(a) == list(range(41))
    good = np.ones(41, np.int32)
    good[[3, 7]] = 0
    c = E.projection_index_list(E.PLT_NORMAL, tilt, good)
    assert list(c) == [i for i in range(41) if i not in (3, 7)]
