"""Parity of the reformulated ("fast") kernels.

Forward projection: the closed-form cell sums use the reference's sample
positions without the reference's per-sample position rounding (~1e-3 voxel
jitter). Against the FP32 and FP64 oracles: rel-L2 <= 1e-4.

Back-projection: the fast kernel computes exact chords. The reference's FP32
chords carry rounding noise from ray origins 1e5 units away. On random
images a single update differs from the exact (FP64) update by 0.3-1%
rel-L2, and the FP32 oracle reproduces that noise. The fast kernel is held to
the FP64 oracle per update (rel-L2 <= 1e-5) and to both oracles on SART
volumes, the parity measure (FP32: <= 1e-3; FP64: <= 2e-4).
"""
import numpy as np
import pytest

from tests.helpers import cuda, host, rel_l2, small_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    return small_case(shift=1.5, psi=0.3)


def _orc(case, i, for_bp=False, aniso=None):
    from oracle import geometry as G

    m, mi = (None, None) if aniso is None else aniso
    return G.orc_geom(case["og"][i], case["vo"], m, mi, for_bp=for_bp)


@pytest.mark.parametrize("voxel", ["f32", "bf16"])
def test_fast_forward_projection(case, voxel):
    import torch

    import artiatomi_b200 as E
    from oracle import driver as D, lib as OL

    W, H = case["W"], case["H"]
    vol32 = case["vol"]
    if voxel == "f32":
        vol_d, vol_o, code = cuda(vol32), vol32, 0
    else:
        vol_d = cuda(vol32).to(torch.bfloat16)
        vol_o, code = np.zeros(vol32.shape, np.uint16), 2
        OL.olib.orc_float_to_bf16(OL.addr(vol32), OL.addr(vol_o), vol32.size)
    m = E.mag_aniso_matrix(1.02, 30.0, W, H)
    mi = E.mag_aniso_matrix(1.0 / 1.02, 30.0, W, H)
    for aniso in (None, (m, mi)):
        for i in range(len(case["tilt"])):
            c = E.set_constant_values(case["pg"][i], case["vg"], *(aniso or (None, None)))
            proj = torch.zeros((H, W), device="cuda")
            dist = torch.zeros((H, W), device="cuda")
            E.forward_project(c, vol_d, proj, dist, fast=True)
            for prec in (0, 1):
                po = np.zeros((H, W), np.float32)
                do = np.zeros((H, W), np.float32)
                D.fp_march(_orc(case, i, aniso=aniso), vol_o, code, W, H, po, do, precision=prec)
                e = rel_l2(host(proj), po)
                # FP32: the reference's float ray positions (start point s + t*n
                # at |t| ~ 1e4) are shared; FP64 positions differ by ~1e-3 voxel
                assert e <= (1e-4 if prec == 0 else 5e-4), (i, prec, e)
                # ray lengths: the FP32 values are the reference's (t ~ 1e4 rounds
                # to ~1e-3); FP64 lengths differ from them by that rounding
                e = rel_l2(host(dist), do)
                assert e <= (1e-6 if prec == 0 else 5e-4), (i, prec, e)


def test_fast_slicer(case):
    import torch

    import artiatomi_b200 as E
    from oracle import driver as D
    from oracle import geometry as G

    W, H = case["W"], case["H"]
    vol_d = cuda(case["vol"])
    for i in range(len(case["tilt"])):
        t0, t1 = G.defocus_distances(case["og"][i], case["vo"])
        for a, b in ((t0, t0 + 7.5), (0.5 * (t0 + t1) - 3.0, 0.5 * (t0 + t1) + 9.0), (t1 - 4.0, t1 + 20.0)):
            c = E.set_constant_values(case["pg"][i], case["vg"])
            proj = torch.zeros((H, W), device="cuda")
            E.forward_project_slab(c, vol_d, proj, a, b, fast=True)
            po = np.zeros((H, W), np.float32)
            D.fp_slicer(_orc(case, i), case["vol"], 0, W, H, po, a, b)
            e = rel_l2(host(proj), po)
            assert e <= 1e-4, (i, a, b, e)


@pytest.mark.parametrize("os_,linear,slab", [(1, False, False), (2, False, False), (2, True, True), (3, True, False)])
def test_fast_back_projection_exact_chords(case, os_, linear, slab):
    import artiatomi_b200 as E
    from oracle import driver as D
    from oracle import geometry as G

    W, H = case["W"], case["H"]
    rng = np.random.default_rng(17)
    vol0 = rng.normal(size=case["vol"].shape).astype(np.float32)
    for i in range(len(case["tilt"])):
        img = rng.normal(size=(H, W)).astype(np.float32)
        dmin, dmax = 0.0, 9999999999999.0
        if slab:
            t0, t1 = G.defocus_distances(case["og"][i], case["vo"])
            dmin, dmax = 0.5 * (t0 + t1) - 8.0, 0.5 * (t0 + t1) + 8.0
        v_d = cuda(vol0)
        E.back_project(E.set_constant_values(case["pg"][i], case["vg"], for_bp=True), v_d, cuda(img), 0.37, os_, dmin,
                       dmax, linear, fast=True)
        vo = vol0.copy()
        D.bp(_orc(case, i, for_bp=True), vo, 0, img, 0.37, os_, dmin, dmax, int(linear), precision=1)
        e = rel_l2(host(v_d) - vol0, vo - vol0)
        # the sub-pixel grid is the reference's float recurrence from the
        # quad's macro-cell corner (exact lattice for power-of-two OS only)
        assert e <= 1e-5, (i, e)


@pytest.mark.parametrize("sirt,os_,aniso", [(1, 1, False), (3, 2, False), (2, 3, False), (3, 2, True)])
def test_fast_sart_volume(sirt, os_, aniso):
    """FAST SART against the oracle (FP32 1e-3, FP64 2e-4). Oversampling 3
    and magnification anisotropy take the back-projector that filters the
    residual itself (no pre-sampled images)."""
    import artiatomi_b200 as E
    from oracle.driver import OracleReconstructor
    from tests.test_parity_recon import _projections

    case = small_case(n_proj=9, shift=1.0, psi=0.2)
    W, H = case["W"], case["H"]
    projs = _projections(case)
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
    cfgd = dict(lambda_=0.5, oversampling=os_, cut_length=(1.0, 1.0), dim_length=(3.0, 3.0),
                crop=(1.0, 2.0, 1.0, 2.0), crop_dim=(3.0, 3.0, 3.0, 3.0))
    m = mi = None
    if aniso:
        m, mi = E.mag_aniso_matrix(1.03, 25.0, W, H), E.mag_aniso_matrix(1.0 / 1.03, 25.0, W, H)
    rec = E.Reconstructor(E.ReconConfig(W, H, len(case["tilt"]), variant=E.VARIANT_FAST, **cfgd), case["pg"],
                          case["tilt"], None, m, mi)
    vol_d = cuda(np.zeros(case["vol"].shape, np.float32))
    rec.sart(case["vg"], vol_d, cuda(projs), il, iterations=2, sirt_count=sirt)
    got = host(vol_d)
    for prec, tol in ((0, 1e-3), (1, 2e-4)):
        orc = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], aniso=m, aniso_inv=mi, precision=prec)
        vo = np.zeros(case["vol"].shape, np.float32)
        orc.sart(case["vo"], vo, 0, projs, il, 2, sirt)
        e = rel_l2(got, vo)
        assert e <= tol, (prec, e)


def _defocus(n, seed):
    rng = np.random.default_rng(seed)
    d = np.stack([rng.uniform(2900, 3100, n), rng.uniform(3100, 3200, n), rng.uniform(0, 180, n)], 1)
    return d.astype(np.float32).ravel()


def test_fast_ctf_forward_and_back_projection():
    """Fused multi-slab slicer + per-slab CTF, and the fused slab back-projection."""
    import artiatomi_b200 as E
    from oracle.driver import OracleReconstructor
    from tests.test_parity_recon import _ctf_cfg

    case = small_case(dims=(64, 64, 24), n_proj=5, shift=1.0)
    W, H = case["W"], case["H"]
    n = len(case["tilt"])
    defocus = _defocus(n, 5)
    cfgd = _ctf_cfg(W)
    rec = E.Reconstructor(E.ReconConfig(W, H, n, variant=E.VARIANT_FAST, **cfgd), case["pg"], case["tilt"], defocus)
    vol_d = cuda(case["vol"])
    proj_v, dist_v, _ = rec.views()
    for prec in (0, 1):
        orc = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], defocus, precision=prec)
        for i in range(n):
            rec.reset_projections()
            rec.forward_projection(case["vg"], vol_d, i, False)
            orc.reset()
            orc.forward_projection(case["vo"], case["vol"], 0, i, False)
            e = rel_l2(host(proj_v), orc.proj)
            assert e <= 1e-4, (prec, i, e)
    rng = np.random.default_rng(6)
    vol_b = cuda(np.zeros(case["vol"].shape, np.float32))
    vo = np.zeros(case["vol"].shape, np.float32)
    orc = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], defocus, precision=1)
    for i in range(n):
        res = rng.normal(size=(H, W)).astype(np.float32)
        proj_v.copy_(cuda(res))
        rec.back_projection(case["vg"], vol_b, i, 2.0)
        orc.back_projection(case["vo"], vo, 0, i, 2.0, img=res.copy())
    e = rel_l2(host(vol_b), vo)
    assert e <= 1e-4, e


def test_fast_sart_ctf():
    import artiatomi_b200 as E
    from oracle.driver import OracleReconstructor
    from tests.test_parity_recon import _ctf_cfg, _projections

    case = small_case(dims=(64, 64, 24), n_proj=5, shift=0.5)
    W, H = case["W"], case["H"]
    n = len(case["tilt"])
    defocus = _defocus(n, 15)
    projs = _projections(case)
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
    cfgd = dict(_ctf_cfg(W), lambda_=0.5, oversampling=2)
    rec = E.Reconstructor(E.ReconConfig(W, H, n, variant=E.VARIANT_FAST, **cfgd), case["pg"], case["tilt"], defocus)
    vol_d = cuda(np.zeros(case["vol"].shape, np.float32))
    rec.sart(case["vg"], vol_d, cuda(projs), il, iterations=2, sirt_count=2)
    got = host(vol_d)
    for prec, tol in ((0, 1e-3), (1, 2e-4)):
        orc = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], defocus, precision=prec)
        vo = np.zeros(case["vol"].shape, np.float32)
        orc.sart(case["vo"], vo, 0, projs, il, 2, 2)
        e = rel_l2(got, vo)
        assert e <= tol, (prec, e)


def _subvolume_case(ctf, sizes, n=7, seed=31, psi_deg=0.0):
    import artiatomi_b200 as E
    from artiatomi_b200 import _lib as L
    from oracle import geometry as G

    W = H = 96
    tilt = np.linspace(-60, 60, n).astype(np.float32)
    psi = np.full(n, psi_deg, np.float32)
    rng = np.random.default_rng(seed)
    projs = rng.normal(size=(n, H, W)).astype(np.float32)
    full, fo = E.volume_geometry((96, 96, 40)), G.volume_geometry((96, 96, 40))
    pos = rng.uniform(20, 76, size=(len(sizes), 3))
    pos[:, 2] = rng.uniform(10, 30, len(sizes))
    shifts = rng.uniform(-1.5, 1.5, size=(len(sizes), n, 2)).astype(np.float32)
    sub = [E.subvolume_geometry(s, 1.0, full, p) for s, p in zip(sizes, pos)]
    subo = [G.subvolume_geometry(s, 1.0, fo, p) for s, p in zip(sizes, pos)]
    pair = (L.ProjGeom * (len(sizes) * n))()
    pair_o = []
    for p in range(len(sizes)):
        g = E.projection_geometry(E.Markers(tilt, rotation_psi=psi), W, H, extra_shift=shifts[p])
        for i in range(n):
            pair[p * n + i] = g[i]
        pair_o.append(G.projection_geometry(tilt, psi=psi, width=W, height=H, extra_shift=shifts[p]))
    defocus = np.stack([np.full(n, 3000.0), np.full(n, 3100.0), np.full(n, 20.0)], 1).astype(np.float32).ravel()
    cfgd = dict(oversampling=2, ctf_mode=ctf, pixel_size_nm=0.27, ctf_slice_thickness_nm=4.0,
                ctf_beta_fac=(10.0, 0.0, 0.008, 0.0))
    return dict(W=W, H=H, n=n, tilt=tilt, psi=psi, projs=projs, full=full, fo=fo, sub=sub, subo=subo, pair=pair,
                pair_o=pair_o, defocus=defocus if ctf else None, cfgd=cfgd, shifts=shifts, sizes=sizes)


def _subvolume_gpu(c, batched, index_list, active=None, patches=None):
    import artiatomi_b200 as E

    W, H, n = c["W"], c["H"], c["n"]
    pg = E.projection_geometry(E.Markers(c["tilt"], rotation_psi=c["psi"]), W, H)
    rec = E.Reconstructor(E.ReconConfig(W, H, n, variant=E.VARIANT_FAST, **c["cfgd"]), pg, c["tilt"], c["defocus"])
    if patches is not None:
        rec.subvolume_patches(patches)
    boxes = [cuda(np.zeros((s, s, s), np.float32)) for s in c["sizes"]]
    rec.subvolume_wbp(c["full"], c["sub"], c["pair"], boxes, cuda(c["projs"]), index_list, active=active,
                      batched=batched)
    return [host(b) for b in boxes]


def _subvolume_oracle(c, index_list, active=None, precision=1):
    from oracle import geometry as G
    from oracle.driver import OracleReconstructor

    W, H = c["W"], c["H"]
    orc = OracleReconstructor(c["cfgd"], W, H, G.projection_geometry(c["tilt"], psi=c["psi"], width=W, height=H),
                              c["tilt"], c["defocus"], precision=precision)
    bo = [np.zeros((s, s, s), np.float32) for s in c["sizes"]]
    orc.subvolume_wbp(c["fo"], c["subo"], c["pair_o"], bo, c["projs"], index_list, active=active)
    return bo


@pytest.mark.parametrize("ctf,batched", [(False, False), (True, False), (False, True), (True, True)])
def test_fast_subvolume_wbp(ctf, batched):
    c = _subvolume_case(ctf, [16, 24, 16, 32])
    il = np.arange(c["n"], dtype=np.int32)
    got = _subvolume_gpu(c, batched, il)
    for b, o in zip(got, _subvolume_oracle(c, il)):
        e = rel_l2(b, o)
        assert e <= 1e-4, e


@pytest.mark.parametrize("ctf", [False, True])
def test_batched_subvolume_matches_per_particle(ctf):
    """One persistent launch over mixed boxes matches one launch per particle
    per tilt: the same per-voxel sums added in the same order (tilts in list
    order, inactive pairs skipped). The two kernels are compiled separately
    and may contract multiply-adds differently, so agreement is to float
    rounding, not bit-exact."""
    c = _subvolume_case(ctf, [16, 24, 32, 48, 16, 24], n=9, seed=5)
    il = np.random.default_rng(1).permutation(c["n"]).astype(np.int32)
    active = (np.linalg.norm(c["shifts"], axis=2) < 1.5).astype(np.uint8)
    plain = _subvolume_gpu(c, False, il, active)
    batch = _subvolume_gpu(c, True, il, active)
    for a, b in zip(plain, batch):
        assert np.abs(a).sum() > 0
        assert rel_l2(b, a) <= 1e-5
        assert np.abs(b - a).max() <= 1e-5 * np.abs(a).max()
    # Against the FP64 oracle: 1e-4 without CTF. With CTF a quad takes the
    # slab of its first corner's depth, computed in float here as in the
    # reference and in double by the FP64 oracle; quads on a slab boundary
    # then read different slab images (the reference's own float result is
    # 2-3e-3 from the FP64 oracle on this case), so the bar is the 1e-3 of a
    # reference-parity result.
    tol = 1e-3 if ctf else 1e-4
    for b, o in zip(batch, _subvolume_oracle(c, il, active)):
        assert rel_l2(b, o) <= tol


@pytest.mark.parametrize("psi_deg", [0.0, 0.7])
def test_subvolume_ctf_patches_match_per_tilt(psi_deg):
    """With CTF the batched call gathers, after each tilt's CTF chain, the
    patch of the slab images each box reads, and adds all tilts in one
    launch (esb_reconstructor_subvolume_patches). One launch per tilt over
    the whole slab images gives the same boxes bit for bit: the same sums in
    the same order, patch texels equal to the clamped image texels (boxes
    here reach past the detector edge). 4 nm slabs: boxes span several."""
    c = _subvolume_case(True, [16, 24, 32, 48, 16, 24], n=9, seed=5, psi_deg=psi_deg)
    il = np.random.default_rng(1).permutation(c["n"]).astype(np.int32)
    active = (np.linalg.norm(c["shifts"], axis=2) < 1.5).astype(np.uint8)
    one = _subvolume_gpu(c, True, il, active, patches=True)
    per_tilt = _subvolume_gpu(c, True, il, active, patches=False)
    for a, b in zip(per_tilt, one):
        assert np.abs(a).sum() > 0
        np.testing.assert_array_equal(b, a)


def test_batched_subvolume_ragged_box_runs_per_particle():
    """A box whose x extent is not a multiple of 4 cannot take the batched
    kernel's float4 layout; the call then runs the per-particle launches."""
    c = _subvolume_case(False, [16, 18, 24], n=5, seed=8)
    il = np.arange(c["n"], dtype=np.int32)
    got = _subvolume_gpu(c, True, il)
    for b, o in zip(got, _subvolume_oracle(c, il)):
        assert rel_l2(b, o) <= 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("ctf", [False, True])
def test_sart_graph_replay_equals_eager(ctf):
    """esb_sart_run with CUDA graphs (iteration 1 eager, 2 captured, 3.. replayed)
    gives the eager result bit for bit: the same kernels run in the same order."""
    import artiatomi_b200 as E
    from tests.test_parity_recon import _ctf_cfg, _projections

    case = small_case(dims=(64, 64, 24), n_proj=5, shift=0.5)
    W, H = case["W"], case["H"]
    n = len(case["tilt"])
    defocus = _defocus(n, 15) if ctf else None
    projs = cuda(_projections(case))
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
    cfgd = dict(_ctf_cfg(W), lambda_=0.5, oversampling=2) if ctf else dict(lambda_=0.5, oversampling=2)
    vols = []
    for graphs in (False, True):
        rec = E.Reconstructor(E.ReconConfig(W, H, n, variant=E.VARIANT_FAST, **cfgd), case["pg"], case["tilt"], defocus)
        rec.enable_graphs(graphs)
        v = cuda(np.zeros(case["vol"].shape, np.float32))
        rec.sart(case["vg"], v, projs, il, iterations=4, sirt_count=2)
        vols.append(host(v))
        rec.close()
    assert np.abs(vols[0]).max() > 0
    np.testing.assert_array_equal(vols[1], vols[0])
