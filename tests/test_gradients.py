"""Adjoint and gradients of the projection model (differentiation).

The model is the fast projector's projection A(x) with a per-tilt detector
offset s in pixels applied as a rigid in-plane translation of the samples
(`esb_projection_loss_grad`, `esb_fp_adjoint`; `orc_model_loss_grad` is its
FP64 CPU counterpart). Checks:

* the FP64 oracle's gradient against central finite differences of its own
  loss (CPU);
* the dot-product test <A x, y> = <x, A^T y> on the GPU (1e-5 of <A x, y>
  for y correlated with A x, of |A x| |y| for independent y);
* the GPU loss, volume gradient, shift gradient and Gauss-Newton terms
  against the FP64 oracle;
* central finite differences (h = 1e-3) on 64 random voxels and on all
  shifts against the GPU gradient;
* 20 Gauss-Newton steps of shift refinement recovering injected shifts to
  < 0.1 px;
* a torch.autograd.Function (test harness only) whose backward is the
  adjoint gives the same volume gradient as the fused loss kernel.
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import cuda, host, rel_l2, small_case

MAG = np.array([1.004, 0.003, 0.0, -0.002, 0.997, 0.0, 0.0, 0.0, 1.0], np.float32)


def _case(dims=(40, 36, 20), n_proj=5, W=40, H=40, seed=5, **kw):
    return small_case(dims=dims, n_proj=n_proj, W=W, H=H, seed=seed, n_ell=12, shift=1.5, psi=0.4, **kw)


def _oracle_loss(case, i, vol, meas, shift, grad=True, mag=None):
    from oracle import geometry as G
    from oracle.lib import NTHREADS, addr, olib

    g = G.orc_geom(case["og"][i], case["vo"], *((mag, np.linalg.inv(mag.reshape(3, 3)).ravel().astype(np.float32))
                                                if mag is not None else (None, None)))
    W, H = case["W"], case["H"]
    out = np.zeros(6, np.float64)
    gv = np.zeros(vol.shape, np.float64) if grad else None
    proj = np.zeros((H, W), np.float32)
    olib.orc_model_loss_grad(C.byref(g), addr(np.ascontiguousarray(vol, np.float32)), W, H,
                             None if meas is None else addr(np.ascontiguousarray(meas, np.float32)),
                             float(shift[0]), float(shift[1]), None if gv is None else addr(gv), addr(proj),
                             addr(out), NTHREADS)
    return out, gv, proj


# ------------------------------------------------------------------ CPU
def test_oracle_gradient_matches_finite_differences():
    case = _case()
    rng = np.random.default_rng(0)
    x = case["vol"].astype(np.float64)
    meas = rng.normal(size=(case["H"], case["W"])).astype(np.float32) * 5
    shift = (0.37, -0.61)
    for i in (0, 2, 4):
        out, gv, _ = _oracle_loss(case, i, x, meas, shift)
        # volume: L is quadratic in x, central differences are exact up to rounding
        idx = rng.choice(x.size, 8, replace=False)
        for k in idx:
            xp, xm = x.copy(), x.copy()
            h = 1e-3
            xp.flat[k] += h
            xm.flat[k] -= h
            lp = _oracle_loss(case, i, xp, meas, shift, grad=False)[0][0]
            lm = _oracle_loss(case, i, xm, meas, shift, grad=False)[0][0]
            fd = (lp - lm) / (2 * h)
            assert abs(fd - gv.flat[k]) <= 1e-4 * max(1.0, abs(gv.flat[k])), (i, k, fd, gv.flat[k])
        # shifts
        for a in (0, 1):
            h = 1e-4
            sp, sm = list(shift), list(shift)
            sp[a] += h
            sm[a] -= h
            fd = (_oracle_loss(case, i, x, meas, sp, grad=False)[0][0] -
                  _oracle_loss(case, i, x, meas, sm, grad=False)[0][0]) / (2 * h)
            assert abs(fd - out[1 + a]) <= 1e-3 * max(1.0, abs(out[1 + a])), (i, a, fd, out[1 + a])


def test_oracle_adjoint_dot_product():
    case = _case()
    rng = np.random.default_rng(1)
    x = rng.normal(size=case["vol"].shape).astype(np.float32)
    y = rng.normal(size=(case["H"], case["W"])).astype(np.float32)
    for i in range(len(case["tilt"])):
        _, _, ax = _oracle_loss(case, i, x, None, (0.2, -0.3), grad=False)
        # residual A x - (A x - y) = y: the volume gradient is A^T y
        _, aty, _ = _oracle_loss(case, i, x, ax - y, (0.2, -0.3))
        lhs = float(np.dot(ax.ravel().astype(np.float64), y.ravel()))
        rhs = float(np.dot(x.ravel().astype(np.float64), aty.ravel()))
        # y enters through float images (A x and A x - y are rounded to
        # float), hence the 1e-5 bar rather than double precision
        assert abs(lhs - rhs) <= 1e-5 * abs(lhs), (i, lhs, rhs)


# ------------------------------------------------------------------ GPU
def _consts(case, i, mag=None):
    import artiatomi_b200 as E

    if mag is None:
        return E.set_constant_values(case["pg"][i], case["vg"])
    return E.set_constant_values(case["pg"][i], case["vg"], mag, np.linalg.inv(mag.reshape(3, 3)).ravel())


def _gpu_loss(case, i, vol_d, meas, shift, grad_d=None, proj_d=None, mag=None):
    import torch

    import artiatomi_b200 as E

    out = torch.zeros(6, dtype=torch.float64, device="cuda")
    E.projection_loss_grad(_consts(case, i, mag), vol_d, meas, out, shift=shift, grad=grad_d, proj_out=proj_d,
                           width=case["W"], height=case["H"])
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("mag", [None, MAG])
def test_adjoint_dot_product(mag):
    import torch

    import artiatomi_b200 as E

    case = _case(n_proj=7)
    rng = np.random.default_rng(2)
    x = cuda(rng.normal(size=case["vol"].shape).astype(np.float32))
    W, H = case["W"], case["H"]
    for i in range(len(case["tilt"])):
        c = _consts(case, i, mag)
        for shift in ((0.0, 0.0), (0.8, -1.3)):
            ax = torch.zeros((H, W), device="cuda")
            if shift == (0.0, 0.0):
                E.forward_project(c, x, ax, torch.zeros_like(ax), fast=True)
            else:
                _gpu_loss(case, i, x, None, shift, proj_d=ax, mag=mag)
            # y correlated with A x (a well-conditioned <A x, y>, bar relative
            # to it) and y independent of it (bar relative to |A x| |y|, the
            # scale of the terms of the sum)
            y1 = ax + cuda(rng.normal(size=(H, W)).astype(np.float32)) * float(ax.std())
            y2 = cuda(rng.normal(size=(H, W)).astype(np.float32))
            for y, independent in ((y1, False), (y2, True)):
                aty = torch.zeros_like(x)
                E.fp_adjoint(c, aty, y, shift=shift)
                lhs = float((ax.double() * y.double()).sum())
                rhs = float((x.double() * aty.double()).sum())
                ref = float(ax.double().norm() * y.double().norm()) if independent else abs(lhs)
                assert abs(lhs - rhs) <= 1e-5 * ref, (i, shift, independent, lhs, rhs)


@pytest.mark.gpu
def test_zero_shift_model_equals_fast_projector():
    import torch

    import artiatomi_b200 as E

    case = _case()
    x = cuda(case["vol"])
    for i in range(len(case["tilt"])):
        a = torch.zeros((case["H"], case["W"]), device="cuda")
        E.forward_project(_consts(case, i), x, a, torch.zeros_like(a), fast=True)
        b = torch.zeros_like(a)
        _gpu_loss(case, i, x, None, (0.0, 0.0), proj_d=b)
        assert rel_l2(host(b), host(a)) <= 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("mag", [None, MAG])
def test_loss_grad_matches_fp64_oracle(mag):
    import torch

    case = _case()
    rng = np.random.default_rng(3)
    meas = (rng.normal(size=(case["H"], case["W"])) * 5).astype(np.float32)
    x = case["vol"]
    gsum = torch.zeros(x.shape, device="cuda")
    osum = np.zeros(6)
    g64 = np.zeros(x.shape)
    o64 = np.zeros(6)
    for i in range(len(case["tilt"])):
        shift = (0.3 * i - 0.5, 0.7 - 0.2 * i)
        osum += _gpu_loss(case, i, cuda(x), cuda(meas), shift, grad_d=gsum, mag=mag)
        o, g, _ = _oracle_loss(case, i, x, meas, shift, mag=mag)
        o64 += o
        g64 += g
    assert abs(osum[0] - o64[0]) <= 1e-5 * abs(o64[0])
    assert rel_l2(host(gsum), g64) <= 1e-4
    # dL/ds = sum r dp/ds has random-sign terms: its bar is relative to the
    # Cauchy-Schwarz scale sqrt(sum r^2 sum (dp/ds)^2); the Gauss-Newton sums
    # relative to themselves (or to sqrt(Huu Hvv) for the cross term)
    L, Huu, Huv, Hvv = o64[0], o64[3], o64[4], o64[5]
    scale = [None, np.sqrt(2 * L * Huu), np.sqrt(2 * L * Hvv), Huu, np.sqrt(Huu * Hvv), Hvv]
    for k in range(1, 6):
        assert abs(osum[k] - o64[k]) <= 1e-4 * scale[k], (k, osum[k], o64[k], scale[k])


@pytest.mark.gpu
def test_loss_grad_finite_differences():
    import torch

    case = _case()
    rng = np.random.default_rng(4)
    meas = (rng.normal(size=(case["H"], case["W"])) * 5).astype(np.float32)
    x = case["vol"].astype(np.float32)
    m_d = cuda(meas)
    for i in (0, 2, 4):
        shift = (0.41, -0.23)
        grad = torch.zeros(x.shape, device="cuda")
        out = _gpu_loss(case, i, cuda(x), m_d, shift, grad_d=grad)
        g = host(grad)
        idx = rng.choice(x.size, 64, replace=False)
        h = 1e-3
        scale = np.sqrt(np.mean(g.ravel()[idx] ** 2)) + 1e-12
        for k in idx:
            xp, xm = x.copy(), x.copy()
            xp.flat[k] += h
            xm.flat[k] -= h
            fd = (_gpu_loss(case, i, cuda(xp), m_d, shift)[0] - _gpu_loss(case, i, cuda(xm), m_d, shift)[0]) / (2 * h)
            assert abs(fd - g.flat[k]) <= 2e-2 * max(scale, abs(g.flat[k])), (i, k, fd, g.flat[k])
        x_d = cuda(x)
        for a in (0, 1):
            sp, sm = list(shift), list(shift)
            sp[a] += h
            sm[a] -= h
            fd = (_gpu_loss(case, i, x_d, m_d, sp)[0] - _gpu_loss(case, i, x_d, m_d, sm)[0]) / (2 * h)
            assert abs(fd - out[1 + a]) <= 1e-2 * max(abs(out[1 + a]), 1e-3 * out[0]), (i, a, fd, out[1 + a])


@pytest.mark.gpu
def test_shift_refinement_recovers_injected_shifts():
    """20 Gauss-Newton steps on the per-tilt offsets, volume known: the
    injected offsets U(+-3 px) come back to < 0.1 px."""
    import torch

    case = small_case(dims=(96, 96, 32), n_proj=41, W=96, H=96, seed=11, n_ell=40)
    n = len(case["tilt"])
    rng = np.random.default_rng(7)
    true = rng.uniform(-3, 3, size=(n, 2))
    x = cuda(case["vol"])
    meas = []
    for i in range(n):
        p = torch.zeros((case["H"], case["W"]), device="cuda")
        _gpu_loss(case, i, x, None, tuple(true[i]), proj_d=p)
        meas.append(p)
    s = np.zeros((n, 2))
    for _ in range(20):
        for i in range(n):
            o = _gpu_loss(case, i, x, meas[i], tuple(s[i]))
            Hm = np.array([[o[3], o[4]], [o[4], o[5]]])
            Hm += np.eye(2) * 1e-6 * np.trace(Hm)
            step = np.linalg.solve(Hm, o[1:3])
            nrm = np.linalg.norm(step)
            if nrm > 1.0:
                step /= nrm
            s[i] -= step
    err = np.abs(s - true).max()
    assert err < 0.1, err


@pytest.mark.gpu
def test_autograd_function_uses_the_adjoint():
    import torch

    import artiatomi_b200 as E

    case = _case()
    c = _consts(case, 1)
    W, H = case["W"], case["H"]

    class Project(torch.autograd.Function):
        @staticmethod
        def forward(ctx, vol):
            p = torch.zeros((H, W), device="cuda")
            E.forward_project(c, vol.detach().contiguous(), p, torch.zeros_like(p), fast=True)
            return p

        @staticmethod
        def backward(ctx, gp):
            g = torch.zeros((case["dims"][2], case["dims"][1], case["dims"][0]), device="cuda")
            E.fp_adjoint(c, g, gp.contiguous())
            return g

    rng = np.random.default_rng(9)
    meas = cuda((rng.normal(size=(H, W)) * 3).astype(np.float32))
    x = cuda(case["vol"]).requires_grad_(True)
    loss = 0.5 * ((Project.apply(x) - meas) ** 2).sum()
    loss.backward()
    g = torch.zeros(x.shape, device="cuda")
    out = _gpu_loss(case, 1, x.detach(), meas, (0.0, 0.0), grad_d=g)
    assert abs(float(loss.detach()) - out[0]) <= 1e-5 * out[0]
    assert rel_l2(host(x.grad), host(g)) <= 1e-5
