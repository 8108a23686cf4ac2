"""numpy restatement of the reference's host geometry (TEST INFRASTRUCTURE).

Follows src/EmSART/Projection.cpp and src/EmSART/Volume.cpp, using float32
scalars where the reference uses float and Python floats where it uses double,
so the results match the reference's rounding.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .lib import OrcGeom

f = np.float32
DIST = f(-10000.0)  # Constants.h:42


def _roundf(x):
    """C roundf: halves away from zero (numpy rounds halves to even)."""
    x = f(x)
    r = f(math.floor(abs(float(x)) + 0.5))
    return r if x >= 0 else -r


def _mmul(A, B):  # Matrix<double>::Mul (Matrix.cpp:625-640)
    return [[((0.0 + A[r][0] * B[0][c]) + A[r][1] * B[1][c]) + A[r][2] * B[2][c] for c in range(3)] for r in range(3)]


def _mvec(A, v):
    return [((0.0 + A[r][0] * v[0]) + A[r][1] * v[1]) + A[r][2] * v[2] for r in range(3)]


def _rotate(tilt, psi, cfg, vec):
    """Projection::RotateMatrix (Projection.cpp:80-143)."""
    tilt_a = float(f(tilt) + f(cfg.get("add_tilt_angle", 0.0))) / 180.0 * math.pi
    tiltx = float(f(cfg.get("add_tilt_x_angle", 0.0))) / 180.0 * math.pi
    psi_a = float(-f(psi)) / 180.0 * math.pi
    if cfg.get("use_fix_psi_angle", False):
        psi_a = float(-f(cfg.get("psi_angle", 0.0))) / 180.0 * math.pi
    phi = float(f(cfg.get("phi_angle", 0.0))) / 180.0 * math.pi
    adj = [[0, -1, 0], [1, 0, 0], [0, 0, -1]]
    mpsi = [[math.cos(psi_a), -math.sin(psi_a), 0], [math.sin(psi_a), math.cos(psi_a), 0], [0, 0, 1]]
    mphi = [[1, 0, 0], [0, math.cos(phi), -math.sin(phi)], [0, math.sin(phi), math.cos(phi)]]
    mth = [[math.cos(tilt_a), 0, math.sin(tilt_a)], [0, 1, 0], [-math.sin(tilt_a), 0, math.cos(tilt_a)]]
    mx = [[1, 0, 0], [0, math.cos(tiltx), -math.sin(tiltx)], [0, math.sin(tiltx), math.cos(tiltx)]]
    mphit = [[mphi[c][r] for c in range(3)] for r in range(3)]
    mth = _mmul(mphi, _mmul(mth, mphit))
    v = [float(vec[0]), float(vec[1]), float(vec[2])]
    d = _mvec(mx, _mvec(mth, _mvec(mpsi, _mvec(adj, v))))
    return np.array(d, dtype=np.float32)


def _normalize(v):
    v = v.astype(np.float32)
    dot = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]
    inv = f(1.0) / np.sqrt(f(dot))
    return (v * inv).astype(np.float32)


def _detector_matrix(u, v, n, d, os=1.0):
    """Projection::GetDetectorMatrix (Projection.cpp:289-404); see libesb's
    restatement for the storage order."""
    e = [float(u[0]) / os, float(u[1]) / os, float(u[2]) / os, 0.0, float(v[0]) / os, float(v[1]) / os,
         float(v[2]) / os, 0.0, float(n[0]), float(n[1]), float(n[2]), 0.0, float(d[0]), float(d[1]), float(d[2]), 1.0]
    a0 = e[0] * e[5] - e[1] * e[4]; a1 = e[0] * e[6] - e[2] * e[4]; a2 = e[0] * e[7] - e[3] * e[4]
    a3 = e[1] * e[6] - e[2] * e[5]; a4 = e[1] * e[7] - e[3] * e[5]; a5 = e[2] * e[7] - e[3] * e[6]
    b0 = e[8] * e[13] - e[9] * e[12]; b1 = e[8] * e[14] - e[10] * e[12]; b2 = e[8] * e[15] - e[11] * e[12]
    b3 = e[9] * e[14] - e[10] * e[13]; b4 = e[9] * e[15] - e[11] * e[13]; b5 = e[10] * e[15] - e[11] * e[14]
    det = a0 * b5 - a1 * b4 + a2 * b3 + a3 * b2 - a4 * b1 + a5 * b0
    m = [+e[5] * b5 - e[6] * b4 + e[7] * b3, -e[4] * b5 + e[6] * b2 - e[7] * b1, +e[4] * b4 - e[5] * b2 + e[7] * b0,
         -e[4] * b3 + e[5] * b1 - e[6] * b0, -e[1] * b5 + e[2] * b4 - e[3] * b3, +e[0] * b5 - e[2] * b2 + e[3] * b1,
         -e[0] * b4 + e[1] * b2 - e[3] * b0, +e[0] * b3 - e[1] * b1 + e[2] * b0, +e[13] * a5 - e[14] * a4 + e[15] * a3,
         -e[12] * a5 + e[14] * a2 - e[15] * a1, +e[12] * a4 - e[13] * a2 + e[15] * a0,
         -e[12] * a3 + e[13] * a1 - e[14] * a0, -e[9] * a5 + e[10] * a4 - e[11] * a3,
         +e[8] * a5 - e[10] * a2 + e[11] * a1, -e[8] * a4 + e[9] * a2 - e[11] * a0, +e[8] * a3 - e[9] * a1 + e[10] * a0]
    inv = 1.0 / det
    return np.array([x * inv for x in m], dtype=np.float32)


def projection_geometry(tilt, x_shift=None, y_shift=None, mag=None, psi=None, width=256, height=256, cfg=None,
                        extra_shift=None):
    """Per projection dict(det, u, v, n, detMat) (Projection.cpp:167-404)."""
    cfg = cfg or {}
    n = len(tilt)
    z = np.zeros(n, np.float32)
    x_shift = z if x_shift is None else np.asarray(x_shift, np.float32)
    y_shift = z if y_shift is None else np.asarray(y_shift, np.float32)
    mag = np.ones(n, np.float32) if mag is None else np.asarray(mag, np.float32)
    psi = z if psi is None else np.asarray(psi, np.float32)
    es = np.zeros((n, 2), np.float32) if extra_shift is None else np.asarray(extra_shift, np.float32).reshape(n, 2)
    out = []
    for i in range(n):
        m = f(mag[i])
        ok = m > f(0.8)
        uu = _rotate(tilt[i], psi[i], cfg, [m if ok else f(1), 0, 0])
        vv = _rotate(tilt[i], psi[i], cfg, [0, m if ok else f(1), 0])
        if ok:
            pos = [f(-0.5) * f(width) * m, f(-0.5) * f(height) * m, DIST]
        else:
            pos = [f(-0.5) * f(width), f(-0.5) * f(height), DIST]
        sx = f(x_shift[i]) + f(es[i, 0])
        sy = f(y_shift[i]) + f(es[i, 1])
        pr = _rotate(tilt[i], psi[i], cfg, pos)
        det = ((pr - (uu * sx).astype(np.float32)).astype(np.float32) - (vv * sy).astype(np.float32)).astype(np.float32)
        un, vn = _normalize(uu), _normalize(vv)
        nrm = np.array([un[2] * vn[1] - un[1] * vn[2], un[0] * vn[2] - un[2] * vn[0], un[1] * vn[0] - un[0] * vn[1]],
                       np.float32)
        nrm = _normalize(nrm)
        out.append(dict(det=det, u=uu, v=vv, n=nrm, detMat=_detector_matrix(uu, vv, nrm, det)))
    return out


@dataclass
class VolGeom:
    bbMin: np.ndarray
    bbMax: np.ndarray
    bbRcp: np.ndarray
    dim: np.ndarray
    vs: np.ndarray
    zShift: float
    full_dim: np.ndarray
    full_min: np.ndarray
    full_max: np.ndarray


def volume_geometry(dims, voxel_size=(1, 1, 1), volume_shift=(0, 0, 0), count=1, part=0) -> VolGeom:
    """Volume(dim, count, part) + PositionInSpace (Volume.cpp:82-114, 270-287)."""
    vs = np.asarray(voxel_size, np.float32)
    sh = np.asarray(volume_shift, np.float32)
    sizeZ = int(math.ceil(dims[2] / count))
    rest = dims[2] - sizeZ * (count - 1)
    pos = np.array([vs[0] * (f(-0.5) * f(dims[0])) + f(0) - sh[0], vs[1] * (f(-0.5) * f(dims[1])) + f(0) - sh[1],
                    vs[2] * (f(-0.5) * f(dims[2])) - sh[2]], np.float32)
    before = sizeZ * part
    subz = rest if part == count - 1 else sizeZ
    mn = pos.copy()
    mn[2] = f(pos[2] + vs[2] * f(before))
    dim = np.array([dims[0], dims[1], subz], np.float32)
    mx = (mn + (dim * vs).astype(np.float32)).astype(np.float32)
    rcp = (f(1) / (dim * vs).astype(np.float32)).astype(np.float32)
    full = np.array(dims, np.float32)
    return VolGeom(mn, mx, rcp, dim, vs, float(before), full, pos, (pos + (full * vs).astype(np.float32)).astype(np.float32))


def subvolume_geometry(size, vs_sub, vol: VolGeom, pos, shift=(0, 0, 0)) -> VolGeom:
    """Volume::PositionInSpace for a particle box (Volume.cpp:289-306)."""
    p = np.zeros(3, np.float32)
    for k in range(3):
        p[k] = ((f(vs_sub) * (f(-0.5) * f(size)) + vol.vs[k] * (f(pos[k]) - f(1))) + f(shift[k]) * vol.vs[k]) + vol.full_min[k]
    dim = np.full(3, size, np.float32)
    vs = np.full(3, vs_sub, np.float32)
    mx = (p + (dim * vs).astype(np.float32)).astype(np.float32)
    rcp = (f(1) / (dim * vs).astype(np.float32)).astype(np.float32)
    return VolGeom(p, mx, rcp, dim, vs, 0.0, dim.copy(), p.copy(), mx.copy())


def orc_geom(pg: dict, vg: VolGeom, aniso=None, aniso_inv=None, for_bp=False) -> OrcGeom:
    """SetConstantValues (Kernels.cpp:949-1101) as an OrcGeom."""
    g = OrcGeom()
    g.det[:] = list(map(float, pg["det"]))
    g.u[:] = list(map(float, pg["u"]))
    g.v[:] = list(map(float, pg["v"]))
    g.n[:] = list(map(float, pg["n"]))
    g.detMat[:] = list(map(float, pg["detMat"]))
    g.bbMin[:] = list(map(float, vg.bbMin))
    g.bbMax[:] = list(map(float, vg.bbMax))
    g.bbRcp[:] = list(map(float, vg.bbRcp))
    g.dim[:] = list(map(float, vg.dim))
    g.vs[:] = list(map(float, vg.vs))
    g.zShift = float(vg.zShift) if for_bp else 0.0
    g.dimXQuarter = int(vg.full_dim[0]) // 4
    ident = [1, 0, 0, 0, 1, 0, 0, 0, 1]
    g.aniso[:] = list(map(float, ident if aniso is None else aniso))
    g.anisoInv[:] = list(map(float, ident if aniso_inv is None else aniso_inv))
    return g


def _detmul(M, p):
    M = np.asarray(M, np.float32)
    return np.array([M[4 * r] * p[0] + M[4 * r + 1] * p[1] + M[4 * r + 2] * p[2] + f(1) * M[4 * r + 3] for r in range(3)],
                    np.float32)


def compute_hit_points(pg: dict, vg: VolGeom):
    """Projection::ComputeHitPoints (Projection.cpp:850-1049)."""
    mn, mx, det, n = vg.full_min, vg.full_max, pg["det"], pg["n"]
    P = []
    for c in range(8):
        q = np.array([mn[0] + (mx[0] - mn[0]) if c & 4 else mn[0], mn[1] + (mx[1] - mn[1]) if c & 2 else mn[1],
                      mn[2] + (mx[2] - mn[2]) if c & 1 else mn[2]], np.float32)
        t = f(f(n[0] * q[0] + n[1] * q[1]) + n[2] * q[2])
        t = f(t + f(f(f(-n[0] * det[0]) - n[1] * det[1]) - n[2] * det[2]))
        t = abs(t)
        hp = np.array([t * -n[k] + q[k] for k in range(3)], np.float32)
        P.append(_detmul(pg["detMat"], hp))
    pick = lambda a, b: int(a if abs(a) < abs(b) else b)
    return [pick(P[0][0], P[1][0]), pick(P[0][1], P[1][1]), pick(P[2][0], P[3][0]), pick(P[2][1], P[3][1]),
            pick(P[4][0], P[5][0]), pick(P[4][1], P[5][1]), pick(P[6][0], P[7][0]), pick(P[6][1], P[7][1])]


def defocus_distances(pg: dict, vg: VolGeom):
    """Reconstructor::GetDefocusDistances (Reconstructor.cpp:53-173)."""
    n, det = pg["n"], pg["det"]
    mn, mx, vd, vs = vg.full_min, vg.full_max, vg.full_dim, vg.vs
    c = np.array([mn[k] + (vd[k] * vs[k] * f(0.5)) for k in range(3)], np.float32)
    t = f(f(n[0] * c[0] + n[1] * c[1]) + n[2] * c[2])
    t = f(t + f(f(f(-n[0] * det[0]) - n[1] * det[1]) - n[2] * det[2]))
    t = abs(t)
    hit = _detmul(pg["detMat"], np.array([t * -n[k] + c[k] for k in range(3)], np.float32))
    hx, hy = int(_roundf(hit[0])), int(_roundf(hit[1]))
    pos = ((det + (pg["u"] * f(hx)).astype(np.float32)).astype(np.float32) + (pg["v"] * f(hy)).astype(np.float32)).astype(np.float32)
    tin, tout = f(20000.0), f(-20000.0)
    for x in (0, 1):
        for y in (0, 1):
            for z in (0, 1):
                tt = f(f(n[0] * (mn[0] + f(x) * (mx[0] - mn[0])) + n[1] * (mn[1] + f(y) * (mx[1] - mn[1]))) +
                       n[2] * (mn[2] + f(z) * (mx[2] - mn[2])))
                tt = f(tt + f(f(f(-n[0] * pos[0]) - n[1] * pos[1]) - n[2] * pos[2]))
                tin = min(tin, tt)
                tout = max(tout, tt)
    return float(tin), float(tout)


def defocus_min_max(ray, dmin, dmax, tilt, add_tilt, ps, T, vshift_z=0.0, ignore_z=False, switch=False):
    """Reconstructor::GetDefocusMinMax (Reconstructor.cpp:178-201)."""
    ta = f(f(f(tilt) + f(add_tilt)) / f(180.0) * f(math.pi))
    d = f(f(ray) + DIST)
    base = f(f(_roundf(f(f(d * f(ps)) * f(T)))) / f(T)) + f(T) / f(2)
    if ignore_z:
        d = f(base)
    else:
        d = f(base - f(f(f(vshift_z) * f(ps)) * f(np.cos(ta))))
    if switch:
        d = -d
    return float(f(f(dmin) + d)), float(f(f(dmax) + d))


def mag_aniso(amount, angle_deg, dimx, dimy):
    """Reconstructor::GetMagAnistropyMatrix (Reconstructor.cpp:386-426), float."""
    a = f(f(angle_deg) / f(180.0) * f(math.pi))
    def rz(t):
        return np.array([[np.cos(t), -np.sin(t), 0], [np.sin(t), np.cos(t), 0], [0, 0, 1]], np.float32)
    sc = np.array([[1, 0, -f(dimx) / f(2)], [0, 1, -f(dimy) / f(2)], [0, 0, 1]], np.float32)
    sb = np.array([[1, 0, f(dimx) / f(2)], [0, 1, f(dimy) / f(2)], [0, 0, 1]], np.float32)
    st = np.array([[amount, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    def mm(A, B):
        R = np.zeros((3, 3), np.float32)
        for r in range(3):
            for c in range(3):
                v = f(0)
                for i in range(3):
                    v = f(v + f(A[r, i] * B[i, c]))
                R[r, c] = v
        return R
    acc = mm(mm(mm(mm(sb, rz(-a)), st), rz(a)), sc)
    return acc.ravel()


def rotation_matrix(phi, psi, theta):
    """RotKernel::computeRotMat (Kernels.cpp:1227-1327), float: multiples of
    30 and 45 degrees in [0, 330] take exact table values, other angles the
    float cosine / sine of the angle in radians. Row-major [3][3]."""
    r3, r2 = f(f(np.sqrt(f(3))) / f(2)), f(f(np.sqrt(f(2))) / f(2))
    table = {0: (1, 0), 30: (r3, 0.5), 45: (r2, r2), 60: (0.5, r3), 90: (0, 1), 120: (-0.5, r3), 135: (-r2, r2),
             150: (-r3, 0.5), 180: (-1, 0), 210: (-r3, -0.5), 225: (-r2, -r2), 240: (-0.5, -r3), 270: (0, -1),
             300: (0.5, -r3), 315: (r2, -r2), 330: (r3, -0.5)}

    def cs(a):
        a = f(a)
        for d, (c, s) in table.items():
            if a == f(d):
                return f(c), f(s)
        r = f(f(a * f(math.pi)) / f(180))
        return f(np.cos(r)), f(np.sin(r))

    cphi, sphi = cs(phi)
    cpsi, spsi = cs(psi)
    cth, sth = cs(theta)
    R = np.zeros((3, 3), np.float32)
    R[0, 0] = f(f(cpsi * cphi) - f(f(cth * spsi) * sphi))
    R[1, 0] = f(f(spsi * cphi) + f(f(cth * cpsi) * sphi))
    R[2, 0] = f(sth * sphi)
    R[0, 1] = f(f(-cpsi * sphi) - f(f(cth * spsi) * cphi))
    R[1, 1] = f(f(-spsi * sphi) + f(f(cth * cpsi) * cphi))
    R[2, 1] = f(sth * cphi)
    R[0, 2] = f(sth * spsi)
    R[1, 2] = f(-sth * cpsi)
    R[2, 2] = cth
    return R


def index_list_random_start_zero(tilt, good=None):
    """Projection::CreateProjectionIndexList(PLT_RANDOM_START_ZERO_TILT)
    (Projection.cpp:592-624) with the C library's srand(0)/rand()."""
    import ctypes
    libc = ctypes.CDLL(None)
    n = len(tilt)
    lst = [i for i in range(n) if good is None or good[i]]
    libc.srand(0)
    for i in range(len(lst) - 1):
        r = i + libc.rand() % (len(lst) - i)
        lst[i], lst[r] = lst[r], lst[i]
    mt, mi = np.float32(np.finfo(np.float32).max), 0
    for i in range(n):
        if abs(np.float32(tilt[i])) < mt:
            mt, mi = abs(np.float32(tilt[i])), i
    for i in range(len(lst)):
        if lst[i] == mi:
            lst[0], lst[i] = lst[i], lst[0]
            break
    return np.array(lst, np.int32)
