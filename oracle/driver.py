"""Restatement of the reference's Reconstructor sequences and driver loops on
the oracle kernels (TEST INFRASTRUCTURE).

Follows Reconstructor::ForwardProjectionNoCTF / ForwardProjectionCTF
(Reconstructor.cpp:429-644), Compare (:1386-1405), BackProjectionNoCTF /
BackProjectionCTF (:871-969), the sub-volume back-projections (:893-1033),
the SART loop of EmSart.cpp:579-675 and the batch loop of
EmSartSubVolumes.cpp:611-705.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import geometry as G
from .lib import NTHREADS, addr, f32, olib

f = np.float32


def fp_march(g, vol, dtype, W, H, proj, dist, precision=0, q9=0, exact_step=0, roi=None):
    x0, y0, x1, y1 = roi if roi is not None else (0, 0, W, H)
    olib.orc_fp_march(C.byref(g), addr(vol), dtype, W, H, addr(proj), addr(dist), x0, y0, x1, y1, precision, q9,
                      exact_step, NTHREADS)


def fp_slicer(g, vol, dtype, W, H, proj, tmin, tmax, precision=0, q9=0, fix_first=0):
    olib.orc_fp_slicer(C.byref(g), addr(vol), dtype, W, H, addr(proj), tmin, tmax, precision, q9, fix_first, NTHREADS)


def travlen(g, W, H, dist, precision=0):
    olib.orc_vol_traversal_length(C.byref(g), W, H, addr(dist), precision, NTHREADS)


def compare(real, virt, dist, real_length, crop, crop_dim, scale):
    H, W = virt.shape
    olib.orc_compare(W, H, addr(real), addr(virt), addr(dist), real_length, addr(f32(crop)), addr(f32(crop_dim)), scale)


def crop_border(img, cut, dim, p):
    H, W = img.shape
    olib.orc_crop_border(W, H, addr(img), addr(f32(cut)), addr(f32(dim)), addr(np.asarray(p, np.int32)))


def bp(g, vol, dtype, img, lam, os_, dmin=0.0, dmax=9999999999999.0, linear=0, precision=0, q9=0):
    H, W = img.shape
    olib.orc_bp(C.byref(g), addr(vol), dtype, addr(img), W, H, lam, os_, dmin, dmax, linear, precision, q9, NTHREADS)


def make_square(img, N, bx, by, mirror=0, fill_zero=1):
    H, W = img.shape
    out = np.zeros((N, N), np.float32)
    olib.orc_make_square(W, H, N, W, addr(img), addr(out), bx, by, mirror, fill_zero)
    return out


def r2c(sq):
    N = sq.shape[0]
    out = np.zeros((N, N // 2 + 1, 2), np.float32)
    olib.orc_r2c(addr(sq), addr(out), N, NTHREADS)
    return out


def c2r(spec):
    N = spec.shape[0]
    out = np.zeros((N, N), np.float32)
    olib.orc_c2r(addr(spec), addr(out), N, NTHREADS)
    return out


def ctf(spec, dmin, dmax, angle, for_fp, cfg, precision=1):
    N = spec.shape[0]
    olib.orc_ctf(addr(spec), N, dmin, dmax, angle, int(for_fp), int(cfg["phase_flip_only"]), cfg["wiener_noise_level"],
                 addr(f32(cfg["ctf_beta_fac"])), cfg["cs_mm"], cfg["voltage_kv"], cfg["amp_contrast"],
                 cfg["pixel_size_nm"], precision)


DEFAULT_CFG = dict(lambda_=1.0, oversampling=1, ctf_mode=False, cut_length=(0.0, 0.0), dim_length=(1.0, 1.0),
                   crop=(0.0, 0.0, 0.0, 0.0), crop_dim=(1.0, 1.0, 1.0, 1.0), projection_scale_factor=1.0,
                   pixel_size_nm=1.0, cs_mm=2.7, voltage_kv=300.0, amp_contrast=0.0, ctf_slice_thickness_nm=50.0,
                   ctf_beta_fac=(200.0, 0.0, 0.008, 0.0), wiener_noise_level=0.1, phase_flip_only=False,
                   ignore_z_shift_for_ctf=False, switch_ctf_direction=False, volume_shift=(0.0, 0.0, 0.0),
                   add_tilt_angle=0.0)


class OracleReconstructor:
    """Reconstructor (Reconstructor.cpp:203-372) on the CPU oracle."""

    def __init__(self, cfg: dict, W, H, geoms, tilt, defocus=None, aniso=None, aniso_inv=None, precision=0, q9=0):
        self.cfg = dict(DEFAULT_CFG, **cfg)
        self.W, self.H = W, H
        self.geoms, self.tilt = geoms, np.asarray(tilt, np.float32)
        self.defocus = None if defocus is None else np.asarray(defocus, np.float32).reshape(-1, 3)
        self.aniso, self.aniso_inv = aniso, aniso_inv
        self.precision, self.q9 = precision, q9
        self.N = max(W, H)
        self.bx, self.by = (self.N - W) // 2, (self.N - H) // 2
        self.proj = np.zeros((H, W), np.float32)
        self.dist = np.zeros((H, W), np.float32)

    def reset(self):
        self.proj[:] = 0
        self.dist[:] = 0

    def _ctf_chain(self, img, crop_in, p_in, index, dmin, dmax, for_fp, crop_out, p_out):
        c = self.cfg
        if crop_in:
            crop_border(img, c["cut_length"], c["dim_length"], p_in)
        sq = make_square(img, self.N, self.bx, self.by, 0, 1)
        spec = r2c(sq)
        ctf(spec, dmin, dmax, float(self.defocus[index, 2]), for_fp, c)
        sq = c2r(spec)
        out = (sq[self.by:self.by + self.H, self.bx:self.bx + self.W] * f(1.0 / (self.N * self.N))).astype(np.float32)
        out = np.ascontiguousarray(out)
        if crop_out:
            crop_border(out, c["cut_length"], c["dim_length"], p_out)
        return out

    def _slabs(self, index, vg):
        t_in, t_out = G.defocus_distances(self.geoms[index], vg)
        step = f(f(self.cfg["ctf_slice_thickness_nm"]) / f(self.cfg["pixel_size_nm"]))
        ray = f(t_in)
        while ray < f(t_out):
            yield float(ray), float(f(ray + step))
            ray = f(ray + step)

    def _dminmax(self, ray, index):
        c = self.cfg
        return G.defocus_min_max(ray, self.defocus[index, 0], self.defocus[index, 1], self.tilt[index],
                                 c["add_tilt_angle"], c["pixel_size_nm"], c["ctf_slice_thickness_nm"],
                                 c["volume_shift"][2], c["ignore_z_shift_for_ctf"], c["switch_ctf_direction"])

    def forward_projection(self, vg, vol, dtype, index, volume_is_empty):
        """Reconstructor::ForwardProjection (Reconstructor.cpp:1411-1421)."""
        g = G.orc_geom(self.geoms[index], vg, self.aniso, self.aniso_inv)
        W, H = self.W, self.H
        if volume_is_empty:
            travlen(g, W, H, self.dist, self.precision)
            return
        if not self.cfg["ctf_mode"]:
            fp_march(g, vol, dtype, W, H, self.proj, self.dist, self.precision, self.q9)
            return
        full = [0, H - 1, W - 1, H - 1, 0, 0, W - 1, 0]
        for ray, ray1 in self._slabs(index, vg):
            dmin, dmax = self._dminmax(ray, index)
            self.dist[:] = 0
            fp_slicer(g, vol, dtype, W, H, self.dist, ray, ray1, self.precision, self.q9)
            out = self._ctf_chain(self.dist, 1, full, index, dmin, dmax, True, 1, full)
            self.proj += out
        self.dist[:] = 0
        travlen(g, W, H, self.dist, self.precision)

    def compare(self, vg, real, index):
        """Reconstructor::Compare (Reconstructor.cpp:1386-1405)."""
        zdir = f(self.geoms[index]["n"][2])
        zmin, zmax = vg.full_min[2], vg.full_max[2]
        length = abs(f(f(G.DIST - zmin) / zdir) - f(f(G.DIST - zmax) / zdir))
        c = self.cfg
        compare(np.ascontiguousarray(real, np.float32), self.proj, self.dist, float(length), c["crop"], c["crop_dim"],
                c["projection_scale_factor"])

    def back_projection(self, vg, vol, dtype, index, sirt_count, img=None):
        """Reconstructor::BackProjection (Reconstructor.cpp:871-887, 920-969)."""
        img = self.proj if img is None else img
        c = self.cfg
        p = G.compute_hit_points(self.geoms[index], vg)
        g = G.orc_geom(self.geoms[index], vg, self.aniso, self.aniso_inv, for_bp=True)
        lam = float(f(f(c["lambda_"]) / f(sirt_count)))
        if not c["ctf_mode"]:
            crop_border(img, c["cut_length"], c["dim_length"], p)
            bp(g, vol, dtype, img, lam, c["oversampling"], 0.0, 9999999999999.0, 0, self.precision, self.q9)
            return
        for ray, ray1 in self._slabs(index, vg):
            dmin, dmax = self._dminmax(ray, index)
            filt = self._ctf_chain(img, 1, p, index, dmin, dmax, False, 1, p)
            bp(g, vol, dtype, filt, lam, c["oversampling"], ray, ray1, 1, self.precision, self.q9)

    def sart(self, vg, vol, dtype, projections, index_list, iterations, sirt_count, volume_is_empty=True):
        """EmSart.cpp:579-675."""
        n = len(index_list)
        for _ in range(iterations):
            for s in range((n + sirt_count - 1) // sirt_count):
                buf = {}
                for i in range(sirt_count):
                    if s * sirt_count + i >= n:
                        continue
                    index = int(index_list[s * sirt_count + i])
                    self.reset()
                    self.forward_projection(vg, vol, dtype, index, volume_is_empty)
                    self.compare(vg, projections[index], index)
                    buf[i] = self.proj.copy()
                for i in range(sirt_count):
                    if s * sirt_count + i >= n:
                        continue
                    volume_is_empty = False
                    index = int(index_list[s * sirt_count + i])
                    self.back_projection(vg, vol, dtype, index, float(sirt_count), img=buf[i])
        return volume_is_empty

    def subvolume_wbp(self, full_vg, sub_geoms, pair_geoms, boxes, projections, index_list, active=None):
        """EmSartSubVolumes.cpp:626-683 with Reconstructor.cpp:893-914/975-1033.
        pair_geoms[p][index] are per particle detector frames with its extra
        shift; boxes are float32 arrays accumulated in place."""
        c = self.cfg
        for index in index_list:
            index = int(index)
            proj = np.ascontiguousarray(projections[index], np.float32)
            if not c["ctf_mode"]:
                for p, box in enumerate(boxes):
                    if active is not None and not active[p][index]:
                        continue
                    g = G.orc_geom(pair_geoms[p][index], sub_geoms[p], self.aniso, self.aniso_inv, for_bp=True)
                    bp(g, box, 0, proj, 1.0, c["oversampling"], 0.0, 9999999999999.0, 0, self.precision, self.q9)
                continue
            for ray, ray1 in self._slabs(index, full_vg):
                dmin, dmax = self._dminmax(ray, index)
                filt = self._ctf_chain(proj.copy(), 0, None, index, dmin, dmax, False, 0, None)
                for p, box in enumerate(boxes):
                    if active is not None and not active[p][index]:
                        continue
                    g = G.orc_geom(pair_geoms[p][index], sub_geoms[p], self.aniso, self.aniso_inv, for_bp=True)
                    bp(g, box, 0, filt, 1.0, c["oversampling"], ray, ray1, 1, self.precision, self.q9)


def _mean_std(a):
    a = np.asarray(a, np.float64)
    mu = a.sum() / a.size
    var = (a * a).sum() / a.size - mu * mu
    return np.float32(mu), np.float32(np.sqrt(max(var, 0.0)))


def prepare_projection(raw, N, pc: dict):
    """Reconstructor::PrepareProjection (Reconstructor.cpp:1158-1383) on one
    raw W x H projection; pc has the fields of esb_prepare_config. Returns
    (normalised float image, mean, std, bad pixel count). Mean and standard
    deviation are FP64 sums (population variance), where the reference calls
    NPP."""
    H, W = raw.shape
    bx, by = (N - W) // 2, (N - H) // 2
    img = np.ascontiguousarray(raw.astype(np.float32))
    sq = make_square(img, N, bx, by, int(pc.get("mirror_y", 0)), 0)
    meanValue = np.float32(sq.astype(np.float64).sum() / sq.size)
    bad = 0
    if pc.get("correct_bad_pixels", 0):
        mask = sq > np.float32(np.float32(pc["bad_pixel_value"]) * meanValue)
        bad = int(mask.sum())
        sq[mask] = meanValue
    stdValue = np.float32(0)
    norm = pc.get("normalization", 1)
    if pc.get("wbp", 0):
        win = np.ascontiguousarray(sq[by:by + H, bx:bx + W] / np.float32(1.0))
        meanValue, stdValue = _mean_std(win)
        std_hf, mean_hf = stdValue, meanValue
        if norm == 0:
            std_hf = meanValue
        if norm == 2:
            std_hf, mean_hf = np.float32(1), np.float32(0)
        if pc.get("down_weight_tilts", 0):
            std_hf = np.float32(std_hf / np.float32(np.cos(np.float32(abs(pc["tilt_deg"])) / np.float32(180.0) *
                                                            np.float32(np.pi))))
        out = ((win - mean_hf) / (-std_hf)).astype(np.float32)
        sq = make_square(np.ascontiguousarray(out), N, bx, by, 0, 0)
    normVal = np.float32(1.0)
    if not pc.get("skip_filter", 0) or pc.get("wbp", 0):
        spec = r2c(sq)
        if not pc.get("skip_filter", 0):
            olib.orc_fourier_filter(addr(spec), N, pc.get("lp", 0.0), pc.get("hp", 0.0), pc.get("lps", 0.0),
                                    pc.get("hps", 0.0))
        if pc.get("dose_weighting", 0):
            olib.orc_dose_weighting(addr(spec), N, pc["accumulated_dose"], np.float32(pc["pixel_size_nm"]) *
                                    np.float32(10.0))
        if pc.get("wbp", 0):
            olib.orc_wbp_weighting(addr(spec), N, pc.get("psi_deg", 0.0), pc.get("wbp_filter", 0))
        sq = c2r(spec)
        normVal = np.float32(N) * np.float32(N)
    win = (sq[by:by + H, bx:bx + W] / normVal).astype(np.float32)
    if pc.get("wbp", 0):
        return np.ascontiguousarray(win), meanValue, stdValue, bad
    if norm == 2:
        meanValue, stdValue = _mean_std(win[H // 4:H // 4 + H // 2, W // 4:W // 4 + W // 2])
    else:
        meanValue, stdValue = _mean_std(win)
    std_hf, mean_hf = stdValue, meanValue
    if norm == 0:
        std_hf = meanValue
    if norm == 2:
        std_hf = np.float32(1)
    out = ((win - mean_hf) / (-std_hf)).astype(np.float32)
    return np.ascontiguousarray(out), meanValue, stdValue, bad
