// Host geometry of the reconstruction: detector frames per projection,
// (sub-)volume placement, kernel constants, volume-shadow hit points and the
// CTF slab bookkeeping. Each function restates the reference member it
// replaces (file:line in the comments) with the same float/double rounding
// steps, so that the kernel constants match the reference's bit for bit in
// the common case.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cfloat>
#include <string>

#include "../../include/esb.h"
#include "esb_internal.h"

namespace {

const float DIST = -10000.0f;  // Constants.h:42 (detector distance)

struct F3 {
  float x, y, z;
};
inline F3 f3(float x, float y, float z) { return F3{x, y, z}; }
inline F3 sub(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline F3 add(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline F3 mul(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 normalize(F3 v) {  // cutil_math normalize: v * (1/sqrtf(dot(v,v)))
  float inv = 1.0f / sqrtf(dot(v, v));
  return mul(v, inv);
}

struct M3d {
  double a[3][3];
};
M3d mmul(const M3d& A, const M3d& B) {  // Matrix<T>::Mul (Matrix.cpp:625-640)
  M3d R;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double v = 0;
      for (int i = 0; i < 3; ++i) v += A.a[r][i] * B.a[i][c];
      R.a[r][c] = v;
    }
  return R;
}
void mvec(const M3d& A, const double in[3], double out[3]) {
  for (int r = 0; r < 3; ++r) {
    double v = 0;
    for (int i = 0; i < 3; ++i) v += A.a[r][i] * in[i];
    out[r] = v;
  }
}
M3d mtrans(const M3d& A) {
  M3d R;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) R.a[r][c] = A.a[c][r];
  return R;
}

struct TiltInput {
  float tilt, sx, sy, mag, psi, ex, ey;
};

// Projection::RotateMatrix (Projection.cpp:80-143).
F3 rotate(const TiltInput& t, const esb_tilt_config& cfg, F3 in) {
  double tiltAngle = (double)(t.tilt + cfg.add_tilt_angle) / 180.0 * (double)M_PI;
  double tiltXAngle = (double)cfg.add_tilt_x_angle / 180.0 * (double)M_PI;
  double psiAngle = (double)(-t.psi) / 180.0 * (double)M_PI;
  if (cfg.use_fix_psi_angle) psiAngle = (double)(-cfg.psi_angle) / 180.0 * (double)M_PI;
  double phiAngle = (double)cfg.phi_angle / 180.0 * (double)M_PI;
  M3d adj = {{{0, -1, 0}, {1, 0, 0}, {0, 0, -1}}};
  M3d psi = {{{cos(psiAngle), -sin(psiAngle), 0}, {sin(psiAngle), cos(psiAngle), 0}, {0, 0, 1}}};
  M3d phi = {{{1, 0, 0}, {0, cos(phiAngle), -sin(phiAngle)}, {0, sin(phiAngle), cos(phiAngle)}}};
  M3d th = {{{cos(tiltAngle), 0, sin(tiltAngle)}, {0, 1, 0}, {-sin(tiltAngle), 0, cos(tiltAngle)}}};
  M3d xt = {{{1, 0, 0}, {0, cos(tiltXAngle), -sin(tiltXAngle)}, {0, sin(tiltXAngle), cos(tiltXAngle)}}};
  th = mmul(phi, mmul(th, mtrans(phi)));
  double v[3] = {in.x, in.y, in.z}, a[3], b[3], c[3], d[3];
  mvec(adj, v, a);
  mvec(psi, a, b);
  mvec(th, b, c);
  mvec(xt, c, d);
  return f3((float)d[0], (float)d[1], (float)d[2]);
}

bool mag_ok(float m) { return m > 0.8f && m > 0.8f; }

F3 u_pitch(const TiltInput& t, const esb_tilt_config& cfg) {  // Projection.cpp:199-222
  F3 u = f3(mag_ok(t.mag) ? 1 * t.mag : 1.0f, 0, 0);
  return rotate(t, cfg, u);
}
F3 v_pitch(const TiltInput& t, const esb_tilt_config& cfg) {  // Projection.cpp:224-246
  F3 v = f3(0, mag_ok(t.mag) ? 1 * t.mag : 1.0f, 0);
  return rotate(t, cfg, v);
}
F3 position(const TiltInput& t, const esb_tilt_config& cfg, int w, int h) {  // Projection.cpp:167-197
  F3 pos;
  if (mag_ok(t.mag)) pos = f3(-0.5f * w * t.mag, -0.5f * h * t.mag, DIST);
  else pos = f3(-0.5f * w, -0.5f * h, DIST);
  float shiftX = t.sx + t.ex;
  float shiftY = t.sy + t.ey;
  pos = rotate(t, cfg, pos);
  F3 up = u_pitch(t, cfg), vp = v_pitch(t, cfg);
  return sub(sub(pos, mul(up, shiftX)), mul(vp, shiftY));
}
F3 normal(const TiltInput& t, const esb_tilt_config& cfg) {  // Projection.cpp:248-287
  F3 u = normalize(u_pitch(t, cfg));
  F3 v = normalize(v_pitch(t, cfg));
  F3 n = f3(u.z * v.y - u.y * v.z, u.x * v.z - u.z * v.x, u.y * v.x - u.x * v.y);
  return normalize(n);
}

// Projection::GetDetectorMatrix (Projection.cpp:289-404): inverse of the
// detector frame (rows u, v, n, detector) in double, by the 2x2-minor
// expansion of a 4x4 inverse; stored so that row r of the result dotted with
// (p, 1) is detector coordinate r of point p.
void detector_matrix(F3 uf, F3 vf, F3 nf, F3 df, float os, float out[16]) {
  double e[16] = {(double)uf.x / (double)os, (double)uf.y / (double)os, (double)uf.z / (double)os, 0.0,
                  (double)vf.x / (double)os, (double)vf.y / (double)os, (double)vf.z / (double)os, 0.0,
                  nf.x, nf.y, nf.z, 0.0,
                  df.x, df.y, df.z, 1.0};
  double a0 = e[0] * e[5] - e[1] * e[4], a1 = e[0] * e[6] - e[2] * e[4], a2 = e[0] * e[7] - e[3] * e[4];
  double a3 = e[1] * e[6] - e[2] * e[5], a4 = e[1] * e[7] - e[3] * e[5], a5 = e[2] * e[7] - e[3] * e[6];
  double b0 = e[8] * e[13] - e[9] * e[12], b1 = e[8] * e[14] - e[10] * e[12], b2 = e[8] * e[15] - e[11] * e[12];
  double b3 = e[9] * e[14] - e[10] * e[13], b4 = e[9] * e[15] - e[11] * e[13], b5 = e[10] * e[15] - e[11] * e[14];
  double det = a0 * b5 - a1 * b4 + a2 * b3 + a3 * b2 - a4 * b1 + a5 * b0;
  double m[16];
  // column c of the inverse goes to row c of m
  m[0] = +e[5] * b5 - e[6] * b4 + e[7] * b3;
  m[1] = -e[4] * b5 + e[6] * b2 - e[7] * b1;
  m[2] = +e[4] * b4 - e[5] * b2 + e[7] * b0;
  m[3] = -e[4] * b3 + e[5] * b1 - e[6] * b0;
  m[4] = -e[1] * b5 + e[2] * b4 - e[3] * b3;
  m[5] = +e[0] * b5 - e[2] * b2 + e[3] * b1;
  m[6] = -e[0] * b4 + e[1] * b2 - e[3] * b0;
  m[7] = +e[0] * b3 - e[1] * b1 + e[2] * b0;
  m[8] = +e[13] * a5 - e[14] * a4 + e[15] * a3;
  m[9] = -e[12] * a5 + e[14] * a2 - e[15] * a1;
  m[10] = +e[12] * a4 - e[13] * a2 + e[15] * a0;
  m[11] = -e[12] * a3 + e[13] * a1 - e[14] * a0;
  m[12] = -e[9] * a5 + e[10] * a4 - e[11] * a3;
  m[13] = +e[8] * a5 - e[10] * a2 + e[11] * a1;
  m[14] = -e[8] * a4 + e[9] * a2 - e[11] * a0;
  m[15] = +e[8] * a3 - e[9] * a1 + e[10] * a0;
  double inv = (1.0f) / det;
  for (int i = 0; i < 16; ++i) out[i] = (float)(m[i] * inv);
}

F3 detmul(const float* M, F3 p) {  // MatrixVector3Mul (Projection.cpp:637-644)
  return f3(M[0] * p.x + M[1] * p.y + M[2] * p.z + 1.f * M[3], M[4] * p.x + M[5] * p.y + M[6] * p.z + 1.f * M[7],
            M[8] * p.x + M[9] * p.y + M[10] * p.z + 1.f * M[11]);
}

F3 from(const float* a) { return f3(a[0], a[1], a[2]); }
void put(float* a, F3 v) {
  a[0] = v.x;
  a[1] = v.y;
  a[2] = v.z;
}

}  // namespace

extern "C" {

int esb_projection_geometry(int n_proj, int width, int height, const float* tilt_deg, const float* x_shift,
                            const float* y_shift, const float* magnification, const float* psi_deg,
                            const float* extra_shift, const esb_tilt_config* cfg, esb_proj_geom* out) {
  if (n_proj < 0 || width <= 0 || height <= 0 || !tilt_deg || !out || !cfg)
    return esb::fail(ESB_ERR_INVALID_ARGUMENT, "esb_projection_geometry: invalid argument");
  for (int i = 0; i < n_proj; ++i) {
    TiltInput t;
    t.tilt = tilt_deg[i];
    t.sx = x_shift ? x_shift[i] : 0.f;
    t.sy = y_shift ? y_shift[i] : 0.f;
    t.mag = magnification ? magnification[i] : 1.f;
    t.psi = psi_deg ? psi_deg[i] : 0.f;
    t.ex = extra_shift ? extra_shift[2 * i] : 0.f;
    t.ey = extra_shift ? extra_shift[2 * i + 1] : 0.f;
    F3 u = u_pitch(t, *cfg), v = v_pitch(t, *cfg), n = normal(t, *cfg), d = position(t, *cfg, width, height);
    esb_proj_geom& g = out[i];
    put(g.detektor, d);
    put(g.u_pitch, u);
    put(g.v_pitch, v);
    put(g.proj_norm, n);
    detector_matrix(u, v, n, d, 1.0f, g.detector_matrix);
    double det4 = 0;
    (void)det4;
  }
  return esb::ok();
}

int esb_volume_geometry(const int dim[3], int subvol_count, int subvol, const float voxel_size[3],
                        const float volume_shift[3], esb_vol_geom* out) {
  if (!dim || !voxel_size || !out || subvol_count < 1 || subvol < 0 || subvol >= subvol_count || dim[0] <= 0 ||
      dim[1] <= 0 || dim[2] <= 0)
    return esb::fail(ESB_ERR_INVALID_ARGUMENT, "esb_volume_geometry: invalid argument");
  // Volume(aDim, aSubVolCount, aSubVol) (Volume.cpp:82-114)
  int sizeZ = (int)ceil((double)dim[2] / (double)subvol_count);
  int rest = dim[2] - sizeZ * (subvol_count - 1);
  if (rest <= 0) return esb::fail(ESB_ERR_INVALID_ARGUMENT, "esb_volume_geometry: too many sub-volumes for dim.z");
  float vs[3] = {voxel_size[0], voxel_size[1], voxel_size[2]};
  float sh[3] = {volume_shift ? volume_shift[0] : 0.f, volume_shift ? volume_shift[1] : 0.f,
                 volume_shift ? volume_shift[2] : 0.f};
  // PositionInSpace(aVoxelSize, aVolShift, aShiftXY = 0) (Volume.cpp:270-287)
  float pos[3];
  pos[0] = vs[0] * (-0.5f * (float)(unsigned)dim[0]) + 0.0f - sh[0];
  pos[1] = vs[1] * (-0.5f * (float)(unsigned)dim[1]) + 0.0f - sh[1];
  pos[2] = vs[2] * (-0.5f * (float)(unsigned)dim[2]) - sh[2];
  int before = 0;
  for (int i = 0; i < subvol; ++i) before += sizeZ;
  int subz = (subvol == subvol_count - 1) ? rest : sizeZ;
  esb_vol_geom& g = *out;
  g.bbox_min[0] = pos[0];
  g.bbox_min[1] = pos[1];
  g.bbox_min[2] = pos[2] + vs[2] * (float)before;
  g.dim[0] = (float)dim[0];
  g.dim[1] = (float)dim[1];
  g.dim[2] = (float)subz;
  for (int k = 0; k < 3; ++k) {
    float bb = g.dim[k] * vs[k];
    g.bbox_max[k] = g.bbox_min[k] + bb;
    g.bbox_rcp[k] = 1.0f / (g.dim[k] * vs[k]);
    g.voxel_size[k] = vs[k];
    g.full_dim[k] = (float)dim[k];
    g.full_bbox_min[k] = pos[k];
    g.full_bbox_max[k] = pos[k] + (float)dim[k] * vs[k];
  }
  g.z_shift = (float)before;  // Volume::GetSubVolumeZShift (Volume.cpp:152-161)
  return esb::ok();
}

int esb_subvolume_geometry(int size, float vs_sub, const esb_vol_geom* vol, const float pos[3], const float shift[3],
                           esb_vol_geom* out) {
  if (size <= 0 || !vol || !pos || !out)
    return esb::fail(ESB_ERR_INVALID_ARGUMENT, "esb_subvolume_geometry: invalid argument");
  // Volume::PositionInSpace(aVoxelSize, aVoxelSizeSubVolume, vol, pos, shift) (Volume.cpp:289-306)
  float s[3] = {shift ? shift[0] : 0.f, shift ? shift[1] : 0.f, shift ? shift[2] : 0.f};
  esb_vol_geom& g = *out;
  for (int k = 0; k < 3; ++k) {
    float p = vs_sub * (-0.5f * (float)(unsigned)size) + vol->voxel_size[k] * (pos[k] - 1) + s[k] * vol->voxel_size[k] +
              vol->full_bbox_min[k];
    g.bbox_min[k] = p;
    g.dim[k] = (float)size;
    g.voxel_size[k] = vs_sub;
    g.bbox_max[k] = p + (float)size * vs_sub;
    g.bbox_rcp[k] = 1.0f / ((float)size * vs_sub);
    g.full_dim[k] = (float)size;
    g.full_bbox_min[k] = p;
    g.full_bbox_max[k] = g.bbox_max[k];
  }
  g.z_shift = 0.f;
  return esb::ok();
}

int esb_mag_aniso_matrix(float amount, float angle_deg, float dim_x, float dim_y, float out[9]) {
  if (!out) return esb::fail(ESB_ERR_INVALID_ARGUMENT, "esb_mag_aniso_matrix: out is NULL");
  // Reconstructor::GetMagAnistropyMatrix (Reconstructor.cpp:386-426), float matrices
  float angle = angle_deg / 180.0f * (float)M_PI;
  auto rotz = [](float a, float m[3][3]) {
    float c = cosf(a), s = sinf(a);
    float r[3][3] = {{c, -s, 0}, {s, c, 0}, {0, 0, 1}};
    memcpy(m, r, sizeof(r));
  };
  auto mm = [](const float A[3][3], const float B[3][3], float C[3][3]) {
    float T[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        float v = 0;
        for (int i = 0; i < 3; ++i) v += A[r][i] * B[i][c];
        T[r][c] = v;
      }
    memcpy(C, T, sizeof(T));
  };
  float sc[3][3] = {{1, 0, -dim_x / 2.0f}, {0, 1, -dim_y / 2.0f}, {0, 0, 1}};
  float sb[3][3] = {{1, 0, dim_x / 2.0f}, {0, 1, dim_y / 2.0f}, {0, 0, 1}};
  float st[3][3] = {{amount, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  float r1[3][3], r2[3][3], acc[3][3];
  rotz(angle, r1);
  rotz(-angle, r2);
  mm(sb, r2, acc);
  mm(acc, st, acc);
  mm(acc, r1, acc);
  mm(acc, sc, acc);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) out[3 * r + c] = acc[r][c];
  return esb::ok();
}

int esb_rotation_matrix(float phi, float psi, float theta, float out[9]) {
  if (!out) return esb::fail(ESB_ERR_INVALID_ARGUMENT, "esb_rotation_matrix: out is NULL");
  // RotKernel::computeRotMat (Kernels.cpp:1227-1327): ZXZ Euler angles in
  // degrees; multiples of 30 and 45 degrees in [0, 330] take exact cosines
  // and sines (the square roots in float), other angles cosf / sinf of the
  // angle in radians.
  const float r3 = sqrtf(3.0f) / 2.0f, r2 = sqrtf(2.0f) / 2.0f;
  static const float deg[16] = {0, 30, 45, 60, 90, 120, 135, 150, 180, 210, 225, 240, 270, 300, 315, 330};
  const float cs[16] = {1.0f, r3, r2, 0.5f, 0.0f, -0.5f, -r2, -r3, -1.0f, -r3, -r2, -0.5f, 0.0f, 0.5f, r2, r3};
  const float sn[16] = {0.0f, 0.5f, r2, r3, 1.0f, r3, r2, 0.5f, 0.0f, -0.5f, -r2, -r3, -1.0f, -r3, -r2, -0.5f};
  auto cos_sin = [&](float a, float& c, float& s) {
    for (int i = 0; i < 16; ++i)
      if (deg[i] == a) {
        c = cs[i];
        s = sn[i];
        return;
      }
    const float r = a * (float)M_PI / 180.0f;
    c = cosf(r);
    s = sinf(r);
  };
  float cphi, sphi, cpsi, spsi, cth, sth;
  cos_sin(phi, cphi, sphi);
  cos_sin(psi, cpsi, spsi);
  cos_sin(theta, cth, sth);
  float R[3][3];
  R[0][0] = cpsi * cphi - cth * spsi * sphi;
  R[1][0] = spsi * cphi + cth * cpsi * sphi;
  R[2][0] = sth * sphi;
  R[0][1] = -cpsi * sphi - cth * spsi * cphi;
  R[1][1] = -spsi * sphi + cth * cpsi * cphi;
  R[2][1] = sth * cphi;
  R[0][2] = sth * spsi;
  R[1][2] = -sth * cpsi;
  R[2][2] = cth;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) out[3 * r + c] = R[r][c];
  return esb::ok();
}

int esb_set_constant_values(const esb_proj_geom* p, const esb_vol_geom* v, const float mag_aniso[9],
                            const float mag_aniso_inv[9], int for_bp, esb_constants* out) {
  if (!p || !v || !out) return esb::fail(ESB_ERR_INVALID_ARGUMENT, "esb_set_constant_values: NULL argument");
  memset(out, 0, sizeof(*out));
  for (int k = 0; k < 3; ++k) {
    out->proj_norm[k] = p->proj_norm[k];
    out->detektor[k] = p->detektor[k];
    out->u_pitch[k] = p->u_pitch[k];
    out->v_pitch[k] = p->v_pitch[k];
    out->bbox_min[k] = v->bbox_min[k];
    out->bbox_max[k] = v->bbox_max[k];
    out->bbox_rcp[k] = v->bbox_rcp[k];
    out->volume_dim[k] = v->dim[k];
    out->voxel_size[k] = v->voxel_size[k];
  }
  out->z_shift = for_bp ? v->z_shift : 0.0f;
  out->volume_dim_x_quarter = (int)v->full_dim[0] / 4;
  memcpy(out->detector_matrix, p->detector_matrix, sizeof(out->detector_matrix));
  static const float ident[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  memcpy(out->mag_aniso, mag_aniso ? mag_aniso : ident, sizeof(out->mag_aniso));
  memcpy(out->mag_aniso_inv, mag_aniso_inv ? mag_aniso_inv : ident, sizeof(out->mag_aniso_inv));
  return esb::ok();
}

int esb_compute_hit_points(const esb_proj_geom* p, const esb_vol_geom* v, int out[8]) {
  if (!p || !v || !out) return esb::fail(ESB_ERR_INVALID_ARGUMENT, "esb_compute_hit_points: NULL argument");
  // Projection::ComputeHitPoints (Projection.cpp:850-1049), on the whole volume's bbox
  F3 mn = from(v->full_bbox_min), mx = from(v->full_bbox_max);
  F3 det = from(p->detektor), n = from(p->proj_norm);
  F3 P[8];
  for (int c = 0; c < 8; ++c) {
    F3 q = f3((c & 4) ? mn.x + (mx.x - mn.x) : mn.x, (c & 2) ? mn.y + (mx.y - mn.y) : mn.y,
              (c & 1) ? mn.z + (mx.z - mn.z) : mn.z);
    float t = (n.x * q.x + n.y * q.y + n.z * q.z);
    t += (-n.x * det.x - n.y * det.y - n.z * det.z);
    t = fabsf(t);
    P[c] = f3(t * (-n.x) + q.x, t * (-n.y) + q.y, t * (-n.z) + q.z);
    P[c] = detmul(p->detector_matrix, P[c]);
  }
  auto pick = [](float a, float b) -> int { return (int)(fabsf(a) < fabsf(b) ? a : b); };
  out[0] = pick(P[0].x, P[1].x);
  out[1] = pick(P[0].y, P[1].y);
  out[2] = pick(P[2].x, P[3].x);
  out[3] = pick(P[2].y, P[3].y);
  out[4] = pick(P[4].x, P[5].x);
  out[5] = pick(P[4].y, P[5].y);
  out[6] = pick(P[6].x, P[7].x);
  out[7] = pick(P[6].y, P[7].y);
  return esb::ok();
}

int esb_defocus_distances(const esb_proj_geom* p, const esb_vol_geom* v, int width, int height, float* t_in,
                          float* t_out) {
  if (!p || !v || !t_in || !t_out) return esb::fail(ESB_ERR_INVALID_ARGUMENT, "esb_defocus_distances: NULL argument");
  // Reconstructor::GetDefocusDistances (Reconstructor.cpp:53-173)
  F3 n = from(p->proj_norm), det = from(p->detektor);
  F3 mn = from(v->full_bbox_min), mx = from(v->full_bbox_max), vd = from(v->full_dim), vs = from(v->voxel_size);
  F3 c = f3(mn.x + (vd.x * vs.x * 0.5f), mn.y + (vd.y * vs.y * 0.5f), mn.z + (vd.z * vs.z * 0.5f));
  float t = (n.x * c.x + n.y * c.y + n.z * c.z);
  t += (-n.x * det.x - n.y * det.y - n.z * det.z);
  t = fabsf(t);
  F3 hit = f3(t * (-n.x) + c.x, t * (-n.y) + c.y, t * (-n.z) + c.z);
  hit = detmul(p->detector_matrix, hit);
  int hitX = (int)roundf(hit.x), hitY = (int)roundf(hit.y);
  F3 u = from(p->u_pitch), vv = from(p->v_pitch);
  F3 pos = add(add(det, mul(u, (float)hitX)), mul(vv, (float)hitY));
  (void)width;
  (void)height;
  float tin = 2 * -DIST, tout = 2 * DIST;
  for (int x = 0; x <= 1; x++)
    for (int y = 0; y <= 1; y++)
      for (int z = 0; z <= 1; z++) {
        float tt = (n.x * (mn.x + x * (mx.x - mn.x)) + n.y * (mn.y + y * (mx.y - mn.y)) + n.z * (mn.z + z * (mx.z - mn.z)));
        tt += (-n.x * pos.x - n.y * pos.y - n.z * pos.z);
        if (tt < tin) tin = tt;
        if (tt > tout) tout = tt;
      }
  *t_in = tin;
  *t_out = tout;
  return esb::ok();
}

int esb_defocus_min_max(float ray, float defocus_min_nm, float defocus_max_nm, float tilt_deg, float add_tilt_deg,
                        float pixel_size_nm, float slice_thickness_nm, float volume_shift_z, int ignore_z_shift,
                        int switch_direction, float* out_min, float* out_max) {
  if (!out_min || !out_max) return esb::fail(ESB_ERR_INVALID_ARGUMENT, "esb_defocus_min_max: NULL argument");
  // Reconstructor::GetDefocusMinMax (Reconstructor.cpp:178-201)
  float tiltAngle = (tilt_deg + add_tilt_deg) / 180.0f * (float)M_PI;
  float d = ray + DIST;
  const float T = slice_thickness_nm;
  if (ignore_z_shift)
    d = (roundf(d * pixel_size_nm * T) / T) + T / 2.0f;
  else
    d = (roundf(d * pixel_size_nm * T) / T) + T / 2.0f - (volume_shift_z * pixel_size_nm * cosf(tiltAngle));
  if (switch_direction) d *= -1;
  *out_min = defocus_min_nm + d;
  *out_max = defocus_max_nm + d;
  return esb::ok();
}

int esb_projection_index_list(int type, int n_proj, const float* tilt_deg, const int* good, int* out, int* count) {
  if (n_proj <= 0 || !out || !count || (type == 2 && !tilt_deg))
    return esb::fail(ESB_ERR_INVALID_ARGUMENT, "esb_projection_index_list: invalid argument");
  // Projection::CreateProjectionIndexList (Projection.cpp:561-640)
  int cnt = 0;
  for (int i = 0; i < n_proj; ++i)
    if (!good || good[i]) out[cnt++] = i;
  if (type == 1 || type == 2) {
    srand(0);
    for (int i = 0; i < cnt - 1; i++) {
      int r = i + (rand() % (cnt - i));
      std::swap(out[i], out[r]);
    }
  }
  if (type == 2) {
    // Projection::GetMinimumTiltIndex (Projection.cpp:405-423): first |tilt| minimum
    float minTilt = FLT_MAX;
    int minIdx = 0;
    for (int i = 0; i < n_proj; i++)
      if (fabsf(tilt_deg[i]) < minTilt) {
        minTilt = fabsf(tilt_deg[i]);
        minIdx = i;
      }
    for (int i = 0; i < cnt; i++)
      if (out[i] == minIdx) {
        std::swap(out[0], out[i]);
        break;
      }
  } else if (type != 0 && type != 1) {
    return esb::fail(ESB_ERR_INVALID_ARGUMENT, "esb_projection_index_list: unknown list type");
  }
  *count = cnt;
  return esb::ok();
}

}  // extern "C"
