// Test harness around the reference's own host geometry: Projection
// (src/EmSART/Projection.cpp: RotateMatrix, GetPosition, GetPixelUPitch,
// GetPixelVPitch, GetNormalVector, GetDetectorMatrix, ComputeHitPoints) and
// Volume (src/EmSART/Volume.cpp: the z-slab partition and PositionInSpace),
// configured by the reference's Config (src/EmSART/utils/Config.cpp) and
// MarkerFile (src/EmTools/FileIO/MarkerFile.cpp), all compiled unmodified
// from the reference tree by oracle/ref_geometry/build.py.
//
// TEST INFRASTRUCTURE ONLY: tests/golden/make_geometry_golden.py and
// tests/test_geometry_reference.py run it to pin the library's geometry
// (esb_projection_geometry, esb_volume_geometry, esb_compute_hit_points) to
// the reference's, bit for bit.
//
//   ref_geometry CONFIG MARKERS W H PIXELSIZE_NM NX NY NZ SUBVOLS
//
// prints, per z-slab s: "vol s" and the slab's bbox min, max, rcp,
// dimension and z shift; per projection i: "proj i" and detector corner,
// u and v pitch, normal, detector matrix (os 1), and per slab the hit
// points pA pB pC pD. Floats as C hex literals (%a), exact.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "MarkerFile.h"
#include "Projection.h"
#include "Volume.h"
#include "utils/Config.h"

// The projection stack's metadata (ProjectionSource) without image data:
// the geometry reads only the count, the size and the pixel size.
class ShapeOnlySource : public ProjectionSource {
 public:
  ShapeOnlySource(int n, int w, int h, float ps) : n_(n), w_(w), h_(h), ps_(ps) {}
  DataType_enum GetDataType() { return DT_FLOAT; }
  char* GetProjection(uint) { return nullptr; }
  float GetPixelSize() { return ps_; }
  int GetWidth() { return w_; }
  int GetHeight() { return h_; }
  int GetProjectionCount() { return n_; }

 private:
  int n_, w_, h_;
  float ps_;
};

static void pf3(const char* tag, float3 v) { printf(" %s %a %a %a", tag, v.x, v.y, v.z); }

int main(int argc, char** argv) {
  if (argc < 10) {
    fprintf(stderr, "usage: ref_geometry CONFIG MARKERS W H PIXELSIZE_NM NX NY NZ SUBVOLS\n");
    return 2;
  }
  Configuration::Config& cfg = Configuration::Config::GetConfig(argv[1], 0, nullptr, 0);
  MarkerFile markers(argv[2], cfg.ReferenceMarker);
  const int W = atoi(argv[3]), H = atoi(argv[4]);
  const float ps = (float)atof(argv[5]);
  uint3 dim = make_uint3((unsigned)atoi(argv[6]), (unsigned)atoi(argv[7]), (unsigned)atoi(argv[8]));
  const int nsub = atoi(argv[9]);
  ShapeOnlySource src(markers.GetProjectionCount(), W, H, ps);
  Projection proj(&src, &markers);
  std::vector<Volume<float>*> vols;
  for (int s = 0; s < nsub; ++s) {
    Volume<float>* v = new Volume<float>(dim, nsub, -1);
    v->PositionInSpace(cfg.VoxelSize, cfg.VolumeShift);
    vols.push_back(v);
    printf("vol %d", s);
    pf3("min", v->GetSubVolumeBBoxMin(s));
    pf3("max", v->GetSubVolumeBBoxMax(s));
    pf3("rcp", v->GetSubVolumeBBoxRcp(s));
    pf3("dim", v->GetSubVolumeDimension(s));
    printf(" zshift %a\n", v->GetSubVolumeZShift(s));
  }
  for (int i = 0; i < markers.GetProjectionCount(); ++i) {
    printf("proj %d", i);
    pf3("det", proj.GetPosition(i));
    pf3("u", proj.GetPixelUPitch(i));
    pf3("v", proj.GetPixelVPitch(i));
    pf3("n", proj.GetNormalVector(i));
    float m[16];
    proj.GetDetectorMatrix(i, m, 1);
    printf(" mat");
    for (int k = 0; k < 16; ++k) printf(" %a", m[k]);
    printf("\n");
    for (int s = 0; s < nsub; ++s) {
      int2 a, b, c, d;
      proj.ComputeHitPoints(*vols[s], i, a, b, c, d);
      printf("hit %d %d %d %d %d %d %d %d %d %d\n", i, s, a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y);
    }
  }
  return 0;
}
