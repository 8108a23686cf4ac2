// Test harness around the reference's own file readers and writers
// (src/EmTools/FileIO/{EmFile,MRCFile,MarkerFile,CtfFile}.cpp, compiled
// unmodified from the reference tree by oracle/ref_fileio/build.py).
//
// TEST INFRASTRUCTURE ONLY: tests/test_fileio.py runs it to check that the
// files artiatomi_b200.fileio writes read back identically through the
// reference's classes, and that files the reference writes read back
// identically through artiatomi_b200.fileio.
//
//   ref_fileio read FILE                     header and data summary
//   ref_fileio write_em FILE nx ny nz ps     float ramp data, EmFile writer
//   ref_fileio write_mrc FILE nx ny nz ps    float ramp data, MRCFile writer
//   ref_fileio markers FILE ref              per projection: tilt xshift yshift mag psi good
//   ref_fileio ctf FILE n                    per projection: min max angle
//   ref_fileio motl FILE scale_pos scale_shift  per particle: coords, shifts, index coding
//   ref_fileio shifts FILE                   per projection and motive: extra shift x y
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "CtfFile.h"
#include "EmFile.h"
#include "MRCFile.h"
#include "MarkerFile.h"
#include "MotiveListe.h"
#include "ShiftFile.h"

static double sum_of(void* data, DataType_enum t, size_t n) {
  double s = 0;
  for (size_t i = 0; i < n; ++i) {
    switch (t) {
      case DT_UCHAR: s += ((unsigned char*)data)[i]; break;
      case DT_SHORT: s += ((short*)data)[i]; break;
      case DT_USHORT: s += ((unsigned short*)data)[i]; break;
      case DT_INT: s += ((int*)data)[i]; break;
      case DT_FLOAT: s += ((float*)data)[i]; break;
      case DT_DOUBLE: s += ((double*)data)[i]; break;
      default: break;
    }
  }
  return s;
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  std::string op = argv[1], path = argv[2];
  if (op == "read") {
    if (path.find(".em") != std::string::npos) {
      EmFile f(path);
      if (!f.OpenAndRead()) return 3;
      EmHeader& h = f.GetFileHeader();
      size_t n = (size_t)h.DimX * h.DimY * h.DimZ;
      printf("%d %d %d %d %d %.17g\n", h.DimX, h.DimY, h.DimZ, (int)f.GetDataType(), h.ObjectPixelSize,
             sum_of(f.GetData(), f.GetDataType(), n));
    } else {
      MRCFile f(path);
      if (!f.OpenAndRead()) return 3;
      MrcHeader& h = f.GetFileHeader();
      size_t n = (size_t)h.NX * h.NY * h.NZ;
      printf("%d %d %d %d %.9g %.17g\n", (int)h.NX, (int)h.NY, (int)h.NZ, (int)f.GetDataType(), f.GetPixelsize(),
             sum_of(f.GetData(), f.GetDataType(), n));
    }
    return 0;
  }
  if ((op == "write_em" || op == "write_mrc") && argc >= 7) {
    int nx = atoi(argv[3]), ny = atoi(argv[4]), nz = atoi(argv[5]);
    float ps = (float)atof(argv[6]);
    std::vector<float> d((size_t)nx * ny * nz);
    for (size_t i = 0; i < d.size(); ++i) d[i] = 0.5f * (float)i - 7.0f;
    bool ok = op == "write_em" ? EmFile::InitHeader(path, nx, ny, nz, ps, DT_FLOAT) &&
                                     EmFile::WriteRawData(path, d.data(), d.size() * sizeof(float))
                               : MRCFile::InitHeaders(path, nx, ny, nz, ps, DT_FLOAT, false) &&
                                     MRCFile::WriteRawData(path, d.data(), d.size() * sizeof(float));
    return ok ? 0 : 3;
  }
  if (op == "markers" && argc >= 4) {
    MarkerFile m(path, atoi(argv[3]));
    for (int p = 0; p < m.GetTotalProjectionCount(); ++p)
      printf("%.9g %.9g %.9g %.9g %.9g %d\n", m(MFI_TiltAngle, p, 0), m(MFI_X_Shift, p, 0), m(MFI_Y_Shift, p, 0),
             m(MFI_Magnifiaction, p, 0), m(MFI_RotationPsi, p, 0), (int)m.CheckIfProjIndexIsGood(p));
    return 0;
  }
  if (op == "ctf" && argc >= 4) {
    CtfFile c(path);
    for (int i = 0; i < atoi(argv[3]); ++i)
      printf("%.9g %.9g %.9g\n", c.GetMinDefocus(i), c.GetMaxDefocus(i), c.GetAstigmatismAngle(i));
    return 0;
  }
  if (op == "motl" && argc >= 5) {
    MotiveList ml(path, (float)atof(argv[3]), (float)atof(argv[4]));
    for (int i = 0; i < ml.GetParticleCount(); ++i) {
      motive m = ml.GetAt(i);
      printf("%.9g %.9g %.9g %.9g %.9g %.9g %s %s\n", m.x_Coord, m.y_Coord, m.z_Coord, m.x_Shift, m.y_Shift,
             m.z_Shift, m.GetIndexCoding(MotiveList::NC_ParticleOnly).c_str(),
             m.GetIndexCoding(MotiveList::NC_TomogramParticle).c_str());
    }
    return 0;
  }
  if (op == "shifts") {
    ShiftFile sf(path);
    for (int p = 0; p < sf.GetProjectionCount(); ++p)
      for (int m = 0; m < sf.GetMotiveCount(); ++m) {
        my_float2 v = sf(p, m);
        printf("%.9g %.9g\n", v.x, v.y);
      }
    return 0;
  }
  return 2;
}
