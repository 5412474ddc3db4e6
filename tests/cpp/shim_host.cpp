// Host-side checks of the C++ template API in include/raptr_b200.hpp:
// the transform unit cases of src/tests/MeasurementSetupTrafo2CartCoordUT.cu
// (exact, double), index functor bijections and float transforms printed
// for comparison with the oracle.  Prints "ok <name>" / "FAIL <name>" lines.
#include <cmath>
#include <cstdio>

#include "raptr_b200.hpp"

typedef double val_t;
typedef DefaultMeasurementSetup<val_t> MS;
typedef DefaultMeasurementSetupTrafo2CartCoordFirstPixel<val_t, MS> Trafo0;
typedef DefaultMeasurementSetupTrafo2CartCoordSecndPixel<val_t, MS> Trafo1;
typedef DefaultMeasurementSetupTrafo2CartCoordFirstPixel_inplace<val_t, MS> Trafo0i;
typedef DefaultMeasurementSetupTrafo2CartCoordSecndPixel_inplace<val_t, MS> Trafo1i;

static int failures = 0;
static void report(bool ok, const char* name) {
  std::printf("%s %s\n", ok ? "ok" : "FAIL", name);
  if (!ok) failures++;
}

// Setup of the unit test: 4x4 segments, 6 angles of 60 degrees, +-3.5, 1.0 edges.
static MS ut_setup() { return MS(-3.5, 3.5, 6, 4, 4, 4, 4, 60.0, 1.0, 1.0, 1.0); }

static void check_norot(int det, int inplace, double dx, double dy, double dz, const char* name) {
  MS s = ut_setup();
  double pos = det == 0 ? s.pos0x() : s.pos1x();
  int ny = det == 0 ? s.n0y() : s.n1y(), nz = det == 0 ? s.n0z() : s.n1z();
  double want[3] = {pos + (-0.5 + dx) * s.segx(), ((-0.5 * ny + 0) + dy) * s.segy(), ((-0.5 * nz + 0) + dz) * s.segz()};
  double dice[3] = {dx, dy, dz}, out[3] = {0, 0, 0};
  if (inplace) {
    out[0] = dx; out[1] = dy; out[2] = dz;
    if (det == 0) Trafo0i()(out, 0, 0, 0, &s);
    else Trafo1i()(out, 0, 0, 0, &s);
  } else {
    if (det == 0) Trafo0()(out, dice, 0, 0, 0, &s);
    else Trafo1()(out, dice, 0, 0, 0, &s);
  }
  bool eq = out[0] == want[0] && out[1] == want[1] && out[2] == want[2];
  bool screwed = out[0] != want[0] + 1. && out[1] != want[1] + 1. && out[2] != want[2] + 1.;
  report(eq && screwed, name);
}

int main() {
  const double corners[5][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {0.1, 0.1, 0.1}};
  char name[64];
  for (int det = 0; det < 2; det++)
    for (int inplace = 0; inplace < 2; inplace++)
      for (int k = 0; k < 5; k++) {
        std::snprintf(name, sizeof(name), "trafo_det%d_inplace%d_case%d", det, inplace, k);
        check_norot(det, inplace, corners[k][0], corners[k][1], corners[k][2], name);
      }
  {  // rotation 1, corner 000 of det0 (test_MeasurementSetupTrafo2CartCoord_025)
    MS s = ut_setup();
    double dice[3] = {0, 0, 0}, out[3];
    Trafo0()(out, dice, 0, 0, 1, &s);
    double ox = s.pos0x() - 0.5 * s.segx(), oz = -0.5 * s.n0z() * s.segz();
    double sn = sinf(M_PI / 180. * 1 * s.da()), cs = cosf(M_PI / 180. * 1 * s.da());
    double want[3] = {sn * oz + cs * ox, -0.5 * s.n0y() * s.segy(), cs * oz - sn * ox};
    report(std::fabs(out[0] - want[0]) < 1e-12 && std::fabs(out[1] - want[1]) < 1e-12 &&
               std::fabs(out[2] - want[2]) < 1e-12,
           "trafo_rotated_case025");
  }
  {  // channel and voxel index bijections on the full setup and grid
    DefaultMeasurementSetup<float> s(-0.24f, 0.24f, 180, 13, 13, 13, 13, 2.f, 0.02f, 0.004f, 0.004f);
    DefaultMeasurementSetupLinId<DefaultMeasurementSetup<float> > lin;
    bool ok = true;
    for (int c = 0; c < 180 * 28561; c += 977) {
      int id0z = DefaultMeasurementSetupId0z<DefaultMeasurementSetup<float> >()(c, &s);
      int id0y = DefaultMeasurementSetupId0y<DefaultMeasurementSetup<float> >()(c, &s);
      int id1z = DefaultMeasurementSetupId1z<DefaultMeasurementSetup<float> >()(c, &s);
      int id1y = DefaultMeasurementSetupId1y<DefaultMeasurementSetup<float> >()(c, &s);
      int ida = DefaultMeasurementSetupIda<DefaultMeasurementSetup<float> >()(c, &s);
      ok = ok && lin(id0z, id0y, id1z, id1y, ida, &s) == c;
    }
    report(ok, "channel_index_bijection");
    DefaultVoxelGrid<float> g(0.1f, 0.2f, 0.3f, 1.f, 2.f, 3.f, 5, 6, 7);
    ok = true;
    for (int v = 0; v < 5 * 6 * 7; v++) {
      int x = DefaultVoxelGridIdx<DefaultVoxelGrid<float> >()(v, &g);
      int y = DefaultVoxelGridIdy<DefaultVoxelGrid<float> >()(v, &g);
      int z = DefaultVoxelGridIdz<DefaultVoxelGrid<float> >()(v, &g);
      ok = ok && DefaultVoxelGridLinId<DefaultVoxelGrid<float> >()(x, y, z, &g) == v && v == x * 42 + y * 7 + z;
    }
    report(ok, "voxel_index_bijection");
    GridAdapter<DefaultVoxelGrid<float>, float> ga(&g);
    float o[3];
    int n[3];
    ga.getOrigin(o);
    ga.getNumberOfVoxels(n);
    report(o[1] == 0.2f && n[2] == 7, "grid_adapter");
  }
  {  // float transforms of the full setup, printed for the oracle comparison
    DefaultMeasurementSetup<float> s(-0.24f, 0.24f, 180, 13, 13, 13, 13, 2.f, 0.02f, 0.004f, 0.004f);
    DefaultMeasurementSetupTrafo2CartCoordFirstPixel_inplace<float, DefaultMeasurementSetup<float> > t0;
    DefaultMeasurementSetupTrafo2CartCoordSecndPixel_inplace<float, DefaultMeasurementSetup<float> > t1;
    for (int k = 0; k < 8; k++) {
      float p[3] = {0.125f * k, 0.5f, 1.0f - 0.1f * k};
      float q[3] = {p[0], p[1], p[2]};
      t0(p, k, 12 - k, 17 * k, &s);
      t1(q, 12 - k, k, 17 * k, &s);
      std::printf("trafo_f %d %a %a %a %a %a %a\n", k, p[0], p[1], p[2], q[0], q[1], q[2]);
    }
  }
  std::printf("failures %d\n", failures);
  return failures ? 1 : 0;
}
