// Oracle (test infrastructure only): thin C driver around the reference's own
// hex8 geometry templates, compiled straight from the reference tree
// (external/nalu/include/master_element/Hex8GeometryFunctions.h) into
// oracle/_ref/libnalu_hex8_ref.so by `make -C oracle ref`.
//
// The loops below are HexSCS::determinant and HexSCV::determinant
// (external/nalu/src/master_element/Hex8CVFEM.C:547-581 and :149-178) with
// their subdivision tables; the arithmetic is the reference's
// subdivide_hex_8, quad_area_by_triangulation and hex_volume_grandy. Used to
// pin the oracle restatement (oracle/hex8_master.hpp) in tests.
#include <master_element/Hex8GeometryFunctions.h>

namespace {

struct View2 {  // minimal (i, j) accessor standing in for SharedMemView<double**>
  using value_type = double;
  double* p;
  int ld;
  double& operator()(int i, int j) const { return p[i * ld + j]; }
};

}  // namespace

extern "C" {

void ref_hex8_scs_areav(const double* x, double* areav) {
  constexpr int facet[12][4] = {{20, 8, 12, 26},  {24, 9, 12, 26},  {10, 12, 26, 23}, {11, 25, 26, 12},
                                {13, 20, 26, 17}, {17, 14, 24, 26}, {17, 15, 23, 26}, {16, 17, 26, 25},
                                {19, 20, 26, 25}, {20, 18, 24, 26}, {22, 23, 26, 24}, {21, 25, 26, 23}};
  View2 c{const_cast<double*>(x), 3};
  View2 a{areav, 3};
  double coordv[27][3];
  sierra::nalu::subdivide_hex_8(c, coordv);
  for (int ics = 0; ics < 12; ++ics) {
    double q[4][3];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) q[n][d] = coordv[facet[ics][n]][d];
    sierra::nalu::quad_area_by_triangulation(ics, q, a);
  }
}

void ref_hex8_scv_volumes(const double* x, double* vol) {
  constexpr int sub[8][8] = {{0, 8, 12, 11, 19, 20, 26, 25}, {8, 1, 9, 12, 20, 18, 24, 26},
                             {12, 9, 2, 10, 26, 24, 22, 23}, {11, 12, 10, 3, 25, 26, 23, 21},
                             {19, 20, 26, 25, 4, 13, 17, 16}, {20, 18, 24, 26, 13, 5, 14, 17},
                             {26, 24, 22, 23, 17, 14, 6, 15}, {25, 26, 23, 21, 16, 17, 15, 7}};
  View2 c{const_cast<double*>(x), 3};
  double coordv[27][3];
  sierra::nalu::subdivide_hex_8(c, coordv);
  for (int ip = 0; ip < 8; ++ip) {
    double h[8][3];
    for (int n = 0; n < 8; ++n)
      for (int d = 0; d < 3; ++d) h[n][d] = coordv[sub[ip][n]][d];
    vol[ip] = sierra::nalu::hex_volume_grandy(h);
  }
}

}  // extern "C"
