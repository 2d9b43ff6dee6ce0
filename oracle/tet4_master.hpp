// Oracle (test infrastructure only): CPU FP64 restatement of the tet4
// control-volume master element (Nalu TetSCS / TetSCV and the tri3 face
// element Tri3DSCS) as OpenAccel's assemblers call it.
//
// This file is a checker, never part of the shipped GPU path. It restates:
//   - ip tables            external/nalu/src/master_element/Tet4CVFEM.C:321-446
//                          (lrscv_, intgLoc_, intgLocShift_, ipNodeMap_,
//                          sideNodeOrdinals_) and :59-90 (TetSCV)
//   - SCS area vectors     MasterElementWork.F:608-752 (tet_scs_det),
//                          CalculateQuadArea.F (quadAreaByTriangleFacets)
//   - SCV volumes          MasterElementWork.F:459-606 (tet_scv_det),
//                          CalculateHexVolume.F, CalculatePolyhedralVolume.F
//   - derivatives          MasterElementWork.F:2539-2582 (tet_derivative)
//   - gradient operator    MasterElementWork.F:3061-3216 (tet_gradient_operator)
//   - shape functions      Tet4CVFEM.C:836-853 (TetSCS::tet_shape_fcn)
//   - boundary faces       MasterElement.C:610-716 (Tri3DSCS tables and
//                          tri_shape_fcn), MasterElementWork.F:1589-1698
//                          (tri3d_scs_det)
// Layouts: coords[node][3], areav[ip][3], gradop[node][3] (the tet4 gradient is
// the same at every ip), shape[ip][node].
#pragma once
#include "hex8_master.hpp"

namespace oracle {
namespace tet4 {

constexpr int NPE = 4;
constexpr int NSCS = 6;
constexpr int NSCV = 4;

// L/R node pair of each SCS ip (Tet4CVFEM.C:329-335).
constexpr int LR[NSCS][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};

// Standard and shifted (edge-midpoint) ip locations (Tet4CVFEM.C:365-382).
constexpr double IP_STD[NSCS][3] = {
    {13.0 / 36.0, 5.0 / 36.0, 5.0 / 36.0},  {13.0 / 36.0, 13.0 / 36.0, 5.0 / 36.0},
    {5.0 / 36.0, 13.0 / 36.0, 5.0 / 36.0},  {5.0 / 36.0, 5.0 / 36.0, 13.0 / 36.0},
    {13.0 / 36.0, 5.0 / 36.0, 13.0 / 36.0}, {5.0 / 36.0, 13.0 / 36.0, 13.0 / 36.0}};
constexpr double IP_SHIFT[NSCS][3] = {{0.5, 0.0, 0.0}, {0.5, 0.5, 0.0}, {0.0, 0.5, 0.0},
                                      {0.0, 0.0, 0.5}, {0.5, 0.0, 0.5}, {0.0, 0.5, 0.5}};

// Face ordinal -> element nodes, outward orientation (Tet4CVFEM.C:416-421).
// Boundary ip k of a face is nearest to element node SIDE_NODES[f][k]
// (ipNodeMap_, Tet4CVFEM.C:406-414).
constexpr int SIDE_NODES[4][3] = {{0, 1, 3}, {1, 2, 3}, {0, 3, 2}, {0, 2, 1}};

// Sub-surface quads and sub-volume hexes within the 15-point subdivision
// (tet_scs_det TetEdgeFacetTable, tet_scv_det TetSubcontrolNodeTable; 0-based).
constexpr int SCS_QUAD[NSCS][4] = {{4, 7, 14, 13},  {7, 14, 10, 5}, {6, 12, 14, 7},
                                   {11, 13, 14, 12}, {13, 9, 10, 14}, {10, 8, 12, 14}};
constexpr int SCV_HEX[NSCV][8] = {{0, 4, 7, 6, 11, 13, 14, 12},
                                  {1, 5, 7, 4, 9, 10, 14, 13},
                                  {2, 6, 7, 5, 8, 12, 14, 10},
                                  {3, 9, 13, 11, 8, 10, 14, 12}};

// 0-3 vertices, 4-6 and 8,9,11 edge midpoints, 7,10,12,13 face centroids,
// 14 the centroid, with the reference's operation order.
inline void subdivide(const double* x /*[4][3]*/, double p[15][3]) {
  const double half = 0.5, third = 1.0 / 3.0;
  for (int n = 0; n < 4; ++n)
    for (int k = 0; k < 3; ++k) p[n][k] = x[3 * n + k];
  for (int k = 0; k < 3; ++k) {
    const double x0 = x[k], x1 = x[3 + k], x2 = x[6 + k], x3 = x[9 + k];
    p[4][k] = half * (x0 + x1);
    p[5][k] = half * (x1 + x2);
    p[6][k] = half * (x2 + x0);
    p[7][k] = third * (x0 + x1 + x2);
    p[8][k] = half * (x2 + x3);
    p[9][k] = half * (x3 + x1);
    p[10][k] = third * (x1 + x2 + x3);
    p[11][k] = half * (x0 + x3);
    p[12][k] = third * (x0 + x2 + x3);
    p[13][k] = third * (x0 + x1 + x3);
    double c = 0.0;
    c = c + 0.25 * x0;
    c = c + 0.25 * x1;
    c = c + 0.25 * x2;
    c = c + 0.25 * x3;
    p[14][k] = c;
  }
}

// SCS area vectors areav[6][3], pointing from L to R.
inline void scs_areav(const double* x, double* areav) {
  double p[15][3];
  subdivide(x, p);
  for (int ip = 0; ip < NSCS; ++ip) {
    double q[4][3];
    for (int v = 0; v < 4; ++v)
      for (int k = 0; k < 3; ++k) q[v][k] = p[SCS_QUAD[ip][v]][k];
    hex8::quad_area(q, &areav[3 * ip]);
  }
}

// SCV volumes vol[4]; returns true when all are non-negative.
inline bool scv_volumes(const double* x, double* vol) {
  double p[15][3];
  subdivide(x, p);
  bool ok = true;
  for (int c = 0; c < NSCV; ++c) {
    double v[8][3];
    for (int n = 0; n < 8; ++n)
      for (int k = 0; k < 3; ++k) v[n][k] = p[SCV_HEX[c][n]][k];
    vol[c] = hex8::hex_volume(v);
    if (vol[c] < 0.0) ok = false;
  }
  return ok;
}

// Constant shape-function derivative table (tet_derivative).
constexpr double DERIV[4][3] = {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};

// dN/dx gradop[4][3] (tet_gradient_operator). Returns 1 when the Jacobian
// determinant is <= 1e6 * DBL_MIN (the determinant is then taken as 1).
inline int grad_op(const double* x, double* g) {
  double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // J[coord][param]
  for (int n = 0; n < 4; ++n)
    for (int c = 0; c < 3; ++c)
      for (int s = 0; s < 3; ++s) J[c][s] = J[c][s] + DERIV[n][s] * x[3 * n + c];
  const double dx1 = J[0][0], dx2 = J[0][1], dx3 = J[0][2];
  const double dy1 = J[1][0], dy2 = J[1][1], dy3 = J[1][2];
  const double dz1 = J[2][0], dz2 = J[2][1], dz3 = J[2][2];
  double det = dx1 * (dy2 * dz3 - dz2 * dy3) + dy1 * (dz2 * dx3 - dx2 * dz3) + dz1 * (dx2 * dy3 - dy2 * dx3);
  int err = 0;
  if (det <= 1.0e6 * 2.2250738585072014e-308) {
    det = 1.0;
    err = 1;
  }
  const double d = 1.0 / det;
  const double s1x = d * (dy2 * dz3 - dz2 * dy3), s2x = d * (dz1 * dy3 - dy1 * dz3),
               s3x = d * (dy1 * dz2 - dz1 * dy2);
  const double s1y = d * (dz2 * dx3 - dx2 * dz3), s2y = d * (dx1 * dz3 - dz1 * dx3),
               s3y = d * (dz1 * dx2 - dx1 * dz2);
  const double s1z = d * (dx2 * dy3 - dy2 * dx3), s2z = d * (dy1 * dx3 - dx1 * dy3),
               s3z = d * (dx1 * dy2 - dy1 * dx2);
  for (int n = 0; n < 4; ++n) {
    const double* D = DERIV[n];
    g[3 * n + 0] = D[0] * s1x + D[1] * s2x + D[2] * s3x;
    g[3 * n + 1] = D[0] * s1y + D[1] * s2y + D[2] * s3y;
    g[3 * n + 2] = D[0] * s1z + D[1] * s2z + D[2] * s3z;
  }
  return err;
}

// Barycentric shape functions at the SCS ips, shape[6][4].
inline void scs_shape(double* N, bool shifted) {
  for (int ip = 0; ip < NSCS; ++ip) {
    const double* q = shifted ? IP_SHIFT[ip] : IP_STD[ip];
    N[4 * ip + 0] = 1.0 - q[0] - q[1] - q[2];
    N[4 * ip + 1] = q[0];
    N[4 * ip + 2] = q[1];
    N[4 * ip + 3] = q[2];
  }
}

// Tri3 face: ip locations (standard 7/36, 11/18; shifted at the vertices) and
// shape functions shape[3 ip][3 face nodes].
inline void face_shape(double* N, bool shifted) {
  const double a = 7.0 / 36.0, b = 11.0 / 18.0;
  const double std_loc[3][2] = {{a, a}, {b, a}, {a, b}};
  const double sh_loc[3][2] = {{0.0, 0.0}, {1.0, 0.0}, {0.0, 1.0}};
  for (int ip = 0; ip < 3; ++ip) {
    const double* q = shifted ? sh_loc[ip] : std_loc[ip];
    N[3 * ip + 0] = 1.0 - q[0] - q[1];
    N[3 * ip + 1] = q[0];
    N[3 * ip + 2] = q[1];
  }
}

// Exposed-face area vectors areav[3][3] of a tri3 face given its nodes in side
// order (tri3d_scs_det): ip k owns the quad (vertex k, edge mids, centroid).
inline void tri_face_areav(const double* p /*[3][3]*/, double* area) {
  const double half = 0.5, third = 1.0 / 3.0;
  double e[3][3], c[3];
  for (int d = 0; d < 3; ++d) {
    e[0][d] = (p[d] + p[3 + d]) * half;
    e[1][d] = (p[3 + d] + p[6 + d]) * half;
    e[2][d] = (p[6 + d] + p[d]) * half;
    c[d] = (p[d] + p[3 + d] + p[6 + d]) * third;
  }
  // ip k: diagonals (centroid - vertex k) and (e[k-1] - e[k])
  for (int k = 0; k < 3; ++k) {
    const int em = (k + 2) % 3;
    const double dx13 = c[0] - p[3 * k], dx24 = e[em][0] - e[k][0];
    const double dy13 = c[1] - p[3 * k + 1], dy24 = e[em][1] - e[k][1];
    const double dz13 = c[2] - p[3 * k + 2], dz24 = e[em][2] - e[k][2];
    area[3 * k + 0] = half * (dz24 * dy13 - dz13 * dy24);
    area[3 * k + 1] = half * (dx24 * dz13 - dx13 * dz24);
    area[3 * k + 2] = half * (dy24 * dx13 - dy13 * dx24);
  }
}

}  // namespace tet4
}  // namespace oracle
