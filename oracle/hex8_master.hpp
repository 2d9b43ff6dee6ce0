// Oracle (test infrastructure only): CPU FP64 restatement of the hex8
// control-volume master element used by OpenAccel's assemblers.
//
// This file is a checker, never part of the shipped GPU path. It restates,
// in plain C++, the vendored Nalu master-element arithmetic:
//   - ip tables            external/nalu/src/master_element/Hex8CVFEM.C:255-446
//   - SCS area vectors     MasterElementWork.F:1-231 (hex_scs_det),
//                          CalculateQuadArea.F (quadAreaByTriangleFacets)
//   - SCV volumes          MasterElementWork.F:233-457 (hex_scv_det),
//                          CalculateHexVolume.F, CalculatePolyhedralVolume.F
//   - shape functions      MasterElementWork.F:2344-2402 (hex_shape_fcn)
//   - derivatives          MasterElementWork.F:2404-2484 (hex_derivative)
//   - gradient operator    MasterElementWork.F:2623-2774 (hex_gradient_operator)
//   - quad face areas      MasterElementWork.F:1467-1587 (quad3d_scs_det)
//   - quad face shape fns  MasterElementWork.F:3651-3696 (quad3d_shape_fcn)
// Layouts follow the reference call sites: coords[node][3], areav[ip][3],
// gradop[ip][node][3], shape[ip][node].
#pragma once
#include <cmath>

namespace oracle {
namespace hex8 {

constexpr int NPE = 8;    // nodes per element
constexpr int NSCS = 12;  // sub-control surfaces (interior ips)
constexpr int NSCV = 8;   // sub-control volumes

// L/R node pair of each SCS ip (Hex8CVFEM.C:264-276).
constexpr int LR[NSCS][2] = {{0, 1}, {1, 2}, {2, 3}, {0, 3}, {4, 5}, {5, 6},
                             {6, 7}, {4, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

// Standard ip locations on the [-1/2,1/2]^3 reference cube (Hex8CVFEM.C:318-330).
constexpr double IP_STD[NSCS][3] = {
    {0.00, -0.25, -0.25}, {0.25, 0.00, -0.25}, {0.00, 0.25, -0.25},
    {-0.25, 0.00, -0.25}, {0.00, -0.25, 0.25}, {0.25, 0.00, 0.25},
    {0.00, 0.25, 0.25},   {-0.25, 0.00, 0.25}, {-0.25, -0.25, 0.00},
    {0.25, -0.25, 0.00},  {0.25, 0.25, 0.00},  {-0.25, 0.25, 0.00}};

// Shifted ("linear_linear") ip locations: edge midpoints (Hex8CVFEM.C:333-345).
constexpr double IP_SHIFT[NSCS][3] = {
    {0.00, -0.50, -0.50}, {0.50, 0.00, -0.50}, {0.00, 0.50, -0.50},
    {-0.50, 0.00, -0.50}, {0.00, -0.50, 0.50}, {0.50, 0.00, 0.50},
    {0.00, 0.50, 0.50},   {-0.50, 0.00, 0.50}, {-0.50, -0.50, 0.00},
    {0.50, -0.50, 0.00},  {0.50, 0.50, 0.00},  {-0.50, 0.50, 0.00}};

// Corner locations of the reference cube.
constexpr double NODE_LOC[NPE][3] = {{-0.5, -0.5, -0.5}, {0.5, -0.5, -0.5},
                                     {0.5, 0.5, -0.5},   {-0.5, 0.5, -0.5},
                                     {-0.5, -0.5, 0.5},  {0.5, -0.5, 0.5},
                                     {0.5, 0.5, 0.5},    {-0.5, 0.5, 0.5}};

// Face ordinal -> element node ordinals, outward orientation (Hex8CVFEM.C:415-422).
constexpr int FACE_NODES[6][4] = {{0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6},
                                  {0, 4, 7, 3}, {0, 3, 2, 1}, {4, 5, 6, 7}};

// Standard exposed-face ip locations, 4 per face (Hex8CVFEM.C:348-378).
constexpr double FACE_IP_STD[6][4][3] = {
    {{-0.25, -0.50, -0.25}, {0.25, -0.50, -0.25}, {0.25, -0.50, 0.25}, {-0.25, -0.50, 0.25}},
    {{0.50, -0.25, -0.25}, {0.50, 0.25, -0.25}, {0.50, 0.25, 0.25}, {0.50, -0.25, 0.25}},
    {{0.25, 0.50, -0.25}, {-0.25, 0.50, -0.25}, {-0.25, 0.50, 0.25}, {0.25, 0.50, 0.25}},
    {{-0.50, -0.25, -0.25}, {-0.50, -0.25, 0.25}, {-0.50, 0.25, 0.25}, {-0.50, 0.25, -0.25}},
    {{-0.25, -0.25, -0.50}, {-0.25, 0.25, -0.50}, {0.25, 0.25, -0.50}, {0.25, -0.25, -0.50}},
    {{-0.25, -0.25, 0.50}, {0.25, -0.25, 0.50}, {0.25, 0.25, 0.50}, {-0.25, 0.25, 0.50}}};

// Exposed-face ip k of a face sits nearest to face node k (Hex8CVFEM.C:381-393),
// i.e. element node FACE_NODES[f][k].

// The 27-point subdivision used by hex_scs_det/hex_scv_det
// (MasterElementWork.F:60-200): 0-7 vertices, then edge midpoints, face
// centroids and the element centroid, in the reference's numbering.
inline void subdivide(const double* x /*[8][3]*/, double p[27][3]) {
  for (int n = 0; n < 8; ++n)
    for (int k = 0; k < 3; ++k) p[n][k] = x[3 * n + k];
  auto mid = [&](int o, int a, int b) {
    for (int k = 0; k < 3; ++k) p[o][k] = 0.5 * (x[3 * a + k] + x[3 * b + k]);
  };
  auto quad = [&](int o, int a, int b, int c, int d) {
    for (int k = 0; k < 3; ++k)
      p[o][k] = 0.25 * (x[3 * a + k] + x[3 * b + k] + x[3 * c + k] + x[3 * d + k]);
  };
  mid(8, 0, 1);
  mid(9, 1, 2);
  mid(10, 2, 3);
  mid(11, 3, 0);
  quad(12, 0, 1, 2, 3);
  mid(13, 4, 5);
  mid(14, 5, 6);
  mid(15, 6, 7);
  mid(16, 7, 4);
  quad(17, 4, 5, 6, 7);
  mid(18, 1, 5);
  mid(19, 0, 4);
  quad(20, 0, 1, 4, 5);
  mid(21, 3, 7);
  mid(22, 2, 6);
  quad(23, 2, 3, 6, 7);
  quad(24, 1, 2, 5, 6);
  quad(25, 0, 3, 4, 7);
  for (int k = 0; k < 3; ++k) {
    double s = 0.0;
    for (int n = 0; n < 8; ++n) s += x[3 * n + k];
    p[26][k] = 0.125 * s;
  }
}

// Vertices of each SCS quad within the subdivision (MasterElementWork.F:38-50,
// converted to 0-based).
constexpr int SCS_QUAD[NSCS][4] = {{20, 8, 12, 26},  {24, 9, 12, 26},
                                   {10, 12, 26, 23}, {11, 25, 26, 12},
                                   {13, 20, 26, 17}, {17, 14, 24, 26},
                                   {17, 15, 23, 26}, {16, 17, 26, 25},
                                   {19, 20, 26, 25}, {20, 18, 24, 26},
                                   {22, 23, 26, 24}, {21, 25, 26, 23}};

// Vertices of each SCV sub-hex within the subdivision (MasterElementWork.F:262-270).
constexpr int SCV_HEX[NSCV][8] = {
    {0, 8, 12, 11, 19, 20, 26, 25}, {8, 1, 9, 12, 20, 18, 24, 26},
    {12, 9, 2, 10, 26, 24, 22, 23}, {11, 12, 10, 3, 25, 26, 23, 21},
    {19, 20, 26, 25, 4, 13, 17, 16}, {20, 18, 24, 26, 13, 5, 14, 17},
    {26, 24, 22, 23, 17, 14, 6, 15}, {25, 26, 23, 21, 16, 17, 15, 7}};

// Area vector of a quad by four triangles about its vertex mean
// (CalculateQuadArea.F).
inline void quad_area(const double q[4][3], double a[3]) {
  double m[3];
  for (int k = 0; k < 3; ++k) m[k] = 0.25 * (q[0][k] + q[1][k] + q[2][k] + q[3][k]);
  a[0] = a[1] = a[2] = 0.0;
  double r2[3] = {q[0][0] - m[0], q[0][1] - m[1], q[0][2] - m[2]};
  for (int t = 0; t < 4; ++t) {
    const int nxt = (t + 1) % 4;
    const double r1[3] = {r2[0], r2[1], r2[2]};
    for (int k = 0; k < 3; ++k) r2[k] = q[nxt][k] - m[k];
    a[0] += r1[1] * r2[2] - r2[1] * r1[2];
    a[1] += r1[2] * r2[0] - r2[2] * r1[0];
    a[2] += r1[0] * r2[1] - r2[0] * r1[1];
  }
  for (int k = 0; k < 3; ++k) a[k] *= 0.5;
}

// SCS area vectors, areav[ip][3], pointing from L to R (hex_scs_det).
inline void scs_areav(const double* x, double* areav) {
  double p[27][3];
  subdivide(x, p);
  for (int ip = 0; ip < NSCS; ++ip) {
    double q[4][3];
    for (int v = 0; v < 4; ++v)
      for (int k = 0; k < 3; ++k) q[v][k] = p[SCS_QUAD[ip][v]][k];
    quad_area(q, &areav[3 * ip]);
  }
}

// Hex volume by 24 triangular facets (Grandy's method; CalculateHexVolume.F
// + polyhedralVolumeByFaces in CalculatePolyhedralVolume.F).
constexpr int HEXVOL_TRI[24][3] = {
    {0, 8, 1},  {8, 2, 1},  {3, 2, 8},  {3, 8, 0},  {6, 9, 5},   {7, 9, 6},
    {4, 9, 7},  {4, 5, 9},  {10, 0, 1}, {5, 10, 1}, {4, 10, 5},  {4, 0, 10},
    {7, 6, 11}, {6, 2, 11}, {2, 3, 11}, {3, 7, 11}, {6, 12, 2},  {5, 12, 6},
    {5, 1, 12}, {1, 2, 12}, {0, 4, 13}, {4, 7, 13}, {7, 3, 13},  {3, 0, 13}};

inline double hex_volume(const double v[8][3]) {
  double c[14][3];
  for (int n = 0; n < 8; ++n)
    for (int k = 0; k < 3; ++k) c[n][k] = v[n][k];
  auto quad = [&](int o, int a, int b, int cc, int d) {
    for (int k = 0; k < 3; ++k) c[o][k] = 0.25 * (v[a][k] + v[b][k] + v[cc][k] + v[d][k]);
  };
  quad(8, 0, 1, 2, 3);
  quad(9, 4, 5, 6, 7);
  quad(10, 0, 1, 5, 4);
  quad(11, 3, 2, 6, 7);
  quad(12, 1, 2, 6, 5);
  quad(13, 0, 3, 7, 4);
  double vol = 0.0;
  for (int t = 0; t < 24; ++t) {
    const double* P = c[HEXVOL_TRI[t][0]];
    const double* Q = c[HEXVOL_TRI[t][1]];
    const double* R = c[HEXVOL_TRI[t][2]];
    const double f0 = P[0] + Q[0] + R[0], f1 = P[1] + Q[1] + R[1], f2 = P[2] + Q[2] + R[2];
    vol += f0 * ((Q[1] - P[1]) * (R[2] - P[2]) - (R[1] - P[1]) * (Q[2] - P[2])) -
           f1 * ((Q[0] - P[0]) * (R[2] - P[2]) - (R[0] - P[0]) * (Q[2] - P[2])) +
           f2 * ((Q[0] - P[0]) * (R[1] - P[1]) - (R[0] - P[0]) * (Q[1] - P[1]));
  }
  return vol / 18.0;
}

// SCV volumes vol[8] (hex_scv_det). Returns true when all are positive.
inline bool scv_volumes(const double* x, double* vol) {
  double p[27][3];
  subdivide(x, p);
  bool ok = true;
  for (int c = 0; c < NSCV; ++c) {
    double v[8][3];
    for (int n = 0; n < 8; ++n)
      for (int k = 0; k < 3; ++k) v[n][k] = p[SCV_HEX[c][n]][k];
    vol[c] = hex_volume(v);
    if (vol[c] < 0.0) ok = false;
  }
  return ok;
}

// Trilinear shape functions at parametric point s (hex_shape_fcn).
inline void shape(const double* s, double N[8]) {
  const double s1 = s[0], s2 = s[1], s3 = s[2];
  const double h = 0.5, q = 0.25, e = 0.125;
  N[0] = e + q * (-s1 - s2 - s3) + h * (s2 * s3 + s3 * s1 + s1 * s2) - s1 * s2 * s3;
  N[1] = e + q * (s1 - s2 - s3) + h * (s2 * s3 - s3 * s1 - s1 * s2) + s1 * s2 * s3;
  N[2] = e + q * (s1 + s2 - s3) + h * (-s2 * s3 - s3 * s1 + s1 * s2) - s1 * s2 * s3;
  N[3] = e + q * (-s1 + s2 - s3) + h * (-s2 * s3 + s3 * s1 - s1 * s2) + s1 * s2 * s3;
  N[4] = e + q * (-s1 - s2 + s3) + h * (-s2 * s3 - s3 * s1 + s1 * s2) + s1 * s2 * s3;
  N[5] = e + q * (s1 - s2 + s3) + h * (-s2 * s3 + s3 * s1 - s1 * s2) - s1 * s2 * s3;
  N[6] = e + q * (s1 + s2 + s3) + h * (s2 * s3 + s3 * s1 + s1 * s2) + s1 * s2 * s3;
  N[7] = e + q * (-s1 + s2 + s3) + h * (s2 * s3 - s3 * s1 - s1 * s2) - s1 * s2 * s3;
}

// Parametric derivatives dN[n][d] at s (hex_derivative).
inline void deriv(const double* s, double dN[8][3]) {
  const double s1 = s[0], s2 = s[1], s3 = s[2];
  const double h = 0.5, q = 0.25;
  const double s12 = s1 * s2, s23 = s2 * s3, s13 = s1 * s3;
  dN[0][0] = h * (s3 + s2) - s23 - q;
  dN[1][0] = h * (-s3 - s2) + s23 + q;
  dN[2][0] = h * (-s3 + s2) - s23 + q;
  dN[3][0] = h * (s3 - s2) + s23 - q;
  dN[4][0] = h * (-s3 + s2) + s23 - q;
  dN[5][0] = h * (s3 - s2) - s23 + q;
  dN[6][0] = h * (s3 + s2) + s23 + q;
  dN[7][0] = h * (-s3 - s2) - s23 - q;
  dN[0][1] = h * (s3 + s1) - s13 - q;
  dN[1][1] = h * (s3 - s1) + s13 - q;
  dN[2][1] = h * (-s3 + s1) - s13 + q;
  dN[3][1] = h * (-s3 - s1) + s13 + q;
  dN[4][1] = h * (-s3 + s1) + s13 - q;
  dN[5][1] = h * (-s3 - s1) - s13 - q;
  dN[6][1] = h * (s3 + s1) + s13 + q;
  dN[7][1] = h * (s3 - s1) - s13 + q;
  dN[0][2] = h * (s2 + s1) - s12 - q;
  dN[1][2] = h * (s2 - s1) + s12 - q;
  dN[2][2] = h * (-s2 - s1) - s12 - q;
  dN[3][2] = h * (-s2 + s1) + s12 - q;
  dN[4][2] = h * (-s2 - s1) + s12 + q;
  dN[5][2] = h * (-s2 + s1) - s12 + q;
  dN[6][2] = h * (s2 + s1) + s12 + q;
  dN[7][2] = h * (s2 - s1) - s12 + q;
}

// Physical gradients g[n][3] of the shape functions at parametric point s
// (hex_gradient_operator). Returns det(J); a determinant below 1e6*realmin is
// flagged (err=1) and replaced by 1, as in the reference.
inline double grad_op_at(const double* s, const double* x, double* g /*[8][3]*/, int* err) {
  double dN[8][3];
  deriv(s, dN);
  double xs1 = 0, xs2 = 0, xs3 = 0, ys1 = 0, ys2 = 0, ys3 = 0, zs1 = 0, zs2 = 0, zs3 = 0;
  for (int n = 0; n < 8; ++n) {
    xs1 += dN[n][0] * x[3 * n + 0];
    xs2 += dN[n][1] * x[3 * n + 0];
    xs3 += dN[n][2] * x[3 * n + 0];
    ys1 += dN[n][0] * x[3 * n + 1];
    ys2 += dN[n][1] * x[3 * n + 1];
    ys3 += dN[n][2] * x[3 * n + 1];
    zs1 += dN[n][0] * x[3 * n + 2];
    zs2 += dN[n][1] * x[3 * n + 2];
    zs3 += dN[n][2] * x[3 * n + 2];
  }
  const double det = xs1 * (ys2 * zs3 - zs2 * ys3) + ys1 * (zs2 * xs3 - xs2 * zs3) +
                     zs1 * (xs2 * ys3 - ys2 * xs3);
  double t = det;
  if (t <= 1.0e6 * 2.2250738585072014e-308) {
    t = 1.0;
    if (err) *err = 1;
  }
  const double d = 1.0 / t;
  const double s1x = d * (ys2 * zs3 - zs2 * ys3), s2x = d * (zs1 * ys3 - ys1 * zs3),
               s3x = d * (ys1 * zs2 - zs1 * ys2);
  const double s1y = d * (zs2 * xs3 - xs2 * zs3), s2y = d * (xs1 * zs3 - zs1 * xs3),
               s3y = d * (zs1 * xs2 - xs1 * zs2);
  const double s1z = d * (xs2 * ys3 - ys2 * xs3), s2z = d * (ys1 * xs3 - xs1 * ys3),
               s3z = d * (xs1 * ys2 - ys1 * xs2);
  for (int n = 0; n < 8; ++n) {
    g[3 * n + 0] = dN[n][0] * s1x + dN[n][1] * s2x + dN[n][2] * s3x;
    g[3 * n + 1] = dN[n][0] * s1y + dN[n][1] * s2y + dN[n][2] * s3y;
    g[3 * n + 2] = dN[n][0] * s1z + dN[n][1] * s2z + dN[n][2] * s3z;
  }
  return det;
}

// gradop[ip][node][3] at all 12 SCS ips (grad_op / shifted_grad_op).
inline int grad_op(const double* x, double* gradop, bool shifted) {
  int err = 0;
  for (int ip = 0; ip < NSCS; ++ip)
    grad_op_at(shifted ? IP_SHIFT[ip] : IP_STD[ip], x, &gradop[24 * ip], &err);
  return err;
}

// shape[ip][node] at the 12 SCS ips (shape_fcn / shifted_shape_fcn).
inline void scs_shape(double* N /*[12][8]*/, bool shifted) {
  for (int ip = 0; ip < NSCS; ++ip) shape(shifted ? IP_SHIFT[ip] : IP_STD[ip], &N[8 * ip]);
}

// Face gradient operator at the 4 exposed ips of face f (face_grad_op /
// shifted_face_grad_op, Hex8CVFEM.C:695-780): the shifted form evaluates at
// the face nodes themselves.
inline int face_grad_op(int f, const double* x, double* gradop /*[4][8][3]*/, bool shifted) {
  int err = 0;
  for (int k = 0; k < 4; ++k) {
    const double* s = shifted ? NODE_LOC[FACE_NODES[f][k]] : FACE_IP_STD[f][k];
    grad_op_at(s, x, &gradop[24 * k], &err);
  }
  return err;
}

// Quad4 face: area vectors of the 4 sub-faces (quad3d_scs_det); xf[4][3] in
// face-node order.
inline void quad_face_areav(const double* xf, double* areav /*[4][3]*/) {
  double e[4][3], c[3];
  for (int k = 0; k < 3; ++k) {
    e[0][k] = (xf[0 * 3 + k] + xf[1 * 3 + k]) * 0.5;
    e[1][k] = (xf[1 * 3 + k] + xf[2 * 3 + k]) * 0.5;
    e[2][k] = (xf[2 * 3 + k] + xf[3 * 3 + k]) * 0.5;
    e[3][k] = (xf[3 * 3 + k] + xf[0 * 3 + k]) * 0.5;
    c[k] = (xf[0 * 3 + k] + xf[1 * 3 + k] + xf[2 * 3 + k] + xf[3 * 3 + k]) * 0.25;
  }
  for (int i = 0; i < 4; ++i) {
    const int prv = (i + 3) % 4;
    const double d13x = c[0] - xf[3 * i + 0], d13y = c[1] - xf[3 * i + 1], d13z = c[2] - xf[3 * i + 2];
    const double d24x = e[prv][0] - e[i][0], d24y = e[prv][1] - e[i][1], d24z = e[prv][2] - e[i][2];
    areav[3 * i + 0] = 0.5 * (d24z * d13y - d13z * d24y);
    areav[3 * i + 1] = 0.5 * (d24x * d13z - d13x * d24z);
    areav[3 * i + 2] = 0.5 * (d24y * d13x - d13y * d24x);
  }
}

// Bilinear face shape functions on [-1/2,1/2]^2 (quad3d_shape_fcn); the
// standard face ips sit at (+-1/4,+-1/4) in face order, the shifted ones at the
// face nodes (identity).
constexpr double QUAD_IP_STD[4][2] = {{-0.25, -0.25}, {0.25, -0.25}, {0.25, 0.25}, {-0.25, 0.25}};
inline void face_shape(double* N /*[4][4]*/, bool shifted) {
  for (int ip = 0; ip < 4; ++ip) {
    if (shifted) {
      for (int n = 0; n < 4; ++n) N[4 * ip + n] = (n == ip) ? 1.0 : 0.0;
      continue;
    }
    const double s1 = QUAD_IP_STD[ip][0], s2 = QUAD_IP_STD[ip][1];
    N[4 * ip + 0] = 0.25 + 0.5 * (-s1 - s2) + s1 * s2;
    N[4 * ip + 1] = 0.25 + 0.5 * (s1 - s2) - s1 * s2;
    N[4 * ip + 2] = 0.25 + 0.5 * (s1 + s2) + s1 * s2;
    N[4 * ip + 3] = 0.25 + 0.5 * (-s1 + s2) - s1 * s2;
  }
}

}  // namespace hex8
}  // namespace oracle
