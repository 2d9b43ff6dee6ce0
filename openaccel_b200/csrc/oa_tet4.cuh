// tet4 control-volume master element (device).
//
// Tables restate external/nalu/src/master_element/Tet4CVFEM.C (lrscv_ :329-335,
// intgLoc_ / intgLocShift_ :365-382, sideNodeOrdinals_ :416-421) and the
// subdivision of MasterElementWork.F tet_scs_det (:608-752) / tet_scv_det
// (:459-606). A corner of an element is seen through the even permutation of
// the element's nodes that brings it to local node 0 (orientation is
// preserved), so the three sub-control surfaces around it are always ips 0
// (0->1), 2 (0->2) and 3 (0->3), each with its area vector pointing away from
// the corner; scs_areas6 evaluates all six surfaces of an element once in
// those frames.
#pragma once
#include <cstdint>

#include "oa_geom.cuh"

namespace oa {
namespace tet4 {

// Even permutations taking corner a to local node 0, packed 2 bits per node.
__host__ __device__ __forceinline__ int perm_at(int a, int k) {
  // a=0: 0123, a=1: 1032, a=2: 2301, a=3: 3210
  return (a ^ k) & 3;
}

// Boundary face ordinal -> element nodes in side order, and the node opposite.
__host__ __device__ __forceinline__ int side_node(int f, int k) {
  // {0,1,3}, {1,2,3}, {0,3,2}, {0,2,1}
  constexpr uint32_t W = (0u | 1u << 2 | 3u << 4) | (1u | 2u << 2 | 3u << 4) << 6 |
                         (0u | 3u << 2 | 2u << 4) << 12 | (0u | 2u << 2 | 1u << 4) << 18;
  return (W >> (6 * f + 2 * k)) & 3u;
}
__host__ __device__ __forceinline__ int opposite_node(int f) { return (0x3102u >> (4 * f)) & 0xFu; }

// Area vectors of all six sub-control surfaces of the element, one per edge,
// in the order (0,1), (0,2), (0,3), (1,3), (1,2), (2,3), each pointing away
// from the edge's first node. In the frame of a corner (nodes p0 p1 p2 p3,
// p0 the corner) the surfaces around it are the quads (m01, f012, c, f013),
// (m02, f023, c, f012) and (m03, f013, c, f023) of the 15-point subdivision
// (edge midpoints m, face centroids f, element centroid c); each edge is
// evaluated in the frame of its first node (corner 0: nodes 0123, corner 1:
// 1032, corner 2: 2301), and the surface seen from the other node is the same
// quad in reverse order, i.e. the negated vector.
__device__ __forceinline__ void scs_areas6(const double (&x)[4][3], double (&A)[6][3]) {
  double m01[3], m02[3], m03[3], m12[3], m13[3], m23[3], f012[3], f013[3], f023[3], f123[3], c[3];
  const double half = 0.5, third = 1.0 / 3.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double x0 = x[0][k], x1 = x[1][k], x2 = x[2][k], x3 = x[3][k];
    m01[k] = half * (x0 + x1);
    m02[k] = half * (x2 + x0);
    m03[k] = half * (x0 + x3);
    m12[k] = half * (x1 + x2);
    m13[k] = half * (x1 + x3);
    m23[k] = half * (x2 + x3);
    f012[k] = third * (x0 + x1 + x2);
    f023[k] = third * (x0 + x2 + x3);
    f013[k] = third * (x0 + x1 + x3);
    f123[k] = third * (x1 + x2 + x3);
    double s = 0.0;
    s = s + 0.25 * x0;
    s = s + 0.25 * x1;
    s = s + 0.25 * x2;
    s = s + 0.25 * x3;
    c[k] = s;
  }
  quad_area(m01, f012, c, f013, A[0]);
  quad_area(m02, f023, c, f012, A[1]);
  quad_area(m03, f013, c, f023, A[2]);
  quad_area(m13, f123, c, f013, A[3]);
  quad_area(m12, f012, c, f123, A[4]);
  quad_area(m23, f023, c, f123, A[5]);
}

// Edge of scs_areas6 joining corner a to node perm_at(a, k) (k = 1..3), with
// the sign that makes its area point away from a.
__host__ __device__ constexpr int corner_edge(int a, int k) {
  constexpr int E[4][3] = {{0, 1, 2}, {0, 3, 4}, {5, 1, 4}, {5, 3, 2}};
  return E[a][k - 1];
}
__host__ __device__ constexpr double corner_edge_sign(int a, int k) {
  constexpr int S[4][3] = {{1, 1, 1}, {-1, 1, 1}, {1, -1, -1}, {-1, -1, -1}};
  return S[a][k - 1];
}

// Constant dN/dx of the four nodes (tet_gradient_operator). Returns false when
// the Jacobian determinant is <= 1e6 * DBL_MIN (the determinant is then 1).
__device__ __forceinline__ bool grad_op(const double (&x)[4][3], double (&g)[4][3]) {
  const double dx1 = x[1][0] - x[0][0], dx2 = x[2][0] - x[0][0], dx3 = x[3][0] - x[0][0];
  const double dy1 = x[1][1] - x[0][1], dy2 = x[2][1] - x[0][1], dy3 = x[3][1] - x[0][1];
  const double dz1 = x[1][2] - x[0][2], dz2 = x[2][2] - x[0][2], dz3 = x[3][2] - x[0][2];
  double det = dx1 * (dy2 * dz3 - dz2 * dy3) + dy1 * (dz2 * dx3 - dx2 * dz3) + dz1 * (dx2 * dy3 - dy2 * dx3);
  bool ok = true;
  if (det <= 1.0e6 * 2.2250738585072014e-308) {
    det = 1.0;
    ok = false;
  }
  const double d = 1.0 / det;
  g[1][0] = d * (dy2 * dz3 - dz2 * dy3);
  g[2][0] = d * (dz1 * dy3 - dy1 * dz3);
  g[3][0] = d * (dy1 * dz2 - dz1 * dy2);
  g[1][1] = d * (dz2 * dx3 - dx2 * dz3);
  g[2][1] = d * (dx1 * dz3 - dz1 * dx3);
  g[3][1] = d * (dz1 * dx2 - dx1 * dz2);
  g[1][2] = d * (dx2 * dy3 - dy2 * dx3);
  g[2][2] = d * (dy1 * dx3 - dx1 * dy3);
  g[3][2] = d * (dx1 * dy2 - dy1 * dx2);
#pragma unroll
  for (int j = 0; j < 3; ++j) g[0][j] = -g[1][j] - g[2][j] - g[3][j];
  return ok;
}

// Sub-control volumes of all four corners (tet_scv_det).
__device__ __forceinline__ void scv_volumes(const double (&x)[4][3], double (&vol)[4]) {
  constexpr int H[4][8] = {{0, 4, 7, 6, 11, 13, 14, 12},
                           {1, 5, 7, 4, 9, 10, 14, 13},
                           {2, 6, 7, 5, 8, 12, 14, 10},
                           {3, 9, 13, 11, 8, 10, 14, 12}};
  double p[15][3];
  const double half = 0.5, third = 1.0 / 3.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double x0 = x[0][k], x1 = x[1][k], x2 = x[2][k], x3 = x[3][k];
    p[0][k] = x0;
    p[1][k] = x1;
    p[2][k] = x2;
    p[3][k] = x3;
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
    double s = 0.0;
    s = s + 0.25 * x0;
    s = s + 0.25 * x1;
    s = s + 0.25 * x2;
    s = s + 0.25 * x3;
    p[14][k] = s;
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    double v[8][3];
#pragma unroll
    for (int n = 0; n < 8; ++n)
#pragma unroll
      for (int k = 0; k < 3; ++k) v[n][k] = p[H[c][n]][k];
    vol[c] = hex_volume(v);
  }
}

// Exposed-face area vectors of the three boundary ips of a tri3 face with
// nodes p[3][3] in side order (tri3d_scs_det, MasterElementWork.F:1589-1698):
// ip k owns the quad (vertex k, edge midpoints, centroid).
__device__ __forceinline__ void tri_face_areas(const double (&p)[3][3], double (&A)[3][3]) {
  const double half = 0.5, third = 1.0 / 3.0;
  double c[3], e[3][3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    e[0][d] = (p[0][d] + p[1][d]) * half;
    e[1][d] = (p[1][d] + p[2][d]) * half;
    e[2][d] = (p[2][d] + p[0][d]) * half;
    c[d] = (p[0][d] + p[1][d] + p[2][d]) * third;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int km = k == 0 ? 2 : k - 1;
    double d13[3], d24[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      d13[d] = c[d] - p[k][d];
      d24[d] = e[km][d] - e[k][d];
    }
    A[k][0] = half * (d24[2] * d13[1] - d13[2] * d24[1]);
    A[k][1] = half * (d24[0] * d13[2] - d13[0] * d24[2]);
    A[k][2] = half * (d24[1] * d13[0] - d13[1] * d24[0]);
  }
}

}  // namespace tet4
}  // namespace oa
