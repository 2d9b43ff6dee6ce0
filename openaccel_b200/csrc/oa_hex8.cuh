// hex8 control-volume master element on the device, evaluated in a
// per-lane canonical frame.
//
// Geometry follows the Nalu hex8 master element used by the reference
// (external/nalu/src/master_element/Hex8CVFEM.C:255-446 tables,
// MasterElementWork.F:1-457 SCS/SCV, :2344-2484 shape functions and
// derivatives, :2623-2774 gradient operator, CalculateQuadArea.F).
//
// Row-owner assembly: the lane that owns CSR row n for incident element e sees
// n at element corner c. It relabels the element's nodes through a proper cube
// rotation that takes corner c to corner 0 (ROT_PERM), so every lane runs the
// same straight-line code for corner 0: the three SCS ips 0 (0->1), 3 (0->3)
// and 8 (0->4), and the three faces 0, 3, 4 that touch corner 0. Because the
// ip index and ip location are compile-time constants, zero shape-function
// derivatives fold away at compile time.
#pragma once
#include <cstdint>

#include "oa_geom.cuh"

namespace oa {
namespace hex8 {

// ROT_PERM[c][k]: original element node that plays canonical node k for a
// lane sitting at corner c (a proper rotation, so orientation is preserved).
__constant__ int8_t ROT_PERM[8][8] = {
    {0, 1, 2, 3, 4, 5, 6, 7}, {1, 0, 4, 5, 2, 3, 7, 6}, {2, 3, 0, 1, 6, 7, 4, 5},
    {3, 2, 6, 7, 0, 1, 5, 4}, {4, 5, 1, 0, 7, 6, 2, 3}, {5, 4, 7, 6, 1, 0, 3, 2},
    {6, 7, 3, 2, 5, 4, 0, 1}, {7, 6, 5, 4, 3, 2, 1, 0}};
// ROT_IP[c][q]: original SCS ip of canonical ip {0,3,8}[q] and its sign
// (+1 when the original ip also runs away from corner c), packed ip*2+(sign<0).
__constant__ int8_t ROT_IP[8][3] = {{0, 6, 16},  {1, 18, 2},  {4, 3, 20},  {5, 22, 7},
                                    {8, 17, 14}, {9, 10, 19}, {12, 21, 11}, {13, 15, 23}};
// ROT_FACE[c][q]: original face ordinal of canonical face {0,3,4}[q].
__constant__ int8_t ROT_FACE[8][3] = {{0, 3, 4}, {4, 1, 0}, {2, 1, 4}, {4, 3, 2},
                                      {5, 3, 0}, {0, 1, 5}, {5, 1, 2}, {2, 3, 5}};

// L/R pairs of the 12 SCS ips (Hex8CVFEM.C:264-276).
__host__ __device__ constexpr int lr(int ip, int side) {
  constexpr int t[12][2] = {{0, 1}, {1, 2}, {2, 3}, {0, 3}, {4, 5}, {5, 6},
                            {6, 7}, {4, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  return t[ip][side];
}

// SCS ip parametric location, standard (+-1/4) or shifted (edge midpoint).
__host__ __device__ constexpr double ip_loc(int ip, int d, bool shifted) {
  constexpr double t[12][3] = {
      {0.00, -0.25, -0.25}, {0.25, 0.00, -0.25}, {0.00, 0.25, -0.25}, {-0.25, 0.00, -0.25},
      {0.00, -0.25, 0.25},  {0.25, 0.00, 0.25},  {0.00, 0.25, 0.25},  {-0.25, 0.00, 0.25},
      {-0.25, -0.25, 0.00}, {0.25, -0.25, 0.00}, {0.25, 0.25, 0.00},  {-0.25, 0.25, 0.00}};
  return shifted ? 2.0 * t[ip][d] : t[ip][d];
}

__host__ __device__ constexpr double node_loc(int n, int d) {
  constexpr double t[8][3] = {{-0.5, -0.5, -0.5}, {0.5, -0.5, -0.5}, {0.5, 0.5, -0.5},
                              {-0.5, 0.5, -0.5},  {-0.5, -0.5, 0.5}, {0.5, -0.5, 0.5},
                              {0.5, 0.5, 0.5},    {-0.5, 0.5, 0.5}};
  return t[n][d];
}

// Standard exposed-face ip of face f nearest face node k (Hex8CVFEM.C:348-378).
__host__ __device__ constexpr double face_ip_loc(int f, int k, int d) {
  constexpr double t[6][4][3] = {
      {{-0.25, -0.50, -0.25}, {0.25, -0.50, -0.25}, {0.25, -0.50, 0.25}, {-0.25, -0.50, 0.25}},
      {{0.50, -0.25, -0.25}, {0.50, 0.25, -0.25}, {0.50, 0.25, 0.25}, {0.50, -0.25, 0.25}},
      {{0.25, 0.50, -0.25}, {-0.25, 0.50, -0.25}, {-0.25, 0.50, 0.25}, {0.25, 0.50, 0.25}},
      {{-0.50, -0.25, -0.25}, {-0.50, -0.25, 0.25}, {-0.50, 0.25, 0.25}, {-0.50, 0.25, -0.25}},
      {{-0.25, -0.25, -0.50}, {-0.25, 0.25, -0.50}, {0.25, 0.25, -0.50}, {0.25, -0.25, -0.50}},
      {{-0.25, -0.25, 0.50}, {0.25, -0.25, 0.50}, {0.25, 0.25, 0.50}, {-0.25, 0.25, 0.50}}};
  return t[f][k][d];
}

__host__ __device__ constexpr int face_node(int f, int k) {
  constexpr int t[6][4] = {{0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6},
                           {0, 4, 7, 3}, {0, 3, 2, 1}, {4, 5, 6, 7}};
  return t[f][k];
}

// Trilinear shape function N_n at (s1,s2,s3) (hex_shape_fcn).
__host__ __device__ constexpr double shape(int n, double s1, double s2, double s3) {
  const double h = 0.5, q = 0.25, e = 0.125;
  switch (n) {
    case 0: return e + q * (-s1 - s2 - s3) + h * (s2 * s3 + s3 * s1 + s1 * s2) - s1 * s2 * s3;
    case 1: return e + q * (s1 - s2 - s3) + h * (s2 * s3 - s3 * s1 - s1 * s2) + s1 * s2 * s3;
    case 2: return e + q * (s1 + s2 - s3) + h * (-s2 * s3 - s3 * s1 + s1 * s2) - s1 * s2 * s3;
    case 3: return e + q * (-s1 + s2 - s3) + h * (-s2 * s3 + s3 * s1 - s1 * s2) + s1 * s2 * s3;
    case 4: return e + q * (-s1 - s2 + s3) + h * (-s2 * s3 - s3 * s1 + s1 * s2) + s1 * s2 * s3;
    case 5: return e + q * (s1 - s2 + s3) + h * (-s2 * s3 + s3 * s1 - s1 * s2) - s1 * s2 * s3;
    case 6: return e + q * (s1 + s2 + s3) + h * (s2 * s3 + s3 * s1 + s1 * s2) + s1 * s2 * s3;
    default: return e + q * (-s1 + s2 + s3) + h * (s2 * s3 - s3 * s1 - s1 * s2) - s1 * s2 * s3;
  }
}

// Parametric derivative dN_n/ds_d at (s1,s2,s3) (hex_derivative).
__host__ __device__ constexpr double dshape(int n, int d, double s1, double s2, double s3) {
  const double h = 0.5, q = 0.25;
  const double s12 = s1 * s2, s23 = s2 * s3, s13 = s1 * s3;
  if (d == 0) {
    switch (n) {
      case 0: return h * (s3 + s2) - s23 - q;
      case 1: return h * (-s3 - s2) + s23 + q;
      case 2: return h * (-s3 + s2) - s23 + q;
      case 3: return h * (s3 - s2) + s23 - q;
      case 4: return h * (-s3 + s2) + s23 - q;
      case 5: return h * (s3 - s2) - s23 + q;
      case 6: return h * (s3 + s2) + s23 + q;
      default: return h * (-s3 - s2) - s23 - q;
    }
  } else if (d == 1) {
    switch (n) {
      case 0: return h * (s3 + s1) - s13 - q;
      case 1: return h * (s3 - s1) + s13 - q;
      case 2: return h * (-s3 + s1) - s13 + q;
      case 3: return h * (-s3 - s1) + s13 + q;
      case 4: return h * (-s3 + s1) + s13 - q;
      case 5: return h * (-s3 - s1) - s13 - q;
      case 6: return h * (s3 + s1) + s13 + q;
      default: return h * (s3 - s1) - s13 + q;
    }
  }
  switch (n) {
    case 0: return h * (s2 + s1) - s12 - q;
    case 1: return h * (s2 - s1) + s12 - q;
    case 2: return h * (-s2 - s1) - s12 - q;
    case 3: return h * (-s2 + s1) + s12 - q;
    case 4: return h * (-s2 - s1) + s12 + q;
    case 5: return h * (-s2 + s1) - s12 + q;
    case 6: return h * (s2 + s1) + s12 + q;
    default: return h * (s2 - s1) - s12 + q;
  }
}

// Inverse-Jacobian rows at a parametric point: ds_k/dx_i stored as
// inv[k][i]; returns det(J). Same algebra and singular-Jacobian guard as
// hex_gradient_operator (det <= 1e6*realmin -> treated as 1, flag raised).
// Inverse Jacobian at a point, in the arithmetic type R (FP64 everywhere but
// the mixed form's momentum fluxes, which use FP32 on element-local
// coordinates).
template <class R>
struct InvJacR {
  R s[3][3];  // s[k][i] = d s_k / d x_i
  R det;
};
using InvJac = InvJacR<double>;

template <class PT, class R = double>
__device__ __forceinline__ InvJacR<R> inv_jacobian(const R (&x)[8][3], int* err) {
  R J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // J[i][d] = dx_i/ds_d
#pragma unroll
  for (int n = 0; n < 8; ++n) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double v = dshape(n, d, PT::s(0), PT::s(1), PT::s(2));
      if (v != 0.0) {
#pragma unroll
        for (int i = 0; i < 3; ++i) J[i][d] += R(v) * x[n][i];
      }
    }
  }
  const R xs1 = J[0][0], xs2 = J[0][1], xs3 = J[0][2];
  const R ys1 = J[1][0], ys2 = J[1][1], ys3 = J[1][2];
  const R zs1 = J[2][0], zs2 = J[2][1], zs3 = J[2][2];
  InvJacR<R> r;
  r.det = xs1 * (ys2 * zs3 - zs2 * ys3) + ys1 * (zs2 * xs3 - xs2 * zs3) + zs1 * (xs2 * ys3 - ys2 * xs3);
  R t = r.det;
  // determinant guard of hex_gradient_operator: 1e6 times the smallest normal
  // number of the arithmetic type
  if (t <= R(1.0e6) * (sizeof(R) == 4 ? R(1.1754943508222875e-38) : R(2.2250738585072014e-308))) {
    t = R(1);
    *err = 1;
  }
  const R d = R(1) / t;
  r.s[0][0] = d * (ys2 * zs3 - zs2 * ys3);
  r.s[1][0] = d * (zs1 * ys3 - ys1 * zs3);
  r.s[2][0] = d * (ys1 * zs2 - zs1 * ys2);
  r.s[0][1] = d * (zs2 * xs3 - xs2 * zs3);
  r.s[1][1] = d * (xs1 * zs3 - zs1 * xs3);
  r.s[2][1] = d * (zs1 * xs2 - xs1 * zs2);
  r.s[0][2] = d * (xs2 * ys3 - ys2 * xs3);
  r.s[1][2] = d * (ys1 * xs3 - xs1 * ys3);
  r.s[2][2] = d * (xs1 * ys2 - ys1 * xs2);
  return r;
}

// Physical gradient of N_n at the point PT: g_i = sum_k dN_n/ds_k * ds_k/dx_i.
template <class PT, int N, class R = double>
__device__ __forceinline__ void grad_n(const InvJacR<R>& J, R g[3]) {
  constexpr double d0 = dshape(N, 0, PT::s(0), PT::s(1), PT::s(2));
  constexpr double d1 = dshape(N, 1, PT::s(0), PT::s(1), PT::s(2));
  constexpr double d2 = dshape(N, 2, PT::s(0), PT::s(1), PT::s(2));
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    R v = R(0);
    if (d0 != 0.0) v += R(d0) * J.s[0][i];
    if (d1 != 0.0) v += R(d1) * J.s[1][i];
    if (d2 != 0.0) v += R(d2) * J.s[2][i];
    g[i] = v;
  }
}

template <class PT, int N>
__host__ __device__ constexpr bool grad_is_zero() {
  return dshape(N, 0, PT::s(0), PT::s(1), PT::s(2)) == 0.0 &&
         dshape(N, 1, PT::s(0), PT::s(1), PT::s(2)) == 0.0 &&
         dshape(N, 2, PT::s(0), PT::s(1), PT::s(2)) == 0.0;
}

// Compile-time parametric points.
template <int IP, bool SHIFT>
struct ScsPt {
  __host__ __device__ static constexpr double s(int d) { return ip_loc(IP, d, SHIFT); }
};
template <int F, int K, bool SHIFT>
struct FacePt {  // exposed ip of face F at face node K (shifted: the node itself)
  __host__ __device__ static constexpr double s(int d) {
    return SHIFT ? node_loc(face_node(F, K), d) : face_ip_loc(F, K, d);
  }
};

template <class PT, int N>
__host__ __device__ constexpr double shape_at() {
  return shape(N, PT::s(0), PT::s(1), PT::s(2));
}


// Subdivision points a canonical corner-0 lane needs: edge midpoints to nodes
// 1, 3, 4; centroids of faces (0,1,2,3), (0,1,4,5), (0,3,4,7); element centroid.
struct Corner0Points {
  double m01[3], m03[3], m04[3], fB[3], fF[3], fL[3], cen[3];
};

__device__ __forceinline__ void corner0_points(const double (&x)[8][3], Corner0Points& p) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    p.m01[k] = 0.5 * (x[0][k] + x[1][k]);
    p.m03[k] = 0.5 * (x[3][k] + x[0][k]);
    p.m04[k] = 0.5 * (x[0][k] + x[4][k]);
    p.fB[k] = 0.25 * (x[0][k] + x[1][k] + x[2][k] + x[3][k]);
    p.fF[k] = 0.25 * (x[0][k] + x[1][k] + x[4][k] + x[5][k]);
    p.fL[k] = 0.25 * (x[0][k] + x[3][k] + x[4][k] + x[7][k]);
    double s = 0.0;
#pragma unroll
    for (int n = 0; n < 8; ++n) s += x[n][k];
    p.cen[k] = 0.125 * s;
  }
}

// SCS area vectors of canonical ips 0, 3, 8 (hex_scs_det facet table rows
// 1, 4, 9), each pointing away from corner 0.
__device__ __forceinline__ void corner0_areas(const Corner0Points& p, double A0[3], double A3[3],
                                              double A8[3]) {
  quad_area(p.fF, p.m01, p.fB, p.cen, A0);
  quad_area(p.m03, p.fL, p.cen, p.fB, A3);
  quad_area(p.m04, p.fF, p.cen, p.fL, A8);
}

// Exposed-face sub-area at face node 0 of a quad whose nodes are listed
// cyclically starting at corner 0 (quad3d_scs_det, first sub-face).
template <class R>
__device__ __forceinline__ void face_area_at_first(const R* p0, const R* p1, const R* p2, const R* p3, R A[3]) {
  R e0[3], e3[3], c[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    e0[k] = (p0[k] + p1[k]) * R(0.5);
    e3[k] = (p3[k] + p0[k]) * R(0.5);
    c[k] = (p0[k] + p1[k] + p2[k] + p3[k]) * R(0.25);
  }
  const R d13x = c[0] - p0[0], d13y = c[1] - p0[1], d13z = c[2] - p0[2];
  const R d24x = e3[0] - e0[0], d24y = e3[1] - e0[1], d24z = e3[2] - e0[2];
  A[0] = R(0.5) * (d24z * d13y - d13z * d24y);
  A[1] = R(0.5) * (d24x * d13z - d13x * d24z);
  A[2] = R(0.5) * (d24y * d13x - d13y * d24x);
}

}  // namespace hex8
}  // namespace oa
