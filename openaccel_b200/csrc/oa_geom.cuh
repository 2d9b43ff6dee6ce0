// Shared FP64 control-volume geometry helpers (device).
#pragma once
#include <cuda_runtime.h>

namespace oa {

// Grandy hex volume by 24 triangular facets (CalculateHexVolume.F).
__device__ __forceinline__ double hex_volume(const double (&v)[8][3]) {
  constexpr int T[24][3] = {{0, 8, 1},  {8, 2, 1},  {3, 2, 8},  {3, 8, 0},  {6, 9, 5},  {7, 9, 6},
                            {4, 9, 7},  {4, 5, 9},  {10, 0, 1}, {5, 10, 1}, {4, 10, 5}, {4, 0, 10},
                            {7, 6, 11}, {6, 2, 11}, {2, 3, 11}, {3, 7, 11}, {6, 12, 2}, {5, 12, 6},
                            {5, 1, 12}, {1, 2, 12}, {0, 4, 13}, {4, 7, 13}, {7, 3, 13}, {3, 0, 13}};
  constexpr int Q[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4},
                           {3, 2, 6, 7}, {1, 2, 6, 5}, {0, 3, 7, 4}};
  double c[14][3];
#pragma unroll
  for (int n = 0; n < 8; ++n)
#pragma unroll
    for (int k = 0; k < 3; ++k) c[n][k] = v[n][k];
#pragma unroll
  for (int f = 0; f < 6; ++f)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      c[8 + f][k] = 0.25 * (v[Q[f][0]][k] + v[Q[f][1]][k] + v[Q[f][2]][k] + v[Q[f][3]][k]);
  double vol = 0.0;
#pragma unroll
  for (int t = 0; t < 24; ++t) {
    const double* P = c[T[t][0]];
    const double* R1 = c[T[t][1]];
    const double* R2 = c[T[t][2]];
    const double f0 = P[0] + R1[0] + R2[0], f1 = P[1] + R1[1] + R2[1], f2 = P[2] + R1[2] + R2[2];
    vol += f0 * ((R1[1] - P[1]) * (R2[2] - P[2]) - (R2[1] - P[1]) * (R1[2] - P[2])) -
           f1 * ((R1[0] - P[0]) * (R2[2] - P[2]) - (R2[0] - P[0]) * (R1[2] - P[2])) +
           f2 * ((R1[0] - P[0]) * (R2[1] - P[1]) - (R2[0] - P[0]) * (R1[1] - P[1]));
  }
  return vol / 18.0;
}


// Area vector of quad (a,b,c,d) by four triangles about the vertex mean
// (CalculateQuadArea.F).
__device__ __forceinline__ void quad_area(const double* a, const double* b, const double* c,
                                          const double* d, double A[3]) {
  double m[3], r1[3], r2[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) m[k] = 0.25 * (a[k] + b[k] + c[k] + d[k]);
  A[0] = A[1] = A[2] = 0.0;
  const double* q[5] = {a, b, c, d, a};
#pragma unroll
  for (int k = 0; k < 3; ++k) r2[k] = a[k] - m[k];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      r1[k] = r2[k];
      r2[k] = q[t + 1][k] - m[k];
    }
    A[0] += r1[1] * r2[2] - r2[1] * r1[2];
    A[1] += r1[2] * r2[0] - r2[2] * r1[0];
    A[2] += r1[0] * r2[1] - r2[0] * r1[1];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) A[k] *= 0.5;
}

}  // namespace oa
