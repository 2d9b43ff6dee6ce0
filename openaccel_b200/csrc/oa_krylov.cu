// Pressure-correction / momentum Krylov solve on the device: BiCGStab
// (van der Vorst 1992) right-preconditioned by point or 3x3 block Jacobi, or
// for scalar systems by the aggregation-AMG V-cycle of oa_amg.cu; for scalar
// AMG-preconditioned systems also GCR(2), one V-cycle per iteration.
//
// The reference hands its systems to liblinsolve (PETSc / Trilinos / HYPRE,
// src/equation/linearSystem.h:416-462), which is absent from the reference
// checkout; the algorithm here is the published one. All scalars live on the
// device and every reduction is a fixed two-stage tree (block partials, then
// an ordered single-block sum), so results are bitwise reproducible run to
// run. A device "done" flag lets chunks of iterations be launched without
// host round trips; kernels after convergence return immediately.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

#include <cmath>
#include <type_traits>

#include "oa_internal.h"
#include "oa_krylov.h"

namespace oa {

constexpr int KB = 256;        // threads per block for vector kernels
constexpr int MAX_PARTIALS = 2048;

template <class T>
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// block-level fixed-order reduction of up to 3 values; thread 0 writes partials
template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double* partials, int nblocks_stride) {
  __shared__ double sh[NV][KB / 32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double s = warp_sum<double>(v[k]);
    if (l == 0) sh[k][w] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = 0.0;
      for (int i = 0; i < KB / 32; ++i) s += sh[k][i];
      partials[k * nblocks_stride + blockIdx.x] = s;
    }
  }
}

// ordered final sum of the partials by one block
template <int NV>
__device__ __forceinline__ void final_reduce(const double* partials, int nb, double (&out)[NV]) {
  __shared__ double sh[NV][KB];
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double s = 0.0;
    for (int i = threadIdx.x; i < nb; i += KB) s += partials[k * MAX_PARTIALS + i];
    sh[k][threadIdx.x] = s;
  }
  __syncthreads();
  for (int st = KB / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
#pragma unroll
      for (int k = 0; k < NV; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + st];
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < NV; ++k) out[k] = sh[k][0];
}

// y = A x for a BSR matrix with BxB row-major blocks; optional partial dots
// (y.w1 and, for ND = 2, y.y).
template <int B, class TM, class TV, int ND>
__global__ void __launch_bounds__(KB) k_spmv(int nn, const int* __restrict__ rp, const int* __restrict__ cols,
                                              const TM* __restrict__ A, const TV* __restrict__ x,
                                              TV* __restrict__ y, const TV* __restrict__ w1,
                                              const TV* __restrict__ w2, double* partials, const KScal* sc) {
  if (sc && sc->done) return;
  double v[ND > 0 ? ND : 1];
#pragma unroll
  for (int k = 0; k < (ND > 0 ? ND : 1); ++k) v[k] = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nn * B; t += gridDim.x * blockDim.x) {
    const int i = t / B, m = t - i * B;
    double s = 0.0;
    const int a = __ldg(rp + i), bnd = __ldg(rp + i + 1);
    for (int k = a; k < bnd; ++k) {
      const int j = __ldg(cols + k);
#pragma unroll
      for (int q = 0; q < B; ++q) s += double(A[(size_t)k * B * B + B * m + q]) * double(x[B * j + q]);
    }
    const TV ys = TV(s);
    y[t] = ys;
    // second dot is y.y, taken from the register (never re-read through y)
    if (ND > 0) v[0] += double(ys) * double(w1[t]);
    if (ND > 1) v[1] += double(ys) * double(ys);
  }
  if (ND > 0) block_reduce_store<ND>(reinterpret_cast<double(&)[ND]>(v), partials, MAX_PARTIALS);
}

// z = Minv v (point or 3x3 block Jacobi); the inverse is stored in the
// precision of the Krylov vectors (FP32 in the mixed form's inner solves)
template <int B, class TV>
__global__ void k_prec(int nn, const TV* __restrict__ Minv, const TV* __restrict__ v, TV* __restrict__ z,
                       const KScal* sc) {
  if (sc->done) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nn * B) return;
  if (B == 1) {
    z[t] = TV(double(Minv[t]) * double(v[t]));
  } else {
    const int i = t / 3, m = t - 3 * i;
    const TV* M = Minv + 9 * (size_t)i + 3 * m;
    z[t] = TV(double(M[0]) * double(v[3 * i]) + double(M[1]) * double(v[3 * i + 1]) +
              double(M[2]) * double(v[3 * i + 2]));
  }
}

template <int B, class TM, class TP>
__global__ void k_build_minv(int nn, const int* __restrict__ rp, const int* __restrict__ dg, const TM* __restrict__ A,
                             TP* Minv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const TM* d = A + (size_t)(rp[i] + dg[i]) * B * B;
  if (B == 1) {
    Minv[i] = TP(1.0 / double(d[0]));
  } else {
    double a[9];
    for (int k = 0; k < 9; ++k) a[k] = double(d[k]);
    const double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                       a[2] * (a[3] * a[7] - a[4] * a[6]);
    const double id = 1.0 / det;
    TP* r = Minv + 9 * (size_t)i;
    r[0] = TP((a[4] * a[8] - a[5] * a[7]) * id);
    r[1] = TP((a[2] * a[7] - a[1] * a[8]) * id);
    r[2] = TP((a[1] * a[5] - a[2] * a[4]) * id);
    r[3] = TP((a[5] * a[6] - a[3] * a[8]) * id);
    r[4] = TP((a[0] * a[8] - a[2] * a[6]) * id);
    r[5] = TP((a[2] * a[3] - a[0] * a[5]) * id);
    r[6] = TP((a[3] * a[7] - a[4] * a[6]) * id);
    r[7] = TP((a[1] * a[6] - a[0] * a[7]) * id);
    r[8] = TP((a[0] * a[4] - a[1] * a[3]) * id);
  }
}

// init: x = 0, r = rh = b, p = v = 0; partial ||b||^2
template <class TV, class TB>
__global__ void __launch_bounds__(KB) k_init(int n, const TB* __restrict__ b, TV* x, TV* r, TV* rh, TV* p, TV* v,
                                              double* partials) {
  double s[1] = {0.0};
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const TV bv = TV(b[t]);
    x[t] = TV(0);
    r[t] = bv;
    rh[t] = bv;
    p[t] = TV(0);
    v[t] = TV(0);
    s[0] += double(bv) * double(bv);
  }
  block_reduce_store<1>(s, partials, MAX_PARTIALS);
}

// rtol_dev / maxit_dev (when not null) replace rtol / maxit: the inner solves
// of a graph-captured iterative refinement take them from the refinement state
__global__ void __launch_bounds__(KB) k_init_scalars(KScal* sc, const double* partials, int nb, double rtol,
                                                      int maxit, const double* rtol_dev, const int* maxit_dev) {
  double o[1];
  final_reduce<1>(partials, nb, o);
  if (threadIdx.x == 0) {
    sc->rtol = rtol_dev ? *rtol_dev : rtol;
    sc->maxit = maxit_dev ? *maxit_dev : maxit;
    sc->bnorm = sqrt(o[0]);
    sc->rnorm = sc->bnorm;
    sc->rho = sc->alpha = sc->omega = 1.0;
    sc->d0 = o[0];  // rh.r for the first iteration equals ||b||^2
    sc->iters = 0;
    sc->status = 0;
    sc->done = (sc->bnorm == 0.0 || !(sc->bnorm < INFINITY)) ? 1 : 0;
    if (!(sc->bnorm < INFINITY)) sc->status = 2;
  }
}

// p = r + beta (p - omega v), beta = (rho1/rho)(alpha/omega), rho1 = sc->d0
template <class TV>
__global__ void k_p_update(int n, TV* p, const TV* r, const TV* v, const KScal* sc) {
  if (sc->done) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double beta = (sc->d0 / sc->rho) * (sc->alpha / sc->omega);
  p[t] = TV(double(r[t]) + beta * (double(p[t]) - sc->omega * double(v[t])));
}

// alpha = rho1 / (rh.v)
__global__ void __launch_bounds__(KB) k_alpha(KScal* sc, const double* partials, int nb) {
  if (sc->done) return;
  double o[1];
  final_reduce<1>(partials, nb, o);
  if (threadIdx.x == 0) {
    if (o[0] == 0.0 || !(fabs(o[0]) < INFINITY)) {
      sc->done = 1;
      sc->status = 1;
      return;
    }
    sc->alpha = sc->d0 / o[0];
  }
}

// s = r - alpha v (stored in r)
template <class TV>
__global__ void k_s_update(int n, TV* r, const TV* v, const KScal* sc) {
  if (sc->done) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  r[t] = TV(double(r[t]) - sc->alpha * double(v[t]));
}

// omega = (t.s)/(t.t)
__global__ void __launch_bounds__(KB) k_omega(KScal* sc, const double* partials, int nb) {
  if (sc->done) return;
  double o[2];
  final_reduce<2>(partials, nb, o);
  if (threadIdx.x == 0) sc->omega = o[1] > 0.0 ? o[0] / o[1] : 0.0;
}

// x += alpha ph + omega sh; r = s - omega t; partials r.r, rh.r
template <class TV>
__global__ void __launch_bounds__(KB) k_x_update(int n, TV* x, TV* r, const TV* ph, const TV* sh, const TV* t,
                                                  const TV* rh, double* partials, const KScal* sc) {
  if (sc->done) return;
  double v[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = TV(double(x[i]) + sc->alpha * double(ph[i]) + sc->omega * double(sh[i]));
    const TV rn = TV(double(r[i]) - sc->omega * double(t[i]));
    r[i] = rn;
    v[0] += double(rn) * double(rn);
    v[1] += double(rh[i]) * double(rn);
  }
  block_reduce_store<2>(v, partials, MAX_PARTIALS);
}

// Largest sqrt(r2[s] / b2[s]) over the segments (0 where b2 = 0), by the
// whole block; 0 when nseg <= 1.
__device__ __forceinline__ double block_seg_max(const double* r2, const double* b2, int nseg) {
  __shared__ double sm[KB];
  double m = 0.0;
  if (nseg > 1)
    for (int q = threadIdx.x; q < nseg; q += KB) {
      const double b = b2[q];
      if (b > 0.0) m = fmax(m, sqrt(r2[q] / b));
    }
  sm[threadIdx.x] = m;
  __syncthreads();
  for (int st = KB / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + st]);
    __syncthreads();
  }
  return sm[0];
}

// per-segment sums of squares, one block per segment, fixed-order tree
template <class T>
__global__ void __launch_bounds__(KB) k_seg_sumsq(const int* __restrict__ ptr, const int* __restrict__ rows,
                                                   const T* __restrict__ v, double* out, const int* done) {
  if (done && *done) return;
  __shared__ double sm[KB];
  const int sg = blockIdx.x;
  double a = 0.0;
  for (int q = ptr[sg] + threadIdx.x; q < ptr[sg + 1]; q += KB) {
    const double x = double(v[rows[q]]);
    a += x * x;
  }
  sm[threadIdx.x] = a;
  __syncthreads();
  for (int st = KB / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) sm[threadIdx.x] += sm[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[sg] = sm[0];
}

__global__ void __launch_bounds__(KB) k_seg_max_ratio(const double* r2, const double* b2, int nseg, double* out) {
  const double m = block_seg_max(r2, b2, nseg);
  if (threadIdx.x == 0) *out = m;
}

// rho <- rho1; rho1 <- rh.r; convergence test (per segment for batched systems)
__global__ void __launch_bounds__(KB) k_end_iter(KScal* sc, const double* partials, int nb, const double* seg_r2,
                                                  const double* seg_b2, int nseg) {
  if (sc->done) return;
  double o[2];
  final_reduce<2>(partials, nb, o);
  const double segmax = block_seg_max(seg_r2, seg_b2, nseg);
  if (threadIdx.x == 0) {
    sc->seg_rel = segmax;
    const bool conv = nseg > 1 ? segmax <= sc->rtol : false;
    sc->rho = sc->d0;
    sc->d0 = o[1];
    sc->rnorm = sqrt(o[0]);
    sc->iters += 1;
    if (!(sc->rnorm < INFINITY)) {
      sc->done = 1;
      sc->status = 2;
    } else if (sc->rnorm > 1e3 * sc->bnorm) {
      sc->done = 1;  // diverging (seen with FP32 vectors on stiff systems)
      sc->status = 3;
    } else if ((nseg > 1 ? conv : sc->rnorm <= sc->rtol * sc->bnorm) || sc->iters >= sc->maxit) {
      sc->done = 1;
    } else if (sc->omega == 0.0 || sc->d0 == 0.0) {
      sc->done = 1;
      sc->status = 1;
    }
  }
}

// ---------------------------------------------------------------------------
// GCR(2) for scalar systems with a variable-free right preconditioner (Eisenstat,
// Elman and Schultz 1983, truncated to the two latest directions): z = M^-1 r,
// q = A z, orthogonalised against the stored A-images Q0, Q1 (orthonormal)
// with the same combination applied to z, normalised, then x += alpha P,
// r -= alpha Q with alpha = r.Q. One preconditioner application and one SpMV
// per iteration instead of BiCGStab's two of each; the residual norm is
// monotone.

// q = A z (scalar CSR); partial q.Q0, q.Q1
template <class TM, class TV>
__global__ void __launch_bounds__(KB) k_spmv_gcr(int nn, const int* __restrict__ rp, const int* __restrict__ cols,
                                                  const TM* __restrict__ A, const TV* __restrict__ z,
                                                  TV* __restrict__ q, const TV* __restrict__ Q0,
                                                  const TV* __restrict__ Q1, double* partials, const KScal* sc) {
  if (sc->done) return;
  double v[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = __ldg(rp + i); k < __ldg(rp + i + 1); ++k) s += double(A[k]) * double(z[__ldg(cols + k)]);
    const TV qs = TV(s);
    q[i] = qs;
    v[0] += double(qs) * double(Q0[i]);
    v[1] += double(qs) * double(Q1[i]);
  }
  block_reduce_store<2>(v, partials, MAX_PARTIALS);
}

// beta_j = q.Q_j (d0, d1)
__global__ void __launch_bounds__(KB) k_gcr_beta(KScal* sc, const double* partials, int nb) {
  if (sc->done) return;
  double o[2];
  final_reduce<2>(partials, nb, o);
  if (threadIdx.x == 0) {
    sc->d0 = o[0];
    sc->d1 = o[1];
  }
}

// z -= beta0 P0 + beta1 P1, q -= beta0 Q0 + beta1 Q1; partial q.q, r.q
template <class TV>
__global__ void __launch_bounds__(KB) k_gcr_orth(int n, TV* z, TV* q, const TV* P0, const TV* P1, const TV* Q0,
                                                  const TV* Q1, const TV* r, double* partials, const KScal* sc) {
  if (sc->done) return;
  const double b0 = sc->d0, b1 = sc->d1;
  double v[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    z[i] = TV(double(z[i]) - b0 * double(P0[i]) - b1 * double(P1[i]));
    const TV qn = TV(double(q[i]) - b0 * double(Q0[i]) - b1 * double(Q1[i]));
    q[i] = qn;
    v[0] += double(qn) * double(qn);
    v[1] += double(r[i]) * double(qn);
  }
  block_reduce_store<2>(v, partials, MAX_PARTIALS);
}

// 1/|q| (omega) and alpha = r.q / |q|; a vanishing q is a breakdown
__global__ void __launch_bounds__(KB) k_gcr_alpha(KScal* sc, const double* partials, int nb) {
  if (sc->done) return;
  double o[2];
  final_reduce<2>(partials, nb, o);
  if (threadIdx.x == 0) {
    const double nq = sqrt(o[0]);
    if (!(nq > 0.0) || !(nq < INFINITY)) {
      sc->done = 1;
      sc->status = nq < INFINITY ? 1 : 2;
      return;
    }
    sc->omega = 1.0 / nq;
    sc->alpha = o[1] / nq;
  }
}

// P = z / |q|, Q = q / |q| into the oldest slot; x += alpha P, r -= alpha Q;
// partial r.r
template <class TV>
__global__ void __launch_bounds__(KB) k_gcr_update(int n, TV* x, TV* r, const TV* z, const TV* q, TV* P, TV* Q,
                                                    double* partials, const KScal* sc) {
  if (sc->done) return;
  const double inv = sc->omega, al = sc->alpha;
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const TV pi = TV(double(z[i]) * inv), qi = TV(double(q[i]) * inv);
    P[i] = pi;
    Q[i] = qi;
    x[i] = TV(double(x[i]) + al * double(pi));
    const TV rn = TV(double(r[i]) - al * double(qi));
    r[i] = rn;
    v[0] += double(rn) * double(rn);
  }
  block_reduce_store<1>(v, partials, MAX_PARTIALS);
}

// residual norm and convergence test; an iteration that leaves the residual
// where it was (truncated GCR can stagnate when the preconditioned operator's
// symmetric part is not definite) ends the solve with status 1, and the
// caller falls back to BiCGStab
__global__ void __launch_bounds__(KB) k_gcr_end(KScal* sc, const double* partials, int nb, const double* seg_r2,
                                                 const double* seg_b2, int nseg) {
  if (sc->done) return;
  double o[1];
  final_reduce<1>(partials, nb, o);
  const double segmax = block_seg_max(seg_r2, seg_b2, nseg);
  if (threadIdx.x == 0) {
    sc->seg_rel = segmax;
    const double prev = sc->rnorm;
    sc->rnorm = sqrt(o[0]);
    sc->iters += 1;
    if (!(sc->rnorm < INFINITY)) {
      sc->done = 1;
      sc->status = 2;
    } else if ((nseg > 1 ? segmax <= sc->rtol : sc->rnorm <= sc->rtol * sc->bnorm) || sc->iters >= sc->maxit) {
      sc->done = 1;
    } else if (sc->rnorm > 0.9999 * prev) {
      sc->done = 1;
      sc->status = 1;
    }
  }
}

// ---------------------------------------------------------------------------
template <int B, class TM, class TV>
int KrylovSolver<B, TM, TV>::setup(int nn_, const int* rp_, const int* cols_, const int* dg_, cudaStream_t st_) {
  if (nn == nn_ && rp == rp_) return OA_OK;
  release();
  nn = nn_;
  rp = rp_;
  cols = cols_;
  dg = dg_;
  st = st_;
  const size_t n = (size_t)B * nn;
  for (int k = 0; k < 8; ++k) OA_CUDA(cudaMalloc(&vec[k], sizeof(TV) * n));
  OA_CUDA(cudaMalloc(&Minv, sizeof(double) * (size_t)B * B * nn));
  OA_CUDA(cudaMalloc(&partials, sizeof(double) * 3 * MAX_PARTIALS));
  OA_CUDA(cudaMalloc(&scal, sizeof(KScal)));
  OA_CUDA(cudaMallocHost(&hscal, sizeof(KScal)));
  return OA_OK;
}

template <int B, class TM, class TV>
size_t KrylovSolver<B, TM, TV>::storage_bytes(int nn_) {
  const size_t n = (size_t)B * nn_;
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  return 8 * up(sizeof(TV) * n) + up(sizeof(double) * (size_t)B * B * nn_) + up(sizeof(double) * 3 * MAX_PARTIALS) +
         up(sizeof(KScal));
}

template <int B, class TM, class TV>
int KrylovSolver<B, TM, TV>::attach(int nn_, const int* rp_, const int* cols_, const int* dg_, cudaStream_t st_,
                                    void* storage, size_t bytes) {
  release();
  if (bytes < storage_bytes(nn_)) return fail(OA_ERR_ARG, "Krylov: caller storage too small");
  nn = nn_;
  rp = rp_;
  cols = cols_;
  dg = dg_;
  st = st_;
  external = true;
  const size_t n = (size_t)B * nn;
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  char* p = static_cast<char*>(storage);
  for (int k = 0; k < 8; ++k) {
    vec[k] = p;
    p += up(sizeof(TV) * n);
  }
  Minv = reinterpret_cast<double*>(p);
  p += up(sizeof(double) * (size_t)B * B * nn);
  partials = reinterpret_cast<double*>(p);
  p += up(sizeof(double) * 3 * MAX_PARTIALS);
  scal = p;
  return OA_OK;
}

template <int B, class TM, class TV>
void KrylovSolver<B, TM, TV>::release() {
  if (!external) {
    for (auto& v : vec)
      if (v) cudaFree(v);
    if (Minv) cudaFree(Minv);
    if (partials) cudaFree(partials);
    if (scal) cudaFree(scal);
  }
  for (auto& v : vec) v = nullptr;
  external = false;
  if (hscal) cudaFreeHost(hscal);
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  graph_exec = nullptr;
  graph_A = nullptr;
  graph_amg = nullptr;
  Minv = nullptr;
  partials = nullptr;
  scal = nullptr;
  hscal = nullptr;
  nn = 0;
  rp = nullptr;
}

template <int B, class TM, class TV>
int KrylovSolver<B, TM, TV>::precond(const TV* in, TV* out) {
  constexpr bool kAmgOk = (B == 1) && std::is_same<TM, TV>::value;
  KScal* sc = static_cast<KScal*>(scal);
  if constexpr (kAmgOk) {
    if (amg) return amg->apply(reinterpret_cast<const TV*>(in), out, &sc->done, st);
  }
  const int gfull = (B * nn + KB - 1) / KB;
  k_prec<B, TV><<<gfull, KB, 0, st>>>(nn, reinterpret_cast<const TV*>(Minv), in, out, sc);
  count_launches(1);
  return OA_OK;
}

// x = 0, r = rh = b, p = v = 0, inverse (block) diagonal, device scalars; the
// GCR(2) direction slots start at zero (no stored directions yet)
template <int B, class TM, class TV>
template <class TB>
int KrylovSolver<B, TM, TV>::prologue(const TM* A, const TB* b, double rtol, int maxit, const double* rtol_dev,
                                      const int* maxit_dev, bool use_gcr) {
  const int n = B * nn;
  TV *x = static_cast<TV*>(vec[0]), *r = static_cast<TV*>(vec[1]), *rh = static_cast<TV*>(vec[2]),
     *p = static_cast<TV*>(vec[3]), *v = static_cast<TV*>(vec[4]);
  KScal* sc = static_cast<KScal*>(scal);
  const int gfull = (n + KB - 1) / KB;
  const int gv = gfull < MAX_PARTIALS ? gfull : MAX_PARTIALS;
  const int gr = (nn + KB - 1) / KB;
  k_build_minv<B, TM, TV><<<gr, KB, 0, st>>>(nn, rp, dg, A, reinterpret_cast<TV*>(Minv));
  k_init<TV, TB><<<gv, KB, 0, st>>>(n, b, x, r, rh, p, v, partials);
  k_init_scalars<<<1, KB, 0, st>>>(sc, partials, gv, rtol, maxit, rtol_dev, maxit_dev);
  count_launches(3);
  if (seg.on()) {
    k_seg_sumsq<TB><<<seg.nseg, KB, 0, st>>>(seg.ptr, seg.rows, b, seg.b2, nullptr);
    count_launches(1);
  }
  OA_CUDA(cudaGetLastError());
  if (use_gcr)
    for (int k = 4; k < 8; ++k) OA_CUDA(cudaMemsetAsync(vec[k], 0, sizeof(TV) * (size_t)n, st));
  return OA_OK;
}

// one chunk of check_every iterations; every kernel reads its scalars and the
// tolerance from device memory, so a chunk can be captured once and replayed
template <int B, class TM, class TV>
int KrylovSolver<B, TM, TV>::chunk(const TM* A, int check_every, bool use_gcr) {
  const int n = B * nn;
  TV *x = static_cast<TV*>(vec[0]), *r = static_cast<TV*>(vec[1]), *rh = static_cast<TV*>(vec[2]),
     *p = static_cast<TV*>(vec[3]), *v = static_cast<TV*>(vec[4]), *ph = static_cast<TV*>(vec[5]),
     *sh = static_cast<TV*>(vec[6]), *t = static_cast<TV*>(vec[7]);
  KScal* sc = static_cast<KScal*>(scal);
  const int gfull = (n + KB - 1) / KB;
  const int gv = gfull < MAX_PARTIALS ? gfull : MAX_PARTIALS;
  if (use_gcr) {
    // GCR(2) work vectors in the same buffers: x r z q P0 P1 Q0 Q1
    TV *gz = rh, *gq = p, *gP[2] = {v, ph}, *gQ[2] = {sh, t};
    for (int it = 0; it < check_every; ++it) {
      const int slot = it & 1;  // the older of the two stored directions
      if (int s = precond(r, gz)) return s;
      k_spmv_gcr<TM, TV><<<gv, KB, 0, st>>>(nn, rp, cols, A, gz, gq, gQ[0], gQ[1], partials, sc);
      k_gcr_beta<<<1, KB, 0, st>>>(sc, partials, gv);
      k_gcr_orth<TV><<<gv, KB, 0, st>>>(n, gz, gq, gP[0], gP[1], gQ[0], gQ[1], r, partials, sc);
      k_gcr_alpha<<<1, KB, 0, st>>>(sc, partials, gv);
      k_gcr_update<TV><<<gv, KB, 0, st>>>(n, x, r, gz, gq, gP[slot], gQ[slot], partials, sc);
      if (seg.on()) {
        k_seg_sumsq<TV><<<seg.nseg, KB, 0, st>>>(seg.ptr, seg.rows, r, seg.r2, &sc->done);
        count_launches(1);
      }
      k_gcr_end<<<1, KB, 0, st>>>(sc, partials, gv, seg.r2, seg.b2, seg.on() ? seg.nseg : 0);
    }
    count_launches(6L * check_every);
    OA_CUDA(cudaGetLastError());
    return OA_OK;
  }
  for (int it = 0; it < check_every; ++it) {
    k_p_update<TV><<<gfull, KB, 0, st>>>(n, p, r, v, sc);
    if (int s = precond(p, ph)) return s;
    k_spmv<B, TM, TV, 1><<<gv, KB, 0, st>>>(nn, rp, cols, A, ph, v, rh, nullptr, partials, sc);
    k_alpha<<<1, KB, 0, st>>>(sc, partials, gv);
    k_s_update<TV><<<gfull, KB, 0, st>>>(n, r, v, sc);
    if (int s = precond(r, sh)) return s;
    k_spmv<B, TM, TV, 2><<<gv, KB, 0, st>>>(nn, rp, cols, A, sh, t, r, nullptr, partials, sc);
    k_omega<<<1, KB, 0, st>>>(sc, partials, gv);
    k_x_update<TV><<<gv, KB, 0, st>>>(n, x, r, ph, sh, t, rh, partials, sc);
    if (seg.on()) {
      k_seg_sumsq<TV><<<seg.nseg, KB, 0, st>>>(seg.ptr, seg.rows, r, seg.r2, &sc->done);
      count_launches(1);
    }
    k_end_iter<<<1, KB, 0, st>>>(sc, partials, gv, seg.r2, seg.b2, seg.on() ? seg.nseg : 0);
  }
  count_launches(8L * check_every);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

template <int B, class TM, class TV>
template <class TB>
int KrylovSolver<B, TM, TV>::solve(const TM* A, const TB* b, TV*& xout, double rtol, int maxit, int* iters,
                                   double* res, int check_every, bool reuse_precond) {
  constexpr bool kAmgOk = (B == 1) && std::is_same<TM, TV>::value;
  KScal* sc = static_cast<KScal*>(scal);
  const bool use_gcr = gcr && B == 1;
  if (use_gcr && check_every % 2) return fail(OA_ERR_ARG, "GCR: iteration chunks must hold an even number of iterations");
  // OA_DEBUG: device time of the preconditioner set-up and of the whole solve
  const bool dbg = std::getenv("OA_DEBUG") != nullptr;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  if (dbg)
    for (auto& e : ev) {
      cudaEventCreate(&e);
    }
  if (dbg) cudaEventRecord(ev[0], st);
  if constexpr (kAmgOk) {
    if (amg && !reuse_precond) {
      if (int s = amg->numeric(reinterpret_cast<const TV*>(A), st)) return s;
    }
  }
  if (dbg) cudaEventRecord(ev[1], st);
  if (int s = prologue<TB>(A, b, rtol, maxit, nullptr, nullptr, use_gcr)) return s;
  if (use_graph && (graph_exec == nullptr || graph_A != (const void*)A || graph_chunk != check_every ||
                    graph_amg != (const void*)amg || graph_gcr != use_gcr)) {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
    cudaGraph_t g;
    OA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const long long l0 = launch_total();
    const int cs = chunk(A, check_every, use_gcr);
    const long long per_chunk = launch_total() - l0;
    const cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (cs) return cs;
    if (ce != cudaSuccess) return fail(OA_ERR_CUDA, std::string("Krylov chunk capture: ") + cudaGetErrorString(ce));
    OA_CUDA(cudaGraphInstantiate(&graph_exec, g, 0));
    cudaGraphDestroy(g);
    graph_A = A;
    graph_amg = amg;
    graph_chunk = check_every;
    graph_gcr = use_gcr;
    graph_launches = per_chunk;
    count_launches(-per_chunk);  // captured, not launched
  }
  int done_iters = 0;
  while (true) {
    if (use_graph) {
      OA_CUDA(cudaGraphLaunch(graph_exec, st));
      count_launches(graph_launches);
    } else if (int s = chunk(A, check_every, use_gcr)) {
      return s;
    }
    done_iters += check_every;
    // pinned staging when the solver owns its storage, else plain host memory
    void* hdst = hscal ? hscal : static_cast<void*>(hbuf);
    OA_CUDA(cudaMemcpyAsync(hdst, sc, sizeof(KScal), cudaMemcpyDeviceToHost, st));
    OA_CUDA(cudaStreamSynchronize(st));
    const KScal* h = static_cast<const KScal*>(hdst);
    if (h->done || done_iters >= maxit) break;
  }
  const KScal* h = static_cast<const KScal*>(hscal ? hscal : static_cast<void*>(hbuf));
  static_assert(sizeof(KScal) <= sizeof(hbuf), "host staging buffer too small");
  if (iters) *iters = h->iters;
  if (res) *res = seg.on() ? h->seg_rel : (h->bnorm > 0 ? h->rnorm / h->bnorm : 0.0);
  xout = static_cast<TV*>(vec[0]);
  last_status = h->status;
  if (dbg) {
    cudaEventRecord(ev[2], st);
    cudaEventSynchronize(ev[2]);
    float t_setup = 0.f, t_all = 0.f;
    cudaEventElapsedTime(&t_setup, ev[0], ev[1]);
    cudaEventElapsedTime(&t_all, ev[0], ev[2]);
    std::fprintf(stderr, "[oa] %s<%d,%s> n %d iters %d: precond set-up %.3f ms, solve %.3f ms\n",
                 use_gcr ? "GCR(2)" : "BiCGStab", B, sizeof(TV) == 4 ? "f32" : "f64", nn, h->iters, t_setup, t_all);
    for (auto& e : ev) cudaEventDestroy(e);
  }
  if (h->status == 2) return fail(OA_ERR_SOLVER, use_gcr ? "GCR: non-finite residual" : "BiCGStab: non-finite residual");
  return OA_OK;
}

template <int B, class TM, class TV>
template <class TB>
int KrylovSolver<B, TM, TV>::emit(GraphBuild& gb, cudaGraph_t g, Deps& d, int body, const TM* A, const TB* b,
                                  double rtol, int maxit, const double* rtol_dev, const int* maxit_dev, int maxit_cap,
                                  int check_every, bool gcr_mode, int branch_body) {
  const bool use_gcr = gcr_mode && B == 1;
  if (use_gcr && check_every % 2) return fail(OA_ERR_ARG, "GCR: iteration chunks must hold an even number of iterations");
  if (st != gb.st) return fail(OA_ERR_ARG, "Krylov graph: the solver's stream is not the capturing stream");
  const int lb = gb.new_body();
  if (lb < 0) return fail(OA_ERR_ARG, "Krylov graph: too many conditional bodies");
  cudaGraphConditionalHandle h;
  if (int s = gb.handle(g, &h)) return s;
  if (int s = gb.seg(g, d, body, [&]() -> int {
        if (int s2 = prologue<TB>(A, b, rtol, maxit, rtol_dev, maxit_dev, use_gcr)) return s2;
        return launch_loop_enter(gb, h, scal, lb, branch_body);
      }))
    return s;
  cudaGraph_t wb = nullptr;
  if (int s = gb.cond(g, d, h, cudaGraphCondTypeWhile, 1, &wb)) return s;
  Deps bd;
  const int cap = (maxit_cap + check_every - 1) / check_every + 2;
  return gb.seg(wb, bd, lb, [&]() -> int {
    if (int s2 = chunk(A, check_every, use_gcr)) return s2;
    return launch_loop_next(gb, h, scal, lb, cap);
  });
}

template struct KrylovSolver<1, double, double>;
template struct KrylovSolver<3, double, double>;
template struct KrylovSolver<1, float, float>;
template struct KrylovSolver<3, float, float>;
template int KrylovSolver<1, double, double>::solve<double>(const double*, const double*, double*&, double, int, int*, double*, int, bool);
template int KrylovSolver<3, double, double>::solve<double>(const double*, const double*, double*&, double, int, int*, double*, int, bool);
template int KrylovSolver<1, float, float>::solve<double>(const float*, const double*, float*&, double, int, int*, double*, int, bool);
template int KrylovSolver<1, float, float>::solve<float>(const float*, const float*, float*&, double, int, int*, double*, int, bool);
template int KrylovSolver<3, float, float>::solve<float>(const float*, const float*, float*&, double, int, int*, double*, int, bool);
#define OA_EMIT(B, TM, TV, TB)                                                                                   \
  template int KrylovSolver<B, TM, TV>::emit<TB>(GraphBuild&, cudaGraph_t, Deps&, int, const TM*, const TB*, double, \
                                                 int, const double*, const int*, int, int, bool, int);
OA_EMIT(1, double, double, double)
OA_EMIT(3, double, double, double)
OA_EMIT(1, float, float, float)
OA_EMIT(3, float, float, float)
#undef OA_EMIT

// ---------------------------------------------------------------------------
// FP64 residual for iterative refinement: r = b - A x (A in its stored
// precision, arithmetic in FP64), with partial ||r||^2.
template <class TM>
__global__ void __launch_bounds__(KB) k_residual(int nn, const int* __restrict__ rp, const int* __restrict__ cols,
                                                  const TM* __restrict__ A, const double* __restrict__ x,
                                                  const double* __restrict__ b, double* __restrict__ r,
                                                  double* partials) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) s += double(A[k]) * x[cols[k]];
    const double ri = b[i] - s;
    r[i] = ri;
    v[0] += ri * ri;
  }
  block_reduce_store<1>(v, partials, MAX_PARTIALS);
}

__global__ void __launch_bounds__(KB) k_norm_out(const double* partials, int nb, double* out) {
  double o[1];
  final_reduce<1>(partials, nb, o);
  if (threadIdx.x == 0) *out = sqrt(o[0]);
}

template <class TV>
__global__ void k_add_correction(int n, double* x, const TV* d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += double(d[i]);
}

template <class TM>
int fp64_residual(int nn, const int* rp, const int* cols, const TM* A, const double* x, const double* b, double* r,
                  double* partials, double* norm_dev, cudaStream_t st) {
  const int gf = (nn + KB - 1) / KB;
  const int g = gf < MAX_PARTIALS ? gf : MAX_PARTIALS;
  k_residual<TM><<<g, KB, 0, st>>>(nn, rp, cols, A, x, b, r, partials);
  k_norm_out<<<1, KB, 0, st>>>(partials, g, norm_dev);
  count_launches(2);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}
template int fp64_residual<float>(int, const int*, const int*, const float*, const double*, const double*, double*,
                                  double*, double*, cudaStream_t);
template int fp64_residual<double>(int, const int*, const int*, const double*, const double*, const double*, double*,
                                   double*, double*, cudaStream_t);

__global__ void __launch_bounds__(KB) k_sumsq_partial(int n, const double* __restrict__ v, double* partials) {
  double s[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s[0] += v[i] * v[i];
  block_reduce_store<1>(s, partials, MAX_PARTIALS);
}

__global__ void __launch_bounds__(KB) k_sum_out(const double* partials, int nb, double* out) {
  double o[1];
  final_reduce<1>(partials, nb, o);
  if (threadIdx.x == 0) *out = o[0];
}

int device_sumsq(int n, const double* v, double* out, double* partials, cudaStream_t st) {
  const int gf = (n + KB - 1) / KB;
  const int g = gf < MAX_PARTIALS ? gf : MAX_PARTIALS;
  k_sumsq_partial<<<g, KB, 0, st>>>(n, v, partials);
  k_sum_out<<<1, KB, 0, st>>>(partials, g, out);
  count_launches(2);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

int partials_size() { return 3 * MAX_PARTIALS; }

// per-component sums of squares of a [nn][3] vector (ordered two-stage tree)
template <class T>
__global__ void __launch_bounds__(KB) k_comp_sumsq3(int nn, const T* __restrict__ v, double* partials) {
  double s[3] = {0.0, 0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double a = double(v[3 * (size_t)i + k]);
      s[k] += a * a;
    }
  block_reduce_store<3>(s, partials, MAX_PARTIALS);
}

__global__ void __launch_bounds__(KB) k_sum3_out(const double* partials, int nb, double* out) {
  double o[3];
  final_reduce<3>(partials, nb, o);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) out[k] = o[k];
}

template <class T>
int device_comp_sumsq3(int nn, const T* v, double* out, double* partials, cudaStream_t st) {
  const int gf = (nn + KB - 1) / KB;
  const int g = gf < MAX_PARTIALS ? gf : MAX_PARTIALS;
  k_comp_sumsq3<T><<<g, KB, 0, st>>>(nn, v, partials);
  k_sum3_out<<<1, KB, 0, st>>>(partials, g, out);
  count_launches(2);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}
template int device_comp_sumsq3<float>(int, const float*, double*, double*, cudaStream_t);
template int device_comp_sumsq3<double>(int, const double*, double*, double*, cudaStream_t);

template <class TV>
int add_correction(int n, double* x, const TV* d, cudaStream_t st) {
  k_add_correction<TV><<<(n + KB - 1) / KB, KB, 0, st>>>(n, x, d);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}
template int add_correction<float>(int, double*, const float*, cudaStream_t);
template int add_correction<double>(int, double*, const double*, cudaStream_t);

template <class T>
int segment_sumsq(const Segments& sg, const T* v, double* out, cudaStream_t st) {
  if (!sg.on()) return OA_OK;
  k_seg_sumsq<T><<<sg.nseg, KB, 0, st>>>(sg.ptr, sg.rows, v, out, nullptr);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}
template int segment_sumsq<float>(const Segments&, const float*, double*, cudaStream_t);
template int segment_sumsq<double>(const Segments&, const double*, double*, cudaStream_t);

int segment_max_ratio(const Segments& sg, double* out, cudaStream_t st) {
  k_seg_max_ratio<<<1, KB, 0, st>>>(sg.r2, sg.b2, sg.nseg, out);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

// ---------------------------------------------------------------------------
// Control kernels of the conditional nodes of whole-iteration graphs (one
// thread each; the condition is set by the graph that holds the node, or by
// the node's own body).
namespace {
__global__ void k_set_if(cudaGraphConditionalHandle h, const int* flag, int negate) {
  cudaGraphSetConditional(h, ((*flag != 0) != (negate != 0)) ? 1u : 0u);
}
__global__ void k_count_body(BodyCounters* c, int body) { c->total[body] += 1; }
__global__ void k_loop_enter(cudaGraphConditionalHandle h, const KScal* sc, BodyCounters* c, int body,
                             int branch_body) {
  c->cur[body] = 0;
  if (branch_body >= 0) c->total[branch_body] += 1;
  cudaGraphSetConditional(h, sc->done ? 0u : 1u);
}
__global__ void k_loop_next(cudaGraphConditionalHandle h, const KScal* sc, BodyCounters* c, int body, int cap) {
  const int n = ++c->cur[body];
  c->total[body] += 1;
  cudaGraphSetConditional(h, (!sc->done && n < cap) ? 1u : 0u);
}
}  // namespace

int launch_set_if(GraphBuild& gb, cudaGraphConditionalHandle h, const int* flag, bool negate) {
  k_set_if<<<1, 1, 0, gb.st>>>(h, flag, negate ? 1 : 0);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}
int launch_count_body(GraphBuild& gb, int body) {
  k_count_body<<<1, 1, 0, gb.st>>>(gb.ctr, body);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}
int launch_loop_enter(GraphBuild& gb, cudaGraphConditionalHandle h, const void* kscal, int body, int branch_body) {
  k_loop_enter<<<1, 1, 0, gb.st>>>(h, static_cast<const KScal*>(kscal), gb.ctr, body, branch_body);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}
int launch_loop_next(GraphBuild& gb, cudaGraphConditionalHandle h, const void* kscal, int body, int cap) {
  k_loop_next<<<1, 1, 0, gb.st>>>(h, static_cast<const KScal*>(kscal), gb.ctr, body, cap);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}
int launch_counters_reset(GraphBuild& gb) {
  OA_CUDA(cudaMemsetAsync(gb.ctr, 0, sizeof(BodyCounters), gb.st));
  return OA_OK;
}

}  // namespace oa
