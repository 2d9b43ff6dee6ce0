// Scalar linear solve with optional FP32 inner iterations and FP64 iterative
// refinement (shared by the pressure-correction and scalar-diffusion paths).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "oa_internal.h"
#include "oa_scalar_solve.h"

namespace oa {

namespace {
__global__ void k_narrow(int n, const double* __restrict__ a, float* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = float(a[i]);
}
}  // namespace

int ScalarSolve::init(int nn) {
  if (const char* e = std::getenv("OA_AMG_REFRESH")) refresh = std::max(1, std::atoi(e));
  if (const char* e = std::getenv("OA_IR_INNER")) inner_floor = std::atof(e);
  if (const char* e = std::getenv("OA_KRYLOV")) gcr = std::strcmp(e, "bicgstab") != 0;
  if (const char* e = std::getenv("OA_GCR_CHUNK")) gcr_chunk = std::max(2, std::atoi(e) / 2 * 2);
  if (n == nn && r) return OA_OK;
  release();
  n = nn;
  if (cudaMalloc(&r, sizeof(double) * (nn ? nn : 1)) != cudaSuccess ||
      cudaMalloc(&r32, sizeof(float) * (nn ? nn : 1)) != cudaSuccess ||
      cudaMalloc(&scal, sizeof(double) * 2) != cudaSuccess ||
      cudaMalloc(&partials, sizeof(double) * partials_size()) != cudaSuccess ||
      cudaMallocHost(&hscal, sizeof(double) * 2) != cudaSuccess) {
    release();
    return fail(OA_ERR_CUDA, "scalar solve: device allocation failed");
  }
  return OA_OK;
}

void ScalarSolve::release() {
  if (r) cudaFree(r);
  if (r32) cudaFree(r32);
  if (scal) cudaFree(scal);
  if (partials) cudaFree(partials);
  if (hscal) cudaFreeHost(hscal);
  r = nullptr;
  r32 = nullptr;
  scal = nullptr;
  partials = nullptr;
  hscal = nullptr;
  n = 0;
  k64.release();
  k32.release();
  amg64.release();
  amg32.release();
}

int ScalarSolve::solve(const ScalarGraph& g, bool mixed, bool amg, bool graphs, const void* A, const double* b,
                       double* x, double rtol, int maxit, int* iters, double* res, int* refinements, cudaStream_t st,
                       const char* what) {
  if (int s = init(g.nn)) return s;
  if (amg) {
    if (!mixed && !amg64.ready)
      if (int s = amg64.setup(g.nn, g.h_rp, g.h_cols, g.h_diag, g.rp, g.cols, g.diag)) return s;
    if (mixed && !amg32.ready)
      if (int s = amg32.setup(g.nn, g.h_rp, g.h_cols, g.h_diag, g.rp, g.cols, g.diag)) return s;
    k64.amg = mixed ? nullptr : &amg64;
    k32.amg = mixed ? &amg32 : nullptr;
  } else {
    k64.amg = nullptr;
    k32.amg = nullptr;
  }
  k64.use_graph = k32.use_graph = graphs;
  // with the AMG: GCR(2), one V-cycle per iteration (chunks of 4); with point
  // Jacobi: BiCGStab
  k64.gcr = k32.gcr = amg && gcr;
  int check_every = amg ? (gcr ? gcr_chunk : 5) : 20;
  // AMG numeric phase every refresh-th solve (the fine matrix is always the
  // current one; the coarse operators may lag by refresh - 1 assemblies)
  const bool reuse = amg && refresh > 1 && (solves++ % refresh) != 0;
  if (!mixed) {
    if (int s = k64.setup(g.nn, g.rp, g.cols, g.diag, st)) return s;
    double* xs = nullptr;
    if (int s = k64.solve<double>(static_cast<const double*>(A), b, xs, rtol, maxit, iters, res, check_every, reuse))
      return s;
    if (k64.gcr && k64.last_status == 1) {
      // GCR stagnated or broke down: BiCGStab from now on, and for this system;
      // the reported count includes the GCR iterations already spent
      gcr = false;
      k64.gcr = false;
      const int spent = iters ? *iters : 0;
      if (int s = k64.solve<double>(static_cast<const double*>(A), b, xs, rtol, maxit, iters, res, 5, true)) return s;
      if (iters) *iters += spent;
      ++fallbacks;
    }
    OA_CUDA(cudaMemcpyAsync(x, xs, sizeof(double) * g.nn, cudaMemcpyDeviceToDevice, st));
    if (refinements) *refinements = 0;
    return OA_OK;
  }
  if (int s = k32.setup(g.nn, g.rp, g.cols, g.diag, st)) return s;
  const float* A32 = static_cast<const float*>(A);
  OA_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * g.nn, st));
  if (int s = device_sumsq(g.nn, b, scal, partials, st)) return s;
  OA_CUDA(cudaMemcpyAsync(hscal, scal, sizeof(double), cudaMemcpyDeviceToHost, st));
  OA_CUDA(cudaStreamSynchronize(st));
  const double bnorm = std::sqrt(hscal[0]);
  if (!(bnorm < INFINITY)) return fail(OA_ERR_SOLVER, std::string(what) + ": non-finite right-hand side");
  int total = 0, nref = 0;
  double rel = bnorm > 0 ? 1.0 : 0.0;
  OA_CUDA(cudaMemcpyAsync(r, b, sizeof(double) * g.nn, cudaMemcpyDeviceToDevice, st));
  constexpr int INNER_CAP = 300;  // FP32 Krylov iterations per refinement
  while (rel > rtol && total < maxit && nref < 40) {
    k_narrow<<<(g.nn + 255) / 256, 256, 0, st>>>(g.nn, r, r32);
    count_launches(1);
    float* d = nullptr;
    int it = 0;
    double r_in = 0.0;
    // inner tolerance: enough digits for FP32 without stalling
    const double inner = std::max(rtol / rel, inner_floor > 0 ? inner_floor : (amg ? 1e-4 : 2e-4));
    if (int s = k32.solve<float>(A32, r32, d, std::min(inner, 0.1), std::min(INNER_CAP, maxit - total), &it, &r_in,
                                 check_every, reuse || nref > 0))
      return s;
    total += it;
    if (k32.gcr && k32.last_status == 1 && r_in > 10.0 * std::min(inner, 0.1)) {
      // GCR stagnated or broke down far from its target (its partial
      // correction still reduced the residual): BiCGStab for the remaining
      // passes and later solves. A stall within a decade of the target is the
      // FP32 floor and only ends the pass.
      gcr = false;
      k32.gcr = false;
      check_every = 5;
      ++fallbacks;
    }
    // a diverged inner solve contributes nothing; the next pass restarts from
    // the FP64 residual
    if (k32.last_status != 3 && r_in < 1.0) add_correction<float>(g.nn, x, d, st);
    if (int s = fp64_residual<float>(g.nn, g.rp, g.cols, A32, x, b, r, k32.partials, scal + 1, st)) return s;
    OA_CUDA(cudaMemcpyAsync(hscal + 1, scal + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    OA_CUDA(cudaStreamSynchronize(st));
    rel = bnorm > 0 ? hscal[1] / bnorm : 0.0;
    if (std::getenv("OA_DEBUG"))
      std::fprintf(stderr, "[oa] %s refinement %d: inner iters %d inner res %.3e |b| %.3e rel %.3e\n", what, nref, it,
                   r_in, bnorm, rel);
    ++nref;
    if (!(rel < INFINITY)) return fail(OA_ERR_SOLVER, std::string(what) + " refinement: non-finite residual");
    if (it == 0) break;
  }
  if (iters) *iters = total;
  if (res) *res = rel;
  if (refinements) *refinements = nref;
  return OA_OK;
}

}  // namespace oa
