// Allocation-free pressure-correction solve.
//
// Some callers cannot allocate device memory at the point where they need a
// solve: host applications that reserve the whole device up front and hand
// out slices of it themselves (a cudaMalloc would fail or break their
// accounting), and solver plug-ins called from a framework that forbids
// allocation on its hot path (an allocation there can synchronise the device
// or fragment the pool the framework manages). oa_pcorr_solve_static serves
// them: the caller passes the system and the solution in device memory it
// already owns, and the BiCGStab work vectors live in one file-scope device
// array of fixed size instead of cudaMalloc'd buffers. Nothing here calls
// cudaMalloc, cudaFree or an allocating library routine.
//
// Limits and sharing rules:
//  - at most OA_STATIC_SOLVE_MAX_ROWS rows; larger systems are rejected;
//  - the array (about 9.5 MB) stays resident on every GPU that loads this
//    library, until the process exits;
//  - every call on a device uses the same array, so calls whose work overlaps
//    on the GPU (different streams or threads) race and corrupt each other;
//    serialise them. The array keeps the previous call's contents; the solver
//    overwrites every region it reads before reading it (the iterate and the
//    search directions start from zero fills it issues itself);
//  - the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) and caches it;
//  - a breakdown, a diverging iteration or a solve that ends above rtol
//    returns OA_ERR_SOLVER (the status is named in oa_last_error); x then
//    holds the last iterate.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "oa_internal.h"
#include "oa_krylov.h"

namespace {

constexpr int kMaxRows = OA_STATIC_SOLVE_MAX_ROWS;
// 8 Krylov vectors + Jacobi inverse + reduction partials + scalars, with the
// 256-byte sub-allocation padding KrylovSolver::attach uses
constexpr size_t kScratchDoubles = 9 * (size_t)kMaxRows + 3 * 2048 + 4096;

static __device__ __align__(256) double g_static_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of g_static_scratch on the current device (resolved once per
// device). In host code g_static_scratch itself is only a host-side stand-in.
int scratch_for_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return oa::fail(OA_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return oa::fail(OA_ERR_ARG, "oa_pcorr_solve_static: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    double* p = nullptr;
    e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_static_scratch);
    if (e != cudaSuccess)
      return oa::fail(OA_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return OA_OK;
}

}  // namespace

extern "C" int oa_pcorr_solve_static(int nn, const int* row_ptr, const int* cols, const int* diag, const double* A,
                                     const double* b, double* x, double rtol, int maxit, int* iters, double* res,
                                     void* stream) {
  if (nn <= 0 || !row_ptr || !cols || !diag || !A || !b || !x || maxit <= 0)
    return oa::fail(OA_ERR_ARG, "oa_pcorr_solve_static: bad arguments");
  if (nn > kMaxRows)
    return oa::fail(OA_ERR_ARG, "oa_pcorr_solve_static: " + std::to_string(nn) + " rows exceed the static limit of " +
                                    std::to_string(kMaxRows));
  double* scratch = nullptr;
  if (int s = scratch_for_current_device(&scratch)) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  oa::KrylovSolver<1, double, double> ks;  // no storage of its own: attached below
  if (int s = ks.attach(nn, row_ptr, cols, diag, st, scratch, sizeof(double) * kScratchDoubles)) return s;
  double* xs = nullptr;
  double r = 0.0;
  int s = ks.solve<double>(A, b, xs, rtol, maxit, iters, &r, 20);
  if (res) *res = r;
  if (s == OA_OK) {
    cudaError_t e = cudaMemcpyAsync(x, xs, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) s = oa::fail(OA_ERR_CUDA, std::string("oa_pcorr_solve_static: ") + cudaGetErrorString(e));
  }
  if (s == OA_OK && (ks.last_status == 1 || ks.last_status == 3 || !(r <= rtol))) {
    const char* why = ks.last_status == 1 ? "breakdown (status 1)"
                      : ks.last_status == 3 ? "diverging residual (status 3)"
                                            : "not converged within maxit (status 0)";
    char msg[160];
    std::snprintf(msg, sizeof msg, "oa_pcorr_solve_static: BiCGStab %s, relative residual %.3e > rtol %.3e", why, r,
                  rtol);
    s = oa::fail(OA_ERR_SOLVER, msg);
  }
  ks.release();
  return s;
}
