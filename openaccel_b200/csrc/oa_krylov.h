// Device Krylov solver interface (internal).
#pragma once
#include <cuda_runtime.h>

#include "oa_amg.h"
#include "oa_graph.h"

namespace oa {

// Device scalars of one Krylov solve (read by every iteration kernel).
struct KScal {
  double rho, alpha, omega, bnorm, rnorm;
  double d0, d1, d2;  // reduced dots of the current phase
  double rtol;
  int maxit;
  int done, iters, status;
  double seg_rel;  // segmented solves: largest per-segment ||r|| / ||b|| at the last test
};

// Independent systems solved as one (a batch of disjoint meshes): the rows of
// each segment (seg_rows[seg_ptr[s] .. seg_ptr[s+1])) and scratch for the
// per-segment sums of squares of b and r. With nseg > 1 a solve has converged
// when every segment's ||r_s|| <= rtol ||b_s||, not when the whole batch's
// norm is.
struct Segments {
  int nseg = 0;
  const int* ptr = nullptr;
  const int* rows = nullptr;
  double* b2 = nullptr;  // [nseg]
  double* r2 = nullptr;  // [nseg]
  bool on() const { return nseg > 1; }
};
// per-segment sums of squares of v into out[nseg] (one block per segment,
// fixed order)
template <class T>
int segment_sumsq(const Segments& sg, const T* v, double* out, cudaStream_t st);
// largest sqrt(r2[s] / b2[s]) over segments (0 where b2 = 0) into *out
int segment_max_ratio(const Segments& sg, double* out, cudaStream_t st);

// BiCGStab on a BSR matrix with BxB blocks; matrix values TM, vectors TV.
template <int B, class TM, class TV>
struct KrylovSolver {
  int nn = 0;
  const int *rp = nullptr, *cols = nullptr, *dg = nullptr;
  cudaStream_t st = nullptr;
  void* vec[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  double* Minv = nullptr;  // Jacobi inverse, B*B*nn values stored as TV (room for FP64)
  double* partials = nullptr;
  void* scal = nullptr;
  void* hscal = nullptr;
  int last_status = 0;  // 0 ok, 1 breakdown, 2 non-finite, 3 diverging
  // optional AMG preconditioner (scalar systems); null = point/block Jacobi
  Amg<TV>* amg = nullptr;
  bool gcr = false;  // scalar systems: GCR(2) instead of BiCGStab (chunks of an even iteration count)
  // CUDA-graph replay of the iteration chunk (captured on first use)
  bool use_graph = false;
  cudaGraphExec_t graph_exec = nullptr;
  const void* graph_A = nullptr;
  const void* graph_amg = nullptr;
  int graph_chunk = 0;
  bool graph_gcr = false;
  long long graph_launches = 0;

  // per-segment convergence (batched disjoint systems); off by default
  Segments seg;
  // storage carved from caller memory instead of cudaMalloc (no allocation)
  bool external = false;
  alignas(16) unsigned char hbuf[128];  // host copy of the scalars when not pinned

  // the solver's residual vector (b - A x, updated by recurrence) after solve()
  const TV* residual() const { return static_cast<const TV*>(vec[1]); }
  int setup(int nn, const int* rp, const int* cols, const int* dg, cudaStream_t st);
  static size_t storage_bytes(int nn);
  int attach(int nn, const int* rp, const int* cols, const int* dg, cudaStream_t st, void* storage, size_t bytes);
  void release();
  ~KrylovSolver() { release(); }
  // Solve A x = b from x0 = 0; xout points at the solver-owned solution.
  template <class TB>
  // reuse_precond: keep the preconditioner built for the same A by the
  // previous call (iterative-refinement passes)
  int solve(const TM* A, const TB* b, TV*& xout, double rtol, int maxit, int* iters, double* res,
            int check_every, bool reuse_precond = false);

  // Graph form of solve() (whole-iteration graphs): its prologue (x = 0,
  // r = b, device scalars; rtol and maxit read on the device when rtol_dev /
  // maxit_dev are given) and a WHILE node over chunks of check_every
  // iterations, captured into g after d. The preconditioner's numeric phase is
  // left to the caller. gcr_mode: GCR(2) (scalar AMG systems) or BiCGStab.
  // The loop is capped at maxit_cap / check_every + 2 passes on the device.
  // branch_body >= 0: g is that IF body, counted once per execution here.
  template <class TB>
  int emit(GraphBuild& gb, cudaGraph_t g, Deps& d, int body, const TM* A, const TB* b, double rtol, int maxit,
           const double* rtol_dev, const int* maxit_dev, int maxit_cap, int check_every, bool gcr_mode,
           int branch_body);
  const KScal* scalars() const { return static_cast<const KScal*>(scal); }
  // forget the captured chunk (its preconditioner launches changed)
  void drop_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
  }
  TV* solution() const { return static_cast<TV*>(vec[0]); }

 private:
  int precond(const TV* in, TV* out);
  template <class TB>
  int prologue(const TM* A, const TB* b, double rtol, int maxit, const double* rtol_dev, const int* maxit_dev,
               bool use_gcr);
  int chunk(const TM* A, int check_every, bool use_gcr);
};

// r = b - A x in FP64 arithmetic (A scalar CSR in its stored precision);
// ||r|| written to norm_dev.
template <class TM>
int fp64_residual(int nn, const int* rp, const int* cols, const TM* A, const double* x, const double* b, double* r,
                  double* partials, double* norm_dev, cudaStream_t st);
template <class TV>
int add_correction(int n, double* x, const TV* d, cudaStream_t st);
// sum of squares of v into *out (device), ordered two-stage reduction;
// partials must hold partials_size() doubles
int device_sumsq(int n, const double* v, double* out, double* partials, cudaStream_t st);
// per-component sums of squares of a [nn][3] vector into out[3] (device)
template <class T>
int device_comp_sumsq3(int nn, const T* v, double* out, double* partials, cudaStream_t st);
int partials_size();

}  // namespace oa
