// Aggregation algebraic multigrid preconditioner (internal).
//
// The reference's pressure-correction systems go to liblinsolve's PETSc /
// Trilinos (ILU) / HYPRE (BoomerAMG) back ends (examples/cavity/input.i:61-77),
// which are absent. This is an unsmoothed-aggregation AMG V-cycle built for
// the device: the hierarchy's structure (aggregates, coarse graphs and the
// fine-entry -> coarse-entry gather lists) depends only on the CSR graph and is
// built once on the host; the numeric Galerkin products run on the device
// every time the fine matrix is reassembled, as deterministic owner gathers.
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace oa {

template <class T>
struct AmgLevel {
  int n = 0, nnz = 0;
  int *rp = nullptr, *cols = nullptr, *diag = nullptr;  // device CSR graph
  T* A = nullptr;                                       // values (level 0: borrowed)
  T* dinv = nullptr;                                    // 1 / diagonal
  // restriction/prolongation to the next level (piecewise constant)
  int* agg = nullptr;                  // [n] coarse index of each row
  int *mptr = nullptr, *mlist = nullptr;  // coarse row -> member rows
  // Galerkin gather of the NEXT level's values: coarse entry c sums this
  // level's entries glist[gptr[c] .. gptr[c+1])
  int *gptr = nullptr, *glist = nullptr;
  // cycle work vectors: x (output, levels > 0), b (input, levels > 0), r
  // (residual), t (pre-smoothed iterate)
  T *x = nullptr, *b = nullptr, *r = nullptr, *t = nullptr;
  bool own_A = false;
};

template <class T>
struct Amg {
  std::vector<AmgLevel<T>> L;
  double* dense_inv = nullptr;    // coarsest level inverse (FP64, n x n)
  double* h_dense = nullptr;      // pinned staging
  int coarse_n = 0;
  double omega = 0.7;             // Jacobi damping
  double alpha = 1.8;             // coarse-correction scaling (over-correction of the
                                  // piecewise-constant prolongation; 1.8-2 halves the
                                  // Krylov iterations on the 128^3 cavity)
  int pre = 1, post = 1;          // smoothing sweeps
  bool ready = false;

  // structure from the fine graph (host arrays); device pointers of the fine
  // graph are borrowed for level 0
  int setup(int n, const int* h_rp, const int* h_cols, const int* h_diag, int* d_rp, int* d_cols, int* d_diag);
  // numeric: coarse operators and inverse diagonals from the fine values
  int numeric(const T* A_fine, cudaStream_t st);
  // z = M^-1 v (one V-cycle from zero initial guess); kernels return early when *done
  int apply(const T* v, T* z, const int* done, cudaStream_t st);
  void release();
  ~Amg() { release(); }
};

}  // namespace oa
