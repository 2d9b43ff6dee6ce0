// Aggregation algebraic multigrid preconditioner (internal).
//
// The reference's pressure-correction systems go to liblinsolve's PETSc /
// Trilinos (ILU) / HYPRE (BoomerAMG) back ends (examples/cavity/input.i:61-77),
// which are absent. This is an aggregation AMG V-cycle built for the device,
// with either the smoothed prolongation P = (I - wp Dinv A) P_tent (default)
// or the piecewise-constant one with an over-corrected coarse correction. The
// hierarchy's structure (aggregates, coarse graphs, and the term lists of P,
// A P and P^T A P) depends only on the CSR graph and is built once on the host;
// the numeric products run on the device every time the fine matrix is
// reassembled, as deterministic owner sums.
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
  // smoothed prolongation P (CSR, n x nc): columns, offset of the row's own
  // aggregate, per entry the A entries whose column lies in that aggregate,
  // and values; P^T by coarse row (fine rows, P entry of each)
  int *p_rp = nullptr, *p_cols = nullptr, *p_diag = nullptr, *pg_ptr = nullptr, *pg_list = nullptr;
  T* pv = nullptr;
  int *pt_rp = nullptr, *pt_rows = nullptr, *pt_src = nullptr;
  T* ptv = nullptr;  // P^T values in coarse-row order
  int nnz_p = 0;
  // lanes per row of the row-parallel kernels (1, 8 or 32, from the average
  // row length): A, P, P^T, and the T / coarse term lists
  int lpr_a = 1, lpr_p = 1, lpr_pt = 1, lpr_t = 1, lpr_c = 1;
  // T = A P values and term lists (A entry, P entry); the next level's values
  // from term lists (P entry, T entry)
  int nnz_t = 0;
  T* tv = nullptr;
  int *tt_ptr = nullptr, *tt_a = nullptr, *tt_p = nullptr;
  int *ct_ptr = nullptr, *ct_p = nullptr, *ct_t = nullptr;
  // cycle work vectors: x (output, levels > 0), b (input, levels > 0), r
  // (residual), t (pre-smoothed iterate)
  T *x = nullptr, *b = nullptr, *r = nullptr, *t = nullptr;
  // Chebyshev smoother (small levels): preconditioned residual, two direction
  // buffers; the power-iteration estimate of the spectral radius of Dinv A
  // (lmax[1]) and its FP64 work arrays (matrix and Dinv copies, two vectors,
  // block partials)
  bool cheb = false;
  T *cr = nullptr, *cd0 = nullptr, *cd1 = nullptr;
  double* lmax = nullptr;
  double *pw_a = nullptr, *pw_dinv = nullptr, *pw_v = nullptr, *pw_w = nullptr, *pw_part = nullptr;
  bool own_A = false;
};

template <class T>
struct Amg {
  std::vector<AmgLevel<T>> L;
  double* dense_inv = nullptr;    // coarsest level inverse (FP64, n x n)
  double* h_dense = nullptr;      // pinned staging
  int coarse_n = 0;
  bool smoothed = true;           // smoothed (true) or piecewise-constant prolongation
  double omega = 0.8;             // Jacobi damping of the smoother
  double omega_p = 0.74;          // prolongation smoothing, 4 / (3 rho(Dinv A)) with rho ~ 1.8
  double alpha = 1.0;             // coarse-correction scaling (1.8 for the piecewise-constant
                                  // prolongation, whose over-correction halves the Krylov
                                  // iterations on the 128^3 cavity)
  int pre = 1, post = 1;          // smoothing sweeps
  // Chebyshev smoothing of the given degree (0: Jacobi everywhere) on every
  // coarse level above the coarsest with at most cheb_rows rows, over the interval
  // [lambda / cheb_ratio, lambda] of Dinv A, lambda 1.1 times its power
  // iteration estimate
  int cheb_degree = 3;
  int cheb_rows = 50000;
  double cheb_ratio = 30.0;
  long long cheb_launches = 0;    // extra launches per V-cycle of the Chebyshev levels
  bool ready = false;

  // structure from the fine graph (host arrays); device pointers of the fine
  // graph are borrowed for level 0
  int setup(int n, const int* h_rp, const int* h_cols, const int* h_diag, int* d_rp, int* d_cols, int* d_diag);
  // numeric: coarse operators and inverse diagonals from the fine values
  int numeric(const T* A_fine, cudaStream_t st);
  // z = M^-1 v (one V-cycle from zero initial guess); kernels return early when *done
  int apply(const T* v, T* z, const int* done, cudaStream_t st);
  // Chebyshev degree of the coarse-level smoother and prolongation damping;
  // before set-up they shape it, after it they take effect with the next
  // numeric phase (degree) and apply (launch count)
  int set_smoothing(int degree, double prolongation_damping);
  void release();
  ~Amg() { release(); }
};

}  // namespace oa
