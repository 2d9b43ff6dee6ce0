/* C++ surface of the reference's linear-solver context, for the drop-in
 * binding of the openaccel_b200 C-ABI behind OpenAccel's assemblers.
 *
 * The reference's assemblers and linear systems talk to an external library
 * (liblinsolve, an empty submodule in the reference checkout) through
 * linearSolver::Context<N> and its Matrix / Vector; this header rebuilds that
 * surface from its call sites in the reference:
 *   Context: getAMatrix, getBVector, getXVector, getRVector, zeroSystemStorage,
 *            getControlData, getResidualScales, getControlResidual,
 *            getCallCount, getSystemName (src/equation/linearSystem.h:416-571,
 *            src/assemble/assembler.h:21-309);
 *   Matrix:  rowVals(lid) (N*N*len values of a block row), rowCols(lid) (its
 *            sorted column ids), diag(lid) (the N x N diagonal block),
 *            dofDiag(lid, dof), diagOffsetRef(), nRows(),
 *            getGraph()->isLocalColumnOrder() (src/assemble/assembler.h:311-453
 *            and the assemblers' boundary code);
 *   Vector:  operator[], size(), data();
 *   ControlData: n_iterations, solver_initial_res, solver_final_res,
 *            scaled_initial_res (src/equation/linearSystem.h:473-488).
 * Storage is the reference's layout: block-CSR rows in node order, columns
 * sorted ascending, N x N row-major blocks, one diagonal offset per row. The
 * matrices live on the host here; the device copies belong to the oa_flow
 * handle, and openaccel_b200::assemble_into / solve below move data between
 * the two only when the caller asks (the reference dumps its systems the same
 * way). Errors from the C-ABI become std::runtime_error with oa_last_error(),
 * the reference's errorMsg convention (src/basic/macros.cpp:21-24).
 *
 * Header only; C++20 (std::span), as the reference itself. */
#ifndef OPENACCEL_B200_COMPAT_LINEAR_SOLVER_CONTEXT_H
#define OPENACCEL_B200_COMPAT_LINEAR_SOLVER_CONTEXT_H

#include <array>
#include <cstddef>
#include <span>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../openaccel_b200.h"

namespace linearSolver {

/* CSR node graph (the reference's CRSNodeGraph): rowPtr[n+1], sorted cols,
 * the diagonal's offset within each row. */
struct CRSNodeGraph {
  std::vector<int> rowPtr, cols, diagOffset;
  bool localColumnOrder = true;
  bool isLocalColumnOrder() const { return localColumnOrder; }
  int nRows() const { return rowPtr.empty() ? 0 : static_cast<int>(rowPtr.size()) - 1; }
  int nnz() const { return rowPtr.empty() ? 0 : rowPtr.back(); }
};

template <std::size_t N>
class Matrix {
 public:
  explicit Matrix(const CRSNodeGraph* g) : graph_(g), vals_(N * N * static_cast<std::size_t>(g->nnz()), 0.0) {}
  std::span<double> rowVals(int lid) {
    const std::size_t a = graph_->rowPtr[lid], b = graph_->rowPtr[lid + 1];
    return {vals_.data() + N * N * a, N * N * (b - a)};
  }
  std::span<const int> rowCols(int lid) const {
    const std::size_t a = graph_->rowPtr[lid], b = graph_->rowPtr[lid + 1];
    return {graph_->cols.data() + a, b - a};
  }
  double* diag(int lid) { return vals_.data() + N * N * (graph_->rowPtr[lid] + graph_->diagOffset[lid]); }
  double& dofDiag(int lid, int dof) { return diag(lid)[N * dof + dof]; }
  const std::vector<int>& diagOffsetRef() const { return graph_->diagOffset; }
  int nRows() const { return graph_->nRows(); }
  const CRSNodeGraph* getGraph() const { return graph_; }
  double* data() { return vals_.data(); }
  std::size_t size() const { return vals_.size(); }
  void zero() { std::fill(vals_.begin(), vals_.end(), 0.0); }

 private:
  const CRSNodeGraph* graph_;
  std::vector<double> vals_;
};

template <std::size_t N>
class Vector {
 public:
  explicit Vector(std::size_t rows) : v_(N * rows, 0.0) {}
  double& operator[](std::size_t i) { return v_[i]; }
  const double& operator[](std::size_t i) const { return v_[i]; }
  std::size_t size() const { return v_.size(); }
  double* data() { return v_.data(); }
  void zero() { std::fill(v_.begin(), v_.end(), 0.0); }

 private:
  std::vector<double> v_;
};

/* Coefficient scaling the linear system applies before a solve when asked
 * (linearSystem::solveSystem_, src/equation/linearSystem.h:416-462: normalize,
 * diagonalScale). The absent library's own definitions are not in the
 * reference checkout; this reconstruction scales every equation (row i, dof
 * m) of A and b by the inverse of its diagonal coefficient, so the diagonal
 * becomes 1 and the solution is unchanged, for both calls. */
template <std::size_t N>
class Coefficients {
 public:
  Coefficients(Matrix<N>& A, Vector<N>& b) : A_(A), b_(b) {}
  void normalize() { scale_rows(); }
  void diagonalScale() { scale_rows(); }

 private:
  void scale_rows() {
    for (int i = 0; i < A_.nRows(); ++i) {
      const auto vals = A_.rowVals(i);
      const std::size_t len = vals.size() / (N * N);
      for (std::size_t m = 0; m < N; ++m) {
        const double d = A_.dofDiag(i, static_cast<int>(m));
        if (d == 0.0) continue;
        const double inv = 1.0 / d;
        for (std::size_t k = 0; k < len; ++k)
          for (std::size_t q = 0; q < N; ++q) vals[N * N * k + N * m + q] *= inv;
        b_[N * static_cast<std::size_t>(i) + m] *= inv;
      }
    }
  }
  Matrix<N>& A_;
  Vector<N>& b_;
};

template <std::size_t N>
struct ControlData {
  int n_iterations = 0;
  std::array<double, N> solver_initial_res{}, solver_final_res{}, scaled_initial_res{};
};

template <std::size_t N>
class Context {
 public:
  static constexpr int BLOCKSIZE = static_cast<int>(N);
  using Matrix = linearSolver::Matrix<N>;
  using Vector = linearSolver::Vector<N>;
  using Array = std::array<double, N>;
  using Index = int;  // column id type of rowCols (32-bit ids: one rank, local = global order)

  Context(std::string name, const CRSNodeGraph* g)
      : name_(std::move(name)), A_(g), b_(g->nRows()), x_(g->nRows()), r_(g->nRows()) {
    scales_.fill(1.0);
  }
  Matrix& getAMatrix() { return A_; }
  Vector& getBVector() { return b_; }
  Vector& getXVector() { return x_; }
  Vector& getRVector() { return r_; }
  void zeroSystemStorage() {
    A_.zero();
    b_.zero();
    x_.zero();
    r_.zero();
  }
  Coefficients<N> getCoefficients() { return Coefficients<N>(A_, b_); }
  ControlData<N>& getControlData() { return cdata_; }
  Array& getResidualScales() { return scales_; }
  Array& getControlResidual() { return control_; }
  int getCallCount() const { return calls_; }
  void countCall() { ++calls_; }
  const std::string& getSystemName() const { return name_; }

 private:
  std::string name_;
  Matrix A_;
  Vector b_, x_, r_;
  ControlData<N> cdata_;
  Array scales_{}, control_{};
  int calls_ = 0;
};

}  // namespace linearSolver

namespace openaccel_b200 {

/* C-ABI status -> std::runtime_error with oa_last_error() (errorMsg). */
inline void check(int status) {
  if (status != OA_OK) throw std::runtime_error(std::string("openaccel_b200: ") + oa_last_error());
}

/* The CSR graph of a device mesh, with the diagonal offsets. */
inline linearSolver::CRSNodeGraph graph_of(const oa_mesh* m, int nn) {
  linearSolver::CRSNodeGraph g;
  int nnz = 0;
  check(oa_mesh_nnz(m, &nnz));
  g.rowPtr.resize(static_cast<std::size_t>(nn) + 1);
  g.cols.resize(static_cast<std::size_t>(nnz));
  check(oa_mesh_graph(m, g.rowPtr.data(), g.cols.data()));
  g.diagOffset.resize(static_cast<std::size_t>(nn));
  for (int i = 0; i < nn; ++i)
    for (int k = g.rowPtr[i]; k < g.rowPtr[i + 1]; ++k)
      if (g.cols[k] == i) g.diagOffset[i] = k - g.rowPtr[i];
  return g;
}

/* Assemble on the device and copy the system into the Context: N = 3 the
 * momentum system (navierStokesAssembler::assemble), N = 1 the pressure
 * correction (pressureCorrectionAssembler::assemble with the pressure-level
 * row). The device copy stays the one oa_solve uses. */
template <std::size_t N>
void assemble_into(oa_flow* f, linearSolver::Context<N>& ctx) {
  static_assert(N == 1 || N == 3, "momentum (3) or pressure correction (1)");
  ctx.zeroSystemStorage();
  if constexpr (N == 3)
    check(oa_assemble_momentum(f, ctx.getAMatrix().data(), ctx.getBVector().data()));
  else
    check(oa_assemble_pcorr(f, ctx.getAMatrix().data(), ctx.getBVector().data()));
}

/* Solve the last assembled system on the device (linearSystem::solve), copy
 * the solution into the Context's X vector and its ControlData. */
template <std::size_t N>
void solve(oa_flow* f, linearSolver::Context<N>& ctx, double rtol, int maxit) {
  static_assert(N == 1 || N == 3, "momentum (3) or pressure correction (1)");
  const int sys = N == 3 ? 0 : 1;
  int iters = 0;
  double res = 0.0;
  check(oa_solve(f, sys, rtol, maxit, ctx.getXVector().data(), &iters, &res));
  oa_control_data cd{};
  check(oa_flow_last_control(f, sys, &cd));
  auto& out = ctx.getControlData();
  out.n_iterations = cd.n_iterations;
  for (std::size_t i = 0; i < N; ++i) {
    out.solver_initial_res[i] = cd.solver_initial_res[i];
    out.solver_final_res[i] = cd.solver_final_res[i];
    out.scaled_initial_res[i] = cd.scaled_initial_res[i];
  }
  ctx.countCall();
}

}  // namespace openaccel_b200

#endif
