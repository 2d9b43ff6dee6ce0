// Oracle (test infrastructure only): the reference's own
// assembler<N>::applyCoeff_ (src/assemble/assembler.h:311-453), compiled from
// the read-only reference tree against the stand-ins in oracle/refshim_asm/
// into oracle/_ref/libref_assembler.so by `make -C oracle ref`. Tests feed it
// the same element lhs / rhs as the oracle's restatement and compare.
#include <cstring>

#include "assembler.h"

namespace {

template <std::size_t N>
struct Probe : accel::assembler<N> {
  explicit Probe(accel::fieldBroker* fb) : accel::assembler<N>(fb) {}
  void assemble_(const accel::domain*, typename accel::assembler<N>::Context*) override {}
  using accel::assembler<N>::applyCoeff_;
};

template <std::size_t N>
int run(int nn, const int* rp, const int* cols, const int* diag_off, double* A, double* b, const int* nodes, int n,
        const double* rhs, const double* lhs, int deduct) {
  linearSolver::CRSNodeGraph g;
  g.rowPtr.assign(rp, rp + nn + 1);
  g.cols.assign(cols, cols + rp[nn]);
  g.diagOffset.assign(diag_off, diag_off + nn);
  linearSolver::Context<N> ctx("probe", &g);
  std::memcpy(ctx.getAMatrix().data(), A, sizeof(double) * ctx.getAMatrix().size());
  std::memcpy(ctx.getBVector().data(), b, sizeof(double) * ctx.getBVector().size());
  accel::fieldBroker fb(nn);
  Probe<N> p(&fb);
  std::vector<stk::mesh::Entity> nodesE(n);
  for (int k = 0; k < n; ++k) nodesE[k].id = static_cast<unsigned>(nodes[k]);
  std::vector<label> scratchIds;
  std::vector<scalar> scratchVals;
  std::vector<scalar> r(rhs, rhs + N * n), l(lhs, lhs + N * N * n * n);
  p.applyCoeff_(ctx.getAMatrix(), ctx.getBVector(), nodesE, scratchIds, scratchVals, r, l, deduct != 0);
  std::memcpy(A, ctx.getAMatrix().data(), sizeof(double) * ctx.getAMatrix().size());
  std::memcpy(b, ctx.getBVector().data(), sizeof(double) * ctx.getBVector().size());
  return 0;
}

}  // namespace

extern "C" int ref_apply_coeff(int N, int nn, const int* rp, const int* cols, const int* diag_off, double* A,
                               double* b, const int* nodes, int n, const double* rhs, const double* lhs, int deduct) {
  if (N == 1) return run<1>(nn, rp, cols, diag_off, A, b, nodes, n, rhs, lhs, deduct);
  if (N == 3) return run<3>(nn, rp, cols, diag_off, A, b, nodes, n, rhs, lhs, deduct);
  return 1;
}
