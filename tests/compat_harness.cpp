// C++ check of the drop-in binding: include/compat/linearSolverContext.h and
// the C-ABI, used the way a reference-side subclass would use them.
//
//   compat_harness cpu          host-only checks (no device needed)
//   compat_harness gpu DIR      assemble and solve a pressure correction on the
//                               device through the subclass below, on the mesh
//                               stored in DIR (coords.f64 [nn][3], conn.i32
//                               [ne][8], faces.i32 [nf][3], bnd.f64 [nb][3],
//                               sizes.i32 {nn, ne, nf, nb}); writes A.f64,
//                               b.f64, x.f64 and control.txt into DIR
//
// The reference's own assembler classes cannot be compiled here (they need
// Trilinos/STK), so minimal stand-ins with the same virtual signatures
// (src/assemble/assembler.h:21-309, pressureCorrectionAssembler.h:43) take
// their place; the subclass is the one INTEGRATION.md shows.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <stdexcept>
#include <string>
#include <vector>

#include "compat/linearSolverContext.h"

namespace accel {
struct domain {};
[[noreturn]] inline void errorMsg(const std::string& m) { throw std::runtime_error(m); }
template <std::size_t N>
class assembler {
 public:
  using Context = ::linearSolver::Context<N>;
  using Matrix = typename Context::Matrix;
  using Vector = typename Context::Vector;
  virtual ~assembler() = default;
  virtual void assemble(const domain* domain, Context* ctx) = 0;
};
class pressureCorrectionAssembler : public assembler<1> {
 public:
  virtual void adjustMatrixForPressureReference(const domain*, Context*) {}
};

// the binding a maintainer adds on the reference side
class gpuPressureCorrectionAssembler : public pressureCorrectionAssembler {
 public:
  explicit gpuPressureCorrectionAssembler(oa_flow* flow) : flow_(flow) {}
  void assemble(const domain*, Context* ctx) override { openaccel_b200::assemble_into(flow_, *ctx); }
  void adjustMatrixForPressureReference(const domain*, Context*) override {
    // done inside oa_assemble_pcorr (the flow's pressure-level rows)
  }

 private:
  oa_flow* flow_;
};
}  // namespace accel

#define EXPECT(c)                                                        \
  do {                                                                   \
    if (!(c)) {                                                          \
      std::fprintf(stderr, "%s:%d: expectation failed: %s\n", __FILE__, __LINE__, #c); \
      return 1;                                                          \
    }                                                                    \
  } while (0)

static int cpu_checks() {
  // block-CSR layout of a 3-node chain 0-1-2, N = 3
  linearSolver::CRSNodeGraph g;
  g.rowPtr = {0, 2, 5, 7};
  g.cols = {0, 1, 0, 1, 2, 1, 2};
  g.diagOffset = {0, 1, 1};
  linearSolver::Context<3> ctx("momentum", &g);
  auto& A = ctx.getAMatrix();
  EXPECT(A.nRows() == 3 && A.size() == 9u * 7u);
  EXPECT(A.rowVals(1).size() == 27u && A.rowCols(1).size() == 3u && A.rowCols(1)[2] == 2);
  EXPECT(A.diag(1) == A.rowVals(1).data() + 9);
  A.dofDiag(2, 1) = 5.0;
  EXPECT(A.data()[9 * 6 + 4] == 5.0);
  EXPECT(A.getGraph()->isLocalColumnOrder());
  ctx.getBVector()[8] = 1.0;
  EXPECT(ctx.getBVector().size() == 9u);
  ctx.zeroSystemStorage();
  EXPECT(A.data()[9 * 6 + 4] == 0.0 && ctx.getBVector()[8] == 0.0);
  // C-ABI errors surface as std::runtime_error carrying oa_last_error()
  bool threw = false;
  try {
    openaccel_b200::check(oa_flow_sync(nullptr));
  } catch (const std::runtime_error& e) {
    threw = std::strstr(e.what(), "null handle") != nullptr;
  }
  EXPECT(threw);
  oa_control_data cd{};
  EXPECT(oa_flow_last_control(nullptr, 1, &cd) == OA_ERR_ARG);
  EXPECT(oa_mesh_create(nullptr, 0, nullptr, 0, OA_TOPO_HEX8, nullptr, nullptr, nullptr, 0, nullptr) == OA_ERR_ARG);
  EXPECT(std::strstr(oa_version(), "sm_100a") != nullptr);
  std::printf("compat cpu ok\n");
  return 0;
}

template <class T>
static std::vector<T> read_file(const std::string& path, std::size_t n) {
  std::vector<T> v(n);
  std::ifstream f(path, std::ios::binary);
  if (!f.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(sizeof(T) * n)))
    throw std::runtime_error("cannot read " + path);
  return v;
}

template <class T>
static void write_file(const std::string& path, const T* p, std::size_t n) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(p), static_cast<std::streamsize>(sizeof(T) * n));
}

static int gpu_checks(const std::string& dir) {
  const auto sz = read_file<int>(dir + "/sizes.i32", 4);
  const int nn = sz[0], ne = sz[1], nf = sz[2], nb = sz[3];
  const auto x = read_file<double>(dir + "/coords.f64", 3ul * nn);
  const auto conn = read_file<int>(dir + "/conn.i32", 8ul * ne);
  const auto faces = read_file<int>(dir + "/faces.i32", 3ul * nf);
  const auto bnd = read_file<double>(dir + "/bnd.f64", 3ul * nb);
  std::vector<int> fe(nf), fo(nf), fb(nf);
  for (int k = 0; k < nf; ++k) {
    fe[k] = faces[3 * k];
    fo[k] = faces[3 * k + 1];
    fb[k] = faces[3 * k + 2];
  }
  oa_mesh* mesh = nullptr;
  openaccel_b200::check(oa_mesh_create(x.data(), nn, conn.data(), ne, OA_TOPO_HEX8, fe.data(), fo.data(), fb.data(),
                                       nf, &mesh));
  oa_flow_settings s{};
  s.rho = 1.0;
  s.mu = 0.01;
  s.urf_u = 0.9;
  s.urf_p = 0.1;
  s.dt = 1.0;
  s.grad_urf = 0.5625;
  s.mdot_urf = 1.0;
  s.wall_rhs_relax = 0.75;
  s.u_shifted = s.u_grad_shifted = s.p_shifted = s.p_grad_shifted = 1;
  s.ref_node = 0;
  s.mom_maxit = 200;
  s.mom_rtol = 1e-6;
  s.pc_maxit = 5000;
  s.pc_rtol = 1e-8;
  s.precision = OA_PREC_FP64;
  s.pc_amg = 1;
  s.use_graphs = 0;
  s.hr = 0;
  s.beta_max = 1.0;
  s.du_mode = 0;
  oa_flow* flow = nullptr;
  openaccel_b200::check(oa_flow_create(mesh, &s, bnd.data(), nb, &flow));
  openaccel_b200::check(oa_flow_initialize(flow));
  openaccel_b200::check(oa_simple_iterate(flow, 1, nullptr));

  const linearSolver::CRSNodeGraph g = openaccel_b200::graph_of(mesh, nn);
  linearSolver::Context<1> ctx("pressure_correction", &g);
  accel::gpuPressureCorrectionAssembler asmb(flow);
  accel::domain dom;
  asmb.assemble(&dom, &ctx);
  asmb.adjustMatrixForPressureReference(&dom, &ctx);
  openaccel_b200::solve<1>(flow, ctx, 1e-12, 5000);
  const auto& cd = ctx.getControlData();
  EXPECT(cd.n_iterations > 0 && cd.solver_final_res[0] <= 1e-12 * cd.solver_initial_res[0] * 1.0001);
  EXPECT(ctx.getCallCount() == 1);
  write_file(dir + "/A.f64", ctx.getAMatrix().data(), ctx.getAMatrix().size());
  write_file(dir + "/b.f64", ctx.getBVector().data(), ctx.getBVector().size());
  write_file(dir + "/x.f64", ctx.getXVector().data(), ctx.getXVector().size());
  std::ofstream ctl(dir + "/control.txt");
  ctl << std::setprecision(17) << cd.n_iterations << " " << cd.solver_initial_res[0] << " " << cd.solver_final_res[0]
      << " " << cd.scaled_initial_res[0] << "\n";
  ctl.close();
  oa_flow_destroy(flow);
  oa_mesh_destroy(mesh);
  std::printf("compat gpu ok\n");
  return 0;
}

int main(int argc, char** argv) {
  const std::string mode = argc > 1 ? argv[1] : "cpu";
  try {
    if (mode == "cpu") return cpu_checks();
    if (mode == "gpu" && argc > 2) return gpu_checks(argv[2]);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 2;
  }
  std::fprintf(stderr, "usage: compat_harness cpu | gpu DIR\n");
  return 2;
}
