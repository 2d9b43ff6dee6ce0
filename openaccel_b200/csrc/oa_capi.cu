// C-ABI of the B200 CVFEM engine: mesh and flow handles, assembly entry
// points, Krylov solves and the SIMPLE outer iteration driver.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "oa_hex_orient.h"
#include "oa_internal.h"
#include "oa_krylov.h"
#include "oa_rowlane.cuh"
#include "oa_scalar_solve.h"

namespace oa {

static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};
void count_launches(long long n) { g_launches += n; }
long long launch_total() { return g_launches.load(); }
void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

// correctField_ with CLIP, relaxation 1 and no upper bound (src/equation/equation.h:204-286):
// phi += x, and a value below lo becomes phi + (lo - phi)
__global__ void k_correct_clip(int n, double* phi, const double* x, double lo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double o = phi[i];
  double v = o + 1.0 * x[i];
  if (v < lo) v = o + 1.0 * (lo - o);
  phi[i] = v;
}

__global__ void k_axpy(int n, double* y, const double* x, double a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += a * x[i];
}
template <class T>
__global__ void k_to_double(size_t n, const T* a, double* b) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = double(a[i]);
}
template <class T>
__global__ void k_from_double(size_t n, const double* a, T* b) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = T(a[i]);
}
}  // namespace oa

using namespace oa;

// What a captured outer-iteration graph baked into its kernel arguments and
// node structure; a change of any of it means a new capture.
struct IterGraphKey {
  oa_flow_settings s;
  int bs_rows, bs_elems, bs_asm;
  int time_order;
  double tk[3], dt_step;
  int pc_gcr, pc_chunk, pc_refresh, pc_cheb;
  double pc_floor, pc_damping;
  bool operator==(const IterGraphKey& o) const { return std::memcmp(this, &o, sizeof(*this)) == 0; }
};

// The whole SIMPLE outer iteration as one CUDA graph (settings.use_graphs =
// 2): assembly kernels, the momentum and pressure-correction solves with
// their convergence loops as conditional device-side nodes, the corrections,
// and copies of every scalar the host reports into one pinned block.
struct IterGraph {
  cudaGraphExec_t exec = nullptr;
  GraphBuild gb;
  IterGraphKey key;
  BodyCounters* ctr = nullptr;       // device
  BodyCounters* ctr_host = nullptr;  // pinned
  double* dsum = nullptr;            // device [8]: momentum |b|^2, |r|^2 per component, |b_pc|^2
  double* hsum = nullptr;            // pinned [8]
  KScal* mom_host = nullptr;         // pinned copy of the momentum solver's scalars
  int* herr = nullptr;               // pinned copy of the flow's error flag
  cudaEvent_t ev[6] = {};            // phase boundaries (event nodes)
  void drop() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
  }
  void release() {
    drop();
    if (ctr) cudaFree(ctr);
    if (dsum) cudaFree(dsum);
    if (ctr_host) cudaFreeHost(ctr_host);
    if (hsum) cudaFreeHost(hsum);
    if (mom_host) cudaFreeHost(mom_host);
    if (herr) cudaFreeHost(herr);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    ctr = nullptr;
    dsum = nullptr;
    ctr_host = nullptr;
    hsum = nullptr;
    mom_host = nullptr;
    herr = nullptr;
    for (auto& e : ev) e = nullptr;
  }
};

struct oa_flow {
  Flow f;
  KrylovSolver<3, double, double> mom64;
  KrylovSolver<3, float, float> mom32;
  ScalarSolve pc;           // pressure-correction solve
  double* scal = nullptr;   // [8] device scalars
  double* hscal = nullptr;  // pinned
  IterGraph ig;
  int eager_iters = 0;      // outer iterations run without the whole-iteration graph
  // k / omega solves of the fused turbulence assembly: Jacobi BiCGStab (FP32
  // inner iterations under FP64 refinement in the mixed form), FP64 rhs and
  // solution scratch
  ScalarSolve tsolve;
  double *t_b64 = nullptr, *t_x = nullptr;
};

namespace {

template <class T>
int dalloc(T** p, size_t n) {
  cudaError_t e = cudaMalloc(p, sizeof(T) * (n ? n : 1));
  if (e != cudaSuccess) return fail(OA_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  return OA_OK;
}

bool mixed(const Flow& f) { return f.s.precision == OA_PREC_MIXED; }

int check_err_flag(Flow& f, const char* what) {
  int h = 0;
  OA_CUDA(cudaMemcpyAsync(&h, f.err_dev, sizeof(int), cudaMemcpyDeviceToHost, f.stream));
  OA_CUDA(cudaStreamSynchronize(f.stream));
  if (h) {
    OA_CUDA(cudaMemsetAsync(f.err_dev, 0, sizeof(int), f.stream));
    OA_CUDA(cudaStreamSynchronize(f.stream));
    return fail(OA_ERR_GEOMETRY, std::string(what) + ": singular Jacobian (det <= 1e6*realmin)");
  }
  return OA_OK;
}

int copy_out_matrix(Flow& f, const void* dev, size_t n, double* host) {
  if (!host) return OA_OK;
  if (mixed(f)) {
    double* tmp = nullptr;
    if (int s = dalloc(&tmp, n)) return s;
    k_to_double<float><<<(unsigned)((n + 255) / 256), 256, 0, f.stream>>>(n, static_cast<const float*>(dev), tmp);
    OA_CUDA(cudaMemcpyAsync(host, tmp, sizeof(double) * n, cudaMemcpyDeviceToHost, f.stream));
    OA_CUDA(cudaStreamSynchronize(f.stream));
    cudaFree(tmp);
  } else {
    OA_CUDA(cudaMemcpyAsync(host, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, f.stream));
    OA_CUDA(cudaStreamSynchronize(f.stream));
  }
  return OA_OK;
}

double* field_ptr(Flow& f, const std::string& n, size_t* len) {
  const size_t nn = f.mesh->nn, ne = f.mesh->ne;
  if (n == "U") { *len = 3 * nn; return f.U; }
  if (n == "p") { *len = nn; return f.p; }
  if (n == "gradU") { *len = 9 * nn; return f.gradU; }
  if (n == "gradP") { *len = 3 * nn; return f.gradP; }
  if (n == "du") { *len = 3 * nn; return f.du; }
  if (n == "div") { *len = nn; return f.div; }
  if (n == "mDot") { *len = 12 * ne; return f.mDot; }
  if (n == "sideU") { *len = 3 * nn; return f.sideU; }
  if (n == "rho") { *len = nn; return f.rho; }
  if (n == "mu") { *len = nn; return f.mu; }
  if (f.betaU && n == "betaU") { *len = 3 * nn; return f.betaU; }
  if (f.minU && n == "minU") { *len = 3 * nn; return f.minU; }
  if (f.maxU && n == "maxU") { *len = 3 * nn; return f.maxU; }
  if (f.duT && n == "duTilde") { *len = 3 * nn; return f.duT; }
  if (f.Uold && n == "Uold") { *len = 3 * nn; return f.Uold; }
  if (f.Uoldold && n == "Uoldold") { *len = 3 * nn; return f.Uoldold; }
  if (f.mut && (n == "mut" || n == "F1" || n == "Pk")) {
    *len = nn;
    return n == "mut" ? f.mut : (n == "F1" ? f.F1 : f.Pk);
  }
  if (f.turb && (n == "gradK" || n == "gradOmega")) {
    *len = 3 * nn;
    return n == "gradK" ? f.gradK : f.gradW;
  }
  if (f.turb) {
    *len = nn;
    if (n == "k") return f.kf;
    if (n == "omega") return f.wf;
    if (n == "gammaK") return f.gkf;
    if (n == "gammaOmega") return f.gwf;
    if (n == "srcDiagK") return f.sdk;
    if (n == "srcRhsK") return f.srk;
    if (n == "srcDiagOmega") return f.sdw;
    if (n == "srcRhsOmega") return f.srw;
  }
  *len = 0;
  return nullptr;
}

// Per-component RMS of the momentum rhs (initial residual, x0 = 0) and of the
// solver's exit residual into the ControlData record.
template <class T>
int momentum_control(oa_flow* h, const T* b, const T* r, int iters) {
  Flow& f = h->f;
  const int nn = f.mesh->nn;
  if (int s = device_comp_sumsq3<T>(nn, b, h->scal + 2, f.red, f.stream)) return s;
  if (int s = device_comp_sumsq3<T>(nn, r, h->scal + 5, f.red, f.stream)) return s;
  OA_CUDA(cudaMemcpyAsync(h->hscal + 2, h->scal + 2, 6 * sizeof(double), cudaMemcpyDeviceToHost, f.stream));
  OA_CUDA(cudaStreamSynchronize(f.stream));
  oa_control_data& cd = f.cd_mom;
  cd = oa_control_data{};
  cd.n_iterations = iters;
  for (int k = 0; k < 3; ++k) {
    cd.solver_initial_res[k] = std::sqrt(h->hscal[2 + k] / nn);
    cd.solver_final_res[k] = std::sqrt(h->hscal[5 + k] / nn);
    cd.scaled_initial_res[k] = cd.solver_initial_res[k] / f.mom_scale;
  }
  return OA_OK;
}

// Momentum solve: BiCGStab with 3x3 block Jacobi; U += x (correctField_ with
// relaxation 1, navierStokesEquation.cpp:186-201).
int solve_momentum(oa_flow* h, double rtol, int maxit, int* iters, double* res, bool apply) {
  Flow& f = h->f;
  DeviceMesh& m = *f.mesh;
  h->mom64.use_graph = h->mom32.use_graph = f.s.use_graphs != 0;
  int it = 0;
  if (mixed(f)) {
    if (int s = h->mom32.setup(m.nn, m.row_ptr, m.cols, m.diag, f.stream)) return s;
    float* x = nullptr;
    if (int s = h->mom32.solve<float>(static_cast<const float*>(f.b.A_mom), static_cast<const float*>(f.b.b_mom), x,
                                      rtol, maxit, &it, res, 10))
      return s;
    k_to_double<float><<<(3 * m.nn + 255) / 256, 256, 0, f.stream>>>(3 * (size_t)m.nn, x, f.b.x_mom);
    count_launches(1);
    if (int s = momentum_control<float>(h, static_cast<const float*>(f.b.b_mom), h->mom32.residual(), it)) return s;
  } else {
    if (int s = h->mom64.setup(m.nn, m.row_ptr, m.cols, m.diag, f.stream)) return s;
    double* x = nullptr;
    if (int s = h->mom64.solve<double>(static_cast<const double*>(f.b.A_mom),
                                       static_cast<const double*>(f.b.b_mom), x, rtol, maxit, &it, res, 10))
      return s;
    OA_CUDA(cudaMemcpyAsync(f.b.x_mom, x, sizeof(double) * 3 * m.nn, cudaMemcpyDeviceToDevice, f.stream));
    if (int s = momentum_control<double>(h, static_cast<const double*>(f.b.b_mom), h->mom64.residual(), it)) return s;
  }
  if (iters) *iters = it;
  if (apply) k_axpy<<<(3 * m.nn + 255) / 256, 256, 0, f.stream>>>(3 * m.nn, f.U, f.b.x_mom, 1.0);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

// RMS over nodes of the pressure-correction rhs (the nodal mass imbalance).
int pc_rhs_rms(oa_flow* h, double* out) {
  Flow& f = h->f;
  if (int s = device_sumsq(f.mesh->nn, f.b.b_pc, h->scal + 2, f.red, f.stream)) return s;
  OA_CUDA(cudaMemcpyAsync(h->hscal + 2, h->scal + 2, sizeof(double), cudaMemcpyDeviceToHost, f.stream));
  OA_CUDA(cudaStreamSynchronize(f.stream));
  *out = std::sqrt(h->hscal[2] / f.mesh->nn);
  return OA_OK;
}

// Pressure-correction solve into f.b.x_pc (ScalarSolve: FP64 Krylov, or FP32
// inner iterations under FP64 iterative refinement), with its ControlData
// record. rhs_rms: RMS of the rhs when the caller has it already (< 0: formed
// here).
ScalarGraph pc_graph(const DeviceMesh& m) {
  ScalarGraph g;
  g.nn = m.nn;
  g.rp = m.row_ptr;
  g.cols = m.cols;
  g.diag = m.diag;
  g.h_rp = m.h_row_ptr.data();
  g.h_cols = m.h_cols.data();
  g.h_diag = m.h_diag.data();
  return g;
}

int solve_pcorr(oa_flow* h, double rtol, int maxit, int* iters, double* res, int* refinements, double rhs_rms = -1.0) {
  Flow& f = h->f;
  const ScalarGraph g = pc_graph(*f.mesh);
  if (rhs_rms < 0)
    if (int s = pc_rhs_rms(h, &rhs_rms)) return s;
  const int fb0 = h->pc.fallbacks;
  int it = 0;
  double r = 0.0;
  if (int s = h->pc.solve(g, mixed(f), f.s.pc_amg != 0, f.s.use_graphs != 0, f.b.A_pc, f.b.b_pc, f.b.x_pc, rtol,
                          maxit, &it, &r, refinements, f.stream, "pressure"))
    return s;
  oa_control_data& cd = f.cd_pc;
  cd = oa_control_data{};
  cd.n_iterations = it;
  cd.fallback = h->pc.fallbacks != fb0;
  cd.solver_initial_res[0] = rhs_rms;
  cd.solver_final_res[0] = r * rhs_rms;  // r = ||b - A x|| / ||b||, and x0 = 0
  cd.scaled_initial_res[0] = rhs_rms / f.mass_scale;
  if (iters) *iters = it;
  if (res) *res = r;
  return OA_OK;
}

IterGraphKey iter_graph_key(oa_flow* h) {
  IterGraphKey k;
  std::memset(&k, 0, sizeof(k));
  const Flow& f = h->f;
  k.s = f.s;
  k.bs_rows = f.bs_rows;
  k.bs_elems = f.bs_elems;
  k.bs_asm = f.bs_asm;
  k.time_order = f.time_order;
  for (int i = 0; i < 3; ++i) k.tk[i] = f.tk[i];
  k.dt_step = f.dt_step;
  k.pc_gcr = h->pc.gcr ? 1 : 0;
  k.pc_chunk = h->pc.gcr_chunk;
  k.pc_refresh = h->pc.refresh;
  k.pc_floor = h->pc.inner_floor;
  k.pc_cheb = h->pc.amg64.cheb_degree;
  k.pc_damping = h->pc.amg64.omega_p;
  return k;
}

// Capture one outer iteration (the steps of oa_simple_iterate, in its order)
// into a graph with device-side loops; the solvers were set up by an eager
// iteration before.
int build_iteration_graph(oa_flow* h) {
  Flow& f = h->f;
  DeviceMesh& m = *f.mesh;
  IterGraph& G = h->ig;
  const bool mx = mixed(f);
  if (!G.ctr) {
    if (cudaMalloc(&G.ctr, sizeof(BodyCounters)) != cudaSuccess || cudaMalloc(&G.dsum, 8 * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&G.ctr_host, sizeof(BodyCounters)) != cudaSuccess ||
        cudaMallocHost(&G.hsum, 8 * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&G.mom_host, sizeof(KScal)) != cudaSuccess || cudaMallocHost(&G.herr, sizeof(int)) != cudaSuccess)
      return fail(OA_ERR_CUDA, "iteration graph: allocation failed");
    for (auto& e : G.ev) OA_CUDA(cudaEventCreate(&e));
  }
  G.drop();
  G.gb = GraphBuild{};
  G.gb.st = f.stream;
  G.gb.ctr = G.ctr;
  GraphBuild& gb = G.gb;
  cudaGraph_t g = nullptr;
  OA_CUDA(cudaGraphCreate(&g, 0));
  struct GraphGuard {
    cudaGraph_t g;
    ~GraphGuard() {
      if (g) cudaGraphDestroy(g);
    }
  } guard{g};
  Deps d;
  auto mark = [&](int k) -> int {
    OA_CUDA(cudaEventRecordWithFlags(G.ev[k], f.stream, cudaEventRecordExternal));
    return OA_OK;
  };
  const int n3 = 3 * m.nn;
  // momentum predictor: assembly, then the solve as a device-side loop
  if (int s = gb.seg(g, d, -1, [&]() -> int {
        if (int s2 = launch_counters_reset(gb)) return s2;
        if (int s2 = mark(0)) return s2;
        if (int s2 = launch_momentum(f, mx)) return s2;
        return mark(1);
      }))
    return s;
  constexpr int MOM_CHUNK = 2;  // device-side checks are cheap: short chunks
  if (mx) {
    h->mom32.amg = nullptr;
    if (int s = h->mom32.setup(m.nn, m.row_ptr, m.cols, m.diag, f.stream)) return s;
    if (int s = h->mom32.emit<float>(gb, g, d, -1, static_cast<const float*>(f.b.A_mom),
                                     static_cast<const float*>(f.b.b_mom), f.s.mom_rtol, f.s.mom_maxit, nullptr,
                                     nullptr, f.s.mom_maxit, MOM_CHUNK, false, -1))
      return s;
  } else {
    h->mom64.amg = nullptr;
    if (int s = h->mom64.setup(m.nn, m.row_ptr, m.cols, m.diag, f.stream)) return s;
    if (int s = h->mom64.emit<double>(gb, g, d, -1, static_cast<const double*>(f.b.A_mom),
                                      static_cast<const double*>(f.b.b_mom), f.s.mom_rtol, f.s.mom_maxit, nullptr,
                                      nullptr, f.s.mom_maxit, MOM_CHUNK, false, -1))
      return s;
  }
  // U += x, the momentum ControlData sums; mass flow and pressure-correction
  // assembly with the rhs norm
  if (int s = gb.seg(g, d, -1, [&]() -> int {
        if (mx) {
          k_to_double<float><<<(n3 + 255) / 256, 256, 0, f.stream>>>((size_t)n3, h->mom32.solution(), f.b.x_mom);
          count_launches(1);
          if (int s2 = device_comp_sumsq3<float>(m.nn, static_cast<const float*>(f.b.b_mom), G.dsum, f.red, f.stream))
            return s2;
          if (int s2 = device_comp_sumsq3<float>(m.nn, h->mom32.residual(), G.dsum + 3, f.red, f.stream)) return s2;
          OA_CUDA(cudaMemcpyAsync(G.mom_host, h->mom32.scalars(), sizeof(KScal), cudaMemcpyDeviceToHost, f.stream));
        } else {
          OA_CUDA(cudaMemcpyAsync(f.b.x_mom, h->mom64.solution(), sizeof(double) * n3, cudaMemcpyDeviceToDevice,
                                  f.stream));
          if (int s2 = device_comp_sumsq3<double>(m.nn, static_cast<const double*>(f.b.b_mom), G.dsum, f.red,
                                                  f.stream))
            return s2;
          if (int s2 = device_comp_sumsq3<double>(m.nn, h->mom64.residual(), G.dsum + 3, f.red, f.stream)) return s2;
          OA_CUDA(cudaMemcpyAsync(G.mom_host, h->mom64.scalars(), sizeof(KScal), cudaMemcpyDeviceToHost, f.stream));
        }
        k_axpy<<<(n3 + 255) / 256, 256, 0, f.stream>>>(n3, f.U, f.b.x_mom, 1.0);
        count_launches(1);
        if (int s2 = mark(2)) return s2;
        if (int s2 = launch_update_mdot(f, true)) return s2;
        if (int s2 = launch_pcorr(f, mx, true)) return s2;
        if (int s2 = device_sumsq(m.nn, f.b.b_pc, G.dsum + 6, f.red, f.stream)) return s2;
        return mark(3);
      }))
    return s;
  // pressure-correction solve
  const ScalarGraph pg = pc_graph(m);
  if (int s = h->pc.emit(gb, g, d, pg, mx, f.s.pc_amg != 0, f.b.A_pc, f.b.b_pc, f.b.x_pc, f.s.pc_rtol, f.s.pc_maxit,
                         f.stream))
    return s;
  // corrections and gradients; the scalars the host reads
  if (int s = gb.seg(g, d, -1, [&]() -> int {
        if (int s2 = mark(4)) return s2;
        k_axpy<<<(m.nn + 255) / 256, 256, 0, f.stream>>>(m.nn, f.p, f.b.x_pc, f.s.urf_p);
        count_launches(1);
        if (int s2 = launch_update_mdot(f)) return s2;
        if (int s2 = launch_div(f)) return s2;
        if (int s2 = launch_axpy_du_gradp(f, +1.0)) return s2;
        if (int s2 = launch_gradient(f, 0)) return s2;
        if (int s2 = launch_axpy_du_gradp(f, -1.0)) return s2;
        if (int s2 = launch_gradient(f, 1)) return s2;
        if (f.s.hr)
          if (int s2 = launch_blend_u(f)) return s2;
        if (int s2 = mark(5)) return s2;
        OA_CUDA(cudaMemcpyAsync(G.hsum, G.dsum, 8 * sizeof(double), cudaMemcpyDeviceToHost, f.stream));
        OA_CUDA(cudaMemcpyAsync(G.herr, f.err_dev, sizeof(int), cudaMemcpyDeviceToHost, f.stream));
        OA_CUDA(cudaMemcpyAsync(G.ctr_host, G.ctr, sizeof(BodyCounters), cudaMemcpyDeviceToHost, f.stream));
        return OA_OK;
      }))
    return s;
  const cudaError_t ie = cudaGraphInstantiate(&G.exec, g, 0);
  if (ie != cudaSuccess) {
    G.exec = nullptr;
    return fail(OA_ERR_CUDA, std::string("iteration graph instantiate: ") + cudaGetErrorString(ie));
  }
  G.key = iter_graph_key(h);
  return OA_OK;
}

// One outer iteration by the graph; the same statistics and ControlData as
// the eager path, from the pinned copies the graph wrote.
int iterate_graph(oa_flow* h, oa_iter_stats* out) {
  Flow& f = h->f;
  IterGraph& G = h->ig;
  const int nn = f.mesh->nn;
  if (G.exec && !(iter_graph_key(h) == G.key)) G.drop();
  if (!G.exec)
    if (int s = build_iteration_graph(h)) {
      G.drop();
      return s;
    }
  if (int s = h->pc.graph_prepare(f.stream)) return s;
  OA_CUDA(cudaGraphLaunch(G.exec, f.stream));
  OA_CUDA(cudaStreamSynchronize(f.stream));
  count_launches(G.gb.launches(*G.ctr_host));
  if (*G.herr) {
    OA_CUDA(cudaMemsetAsync(f.err_dev, 0, sizeof(int), f.stream));
    OA_CUDA(cudaStreamSynchronize(f.stream));
    return fail(OA_ERR_GEOMETRY, "oa_simple_iterate: singular Jacobian (det <= 1e6*realmin)");
  }
  oa_iter_stats st{};
  const KScal& K = *G.mom_host;
  if (K.status == 2) return fail(OA_ERR_SOLVER, "BiCGStab: non-finite residual");
  st.mom_iters = K.iters;
  st.mom_res = K.bnorm > 0 ? K.rnorm / K.bnorm : 0.0;
  oa_control_data& cm = f.cd_mom;
  cm = oa_control_data{};
  cm.n_iterations = K.iters;
  for (int k = 0; k < 3; ++k) {
    cm.solver_initial_res[k] = std::sqrt(G.hsum[k] / nn);
    cm.solver_final_res[k] = std::sqrt(G.hsum[3 + k] / nn);
    cm.scaled_initial_res[k] = cm.solver_initial_res[k] / f.mom_scale;
  }
  st.continuity_rms_raw = std::sqrt(G.hsum[6] / nn);
  st.continuity_rms = st.continuity_rms_raw / f.mass_scale;
  bool recapture = false;
  const int fb0 = h->pc.fallbacks;
  const int ps = h->pc.graph_result(mixed(f), &st.pc_iters, &st.pc_res, &st.pc_refinements, &recapture, "pressure");
  if (recapture) G.drop();
  if (ps) return ps;
  oa_control_data& cp = f.cd_pc;
  cp = oa_control_data{};
  cp.n_iterations = st.pc_iters;
  cp.fallback = h->pc.fallbacks != fb0;
  cp.solver_initial_res[0] = st.continuity_rms_raw;
  cp.solver_final_res[0] = st.pc_res * st.continuity_rms_raw;
  cp.scaled_initial_res[0] = st.continuity_rms_raw / f.mass_scale;
  if (out) {
    float t[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    for (int k = 0; k < 5; ++k) cudaEventElapsedTime(&t[k], G.ev[k], G.ev[k + 1]);
    st.ms_momentum_assembly = t[0];
    st.ms_momentum_solve = t[1];
    st.ms_pcorr_assembly = t[2];
    st.ms_pcorr_solve = t[3];
    st.ms_corrections = t[4];
    st.mom = f.cd_mom;
    st.pc = f.cd_pc;
    *out = st;
  }
  return OA_OK;
}

}  // namespace

extern "C" {

const char* oa_last_error(void) { return g_last_error.c_str(); }
const char* oa_version(void) { return "openaccel_b200 0.1 (sm_100a)"; }

int oa_mesh_create(const double* coords, int nn, const int* conn, int ne, int topo, const int* face_elem,
                   const int* face_ord, const int* face_bnd, int nf, oa_mesh** out) {
  if (!out || !coords || !conn || nn <= 0 || ne <= 0 || nf < 0) return fail(OA_ERR_ARG, "oa_mesh_create: bad arguments");
  if (topo != OA_TOPO_HEX8 && topo != OA_TOPO_TET4) return fail(OA_ERR_MESH, "oa_mesh_create: unknown topology");
  *out = nullptr;
  if (topo == OA_TOPO_TET4) {
    oa_mesh* M = new oa_mesh();
    if (int s = create_tet4_mesh(M, coords, nn, conn, ne, face_elem, face_ord, face_bnd, nf)) {
      oa_mesh_destroy(M);
      return s;
    }
    *out = M;
    return OA_OK;
  }
  for (long k = 0; k < 8L * ne; ++k)
    if (conn[k] < 0 || conn[k] >= nn) return fail(OA_ERR_MESH, "oa_mesh_create: connectivity index out of range");
  for (int f = 0; f < nf; ++f)
    if (face_elem[f] < 0 || face_elem[f] >= ne || face_ord[f] < 0 || face_ord[f] > 5)
      return fail(OA_ERR_MESH, "oa_mesh_create: boundary face out of range");
  static const int LRt[12][2] = {{0, 1}, {1, 2}, {2, 3}, {0, 3}, {4, 5}, {5, 6},
                                 {6, 7}, {4, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  static const int FN[6][4] = {{0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {0, 4, 7, 3}, {0, 3, 2, 1}, {4, 5, 6, 7}};
  // relabel elements whose corner numbering starts elsewhere (one of the 24
  // proper cube rotations each) so the mesh is a consistently oriented block;
  // boundary-face ordinals follow their element
  std::vector<int> oconn;
  std::vector<uint8_t> rot;
  std::vector<int> oface(face_ord, face_ord + nf);
  bool consistent = true;
  bool general = false;  // not a consistently oriented block: incident-list lanes
  if (ne > (1 << 28)) return fail(OA_ERR_MESH, "oa_mesh_create: more than 2^28 elements");
  {
    std::vector<uint8_t> seen(8L * nn, 0);
    for (long k = 0; k < 8L * ne && consistent; ++k) {
      uint8_t& v = seen[8L * conn[k] + (k & 7)];
      if (v) consistent = false;
      v = 1;
    }
  }
  if (!consistent) {  // only meshes that need it pay for the face walk
    std::string why;
    bool invalid = false;
    if (hexorient::orient(nn, ne, conn, oconn, rot, &why, &invalid)) {
      for (int f = 0; f < nf; ++f) oface[f] = hexorient::face_map(rot[face_elem[f]], face_ord[f]);
      conn = oconn.data();
      face_ord = oface.data();
    } else if (invalid) {
      return fail(OA_ERR_MESH, "oa_mesh_create: invalid hex mesh (" + why + ")");
    } else {
      general = true;  // the caller's labelling, incident-list lanes
      rot.clear();
    }
  }
  oa_mesh* M = new oa_mesh();
  DeviceMesh& m = M->m;
  if (std::any_of(rot.begin(), rot.end(), [](uint8_t r) { return r != 0; })) m.h_rot.swap(rot);
  m.nn = nn;
  m.ne = ne;
  m.nf = nf;
  // node -> incident (element, corner) table, lpr entries per node:
  // entry c = the element where the node is corner c on a block mesh, the
  // incident elements in element order otherwise
  int lpr = 8;
  std::vector<int> n2e;
  if (!general) {
    n2e.assign(8L * nn, -1);
    for (int e = 0; e < ne; ++e)
      for (int a = 0; a < 8; ++a) {
        int& slot = n2e[8L * conn[8L * e + a] + a];
        if (slot != -1) {
          delete M;
          return fail(OA_ERR_MESH, "oa_mesh_create: a node is the same local corner of two elements");
        }
        slot = 8 * e + a;
      }
  } else {
    std::vector<int> inc(nn, 0);
    int most = 0;
    for (long k = 0; k < 8L * ne; ++k) most = std::max(most, ++inc[conn[k]]);
    if (most > 16) {
      delete M;
      return fail(OA_ERR_MESH, "oa_mesh_create: a node with more than 16 incident hex elements");
    }
    lpr = most <= 8 ? 8 : 16;
    n2e.assign((size_t)lpr * nn, -1);
    std::fill(inc.begin(), inc.end(), 0);
    for (int e = 0; e < ne; ++e)
      for (int a = 0; a < 8; ++a) {
        const int nd = conn[8L * e + a];
        n2e[(size_t)lpr * nd + inc[nd]++] = 8 * e + a;
      }
  }
  m.lpr = lpr;
  // reduced-stencil graph: row i = {i} U {j : (i,j) is an SCS L/R pair}
  std::vector<int> cnt(nn + 1, 0);
  for (int e = 0; e < ne; ++e)
    for (int ip = 0; ip < 12; ++ip) {
      cnt[conn[8L * e + LRt[ip][0]] + 1] += 1;
      cnt[conn[8L * e + LRt[ip][1]] + 1] += 1;
    }
  for (int i = 0; i < nn; ++i) cnt[i + 1] += cnt[i] + 0;
  std::vector<int> nbr(cnt[nn]);
  std::vector<int> pos(cnt.begin(), cnt.end() - 1);
  for (int e = 0; e < ne; ++e)
    for (int ip = 0; ip < 12; ++ip) {
      const int L = conn[8L * e + LRt[ip][0]], R = conn[8L * e + LRt[ip][1]];
      nbr[pos[L]++] = R;
      nbr[pos[R]++] = L;
    }
  m.h_row_ptr.assign(nn + 1, 0);
  m.h_diag.assign(nn, 0);
  m.h_cols.clear();
  m.h_cols.reserve((size_t)nn * 7);
  std::vector<int> tmp;
  for (int i = 0; i < nn; ++i) {
    tmp.assign(nbr.begin() + cnt[i], nbr.begin() + cnt[i + 1]);
    tmp.push_back(i);
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    for (size_t k = 0; k < tmp.size(); ++k)
      if (tmp[k] == i) m.h_diag[i] = (int)k;
    m.h_cols.insert(m.h_cols.end(), tmp.begin(), tmp.end());
    m.h_row_ptr[i + 1] = (int)m.h_cols.size();
  }
  m.nnz = m.h_row_ptr[nn];
  // slot maps of the row write-out: which corner-lane neighbour blocks sum
  // into each off-diagonal CSR entry (a row's lanes then add them in bit
  // order, the same ascending (lane, neighbour) order as a search would)
  std::vector<unsigned long long> smask(m.nnz, 0ull);
  for (int i = 0; i < nn; ++i) {
    const int* rb = m.h_cols.data() + m.h_row_ptr[i];
    const int* re = m.h_cols.data() + m.h_row_ptr[i + 1];
    for (int l = 0; l < lpr; ++l) {
      const int ec = n2e[(size_t)lpr * i + l];
      if (ec < 0) continue;
      const int e = ec >> 3, c = ec & 7;
      for (int k = 0; k < 3; ++k) {
        const int j = conn[8L * e + edge_nbr(c, k)];
        const int* q = std::lower_bound(rb, re, j);
        if (q == re || *q != j) {
          delete M;
          return fail(OA_ERR_MESH, "oa_mesh_create: an element edge is missing from the stencil graph");
        }
        smask[q - m.h_cols.data()] |= 1ull << (3 * l + k);
      }
    }
  }
  std::vector<uint32_t> smask32;
  if (lpr == 8) smask32.assign(smask.begin(), smask.end());
  {
    // mean element edge length (the 12 edges are the SCS L/R pairs)
    double sum = 0.0;
    for (int e = 0; e < ne; ++e)
      for (int ip = 0; ip < 12; ++ip) {
        const double* a = coords + 3L * conn[8L * e + LRt[ip][0]];
        const double* b = coords + 3L * conn[8L * e + LRt[ip][1]];
        sum += std::sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
      }
    m.h_mean = sum / (12.0 * ne);
  }
  m.h_conn.assign(conn, conn + 8L * ne);
  m.h_face_elem.assign(face_elem, face_elem + nf);
  m.h_face_ord.assign(face_ord, face_ord + nf);
  m.h_face_bnd.assign(face_bnd, face_bnd + nf);
  // boundary faces
  std::vector<uint8_t> fmask(ne, 0);
  std::vector<int> wall(nn, 0);
  for (int f = 0; f < nf; ++f) {
    fmask[face_elem[f]] |= (uint8_t)(1u << face_ord[f]);
    for (int k = 0; k < 4; ++k) wall[conn[8L * face_elem[f] + FN[face_ord[f]][k]]] = 1;
  }
  int st = OA_OK;
  if ((st = dalloc(&m.x, 3L * nn)) || (st = dalloc(&m.conn, 8L * ne)) || (st = dalloc(&m.n2e, (size_t)lpr * nn)) ||
      (st = dalloc(&m.row_ptr, nn + 1L)) || (st = dalloc(&m.cols, (size_t)m.nnz)) || (st = dalloc(&m.diag, (size_t)nn)) ||
      (lpr == 8 ? (st = dalloc(&m.slot_mask, (size_t)m.nnz)) : (st = dalloc(&m.slot_mask64, (size_t)m.nnz))) ||
      (st = dalloc(&m.face_mask, (size_t)ne)) || (st = dalloc(&m.vol, (size_t)nn)) || (st = dalloc(&m.wscv, 8L * ne)) ||
      (st = dalloc(&m.scs_area, 36L * ne)) ||
      (st = dalloc(&m.wall_node, (size_t)nn))) {
    oa_mesh_destroy(M);
    return st;
  }
  cudaStreamCreateWithFlags(&M->st, cudaStreamNonBlocking);
  cudaMemcpy(m.x, coords, sizeof(double) * 3 * nn, cudaMemcpyHostToDevice);
  cudaMemcpy(m.conn, conn, sizeof(int) * 8 * ne, cudaMemcpyHostToDevice);
  cudaMemcpy(m.n2e, n2e.data(), sizeof(int) * n2e.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(m.row_ptr, m.h_row_ptr.data(), sizeof(int) * (nn + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(m.cols, m.h_cols.data(), sizeof(int) * m.nnz, cudaMemcpyHostToDevice);
  cudaMemcpy(m.diag, m.h_diag.data(), sizeof(int) * nn, cudaMemcpyHostToDevice);
  if (lpr == 8) cudaMemcpy(m.slot_mask, smask32.data(), sizeof(uint32_t) * m.nnz, cudaMemcpyHostToDevice);
  else cudaMemcpy(m.slot_mask64, smask.data(), sizeof(unsigned long long) * m.nnz, cudaMemcpyHostToDevice);
  cudaMemcpy(m.face_mask, fmask.data(), ne, cudaMemcpyHostToDevice);
  cudaMemcpy(m.wall_node, wall.data(), sizeof(int) * nn, cudaMemcpyHostToDevice);
  cudaError_t ce = cudaDeviceSynchronize();
  if (ce == cudaSuccess) ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    oa_mesh_destroy(M);
    return fail(OA_ERR_CUDA, std::string("mesh upload: ") + cudaGetErrorString(ce));
  }
  if ((st = launch_geometry(m, M->st))) {
    oa_mesh_destroy(M);
    return st;
  }
  *out = M;
  return OA_OK;
}

void oa_mesh_destroy(oa_mesh* M) {
  if (!M) return;
  DeviceMesh& m = M->m;
  void* ptrs[] = {m.x,       m.conn,      m.n2e,      m.n2e_ptr,  m.n2f,       m.n2f_ptr, m.face_elem, m.face_ord,
                  m.face_bnd, m.row_ptr, m.cols,     m.diag,     m.face_mask, m.vol,     m.wscv,      m.wall_node,
                  m.scs_area, m.slot_mask, m.slot_mask64};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (M->st) cudaStreamDestroy(M->st);
  delete M;
}

int oa_mesh_nnz(const oa_mesh* M, int* nnz) {
  if (!M || !nnz) return fail(OA_ERR_ARG, "oa_mesh_nnz: null argument");
  *nnz = M->m.nnz;
  return OA_OK;
}

int oa_mesh_graph(const oa_mesh* M, int* row_ptr, int* cols) {
  if (!M || !row_ptr || !cols) return fail(OA_ERR_ARG, "oa_mesh_graph: null argument");
  std::memcpy(row_ptr, M->m.h_row_ptr.data(), sizeof(int) * (M->m.nn + 1));
  std::memcpy(cols, M->m.h_cols.data(), sizeof(int) * M->m.nnz);
  return OA_OK;
}

int oa_mesh_dual_volume(const oa_mesh* M, double* vol) {
  if (!M || !vol) return fail(OA_ERR_ARG, "oa_mesh_dual_volume: null argument");
  OA_CUDA(cudaMemcpy(vol, M->m.vol, sizeof(double) * M->m.nn, cudaMemcpyDeviceToHost));
  return OA_OK;
}

int oa_flow_create(oa_mesh* M, const oa_flow_settings* s, const double* bnd_velocity, int nbnd, oa_flow** out) {
  if (!M || !s || !out || nbnd < 0 || (nbnd > 0 && !bnd_velocity)) return fail(OA_ERR_ARG, "oa_flow_create: bad arguments");
  if (s->urf_u <= 0 || s->urf_p <= 0 || s->dt <= 0) return fail(OA_ERR_ARG, "oa_flow_create: relaxation/timescale must be > 0");
  if (s->precision != OA_PREC_FP64 && s->precision != OA_PREC_MIXED) return fail(OA_ERR_ARG, "oa_flow_create: unknown precision");
  if (s->use_graphs < 0 || s->use_graphs > 2) return fail(OA_ERR_ARG, "oa_flow_create: use_graphs must be 0, 1 or 2");
  if (s->hr != 0 && s->hr != 1) return fail(OA_ERR_ARG, "oa_flow_create: advection scheme must be 0 (upwind) or 1 (high resolution)");
  if (s->hr && !(s->beta_max > 0)) return fail(OA_ERR_ARG, "oa_flow_create: beta_max must be > 0 for high resolution");
  if (s->du_mode < 0 || s->du_mode > 2)
    return fail(OA_ERR_ARG, "oa_flow_create: du_mode must be 0 (SIMPLE), 1 (SIMPLEC) or 2 (fractional step)");
  if (s->ref_node >= M->m.nn) return fail(OA_ERR_ARG, "oa_flow_create: ref_node out of range");
  if (M->m.topo != OA_TOPO_HEX8) return fail(OA_ERR_MESH, "oa_flow_create: the flow path needs a hex8 mesh");
  *out = nullptr;
  oa_flow* H = new oa_flow();
  Flow& f = H->f;
  f.mesh = &M->m;
  f.s = *s;
  f.h_bnd_velocity.assign(bnd_velocity, bnd_velocity + 3L * nbnd);
  f.h_bnd_type.assign(nbnd, OA_BTYPE_WALL);
  {
    double u = 0.0;
    for (int k = 0; k < nbnd; ++k) {
      const double* v = bnd_velocity + 3L * k;
      u = std::max(u, std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
    }
    f.u_ref = u > 0.0 ? u : 1.0;
    const double h2 = M->m.h_mean * M->m.h_mean;
    f.mass_scale = s->rho * f.u_ref * h2;
    f.mom_scale = s->rho * f.u_ref * f.u_ref * h2;
    f.cd_mom.n_iterations = f.cd_pc.n_iterations = -1;  // no solve yet
  }
  const size_t nn = M->m.nn, ne = M->m.ne, nnz = M->m.nnz;
  const size_t tm = s->precision == OA_PREC_MIXED ? sizeof(float) : sizeof(double);
  int st = OA_OK;
  if ((st = dalloc(&f.U, 3 * nn)) || (st = dalloc(&f.p, nn)) || (st = dalloc(&f.gradU, 9 * nn)) ||
      (st = dalloc(&f.gradP, 3 * nn)) || (st = dalloc(&f.du, 3 * nn)) || (st = dalloc(&f.div, nn)) ||
      (st = dalloc(&f.mDot, 12 * ne)) || (st = dalloc(&f.pc_flux, 12 * ne)) || (st = dalloc(&f.rho, nn)) ||
      (st = dalloc(&f.mu, nn)) ||
      (st = dalloc(&f.sideU, 3 * nn)) || (st = dalloc(&f.b.b_pc, nn)) || (st = dalloc(&f.b.x_mom, 3 * nn)) ||
      (st = dalloc(&f.b.x_pc, nn)) || (st = dalloc(&f.err_dev, 1)) || (st = dalloc(&H->scal, 8)) ||
      (st = dalloc(&f.red, (size_t)partials_size())) || (st = dalloc(&f.ref_flag, nn)) ||
      (s->hr && ((st = dalloc(&f.betaU, 3 * nn)) || (st = dalloc(&f.minU, 3 * nn)) ||
                 (st = dalloc(&f.maxU, 3 * nn)))) ||
      (s->du_mode == 1 && (st = dalloc(&f.duT, 3 * nn)))) {
    oa_flow_destroy(H);
    return st;
  }
  if (cudaMalloc(&f.b.A_mom, tm * 9 * nnz) != cudaSuccess || cudaMalloc(&f.b.b_mom, tm * 3 * nn) != cudaSuccess ||
      cudaMalloc(&f.b.A_pc, tm * nnz) != cudaSuccess || cudaMalloc(&f.pc_coef, tm * 24 * ne) != cudaSuccess ||
      cudaMallocHost(&H->hscal, 8 * sizeof(double)) != cudaSuccess ||
      (s->precision == OA_PREC_MIXED && (cudaMalloc(&f.xloc32, sizeof(float4) * 8 * ne) != cudaSuccess ||
                                         cudaMalloc(&f.umu32, sizeof(float4) * nn) != cudaSuccess))) {
    oa_flow_destroy(H);
    return fail(OA_ERR_CUDA, "oa_flow_create: device allocation failed");
  }
  cudaStreamCreateWithFlags(&f.stream, cudaStreamNonBlocking);
  if (f.xloc32) {
    st = launch_xloc(f);
    if (!st && cudaStreamSynchronize(f.stream) != cudaSuccess)
      st = fail(OA_ERR_CUDA, "oa_flow_create: corner offsets failed");
    if (st) {
      oa_flow_destroy(H);
      return st;
    }
  }
  // constant properties, zero fields
  std::vector<double> h(nn, s->rho);
  cudaMemcpy(f.rho, h.data(), sizeof(double) * nn, cudaMemcpyHostToDevice);
  std::fill(h.begin(), h.end(), s->mu);
  cudaMemcpy(f.mu, h.data(), sizeof(double) * nn, cudaMemcpyHostToDevice);
  cudaMemset(f.U, 0, sizeof(double) * 3 * nn);
  cudaMemset(f.p, 0, sizeof(double) * nn);
  cudaMemset(f.gradU, 0, sizeof(double) * 9 * nn);
  cudaMemset(f.gradP, 0, sizeof(double) * 3 * nn);
  cudaMemset(f.du, 0, sizeof(double) * 3 * nn);
  cudaMemset(f.div, 0, sizeof(double) * nn);
  cudaMemset(f.mDot, 0, sizeof(double) * 12 * ne);
  cudaMemset(f.err_dev, 0, sizeof(int));
  if (f.duT) cudaMemset(f.duT, 0, sizeof(double) * 3 * nn);
  if (f.betaU) {
    // setupBlendingFactorField starts the blending factor at zero
    // (src/field/nodeField/nodeField.hpp:733-745)
    cudaMemset(f.betaU, 0, sizeof(double) * 3 * nn);
    cudaMemset(f.minU, 0, sizeof(double) * 3 * nn);
    cudaMemset(f.maxU, 0, sizeof(double) * 3 * nn);
  }
  cudaMemset(f.ref_flag, 0, nn);
  if (s->ref_node >= 0) {
    const uint8_t one = 1;
    cudaMemcpy(f.ref_flag + s->ref_node, &one, 1, cudaMemcpyHostToDevice);
  }
  // node-side wall velocity, boundary by boundary in index order
  // (nodeField::updateBoundarySideFieldSpecifiedValue sets parts in turn)
  std::vector<double> side(3 * nn, 0.0);
  {
    static const int FN[6][4] = {{0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {0, 4, 7, 3}, {0, 3, 2, 1}, {4, 5, 6, 7}};
    const DeviceMesh& m = M->m;
    for (int bnd = 0; bnd < nbnd; ++bnd)
      for (int fc = 0; fc < m.nf; ++fc) {
        if (m.h_face_bnd[fc] != bnd) continue;
        for (int k = 0; k < 4; ++k) {
          const int nd = m.h_conn[8L * m.h_face_elem[fc] + FN[m.h_face_ord[fc]][k]];
          for (int d = 0; d < 3; ++d) side[3L * nd + d] = bnd_velocity[3 * bnd + d];
        }
      }
  }
  cudaMemcpy(f.sideU, side.data(), sizeof(double) * 3 * nn, cudaMemcpyHostToDevice);
  cudaError_t ce = cudaDeviceSynchronize();
  if (ce == cudaSuccess) ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    oa_flow_destroy(H);
    return fail(OA_ERR_CUDA, std::string("oa_flow_create: ") + cudaGetErrorString(ce));
  }
  *out = H;
  return OA_OK;
}

void oa_flow_destroy(oa_flow* H) {
  if (!H) return;
  Flow& f = H->f;
  void* ptrs[] = {f.U,       f.p,       f.gradU,   f.gradP,   f.du,      f.div,    f.mDot,  f.pc_flux,
                  f.pc_coef, f.xloc32,  f.umu32,   f.rho,     f.mu,      f.sideU,  f.b.A_mom, f.b.b_mom,
                  f.b.A_pc,  f.b.b_pc,  f.b.x_mom, f.b.x_pc,  f.err_dev, H->scal,  f.red,   f.ref_flag,
                  f.betaU,   f.minU,    f.maxU,    f.duT,     f.Uold,    f.Uoldold, f.kf,      f.wf,
                  f.gkf,     f.gwf,     f.sdk,     f.srk,     f.sdw,     f.srw,     f.A_k,     f.b_k,
                  f.A_w,     f.b_w,     f.sym_mask, f.sym_nodes, f.sym_area, f.wall_face_node,
                  f.gradK,   f.gradW,   f.mut,     f.F1,      f.Pk,      f.k_prev};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (H->hscal) cudaFreeHost(H->hscal);
  H->ig.release();
  H->tsolve.release();
  if (H->t_b64) cudaFree(H->t_b64);
  if (H->t_x) cudaFree(H->t_x);
  H->pc.release();
  H->mom64.release();
  H->mom32.release();
  if (f.stream) cudaStreamDestroy(f.stream);
  delete H;
}

// Mass flows of relabelled elements: the device keeps them in the element's
// new ip order; the caller sees its own (ip q of the new labelling is old ip
// o, with the sign of the L -> R direction).
static void mdot_to_device_order(const DeviceMesh& m, const double* in, double* out) {
  for (int e = 0; e < m.ne; ++e)
    for (int q = 0; q < 12; ++q) {
      int o = q, sg = 1;
      if (m.h_rot[e]) hexorient::ip_map(m.h_rot[e], q, &o, &sg);
      out[12L * e + q] = sg * in[12L * e + o];
    }
}
static void mdot_to_caller_order(const DeviceMesh& m, const double* in, double* out) {
  for (int e = 0; e < m.ne; ++e)
    for (int q = 0; q < 12; ++q) {
      int o = q, sg = 1;
      if (m.h_rot[e]) hexorient::ip_map(m.h_rot[e], q, &o, &sg);
      out[12L * e + o] = sg * in[12L * e + q];
    }
}

int oa_flow_set_field(oa_flow* H, const char* name, const double* host, long n) {
  if (!H || !name || !host) return fail(OA_ERR_ARG, "oa_flow_set_field: null argument");
  size_t len = 0;
  double* d = field_ptr(H->f, name, &len);
  if (!d) return fail(OA_ERR_ARG, std::string("oa_flow_set_field: unknown field ") + name);
  if ((size_t)n != len) return fail(OA_ERR_ARG, std::string("oa_flow_set_field: size mismatch for ") + name);
  std::vector<double> tmp;
  if (!H->f.mesh->h_rot.empty() && std::string(name) == "mDot") {
    tmp.resize(len);
    mdot_to_device_order(*H->f.mesh, host, tmp.data());
    host = tmp.data();
  }
  OA_CUDA(cudaMemcpyAsync(d, host, sizeof(double) * len, cudaMemcpyHostToDevice, H->f.stream));
  OA_CUDA(cudaStreamSynchronize(H->f.stream));
  return OA_OK;
}

int oa_flow_get_field(oa_flow* H, const char* name, double* host, long n) {
  if (!H || !name || !host) return fail(OA_ERR_ARG, "oa_flow_get_field: null argument");
  size_t len = 0;
  double* d = field_ptr(H->f, name, &len);
  if (!d) return fail(OA_ERR_ARG, std::string("oa_flow_get_field: unknown field ") + name);
  if ((size_t)n != len) return fail(OA_ERR_ARG, std::string("oa_flow_get_field: size mismatch for ") + name);
  OA_CUDA(cudaMemcpyAsync(host, d, sizeof(double) * len, cudaMemcpyDeviceToHost, H->f.stream));
  OA_CUDA(cudaStreamSynchronize(H->f.stream));
  if (!H->f.mesh->h_rot.empty() && std::string(name) == "mDot") {
    std::vector<double> tmp(host, host + len);
    mdot_to_caller_order(*H->f.mesh, tmp.data(), host);
  }
  return OA_OK;
}

int oa_flow_field_device_ptr(oa_flow* H, const char* name, double** dev) {
  if (!H || !name || !dev) return fail(OA_ERR_ARG, "oa_flow_field_device_ptr: null argument");
  size_t len = 0;
  *dev = field_ptr(H->f, name, &len);
  if (!*dev) return fail(OA_ERR_ARG, std::string("oa_flow_field_device_ptr: unknown field ") + name);
  return OA_OK;
}

int oa_flow_set_reference_nodes(oa_flow* H, const int* nodes, int count) {
  if (!H || count < 0 || (count > 0 && !nodes)) return fail(OA_ERR_ARG, "oa_flow_set_reference_nodes: bad arguments");
  Flow& f = H->f;
  std::vector<uint8_t> flag(f.mesh->nn, 0);
  for (int k = 0; k < count; ++k) {
    if (nodes[k] < 0 || nodes[k] >= f.mesh->nn) return fail(OA_ERR_ARG, "oa_flow_set_reference_nodes: node out of range");
    flag[nodes[k]] = 1;
  }
  OA_CUDA(cudaMemcpyAsync(f.ref_flag, flag.data(), f.mesh->nn, cudaMemcpyHostToDevice, f.stream));
  OA_CUDA(cudaStreamSynchronize(f.stream));
  // closed domains of a batched (disjoint-union) mesh: the connected
  // components of the stencil graph, numbered by their first node; the
  // pressure-correction solve then converges when each of them does
  const DeviceMesh& m = *f.mesh;
  std::vector<int> comp(m.nn, -1), order;
  order.reserve(m.nn);
  std::vector<int> ptr(1, 0);
  for (int r0 = 0; r0 < m.nn; ++r0) {
    if (comp[r0] >= 0) continue;
    const int c = (int)ptr.size() - 1;
    const size_t first = order.size();
    comp[r0] = c;
    order.push_back(r0);
    for (size_t q = first; q < order.size(); ++q) {
      const int i = order[q];
      for (int k = m.h_row_ptr[i]; k < m.h_row_ptr[i + 1]; ++k) {
        const int j = m.h_cols[k];
        if (comp[j] < 0) {
          comp[j] = c;
          order.push_back(j);
        }
      }
    }
    std::sort(order.begin() + first, order.end());
    ptr.push_back((int)order.size());
  }
  if (int s = H->pc.set_segments(ptr, order)) return s;
  H->ig.drop();  // the captured solve loops carry the segment tests
  return OA_OK;
}

int oa_flow_set_boundary_types(oa_flow* H, const int* types, int nbnd, int correct_gradients) {
  if (!H || nbnd < 0 || (nbnd > 0 && !types)) return fail(OA_ERR_ARG, "oa_flow_set_boundary_types: bad arguments");
  Flow& f = H->f;
  if (nbnd != (int)f.h_bnd_type.size())
    return fail(OA_ERR_ARG, "oa_flow_set_boundary_types: one type per boundary index of oa_flow_create");
  for (int k = 0; k < nbnd; ++k)
    if (types[k] != OA_BTYPE_WALL && types[k] != OA_BTYPE_SYMMETRY)
      return fail(OA_ERR_ARG, "oa_flow_set_boundary_types: a type is neither OA_BTYPE_WALL nor OA_BTYPE_SYMMETRY");
  const DeviceMesh& m = *f.mesh;
  static const int FN[6][4] = {{0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {0, 4, 7, 3}, {0, 3, 2, 1}, {4, 5, 6, 7}};
  // element masks of the symmetry faces, the symmetry nodes, the wall-face
  // nodes; the node side velocity again from the wall boundaries alone, in
  // index order (nodeField::updateBoundarySideField leaves symmetry parts
  // untouched, nodeField.hpp:1128)
  std::vector<uint8_t> smask(m.ne, 0);
  std::vector<int> wallf(m.nn, 0), sym_nodes;
  std::vector<char> sym(m.nn, 0);
  std::vector<double> side(3L * m.nn, 0.0);
  for (int fc = 0; fc < m.nf; ++fc) {
    const bool sf = types[m.h_face_bnd[fc]] == OA_BTYPE_SYMMETRY;
    if (sf) smask[m.h_face_elem[fc]] |= (uint8_t)(1u << m.h_face_ord[fc]);
    for (int k = 0; k < 4; ++k) {
      const int nd = m.h_conn[8L * m.h_face_elem[fc] + FN[m.h_face_ord[fc]][k]];
      if (sf) sym[nd] = 1;
      else wallf[nd] = 1;
    }
  }
  for (int bnd = 0; bnd < nbnd; ++bnd) {
    if (types[bnd] == OA_BTYPE_SYMMETRY) continue;
    for (int fc = 0; fc < m.nf; ++fc) {
      if (m.h_face_bnd[fc] != bnd) continue;
      for (int k = 0; k < 4; ++k) {
        const int nd = m.h_conn[8L * m.h_face_elem[fc] + FN[m.h_face_ord[fc]][k]];
        for (int d = 0; d < 3; ++d) side[3L * nd + d] = f.h_bnd_velocity[3L * bnd + d];
      }
    }
  }
  for (int i = 0; i < m.nn; ++i)
    if (sym[i]) sym_nodes.push_back(i);
  // drop the old symmetry state (and the captured iteration, which holds its
  // launches), then upload the new one
  OA_CUDA(cudaStreamSynchronize(f.stream));
  H->ig.drop();
  for (void** p : {(void**)&f.sym_mask, (void**)&f.sym_nodes, (void**)&f.sym_area, (void**)&f.wall_face_node}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  f.nsym = 0;
  f.h_bnd_type.assign(types, types + nbnd);
  f.correct_grad = correct_gradients != 0;
  OA_CUDA(cudaMemcpyAsync(f.sideU, side.data(), sizeof(double) * side.size(), cudaMemcpyHostToDevice, f.stream));
  if (!sym_nodes.empty()) {
    const int ns = (int)sym_nodes.size();
    double* area_nn = nullptr;
    int st = OA_OK;
    if ((st = dalloc(&f.sym_mask, (size_t)m.ne)) || (st = dalloc(&f.sym_nodes, (size_t)ns)) ||
        (st = dalloc(&f.sym_area, 3L * ns)) || (st = dalloc(&f.wall_face_node, (size_t)m.nn)) ||
        (st = dalloc(&area_nn, 3L * m.nn))) {
      if (area_nn) cudaFree(area_nn);
      return st;
    }
    OA_CUDA(cudaMemcpyAsync(f.sym_mask, smask.data(), m.ne, cudaMemcpyHostToDevice, f.stream));
    OA_CUDA(cudaMemcpyAsync(f.sym_nodes, sym_nodes.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, f.stream));
    OA_CUDA(cudaMemcpyAsync(f.wall_face_node, wallf.data(), sizeof(int) * m.nn, cudaMemcpyHostToDevice, f.stream));
    if ((st = launch_sym_area(f, area_nn))) {
      cudaFree(area_nn);
      return st;
    }
    std::vector<double> all(3L * m.nn), cmp(3L * ns);
    OA_CUDA(cudaMemcpyAsync(all.data(), area_nn, sizeof(double) * all.size(), cudaMemcpyDeviceToHost, f.stream));
    OA_CUDA(cudaStreamSynchronize(f.stream));
    cudaFree(area_nn);
    for (int k = 0; k < ns; ++k)
      for (int d = 0; d < 3; ++d) cmp[3L * k + d] = all[3L * sym_nodes[k] + d];
    OA_CUDA(cudaMemcpyAsync(f.sym_area, cmp.data(), sizeof(double) * cmp.size(), cudaMemcpyHostToDevice, f.stream));
    f.nsym = ns;
  }
  OA_CUDA(cudaStreamSynchronize(f.stream));
  return OA_OK;
}

int oa_flow_initialize(oa_flow* H) {
  if (!H) return fail(OA_ERR_ARG, "oa_flow_initialize: null handle");
  Flow& f = H->f;
  int s;
  // navierStokesEquation::initialize: velocity gradient, then (high
  // resolution) the blending factor
  if ((s = launch_gradient(f, 1)) || (f.s.hr && (s = launch_blend_u(f))) || (s = launch_init_mdot(f)) ||
      (s = launch_div(f)) || (s = launch_gradient(f, 0)))
    return s;
  return check_err_flag(f, "oa_flow_initialize");
}

int oa_assemble_momentum(oa_flow* H, double* A, double* b) {
  if (!H) return fail(OA_ERR_ARG, "oa_assemble_momentum: null handle");
  Flow& f = H->f;
  if (int s = launch_momentum(f, mixed(f))) return s;
  if (int s = check_err_flag(f, "oa_assemble_momentum")) return s;
  if (int s = copy_out_matrix(f, f.b.A_mom, 9 * (size_t)f.mesh->nnz, A)) return s;
  return copy_out_matrix(f, f.b.b_mom, 3 * (size_t)f.mesh->nn, b);
}

int oa_assemble_pcorr(oa_flow* H, double* A, double* b) {
  if (!H) return fail(OA_ERR_ARG, "oa_assemble_pcorr: null handle");
  Flow& f = H->f;
  if (int s = launch_pcorr(f, mixed(f))) return s;
  if (int s = check_err_flag(f, "oa_assemble_pcorr")) return s;
  if (int s = copy_out_matrix(f, f.b.A_pc, (size_t)f.mesh->nnz, A)) return s;
  if (b) {
    OA_CUDA(cudaMemcpyAsync(b, f.b.b_pc, sizeof(double) * f.mesh->nn, cudaMemcpyDeviceToHost, f.stream));
    OA_CUDA(cudaStreamSynchronize(f.stream));
  }
  return OA_OK;
}

int oa_update_mdot(oa_flow* H) {
  if (!H) return fail(OA_ERR_ARG, "oa_update_mdot: null handle");
  if (int s = launch_update_mdot(H->f)) return s;
  return check_err_flag(H->f, "oa_update_mdot");
}

int oa_update_div(oa_flow* H) {
  if (!H) return fail(OA_ERR_ARG, "oa_update_div: null handle");
  return launch_div(H->f);
}

int oa_update_gradient(oa_flow* H, int which) {
  if (!H || which < 0 || which > 3) return fail(OA_ERR_ARG, "oa_update_gradient: bad arguments");
  if (which >= 2 && !H->f.turb)
    return fail(OA_ERR_NOT_READY, "oa_update_gradient: k / omega gradients need oa_flow_enable_turbulence");
  return launch_gradient(H->f, which);
}

int oa_solve(oa_flow* H, int sys, double rtol, int maxit, double* x, int* iters, double* res) {
  if (!H || (sys != 0 && sys != 1) || maxit <= 0) return fail(OA_ERR_ARG, "oa_solve: bad arguments");
  Flow& f = H->f;
  int s;
  if (sys == 0) {
    if ((s = solve_momentum(H, rtol, maxit, iters, res, false))) return s;
    if (x) {
      OA_CUDA(cudaMemcpyAsync(x, f.b.x_mom, sizeof(double) * 3 * f.mesh->nn, cudaMemcpyDeviceToHost, f.stream));
    }
  } else {
    if ((s = solve_pcorr(H, rtol, maxit, iters, res, nullptr))) return s;
    if (x) {
      OA_CUDA(cudaMemcpyAsync(x, f.b.x_pc, sizeof(double) * f.mesh->nn, cudaMemcpyDeviceToHost, f.stream));
    }
  }
  OA_CUDA(cudaStreamSynchronize(f.stream));
  return OA_OK;
}

// segregatedFlowEquations::solve (segregatedFlowEquations.cpp:76-297): momentum
// predictor, one pressure-correction sub-iteration, mass-flow and velocity
// corrections, gradient updates.
int oa_simple_iterate(oa_flow* H, int n, oa_iter_stats* stats) {
  if (!H || n < 0) return fail(OA_ERR_ARG, "oa_simple_iterate: bad arguments");
  Flow& f = H->f;
  const bool mx = mixed(f);
  // Phase boundaries (device time, recorded only when stats are asked for):
  // momentum assembly | momentum solve | mass flow + pressure-correction
  // assembly | pressure-correction solve | corrections and gradients. NVTX
  // ranges name the same phases for profilers.
  cudaEvent_t ev[6] = {};
  if (stats)
    for (auto& e : ev) OA_CUDA(cudaEventCreate(&e));
  auto mark = [&](int k) {
    if (stats) cudaEventRecord(ev[k], f.stream);
  };
  int s = OA_OK;
  for (int it = 0; it < n && s == OA_OK; ++it) {
    if (f.s.use_graphs == 2 && H->eager_iters > 0) {
      // the whole outer iteration as one graph (the first iteration ran eagerly
      // and set up the solvers and the AMG hierarchy)
      nvtxRangePushA("oa_simple_iterate (graph)");
      s = iterate_graph(H, stats ? stats + it : nullptr);
      nvtxRangePop();
      continue;
    }
    oa_iter_stats st{};
    nvtxRangePushA("oa_simple_iterate");
    // momentum predictor (navierStokesEquation::solve)
    mark(0);
    nvtxRangePushA("momentum assembly");
    s = launch_momentum(f, mx);
    nvtxRangePop();
    mark(1);
    nvtxRangePushA("momentum solve");
    if (!s) s = solve_momentum(H, f.s.mom_rtol, f.s.mom_maxit, &st.mom_iters, &st.mom_res, true);
    nvtxRangePop();
    mark(2);
    // pressure correction (pressureCorrectionEquation::solve)
    nvtxRangePushA("mass flow and pressure-correction assembly");
    if (!s) s = launch_update_mdot(f, true);
    if (!s) s = launch_pcorr(f, mx, true);
    if (!s) s = pc_rhs_rms(H, &st.continuity_rms_raw);
    st.continuity_rms = st.continuity_rms_raw / f.mass_scale;
    nvtxRangePop();
    mark(3);
    nvtxRangePushA("pressure-correction solve");
    if (!s)
      s = solve_pcorr(H, f.s.pc_rtol, f.s.pc_maxit, &st.pc_iters, &st.pc_res, &st.pc_refinements,
                      st.continuity_rms_raw);
    nvtxRangePop();
    mark(4);
    // corrections
    nvtxRangePushA("corrections and gradients");
    if (!s) {
      k_axpy<<<(f.mesh->nn + 255) / 256, 256, 0, f.stream>>>(f.mesh->nn, f.p, f.b.x_pc, f.s.urf_p);
      count_launches(1);
      if (!(s = launch_update_mdot(f)) && !(s = launch_div(f)) && !(s = launch_axpy_du_gradp(f, +1.0)) &&
          !(s = launch_gradient(f, 0)) && !(s = launch_axpy_du_gradp(f, -1.0)) && !(s = launch_gradient(f, 1)) &&
          f.s.hr)
        s = launch_blend_u(f);  // segregatedFlowEquations.cpp:287-288
    }
    nvtxRangePop();
    mark(5);
    nvtxRangePop();
    if (!s) s = check_err_flag(f, "oa_simple_iterate");  // synchronises the stream
    if (!s) ++H->eager_iters;
    if (!s && stats) {
      float t[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
      for (int k = 0; k < 5; ++k) cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]);
      st.ms_momentum_assembly = t[0];
      st.ms_momentum_solve = t[1];
      st.ms_pcorr_assembly = t[2];
      st.ms_pcorr_solve = t[3];
      st.ms_corrections = t[4];
      st.mom = f.cd_mom;
      st.pc = f.cd_pc;
      stats[it] = st;
    }
  }
  if (stats)
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  return s;
}

int oa_flow_enable_turbulence(oa_flow* H, double urf_k, double urf_omega) {
  if (!H || !(urf_k > 0 && urf_k <= 1) || !(urf_omega > 0 && urf_omega <= 1))
    return fail(OA_ERR_ARG, "oa_flow_enable_turbulence: relaxation factors must be in (0, 1]");
  Flow& f = H->f;
  if (f.s.hr || f.s.du_mode || f.time_scheme)
    return fail(OA_ERR_ARG, "oa_flow_enable_turbulence: the fused transport variant is steady upwind SIMPLE only");
  f.urf_k = urf_k;
  f.urf_w = urf_omega;
  if (f.turb) return OA_OK;
  const size_t nn = f.mesh->nn, nnz = f.mesh->nnz;
  const size_t ws = mixed(f) ? sizeof(float) : sizeof(double);
  double** fields[] = {&f.kf, &f.wf, &f.gkf, &f.gwf, &f.sdk, &f.srk, &f.sdw, &f.srw};
  // a retry after a failed allocation keeps what the first attempt got
  for (double** p : fields) {
    if (*p) continue;
    if (int s = dalloc(p, nn)) return s;
    OA_CUDA(cudaMemset(*p, 0, sizeof(double) * nn));
  }
  for (double** p : {&f.gradK, &f.gradW}) {
    if (*p) continue;
    if (int s = dalloc(p, 3 * nn)) return s;
    OA_CUDA(cudaMemset(*p, 0, sizeof(double) * 3 * nn));
  }
  void** sys[] = {&f.A_k, &f.A_w};
  for (void** p : sys)
    if (!*p) OA_CUDA(cudaMalloc(p, ws * (nnz ? nnz : 1)));
  void** rhs[] = {&f.b_k, &f.b_w};
  for (void** p : rhs)
    if (!*p) OA_CUDA(cudaMalloc(p, ws * (nn ? nn : 1)));
  f.turb = true;
  H->ig.drop();
  return OA_OK;
}

int oa_flow_turbulence_systems(oa_flow* H, double* A_k, double* b_k, double* A_omega, double* b_omega) {
  if (!H) return fail(OA_ERR_ARG, "oa_flow_turbulence_systems: null handle");
  Flow& f = H->f;
  if (!f.turb) return fail(OA_ERR_NOT_READY, "oa_flow_turbulence_systems: turbulence transport not enabled");
  const size_t nn = f.mesh->nn, nnz = f.mesh->nnz;
  if (int s = copy_out_matrix(f, f.A_k, nnz, A_k)) return s;
  if (int s = copy_out_matrix(f, f.b_k, nn, b_k)) return s;
  if (int s = copy_out_matrix(f, f.A_w, nnz, A_omega)) return s;
  return copy_out_matrix(f, f.b_w, nn, b_omega);
}

int oa_flow_solve_turbulence(oa_flow* H, double rtol, int maxit, int* iters_k, int* iters_omega) {
  if (!H || !(rtol > 0) || maxit <= 0) return fail(OA_ERR_ARG, "oa_flow_solve_turbulence: bad arguments");
  Flow& f = H->f;
  if (!f.turb) return fail(OA_ERR_NOT_READY, "oa_flow_solve_turbulence: turbulence transport not enabled");
  const int nn = f.mesh->nn;
  if (!H->t_b64) {
    if (int s = dalloc(&H->t_b64, (size_t)nn)) return s;
    if (int s = dalloc(&H->t_x, (size_t)nn)) return s;
  }
  const ScalarGraph g = pc_graph(*f.mesh);
  // the k and omega systems are strongly diagonal (their node sources): FP32
  // Jacobi BiCGStab reaches 1e-6 per refinement pass, and asking for it saves
  // restarts (256 x 96 x 96 channel, rtol 1e-6: 4.5 against 6.8 ms for both
  // solves with the pressure solve's Jacobi default of 2e-4); OA_IR_INNER
  // overrides
  if (!std::getenv("OA_IR_INNER")) H->tsolve.inner_floor = 1e-6;
  constexpr double CLIP_LO = 2.220446049250313e-16;  // accel::SMALL, the reference's lower clip value
  for (int t = 0; t < 2; ++t) {
    const void* bt = t ? f.b_w : f.b_k;
    if (mixed(f)) {
      k_to_double<float><<<(nn + 255) / 256, 256, 0, f.stream>>>((size_t)nn, static_cast<const float*>(bt), H->t_b64);
      count_launches(1);
    } else {
      OA_CUDA(cudaMemcpyAsync(H->t_b64, bt, sizeof(double) * nn, cudaMemcpyDeviceToDevice, f.stream));
    }
    int it = 0;
    double res = 0.0;
    if (int s = H->tsolve.solve(g, mixed(f), false, f.s.use_graphs != 0, t ? f.A_w : f.A_k, H->t_b64, H->t_x, rtol,
                                maxit, &it, &res, nullptr, f.stream, t ? "omega" : "k"))
      return s;
    k_correct_clip<<<(nn + 255) / 256, 256, 0, f.stream>>>(nn, t ? f.wf : f.kf, H->t_x, CLIP_LO);
    count_launches(1);
    if (t == 0 && iters_k) *iters_k = it;
    if (t == 1 && iters_omega) *iters_omega = it;
  }
  OA_CUDA(cudaGetLastError());
  OA_CUDA(cudaStreamSynchronize(f.stream));
  return OA_OK;
}

int oa_flow_sst_iterate(oa_flow* H, int n, const oa_sst_constants* c, const double* ymin, const int* wall_node,
                        const double* mu_lam, double mut_urf, double rtol, int maxit, oa_iter_stats* stats) {
  if (!H || n < 0 || !c || !ymin || !wall_node || !mu_lam || !(mut_urf > 0 && mut_urf <= 1) || !(rtol > 0) ||
      maxit <= 0)
    return fail(OA_ERR_ARG, "oa_flow_sst_iterate: bad arguments");
  Flow& f = H->f;
  if (!f.turb) return fail(OA_ERR_NOT_READY, "oa_flow_sst_iterate: turbulence transport not enabled");
  const size_t nn = f.mesh->nn;
  for (double** p : {&f.mut, &f.F1, &f.Pk, &f.k_prev}) {
    if (*p) continue;
    if (int s = dalloc(p, nn)) return s;
    OA_CUDA(cudaMemsetAsync(*p, 0, sizeof(double) * nn, f.stream));
  }
  for (int it = 0; it < n; ++it) {
    // the previous-iteration k of the omega node terms (k.prevIter)
    OA_CUDA(cudaMemcpyAsync(f.k_prev, f.kf, sizeof(double) * nn, cudaMemcpyDeviceToDevice, f.stream));
    // flow: u/v/w/k/omega assembled in one launch, momentum and pressure
    // correction solved and corrected
    if (int s = oa_simple_iterate(H, 1, stats ? stats + it : nullptr)) return s;
    // k and omega solved and corrected, then their gradients
    if (int s = oa_flow_solve_turbulence(H, rtol, maxit, nullptr, nullptr)) return s;
    if (int s = launch_gradient(f, 2)) return s;
    if (int s = launch_gradient(f, 3)) return s;
    // mu_t, F1, production and the node terms of the next assembly, then
    // mu_eff and the diffusivities
    oa_sst_fields sf{};
    sf.k = f.kf;
    sf.omega = f.wf;
    sf.k_prev = f.k_prev;
    sf.rho = f.rho;
    sf.mu = mu_lam;
    sf.ymin = ymin;
    sf.gradU = f.gradU;
    sf.gradK = f.gradK;
    sf.gradW = f.gradW;
    sf.div = f.div;
    sf.vol = f.mesh->vol;
    sf.mut_old = f.mut;
    sf.pk_wall = nullptr;
    sf.wall_node = wall_node;
    sf.mut = f.mut;
    sf.F1 = f.F1;
    sf.Pk = f.Pk;
    sf.k_diag = f.sdk;
    sf.k_rhs = f.srk;
    sf.w_diag = f.sdw;
    sf.w_rhs = f.srw;
    if (int s = oa_sst_node_update((int)nn, c, f.s.dt, mut_urf, &sf, f.stream)) return s;
    if (int s = oa_sst_diffusivities((int)nn, c, mu_lam, f.mut, f.F1, f.mu, f.gkf, f.gwf, f.stream)) return s;
  }
  OA_CUDA(cudaStreamSynchronize(f.stream));
  return check_err_flag(f, "oa_flow_sst_iterate");
}

int oa_flow_set_tuning(oa_flow* H, const oa_tuning* t) {
  if (!H || !t) return fail(OA_ERR_ARG, "oa_flow_set_tuning: null argument");
  auto ok_bs = [](int b) { return b == 32 || b == 64 || b == 128; };
  if (!ok_bs(t->block_rows) || !ok_bs(t->block_elements) || !ok_bs(t->block_assembly) || t->gcr_chunk < 2 ||
      t->gcr_chunk % 2 || t->amg_refresh < 1)
    return fail(OA_ERR_ARG, "oa_flow_set_tuning: block sizes 32/64/128, even GCR chunk >= 2, AMG refresh >= 1");
  Flow& f = H->f;
  f.bs_rows = t->block_rows;
  f.bs_elems = t->block_elements;
  f.bs_asm = t->block_assembly;
  H->pc.gcr_chunk = t->gcr_chunk;
  H->pc.refresh = t->amg_refresh;
  if (t->amg_cheb_degree != 0 || t->amg_prolong_damping != 0.0) {
    const int deg = t->amg_cheb_degree ? t->amg_cheb_degree : std::max(2, H->pc.amg64.cheb_degree);
    const double wp = t->amg_prolong_damping != 0.0 ? t->amg_prolong_damping : H->pc.amg64.omega_p;
    if (int s = H->pc.set_smoothing(deg, wp)) return s;
  }
  return OA_OK;
}

int oa_flow_autotune(oa_flow* H, int iters, oa_tuning* out) {
  if (!H || iters < 1) return fail(OA_ERR_ARG, "oa_flow_autotune: bad arguments");
  Flow& f = H->f;
  const size_t nn = f.mesh->nn, ne = f.mesh->ne;
  // the state the trials start from, restored after each and at the end
  struct Saved {
    double* dev;
    double* copy;
    size_t n;
  };
  std::vector<Saved> saved;
  double* fields[] = {f.U, f.p, f.gradU, f.gradP, f.du, f.div, f.mDot, f.betaU, f.minU, f.maxU, f.duT};
  const size_t sizes[] = {3 * nn, nn, 9 * nn, 3 * nn, 3 * nn, nn, 12 * ne, 3 * nn, 3 * nn, 3 * nn, 3 * nn};
  int st = OA_OK;
  for (int k = 0; k < 11 && !st; ++k) {
    if (!fields[k]) continue;
    Saved sv{fields[k], nullptr, sizes[k]};
    if (cudaMalloc(&sv.copy, sizeof(double) * sv.n) != cudaSuccess) {
      st = fail(OA_ERR_CUDA, "oa_flow_autotune: could not save the state");
      break;
    }
    saved.push_back(sv);
    if (cudaMemcpyAsync(sv.copy, sv.dev, sizeof(double) * sv.n, cudaMemcpyDeviceToDevice, f.stream) != cudaSuccess)
      st = fail(OA_ERR_CUDA, "oa_flow_autotune: state copy failed");
  }
  auto restore = [&]() -> int {
    for (auto& sv : saved)
      OA_CUDA(cudaMemcpyAsync(sv.dev, sv.copy, sizeof(double) * sv.n, cudaMemcpyDeviceToDevice, f.stream));
    return OA_OK;
  };
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (!st && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
    st = fail(OA_ERR_CUDA, "oa_flow_autotune: event creation failed");
  const long long solves0 = H->pc.solves;
  // one trial: restore, one untimed iteration, `iters` timed ones
  auto trial = [&](double* ms) -> int {
    if (int s = restore()) return s;
    H->pc.solves = 0;  // the first solve of a trial refreshes the AMG numeric phase
    if (int s = oa_simple_iterate(H, 1, nullptr)) return s;
    OA_CUDA(cudaEventRecord(e0, f.stream));
    if (int s = oa_simple_iterate(H, iters, nullptr)) return s;
    OA_CUDA(cudaEventRecord(e1, f.stream));
    OA_CUDA(cudaEventSynchronize(e1));
    float t = 0.f;
    OA_CUDA(cudaEventElapsedTime(&t, e0, e1));
    *ms = t / iters;
    return OA_OK;
  };
  oa_tuning best{f.bs_rows, f.bs_elems, f.bs_asm, H->pc.gcr_chunk, H->pc.refresh, 0.0, 0.0,
                 std::max(2, H->pc.amg64.cheb_degree), H->pc.amg64.omega_p};
  double best_ms = 0.0;
  if (!st) st = trial(&best_ms);
  const double before = best_ms;
  // coordinate descent, one knob at a time
  const int bss[3] = {32, 64, 128};
  const int chunks[2] = {2, 4};
  const int refreshes[3] = {4, 8, 16};
  const int chebs[2] = {3, 4};
  // the AMG smoother: a degree-4 Chebyshev polynomial with prolongation
  // damping 0.85 takes 19 instead of 21 V-cycles on the 128^3 cavity (+4 %),
  // but costs 8 % on the 64^3 one, where fewer V-cycles are needed anyway
  const double dampings[2] = {0.74, 0.85};
  for (int knob = 0; knob < 7 && !st; ++knob) {
    const int* cand = knob < 3 ? bss : (knob == 3 ? chunks : (knob == 4 ? refreshes : chebs));
    const int nc = knob == 3 || knob >= 5 ? 2 : 3;
    for (int c = 0; c < nc && !st; ++c) {
      oa_tuning t = best;
      if (knob == 6) {
        if (t.amg_prolong_damping == dampings[c]) continue;
        t.amg_prolong_damping = dampings[c];
      } else {
        int* slot = knob == 0   ? &t.block_rows
                    : knob == 1 ? &t.block_elements
                    : knob == 2 ? &t.block_assembly
                    : knob == 3 ? &t.gcr_chunk
                    : knob == 4 ? &t.amg_refresh
                                : &t.amg_cheb_degree;
        if (*slot == cand[c]) continue;
        *slot = cand[c];
      }
      if ((st = oa_flow_set_tuning(H, &t))) break;
      double ms = 0.0;
      if ((st = trial(&ms))) break;
      if (ms < best_ms) {
        best_ms = ms;
        best = t;
      }
    }
    if (!st) st = oa_flow_set_tuning(H, &best);
  }
  if (!st) st = restore();
  if (!st && cudaStreamSynchronize(f.stream) != cudaSuccess) st = fail(OA_ERR_CUDA, "oa_flow_autotune: sync failed");
  H->pc.solves = 0;
  (void)solves0;
  for (auto& sv : saved) cudaFree(sv.copy);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) return st;
  best.ms_per_iteration_before = before;
  best.ms_per_iteration_after = best_ms;
  if (out) *out = best;
  return OA_OK;
}

int oa_flow_advance_time(oa_flow* H, int scheme, double dt) {
  if (!H || (scheme != OA_TIME_BDF1 && scheme != OA_TIME_BDF2) || !(dt > 0))
    return fail(OA_ERR_ARG, "oa_flow_advance_time: scheme must be OA_TIME_BDF1 or OA_TIME_BDF2 and dt > 0");
  Flow& f = H->f;
  if (f.turb) return fail(OA_ERR_ARG, "oa_flow_advance_time: the fused turbulence transport is steady only");
  const size_t n3 = 3 * (size_t)f.mesh->nn;
  if (!f.Uold) {
    if (int s = dalloc(&f.Uold, n3)) return s;
    if (int s = dalloc(&f.Uoldold, n3)) return s;
    OA_CUDA(cudaMemsetAsync(f.Uold, 0, sizeof(double) * n3, f.stream));
  }
  // time levels: old -> old-old, current -> old (the reference's preWork)
  OA_CUDA(cudaMemcpyAsync(f.Uoldold, f.Uold, sizeof(double) * n3, cudaMemcpyDeviceToDevice, f.stream));
  OA_CUDA(cudaMemcpyAsync(f.Uold, f.U, sizeof(double) * n3, cudaMemcpyDeviceToDevice, f.stream));
  f.dt_prev = f.time_steps ? f.dt_step : dt;
  f.dt_step = dt;
  f.time_scheme = scheme;
  ++f.time_steps;
  // BDF1 {1, -1} (src/basic/types.cpp:392-396); BDF2 with w = dt / dt_prev
  // (:398-410), BDF1 on the first step
  if (scheme == OA_TIME_BDF2 && f.time_steps >= 2) {
    const double w = f.dt_step / f.dt_prev;
    f.tk[0] = (1.0 + 2.0 * w) / (1.0 + w);
    f.tk[1] = -(1.0 + w);
    f.tk[2] = w * w / (1.0 + w);
    f.time_order = 2;
  } else {
    f.tk[0] = 1.0;
    f.tk[1] = -1.0;
    f.tk[2] = 0.0;
    f.time_order = 1;
  }
  OA_CUDA(cudaStreamSynchronize(f.stream));
  return OA_OK;
}

int oa_flow_last_control(oa_flow* H, int sys, oa_control_data* out) {
  if (!H || !out || (sys != 0 && sys != 1)) return fail(OA_ERR_ARG, "oa_flow_last_control: bad arguments");
  const oa_control_data& cd = sys == 0 ? H->f.cd_mom : H->f.cd_pc;
  if (cd.n_iterations < 0) return fail(OA_ERR_NOT_READY, "oa_flow_last_control: no solve of this system yet");
  *out = cd;
  return OA_OK;
}

int oa_flow_scales(oa_flow* H, double* u_ref, double* mass_scale, double* mom_scale) {
  if (!H) return fail(OA_ERR_ARG, "oa_flow_scales: null handle");
  if (u_ref) *u_ref = H->f.u_ref;
  if (mass_scale) *mass_scale = H->f.mass_scale;
  if (mom_scale) *mom_scale = H->f.mom_scale;
  return OA_OK;
}

int oa_flow_stream(oa_flow* H, void** stream) {
  if (!H || !stream) return fail(OA_ERR_ARG, "oa_flow_stream: null argument");
  *stream = (void*)H->f.stream;
  return OA_OK;
}

int oa_launch_count(long long* count) {
  if (!count) return fail(OA_ERR_ARG, "oa_launch_count: null argument");
  *count = g_launches.load();
  return OA_OK;
}

int oa_time_kernel(oa_flow* H, int which, int reps, double* ms) {
  if (!H || !ms || reps <= 0 || which < 0 || which > 3) return fail(OA_ERR_ARG, "oa_time_kernel: bad arguments");
  Flow& f = H->f;
  cudaEvent_t e0, e1;
  OA_CUDA(cudaEventCreate(&e0));
  OA_CUDA(cudaEventCreate(&e1));
  // one untimed launch, then reps timed ones
  for (int r = 0; r <= reps; ++r) {
    if (r == 1) OA_CUDA(cudaEventRecord(e0, f.stream));
    int s = OA_OK;
    if (which == 0) s = launch_momentum(f, mixed(f));
    else if (which == 1) s = launch_pcorr(f, mixed(f));
    else if (which == 2) s = launch_update_mdot(f);
    else s = launch_gradient(f, 1);
    if (s) return s;
  }
  OA_CUDA(cudaEventRecord(e1, f.stream));
  OA_CUDA(cudaEventSynchronize(e1));
  float t = 0.f;
  OA_CUDA(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = t / reps;
  return check_err_flag(f, "oa_time_kernel");
}

int oa_flow_sync(oa_flow* H) {
  if (!H) return fail(OA_ERR_ARG, "oa_flow_sync: null handle");
  OA_CUDA(cudaStreamSynchronize(H->f.stream));
  return OA_OK;
}

}  // extern "C"
