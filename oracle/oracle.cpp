// Oracle (test infrastructure only): CPU FP64 restatement of OpenAccel's
// CVFEM assembly + SIMPLE pressure-correction hot path for hex8 meshes.
// Only tests, the smoke check and the bench CPU-baseline leg use it.
//
// Each routine names the reference routine it restates (paths relative to the
// reference project root). Element loops are element-centric exactly as in the
// reference and scatter through a literal restatement of
// assembler<N>::applyCoeff_ (src/assemble/assembler.h:311-453), including the
// reduced-stencil lumping of missing columns into the diagonal block.
#include "oracle.h"

#include <algorithm>
#include <cstdint>
#include <cmath>
#include <cstring>
#include <numeric>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "hex8_master.hpp"
#include "pool.hpp"

namespace {

using oracle::hex8::LR;
using oracle::hex8::NPE;
using oracle::hex8::NSCS;
constexpr double SMALL = 2.220446049250313e-16;  // src/basic/types.h:179

int g_threads = 1;

// Static-chunked parallel loop on the persistent pool (serial below 4096
// items or with one thread).
template <class F>
void parallel_for(long n, F f) {
  if (g_threads <= 1 || n < 4096) {
    for (long i = 0; i < n; ++i) f(i);
    return;
  }
  oracle::Pool& P = oracle::Pool::get();
  P.run([&](int t) {
    long lo, hi;
    oracle::chunk_range(n, P.size(), t, &lo, &hi);
    for (long i = lo; i < hi; ++i) f(i);
  });
}

struct Case {
  orc_settings s;
  int nn, ne, nf, nbnd;
  std::vector<double> x;
  std::vector<int> conn;
  std::vector<int> fElem, fOrd, fBnd;
  std::vector<double> bndU;
  // geometry
  std::vector<double> vol, faceArea;  // vol[nn], faceArea[nf][4][3]
  // graph (reduced stencil, sorted columns)
  std::vector<int> rowPtr, cols, diagOff;
  // fields
  std::vector<double> U, p, gradU, gradP, du, div, mDot, rho, mu, sideU, wallNode;
  // high-resolution advection: velocity blending factor and its extrema
  // fields, [nn][3] each (nodeField blendingFactor / minValue / maxValue)
  std::vector<double> betaU, minU, maxU;
  // SIMPLEC: the consistent coefficient D~ [nn][3] (flowModel duTilde)
  std::vector<double> duT;
  // transient runs: scheme (0 steady, 1 BDF1, 2 BDF2), time steps taken, the
  // current and previous step sizes, velocity at the two previous time levels
  int timeScheme = 0, timeSteps = 0;
  double dtStep = 0.0, dtPrev = 0.0;
  std::vector<double> Uold, Uoldold;
  // element colours (no two elements of a colour share a node), for the
  // threaded CPU-baseline path
  std::vector<std::vector<int>> colors;
  // pressure-level rows (settings.ref_node, or a list for batched meshes)
  std::vector<int> refNodes;
  // boundary physical type by boundary index (ORC_BTYPE_WALL no-slip wall,
  // ORC_BTYPE_SYMMETRY symmetry plane); all walls until set
  std::vector<int> bndType;
  // symmetry planes: the nodes on a symmetry face, the assembled symmetry
  // area vector [nn][3] (sum of the exposed-area vectors of the face ips
  // nearest each node, mesh::updateAssembledSymmetryAreaField_,
  // src/mesh/meshGeometry.cpp:1787-1880) and the nodes on a wall face
  std::vector<int> symNodes;
  std::vector<double> symArea;
  std::vector<char> wallFaceNode;
  // expertParameters_.correctGradients_ (default off): gradients at symmetry
  // nodes lose their normal part (node*Field::correctGradientField_)
  bool correctGrad = false;
  // last assembled systems (for the solver inside simple_iteration)
  std::vector<double> Am, bm, xm, Ap, bp, xp;
  // continuity-residual scale rho U_ref h^2 (the residual normalisation of
  // the cavity benchmark; the reference's own lives in the absent liblinsolve)
  double massScale = 1.0;
  // linear solvers of simple_iteration: 0 Jacobi-BiCGStab (the parity
  // reference), 1 the reference example's configuration (GMRES + block ILU(0))
  int solverKind = 0;
};

// Greedy element colouring over shared nodes (built once per case).
void build_colors(Case& c) {
  std::vector<uint32_t> used(c.nn, 0u);
  std::vector<int> col(c.ne);
  int nc = 0;
  for (int e = 0; e < c.ne; ++e) {
    uint32_t m = 0;
    for (int a = 0; a < 8; ++a) m |= used[c.conn[8 * e + a]];
    int k = 0;
    while (k < 32 && (m >> k) & 1u) ++k;
    col[e] = k;
    nc = std::max(nc, k + 1);
    for (int a = 0; a < 8; ++a) used[c.conn[8 * e + a]] |= (1u << k);
  }
  c.colors.assign(nc, {});
  for (int e = 0; e < c.ne; ++e) c.colors[col[e]].push_back(e);
}

// Element loop that scatters into nodal/CSR storage. Serial: element order,
// exactly as the reference's bucket loop. Threaded: colour by colour, so each
// entry receives its contributions in colour order whatever the thread count.
template <class F>
void for_elements(const Case& c, F f) {
  if (g_threads <= 1) {
    for (int e = 0; e < c.ne; ++e) f(e);
    return;
  }
  for (const auto& cl : c.colors) parallel_for((long)cl.size(), [&](long i) { f(cl[i]); });
}

// Ordered dot product: per-thread partial sums added in thread order.
double pdot(long n, const double* a, const double* b) {
  if (g_threads <= 1 || n < 65536) {
    double s = 0.0;
    for (long i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
  }
  oracle::Pool& P = oracle::Pool::get();
  std::vector<double> part(P.size(), 0.0);
  P.run([&](int t) {
    long lo, hi;
    oracle::chunk_range(n, P.size(), t, &lo, &hi);
    double s = 0.0;
    for (long i = lo; i < hi; ++i) s += a[i] * b[i];
    part[t] = s;
  });
  double s = 0.0;
  for (double v : part) s += v;
  return s;
}

// ---------------------------------------------------------------------------
// graph: nodeGraph::buildGraph_ reduced stencil (src/mesh/graph/nodeGraph.cpp:29-98)
void build_graph(Case& c) {
  std::vector<std::set<int>> st(c.nn);
  for (int e = 0; e < c.ne; ++e) {
    const int* en = &c.conn[8 * e];
    for (int ip = 0; ip < NSCS; ++ip) {
      const int L = en[LR[ip][0]], R = en[LR[ip][1]];
      st[L].insert(L);
      st[L].insert(R);
      st[R].insert(L);
      st[R].insert(R);
    }
  }
  c.rowPtr.assign(c.nn + 1, 0);
  for (int i = 0; i < c.nn; ++i) c.rowPtr[i + 1] = c.rowPtr[i] + (int)st[i].size();
  c.cols.resize(c.rowPtr[c.nn]);
  c.diagOff.resize(c.nn);
  for (int i = 0; i < c.nn; ++i) {
    int k = c.rowPtr[i];
    for (int j : st[i]) {
      if (j == i) c.diagOff[i] = k - c.rowPtr[i];
      c.cols[k++] = j;
    }
  }
}

// applyCoeff_ (src/assemble/assembler.h:311-453): element nodes sorted by
// column id; for each row the sorted columns are searched monotonically in the
// row's sorted column list; a column absent from the row is added to the
// diagonal block (deductUnfound). lhs is [(n*N)x(n*N)] row-major with
// row = node*N+m, col = node*N+n.
template <int N>
void apply_coeff(Case& c, double* A, double* b, const int* nodes, int n, const double* rhs,
                 const double* lhs) {
  int perm[8];
  std::iota(perm, perm + n, 0);
  std::sort(perm, perm + n, [&](int a, int bb) { return nodes[a] < nodes[bb]; });
  for (int r = 0; r < n; ++r) {
    const int pr = perm[r];
    const int row = nodes[pr];
    const double* lrow = &lhs[N * N * pr * n];
    const double* rr = &rhs[N * pr];
    const int beg = c.rowPtr[row], len = c.rowPtr[row + 1] - beg;
    double* vals = &A[(long)N * N * beg];
    double* diag = &A[(long)N * N * (beg + c.diagOff[row])];
    int off = 0, offOld = 0;
    for (int j = 0; j < n; ++j) {
      const int pj = perm[j];
      const int col = nodes[pj];
      while (off < len && c.cols[beg + off] != col) ++off;
      if (off < len) {
        for (int m = 0; m < N; ++m)
          for (int q = 0; q < N; ++q) vals[N * N * off + N * m + q] += lrow[N * n * m + N * pj + q];
        offOld = off;
      } else {
        for (int m = 0; m < N; ++m)
          for (int q = 0; q < N; ++q) diag[N * m + q] += lrow[N * n * m + N * pj + q];
        off = offOld;
      }
    }
    for (int k = 0; k < N; ++k) b[N * row + k] += rr[k];
  }
}

bool is_symmetry_face(const Case& c, int f) {
  return !c.bndType.empty() && c.bndType[c.fBnd[f]] == ORC_BTYPE_SYMMETRY;
}

// unit vector of node i's assembled symmetry area (amag from the vector itself)
void sym_normal(const Case& c, int i, double* n) {
  const double* a = &c.symArea[3L * i];
  const double amag = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  for (int k = 0; k < 3; ++k) n[k] = a[k] / amag;
}

void gather_coords(const Case& c, int e, double* xe) {
  for (int a = 0; a < 8; ++a)
    for (int k = 0; k < 3; ++k) xe[3 * a + k] = c.x[3 * c.conn[8 * e + a] + k];
}

// Time-integration coefficients of the current step: BDF1 {1, -1}
// (src/basic/types.cpp:392-396), BDF2 {(1 + 2w)/(1 + w), -(1 + w), w^2/(1 + w)}
// with w = dt / dt_prev (:398-410); BDF2 takes BDF1 on the first step, when no
// second old level exists.
int time_coeffs(const Case& c, double* k) {
  if (c.timeScheme == 2 && c.timeSteps >= 2) {
    const double w = c.dtStep / c.dtPrev;
    k[0] = (1.0 + 2.0 * w) / (1.0 + w);
    k[1] = -(1.0 + w);
    k[2] = w * w / (1.0 + w);
    return 2;
  }
  k[0] = 1.0;
  k[1] = -1.0;
  k[2] = 0.0;
  return 1;
}

// mesh::updateDualNodalVolumeField_ (src/mesh/meshGeometry.cpp:1277-1345)
void dual_volume(Case& c) {
  c.vol.assign(c.nn, 0.0);
  for (int e = 0; e < c.ne; ++e) {
    double xe[24], v[8];
    gather_coords(c, e, xe);
    oracle::hex8::scv_volumes(xe, v);
    for (int a = 0; a < 8; ++a) c.vol[c.conn[8 * e + a]] += v[a];
  }
}

// mesh::updateExposedAreaVectorField_ (src/mesh/meshGeometry.cpp:1441-1527)
void exposed_areas(Case& c) {
  c.faceArea.assign(12 * c.nf, 0.0);
  for (int f = 0; f < c.nf; ++f) {
    const int e = c.fElem[f], o = c.fOrd[f];
    double xf[12];
    for (int k = 0; k < 4; ++k) {
      const int nd = c.conn[8 * e + oracle::hex8::FACE_NODES[o][k]];
      for (int d = 0; d < 3; ++d) xf[3 * k + d] = c.x[3 * nd + d];
    }
    oracle::hex8::quad_face_areav(xf, &c.faceArea[12 * f]);
  }
}

// ---------------------------------------------------------------------------
// flowModel::initializeMassFlowRateInterior_ (src/model/flow/flowModel.cpp:3303-3470)
void init_mdot(Case& c) {
  double N[96];
  oracle::hex8::scs_shape(N, c.s.u_shifted);
  parallel_for(c.ne, [&](long e) {
    double xe[24], A[36];
    gather_coords(c, (int)e, xe);
    oracle::hex8::scs_areav(xe, A);
    const int* en = &c.conn[8 * e];
    for (int ip = 0; ip < NSCS; ++ip) {
      double u[3] = {0, 0, 0}, rhoIp = 0.0;
      for (int a = 0; a < 8; ++a) {
        const double r = N[8 * ip + a];
        rhoIp += r * c.rho[en[a]];
        for (int j = 0; j < 3; ++j) u[j] += r * c.U[3 * en[a] + j];
      }
      double m = 0.0;
      for (int j = 0; j < 3; ++j) m += rhoIp * u[j] * A[3 * ip + j];
      c.mDot[12 * e + ip] = m;
    }
  });
}

// flowModel::updateMassFlowRateInterior_ (src/model/flow/flowModel.cpp:5272-5687),
// incompressible stationary frame: rhoHR = upwind density (the blending factor
// of rho is the zero dummy field, so the deferred correction vanishes).
void update_mdot(Case& c) {
  double Nv[96], Nc[96];
  oracle::hex8::scs_shape(Nv, c.s.u_shifted);
  oracle::hex8::scs_shape(Nc, false);
  parallel_for(c.ne, [&](long e) {
    const int* en = &c.conn[8 * e];
    double xe[24], A[36], g[288], v[8], w[8];
    gather_coords(c, (int)e, xe);
    oracle::hex8::scs_areav(xe, A);
    oracle::hex8::scv_volumes(xe, v);
    double Vel = 0.0;
    for (int a = 0; a < 8; ++a) Vel += v[a];
    const double iV = 1.0 / Vel;
    for (int a = 0; a < 8; ++a) w[a] = 0.0;
    for (int a = 0; a < 8; ++a) w[a] += v[a] * iV;
    oracle::hex8::grad_op(xe, g, c.s.p_grad_shifted);
    for (int ip = 0; ip < NSCS; ++ip) {
      const int il = LR[ip][0], ir = LR[ip][1];
      double du[3] = {0, 0, 0}, u[3] = {0, 0, 0}, dp[3] = {0, 0, 0}, Gp[3] = {0, 0, 0};
      double rhoIp = 0.0;
      for (int a = 0; a < 8; ++a) {
        const double r = Nv[8 * ip + a];
        rhoIp += r * c.rho[en[a]];
        for (int j = 0; j < 3; ++j) {
          du[j] += r * c.du[3 * en[a] + j];
          u[j] += r * c.U[3 * en[a] + j];
          dp[j] += g[24 * ip + 3 * a + j] * c.p[en[a]];
          Gp[j] += w[a] * c.gradP[3 * en[a] + j];
        }
      }
      const double tU = c.mDot[12 * e + ip] / rhoIp;
      const double rhoUp = tU > 0 ? c.rho[en[il]] : c.rho[en[ir]];
      double m = 0.0;
      for (int j = 0; j < 3; ++j) {
        m += rhoUp * u[j] * A[3 * ip + j];
        m -= rhoUp * du[j] * (dp[j] - Gp[j]) * A[3 * ip + j];
      }
      c.mDot[12 * e + ip] = c.s.mdot_urf * m + (1.0 - c.s.mdot_urf) * c.mDot[12 * e + ip];
    }
  });
}

// flowModel::updateMassDivergenceField_ interior part (flowModel.cpp:13710-13760);
// wall side mass flows are zero.
void update_div(Case& c) {
  std::fill(c.div.begin(), c.div.end(), 0.0);
  for_elements(c, [&](int e) {
    const int* en = &c.conn[8 * e];
    for (int ip = 0; ip < NSCS; ++ip) {
      const double m = c.mDot[12 * e + ip];
      c.div[en[LR[ip][0]]] += m;
      c.div[en[LR[ip][1]]] -= m;
    }
  });
  // transient contribution (flowModel.cpp:13556-13700, fixed mesh): the
  // density at every time level is the current one (constant density)
  if (c.timeScheme) {
    double k[3];
    const int order = time_coeffs(c, k);
    for (int i = 0; i < c.nn; ++i) {
      const double rho = c.rho[i];
      if (order == 1)
        c.div[i] += (k[0] * rho + k[1] * rho) * c.vol[i] / c.dtStep;
      else
        c.div[i] += (k[0] * rho + k[1] * rho + k[2] * rho) * c.vol[i] / c.dtStep;
    }
  }
}

// Gradient at a symmetry node without its normal part, at the end of
// updateGradientField (nodeField.hpp:4939-4943): a scalar's G - (G.n) n
// (nodeScalarField.cpp:44-112); a vector's G - (G n) n^T - n (n^T G)
// + 2 (n^T G n) n n^T (nodeVectorField.cpp:44-148).
template <int NC>
void correct_gradient(const Case& c, int node, double* G) {
  double n[3];
  sym_normal(c, node, n);
  if (NC == 1) {
    const double dot = G[0] * n[0] + G[1] * n[1] + G[2] * n[2];
    for (int j = 0; j < 3; ++j) G[j] -= dot * n[j];
    return;
  }
  double Gn[3] = {0, 0, 0}, nG[3] = {0, 0, 0};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      Gn[i] += G[3 * i + j] * n[j];
      nG[j] += G[3 * i + j] * n[i];
    }
  const double nGn = nG[0] * n[0] + nG[1] * n[1] + nG[2] * n[2];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      G[3 * i + j] -= Gn[i] * n[j];
      G[3 * i + j] -= n[i] * nG[j];
      G[3 * i + j] += 2.0 * n[i] * n[j] * nGn;
    }
}

// nodeField::updateGradientField (src/field/nodeField/nodeField.hpp:3253-3445
// interior, :4732-4930 boundary, :6362-6398 relax). NC = field components.
template <int NC>
void update_gradient(Case& c, const std::vector<double>& phi, std::vector<double>& grad, bool shifted) {
  const double g = c.s.grad_urf;
  for (auto& v : grad) v *= (1.0 - g);
  double N[96];
  oracle::hex8::scs_shape(N, shifted);
  for_elements(c, [&](int e) {
    const int* en = &c.conn[8 * e];
    double xe[24], A[36];
    gather_coords(c, e, xe);
    oracle::hex8::scs_areav(xe, A);
    for (int ip = 0; ip < NSCS; ++ip) {
      const int L = en[LR[ip][0]], R = en[LR[ip][1]];
      double pip[NC];
      for (int j = 0; j < NC; ++j) pip[j] = 0.0;
      for (int a = 0; a < 8; ++a)
        for (int j = 0; j < NC; ++j) pip[j] += N[8 * ip + a] * phi[NC * en[a] + j];
      const double ivL = 1.0 / c.vol[L], ivR = 1.0 / c.vol[R];
      for (int i = 0; i < NC; ++i)
        for (int j = 0; j < 3; ++j) {
          grad[3 * NC * L + 3 * i + j] += g * (pip[i] - phi[NC * L + i]) * A[3 * ip + j] * ivL;
          grad[3 * NC * R + 3 * i + j] -= g * (pip[i] - phi[NC * R + i]) * A[3 * ip + j] * ivR;
        }
    }
  });
  double Nf[16];
  oracle::hex8::face_shape(Nf, shifted);
  for (int f = 0; f < c.nf; ++f) {
    // symmetry faces add nothing (nodeField.hpp:4764)
    if (is_symmetry_face(c, f)) continue;
    const int e = c.fElem[f], o = c.fOrd[f];
    int fn[4];
    for (int k = 0; k < 4; ++k) fn[k] = c.conn[8 * e + oracle::hex8::FACE_NODES[o][k]];
    for (int ip = 0; ip < 4; ++ip) {
      const int nn = fn[ip];
      double pip[NC];
      for (int j = 0; j < NC; ++j) pip[j] = 0.0;
      for (int k = 0; k < 4; ++k)
        for (int j = 0; j < NC; ++j) pip[j] += Nf[4 * ip + k] * phi[NC * fn[k] + j];
      const double iv = 1.0 / c.vol[nn];
      for (int i = 0; i < NC; ++i)
        for (int j = 0; j < 3; ++j)
          grad[3 * NC * nn + 3 * i + j] +=
              g * (pip[i] - phi[NC * nn + i]) * c.faceArea[12 * f + 3 * ip + j] * iv;
    }
  }
  if (c.correctGrad)
    for (int i : c.symNodes) correct_gradient<NC>(c, i, &grad[3L * NC * i]);
}

// ---------------------------------------------------------------------------
// pressureCorrectionAssembler::assembleElemTermsInterior_
// (src/assemble/flow/segregatedFlow/pressureCorrectionAssembler/
//  pressureCorrectionAssemblerElemTerms.cpp:17-616), incompressible,
// stationary frame; adjustMatrixForPressureReference
// (pressureCorrectionAssembler.cpp:19-63). No-slip wall faces add rho*U_bc.A
// with U_bc tangential to the flat walls, i.e. exact zeros, so they are omitted.
// Velocity blending factor of the high-resolution scheme:
// nodeField::updateMinMaxFields (src/field/nodeField/nodeField.hpp:1843-2066,
// defaults: no extrema expansion, no smoothing) followed by
// nodeField::updateBlendingFactorField (:2069-2410 interior and boundary ips,
// then the relaxation beta = 0.75 beta_prev + 0.25 beta, :2410+). Interior
// ips: the extrema over the edge neighbours, then the limiter at both ends of
// every SCS ip with dx = x_ip - x_node (x_ip from the standard trilinear
// coordinate shape functions); boundary faces: the limiter at each face ip's
// nearest node (standard face shape functions for x_ip).
void update_blending_u(Case& c) {
  const long n3 = 3L * c.nn;
  c.minU.assign(c.U.begin(), c.U.end());
  c.maxU.assign(c.U.begin(), c.U.end());
  for (int e = 0; e < c.ne; ++e) {
    const int* en = &c.conn[8 * e];
    for (int ip = 0; ip < NSCS; ++ip) {
      const int L = en[LR[ip][0]], R = en[LR[ip][1]];
      for (int i = 0; i < 3; ++i) {
        c.minU[3 * L + i] = std::min(c.minU[3 * L + i], c.U[3 * R + i]);
        c.maxU[3 * L + i] = std::max(c.maxU[3 * L + i], c.U[3 * R + i]);
        c.minU[3 * R + i] = std::min(c.minU[3 * R + i], c.U[3 * L + i]);
        c.maxU[3 * R + i] = std::max(c.maxU[3 * R + i], c.U[3 * L + i]);
      }
    }
  }
  const std::vector<double> prev = c.betaU;
  std::vector<double> beta(n3, c.s.beta_max);
  // limiter at node nd for the point xip (reference formulas, both loops)
  auto limit = [&](int nd, const double* xip) {
    double dx[3];
    for (int j = 0; j < 3; ++j) dx[j] = xip[j] - c.x[3 * nd + j];
    for (int i = 0; i < 3; ++i) {
      double rgrad = 0.0;
      for (int j = 0; j < 3; ++j) rgrad += c.gradU[9 * nd + 3 * i + j] * dx[j];
      if (rgrad > 0)
        rgrad = rgrad + SMALL;
      else
        rgrad = rgrad - SMALL;
      const double dmax = c.maxU[3 * nd + i] - c.U[3 * nd + i];
      const double dmin = c.minU[3 * nd + i] - c.U[3 * nd + i];
      const double betaLocal = std::max(dmax / rgrad, dmin / rgrad);
      const double beta12Local = std::max(-dmax / rgrad, -dmin / rgrad);
      double y = std::min(betaLocal, beta12Local);
      if (c.s.beta_max < 2.0 - SMALL) y = ((y * y + 2.0 * y) / (y * y + y + 2.0));
      if ((rgrad > 100 * SMALL) || (rgrad < -100 * SMALL)) beta[3 * nd + i] = std::min(beta[3 * nd + i], y);
    }
  };
  double Nc[96];
  oracle::hex8::scs_shape(Nc, false);
  for (int e = 0; e < c.ne; ++e) {
    const int* en = &c.conn[8 * e];
    for (int ip = 0; ip < NSCS; ++ip) {
      double xip[3] = {0.0, 0.0, 0.0};
      for (int a = 0; a < 8; ++a)
        for (int j = 0; j < 3; ++j) xip[j] += Nc[8 * ip + a] * c.x[3 * en[a] + j];
      limit(en[LR[ip][0]], xip);
      limit(en[LR[ip][1]], xip);
    }
  }
  double Nf[16];
  oracle::hex8::face_shape(Nf, false);
  for (int f = 0; f < c.nf; ++f) {
    const int* en = &c.conn[8 * c.fElem[f]];
    const int o = c.fOrd[f];
    for (int ip = 0; ip < 4; ++ip) {
      double xip[3] = {0.0, 0.0, 0.0};
      for (int k = 0; k < 4; ++k)
        for (int j = 0; j < 3; ++j) xip[j] += Nf[4 * ip + k] * c.x[3 * en[oracle::hex8::FACE_NODES[o][k]] + j];
      limit(en[oracle::hex8::FACE_NODES[o][ip]], xip);
    }
  }
  for (long k = 0; k < n3; ++k) c.betaU[k] = 0.75 * prev[k] + 0.25 * beta[k];
}

void assemble_pcorr(Case& c, double* A, double* b) {
  const int nnz = c.rowPtr[c.nn];
  std::fill(A, A + nnz, 0.0);
  std::fill(b, b + c.nn, 0.0);
  double Nv[96], Nc[96];
  oracle::hex8::scs_shape(Nv, c.s.u_shifted);
  oracle::hex8::scs_shape(Nc, false);
  for_elements(c, [&](int e) {
    const int* en = &c.conn[8 * e];
    double xe[24], Ar[36], g[288], v[8], w[8], lhs[64], rhs[8];
    std::fill(lhs, lhs + 64, 0.0);
    std::fill(rhs, rhs + 8, 0.0);
    gather_coords(c, e, xe);
    oracle::hex8::scs_areav(xe, Ar);
    oracle::hex8::scv_volumes(xe, v);
    double Vel = 0.0;
    for (int a = 0; a < 8; ++a) Vel += v[a];
    const double iV = 1.0 / Vel;
    for (int a = 0; a < 8; ++a) w[a] = 0.0;
    for (int a = 0; a < 8; ++a) w[a] += v[a] * iV;
    oracle::hex8::grad_op(xe, g, c.s.p_grad_shifted);
    for (int ip = 0; ip < NSCS; ++ip) {
      const int il = LR[ip][0], ir = LR[ip][1];
      const double tm = c.mDot[12 * e + ip];
      // the lhs diffusivity is D~ with SIMPLEC, the rhs keeps D
      // (pressureCorrectionAssemblerElemTerms.cpp:126-134)
      const std::vector<double>& dl = c.s.du_mode == 1 ? c.duT : c.du;
      double u[3] = {0, 0, 0}, du[3] = {0, 0, 0}, dul[3] = {0, 0, 0}, dp[3] = {0, 0, 0}, Gp[3] = {0, 0, 0};
      for (int a = 0; a < 8; ++a) {
        const double r = Nv[8 * ip + a];
        for (int j = 0; j < 3; ++j) {
          u[j] += r * c.U[3 * en[a] + j];
          du[j] += r * c.du[3 * en[a] + j];
          dul[j] += r * dl[3 * en[a] + j];
          dp[j] += g[24 * ip + 3 * a + j] * c.p[en[a]];
          Gp[j] += w[a] * c.gradP[3 * en[a] + j];
        }
      }
      const double rhoHR = tm > 0 ? c.rho[en[il]] : c.rho[en[ir]];
      for (int a = 0; a < 8; ++a) {
        double f = 0.0;
        for (int j = 0; j < 3; ++j) f += -rhoHR * dul[j] * g[24 * ip + 3 * a + j] * Ar[3 * ip + j];
        lhs[8 * il + a] += f;
        lhs[8 * ir + a] -= f;
      }
      double m = 0.0;
      for (int j = 0; j < 3; ++j) {
        m += rhoHR * u[j] * Ar[3 * ip + j];
        m -= rhoHR * du[j] * (dp[j] - Gp[j]) * Ar[3 * ip + j];
      }
      rhs[il] -= m;
      rhs[ir] += m;
    }
    apply_coeff<1>(c, A, b, en, 8, rhs, lhs);
  });
  for (const int r : c.refNodes) {
    const double d = A[c.rowPtr[r] + c.diagOff[r]];
    for (int k = c.rowPtr[r]; k < c.rowPtr[r + 1]; ++k) A[k] = 0.0;
    A[c.rowPtr[r] + c.diagOff[r]] = d;
    b[r] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// navierStokesAssembler momentum system:
//  node terms   navierStokesAssemblerNodeTerms.cpp:16-149 (steady, no body force,
//               stationary frame)
//  interior     navierStokesAssemblerElemTerms.cpp:15-441 (upwind, beta = 0 dummy,
//               incompressible)
//  no-slip wall navierStokesAssemblerElemBoundaryConditions.cpp:2659-2981 with
//               IP_ZERO_NORMAL_STRESS_FIXED_VEL__ (:592-654), laminar
//  post         phiAssembler.h:748-753 + :967-1006 (diag / urf),
//               navierStokesAssembler.cpp:234-385 (wall-node rhs * 0.75)
//  DU           navierStokesAssembler.cpp:84-232 (SIMPLE, steady)
// navierStokesAssembler::assembleElemTermsBoundarySymmetry_
// (src/assemble/flow/segregatedFlow/navierStokesAssembler/
//  navierStokesAssemblerElemBoundaryConditions.cpp:2082-2375): at each face
// ip, the full viscous stress -mu (dU_i/dx_j + dU_j/dx_i) A_j of the element's
// own velocities (IP_FULL_STRESS__, :295-344; the bulk term vanishes for the
// incompressible fluid), mu at the ip by the face shape functions.
void symmetry_face(const Case& c, int f, const double* Nf, double* lhs, double* rhs) {
  const int e = c.fElem[f], o = c.fOrd[f];
  const int* en = &c.conn[8 * e];
  double xe[24], g[96], muf[4];
  gather_coords(c, e, xe);
  for (int k = 0; k < 4; ++k) muf[k] = c.mu[en[oracle::hex8::FACE_NODES[o][k]]];
  oracle::hex8::face_grad_op(o, xe, g, c.s.u_grad_shifted);
  const double* av = &c.faceArea[12 * f];
  for (int ip = 0; ip < 4; ++ip) {
    const int nn = oracle::hex8::FACE_NODES[o][ip];
    double muB = 0.0;
    for (int k = 0; k < 4; ++k) muB += Nf[4 * ip + k] * muf[k];
    for (int a = 0; a < 8; ++a) {
      const double* ga = &g[24 * ip + 3 * a];
      const double* Ua = &c.U[3L * en[a]];
      for (int i = 0; i < 3; ++i) {
        const int iR = 3 * nn + i, rowR = iR * 24;
        for (int j = 0; j < 3; ++j) {
          const double Aj = av[3 * ip + j];
          double lf = -muB * ga[j] * Aj;
          lhs[rowR + 3 * a + i] += lf;
          rhs[iR] -= lf * Ua[i];
          lf = -muB * ga[i] * Aj;
          lhs[rowR + 3 * a + j] += lf;
          rhs[iR] -= lf * Ua[j];
        }
      }
    }
  }
}

void assemble_momentum(Case& c, double* A, double* b) {
  const int nnz = c.rowPtr[c.nn];
  std::fill(A, A + 9L * nnz, 0.0);
  std::fill(b, b + 3L * c.nn, 0.0);
  // node terms, one applyCoeff_ per node
  double tk[3];
  const int order = c.timeScheme ? time_coeffs(c, tk) : 0;
  for (int i = 0; i < c.nn; ++i) {
    double lhs[9] = {0}, rhs[3] = {0};
    const double rho = c.rho[i], vol = c.vol[i], dv = c.div[i];
    if (order == 0) {
      // steady: false transient with the physical timescale (...NodeTerms.cpp:16-149)
      const double lf = rho * vol / c.s.dt;
      for (int k = 0; k < 3; ++k) {
        if (dv < 0) lhs[4 * k] += -dv;
        rhs[k] -= -dv * c.U[3 * i + k];
        rhs[k] -= c.gradP[3 * i + k] * vol;
        lhs[4 * k] += lf;
      }
    } else {
      // BDF1 / BDF2 (...NodeTerms.cpp:151-427); density constant in time
      const double lhsfac = tk[0] * rho * vol / c.dtStep;
      const double lhsfacOld = tk[1] * rho * vol / c.dtStep;
      const double lhsfacOldOld = tk[2] * rho * vol / c.dtStep;
      for (int k = 0; k < 3; ++k) {
        lhs[4 * k] += lhsfac;
        if (order == 1)
          rhs[k] -= (lhsfac * c.U[3 * i + k] + lhsfacOld * c.Uold[3 * i + k]);
        else
          rhs[k] -= (lhsfac * c.U[3 * i + k] + lhsfacOld * c.Uold[3 * i + k] + lhsfacOldOld * c.Uoldold[3 * i + k]);
        if (dv < 0) lhs[4 * k] += -dv;
        rhs[k] -= -dv * c.U[3 * i + k];
        rhs[k] -= c.gradP[3 * i + k] * vol;
      }
    }
    apply_coeff<3>(c, A, b, &i, 1, rhs, lhs);
  }
  // interior elements
  double Nv[96], Nc[96];
  oracle::hex8::scs_shape(Nv, c.s.u_shifted);
  oracle::hex8::scs_shape(Nc, false);
  for_elements(c, [&](int e) {
    const int* en = &c.conn[8 * e];
    std::vector<double> lhs(576, 0.0), rhs(24, 0.0);
    double xe[24], Ar[36], g[288], Ue[24], mue[8];
    gather_coords(c, e, xe);
    for (int a = 0; a < 8; ++a) {
      mue[a] = c.mu[en[a]];
      for (int k = 0; k < 3; ++k) Ue[3 * a + k] = c.U[3 * en[a] + k];
    }
    oracle::hex8::scs_areav(xe, Ar);
    oracle::hex8::grad_op(xe, g, c.s.u_grad_shifted);
    for (int ip = 0; ip < NSCS; ++ip) {
      const int il = LR[ip][0], ir = LR[ip][1];
      const double tm = c.mDot[12 * e + ip];
      double muIp = 0.0;
      for (int a = 0; a < 8; ++a) muIp += Nv[8 * ip + a] * mue[a];
      // high resolution: deferred correction beta_up,i (x_ip - x_up) . grad u_i,up
      // (navierStokesAssemblerElemTerms.cpp:287-330), x_ip from the standard
      // coordinate shape functions
      double xip[3] = {0.0, 0.0, 0.0};
      if (c.s.hr)
        for (int a = 0; a < 8; ++a)
          for (int j = 0; j < 3; ++j) xip[j] += Nc[8 * ip + a] * xe[3 * a + j];
      for (int i = 0; i < 3; ++i) {
        const double up = tm > 0 ? Ue[3 * il + i] : Ue[3 * ir + i];
        double dcorr = 0.0;
        if (c.s.hr) {
          const int iu = tm > 0 ? il : ir;
          const int nu = en[iu];
          for (int j = 0; j < 3; ++j)
            dcorr += c.betaU[3 * nu + i] * (xip[j] - xe[3 * iu + j]) * c.gradU[9 * nu + 3 * i + j];
        }
        const double af = tm * (up + dcorr);
        const int iL = 3 * il + i, iR = 3 * ir + i;
        const int rowL = iL * 24, rowR = iR * 24;
        rhs[iL] -= af;
        rhs[iR] += af;
        const double fl = 0.5 * (tm + std::fabs(tm));
        lhs[rowL + 3 * il + i] += fl;
        lhs[rowR + 3 * il + i] -= fl;
        const double fr = 0.5 * (tm - std::fabs(tm));
        lhs[rowR + 3 * ir + i] -= fr;
        lhs[rowL + 3 * ir + i] += fr;
      }
      for (int a = 0; a < 8; ++a) {
        const double* ga = &g[24 * ip + 3 * a];
        for (int i = 0; i < 3; ++i) {
          const int iL = 3 * il + i, iR = 3 * ir + i;
          const int rowL = iL * 24, rowR = iR * 24;
          double lc = 0.0;
          for (int j = 0; j < 3; ++j) {
            const double axj = Ar[3 * ip + j];
            const double uj = Ue[3 * a + j];
            lc += -muIp * ga[j] * axj;
            const double fj = -muIp * ga[i] * axj;
            lhs[rowL + 3 * a + j] += fj;
            lhs[rowR + 3 * a + j] -= fj;
            rhs[iL] -= fj * uj;
            rhs[iR] += fj * uj;
          }
          lhs[rowL + 3 * a + i] += lc;
          lhs[rowR + 3 * a + i] -= lc;
          rhs[iL] -= lc * Ue[3 * a + i];
          rhs[iR] += lc * Ue[3 * a + i];
        }
      }
    }
    apply_coeff<3>(c, A, b, en, 8, rhs.data(), lhs.data());
  });
  // no-slip walls (laminar): zero normal stress with fixed velocity
  double Nf[16];
  oracle::hex8::face_shape(Nf, c.s.u_shifted);
  std::vector<double> lhs(576), rhs(24);
  for (int f = 0; f < c.nf; ++f) {
    const int e = c.fElem[f], o = c.fOrd[f];
    const int* en = &c.conn[8 * e];
    std::fill(lhs.begin(), lhs.end(), 0.0);
    std::fill(rhs.begin(), rhs.end(), 0.0);
    if (is_symmetry_face(c, f)) {
      symmetry_face(c, f, Nf, lhs.data(), rhs.data());
      apply_coeff<3>(c, A, b, en, 8, rhs.data(), lhs.data());
      continue;
    }
    double xe[24], g[96], Ue[24], bcm[8], muf[4];
    gather_coords(c, e, xe);
    for (int a = 0; a < 8; ++a) {
      bcm[a] = 1.0;
      for (int k = 0; k < 3; ++k) Ue[3 * a + k] = c.U[3 * en[a] + k];
    }
    for (int k = 0; k < 4; ++k) {
      const int ic = oracle::hex8::FACE_NODES[o][k];
      muf[k] = c.mu[en[ic]];
      bcm[ic] = 0.0;
      for (int d = 0; d < 3; ++d) Ue[3 * ic + d] = c.sideU[3 * en[ic] + d];
    }
    oracle::hex8::face_grad_op(o, xe, g, c.s.u_grad_shifted);
    const double* av = &c.faceArea[12 * f];
    for (int ip = 0; ip < 4; ++ip) {
      const int nn = oracle::hex8::FACE_NODES[o][ip];
      double asq = 0.0;
      for (int j = 0; j < 3; ++j) asq += av[3 * ip + j] * av[3 * ip + j];
      const double amag = std::sqrt(asq);
      double muB = 0.0;
      for (int k = 0; k < 4; ++k) muB += Nf[4 * ip + k] * muf[k];
      double nx[3];
      for (int i = 0; i < 3; ++i) nx[i] = av[3 * ip + i] / amag;
      for (int a = 0; a < 8; ++a) {
        const double* ga = &g[24 * ip + 3 * a];
        for (int j = 0; j < 3; ++j) {
          const double axj = av[3 * ip + j];
          const double gj = ga[j];
          const double uj = Ue[3 * a + j];
          for (int i = 0; i < 3; ++i) {
            const int iR = 3 * nn + i, rowR = iR * 24;
            const double gi = ga[i], ui = Ue[3 * a + i], ni = nx[i];
            const double om = 1.0 - ni * ni;
            double lf = -muB * gj * axj * om;
            lhs[rowR + 3 * a + i] += lf * bcm[a];
            rhs[iR] -= lf * ui;
            lf = -muB * gi * axj * om;
            lhs[rowR + 3 * a + j] += lf * bcm[a];
            rhs[iR] -= lf * uj;
            for (int l = 0; l < 3; ++l) {
              if (i == l) continue;
              const double nil = ni * nx[l];
              const double ul = Ue[3 * a + l], gl = ga[l];
              lf = muB * gj * axj * nil;
              lhs[rowR + 3 * a + l] += lf * bcm[a];
              rhs[iR] -= lf * ul;
              lf = muB * gl * axj * nil;
              lhs[rowR + 3 * a + j] += lf * bcm[a];
              rhs[iR] -= lf * uj;
            }
          }
        }
      }
    }
    apply_coeff<3>(c, A, b, en, 8, rhs.data(), lhs.data());
  }
  // relaxation of the diagonal, wall-node rhs relaxation
  const double ui = 1.0 / c.s.urf_u;
  for (int i = 0; i < c.nn; ++i) {
    double* d = &A[9L * (c.rowPtr[i] + c.diagOff[i])];
    for (int k = 0; k < 3; ++k) d[4 * k] *= ui;
  }
  // navierStokesAssembler::assembleBoundaryRelaxation_ (navierStokesAssembler.cpp:241-385):
  // every boundary node in steady runs, the no-slip wall nodes alone in
  // transient ones
  const bool wall_only = c.timeScheme != 0 && !c.symNodes.empty();
  for (int i = 0; i < c.nn; ++i)
    if (wall_only ? c.wallFaceNode[i] != 0 : c.wallNode[i] != 0.0)
      for (int k = 0; k < 3; ++k) b[3 * i + k] *= c.s.wall_rhs_relax;
  // applySymmetryConditions_ (navierStokesAssembler.cpp:387-471): the rhs of a
  // symmetry node loses its component along the assembled symmetry normal
  for (int i : c.symNodes) {
    double n[3];
    sym_normal(c, i, n);
    const double dot = b[3 * i] * n[0] + b[3 * i + 1] * n[1] + b[3 * i + 2] * n[2];
    for (int k = 0; k < 3; ++k) b[3 * i + k] -= dot * n[k];
  }
  // DU coefficients: navierStokesAssembler::computeDUCoefficients
  // (src/assemble/flow/segregatedFlow/navierStokesAssembler/navierStokesAssembler.cpp:84-232):
  // D = V / (a_ii + SMALL), or dt / rho for the fractional-step method (steady:
  // gamma1 = 1, dt the physical timescale); SIMPLEC also D~ = V / (a_ii + sum
  // of the row's off-diagonal (i, i) coefficients + SMALL)
  for (int i = 0; i < c.nn; ++i) {
    const double* d = &A[9L * (c.rowPtr[i] + c.diagOff[i])];
    for (int k = 0; k < 3; ++k)
      c.du[3 * i + k] = c.s.du_mode == 2 ? (order ? c.dtStep / tk[0] / c.rho[i] : c.s.dt / c.rho[i])
                                          : c.vol[i] / (d[4 * k] + SMALL);
    if (c.s.du_mode == 1)
      for (int k = 0; k < 3; ++k) {
        double off = 0.0;
        for (int q = c.rowPtr[i]; q < c.rowPtr[i + 1]; ++q)
          if (q - c.rowPtr[i] != c.diagOff[i]) off += A[9L * q + 4 * k];
        c.duT[3 * i + k] = c.vol[i] / (d[4 * k] + off + SMALL);
      }
  }
  // assembleNormalRelaxation (navierStokesAssembler.cpp:473-699, urf 0.75 from
  // navierStokesEquation.cpp:169), after the DU coefficients: the diagonal
  // block D of a symmetry node gains (1 - urf) D n n^T
  for (int i : c.symNodes) {
    double n[3], T[9], M[9];
    sym_normal(c, i, n);
    for (int a = 0; a < 3; ++a)
      for (int q = 0; q < 3; ++q) T[3 * a + q] = n[a] * n[q];
    double* d = &A[9L * (c.rowPtr[i] + c.diagOff[i])];
    for (int a = 0; a < 3; ++a)
      for (int q = 0; q < 3; ++q) {
        M[3 * a + q] = 0.0;
        for (int k = 0; k < 3; ++k) M[3 * a + q] += d[3 * a + k] * T[3 * k + q];
      }
    for (int k = 0; k < 9; ++k) d[k] += (1.0 - 0.75) * M[k];
  }
}

// ---------------------------------------------------------------------------
// Scalar transport of a turbulence field (k or omega of the SST model):
// phiAssembler<1>::assembleElemTermsInterior_
// (src/assemble/phiAssembler/phiAssemblerElemTerms.hpp:11-413) with upwind
// advection (the blending factor of both fields is zero) and diffusion with the
// nodal diffusivity interpolated to the ip, on the velocity's shape functions
// and gradient operator. Walls are zero-gradient for k and omega
// (turbulent*SSTAssemblerElemBoundaryConditions.cpp: no boundary element
// terms). Node terms are given per node (sdiag, srhs: the SST node update's
// sources), added by one applyCoeff_ per node before the elements; then the
// diagonal is relaxed by 1/urf (phiAssembler.h:967-1006).
void assemble_scalar_transport(Case& c, const double* phi, const double* gam, const double* sdiag,
                               const double* srhs, double urf, double* A, double* b) {
  const int nnz = c.rowPtr[c.nn];
  std::fill(A, A + nnz, 0.0);
  std::fill(b, b + c.nn, 0.0);
  for (int i = 0; i < c.nn; ++i) {
    double lhs[1] = {sdiag[i]}, rhs[1] = {srhs[i]};
    apply_coeff<1>(c, A, b, &i, 1, rhs, lhs);
  }
  double Nv[96];
  oracle::hex8::scs_shape(Nv, c.s.u_shifted);
  for_elements(c, [&](int e) {
    const int* en = &c.conn[8 * e];
    double lhs[64] = {0.0}, rhs[8] = {0.0};
    double xe[24], Ar[36], g[288], pe[8], ge[8];
    gather_coords(c, e, xe);
    for (int a = 0; a < 8; ++a) {
      pe[a] = phi[en[a]];
      ge[a] = gam[en[a]];
    }
    oracle::hex8::scs_areav(xe, Ar);
    oracle::hex8::grad_op(xe, g, c.s.u_grad_shifted);
    for (int ip = 0; ip < NSCS; ++ip) {
      const int il = LR[ip][0], ir = LR[ip][1];
      const double tm = c.mDot[12 * e + ip];
      double gIp = 0.0;
      for (int a = 0; a < 8; ++a) gIp += Nv[8 * ip + a] * ge[a];
      // advection, upwind
      const double af = tm * (tm > 0 ? pe[il] : pe[ir]);
      rhs[il] -= af;
      rhs[ir] += af;
      const double fl = 0.5 * (tm + std::fabs(tm));
      lhs[8 * il + il] += fl;
      lhs[8 * ir + il] -= fl;
      const double fr = 0.5 * (tm - std::fabs(tm));
      lhs[8 * ir + ir] -= fr;
      lhs[8 * il + ir] += fr;
      // diffusion: -Gamma_ip dN_ic/dx_j A_j
      for (int a = 0; a < 8; ++a) {
        double lc = 0.0;
        for (int j = 0; j < 3; ++j) lc += -gIp * g[24 * ip + 3 * a + j] * Ar[3 * ip + j];
        lhs[8 * il + a] += lc;
        lhs[8 * ir + a] -= lc;
        rhs[il] -= lc * pe[a];
        rhs[ir] += lc * pe[a];
      }
    }
    apply_coeff<1>(c, A, b, en, 8, rhs, lhs);
  });
  const double ui = 1.0 / urf;
  for (int i = 0; i < c.nn; ++i) A[c.rowPtr[i] + c.diagOff[i]] *= ui;
}

// ---------------------------------------------------------------------------
// Krylov: BiCGStab, right-preconditioned by (block-)Jacobi. The reference's
// solver library (liblinsolve over PETSc/Trilinos/HYPRE) is absent; this is the
// published van der Vorst algorithm.
void spmv(const Case& c, int bs, const double* A, const double* x, double* y) {
  parallel_for(c.nn, [&](long i) {
    for (int m = 0; m < bs; ++m) {
      double s = 0.0;
      for (int k = c.rowPtr[i]; k < c.rowPtr[i + 1]; ++k) {
        const int j = c.cols[k];
        for (int q = 0; q < bs; ++q) s += A[(long)bs * bs * k + bs * m + q] * x[bs * j + q];
      }
      y[bs * i + m] = s;
    }
  });
}

void invert3(const double* a, double* r) {
  const double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                     a[2] * (a[3] * a[7] - a[4] * a[6]);
  const double id = 1.0 / det;
  r[0] = (a[4] * a[8] - a[5] * a[7]) * id;
  r[1] = (a[2] * a[7] - a[1] * a[8]) * id;
  r[2] = (a[1] * a[5] - a[2] * a[4]) * id;
  r[3] = (a[5] * a[6] - a[3] * a[8]) * id;
  r[4] = (a[0] * a[8] - a[2] * a[6]) * id;
  r[5] = (a[2] * a[3] - a[0] * a[5]) * id;
  r[6] = (a[3] * a[7] - a[4] * a[6]) * id;
  r[7] = (a[1] * a[6] - a[0] * a[7]) * id;
  r[8] = (a[0] * a[4] - a[1] * a[3]) * id;
}

double dot(long n, const double* a, const double* b) { return pdot(n, a, b); }

// BiCGStab core with a right preconditioner prec(v, z): z = M^-1 v.
template <class Prec>
int bicgstab_core(const Case& c, int bs, const double* A, const double* b, double* x, double rtol, int maxit,
                  double* res, Prec prec) {
  const long n = (long)bs * c.nn;
  std::vector<double> r(n), rh(n), pv(n, 0.0), v(n, 0.0), s(n), t(n), ph(n), sh(n);
  std::fill(x, x + n, 0.0);
  for (long i = 0; i < n; ++i) r[i] = b[i];
  const double bn = std::sqrt(dot(n, b, b));
  if (bn == 0.0) {
    *res = 0.0;
    return 0;
  }
  rh = r;
  double rho = 1, alpha = 1, omega = 1;
  int it = 0;
  double rn = bn;
  for (it = 0; it < maxit; ++it) {
    if (rn <= rtol * bn) break;
    const double rho1 = dot(n, rh.data(), r.data());
    if (rho1 == 0.0) break;
    const double beta = (rho1 / rho) * (alpha / omega);
    parallel_for(n, [&](long i) { pv[i] = r[i] + beta * (pv[i] - omega * v[i]); });
    prec(pv.data(), ph.data());
    spmv(c, bs, A, ph.data(), v.data());
    alpha = rho1 / dot(n, rh.data(), v.data());
    parallel_for(n, [&](long i) { s[i] = r[i] - alpha * v[i]; });
    prec(s.data(), sh.data());
    spmv(c, bs, A, sh.data(), t.data());
    const double tt = dot(n, t.data(), t.data());
    omega = tt > 0 ? dot(n, t.data(), s.data()) / tt : 0.0;
    parallel_for(n, [&](long i) {
      x[i] += alpha * ph[i] + omega * sh[i];
      r[i] = s[i] - omega * t[i];
    });
    rho = rho1;
    rn = std::sqrt(dot(n, r.data(), r.data()));
    if (omega == 0.0) {
      ++it;
      break;
    }
  }
  *res = rn / bn;
  return it;
}

// Jacobi (bs 1) or 3x3 block-Jacobi (bs 3) preconditioned BiCGStab.
int bicgstab(const Case& c, int bs, const double* A, const double* b, double* x, double rtol, int maxit,
             double* res) {
  std::vector<double> Minv((long)bs * bs * c.nn);
  for (int i = 0; i < c.nn; ++i) {
    const double* d = &A[(long)bs * bs * (c.rowPtr[i] + c.diagOff[i])];
    if (bs == 1)
      Minv[i] = 1.0 / d[0];
    else
      invert3(d, &Minv[9L * i]);
  }
  auto prec = [&](const double* v, double* z) {
    parallel_for(c.nn, [&](long i) {
      if (bs == 1) {
        z[i] = Minv[i] * v[i];
      } else {
        for (int m = 0; m < 3; ++m)
          z[3 * i + m] = Minv[9L * i + 3 * m] * v[3 * i] + Minv[9L * i + 3 * m + 1] * v[3 * i + 1] +
                         Minv[9L * i + 3 * m + 2] * v[3 * i + 2];
      }
    });
  };
  return bicgstab_core(c, bs, A, b, x, rtol, maxit, res, prec);
}

// ---------------------------------------------------------------------------
// The reference cavity example's solver configuration
// (examples/cavity/input.i:61-77): momentum by PETSc fgmres with bjacobi
// (block Jacobi, ILU(0) on each block: PETSc's sub-solver default), pressure
// correction by Trilinos Belos GMRES with Ifpack2 ILU (one ILU(0) block per
// MPI rank). Restated from the published algorithms (Saad, Iterative Methods
// for Sparse Linear Systems, 2nd ed.: ILU(0) Alg. 10.4 in its IKJ form,
// restarted GMRES Alg. 6.9 with right preconditioning and Givens rotations):
// one block of contiguous rows per thread, as one block per rank; couplings
// to rows outside the block are dropped from the factors (block Jacobi);
// block ILU(0) on the 3x3 blocks of the momentum BSR matrix.
template <int B>
struct BlockIlu0 {
  const Case* c = nullptr;
  int nblk = 1;
  std::vector<double> lu;    // factors in the CSR layout of A (B*B per entry)
  std::vector<double> dinv;  // inverse of each row's factored diagonal block

  static void mul(const double* a, const double* b, double* out) {  // out = a b
    for (int i = 0; i < B; ++i)
      for (int j = 0; j < B; ++j) {
        double s = 0.0;
        for (int k = 0; k < B; ++k) s += a[B * i + k] * b[B * k + j];
        out[B * i + j] = s;
      }
  }
  static void inv(const double* a, double* r) {
    if (B == 1)
      r[0] = 1.0 / a[0];
    else
      invert3(a, r);
  }

  void factor(const Case& cs, const double* A, int blocks) {
    c = &cs;
    nblk = std::max(1, std::min(blocks, oracle::Pool::get().size()));
    const long nnz = cs.rowPtr[cs.nn];
    lu.assign(A, A + (long)B * B * nnz);
    dinv.assign((long)B * B * cs.nn, 0.0);
    auto body = [&](int t) {
      long r0, r1;
      oracle::chunk_range(cs.nn, nblk, t, &r0, &r1);
      std::vector<int> w(std::max<long>(r1 - r0, 1), -1);
      double tmp[B * B], upd[B * B];
      for (long i = r0; i < r1; ++i) {
        const int a = cs.rowPtr[i], e = cs.rowPtr[i + 1];
        for (int k = a; k < e; ++k)
          if (cs.cols[k] >= r0 && cs.cols[k] < r1) w[cs.cols[k] - r0] = k;
        for (int k = a; k < e; ++k) {
          const int j = cs.cols[k];
          if (j >= i) break;
          if (j < r0) continue;
          // L_ij = A_ij U_jj^-1, then A_il -= L_ij U_jl for the kept l > j
          mul(&lu[(long)B * B * k], &dinv[(long)B * B * j], tmp);
          std::copy(tmp, tmp + B * B, &lu[(long)B * B * k]);
          for (int kk = cs.rowPtr[j]; kk < cs.rowPtr[j + 1]; ++kk) {
            const int cc = cs.cols[kk];
            if (cc <= j || cc >= r1) continue;
            const int pos = w[cc - r0];
            if (pos < 0) continue;
            mul(&lu[(long)B * B * k], &lu[(long)B * B * kk], upd);
            for (int q = 0; q < B * B; ++q) lu[(long)B * B * pos + q] -= upd[q];
          }
        }
        inv(&lu[(long)B * B * (a + cs.diagOff[i])], &dinv[(long)B * B * i]);
        for (int k = a; k < e; ++k)
          if (cs.cols[k] >= r0 && cs.cols[k] < r1) w[cs.cols[k] - r0] = -1;
      }
    };
    if (nblk == 1)
      body(0);
    else
      oracle::Pool::get().run([&](int t) {
        if (t < nblk) body(t);
      });
  }

  // z = (LU)^-1 v, each block on its own
  void apply(const double* v, double* z) const {
    const Case& cs = *c;
    auto body = [&](int t) {
      long r0, r1;
      oracle::chunk_range(cs.nn, nblk, t, &r0, &r1);
      for (long i = r0; i < r1; ++i) {  // L y = v (unit lower)
        double y[B];
        for (int m = 0; m < B; ++m) y[m] = v[B * i + m];
        for (int k = cs.rowPtr[i]; k < cs.rowPtr[i + 1]; ++k) {
          const int j = cs.cols[k];
          if (j >= i) break;
          if (j < r0) continue;
          const double* L = &lu[(long)B * B * k];
          for (int m = 0; m < B; ++m)
            for (int q = 0; q < B; ++q) y[m] -= L[B * m + q] * z[B * j + q];
        }
        for (int m = 0; m < B; ++m) z[B * i + m] = y[m];
      }
      for (long i = r1 - 1; i >= r0; --i) {  // U x = y
        double y[B];
        for (int m = 0; m < B; ++m) y[m] = z[B * i + m];
        for (int k = cs.rowPtr[i] + cs.diagOff[i] + 1; k < cs.rowPtr[i + 1]; ++k) {
          const int j = cs.cols[k];
          if (j >= r1) break;
          const double* U = &lu[(long)B * B * k];
          for (int m = 0; m < B; ++m)
            for (int q = 0; q < B; ++q) y[m] -= U[B * m + q] * z[B * j + q];
        }
        const double* D = &dinv[(long)B * B * i];
        for (int m = 0; m < B; ++m) {
          double s = 0.0;
          for (int q = 0; q < B; ++q) s += D[B * m + q] * y[q];
          z[B * i + m] = s;
        }
      }
    };
    if (nblk == 1)
      body(0);
    else
      oracle::Pool::get().run([&](int t) {
        if (t < nblk) body(t);
      });
  }
};

// Restarted GMRES(m), right-preconditioned by block ILU(0); x0 = 0. Returns
// the iteration count; *res = ||b - A x|| / ||b|| at exit.
template <int B>
int gmres_ilu(const Case& c, const double* A, const double* b, double* x, double rtol, int maxit, int m,
              double* res) {
  const long n = (long)B * c.nn;
  BlockIlu0<B> M;
  M.factor(c, A, g_threads);
  std::fill(x, x + n, 0.0);
  const double bn = std::sqrt(dot(n, b, b));
  if (bn == 0.0) {
    *res = 0.0;
    return 0;
  }
  std::vector<double> V((long)(m + 1) * n), z(n), w(n), r(b, b + n);
  std::vector<double> H((long)(m + 1) * m, 0.0), cs(m), sn(m), g(m + 1);
  double beta = bn;
  int it = 0;
  while (true) {
    for (int k = 0; k <= m; ++k) g[k] = 0.0;
    g[0] = beta;
    parallel_for(n, [&](long i) { V[i] = r[i] / beta; });
    int j = 0;
    for (; j < m && it < maxit;) {
      M.apply(&V[(long)j * n], z.data());
      spmv(c, B, A, z.data(), w.data());
      for (int i = 0; i <= j; ++i) {  // modified Gram-Schmidt
        const double* vi = &V[(long)i * n];
        const double h = dot(n, w.data(), vi);
        H[(long)i * m + j] = h;
        parallel_for(n, [&](long q) { w[q] -= h * vi[q]; });
      }
      const double hn = std::sqrt(dot(n, w.data(), w.data()));
      if (hn > 0.0) {
        double* vj = &V[(long)(j + 1) * n];
        parallel_for(n, [&](long q) { vj[q] = w[q] / hn; });
      }
      for (int i = 0; i < j; ++i) {  // earlier rotations on the new column
        const double a = H[(long)i * m + j], bb = H[(long)(i + 1) * m + j];
        H[(long)i * m + j] = cs[i] * a + sn[i] * bb;
        H[(long)(i + 1) * m + j] = -sn[i] * a + cs[i] * bb;
      }
      const double a = H[(long)j * m + j];
      const double d = std::sqrt(a * a + hn * hn);
      cs[j] = d > 0.0 ? a / d : 1.0;
      sn[j] = d > 0.0 ? hn / d : 0.0;
      H[(long)j * m + j] = d;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      ++it;
      ++j;
      if (std::fabs(g[j]) <= rtol * bn || hn == 0.0) break;
    }
    // y = H^-1 g (upper triangular j x j); x += M^-1 (V y)
    std::vector<double> y(j, 0.0);
    for (int i = j - 1; i >= 0; --i) {
      double s = g[i];
      for (int k = i + 1; k < j; ++k) s -= H[(long)i * m + k] * y[k];
      y[i] = s / H[(long)i * m + i];
    }
    parallel_for(n, [&](long q) {
      double s = 0.0;
      for (int k = 0; k < j; ++k) s += y[k] * V[(long)k * n + q];
      w[q] = s;
    });
    M.apply(w.data(), z.data());
    parallel_for(n, [&](long q) { x[q] += z[q]; });
    spmv(c, B, A, x, w.data());
    parallel_for(n, [&](long q) { r[q] = b[q] - w[q]; });
    beta = std::sqrt(dot(n, r.data(), r.data()));
    if (beta <= rtol * bn || it >= maxit || !(beta < INFINITY)) break;
  }
  *res = beta / bn;
  return it;
}

// BiCGStab right-preconditioned by block-Jacobi ILU(0) (one block per thread).
template <int B>
int bicgstab_ilu(const Case& c, const double* A, const double* b, double* x, double rtol, int maxit, double* res) {
  BlockIlu0<B> M;
  M.factor(c, A, g_threads);
  return bicgstab_core(c, B, A, b, x, rtol, maxit, res, [&](const double* v, double* z) { M.apply(v, z); });
}

// ---------------------------------------------------------------------------
// One SIMPLE outer iteration: segregatedFlowEquations::solve
// (src/equation/flow/segregatedFlowEquations.cpp:76-297) with
// navierStokesEquation::solve (navierStokesEquation.cpp:157-222) and
// pressureCorrectionEquation::solve (pressureCorrectionEquation.cpp:89-150),
// one pressure sub-iteration, no compressibility, no frame motion.
void simple_iteration(Case& c, orc_iter_stats* st) {
  const int nnz = c.rowPtr[c.nn];
  c.Am.resize(9L * nnz);
  c.bm.resize(3L * c.nn);
  c.xm.resize(3L * c.nn);
  c.Ap.resize(nnz);
  c.bp.resize(c.nn);
  c.xp.resize(c.nn);
  // momentum predictor
  assemble_momentum(c, c.Am.data(), c.bm.data());
  double res = 0.0;
  const int mi =
      c.solverKind == 1   ? gmres_ilu<3>(c, c.Am.data(), c.bm.data(), c.xm.data(), c.s.mom_rtol, c.s.mom_maxit, 30, &res)
      : c.solverKind == 2 ? bicgstab_ilu<3>(c, c.Am.data(), c.bm.data(), c.xm.data(), c.s.mom_rtol, c.s.mom_maxit, &res)
                          : bicgstab(c, 3, c.Am.data(), c.bm.data(), c.xm.data(), c.s.mom_rtol, c.s.mom_maxit, &res);
  for (long i = 0; i < 3L * c.nn; ++i) c.U[i] += c.xm[i];
  update_mdot(c);
  if (st) {
    st->mom_iters[0] = mi;
    st->mom_res = res;
  }
  // pressure correction
  assemble_pcorr(c, c.Ap.data(), c.bp.data());
  if (st) {
    double s2 = 0.0;
    for (int i = 0; i < c.nn; ++i) s2 += c.bp[i] * c.bp[i];
    st->continuity_raw = std::sqrt(s2 / c.nn);
    st->continuity_rms = st->continuity_raw / c.massScale;
  }
  const int pi =
      c.solverKind == 1   ? gmres_ilu<1>(c, c.Ap.data(), c.bp.data(), c.xp.data(), c.s.pc_rtol, c.s.pc_maxit, 50, &res)
      : c.solverKind == 2 ? bicgstab_ilu<1>(c, c.Ap.data(), c.bp.data(), c.xp.data(), c.s.pc_rtol, c.s.pc_maxit, &res)
                          : bicgstab(c, 1, c.Ap.data(), c.bp.data(), c.xp.data(), c.s.pc_rtol, c.s.pc_maxit, &res);
  for (int i = 0; i < c.nn; ++i) c.p[i] += c.s.urf_p * c.xp[i];
  if (st) {
    st->pc_iters = pi;
    st->pc_res = res;
  }
  update_mdot(c);
  update_div(c);
  // velocity correction with D, or D~ with SIMPLEC (segregatedFlowEquations.cpp:134-278)
  const double iu = 1.0 / c.s.urf_p;
  const std::vector<double>& dc = c.s.du_mode == 1 ? c.duT : c.du;
  for (long i = 0; i < 3L * c.nn; ++i) c.U[i] += iu * dc[i] * c.gradP[i];
  update_gradient<1>(c, c.p, c.gradP, c.s.p_shifted);
  for (long i = 0; i < 3L * c.nn; ++i) c.U[i] -= iu * dc[i] * c.gradP[i];
  update_gradient<3>(c, c.U, c.gradU, c.s.u_shifted);
  if (c.s.hr) update_blending_u(c);  // segregatedFlowEquations.cpp:287-288
}

}  // namespace

extern "C" {

void orc_set_threads(int n) {
  g_threads = n < 1 ? 1 : n;
  oracle::Pool::get().resize(g_threads);
}
int orc_get_threads(void) { return g_threads; }

void orc_hex8_scs_areav(const double* x, double* areav) { oracle::hex8::scs_areav(x, areav); }
int orc_hex8_scv_volumes(const double* x, double* vol) {
  return oracle::hex8::scv_volumes(x, vol) ? 0 : 1;
}
int orc_hex8_grad_op(const double* x, double* gradop, int shifted) {
  return oracle::hex8::grad_op(x, gradop, shifted != 0);
}
void orc_hex8_shape(double* shape, int shifted) { oracle::hex8::scs_shape(shape, shifted != 0); }

void* orc_case_create(int nn, int ne, const double* x, const int* conn, int nf, const int* face_elem,
                      const int* face_ord, const int* face_bnd, int nbnd, const double* bnd_velocity,
                      const orc_settings* s) {
  Case* c = new Case();
  c->s = *s;
  c->nn = nn;
  c->ne = ne;
  c->nf = nf;
  c->nbnd = nbnd;
  c->x.assign(x, x + 3L * nn);
  c->conn.assign(conn, conn + 8L * ne);
  c->fElem.assign(face_elem, face_elem + nf);
  c->fOrd.assign(face_ord, face_ord + nf);
  c->fBnd.assign(face_bnd, face_bnd + nf);
  c->bndU.assign(bnd_velocity, bnd_velocity + 3L * nbnd);
  build_graph(*c);
  build_colors(*c);
  dual_volume(*c);
  exposed_areas(*c);
  c->U.assign(3L * nn, 0.0);
  c->p.assign(nn, 0.0);
  c->gradU.assign(9L * nn, 0.0);
  c->gradP.assign(3L * nn, 0.0);
  c->du.assign(3L * nn, 0.0);
  c->div.assign(nn, 0.0);
  c->mDot.assign(12L * ne, 0.0);
  c->rho.assign(nn, s->rho);
  c->mu.assign(nn, s->mu);
  c->sideU.assign(3L * nn, 0.0);
  c->wallNode.assign(nn, 0.0);
  c->duT.assign(3L * nn, 0.0);
  c->betaU.assign(3L * nn, 0.0);  // setupBlendingFactorField: zero (nodeField.hpp:733-745)
  c->minU.assign(3L * nn, 0.0);
  c->maxU.assign(3L * nn, 0.0);
  if (s->ref_node >= 0) c->refNodes.push_back(s->ref_node);
  {
    // mean element edge length over every element's 12 edges (element order)
    // and the largest wall speed
    double sum = 0.0;
    for (int e = 0; e < ne; ++e)
      for (int ip = 0; ip < 12; ++ip) {
        const double* a = &c->x[3L * c->conn[8L * e + oracle::hex8::LR[ip][0]]];
        const double* b = &c->x[3L * c->conn[8L * e + oracle::hex8::LR[ip][1]]];
        sum += std::sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
      }
    const double h = sum / (12.0 * ne);
    double u = 0.0;
    for (int k = 0; k < nbnd; ++k)
      u = std::max(u, std::sqrt(bnd_velocity[3 * k] * bnd_velocity[3 * k] + bnd_velocity[3 * k + 1] * bnd_velocity[3 * k + 1] +
                                bnd_velocity[3 * k + 2] * bnd_velocity[3 * k + 2]));
    c->massScale = s->rho * (u > 0.0 ? u : 1.0) * h * h;
  }
  // node side velocity: boundaries applied in order, later ones overwrite shared
  // nodes (nodeField::updateBoundarySideFieldSpecifiedValue, setToValue per part)
  for (int bnd = 0; bnd < nbnd; ++bnd)
    for (int f = 0; f < nf; ++f) {
      if (c->fBnd[f] != bnd) continue;
      for (int k = 0; k < 4; ++k) {
        const int nd = c->conn[8 * c->fElem[f] + oracle::hex8::FACE_NODES[c->fOrd[f]][k]];
        for (int d = 0; d < 3; ++d) c->sideU[3 * nd + d] = c->bndU[3 * bnd + d];
        c->wallNode[nd] = 1.0;
      }
    }
  return c;
}

int orc_set_boundary_types(void* h, const int* types, int nbnd, int correct_gradients) {
  Case& c = *static_cast<Case*>(h);
  c.correctGrad = correct_gradients != 0;
  if (nbnd != c.nbnd) return 1;
  for (int k = 0; k < nbnd; ++k)
    if (types[k] != ORC_BTYPE_WALL && types[k] != ORC_BTYPE_SYMMETRY) return 1;
  c.bndType.assign(types, types + nbnd);
  c.symArea.assign(3L * c.nn, 0.0);
  c.wallFaceNode.assign(c.nn, 0);
  std::vector<char> sym(c.nn, 0);
  for (int f = 0; f < c.nf; ++f) {
    const int* en = &c.conn[8 * c.fElem[f]];
    const bool s = is_symmetry_face(c, f);
    for (int ip = 0; ip < 4; ++ip) {
      const int nd = en[oracle::hex8::FACE_NODES[c.fOrd[f]][ip]];
      if (s) {
        sym[nd] = 1;
        for (int d = 0; d < 3; ++d) c.symArea[3L * nd + d] += c.faceArea[12 * f + 3 * ip + d];
      } else {
        c.wallFaceNode[nd] = 1;
      }
    }
  }
  c.symNodes.clear();
  for (int i = 0; i < c.nn; ++i)
    if (sym[i]) c.symNodes.push_back(i);
  // side velocity from the wall boundaries alone (nodeField::updateBoundarySideField
  // leaves symmetry parts untouched, nodeField.hpp:1128)
  std::fill(c.sideU.begin(), c.sideU.end(), 0.0);
  for (int bnd = 0; bnd < c.nbnd; ++bnd) {
    if (c.bndType[bnd] == ORC_BTYPE_SYMMETRY) continue;
    for (int f = 0; f < c.nf; ++f) {
      if (c.fBnd[f] != bnd) continue;
      for (int k = 0; k < 4; ++k) {
        const int nd = c.conn[8 * c.fElem[f] + oracle::hex8::FACE_NODES[c.fOrd[f]][k]];
        for (int d = 0; d < 3; ++d) c.sideU[3 * nd + d] = c.bndU[3 * bnd + d];
      }
    }
  }
  return 0;
}

void orc_case_destroy(void* h) { delete static_cast<Case*>(h); }

double orc_case_mass_scale(void* h) { return static_cast<Case*>(h)->massScale; }

void orc_set_ref_nodes(void* h, const int* nodes, int n) {
  Case* c = static_cast<Case*>(h);
  c->refNodes.assign(nodes, nodes + n);
}

double* orc_case_field(void* h, const char* name, long* len) {
  Case* c = static_cast<Case*>(h);
  std::vector<double>* v = nullptr;
  const std::string n(name);
  if (n == "U") v = &c->U;
  else if (n == "p") v = &c->p;
  else if (n == "gradU") v = &c->gradU;
  else if (n == "gradP") v = &c->gradP;
  else if (n == "du") v = &c->du;
  else if (n == "div") v = &c->div;
  else if (n == "mDot") v = &c->mDot;
  else if (n == "rho") v = &c->rho;
  else if (n == "mu") v = &c->mu;
  else if (n == "vol") v = &c->vol;
  else if (n == "faceArea") v = &c->faceArea;
  else if (n == "sideU") v = &c->sideU;
  else if (n == "wallNode") v = &c->wallNode;
  else if (n == "symArea") v = &c->symArea;
  else if (n == "x") v = &c->x;
  else if (n == "betaU") v = &c->betaU;
  else if (n == "duTilde") v = &c->duT;
  else if (n == "minU") v = &c->minU;
  else if (n == "maxU") v = &c->maxU;
  if (!v) {
    *len = 0;
    return nullptr;
  }
  *len = (long)v->size();
  return v->data();
}

int orc_case_nnz(void* h) {
  Case* c = static_cast<Case*>(h);
  return c->rowPtr[c->nn];
}

void orc_case_graph(void* h, int* row_ptr, int* cols) {
  Case* c = static_cast<Case*>(h);
  std::copy(c->rowPtr.begin(), c->rowPtr.end(), row_ptr);
  std::copy(c->cols.begin(), c->cols.end(), cols);
}

// navierStokesEquation::initialize/postInitialize and
// pressureCorrectionEquation::initialize (velocity gradient, pressure gradient,
// mass flow rate, divergence).
void orc_initialize(void* h) {
  Case* c = static_cast<Case*>(h);
  update_gradient<3>(*c, c->U, c->gradU, c->s.u_shifted);
  if (c->s.hr) update_blending_u(*c);  // navierStokesEquation::initialize
  init_mdot(*c);
  update_div(*c);
  update_gradient<1>(*c, c->p, c->gradP, c->s.p_shifted);
}

void orc_assemble_momentum(void* h, double* A, double* b) {
  assemble_momentum(*static_cast<Case*>(h), A, b);
}
void orc_assemble_pcorr(void* h, double* A, double* b) {
  assemble_pcorr(*static_cast<Case*>(h), A, b);
}
void orc_assemble_scalar_transport(void* h, const double* phi, const double* gam, const double* sdiag,
                                   const double* srhs, double urf, double* A, double* b) {
  assemble_scalar_transport(*static_cast<Case*>(h), phi, gam, sdiag, srhs, urf, A, b);
}
void orc_update_mdot(void* h) { update_mdot(*static_cast<Case*>(h)); }
void orc_update_div(void* h) { update_div(*static_cast<Case*>(h)); }
void orc_update_grad_p(void* h) {
  Case* c = static_cast<Case*>(h);
  update_gradient<1>(*c, c->p, c->gradP, c->s.p_shifted);
}
void orc_update_blending_u(void* h) { update_blending_u(*static_cast<Case*>(h)); }

void orc_update_grad_u(void* h) {
  Case* c = static_cast<Case*>(h);
  update_gradient<3>(*c, c->U, c->gradU, c->s.u_shifted);
}
int orc_bicgstab(void* h, int bs, const double* A, const double* b, double* x, double rtol, int maxit,
                 double* res) {
  return bicgstab(*static_cast<Case*>(h), bs, A, b, x, rtol, maxit, res);
}
void orc_simple_iteration(void* h, orc_iter_stats* st) { simple_iteration(*static_cast<Case*>(h), st); }

void orc_apply_coeff(void* h, int bs, double* A, double* b, const int* nodes, int n, const double* rhs,
                     const double* lhs) {
  Case& c = *static_cast<Case*>(h);
  if (n < 1 || n > 8) return;  // hex8 / tet4 elements
  if (bs == 3)
    apply_coeff<3>(c, A, b, nodes, n, rhs, lhs);
  else
    apply_coeff<1>(c, A, b, nodes, n, rhs, lhs);
}

void orc_advance_time(void* h, int scheme, double dt) {
  Case& c = *static_cast<Case*>(h);
  if (c.Uold.empty()) {
    c.Uold.assign(3L * c.nn, 0.0);
    c.Uoldold.assign(3L * c.nn, 0.0);
  }
  c.Uoldold = c.Uold;
  c.Uold = c.U;
  c.dtPrev = c.timeSteps ? c.dtStep : dt;
  c.dtStep = dt;
  c.timeScheme = scheme == 2 ? 2 : 1;
  ++c.timeSteps;
}

void orc_set_solver(void* h, int kind) { static_cast<Case*>(h)->solverKind = (kind == 1 || kind == 2) ? kind : 0; }

int orc_gmres_ilu(void* h, int bs, const double* A, const double* b, double* x, double rtol, int maxit, int restart,
                  double* res) {
  const Case& c = *static_cast<Case*>(h);
  return bs == 3 ? gmres_ilu<3>(c, A, b, x, rtol, maxit, restart, res)
                 : gmres_ilu<1>(c, A, b, x, rtol, maxit, restart, res);
}

}  // extern "C"
