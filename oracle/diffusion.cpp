// Oracle (test infrastructure only): CPU FP64 restatement of OpenAccel's tet4
// scalar-diffusion path (a solid-domain energy equation: pure diffusion with a
// volumetric source, fixed-value and zero-flux walls) and of a Krylov solve of
// the assembled system. Only tests, the smoke check and the bench CPU-baseline
// leg use it.
//
// Reference routines restated (paths relative to the reference project root):
//   - element terms        src/assemble/phiAssembler/phiAssemblerElemTerms.hpp:11-413
//                          (diffusion only: solid domain, :14-15)
//   - fixed-value walls    src/assemble/phiAssembler/phiAssemblerElemBoundaryConditions.hpp:112-410
//   - node terms           src/assemble/heatTransfer/thermalEnergy/thermalEnergyAssemblerNodeTerms.cpp:25-97
//                          (solid: rhs += source * dual volume)
//   - post-assembly        src/assemble/phiAssembler/phiAssembler.h:748-753,967-1006
//                          (diagonal / urf) and thermalEnergyAssembler.h:39-43 +
//                          phiAssembler.h:1008-1152 (rhs *= 0.75 on wall nodes)
//   - scatter              src/assemble/assembler.h:311-453 (applyCoeff_)
//   - field correction     src/equation/heatTransfer/thermalEnergy/thermalEnergyEquation.cpp:190-247,
//                          src/equation/equation.h:204-286 (phi += x, clipped below at 0)
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "oracle.h"
#include "tet4_master.hpp"

namespace {

using oracle::tet4::LR;
using oracle::tet4::NSCS;
using oracle::tet4::SIDE_NODES;

template <class F>
void pfor(long n, F f) {
  const int nt = orc_get_threads();
  if (nt <= 1 || n < 4096) {
    for (long i = 0; i < n; ++i) f(i);
    return;
  }
  std::vector<std::thread> th;
  const long chunk = (n + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    const long a = t * chunk, b = std::min(n, a + chunk);
    if (a >= b) break;
    th.emplace_back([=, &f] {
      for (long i = a; i < b; ++i) f(i);
    });
  }
  for (auto& x : th) x.join();
}

double pdot(long n, const double* a, const double* b) {
  const int nt = orc_get_threads();
  if (nt <= 1 || n < 65536) {
    double s = 0.0;
    for (long i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
  }
  std::vector<double> part(nt, 0.0);
  std::vector<std::thread> th;
  const long chunk = (n + nt - 1) / nt;
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&, t] {
      const long lo = t * chunk, hi = std::min(n, lo + chunk);
      double s = 0.0;
      for (long i = lo; i < hi; ++i) s += a[i] * b[i];
      part[t] = s;
    });
  for (auto& x : th) x.join();
  double s = 0.0;
  for (double v : part) s += v;
  return s;
}

struct DiffCase {
  orc_diff_settings s;
  int nn, ne, nf, nbnd;
  std::vector<double> x;
  std::vector<int> conn;  // [ne][4]
  std::vector<int> fElem, fOrd, fBnd;
  std::vector<int> bndKind;       // ORC_BND_FIXED_VALUE / ORC_BND_ZERO_FLUX
  std::vector<double> bndValue;   // fixed value per boundary
  std::vector<double> vol, faceArea;  // vol[nn], faceArea[nf][3][3]
  std::vector<int> rowPtr, cols, diagOff;
  std::vector<double> phi, gamma, src, sidePhi, wallNode;
  std::vector<std::vector<int>> colors;
};

// nodeGraph::buildGraph_ (src/mesh/graph/nodeGraph.cpp:29-98): the tet4 edge
// stencil, which is every node pair of an element.
void build_graph(DiffCase& c) {
  std::vector<std::set<int>> st(c.nn);
  for (int e = 0; e < c.ne; ++e) {
    const int* en = &c.conn[4 * e];
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) st[en[a]].insert(en[b]);
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

void build_colors(DiffCase& c) {
  std::vector<uint64_t> used(c.nn, 0u);
  std::vector<int> col(c.ne);
  int nc = 0;
  for (int e = 0; e < c.ne; ++e) {
    uint64_t m = 0;
    for (int a = 0; a < 4; ++a) m |= used[c.conn[4 * e + a]];
    int k = 0;
    while (k < 64 && (m >> k) & 1u) ++k;
    col[e] = k;
    nc = std::max(nc, k + 1);
    for (int a = 0; a < 4; ++a) used[c.conn[4 * e + a]] |= (uint64_t(1) << k);
  }
  c.colors.assign(nc, {});
  for (int e = 0; e < c.ne; ++e) c.colors[col[e]].push_back(e);
}

template <class F>
void for_elements(const DiffCase& c, F f) {
  if (orc_get_threads() <= 1) {
    for (int e = 0; e < c.ne; ++e) f(e);
    return;
  }
  for (const auto& cl : c.colors) pfor((long)cl.size(), [&](long i) { f(cl[i]); });
}

// applyCoeff_ for a scalar equation (src/assemble/assembler.h:311-453).
void apply_coeff(DiffCase& c, double* A, double* b, const int* nodes, int n, const double* rhs,
                 const double* lhs) {
  int perm[4];
  std::iota(perm, perm + n, 0);
  std::sort(perm, perm + n, [&](int a, int bb) { return nodes[a] < nodes[bb]; });
  for (int r = 0; r < n; ++r) {
    const int pr = perm[r];
    const int row = nodes[pr];
    const int beg = c.rowPtr[row], len = c.rowPtr[row + 1] - beg;
    int off = 0, offOld = 0;
    for (int j = 0; j < n; ++j) {
      const int pj = perm[j];
      const int col = nodes[pj];
      while (off < len && c.cols[beg + off] != col) ++off;
      if (off < len) {
        A[beg + off] += lhs[n * pr + pj];
        offOld = off;
      } else {
        A[beg + c.diagOff[row]] += lhs[n * pr + pj];
        off = offOld;
      }
    }
    b[row] += rhs[pr];
  }
}

void gather_coords(const DiffCase& c, int e, double* xe) {
  for (int a = 0; a < 4; ++a)
    for (int k = 0; k < 3; ++k) xe[3 * a + k] = c.x[3 * c.conn[4 * e + a] + k];
}

// mesh::updateDualNodalVolumeField_ (src/mesh/meshGeometry.cpp:1277-1345).
void dual_volume(DiffCase& c) {
  c.vol.assign(c.nn, 0.0);
  for (int e = 0; e < c.ne; ++e) {
    double xe[12], v[4];
    gather_coords(c, e, xe);
    oracle::tet4::scv_volumes(xe, v);
    for (int a = 0; a < 4; ++a) c.vol[c.conn[4 * e + a]] += v[a];
  }
}

// mesh::updateExposedAreaVectorField_ (src/mesh/meshGeometry.cpp:1441-1527)
// with the tri3 face element; face nodes in side order.
void exposed_areas(DiffCase& c) {
  c.faceArea.assign(9L * c.nf, 0.0);
  for (int f = 0; f < c.nf; ++f) {
    double p[9];
    const int e = c.fElem[f], o = c.fOrd[f];
    for (int k = 0; k < 3; ++k)
      for (int d = 0; d < 3; ++d) p[3 * k + d] = c.x[3 * c.conn[4 * e + SIDE_NODES[o][k]] + d];
    oracle::tet4::tri_face_areav(p, &c.faceArea[9L * f]);
  }
}

void assemble(DiffCase& c, double* A, double* b) {
  const int nnz = c.rowPtr[c.nn];
  std::fill(A, A + nnz, 0.0);
  std::fill(b, b + c.nn, 0.0);
  const bool sh = c.s.shifted != 0;
  double N[NSCS * 4], Nf[9];
  oracle::tet4::scs_shape(N, sh);
  oracle::tet4::face_shape(Nf, sh);

  // node terms (solid energy source): rhs += S * V, lhs 0 on the diagonal
  for (int i = 0; i < c.nn; ++i) {
    const double lhs0 = 0.0, rhs0 = 0.0 + c.src[i] * c.vol[i];
    apply_coeff(c, A, b, &i, 1, &rhs0, &lhs0);
  }

  // interior element terms (diffusion)
  for_elements(c, [&](int e) {
    const int* en = &c.conn[4 * e];
    double xe[12], areav[18], g[12], ph[4], gm[4], lhs[16] = {0}, rhs[4] = {0};
    gather_coords(c, e, xe);
    for (int a = 0; a < 4; ++a) {
      ph[a] = c.phi[en[a]];
      gm[a] = c.gamma[en[a]];
    }
    oracle::tet4::scs_areav(xe, areav);
    oracle::tet4::grad_op(xe, g);
    for (int ip = 0; ip < NSCS; ++ip) {
      const int il = LR[ip][0], ir = LR[ip][1];
      double G = 0.0;
      for (int ic = 0; ic < 4; ++ic) G += N[4 * ip + ic] * gm[ic];
      for (int ic = 0; ic < 4; ++ic) {
        double l = 0.0;
        for (int j = 0; j < 3; ++j) l += -G * g[3 * ic + j] * areav[3 * ip + j];
        lhs[4 * il + ic] += l;
        lhs[4 * ir + ic] -= l;
        rhs[il] -= l * ph[ic];
        rhs[ir] += l * ph[ic];
      }
    }
    apply_coeff(c, A, b, en, 4, rhs, lhs);
  });

  // fixed-value walls, boundary by boundary in face order
  for (int f = 0; f < c.nf; ++f) {
    if (c.bndKind[c.fBnd[f]] != ORC_BND_FIXED_VALUE) continue;
    const int e = c.fElem[f], o = c.fOrd[f];
    const int* en = &c.conn[4 * e];
    double xe[12], g[12], ph[4], bcm[4], gf[3], lhs[16] = {0}, rhs[4] = {0};
    gather_coords(c, e, xe);
    for (int a = 0; a < 4; ++a) {
      ph[a] = c.phi[en[a]];
      bcm[a] = 1.0;
    }
    for (int k = 0; k < 3; ++k) {
      const int ic = SIDE_NODES[o][k];
      gf[k] = c.gamma[en[ic]];
      bcm[ic] = 0.0;
      ph[ic] = c.sidePhi[en[ic]];
    }
    oracle::tet4::grad_op(xe, g);
    const double* av = &c.faceArea[9L * f];
    for (int ip = 0; ip < 3; ++ip) {
      const int nearest = SIDE_NODES[o][ip];
      double G = 0.0;
      for (int k = 0; k < 3; ++k) G += Nf[3 * ip + k] * gf[k];
      for (int ic = 0; ic < 4; ++ic)
        for (int j = 0; j < 3; ++j) {
          const double lf = -G * g[3 * ic + j] * av[3 * ip + j];
          lhs[4 * nearest + ic] += lf * bcm[ic];
          rhs[nearest] -= lf * ph[ic];
        }
    }
    apply_coeff(c, A, b, en, 4, rhs, lhs);
  }

  // relaxation of the diagonal, then of the wall-node rhs
  const double urf_inv = 1.0 / c.s.urf;
  for (int i = 0; i < c.nn; ++i) A[c.rowPtr[i] + c.diagOff[i]] *= urf_inv;
  for (int i = 0; i < c.nn; ++i)
    if (c.wallNode[i] != 0.0) b[i] *= c.s.wall_rhs_relax;
}

void spmv(const DiffCase& c, const double* A, const double* x, double* y) {
  pfor(c.nn, [&](long i) {
    double s = 0.0;
    for (int k = c.rowPtr[i]; k < c.rowPtr[i + 1]; ++k) s += A[k] * x[c.cols[k]];
    y[i] = s;
  });
}

// Jacobi-preconditioned conjugate gradients (Hestenes-Stiefel), x0 = 0,
// stopping at ||r|| <= rtol ||b||. The reference's solver library is absent;
// this is the published algorithm.
int cg(const DiffCase& c, const double* A, const double* b, double* x, double rtol, int maxit,
       double* res) {
  const long n = c.nn;
  std::vector<double> dinv(n), r(n), z(n), p(n), q(n);
  for (long i = 0; i < n; ++i) dinv[i] = 1.0 / A[c.rowPtr[i] + c.diagOff[i]];
  std::fill(x, x + n, 0.0);
  for (long i = 0; i < n; ++i) r[i] = b[i];
  const double bn = std::sqrt(pdot(n, b, b));
  if (bn == 0.0) {
    *res = 0.0;
    return 0;
  }
  pfor(n, [&](long i) { z[i] = dinv[i] * r[i]; });
  p = z;
  double rz = pdot(n, r.data(), z.data());
  double rn = bn;
  int it = 0;
  for (it = 0; it < maxit; ++it) {
    if (rn <= rtol * bn) break;
    spmv(c, A, p.data(), q.data());
    const double alpha = rz / pdot(n, p.data(), q.data());
    pfor(n, [&](long i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
      z[i] = dinv[i] * r[i];
    });
    const double rz1 = pdot(n, r.data(), z.data());
    const double beta = rz1 / rz;
    rz = rz1;
    pfor(n, [&](long i) { p[i] = z[i] + beta * p[i]; });
    rn = std::sqrt(pdot(n, r.data(), r.data()));
  }
  *res = rn / bn;
  return it;
}

// Jacobi right-preconditioned BiCGStab (van der Vorst), x0 = 0, stopping at
// ||r|| <= rtol ||b||: the assembled operator is not symmetric (Gamma varies
// between the SCS ips of an element and the fixed-value rows carry the
// boundary flux only), so CG does not apply to it.
int bicgstab(const DiffCase& c, const double* A, const double* b, double* x, double rtol, int maxit,
             double* res) {
  const long n = c.nn;
  std::vector<double> dinv(n), r(n), rh(n), pv(n, 0.0), v(n, 0.0), s(n), t(n), ph(n), sh(n);
  for (long i = 0; i < n; ++i) dinv[i] = 1.0 / A[c.rowPtr[i] + c.diagOff[i]];
  std::fill(x, x + n, 0.0);
  for (long i = 0; i < n; ++i) r[i] = b[i];
  const double bn = std::sqrt(pdot(n, b, b));
  if (bn == 0.0) {
    *res = 0.0;
    return 0;
  }
  rh = r;
  double rho = 1, alpha = 1, omega = 1, rn = bn;
  int it = 0;
  for (it = 0; it < maxit; ++it) {
    if (rn <= rtol * bn) break;
    const double rho1 = pdot(n, rh.data(), r.data());
    if (rho1 == 0.0) break;
    const double beta = (rho1 / rho) * (alpha / omega);
    pfor(n, [&](long i) {
      pv[i] = r[i] + beta * (pv[i] - omega * v[i]);
      ph[i] = dinv[i] * pv[i];
    });
    spmv(c, A, ph.data(), v.data());
    alpha = rho1 / pdot(n, rh.data(), v.data());
    pfor(n, [&](long i) {
      s[i] = r[i] - alpha * v[i];
      sh[i] = dinv[i] * s[i];
    });
    spmv(c, A, sh.data(), t.data());
    const double tt = pdot(n, t.data(), t.data());
    omega = tt > 0 ? pdot(n, t.data(), s.data()) / tt : 0.0;
    pfor(n, [&](long i) {
      x[i] += alpha * ph[i] + omega * sh[i];
      r[i] = s[i] - omega * t[i];
    });
    rho = rho1;
    rn = std::sqrt(pdot(n, r.data(), r.data()));
    if (omega == 0.0) {
      ++it;
      break;
    }
  }
  *res = rn / bn;
  return it;
}

}  // namespace

extern "C" {

void orc_tet4_scs_areav(const double* x, double* areav) { oracle::tet4::scs_areav(x, areav); }
int orc_tet4_scv_volumes(const double* x, double* vol) {
  return oracle::tet4::scv_volumes(x, vol) ? 0 : 1;
}
int orc_tet4_grad_op(const double* x, double* gradop) { return oracle::tet4::grad_op(x, gradop); }
void orc_tet4_shape(double* shape, int shifted) { oracle::tet4::scs_shape(shape, shifted != 0); }
void orc_tri3_face_areav(const double* p, double* areav) { oracle::tet4::tri_face_areav(p, areav); }

void* orc_diff_create(int nn, int ne, const double* x, const int* conn, int nf, const int* face_elem,
                      const int* face_ord, const int* face_bnd, int nbnd, const int* bnd_kind,
                      const double* bnd_value, const orc_diff_settings* s) {
  DiffCase* c = new DiffCase();
  c->s = *s;
  c->nn = nn;
  c->ne = ne;
  c->nf = nf;
  c->nbnd = nbnd;
  c->x.assign(x, x + 3L * nn);
  c->conn.assign(conn, conn + 4L * ne);
  c->fElem.assign(face_elem, face_elem + nf);
  c->fOrd.assign(face_ord, face_ord + nf);
  c->fBnd.assign(face_bnd, face_bnd + nf);
  c->bndKind.assign(bnd_kind, bnd_kind + nbnd);
  c->bndValue.assign(bnd_value, bnd_value + nbnd);
  build_graph(*c);
  build_colors(*c);
  dual_volume(*c);
  exposed_areas(*c);
  c->phi.assign(nn, 0.0);
  c->gamma.assign(nn, 1.0);
  c->src.assign(nn, 0.0);
  c->sidePhi.assign(nn, 0.0);
  c->wallNode.assign(nn, 0.0);
  // side values of the fixed-value boundaries, applied in boundary order; every
  // boundary node of a solid domain is a wall node for the rhs relaxation
  for (int bnd = 0; bnd < nbnd; ++bnd)
    for (int f = 0; f < nf; ++f) {
      if (c->fBnd[f] != bnd) continue;
      for (int k = 0; k < 3; ++k) {
        const int nd = c->conn[4 * c->fElem[f] + SIDE_NODES[c->fOrd[f]][k]];
        if (c->bndKind[bnd] == ORC_BND_FIXED_VALUE) c->sidePhi[nd] = c->bndValue[bnd];
        c->wallNode[nd] = 1.0;
      }
    }
  return c;
}

void orc_diff_destroy(void* h) { delete static_cast<DiffCase*>(h); }

double* orc_diff_field(void* h, const char* name, long* len) {
  DiffCase* c = static_cast<DiffCase*>(h);
  std::vector<double>* v = nullptr;
  const std::string n(name);
  if (n == "phi") v = &c->phi;
  else if (n == "gamma") v = &c->gamma;
  else if (n == "src") v = &c->src;
  else if (n == "sidePhi") v = &c->sidePhi;
  else if (n == "vol") v = &c->vol;
  else if (n == "wallNode") v = &c->wallNode;
  else if (n == "faceArea") v = &c->faceArea;
  else if (n == "x") v = &c->x;
  if (!v) {
    *len = 0;
    return nullptr;
  }
  *len = (long)v->size();
  return v->data();
}

int orc_diff_nnz(void* h) {
  DiffCase* c = static_cast<DiffCase*>(h);
  return c->rowPtr[c->nn];
}

void orc_diff_graph(void* h, int* row_ptr, int* cols) {
  DiffCase* c = static_cast<DiffCase*>(h);
  std::copy(c->rowPtr.begin(), c->rowPtr.end(), row_ptr);
  std::copy(c->cols.begin(), c->cols.end(), cols);
}

void orc_diff_assemble(void* h, double* A, double* b) { assemble(*static_cast<DiffCase*>(h), A, b); }

int orc_diff_cg(void* h, const double* A, const double* b, double* x, double rtol, int maxit, double* res) {
  return cg(*static_cast<DiffCase*>(h), A, b, x, rtol, maxit, res);
}

int orc_diff_bicgstab(void* h, const double* A, const double* b, double* x, double rtol, int maxit,
                      double* res) {
  return bicgstab(*static_cast<DiffCase*>(h), A, b, x, rtol, maxit, res);
}

void orc_diff_spmv(void* h, const double* A, const double* x, double* y) {
  spmv(*static_cast<DiffCase*>(h), A, x, y);
}

// thermalEnergyEquation::solve (thermalEnergyEquation.cpp:190-247): assemble,
// solve (BiCGStab), phi += x with the lower clip at 0 (equation.h:204-286).
int orc_diff_step(void* h, double* res) {
  DiffCase* c = static_cast<DiffCase*>(h);
  const int nnz = c->rowPtr[c->nn];
  std::vector<double> A(nnz), b(c->nn), x(c->nn);
  assemble(*c, A.data(), b.data());
  const int it = bicgstab(*c, A.data(), b.data(), x.data(), c->s.rtol, c->s.maxit, res);
  for (int i = 0; i < c->nn; ++i) {
    double v = c->phi[i] + 1.0 * (x[i] + 0.0);
    if (v < c->s.lower_clip) v = c->phi[i] + 1.0 * (c->s.lower_clip - c->phi[i]);
    c->phi[i] = v;
  }
  return it;
}

}  // extern "C"
