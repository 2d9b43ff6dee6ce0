// tet4 scalar-diffusion path of the B200 CVFEM engine: tet4 mesh set-up,
// the diffusion assembly (element pass, face pass and CSR-entry gather over
// contribution lists built at set-up), and the C-ABI of the diffusion
// handle (a solid-domain energy equation: Gamma-diffusion with a volumetric
// source, fixed-value and zero-flux walls).
//
// Reference: src/assemble/phiAssembler/phiAssemblerElemTerms.hpp:11-413
// (diffusion branch), phiAssemblerElemBoundaryConditions.hpp:112-410
// (fixed-value wall), src/assemble/heatTransfer/thermalEnergy/
// thermalEnergyAssemblerNodeTerms.cpp:25-97 (solid source), phiAssembler.h:
// 748-753,967-1152 and thermalEnergyAssembler.h:39-43 (relaxation), and
// src/equation/heatTransfer/thermalEnergy/thermalEnergyEquation.cpp:190-247
// (assemble, solve, clipped correction).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "oa_internal.h"
#include "oa_scalar_solve.h"
#include "oa_tet4.cuh"
#include "oa_tet4_lists.h"

namespace oa {

namespace {


template <class T>
int dalloc(T** p, size_t n) {
  cudaError_t e = cudaMalloc(p, sizeof(T) * (n ? n : 1));
  if (e != cudaSuccess) return fail(OA_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  return OA_OK;
}

__device__ __forceinline__ void load3(const double* __restrict__ p, int n, double (&v)[3]) {
  v[0] = __ldg(p + 3 * n);
  v[1] = __ldg(p + 3 * n + 1);
  v[2] = __ldg(p + 3 * n + 2);
}

// ---------------------------------------------------------------------------
// geometry set-up: SCV volumes per element, then dual volumes per node

__global__ void k_tet_scv(MeshView m, double* __restrict__ scv, int* err) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.ne) return;
  double x[4][3], v[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) load3(m.x, __ldg(m.conn + 4 * e + k), x[k]);
  tet4::scv_volumes(x, v);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (!(v[k] > 0.0)) err[0] = 1;
    scv[4 * e + k] = v[k];
  }
}

// mesh::updateDualNodalVolumeField_ (src/mesh/meshGeometry.cpp:1277-1345),
// summed in ascending element order.
__global__ void k_tet_dual_volume(MeshView m, const double* __restrict__ scv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nn) return;
  double v = 0.0;
  for (int k = m.n2e_ptr[i]; k < m.n2e_ptr[i + 1]; ++k) v += scv[m.n2e[k]];
  m.vol[i] = v;
}

}  // namespace

int create_tet4_mesh(oa_mesh* M, const double* coords, int nn, const int* conn, int ne, const int* face_elem,
                     const int* face_ord, const int* face_bnd, int nf) {
  DeviceMesh& m = M->m;
  for (long k = 0; k < 4L * ne; ++k)
    if (conn[k] < 0 || conn[k] >= nn) return fail(OA_ERR_MESH, "oa_mesh_create: connectivity index out of range");
  for (int f = 0; f < nf; ++f)
    if (face_elem[f] < 0 || face_elem[f] >= ne || face_ord[f] < 0 || face_ord[f] > 3 || face_bnd[f] < 0)
      return fail(OA_ERR_MESH, "oa_mesh_create: boundary face out of range");
  if (4L * ne > INT_MAX / 2) return fail(OA_ERR_MESH, "oa_mesh_create: too many elements for 32-bit incidence codes");
  m.topo = OA_TOPO_TET4;
  m.nn = nn;
  m.ne = ne;
  m.nf = nf;
  // node -> (element, corner), ascending element
  std::vector<int> n2e_ptr(nn + 1, 0), n2e(4L * ne);
  for (long k = 0; k < 4L * ne; ++k) n2e_ptr[conn[k] + 1] += 1;
  for (int i = 0; i < nn; ++i) n2e_ptr[i + 1] += n2e_ptr[i];
  {
    std::vector<int> pos(n2e_ptr.begin(), n2e_ptr.end() - 1);
    for (int e = 0; e < ne; ++e)
      for (int a = 0; a < 4; ++a) n2e[pos[conn[4L * e + a]]++] = 4 * e + a;
  }
  // node -> (boundary face, side position), ascending face
  std::vector<int> n2f_ptr(nn + 1, 0), n2f(3L * nf);
  std::vector<int> wall(nn, 0);
  for (int f = 0; f < nf; ++f)
    for (int k = 0; k < 3; ++k) {
      const int nd = conn[4L * face_elem[f] + tet4::side_node(face_ord[f], k)];
      n2f_ptr[nd + 1] += 1;
      wall[nd] = 1;
    }
  for (int i = 0; i < nn; ++i) n2f_ptr[i + 1] += n2f_ptr[i];
  {
    std::vector<int> pos(n2f_ptr.begin(), n2f_ptr.end() - 1);
    for (int f = 0; f < nf; ++f)
      for (int k = 0; k < 3; ++k) n2f[pos[conn[4L * face_elem[f] + tet4::side_node(face_ord[f], k)]]++] = 4 * f + k;
  }
  // edge graph (every node pair of an element), sorted columns
  m.h_row_ptr.assign(nn + 1, 0);
  m.h_diag.assign(nn, 0);
  m.h_cols.clear();
  m.h_cols.reserve((size_t)nn * 16);
  std::vector<int> tmp;
  for (int i = 0; i < nn; ++i) {
    tmp.clear();
    for (int k = n2e_ptr[i]; k < n2e_ptr[i + 1]; ++k) {
      const int e = n2e[k] >> 2;
      for (int a = 0; a < 4; ++a) tmp.push_back(conn[4L * e + a]);
    }
    tmp.push_back(i);
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    for (size_t k = 0; k < tmp.size(); ++k)
      if (tmp[k] == i) m.h_diag[i] = (int)k;
    m.h_cols.insert(m.h_cols.end(), tmp.begin(), tmp.end());
    m.h_row_ptr[i + 1] = (int)m.h_cols.size();
  }
  m.nnz = m.h_row_ptr[nn];
  m.h_conn.assign(conn, conn + 4L * ne);
  m.h_face_elem.assign(face_elem, face_elem + nf);
  m.h_face_ord.assign(face_ord, face_ord + nf);
  m.h_face_bnd.assign(face_bnd, face_bnd + nf);
  int st = OA_OK;
  if ((st = dalloc(&m.x, 3L * nn)) || (st = dalloc(&m.conn, 4L * ne)) || (st = dalloc(&m.n2e, 4L * ne)) ||
      (st = dalloc(&m.n2e_ptr, nn + 1L)) || (st = dalloc(&m.n2f, 3L * nf)) || (st = dalloc(&m.n2f_ptr, nn + 1L)) ||
      (st = dalloc(&m.face_elem, (size_t)nf)) || (st = dalloc(&m.face_ord, (size_t)nf)) ||
      (st = dalloc(&m.face_bnd, (size_t)nf)) || (st = dalloc(&m.row_ptr, nn + 1L)) ||
      (st = dalloc(&m.cols, (size_t)m.nnz)) || (st = dalloc(&m.diag, (size_t)nn)) || (st = dalloc(&m.vol, (size_t)nn)) ||
      (st = dalloc(&m.wall_node, (size_t)nn)))
    return st;
  cudaStreamCreateWithFlags(&M->st, cudaStreamNonBlocking);
  cudaMemcpy(m.x, coords, sizeof(double) * 3 * nn, cudaMemcpyHostToDevice);
  cudaMemcpy(m.conn, conn, sizeof(int) * 4 * (size_t)ne, cudaMemcpyHostToDevice);
  cudaMemcpy(m.n2e, n2e.data(), sizeof(int) * n2e.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(m.n2e_ptr, n2e_ptr.data(), sizeof(int) * (nn + 1), cudaMemcpyHostToDevice);
  if (nf) {
    cudaMemcpy(m.n2f, n2f.data(), sizeof(int) * n2f.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(m.face_elem, face_elem, sizeof(int) * nf, cudaMemcpyHostToDevice);
    cudaMemcpy(m.face_ord, face_ord, sizeof(int) * nf, cudaMemcpyHostToDevice);
    cudaMemcpy(m.face_bnd, face_bnd, sizeof(int) * nf, cudaMemcpyHostToDevice);
  }
  cudaMemcpy(m.n2f_ptr, n2f_ptr.data(), sizeof(int) * (nn + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(m.row_ptr, m.h_row_ptr.data(), sizeof(int) * (nn + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(m.cols, m.h_cols.data(), sizeof(int) * m.nnz, cudaMemcpyHostToDevice);
  cudaMemcpy(m.diag, m.h_diag.data(), sizeof(int) * nn, cudaMemcpyHostToDevice);
  cudaMemcpy(m.wall_node, wall.data(), sizeof(int) * nn, cudaMemcpyHostToDevice);
  cudaError_t ce = cudaDeviceSynchronize();
  if (ce == cudaSuccess) ce = cudaGetLastError();
  if (ce != cudaSuccess) return fail(OA_ERR_CUDA, std::string("tet4 mesh upload: ") + cudaGetErrorString(ce));
  // dual volumes
  double* scv = nullptr;
  int* err = nullptr;
  if ((st = dalloc(&scv, 4L * ne)) || (st = dalloc(&err, 1))) {
    if (scv) cudaFree(scv);
    return st;
  }
  cudaMemset(err, 0, sizeof(int));
  k_tet_scv<<<(ne + 127) / 128, 128>>>(m.view(), scv, err);
  k_tet_dual_volume<<<(nn + 127) / 128, 128>>>(m.view(), scv);
  count_launches(2);
  int herr = 0;
  ce = cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(scv);
  cudaFree(err);
  if (ce != cudaSuccess) return fail(OA_ERR_CUDA, std::string("tet4 geometry: ") + cudaGetErrorString(ce));
  m.geom_err = herr;
  if (herr) return fail(OA_ERR_GEOMETRY, "non-positive sub-control volume in tet4 mesh");
  return OA_OK;
}

namespace {

// Per-handle view of the diffusion fields.
struct DiffView {
  const double* phi;
  const double* gamma;
  const double* src;
  const double* side;      // node-side values of the fixed-value boundaries
  const int* bnd_kind;     // OA_BND_* per boundary index
  int nbnd;
  double urf_inv;          // 1 / diagonal relaxation
  double wall_relax;       // wall-node rhs factor
};

// Diffusion assembly in three passes, deterministic and without atomics.
//
// 1. Element owner (k_tet_elem): one thread per tet evaluates, for each of
//    its four corners a, what the corner's control volume receives from the
//    element: with S_a = sum over the three SCS ips around a of Gamma_ip A_ip
//    (A pointing away from a), the coefficients c_a[k] = -dN_k/dx . S_a of the
//    four element nodes and the defect rhs -sum_k c_a[k] phi_k. The corner is
//    evaluated in the frame of the even permutation that brings it to local
//    node 0, with the same arithmetic the oracle's element loop uses per
//    corner. Stored as lhs[16 e + 4 a + k] and rhs[4 e + a].
// 2. Face owner (k_tet_face): one thread per boundary face; on a fixed-value
//    face each side node k gets the flux of its boundary ip: lhs on the
//    off-face node only (the side nodes' columns carry bcMultiplier 0) and
//    rhs Gamma_bip grad(phi~) . A_bip with phi~ the side values on the face
//    nodes. Stored after the element records; zero-flux faces store zeros.
// 3. Gathers: every CSR entry sums its staged contributions in the fixed
//    order of a precomputed list (k_tet_gather; the diagonal is then divided
//    by the relaxation factor), and every row sums the rhs of its element and
//    face items in n2e / n2f order (k_tet_rhs).
template <bool SH, class TM>
__global__ void __launch_bounds__(128) k_tet_elem(MeshView m, DiffView d, TM* __restrict__ lhs,
                                                  double* __restrict__ rhs, int* err) {
  // the records are assembled in shared memory (rows padded against bank
  // conflicts) and each warp stores its 32 elements' records as one
  // contiguous, coalesced block
  __shared__ TM s_lhs[128 * 17];
  __shared__ double s_rhs[128 * 5];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, wbase = threadIdx.x & ~31;
  const long long e0 = (long long)blockIdx.x * blockDim.x + wbase;
  if (e0 >= m.ne) return;  // whole warp
  const int nvalid = (int)min(32LL, (long long)m.ne - e0);
  if (e < m.ne) {
    // shape-function weights of Gamma at an SCS ip (edge nodes, other nodes)
    const double wn = SH ? 0.5 : 13.0 / 36.0, wf = SH ? 0.0 : 5.0 / 36.0;
    double x[4][3], ph[4], gm[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int n = __ldg(m.conn + 4 * e + k);
      load3(m.x, n, x[k]);
      ph[k] = __ldg(d.phi + n);
      gm[k] = __ldg(d.gamma + n);
    }
    // the element's six SCS areas and its gradient operator, once
    double A6[6][3], g[4][3];
    tet4::scs_areas6(x, A6);
    const bool bad = !tet4::grad_op(x, g);
    // Gamma at the ip of each edge: its two nodes with weight wn, the others wf
    constexpr int EN[6][4] = {{0, 1, 2, 3}, {0, 2, 1, 3}, {0, 3, 1, 2}, {1, 3, 0, 2}, {1, 2, 0, 3}, {2, 3, 0, 1}};
    double Ge[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) Ge[q] = wn * (gm[EN[q][0]] + gm[EN[q][1]]) + wf * (gm[EN[q][2]] + gm[EN[q][3]]);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      // S = sum over the corner's three ips of Gamma_ip A_ip, A away from a
      double S[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int k = 1; k < 4; ++k) {
        const int q = tet4::corner_edge(a, k);
        const double w = tet4::corner_edge_sign(a, k) * Ge[q];
#pragma unroll
        for (int j = 0; j < 3; ++j) S[j] += w * A6[q][j];
      }
      double c[4], r = 0.0;
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        c[n] = -(g[n][0] * S[0] + g[n][1] * S[1] + g[n][2] * S[2]);
        r -= c[n] * ph[n];
      }
      s_rhs[threadIdx.x * 5 + a] = r;
#pragma unroll
      for (int n = 0; n < 4; ++n) s_lhs[threadIdx.x * 17 + 4 * a + n] = TM(c[n]);
    }
    if (bad) err[0] = 1;
  }
  __syncwarp();
  for (int i = lane; i < 16 * nvalid; i += 32) lhs[16 * e0 + i] = s_lhs[(wbase + (i >> 4)) * 17 + (i & 15)];
  for (int i = lane; i < 4 * nvalid; i += 32) rhs[4 * e0 + i] = s_rhs[(wbase + (i >> 2)) * 5 + (i & 3)];
}

template <bool SH, class TM>
__global__ void __launch_bounds__(128) k_tet_face(MeshView m, DiffView d, TM* __restrict__ lhs,
                                                  double* __restrict__ rhs, int* err) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nf) return;
  const int bnd = __ldg(m.face_bnd + f);
  if (!(bnd < d.nbnd && __ldg(d.bnd_kind + bnd) == OA_BND_FIXED_VALUE)) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lhs[3 * (size_t)f + k] = TM(0);
      rhs[3 * (size_t)f + k] = 0.0;
    }
    return;
  }
  // shape-function weights of Gamma at a tri3 boundary ip (own node, others)
  const double fo = SH ? 1.0 : 1.0 - 7.0 / 36.0 - 7.0 / 36.0, ff = SH ? 0.0 : 7.0 / 36.0;
  const int e = __ldg(m.face_elem + f), o = __ldg(m.face_ord + f);
  // element nodes as (opposite node, side nodes in side order): a positively
  // oriented ordering with the face opposite local node 0
  double x[4][3], g[4][3], p[3][3];
  int nd[4];
  nd[0] = __ldg(m.conn + 4 * e + tet4::opposite_node(o));
#pragma unroll
  for (int q = 0; q < 3; ++q) nd[q + 1] = __ldg(m.conn + 4 * e + tet4::side_node(o, q));
#pragma unroll
  for (int q = 0; q < 4; ++q) load3(m.x, nd[q], x[q]);
  if (!tet4::grad_op(x, g)) err[0] = 1;
  double gs[3], grad_t[3];
  const double po = __ldg(d.phi + nd[0]);
#pragma unroll
  for (int j = 0; j < 3; ++j) grad_t[j] = po * g[0][j];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
#pragma unroll
    for (int j = 0; j < 3; ++j) p[q][j] = x[q + 1][j];
    gs[q] = __ldg(d.gamma + nd[q + 1]);
    const double ps = __ldg(d.side + nd[q + 1]);
#pragma unroll
    for (int j = 0; j < 3; ++j) grad_t[j] += ps * g[q + 1][j];
  }
  double Aall[3][3];
  tet4::tri_face_areas(p, Aall);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double G = fo * gs[k] + ff * (gs[0] + gs[1] + gs[2] - gs[k]);
    lhs[3 * (size_t)f + k] = TM(-G * (g[0][0] * Aall[k][0] + g[0][1] * Aall[k][1] + g[0][2] * Aall[k][2]));
    rhs[3 * (size_t)f + k] = G * (grad_t[0] * Aall[k][0] + grad_t[1] * Aall[k][1] + grad_t[2] * Aall[k][2]);
  }
}

// A[s] = sum of the staged contributions listed for entry s, in list order;
// diagonal entries divided by the relaxation factor
template <class TM>
__global__ void __launch_bounds__(256) k_tet_gather(int nnz, const int* __restrict__ eptr,
                                                    const int* __restrict__ eidx, const uint8_t* __restrict__ ediag,
                                                    const TM* __restrict__ lhs, double urf_inv, TM* __restrict__ A) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nnz) return;
  // four list items per pass with every load issued before the adds (items
  // past the end clamped and dropped); the sum keeps list order
  const int q0 = __ldg(eptr + s), q1 = __ldg(eptr + s + 1);
  double acc = 0.0;
  for (int q = q0; q < q1; q += 4) {
    int id[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) id[u] = __ldg(eidx + min(q + u, q1 - 1));
    double v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = double(__ldg(lhs + id[u]));
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (q + u < q1) acc += v[u];
  }
  if (__ldg(ediag + s)) acc *= urf_inv;
  A[s] = TM(acc);
}

// b[row] = source * volume + the row's element and face rhs (n2e, then n2f
// order), times the wall relaxation on wall nodes
__global__ void __launch_bounds__(256) k_tet_rhs(MeshView m, DiffView d, const double* __restrict__ rhs_e,
                                                 const double* __restrict__ rhs_f, double* __restrict__ b) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= m.nn) return;
  double r = 0.0;
  const int q0 = __ldg(m.n2e_ptr + row), q1 = __ldg(m.n2e_ptr + row + 1);
  for (int q = q0; q < q1; q += 4) {  // as in k_tet_gather: four items in flight, order kept
    int id[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) id[u] = __ldg(m.n2e + min(q + u, q1 - 1));
    double v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = __ldg(rhs_e + id[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (q + u < q1) r += v[u];
  }
  for (int q = __ldg(m.n2f_ptr + row); q < __ldg(m.n2f_ptr + row + 1); ++q) {
    const int code = __ldg(m.n2f + q);
    r += __ldg(rhs_f + 3 * (code >> 2) + (code & 3));
  }
  double bb = __ldg(d.src + row) * __ldg(m.vol + row) + r;
  if (__ldg(m.wall_node + row)) bb *= d.wall_relax;
  b[row] = bb;
}

// phi <- phi + x, clipped below (equation::correctField_ with CLIP,
// src/equation/equation.h:204-286).
__global__ void k_correct_clip(int n, double* __restrict__ phi, const double* __restrict__ x, double lo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double p = phi[i];
  double v = p + 1.0 * (x[i] + 0.0);
  if (v < lo) v = p + 1.0 * (lo - p);
  phi[i] = v;
}

template <class T>
__global__ void k_widen(size_t n, const T* a, double* b) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = double(a[i]);
}

}  // namespace
}  // namespace oa

using namespace oa;

struct oa_diffusion {
  DeviceMesh* mesh = nullptr;
  oa_diffusion_settings s{};
  cudaStream_t stream = nullptr;
  double *phi = nullptr, *gamma = nullptr, *src = nullptr, *side = nullptr;
  int* bnd_kind = nullptr;
  int nbnd = 0;
  void* A = nullptr;       // [nnz] FP64 or FP32
  double* b = nullptr;     // [nn]
  double* x = nullptr;     // [nn]
  int* err = nullptr;
  bool assembled = false;
  ScalarSolve solver;
  // staged contributions: [16 ne] element lhs then [3 nf] face lhs (matrix
  // precision), [4 ne] element rhs then [3 nf] face rhs (FP64)
  void* lhs_st = nullptr;
  double* rhs_st = nullptr;
  // per CSR entry, the ordered list of staged lhs contributions, and a mark
  // on the diagonal entries
  int *eptr = nullptr, *eidx = nullptr;
  uint8_t* ediag = nullptr;
};

namespace {

bool dmixed(const oa_diffusion* H) { return H->s.precision == OA_PREC_MIXED; }

// Contribution lists of the CSR entries (oa_tet4_lists.h) from the mesh's
// host copies; the faces' side and opposite nodes come from the tet4 tables.
int build_entry_lists(const DeviceMesh& m, const int* bnd_kind, int nbnd, std::vector<int>& eptr,
                      std::vector<int>& eidx, std::vector<uint8_t>& ediag) {
  std::vector<int> side(3 * (size_t)m.nf), opp(m.nf);
  std::vector<uint8_t> fixed(m.nf, 0);
  for (int f = 0; f < m.nf; ++f) {
    const long long e = m.h_face_elem[f];
    const int o = m.h_face_ord[f], bnd = m.h_face_bnd[f];
    fixed[f] = (bnd < nbnd && bnd_kind[bnd] == OA_BND_FIXED_VALUE) ? 1 : 0;
    opp[f] = m.h_conn[4 * e + tet4::opposite_node(o)];
    for (int q = 0; q < 3; ++q) side[3 * f + q] = m.h_conn[4 * e + tet4::side_node(o, q)];
  }
  tet4lists::Input in;
  in.nn = m.nn;
  in.ne = m.ne;
  in.nf = m.nf;
  in.row_ptr = m.h_row_ptr.data();
  in.cols = m.h_cols.data();
  in.diag = m.h_diag.data();
  in.conn = m.h_conn.data();
  in.face_side = side.data();
  in.face_opp = opp.data();
  in.face_fixed = fixed.data();
  if (!tet4lists::build(in, eptr, eidx, ediag))
    return fail(OA_ERR_ARG, "oa_diffusion_create: mesh too large for 32-bit lists");
  return OA_OK;
}

double* diff_field(oa_diffusion* H, const std::string& n) {
  if (n == "phi") return H->phi;
  if (n == "gamma") return H->gamma;
  if (n == "src") return H->src;
  if (n == "sidePhi") return H->side;
  return nullptr;
}

template <bool SH, class TM>
void launch_diffusion_t(oa_diffusion* H, const DiffView& d) {
  DeviceMesh& m = *H->mesh;
  TM* lhs = static_cast<TM*>(H->lhs_st);
  double* rhs = H->rhs_st;
  const size_t ne = m.ne;
  k_tet_elem<SH, TM><<<(m.ne + 127) / 128, 128, 0, H->stream>>>(m.view(), d, lhs, rhs, H->err);
  if (m.nf) k_tet_face<SH, TM><<<(m.nf + 127) / 128, 128, 0, H->stream>>>(m.view(), d, lhs + 16 * ne, rhs + 4 * ne, H->err);
  k_tet_gather<TM><<<(m.nnz + 255) / 256, 256, 0, H->stream>>>(m.nnz, H->eptr, H->eidx, H->ediag, lhs, d.urf_inv,
                                                                static_cast<TM*>(H->A));
  k_tet_rhs<<<(m.nn + 255) / 256, 256, 0, H->stream>>>(m.view(), d, rhs, rhs + 4 * ne, H->b);
  count_launches(m.nf ? 4 : 3);
}

int launch_diffusion(oa_diffusion* H) {
  DiffView d{H->phi, H->gamma, H->src, H->side, H->bnd_kind, H->nbnd, 1.0 / H->s.urf, H->s.wall_rhs_relax};
  const bool sh = H->s.shifted != 0;
  if (dmixed(H)) {
    if (sh) launch_diffusion_t<true, float>(H, d);
    else launch_diffusion_t<false, float>(H, d);
  } else {
    if (sh) launch_diffusion_t<true, double>(H, d);
    else launch_diffusion_t<false, double>(H, d);
  }
  OA_CUDA(cudaGetLastError());
  H->assembled = true;
  return OA_OK;
}

int diff_check_err(oa_diffusion* H, const char* what) {
  int h = 0;
  OA_CUDA(cudaMemcpyAsync(&h, H->err, sizeof(int), cudaMemcpyDeviceToHost, H->stream));
  OA_CUDA(cudaStreamSynchronize(H->stream));
  if (h) {
    OA_CUDA(cudaMemsetAsync(H->err, 0, sizeof(int), H->stream));
    OA_CUDA(cudaStreamSynchronize(H->stream));
    return fail(OA_ERR_GEOMETRY, std::string(what) + ": singular Jacobian (det <= 1e6*realmin)");
  }
  return OA_OK;
}

int diff_solve(oa_diffusion* H, double rtol, int maxit, int* iters, double* res, int* refinements) {
  DeviceMesh& m = *H->mesh;
  ScalarGraph g;
  g.nn = m.nn;
  g.rp = m.row_ptr;
  g.cols = m.cols;
  g.diag = m.diag;
  g.h_rp = m.h_row_ptr.data();
  g.h_cols = m.h_cols.data();
  g.h_diag = m.h_diag.data();
  return H->solver.solve(g, dmixed(H), H->s.amg != 0, H->s.use_graphs != 0, H->A, H->b, H->x, rtol, maxit, iters,
                         res, refinements, H->stream, "diffusion");
}

}  // namespace

extern "C" {

int oa_diffusion_create(oa_mesh* M, const oa_diffusion_settings* s, const int* bnd_kind, const double* bnd_value,
                        int nbnd, oa_diffusion** out) {
  if (!M || !s || !out || nbnd < 0 || (nbnd > 0 && (!bnd_kind || !bnd_value)))
    return fail(OA_ERR_ARG, "oa_diffusion_create: bad arguments");
  *out = nullptr;
  if (M->m.topo != OA_TOPO_TET4) return fail(OA_ERR_MESH, "oa_diffusion_create: the diffusion path needs a tet4 mesh");
  if (!(s->urf > 0.0)) return fail(OA_ERR_ARG, "oa_diffusion_create: relaxation must be > 0");
  if (s->precision != OA_PREC_FP64 && s->precision != OA_PREC_MIXED)
    return fail(OA_ERR_ARG, "oa_diffusion_create: unknown precision");
  for (int i = 0; i < nbnd; ++i)
    if (bnd_kind[i] != OA_BND_FIXED_VALUE && bnd_kind[i] != OA_BND_ZERO_FLUX)
      return fail(OA_ERR_ARG, "oa_diffusion_create: unknown boundary kind");
  const DeviceMesh& m = M->m;
  for (int f = 0; f < m.nf; ++f)
    if (m.h_face_bnd[f] >= nbnd) return fail(OA_ERR_ARG, "oa_diffusion_create: a face names a boundary index >= nbnd");
  oa_diffusion* H = new oa_diffusion();
  // BiCGStab by default: on the tet4 conduction GCR(2) needs as many V-cycles
  // as BiCGStab (26 against 13 x 2 at 96^3 x 6) and is 7 % slower per step
  H->solver.gcr = false;
  H->mesh = &M->m;
  H->s = *s;
  H->nbnd = nbnd;
  const size_t nn = m.nn, nnz = m.nnz;
  const size_t tm = s->precision == OA_PREC_MIXED ? sizeof(float) : sizeof(double);
  int st = OA_OK;
  if ((st = dalloc(&H->phi, nn)) || (st = dalloc(&H->gamma, nn)) || (st = dalloc(&H->src, nn)) ||
      (st = dalloc(&H->side, nn)) || (st = dalloc(&H->bnd_kind, (size_t)std::max(nbnd, 1))) ||
      (st = dalloc(&H->b, nn)) || (st = dalloc(&H->x, nn)) || (st = dalloc(&H->err, 1))) {
    oa_diffusion_destroy(H);
    return st;
  }
  if (cudaMalloc(&H->A, tm * nnz) != cudaSuccess) {
    oa_diffusion_destroy(H);
    return fail(OA_ERR_CUDA, "oa_diffusion_create: device allocation failed");
  }
  {
    std::vector<int> eptr, eidx;
    std::vector<uint8_t> ediag;
    const size_t ne = m.ne, nf = m.nf;
    if ((st = build_entry_lists(m, bnd_kind, nbnd, eptr, eidx, ediag)) || (st = dalloc(&H->eptr, eptr.size())) ||
        (st = dalloc(&H->eidx, eidx.size())) || (st = dalloc(&H->ediag, ediag.size())) ||
        (st = dalloc(&H->rhs_st, 4 * ne + 3 * nf))) {
      oa_diffusion_destroy(H);
      return st;
    }
    if (cudaMalloc(&H->lhs_st, tm * (16 * ne + 3 * nf + 1)) != cudaSuccess) {
      oa_diffusion_destroy(H);
      return fail(OA_ERR_CUDA, "oa_diffusion_create: device allocation failed");
    }
    cudaMemcpy(H->eptr, eptr.data(), sizeof(int) * eptr.size(), cudaMemcpyHostToDevice);
    if (!eidx.empty()) cudaMemcpy(H->eidx, eidx.data(), sizeof(int) * eidx.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(H->ediag, ediag.data(), ediag.size(), cudaMemcpyHostToDevice);
  }
  cudaStreamCreateWithFlags(&H->stream, cudaStreamNonBlocking);
  std::vector<double> h(nn, 0.0);
  // node-side values of the fixed-value boundaries, boundary by boundary in
  // index order (nodeField::updateBoundarySideFieldSpecifiedValue sets parts in
  // turn); zero-flux boundaries write none
  std::vector<double> side(nn, 0.0);
  for (int bnd = 0; bnd < nbnd; ++bnd) {
    if (bnd_kind[bnd] != OA_BND_FIXED_VALUE) continue;
    for (int f = 0; f < m.nf; ++f) {
      if (m.h_face_bnd[f] != bnd) continue;
      for (int k = 0; k < 3; ++k)
        side[m.h_conn[4L * m.h_face_elem[f] + tet4::side_node(m.h_face_ord[f], k)]] = bnd_value[bnd];
    }
  }
  cudaMemcpy(H->phi, h.data(), sizeof(double) * nn, cudaMemcpyHostToDevice);
  cudaMemcpy(H->src, h.data(), sizeof(double) * nn, cudaMemcpyHostToDevice);
  std::fill(h.begin(), h.end(), 1.0);
  cudaMemcpy(H->gamma, h.data(), sizeof(double) * nn, cudaMemcpyHostToDevice);
  cudaMemcpy(H->side, side.data(), sizeof(double) * nn, cudaMemcpyHostToDevice);
  if (nbnd) cudaMemcpy(H->bnd_kind, bnd_kind, sizeof(int) * nbnd, cudaMemcpyHostToDevice);
  cudaMemset(H->err, 0, sizeof(int));
  cudaError_t ce = cudaDeviceSynchronize();
  if (ce == cudaSuccess) ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    oa_diffusion_destroy(H);
    return fail(OA_ERR_CUDA, std::string("oa_diffusion_create: ") + cudaGetErrorString(ce));
  }
  *out = H;
  return OA_OK;
}

void oa_diffusion_destroy(oa_diffusion* H) {
  if (!H) return;
  void* ptrs[] = {H->phi, H->gamma, H->src,   H->side, H->bnd_kind, H->A,    H->b,
                  H->x,   H->err,   H->lhs_st, H->rhs_st, H->eptr,    H->eidx, H->ediag};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  H->solver.release();
  if (H->stream) cudaStreamDestroy(H->stream);
  delete H;
}

int oa_diffusion_set_field(oa_diffusion* H, const char* name, const double* host, long n) {
  if (!H || !name || !host) return fail(OA_ERR_ARG, "oa_diffusion_set_field: null argument");
  double* p = diff_field(H, name);
  if (!p) return fail(OA_ERR_ARG, std::string("oa_diffusion_set_field: unknown field ") + name);
  if (n != H->mesh->nn) return fail(OA_ERR_ARG, std::string("oa_diffusion_set_field: size mismatch for ") + name);
  OA_CUDA(cudaMemcpyAsync(p, host, sizeof(double) * n, cudaMemcpyHostToDevice, H->stream));
  OA_CUDA(cudaStreamSynchronize(H->stream));
  return OA_OK;
}

int oa_diffusion_get_field(oa_diffusion* H, const char* name, double* host, long n) {
  if (!H || !name || !host) return fail(OA_ERR_ARG, "oa_diffusion_get_field: null argument");
  double* p = diff_field(H, name);
  if (!p) return fail(OA_ERR_ARG, std::string("oa_diffusion_get_field: unknown field ") + name);
  if (n != H->mesh->nn) return fail(OA_ERR_ARG, std::string("oa_diffusion_get_field: size mismatch for ") + name);
  OA_CUDA(cudaMemcpyAsync(host, p, sizeof(double) * n, cudaMemcpyDeviceToHost, H->stream));
  OA_CUDA(cudaStreamSynchronize(H->stream));
  return OA_OK;
}

int oa_diffusion_field_device_ptr(oa_diffusion* H, const char* name, double** dev) {
  if (!H || !name || !dev) return fail(OA_ERR_ARG, "oa_diffusion_field_device_ptr: null argument");
  double* p = diff_field(H, name);
  if (!p) return fail(OA_ERR_ARG, std::string("oa_diffusion_field_device_ptr: unknown field ") + name);
  *dev = p;
  return OA_OK;
}

int oa_diffusion_assemble(oa_diffusion* H, double* A, double* b) {
  if (!H) return fail(OA_ERR_ARG, "oa_diffusion_assemble: null handle");
  if (int s = launch_diffusion(H)) return s;
  if (int s = diff_check_err(H, "oa_diffusion_assemble")) return s;
  const size_t nnz = H->mesh->nnz, nn = H->mesh->nn;
  if (A) {
    if (dmixed(H)) {
      double* tmp = nullptr;
      if (int s = dalloc(&tmp, nnz)) return s;
      k_widen<float><<<(unsigned)((nnz + 255) / 256), 256, 0, H->stream>>>(nnz, (const float*)H->A, tmp);
      OA_CUDA(cudaMemcpyAsync(A, tmp, sizeof(double) * nnz, cudaMemcpyDeviceToHost, H->stream));
      OA_CUDA(cudaStreamSynchronize(H->stream));
      cudaFree(tmp);
    } else {
      OA_CUDA(cudaMemcpyAsync(A, H->A, sizeof(double) * nnz, cudaMemcpyDeviceToHost, H->stream));
    }
  }
  if (b) OA_CUDA(cudaMemcpyAsync(b, H->b, sizeof(double) * nn, cudaMemcpyDeviceToHost, H->stream));
  OA_CUDA(cudaStreamSynchronize(H->stream));
  return OA_OK;
}

int oa_diffusion_solve(oa_diffusion* H, double rtol, int maxit, double* x, int* iters, double* res,
                       int* refinements) {
  if (!H || maxit <= 0 || !(rtol > 0.0)) return fail(OA_ERR_ARG, "oa_diffusion_solve: bad arguments");
  if (!H->assembled) return fail(OA_ERR_NOT_READY, "oa_diffusion_solve: no assembled system");
  if (int s = diff_solve(H, rtol, maxit, iters, res, refinements)) return s;
  if (x) OA_CUDA(cudaMemcpyAsync(x, H->x, sizeof(double) * H->mesh->nn, cudaMemcpyDeviceToHost, H->stream));
  OA_CUDA(cudaStreamSynchronize(H->stream));
  return OA_OK;
}

int oa_diffusion_step(oa_diffusion* H, int* iters, double* res, int* refinements) {
  if (!H) return fail(OA_ERR_ARG, "oa_diffusion_step: null handle");
  if (int s = launch_diffusion(H)) return s;
  if (int s = diff_check_err(H, "oa_diffusion_step")) return s;
  if (int s = diff_solve(H, H->s.rtol, H->s.maxit, iters, res, refinements)) return s;
  const int n = H->mesh->nn;
  k_correct_clip<<<(n + 255) / 256, 256, 0, H->stream>>>(n, H->phi, H->x, H->s.lower_clip);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  OA_CUDA(cudaStreamSynchronize(H->stream));
  return OA_OK;
}

int oa_diffusion_stream(oa_diffusion* H, void** stream) {
  if (!H || !stream) return fail(OA_ERR_ARG, "oa_diffusion_stream: null argument");
  *stream = (void*)H->stream;
  return OA_OK;
}

int oa_diffusion_time_assembly(oa_diffusion* H, int reps, double* ms) {
  if (!H || !ms || reps <= 0) return fail(OA_ERR_ARG, "oa_diffusion_time_assembly: bad arguments");
  cudaEvent_t e0, e1;
  OA_CUDA(cudaEventCreate(&e0));
  OA_CUDA(cudaEventCreate(&e1));
  if (int s = launch_diffusion(H)) return s;
  OA_CUDA(cudaEventRecord(e0, H->stream));
  for (int i = 0; i < reps; ++i)
    if (int s = launch_diffusion(H)) return s;
  OA_CUDA(cudaEventRecord(e1, H->stream));
  OA_CUDA(cudaEventSynchronize(e1));
  float t = 0.f;
  OA_CUDA(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = double(t) / reps;
  return diff_check_err(H, "oa_diffusion_time_assembly");
}

}  // extern "C"
