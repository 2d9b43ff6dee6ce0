// Hand-written sm_100a kernels of the hex8 CVFEM hot path: geometry
// precompute, pressure-correction and momentum assembly (row-owner, written
// once per CSR row), mass-flow update, divergence and Green-Gauss gradients.
#include <cuda_runtime.h>

#include <cstdint>

#include "oa_internal.h"
#include "oa_geom.cuh"
#include "oa_rowlane.cuh"

namespace oa {

using namespace hex8;

constexpr double SMALL = 2.220446049250313e-16;  // src/basic/types.h:179
constexpr int BLOCK = 128;                        // 16 rows per block

template <int I, int N>
struct StaticFor {
  template <class F>
  __device__ __forceinline__ static void run(F&& f) {
    f(std::integral_constant<int, I>{});
    StaticFor<I + 1, N>::run(f);
  }
};
template <int N>
struct StaticFor<N, N> {
  template <class F>
  __device__ __forceinline__ static void run(F&&) {}
};

__device__ __forceinline__ void load3(const double* __restrict__ p, int n, double (&v)[3]) {
  v[0] = __ldg(p + 3 * n);
  v[1] = __ldg(p + 3 * n + 1);
  v[2] = __ldg(p + 3 * n + 2);
}

// SCS area vector of the ip packed in an ip word entry (original ip << 1 |
// sign), from the per-element table, pointing away from the lane's corner.
__device__ __forceinline__ void load_area(const MeshView& m, int e, int pk, double (&A)[3]) {
  const double* a = m.scs_area + 36L * e + 3 * (pk >> 1);
  const double sg = (pk & 1) ? -1.0 : 1.0;
  A[0] = sg * __ldg(a);
  A[1] = sg * __ldg(a + 1);
  A[2] = sg * __ldg(a + 2);
}

// ---------------------------------------------------------------------------
// Geometry precompute (FP64, once per mesh)

// SCV volume of corner 0 in the canonical frame: sub-hex
// {0, mid01, face0123, mid03, mid04, face0145, centroid, face0347}
// (hex_scv_det table row 1).
__device__ __forceinline__ double corner0_scv(const double (&x)[8][3], const Corner0Points& p) {
  double v[8][3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    v[0][k] = x[0][k];
    v[1][k] = p.m01[k];
    v[2][k] = p.fB[k];
    v[3][k] = p.m03[k];
    v[4][k] = p.m04[k];
    v[5][k] = p.fF[k];
    v[6][k] = p.cen[k];
    v[7][k] = p.fL[k];
  }
  return hex_volume(v);
}

__device__ __forceinline__ void gather_x(const MeshView& m, int e, uint32_t pw, double (&x)[8][3],
                                         int (&nd)[8]) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    nd[k] = __ldg(m.conn + 8 * e + perm_at(pw, k));
    load3(m.x, nd[k], x[k]);
  }
}

struct GeoArgs {
  MeshView m;
  double* scv;  // [ne][8] raw SCV volumes (scratch)
  int* err;
};

// Element kernel: SCV volumes of all 8 corners, stored as volume fractions
// (the scv weights of pressureCorrectionAssemblerElemTerms.cpp:349-368).
__global__ void __launch_bounds__(BLOCK) k_scv(GeoArgs a) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.m.ne) return;
  double vols[8];
  double Vel = 0.0;
#pragma unroll 1
  for (int c = 0; c < 8; ++c) {
    double x[8][3];
    int nd[8];
    gather_x(a.m, e, perm_word(c), x, nd);
    Corner0Points p;
    corner0_points(x, p);
    vols[c] = corner0_scv(x, p);
    if (!(vols[c] > 0.0)) a.err[0] = 1;
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) Vel += vols[c];
  const double iV = 1.0 / Vel;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    a.scv[8 * e + c] = vols[c];
    a.m.wscv[8 * e + c] = vols[c] * iV;
  }
}

// Row kernel: dual nodal volume = sum of incident SCV volumes
// (mesh::updateDualNodalVolumeField_).
template <int LPR>
__global__ void __launch_bounds__(BLOCK) k_dual_volume(GeoArgs a) {
  const RowLane<LPR> rl = row_lane<LPR>(a.m);
  double v = (rl.e >= 0) ? a.scv[8 * rl.e + rl.c] : 0.0;
  v = rowsum<LPR>(v);
  if (rl.rv && rl.li == 0) a.m.vol[rl.row] = v;
}

int launch_scs_area(DeviceMesh& m, cudaStream_t st);

int launch_geometry(DeviceMesh& m, cudaStream_t st) {
  if (int s = launch_scs_area(m, st)) return s;
  GeoArgs a{m.view(), nullptr, nullptr};
  OA_CUDA(cudaMallocAsync(&a.scv, sizeof(double) * 8 * (size_t)m.ne, st));
  OA_CUDA(cudaMallocAsync(&a.err, sizeof(int), st));
  OA_CUDA(cudaMemsetAsync(a.err, 0, sizeof(int), st));
  k_scv<<<(m.ne + BLOCK - 1) / BLOCK, BLOCK, 0, st>>>(a);
  const unsigned gdv = (unsigned)(((size_t)m.nn * m.lpr + BLOCK - 1) / BLOCK);
  if (m.lpr == 16) k_dual_volume<16><<<gdv, BLOCK, 0, st>>>(a);
  else k_dual_volume<8><<<gdv, BLOCK, 0, st>>>(a);
  OA_CUDA(cudaGetLastError());
  int herr = 0;
  OA_CUDA(cudaMemcpyAsync(&herr, a.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  OA_CUDA(cudaFreeAsync(a.scv, st));
  OA_CUDA(cudaFreeAsync(a.err, st));
  OA_CUDA(cudaStreamSynchronize(st));
  m.geom_err = herr;
  if (herr) return fail(OA_ERR_GEOMETRY, "non-positive sub-control volume in mesh");
  return OA_OK;
}

// ---------------------------------------------------------------------------
// CSR row write-out shared by the assembly kernels. Each lane publishes its
// three edge-neighbour blocks; lane s of the row then emits CSR slot s (s,
// s+8, ...), summing the blocks its precomputed slot mask names in ascending
// (lane, neighbour) order. The diagonal block is already reduced in every lane.
template <int B, class TM, int LPR>
__device__ __forceinline__ void write_row(int row, bool rv, int li, int lane, const TM (&diag)[B],
                                          const TM (&nb)[3][B], const MeshView& m, TM* __restrict__ A,
                                          TM* sh_val, bool offdiag_zero) {
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int b = 0; b < B; ++b) sh_val[(lane * 3 + k) * B + b] = nb[k][b];
  __syncwarp();
  if (rv) {
    const int rp = __ldg(m.row_ptr + row);
    const int len = __ldg(m.row_ptr + row + 1) - rp;
    const int dof = __ldg(m.diag + row);
    const TM* row_vals = sh_val + (lane & ~(LPR - 1)) * 3 * B;
    for (int s = li; s < len; s += LPR) {
      TM out[B];
      if (s == dof) {
#pragma unroll
        for (int b = 0; b < B; ++b) out[b] = diag[b];
      } else {
#pragma unroll
        for (int b = 0; b < B; ++b) out[b] = TM(0);
        unsigned long long mk = 0ull;
        if (!offdiag_zero) mk = LPR == 8 ? __ldg(m.slot_mask + rp + s) : __ldg(m.slot_mask64 + rp + s);
        while (mk) {
          const TM* v = row_vals + (__ffsll(mk) - 1) * B;
          mk &= mk - 1;
#pragma unroll
          for (int b = 0; b < B; ++b) out[b] += v[b];
        }
      }
#pragma unroll
      for (int b = 0; b < B; ++b) A[(size_t)(rp + s) * B + b] = out[b];
    }
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// Pressure-correction assembly
// (pressureCorrectionAssemblerElemTerms.cpp:17-616, incompressible, stationary
// frame; adjustMatrixForPressureReference, pressureCorrectionAssembler.cpp:19-63).
//
// Split in two: the element-owner mass-flow kernel (k_mdot below) evaluates
// every SCS ip once and stages, per element corner, the lhs coefficients of
// the corner's three edge neighbours summed over the corner's three ips
// ([ne][8][3], in the order of edge_nbr) and, per ip, the Rhie-Chow flux of the
// rhs ([ne][12]); this row kernel gathers its row's eight corner records and
// writes the CSR row. The diagonal is minus the sum of the kept neighbour
// coefficients (partition of unity, sum_n grad N_n = 0: every column outside
// the edge stencil is lumped into it).
struct PcArgs {
  MeshView m;
  const void* coef;    // [ne][8][3] staged lhs coefficients (TF)
  const double* flux;  // [ne][12] Rhie-Chow ip mass fluxes with the upwind density
  void* A;
  double* b;
  const uint8_t* ref_flag;  // [nn] 1 on pressure-level rows
};

template <int LPR, class TF>
__global__ void __launch_bounds__(BLOCK) k_pcorr(PcArgs a) {
  __shared__ TF sh_val[BLOCK * 3];
  const int lane = threadIdx.x & 31;
  const int warp_base = threadIdx.x & ~31;
  const RowLane<LPR> rl = row_lane<LPR>(a.m);
  const int row = rl.row, li = rl.li, e = rl.e, c = rl.c;
  const bool rv = rl.rv;
  TF diag[1] = {TF(0)};
  TF nb[3][1] = {{TF(0)}, {TF(0)}, {TF(0)}};
  double rhs = 0.0;
  if (e >= 0) {
    const TF* cf = static_cast<const TF*>(a.coef) + 24 * (size_t)e + 3 * c;
#pragma unroll
    for (int s = 0; s < 3; ++s) nb[s][0] = __ldg(cf + s);
    diag[0] = -(nb[0][0] + nb[1][0] + nb[2][0]);
    const uint32_t iw = ip_word(c);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int pk = (iw >> (5 * q)) & 31;
      const double fl = __ldg(a.flux + 12 * e + (pk >> 1));
      rhs -= (pk & 1) ? -fl : fl;
    }
  }
  diag[0] = rowsum<LPR>(diag[0]);
  rhs = rowsum<LPR>(rhs);
  const bool refrow = rv && __ldg(a.ref_flag + row) != 0;
  write_row<1, TF, LPR>(row, rv, li, lane, diag, nb, a.m, static_cast<TF*>(a.A), sh_val + warp_base * 3, refrow);
  if (rv && li == 0) a.b[row] = refrow ? 0.0 : rhs;
}

// ---------------------------------------------------------------------------
// Momentum assembly (navierStokesAssemblerElemTerms.cpp:15-441 upwind,
// incompressible; no-slip walls ...ElemBoundaryConditions.cpp:2659-2981 with
// IP_ZERO_NORMAL_STRESS_FIXED_VEL__; node terms ...NodeTerms.cpp:16-149;
// postAssemble_ relaxation phiAssembler.h:967-1006 and wall rhs relaxation
// navierStokesAssembler.cpp:241-385; computeDUCoefficients :84-232).
struct MomArgs {
  MeshView m;
  const double *U, *gradP, *div, *mDot, *rho, *mu, *sideU;
  // high-resolution advection: velocity blending factor [nn][3] and nodal
  // velocity gradient [nn][9] of the deferred correction
  const double *betaU, *gradU;
  const float4* xloc;  // mixed form: [ne][8] FP32 corner offsets from corner 0
  const float4* umu;   // mixed form: [nn] FP32 (U, mu)
  void* A;
  void* b;
  double* du;
  double* duT;   // SIMPLEC: D~ [nn][3]
  double dt, urf_inv, wall_relax;
  int du_mode;   // 0 SIMPLE, 1 SIMPLEC, 2 fractional step
  int hr;        // high-resolution deferred correction
  // transient runs: BDF order (0 steady: dt is the false-transient physical
  // timescale; 1, 2: dt is the time step), coefficients, old velocity levels
  int order;
  double tk0, tk1, tk2;
  const double *Uold, *Uoldold;
  int* err;
  // fused turbulence transport (VAR 2): k, omega, their nodal diffusivities
  // and node source terms; systems in the matrix precision
  const double *kf, *wf, *gkf, *gwf, *sdk, *srk, *sdw, *srw;
  void *Ak, *bk, *Aw, *bw;
  double urf_k_inv, urf_w_inv;
};

// Zero-normal-stress wall term at the exposed ip of canonical face FC nearest
// corner 0 (IP_ZERO_NORMAL_STRESS_FIXED_VEL__).
template <int FC, bool USH, bool UGSH, class TF>
__device__ __forceinline__ void wall_face(const MomArgs& a, const TF (&x)[8][3], const int (&nd)[8],
                                          const TF (&Uc)[8][3], const TF (&mu)[8], TF (&diag)[9],
                                          TF (&nb)[3][9], TF (&rhs)[3], int* err) {
  constexpr int f0 = face_node(FC, 0), f1 = face_node(FC, 1), f2 = face_node(FC, 2), f3 = face_node(FC, 3);
  TF Af[3];
  face_area_at_first<TF>(x[f0], x[f1], x[f2], x[f3], Af);
  using PT = FacePt<FC, 0, UGSH>;
  const InvJacR<TF> J = inv_jacobian<PT, TF>(x, err);
  // face-node velocities replaced by the wall (node-side) values
  TF Ue[8][3];
#pragma unroll
  for (int n = 0; n < 8; ++n)
#pragma unroll
    for (int k = 0; k < 3; ++k) Ue[n][k] = Uc[n][k];
  StaticFor<0, 4>::run([&](auto kc) {
    constexpr int fn = face_node(FC, decltype(kc)::value);
    double s[3];
    load3(a.sideU, nd[fn], s);
#pragma unroll
    for (int k = 0; k < 3; ++k) Ue[fn][k] = TF(s[k]);
  });
  // bilinear face shape at the face ip (identity when shifted)
  TF muB;
  if (USH) {
    muB = mu[f0];
  } else {
    muB = TF(0.5625) * mu[f0] + TF(0.1875) * mu[f1] + TF(0.0625) * mu[f2] + TF(0.1875) * mu[f3];
  }
  const TF amag = sqrt(Af[0] * Af[0] + Af[1] * Af[1] + Af[2] * Af[2]);
  TF nx[3], ax[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    nx[i] = Af[i] / amag;
    ax[i] = Af[i];
  }
  StaticFor<0, 8>::run([&](auto nc) {
    constexpr int n = decltype(nc)::value;
    if (!grad_is_zero<PT, n>()) {
      constexpr bool on_face = (n == f0 || n == f1 || n == f2 || n == f3);
      constexpr int sl = nb_slot(n);
      TF g[3];
      grad_n<PT, n, TF>(J, g);
#pragma unroll
      for (int j = 0; j < 3; ++j) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const TF om = TF(1) - nx[i] * nx[i];
          TF lf = -muB * g[j] * ax[j] * om;
          if (!on_face) {
            if (sl < 0) diag[3 * i + i] += lf; else nb[sl][3 * i + i] += lf;
          }
          rhs[i] -= lf * Ue[n][i];
          lf = -muB * g[i] * ax[j] * om;
          if (!on_face) {
            if (sl < 0) diag[3 * i + j] += lf; else nb[sl][3 * i + j] += lf;
          }
          rhs[i] -= lf * Ue[n][j];
#pragma unroll
          for (int l = 0; l < 3; ++l) {
            if (l == i) continue;
            const TF nil = nx[i] * nx[l];
            lf = muB * g[j] * ax[j] * nil;
            if (!on_face) {
              if (sl < 0) diag[3 * i + l] += lf; else nb[sl][3 * i + l] += lf;
            }
            rhs[i] -= lf * Ue[n][l];
            lf = muB * g[l] * ax[j] * nil;
            if (!on_face) {
              if (sl < 0) diag[3 * i + j] += lf; else nb[sl][3 * i + j] += lf;
            }
            rhs[i] -= lf * Ue[n][j];
          }
        }
      }
    }
  });
}

// Symmetry-plane term at the exposed ip of canonical face FC nearest corner 0
// (navierStokesAssemblerElemBoundaryConditions.cpp:2082-2375 with
// IP_FULL_STRESS__, :295-344): the full viscous stress of the element's own
// velocities, -mu (dU_i/dx_j + dU_j/dx_i) A_j, every node's coefficient in
// the row (the bulk term vanishes for the incompressible fluid).
template <int FC, bool USH, bool UGSH, class TF>
__device__ __forceinline__ void sym_face(const TF (&x)[8][3], const TF (&Uc)[8][3], const TF (&mu)[8],
                                         TF (&diag)[9], TF (&nb)[3][9], TF (&rhs)[3], int* err) {
  constexpr int f0 = face_node(FC, 0), f1 = face_node(FC, 1), f2 = face_node(FC, 2), f3 = face_node(FC, 3);
  TF Af[3];
  face_area_at_first<TF>(x[f0], x[f1], x[f2], x[f3], Af);
  using PT = FacePt<FC, 0, UGSH>;
  const InvJacR<TF> J = inv_jacobian<PT, TF>(x, err);
  TF muB;
  if (USH) {
    muB = mu[f0];
  } else {
    muB = TF(0.5625) * mu[f0] + TF(0.1875) * mu[f1] + TF(0.0625) * mu[f2] + TF(0.1875) * mu[f3];
  }
  StaticFor<0, 8>::run([&](auto nc) {
    constexpr int n = decltype(nc)::value;
    if (!grad_is_zero<PT, n>()) {
      constexpr int sl = nb_slot(n);
      TF g[3];
      grad_n<PT, n, TF>(J, g);
      const TF ga = g[0] * Af[0] + g[1] * Af[1] + g[2] * Af[2];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const TF lf = -muB * g[i] * Af[j] + (i == j ? -muB * ga : TF(0));
          if (sl < 0) diag[3 * i + j] += lf; else nb[sl][3 * i + j] += lf;
          rhs[i] -= lf * Uc[n][j];
        }
      }
    }
  });
}

// VAR 1: the variant with the optional terms (high-resolution deferred
// correction, transient node terms, SIMPLEC / fractional-step coefficients),
// each switched at run time; VAR 2: the fused u/v/w/k/omega variant, which
// also assembles the two turbulence transport equations from the same ip
// geometry (upwind advection with the same mass flows, diffusion with the
// nodal diffusivities at the ips: phiAssemblerElemTerms.hpp:11-413, N = 1);
// VAR 0 is the steady upwind SIMPLE assembly with nothing else in its
// register budget.
template <int LPR, bool USH, bool UGSH, class TF, int VAR = 0>
__global__ void __launch_bounds__(BLOCK, sizeof(TF) == 4 ? (UGSH ? 4 : 3) : 1)
    k_momentum(MomArgs a) {
  constexpr bool EXT = VAR == 1;
  constexpr bool TURB = VAR == 2;
  __shared__ TF sh_val[BLOCK * 3 * 9];
  const int lane = threadIdx.x & 31;
  const int warp_base = threadIdx.x & ~31;
  const RowLane<LPR> rl = row_lane<LPR>(a.m);
  const int row = rl.row, li = rl.li, e = rl.e, c = rl.c;
  const bool rv = rl.rv;
  TF diag[9], nb[3][9], rhs[3];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    diag[k] = TF(0);
    nb[0][k] = nb[1][k] = nb[2][k] = TF(0);
  }
  rhs[0] = rhs[1] = rhs[2] = TF(0);
  // element corner nodes and coordinates in the lane's canonical frame (kept
  // for the turbulence pass of the fused variant)
  int nd[8];
  TF x[8][3];
  if (e >= 0) {
    const uint32_t pw = perm_word(c);
    const uint32_t iw = ip_word(c);
    // coordinates of the flux arithmetic: FP64 as gathered, or, in the mixed
    // form, the element's FP32 corner offsets from its corner 0 (the Jacobians
    // are translation invariant), one 16-byte load per corner, with U and mu
    // from the FP32 node copy (one 16-byte load per node)
    TF Uc[8][3], mu[8];
    if constexpr (sizeof(TF) == 4) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int pk = perm_at(pw, k);
        nd[k] = __ldg(a.m.conn + 8 * e + pk);
        const float4 t = __ldg(a.xloc + 8 * (size_t)e + pk);
        x[k][0] = t.x;
        x[k][1] = t.y;
        x[k][2] = t.z;
        const float4 u = __ldg(a.umu + nd[k]);
        Uc[k][0] = u.x;
        Uc[k][1] = u.y;
        Uc[k][2] = u.z;
        mu[k] = u.w;
      }
    } else {
      double xg[8][3];
      gather_x(a.m, e, pw, xg, nd);
#pragma unroll
      for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int i = 0; i < 3; ++i) x[k][i] = TF(xg[k][i]);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        double u[3];
        load3(a.U, nd[k], u);
        Uc[k][0] = TF(u[0]);
        Uc[k][1] = TF(u[1]);
        Uc[k][2] = TF(u[2]);
        mu[k] = TF(__ldg(a.mu + nd[k]));
      }
    }
    int err = 0;
    StaticFor<0, 3>::run([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      constexpr int IP = q == 0 ? 0 : (q == 1 ? 3 : 8);
      // this ip's SCS area from the static per-element table
      double Aip[3];
      load_area(a.m, e, (iw >> (5 * q)) & 31, Aip);
      constexpr int R = q == 0 ? 1 : (q == 1 ? 3 : 4);
      constexpr int RS = nb_slot(R);
      using PG = ScsPt<IP, UGSH>;
      using PV = ScsPt<IP, USH>;
      const int pk = (iw >> (5 * q)) & 31;
      const double tmd = (pk & 1) ? -__ldg(a.mDot + 12 * e + (pk >> 1)) : __ldg(a.mDot + 12 * e + (pk >> 1));
      const TF tm = TF(tmd);
      TF muIp = TF(0);
      StaticFor<0, 8>::run([&](auto nc) {
        constexpr int n = decltype(nc)::value;
        constexpr double N = shape_at<PV, n>();
        if (N != 0.0) muIp += TF(N) * mu[n];
      });
      // upwind advection (row L = corner 0)
      const TF fl = TF(0.5) * (tm + fabs(tm));
      const TF fr = TF(0.5) * (tm - fabs(tm));
      // high resolution: deferred correction beta_up,i (x_ip - x_up) . grad
      // u_i,up on the rhs (navierStokesAssemblerElemTerms.cpp:287-330), x_ip
      // from the standard trilinear coordinate shape functions
      TF dcorr[3] = {TF(0), TF(0), TF(0)};
      if (EXT && a.hr) {
        using PC = ScsPt<IP, false>;
        TF dx[3];
        const int ku = tmd > 0 ? 0 : R;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          TF xi = TF(0);
          StaticFor<0, 8>::run([&](auto nc) {
            constexpr int n = decltype(nc)::value;
            constexpr double N = shape_at<PC, n>();
            if (N != 0.0) xi += TF(N) * x[n][j];
          });
          dx[j] = xi - (tmd > 0 ? x[0][j] : x[R][j]);
        }
        const int nu = ku == 0 ? row : __ldg(a.m.conn + 8 * e + perm_at(pw, R));
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const TF bu = TF(__ldg(a.betaU + 3 * nu + i));
          TF g = TF(0);
#pragma unroll
          for (int j = 0; j < 3; ++j) g += TF(__ldg(a.gradU + 9 * nu + 3 * i + j)) * dx[j];
          dcorr[i] = bu * g;
        }
      }
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const TF up = tmd > 0 ? Uc[0][i] : Uc[R][i];
        rhs[i] -= tm * (up + dcorr[i]);
        diag[3 * i + i] += fl;
        nb[RS][3 * i + i] += fr;
      }
      // viscous stress incl. transpose. Block of column n:
      //   -mu_ip (g_n . A) I - mu_ip A (x) g_n   (rows i, columns j: g_n,i A_j)
      // Its defect contribution summed over the eight columns is
      //   rhs += mu_ip (G A + G^T A), G = grad U at the ip,
      // taken through the parametric gradient; only the three edge neighbours
      // keep their own blocks, and the diagonal block, which takes every other
      // column, is minus their sum (partition of unity: sum_n g_n = 0).
      const InvJacR<TF> J = inv_jacobian<PG, TF>(x, &err);
      TF ax[3] = {TF(Aip[0]), TF(Aip[1]), TF(Aip[2])};
      TF Gs[3][3] = {{TF(0), TF(0), TF(0)}, {TF(0), TF(0), TF(0)}, {TF(0), TF(0), TF(0)}};
      StaticFor<0, 8>::run([&](auto nc) {
        constexpr int n = decltype(nc)::value;
        constexpr double d0 = dshape(n, 0, PG::s(0), PG::s(1), PG::s(2));
        constexpr double d1 = dshape(n, 1, PG::s(0), PG::s(1), PG::s(2));
        constexpr double d2 = dshape(n, 2, PG::s(0), PG::s(1), PG::s(2));
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          if (d0 != 0.0) Gs[i][0] += TF(d0) * Uc[n][i];
          if (d1 != 0.0) Gs[i][1] += TF(d1) * Uc[n][i];
          if (d2 != 0.0) Gs[i][2] += TF(d2) * Uc[n][i];
        }
      });
      TF G[3][3];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) G[i][j] = Gs[i][0] * J.s[0][j] + Gs[i][1] * J.s[1][j] + Gs[i][2] * J.s[2][j];
#pragma unroll
      for (int i = 0; i < 3; ++i)
        rhs[i] += muIp * (G[i][0] * ax[0] + G[i][1] * ax[1] + G[i][2] * ax[2] + G[0][i] * ax[0] + G[1][i] * ax[1] +
                          G[2][i] * ax[2]);
      StaticFor<1, 5>::run([&](auto nc) {
        constexpr int n = decltype(nc)::value;
        constexpr int sl = nb_slot(n);
        if (sl >= 0 && !grad_is_zero<PG, n>()) {
          TF g[3];
          grad_n<PG, n, TF>(J, g);
          const TF ga = g[0] * ax[0] + g[1] * ax[1] + g[2] * ax[2];
#pragma unroll
          for (int i = 0; i < 3; ++i) {
#pragma unroll
            for (int j = 0; j < 3; ++j) {
              const TF fj = -muIp * g[i] * ax[j] + (i == j ? -muIp * ga : TF(0));
              nb[sl][3 * i + j] += fj;
              diag[3 * i + j] -= fj;
            }
          }
        }
      });
    });
    // no-slip wall faces and symmetry faces touching this corner
    const uint8_t sm = a.m.sym_mask ? __ldg(a.m.sym_mask + e) : uint8_t(0);
    const uint8_t fm = __ldg(a.m.face_mask + e) & uint8_t(~sm);
    if (fm) {
      const uint32_t fw = face_word(c);
      if (fm & (1u << ((fw >> 0) & 7))) wall_face<0, USH, UGSH, TF>(a, x, nd, Uc, mu, diag, nb, rhs, &err);
      if (fm & (1u << ((fw >> 3) & 7))) wall_face<3, USH, UGSH, TF>(a, x, nd, Uc, mu, diag, nb, rhs, &err);
      if (fm & (1u << ((fw >> 6) & 7))) wall_face<4, USH, UGSH, TF>(a, x, nd, Uc, mu, diag, nb, rhs, &err);
    }
    if (sm) {
      const uint32_t fw = face_word(c);
      if (sm & (1u << ((fw >> 0) & 7))) sym_face<0, USH, UGSH, TF>(x, Uc, mu, diag, nb, rhs, &err);
      if (sm & (1u << ((fw >> 3) & 7))) sym_face<3, USH, UGSH, TF>(x, Uc, mu, diag, nb, rhs, &err);
      if (sm & (1u << ((fw >> 6) & 7))) sym_face<4, USH, UGSH, TF>(x, Uc, mu, diag, nb, rhs, &err);
    }
    if (err) a.err[0] = 1;
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) diag[k] = rowsum<LPR>(diag[k]);
#pragma unroll
  for (int k = 0; k < 3; ++k) rhs[k] = rowsum<LPR>(rhs[k]);
  // SIMPLEC: sum of the row's off-diagonal (i, i) coefficients (the CSR
  // off-diagonal entries are the lanes' neighbour blocks summed)
  double off[3] = {0.0, 0.0, 0.0};
  if (EXT && a.du_mode == 1)
#pragma unroll
    for (int k = 0; k < 3; ++k) off[k] = double(rowsum<LPR>(TF(nb[0][4 * k] + nb[1][4 * k] + nb[2][4 * k])));
  if (rv) {
    // node terms, relaxation, wall rhs relaxation, DU
    const double vol = __ldg(a.m.vol + row);
    const double dv = __ldg(a.div + row);
    const double rho = __ldg(a.rho + row);
    const double lf = rho * vol / a.dt;
    double un[3], gp[3], uo[3] = {0.0, 0.0, 0.0}, uoo[3] = {0.0, 0.0, 0.0};
    load3(a.U, row, un);
    load3(a.gradP, row, gp);
    const int order = EXT ? a.order : 0;
    if (order >= 1) load3(a.Uold, row, uo);
    if (order == 2) load3(a.Uoldold, row, uoo);
    const bool wall = __ldg(a.m.wall_node + row) != 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double d = double(diag[4 * k]);
      double r = double(rhs[k]);
      if (order == 0) {
        // steady: false transient with the physical timescale
        if (dv < 0) d += -dv;
        d += lf;
      } else {
        // BDF1 / BDF2 node terms (navierStokesAssemblerNodeTerms.cpp:151-427),
        // density constant in time
        const double f0 = a.tk0 * lf, f1 = a.tk1 * lf, f2 = a.tk2 * lf;
        d += f0;
        r -= order == 1 ? (f0 * un[k] + f1 * uo[k]) : (f0 * un[k] + f1 * uo[k] + f2 * uoo[k]);
        if (dv < 0) d += -dv;
      }
      d *= a.urf_inv;
      diag[4 * k] = TF(d);
      r -= -dv * un[k];
      r -= gp[k] * vol;
      if (wall) r *= a.wall_relax;
      rhs[k] = TF(r);
    }
    if (li == 0) {
      // computeDUCoefficients (navierStokesAssembler.cpp:84-232): V / (a_ii +
      // SMALL), or dt / rho (fractional step, steady gamma1 = 1); SIMPLEC also
      // D~ = V / (a_ii + off-diagonal sum + SMALL)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int du_mode = EXT ? a.du_mode : 0;
        a.du[3 * row + k] = du_mode == 2 ? (order ? a.dt / a.tk0 / rho : a.dt / rho)
                                         : vol / (double(diag[4 * k]) + SMALL);
        if (du_mode == 1) a.duT[3 * row + k] = vol / (double(diag[4 * k]) + off[k] + SMALL);
        static_cast<TF*>(a.b)[3 * row + k] = rhs[k];
      }
    }
  }
  write_row<9, TF, LPR>(row, rv, li, lane, diag, nb, a.m, static_cast<TF*>(a.A), sh_val + warp_base * 3 * 9, false);
  if constexpr (TURB) {
    // Second pass over the lane's three ips for k and omega, after the momentum
    // row is written (its accumulators are dead, so the pass fits the same
    // register budget): the inverse Jacobian is formed again from the corner
    // coordinates still held, the mass flow and area come back from L1/L2.
    // Upwind advection with the momentum's mass flows; diffusion -Gamma_ip
    // grad N . A with the diffusivities at the ip on the velocity's shape
    // functions; [0] k, [1] omega.
    TF tdiag[2] = {TF(0), TF(0)}, tnb[2][3] = {{TF(0), TF(0), TF(0)}, {TF(0), TF(0), TF(0)}};
    TF trhs[2] = {TF(0), TF(0)};
    if (e >= 0) {
      const uint32_t iw = ip_word(c);
      TF tph[2][8], tgam[2][8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        tph[0][k] = TF(__ldg(a.kf + nd[k]));
        tph[1][k] = TF(__ldg(a.wf + nd[k]));
        tgam[0][k] = TF(__ldg(a.gkf + nd[k]));
        tgam[1][k] = TF(__ldg(a.gwf + nd[k]));
      }
      int err = 0;
      StaticFor<0, 3>::run([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        constexpr int IP = q == 0 ? 0 : (q == 1 ? 3 : 8);
        constexpr int R = q == 0 ? 1 : (q == 1 ? 3 : 4);
        constexpr int RS = nb_slot(R);
        using PG = ScsPt<IP, UGSH>;
        using PV = ScsPt<IP, USH>;
        double Aip[3];
        load_area(a.m, e, (iw >> (5 * q)) & 31, Aip);
        const TF ax[3] = {TF(Aip[0]), TF(Aip[1]), TF(Aip[2])};
        const int pk = (iw >> (5 * q)) & 31;
        const double tmd = (pk & 1) ? -__ldg(a.mDot + 12 * e + (pk >> 1)) : __ldg(a.mDot + 12 * e + (pk >> 1));
        const TF tm = TF(tmd);
        const TF fl = TF(0.5) * (tm + fabs(tm));
        const TF fr = TF(0.5) * (tm - fabs(tm));
        const InvJacR<TF> J = inv_jacobian<PG, TF>(x, &err);
        TF tgIp[2] = {TF(0), TF(0)};
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          StaticFor<0, 8>::run([&](auto nc) {
            constexpr int n = decltype(nc)::value;
            constexpr double N = shape_at<PV, n>();
            if (N != 0.0) tgIp[t] += TF(N) * tgam[t][n];
          });
          trhs[t] -= tm * (tmd > 0 ? tph[t][0] : tph[t][R]);
          tdiag[t] += fl;
          tnb[t][RS] += fr;
        }
        {
          // diffusion defect: rhs += Gamma_ip grad(phi)_ip . A
#pragma unroll
          for (int t = 0; t < 2; ++t) {
            TF Gp[3] = {TF(0), TF(0), TF(0)};
            StaticFor<0, 8>::run([&](auto nc) {
              constexpr int n = decltype(nc)::value;
              constexpr double d0 = dshape(n, 0, PG::s(0), PG::s(1), PG::s(2));
              constexpr double d1 = dshape(n, 1, PG::s(0), PG::s(1), PG::s(2));
              constexpr double d2 = dshape(n, 2, PG::s(0), PG::s(1), PG::s(2));
              if (d0 != 0.0) Gp[0] += TF(d0) * tph[t][n];
              if (d1 != 0.0) Gp[1] += TF(d1) * tph[t][n];
              if (d2 != 0.0) Gp[2] += TF(d2) * tph[t][n];
            });
            TF gax = TF(0);
#pragma unroll
            for (int j = 0; j < 3; ++j) gax += (Gp[0] * J.s[0][j] + Gp[1] * J.s[1][j] + Gp[2] * J.s[2][j]) * ax[j];
            trhs[t] += tgIp[t] * gax;
          }
        }
        StaticFor<1, 5>::run([&](auto nc) {
          constexpr int n = decltype(nc)::value;
          constexpr int sl = nb_slot(n);
          if (sl >= 0 && !grad_is_zero<PG, n>()) {
            TF g[3];
            grad_n<PG, n, TF>(J, g);
            const TF ga = g[0] * ax[0] + g[1] * ax[1] + g[2] * ax[2];
#pragma unroll
            for (int t = 0; t < 2; ++t) {
              const TF ft = -tgIp[t] * ga;
              tnb[t][sl] += ft;
              tdiag[t] -= ft;
            }
          }
        });
      });
      if (err) a.err[0] = 1;
    }
    // k and omega rows: node source terms (the SST node update's diagonal and
    // rhs), relaxation of the diagonal (phiAssembler.h:967-1006)
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      TF td[1] = {rowsum<LPR>(tdiag[t])};
      TF tr = rowsum<LPR>(trhs[t]);
      if (rv) {
        const double d = (double(td[0]) + __ldg((t ? a.sdw : a.sdk) + row)) * (t ? a.urf_w_inv : a.urf_k_inv);
        td[0] = TF(d);
        tr = TF(double(tr) + __ldg((t ? a.srw : a.srk) + row));
        if (li == 0) static_cast<TF*>(t ? a.bw : a.bk)[row] = tr;
      }
      TF tnbt[3][1] = {{tnb[t][0]}, {tnb[t][1]}, {tnb[t][2]}};
      write_row<1, TF, LPR>(row, rv, li, lane, td, tnbt, a.m, static_cast<TF*>(t ? a.Aw : a.Ak),
                            sh_val + warp_base * 3 * 9, false);
    }
  }
}

// ---------------------------------------------------------------------------
// Mass flow: element kernels over all 12 SCS ips.
struct MdotArgs {
  MeshView m;
  const double *U, *p, *gradP, *du, *rho;
  const double* du_lhs;  // diffusivity of the pressure-correction lhs: D, or D~ with SIMPLEC
  double* mDot;
  double* flux;  // [ne][12] pressure-correction ip fluxes (staging modes)
  void* coef;    // [ne][8][3] pressure-correction lhs coefficients per corner (staging modes)
  double urf;
  int init;       // initial mass flow rho U.A (no Rhie-Chow term, no fluxes)
  int flux_only;  // write the fluxes from the current mass flow, leave it unchanged
  int* err;
};

// Full 27-point subdivision and 12 SCS area vectors (hex_scs_det).
__device__ __forceinline__ void scs_areas_all(const double (&x)[8][3], double (&A)[12][3]) {
  double p[27][3];
#pragma unroll
  for (int n = 0; n < 8; ++n)
#pragma unroll
    for (int k = 0; k < 3; ++k) p[n][k] = x[n][k];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    p[8][k] = 0.5 * (x[0][k] + x[1][k]);
    p[9][k] = 0.5 * (x[1][k] + x[2][k]);
    p[10][k] = 0.5 * (x[2][k] + x[3][k]);
    p[11][k] = 0.5 * (x[3][k] + x[0][k]);
    p[12][k] = 0.25 * (x[0][k] + x[1][k] + x[2][k] + x[3][k]);
    p[13][k] = 0.5 * (x[4][k] + x[5][k]);
    p[14][k] = 0.5 * (x[5][k] + x[6][k]);
    p[15][k] = 0.5 * (x[6][k] + x[7][k]);
    p[16][k] = 0.5 * (x[7][k] + x[4][k]);
    p[17][k] = 0.25 * (x[4][k] + x[5][k] + x[6][k] + x[7][k]);
    p[18][k] = 0.5 * (x[1][k] + x[5][k]);
    p[19][k] = 0.5 * (x[0][k] + x[4][k]);
    p[20][k] = 0.25 * (x[0][k] + x[1][k] + x[4][k] + x[5][k]);
    p[21][k] = 0.5 * (x[3][k] + x[7][k]);
    p[22][k] = 0.5 * (x[2][k] + x[6][k]);
    p[23][k] = 0.25 * (x[2][k] + x[3][k] + x[6][k] + x[7][k]);
    p[24][k] = 0.25 * (x[1][k] + x[2][k] + x[5][k] + x[6][k]);
    p[25][k] = 0.25 * (x[0][k] + x[3][k] + x[4][k] + x[7][k]);
    double s = 0.0;
#pragma unroll
    for (int n = 0; n < 8; ++n) s += x[n][k];
    p[26][k] = 0.125 * s;
  }
  constexpr int Q[12][4] = {{20, 8, 12, 26},  {24, 9, 12, 26},  {10, 12, 26, 23}, {11, 25, 26, 12},
                            {13, 20, 26, 17}, {17, 14, 24, 26}, {17, 15, 23, 26}, {16, 17, 26, 25},
                            {19, 20, 26, 25}, {20, 18, 24, 26}, {22, 23, 26, 24}, {21, 25, 26, 23}};
#pragma unroll
  for (int ip = 0; ip < 12; ++ip) quad_area(p[Q[ip][0]], p[Q[ip][1]], p[Q[ip][2]], p[Q[ip][3]], A[ip]);
}

// Static SCS area table [ne][12][3] (hex_scs_det; the mesh does not move), read
// by the assembly, mass-flow and gradient kernels instead of recomputing the
// element subdivision in every lane.
__global__ void __launch_bounds__(BLOCK) k_scs_area(MeshView m) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.ne) return;
  double x[8][3];
  int nd[8];
  gather_x(m, e, perm_word(0), x, nd);
  double A[12][3];
  scs_areas_all(x, A);
#pragma unroll
  for (int ip = 0; ip < 12; ++ip)
#pragma unroll
    for (int k = 0; k < 3; ++k) m.scs_area[36L * e + 3 * ip + k] = A[ip][k];
}

int launch_scs_area(DeviceMesh& m, cudaStream_t st) {
  k_scs_area<<<(m.ne + BLOCK - 1) / BLOCK, BLOCK, 0, st>>>(m.view());
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

// initializeMassFlowRateInterior_ (flowModel.cpp:3303-3470) when init != 0,
// otherwise updateMassFlowRateInterior_ (flowModel.cpp:5272-5687).
//
// STAGE: also write the pressure-correction ip fluxes and corner coefficients
// (TC: the matrix precision); without it the kernel keeps the register budget
// of four blocks per SM.
// SC (staging with SIMPLEC): the staged lhs coefficients take D~ (du_lhs)
// while the fluxes keep D.
template <bool USH, bool PGSH, class TC, bool STAGE, bool SC = false>
__global__ void __launch_bounds__(BLOCK, STAGE ? 3 : 4) k_mdot(MdotArgs a) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.m.ne) return;
  double x[8][3];
  int nd[8];
  gather_x(a.m, e, perm_word(0), x, nd);
  double Gp[3] = {0.0, 0.0, 0.0}, pn[8];
  if (!a.init) {
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      const double w = __ldg(a.m.wscv + 8 * e + n);
      double gp[3];
      load3(a.gradP, nd[n], gp);
#pragma unroll
      for (int j = 0; j < 3; ++j) Gp[j] += w * gp[j];
      pn[n] = __ldg(a.p + nd[n]);
    }
  }
  int err = 0;
  TC coef[8][3];
#pragma unroll
  for (int k = 0; k < 8; ++k) coef[k][0] = coef[k][1] = coef[k][2] = TC(0);
  StaticFor<0, 12>::run([&](auto ic) {
    constexpr int IP = decltype(ic)::value;
    using PV = ScsPt<IP, USH>;
    using PG = ScsPt<IP, PGSH>;
    double u[3] = {0, 0, 0}, duip[3] = {0, 0, 0}, dulip[3] = {0, 0, 0}, rhoIp = 0.0;
    constexpr bool simplec = STAGE && SC;
    StaticFor<0, 8>::run([&](auto nc) {
      constexpr int n = decltype(nc)::value;
      constexpr double N = shape_at<PV, n>();
      if (N != 0.0) {
        double un[3];
        load3(a.U, nd[n], un);
        rhoIp += N * __ldg(a.rho + nd[n]);
#pragma unroll
        for (int j = 0; j < 3; ++j) u[j] += N * un[j];
        if (!a.init) {
          double dn[3];
          load3(a.du, nd[n], dn);
#pragma unroll
          for (int j = 0; j < 3; ++j) duip[j] += N * dn[j];
          if (simplec) {
            load3(a.du_lhs, nd[n], dn);
#pragma unroll
            for (int j = 0; j < 3; ++j) dulip[j] += N * dn[j];
          }
        }
      }
    });
    if (!simplec)
#pragma unroll
      for (int j = 0; j < 3; ++j) dulip[j] = duip[j];
    double Aip[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) Aip[k] = __ldg(a.m.scs_area + 36L * e + 3 * IP + k);
    double m = 0.0;
    if (a.init) {
#pragma unroll
      for (int j = 0; j < 3; ++j) m += rhoIp * u[j] * Aip[j];
      a.mDot[12 * e + IP] = m;
    } else {
      const InvJac J = inv_jacobian<PG>(x, &err);
      // grad p at the ip through the parametric gradient: dp = J^-T sum_n dN_n/ds p_n
      double dps[3] = {0.0, 0.0, 0.0};
      StaticFor<0, 8>::run([&](auto nc) {
        constexpr int n = decltype(nc)::value;
        constexpr double d0 = dshape(n, 0, PG::s(0), PG::s(1), PG::s(2));
        constexpr double d1 = dshape(n, 1, PG::s(0), PG::s(1), PG::s(2));
        constexpr double d2 = dshape(n, 2, PG::s(0), PG::s(1), PG::s(2));
        if (d0 != 0.0) dps[0] += d0 * pn[n];
        if (d1 != 0.0) dps[1] += d1 * pn[n];
        if (d2 != 0.0) dps[2] += d2 * pn[n];
      });
      double dp[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) dp[i] = J.s[0][i] * dps[0] + J.s[1][i] * dps[1] + J.s[2][i] * dps[2];
      const double old = a.mDot[12 * e + IP];
      double now = old;
      if (!a.flux_only) {
        const double tU = old / rhoIp;
        const double rhoUp = tU > 0 ? __ldg(a.rho + nd[lr(IP, 0)]) : __ldg(a.rho + nd[lr(IP, 1)]);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          m += rhoUp * u[j] * Aip[j];
          m -= rhoUp * duip[j] * (dp[j] - Gp[j]) * Aip[j];
        }
        now = a.urf * m + (1.0 - a.urf) * old;
        a.mDot[12 * e + IP] = now;
      }
      if constexpr (STAGE) {
        // the pressure-correction right-hand side's flux at this ip: the same
        // Rhie-Chow velocity with the density upwinded by the new mass flow
        // (pressureCorrectionAssemblerElemTerms.cpp:17-616, as the oracle's
        // assemble_pcorr forms it per ip)
        const double rhoHR = now > 0 ? __ldg(a.rho + nd[lr(IP, 0)]) : __ldg(a.rho + nd[lr(IP, 1)]);
        double mm = 0.0;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          mm += rhoHR * u[j] * Aip[j];
          mm -= rhoHR * duip[j] * (dp[j] - Gp[j]) * Aip[j];
        }
        a.flux[12 * e + IP] = mm;
        // lhs: the flux's dependence on the pressure correction, -rhoHR DU_ip
        // A . grad N_n, for the edge neighbours of L (added to L's row) and of
        // R (subtracted from R's row: the ip's area points away from L)
        constexpr int L = lr(IP, 0), R = lr(IP, 1);
        const double w[3] = {-rhoHR * dulip[0] * Aip[0], -rhoHR * dulip[1] * Aip[1], -rhoHR * dulip[2] * Aip[2]};
        StaticFor<0, 3>::run([&](auto sc) {
          constexpr int sl = decltype(sc)::value;
          constexpr int nl = edge_nbr(L, sl), nr = edge_nbr(R, sl);
          if (!grad_is_zero<PG, nl>()) {
            double g[3];
            grad_n<PG, nl>(J, g);
            coef[L][sl] += TC(w[0] * g[0] + w[1] * g[1] + w[2] * g[2]);
          }
          if (!grad_is_zero<PG, nr>()) {
            double g[3];
            grad_n<PG, nr>(J, g);
            coef[R][sl] -= TC(w[0] * g[0] + w[1] * g[1] + w[2] * g[2]);
          }
        });
      }
    }
  });
  if constexpr (STAGE) {
    TC* out = static_cast<TC*>(a.coef) + 24 * (size_t)e;
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
      for (int sl = 0; sl < 3; ++sl) out[3 * k + sl] = coef[k][sl];
  }
  if (err) a.err[0] = 1;
}

// ---------------------------------------------------------------------------
// Divergence: div_n = sum of outgoing SCS mass flows (interior part of
// updateMassDivergenceField_; wall side flows are zero).
struct DivArgs {
  MeshView m;
  const double* mDot;
  double* div;
  // transient contribution (flowModel.cpp:13556-13700, fixed mesh, density
  // constant in time): (tk0 + tk1 [+ tk2]) rho V / dt
  const double* rho;
  int order;
  double tk0, tk1, tk2, dt;
};

template <int LPR>
__global__ void __launch_bounds__(BLOCK) k_div(DivArgs a) {
  const RowLane<LPR> rl = row_lane<LPR>(a.m);
  const int row = rl.row, li = rl.li, e = rl.e, c = rl.c;
  const bool rv = rl.rv;
  double s = 0.0;
  if (e >= 0) {
    const uint32_t iw = ip_word(c);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int pk = (iw >> (5 * q)) & 31;
      const double m = __ldg(a.mDot + 12 * e + (pk >> 1));
      s += (pk & 1) ? -m : m;
    }
  }
  s = rowsum<LPR>(s);
  if (rv && li == 0) {
    if (a.order) {
      const double rho = __ldg(a.rho + row), vol = __ldg(a.m.vol + row);
      s += (a.order == 1 ? (a.tk0 * rho + a.tk1 * rho) : (a.tk0 * rho + a.tk1 * rho + a.tk2 * rho)) * vol / a.dt;
    }
    a.div[row] = s;
  }
}

// ---------------------------------------------------------------------------
// Green-Gauss nodal gradient with under-relaxation and incremental form
// (nodeField::updateGradientField, nodeField.hpp:3253-3445 interior,
// :4732-4930 boundary faces). NC = field components.
struct GradArgs {
  MeshView m;
  const double* phi;
  double* grad;
  double gurf;
};

template <int LPR, int NC, bool SH>
__global__ void __launch_bounds__(BLOCK) k_gradient(GradArgs a) {
  const RowLane<LPR> rl = row_lane<LPR>(a.m);
  const int row = rl.row, li = rl.li, e = rl.e, c = rl.c;
  const bool rv = rl.rv;
  double acc[NC][3];
#pragma unroll
  for (int i = 0; i < NC; ++i) acc[i][0] = acc[i][1] = acc[i][2] = 0.0;
  if (e >= 0) {
    const uint32_t pw = perm_word(c);
    double x[8][3];
    int nd[8];
    gather_x(a.m, e, pw, x, nd);
    double ph[8][NC];
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
      for (int i = 0; i < NC; ++i) ph[k][i] = __ldg(a.phi + NC * nd[k] + i);
    const uint32_t iw = ip_word(c);
    double Aq[3][3];
#pragma unroll
    for (int q = 0; q < 3; ++q) load_area(a.m, e, (iw >> (5 * q)) & 31, Aq[q]);
    StaticFor<0, 3>::run([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      constexpr int IP = q == 0 ? 0 : (q == 1 ? 3 : 8);
      using PV = ScsPt<IP, SH>;
      double pip[NC];
#pragma unroll
      for (int i = 0; i < NC; ++i) pip[i] = 0.0;
      StaticFor<0, 8>::run([&](auto nc) {
        constexpr int n = decltype(nc)::value;
        constexpr double N = shape_at<PV, n>();
        if (N != 0.0) {
#pragma unroll
          for (int i = 0; i < NC; ++i) pip[i] += N * ph[n][i];
        }
      });
#pragma unroll
      for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) acc[i][j] += (pip[i] - ph[0][i]) * Aq[q][j];
    });
    if (!SH) {
      // boundary faces: bilinear face value at the face ip nearest the node;
      // symmetry faces add nothing (nodeField.hpp:4764)
      const uint8_t fm = __ldg(a.m.face_mask + e) & uint8_t(a.m.sym_mask ? ~__ldg(a.m.sym_mask + e) : 0xff);
      if (fm) {
        const uint32_t fw = face_word(c);
        StaticFor<0, 3>::run([&](auto qc) {
          constexpr int q = decltype(qc)::value;
          constexpr int FC = q == 0 ? 0 : (q == 1 ? 3 : 4);
          if (fm & (1u << ((fw >> (3 * q)) & 7))) {
            constexpr int f0 = face_node(FC, 0), f1 = face_node(FC, 1), f2 = face_node(FC, 2),
                          f3 = face_node(FC, 3);
            double Af[3];
            face_area_at_first(x[f0], x[f1], x[f2], x[f3], Af);
#pragma unroll
            for (int i = 0; i < NC; ++i) {
              const double pip = 0.5625 * ph[f0][i] + 0.1875 * ph[f1][i] + 0.0625 * ph[f2][i] +
                                 0.1875 * ph[f3][i];
#pragma unroll
              for (int j = 0; j < 3; ++j) acc[i][j] += (pip - ph[0][i]) * Af[j];
            }
          }
        });
      }
    }
  }
#pragma unroll
  for (int i = 0; i < NC; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) acc[i][j] = rowsum<LPR>(acc[i][j]);
  if (rv && li == 0) {
    const double iv = 1.0 / __ldg(a.m.vol + row);
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const size_t k = (size_t)3 * NC * row + 3 * i + j;
        a.grad[k] = (1.0 - a.gurf) * a.grad[k] + a.gurf * acc[i][j] * iv;
      }
  }
}

// ---------------------------------------------------------------------------
// High-resolution advection: velocity blending factor
// (nodeField::updateMinMaxFields, src/field/nodeField/nodeField.hpp:1843-2066,
// and nodeField::updateBlendingFactorField, :2069-2410 and the relaxation
// after it), row-owner like the assembly: lane c looks at the incident
// element where the row node is corner c.
struct BlendArgs {
  MeshView m;
  const double *U, *gradU;
  double *minU, *maxU, *beta;
  double beta_max;
};

// extrema of every velocity component over the row node and its edge
// neighbours (each SCS ip gives its L node the R value and vice versa)
template <int LPR>
__global__ void __launch_bounds__(BLOCK) k_minmax_u(BlendArgs a) {
  const RowLane<LPR> rl = row_lane<LPR>(a.m);
  const int row = rl.row, li = rl.li, e = rl.e, c = rl.c;
  const bool rv = rl.rv;
  double lo[3], hi[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) lo[i] = hi[i] = rv ? __ldg(a.U + 3 * row + i) : 0.0;
  if (e >= 0) {
    const uint32_t pw = perm_word(c);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int nd = __ldg(a.m.conn + 8 * e + perm_at(pw, k == 0 ? 1 : (k == 1 ? 3 : 4)));
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double v = __ldg(a.U + 3 * nd + i);
        lo[i] = fmin(lo[i], v);
        hi[i] = fmax(hi[i], v);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int o = 1; o < LPR; o <<= 1) {
      lo[i] = fmin(lo[i], __shfl_xor_sync(FULL_MASK, lo[i], o));
      hi[i] = fmax(hi[i], __shfl_xor_sync(FULL_MASK, hi[i], o));
    }
  if (rv && li == 0)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      a.minU[3 * row + i] = lo[i];
      a.maxU[3 * row + i] = hi[i];
    }
}

// limiter of the row node for the point at dx from it (the reference's
// formulas: SMALL-stabilised projected increment, the two-sided ratio, the
// smooth Venkatakrishnan-type map when beta_max < 2)
__device__ __forceinline__ void blend_limit(const BlendArgs& a, const double (&phi)[3], const double (&lo)[3],
                                            const double (&hi)[3], const double (&G)[9], const double (&dx)[3],
                                            double (&beta)[3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double rgrad = G[3 * i] * dx[0] + G[3 * i + 1] * dx[1] + G[3 * i + 2] * dx[2];
    rgrad = rgrad > 0 ? rgrad + SMALL : rgrad - SMALL;
    const double dmax = hi[i] - phi[i], dmin = lo[i] - phi[i];
    const double bl = fmax(dmax / rgrad, dmin / rgrad);
    const double bl12 = fmax(-dmax / rgrad, -dmin / rgrad);
    double y = fmin(bl, bl12);
    if (a.beta_max < 2.0 - SMALL) y = (y * y + 2.0 * y) / (y * y + y + 2.0);
    if (rgrad > 100 * SMALL || rgrad < -100 * SMALL) beta[i] = fmin(beta[i], y);
  }
}

template <int LPR>
__global__ void __launch_bounds__(BLOCK) k_blend_u(BlendArgs a) {
  const RowLane<LPR> rl = row_lane<LPR>(a.m);
  const int row = rl.row, li = rl.li, e = rl.e, c = rl.c;
  const bool rv = rl.rv;
  double beta[3] = {a.beta_max, a.beta_max, a.beta_max};
  if (e >= 0) {
    double phi[3], lo[3], hi[3], G[9];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      phi[i] = __ldg(a.U + 3 * row + i);
      lo[i] = __ldg(a.minU + 3 * row + i);
      hi[i] = __ldg(a.maxU + 3 * row + i);
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) G[k] = __ldg(a.gradU + 9 * row + k);
    double x[8][3];
    int nd[8];
    gather_x(a.m, e, perm_word(c), x, nd);
    // interior SCS ips touching the row node (canonical ips 0, 3, 8)
    StaticFor<0, 3>::run([&](auto qc) {
      constexpr int IP = decltype(qc)::value == 0 ? 0 : (decltype(qc)::value == 1 ? 3 : 8);
      using PC = ScsPt<IP, false>;
      double dx[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        double xi = 0.0;
        StaticFor<0, 8>::run([&](auto nc) {
          constexpr int n = decltype(nc)::value;
          constexpr double N = shape_at<PC, n>();
          if (N != 0.0) xi += N * x[n][j];
        });
        dx[j] = xi - x[0][j];
      }
      blend_limit(a, phi, lo, hi, G, dx, beta);
    });
    // boundary faces at the row node: the face ip nearest to it (standard
    // bilinear face shape functions: 9/16, 3/16, 1/16, 3/16)
    const uint8_t fm = __ldg(a.m.face_mask + e);
    if (fm) {
      const uint32_t fw = face_word(c);
      StaticFor<0, 3>::run([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        constexpr int FC = q == 0 ? 0 : (q == 1 ? 3 : 4);
        if (fm & (1u << ((fw >> (3 * q)) & 7))) {
          constexpr int f1 = face_node(FC, 1), f2 = face_node(FC, 2), f3 = face_node(FC, 3);
          double dx[3];
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const double xi = 0.5625 * x[0][j] + 0.1875 * x[f1][j] + 0.0625 * x[f2][j] + 0.1875 * x[f3][j];
            dx[j] = xi - x[0][j];
          }
          blend_limit(a, phi, lo, hi, G, dx, beta);
        }
      });
    }
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int o = 1; o < LPR; o <<= 1) beta[i] = fmin(beta[i], __shfl_xor_sync(FULL_MASK, beta[i], o));
  if (rv && li == 0)
#pragma unroll
    for (int i = 0; i < 3; ++i) a.beta[3 * row + i] = 0.75 * a.beta[3 * row + i] + 0.25 * beta[i];
}

// U += sign * du * gradP / urf_p on all nodes (segregatedFlowEquations.cpp:134-278)
__global__ void k_vel_correct(int n3, double* U, const double* du, const double* gradP, double f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) U[i] += f * du[i] * gradP[i];
}

// ---------------------------------------------------------------------------
// launchers
// grids: 8 lanes per row, bs threads per block (a multiple of 32, at most the
// BLOCK the kernels are compiled for)
// ---------------------------------------------------------------------------
// Symmetry planes.
//
// Assembled symmetry area of each row node (mesh::updateAssembledSymmetryAreaField_,
// src/mesh/meshGeometry.cpp:1787-1880): the exposed-area vectors of the
// symmetry face ips nearest the node, summed over its incident elements (each
// lane its element's symmetry faces at its corner). Set-up only.
template <int LPR>
__global__ void __launch_bounds__(BLOCK) k_sym_area(MeshView m, double* area) {
  const RowLane<LPR> rl = row_lane<LPR>(m);
  double A[3] = {0.0, 0.0, 0.0};
  if (rl.e >= 0 && m.sym_mask) {
    const uint8_t sm = __ldg(m.sym_mask + rl.e);
    if (sm) {
      const uint32_t fw = face_word(rl.c);
      double x[8][3];
      int nd[8];
      gather_x(m, rl.e, perm_word(rl.c), x, nd);
      StaticFor<0, 3>::run([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        constexpr int FC = q == 0 ? 0 : (q == 1 ? 3 : 4);
        if (sm & (1u << ((fw >> (3 * q)) & 7))) {
          double Af[3];
          face_area_at_first<double>(x[face_node(FC, 0)], x[face_node(FC, 1)], x[face_node(FC, 2)],
                                     x[face_node(FC, 3)], Af);
#pragma unroll
          for (int k = 0; k < 3; ++k) A[k] += Af[k];
        }
      });
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) A[k] = rowsum<LPR>(A[k]);
  if (rl.rv && rl.li == 0)
#pragma unroll
    for (int k = 0; k < 3; ++k) area[3L * rl.row + k] = A[k];
}

__device__ __forceinline__ void sym_unit(const double* a, double (&n)[3]) {
  const double amag = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
#pragma unroll
  for (int k = 0; k < 3; ++k) n[k] = a[k] / amag;
}

// Symmetry rows after the momentum assembly, one thread per symmetry node:
// applySymmetryConditions_ (navierStokesAssembler.cpp:387-471) removes the rhs
// component along the assembled symmetry normal n; assembleNormalRelaxation
// (:473-699, urf 0.75 from navierStokesEquation.cpp:169, after the DU
// coefficients) adds (1 - urf) D n n^T to the diagonal block D.
template <class TF>
__global__ void __launch_bounds__(BLOCK) k_sym_rows(int nsym, const int* __restrict__ nodes,
                                                    const double* __restrict__ area, const int* __restrict__ row_ptr,
                                                    const int* __restrict__ diag, TF* A, TF* b) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nsym) return;
  const int i = nodes[k];
  double n[3];
  sym_unit(area + 3L * k, n);
  TF* bb = b + 3L * i;
  const double r[3] = {double(bb[0]), double(bb[1]), double(bb[2])};
  const double dot = r[0] * n[0] + r[1] * n[1] + r[2] * n[2];
#pragma unroll
  for (int q = 0; q < 3; ++q) bb[q] = TF(r[q] - dot * n[q]);
  TF* D = A + 9L * (row_ptr[i] + diag[i]);
  double d[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) d[q] = double(D[q]);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double m = 0.0;
#pragma unroll
      for (int q = 0; q < 3; ++q) m += d[3 * a + q] * (n[q] * n[c]);
      D[3 * a + c] = TF(d[3 * a + c] + (1.0 - 0.75) * m);
    }
}

// Gradient at a symmetry node without its normal part (the correctGradients_
// switch, end of nodeField::updateGradientField, nodeField.hpp:4939-4943): a
// scalar's G - (G.n) n (nodeScalarField.cpp:44-112), a vector's
// G - (G n) n^T - n (n^T G) + 2 (n^T G n) n n^T (nodeVectorField.cpp:44-148).
template <int NC>
__global__ void __launch_bounds__(BLOCK) k_sym_grad(int nsym, const int* __restrict__ nodes,
                                                    const double* __restrict__ area, double* grad) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nsym) return;
  double n[3];
  sym_unit(area + 3L * k, n);
  double* G = grad + 3L * NC * nodes[k];
  if (NC == 1) {
    const double dot = G[0] * n[0] + G[1] * n[1] + G[2] * n[2];
#pragma unroll
    for (int j = 0; j < 3; ++j) G[j] -= dot * n[j];
    return;
  }
  double g[9], Gn[3] = {0.0, 0.0, 0.0}, nG[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int q = 0; q < 9; ++q) g[q] = G[q];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      Gn[i] += g[3 * i + j] * n[j];
      nG[j] += g[3 * i + j] * n[i];
    }
  const double nGn = nG[0] * n[0] + nG[1] * n[1] + nG[2] * n[2];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double v = g[3 * i + j];
      v -= Gn[i] * n[j];
      v -= n[i] * nG[j];
      v += 2.0 * n[i] * n[j] * nGn;
      G[3 * i + j] = v;
    }
}

static int grid_rows(const DeviceMesh& m, int bs = BLOCK) { return (int)(((size_t)m.nn * m.lpr + bs - 1) / bs); }

static int launch_mdot_impl(Flow& f, int mode);

int launch_pcorr(Flow& f, bool mixed, bool flux_fresh) {
  // the staged coefficients are written in the flow's matrix precision
  if (mixed != (f.s.precision == OA_PREC_MIXED))
    return fail(OA_ERR_ARG, "pressure-correction assembly: precision differs from the flow's");
  if (!flux_fresh)
    if (int s = launch_mdot_impl(f, 2)) return s;
  PcArgs a{f.mesh->view(), f.pc_coef, f.pc_flux, f.b.A_pc, f.b.b_pc, f.ref_flag};
  const int bs = f.bs_asm;
  const int g = grid_rows(*f.mesh, bs);
  if (mixed)
    if (f.mesh->lpr == 16) k_pcorr<16, float><<<g, bs, 0, f.stream>>>(a);
    else k_pcorr<8, float><<<g, bs, 0, f.stream>>>(a);
  else
    if (f.mesh->lpr == 16) k_pcorr<16, double><<<g, bs, 0, f.stream>>>(a);
    else k_pcorr<8, double><<<g, bs, 0, f.stream>>>(a);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

// FP32 corner offsets of every element from its corner 0 (mixed form, once
// per flow: the offsets are formed in FP64 and rounded once)
__global__ void k_xloc(MeshView m, float4* xloc) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 8LL * m.ne) return;
  const int e = (int)(t >> 3);
  const int n0 = m.conn[8 * e], nk = m.conn[t];
  xloc[t] = make_float4(float(m.x[3 * nk] - m.x[3 * n0]), float(m.x[3 * nk + 1] - m.x[3 * n0 + 1]),
                        float(m.x[3 * nk + 2] - m.x[3 * n0 + 2]), 0.f);
}

// FP32 node copy of (U, mu) for the mixed momentum kernel
__global__ void k_pack_umu(int nn, const double* __restrict__ U, const double* __restrict__ mu, float4* umu) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nn) umu[i] = make_float4(float(U[3 * i]), float(U[3 * i + 1]), float(U[3 * i + 2]), float(mu[i]));
}

int launch_xloc(Flow& f) {
  const long long n = 8LL * f.mesh->ne;
  k_xloc<<<(unsigned)((n + 255) / 256), 256, 0, f.stream>>>(f.mesh->view(), f.xloc32);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

int launch_momentum(Flow& f, bool mixed) {
  if (mixed) {
    if (!f.xloc32 || !f.umu32) return fail(OA_ERR_ARG, "momentum assembly: mixed-form buffers missing");
    k_pack_umu<<<(f.mesh->nn + 255) / 256, 256, 0, f.stream>>>(f.mesh->nn, f.U, f.mu, f.umu32);
    count_launches(1);
  }
  MomArgs a{f.view(),       f.U,       f.gradP, f.div,  f.mDot,          f.rho,
            f.mu,           f.sideU,   f.betaU, f.gradU, f.xloc32, f.umu32, f.b.A_mom, f.b.b_mom,
            f.du,           f.duT,     f.time_order ? f.dt_step : f.s.dt,  1.0 / f.s.urf_u, f.s.wall_rhs_relax,
            f.s.du_mode,    f.s.hr,    f.time_order, f.tk[0], f.tk[1], f.tk[2], f.Uold, f.Uoldold, f.err_dev};
  const int bs = f.bs_asm;
  const int g = grid_rows(*f.mesh, bs);
  const bool us = f.s.u_shifted, gs = f.s.u_grad_shifted;
  const bool hr = f.s.hr != 0 || f.time_order != 0 || f.s.du_mode != 0;  // the optional-terms variant
  if (f.turb) {
    if (hr) return fail(OA_ERR_ARG, "momentum assembly: the fused turbulence variant is steady upwind SIMPLE only");
    a.kf = f.kf;
    a.wf = f.wf;
    a.gkf = f.gkf;
    a.gwf = f.gwf;
    a.sdk = f.sdk;
    a.srk = f.srk;
    a.sdw = f.sdw;
    a.srw = f.srw;
    a.Ak = f.A_k;
    a.bk = f.b_k;
    a.Aw = f.A_w;
    a.bw = f.b_w;
    a.urf_k_inv = 1.0 / f.urf_k;
    a.urf_w_inv = 1.0 / f.urf_w;
  }
  const int var = f.turb ? 2 : (hr ? 1 : 0);
  auto go = [&](auto lanes) {
    constexpr int L = decltype(lanes)::value;
#define OA_MOM(US, GS, T)                                                                   \
  if (us == US && gs == GS) {                                                               \
    if (var == 1)                                                                           \
      k_momentum<L, US, GS, T, 1><<<g, bs, 0, f.stream>>>(a);                               \
    else if (var == 2)                                                                      \
      k_momentum<L, US, GS, T, 2><<<g, bs, 0, f.stream>>>(a);                               \
    else                                                                                    \
      k_momentum<L, US, GS, T, 0><<<g, bs, 0, f.stream>>>(a);                               \
  }
    if (mixed) {
      OA_MOM(true, true, float) OA_MOM(true, false, float) OA_MOM(false, true, float) OA_MOM(false, false, float)
    } else {
      OA_MOM(true, true, double) OA_MOM(true, false, double) OA_MOM(false, true, double) OA_MOM(false, false, double)
    }
#undef OA_MOM
  };
  if (f.mesh->lpr == 16) go(std::integral_constant<int, 16>{});
  else go(std::integral_constant<int, 8>{});
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  if (f.nsym) {
    const unsigned gs = (unsigned)((f.nsym + BLOCK - 1) / BLOCK);
    const DeviceMesh& m = *f.mesh;
    if (mixed)
      k_sym_rows<float><<<gs, BLOCK, 0, f.stream>>>(f.nsym, f.sym_nodes, f.sym_area, m.row_ptr, m.diag,
                                                     static_cast<float*>(f.b.A_mom), static_cast<float*>(f.b.b_mom));
    else
      k_sym_rows<double><<<gs, BLOCK, 0, f.stream>>>(f.nsym, f.sym_nodes, f.sym_area, m.row_ptr, m.diag,
                                                      static_cast<double*>(f.b.A_mom), static_cast<double*>(f.b.b_mom));
    count_launches(1);
    OA_CUDA(cudaGetLastError());
  }
  return OA_OK;
}

// mode 0: update the mass flow; 1: initial mass flow; 2: pressure-correction
// staging only (ip fluxes and corner coefficients from the current mass flow,
// which stays unchanged); 3: update and staging
static int launch_mdot_impl(Flow& f, int mode) {
  MdotArgs a{f.mesh->view(), f.U,          f.p,          f.gradP,   f.du,     f.rho,
             f.s.du_mode == 1 ? f.duT : f.du, f.mDot, f.pc_flux,
             f.pc_coef,      f.s.mdot_urf, mode == 1 ? 1 : 0, mode == 2 ? 1 : 0, f.err_dev};
  const int bs = f.bs_elems;
  const int g = (f.mesh->ne + bs - 1) / bs;
  const bool us = f.s.u_shifted, ps = f.s.p_grad_shifted;
#define OA_MD(T, ST, SC)                                                                \
  if (us && ps) k_mdot<true, true, T, ST, SC><<<g, bs, 0, f.stream>>>(a);            \
  else if (us && !ps) k_mdot<true, false, T, ST, SC><<<g, bs, 0, f.stream>>>(a);     \
  else if (!us && ps) k_mdot<false, true, T, ST, SC><<<g, bs, 0, f.stream>>>(a);     \
  else k_mdot<false, false, T, ST, SC><<<g, bs, 0, f.stream>>>(a);
  const bool sc = f.s.du_mode == 1;
  if (mode == 0 || mode == 1) {
    OA_MD(double, false, false)
  } else if (f.s.precision == OA_PREC_MIXED) {
    if (sc) {
      OA_MD(float, true, true)
    } else {
      OA_MD(float, true, false)
    }
  } else {
    if (sc) {
      OA_MD(double, true, true)
    } else {
      OA_MD(double, true, false)
    }
  }
#undef OA_MD
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}
int launch_init_mdot(Flow& f) { return launch_mdot_impl(f, 1); }
int launch_update_mdot(Flow& f, bool stage) { return launch_mdot_impl(f, stage ? 3 : 0); }

int launch_div(Flow& f) {
  DivArgs a{f.mesh->view(), f.mDot, f.div, f.rho, f.time_order, f.tk[0], f.tk[1], f.tk[2], f.dt_step};
  if (f.mesh->lpr == 16) k_div<16><<<grid_rows(*f.mesh, f.bs_rows), f.bs_rows, 0, f.stream>>>(a);
  else k_div<8><<<grid_rows(*f.mesh, f.bs_rows), f.bs_rows, 0, f.stream>>>(a);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

int launch_sym_area(Flow& f, double* area_nn) {
  // the mesh view with the flow's symmetry mask, which f.view() exposes only
  // once the symmetry nodes are set up
  if (!f.sym_mask) return fail(OA_ERR_ARG, "symmetry area: no symmetry face mask");
  MeshView v = f.mesh->view();
  v.sym_mask = f.sym_mask;
  const unsigned g = (unsigned)(((size_t)f.mesh->nn * f.mesh->lpr + BLOCK - 1) / BLOCK);
  if (f.mesh->lpr == 16) k_sym_area<16><<<g, BLOCK, 0, f.stream>>>(v, area_nn);
  else k_sym_area<8><<<g, BLOCK, 0, f.stream>>>(v, area_nn);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

static int launch_sym_grad(Flow& f, int which) {
  if (!f.nsym || !f.correct_grad) return OA_OK;
  const unsigned g = (unsigned)((f.nsym + BLOCK - 1) / BLOCK);
  if (which == 1) k_sym_grad<3><<<g, BLOCK, 0, f.stream>>>(f.nsym, f.sym_nodes, f.sym_area, f.gradU);
  else
    k_sym_grad<1><<<g, BLOCK, 0, f.stream>>>(f.nsym, f.sym_nodes, f.sym_area,
                                             which == 0 ? f.gradP : (which == 2 ? f.gradK : f.gradW));
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

int launch_gradient(Flow& f, int which) {
  const int bs = f.bs_rows;
  const int g = grid_rows(*f.mesh, bs);
  if (which >= 2) {
    // k (2) and omega (3): the turbulence fields' default interpolation is
    // linear_linear (controls.h:97-102), the shifted gradient operator
    if (!f.turb) return fail(OA_ERR_NOT_READY, "gradient of k / omega: turbulence transport not enabled");
    GradArgs a{f.view(), which == 2 ? f.kf : f.wf, which == 2 ? f.gradK : f.gradW, f.s.grad_urf};
    if (f.mesh->lpr == 16) k_gradient<16, 1, true><<<g, bs, 0, f.stream>>>(a);
    else k_gradient<8, 1, true><<<g, bs, 0, f.stream>>>(a);
  } else if (which == 0) {
    GradArgs a{f.view(), f.p, f.gradP, f.s.grad_urf};
    if (f.mesh->lpr == 16) {
      if (f.s.p_shifted) k_gradient<16, 1, true><<<g, bs, 0, f.stream>>>(a);
      else k_gradient<16, 1, false><<<g, bs, 0, f.stream>>>(a);
    } else {
      if (f.s.p_shifted) k_gradient<8, 1, true><<<g, bs, 0, f.stream>>>(a);
      else k_gradient<8, 1, false><<<g, bs, 0, f.stream>>>(a);
    }
  } else {
    GradArgs a{f.view(), f.U, f.gradU, f.s.grad_urf};
    if (f.mesh->lpr == 16) {
      if (f.s.u_shifted) k_gradient<16, 3, true><<<g, bs, 0, f.stream>>>(a);
      else k_gradient<16, 3, false><<<g, bs, 0, f.stream>>>(a);
    } else {
      if (f.s.u_shifted) k_gradient<8, 3, true><<<g, bs, 0, f.stream>>>(a);
      else k_gradient<8, 3, false><<<g, bs, 0, f.stream>>>(a);
    }
  }
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return launch_sym_grad(f, which);
}

int launch_blend_u(Flow& f) {
  BlendArgs a{f.mesh->view(), f.U, f.gradU, f.minU, f.maxU, f.betaU, f.s.beta_max};
  const int g = grid_rows(*f.mesh, f.bs_rows);
  if (f.mesh->lpr == 16) {
    k_minmax_u<16><<<g, f.bs_rows, 0, f.stream>>>(a);
    k_blend_u<16><<<g, f.bs_rows, 0, f.stream>>>(a);
  } else {
    k_minmax_u<8><<<g, f.bs_rows, 0, f.stream>>>(a);
    k_blend_u<8><<<g, f.bs_rows, 0, f.stream>>>(a);
  }
  count_launches(2);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

int launch_axpy_du_gradp(Flow& f, double sign) {
  const int n3 = 3 * f.mesh->nn;
  // D, or D~ with SIMPLEC (segregatedFlowEquations.cpp:134-278)
  k_vel_correct<<<(n3 + 255) / 256, 256, 0, f.stream>>>(n3, f.U, f.s.du_mode == 1 ? f.duT : f.du, f.gradP,
                                                         sign / f.s.urf_p);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

}  // namespace oa
