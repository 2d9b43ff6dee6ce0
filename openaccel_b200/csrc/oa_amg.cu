// Aggregation AMG V-cycle for the pressure-correction system (see oa_amg.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "oa_amg.h"
#include "oa_amg_symbolic.h"
#include "oa_internal.h"

namespace oa {

constexpr int AB = 256;          // threads per block
constexpr int COARSE_MAX = 256;  // coarsest level solved by a dense inverse
constexpr int MAX_CHEB = 6;      // highest Chebyshev smoothing degree

// Lanes per row of the row-parallel kernels (1, 4, 8 or 32): levels with many
// rows keep one lane per row for short rows and take 8 for long ones (the
// first coarse level of the 128^3 cavity: 31 entries per row, 8 lanes measured
// fastest against 1, 4 and 32); small levels spread each row over a group of
// lanes so that the few rows still fill the SMs. OA_AMG_LANES_BIG overrides
// the choice for long rows on large levels.
static int lanes_for(double avg, long long rows) {
  if (rows >= 100000) {
    if (avg <= 16.0) return 1;
    static const int big = [] {
      const char* e = std::getenv("OA_AMG_LANES_BIG");
      const int v = e ? std::atoi(e) : 0;
      return (v == 1 || v == 4 || v == 8 || v == 32) ? v : 0;
    }();
    if (big) return big;
    return 8;
  }
  return avg <= 4.0 ? 1 : (avg <= 24.0 ? 8 : 32);
}

static unsigned grid_for(long long rows, int lpr) { return (unsigned)((rows * lpr + AB - 1) / AB); }


template <class T>
static int upload(T** d, const std::vector<T>& h) {
  if (cudaMalloc(d, sizeof(T) * std::max<size_t>(1, h.size())) != cudaSuccess)
    return fail(OA_ERR_CUDA, "AMG: device allocation failed");
  if (!h.empty() && cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(OA_ERR_CUDA, "AMG: upload failed");
  return OA_OK;
}

template <class T>
static int dalloc(T** d, size_t n) {
  if (cudaMalloc(d, sizeof(T) * std::max<size_t>(1, n)) != cudaSuccess)
    return fail(OA_ERR_CUDA, "AMG: device allocation failed");
  return OA_OK;
}

template <class T>
int Amg<T>::setup(int n, const int* h_rp, const int* h_cols, const int* h_diag, int* d_rp, int* d_cols, int* d_diag) {
  release();
  // tuning knobs: prolongation type, Jacobi damping, coarse-correction scaling
  if (const char* e = std::getenv("OA_AMG_SMOOTHED")) smoothed = std::atoi(e) != 0;
  omega = smoothed ? 0.8 : 0.7;
  alpha = smoothed ? 1.0 : 1.8;
  if (const char* e = std::getenv("OA_AMG_OMEGA")) omega = std::atof(e);
  if (const char* e = std::getenv("OA_AMG_ALPHA")) alpha = std::atof(e);
  if (const char* e = std::getenv("OA_AMG_OMEGA_P")) omega_p = std::atof(e);
  if (const char* e = std::getenv("OA_AMG_CHEB_DEGREE")) cheb_degree = std::atoi(e);
  if (const char* e = std::getenv("OA_AMG_CHEB_ROWS")) cheb_rows = std::atoi(e);
  if (const char* e = std::getenv("OA_AMG_CHEB_RATIO")) cheb_ratio = std::max(1.5, std::atof(e));
  if (cheb_degree < 2 || !smoothed) cheb_degree = 0;
  if (cheb_degree > MAX_CHEB) return fail(OA_ERR_ARG, "AMG: Chebyshev degree above the supported maximum");
  cheb_launches = 0;
  std::vector<int> rp(h_rp, h_rp + n + 1), cols(h_cols, h_cols + h_rp[n]), dg(h_diag, h_diag + n);
  int cur = n;
  for (int lev = 0;; ++lev) {
    // the level joins L before anything is allocated for it, so an error
    // return leaves every allocation where release() finds it
    L.emplace_back();
    AmgLevel<T>& lv = L.back();
    lv.n = cur;
    lv.nnz = rp[cur];
    if (lev == 0) {
      lv.rp = d_rp;
      lv.cols = d_cols;
      lv.diag = d_diag;
    } else {
      int s;
      if ((s = upload(&lv.rp, rp)) || (s = upload(&lv.cols, cols)) || (s = upload(&lv.diag, dg))) return s;
      if ((s = dalloc(&lv.A, (size_t)lv.nnz))) return s;
      lv.own_A = true;
    }
    int s;
    if ((s = dalloc(&lv.dinv, cur)) || (s = dalloc(&lv.r, cur)) || (s = dalloc(&lv.t, cur))) return s;
    if (lev > 0 && ((s = dalloc(&lv.x, cur)) || (s = dalloc(&lv.b, cur)))) return s;
    lv.lpr_a = lanes_for(double(lv.nnz) / std::max(1, cur), cur);
    const bool last = cur <= COARSE_MAX || lev >= 14;
    if (last) break;
    // not on the finest level: its matrix is always the caller's current one,
    // while the spectral estimate (like Dinv) is refreshed only with the
    // hierarchy; a coarse level's matrix, Dinv and estimate come from the same
    // numeric phase
    if (cheb_degree >= 2 && lev > 0 && cur <= cheb_rows) {
      lv.cheb = true;
      if ((s = dalloc(&lv.cr, cur)) || (s = dalloc(&lv.cd0, cur)) || (s = dalloc(&lv.cd1, cur)) ||
          (s = dalloc(&lv.lmax, 2)) || (s = dalloc(&lv.pw_a, (size_t)lv.nnz)) || (s = dalloc(&lv.pw_dinv, cur)) ||
          (s = dalloc(&lv.pw_v, cur)) || (s = dalloc(&lv.pw_w, cur)) ||
          (s = dalloc(&lv.pw_part, grid_for(cur, lv.lpr_a))))
        return s;
      cheb_launches += 2LL * (cheb_degree - 1);
    }
    int nc = 0;
    std::vector<int> crp, ccols, cdg;
    if (smoothed) {
      sa::Level H;
      if (!sa::build(cur, rp, cols, H))
        return fail(OA_ERR_SOLVER, "AMG: smoothed-aggregation term lists exceed 32-bit offsets");
      nc = H.nc;
      if (nc >= cur) return fail(OA_ERR_SOLVER, "AMG: aggregation made no progress");
      lv.nnz_t = H.trp[cur];
      lv.nnz_p = H.prp[cur];
      lv.lpr_p = lanes_for(double(lv.nnz_p) / cur, cur);
      lv.lpr_pt = lanes_for(double(lv.nnz_p) / H.nc, H.nc);
      lv.lpr_t = lanes_for(double(H.tta.size()) / std::max(1, lv.nnz_t), lv.nnz_t);
      lv.lpr_c = lanes_for(double(H.ctp.size()) / std::max(1, H.crp[H.nc]), H.crp[H.nc]);
      if ((s = upload(&lv.p_rp, H.prp)) || (s = upload(&lv.p_cols, H.pcols)) || (s = upload(&lv.p_diag, H.pdiag)) ||
          (s = upload(&lv.pg_ptr, H.pgptr)) || (s = upload(&lv.pg_list, H.pglist)) ||
          (s = upload(&lv.pt_rp, H.ptrp)) || (s = upload(&lv.pt_rows, H.ptrows)) || (s = upload(&lv.pt_src, H.ptsrc)) ||
          (s = upload(&lv.tt_ptr, H.ttptr)) || (s = upload(&lv.tt_a, H.tta)) || (s = upload(&lv.tt_p, H.ttp)) ||
          (s = upload(&lv.ct_ptr, H.ctptr)) || (s = upload(&lv.ct_p, H.ctp)) || (s = upload(&lv.ct_t, H.ctt)) ||
          (s = dalloc(&lv.pv, H.pcols.size())) || (s = dalloc(&lv.ptv, H.pcols.size())) ||
          (s = dalloc(&lv.tv, (size_t)lv.nnz_t)))
        return s;
      crp.swap(H.crp);
      ccols.swap(H.ccols);
      cdg.swap(H.cdg);
    } else {
      std::vector<int> agg;
      nc = sa::aggregate(cur, rp, cols, agg);
      if (nc >= cur) return fail(OA_ERR_SOLVER, "AMG: aggregation made no progress");
      // members of each aggregate, in row order
      std::vector<int> mptr(nc + 1, 0), mlist(cur);
      for (int i = 0; i < cur; ++i) mptr[agg[i] + 1]++;
      for (int c = 0; c < nc; ++c) mptr[c + 1] += mptr[c];
      {
        std::vector<int> pos(mptr.begin(), mptr.end() - 1);
        for (int i = 0; i < cur; ++i) mlist[pos[agg[i]]++] = i;
      }
      // coarse graph (sorted columns) and the gather list of each coarse entry
      crp.assign(nc + 1, 0);
      cdg.assign(nc, 0);
      std::vector<int> tmp;
      for (int c = 0; c < nc; ++c) {
        tmp.clear();
        for (int m = mptr[c]; m < mptr[c + 1]; ++m) {
          const int i = mlist[m];
          for (int k = rp[i]; k < rp[i + 1]; ++k) tmp.push_back(agg[cols[k]]);
        }
        std::sort(tmp.begin(), tmp.end());
        tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
        for (size_t q = 0; q < tmp.size(); ++q)
          if (tmp[q] == c) cdg[c] = (int)q;
        ccols.insert(ccols.end(), tmp.begin(), tmp.end());
        crp[c + 1] = (int)ccols.size();
      }
      const int cnnz = crp[nc];
      std::vector<int> gcnt(cnnz + 1, 0), target(rp[cur]);
      for (int c = 0; c < nc; ++c)
        for (int m = mptr[c]; m < mptr[c + 1]; ++m) {
          const int i = mlist[m];
          for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int cj = agg[cols[k]];
            const int pos =
                (int)(std::lower_bound(ccols.begin() + crp[c], ccols.begin() + crp[c + 1], cj) - ccols.begin());
            target[k] = pos;
            gcnt[pos + 1]++;
          }
        }
      for (int q = 0; q < cnnz; ++q) gcnt[q + 1] += gcnt[q];
      std::vector<int> glist(rp[cur]);
      {
        std::vector<int> pos(gcnt.begin(), gcnt.end() - 1);
        for (int c = 0; c < nc; ++c)
          for (int m = mptr[c]; m < mptr[c + 1]; ++m) {
            const int i = mlist[m];
            for (int k = rp[i]; k < rp[i + 1]; ++k) glist[pos[target[k]]++] = k;
          }
      }
      if ((s = upload(&lv.agg, agg)) || (s = upload(&lv.mptr, mptr)) || (s = upload(&lv.mlist, mlist)) ||
          (s = upload(&lv.gptr, gcnt)) || (s = upload(&lv.glist, glist)))
        return s;
    }
    rp.swap(crp);
    cols.swap(ccols);
    dg.swap(cdg);
    cur = nc;
  }
  coarse_n = L.back().n;
  if (cudaMalloc(&dense_inv, sizeof(double) * 2 * (size_t)coarse_n * coarse_n) != cudaSuccess)
    return fail(OA_ERR_CUDA, "AMG: dense coarse allocation failed");
  ready = true;
  return OA_OK;
}

template <class T>
void Amg<T>::release() {
  for (size_t l = 0; l < L.size(); ++l) {
    AmgLevel<T>& v = L[l];
    if (l > 0) {
      cudaFree(v.rp);
      cudaFree(v.cols);
      cudaFree(v.diag);
    }
    if (v.own_A) cudaFree(v.A);
    void* p[] = {v.dinv,   v.agg,   v.mptr,   v.mlist, v.gptr,   v.glist, v.r,      v.t,    v.p_rp,
                 v.p_cols, v.p_diag, v.pg_ptr, v.pg_list, v.pv, v.ptv, v.pt_rp, v.pt_rows, v.pt_src, v.tv,
                 v.tt_ptr, v.tt_a,   v.tt_p,   v.ct_ptr, v.ct_p, v.ct_t, v.cr,      v.cd0,  v.cd1,
                 v.lmax,   v.pw_a,  v.pw_dinv, v.pw_v, v.pw_w,   v.pw_part};
    for (void* q : p)
      if (q) cudaFree(q);
    if (l > 0) {
      cudaFree(v.x);
      cudaFree(v.b);
    }
  }
  L.clear();
  if (dense_inv) cudaFree(dense_inv);
  dense_inv = nullptr;
  ready = false;
}

// ---------------------------------------------------------------------------
// kernels
template <class T>
__global__ void k_galerkin(int nnz_c, const int* __restrict__ gptr, const int* __restrict__ glist,
                           const T* __restrict__ Af, T* __restrict__ Ac) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nnz_c) return;
  double s = 0.0;
  for (int q = gptr[c]; q < gptr[c + 1]; ++q) s += double(Af[glist[q]]);
  Ac[c] = T(s);
}

template <class T>
__global__ void k_widen(int n, const T* __restrict__ a, double* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = double(a[i]);
}

template <class T>
__global__ void k_dinv(int n, const int* __restrict__ rp, const int* __restrict__ dg, const T* __restrict__ A,
                       T* __restrict__ dinv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dinv[i] = T(1.0 / double(A[rp[i] + dg[i]]));
}

// dense copy of the coarsest matrix, augmented with the identity: [A | I]
template <class T>
__global__ void k_dense_fill(int n, const int* __restrict__ rp, const int* __restrict__ cols, const T* __restrict__ A,
                             double* M) {
  const int i = blockIdx.x;
  for (int j = threadIdx.x; j < 2 * n; j += blockDim.x) M[(size_t)i * 2 * n + j] = (j - n == i) ? 1.0 : 0.0;
  __syncthreads();
  for (int k = rp[i] + threadIdx.x; k < rp[i + 1]; k += blockDim.x) M[(size_t)i * 2 * n + cols[k]] = double(A[k]);
}

// Gauss-Jordan elimination without pivoting (the coarse Galerkin operators of
// the grounded Rhie-Chow Laplacian are M-matrices), one block; leaves A^-1 in
// the right half. At step k the pivot row is zero left of column k (earlier
// steps cleared it) and right of column n + k (the identity's later columns
// are still untouched there), so only its n + 1 columns k .. n + k are
// normalised and used: the skipped updates would subtract exact zeros.
__global__ void k_gauss_jordan(int n, double* M) {
  const int w = 2 * n;
  for (int k = 0; k < n; ++k) {
    __syncthreads();
    const double piv = M[(size_t)k * w + k];
    __syncthreads();
    for (int j = k + threadIdx.x; j <= n + k; j += blockDim.x) M[(size_t)k * w + j] /= piv;
    __syncthreads();
    // columns k + 1 .. n + k of every other row (n of them)
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
      const int i = idx / n, j = k + 1 + (idx - i * n);
      if (i == k) continue;
      M[(size_t)i * w + j] -= M[(size_t)i * w + k] * M[(size_t)k * w + j];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      if (i != k) M[(size_t)i * w + k] = 0.0;
  }
}

// Sum of one value per lane over a group of LPR consecutive lanes (a row's
// lanes), by a fixed xor butterfly: the same order every run.
template <int LPR>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = LPR / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Downward step, LPR lanes per row: pre-smooth from zero, xs_i = w Dinv_i b_i,
// and the residual r_i = b_i - sum_j a_ij xs_j (neighbours' xs formed from b).
template <class T, int LPR>
__global__ void __launch_bounds__(AB) k_smooth_resid(int n, const int* __restrict__ rp, const int* __restrict__ cols,
                                                     const T* __restrict__ A, const T* __restrict__ dinv,
                                                     const T* __restrict__ b, T* __restrict__ xs, T* __restrict__ r,
                                                     double w, const int* done) {
  if (*done) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = g / LPR, lane = g % LPR;
  double s = 0.0;
  if (i < n)
    for (int k = rp[i] + lane; k < rp[i + 1]; k += LPR) {
      const int j = cols[k];
      s += double(A[k]) * (w * double(dinv[j]) * double(b[j]));
    }
  s = group_sum<LPR>(s);
  if (i >= n || lane) return;
  const double bi = double(b[i]);
  xs[i] = T(w * double(dinv[i]) * bi);
  r[i] = T(bi - s);
}

// restriction by the piecewise-constant prolongation: bc_c = sum of the
// members' residuals, in member order
template <class T>
__global__ void k_restrict(int nc, const int* __restrict__ mptr, const int* __restrict__ mlist, const T* __restrict__ r,
                           T* __restrict__ bc, const int* done) {
  if (*done) return;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double s = 0.0;
  for (int m = mptr[c]; m < mptr[c + 1]; ++m) s += double(r[mlist[m]]);
  bc[c] = T(s);
}

// Fused upward step: prolong (t = xs + alpha P xc, formed on the fly for each
// neighbour) and post-smooth, x_i = t_i + w Dinv_i (b_i - sum_j a_ij t_j).
// Reads xs, writes x: out of place, no race between rows.
template <class T>
__global__ void __launch_bounds__(AB) k_up(int n, const int* __restrict__ rp, const int* __restrict__ cols,
                                           const T* __restrict__ A, const T* __restrict__ dinv,
                                           const int* __restrict__ agg, const T* __restrict__ b,
                                           const T* __restrict__ xs, const T* __restrict__ xc, T* __restrict__ x,
                                           double w, double alpha, const int* done) {
  if (*done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const int j = cols[k];
    s += double(A[k]) * (double(xs[j]) + alpha * double(xc[agg[j]]));
  }
  const double ti = double(xs[i]) + alpha * double(xc[agg[i]]);
  x[i] = T(ti + w * double(dinv[i]) * (double(b[i]) - s));
}

template <class T>
__global__ void __launch_bounds__(AB) k_dense_apply(int n, const double* __restrict__ M, const T* __restrict__ b,
                                                    T* __restrict__ x, const int* done) {
  if (*done) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = g / 32, lane = g % 32;  // one warp per row of the coarsest inverse
  double s = 0.0;
  if (i < n) {
    const double* row = M + (size_t)i * 2 * n + n;
    for (int j = lane; j < n; j += 32) s += row[j] * double(b[j]);
  }
  s = group_sum<32>(s);
  if (i < n && lane == 0) x[i] = T(s);
}

// Smoothed prolongation: P_iJ = [J == agg(i)] - wp Dinv_i sum of the row's A
// entries whose column lies in aggregate J; LPR lanes share a row's entries.
template <class T, int LPR>
__global__ void __launch_bounds__(AB) k_sa_prolongator(int n, const int* __restrict__ p_rp,
                                                       const int* __restrict__ p_diag, const int* __restrict__ pg_ptr,
                                                       const int* __restrict__ pg_list, const T* __restrict__ A,
                                                       const T* __restrict__ dinv, double wp, T* __restrict__ pv) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = g / LPR, lane = g % LPR;
  if (i >= n) return;
  const double di = double(dinv[i]);
  const int e0 = p_rp[i];
  for (int e = e0 + lane; e < p_rp[i + 1]; e += LPR) {
    double s = 0.0;
    for (int q = pg_ptr[e]; q < pg_ptr[e + 1]; ++q) s += double(A[pg_list[q]]);
    pv[e] = T((e - e0 == p_diag[i] ? 1.0 : 0.0) - wp * di * s);
  }
}

// out_e = sum over the entry's term list of a[ia] * b[ib], LPR lanes per entry.
template <class T, int LPR>
__global__ void __launch_bounds__(AB) k_pair_sum(int n_out, const int* __restrict__ ptr, const int* __restrict__ ia,
                                                 const int* __restrict__ ib, const T* __restrict__ a,
                                                 const T* __restrict__ b, T* __restrict__ out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int e = g / LPR, lane = g % LPR;
  double s = 0.0;
  if (e < n_out)
    for (int q = ptr[e] + lane; q < ptr[e + 1]; q += LPR) s += double(a[ia[q]]) * double(b[ib[q]]);
  s = group_sum<LPR>(s);
  if (e < n_out && lane == 0) out[e] = T(s);
}

// P^T values in coarse-row order (contiguous for the restriction)
template <class T>
__global__ void k_gather(int n, const int* __restrict__ idx, const T* __restrict__ src, T* __restrict__ dst) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) dst[q] = src[idx[q]];
}

// restriction bc = P^T r, LPR lanes per coarse row
template <class T, int LPR>
__global__ void __launch_bounds__(AB) k_sa_restrict(int nc, const int* __restrict__ pt_rp,
                                                    const int* __restrict__ pt_rows, const T* __restrict__ ptv,
                                                    const T* __restrict__ r, T* __restrict__ bc, const int* done) {
  if (*done) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = g / LPR, lane = g % LPR;
  double s = 0.0;
  if (c < nc)
    for (int q = pt_rp[c] + lane; q < pt_rp[c + 1]; q += LPR) s += double(ptv[q]) * double(r[pt_rows[q]]);
  s = group_sum<LPR>(s);
  if (c < nc && lane == 0) bc[c] = T(s);
}

// coarse correction in place: t_i += alpha (P xc)_i, LPR lanes per row
template <class T, int LPR>
__global__ void __launch_bounds__(AB) k_sa_prolong_add(int n, const int* __restrict__ p_rp,
                                                       const int* __restrict__ p_cols, const T* __restrict__ pv,
                                                       const T* __restrict__ xc, T* __restrict__ t, double alpha,
                                                       const int* done) {
  if (*done) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = g / LPR, lane = g % LPR;
  double s = 0.0;
  if (i < n)
    for (int e = p_rp[i] + lane; e < p_rp[i + 1]; e += LPR) s += double(pv[e]) * double(xc[p_cols[e]]);
  s = group_sum<LPR>(s);
  if (i < n && lane == 0) t[i] = T(double(t[i]) + alpha * s);
}

// post-smooth out of place, LPR lanes per row:
// x_i = t_i + w Dinv_i (b_i - sum_j a_ij t_j)
template <class T, int LPR>
__global__ void __launch_bounds__(AB) k_post_smooth(int n, const int* __restrict__ rp, const int* __restrict__ cols,
                                                    const T* __restrict__ A, const T* __restrict__ dinv,
                                                    const T* __restrict__ b, const T* __restrict__ t,
                                                    T* __restrict__ x, double w, const int* done) {
  if (*done) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = g / LPR, lane = g % LPR;
  double s = 0.0;
  if (i < n)
    for (int k = rp[i] + lane; k < rp[i + 1]; k += LPR) s += double(A[k]) * double(t[cols[k]]);
  s = group_sum<LPR>(s);
  if (i < n && lane == 0) x[i] = T(double(t[i]) + w * double(dinv[i]) * (double(b[i]) - s));
}

// Chebyshev smoothing (Saad, Iterative Methods for Sparse Linear Systems,
// 2nd ed., Algorithm 12.1, applied to Dinv A) over [lambda / ratio, lambda]:
// with theta and delta the interval's centre and half width, sigma = theta /
// delta and rho_0 = 1 / sigma, step k >= 1 takes rho_k = 1 / (2 sigma -
// rho_{k-1}), r_k = r_{k-1} - Dinv A d_{k-1}, d_k = rho_k rho_{k-1} d_{k-1} +
// (2 rho_k / delta) r_k and x += d_k, from r_0 = Dinv (b - A x), d_0 = r_0 /
// theta. The step coefficients are formed from lambda by every thread.
struct ChebStep {
  double inv_theta, c1, c2;
};

__device__ __forceinline__ ChebStep cheb_step(double lmax, double ratio, int k) {
  const double lmin = lmax / ratio, theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
  const double sigma = theta / delta;
  double rho = 1.0 / sigma, c1 = 0.0, c2 = 0.0;
  for (int j = 1; j <= k; ++j) {
    const double rho1 = 1.0 / (2.0 * sigma - rho);
    c1 = rho1 * rho;
    c2 = 2.0 * rho1 / delta;
    rho = rho1;
  }
  return {1.0 / theta, c1, c2};
}

// Spectral radius of Dinv A by power iteration from a fixed pseudo-random
// vector: POWER_STEPS products w = Dinv A (v / |v|), each followed by an
// ordered reduction of |w|^2; the last |w|, times a safety factor of 1.1,
// bounds the smoothing interval. State in est[]: est[0] = 1 / |v| of the
// vector being multiplied, est[1] = the bound.
constexpr int POWER_STEPS = 15;

__global__ void k_power_init(int n, double* v, double* est) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    unsigned h = (unsigned)i * 2654435761u;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    v[i] = double(h) * (2.0 / 4294967296.0) - 1.0;
  }
  if (i == 0) est[0] = 1.0;
}

template <int LPR>
__global__ void __launch_bounds__(AB) k_power_apply(int n, const int* __restrict__ rp, const int* __restrict__ cols,
                                                    const double* __restrict__ Ad, const double* __restrict__ dinv,
                                                    const double* __restrict__ v, const double* __restrict__ est,
                                                    double* __restrict__ w, double* __restrict__ partials) {
  __shared__ double sh[AB];
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = g / LPR, lane = g % LPR;
  double s = 0.0;
  if (i < n)
    for (int k = rp[i] + lane; k < rp[i + 1]; k += LPR) s += Ad[k] * v[cols[k]];
  s = group_sum<LPR>(s);
  double q = 0.0;
  if (i < n && lane == 0) {
    const double wi = dinv[i] * s * est[0];
    w[i] = wi;
    q = wi * wi;
  }
  sh[threadIdx.x] = q;
  __syncthreads();
  for (int o = AB / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

__global__ void k_power_norm(int nb, const double* __restrict__ partials, double* est) {
  __shared__ double sh[AB];
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += AB) s += partials[b];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = AB / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double nrm = sqrt(sh[0]);
    est[0] = nrm > 0.0 ? 1.0 / nrm : 1.0;
    est[1] = 1.1 * nrm;
  }
}

// Pre-smoothing from a zero iterate, steps 0 and 1 together: d_0 = Dinv b /
// theta (formed for the neighbours from b), r_1 = Dinv b - Dinv A d_0, d_1 and
// x = d_0 + d_1.
template <class T, int LPR>
__global__ void __launch_bounds__(AB) k_cheb_first(int n, const int* __restrict__ rp, const int* __restrict__ cols,
                                                   const T* __restrict__ A, const T* __restrict__ dinv,
                                                   const T* __restrict__ b, const double* __restrict__ lmax,
                                                   double ratio, T* __restrict__ cr, T* __restrict__ d1,
                                                   T* __restrict__ x, const int* done) {
  if (*done) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = g / LPR, lane = g % LPR;
  double s = 0.0;
  if (i < n)
    for (int k = rp[i] + lane; k < rp[i + 1]; k += LPR) s += double(A[k]) * (double(dinv[cols[k]]) * double(b[cols[k]]));
  s = group_sum<LPR>(s);
  if (i >= n || lane) return;
  const ChebStep c = cheb_step(lmax[1], ratio, 1);
  const double di = double(dinv[i]), db = di * double(b[i]);
  const double r1 = db - di * s * c.inv_theta, d0 = db * c.inv_theta;
  const double dn = c.c1 * d0 + c.c2 * r1;
  cr[i] = T(r1);
  d1[i] = T(dn);
  x[i] = T(d0 + dn);
}

// Post-smoothing, step 0 from the iterate t: r_0 = Dinv (b - A t), d_0 = r_0 /
// theta, x = t + d_0.
template <class T, int LPR>
__global__ void __launch_bounds__(AB) k_cheb_start(int n, const int* __restrict__ rp, const int* __restrict__ cols,
                                                   const T* __restrict__ A, const T* __restrict__ dinv,
                                                   const T* __restrict__ b, const T* __restrict__ t,
                                                   const double* __restrict__ lmax, double ratio,
                                                   T* __restrict__ cr, T* __restrict__ d0, T* __restrict__ x,
                                                   const int* done) {
  if (*done) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = g / LPR, lane = g % LPR;
  double s = 0.0;
  if (i < n)
    for (int k = rp[i] + lane; k < rp[i + 1]; k += LPR) s += double(A[k]) * double(t[cols[k]]);
  s = group_sum<LPR>(s);
  if (i >= n || lane) return;
  const ChebStep c = cheb_step(lmax[1], ratio, 0);
  const double r0 = double(dinv[i]) * (double(b[i]) - s), d = r0 * c.inv_theta;
  cr[i] = T(r0);
  d0[i] = T(d);
  x[i] = T(double(t[i]) + d);
}

// Step k >= 1: r -= Dinv A d_in, d_out = c1 d_in + c2 r, x += d_out (each row
// updates only its own r and x; the neighbours are read from d_in)
template <class T, int LPR>
__global__ void __launch_bounds__(AB) k_cheb_next(int n, const int* __restrict__ rp, const int* __restrict__ cols,
                                                  const T* __restrict__ A, const T* __restrict__ dinv,
                                                  const T* __restrict__ d_in, const double* __restrict__ lmax,
                                                  double ratio, int step, T* __restrict__ cr, T* __restrict__ d_out,
                                                  T* __restrict__ x, const int* done) {
  if (*done) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = g / LPR, lane = g % LPR;
  double s = 0.0;
  if (i < n)
    for (int k = rp[i] + lane; k < rp[i + 1]; k += LPR) s += double(A[k]) * double(d_in[cols[k]]);
  s = group_sum<LPR>(s);
  if (i >= n || lane) return;
  const ChebStep c = cheb_step(lmax[1], ratio, step);
  const double r = double(cr[i]) - double(dinv[i]) * s;
  const double dn = c.c1 * double(d_in[i]) + c.c2 * r;
  cr[i] = T(r);
  d_out[i] = T(dn);
  x[i] = T(double(x[i]) + dn);
}

// residual r = b - A x
template <class T, int LPR>
__global__ void __launch_bounds__(AB) k_resid(int n, const int* __restrict__ rp, const int* __restrict__ cols,
                                              const T* __restrict__ A, const T* __restrict__ b,
                                              const T* __restrict__ x, T* __restrict__ r, const int* done) {
  if (*done) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = g / LPR, lane = g % LPR;
  double s = 0.0;
  if (i < n)
    for (int k = rp[i] + lane; k < rp[i + 1]; k += LPR) s += double(A[k]) * double(x[cols[k]]);
  s = group_sum<LPR>(s);
  if (i < n && lane == 0) r[i] = T(double(b[i]) - s);
}

#define OA_LPR_LAUNCH(lpr, kernel, T, rows, st, ...)                                         \
  do {                                                                                        \
    if ((lpr) == 1)                                                                           \
      kernel<T, 1><<<grid_for(rows, 1), AB, 0, st>>>(__VA_ARGS__);                            \
    else if ((lpr) == 4)                                                                      \
      kernel<T, 4><<<grid_for(rows, 4), AB, 0, st>>>(__VA_ARGS__);                            \
    else if ((lpr) == 8)                                                                      \
      kernel<T, 8><<<grid_for(rows, 8), AB, 0, st>>>(__VA_ARGS__);                            \
    else                                                                                      \
      kernel<T, 32><<<grid_for(rows, 32), AB, 0, st>>>(__VA_ARGS__);                          \
  } while (0)

// ---------------------------------------------------------------------------
template <class T>
int Amg<T>::numeric(const T* A_fine, cudaStream_t st) {
  if (!ready) return fail(OA_ERR_NOT_READY, "AMG: numeric before setup");
  L[0].A = const_cast<T*>(A_fine);
  for (size_t l = 0; l < L.size(); ++l) {
    AmgLevel<T>& v = L[l];
    k_dinv<T><<<(v.n + AB - 1) / AB, AB, 0, st>>>(v.n, v.rp, v.diag, v.A, v.dinv);
    count_launches(1);
    if (v.cheb) {
      // the estimate runs in FP64 on an FP64 copy of the level (small by
      // construction: at most cheb_rows rows)
      k_widen<T><<<(v.nnz + AB - 1) / AB, AB, 0, st>>>(v.nnz, v.A, v.pw_a);
      k_widen<T><<<(v.n + AB - 1) / AB, AB, 0, st>>>(v.n, v.dinv, v.pw_dinv);
      k_power_init<<<(v.n + AB - 1) / AB, AB, 0, st>>>(v.n, v.pw_v, v.lmax);
      const int nb = (int)grid_for(v.n, v.lpr_a);
      for (int it = 0; it < POWER_STEPS; ++it) {
        const double* vin = (it & 1) ? v.pw_w : v.pw_v;
        double* wout = (it & 1) ? v.pw_v : v.pw_w;
        switch (v.lpr_a) {
          case 1: k_power_apply<1><<<nb, AB, 0, st>>>(v.n, v.rp, v.cols, v.pw_a, v.pw_dinv, vin, v.lmax, wout, v.pw_part); break;
          case 4: k_power_apply<4><<<nb, AB, 0, st>>>(v.n, v.rp, v.cols, v.pw_a, v.pw_dinv, vin, v.lmax, wout, v.pw_part); break;
          case 8: k_power_apply<8><<<nb, AB, 0, st>>>(v.n, v.rp, v.cols, v.pw_a, v.pw_dinv, vin, v.lmax, wout, v.pw_part); break;
          default: k_power_apply<32><<<nb, AB, 0, st>>>(v.n, v.rp, v.cols, v.pw_a, v.pw_dinv, vin, v.lmax, wout, v.pw_part);
        }
        k_power_norm<<<1, AB, 0, st>>>(nb, v.pw_part, v.lmax);
      }
      count_launches(3 + 2 * POWER_STEPS);
    }
    if (l + 1 < L.size()) {
      AmgLevel<T>& c = L[l + 1];
      if (smoothed) {
        OA_LPR_LAUNCH(v.lpr_p, k_sa_prolongator, T, v.n, st, v.n, v.p_rp, v.p_diag, v.pg_ptr, v.pg_list, v.A,
                      v.dinv, omega_p, v.pv);
        k_gather<T><<<(v.nnz_p + AB - 1) / AB, AB, 0, st>>>(v.nnz_p, v.pt_src, v.pv, v.ptv);
        OA_LPR_LAUNCH(v.lpr_t, k_pair_sum, T, v.nnz_t, st, v.nnz_t, v.tt_ptr, v.tt_a, v.tt_p, v.A, v.pv, v.tv);
        OA_LPR_LAUNCH(v.lpr_c, k_pair_sum, T, c.nnz, st, c.nnz, v.ct_ptr, v.ct_p, v.ct_t, v.pv, v.tv, c.A);
        count_launches(4);
      } else {
        k_galerkin<T><<<(c.nnz + AB - 1) / AB, AB, 0, st>>>(c.nnz, v.gptr, v.glist, v.A, c.A);
        count_launches(1);
      }
    }
  }
  const AmgLevel<T>& cl = L.back();
  k_dense_fill<T><<<cl.n, 128, 0, st>>>(cl.n, cl.rp, cl.cols, cl.A, dense_inv);
  k_gauss_jordan<<<1, 1024, 0, st>>>(cl.n, dense_inv);
  count_launches(2);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

template <class T>
int Amg<T>::apply(const T* v, T* z, const int* done, cudaStream_t st) {
  const int nl = (int)L.size();
  // downward pass: smooth + residual (row parallel), then restriction
  for (int l = 0; l < nl; ++l) {
    AmgLevel<T>& lv = L[l];
    const T* b = l == 0 ? v : lv.b;
    if (l == nl - 1) {
      T* x = l == 0 ? z : lv.x;
      k_dense_apply<T><<<grid_for(lv.n, 32), AB, 0, st>>>(lv.n, dense_inv, b, x, done);
      break;
    }
    AmgLevel<T>& c = L[l + 1];
    if (lv.cheb) {
      OA_LPR_LAUNCH(lv.lpr_a, k_cheb_first, T, lv.n, st, lv.n, lv.rp, lv.cols, lv.A, lv.dinv, b, lv.lmax, cheb_ratio,
                    lv.cr, lv.cd1, lv.t, done);
      for (int k = 2; k < cheb_degree; ++k) {
        const T* din = (k & 1) ? lv.cd0 : lv.cd1;
        T* dout = (k & 1) ? lv.cd1 : lv.cd0;
        OA_LPR_LAUNCH(lv.lpr_a, k_cheb_next, T, lv.n, st, lv.n, lv.rp, lv.cols, lv.A, lv.dinv, din, lv.lmax,
                      cheb_ratio, k, lv.cr, dout, lv.t, done);
      }
      OA_LPR_LAUNCH(lv.lpr_a, k_resid, T, lv.n, st, lv.n, lv.rp, lv.cols, lv.A, b, lv.t, lv.r, done);
    } else {
      OA_LPR_LAUNCH(lv.lpr_a, k_smooth_resid, T, lv.n, st, lv.n, lv.rp, lv.cols, lv.A, lv.dinv, b, lv.t, lv.r,
                    omega, done);
    }
    if (smoothed)
      OA_LPR_LAUNCH(lv.lpr_pt, k_sa_restrict, T, c.n, st, c.n, lv.pt_rp, lv.pt_rows, lv.ptv, lv.r, c.b, done);
    else
      k_restrict<T><<<(c.n + AB - 1) / AB, AB, 0, st>>>(c.n, lv.mptr, lv.mlist, lv.r, c.b, done);
  }
  // upward pass: prolongation + post-smooth (one fused kernel for the
  // piecewise-constant prolongation, two for the smoothed one)
  for (int l = nl - 2; l >= 0; --l) {
    AmgLevel<T>& lv = L[l];
    const T* b = l == 0 ? v : lv.b;
    T* x = l == 0 ? z : lv.x;
    if (smoothed) {
      OA_LPR_LAUNCH(lv.lpr_p, k_sa_prolong_add, T, lv.n, st, lv.n, lv.p_rp, lv.p_cols, lv.pv, L[l + 1].x, lv.t,
                    alpha, done);
      if (lv.cheb) {
        OA_LPR_LAUNCH(lv.lpr_a, k_cheb_start, T, lv.n, st, lv.n, lv.rp, lv.cols, lv.A, lv.dinv, b, lv.t, lv.lmax,
                      cheb_ratio, lv.cr, lv.cd0, x, done);
        for (int k = 1; k < cheb_degree; ++k) {
          const T* din = (k & 1) ? lv.cd0 : lv.cd1;
          T* dout = (k & 1) ? lv.cd1 : lv.cd0;
          OA_LPR_LAUNCH(lv.lpr_a, k_cheb_next, T, lv.n, st, lv.n, lv.rp, lv.cols, lv.A, lv.dinv, din, lv.lmax,
                        cheb_ratio, k, lv.cr, dout, x, done);
        }
      } else {
        OA_LPR_LAUNCH(lv.lpr_a, k_post_smooth, T, lv.n, st, lv.n, lv.rp, lv.cols, lv.A, lv.dinv, b, lv.t, x, omega,
                      done);
      }
    } else {
      k_up<T><<<(lv.n + AB - 1) / AB, AB, 0, st>>>(lv.n, lv.rp, lv.cols, lv.A, lv.dinv, lv.agg, b, lv.t, L[l + 1].x,
                                                    x, omega, alpha, done);
    }
  }
  count_launches((smoothed ? 4 : 3) * (long long)(nl - 1) + 1 + cheb_launches);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

template <class T>
int Amg<T>::set_smoothing(int degree, double prolongation_damping) {
  if (degree < 2 || degree > MAX_CHEB || !(prolongation_damping > 0.0 && prolongation_damping < 1.5))
    return fail(OA_ERR_ARG, "AMG: Chebyshev degree 2..6 and prolongation damping in (0, 1.5)");
  omega_p = prolongation_damping;
  if (!smoothed) return OA_OK;
  cheb_degree = degree;
  cheb_launches = 0;
  for (const AmgLevel<T>& lv : L)
    if (lv.cheb) cheb_launches += 2LL * (cheb_degree - 1);
  return OA_OK;
}

template struct Amg<double>;
template struct Amg<float>;

}  // namespace oa
