// Aggregation AMG V-cycle for the pressure-correction system (see oa_amg.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "oa_amg.h"
#include "oa_internal.h"

namespace oa {

constexpr int AB = 256;          // threads per block
constexpr int COARSE_MAX = 256;  // coarsest level solved by a dense inverse

// ---------------------------------------------------------------------------
// host: greedy aggregation of a CSR graph (root + all its free neighbours,
// then leftover rows join an adjacent aggregate)
static int aggregate(int n, const std::vector<int>& rp, const std::vector<int>& cols, std::vector<int>& agg) {
  agg.assign(n, -1);
  int nc = 0;
  for (int i = 0; i < n; ++i) {
    if (agg[i] != -1) continue;
    bool free_nb = true;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (cols[k] != i && agg[cols[k]] != -1) {
        free_nb = false;
        break;
      }
    if (!free_nb) continue;
    agg[i] = nc;
    for (int k = rp[i]; k < rp[i + 1]; ++k) agg[cols[k]] = nc;
    ++nc;
  }
  std::vector<int> pass1(agg);
  for (int i = 0; i < n; ++i) {
    if (agg[i] != -1) continue;
    int best = -1;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (pass1[cols[k]] != -1) {
        best = pass1[cols[k]];
        break;
      }
    agg[i] = best >= 0 ? best : nc++;
  }
  return nc;
}

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
  std::vector<int> rp(h_rp, h_rp + n + 1), cols(h_cols, h_cols + h_rp[n]), dg(h_diag, h_diag + n);
  int cur = n;
  for (int lev = 0;; ++lev) {
    AmgLevel<T> lv;
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
    const bool last = cur <= COARSE_MAX || lev >= 14;
    if (last) {
      L.push_back(lv);
      break;
    }
    std::vector<int> agg;
    const int nc = aggregate(cur, rp, cols, agg);
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
    std::vector<int> crp(nc + 1, 0), ccols, cdg(nc, 0);
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
          const int pos = (int)(std::lower_bound(ccols.begin() + crp[c], ccols.begin() + crp[c + 1], cj) - ccols.begin());
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
    L.push_back(lv);
    rp.swap(crp);
    cols.swap(ccols);
    dg.swap(cdg);
    cur = nc;
  }
  coarse_n = L.back().n;
  if (cudaMalloc(&dense_inv, sizeof(double) * 2 * (size_t)coarse_n * coarse_n) != cudaSuccess)
    return fail(OA_ERR_CUDA, "AMG: dense coarse allocation failed");
  // tuning knobs (Jacobi damping, coarse-correction scaling)
  if (const char* e = std::getenv("OA_AMG_OMEGA")) omega = std::atof(e);
  if (const char* e = std::getenv("OA_AMG_ALPHA")) alpha = std::atof(e);
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
    void* p[] = {v.dinv, v.agg, v.mptr, v.mlist, v.gptr, v.glist, v.r, v.t};
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
// the right half.
__global__ void k_gauss_jordan(int n, double* M) {
  const int w = 2 * n;
  for (int k = 0; k < n; ++k) {
    __syncthreads();
    const double piv = M[(size_t)k * w + k];
    __syncthreads();
    for (int j = threadIdx.x; j < w; j += blockDim.x) M[(size_t)k * w + j] /= piv;
    __syncthreads();
    for (int idx = threadIdx.x; idx < n * w; idx += blockDim.x) {
      const int i = idx / w, j = idx - i * w;
      if (i == k || j == k) continue;
      M[(size_t)i * w + j] -= M[(size_t)i * w + k] * M[(size_t)k * w + j];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      if (i != k) M[(size_t)i * w + k] = 0.0;
  }
}

// Downward step, row parallel: pre-smooth from zero, xs_i = w Dinv_i b_i, and
// the residual r_i = b_i - sum_j a_ij xs_j (neighbours' xs formed from b).
template <class T>
__global__ void __launch_bounds__(AB) k_smooth_resid(int n, const int* __restrict__ rp, const int* __restrict__ cols,
                                                     const T* __restrict__ A, const T* __restrict__ dinv,
                                                     const T* __restrict__ b, T* __restrict__ xs, T* __restrict__ r,
                                                     double w, const int* done) {
  if (*done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const int j = cols[k];
    s += double(A[k]) * (w * double(dinv[j]) * double(b[j]));
  }
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
__global__ void k_dense_apply(int n, const double* __restrict__ M, const T* __restrict__ b, T* __restrict__ x,
                              const int* done) {
  if (*done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* row = M + (size_t)i * 2 * n + n;
  double s = 0.0;
  for (int j = 0; j < n; ++j) s += row[j] * double(b[j]);
  x[i] = T(s);
}

// ---------------------------------------------------------------------------
template <class T>
int Amg<T>::numeric(const T* A_fine, cudaStream_t st) {
  if (!ready) return fail(OA_ERR_NOT_READY, "AMG: numeric before setup");
  L[0].A = const_cast<T*>(A_fine);
  for (size_t l = 0; l < L.size(); ++l) {
    AmgLevel<T>& v = L[l];
    k_dinv<T><<<(v.n + AB - 1) / AB, AB, 0, st>>>(v.n, v.rp, v.diag, v.A, v.dinv);
    if (l + 1 < L.size()) {
      AmgLevel<T>& c = L[l + 1];
      k_galerkin<T><<<(c.nnz + AB - 1) / AB, AB, 0, st>>>(c.nnz, v.gptr, v.glist, v.A, c.A);
    }
  }
  const AmgLevel<T>& cl = L.back();
  k_dense_fill<T><<<cl.n, 128, 0, st>>>(cl.n, cl.rp, cl.cols, cl.A, dense_inv);
  k_gauss_jordan<<<1, 1024, 0, st>>>(cl.n, dense_inv);
  count_launches(2 * (long long)L.size() + 1);
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
      k_dense_apply<T><<<(lv.n + AB - 1) / AB, AB, 0, st>>>(lv.n, dense_inv, b, x, done);
      break;
    }
    AmgLevel<T>& c = L[l + 1];
    k_smooth_resid<T><<<(lv.n + AB - 1) / AB, AB, 0, st>>>(lv.n, lv.rp, lv.cols, lv.A, lv.dinv, b, lv.t, lv.r, omega,
                                                            done);
    k_restrict<T><<<(c.n + AB - 1) / AB, AB, 0, st>>>(c.n, lv.mptr, lv.mlist, lv.r, c.b, done);
  }
  // upward pass: one fused prolong/post-smooth kernel per level
  for (int l = nl - 2; l >= 0; --l) {
    AmgLevel<T>& lv = L[l];
    const T* b = l == 0 ? v : lv.b;
    T* x = l == 0 ? z : lv.x;
    k_up<T><<<(lv.n + AB - 1) / AB, AB, 0, st>>>(lv.n, lv.rp, lv.cols, lv.A, lv.dinv, lv.agg, b, lv.t, L[l + 1].x,
                                                  x, omega, alpha, done);
  }
  count_launches(3 * (long long)(nl - 1) + 1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

template struct Amg<double>;
template struct Amg<float>;

}  // namespace oa
