// Scalar linear solve with optional FP32 inner iterations and FP64 iterative
// refinement (shared by the pressure-correction and scalar-diffusion paths).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "oa_internal.h"
#include "oa_scalar_solve.h"

namespace oa {

constexpr int INNER_CAP = 300;  // FP32 Krylov iterations per refinement pass

namespace {
__global__ void k_narrow(int n, const double* __restrict__ a, float* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = float(a[i]);
}

// ---- graph form: the host decisions of solve() as one-thread kernels ----

// Largest relative change of the diagonal since the last numeric refresh,
// max_i |a_ii / ref_i - 1|, into *out (zeroed before) as the bits of a
// non-negative double, whose integer order is the numeric one.
template <class T>
__global__ void k_diag_drift(int n, const int* __restrict__ rp, const int* __restrict__ dg, const T* __restrict__ A,
                             const double* __restrict__ ref, unsigned long long* out) {
  double m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double d = double(A[rp[i] + dg[i]]), r = ref[i];
    const double c = r != 0.0 ? fabs(d / r - 1.0) : (d != 0.0 ? INFINITY : 0.0);
    m = fmax(m, c);
  }
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// the diagonal the next drift test compares against
template <class T>
__global__ void k_diag_store(int n, const int* __restrict__ rp, const int* __restrict__ dg, const T* __restrict__ A,
                             double* __restrict__ ref) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ref[i] = double(A[rp[i] + dg[i]]);
}

// AMG numeric phase on every refresh-th solve (the counter persists across
// graph launches) and on any solve whose matrix drifted
__global__ void k_refresh_if(cudaGraphConditionalHandle h, ScalarGraphState* S, int refresh,
                             const unsigned long long* drift, double drift_max) {
  const double dr = __longlong_as_double((long long)*drift);
  const int go = refresh <= 1 || (S->refresh_ctr % refresh) == 0 || dr > drift_max;
  S->refresh_ctr += 1;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

constexpr int DRIFT_BLOCKS = 4 * 148;

template <class T>
int launch_drift(const ScalarGraph& g, const void* A, const double* ref, unsigned long long* drift, cudaStream_t st) {
  OA_CUDA(cudaMemsetAsync(drift, 0, sizeof(unsigned long long), st));
  k_diag_drift<T><<<DRIFT_BLOCKS, 256, 0, st>>>(g.nn, g.rp, g.diag, static_cast<const T*>(A), ref, drift);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

template <class T>
int launch_store(const ScalarGraph& g, const void* A, double* ref, cudaStream_t st) {
  k_diag_store<T><<<(g.nn + 255) / 256, 256, 0, st>>>(g.nn, g.rp, g.diag, static_cast<const T*>(A), ref);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

// FP64: a GCR(2) solve that stagnated or broke down is redone by BiCGStab
__global__ void k_fallback_if(cudaGraphConditionalHandle h, const KScal* sc, ScalarGraphState* S) {
  const int fb = sc->status == 1;
  S->fallback = fb;
  S->spent = fb ? sc->iters : 0;
  cudaGraphSetConditional(h, fb ? 1u : 0u);
}

// mixed: entry of the refinement loop (||b|| from the reduction before it)
__global__ void k_ir_begin(cudaGraphConditionalHandle h, ScalarGraphState* S, double rtol, int maxit, double floor,
                           int use_gcr, int seg) {
  const double bn = sqrt(S->bsq);
  S->seg = seg;
  S->bnorm = bn;
  S->rtol = rtol;
  S->maxit = maxit;
  S->floor = floor;
  S->use_gcr = use_gcr;
  S->total = 0;
  S->nref = 0;
  S->fallback = 0;
  S->it_last = 0;
  S->apply = 0;
  S->spent = 0;
  S->status = bn < INFINITY ? 0 : 3;  // 3: non-finite right-hand side
  S->rel = bn > 0 ? 1.0 : 0.0;
  cudaGraphSetConditional(h, (S->status == 0 && S->rel > rtol && maxit > 0) ? 1u : 0u);
}

// inner tolerance and iteration budget of a pass; selects GCR(2) or BiCGStab
__global__ void k_ir_params(cudaGraphConditionalHandle hsel, ScalarGraphState* S) {
  const double inner = fmax(S->rtol / S->rel, S->floor);
  S->inner_rtol = fmin(inner, 0.1);
  S->inner_maxit = min(INNER_CAP, S->maxit - S->total);
  cudaGraphSetConditional(hsel, S->use_gcr ? 1u : 0u);
}

// after the inner solve: iteration count, the switch to BiCGStab for a GCR(2)
// stall far from its target, and whether the correction is applied
__global__ void k_ir_after(ScalarGraphState* S, const KScal* sc) {
  const int it = sc->iters;
  const double r_in = sc->bnorm > 0 ? sc->rnorm / sc->bnorm : 0.0;
  S->it_last = it;
  S->r_in = r_in;
  S->total += it;
  if (S->use_gcr && sc->status == 1 && r_in > 10.0 * S->inner_rtol) {
    S->use_gcr = 0;
    S->fallback += 1;
  }
  if (sc->status == 2 && S->status == 0) S->status = 4;  // 4: non-finite inner residual
  S->apply = (sc->status != 3 && r_in < 1.0) ? 1 : 0;
}

template <class TV>
__global__ void k_add_correction_if(int n, double* x, const TV* d, const ScalarGraphState* S) {
  if (!S->apply) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += double(d[i]);
}

// end of a pass: relative FP64 residual, loop condition
__global__ void k_ir_next(cudaGraphConditionalHandle h, ScalarGraphState* S, BodyCounters* c, int body) {
  c->total[body] += 1;
  double rel = S->bnorm > 0 ? S->rnorm_out / S->bnorm : 0.0;
  if (S->seg && rel < INFINITY) rel = S->rel_seg;  // the worst segment of a batch
  S->rel = rel;
  S->nref += 1;
  if (!(rel < INFINITY) && S->status == 0) S->status = 2;
  const bool go = S->status == 0 && rel > S->rtol && S->total < S->maxit && S->nref < 40 && S->it_last != 0;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}
}  // namespace

int ScalarSolve::init(int nn) {
  if (const char* e = std::getenv("OA_AMG_REFRESH")) refresh = std::max(1, std::atoi(e));
  if (const char* e = std::getenv("OA_AMG_DRIFT")) drift_max = std::atof(e);
  if (const char* e = std::getenv("OA_IR_INNER")) inner_floor = std::atof(e);
  if (const char* e = std::getenv("OA_KRYLOV")) gcr = std::strcmp(e, "bicgstab") != 0;
  if (const char* e = std::getenv("OA_GCR_CHUNK")) gcr_chunk = std::max(2, std::atoi(e) / 2 * 2);
  if (n == nn && r) return OA_OK;
  release();
  n = nn;
  if (cudaMalloc(&r, sizeof(double) * (nn ? nn : 1)) != cudaSuccess ||
      cudaMalloc(&r32, sizeof(float) * (nn ? nn : 1)) != cudaSuccess ||
      cudaMalloc(&scal, sizeof(double) * 2) != cudaSuccess ||
      cudaMalloc(&partials, sizeof(double) * partials_size()) != cudaSuccess ||
      cudaMalloc(&diag_ref, sizeof(double) * (nn ? nn : 1)) != cudaSuccess ||
      cudaMalloc(&drift, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMallocHost(&hdrift, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMallocHost(&hscal, sizeof(double) * 2) != cudaSuccess) {
    release();
    return fail(OA_ERR_CUDA, "scalar solve: device allocation failed");
  }
  return OA_OK;
}

int ScalarSolve::set_segments(const std::vector<int>& ptr, const std::vector<int>& rows) {
  release_segments();
  const int nseg = (int)ptr.size() - 1;
  if (nseg <= 1) return OA_OK;
  if (cudaMalloc(&seg_dev, sizeof(int) * (ptr.size() + rows.size())) != cudaSuccess ||
      cudaMalloc(&seg_buf, sizeof(double) * 4 * nseg) != cudaSuccess ||
      cudaMalloc(&seg_rel, sizeof(double)) != cudaSuccess) {
    release_segments();
    return fail(OA_ERR_CUDA, "scalar solve: segment allocation failed");
  }
  OA_CUDA(cudaMemcpy(seg_dev, ptr.data(), sizeof(int) * ptr.size(), cudaMemcpyHostToDevice));
  OA_CUDA(cudaMemcpy(seg_dev + ptr.size(), rows.data(), sizeof(int) * rows.size(), cudaMemcpyHostToDevice));
  seg_in.nseg = seg_out.nseg = nseg;
  seg_in.ptr = seg_out.ptr = seg_dev;
  seg_in.rows = seg_out.rows = seg_dev + ptr.size();
  seg_in.b2 = seg_buf;
  seg_in.r2 = seg_buf + nseg;
  seg_out.b2 = seg_buf + 2 * nseg;
  seg_out.r2 = seg_buf + 3 * nseg;
  return OA_OK;
}

void ScalarSolve::release_segments() {
  if (seg_dev) cudaFree(seg_dev);
  if (seg_buf) cudaFree(seg_buf);
  if (seg_rel) cudaFree(seg_rel);
  seg_dev = nullptr;
  seg_buf = nullptr;
  seg_rel = nullptr;
  seg_in = Segments{};
  seg_out = Segments{};
  k64.seg = Segments{};
  k32.seg = Segments{};
}

void ScalarSolve::release() {
  if (gs) cudaFree(gs);
  if (gs_host) cudaFreeHost(gs_host);
  if (k_host) cudaFreeHost(k_host);
  gs = nullptr;
  gs_host = nullptr;
  k_host = nullptr;
  if (diag_ref) cudaFree(diag_ref);
  if (drift) cudaFree(drift);
  if (hdrift) cudaFreeHost(hdrift);
  diag_ref = nullptr;
  drift = nullptr;
  hdrift = nullptr;
  if (r) cudaFree(r);
  if (r32) cudaFree(r32);
  if (scal) cudaFree(scal);
  if (partials) cudaFree(partials);
  if (hscal) cudaFreeHost(hscal);
  r = nullptr;
  r32 = nullptr;
  scal = nullptr;
  partials = nullptr;
  hscal = nullptr;
  n = 0;
  k64.release();
  k32.release();
  amg64.release();
  amg32.release();
}

int ScalarSolve::solve(const ScalarGraph& g, bool mixed, bool amg, bool graphs, const void* A, const double* b,
                       double* x, double rtol, int maxit, int* iters, double* res, int* refinements, cudaStream_t st,
                       const char* what) {
  if (int s = init(g.nn)) return s;
  if (amg) {
    if (!mixed && !amg64.ready)
      if (int s = amg64.setup(g.nn, g.h_rp, g.h_cols, g.h_diag, g.rp, g.cols, g.diag)) return s;
    if (mixed && !amg32.ready)
      if (int s = amg32.setup(g.nn, g.h_rp, g.h_cols, g.h_diag, g.rp, g.cols, g.diag)) return s;
    k64.amg = mixed ? nullptr : &amg64;
    k32.amg = mixed ? &amg32 : nullptr;
  } else {
    k64.amg = nullptr;
    k32.amg = nullptr;
  }
  k64.use_graph = k32.use_graph = graphs;
  k64.seg = k32.seg = seg_in;
  // with the AMG: GCR(2), one V-cycle per iteration (chunks of 4); with point
  // Jacobi: BiCGStab
  k64.gcr = k32.gcr = amg && gcr;
  int check_every = amg ? (gcr ? gcr_chunk : 5) : 20;
  // AMG numeric phase every refresh-th solve (the fine matrix is always the
  // current one; the coarse operators may lag by refresh - 1 assemblies)
  bool reuse = amg && refresh > 1 && (solves++ % refresh) != 0;
  if (reuse) {
    // a matrix that drifted from the hierarchy's refreshes it early
    if (int s = mixed ? launch_drift<float>(g, A, diag_ref, drift, st) : launch_drift<double>(g, A, diag_ref, drift, st))
      return s;
    OA_CUDA(cudaMemcpyAsync(hdrift, drift, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    OA_CUDA(cudaStreamSynchronize(st));
    double dr;
    std::memcpy(&dr, hdrift, sizeof(double));
    if (dr > drift_max) reuse = false;
  }
  if (amg && !reuse)
    if (int s = mixed ? launch_store<float>(g, A, diag_ref, st) : launch_store<double>(g, A, diag_ref, st)) return s;
  if (!mixed) {
    if (int s = k64.setup(g.nn, g.rp, g.cols, g.diag, st)) return s;
    double* xs = nullptr;
    if (int s = k64.solve<double>(static_cast<const double*>(A), b, xs, rtol, maxit, iters, res, check_every, reuse))
      return s;
    if (k64.gcr && k64.last_status == 1) {
      // GCR stagnated or broke down: BiCGStab from now on, and for this system;
      // the reported count includes the GCR iterations already spent
      gcr = false;
      k64.gcr = false;
      const int spent = iters ? *iters : 0;
      if (int s = k64.solve<double>(static_cast<const double*>(A), b, xs, rtol, maxit, iters, res, 5, true)) return s;
      if (iters) *iters += spent;
      ++fallbacks;
    }
    OA_CUDA(cudaMemcpyAsync(x, xs, sizeof(double) * g.nn, cudaMemcpyDeviceToDevice, st));
    if (refinements) *refinements = 0;
    return OA_OK;
  }
  if (int s = k32.setup(g.nn, g.rp, g.cols, g.diag, st)) return s;
  const float* A32 = static_cast<const float*>(A);
  OA_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * g.nn, st));
  if (int s = device_sumsq(g.nn, b, scal, partials, st)) return s;
  OA_CUDA(cudaMemcpyAsync(hscal, scal, sizeof(double), cudaMemcpyDeviceToHost, st));
  OA_CUDA(cudaStreamSynchronize(st));
  const double bnorm = std::sqrt(hscal[0]);
  if (!(bnorm < INFINITY)) return fail(OA_ERR_SOLVER, std::string(what) + ": non-finite right-hand side");
  int total = 0, nref = 0;
  double rel = bnorm > 0 ? 1.0 : 0.0;
  OA_CUDA(cudaMemcpyAsync(r, b, sizeof(double) * g.nn, cudaMemcpyDeviceToDevice, st));
  if (seg_out.on())
    if (int s = segment_sumsq<double>(seg_out, b, seg_out.b2, st)) return s;
  const double floor0 = floor_default(amg);  // fixed for the whole solve, as in the graph form
  while (rel > rtol && total < maxit && nref < 40) {
    k_narrow<<<(g.nn + 255) / 256, 256, 0, st>>>(g.nn, r, r32);
    count_launches(1);
    float* d = nullptr;
    int it = 0;
    double r_in = 0.0;
    // inner tolerance: enough digits for FP32 without stalling
    const double inner = std::max(rtol / rel, floor0);
    if (int s = k32.solve<float>(A32, r32, d, std::min(inner, 0.1), std::min(INNER_CAP, maxit - total), &it, &r_in,
                                 check_every, reuse || nref > 0))
      return s;
    total += it;
    if (k32.gcr && k32.last_status == 1 && r_in > 10.0 * std::min(inner, 0.1)) {
      // GCR stagnated or broke down far from its target (its partial
      // correction still reduced the residual): BiCGStab for the remaining
      // passes and later solves. A stall within a decade of the target is the
      // FP32 floor and only ends the pass.
      gcr = false;
      k32.gcr = false;
      check_every = 5;
      ++fallbacks;
    }
    // a diverged inner solve contributes nothing; the next pass restarts from
    // the FP64 residual
    if (k32.last_status != 3 && r_in < 1.0) add_correction<float>(g.nn, x, d, st);
    if (int s = fp64_residual<float>(g.nn, g.rp, g.cols, A32, x, b, r, k32.partials, scal + 1, st)) return s;
    OA_CUDA(cudaMemcpyAsync(hscal + 1, scal + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (seg_out.on()) {
      // batched disjoint systems: the worst segment's relative residual
      if (int s = segment_sumsq<double>(seg_out, r, seg_out.r2, st)) return s;
      if (int s = segment_max_ratio(seg_out, seg_rel, st)) return s;
      OA_CUDA(cudaMemcpyAsync(hscal, seg_rel, sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    OA_CUDA(cudaStreamSynchronize(st));
    rel = seg_out.on() ? hscal[0] : (bnorm > 0 ? hscal[1] / bnorm : 0.0);
    if (!(hscal[1] < INFINITY)) rel = hscal[1];
    if (std::getenv("OA_DEBUG"))
      std::fprintf(stderr, "[oa] %s refinement %d: inner iters %d inner res %.3e |b| %.3e rel %.3e\n", what, nref, it,
                   r_in, bnorm, rel);
    ++nref;
    if (!(rel < INFINITY)) return fail(OA_ERR_SOLVER, std::string(what) + " refinement: non-finite residual");
    if (it == 0) break;
  }
  if (iters) *iters = total;
  if (res) *res = rel;
  if (refinements) *refinements = nref;
  return OA_OK;
}

int ScalarSolve::emit(GraphBuild& gb, cudaGraph_t g, Deps& d, const ScalarGraph& gr, bool mixed, bool amg,
                      const void* A, const double* b, double* x, double rtol, int maxit, cudaStream_t st) {
  if (int s = init(gr.nn)) return s;
  if (amg && !(mixed ? amg32.ready : amg64.ready))
    return fail(OA_ERR_NOT_READY, "scalar solve graph: the preconditioner is set up by a first eager solve");
  if (!gs) {
    if (cudaMalloc(&gs, sizeof(ScalarGraphState)) != cudaSuccess ||
        cudaMallocHost(&gs_host, sizeof(ScalarGraphState)) != cudaSuccess ||
        cudaMallocHost(&k_host, sizeof(KScal)) != cudaSuccess)
      return fail(OA_ERR_CUDA, "scalar solve graph: allocation failed");
    OA_CUDA(cudaMemsetAsync(gs, 0, sizeof(ScalarGraphState), st));
  }
  k64.amg = amg && !mixed ? &amg64 : nullptr;
  k32.amg = amg && mixed ? &amg32 : nullptr;
  k64.seg = k32.seg = seg_in;
  if (mixed) {
    if (int s = k32.setup(gr.nn, gr.rp, gr.cols, gr.diag, st)) return s;
  } else if (int s = k64.setup(gr.nn, gr.rp, gr.cols, gr.diag, st)) {
    return s;
  }
  const bool use_gcr = amg && gcr;
  const int chunk_gcr = gcr_chunk;
  // AMG numeric phase under the refresh IF
  if (amg) {
    cudaGraphConditionalHandle hn;
    if (int s = gb.handle(g, &hn)) return s;
    if (int s = gb.seg(g, d, -1, [&]() -> int {
          if (refresh > 1)
            if (int s2 = mixed ? launch_drift<float>(gr, A, diag_ref, drift, st)
                               : launch_drift<double>(gr, A, diag_ref, drift, st))
              return s2;
          k_refresh_if<<<1, 1, 0, st>>>(hn, gs, refresh, drift, refresh > 1 ? drift_max : INFINITY);
          count_launches(1);
          return OA_OK;
        }))
      return s;
    cudaGraph_t nb = nullptr;
    if (int s = gb.cond(g, d, hn, cudaGraphCondTypeIf, 1, &nb)) return s;
    const int bid = gb.new_body();
    if (bid < 0) return fail(OA_ERR_ARG, "scalar solve graph: too many conditional bodies");
    Deps nd;
    if (int s = gb.seg(nb, nd, bid, [&]() -> int {
          if (int s2 = launch_count_body(gb, bid)) return s2;
          if (int s2 = mixed ? launch_store<float>(gr, A, diag_ref, st) : launch_store<double>(gr, A, diag_ref, st))
            return s2;
          return mixed ? amg32.numeric(static_cast<const float*>(A), st)
                       : amg64.numeric(static_cast<const double*>(A), st);
        }))
      return s;
  }
  if (!mixed) {
    const double* A64 = static_cast<const double*>(A);
    if (int s = k64.emit<double>(gb, g, d, -1, A64, b, rtol, maxit, nullptr, nullptr, maxit,
                                 use_gcr ? chunk_gcr : (amg ? 5 : 20), use_gcr, -1))
      return s;
    if (use_gcr) {
      // the BiCGStab fallback of a stagnated GCR(2) solve
      cudaGraphConditionalHandle hf;
      if (int s = gb.handle(g, &hf)) return s;
      if (int s = gb.seg(g, d, -1, [&]() -> int {
            k_fallback_if<<<1, 1, 0, st>>>(hf, k64.scalars(), gs);
            count_launches(1);
            return OA_OK;
          }))
        return s;
      cudaGraph_t fb = nullptr;
      if (int s = gb.cond(g, d, hf, cudaGraphCondTypeIf, 1, &fb)) return s;
      const int bid = gb.new_body();
      if (bid < 0) return fail(OA_ERR_ARG, "scalar solve graph: too many conditional bodies");
      Deps fd;
      if (int s = k64.emit<double>(gb, fb, fd, bid, A64, b, rtol, maxit, nullptr, nullptr, maxit, 5, false, bid))
        return s;
    } else {
      if (int s = gb.seg(g, d, -1, [&]() -> int {
            OA_CUDA(cudaMemsetAsync(&gs->fallback, 0, sizeof(int), st));
            OA_CUDA(cudaMemsetAsync(&gs->spent, 0, sizeof(int), st));
            return OA_OK;
          }))
        return s;
    }
    return gb.seg(g, d, -1, [&]() -> int {
      OA_CUDA(cudaMemcpyAsync(x, k64.solution(), sizeof(double) * gr.nn, cudaMemcpyDeviceToDevice, st));
      OA_CUDA(cudaMemcpyAsync(k_host, k64.scalars(), sizeof(KScal), cudaMemcpyDeviceToHost, st));
      OA_CUDA(cudaMemcpyAsync(gs_host, gs, sizeof(ScalarGraphState), cudaMemcpyDeviceToHost, st));
      return OA_OK;
    });
  }
  // mixed: FP64 iterative refinement around FP32 inner solves
  const float* A32 = static_cast<const float*>(A);
  const double floor = floor_default(amg);
  cudaGraphConditionalHandle hir;
  if (int s = gb.handle(g, &hir)) return s;
  if (int s = gb.seg(g, d, -1, [&]() -> int {
        OA_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * gr.nn, st));
        if (int s2 = device_sumsq(gr.nn, b, &gs->bsq, partials, st)) return s2;
        OA_CUDA(cudaMemcpyAsync(r, b, sizeof(double) * gr.nn, cudaMemcpyDeviceToDevice, st));
        if (seg_out.on())
          if (int s2 = segment_sumsq<double>(seg_out, b, seg_out.b2, st)) return s2;
        k_ir_begin<<<1, 1, 0, st>>>(hir, gs, rtol, maxit, floor, use_gcr ? 1 : 0, seg_out.on() ? 1 : 0);
        count_launches(1);
        return OA_OK;
      }))
    return s;
  cudaGraph_t irb = nullptr;
  if (int s = gb.cond(g, d, hir, cudaGraphCondTypeWhile, 1, &irb)) return s;
  const int ir_body = gb.new_body();
  if (ir_body < 0) return fail(OA_ERR_ARG, "scalar solve graph: too many conditional bodies");
  Deps bd;
  cudaGraphConditionalHandle hsel;
  if (int s = gb.handle(irb, &hsel)) return s;
  if (int s = gb.seg(irb, bd, ir_body, [&]() -> int {
        k_narrow<<<(gr.nn + 255) / 256, 256, 0, st>>>(gr.nn, r, r32);
        k_ir_params<<<1, 1, 0, st>>>(hsel, gs);
        count_launches(2);
        return OA_OK;
      }))
    return s;
  // GCR(2) while the solve has not fallen back, else BiCGStab
  cudaGraph_t sel[2] = {nullptr, nullptr};
  if (int s = gb.cond(irb, bd, hsel, cudaGraphCondTypeIf, 2, sel)) return s;
  const int b_gcr = gb.new_body(), b_bicg = gb.new_body();
  if (b_gcr < 0 || b_bicg < 0) return fail(OA_ERR_ARG, "scalar solve graph: too many conditional bodies");
  {
    Deps d0, d1;
    if (int s = k32.emit<float>(gb, sel[0], d0, b_gcr, A32, r32, 0.0, 0, &gs->inner_rtol, &gs->inner_maxit, INNER_CAP,
                                chunk_gcr, true, b_gcr))
      return s;
    if (int s = k32.emit<float>(gb, sel[1], d1, b_bicg, A32, r32, 0.0, 0, &gs->inner_rtol, &gs->inner_maxit,
                                INNER_CAP, 5, false, b_bicg))
      return s;
  }
  if (int s = gb.seg(irb, bd, ir_body, [&]() -> int {
        k_ir_after<<<1, 1, 0, st>>>(gs, k32.scalars());
        k_add_correction_if<float><<<(gr.nn + 255) / 256, 256, 0, st>>>(gr.nn, x, k32.solution(), gs);
        count_launches(2);
        if (int s2 = fp64_residual<float>(gr.nn, gr.rp, gr.cols, A32, x, b, r, k32.partials, &gs->rnorm_out, st))
          return s2;
        if (seg_out.on()) {
          if (int s2 = segment_sumsq<double>(seg_out, r, seg_out.r2, st)) return s2;
          if (int s2 = segment_max_ratio(seg_out, &gs->rel_seg, st)) return s2;
        }
        k_ir_next<<<1, 1, 0, st>>>(hir, gs, gb.ctr, ir_body);
        count_launches(1);
        return OA_OK;
      }))
    return s;
  return gb.seg(g, d, -1, [&]() -> int {
    OA_CUDA(cudaMemcpyAsync(gs_host, gs, sizeof(ScalarGraphState), cudaMemcpyDeviceToHost, st));
    return OA_OK;
  });
}

int ScalarSolve::graph_prepare(cudaStream_t st) {
  if (!gs) return fail(OA_ERR_NOT_READY, "scalar solve graph: not captured");
  gs_host->refresh_ctr = (int)solves;
  OA_CUDA(cudaMemcpyAsync(&gs->refresh_ctr, &gs_host->refresh_ctr, sizeof(int), cudaMemcpyHostToDevice, st));
  return OA_OK;
}

int ScalarSolve::graph_result(bool mixed, int* iters, double* res, int* refinements, bool* recapture,
                              const char* what) {
  const ScalarGraphState& S = *gs_host;
  ++solves;  // the device refresh counter advanced once
  if (recapture) *recapture = false;
  if (mixed) {
    if (S.fallback) {
      gcr = false;
      k32.gcr = false;
      fallbacks += S.fallback;
      if (recapture) *recapture = true;
    }
    if (S.status == 3) return fail(OA_ERR_SOLVER, std::string(what) + ": non-finite right-hand side");
    if (S.status == 2) return fail(OA_ERR_SOLVER, std::string(what) + " refinement: non-finite residual");
    if (S.status == 4) return fail(OA_ERR_SOLVER, std::string(what) + ": non-finite residual in an inner solve");
    if (iters) *iters = S.total;
    if (res) *res = S.rel;
    if (refinements) *refinements = S.nref;
    return OA_OK;
  }
  const KScal& K = *k_host;
  if (S.fallback) {
    gcr = false;
    k64.gcr = false;
    ++fallbacks;
    if (recapture) *recapture = true;
  }
  if (K.status == 2) return fail(OA_ERR_SOLVER, std::string(what) + ": non-finite residual");
  if (iters) *iters = K.iters + S.spent;
  if (res) *res = seg_in.on() ? K.seg_rel : (K.bnorm > 0 ? K.rnorm / K.bnorm : 0.0);
  if (refinements) *refinements = 0;
  return OA_OK;
}

}  // namespace oa
