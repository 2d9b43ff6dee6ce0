// Scalar (1 dof per node) linear solve shared by the pressure-correction and
// the scalar-diffusion paths (internal).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "oa_amg.h"
#include "oa_krylov.h"

namespace oa {

// CSR graph of a scalar system: device arrays and the host copies the AMG
// set-up reads.
struct ScalarGraph {
  int nn = 0;
  int *rp = nullptr, *cols = nullptr, *diag = nullptr;
  const int *h_rp = nullptr, *h_cols = nullptr, *h_diag = nullptr;
};

// Device state of a graph-captured scalar solve: the refinement loop of the
// mixed form, the AMG refresh counter and the fallback bookkeeping.
struct ScalarGraphState {
  double bsq, bnorm, rel, rtol, floor, inner_rtol, r_in, rnorm_out;
  int maxit, total, nref, inner_maxit, use_gcr, fallback, status, it_last, apply;
  int refresh_ctr, refresh, spent;
  int seg;         // per-segment convergence (batched disjoint systems)
  double rel_seg;  // largest per-segment ||r|| / ||b|| of the FP64 residual
};

// FP64: BiCGStab (AMG- or Jacobi-preconditioned) to rtol. Mixed: iterative
// refinement with the FP64 residual r = b - A x (A in its stored FP32 values),
// FP32 BiCGStab on A d = r to a loose inner tolerance, x += d, until
// ||r|| <= rtol ||b||. The preconditioner hierarchy is built on first use and
// its numeric part refreshed on every solve.
struct ScalarSolve {
  KrylovSolver<1, double, double> k64;
  KrylovSolver<1, float, float> k32;
  Amg<double> amg64;
  Amg<float> amg32;
  double* r = nullptr;      // FP64 residual
  float* r32 = nullptr;     // its FP32 copy
  double* scal = nullptr;   // [2] device scalars
  double* hscal = nullptr;  // [2] pinned
  double* partials = nullptr;
  int n = 0;
  // AMG numeric phase (coarse operators, prolongation, inverse diagonals,
  // Chebyshev bounds) every refresh-th solve; between refreshes the fine
  // matrix is the current one and only the coarse operators lag. On the 128^3
  // cavity 4 kept the iteration counts of 1 and saved 5 % of the outer
  // iteration; with GCR(2) 8 still keeps them (22 per outer iteration) and
  // saves another 2 % (OA_AMG_REFRESH overrides)
  int refresh = 8;
  // ...and earlier when the matrix has drifted: a solve refreshes whenever
  // some diagonal entry moved by more than drift_max (relative) since the last
  // refresh. A hierarchy left from a much different matrix can make the
  // Chebyshev smoother diverge: on a 64 x 24 x 24 channel at mu = 1e-5 the
  // pressure solve of the second outer iteration hit maxit with refresh 8 and
  // took 13 iterations with a refresh on every solve (OA_AMG_DRIFT overrides).
  double drift_max = 0.5;
  double* diag_ref = nullptr;           // [n] FP64 diagonal at the last refresh
  unsigned long long* drift = nullptr;  // device: largest relative change (double bits)
  unsigned long long* hdrift = nullptr; // pinned mirror
  // lowest relative tolerance asked of an FP32 inner solve (0: the default of
  // floor_default); OA_IR_INNER overrides
  double inner_floor = 0.0;
  // GCR(2) with the AMG reaches 1e-5 in FP32 without stalling, and asking for
  // it leaves fewer refinement restarts: on the 128^3 cavity 73.3 against 71.3
  // outer iterations/s for 1e-4 (3e-5: 72.2, 3e-6: 73.0); BiCGStab keeps 1e-4
  // with the AMG and 2e-4 with Jacobi
  double floor_default(bool amg) const {
    if (inner_floor > 0) return inner_floor;
    return amg ? (gcr ? 1e-5 : 1e-4) : 2e-4;
  }
  // Krylov method with the AMG: GCR(2) (one V-cycle per iteration; the
  // pressure correction's default: 22 instead of 26 V-cycles per outer
  // iteration on the 128^3 cavity) or BiCGStab (two per iteration). The
  // OA_KRYLOV environment variable overrides ("bicgstab", else GCR); a GCR
  // solve that stagnates switches this solver to BiCGStab for good.
  bool gcr = true;
  // GCR iterations per device-resident chunk (even; OA_GCR_CHUNK): short
  // chunks launch fewer iterations past convergence (each a V-cycle of early
  // exits) at the price of more host checks; on the 128^3 cavity 2 beat 4, 6
  // and 8 (with refresh 8: 68.1 against 65.6 outer iterations/s for 4 and
  // refresh 4)
  int gcr_chunk = 2;
  long long solves = 0;
  // GCR(2) solves that stagnated and were finished by BiCGStab (in either
  // precision); reported so callers can see the switch happen
  int fallbacks = 0;

  // graph form (whole-iteration graphs)
  ScalarGraphState* gs = nullptr;       // device
  ScalarGraphState* gs_host = nullptr;  // pinned mirror, written by the graph's last nodes
  KScal* k_host = nullptr;              // pinned mirror of the FP64 solver's scalars

  // disjoint systems solved as one: a solve converges when every segment
  // does (inner Krylov tests on seg_in, the refinement test on seg_out)
  Segments seg_in, seg_out;
  int* seg_dev = nullptr;      // [nseg + 1 + nn] row pointers and rows
  double* seg_buf = nullptr;   // [4 nseg] sums of squares
  double* seg_rel = nullptr;   // device scalar: refinement's largest segment ratio
  int set_segments(const std::vector<int>& ptr, const std::vector<int>& rows);
  void release_segments();

  // coarse-level Chebyshev degree and prolongation damping of both
  // precisions' hierarchies (autotuned; defaults 3 and 0.74)
  int set_smoothing(int degree, double prolongation_damping) {
    if (int s = amg64.set_smoothing(degree, prolongation_damping)) return s;
    if (int s = amg32.set_smoothing(degree, prolongation_damping)) return s;
    k64.drop_graph();
    k32.drop_graph();
    return 0;
  }

  int init(int n);
  // A: const double* (mixed = false) or const float* (mixed = true); b and x
  // FP64 device vectors of g.nn; x is overwritten. refinements may be null.
  int solve(const ScalarGraph& g, bool mixed, bool amg, bool graphs, const void* A, const double* b, double* x,
            double rtol, int maxit, int* iters, double* res, int* refinements, cudaStream_t st, const char* what);
  // Graph form of solve(): the same steps with every host decision moved to
  // the device (refresh IF, Krylov WHILE loops, the BiCGStab fallback IF, the
  // refinement WHILE loop), captured into g after d on the stream st. The
  // preconditioner must have been set up by an earlier solve(). After the
  // graph ran, graph_result() reads the outcome from the pinned mirrors;
  // *recapture is set when the solve switched to BiCGStab for good.
  int emit(GraphBuild& gb, cudaGraph_t g, Deps& d, const ScalarGraph& gr, bool mixed, bool amg, const void* A,
           const double* b, double* x, double rtol, int maxit, cudaStream_t st);
  int graph_result(bool mixed, int* iters, double* res, int* refinements, bool* recapture, const char* what);
  // before each launch of a graph holding emit()'s nodes: the device refresh
  // counter takes the host's solve count (which a caller may have reset)
  int graph_prepare(cudaStream_t st);
  void release();
  ~ScalarSolve() {
    release();
    release_segments();
  }
};

}  // namespace oa
