// Building one CUDA graph for a whole SIMPLE outer iteration (internal).
//
// The host-side convergence checks of the iterative solves become device-side
// conditional nodes: a WHILE node per Krylov loop, whose body is one chunk of
// iterations followed by a one-thread kernel that sets the loop's condition
// from the solver's device "done" flag, and IF nodes for the refresh of the
// AMG numeric phase and for the BiCGStab fallback of a stagnated GCR(2)
// solve. Stream work between the conditional nodes is captured straight into
// the graph (or into a body graph) with cudaStreamBeginCaptureToGraph, so the
// launch helpers of the eager path are reused unchanged.
//
// Every loop is bounded twice: by the solver's own iteration limit (its done
// flag) and by a pass cap counted on the device, so a WHILE node ends even if
// a solver never raised its flag.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/openaccel_b200.h"

namespace oa {

int fail(int code, const std::string& msg);
void count_launches(long long n);
long long launch_total();

using Deps = std::vector<cudaGraphNode_t>;

// Device counters of the conditional bodies of one graph: for each body, the
// passes of its current entry (WHILE bodies, against the cap) and the
// executions since the graph was launched (for the launch count).
constexpr int MAX_BODIES = 24;
struct BodyCounters {
  int cur[MAX_BODIES];
  int total[MAX_BODIES];
};

struct GraphBuild {
  cudaStream_t st = nullptr;
  BodyCounters* ctr = nullptr;  // device
  int nbodies = 0;
  long long top_launches = 0;                   // kernels outside every body
  long long body_launches[MAX_BODIES] = {};     // kernels per execution of a body

  // a new body id (its counters are reset when the graph starts)
  int new_body() {
    if (nbodies >= MAX_BODIES) return -1;
    return nbodies++;
  }

  // Capture f()'s stream work into g after the nodes d; d becomes the leaves
  // of what was captured (unchanged when f launched nothing). body: the id of
  // the conditional body g is (-1: the top-level graph), for the launch count.
  template <class F>
  int seg(cudaGraph_t g, Deps& d, int body, F&& f) {
    cudaError_t e = cudaStreamBeginCaptureToGraph(st, g, d.empty() ? nullptr : d.data(), nullptr, d.size(),
                                                  cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return fail(OA_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    const long long l0 = launch_total();
    const int s = f();
    const long long dl = launch_total() - l0;
    count_launches(-dl);  // captured, not launched
    if (body < 0) top_launches += dl;
    else body_launches[body] += dl;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const cudaGraphNode_t* leaves = nullptr;
    size_t nleaves = 0;
    const cudaError_t ei = cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &leaves, &nleaves);
    Deps next;
    if (ei == cudaSuccess && leaves) next.assign(leaves, leaves + nleaves);
    cudaGraph_t out = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(st, &out);
    if (s) return s;
    if (ei != cudaSuccess) return fail(OA_ERR_CUDA, std::string("graph capture info: ") + cudaGetErrorString(ei));
    if (ee != cudaSuccess) return fail(OA_ERR_CUDA, std::string("graph capture end: ") + cudaGetErrorString(ee));
    d.swap(next);
    return 0;
  }

  // A conditional node after d (d becomes {node}); its body graphs, owned by
  // the node, are written to bodies[0 .. size).
  int cond(cudaGraph_t g, Deps& d, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type, unsigned size,
           cudaGraph_t* bodies) {
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = size;
    cudaGraphNode_t node = nullptr;
    const cudaError_t e = cudaGraphAddNode(&node, g, d.empty() ? nullptr : d.data(), d.size(), &p);
    if (e != cudaSuccess) return fail(OA_ERR_CUDA, std::string("conditional graph node: ") + cudaGetErrorString(e));
    for (unsigned k = 0; k < size; ++k) bodies[k] = p.conditional.phGraph_out[k];
    d.assign(1, node);
    return 0;
  }

  int handle(cudaGraph_t g, cudaGraphConditionalHandle* h) {
    const cudaError_t e = cudaGraphConditionalHandleCreate(h, g, 0, 0);
    if (e != cudaSuccess) return fail(OA_ERR_CUDA, std::string("conditional handle: ") + cudaGetErrorString(e));
    return 0;
  }

  // kernel launches of one graph execution, from the body execution counts
  long long launches(const BodyCounters& host) const {
    long long n = top_launches;
    for (int k = 0; k < nbodies; ++k) n += body_launches[k] * host.total[k];
    return n;
  }
};

// One-thread control kernels (oa_krylov.cu), launched on gb.st.
// Condition of an IF node: (*flag != 0) != negate.
int launch_set_if(GraphBuild& gb, cudaGraphConditionalHandle h, const int* flag, bool negate);
// Counts one execution of an IF body (its first node).
int launch_count_body(GraphBuild& gb, int body);
// Entry of a WHILE node over a Krylov solve: pass counter reset, condition =
// the solve is not done yet. branch_body (>= 0) counts an execution of the IF
// branch this entry sits in.
int launch_loop_enter(GraphBuild& gb, cudaGraphConditionalHandle h, const void* kscal, int body, int branch_body);
// End of a pass: condition = not done and fewer than cap passes.
int launch_loop_next(GraphBuild& gb, cudaGraphConditionalHandle h, const void* kscal, int body, int cap);
// Counters reset (a memset node at the start of the graph).
int launch_counters_reset(GraphBuild& gb);

}  // namespace oa
