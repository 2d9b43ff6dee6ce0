// Internal structures of the B200 CVFEM engine (not part of the C-ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/openaccel_b200.h"

namespace oa {

// Device-resident mesh: connectivity, node -> incident-element table,
// reduced-stencil CSR graph, wall faces and static FP64 geometry.
// POD view of the device arrays, passed to kernels by value.
//   hex8: n2e is [nn][lpr]: element * 8 + corner of the node's incident
//         elements (or -1); on block meshes entry c is the element where the
//         node is corner c.
//   tet4: n2e[n2e_ptr[i] .. n2e_ptr[i+1]) lists 4*element + corner for every
//         element incident to node i, by ascending element; n2f likewise
//         lists 4*face + k for every boundary face whose side node k is i.
struct MeshView {
  int nn = 0, ne = 0, nf = 0, nnz = 0;
  double* x = nullptr;         // [nn][3]
  int* conn = nullptr;         // [ne][8] (hex8) or [ne][4] (tet4)
  int* n2e = nullptr;
  int* n2e_ptr = nullptr;      // [nn+1] (tet4)
  int* n2f = nullptr;          // (tet4)
  int* n2f_ptr = nullptr;      // [nn+1] (tet4)
  int* face_elem = nullptr;    // [nf] (tet4)
  int* face_ord = nullptr;     // [nf] (tet4)
  int* face_bnd = nullptr;     // [nf] (tet4)
  int* row_ptr = nullptr;      // [nn+1]
  int* cols = nullptr;         // [nnz]
  int* diag = nullptr;         // [nn] offset of the diagonal within the row
  // hex8: per off-diagonal CSR entry, the row's corner-lane contributions that
  // land in it: bit 3c + k is lane c's edge neighbour k (edge_nbr order)
  uint32_t* slot_mask = nullptr;  // [nnz]
  // the same with 16 lanes per row (meshes that are not consistently
  // oriented blocks; bit 3 lane + neighbour)
  unsigned long long* slot_mask64 = nullptr;  // [nnz]
  // hex8 lanes per row: 8 (block mesh, lane = corner) or 16 (general)
  int lpr = 8;
  uint8_t* face_mask = nullptr;  // [ne] bit f: face f is a boundary face
  // [ne] bit f: face f is on a symmetry plane (a flow's boundary types; null
  // when it has none). The no-slip wall faces are face_mask & ~sym_mask.
  uint8_t* sym_mask = nullptr;
  double* vol = nullptr;       // [nn] dual nodal volume
  double* wscv = nullptr;      // [ne][8] SCV volume fractions (hex8)
  double* scs_area = nullptr;  // [ne][12][3] SCS area vectors, L -> R (hex8)
  int* wall_node = nullptr;    // [nn] 1 on wall nodes
};

struct DeviceMesh : MeshView {
  int topo = OA_TOPO_HEX8;
  int geom_err = 0;
  // mean element edge length (every element's 12 edges, summed in element
  // order on the host): the h of the continuity-residual scale rho U_ref h^2
  double h_mean = 0.0;
  // hex8 elements relabelled into a consistently oriented block: the cube
  // rotation applied to each (empty when none was needed)
  std::vector<uint8_t> h_rot;
  // host copies needed for set-up and parity dumps
  std::vector<int> h_row_ptr, h_cols, h_diag;
  std::vector<int> h_conn, h_face_elem, h_face_ord, h_face_bnd;
  const MeshView& view() const { return *this; }
};

struct Buffers {
  // matrices / vectors in the working precision
  void* A_mom = nullptr;   // [nnz][9]
  void* b_mom = nullptr;   // [nn][3]
  void* A_pc = nullptr;    // [nnz]
  double* b_pc = nullptr;  // [nn]
  double* x_mom = nullptr; // [nn][3]
  double* x_pc = nullptr;  // [nn]
};

struct Flow {
  DeviceMesh* mesh = nullptr;
  oa_flow_settings s{};
  cudaStream_t stream = nullptr;
  // fields (FP64)
  double *U = nullptr, *p = nullptr, *gradU = nullptr, *gradP = nullptr, *du = nullptr,
         *div = nullptr, *mDot = nullptr, *rho = nullptr, *mu = nullptr, *sideU = nullptr;
  // high-resolution advection (settings.hr): velocity blending factor and the
  // extrema it is limited by, [nn][3] each
  double *betaU = nullptr, *minU = nullptr, *maxU = nullptr;
  // SIMPLEC (settings.du_mode == 1): the consistent coefficient D~ [nn][3]
  double* duT = nullptr;
  // transient runs (oa_flow_advance_time): scheme (0 steady, 1 BDF1, 2 BDF2),
  // time steps taken, the order and coefficients of the current step, its
  // size and the previous one, velocity at the two previous time levels
  int time_scheme = 0, time_steps = 0, time_order = 0;
  double tk[3] = {0.0, 0.0, 0.0};
  double dt_step = 0.0, dt_prev = 0.0;
  double *Uold = nullptr, *Uoldold = nullptr;
  // launch shapes chosen by oa_flow_autotune (threads per block; multiples
  // of 32 up to the kernels' compiled 128): row kernels without shared
  // memory (gradients, divergence, blending), the element-owner mass-flow
  // kernel, the assembly row kernels (momentum, pressure correction)
  int bs_rows = 128, bs_elems = 128, bs_asm = 128;
  // k-omega transport assembled in the momentum launch (oa_flow_enable_turbulence):
  // k, omega, their nodal diffusivities and node source terms ([nn] FP64), the
  // two systems in the matrix precision, their relaxation factors
  bool turb = false;
  double *kf = nullptr, *wf = nullptr, *gkf = nullptr, *gwf = nullptr;
  double *sdk = nullptr, *srk = nullptr, *sdw = nullptr, *srw = nullptr;
  void *A_k = nullptr, *b_k = nullptr, *A_w = nullptr, *b_w = nullptr;
  // gradients of k and omega [nn][3] (oa_update_gradient 2 and 3)
  double *gradK = nullptr, *gradW = nullptr;
  // SST outer loop (oa_flow_sst_iterate): turbulent viscosity, F1 blending,
  // production and the previous-iteration k [nn]
  double *mut = nullptr, *F1 = nullptr, *Pk = nullptr, *k_prev = nullptr;
  double urf_k = 1.0, urf_w = 1.0;
  // [ne][12] Rhie-Chow mass flux of each SCS ip with the pressure-correction
  // equation's upwind density (its right-hand side), written by the mass-flow
  // kernel and summed per row by the pressure-correction kernel
  double* pc_flux = nullptr;
  // [ne][8][3] pressure-correction lhs coefficients per element corner (edge
  // neighbours in the row-slot order), matrix precision, staged the same way
  void* pc_coef = nullptr;
  // mixed form only: [ne][8] FP32 corner offsets from corner 0 (static) and
  // the [nn] FP32 (U, mu) copy packed before each momentum assembly
  float4* xloc32 = nullptr;
  float4* umu32 = nullptr;
  Buffers b;
  // Krylov workspace (allocated on first solve)
  std::vector<void*> work;
  double* red = nullptr;        // reduction partials
  double* red_host = nullptr;   // pinned
  int* err_dev = nullptr;       // device error flags
  uint8_t* ref_flag = nullptr;  // [nn] pressure-level rows (one per closed domain)
  // residual scales: U_ref = largest wall speed (1 when all walls rest),
  // mass-flux scale rho U_ref h^2, momentum-flux scale rho U_ref^2 h^2
  double u_ref = 1.0, mass_scale = 1.0, mom_scale = 1.0;
  // convergence record of the last momentum / pressure-correction solve
  oa_control_data cd_mom{}, cd_pc{};
  // boundary physical types (oa_flow_set_boundary_types): per boundary index,
  // the wall velocities given at creation; with symmetry planes, the element
  // face mask of the symmetry faces, the symmetry nodes and their assembled
  // symmetry area vectors [nsym][3], the nodes on a wall face [nn] (the
  // boundary rhs relaxation of transient runs), the gradient-correction switch
  std::vector<int> h_bnd_type;
  std::vector<double> h_bnd_velocity;
  uint8_t* sym_mask = nullptr;
  int nsym = 0;
  int* sym_nodes = nullptr;
  double* sym_area = nullptr;
  int* wall_face_node = nullptr;
  bool correct_grad = false;
  // the mesh view of this flow's kernels: the mesh's, with the symmetry face
  // mask, and in transient runs with symmetry planes the wall-face nodes as the
  // relaxed boundary rows
  MeshView view() const {
    MeshView v = mesh->view();
    v.sym_mask = nsym ? sym_mask : nullptr;
    if (nsym && time_order) v.wall_node = wall_face_node;
    return v;
  }
};

void set_error(const std::string& msg);
void count_launches(long long n);
long long launch_total();
int fail(int code, const std::string& msg);

#define OA_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return ::oa::fail(OA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

}  // namespace oa

struct oa_mesh {
  oa::DeviceMesh m;
  cudaStream_t st = nullptr;
};

namespace oa {

// tet4 mesh set-up (oa_diffusion.cu): graph, incidence lists, dual volumes.
int create_tet4_mesh(oa_mesh* M, const double* coords, int nn, const int* conn, int ne, const int* face_elem,
                     const int* face_ord, const int* face_bnd, int nf);

// kernels / launchers (oa_kernels.cu)
int launch_geometry(DeviceMesh& m, cudaStream_t st);
// flux_fresh: pc_flux already holds this state's fluxes (the mass-flow update
// ran last on the stream); otherwise a flux-only mass-flow pass runs first
int launch_pcorr(Flow& f, bool mixed, bool flux_fresh = false);
int launch_momentum(Flow& f, bool mixed);
int launch_init_mdot(Flow& f);
int launch_xloc(Flow& f);
// stage: also write the pressure-correction ip fluxes and corner coefficients
int launch_update_mdot(Flow& f, bool stage = false);
int launch_div(Flow& f);
int launch_gradient(Flow& f, int which);
int launch_axpy_du_gradp(Flow& f, double sign);
// velocity extrema and blending factor of the high-resolution scheme
int launch_blend_u(Flow& f);
// assembled symmetry area [nn][3] of every node (zero off the symmetry planes)
int launch_sym_area(Flow& f, double* area_nn);

}  // namespace oa
