/* Oracle (test infrastructure only): C interface of the CPU FP64 restatement
 * of OpenAccel's CVFEM assembly and SIMPLE pressure-correction path.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library, and only as the checker. The shipped GPU path never calls it.
 *
 * Every function restates a reference routine; the citing comment sits beside
 * the implementation in oracle.cpp. Parity status: the reference cannot be
 * built here (Trilinos/STK, yaml-cpp, MPI, gfortran and the liblinsolve
 * submodule are absent) and ships no golden vectors, so this restatement is
 * pinned by analytic known-answer tests (tests/test_oracle_kat.py) and by the
 * committed fixtures it generates; parity against the reference binary itself
 * is unpinned.
 */
#ifndef OPENACCEL_ORACLE_H
#define OPENACCEL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Settings of the laminar, steady, incompressible segregated-flow case; the
 * defaults in the Python mirror follow controls.h and examples/cavity/input.i. */
typedef struct orc_settings {
  double rho;          /* density */
  double mu;           /* dynamic viscosity */
  double urf_u;        /* velocity relaxation factor */
  double urf_p;        /* pressure relaxation factor */
  double dt;           /* physical timescale (false transient) */
  double grad_urf;     /* gradient under-relaxation (nodeField.h:152) */
  double mdot_urf;     /* mass-flow relaxation (relaxMass_) */
  double wall_rhs_relax; /* boundary rhs relaxation (navierStokesAssembler.cpp:237) */
  int u_shifted;       /* velocity interpolation linear_linear */
  int u_grad_shifted;  /* velocity gradient interpolation linear_linear */
  int p_shifted;       /* pressure interpolation linear_linear */
  int p_grad_shifted;  /* pressure gradient interpolation linear_linear */
  int ref_node;        /* pressure-level node (row fixed), -1 for none */
  int mom_maxit;
  double mom_rtol;
  int pc_maxit;
  double pc_rtol;
  int hr;              /* advection scheme: 0 upwind, 1 high resolution (Barth-Jespersen blended deferred correction) */
  double beta_max;     /* upper limit of the blending factor (nodeField.h:150) */
  int du_mode;         /* pressure-velocity coupling: 0 SIMPLE, 1 SIMPLEC (consistent_), 2 fractional step */
} orc_settings;

typedef struct orc_iter_stats {
  int mom_iters[1];
  double mom_res;
  int pc_iters;
  double pc_res;
  double continuity_rms; /* RMS of the PC rhs before the solve / (rho U_ref h^2) */
  double continuity_raw; /* the RMS itself */
} orc_iter_stats;

/* ---- stateless geometry kernels (per element) ---- */
void orc_hex8_scs_areav(const double* x /*[8][3]*/, double* areav /*[12][3]*/);
int orc_hex8_scv_volumes(const double* x, double* vol /*[8]*/);
int orc_hex8_grad_op(const double* x, double* gradop /*[12][8][3]*/, int shifted);
void orc_hex8_shape(double* shape /*[12][8]*/, int shifted);

/* ---- case object ---- */
void* orc_case_create(int nn, int ne, const double* x, const int* conn, int nf,
                      const int* face_elem, const int* face_ord, const int* face_bnd,
                      int nbnd, const double* bnd_velocity, const orc_settings* s);
void orc_case_destroy(void* h);
/* pressure-level rows (replaces settings.ref_node; one per closed domain) */
void orc_set_ref_nodes(void* h, const int* nodes, int n);
/* boundary physical types by boundary index (types[nbnd]): no-slip wall or
 * symmetry plane (boundaryPhysicalType::wall / ::symmetry). A symmetry
 * boundary's velocity row is ignored; the node side velocity is set again
 * from the wall boundaries alone, in index order. correct_gradients: the
 * solver's correctGradients_ expert switch (gradients at symmetry nodes lose
 * their normal part). Returns nonzero on a bad type or count. */
enum { ORC_BTYPE_WALL = 0, ORC_BTYPE_SYMMETRY = 1 };
int orc_set_boundary_types(void* h, const int* types, int nbnd, int correct_gradients);
/* Pointer to a named field of the case (see oracle.cpp for the list); *len
 * receives the number of doubles. */
double* orc_case_field(void* h, const char* name, long* len);
int orc_case_nnz(void* h);
/* continuity-residual scale rho U_ref h^2: rho = settings.rho, U_ref = largest
 * wall speed (1 when every wall is at rest), h = mean element edge length */
double orc_case_mass_scale(void* h);
void orc_case_graph(void* h, int* row_ptr /*nn+1*/, int* cols /*nnz*/);

/* initialisation: mDot from U, gradients, divergence */
void orc_initialize(void* h);
/* assembled momentum system (BSR 3x3, row-major blocks) incl. node terms,
 * interior, no-slip walls, symmetry planes (face terms, rhs projection and
 * normal relaxation), relaxation; also updates du */
void orc_assemble_momentum(void* h, double* A, double* b);
/* pressure-correction system incl. reference-pressure row */
void orc_assemble_pcorr(void* h, double* A, double* b);
/* k / omega transport system (phiAssemblerElemTerms.hpp:11-413, upwind,
 * zero-gradient walls) with per-node source terms and relaxation 1/urf. */
void orc_assemble_scalar_transport(void* h, const double* phi, const double* gam, const double* sdiag,
                                   const double* srhs, double urf, double* A, double* b);
void orc_update_mdot(void* h);
void orc_update_div(void* h);
void orc_update_grad_p(void* h);
void orc_update_grad_u(void* h);
/* high-resolution velocity blending factor (min/max fields, limiter,
 * relaxation) from the current U and grad U: field "betaU" */
void orc_update_blending_u(void* h);
/* BiCGStab with (block-)Jacobi preconditioning; returns iterations, res = final
 * relative residual. bs = 1 or 3. */
int orc_bicgstab(void* h, int bs, const double* A, const double* b, double* x,
                 double rtol, int maxit, double* res);
/* the oracle's applyCoeff_ restatement on the case's graph: adds an element's
 * lhs [(n*bs)^2] and rhs [n*bs] (node-major, assembler.h layout) into A (BSR,
 * bs = 1 or 3) and b; columns missing from a row go to the diagonal block */
void orc_apply_coeff(void* h, int bs, double* A, double* b, const int* nodes, int n, const double* rhs,
                     const double* lhs);
/* one SIMPLE outer iteration (segregatedFlowEquations::solve) */
void orc_simple_iteration(void* h, orc_iter_stats* st);
/* start a time step (simulation::runTransient preWork): the velocity moves to
 * the old level (old to old-old), the step is dt, scheme 1 = BDF1, 2 = BDF2
 * (BDF1 on the first step); later iterations use the transient node terms */
void orc_advance_time(void* h, int scheme, double dt);
/* linear solvers of orc_simple_iteration: 0 = Jacobi-preconditioned BiCGStab
 * (default, the parity reference), 1 = the reference cavity example's
 * configuration (examples/cavity/input.i:61-77): momentum FGMRES(30) and
 * pressure correction GMRES(50), both right-preconditioned by block-Jacobi
 * ILU(0) with one block of contiguous rows per thread */
void orc_set_solver(void* h, int kind);
/* restarted GMRES with block-Jacobi ILU(0) on the case's graph (bs 1 or 3) */
int orc_gmres_ilu(void* h, int bs, const double* A, const double* b, double* x, double rtol, int maxit,
                  int restart, double* res);
/* thread count used by the element loops and SpMV (1 = serial) */
void orc_set_threads(int n);
int orc_get_threads(void);

/* ---- tet4 scalar diffusion (diffusion.cpp) ---- */
enum { ORC_BND_FIXED_VALUE = 0, ORC_BND_ZERO_FLUX = 1 };

typedef struct orc_diff_settings {
  int shifted;           /* linear_linear interpolation of Gamma (temperature default) */
  double urf;            /* diagonal relaxation (energy relaxation factor) */
  double wall_rhs_relax; /* wall-node rhs relaxation (thermalEnergyAssembler.h:42) */
  double lower_clip;     /* lower clip of the corrected field */
  int maxit;
  double rtol;
} orc_diff_settings;

void orc_tet4_scs_areav(const double* x /*[4][3]*/, double* areav /*[6][3]*/);
int orc_tet4_scv_volumes(const double* x, double* vol /*[4]*/);
int orc_tet4_grad_op(const double* x, double* gradop /*[4][3]*/);
void orc_tet4_shape(double* shape /*[6][4]*/, int shifted);
void orc_tri3_face_areav(const double* p /*[3][3]*/, double* areav /*[3][3]*/);

/* bnd_kind[nbnd] (ORC_BND_*), bnd_value[nbnd] (fixed values) */
void* orc_diff_create(int nn, int ne, const double* x, const int* conn, int nf, const int* face_elem,
                      const int* face_ord, const int* face_bnd, int nbnd, const int* bnd_kind,
                      const double* bnd_value, const orc_diff_settings* s);
void orc_diff_destroy(void* h);
/* fields: phi, gamma, src (per node), sidePhi, vol, wallNode, faceArea, x */
double* orc_diff_field(void* h, const char* name, long* len);
int orc_diff_nnz(void* h);
void orc_diff_graph(void* h, int* row_ptr, int* cols);
void orc_diff_assemble(void* h, double* A, double* b);
int orc_diff_cg(void* h, const double* A, const double* b, double* x, double rtol, int maxit, double* res);
int orc_diff_bicgstab(void* h, const double* A, const double* b, double* x, double rtol, int maxit,
                      double* res);
void orc_diff_spmv(void* h, const double* A, const double* x, double* y);
/* one thermalEnergyEquation::solve step: assemble, BiCGStab, correct; returns iterations */
int orc_diff_step(void* h, double* res);

/* ---- k-omega SST node-level updates (sst.cpp) ---- */
typedef struct orc_sst_constants {
  double sigma_k1, sigma_k2, sigma_w1, sigma_w2, beta1, beta2, gamma1, gamma2, a1, beta_star, prod_limit, cmu;
} orc_sst_constants;

typedef struct orc_sst_in {
  const double *k, *omega, *k_prev, *rho, *mu, *ymin, *gradU /*[nn][9]*/, *gradK /*[nn][3]*/, *gradW /*[nn][3]*/,
      *div, *vol, *mut_old, *pk_wall;
  const int* wall_node;
} orc_sst_in;

typedef struct orc_sst_out {
  double *mut, *F1, *Pk, *k_diag, *k_rhs, *w_diag, *w_rhs;
} orc_sst_out;

void orc_sst_default_constants(orc_sst_constants* c);
/* mu_t, F1, P_k and the steady k / omega node-term diagonal and rhs per node */
void orc_sst_nodes(int nn, const orc_sst_constants* c, double dt, double mut_urf, const orc_sst_in* in,
                   orc_sst_out* out);
/* mu_eff = mu + mu_t and the F1-blended k / omega diffusivities per node */
void orc_sst_diffusivities(int nn, const orc_sst_constants* c, const double* mu, const double* mut, const double* F1,
                           double* mu_eff, double* gamma_k, double* gamma_w);

#ifdef __cplusplus
}
#endif
#endif
