/* openaccel_b200 — C-ABI of the B200 (sm_100a) CVFEM assembly and SIMPLE
 * pressure-correction engine.
 *
 * The entry points replace OpenAccel's element assembly, CSR scatter and
 * pressure-correction linear solve behind the reference's assembler /
 * linear-system API. Each declaration names the reference interface it stands
 * in for (paths relative to the reference project root). Plain pointers and
 * sizes only; every function returns an oa_status (0 = success) and leaves a
 * message for oa_last_error() on failure, mirroring errorMsg()
 * (src/basic/macros.cpp:21-24), which throws std::runtime_error.
 *
 * Threading: a handle is not re-entrant; each flow handle owns one CUDA stream
 * and all its work is ordered on it.
 */
#ifndef OPENACCEL_B200_H
#define OPENACCEL_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum oa_status {
  OA_OK = 0,
  OA_ERR_ARG = 1,         /* invalid argument or size */
  OA_ERR_MESH = 2,        /* unsupported or invalid mesh (orientation, topology) */
  OA_ERR_GEOMETRY = 3,    /* non-positive Jacobian / volume */
  OA_ERR_CUDA = 4,        /* CUDA runtime error */
  OA_ERR_SOLVER = 5,      /* Krylov breakdown, stagnation or non-finite residual */
  OA_ERR_NOT_READY = 6    /* call out of sequence */
} oa_status;

enum { OA_TOPO_HEX8 = 8, OA_TOPO_TET4 = 4 };
enum { OA_PREC_FP64 = 0, OA_PREC_MIXED = 1 };

typedef struct oa_mesh oa_mesh;
typedef struct oa_flow oa_flow;

/* Settings of the steady laminar segregated-flow solve. Field meanings follow
 * the reference controls (src/controls/controls.h:60-245) and the cavity example
 * (examples/cavity/input.i). */
typedef struct oa_flow_settings {
  double rho, mu;               /* density, dynamic viscosity */
  double urf_u, urf_p;          /* velocity / pressure relaxation factors */
  double dt;                    /* physical timescale (false transient) */
  double grad_urf;              /* gradient under-relaxation (nodeField.h:152) */
  double mdot_urf;              /* mass-flow relaxation (relaxMass_) */
  double wall_rhs_relax;        /* wall-node rhs relaxation (navierStokesAssembler.cpp:237) */
  int u_shifted, u_grad_shifted, p_shifted, p_grad_shifted; /* linear_linear interpolation */
  int ref_node;                 /* pressure-level node, -1 for none */
  int mom_maxit;
  double mom_rtol;
  int pc_maxit;
  double pc_rtol;
  int precision;                /* OA_PREC_FP64 or OA_PREC_MIXED */
  int pc_amg;                   /* 1: aggregation-AMG preconditioned GCR(2) pressure solve (BiCGStab
                                   if GCR stagnates or OA_KRYLOV=bicgstab), 0: Jacobi BiCGStab */
  int use_graphs;               /* 1: replay Krylov iteration chunks as CUDA graphs; 2: run each
                                   outer iteration of oa_simple_iterate after the first as one CUDA
                                   graph whose solver loops are device-side conditional nodes (no
                                   host round trip inside the iteration; recaptured when tuning,
                                   time step or solver fallback change what it holds) */
  int hr;                       /* advection: 0 upwind, 1 high resolution (advectionSchemeType::highResolution:
                                   blended deferred correction, nodeField::updateBlendingFactorField) */
  double beta_max;              /* upper limit of the blending factor (nodeField.h:150, default 1) */
  int du_mode;                  /* pressure-velocity coupling coefficient (computeDUCoefficients,
                                   navierStokesAssembler.cpp:84-232): 0 SIMPLE D = V/a_ii, 1 SIMPLEC (consistent_:
                                   D~ = V/(a_ii + sum of off-diagonals) on the pressure-correction lhs and in the
                                   velocity correction), 2 fractional step D = dt/rho */
} oa_flow_settings;

/* Convergence record of one linear solve: the ControlData that liblinsolve
 * hands to linearSystem::convergenceReport_ (src/equation/linearSystem.h:464-571,
 * fields read at :473-488). Component i is velocity component i for the
 * momentum system and [0] for the scalar pressure correction (the other
 * entries are 0). Residuals are RMS over the rows of the component:
 *   solver_initial_res[i] = RMS_i(b - A x0), x0 = 0 (defect form), i.e. RMS_i(b);
 *   solver_final_res[i]   = RMS_i of the solver's residual at exit (the FP64
 *                           residual b - A x of the last refinement pass in
 *                           the mixed pressure solve);
 *   scaled_initial_res[i] = solver_initial_res[i] / flux scale, with the
 *                           mass-flux scale rho U_ref h^2 (pressure correction:
 *                           this is the continuity residual) and the
 *                           momentum-flux scale rho U_ref^2 h^2 (momentum);
 *                           rho = settings.rho, U_ref = the largest wall speed
 *                           given to oa_flow_create (1 when every wall is at
 *                           rest), h = the mean element edge length.
 * The reference multiplies scaled_initial_res by its residual_scales
 * (1 / field scale, navierStokesEquation.cpp:230-238,
 * pressureCorrectionEquation.cpp:165-169) to form the control residual; the
 * scale normalisation inside liblinsolve is not in the reference checkout, so
 * the one above is this library's definition. */
typedef struct oa_control_data {
  int n_iterations;               /* Krylov iterations (GCR(2): V-cycles; BiCGStab: two per iteration) */
  int fallback;                   /* 1 when a stagnated GCR(2) solve was finished by BiCGStab */
  double solver_initial_res[3];
  double solver_final_res[3];
  double scaled_initial_res[3];
} oa_control_data;

typedef struct oa_iter_stats {
  int mom_iters, pc_iters, pc_refinements;
  double mom_res, pc_res;         /* relative residuals ||r|| / ||b|| at exit */
  /* continuity residual: RMS over nodes of the pressure-correction rhs (the
   * nodal mass imbalance) before the solve, divided by rho U_ref h^2 (see
   * oa_control_data); continuity_rms_raw is the RMS itself */
  double continuity_rms;
  /* device time of the iteration's phases in ms (CUDA events on the flow's
   * stream), the counterpart of the reference's Profiler push/pop around
   * assembly and solve (src/equation/linearSystem.h:452-454) */
  double ms_momentum_assembly, ms_momentum_solve, ms_pcorr_assembly, ms_pcorr_solve, ms_corrections;
  double continuity_rms_raw;
  oa_control_data mom, pc;        /* ControlData of the iteration's two solves */
} oa_iter_stats;

/* Last error message of the calling thread ("" when none). */
const char* oa_last_error(void);
/* Library version string. */
const char* oa_version(void);

/* Mesh set-up: replaces the STK mesh + mesh::updateDualNodalVolumeField_ /
 * updateExposedAreaVectorField_ (src/mesh/meshGeometry.cpp:1277-1527) and the
 * reduced-stencil CSR graph of nodeGraph::buildGraph_
 * (src/mesh/graph/nodeGraph.cpp:29-469). coords[nn][3], conn[ne][8] (Nalu hex8
 * ordering), boundary faces as (element, face ordinal, boundary index).
 * hex8: elements whose corner numbering starts at another corner or axis than
 * their neighbours' are relabelled by a proper cube rotation (the geometry and
 * Jacobian sign do not change) so that the mesh is a consistently oriented
 * block. A hex mesh that admits no such labelling (three or five elements
 * around an interior edge, as where blocks of a multi-block mesh meet) keeps
 * the caller's labelling and its row kernels take each node's incident
 * elements from a list (up to 16 per node; more is OA_ERR_MESH, as is a face
 * shared by three elements). Element fields ("mDot") are exchanged in the
 * caller's labelling. */
int oa_mesh_create(const double* coords, int nn, const int* conn, int ne, int topo,
                   const int* face_elem, const int* face_ord, const int* face_bnd, int nf,
                   oa_mesh** out);
void oa_mesh_destroy(oa_mesh* m);
/* CSR graph of the mesh (columns sorted ascending): nnz, then row_ptr[nn+1],
 * cols[nnz]. Mirrors the CRSNodeGraph consumed by Matrix::rowCols(). */
int oa_mesh_nnz(const oa_mesh* m, int* nnz);
int oa_mesh_graph(const oa_mesh* m, int* row_ptr, int* cols);
/* Dual nodal volumes (host copy), mesh::updateDualNodalVolumeField_. */
int oa_mesh_dual_volume(const oa_mesh* m, double* vol);

/* Flow state: replaces the fieldBroker/flowModel fields U, p, mDot, du, grad U,
 * grad p, div (src/realm/fieldBroker.cpp) for one domain whose boundaries are
 * no-slip walls (oa_flow_set_boundary_types may make some symmetry planes).
 * bnd_velocity[nbnd][3] are the wall velocities by boundary index. */
int oa_flow_create(oa_mesh* m, const oa_flow_settings* s, const double* bnd_velocity, int nbnd,
                   oa_flow** out);
void oa_flow_destroy(oa_flow* f);
/* Host <-> device copies of a named field: "U" [nn][3], "p" [nn], "gradU"
 * [nn][9], "gradP" [nn][3], "du" [nn][3], "div" [nn], "mDot" [ne][12],
 * "sideU" [nn][3], "rho" [nn], "mu" [nn]; with settings.hr also the velocity
 * blending factor "betaU" and its extrema fields "minU", "maxU" [nn][3]; with
 * SIMPLEC (du_mode 1) "duTilde" [nn][3].
 * n is the number of doubles. */
int oa_flow_set_field(oa_flow* f, const char* name, const double* host, long n);
int oa_flow_get_field(oa_flow* f, const char* name, double* host, long n);
/* Device pointer of a named field (for callers that keep data resident;
 * "mDot" of a relabelled mesh is stored in the relabelled ip order). */
int oa_flow_field_device_ptr(oa_flow* f, const char* name, double** dev);
/* Pressure-level rows: replaces settings.ref_node with a list, one row per
 * closed domain of a batched (disjoint-union) mesh. Mirrors
 * domain::pressureLevelNodeId / adjustMatrixForPressureReference
 * (src/assemble/flow/segregatedFlow/pressureCorrectionAssembler/pressureCorrectionAssembler.cpp:19-63)
 * applied per domain. count = 0 removes all reference rows. The connected
 * components of the stencil graph become segments of the pressure-correction
 * solve: with more than one, a solve converges only when each component's
 * ||r|| <= rtol ||b|| (its reported residual is the worst component's). */
int oa_flow_set_reference_nodes(oa_flow* f, const int* nodes, int count);

/* Boundary physical types by boundary index (types[nbnd], nbnd as given to
 * oa_flow_create): a no-slip wall (the default) or a symmetry plane
 * (boundaryPhysicalType::wall / ::symmetry, zone/boundary/boundary.h). A
 * symmetry face carries no mass flow and no gradient contribution
 * (nodeField.hpp:4764), and its momentum term is the full viscous stress of the
 * element's velocities (navierStokesAssemblerElemBoundaryConditions.cpp:2082-2375);
 * after each momentum assembly a symmetry node's rhs loses its component along
 * the assembled symmetry normal (navierStokesAssembler::applySymmetryConditions_,
 * navierStokesAssembler.cpp:387-471) and its diagonal block D gains 0.25 D n n^T
 * (assembleNormalRelaxation, :473-699). The symmetry boundary's row of
 * bnd_velocity is ignored: the node side velocity is set again from the wall
 * boundaries alone, in index order. In transient runs only wall-face nodes get
 * the boundary rhs relaxation (assembleBoundaryRelaxation_, :241-385).
 * correct_gradients = 1 is the solver's correctGradients_ expert switch: the
 * velocity and pressure gradients at symmetry nodes lose their normal part
 * (node{Scalar,Vector}Field::correctGradientField_). hex8 flows. Drops a
 * captured iteration graph. */
enum { OA_BTYPE_WALL = 0, OA_BTYPE_SYMMETRY = 1 };
int oa_flow_set_boundary_types(oa_flow* f, const int* types, int nbnd, int correct_gradients);

/* navierStokesEquation::initialize / postInitialize and
 * pressureCorrectionEquation::initialize
 * (src/equation/flow/navierStokes/navierStokesEquation.cpp:86-133,
 *  src/equation/flow/pressureCorrection/pressureCorrectionEquation.cpp:60-71):
 * velocity and pressure gradients, initial mass flow, divergence. */
int oa_flow_initialize(oa_flow* f);

/* Momentum assembly: navierStokesAssembler::assemble + computeDUCoefficients
 * (src/assemble/flow/segregatedFlow/navierStokesAssembler/navierStokesAssembler.cpp:84-239,
 *  ...ElemTerms.cpp:15-441, ...NodeTerms.cpp:16-149,
 *  ...ElemBoundaryConditions.cpp:2659-2981). The system stays on the device;
 * when A (BSR 3x3, [nnz][9]) / b ([nn][3]) are non-null FP64 host copies are
 * written (the Context getAMatrix()/getBVector() dump). */
int oa_assemble_momentum(oa_flow* f, double* A, double* b);
/* Pressure-correction assembly: pressureCorrectionAssembler::assemble +
 * adjustMatrixForPressureReference
 * (src/assemble/flow/segregatedFlow/pressureCorrectionAssembler/pressureCorrectionAssemblerElemTerms.cpp:17-616,
 *  pressureCorrectionAssembler.cpp:19-63). Optional FP64 host copies of A [nnz], b [nn]. */
int oa_assemble_pcorr(oa_flow* f, double* A, double* b);
/* flowModel::updateMassFlowRateInterior_ (src/model/flow/flowModel.cpp:5272-5687). */
int oa_update_mdot(oa_flow* f);
/* flowModel::updateMassDivergenceField_ (flowModel.cpp:13541-14948, interior). */
int oa_update_div(oa_flow* f);
/* nodeField::updateGradientField (src/field/nodeField/nodeField.hpp:3253-4948);
 * which = 0: pressure, 1: velocity, 2: k, 3: omega (fields "gradK",
 * "gradOmega" [nn][3] after oa_flow_enable_turbulence, else OA_ERR_NOT_READY;
 * the SST driver's updateTurbulent{KineticEnergy,EddyFrequency}GradientField,
 * segregatedShearStressTransportEquations.cpp:96-98, with the turbulence
 * fields' default linear_linear interpolation, controls.h:97-102). */
int oa_update_gradient(oa_flow* f, int which);
/* Linear solve of the last assembled system: linearSystem::solve()
 * (src/equation/linearSystem.h:416-462). sys = 0 momentum (x [nn][3]), 1
 * pressure correction (x [nn]); x may be NULL (result kept on the device).
 * iters counts Krylov iterations of the method in use (GCR(2): one
 * preconditioner application each; BiCGStab: two). */
int oa_solve(oa_flow* f, int sys, double rtol, int maxit, double* x, int* iters, double* res);
/* Transient runs: start a time step of size dt (simulation::runTransient's
 * preWork and time advance, src/simulation/simulation.cpp:222-312): the
 * velocity moves to the old time level (old to old-old), and the following
 * oa_simple_iterate calls (the step's coefficient iterations) assemble the
 * BDF1 or BDF2 momentum node terms
 * (src/assemble/flow/segregatedFlow/navierStokesAssembler/navierStokesAssemblerNodeTerms.cpp:151-427)
 * and the transient part of the mass divergence (src/model/flow/flowModel.cpp:13556-13700)
 * instead of the steady false transient; BDF2 uses variable-step
 * coefficients (src/basic/types.cpp:398-410) and BDF1 on its first step.
 * The density is constant in time (incompressible). Fields "Uold",
 * "Uoldold" become readable. */
enum { OA_TIME_BDF1 = 1, OA_TIME_BDF2 = 2 };
int oa_flow_advance_time(oa_flow* f, int scheme, double dt);
/* Autotuning of the flow's launch shapes and pressure-solve schedule (no
 * counterpart in the reference, which has no device). Coordinate descent over
 * the threads per block of the row kernels without shared memory (gradients,
 * divergence, blending factor), of the element-owner mass-flow kernel and of
 * the assembly row kernels (each 32, 64 or 128), the GCR(2) iterations per
 * device-resident chunk (2 or 4), the AMG numeric refresh interval (4, 8 or
 * 16 solves), the degree of the AMG's coarse-level Chebyshev smoother (3 or 4)
 * and its prolongation damping (0.74 or 0.85), each candidate timed over
 * `iters` SIMPLE outer iterations (CUDA
 * events on the flow's stream, after one untimed iteration) from the same
 * saved state; the flow's fields are restored afterwards and the next
 * pressure solve rebuilds the AMG numeric phase. Block sizes do not change
 * results; the solve schedule changes iterates within the solve tolerance. */
typedef struct oa_tuning {
  int block_rows, block_elements, block_assembly;  /* threads per block */
  int gcr_chunk, amg_refresh;
  double ms_per_iteration_before, ms_per_iteration_after;
  int amg_cheb_degree;            /* 2..6; 0 in oa_flow_set_tuning: keep the current one */
  double amg_prolong_damping;     /* (0, 1.5); 0 in oa_flow_set_tuning: keep the current one */
} oa_tuning;
int oa_flow_autotune(oa_flow* f, int iters, oa_tuning* out);
/* Apply a tuning found earlier (ms fields ignored). */
int oa_flow_set_tuning(oa_flow* f, const oa_tuning* t);
/* ControlData of the last solve of system sys (0 momentum, 1 pressure
 * correction) made by oa_solve or oa_simple_iterate: Context::getControlData()
 * as linearSystem::convergenceReport_ reads it (src/equation/linearSystem.h:473-488).
 * OA_ERR_NOT_READY before the first solve of that system. */
int oa_flow_last_control(oa_flow* f, int sys, oa_control_data* out);
/* Residual scales of the flow: U_ref, the mass-flux scale rho U_ref h^2 and the
 * momentum-flux scale rho U_ref^2 h^2 (see oa_control_data); any pointer may be NULL. */
int oa_flow_scales(oa_flow* f, double* u_ref, double* mass_scale, double* mom_scale);
/* n SIMPLE outer iterations: segregatedFlowEquations::solve
 * (src/equation/flow/segregatedFlowEquations.cpp:76-297). stats may be NULL. */
int oa_simple_iterate(oa_flow* f, int n, oa_iter_stats* stats);
/* Wait for the flow's stream. */
int oa_flow_sync(oa_flow* f);

/* Measurement hooks (no counterpart in the reference, which has no device):
 * the cudaStream_t all of the flow's work is ordered on (so callers can time
 * it with CUDA events), the number of kernels this library has launched so
 * far, and the mean device time of `reps` back-to-back launches of one
 * assembly kernel (which = 0 momentum, 1 pressure correction, 2 mass flow,
 * 3 velocity gradient) timed with CUDA events on the flow's stream. */
int oa_flow_stream(oa_flow* f, void** stream);
int oa_launch_count(long long* count);
int oa_time_kernel(oa_flow* f, int which, int reps, double* ms_per_launch);

/* Allocation-free pressure-correction solve. No counterpart in the reference:
 * it exists for callers that cannot allocate device memory when they solve,
 * such as a host application that reserves all device memory up front and
 * hands out slices itself, or a solver plug-in called from a framework that
 * forbids allocation on its hot path. Everything is a device pointer the
 * caller owns: the CSR graph (row_ptr[nn+1], cols, diag = offset of the
 * diagonal within each row), A (FP64 values), b and the solution x [nn].
 * BiCGStab with Jacobi preconditioning, FP64, to rtol relative to ||b||. Its
 * work vectors live in one file-scope device array sized for
 * OA_STATIC_SOLVE_MAX_ROWS rows (about 9.5 MB, held by every GPU that loads the
 * library until exit); larger systems are rejected with OA_ERR_ARG, and the
 * call allocates nothing. All calls on a device share that array, so calls
 * that overlap on the GPU race: the caller must serialise them. The first call
 * on a device resolves the array's device address (cudaGetSymbolAddress) and
 * caches it; make that first call before any stream capture. A breakdown, a
 * diverging iteration or a solve that ends above rtol returns OA_ERR_SOLVER
 * (oa_last_error names the status) with the last iterate in x. The call
 * synchronises `stream` before it returns. stream may be NULL (default
 * stream). */
#define OA_STATIC_SOLVE_MAX_ROWS 131072
int oa_pcorr_solve_static(int nn, const int* row_ptr, const int* cols, const int* diag, const double* A,
                          const double* b, double* x, double rtol, int maxit, int* iters, double* res,
                          void* stream);

/* ---- tet4 scalar diffusion (solid-domain energy equation) ----
 * Replaces phiAssembler<1> in diffusion mode as the thermal energy assembler
 * drives it in a solid domain: element terms
 * (src/assemble/phiAssembler/phiAssemblerElemTerms.hpp:11-413), fixed-value
 * walls (phiAssemblerElemBoundaryConditions.hpp:112-410), the solid source
 * (src/assemble/heatTransfer/thermalEnergy/thermalEnergyAssemblerNodeTerms.cpp:25-97,
 * generalised from one domain value to a value per node), relaxation
 * (phiAssembler.h:748-753,967-1006; thermalEnergyAssembler.h:39-43), and the
 * solve + clipped correction of thermalEnergyEquation::solve
 * (src/equation/heatTransfer/thermalEnergy/thermalEnergyEquation.cpp:190-247).
 * The mesh comes from oa_mesh_create with OA_TOPO_TET4 (conn[ne][4], face
 * ordinals 0..3 of the Nalu tet4 element, Tet4CVFEM.C:416-421). */
typedef struct oa_diffusion oa_diffusion;
enum { OA_BND_FIXED_VALUE = 0, OA_BND_ZERO_FLUX = 1 };

typedef struct oa_diffusion_settings {
  int shifted;            /* linear_linear interpolation of Gamma (controls.h:95 temperature default) */
  double urf;             /* diagonal relaxation (energy relaxation factor, controls.h:73) */
  double wall_rhs_relax;  /* wall-node rhs relaxation (thermalEnergyAssembler.h:42) */
  double lower_clip;      /* lower clip of the corrected field (thermalEnergyEquation.cpp:212-213) */
  int maxit;
  double rtol;
  int precision;          /* OA_PREC_FP64 or OA_PREC_MIXED */
  int amg;                /* 1: aggregation-AMG preconditioned BiCGStab, 0: Jacobi */
  int use_graphs;         /* 1: replay Krylov iteration chunks as CUDA graphs */
} oa_diffusion_settings;

/* bnd_kind[nbnd] (OA_BND_*) and bnd_value[nbnd] (fixed values) by boundary
 * index; node-side values are applied boundary by boundary in index order.
 * Set-up builds, on the host, the assembly's contribution list of every CSR
 * entry (4 bytes per element-corner-node triple, 64 bytes per element) and
 * keeps it on the device with the staging buffers of the element pass
 * (16 matrix values and 4 FP64 rhs values per element). */
int oa_diffusion_create(oa_mesh* m, const oa_diffusion_settings* s, const int* bnd_kind, const double* bnd_value,
                        int nbnd, oa_diffusion** out);
void oa_diffusion_destroy(oa_diffusion* d);
/* Node fields [nn]: "phi" (the transported scalar), "gamma" (diffusivity at
 * nodes, phiAssembler.h:218-224), "src" (volumetric source), "sidePhi". */
int oa_diffusion_set_field(oa_diffusion* d, const char* name, const double* host, long n);
int oa_diffusion_get_field(oa_diffusion* d, const char* name, double* host, long n);
int oa_diffusion_field_device_ptr(oa_diffusion* d, const char* name, double** dev);
/* Assembly into the handle's CSR system (defect form); optional FP64 host
 * copies of A [nnz] and b [nn]. */
int oa_diffusion_assemble(oa_diffusion* d, double* A, double* b);
/* Solve the last assembled system to rtol (linearSystem::solve(),
 * src/equation/linearSystem.h:416-462); x [nn] may be NULL. */
int oa_diffusion_solve(oa_diffusion* d, double rtol, int maxit, double* x, int* iters, double* res,
                       int* refinements);
/* One thermalEnergyEquation::solve step: assemble, solve to settings.rtol,
 * phi += x clipped below at settings.lower_clip. */
int oa_diffusion_step(oa_diffusion* d, int* iters, double* res, int* refinements);
/* Measurement hooks (no reference counterpart): the handle's cudaStream_t and
 * the mean device time of `reps` assembly launches. */
int oa_diffusion_stream(oa_diffusion* d, void** stream);
int oa_diffusion_time_assembly(oa_diffusion* d, int reps, double* ms_per_launch);

/* ---- k-omega SST node-level model updates ----
 * One fused node kernel replacing shearStressTransportModel::
 * updateTurbulentDynamicViscosity (src/model/turbulence/RANS/shearStressTransport/
 * shearStressTransportModel.cpp:597-678), updateFOneBlending (:95-174),
 * updateTurbulentProduction (:176-420; incompressible, fixed frame; at wall
 * nodes the production is the caller's wall-function value, or 0) and the
 * steady node terms of the k and omega SST assemblers
 * (src/assemble/turbulence/RANS/shearStressTransport/segregatedShearStressTransport/
 * turbulentKineticEnergy/turbulentKineticEnergySSTAssemblerNodeTerms.cpp:13-127,
 * turbulentEddyFrequency/turbulentEddyFrequencySSTAssemblerNodeTerms.cpp:13-218).
 * Defaults of the constants: shearStressTransportModel.h:21-37, RANSModel.h:20-22,
 * turbulenceModel.h:20. */
typedef struct oa_sst_constants {
  double sigma_k1, sigma_k2, sigma_w1, sigma_w2, beta1, beta2, gamma1, gamma2, a1, beta_star, prod_limit, cmu;
} oa_sst_constants;

/* Device pointers, [nn] unless noted. mut may alias mut_old (in-place
 * relaxation mut = urf * new + (1 - urf) * old); pk_wall may be NULL. */
typedef struct oa_sst_fields {
  const double *k, *omega, *k_prev, *rho, *mu, *ymin;
  const double *gradU;         /* [nn][9], row-major d u_i / d x_j */
  const double *gradK, *gradW; /* [nn][3] */
  const double *div, *vol, *mut_old, *pk_wall;
  const int* wall_node;        /* 1 on no-slip wall nodes */
  double *mut, *F1, *Pk;
  double *k_diag, *k_rhs;      /* node-term diagonal / rhs of the k equation */
  double *w_diag, *w_rhs;      /* same for omega */
} oa_sst_fields;

void oa_sst_default_constants(oa_sst_constants* c);
/* Launch on `stream` (NULL: default stream); asynchronous. */
int oa_sst_node_update(int nn, const oa_sst_constants* c, double dt, double mut_urf, const oa_sst_fields* f,
                       void* stream);
/* The SST driver's viscosity updates (segregatedShearStressTransportEquations
 * preSolve and the k / omega equations' diffusivity setup): mu_eff = mu + mu_t
 * (turbulenceModel::updateEffectiveDynamicViscosity,
 * src/model/turbulence/turbulenceModel.cpp:121-150) and the diffusivities
 * gamma_k = mu + mu_t (F1 sigma_k1 + (1 - F1) sigma_k2), gamma_w likewise with
 * sigma_w1 / sigma_w2 (turbulentKineticEnergySSTEquation.cpp:55-75,
 * turbulentEddyFrequencySSTEquation.cpp:55-75). mu is the laminar viscosity.
 * Device pointers [nn]; outputs may be a flow's "mu", "gammaK" and
 * "gammaOmega" fields (oa_flow_field_device_ptr), but not alias the inputs.
 * Launch on `stream` (NULL: default stream); asynchronous. */
int oa_sst_diffusivities(int nn, const oa_sst_constants* c, const double* mu, const double* mut, const double* F1,
                         double* mu_eff, double* gamma_k, double* gamma_w, void* stream);

/* Fused u/v/w/k/omega assembly. After this call every momentum assembly of the
 * flow (oa_assemble_momentum, oa_simple_iterate) assembles in the same launch
 * the k and omega transport systems of the SST equations' element terms
 * (phiAssembler<1>::assembleElemTermsInterior_,
 * src/assemble/phiAssembler/phiAssemblerElemTerms.hpp:11-413: upwind advection
 * with the flow's mass flows, diffusion with the nodal diffusivities
 * "gammaK" / "gammaOmega" interpolated to the ips on the velocity's shape
 * functions and gradient operator), reusing the momentum kernel's ip geometry.
 * Walls are zero-gradient for both fields
 * (turbulent*SSTAssemblerElemBoundaryConditions.cpp), so they add no element
 * terms. The node terms are the flow fields "srcDiagK" / "srcRhsK" /
 * "srcDiagOmega" / "srcRhsOmega" (for instance the k_diag / k_rhs / w_diag /
 * w_rhs outputs of oa_sst_node_update written to their device pointers); the
 * diagonal is then relaxed by 1/urf (phiAssembler.h:967-1006). k and omega are
 * the fields "k" and "omega", their gradients "gradK" / "gradOmega" [nn][3]
 * (oa_update_gradient 2 / 3, the SST node update's gradK / gradW inputs).
 * Creates these fields (zero); steady upwind SIMPLE
 * flows only (no high resolution, SIMPLEC, fractional step or time stepping:
 * OA_ERR_ARG). */
int oa_flow_enable_turbulence(oa_flow* f, double urf_k, double urf_omega);
/* Host copies of the k and omega systems of the last momentum assembly (same
 * CSR layout as the pressure correction); any pointer may be NULL.
 * OA_ERR_NOT_READY before oa_flow_enable_turbulence. */
int oa_flow_turbulence_systems(oa_flow* f, double* A_k, double* b_k, double* A_omega, double* b_omega);
/* Solve the k and omega systems of the last fused assembly to rtol (BiCGStab
 * with Jacobi; FP32 inner iterations under FP64 refinement in the mixed form)
 * and correct the fields as turbulentKineticEnergySSTEquation::solve /
 * turbulentEddyFrequencySSTEquation::solve do (correctField_ with relaxation 1
 * and the lower clip SMALL, src/equation/equation.h:204-286). Iteration counts
 * may be NULL. OA_ERR_NOT_READY before oa_flow_enable_turbulence. */
int oa_flow_solve_turbulence(oa_flow* f, double rtol, int maxit, int* iters_k, int* iters_omega);
/* n outer iterations of the flow with the k-omega SST equations
 * (segregatedFlowEquations::solve followed by
 * segregatedShearStressTransportEquations::preSolve / solve,
 * segregatedShearStressTransportEquations.cpp:63-99), all on the device. Each
 * iteration: k.prevIter = k; one SIMPLE outer iteration whose momentum launch
 * also assembles the k and omega systems (oa_simple_iterate; stats[it] when
 * stats is not NULL); the k and omega solves to rtol with the clipped
 * correction (oa_flow_solve_turbulence); their gradients (oa_update_gradient 2
 * and 3); the SST node update (oa_sst_node_update with dt = settings.dt, the
 * flow's k, omega, gradients, U gradient, divergence, density and dual volumes,
 * the caller's laminar viscosity mu_lam, wall distance ymin and wall flags,
 * mu_t relaxed by mut_urf against its previous value, node terms into the
 * flow's source fields); then mu_eff into the flow's "mu" and the diffusivities
 * into "gammaK" / "gammaOmega" (oa_sst_diffusivities). The flow owns mu_t, F1
 * and P_k (fields "mut", "F1", "Pk" [nn], zero before the first call). The k
 * and omega systems of an iteration are assembled from the node terms of the
 * previous update, on the iteration's starting mass flows (the reference
 * assembles them after the pressure correction). Wall functions are not
 * modelled: wall production comes from the node kernel's wall treatment.
 * ymin, wall_node, mu_lam: device pointers [nn]. OA_ERR_NOT_READY before
 * oa_flow_enable_turbulence. */
int oa_flow_sst_iterate(oa_flow* f, int n, const oa_sst_constants* c, const double* ymin, const int* wall_node,
                        const double* mu_lam, double mut_urf, double rtol, int maxit, oa_iter_stats* stats);

#ifdef __cplusplus
}
#endif
#endif
