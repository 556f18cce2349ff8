/*
 * pism_ssa_gpu.h — C-ABI of the B200 finite-difference SSA (SSAFD) solver.
 *
 * This is the boundary a PISM host binds to in place of SSAFD's PETSc path.
 * Every entry point takes plain pointers and sizes and returns an int status
 * (0 = success, see PISM_GPU_SSA_E*); nothing throws across this boundary.
 * The message of the last failure of a handle is pism_gpu_ssa_last_error().
 *
 * Field layout (all FP64 unless stated): a scalar field is Mx*My values indexed
 * [i][j] with j (the y index) contiguous, i.e. element i*My + j — the layout of a
 * PETSc DMDA local array without ghosts (src/base/util/IceGrid.cc:800-823).  A
 * vector field (velocity, boundary values, driving stress) interleaves (u, v)
 * per cell (2*Mx*My values, IceModelVec2V); a staggered field stores
 * (east face i+1/2, north face j+1/2) per cell (IceModelVec2Stag).  Neighbour
 * accesses wrap periodically at every domain edge, as the reference's DMDA does.
 *
 * Units are SI: m, m/s, Pa, Pa s m, J/kg.
 */
#ifndef PISM_SSA_GPU_H
#define PISM_SSA_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define PISM_GPU_SSA_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------- */
enum {
  PISM_GPU_SSA_OK = 0,
  PISM_GPU_SSA_EINVAL = 1,          /* bad argument (null pointer, size, enum)          */
  PISM_GPU_SSA_ECUDA = 2,           /* CUDA runtime error; context may be unusable      */
  PISM_GPU_SSA_ENOMEM = 3,          /* device allocation failed                         */
  PISM_GPU_SSA_EKSP = 4,            /* KSPFailure: Krylov solve failed (SSAFD.hh:115)   */
  PISM_GPU_SSA_EPICARD = 5,         /* PicardFailure (SSAFD.hh:120)                     */
  PISM_GPU_SSA_EZERODIAG = 6,       /* zero diagonal at a regular location (SSAFD.cc:766-776) */
  PISM_GPU_SSA_ENAN = 7,            /* non-finite value in a residual / inputs          */
  PISM_GPU_SSA_ESTATE = 8,          /* call order violated (e.g. solve before inputs)   */
  PISM_GPU_SSA_ETOOLARGE = 9        /* grid exceeds PISM_GPU_SSA_NOALLOC_MAX_CELLS      */
};

/* ---- enumerations -------------------------------------------------------- */
/* flow laws accepted by the SSA (src/base/rheology/flowlaw_factory.hh:31-37,
 * Goldsby-Kohlstedt excluded as in SSA.cc:107-109) */
enum {
  PISM_FLOW_LAW_ISOTHERMAL_GLEN = 0,
  PISM_FLOW_LAW_PB = 1,
  PISM_FLOW_LAW_GPBLD = 2,
  PISM_FLOW_LAW_ARR = 3,
  PISM_FLOW_LAW_ARRWARM = 4,
  PISM_FLOW_LAW_HOOKE = 5
};

/* grid periodicity (IceGrid.hh, Periodicity) */
enum { PISM_NOT_PERIODIC = 0, PISM_X_PERIODIC = 1, PISM_Y_PERIODIC = 2, PISM_XY_PERIODIC = 3 };

/* Krylov method (replaces PETSc KSPSolve, SSAFD.cc:1018) */
enum { PISM_KSP_BICGSTAB = 0, PISM_KSP_GMRES = 1 };

/* preconditioner (replaces PCBJACOBI/ILU(0) and PCASM/LU, SSAFD.cc:136-219):
 *   BLOCK_JACOBI  the inverse 2 x 2 diagonal block of each cell
 *   MULTIGRID     an FP32 aggregation-multigrid V(1,1) cycle
 *   LINE          line block Jacobi: the 2 x 2-block tridiagonal couplings of each grid line
 *                 of constant i (j - 1, j, j + 1; none across the line's ends) solved exactly
 * A KSP failure retries with MULTIGRID (BLOCK_JACOBI after a MULTIGRID failure). */
enum { PISM_PC_BLOCK_JACOBI = 0, PISM_PC_MULTIGRID = 1, PISM_PC_LINE = 2 };

/* arithmetic of the inner Krylov iterations */
enum { PISM_PRECISION_FP64 = 0, PISM_PRECISION_MIXED = 1 };

/* where the pointers handed to set_inputs / solve live */
enum { PISM_MEM_HOST = 0, PISM_MEM_DEVICE = 1 };

/* ---- grid -------------------------------------------------------------- */
typedef struct pism_gpu_grid {
  int Mx, My;            /* points in x (i) and y (j); both >= 3                  */
  double dx, dy;         /* spacing (IceGrid::dx(), dy())                          */
  int periodicity;       /* PISM_*_PERIODIC; only affects the one-sided edge
                            differences of compute_surf_grad_inward_ssa            */
  int Mz;                /* vertical levels of the enthalpy columns (0 = none)     */
  const double *z;       /* host array of Mz levels, z[0] = 0 (IceGrid::z())       */
} pism_gpu_grid;

/* ---- SSA configuration: the pism_config.cdl parameters the path reads ---- */
typedef struct pism_gpu_ssa_config {
  double ice_density, sea_water_density, standard_gravity, sea_level;
  double epsilon_ssa;                              /* nu*H regularisation            */
  double ssafd_relative_convergence;               /* Picard tolerance (-ssa_rtol)   */
  int    max_iterations_ssafd;                     /* -ssa_maxi                      */
  double ssafd_nuH_iter_failure_underrelaxation;
  double min_thickness_strength_extension_ssa;
  double constant_nu_strength_extension_ssa;
  double plastic_regularization;                   /* m/s                            */
  int    do_pseudo_plastic_till;
  double pseudo_plastic_q, pseudo_plastic_uthreshold, sliding_scale_factor_reduces_tauc;
  double beta_ice_free_bedrock;
  int    calving_front_stress_boundary_condition;  /* -cfbc                          */
  int    ssa_dirichlet_bc;
  int    sub_groundingline;
  int    nu_bedrock_set;
  double nu_bedrock;
  int    surface_gradient_eta;                     /* surface_gradient_method == eta */
  int    compute_surf_grad_inward_ssa;
  int    flow_law;                                 /* PISM_FLOW_LAW_*                */
  double ssa_Glen_exponent, ssa_enhancement_factor, ice_softness;
  double Schoof_regularizing_length, Schoof_regularizing_velocity;   /* m, m/s     */
  double Paterson_Budd_A_cold, Paterson_Budd_A_warm, Paterson_Budd_Q_cold, Paterson_Budd_Q_warm;
  double Paterson_Budd_critical_temperature, ideal_gas_constant;
  double gpbld_water_frac_coeff, gpbld_water_frac_observed_limit;
  double Hooke_A, Hooke_Q, Hooke_C, Hooke_k, Hooke_Tr;
  double beta_CC, ice_specific_heat_capacity, water_latent_heat_fusion, surface_pressure;
  double water_melting_point_temperature, enthalpy_converter_reference_temperature;
  int    do_fracture_density;
  double fracture_density_softening_lower_limit;
  int    brutal_sliding;
  double brutal_sliding_scale;
  /* linear solver: the -ssafd_ksp_* / -ssafd_pc_* options of the reference */
  int    ksp_type;                                 /* PISM_KSP_*                     */
  int    pc_type;                                  /* PISM_PC_*                      */
  double ksp_rtol;                                 /* -ssafd_ksp_rtol (PETSc 1e-5)   */
  int    ksp_max_it;                               /* PETSc default 10000            */
  int    gmres_restart;                            /* PETSc default 30               */
  int    precision;                                /* PISM_PRECISION_*               */
  double mixed_inner_rtol;                         /* inner FP32 solve tolerance     */
  double mg_omega;                                 /* multigrid smoother damping     */
  double mg_correction;                            /* coarse-correction scaling      */
  /* inexact Picard: KSP rtol of iteration k = clamp(ksp_rtol_factor * (last relative nu*H
     change), ksp_rtol, ksp_rtol_max); the accepted last iteration is always solved to ksp_rtol */
  int    ksp_rtol_adaptive;                        /* 0: every solve to ksp_rtol     */
  double ksp_rtol_max;
  double ksp_rtol_factor;
  /* launch mode of the Krylov iterations: 2 a graph-resident loop per solve (a CUDA graph
     with a conditional WHILE node), 1 captured graphs of a few iterations, 0 direct launches
     (kernel profilers that cannot look into conditional graphs need 0 or 1).
     3 (BiCGStab only, otherwise as 2): the whole Picard loop of a solve is one CUDA graph
     with nested conditional nodes, its decisions taken on the device, one launch and one
     read-back per solve; the same results as 2, bit for bit */
  int    graphs;
  int    verbosity;                                /* 0 silent .. 3 per-iteration    */
  /* resident blocks per SM that the coarse-level multigrid post-smoothing grid is sized for
     (1..4; 0 = 4, the other tile kernels' size): a launch-shape knob for the autotuner */
  int    mg_post_blocks_per_sm;
  /* lagged multigrid coarse levels (0 = rebuilt every Picard iteration, as PETSc sets its
     preconditioner up on every KSPSolve): the coarse Galerkin operators and the coarsest
     inverse are rebuilt on the first Picard iteration of a solve and then once the relative
     nu*H changes summed since the last build reach this value.  The fine level and the
     Krylov operator always use the current nu*H, so a lagged coarse level changes the
     iteration counts, not the tolerance the solve meets */
  double mg_rebuild_rtol;
  /* the multigrid's small levels in one thread-block cluster: 0 the levels of <= 4096
     cells, every CTA staging from L2 the rows its share of each step reads; 1 the same levels
     with each CTA holding a block of every level in its shared memory (operators staged by
     bulk asynchronous copies, halos read from the neighbouring CTAs' shared memory), where
     the blocks fit; 0 and 1 give the same results, bit for bit (a launch-shape knob).  2 as 0
     but from the first level of <= 16384 cells (the 101^2 level of an 801^2 grid joins the
     cluster instead of two tiled passes); its residual sums at that level are added in
     another order, so its results differ in the last bits */
  int    mg_small_kernel;
  /* mixed precision with multigrid, the FP32 operator apply that BiCGStab performs on each
     V-cycle's result: 0 a kernel of its own loading each tile with plain loads; 1 the same
     kernel with interior tiles staged by bulk asynchronous copies, the next tile in flight;
     2 fused into the V-cycle's fine-level pass (one kernel per V-cycle fewer, the halo of the
     smoothed iterate recomputed instead of read back; the default).  All give the same
     results, bit for bit; the whole 801^2 fast solve took 225.6 / 233.0 / 224.2 ms with
     0 / 1 / 2 on one B200: a launch-shape knob */
  int    mixed_apply_kernel;
} pism_gpu_ssa_config;

/* ---- input fields (SSA::init_impl, SSA.cc:134-184; SSAFD::update) -------- */
typedef struct pism_gpu_ssa_inputs {
  int where;                      /* PISM_MEM_HOST or PISM_MEM_DEVICE                  */
  const double *thickness;        /* land_ice_thickness                    (required) */
  const double *surface;          /* surface_altitude                      (required) */
  const double *bed;              /* bedrock_altitude                      (required) */
  const double *mask;             /* mask, doubles rounded by as_int()     (required) */
  const double *tauc;             /* tauc (yield stress)                   (required) */
  const double *bc_mask;          /* bc_mask; NULL = no Dirichlet locations          */
  const double *bc_values;        /* vel_ssa_bc, interleaved; NULL with bc_mask NULL */
  const double *melange;          /* melange back pressure fraction; NULL = 0        */
  const double *gl_mask;          /* gl_mask; required if sub_groundingline          */
  const double *enthalpy;         /* Mx*My*Mz, [i][j][k]; required unless the flow
                                     law is isothermal_glen or hardness is given     */
  const double *hardness_stag;    /* optional precomputed staggered hardness (2*Mx*My);
                                     replaces compute_hardav_staggered when non-NULL */
  const double *fracture_density; /* required if do_fracture_density                 */
} pism_gpu_ssa_inputs;

/* ---- per-solve statistics (the SSAFD stdout report, SSAFD.cc:994-1118) ---- */
typedef struct pism_gpu_ssa_stats {
  int    status;                   /* PISM_GPU_SSA_* of the solve                     */
  int    converged;                /* 1 if a Picard strategy met the tolerance        */
  int    strategy;                 /* 0 default, 1 under-relaxation, 2 regularisation */
  int    picard_iterations;        /* outer iterations of the accepted strategy       */
  int    ksp_iterations;           /* Krylov iterations, all strategies               */
  int    ksp_failures;             /* KSP failures that switched the solver           */
  int    refinement_steps;         /* FP64 refinement steps (mixed precision)         */
  double nuH_norm, nuH_norm_change;
  double final_linear_residual;    /* ||b - A x|| / ||b|| of the last linear solve    */
  double solve_ms;                 /* wall time of pism_gpu_ssa_solve                 */
  double kernel_ms;                /* device time (CUDA events) of the solve          */
  long long kernel_launches;       /* kernels launched by the solve                   */
  int    mg_rebuilds;              /* multigrid coarse-level builds (mg_rebuild_rtol)   */
} pism_gpu_ssa_stats;

/* ---- one member of an ensemble (pism_gpu_ssa_solve_batch) ---- */
typedef struct pism_gpu_ssa_member {
  pism_gpu_ssa_inputs inputs;     /* the member's fields on the handle's grid         */
  double ice_softness;            /* > 0: this member's isothermal Glen softness
                                     (Pa^-3 s^-1); <= 0: the configuration's          */
  double *velocity;               /* 2*Mx*My, in inputs.where memory: the initial guess
                                     on entry (unless a network gives it), the
                                     solution on return                               */
} pism_gpu_ssa_member;

typedef struct pism_gpu_ssa pism_gpu_ssa;   /* opaque handle: owns device scratch */

/* Fill *cfg with the pism_config.cdl defaults.  Replaces Config::get_* reads. */
int pism_gpu_ssa_config_defaults(pism_gpu_ssa_config *cfg);

/* Create a solver for one grid on CUDA device `device`.  Replaces the SSAFD
 * constructor + SSAFD::init_impl (SSAFD.cc:59-129, 221-258) and the factory
 * SSAFDFactory (SSAFD.cc:47-49, typedef SSAFactory SSA.hh:77). */
int pism_gpu_ssa_create(const pism_gpu_grid *grid, const pism_gpu_ssa_config *cfg,
                        int device, pism_gpu_ssa **out);

/* Destroy a handle and free its device memory. */
int pism_gpu_ssa_destroy(pism_gpu_ssa *h);

/* Last error message of the handle ("" if none); valid until the next call. */
const char *pism_gpu_ssa_last_error(const pism_gpu_ssa *h);

/* Run the handle's work on a caller-owned cudaStream_t (NULL = the handle's own). */
int pism_gpu_ssa_set_stream(pism_gpu_ssa *h, void *cuda_stream);

/* Replace the configuration (e.g. epsilon_ssa set after init, as ssa_testi.cc:99-100). */
int pism_gpu_ssa_set_config(pism_gpu_ssa *h, const pism_gpu_ssa_config *cfg);

/* Copy the input fields (borrowed for the duration of the call).  Replaces the
 * m_grid->variables() lookups of SSA::init_impl (SSA.cc:134-184), the
 * ShallowStressBalance::set_boundary_conditions call and the melange pointer of
 * SSAFD::update (SSAFD.cc:260-264). */
int pism_gpu_ssa_set_inputs(pism_gpu_ssa *h, const pism_gpu_ssa_inputs *in);

/* SSA::set_initial_guess (SSA.cc:361-363): velocity (2*Mx*My, host or device per
 * `where`). */
int pism_gpu_ssa_set_initial_guess(pism_gpu_ssa *h, const double *velocity, int where);

/* SSAFD::solve (SSAFD.cc:869-924) with the Picard strategy ladder, followed by
 * compute_basal_frictional_heating as in SSA::update (SSA.cc:188-196).  Writes the
 * velocity (2*Mx*My) to velocity_out (host or device per `where`; may be NULL)
 * and fills *stats (may be NULL).  Blocks until the solve is done. */
int pism_gpu_ssa_solve(pism_gpu_ssa *h, double *velocity_out, int where,
                       pism_gpu_ssa_stats *stats);

/* An ensemble of independent sheets on the handle's grid (no reference counterpart; PISM
 * runs ensemble members as separate model runs).  Member q: its inputs, its softness, the
 * learned initial guess when net != NULL (features at `stride`, see pism_unet_gpu.h) or
 * its velocity otherwise, then pism_gpu_ssa_solve; stats[q] (may be NULL) gets its
 * statistics.  Members run one after another on the handle's stream.  A member whose
 * solve fails (KSP, Picard, NaN, zero diagonal) is recorded in stats[q].status and the
 * batch goes on; the first such status is returned.  Argument and CUDA errors stop the
 * batch.  The configuration's softness is restored on return. */
int pism_gpu_ssa_solve_batch(pism_gpu_ssa *h, struct pism_gpu_unet *net, int stride, int n,
                             pism_gpu_ssa_member *members, pism_gpu_ssa_stats *stats);

/* Field getters (host or device destination per `where`). */
enum {
  PISM_FIELD_VELOCITY = 0,        /* 2N  m_velocity                                   */
  PISM_FIELD_TAUD = 1,            /* 2N  driving stress (SSA_taud, SSA.cc:402-432)    */
  PISM_FIELD_RHS = 2,             /* 2N  m_b (SSAFD::assemble_rhs)                    */
  PISM_FIELD_HARDNESS = 3,        /* 2N  staggered hardness                           */
  PISM_FIELD_NUH = 4,             /* 2N  nu*H (SSAFD_nuH diagnostic, SSAFD.cc:1790)   */
  PISM_FIELD_BETA = 5,            /* N   basal drag coefficient of the last assembly  */
  PISM_FIELD_BFRICT = 6           /* N   basal frictional heating                     */
};
int pism_gpu_ssa_get_field(pism_gpu_ssa *h, int field, double *out, int where);

/* The consumers of the SSA velocity in StressBalance::update with a full update
 * (PISMStressBalance.cc:79-116, fast == false), from the handle's current velocity (the last
 * solve's, or the initial guess), mask, thickness and enthalpy:
 *   u3, v3          ConstantInColumn::update (SSB_Modifier.cc:126-152): every level of the
 *                   3-D horizontal velocity is the column's SSA velocity
 *   strain_heating  StressBalance::compute_volumetric_strain_heating
 *                   (PISMStressBalance.cc:369-499), zero above kBelowHeight(H)
 *   w3              StressBalance::compute_vertical_velocity (PISMStressBalance.cc:192-287),
 *                   w(0) = -basal_melt_rate (Mx*My, m/s) or 0 when basal_melt_rate is NULL
 *                   (include_bmr_in_continuity false)
 * Each output is Mx*My*Mz doubles, [i][j][k] (IceModelVec3's column order); any may be NULL.
 * All pointers are host or device per `where`.  Needs a grid with 2 <= Mz <= 800 levels and, for
 * the strain heating under an enthalpy-dependent flow law, the inputs' enthalpy.  Blocks
 * until done. */
int pism_gpu_ssa_stress_balance_3d(pism_gpu_ssa *h, const double *basal_melt_rate, double *u3, double *v3,
                                   double *w3, double *strain_heating, int where);

/* Mass transport consuming the SSA velocity: IceModel::massContExplicitStep
 * (iMgeometry.cc:497-819) over dt seconds on the handle's velocity, mask, thickness and (with
 * ssa_dirichlet_bc) Dirichlet data, with the ConstantInColumn modifier (no diffusive flux) and
 * part_grid off: the upwinded SSA flux divergence (face velocities of cell_interface_fluxes,
 * iMgeometry.cc:309-410), the climatic mass balance (kg m-2 s-1) and, when
 * basal_melt_rate != NULL (include_bmr_in_continuity), the basal melt rate (m s-1) as sources
 * (neither on ice-free ocean nor at Dirichlet locations), the non-negativity rule; then
 * updateSurfaceElevationAndMask (iMgeometry.cc:56-68) on the new thickness with the
 * GeometryCalculator thresholds mask_icefree_thickness_standard and
 * mask_is_floating_thickness_standard (dry simulation off).  cell_area may be NULL (dx dy).
 * Outputs (Mx*My each; only thickness_out is required): the new thickness, mask (as
 * doubles) and surface, and the flux divergence (m s-1); totals (host, 8 doubles, may be
 * NULL) gets the step's grounded basal, non-negativity, sub-shelf, surface, SIA and SSA
 * divergence, Href-to-H and H-to-Href fluxes in kg (iMgeometry.cc:778-787 order).  The
 * handle's own fields are not changed: pass the new ones to pism_gpu_ssa_set_inputs for
 * the next solve.  Arrays are host or device per `where`.  Blocks until done. */
int pism_gpu_ssa_mass_continuity_step(pism_gpu_ssa *h, double dt, const double *climatic_mass_balance,
                                      const double *basal_melt_rate, const double *cell_area,
                                      double icefree_thickness, double is_floating_thickness, double *thickness_out,
                                      double *mask_out, double *surface_out, double *flux_divergence,
                                      double *totals, int where);

/* The strain rates and 2-D stresses of the handle's velocity:
 *   edot      ShallowStressBalance::compute_2D_principal_strain_rates
 *             (ShallowStressBalance.cc:224-305): the eigenvalues (max, min) of the vertically
 *             integrated horizontal strain rate tensor (1/s), Mx*My*2, [i][j][2]
 *   stresses  ShallowStressBalance::compute_2D_stresses (:308-386): nu (u_x, v_y,
 *             (u_y + v_x) / 2) with nu the effective viscosity of the constant hardness
 *             ice_softness^(-1/ssa_Glen_exponent) (Pa), Mx*My*3, [i][j][3]
 * Differences are one-sided next to ice-free cells; both are zero on ice-free cells.  mask
 * (Mx*My doubles, PISM's mask values) may be NULL for the handle's mask.  Either output may
 * be NULL.  Arrays are host or device per `where`.  Blocks until done. */
int pism_gpu_ssa_strain_rates(pism_gpu_ssa *h, const double *mask, double *edot, double *stresses, int where);

/* EigenCalving::update (PISMEigenCalving.cc:77-235) over dt seconds with the constant K
 * (eigen_calving_K, m s) on the handle's velocity: at each ice-free ocean cell next to
 * floating ice the calving rate K e1 e2 H_average / dx (e1, e2 the principal strain rates
 * averaged over the floating, non-margin cells two cells away) lowers Href; where Href goes
 * negative the rest is shared among the floating neighbours, which are cut (thickness 0,
 * ice-free ocean, Href = max(H - loss, 0)); then remove_narrow_tongues (:420-493) in the
 * reference's (i, j) order.  mask (as doubles), Href and thickness (Mx*My each) are read and
 * overwritten, host or device per `where`.  The grid is taken as one process's: a strain
 * rate two cells across the grid's edge reads 0 (the reference's never-refreshed ghosts).
 * Blocks until done. */
int pism_gpu_ssa_eigen_calving(pism_gpu_ssa *h, double dt, double K, double *mask, double *Href, double *thickness,
                               int where);

/* EigenCalving::max_timestep (PISMEigenCalving.cc:249-341) on the handle's velocity and this
 * mask: result (host, 4 doubles) = {the time step allowed (s), the maximum horizontal
 * calving rate (m/s), their mean, the number of cells where the calving law applies}.  The
 * caller applies it only with cfl_eigen_calving.  mask is host or device per `where`. */
int pism_gpu_ssa_eigen_calving_max_timestep(pism_gpu_ssa *h, double K, const double *mask, double *result,
                                            int where);

/* ---- SSAFEM: the Q1 finite-element SSA (SSAFEM.cc:151-840) on the same handle ----------- */

/* The nonlinear and linear solver settings of SSAFEM::solve.  The reference hands F(u) = 0
 * to PETSc's SNES (Newton with a line search); here Newton steps with a backtracking line
 * search on ||F||, each linear solve by conjugate gradients preconditioned by the inverse
 * 2 x 2 diagonal blocks (the regression tests' -ksp_type cg). */
typedef struct pism_gpu_ssafem_options {
  double snes_rtol;              /* converged when ||F|| <= snes_rtol ||F(u0)|| (PETSc 1e-8)    */
  double snes_stol;              /* ... or when a step is below snes_stol ||u|| (PETSc 1e-8)    */
  int snes_max_it;               /* Newton steps (200, SSAFEM.cc:91-95)                        */
  double ksp_rtol;               /* linear solve: ||r|| <= ksp_rtol ||F|| (PETSc 1e-5)          */
  int ksp_max_it;                /* CG iterations per Newton step (10000)                      */
  double dirichlet_scale;        /* -ssa_fe_dirichlet_scale (1e9, SSAFEM.cc:128-131)           */
  double icefree_thickness;      /* mask_icefree_thickness_standard (GeometryCalculator)       */
  double is_floating_thickness;  /* mask_is_floating_thickness_standard                        */
} pism_gpu_ssafem_options;

typedef struct pism_gpu_ssafem_stats {
  int converged;                 /* 1: ||F|| test, 2: step test; 0: not converged               */
  int newton_iterations, ksp_iterations;
  double fnorm0, fnorm;          /* ||F|| at the initial guess and at the answer                */
} pism_gpu_ssafem_stats;

void pism_gpu_ssafem_options_defaults(pism_gpu_ssafem_options *o);

/* SSAFEM::solve (SSAFEM.cc:170-232): the coefficients at the quadrature points
 * (cacheQuadPtValues, SSAFEM.cc:233-375: thickness, bed, tau_c, the driving stress
 * -rho g H grad(surface), the GeometryCalculator mask and the column-averaged hardness), then
 * Newton on the weak-form residual (compute_local_function, :441-532) with its Jacobian
 * (compute_local_jacobian, :571-700), from the handle's current velocity (its initial guess or
 * the last solve's answer) to the handle's velocity.  Inputs are those of
 * pism_gpu_ssa_set_inputs (mask, melange and the CFBC are not used by this discretisation);
 * Dirichlet data where bc_mask is 1.  stats may be NULL.  Returns PISM_GPU_SSA_EPICARD when
 * the nonlinear solve does not converge ("SSAFEM solve failed to converge") and
 * PISM_GPU_SSA_EKSP when a linear solve breaks down or reaches ksp_max_it; after a failure the
 * handle's velocity is the one the solve started from (SSAFEM.cc:215-228). */
int pism_gpu_ssafem_solve(pism_gpu_ssa *h, const pism_gpu_ssafem_options *o, pism_gpu_ssafem_stats *stats);

/* Stage entry points, each the device restatement of one reference method, for
 * stage-by-stage checking:
 *   assemble_rhs       -> SSA::compute_driving_stress + SSAFD::assemble_rhs
 *   compute_hardness   -> SSAFD::compute_hardav_staggered (+ fracture softening)
 *   compute_nuH        -> SSAFD::compute_nuH_staggered[_cfbc] at the current
 *                         velocity, with regularisation `reg`; also refreshes beta
 *   apply              -> y = A x with the matrix SSAFD::assemble_matrix would
 *                         build from the current nu*H and beta (device pointers) */
int pism_gpu_ssa_assemble_rhs(pism_gpu_ssa *h);
int pism_gpu_ssa_compute_hardness(pism_gpu_ssa *h);
int pism_gpu_ssa_compute_nuH(pism_gpu_ssa *h, double reg);
int pism_gpu_ssa_apply(pism_gpu_ssa *h, const double *x_dev, double *y_dev);

/* z = M^-1 r with the active preconditioner, set up at the current nu*H / beta (PETSc's
 * PCSetUp + PCApply inside KSPSolve, SSAFD.cc:1018).  Device pointers, 2N each, not the same. */
int pism_gpu_ssa_apply_preconditioner(pism_gpu_ssa *h, const double *r_dev, double *z_dev);

/* One linear solve A x = b at the current nu*H / beta with the configured
 * Krylov method (the body of KSPSolve, SSAFD.cc:1018).  x (device, 2N) holds the
 * initial guess on entry.  *iterations and *rel_residual may be NULL. */
int pism_gpu_ssa_linear_solve(pism_gpu_ssa *h, double *x_dev, int *iterations,
                              double *rel_residual);

/* The same linear solve for the caller's right-hand side b (device, 2N; not x_dev): PETSc's
 * KSPSolve with any b (SSAFD.cc:1018 passes m_b).  Used to build the learned preconditioner's
 * training pairs (pism_unet_gpu.h). */
int pism_gpu_ssa_linear_solve_rhs(pism_gpu_ssa *h, const double *b_dev, double *x_dev, int *iterations,
                                  double *rel_residual);

/* ---- allocation-free entry point ------------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * hosts that route every device allocation through their own pool or arena,
 * code that works under a memory budget that forbids new allocations, and
 * bindings without access to the CUDA allocator.  It computes what pism_gpu_ssa_compute_nuH computes for the plain
 * (non-CFBC) stencil — nu*H on the staggered grid, under-relaxed against the
 * values in `nuH` when underrelax != 1 (SSAFD.cc:1061-1064), and the basal drag
 * coefficient of the next assembly — and writes the two L1 norms of the Picard
 * test, |nuH| and |nuH_before - nuH| (SSAFD.cc:1170-1189), to norms[0..1].
 *
 * All pointers are device memory: velocity (2N), thickness (N), hardness_stag
 * (2N), mask (N, doubles rounded as IceModelVec2Int::as_int does), tauc (N),
 * gl_mask (N; only read with sub_groundingline), nuH (2N, in: the previous
 * values, out: the new ones), beta (N, out), norms (2, out).  The work is
 * enqueued on `cuda_stream` (NULL = the legacy default stream) and the call
 * returns without waiting for it.
 *
 * It allocates nothing: its scratch is a fixed 512 KiB device array inside the
 * library, which every GPU that loads the library holds until the process exits.
 * So the grid may have at most PISM_GPU_SSA_NOALLOC_MAX_CELLS cells, in any shape
 * (larger grids return PISM_GPU_SSA_ETOOLARGE), and because every call shares that
 * array, calls whose work overlaps on the GPU (other streams, other host threads)
 * race: order them on one stream.  The first call on a device looks up the array's
 * device address; make that first call before any stream capture.  The return value
 * is this call's own status: an error that earlier work left pending in the CUDA
 * runtime (cudaGetLastError) is neither read nor cleared.
 * CFBC configurations return PISM_GPU_SSA_EINVAL (use the handle API). */
#define PISM_GPU_SSA_NOALLOC_MAX_CELLS (2048 * 2048)
int pism_gpu_ssa_nuH_noalloc(const pism_gpu_grid *grid, const pism_gpu_ssa_config *cfg,
                             const double *velocity, const double *thickness, const double *hardness_stag,
                             const double *mask, const double *tauc, const double *gl_mask,
                             double nuH_regularization, double underrelax, double *nuH, double *beta,
                             double *norms, void *cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* PISM_SSA_GPU_H */
