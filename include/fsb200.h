/*
 * fsb200.h -- C ABI of the B200 (sm_100a) SIMPLE inner loop.
 *
 * The entry points below replace the leaf and driver subroutines that the
 * Fortran solver fadlmoukalled/FlowSolverSourceCode calls once per outer
 * iteration (MainProgram/MainProgram.for:257-348).  Each declaration names
 * the reference interface it stands in for.  All state lives on the GPU in
 * an opaque context; Fortran (through ISO_C_BINDING) or
 * C/C++/Python (ctypes) hold only the context pointer and plain host arrays.
 *
 * Conventions
 *   - Indices are 0-based here (the reference is 1-based).  Face and cell
 *     numbering is the polyMesh order: interior faces first, then boundary
 *     faces patch by patch (ReadFoamMesh.f90:277-297).  The linear boundary
 *     face index b = sum(NBFaces(s<set)) + j is the reference's
 *     i4-NIFaces (AssembleGolbalElementAndFaceFluxes.for:83-92).
 *   - Every call returns an int status: FS_OK (0) or a negative FS_E_* code.
 *     Nothing traps; device waits are bounded and report FS_E_TIMEOUT.
 *   - Character dummies of the reference (Variable, solver, schemes) become
 *     the integer enums below.
 *   - One context is single-caller and non-reentrant (one CUDA stream).
 */
#ifndef FSB200_H
#define FSB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------------- status */
#define FS_OK             0
#define FS_E_ARG         -1   /* bad argument / size */
#define FS_E_CUDA        -2   /* CUDA runtime error */
#define FS_E_NOMEM       -3   /* device allocation failed */
#define FS_E_NAN         -4   /* NaN/Inf detected in a residual */
#define FS_E_DIVERGED    -5   /* stop metric grew by > FS_DIVERGENCE_FACTOR */
#define FS_E_TIMEOUT     -6   /* bounded device wait gave up */
#define FS_E_MESH        -7   /* inconsistent mesh */
#define FS_E_UNSUPPORTED -8   /* option not implemented */
#define FS_E_TOO_LARGE   -9   /* problem larger than a fixed-size scratch allows */

/* An outer iteration whose stop metric exceeds FS_DIVERGENCE_FACTOR times
 * the largest stop metric of the context's earlier outer iterations (of the
 * current time step, for unsteady runs) returns FS_E_DIVERGED.  The
 * reference has no such check (it prints and continues). */
#define FS_DIVERGENCE_FACTOR 1e6

/* ------------------------------------------------------- variable ids (NF)
 * GetNFfromVariable (AlgebraicSolvers/AssignNFvaluesToVariables.for:4):
 * velx=1, vely=2, velz=3, pressc=4, continuity residual slot 5. */
#define FS_VAR_U      1
#define FS_VAR_V      2
#define FS_VAR_W      3
#define FS_VAR_PC     4
#define FS_VAR_MASS   5
#define FS_VAR_TEMP   6   /* 'temp' (AssignNFvaluesToVariables.for:45), the temperature equation */
#define FS_VAR_TKE    8   /* 'tke' (AssignNFvaluesToVariables.for:55) */
#define FS_VAR_TED    9   /* 'ted' (AssignNFvaluesToVariables.for:60) */
#define FS_VAR_RHOK  10   /* 'rhok' = 2/3 rho k (gradient calls only, AssembleMinusTwoThirdsRhoK.for) */
#define FS_VAR_P     20   /* 'press' (pressure itself, gradient calls only; the reference's
                           * 'press' shares NF 5 with the continuity residual, so it takes
                           * an id of its own here) */

/* ------------------------------------------------------ field ids (get/set) */
enum fs_field {
  FS_F_U = 0, FS_F_V, FS_F_W, FS_F_P, FS_F_PC,      /* cell fields (N) */
  FS_F_MDOT,                                         /* interior faces (F) */
  FS_F_BU, FS_F_BV, FS_F_BW, FS_F_BP, FS_F_BPC,      /* boundary faces (B) */
  FS_F_BMDOT,
  FS_F_AC, FS_F_BC, FS_F_ANB,                        /* last assembled system (N, N, W*N slot-major) */
  FS_F_DU1, FS_F_DV1, FS_F_DW1, FS_F_DU2, FS_F_DV2, FS_F_DW2,
  FS_F_UGRAD, FS_F_VGRAD, FS_F_WGRAD, FS_F_PGRAD, FS_F_PCGRAD, /* 3N each: x block, y block, z block */
  FS_F_VOLUME, FS_F_XC,                              /* N, 3N geometry */
  FS_F_GFACTOR, FS_F_SF, FS_F_GDIFF, FS_F_FT,        /* F, 3F, F, 3F */
  FS_F_BSF,                                          /* 3B */
  FS_F_DPHI,                                         /* N: last linear solution */
  FS_F_TKE, FS_F_TED, FS_F_MUT,                      /* N: k, epsilon, turbulent viscosity */
  FS_F_BTKE, FS_F_BTED, FS_F_BMUT,                   /* B */
  FS_F_KX,                                           /* N: BICGSTAB_OMP's persistent solution vector */
  FS_F_UTAU, FS_F_YPLUS,                             /* B: wall-function state (uTau, yplus) */
  FS_F_OLD, FS_F_OLDOLD,                             /* 7N: u v w p k epsilon T at time levels n-1, n-2 (unsteady) */
  FS_F_BOLD,                                         /* 7B: their boundary values at n-1 */
  FS_F_T, FS_F_BT,                                   /* N, B: temperature (energy equation) */
  FS_F_TGRAD,                                        /* 3N: its gradient */
  FS_F_COUNT
};

/* -------------------------------------------------------- boundary types
 * BCType + wallTypeMomentum / inletTypeMomentum / outletTypeMomentum
 * (SetBoundaryPatches/SetBoundaryConditionPatches.for:88-200). */
enum fs_bc {
  FS_BC_WALL_NOSLIP = 0,   /* 'wall','noslip' (velocity given per patch: lid) */
  FS_BC_WALL_SLIP   = 1,   /* 'wall','slip' */
  FS_BC_SYMMETRY    = 2,   /* 'symmetry' */
  FS_BC_INLET_VEL   = 3,   /* 'inlet','specifiedvelocity' */
  FS_BC_OUTLET_FD   = 4,   /* 'outlet','fullydeveloped' */
  FS_BC_OUTLET_SP   = 5,   /* 'outlet','specifiedstaticpressure' (patch_pressure) */
  FS_BC_INLET_MASS  = 6,   /* 'inlet','specifiedmassflowrate': patch_vel is the velocity
                            * direction (xVeldirection...), patch_mass_flow the inflow */
  FS_BC_INLET_SP    = 7,   /* 'inlet','specifiedstaticpressure': patch_pressure, and
                            * patch_vel the velocity direction */
  FS_BC_OUTLET_MASS = 8,   /* 'outlet','specifiedmassflowrate': patch_mass_flow leaves the
                            * domain, along the owner cell's velocity */
  FS_BC_OUTLET_ASP  = 9,   /* 'outlet','specifiedaveragestaticpressure': treated as a static-pressure
                            * outlet, except that after each pressure correction the face pressure
                            * is the owner's, shifted so that its area average is patch_pressure
                            * (CorrectPressure.for:169-205) */
  FS_BC_OUTLET_RES  = 10,  /* 'outlet','specifiedresistance': the static-pressure outlet's flux and
                            * velocity; p'_b = R sum(gd p'_C)/(1 + R sum gd) over the patch, the p'
                            * diagonal coupled through it (AssemblePressureCorrectionFluxes.for:400-500,
                            * UpdatePressureCorrectionAtBoundaries.for:144-175) and p_b += urfP p'_b;
                            * R = patch_resistance (ArteryResistance), patch_pressure the initial p_b */
  FS_BC_INLET_STAG  = 11   /* 'inlet','specifiedstagnationpressure': the static-pressure inlet's flux
                            * and velocity (patch_vel the direction); after AssembleMdot
                            * p_b = max(p0 - rho |U_b|^2 / 2, 0) (TotalConditionsBoundary.for:25-45),
                            * the p' coefficients of AssemblePressureCorrectionFluxes.for:663-720 and
                            * UpdatePressureCorrectionAtBoundaries.for:97-112; patch_pressure = p0 */
};

/* ------------------------------------------------ thermal boundary types
 * The temperature equation's boundary sets (BoundaryConditions1: IWallDirichlet,
 * IWallVonNeumann, IWallRobin, IinletSpecifiedStaticTemperature,
 * IinletSpecifiedStagnationTemperature, IoutletFullyDevelopedEnergy, Isymmetry),
 * one per patch.  FS_TBC_DEFAULT takes the flow type's counterpart: walls von
 * Neumann with patch_heat_flux (adiabatic at 0), inlets static temperature,
 * outlets fully developed, symmetry planes symmetry. */
enum fs_tbc {
  FS_TBC_DEFAULT = 0,
  FS_TBC_WALL_DIRICHLET = 1,   /* wall temperature patch_temperature */
  FS_TBC_WALL_NEUMANN = 2,     /* heat flux patch_heat_flux into the domain per unit area */
  FS_TBC_WALL_ROBIN = 3,       /* HinfinityRobin = patch_h_inf, TinfinityRobin = patch_temperature */
  FS_TBC_INLET_STATIC = 4,     /* 'specifiedstatictemperature': patch_temperature */
  FS_TBC_INLET_STAGNATION = 5, /* 'specifiedstagnationtemperature': T = patch_temperature - |U_b|^2/(2 cp) */
  FS_TBC_OUTLET_FD = 6,        /* 'fullydevelopedenergy': T_b = T_owner */
  FS_TBC_SYMMETRY = 7          /* T_b = T_owner, no flux */
};

/* ---------------------------------------------------------- scheme enums */
enum fs_gradinterp { FS_GI_AVERAGE = 0, FS_GI_UPWIND, FS_GI_DOWNWIND, FS_GI_AVERAGECORRECTED };
enum fs_hr { FS_HR_NONE = 0, FS_HR_TVD = 1 };
/* TVDLimiter (Convection/LimitersTVDType.for:4) scheme names */
enum fs_tvd {
  FS_TVD_UPWIND = 0, FS_TVD_DOWNWIND, FS_TVD_FROMM, FS_TVD_SOU, FS_TVD_CD,
  FS_TVD_QUICK, FS_TVD_SUPERBEE, FS_TVD_MINMOD, FS_TVD_OSHER, FS_TVD_VANLEER,
  FS_TVD_MUSCL, FS_TVD_SMART, FS_TVD_HQUICK, FS_TVD_UMIST, FS_TVD_CHARM
};
/* ASSolver* (SolveAlegbraicEquations.for:105-175) plus the GPU-only forms */
enum fs_solver {
  FS_SOLVER_SOR = 0,       /* 'sor': symmetric Gauss-Seidel sweeps (GPU: multicolour order) */
  FS_SOLVER_BICGS = 1,     /* 'bicgs': BICGSTAB_OMP restated (matrixSolverOMP.f90:306) */
  FS_SOLVER_AMG = 2,       /* LMultigrid=.true., MGType='geometricelement' */
  FS_SOLVER_AMG_BICGS = 3, /* FP64 BiCGSTAB right-preconditioned by one AMG V-cycle (no reference row) */
  FS_SOLVER_AMG32_BICGS = 4,/* same with an FP32 AMG hierarchy (iterative refinement, no reference row) */
  FS_SOLVER_GMRES = 5,     /* 'gmres': GMRES_RESTARTED_OMP_RETURNR restated (matrixSolverOMP.f90:48) */
  FS_SOLVER_ILU = 6,       /* 'ilu': D-ILU factorisation once, then ILU sweeps until rrF or itmax
                            * (FactorizeUsingILU.for:4, ILUMethod.for:4, SolveAlegbraicEquations.for:122-133) */
  FS_SOLVER_AMG32GS_BICGS = 7,/* FP64 BiCGSTAB preconditioned by an FP32 V-cycle with symmetric multicolour
                            * Gauss-Seidel smoothing (no reference row) */
  FS_SOLVER_PBCG = 8       /* 'pbcg': biconjugate gradient, minimum-residual form, preconditioned by the
                            * D-ILU diagonal, one iteration per CheckConvergence until rrF or itmax
                            * (PBCGMethod.for:96-180, SolveAlegbraicEquations.for:138-152) */
};
enum fs_algorithm { FS_SIMPLE = 0, FS_SIMPLEC = 1 };

#define FS_MAX_PATCHES 32

/* Case description: the knobs of User0.F90 / DescribeProblem that the inner
 * loop reads (ProblemDescriptionRoutine.for:201-524). */
typedef struct fs_case {
  double rho;                    /* Density (constant) */
  double mu;                     /* Viscosity (constant, laminar) */
  int    algorithm;              /* Algorithm: FS_SIMPLE / FS_SIMPLEC */
  int    relax_momentum;         /* LRelaxMomentum */
  double urf_momentum;           /* urfMomentum */
  double urf_pressure;           /* urfPressure (always applied, CorrectPressure.for:42) */
  int    method_grad_mom;        /* MethodCalcGradientMomentum (1 or 2) */
  int    method_grad_cont;       /* MethodCalcGradientContinuity (1 or 2) */
  int    niter_grad_mom;         /* nIterGradientMomentum */
  int    niter_grad_cont;        /* nIterGradientContinuity */
  int    grad_interp_mom;        /* GradientInterpolationSchemeMomentum */
  int    grad_interp_cont;       /* GradientInterpolationSchemeContinuity */
  int    method_decompose_s;     /* MethodDecomposeS (1,2,3); geometry + Rhie-Chow */
  int    hr_framework;           /* HRFrameworkMomentum */
  int    conv_scheme;            /* ConvectionSchemeMomentum (fs_tvd) */
  int    niter_start_hr;         /* nIterStartApplyingHR */
  double bleed;                  /* BleedMomentum */
  int    solver_mom;             /* ASSolverMomentum / LMultigridMomentum */
  int    solver_cont;            /* ASSolverContinuity / LMultigridContinuity */
  double rrf_mom, rrf_cont;      /* rrFMomentum, rrFContinuity */
  int    itmax_mom, itmax_cont;  /* ASIterMomentum, ASIterContinuity */
  int    nstop_type;             /* NstopType 1..4 */
  double max_residual;           /* maximumResidual */
  int    ref_pressure_cell;      /* ReferencePressureLocation (0-based) */
  int    set_reference_pressure; /* LSetReferencePressure (0/1) */
  int    inviscid;               /* Linviscid */
  /* multigrid (MultiGrid*, ProblemDescriptionRoutine.for:392-430) */
  int    mg_cycle;               /* 0 V, 1 F, 2 W  (MultiGridCycleType) */
  int    mg_pre, mg_post;        /* MultiGridpreSweep / MultiGridpostSweep */
  int    mg_max_cycles;          /* MaxMultiGridCycles */
  int    mg_min_parents;         /* minNumberofParents */
  int    mg_max_levels;          /* maxNumberofCoarseLevels */
  double mg_rrf;                 /* MultiGridrrf */
  /* krylov (BICGSTAB_OMP(N,100,1.d-5)) */
  int    krylov_maxit;
  double krylov_tol;
  /* patches, in polyMesh boundary order */
  int    n_patches;
  int    patch_type[FS_MAX_PATCHES];      /* fs_bc */
  double patch_vel[FS_MAX_PATCHES][3];    /* wall / inlet velocity */
  /* multi-RHS momentum (no reference row): assemble X, Y and Z from the same
   * velocities and solve them together (one Gauss-Seidel kernel, shared anb);
   * the Y/Z wall cross terms then use the previous iteration's u, v.  Only
   * with solver_mom = FS_SOLVER_SOR. */
  int    batched_momentum;
  /* outlets 'fullydeveloped': MassFlowFraction per patch (AdjustFlowAtOuletBoundary.for:38-55) */
  double mass_flow_fraction[FS_MAX_PATCHES];
  /* k-epsilon (TurbulenceModel='kepsilon', WallTreatment='wallfunctions',
   * WallFunctionKind='equilibrium', MomentumWallFunctionType 'standard', 'scalable' or 'automatic';
   * SolveSelectedTurbulenceModelEquations.for:21-30).  0 = laminar. */
  int    turbulence;
  int    solver_turb;            /* ASSolverTKE = ASSolverTED */
  double rrf_tke, rrf_ted;       /* rrfTKE, rrfTED */
  int    itmax_tke, itmax_ted;   /* ASIterTKE, ASIterTED */
  double urf_tke, urf_ted;       /* urfTKE, urfTED (LRelaxTKE/TED) */
  double urf_tvisc;              /* urfTViscosity */
  double max_visc_ratio;         /* MaximumViscosityRatio */
  int    limit_production;       /* LimitTurbulenceProduction */
  int    conv_scheme_tke, conv_scheme_ted; /* ConvectionSchemeTKE/TED (fs_tvd; HR framework tvd) */
  double inlet_intensity[FS_MAX_PATCHES];  /* inletTurbulenceIntensity, inletTypeT='specifiedil' */
  double inlet_length[FS_MAX_PATCHES];     /* inletTurbulenceLengthScale */
  int    wall_function;          /* MomentumWallFunctionType: 0 'standard', 1 'scalable', 2 'automatic' */
  double patch_pressure[FS_MAX_PATCHES];  /* static pressure of 'specifiedstaticpressure' outlets */
  /* unsteady runs (LUnsteady, TransientScheme, dt; ProblemDescriptionRoutine.for:539):
   * the transient term of the momentum, k and epsilon equations
   * (AssembleTheTransientTerm.for:52-330).  Time steps are advanced by
   * fs_advance_time; 0 = steady. */
  int    unsteady;
  int    transient_scheme;       /* fs_transient */
  double dt;                     /* first time step */
  /* 'specifiedmassflowrate' inlets and outlets: mass flow into (inlets) or
   * out of (outlets) the domain per patch, spread over the faces by area as
   * the initial Bmdot (the reference leaves the face values to
   * DescribeProblem: set FS_F_BMDOT to override) */
  double patch_mass_flow[FS_MAX_PATCHES];
  /* 'specifiedresistance' outlets: ArteryResistance per patch */
  double patch_resistance[FS_MAX_PATCHES];
  /* temperature equation (LSolveEnergy, EnergyEquation='temperature';
   * Energy/SolveTemperatureEquation.for:4-291), solved after the turbulence
   * equations of each outer iteration (MainProgram.for:281): constant rho, cp
   * and conductivity, isotropic diffusion.  0 = isothermal. */
  int    energy;
  double cp;                     /* SpecificHeat */
  double conductivity;           /* Conductivity */
  double temp_init;              /* initial temperature of the cells and of the faces no boundary type sets */
  int    solver_energy;          /* ASSolverEnergy */
  double rrf_energy;             /* rrfEnergy */
  int    itmax_energy;           /* ASIterEnergy */
  int    relax_energy;           /* LRelaxEnergy */
  double urf_energy;             /* urfEnergy */
  int    conv_scheme_energy;     /* ConvectionSchemeEnergy (fs_tvd, HRFrameworkEnergy 'tvd') */
  double bleed_energy;           /* BleedEnergy */
  int    method_grad_energy;     /* MethodCalcGradientEnergy (1 or 2) */
  int    niter_grad_energy;      /* nIterGradientEnergy */
  int    grad_interp_energy;     /* GradientInterpolationSchemeEnergy (fs_gradinterp) */
  int    gamma_interp_energy;    /* InterpolationSchemeGamaEnergy: 0 'average', 1 'upwind',
                                  * 2 'downwind', 3 'harmonic' (InterpolateFromElementToFace.for:17-60) */
  double energy_sc, energy_sb;   /* ScEnergy, SbEnergy, uniform: the source Sb + Sc T per unit volume */
  int    limit_temperature;      /* LimitTemperature */
  double temp_min, temp_max;     /* tempmin, tempmax */
  double sigma_t;                /* SigT, the turbulent Prandtl number of k-epsilon runs */
  int    energy_wall_function;   /* EnergyWallFunctionType of k-epsilon runs: 0 'standard', 1 'scalable', 2 'automatic' */
  int    patch_thermal[FS_MAX_PATCHES];      /* fs_tbc */
  double patch_temperature[FS_MAX_PATCHES];  /* wall, inlet static or stagnation temperature; TinfinityRobin */
  double patch_heat_flux[FS_MAX_PATCHES];    /* HeatFlux of von Neumann walls */
  double patch_h_inf[FS_MAX_PATCHES];        /* HinfinityRobin */
  /* p' initial guess from the pc_history (0..7) previous p' solutions
   * (fs_set_pc_history; no reference counterpart); 0 = zero start */
  int    pc_history;
  /* AMG-BiCGSTAB preconditioner reuse: the coarse matrices and the dense
   * coarsest inverse are rebuilt every pc_refresh solves of the same system
   * and kept in between (level 0 is always the current system); 0 or 1 =
   * every solve.  No reference counterpart. */
  int    pc_refresh;
} fs_case;

/* TransientScheme values (AssembleTheTransientTerm.for:52,124,199,290). */
enum fs_transient {
  FS_TRANSIENT_EULER          = 0,   /* 'euler' */
  FS_TRANSIENT_CRANKNICOLSON1 = 1,   /* 'cranknicolson1': Euler over dt/2, then extrapolate */
  FS_TRANSIENT_CRANKNICOLSON2 = 2,   /* 'cranknicolson2': three time levels */
  FS_TRANSIENT_ADAMSMOULTON   = 3    /* 'adamsmoulton': three time levels */
};

/* Mesh in polyMesh form (0-based), the input Readit parses
 * (GridAndGeometry/ReadFoamMesh.f90:31-297). */
typedef struct fs_mesh_in {
  int32_t        n_nodes;
  const double  *points;      /* 3*n_nodes, xyz interleaved */
  int32_t        n_faces;     /* all faces */
  const int32_t *face_ptr;    /* n_faces+1 offsets into face_nodes */
  const int32_t *face_nodes;
  const int32_t *owner;       /* n_faces */
  int32_t        n_internal;  /* faces [0,n_internal) have a neighbour */
  const int32_t *neighbour;   /* n_internal */
  int32_t        n_patches;
  const int32_t *patch_start; /* n_patches, face index of first patch face */
  const int32_t *patch_size;  /* n_patches */
  /* Optional (NULL: the polyMesh order of Readit, ReadFoamMesh.f90:311-458).
   * A mesh built by GlobalConnectivity (Gambit neutral files) keeps each
   * element's faces in its local face order (NGlobalEFaces,
   * GlobalGridConnectivity.for:125-345) and its nodes in file order
   * (ListOfElementNodes, ReadGridFromNeutralFile.for): both set the order of
   * the per-cell sums, so they are passed as given.  fs_neu_connectivity
   * returns them. */
  const int32_t *cell_face_ptr; /* n_cells+1 offsets into cell_faces */
  const int32_t *cell_faces;    /* face ids, each interior face once per side, each boundary face once */
  const int32_t *cell_node_ptr; /* n_cells+1 offsets into cell_nodes */
  const int32_t *cell_nodes;
} fs_mesh_in;

/* Gambit neutral-file elements (ReadNeutralGrid, ReadGridFromNeutralFile.for)
 * for fs_neu_connectivity.  0-based node and element ids; bc_face is the
 * element-local face, 0-based, in the face numbering of GlobalConnectivity
 * (GlobalGridConnectivity.for:21-120). */
typedef struct fs_neu_in {
  int32_t        n_elements;
  const int32_t *type;          /* NTypeGeometry: 4 brick, 5 wedge, 6 tetrahedron, 7 pyramid */
  const int32_t *node_ptr;      /* n_elements+1 offsets into nodes */
  const int32_t *nodes;         /* element nodes in file order */
  int32_t        n_sets;        /* NumberOfBCSets */
  const int32_t *set_size;      /* NBCDataRecords per set */
  const int32_t *bc_element;    /* NElementBC, sets concatenated */
  const int32_t *bc_face;       /* NElementBCFace */
} fs_neu_in;

/* Residual block (Residuals1.F90), indexed by NF-1 for NF=1..5. */
typedef struct fs_residuals {
  double abs_[5], max_[5], rms[5], scaled[5];
  double overall_imbalance;   /* OverallImbalance */
  int    imax_imbalance;      /* iMaxImbalance (0-based) */
  int    lin_iters[5];        /* linear iterations spent per NF this outer iteration */
  double source;              /* stop metric of PrintConvergenceHistory */
  /* k and epsilon equations (NF 8, 9), filled when the case is turbulent */
  double turb_abs[2], turb_max[2], turb_rms[2], turb_scaled[2];
  int    turb_lin_iters[2];
  /* temperature equation (NF 6), filled when the case solves it */
  double temp_abs, temp_max, temp_rms, temp_scaled;
  int    temp_lin_iters;
} fs_residuals;

typedef struct fs_ctx fs_ctx;

/* ---------------------------------------------------------- lifetime
 * Replaces Grid + allocateStorage + SetBCPatches + CalculateInitialmdot
 * (MainProgram.for:57-73,142).  Builds connectivity on the host (bit-exact
 * with Readit), computes geometry on the GPU (ProcessGeometryRoutine.for:3),
 * sets the initial state u=v=w=p=0 with patch velocities on the boundary,
 * and the initial mdot (InitializaMdot.for:4). */
int fs_create(const fs_mesh_in *mesh, const fs_case *cfg, int device, fs_ctx **out);
int fs_destroy(fs_ctx *ctx);
int fs_sizes(const fs_ctx *ctx, int32_t *n_cells, int32_t *n_ifaces,
             int32_t *n_bfaces, int32_t *max_faces);
const char *fs_last_error(const fs_ctx *ctx);

/* ------------------------------------------------------- driver routines */
/* SolveMomentumX/Y/Z (Momentum/SolveXMomentumEquation.for:4,
 * SolveYMomentumEquation.for:4, SolveZMomentumEquation.for:4). comp=0,1,2. */
int fs_solve_momentum(fs_ctx *ctx, int comp);
/* SolveContinuity (ContinuityEquation/SolveContinuityEquation.for:4). */
int fs_solve_continuity(fs_ctx *ctx);
/* p' initial guess from the m (0..7) previous p' solutions (no reference
 * counterpart: the reference starts p' from zero).  The AMG-BiCGSTAB solvers
 * start from the combination of those solutions (and of the learned guess,
 * when it is on) that minimises |b - A x0| -- least squares over their span,
 * so the starting residual never exceeds |b| -- and iterate to the same
 * tolerance.  m = 0 (the default) starts from zero; other solvers ignore it. */
int fs_set_pc_history(fs_ctx *ctx, int m);
/* SolveEnergy, EnergyEquation='temperature' (Energy/SelectEnergyEquationToSolve.for:4,
 * SolveTemperatureEquation.for:4): one temperature solve on the current
 * velocities and mass fluxes.  FS_E_ARG when the case has energy = 0. */
int fs_solve_energy(fs_ctx *ctx);
/* One outer iteration of MainProgram.for:257-325 (momentum x,y,z,
 * continuity, k-epsilon, temperature, PrintConvergenceHistory's stop metric). */
int fs_simple_iteration(fs_ctx *ctx, fs_residuals *res);
/* Same, but the state arrays live on the HOST: they are copied in, the
 * iteration runs, and they are copied back (the Fortran-owned layout of a
 * drop-in: u,v,w,p [N], mdot [F], bu,bv,bw,bp,bmdot [B]). */
int fs_simple_iteration_host(fs_ctx *ctx, double *u, double *v, double *w,
                             double *p, double *mdot, double *bu, double *bv,
                             double *bw, double *bp, double *bmdot,
                             fs_residuals *res);

/* The two halves of each driver around its SolveEquation call, for callers
 * that run their own solver (and for per-kernel parity checks):
 * fs_assemble_momentum = SolveXMomentumEquation.for:177-292 (fluxes,
 * gradients in X, assembly, UnderRelaxEquation, storeDvalues);
 * fs_assemble_continuity = SolveContinuityEquation.for:37-74;
 * fs_correct_continuity = SolveContinuityEquation.for:79-100. */
int fs_assemble_momentum(fs_ctx *ctx, int comp);
int fs_assemble_continuity(fs_ctx *ctx);
int fs_correct_continuity(fs_ctx *ctx);
/* MultiGrid2 nIter (gates nIterStartApplyingHR). */
int fs_set_iteration(fs_ctx *ctx, int n_iter);
/* CalculateInitialmdot (ContinuityEquation/InitializaMdot.for:4): mdot and
 * Bmdot from the current cell and boundary velocities, for a caller that set
 * an initial field with fs_set_field (fs_create already ran it once). */
int fs_initialize_mdot(fs_ctx *ctx);

/* GlobalConnectivity (GlobalGridConnectivity.for:4-523) in O(N) with a hash
 * of sorted face nodes instead of the O(N^2) search, the same face order:
 * elements in order, local faces in order; a face not on a boundary record
 * and not seen before becomes the next interior face (nodes in the creating
 * element's local order, owner = lower element id); boundary faces follow,
 * set by set, record by record.  Host-only (no GPU).  Outputs, sized by the
 * caller for F_max = sum of local faces over elements: face_ptr (F_max+1),
 * face_nodes (4 F_max), owner (F_max), neighbour (F_max), cell_face_ptr
 * (n_elements+1), cell_faces (F_max); n_internal and n_faces are written.
 * Returns FS_E_MESH for an unknown element type, a bad boundary record or a
 * face shared by more than two elements. */
int fs_neu_connectivity(const fs_neu_in *in, int32_t *n_internal, int32_t *n_faces,
                        int32_t *face_ptr, int32_t *face_nodes, int32_t *owner, int32_t *neighbour,
                        int32_t *cell_face_ptr, int32_t *cell_faces);

/* Time-step prologue of the unsteady loop (MainProgram.for:184-245): the
 * first step of 'cranknicolson2'/'adamsmoulton' runs as 'euler'; from the
 * second step on 'cranknicolson1' first extrapolates every solved field
 * (CrankNicolsonRoutine.for:4: phi = 2 phi - phiOld, boundary values too) and
 * re-assembles the face mass fluxes (AssembleMdot); then the time levels are
 * shifted (updateVariablesInTime, AdvanceVariablesInTime.for:4), dtOldOld =
 * dtOld = dt, dt = dt_next, time += dt and the outer-iteration counter
 * restarts (do nIter=1,IterMax).  Requires cfg.unsteady. */
int fs_advance_time(fs_ctx *ctx, double dt_next);
/* AdaptiveTimeStep (CalculateAdaptiveTimeStep.for:4-200; called from the time
 * loop when LadaptiveTimeStep, MainProgram.for:235-241) for a laminar,
 * isothermal unsteady case: the 'velx' limit of CalculateAdaptiveTimeStepValue
 * (:203-1758) from the current mass fluxes -- per cell the diffusion sum
 * gamf gDiff of its faces with the boundary terms of no-slip walls, inlets,
 * mass-flow outlets and symmetry, plus the convection max(mdot, 0) terms --
 * dtlocal = courant / max over cells of that sum / (rho V), and
 * *dt_next = min(max(dtlocal, min_factor dt), max_factor dt) with dt the
 * current time step.  The reference's defaults are GlobalCourantNumber 2,
 * minimumdtChangeFactor 0.5, maximumdtChangeFactor 5
 * (ProblemDescriptionRoutine.for:544-546).  Pass *dt_next to
 * fs_advance_time.  FS_E_ARG for steady, turbulent or energy cases (their
 * k, epsilon and temperature limits are not built).  Synchronises ctx's stream. */
int fs_adaptive_time_step(fs_ctx *ctx, double courant, double min_factor, double max_factor, double *dt_next);
/* Time state: t[0] time, t[1] dt, t[2] dtOld, t[3] dtOldOld, and ndt (the
 * number of time steps taken).  fs_set_time restores it for a restart
 * (readSolution, ReadSolutionToContinue.for:59-108, restores the old time
 * levels, which are the fields FS_F_OLD, FS_F_OLDOLD and FS_F_BOLD). */
int fs_get_time(fs_ctx *ctx, double t[4], int32_t *n_steps);
int fs_set_time(fs_ctx *ctx, const double t[4], int32_t n_steps);

/* ---------------------------------------------------------- leaf routines */
/* Gradient (GradientFiles/CalculateGradients.for:3) of field var
 * (FS_VAR_U/V/W/P/PC) into its gradient arrays, method 1 or 2. */
int fs_gradient(fs_ctx *ctx, int var, int method, int n_iter);
/* Gradient of host arrays phi [N] / bphi [B] -> grad [3N] / bgrad [3B]
 * (x block, y block, z block).  var selects the boundary corrections. */
int fs_gradient_host(fs_ctx *ctx, int var, int method, int n_iter,
                     const double *phi, const double *bphi,
                     double *grad, double *bgrad);
/* UnderRelaxEquation (UnderRelaxVariables/UnderRelaxation.for:4) on the
 * currently assembled system. */
int fs_under_relax(fs_ctx *ctx, double urf);
/* SolveEquation (AlgebraicSolvers/SolveAlegbraicEquations.for:4) on the
 * currently assembled system for variable var; updates the field by dphi. */
int fs_solve_equation(fs_ctx *ctx, int var, double rrf, int itmax, int solver);
/* Solve a host-given system ac [N], anb [W*N slot-major], bc [N] for dphi [N]
 * with the given solver (the matrix layout of Variables2.F90). */
int fs_solve_system_host(fs_ctx *ctx, const double *ac, const double *anb,
                         const double *bc, double *dphi, double rrf, int itmax,
                         int solver, int *iters);
/* CalculateResiduals (CalculateResidualsRoutine.for:3) of the assembled
 * system at dphi=0 for field var; fills res slot var-1. */
int fs_residuals_get(fs_ctx *ctx, fs_residuals *res);

/* ----------------------------------------------------- state transfer */
int fs_get_field(fs_ctx *ctx, int field, double *host, size_t n);
int fs_set_field(fs_ctx *ctx, int field, const double *host, size_t n);
/* Connectivity produced by the Readit restatement (0-based):
 * n_cell_faces [N], cell_faces [W*N slot-major, -1 unused],
 * cell_nbr [W*N, -1 boundary/unused], own_slot [F], nbr_slot [F]. */
int fs_get_connectivity(fs_ctx *ctx, int32_t *n_cell_faces, int32_t *cell_faces,
                        int32_t *cell_nbr, int32_t *own_slot, int32_t *nbr_slot);
/* Multigrid hierarchy (geometric-element agglomeration): number of levels,
 * level sizes, and the parent map of level l -> l+1 (0-based). */
int fs_mg_levels(fs_ctx *ctx, int32_t *n_levels, int32_t *level_sizes, int max_levels);
int fs_mg_parents(fs_ctx *ctx, int level, int32_t *parents, size_t n);
/* Level shapes (no reference counterpart; diagnostics and the byte counts of
 * the bench roofline): ELL width of each level and the coarsest level the
 * AMG preconditioner cycles to (inverted densely when *direct is 1). */
int fs_mg_info(fs_ctx *ctx, int32_t *widths, int max_levels, int32_t *prec_coarsest, int32_t *direct);
/* AssembleAgglomeratedLHS (AssembleElementBasedAgglomoratedLHS.for:45-150) of
 * the last assembled system, read back for level `level` >= 1: ac [n],
 * n_nbr [n], nbr and anb [w*n slot-major, nbr -1 past n_nbr[i]], with n and
 * w the level's size and ELL width (fs_mg_levels, fs_mg_info). */
int fs_mg_coarse_matrix(fs_ctx *ctx, int level, double *ac, int32_t *n_nbr, int32_t *nbr, double *anb,
                        size_t n, size_t w);

/* ----------------------------------------------------- learned p' initial guess
 * No reference counterpart: the reference starts every p' solve from zero.
 * A 4-layer message-passing network on the cell graph (hidden width 64, BF16
 * tensor-core layer products with FP32 accumulation) maps features of the p'
 * system (mass imbalance, coefficients, velocity-gradient diagonal, previous
 * p') to an initial guess for the AMG-preconditioned BiCGSTAB solvers, which
 * scale it by the c minimising |b - c A x0| (so |r0| <= |b|) and still
 * iterate to their tolerance relative to |b|.
 *   fs_nn_create     network (seeded init, untrained guess = 0) and room for
 *                    snapshot_capacity training snapshots of this mesh
 *   fs_nn_mode       capture: store (features, edge weights, converged p')
 *                    after every p' solve; use: seed the p' solves
 *   fs_nn_train      epochs of Adam over the stored snapshots on the GPU;
 *                    mean relative loss of the first and last epoch
 *   fs_nn_params     copy the FS_NN_NPARAM parameters out (get) and/or in (set)
 *   fs_nn_eval_host  forward (and, with target, loss + gradient) on host
 *                    inputs X [N x 8], edge weights [W*N slot-major], target [N]
 *   fs_nn_stats      p' solves seeded by the network, and how many fell back
 *                    to zero (scale c zero or not finite)
 *   fs_nn_policy     the guess is used only while it reduces iterations
 *                    against zero-start probes (every 4th solve): average
 *                    p' iterations with the guess and from zero, and how often
 *                    the guess was parked */
#define FS_NN_NPARAM 33665
int fs_nn_create(fs_ctx *ctx, int snapshot_capacity, uint64_t seed);
int fs_nn_mode(fs_ctx *ctx, int capture, int use);
int fs_nn_snapshots(fs_ctx *ctx, int32_t *count);
int fs_nn_train(fs_ctx *ctx, int epochs, float lr, uint64_t seed, float *loss_first, float *loss_last);
int fs_nn_params(fs_ctx *ctx, float *get, const float *set, size_t n);
int fs_nn_eval_host(fs_ctx *ctx, const float *X, const float *wgt, const float *target, float *loss, float *grad,
                    float *y);
int fs_nn_stats(fs_ctx *ctx, int32_t *uses, int32_t *fallbacks);
int fs_nn_policy(fs_ctx *ctx, double *avg_guessed, double *avg_zero, int32_t *parked);

/* ----------------------------------------------------- ensemble and launch shape
 * No reference counterparts.
 * fs_set_launch_shape: threads per SM of the persistent cooperative solver
 *   kernels, in units of 256 (1..4; 0 = 1024): every cooperative launch puts
 *   one CTA of 256 * shape threads on each SM; the project's autotuner
 *   (flowsolversourcecode_b200/ensemble.py) picks it per case by timing.
 * fs_ensemble_run: `iters` SIMPLE iterations of each of n independent cases
 *   (contexts on one GPU) captured into one CUDA graph, cases in sequence so
 *   their cooperative kernels never overlap, launched `launches` times with one
 *   host synchronisation per launch.  source_out [n * iters * launches]
 *   (case-major) receives the stop metric after every iteration, pc_iters_out
 *   (optional, same shape) the p' iterations, ms_out the device time.  One
 *   ordinary iteration per case runs first (hierarchies, colourings, grids);
 *   the learned guess is not used inside the graph. */
int fs_set_launch_shape(fs_ctx *ctx, int shape);
/* Test of the bounded device waits (no reference counterpart): with extra > 0
 * the AMG preconditioner's team barriers wait for `extra` more CTAs than take
 * part, so their bounded polls run out (well under a second); the iteration
 * then returns FS_E_TIMEOUT and its results are not valid.  0 restores normal
 * operation. */
int fs_test_wait_timeout(fs_ctx *ctx, int extra);
int fs_ensemble_run(fs_ctx **ctxs, int n, int iters, int launches, double *source_out, int32_t *pc_iters_out,
                    float *ms_out);
/* fs_ensemble_run_batched: the same with the cases concurrent.  Inside each
 * iteration the p' solves of all cases (initial-guess fit, then the Krylov
 * solve) run as ONE cooperative launch in which each case has its own group of
 * CTAs (sized in proportion to its cells times its p' iterations in the
 * warm-up) and its own bounded barriers; when every case uses the multi-RHS
 * momentum SOR, the momentum solves are one such launch too (groups by cells),
 * and the cases' other kernels run as concurrent graph branches between the
 * launches (the part after the p' solve stays in sequence for cases with
 * k-epsilon or the temperature equation).  All cases must use the same
 * AMG-BiCGSTAB p' solver form (FS_E_UNSUPPORTED otherwise).  A case's sums then
 * run over its group rather than the whole grid, so results differ from
 * fs_ensemble_run's within the linear solvers' tolerances. */
int fs_ensemble_run_batched(fs_ctx **ctxs, int n, int iters, int launches, double *source_out,
                            int32_t *pc_iters_out, float *ms_out);
/* fs_ensemble_split: the CTA groups of fs_ensemble_run_batched calls whose
 * first context is ctx are sized in proportion to cells^exponent (momentum) and
 * cells^exponent x warm-up p' iterations (p'); exponent in [0, 2], 1 by default.
 * Below 1 small cases get more CTAs than their share of cells, which pays when
 * their latency-bound phases, not bandwidth, set a group's time.  The project's
 * autotuner (ensemble.py) picks it by timing.  No reference counterpart. */
int fs_ensemble_split(fs_ctx *ctx, double exponent);

/* Timing of the last outer iteration's phases in milliseconds (CUDA events):
 * [0] momentum assembly, [1] momentum solves, [2] continuity assembly,
 * [3] p' solve, [4] corrections+residuals. */
int fs_phase_times(fs_ctx *ctx, float *ms5);
/* CUDA-event timer on the context stream: fs_timer_start records the start
 * event; fs_timer_stop records the stop event, waits for it and returns the
 * elapsed device time in milliseconds. */
int fs_timer_start(fs_ctx *ctx);
int fs_timer_stop(fs_ctx *ctx, float *ms);
/* Linear-solver statistics accumulated since the last reset, per NF 1..5:
 * device time of the solver kernels (CUDA events around each launch, in ms),
 * solver iterations, and calls.  reset=1 clears them after reading. */
int fs_solver_stats(fs_ctx *ctx, float *ms5, int32_t *iters5, int32_t *calls5, int reset);
/* Milliseconds of the main cooperative solver kernel alone (no set-up
 * kernels) per NF, accumulated like fs_solver_stats and reset with it.  No
 * reference counterpart (roofline timing). */
int fs_solver_kernel_ms(fs_ctx *ctx, float *ms5);
/* Number of kernel launches issued by this context since creation. */
int64_t fs_launch_count(const fs_ctx *ctx);
/* Synchronise the context stream. */
int fs_sync(fs_ctx *ctx);

/* BiCGSTAB without any device allocation.  No counterpart in the reference:
 * it is the k_bicgstab solve of fs_solve_system_host for callers that cannot
 * call cudaMalloc (a host whose device memory is owned by another allocator,
 * or that must not allocate once running).  All pointers are device memory
 * owned by the caller, in the layout of fs_solve_system_host: ncf [n],
 * cn and anb [w*n slot-major], ac and bc [n]; x [n] holds the initial guess on
 * entry and the solution on return; iters (device int32, may be NULL) gets
 * the iteration count.  The work vectors live in one fixed device array of
 * the library, so n may not exceed FS_NOALLOC_MAX_ROWS (FS_E_TOO_LARGE
 * otherwise).  The solve is queued on `stream` (a cudaStream_t, NULL for the
 * default stream) and the call returns without waiting.  Every call on a
 * device shares that array: calls that overlap on the GPU race on it.  The
 * first call on a device does a one-time set-up: it looks the array's device
 * address up with cudaGetSymbolAddress and keeps it for the CUDA context
 * current at the call (a call under another context of the device repeats
 * it); make that first call before any stream capture begins. */
#define FS_NOALLOC_MAX_ROWS 262144
int fs_bicgstab_noalloc(int32_t n, int32_t w, const int32_t *ncf, const int32_t *cn,
                        const double *ac, const double *anb, const double *bc, double *x,
                        int32_t maxit, double tol, int32_t *iters, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* FSB200_H */
