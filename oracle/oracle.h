/*
 * oracle.h -- CPU restatement of the reference SIMPLE inner loop.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this
 * code; only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * --impl reference legs load it, as the checker and as the timed CPU
 * baseline.
 *
 * PARITY UNPINNED: the reference (fadlmoukalled/FlowSolverSourceCode) is
 * Fortran, no Fortran compiler exists in this image, and the reference ships
 * no tests, golden vectors or fixtures.  This file restates the reference's
 * subroutines line by line (each function cites file:line) and is pinned
 * only by the analytic invariants checked in tests/test_oracle.py.
 *
 * Indices are 0-based; slot-major 2-D arrays (anb, cell_faces, cell_nbr) are
 * stored as a[j*N + i], i.e. exactly the column-major Fortran anb(i,j).
 */
#ifndef FS_ORACLE_H
#define FS_ORACLE_H
#include "../include/fsb200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct om om;

om    *om_create(const fs_mesh_in *mesh, const fs_case *cfg);
void   om_destroy(om *m);
/* Direct pointer to a named internal array (see om_arrays in oracle.c);
 * *len receives its element count, *is_int 1 for int32 arrays. */
void  *om_array(om *m, const char *name, long *len, int *is_int);
int    om_sizes(om *m, int *N, int *F, int *B, int *W);

/* SIMPLE driver pieces (MainProgram.for:257-325) */
void   om_momentum(om *m, int comp);           /* SolveMomentumX/Y/Z */
void   om_continuity(om *m);                   /* SolveContinuity */
double om_simple_iteration(om *m);             /* one outer iteration, returns source */
void   om_set_iter(om *m, int nIter);          /* MultiGrid2 nIter */
void   om_residuals(om *m, double out[20]);    /* ResorAbs/Max/RMS/Scaled x5 */
int    om_lin_iters(om *m, int nf);            /* linear iterations last solve of NF */
void   om_energy(om *m);                      /* SolveEnergy ('temperature') on the current flow */
void   om_residuals_temp(om *m, double out[4]);/* abs/max/rms/scaled of the temperature (NF 6) */
void   om_residuals_turb(om *m, double out[8]);/* abs/max/rms/scaled of k, epsilon (NF 8, 9) */
void   om_initialize_mdot(om *m);              /* CalculateInitialmdot from the current fields */
int    om_neu_connectivity_literal(const fs_neu_in *in, int *n_internal, int *n_faces, int *face_ptr,
                                   int *face_nodes, int *owner, int *neighbour, int *cell_face_ptr,
                                   int *cell_faces);   /* GlobalConnectivity, O(N^2) as written */
void   om_advance_time(om *m, double dt_next);  /* time-step prologue (MainProgram.for:184-245) */
double om_adaptive_dt(om *m, double courant, double min_factor, double max_factor);  /* AdaptiveTimeStep, laminar */
void   om_get_time(om *m, double t[4], int *ndt);        /* time, dt, dtOld, dtOldOld; ndt */
void   om_set_time(om *m, const double t[4], int ndt);
void   om_turb_production(om *m);              /* strain rate + k-epsilon production (into "prod") */

/* leaf operators (exposed for per-kernel parity tests) */
void   om_gradient(om *m, int var, int method, int niter,
                   const double *phi, const double *bphi,
                   double *g, double *bg);     /* g: 3*N (x,y,z blocks), bg: 3*B */
void   om_assemble_momentum(om *m, int comp);  /* everything of SolveMomentum* but the solve */
void   om_assemble_continuity(om *m);          /* SolveContinuity up to the p' solve */
void   om_correct_continuity(om *m);           /* SolveContinuity after the p' solve */
void   om_solve_equation(om *m, int nf, double *fi, double rrf, int itmax, int solver);
int    om_bicgstab(om *m, int maxit, double tol); /* returns iterations */
int    om_gmres(om *m);                            /* returns Arnoldi steps */
void   om_calc_residuals(om *m, int nf, const double *fi);

/* geometric-element agglomeration multigrid */
int    om_mg_setup(om *m);                     /* returns number of levels */
int    om_mg_level_size(om *m, int level);
const int *om_mg_parents(om *m, int level);    /* level l cell -> level l+1 parent (0-based) */
int    om_mg_width(om *m, int level);          /* ELL width of a level */
int    om_set_threads(int n);                  /* AxOMP threads (n <= 0: keep); returns the count */
/* AssembleAgglomeratedLHS of the current system up to `level` >= 1, copied out:
 * ac [n], n_nbr [n], nbr and anb [w*n slot-major] of that level */
int    om_mg_coarse_matrix(om *m, int level, double *ac, int *n_nbr, int *nbr, double *anb);

#ifdef __cplusplus
}
#endif
#endif
