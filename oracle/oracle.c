/*
 * oracle.c -- sequential FP64 restatement of the reference SIMPLE loop.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline); the
 * product never links it.  PARITY UNPINNED: there is no Fortran compiler in
 * this image and the reference ships no golden vectors, so the restatement is
 * pinned only by analytic invariants (tests/test_oracle.py).
 *
 * Reference paths are relative to the reference project root.  Loop order,
 * operation order and the reference's single-precision literals are kept:
 *   - `-2./3.` (Diffusion/AssembleBulkViscosity.for:36) is REAL(4): OM_M23.
 *   - `1.e-9`  (Convection/AssembleHRSchemeCorrection.for:70,92): OM_EPS9.
 * Quirks kept on purpose:
 *   - CorrectGradientAtOulet and CorrectPressureGradientAtSymmetryBoundary
 *     read nz=BFaceAreanz(i,i) (set index twice, CorrectGradients.for:222,272).
 *   - BICGSTAB_OMP keeps its solution vector x between calls and between
 *     variables (matrixSolverOMP.f90:560,607); x starts at 0 here.
 *   - BICGSTAB_OMP ignores rrF/itmax (fixed 100 iterations, 1e-5,
 *     matrixSolverOMP.f90:607) -- cfg.krylov_maxit/krylov_tol carry them.
 */
#include "oracle.h"
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#define OM_M23   ((double)(-2.0f / 3.0f))
#define OM_EPS9  ((double)1.e-9f)
#define OM_TINY  1.0e-15              /* Constants1.F90: tiny=1.d-15 */
#define OM_TWOTHIRD ((double)(2.0f / 3.0f))   /* Constants1.F90:12 TwoThird, a REAL(4) literal */
/* 'specifiedvelocity' and 'specifiedmassflowrate' inlets take the same
 * momentum, p' and k-epsilon treatment (AssembleIsotropicDiffusion.for:254-300,
 * AssembleConvection.for:260-300, AssemblePressureCorrectionFluxes.for:545-575) */
#define OM_INLET(t) ((t) == FS_BC_INLET_VEL || (t) == FS_BC_INLET_MASS || (t) == FS_BC_INLET_SP || (t) == FS_BC_INLET_STAG)
/* static- and stagnation-pressure inlets: the same loop bodies (incompressible)
 * but for the boundary pressure and the p' coefficients */
#define OM_P_INLET(t) ((t) == FS_BC_INLET_SP || (t) == FS_BC_INLET_STAG)
/* static pressure specified: Rhie-Chow boundary flux, p'_b = 0 (AssembleMdotUsingRhieChow.for:1441-1598, 2105-2283) */
#define OM_PRESSURE(t) ((t) == FS_BC_OUTLET_SP || (t) == FS_BC_INLET_SP || (t) == FS_BC_OUTLET_ASP || \
                        (t) == FS_BC_OUTLET_RES || (t) == FS_BC_INLET_STAG)
/* 'specifiedstaticpressure' and 'specifiedaveragestaticpressure' outlets share
 * every loop body but CorrectPressure's (AssembleMdotUsingRhieChow.for:1441-1812,
 * AssemblePressureCorrectionFluxes.for:244-400, CorrectMdotandVelocity.for:264-320, ...) */
#define OM_SP_OUTLET(t) ((t) == FS_BC_OUTLET_SP || (t) == FS_BC_OUTLET_ASP || (t) == FS_BC_OUTLET_RES)
/* Dirichlet momentum diffusion and plain upwind convection at the face
 * (AssembleIsotropicDiffusion.for:254-300, 507-525; AssembleConvection.for:260-330, 505-520) */
#define OM_GIVEN_FLOW(t) (OM_INLET(t) || (t) == FS_BC_OUTLET_MASS)
/* the direction of the inlet velocity is given (xVeldirection...) */
#define OM_DIRECTED(t) ((t) == FS_BC_INLET_MASS || OM_P_INLET(t))

struct om {
  fs_case cfg;
  int N, F, B, NS, W, nnodes;
  int nIter;
  /* polyMesh input copy */
  double *pts; int *face_ptr, *face_nodes;
  /* connectivity (ReadFoamMesh.f90:277-660) */
  int *if_own, *if_nbr;     /* F */
  int *bf_own, *bf_set;     /* B */
  int *bset_start, *bset_n; /* NS */
  int *ncf;                 /* NumbOfElementFaces [N] */
  int *cf;                  /* NGlobalEFaces [j*N+i], global face id, -1 unused */
  int *cn;                  /* ElementNeighbor [j*N+i], -1 = boundary/unused */
  int *own_slot, *nbr_slot; /* iOwnerNeighbor, iNeighborOwner [F] */
  int *cnode_ptr, *cnodes;  /* ListOfElementNodes (CSR) */
  /* interior geometry (ProcessGeometryRoutine.for) */
  double *fcx, *fcy, *fcz, *fa, *sx, *sy, *sz, *nx, *ny, *nz;
  double *dcfx, *dcfy, *dcfz, *dcf, *ex, *ey, *ez, *gf;
  double *Ex, *Ey, *Ez, *E, *gdiff, *Tx, *Ty, *Tz, *T;
  /* boundary geometry (linear boundary index) */
  double *bfcx, *bfcy, *bfcz, *bfa, *bsx, *bsy, *bsz, *bnx, *bny, *bnz;
  double *bdx, *bdy, *bdz, *bd, *bex, *bey, *bez;
  double *bEx, *bEy, *bEz, *bE, *bgdiff, *bTx, *bTy, *bTz, *bT;
  double *vol, *xc, *yc, *zc;
  /* boundary conditions */
  int *btype;
  /* state */
  double *u, *v, *w, *p, *pc, *mdot;
  double *bu, *bv, *bw, *bp, *bpc, *bmdot;
  double *ug, *vg, *wg, *pg, *pcg;          /* 3N each */
  double *bug, *bvg, *bwg, *bpg, *bpcg;     /* 3B each */
  double *ugf, *vgf, *wgf, *pgf;            /* 3F face gradients */
  double *du1, *dv1, *dw1, *du2, *dv2, *dw2;
  double *us, *vs, *ws;                     /* u* */
  double *gstar;                            /* 3N SaveGradient */
  /* assembly */
  double *fcf, *fff, *fvf, *ftf;            /* FluxCf/Ff/Vf/Tf [F+B] */
  double *fce, *fte;                        /* FluxCE, FluxTE [N] */
  double *effdiv;
  double *ac, *anb, *bc, *dphi;
  /* residuals (Residuals1.F90), NF 1..9 */
  double rabs[9], rmax[9], rrms[9], rscl[9];
  double overall_imbalance; int imax_imbalance;
  int lin_iters[9];
  /* outlets (FlowInOut1.F90) */
  double mdot_in, *mdot1, *mdot_out;        /* mdotIn, mdot1(NS), mdotOut(NS) */
  /* k-epsilon (Variables1, PhysicalProperties1, Turbulence1, WallDistance1) */
  double *tke, *ted, *mut, *btke, *bted, *bmut;
  double *tkeg, *tedg, *btkeg, *btedg, *tkegf, *tedgf;
  double *edif, *bedif;                     /* eDiffCoefficient, BeDiffCoefficient */
  double *prod, *bprod;                     /* TurbulenceProduction, BTurbulenceProduction */
  double *s11, *s12, *s13, *s22, *s23, *s33;
  double *rhok, *brhok, *drk, *bdrk;        /* MinusTwoThirdsRhoK */
  double *wdist; int *itau;                 /* WallDistance, iTau (boundary index) */
  double *bdir;                             /* xVeldirection.. of 'specifiedmassflowrate' inlets [3B] */
  double *utau, *yplus, *uplus, *dupdyp, *tauw, *wallvisc;   /* per wall face */
  /* BICGSTAB_OMP persistent storage (SparseMatricesVariables) */
  int csr_built; long *csr_ptr; int *csr_j; int *csr_slot; double *csr_val;
  double *kx, *kr, *kb;
  /* 'specifiedstagnationpressure' p0 per boundary face (BStagnationPressure);
   * 'specifiedresistance' geoDiffB per face and geoDiffSum per patch (ArteryResistance1) */
  double *bp0, *bgd, gdsum[FS_MAX_PATCHES];
  /* ILU (Variables2 dc, rc) */
  double *ilu_dc, *ilu_rc;
  /* multigrid */
  int mg_nlev; int mg_built; void *mgt;
  /* temperature (Variables1 Temperature, BTemperature, TempGrad*; BStagnationTemperature;
   * the thermal boundary set of each face) */
  double *tmp, *btmp, *tmpg, *btmpg, *tmpgf, *bt0; int *tbc;
  /* unsteady (Variables1 ...Old and ...OldOld, Transient1 dt, dtOld, dtOldOld; time, ndt) */
  double *old, *oldold, *bold;
  double dt, dto, dtoo, time;
  int ndt, tscheme;                         /* tscheme: the TransientScheme in effect */
};

#define OM_NLEVELS 7                  /* time levels: u v w p k epsilon T */
static double *dz_(long n) { return (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }
static void om_momentum_wall_functions(om *m);   /* oracle_turb.inc */
static int *iz_(long n) { return (int *)calloc((size_t)(n > 0 ? n : 1), sizeof(int)); }
#include "oracle_transient.inc"
#include "oracle_neutral.inc"

/* ===================================================================== */
/*  Connectivity: Readit (GridAndGeometry/ReadFoamMesh.f90:277-660)       */
/* ===================================================================== */
static void om_connectivity(om *m, const fs_mesh_in *mi)
{
  int nf = mi->n_faces, F = mi->n_internal, B = nf - F, N = -1;
  /* NumberOfElements = max owner/neighbour (ReadFoamMesh.f90:283-286) */
  for (int i = 0; i < nf; i++) {
    if (mi->owner[i] + 1 > N) N = mi->owner[i] + 1;
    if (i < F && mi->neighbour[i] + 1 > N) N = mi->neighbour[i] + 1;
  }
  m->N = N; m->F = F; m->B = B; m->NS = mi->n_patches; m->nnodes = mi->n_nodes;
  m->if_own = iz_(F); m->if_nbr = iz_(F);
  for (int i = 0; i < F; i++) { m->if_own[i] = mi->owner[i]; m->if_nbr[i] = mi->neighbour[i]; }
  m->bf_own = iz_(B); m->bf_set = iz_(B);
  m->bset_start = iz_(m->NS); m->bset_n = iz_(m->NS);
  int k = 0;
  for (int s = 0; s < m->NS; s++) {
    m->bset_start[s] = k; m->bset_n[s] = mi->patch_size[s];
    for (int j = 0; j < mi->patch_size[s]; j++, k++) {
      m->bf_own[k] = mi->owner[F + k]; m->bf_set[k] = s;
    }
  }
  /* NumbOfElementFaces (ReadFoamMesh.f90:311-322); a neutral-file mesh
   * gives its element-local face lists (NGlobalEFaces of GlobalConnectivity) */
  m->ncf = iz_(N);
  if (mi->cell_face_ptr) for (int i = 0; i < N; i++) m->ncf[i] = mi->cell_face_ptr[i + 1] - mi->cell_face_ptr[i];
  else {
    for (int i = 0; i < F; i++) { m->ncf[mi->owner[i]]++; m->ncf[mi->neighbour[i]]++; }
    for (int i = F; i < nf; i++) m->ncf[mi->owner[i]]++;
  }
  int W = -1;
  for (int i = 0; i < N; i++) if (m->ncf[i] > W) W = m->ncf[i];
  m->W = W;
  /* NGlobalEFaces: interior faces in file order, then boundary faces (:326-342) */
  m->cf = iz_((long)W * N); m->cn = iz_((long)W * N);
  for (long q = 0; q < (long)W * N; q++) { m->cf[q] = -1; m->cn[q] = -1; }
  if (mi->cell_face_ptr) {
    for (int i = 0; i < N; i++)
      for (int j = 0; j < m->ncf[i]; j++) m->cf[(long)j * N + i] = mi->cell_faces[mi->cell_face_ptr[i] + j];
  } else {
    int *cnt = iz_(N);
    for (int i = 0; i < F; i++) {
      int o = mi->owner[i], nb = mi->neighbour[i];
      m->cf[(long)cnt[o] * N + o] = i; cnt[o]++;
      m->cf[(long)cnt[nb] * N + nb] = i; cnt[nb]++;
    }
    for (int i = F; i < nf; i++) { int o = mi->owner[i]; m->cf[(long)cnt[o] * N + o] = i; cnt[o]++; }
    free(cnt);
  }
  /* iOwnerNeighbor / iNeighborOwner / ElementNeighbor (:597-635) */
  m->own_slot = iz_(F); m->nbr_slot = iz_(F);
  for (int i = 0; i < F; i++) {
    int e = m->if_own[i], nb = m->if_nbr[i];
    for (int j = 0; j < m->ncf[e]; j++)
      if (m->cf[(long)j * N + e] == i) { m->own_slot[i] = j; m->cn[(long)j * N + e] = nb; break; }
    for (int j = 0; j < m->ncf[nb]; j++)
      if (m->cf[(long)j * N + nb] == i) { m->nbr_slot[i] = j; m->cn[(long)j * N + nb] = e; break; }
  }
  /* ListOfElementNodes, second (ordered) fill (:430-458): nodes of the first
   * face in face order, then new nodes of later faces.  The first pass
   * (:380-410) only counts unique nodes, which the second pass reproduces. */
  m->cnode_ptr = iz_(N + 1);
  if (mi->cell_node_ptr) {   /* ListOfElementNodes as read from a neutral file */
    memcpy(m->cnode_ptr, mi->cell_node_ptr, sizeof(int) * (N + 1));
    m->cnodes = iz_(mi->cell_node_ptr[N]);
    memcpy(m->cnodes, mi->cell_nodes, sizeof(int) * mi->cell_node_ptr[N]);
    return;
  }
  int cap = 0;
  for (int i = 0; i < N; i++) {
    int c = 0;
    for (int j = 0; j < m->ncf[i]; j++) { int f = m->cf[(long)j * N + i]; c += mi->face_ptr[f + 1] - mi->face_ptr[f]; }
    cap += c;
  }
  m->cnodes = iz_(cap);
  int pos = 0;
  for (int i = 0; i < N; i++) {
    m->cnode_ptr[i] = pos;
    int start = pos;
    for (int j = 0; j < m->ncf[i]; j++) {
      int f = m->cf[(long)j * N + i];
      for (int q = mi->face_ptr[f]; q < mi->face_ptr[f + 1]; q++) {
        int nd = mi->face_nodes[q], seen = 0;
        if (j > 0) for (int r = start; r < pos; r++) if (m->cnodes[r] == nd) { seen = 1; break; }
        if (!seen) m->cnodes[pos++] = nd;
      }
    }
  }
  m->cnode_ptr[N] = pos;
}

/* ===================================================================== */
/*  Geometry: ProcessGeometry (GridAndGeometry/ProcessGeometryRoutine.for) */
/* ===================================================================== */
static void face_area_centroid(const om *m, int f, double *ax, double *ay, double *az,
                               double *a, double *cx, double *cy, double *cz)
{
  const double *P = m->pts;
  int q0 = m->face_ptr[f], q1 = m->face_ptr[f + 1], n = q1 - q0;
  double centerx = 0., centery = 0., centerz = 0.;
  for (int q = q0; q < q1; q++) { int j1 = m->face_nodes[q]; centerx += P[3*j1]; centery += P[3*j1+1]; centerz += P[3*j1+2]; }
  centerx /= n; centery /= n; centerz /= n;
  double Sx = 0, Sy = 0, Sz = 0, A = 0, Cx = 0, Cy = 0, Cz = 0;
  for (int q = q0; q < q1; q++) {
    int j2 = m->face_nodes[q], j3 = (q < q1 - 1) ? m->face_nodes[q + 1] : m->face_nodes[q0];
    double x2 = P[3*j2], y2 = P[3*j2+1], z2 = P[3*j2+2];
    double x3 = P[3*j3], y3 = P[3*j3+1], z3 = P[3*j3+2];
    /* ProcessGeometryRoutine.for:84-93 */
    double sx1 = 0.5 * ((y2 - centery) * (z3 - centerz) - (y3 - centery) * (z2 - centerz));
    double sy1 = -0.5 * ((x2 - centerx) * (z3 - centerz) - (x3 - centerx) * (z2 - centerz));
    double sz1 = 0.5 * ((x2 - centerx) * (y3 - centery) - (x3 - centerx) * (y2 - centery));
    double area1 = sqrt(sx1 * sx1 + sy1 * sy1 + sz1 * sz1);
    double x1 = (centerx + x2 + x3) / 3., y1 = (centery + y2 + y3) / 3., z1 = (centerz + z2 + z3) / 3.;
    Sx += sx1; Sy += sy1; Sz += sz1; A += area1;
    Cx += x1 * area1; Cy += y1 * area1; Cz += z1 * area1;
  }
  *ax = Sx; *ay = Sy; *az = Sz; *a = A; *cx = Cx / A; *cy = Cy / A; *cz = Cz / A;
}

static void om_geometry(om *m)
{
  int N = m->N, F = m->F, B = m->B;
  double **fa_[] = {&m->fcx,&m->fcy,&m->fcz,&m->fa,&m->sx,&m->sy,&m->sz,&m->nx,&m->ny,&m->nz,
                    &m->dcfx,&m->dcfy,&m->dcfz,&m->dcf,&m->ex,&m->ey,&m->ez,&m->gf,
                    &m->Ex,&m->Ey,&m->Ez,&m->E,&m->gdiff,&m->Tx,&m->Ty,&m->Tz,&m->T};
  for (unsigned q = 0; q < sizeof(fa_)/sizeof(fa_[0]); q++) *fa_[q] = dz_(F);
  double **ba_[] = {&m->bfcx,&m->bfcy,&m->bfcz,&m->bfa,&m->bsx,&m->bsy,&m->bsz,&m->bnx,&m->bny,&m->bnz,
                    &m->bdx,&m->bdy,&m->bdz,&m->bd,&m->bex,&m->bey,&m->bez,
                    &m->bEx,&m->bEy,&m->bEz,&m->bE,&m->bgdiff,&m->bTx,&m->bTy,&m->bTz,&m->bT};
  for (unsigned q = 0; q < sizeof(ba_)/sizeof(ba_[0]); q++) *ba_[q] = dz_(B);
  m->vol = dz_(N); m->xc = dz_(N); m->yc = dz_(N); m->zc = dz_(N);
  /* interior faces (:61-104) */
  for (int i = 0; i < F; i++)
    face_area_centroid(m, i, &m->sx[i], &m->sy[i], &m->sz[i], &m->fa[i], &m->fcx[i], &m->fcy[i], &m->fcz[i]);
  /* boundary faces (:129-183) */
  for (int b = 0; b < B; b++)
    face_area_centroid(m, F + b, &m->bsx[b], &m->bsy[b], &m->bsz[b], &m->bfa[b], &m->bfcx[b], &m->bfcy[b], &m->bfcz[b]);
  /* element volume and centroid (:186-237) */
  const double *P = m->pts;
  for (int i = 0; i < N; i++) {
    double x1 = 0, y1 = 0, z1 = 0;
    int nn = m->cnode_ptr[i + 1] - m->cnode_ptr[i];
    for (int q = m->cnode_ptr[i]; q < m->cnode_ptr[i + 1]; q++) { int k = m->cnodes[q]; x1 += P[3*k]; y1 += P[3*k+1]; z1 += P[3*k+2]; }
    x1 /= nn; y1 /= nn; z1 /= nn;
    double V = 0., px = 0., py = 0., pz = 0.;
    for (int j = 0; j < m->ncf[i]; j++) {
      int f = m->cf[(long)j * N + i];
      double Abx, Aby, Abz, x2, y2, z2;
      if (f >= F) { int b = f - F; Abx = m->bsx[b]; Aby = m->bsy[b]; Abz = m->bsz[b]; x2 = m->bfcx[b]; y2 = m->bfcy[b]; z2 = m->bfcz[b]; }
      else { Abx = m->sx[f]; Aby = m->sy[f]; Abz = m->sz[f]; x2 = m->fcx[f]; y2 = m->fcy[f]; z2 = m->fcz[f]; }
      double dx = x2 - x1, dy = y2 - y1, dz = z2 - z1;
      double xcp = 0.75 * x2 + 0.25 * x1, ycp = 0.75 * y2 + 0.25 * y1, zcp = 0.75 * z2 + 0.25 * z1;
      double vt = fabs(Abx * dx + Aby * dy + Abz * dz) / 3.;
      V += vt; px += xcp * vt; py += ycp * vt; pz += zcp * vt;
    }
    m->vol[i] = V; m->xc[i] = px / V; m->yc[i] = py / V; m->zc[i] = pz / V;
  }
  /* CF vectors (:247-258), orientation + unit normal (:260-271), g (:273-282) */
  for (int k = 0; k < F; k++) {
    int i = m->if_own[k], j = m->if_nbr[k];
    m->dcfx[k] = m->xc[j] - m->xc[i]; m->dcfy[k] = m->yc[j] - m->yc[i]; m->dcfz[k] = m->zc[j] - m->zc[i];
    m->dcf[k] = sqrt(m->dcfx[k] * m->dcfx[k] + m->dcfy[k] * m->dcfy[k] + m->dcfz[k] * m->dcfz[k]);
    m->ex[k] = m->dcfx[k] / m->dcf[k]; m->ey[k] = m->dcfy[k] / m->dcf[k]; m->ez[k] = m->dcfz[k] / m->dcf[k];
  }
  for (int k = 0; k < F; k++) {
    double dp = m->dcfx[k] * m->sx[k] + m->dcfy[k] * m->sy[k] + m->dcfz[k] * m->sz[k];
    if (dp < 0.) { m->sx[k] = -m->sx[k]; m->sy[k] = -m->sy[k]; m->sz[k] = -m->sz[k]; }
    m->nx[k] = m->sx[k] / m->fa[k]; m->ny[k] = m->sy[k] / m->fa[k]; m->nz[k] = m->sz[k] / m->fa[k];
  }
  for (int k = 0; k < F; k++) {
    int i = m->if_own[k], j = m->if_nbr[k];
    double d1 = sqrt((m->fcx[k]-m->xc[i])*(m->fcx[k]-m->xc[i]) + (m->fcy[k]-m->yc[i])*(m->fcy[k]-m->yc[i]) + (m->fcz[k]-m->zc[i])*(m->fcz[k]-m->zc[i]));
    double d2 = sqrt((m->fcx[k]-m->xc[j])*(m->fcx[k]-m->xc[j]) + (m->fcy[k]-m->yc[j])*(m->fcy[k]-m->yc[j]) + (m->fcz[k]-m->zc[j])*(m->fcz[k]-m->zc[j]));
    m->gf[k] = d2 / (d1 + d2);
  }
  /* boundary distance, orientation, unit normal (:284-309) */
  for (int b = 0; b < B; b++) {
    int n = m->bf_own[b];
    m->bdx[b] = m->bfcx[b] - m->xc[n]; m->bdy[b] = m->bfcy[b] - m->yc[n]; m->bdz[b] = m->bfcz[b] - m->zc[n];
    m->bd[b] = sqrt(m->bdx[b] * m->bdx[b] + m->bdy[b] * m->bdy[b] + m->bdz[b] * m->bdz[b]);
    m->bex[b] = m->bdx[b] / m->bd[b]; m->bey[b] = m->bdy[b] / m->bd[b]; m->bez[b] = m->bdz[b] / m->bd[b];
    double dp = m->bdx[b] * m->bsx[b] + m->bdy[b] * m->bsy[b] + m->bdz[b] * m->bsz[b];
    if (dp < 0.) { m->bsx[b] = -m->bsx[b]; m->bsy[b] = -m->bsy[b]; m->bsz[b] = -m->bsz[b]; }
    m->bnx[b] = m->bsx[b] / m->bfa[b]; m->bny[b] = m->bsy[b] / m->bfa[b]; m->bnz[b] = m->bsz[b] / m->bfa[b];
  }
  /* E/T decomposition (:313-366 interior, :379-444 boundary) */
  int msd = m->cfg.method_decompose_s;
  for (int k = 0; k < F; k++) {
    if (msd == 1) {
      double dp = m->ex[k] * m->sx[k] + m->ey[k] * m->sy[k] + m->ez[k] * m->sz[k];
      m->Ex[k] = dp * m->ex[k]; m->Ey[k] = dp * m->ey[k]; m->Ez[k] = dp * m->ez[k]; m->E[k] = fabs(dp);
    } else if (msd == 2) {
      m->Ex[k] = m->fa[k] * m->ex[k]; m->Ey[k] = m->fa[k] * m->ey[k]; m->Ez[k] = m->fa[k] * m->ez[k]; m->E[k] = m->fa[k];
    } else {
      double dp = m->ex[k] * m->sx[k] + m->ey[k] * m->sy[k] + m->ez[k] * m->sz[k];
      double a2 = m->fa[k] * m->fa[k];
      m->Ex[k] = (a2 / dp) * m->ex[k]; m->Ey[k] = (a2 / dp) * m->ey[k]; m->Ez[k] = (a2 / dp) * m->ez[k];
      m->E[k] = sqrt(m->Ex[k] * m->Ex[k] + m->Ey[k] * m->Ey[k] + m->Ez[k] * m->Ez[k]);
    }
    m->gdiff[k] = m->E[k] / m->dcf[k];
    m->Tx[k] = m->sx[k] - m->Ex[k]; m->Ty[k] = m->sy[k] - m->Ey[k]; m->Tz[k] = m->sz[k] - m->Ez[k];
    m->T[k] = sqrt(m->Tx[k] * m->Tx[k] + m->Ty[k] * m->Ty[k] + m->Tz[k] * m->Tz[k]);
  }
  for (int b = 0; b < B; b++) {
    if (msd == 1) {
      double dp = m->bex[b] * m->bsx[b] + m->bey[b] * m->bsy[b] + m->bez[b] * m->bsz[b];
      m->bEx[b] = dp * m->bex[b]; m->bEy[b] = dp * m->bey[b]; m->bEz[b] = dp * m->bez[b]; m->bE[b] = fabs(dp);
    } else if (msd == 2) {
      m->bEx[b] = m->bfa[b] * m->bex[b]; m->bEy[b] = m->bfa[b] * m->bey[b]; m->bEz[b] = m->bfa[b] * m->bez[b]; m->bE[b] = m->bfa[b];
    } else {
      double dp = m->bex[b] * m->bsx[b] + m->bey[b] * m->bsy[b] + m->bez[b] * m->bsz[b];
      double a2 = m->bfa[b] * m->bfa[b];
      m->bEx[b] = (a2 / dp) * m->bex[b]; m->bEy[b] = (a2 / dp) * m->bey[b]; m->bEz[b] = (a2 / dp) * m->bez[b];
      m->bE[b] = sqrt(m->bEx[b] * m->bEx[b] + m->bEy[b] * m->bEy[b] + m->bEz[b] * m->bEz[b]);
    }
    m->bgdiff[b] = m->bE[b] / m->bd[b];
    m->bTx[b] = m->bsx[b] - m->bEx[b]; m->bTy[b] = m->bsy[b] - m->bEy[b]; m->bTz[b] = m->bsz[b] - m->bEz[b];
    m->bT[b] = sqrt(m->bTx[b] * m->bTx[b] + m->bTy[b] * m->bTy[b] + m->bTz[b] * m->bTz[b]);
  }
}

/* ===================================================================== */
/*  Gradients (GradientFiles/)                                            */
/* ===================================================================== */
/* StandardGreenGauss (StandardGreenGaussGradient.for:3) and
 * StandardGreenGaussFaceCorrection1 (StandardGreenGaussCorrection1Gradient.for:3) */
static void om_gg(om *m, int method, int niter, const double *phi, const double *bphi,
                  double *gx, double *gy, double *gz, double *bgx, double *bgy, double *bgz)
{
  int N = m->N, F = m->F, B = m->B;
  for (int i = 0; i < N; i++) { gx[i] = 0.; gy[i] = 0.; gz[i] = 0.; }
  for (int b = 0; b < B; b++) { bgx[b] = 0.; bgy[b] = 0.; bgz[b] = 0.; }
  double *fip = dz_(F);
  for (int k = 0; k < F; k++) {
    int j = m->if_own[k], kk = m->if_nbr[k];
    fip[k] = phi[j] * m->gf[k] + phi[kk] * (1. - m->gf[k]);
    double fx = fip[k] * m->sx[k], fy = fip[k] * m->sy[k], fz = fip[k] * m->sz[k];
    gx[j] += fx; gy[j] += fy; gz[j] += fz;
    gx[kk] -= fx; gy[kk] -= fy; gz[kk] -= fz;
  }
  for (int b = 0; b < B; b++) {
    int k = m->bf_own[b];
    gx[k] += bphi[b] * m->bsx[b]; gy[k] += bphi[b] * m->bsy[b]; gz[k] += bphi[b] * m->bsz[b];
  }
  for (int i = 0; i < N; i++) { gx[i] /= m->vol[i]; gy[i] /= m->vol[i]; gz[i] /= m->vol[i]; }
  if (method == 2) {
    double *fx_ = dz_(N), *fy_ = dz_(N), *fz_ = dz_(N);
    for (int it = 0; it < niter; it++) {
      memset(fx_, 0, sizeof(double) * N); memset(fy_, 0, sizeof(double) * N); memset(fz_, 0, sizeof(double) * N);
      for (int k = 0; k < F; k++) {
        int j = m->if_own[k], kk = m->if_nbr[k];
        /* StandardGreenGaussCorrection1Gradient.for:113-130 */
        double eDOTn = m->Ex[k] * m->nx[k] + m->Ey[k] * m->ny[k] + m->Ez[k] * m->nz[k];
        double rfn = (m->fcx[k] - m->xc[j]) * m->nx[k] + (m->fcy[k] - m->yc[j]) * m->ny[k] + (m->fcz[k] - m->zc[j]) * m->nz[k];
        double xfp = m->xc[j] + (rfn / eDOTn) * m->Ex[k];
        double yfp = m->yc[j] + (rfn / eDOTn) * m->Ey[k];
        double zfp = m->zc[j] + (rfn / eDOTn) * m->Ez[k];
        double g = m->gf[k];
        double cx = gx[j] * g + gx[kk] * (1. - g); cx = cx * (m->fcx[k] - xfp);
        double cy = gy[j] * g + gy[kk] * (1. - g); cy = cy * (m->fcy[k] - yfp);
        double cz = gz[j] * g + gz[kk] * (1. - g); cz = cz * (m->fcz[k] - zfp);
        double phif = fip[k] + cx + cy + cz;
        double sxp = phif * m->sx[k], syp = phif * m->sy[k], szp = phif * m->sz[k];
        fx_[j] += sxp; fy_[j] += syp; fz_[j] += szp;
        fx_[kk] -= sxp; fy_[kk] -= syp; fz_[kk] -= szp;
      }
      for (int b = 0; b < B; b++) {
        int k = m->bf_own[b];
        fx_[k] += bphi[b] * m->bsx[b]; fy_[k] += bphi[b] * m->bsy[b]; fz_[k] += bphi[b] * m->bsz[b];
      }
      for (int i = 0; i < N; i++) { gx[i] = fx_[i] / m->vol[i]; gy[i] = fy_[i] / m->vol[i]; gz[i] = fz_[i] / m->vol[i]; }
    }
    free(fx_); free(fy_); free(fz_);
  }
  free(fip);
  for (int b = 0; b < B; b++) { int k = m->bf_own[b]; bgx[b] = gx[k]; bgy[b] = gy[k]; bgz[b] = gz[k]; }
}

/* tangential projection used by CorrectGradientAtOulet / symmetry / walls */
static void tproj(double nx, double ny, double nz, double gx, double gy, double gz,
                  double *ox, double *oy, double *oz, int wall_form)
{
  if (wall_form) { /* CorrectGradients.for:34-39 */
    *ox = (1 - nx * nx) * gx - nx * ny * gy - nx * nz * gz;
    *oy = (1 - ny * ny) * gy - ny * nx * gx - ny * nz * gz;
    *oz = (1 - nz * nz) * gz - nz * nx * gx - nz * ny * gy;
  } else {         /* CorrectGradients.for:224-229 */
    *ox = gx * (1. - nx * nx) - gy * nx * ny - gz * nx * nz;
    *oy = gy * (1. - ny * ny) - gx * ny * nx - gz * ny * nz;
    *oz = gz * (1. - nz * nz) - gx * nz * nx - gy * nz * ny;
  }
}

/* BFaceAreanz(i,i) of the reference's (set,face) array, 0-based set s */
static double nz_ii(const om *m, int s)
{
  if (s < m->bset_n[s]) return m->bnz[m->bset_start[s] + s];
  return 0.;
}

/* Gradient (CalculateGradients.for:3-272) */
void om_gradient(om *m, int var, int method, int niter, const double *phi, const double *bphi,
                 double *g, double *bg)
{
  int N = m->N, B = m->B;
  double *gx = g, *gy = g + N, *gz = g + 2 * (long)N;
  double *bgx = bg, *bgy = bg + B, *bgz = bg + 2 * (long)B;
  memcpy(m->gstar, g, sizeof(double) * 3 * (size_t)N);    /* SaveGradient */
  om_gg(m, method, niter, phi, bphi, gx, gy, gz, bgx, bgy, bgz);
  /* RelaxGradient: all LrelaxGradient* are .false. (User0.F90:164-179) -> return */
  /* CorrectGradientAtOulet for velocities (CorrectGradients.for:188-238) */
  if (var == FS_VAR_U || var == FS_VAR_V || var == FS_VAR_W) {
    for (int b = 0; b < B; b++) if (m->btype[b] == FS_BC_OUTLET_FD || OM_SP_OUTLET(m->btype[b])) {
      int k = m->bf_own[b], s = m->bf_set[b];
      tproj(m->bnx[b], m->bny[b], nz_ii(m, s), gx[k], gy[k], gz[k], &bgx[b], &bgy[b], &bgz[b], 0);
    }
  }
  if (var == FS_VAR_P || var == FS_VAR_RHOK) {   /* 'press' and 'rhok' (CalculateGradients.for:266-271) */
    /* CorrectPressureGradientAtSymmetryBoundary (CorrectGradients.for:244-288) */
    for (int b = 0; b < B; b++) if (m->btype[b] == FS_BC_SYMMETRY) {
      int k = m->bf_own[b], s = m->bf_set[b];
      tproj(m->bnx[b], m->bny[b], nz_ii(m, s), gx[k], gy[k], gz[k], &bgx[b], &bgy[b], &bgz[b], 0);
    }
    /* CorrectPresureGradientAtWalls (CorrectGradients.for:3-62): slip then noslip */
    for (int pass = 0; pass < 2; pass++)
      for (int b = 0; b < B; b++) {
        int t = m->btype[b];
        if ((pass == 0 && t == FS_BC_WALL_SLIP) || (pass == 1 && t == FS_BC_WALL_NOSLIP)) {
          int k = m->bf_own[b];
          tproj(m->bnx[b], m->bny[b], m->bnz[b], gx[k], gy[k], gz[k], &bgx[b], &bgy[b], &bgz[b], 1);
        }
      }
  }
}

/* InterpolateGradientToFace (Interpolation/InterpolateGradientFromElementToFace.for:3) */
static void om_interp_grad(om *m, int scheme, const double *phi, const double *g, double *gfc)
{
  int N = m->N, F = m->F;
  const double *gx = g, *gy = g + N, *gz = g + 2 * (long)N;
  double *fx = gfc, *fy = gfc + F, *fz = gfc + 2 * (long)F;
  for (int k = 0; k < F; k++) {
    int i = m->if_own[k], j = m->if_nbr[k];
    double g_;
    if (scheme == FS_GI_UPWIND) g_ = (m->mdot[k] > 0.) ? 1. : 0.;
    else if (scheme == FS_GI_DOWNWIND) g_ = (m->mdot[k] > 0.) ? 0. : 1.;
    else g_ = m->gf[k];
    fx[k] = g_ * gx[i] + (1. - g_) * gx[j];
    fy[k] = g_ * gy[i] + (1. - g_) * gy[j];
    fz[k] = g_ * gz[i] + (1. - g_) * gz[j];
    if (scheme == FS_GI_AVERAGECORRECTED) {
      double corr = (phi[j] - phi[i]) / m->dcf[k];
      corr = corr - (fx[k] * m->ex[k] + fy[k] * m->ey[k] + fz[k] * m->ez[k]);
      fx[k] = fx[k] + corr * m->ex[k]; fy[k] = fy[k] + corr * m->ey[k]; fz[k] = fz[k] + corr * m->ez[k];
    }
  }
}

/* InterpolateElementToFace 'average' (InterpolateFromElementToFace.for:3-31) */
static inline double avgf(const om *m, int k, const double *a)
{
  double g = m->gf[k];
  return g * a[m->if_own[k]] + (1. - g) * a[m->if_nbr[k]];
}

/* TVDLimiter (Convection/LimitersTVDType.for:4) */
static double tvd_psi(int s, double rf)
{
  double t;
  switch (s) {
  case FS_TVD_UPWIND: return 0.;
  case FS_TVD_DOWNWIND: return 2.;
  case FS_TVD_FROMM: return 0.5 * (1. + rf);
  case FS_TVD_SOU: return rf;
  case FS_TVD_CD: return 1.;
  case FS_TVD_QUICK: return (3. + rf) / 4.;
  case FS_TVD_SUPERBEE: t = fmin(1., 2. * rf); return fmax(fmax(0., t), fmin(2., rf));
  case FS_TVD_MINMOD: return fmax(0., fmin(1., rf));
  case FS_TVD_OSHER: return fmax(0., fmin(2., rf));
  case FS_TVD_VANLEER: return (rf + fabs(rf)) / (1. + fabs(rf));
  case FS_TVD_MUSCL: return fmax(0., fmin(fmin(2. * rf, 0.5 * (1. + rf)), 2.));
  case FS_TVD_SMART: return fmax(0., fmin(fmin(2. * rf, 0.75 * rf + 0.25), 4.));
  case FS_TVD_HQUICK: return 2. * (rf + fabs(rf)) / (rf + 3.);
  case FS_TVD_UMIST: return fmax(0., fmin(fmin(fmin(2. * rf, 0.25 + 0.75 * rf), 0.75 + 0.25 * rf), 2.));
  case FS_TVD_CHARM: return (rf <= 0.) ? 0. : rf * (3. * rf + 1.) / ((rf + 1.) * (rf + 1.));
  }
  return 0.;
}

/* ===================================================================== */
/*  Momentum (Momentum/SolveXMomentumEquation.for:4 and Y/Z)              */
/* ===================================================================== */
static void init_fluxes(om *m)   /* InitializeFluxes / InitializeCoefficients */
{
  long FB = (long)m->F + m->B;
  memset(m->fcf, 0, sizeof(double) * FB); memset(m->fff, 0, sizeof(double) * FB);
  memset(m->fvf, 0, sizeof(double) * FB); memset(m->ftf, 0, sizeof(double) * FB);
  memset(m->fce, 0, sizeof(double) * m->N); memset(m->fte, 0, sizeof(double) * m->N);
  memset(m->ac, 0, sizeof(double) * m->N); memset(m->bc, 0, sizeof(double) * m->N);
  memset(m->anb, 0, sizeof(double) * (size_t)m->N * m->W);
}

/* AssembleGlobalMatrixFaceFluxes / ElementFluxes (AssembleGolbalElementAndFaceFluxes.for:4-98) */
static void global_assembly(om *m)
{
  int N = m->N, F = m->F;
  for (int k = 0; k < F; k++) {
    int i = m->if_own[k], j = m->if_nbr[k], i1 = m->own_slot[k], j1 = m->nbr_slot[k];
    m->ac[i] += m->fcf[k]; m->anb[(long)i1 * N + i] += m->fff[k]; m->bc[i] -= m->ftf[k];
    m->ac[j] -= m->fff[k]; m->anb[(long)j1 * N + j] -= m->fcf[k]; m->bc[j] += m->ftf[k];
  }
  for (int b = 0; b < m->B; b++) {
    int k = m->bf_own[b];
    m->ac[k] += m->fcf[F + b]; m->bc[k] -= m->ftf[F + b];
  }
  for (int i = 0; i < N; i++) { m->ac[i] += m->fce[i]; m->bc[i] -= m->fte[i]; }
}

void om_assemble_momentum(om *m, int comp)
{
  int N = m->N, F = m->F, B = m->B;
  const fs_case *c = &m->cfg;
  double *fi = comp == 0 ? m->u : comp == 1 ? m->v : m->w;
  double *bfi = comp == 0 ? m->bu : comp == 1 ? m->bv : m->bw;
  double *fg = comp == 0 ? m->ug : comp == 1 ? m->vg : m->wg;
  double *bfg = comp == 0 ? m->bug : comp == 1 ? m->bvg : m->bwg;
  double *fgf = comp == 0 ? m->ugf : comp == 1 ? m->vgf : m->wgf;
  init_fluxes(m);
  if (comp == 0) {   /* gradients only in X (SolveXMomentumEquation.for:182-222) */
    om_gradient(m, FS_VAR_U, c->method_grad_mom, c->niter_grad_mom, m->u, m->bu, m->ug, m->bug);
    om_gradient(m, FS_VAR_V, c->method_grad_mom, c->niter_grad_mom, m->v, m->bv, m->vg, m->bvg);
    om_gradient(m, FS_VAR_W, c->method_grad_mom, c->niter_grad_mom, m->w, m->bw, m->wg, m->bwg);
    om_gradient(m, FS_VAR_P, c->method_grad_cont, c->niter_grad_cont, m->p, m->bp, m->pg, m->bpg);
    om_interp_grad(m, c->grad_interp_mom, m->u, m->ug, m->ugf);
    om_interp_grad(m, c->grad_interp_mom, m->v, m->vg, m->vgf);
    om_interp_grad(m, c->grad_interp_mom, m->w, m->wg, m->wgf);
    om_interp_grad(m, c->grad_interp_cont, m->p, m->pg, m->pgf);
  }
  const double *fgx = fgf, *fgy = fgf + F, *fgz = fgf + 2 * (long)F;
  if (!c->inviscid) {
    /* CalculateEffectiveDiffusionCoefficient('vel?') (ComputeEffectiveDiffusionCoefficient.for:24-48,
     * 580-596): mu (+ mu_t and the momentum wall functions when turbulent) */
    if (c->turbulence) {
      for (int i = 0; i < N; i++) m->edif[i] = c->mu + m->mut[i];
      for (int b = 0; b < B; b++) m->bedif[b] = c->mu + m->bmut[b];
      om_momentum_wall_functions(m);
    } else {
      for (int i = 0; i < N; i++) m->edif[i] = c->mu;
      for (int b = 0; b < B; b++) m->bedif[b] = c->mu;
    }
    /* AssembleDiffusionTerm interior (AssembleIsotropicDiffusion.for:99-117);
     * GamaFace = 'average' of eDiffCoefficient (InterpolateGamaFromCentroidToFace.for) */
    for (int k = 0; k < F; k++) {
      int i = m->if_own[k], j = m->if_nbr[k];
      double gamf = m->gf[k] * m->edif[i] + (1. - m->gf[k]) * m->edif[j];
      double fcl = gamf * m->gdiff[k], ffl = -gamf * m->gdiff[k];
      double fvl = -(gamf * (fgx[k] * m->Tx[k] + fgy[k] * m->Ty[k] + fgz[k] * m->Tz[k]));
      m->fcf[k] += fcl; m->fff[k] += ffl; m->fvf[k] += fvl;
      m->ftf[k] += fcl * fi[i] + ffl * fi[j] + fvl;
    }
    /* boundary faces (AssembleIsotropicDiffusion.for:123-627) */
    for (int b = 0; b < B; b++) {
      int i1 = m->bf_own[b], t = m->btype[b];
      long i4 = F + b;
      double gamf = m->bedif[b];
      if (t == FS_BC_WALL_NOSLIP) {
        double dN = m->bdx[b] * m->bnx[b] + m->bdy[b] * m->bny[b] + m->bdz[b] * m->bnz[b];
        double area = m->bfa[b], nx = m->bnx[b], ny = m->bny[b], nz = m->bnz[b];
        double fcl, fvl;
        if (comp == 0) {
          fcl = gamf * area * (1. - nx * nx) / dN;
          fvl = -((gamf * area / dN) * (bfi[b] * (1. - nx * nx) + (m->v[i1] - m->bv[b]) * nx * ny + (m->w[i1] - m->bw[b]) * nx * nz));
        } else if (comp == 1) {
          fcl = gamf * area * (1. - ny * ny) / dN;
          fvl = -((gamf * area / dN) * ((m->u[i1] - m->bu[b]) * nx * ny + bfi[b] * (1. - ny * ny) + (m->w[i1] - m->bw[b]) * nz * ny));
        } else {
          fcl = gamf * area * (1. - nz * nz) / dN;
          fvl = -((gamf * area / dN) * ((m->u[i1] - m->bu[b]) * nx * nz + (m->v[i1] - m->bv[b]) * ny * nz + bfi[b] * (1. - nz * nz)));
        }
        m->fcf[i4] += fcl; m->fvf[i4] += fvl;
        m->ftf[i4] += fcl * fi[i1] + 0. * bfi[b] + fvl;
      } else if (t == FS_BC_SYMMETRY) {
        double dN = m->bdx[b] * m->bnx[b] + m->bdy[b] * m->bny[b] + m->bdz[b] * m->bnz[b];
        double area = m->bfa[b], nx = m->bnx[b], ny = m->bny[b], nz = m->bnz[b];
        double fcl, fvl;
        if (comp == 0) { fcl = 2. * gamf * area * (nx * nx) / dN; fvl = -((-2. * gamf * area / dN) * (m->v[i1] * ny + m->w[i1] * nz) * nx); }
        else if (comp == 1) { fcl = 2. * gamf * area * (ny * ny) / dN; fvl = -((-2. * gamf * area / dN) * (m->u[i1] * nx + m->w[i1] * nz) * ny); }
        else { fcl = 2. * gamf * area * (nz * nz) / dN; fvl = -((-2. * gamf * area / dN) * (m->u[i1] * nx + m->v[i1] * ny) * nz); }
        m->fcf[i4] += fcl; m->fvf[i4] += fvl;
        m->ftf[i4] += fcl * fi[i1] + 0. * bfi[b] + fvl;
      } else if (OM_GIVEN_FLOW(t)) {   /* :254-300, 507-525 */
        const double *bgx = bfg, *bgy = bfg + B, *bgz = bfg + 2 * (long)B;
        double fcl = gamf * m->bgdiff[b], ffl = -gamf * m->bgdiff[b];
        double fvl = -(gamf * (bgx[b] * m->bTx[b] + bgy[b] * m->bTy[b] + bgz[b] * m->bTz[b]));
        m->fcf[i4] += fcl; m->fff[i4] += ffl; m->fvf[i4] += fvl;
        m->ftf[i4] += fcl * fi[i1] + ffl * bfi[b] + fvl;
      } /* slip wall, fully developed outlet: zero (:126-146, :540-560) */
    }
    /* AssembleExplicitDiffusionTerm (AssembleExplicitDiffusion.for:22-176) */
    const double *Gx = comp == 0 ? m->ugf : comp == 1 ? m->ugf + F : m->ugf + 2 * (long)F;
    const double *Gy = comp == 0 ? m->vgf : comp == 1 ? m->vgf + F : m->vgf + 2 * (long)F;
    const double *Gz = comp == 0 ? m->wgf : comp == 1 ? m->wgf + F : m->wgf + 2 * (long)F;
    for (int k = 0; k < F; k++) {
      double gamf = m->gf[k] * m->edif[m->if_own[k]] + (1. - m->gf[k]) * m->edif[m->if_nbr[k]];
      double fvl = -(gamf * (Gx[k] * m->sx[k] + Gy[k] * m->sy[k] + Gz[k] * m->sz[k]));
      m->fvf[k] += fvl; m->ftf[k] += fvl;
    }
    const double *BGx = comp == 0 ? m->bug : comp == 1 ? m->bug + B : m->bug + 2 * (long)B;
    const double *BGy = comp == 0 ? m->bvg : comp == 1 ? m->bvg + B : m->bvg + 2 * (long)B;
    const double *BGz = comp == 0 ? m->bwg : comp == 1 ? m->bwg + B : m->bwg + 2 * (long)B;
    for (int b = 0; b < B; b++) {
      double gamf = m->bedif[b];
      double fvl = -(gamf * (BGx[b] * m->bsx[b] + BGy[b] * m->bsy[b] + BGz[b] * m->bsz[b]));
      m->fvf[F + b] += fvl; m->ftf[F + b] += fvl;
    }
    /* AssembleBulkViscosityTerm (AssembleBulkViscosity.for:22-172) */
    for (int k = 0; k < F; k++) {
      double gamf = m->gf[k] * m->edif[m->if_own[k]] + (1. - m->gf[k]) * m->edif[m->if_nbr[k]];
      double div = m->ugf[k] + m->vgf[F + k] + m->wgf[2 * (long)F + k];
      double s = comp == 0 ? m->sx[k] : comp == 1 ? m->sy[k] : m->sz[k];
      double fvl = -(OM_M23 * gamf * div * s);
      m->fvf[k] += fvl; m->ftf[k] += fvl;
    }
    for (int b = 0; b < B; b++) {
      double gamf = m->bedif[b];
      double div = m->bug[b] + m->bvg[B + b] + m->bwg[2 * (long)B + b];
      double s = comp == 0 ? m->bsx[b] : comp == 1 ? m->bsy[b] : m->bsz[b];
      double fvl = -(OM_M23 * gamf * div * s);
      m->fvf[F + b] += fvl; m->ftf[F + b] += fvl;
    }
  }
  /* AssembleConvectionTerm (Convection/AssembleConvection.for:72-88) */
  for (int k = 0; k < F; k++) {
    int i = m->if_own[k], j = m->if_nbr[k];
    double fcl = fmax(m->mdot[k], 0.), ffl = -fmax(-m->mdot[k], 0.);
    m->fcf[k] += fcl; m->fff[k] += ffl;
    m->ftf[k] += fcl * fi[i] + ffl * fi[j];
  }
  /* HRSchemesCorrections (AssembleHRSchemeCorrection.for:36-134) */
  if (c->hr_framework == FS_HR_TVD && m->nIter >= c->niter_start_hr && c->conv_scheme != FS_TVD_UPWIND) {
    const double *gx = fg, *gy = fg + N, *gz = fg + 2 * (long)N;
    for (int k = 0; k < F; k++) {
      int i = m->if_own[k], j = m->if_nbr[k], iu;
      double phic, phid, dx, dy, dz;
      if (m->mdot[k] > 0.) { iu = i; phic = fi[i]; phid = fi[j]; dx = m->dcfx[k]; dy = m->dcfy[k]; dz = m->dcfz[k]; }
      else { iu = j; phic = fi[j]; phid = fi[i]; dx = -m->dcfx[k]; dy = -m->dcfy[k]; dz = -m->dcfz[k]; }
      double phiu = phid - 2. * (gx[iu] * dx + gy[iu] * dy + gz[iu] * dz);
      double diff = phid - phic, rf;
      if (fabs(diff) < OM_EPS9) rf = 0.; else rf = (phic - phiu) / diff;
      double psi = tvd_psi(c->conv_scheme, rf);
      double phiHR = phic + 0.5 * psi * diff;
      phiHR = (1. - c->bleed) * phiHR + c->bleed * phic;
      m->ftf[k] += m->mdot[k] * (phiHR - phic) * 1.;
    }
  }
  /* ComputeEffectiveDivergence (CalculateEffectiveDivergence.for:20-45) */
  memset(m->effdiv, 0, sizeof(double) * N);
  for (int k = 0; k < F; k++) { m->effdiv[m->if_own[k]] += m->mdot[k]; m->effdiv[m->if_nbr[k]] -= m->mdot[k]; }
  for (int b = 0; b < B; b++) m->effdiv[m->bf_own[b]] += m->bmdot[b];
  for (int i = 0; i < N; i++) {   /* AssembleConvection.for:165-178 */
    double fce = fmax(m->effdiv[i], 0.0) - m->effdiv[i];
    double fve = -(fmax(m->effdiv[i], 0.0) * fi[i]);
    double fte = fce * fi[i] + fve;
    m->fce[i] += fce; m->fte[i] += fte;
  }
  /* boundary convection (AssembleConvection.for:182-580): inlet specified velocity, outlet FD */
  for (int b = 0; b < B; b++) {
    int i1 = m->bf_own[b], t = m->btype[b]; long i4 = F + b;
    if (OM_GIVEN_FLOW(t)) {
      double fcl = fmax(m->bmdot[b], 0.), ffl = -fmax(-m->bmdot[b], 0.);
      m->fcf[i4] += fcl; m->fff[i4] += ffl; m->ftf[i4] += fcl * fi[i1] + ffl * bfi[b];
    } else if (t == FS_BC_OUTLET_FD || OM_SP_OUTLET(t)) {   /* :421-476 the same for all three */
      const double *bgx = bfg, *bgy = bfg + B, *bgz = bfg + 2 * (long)B;
      double fcl = fmax(m->bmdot[b], 0.), ffl = -fmax(-m->bmdot[b], 0.);
      double fvl = m->bmdot[b] * (bgx[b] * m->bdx[b] + bgy[b] * m->bdy[b] + bgz[b] * m->bdz[b]);
      m->fcf[i4] += fcl; m->fff[i4] += ffl; m->ftf[i4] += fcl * fi[i1] + ffl * bfi[b] + fvl;
    }
  }
  /* AssembleTransientTerm (SolveXMomentumEquation.for:247-251) */
  om_transient_term(m, fi, comp);
  /* AssembleSourceTerm: Sc=Sb=0 for these cases (AssembleSources.for:20-33) adds nothing */
  /* AssemblePressureGradientTerm (AssemblePressureGradient.for:17-22) */
  const double *dp = m->pg + (long)comp * N;
  for (int i = 0; i < N; i++) m->fte[i] += dp[i] * m->vol[i];
  /* MinusTwoThirdsRhoK (AssembleMinusTwoThirdsRhoK.for:40-110): gradient of 2/3 rho k in X */
  if (c->turbulence) {
    if (comp == 0) {
      for (int i = 0; i < N; i++) m->rhok[i] = OM_TWOTHIRD * c->rho * m->tke[i];
      for (int b = 0; b < B; b++) m->brhok[b] = OM_TWOTHIRD * c->rho * m->btke[b];
      om_gradient(m, FS_VAR_RHOK, c->method_grad_mom, c->niter_grad_mom, m->rhok, m->brhok, m->drk, m->bdrk);
    }
    const double *dk = m->drk + (long)comp * N;
    for (int i = 0; i < N; i++) m->fte[i] += dk[i] * m->vol[i];
  }
  global_assembly(m);
  /* UnderRelaxEquation (UnderRelaxation.for:21) */
  if (c->relax_momentum) for (int i = 0; i < N; i++) m->ac[i] = m->ac[i] / c->urf_momentum;
  /* storeDvalues (StoreTheDValues.for:20-48) */
  double *d1 = comp == 0 ? m->du1 : comp == 1 ? m->dv1 : m->dw1;
  double *d2 = comp == 0 ? m->du2 : comp == 1 ? m->dv2 : m->dw2;
  double *st = comp == 0 ? m->us : comp == 1 ? m->vs : m->ws;
  for (int i = 0; i < N; i++) {
    d1[i] = m->vol[i] / m->ac[i];
    if (c->algorithm == FS_SIMPLE) d2[i] = d1[i];
    else {
      double s = m->ac[i];
      for (int j = 0; j < m->ncf[i]; j++) s += m->anb[(long)j * N + i];
      d2[i] = m->vol[i] / s;
    }
    st[i] = fi[i];
  }
}

void om_momentum(om *m, int comp)
{
  double *fi = comp == 0 ? m->u : comp == 1 ? m->v : m->w;
  om_assemble_momentum(m, comp);
  om_solve_equation(m, comp + 1, fi, m->cfg.rrf_mom, m->cfg.itmax_mom, m->cfg.solver_mom);
}

/* ===================================================================== */
/*  Continuity (ContinuityEquation/)                                      */
/* ===================================================================== */
static double geo_diff(int msd, double Du, double Dv, double Dw, double sx, double sy, double sz,
                       double ex, double ey, double ez, double cf, double *tx, double *ty, double *tz)
{ /* AssembleMdotUsingRhieChow.for:579-611 / AssemblePressureCorrectionFluxes.for:96-140 */
  double DuSf = Du * sx, DvSf = Dv * sy, DwSf = Dw * sz, DuEf, DvEf, DwEf;
  if (msd == 1) {
    double dp = ex * DuSf + ey * DvSf + ez * DwSf;
    DuEf = dp * ex; DvEf = dp * ey; DwEf = dp * ez;
  } else if (msd == 2) {
    double mag = sqrt(DuSf * DuSf + DvSf * DvSf + DwSf * DwSf);
    DuEf = ex * mag; DvEf = ey * mag; DwEf = ez * mag;
  } else {
    double mag = sqrt(DuSf * DuSf + DvSf * DvSf + DwSf * DwSf);
    double eu = DuSf / mag, ev = DvSf / mag, ew = DwSf / mag;
    double dp = ex * eu + ey * ev + ez * ew;
    DuEf = mag * ex / dp; DvEf = mag * ey / dp; DwEf = mag * ez / dp;
  }
  double gd = sqrt(DuEf * DuEf + DvEf * DvEf + DwEf * DwEf) / cf;
  if (tx) { *tx = DuSf - DuEf; *ty = DvSf - DvEf; *tz = DwSf - DwEf; }
  return gd;
}

/* FlowIn (CalculateFlowIn.for:4-40), FlowOut (CalculateFlowOut.for:4-55) and
 * AdjustFlow (AdjustFlowAtOuletBoundary.for:4-75), incompressible, when every
 * outlet is 'fullydeveloped' */
static void om_flow_in_out(om *m)
{
  int NS = m->NS, F = m->F;
  const fs_case *c = &m->cfg;
  int nfd = 0, other = 0;
  for (int s = 0; s < NS; s++) {
    if (c->patch_type[s] == FS_BC_OUTLET_FD) nfd++;
    if (OM_SP_OUTLET(c->patch_type[s]) || c->patch_type[s] == FS_BC_OUTLET_MASS) other++;
  }
  /* FlowOut/AdjustFlow return at once unless every outlet is fully developed */
  if (nfd == 0 || other) return;
  /* FlowIn returns at once when an inlet is a static- or stagnation-pressure
   * one (CalculateFlowIn.for:19-31): mdotIn keeps the value the last
   * CalculateResidualsContinuity left (every inlet face, :195-203) */
  int p_inlet = 0;
  for (int s = 0; s < NS; s++) p_inlet |= OM_P_INLET(c->patch_type[s]);
  if (!p_inlet) {
    m->mdot_in = 0.;
    for (int s = 0; s < NS; s++)   /* velocity and mass-flow inlets (CalculateFlowIn.for:37-48) */
      if (c->patch_type[s] == FS_BC_INLET_VEL || c->patch_type[s] == FS_BC_INLET_MASS)
        for (int j = 0; j < m->bset_n[s]; j++) m->mdot_in = m->mdot_in + m->bmdot[m->bset_start[s] + j];
  }
  for (int s = 0; s < NS; s++) if (c->patch_type[s] == FS_BC_OUTLET_FD) {
    m->mdot1[s] = 0.;
    for (int j = 0; j < m->bset_n[s]; j++) {
      int b = m->bset_start[s] + j;
      m->bmdot[b] = c->rho * (m->bu[b] * m->bsx[b] + m->bv[b] * m->bsy[b] + m->bw[b] * m->bsz[b]);
      if (m->bmdot[b] < m->mdot1[s]) m->mdot1[s] = m->bmdot[b];
    }
    m->mdot1[s] = fabs(m->mdot1[s]);
  }
  for (int s = 0; s < NS; s++) if (c->patch_type[s] == FS_BC_OUTLET_FD) {
    m->mdot_out[s] = 0.;
    for (int j = 0; j < m->bset_n[s]; j++) m->mdot_out[s] = m->mdot_out[s] + m->mdot1[s] + m->bmdot[m->bset_start[s] + j];
  }
  double tff = 0.;
  for (int s = 0; s < NS; s++) if (c->patch_type[s] == FS_BC_OUTLET_FD) tff = tff + c->mass_flow_fraction[s];
  for (int s = 0; s < NS; s++) if (c->patch_type[s] == FS_BC_OUTLET_FD) {
    double ratio = (c->mass_flow_fraction[s] / (tff + OM_TINY)) * fabs(m->mdot_in / (m->mdot_out[s] + OM_TINY));
    for (int j = 0; j < m->bset_n[s]; j++) {
      int b = m->bset_start[s] + j, k = m->bf_own[b];
      m->bmdot[b] = ratio * (m->bmdot[b] + m->mdot1[s]);
      /* boundary velocity from the owner and the boundary gradient; AssembleMdot
       * overwrites it with the owner velocity right after */
      m->bu[b] = m->u[k] + (m->bug[b] * m->bdx[b] + m->bug[m->B + b] * m->bdy[b] + m->bug[2L * m->B + b] * m->bdz[b]);
      m->bv[b] = m->v[k] + (m->bvg[b] * m->bdx[b] + m->bvg[m->B + b] * m->bdy[b] + m->bvg[2L * m->B + b] * m->bdz[b]);
      m->bw[b] = m->w[k] + (m->bwg[b] * m->bdx[b] + m->bwg[m->B + b] * m->bdy[b] + m->bwg[2L * m->B + b] * m->bdz[b]);
    }
  }
  (void)F;
}

/* the velocity of an inlet with a given direction from its Bmdot
 * (AssembleMdotUsingRhieChow.for:2089-2099) */
static void om_directed_velocity(om *m, int b)
{
  const double *d = m->bdir + 3L * b;
  double vm = m->bmdot[b] / (m->cfg.rho * (d[0] * m->bsx[b] + d[1] * m->bsy[b] + d[2] * m->bsz[b]));
  m->bu[b] = vm * d[0]; m->bv[b] = vm * d[1]; m->bw[b] = vm * d[2];
}

/* AssembleMdot (AssembleMdotUsingRhieChow.for:262-292, 554-759, 1441-1598, 2033-2283) */
static void om_assemble_mdot(om *m)
{
  int N = m->N, F = m->F, B = m->B;
  const fs_case *c = &m->cfg;
  double *pgbar = dz_(3 * (long)F);
  om_interp_grad(m, FS_GI_AVERAGE, m->p, m->pg, pgbar);
  const double *pbx = pgbar, *pby = pgbar + F, *pbz = pgbar + 2 * (long)F;
  const double *pfx = m->pgf, *pfy = m->pgf + F, *pfz = m->pgf + 2 * (long)F;
  /* k-epsilon: the 2/3 rho k gradient enters like the pressure
   * (AssembleMdotUsingRhieChow.for:296-305, 627-634): 'average' and
   * 'averagecorrected' face gradients of rhok from MinusTwoThirdsRhoK */
  double *rkbar = NULL, *rkf = NULL;
  if (c->turbulence) {
    rkbar = dz_(3 * (long)F); rkf = dz_(3 * (long)F);
    om_interp_grad(m, FS_GI_AVERAGE, m->rhok, m->drk, rkbar);
    om_interp_grad(m, FS_GI_AVERAGECORRECTED, m->rhok, m->drk, rkf);
  }
  for (int k = 0; k < F; k++) {
    int i = m->if_own[k], j = m->if_nbr[k];
    double rhof = c->rho, sx = m->sx[k], sy = m->sy[k], sz = m->sz[k];
    double du = avgf(m, k, m->du1), dv = avgf(m, k, m->dv1), dw = avgf(m, k, m->dw1);
    double mbar = avgf(m, k, m->u) * sx + avgf(m, k, m->v) * sy + avgf(m, k, m->w) * sz;
    double fvl = rhof * mbar;
    double tx, ty, tz;
    double gd = geo_diff(c->method_decompose_s, du, dv, dw, sx, sy, sz, m->ex[k], m->ey[k], m->ez[k], m->dcf[k], &tx, &ty, &tz);
    double fcl = rhof * gd, ffl = -rhof * gd;
    fvl = fvl - rhof * (pfx[k] * tx + pfy[k] * ty + pfz[k] * tz);
    fvl = fvl + rhof * (pbx[k] * (du * sx) + pby[k] * (dv * sy) + pbz[k] * (dw * sz));
    if (c->turbulence) {
      fvl = fvl - rhof * (rkf[k] * tx + rkf[F + k] * ty + rkf[2L * F + k] * tz);
      fvl = fvl + rhof * (rkbar[k] * (du * sx) + rkbar[F + k] * (dv * sy) + rkbar[2L * F + k] * (dw * sz));
      fvl = fvl + fcl * m->rhok[i] + ffl * m->rhok[j];
    }
    if (c->relax_momentum) {
      double ms = rhof * (avgf(m, k, m->us) * sx + avgf(m, k, m->vs) * sy + avgf(m, k, m->ws) * sz);
      fvl = fvl + (1. - c->urf_momentum) * (m->mdot[k] - ms);
    }
    m->mdot[k] = fcl * m->p[i] + ffl * m->p[j] + fvl;
  }
  free(pgbar); free(rkbar); free(rkf);
  /* 'specifiedstaticpressure' outlets (AssembleMdotUsingRhieChow.for:1441-1598) and
   * inlets (:2105-2283): the same Rhie-Chow boundary flux; the outlet first
   * extrapolates its velocity, the inlet's follows from Bmdot along its direction */
  for (int b = 0; b < B; b++) if (OM_PRESSURE(m->btype[b])) {
    int i1 = m->bf_own[b];
    double rhof = c->rho, sx = m->bsx[b], sy = m->bsy[b], sz = m->bsz[b];
    if (OM_SP_OUTLET(m->btype[b])) {
      m->bu[b] = m->u[i1] + (m->bug[b] * m->bdx[b] + m->bug[B + b] * m->bdy[b] + m->bug[2L * B + b] * m->bdz[b]);
      m->bv[b] = m->v[i1] + (m->bvg[b] * m->bdx[b] + m->bvg[B + b] * m->bdy[b] + m->bvg[2L * B + b] * m->bdz[b]);
      m->bw[b] = m->w[i1] + (m->bwg[b] * m->bdx[b] + m->bwg[B + b] * m->bdy[b] + m->bwg[2L * B + b] * m->bdz[b]);
    }
    double mbar = m->u[i1] * sx + m->v[i1] * sy + m->w[i1] * sz;
    double fvl = rhof * mbar;
    double du = m->du1[i1], dv = m->dv1[i1], dw = m->dw1[i1], tx, ty, tz;
    double gd = geo_diff(c->method_decompose_s, du, dv, dw, sx, sy, sz, m->bex[b], m->bey[b], m->bez[b], m->bd[b], &tx, &ty, &tz);
    double fcl = rhof * gd, ffl = -rhof * gd;
    fvl = fvl - rhof * (m->bpg[b] * tx + m->bpg[B + b] * ty + m->bpg[2L * B + b] * tz);
    fvl = fvl + rhof * (m->pg[i1] * (du * sx) + m->pg[N + i1] * (dv * sy) + m->pg[2L * N + i1] * (dw * sz));
    if (c->turbulence) {
      fvl = fvl - rhof * (m->bdrk[b] * tx + m->bdrk[B + b] * ty + m->bdrk[2L * B + b] * tz);
      fvl = fvl + rhof * (m->drk[i1] * (du * sx) + m->drk[N + i1] * (dv * sy) + m->drk[2L * N + i1] * (dw * sz));
      fvl = fvl + fcl * m->rhok[i1] + ffl * m->brhok[b];
    }
    if (c->relax_momentum) {
      double ms = rhof * (m->us[i1] * sx + m->vs[i1] * sy + m->ws[i1] * sz);
      fvl = fvl + (1. - c->urf_momentum) * (m->bmdot[b] - ms);
    }
    m->bmdot[b] = fcl * m->p[i1] + ffl * m->bp[b] + fvl;
    if (OM_P_INLET(m->btype[b])) om_directed_velocity(m, b);   /* :2277-2282, 2455-2460 */
  }
  /* inlet specified velocity Bmdot (AssembleMdotUsingRhieChow.for:2054-2075) */
  for (int b = 0; b < B; b++) if (m->btype[b] == FS_BC_INLET_VEL)
    m->bmdot[b] = c->rho * (m->bu[b] * m->bsx[b] + m->bv[b] * m->bsy[b] + m->bw[b] * m->bsz[b]);
  /* fully developed outlet velocity (AssembleMdotUsingRhieChow.for:2033-2050) */
  for (int b = 0; b < B; b++) if (m->btype[b] == FS_BC_OUTLET_FD) {
    int i1 = m->bf_own[b];
    m->bu[b] = m->u[i1]; m->bv[b] = m->v[i1]; m->bw[b] = m->w[i1];
  }
  /* 'specifiedmassflowrate' inlet velocity from Bmdot along the given
   * direction (AssembleMdotUsingRhieChow.for:2077-2100) */
  for (int b = 0; b < B; b++) if (m->btype[b] == FS_BC_INLET_MASS) om_directed_velocity(m, b);
  /* 'specifiedmassflowrate' outlets: along the owner's velocity (:1999-2031) */
  for (int b = 0; b < B; b++) if (m->btype[b] == FS_BC_OUTLET_MASS) {
    int i1 = m->bf_own[b];
    double vel = sqrt(m->u[i1] * m->u[i1] + m->v[i1] * m->v[i1] + m->w[i1] * m->w[i1]);
    double dx = m->u[i1] / (vel + OM_TINY), dy = m->v[i1] / (vel + OM_TINY), dz = m->w[i1] / (vel + OM_TINY);
    double vm = m->bmdot[b] / (c->rho * (dx * m->bsx[b] + dy * m->bsy[b] + dz * m->bsz[b]));
    m->bu[b] = vm * dx; m->bv[b] = vm * dy; m->bw[b] = vm * dz;
  }
}

void om_assemble_continuity(om *m)
{
  int N = m->N, F = m->F, B = m->B;
  const fs_case *c = &m->cfg;
  init_fluxes(m);
  memset(m->pc, 0, sizeof(double) * N);          /* InitializePressureCorrection */
  om_flow_in_out(m);                             /* FlowIn, FlowOut, AdjustFlow */
  om_assemble_mdot(m);
  /* UpdateBoundaryForTotalConditions (TotalConditionsBoundary.for:25-45), incompressible */
  for (int b = 0; b < B; b++) if (m->btype[b] == FS_BC_INLET_STAG) {
    const double vel2 = m->bu[b] * m->bu[b] + m->bv[b] * m->bv[b] + m->bw[b] * m->bw[b];
    m->bp[b] = fmax(m->bp0[b] - 0.5 * c->rho * vel2, 0.);
  }
  /* AssemblePressureCorrection (AssemblePressureCorrectionFluxes.for:85-164) */
  for (int k = 0; k < F; k++) {
    double du = avgf(m, k, m->du2), dv = avgf(m, k, m->dv2), dw = avgf(m, k, m->dw2);
    double gd = geo_diff(c->method_decompose_s, du, dv, dw, m->sx[k], m->sy[k], m->sz[k], m->ex[k], m->ey[k], m->ez[k], m->dcf[k], 0, 0, 0);
    m->fcf[k] = c->rho * gd; m->fff[k] = -(c->rho * gd); m->ftf[k] = m->mdot[k];
  }
  for (int b = 0; b < B; b++) m->ftf[F + b] = m->bmdot[b];
  /* 'specifiedstaticpressure' outlets and inlets: p'_b = 0, FluxCf = FluxFf = rho geoDiff(D2)
   * (AssemblePressureCorrectionFluxes.for:244-313, 585-657) */
  for (int b = 0; b < B; b++) if (OM_PRESSURE(m->btype[b])) {
    int i1 = m->bf_own[b];
    double gd = geo_diff(c->method_decompose_s, m->du2[i1], m->dv2[i1], m->dw2[i1], m->bsx[b], m->bsy[b], m->bsz[b],
                         m->bex[b], m->bey[b], m->bez[b], m->bd[b], 0, 0, 0);
    m->fcf[F + b] = c->rho * gd; m->fff[F + b] = c->rho * gd;
    m->bgd[b] = gd;
  }
  /* 'specifiedresistance' outlets (:400-500): geoDiffSum per patch, FluxCf
   * rho geoDiff (1 + (geoDiffSum - geoDiff) R) / (1 + R geoDiffSum) */
  for (int s = 0; s < m->NS; s++) if (c->patch_type[s] == FS_BC_OUTLET_RES) {
    m->gdsum[s] = 0.;
    for (int j = 0; j < m->bset_n[s]; j++) m->gdsum[s] = m->gdsum[s] + m->bgd[m->bset_start[s] + j];
    const double R = c->patch_resistance[s];
    for (int j = 0; j < m->bset_n[s]; j++) {
      const int b = m->bset_start[s] + j;
      double fcl = c->rho * m->bgd[b];
      fcl = fcl * (1 + (m->gdsum[s] - m->bgd[b]) * R) / (1. + R * m->gdsum[s]);
      m->fcf[F + b] = fcl;
    }
  }
  /* 'specifiedstagnationpressure' inlets (:663-720): FluxCf Bmdot FluxFf / (Bmdot - FluxFf rho |U_b|^2) */
  for (int b = 0; b < B; b++) if (m->btype[b] == FS_BC_INLET_STAG) {
    const double vel2 = m->bu[b] * m->bu[b] + m->bv[b] * m->bv[b] + m->bw[b] * m->bw[b];
    const double ff = m->fff[F + b];
    m->fcf[F + b] = m->bmdot[b] * ff / (m->bmdot[b] - ff * c->rho * vel2);
  }
  /* specified-velocity inlet: FluxCf=FluxFf=0 (AssemblePressureCorrectionFluxes.for:545-563) */
  global_assembly(m);
  if (0) {   /* LfixPressure (FixPressure, ReferenceAndSetPressureRoutines.for:64) is not used by these cases */
    int i = c->ref_pressure_cell;
    m->bc[i] = 0;
    for (int j = 0; j < m->ncf[i]; j++) m->anb[(long)j * N + i] = 0.;
  }
}

void om_correct_continuity(om *m)
{
  int N = m->N, F = m->F, B = m->B;
  const fs_case *c = &m->cfg;
  /* UpdateBoundaryPressureCorrection (UpdatePressureCorrectionAtBoundaries.for) */
  for (int b = 0; b < B; b++) {
    const int t = m->btype[b];
    if (t == FS_BC_INLET_STAG) {   /* :97-112, geoDiff = FluxFf */
      const double gd = m->fff[F + b];
      const double vel2 = m->bu[b] * m->bu[b] + m->bv[b] * m->bv[b] + m->bw[b] * m->bw[b];
      m->bpc[b] = -c->rho * vel2 * gd * m->pc[m->bf_own[b]] / (m->bmdot[b] - gd * c->rho * vel2);
    } else if (t != FS_BC_OUTLET_RES) {
      m->bpc[b] = (t == FS_BC_OUTLET_SP || t == FS_BC_INLET_SP || t == FS_BC_OUTLET_ASP) ? 0. : m->pc[m->bf_own[b]];   /* :85-90, 126-143 */
    }
  }
  /* 'specifiedresistance' (:144-175): R sum(geoDiffB p'_C) / (1 + R geoDiffSum) on the patch */
  for (int s = 0; s < m->NS; s++) if (c->patch_type[s] == FS_BC_OUTLET_RES) {
    double pcr = 0.;
    for (int j = 0; j < m->bset_n[s]; j++) {
      const int b = m->bset_start[s] + j;
      pcr = pcr + m->bgd[b] * m->pc[m->bf_own[b]];
    }
    const double R = c->patch_resistance[s];
    pcr = R * pcr / (1. + R * m->gdsum[s]);
    for (int j = 0; j < m->bset_n[s]; j++) m->bpc[m->bset_start[s] + j] = pcr;
  }
  /* CorrectPressure (CorrectPressure.for:4-42) */
  double rpc = (c->ref_pressure_cell >= 0) ? m->pc[c->ref_pressure_cell] : 0.;
  if (c->set_reference_pressure == 1) rpc = 0.;
  for (int i = 0; i < N; i++) m->p[i] = m->p[i] + c->urf_pressure * (m->pc[i] - rpc);
  /* CorrectVelocity (CorrectMdotandVelocity.for:722-779) */
  om_gradient(m, FS_VAR_PC, c->method_grad_cont, c->niter_grad_cont, m->pc, m->bpc, m->pcg, m->bpcg);
  for (int i = 0; i < N; i++) {
    m->u[i] = m->u[i] - m->du2[i] * m->pcg[i];
    m->v[i] = m->v[i] - m->dv2[i] * m->pcg[N + i];
    m->w[i] = m->w[i] - m->dw2[i] * m->pcg[2 * (long)N + i];
  }
  /* Correctmdot (CorrectMdotandVelocity.for:55-63) */
  for (int k = 0; k < F; k++)
    m->mdot[k] = m->mdot[k] + m->fcf[k] * m->pc[m->if_own[k]] + m->fff[k] * m->pc[m->if_nbr[k]];
  /* CorrectBoundarymdot, 'specifiedstaticpressure' outlets (CorrectMdotandVelocity.for:264-280)
   * and inlets (:180-205: the velocity again from Bmdot along its direction) */
  for (int b = 0; b < B; b++) if (OM_PRESSURE(m->btype[b])) {
    int i1 = m->bf_own[b];
    double gd = m->fff[F + b];
    m->bmdot[b] = m->bmdot[b] - gd * (m->bpc[b] - m->pc[i1]);
    if (OM_P_INLET(m->btype[b])) { om_directed_velocity(m, b); continue; }
    m->bu[b] = m->bu[b] - m->du2[i1] * m->pcg[i1];
    m->bv[b] = m->bv[b] - m->dv2[i1] * m->pcg[N + i1];
    m->bw[b] = m->bw[b] - m->dw2[i1] * m->pcg[2L * N + i1];
  }
  /* CorrectBoundarymdot, 'specifiedmassflowrate' inlets and outlets: velocity only
   * (CorrectMdotandVelocity.for:165-175, 354-364) */
  for (int b = 0; b < B; b++) if (m->btype[b] == FS_BC_INLET_MASS || m->btype[b] == FS_BC_OUTLET_MASS) {
    int i1 = m->bf_own[b];
    m->bu[b] = m->bu[b] - m->du2[i1] * m->pcg[i1];
    m->bv[b] = m->bv[b] - m->dv2[i1] * m->pcg[N + i1];
    m->bw[b] = m->bw[b] - m->dw2[i1] * m->pcg[2L * N + i1];
  }
  /* UpdateBoundaryPressure (CorrectPressure.for:49-190): walls and symmetry */
  for (int b = 0; b < B; b++) {
    int t = m->btype[b], i1 = m->bf_own[b];
    if (t == FS_BC_WALL_SLIP || t == FS_BC_WALL_NOSLIP || t == FS_BC_SYMMETRY)
      m->bp[b] = m->p[i1] + m->bpg[b] * m->bdx[b] + m->bpg[B + b] * m->bdy[b] + m->bpg[2 * (long)B + b] * m->bdz[b];
    else if (t == FS_BC_INLET_VEL || t == FS_BC_INLET_MASS || t == FS_BC_OUTLET_FD || t == FS_BC_OUTLET_MASS)   /* :120-138, 220-226; static pressures stay */
      m->bp[b] = m->bp[b] + c->urf_pressure * (m->bpc[b] - rpc);
    else if (t == FS_BC_OUTLET_ASP)   /* :169-176 */
      m->bp[b] = m->p[i1];
    else if (t == FS_BC_OUTLET_RES || t == FS_BC_INLET_STAG)   /* :152-160, 206-214 */
      m->bp[b] = m->bp[b] + c->urf_pressure * (m->bpc[b] - rpc);
  }
  /* 'specifiedaveragestaticpressure': the face pressures shifted so that their
   * area average is AverageOutletPressure (:178-203) */
  for (int s = 0; s < m->NS; s++) if (c->patch_type[s] == FS_BC_OUTLET_ASP) {
    double avg = 0., area = 0.;
    for (int j = 0; j < m->bset_n[s]; j++) {
      int b = m->bset_start[s] + j;
      avg = avg + m->bfa[b] * m->bp[b];
      area = area + m->bfa[b];
    }
    avg = avg / (area + OM_TINY);
    avg = c->patch_pressure[s] - avg;
    for (int j = 0; j < m->bset_n[s]; j++) { int b = m->bset_start[s] + j; m->bp[b] = m->bp[b] + avg; }
  }
  /* CalculateResidualsContinuity (CalculateContinuityResiduals.for:130-235) */
  double *mi = dz_(N);
  for (int k = 0; k < F; k++) { mi[m->if_own[k]] += m->mdot[k]; mi[m->if_nbr[k]] -= m->mdot[k]; }
  for (int b = 0; b < B; b++) mi[m->bf_own[b]] += m->bmdot[b];
  if (c->unsteady) {   /* + d rho/dt V (CalculateContinuityResiduals.for:159-170) */
    double drhodt = om_drhodt(m);
    for (int i = 0; i < N; i++) mi[i] = mi[i] + drhodt * m->vol[i];
  }
  double mx = 0., ov = 0., ab = 0., rms = 0.; int imx = 0;
  for (int i = 0; i < N; i++) {
    ov += mi[i]; ab += fabs(mi[i]);
    mx = fmax(mx, fabs(mi[i]));
    if (mx == fabs(mi[i])) imx = i;
    rms += mi[i] * mi[i];
  }
  m->rmax[4] = mx; m->rabs[4] = ab; m->rrms[4] = sqrt(rms / N);
  m->overall_imbalance = ov; m->imax_imbalance = imx;
  double min_ = 0.;
  for (int b = 0; b < B; b++) if (OM_INLET(m->btype[b])) min_ += m->bmdot[b];   /* every 'inlet' face (:195-203) */
  m->mdot_in = min_;                                                                /* the module's mdotIn */
  m->rscl[4] = (min_ == 0.) ? 0. : m->rmax[4] / fabs(min_);
  free(mi);
  /* UpdateSymmetry (SymmetryAndAxisBoundary.for:4-33), UpdateSlipWallBoundary */
  for (int b = 0; b < B; b++) {
    int t = m->btype[b], i1 = m->bf_own[b];
    if (t == FS_BC_SYMMETRY || t == FS_BC_WALL_SLIP) {
      double nx = m->bnx[b], ny = m->bny[b], nz = m->bnz[b];
      double a = m->u[i1] * nx + m->v[i1] * ny + m->w[i1] * nz;
      m->bu[b] = m->u[i1] - a * nx; m->bv[b] = m->v[i1] - a * ny; m->bw[b] = m->w[i1] - a * nz;
    }
  }
}

void om_continuity(om *m)
{
  om_assemble_continuity(m);
  om_solve_equation(m, FS_VAR_PC, m->pc, m->cfg.rrf_cont, m->cfg.itmax_cont, m->cfg.solver_cont);
  om_correct_continuity(m);
}

/* ===================================================================== */
/*  Linear solvers (AlgebraicSolvers/)                                    */
/* ===================================================================== */
/* CalculateResiduals (CalculateResidualsRoutine.for:3-67) */
void om_calc_residuals(om *m, int nf, const double *fi)
{
  int N = m->N, q = nf - 1;
  m->rabs[q] = 0.; m->rmax[q] = -1.; m->rscl[q] = -1;
  if (nf == 4) m->rscl[q] = 0.;
  double rmsr = 0., acphic = -1.;
  for (int i = 0; i < N; i++) acphic = fmax(acphic, fabs(m->ac[i] * fi[i]));
  for (int i = 0; i < N; i++) {
    double r = m->bc[i] - m->ac[i] * m->dphi[i];
    for (int j = 0; j < m->ncf[i]; j++) {
      int k = m->cn[(long)j * N + i];
      if (k >= 0) r = r - m->anb[(long)j * N + i] * m->dphi[k];
    }
    r = fabs(r);
    m->rabs[q] += r; m->rmax[q] = fmax(m->rmax[q], r); rmsr += r * r;
    if (nf != 4) m->rscl[q] = fmax(m->rscl[q], r / (acphic + OM_TINY));
  }
  m->rrms[q] = sqrt(rmsr / N);
}

static double check_convergence(om *m)   /* CheckConvergenceRoutine.for:3 */
{
  int N = m->N; double s = 0.;
  for (int i = 0; i < N; i++) {
    double r = m->bc[i] - m->ac[i] * m->dphi[i];
    for (int j = 0; j < m->ncf[i]; j++) {
      int k = m->cn[(long)j * N + i];
      if (k >= 0) r = r - m->anb[(long)j * N + i] * m->dphi[k];
    }
    s += fabs(r);
  }
  return s;
}

static void sor_sweep(om *m)   /* SolveEquationsUsingSOR (SORMethod.for:20-60) */
{
  int N = m->N;
  for (int pass = 0; pass < 2; pass++)
    for (int ii = 0; ii < N; ii++) {
      int i = pass == 0 ? ii : N - 1 - ii;
      double l = m->bc[i];
      for (int j = 0; j < m->ncf[i]; j++) {
        int k = m->cn[(long)j * N + i];
        if (k >= 0) l = l - m->anb[(long)j * N + i] * m->dphi[k];
      }
      m->dphi[i] = l / m->ac[i];
    }
}

/* the first slot of row j whose neighbour is i (the reference's search loops,
 * FactorizeUsingILU.for:47-51, ILUMethod.for:86-92); -1 when there is none */
static int slot_of(const om *m, int j, int i)
{
  const int N = m->N;
  for (int q = 0; q < m->ncf[j]; q++) if (m->cn[(long)q * N + j] == i) return q;
  return -1;
}

/* ILUFactorization (FactorizeUsingILU.for:4-75): the diagonal of the D-ILU
 * factorisation, dc = 1/(ac - sum over earlier neighbours), in element order.
 * Quirk kept: element NumberOfElements-1 (1-based; 0-based N-2) does not
 * update its later neighbours (:36). */
static void ilu_factor(om *m)
{
  const int N = m->N;
  if (!m->ilu_dc) { m->ilu_dc = dz_(N); m->ilu_rc = dz_(N); }
  double *dc = m->ilu_dc;
  for (int i = 0; i < N; i++) dc[i] = m->ac[i];
  for (int i1 = 0; i1 < N; i1++) {
    dc[i1] = 1.0 / dc[i1];
    m->ilu_rc[i1] = m->bc[i1];
    if (i1 == N - 2) continue;
    for (int j2 = 0; j2 < m->ncf[i1]; j2++) {
      const int j4 = m->cn[(long)j2 * N + i1];
      if (j4 > i1 && j4 < N) {
        const int i2 = slot_of(m, j4, i1);
        if (i2 >= 0) dc[j4] = dc[j4] - m->anb[(long)i2 * N + j4] * dc[i1] * m->anb[(long)j2 * N + i1];
        else fprintf(stderr, "the index for i in j is not found\n");
      }
    }
  }
}

/* SolveEquationsUsingILU (ILUMethod.for:4-170): residual, forward
 * substitution through the earlier neighbours, backward substitution through
 * the later ones, dphi += D r */
static void ilu_sweep(om *m)
{
  const int N = m->N;
  double *dc = m->ilu_dc, *rc = m->ilu_rc, *dphi = m->dphi;
  for (int i = 0; i < N; i++) {
    double res = -m->ac[i] * dphi[i] + m->bc[i];
    for (int j = 0; j < m->ncf[i]; j++) {
      const int k = m->cn[(long)j * N + i];
      if (k >= 0) res = res - m->anb[(long)j * N + i] * dphi[k];
    }
    rc[i] = res;
  }
  for (int i1 = 0; i1 < N; i1++) {
    const double product1 = dc[i1] * rc[i1];
    for (int j2 = 0; j2 < m->ncf[i1]; j2++) {
      const int j1 = m->cn[(long)j2 * N + i1];
      if (j1 >= 0 && j1 > i1 && j1 < N) {
        const int i2 = slot_of(m, j1, i1);
        if (i2 >= 0) {
          const double product2 = m->anb[(long)i2 * N + j1] * product1;
          rc[j1] = rc[j1] - product2;
        } else {
          fprintf(stderr, "ILU Solver Error The index for i in element j is not found\n");
        }
      }
    }
  }
  for (int i1 = N - 1; i1 >= 0; i1--) {
    if (i1 < N - 1)
      for (int j2 = 0; j2 < m->ncf[i1]; j2++) {
        const int j = m->cn[(long)j2 * N + i1];
        if (j > i1) rc[i1] = rc[i1] - m->anb[(long)j2 * N + i1] * rc[j];
      }
    const double product1 = dc[i1] * rc[i1];
    rc[i1] = product1;
    dphi[i1] = dphi[i1] + product1;
  }
}

/* PBCG (PBCGMethod.for): Numerical Recipes' biconjugate gradient in its
 * minimum-residual form (rr = A r at the start), both systems preconditioned
 * by the D-ILU diagonal dc (asolve, :196-212).  A is sprsin's copy of the
 * system (:290-333): the diagonal ac, then every neighbour slot of each row
 * in slot order (thresh 0 keeps zero coefficients).  dsprsax (A x) sums a
 * row as the diagonal term, then the off-diagonal terms in slot order;
 * dsprstx (A^T x) starts from the diagonal terms and adds every row's
 * off-diagonal terms to their columns, rows in element order.  bkden is a
 * local of SolveEquationsUsingPBCG without SAVE: it is kept from one call
 * (iteration) to the next here, the only reading under which the recurrence
 * is defined. */
struct om_pbcg { double *p, *pp, *r, *rr, *z, *zz, bkden; };

static void pbcg_atimes(const om *m, int trn, const double *b, double *x)
{
  const int N = m->N;
  if (!trn) {
    for (int i = 0; i < N; i++) {
      double t = m->ac[i] * b[i];
      for (int j = 0; j < m->ncf[i]; j++) {
        const int k = m->cn[(long)j * N + i];
        if (k >= 0 && k != i) t = t + m->anb[(long)j * N + i] * b[k];
      }
      x[i] = t;
    }
  } else {
    for (int i = 0; i < N; i++) x[i] = m->ac[i] * b[i];
    for (int i = 0; i < N; i++)
      for (int j = 0; j < m->ncf[i]; j++) {
        const int k = m->cn[(long)j * N + i];
        if (k >= 0 && k != i) x[k] = x[k] + m->anb[(long)j * N + i] * b[i];
      }
  }
}

/* SolveEquationsUsingPBCG (PBCGMethod.for:96-180), one call = one iteration */
static void pbcg_step(om *m, struct om_pbcg *w, int iter)
{
  const int N = m->N;
  const double *dc = m->ilu_dc;
  if (iter == 0) {
    pbcg_atimes(m, 0, m->dphi, w->r);
    for (int j = 0; j < N; j++) { w->r[j] = m->bc[j] - w->r[j]; w->rr[j] = w->r[j]; }
    pbcg_atimes(m, 0, w->r, w->rr);          /* the minimum-residual variant */
  }
  for (int i = 0; i < N; i++) w->z[i] = w->r[i] * dc[i];
  for (int i = 0; i < N; i++) w->zz[i] = w->rr[i] * dc[i];
  double bknum = 0.;
  for (int j = 0; j < N; j++) bknum = bknum + w->z[j] * w->rr[j];
  if (iter == 0) {
    for (int j = 0; j < N; j++) { w->p[j] = w->z[j]; w->pp[j] = w->zz[j]; }
  } else {
    const double bk = bknum / (w->bkden + 1.e-10);
    for (int j = 0; j < N; j++) { w->p[j] = bk * w->p[j] + w->z[j]; w->pp[j] = bk * w->pp[j] + w->zz[j]; }
  }
  w->bkden = bknum;
  pbcg_atimes(m, 0, w->p, w->z);
  double akden = 0.;
  for (int j = 0; j < N; j++) akden = akden + w->z[j] * w->pp[j];
  const double ak = bknum / (akden + 1.e-10);
  pbcg_atimes(m, 1, w->pp, w->zz);
  for (int j = 0; j < N; j++) {
    m->dphi[j] = m->dphi[j] + ak * w->p[j];
    w->r[j] = w->r[j] - ak * w->z[j];
    w->rr[j] = w->rr[j] - ak * w->zz[j];
  }
}

/* SolveAlgebraicSystemInParallel CSR (matrixSolverOMP.f90:462-584) + AxOMP (:390-423) */
static void csr_build(om *m)
{
  int N = m->N;
  if (!m->csr_built) {
    m->csr_ptr = (long *)calloc((size_t)N + 1, sizeof(long));
    long nnz = 0;
    for (int i = 0; i < N; i++) {
      m->csr_ptr[i] = nnz; nnz++;
      for (int j = 0; j < m->ncf[i]; j++) if (m->cn[(long)j * N + i] >= 0) nnz++;
    }
    m->csr_ptr[N] = nnz;
    m->csr_j = iz_(nnz); m->csr_slot = iz_(nnz); m->csr_val = dz_(nnz);
    for (int i = 0; i < N; i++) {
      long q = m->csr_ptr[i];
      m->csr_j[q] = i; m->csr_slot[q] = -1; q++;
      for (int j = 0; j < m->ncf[i]; j++) {
        int k = m->cn[(long)j * N + i];
        if (k >= 0) { m->csr_j[q] = k; m->csr_slot[q] = j; q++; }
      }
    }
    m->kx = dz_(N); m->kr = dz_(N); m->kb = dz_(N);
    m->csr_built = 1;
  }
  for (int i = 0; i < N; i++) {
    long q = m->csr_ptr[i];
    m->csr_val[q] = m->ac[i];
    for (q = q + 1; q < m->csr_ptr[i + 1]; q++) m->csr_val[q] = m->anb[(long)m->csr_slot[q] * N + i];
  }
}

/* AxOMP (matrixSolverOMP.f90:390-423): the one loop of the reference that
 * runs on several threads (its OpenMP loop over rows, statically split; here
 * POSIX threads over equal row ranges).  Every row is summed as in the
 * sequential loop, so the result does not depend on the thread count.  The
 * dot products of BICGSTAB_OMP sit in orphaned WORKSHARE constructs outside
 * any parallel region, which one thread executes: they stay sequential. */
static int g_axomp_threads = 1;
typedef struct { const om *m; const double *x; double *y; int i0, i1; } ax_job;

static void ax_rows(const om *m, const double *x, double *y, int i0, int i1)
{
  for (int i = i0; i < i1; i++) {
    double t = 0.0;
    for (long q = m->csr_ptr[i]; q < m->csr_ptr[i + 1]; q++) t = t + m->csr_val[q] * x[m->csr_j[q]];
    y[i] = t;
  }
}

static void *ax_thread(void *p)
{
  ax_job *j = (ax_job *)p;
  ax_rows(j->m, j->x, j->y, j->i0, j->i1);
  return NULL;
}

static void axomp(const om *m, const double *x, double *y)
{
  int T = g_axomp_threads;
  if (T <= 1 || m->N < 65536) { ax_rows(m, x, y, 0, m->N); return; }
  if (T > 256) T = 256;
  pthread_t th[256];
  ax_job jb[256];
  int started = 0;
  for (int t = 0; t < T; t++) {
    jb[t].m = m; jb[t].x = x; jb[t].y = y;
    jb[t].i0 = (int)((long)m->N * t / T); jb[t].i1 = (int)((long)m->N * (t + 1) / T);
    if (t == 0) continue;
    if (pthread_create(&th[t], NULL, ax_thread, &jb[t]) != 0) { ax_rows(m, x, y, jb[t].i0, jb[t].i1); jb[t].i0 = -1; }
    else started++;
  }
  ax_rows(m, x, y, jb[0].i0, jb[0].i1);
  for (int t = 1; t < T; t++) if (jb[t].i0 >= 0) pthread_join(th[t], NULL);
  (void)started;
}

static double dot(const double *a, const double *b, int n)
{
  double s = 0.; for (int i = 0; i < n; i++) s += a[i] * b[i]; return s;
}

/* BICGSTAB_OMP (matrixSolverOMP.f90:306-386) on the CSR of ac/anb/bc */
int om_bicgstab(om *m, int nIter, double res)
{
  int n = m->N;
  csr_build(m);
  memcpy(m->kb, m->bc, sizeof(double) * n);
  double *x = m->kx, *r = m->kr, *b = m->kb;
  double *r0 = dz_(n), *p = dz_(n), *s = dz_(n), *v = dz_(n), *As = dz_(n);
  axomp(m, x, r0);
  for (int i = 0; i < n; i++) { r0[i] = b[i] - r0[i]; r[i] = r0[i]; }
  double rhoPrev = dot(r, r0, n);
  double resnorm = sqrt(fabs(rhoPrev));
  memcpy(p, r0, sizeof(double) * n);
  double normb = sqrt(dot(b, b, n));
  int k = 1;
  while (k < nIter && resnorm > res * normb) {
    k = k + 1;
    axomp(m, p, v);
    double dp0 = dot(v, r0, n);
    double alpha = rhoPrev / dp0;
    for (int i = 0; i < n; i++) s[i] = r[i] - alpha * v[i];
    axomp(m, s, As);
    double dp1 = dot(As, s, n), dp2 = dot(As, As, n);
    double omega = dp1 / dp2;
    for (int i = 0; i < n; i++) { x[i] = x[i] + alpha * p[i] + omega * s[i]; r[i] = s[i] - omega * As[i]; }
    double rho = dot(r, r0, n);
    double beta = (rho / rhoPrev) * (alpha / omega); rhoPrev = rho;
    for (int i = 0; i < n; i++) p[i] = r[i] + beta * (p[i] - omega * v[i]);
    resnorm = sqrt(fabs(rho));
  }
  free(r0); free(p); free(s); free(v); free(As);
  memcpy(m->dphi, x, sizeof(double) * n);     /* dphi=x */
  return k - 1;
}

/* GMRES_RESTARTED_OMP_RETURNR (matrixSolverOMP.f90:48-304) with the caller's
 * parameters GMRES_ninner=20, GMRES_nouter=1000, GMRES_tol=1e-9
 * (matrixSolverOMP.f90:4-6,604): the system is normalised by |b|; restart
 * lengths mm = 5, 10, 15, 20 (each round from x = 0: resetFlag is never
 * cleared, :81,120); within a round, Arnoldi with modified Gram-Schmidt and
 * Givens rotations (:145-181), the best iterate kept (:219-229), and the
 * restart length reduced by 5 (above 10) or 1 when a cycle gains less than
 * 10 % or loses (:231-238); a round with m = 1 ends when a cycle gains less
 * than 1 % or after 100 cycles (:215-216).  The next round runs only if this
 * one improved the best residual (:256-263).  A zero right-hand side gives
 * x = 0 (the reference divides by |b| = 0).  Returns the Arnoldi steps. */
int om_gmres(om *m)
{
  const int n = m->N, mMax = 20;
  const double res = 1.0e-9;
  csr_build(m);
  double *b = dz_(n), *x = m->kx, *r = m->kr;
  memcpy(b, m->bc, sizeof(double) * n);
  double normb0 = sqrt(dot(b, b, n));
  int total = 0;
  if (normb0 == 0.) {
    memset(x, 0, sizeof(double) * n);
    memcpy(m->dphi, x, sizeof(double) * n);
    free(b);
    return 0;
  }
  for (int i = 0; i < n; i++) b[i] = b[i] / normb0;
  const double normb = 1.0;
  double *w = dz_(n), *x1 = dz_(n), *xOpt = dz_(n), *rOpt = dz_(n), *xG = dz_(n), *rG = dz_(n);
  double *V = dz_((size_t)n * (mMax + 1));
  double H[21][20], g[21], c[20], s[20], y[20];
  double normminG = 1.0e30;
  int mm = 5;
  while (mm <= mMax) {
    double normmin = 1.0e30;
    int mcur = mm, iter = 0, leave = 0;
    memset(x, 0, sizeof(double) * n);
    memcpy(r, b, sizeof(double) * n);
    double normr = sqrt(dot(r, r, n));
    double normrPrev = normr;
    while (normmin > res * normb && leave == 0) {
      iter++;
      int mloc = mcur;
      for (int i = 0; i < n; i++) V[i] = r[i] / normr;
      for (int a = 0; a <= mMax; a++) { g[a] = 0.; for (int q = 0; q < mMax; q++) H[a][q] = 0.; }
      g[0] = normr;
      for (int j = 0; j < mloc; j++) {
        total++;
        axomp(m, V + (size_t)j * n, w);
        for (int i = 0; i <= j; i++) {
          H[i][j] = dot(w, V + (size_t)i * n, n);
          const double h = H[i][j], *vi = V + (size_t)i * n;
          for (int q = 0; q < n; q++) w[q] = w[q] - h * vi[q];
        }
        H[j + 1][j] = sqrt(dot(w, w, n));
        if (H[j + 1][j] == 0.) { mloc = j + 1; break; }
        for (int q = 0; q < n; q++) V[(size_t)(j + 1) * n + q] = w[q] / H[j + 1][j];
        for (int i = 0; i < j; i++) {
          double hi = c[i] * H[i][j] + s[i] * H[i + 1][j], hi1 = -s[i] * H[i][j] + c[i] * H[i + 1][j];
          H[i][j] = hi; H[i + 1][j] = hi1;
        }
        double d = sqrt(H[j][j] * H[j][j] + H[j + 1][j] * H[j + 1][j]);
        s[j] = H[j + 1][j] / d; c[j] = H[j][j] / d;
        for (int q = 0; q < mloc; q++) {
          double hj = c[j] * H[j][q] + s[j] * H[j + 1][q], hj1 = -s[j] * H[j][q] + c[j] * H[j + 1][q];
          H[j][q] = hj; H[j + 1][q] = hj1;
        }
        double gj = c[j] * g[j] + s[j] * g[j + 1], gj1 = -s[j] * g[j] + c[j] * g[j + 1];
        g[j] = gj; g[j + 1] = gj1;
      }
      mcur = mloc;
      y[mcur - 1] = g[mcur - 1] / H[mcur - 1][mcur - 1];
      for (int j = mcur - 2; j >= 0; j--) {
        double dp = 0.;
        for (int q = j + 1; q < mcur; q++) dp += H[j][q] * y[q];
        y[j] = (g[j] - dp) / H[j][j];
      }
      for (int i = 0; i < n; i++) {
        double t = 0.;
        for (int q = 0; q < mcur; q++) t += V[(size_t)q * n + i] * y[q];
        w[i] = t;
      }
      for (int i = 0; i < n; i++) x1[i] = x[i] + w[i];
      axomp(m, x1, r);
      for (int i = 0; i < n; i++) r[i] = b[i] - r[i];
      normr = sqrt(dot(r, r, n));
      if ((normr - normrPrev) / normrPrev > -0.01 && mcur == 1) leave = 1;
      if (mcur == 1 && iter > 100) leave = 1;
      if (normr < normmin) {
        normmin = normr;
        memcpy(xOpt, x1, sizeof(double) * n);
        memcpy(rOpt, r, sizeof(double) * n);
      }
      if (normr < normrPrev) memcpy(x, x1, sizeof(double) * n);
      else { memcpy(x, xOpt, sizeof(double) * n); memcpy(r, rOpt, sizeof(double) * n); }
      if ((fabs((normr - normrPrev) / normr) < 0.1 || normr > normrPrev) && mcur > 1) {
        mcur = mcur > 10 ? mcur - 5 : mcur - 1;
        iter = 0;
      }
      normrPrev = normr;
    }
    if (normmin < normminG) {
      normminG = normmin;
      memcpy(xG, xOpt, sizeof(double) * n);
      memcpy(rG, rOpt, sizeof(double) * n);
      mm += 5;
    } else {
      mm = mMax + 5;
    }
    if (normminG <= res) mm = mMax + 5;
  }
  for (int i = 0; i < n; i++) x[i] = xG[i] * normb0;
  memcpy(m->dphi, x, sizeof(double) * n);     /* dphi=x */
  free(b); free(w); free(x1); free(xOpt); free(rOpt); free(xG); free(rG); free(V);
  return total;
}

int om_mg_solve(om *m, double rrF, double IRes);   /* below */

/* SolveEquation (SolveAlegbraicEquations.for:4-180) */
void om_solve_equation(om *m, int nf, double *fi, double rrf, int itmax, int solver)
{
  int N = m->N;
  memset(m->dphi, 0, sizeof(double) * N);
  om_calc_residuals(m, nf, fi);
  double IRes = m->rabs[nf - 1], FRes = IRes;
  int iter = 0;
  if (solver == FS_SOLVER_SOR) {
    while (FRes > rrf * IRes && iter < itmax) { sor_sweep(m); FRes = check_convergence(m); iter++; }
  } else if (solver == FS_SOLVER_ILU) {   /* SolveAlegbraicEquations.for:122-133 */
    ilu_factor(m);
    while (FRes > rrf * IRes && iter < itmax) { ilu_sweep(m); FRes = check_convergence(m); iter++; }
  } else if (solver == FS_SOLVER_PBCG) {  /* SolveAlegbraicEquations.for:138-152 */
    struct om_pbcg w;
    w.p = dz_(N); w.pp = dz_(N); w.r = dz_(N); w.rr = dz_(N); w.z = dz_(N); w.zz = dz_(N); w.bkden = 0.;
    ilu_factor(m);
    while (FRes > rrf * IRes && iter < itmax) { pbcg_step(m, &w, iter); FRes = check_convergence(m); iter++; }
    free(w.p); free(w.pp); free(w.r); free(w.rr); free(w.z); free(w.zz);
  } else if (solver == FS_SOLVER_BICGS) {
    iter = om_bicgstab(m, m->cfg.krylov_maxit, m->cfg.krylov_tol);
  } else if (solver == FS_SOLVER_AMG) {
    iter = om_mg_solve(m, rrf, IRes);
  } else if (solver == FS_SOLVER_GMRES) {
    iter = om_gmres(m);
  } else {
    fprintf(stderr, "oracle: solver %d not restated\n", solver);
  }
  m->lin_iters[nf - 1] = iter;
  for (int i = 0; i < N; i++) fi[i] = fi[i] + m->dphi[i];
}

/* ===================================================================== */
/*  k-epsilon (Turbulence/)                                               */
/* ===================================================================== */
#include "oracle_turb.inc"
#include "oracle_energy.inc"

/* ===================================================================== */
/*  Stop metric (PrintConvergenceToFileAndScreen.for:613-700)             */
/* ===================================================================== */
static double stop_metric(om *m)
{
  const double *r = m->cfg.nstop_type == 1 ? m->rabs : m->cfg.nstop_type == 2 ? m->rmax :
                    m->cfg.nstop_type == 3 ? m->rrms : m->rscl;
  double s = 0.;
  s = fmax(s, fmax(fabs(r[0]), fmax(fabs(r[1]), fabs(r[2]))));
  s = fmax(s, fabs(r[4]));
  if (m->cfg.turbulence) { s = fmax(s, fabs(r[7])); s = fmax(s, fabs(r[8])); }
  if (m->cfg.energy) s = fmax(s, fabs(r[FS_VAR_TEMP - 1]));
  return s;
}

double om_simple_iteration(om *m)
{
  m->nIter++;
  om_momentum(m, 0); om_momentum(m, 1); om_momentum(m, 2);
  om_continuity(m);
  if (m->cfg.turbulence) om_effects_of_turbulence(m);
  if (m->cfg.energy) om_solve_temperature(m);   /* SolveEnergy (MainProgram.for:281) */
  return stop_metric(m);
}

/* CalculateStrainRateTensor + CalculateTurbulenceProduction on the current
 * velocity gradients, k, epsilon and mu_t (into "prod"), for the unit tests */
void om_turb_production(om *m) { om_strain_rate(m); om_production(m); }

/* SolveEnergy alone, on the current mdot and velocities */
void om_energy(om *m) { om_solve_temperature(m); }

void om_residuals_temp(om *m, double out[4])
{
  int q = FS_VAR_TEMP - 1;
  out[0] = m->rabs[q]; out[1] = m->rmax[q]; out[2] = m->rrms[q]; out[3] = m->rscl[q];
}

void om_residuals_turb(om *m, double out[8])
{
  for (int q = 0; q < 2; q++) { out[q] = m->rabs[7 + q]; out[2 + q] = m->rmax[7 + q]; out[4 + q] = m->rrms[7 + q]; out[6 + q] = m->rscl[7 + q]; }
}

/* CalculateInitialmdot (InitializaMdot.for:20-60), Densityf = rho */
void om_initialize_mdot(om *m)
{
  const fs_case *cfg = &m->cfg;
  for (int k = 0; k < m->F; k++) {
    double uf = m->gf[k] * m->u[m->if_own[k]] + (1. - m->gf[k]) * m->u[m->if_nbr[k]];
    double vf = m->gf[k] * m->v[m->if_own[k]] + (1. - m->gf[k]) * m->v[m->if_nbr[k]];
    double wf = m->gf[k] * m->w[m->if_own[k]] + (1. - m->gf[k]) * m->w[m->if_nbr[k]];
    m->mdot[k] = cfg->rho * (uf * m->sx[k] + vf * m->sy[k] + wf * m->sz[k]);
  }
  for (int b = 0; b < m->B; b++) {
    if (m->btype[b] == FS_BC_WALL_NOSLIP || m->btype[b] == FS_BC_WALL_SLIP) m->bmdot[b] = 0.;
    else if (m->btype[b] == FS_BC_INLET_MASS || m->btype[b] == FS_BC_OUTLET_MASS) continue;   /* specified (InitializaMdot.for:55,66) */
    else m->bmdot[b] = cfg->rho * (m->bsx[b] * m->bu[b] + m->bsy[b] * m->bv[b] + m->bsz[b] * m->bw[b]);
  }
}

void om_set_iter(om *m, int nIter) { m->nIter = nIter; }

/* threads of the AxOMP loop (OMP_NUM_THREADS of the reference build; 1 by
 * default); returns the count in effect */
int om_set_threads(int n)
{
  if (n > 0) g_axomp_threads = n;
  return g_axomp_threads;
}
void om_residuals(om *m, double out[20])
{
  for (int q = 0; q < 5; q++) { out[q] = m->rabs[q]; out[5 + q] = m->rmax[q]; out[10 + q] = m->rrms[q]; out[15 + q] = m->rscl[q]; }
}
int om_lin_iters(om *m, int nf) { return m->lin_iters[nf - 1]; }

/* ===================================================================== */
/*  Multigrid (AlgebraicMultiGrid/) -- see oracle_mg.c                    */
/* ===================================================================== */
#include "oracle_mg.inc"

/* ===================================================================== */
/*  Create / arrays                                                       */
/* ===================================================================== */
om *om_create(const fs_mesh_in *mi, const fs_case *cfg)
{
  om *m = (om *)calloc(1, sizeof(om));
  m->cfg = *cfg;
  long np = (long)mi->n_nodes * 3, nq = mi->face_ptr[mi->n_faces];
  m->pts = dz_(np); memcpy(m->pts, mi->points, sizeof(double) * np);
  m->face_ptr = iz_(mi->n_faces + 1); memcpy(m->face_ptr, mi->face_ptr, sizeof(int) * (mi->n_faces + 1));
  m->face_nodes = iz_(nq); memcpy(m->face_nodes, mi->face_nodes, sizeof(int) * nq);
  om_connectivity(m, mi);
  om_geometry(m);
  int N = m->N, F = m->F, B = m->B;
  m->btype = iz_(B);
  double *bvx = dz_(B), *bvy = dz_(B), *bvz = dz_(B);
  for (int b = 0; b < B; b++) {
    int s = m->bf_set[b];
    m->btype[b] = cfg->patch_type[s];
    if (cfg->patch_type[s] == FS_BC_WALL_NOSLIP || cfg->patch_type[s] == FS_BC_INLET_VEL) {
      bvx[b] = cfg->patch_vel[s][0]; bvy[b] = cfg->patch_vel[s][1]; bvz[b] = cfg->patch_vel[s][2];
    }
  }
  m->u = dz_(N); m->v = dz_(N); m->w = dz_(N); m->p = dz_(N); m->pc = dz_(N); m->mdot = dz_(F);
  m->bu = bvx; m->bv = bvy; m->bw = bvz; m->bp = dz_(B); m->bpc = dz_(B); m->bmdot = dz_(B);
  /* specified static pressure on its outlets; SetReferencePressure
   * (ReferenceAndSetPressureRoutines.for:4-50): a pressure-specified patch
   * fixes the level, no reference cell */
  int has_sp = 0;
  m->bp0 = dz_(B); m->bgd = dz_(B);
  for (int b = 0; b < B; b++) if (OM_PRESSURE(m->btype[b])) {
    m->bp[b] = cfg->patch_pressure[m->bf_set[b]]; m->bp0[b] = m->bp[b]; has_sp = 1;
  }
  if (m->cfg.set_reference_pressure < 0) m->cfg.set_reference_pressure = has_sp;
  m->ug = dz_(3L*N); m->vg = dz_(3L*N); m->wg = dz_(3L*N); m->pg = dz_(3L*N); m->pcg = dz_(3L*N);
  m->bug = dz_(3L*B); m->bvg = dz_(3L*B); m->bwg = dz_(3L*B); m->bpg = dz_(3L*B); m->bpcg = dz_(3L*B);
  m->ugf = dz_(3L*F); m->vgf = dz_(3L*F); m->wgf = dz_(3L*F); m->pgf = dz_(3L*F);
  m->du1 = dz_(N); m->dv1 = dz_(N); m->dw1 = dz_(N); m->du2 = dz_(N); m->dv2 = dz_(N); m->dw2 = dz_(N);
  m->us = dz_(N); m->vs = dz_(N); m->ws = dz_(N); m->gstar = dz_(3L*N);
  m->fcf = dz_(F + B); m->fff = dz_(F + B); m->fvf = dz_(F + B); m->ftf = dz_(F + B);
  m->fce = dz_(N); m->fte = dz_(N); m->effdiv = dz_(N);
  m->ac = dz_(N); m->bc = dz_(N); m->dphi = dz_(N); m->anb = dz_((long)N * m->W);
  m->mdot1 = dz_(m->NS); m->mdot_out = dz_(m->NS);
  m->edif = dz_(N); m->bedif = dz_(B);
  m->tke = dz_(N); m->ted = dz_(N); m->mut = dz_(N); m->btke = dz_(B); m->bted = dz_(B); m->bmut = dz_(B);
  m->tkeg = dz_(3L*N); m->tedg = dz_(3L*N); m->btkeg = dz_(3L*B); m->btedg = dz_(3L*B);
  m->tkegf = dz_(3L*F); m->tedgf = dz_(3L*F);
  m->prod = dz_(N); m->bprod = dz_(B);
  m->s11 = dz_(N); m->s12 = dz_(N); m->s13 = dz_(N); m->s22 = dz_(N); m->s23 = dz_(N); m->s33 = dz_(N);
  m->rhok = dz_(N); m->brhok = dz_(B); m->drk = dz_(3L*N); m->bdrk = dz_(3L*B);
  m->wdist = dz_(N); m->itau = iz_(N);
  m->utau = dz_(B); m->yplus = dz_(B); m->uplus = dz_(B); m->dupdyp = dz_(B); m->tauw = dz_(B); m->wallvisc = dz_(B);
  om_wall_distance(m);
  /* 'specifiedmassflowrate' inlets: direction per face, Bmdot = -mdot |S_f| / sum |S| in face order */
  m->bdir = dz_(3L * B);
  for (int s = 0; s < m->NS; s++) if (OM_P_INLET(cfg->patch_type[s]))
    for (int j = 0; j < m->bset_n[s]; j++)
      for (int q = 0; q < 3; q++) m->bdir[3L * (m->bset_start[s] + j) + q] = cfg->patch_vel[s][q];
  for (int s = 0; s < m->NS; s++) if (cfg->patch_type[s] == FS_BC_OUTLET_MASS) {   /* outflow: Bmdot > 0 */
    double area = 0.;
    for (int j = 0; j < m->bset_n[s]; j++) area = area + m->bfa[m->bset_start[s] + j];
    for (int j = 0; j < m->bset_n[s]; j++) m->bmdot[m->bset_start[s] + j] = cfg->patch_mass_flow[s] * m->bfa[m->bset_start[s] + j] / area;
  }
  for (int s = 0; s < m->NS; s++) if (cfg->patch_type[s] == FS_BC_INLET_MASS) {
    double area = 0.;
    for (int j = 0; j < m->bset_n[s]; j++) area = area + m->bfa[m->bset_start[s] + j];
    for (int j = 0; j < m->bset_n[s]; j++) {
      int b = m->bset_start[s] + j;
      const double *d = m->bdir + 3L * b;
      for (int q = 0; q < 3; q++) m->bdir[3L * b + q] = cfg->patch_vel[s][q];
      m->bmdot[b] = -(cfg->patch_mass_flow[s] * m->bfa[b] / area);
      double vm = m->bmdot[b] / (cfg->rho * (d[0] * m->bsx[b] + d[1] * m->bsy[b] + d[2] * m->bsz[b]));
      m->bu[b] = vm * d[0]; m->bv[b] = vm * d[1]; m->bw[b] = vm * d[2];
    }
  }
  om_initialize_mdot(m);
  om_energy_init(m);
  om_transient_init(m);
  return m;
}

void om_destroy(om *m)
{
  if (!m) return;
  /* process exit reclaims the rest; the oracle is short-lived test code */
  free(m);
}

int om_sizes(om *m, int *N, int *F, int *B, int *W)
{
  *N = m->N; *F = m->F; *B = m->B; *W = m->W; return 0;
}

void *om_array(om *m, const char *name, long *len, int *is_int)
{
  long N = m->N, F = m->F, B = m->B, W = m->W;
  struct { const char *n; void *p; long len; int isint; } t[] = {
    {"u", m->u, N, 0}, {"v", m->v, N, 0}, {"w", m->w, N, 0}, {"p", m->p, N, 0}, {"pc", m->pc, N, 0},
    {"mdot", m->mdot, F, 0}, {"bu", m->bu, B, 0}, {"bv", m->bv, B, 0}, {"bw", m->bw, B, 0},
    {"bp", m->bp, B, 0}, {"bpc", m->bpc, B, 0}, {"bmdot", m->bmdot, B, 0},
    {"ug", m->ug, 3*N, 0}, {"vg", m->vg, 3*N, 0}, {"wg", m->wg, 3*N, 0}, {"pg", m->pg, 3*N, 0}, {"pcg", m->pcg, 3*N, 0},
    {"bug", m->bug, 3*B, 0}, {"bvg", m->bvg, 3*B, 0}, {"bwg", m->bwg, 3*B, 0}, {"bpg", m->bpg, 3*B, 0}, {"bpcg", m->bpcg, 3*B, 0},
    {"ugf", m->ugf, 3*F, 0}, {"vgf", m->vgf, 3*F, 0}, {"wgf", m->wgf, 3*F, 0}, {"pgf", m->pgf, 3*F, 0},
    {"du1", m->du1, N, 0}, {"dv1", m->dv1, N, 0}, {"dw1", m->dw1, N, 0},
    {"du2", m->du2, N, 0}, {"dv2", m->dv2, N, 0}, {"dw2", m->dw2, N, 0},
    {"us", m->us, N, 0}, {"vs", m->vs, N, 0}, {"ws", m->ws, N, 0},
    {"ac", m->ac, N, 0}, {"bc", m->bc, N, 0}, {"anb", m->anb, N*W, 0}, {"dphi", m->dphi, N, 0},
    {"fcf", m->fcf, F+B, 0}, {"fff", m->fff, F+B, 0}, {"ftf", m->ftf, F+B, 0},
    {"vol", m->vol, N, 0}, {"xc", m->xc, N, 0}, {"yc", m->yc, N, 0}, {"zc", m->zc, N, 0},
    {"gf", m->gf, F, 0}, {"sx", m->sx, F, 0}, {"sy", m->sy, F, 0}, {"sz", m->sz, F, 0},
    {"fa", m->fa, F, 0}, {"fcx", m->fcx, F, 0}, {"fcy", m->fcy, F, 0}, {"fcz", m->fcz, F, 0},
    {"dcf", m->dcf, F, 0}, {"gdiff", m->gdiff, F, 0}, {"Tx", m->Tx, F, 0}, {"Ty", m->Ty, F, 0}, {"Tz", m->Tz, F, 0},
    {"Ex", m->Ex, F, 0}, {"Ey", m->Ey, F, 0}, {"Ez", m->Ez, F, 0},
    {"bsx", m->bsx, B, 0}, {"bsy", m->bsy, B, 0}, {"bsz", m->bsz, B, 0}, {"bfa", m->bfa, B, 0},
    {"bfcx", m->bfcx, B, 0}, {"bfcy", m->bfcy, B, 0}, {"bfcz", m->bfcz, B, 0},
    {"bdx", m->bdx, B, 0}, {"bdy", m->bdy, B, 0}, {"bdz", m->bdz, B, 0}, {"bgdiff", m->bgdiff, B, 0},
    {"bTx", m->bTx, B, 0}, {"bTy", m->bTy, B, 0}, {"bTz", m->bTz, B, 0},
    {"ncf", m->ncf, N, 1}, {"cf", m->cf, N*W, 1}, {"cn", m->cn, N*W, 1},
    {"own_slot", m->own_slot, F, 1}, {"nbr_slot", m->nbr_slot, F, 1},
    {"if_own", m->if_own, F, 1}, {"if_nbr", m->if_nbr, F, 1}, {"bf_own", m->bf_own, B, 1},
    {"btype", m->btype, B, 1}, {"kx", m->kx, m->kx ? N : 0, 0}, {"ilu_dc", m->ilu_dc, m->ilu_dc ? N : 0, 0},
    {"tke", m->tke, N, 0}, {"ted", m->ted, N, 0}, {"mut", m->mut, N, 0},
    {"btke", m->btke, B, 0}, {"bted", m->bted, B, 0}, {"bmut", m->bmut, B, 0},
    {"tkeg", m->tkeg, 3*N, 0}, {"tedg", m->tedg, 3*N, 0}, {"prod", m->prod, N, 0},
    {"edif", m->edif, N, 0}, {"bedif", m->bedif, B, 0}, {"drk", m->drk, 3*N, 0},
    {"wdist", m->wdist, N, 0}, {"itau", m->itau, N, 1},
    {"utau", m->utau, B, 0}, {"yplus", m->yplus, B, 0}, {"uplus", m->uplus, B, 0},
    {"dupdyp", m->dupdyp, B, 0}, {"wallvisc", m->wallvisc, B, 0}, {"bprod", m->bprod, B, 0},
    {"old", m->old, OM_NLEVELS*N, 0}, {"oldold", m->oldold, OM_NLEVELS*N, 0}, {"bold", m->bold, OM_NLEVELS*B, 0},
    {"temp", m->tmp, N, 0}, {"btemp", m->btmp, B, 0}, {"tempg", m->tmpg, 3*N, 0}, {"btempg", m->btmpg, 3*B, 0},
  };
  for (unsigned q = 0; q < sizeof(t) / sizeof(t[0]); q++)
    if (strcmp(t[q].n, name) == 0) { *len = t[q].len; *is_int = t[q].isint; return t[q].p; }
  *len = 0; *is_int = 0; return NULL;
}
