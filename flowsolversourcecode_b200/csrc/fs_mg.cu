// fs_mg.cu -- element-agglomeration multigrid on the GPU.
//
// Hierarchy (host, once per context): AgglomorateLevelGeometricallyElement
// (AlgebraicMultiGrid/AgglomorateALevelGeometricallyElementBased.for:4-318)
// restated in C++ -- greedy seeds in cell order, immediate neighbours, then
// neighbours of neighbours, capped at 8/4/3/2 children by level, orphans
// joined with and then without the cap -- and the coarse connectivity in the
// reference's discovery order.  Coarsening stops as in Agglomorate
// (AgglomorateGrid.for:36-72).  The parent maps depend on connectivity only.
//
// Per solve: coarse matrices by a per-parent gather (AssembleElementBasedAgglomoratedLHS.for:45-150)
// in the reference's summation order (seed, then children, each with its
// slots), so they are bit-identical to the CPU restatement.
//
// Cycles run inside ONE persistent cooperative kernel.  Levels with more than
// FS_MG_SMALL rows are processed by the whole grid (grid barriers between
// colours of the Gauss-Seidel sweeps); smaller levels by CTA 0 alone with
// block barriers, so the coarse tail of a cycle costs no grid barriers.  A
// phase of a latency-bound sweep costs about one dependent-load chain per row a
// thread handles, so CTA 0 wins below ~8 rows per thread (2048 rows).
//   k_mg_solve      : AlgebraicMultigrid (AlgebraicMultiGridMainRoutine.for:330-345)
//                     with V/F/W cycles (MultiGridCycle.for), smoothing sweeps
//                     that stop on sum|r| <= rrF*IResiduals (SolveEquationsWithMultiGrid.for),
//                     multicolour symmetric Gauss-Seidel in place of the
//                     sequential sweep, coarse corrections kept between cycles
//                     as the reference does.
//   k_amg_bicgstab  : FP64 BiCGSTAB right-preconditioned by one V-cycle
//                     (PCycle: damped Jacobi, fused restrict/prolong phases,
//                     dense FP64 inverse of the coarsest level) -- no reference
//                     row; templated on the V-cycle precision (double, or float
//                     with FP32 copies of every level's matrix: iterative
//                     refinement).
#include "fs_internal.cuh"
#include <cooperative_groups.h>
#include <algorithm>
#include <cstring>
#include <type_traits>

namespace cg = cooperative_groups;

#define FS_MG_SMALL 2048
#define FS_MG_DIRECT 160   // largest coarsest level inverted densely (n^2 doubles in shared memory)
#define FS_MG_MAXLEV 16
#define FS_SUMK (FS_GUESS_MAX * (FS_GUESS_MAX + 1) / 2 + FS_GUESS_MAX + 1)   // sums of the guess fit
// preconditioner V-cycle: Jacobi weight and coarse-correction factor
// (over-correction compensates the energy of piecewise-constant prolongation)
#ifndef FS_MG_OMEGA
#define FS_MG_OMEGA 0.9
#endif
// CTAs per SM the preconditioned Krylov kernel is compiled for (register cap)
#ifndef FS_AMG_MINB
#define FS_AMG_MINB 1
#endif
#ifndef FS_MG_ALPHA
#define FS_MG_ALPHA 1.8
#endif
// level 0 (the fine matrix) may take its own weight and correction factor
#ifndef FS_MG_OMEGA0
#define FS_MG_OMEGA0 0.8
#endif
#ifndef FS_MG_ALPHA0
#define FS_MG_ALPHA0 FS_MG_ALPHA
#endif

template <class R>
struct LevelDev {
  int n, w, ncolors;
  const int32_t *ncf, *nbr, *color_ptr, *color_rows;
  const R *ac, *anb;
  R *b, *x, *r, *t;
  const int32_t *parent;        // this level -> next coarser (nullptr on the coarsest)
  const int32_t *rptr, *rlist;  // restriction into this level: finer rows per coarse row, ascending
  // warp chunks of this level's rows for the fused restriction into it:
  // chunk k is rows [chunk[k], chunk[k+1]), at most 32 rows and, unless one
  // row alone has more, at most 64 finer rows (children) in all
  const int32_t *chunk;
  int nchunk;
};

template <class R>
struct AmgKArgs {
  int N, W;
  const int32_t *ncf, *cn;
  const double *ac, *anb, *bc;
  double *x, *r, *r0, *p, *v, *s, *t, *y, *z, *dphi;
  const LevelDev<R> *lev;
  int lc, direct, pre, post, maxit;
  const double *sinv;
  double tol;
  double *part;
  int32_t *iters;
  double *diag;
  const double *xs[FS_GUESS_MAX];   // initial-guess basis: previous p' solutions, the network's guess
  int nx;             // vectors in xs (0: zero start)
  int32_t *fit;       // [0]: k_guess_fit found a guess (device)
  int32_t *nncnt;     // [fallbacks, uses] of the initial guess, or nullptr
  unsigned *teambar;  // team barrier words of the V-cycle (zeroed before the launch)
  int32_t *status;    // [0] team-barrier timeout flag
  int team_extra;     // fs_test_wait_timeout
};

struct fs_mg_dev {
  int nlev = 0;
  int n[FS_MG_MAXLEV] = {}, w[FS_MG_MAXLEV] = {}, ncol[FS_MG_MAXLEV] = {};
  std::vector<int32_t> h_parent[FS_MG_MAXLEV];
  // device
  int32_t *nnb[FS_MG_MAXLEV] = {}, *nbr[FS_MG_MAXLEV] = {}, *parent[FS_MG_MAXLEV] = {};
  int32_t *cptr[FS_MG_MAXLEV] = {}, *clist[FS_MG_MAXLEV] = {}, *cmap[FS_MG_MAXLEV] = {};
  int32_t *rptr[FS_MG_MAXLEV] = {}, *rlist[FS_MG_MAXLEV] = {};
  int32_t *colors[FS_MG_MAXLEV] = {};   // rows by colour, then ncol+1 offsets
  int32_t *chunk[FS_MG_MAXLEV] = {};    // warp chunks of coarse rows (fused restriction)
  int nchunk[FS_MG_MAXLEV] = {};
  double *ac[FS_MG_MAXLEV] = {}, *anb[FS_MG_MAXLEV] = {}, *b[FS_MG_MAXLEV] = {}, *x[FS_MG_MAXLEV] = {}, *r[FS_MG_MAXLEV] = {};
  double *t[FS_MG_MAXLEV] = {};
  float *acf[FS_MG_MAXLEV] = {}, *anbf[FS_MG_MAXLEV] = {}, *bf[FS_MG_MAXLEV] = {}, *xf[FS_MG_MAXLEV] = {}, *rf[FS_MG_MAXLEV] = {};
  float *tf[FS_MG_MAXLEV] = {};
  int lc = 0;                           // coarsest level of the preconditioner
  bool direct = false;                  // lev[lc] inverted densely
  double *sinv = nullptr;
  LevelDev<double> *lev64 = nullptr;
  LevelDev<float> *lev32 = nullptr;
  double *red = nullptr;                // partial sums
  int per_sm = 0;                       // co-resident CTAs per SM of the multigrid kernels
  // preconditioner reuse (pc_refresh): the system and precision the coarse
  // levels and the dense inverse were last built for, and the solves since
  int built_nf = 0, age = 0;
  bool built_f32 = false;
  // the Krylov launch a deferred solve prepared (pc_defer): its arguments and
  // form (fs_pc_batch_form), for fs_pc_batch_launch
  AmgKArgs<double> pend64{};
  AmgKArgs<float> pend32{};
  int pend_form = -1;
};

namespace {

// ---------------------------------------------------------------- device helpers
__device__ __forceinline__ double wsum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
// block sum broadcast to the whole block
__device__ double bsum(double v) {
  __shared__ double sh[33];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = wsum(v);
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    double r = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.;
    r = wsum(r);
    if (lane == 0) sh[32] = r;
  }
  __syncthreads();
  double r = sh[32];
  __syncthreads();
  return r;
}


// V-cycle work split (PCycle): levels up to FS_PC_SMALL rows on CTA 0 alone,
// up to FS_PC_TEAM_MAX rows on a team of the first FS_PC_TEAM CTAs with a
// bounded barrier of its own, larger ones on every CTA
#ifndef FS_PC_TEAM
#define FS_PC_TEAM 32
#endif
#define FS_PC_SMALL 256
#ifndef FS_PC_TEAM_MAX
#define FS_PC_TEAM_MAX 4096   // levels up to this many rows run on the CTA team
#endif
#define FS_PC_SPIN_LIMIT (1L << 20)   // polls of a team barrier before it reports a timeout
#ifndef FS_PC_GS_LEVELS
#define FS_PC_GS_LEVELS 1     // amg32gs_bicgs: Gauss-Seidel on the levels below this one, Jacobi above
#endif
#ifndef FS_PC_FUSE_DOWN
#define FS_PC_FUSE_DOWN 0     // restrictions from levels below this one form the residual on the fly
#endif

// the same Krylov/V-cycle code for one system on the whole grid (g1) and for
// groups of CTAs that each solve their own system (gb)
namespace g1 {
#define FS_GROUPS 0
#include "fs_amg_core.cuh"
#undef FS_GROUPS
}  // namespace g1
namespace gb {
#define FS_GROUPS 1
#include "fs_amg_core.cuh"
#undef FS_GROUPS
}  // namespace gb
using namespace g1;

template <class R>
__device__ __forceinline__ Scope scope_of(const LevelDev<R> &L) { Scope s; s.grid = L.n > FS_MG_SMALL; return s; }

__device__ __forceinline__ void scope_sync(Sync &S, const Scope &sc) {
  if (sc.grid) S.all(); else __syncthreads();
}

// sum over a level: grid-wide or CTA 0
__device__ double scope_sum(Sync &S, const Scope &sc, double v) {
  if (sc.grid) { double o, d; S.sum2(v, 0., o, d); return o; }
  return bsum(v);
}

// one symmetric multicolour Gauss-Seidel sweep (SORMultiGrid.for:20-66)
template <class R>
// `last`: colour of the previous pass over x; a pass repeating it (the
// backward pass's first colour, the next sweep's first) would rewrite the same
// values -- rows of one colour read only other colours -- and is skipped
__device__ void gs_sweep(Sync &S, const Scope &sc, const LevelDev<R> L, const R *b, R *x, int &last) {
  const int n = L.n;
  for (int pass = 0; pass < 2; pass++)
    for (int cc = 0; cc < L.ncolors; cc++) {
      int c = pass == 0 ? cc : L.ncolors - 1 - cc;
      if (c == last) continue;
      last = c;
      int r0 = L.color_ptr[c], r1 = L.color_ptr[c + 1];
      for (long q = r0 + sc.tid0(); q < r1; q += sc.nth()) {
        int i = L.color_rows[q];
        R l = ell_acc<8, true>(b[i], n, L.w, L.nbr, L.anb, i, [&](int k) { return x[k]; });
        x[i] = l / L.ac[i];
      }
      scope_sync(S, sc);
    }
}

// r = b - A x on a level; returns sum |r| (CalculateResidualsMG + CheckConvergenceMG)
template <class R>
__device__ double residual(Sync &S, const Scope &sc, const LevelDev<R> L, const R *b, const R *x, R *r) {
  const int n = L.n;
  double s = 0.;
  for (long i = sc.tid0(); i < n; i += sc.nth()) {
    R t = ell_acc<8, true>(b[i] - L.ac[i] * x[i], n, L.w, L.nbr, L.anb, i, [&](int k) { return x[k]; });
    r[i] = t;
    s += fabs((double)t);
  }
  return scope_sum(S, sc, s);
}

// SolveEquationMG: sweeps until sum|r| <= rrF*IRes or itmax (checked=true), or
// exactly itmax sweeps (checked=false)
template <class R>
__device__ void smooth(Sync &S, const Scope &sc, const LevelDev<R> &L, const R *b, R *x, R *r,
                       double rrf, double ires, int itmax, bool checked) {
  double fres = ires;
  int iter = 0, last = -1;
  while ((!checked || fres > rrf * ires) && iter < itmax) {
    gs_sweep(S, sc, L, b, x, last);
    if (checked) fres = residual(S, sc, L, b, x, r);
    iter++;
  }
}

// b_{l+1}[P] = sum of r_l over P's fine rows in ascending order (AssembleAgglomeratedRHS)
template <class R>
__device__ void restrict_rhs(const Scope &sc, const LevelDev<R> &Lc, const R *r_f) {
  for (long P = sc.tid0(); P < Lc.n; P += sc.nth()) {
    R s = 0.;
    for (int q = Lc.rptr[P]; q < Lc.rptr[P + 1]; q++) s = s + r_f[Lc.rlist[q]];
    Lc.b[P] = s;
  }
}

// x_l[i] += x_{l+1}[parent[i]] (CorrectFinerLevelSolution)
template <class R>
__device__ void prolong(const Scope &sc, const LevelDev<R> &Lf, R *x_f, const R *x_c) {
  for (long i = sc.tid0(); i < Lf.n; i += sc.nth()) x_f[i] = x_f[i] + x_c[Lf.parent[i]];
}

// a V/F/W cycle; level 0 uses (b0, x0, r0), coarser levels their own arrays.
// Every CTA walks the same sequence of operations; an operation on a small
// level is done by CTA 0 while the others skip to the next grid barrier.
template <class R>
struct Cycle {
  Sync &S;
  const LevelDev<R> *lev;
  int nlev;
  const R *b0; R *x0; R *r0;
  double rrf, ires;
  int pre, post;
  bool checked;
  bool last_grid;   // scope of the previous operation
  __device__ const R *B(int l) const { return l == 0 ? b0 : lev[l].b; }
  __device__ R *X(int l) const { return l == 0 ? x0 : lev[l].x; }
  __device__ R *Rr(int l) const { return l == 0 ? r0 : lev[l].r; }
  __device__ void enter(const Scope &sc) {
    // a grid barrier whenever the whole grid is involved on either side,
    // else a block barrier (CTA 0 works alone on small levels)
    if (sc.grid || last_grid) S.all(); else __syncthreads();
    last_grid = sc.grid;
  }
  __device__ void op_smooth(int l, int itmax) {
    Scope sc = scope_of(lev[l]);
    enter(sc);
    if (sc.active()) smooth(S, sc, lev[l], B(l), X(l), Rr(l), rrf, ires, itmax, checked);
  }
  __device__ void op_residual(int l) {
    Scope sc = scope_of(lev[l]);
    enter(sc);
    if (sc.active()) residual(S, sc, lev[l], B(l), X(l), Rr(l));
  }
  __device__ void op_restrict(int l) {   // Restrict(l): smooth, residual, coarse rhs
    op_smooth(l, pre);
    op_residual(l);
    Scope sc = scope_of(lev[l + 1]);
    Scope sf = scope_of(lev[l]);
    Scope su; su.grid = sc.grid || sf.grid;
    enter(su);
    if (su.active()) restrict_rhs(su, lev[l + 1], Rr(l));
  }
  __device__ void op_prolong(int lc) {   // Prolongate(lc): correct level lc-1, smooth it
    int l = lc - 1;
    Scope sf = scope_of(lev[l]);
    enter(sf);
    if (sf.active()) prolong(sf, lev[l], X(l), X(lc));
    op_smooth(l, post);
  }
  __device__ void run(int type) {
    int L = nlev - 1;
    for (int l = 0; l < L; l++) op_restrict(l);
    op_smooth(L, post);
    op_residual(L);
    if (type != 0) {
      for (int l1 = L - 1; l1 >= 1; l1--) {
        for (int l = L; l >= l1 + 1; l--) op_prolong(l);
        for (int l = l1; l < L; l++) op_restrict(l);
        op_smooth(L, post);
        op_residual(L);
      }
      if (type == 2)
        for (int l1 = 2; l1 <= L - 1; l1++) {
          for (int l = L; l >= l1 + 1; l--) op_prolong(l);
          for (int l = l1; l < L; l++) op_restrict(l);
          op_smooth(L, post);
          op_residual(L);
        }
    }
    for (int l = L; l >= 1; l--) op_prolong(l);
    Scope g; g.grid = true;
    enter(g);     // final barrier: level-0 x complete
  }
};

struct MgSolveArgs {
  const LevelDev<double> *lev;
  int nlev, type, pre, post, maxcycles;
  const double *b0; double *x0; double *r0;
  double rrf; const double *ires;
  double *part;
  int32_t *iters;
};

// AlgebraicMultigrid cycle loop (AlgebraicMultiGridMainRoutine.for:330-345)
__global__ void __launch_bounds__(FS_COOP_BLOCK) k_mg_solve(MgSolveArgs a) {
  Sync S(a.part);
  // dphiMG = 0 on every level
  for (int l = 0; l < a.nlev; l++) {
    Scope sc; sc.grid = true;
    double *x = l == 0 ? a.x0 : a.lev[l].x;
    for (long i = sc.tid0(); i < a.lev[l].n; i += sc.nth()) x[i] = 0.;
  }
  S.all();
  double ires = *a.ires, fres = ires;
  Cycle<double> C{S, a.lev, a.nlev, a.b0, a.x0, a.r0, a.rrf, ires, a.pre, a.post, true, true};
  int ncycle = 1;
  while (ncycle <= a.maxcycles && fres > a.rrf * ires) {
    C.last_grid = true;
    C.run(a.type);
    Scope g; g.grid = true;
    fres = residual(S, g, a.lev[0], a.b0, a.x0, a.r0);
    ncycle++;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *a.iters = ncycle - 1;
}

// the initial guess of k_amg_bicgstab on the whole cooperative grid
// (guess_fit_body in fs_amg_core.cuh)
template <class R, int NX>
__global__ void __launch_bounds__(FS_COOP_BLOCK, 1) k_guess_fit(AmgKArgs<R> a) {
  g1::guess_fit_body<R, NX>(a);
}

// right-preconditioned BiCGSTAB with the V-cycle on the whole cooperative grid
// (amg_bicgstab_body in fs_amg_core.cuh)
template <class R, int MODE>
__global__ void __launch_bounds__(FS_COOP_BLOCK, FS_AMG_MINB) k_amg_bicgstab(AmgKArgs<R> a) {
  g1::amg_bicgstab_body<R, MODE>(a);
}

// the same solve for n systems at once (the p' solves of an ensemble, one
// cooperative launch): CTAs [start[q], start[q+1]) solve system q with their
// own bounded barriers (gbar[2q..2q+1], zero at launch), so systems of uneven
// size share the GPU instead of each holding all of it in turn
template <class R, int MODE>
__global__ void __launch_bounds__(FS_COOP_BLOCK, FS_AMG_MINB)
    k_amg_bicgstab_batch(const AmgKArgs<R> *__restrict__ as, const int32_t *__restrict__ start, int n,
                         unsigned *gbar) {
  gb::GroupState &G = gb::gstate();
  if (threadIdx.x == 0) {
    int q = 0;
    while (q + 1 < n && (int)blockIdx.x >= start[q + 1]) q++;
    G.q = q;
    G.cta = (int)blockIdx.x - start[q];
    G.ncta = start[q + 1] - start[q];
    G.gen = 0;
    G.bar = gbar + 2 * q;
    G.status = as[q].status;
  }
  __syncthreads();
  const AmgKArgs<R> a = as[G.q];
  gb::amg_bicgstab_body<R, MODE>(a);
}

// the initial guesses of the batched solves, in the same CTA groups (a group
// whose system has no basis vectors does nothing)
template <class R, int NX>
__global__ void __launch_bounds__(FS_COOP_BLOCK, 1)
    k_guess_fit_batch(const AmgKArgs<R> *__restrict__ as, const int32_t *__restrict__ start, int n, unsigned *gbar) {
  gb::GroupState &G = gb::gstate();
  if (threadIdx.x == 0) {
    int q = 0;
    while (q + 1 < n && (int)blockIdx.x >= start[q + 1]) q++;
    G.q = q;
    G.cta = (int)blockIdx.x - start[q];
    G.ncta = start[q + 1] - start[q];
    G.gen = 0;
    G.bar = gbar + 2 * q;
    G.status = as[q].status;
  }
  __syncthreads();
  const AmgKArgs<R> a = as[G.q];
  if (a.nx == NX) gb::guess_fit_body<R, NX>(a);   // groups of other basis sizes take another launch
}

// the fit kernels by basis size (1 .. FS_GUESS_MAX): each instance keeps its
// sums in registers
template <class R>
static const void *guess_fit_kernel(int nx) {
  switch (nx) {
    case 1: return (const void *)k_guess_fit<R, 1>;
    case 2: return (const void *)k_guess_fit<R, 2>;
    case 3: return (const void *)k_guess_fit<R, 3>;
    case 4: return (const void *)k_guess_fit<R, 4>;
    case 5: return (const void *)k_guess_fit<R, 5>;
    case 6: return (const void *)k_guess_fit<R, 6>;
    case 7: return (const void *)k_guess_fit<R, 7>;
    case 8: return (const void *)k_guess_fit<R, 8>;
  }
  return nullptr;
}
template <class R>
static const void *guess_fit_batch_kernel(int nx) {
  switch (nx) {
    case 1: return (const void *)k_guess_fit_batch<R, 1>;
    case 2: return (const void *)k_guess_fit_batch<R, 2>;
    case 3: return (const void *)k_guess_fit_batch<R, 3>;
    case 4: return (const void *)k_guess_fit_batch<R, 4>;
    case 5: return (const void *)k_guess_fit_batch<R, 5>;
    case 6: return (const void *)k_guess_fit_batch<R, 6>;
    case 7: return (const void *)k_guess_fit_batch<R, 7>;
    case 8: return (const void *)k_guess_fit_batch<R, 8>;
  }
  return nullptr;
}

// coarse matrix of level lc from level lc-1 (AssembleElementBasedAgglomoratedLHS.for:45-150)
// one thread per coarse row (AssembleElementBasedAgglomoratedLHS.for:45-150):
// the children in list order, each child's diagonal then its neighbour slots in
// slot order, so every coarse entry is summed in the reference's order.  The
// coarse row's off-diagonal sums live in shared memory (wc doubles per thread,
// column-major across the block).  WF > 0 bounds the fine width: a child's
// slots are then loaded all at once (independent loads in flight) before the
// additions, instead of one dependent load chain per slot.
template <int WF>
__global__ void k_mg_lhs(int nf, const int32_t *__restrict__ ncf_f, const double *__restrict__ ac_f,
                         const double *__restrict__ anb_f, int nc, int wc, const int32_t *__restrict__ cptr,
                         const int32_t *__restrict__ clist, const int32_t *__restrict__ cmap,
                         double *__restrict__ ac_c, double *__restrict__ anb_c,
                         float *__restrict__ acf_c, float *__restrict__ anbf_c) {
  extern __shared__ double sacc[];
  int P = blockIdx.x * blockDim.x + threadIdx.x;
  const int T = blockDim.x;
  double *acc_nb = sacc + threadIdx.x;
  for (int k = 0; k < wc; k++) acc_nb[(long)k * T] = 0.;
  if (P >= nc) return;
  double acc = 0.;
  const int q0 = cptr[P], q1 = cptr[P + 1];
  for (int q = q0; q < q1; q++) {
    const int c = clist[q];
    const double a0 = ac_f[c];
    const int nn = ncf_f[c];
    if (WF > 0) {
      int t[WF > 0 ? WF : 1];
      double a[WF > 0 ? WF : 1];
#pragma unroll
      for (int j = 0; j < WF; j++) {
        t[j] = -1; a[j] = 0.;
        if (j < nn) { t[j] = cmap[(long)j * nf + c]; a[j] = anb_f[(long)j * nf + c]; }
      }
      acc = acc + a0;
#pragma unroll
      for (int j = 0; j < WF; j++) {
        if (t[j] == -2) acc = acc + a[j];
        else if (t[j] >= 0) acc_nb[(long)t[j] * T] = acc_nb[(long)t[j] * T] + a[j];
      }
    } else {
      acc = acc + a0;
      for (int j = 0; j < nn; j++) {
        const int tj = cmap[(long)j * nf + c];
        const double aj = anb_f[(long)j * nf + c];
        if (tj == -2) acc = acc + aj;
        else if (tj >= 0) acc_nb[(long)tj * T] = acc_nb[(long)tj * T] + aj;
      }
    }
  }
  ac_c[P] = acc;
  for (int k = 0; k < wc; k++) anb_c[(long)k * nc + P] = acc_nb[(long)k * T];
  if (acf_c) {   // the FP32 copy of the coarse level, when the preconditioner is FP32
    acf_c[P] = (float)acc;
    for (int k = 0; k < wc; k++) anbf_c[(long)k * nc + P] = (float)acc_nb[(long)k * T];
  }
}

__global__ void k_to_f32(long n, const double *a, float *b) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

// Dense inverse of the coarsest level (one CTA, matrix in shared memory):
// in-place Gauss-Jordan without pivoting, two block barriers per pivot.  The
// agglomerated matrices are diagonally dominant.  A pure-Neumann level (every
// row sum ~0: the pressure correction with walls only) is singular with the
// constant null space; its last equation is replaced by x_{n-1} = 0 and the last
// column of the inverse is zeroed, so sinv*b solves the remaining equations --
// the consistent systems the V-cycle restricts.  A zero pivot drops its unknown.
__global__ void __launch_bounds__(1024) k_mg_dense_inverse(int n, const int32_t *ncf, const int32_t *nbr,
                                                           const double *ac, const double *anb, double *sinv) {
  extern __shared__ double sm[];
  double *A = sm, *col = sm + (long)n * n;
  __shared__ int singular;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int q = tid; q < n * n; q += nt) A[q] = 0.;
  if (tid == 0) singular = 1;
  __syncthreads();
  for (int i = tid; i < n; i += nt) {
    double d = ac[i], rs = d;
    A[(long)i * n + i] = d;
    for (int j = 0; j < ncf[i]; j++) {
      int k = nbr[(long)j * n + i];
      if (k >= 0) { double a = anb[(long)j * n + i]; A[(long)i * n + k] += a; rs += a; }
    }
    if (fabs(rs) > 1e-9 * fabs(d)) singular = 0;
  }
  __syncthreads();
  const bool sing = singular != 0;
  if (sing)
    for (int j = tid; j < n; j += nt) A[(long)(n - 1) * n + j] = j == n - 1 ? 1. : 0.;
  __syncthreads();
  // warps take rows, lanes take columns.  The pivot row and column of step k
  // are read from buffers (prow/pcol, double-buffered by the parity of k) that
  // the update of step k-1 filled, so one block barrier per pivot suffices;
  // every entry goes through the same operations as an in-place elimination.
  const int lane = tid & 31, wid = tid >> 5, nwarp = nt >> 5;
  double *prow = col + n, *pcol = prow + 2 * n;   // [2][n] each
  for (int j = tid; j < n; j += nt) { prow[j] = A[j]; pcol[j] = A[(long)j * n]; }
  __syncthreads();
  for (int k = 0; k < n; k++) {
    const int b = k & 1;
    const double *pr = prow + b * n, *pc = pcol + b * n;
    double *nr = prow + (b ^ 1) * n, *nc = pcol + (b ^ 1) * n;
    const double d = pr[k];
    const double p = d != 0. ? 1. / d : 0.;
    for (int i = wid; i < n; i += nwarp) {
      double *ri = A + (long)i * n;
      const double ci = pc[i];
      for (int j = lane; j < n; j += 32) {
        const double rkj = j == k ? p : pr[j] * p;
        double v;
        if (i == k) v = rkj;
        else v = j == k ? -ci * p : ri[j] - ci * rkj;
        ri[j] = v;
        if (i == k + 1) nr[j] = v;
        if (j == k + 1) nc[i] = v;
      }
    }
    __syncthreads();
  }
  if (sing)
    for (int i = tid; i < n; i += nt) A[(long)i * n + n - 1] = 0.;
  __syncthreads();
  for (int q = tid; q < n * n; q += nt) sinv[q] = A[q];
}

}  // namespace

// ================================================================ host: hierarchy
struct HostLevel {
  int n = 0, w = 0;
  std::vector<int32_t> nnb, nbr;   // nbr[j*n+i]
};

// AgglomorateLevelGeometricallyElement restated (see file header); fills the
// coarse level and the parent map / child lists of the fine one.
static void agglomerate(const HostLevel &f, int lc, HostLevel &c, std::vector<int32_t> &parent,
                        std::vector<int32_t> &cptr, std::vector<int32_t> &clist) {
  const int n = f.n;
  const int maxc = lc == 1 ? 8 : lc == 2 ? 4 : lc == 3 ? 3 : 2;
  parent.assign(n, -1);
  std::vector<int32_t> seed;
  std::vector<std::vector<int32_t>> ch;
  for (int s = 0; s < n; s++) {
    if (parent[s] != -1) continue;
    int ip = (int)seed.size();
    parent[s] = ip;
    std::vector<int32_t> list;
    int cnt = 0;
    for (int j = 0; j < f.nnb[s]; j++) {
      int q = f.nbr[(size_t)j * n + s];
      if (q >= 0 && parent[q] == -1) {
        if (cnt >= maxc) break;
        parent[q] = ip; list.push_back(q); cnt++;
      }
    }
    int cnt2 = cnt;
    if (cnt < maxc)
      for (int k = 0; k < cnt2; k++) {
        if (cnt >= maxc) break;
        int cc = list[k];
        for (int j = 0; j < f.nnb[cc]; j++) {
          if (cnt >= maxc) break;
          int q = f.nbr[(size_t)j * n + cc];
          if (q >= 0 && parent[q] == -1) { parent[q] = ip; list.push_back(q); cnt++; }
        }
      }
    if (cnt == 0) parent[s] = -1;
    else { seed.push_back(s); ch.push_back(list); }
  }
  for (int pass = 0; pass < 2; pass++)
    for (int o = 0; o < n; o++) {
      if (parent[o] == -1) {
        bool found = false;
        for (int j = 0; j < f.nnb[o]; j++) {
          int q = f.nbr[(size_t)j * n + o];
          if (q >= 0 && parent[q] != -1 && !found) {
            found = true;
            int P = parent[q];
            if (pass == 0 && (int)ch[P].size() >= maxc) continue;
            parent[o] = P; ch[P].push_back(o);
          }
        }
      }
      if (pass == 1 && parent[o] == -1) {
        parent[o] = (int)seed.size(); seed.push_back(o); ch.emplace_back();
      }
    }
  const int nc = (int)seed.size();
  std::vector<std::vector<int32_t>> cn(nc);
  for (int e = 0; e < n; e++)
    for (int j = 0; j < f.nnb[e]; j++) {
      int q = f.nbr[(size_t)j * n + e];
      if (q < 0 || parent[e] == parent[q]) continue;
      auto &v = cn[parent[e]];
      if (std::find(v.begin(), v.end(), parent[q]) == v.end()) v.push_back(parent[q]);
    }
  int wc = 1;
  for (auto &v : cn) wc = std::max(wc, (int)v.size());
  c.n = nc; c.w = wc;
  c.nnb.assign(nc, 0);
  c.nbr.assign((size_t)wc * nc, -1);
  for (int P = 0; P < nc; P++) {
    c.nnb[P] = (int)cn[P].size();
    for (int k = 0; k < c.nnb[P]; k++) c.nbr[(size_t)k * nc + P] = cn[P][k];
  }
  cptr.assign(nc + 1, 0);
  clist.clear();
  for (int P = 0; P < nc; P++) {
    cptr[P] = (int)clist.size();
    clist.push_back(seed[P]);
    clist.insert(clist.end(), ch[P].begin(), ch[P].end());
  }
  cptr[nc] = (int)clist.size();
}

static std::vector<int32_t> color_level(const HostLevel &L, int &ncol) {
  std::vector<int> col(L.n, -1);
  ncol = 0;
  for (int i = 0; i < L.n; i++) {
    uint64_t used = 0;
    for (int j = 0; j < L.nnb[i]; j++) {
      int k = L.nbr[(size_t)j * L.n + i];
      if (k >= 0 && col[k] >= 0 && col[k] < 64) used |= 1ull << col[k];
    }
    int c = 0;
    while (c < 63 && (used & (1ull << c))) c++;
    col[i] = c;
    ncol = std::max(ncol, c + 1);
  }
  std::vector<int32_t> ptr(ncol + 1, 0), rows(L.n);
  for (int i = 0; i < L.n; i++) ptr[col[i] + 1]++;
  for (int c = 0; c < ncol; c++) ptr[c + 1] += ptr[c];
  std::vector<int32_t> pos(ptr.begin(), ptr.end() - 1);
  for (int i = 0; i < L.n; i++) rows[pos[col[i]]++] = i;
  rows.insert(rows.end(), ptr.begin(), ptr.end());
  return rows;
}

template <class T>
static int upv(fs_ctx *ctx, T **d, const std::vector<T> &h) {
  FS_CK(cudaMalloc((void **)d, std::max<size_t>(h.size(), 1) * sizeof(T)));
  if (!h.empty()) FS_CK(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return FS_OK;
}

int fs_mg_build(fs_ctx *ctx) {
  if (ctx->mg) return FS_OK;
  fs_mg_dev *M = new fs_mg_dev();
  ctx->mg = M;
  std::vector<HostLevel> H(1);
  H[0].n = ctx->N; H[0].w = ctx->W; H[0].nnb = ctx->h_ncf; H[0].nbr = ctx->h_cn;
  std::vector<std::vector<int32_t>> cptr(FS_MG_MAXLEV), clist(FS_MG_MAXLEV);
  int l = 0;
  const int maxlev = std::min(ctx->cfg.mg_max_levels, FS_MG_MAXLEV);
  while (l + 1 < maxlev && H[l].n > 2 * ctx->cfg.mg_min_parents) {
    H.emplace_back();
    agglomerate(H[l], l + 1, H[l + 1], M->h_parent[l], cptr[l], clist[l]);
    l++;
  }
  M->nlev = l + 1;
  int rc;
  std::vector<LevelDev<double>> L64(M->nlev);
  std::vector<LevelDev<float>> L32(M->nlev);
  for (int q = 0; q < M->nlev; q++) {
    const HostLevel &h = H[q];
    M->n[q] = h.n; M->w[q] = h.w;
    std::vector<int32_t> colors = color_level(h, M->ncol[q]);
    if ((rc = upv(ctx, &M->colors[q], colors))) return rc;
    if (q == 0) { M->nnb[0] = ctx->ncf; M->nbr[0] = ctx->cn; }
    else {
      if ((rc = upv(ctx, &M->nnb[q], h.nnb))) return rc;
      if ((rc = upv(ctx, &M->nbr[q], h.nbr))) return rc;
    }
    if (q + 1 < M->nlev) {
      if ((rc = upv(ctx, &M->parent[q], M->h_parent[q]))) return rc;
      // LHS lists and slot map (fine slot -> coarse slot / internal / none)
      if ((rc = upv(ctx, &M->cptr[q + 1], cptr[q]))) return rc;
      if ((rc = upv(ctx, &M->clist[q + 1], clist[q]))) return rc;
      const HostLevel &c = H[q + 1];
      std::vector<int32_t> cmap((size_t)h.w * h.n, -1);
      for (int i = 0; i < h.n; i++) {
        int P = M->h_parent[q][i];
        for (int j = 0; j < h.nnb[i]; j++) {
          int nb = h.nbr[(size_t)j * h.n + i];
          if (nb < 0) continue;
          int Q = M->h_parent[q][nb];
          if (Q == P) { cmap[(size_t)j * h.n + i] = -2; continue; }
          for (int k = 0; k < c.nnb[P]; k++)
            if (c.nbr[(size_t)k * c.n + P] == Q) { cmap[(size_t)j * h.n + i] = k; break; }
        }
      }
      if ((rc = upv(ctx, &M->cmap[q + 1], cmap))) return rc;
      // restriction lists: fine rows of each coarse row in ascending order
      std::vector<int32_t> rptr(c.n + 1, 0), rlist(h.n);
      for (int i = 0; i < h.n; i++) rptr[M->h_parent[q][i] + 1]++;
      for (int P = 0; P < c.n; P++) rptr[P + 1] += rptr[P];
      std::vector<int32_t> pos(rptr.begin(), rptr.end() - 1);
      for (int i = 0; i < h.n; i++) rlist[pos[M->h_parent[q][i]]++] = i;
      if ((rc = upv(ctx, &M->rptr[q + 1], rptr))) return rc;
      if ((rc = upv(ctx, &M->rlist[q + 1], rlist))) return rc;
      // warp chunks of the coarse rows: consecutive rows, <= 32 of them and
      // <= 64 children in all (a row with more children is a chunk alone)
      std::vector<int32_t> ck(1, 0);
      for (int P = 0, rows = 0, kids = 0; P < c.n; P++) {
        const int k = rptr[P + 1] - rptr[P];
        if (rows > 0 && (rows == 32 || kids + k > 64)) { ck.push_back(P); rows = 0; kids = 0; }
        rows++; kids += k;
      }
      ck.push_back(c.n);
      M->nchunk[q + 1] = (int)ck.size() - 1;
      if ((rc = upv(ctx, &M->chunk[q + 1], ck))) return rc;
    }
    size_t n = h.n, nw = (size_t)h.w * h.n;
    if (q == 0) { M->ac[0] = ctx->ac; M->anb[0] = ctx->anb; }
    else {
      FS_CK(cudaMalloc(&M->ac[q], sizeof(double) * n));
      FS_CK(cudaMalloc(&M->anb[q], sizeof(double) * nw));
      FS_CK(cudaMemset(M->anb[q], 0, sizeof(double) * nw));
    }
    FS_CK(cudaMalloc(&M->b[q], sizeof(double) * n));
    FS_CK(cudaMalloc(&M->x[q], sizeof(double) * n));
    FS_CK(cudaMalloc(&M->r[q], sizeof(double) * n));
    FS_CK(cudaMalloc(&M->t[q], sizeof(double) * n));
    FS_CK(cudaMalloc(&M->tf[q], sizeof(float) * n));
    FS_CK(cudaMalloc(&M->acf[q], sizeof(float) * n));
    FS_CK(cudaMalloc(&M->anbf[q], sizeof(float) * nw));
    FS_CK(cudaMalloc(&M->bf[q], sizeof(float) * n));
    FS_CK(cudaMalloc(&M->xf[q], sizeof(float) * n));
    FS_CK(cudaMalloc(&M->rf[q], sizeof(float) * n));
  }
  for (int q = 0; q < M->nlev; q++) {
    int32_t *cols = M->colors[q];
    LevelDev<double> d{};
    d.n = M->n[q]; d.w = M->w[q]; d.ncolors = M->ncol[q];
    d.ncf = M->nnb[q]; d.nbr = M->nbr[q]; d.color_rows = cols; d.color_ptr = cols + M->n[q];
    d.ac = M->ac[q]; d.anb = M->anb[q]; d.b = M->b[q]; d.x = M->x[q]; d.r = M->r[q]; d.t = M->t[q];
    d.parent = (q + 1 < M->nlev) ? M->parent[q] : nullptr;
    d.rptr = M->rptr[q]; d.rlist = M->rlist[q];
    d.chunk = M->chunk[q]; d.nchunk = M->nchunk[q];
    L64[q] = d;
    LevelDev<float> e{};
    e.n = d.n; e.w = d.w; e.ncolors = d.ncolors; e.ncf = d.ncf; e.nbr = d.nbr; e.color_rows = d.color_rows;
    e.color_ptr = d.color_ptr; e.ac = M->acf[q]; e.anb = M->anbf[q]; e.b = M->bf[q]; e.x = M->xf[q]; e.r = M->rf[q];
    e.t = M->tf[q];
    e.parent = d.parent; e.rptr = d.rptr; e.rlist = d.rlist;
    e.chunk = d.chunk; e.nchunk = d.nchunk;
    L32[q] = e;
  }
  FS_CK(cudaMalloc(&M->lev64, sizeof(LevelDev<double>) * M->nlev));
  FS_CK(cudaMemcpy(M->lev64, L64.data(), sizeof(LevelDev<double>) * M->nlev, cudaMemcpyHostToDevice));
  FS_CK(cudaMalloc(&M->lev32, sizeof(LevelDev<float>) * M->nlev));
  FS_CK(cudaMemcpy(M->lev32, L32.data(), sizeof(LevelDev<float>) * M->nlev, cudaMemcpyHostToDevice));
  FS_CK(cudaMalloc(&M->red, sizeof(double) * (6 + FS_SUMK + 9) * FS_RED_BLOCKS));
  // preconditioner: stop at the first level small enough for the dense inverse
  M->lc = M->nlev - 1;
  for (int q = 0; q < M->nlev; q++)
    if (q > 0 && M->n[q] <= FS_MG_DIRECT) { M->lc = q; break; }
  M->direct = M->lc > 0 && M->n[M->lc] <= FS_MG_DIRECT;
  if (M->direct) {
    size_t nn = (size_t)M->n[M->lc] * M->n[M->lc];
    FS_CK(cudaMalloc(&M->sinv, sizeof(double) * nn));
    // the attribute belongs to the function, shared by every context of the
    // process: set it for the largest coarsest level any context may have
    FS_CK(cudaFuncSetAttribute((const void *)k_mg_dense_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(sizeof(double) * ((size_t)FS_MG_DIRECT * FS_MG_DIRECT + 5 * FS_MG_DIRECT))));
  }
  // cooperative grid: smallest co-resident count of the three kernels, <= 4 CTAs/SM
  int a = 0, b = 0, c = 0;
  FS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, (void *)k_mg_solve, FS_COOP_BLOCK, 0));
  int b2 = 0, c2 = 0, c3 = 0;
  FS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (void *)k_amg_bicgstab<double, 0>, FS_COOP_BLOCK, 0));
  FS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, (void *)k_amg_bicgstab<float, 0>, FS_COOP_BLOCK, 0));
  FS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, (void *)k_amg_bicgstab<double, 1>, FS_COOP_BLOCK, 0));
  FS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c2, (void *)k_amg_bicgstab<float, 1>, FS_COOP_BLOCK, 0));
  FS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c3, (void *)k_amg_bicgstab<float, 2>, FS_COOP_BLOCK, 0));
  int per = std::min(std::min(a, std::min(b, c)), std::min(std::min(b2, c2), c3));
  if (per < 1) { ctx->err = "multigrid kernels do not fit on an SM"; return FS_E_CUDA; }
  M->per_sm = per;   // occupancy limit; the grid follows the launch shape at each solve
  return FS_OK;
}

int fs_mg_free(fs_ctx *ctx) {
  fs_mg_dev *M = ctx->mg;
  if (!M) return FS_OK;
  for (int q = 0; q < M->nlev; q++) {
    void *p[] = {M->colors[q], M->chunk[q], q ? M->nnb[q] : nullptr, q ? M->nbr[q] : nullptr, M->parent[q], M->cptr[q], M->clist[q],
                 M->cmap[q], M->rptr[q], M->rlist[q], q ? M->ac[q] : nullptr, q ? M->anb[q] : nullptr, M->b[q], M->x[q],
                 M->r[q], M->acf[q], M->anbf[q], M->bf[q], M->xf[q], M->rf[q], M->t[q], M->tf[q]};
    for (void *x : p) if (x) cudaFree(x);
  }
  cudaFree(M->lev64); cudaFree(M->lev32); cudaFree(M->red); cudaFree(M->sinv);
  delete M;
  ctx->mg = nullptr;
  return FS_OK;
}

// coarse matrices of levels 1..last for the current fine system (every call:
// the fine matrix changes), FP32 copies of levels 0..last when asked
static int mg_coarse_matrices(fs_ctx *ctx, int last, bool f32) {
  fs_mg_dev *M = ctx->mg;
  for (int q = 1; q <= last; q++) {
    // block of T threads with T * w doubles of shared accumulators (<= 48 KB)
    int T = 128;
    while (T > 32 && (size_t)T * M->w[q] * sizeof(double) > 48 * 1024) T /= 2;
    const size_t sm = (size_t)T * M->w[q] * sizeof(double);
    if (sm > 48 * 1024) { ctx->err = "coarse level too wide for the coarse-matrix kernel"; return FS_E_UNSUPPORTED; }
    const int wf = M->w[q - 1];
#define FS_LHS_ARGS M->n[q - 1], M->nnb[q - 1], M->ac[q - 1], M->anb[q - 1], M->n[q], M->w[q], M->cptr[q], \
                    M->clist[q], M->cmap[q], M->ac[q], M->anb[q], f32 ? M->acf[q] : nullptr, f32 ? M->anbf[q] : nullptr
    if (wf <= 8) k_mg_lhs<8><<<fs_grid(M->n[q], T), T, sm, ctx->st>>>(FS_LHS_ARGS);
    else if (wf <= 32) k_mg_lhs<32><<<fs_grid(M->n[q], T), T, sm, ctx->st>>>(FS_LHS_ARGS);
    else k_mg_lhs<0><<<fs_grid(M->n[q], T), T, sm, ctx->st>>>(FS_LHS_ARGS);
#undef FS_LHS_ARGS
    FS_LAUNCH_CHECK();
  }
  if (f32)
    for (int q = 0; q <= 0; q++) {   // coarse levels got their FP32 copy from k_mg_lhs
      long n = M->n[q], nw = (long)M->w[q] * M->n[q];
      k_to_f32<<<fs_grid(n), FS_BLOCK, 0, ctx->st>>>(n, M->ac[q], M->acf[q]);
      FS_LAUNCH_CHECK();
      k_to_f32<<<fs_grid(nw), FS_BLOCK, 0, ctx->st>>>(nw, M->anb[q], M->anbf[q]);
      FS_LAUNCH_CHECK();
    }
  return FS_OK;
}

int fs_mg_solve(fs_ctx *ctx, int nf, double rrf, int solver) {
  int rc = fs_mg_build(ctx);
  if (rc) return rc;
  fs_mg_dev *M = ctx->mg;
  const bool gs = solver == FS_SOLVER_AMG32GS_BICGS;
  const bool f32 = solver == FS_SOLVER_AMG32_BICGS || gs;
  if (gs && !(M->direct && M->lc > 0)) {
    ctx->err = "the Gauss-Seidel V-cycle needs a coarsest level small enough for the dense inverse";
    return FS_E_UNSUPPORTED;
  }
  const int G = std::min(ctx->num_sms * fs_coop_per_sm(ctx, M->per_sm), FS_RED_BLOCKS);
  if (solver == FS_SOLVER_AMG) {
    if ((rc = mg_coarse_matrices(ctx, M->nlev - 1, false))) return rc;
    M->built_nf = 0;
    MgSolveArgs a{};
    a.lev = M->lev64; a.nlev = M->nlev; a.type = ctx->cfg.mg_cycle; a.pre = ctx->cfg.mg_pre; a.post = ctx->cfg.mg_post;
    a.maxcycles = ctx->cfg.mg_max_cycles; a.b0 = ctx->bc; a.x0 = ctx->dphi; a.r0 = M->r[0];
    a.rrf = rrf; a.ires = ctx->resblk + RB_ABS + (nf - 1); a.part = M->red; a.iters = ctx->d_iters + (nf - 1);
    void *args[] = {&a};
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][0], ctx->st)));
    FS_CK(fs_coop_launch((const void *)k_mg_solve, G, fs_coop_block(ctx), args, ctx->st));
    FS_LAUNCH_CHECK();
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][1], ctx->st)));
    return FS_OK;
  }
  // coarse levels and the dense coarsest inverse: rebuilt every pc_refresh solves
  // of the same system (1: every solve); in between the V-cycle keeps them and
  // only level 0 (the current system) is new -- a fixed preconditioner within
  // each solve, which still runs to its tolerance
  const int refresh = std::max(1, ctx->cfg.pc_refresh);
  const bool reuse = M->built_nf == nf && M->built_f32 == f32 && M->age + 1 < refresh;
  if (reuse) {
    M->age++;
    if (f32) {   // level 0 in FP32 from the current system
      const long n = M->n[0], nw = (long)M->w[0] * M->n[0];
      k_to_f32<<<fs_grid(n), FS_BLOCK, 0, ctx->st>>>(n, M->ac[0], M->acf[0]);
      FS_LAUNCH_CHECK();
      k_to_f32<<<fs_grid(nw), FS_BLOCK, 0, ctx->st>>>(nw, M->anb[0], M->anbf[0]);
      FS_LAUNCH_CHECK();
    }
  } else {
    if ((rc = mg_coarse_matrices(ctx, M->lc, f32))) return rc;
    M->built_nf = nf; M->built_f32 = f32; M->age = 0;
  }
  // team-barrier counters of the V-cycle start at zero for every launch
  FS_CK(cudaMemsetAsync(ctx->d_status + 4, 0, sizeof(int32_t) * 2, ctx->st));
  if (M->direct && !reuse) {
    const int n = M->n[M->lc];
    k_mg_dense_inverse<<<1, 1024, sizeof(double) * ((size_t)n * n + 5 * (size_t)n), ctx->st>>>(
        n, M->nnb[M->lc], M->nbr[M->lc], M->ac[M->lc], M->anb[M->lc], M->sinv);
    FS_LAUNCH_CHECK();
  }
  auto fill = [&](auto &a) {
    a.N = ctx->N; a.W = ctx->W; a.ncf = ctx->ncf; a.cn = ctx->cn; a.ac = ctx->ac; a.anb = ctx->anb; a.bc = ctx->bc;
    a.x = ctx->kx; a.r = ctx->kr; a.r0 = ctx->kr0; a.p = ctx->kp; a.v = ctx->kv; a.s = ctx->ks; a.t = ctx->kt;
    a.y = ctx->ky; a.z = ctx->kz; a.dphi = ctx->dphi;
    // one V-cycle per application: one pre- and one post-sweep (MultiGridpreSweep)
    a.lc = M->lc; a.direct = M->direct; a.sinv = M->sinv;
    a.pre = std::max(1, ctx->cfg.mg_pre); a.post = std::max(1, ctx->cfg.mg_pre);
    a.maxit = ctx->cfg.krylov_maxit; a.tol = ctx->cfg.krylov_tol; a.part = M->red;
    a.iters = ctx->d_iters + (nf - 1); a.diag = ctx->resblk + RB_DIAG;
    a.nx = 0;
    if (nf == FS_VAR_PC)
      for (int j = 0; j < ctx->pc_nguess && j < FS_GUESS_MAX; j++) a.xs[a.nx++] = ctx->pc_guess[j];
    a.fit = ctx->d_status + 6;
    a.nncnt = ctx->pc_nn ? fs_nn_counters(ctx) : nullptr;   // the network's guess is in the basis
    a.teambar = (unsigned *)(ctx->d_status + 4);
    a.status = ctx->d_status;
    a.team_extra = ctx->test_wait_extra;
  };
  // the fused V-cycle needs one pre- and one post-sweep and a dense coarsest level
  const bool fused = std::max(1, ctx->cfg.mg_pre) == 1 && M->direct && M->lc > 0;
  if (ctx->pc_defer && nf == FS_VAR_PC) {   // prepared here, launched with other contexts' by fs_pc_batch_launch
    int form = -1;
    if ((rc = fs_pc_batch_form(ctx, &form))) return rc;
    if (form < 0) { ctx->err = "this p' solver cannot join a batched launch"; return FS_E_UNSUPPORTED; }
    M->pend_form = form;   // the initial-guess fit runs in the batched launch too
    if (!f32) {
      M->pend64 = AmgKArgs<double>{};
      fill(M->pend64);
      M->pend64.lev = M->lev64;
    } else {
      M->pend32 = AmgKArgs<float>{};
      fill(M->pend32);
      M->pend32.lev = M->lev32;
    }
    return FS_OK;
  }
  if (!f32) {
    AmgKArgs<double> a{};
    fill(a);
    a.lev = M->lev64;
    void *args[] = {&a};
    if (a.nx > 0) FS_CK(fs_coop_launch(guess_fit_kernel<double>(a.nx), G, fs_coop_block(ctx), args, ctx->st));
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][0], ctx->st)));
    FS_CK(fs_coop_launch(fused ? (const void *)k_amg_bicgstab<double, 1> : (const void *)k_amg_bicgstab<double, 0>,
                         G, fs_coop_block(ctx), args, ctx->st));
  } else {
    AmgKArgs<float> a{};
    fill(a);
    a.lev = M->lev32;
    void *args[] = {&a};
    if (a.nx > 0) FS_CK(fs_coop_launch(guess_fit_kernel<float>(a.nx), G, fs_coop_block(ctx), args, ctx->st));
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][0], ctx->st)));
    const void *k = gs ? (const void *)k_amg_bicgstab<float, 2>
                    : fused ? (const void *)k_amg_bicgstab<float, 1> : (const void *)k_amg_bicgstab<float, 0>;
    FS_CK(fs_coop_launch(k, G, fs_coop_block(ctx), args, ctx->st));
  }
  FS_LAUNCH_CHECK();
  FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][1], ctx->st)));
  (void)rrf;
  return FS_OK;
}

extern "C" int fs_mg_levels(fs_ctx *ctx, int32_t *n_levels, int32_t *level_sizes, int max_levels) {
  if (!ctx) return FS_E_ARG;
  int rc = fs_mg_build(ctx);
  if (rc) return rc;
  if (n_levels) *n_levels = ctx->mg->nlev;
  if (level_sizes)
    for (int q = 0; q < ctx->mg->nlev && q < max_levels; q++) level_sizes[q] = ctx->mg->n[q];
  return FS_OK;
}

extern "C" int fs_mg_parents(fs_ctx *ctx, int level, int32_t *parents, size_t n) {
  if (!ctx || !parents) return FS_E_ARG;
  int rc = fs_mg_build(ctx);
  if (rc) return rc;
  if (level < 0 || level + 1 >= ctx->mg->nlev || n != ctx->mg->h_parent[level].size()) return FS_E_ARG;
  memcpy(parents, ctx->mg->h_parent[level].data(), sizeof(int32_t) * n);
  return FS_OK;
}

extern "C" int fs_mg_info(fs_ctx *ctx, int32_t *widths, int max_levels, int32_t *prec_coarsest, int32_t *direct) {
  if (!ctx) return FS_E_ARG;
  int rc = fs_mg_build(ctx);
  if (rc) return rc;
  if (widths)
    for (int q = 0; q < ctx->mg->nlev && q < max_levels; q++) widths[q] = ctx->mg->w[q];
  if (prec_coarsest) *prec_coarsest = ctx->mg->lc;
  if (direct) *direct = ctx->mg->direct ? 1 : 0;
  return FS_OK;
}

extern "C" int fs_mg_coarse_matrix(fs_ctx *ctx, int level, double *ac, int32_t *n_nbr, int32_t *nbr, double *anb,
                                   size_t n, size_t w) {
  if (!ctx || !ac || !n_nbr || !nbr || !anb) return FS_E_ARG;
  int rc = fs_mg_build(ctx);
  if (rc) return rc;
  fs_mg_dev *M = ctx->mg;
  if (level < 1 || level >= M->nlev || n != (size_t)M->n[level] || w != (size_t)M->w[level]) return FS_E_ARG;
  cudaSetDevice(ctx->dev);
  if ((rc = mg_coarse_matrices(ctx, level, false))) return rc;
  FS_CK(cudaMemcpyAsync(ac, M->ac[level], sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
  FS_CK(cudaMemcpyAsync(anb, M->anb[level], sizeof(double) * n * w, cudaMemcpyDeviceToHost, ctx->st));
  FS_CK(cudaMemcpyAsync(n_nbr, M->nnb[level], sizeof(int32_t) * n, cudaMemcpyDeviceToHost, ctx->st));
  FS_CK(cudaMemcpyAsync(nbr, M->nbr[level], sizeof(int32_t) * n * w, cudaMemcpyDeviceToHost, ctx->st));
  FS_CK(cudaStreamSynchronize(ctx->st));
  return FS_OK;
}

// Test of the bounded device waits (no reference counterpart): with extra > 0
// the multigrid team barriers wait for more CTAs than the team has, so their
// polls run out; the solve then ends and the iteration reports FS_E_TIMEOUT.
extern "C" int fs_test_wait_timeout(fs_ctx *ctx, int extra) {
  if (!ctx || extra < 0 || extra > 64) return FS_E_ARG;
  ctx->test_wait_extra = extra;
  return FS_OK;
}

// ------------------------------------------------------------ batched p' solves
// Several contexts' AMG-BiCGSTAB solves in one cooperative launch of
// k_amg_bicgstab_batch (no reference counterpart; the ensemble form).  Form:
// 0/1 FP64 V-cycle run()/fused, 2/3 FP32 run()/fused, 4 FP32 Gauss-Seidel; -1
// when the context's p' solver is not an AMG-BiCGSTAB one.
int fs_pc_batch_form(fs_ctx *ctx, int *form) {
  if (!ctx || !form) return FS_E_ARG;
  *form = -1;
  const int sv = ctx->cfg.solver_cont;
  if (sv != FS_SOLVER_AMG_BICGS && sv != FS_SOLVER_AMG32_BICGS && sv != FS_SOLVER_AMG32GS_BICGS) return FS_OK;
  int rc = fs_mg_build(ctx);
  if (rc) return rc;
  const fs_mg_dev *M = ctx->mg;
  const bool gs = sv == FS_SOLVER_AMG32GS_BICGS, f32 = sv != FS_SOLVER_AMG_BICGS;
  if (gs && !(M->direct && M->lc > 0)) return FS_OK;
  const bool fused = std::max(1, ctx->cfg.mg_pre) == 1 && M->direct && M->lc > 0;
  *form = !f32 ? (fused ? 1 : 0) : gs ? 4 : fused ? 3 : 2;
  return FS_OK;
}

struct fs_pc_batch {
  int n = 0, form = -1, ncta = 0;
  size_t argsz = 0;
  void *h_args = nullptr;       // pinned: the n argument blocks, copied to d_args by each launch
  void *d_args = nullptr;
  int32_t *d_start = nullptr;   // n + 1 CTA offsets
  unsigned *d_words = nullptr;  // 2n team-barrier words, then 2n group-barrier words (zero at each launch)
  std::vector<int32_t> start;
};

static const void *batch_kernel(int form) {
  switch (form) {
    case 0: return (const void *)k_amg_bicgstab_batch<double, 0>;
    case 1: return (const void *)k_amg_bicgstab_batch<double, 1>;
    case 2: return (const void *)k_amg_bicgstab_batch<float, 0>;
    case 3: return (const void *)k_amg_bicgstab_batch<float, 1>;
    case 4: return (const void *)k_amg_bicgstab_batch<float, 2>;
  }
  return nullptr;
}

void fs_pc_batch_free(fs_pc_batch *B) {
  if (!B) return;
  if (B->h_args) cudaFreeHost(B->h_args);
  if (B->d_args) cudaFree(B->d_args);
  if (B->d_start) cudaFree(B->d_start);
  if (B->d_words) cudaFree(B->d_words);
  delete B;
}

// CTAs of one co-resident launch (1024 threads each, one per SM) split among
// the n contexts in proportion to weight[q] (fs_cta_split)
int fs_pc_batch_create(fs_ctx **cs, int n, const double *weight, fs_pc_batch **out) {
  if (!cs || n < 1 || !weight || !out) return FS_E_ARG;
  *out = nullptr;
  fs_ctx *ctx = cs[0];
  int form = -1;
  for (int q = 0; q < n; q++) {
    int f = -1;
    int rc = fs_pc_batch_form(cs[q], &f);
    if (rc) { if (cs[q] != ctx) ctx->err = cs[q]->err; return rc; }
    if (f < 0 || (q > 0 && f != form)) { ctx->err = "contexts cannot share a batched p' launch"; return FS_E_UNSUPPORTED; }
    form = f;
  }
  int occ = 0;
  FS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel(form), FS_COOP_BLOCK, 0));
  const int cap = std::min(ctx->num_sms * std::max(occ, 0), FS_RED_BLOCKS);
  if (cap < n) { ctx->err = "more contexts than co-resident CTAs for a batched p' launch"; return FS_E_UNSUPPORTED; }
  const std::vector<int32_t> split = fs_cta_split(cap, weight, n);
  fs_pc_batch *B = new fs_pc_batch;
  B->n = n; B->form = form;
  B->argsz = form <= 1 ? sizeof(AmgKArgs<double>) : sizeof(AmgKArgs<float>);
  B->start = split;
  B->ncta = B->start[n];
  cudaError_t e;
  if ((e = cudaHostAlloc(&B->h_args, B->argsz * n, cudaHostAllocDefault)) != cudaSuccess ||
      (e = cudaMalloc(&B->d_args, B->argsz * n)) != cudaSuccess ||
      (e = cudaMalloc(&B->d_start, sizeof(int32_t) * (n + 1))) != cudaSuccess ||
      (e = cudaMalloc(&B->d_words, sizeof(unsigned) * 4 * n)) != cudaSuccess ||
      (e = cudaMemcpy(B->d_start, B->start.data(), sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice)) != cudaSuccess) {
    ctx->err = std::string("batched p' set-up: ") + cudaGetErrorString(e);
    fs_pc_batch_free(B);
    return FS_E_CUDA;
  }
  *out = B;
  return FS_OK;
}

// launch the solves every context prepared with pc_defer (fs_mg_solve), on st;
// each context's status word records a barrier timeout as in its own launches
int fs_pc_batch_launch(fs_pc_batch *B, fs_ctx **cs, int n, cudaStream_t st) {
  if (!B || !cs || n != B->n) return FS_E_ARG;
  fs_ctx *ctx = cs[0];
  unsigned nx_mask = 0;
  for (int q = 0; q < n; q++) {
    fs_mg_dev *M = cs[q]->mg;
    if (!M || M->pend_form != B->form) { ctx->err = "batched p' launch: a context prepared no matching solve"; return FS_E_ARG; }
    char *dst = (char *)B->h_args + B->argsz * q;
    if (B->form <= 1) {
      AmgKArgs<double> a = M->pend64;
      a.teambar = B->d_words + 2 * q;
      if (a.nx > 0 && a.nx <= FS_GUESS_MAX) nx_mask |= 1u << a.nx;
      memcpy(dst, &a, sizeof(a));
    } else {
      AmgKArgs<float> a = M->pend32;
      a.teambar = B->d_words + 2 * q;
      if (a.nx > 0 && a.nx <= FS_GUESS_MAX) nx_mask |= 1u << a.nx;
      memcpy(dst, &a, sizeof(a));
    }
    M->pend_form = -1;
  }
  FS_CK(cudaMemcpyAsync(B->d_args, B->h_args, B->argsz * n, cudaMemcpyHostToDevice, st));
  unsigned *gw = B->d_words + 2 * n;
  void *args[] = {&B->d_args, &B->d_start, &B->n, &gw};
  // the initial guesses, same groups: one launch per basis size present (a
  // group sits out the launches of other sizes); the barrier words start from
  // zero for each launch
  for (int nx = 1; nx <= FS_GUESS_MAX; nx++) {
    if (!(nx_mask & (1u << nx))) continue;
    FS_CK(cudaMemsetAsync(B->d_words, 0, sizeof(unsigned) * 4 * n, st));
    FS_CK(fs_coop_launch(B->form <= 1 ? guess_fit_batch_kernel<double>(nx) : guess_fit_batch_kernel<float>(nx),
                         B->ncta, FS_COOP_BLOCK, args, st));
    FS_LAUNCH_CHECK();
  }
  FS_CK(cudaMemsetAsync(B->d_words, 0, sizeof(unsigned) * 4 * n, st));
  FS_CK(fs_coop_launch(batch_kernel(B->form), B->ncta, FS_COOP_BLOCK, args, st));
  FS_LAUNCH_CHECK();
  return FS_OK;
}
