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

struct Sync {
  cg::grid_group grid;
  double *part;
  int buf, buf3;
  __device__ Sync(double *p) : grid(cg::this_grid()), part(p), buf(0), buf3(0) {}
  __device__ void all() { grid.sync(); }
  // grid-deterministic sum of two values (every CTA gets the same result)
  __device__ void sum2(double a0, double a1, double &o0, double &o1) {
    int G = gridDim.x;
    double b0 = bsum(a0), b1 = bsum(a1);
    if (threadIdx.x == 0) { part[(2 * buf) * G + blockIdx.x] = b0; part[(2 * buf + 1) * G + blockIdx.x] = b1; }
    grid.sync();
    double s0 = 0., s1 = 0.;
    for (int q = threadIdx.x; q < G; q += blockDim.x) { s0 += part[(2 * buf) * G + q]; s1 += part[(2 * buf + 1) * G + q]; }
    o0 = bsum(s0); o1 = bsum(s1);
    buf = (buf + 1) % 3;
  }
  // grid-deterministic sums of K <= FS_SUMK values, in the partial slots after
  // the three buffers of sum2 (every CTA gets the same results)
  __device__ void sumK(const double *in, double *out, int K) {
    const int G = gridDim.x;
    double *pk = part + 6L * G;
    for (int k = 0; k < K; k++) {
      const double b = bsum(in[k]);
      if (threadIdx.x == 0) pk[(long)k * G + blockIdx.x] = b;
    }
    grid.sync();
    for (int k = 0; k < K; k++) {
      double t = 0.;
      for (int q = threadIdx.x; q < G; q += blockDim.x) t += pk[(long)k * G + q];
      out[k] = bsum(t);
    }
  }
  // grid-deterministic sums of three values, in three rotating buffers of
  // their own after the sumK slots
  __device__ void sum3(double a0, double a1, double a2, double &o0, double &o1, double &o2) {
    const int G = gridDim.x;
    double *pb = part + (6L + FS_SUMK + 3L * buf3) * G;
    const double b0 = bsum(a0), b1 = bsum(a1), b2 = bsum(a2);
    if (threadIdx.x == 0) { pb[blockIdx.x] = b0; pb[G + blockIdx.x] = b1; pb[2 * G + blockIdx.x] = b2; }
    grid.sync();
    double s0 = 0., s1 = 0., s2 = 0.;
    for (int q = threadIdx.x; q < G; q += blockDim.x) { s0 += pb[q]; s1 += pb[G + q]; s2 += pb[2 * G + q]; }
    o0 = bsum(s0); o1 = bsum(s1); o2 = bsum(s2);
    buf3 = (buf3 + 1) % 3;
  }
};

// which threads work on a level, and how they synchronise
// the first FS_PC_TEAM CTAs: mid-sized preconditioner levels (PCycle)
#ifndef FS_PC_TEAM
#define FS_PC_TEAM 32
#endif
__device__ __forceinline__ int team_size() { return gridDim.x < FS_PC_TEAM ? (int)gridDim.x : FS_PC_TEAM; }

struct Scope {
  bool grid = false;   // whole grid
  bool team = false;   // else the first team_size() CTAs; else CTA 0 only
  __device__ bool active() const { return grid || (team ? (int)blockIdx.x < team_size() : blockIdx.x == 0); }
  __device__ long tid0() const {
    return (grid || team) ? (long)blockIdx.x * blockDim.x + threadIdx.x : (long)threadIdx.x;
  }
  __device__ long nth() const {
    return grid ? (long)gridDim.x * blockDim.x : team ? (long)team_size() * blockDim.x : (long)blockDim.x;
  }
};

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

// One V-cycle with zero initial guesses as the preconditioner M^-1 of the Krylov
// solver.  Damped Jacobi (omega) on every level, so each sweep is one phase of
// independent rows; the first pre-sweep from zero is fused into the restriction
// that makes the level's rhs, and the coarsest level is solved by a dense FP64
// inverse (k_mg_dense_inverse).  The coarse correction is over-weighted,
// x += alpha*x_c[parent] with alpha > 1, which compensates the energy of
// piecewise-constant prolongation.  On levels with a thread per row the
// prolongation is a phase of its own before the first post-sweep; on levels
// with G lanes per row it is formed on the fly inside the sweep for the row and
// its neighbours.  A cycle over levels 0..lc costs 3*lc+2 barrier phases plus one
// per thread-per-row level.  Level-0 rhs and result are FP64 in either
// precision; up-leg results go to each level's r.
//
// Rows with fewer than two threads each are handled a thread per row, two rows
// per step (ell_acc2).  Coarse rows have 10-30 neighbours and coarse levels
// fewer rows than the grid has threads, so there a row is handled by G
// consecutive lanes (G = 2..8 from the threads per row) that split its
// neighbour loop and combine by shuffles.  Levels up to FS_PC_SMALL rows run on
// CTA 0 alone; levels up to FS_PC_TEAM_MAX rows on a team of the first
// FS_PC_TEAM CTAs with a bounded barrier of their own in global memory -- a
// barrier over all CTAs costs several microseconds, and those phases have too
// little work to use the whole grid anyway.
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

template <class R>
__device__ __forceinline__ Scope pc_scope(const LevelDev<R> &L) {
  Scope s;
  s.grid = L.n > FS_PC_TEAM_MAX;
  s.team = !s.grid && L.n > FS_PC_SMALL;
  return s;
}

template <int G, class T>
__device__ __forceinline__ T gsum(T v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// rows [0,n) by groups of G consecutive lanes; the trip count is uniform per
// warp, so every lane reaches the group shuffles (f must not return early)
template <int G, class F>
__device__ __forceinline__ void group_rows(const Scope &sc, int n, F &f) {
  constexpr int GPW = 32 / G;
  const long w0 = sc.tid0() >> 5, nw = sc.nth() >> 5;
  const int lane = threadIdx.x & 31, grp = lane / G, q = lane % G;
  for (long wb = w0 * GPW; wb < n; wb += nw * GPW) {
    long i = wb + grp;
    f(std::integral_constant<int, G>{}, i, i < n, q);
  }
}

// G from the threads per row (callers handle fewer than 2 threads per row)
template <class F>
__device__ __forceinline__ void level_rows(const Scope &sc, int n, int level, F &&f) {
  const long per = sc.nth() / (n > 0 ? n : 1);
  (void)level;
  if (per < 4) group_rows<2>(sc, n, f);
  else if (per < 8) group_rows<4>(sc, n, f);
  else group_rows<8>(sc, n, f);
}

template <class R>
struct PCycle {
  Sync &S;
  const LevelDev<R> *lev;
  int lc;              // coarsest level used by the preconditioner
  bool direct;         // coarsest by the dense inverse, else coarse_sweeps sweeps
  const double *sinv;  // lev[lc].n^2, row-major
  int pre, post, coarse_sweeps;
  R omega, alpha;        // Jacobi weight and coarse-correction factor on levels >= 1
  Scope last;            // scope of the previous phase
  R omega0, alpha0;      // the same on level 0
  unsigned *bar;         // team barrier: [0] arrivals, [1] generation (zero at launch)
  int32_t *status;       // [0] set when a team barrier timed out
  unsigned gen;          // generation this CTA waits to leave
  int extra;             // arrivals waited for beyond the team (0; >0 only to test the timeout)
  bool synced;           // the next enter() needs no barrier (the caller has just passed one)
  __device__ R om(int l) const { return l == 0 ? omega0 : omega; }
  __device__ R al(int l) const { return l == 0 ? alpha0 : alpha; }
  // barrier among the team CTAs: the arrival count in global memory, the last
  // arrival resets it and bumps the generation the others poll; polls are
  // bounded, and a timeout is recorded (later team barriers then stop
  // waiting).  The FP64 cycle calls it out of line (inlined at every phase it
  // doubled that kernel's register spills); the FP32 cycle, with fewer live
  // registers, runs faster with it inline.
  __device__ __noinline__ void team_sync_call() { team_sync_body(); }
  __device__ __forceinline__ void team_sync() {
    if (sizeof(R) == sizeof(double)) team_sync_call();
    else team_sync_body();
  }
  __device__ __forceinline__ void team_sync_body() {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned g = gen, T = (unsigned)(team_size() + extra);
      if (atomicAdd(&bar[0], 1u) == T - 1) {
        atomicExch(&bar[0], 0u);
        __threadfence();
        atomicAdd(&bar[1], 1u);
      } else {
        const volatile unsigned *vg = bar + 1;
        const volatile int32_t *vs = status;
        long spins = 0;
        while (*vg == g && *vs == 0) {
          if (++spins > FS_PC_SPIN_LIMIT) { atomicExch(status, 1); break; }
          __nanosleep(64);
        }
      }
      __threadfence();
    }
    gen++;
    __syncthreads();
  }
  // the barrier before a phase: grid-wide when the grid is involved on either
  // side, among the team when the team is, else within CTA 0
  __device__ void enter(const Scope &sc) {
    if (synced) synced = false;
    else if (sc.grid || last.grid) S.all();
    else if (sc.team || last.team) { if ((int)blockIdx.x < team_size()) team_sync(); }
    else __syncthreads();
    last = sc;
  }
  // r (into dst) = b - A x on level l; level 0 takes b from `in`
  __device__ void residual(int l, const double *__restrict__ in, const R *__restrict__ x, R *__restrict__ dst) {
    const LevelDev<R> L = lev[l];
    Scope sc = pc_scope(L);
    enter(sc);
    if (!sc.active()) return;
    if (l == 0 || sc.nth() < 2L * L.n) {   // a thread per row, two rows per step
      const long t0 = sc.tid0(), nt = sc.nth();
      for (long i = t0; i < L.n; i += 2 * nt) {
        const long i2 = i + nt;
        const bool h2 = i2 < L.n;
        R t1 = 0., t2 = 0.;
        ell_acc2<6, false>(t1, t2, L.n, L.w, L.nbr, L.anb, i, i2, h2, [&](int k) { return x[k]; });
        dst[i] = (l == 0 ? (R)in[i] : L.b[i]) - L.ac[i] * x[i] - t1;
        if (h2) dst[i2] = (l == 0 ? (R)in[i2] : L.b[i2]) - L.ac[i2] * x[i2] - t2;
      }
      return;
    }
    level_rows(sc, L.n, l, [&](auto g, long i, bool act, int q) {
      constexpr int G = decltype(g)::value;
      R t = 0.;
      if (act) t = ell_part<G, G == 1 ? 8 : 4>(L.n, L.w, L.nbr, L.anb, i, q, [&](int k) { return x[k]; });
      t = gsum<G>(t);
      if (act && q == 0) dst[i] = (l == 0 ? (R)in[i] : L.b[i]) - L.ac[i] * x[i] - t;
    });
  }
  // further Jacobi sweeps in place: residual into t, then the update
  __device__ void sweeps(int l, const double *in, R *x, int n) {
    const LevelDev<R> L = lev[l];
    Scope sc = pc_scope(L);
    for (int s = 0; s < n; s++) {
      residual(l, in, x, L.t);
      enter(sc);
      if (sc.active()) for (long i = sc.tid0(); i < L.n; i += sc.nth()) x[i] = x[i] + om(l) * L.t[i] / L.ac[i];
    }
  }
  // out = M^-1 in.  Callers have made `in` visible grid-wide.
  __device__ void run(const double *__restrict__ in, double *__restrict__ out) {
    Scope g; g.grid = true;
    {
      const LevelDev<R> L0 = lev[0];
      for (long i = g.tid0(); i < L0.n; i += g.nth()) L0.x[i] = omega0 * (R)in[i] / L0.ac[i];
    }
    last.grid = true;
    last.team = false;
    sweeps(0, in, lev[0].x, pre - 1);
    for (int l = 0; l < lc; l++) {
      const LevelDev<R> L = lev[l], C = lev[l + 1];
      residual(l, in, L.x, L.r);
      Scope scc = pc_scope(C);
      enter(scc);
      const bool first_sweep = l + 1 < lc || !direct;
      if (scc.active() && scc.nth() < 2L * C.n) {   // a thread per coarse row
        for (long P = scc.tid0(); P < C.n; P += scc.nth()) {
          R s = 0.;
          const int c0 = C.rptr[P], c1 = C.rptr[P + 1];
          for (int c = c0; c < c1; c++) s = s + L.r[C.rlist[c]];
          C.b[P] = s;
          if (first_sweep) C.x[P] = om(l + 1) * s / C.ac[P];
        }
      } else if (scc.active())
        level_rows(scc, C.n, l + 1, [&](auto gg, long P, bool act, int q) {
          constexpr int G = decltype(gg)::value;
          R s = 0.;
          if (act)
            for (int c = C.rptr[P] + q; c < C.rptr[P + 1]; c += G) s = s + L.r[C.rlist[c]];
          s = gsum<G>(s);
          if (act && q == 0) {
            C.b[P] = s;
            if (first_sweep) C.x[P] = om(l + 1) * s / C.ac[P];
          }
        });
      if (l + 1 < lc) sweeps(l + 1, in, C.x, pre - 1);
    }
    const LevelDev<R> Cc = lev[lc];
    if (direct) {
      Scope c0; c0.grid = false;
      enter(c0);
      if (blockIdx.x == 0) {
        const int n = Cc.n, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
        for (int i = threadIdx.x >> 5; i < n; i += nw) {
          double t = 0.;
          for (int j = lane; j < n; j += 32) t += sinv[(long)i * n + j] * (double)Cc.b[j];
          t = wsum(t);
          if (lane == 0) Cc.r[i] = (R)t;
        }
      }
    } else {
      sweeps(lc, in, Cc.x, coarse_sweeps - 1);
      Scope sc = pc_scope(Cc);
      enter(sc);
      if (sc.active()) for (long i = sc.tid0(); i < Cc.n; i += sc.nth()) Cc.r[i] = Cc.x[i];
    }
    for (int l = lc - 1; l >= 0; l--) {
      const LevelDev<R> L = lev[l];
      const R *__restrict__ xc = lev[l + 1].r;
      Scope sl = pc_scope(L);
      const bool to_out = l == 0 && post == 1;
      enter(sl);
      if (sl.active() && (l == 0 || sl.nth() < 2L * L.n)) {
        // a thread per row: prolong in place (x += alpha x_c[parent], each row
        // its own), then the smoothing sweep gathers x directly -- two memory
        // latencies per slot round instead of three
        const long t0 = sl.tid0(), nt = sl.nth();
        for (long i = t0; i < L.n; i += nt) L.x[i] = L.x[i] + al(l) * xc[L.parent[i]];
        enter(sl);
        for (long i = t0; i < L.n; i += 2 * nt) {
          const long i2 = i + nt;
          const bool h2 = i2 < L.n;
          R t1 = 0., t2 = 0.;
          ell_acc2<6, false>(t1, t2, L.n, L.w, L.nbr, L.anb, i, i2, h2, [&](int k) { return L.x[k]; });
          R xi = L.x[i], bi = l == 0 ? (R)in[i] : L.b[i];
          R xn = xi + om(l) * (bi - L.ac[i] * xi - t1) / L.ac[i];
          if (to_out) out[i] = (double)xn; else L.r[i] = xn;
          if (h2) {
            R xj = L.x[i2], bj = l == 0 ? (R)in[i2] : L.b[i2];
            R xm = xj + om(l) * (bj - L.ac[i2] * xj - t2) / L.ac[i2];
            if (to_out) out[i2] = (double)xm; else L.r[i2] = xm;
          }
        }
      } else if (sl.active())
        level_rows(sl, L.n, l, [&](auto gg, long i, bool act, int q) {
          constexpr int G = decltype(gg)::value;
          R t = 0.;
          if (act)
            t = ell_part<G, G == 1 ? 8 : 4>(L.n, L.w, L.nbr, L.anb, i, q,
                                            [&](int k) { return L.x[k] + al(l) * xc[L.parent[k]]; });
          t = gsum<G>(t);
          if (act && q == 0) {
            R xi = L.x[i] + al(l) * xc[L.parent[i]];
            R bi = l == 0 ? (R)in[i] : L.b[i];
            R xn = xi + om(l) * (bi - L.ac[i] * xi - t) / L.ac[i];
            if (to_out) out[i] = (double)xn; else L.r[i] = xn;
          }
        });
      if (!to_out) sweeps(l, in, L.r, post - 1);
    }
    if (post > 1) {
      enter(g);
      const LevelDev<R> L0 = lev[0];
      for (long i = g.tid0(); i < L0.n; i += g.nth()) out[i] = (double)L0.r[i];
    }
    enter(g);
  }

  // ------------------------------------------------------------ fused V-cycle
  // The same V-cycle (one pre- and one post-sweep, dense coarsest inverse) in
  // one barrier phase per level and leg, with the same arithmetic in the same
  // order as run():
  //   down: the restriction into level l+1 forms the residual of each child
  //     on the fly (no residual array, no phase of its own) for the first
  //     FS_PC_FUSE_DOWN levels; a warp takes a chunk of coarse rows, a lane
  //     two children, and each coarse row sums its children's residuals in
  //     ascending order through shuffles;
  //   up: the sweep of a row of level l >= 2 scatters its new value, times
  //     alpha, to the row's children on level l-1 (the prolongation: every
  //     finer row has one parent, so no two writes meet), and the coarsest
  //     level's dense solve does the same; level 1's sweep keeps its values
  //     and level 0 gathers them through parent (prolong0); level 0's sweep
  //     writes `out`.  (The restriction fused with the residual measured
  //     slower than the two phases on every level, so FS_PC_FUSE_DOWN is 0.)
  // The caller has set x_0 = omega0 in / ac_0 and passed a grid barrier.
  __device__ void restrict_fused(int l, const double *__restrict__ in) {
    const LevelDev<R> L = lev[l], C = lev[l + 1];
    Scope sc = pc_scope(L);
    enter(sc);
    if (!sc.active()) return;
    const bool first_sweep = l + 1 < lc || !direct;
    const R omc = om(l + 1);
    const int lane = threadIdx.x & 31;
    const long w0 = sc.tid0() >> 5, nw = sc.nth() >> 5;
    for (long k = w0; k < C.nchunk; k += nw) {
      const int P0 = C.chunk[k], P1 = C.chunk[k + 1];
      const int e0 = C.rptr[P0], e1 = C.rptr[P1];
      const int P = P0 + lane;
      const bool hasP = P < P1;
      const int ra0 = hasP ? C.rptr[P] : e1, ra1 = hasP ? C.rptr[P + 1] : e1;
      R s = 0.;
      for (int base = e0; base < e1; base += 64) {
        const int ea = base + lane, eb = ea + 32;
        const bool hb = eb < e1;
        const long ia = C.rlist[ea < e1 ? ea : e0], ib = C.rlist[hb ? eb : e0];
        R t1 = 0., t2 = 0.;
        ell_acc2<6, false>(t1, t2, L.n, L.w, L.nbr, L.anb, ia, ib, hb, [&](int q) { return L.x[q]; });
        const R va = (l == 0 ? (R)in[ia] : L.b[ia]) - L.ac[ia] * L.x[ia] - t1;
        R vb = 0.;
        if (hb) vb = (l == 0 ? (R)in[ib] : L.b[ib]) - L.ac[ib] * L.x[ib] - t2;
        // this lane's coarse row: its children inside [base, base+64), in order
        const int lo = ra0 > base ? ra0 : base, hi = ra1 < base + 64 ? ra1 : base + 64;
        const int cnt = hi > lo ? hi - lo : 0;
        const int mx = __reduce_max_sync(0xffffffffu, cnt);
        for (int m = 0; m < mx; m++) {
          const int off = lo + m - base;
          const R xa = __shfl_sync(0xffffffffu, va, off & 31);
          const R xb = __shfl_sync(0xffffffffu, vb, off & 31);
          if (m < cnt) s = s + (off < 32 ? xa : xb);
        }
      }
      if (hasP) {
        C.b[P] = s;
        if (first_sweep) C.x[P] = omc * s / C.ac[P];
      }
    }
  }
  // the residual phase and the restriction of run() (levels past FS_PC_FUSE_DOWN)
  __device__ void restrict_plain(int l, const double *__restrict__ in) {
    const LevelDev<R> L = lev[l], C = lev[l + 1];
    residual(l, in, L.x, L.r);
    Scope scc = pc_scope(C);
    enter(scc);
    if (!scc.active()) return;
    const bool first_sweep = l + 1 < lc || !direct;
    if (scc.nth() < 2L * C.n) {
      for (long P = scc.tid0(); P < C.n; P += scc.nth()) {
        R s = 0.;
        const int c0 = C.rptr[P], c1 = C.rptr[P + 1];
        // children's residuals eight at a time: their list entries, then their
        // values, all in flight before the (ascending) sum
        for (int c = c0; c < c1; c += 8) {
          int f[8];
          R v[8];
#pragma unroll
          for (int u = 0; u < 8; u++) f[u] = c + u < c1 ? C.rlist[c + u] : -1;
#pragma unroll
          for (int u = 0; u < 8; u++) v[u] = f[u] >= 0 ? L.r[f[u]] : (R)0.;
#pragma unroll
          for (int u = 0; u < 8; u++) if (f[u] >= 0) s = s + v[u];
        }
        C.b[P] = s;
        if (first_sweep) C.x[P] = om(l + 1) * s / C.ac[P];
      }
    } else
      level_rows(scc, C.n, l + 1, [&](auto gg, long P, bool act, int q) {
        constexpr int G = decltype(gg)::value;
        R s = 0.;
        if (act)
          for (int c = C.rptr[P] + q; c < C.rptr[P + 1]; c += G) s = s + L.r[C.rlist[c]];
        s = gsum<G>(s);
        if (act && q == 0) {
          C.b[P] = s;
          if (first_sweep) C.x[P] = om(l + 1) * s / C.ac[P];
        }
      });
  }
  // x_{l-1}[c] += d for the children c of row i of level l (d = alpha x_l[i])
  __device__ __forceinline__ void scatter_children(const LevelDev<R> &L, R *__restrict__ xf, long i, R d, int q0,
                                                   int step) {
    const int c1 = L.rptr[i + 1];
    for (int c = L.rptr[i] + q0; c < c1; c += 4 * step) {
      int f[4];
      R v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) f[u] = c + u * step < c1 ? L.rlist[c + u * step] : -1;
#pragma unroll
      for (int u = 0; u < 4; u++) if (f[u] >= 0) v[u] = xf[f[u]];
#pragma unroll
      for (int u = 0; u < 4; u++) if (f[u] >= 0) xf[f[u]] = v[u] + d;
    }
  }
  // the post-sweep of level l, then its prolongation into level l-1 (l >= 1)
  // or the result into `out` (l = 0)
  __device__ void smooth_scatter(int l, const double *__restrict__ in, double *__restrict__ out) {
    const LevelDev<R> L = lev[l];
    Scope sl = pc_scope(L);
    enter(sl);
    if (!sl.active()) return;
    R *__restrict__ xf = l > 0 ? lev[l - 1].x : nullptr;
    const R af = l > 0 ? al(l - 1) : (R)0.;
    if (l == 0 || sl.nth() < 2L * L.n) {   // a thread per row, two rows per step
      const long t0 = sl.tid0(), nt = sl.nth();
      for (long i = t0; i < L.n; i += 2 * nt) {
        const long i2 = i + nt;
        const bool h2 = i2 < L.n;
        R t1 = 0., t2 = 0.;
        ell_acc2<6, false>(t1, t2, L.n, L.w, L.nbr, L.anb, i, i2, h2, [&](int k) { return L.x[k]; });
        R xi = L.x[i], bi = l == 0 ? (R)in[i] : L.b[i];
        R xn = xi + om(l) * (bi - L.ac[i] * xi - t1) / L.ac[i];
        R xm = 0.;
        if (h2) {
          R xj = L.x[i2], bj = l == 0 ? (R)in[i2] : L.b[i2];
          xm = xj + om(l) * (bj - L.ac[i2] * xj - t2) / L.ac[i2];
        }
        if (l == 0) {
          out[i] = (double)xn;
          if (h2) out[i2] = (double)xm;
        } else if (gather_into(l)) {
          L.r[i] = xn;
          if (h2) L.r[i2] = xm;
        } else {
          scatter_children(L, xf, i, af * xn, 0, 1);
          if (h2) scatter_children(L, xf, i2, af * xm, 0, 1);
        }
      }
      return;
    }
    level_rows(sl, L.n, l, [&](auto gg, long i, bool act, int q) {
      constexpr int G = decltype(gg)::value;
      R t = 0.;
      if (act) t = ell_part<G, G == 1 ? 8 : 4>(L.n, L.w, L.nbr, L.anb, i, q, [&](int k) { return L.x[k]; });
      t = gsum<G>(t);
      if (act) {
        R xi = L.x[i], bi = L.b[i];
        R xn = xi + om(l) * (bi - L.ac[i] * xi - t) / L.ac[i];
        if (!gather_into(l)) scatter_children(L, xf, i, af * xn, q, G);
        else if (q == 0) L.r[i] = xn;
      }
    });
  }
  // level 1's post-sweep leaves its result in its r, and level 0 gathers the
  // correction through parent in a phase of its own (x_0 += alpha x_1[parent],
  // the same sum the scatter forms): a coalesced pass over the fine rows
  // instead of one read-modify-write per fine row in agglomerate order.  At
  // 128^3 the extra grid barrier costs less than the scattered writes: the
  // FP64 p' solve 2 % faster, and the FP32 one, which ran the unfused cycle
  // before, 10 %.
  __device__ __forceinline__ bool gather_into(int l) const { return l == 1 && lc >= 2; }
  __device__ void prolong0() {
    const LevelDev<R> L = lev[0];
    const R *__restrict__ xc = lev[1].r;
    Scope g;
    g.grid = true;
    enter(g);
    const R a0 = al(0);
    for (long i = g.tid0(); i < L.n; i += g.nth()) L.x[i] = L.x[i] + a0 * xc[L.parent[i]];
  }
  // the dense coarsest solve (CTA 0, warps on rows), scattered into level lc-1
  __device__ void coarsest_scatter() {
    Scope c0;
    c0.grid = false;
    enter(c0);
    if (blockIdx.x != 0) return;
    const LevelDev<R> Cc = lev[lc];
    R *__restrict__ xf = lev[lc - 1].x;
    const R af = al(lc - 1);
    const int n = Cc.n, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = threadIdx.x >> 5; i < n; i += nw) {
      double t = 0.;
      for (int j = lane; j < n; j += 32) t += sinv[(long)i * n + j] * (double)Cc.b[j];
      t = wsum(t);
      t = __shfl_sync(0xffffffffu, t, 0);
      scatter_children(Cc, xf, i, af * (R)t, lane, 32);
    }
  }
  // ------------------------------------------------------------ Gauss-Seidel V-cycle
  // One multicolour Gauss-Seidel pass over level l in place: the colours in
  // order (forward) or reversed (backward); rows of one colour read only
  // rows of other colours, so each colour is one phase of independent rows.
  __device__ void gs_colours(int l, const double *__restrict__ in, R *__restrict__ x, bool backward) {
    const LevelDev<R> L = lev[l];
    Scope sc = pc_scope(L);
    for (int cc = 0; cc < L.ncolors; cc++) {
      const int c = backward ? L.ncolors - 1 - cc : cc;
      enter(sc);
      if (!sc.active()) continue;
      const int r0 = L.color_ptr[c], r1 = L.color_ptr[c + 1];
      for (long q = r0 + sc.tid0(); q < r1; q += sc.nth()) {
        const int i = L.color_rows[q];
        const R t = ell_acc<6, false>((R)0., L.n, L.w, L.nbr, L.anb, i, [&](int k) { return x[k]; });
        const R bi = l == 0 ? (R)in[i] : L.b[i];
        x[i] = (bi - t) / L.ac[i];
      }
    }
  }
  // The V-cycle with symmetric multicolour Gauss-Seidel smoothing on the
  // levels below FS_PC_GS_LEVELS (a forward pass from zero before the
  // restriction and, after the correction x += alpha x_c[parent], a backward
  // pass) and the damped Jacobi sweeps of run() on the others; the coarsest
  // level by the dense inverse.  Results stay in each level's x.  out =
  // M^-1 in; callers have made `in` visible.
  __device__ void run_gs(const double *__restrict__ in, double *__restrict__ out) {
    Scope g;
    g.grid = true;
    const LevelDev<R> L0 = lev[0];
    for (long i = g.tid0(); i < L0.n; i += g.nth()) L0.x[i] = (R)0.;
    last.grid = true;
    last.team = false;
    gs_colours(0, in, L0.x, false);
    for (int l = 0; l < lc; l++) {
      const LevelDev<R> L = lev[l], C = lev[l + 1];
      residual(l, in, L.x, L.r);
      Scope scc = pc_scope(C);
      enter(scc);
      const bool gsc = l + 1 < FS_PC_GS_LEVELS;
      const R omc = (gsc || l + 1 == lc) ? (R)0. : om(l + 1);   // Jacobi: the first sweep from zero
      if (scc.active())
        for (long P = scc.tid0(); P < C.n; P += scc.nth()) {
          R s = 0.;
          for (int c = C.rptr[P]; c < C.rptr[P + 1]; c++) s = s + L.r[C.rlist[c]];
          C.b[P] = s;
          C.x[P] = omc * s / C.ac[P];
        }
      if (l + 1 < lc && gsc) gs_colours(l + 1, in, C.x, false);
    }
    {
      Scope c0;
      c0.grid = false;
      enter(c0);
      if (blockIdx.x == 0) {
        const LevelDev<R> Cc = lev[lc];
        const int n = Cc.n, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
        for (int i = threadIdx.x >> 5; i < n; i += nw) {
          double t = 0.;
          for (int j = lane; j < n; j += 32) t += sinv[(long)i * n + j] * (double)Cc.b[j];
          t = wsum(t);
          if (lane == 0) Cc.x[i] = (R)t;
        }
      }
    }
    for (int l = lc - 1; l >= 0; l--) {
      const LevelDev<R> L = lev[l];
      const R *__restrict__ xc = lev[l + 1].x;
      Scope sl = pc_scope(L);
      enter(sl);
      if (sl.active())
        for (long i = sl.tid0(); i < L.n; i += sl.nth()) L.x[i] = L.x[i] + al(l) * xc[L.parent[i]];
      if (l < FS_PC_GS_LEVELS) {
        gs_colours(l, in, L.x, true);
      } else {   // one damped Jacobi sweep in place: residual into t, then the update
        residual(l, in, L.x, L.t);
        enter(sl);
        if (sl.active()) for (long i = sl.tid0(); i < L.n; i += sl.nth()) L.x[i] = L.x[i] + om(l) * L.t[i] / L.ac[i];
      }
    }
    enter(g);
    for (long i = g.tid0(); i < L0.n; i += g.nth()) out[i] = (double)L0.x[i];
    enter(g);
  }

  __device__ void run_fused(const double *__restrict__ in, double *__restrict__ out) {
    Scope g;
    g.grid = true;
    last.grid = true;
    last.team = false;
    synced = true;   // the caller's grid barrier stands for the first phase's
    for (int l = 0; l < lc; l++) {
      if (l < FS_PC_FUSE_DOWN) restrict_fused(l, in);
      else restrict_plain(l, in);
    }
    coarsest_scatter();
    for (int l = lc - 1; l >= 0; l--) {
      if (l == 0 && gather_into(1)) prolong0();
      smooth_scatter(l, in, out);
    }
    enter(g);
  }
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

// rows i and i2 (when h2) of A x at once (ell_acc2)
template <class A>
__device__ __forceinline__ void row_ax2(const A &a, long i, long i2, bool h2, const double *x, double &t1, double &t2) {
  t1 = 0.0;
  t1 = t1 + a.ac[i] * x[i];
  t2 = 0.0;
  if (h2) t2 = t2 + a.ac[i2] * x[i2];
  ell_acc2<6, false>(t1, t2, a.N, a.W, a.cn, a.anb, i, i2, h2, [&](int k) { return x[k]; });
}

// apply the preconditioner: out (FP64) = M^-1 in (FP64), via the R-precision
// V-cycle; `fused`: the caller has set x_0 = omega0 in / ac_0 (run_fused)
// MODE: 0 the V-cycle of run(), 1 run_fused(), 2 run_gs()
template <class R, int MODE>
__device__ void apply_prec(Sync &S, const AmgKArgs<R> &a, const double *in, double *out, unsigned &gen) {
  Scope all;
  all.grid = true;
  PCycle<R> C{S, a.lev, a.lc, a.direct != 0, a.sinv, a.pre, a.post, 20, (R)FS_MG_OMEGA, (R)FS_MG_ALPHA, all,
               (R)FS_MG_OMEGA0, (R)FS_MG_ALPHA0, a.teambar, a.status, gen, a.team_extra, false};
  if (MODE == 1) C.run_fused(in, out);
  else if (MODE == 2) C.run_gs(in, out);
  else C.run(in, out);
  gen = C.gen;
}

// mean of the right-hand side of a pure-Neumann system (every row sums to
// zero), else 0; the same grid-deterministic sums in every kernel that calls it
template <class R>
__device__ double rhs_mean(Sync &S, const AmgKArgs<R> &a) {
  const int N = a.N;
  const long t0 = (long)blockIdx.x * blockDim.x + threadIdx.x, nt = (long)gridDim.x * blockDim.x;
  double nonsing = 0., bsum = 0.;
  for (long i = t0; i < N; i += nt) {
    double rs = a.ac[i];
    for (int j = 0; j < a.W; j++)
      if (a.cn[(long)j * N + i] >= 0) rs += a.anb[(long)j * N + i];
    nonsing += fabs(rs) > 1e-9 * fabs(a.ac[i]) ? 1. : 0.;
    bsum += a.bc[i];
  }
  double n_nonsing, b_total;
  S.sum2(nonsing, bsum, n_nonsing, b_total);
  return n_nonsing == 0. ? b_total / N : 0.;
}

// The initial guess of k_amg_bicgstab, one cooperative launch before it: the
// combination x = sum_j c_j x_j of the basis vectors (previous p' solutions,
// the network's guess) that minimises |b - A x|, least squares over their
// span, so |b - A x| <= |b|.  The normal equations (Gram matrix of the A x_j)
// are solved by every CTA alike from grid-deterministic sums, by a Cholesky
// factorisation with a relative diagonal shift.  x goes to a.x and fit[0] = 1;
// a failed factorisation leaves fit[0] = 0 (the solve starts from zero).
template <class R>
__global__ void __launch_bounds__(FS_COOP_BLOCK, 1) k_guess_fit(AmgKArgs<R> a) {
  Sync S(a.part);
  const int N = a.N, nx = a.nx;
  const long t0 = (long)blockIdx.x * blockDim.x + threadIdx.x, nt = (long)gridDim.x * blockDim.x;
  const double bmean = rhs_mean(S, a);
  double c[FS_GUESS_MAX];
  for (int j = 0; j < FS_GUESS_MAX; j++) c[j] = 0.;
  bool fell_back = false;
  {
    // Gram matrix G_jk = (A x_j).(A x_k) (upper triangle), g_j = (A x_j).b, |b|^2
    double acc[FS_SUMK];
    const int ng = nx * (nx + 1) / 2;
    for (int k = 0; k < ng + nx + 1; k++) acc[k] = 0.;
    for (long i = t0; i < N; i += nt) {
      double y[FS_GUESS_MAX];
      for (int j = 0; j < nx; j++) {
        const double *xj = a.xs[j];
        double t = 0.;
        t = t + a.ac[i] * xj[i];
        y[j] = ell_acc<8, false>(t, a.N, a.W, a.cn, a.anb, i, [&](int k) { return xj[k]; });
      }
      const double b1 = a.bc[i] - bmean;
      int q = 0;
      for (int j = 0; j < nx; j++)
        for (int k = j; k < nx; k++) acc[q++] += y[j] * y[k];
      for (int j = 0; j < nx; j++) acc[ng + j] += y[j] * b1;
      acc[ng + nx] += b1 * b1;
    }
    double tot[FS_SUMK];
    S.sumK(acc, tot, ng + nx + 1);
    // Cholesky of G + 1e-12 max(diag) I, then the two triangular solves (row-major L)
    double L[FS_GUESS_MAX * FS_GUESS_MAX];
    double dmax = 0.;
    {
      int q = 0;
      for (int j = 0; j < nx; j++)
        for (int k = j; k < nx; k++) { L[k * FS_GUESS_MAX + j] = tot[q]; if (k == j) dmax = fmax(dmax, tot[q]); q++; }
    }
    bool ok = dmax > 0. && isfinite(dmax);
    for (int j = 0; j < nx && ok; j++) {
      double d = L[j * FS_GUESS_MAX + j] + 1e-12 * dmax;
      for (int k = 0; k < j; k++) d -= L[j * FS_GUESS_MAX + k] * L[j * FS_GUESS_MAX + k];
      if (!(d > 1e-14 * dmax)) { ok = false; break; }
      d = sqrt(d);
      L[j * FS_GUESS_MAX + j] = d;
      for (int r = j + 1; r < nx; r++) {
        double v = L[r * FS_GUESS_MAX + j];
        for (int k = 0; k < j; k++) v -= L[r * FS_GUESS_MAX + k] * L[j * FS_GUESS_MAX + k];
        L[r * FS_GUESS_MAX + j] = v / d;
      }
    }
    if (ok) {
      double z[FS_GUESS_MAX];
      for (int j = 0; j < nx; j++) {
        double v = tot[ng + j];
        for (int k = 0; k < j; k++) v -= L[j * FS_GUESS_MAX + k] * z[k];
        z[j] = v / L[j * FS_GUESS_MAX + j];
      }
      for (int j = nx - 1; j >= 0; j--) {
        double v = z[j];
        for (int k = j + 1; k < nx; k++) v -= L[k * FS_GUESS_MAX + j] * c[k];
        c[j] = v / L[j * FS_GUESS_MAX + j];
      }
      for (int j = 0; j < nx; j++) if (!isfinite(c[j])) ok = false;
    }
    if (!ok) for (int j = 0; j < nx; j++) c[j] = 0.;
    fell_back = !ok;
    for (long i = t0; i < N; i += nt) {
      double xi = 0.;
      for (int j = 0; j < nx; j++) xi += c[j] * a.xs[j][i];
      a.x[i] = xi;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.fit[0] = fell_back ? 0 : 1;
    if (a.nncnt) { a.nncnt[1] += 1; if (fell_back) a.nncnt[0] += 1; }
  }
}

// right-preconditioned BiCGSTAB (van der Vorst 1992) with a multigrid V-cycle:
// MODE 0 run(), 2 run_gs() (multicolour Gauss-Seidel smoothing), 1 the fused
// V-cycle (one pre- and one post-sweep, dense coarsest level), whose first
// sweep from zero, x_0 = omega0 in / ac_0, rides on the loops that form p and s.
// Four grid synchronisations per iteration besides the V-cycles': the sums
// after v = A y and after s, the sums after t = A z, and the barrier after one
// pass that updates x and r and forms the next p.  That pass needs beta
// before |r|^2 and r0.r of the new r are summed; both come from the t-pass
// sums instead: r0.r_new = r0.s - omega r0.t, and |s - omega t|^2 = |s|^2 -
// omega t.s (omega = t.s / t.t), with |s|^2 summed fresh from s, so the
// estimate's rounding is relative to |s|^2 of this iteration.  Only an
// iteration whose estimate says it has converged (or the last one) sums |r|^2
// and r0.r of the stored r instead, so the exit is always decided on a
// residual summed from its vector, and a solve that has not really converged
// continues with p formed in a separate pass.
template <class R, int MODE>
__global__ void __launch_bounds__(FS_COOP_BLOCK, FS_AMG_MINB) k_amg_bicgstab(AmgKArgs<R> a) {
  Sync S(a.part);
  unsigned gen = 0;   // team-barrier generation (the counters are zeroed before the launch)
  const int N = a.N;
  Scope g; g.grid = true;
  const long t0 = g.tid0(), nt = g.nth();
  R *__restrict__ x0v = a.lev[0].x;
  const R *__restrict__ ac0 = a.lev[0].ac;
  const R om0 = (R)FS_MG_OMEGA0;
  // start from the initial guess k_guess_fit left in x (the least-squares
  // combination of the basis vectors; fit[0] = 0 when it fell back), or from zero.
  // A pure-Neumann system (every row sums to zero: the closed-cavity p'
  // system) is singular.  Its right-hand side is taken with its mean removed,
  // the part a solution can match; otherwise, once the outer iterations have
  // converged the mean (rounding in the mass fluxes) is no longer small
  // against |b|, the tolerance cannot be met and the iterates drift.  The
  // constant null vector is left to the caller (pressure reference cell).
  const double bmean = rhs_mean(S, a);
  const bool has_x = a.nx > 0 && a.fit[0] != 0;
  double l0 = 0., l1 = 0., l2 = 0.;
  for (long i = t0; i < N; i += nt) {
    const double b1 = a.bc[i] - bmean;
    double ri = b1;
    if (has_x) {
      double t = 0.;
      t = t + a.ac[i] * a.x[i];
      t = ell_acc<8, false>(t, a.N, a.W, a.cn, a.anb, i, [&](int k) { return a.x[k]; });
      ri = ri - t;
    } else {
      a.x[i] = 0.;
    }
    // the first p is r (beta's factors are 1 and p = v = 0 before it)
    a.r[i] = ri; a.r0[i] = ri; a.p[i] = ri; a.v[i] = 0.;
    if (MODE == 1) x0v[i] = om0 * (R)ri / ac0[i];
    l0 += ri * ri;
    l1 += b1 * b1;
  }
  double rr, bb, dum;
  S.sum2(l0, l1, rr, bb);
  double normb = sqrt(bb), alpha = 1., omega = 1.;
  int k = 0;
  double resn = sqrt(rr);
  // rho = r0 . r of the iteration; rho_next that of the next one, summed from
  // the stored r when p still has to be formed (p_ready false)
  double rho = rr, rho_next = rr;
  bool p_ready = true;
  if (!(rr != 0.) || !isfinite(rr)) p_ready = false;   // the loop's breakdown test takes it
  while (k < a.maxit && resn > a.tol * normb && normb > 0.) {
    k++;
    if (!p_ready) {
      const double rho1 = rho_next;
      // breakdown (r0 . r vanished: r at round-off): keep x.  Every CTA holds
      // the same sums, so every CTA takes the same branch.
      if (!(rho1 != 0.) || !isfinite(rho1)) break;
      const double beta = (rho1 / rho) * (alpha / omega);
      rho = rho1;
      for (long i = t0; i < N; i += nt) {
        const double pi = a.r[i] + beta * (a.p[i] - omega * a.v[i]);
        a.p[i] = pi;
        if (MODE == 1) x0v[i] = om0 * (R)pi / ac0[i];
      }
      S.all();
    }
    p_ready = false;
    apply_prec<R, MODE>(S, a, a.p, a.y, gen);                       // y = M^-1 p
    l0 = 0.;
    for (long i = t0; i < N; i += 2 * nt) {
      const long i2 = i + nt;
      const bool h2 = i2 < N;
      double v1, v2;
      row_ax2(a, i, i2, h2, a.y, v1, v2);
      a.v[i] = v1; l0 += a.r0[i] * v1;
      if (h2) { a.v[i2] = v2; l0 += a.r0[i2] * v2; }
    }
    double rv;
    S.sum2(l0, 0., rv, dum);
    if (!(rv != 0.) || !isfinite(rho / rv)) break;
    alpha = rho / rv;
    l0 = 0.; l1 = 0.;
    for (long i = t0; i < N; i += nt) {
      const double si = a.r[i] - alpha * a.v[i];
      a.s[i] = si;
      l0 += si * si;
      l1 += a.r0[i] * si;
      if (MODE == 1) x0v[i] = om0 * (R)si / ac0[i];
    }
    double ss, r0s;
    S.sum2(l0, l1, ss, r0s);
    if (sqrt(ss) <= a.tol * normb) {
      for (long i = t0; i < N; i += nt) a.x[i] = a.x[i] + alpha * a.y[i];
      resn = sqrt(ss);
      break;
    }
    apply_prec<R, MODE>(S, a, a.s, a.z, gen);                       // z = M^-1 s
    l0 = 0.; l1 = 0.; l2 = 0.;
    for (long i = t0; i < N; i += 2 * nt) {
      const long i2 = i + nt;
      const bool h2 = i2 < N;
      double t1, t2;
      row_ax2(a, i, i2, h2, a.z, t1, t2);
      a.t[i] = t1; l0 += t1 * a.s[i]; l1 += t1 * t1; l2 += a.r0[i] * t1;
      if (h2) { a.t[i2] = t2; l0 += t2 * a.s[i2]; l1 += t2 * t2; l2 += a.r0[i2] * t2; }
    }
    double ts, tt, r0t;
    S.sum3(l0, l1, l2, ts, tt, r0t);
    if (!(tt > 0.) || !(ts != 0.) || !isfinite(ts / tt)) {
      // t = A z vanished or is orthogonal to s: take the half step and stop
      for (long i = t0; i < N; i += nt) a.x[i] = a.x[i] + alpha * a.y[i];
      resn = sqrt(ss);
      break;
    }
    omega = ts / tt;
    const double rn_est = fmax(ss - omega * ts, 0.);
    const double rho_est = r0s - omega * r0t;
    if (k < a.maxit && sqrt(rn_est) > a.tol * normb && rho_est != 0. && isfinite(rho_est)) {
      // x and r of this iteration and p of the next in one pass
      const double beta = (rho_est / rho) * (alpha / omega);
      rho = rho_est;
      for (long i = t0; i < N; i += nt) {
        a.x[i] = a.x[i] + alpha * a.y[i] + omega * a.z[i];
        const double ri = a.s[i] - omega * a.t[i];
        a.r[i] = ri;
        const double pi = ri + beta * (a.p[i] - omega * a.v[i]);
        a.p[i] = pi;
        if (MODE == 1) x0v[i] = om0 * (R)pi / ac0[i];
      }
      S.all();
      resn = sqrt(rn_est);
      p_ready = true;
    } else {
      l0 = 0.; l1 = 0.;
      for (long i = t0; i < N; i += nt) {
        a.x[i] = a.x[i] + alpha * a.y[i] + omega * a.z[i];
        const double ri = a.s[i] - omega * a.t[i];
        a.r[i] = ri;
        l0 += ri * ri;
        l1 += a.r0[i] * ri;
      }
      double rn;
      S.sum2(l0, l1, rn, rho_next);
      resn = sqrt(rn);
    }
  }
  S.all();
  for (long i = t0; i < N; i += nt) a.dphi[i] = a.x[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) { *a.iters = k; a.diag[0] = resn; a.diag[1] = normb; }
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
  if (!f32) {
    AmgKArgs<double> a{};
    fill(a);
    a.lev = M->lev64;
    void *args[] = {&a};
    if (a.nx > 0) FS_CK(fs_coop_launch((const void *)k_guess_fit<double>, G, fs_coop_block(ctx), args, ctx->st));
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][0], ctx->st)));
    FS_CK(fs_coop_launch(fused ? (const void *)k_amg_bicgstab<double, 1> : (const void *)k_amg_bicgstab<double, 0>,
                         G, fs_coop_block(ctx), args, ctx->st));
  } else {
    AmgKArgs<float> a{};
    fill(a);
    a.lev = M->lev32;
    void *args[] = {&a};
    if (a.nx > 0) FS_CK(fs_coop_launch((const void *)k_guess_fit<float>, G, fs_coop_block(ctx), args, ctx->st));
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
