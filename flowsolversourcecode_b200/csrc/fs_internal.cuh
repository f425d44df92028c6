// fs_internal.cuh -- device context of the B200 SIMPLE inner loop.
//
// Data layout in HBM (all FP64 unless noted, SoA so every kernel streams
// contiguous arrays):
//   cells  (N):  vol, xc/yc/zc, u/v/w/p/pc, gradients as 3 blocks of N
//   slots (W*N, slot-major like the reference's anb(N,NElementFaces)):
//          slot[j*N+i] = (face<<1)|side  (face < F interior, F+b boundary;
//          side 1 = this cell is the face's neighbour), -1 unused;
//          cn[j*N+i]   = neighbour cell or -1 (ElementNeighbor)
//   interior faces (F): own/nbr (int32), gf, S, dCF vector and length,
//          gDiff, T vector, dfp = r_f - r_f' (Green-Gauss correction vector)
//   boundary faces (B, linear patch-major index = reference i4-NIFaces):
//          own, type (int32), S, |S|, n, dCF (BDistanceCF), gDiff, T, nz(i,i)
//   matrix: ac (N), anb (W*N slot-major), bc (N)
#pragma once
#include "../../include/fsb200.h"
#include <cuda_runtime.h>
#include <string>
#include <vector>
#include <cstdint>

// 'specifiedvelocity' and 'specifiedmassflowrate' inlets share the momentum,
// p' and k-epsilon treatment (AssembleIsotropicDiffusion.for:254-300,
// AssembleConvection.for:260-300, AssemblePressureCorrectionFluxes.for:545-575)
__host__ __device__ inline bool fs_is_inlet(int t) {
  return t == FS_BC_INLET_VEL || t == FS_BC_INLET_MASS || t == FS_BC_INLET_SP || t == FS_BC_INLET_STAG;
}
// static- and stagnation-pressure inlets: the same loop bodies everywhere but
// in the boundary pressure and the p' coefficients (incompressible)
__host__ __device__ inline bool fs_is_p_inlet(int t) { return t == FS_BC_INLET_SP || t == FS_BC_INLET_STAG; }
// static pressure specified: Rhie-Chow boundary flux and p'_b = 0
// (AssembleMdotUsingRhieChow.for:1441-1598, 2105-2283)
__host__ __device__ inline bool fs_is_pressure(int t) {
  return t == FS_BC_OUTLET_SP || t == FS_BC_INLET_SP || t == FS_BC_OUTLET_ASP || t == FS_BC_OUTLET_RES ||
         t == FS_BC_INLET_STAG;
}
// static-pressure, average-static-pressure and resistance outlets: one
// treatment in every routine but the p' coefficients, the p' boundary values
// and CorrectPressure (the other loops of the three types are the same text)
__host__ __device__ inline bool fs_is_sp_outlet(int t) {
  return t == FS_BC_OUTLET_SP || t == FS_BC_OUTLET_ASP || t == FS_BC_OUTLET_RES;
}
// p'_b = 0 (UpdatePressureCorrectionAtBoundaries.for:85-90, 126-143)
__host__ __device__ inline bool fs_pc_dirichlet(int t) {
  return t == FS_BC_OUTLET_SP || t == FS_BC_INLET_SP || t == FS_BC_OUTLET_ASP;
}
// the velocity follows from Bmdot along a given direction (AssembleMdotUsingRhieChow.for:2089-2099)
__device__ __forceinline__ void fs_directed_velocity(const double *bdir, const double *bsf, double rho, int B, int b,
                                                     double bm, double *bu, double *bv, double *bw) {
  const double dx = bdir[3L * b], dy = bdir[3L * b + 1], dz = bdir[3L * b + 2];
  const double vm = bm / (rho * (dx * bsf[b] + dy * bsf[B + b] + dz * bsf[2L * B + b]));
  bu[b] = vm * dx; bv[b] = vm * dy; bw[b] = vm * dz;
}

#define FS_BLOCK 256
#ifndef FS_COOP_BLOCK
#define FS_COOP_BLOCK 1024           // most threads per CTA of the persistent cooperative solvers
#endif
#define FS_RED_BLOCKS 1184           // 148 SMs x 8: partial-sum slots of the grid reductions

// reduction slots in ctx->red (double); each quantity has FS_RED_BLOCKS partials
enum { RED_SUM0 = 0, RED_SUM1, RED_SUM2, RED_MAX0, RED_MAX1, RED_NQ };

struct fs_mg_dev;  // multigrid hierarchy (fs_mg.cu)
struct fs_turb;    // k-epsilon state (fs_turb.cu)
struct fs_energy;  // temperature equation state (fs_energy.cu)
struct fs_nn;      // learned p' initial guess (fs_nn.cu)
struct fs_ilu;     // D-ILU level schedule (fs_solvers.cu)

#define FS_NEQ 9        // equations with residual slots: NF 1..9
#define FS_NLEVELS 7    // unsteady time levels: u v w p k epsilon T
#define FS_GUESS_MAX 8  // vectors of the p' initial-guess fit (history + the network's guess)
#define FS_NITERS 16     // int32 iteration-count slots (NF - 1 indexed)

struct fs_ctx {
  int dev = 0;
  cudaStream_t st = nullptr;
  fs_case cfg{};
  int N = 0, F = 0, B = 0, W = 0, NS = 0;
  int nIter = 0;
  double div_ref = 0.;   // largest stop metric so far (divergence check), 0 = none yet
  int64_t launches = 0;
  std::string err;
  int num_sms = 148;

  // host copies (connectivity restated from Readit, 0-based)
  std::vector<int32_t> h_ncf, h_cf, h_cn, h_own_slot, h_nbr_slot, h_fown, h_fnbr, h_bown, h_bset;
  std::vector<int32_t> h_bset_start, h_bset_n, h_btype;
  std::vector<int32_t> h_color_ptr, h_color_rows;  // multicolour ordering for GS
  int ncolors = 0;

  // connectivity (device)
  int32_t *slot = nullptr, *cn = nullptr, *ncf = nullptr;
  int32_t *fown = nullptr, *fnbr = nullptr, *bown = nullptr, *btype = nullptr;
  int32_t *color_rows = nullptr;
  // colour-major copy of the matrix for the Gauss-Seidel sweeps: position p holds
  // row color_rows[p]; cnP/ncfP are fixed per mesh, acP/bcP/anbP/dphiP per solve
  int32_t *cposP = nullptr, *cnP = nullptr, *ncfP = nullptr;
  double *acP = nullptr, *bcP = nullptr, *anbP = nullptr, *dphiP = nullptr;
  // multi-RHS momentum: the three systems (3N each) in cell and colour-major order
  double *ac3 = nullptr, *bc3 = nullptr, *ac3P = nullptr, *bc3P = nullptr, *x3P = nullptr;

  // geometry (device)
  double *vol = nullptr, *xc = nullptr;                     // xc: 3N
  double *gf = nullptr, *sf = nullptr, *dcfv = nullptr, *dcf = nullptr, *gdiff = nullptr;  // sf,dcfv: 3F
  double *tf = nullptr, *dfp = nullptr, *fa = nullptr;      // 3F, 3F, F
  double *bsf = nullptr, *bfa = nullptr, *bnf = nullptr, *bdv = nullptr, *bgdiff = nullptr, *btf = nullptr, *bnzii = nullptr;

  // state (device)
  double *u = nullptr, *v = nullptr, *w = nullptr, *p = nullptr, *pc = nullptr, *mdot = nullptr;
  double *bu = nullptr, *bv = nullptr, *bw = nullptr, *bp = nullptr, *bpc = nullptr, *bmdot = nullptr;
  double *ug = nullptr, *vg = nullptr, *wg = nullptr, *pg = nullptr, *pcg = nullptr;      // 3N
  double *bug = nullptr, *bvg = nullptr, *bwg = nullptr, *bpg = nullptr, *bpcg = nullptr; // 3B
  double *gtmp = nullptr;                                  // 12N double buffer for GG passes
  double *du1 = nullptr, *dv1 = nullptr, *dw1 = nullptr, *du2 = nullptr, *dv2 = nullptr, *dw2 = nullptr;
  double *us = nullptr, *vs = nullptr, *ws = nullptr;

  // assembly (device)
  double *ac = nullptr, *anb = nullptr, *bc = nullptr, *dphi = nullptr;
  double *ac_int = nullptr, *bc_int = nullptr, *effdiv = nullptr;  // bc_int: 3N
  double *pcoef = nullptr;                                         // F: p' face coefficient
  double *bpcoef = nullptr;                                        // B: p' coefficient of pressure outlets (FluxFf)
  double *bpcoefc = nullptr;                                       // B: its diagonal part FluxCf (resistance, stagnation)
  double *bgd = nullptr;                                           // B: geoDiff of 'specifiedresistance' faces
  double *bp0 = nullptr;                                           // B: patch_pressure per face (stagnation p0)
  double *d_patch = nullptr;                                       // 2*FS_MAX_PATCHES: resistance R, then sum geoDiff
  bool has_res = false, has_stag = false;                          // resistance outlets, stagnation inlets
  bool has_sp = false;                                             // a 'specifiedstaticpressure' outlet exists
  double *bdir = nullptr;                                          // 3B: direction of 'specifiedmassflowrate' inlets
  // krylov work (device)
  double *kx = nullptr, *kr = nullptr, *kr0 = nullptr, *kp = nullptr, *kv = nullptr, *ks = nullptr, *kt = nullptr;
  double *kz = nullptr, *ky = nullptr;   // preconditioned vectors (AMG-BiCGSTAB)
  double *sysx = nullptr;                // fs_solve_system_host: the field the update is added to
  double *gm = nullptr;                  // GMRES work: 21 Krylov vectors + 7 (allocated on first use)
  // reductions
  double *red = nullptr;        // RED_NQ * FS_RED_BLOCKS partials
  int64_t *redi = nullptr;      // FS_RED_BLOCKS argmax partials
  double *resblk = nullptr;     // device residual block, layout of fs_residuals' first 20 doubles + extras
  int32_t *d_iters = nullptr;   // linear iterations per NF (FS_NITERS slots, NF 1..9 used)
  int32_t *d_status = nullptr;  // device-side status flags

  // boundary patch per boundary face (device), outlet mass-flow scratch:
  // [0] mdotIn, [1 + s] mdot1(s), [1 + FS_MAX_PATCHES + s] mdotOut(s)
  int32_t *d_bset = nullptr;
  double *flow = nullptr;
  // unsteady runs: u v w p k epsilon T at time levels n-1, n-2 (FS_NLEVELS N each),
  // their boundary values at n-1 (FS_NLEVELS B), p at the last X-momentum gradient ('cranknicolson1')
  double *old = nullptr, *oldold = nullptr, *bold = nullptr, *p_mx = nullptr;
  double dt = 0., dto = 0., dtoo = 0., time = 0.;
  int ndt = 0, tscheme = 0;      // tscheme: the TransientScheme in effect
  // k-epsilon (nullptr: laminar)
  fs_turb *turb = nullptr;
  fs_energy *energy = nullptr;
  // multigrid
  fs_mg_dev *mg = nullptr;
  // level schedule and factor of the 'ilu' solver (built on first use)
  fs_ilu *ilu = nullptr;
  // learned initial guess of the p' solve (nullptr: zero guess)
  fs_nn *nn = nullptr;
  // initial-guess basis of the p' solve (set around it only): previous p'
  // solutions, then the network's guess
  const double *pc_guess[FS_GUESS_MAX] = {};
  int pc_nguess = 0;
  bool pc_nn = false;   // the last basis vector is the network's guess
  // previous p' solutions kept for the guess (fs_set_pc_history): hist_cap
  // slots of N, slot 0 the newest, hist_cnt filled
  double *hist = nullptr;
  int hist_cap = 0, hist_cnt = 0;

  // timing
  cudaEvent_t tev[2] = {};                 // fs_timer_start / fs_timer_stop
  cudaEvent_t sev[FS_NEQ][2] = {};         // around the solver launch of each NF
  bool s_pending[FS_NEQ] = {};
  float s_ms[FS_NEQ] = {};
  cudaEvent_t kev[FS_NEQ][2] = {};         // around the main cooperative kernel of each solve
  float k_ms[FS_NEQ] = {};
  int32_t s_its[FS_NEQ] = {}, s_calls[FS_NEQ] = {};
  cudaEvent_t ev[6] = {};
  float phase_ms[5] = {};
  int coop_grid = 0;            // blocks of a cooperative solver launch
  int coop_per_sm = 0;          // launch shape: cooperative CTAs per SM (0: up to 4; fs_set_launch_shape)
  bool graph_mode = false;      // enqueueing for stream capture: no host syncs, no timing events
  bool pc_defer = false;        // the AMG-BiCGSTAB solve prepares its launch and leaves it to fs_pc_batch_launch
  bool mom_defer = false;       // the multi-RHS momentum solve prepares its launch for fs_mom_batch_launch
  double ens_split = 1.;        // batched ensembles: CTA groups in proportion to cells^ens_split (x p' iterations)
  bool mom_pending = false;
  alignas(8) unsigned char mom_pend[160];   // the prepared launch's arguments (Sor3Args)
  int test_wait_extra = 0;      // fs_test_wait_timeout: extra arrivals the team barrier waits for
};

// timing events and their host-side bookkeeping are skipped while a graph is captured
#define FS_TIMING(stmt)                                                      \
  do {                                                                       \
    if (!ctx->graph_mode) { stmt; }                                          \
  } while (0)

// residual block layout on the device (double resblk[RB_SIZE]): four norms of
// NF 1..9 (u, v, w, p', mass, -, -, k, epsilon), the overall imbalance and its
// cell, the last linear solve's final residual and |b|, and the inlet mass
// flow of the last continuity residual (the module's mdotIn)
enum { RB_ABS = 0, RB_MAX = 9, RB_RMS = 18, RB_SCL = 27, RB_OVERALL = 36, RB_IMAX = 37,
       RB_DIAG = 38, RB_MDOTIN = 40, RB_SIZE = 41 };

#define FS_CK(call)                                                          \
  do {                                                                       \
    cudaError_t e__ = (call);                                                \
    if (e__ != cudaSuccess) {                                                \
      ctx->err = std::string(#call) + ": " + cudaGetErrorString(e__);        \
      return FS_E_CUDA;                                                      \
    }                                                                        \
  } while (0)

#define FS_STR2(x) #x
#define FS_STR(x) FS_STR2(x)
#define FS_LAUNCH_CHECK()                                                    \
  do {                                                                       \
    ctx->launches++;                                                         \
    cudaError_t e__ = cudaGetLastError();                                    \
    if (e__ != cudaSuccess) {                                                \
      ctx->err = std::string("launch (" __FILE__ ":" FS_STR(__LINE__) "): ") + cudaGetErrorString(e__); \
      return FS_E_CUDA;                                                      \
    }                                                                        \
  } while (0)

// A cooperative (grid-synchronising) launch in the form stream capture
// accepts: cudaLaunchKernelExC with the cooperative launch attribute.
static inline cudaError_t fs_coop_launch(const void *fn, int grid, int block, void **args, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, fn, args);
}

static inline int fs_grid(long n, int block = FS_BLOCK) {
  long g = (n + block - 1) / block;
  return (int)(g < 1 ? 1 : g);
}

// entry points shared between translation units
int fs_geometry_build(fs_ctx *ctx, const fs_mesh_in *mi);
int fs_gradient_dev(fs_ctx *ctx, int nfld, const int *vars, const double *const *phi,
                    const double *const *bphi, double *const *g, double *const *bg,
                    const int *method, const int *niter);
int fs_momentum_assemble(fs_ctx *ctx, int comp);
int fs_momentum_assemble_to(fs_ctx *ctx, int comp, double *ac, double *bc);
int fs_momentum_assemble3(fs_ctx *ctx);   // u, v, w into ac3/bc3 (multi-RHS form)
int fs_momentum_batched_solve(fs_ctx *ctx);
int fs_continuity_assemble(fs_ctx *ctx);
int fs_continuity_correct(fs_ctx *ctx);
int fs_residual_reduce(fs_ctx *ctx, int nf);   // CalculateResiduals partials -> resblk slot
int fs_linear_solve(fs_ctx *ctx, int nf, double *fi, double rrf, int itmax, int solver);
// k-epsilon and outlets (fs_turb.cu)
// Transient term of one equation (AssembleTheTransientTerm.for:52-330), by value in kernel arguments:
// two-level (three = 0): FluxCE = rho V / d, FluxCEold = -(rho V / d);
// three-level: FluxCE = f1 rho V, FluxCEold = s2 (f2 rho V), FluxCEoldold = f3 rho V.
struct FsTransient {
  int on, three;
  double rho, d, f1, f2, f3, s2;
  const double *old, *oldold;    // FS_NLEVELS blocks of N: u v w p k epsilon T
};
FsTransient fs_transient_args(const fs_ctx *ctx);
double fs_drhodt(const fs_ctx *ctx);                   // d rho/dt of the continuity residual
int fs_transient_create(fs_ctx *ctx);
void fs_transient_free(fs_ctx *ctx);
int fs_assemble_mdot(fs_ctx *ctx, const double *p_face);   // AssembleMdot alone
int fs_turb_create(fs_ctx *ctx);
void fs_turb_free(fs_ctx *ctx);
double *fs_turb_field(fs_ctx *ctx, int field, size_t *n);
void fs_turb_momentum_ptrs(fs_ctx *ctx, const double **mut, const double **bedif, const double **drk);
void fs_turb_rhok_ptrs(fs_ctx *ctx, const double **rhok, const double **drk);
void fs_turb_brhok_ptrs(fs_ctx *ctx, const double **brhok, const double **bdrk);
int fs_turb_wall_functions(fs_ctx *ctx);
int fs_turb_rhok_gradient(fs_ctx *ctx);
int fs_turb_effects(fs_ctx *ctx);
double *fs_turb_wall_distance(fs_ctx *ctx);            // WallDistance (N), nullptr when laminar
// temperature equation (fs_energy.cu)
int fs_energy_create(fs_ctx *ctx);
void fs_energy_free(fs_ctx *ctx);
double *fs_energy_field(fs_ctx *ctx, int field, size_t *n);
double *fs_energy_bgrad(fs_ctx *ctx);                   // BTempGrad (3B)
int fs_energy_solve(fs_ctx *ctx);
int fs_flow_in_out(fs_ctx *ctx);
int fs_mg_build(fs_ctx *ctx);
int fs_mg_free(fs_ctx *ctx);
void fs_ilu_free(fs_ctx *ctx);
int fs_mg_solve(fs_ctx *ctx, int nf, double rrf, int solver);
int fs_solver_stats_collect(fs_ctx *ctx);
int fs_coop_per_sm(fs_ctx *ctx, int occupancy);         // CTAs per SM for a cooperative launch (1)
int fs_coop_block(const fs_ctx *ctx);                   // threads per CTA of a cooperative launch
// batched AMG-BiCGSTAB p' solves of several contexts in one cooperative launch
// (ensembles): fs_pc_batch_form reports whether a context's p' solver can take
// part and in which kernel form; fs_pc_batch_create splits the co-resident
// CTAs among the contexts by weight; fs_pc_batch_launch launches the solves
// the contexts prepared with pc_defer set
struct fs_pc_batch;
int fs_linear_solve_finish(fs_ctx *ctx, int nf, double *fi);
// the multi-RHS momentum solves of several contexts in one cooperative launch
// (ensembles), as the p' solves above; fs_momentum_batched_finish moves a
// deferred solve's result back to cell order
struct fs_mom_batch;
int fs_momentum_batched_finish(fs_ctx *ctx);
int fs_mom_batch_create(fs_ctx **cs, int n, const double *weight, fs_mom_batch **out);
int fs_mom_batch_launch(fs_mom_batch *B, fs_ctx **cs, int n, cudaStream_t st);
void fs_mom_batch_free(fs_mom_batch *B);
// CTA offsets of n groups sharing `cap` co-resident CTAs in proportion to
// weight (at least one each; largest remainders, so the split is reproducible)
std::vector<int32_t> fs_cta_split(int cap, const double *weight, int n);
int fs_pc_batch_form(fs_ctx *ctx, int *form);
int fs_pc_batch_create(fs_ctx **cs, int n, const double *weight, fs_pc_batch **out);
int fs_pc_batch_launch(fs_pc_batch *B, fs_ctx **cs, int n, cudaStream_t st);
void fs_pc_batch_free(fs_pc_batch *B);
int fs_nn_before_pc(fs_ctx *ctx, const double **x0);   // features (+ guess) before the p' solve
int fs_nn_after_pc(fs_ctx *ctx);                        // snapshot capture, previous p'
void fs_nn_free(fs_ctx *ctx);
int32_t *fs_nn_counters(fs_ctx *ctx);                   // device [fallbacks, uses] or nullptr
void fs_nn_note_iters(fs_ctx *ctx, int pc_iters);       // iterations of the last p' solve (policy)   // after a stream sync: fold pending solver events

#ifdef __CUDACC__
// Row i of a slot-major ELL table (n rows, width w; unused slots hold index -1):
// acc (+ or -) coef_ij * x(k_ij) over the valid slots in ascending slot order,
// i.e. the summation order of the sequential slot loop, so results are
// bit-identical to it.  U slots per round: the index and coefficient loads of
// a round are issued before its gathers, so a row costs about two memory
// latencies per round rather than two per slot.
template <int U, bool SUB, class T, class XF>
__device__ __forceinline__ T ell_acc(T acc, long n, int w, const int32_t *__restrict__ idx,
                                     const T *__restrict__ coef, long i, XF &&xv) {
  for (int j0 = 0; j0 < w; j0 += U) {
    int k[U];
    T a[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int j = j0 + u;
      k[u] = j < w ? idx[(long)j * n + i] : -1;
      a[u] = j < w ? coef[(long)j * n + i] : (T)0;
    }
#pragma unroll
    for (int u = 0; u < U; u++)
      if (k[u] >= 0) acc = SUB ? acc - a[u] * xv(k[u]) : acc + a[u] * xv(k[u]);
  }
  return acc;
}

// the slots j = q, q+G, ... of row i (lane q of a G-lane group); a partial sum
template <int G, int U, class T, class XF>
__device__ __forceinline__ T ell_part(long n, int w, const int32_t *__restrict__ idx, const T *__restrict__ coef,
                                      long i, int q, XF &&xv) {
  T acc = (T)0;
  for (int j0 = q; j0 < w; j0 += U * G) {
    int k[U];
    T a[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int j = j0 + u * G;
      k[u] = j < w ? idx[(long)j * n + i] : -1;
      a[u] = j < w ? coef[(long)j * n + i] : (T)0;
    }
#pragma unroll
    for (int u = 0; u < U; u++)
      if (k[u] >= 0) acc = acc + a[u] * xv(k[u]);
  }
  return acc;
}
#endif

#ifdef __CUDACC__
// Rows i and i2 (i2 = i + stride, valid when h2) of the ELL product at once:
// the index and coefficient loads of both rows are issued before their
// gathers.  Inside the persistent cooperative kernels a grid-stride loop of
// one row per step runs well below the bandwidth a plain launch reaches; two
// independent rows per step restore the memory-level parallelism.  Per-row
// summation order is that of ell_acc.
template <int U, bool SUB, class T, class XF>
__device__ __forceinline__ void ell_acc2(T &acc1, T &acc2, long n, int w, const int32_t *__restrict__ idx,
                                         const T *__restrict__ coef, long i, long i2, bool h2, XF &&xv) {
  for (int j0 = 0; j0 < w; j0 += U) {
    int k1[U], k2[U];
    T a1[U], a2[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int j = j0 + u;
      const bool in = j < w, in2 = in && h2;
      k1[u] = in ? idx[(long)j * n + i] : -1;
      a1[u] = in ? coef[(long)j * n + i] : (T)0;
      k2[u] = in2 ? idx[(long)j * n + i2] : -1;
      a2[u] = in2 ? coef[(long)j * n + i2] : (T)0;
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (k1[u] >= 0) acc1 = SUB ? acc1 - a1[u] * xv(k1[u]) : acc1 + a1[u] * xv(k1[u]);
      if (k2[u] >= 0) acc2 = SUB ? acc2 - a2[u] * xv(k2[u]) : acc2 + a2[u] * xv(k2[u]);
    }
  }
}
#endif
