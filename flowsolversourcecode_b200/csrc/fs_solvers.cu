// fs_solvers.cu -- SolveEquation (AlgebraicSolvers/SolveAlegbraicEquations.for:4-180)
// on the GPU.
//
// Each solve is ONE persistent cooperative kernel (one or more CTAs per SM,
// grid-wide barriers between dependent steps), so an entire BiCGSTAB or
// Gauss-Seidel solve including its convergence test runs without a host
// round trip.  Dot products and norms are FP64 and deterministic: every CTA
// writes a partial, and after the barrier every CTA sums the same partials
// in the same fixed order, so all CTAs hold the same value.
//
// Matrix: ac (N), anb (W*N slot-major), neighbour table cn (W*N), i.e. the
// reference's Variables2 layout.  The product row i: ac_i x_i + sum_j anb_ij
// x_cn(i,j) in slot order is the CSR row order of matrixSolverOMP.f90:517-583.
#include "fs_internal.cuh"
#include <cooperative_groups.h>
#include <algorithm>
#include <array>
#include <cstring>

namespace cg = cooperative_groups;

// CTAs per SM the BiCGSTAB kernel is compiled for (register cap: the shared
// cooperative grid takes the smallest occupancy of the solver kernels)
#ifndef FS_KRYLOV_MINB
#define FS_KRYLOV_MINB 1
#endif

namespace {

struct SolveArgs {
  int N, W;
  const int32_t *ncf, *cn;
  const double *ac, *anb, *bc;
  double *x, *r, *r0, *p, *v, *s, *t, *dphi;
  double *part;        // 8 * grid partial slots
  const double *ires;  // IResiduals (ResorAbs of the system at dphi=0)
  double rrf, tol;
  int itmax;
  const int32_t *color_rows;
  const int32_t *color_ptr;  // device copy (ncolors+1)
  int ncolors;
  int32_t *iters;
  double *diag;        // [0]=final residual norm, [1]=normb
};

__device__ __forceinline__ double row_ax(const SolveArgs &a, int i, const double *x) {
  double t = 0.0;
  t = t + a.ac[i] * x[i];
  return ell_acc<8, false>(t, a.N, a.W, a.cn, a.anb, i, [&](int k) { return x[k]; });
}

// rows i and i2 = i + stride (when h2) at once (ell_acc2)
__device__ __forceinline__ void row_ax2(const SolveArgs &a, long i, long i2, bool h2, const double *x, double &t1,
                                        double &t2) {
  t1 = 0.0;
  t1 = t1 + a.ac[i] * x[i];
  t2 = 0.0;
  if (h2) t2 = t2 + a.ac[i2] * x[i2];
  ell_acc2<6, false>(t1, t2, a.N, a.W, a.cn, a.anb, i, i2, h2, [&](int k) { return x[k]; });
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// block sum of per-thread values, broadcast to every thread of the block
__device__ double block_sum_all(double v) {
  __shared__ double sh[33];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    double r = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.;
    r = warp_sum(r);
    if (lane == 0) sh[32] = r;
  }
  __syncthreads();
  double r = sh[32];
  __syncthreads();
  return r;
}

// grid-deterministic reduction of up to 2 values: write partials at slot `buf`,
// barrier, then every CTA sums all partials in the same order
__device__ void grid_sum2(cg::grid_group &grid, double *part, int buf, double a0, double a1,
                          double &o0, double &o1) {
  int G = gridDim.x;
  double b0 = block_sum_all(a0), b1 = block_sum_all(a1);
  if (threadIdx.x == 0) { part[(2 * buf) * G + blockIdx.x] = b0; part[(2 * buf + 1) * G + blockIdx.x] = b1; }
  grid.sync();
  double s0 = 0., s1 = 0.;
  for (int q = threadIdx.x; q < G; q += blockDim.x) { s0 += part[(2 * buf) * G + q]; s1 += part[(2 * buf + 1) * G + q]; }
  o0 = block_sum_all(s0);
  o1 = block_sum_all(s1);
}

// BICGSTAB_OMP (matrixSolverOMP.f90:306-386): unpreconditioned, x kept between
// calls (the reference's module vector x), stop when sqrt|r.r0| <= tol*|b|
// or after maxit-1 iterations.  Every row loop takes rows i and i + nth per
// step (ell_acc2); a thread's partial sums still run over its rows in
// ascending order.
__global__ void __launch_bounds__(FS_COOP_BLOCK, FS_KRYLOV_MINB) k_bicgstab(SolveArgs a) {
  cg::grid_group grid = cg::this_grid();
  const int N = a.N;
  const long tid0 = (long)blockIdx.x * blockDim.x + threadIdx.x, nth = (long)gridDim.x * blockDim.x;
  double l0 = 0., l1 = 0.;
  for (long i = tid0; i < N; i += 2 * nth) {
    const long i2 = i + nth;
    const bool h2 = i2 < N;
    double t1, t2;
    row_ax2(a, i, i2, h2, a.x, t1, t2);
    double r0 = a.bc[i] - t1;
    a.r0[i] = r0; a.r[i] = r0; a.p[i] = r0;
    l0 += r0 * r0;
    l1 += a.bc[i] * a.bc[i];
    if (h2) {
      double r2 = a.bc[i2] - t2;
      a.r0[i2] = r2; a.r[i2] = r2; a.p[i2] = r2;
      l0 += r2 * r2;
      l1 += a.bc[i2] * a.bc[i2];
    }
  }
  double rhoPrev, bb;
  grid_sum2(grid, a.part, 0, l0, l1, rhoPrev, bb);
  double resnorm = sqrt(fabs(rhoPrev)), normb = sqrt(bb);
  int k = 1;
  int buf = 1;
  while (k < a.itmax && resnorm > a.tol * normb) {
    k = k + 1;
    // v = A p ; dp0 = v.r0
    l0 = 0.;
    for (long i = tid0; i < N; i += 2 * nth) {
      const long i2 = i + nth;
      const bool h2 = i2 < N;
      double v1, v2;
      row_ax2(a, i, i2, h2, a.p, v1, v2);
      a.v[i] = v1; l0 += v1 * a.r0[i];
      if (h2) { a.v[i2] = v2; l0 += v2 * a.r0[i2]; }
    }
    double dp0, dum;
    grid_sum2(grid, a.part, buf, l0, 0., dp0, dum); buf ^= 3;
    double alpha = rhoPrev / dp0;
    for (long i = tid0; i < N; i += 2 * nth) {
      const long i2 = i + nth;
      const bool h2 = i2 < N;
      double r1 = a.r[i], v1 = a.v[i], r2 = h2 ? a.r[i2] : 0., v2 = h2 ? a.v[i2] : 0.;
      a.s[i] = r1 - alpha * v1;
      if (h2) a.s[i2] = r2 - alpha * v2;
    }
    grid.sync();
    // As = A s ; dp1 = As.s ; dp2 = As.As
    l0 = 0.; l1 = 0.;
    for (long i = tid0; i < N; i += 2 * nth) {
      const long i2 = i + nth;
      const bool h2 = i2 < N;
      double t1, t2;
      row_ax2(a, i, i2, h2, a.s, t1, t2);
      a.t[i] = t1; l0 += t1 * a.s[i]; l1 += t1 * t1;
      if (h2) { a.t[i2] = t2; l0 += t2 * a.s[i2]; l1 += t2 * t2; }
    }
    double dp1, dp2;
    grid_sum2(grid, a.part, buf, l0, l1, dp1, dp2); buf ^= 3;
    double omega = dp1 / dp2;
    l0 = 0.;
    for (long i = tid0; i < N; i += 2 * nth) {
      const long i2 = i + nth;
      const bool h2 = i2 < N;
      double x1 = a.x[i], p1 = a.p[i], s1 = a.s[i], t1 = a.t[i], q1 = a.r0[i];
      double x2 = 0., p2 = 0., s2 = 0., t2 = 0., q2 = 0.;
      if (h2) { x2 = a.x[i2]; p2 = a.p[i2]; s2 = a.s[i2]; t2 = a.t[i2]; q2 = a.r0[i2]; }
      a.x[i] = x1 + alpha * p1 + omega * s1;
      double ri = s1 - omega * t1;
      a.r[i] = ri;
      l0 += ri * q1;
      if (h2) {
        a.x[i2] = x2 + alpha * p2 + omega * s2;
        double rj = s2 - omega * t2;
        a.r[i2] = rj;
        l0 += rj * q2;
      }
    }
    double rho;
    grid_sum2(grid, a.part, buf, l0, 0., rho, dum); buf ^= 3;
    double beta = (rho / rhoPrev) * (alpha / omega);
    rhoPrev = rho;
    for (long i = tid0; i < N; i += 2 * nth) {
      const long i2 = i + nth;
      const bool h2 = i2 < N;
      double r1 = a.r[i], p1 = a.p[i], v1 = a.v[i];
      double r2 = 0., p2 = 0., v2 = 0.;
      if (h2) { r2 = a.r[i2]; p2 = a.p[i2]; v2 = a.v[i2]; }
      a.p[i] = r1 + beta * (p1 - omega * v1);
      if (h2) a.p[i2] = r2 + beta * (p2 - omega * v2);
    }
    resnorm = sqrt(fabs(rho));
    grid.sync();
  }
  for (long i = tid0; i < N; i += nth) a.dphi[i] = a.x[i];
  if (tid0 == 0) { *a.iters = k - 1; a.diag[0] = resnorm; a.diag[1] = normb; }
}

// SolveEquationsUsingSOR sweeps (SORMethod.for:20-60) in multicolour order:
// forward over colours 0..C-1, backward C-1..0, each colour an independent
// set, then CheckConvergence (CheckConvergenceRoutine.for:3) -- until
// sum|r| <= rrF * IResiduals or itmax sweeps (SolveAlegbraicEquations.for:108-117).
// The sweeps run on the colour-major copy: colour c occupies positions
// [color_ptr[c], color_ptr[c+1]) contiguously, so every pass streams its rows
struct SorPArgs {
  int N, W;
  const int32_t *ncf, *cn, *color_ptr;
  const double *ac, *anb, *bc;
  double *x;
  double *part;
  const double *ires;
  double rrf;
  int itmax, ncolors;
  int32_t *iters;
  double *diag;
};

__global__ void __launch_bounds__(FS_COOP_BLOCK, FS_KRYLOV_MINB) k_sor_colour(SorPArgs a) {
  cg::grid_group grid = cg::this_grid();
  const int N = a.N;
  const long tid0 = (long)blockIdx.x * blockDim.x + threadIdx.x, nth = (long)gridDim.x * blockDim.x;
  const int32_t *__restrict__ cn = a.cn;
  const double *__restrict__ anb = a.anb;
  double ires = *a.ires, fres = ires;
  int iter = 0, buf = 0;
  // a pass repeating the previous pass's colour (the backward pass's first
  // colour, the next sweep's first) would rewrite the same values -- rows of
  // one colour read only other colours -- and is skipped: results unchanged
  int last = -1;
  while (fres > a.rrf * ires && iter < a.itmax) {
    for (int pass = 0; pass < 2; pass++) {
      for (int cc = 0; cc < a.ncolors; cc++) {
        int c = pass == 0 ? cc : a.ncolors - 1 - cc;
        if (c == last) continue;
        last = c;
        int r0 = a.color_ptr[c], r1 = a.color_ptr[c + 1];
        // rows of one colour are independent: two per step (ell_acc2)
        for (long i = r0 + tid0; i < r1; i += 2 * nth) {
          const long i2 = i + nth;
          const bool h2 = i2 < r1;
          double l1 = a.bc[i], l2 = h2 ? a.bc[i2] : 0.;
          ell_acc2<6, true>(l1, l2, N, a.W, cn, anb, i, i2, h2, [&](int k) { return a.x[k]; });
          a.x[i] = l1 / a.ac[i];
          if (h2) a.x[i2] = l2 / a.ac[i2];
        }
        grid.sync();
      }
    }
    // sum of |residual|: the rows of the colour just solved satisfy their
    // equations up to rounding (solved from neighbours of other colours,
    // unchanged since), so only the other colours' rows are summed
    double l0 = 0., dum;
    const long lr0 = a.color_ptr[last], lr1 = a.color_ptr[last + 1];
    for (int part = 0; part < 2; part++) {
      const long q0 = part == 0 ? 0 : lr1, qe = part == 0 ? lr0 : N;
      for (long i = q0 + tid0; i < qe; i += 2 * nth) {
        const long i2 = i + nth;
        const bool h2 = i2 < qe;
        double q1 = a.bc[i] - a.ac[i] * a.x[i], q2 = h2 ? a.bc[i2] - a.ac[i2] * a.x[i2] : 0.;
        ell_acc2<6, true>(q1, q2, N, a.W, cn, anb, i, i2, h2, [&](int k) { return a.x[k]; });
        l0 += fabs(q1);
        if (h2) l0 += fabs(q2);
      }
    }
    grid_sum2(grid, a.part, buf, l0, 0., fres, dum); buf ^= 1;
    iter++;
  }
  if (tid0 == 0) { *a.iters = iter; a.diag[0] = fres; a.diag[1] = ires; }
}

// gather the assembled system into colour-major order; zero the start vector
__global__ void k_to_colour(int N, int W, const int32_t *__restrict__ rows, const int32_t *__restrict__ ncfP,
                            const double *__restrict__ ac, const double *__restrict__ bc,
                            const double *__restrict__ anb, double *acP, double *bcP, double *anbP, double *xP) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  int i = rows[q];
  acP[q] = ac[i]; bcP[q] = bc[i]; xP[q] = 0.;
  int nc = ncfP[q];
  for (int j = 0; j < nc; j++) anbP[(long)j * N + q] = anb[(long)j * N + i];
}

// dphi back to cell order and FiT = FiT + dphi (SolveAlegbraicEquations.for:180)
__global__ void k_from_colour(int N, const int32_t *__restrict__ pos, const double *__restrict__ xP, double *dphi) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) dphi[i] = xP[pos[i]];
}

// multi-RHS momentum: X, Y, Z systems share anb/cn; each keeps its own ac, bc
// and convergence test (SolveAlegbraicEquations.for:108-117 per component)
struct Sor3Args {
  int N, W;
  const int32_t *ncf, *cn, *color_ptr;
  const double *ac3, *anb, *bc3;
  double *x3;
  double *part;
  const double *ires3;   // ResorAbs of the three systems
  double rrf;
  int itmax, ncolors;
  int32_t *iters3;
};

// l_c -= anb_ij x_c[k_ij] (m for row i2) for the three components sharing
// anb, slots in ascending order, rows i and i2 (when h2) at once
__device__ __forceinline__ void sub3x2(long N, int W, const int32_t *__restrict__ cn, const double *__restrict__ anb,
                                       long i, long i2, bool h2, const double *x3, double *l, double *m) {
  for (int j0 = 0; j0 < W; j0 += 4) {
    int k[4], k2[4];
    double w[4], w2[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int j = j0 + u;
      const bool in = j < W, in2 = in && h2;
      k[u] = in ? cn[(long)j * N + i] : -1;
      w[u] = in ? anb[(long)j * N + i] : 0.;
      k2[u] = in2 ? cn[(long)j * N + i2] : -1;
      w2[u] = in2 ? anb[(long)j * N + i2] : 0.;
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      if (k[u] >= 0) {
        l[0] = l[0] - w[u] * x3[k[u]]; l[1] = l[1] - w[u] * x3[N + k[u]]; l[2] = l[2] - w[u] * x3[2 * N + k[u]];
      }
      if (k2[u] >= 0) {
        m[0] = m[0] - w2[u] * x3[k2[u]]; m[1] = m[1] - w2[u] * x3[N + k2[u]]; m[2] = m[2] - w2[u] * x3[2 * N + k2[u]];
      }
    }
  }
}

// the CTAs a multi-RHS SOR solve runs on: the whole cooperative grid, or one
// group of a batched launch (CTAs [c0, c0 + n) with a bounded barrier of their
// own in global memory: bar[0] arrivals, bar[1] generation, zero at launch; a
// timeout sets status[0] and later barriers stop waiting)
struct GridCtas {
  cg::grid_group g;
  __device__ GridCtas() : g(cg::this_grid()) {}
  __device__ __forceinline__ int cta() const { return (int)blockIdx.x; }
  __device__ __forceinline__ int ncta() const { return (int)gridDim.x; }
  __device__ __forceinline__ void sync() { g.sync(); }
};
#define FS_GROUP_SPIN_LIMIT (1L << 20)
struct GroupCtas {
  int c, n;
  unsigned *bar;
  int32_t *status;
  unsigned gen;
  __device__ __forceinline__ int cta() const { return c; }
  __device__ __forceinline__ int ncta() const { return n; }
  __device__ void sync() {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      if (atomicAdd(&bar[0], 1u) == (unsigned)n - 1) {
        atomicExch(&bar[0], 0u);
        __threadfence();
        atomicAdd(&bar[1], 1u);
      } else {
        const volatile unsigned *vg = bar + 1;
        const volatile int32_t *vs = status;
        long spins = 0;
        while (*vg == gen && *vs == 0) {
          if (++spins > FS_GROUP_SPIN_LIMIT) { atomicExch(status, 1); break; }
          __nanosleep(64);
        }
      }
      __threadfence();
    }
    gen++;
    __syncthreads();
  }
};

// grid_sum2 over the CTAs of C
template <class CT>
__device__ void ctas_sum2(CT &C, double *part, int buf, double a0, double a1, double &o0, double &o1) {
  const int G = C.ncta();
  double b0 = block_sum_all(a0), b1 = block_sum_all(a1);
  if (threadIdx.x == 0) { part[(2 * buf) * G + C.cta()] = b0; part[(2 * buf + 1) * G + C.cta()] = b1; }
  C.sync();
  double s0 = 0., s1 = 0.;
  for (int q = threadIdx.x; q < G; q += blockDim.x) { s0 += part[(2 * buf) * G + q]; s1 += part[(2 * buf + 1) * G + q]; }
  o0 = block_sum_all(s0);
  o1 = block_sum_all(s1);
}

template <class CT>
__device__ __forceinline__ void sor3_body(const Sor3Args &a, CT &C) {
  const int N = a.N;
  const long tid0 = (long)C.cta() * blockDim.x + threadIdx.x, nth = (long)C.ncta() * blockDim.x;
  const int32_t *__restrict__ cn = a.cn;
  const double *__restrict__ anb = a.anb;
  double ires[3], fres[3];
  int iters[3];
  for (int c = 0; c < 3; c++) { ires[c] = a.ires3[c]; fres[c] = ires[c]; iters[c] = 0; }
  int buf = 0;
  int last = -1;   // repeated colour passes are skipped, as in k_sor_colour
  for (;;) {
    bool act[3];
    bool any = false;
    for (int c = 0; c < 3; c++) { act[c] = fres[c] > a.rrf * ires[c] && iters[c] < a.itmax; any |= act[c]; }
    if (!any) break;
    for (int pass = 0; pass < 2; pass++) {
      for (int cc = 0; cc < a.ncolors; cc++) {
        int col = pass == 0 ? cc : a.ncolors - 1 - cc;
        if (col == last) continue;
        last = col;
        int r0 = a.color_ptr[col], r1 = a.color_ptr[col + 1];
        for (long i = r0 + tid0; i < r1; i += 2 * nth) {
          const long i2 = i + nth;
          const bool h2 = i2 < r1;
          double l[3] = {a.bc3[i], a.bc3[N + i], a.bc3[2L * N + i]};
          double m[3] = {0., 0., 0.};
          if (h2) { m[0] = a.bc3[i2]; m[1] = a.bc3[N + i2]; m[2] = a.bc3[2L * N + i2]; }
          sub3x2(N, a.W, cn, anb, i, i2, h2, a.x3, l, m);
#pragma unroll
          for (int c = 0; c < 3; c++) {
            if (act[c]) a.x3[c * (long)N + i] = l[c] / a.ac3[c * (long)N + i];
            if (act[c] && h2) a.x3[c * (long)N + i2] = m[c] / a.ac3[c * (long)N + i2];
          }
        }
        C.sync();
      }
    }
    // |residual| sums of the active components.  The rows of the colour just
    // solved satisfy their equations up to rounding (each was solved from
    // neighbours of other colours, unchanged since), so only the other
    // colours' rows are summed: half the pass on a two-colour mesh
    double s0 = 0., s1 = 0., s2 = 0.;
    const long lr0 = a.color_ptr[last], lr1 = a.color_ptr[last + 1];
    for (int part = 0; part < 2; part++) {
      const long q0 = part == 0 ? 0 : lr1, q1 = part == 0 ? lr0 : N;
      for (long i = q0 + tid0; i < q1; i += 2 * nth) {
        const long i2 = i + nth;
        const bool h2 = i2 < q1;
        double l[3], m[3] = {0., 0., 0.};
#pragma unroll
        for (int c = 0; c < 3; c++) {
          l[c] = a.bc3[c * (long)N + i] - a.ac3[c * (long)N + i] * a.x3[c * (long)N + i];
          if (h2) m[c] = a.bc3[c * (long)N + i2] - a.ac3[c * (long)N + i2] * a.x3[c * (long)N + i2];
        }
        sub3x2(N, a.W, cn, anb, i, i2, h2, a.x3, l, m);
        s0 += fabs(l[0]); s1 += fabs(l[1]); s2 += fabs(l[2]);
        if (h2) { s0 += fabs(m[0]); s1 += fabs(m[1]); s2 += fabs(m[2]); }
      }
    }
    double o0, o1, o2, d;
    ctas_sum2(C, a.part, buf, s0, s1, o0, o1);
    ctas_sum2(C, a.part, buf + 1, s2, 0., o2, d);
    buf = buf == 0 ? 2 : 0;
    double o[3] = {o0, o1, o2};
    for (int c = 0; c < 3; c++) if (act[c]) { fres[c] = o[c]; iters[c]++; }
  }
  if (tid0 == 0) for (int c = 0; c < 3; c++) a.iters3[c] = iters[c];
}

__global__ void __launch_bounds__(FS_COOP_BLOCK, FS_KRYLOV_MINB) k_sor3_colour(Sor3Args a) {
  GridCtas C;
  sor3_body(a, C);
}

// the multi-RHS SOR solves of n systems in one cooperative launch: CTAs
// [start[q], start[q+1]) solve system q (an ensemble's momentum solves); a
// system's barrier timeout is recorded in status[q][0]
__global__ void __launch_bounds__(FS_COOP_BLOCK, FS_KRYLOV_MINB)
    k_sor3_colour_batch(const Sor3Args *__restrict__ as, const int32_t *__restrict__ start, int n, unsigned *gbar,
                        int32_t *const *__restrict__ status) {
  __shared__ int sq;
  if (threadIdx.x == 0) {
    int q = 0;
    while (q + 1 < n && (int)blockIdx.x >= start[q + 1]) q++;
    sq = q;
  }
  __syncthreads();
  const int q = sq;
  GroupCtas C{(int)blockIdx.x - start[q], start[q + 1] - start[q], gbar + 2 * q, status[q], 0u};
  const Sor3Args a = as[q];
  sor3_body(a, C);
}

__global__ void k_to_colour3(int N, const int32_t *__restrict__ rows, const int32_t *__restrict__ ncfP,
                             const double *__restrict__ ac3, const double *__restrict__ bc3,
                             const double *__restrict__ anb, double *ac3P, double *bc3P, double *anbP, double *x3P) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  int i = rows[q];
  for (int c = 0; c < 3; c++) {
    ac3P[(long)c * N + q] = ac3[(long)c * N + i];
    bc3P[(long)c * N + q] = bc3[(long)c * N + i];
    x3P[(long)c * N + q] = 0.;
  }
  int nc = ncfP[q];
  for (int j = 0; j < nc; j++) anbP[(long)j * N + q] = anb[(long)j * N + i];
}

__global__ void k_from_colour3(int N, const int32_t *__restrict__ pos, const double *__restrict__ x3P,
                               double *u, double *v, double *w) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int q = pos[i];
  u[i] = u[i] + x3P[q];
  v[i] = v[i] + x3P[N + q];
  w[i] = w[i] + x3P[2L * N + q];
}

__global__ void k_axpy_field(int N, double *fi, const double *dphi) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) fi[i] = fi[i] + dphi[i];
}

}  // namespace

// one grid size for every cooperative solver kernel of a context: the smallest
// co-resident CTA count of the three, at most 4 per SM

// GMRES_RESTARTED_OMP_RETURNR (matrixSolverOMP.f90:48-304) with the caller's
// GMRES_ninner = 20, GMRES_tol = 1e-9 (:4-6, :604), as one cooperative kernel:
// the system normalised by |b|; restart lengths mm = 5, 10, 15, 20, each round
// from x = 0 (resetFlag is never cleared, :81,120); Arnoldi with modified
// Gram-Schmidt (one grid reduction per projection) and Givens rotations; the
// best iterate kept; the restart length reduced by 5 (above 10) or 1 when a
// cycle gains less than 10 % or loses; a round with m = 1 ends when a cycle
// gains less than 1 % or after 100 cycles; the next round only if this one
// improved the best residual.  Every CTA keeps the Hessenberg matrix, the
// rotations and the least-squares solution in shared memory, updated by its
// thread 0 from the same grid-deterministic sums, so all CTAs take the same
// branches.  A zero right-hand side gives x = 0 (the reference divides by
// |b| = 0).  As the reference's module vector x, the result also stays in x.
#define FS_GM_M 20
#define FS_GM_CYCLES 20000   // bound on cycles per round (the reference's loop always ends; this only bounds a kernel)
struct GmresArgs {
  int N, W;
  const int32_t *cn;
  const double *ac, *anb, *bc;
  double *V, *w, *x1, *xOpt, *rOpt, *xG, *rG, *bn, *x, *r, *dphi;
  double *part;
  int32_t *iters;
  double *diag;
};

__device__ __forceinline__ void gm_ax2(const GmresArgs &a, long i, long i2, bool h2, const double *x, double &t1,
                                       double &t2) {
  t1 = 0.0;
  t1 = t1 + a.ac[i] * x[i];
  t2 = 0.0;
  if (h2) t2 = t2 + a.ac[i2] * x[i2];
  ell_acc2<6, false>(t1, t2, a.N, a.W, a.cn, a.anb, i, i2, h2, [&](int k) { return x[k]; });
}

__global__ void __launch_bounds__(FS_COOP_BLOCK, FS_KRYLOV_MINB) k_gmres(GmresArgs a) {
  cg::grid_group grid = cg::this_grid();
  const int N = a.N;
  const long tid0 = (long)blockIdx.x * blockDim.x + threadIdx.x, nth = (long)gridDim.x * blockDim.x;
  __shared__ double H[FS_GM_M + 1][FS_GM_M], g[FS_GM_M + 1], c[FS_GM_M], s[FS_GM_M], y[FS_GM_M];
  const double res = 1.0e-9, normb = 1.0;
  int buf = 1;
  double l0 = 0., dum;
  for (long i = tid0; i < N; i += nth) l0 += a.bc[i] * a.bc[i];
  double bb;
  grid_sum2(grid, a.part, 0, l0, 0., bb, dum);
  const double normb0 = sqrt(bb);
  if (normb0 == 0.) {
    for (long i = tid0; i < N; i += nth) { a.x[i] = 0.; a.dphi[i] = 0.; }
    if (tid0 == 0) { *a.iters = 0; a.diag[0] = 0.; a.diag[1] = 0.; }
    return;
  }
  for (long i = tid0; i < N; i += nth) a.bn[i] = a.bc[i] / normb0;
  int total = 0, mm = 5;
  double normminG = 1.0e30;
  while (mm <= FS_GM_M) {
    double normmin = 1.0e30;
    int mcur = mm, iter = 0, leave = 0, cycles = 0;
    l0 = 0.;
    for (long i = tid0; i < N; i += nth) { a.x[i] = 0.; const double ri = a.bn[i]; a.r[i] = ri; l0 += ri * ri; }
    double rr;
    grid_sum2(grid, a.part, buf, l0, 0., rr, dum); buf ^= 3;
    double normr = sqrt(rr), normrPrev = normr;
    while (normmin > res * normb && leave == 0 && cycles < FS_GM_CYCLES) {
      cycles++;
      iter++;
      int mloc = mcur;
      for (long i = tid0; i < N; i += nth) a.V[i] = a.r[i] / normr;
      if (threadIdx.x == 0) {
        for (int p = 0; p <= FS_GM_M; p++) { g[p] = 0.; for (int q = 0; q < FS_GM_M; q++) H[p][q] = 0.; }
        g[0] = normr;
      }
      __syncthreads();
      for (int j = 0; j < mloc; j++) {
        total++;
        const double *vj = a.V + (size_t)j * N;
        grid.sync();   // v_j complete before its neighbours are gathered
        for (long i = tid0; i < N; i += 2 * nth) {
          const long i2 = i + nth;
          const bool h2 = i2 < N;
          double t1, t2;
          gm_ax2(a, i, i2, h2, vj, t1, t2);
          a.w[i] = t1;
          if (h2) a.w[i2] = t2;
        }
        for (int i = 0; i <= j; i++) {
          const double *vi = a.V + (size_t)i * N;
          l0 = 0.;
          for (long q = tid0; q < N; q += nth) l0 += a.w[q] * vi[q];
          double h;
          grid_sum2(grid, a.part, buf, l0, 0., h, dum); buf ^= 3;
          for (long q = tid0; q < N; q += nth) a.w[q] = a.w[q] - h * vi[q];
          if (threadIdx.x == 0) H[i][j] = h;
        }
        l0 = 0.;
        for (long q = tid0; q < N; q += nth) l0 += a.w[q] * a.w[q];
        double ww;
        grid_sum2(grid, a.part, buf, l0, 0., ww, dum); buf ^= 3;
        const double hn = sqrt(ww);
        if (threadIdx.x == 0) H[j + 1][j] = hn;
        if (hn == 0.) { mloc = j + 1; __syncthreads(); break; }
        double *vn = a.V + (size_t)(j + 1) * N;
        for (long q = tid0; q < N; q += nth) vn[q] = a.w[q] / hn;
        if (threadIdx.x == 0) {
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
        __syncthreads();
      }
      mcur = mloc;
      if (threadIdx.x == 0) {
        y[mcur - 1] = g[mcur - 1] / H[mcur - 1][mcur - 1];
        for (int j = mcur - 2; j >= 0; j--) {
          double dp = 0.;
          for (int q = j + 1; q < mcur; q++) dp += H[j][q] * y[q];
          y[j] = (g[j] - dp) / H[j][j];
        }
      }
      __syncthreads();
      for (long i = tid0; i < N; i += nth) {
        double t = 0.;
        for (int q = 0; q < mcur; q++) t += a.V[(size_t)q * N + i] * y[q];
        a.x1[i] = a.x[i] + t;
      }
      grid.sync();   // x1 complete before its neighbours are gathered
      l0 = 0.;
      for (long i = tid0; i < N; i += 2 * nth) {
        const long i2 = i + nth;
        const bool h2 = i2 < N;
        double t1, t2;
        gm_ax2(a, i, i2, h2, a.x1, t1, t2);
        const double r1 = a.bn[i] - t1;
        a.r[i] = r1;
        l0 += r1 * r1;
        if (h2) { const double r2 = a.bn[i2] - t2; a.r[i2] = r2; l0 += r2 * r2; }
      }
      grid_sum2(grid, a.part, buf, l0, 0., rr, dum); buf ^= 3;
      normr = sqrt(rr);
      if ((normr - normrPrev) / normrPrev > -0.01 && mcur == 1) leave = 1;
      if (mcur == 1 && iter > 100) leave = 1;
      const bool best = normr < normmin, step = normr < normrPrev;
      if (best) normmin = normr;
      for (long i = tid0; i < N; i += nth) {
        if (best) { a.xOpt[i] = a.x1[i]; a.rOpt[i] = a.r[i]; }
        if (step) a.x[i] = a.x1[i];
        else { a.x[i] = a.xOpt[i]; a.r[i] = a.rOpt[i]; }
      }
      if ((fabs((normr - normrPrev) / normr) < 0.1 || normr > normrPrev) && mcur > 1) {
        mcur = mcur > 10 ? mcur - 5 : mcur - 1;
        iter = 0;
      }
      normrPrev = normr;
    }
    if (normmin < normminG) {
      normminG = normmin;
      for (long i = tid0; i < N; i += nth) { a.xG[i] = a.xOpt[i]; a.rG[i] = a.rOpt[i]; }
      mm += 5;
    } else {
      mm = FS_GM_M + 5;
    }
    if (normminG <= res) mm = FS_GM_M + 5;
  }
  for (long i = tid0; i < N; i += nth) { const double xi = a.xG[i] * normb0; a.x[i] = xi; a.dphi[i] = xi; }
  if (tid0 == 0) { *a.iters = total; a.diag[0] = normminG * normb0; a.diag[1] = normb0; }
}

struct IluArgs;
__global__ void k_ilu(IluArgs a);
struct PbcgArgs;
__global__ void k_pbcg(PbcgArgs a);

static int coop_grid_size(fs_ctx *ctx) {
  if (ctx->coop_grid > 0) return FS_OK;
  int a = 0, b = 0, c = 0;
  FS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, (void *)k_bicgstab, FS_COOP_BLOCK, 0));
  b = a;
  FS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, (void *)k_sor_colour, FS_COOP_BLOCK, 0));
  int d = 0, e = 0;
  FS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d, (void *)k_sor3_colour, FS_COOP_BLOCK, 0));
  FS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&e, (void *)k_gmres, FS_COOP_BLOCK, 0));
  FS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (void *)k_ilu, FS_COOP_BLOCK, 0));
  int f = 0;
  FS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&f, (void *)k_pbcg, FS_COOP_BLOCK, 0));
  int per_sm = std::min(std::min(std::min(a, d), std::min(b, c)), std::min(e, f));
  if (per_sm < 1) { ctx->err = "cooperative kernel does not fit on an SM"; return FS_E_CUDA; }
  ctx->coop_grid = ctx->num_sms * fs_coop_per_sm(ctx, per_sm);
  return FS_OK;
}

// Cooperative launches put one CTA on every SM: a grid barrier costs about
// one arrival per CTA, and at 128^3 one CTA of 1024 threads per SM ran the
// AMG Krylov solve 5-6 % faster than four CTAs of 256 (same threads, same
// registers).  The launch shape (fs_set_launch_shape, 1-4) sets the threads
// per CTA, 256 per unit: small ensemble cases run faster with fewer.
int fs_coop_per_sm(fs_ctx *ctx, int occupancy) {
  (void)ctx;
  return occupancy >= 1 ? 1 : 0;
}
int fs_coop_block(const fs_ctx *ctx) {
  const int k = ctx->coop_per_sm > 0 ? ctx->coop_per_sm : FS_COOP_BLOCK / 256;
  return 256 * std::max(1, std::min(k, FS_COOP_BLOCK / 256));
}

extern "C" int fs_set_launch_shape(fs_ctx *ctx, int shape) {
  if (!ctx || shape < 0 || shape > FS_COOP_BLOCK / 256) return FS_E_ARG;
  ctx->coop_per_sm = shape;
  ctx->coop_grid = 0;   // recomputed at the next solve
  return FS_OK;
}

static int coop_launch(fs_ctx *ctx, void *fn, SolveArgs &a) {
  int rc = coop_grid_size(ctx);
  if (rc) return rc;
  int G = ctx->coop_grid;
  const int T = fs_coop_block(ctx);
  long need = (ctx->N + T - 1) / T;
  if (need < G) G = (int)(need < 1 ? 1 : need);
  void *args[] = {&a};
  FS_CK(fs_coop_launch(fn, G, T, args, ctx->st));
  FS_LAUNCH_CHECK();
  return FS_OK;
}

// ======================================================================
// 'ilu' (SolveAlegbraicEquations.for:122-133): ILUFactorization once
// (FactorizeUsingILU.for:4-75), then SolveEquationsUsingILU sweeps
// (ILUMethod.for:4-170) and CheckConvergence until sum|r| <= rrF*IResiduals
// or itmax.  The factorisation and both substitutions are sequential in
// element order; here each runs level by level (a row's level is one more
// than that of the rows it waits for), one grid barrier per level, and every
// row applies its terms in the order the sequential loops apply them, so the
// factor and the sweeps are those of the element-order loops bit for bit.
//   lower list of row j: entries (i, sj, si) for every slot si of an earlier
//     neighbour i that points to j, sorted by (i, si); sj is the first slot
//     of j pointing to i (the reference's search loops)
//   forward levels: over the lower lists; backward levels: over the later
//     neighbours in the slot table
struct fs_ilu {
  int nlf = 0, nlb = 0;
  int32_t *lo_ptr = nullptr, *lo_i = nullptr, *lo_sj = nullptr, *lo_si = nullptr;
  int32_t *fl_ptr = nullptr, *fl_rows = nullptr, *bl_ptr = nullptr, *bl_rows = nullptr;
  double *dc = nullptr, *rc = nullptr;
  // 'pbcg': the transpose lists, every (row i, slot si) whose neighbour is j, sorted by (i, si)
  int32_t *tr_ptr = nullptr, *tr_i = nullptr, *tr_si = nullptr;
};

// ILUFactorization: dc = 1/(ac - sum a_ji dc_i a_ij) level by level; element
// N-2 (the reference's NumberOfElements-1) updates none of its later neighbours
__device__ void ilu_factor_levels(cg::grid_group &grid, int N, int nlf, const int32_t *fl_ptr, const int32_t *fl_rows,
                                  const int32_t *lo_ptr, const int32_t *lo_i, const int32_t *lo_sj,
                                  const int32_t *lo_si, const double *ac, const double *__restrict__ anb, double *dc,
                                  long tid0, long nth) {
  for (int L = 0; L < nlf; L++) {
    for (long q = fl_ptr[L] + tid0; q < fl_ptr[L + 1]; q += nth) {
      const int j = fl_rows[q];
      double d = ac[j];
      for (int e = lo_ptr[j]; e < lo_ptr[j + 1]; e++) {
        const int i = lo_i[e];
        if (i == N - 2) continue;
        d = d - anb[(long)lo_sj[e] * N + j] * dc[i] * anb[(long)lo_si[e] * N + i];
      }
      dc[j] = 1.0 / d;
    }
    grid.sync();
  }
}

struct IluArgs {
  int N, W, nlf, nlb, itmax;
  const int32_t *ncf, *cn, *lo_ptr, *lo_i, *lo_sj, *lo_si, *fl_ptr, *fl_rows, *bl_ptr, *bl_rows;
  const double *ac, *anb, *bc;
  double *x, *dc, *rc, *part;
  const double *ires;
  double rrf;
  int32_t *iters;
  double *diag;
};

__global__ void __launch_bounds__(FS_COOP_BLOCK, FS_KRYLOV_MINB) k_ilu(IluArgs a) {
  cg::grid_group grid = cg::this_grid();
  const int N = a.N;
  const long tid0 = (long)blockIdx.x * blockDim.x + threadIdx.x, nth = (long)gridDim.x * blockDim.x;
  const int32_t *__restrict__ cn = a.cn;
  const double *__restrict__ anb = a.anb;
  ilu_factor_levels(grid, N, a.nlf, a.fl_ptr, a.fl_rows, a.lo_ptr, a.lo_i, a.lo_sj, a.lo_si, a.ac, anb, a.dc, tid0, nth);
  double ires = *a.ires, fres = ires;
  int iter = 0, buf = 0;
  while (fres > a.rrf * ires && iter < a.itmax) {
    // residual (ILUMethod.for:20-40)
    for (long i = tid0; i < N; i += nth) {
      double res = -a.ac[i] * a.x[i] + a.bc[i];
      for (int j = 0; j < a.ncf[i]; j++) {
        const int k = cn[(long)j * N + i];
        if (k >= 0) res = res - anb[(long)j * N + i] * a.x[k];
      }
      a.rc[i] = res;
    }
    grid.sync();
    // forward substitution (:44-100): row j takes dc_i rc_i of each earlier neighbour
    for (int L = 0; L < a.nlf; L++) {
      for (long q = a.fl_ptr[L] + tid0; q < a.fl_ptr[L + 1]; q += nth) {
        const int j = a.fl_rows[q];
        double r = a.rc[j];
        for (int e = a.lo_ptr[j]; e < a.lo_ptr[j + 1]; e++) {
          const int i = a.lo_i[e];
          const double product1 = a.dc[i] * a.rc[i];
          r = r - anb[(long)a.lo_sj[e] * N + j] * product1;
        }
        a.rc[j] = r;
      }
      grid.sync();
    }
    // backward substitution (:104-150): later neighbours in slot order, then dphi += dc rc
    for (int L = 0; L < a.nlb; L++) {
      for (long q = a.bl_ptr[L] + tid0; q < a.bl_ptr[L + 1]; q += nth) {
        const int i = a.bl_rows[q];
        double r = a.rc[i];
        if (i < N - 1)
          for (int j2 = 0; j2 < a.ncf[i]; j2++) {
            const int j = cn[(long)j2 * N + i];
            if (j > i) r = r - anb[(long)j2 * N + i] * a.rc[j];
          }
        const double product1 = a.dc[i] * r;
        a.rc[i] = product1;
        a.x[i] = a.x[i] + product1;
      }
      grid.sync();
    }
    // CheckConvergence
    double l0 = 0., dum;
    for (long i = tid0; i < N; i += 2 * nth) {
      const long i2 = i + nth;
      const bool h2 = i2 < N;
      double q1 = a.bc[i] - a.ac[i] * a.x[i], q2 = h2 ? a.bc[i2] - a.ac[i2] * a.x[i2] : 0.;
      ell_acc2<6, true>(q1, q2, N, a.W, cn, anb, i, i2, h2, [&](int k) { return a.x[k]; });
      l0 += fabs(q1);
      if (h2) l0 += fabs(q2);
    }
    grid_sum2(grid, a.part, buf, l0, 0., fres, dum); buf ^= 1;
    iter++;
  }
  if (tid0 == 0) { *a.iters = iter; a.diag[0] = fres; a.diag[1] = ires; }
}

// 'pbcg' (SolveAlegbraicEquations.for:138-152): sprsin, ILUFactorization, then
// SolveEquationsUsingPBCG (PBCGMethod.for:96-180) and CheckConvergence until
// sum|r| <= rrF*IResiduals or itmax.  Numerical Recipes' biconjugate gradient
// in its minimum-residual form (rr = A r), both systems preconditioned by the
// D-ILU diagonal; A x sums each row's diagonal then its slots in order
// (dsprsax), A^T x each column's diagonal then the rows that reference it in
// element order (dsprstx, through the transpose lists).  bkden carries from
// one iteration to the next.  Per iteration: p, pp update | A p, A^T pp and
// the denominator | x, r, rr update | residual sum and the next numerator.
struct PbcgArgs {
  int N, W, nlf, itmax;
  const int32_t *ncf, *cn, *lo_ptr, *lo_i, *lo_sj, *lo_si, *fl_ptr, *fl_rows, *tr_ptr, *tr_i, *tr_si;
  const double *ac, *anb, *bc;
  double *x, *dc, *r, *rr, *p, *pp, *z, *zz, *part;
  const double *ires;
  double rrf;
  int32_t *iters;
  double *diag;
};

__device__ __forceinline__ double pbcg_ax(const PbcgArgs &a, long i, const double *x) {
  double t = a.ac[i] * x[i];
  return ell_acc<8, false>(t, a.N, a.W, a.cn, a.anb, i, [&](int k) { return x[k]; });
}

__device__ __forceinline__ double pbcg_atx(const PbcgArgs &a, long j, const double *x) {
  double t = a.ac[j] * x[j];
  for (int e = a.tr_ptr[j]; e < a.tr_ptr[j + 1]; e++) {
    const int i = a.tr_i[e];
    t = t + a.anb[(long)a.tr_si[e] * a.N + i] * x[i];
  }
  return t;
}

__global__ void __launch_bounds__(FS_COOP_BLOCK, FS_KRYLOV_MINB) k_pbcg(PbcgArgs a) {
  cg::grid_group grid = cg::this_grid();
  const int N = a.N;
  const long tid0 = (long)blockIdx.x * blockDim.x + threadIdx.x, nth = (long)gridDim.x * blockDim.x;
  ilu_factor_levels(grid, N, a.nlf, a.fl_ptr, a.fl_rows, a.lo_ptr, a.lo_i, a.lo_sj, a.lo_si, a.ac, a.anb, a.dc,
                    tid0, nth);
  // iter 0: r = bc - A x, then the minimum-residual shadow rr = A r
  for (long i = tid0; i < N; i += nth) {
    const double ri = a.bc[i] - pbcg_ax(a, i, a.x);
    a.r[i] = ri;
  }
  grid.sync();
  double l0 = 0., l1 = 0., dum;
  for (long i = tid0; i < N; i += nth) {
    const double rri = pbcg_ax(a, i, a.r);
    a.rr[i] = rri;
    const double zi = a.r[i] * a.dc[i], zzi = rri * a.dc[i];
    a.z[i] = zi; a.zz[i] = zzi;
    l0 += zi * rri;
  }
  int buf = 0;
  double bknum, bkden = 0.;
  grid_sum2(grid, a.part, buf, l0, 0., bknum, dum); buf ^= 1;
  const double ires = *a.ires;
  double fres = ires;
  int iter = 0;
  while (fres > a.rrf * ires && iter < a.itmax) {
    const double bk = bknum / (bkden + 1.e-10);
    for (long i = tid0; i < N; i += nth) {
      if (iter == 0) { a.p[i] = a.z[i]; a.pp[i] = a.zz[i]; }
      else { a.p[i] = bk * a.p[i] + a.z[i]; a.pp[i] = bk * a.pp[i] + a.zz[i]; }
    }
    bkden = bknum;
    grid.sync();
    l0 = 0.;
    for (long i = tid0; i < N; i += nth) {
      const double zi = pbcg_ax(a, i, a.p), zzi = pbcg_atx(a, i, a.pp);
      a.z[i] = zi; a.zz[i] = zzi;
      l0 += zi * a.pp[i];
    }
    double akden;
    grid_sum2(grid, a.part, buf, l0, 0., akden, dum); buf ^= 1;
    const double ak = bknum / (akden + 1.e-10);
    for (long i = tid0; i < N; i += nth) {
      a.x[i] = a.x[i] + ak * a.p[i];
      a.r[i] = a.r[i] - ak * a.z[i];
      a.rr[i] = a.rr[i] - ak * a.zz[i];
    }
    grid.sync();
    // CheckConvergence, and the next call's z = dc r, zz = dc rr, bknum = z.rr
    l0 = 0.; l1 = 0.;
    for (long i = tid0; i < N; i += nth) {
      double q = a.bc[i] - a.ac[i] * a.x[i];
      q = ell_acc<8, true>(q, N, a.W, a.cn, a.anb, i, [&](int k) { return a.x[k]; });
      l0 += fabs(q);
      const double zi = a.r[i] * a.dc[i], zzi = a.rr[i] * a.dc[i];
      a.z[i] = zi; a.zz[i] = zzi;
      l1 += zi * a.rr[i];
    }
    grid_sum2(grid, a.part, buf, l0, l1, fres, bknum); buf ^= 1;
    iter++;
  }
  if (tid0 == 0) { *a.iters = iter; a.diag[0] = fres; a.diag[1] = ires; }
}

// the transpose lists of 'pbcg', built once per context after the ILU levels
static int pbcg_build(fs_ctx *ctx) {
  fs_ilu *I = ctx->ilu;
  if (I->tr_ptr) return FS_OK;
  const int N = ctx->N;
  const std::vector<int32_t> &ncf = ctx->h_ncf, &cn = ctx->h_cn;
  std::vector<int32_t> ptr(N + 1, 0);
  for (int i = 0; i < N; i++)
    for (int si = 0; si < ncf[i]; si++) {
      const int j = cn[(size_t)si * N + i];
      if (j >= 0 && j != i) ptr[j + 1]++;
    }
  for (int j = 0; j < N; j++) ptr[j + 1] += ptr[j];
  std::vector<int32_t> ti(ptr[N]), ts(ptr[N]), pos(ptr.begin(), ptr.end() - 1);
  for (int i = 0; i < N; i++)   // rows in element order, slots in order: (i, si) sorted per column
    for (int si = 0; si < ncf[i]; si++) {
      const int j = cn[(size_t)si * N + i];
      if (j >= 0 && j != i) { ti[pos[j]] = i; ts[pos[j]] = si; pos[j]++; }
    }
  auto up = [&](int32_t **d, const std::vector<int32_t> &h) -> int {
    FS_CK(cudaMalloc((void **)d, std::max<size_t>(h.size(), 1) * sizeof(int32_t)));
    if (!h.empty()) FS_CK(cudaMemcpy(*d, h.data(), h.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    return FS_OK;
  };
  int rc;
  if ((rc = up(&I->tr_ptr, ptr)) || (rc = up(&I->tr_i, ti)) || (rc = up(&I->tr_si, ts))) return rc;
  return FS_OK;
}

static int ilu_build(fs_ctx *ctx) {
  if (ctx->ilu) return FS_OK;
  const int N = ctx->N, W = ctx->W;
  const std::vector<int32_t> &ncf = ctx->h_ncf, &cn = ctx->h_cn;
  std::vector<std::vector<std::array<int32_t, 3>>> lo(N);
  for (int i = 0; i < N; i++)
    for (int si = 0; si < ncf[i]; si++) {
      const int j = cn[(size_t)si * N + i];
      if (j > i && j < N) {
        int sj = -1;
        for (int q = 0; q < ncf[j]; q++) if (cn[(size_t)q * N + j] == i) { sj = q; break; }
        if (sj < 0) { ctx->err = "ilu: a neighbour does not list the cell back"; return FS_E_MESH; }
        lo[j].push_back({i, sj, si});   // visited in (i, si) order already
      }
    }
  std::vector<int32_t> lo_ptr(N + 1, 0), lo_i, lo_sj, lo_si, lf(N, 0), lb(N, 0);
  int nlf = 0, nlb = 0;
  for (int j = 0; j < N; j++) {
    lo_ptr[j + 1] = lo_ptr[j] + (int)lo[j].size();
    int L = 0;
    for (auto &e : lo[j]) { lo_i.push_back(e[0]); lo_sj.push_back(e[1]); lo_si.push_back(e[2]); L = std::max(L, lf[e[0]] + 1); }
    lf[j] = L; nlf = std::max(nlf, L + 1);
  }
  for (int i = N - 1; i >= 0; i--) {
    int L = 0;
    for (int q = 0; q < ncf[i]; q++) { const int j = cn[(size_t)q * N + i]; if (j > i) L = std::max(L, lb[j] + 1); }
    lb[i] = L; nlb = std::max(nlb, L + 1);
  }
  auto by_level = [&](const std::vector<int32_t> &lev, int nl, std::vector<int32_t> &ptr, std::vector<int32_t> &rows) {
    ptr.assign(nl + 1, 0);
    for (int r = 0; r < N; r++) ptr[lev[r] + 1]++;
    for (int L = 0; L < nl; L++) ptr[L + 1] += ptr[L];
    std::vector<int32_t> pos(ptr.begin(), ptr.end() - 1);
    rows.assign(N, 0);
    for (int r = 0; r < N; r++) rows[pos[lev[r]]++] = r;
  };
  std::vector<int32_t> fl_ptr, fl_rows, bl_ptr, bl_rows;
  by_level(lf, nlf, fl_ptr, fl_rows);
  by_level(lb, nlb, bl_ptr, bl_rows);
  fs_ilu *I = new fs_ilu();
  ctx->ilu = I;
  I->nlf = nlf; I->nlb = nlb;
  auto up = [&](int32_t **d, const std::vector<int32_t> &h) -> int {
    FS_CK(cudaMalloc((void **)d, std::max<size_t>(h.size(), 1) * sizeof(int32_t)));
    if (!h.empty()) FS_CK(cudaMemcpy(*d, h.data(), h.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    return FS_OK;
  };
  int rc;
  if ((rc = up(&I->lo_ptr, lo_ptr)) || (rc = up(&I->lo_i, lo_i)) || (rc = up(&I->lo_sj, lo_sj)) ||
      (rc = up(&I->lo_si, lo_si)) || (rc = up(&I->fl_ptr, fl_ptr)) || (rc = up(&I->fl_rows, fl_rows)) ||
      (rc = up(&I->bl_ptr, bl_ptr)) || (rc = up(&I->bl_rows, bl_rows)))
    return rc;
  FS_CK(cudaMalloc(&I->dc, sizeof(double) * N));
  FS_CK(cudaMalloc(&I->rc, sizeof(double) * N));
  (void)W;
  return FS_OK;
}

void fs_ilu_free(fs_ctx *ctx) {
  fs_ilu *I = ctx->ilu;
  if (!I) return;
  void *p[] = {I->lo_ptr, I->lo_i, I->lo_sj, I->lo_si, I->fl_ptr, I->fl_rows, I->bl_ptr, I->bl_rows, I->dc, I->rc,
               I->tr_ptr, I->tr_i, I->tr_si};
  for (void *x : p) if (x) cudaFree(x);
  delete I;
  ctx->ilu = nullptr;
}

static SolveArgs solve_args(fs_ctx *ctx, int nf, double rrf, int itmax) {
  SolveArgs a{};
  a.N = ctx->N; a.W = ctx->W; a.ncf = ctx->ncf; a.cn = ctx->cn;
  a.ac = ctx->ac; a.anb = ctx->anb; a.bc = ctx->bc;
  a.x = ctx->kx; a.r = ctx->kr; a.r0 = ctx->kr0; a.p = ctx->kp; a.v = ctx->kv; a.s = ctx->ks; a.t = ctx->kt;
  a.dphi = ctx->dphi;
  a.part = ctx->red;
  a.ires = ctx->resblk + RB_ABS + (nf - 1);
  a.rrf = rrf; a.itmax = itmax; a.tol = ctx->cfg.krylov_tol;
  a.color_rows = ctx->color_rows;
  a.ncolors = ctx->ncolors;
  a.iters = ctx->d_iters + (nf - 1);
  a.diag = ctx->resblk + RB_DIAG;
  return a;
}

int fs_linear_solve(fs_ctx *ctx, int nf, double *fi, double rrf, int itmax, int solver) {
  const int N = ctx->N;
  FS_CK(cudaMemsetAsync(ctx->dphi, 0, sizeof(double) * N, ctx->st));
  SolveArgs a = solve_args(ctx, nf, rrf, itmax);
  int rc = FS_OK;
  if (ctx->s_pending[nf - 1] && !ctx->graph_mode) { FS_CK(cudaStreamSynchronize(ctx->st)); fs_solver_stats_collect(ctx); }
  FS_TIMING(FS_CK(cudaEventRecord(ctx->sev[nf - 1][0], ctx->st)));
  if (solver == FS_SOLVER_SOR) {
    // colour-major copy, sweeps on it, back to cell order
    k_to_colour<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(N, ctx->W, ctx->color_rows, ctx->ncfP, ctx->ac, ctx->bc,
                                                     ctx->anb, ctx->acP, ctx->bcP, ctx->anbP, ctx->dphiP);
    FS_LAUNCH_CHECK();
    if ((rc = coop_grid_size(ctx))) return rc;
    SorPArgs sp{};
    sp.N = N; sp.W = ctx->W; sp.ncf = ctx->ncfP; sp.cn = ctx->cnP; sp.color_ptr = ctx->color_rows + N;
    sp.ac = ctx->acP; sp.anb = ctx->anbP; sp.bc = ctx->bcP; sp.x = ctx->dphiP; sp.part = ctx->red;
    sp.ires = a.ires; sp.rrf = rrf; sp.itmax = itmax; sp.ncolors = ctx->ncolors; sp.iters = a.iters; sp.diag = a.diag;
    int G = ctx->coop_grid;
    long need = (N + fs_coop_block(ctx) - 1) / fs_coop_block(ctx);
    if (need < G) G = (int)(need < 1 ? 1 : need);
    void *args[] = {&sp};
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][0], ctx->st)));
    FS_CK(fs_coop_launch((const void *)k_sor_colour, G, fs_coop_block(ctx), args, ctx->st));
    FS_LAUNCH_CHECK();
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][1], ctx->st)));
    k_from_colour<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(N, ctx->cposP, ctx->dphiP, ctx->dphi);
    FS_LAUNCH_CHECK();
  } else if (solver == FS_SOLVER_ILU) {
    if ((rc = ilu_build(ctx))) return rc;
    if ((rc = coop_grid_size(ctx))) return rc;
    fs_ilu *I = ctx->ilu;
    IluArgs g{};
    g.N = N; g.W = ctx->W; g.nlf = I->nlf; g.nlb = I->nlb; g.itmax = itmax;
    g.ncf = ctx->ncf; g.cn = ctx->cn; g.lo_ptr = I->lo_ptr; g.lo_i = I->lo_i; g.lo_sj = I->lo_sj; g.lo_si = I->lo_si;
    g.fl_ptr = I->fl_ptr; g.fl_rows = I->fl_rows; g.bl_ptr = I->bl_ptr; g.bl_rows = I->bl_rows;
    g.ac = ctx->ac; g.anb = ctx->anb; g.bc = ctx->bc; g.x = ctx->dphi; g.dc = I->dc; g.rc = I->rc; g.part = ctx->red;
    g.ires = a.ires; g.rrf = rrf; g.iters = a.iters; g.diag = a.diag;
    int G = ctx->coop_grid;
    long need = (N + fs_coop_block(ctx) - 1) / fs_coop_block(ctx);
    if (need < G) G = (int)(need < 1 ? 1 : need);
    void *args[] = {&g};
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][0], ctx->st)));
    FS_CK(fs_coop_launch((const void *)k_ilu, G, fs_coop_block(ctx), args, ctx->st));
    FS_LAUNCH_CHECK();
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][1], ctx->st)));
  } else if (solver == FS_SOLVER_PBCG) {
    if ((rc = ilu_build(ctx)) || (rc = pbcg_build(ctx))) return rc;
    if ((rc = coop_grid_size(ctx))) return rc;
    fs_ilu *I = ctx->ilu;
    PbcgArgs g{};
    g.N = N; g.W = ctx->W; g.nlf = I->nlf; g.itmax = itmax;
    g.ncf = ctx->ncf; g.cn = ctx->cn; g.lo_ptr = I->lo_ptr; g.lo_i = I->lo_i; g.lo_sj = I->lo_sj; g.lo_si = I->lo_si;
    g.fl_ptr = I->fl_ptr; g.fl_rows = I->fl_rows; g.tr_ptr = I->tr_ptr; g.tr_i = I->tr_i; g.tr_si = I->tr_si;
    g.ac = ctx->ac; g.anb = ctx->anb; g.bc = ctx->bc; g.x = ctx->dphi; g.dc = I->dc;
    g.r = ctx->kr; g.rr = ctx->kr0; g.p = ctx->kp; g.pp = ctx->kv; g.z = ctx->ks; g.zz = ctx->kt; g.part = ctx->red;
    g.ires = a.ires; g.rrf = rrf; g.iters = a.iters; g.diag = a.diag;
    int G = ctx->coop_grid;
    long need = (N + fs_coop_block(ctx) - 1) / fs_coop_block(ctx);
    if (need < G) G = (int)(need < 1 ? 1 : need);
    void *args[] = {&g};
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][0], ctx->st)));
    FS_CK(fs_coop_launch((const void *)k_pbcg, G, fs_coop_block(ctx), args, ctx->st));
    FS_LAUNCH_CHECK();
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][1], ctx->st)));
  } else if (solver == FS_SOLVER_BICGS) {
    a.itmax = ctx->cfg.krylov_maxit;
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][0], ctx->st)));
    rc = coop_launch(ctx, (void *)k_bicgstab, a);
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][1], ctx->st)));
  } else if (solver == FS_SOLVER_GMRES) {
    if (!ctx->gm) FS_CK(cudaMalloc(&ctx->gm, sizeof(double) * (size_t)(FS_GM_M + 8) * N));
    GmresArgs g{};
    g.N = N; g.W = ctx->W; g.cn = ctx->cn; g.ac = ctx->ac; g.anb = ctx->anb; g.bc = ctx->bc;
    double *p = ctx->gm;
    g.V = p; p += (size_t)(FS_GM_M + 1) * N;
    g.w = p; p += N; g.x1 = p; p += N; g.xOpt = p; p += N; g.rOpt = p; p += N;
    g.xG = p; p += N; g.rG = p; p += N; g.bn = p;
    g.x = ctx->kx; g.r = ctx->kr; g.dphi = ctx->dphi; g.part = ctx->red;
    g.iters = a.iters; g.diag = a.diag;
    if ((rc = coop_grid_size(ctx))) return rc;
    int G = ctx->coop_grid;
    long need = (N + fs_coop_block(ctx) - 1) / fs_coop_block(ctx);
    if (need < G) G = (int)(need < 1 ? 1 : need);
    void *args[] = {&g};
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][0], ctx->st)));
    FS_CK(fs_coop_launch((const void *)k_gmres, G, fs_coop_block(ctx), args, ctx->st));
    FS_LAUNCH_CHECK();
    FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[nf - 1][1], ctx->st)));
  } else if (solver == FS_SOLVER_AMG || solver == FS_SOLVER_AMG_BICGS || solver == FS_SOLVER_AMG32_BICGS ||
             solver == FS_SOLVER_AMG32GS_BICGS) {
    rc = fs_mg_solve(ctx, nf, rrf, solver);
  } else {
    ctx->err = "unknown solver";
    return FS_E_ARG;
  }
  if (rc) return rc;
  if (ctx->pc_defer && nf == FS_VAR_PC) return FS_OK;   // fs_linear_solve_finish after the batched launch
  FS_TIMING(FS_CK(cudaEventRecord(ctx->sev[nf - 1][1], ctx->st)); ctx->s_pending[nf - 1] = true);
  k_axpy_field<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(N, fi, ctx->dphi);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

// the end of a solve whose Krylov launch was deferred (pc_defer): fi += dphi
int fs_linear_solve_finish(fs_ctx *ctx, int nf, double *fi) {
  (void)nf;
  const int N = ctx->N;
  k_axpy_field<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(N, fi, ctx->dphi);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

int fs_solver_stats_collect(fs_ctx *ctx) {
  int32_t it[FS_NITERS];
  bool any = false;
  for (int q = 0; q < FS_NEQ; q++) any |= ctx->s_pending[q];
  if (!any) return FS_OK;
  FS_CK(cudaMemcpy(it, ctx->d_iters, sizeof(it), cudaMemcpyDeviceToHost));
  for (int q = 0; q < FS_NEQ; q++) {
    if (!ctx->s_pending[q]) continue;
    float ms = 0.f;
    FS_CK(cudaEventElapsedTime(&ms, ctx->sev[q][0], ctx->sev[q][1]));
    ctx->s_ms[q] += ms; ctx->s_its[q] += it[q]; ctx->s_calls[q] += 1;
    float kms = 0.f;
    if (cudaEventElapsedTime(&kms, ctx->kev[q][0], ctx->kev[q][1]) == cudaSuccess) ctx->k_ms[q] += kms;
    else cudaGetLastError();
    ctx->s_pending[q] = false;
  }
  return FS_OK;
}

// ======================================================================
// fs_bicgstab_noalloc: the BiCGSTAB solve for callers that cannot allocate.
//
// Some callers cannot call cudaMalloc at all: a Fortran host that must stay
// inside a memory budget fixed by another framework's allocator, code running
// while a CUDA graph is being captured elsewhere in the process, or a plugin
// host that forbids device allocations after start-up.  They still own the
// matrix, the right-hand side and the solution in device memory, but not the
// six Krylov work vectors.  This entry point runs the same k_bicgstab kernel
// with its work vectors, partial sums and counters in one fixed file-scope
// device array, so it allocates nothing.
//
// Limits and rules:
//   - at most FS_NOALLOC_MAX_ROWS rows; larger systems are rejected with
//     FS_E_TOO_LARGE before anything is launched;
//   - the array is shared by every call on a device: two calls whose kernels
//     overlap on the GPU (different streams, or different host threads on one
//     device) race on it and give wrong answers; serialise them;
//   - nothing in the array has to start at zero: the kernel writes every work
//     entry (r0, r, p first, then v, s, t, then the partial sums) before it
//     reads it in the same call, so the previous call's contents are ignored;
//   - the first call on a device does the set-up: with that device current
//     it looks up the array's device address with cudaGetSymbolAddress and
//     caches it, keyed on the CUDA context current at the call.  A call under
//     another context of the same device (a driver-API context, or the
//     primary context re-created after cudaDeviceReset) repeats the set-up.
//     Make the first call on a device before any stream capture begins.
// ======================================================================
#define FS_NOALLOC_VECS 6
#define FS_NOALLOC_PARTS (6 * FS_RED_BLOCKS)

static __device__ __align__(256) double g_noalloc_scratch[FS_NOALLOC_VECS * (size_t)FS_NOALLOC_MAX_ROWS +
                                                          FS_NOALLOC_PARTS + 16];

#include <mutex>
namespace {
struct NoallocDev { double *base = nullptr; int grid = 0; void *cuctx = nullptr; };
std::mutex g_noalloc_mu;
NoallocDev g_noalloc_dev[64];

// the CUDA context current on this thread (cuCtxGetCurrent through the
// runtime's driver entry point, so the library needs no link to libcuda)
int noalloc_current_context(void **cuctx) {
  typedef int (*CtxGetCurrent)(void **);
  static CtxGetCurrent fn = nullptr;
  if (!fn) {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !f)
      return FS_E_CUDA;
    fn = (CtxGetCurrent)f;
  }
  *cuctx = nullptr;
  return fn(cuctx) == 0 ? FS_OK : FS_E_CUDA;   // null when no context is current yet
}
}  // namespace

extern "C" int fs_bicgstab_noalloc(int32_t n, int32_t w, const int32_t *ncf, const int32_t *cn,
                                   const double *ac, const double *anb, const double *bc, double *x,
                                   int32_t maxit, double tol, int32_t *iters, void *stream) {
  if (n <= 0 || w <= 0 || !ncf || !cn || !ac || !anb || !bc || !x || maxit < 1) return FS_E_ARG;
  if (n > FS_NOALLOC_MAX_ROWS) return FS_E_TOO_LARGE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return FS_E_CUDA;
  void *cuctx = nullptr;
  NoallocDev d;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (noalloc_current_context(&cuctx) != FS_OK) return FS_E_CUDA;
    if (!cuctx || !g_noalloc_dev[dev].base || g_noalloc_dev[dev].cuctx != cuctx) {
      // once per device and context, with that device current: the symbol's
      // device address (the lookup also makes the primary context current
      // when no context was)
      double *ptr = nullptr;
      if (cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return FS_E_CUDA;
      if (noalloc_current_context(&cuctx) != FS_OK || !cuctx) return FS_E_CUDA;
      int per_sm = 0, per_sm2 = 0, sms = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k_bicgstab, FS_COOP_BLOCK, 0) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, (const void *)k_sor_colour, FS_COOP_BLOCK, 0) != cudaSuccess ||
          cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return FS_E_CUDA;
      if (per_sm2 < per_sm) per_sm = per_sm2;
      if (per_sm < 1) return FS_E_CUDA;
      int g = sms * (per_sm > 4 ? 4 : per_sm);   // the grid the context solvers use
      if (g > FS_RED_BLOCKS) g = FS_RED_BLOCKS;
      g_noalloc_dev[dev].base = ptr;
      g_noalloc_dev[dev].grid = g;
      g_noalloc_dev[dev].cuctx = cuctx;
    }
    d = g_noalloc_dev[dev];
  }
  const size_t M = (size_t)FS_NOALLOC_MAX_ROWS;
  double *base = d.base;
  SolveArgs a{};
  a.N = n; a.W = w; a.ncf = ncf; a.cn = cn; a.ac = ac; a.anb = anb; a.bc = bc;
  a.x = x; a.dphi = x;
  a.r = base; a.r0 = base + M; a.p = base + 2 * M; a.v = base + 3 * M; a.s = base + 4 * M; a.t = base + 5 * M;
  a.part = base + FS_NOALLOC_VECS * M;
  a.diag = a.part + FS_NOALLOC_PARTS;
  a.iters = iters ? iters : (int32_t *)(a.diag + 4);
  a.ires = a.diag;
  a.tol = tol; a.itmax = maxit;
  int G = d.grid;
  long need = ((long)n + FS_COOP_BLOCK - 1) / FS_COOP_BLOCK;
  if (need < G) G = (int)need;
  void *args[] = {&a};
  if (cudaLaunchCooperativeKernel((const void *)k_bicgstab, dim3(G), dim3(FS_COOP_BLOCK), args, 0,
                                  (cudaStream_t)stream) != cudaSuccess)
    return FS_E_CUDA;
  return FS_OK;
}

// the three momentum solves in one cooperative launch (multi-RHS form)
int fs_momentum_batched_solve(fs_ctx *ctx) {
  const int N = ctx->N;
  int rc = coop_grid_size(ctx);
  if (rc) return rc;
  for (int c = 0; c < 3; c++) {
    if (ctx->s_pending[c] && !ctx->graph_mode) { FS_CK(cudaStreamSynchronize(ctx->st)); fs_solver_stats_collect(ctx); }
  }
  FS_TIMING(FS_CK(cudaEventRecord(ctx->sev[0][0], ctx->st)));
  k_to_colour3<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(N, ctx->color_rows, ctx->ncfP, ctx->ac3, ctx->bc3, ctx->anb,
                                                    ctx->ac3P, ctx->bc3P, ctx->anbP, ctx->x3P);
  FS_LAUNCH_CHECK();
  Sor3Args a{};
  a.N = N; a.W = ctx->W; a.ncf = ctx->ncfP; a.cn = ctx->cnP; a.color_ptr = ctx->color_rows + N;
  a.ac3 = ctx->ac3P; a.anb = ctx->anbP; a.bc3 = ctx->bc3P; a.x3 = ctx->x3P; a.part = ctx->red;
  a.ires3 = ctx->resblk + RB_ABS; a.rrf = ctx->cfg.rrf_mom; a.itmax = ctx->cfg.itmax_mom; a.ncolors = ctx->ncolors;
  a.iters3 = ctx->d_iters;
  if (ctx->mom_defer) {   // launched with other contexts' by fs_mom_batch_launch, then fs_momentum_batched_finish
    static_assert(sizeof(Sor3Args) <= sizeof(ctx->mom_pend), "mom_pend too small");
    memcpy(ctx->mom_pend, &a, sizeof(a));
    ctx->mom_pending = true;
    return FS_OK;
  }
  int G = ctx->coop_grid;
  long need = (N + fs_coop_block(ctx) - 1) / fs_coop_block(ctx);
  if (need < G) G = (int)(need < 1 ? 1 : need);
  void *args[] = {&a};
  FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[0][0], ctx->st)));
  FS_CK(fs_coop_launch((const void *)k_sor3_colour, G, fs_coop_block(ctx), args, ctx->st));
  FS_TIMING(FS_CK(cudaEventRecord(ctx->kev[0][1], ctx->st)));
  FS_LAUNCH_CHECK();
  return fs_momentum_batched_finish(ctx);
}

int fs_momentum_batched_finish(fs_ctx *ctx) {
  const int N = ctx->N;
  k_from_colour3<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(N, ctx->cposP, ctx->x3P, ctx->u, ctx->v, ctx->w);
  FS_LAUNCH_CHECK();
  FS_TIMING(FS_CK(cudaEventRecord(ctx->sev[0][1], ctx->st)); ctx->s_pending[0] = true);
  return FS_OK;
}

std::vector<int32_t> fs_cta_split(int cap, const double *weight, int n) {
  double wsum = 0.;
  for (int q = 0; q < n; q++) wsum += std::max(weight[q], 0.);
  std::vector<int> cnt(n, 1);
  const int left = cap - n;
  if (wsum > 0. && left > 0) {
    std::vector<double> rem(n);
    int given = 0;
    for (int q = 0; q < n; q++) {
      const double share = left * std::max(weight[q], 0.) / wsum;
      const int k = (int)share;
      cnt[q] += k; given += k; rem[q] = share - k;
    }
    std::vector<int> order(n);
    for (int q = 0; q < n; q++) order[q] = q;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return rem[x] > rem[y]; });
    for (int j = 0; j < left - given && j < n; j++) cnt[order[j]]++;
  }
  std::vector<int32_t> start(n + 1, 0);
  for (int q = 0; q < n; q++) start[q + 1] = start[q] + cnt[q];
  return start;
}

struct fs_mom_batch {
  int n = 0, ncta = 0;
  Sor3Args *h_args = nullptr;   // pinned, copied to d_args by each launch
  Sor3Args *d_args = nullptr;
  int32_t *d_start = nullptr;
  unsigned *d_words = nullptr;  // 2n group-barrier words (zero at each launch)
  int32_t **d_status = nullptr;
};

void fs_mom_batch_free(fs_mom_batch *B) {
  if (!B) return;
  if (B->h_args) cudaFreeHost(B->h_args);
  if (B->d_args) cudaFree(B->d_args);
  if (B->d_start) cudaFree(B->d_start);
  if (B->d_words) cudaFree(B->d_words);
  if (B->d_status) cudaFree(B->d_status);
  delete B;
}

int fs_mom_batch_create(fs_ctx **cs, int n, const double *weight, fs_mom_batch **out) {
  if (!cs || n < 1 || !weight || !out) return FS_E_ARG;
  *out = nullptr;
  fs_ctx *ctx = cs[0];
  for (int q = 0; q < n; q++)
    if (!cs[q]->cfg.batched_momentum || cs[q]->cfg.solver_mom != FS_SOLVER_SOR) {
      ctx->err = "a batched momentum launch needs the multi-RHS SOR solve in every context";
      return FS_E_UNSUPPORTED;
    }
  int occ = 0;
  FS_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void *)k_sor3_colour_batch, FS_COOP_BLOCK, 0));
  const int cap = std::min(ctx->num_sms * std::max(occ, 0), FS_RED_BLOCKS);
  if (cap < n) { ctx->err = "more contexts than co-resident CTAs for a batched momentum launch"; return FS_E_UNSUPPORTED; }
  const std::vector<int32_t> start = fs_cta_split(cap, weight, n);
  std::vector<int32_t *> st(n);
  for (int q = 0; q < n; q++) st[q] = cs[q]->d_status;
  fs_mom_batch *B = new fs_mom_batch;
  B->n = n; B->ncta = start[n];
  cudaError_t e;
  if ((e = cudaHostAlloc((void **)&B->h_args, sizeof(Sor3Args) * n, cudaHostAllocDefault)) != cudaSuccess ||
      (e = cudaMalloc(&B->d_args, sizeof(Sor3Args) * n)) != cudaSuccess ||
      (e = cudaMalloc(&B->d_start, sizeof(int32_t) * (n + 1))) != cudaSuccess ||
      (e = cudaMalloc(&B->d_words, sizeof(unsigned) * 2 * n)) != cudaSuccess ||
      (e = cudaMalloc(&B->d_status, sizeof(int32_t *) * n)) != cudaSuccess ||
      (e = cudaMemcpy(B->d_start, start.data(), sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(B->d_status, st.data(), sizeof(int32_t *) * n, cudaMemcpyHostToDevice)) != cudaSuccess) {
    ctx->err = std::string("batched momentum set-up: ") + cudaGetErrorString(e);
    fs_mom_batch_free(B);
    return FS_E_CUDA;
  }
  *out = B;
  return FS_OK;
}

int fs_mom_batch_launch(fs_mom_batch *B, fs_ctx **cs, int n, cudaStream_t st) {
  if (!B || !cs || n != B->n) return FS_E_ARG;
  fs_ctx *ctx = cs[0];
  for (int q = 0; q < n; q++) {
    if (!cs[q]->mom_pending) { ctx->err = "batched momentum launch: a context prepared no solve"; return FS_E_ARG; }
    memcpy(&B->h_args[q], cs[q]->mom_pend, sizeof(Sor3Args));
    cs[q]->mom_pending = false;
  }
  FS_CK(cudaMemcpyAsync(B->d_args, B->h_args, sizeof(Sor3Args) * n, cudaMemcpyHostToDevice, st));
  FS_CK(cudaMemsetAsync(B->d_words, 0, sizeof(unsigned) * 2 * n, st));
  void *args[] = {&B->d_args, &B->d_start, &B->n, &B->d_words, &B->d_status};
  FS_CK(fs_coop_launch((const void *)k_sor3_colour_batch, B->ncta, FS_COOP_BLOCK, args, st));
  FS_LAUNCH_CHECK();
  return FS_OK;
}
