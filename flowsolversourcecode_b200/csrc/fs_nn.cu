// fs_nn.cu -- learned initial guess for the pressure-correction solve (no
// reference counterpart: the reference always starts p' from zero).
//
// A message-passing network on the cell graph of the mesh (nodes = cells,
// edges = interior faces through the slot-major neighbour table cn):
//
//   X (N x 8)  node features of the p' system at solve time:
//              b/s_b, ac/mean(ac) - 1, sum(face coefficients)/ac - 1,
//              du/dx, dv/dy, dw/dz (/ rms), previous p' (mean removed, / rms), 1
//   w_ij       = c_f / sqrt(ac_i ac_j), c_f the p' face coefficient: symmetric
//   h0         = relu(X W_in + b_in)                                  (N x 64)
//   layer l    m = sum_j w_ij h_j ;  h <- h + relu([h, m] W_l + b_l)  (4 layers)
//   y          = h w_out + b_out ;  guess = (y - mean y) * rms(previous p')
//
// The layer products [h, m] (N x 128) x W_l (128 x 64) and their backward
// products (dW = A^T dz, dA = dz W^T) run on the 5th-generation tensor cores
// (tcgen05.mma, BF16 operands staged in shared memory in the UMMA canonical
// layout, FP32 accumulators in TMEM); activations, the gather, the small
// input/output layers and the optimiser are FP32.  The products are skinny
// (K = 128, N = 64) and the layer kernels move ~0.5 KB per row, so they are
// bounded by the neighbour gather, not by the tensor pipe.
//
// The p' solver takes the guess into the basis of its least-squares initial
// guess (k_guess_fit) and iterates to its usual tolerance; a host policy
// (fs_nn_before_pc) keeps the guess only while it reduces iterations against
// zero-start probes.
//
// Training: supervised on snapshots the plain solver captures (features,
// edge weights, converged p' normalised by rms(previous p')), loss
// sum((y - mean y) - t)^2 / sum t^2 per snapshot, Adam, all on the GPU with
// the kernels below.  Deterministic: per-CTA partial gradients are summed in a
// fixed order.
#include "fs_internal.cuh"
#include <cuda_bf16.h>
#include <algorithm>
#include <random>

#define NN_F 8
#define NN_H 64
#define NN_K (2 * NN_H)
#define NN_L 4
#define NN_TM 128           // rows per tile of the layer kernels
#define NN_THREADS 256
#define NN_RED 296          // CTAs of the reduction-style kernels

#define NN_OFF_WIN 0
#define NN_OFF_BIN (NN_F * NN_H)
#define NN_OFF_L(l) (NN_OFF_BIN + NN_H + (l) * (NN_K * NN_H + NN_H))
#define NN_OFF_WOUT NN_OFF_L(NN_L)
#define NN_OFF_BOUT (NN_OFF_WOUT + NN_H)
#define NN_NP (NN_OFF_BOUT + 1)
static_assert(NN_NP == FS_NN_NPARAM, "parameter count");

typedef __nv_bfloat16 bf16;

struct fs_nn {
  int N = 0, W = 0;
  float *theta = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
  bf16 *wt = nullptr;     // per layer W^T (64 x 128) bf16
  bf16 *wr = nullptr;     // per layer W   (128 x 64) bf16
  float *X = nullptr, *wgt = nullptr;
  float *H[NN_L + 1] = {};
  uint8_t *mask[NN_L + 1] = {};
  float *dH = nullptr, *dH2 = nullptr, *DM = nullptr, *y = nullptr, *dy = nullptr;
  float *part = nullptr;  // NN_RED x (NN_K*NN_H + NN_H) partial gradients
  double *sc = nullptr;   // scalars: [0] s_b [1] mean ac [2] s_g [3] mean prev [4] s_p [5] mean y [6] sum t^2 [7] loss
  double *redp = nullptr; // NN_RED x 8 partial sums
  double *prev = nullptr, *guess = nullptr;
  int cap = 0, count = 0, next = 0;
  float *snapX = nullptr, *snapW = nullptr, *snapT = nullptr;
  std::vector<double> snap_tt;
  bool have_prev = false, use = false, capture = false, feat_valid = false;
  int step = 0;
  int32_t *d_cnt = nullptr;  // [fallbacks, uses], counted by the p' solver
  float *tbuf = nullptr;     // target staging of fs_nn_eval_host
  // policy: guess only while it reduces iterations against zero-start probes
  bool pending = false, last_guessed = false;
  double z_last = 0., gain = 0., g_avg = 0., z_avg = 0.;
  int n_g = 0, n_z = 0, since_probe = 0, park = 0;
  int32_t parked_total = 0;
};

namespace {

// ---------------------------------------------------------------- reductions
__device__ double nn_block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.;
  if (threadIdx.x == 0)
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) r += sh[q];
  return r;  // valid in thread 0
}

// per-block partials of up to 5 row sums (fixed grid, fixed order)
struct SumArgs {
  int N, nq;
  const double *a[5];
  int kind[5];   // 0: a, 1: a^2, 2: sum of squares of three comp-major vectors (a = 3N)
};
__global__ void k_nn_sums(SumArgs s, double *redp) {
  __shared__ double sh[32];
  double acc[5] = {0., 0., 0., 0., 0.};
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < s.N; i += (long)gridDim.x * blockDim.x)
    for (int q = 0; q < s.nq; q++) {
      const double *a = s.a[q];
      if (s.kind[q] == 0) acc[q] += a[i];
      else if (s.kind[q] == 1) acc[q] += a[i] * a[i];
      else acc[q] += a[i] * a[i] + a[s.N + i] * a[s.N + i] + a[2L * s.N + i] * a[2L * s.N + i];
    }
  for (int q = 0; q < s.nq; q++) {
    double r = nn_block_sum(acc[q], sh);
    if (threadIdx.x == 0) redp[blockIdx.x * 8 + q] = r;
  }
}
__global__ void k_nn_sums_f(int N, const float *a, const float *b, double *redp) {
  __shared__ double sh[32];
  double s0 = 0., s1 = 0.;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    s0 += a[i];
    if (b) s1 += (double)b[i] * b[i];
  }
  double r0 = nn_block_sum(s0, sh), r1 = nn_block_sum(s1, sh);
  if (threadIdx.x == 0) { redp[blockIdx.x * 8] = r0; redp[blockIdx.x * 8 + 1] = r1; }
}
// out[q] = f(sum over blocks of partial q), one thread per q
__global__ void k_nn_final(const double *redp, int nblk, int nq, int N, double *out, int mode) {
  const int q = threadIdx.x;
  double s = 0.;
  if (q < nq)
    for (int b = 0; b < nblk; b++) s += redp[b * 8 + q];
  // mode 0 (features): s_b = rms(b), mean ac, s_g = rms of the components of grad u,
  //   mean prev, s_p = rms(prev - mean prev); otherwise the raw sums
  __shared__ double t[32];
  t[q] = s;
  __syncthreads();
  if (q != 0) return;
  if (mode == 0) {
    double sb = sqrt(t[0] / N), mac = t[1] / N, sg = sqrt(t[2] / (3.0 * N)), mp = t[3] / N;
    double vp = t[4] / N - mp * mp;
    out[0] = sb > 0. ? sb : 1.;
    out[1] = mac != 0. ? mac : 1.;
    out[2] = sg > 0. ? sg : 1.;
    out[3] = mp;
    out[4] = vp > 0. ? sqrt(vp) : 0.;
  } else {
    for (int k = 0; k < nq; k++) out[k] = t[k];
  }
}

// ---------------------------------------------------------------- features
struct FeatArgs {
  int N, W, F;
  const int32_t *slot, *cn;
  const double *ac, *bc, *pcoef, *ug, *vg, *wg, *prev;
  const double *sc;
  float *X, *wgt;
};
__global__ void k_nn_features(FeatArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  const double sb = a.sc[0], mac = a.sc[1], sg = a.sc[2], mp = a.sc[3], sp = a.sc[4];
  const double aci = a.ac[i];
  double csum = 0.;
  for (int j = 0; j < a.W; j++) {
    int k = a.cn[(long)j * a.N + i];
    float w = 0.f;
    if (k >= 0) {
      int f = a.slot[(long)j * a.N + i] >> 1;
      double c = a.pcoef[f];
      csum += c;
      w = (float)(c / sqrt(aci * a.ac[k]));
    }
    a.wgt[(long)j * a.N + i] = w;
  }
  float *x = a.X + (long)i * NN_F;
  x[0] = (float)(a.bc[i] / sb);
  x[1] = (float)(aci / mac - 1.);
  x[2] = (float)(aci != 0. ? csum / aci - 1. : 0.);
  x[3] = (float)(a.ug[i] / sg);
  x[4] = (float)(a.vg[a.N + i] / sg);
  x[5] = (float)(a.wg[2L * a.N + i] / sg);
  x[6] = (float)(sp > 0. ? (a.prev[i] - mp) / sp : 0.);
  x[7] = 1.f;
}

// target of a snapshot: t = (dphi - mean dphi) / s_p
__global__ void k_nn_target(int N, const double *dphi, const double *mean, const double *sc, float *t) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) t[i] = (float)((dphi[i] - mean[0]) / sc[4]);
}

// ---------------------------------------------------------------- input / output layers (FP32)
__global__ void k_nn_in_fwd(int N, const float *X, const float *th, float *H0, uint8_t *mask) {
  long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long)N * NN_H) return;
  long i = q / NN_H;
  int c = (int)(q - i * NN_H);
  float z = th[NN_OFF_BIN + c];
#pragma unroll
  for (int f = 0; f < NN_F; f++) z += X[i * NN_F + f] * th[NN_OFF_WIN + f * NN_H + c];
  H0[q] = z > 0.f ? z : 0.f;
  if (mask) mask[q] = z > 0.f;
}

__global__ void k_nn_out_fwd(int N, const float *H, const float *th, float *y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float4 *h = (const float4 *)(H + (long)i * NN_H);
  float s = th[NN_OFF_BOUT];
#pragma unroll
  for (int c = 0; c < NN_H / 4; c++) {
    float4 v = h[c];
    s += v.x * th[NN_OFF_WOUT + 4 * c] + v.y * th[NN_OFF_WOUT + 4 * c + 1] + v.z * th[NN_OFF_WOUT + 4 * c + 2] +
         v.w * th[NN_OFF_WOUT + 4 * c + 3];
  }
  y[i] = s;
}

// loss and dy: sc[5] = sum y (-> mean), tt = sum t^2 of the snapshot
__global__ void k_nn_loss(int N, const float *y, const float *t, const double *sumy, double tt, float *dy,
                          double *redp) {
  __shared__ double sh[32];
  const double my = sumy[0] / N;
  double l = 0.;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    double d = ((double)y[i] - my) - t[i];
    l += d * d;
    dy[i] = (float)(2. * d / tt);
  }
  double r = nn_block_sum(l, sh);
  if (threadIdx.x == 0) redp[blockIdx.x * 8] = r;
}

// out layer backward: dH = dy w_out^T ; partials of dw_out (64) and db_out (1)
__global__ void __launch_bounds__(NN_THREADS) k_nn_out_bwd(int N, const float *H, const float *dy, const float *th,
                                                           float *dH, float *part, int pstride) {
  __shared__ float sh[4][NN_H + 1];
  const int c = threadIdx.x & (NN_H - 1), rg = threadIdx.x >> 6;
  float gw = 0.f, gb = 0.f;
  const float wc = th[NN_OFF_WOUT + c];
  for (long i = (long)blockIdx.x * 4 + rg; i < N; i += (long)gridDim.x * 4) {
    float d = dy[i];
    gw += H[i * NN_H + c] * d;
    gb += d;
    dH[i * NN_H + c] = d * wc;
  }
  sh[rg][c] = gw;
  sh[rg][NN_H] = 0.f;
  __syncthreads();
  if (rg == 0) {
    float s = sh[0][c] + sh[1][c] + sh[2][c] + sh[3][c];
    part[(long)blockIdx.x * pstride + c] = s;
  }
  __syncthreads();
  if (c == 0) sh[rg][NN_H] = gb;
  __syncthreads();
  if (threadIdx.x == 0) part[(long)blockIdx.x * pstride + NN_H] = sh[0][NN_H] + sh[1][NN_H] + sh[2][NN_H] + sh[3][NN_H];
}

// input layer backward: dz0 = dH0 * mask0 ; partials of dW_in (8 x 64) and db_in (64)
__global__ void __launch_bounds__(NN_THREADS) k_nn_in_bwd(int N, const float *X, const float *dH, const uint8_t *mask,
                                                          float *part, int pstride) {
  __shared__ float sh[4][NN_F + 1][NN_H];
  const int c = threadIdx.x & (NN_H - 1), rg = threadIdx.x >> 6;
  float g[NN_F + 1] = {};
  for (long i = (long)blockIdx.x * 4 + rg; i < N; i += (long)gridDim.x * 4) {
    float dz = mask[i * NN_H + c] ? dH[i * NN_H + c] : 0.f;
#pragma unroll
    for (int f = 0; f < NN_F; f++) g[f] += X[i * NN_F + f] * dz;
    g[NN_F] += dz;
  }
#pragma unroll
  for (int f = 0; f <= NN_F; f++) sh[rg][f][c] = g[f];
  __syncthreads();
  if (rg == 0)
    for (int f = 0; f <= NN_F; f++)
      part[(long)blockIdx.x * pstride + f * NN_H + c] = sh[0][f][c] + sh[1][f][c] + sh[2][f][c] + sh[3][f][c];
}

// ---------------------------------------------------------------- tensor-core helpers
__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// ---------------------------------------------------------------- layer forward (tcgen05)
// Hout = Hin + relu([Hin, m] W + b); mask (training) = z > 0.  One 128-row tile
// per CTA on the 5th-generation tensor cores: the [h, m] tile (128 x 128) and
// W^T (64 x 128) sit in shared memory in the K-major, no-swizzle canonical
// layout of the UMMA descriptors (8-row x 16-byte core matrices: a K chunk of 8
// every 128 bytes, an 8-row group every 2048 bytes), one thread issues the eight
// K=16 steps of tcgen05.mma (M=128, N=64, BF16 x BF16 -> FP32) into a 64-column
// TMEM accumulator, tcgen05.commit arrives on an mbarrier, and every warp reads
// its 32 lanes x 32 columns back with tcgen05.ld for the epilogue.  The wait on
// the mbarrier is bounded: on a timeout the CTA records it in *status, skips the
// epilogue and still frees its TMEM.
#define NN_TC_COLS 64            // TMEM columns of the accumulator (power of 2, >= 32)
#define NN_TC_SPIN (1L << 22)    // polls of the MMA-completion mbarrier before giving up

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (row, k) of a K-major canonical tile with 16 K chunks per row group
__device__ __forceinline__ int canon_off(int row, int k) { return (row >> 3) * 2048 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2; }

// UMMA shared-memory descriptor: K-major, SWIZZLE_NONE, LBO = 128 B (next K chunk),
// SBO = 2048 B (next 8-row group), version 1
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(2048 >> 4) << 32) |
         ((uint64_t)1 << 46);
}

// instruction descriptor: D FP32, A and B BF16, both K-major, N = 64, M = 128
constexpr uint32_t NN_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NN_H >> 3) << 17) |
                              ((uint32_t)(NN_TM >> 4) << 24);

__device__ __forceinline__ void pack8_store(unsigned char *dst, const float *v) {
  uint4 u;
  u.x = pack2(__float2bfloat16(v[0]), __float2bfloat16(v[1]));
  u.y = pack2(__float2bfloat16(v[2]), __float2bfloat16(v[3]));
  u.z = pack2(__float2bfloat16(v[4]), __float2bfloat16(v[5]));
  u.w = pack2(__float2bfloat16(v[6]), __float2bfloat16(v[7]));
  *(uint4 *)dst = u;
}

// stage the [h, m] tile (rows i0..i0+127) as bf16 in the canonical layout: m = sum_j w_ij h_j
__device__ void stage_hm_canon(int N, int W, const int32_t *__restrict__ cn, const float *__restrict__ wgt,
                               const float *__restrict__ H, long i0, unsigned char *A) {
  const int rr = threadIdx.x >> 1, q = threadIdx.x & 1;
  const long i = i0 + rr;
  float hv[32], acc[32];
#pragma unroll
  for (int c = 0; c < 32; c++) { hv[c] = 0.f; acc[c] = 0.f; }
  if (i < N) {
    const float4 *hs = (const float4 *)(H + i * NN_H + q * 32);
#pragma unroll
    for (int c = 0; c < 8; c++) {
      float4 v = hs[c];
      hv[4 * c] = v.x; hv[4 * c + 1] = v.y; hv[4 * c + 2] = v.z; hv[4 * c + 3] = v.w;
    }
    for (int j = 0; j < W; j++) {
      int k = cn[(long)j * N + i];
      if (k < 0) continue;
      float w = wgt[(long)j * N + i];
      const float4 *hk = (const float4 *)(H + (long)k * NN_H + q * 32);
#pragma unroll
      for (int c = 0; c < 8; c++) {
        float4 v = hk[c];
        acc[4 * c] += w * v.x; acc[4 * c + 1] += w * v.y; acc[4 * c + 2] += w * v.z; acc[4 * c + 3] += w * v.w;
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 4; c++) {
    pack8_store(A + canon_off(rr, q * 32 + 8 * c), hv + 8 * c);
    pack8_store(A + canon_off(rr, NN_H + q * 32 + 8 * c), acc + 8 * c);
  }
}

__global__ void __launch_bounds__(NN_THREADS) k_nn_layer_fwd(int N, int W, const int32_t *__restrict__ cn,
                                                             const float *__restrict__ wgt, const float *Hin,
                                                             const bf16 *__restrict__ wt, const float *__restrict__ bias,
                                                             float *Hout, uint8_t *mask, int32_t *status) {
  extern __shared__ __align__(16) unsigned char smem[];
  // tiles on a 128-byte boundary (the launch adds 128 bytes of slack)
  unsigned char *A = smem + ((128u - (smem_u32(smem) & 127u)) & 127u);   // 128 x 128 bf16, canonical (32 KB)
  unsigned char *WT = A + NN_TM * NN_K * 2;                              // 64 x 128 bf16, canonical (16 KB)
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long i0 = (long)blockIdx.x * NN_TM;
  if (warp == 0) {   // TMEM accumulator: one warp allocates, the address lands in tbase
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tbase)),
                 "r"(NN_TC_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int c = threadIdx.x; c < NN_H * (NN_K / 8); c += blockDim.x) {   // W^T, 16-byte chunks
    const int n = c / (NN_K / 8), kc = c - n * (NN_K / 8);
    *(uint4 *)(WT + (n >> 3) * 2048 + kc * 128 + (n & 7) * 16) = *(const uint4 *)(wt + n * NN_K + kc * 8);
  }
  stage_hm_canon(N, W, cn, wgt, Hin, i0, A);
  // the tensor cores read shared memory through the async proxy
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tbase;
  if (threadIdx.x == 0) {
    const uint32_t a0 = smem_u32(A), b0 = smem_u32(WT);
#pragma unroll
    for (int kk = 0; kk < NN_K / 16; kk++) {
      const uint64_t da = umma_desc(a0 + kk * 256), db = umma_desc(b0 + kk * 256);
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "setp.ne.b32 p, %4, 0;\n\t"
          "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
          "}\n" ::"r"(tmem),
          "l"(da), "l"(db), "r"(NN_IDESC), "r"(kk) : "memory");
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(&mbar))
                 : "memory");
  }
  // bounded wait for the accumulator (phase 0 of the mbarrier)
  uint32_t done = 0;
  for (long spin = 0; spin < NN_TC_SPIN && !done; spin++) {
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(smem_u32(&mbar)), "r"(0)
        : "memory");
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!done) {
    if (lane == 0) atomicExch(status, 1);
  } else {
    // warp w reads TMEM lanes 32 (w % 4) .. +31 (its rows), columns 32 (w / 4) .. +31
    const int rowq = warp & 3, colh = warp >> 2;
    uint32_t v[32];
    const uint32_t ta = tmem + ((uint32_t)(32 * rowq) << 16) + (uint32_t)(32 * colh);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(ta)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    const long i = i0 + 32 * rowq + lane;
    if (i < N) {
      const int c0 = 32 * colh;
      const float4 *hin = (const float4 *)(Hin + i * NN_H + c0);
      float4 *hout = (float4 *)(Hout + i * NN_H + c0);
      uint32_t mb[8];
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const float4 h = hin[c];
        float z[4], o[4];
        const float hh[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
        for (int e = 0; e < 4; e++) {
          z[e] = __uint_as_float(v[4 * c + e]) + bias[c0 + 4 * c + e];
          o[e] = hh[e] + (z[e] > 0.f ? z[e] : 0.f);
        }
        hout[c] = make_float4(o[0], o[1], o[2], o[3]);
        mb[c] = (uint32_t)(z[0] > 0.f) | ((uint32_t)(z[1] > 0.f) << 8) | ((uint32_t)(z[2] > 0.f) << 16) |
                ((uint32_t)(z[3] > 0.f) << 24);
      }
      if (mask) {
        uint4 *m4 = (uint4 *)(mask + i * NN_H + c0);
        m4[0] = make_uint4(mb[0], mb[1], mb[2], mb[3]);
        m4[1] = make_uint4(mb[4], mb[5], mb[6], mb[7]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NN_TC_COLS) : "memory");
}

// ---------------------------------------------------------------- layer backward (tcgen05)
// The same backward on the 5th-generation tensor cores, persistent over tiles:
//   dW (128 x 64) += [h, m]^T dz: UMMA M = 128 features, N = 64, K = the tile's
//     128 rows; operands [h, m]^T and dz^T staged K-major (rows contiguous),
//     accumulated in TMEM columns 128..191 across all of the CTA's tiles;
//   dA (128 x 128) = dz W^T: UMMA M = 128 rows, N = 128 features, K = 64;
//     operands dz and W staged K-major (outputs contiguous), TMEM columns 0..127,
//     read back per tile: dHin = dHout + dA[:, :64], DM = dA[:, 64:].
// One thread issues the twelve K=16 steps of a tile and commits them to an
// mbarrier (one phase per tile); the waits are bounded as in the forward.
__device__ __forceinline__ int canon64_off(int row, int k) { return (row >> 3) * 1024 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2; }
__device__ __forceinline__ uint64_t umma_desc64(uint32_t saddr) {   // K-major, 8 K chunks per row group
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46);
}
constexpr uint32_t NN_IDESC_DA = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NN_K >> 3) << 17) |
                                 ((uint32_t)(NN_TM >> 4) << 24);   // M = 128, N = 128
#define NN_TC_BWD_COLS 256   // dA in columns 0..127, dW in 128..191

__device__ __forceinline__ void tmem_ld32(uint32_t ta, uint32_t *v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(ta)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void umma_f16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, int acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
      "}\n" ::"r"(tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
}

__global__ void __launch_bounds__(NN_THREADS) k_nn_layer_bwd_tc(int N, int W, const int32_t *__restrict__ cn,
                                                                const float *__restrict__ wgt, const float *Hin,
                                                                const uint8_t *__restrict__ mask, const float *dHout,
                                                                const bf16 *__restrict__ wr, float *dHin, float *DM,
                                                                float *part, int pstride, int32_t *status) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char *AT = smem + ((128u - (smem_u32(smem) & 127u)) & 127u);   // [h, m]^T: 128 features x 128 rows (32 KB)
  unsigned char *DZT = AT + NN_K * NN_TM * 2;                             // dz^T: 64 outputs x 128 rows (16 KB)
  unsigned char *DZ = DZT + NN_H * NN_TM * 2;                             // dz: 128 rows x 64 outputs (16 KB)
  unsigned char *WC = DZ + NN_TM * NN_H * 2;                              // W: 128 features x 64 outputs (16 KB)
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase;
  __shared__ float shb[4][NN_H];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tbase)),
                 "r"(NN_TC_BWD_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int q = threadIdx.x; q < NN_K * NN_H; q += blockDim.x) {   // W, rows = input features
    const int f = q / NN_H, o = q - f * NN_H;
    *(bf16 *)(WC + canon64_off(f, o)) = wr[q];
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tbase;
  const int c = threadIdx.x & (NN_H - 1), rg = threadIdx.x >> 6;
  float db = 0.f;
  bool ok = true;
  int it = 0;
  const long ntiles = ((long)N + NN_TM - 1) / NN_TM;
  for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, it++) {
    const long i0 = tile * NN_TM;
    // [h, m]^T: each thread forms half of one row's 128 features, stored transposed
    {
      const int rr = threadIdx.x >> 1, qh = threadIdx.x & 1;
      const long i = i0 + rr;
      float hv[32], acc[32];
#pragma unroll
      for (int e = 0; e < 32; e++) { hv[e] = 0.f; acc[e] = 0.f; }
      if (i < N) {
        const float4 *hs = (const float4 *)(Hin + i * NN_H + qh * 32);
#pragma unroll
        for (int e = 0; e < 8; e++) {
          const float4 v = hs[e];
          hv[4 * e] = v.x; hv[4 * e + 1] = v.y; hv[4 * e + 2] = v.z; hv[4 * e + 3] = v.w;
        }
        for (int j = 0; j < W; j++) {
          const int k = cn[(long)j * N + i];
          if (k < 0) continue;
          const float w = wgt[(long)j * N + i];
          const float4 *hk = (const float4 *)(Hin + (long)k * NN_H + qh * 32);
#pragma unroll
          for (int e = 0; e < 8; e++) {
            const float4 v = hk[e];
            acc[4 * e] += w * v.x; acc[4 * e + 1] += w * v.y; acc[4 * e + 2] += w * v.z; acc[4 * e + 3] += w * v.w;
          }
        }
      }
#pragma unroll
      for (int e = 0; e < 32; e++) {
        *(bf16 *)(AT + canon_off(qh * 32 + e, rr)) = __float2bfloat16(hv[e]);
        *(bf16 *)(AT + canon_off(NN_H + qh * 32 + e, rr)) = __float2bfloat16(acc[e]);
      }
    }
    // dz = dHout * mask, as dz (rows x outputs) and dz^T
    for (int rr = rg; rr < NN_TM; rr += 4) {
      const long i = i0 + rr;
      float dz = 0.f;
      if (i < N && mask[i * NN_H + c]) dz = dHout[i * NN_H + c];
      db += dz;
      const bf16 b = __float2bfloat16(dz);
      *(bf16 *)(DZ + canon64_off(rr, c)) = b;
      *(bf16 *)(DZT + canon_off(c, rr)) = b;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (threadIdx.x == 0) {
      const uint32_t at = smem_u32(AT), dzt = smem_u32(DZT), dz = smem_u32(DZ), wc = smem_u32(WC);
#pragma unroll
      for (int kk = 0; kk < NN_TM / 16; kk++)
        umma_f16(tmem + 128, umma_desc(at + kk * 256), umma_desc(dzt + kk * 256), NN_IDESC, (it > 0 || kk > 0) ? 1 : 0);
#pragma unroll
      for (int kk = 0; kk < NN_H / 16; kk++)
        umma_f16(tmem, umma_desc64(dz + kk * 256), umma_desc64(wc + kk * 256), NN_IDESC_DA, kk > 0 ? 1 : 0);
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(&mbar))
                   : "memory");
    }
    uint32_t done = 0;
    for (long spin = 0; spin < NN_TC_SPIN && !done; spin++) {
      asm volatile(
          "{\n\t.reg .pred P1;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
          "selp.b32 %0, 1, 0, P1;\n\t"
          "}\n"
          : "=r"(done)
          : "r"(smem_u32(&mbar)), "r"((uint32_t)(it & 1))
          : "memory");
    }
    // one verdict for the whole CTA, so every thread takes the same path
    // through the remaining block barriers
    done = __syncthreads_and(done);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!done) {
      if (threadIdx.x == 0) atomicExch(status, 1);
      ok = false;
    } else {
      // warp w: TMEM lanes 32 (w % 4) .. +31 (rows of the tile), columns 64 (w / 4) .. +63 of dA
      const int rowq = warp & 3, half = warp >> 2;
      const long i = i0 + 32 * rowq + lane;
#pragma unroll
      for (int part32 = 0; part32 < 2; part32++) {
        uint32_t v[32];
        const int col0 = 64 * half + 32 * part32;
        tmem_ld32(tmem + ((uint32_t)(32 * rowq) << 16) + (uint32_t)col0, v);
        if (i < N) {
          if (half == 0) {
            const float4 *dh = (const float4 *)(dHout + i * NN_H + col0);
            float4 *out = (float4 *)(dHin + i * NN_H + col0);
#pragma unroll
            for (int e = 0; e < 8; e++) {
              const float4 d = dh[e];
              out[e] = make_float4(d.x + __uint_as_float(v[4 * e]), d.y + __uint_as_float(v[4 * e + 1]),
                                   d.z + __uint_as_float(v[4 * e + 2]), d.w + __uint_as_float(v[4 * e + 3]));
            }
          } else {
            float4 *out = (float4 *)(DM + i * NN_H + (col0 - NN_H));
#pragma unroll
            for (int e = 0; e < 8; e++)
              out[e] = make_float4(__uint_as_float(v[4 * e]), __uint_as_float(v[4 * e + 1]),
                                   __uint_as_float(v[4 * e + 2]), __uint_as_float(v[4 * e + 3]));
          }
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  // partials: dW (128 features x 64) from TMEM, then db (64)
  float *pp = part + (long)blockIdx.x * pstride;
  if (ok) {
    const int rowq = warp & 3, half = warp >> 2;
    uint32_t v[32];
    tmem_ld32(tmem + ((uint32_t)(32 * rowq) << 16) + (uint32_t)(128 + 32 * half), v);
    const int f = 32 * rowq + lane;
#pragma unroll
    for (int e = 0; e < 32; e++) pp[f * NN_H + 32 * half + e] = it > 0 ? __uint_as_float(v[e]) : 0.f;
  }
  shb[rg][c] = db;
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (rg == 0) pp[NN_K * NN_H + c] = shb[0][c] + shb[1][c] + shb[2][c] + shb[3][c];
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NN_TC_BWD_COLS) : "memory");
}

// layer backward (b): dHin[j] += sum_s w_js DM[cn(j,s)] (the aggregation is symmetric)
__global__ void k_nn_layer_bwd_gather(int N, int W, const int32_t *__restrict__ cn, const float *__restrict__ wgt,
                                      const float *__restrict__ DM, float *dHin) {
  long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long)N * (NN_H / 4)) return;
  long i = q / (NN_H / 4);
  int c4 = (int)(q - i * (NN_H / 4));
  float4 s = ((float4 *)(dHin + i * NN_H))[c4];
  for (int j = 0; j < W; j++) {
    int k = cn[(long)j * N + i];
    if (k < 0) continue;
    float w = wgt[(long)j * N + i];
    float4 d = ((const float4 *)(DM + (long)k * NN_H))[c4];
    s.x += w * d.x; s.y += w * d.y; s.z += w * d.z; s.w += w * d.w;
  }
  ((float4 *)(dHin + i * NN_H))[c4] = s;
}

// grad[off + p] = sum over CTAs g of part[g * pstride + p] (fixed order)
__global__ void k_nn_reduce(const float *part, int nblk, int pstride, int count, float *grad) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= count) return;
  float s = 0.f;
  for (int b = 0; b < nblk; b++) s += part[(long)b * pstride + p];
  grad[p] = s;
}

__global__ void k_nn_adam(int n, float *th, const float *gr, float *m1, float *m2, float lr, float c1, float c2) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  float g = gr[p];
  float a = 0.9f * m1[p] + 0.1f * g, b = 0.999f * m2[p] + 0.001f * g * g;
  m1[p] = a; m2[p] = b;
  th[p] -= lr * (a / c1) / (sqrtf(b / c2) + 1e-8f);
}

// bf16 copies of the layer matrices: wt = W^T (64 x 128), wr = W (128 x 64)
__global__ void k_nn_pack(const float *th, bf16 *wt, bf16 *wr) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= NN_L * NN_K * NN_H) return;
  int l = q / (NN_K * NN_H), r = q - l * NN_K * NN_H;
  int k = r / NN_H, n = r - k * NN_H;  // W[k][n]
  float w = th[NN_OFF_L(l) + k * NN_H + n];
  wr[(long)l * NN_K * NN_H + k * NN_H + n] = __float2bfloat16(w);
  wt[(long)l * NN_K * NN_H + n * NN_K + k] = __float2bfloat16(w);
}

// guess = (y - mean y) * s_p
__global__ void k_nn_guess(int N, const float *y, const double *sumy, const double *sc, double *guess) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) guess[i] = ((double)y[i] - sumy[0] / N) * sc[4];
}

}  // namespace

// ================================================================ host
static const size_t NN_SMEM_FWD = sizeof(bf16) * (NN_TM * NN_K + NN_H * NN_K) + 128;   // canonical tiles + alignment slack
static const size_t NN_SMEM_BWD = sizeof(bf16) * (NN_K * NN_TM + 2 * NN_H * NN_TM + NN_K * NN_H) + 128;   // canonical tiles + slack
static const int NN_PSTRIDE = NN_K * NN_H + NN_H;

static int nn_sum_rows(fs_ctx *ctx, fs_nn *nn, SumArgs s, double *out, int mode) {
  k_nn_sums<<<NN_RED, FS_BLOCK, 0, ctx->st>>>(s, nn->redp);
  FS_LAUNCH_CHECK();
  k_nn_final<<<1, 32, 0, ctx->st>>>(nn->redp, NN_RED, s.nq, ctx->N, out, mode);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

// features of the current p' system into nn->X / nn->wgt (and scales into sc[0..4])
static int nn_features(fs_ctx *ctx) {
  fs_nn *nn = ctx->nn;
  const int N = ctx->N;
  SumArgs s{};
  s.N = N; s.nq = 5;
  s.a[0] = ctx->bc; s.kind[0] = 1;
  s.a[1] = ctx->ac; s.kind[1] = 0;
  s.a[2] = ctx->ug; s.kind[2] = 2;   // sum of squares of the components of grad u: its rms scales the
  s.a[3] = nn->prev; s.kind[3] = 0;  // velocity-gradient features
  s.a[4] = nn->prev; s.kind[4] = 1;
  int rc;
  if ((rc = nn_sum_rows(ctx, nn, s, nn->sc, 0))) return rc;
  FeatArgs a{};
  a.N = N; a.W = ctx->W; a.F = ctx->F; a.slot = ctx->slot; a.cn = ctx->cn; a.ac = ctx->ac; a.bc = ctx->bc;
  a.pcoef = ctx->pcoef; a.ug = ctx->ug; a.vg = ctx->vg; a.wg = ctx->wg; a.prev = nn->prev; a.sc = nn->sc;
  a.X = nn->X; a.wgt = nn->wgt;
  k_nn_features<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(a);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

// forward through the network on (X, wgt); train=true keeps masks
static int nn_forward(fs_ctx *ctx, const float *X, const float *wgt, bool train) {
  fs_nn *nn = ctx->nn;
  const int N = ctx->N, W = ctx->W;
  k_nn_in_fwd<<<fs_grid((long)N * NN_H), FS_BLOCK, 0, ctx->st>>>(N, X, nn->theta, nn->H[0], train ? nn->mask[0] : nullptr);
  FS_LAUNCH_CHECK();
  const int tiles = (N + NN_TM - 1) / NN_TM;
  for (int l = 0; l < NN_L; l++) {
    // inference keeps two activation buffers (ping-pong); training keeps all
    float *hin = train ? nn->H[l] : nn->H[l & 1], *hout = train ? nn->H[l + 1] : nn->H[(l + 1) & 1];
    k_nn_layer_fwd<<<tiles, NN_THREADS, NN_SMEM_FWD, ctx->st>>>(N, W, ctx->cn, wgt, hin,
                                                                 nn->wt + (size_t)l * NN_K * NN_H,
                                                                 nn->theta + NN_OFF_L(l) + NN_K * NN_H, hout,
                                                                 train ? nn->mask[l + 1] : nullptr, ctx->d_status);
    FS_LAUNCH_CHECK();
  }
  const float *hl = train ? nn->H[NN_L] : nn->H[NN_L & 1];
  k_nn_out_fwd<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(N, hl, nn->theta, nn->y);
  FS_LAUNCH_CHECK();
  k_nn_sums_f<<<NN_RED, FS_BLOCK, 0, ctx->st>>>(N, nn->y, nullptr, nn->redp);
  FS_LAUNCH_CHECK();
  k_nn_final<<<1, 32, 0, ctx->st>>>(nn->redp, NN_RED, 1, N, nn->sc + 5, 1);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

// loss, backward and the gradient vector nn->grad for target t (sum t^2 = tt)
static int nn_backward(fs_ctx *ctx, const float *X, const float *wgt, const float *t, double tt) {
  fs_nn *nn = ctx->nn;
  const int N = ctx->N, W = ctx->W;
  k_nn_loss<<<NN_RED, FS_BLOCK, 0, ctx->st>>>(N, nn->y, t, nn->sc + 5, tt, nn->dy, nn->redp);
  FS_LAUNCH_CHECK();
  k_nn_final<<<1, 32, 0, ctx->st>>>(nn->redp, NN_RED, 1, N, nn->sc + 7, 1);
  FS_LAUNCH_CHECK();
  k_nn_out_bwd<<<NN_RED, NN_THREADS, 0, ctx->st>>>(N, nn->H[NN_L], nn->dy, nn->theta, nn->dH, nn->part, NN_PSTRIDE);
  FS_LAUNCH_CHECK();
  k_nn_reduce<<<1, 128, 0, ctx->st>>>(nn->part, NN_RED, NN_PSTRIDE, NN_H + 1, nn->grad + NN_OFF_WOUT);
  FS_LAUNCH_CHECK();
  const int tiles = (N + NN_TM - 1) / NN_TM;
  const int G = std::min(tiles, NN_RED);
  float *dcur = nn->dH, *dnext = nn->dH2;
  for (int l = NN_L - 1; l >= 0; l--) {
    k_nn_layer_bwd_tc<<<G, NN_THREADS, NN_SMEM_BWD, ctx->st>>>(N, W, ctx->cn, wgt, nn->H[l], nn->mask[l + 1], dcur,
                                                               nn->wr + (size_t)l * NN_K * NN_H, dnext, nn->DM,
                                                               nn->part, NN_PSTRIDE, ctx->d_status);
    FS_LAUNCH_CHECK();
    k_nn_reduce<<<fs_grid(NN_PSTRIDE), FS_BLOCK, 0, ctx->st>>>(nn->part, G, NN_PSTRIDE, NN_PSTRIDE,
                                                               nn->grad + NN_OFF_L(l));
    FS_LAUNCH_CHECK();
    k_nn_layer_bwd_gather<<<fs_grid((long)N * (NN_H / 4)), FS_BLOCK, 0, ctx->st>>>(N, W, ctx->cn, wgt, nn->DM, dnext);
    FS_LAUNCH_CHECK();
    std::swap(dcur, dnext);
  }
  k_nn_in_bwd<<<NN_RED, NN_THREADS, 0, ctx->st>>>(N, X, dcur, nn->mask[0], nn->part, NN_PSTRIDE);
  FS_LAUNCH_CHECK();
  k_nn_reduce<<<fs_grid((NN_F + 1) * NN_H), FS_BLOCK, 0, ctx->st>>>(nn->part, NN_RED, NN_PSTRIDE, (NN_F + 1) * NN_H,
                                                                    nn->grad + NN_OFF_WIN);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

static int nn_pack(fs_ctx *ctx) {
  fs_nn *nn = ctx->nn;
  k_nn_pack<<<fs_grid(NN_L * NN_K * NN_H), FS_BLOCK, 0, ctx->st>>>(nn->theta, nn->wt, nn->wr);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

void fs_nn_free(fs_ctx *ctx) {
  fs_nn *nn = ctx->nn;
  if (!nn) return;
  void *p[] = {nn->theta, nn->grad, nn->m1, nn->m2, nn->wt, nn->wr, nn->X, nn->wgt, nn->dH, nn->dH2, nn->DM, nn->y,
               nn->dy, nn->part, nn->sc, nn->redp, nn->prev, nn->guess, nn->snapX, nn->snapW, nn->snapT, nn->d_cnt,
               nn->tbuf};
  for (void *x : p) if (x) cudaFree(x);
  for (int l = 0; l <= NN_L; l++) { if (nn->H[l]) cudaFree(nn->H[l]); if (nn->mask[l]) cudaFree(nn->mask[l]); }
  delete nn;
  ctx->nn = nullptr;
}

// Guess policy (the zero start is the fallback whenever the guess does not
// reduce iterations): every 4th solve, and every solve while parked, starts
// from zero and measures the zero-start iteration count.  Iteration counts
// drift over the outer iterations, so each guessed solve is compared with the
// latest zero-start probe (at most three solves earlier); the saving is
// averaged exponentially (weight 1/4), and once four guessed solves save less
// than half an iteration on average the guess is parked for 32 solves (no
// inference while parked).
static bool nn_want_guess(fs_nn *nn) {
  if (!nn->use || !nn->have_prev) return false;
  if (nn->park > 0) { nn->park--; return false; }
  if (nn->n_z < 1 || ++nn->since_probe >= 4) { nn->since_probe = 0; return false; }
  return true;
}

void fs_nn_note_iters(fs_ctx *ctx, int pc_iters) {
  fs_nn *nn = ctx->nn;
  if (!nn || !nn->pending) return;
  nn->pending = false;
  const double v = pc_iters;
  if (nn->last_guessed) {
    const double s = nn->z_last - v;
    nn->gain = nn->n_g ? 0.75 * nn->gain + 0.25 * s : s;
    nn->g_avg = nn->n_g ? 0.75 * nn->g_avg + 0.25 * v : v;
    nn->n_g++;
    if (nn->n_g >= 4 && nn->gain < 0.5) {
      nn->park = 32; nn->n_g = 0; nn->parked_total++;
    }
  } else {
    nn->z_last = v;
    nn->z_avg = nn->n_z ? 0.75 * nn->z_avg + 0.25 * v : v;
    nn->n_z++;
  }
}

// before the p' solve: features (when capturing or guessing) and the guess.
// Returns the guess pointer in *x0 (nullptr: start from zero).
int fs_nn_before_pc(fs_ctx *ctx, const double **x0) {
  *x0 = nullptr;
  fs_nn *nn = ctx->nn;
  if (!nn || !(nn->use || nn->capture)) return FS_OK;
  nn->feat_valid = false;
  const bool guess = nn_want_guess(nn);
  nn->pending = nn->use && nn->have_prev;
  nn->last_guessed = guess;
  if (!nn->have_prev || !(guess || nn->capture)) return FS_OK;
  int rc;
  if ((rc = nn_features(ctx))) return rc;
  nn->feat_valid = true;
  if (!guess) return FS_OK;
  if ((rc = nn_forward(ctx, nn->X, nn->wgt, false))) return rc;
  k_nn_guess<<<fs_grid(ctx->N), FS_BLOCK, 0, ctx->st>>>(ctx->N, nn->y, nn->sc + 5, nn->sc, nn->guess);
  FS_LAUNCH_CHECK();
  *x0 = nn->guess;
  return FS_OK;
}

// after the p' solve (dphi holds p'): capture a snapshot, keep p' as `previous`
int fs_nn_after_pc(fs_ctx *ctx) {
  fs_nn *nn = ctx->nn;
  if (!nn) return FS_OK;
  const int N = ctx->N, W = ctx->W;
  if (nn->capture && nn->feat_valid && nn->cap > 0) {
    double sp = 0.;
    FS_CK(cudaMemcpyAsync(&sp, nn->sc + 4, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    FS_CK(cudaStreamSynchronize(ctx->st));
    if (sp > 0.) {
      const int s = nn->next;
      FS_CK(cudaMemcpyAsync(nn->snapX + (size_t)s * N * NN_F, nn->X, sizeof(float) * N * NN_F,
                            cudaMemcpyDeviceToDevice, ctx->st));
      FS_CK(cudaMemcpyAsync(nn->snapW + (size_t)s * N * W, nn->wgt, sizeof(float) * N * W, cudaMemcpyDeviceToDevice,
                            ctx->st));
      SumArgs a{};
      a.N = N; a.nq = 1; a.a[0] = ctx->dphi; a.kind[0] = 0;
      int rc;
      if ((rc = nn_sum_rows(ctx, nn, a, nn->sc + 6, 1))) return rc;
      // sc[6] = sum dphi -> mean
      double sum = 0.;
      FS_CK(cudaMemcpyAsync(&sum, nn->sc + 6, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
      FS_CK(cudaStreamSynchronize(ctx->st));
      double mean = sum / N;
      FS_CK(cudaMemcpyAsync(nn->sc + 6, &mean, sizeof(double), cudaMemcpyHostToDevice, ctx->st));
      float *t = nn->snapT + (size_t)s * N;
      k_nn_target<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(N, ctx->dphi, nn->sc + 6, nn->sc, t);
      FS_LAUNCH_CHECK();
      k_nn_sums_f<<<NN_RED, FS_BLOCK, 0, ctx->st>>>(N, t, t, nn->redp);
      FS_LAUNCH_CHECK();
      k_nn_final<<<1, 32, 0, ctx->st>>>(nn->redp, NN_RED, 2, N, nn->sc + 6, 1);
      FS_LAUNCH_CHECK();
      double tt[2];
      FS_CK(cudaMemcpyAsync(tt, nn->sc + 6, sizeof(tt), cudaMemcpyDeviceToHost, ctx->st));
      FS_CK(cudaStreamSynchronize(ctx->st));
      nn->snap_tt[s] = tt[1];
      nn->next = (s + 1) % nn->cap;
      nn->count = std::min(nn->count + 1, nn->cap);
    }
  }
  FS_CK(cudaMemcpyAsync(nn->prev, ctx->dphi, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->st));
  nn->have_prev = true;
  return FS_OK;
}

int32_t *fs_nn_counters(fs_ctx *ctx) { return ctx->nn ? ctx->nn->d_cnt : nullptr; }

extern "C" int fs_nn_create(fs_ctx *ctx, int snapshot_capacity, uint64_t seed) {
  if (!ctx || snapshot_capacity < 0) return FS_E_ARG;
  cudaSetDevice(ctx->dev);
  fs_nn_free(ctx);
  fs_nn *nn = new fs_nn();
  ctx->nn = nn;
  const int N = ctx->N, W = ctx->W;
  nn->N = N; nn->W = W;
  auto al = [&](void **p, size_t bytes) -> int {
    FS_CK(cudaMalloc(p, std::max<size_t>(bytes, 16)));
    FS_CK(cudaMemset(*p, 0, std::max<size_t>(bytes, 16)));
    return FS_OK;
  };
  int rc = 0;
  const size_t NH = (size_t)N * NN_H;
  if ((rc = al((void **)&nn->theta, sizeof(float) * NN_NP)) || (rc = al((void **)&nn->grad, sizeof(float) * NN_NP)) ||
      (rc = al((void **)&nn->m1, sizeof(float) * NN_NP)) || (rc = al((void **)&nn->m2, sizeof(float) * NN_NP)) ||
      (rc = al((void **)&nn->wt, sizeof(bf16) * NN_L * NN_K * NN_H)) ||
      (rc = al((void **)&nn->wr, sizeof(bf16) * NN_L * NN_K * NN_H)) ||
      (rc = al((void **)&nn->X, sizeof(float) * N * NN_F)) || (rc = al((void **)&nn->wgt, sizeof(float) * N * W)) ||
      (rc = al((void **)&nn->dH, sizeof(float) * NH)) || (rc = al((void **)&nn->dH2, sizeof(float) * NH)) ||
      (rc = al((void **)&nn->DM, sizeof(float) * NH)) || (rc = al((void **)&nn->y, sizeof(float) * N)) ||
      (rc = al((void **)&nn->dy, sizeof(float) * N)) ||
      (rc = al((void **)&nn->part, sizeof(float) * NN_RED * NN_PSTRIDE)) ||
      (rc = al((void **)&nn->sc, sizeof(double) * 16)) || (rc = al((void **)&nn->redp, sizeof(double) * NN_RED * 8)) ||
      (rc = al((void **)&nn->prev, sizeof(double) * N)) || (rc = al((void **)&nn->guess, sizeof(double) * N)) ||
      (rc = al((void **)&nn->d_cnt, sizeof(int32_t) * 4)) || (rc = al((void **)&nn->tbuf, sizeof(float) * N))) {
    fs_nn_free(ctx);
    return rc;
  }
  for (int l = 0; l <= NN_L; l++)
    if ((rc = al((void **)&nn->H[l], sizeof(float) * NH)) || (rc = al((void **)&nn->mask[l], NH))) {
      fs_nn_free(ctx);
      return rc;
    }
  nn->cap = snapshot_capacity;
  if (nn->cap > 0) {
    if ((rc = al((void **)&nn->snapX, sizeof(float) * (size_t)nn->cap * N * NN_F)) ||
        (rc = al((void **)&nn->snapW, sizeof(float) * (size_t)nn->cap * N * W)) ||
        (rc = al((void **)&nn->snapT, sizeof(float) * (size_t)nn->cap * N))) {
      fs_nn_free(ctx);
      return rc;
    }
    nn->snap_tt.assign(nn->cap, 0.);
  }
  // He-style initialisation from a seeded generator (host), biases zero;
  // the output layer starts at zero so the untrained guess is zero
  std::vector<float> th(NN_NP, 0.f);
  std::mt19937_64 gen(seed);
  auto fill = [&](int off, int fan_in, int count) {
    std::normal_distribution<float> d(0.f, sqrtf(2.f / fan_in));
    for (int q = 0; q < count; q++) th[off + q] = d(gen);
  };
  fill(NN_OFF_WIN, NN_F, NN_F * NN_H);
  for (int l = 0; l < NN_L; l++) {
    std::normal_distribution<float> d(0.f, 0.5f * sqrtf(2.f / NN_K));
    for (int q = 0; q < NN_K * NN_H; q++) th[NN_OFF_L(l) + q] = d(gen);
  }
  FS_CK(cudaMemcpy(nn->theta, th.data(), sizeof(float) * NN_NP, cudaMemcpyHostToDevice));
  FS_CK(cudaFuncSetAttribute((const void *)k_nn_layer_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)NN_SMEM_FWD));
  FS_CK(cudaFuncSetAttribute((const void *)k_nn_layer_bwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)NN_SMEM_BWD));
  if ((rc = nn_pack(ctx))) return rc;
  FS_CK(cudaStreamSynchronize(ctx->st));
  return FS_OK;
}

extern "C" int fs_nn_mode(fs_ctx *ctx, int capture, int use) {
  if (!ctx || !ctx->nn) return FS_E_ARG;
  ctx->nn->capture = capture != 0;
  ctx->nn->use = use != 0;
  return FS_OK;
}

extern "C" int fs_nn_snapshots(fs_ctx *ctx, int32_t *count) {
  if (!ctx || !ctx->nn || !count) return FS_E_ARG;
  *count = ctx->nn->count;
  return FS_OK;
}

extern "C" int fs_nn_train(fs_ctx *ctx, int epochs, float lr, uint64_t seed, float *loss_first, float *loss_last) {
  if (!ctx || !ctx->nn || epochs < 0) return FS_E_ARG;
  fs_nn *nn = ctx->nn;
  if (nn->count == 0) { ctx->err = "no snapshots captured"; return FS_E_ARG; }
  cudaSetDevice(ctx->dev);
  const int N = ctx->N, W = ctx->W;
  std::vector<int> order(nn->count);
  for (int q = 0; q < nn->count; q++) order[q] = q;
  std::mt19937_64 gen(seed);
  int rc;
  for (int e = 0; e < epochs; e++) {
    std::shuffle(order.begin(), order.end(), gen);
    double lsum = 0.;
    for (int s : order) {
      const float *X = nn->snapX + (size_t)s * N * NN_F, *wg = nn->snapW + (size_t)s * N * W,
                  *t = nn->snapT + (size_t)s * N;
      if ((rc = nn_forward(ctx, X, wg, true))) return rc;
      if ((rc = nn_backward(ctx, X, wg, t, nn->snap_tt[s] > 0. ? nn->snap_tt[s] : 1.))) return rc;
      nn->step++;
      const float c1 = 1.f - powf(0.9f, (float)nn->step), c2 = 1.f - powf(0.999f, (float)nn->step);
      k_nn_adam<<<fs_grid(NN_NP), FS_BLOCK, 0, ctx->st>>>(NN_NP, nn->theta, nn->grad, nn->m1, nn->m2, lr, c1, c2);
      FS_LAUNCH_CHECK();
      if ((rc = nn_pack(ctx))) return rc;
      double l = 0.;
      FS_CK(cudaMemcpyAsync(&l, nn->sc + 7, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
      FS_CK(cudaStreamSynchronize(ctx->st));
      lsum += l / (nn->snap_tt[s] > 0. ? nn->snap_tt[s] : 1.);
    }
    float lm = (float)(lsum / nn->count);
    if (e == 0 && loss_first) *loss_first = lm;
    if (loss_last) *loss_last = lm;
  }
  return FS_OK;
}

extern "C" int fs_nn_params(fs_ctx *ctx, float *get, const float *set, size_t n) {
  if (!ctx || !ctx->nn || n != (size_t)NN_NP) return FS_E_ARG;
  cudaSetDevice(ctx->dev);
  FS_CK(cudaStreamSynchronize(ctx->st));
  if (get) FS_CK(cudaMemcpy(get, ctx->nn->theta, sizeof(float) * NN_NP, cudaMemcpyDeviceToHost));
  if (set) {
    FS_CK(cudaMemcpy(ctx->nn->theta, set, sizeof(float) * NN_NP, cudaMemcpyHostToDevice));
    int rc = nn_pack(ctx);
    if (rc) return rc;
    FS_CK(cudaStreamSynchronize(ctx->st));
  }
  return FS_OK;
}

extern "C" int fs_nn_eval_host(fs_ctx *ctx, const float *X, const float *wgt, const float *target, float *loss,
                               float *grad, float *y) {
  if (!ctx || !ctx->nn || !X || !wgt) return FS_E_ARG;
  cudaSetDevice(ctx->dev);
  fs_nn *nn = ctx->nn;
  const int N = ctx->N, W = ctx->W;
  FS_CK(cudaMemcpy(nn->X, X, sizeof(float) * N * NN_F, cudaMemcpyHostToDevice));
  FS_CK(cudaMemcpy(nn->wgt, wgt, sizeof(float) * N * W, cudaMemcpyHostToDevice));
  int rc;
  if ((rc = nn_forward(ctx, nn->X, nn->wgt, true))) return rc;
  if (target) {
    std::vector<double> t(target, target + N);
    double tt = 0.;
    for (double v : t) tt += v * v;
    FS_CK(cudaMemcpy(nn->tbuf, target, sizeof(float) * N, cudaMemcpyHostToDevice));
    if ((rc = nn_backward(ctx, nn->X, nn->wgt, nn->tbuf, tt > 0. ? tt : 1.))) return rc;
    FS_CK(cudaStreamSynchronize(ctx->st));
    double l = 0.;
    FS_CK(cudaMemcpy(&l, nn->sc + 7, sizeof(double), cudaMemcpyDeviceToHost));
    if (loss) *loss = (float)(l / (tt > 0. ? tt : 1.));
    if (grad) FS_CK(cudaMemcpy(grad, nn->grad, sizeof(float) * NN_NP, cudaMemcpyDeviceToHost));
  }
  FS_CK(cudaStreamSynchronize(ctx->st));
  if (y) FS_CK(cudaMemcpy(y, nn->y, sizeof(float) * N, cudaMemcpyDeviceToHost));
  return FS_OK;
}

extern "C" int fs_nn_policy(fs_ctx *ctx, double *avg_guessed, double *avg_zero, int32_t *parked) {
  if (!ctx || !ctx->nn) return FS_E_ARG;
  if (avg_guessed) *avg_guessed = ctx->nn->g_avg;
  if (avg_zero) *avg_zero = ctx->nn->z_avg;
  if (parked) *parked = ctx->nn->parked_total;
  return FS_OK;
}

extern "C" int fs_nn_stats(fs_ctx *ctx, int32_t *uses, int32_t *fallbacks) {
  if (!ctx || !ctx->nn) return FS_E_ARG;
  cudaSetDevice(ctx->dev);
  int32_t c[4];
  FS_CK(cudaStreamSynchronize(ctx->st));
  FS_CK(cudaMemcpy(c, ctx->nn->d_cnt, sizeof(c), cudaMemcpyDeviceToHost));
  if (fallbacks) *fallbacks = c[0];
  if (uses) *uses = c[1];
  return FS_OK;
}
