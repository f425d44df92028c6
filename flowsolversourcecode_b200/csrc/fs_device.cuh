// fs_device.cuh -- device helpers shared by the assembly kernels of
// fs_simple.cu and fs_turb.cu: reference constants, deterministic block
// reductions, the residual statistics of CalculateResiduals, face-gradient
// interpolation and the TVD deferred correction.  Everything is internal to
// the including translation unit.
#pragma once
#include "fs_internal.cuh"

// Slot loops of the cell-centric gathers: the first FS_PF (face, neighbour)
// pairs of a cell are loaded up front, so a face's data loads no longer wait
// behind its own index loads; faces are still visited in slot order.
#define FS_PF 6
#define FS_SLOT_PREFETCH(nc, slot, cn, N, i)                                    \
  int pf_s_[FS_PF], pf_k_[FS_PF];                                               \
  _Pragma("unroll") for (int j_ = 0; j_ < FS_PF; j_++) {                        \
    pf_s_[j_] = j_ < (nc) ? (slot)[(long)j_ * (N) + (i)] : 0;                   \
    pf_k_[j_] = j_ < (nc) ? (cn)[(long)j_ * (N) + (i)] : 0;                     \
  }
#define FS_SLOT_LOOP(nc, slot, cn, N, i, fn)                                    \
  do {                                                                          \
    _Pragma("unroll") for (int j_ = 0; j_ < FS_PF; j_++)                        \
      if (j_ < (nc)) fn(pf_s_[j_], pf_k_[j_]);                                  \
    for (int j_ = FS_PF; j_ < (nc); j_++) fn((slot)[(long)j_ * (N) + (i)], (cn)[(long)j_ * (N) + (i)]); \
  } while (0)
// a rolled loop over the prefetched pairs, passing the slot index too:
// fn(j, slot, neighbour); for bodies too large to unroll (the prefetched
// pairs then sit in thread-local memory, an L1 hit per slot)
#define FS_SLOT_LOOP_J(nc, slot, cn, N, i, fn)                                  \
  do {                                                                          \
    _Pragma("unroll 1") for (int j_ = 0; j_ < (nc); j_++) {                     \
      const int s_ = j_ < FS_PF ? pf_s_[j_] : (slot)[(long)j_ * (N) + (i)];     \
      const int k_ = j_ < FS_PF ? pf_k_[j_] : (cn)[(long)j_ * (N) + (i)];       \
      fn(j_, s_, k_);                                                           \
    }                                                                           \
  } while (0)

namespace {

constexpr double M23 = (double)(-2.0f / 3.0f);   // `-2./3.` is REAL(4) (AssembleBulkViscosity.for:36)
constexpr double EPS9 = (double)1.e-9f;          // `1.e-9` is REAL(4) (AssembleHRSchemeCorrection.for:92)
constexpr double TINY = 1.0e-15;                 // Constants1.F90

// ------------------------------------------------------------ reductions
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}
// deterministic block sum / max (fixed tree for a fixed blockDim); result valid in thread 0
__device__ double block_sum(double v, double *sh) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.;
  if (wid == 0) {
    r = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.;
    r = warp_sum(r);
  }
  return r;
}
__device__ double block_max(double v, double *sh) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = -1.0e300;
  if (wid == 0) {
    r = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : -1.0e300;
    r = warp_max(r);
  }
  return r;
}

// per-cell residual statistics of CalculateResiduals (CalculateResidualsRoutine.for:30-67)
// at dphi=0: r=|bc|.  Writes block partials.
__device__ void residual_partials(double r, double acphi, double *red, int nblk) {
  __shared__ double sh[32];
  double s0 = block_sum(r, sh);
  double s1 = block_sum(r * r, sh);
  double m0 = block_max(r, sh);
  double m1 = block_max(acphi, sh);
  if (threadIdx.x == 0) {
    red[RED_SUM0 * nblk + blockIdx.x] = s0;
    red[RED_SUM1 * nblk + blockIdx.x] = s1;
    red[RED_MAX0 * nblk + blockIdx.x] = m0;
    red[RED_MAX1 * nblk + blockIdx.x] = m1;
  }
}

// single block: partials -> residual block slot q (ResorAbs/Max/RMS/Scaled)
__global__ void k_residual_final(const double *red, int nblk, int N, int q, double *rb) {
  __shared__ double sh[32];
  double s0 = 0., s1 = 0., m0 = -1., m1 = -1.;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    s0 += red[RED_SUM0 * nblk + b];
    s1 += red[RED_SUM1 * nblk + b];
    m0 = fmax(m0, red[RED_MAX0 * nblk + b]);
    m1 = fmax(m1, red[RED_MAX1 * nblk + b]);
  }
  s0 = block_sum(s0, sh); s1 = block_sum(s1, sh);
  m0 = block_max(m0, sh); m1 = block_max(m1, sh);
  if (threadIdx.x == 0) {
    rb[RB_ABS + q] = s0;
    rb[RB_MAX + q] = m0;
    rb[RB_RMS + q] = sqrt(s1 / N);
    rb[RB_SCL + q] = (q == 3) ? 0. : m0 / (m1 + TINY);
  }
}

// ------------------------------------------------------------ interpolation helpers
// InterpolateGradientToFace (InterpolateGradientFromElementToFace.for:3-100),
// owner-perspective: o = owner gradient, n = neighbour gradient.
__device__ __forceinline__ void face_grad(int scheme, double g, double md, double phio, double phin,
                                          double d, double ex, double ey, double ez,
                                          double ox, double oy, double oz, double nx, double ny, double nz,
                                          double &fx, double &fy, double &fz) {
  double gg = g;
  if (scheme == FS_GI_UPWIND) gg = (md > 0.) ? 1. : 0.;
  else if (scheme == FS_GI_DOWNWIND) gg = (md > 0.) ? 0. : 1.;
  fx = gg * ox + (1. - gg) * nx;
  fy = gg * oy + (1. - gg) * ny;
  fz = gg * oz + (1. - gg) * nz;
  if (scheme == FS_GI_AVERAGECORRECTED) {
    double c = (phin - phio) / d;
    c = c - (fx * ex + fy * ey + fz * ez);
    fx = fx + c * ex; fy = fy + c * ey; fz = fz + c * ez;
  }
}

// TVDLimiter (Convection/LimitersTVDType.for:4)
__device__ __forceinline__ double tvd_psi(int s, double rf) {
  switch (s) {
  case FS_TVD_UPWIND: return 0.;
  case FS_TVD_DOWNWIND: return 2.;
  case FS_TVD_FROMM: return 0.5 * (1. + rf);
  case FS_TVD_SOU: return rf;
  case FS_TVD_CD: return 1.;
  case FS_TVD_QUICK: return (3. + rf) / 4.;
  case FS_TVD_SUPERBEE: return fmax(fmax(0., fmin(1., 2. * rf)), fmin(2., rf));
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

// HRSchemesCorrections (AssembleHRSchemeCorrection.for:36-134), TVD framework; cpf is 1
// but for the temperature equation's face specific heat (:121-124)
__device__ __forceinline__ double hr_flux(int scheme, double bleed, double md, double phio, double phin,
                                          const double go[3], const double gn[3], double dx, double dy, double dz,
                                          double cpf = 1.) {
  double phic, phid, gx, gy, gz;
  if (md > 0.) { phic = phio; phid = phin; gx = go[0]; gy = go[1]; gz = go[2]; }
  else { phic = phin; phid = phio; gx = gn[0]; gy = gn[1]; gz = gn[2]; dx = -dx; dy = -dy; dz = -dz; }
  double phiu = phid - 2. * (gx * dx + gy * dy + gz * dz);
  double diff = phid - phic, rf;
  if (fabs(diff) < EPS9) rf = 0.; else rf = (phic - phiu) / diff;
  double psi = tvd_psi(scheme, rf);
  double phiHR = phic + 0.5 * psi * diff;
  phiHR = (1. - bleed) * phiHR + bleed * phic;
  return md * (phiHR - phic) * cpf;
}

// AssembleTransientTerm (AssembleTheTransientTerm.for:52-330) for time-level
// block lvl (0..2 velocity, 4 k, 5 epsilon, 6 temperature) of cell i: adds to
// the cell's FluxCE and FluxTE sums in the reference's order.  cp is the
// temperature equation's SpecificHeat (Density*SpecificHeat*Volume), 1 otherwise
// (multiplying by 1 leaves the other equations' products unchanged).
__device__ __forceinline__ void transient_term(const FsTransient &t, int lvl, long N, long i, double V, double phi,
                                               double &fce, double &fte, double cp = 1.) {
  const double po = t.old[lvl * N + i];
  if (!t.three) {
    const double fcl = t.rho * cp * V / t.d, fcol = -(t.rho * cp * V / t.d);
    fce = fce + fcl;
    fte = fte + fcl * phi + fcol * po;
  } else {
    const double poo = t.oldold[lvl * N + i];
    const double fcl = t.f1 * t.rho * cp * V, fcol = t.s2 * (t.f2 * t.rho * cp * V), fcool = t.f3 * t.rho * cp * V;
    fce = fce + fcl;
    fte = fte + fcl * phi + fcol * po + fcool * poo;
  }
}

}  // namespace
