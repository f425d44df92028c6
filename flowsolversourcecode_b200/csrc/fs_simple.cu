// fs_simple.cu -- the per-face / per-cell kernels of one SIMPLE outer iteration.
//
// Every kernel is cell-centric gather (one thread per cell, looping over the
// cell's face slots in slot order) or face-centric (one thread per face).  A
// cell's slots hold its faces in increasing face index, so a gather visits a
// cell's faces in the same order as the reference's face loops scatter into
// that cell (AssembleGolbalElementAndFaceFluxes.for:60-98): sums are formed
// in the reference's order without atomics, and with --fmad=false the
// assembled coefficients are bit-identical to the CPU restatement.
#include "fs_internal.cuh"
#include "fs_device.cuh"

namespace {

// ------------------------------------------------------------ gradients
struct GradJob {
  int nfld;
  const double *phi[4];
  const double *bphi[4];
  double *out[4];      // 3N destination of this pass
  const double *in[4]; // 3N gradient of the previous pass (correction passes)
};

// CTAs per SM the wide gather kernels are compiled for (register caps):
// uncapped, k_mom_interior took 162 registers (one CTA per SM) and
// k_gg_corr<4> 128; these latency-bound gathers run faster with more resident
// warps even at the cost of a few spilled registers
#ifndef FS_MOM_MINB
#define FS_MOM_MINB 2
#endif
#ifndef FS_GG_MINB
#define FS_GG_MINB 3
#endif
#ifndef FS_GG0_MINB
#define FS_GG0_MINB 3
#endif
#ifndef FS_FACE_MINB
#define FS_FACE_MINB 4
#endif

// StandardGreenGauss / first pass of StandardGreenGaussFaceCorrection1
// (StandardGreenGaussGradient.for:35-79; StandardGreenGaussCorrection1Gradient.for:47-96).
// All NF fields of a call are done in one slot loop, so a face's geometry and
// index are read once per cell for all fields.  A cell's own values stay in
// registers; the other cell of each interior face comes from the slot-major
// neighbour table cn.
template <int NF>
__global__ void __launch_bounds__(FS_BLOCK, FS_GG0_MINB) k_gg0(GradJob J, int N, int F, int B,
    const int32_t *__restrict__ ncf, const int32_t *__restrict__ slot, const int32_t *__restrict__ cn,
    const double *__restrict__ gf, const double *__restrict__ sf,
    const double *__restrict__ bsf, const double *__restrict__ vol) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int nc = ncf[i];
  double V = vol[i];
  double ps[NF], gx[NF], gy[NF], gz[NF];
#pragma unroll
  for (int q = 0; q < NF; q++) { ps[q] = J.phi[q][i]; gx[q] = 0.; gy[q] = 0.; gz[q] = 0.; }
  FS_SLOT_PREFETCH(nc, slot, cn, N, i);
  auto face = [&](int s, int k) {
    int f = s >> 1;
    if (f < F) {
      double g = gf[f], sx = sf[f], sy = sf[F + f], sz = sf[2L * F + f];
      bool nb = s & 1;
#pragma unroll
      for (int q = 0; q < NF; q++) {
        double pk = J.phi[q][k];
        double po = nb ? pk : ps[q], pn = nb ? ps[q] : pk;
        double fip = po * g + pn * (1. - g);
        double fx = fip * sx, fy = fip * sy, fz = fip * sz;
        if (nb) { gx[q] = gx[q] - fx; gy[q] = gy[q] - fy; gz[q] = gz[q] - fz; }
        else { gx[q] = gx[q] + fx; gy[q] = gy[q] + fy; gz[q] = gz[q] + fz; }
      }
    } else {
      int b = f - F;
      double bx = bsf[b], by = bsf[B + b], bz = bsf[2L * B + b];
#pragma unroll
      for (int q = 0; q < NF; q++) {
        double bp = J.bphi[q][b];
        gx[q] = gx[q] + bp * bx; gy[q] = gy[q] + bp * by; gz[q] = gz[q] + bp * bz;
      }
    }
  };
  FS_SLOT_LOOP(nc, slot, cn, N, i, face);
#pragma unroll
  for (int q = 0; q < NF; q++) {
    double *o = J.out[q];
    o[i] = gx[q] / V; o[N + i] = gy[q] / V; o[2L * N + i] = gz[q] / V;
  }
}

// Shared-memory staging of the correction pass (FS_GG_STAGE > 0, off by
// default): a CTA first copies phi and the previous gradient of the cells
// [first - FS_GG_STAGE, last + FS_GG_STAGE] with coalesced loads, and the
// face loop takes a neighbour inside that window from shared memory (on a
// structured ordering the +-1 and +-nx neighbours), the others from global
// memory.  The values are the same either way.  Measured at 128^3 with a
// window of +-128 cells: the assembly phases took 3.73 ms per iteration
// against 3.42 ms unstaged -- the neighbours it serves are L1/L2 hits
// already, and the window load, the barrier and the extra spills cost more.
#ifndef FS_GG_STAGE
#define FS_GG_STAGE 0
#endif
constexpr int GG_WIN = FS_BLOCK + 2 * FS_GG_STAGE;   // staged cells per CTA

// correction pass of StandardGreenGaussFaceCorrection1 (:98-172)
template <int NF>
__global__ void __launch_bounds__(FS_BLOCK, FS_GG_MINB) k_gg_corr(GradJob J, int N, int F, int B,
    const int32_t *__restrict__ ncf, const int32_t *__restrict__ slot, const int32_t *__restrict__ cn,
    const double *__restrict__ gf, const double *__restrict__ sf, const double *__restrict__ dfp,
    const double *__restrict__ bsf, const double *__restrict__ vol) {
#if FS_GG_STAGE > 0
  extern __shared__ double stg[];   // [q][phi, gx, gy, gz][GG_WIN]
  const long w0 = (long)blockIdx.x * blockDim.x - FS_GG_STAGE;
#pragma unroll
  for (int q = 0; q < NF; q++)
    for (int t = threadIdx.x; t < GG_WIN; t += blockDim.x) {
      const long c = w0 + t;
      const bool in = c >= 0 && c < N;
      stg[(4 * q + 0) * GG_WIN + t] = in ? J.phi[q][c] : 0.;
      stg[(4 * q + 1) * GG_WIN + t] = in ? J.in[q][c] : 0.;
      stg[(4 * q + 2) * GG_WIN + t] = in ? J.in[q][N + c] : 0.;
      stg[(4 * q + 3) * GG_WIN + t] = in ? J.in[q][2L * N + c] : 0.;
    }
  __syncthreads();
#endif
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int nc = ncf[i];
  double V = vol[i];
  double ps[NF], gsx[NF], gsy[NF], gsz[NF], gx[NF], gy[NF], gz[NF];
#pragma unroll
  for (int q = 0; q < NF; q++) {
    ps[q] = J.phi[q][i];
    gsx[q] = J.in[q][i]; gsy[q] = J.in[q][N + i]; gsz[q] = J.in[q][2L * N + i];
    gx[q] = 0.; gy[q] = 0.; gz[q] = 0.;
  }
  FS_SLOT_PREFETCH(nc, slot, cn, N, i);
  auto face = [&](int s, int k) {
    int f = s >> 1;
    if (f < F) {
      double g = gf[f], g1 = 1. - g;
      double sx = sf[f], sy = sf[F + f], sz = sf[2L * F + f];
      double dx = dfp[f], dy = dfp[F + f], dz = dfp[2L * F + f];
      bool nb = s & 1;
#if FS_GG_STAGE > 0
      const long lk = k - w0;
      const bool sm = (unsigned long)lk < (unsigned long)GG_WIN;
#endif
#pragma unroll
      for (int q = 0; q < NF; q++) {
        const double *__restrict__ gi = J.in[q];
#if FS_GG_STAGE > 0
        double pk, gkx, gky, gkz;
        if (sm) {
          pk = stg[(4 * q + 0) * GG_WIN + lk]; gkx = stg[(4 * q + 1) * GG_WIN + lk];
          gky = stg[(4 * q + 2) * GG_WIN + lk]; gkz = stg[(4 * q + 3) * GG_WIN + lk];
        } else {
          pk = J.phi[q][k]; gkx = gi[k]; gky = gi[N + k]; gkz = gi[2L * N + k];
        }
#else
        double pk = J.phi[q][k], gkx = gi[k], gky = gi[N + k], gkz = gi[2L * N + k];
#endif
        double po = nb ? pk : ps[q], pn = nb ? ps[q] : pk;
        double gox = nb ? gkx : gsx[q], gnx = nb ? gsx[q] : gkx;
        double goy = nb ? gky : gsy[q], gny = nb ? gsy[q] : gky;
        double goz = nb ? gkz : gsz[q], gnz = nb ? gsz[q] : gkz;
        double fip = po * g + pn * g1;
        double cx = gox * g + gnx * g1; cx = cx * dx;
        double cy = goy * g + gny * g1; cy = cy * dy;
        double cz = goz * g + gnz * g1; cz = cz * dz;
        double phif = fip + cx + cy + cz;
        double fx = phif * sx, fy = phif * sy, fz = phif * sz;
        if (nb) { gx[q] = gx[q] - fx; gy[q] = gy[q] - fy; gz[q] = gz[q] - fz; }
        else { gx[q] = gx[q] + fx; gy[q] = gy[q] + fy; gz[q] = gz[q] + fz; }
      }
    } else {
      int b = f - F;
      double bx = bsf[b], by = bsf[B + b], bz = bsf[2L * B + b];
#pragma unroll
      for (int q = 0; q < NF; q++) {
        double bp = J.bphi[q][b];
        gx[q] = gx[q] + bp * bx; gy[q] = gy[q] + bp * by; gz[q] = gz[q] + bp * bz;
      }
    }
  };
  FS_SLOT_LOOP(nc, slot, cn, N, i, face);
#pragma unroll
  for (int q = 0; q < NF; q++) {
    double *o = J.out[q];
    o[i] = gx[q] / V; o[N + i] = gy[q] / V; o[2L * N + i] = gz[q] / V;
  }
}

// boundary gradients: owner value, then the CorrectGradients.for projections
struct BGradJob { int nfld; int var[4]; const double *g[4]; double *bg[4]; };
__global__ void k_bgrad(BGradJob J, int N, int B, const int32_t *__restrict__ bown,
                        const int32_t *__restrict__ btype, const double *__restrict__ bnf,
                        const double *__restrict__ bnzii) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  int k = bown[b], t = btype[b];
  double nx = bnf[b], ny = bnf[B + b], nz = bnf[2L * B + b], nzi = bnzii[b];
  for (int q = 0; q < J.nfld; q++) {
    const double *g = J.g[q];
    double gx = g[k], gy = g[N + k], gz = g[2L * N + k];
    double ox = gx, oy = gy, oz = gz;
    int var = J.var[q];
    bool vel = (var == FS_VAR_U || var == FS_VAR_V || var == FS_VAR_W);
    bool prs = (var == FS_VAR_P || var == FS_VAR_RHOK);   // 'press' and 'rhok' (CalculateGradients.for:266-271)
    if ((vel && (t == FS_BC_OUTLET_FD || fs_is_sp_outlet(t))) || (prs && t == FS_BC_SYMMETRY)) {
      // CorrectGradientAtOulet / CorrectPressureGradientAtSymmetryBoundary, nz=BFaceAreanz(i,i)
      ox = gx * (1. - nx * nx) - gy * nx * ny - gz * nx * nzi;
      oy = gy * (1. - ny * ny) - gx * ny * nx - gz * ny * nzi;
      oz = gz * (1. - nzi * nzi) - gx * nzi * nx - gy * nzi * ny;
    } else if (prs && (t == FS_BC_WALL_SLIP || t == FS_BC_WALL_NOSLIP)) {
      // CorrectPresureGradientAtWalls (CorrectGradients.for:34-56)
      ox = (1 - nx * nx) * gx - nx * ny * gy - nx * nz * gz;
      oy = (1 - ny * ny) * gy - ny * nx * gx - ny * nz * gz;
      oz = (1 - nz * nz) * gz - nz * nx * gx - nz * ny * gy;
    }
    double *bg = J.bg[q];
    bg[b] = ox; bg[B + b] = oy; bg[2L * B + b] = oz;
  }
}

// ------------------------------------------------------------ momentum
struct MomArgs {
  int N, F, B;
  const int32_t *ncf, *slot, *fown, *fnbr, *bown, *btype, *cn;
  const double *gf, *sf, *dcfv, *dcf, *gdiff, *tf, *vol;
  const double *bsf, *bfa, *bnf, *bdv, *bgdiff, *btf;
  const double *u, *v, *w, *mdot, *bmdot, *bu, *bv, *bw;
  const double *ug, *vg, *wg, *pg, *bug, *bvg, *bwg;
  const double *mut, *bedif, *drk;      // k-epsilon: mu_t (N), BeDiffCoefficient (B), grad(2/3 rho k) (3N)
  double mu, bleed, urf;
  int gi_scheme, hr_on, conv_scheme, inviscid, relax, simplec;
  // outputs
  double *ac_int, *anb, *bc_int, *effdiv;
  double *ac, *bc, *d1, *d2, *star;
  double *red; int nblk;
  FsTransient tr;                        // unsteady runs (tr.on = 0: steady)
};

// Interior-face part of SolveMomentumX/Y/Z for all three components at once:
// diffusion (AssembleIsotropicDiffusion.for:99-117), transpose diffusion
// (AssembleExplicitDiffusion.for:22-44), bulk viscosity (AssembleBulkViscosity.for:22-44),
// upwind convection + HR deferred correction (AssembleConvection.for:72-88,153-162)
// and the effective divergence (CalculateEffectiveDivergence.for:20-45).
// FluxCf/FluxFf (and so ac, anb) are shared by u, v, w; bc differs.
// TURB: eDiffCoefficient = mu + mu_t (ComputeEffectiveDiffusionCoefficient.for:30-32)
template <bool TURB>
__global__ void __launch_bounds__(FS_BLOCK, FS_MOM_MINB) k_mom_interior(MomArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  const int N = a.N, F = a.F;
  const long N2 = 2L * N, F2 = 2L * F;
  int nc = a.ncf[i];
  const double mu = a.mu;
  // this cell's values stay in registers; the other cell of a face is cn(i,j)
  const double us = a.u[i], vs = a.v[i], ws = a.w[i];
  const double mts = TURB ? a.mut[i] : 0.;
  const double gus[3] = {a.ug[i], a.ug[N + i], a.ug[N2 + i]};
  const double gvs[3] = {a.vg[i], a.vg[N + i], a.vg[N2 + i]};
  const double gws[3] = {a.wg[i], a.wg[N + i], a.wg[N2 + i]};
  double ac = 0., bcu = 0., bcv = 0., bcw = 0., ed = 0.;
  FS_SLOT_PREFETCH(nc, a.slot, a.cn, N, i);
  auto face = [&](int j, int s, int k) {
    int f = s >> 1;
    if (f >= F) { ed = ed + a.bmdot[f - F]; return; }
    const bool nb = s & 1;                 // this cell is the face's neighbour
    double g = a.gf[f], md = a.mdot[f];
    double sx = a.sf[f], sy = a.sf[F + f], sz = a.sf[F2 + f];
    const double uk = a.u[k], vk = a.v[k], wk = a.w[k];
    const double guk[3] = {a.ug[k], a.ug[N + k], a.ug[N2 + k]};
    const double gvk[3] = {a.vg[k], a.vg[N + k], a.vg[N2 + k]};
    const double gwk[3] = {a.wg[k], a.wg[N + k], a.wg[N2 + k]};
    // owner (o) / neighbour (n) values in the face's orientation
    double uo = nb ? uk : us, un = nb ? us : uk;
    double vo = nb ? vk : vs, vn = nb ? vs : vk;
    double wo = nb ? wk : ws, wn = nb ? ws : wk;
    double guo[3], gun[3], gvo[3], gvn[3], gwo[3], gwn[3];
    for (int d = 0; d < 3; d++) {
      guo[d] = nb ? guk[d] : gus[d]; gun[d] = nb ? gus[d] : guk[d];
      gvo[d] = nb ? gvk[d] : gvs[d]; gvn[d] = nb ? gvs[d] : gvk[d];
      gwo[d] = nb ? gwk[d] : gws[d]; gwn[d] = nb ? gws[d] : gwk[d];
    }
    double dx = a.dcfv[f], dy = a.dcfv[F + f], dz = a.dcfv[F2 + f], d = a.dcf[f];
    double ex = dx / d, ey = dy / d, ez = dz / d;
    double fcf = 0., fff = 0., tu = 0., tv = 0., tw = 0.;
    if (!a.inviscid) {
      double gamf;
      if (TURB) {
        const double mtk = a.mut[k];
        gamf = g * (mu + (nb ? mtk : mts)) + (1. - g) * (mu + (nb ? mts : mtk));
      } else {
        gamf = g * mu + (1. - g) * mu;
      }
      double gd = a.gdiff[f];
      double tx = a.tf[f], ty = a.tf[F + f], tz = a.tf[F2 + f];
      double fu[3], fv[3], fw[3];
      face_grad(a.gi_scheme, g, md, uo, un, d, ex, ey, ez, guo[0], guo[1], guo[2], gun[0], gun[1], gun[2], fu[0], fu[1], fu[2]);
      face_grad(a.gi_scheme, g, md, vo, vn, d, ex, ey, ez, gvo[0], gvo[1], gvo[2], gvn[0], gvn[1], gvn[2], fv[0], fv[1], fv[2]);
      face_grad(a.gi_scheme, g, md, wo, wn, d, ex, ey, ez, gwo[0], gwo[1], gwo[2], gwn[0], gwn[1], gwn[2], fw[0], fw[1], fw[2]);
      double fcl = gamf * gd, ffl = -gamf * gd;
      fcf = fcl; fff = ffl;
      tu = fcl * uo + ffl * un + -(gamf * (fu[0] * tx + fu[1] * ty + fu[2] * tz));
      tv = fcl * vo + ffl * vn + -(gamf * (fv[0] * tx + fv[1] * ty + fv[2] * tz));
      tw = fcl * wo + ffl * wn + -(gamf * (fw[0] * tx + fw[1] * ty + fw[2] * tz));
      // transpose term
      tu = tu + -(gamf * (fu[0] * sx + fv[0] * sy + fw[0] * sz));
      tv = tv + -(gamf * (fu[1] * sx + fv[1] * sy + fw[1] * sz));
      tw = tw + -(gamf * (fu[2] * sx + fv[2] * sy + fw[2] * sz));
      // bulk viscosity
      double div = fu[0] + fv[1] + fw[2];
      tu = tu + -(M23 * gamf * div * sx);
      tv = tv + -(M23 * gamf * div * sy);
      tw = tw + -(M23 * gamf * div * sz);
    }
    double cc = fmax(md, 0.), cn_ = -fmax(-md, 0.);
    fcf = fcf + cc; fff = fff + cn_;
    tu = tu + (cc * uo + cn_ * un);
    tv = tv + (cc * vo + cn_ * vn);
    tw = tw + (cc * wo + cn_ * wn);
    if (a.hr_on) {
      tu = tu + hr_flux(a.conv_scheme, a.bleed, md, uo, un, guo, gun, dx, dy, dz);
      tv = tv + hr_flux(a.conv_scheme, a.bleed, md, vo, vn, gvo, gvn, dx, dy, dz);
      tw = tw + hr_flux(a.conv_scheme, a.bleed, md, wo, wn, gwo, gwn, dx, dy, dz);
    }
    if (nb) {
      ac = ac - fff;
      a.anb[(long)j * N + i] = 0. - fcf;
      bcu = bcu + tu; bcv = bcv + tv; bcw = bcw + tw;
      ed = ed - md;
    } else {
      ac = ac + fcf;
      a.anb[(long)j * N + i] = 0. + fff;
      bcu = bcu - tu; bcv = bcv - tv; bcw = bcw - tw;
      ed = ed + md;
    }
  };
  FS_SLOT_LOOP_J(nc, a.slot, a.cn, N, i, face);
  a.ac_int[i] = ac;
  a.bc_int[i] = bcu; a.bc_int[N + i] = bcv; a.bc_int[N2 + i] = bcw;
  a.effdiv[i] = ed;
}

// Boundary faces, element terms, under-relaxation and D of one component:
// AssembleIsotropicDiffusion.for:123-627 (walls/symmetry/inlet), explicit and bulk
// boundary terms, AssembleConvection.for:165-178 + 263-556, AssemblePressureGradient.for,
// AssembleGolbalElementAndFaceFluxes.for:83-98 + 4-30, UnderRelaxation.for:21,
// StoreTheDValues.for:20-48, and the residual partials of CalculateResiduals.
// TURB: boundary faces diffuse with BeDiffCoefficient (wall functions on no-slip
// walls) and FluxTE takes MinusTwoThirdsRhoK (AssembleMinusTwoThirdsRhoK.for:96-110).
template <bool TURB>
__device__ __forceinline__ void mom_finish_cell(const MomArgs &a, int comp, int i, double *ac_o, double *bc_o,
                                                double *d1_o, double *d2_o, double *star_o, double &r, double &acphi) {
  {
    const int N = a.N, F = a.F, B = a.B;
    const long N2 = 2L * N, B2 = 2L * B;
    const double mu = a.mu;
    const double *fi = comp == 0 ? a.u : comp == 1 ? a.v : a.w;
    const double *bfi = comp == 0 ? a.bu : comp == 1 ? a.bv : a.bw;
    const double *bfg = comp == 0 ? a.bug : comp == 1 ? a.bvg : a.bwg;
    double phi = fi[i];
    double ac = a.ac_int[i], bc = a.bc_int[(long)comp * N + i];
    int nc = a.ncf[i];
    for (int j = 0; j < nc; j++) {
      int f = a.slot[(long)j * N + i] >> 1;
      if (f < F) continue;
      int b = f - F, t = a.btype[b];
      double fcf = 0., tf = 0.;
      double bsx = a.bsf[b], bsy = a.bsf[B + b], bsz = a.bsf[B2 + b];
      double bp = bfi[b];
      if (!a.inviscid) {
        double gamf = TURB ? a.bedif[b] : mu;
        if (t == FS_BC_WALL_NOSLIP || t == FS_BC_SYMMETRY) {
          double nx = a.bnf[b], ny = a.bnf[B + b], nz = a.bnf[B2 + b];
          double dN = a.bdv[b] * nx + a.bdv[B + b] * ny + a.bdv[B2 + b] * nz;
          double area = a.bfa[b], fcl, fvl;
          if (t == FS_BC_WALL_NOSLIP) {
            if (comp == 0) {
              fcl = gamf * area * (1. - nx * nx) / dN;
              fvl = -((gamf * area / dN) * (bp * (1. - nx * nx) + (a.v[i] - a.bv[b]) * nx * ny + (a.w[i] - a.bw[b]) * nx * nz));
            } else if (comp == 1) {
              fcl = gamf * area * (1. - ny * ny) / dN;
              fvl = -((gamf * area / dN) * ((a.u[i] - a.bu[b]) * nx * ny + bp * (1. - ny * ny) + (a.w[i] - a.bw[b]) * nz * ny));
            } else {
              fcl = gamf * area * (1. - nz * nz) / dN;
              fvl = -((gamf * area / dN) * ((a.u[i] - a.bu[b]) * nx * nz + (a.v[i] - a.bv[b]) * ny * nz + bp * (1. - nz * nz)));
            }
          } else {
            if (comp == 0) { fcl = 2. * gamf * area * (nx * nx) / dN; fvl = -((-2. * gamf * area / dN) * (a.v[i] * ny + a.w[i] * nz) * nx); }
            else if (comp == 1) { fcl = 2. * gamf * area * (ny * ny) / dN; fvl = -((-2. * gamf * area / dN) * (a.u[i] * nx + a.w[i] * nz) * ny); }
            else { fcl = 2. * gamf * area * (nz * nz) / dN; fvl = -((-2. * gamf * area / dN) * (a.u[i] * nx + a.v[i] * ny) * nz); }
          }
          fcf = fcl;
          tf = fcl * phi + 0. * bp + fvl;
        } else if (fs_is_inlet(t) || t == FS_BC_OUTLET_MASS) {   // :254-300, 507-525
          double fcl = gamf * a.bgdiff[b], ffl = -gamf * a.bgdiff[b];
          double fvl = -(gamf * (bfg[b] * a.btf[b] + bfg[B + b] * a.btf[B + b] + bfg[B2 + b] * a.btf[B2 + b]));
          fcf = fcl;
          tf = fcl * phi + ffl * bp + fvl;
        }
        // transpose (explicit) diffusion, all boundary faces
        double gxc = a.bug[(long)comp * B + b], gyc = a.bvg[(long)comp * B + b], gzc = a.bwg[(long)comp * B + b];
        tf = tf + -(gamf * (gxc * bsx + gyc * bsy + gzc * bsz));
        // bulk viscosity, all boundary faces
        double div = a.bug[b] + a.bvg[B + b] + a.bwg[B2 + b];
        double sc = comp == 0 ? bsx : comp == 1 ? bsy : bsz;
        tf = tf + -(M23 * gamf * div * sc);
      }
      if (fs_is_inlet(t) || t == FS_BC_OUTLET_MASS) {
        double bm = a.bmdot[b];
        double fcl = fmax(bm, 0.), ffl = -fmax(-bm, 0.);
        fcf = fcf + fcl;
        tf = tf + (fcl * phi + ffl * bp);
      } else if (t == FS_BC_OUTLET_FD || fs_is_sp_outlet(t)) {
        double bm = a.bmdot[b];
        double fcl = fmax(bm, 0.), ffl = -fmax(-bm, 0.);
        double fvl = bm * (bfg[b] * a.bdv[b] + bfg[B + b] * a.bdv[B + b] + bfg[B2 + b] * a.bdv[B2 + b]);
        fcf = fcf + fcl;
        tf = tf + (fcl * phi + ffl * bp + fvl);
      }
      ac = ac + fcf;
      bc = bc - tf;
    }
    // element terms: effective divergence (AssembleConvection.for:165-178) and pressure gradient
    double e = a.effdiv[i];
    double fce = fmax(e, 0.0) - e;
    double fve = -(fmax(e, 0.0) * phi);
    double fte = fce * phi + fve;
    if (a.tr.on) transient_term(a.tr, comp, N, i, a.vol[i], phi, fce, fte);   // SolveXMomentumEquation.for:247-251
    fte = fte + a.pg[(long)comp * N + i] * a.vol[i];
    if (TURB) fte = fte + a.drk[(long)comp * N + i] * a.vol[i];
    ac = ac + fce;
    bc = bc - fte;
    if (a.relax) ac = ac / a.urf;
    double V = a.vol[i];
    double d1 = V / ac, d2 = d1;
    if (a.simplec) {
      double sa = ac;
      for (int j = 0; j < nc; j++) sa = sa + a.anb[(long)j * N + i];
      d2 = V / sa;
    }
    ac_o[i] = ac; bc_o[i] = bc; d1_o[i] = d1; d2_o[i] = d2; star_o[i] = phi;
    r = fabs(bc);
    acphi = fabs(ac * phi);
  }
}

template <bool TURB>
__global__ void __launch_bounds__(FS_BLOCK, FS_FACE_MINB) k_mom_finish(MomArgs a, int comp) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double r = 0., acphi = -1.;
  if (i < a.N) mom_finish_cell<TURB>(a, comp, i, a.ac, a.bc, a.d1, a.d2, a.star, r, acphi);
  residual_partials(r, acphi, a.red, a.nblk);
}

// the three components in one launch (the multi-RHS form assembles u, v, w
// from the same fields): a thread finishes its cell for u, v, then w, so the
// cell's slots, coefficients and volume come from cache after the first; the
// residual partials of component c go to red + RED_NQ c nblk
struct MomOut3 {
  double *ac[3], *bc[3], *d1[3], *d2[3], *star[3];
};
template <bool TURB>
__global__ void __launch_bounds__(FS_BLOCK, FS_FACE_MINB) k_mom_finish3(MomArgs a, MomOut3 o) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll 1
  for (int comp = 0; comp < 3; comp++) {
    double r = 0., acphi = -1.;
    double *ac_o = comp == 0 ? o.ac[0] : comp == 1 ? o.ac[1] : o.ac[2];
    double *bc_o = comp == 0 ? o.bc[0] : comp == 1 ? o.bc[1] : o.bc[2];
    double *d1_o = comp == 0 ? o.d1[0] : comp == 1 ? o.d1[1] : o.d1[2];
    double *d2_o = comp == 0 ? o.d2[0] : comp == 1 ? o.d2[1] : o.d2[2];
    double *st_o = comp == 0 ? o.star[0] : comp == 1 ? o.star[1] : o.star[2];
    if (i < a.N) mom_finish_cell<TURB>(a, comp, i, ac_o, bc_o, d1_o, d2_o, st_o, r, acphi);
    residual_partials(r, acphi, a.red + (long)RED_NQ * comp * a.nblk, a.nblk);
  }
}

// ------------------------------------------------------------ continuity
struct ContArgs {
  int N, F, B, msd, relax, gi_scheme;
  double rho, urf;
  const int32_t *ncf, *slot, *fown, *fnbr, *bown, *btype;
  const double *gf, *sf, *dcfv, *dcf;
  const double *u, *v, *w, *p, *us, *vs, *ws, *pg;
  const double *pf;   // pressure of the 'averagecorrected' face gradient (fs_assemble_mdot)
  const double *du1, *dv1, *dw1, *du2, *dv2, *dw2;
  double *mdot, *pcoef, *bmdot;
  const double *bu, *bv, *bw, *bsf;
  const double *rhok, *drk;   // k-epsilon: 2/3 rho k and its gradient (3N), nullptr when laminar
  // pressure outlets
  double *bpcoef, *bu_w, *bv_w, *bw_w;
  double *bpcoefc, *bgd, *bp_w;   // FluxCf of the p' diagonal, geoDiff of resistance faces, p_b (stagnation)
  const double *bp0, *patch;      // p0 per face; per patch: resistance R [0,32), sum of geoDiff [32,64)
  const int32_t *bset;            // patch of each boundary face
  const double *bdir;   // 3B direction of 'specifiedmassflowrate' inlets (nullptr: none)
  const double *bug, *bvg, *bwg, *bdv, *bpg, *bp, *brhok, *bdrk;
  double *ac, *anb, *bc;
  double *red; int nblk;
};

__device__ __forceinline__ double geo_diff(int msd, double du, double dv, double dw, double sx, double sy, double sz,
                                           double ex, double ey, double ez, double cf,
                                           double &tx, double &ty, double &tz) {
  double DuSf = du * sx, DvSf = dv * sy, DwSf = dw * sz, DuEf, DvEf, DwEf;
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
  tx = DuSf - DuEf; ty = DvSf - DvEf; tz = DwSf - DwEf;
  return sqrt(DuEf * DuEf + DvEf * DvEf + DwEf * DwEf) / cf;
}

// Rhie-Chow mdot (AssembleMdotUsingRhieChow.for:554-759) and the p' face
// coefficient rho*geoDiff(D2) (AssemblePressureCorrectionFluxes.for:85-153)
template <bool TURB>
__global__ void __launch_bounds__(FS_BLOCK, FS_FACE_MINB) k_mdot(ContArgs a) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.F) return;
  const int N = a.N, F = a.F;
  const long N2 = 2L * N, F2 = 2L * F;
  int i = a.fown[k], j = a.fnbr[k];
  double g = a.gf[k], g1 = 1. - g;
  double rhof = a.rho;
  double sx = a.sf[k], sy = a.sf[F + k], sz = a.sf[F2 + k];
  double dx = a.dcfv[k], dy = a.dcfv[F + k], dz = a.dcfv[F2 + k], cf = a.dcf[k];
  double ex = dx / cf, ey = dy / cf, ez = dz / cf;
  double du = g * a.du1[i] + g1 * a.du1[j];
  double dv = g * a.dv1[i] + g1 * a.dv1[j];
  double dw = g * a.dw1[i] + g1 * a.dw1[j];
  double ub = g * a.u[i] + g1 * a.u[j], vb = g * a.v[i] + g1 * a.v[j], wb = g * a.w[i] + g1 * a.w[j];
  double fvl = rhof * (ub * sx + vb * sy + wb * sz);
  double tx, ty, tz;
  double gd = geo_diff(a.msd, du, dv, dw, sx, sy, sz, ex, ey, ez, cf, tx, ty, tz);
  double fcl = rhof * gd, ffl = -rhof * gd;
  double pi = a.p[i], pj = a.p[j];
  double gox = a.pg[i], goy = a.pg[N + i], goz = a.pg[N2 + i];
  double gnx = a.pg[j], gny = a.pg[N + j], gnz = a.pg[N2 + j];
  double pfx, pfy, pfz;   // PressGradf (GradientInterpolationSchemeContinuity)
  face_grad(a.gi_scheme, g, a.mdot[k], a.pf[i], a.pf[j], cf, ex, ey, ez, gox, goy, goz, gnx, gny, gnz, pfx, pfy, pfz);
  double pbx = g * gox + g1 * gnx, pby = g * goy + g1 * gny, pbz = g * goz + g1 * gnz;  // PressGradBar ('average')
  fvl = fvl - rhof * (pfx * tx + pfy * ty + pfz * tz);
  fvl = fvl + rhof * (pbx * (du * sx) + pby * (dv * sy) + pbz * (dw * sz));
  if (TURB) {
    // k-epsilon: the 2/3 rho k gradient like the pressure (AssembleMdotUsingRhieChow.for:296-305, 627-634)
    const double ki = a.rhok[i], kj = a.rhok[j];
    const double kox = a.drk[i], koy = a.drk[N + i], koz = a.drk[N2 + i];
    const double knx = a.drk[j], kny = a.drk[N + j], knz = a.drk[N2 + j];
    double rfx, rfy, rfz;
    face_grad(FS_GI_AVERAGECORRECTED, g, a.mdot[k], ki, kj, cf, ex, ey, ez, kox, koy, koz, knx, kny, knz, rfx, rfy, rfz);
    const double rbx = g * kox + g1 * knx, rby = g * koy + g1 * kny, rbz = g * koz + g1 * knz;
    fvl = fvl - rhof * (rfx * tx + rfy * ty + rfz * tz);
    fvl = fvl + rhof * (rbx * (du * sx) + rby * (dv * sy) + rbz * (dw * sz));
    fvl = fvl + fcl * ki + ffl * kj;
  }
  double mold = a.mdot[k];
  if (a.relax) {
    double ms = rhof * ((g * a.us[i] + g1 * a.us[j]) * sx + (g * a.vs[i] + g1 * a.vs[j]) * sy + (g * a.ws[i] + g1 * a.ws[j]) * sz);
    fvl = fvl + (1. - a.urf) * (mold - ms);
  }
  a.mdot[k] = fcl * pi + ffl * pj + fvl;
  // p' coefficient with D2 (SIMPLEC) -- identical to D1 for SIMPLE
  double du2 = g * a.du2[i] + g1 * a.du2[j];
  double dv2 = g * a.dv2[i] + g1 * a.dv2[j];
  double dw2 = g * a.dw2[i] + g1 * a.dw2[j];
  double t2x, t2y, t2z;
  a.pcoef[k] = rhof * geo_diff(a.msd, du2, dv2, dw2, sx, sy, sz, ex, ey, ez, cf, t2x, t2y, t2z);
}

// specified-velocity inlets: Bmdot = rho*Ub.S (AssembleMdotUsingRhieChow.for:2054-2075);
// mass-flow inlets and fully developed outlets: the boundary velocity
__global__ void k_bmdot_inlet(ContArgs a) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.B) return;
  const int t = a.btype[b];
  if (t == FS_BC_OUTLET_FD) {
    // fully developed outlet velocity (AssembleMdotUsingRhieChow.for:2033-2050); k_flow_in_out
    // set the same values just before, unless a Crank-Nicolson extrapolation came in between
    const int i1 = a.bown[b];
    a.bu_w[b] = a.u[i1]; a.bv_w[b] = a.v[i1]; a.bw_w[b] = a.w[i1];
    return;
  }
  const int B = a.B;
  if (t == FS_BC_INLET_MASS) {
    // velocity from the specified Bmdot along the given direction (AssembleMdotUsingRhieChow.for:2077-2100)
    fs_directed_velocity(a.bdir, a.bsf, a.rho, B, b, a.bmdot[b], a.bu_w, a.bv_w, a.bw_w);
    return;
  }
  if (t == FS_BC_OUTLET_MASS) {
    // along the owner's velocity (AssembleMdotUsingRhieChow.for:1999-2031)
    const int i1 = a.bown[b];
    const double u = a.u[i1], v = a.v[i1], w = a.w[i1];
    const double vel = sqrt(u * u + v * v + w * w);
    const double dx = u / (vel + TINY), dy = v / (vel + TINY), dz = w / (vel + TINY);
    const double vm = a.bmdot[b] / (a.rho * (dx * a.bsf[b] + dy * a.bsf[B + b] + dz * a.bsf[2L * B + b]));
    a.bu_w[b] = vm * dx; a.bv_w[b] = vm * dy; a.bw_w[b] = vm * dz;
    return;
  }
  if (t != FS_BC_INLET_VEL) return;
  a.bmdot[b] = a.rho * (a.bu[b] * a.bsf[b] + a.bv[b] * a.bsf[B + b] + a.bw[b] * a.bsf[2L * B + b]);
}

// 'specifiedstaticpressure' outlets: boundary velocity, Rhie-Chow Bmdot
// (AssembleMdotUsingRhieChow.for:1441-1598) and the p' coefficient rho geoDiff(D2)
// (AssemblePressureCorrectionFluxes.for:244-313)
__global__ void k_bmdot_sp(ContArgs a) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.B || !fs_is_pressure(a.btype[b])) return;
  const int N = a.N, B = a.B;
  const long N2 = 2L * N, B2 = 2L * B;
  const int i1 = a.bown[b];
  // static- and stagnation-pressure inlets (:2105-2460): the same flux; velocity from Bmdot
  const bool inlet = fs_is_p_inlet(a.btype[b]);
  const double rhof = a.rho, sx = a.bsf[b], sy = a.bsf[B + b], sz = a.bsf[B2 + b];
  const double dx = a.bdv[b], dy = a.bdv[B + b], dz = a.bdv[B2 + b];
  if (!inlet) {
    a.bu_w[b] = a.u[i1] + (a.bug[b] * dx + a.bug[B + b] * dy + a.bug[B2 + b] * dz);
    a.bv_w[b] = a.v[i1] + (a.bvg[b] * dx + a.bvg[B + b] * dy + a.bvg[B2 + b] * dz);
    a.bw_w[b] = a.w[i1] + (a.bwg[b] * dx + a.bwg[B + b] * dy + a.bwg[B2 + b] * dz);
  }
  const double cf = sqrt(dx * dx + dy * dy + dz * dz);
  const double ex = dx / cf, ey = dy / cf, ez = dz / cf;
  double fvl = rhof * (a.u[i1] * sx + a.v[i1] * sy + a.w[i1] * sz);
  const double du = a.du1[i1], dv = a.dv1[i1], dw = a.dw1[i1];
  double tx, ty, tz;
  const double gd = geo_diff(a.msd, du, dv, dw, sx, sy, sz, ex, ey, ez, cf, tx, ty, tz);
  const double fcl = rhof * gd, ffl = -rhof * gd;
  fvl = fvl - rhof * (a.bpg[b] * tx + a.bpg[B + b] * ty + a.bpg[B2 + b] * tz);
  fvl = fvl + rhof * (a.pg[i1] * (du * sx) + a.pg[N + i1] * (dv * sy) + a.pg[N2 + i1] * (dw * sz));
  if (a.rhok) {
    fvl = fvl - rhof * (a.bdrk[b] * tx + a.bdrk[B + b] * ty + a.bdrk[B2 + b] * tz);
    fvl = fvl + rhof * (a.drk[i1] * (du * sx) + a.drk[N + i1] * (dv * sy) + a.drk[N2 + i1] * (dw * sz));
    fvl = fvl + fcl * a.rhok[i1] + ffl * a.brhok[b];
  }
  if (a.relax) {
    const double ms = rhof * (a.us[i1] * sx + a.vs[i1] * sy + a.ws[i1] * sz);
    fvl = fvl + (1. - a.urf) * (a.bmdot[b] - ms);
  }
  a.bmdot[b] = fcl * a.p[i1] + ffl * a.bp[b] + fvl;
  if (inlet) fs_directed_velocity(a.bdir, a.bsf, rhof, B, b, a.bmdot[b], a.bu_w, a.bv_w, a.bw_w);
  double t2x, t2y, t2z;
  const double gd2 = geo_diff(a.msd, a.du2[i1], a.dv2[i1], a.dw2[i1], sx, sy, sz, ex, ey, ez, cf, t2x, t2y, t2z);
  a.bpcoef[b] = rhof * gd2;
  if (a.btype[b] == FS_BC_OUTLET_RES) a.bgd[b] = gd2;   // geoDiffB (AssemblePressureCorrectionFluxes.for:474)
}

// sum of geoDiff over each 'specifiedresistance' patch (geoDiffSum,
// AssemblePressureCorrectionFluxes.for:400-476), one CTA per patch
struct ResPatches { int n; int s[FS_MAX_PATCHES], start[FS_MAX_PATCHES], cnt[FS_MAX_PATCHES]; };
__global__ void __launch_bounds__(1024) k_res_sum(ResPatches rp, const double *__restrict__ bgd, double *patch) {
  __shared__ double sh[32];
  const int q = blockIdx.x;
  const int b0 = rp.start[q], n = rp.cnt[q];
  double t = 0.;
  for (int j = threadIdx.x; j < n; j += blockDim.x) t = t + bgd[b0 + j];
  t = block_sum(t, sh);
  if (threadIdx.x == 0) patch[FS_MAX_PATCHES + rp.s[q]] = t;
}

// UpdateBoundaryForTotalConditions (TotalConditionsBoundary.for:25-45) and the
// boundary FluxCf of the p' system (AssemblePressureCorrectionFluxes.for:
// 244-313 static, 322-400 average, 476-500 resistance, 585-720 inlets):
// FluxFf stays rho geoDiff; FluxCf is rho geoDiff (1 + (S - geoDiff) R) /
// (1 + R S) on a resistance outlet, Bmdot FluxFf / (Bmdot - FluxFf rho |U_b|^2)
// on a stagnation-pressure inlet after p_b = max(p0 - rho |U_b|^2 / 2, 0)
__global__ void k_pc_bcoef(ContArgs a) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.B) return;
  const int t = a.btype[b];
  if (!fs_is_pressure(t)) return;
  const double ff = a.bpcoef[b];
  double fc = ff;
  if (t == FS_BC_INLET_STAG) {
    const double u = a.bu_w[b], v = a.bv_w[b], w = a.bw_w[b];
    const double vel2 = u * u + v * v + w * w;
    a.bp_w[b] = fmax(a.bp0[b] - 0.5 * a.rho * vel2, 0.);
    const double bm = a.bmdot[b];
    fc = bm * ff / (bm - ff * a.rho * vel2);
  } else if (t == FS_BC_OUTLET_RES) {
    const int s = a.bset[b];
    const double R = a.patch[s], S = a.patch[FS_MAX_PATCHES + s], g = a.bgd[b];
    fc = a.rho * g;
    fc = fc * (1. + (S - g) * R) / (1. + R * S);
  }
  a.bpcoefc[b] = fc;
}

// p' system (AssemblePressureCorrectionFluxes.for + global assembly): ac = sum coef,
// anb = -coef, bc = -(net outflow)
__global__ void __launch_bounds__(FS_BLOCK) k_pc_assemble(ContArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double r = 0.;
  if (i < a.N) {
    const int N = a.N, F = a.F;
    int nc = a.ncf[i];
    double ac = 0., bc = 0.;
    FS_SLOT_PREFETCH(nc, a.slot, a.slot, N, i);
    auto face = [&](int j, int s, int) {
      int f = s >> 1;
      if (f < F) {
        double c = a.pcoef[f], fff = -c, md = a.mdot[f];
        if (s & 1) { ac = ac - fff; a.anb[(long)j * N + i] = 0. - c; bc = bc + md; }
        else { ac = ac + c; a.anb[(long)j * N + i] = 0. + fff; bc = bc - md; }
      } else {
        ac = ac + (fs_is_pressure(a.btype[f - F]) ? a.bpcoefc[f - F] : 0.);
        bc = bc - a.bmdot[f - F];
      }
    };
    FS_SLOT_LOOP_J(nc, a.slot, a.slot, N, i, face);
    ac = ac + 0.; bc = bc - 0.;
    a.ac[i] = ac; a.bc[i] = bc;
    r = fabs(bc);
  }
  residual_partials(r, 0., a.red, a.nblk);
}

// ------------------------------------------------------------ corrections
struct CorrArgs {
  int N, F, B, ref_cell, set_ref;
  double urfp;
  const int32_t *ncf, *slot, *fown, *fnbr, *bown, *btype;
  const double *bdv, *bnf, *pcoef, *du2, *dv2, *dw2, *pcg, *bpg;
  double *u, *v, *w, *p, *pc, *mdot, *bp, *bpc, *bu, *bv, *bw, *bmdot;
  const double *bpcoef;
  double *red; int64_t *redi; int nblk; double *rb;
  const double *vol; double drhodt; int unsteady;   // + d rho/dt V in unsteady runs
  const double *bdir, *bsf; double rho;             // inlets with a given velocity direction
};

// UpdateBoundaryPressureCorrection (UpdatePressureCorrectionAtBoundaries.for):
// 0 at static pressures (:85-90, 126-143), the owner's elsewhere; on a
// stagnation-pressure inlet -rho |U_b|^2 FluxFf p'_C / (Bmdot - FluxFf rho |U_b|^2)
// (:97-112); resistance outlets are set by k_res_pc
__global__ void k_bpc(CorrArgs a) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.B) return;
  const int t = a.btype[b];
  if (t == FS_BC_OUTLET_RES) return;
  if (t == FS_BC_INLET_STAG) {
    const double gd = a.bpcoef[b];
    const double u = a.bu[b], v = a.bv[b], w = a.bw[b];
    const double vel2 = u * u + v * v + w * w;
    a.bpc[b] = -a.rho * vel2 * gd * a.pc[a.bown[b]] / (a.bmdot[b] - gd * a.rho * vel2);
    return;
  }
  a.bpc[b] = fs_pc_dirichlet(t) ? 0. : a.pc[a.bown[b]];
}
// 'specifiedresistance' outlets (UpdatePressureCorrectionAtBoundaries.for:144-175):
// p'_b = R sum(geoDiff p'_C) / (1 + R sum geoDiff) on every face of the patch
struct ResPatchesC { int n; int s[FS_MAX_PATCHES], start[FS_MAX_PATCHES], cnt[FS_MAX_PATCHES]; };
__global__ void __launch_bounds__(1024) k_res_pc(ResPatchesC rp, const double *__restrict__ bgd,
                                                 const int32_t *__restrict__ bown, const double *__restrict__ pc,
                                                 const double *__restrict__ patch, double *bpc) {
  __shared__ double sh[32];
  __shared__ double val;
  const int q = blockIdx.x;
  const int b0 = rp.start[q], n = rp.cnt[q], s = rp.s[q];
  double t = 0.;
  for (int j = threadIdx.x; j < n; j += blockDim.x) t = t + bgd[b0 + j] * pc[bown[b0 + j]];
  t = block_sum(t, sh);
  if (threadIdx.x == 0) {
    const double R = patch[s], S = patch[FS_MAX_PATCHES + s];
    val = R * t / (1. + R * S);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += blockDim.x) bpc[b0 + j] = val;
}
// CorrectPressure (CorrectPressure.for:21-42)
__global__ void k_corr_p(CorrArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  double rpc = (a.ref_cell >= 0) ? a.pc[a.ref_cell] : 0.;
  if (a.set_ref) rpc = 0.;
  a.p[i] = a.p[i] + a.urfp * (a.pc[i] - rpc);
}
// CorrectVelocity (CorrectMdotandVelocity.for:773-779)
__global__ void k_corr_u(CorrArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  const int N = a.N;
  a.u[i] = a.u[i] - a.du2[i] * a.pcg[i];
  a.v[i] = a.v[i] - a.dv2[i] * a.pcg[N + i];
  a.w[i] = a.w[i] - a.dw2[i] * a.pcg[2L * N + i];
}
// Correctmdot (CorrectMdotandVelocity.for:55-63)
__global__ void k_corr_mdot(CorrArgs a) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.F) return;
  double c = a.pcoef[k];
  a.mdot[k] = a.mdot[k] + c * a.pc[a.fown[k]] + (-c) * a.pc[a.fnbr[k]];
}
// UpdateBoundaryPressure (CorrectPressure.for:49-190), UpdateSymmetry
// (SymmetryAndAxisBoundary.for:4-33), UpdateSlipWallBoundary (SlipWallBoundary.for:4)
__global__ void k_bcorr(CorrArgs a) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.B) return;
  const int B = a.B;
  const long B2 = 2L * B;
  int t = a.btype[b], i1 = a.bown[b];
  if (fs_is_pressure(t)) {
    // CorrectBoundarymdot (CorrectMdotandVelocity.for:264-280; inlets :180-205, the velocity
    // again from Bmdot); the static pressure stays (CorrectPressure.for:146-150, 162-166)
    const int N = a.N;
    a.bmdot[b] = a.bmdot[b] - a.bpcoef[b] * (a.bpc[b] - a.pc[i1]);
    if (fs_is_p_inlet(t)) {
      fs_directed_velocity(a.bdir, a.bsf, a.rho, B, b, a.bmdot[b], a.bu, a.bv, a.bw);
    } else {
      a.bu[b] = a.bu[b] - a.du2[i1] * a.pcg[i1];
      a.bv[b] = a.bv[b] - a.dv2[i1] * a.pcg[N + i1];
      a.bw[b] = a.bw[b] - a.dw2[i1] * a.pcg[2L * N + i1];
    }
    if (t == FS_BC_OUTLET_ASP) a.bp[b] = a.p[i1];   // CorrectPressure.for:169-176; k_avg_pressure shifts it
    if (t == FS_BC_OUTLET_RES || t == FS_BC_INLET_STAG) {   // CorrectPressure.for:152-160, 206-214
      double rpc = (a.ref_cell >= 0) ? a.pc[a.ref_cell] : 0.;
      if (a.set_ref) rpc = 0.;
      a.bp[b] = a.bp[b] + a.urfp * (a.bpc[b] - rpc);
    }
  } else if (t == FS_BC_WALL_SLIP || t == FS_BC_WALL_NOSLIP || t == FS_BC_SYMMETRY) {
    a.bp[b] = a.p[i1] + a.bpg[b] * a.bdv[b] + a.bpg[B + b] * a.bdv[B + b] + a.bpg[B2 + b] * a.bdv[B2 + b];
  } else {
    double rpc = (a.ref_cell >= 0) ? a.pc[a.ref_cell] : 0.;
    if (a.set_ref) rpc = 0.;
    a.bp[b] = a.bp[b] + a.urfp * (a.bpc[b] - rpc);
    if (t == FS_BC_INLET_MASS || t == FS_BC_OUTLET_MASS) {   // CorrectBoundarymdot: the velocity only (:165-175, 354-364)
      const int N = a.N;
      a.bu[b] = a.bu[b] - a.du2[i1] * a.pcg[i1];
      a.bv[b] = a.bv[b] - a.dv2[i1] * a.pcg[N + i1];
      a.bw[b] = a.bw[b] - a.dw2[i1] * a.pcg[2L * N + i1];
    }
  }
  if (t == FS_BC_SYMMETRY || t == FS_BC_WALL_SLIP) {
    double nx = a.bnf[b], ny = a.bnf[B + b], nz = a.bnf[B2 + b];
    double q = a.u[i1] * nx + a.v[i1] * ny + a.w[i1] * nz;
    a.bu[b] = a.u[i1] - q * nx; a.bv[b] = a.v[i1] - q * ny; a.bw[b] = a.w[i1] - q * nz;
  }
}

// 'specifiedaveragestaticpressure' outlets (CorrectPressure.for:178-203): the
// face pressures (the owners', set by k_bcorr) shifted so that their area
// average is AverageOutletPressure; one CTA per patch, fixed-order sums
struct AvgPatch { int n; int start[FS_MAX_PATCHES], cnt[FS_MAX_PATCHES]; double target[FS_MAX_PATCHES]; };
__global__ void __launch_bounds__(1024) k_avg_pressure(AvgPatch ap, const double *__restrict__ bfa, double *bp) {
  __shared__ double sh[32];
  __shared__ double shift;
  const int q = blockIdx.x;
  if (q >= ap.n) return;
  const int b0 = ap.start[q], n = ap.cnt[q];
  double s = 0., ar = 0.;
  for (int j = threadIdx.x; j < n; j += blockDim.x) { s = s + bfa[b0 + j] * bp[b0 + j]; ar = ar + bfa[b0 + j]; }
  s = block_sum(s, sh);
  ar = block_sum(ar, sh);
  if (threadIdx.x == 0) shift = ap.target[q] - s / (ar + 1.0e-15);
  __syncthreads();
  const double d = shift;
  for (int j = threadIdx.x; j < n; j += blockDim.x) bp[b0 + j] = bp[b0 + j] + d;
}

// mass imbalance per cell (CalculateContinuityResiduals.for:130-183): partial sums,
// max |m| and the largest index attaining it (iMaxImbalance)
__global__ void __launch_bounds__(FS_BLOCK) k_mass_imbalance(CorrArgs a) {
  __shared__ double sh[32];
  __shared__ int64_t shi[FS_BLOCK];
  __shared__ double shm[FS_BLOCK];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double m = 0.;
  if (i < a.N) {
    const int N = a.N, F = a.F;
    int nc = a.ncf[i];
    for (int j = 0; j < nc; j++) {
      int s = a.slot[(long)j * N + i];
      int f = s >> 1;
      if (f < F) m = (s & 1) ? m - a.mdot[f] : m + a.mdot[f];
      else m = m + a.bmdot[f - F];
    }
    if (a.unsteady) m = m + a.drhodt * a.vol[i];   // CalculateContinuityResiduals.for:159-170
  }
  double s0 = block_sum(m, sh);
  double s1 = block_sum(fabs(m), sh);
  double s2 = block_sum(m * m, sh);
  double am = (i < a.N) ? fabs(m) : -1.;
  shm[threadIdx.x] = am; shi[threadIdx.x] = (i < a.N) ? i : -1;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      double x = shm[threadIdx.x], y = shm[threadIdx.x + o];
      int64_t ix = shi[threadIdx.x], iy = shi[threadIdx.x + o];
      if (y > x || (y == x && iy > ix)) { shm[threadIdx.x] = y; shi[threadIdx.x] = iy; }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    a.red[RED_SUM0 * a.nblk + blockIdx.x] = s0;
    a.red[RED_SUM1 * a.nblk + blockIdx.x] = s1;
    a.red[RED_SUM2 * a.nblk + blockIdx.x] = s2;
    a.red[RED_MAX0 * a.nblk + blockIdx.x] = shm[0];
    a.redi[blockIdx.x] = shi[0];
  }
}

// mdot_in_dev: inlet mass flow on the device (nullptr: no inlet)
__global__ void k_mass_final(CorrArgs a, const double *mdot_in_dev) {
  __shared__ double sh[32];
  __shared__ int64_t shi[1024];
  __shared__ double shm[1024];
  double s0 = 0., s1 = 0., s2 = 0., mx = -1.; int64_t im = -1;
  for (int b = threadIdx.x; b < a.nblk; b += blockDim.x) {
    s0 += a.red[RED_SUM0 * a.nblk + b];
    s1 += a.red[RED_SUM1 * a.nblk + b];
    s2 += a.red[RED_SUM2 * a.nblk + b];
    double y = a.red[RED_MAX0 * a.nblk + b]; int64_t iy = a.redi[b];
    if (y > mx || (y == mx && iy > im)) { mx = y; im = iy; }
  }
  s0 = block_sum(s0, sh); s1 = block_sum(s1, sh); s2 = block_sum(s2, sh);
  shm[threadIdx.x] = mx; shi[threadIdx.x] = im;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      double x = shm[threadIdx.x], y = shm[threadIdx.x + o];
      int64_t ix = shi[threadIdx.x], iy = shi[threadIdx.x + o];
      if (y > x || (y == x && iy > ix)) { shm[threadIdx.x] = y; shi[threadIdx.x] = iy; }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double mdot_in = mdot_in_dev ? *mdot_in_dev : 0.;
    double mxv = shm[0] < 0. ? 0. : shm[0];
    a.rb[RB_ABS + 4] = s1;
    a.rb[RB_MAX + 4] = mxv;
    a.rb[RB_RMS + 4] = sqrt(s2 / a.N);
    a.rb[RB_SCL + 4] = (mdot_in == 0.) ? 0. : mxv / fabs(mdot_in);
    a.rb[RB_OVERALL] = s0;
    a.rb[RB_IMAX] = (double)shi[0];
  }
}

// inlet mass flow: one CTA over the inlet patches' face ranges, strided
// per-thread sums then a fixed tree (deterministic)
struct InletRanges { int n; int start[FS_MAX_PATCHES], cnt[FS_MAX_PATCHES]; };
__global__ void k_sum_inlet(InletRanges r, const double *bmdot, double *out) {
  __shared__ double sh[32];
  double s = 0.;
  for (int q = 0; q < r.n; q++)
    for (int j = threadIdx.x; j < r.cnt[q]; j += blockDim.x) s += bmdot[r.start[q] + j];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) *out = s;
}

}  // namespace

// ======================================================================
// host drivers
// ======================================================================
// dynamic shared memory of a k_gg_corr<nf> launch (the staged window)
static size_t gg_smem(int nf) { return FS_GG_STAGE > 0 ? sizeof(double) * 4 * nf * GG_WIN : 0; }

int fs_gradient_dev(fs_ctx *ctx, int nfld, const int *vars, const double *const *phi,
                    const double *const *bphi, double *const *g, double *const *bg,
                    const int *method, const int *niter) {
  const int N = ctx->N, F = ctx->F, B = ctx->B;
  if (FS_GG_STAGE > 0) {   // windows above 48 KB: a per-function attribute, shared by every context
    static bool attr = false;
    if (!attr) {
      const void *fns[4] = {(const void *)k_gg_corr<1>, (const void *)k_gg_corr<2>, (const void *)k_gg_corr<3>,
                            (const void *)k_gg_corr<4>};
      for (int q = 0; q < 4; q++)
        FS_CK(cudaFuncSetAttribute(fns[q], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gg_smem(q + 1)));
      attr = true;
    }
  }
  int passes[4], maxp = 0;
  for (int q = 0; q < nfld; q++) {
    passes[q] = 1 + (method[q] == 2 ? niter[q] : 0);
    if (method[q] != 1 && method[q] != 2) { ctx->err = "only MethodCalcGradient 1 and 2 are implemented"; return FS_E_UNSUPPORTED; }
    maxp = passes[q] > maxp ? passes[q] : maxp;
  }
  // pass p of field q writes g if (passes-1-p) is even, else the scratch buffer
  for (int pidx = 0; pidx < maxp; pidx++) {
    GradJob J{};
    int n = 0;
    for (int q = 0; q < nfld; q++) {
      if (pidx >= passes[q]) continue;
      double *tmp = ctx->gtmp + 3L * N * q;
      bool to_final = ((passes[q] - 1 - pidx) % 2) == 0;
      J.phi[n] = phi[q]; J.bphi[n] = bphi[q];
      J.out[n] = to_final ? g[q] : tmp;
      J.in[n] = to_final ? tmp : g[q];
      n++;
    }
    J.nfld = n;
#define FS_GG_LAUNCH(NFV)                                                                                           \
  do {                                                                                                              \
    if (pidx == 0)                                                                                                  \
      k_gg0<NFV><<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(J, N, F, B, ctx->ncf, ctx->slot, ctx->cn, ctx->gf, ctx->sf,  \
                                                       ctx->bsf, ctx->vol);                                         \
    else                                                                                                            \
      k_gg_corr<NFV><<<fs_grid(N), FS_BLOCK, gg_smem(NFV), ctx->st>>>(J, N, F, B, ctx->ncf, ctx->slot, ctx->cn,     \
                                                                     ctx->gf, ctx->sf, ctx->dfp, ctx->bsf, ctx->vol); \
  } while (0)
    switch (n) {
    case 1: FS_GG_LAUNCH(1); break;
    case 2: FS_GG_LAUNCH(2); break;
    case 3: FS_GG_LAUNCH(3); break;
    default: FS_GG_LAUNCH(4); break;
    }
#undef FS_GG_LAUNCH
    FS_LAUNCH_CHECK();
  }
  if (B) {
    BGradJob BJ{};
    BJ.nfld = nfld;
    for (int q = 0; q < nfld; q++) { BJ.var[q] = vars[q]; BJ.g[q] = g[q]; BJ.bg[q] = bg[q]; }
    k_bgrad<<<fs_grid(B), FS_BLOCK, 0, ctx->st>>>(BJ, N, B, ctx->bown, ctx->btype, ctx->bnf, ctx->bnzii);
    FS_LAUNCH_CHECK();
  }
  return FS_OK;
}

static MomArgs mom_args(fs_ctx *ctx) {
  MomArgs a{};
  const fs_case &c = ctx->cfg;
  a.N = ctx->N; a.F = ctx->F; a.B = ctx->B;
  a.tr = fs_transient_args(ctx);
  a.ncf = ctx->ncf; a.slot = ctx->slot; a.fown = ctx->fown; a.fnbr = ctx->fnbr; a.bown = ctx->bown; a.btype = ctx->btype;
  a.cn = ctx->cn;
  a.gf = ctx->gf; a.sf = ctx->sf; a.dcfv = ctx->dcfv; a.dcf = ctx->dcf; a.gdiff = ctx->gdiff; a.tf = ctx->tf; a.vol = ctx->vol;
  a.bsf = ctx->bsf; a.bfa = ctx->bfa; a.bnf = ctx->bnf; a.bdv = ctx->bdv; a.bgdiff = ctx->bgdiff; a.btf = ctx->btf;
  a.u = ctx->u; a.v = ctx->v; a.w = ctx->w; a.mdot = ctx->mdot; a.bmdot = ctx->bmdot; a.bu = ctx->bu; a.bv = ctx->bv; a.bw = ctx->bw;
  a.ug = ctx->ug; a.vg = ctx->vg; a.wg = ctx->wg; a.pg = ctx->pg; a.bug = ctx->bug; a.bvg = ctx->bvg; a.bwg = ctx->bwg;
  a.mu = c.mu; a.bleed = c.bleed; a.urf = c.urf_momentum;
  fs_turb_momentum_ptrs(ctx, &a.mut, &a.bedif, &a.drk);
  a.gi_scheme = c.grad_interp_mom;
  a.hr_on = (c.hr_framework == FS_HR_TVD && ctx->nIter >= c.niter_start_hr && c.conv_scheme != FS_TVD_UPWIND) ? 1 : 0;
  a.conv_scheme = c.conv_scheme; a.inviscid = c.inviscid; a.relax = c.relax_momentum; a.simplec = c.algorithm == FS_SIMPLEC;
  a.ac_int = ctx->ac_int; a.anb = ctx->anb; a.bc_int = ctx->bc_int; a.effdiv = ctx->effdiv;
  a.ac = ctx->ac; a.bc = ctx->bc; a.red = ctx->red; a.nblk = fs_grid(ctx->N);
  return a;
}

// SolveMomentumX/Y/Z up to (not including) SolveEquation
int fs_momentum_assemble(fs_ctx *ctx, int comp) { return fs_momentum_assemble_to(ctx, comp, ctx->ac, ctx->bc); }

static int mom_prologue(fs_ctx *ctx);

// u, v and w into ac3/bc3 (the multi-RHS form): the same kernels as three
// fs_momentum_assemble_to calls, with the three finishing launches as one
// (k_mom_finish3) when no k-epsilon wall treatment runs between them
int fs_momentum_assemble3(fs_ctx *ctx) {
  const int N = ctx->N;
  if (ctx->turb) {
    for (int c = 0; c < 3; c++) {
      int rc = fs_momentum_assemble_to(ctx, c, ctx->ac3 + (size_t)c * N, ctx->bc3 + (size_t)c * N);
      if (rc) return rc;
    }
    return FS_OK;
  }
  int rc = mom_prologue(ctx);
  if (rc) return rc;
  MomArgs a = mom_args(ctx);
  MomOut3 o;
  double *d1[3] = {ctx->du1, ctx->dv1, ctx->dw1}, *d2[3] = {ctx->du2, ctx->dv2, ctx->dw2};
  double *st[3] = {ctx->us, ctx->vs, ctx->ws};
  for (int c = 0; c < 3; c++) {
    o.ac[c] = ctx->ac3 + (size_t)c * N; o.bc[c] = ctx->bc3 + (size_t)c * N;
    o.d1[c] = d1[c]; o.d2[c] = d2[c]; o.star[c] = st[c];
  }
  k_mom_finish3<false><<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(a, o);
  FS_LAUNCH_CHECK();
  for (int c = 0; c < 3; c++) {
    k_residual_final<<<1, 1024, 0, ctx->st>>>(ctx->red + (size_t)RED_NQ * c * a.nblk, a.nblk, N, c, ctx->resblk);
    FS_LAUNCH_CHECK();
  }
  return FS_OK;
}

// the same, writing the component's ac/bc to the given arrays
// gradients of u, v, w, p and the fused interior-face assembly of the three
// components (the part of the X-momentum call that the Y and Z calls reuse)
static int mom_prologue(fs_ctx *ctx) {
  const fs_case &c = ctx->cfg;
  const int N = ctx->N;
  {
    int vars[4] = {FS_VAR_U, FS_VAR_V, FS_VAR_W, FS_VAR_P};
    const double *phi[4] = {ctx->u, ctx->v, ctx->w, ctx->p};
    const double *bphi[4] = {ctx->bu, ctx->bv, ctx->bw, ctx->bp};
    double *g[4] = {ctx->ug, ctx->vg, ctx->wg, ctx->pg};
    double *bg[4] = {ctx->bug, ctx->bvg, ctx->bwg, ctx->bpg};
    int meth[4] = {c.method_grad_mom, c.method_grad_mom, c.method_grad_mom, c.method_grad_cont};
    int nit[4] = {c.niter_grad_mom, c.niter_grad_mom, c.niter_grad_mom, c.niter_grad_cont};
    int rc = fs_gradient_dev(ctx, 4, vars, phi, bphi, g, bg, meth, nit);
    if (rc) return rc;
    // 'cranknicolson1': the pressure PressGradf is interpolated from here on
    // (SolveXMomentumEquation.for:214-217), kept for the AssembleMdot after an extrapolation
    if (ctx->p_mx) FS_CK(cudaMemcpyAsync(ctx->p_mx, ctx->p, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->st));
    if (ctx->turb && (rc = fs_turb_rhok_gradient(ctx))) return rc;
    MomArgs a = mom_args(ctx);
    if (ctx->turb) k_mom_interior<true><<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(a);
    else k_mom_interior<false><<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(a);
    FS_LAUNCH_CHECK();
  }
  return FS_OK;
}

int fs_momentum_assemble_to(fs_ctx *ctx, int comp, double *ac_out, double *bc_out) {
  const fs_case &c = ctx->cfg;
  const int N = ctx->N;
  if (comp == 0) {
    int rc = mom_prologue(ctx);
    if (rc) return rc;
  }
  if (ctx->turb && !c.inviscid) {
    int rc = fs_turb_wall_functions(ctx);
    if (rc) return rc;
  }
  MomArgs a = mom_args(ctx);
  a.ac = ac_out; a.bc = bc_out;
  a.d1 = comp == 0 ? ctx->du1 : comp == 1 ? ctx->dv1 : ctx->dw1;
  a.d2 = comp == 0 ? ctx->du2 : comp == 1 ? ctx->dv2 : ctx->dw2;
  a.star = comp == 0 ? ctx->us : comp == 1 ? ctx->vs : ctx->ws;
  if (ctx->turb) k_mom_finish<true><<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(a, comp);
  else k_mom_finish<false><<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(a, comp);
  FS_LAUNCH_CHECK();
  k_residual_final<<<1, 1024, 0, ctx->st>>>(ctx->red, a.nblk, N, comp, ctx->resblk);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

static ContArgs cont_args(fs_ctx *ctx) {
  ContArgs a{};
  const fs_case &c = ctx->cfg;
  a.N = ctx->N; a.F = ctx->F; a.B = ctx->B; a.msd = c.method_decompose_s; a.relax = c.relax_momentum;
  a.gi_scheme = c.grad_interp_cont; a.rho = c.rho; a.urf = c.urf_momentum;
  a.ncf = ctx->ncf; a.slot = ctx->slot; a.fown = ctx->fown; a.fnbr = ctx->fnbr; a.bown = ctx->bown; a.btype = ctx->btype;
  a.gf = ctx->gf; a.sf = ctx->sf; a.dcfv = ctx->dcfv; a.dcf = ctx->dcf;
  a.u = ctx->u; a.v = ctx->v; a.w = ctx->w; a.p = ctx->p; a.us = ctx->us; a.vs = ctx->vs; a.ws = ctx->ws; a.pg = ctx->pg;
  a.pf = ctx->p;
  a.du1 = ctx->du1; a.dv1 = ctx->dv1; a.dw1 = ctx->dw1; a.du2 = ctx->du2; a.dv2 = ctx->dv2; a.dw2 = ctx->dw2;
  a.mdot = ctx->mdot; a.pcoef = ctx->pcoef; a.bmdot = ctx->bmdot;
  a.bu = ctx->bu; a.bv = ctx->bv; a.bw = ctx->bw; a.bsf = ctx->bsf;
  fs_turb_rhok_ptrs(ctx, &a.rhok, &a.drk);
  fs_turb_brhok_ptrs(ctx, &a.brhok, &a.bdrk);
  a.bpcoef = ctx->bpcoef; a.bu_w = ctx->bu; a.bv_w = ctx->bv; a.bw_w = ctx->bw; a.bdir = ctx->bdir;
  a.bpcoefc = ctx->bpcoefc; a.bgd = ctx->bgd; a.bp_w = ctx->bp; a.bp0 = ctx->bp0; a.patch = ctx->d_patch;
  a.bset = ctx->d_bset;
  a.bug = ctx->bug; a.bvg = ctx->bvg; a.bwg = ctx->bwg; a.bdv = ctx->bdv; a.bpg = ctx->bpg; a.bp = ctx->bp;
  a.ac = ctx->ac; a.anb = ctx->anb; a.bc = ctx->bc; a.red = ctx->red; a.nblk = fs_grid(ctx->N);
  return a;
}

// AssembleMdot (AssembleMdotUsingRhieChow.for:262-759, 1441-1598, 2033-2075).
// p_face: the pressure whose 'averagecorrected' face gradient PressGradf
// enters (the X-momentum solve interpolated it, SolveXMomentumEquation.for:214-217);
// the current pressure, except after a Crank-Nicolson extrapolation.
int fs_assemble_mdot(fs_ctx *ctx, const double *p_face) {
  const int F = ctx->F, B = ctx->B;
  ContArgs a = cont_args(ctx);
  a.pf = p_face;
  if (F) {
    if (a.rhok) k_mdot<true><<<fs_grid(F), FS_BLOCK, 0, ctx->st>>>(a);
    else k_mdot<false><<<fs_grid(F), FS_BLOCK, 0, ctx->st>>>(a);
    FS_LAUNCH_CHECK();
  }
  if (B) { k_bmdot_inlet<<<fs_grid(B), FS_BLOCK, 0, ctx->st>>>(a); FS_LAUNCH_CHECK(); }
  if (B && ctx->has_sp) { k_bmdot_sp<<<fs_grid(B), FS_BLOCK, 0, ctx->st>>>(a); FS_LAUNCH_CHECK(); }
  return FS_OK;
}

// SolveContinuity up to (not including) SolveEquation
int fs_continuity_assemble(fs_ctx *ctx) {
  const int N = ctx->N, F = ctx->F, B = ctx->B;
  FS_CK(cudaMemsetAsync(ctx->pc, 0, sizeof(double) * N, ctx->st));   // InitializePressureCorrection
  int rc = fs_flow_in_out(ctx);                                        // FlowIn, FlowOut, AdjustFlow
  if (rc) return rc;
  rc = fs_assemble_mdot(ctx, ctx->p);
  if (rc) return rc;
  ContArgs a = cont_args(ctx);
  if (ctx->has_res) {
    ResPatches rp{};
    for (int s = 0; s < ctx->NS; s++)
      if (ctx->cfg.patch_type[s] == FS_BC_OUTLET_RES) {
        rp.s[rp.n] = s; rp.start[rp.n] = ctx->h_bset_start[s]; rp.cnt[rp.n] = ctx->h_bset_n[s]; rp.n++;
      }
    k_res_sum<<<rp.n, 1024, 0, ctx->st>>>(rp, ctx->bgd, ctx->d_patch);
    FS_LAUNCH_CHECK();
  }
  if (B && ctx->has_sp) { k_pc_bcoef<<<fs_grid(B), FS_BLOCK, 0, ctx->st>>>(a); FS_LAUNCH_CHECK(); }
  k_pc_assemble<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(a);
  FS_LAUNCH_CHECK();
  k_residual_final<<<1, 1024, 0, ctx->st>>>(ctx->red, a.nblk, N, 3, ctx->resblk);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

static CorrArgs corr_args(fs_ctx *ctx) {
  CorrArgs a{};
  const fs_case &c = ctx->cfg;
  a.N = ctx->N; a.F = ctx->F; a.B = ctx->B; a.ref_cell = c.ref_pressure_cell; a.set_ref = c.set_reference_pressure;
  a.urfp = c.urf_pressure;
  a.ncf = ctx->ncf; a.slot = ctx->slot; a.fown = ctx->fown; a.fnbr = ctx->fnbr; a.bown = ctx->bown; a.btype = ctx->btype;
  a.bdv = ctx->bdv; a.bnf = ctx->bnf; a.pcoef = ctx->pcoef; a.du2 = ctx->du2; a.dv2 = ctx->dv2; a.dw2 = ctx->dw2;
  a.pcg = ctx->pcg; a.bpg = ctx->bpg;
  a.u = ctx->u; a.v = ctx->v; a.w = ctx->w; a.p = ctx->p; a.pc = ctx->pc; a.mdot = ctx->mdot; a.bp = ctx->bp; a.bpc = ctx->bpc;
  a.bu = ctx->bu; a.bv = ctx->bv; a.bw = ctx->bw; a.bmdot = ctx->bmdot; a.bpcoef = ctx->bpcoef;
  a.red = ctx->red; a.redi = ctx->redi; a.nblk = fs_grid(ctx->N); a.rb = ctx->resblk;
  a.vol = ctx->vol; a.unsteady = c.unsteady; a.drhodt = c.unsteady ? fs_drhodt(ctx) : 0.;
  a.bdir = ctx->bdir; a.bsf = ctx->bsf; a.rho = c.rho;
  return a;
}

// SolveContinuity after SolveEquation: corrections, residuals, symmetry update
int fs_continuity_correct(fs_ctx *ctx) {
  const int N = ctx->N, F = ctx->F, B = ctx->B;
  const fs_case &c = ctx->cfg;
  CorrArgs a = corr_args(ctx);
  if (B) { k_bpc<<<fs_grid(B), FS_BLOCK, 0, ctx->st>>>(a); FS_LAUNCH_CHECK(); }
  if (ctx->has_res) {
    ResPatchesC rp{};
    for (int s = 0; s < ctx->NS; s++)
      if (c.patch_type[s] == FS_BC_OUTLET_RES) {
        rp.s[rp.n] = s; rp.start[rp.n] = ctx->h_bset_start[s]; rp.cnt[rp.n] = ctx->h_bset_n[s]; rp.n++;
      }
    k_res_pc<<<rp.n, 1024, 0, ctx->st>>>(rp, ctx->bgd, ctx->bown, ctx->pc, ctx->d_patch, ctx->bpc);
    FS_LAUNCH_CHECK();
  }
  k_corr_p<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(a);
  FS_LAUNCH_CHECK();
  int var = FS_VAR_PC, meth = c.method_grad_cont, nit = c.niter_grad_cont;
  const double *phi = ctx->pc, *bphi = ctx->bpc;
  double *g = ctx->pcg, *bg = ctx->bpcg;
  int rc = fs_gradient_dev(ctx, 1, &var, &phi, &bphi, &g, &bg, &meth, &nit);
  if (rc) return rc;
  k_corr_u<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(a);
  FS_LAUNCH_CHECK();
  if (F) { k_corr_mdot<<<fs_grid(F), FS_BLOCK, 0, ctx->st>>>(a); FS_LAUNCH_CHECK(); }
  if (B) { k_bcorr<<<fs_grid(B), FS_BLOCK, 0, ctx->st>>>(a); FS_LAUNCH_CHECK(); }
  AvgPatch ap{};
  for (int s = 0; s < ctx->NS; s++)
    if (c.patch_type[s] == FS_BC_OUTLET_ASP) {
      ap.start[ap.n] = ctx->h_bset_start[s]; ap.cnt[ap.n] = ctx->h_bset_n[s]; ap.target[ap.n] = c.patch_pressure[s]; ap.n++;
    }
  if (ap.n) { k_avg_pressure<<<ap.n, 1024, 0, ctx->st>>>(ap, ctx->bfa, ctx->bp); FS_LAUNCH_CHECK(); }
  k_mass_imbalance<<<a.nblk, FS_BLOCK, 0, ctx->st>>>(a);
  FS_LAUNCH_CHECK();
  InletRanges ir{};
  for (int s = 0; s < ctx->NS; s++)
    if (fs_is_inlet(c.patch_type[s])) { ir.start[ir.n] = ctx->h_bset_start[s]; ir.cnt[ir.n] = ctx->h_bset_n[s]; ir.n++; }
  double *d_in = nullptr;
  if (ir.n) {
    // inlet mass flow, used only through ResorScaled(5); stays on the device
    d_in = ctx->resblk + RB_MDOTIN;
    k_sum_inlet<<<1, 1024, 0, ctx->st>>>(ir, ctx->bmdot, d_in);
    FS_LAUNCH_CHECK();
  }
  k_mass_final<<<1, 1024, 0, ctx->st>>>(a, d_in);
  FS_LAUNCH_CHECK();
  return FS_OK;
}
