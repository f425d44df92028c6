// fs_turb.cu -- standard k-epsilon with equilibrium 'standard', 'scalable' or
// 'automatic' momentum wall functions (Turbulence/ of the reference, TurbulenceModel='kepsilon'), and
// the 'fullydeveloped' outlet mass-flow adjustment of SolveContinuity.
//
// The k and epsilon equations go through one cell-centric gather kernel each
// (diffusion, upwind convection + TVD deferred correction, effective
// divergence, model sources, wall treatment, global assembly, under-relaxation
// and the residual statistics), in the same per-cell summation order as the
// reference's face-loop scatter, so the assembled systems are bit-identical to
// the CPU restatement.  The model constants are REAL(4) literals assigned to
// double precision variables (SetModelCoefficients.for:23-38).
#include "fs_internal.cuh"
#include "fs_device.cuh"

struct fs_turb {
  double *tke = nullptr, *ted = nullptr, *mut = nullptr;        // N
  double *btke = nullptr, *bted = nullptr, *bmut = nullptr;     // B
  double *tkeg = nullptr, *tedg = nullptr;                      // 3N
  double *btkeg = nullptr, *btedg = nullptr;                    // 3B
  double *bedif = nullptr;                                      // B: BeDiffCoefficient of the momentum equations
  double *prod = nullptr;                                       // N: TurbulenceProduction
  double *rhok = nullptr, *brhok = nullptr, *drk = nullptr, *bdrk = nullptr;   // N, B, 3N, 3B
  double *wdist = nullptr;                                      // N: WallDistance (wall-adjacent cells)
  int32_t *itau = nullptr;                                      // N: iTau, boundary face index or -1
  double *utau = nullptr, *yplus = nullptr, *uplus = nullptr, *dupdyp = nullptr;   // B, wall faces
};

// CTAs per SM the k / epsilon gather kernel is compiled for (register cap)
#ifndef FS_TURB_MINB
#define FS_TURB_MINB 3
#endif

namespace {

constexpr double KE_CMU = (double)0.09f;
constexpr double KE_CE1 = (double)1.44f;
constexpr double KE_CE2 = (double)1.92f;
constexpr double KE_SIGK = (double)1.0f;
constexpr double KE_SIGE = (double)1.3f;
constexpr double KE_CTRANS = (double)11.63f;
constexpr double KE_KAPPA = (double)0.41f;
constexpr double KE_CC = (double)5.2f;
constexpr double KE_C1LIM = (double)10.f;
constexpr double KE_YPMIN = (double)0.2f;                       // yplusmin (WallFunctions.for:1904)
constexpr double TWOTHIRD = (double)(2.0f / 3.0f);              // Constants1.F90 TwoThird, REAL(4) literal

struct TurbArgs {
  int N, F, B;
  double rho, mu, urf, bleed, cmu75, tvisc_urf, max_ratio;
  int scheme, hr_on, limit, first, wfun;   // wfun: 0 standard, 1 scalable, 2 automatic
  const int32_t *ncf, *slot, *cn, *bown, *btype, *bset;
  const double *gf, *sf, *dcfv, *gdiff, *tf, *vol;
  const double *bsf, *bnf, *bdv, *bgdiff, *btf;
  const double *u, *v, *w, *bu, *bv, *bw, *ug, *vg, *wg, *mdot, *bmdot;
  double *tke, *ted, *mut, *btke, *bted, *bmut;
  double *phi, *bphi;                 // the transported field (k or epsilon)
  const double *phig;                 // its cell gradient (3N)
  double *prod, *bedif, *wdist;
  int32_t *itau;
  double *utau, *yplus, *uplus, *dupdyp;
  double *ac, *anb, *bc, *red;
  int nblk;
  double in_i[FS_MAX_PATCHES], in_l[FS_MAX_PATCHES];
  FsTransient tr;                     // unsteady runs (tr.on = 0: steady)
};

// TangentialVelocity (NormalAndTangentialVelocities/CalculateTangentialVelocity.for:4-35)
__device__ __forceinline__ double tang_vel(const TurbArgs &a, int i1) {
  const int B = a.B;
  int b = a.itau[i1];
  double nx = a.bnf[b], ny = a.bnf[B + b], nz = a.bnf[2L * B + b];
  double uw = a.bu[b] - a.u[i1], vw = a.bv[b] - a.v[i1], ww = a.bw[b] - a.w[i1];
  double dp = uw * nx + vw * ny + ww * nz;
  uw = uw - dp * nx; vw = vw - dp * ny; ww = ww - dp * nz;
  return sqrt(uw * uw + vw * vw + ww * ww);
}

// wall-adjacent part of CalculateNormalDistanceToWall (CalculateDistanceToWall.for:520-535):
// d = dCF.n of the cell's last wall face, which also becomes iTau
__global__ void k_wall_distance(TurbArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  const int N = a.N, F = a.F, B = a.B;
  double d = 0.;
  int it = -1;
  for (int j = 0; j < a.ncf[i]; j++) {
    int f = a.slot[(long)j * N + i] >> 1;
    if (f < F) continue;
    int b = f - F;
    if (a.btype[b] != FS_BC_WALL_NOSLIP) continue;
    d = a.bdv[b] * a.bnf[b] + a.bdv[B + b] * a.bnf[B + b] + a.bdv[2L * B + b] * a.bnf[2L * B + b];
    it = b;
  }
  a.wdist[i] = d;
  a.itau[i] = it;
}

// CalculateEffectiveDiffusionCoefficient('vel?') boundary part
// (ComputeEffectiveDiffusionCoefficient.for:34-46) and
// EquilibriumMomentumWallFunctions (WallFunctions.for:1846-2025): 'standard'
// (:1918-1960), 'scalable' (:1961-1993, y+ clipped to ctrans + tiny) or
// 'automatic' (:1994-2025, viscous and log u_tau blended by fourth powers)
__global__ void k_wall_fn(TurbArgs a) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.B) return;
  if (a.btype[b] != FS_BC_WALL_NOSLIP) { a.bedif[b] = a.mu + a.bmut[b]; return; }
  const double rho = a.rho, mu = a.mu;
  int i1 = a.bown[b];
  double dn = a.wdist[i1], wv = tang_vel(a, i1);
  if (a.first) {
    a.utau[b] = sqrt((mu + a.mut[i1]) * wv / (dn * rho));
    a.yplus[b] = rho * a.utau[b] * dn / mu;
  }
  double yp1 = dn * rho * a.utau[b] / mu;
  double yp, up, ut, dd;
  if (a.wfun == 2) {
    const double utv = sqrt(mu * wv / (rho * dn));
    const double utl = wv / (log(a.yplus[b]) / KE_KAPPA + KE_CC);
    const double v2 = utv * utv, l2 = utl * utl;
    ut = pow(v2 * v2 + l2 * l2, (double)0.25f);
    up = wv / fmax(ut, TINY);
    yp = rho * ut * dn / mu;
    const double y2 = yp * yp;
    const double factor = (double)0.01f * (y2 * y2) / (1. + 5. * yp) + TINY;
    dd = 1. * exp(-factor) + (1. / (KE_KAPPA * yp)) * exp(-1. / factor);
  } else if (a.wfun == 1) {
    yp = fmax(yp1, KE_CTRANS + TINY);
    dd = 1. / (KE_KAPPA * yp);
    up = log(yp) / KE_KAPPA + KE_CC;
    ut = wv / up;
  } else {
    yp = fmax(yp1, KE_YPMIN);
    if (yp < KE_CTRANS) { up = yp; ut = wv / up; dd = 1.; }
    else { up = log(yp) / KE_KAPPA + KE_CC; ut = wv / up; dd = 1. / (KE_KAPPA * yp); }
  }
  a.yplus[b] = yp; a.uplus[b] = up; a.utau[b] = ut; a.dupdyp[b] = dd;
  double tw = rho * ut * ut;
  double wvis = tw * dn / fmax(wv, TINY);
  a.bmut[b] = fmax(wvis - mu, 0.);
  a.bedif[b] = fmax(wvis, mu);
}

// rhok = 2/3 rho k on cells and boundary faces (AssembleMinusTwoThirdsRhoK.for:58-70)
__global__ void k_rhok(int N, int B, double rho, const double *tke, const double *btke, double *rhok, double *brhok) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < N) rhok[t] = TWOTHIRD * rho * tke[t];
  if (t < B) brhok[t] = TWOTHIRD * rho * btke[t];
}

// CalculateInletTurbulence, 'specifiedil' (CalculateTurbulenceAtBoundary.for:20-40)
__global__ void k_inlet_turb(TurbArgs a) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.B || !fs_is_inlet(a.btype[b])) return;
  int s = a.bset[b];
  double bv2 = a.bu[b] * a.bu[b] + a.bv[b] * a.bv[b] + a.bw[b] * a.bw[b];
  double in2 = a.in_i[s] * a.in_i[s];
  double k = 1.5 * bv2 * in2;
  double e = a.cmu75 * pow(fmax(k, 0.), 1.5) / a.in_l[s];
  a.btke[b] = k; a.bted[b] = e;
  a.bmut[b] = (1. - a.tvisc_urf) * a.bmut[b] + KE_CMU * a.tvisc_urf * a.rho * (k * k) / fmax(e, TINY);
}

// wall-adjacent epsilon (AssembleTEDSources.for:78-120): the cell's last wall face decides
__global__ void k_ted_wall(TurbArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  int b = a.itau[i];
  if (b < 0) return;
  if (a.wfun == 2) return;   // 'automatic': no branch sets the wall-cell epsilon
  double dn = a.wdist[i], k = fmax(a.tke[i], 0.);
  if (a.wfun == 1) {
    dn = a.yplus[b] * a.mu / (a.rho * a.utau[b]);
    a.ted[i] = a.cmu75 * pow(k, 1.5) / (KE_KAPPA * dn);
  } else if (a.yplus[b] < KE_CTRANS) a.ted[i] = 2. * a.mu * k / (a.rho * (dn * dn));
  else a.ted[i] = a.cmu75 * pow(k, 1.5) / (KE_KAPPA * dn);
}

// SolveTKE / SolveTED between the gradient and SolveEquation, one thread per
// cell: AssembleTurbulentKESources / AssembleTurbulentEDSources (kepsilon),
// AssembleDiffusionTerm 'tke'/'ted' (AssembleIsotropicDiffusion.for:99-117,
// inlet faces :2172-2507), AssembleConvectionTerm (AssembleConvection.for:90-110,
// 153-178, 808-892), global assembly, UnderRelaxEquation, for epsilon
// ModifyCoefficientsAlongWalls (ModifyWallCoefficients.for:21-33), and the
// residual statistics of CalculateResiduals at dphi = 0.
template <bool TED>
__global__ void __launch_bounds__(FS_BLOCK, FS_TURB_MINB) k_turb_assemble(TurbArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double r = 0., acphi = -1.;
  if (i < a.N) {
    const int N = a.N, F = a.F, B = a.B;
    const double sig = TED ? KE_SIGE : KE_SIGK;
    const double rho = a.rho, mu = a.mu, V = a.vol[i];
    const double ps = a.phi[i];
    const double gs[3] = {a.phig[i], a.phig[N + i], a.phig[2L * N + i]};
    const double es = mu + a.mut[i] / sig;
    const int nc = a.ncf[i];
    // ---- model sources (into FluxCE / FluxTE)
    double fce, fte;
    if (!TED) {
      // CalculateTurbulenceProduction via CalculatePkTerm / calculateShearStress
      const double ev = a.mut[i] + mu;
      const double ux = a.ug[i], uy = a.ug[N + i], uz = a.ug[2L * N + i];
      const double vx = a.vg[i], vy = a.vg[N + i], vz = a.vg[2L * N + i];
      const double wx = a.wg[i], wy = a.wg[N + i], wz = a.wg[2L * N + i];
      const double s11 = ux, s12 = 0.5 * (uy + vx), s13 = 0.5 * (uz + wx);
      const double s22 = vy, s23 = 0.5 * (vz + wy), s33 = wz;
      double t11 = ev * 2. * s11, t12 = ev * 2. * s12, t13 = ev * 2. * s13;
      double t22 = ev * 2. * s22, t23 = ev * 2. * s23, t33 = ev * 2. * s33;
      const double k1 = fmax(a.tke[i], 0.);
      t11 = t11 - TWOTHIRD * rho * k1;
      t22 = t22 - TWOTHIRD * rho * k1;
      t33 = t33 - TWOTHIRD * rho * k1;
      double P = fmax(t11 * ux + t12 * uy + t13 * uz + t12 * vx + t22 * vy + t23 * vz + t13 * wx + t23 * wy + t33 * wz, 0.);
      if (a.limit) P = fmin(P, KE_C1LIM * rho * fmax(a.ted[i], 0.));
      const double rt = rho * fmax(a.ted[i], 0.) / fmax(a.tke[i], TINY);
      fce = 0. + rt * V;
      fte = 0. - P * V + rt * V * fmax(a.tke[i], TINY);
      // production along walls (AssembleTKESources.for:120-148), wall faces in boundary order
      for (int j = 0; j < nc; j++) {
        int f = a.slot[(long)j * N + i] >> 1;
        if (f < F) continue;
        int b = f - F;
        if (a.btype[b] != FS_BC_WALL_NOSLIP) continue;
        double wv = tang_vel(a, i), wv2 = wv * wv;
        double q = a.utau[b] / a.uplus[b];
        double bp = (rho * rho) * a.dupdyp[b] * (q * q) * wv2 / mu;
        fte = fte + P * V;
        if (a.limit) bp = fmin(bp, KE_C1LIM * rho * fmax(a.bted[b], 0.));
        P = bp;
        fte = fte - P * V;
        a.btke[b] = a.tke[i];
      }
      a.prod[i] = P;
    } else {
      const double t1 = rho * KE_CMU * fmax(a.tke[i], 0.) * V / fmax(a.mut[i], TINY);
      fce = 0. + KE_CE2 * t1 * rho;
      fte = 0. - fmax(KE_CE1 * t1 * a.prod[i], 0.) + KE_CE2 * t1 * rho * fmax(a.ted[i], 0.);
    }
    // ---- faces, slot order = the reference's face order for this cell
    double ac = 0., bc = 0., ed = 0.;
    FS_SLOT_PREFETCH(nc, a.slot, a.cn, N, i);
    auto face = [&](int j, int s, int k) {
      int f = s >> 1;
      if (f >= F) {
        int b = f - F, t = a.btype[b];
        double bm = a.bmdot[b];
        ed = ed + bm;
        double fcf = 0., tf = 0.;
        if (fs_is_inlet(t)) {
          double gamf = mu + a.bmut[b] / sig;          // BeDiffCoefficient of the equation
          double gd = a.bgdiff[b];
          double fcl = gamf * gd, ffl = -gamf * gd;
          double fvl = -(gamf * (gs[0] * a.btf[b] + gs[1] * a.btf[B + b] + gs[2] * a.btf[2L * B + b]));
          fcf = fcl;
          tf = fcl * ps + ffl * a.bphi[b] + fvl;
        }
        if (fs_is_inlet(t) || t == FS_BC_OUTLET_FD || fs_is_sp_outlet(t) || t == FS_BC_OUTLET_MASS) {
          double cc = fmax(bm, 0.), cn_ = -fmax(-bm, 0.);
          fcf = fcf + cc;
          tf = tf + (cc * ps + cn_ * a.bphi[b]);
        }
        ac = ac + fcf;
        bc = bc - tf;
        return;
      }
      const bool nb = s & 1;
      const double g = a.gf[f], md = a.mdot[f];
      const double pk = a.phi[k];
      const double gk[3] = {a.phig[k], a.phig[N + k], a.phig[2L * N + k]};
      const double ek = mu + a.mut[k] / sig;
      double po = nb ? pk : ps, pn = nb ? ps : pk;
      double eo = nb ? ek : es, en = nb ? es : ek;
      double go[3], gn[3];
      for (int d = 0; d < 3; d++) { go[d] = nb ? gk[d] : gs[d]; gn[d] = nb ? gs[d] : gk[d]; }
      double gamf = g * eo + (1. - g) * en;
      double gd = a.gdiff[f];
      double fx = g * go[0] + (1. - g) * gn[0];
      double fy = g * go[1] + (1. - g) * gn[1];
      double fz = g * go[2] + (1. - g) * gn[2];
      double fcl = gamf * gd, ffl = -gamf * gd;
      double fvl = -(gamf * (fx * a.tf[f] + fy * a.tf[F + f] + fz * a.tf[2L * F + f]));
      double fcf = fcl, fff = ffl;
      double tf = fcl * po + ffl * pn + fvl;
      double cc = fmax(md, 0.), cn_ = -fmax(-md, 0.);
      fcf = fcf + cc; fff = fff + cn_;
      tf = tf + (cc * po + cn_ * pn);
      if (a.hr_on)
        tf = tf + hr_flux(a.scheme, a.bleed, md, po, pn, go, gn, a.dcfv[f], a.dcfv[F + f], a.dcfv[2L * F + f]);
      if (nb) {
        ac = ac - fff;
        a.anb[(long)j * N + i] = 0. - fcf;
        bc = bc + tf;
        ed = ed - md;
      } else {
        ac = ac + fcf;
        a.anb[(long)j * N + i] = 0. + fff;
        bc = bc - tf;
        ed = ed + md;
      }
    };
    FS_SLOT_LOOP_J(nc, a.slot, a.cn, N, i, face);
    // effective divergence (AssembleConvection.for:165-178)
    double fce2 = fmax(ed, 0.0) - ed;
    double fve = -(fmax(ed, 0.0) * ps);
    double fte2 = fce2 * ps + fve;
    fce = fce + fce2;
    fte = fte + fte2;
    if (a.tr.on) transient_term(a.tr, TED ? 5 : 4, N, i, V, ps, fce, fte);   // SolveTKE.for:194-199
    ac = ac + fce;
    bc = bc - fte;
    ac = ac / a.urf;
    if (TED && a.itau[i] >= 0) {
      ac = 1.; bc = 0.;
      for (int j = 0; j < nc; j++) {
        a.anb[(long)j * N + i] = 0.;
        int f = a.slot[(long)j * N + i] >> 1;
        if (f >= F && a.btype[f - F] == FS_BC_WALL_NOSLIP) a.bted[f - F] = ps;
      }
    }
    a.ac[i] = ac; a.bc[i] = bc;
    r = fabs(bc);
    acphi = fabs(ac * ps);
  }
  residual_partials(r, acphi, a.red, a.nblk);
}

// BoundTurbulentKE / BoundTurbulentED (BoundTurbulentVariables.for:4-45) and
// updateValuesFromBoundaryConditions 'tke'/'ted' (UpdateVariablesFromBoundaryConditions.for:76-99,502-525)
__global__ void k_turb_bound(int N, int B, const int32_t *bown, const int32_t *btype, double *phi, double *bphi) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < N) phi[t] = fmax(phi[t], TINY);
  if (t < B) {
    int ty = btype[t];
    if (ty == FS_BC_OUTLET_FD || fs_is_sp_outlet(ty) || ty == FS_BC_OUTLET_MASS || ty == FS_BC_SYMMETRY)
      bphi[t] = fmax(phi[bown[t]], TINY);
    else bphi[t] = fmax(bphi[t], 0.);
  }
}

// CalculateTurbulentViscosity, kepsilon (CalculateTurbulentViscosity.for:171-194, 925-945)
__global__ void k_turb_visc(TurbArgs a) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const double cap = a.max_ratio * a.mu;
  if (t < a.N) {
    double m = (1. - a.tvisc_urf) * a.mut[t] + KE_CMU * a.tvisc_urf * a.rho * (a.tke[t] * a.tke[t]) / fmax(a.ted[t], TINY);
    a.mut[t] = fmin(m, cap);
  }
  if (t < a.B) {
    double m = (1. - a.tvisc_urf) * a.bmut[t] + KE_CMU * a.tvisc_urf * a.rho * (a.btke[t] * a.btke[t]) / fmax(a.bted[t], TINY);
    a.bmut[t] = fmin(m, cap);
  }
}

// ---------------------------------------------------------------- outlets
struct FlowArgs {
  int B, NS;
  double rho;
  int ptype[FS_MAX_PATCHES], pstart[FS_MAX_PATCHES], pn[FS_MAX_PATCHES];
  double frac[FS_MAX_PATCHES];   // MassFlowFraction / (total + tiny)
  const int32_t *bown;
  const double *bsf, *u, *v, *w;
  double *bu, *bv, *bw, *bmdot, *flow;
  // FlowIn returns at once when an inlet is a static- or stagnation-pressure
  // one (CalculateFlowIn.for:19-31): mdotIn is then the inlet flow the last
  // continuity residual summed (every inlet face), or 0 before the first
  const double *mdot_in_prev;   // nullptr: FlowIn sums velocity and mass-flow inlets
};

// FlowIn (CalculateFlowIn.for:4-40), FlowOut (CalculateFlowOut.for:4-55),
// AdjustFlow (AdjustFlowAtOuletBoundary.for:4-75) and the 'fullydeveloped'
// outlet velocity of AssembleMdot (AssembleMdotUsingRhieChow.for:2033-2050),
// one CTA: sums in a fixed order (strided per thread, then a fixed tree).
// AdjustFlow's boundary velocity (owner value + gradient . dCF) is not
// formed: AssembleMdot replaces it with the owner velocity before any read.
__global__ void __launch_bounds__(1024) k_flow_in_out(FlowArgs a) {
  __shared__ double sh[32];
  __shared__ double bcast;
  const int B = a.B;
  double s = 0.;
  if (!a.mdot_in_prev)
    for (int q = 0; q < a.NS; q++)
      if (a.ptype[q] == FS_BC_INLET_VEL || a.ptype[q] == FS_BC_INLET_MASS)   // CalculateFlowIn.for:37-48
        for (int j = threadIdx.x; j < a.pn[q]; j += blockDim.x) s = s + a.bmdot[a.pstart[q] + j];
  s = block_sum(s, sh);
  if (a.mdot_in_prev) s = *a.mdot_in_prev;
  if (threadIdx.x == 0) { a.flow[0] = s; bcast = s; }
  __syncthreads();
  const double mdot_in = bcast;
  for (int q = 0; q < a.NS; q++) {
    if (a.ptype[q] != FS_BC_OUTLET_FD) continue;
    double mn = 0.;
    for (int j = threadIdx.x; j < a.pn[q]; j += blockDim.x) {
      int b = a.pstart[q] + j;
      double bm = a.rho * (a.bu[b] * a.bsf[b] + a.bv[b] * a.bsf[B + b] + a.bw[b] * a.bsf[2L * B + b]);
      a.bmdot[b] = bm;
      mn = fmin(mn, bm);
    }
    mn = -block_max(-mn, sh);
    if (threadIdx.x == 0) bcast = fabs(fmin(mn, 0.));
    __syncthreads();
    const double m1 = bcast;
    __syncthreads();
    double so = 0.;
    for (int j = threadIdx.x; j < a.pn[q]; j += blockDim.x) so = so + m1 + a.bmdot[a.pstart[q] + j];
    so = block_sum(so, sh);
    if (threadIdx.x == 0) { bcast = so; a.flow[1 + q] = m1; a.flow[1 + FS_MAX_PATCHES + q] = so; }
    __syncthreads();
    const double mout = bcast;
    __syncthreads();
    const double ratio = a.frac[q] * fabs(mdot_in / (mout + TINY));
    for (int j = threadIdx.x; j < a.pn[q]; j += blockDim.x) {
      int b = a.pstart[q] + j, k = a.bown[b];
      a.bmdot[b] = ratio * (a.bmdot[b] + m1);
      a.bu[b] = a.u[k]; a.bv[b] = a.v[k]; a.bw[b] = a.w[k];
    }
    __syncthreads();
  }
}

TurbArgs turb_args(fs_ctx *ctx) {
  TurbArgs a{};
  const fs_case &c = ctx->cfg;
  fs_turb *T = ctx->turb;
  a.N = ctx->N; a.F = ctx->F; a.B = ctx->B;
  a.rho = c.rho; a.mu = c.mu; a.bleed = c.bleed;
  a.tr = fs_transient_args(ctx);
  a.cmu75 = sqrt(sqrt(KE_CMU)); a.cmu75 = a.cmu75 * a.cmu75 * a.cmu75;
  a.tvisc_urf = c.urf_tvisc; a.max_ratio = c.max_visc_ratio; a.limit = c.limit_production;
  a.wfun = c.wall_function;
  a.ncf = ctx->ncf; a.slot = ctx->slot; a.cn = ctx->cn; a.bown = ctx->bown; a.btype = ctx->btype; a.bset = ctx->d_bset;
  a.gf = ctx->gf; a.sf = ctx->sf; a.dcfv = ctx->dcfv; a.gdiff = ctx->gdiff; a.tf = ctx->tf; a.vol = ctx->vol;
  a.bsf = ctx->bsf; a.bnf = ctx->bnf; a.bdv = ctx->bdv; a.bgdiff = ctx->bgdiff; a.btf = ctx->btf;
  a.u = ctx->u; a.v = ctx->v; a.w = ctx->w; a.bu = ctx->bu; a.bv = ctx->bv; a.bw = ctx->bw;
  a.ug = ctx->ug; a.vg = ctx->vg; a.wg = ctx->wg; a.mdot = ctx->mdot; a.bmdot = ctx->bmdot;
  a.tke = T->tke; a.ted = T->ted; a.mut = T->mut; a.btke = T->btke; a.bted = T->bted; a.bmut = T->bmut;
  a.prod = T->prod; a.bedif = T->bedif; a.wdist = T->wdist; a.itau = T->itau;
  a.utau = T->utau; a.yplus = T->yplus; a.uplus = T->uplus; a.dupdyp = T->dupdyp;
  a.ac = ctx->ac; a.anb = ctx->anb; a.bc = ctx->bc; a.red = ctx->red; a.nblk = fs_grid(ctx->N);
  for (int s = 0; s < FS_MAX_PATCHES; s++) { a.in_i[s] = c.inlet_intensity[s]; a.in_l[s] = c.inlet_length[s]; }
  return a;
}

}  // namespace

// ================================================================ host side
static int talloc(fs_ctx *ctx, double **p, size_t n) {
  FS_CK(cudaMalloc((void **)p, sizeof(double) * (n ? n : 1)));
  FS_CK(cudaMemsetAsync(*p, 0, sizeof(double) * (n ? n : 1), ctx->st));
  return FS_OK;
}

int fs_turb_create(fs_ctx *ctx) {
  if (!ctx->cfg.turbulence) return FS_OK;
  if (ctx->cfg.batched_momentum) { ctx->err = "k-epsilon runs with the per-component momentum solves"; return FS_E_UNSUPPORTED; }
  fs_turb *T = new (std::nothrow) fs_turb();
  if (!T) return FS_E_NOMEM;
  ctx->turb = T;
  const size_t N = ctx->N, B = ctx->B;
  int rc;
  double **n1[] = {&T->tke, &T->ted, &T->mut, &T->prod, &T->rhok, &T->wdist};
  for (auto p : n1) if ((rc = talloc(ctx, p, N))) return rc;
  double **n3[] = {&T->tkeg, &T->tedg, &T->drk};
  for (auto p : n3) if ((rc = talloc(ctx, p, 3 * N))) return rc;
  double **b1[] = {&T->btke, &T->bted, &T->bmut, &T->bedif, &T->brhok, &T->utau, &T->yplus, &T->uplus, &T->dupdyp};
  for (auto p : b1) if ((rc = talloc(ctx, p, B))) return rc;
  double **b3[] = {&T->btkeg, &T->btedg, &T->bdrk};
  for (auto p : b3) if ((rc = talloc(ctx, p, 3 * B))) return rc;
  FS_CK(cudaMalloc((void **)&T->itau, sizeof(int32_t) * (N ? N : 1)));
  TurbArgs a = turb_args(ctx);
  k_wall_distance<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(a);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

void fs_turb_free(fs_ctx *ctx) {
  fs_turb *T = ctx->turb;
  if (!T) return;
  void *ptrs[] = {T->tke, T->ted, T->mut, T->btke, T->bted, T->bmut, T->tkeg, T->tedg, T->btkeg, T->btedg,
                  T->bedif, T->prod, T->rhok, T->brhok, T->drk, T->bdrk, T->wdist, T->itau,
                  T->utau, T->yplus, T->uplus, T->dupdyp};
  for (void *p : ptrs) if (p) cudaFree(p);
  delete T;
  ctx->turb = nullptr;
}

double *fs_turb_field(fs_ctx *ctx, int field, size_t *n) {
  fs_turb *T = ctx->turb;
  *n = 0;
  if (!T) return nullptr;
  switch (field) {
  case FS_F_TKE: *n = ctx->N; return T->tke;
  case FS_F_TED: *n = ctx->N; return T->ted;
  case FS_F_MUT: *n = ctx->N; return T->mut;
  case FS_F_BTKE: *n = ctx->B; return T->btke;
  case FS_F_BTED: *n = ctx->B; return T->bted;
  case FS_F_BMUT: *n = ctx->B; return T->bmut;
  case FS_F_UTAU: *n = ctx->B; return T->utau;
  case FS_F_YPLUS: *n = ctx->B; return T->yplus;
  }
  return nullptr;
}

double *fs_turb_wall_distance(fs_ctx *ctx) { return ctx->turb ? ctx->turb->wdist : nullptr; }

// pointers the momentum kernels read: mu_t (N), BeDiffCoefficient (B), grad(2/3 rho k) (3N)
void fs_turb_momentum_ptrs(fs_ctx *ctx, const double **mut, const double **bedif, const double **drk) {
  fs_turb *T = ctx->turb;
  *mut = T ? T->mut : nullptr;
  *bedif = T ? T->bedif : nullptr;
  *drk = T ? T->drk : nullptr;
}

// 2/3 rho k and its gradient for the Rhie-Chow interpolation (nullptr when laminar)
void fs_turb_rhok_ptrs(fs_ctx *ctx, const double **rhok, const double **drk) {
  fs_turb *T = ctx->turb;
  *rhok = T ? T->rhok : nullptr;
  *drk = T ? T->drk : nullptr;
}

// boundary values of 2/3 rho k and of its gradient (nullptr when laminar)
void fs_turb_brhok_ptrs(fs_ctx *ctx, const double **brhok, const double **bdrk) {
  fs_turb *T = ctx->turb;
  *brhok = T ? T->brhok : nullptr;
  *bdrk = T ? T->bdrk : nullptr;
}

// CalculateEffectiveDiffusionCoefficient('vel?') with the momentum wall
// functions, before the boundary terms of each momentum component
int fs_turb_wall_functions(fs_ctx *ctx) {
  if (!ctx->turb || !ctx->B) return FS_OK;
  TurbArgs a = turb_args(ctx);
  a.first = ctx->nIter == 1;
  k_wall_fn<<<fs_grid(ctx->B), FS_BLOCK, 0, ctx->st>>>(a);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

// MinusTwoThirdsRhoK, X momentum: gradient of 2/3 rho k (AssembleMinusTwoThirdsRhoK.for:40-80)
int fs_turb_rhok_gradient(fs_ctx *ctx) {
  fs_turb *T = ctx->turb;
  if (!T) return FS_OK;
  const fs_case &c = ctx->cfg;
  long n = ctx->N > ctx->B ? ctx->N : ctx->B;
  k_rhok<<<fs_grid(n), FS_BLOCK, 0, ctx->st>>>(ctx->N, ctx->B, c.rho, T->tke, T->btke, T->rhok, T->brhok);
  FS_LAUNCH_CHECK();
  int var = FS_VAR_RHOK, meth = c.method_grad_mom, nit = c.niter_grad_mom;
  const double *phi = T->rhok, *bphi = T->brhok;
  double *g = T->drk, *bg = T->bdrk;
  return fs_gradient_dev(ctx, 1, &var, &phi, &bphi, &g, &bg, &meth, &nit);
}

// one of SolveTurbulenceKineticEnergy (SolveTKE.for:148-229) /
// SolveTurbulenceDissipationRate (SolveTED.for:150-223)
static int solve_turb(fs_ctx *ctx, bool ted) {
  fs_turb *T = ctx->turb;
  const fs_case &c = ctx->cfg;
  const int N = ctx->N, B = ctx->B;
  TurbArgs a = turb_args(ctx);
  if (!ted && B) {
    k_inlet_turb<<<fs_grid(B), FS_BLOCK, 0, ctx->st>>>(a);
    FS_LAUNCH_CHECK();
  }
  int var = ted ? FS_VAR_TED : FS_VAR_TKE, meth = 2, nit = 2;
  const double *phi = ted ? T->ted : T->tke, *bphi = ted ? T->bted : T->btke;
  double *g = ted ? T->tedg : T->tkeg, *bg = ted ? T->btedg : T->btkeg;
  int rc = fs_gradient_dev(ctx, 1, &var, &phi, &bphi, &g, &bg, &meth, &nit);
  if (rc) return rc;
  if (ted) {
    k_ted_wall<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(a);
    FS_LAUNCH_CHECK();
  }
  a.phi = ted ? T->ted : T->tke; a.bphi = ted ? T->bted : T->btke; a.phig = g;
  a.urf = ted ? c.urf_ted : c.urf_tke;
  a.scheme = ted ? c.conv_scheme_ted : c.conv_scheme_tke;
  a.hr_on = (ctx->nIter >= c.niter_start_hr && a.scheme != FS_TVD_UPWIND) ? 1 : 0;
  if (ted) k_turb_assemble<true><<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(a);
  else k_turb_assemble<false><<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(a);
  FS_LAUNCH_CHECK();
  k_residual_final<<<1, 1024, 0, ctx->st>>>(ctx->red, a.nblk, N, var - 1, ctx->resblk);
  FS_LAUNCH_CHECK();
  rc = fs_linear_solve(ctx, var, a.phi, ted ? c.rrf_ted : c.rrf_tke, ted ? c.itmax_ted : c.itmax_tke, c.solver_turb);
  if (rc) return rc;
  long n = N > B ? N : B;
  k_turb_bound<<<fs_grid(n), FS_BLOCK, 0, ctx->st>>>(N, B, ctx->bown, ctx->btype, a.phi, a.bphi);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

// CalculateEffectsOfTurbulence, kepsilon (SolveSelectedTurbulenceModelEquations.for:4-30);
// the strain rate is formed from the velocity gradients inside the k assembly
int fs_turb_effects(fs_ctx *ctx) {
  if (!ctx->turb) return FS_OK;
  int rc;
  if ((rc = solve_turb(ctx, false))) return rc;
  if ((rc = solve_turb(ctx, true))) return rc;
  TurbArgs a = turb_args(ctx);
  long n = ctx->N > ctx->B ? ctx->N : ctx->B;
  k_turb_visc<<<fs_grid(n), FS_BLOCK, 0, ctx->st>>>(a);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

// FlowIn / FlowOut / AdjustFlow when every outlet is 'fullydeveloped'
int fs_flow_in_out(fs_ctx *ctx) {
  const fs_case &c = ctx->cfg;
  int nfd = 0, other = 0;
  for (int s = 0; s < ctx->NS; s++) { nfd += c.patch_type[s] == FS_BC_OUTLET_FD; other += fs_is_sp_outlet(c.patch_type[s]) || c.patch_type[s] == FS_BC_OUTLET_MASS; }
  if (!nfd || other) return FS_OK;   // FlowOut / AdjustFlow act only when every outlet is fully developed
  FlowArgs a{};
  a.B = ctx->B; a.NS = ctx->NS; a.rho = c.rho;
  double tff = 0.;
  for (int s = 0; s < ctx->NS; s++) if (c.patch_type[s] == FS_BC_OUTLET_FD) tff = tff + c.mass_flow_fraction[s];
  for (int s = 0; s < ctx->NS; s++) {
    a.ptype[s] = c.patch_type[s]; a.pstart[s] = ctx->h_bset_start[s]; a.pn[s] = ctx->h_bset_n[s];
    a.frac[s] = c.mass_flow_fraction[s] / (tff + TINY);
  }
  a.bown = ctx->bown; a.bsf = ctx->bsf; a.u = ctx->u; a.v = ctx->v; a.w = ctx->w;
  for (int s = 0; s < ctx->NS; s++)
    if (fs_is_p_inlet(c.patch_type[s])) a.mdot_in_prev = ctx->resblk + RB_MDOTIN;
  a.bu = ctx->bu; a.bv = ctx->bv; a.bw = ctx->bw; a.bmdot = ctx->bmdot; a.flow = ctx->flow;
  k_flow_in_out<<<1, 1024, 0, ctx->st>>>(a);
  FS_LAUNCH_CHECK();
  return FS_OK;
}
