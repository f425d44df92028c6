// fs_energy.cu -- the temperature equation (LSolveEnergy, EnergyEquation =
// 'temperature'; Energy/SolveTemperatureEquation.for:169-290) at constant rho,
// cp and conductivity with isotropic diffusion, solved after the turbulence
// equations of each outer iteration (MainProgram.for:281).
//
// Three kernels around the shared gradient and linear-solver paths:
//   k_energy_bface     boundary faces before the gradient: the static
//                      temperature of stagnation-temperature inlets and the
//                      boundary diffusion coefficient (thermal wall functions
//                      of k-epsilon runs);
//   k_energy_assemble  one thread per cell, the cell's faces in the
//                      reference's face order: diffusion, cp-weighted upwind
//                      convection with the TVD deferred correction, effective
//                      divergence, transient and source terms, global
//                      assembly, under-relaxation and residual statistics;
//   k_energy_finish    BoundTemperature and updateValuesFromBoundaryConditions.
// Each face's fluxes are summed in the reference's association order
// (X = X + a + b is (X + a) + b), so the assembled system matches the CPU
// restatement to rounding of the per-cell sums.
#include "fs_internal.cuh"
#include "fs_device.cuh"

struct fs_energy {
  double *t = nullptr, *bt = nullptr;       // Temperature (N), BTemperature (B)
  double *tg = nullptr, *btg = nullptr;     // TempGrad (3N), BTempGrad (3B)
  double *bt0 = nullptr;                    // BStagnationTemperature (B)
  double *bedif = nullptr;                  // BeDiffCoefficient of 'temp' (B)
  int32_t *tbc = nullptr;                   // thermal boundary set per face (fs_tbc, resolved)
};

#ifndef FS_ENERGY_MINB
#define FS_ENERGY_MINB 3
#endif

namespace {

constexpr double SIGT_DEFAULT = (double)0.9f;   // SetModelCoefficients.for:27 sigT=0.9
constexpr double EW_CTRANS = (double)11.63f;    // ctrans (SetModelCoefficients.for:37)

struct EnergyArgs {
  int N, F, B;
  double rho, mu, cp, kc, st, urf, bleed, sc, sb, tmin, tmax;
  int scheme, hr_on, gi, gam, turb, relax, inviscid, wfun, limit;
  const int32_t *ncf, *slot, *cn, *bown, *btype, *bset, *tbc;
  const double *gf, *dcfv, *dcf, *gdiff, *tf, *vol;
  const double *bfa, *bgdiff, *btf;
  const double *bu, *bv, *bw, *mdot, *bmdot;
  const double *mut, *bmut, *wdist, *utau, *yplus;   // k-epsilon runs (nullptr when laminar)
  double *t, *bt, *bedif;
  const double *tg, *bt0;
  double *ac, *anb, *bc, *red;
  int nblk;
  double qh[FS_MAX_PATCHES], hinf[FS_MAX_PATCHES], tinf[FS_MAX_PATCHES];
  FsTransient tr;
};

// CalculateEffectiveDiffusionCoefficient('temp') of a cell
// (ComputeEffectiveDiffusionCoefficient.for:75-81, 601-605)
__device__ __forceinline__ double cell_gamma(const EnergyArgs &a, int i) {
  return a.turb ? a.kc + a.cp * a.mut[i] / a.st : a.kc;
}

// InterpolateElementToFace of the diffusion coefficient by InterpolationSchemeGamaEnergy
// (InterpolateFromElementToFace.for:17-60; 'harmonic' divides by the arithmetic weight, as written there)
__device__ __forceinline__ double face_gamma(int scheme, double g, double md, double eo, double en) {
  double w;
  switch (scheme) {
  case 1: w = md > 0. ? 1. : 0.; return w * eo + (1. - w) * en;
  case 2: w = md > 0. ? 0. : 1.; return w * eo + (1. - w) * en;
  case 3: {
    double r = eo * en;
    if (r != 0.) r = r / (g * eo + (1. - g) * en);
    return r;
  }
  default: return g * eo + (1. - g) * en;
  }
}

// EquilibriumEnergyWallFunctions (WallFunctions.for:743-1005), incompressible:
// the no-slip wall face's BeDiffCoefficient from the thermal law of the wall,
// with the uTau and yplus the momentum wall functions left.  The HeatFlux of
// Dirichlet walls derived there is output only, and the von Neumann wall
// temperature set there is replaced after the solve before anything reads it.
__device__ double thermal_wall(const EnergyArgs &a, int b) {
  const int i1 = a.bown[b];
  const double cp = a.cp, dn = a.wdist[i1];
  const double pr = a.mu * cp / a.kc;
  const double q = (double)3.85f * pow(pr, (double)(1.f / 3.f)) - (double)1.3f;
  const double prp = q * q;
  double pry, tplus, wvt;
  if (a.wfun == 1) {            // 'scalable' (:840-875)
    pry = fmax(pr * a.yplus[b], EW_CTRANS);
    tplus = (double)2.12f * log(pry) + prp;
    wvt = a.utau[b] * a.rho * cp * dn / tplus;
  } else if (a.wfun == 2) {     // 'automatic' (:877-912)
    pry = pr * a.yplus[b];
    const double p2 = pry * pry;
    const double gam = (double)0.01f * (p2 * p2) / (1. + 5. * pr * pr * pry) + TINY;
    tplus = pry * exp(-gam) + ((double)2.12f * log(pry) + prp) * exp(-1. / gam);
    wvt = a.utau[b] * a.rho * cp * dn / fmax(tplus, TINY);
  } else {                      // 'standard' (:796-838)
    pry = pr * a.yplus[b];
    tplus = pry < EW_CTRANS ? pry : (double)2.12f * log(pry) + prp;
    wvt = a.utau[b] * a.rho * cp * dn / fmax(tplus, TINY);
  }
  return fmax(wvt, a.kc);
}

// UpdateStaticTemperatureFromTotal (UpdateInletStaticTemperatureFromTotalTemperature.for:27-47)
// and the boundary part of CalculateEffectiveDiffusionCoefficient('temp')
__global__ void k_energy_bface(EnergyArgs a) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.B) return;
  if (a.tbc[b] == FS_TBC_INLET_STAGNATION) {
    const double v2 = a.bu[b] * a.bu[b] + a.bv[b] * a.bv[b] + a.bw[b] * a.bw[b];
    a.bt[b] = a.bt0[b] - 0.5 * v2 / a.cp;
  }
  double e = a.kc;
  if (a.turb) {
    e = a.kc + a.cp * a.bmut[b] / a.st;
    if (a.btype[b] == FS_BC_WALL_NOSLIP) e = thermal_wall(a, b);
  }
  a.bedif[b] = e;
}

// SolveTemperature between the gradient and SolveEquation: AssembleDiffusionTerm
// (AssembleIsotropicDiffusion.for:99-117, 2508-2922), AssembleConvectionTerm
// (AssembleConvection.for:111-131, 153-178, 967-1186), HRSchemesCorrections
// (AssembleHRSchemeCorrection.for:109-132), AssembleTransientTerm, AssembleSourceTerm
// (AssembleSources.for:18-27), the global assembly and UnderRelaxEquation, and
// the residual statistics of CalculateResiduals at dphi = 0.
__global__ void __launch_bounds__(FS_BLOCK, FS_ENERGY_MINB) k_energy_assemble(EnergyArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double r = 0., acphi = -1.;
  if (i < a.N) {
    const int N = a.N, F = a.F, B = a.B;
    const double cp = a.cp, V = a.vol[i];
    const double ts = a.t[i];
    const double gs[3] = {a.tg[i], a.tg[N + i], a.tg[2L * N + i]};
    const double es = cell_gamma(a, i);
    const int nc = a.ncf[i];
    double ac = 0., bc = 0., ed = 0.;
    FS_SLOT_PREFETCH(nc, a.slot, a.cn, N, i);
    auto face = [&](int j, int s, int k) {
      int f = s >> 1;
      if (f >= F) {
        const int b = f - F, t = a.tbc[b], set = a.bset[b];
        const double bm = a.bmdot[b], bT = a.bt[b];
        ed = ed + bm * cp;
        double fcf = 0., tf = 0.;
        if (!a.inviscid) {
          // BGamaFace = BeDiffCoefficient, boundary gradient = the owner's
          const double gamf = a.bedif[b];
          const double dot = gs[0] * a.btf[b] + gs[1] * a.btf[B + b] + gs[2] * a.btf[2L * B + b];
          if (t == FS_TBC_WALL_DIRICHLET || t == FS_TBC_INLET_STATIC || t == FS_TBC_INLET_STAGNATION) {
            const double gd = a.bgdiff[b];
            const double fcl = gamf * gd, ffl = -gamf * gd, fvl = -(gamf * dot);
            fcf = fcf + fcl;
            tf = tf + fcl * ts + ffl * bT + fvl;
          } else if (t == FS_TBC_WALL_NEUMANN) {
            tf = tf + -(a.qh[set] * a.bfa[b]);
          } else if (t == FS_TBC_WALL_ROBIN) {
            const double h = a.hinf[set], gd = a.bgdiff[b], A = a.bfa[b];
            const double term1 = h * A + gamf * gd;
            const double fcl = h * A * gd * gamf / term1;
            const double fvl = -(a.tinf[set] * fcl) - h * A * gamf * dot / term1;
            fcf = fcf + fcl;
            tf = tf + fcl * ts + fvl;
          } else if (t == FS_TBC_SYMMETRY) {
            a.bt[b] = ts;   // BFiT = FiT(i1) (AssembleIsotropicDiffusion.for:2837)
          }
        }
        if (t == FS_TBC_INLET_STATIC || t == FS_TBC_INLET_STAGNATION || t == FS_TBC_OUTLET_FD) {
          const double cc = cp * fmax(bm, 0.), cn_ = -(cp * fmax(-bm, 0.));
          fcf = fcf + cc;
          tf = tf + cc * ts + cn_ * bT;
        }
        ac = ac + fcf;
        bc = bc - tf;
        return;
      }
      const bool nb = s & 1;                 // this cell is the face's neighbour
      const double g = a.gf[f], md = a.mdot[f];
      const double tk = a.t[k];
      const double gk[3] = {a.tg[k], a.tg[N + k], a.tg[2L * N + k]};
      const double po = nb ? tk : ts, pn = nb ? ts : tk;
      double go[3], gn[3];
      for (int d = 0; d < 3; d++) { go[d] = nb ? gk[d] : gs[d]; gn[d] = nb ? gs[d] : gk[d]; }
      double fcf = 0., fff = 0., tf = 0.;
      if (!a.inviscid) {
        const double ek = cell_gamma(a, k);
        const double gamf = face_gamma(a.gam, g, md, nb ? ek : es, nb ? es : ek);
        const double dx = a.dcfv[f], dy = a.dcfv[F + f], dz = a.dcfv[2L * F + f], d = a.dcf[f];
        double fx, fy, fz;   // TempGradf (GradientInterpolationSchemeEnergy)
        face_grad(a.gi, g, md, po, pn, d, dx / d, dy / d, dz / d, go[0], go[1], go[2], gn[0], gn[1], gn[2], fx, fy, fz);
        const double gd = a.gdiff[f];
        const double fcl = gamf * gd, ffl = -gamf * gd;
        const double fvl = -(gamf * (fx * a.tf[f] + fy * a.tf[F + f] + fz * a.tf[2L * F + f]));
        fcf = fcf + fcl; fff = fff + ffl;
        tf = tf + fcl * po + ffl * pn + fvl;
      }
      const double cpf = g * cp + (1. - g) * cp;
      const double cc = fmax(md, 0.) * cpf, cn_ = -fmax(-md, 0.) * cpf;
      fcf = fcf + cc; fff = fff + cn_;
      tf = tf + cc * po + cn_ * pn;
      if (a.hr_on)
        tf = tf + hr_flux(a.scheme, a.bleed, md, po, pn, go, gn, a.dcfv[f], a.dcfv[F + f], a.dcfv[2L * F + f], cpf);
      if (nb) {
        ac = ac - fff;
        a.anb[(long)j * N + i] = 0. - fcf;
        bc = bc + tf;
        ed = ed - md * cpf;
      } else {
        ac = ac + fcf;
        a.anb[(long)j * N + i] = 0. + fff;
        bc = bc - tf;
        ed = ed + md * cpf;
      }
    };
    FS_SLOT_LOOP_J(nc, a.slot, a.cn, N, i, face);
    // convection-divergence term with the cp-weighted effective divergence
    // (AssembleConvection.for:165-178, CalculateEffectiveDivergence.for 'temp')
    double fce = 0., fte = 0.;
    const double fce2 = fmax(ed, 0.0) - ed;
    const double fve = -(fmax(ed, 0.0) * ts);
    fce = fce + fce2;
    fte = fte + (fce2 * ts + fve);
    if (a.tr.on) transient_term(a.tr, 6, N, i, V, ts, fce, fte, cp);   // rho cp V (AssembleTheTransientTerm.for 'temp')
    // AssembleSourceTerm(ScEnergy, SbEnergy)
    if (a.sc < 0.) fce = fce - a.sc * V;
    else fce = fce + 0.;
    fte = fte - (a.sb + a.sc * ts) * V;
    ac = ac + fce;
    bc = bc - fte;
    if (a.relax) ac = ac / a.urf;
    a.ac[i] = ac; a.bc[i] = bc;
    r = fabs(bc);
    acphi = fabs(ac * ts);
  }
  residual_partials(r, acphi, a.red, a.nblk);
}

// BoundTemperature (BoundTemperatureValues.for:18-32) and
// updateValuesFromBoundaryConditions('temp'), isotropic
// (UpdateVariablesFromBoundaryConditions.for:820-880).  A face thread clamps
// its owner's value itself (the clamp is idempotent, so it reads the same value
// whether or not the cell's thread has stored it yet).
__global__ void k_energy_finish(EnergyArgs a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x < a.N && a.limit) {
    double v = fmax(a.tmin, a.t[x]);
    a.t[x] = fmin(a.tmax, v);
  }
  if (x >= a.B) return;
  const int b = x, ty = a.tbc[b], i1 = a.bown[b], set = a.bset[b];
  double tc = a.t[i1];
  double bt = a.bt[b];
  if (a.limit) {
    tc = fmin(a.tmax, fmax(a.tmin, tc));
    bt = fmin(a.tmax, fmax(a.tmin, bt));
  }
  const double gamf = a.bedif[b], gd = a.bgdiff[b];
  if (ty == FS_TBC_WALL_NEUMANN) {
    bt = tc - a.qh[set] / (gamf * gd + TINY);
  } else if (ty == FS_TBC_WALL_ROBIN) {
    const int N = a.N, B = a.B;
    const double h = a.hinf[set], A = a.bfa[b];
    const double term1 = h * A + gamf * gd;
    const double term2 = gamf * (a.tg[i1] * a.btf[b] + a.tg[N + i1] * a.btf[B + b] + a.tg[2L * N + i1] * a.btf[2L * B + b]);
    bt = (h * A * a.tinf[set] + gamf * gd * tc - term2) / (term1 + TINY);
  } else if (ty == FS_TBC_OUTLET_FD || ty == FS_TBC_SYMMETRY) {
    bt = tc;
  }
  a.bt[b] = bt;
}

EnergyArgs energy_args(fs_ctx *ctx) {
  EnergyArgs a{};
  const fs_case &c = ctx->cfg;
  fs_energy *E = ctx->energy;
  a.N = ctx->N; a.F = ctx->F; a.B = ctx->B;
  a.rho = c.rho; a.mu = c.mu; a.cp = c.cp; a.kc = c.conductivity;
  a.st = c.sigma_t > 0. ? c.sigma_t : SIGT_DEFAULT;
  a.urf = c.urf_energy; a.relax = c.relax_energy; a.bleed = c.bleed_energy;
  a.sc = c.energy_sc; a.sb = c.energy_sb;
  a.limit = c.limit_temperature; a.tmin = c.temp_min; a.tmax = c.temp_max;
  a.scheme = c.conv_scheme_energy;
  a.hr_on = (ctx->nIter >= c.niter_start_hr && c.conv_scheme_energy != FS_TVD_UPWIND) ? 1 : 0;
  a.gi = c.grad_interp_energy; a.gam = c.gamma_interp_energy;
  a.turb = ctx->turb ? 1 : 0; a.inviscid = c.inviscid; a.wfun = c.energy_wall_function;
  a.ncf = ctx->ncf; a.slot = ctx->slot; a.cn = ctx->cn; a.bown = ctx->bown; a.btype = ctx->btype;
  a.bset = ctx->d_bset; a.tbc = E->tbc;
  a.gf = ctx->gf; a.dcfv = ctx->dcfv; a.dcf = ctx->dcf; a.gdiff = ctx->gdiff; a.tf = ctx->tf; a.vol = ctx->vol;
  a.bfa = ctx->bfa; a.bgdiff = ctx->bgdiff; a.btf = ctx->btf;
  a.bu = ctx->bu; a.bv = ctx->bv; a.bw = ctx->bw; a.mdot = ctx->mdot; a.bmdot = ctx->bmdot;
  if (ctx->turb) {
    size_t n;
    a.mut = fs_turb_field(ctx, FS_F_MUT, &n);
    a.bmut = fs_turb_field(ctx, FS_F_BMUT, &n);
    a.utau = fs_turb_field(ctx, FS_F_UTAU, &n);
    a.yplus = fs_turb_field(ctx, FS_F_YPLUS, &n);
    a.wdist = fs_turb_wall_distance(ctx);
  }
  a.t = E->t; a.bt = E->bt; a.bedif = E->bedif; a.tg = E->tg; a.bt0 = E->bt0;
  a.ac = ctx->ac; a.anb = ctx->anb; a.bc = ctx->bc; a.red = ctx->red; a.nblk = fs_grid(ctx->N);
  for (int s = 0; s < FS_MAX_PATCHES; s++) {
    a.qh[s] = c.patch_heat_flux[s]; a.hinf[s] = c.patch_h_inf[s]; a.tinf[s] = c.patch_temperature[s];
  }
  a.tr = fs_transient_args(ctx);
  return a;
}

// the thermal boundary set of a patch (FS_TBC_DEFAULT follows the flow type)
int thermal_type(const fs_case &c, int s) {
  const int t = c.patch_thermal[s], f = c.patch_type[s];
  if (t != FS_TBC_DEFAULT) return t;
  if (f == FS_BC_WALL_NOSLIP || f == FS_BC_WALL_SLIP) return FS_TBC_WALL_NEUMANN;
  if (fs_is_inlet(f)) return FS_TBC_INLET_STATIC;
  if (f == FS_BC_SYMMETRY) return FS_TBC_SYMMETRY;
  return FS_TBC_OUTLET_FD;
}

}  // namespace

// ================================================================ host side
int fs_energy_create(fs_ctx *ctx) {
  const fs_case &c = ctx->cfg;
  if (!c.energy) return FS_OK;
  if (c.inviscid) { ctx->err = "the temperature equation is not restated for inviscid runs"; return FS_E_UNSUPPORTED; }
  if (!(c.cp > 0.) || !(c.conductivity > 0.)) { ctx->err = "energy: cp and conductivity must be > 0"; return FS_E_ARG; }
  if (c.relax_energy && !(c.urf_energy > 0.)) { ctx->err = "energy: urf_energy must be > 0"; return FS_E_ARG; }
  if (c.gamma_interp_energy < 0 || c.gamma_interp_energy > 3 || c.energy_wall_function < 0 || c.energy_wall_function > 2) {
    ctx->err = "energy: gamma_interp_energy 0..3, energy_wall_function 0..2";
    return FS_E_ARG;
  }
  for (int s = 0; s < ctx->NS; s++)
    if (c.patch_thermal[s] < FS_TBC_DEFAULT || c.patch_thermal[s] > FS_TBC_SYMMETRY) {
      ctx->err = "energy: patch_thermal must be one of fs_tbc";
      return FS_E_ARG;
    }
  fs_energy *E = new (std::nothrow) fs_energy();
  if (!E) return FS_E_NOMEM;
  ctx->energy = E;
  const size_t N = ctx->N, B = ctx->B;
  const size_t nb = B ? B : 1;
  FS_CK(cudaMalloc((void **)&E->t, sizeof(double) * N));
  FS_CK(cudaMalloc((void **)&E->bt, sizeof(double) * nb));
  FS_CK(cudaMalloc((void **)&E->tg, sizeof(double) * 3 * N));
  FS_CK(cudaMalloc((void **)&E->btg, sizeof(double) * 3 * nb));
  FS_CK(cudaMalloc((void **)&E->bt0, sizeof(double) * nb));
  FS_CK(cudaMalloc((void **)&E->bedif, sizeof(double) * nb));
  FS_CK(cudaMalloc((void **)&E->tbc, sizeof(int32_t) * nb));
  FS_CK(cudaMemsetAsync(E->tg, 0, sizeof(double) * 3 * N, ctx->st));
  FS_CK(cudaMemsetAsync(E->btg, 0, sizeof(double) * 3 * nb, ctx->st));
  FS_CK(cudaMemsetAsync(E->bedif, 0, sizeof(double) * nb, ctx->st));
  // initial values: cells and unset faces temp_init; Dirichlet walls and inlets their patch temperature
  std::vector<double> ht(N, c.temp_init), hbt(nb, c.temp_init), hb0(nb, 0.);
  std::vector<int32_t> htbc(nb, FS_TBC_DEFAULT);
  for (size_t b = 0; b < B; b++) {
    const int s = ctx->h_bset[b], t = thermal_type(c, s);
    htbc[b] = t;
    if (t == FS_TBC_WALL_DIRICHLET || t == FS_TBC_INLET_STATIC || t == FS_TBC_INLET_STAGNATION) hbt[b] = c.patch_temperature[s];
    hb0[b] = c.patch_temperature[s];
  }
  FS_CK(cudaMemcpyAsync(E->t, ht.data(), sizeof(double) * N, cudaMemcpyHostToDevice, ctx->st));
  FS_CK(cudaMemcpyAsync(E->bt, hbt.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, ctx->st));
  FS_CK(cudaMemcpyAsync(E->bt0, hb0.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, ctx->st));
  FS_CK(cudaMemcpyAsync(E->tbc, htbc.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice, ctx->st));
  // the host vectors must outlive the copies
  FS_CK(cudaStreamSynchronize(ctx->st));
  return FS_OK;
}

void fs_energy_free(fs_ctx *ctx) {
  fs_energy *E = ctx->energy;
  if (!E) return;
  void *ptrs[] = {E->t, E->bt, E->tg, E->btg, E->bt0, E->bedif, E->tbc};
  for (void *p : ptrs) if (p) cudaFree(p);
  delete E;
  ctx->energy = nullptr;
}

double *fs_energy_field(fs_ctx *ctx, int field, size_t *n) {
  fs_energy *E = ctx->energy;
  *n = 0;
  if (!E) return nullptr;
  switch (field) {
  case FS_F_T: *n = ctx->N; return E->t;
  case FS_F_BT: *n = ctx->B; return E->bt;
  case FS_F_TGRAD: *n = 3 * (size_t)ctx->N; return E->tg;
  }
  return nullptr;
}

double *fs_energy_bgrad(fs_ctx *ctx) { return ctx->energy ? ctx->energy->btg : nullptr; }

// SolveEnergy, 'temperature' (SelectEnergyEquationToSolve.for:12-14; SolveTemperatureEquation.for:169-290)
int fs_energy_solve(fs_ctx *ctx) {
  fs_energy *E = ctx->energy;
  if (!E) return FS_OK;
  const fs_case &c = ctx->cfg;
  const int N = ctx->N, B = ctx->B;
  EnergyArgs a = energy_args(ctx);
  if (B) {
    k_energy_bface<<<fs_grid(B), FS_BLOCK, 0, ctx->st>>>(a);
    FS_LAUNCH_CHECK();
  }
  int var = FS_VAR_TEMP, meth = c.method_grad_energy, nit = c.niter_grad_energy;
  const double *phi = E->t, *bphi = E->bt;
  double *g = E->tg, *bg = E->btg;
  int rc = fs_gradient_dev(ctx, 1, &var, &phi, &bphi, &g, &bg, &meth, &nit);
  if (rc) return rc;
  k_energy_assemble<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(a);
  FS_LAUNCH_CHECK();
  k_residual_final<<<1, 1024, 0, ctx->st>>>(ctx->red, a.nblk, N, FS_VAR_TEMP - 1, ctx->resblk);
  FS_LAUNCH_CHECK();
  rc = fs_linear_solve(ctx, FS_VAR_TEMP, E->t, c.rrf_energy, c.itmax_energy, c.solver_energy);
  if (rc) return rc;
  long n = N > B ? N : B;
  k_energy_finish<<<fs_grid(n), FS_BLOCK, 0, ctx->st>>>(a);
  FS_LAUNCH_CHECK();
  return FS_OK;
}
