// fs_time.cu -- unsteady runs: the time levels of the solved fields, the
// coefficients of the transient term (AssembleTheTransientTerm.for:52-330)
// and the time-step prologue of the reference's time loop
// (MainProgram.for:184-245: CrankNicolson, updateVariablesInTime, dt
// bookkeeping).  Density, DensityOld and DensityOldOld are the constant rho.
//
// Layout: old / oldold hold u, v, w, p, k, epsilon, T in blocks of N (time
// levels n-1 and n-2); bold the boundary values at n-1 in blocks of B.  The
// k and epsilon blocks stay zero in laminar runs, the T block in isothermal ones.
#include "fs_internal.cuh"

namespace {

// phi = 2 phi - phiOld (CrankNicolsonRoutine.for:51-80), cells or boundary faces
__global__ void k_cn_extrapolate(double *x, const double *old, long n) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) x[i] = 2. * x[i] - old[i];
}

// factor1..3 of 'cranknicolson2' (AssembleTheTransientTerm.for:201-203) and
// 'adamsmoulton' (:292-294)
void time_factors(int scheme, double dt, double dto, double dtoo, double f[3]) {
  if (scheme == FS_TRANSIENT_CRANKNICOLSON2) {
    f[0] = (dto / dt) / (dt + dto);
    f[1] = 1. / (dt + dto) - (dtoo / dt) / (dto + dtoo);
    f[2] = -(dto / dt) / (dto + dtoo);
  } else {
    f[0] = 1. / dt + 1. / (dt + dto);
    f[2] = (dto / dt) / (dto + dtoo);
    f[1] = f[0] + f[2];
  }
}

// the solved fields of the time levels (cell values, or boundary values with
// bnd); nullptr for k, epsilon or T when their equation is not solved
double *level_field(fs_ctx *ctx, int q, bool bnd) {
  size_t n = 0;
  switch (q) {
  case 0: return bnd ? ctx->bu : ctx->u;
  case 1: return bnd ? ctx->bv : ctx->v;
  case 2: return bnd ? ctx->bw : ctx->w;
  case 3: return bnd ? ctx->bp : ctx->p;
  case 4: return fs_turb_field(ctx, bnd ? FS_F_BTKE : FS_F_TKE, &n);
  case 5: return fs_turb_field(ctx, bnd ? FS_F_BTED : FS_F_TED, &n);
  default: return fs_energy_field(ctx, bnd ? FS_F_BT : FS_F_T, &n);
  }
}

int scheme_in_effect(int scheme, int ndt_before) {
  // the first step of the three-level schemes runs as 'euler' (MainProgram.for:201-224)
  if (ndt_before == 0 && (scheme == FS_TRANSIENT_CRANKNICOLSON2 || scheme == FS_TRANSIENT_ADAMSMOULTON))
    return FS_TRANSIENT_EULER;
  return scheme;
}

}  // namespace

FsTransient fs_transient_args(const fs_ctx *ctx) {
  FsTransient t{};
  if (!ctx->cfg.unsteady || !ctx->old) return t;
  t.on = 1;
  t.rho = ctx->cfg.rho;
  t.old = ctx->old;
  t.oldold = ctx->oldold;
  if (ctx->tscheme == FS_TRANSIENT_EULER || ctx->tscheme == FS_TRANSIENT_CRANKNICOLSON1) {
    t.three = 0;
    t.d = ctx->tscheme == FS_TRANSIENT_EULER ? ctx->dt : ctx->dt / 2.;   // dtCN = dt/2 (:126)
  } else {
    double f[3];
    time_factors(ctx->tscheme, ctx->dt, ctx->dto, ctx->dtoo, f);
    t.three = 1;
    t.f1 = f[0]; t.f2 = f[1]; t.f3 = f[2];
    t.s2 = ctx->tscheme == FS_TRANSIENT_ADAMSMOULTON ? -1. : 1.;        // :300 -factor2
  }
  return t;
}

// ComputeTransientGradient of the density (CalculateTransientGradient.for:19-60)
double fs_drhodt(const fs_ctx *ctx) {
  const double rho = ctx->cfg.rho, dt = ctx->dt;
  switch (ctx->tscheme) {
  case FS_TRANSIENT_EULER: return (rho - rho) / dt;
  case FS_TRANSIENT_CRANKNICOLSON1: return (rho - rho) / (dt / 2.);
  default: {
    double f[3];
    time_factors(ctx->tscheme, dt, ctx->dto, ctx->dtoo, f);
    if (ctx->tscheme == FS_TRANSIENT_CRANKNICOLSON2) return f[0] * rho + f[1] * rho + f[2] * rho;
    return f[0] * rho - f[1] * rho + f[2] * rho;
  }
  }
}

// InitializeOldVariables (OldVariablesInitialization.for:129-170): every
// time level starts from the current fields
int fs_transient_create(fs_ctx *ctx) {
  const fs_case &c = ctx->cfg;
  if (!c.unsteady) return FS_OK;
  if (!(c.dt > 0.) || c.transient_scheme < FS_TRANSIENT_EULER || c.transient_scheme > FS_TRANSIENT_ADAMSMOULTON) {
    ctx->err = "unsteady case: dt must be > 0 and transient_scheme one of fs_transient";
    return FS_E_ARG;
  }
  const size_t N = ctx->N, B = ctx->B;
  if (cudaMalloc(&ctx->old, sizeof(double) * FS_NLEVELS * N) != cudaSuccess ||
      cudaMalloc(&ctx->oldold, sizeof(double) * FS_NLEVELS * N) != cudaSuccess ||
      cudaMalloc(&ctx->bold, sizeof(double) * FS_NLEVELS * (B ? B : 1)) != cudaSuccess)
    return FS_E_NOMEM;
  if (c.transient_scheme == FS_TRANSIENT_CRANKNICOLSON1 && cudaMalloc(&ctx->p_mx, sizeof(double) * N) != cudaSuccess)
    return FS_E_NOMEM;
  FS_CK(cudaMemsetAsync(ctx->old, 0, sizeof(double) * FS_NLEVELS * N, ctx->st));
  FS_CK(cudaMemsetAsync(ctx->bold, 0, sizeof(double) * FS_NLEVELS * (B ? B : 1), ctx->st));
  if (ctx->p_mx) FS_CK(cudaMemsetAsync(ctx->p_mx, 0, sizeof(double) * N, ctx->st));
  for (int q = 0; q < FS_NLEVELS; q++) {
    const double *x = level_field(ctx, q, false), *bx = level_field(ctx, q, true);
    if (x) FS_CK(cudaMemcpyAsync(ctx->old + q * N, x, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->st));
    if (bx && B) FS_CK(cudaMemcpyAsync(ctx->bold + q * B, bx, sizeof(double) * B, cudaMemcpyDeviceToDevice, ctx->st));
  }
  FS_CK(cudaMemcpyAsync(ctx->oldold, ctx->old, sizeof(double) * FS_NLEVELS * N, cudaMemcpyDeviceToDevice, ctx->st));
  ctx->dt = ctx->dto = ctx->dtoo = c.dt;
  ctx->time = 0.;
  ctx->ndt = 0;
  ctx->tscheme = c.transient_scheme;
  return FS_OK;
}

void fs_transient_free(fs_ctx *ctx) {
  for (double **p : {&ctx->old, &ctx->oldold, &ctx->bold, &ctx->p_mx}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
}

int fs_advance_time(fs_ctx *ctx, double dt_next) {
  if (!ctx) return FS_E_ARG;
  cudaSetDevice(ctx->dev);
  const fs_case &c = ctx->cfg;
  if (!c.unsteady || !ctx->old) { ctx->err = "fs_advance_time: the case is not unsteady"; return FS_E_ARG; }
  if (!(dt_next > 0.)) { ctx->err = "fs_advance_time: dt_next must be > 0"; return FS_E_ARG; }
  const long N = ctx->N, B = ctx->B;
  if (c.transient_scheme == FS_TRANSIENT_CRANKNICOLSON1 && ctx->ndt != 0) {
    // CrankNicolson (CrankNicolsonRoutine.for:51-80,150): extrapolate, then AssembleMdot,
    // whose PressGradf is still the one the last X-momentum solve interpolated
    ctx->tscheme = FS_TRANSIENT_CRANKNICOLSON1;
    for (int q = 0; q < FS_NLEVELS; q++) {
      if (!level_field(ctx, q, false)) continue;   // an equation the case does not solve
      k_cn_extrapolate<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(level_field(ctx, q, false), ctx->old + q * N, N);
      FS_LAUNCH_CHECK();
      if (B) {
        k_cn_extrapolate<<<fs_grid(B), FS_BLOCK, 0, ctx->st>>>(level_field(ctx, q, true), ctx->bold + q * B, B);
        FS_LAUNCH_CHECK();
      }
    }
    int rc = fs_assemble_mdot(ctx, ctx->p_mx);
    if (rc) return rc;
  }
  ctx->tscheme = scheme_in_effect(c.transient_scheme, ctx->ndt);
  // updateVariablesInTime (AdvanceVariablesInTime.for:98-160)
  FS_CK(cudaMemcpyAsync(ctx->oldold, ctx->old, sizeof(double) * FS_NLEVELS * N, cudaMemcpyDeviceToDevice, ctx->st));
  for (int q = 0; q < FS_NLEVELS; q++) {
    if (!level_field(ctx, q, false)) continue;
    FS_CK(cudaMemcpyAsync(ctx->old + q * N, level_field(ctx, q, false), sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->st));
    if (B)
      FS_CK(cudaMemcpyAsync(ctx->bold + q * B, level_field(ctx, q, true), sizeof(double) * B, cudaMemcpyDeviceToDevice, ctx->st));
  }
  // dtOldOld = dtOld; dtOld = dt, in updateVariablesInTime and again in the
  // loop (MainProgram.for:227-228); then SetTimeStepValue
  ctx->dtoo = ctx->dto; ctx->dto = ctx->dt;
  ctx->dtoo = ctx->dto; ctx->dto = ctx->dt;
  ctx->dt = dt_next;
  ctx->time = ctx->time + ctx->dt;
  ctx->ndt++;
  ctx->nIter = 0;
  ctx->div_ref = 0.;   // the divergence check restarts with the time step
  return FS_OK;
}

int fs_get_time(fs_ctx *ctx, double t[4], int32_t *n_steps) {
  if (!ctx || !t || !n_steps) return FS_E_ARG;
  t[0] = ctx->time; t[1] = ctx->dt; t[2] = ctx->dto; t[3] = ctx->dtoo;
  *n_steps = ctx->ndt;
  return FS_OK;
}

int fs_set_time(fs_ctx *ctx, const double t[4], int32_t n_steps) {
  if (!ctx || !t || n_steps < 0) return FS_E_ARG;
  if (!ctx->cfg.unsteady || !ctx->old) { ctx->err = "fs_set_time: the case is not unsteady"; return FS_E_ARG; }
  ctx->time = t[0]; ctx->dt = t[1]; ctx->dto = t[2]; ctx->dtoo = t[3];
  ctx->ndt = n_steps;
  // the scheme the step just taken ran with
  ctx->tscheme = scheme_in_effect(ctx->cfg.transient_scheme, n_steps > 0 ? n_steps - 1 : 0);
  return FS_OK;
}

// ------------------------------------------------ adaptive time step
// AdaptiveTimeStep of a laminar, isothermal case (CalculateAdaptiveTimeStep.for:4-200
// and the 'velx' branch of CalculateAdaptiveTimeStepValue, :203-1758).  The
// reference scatters over faces into TimeStep(cell); here one thread per cell
// gathers its slots (faces in increasing index) in the reference's loop order:
// interior diffusion, the boundary lists in the order the reference visits
// them, interior convection, boundary convection.  Each block writes the max
// of TimeStep / (rho V) over its cells; one CTA reduces the partials.
namespace {

struct DtArgs {
  int N, F, B, inviscid, nblk;
  const int32_t *ncf, *slot, *btype;
  const double *gf, *gdiff, *bfa, *bnf, *bdv, *bgdiff, *mdot, *bmdot, *vol;
  double rho, mu;
  double *part, *out;
};

__device__ __forceinline__ double block_max(double v, double *sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  return sh[0];
}

__global__ void __launch_bounds__(FS_BLOCK) k_adaptive_dt(DtArgs a) {
  __shared__ double sh[FS_BLOCK];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double val = -1.;
  if (i < a.N) {
    const int N = a.N, F = a.F, B = a.B, nc = a.ncf[i];
    const double mu = a.mu;
    double ts = 0.;
    if (!a.inviscid) {
      for (int j = 0; j < nc; j++) {   // :329-346
        const int f = a.slot[(long)j * N + i] >> 1;
        if (f < F) {
          const double g = a.gf[f];
          const double gamf = g * mu + (1. - g) * mu;
          ts = ts + gamf * a.gdiff[f];
        }
      }
      // the boundary lists of :384-589, in that order
      const int order[7] = {FS_BC_WALL_NOSLIP, FS_BC_INLET_VEL, FS_BC_INLET_MASS, FS_BC_INLET_SP,
                            FS_BC_INLET_STAG, FS_BC_OUTLET_MASS, FS_BC_SYMMETRY};
      for (int l = 0; l < 7; l++)
        for (int j = 0; j < nc; j++) {
          const int f = a.slot[(long)j * N + i] >> 1;
          if (f < F) continue;
          const int b = f - F;
          if (a.btype[b] != order[l]) continue;
          if (order[l] == FS_BC_WALL_NOSLIP || order[l] == FS_BC_SYMMETRY) {
            const double nx = a.bnf[b], ny = a.bnf[B + b], nz = a.bnf[2L * B + b];
            const double dN = a.bdv[b] * nx + a.bdv[B + b] * ny + a.bdv[2L * B + b] * nz;
            const double area = a.bfa[b];
            double fl;
            if (order[l] == FS_BC_WALL_NOSLIP) {
              fl = mu * area * (1. - nx * nx) / dN;
              fl = fmax(fl, mu * area * (1. - ny * ny) / dN);
              fl = fmax(fl, mu * area * (1. - nz * nz) / dN);
            } else {
              fl = 2. * mu * area * (nx * nx) / dN;
              fl = fmax(fl, 2. * mu * area * (ny * ny) / dN);
              fl = fmax(fl, 2. * mu * area * (nz * nz) / dN);
            }
            ts = ts + fl;
          } else {
            ts = ts + mu * a.bgdiff[b];
          }
        }
    }
    // convection (:1685-1708); the neighbour side subtracts, as the reference writes it
    for (int j = 0; j < nc; j++) {
      const int s = a.slot[(long)j * N + i], f = s >> 1;
      if (f < F) ts = (s & 1) ? ts - fmax(-a.mdot[f], 0.) : ts + fmax(a.mdot[f], 0.);
    }
    for (int j = 0; j < nc; j++) {
      const int f = a.slot[(long)j * N + i] >> 1;
      if (f >= F) ts = ts + fmax(a.bmdot[f - F], 0.);
    }
    val = ts / (a.rho * a.vol[i]);
  }
  const double m = block_max(val, sh);
  if (threadIdx.x == 0) a.part[blockIdx.x] = m;
}

__global__ void __launch_bounds__(1024) k_adaptive_dt_final(DtArgs a) {
  __shared__ double sh[1024];
  double m = -1.;
  for (int b = threadIdx.x; b < a.nblk; b += blockDim.x) m = fmax(m, a.part[b]);
  m = block_max(m, sh);
  if (threadIdx.x == 0) *a.out = m;
}

}  // namespace

int fs_adaptive_time_step(fs_ctx *ctx, double courant, double min_factor, double max_factor, double *dt_next) {
  if (!ctx || !dt_next) return FS_E_ARG;
  const fs_case &c = ctx->cfg;
  if (!c.unsteady || !ctx->old) { ctx->err = "fs_adaptive_time_step: the case is not unsteady"; return FS_E_ARG; }
  if (c.turbulence || c.energy) {
    ctx->err = "fs_adaptive_time_step: laminar isothermal cases only (the k, epsilon and temperature limits are not built)";
    return FS_E_ARG;
  }
  if (!(courant > 0.) || !(min_factor > 0.) || !(max_factor >= min_factor)) {
    ctx->err = "fs_adaptive_time_step: courant and min_factor must be > 0 and max_factor >= min_factor";
    return FS_E_ARG;
  }
  cudaSetDevice(ctx->dev);
  DtArgs a{};
  a.N = (int)ctx->N; a.F = (int)ctx->F; a.B = (int)ctx->B; a.inviscid = c.inviscid;
  a.nblk = fs_grid(ctx->N);
  a.ncf = ctx->ncf; a.slot = ctx->slot; a.btype = ctx->btype;
  a.gf = ctx->gf; a.gdiff = ctx->gdiff; a.bfa = ctx->bfa; a.bnf = ctx->bnf; a.bdv = ctx->bdv;
  a.bgdiff = ctx->bgdiff; a.mdot = ctx->mdot; a.bmdot = ctx->bmdot; a.vol = ctx->vol;
  a.rho = c.rho; a.mu = c.mu;
  a.part = ctx->red + (long)RED_MAX1 * a.nblk;   // ctx->red holds 16 x nblk doubles
  a.out = ctx->red + (long)RED_NQ * a.nblk;
  k_adaptive_dt<<<a.nblk, FS_BLOCK, 0, ctx->st>>>(a);
  FS_LAUNCH_CHECK();
  k_adaptive_dt_final<<<1, 1024, 0, ctx->st>>>(a);
  FS_LAUNCH_CHECK();
  double mx = 0.;
  FS_CK(cudaMemcpyAsync(&mx, a.out, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  FS_CK(cudaStreamSynchronize(ctx->st));
  // dtlocal = GlobalCourantNumber / max, then the change-factor clamp (:192-193)
  double dtl = courant / mx;
  dtl = fmax(dtl, min_factor * ctx->dt);
  *dt_next = fmin(dtl, max_factor * ctx->dt);
  return FS_OK;
}
