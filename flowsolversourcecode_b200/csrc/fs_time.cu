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
