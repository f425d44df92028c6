// fs_capi.cu -- the extern "C" entry points of include/fsb200.h.
#include "fs_internal.cuh"
#include <cmath>
#include <cstring>
#include <new>

namespace {

__global__ void k_initial_mdot(int N, int F, int B, double rho, const int32_t *fown, const int32_t *fnbr,
                               const double *gf, const double *sf, const double *u, const double *v,
                               const double *w, double *mdot, const int32_t *btype, const double *bsf,
                               const double *bu, const double *bv, const double *bw, double *bmdot) {
  // CalculateInitialmdot (ContinuityEquation/InitializaMdot.for:20-60), Densityf = rho
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < F) {
    int k = (int)t, i = fown[k], j = fnbr[k];
    double g = gf[k];
    double uf = g * u[i] + (1. - g) * u[j];
    double vf = g * v[i] + (1. - g) * v[j];
    double wf = g * w[i] + (1. - g) * w[j];
    mdot[k] = rho * (uf * sf[k] + vf * sf[F + k] + wf * sf[2L * F + k]);
  } else if (t < (long)F + B) {
    int b = (int)(t - F), ty = btype[b];
    if (ty == FS_BC_WALL_NOSLIP || ty == FS_BC_WALL_SLIP) bmdot[b] = 0.;
    else if (ty != FS_BC_INLET_MASS && ty != FS_BC_OUTLET_MASS)   // specified mass flow (InitializaMdot.for:55,66)
      bmdot[b] = rho * (bsf[b] * bu[b] + bsf[B + b] * bv[b] + bsf[2L * B + b] * bw[b]);
  }
}

__global__ void k_divide(int N, double *ac, double urf) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) ac[i] = ac[i] / urf;
}

__device__ double blk_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.;
  if (wid == 0) {
    r = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  return r;
}
__device__ double blk_max(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = -1e300;
  if (wid == 0) {
    r = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : -1e300;
    for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, o));
  }
  return r;
}

// CalculateResiduals at dphi=0 on the current system (CalculateResidualsRoutine.for:30-67)
__global__ void k_residual_partials(int N, const double *ac, const double *bc, const double *fi, double *red, int nblk) {
  __shared__ double sh[32];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double r = 0., acphi = -1.;
  if (i < N) { r = fabs(bc[i]); acphi = fabs(ac[i] * fi[i]); }
  double s0 = blk_sum(r, sh), s1 = blk_sum(r * r, sh), m0 = blk_max(r, sh), m1 = blk_max(acphi, sh);
  if (threadIdx.x == 0) {
    red[RED_SUM0 * nblk + blockIdx.x] = s0; red[RED_SUM1 * nblk + blockIdx.x] = s1;
    red[RED_MAX0 * nblk + blockIdx.x] = m0; red[RED_MAX1 * nblk + blockIdx.x] = m1;
  }
}
__global__ void k_residual_final2(const double *red, int nblk, int N, int q, double *rb) {
  __shared__ double sh[32];
  double s0 = 0., s1 = 0., m0 = -1., m1 = -1.;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    s0 += red[RED_SUM0 * nblk + b]; s1 += red[RED_SUM1 * nblk + b];
    m0 = fmax(m0, red[RED_MAX0 * nblk + b]); m1 = fmax(m1, red[RED_MAX1 * nblk + b]);
  }
  s0 = blk_sum(s0, sh); s1 = blk_sum(s1, sh); m0 = blk_max(m0, sh); m1 = blk_max(m1, sh);
  if (threadIdx.x == 0) {
    rb[RB_ABS + q] = s0; rb[RB_MAX + q] = m0; rb[RB_RMS + q] = sqrt(s1 / N);
    rb[RB_SCL + q] = (q == 3) ? 0. : m0 / (m1 + 1.0e-15);
  }
}

}  // namespace

static double *field_ptr(fs_ctx *c, int f, size_t *n) {
  const size_t N = c->N, F = c->F, B = c->B, W = c->W;
  switch (f) {
  case FS_F_U: *n = N; return c->u;
  case FS_F_V: *n = N; return c->v;
  case FS_F_W: *n = N; return c->w;
  case FS_F_P: *n = N; return c->p;
  case FS_F_PC: *n = N; return c->pc;
  case FS_F_MDOT: *n = F; return c->mdot;
  case FS_F_BU: *n = B; return c->bu;
  case FS_F_BV: *n = B; return c->bv;
  case FS_F_BW: *n = B; return c->bw;
  case FS_F_BP: *n = B; return c->bp;
  case FS_F_BPC: *n = B; return c->bpc;
  case FS_F_BMDOT: *n = B; return c->bmdot;
  case FS_F_AC: *n = N; return c->ac;
  case FS_F_BC: *n = N; return c->bc;
  case FS_F_ANB: *n = W * N; return c->anb;
  case FS_F_DU1: *n = N; return c->du1;
  case FS_F_DV1: *n = N; return c->dv1;
  case FS_F_DW1: *n = N; return c->dw1;
  case FS_F_DU2: *n = N; return c->du2;
  case FS_F_DV2: *n = N; return c->dv2;
  case FS_F_DW2: *n = N; return c->dw2;
  case FS_F_UGRAD: *n = 3 * N; return c->ug;
  case FS_F_VGRAD: *n = 3 * N; return c->vg;
  case FS_F_WGRAD: *n = 3 * N; return c->wg;
  case FS_F_PGRAD: *n = 3 * N; return c->pg;
  case FS_F_PCGRAD: *n = 3 * N; return c->pcg;
  case FS_F_VOLUME: *n = N; return c->vol;
  case FS_F_XC: *n = 3 * N; return c->xc;
  case FS_F_GFACTOR: *n = F; return c->gf;
  case FS_F_SF: *n = 3 * F; return c->sf;
  case FS_F_GDIFF: *n = F; return c->gdiff;
  case FS_F_FT: *n = 3 * F; return c->tf;
  case FS_F_BSF: *n = 3 * B; return c->bsf;
  case FS_F_DPHI: *n = N; return c->dphi;
  case FS_F_KX: *n = N; return c->kx;
  case FS_F_TKE: case FS_F_TED: case FS_F_MUT: case FS_F_BTKE: case FS_F_BTED: case FS_F_BMUT:
  case FS_F_UTAU: case FS_F_YPLUS:
    return fs_turb_field(c, f, n);
  case FS_F_OLD: *n = c->old ? FS_NLEVELS * N : 0; return c->old;
  case FS_F_OLDOLD: *n = c->oldold ? FS_NLEVELS * N : 0; return c->oldold;
  case FS_F_BOLD: *n = c->bold ? FS_NLEVELS * B : 0; return c->bold;
  case FS_F_T: case FS_F_BT: case FS_F_TGRAD:
    return fs_energy_field(c, f, n);
  }
  *n = 0;
  return nullptr;
}

static int alloc0(fs_ctx *ctx, double **p, size_t n) {
  FS_CK(cudaMalloc((void **)p, sizeof(double) * (n ? n : 1)));
  FS_CK(cudaMemsetAsync(*p, 0, sizeof(double) * (n ? n : 1), ctx->st));
  return FS_OK;
}

static void free_all(fs_ctx *c) {
  void *ptrs[] = {c->slot, c->cn, c->ncf, c->fown, c->fnbr, c->bown, c->btype, c->color_rows,
                  c->vol, c->xc, c->gf, c->sf, c->dcfv, c->dcf, c->gdiff, c->tf, c->dfp, c->fa,
                  c->bsf, c->bfa, c->bnf, c->bdv, c->bgdiff, c->btf, c->bnzii,
                  c->u, c->v, c->w, c->p, c->pc, c->mdot, c->bu, c->bv, c->bw, c->bp, c->bpc, c->bmdot,
                  c->ug, c->vg, c->wg, c->pg, c->pcg, c->bug, c->bvg, c->bwg, c->bpg, c->bpcg, c->gtmp,
                  c->du1, c->dv1, c->dw1, c->du2, c->dv2, c->dw2, c->us, c->vs, c->ws,
                  c->ac, c->anb, c->bc, c->dphi, c->ac_int, c->bc_int, c->effdiv, c->pcoef, c->bpcoef,
                  c->kx, c->kr, c->kr0, c->kp, c->kv, c->ks, c->kt, c->kz, c->ky, c->sysx,
                  c->red, c->redi, c->resblk, c->d_iters, c->d_status,
                  c->cposP, c->cnP, c->ncfP, c->acP, c->bcP, c->anbP, c->dphiP,
                  c->ac3, c->bc3, c->ac3P, c->bc3P, c->x3P, c->gm, c->d_bset, c->flow, c->bdir,
                  c->bpcoefc, c->bgd, c->bp0, c->d_patch, c->hist};
  for (void *p : ptrs) if (p) cudaFree(p);
}

extern "C" {

int fs_create(const fs_mesh_in *mesh, const fs_case *cfg, int device, fs_ctx **out) {
  if (!mesh || !cfg || !out) return FS_E_ARG;
  *out = nullptr;
  if (mesh->n_patches != cfg->n_patches || cfg->n_patches > FS_MAX_PATCHES) return FS_E_ARG;
  if (cfg->method_decompose_s < 1 || cfg->method_decompose_s > 3) return FS_E_ARG;
  fs_ctx *ctx = new (std::nothrow) fs_ctx();
  if (!ctx) return FS_E_NOMEM;
  ctx->cfg = *cfg;
  ctx->dev = device;
  int rc = FS_OK;
  auto fail = [&](int r) { fs_transient_free(ctx); fs_energy_free(ctx); fs_turb_free(ctx); free_all(ctx); if (ctx->st) cudaStreamDestroy(ctx->st); delete ctx; return r; };
  if (cudaSetDevice(device) != cudaSuccess) return fail(FS_E_CUDA);
  if (cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking) != cudaSuccess) return fail(FS_E_CUDA);
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  for (auto &e : ctx->ev) cudaEventCreate(&e);
  for (auto &e : ctx->tev) cudaEventCreate(&e);
  for (auto &pr : ctx->sev) { cudaEventCreate(&pr[0]); cudaEventCreate(&pr[1]); }
  for (auto &pr : ctx->kev) { cudaEventCreate(&pr[0]); cudaEventCreate(&pr[1]); }
  for (int s = 0; s < ctx->cfg.n_patches; s++) {
    ctx->has_sp |= fs_is_pressure(ctx->cfg.patch_type[s]);
    ctx->has_res |= ctx->cfg.patch_type[s] == FS_BC_OUTLET_RES;
    ctx->has_stag |= ctx->cfg.patch_type[s] == FS_BC_INLET_STAG;
  }
  // SetReferencePressure (ReferenceAndSetPressureRoutines.for:4-50): a pressure-specified patch fixes the level
  if (ctx->cfg.set_reference_pressure < 0) ctx->cfg.set_reference_pressure = ctx->has_sp ? 1 : 0;
  if ((rc = fs_geometry_build(ctx, mesh))) { std::string e = ctx->err; fprintf(stderr, "fs_create: %s\n", e.c_str()); return fail(rc); }
  const size_t N = ctx->N, F = ctx->F, B = ctx->B, W = ctx->W;
  if (ctx->cfg.ref_pressure_cell >= (int)N) return fail(FS_E_ARG);
  double **cellv[] = {&ctx->u, &ctx->v, &ctx->w, &ctx->p, &ctx->pc, &ctx->du1, &ctx->dv1, &ctx->dw1, &ctx->du2,
                      &ctx->dv2, &ctx->dw2, &ctx->us, &ctx->vs, &ctx->ws, &ctx->ac, &ctx->bc, &ctx->dphi,
                      &ctx->ac_int, &ctx->effdiv, &ctx->kx, &ctx->kr, &ctx->kr0, &ctx->kp, &ctx->kv, &ctx->ks,
                      &ctx->kt, &ctx->kz, &ctx->ky, &ctx->sysx};
  for (auto p : cellv) if ((rc = alloc0(ctx, p, N))) return fail(rc);
  if ((rc = alloc0(ctx, &ctx->acP, N)) || (rc = alloc0(ctx, &ctx->bcP, N)) || (rc = alloc0(ctx, &ctx->dphiP, N)) ||
      (rc = alloc0(ctx, &ctx->anbP, W * N)))
    return fail(rc);
  if (ctx->cfg.batched_momentum &&
      ((rc = alloc0(ctx, &ctx->ac3, 3 * N)) || (rc = alloc0(ctx, &ctx->bc3, 3 * N)) || (rc = alloc0(ctx, &ctx->ac3P, 3 * N)) ||
       (rc = alloc0(ctx, &ctx->bc3P, 3 * N)) || (rc = alloc0(ctx, &ctx->x3P, 3 * N))))
    return fail(rc);
  double **cell3[] = {&ctx->ug, &ctx->vg, &ctx->wg, &ctx->pg, &ctx->pcg, &ctx->bc_int};
  for (auto p : cell3) if ((rc = alloc0(ctx, p, 3 * N))) return fail(rc);
  if ((rc = alloc0(ctx, &ctx->gtmp, 12 * N))) return fail(rc);
  if ((rc = alloc0(ctx, &ctx->anb, W * N))) return fail(rc);
  if ((rc = alloc0(ctx, &ctx->mdot, F)) || (rc = alloc0(ctx, &ctx->pcoef, F)) || (rc = alloc0(ctx, &ctx->bpcoef, B)) ||
      (rc = alloc0(ctx, &ctx->bpcoefc, B)) || (rc = alloc0(ctx, &ctx->bgd, B)) || (rc = alloc0(ctx, &ctx->bp0, B)) ||
      (rc = alloc0(ctx, &ctx->d_patch, 2 * FS_MAX_PATCHES)))
    return fail(rc);
  double **bnd[] = {&ctx->bu, &ctx->bv, &ctx->bw, &ctx->bp, &ctx->bpc, &ctx->bmdot};
  for (auto p : bnd) if ((rc = alloc0(ctx, p, B))) return fail(rc);
  double **bnd3[] = {&ctx->bug, &ctx->bvg, &ctx->bwg, &ctx->bpg, &ctx->bpcg};
  for (auto p : bnd3) if ((rc = alloc0(ctx, p, 3 * B))) return fail(rc);
  size_t nblk = (size_t)fs_grid((long)N);
  size_t nred = 16 * (nblk > FS_RED_BLOCKS ? nblk : FS_RED_BLOCKS);   // three components' partials (k_mom_finish3)
  if ((rc = alloc0(ctx, &ctx->red, nred))) return fail(rc);
  if (cudaMalloc(&ctx->redi, sizeof(int64_t) * (nblk > FS_RED_BLOCKS ? nblk : FS_RED_BLOCKS)) != cudaSuccess) return fail(FS_E_NOMEM);
  if ((rc = alloc0(ctx, &ctx->resblk, RB_SIZE))) return fail(rc);
  if (cudaMalloc(&ctx->d_iters, sizeof(int32_t) * FS_NITERS) != cudaSuccess) return fail(FS_E_NOMEM);
  cudaMemsetAsync(ctx->d_iters, 0, sizeof(int32_t) * FS_NITERS, ctx->st);
  if (cudaMalloc(&ctx->d_status, sizeof(int32_t) * 8) != cudaSuccess) return fail(FS_E_NOMEM);
  cudaMemsetAsync(ctx->d_status, 0, sizeof(int32_t) * 8, ctx->st);
  if ((rc = alloc0(ctx, &ctx->flow, 1 + 2 * FS_MAX_PATCHES))) return fail(rc);
  if (cudaMalloc(&ctx->d_bset, sizeof(int32_t) * (B ? B : 1)) != cudaSuccess) return fail(FS_E_NOMEM);
  if (B) cudaMemcpyAsync(ctx->d_bset, ctx->h_bset.data(), sizeof(int32_t) * B, cudaMemcpyHostToDevice, ctx->st);
  if ((rc = fs_turb_create(ctx))) return fail(rc);
  if ((rc = fs_energy_create(ctx))) { std::string e = ctx->err; fprintf(stderr, "fs_create: %s\n", e.c_str()); return fail(rc); }
  if ((rc = fs_set_pc_history(ctx, ctx->cfg.pc_history))) { ctx->err = "pc_history must be 0..7"; return fail(rc); }
  // boundary values from the patches (setBoundaryConditions): wall / inlet velocities
  std::vector<double> hb(3 * B, 0.);
  for (size_t b = 0; b < B; b++) {
    int s = ctx->h_bset[b], t = ctx->cfg.patch_type[s];
    if (t == FS_BC_WALL_NOSLIP || t == FS_BC_INLET_VEL) {
      hb[b] = ctx->cfg.patch_vel[s][0]; hb[B + b] = ctx->cfg.patch_vel[s][1]; hb[2 * B + b] = ctx->cfg.patch_vel[s][2];
    }
  }
  std::vector<double> hp(B, 0.);   // static pressure of 'specifiedstaticpressure' outlets
  for (size_t b = 0; b < B; b++) {
    int s = ctx->h_bset[b];
    if (fs_is_pressure(ctx->cfg.patch_type[s])) hp[b] = ctx->cfg.patch_pressure[s];
  }
  // 'specifiedmassflowrate' inlets: Bmdot = -mdot |S_f| / sum |S| in face order, and the
  // velocity AssembleMdot derives from it (AssembleMdotUsingRhieChow.for:2077-2100)
  std::vector<double> hm(B, 0.);
  bool has_mass = false;
  for (int s = 0; s < ctx->cfg.n_patches; s++)
    has_mass |= ctx->cfg.patch_type[s] == FS_BC_INLET_MASS || fs_is_p_inlet(ctx->cfg.patch_type[s]) ||
                ctx->cfg.patch_type[s] == FS_BC_OUTLET_MASS;
  if (has_mass && B) {
    std::vector<double> hfa(B), hsf(3 * B), hd(3 * B, 0.);
    if (cudaStreamSynchronize(ctx->st) != cudaSuccess ||
        cudaMemcpy(hfa.data(), ctx->bfa, sizeof(double) * B, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(hsf.data(), ctx->bsf, sizeof(double) * 3 * B, cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(FS_E_CUDA);
    for (int s = 0; s < ctx->cfg.n_patches; s++) {
      const int b0 = ctx->h_bset_start[s], nb = ctx->h_bset_n[s];
      const double *d = ctx->cfg.patch_vel[s], rho = ctx->cfg.rho;
      if (fs_is_p_inlet(ctx->cfg.patch_type[s]))   // direction only
        for (int j = 0; j < nb; j++) for (int q = 0; q < 3; q++) hd[3 * (size_t)(b0 + j) + q] = d[q];
      if (ctx->cfg.patch_type[s] == FS_BC_OUTLET_MASS) {   // outflow: Bmdot > 0; velocity from the first mdot assembly
        double area = 0.;
        for (int j = 0; j < nb; j++) area = area + hfa[b0 + j];
        for (int j = 0; j < nb; j++) hm[b0 + j] = ctx->cfg.patch_mass_flow[s] * hfa[b0 + j] / area;
      }
      if (ctx->cfg.patch_type[s] != FS_BC_INLET_MASS) continue;
      double area = 0.;
      for (int j = 0; j < nb; j++) area = area + hfa[b0 + j];
      for (int j = 0; j < nb; j++) {
        const size_t b = b0 + j;
        for (int q = 0; q < 3; q++) hd[3 * b + q] = d[q];
        hm[b] = -(ctx->cfg.patch_mass_flow[s] * hfa[b] / area);
        const double vm = hm[b] / (rho * (d[0] * hsf[b] + d[1] * hsf[B + b] + d[2] * hsf[2 * B + b]));
        hb[b] = vm * d[0]; hb[B + b] = vm * d[1]; hb[2 * B + b] = vm * d[2];
      }
    }
    if (cudaMalloc(&ctx->bdir, sizeof(double) * 3 * B) != cudaSuccess) return fail(FS_E_NOMEM);
    cudaMemcpyAsync(ctx->bdir, hd.data(), sizeof(double) * 3 * B, cudaMemcpyHostToDevice, ctx->st);
    cudaMemcpyAsync(ctx->bmdot, hm.data(), sizeof(double) * B, cudaMemcpyHostToDevice, ctx->st);
  }
  if (B) {
    cudaMemcpyAsync(ctx->bp, hp.data(), sizeof(double) * B, cudaMemcpyHostToDevice, ctx->st);
    cudaMemcpyAsync(ctx->bp0, hp.data(), sizeof(double) * B, cudaMemcpyHostToDevice, ctx->st);
    // ArteryResistance per patch ('specifiedresistance'); the patch sums of geoDiff follow
    cudaMemcpyAsync(ctx->d_patch, ctx->cfg.patch_resistance, sizeof(double) * FS_MAX_PATCHES, cudaMemcpyHostToDevice,
                    ctx->st);
    cudaMemcpyAsync(ctx->bu, hb.data(), sizeof(double) * B, cudaMemcpyHostToDevice, ctx->st);
    cudaMemcpyAsync(ctx->bv, hb.data() + B, sizeof(double) * B, cudaMemcpyHostToDevice, ctx->st);
    cudaMemcpyAsync(ctx->bw, hb.data() + 2 * B, sizeof(double) * B, cudaMemcpyHostToDevice, ctx->st);
  }
  k_initial_mdot<<<fs_grid((long)F + B), FS_BLOCK, 0, ctx->st>>>((int)N, (int)F, (int)B, ctx->cfg.rho, ctx->fown, ctx->fnbr,
      ctx->gf, ctx->sf, ctx->u, ctx->v, ctx->w, ctx->mdot, ctx->btype, ctx->bsf, ctx->bu, ctx->bv, ctx->bw, ctx->bmdot);
  ctx->launches++;
  if ((rc = fs_transient_create(ctx))) { std::string e = ctx->err; fprintf(stderr, "fs_create: %s\n", e.c_str()); return fail(rc); }
  if (cudaStreamSynchronize(ctx->st) != cudaSuccess || cudaGetLastError() != cudaSuccess) return fail(FS_E_CUDA);
  *out = ctx;
  return FS_OK;
}

int fs_destroy(fs_ctx *ctx) {
  if (!ctx) return FS_OK;
  cudaSetDevice(ctx->dev);
  if (ctx->st) cudaStreamSynchronize(ctx->st);
  fs_mg_free(ctx);
  fs_ilu_free(ctx);
  fs_nn_free(ctx);
  fs_turb_free(ctx);
  fs_energy_free(ctx);
  fs_transient_free(ctx);
  free_all(ctx);
  for (auto &e : ctx->ev) if (e) cudaEventDestroy(e);
  for (auto &e : ctx->tev) if (e) cudaEventDestroy(e);
  for (auto &pr : ctx->sev) { if (pr[0]) cudaEventDestroy(pr[0]); if (pr[1]) cudaEventDestroy(pr[1]); }
  for (auto &pr : ctx->kev) { if (pr[0]) cudaEventDestroy(pr[0]); if (pr[1]) cudaEventDestroy(pr[1]); }
  if (ctx->st) cudaStreamDestroy(ctx->st);
  delete ctx;
  return FS_OK;
}

int fs_sizes(const fs_ctx *ctx, int32_t *n, int32_t *f, int32_t *b, int32_t *w) {
  if (!ctx) return FS_E_ARG;
  if (n) *n = ctx->N;
  if (f) *f = ctx->F;
  if (b) *b = ctx->B;
  if (w) *w = ctx->W;
  return FS_OK;
}

const char *fs_last_error(const fs_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int fs_solve_momentum(fs_ctx *ctx, int comp) {
  if (!ctx || comp < 0 || comp > 2) return FS_E_ARG;
  int rc = fs_momentum_assemble(ctx, comp);
  if (rc) return rc;
  double *fi = comp == 0 ? ctx->u : comp == 1 ? ctx->v : ctx->w;
  return fs_linear_solve(ctx, comp + 1, fi, ctx->cfg.rrf_mom, ctx->cfg.itmax_mom, ctx->cfg.solver_mom);
}

// the p' solve with its initial-guess basis: the previous p' solutions kept
// by fs_set_pc_history (slot 0 the newest) and the network's guess.  The
// slots shift by device copies after each solve, so the pointers stay fixed and
// the solve can be captured into a graph (the network's guess, which needs host
// bookkeeping, is left out there).  With pc_defer the Krylov launch itself is
// left to fs_pc_batch_launch between pc_solve_pre and pc_solve_post.
static int pc_solve_pre(fs_ctx *ctx) {
  const double *x0 = nullptr;
  int rc;
  if (!ctx->graph_mode && (rc = fs_nn_before_pc(ctx, &x0))) return rc;
  const size_t N = ctx->N;
  ctx->pc_nguess = 0;
  for (int q = 0; q < ctx->hist_cnt && ctx->pc_nguess < FS_GUESS_MAX - 1; q++)
    ctx->pc_guess[ctx->pc_nguess++] = ctx->hist + (size_t)q * N;
  ctx->pc_nn = x0 != nullptr;
  if (x0) ctx->pc_guess[ctx->pc_nguess++] = x0;
  rc = fs_linear_solve(ctx, FS_VAR_PC, ctx->pc, ctx->cfg.rrf_cont, ctx->cfg.itmax_cont, ctx->cfg.solver_cont);
  ctx->pc_nguess = 0;
  ctx->pc_nn = false;
  return rc;
}

static int pc_solve_post(fs_ctx *ctx) {
  int rc;
  if (ctx->pc_defer && (rc = fs_linear_solve_finish(ctx, FS_VAR_PC, ctx->pc))) return rc;
  const size_t N = ctx->N;
  if (ctx->hist_cap > 0) {
    for (int q = std::min(ctx->hist_cnt, ctx->hist_cap - 1); q >= 1; q--)
      FS_CK(cudaMemcpyAsync(ctx->hist + (size_t)q * N, ctx->hist + (size_t)(q - 1) * N, sizeof(double) * N,
                            cudaMemcpyDeviceToDevice, ctx->st));
    FS_CK(cudaMemcpyAsync(ctx->hist, ctx->dphi, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->st));
    ctx->hist_cnt = std::min(ctx->hist_cnt + 1, ctx->hist_cap);
  }
  return ctx->graph_mode ? FS_OK : fs_nn_after_pc(ctx);
}

static int pc_solve(fs_ctx *ctx) {
  int rc = pc_solve_pre(ctx);
  if (rc) return rc;
  return pc_solve_post(ctx);
}

int fs_set_pc_history(fs_ctx *ctx, int m) {
  if (!ctx || m < 0 || m > FS_GUESS_MAX - 1) return FS_E_ARG;
  cudaSetDevice(ctx->dev);
  if (ctx->hist) { FS_CK(cudaStreamSynchronize(ctx->st)); cudaFree(ctx->hist); ctx->hist = nullptr; }
  ctx->hist_cap = ctx->hist_cnt = 0;
  if (m == 0) return FS_OK;
  FS_CK(cudaMalloc(&ctx->hist, sizeof(double) * (size_t)m * ctx->N));
  ctx->hist_cap = m;
  return FS_OK;
}

int fs_solve_energy(fs_ctx *ctx) {
  if (!ctx) return FS_E_ARG;
  if (!ctx->energy) { ctx->err = "fs_solve_energy: the case does not solve the temperature equation"; return FS_E_ARG; }
  cudaSetDevice(ctx->dev);
  return fs_energy_solve(ctx);
}

int fs_solve_continuity(fs_ctx *ctx) {
  if (!ctx) return FS_E_ARG;
  int rc = fs_continuity_assemble(ctx);
  if (rc) return rc;
  if ((rc = pc_solve(ctx))) return rc;
  return fs_continuity_correct(ctx);
}

int fs_assemble_momentum(fs_ctx *ctx, int comp) {
  if (!ctx || comp < 0 || comp > 2) return FS_E_ARG;
  return fs_momentum_assemble(ctx, comp);
}
int fs_assemble_continuity(fs_ctx *ctx) { return ctx ? fs_continuity_assemble(ctx) : FS_E_ARG; }
int fs_correct_continuity(fs_ctx *ctx) { return ctx ? fs_continuity_correct(ctx) : FS_E_ARG; }
int fs_set_iteration(fs_ctx *ctx, int n_iter) {
  if (!ctx) return FS_E_ARG;
  ctx->nIter = n_iter;
  return FS_OK;
}

int fs_initialize_mdot(fs_ctx *ctx) {
  if (!ctx) return FS_E_ARG;
  cudaSetDevice(ctx->dev);
  const int N = ctx->N, F = ctx->F, B = ctx->B;
  k_initial_mdot<<<fs_grid((long)F + B), FS_BLOCK, 0, ctx->st>>>(N, F, B, ctx->cfg.rho, ctx->fown, ctx->fnbr,
      ctx->gf, ctx->sf, ctx->u, ctx->v, ctx->w, ctx->mdot, ctx->btype, ctx->bsf, ctx->bu, ctx->bv, ctx->bw, ctx->bmdot);
  FS_LAUNCH_CHECK();
  FS_CK(cudaStreamSynchronize(ctx->st));
  return FS_OK;
}

// PrintConvergenceHistory stop metric (PrintConvergenceToFileAndScreen.for:613-700)
// from a device residual block
static double stop_metric(const fs_case &c, const double *rb) {
  const int o = c.nstop_type == 1 ? RB_ABS : c.nstop_type == 2 ? RB_MAX : c.nstop_type == 3 ? RB_RMS : RB_SCL;
  double s = 0.;
  s = fmax(s, fmax(fabs(rb[o]), fmax(fabs(rb[o + 1]), fabs(rb[o + 2]))));
  s = fmax(s, fabs(rb[o + 4]));
  if (c.turbulence) { s = fmax(s, fabs(rb[o + FS_VAR_TKE - 1])); s = fmax(s, fabs(rb[o + FS_VAR_TED - 1])); }
  if (c.energy) s = fmax(s, fabs(rb[o + FS_VAR_TEMP - 1]));
  return s;
}

static int read_residuals(fs_ctx *ctx, fs_residuals *res) {
  double rb[RB_SIZE];
  int32_t it[FS_NITERS];
  FS_CK(cudaMemcpyAsync(rb, ctx->resblk, sizeof(rb), cudaMemcpyDeviceToHost, ctx->st));
  FS_CK(cudaMemcpyAsync(it, ctx->d_iters, sizeof(it), cudaMemcpyDeviceToHost, ctx->st));
  int32_t status = 0;
  FS_CK(cudaMemcpyAsync(&status, ctx->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->st));
  FS_CK(cudaStreamSynchronize(ctx->st));
  if (status) {
    // a bounded device wait gave up: the iteration's results are not valid
    FS_CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int32_t), ctx->st));
    ctx->err = "a bounded device wait (multigrid team barrier or tensor-core completion) timed out";
    return FS_E_TIMEOUT;
  }
  fs_solver_stats_collect(ctx);
  fs_residuals r{};
  for (int q = 0; q < 5; q++) {
    r.abs_[q] = rb[RB_ABS + q]; r.max_[q] = rb[RB_MAX + q]; r.rms[q] = rb[RB_RMS + q]; r.scaled[q] = rb[RB_SCL + q];
    r.lin_iters[q] = it[q];
  }
  for (int q = 0; q < 2; q++) {
    const int e = FS_VAR_TKE - 1 + q;
    r.turb_abs[q] = rb[RB_ABS + e]; r.turb_max[q] = rb[RB_MAX + e]; r.turb_rms[q] = rb[RB_RMS + e];
    r.turb_scaled[q] = rb[RB_SCL + e]; r.turb_lin_iters[q] = it[e];
  }
  {
    const int e = FS_VAR_TEMP - 1;
    r.temp_abs = rb[RB_ABS + e]; r.temp_max = rb[RB_MAX + e]; r.temp_rms = rb[RB_RMS + e];
    r.temp_scaled = rb[RB_SCL + e]; r.temp_lin_iters = it[e];
  }
  if (ctx->nn) fs_nn_note_iters(ctx, it[FS_VAR_PC - 1]);
  r.overall_imbalance = rb[RB_OVERALL];
  r.imax_imbalance = (int)rb[RB_IMAX];
  r.source = stop_metric(ctx->cfg, rb);
  if (res) *res = r;
  for (int q = 0; q < 5; q++)
    if (!std::isfinite(r.abs_[q])) { ctx->err = "NaN/Inf residual"; return FS_E_NAN; }
  if (ctx->cfg.turbulence)
    for (int q = 0; q < 2; q++)
      if (!std::isfinite(r.turb_abs[q])) { ctx->err = "NaN/Inf residual"; return FS_E_NAN; }
  if (ctx->cfg.energy && !std::isfinite(r.temp_abs)) { ctx->err = "NaN/Inf residual"; return FS_E_NAN; }
  // divergence: the stop metric grew past FS_DIVERGENCE_FACTOR times the largest
  // one of the earlier outer iterations of the run (or of the time step)
  if (std::isfinite(r.source) && r.source > 0.) {
    if (ctx->div_ref > 0. && r.source > FS_DIVERGENCE_FACTOR * ctx->div_ref) {
      ctx->err = "diverged: the stop metric grew by more than 1e6 over its largest earlier value";
      return FS_E_DIVERGED;
    }
    ctx->div_ref = fmax(ctx->div_ref, r.source);
  }
  return FS_OK;
}

// one SIMPLE outer iteration enqueued on the context stream (MainProgram.for:257-325)
// one SIMPLE iteration in two parts around the p' Krylov launch (MainProgram.for:257-348)
// the momentum part (with mom_defer the multi-RHS SOR launch is left to
// fs_mom_batch_launch), then the part up to the p' Krylov launch
static int iteration_mom(fs_ctx *ctx) {
  int rc;
  FS_TIMING(cudaEventRecord(ctx->ev[0], ctx->st));
  if (ctx->cfg.batched_momentum && ctx->cfg.solver_mom == FS_SOLVER_SOR) {
    if ((rc = fs_momentum_assemble3(ctx))) return rc;
    if ((rc = fs_momentum_batched_solve(ctx))) return rc;
  } else {
    for (int c = 0; c < 3; c++) {
      if ((rc = fs_momentum_assemble(ctx, c))) return rc;
      double *fi = c == 0 ? ctx->u : c == 1 ? ctx->v : ctx->w;
      if ((rc = fs_linear_solve(ctx, c + 1, fi, ctx->cfg.rrf_mom, ctx->cfg.itmax_mom, ctx->cfg.solver_mom))) return rc;
    }
  }
  return FS_OK;
}

static int iteration_mid(fs_ctx *ctx) {
  int rc;
  if (ctx->mom_defer && (rc = fs_momentum_batched_finish(ctx))) return rc;
  FS_TIMING(cudaEventRecord(ctx->ev[1], ctx->st));
  if ((rc = fs_continuity_assemble(ctx))) return rc;
  FS_TIMING(cudaEventRecord(ctx->ev[2], ctx->st));
  return pc_solve_pre(ctx);
}

static int iteration_pre(fs_ctx *ctx) {
  int rc = iteration_mom(ctx);
  if (rc) return rc;
  return iteration_mid(ctx);
}

static int iteration_post(fs_ctx *ctx) {
  int rc;
  if ((rc = pc_solve_post(ctx))) return rc;
  FS_TIMING(cudaEventRecord(ctx->ev[3], ctx->st));
  if ((rc = fs_continuity_correct(ctx))) return rc;
  // CalculateEffectsOfTurbulence (MainProgram.for:275-277), SolveEnergy (:281)
  if ((rc = fs_turb_effects(ctx))) return rc;
  if ((rc = fs_energy_solve(ctx))) return rc;
  FS_TIMING(cudaEventRecord(ctx->ev[4], ctx->st));
  return FS_OK;
}

static int iteration_body(fs_ctx *ctx) {
  int rc = iteration_pre(ctx);
  if (rc) return rc;
  return iteration_post(ctx);
}

static int iteration_enqueue(fs_ctx *ctx) {
  ctx->nIter++;
  return iteration_body(ctx);
}

int fs_simple_iteration(fs_ctx *ctx, fs_residuals *res) {
  if (!ctx) return FS_E_ARG;
  cudaSetDevice(ctx->dev);
  ctx->nIter++;
  int rc = iteration_body(ctx);
  if (rc) return rc;
  rc = read_residuals(ctx, res);
  cudaEventElapsedTime(&ctx->phase_ms[0], ctx->ev[0], ctx->ev[1]);
  cudaEventElapsedTime(&ctx->phase_ms[2], ctx->ev[1], ctx->ev[2]);
  cudaEventElapsedTime(&ctx->phase_ms[3], ctx->ev[2], ctx->ev[3]);
  cudaEventElapsedTime(&ctx->phase_ms[4], ctx->ev[3], ctx->ev[4]);
  ctx->phase_ms[1] = 0.f;
  return rc;
}

int fs_simple_iteration_host(fs_ctx *ctx, double *u, double *v, double *w, double *p, double *mdot,
                             double *bu, double *bv, double *bw, double *bp, double *bmdot, fs_residuals *res) {
  if (!ctx || !u || !v || !w || !p || !mdot || !bu || !bv || !bw || !bp || !bmdot) return FS_E_ARG;
  cudaSetDevice(ctx->dev);
  const size_t N = ctx->N, F = ctx->F, B = ctx->B;
  struct { double *h; double *d; size_t n; } t[] = {{u, ctx->u, N}, {v, ctx->v, N}, {w, ctx->w, N}, {p, ctx->p, N},
      {mdot, ctx->mdot, F}, {bu, ctx->bu, B}, {bv, ctx->bv, B}, {bw, ctx->bw, B}, {bp, ctx->bp, B}, {bmdot, ctx->bmdot, B}};
  for (auto &e : t) if (e.n) FS_CK(cudaMemcpyAsync(e.d, e.h, sizeof(double) * e.n, cudaMemcpyHostToDevice, ctx->st));
  int rc = fs_simple_iteration(ctx, res);
  if (rc) return rc;
  for (auto &e : t) if (e.n) FS_CK(cudaMemcpyAsync(e.h, e.d, sizeof(double) * e.n, cudaMemcpyDeviceToHost, ctx->st));
  FS_CK(cudaStreamSynchronize(ctx->st));
  return FS_OK;
}

int fs_gradient(fs_ctx *ctx, int var, int method, int n_iter) {
  if (!ctx) return FS_E_ARG;
  const double *phi, *bphi;
  double *g, *bg;
  switch (var) {
  case FS_VAR_U: phi = ctx->u; bphi = ctx->bu; g = ctx->ug; bg = ctx->bug; break;
  case FS_VAR_V: phi = ctx->v; bphi = ctx->bv; g = ctx->vg; bg = ctx->bvg; break;
  case FS_VAR_W: phi = ctx->w; bphi = ctx->bw; g = ctx->wg; bg = ctx->bwg; break;
  case FS_VAR_P: phi = ctx->p; bphi = ctx->bp; g = ctx->pg; bg = ctx->bpg; break;
  case FS_VAR_PC: phi = ctx->pc; bphi = ctx->bpc; g = ctx->pcg; bg = ctx->bpcg; break;
  case FS_VAR_TEMP: {
    size_t n;
    phi = fs_energy_field(ctx, FS_F_T, &n); bphi = fs_energy_field(ctx, FS_F_BT, &n);
    g = fs_energy_field(ctx, FS_F_TGRAD, &n);
    bg = fs_energy_bgrad(ctx);
    if (!phi) { ctx->err = "fs_gradient: the case does not solve the temperature equation"; return FS_E_ARG; }
    break;
  }
  default: return FS_E_ARG;
  }
  return fs_gradient_dev(ctx, 1, &var, &phi, &bphi, &g, &bg, &method, &n_iter);
}

int fs_gradient_host(fs_ctx *ctx, int var, int method, int n_iter, const double *phi, const double *bphi,
                     double *grad, double *bgrad) {
  if (!ctx || !phi || !bphi || !grad || !bgrad) return FS_E_ARG;
  if (var != FS_VAR_U && var != FS_VAR_V && var != FS_VAR_W && var != FS_VAR_PC && var != FS_VAR_P &&
      var != FS_VAR_TEMP)
    return FS_E_ARG;
  cudaSetDevice(ctx->dev);
  const size_t N = ctx->N, B = ctx->B;
  // stage through the (otherwise unused during this call) Krylov vectors
  double *dphi_ = ctx->kz, *dbphi = nullptr, *dg = ctx->gtmp + 9 * N, *dbg = nullptr;
  FS_CK(cudaMalloc(&dbphi, sizeof(double) * (B ? B : 1)));
  FS_CK(cudaMalloc(&dbg, sizeof(double) * 3 * (B ? B : 1)));
  FS_CK(cudaMemcpyAsync(dphi_, phi, sizeof(double) * N, cudaMemcpyHostToDevice, ctx->st));
  if (B) FS_CK(cudaMemcpyAsync(dbphi, bphi, sizeof(double) * B, cudaMemcpyHostToDevice, ctx->st));
  // the scratch of field slot 0 of the gradient passes is gtmp[0:3N]; dg sits in slot 3
  double *gout = nullptr;
  FS_CK(cudaMalloc(&gout, sizeof(double) * 3 * N));
  const double *pp = dphi_, *bp = dbphi;
  int rc = fs_gradient_dev(ctx, 1, &var, &pp, &bp, &gout, &dbg, &method, &n_iter);
  (void)dg;
  if (!rc) {
    FS_CK(cudaMemcpyAsync(grad, gout, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, ctx->st));
    if (B) FS_CK(cudaMemcpyAsync(bgrad, dbg, sizeof(double) * 3 * B, cudaMemcpyDeviceToHost, ctx->st));
    FS_CK(cudaStreamSynchronize(ctx->st));
  }
  cudaFree(gout); cudaFree(dbphi); cudaFree(dbg);
  return rc;
}

int fs_under_relax(fs_ctx *ctx, double urf) {
  if (!ctx || urf == 0.) return FS_E_ARG;
  k_divide<<<fs_grid(ctx->N), FS_BLOCK, 0, ctx->st>>>(ctx->N, ctx->ac, urf);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

static int residual_of_system(fs_ctx *ctx, int nf, const double *fi) {
  int nblk = fs_grid(ctx->N);
  k_residual_partials<<<nblk, FS_BLOCK, 0, ctx->st>>>(ctx->N, ctx->ac, ctx->bc, fi, ctx->red, nblk);
  FS_LAUNCH_CHECK();
  k_residual_final2<<<1, 1024, 0, ctx->st>>>(ctx->red, nblk, ctx->N, nf - 1, ctx->resblk);
  FS_LAUNCH_CHECK();
  return FS_OK;
}

int fs_solve_equation(fs_ctx *ctx, int var, double rrf, int itmax, int solver) {
  if (!ctx || ((var < FS_VAR_U || var > FS_VAR_PC) && var != FS_VAR_TEMP)) return FS_E_ARG;
  size_t n;
  double *fi = var == FS_VAR_U ? ctx->u : var == FS_VAR_V ? ctx->v : var == FS_VAR_W ? ctx->w :
               var == FS_VAR_TEMP ? fs_energy_field(ctx, FS_F_T, &n) : ctx->pc;
  if (!fi) { ctx->err = "fs_solve_equation: the case does not solve the temperature equation"; return FS_E_ARG; }
  int rc = residual_of_system(ctx, var, fi);
  if (rc) return rc;
  return fs_linear_solve(ctx, var, fi, rrf, itmax, solver);
}

int fs_solve_system_host(fs_ctx *ctx, const double *ac, const double *anb, const double *bc, double *dphi,
                         double rrf, int itmax, int solver, int *iters) {
  if (!ctx || !ac || !anb || !bc || !dphi) return FS_E_ARG;
  cudaSetDevice(ctx->dev);
  const size_t N = ctx->N, W = ctx->W;
  FS_CK(cudaMemcpyAsync(ctx->ac, ac, sizeof(double) * N, cudaMemcpyHostToDevice, ctx->st));
  FS_CK(cudaMemcpyAsync(ctx->anb, anb, sizeof(double) * N * W, cudaMemcpyHostToDevice, ctx->st));
  FS_CK(cudaMemcpyAsync(ctx->bc, bc, sizeof(double) * N, cudaMemcpyHostToDevice, ctx->st));
  // solve into a zero field so the update equals dphi
  double *fz = ctx->sysx;
  FS_CK(cudaMemsetAsync(fz, 0, sizeof(double) * N, ctx->st));
  int rc = residual_of_system(ctx, FS_VAR_PC, fz);
  if (rc) return rc;
  rc = fs_linear_solve(ctx, FS_VAR_PC, fz, rrf, itmax, solver);
  if (rc) return rc;
  int32_t it = 0;
  FS_CK(cudaMemcpyAsync(dphi, fz, sizeof(double) * N, cudaMemcpyDeviceToHost, ctx->st));
  FS_CK(cudaMemcpyAsync(&it, ctx->d_iters + 3, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->st));
  FS_CK(cudaStreamSynchronize(ctx->st));
  if (iters) *iters = it;
  return FS_OK;
}

int fs_residuals_get(fs_ctx *ctx, fs_residuals *res) {
  if (!ctx || !res) return FS_E_ARG;
  return read_residuals(ctx, res);
}

int fs_get_field(fs_ctx *ctx, int field, double *host, size_t n) {
  if (!ctx || !host) return FS_E_ARG;
  size_t m = 0;
  double *d = field_ptr(ctx, field, &m);
  if (!d || n != m) { ctx->err = "field id or size mismatch"; return FS_E_ARG; }
  FS_CK(cudaMemcpyAsync(host, d, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
  FS_CK(cudaStreamSynchronize(ctx->st));
  return FS_OK;
}

int fs_set_field(fs_ctx *ctx, int field, const double *host, size_t n) {
  if (!ctx || !host) return FS_E_ARG;
  size_t m = 0;
  double *d = field_ptr(ctx, field, &m);
  if (!d || n != m) { ctx->err = "field id or size mismatch"; return FS_E_ARG; }
  FS_CK(cudaMemcpyAsync(d, host, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->st));
  FS_CK(cudaStreamSynchronize(ctx->st));
  return FS_OK;
}

int fs_get_connectivity(fs_ctx *ctx, int32_t *ncf, int32_t *cf, int32_t *cn, int32_t *own_slot, int32_t *nbr_slot) {
  if (!ctx) return FS_E_ARG;
  const size_t N = ctx->N, W = ctx->W, F = ctx->F;
  if (ncf) memcpy(ncf, ctx->h_ncf.data(), sizeof(int32_t) * N);
  if (cf) memcpy(cf, ctx->h_cf.data(), sizeof(int32_t) * N * W);
  if (cn) memcpy(cn, ctx->h_cn.data(), sizeof(int32_t) * N * W);
  if (own_slot) memcpy(own_slot, ctx->h_own_slot.data(), sizeof(int32_t) * F);
  if (nbr_slot) memcpy(nbr_slot, ctx->h_nbr_slot.data(), sizeof(int32_t) * F);
  return FS_OK;
}

int fs_phase_times(fs_ctx *ctx, float *ms5) {
  if (!ctx || !ms5) return FS_E_ARG;
  for (int i = 0; i < 5; i++) ms5[i] = ctx->phase_ms[i];
  return FS_OK;
}

int64_t fs_launch_count(const fs_ctx *ctx) { return ctx ? ctx->launches : -1; }

int fs_timer_start(fs_ctx *ctx) {
  if (!ctx) return FS_E_ARG;
  FS_CK(cudaEventRecord(ctx->tev[0], ctx->st));
  return FS_OK;
}

int fs_timer_stop(fs_ctx *ctx, float *ms) {
  if (!ctx || !ms) return FS_E_ARG;
  FS_CK(cudaEventRecord(ctx->tev[1], ctx->st));
  FS_CK(cudaEventSynchronize(ctx->tev[1]));
  FS_CK(cudaEventElapsedTime(ms, ctx->tev[0], ctx->tev[1]));
  return FS_OK;
}

int fs_solver_stats(fs_ctx *ctx, float *ms5, int32_t *iters5, int32_t *calls5, int reset) {
  if (!ctx) return FS_E_ARG;
  FS_CK(cudaStreamSynchronize(ctx->st));
  fs_solver_stats_collect(ctx);
  for (int q = 0; q < 5; q++) {
    if (ms5) ms5[q] = ctx->s_ms[q];
    if (iters5) iters5[q] = ctx->s_its[q];
    if (calls5) calls5[q] = ctx->s_calls[q];
    if (reset) { ctx->s_ms[q] = 0.f; ctx->s_its[q] = 0; ctx->s_calls[q] = 0; ctx->k_ms[q] = 0.f; }
  }
  return FS_OK;
}

int fs_solver_kernel_ms(fs_ctx *ctx, float *ms5) {
  if (!ctx || !ms5) return FS_E_ARG;
  FS_CK(cudaStreamSynchronize(ctx->st));
  fs_solver_stats_collect(ctx);
  for (int q = 0; q < 5; q++) ms5[q] = ctx->k_ms[q];
  return FS_OK;
}

int fs_sync(fs_ctx *ctx) {
  if (!ctx) return FS_E_ARG;
  FS_CK(cudaStreamSynchronize(ctx->st));
  return FS_OK;
}

// Ensemble of independent cases (no reference counterpart): `iters` SIMPLE
// iterations of every case captured into ONE CUDA graph -- the cases in
// sequence, so their cooperative solver kernels never run concurrently -- and
// the graph launched `launches` times, one host synchronisation per launch.
// Batched: each iteration runs every case up to its p' solve, then all the p'
// solves in one cooperative launch (k_amg_bicgstab_batch: CTA groups sized by
// rows x p' iterations, each solving its case behind its own bounded barrier),
// then the rest of every case's iteration.
// Residual blocks and linear iteration counts of every captured iteration go to
// pinned host memory by copies inside the graph.  source_out[q*T + t] is the
// stop metric of case q after its t-th run iteration (T = iters*launches),
// pc_iters_out (optional) the p' iterations, ms_out the device time of the
// launches.  The p' history guess runs inside the graph; the learned network's
// guess (host bookkeeping per solve) does not.
static int ensemble_run(fs_ctx **cs, int n, int iters, int launches, double *source_out, int32_t *pc_iters_out,
                        float *ms_out, bool batched) {
  if (!cs || n < 1 || iters < 1 || launches < 1 || !source_out) return FS_E_ARG;
  fs_ctx *c0 = cs[0];
  for (int q = 0; q < n; q++)
    if (!cs[q] || cs[q]->dev != c0->dev) return FS_E_ARG;
  cudaSetDevice(c0->dev);
  fs_ctx *ctx = c0;  // FS_CK reports into the first context
  // ordinary iterations per case build hierarchies, colourings and grids
  // (nothing may allocate during capture); the HR start must already be passed
  // and the p' history full (the captured solves take a fixed basis)
  std::vector<double> weight(n, 1.);
  for (int q = 0; q < n; q++) {
    fs_ctx *c = cs[q];
    fs_residuals r;
    do {
      int rc = fs_simple_iteration(c, &r);
      if (rc) { if (c != ctx) ctx->err = c->err; return rc; }
    } while (c->nIter < c->cfg.niter_start_hr || c->hist_cnt < c->hist_cap);
    // the batched p' launch gives each case CTAs in proportion to its rows
    // times its last p' iterations
    weight[q] = std::pow((double)c->N, ctx->ens_split) * std::max(1, r.lin_iters[FS_VAR_PC - 1]);
  }
  // batched: the multi-RHS momentum solves also go into one launch when every
  // case uses them; the parts of an iteration that have no cooperative kernel
  // then run as concurrent branches, one per case (cases with k-epsilon or the
  // temperature equation solve those with cooperative kernels, so their last
  // part stays in sequence)
  bool mom_b = batched, fork_post = batched;
  std::vector<double> mom_w(n);
  for (int q = 0; q < n; q++) {
    mom_b = mom_b && cs[q]->cfg.batched_momentum && cs[q]->cfg.solver_mom == FS_SOLVER_SOR;
    fork_post = fork_post && !cs[q]->turb && !cs[q]->energy;
    mom_w[q] = std::pow((double)cs[q]->N, ctx->ens_split);
  }
  fs_pc_batch *PB = nullptr;
  fs_mom_batch *MB = nullptr;
  std::vector<cudaEvent_t> ev(n, nullptr);
  if (batched) {
    int rc = fs_pc_batch_create(cs, n, weight.data(), &PB);
    if (rc) return rc;
    if (mom_b && (rc = fs_mom_batch_create(cs, n, mom_w.data(), &MB))) { fs_pc_batch_free(PB); return rc; }
  }
  const size_t slot = RB_SIZE + FS_NITERS / 2;  // residual block, then the int32 iteration counts
  double *h = nullptr;
  FS_CK(cudaHostAlloc((void **)&h, sizeof(double) * slot * n * iters, cudaHostAllocDefault));
  cudaStream_t S = nullptr;
  cudaEvent_t ej = nullptr, e0 = nullptr, e1 = nullptr;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t x = nullptr;
  std::vector<int> nit0(n);
  int rc = FS_OK;
  auto cleanup = [&]() {
    fs_pc_batch_free(PB);
    fs_mom_batch_free(MB);
    for (auto &v : ev) if (v) cudaEventDestroy(v);
    if (x) cudaGraphExecDestroy(x);
    if (g) cudaGraphDestroy(g);
    if (ej) cudaEventDestroy(ej);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (S) cudaStreamDestroy(S);
    cudaFreeHost(h);
  };
  auto fail = [&](const char *what, cudaError_t e) {
    ctx->err = std::string(what) + ": " + cudaGetErrorString(e);
    cleanup();
    return FS_E_CUDA;
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&S, cudaStreamNonBlocking)) != cudaSuccess) return fail("stream", e);
  if ((e = cudaEventCreateWithFlags(&ej, cudaEventDisableTiming)) != cudaSuccess) return fail("event", e);
  if ((e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess) return fail("event", e);
  if (batched)
    for (int q = 0; q < n; q++)
      if ((e = cudaEventCreateWithFlags(&ev[q], cudaEventDisableTiming)) != cudaSuccess) return fail("event", e);
  for (int q = 0; q < n; q++) nit0[q] = cs[q]->nIter;
  for (int q = 0; q < n; q++)
    if ((e = cudaStreamSynchronize(cs[q]->st)) != cudaSuccess) return fail("before capture", e);
  (void)cudaGetLastError();  // no stale error may be reported by a launch check inside the capture
  if ((e = cudaStreamBeginCapture(S, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return fail("capture", e);
  const char *what = nullptr;
  // one part of case q's iteration on its stream, joined to S before and after
  auto on_case = [&](fs_ctx *c, auto &&part) -> bool {
    if ((e = cudaEventRecord(ej, S)) != cudaSuccess) { what = "join record"; return false; }
    if ((e = cudaStreamWaitEvent(c->st, ej, 0)) != cudaSuccess) { what = "join wait"; return false; }
    c->graph_mode = true;
    c->pc_defer = batched;
    rc = part(c);
    c->graph_mode = false;
    c->pc_defer = false;
    if (rc != FS_OK) { if (c != ctx) ctx->err = c->err; return false; }
    if ((e = cudaEventRecord(ej, c->st)) != cudaSuccess) { what = "rejoin record"; return false; }
    if ((e = cudaStreamWaitEvent(S, ej, 0)) != cudaSuccess) { what = "rejoin wait"; return false; }
    return true;
  };
  // one part of every case's iteration as concurrent branches off S (no
  // cooperative kernel may be in such a part), joined back into S
  auto on_all = [&](auto &&part) -> bool {
    if ((e = cudaEventRecord(ej, S)) != cudaSuccess) { what = "fork record"; return false; }
    for (int q = 0; q < n; q++) {
      fs_ctx *c = cs[q];
      if ((e = cudaStreamWaitEvent(c->st, ej, 0)) != cudaSuccess) { what = "fork wait"; return false; }
      c->graph_mode = true;
      c->pc_defer = true;
      c->mom_defer = mom_b;
      rc = part(c);
      c->graph_mode = false;
      c->pc_defer = false;
      c->mom_defer = false;
      if (rc != FS_OK) { if (c != ctx) ctx->err = c->err; return false; }
      if ((e = cudaEventRecord(ev[q], c->st)) != cudaSuccess) { what = "join record"; return false; }
    }
    for (int q = 0; q < n; q++)
      if ((e = cudaStreamWaitEvent(S, ev[q], 0)) != cudaSuccess) { what = "join wait"; return false; }
    return true;
  };
  for (int t = 0; t < iters && rc == FS_OK && !what; t++) {
    if (batched) {
      // every case up to its p' solve (the momentum solves in one launch when
      // mom_b), all p' solves in one launch, then the rest
      bool ok = true;
      if (mom_b) {
        ok = on_all([](fs_ctx *c) { c->nIter++; return iteration_mom(c); });
        if (!ok) break;
        if ((rc = fs_mom_batch_launch(MB, cs, n, S)) != FS_OK) break;
        ok = on_all([](fs_ctx *c) { return iteration_mid(c); });
      } else {
        for (int q = 0; q < n && ok; q++)
          ok = on_case(cs[q], [](fs_ctx *c) { c->nIter++; return iteration_pre(c); });
      }
      if (!ok) break;
      if ((rc = fs_pc_batch_launch(PB, cs, n, S)) != FS_OK) break;
      if (fork_post && !on_all([](fs_ctx *c) { return iteration_post(c); })) break;
    }
    for (int q = 0; q < n && rc == FS_OK && !what; q++) {
      fs_ctx *c = cs[q];
      bool ok = true;
      if (!batched) ok = on_case(c, [](fs_ctx *cc) { return iteration_enqueue(cc); });
      else if (!fork_post) ok = on_case(c, [](fs_ctx *cc) { return iteration_post(cc); });
      if (!ok) break;
      // the residual block and iteration counts of this iteration, on S after the case's work
      double *d = h + ((size_t)q * iters + t) * slot;
      if ((e = cudaMemcpyAsync(d, c->resblk, sizeof(double) * RB_SIZE, cudaMemcpyDeviceToHost, S)) != cudaSuccess ||
          (e = cudaMemcpyAsync(d + RB_SIZE, c->d_iters, sizeof(int32_t) * FS_NITERS, cudaMemcpyDeviceToHost, S)) !=
              cudaSuccess) { what = "residual copy"; break; }
    }
  }
  cudaError_t ec = cudaStreamEndCapture(S, &g);
  for (int q = 0; q < n; q++) cs[q]->nIter = nit0[q];
  if (what) return fail(what, e);
  if (rc != FS_OK) { cleanup(); return rc; }
  if (ec != cudaSuccess) return fail("capture", ec);
  if ((e = cudaGraphInstantiate(&x, g, 0)) != cudaSuccess) return fail("instantiate", e);
  const int T = iters * launches;
  cudaEventRecord(e0, S);
  for (int L = 0; L < launches; L++) {
    if ((e = cudaGraphLaunch(x, S)) != cudaSuccess) return fail("graph launch", e);
    if ((e = cudaStreamSynchronize(S)) != cudaSuccess) return fail("graph run", e);
    for (int q = 0; q < n; q++)
      for (int t = 0; t < iters; t++) {
        const double *d = h + ((size_t)q * iters + t) * slot;
        const int k = L * iters + t;
        source_out[(size_t)q * T + k] = stop_metric(cs[q]->cfg, d);
        if (pc_iters_out) pc_iters_out[(size_t)q * T + k] = ((const int32_t *)(d + RB_SIZE))[FS_VAR_PC - 1];
      }
  }
  cudaEventRecord(e1, S);
  if ((e = cudaEventSynchronize(e1)) != cudaSuccess) return fail("graph run", e);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  if (ms_out) *ms_out = ms;
  for (int q = 0; q < n; q++) cs[q]->nIter = nit0[q] + T;
  cleanup();
  return FS_OK;
}

int fs_ensemble_run(fs_ctx **cs, int n, int iters, int launches, double *source_out, int32_t *pc_iters_out,
                    float *ms_out) {
  return ensemble_run(cs, n, iters, launches, source_out, pc_iters_out, ms_out, false);
}

int fs_ensemble_run_batched(fs_ctx **cs, int n, int iters, int launches, double *source_out, int32_t *pc_iters_out,
                            float *ms_out) {
  return ensemble_run(cs, n, iters, launches, source_out, pc_iters_out, ms_out, true);
}

int fs_ensemble_split(fs_ctx *ctx, double exponent) {
  if (!ctx || !(exponent >= 0.) || exponent > 2.) return FS_E_ARG;
  ctx->ens_split = exponent;
  return FS_OK;
}

}  // extern "C"
