// fs_mg.cu -- element-agglomeration multigrid (placeholder until the hierarchy lands).
#include "fs_internal.cuh"

int fs_mg_build(fs_ctx *ctx) { ctx->err = "multigrid not built"; return FS_E_UNSUPPORTED; }
int fs_mg_free(fs_ctx *ctx) { (void)ctx; return FS_OK; }
int fs_mg_vcycle_solve(fs_ctx *ctx, int nf, double rrf, double *iters_out) {
  (void)nf; (void)rrf; (void)iters_out;
  ctx->err = "multigrid solver not available";
  return FS_E_UNSUPPORTED;
}
extern "C" int fs_mg_levels(fs_ctx *ctx, int32_t *n_levels, int32_t *level_sizes, int max_levels) {
  (void)ctx; (void)level_sizes; (void)max_levels;
  if (n_levels) *n_levels = 0;
  return FS_E_UNSUPPORTED;
}
extern "C" int fs_mg_parents(fs_ctx *ctx, int level, int32_t *parents, size_t n) {
  (void)ctx; (void)level; (void)parents; (void)n;
  return FS_E_UNSUPPORTED;
}
