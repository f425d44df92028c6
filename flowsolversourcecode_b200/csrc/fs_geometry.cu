// fs_geometry.cu -- connectivity (host) and geometry (device) set-up.
//
// Connectivity restates Readit (SolveEquations/GridAndGeometry/
// ReadFoamMesh.f90:277-660) in O(N): a cell's local face slots are its
// interior faces in face order followed by its boundary faces, and the
// owner/neighbour slot maps are recorded while the slots are filled, which
// gives exactly the slots the reference finds by search (:597-635).
//
// Geometry restates ProcessGeometry (ProcessGeometryRoutine.for:3-444) as
// four kernels.  This file is compiled with --fmad=false and keeps the
// reference's operation order, so every geometric array is bit-identical
// to the CPU restatement (IEEE-754 add/mul/div/sqrt, no contraction).
#include "fs_internal.cuh"
#include <algorithm>

namespace {

__global__ void k_face_geom(int nf, int F, const int32_t *__restrict__ fptr,
                            const int32_t *__restrict__ fnodes, const double *__restrict__ P,
                            double *sf, double *fa, double *fc, double *bsf, double *bfa,
                            double *bfc, int B) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  int q0 = fptr[f], q1 = fptr[f + 1], n = q1 - q0;
  double cx = 0., cy = 0., cz = 0.;
  for (int q = q0; q < q1; q++) {
    int j = fnodes[q];
    cx = cx + P[3 * j]; cy = cy + P[3 * j + 1]; cz = cz + P[3 * j + 2];
  }
  cx = cx / n; cy = cy / n; cz = cz / n;
  double Sx = 0, Sy = 0, Sz = 0, A = 0, Cx = 0, Cy = 0, Cz = 0;
  for (int q = q0; q < q1; q++) {
    int j2 = fnodes[q], j3 = (q < q1 - 1) ? fnodes[q + 1] : fnodes[q0];
    double x2 = P[3 * j2], y2 = P[3 * j2 + 1], z2 = P[3 * j2 + 2];
    double x3 = P[3 * j3], y3 = P[3 * j3 + 1], z3 = P[3 * j3 + 2];
    double sx1 = 0.5 * ((y2 - cy) * (z3 - cz) - (y3 - cy) * (z2 - cz));
    double sy1 = -0.5 * ((x2 - cx) * (z3 - cz) - (x3 - cx) * (z2 - cz));
    double sz1 = 0.5 * ((x2 - cx) * (y3 - cy) - (x3 - cx) * (y2 - cy));
    double a1 = sqrt(sx1 * sx1 + sy1 * sy1 + sz1 * sz1);
    double x1 = (cx + x2 + x3) / 3., y1 = (cy + y2 + y3) / 3., z1 = (cz + z2 + z3) / 3.;
    Sx = Sx + sx1; Sy = Sy + sy1; Sz = Sz + sz1; A = A + a1;
    Cx = Cx + x1 * a1; Cy = Cy + y1 * a1; Cz = Cz + z1 * a1;
  }
  if (f < F) {
    sf[f] = Sx; sf[F + f] = Sy; sf[2L * F + f] = Sz; fa[f] = A;
    fc[f] = Cx / A; fc[F + f] = Cy / A; fc[2L * F + f] = Cz / A;
  } else {
    int b = f - F;
    bsf[b] = Sx; bsf[B + b] = Sy; bsf[2L * B + b] = Sz; bfa[b] = A;
    bfc[b] = Cx / A; bfc[B + b] = Cy / A; bfc[2L * B + b] = Cz / A;
  }
}

__global__ void k_cell_geom(int N, int F, int B, const int32_t *__restrict__ cptr,
                            const int32_t *__restrict__ cnodes, const double *__restrict__ P,
                            const int32_t *__restrict__ ncf, const int32_t *__restrict__ slot,
                            const double *__restrict__ sf, const double *__restrict__ fc,
                            const double *__restrict__ bsf, const double *__restrict__ bfc,
                            double *vol, double *xc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double x1 = 0, y1 = 0, z1 = 0;
  int nn = cptr[i + 1] - cptr[i];
  for (int q = cptr[i]; q < cptr[i + 1]; q++) {
    int k = cnodes[q];
    x1 = x1 + P[3 * k]; y1 = y1 + P[3 * k + 1]; z1 = z1 + P[3 * k + 2];
  }
  x1 = x1 / nn; y1 = y1 / nn; z1 = z1 / nn;
  double V = 0., px = 0., py = 0., pz = 0.;
  int nc = ncf[i];
  for (int j = 0; j < nc; j++) {
    int f = slot[(long)j * N + i] >> 1;
    double ax, ay, az, x2, y2, z2;
    if (f >= F) {
      int b = f - F;
      ax = bsf[b]; ay = bsf[B + b]; az = bsf[2L * B + b];
      x2 = bfc[b]; y2 = bfc[B + b]; z2 = bfc[2L * B + b];
    } else {
      ax = sf[f]; ay = sf[F + f]; az = sf[2L * F + f];
      x2 = fc[f]; y2 = fc[F + f]; z2 = fc[2L * F + f];
    }
    double dx = x2 - x1, dy = y2 - y1, dz = z2 - z1;
    double xcp = 0.75 * x2 + 0.25 * x1, ycp = 0.75 * y2 + 0.25 * y1, zcp = 0.75 * z2 + 0.25 * z1;
    double vt = fabs(ax * dx + ay * dy + az * dz) / 3.;
    V = V + vt; px = px + xcp * vt; py = py + ycp * vt; pz = pz + zcp * vt;
  }
  vol[i] = V; xc[i] = px / V; xc[N + i] = py / V; xc[2L * N + i] = pz / V;
}

// interior faces: dCF, orientation, g, E/T, gDiff and the Green-Gauss
// correction vector dfp = r_f - r_f' (StandardGreenGaussCorrection1Gradient.for:113-124)
__global__ void k_iface_post(int N, int F, int msd, const int32_t *__restrict__ own,
                             const int32_t *__restrict__ nbr, const double *__restrict__ xc,
                             const double *__restrict__ fc, const double *__restrict__ fa,
                             double *sf, double *dcfv, double *dcf, double *gf, double *gdiff,
                             double *tf, double *dfp) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= F) return;
  int i = own[k], j = nbr[k];
  double xi = xc[i], yi = xc[N + i], zi = xc[2L * N + i];
  double xj = xc[j], yj = xc[N + j], zj = xc[2L * N + j];
  double dx = xj - xi, dy = yj - yi, dz = zj - zi;
  double d = sqrt(dx * dx + dy * dy + dz * dz);
  double ex = dx / d, ey = dy / d, ez = dz / d;
  double sx = sf[k], sy = sf[F + k], sz = sf[2L * F + k], A = fa[k];
  double dp = dx * sx + dy * sy + dz * sz;
  if (dp < 0.) { sx = -sx; sy = -sy; sz = -sz; }
  double nx = sx / A, ny = sy / A, nz = sz / A;
  double fx = fc[k], fy = fc[F + k], fz = fc[2L * F + k];
  double d1 = sqrt((fx - xi) * (fx - xi) + (fy - yi) * (fy - yi) + (fz - zi) * (fz - zi));
  double d2 = sqrt((fx - xj) * (fx - xj) + (fy - yj) * (fy - yj) + (fz - zj) * (fz - zj));
  double g = d2 / (d1 + d2);
  double Ex, Ey, Ez, E;
  if (msd == 1) {
    double q = ex * sx + ey * sy + ez * sz;
    Ex = q * ex; Ey = q * ey; Ez = q * ez; E = fabs(q);
  } else if (msd == 2) {
    Ex = A * ex; Ey = A * ey; Ez = A * ez; E = A;
  } else {
    double q = ex * sx + ey * sy + ez * sz, a2 = A * A;
    Ex = (a2 / q) * ex; Ey = (a2 / q) * ey; Ez = (a2 / q) * ez;
    E = sqrt(Ex * Ex + Ey * Ey + Ez * Ez);
  }
  sf[k] = sx; sf[F + k] = sy; sf[2L * F + k] = sz;
  dcfv[k] = dx; dcfv[F + k] = dy; dcfv[2L * F + k] = dz; dcf[k] = d;
  gf[k] = g; gdiff[k] = E / d;
  tf[k] = sx - Ex; tf[F + k] = sy - Ey; tf[2L * F + k] = sz - Ez;
  double eDOTn = Ex * nx + Ey * ny + Ez * nz;
  double rfn = (fx - xi) * nx + (fy - yi) * ny + (fz - zi) * nz;
  double xfp = xi + (rfn / eDOTn) * Ex, yfp = yi + (rfn / eDOTn) * Ey, zfp = zi + (rfn / eDOTn) * Ez;
  dfp[k] = fx - xfp; dfp[F + k] = fy - yfp; dfp[2L * F + k] = fz - zfp;
}

__global__ void k_bface_post(int N, int B, int msd, const int32_t *__restrict__ bown,
                             const double *__restrict__ xc, const double *__restrict__ bfc,
                             const double *__restrict__ bfa, double *bsf, double *bnf,
                             double *bdv, double *bgdiff, double *btf) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  int n = bown[b];
  double dx = bfc[b] - xc[n], dy = bfc[B + b] - xc[N + n], dz = bfc[2L * B + b] - xc[2L * N + n];
  double d = sqrt(dx * dx + dy * dy + dz * dz);
  double ex = dx / d, ey = dy / d, ez = dz / d;
  double sx = bsf[b], sy = bsf[B + b], sz = bsf[2L * B + b], A = bfa[b];
  double dp = dx * sx + dy * sy + dz * sz;
  if (dp < 0.) { sx = -sx; sy = -sy; sz = -sz; }
  double Ex, Ey, Ez, E;
  if (msd == 1) {
    double q = ex * sx + ey * sy + ez * sz;
    Ex = q * ex; Ey = q * ey; Ez = q * ez; E = fabs(q);
  } else if (msd == 2) {
    Ex = A * ex; Ey = A * ey; Ez = A * ez; E = A;
  } else {
    double q = ex * sx + ey * sy + ez * sz, a2 = A * A;
    Ex = (a2 / q) * ex; Ey = (a2 / q) * ey; Ez = (a2 / q) * ez;
    E = sqrt(Ex * Ex + Ey * Ey + Ez * Ez);
  }
  bsf[b] = sx; bsf[B + b] = sy; bsf[2L * B + b] = sz;
  bnf[b] = sx / A; bnf[B + b] = sy / A; bnf[2L * B + b] = sz / A;
  bdv[b] = dx; bdv[B + b] = dy; bdv[2L * B + b] = dz;
  bgdiff[b] = E / d;
  btf[b] = sx - Ex; btf[B + b] = sy - Ey; btf[2L * B + b] = sz - Ez;
}

// BFaceAreanz(i,i) read by CorrectGradientAtOulet / CorrectPressureGradientAtSymmetryBoundary
// (CorrectGradients.for:222,272): the z-normal of face #set within patch #set
__global__ void k_bnzii(int B, const int32_t *__restrict__ bset, const int32_t *__restrict__ sstart,
                        const int32_t *__restrict__ sn, const double *__restrict__ bnf, double *nzii) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  int s = bset[b];
  nzii[b] = (s < sn[s]) ? bnf[2L * B + sstart[s] + s] : 0.;
}

}  // namespace

// Greedy colouring in cell order (independent sets for the Gauss-Seidel
// sweeps).  Hex meshes in i-j-k order get the two checkerboard colours.
static void build_colors(fs_ctx *ctx) {
  int N = ctx->N, W = ctx->W;
  std::vector<int> col(N, -1);
  int nc = 0;
  for (int i = 0; i < N; i++) {
    unsigned used = 0;
    for (int j = 0; j < ctx->h_ncf[i]; j++) {
      int k = ctx->h_cn[(long)j * N + i];
      if (k >= 0 && col[k] >= 0 && col[k] < 32) used |= 1u << col[k];
    }
    int c = 0;
    while (used & (1u << c)) c++;
    col[i] = c;
    nc = std::max(nc, c + 1);
  }
  (void)W;
  ctx->ncolors = nc;
  ctx->h_color_ptr.assign(nc + 1, 0);
  for (int i = 0; i < N; i++) ctx->h_color_ptr[col[i] + 1]++;
  for (int c = 0; c < nc; c++) ctx->h_color_ptr[c + 1] += ctx->h_color_ptr[c];
  ctx->h_color_rows.assign(N, 0);
  std::vector<int> pos(ctx->h_color_ptr.begin(), ctx->h_color_ptr.end() - 1);
  for (int i = 0; i < N; i++) ctx->h_color_rows[pos[col[i]]++] = i;
}

template <class T>
static int up(fs_ctx *ctx, T **d, const T *h, size_t n) {
  FS_CK(cudaMalloc((void **)d, std::max<size_t>(n, 1) * sizeof(T)));
  if (n) FS_CK(cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice));
  return FS_OK;
}

int fs_geometry_build(fs_ctx *ctx, const fs_mesh_in *mi) {
  const int nf = mi->n_faces, F = mi->n_internal, B = nf - F;
  if (nf <= 0 || F < 0 || B < 0 || mi->n_nodes <= 0) { ctx->err = "empty mesh"; return FS_E_MESH; }
  int N = -1;
  for (int i = 0; i < nf; i++) {
    if (mi->owner[i] < 0 || mi->owner[i] >= (1 << 30)) { ctx->err = "bad owner"; return FS_E_MESH; }
    N = std::max(N, mi->owner[i] + 1);
    if (i < F) {
      if (mi->neighbour[i] < 0) { ctx->err = "bad neighbour"; return FS_E_MESH; }
      N = std::max(N, mi->neighbour[i] + 1);
    }
  }
  long psum = 0;
  for (int s = 0; s < mi->n_patches; s++) {
    if (mi->patch_start[s] != F + psum) { ctx->err = "patches must follow the interior faces in order"; return FS_E_MESH; }
    psum += mi->patch_size[s];
  }
  if (psum != B) { ctx->err = "patch sizes do not cover the boundary faces"; return FS_E_MESH; }
  for (int q = 0; q < mi->face_ptr[nf]; q++)
    if (mi->face_nodes[q] < 0 || mi->face_nodes[q] >= mi->n_nodes) { ctx->err = "face node out of range"; return FS_E_MESH; }
  ctx->N = N; ctx->F = F; ctx->B = B; ctx->NS = mi->n_patches;

  // ---- Readit restatement (host, O(N)) ----
  std::vector<int32_t> &ncf = ctx->h_ncf;
  ncf.assign(N, 0);
  if (mi->cell_face_ptr) {   // the element-local order of GlobalConnectivity
    if (!mi->cell_faces || mi->cell_face_ptr[0] != 0) { ctx->err = "cell_faces missing"; return FS_E_MESH; }
    for (int i = 0; i < N; i++) ncf[i] = mi->cell_face_ptr[i + 1] - mi->cell_face_ptr[i];
  } else {
    for (int i = 0; i < F; i++) { ncf[mi->owner[i]]++; ncf[mi->neighbour[i]]++; }
    for (int i = F; i < nf; i++) ncf[mi->owner[i]]++;
  }
  int W = 0;
  for (int i = 0; i < N; i++) W = std::max(W, ncf[i]);
  ctx->W = W;
  ctx->h_cf.assign((size_t)W * N, -1);
  ctx->h_cn.assign((size_t)W * N, -1);
  ctx->h_own_slot.assign(F, 0);
  ctx->h_nbr_slot.assign(F, 0);
  std::vector<int32_t> cnt(N, 0), slotv((size_t)W * N, -1);
  if (mi->cell_face_ptr) {
    // every interior face once on its owner's and once on its neighbour's list,
    // every boundary face once on its owner's
    std::vector<int8_t> seen((size_t)nf, 0);
    for (int i = 0; i < N; i++)
      for (int j = 0; j < ncf[i]; j++) {
        int k = mi->cell_faces[mi->cell_face_ptr[i] + j];
        if (k < 0 || k >= nf) { ctx->err = "cell_faces: face id out of range"; return FS_E_MESH; }
        int side;
        if (k < F && mi->owner[k] == i && !(seen[k] & 1)) side = 0;
        else if (k < F && mi->neighbour[k] == i && !(seen[k] & 2)) side = 1;
        else if (k >= F && mi->owner[k] == i && !seen[k]) side = 0;
        else { ctx->err = "cell_faces: face not on this cell or listed twice"; return FS_E_MESH; }
        seen[k] |= (int8_t)(1 << side);
        ctx->h_cf[(size_t)j * N + i] = k;
        slotv[(size_t)j * N + i] = (k << 1) | side;
        if (k < F) {
          ctx->h_cn[(size_t)j * N + i] = side ? mi->owner[k] : mi->neighbour[k];
          (side ? ctx->h_nbr_slot : ctx->h_own_slot)[k] = j;
        }
      }
    for (int k = 0; k < nf; k++)
      if (seen[k] != (k < F ? 3 : 1)) { ctx->err = "cell_faces: a face is missing from its cells"; return FS_E_MESH; }
  } else {
    for (int k = 0; k < F; k++) {
      int o = mi->owner[k], nb = mi->neighbour[k];
      int jo = cnt[o]++, jn = cnt[nb]++;
      ctx->h_cf[(size_t)jo * N + o] = k; ctx->h_cn[(size_t)jo * N + o] = nb; slotv[(size_t)jo * N + o] = k << 1;
      ctx->h_cf[(size_t)jn * N + nb] = k; ctx->h_cn[(size_t)jn * N + nb] = o; slotv[(size_t)jn * N + nb] = (k << 1) | 1;
      ctx->h_own_slot[k] = jo; ctx->h_nbr_slot[k] = jn;
    }
    for (int k = F; k < nf; k++) {
      int o = mi->owner[k], j = cnt[o]++;
      ctx->h_cf[(size_t)j * N + o] = k; slotv[(size_t)j * N + o] = k << 1;
    }
  }
  ctx->h_fown.assign(mi->owner, mi->owner + F);
  ctx->h_fnbr.assign(mi->neighbour, mi->neighbour + F);
  ctx->h_bown.assign(mi->owner + F, mi->owner + nf);
  ctx->h_bset.assign(B, 0);
  ctx->h_bset_start.assign(ctx->NS, 0);
  ctx->h_bset_n.assign(ctx->NS, 0);
  ctx->h_btype.assign(B, 0);
  for (int s = 0, b = 0; s < ctx->NS; s++) {
    ctx->h_bset_start[s] = b; ctx->h_bset_n[s] = mi->patch_size[s];
    for (int j = 0; j < mi->patch_size[s]; j++, b++) {
      ctx->h_bset[b] = s; ctx->h_btype[b] = ctx->cfg.patch_type[s];
    }
  }
  // ordered cell node lists (ReadFoamMesh.f90:430-458), or as given (ListOfElementNodes of a neutral file)
  std::vector<int32_t> cptr(N + 1, 0), cnodes;
  cnodes.reserve((size_t)N * 8);
  if (mi->cell_node_ptr) {
    if (!mi->cell_nodes || mi->cell_node_ptr[0] != 0) { ctx->err = "cell_nodes missing"; return FS_E_MESH; }
    cptr.assign(mi->cell_node_ptr, mi->cell_node_ptr + N + 1);
    cnodes.assign(mi->cell_nodes, mi->cell_nodes + cptr[N]);
    for (int32_t nd : cnodes) if (nd < 0 || nd >= mi->n_nodes) { ctx->err = "cell node out of range"; return FS_E_MESH; }
  }
  for (int i = 0; i < N && !mi->cell_node_ptr; i++) {
    cptr[i] = (int32_t)cnodes.size();
    size_t start = cnodes.size();
    for (int j = 0; j < ncf[i]; j++) {
      int f = ctx->h_cf[(size_t)j * N + i];
      for (int q = mi->face_ptr[f]; q < mi->face_ptr[f + 1]; q++) {
        int nd = mi->face_nodes[q];
        bool seen = false;
        if (j > 0)
          for (size_t r = start; r < cnodes.size(); r++) if (cnodes[r] == nd) { seen = true; break; }
        if (!seen) cnodes.push_back(nd);
      }
    }
  }
  if (!mi->cell_node_ptr) cptr[N] = (int32_t)cnodes.size();
  build_colors(ctx);

  // ---- upload connectivity ----
  int rc;
  if ((rc = up(ctx, &ctx->slot, slotv.data(), slotv.size()))) return rc;
  if ((rc = up(ctx, &ctx->cn, ctx->h_cn.data(), ctx->h_cn.size()))) return rc;
  if ((rc = up(ctx, &ctx->ncf, ncf.data(), (size_t)N))) return rc;
  if ((rc = up(ctx, &ctx->fown, ctx->h_fown.data(), (size_t)F))) return rc;
  if ((rc = up(ctx, &ctx->fnbr, ctx->h_fnbr.data(), (size_t)F))) return rc;
  if ((rc = up(ctx, &ctx->bown, ctx->h_bown.data(), (size_t)B))) return rc;
  if ((rc = up(ctx, &ctx->btype, ctx->h_btype.data(), (size_t)B))) return rc;
  {  // colour-major index maps for the permuted Gauss-Seidel matrix
    std::vector<int32_t> pos(N), cnP((size_t)W * N, -1), ncfP(N);
    for (int q = 0; q < N; q++) pos[ctx->h_color_rows[q]] = q;
    for (int q = 0; q < N; q++) {
      int i = ctx->h_color_rows[q];
      ncfP[q] = ncf[i];
      for (int j = 0; j < ncf[i]; j++) {
        int k = ctx->h_cn[(size_t)j * N + i];
        cnP[(size_t)j * N + q] = k >= 0 ? pos[k] : -1;
      }
    }
    if ((rc = up(ctx, &ctx->cposP, pos.data(), pos.size()))) return rc;
    if ((rc = up(ctx, &ctx->cnP, cnP.data(), cnP.size()))) return rc;
    if ((rc = up(ctx, &ctx->ncfP, ncfP.data(), ncfP.size()))) return rc;
  }
  {  // colour row lists followed by the colour offsets (ncolors+1)
    std::vector<int32_t> cr(ctx->h_color_rows);
    cr.insert(cr.end(), ctx->h_color_ptr.begin(), ctx->h_color_ptr.end());
    if ((rc = up(ctx, &ctx->color_rows, cr.data(), cr.size()))) return rc;
  }

  // ---- geometry kernels ----
  int32_t *d_fptr = nullptr, *d_fnodes = nullptr, *d_cptr = nullptr, *d_cnodes = nullptr;
  int32_t *d_bset = nullptr, *d_sstart = nullptr, *d_sn = nullptr;
  double *d_P = nullptr, *d_fc = nullptr, *d_bfc = nullptr;
  if ((rc = up(ctx, &d_fptr, mi->face_ptr, (size_t)nf + 1))) return rc;
  if ((rc = up(ctx, &d_fnodes, mi->face_nodes, (size_t)mi->face_ptr[nf]))) return rc;
  if ((rc = up(ctx, &d_cptr, cptr.data(), cptr.size()))) return rc;
  if ((rc = up(ctx, &d_cnodes, cnodes.data(), cnodes.size()))) return rc;
  if ((rc = up(ctx, &d_P, mi->points, (size_t)mi->n_nodes * 3))) return rc;
  if ((rc = up(ctx, &d_bset, ctx->h_bset.data(), (size_t)B))) return rc;
  if ((rc = up(ctx, &d_sstart, ctx->h_bset_start.data(), (size_t)ctx->NS))) return rc;
  if ((rc = up(ctx, &d_sn, ctx->h_bset_n.data(), (size_t)ctx->NS))) return rc;
  FS_CK(cudaMalloc(&d_fc, sizeof(double) * 3 * std::max(F, 1)));
  FS_CK(cudaMalloc(&d_bfc, sizeof(double) * 3 * std::max(B, 1)));
  auto dal = [&](double **p, size_t n) -> int {
    FS_CK(cudaMalloc((void **)p, sizeof(double) * std::max<size_t>(n, 1)));
    FS_CK(cudaMemset(*p, 0, sizeof(double) * std::max<size_t>(n, 1)));
    return FS_OK;
  };
  if ((rc = dal(&ctx->vol, N)) || (rc = dal(&ctx->xc, 3L * N)) || (rc = dal(&ctx->gf, F)) ||
      (rc = dal(&ctx->sf, 3L * F)) || (rc = dal(&ctx->dcfv, 3L * F)) || (rc = dal(&ctx->dcf, F)) ||
      (rc = dal(&ctx->gdiff, F)) || (rc = dal(&ctx->tf, 3L * F)) || (rc = dal(&ctx->dfp, 3L * F)) ||
      (rc = dal(&ctx->fa, F)) || (rc = dal(&ctx->bsf, 3L * B)) || (rc = dal(&ctx->bfa, B)) ||
      (rc = dal(&ctx->bnf, 3L * B)) || (rc = dal(&ctx->bdv, 3L * B)) || (rc = dal(&ctx->bgdiff, B)) ||
      (rc = dal(&ctx->btf, 3L * B)) || (rc = dal(&ctx->bnzii, B)))
    return rc;
  int msd = ctx->cfg.method_decompose_s;
  k_face_geom<<<fs_grid(nf), FS_BLOCK, 0, ctx->st>>>(nf, F, d_fptr, d_fnodes, d_P, ctx->sf, ctx->fa, d_fc,
                                                    ctx->bsf, ctx->bfa, d_bfc, B);
  FS_LAUNCH_CHECK();
  k_cell_geom<<<fs_grid(N), FS_BLOCK, 0, ctx->st>>>(N, F, B, d_cptr, d_cnodes, d_P, ctx->ncf, ctx->slot, ctx->sf,
                                                   d_fc, ctx->bsf, d_bfc, ctx->vol, ctx->xc);
  FS_LAUNCH_CHECK();
  if (F) {
    k_iface_post<<<fs_grid(F), FS_BLOCK, 0, ctx->st>>>(N, F, msd, ctx->fown, ctx->fnbr, ctx->xc, d_fc, ctx->fa, ctx->sf,
                                                      ctx->dcfv, ctx->dcf, ctx->gf, ctx->gdiff, ctx->tf, ctx->dfp);
    FS_LAUNCH_CHECK();
  }
  if (B) {
    k_bface_post<<<fs_grid(B), FS_BLOCK, 0, ctx->st>>>(N, B, msd, ctx->bown, ctx->xc, d_bfc, ctx->bfa, ctx->bsf,
                                                      ctx->bnf, ctx->bdv, ctx->bgdiff, ctx->btf);
    FS_LAUNCH_CHECK();
    k_bnzii<<<fs_grid(B), FS_BLOCK, 0, ctx->st>>>(B, d_bset, d_sstart, d_sn, ctx->bnf, ctx->bnzii);
    FS_LAUNCH_CHECK();
  }
  FS_CK(cudaStreamSynchronize(ctx->st));
  cudaFree(d_fptr); cudaFree(d_fnodes); cudaFree(d_cptr); cudaFree(d_cnodes); cudaFree(d_P);
  cudaFree(d_fc); cudaFree(d_bfc); cudaFree(d_bset); cudaFree(d_sstart); cudaFree(d_sn);
  return FS_OK;
}
