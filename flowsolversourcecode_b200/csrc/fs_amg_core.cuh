// Krylov solve with the V-cycle preconditioner (PCycle) and the grid
// reductions it uses.  Included twice by fs_mg.cu:
//   FS_GROUPS 0: the whole cooperative grid solves one system; CTA index and
//     count are the grid's and the grid barrier is the cooperative one;
//   FS_GROUPS 1: the CTAs of one cooperative launch are split into groups, one
//     per system (the batched p' solve of an ensemble); CTA index and count are
//     relative to the group, held in shared memory, and the grid barrier is a
//     bounded barrier among the group's CTAs in global memory.
#if FS_GROUPS
struct GroupState {
  int cta, ncta, q;   // this CTA within its group, the group's CTAs, its system
  unsigned gen;       // generation of the group barrier this CTA waits to leave
  unsigned *bar;      // [0] arrivals, [1] generation (zero at launch)
  int32_t *status;    // [0] set when a barrier timed out
};
__device__ __forceinline__ GroupState &gstate() {
  __shared__ GroupState g;
  return g;
}
__device__ __forceinline__ int cta_id() { return gstate().cta; }
__device__ __forceinline__ int cta_count() { return gstate().ncta; }
// barrier among the group's CTAs: the last arrival resets the count and bumps
// the generation the others poll; polls are bounded, a timeout is recorded in
// the system's status word, and once it is set no barrier waits any more
__device__ void group_sync() {
  GroupState &G = gstate();
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned gen = G.gen;
    if (atomicAdd(&G.bar[0], 1u) == (unsigned)G.ncta - 1) {
      atomicExch(&G.bar[0], 0u);
      __threadfence();
      atomicAdd(&G.bar[1], 1u);
    } else {
      const volatile unsigned *vg = G.bar + 1;
      const volatile int32_t *vs = G.status;
      long spins = 0;
      while (*vg == gen && *vs == 0) {
        if (++spins > FS_PC_SPIN_LIMIT) { atomicExch(G.status, 1); break; }
        __nanosleep(64);
      }
    }
    __threadfence();
    G.gen = gen + 1;
  }
  __syncthreads();
}
#else
__device__ __forceinline__ int cta_id() { return (int)blockIdx.x; }
__device__ __forceinline__ int cta_count() { return (int)gridDim.x; }
#endif

struct Sync {
  cg::grid_group grid;
  double *part;
  int buf, buf3;
  __device__ Sync(double *p) : grid(cg::this_grid()), part(p), buf(0), buf3(0) {}
  __device__ __forceinline__ void gbar() {
#if FS_GROUPS
    group_sync();
#else
    grid.sync();
#endif
  }
  __device__ void all() { gbar(); }
  // grid-deterministic sum of two values (every CTA gets the same result)
  __device__ void sum2(double a0, double a1, double &o0, double &o1) {
    int G = cta_count();
    double b0 = bsum(a0), b1 = bsum(a1);
    if (threadIdx.x == 0) { part[(2 * buf) * G + cta_id()] = b0; part[(2 * buf + 1) * G + cta_id()] = b1; }
    gbar();
    double s0 = 0., s1 = 0.;
    for (int q = threadIdx.x; q < G; q += blockDim.x) { s0 += part[(2 * buf) * G + q]; s1 += part[(2 * buf + 1) * G + q]; }
    o0 = bsum(s0); o1 = bsum(s1);
    buf = (buf + 1) % 3;
  }
  // grid-deterministic sums of K <= FS_SUMK values, in the partial slots after
  // the three buffers of sum2 (every CTA gets the same results), with one
  // block barrier before and one after the grid barrier: warp sums into shared
  // memory, thread k adds the warps' and then the CTAs' partials of value k in
  // a fixed order
  template <int K>
  __device__ void sumKt(const double (&in)[K], double (&out)[K]) {
    __shared__ double sh[K][33];
    const int G = cta_count(), lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double *pk = part + 6L * G;
#pragma unroll
    for (int k = 0; k < K; k++) {
      const double v = wsum(in[k]);
      if (lane == 0) sh[k][wid] = v;
    }
    __syncthreads();
    if ((int)threadIdx.x < K) {
      const int k = threadIdx.x;
      double t = 0.;
      for (int w = 0; w < nw; w++) t += sh[k][w];
      pk[(long)k * G + cta_id()] = t;
    }
    gbar();
    if ((int)threadIdx.x < K) {
      const int k = threadIdx.x;
      double t = 0.;
      for (int q = 0; q < G; q++) t += pk[(long)k * G + q];
      sh[k][32] = t;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; k++) out[k] = sh[k][32];
  }
  // grid-deterministic sums of three values, in three rotating buffers of
  // their own after the sumK slots
  __device__ void sum3(double a0, double a1, double a2, double &o0, double &o1, double &o2) {
    const int G = cta_count();
    double *pb = part + (6L + FS_SUMK + 3L * buf3) * G;
    const double b0 = bsum(a0), b1 = bsum(a1), b2 = bsum(a2);
    if (threadIdx.x == 0) { pb[cta_id()] = b0; pb[G + cta_id()] = b1; pb[2 * G + cta_id()] = b2; }
    gbar();
    double s0 = 0., s1 = 0., s2 = 0.;
    for (int q = threadIdx.x; q < G; q += blockDim.x) { s0 += pb[q]; s1 += pb[G + q]; s2 += pb[2 * G + q]; }
    o0 = bsum(s0); o1 = bsum(s1); o2 = bsum(s2);
    buf3 = (buf3 + 1) % 3;
  }
};

// which threads work on a level, and how they synchronise
// the first FS_PC_TEAM CTAs: mid-sized preconditioner levels (PCycle)
__device__ __forceinline__ int team_size() { return cta_count() < FS_PC_TEAM ? cta_count() : FS_PC_TEAM; }

struct Scope {
  bool grid = false;   // whole grid
  bool team = false;   // else the first team_size() CTAs; else CTA 0 only
  __device__ bool active() const { return grid || (team ? cta_id() < team_size() : cta_id() == 0); }
  __device__ long tid0() const {
    return (grid || team) ? (long)cta_id() * blockDim.x + threadIdx.x : (long)threadIdx.x;
  }
  __device__ long nth() const {
    return grid ? (long)cta_count() * blockDim.x : team ? (long)team_size() * blockDim.x : (long)blockDim.x;
  }
};

// One V-cycle with zero initial guesses as the preconditioner M^-1 of the Krylov
// solver.  Damped Jacobi (omega) on every level, so each sweep is one phase of
// independent rows; the first pre-sweep from zero is fused into the restriction
// that makes the level's rhs, and the coarsest level is solved by a dense FP64
// inverse (k_mg_dense_inverse).  The coarse correction is over-weighted,
// x += alpha*x_c[parent] with alpha > 1, which compensates the energy of
// piecewise-constant prolongation.  On levels with a thread per row the
// prolongation is a phase of its own before the first post-sweep; on levels
// with G lanes per row it is formed on the fly inside the sweep for the row and
// its neighbours.  A cycle over levels 0..lc costs 3*lc+2 barrier phases plus one
// per thread-per-row level.  Level-0 rhs and result are FP64 in either
// precision; up-leg results go to each level's r.
//
// Rows with fewer than two threads each are handled a thread per row, two rows
// per step (ell_acc2).  Coarse rows have 10-30 neighbours and coarse levels
// fewer rows than the grid has threads, so there a row is handled by G
// consecutive lanes (G = 2..8 from the threads per row) that split its
// neighbour loop and combine by shuffles.  Levels up to FS_PC_SMALL rows run on
// CTA 0 alone; levels up to FS_PC_TEAM_MAX rows on a team of the first
// FS_PC_TEAM CTAs with a bounded barrier of their own in global memory -- a
// barrier over all CTAs costs several microseconds, and those phases have too
// little work to use the whole grid anyway.

template <class R>
__device__ __forceinline__ Scope pc_scope(const LevelDev<R> &L) {
  Scope s;
  s.grid = L.n > FS_PC_TEAM_MAX;
  s.team = !s.grid && L.n > FS_PC_SMALL;
  return s;
}

template <int G, class T>
__device__ __forceinline__ T gsum(T v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// rows [0,n) by groups of G consecutive lanes; the trip count is uniform per
// warp, so every lane reaches the group shuffles (f must not return early)
template <int G, class F>
__device__ __forceinline__ void group_rows(const Scope &sc, int n, F &f) {
  constexpr int GPW = 32 / G;
  const long w0 = sc.tid0() >> 5, nw = sc.nth() >> 5;
  const int lane = threadIdx.x & 31, grp = lane / G, q = lane % G;
  for (long wb = w0 * GPW; wb < n; wb += nw * GPW) {
    long i = wb + grp;
    f(std::integral_constant<int, G>{}, i, i < n, q);
  }
}

// G from the threads per row (callers handle fewer than 2 threads per row)
template <class F>
__device__ __forceinline__ void level_rows(const Scope &sc, int n, int level, F &&f) {
  const long per = sc.nth() / (n > 0 ? n : 1);
  (void)level;
  if (per < 4) group_rows<2>(sc, n, f);
  else if (per < 8) group_rows<4>(sc, n, f);
  else group_rows<8>(sc, n, f);
}

template <class R>
struct PCycle {
  Sync &S;
  const LevelDev<R> *lev;
  int lc;              // coarsest level used by the preconditioner
  bool direct;         // coarsest by the dense inverse, else coarse_sweeps sweeps
  const double *sinv;  // lev[lc].n^2, row-major
  int pre, post, coarse_sweeps;
  R omega, alpha;        // Jacobi weight and coarse-correction factor on levels >= 1
  Scope last;            // scope of the previous phase
  R omega0, alpha0;      // the same on level 0
  unsigned *bar;         // team barrier: [0] arrivals, [1] generation (zero at launch)
  int32_t *status;       // [0] set when a team barrier timed out
  unsigned gen;          // generation this CTA waits to leave
  int extra;             // arrivals waited for beyond the team (0; >0 only to test the timeout)
  bool synced;           // the next enter() needs no barrier (the caller has just passed one)
  __device__ R om(int l) const { return l == 0 ? omega0 : omega; }
  __device__ R al(int l) const { return l == 0 ? alpha0 : alpha; }
  // barrier among the team CTAs: the arrival count in global memory, the last
  // arrival resets it and bumps the generation the others poll; polls are
  // bounded, and a timeout is recorded (later team barriers then stop
  // waiting).  The FP64 cycle calls it out of line (inlined at every phase it
  // doubled that kernel's register spills); the FP32 cycle, with fewer live
  // registers, runs faster with it inline.
  __device__ __noinline__ void team_sync_call() { team_sync_body(); }
  __device__ __forceinline__ void team_sync() {
    if (sizeof(R) == sizeof(double)) team_sync_call();
    else team_sync_body();
  }
  __device__ __forceinline__ void team_sync_body() {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned g = gen, T = (unsigned)(team_size() + extra);
      if (atomicAdd(&bar[0], 1u) == T - 1) {
        atomicExch(&bar[0], 0u);
        __threadfence();
        atomicAdd(&bar[1], 1u);
      } else {
        const volatile unsigned *vg = bar + 1;
        const volatile int32_t *vs = status;
        long spins = 0;
        while (*vg == g && *vs == 0) {
          if (++spins > FS_PC_SPIN_LIMIT) { atomicExch(status, 1); break; }
          __nanosleep(64);
        }
      }
      __threadfence();
    }
    gen++;
    __syncthreads();
  }
  // the barrier before a phase: grid-wide when the grid is involved on either
  // side, among the team when the team is, else within CTA 0
  __device__ void enter(const Scope &sc) {
    if (synced) synced = false;
    else if (sc.grid || last.grid) S.all();
    else if (sc.team || last.team) { if (cta_id() < team_size()) team_sync(); }
    else __syncthreads();
    last = sc;
  }
  // r (into dst) = b - A x on level l; level 0 takes b from `in`
  __device__ void residual(int l, const double *__restrict__ in, const R *__restrict__ x, R *__restrict__ dst) {
    const LevelDev<R> L = lev[l];
    Scope sc = pc_scope(L);
    enter(sc);
    if (!sc.active()) return;
    if (l == 0 || sc.nth() < 2L * L.n) {   // a thread per row, two rows per step
      const long t0 = sc.tid0(), nt = sc.nth();
      for (long i = t0; i < L.n; i += 2 * nt) {
        const long i2 = i + nt;
        const bool h2 = i2 < L.n;
        R t1 = 0., t2 = 0.;
        ell_acc2<6, false>(t1, t2, L.n, L.w, L.nbr, L.anb, i, i2, h2, [&](int k) { return x[k]; });
        dst[i] = (l == 0 ? (R)in[i] : L.b[i]) - L.ac[i] * x[i] - t1;
        if (h2) dst[i2] = (l == 0 ? (R)in[i2] : L.b[i2]) - L.ac[i2] * x[i2] - t2;
      }
      return;
    }
    level_rows(sc, L.n, l, [&](auto g, long i, bool act, int q) {
      constexpr int G = decltype(g)::value;
      R t = 0.;
      if (act) t = ell_part<G, G == 1 ? 8 : 4>(L.n, L.w, L.nbr, L.anb, i, q, [&](int k) { return x[k]; });
      t = gsum<G>(t);
      if (act && q == 0) dst[i] = (l == 0 ? (R)in[i] : L.b[i]) - L.ac[i] * x[i] - t;
    });
  }
  // further Jacobi sweeps in place: residual into t, then the update
  __device__ void sweeps(int l, const double *in, R *x, int n) {
    const LevelDev<R> L = lev[l];
    Scope sc = pc_scope(L);
    for (int s = 0; s < n; s++) {
      residual(l, in, x, L.t);
      enter(sc);
      if (sc.active()) for (long i = sc.tid0(); i < L.n; i += sc.nth()) x[i] = x[i] + om(l) * L.t[i] / L.ac[i];
    }
  }
  // out = M^-1 in.  Callers have made `in` visible grid-wide.
  __device__ void run(const double *__restrict__ in, double *__restrict__ out) {
    Scope g; g.grid = true;
    {
      const LevelDev<R> L0 = lev[0];
      for (long i = g.tid0(); i < L0.n; i += g.nth()) L0.x[i] = omega0 * (R)in[i] / L0.ac[i];
    }
    last.grid = true;
    last.team = false;
    sweeps(0, in, lev[0].x, pre - 1);
    for (int l = 0; l < lc; l++) {
      const LevelDev<R> L = lev[l], C = lev[l + 1];
      residual(l, in, L.x, L.r);
      Scope scc = pc_scope(C);
      enter(scc);
      const bool first_sweep = l + 1 < lc || !direct;
      if (scc.active() && scc.nth() < 2L * C.n) {   // a thread per coarse row
        for (long P = scc.tid0(); P < C.n; P += scc.nth()) {
          R s = 0.;
          const int c0 = C.rptr[P], c1 = C.rptr[P + 1];
          for (int c = c0; c < c1; c++) s = s + L.r[C.rlist[c]];
          C.b[P] = s;
          if (first_sweep) C.x[P] = om(l + 1) * s / C.ac[P];
        }
      } else if (scc.active())
        level_rows(scc, C.n, l + 1, [&](auto gg, long P, bool act, int q) {
          constexpr int G = decltype(gg)::value;
          R s = 0.;
          if (act)
            for (int c = C.rptr[P] + q; c < C.rptr[P + 1]; c += G) s = s + L.r[C.rlist[c]];
          s = gsum<G>(s);
          if (act && q == 0) {
            C.b[P] = s;
            if (first_sweep) C.x[P] = om(l + 1) * s / C.ac[P];
          }
        });
      if (l + 1 < lc) sweeps(l + 1, in, C.x, pre - 1);
    }
    const LevelDev<R> Cc = lev[lc];
    if (direct) {
      Scope c0; c0.grid = false;
      enter(c0);
      if (cta_id() == 0) {
        const int n = Cc.n, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
        for (int i = threadIdx.x >> 5; i < n; i += nw) {
          double t = 0.;
          for (int j = lane; j < n; j += 32) t += sinv[(long)i * n + j] * (double)Cc.b[j];
          t = wsum(t);
          if (lane == 0) Cc.r[i] = (R)t;
        }
      }
    } else {
      sweeps(lc, in, Cc.x, coarse_sweeps - 1);
      Scope sc = pc_scope(Cc);
      enter(sc);
      if (sc.active()) for (long i = sc.tid0(); i < Cc.n; i += sc.nth()) Cc.r[i] = Cc.x[i];
    }
    for (int l = lc - 1; l >= 0; l--) {
      const LevelDev<R> L = lev[l];
      const R *__restrict__ xc = lev[l + 1].r;
      Scope sl = pc_scope(L);
      const bool to_out = l == 0 && post == 1;
      enter(sl);
      if (sl.active() && (l == 0 || sl.nth() < 2L * L.n)) {
        // a thread per row: prolong in place (x += alpha x_c[parent], each row
        // its own), then the smoothing sweep gathers x directly -- two memory
        // latencies per slot round instead of three
        const long t0 = sl.tid0(), nt = sl.nth();
        for (long i = t0; i < L.n; i += nt) L.x[i] = L.x[i] + al(l) * xc[L.parent[i]];
        enter(sl);
        for (long i = t0; i < L.n; i += 2 * nt) {
          const long i2 = i + nt;
          const bool h2 = i2 < L.n;
          R t1 = 0., t2 = 0.;
          ell_acc2<6, false>(t1, t2, L.n, L.w, L.nbr, L.anb, i, i2, h2, [&](int k) { return L.x[k]; });
          R xi = L.x[i], bi = l == 0 ? (R)in[i] : L.b[i];
          R xn = xi + om(l) * (bi - L.ac[i] * xi - t1) / L.ac[i];
          if (to_out) out[i] = (double)xn; else L.r[i] = xn;
          if (h2) {
            R xj = L.x[i2], bj = l == 0 ? (R)in[i2] : L.b[i2];
            R xm = xj + om(l) * (bj - L.ac[i2] * xj - t2) / L.ac[i2];
            if (to_out) out[i2] = (double)xm; else L.r[i2] = xm;
          }
        }
      } else if (sl.active())
        level_rows(sl, L.n, l, [&](auto gg, long i, bool act, int q) {
          constexpr int G = decltype(gg)::value;
          R t = 0.;
          if (act)
            t = ell_part<G, G == 1 ? 8 : 4>(L.n, L.w, L.nbr, L.anb, i, q,
                                            [&](int k) { return L.x[k] + al(l) * xc[L.parent[k]]; });
          t = gsum<G>(t);
          if (act && q == 0) {
            R xi = L.x[i] + al(l) * xc[L.parent[i]];
            R bi = l == 0 ? (R)in[i] : L.b[i];
            R xn = xi + om(l) * (bi - L.ac[i] * xi - t) / L.ac[i];
            if (to_out) out[i] = (double)xn; else L.r[i] = xn;
          }
        });
      if (!to_out) sweeps(l, in, L.r, post - 1);
    }
    if (post > 1) {
      enter(g);
      const LevelDev<R> L0 = lev[0];
      for (long i = g.tid0(); i < L0.n; i += g.nth()) out[i] = (double)L0.r[i];
    }
    enter(g);
  }

  // ------------------------------------------------------------ fused V-cycle
  // The same V-cycle (one pre- and one post-sweep, dense coarsest inverse) in
  // one barrier phase per level and leg, with the same arithmetic in the same
  // order as run():
  //   down: the restriction into level l+1 forms the residual of each child
  //     on the fly (no residual array, no phase of its own) for the first
  //     FS_PC_FUSE_DOWN levels; a warp takes a chunk of coarse rows, a lane
  //     two children, and each coarse row sums its children's residuals in
  //     ascending order through shuffles;
  //   up: the sweep of a row of level l >= 2 scatters its new value, times
  //     alpha, to the row's children on level l-1 (the prolongation: every
  //     finer row has one parent, so no two writes meet), and the coarsest
  //     level's dense solve does the same; level 1's sweep keeps its values
  //     and level 0 gathers them through parent (prolong0); level 0's sweep
  //     writes `out`.  (The restriction fused with the residual measured
  //     slower than the two phases on every level, so FS_PC_FUSE_DOWN is 0.)
  // The caller has set x_0 = omega0 in / ac_0 and passed a grid barrier.
  __device__ void restrict_fused(int l, const double *__restrict__ in) {
    const LevelDev<R> L = lev[l], C = lev[l + 1];
    Scope sc = pc_scope(L);
    enter(sc);
    if (!sc.active()) return;
    const bool first_sweep = l + 1 < lc || !direct;
    const R omc = om(l + 1);
    const int lane = threadIdx.x & 31;
    const long w0 = sc.tid0() >> 5, nw = sc.nth() >> 5;
    for (long k = w0; k < C.nchunk; k += nw) {
      const int P0 = C.chunk[k], P1 = C.chunk[k + 1];
      const int e0 = C.rptr[P0], e1 = C.rptr[P1];
      const int P = P0 + lane;
      const bool hasP = P < P1;
      const int ra0 = hasP ? C.rptr[P] : e1, ra1 = hasP ? C.rptr[P + 1] : e1;
      R s = 0.;
      for (int base = e0; base < e1; base += 64) {
        const int ea = base + lane, eb = ea + 32;
        const bool hb = eb < e1;
        const long ia = C.rlist[ea < e1 ? ea : e0], ib = C.rlist[hb ? eb : e0];
        R t1 = 0., t2 = 0.;
        ell_acc2<6, false>(t1, t2, L.n, L.w, L.nbr, L.anb, ia, ib, hb, [&](int q) { return L.x[q]; });
        const R va = (l == 0 ? (R)in[ia] : L.b[ia]) - L.ac[ia] * L.x[ia] - t1;
        R vb = 0.;
        if (hb) vb = (l == 0 ? (R)in[ib] : L.b[ib]) - L.ac[ib] * L.x[ib] - t2;
        // this lane's coarse row: its children inside [base, base+64), in order
        const int lo = ra0 > base ? ra0 : base, hi = ra1 < base + 64 ? ra1 : base + 64;
        const int cnt = hi > lo ? hi - lo : 0;
        const int mx = __reduce_max_sync(0xffffffffu, cnt);
        for (int m = 0; m < mx; m++) {
          const int off = lo + m - base;
          const R xa = __shfl_sync(0xffffffffu, va, off & 31);
          const R xb = __shfl_sync(0xffffffffu, vb, off & 31);
          if (m < cnt) s = s + (off < 32 ? xa : xb);
        }
      }
      if (hasP) {
        C.b[P] = s;
        if (first_sweep) C.x[P] = omc * s / C.ac[P];
      }
    }
  }
  // the residual phase and the restriction of run() (levels past FS_PC_FUSE_DOWN)
  __device__ void restrict_plain(int l, const double *__restrict__ in) {
    const LevelDev<R> L = lev[l], C = lev[l + 1];
    residual(l, in, L.x, L.r);
    Scope scc = pc_scope(C);
    enter(scc);
    if (!scc.active()) return;
    const bool first_sweep = l + 1 < lc || !direct;
    if (scc.nth() < 2L * C.n) {
      for (long P = scc.tid0(); P < C.n; P += scc.nth()) {
        R s = 0.;
        const int c0 = C.rptr[P], c1 = C.rptr[P + 1];
        // children's residuals eight at a time: their list entries, then their
        // values, all in flight before the (ascending) sum
        for (int c = c0; c < c1; c += 8) {
          int f[8];
          R v[8];
#pragma unroll
          for (int u = 0; u < 8; u++) f[u] = c + u < c1 ? C.rlist[c + u] : -1;
#pragma unroll
          for (int u = 0; u < 8; u++) v[u] = f[u] >= 0 ? L.r[f[u]] : (R)0.;
#pragma unroll
          for (int u = 0; u < 8; u++) if (f[u] >= 0) s = s + v[u];
        }
        C.b[P] = s;
        if (first_sweep) C.x[P] = om(l + 1) * s / C.ac[P];
      }
    } else
      level_rows(scc, C.n, l + 1, [&](auto gg, long P, bool act, int q) {
        constexpr int G = decltype(gg)::value;
        R s = 0.;
        if (act)
          for (int c = C.rptr[P] + q; c < C.rptr[P + 1]; c += G) s = s + L.r[C.rlist[c]];
        s = gsum<G>(s);
        if (act && q == 0) {
          C.b[P] = s;
          if (first_sweep) C.x[P] = om(l + 1) * s / C.ac[P];
        }
      });
  }
  // x_{l-1}[c] += d for the children c of row i of level l (d = alpha x_l[i])
  __device__ __forceinline__ void scatter_children(const LevelDev<R> &L, R *__restrict__ xf, long i, R d, int q0,
                                                   int step) {
    const int c1 = L.rptr[i + 1];
    for (int c = L.rptr[i] + q0; c < c1; c += 4 * step) {
      int f[4];
      R v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) f[u] = c + u * step < c1 ? L.rlist[c + u * step] : -1;
#pragma unroll
      for (int u = 0; u < 4; u++) if (f[u] >= 0) v[u] = xf[f[u]];
#pragma unroll
      for (int u = 0; u < 4; u++) if (f[u] >= 0) xf[f[u]] = v[u] + d;
    }
  }
  // the post-sweep of level l, then its prolongation into level l-1 (l >= 1)
  // or the result into `out` (l = 0)
  __device__ void smooth_scatter(int l, const double *__restrict__ in, double *__restrict__ out) {
    const LevelDev<R> L = lev[l];
    Scope sl = pc_scope(L);
    enter(sl);
    if (!sl.active()) return;
    R *__restrict__ xf = l > 0 ? lev[l - 1].x : nullptr;
    const R af = l > 0 ? al(l - 1) : (R)0.;
    if (l == 0 || sl.nth() < 2L * L.n) {   // a thread per row, two rows per step
      const long t0 = sl.tid0(), nt = sl.nth();
      for (long i = t0; i < L.n; i += 2 * nt) {
        const long i2 = i + nt;
        const bool h2 = i2 < L.n;
        R t1 = 0., t2 = 0.;
        ell_acc2<6, false>(t1, t2, L.n, L.w, L.nbr, L.anb, i, i2, h2, [&](int k) { return L.x[k]; });
        R xi = L.x[i], bi = l == 0 ? (R)in[i] : L.b[i];
        R xn = xi + om(l) * (bi - L.ac[i] * xi - t1) / L.ac[i];
        R xm = 0.;
        if (h2) {
          R xj = L.x[i2], bj = l == 0 ? (R)in[i2] : L.b[i2];
          xm = xj + om(l) * (bj - L.ac[i2] * xj - t2) / L.ac[i2];
        }
        if (l == 0) {
          out[i] = (double)xn;
          if (h2) out[i2] = (double)xm;
        } else if (gather_into(l)) {
          L.r[i] = xn;
          if (h2) L.r[i2] = xm;
        } else {
          scatter_children(L, xf, i, af * xn, 0, 1);
          if (h2) scatter_children(L, xf, i2, af * xm, 0, 1);
        }
      }
      return;
    }
    level_rows(sl, L.n, l, [&](auto gg, long i, bool act, int q) {
      constexpr int G = decltype(gg)::value;
      R t = 0.;
      if (act) t = ell_part<G, G == 1 ? 8 : 4>(L.n, L.w, L.nbr, L.anb, i, q, [&](int k) { return L.x[k]; });
      t = gsum<G>(t);
      if (act) {
        R xi = L.x[i], bi = L.b[i];
        R xn = xi + om(l) * (bi - L.ac[i] * xi - t) / L.ac[i];
        if (!gather_into(l)) scatter_children(L, xf, i, af * xn, q, G);
        else if (q == 0) L.r[i] = xn;
      }
    });
  }
  // level 1's post-sweep leaves its result in its r, and level 0 gathers the
  // correction through parent in a phase of its own (x_0 += alpha x_1[parent],
  // the same sum the scatter forms): a coalesced pass over the fine rows
  // instead of one read-modify-write per fine row in agglomerate order.  At
  // 128^3 the extra grid barrier costs less than the scattered writes: the
  // FP64 p' solve 2 % faster, and the FP32 one, which ran the unfused cycle
  // before, 10 %.
  __device__ __forceinline__ bool gather_into(int l) const { return l == 1 && lc >= 2; }
  __device__ void prolong0() {
    const LevelDev<R> L = lev[0];
    const R *__restrict__ xc = lev[1].r;
    Scope g;
    g.grid = true;
    enter(g);
    const R a0 = al(0);
    for (long i = g.tid0(); i < L.n; i += g.nth()) L.x[i] = L.x[i] + a0 * xc[L.parent[i]];
  }
  // the dense coarsest solve (CTA 0, warps on rows), scattered into level lc-1
  __device__ void coarsest_scatter() {
    Scope c0;
    c0.grid = false;
    enter(c0);
    if (cta_id() != 0) return;
    const LevelDev<R> Cc = lev[lc];
    R *__restrict__ xf = lev[lc - 1].x;
    const R af = al(lc - 1);
    const int n = Cc.n, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = threadIdx.x >> 5; i < n; i += nw) {
      double t = 0.;
      for (int j = lane; j < n; j += 32) t += sinv[(long)i * n + j] * (double)Cc.b[j];
      t = wsum(t);
      t = __shfl_sync(0xffffffffu, t, 0);
      scatter_children(Cc, xf, i, af * (R)t, lane, 32);
    }
  }
  // ------------------------------------------------------------ Gauss-Seidel V-cycle
  // One multicolour Gauss-Seidel pass over level l in place: the colours in
  // order (forward) or reversed (backward); rows of one colour read only
  // rows of other colours, so each colour is one phase of independent rows.
  __device__ void gs_colours(int l, const double *__restrict__ in, R *__restrict__ x, bool backward) {
    const LevelDev<R> L = lev[l];
    Scope sc = pc_scope(L);
    for (int cc = 0; cc < L.ncolors; cc++) {
      const int c = backward ? L.ncolors - 1 - cc : cc;
      enter(sc);
      if (!sc.active()) continue;
      const int r0 = L.color_ptr[c], r1 = L.color_ptr[c + 1];
      for (long q = r0 + sc.tid0(); q < r1; q += sc.nth()) {
        const int i = L.color_rows[q];
        const R t = ell_acc<6, false>((R)0., L.n, L.w, L.nbr, L.anb, i, [&](int k) { return x[k]; });
        const R bi = l == 0 ? (R)in[i] : L.b[i];
        x[i] = (bi - t) / L.ac[i];
      }
    }
  }
  // The V-cycle with symmetric multicolour Gauss-Seidel smoothing on the
  // levels below FS_PC_GS_LEVELS (a forward pass from zero before the
  // restriction and, after the correction x += alpha x_c[parent], a backward
  // pass) and the damped Jacobi sweeps of run() on the others; the coarsest
  // level by the dense inverse.  Results stay in each level's x.  out =
  // M^-1 in; callers have made `in` visible.
  __device__ void run_gs(const double *__restrict__ in, double *__restrict__ out) {
    Scope g;
    g.grid = true;
    const LevelDev<R> L0 = lev[0];
    for (long i = g.tid0(); i < L0.n; i += g.nth()) L0.x[i] = (R)0.;
    last.grid = true;
    last.team = false;
    gs_colours(0, in, L0.x, false);
    for (int l = 0; l < lc; l++) {
      const LevelDev<R> L = lev[l], C = lev[l + 1];
      residual(l, in, L.x, L.r);
      Scope scc = pc_scope(C);
      enter(scc);
      const bool gsc = l + 1 < FS_PC_GS_LEVELS;
      const R omc = (gsc || l + 1 == lc) ? (R)0. : om(l + 1);   // Jacobi: the first sweep from zero
      if (scc.active())
        for (long P = scc.tid0(); P < C.n; P += scc.nth()) {
          R s = 0.;
          for (int c = C.rptr[P]; c < C.rptr[P + 1]; c++) s = s + L.r[C.rlist[c]];
          C.b[P] = s;
          C.x[P] = omc * s / C.ac[P];
        }
      if (l + 1 < lc && gsc) gs_colours(l + 1, in, C.x, false);
    }
    {
      Scope c0;
      c0.grid = false;
      enter(c0);
      if (cta_id() == 0) {
        const LevelDev<R> Cc = lev[lc];
        const int n = Cc.n, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
        for (int i = threadIdx.x >> 5; i < n; i += nw) {
          double t = 0.;
          for (int j = lane; j < n; j += 32) t += sinv[(long)i * n + j] * (double)Cc.b[j];
          t = wsum(t);
          if (lane == 0) Cc.x[i] = (R)t;
        }
      }
    }
    for (int l = lc - 1; l >= 0; l--) {
      const LevelDev<R> L = lev[l];
      const R *__restrict__ xc = lev[l + 1].x;
      Scope sl = pc_scope(L);
      enter(sl);
      if (sl.active())
        for (long i = sl.tid0(); i < L.n; i += sl.nth()) L.x[i] = L.x[i] + al(l) * xc[L.parent[i]];
      if (l < FS_PC_GS_LEVELS) {
        gs_colours(l, in, L.x, true);
      } else {   // one damped Jacobi sweep in place: residual into t, then the update
        residual(l, in, L.x, L.t);
        enter(sl);
        if (sl.active()) for (long i = sl.tid0(); i < L.n; i += sl.nth()) L.x[i] = L.x[i] + om(l) * L.t[i] / L.ac[i];
      }
    }
    enter(g);
    for (long i = g.tid0(); i < L0.n; i += g.nth()) out[i] = (double)L0.x[i];
    enter(g);
  }

  __device__ void run_fused(const double *__restrict__ in, double *__restrict__ out) {
    Scope g;
    g.grid = true;
    last.grid = true;
    last.team = false;
    synced = true;   // the caller's grid barrier stands for the first phase's
    for (int l = 0; l < lc; l++) {
      if (l < FS_PC_FUSE_DOWN) restrict_fused(l, in);
      else restrict_plain(l, in);
    }
    coarsest_scatter();
    for (int l = lc - 1; l >= 0; l--) {
      if (l == 0 && gather_into(1)) prolong0();
      smooth_scatter(l, in, out);
    }
    enter(g);
  }
};

// rows i and i2 (when h2) of A x at once (ell_acc2)
template <class A>
__device__ __forceinline__ void row_ax2(const A &a, long i, long i2, bool h2, const double *x, double &t1, double &t2) {
  t1 = 0.0;
  t1 = t1 + a.ac[i] * x[i];
  t2 = 0.0;
  if (h2) t2 = t2 + a.ac[i2] * x[i2];
  ell_acc2<6, false>(t1, t2, a.N, a.W, a.cn, a.anb, i, i2, h2, [&](int k) { return x[k]; });
}

// apply the preconditioner: out (FP64) = M^-1 in (FP64), via the R-precision
// V-cycle; `fused`: the caller has set x_0 = omega0 in / ac_0 (run_fused)
// MODE: 0 the V-cycle of run(), 1 run_fused(), 2 run_gs()
template <class R, int MODE>
__device__ void apply_prec(Sync &S, const AmgKArgs<R> &a, const double *in, double *out, unsigned &gen) {
  Scope all;
  all.grid = true;
  PCycle<R> C{S, a.lev, a.lc, a.direct != 0, a.sinv, a.pre, a.post, 20, (R)FS_MG_OMEGA, (R)FS_MG_ALPHA, all,
               (R)FS_MG_OMEGA0, (R)FS_MG_ALPHA0, a.teambar, a.status, gen, a.team_extra, false};
  if (MODE == 1) C.run_fused(in, out);
  else if (MODE == 2) C.run_gs(in, out);
  else C.run(in, out);
  gen = C.gen;
}

// mean of the right-hand side of a pure-Neumann system (every row sums to
// zero), else 0; the same grid-deterministic sums in every kernel that calls it
template <class R>
__device__ double rhs_mean(Sync &S, const AmgKArgs<R> &a) {
  const int N = a.N;
  const long t0 = (long)cta_id() * blockDim.x + threadIdx.x, nt = (long)cta_count() * blockDim.x;
  double nonsing = 0., bsum = 0.;
  for (long i = t0; i < N; i += nt) {
    double rs = a.ac[i];
    for (int j = 0; j < a.W; j++)
      if (a.cn[(long)j * N + i] >= 0) rs += a.anb[(long)j * N + i];
    nonsing += fabs(rs) > 1e-9 * fabs(a.ac[i]) ? 1. : 0.;
    bsum += a.bc[i];
  }
  double n_nonsing, b_total;
  S.sum2(nonsing, bsum, n_nonsing, b_total);
  return n_nonsing == 0. ? b_total / N : 0.;
}

// The initial guess of k_amg_bicgstab, one cooperative launch before it: the
// combination x = sum_j c_j x_j of the basis vectors (previous p' solutions,
// the network's guess) that minimises |b - A x|, least squares over their
// span, so |b - A x| <= |b|.  The normal equations (Gram matrix of the A x_j)
// are solved by every CTA alike from grid-deterministic sums, by a Cholesky
// factorisation with a relative diagonal shift.  x goes to a.x and fit[0] = 1;
// a failed factorisation leaves fit[0] = 0 (the solve starts from zero).
template <class R, int NX>
__device__ __forceinline__ void guess_fit_body(const AmgKArgs<R> a) {
  constexpr int NG = NX * (NX + 1) / 2, K = NG + NX + 1;
  Sync S(a.part);
  const double bmean = rhs_mean(S, a);
  double c[NX];
  bool fell_back;
  const int N = a.N, W = a.W;
  const long t0 = (long)cta_id() * blockDim.x + threadIdx.x, nt = (long)cta_count() * blockDim.x;
  const double *xs[NX];
#pragma unroll
  for (int j = 0; j < NX; j++) xs[j] = a.xs[j];
  // Gram matrix G_jk = (A x_j).(A x_k) (upper triangle), g_j = (A x_j).b, |b|^2;
  // each row of A is read once for all basis vectors, its slots in order
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; k++) acc[k] = 0.;
  for (long i = t0; i < N; i += nt) {
    double y[NX];
    const double aci = a.ac[i];
#pragma unroll
    for (int j = 0; j < NX; j++) { double t = 0.; t = t + aci * xs[j][i]; y[j] = t; }
    for (int w0 = 0; w0 < W; w0 += 4) {
      int kk[4];
      double av[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const bool in = w0 + u < W;
        kk[u] = in ? a.cn[(long)(w0 + u) * N + i] : -1;
        av[u] = in ? a.anb[(long)(w0 + u) * N + i] : 0.;
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (kk[u] >= 0)
#pragma unroll
          for (int j = 0; j < NX; j++) y[j] = y[j] + av[u] * xs[j][kk[u]];
    }
    const double b1 = a.bc[i] - bmean;
    int q = 0;
#pragma unroll
    for (int j = 0; j < NX; j++)
#pragma unroll
      for (int k = j; k < NX; k++) acc[q++] += y[j] * y[k];
#pragma unroll
    for (int j = 0; j < NX; j++) acc[NG + j] += y[j] * b1;
    acc[NG + NX] += b1 * b1;
  }
  double tot[K];
  S.sumKt<K>(acc, tot);
  // Cholesky of G + 1e-12 max(diag) I, then the two triangular solves (row-major L)
  double L[NX][NX];
  double dmax = 0.;
  {
    int q = 0;
#pragma unroll
    for (int j = 0; j < NX; j++)
#pragma unroll
      for (int k = j; k < NX; k++) { L[k][j] = tot[q]; if (k == j) dmax = fmax(dmax, tot[q]); q++; }
  }
  bool ok = dmax > 0. && isfinite(dmax);
#pragma unroll
  for (int j = 0; j < NX; j++) {
    if (!ok) break;
    double d = L[j][j] + 1e-12 * dmax;
    for (int k = 0; k < j; k++) d -= L[j][k] * L[j][k];
    if (!(d > 1e-14 * dmax)) { ok = false; break; }
    d = sqrt(d);
    L[j][j] = d;
#pragma unroll
    for (int r = j + 1; r < NX; r++) {
      double v = L[r][j];
      for (int k = 0; k < j; k++) v -= L[r][k] * L[j][k];
      L[r][j] = v / d;
    }
  }
  if (ok) {
    double z[NX];
#pragma unroll
    for (int j = 0; j < NX; j++) {
      double v = tot[NG + j];
      for (int k = 0; k < j; k++) v -= L[j][k] * z[k];
      z[j] = v / L[j][j];
    }
#pragma unroll
    for (int j = NX - 1; j >= 0; j--) {
      double v = z[j];
      for (int k = j + 1; k < NX; k++) v -= L[k][j] * c[k];
      c[j] = v / L[j][j];
    }
#pragma unroll
    for (int j = 0; j < NX; j++) if (!isfinite(c[j])) ok = false;
  }
  if (!ok)
#pragma unroll
    for (int j = 0; j < NX; j++) c[j] = 0.;
  fell_back = !ok;
  for (long i = t0; i < N; i += nt) {
    double xi = 0.;
#pragma unroll
    for (int j = 0; j < NX; j++) xi += c[j] * xs[j][i];
    a.x[i] = xi;
  }
  if (cta_id() == 0 && threadIdx.x == 0) {
    a.fit[0] = fell_back ? 0 : 1;
    if (a.nncnt) { a.nncnt[1] += 1; if (fell_back) a.nncnt[0] += 1; }
  }
}


// right-preconditioned BiCGSTAB (van der Vorst 1992) with a multigrid V-cycle:
// MODE 0 run(), 2 run_gs() (multicolour Gauss-Seidel smoothing), 1 the fused
// V-cycle (one pre- and one post-sweep, dense coarsest level), whose first
// sweep from zero, x_0 = omega0 in / ac_0, rides on the loops that form p and s.
// Four grid synchronisations per iteration besides the V-cycles': the sums
// after v = A y and after s, the sums after t = A z, and the barrier after one
// pass that updates x and r and forms the next p.  That pass needs beta
// before |r|^2 and r0.r of the new r are summed; both come from the t-pass
// sums instead: r0.r_new = r0.s - omega r0.t, and |s - omega t|^2 = |s|^2 -
// omega t.s (omega = t.s / t.t), with |s|^2 summed fresh from s, so the
// estimate's rounding is relative to |s|^2 of this iteration.  Only an
// iteration whose estimate says it has converged (or the last one) sums |r|^2
// and r0.r of the stored r instead, so the exit is always decided on a
// residual summed from its vector, and a solve that has not really converged
// continues with p formed in a separate pass.
template <class R, int MODE>
__device__ __forceinline__ void amg_bicgstab_body(const AmgKArgs<R> a) {
  Sync S(a.part);
  unsigned gen = 0;   // team-barrier generation (the counters are zeroed before the launch)
  const int N = a.N;
  Scope g; g.grid = true;
  const long t0 = g.tid0(), nt = g.nth();
  R *__restrict__ x0v = a.lev[0].x;
  const R *__restrict__ ac0 = a.lev[0].ac;
  const R om0 = (R)FS_MG_OMEGA0;
  // start from the initial guess k_guess_fit left in x (the least-squares
  // combination of the basis vectors; fit[0] = 0 when it fell back), or from zero.
  // A pure-Neumann system (every row sums to zero: the closed-cavity p'
  // system) is singular.  Its right-hand side is taken with its mean removed,
  // the part a solution can match; otherwise, once the outer iterations have
  // converged the mean (rounding in the mass fluxes) is no longer small
  // against |b|, the tolerance cannot be met and the iterates drift.  The
  // constant null vector is left to the caller (pressure reference cell).
  const double bmean = rhs_mean(S, a);
  const bool has_x = a.nx > 0 && a.fit[0] != 0;
  double l0 = 0., l1 = 0., l2 = 0.;
  for (long i = t0; i < N; i += nt) {
    const double b1 = a.bc[i] - bmean;
    double ri = b1;
    if (has_x) {
      double t = 0.;
      t = t + a.ac[i] * a.x[i];
      t = ell_acc<8, false>(t, a.N, a.W, a.cn, a.anb, i, [&](int k) { return a.x[k]; });
      ri = ri - t;
    } else {
      a.x[i] = 0.;
    }
    // the first p is r (beta's factors are 1 and p = v = 0 before it)
    a.r[i] = ri; a.r0[i] = ri; a.p[i] = ri; a.v[i] = 0.;
    if (MODE == 1) x0v[i] = om0 * (R)ri / ac0[i];
    l0 += ri * ri;
    l1 += b1 * b1;
  }
  double rr, bb, dum;
  S.sum2(l0, l1, rr, bb);
  double normb = sqrt(bb), alpha = 1., omega = 1.;
  int k = 0;
  double resn = sqrt(rr);
  // rho = r0 . r of the iteration; rho_next that of the next one, summed from
  // the stored r when p still has to be formed (p_ready false)
  double rho = rr, rho_next = rr;
  bool p_ready = true;
  if (!(rr != 0.) || !isfinite(rr)) p_ready = false;   // the loop's breakdown test takes it
  while (k < a.maxit && resn > a.tol * normb && normb > 0.) {
    k++;
    if (!p_ready) {
      const double rho1 = rho_next;
      // breakdown (r0 . r vanished: r at round-off): keep x.  Every CTA holds
      // the same sums, so every CTA takes the same branch.
      if (!(rho1 != 0.) || !isfinite(rho1)) break;
      const double beta = (rho1 / rho) * (alpha / omega);
      rho = rho1;
      for (long i = t0; i < N; i += nt) {
        const double pi = a.r[i] + beta * (a.p[i] - omega * a.v[i]);
        a.p[i] = pi;
        if (MODE == 1) x0v[i] = om0 * (R)pi / ac0[i];
      }
      S.all();
    }
    p_ready = false;
    apply_prec<R, MODE>(S, a, a.p, a.y, gen);                       // y = M^-1 p
    l0 = 0.;
    for (long i = t0; i < N; i += 2 * nt) {
      const long i2 = i + nt;
      const bool h2 = i2 < N;
      double v1, v2;
      row_ax2(a, i, i2, h2, a.y, v1, v2);
      a.v[i] = v1; l0 += a.r0[i] * v1;
      if (h2) { a.v[i2] = v2; l0 += a.r0[i2] * v2; }
    }
    double rv;
    S.sum2(l0, 0., rv, dum);
    if (!(rv != 0.) || !isfinite(rho / rv)) break;
    alpha = rho / rv;
    l0 = 0.; l1 = 0.;
    for (long i = t0; i < N; i += nt) {
      const double si = a.r[i] - alpha * a.v[i];
      a.s[i] = si;
      l0 += si * si;
      l1 += a.r0[i] * si;
      if (MODE == 1) x0v[i] = om0 * (R)si / ac0[i];
    }
    double ss, r0s;
    S.sum2(l0, l1, ss, r0s);
    if (sqrt(ss) <= a.tol * normb) {
      for (long i = t0; i < N; i += nt) a.x[i] = a.x[i] + alpha * a.y[i];
      resn = sqrt(ss);
      break;
    }
    apply_prec<R, MODE>(S, a, a.s, a.z, gen);                       // z = M^-1 s
    l0 = 0.; l1 = 0.; l2 = 0.;
    for (long i = t0; i < N; i += 2 * nt) {
      const long i2 = i + nt;
      const bool h2 = i2 < N;
      double t1, t2;
      row_ax2(a, i, i2, h2, a.z, t1, t2);
      a.t[i] = t1; l0 += t1 * a.s[i]; l1 += t1 * t1; l2 += a.r0[i] * t1;
      if (h2) { a.t[i2] = t2; l0 += t2 * a.s[i2]; l1 += t2 * t2; l2 += a.r0[i2] * t2; }
    }
    double ts, tt, r0t;
    S.sum3(l0, l1, l2, ts, tt, r0t);
    if (!(tt > 0.) || !(ts != 0.) || !isfinite(ts / tt)) {
      // t = A z vanished or is orthogonal to s: take the half step and stop
      for (long i = t0; i < N; i += nt) a.x[i] = a.x[i] + alpha * a.y[i];
      resn = sqrt(ss);
      break;
    }
    omega = ts / tt;
    const double rn_est = fmax(ss - omega * ts, 0.);
    const double rho_est = r0s - omega * r0t;
    if (k < a.maxit && sqrt(rn_est) > a.tol * normb && rho_est != 0. && isfinite(rho_est)) {
      // x and r of this iteration and p of the next in one pass
      const double beta = (rho_est / rho) * (alpha / omega);
      rho = rho_est;
      for (long i = t0; i < N; i += nt) {
        a.x[i] = a.x[i] + alpha * a.y[i] + omega * a.z[i];
        const double ri = a.s[i] - omega * a.t[i];
        a.r[i] = ri;
        const double pi = ri + beta * (a.p[i] - omega * a.v[i]);
        a.p[i] = pi;
        if (MODE == 1) x0v[i] = om0 * (R)pi / ac0[i];
      }
      S.all();
      resn = sqrt(rn_est);
      p_ready = true;
    } else {
      l0 = 0.; l1 = 0.;
      for (long i = t0; i < N; i += nt) {
        a.x[i] = a.x[i] + alpha * a.y[i] + omega * a.z[i];
        const double ri = a.s[i] - omega * a.t[i];
        a.r[i] = ri;
        l0 += ri * ri;
        l1 += a.r0[i] * ri;
      }
      double rn;
      S.sum2(l0, l1, rn, rho_next);
      resn = sqrt(rn);
    }
  }
  S.all();
  for (long i = t0; i < N; i += nt) a.dphi[i] = a.x[i];
  if (cta_id() == 0 && threadIdx.x == 0) { *a.iters = k; a.diag[0] = resn; a.diag[1] = normb; }
}

