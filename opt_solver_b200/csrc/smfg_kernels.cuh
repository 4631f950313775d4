// Device kernels of the numeric phase: value placement, per-level front
// set-up, assembly / extend-add, front factorization by size class, the
// supernodal solves and the residual.
#pragma once
#include "smfg_aptp_host.h"
#include "smfg_internal.cuh"
#include "smfg_tc.cuh"

namespace smfg {

// counters[] slots
enum : int { kCArena = 0, kCRows = 1, kCFlags = 2, kCMaxAbs = 3, kCAux = 4, kCEffSmall = 5,
             kCActive = 6, kCGemmFlops = 7, kCTcFlops = 8, kCDeferBytes = 9, kCDeferUpd = 10,
             kCDeferSmall = 11, kCAptpMiss = 12, kCNegSoFar = 13, kCWorkSoFar = 14, kCCount = 15 };
// error flag bits (counters[kCFlags])
enum : unsigned { kFArena = 1u, kFRows = 2u, kFNonfinite = 4u, kFNotPosdef = 8u, kFNonfiniteD = 16u,
                  kFMap = 32u, kFInternal = 64u, kFTcWait = 128u, kFTcCap = 256u, kFSteps = 512u,
                  kFAptpMiss = 1024u, kFInertia = 2048u, kFWork = 4096u };
// team reduction scratch per large front (2 buffers x 16 CTAs x 6 doubles)
constexpr int kTeamRedDoubles = 256;
// flags after which the rest of a factorization is skipped (retried with
// more room, or reported)
constexpr unsigned kFAbort = kFArena | kFRows | kFTcWait | kFTcCap | kFAptpMiss | kFInertia | kFWork;
// fronts recorded per factorization that grew past the APTP size outside the
// large-front path (they join it, and the factorization is redone)
constexpr int kAptpMissCap = 1024;

__device__ __forceinline__ void set_flag(unsigned long long *cnt, unsigned bit) {
  atomicOr(cnt + kCFlags, (unsigned long long)bit);
}

// ---------------------------------------------------------------------------
// Value placement: map_values_to_permuted + S A S (workspace.cpp:129-281,
// factor_indef.cpp:513-559). Each permuted slot sums its caller entries in
// input order, then takes v * (s_row * s_col). max |S A S| and the
// finiteness of every input value are reduced on the way.
__global__ void k_values(const double *__restrict__ vin, int64_t nnz_in, const int *__restrict__ vptr,
                         const int *__restrict__ vsrc, const int *__restrict__ pcp_col,
                         const int *__restrict__ pri, const int *__restrict__ perm,
                         const double *__restrict__ scale, int64_t nnz, double *__restrict__ pv,
                         double *__restrict__ pv_raw, unsigned long long *cnt) {
  __shared__ double red[32];
  double m = 0.0;
  bool bad = false;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz_in; k += stride)
    bad = bad || !isfinite(vin[k]);
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nnz; s += stride) {
    double v = 0.0;
    for (int k = vptr[s]; k < vptr[s + 1]; ++k) v = __dadd_rn(v, vin[vsrc[k]]);
    pv_raw[s] = v;
    if (scale) v = __dmul_rn(v, __dmul_rn(scale[perm[pri[s]]], scale[perm[pcp_col[s]]]));
    pv[s] = v;
    m = fmax(m, fabs(v));
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) set_flag(cnt, kFNonfinite);
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) atomicMax(cnt + kCMaxAbs, (unsigned long long)__double_as_longlong(m));
  }
}

// eff_small of factor_indef.cpp:631-636 from max |S A S|.
__global__ void k_eff_small(unsigned long long *cnt, double small_pivot) {
  const double m = __longlong_as_double((long long)cnt[kCMaxAbs]);
  const double e = (m > 0.0 && m < small_pivot) ? small_pivot * m : small_pivot;
  cnt[kCEffSmall] = (unsigned long long)__double_as_longlong(e);
}

// ---------------------------------------------------------------------------
// Per-level set-up (one block): realized front sizes (delays in), storage
// offsets by exclusive scan, delay offsets of the children in the parent's
// row list (multifrontal_serial.cpp:510-545), assembly work items.
template <int NT>
__global__ void k_level_setup(DevPlan P, DevFactor X, int lo, int hi, int lvl, int nb) {
  static_assert(NT % 32 == 0 && NT <= 1024, "block size");
  constexpr int NW = NT / 32;
  __shared__ long long wa[NW], wr[NW], wb[NW];
  __shared__ long long base_a, base_r, run_a, run_r, run_b;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long *cnt = X.counters;
  if (threadIdx.x == 0) {
    base_a = (long long)cnt[kCArena];
    base_r = (long long)cnt[kCRows];
    run_a = run_r = run_b = 0;
  }
  __syncthreads();
  for (int c0 = lo; c0 < hi; c0 += NT) {
    const int i = c0 + threadIdx.x;
    long long fa = 0, fr = 0, fb = 0;
    int s = -1, f = 0;
    if (i < hi) {
      s = P.lvl_sn[i];
      int nd = 0;
      for (int t = P.child_ptr[s]; t < P.child_ptr[s + 1]; ++t) {
        X.child_doff[t] = nd;
        nd += X.sn_dout[P.child_idx[t]];
      }
      f = nd + P.sn_fsym[s];
      X.sn_nd[s] = nd;
      X.sn_f[s] = f;
      X.sn_ne[s] = nd + P.sn_width[s];
      fa = (long long)f * f + (long long)f * nb;
      fr = f;
      fb = (f + kAsmCols - 1) / kAsmCols;
    }
    // inclusive block scan of (fa, fr, fb): warp shuffles, then the warps'
    // totals scanned by warp 0
    long long va = fa, vr = fr, vb = fb;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long ya = __shfl_up_sync(0xffffffffu, va, o);
      const long long yr = __shfl_up_sync(0xffffffffu, vr, o);
      const long long yb = __shfl_up_sync(0xffffffffu, vb, o);
      if (lane >= o) {
        va += ya;
        vr += yr;
        vb += yb;
      }
    }
    if (lane == 31) {
      wa[warp] = va;
      wr[warp] = vr;
      wb[warp] = vb;
    }
    __syncthreads();
    if (warp == 0) {
      long long ta = lane < NW ? wa[lane] : 0, tr = lane < NW ? wr[lane] : 0, tb = lane < NW ? wb[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long ya = __shfl_up_sync(0xffffffffu, ta, o);
        const long long yr = __shfl_up_sync(0xffffffffu, tr, o);
        const long long yb = __shfl_up_sync(0xffffffffu, tb, o);
        if (lane >= o) {
          ta += ya;
          tr += yr;
          tb += yb;
        }
      }
      if (lane < NW) {
        wa[lane] = ta;
        wr[lane] = tr;
        wb[lane] = tb;
      }
    }
    __syncthreads();
    if (warp > 0) {
      va += wa[warp - 1];
      vr += wr[warp - 1];
      vb += wb[warp - 1];
    }
    if (i < hi) {
      X.sn_off[s] = base_a + run_a + va - fa;
      X.sn_roff[s] = base_r + run_r + vr - fr;
      X.lvl_blk[i + lvl] = (int)(run_b + vb - fb);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      run_a += wa[NW - 1];
      run_r += wr[NW - 1];
      run_b += wb[NW - 1];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    X.lvl_blk[hi + lvl] = (int)run_b;
    cnt[kCArena] = (unsigned long long)(base_a + run_a);
    cnt[kCRows] = (unsigned long long)(base_r + run_r);
    cnt[kCAux] = (unsigned long long)run_b;
    if (base_a + run_a > X.arena_cap) set_flag(cnt, kFArena);
    if (base_r + run_r > X.rows_cap) set_flag(cnt, kFRows);
  }
}

// Rows of each front (children's delayed rows in child order, then its
// symbolic rows) and each child's contribution-block row map into it.
__global__ void k_level_rows(DevPlan P, DevFactor X, int lo, int hi) {
  if (X.counters[kCFlags] & kFAbort) return;
  const int s = P.lvl_sn[lo + blockIdx.x];
  const int64_t roff = X.sn_roff[s];
  const int nd = X.sn_nd[s], f = X.sn_f[s], fsym = P.sn_fsym[s];
  int *rows = X.rows + roff;
  for (int t = P.child_ptr[s]; t < P.child_ptr[s + 1]; ++t) {
    const int c = P.child_idx[t];
    const int dc = X.sn_dout[c];
    const int pc = X.sn_p[c];
    const int fc = X.sn_f[c];
    const int q = fc - pc;
    const int doff = X.child_doff[t];
    const int *crow = X.rows + X.sn_roff[c] + pc;
    int *cmap = X.cbmap + X.sn_roff[c] + pc;
    const int *cpr = P.cpr_idx + P.cpr_off[t];
    for (int u = threadIdx.x; u < q; u += blockDim.x) {
      if (u < dc) {
        rows[doff + u] = crow[u];
        cmap[u] = doff + u;
      } else {
        cmap[u] = nd + cpr[u - dc];
      }
    }
  }
  const int *fr = P.frow_idx + P.frow_ptr[s];
  for (int u = threadIdx.x; u < fsym; u += blockDim.x) rows[nd + u] = fr[u];
  for (int u = threadIdx.x; u < f; u += blockDim.x) X.tags[roff + u] = 0;
}

// Assembly of one level (process_front, multifrontal_serial.cpp:720-789):
// each work item is a block of kAsmCols columns of one front. It zeroes the
// lower part of its columns, adds the original entries of the pivot columns,
// then extend-adds the children's Schur blocks in child order (the
// reference's order of additions, so every entry is the reference's sum).
// A child's block is read in place from its own front.
// First index in [lo, hi) of the increasing a[] whose value is >= key (hi
// if none), by the 32 lanes of a warp: 32 probes a round (one load
// latency), about three rounds for a few thousand entries.
__device__ __forceinline__ int warp_lower_bound(const int *__restrict__ a, int lo, int hi, int key) {
  const int lane = threadIdx.x & 31;
  while (hi - lo > 32) {
    const int step = (hi - lo + 31) / 32;
    const int pos = min(lo + step * (lane + 1) - 1, hi - 1);
    const int nl = __popc(__ballot_sync(0xffffffffu, a[pos] < key));  // a prefix of the lanes
    const int nlo = min(lo + step * nl, hi);
    hi = nl == 32 ? hi : min(lo + step * (nl + 1), hi);
    lo = nlo;
  }
  const int pos = lo + lane;
  return lo + __popc(__ballot_sync(0xffffffffu, pos < hi && a[pos] < key));
}

__global__ void k_level_assemble(DevPlan P, DevFactor X, int lo, int hi, int lvl) {
  unsigned long long *cnt = X.counters;
  if (cnt[kCFlags] & kFAbort) return;
  const int *pref = X.lvl_blk + lo + lvl;  // m + 1 prefix entries
  const int m = hi - lo;
  const int total = pref[m];
  __shared__ int rng[2];
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    int a = 0, b = m;  // largest i with pref[i] <= w
    while (b - a > 1) {
      const int mid = (a + b) >> 1;
      if (pref[mid] <= w) a = mid;
      else b = mid;
    }
    const int s = P.lvl_sn[lo + a];
    const int f = X.sn_f[s], nd = X.sn_nd[s];
    const int j0 = (w - pref[a]) * kAsmCols;
    const int j1 = min(j0 + kAsmCols, f);
    double *F = X.arena + X.sn_off[s];
    const size_t sf = (size_t)f;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    // 1. zero the lower part of columns [j0, j1): a warp per column
    for (int jj = j0 + warp; jj < j1; jj += nwarp) {
      double *Fj = F + jj * sf;
      for (int i = jj + lane; i < f; i += 32) Fj[i] = 0.0;
    }
    __syncthreads();
    // 2. original entries of the pivot columns in [j0, j1): their slots are
    // one contiguous range (consecutive columns), each slot a distinct entry
    const int cs = P.sn_start[s], wdt = P.sn_width[s];
    const int ca = max(j0 - nd, 0), cb = min(j1 - nd, wdt);
    if (ca < cb) {
      const int k0 = P.pcp[cs + ca], k1 = P.pcp[cs + cb];
      for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        int c = ca;  // the column of slot k (at most kAsmCols candidates)
        while (c + 1 < cb && P.pcp[cs + c + 1] <= k) ++c;
        F[(nd + c) * sf + nd + P.amap[k]] += X.pv[k];
      }
    }
    __syncthreads();
    // 3. children in order
    for (int t = P.child_ptr[s]; t < P.child_ptr[s + 1]; ++t) {
      const int c = P.child_idx[t];
      const int pc = X.sn_p[c], fc = X.sn_f[c];
      const int q = fc - pc;
      if (q <= 0) continue;
      const int *cmap = X.cbmap + X.sn_roff[c] + pc;
      // the child's CB rows mapped into [j0, j1): warp 0 finds the first
      // with cmap >= j0, warp 1 the first with cmap >= j1
      if (warp < 2) {
        const int r = warp_lower_bound(cmap, 0, q, warp == 0 ? j0 : j1);
        if (lane == 0) rng[warp] = r;
      }
      __syncthreads();
      const int ja = rng[0], jb = rng[1];
      const double *Fc = X.arena + X.sn_off[c];
      const size_t sfc = (size_t)fc;
      // the child's block columns [ja, jb): a warp per column, lanes over
      // its rows (contiguous in the child, increasing in the parent), four a
      // lane in flight; its targets are distinct
      for (int jj = ja + warp; jj < jb; jj += nwarp) {
        const int lj = cmap[jj];
        const double *Fcj = Fc + (size_t)(pc + jj) * sfc + pc;
        double *Fj = F + (size_t)lj * sf;
        for (int i0 = jj + lane; i0 < q; i0 += 4 * 32) {
          double sv[4], dv[4];
          int li[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int ii = i0 + 32 * u;
            li[u] = -1;
            sv[u] = dv[u] = 0.0;
            if (ii < q) {
              li[u] = cmap[ii];
              if (li[u] < lj) {
                set_flag(cnt, kFMap);
                li[u] = -1;
              } else {
                sv[u] = Fcj[ii];
                dv[u] = Fj[li[u]];
              }
            }
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (li[u] >= 0) Fj[li[u]] = dv[u] + sv[u];
        }
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
template <int NT, bool SMEM>
__device__ void store_front(DevPlan &P, DevFactor &X, int s, const FrontRef &v, int p,
                            const PivotParams &prm, FrontShared &sh, int *inv, double *Fg,
                            int *rows_g, int8_t *tags_g);

// Fronts of at least this many symbolic rows take the multi-block path.
constexpr int kLargeMin = 384;

// In-place unit-LDL^T of the nbp x nbp lower block T (the SPD panels'
// diagonal blocks), all threads of the block: pivot k's reciprocal to
// linv[k], its multipliers l_kj = t_jk / d_k to lm[k][j], then every entry
// (i, j), k < j <= i, takes t_ij - t_ik l_kj (skipped for l_kj = 0) -- per
// entry the one-warp loop's operations in its order. The strictly lower
// part keeps the unscaled values (its multipliers are lm; the callers read
// only the diagonal of T afterwards). Stops at the first pivot that is not
// positive and finite; returns the pivots taken. Starts and ends at a
// barrier. `zero` (shared, optional) is set to 1 when a multiplier is zero.
template <int NB, int NT = 256>
__device__ __forceinline__ int spd_diag_factor(double (*T)[NB + 1], double (*lm)[NB], double *linv, int nbp,
                                               int *zero = nullptr) {
  const int t = threadIdx.x;
  __syncthreads();
  int np = 0;
  for (int k = 0; k < nbp; ++k) {
    const double d = T[k][k];
    if (!(d > 0.0 && isfinite(d))) break;
    const double inv = __drcp_rn(d);  // 1.0 / d, correctly rounded
    if (t == 0) linv[k] = inv;
    // each entry's thread forms the multiplier it needs itself (column k
    // is read, not written, in this step): one barrier a pivot
    for (int e = t; e < NB * NB; e += NT) {
      const int ti = e / NB, tj = e % NB;
      if (tj > k && tj <= ti && ti < nbp) {
        const double l = __dmul_rn(T[tj][k], inv);
        if (ti == tj) {
          lm[k][tj] = l;
          if (zero && l == 0.0) *zero = 1;
        }
        if (l != 0.0) T[ti][tj] = __dsub_rn(T[ti][tj], __dmul_rn(T[ti][k], l));
      }
    }
    __syncthreads();
    ++np;
  }
  return np;
}

// SPD fronts of the blocked size classes (nb = 16, at least
// blocked_min_front rows) in their one block of threads: the medium
// kernel's pivoting steps (tpp_step_blk, one pivot at a time) replaced by
// the large fronts' panel arithmetic. Panels of 16 pivots: the diagonal
// block factored by all threads (spd_diag_factor), every row of the
// panel's columns by one thread (the multiply-subtract chain of
// k_large_panel_spd2's rows, w kept in W), then the medium kernel's own
// deferred update of the eligible columns and, at the end, its Schur update
// of the contribution block. A pivot that is not positive ends the
// pivoting. Returns the pivots taken.
template <int NT>
__device__ int spd_front_panels(FrontRef &v, const PivotParams &prm, FrontShared &sh) {
  constexpr int NB = 16;
  __shared__ double T[NB][NB + 1], lm[NB][NB], linv[NB];
  const int f = v.f, ne = v.ne;
  const size_t sf = (size_t)v.ld;
  double *F = v.F, *W = v.W;  // W row q (f doubles): w of the panel's pivot q
  int p = 0;
  for (int ps = 0; ps < ne; ps += NB) {
    const int pe = min(ne, ps + NB), nbp = pe - ps;
    for (int t = threadIdx.x; t < NB * NB; t += NT) {
      const int r = t / NB, c = t % NB;
      T[r][c] = (r < nbp && c <= r) ? F[(size_t)(ps + c) * sf + ps + r] : 0.0;
    }
    const int np = spd_diag_factor<NB, NT>(T, lm, linv, nbp);
    for (int i = ps + threadIdx.x; i < f; i += NT) {
      double a[NB];
#pragma unroll
      for (int c = 0; c < NB; ++c) a[c] = (c < nbp && ps + c <= i) ? F[(size_t)(ps + c) * sf + i] : 0.0;
#pragma unroll
      for (int k = 0; k < NB; ++k) {
        if (k < np && i > ps + k) {
          const double w = a[k];
          W[(size_t)k * sf + i] = w;
#pragma unroll
          for (int j = k + 1; j < NB; ++j) {
            if (j < nbp && ps + j <= i) {
              const double l = lm[k][j];
              if (l != 0.0) a[j] = __dsub_rn(a[j], __dmul_rn(w, l));
            }
          }
          a[k] = __dmul_rn(w, linv[k]);
        }
      }
#pragma unroll
      for (int c = 0; c < NB; ++c)
        if (c < nbp && ps + c <= i) F[(size_t)(ps + c) * sf + i] = a[c];
    }
    if (threadIdx.x == 0) {
      for (int k = 0; k < np; ++k) {
        v.tags[ps + k] = 1;
        inertia_1x1(T[k][k], prm.eff_small, sh.st);
        const double rem = (double)(f - (ps + k + 1));
        sh.st.flops += rem + rem * (rem + 1.0);
      }
    }
    p = ps + np;
    __syncthreads();
    if (np < nbp) break;
    // the eligible columns past the panel, every row below: the medium
    // kernel's deferred update
    deferred_update_blk<NT>(v, ps, pe, pe, ne);
  }
  // the contribution block: its Schur update over every pivot, as the
  // medium kernel takes it
  schur_update_blk<NT>(v, 0, p, ne);
  return p;
}

// Front factorization + store (process_front's kernel call and D handling,
// multifrontal_serial.cpp:790-945): one block per front of the size class
// [FMIN, FMAX]; SMEM: the front is copied into shared memory.
template <int NT, bool SMEM>
__device__ void factor_one_front(DevPlan &P, DevFactor &X, int s, const PivotParams &prm0,
                                 double *smem) {
  __shared__ FrontShared sh;
  const int f = X.sn_f[s], ne = X.sn_ne[s], nb = prm0.nb;
  const size_t sf = (size_t)f;
  double *Fg = X.arena + X.sn_off[s];
  int *rows_g = X.rows + X.sn_roff[s];
  int8_t *tags_g = X.tags + X.sn_roff[s];
  PivotParams prm = prm0;
  prm.eff_small = __longlong_as_double((long long)X.counters[kCEffSmall]);
  FrontRef v;
  v.ld = f;
  v.f = f;
  v.ne = ne;
  int *inv;
  if (SMEM) {
    // F, then W only where the blocked path runs (the launch's shared
    // memory holds W only for buckets that can reach it), then the ints
    const bool blocked = f >= prm0.blocked_min_front && nb > 1;
    double *F = smem;
    double *W = F + sf * sf;
    int *rows = (int *)(W + (blocked ? sf * nb : 0));
    int *loc = rows + f;
    inv = loc + f;
    int8_t *tags = (int8_t *)(inv + f);
    for (size_t t = threadIdx.x; t < sf * sf; t += NT) F[t] = Fg[t];
    for (int t = threadIdx.x; t < f; t += NT) {
      rows[t] = rows_g[t];
      loc[t] = t;
      tags[t] = 0;
    }
    v.F = F;
    v.W = W;
    v.rows = rows;
    v.tags = tags;
    v.loc = loc;
  } else {
    v.F = Fg;
    v.W = Fg + sf * sf;
    v.rows = rows_g;
    v.tags = tags_g;
    v.loc = X.ploc + X.sn_roff[s];
    inv = X.ploc + X.rows_cap + X.sn_roff[s];
    for (int t = threadIdx.x; t < f; t += NT) v.loc[t] = t;
  }
  if (threadIdx.x == 0) sh.st = FrontStats{0, 0, 0, 0, 0.0};
  __syncthreads();
  const bool spd_panels = prm.posdef && nb == 16 && f >= prm0.blocked_min_front && NT >= 128;
  const int p = spd_panels ? spd_front_panels<NT>(v, prm, sh) : ldlt_factor_front_blk<NT>(v, prm, sh);
  store_front<NT, SMEM>(P, X, s, v, p, prm, sh, inv, Fg, rows_g, tags_g);
}

// D and the stored L of a factored front, its counts, and its children's
// row maps in pivot order (multifrontal_serial.cpp:884-945).
template <int NT, bool SMEM>
__device__ void store_front(DevPlan &P, DevFactor &X, int s, const FrontRef &v, int p,
                            const PivotParams &prm, FrontShared &sh, int *inv, double *Fg,
                            int *rows_g, int8_t *tags_g) {
  const int f = v.f, ne = v.ne;
  const size_t sf = (size_t)f;
  const bool is_root = P.sn_parent[s] < 0;
  int pstore = p;
  if (is_root && p < ne) {
    for (int c = p + threadIdx.x; c < ne; c += NT) v.tags[c] = 0;
    if (threadIdx.x == 0) sh.st.zero += ne - p;
    pstore = ne;
  }
  __syncthreads();
  if (prm.posdef) {
    if (p < ne && threadIdx.x == 0) set_flag(X.counters, kFNotPosdef);
    // L = L_unit sqrt(D), upper part zero
    for (long long t = threadIdx.x; t < (long long)pstore * f; t += NT) {
      const int c = (int)(t / f), i = (int)(t % f);
      double *Lc = v.F + (size_t)c * sf;
      if (i < c) Lc[i] = 0.0;
      else if (i > c) Lc[i] = __dmul_rn(Lc[i], sqrt(Lc[c]));
    }
    __syncthreads();
    for (int c = threadIdx.x; c < pstore; c += NT) {
      double *Lc = v.F + (size_t)c * sf;
      Lc[c] = sqrt(Lc[c]);
    }
  } else {
    // D inline: d on the diagonal, a 2x2 block's off-diagonal in the upper
    // slot (c, c + 1); zero pivots' columns zero.
    bool bad = false;
    for (int c = threadIdx.x; c < pstore; c += NT) {
      const double *Lc = v.F + (size_t)c * sf;
      const int8_t tag = v.tags[c];
      if (tag == 1) bad = bad || !isfinite(Lc[c]);
      else if (tag == 2) bad = bad || !isfinite(Lc[c]) || !isfinite(Lc[c + 1]) || !isfinite(Lc[sf + c + 1]);
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) set_flag(X.counters, kFNonfiniteD);
    for (int c = threadIdx.x; c < pstore; c += NT) {
      if (v.tags[c] == -1) {  // move d10 from (c, c-1) to the upper slot (c-1, c)
        double *Lc = v.F + (size_t)c * sf;
        Lc[c - 1] = v.F[(size_t)(c - 1) * sf + c];
      }
    }
    __syncthreads();
    for (long long t = threadIdx.x; t < (long long)pstore * f; t += NT) {
      const int c = (int)(t / f), i = (int)(t % f);
      double *Lc = v.F + (size_t)c * sf;
      const int8_t tag = v.tags[c];
      if (tag == 0) {
        if (i >= c) Lc[i] = 0.0;
        else Lc[i] = 0.0;
      } else if (i < c) {
        if (!(tag == -1 && i == c - 1)) Lc[i] = 0.0;
      } else if (tag == 2 && i == c + 1) {
        Lc[i] = 0.0;
      }
    }
  }
  __syncthreads();
  if (SMEM) {
    for (size_t t = threadIdx.x; t < sf * sf; t += NT) Fg[t] = v.F[t];
    for (int t = threadIdx.x; t < f; t += NT) {
      rows_g[t] = v.rows[t];
      tags_g[t] = v.tags[t];
    }
  }
  // The children's row maps, built in assembly order, now point at the
  // rows' final (pivot-order) positions: the solves read them that way.
  for (int t = threadIdx.x; t < f; t += NT) inv[v.loc[t]] = t;
  __syncthreads();
  for (int t = P.child_ptr[s]; t < P.child_ptr[s + 1]; ++t) {
    const int c = P.child_idx[t];
    const int pc = X.sn_p[c];
    int *cmap = X.cbmap + X.sn_roff[c] + pc;
    for (int u = threadIdx.x; u < X.sn_f[c] - pc; u += NT) cmap[u] = inv[cmap[u]];
  }
  if (threadIdx.x == 0) {
    X.sn_p[s] = p;
    X.sn_pstore[s] = pstore;
    X.sn_dout[s] = is_root ? 0 : ne - p;
    int *st = X.sn_stat + 4 * s;
    st[0] = sh.st.pos;
    st[1] = sh.st.neg;
    st[2] = sh.st.zero;
    st[3] = sh.st.two_by_two;
    X.sn_flops[s] = sh.st.flops;
  }
}

template <int NT, int FMIN, int FMAX, bool SMEM>
__global__ void __launch_bounds__(NT) k_factor(DevPlan P, DevFactor X, int lo, int hi, PivotParams prm) {
  extern __shared__ __align__(16) double smem[];
  if (X.counters[kCFlags] & kFAbort) return;
  const int s = P.lvl_sn[lo + blockIdx.x];
  const int f = X.sn_f[s];
  if (f < FMIN || f > FMAX || P.sn_large[s]) return;
  if (!SMEM && prm.aptp_min > 0 && !prm.posdef && f >= prm.aptp_min && prm.u >= kWeakPivotRatio) {
    // delays took the front to the APTP size: it must take the large-front
    // path; recorded, and the factorization is redone
    if (threadIdx.x == 0) {
      const unsigned long long i = atomicAdd(X.counters + kCAptpMiss, 1ull);
      if (i < (unsigned long long)kAptpMissCap) X.aptp_miss[i] = s;
      set_flag(X.counters, kFAptpMiss);
    }
    return;
  }
  factor_one_front<NT, SMEM>(P, X, s, prm, smem);
}

// ---------------------------------------------------------------------------
// Large fronts: one block per front steps the blocked pivoting (tpp_step_blk)
// while all blocks of the GPU run its deferred updates and, at the end, its
// Schur update, as tiled GEMMs whose every entry takes the same fused
// multiply-adds in the same pivot order as the block kernel.

__device__ __forceinline__ FrontRef large_view(DevPlan &P, DevFactor &X, int s) {
  FrontRef v;
  const int f = X.sn_f[s];
  v.F = X.arena + X.sn_off[s];
  v.ld = f;
  v.f = f;
  v.ne = X.sn_ne[s];
  v.rows = X.rows + X.sn_roff[s];
  v.tags = X.tags + X.sn_roff[s];
  v.W = v.F + (size_t)f * f;
  v.loc = X.ploc + X.sn_roff[s];
  v.inv = X.ploc + X.rows_cap + X.sn_roff[s];
  return v;
}

__global__ void k_large_init(DevPlan P, DevFactor X, const int *__restrict__ large, int nlarge,
                             int posdef, int nbo) {
  if (X.counters[kCFlags] & kFAbort) return;
  const int s = large[blockIdx.x];
  if (threadIdx.x == 0) {  // arrival counters of the front's team (both launch parities)
    X.team_bar[2 * blockIdx.x] = 0u;
    X.team_bar[2 * blockIdx.x + 1] = 0u;
  }
  const int f = X.sn_f[s];
  int *loc = X.ploc + X.sn_roff[s];
  int *inv = X.ploc + X.rows_cap + X.sn_roff[s];
  for (int t = threadIdx.x; t < f; t += blockDim.x) {
    loc[t] = t;
    inv[t] = t;
  }
  if (threadIdx.x == 0) {
    TppState S;
    const bool mixed = X.sn_mixed != nullptr && X.sn_mixed[s] != 0 && nbo > 0;
    tpp_init(S, X.sn_ne[s], posdef != 0, mixed, nbo);
    S.pad[0] = 0;  // deferred update pending
    X.tpp[blockIdx.x] = S;
  }
}

// The early stops of an indefinite factorization, after each level
// (multifrontal_serial.cpp:1619-1628, :660-671): the negative pivots and the
// front work (fully summed columns x rows^2, exact integers) of the fronts
// factored so far; past max_negative_pivots (neg_limit >= 0) or past the
// work cap (work_cap >= 0) the rest of the factorization is skipped. Both
// counts only grow, so a run that stops is exactly one whose finished count
// would have passed the limit.
__global__ void k_level_limits(DevPlan P, DevFactor X, int lo, int hi, long long neg_limit, long long work_cap) {
  __shared__ long long red[2][32];
  if (X.counters[kCFlags] & kFAbort) return;
  long long neg = 0, work = 0;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const int s = P.lvl_sn[i];
    const long long f = X.sn_f[s];
    neg += X.sn_stat[4 * s + 1];
    work += (long long)X.sn_ne[s] * f * f;
  }
  for (int o = 16; o > 0; o >>= 1) {
    neg += __shfl_xor_sync(0xffffffffu, neg, o);
    work += __shfl_xor_sync(0xffffffffu, work, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = neg;
    red[1][threadIdx.x >> 5] = work;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    neg = work = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      neg += red[0][w];
      work += red[1][w];
    }
    const long long tn = (long long)atomicAdd(X.counters + kCNegSoFar, (unsigned long long)neg) + neg;
    const long long tw = (long long)atomicAdd(X.counters + kCWorkSoFar, (unsigned long long)work) + work;
    if (neg_limit >= 0 && tn > neg_limit) set_flag(X.counters, kFInertia);
    if (work_cap >= 0 && tw > work_cap) set_flag(X.counters, kFWork);
  }
}

// Realized rows, eligible columns, arena and row offsets of a level's large
// fronts (read by the host to set up their APTP sweep).
__global__ void k_large_sizes(DevFactor X, const int *__restrict__ large, int nlarge, int64_t *__restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nlarge) return;
  const int s = large[q];
  out[4 * q] = X.sn_f[s];
  out[4 * q + 1] = X.sn_ne[s];
  out[4 * q + 2] = X.sn_off[s];
  out[4 * q + 3] = X.sn_roff[s];
}

// The threshold kernel's state of the APTP fronts after their sweep: it
// continues from the APTP pivots on the columns the sweep failed (blocked,
// or unblocked when fewer than blocked_min_front rows remain:
// multifrontal_serial.cpp:810-814, ldlt_kernel.cpp:977), its Schur update
// from those pivots on; the sweep's counts carried, and the position map
// (inv, the inverse of loc, which the sweep permuted) rebuilt. One block per
// front.
__global__ void k_aptp_to_tpp(const aptp::Front *__restrict__ fr, const aptp::State *__restrict__ st,
                              const int *__restrict__ qpos, int64_t rows_cap, TppState *__restrict__ tpp, int bmf) {
  const int i = blockIdx.x;
  const aptp::Front F = fr[i];
  int *inv = F.loc + rows_cap;
  for (int t = threadIdx.x; t < F.f; t += blockDim.x) inv[F.loc[t]] = t;
  if (threadIdx.x != 0) return;
  const aptp::State &A = st[i];
  TppState &T = tpp[qpos[i]];
  T.k = A.num_elim;
  T.live = F.ne;
  T.k_paired = -1;
  T.post = 0;
  T.st = A.st;
  T.pad[3] = A.num_elim;
  T.mixed = 0;
  T.se = 1 << 30;
  T.phase = (A.num_elim >= F.ne) ? 2 : (F.f - A.num_elim < bmf ? 3 : 0);
}

// One blocked-TPP step (tpp_step_blk) of each large front of a level; a
// front is taken by a team of C CTAs launched as one thread-block cluster
// (blockIdx.x / C = the front), the pivot decisions taken by every CTA of
// the team alike and the swaps and panel eliminations split over it.
template <int NT, int C>
__global__ void __launch_bounds__(NT) k_large_panel(DevPlan P, DevFactor X, const int *__restrict__ large,
                                                    PivotParams prm, int iter, unsigned *__restrict__ team_bar) {
  __shared__ FrontShared sh;
  __shared__ int s_abort;
  __shared__ unsigned s_bar_seq;
  __shared__ PairScratch s_pair;
  if (X.counters[kCFlags] & kFAbort) return;
  const int q = blockIdx.x / C;
  const bool lead = team_rank<C>() == 0 && threadIdx.x == 0;
  const int s = large[q];
  TppState S = X.tpp[q];
  if (S.phase == 2) {
    if (lead) X.tpp[q].pad[0] = 0;
    return;
  }
  prm.eff_small = __longlong_as_double((long long)X.counters[kCEffSmall]);
  FrontRef v = large_view(P, X, s);
  // arrival counters: one per launch parity; this launch resets the other
  // (the previous launch's, finished; the next launch's, not started)
  v.team_bar = team_bar + 2 * q + (iter & 1);
  if (lead) team_bar[2 * q + ((iter + 1) & 1)] = 0u;
  v.err = X.counters + kCFlags;
  v.abort = &s_abort;
  v.bar_seq = &s_bar_seq;
  v.pair = &s_pair;
  v.team_red = X.team_red + (size_t)q * kTeamRedDoubles;
  if (threadIdx.x == 0) {
    sh.st = S.st;
    sh.tr_seq = 0;
    s_abort = 0;
    s_bar_seq = 0;
  }
  __syncthreads();
  // every CTA has read the state before the leader may write it back
  if constexpr (C > 1) team_sync<C>(v);
  const bool more = tpp_step_blk<NT, C>(v, prm, sh, S);
  __syncthreads();
  if (lead) {
    S.st = sh.st;
    S.pad[0] = more ? 1 : 0;
    X.tpp[q] = S;
    if (more) {
      atomicMax(X.counters + kCActive, (unsigned long long)(iter + 1));
      // algorithmic flops of the deferred update asked for (2 per FMA)
      // and its bytes (each element read and written once)
      const long long m = S.g_e - S.g_c0, h = v.f - S.g_c0;
      if (m > 0 && S.g_p1 > S.g_p0) {
        const double elems = (double)(m * h - m * (m - 1) / 2);
        atomicAdd(reinterpret_cast<double *>(X.counters + kCGemmFlops), 2.0 * (double)(S.g_p1 - S.g_p0) * elems);
        atomicAdd(reinterpret_cast<double *>(X.counters + kCDeferBytes), 16.0 * elems);
        atomicAdd(X.counters + kCDeferUpd, 1ull);
        if (S.g_p1 - S.g_p0 <= 2) atomicAdd(X.counters + kCDeferSmall, 1ull);
      }
    }
  }
}

// Work items of a level's tiled GEMMs: each large front contributes tiles of
// kGT x kGT over a lower-trapezoidal region [r0, f) x [r0, c1) with tile
// (ti, tj) needed when ti >= tj.
constexpr int kGT = 64;

__device__ __forceinline__ int trap_tiles(int rows, int cols) {  // rows >= cols
  const int rt = (rows + kGT - 1) / kGT, ct = (cols + kGT - 1) / kGT;
  return ct * rt - ct * (ct - 1) / 2;
}

__device__ __forceinline__ void trap_tile(int w, int rows, int cols, int &ti, int &tj) {
  const int rt = (rows + kGT - 1) / kGT;
  tj = 0;
  while (w >= rt - tj) {
    w -= rt - tj;
    ++tj;
  }
  ti = tj + w;
}

// (L D)(j, c) of a front in global memory (fill_ld_column).
__device__ __forceinline__ double ld_entry_g(const double *F, size_t sf, const int8_t *tags, int c, int j) {
  const double *Lc = F + (size_t)c * sf;
  const int8_t tag = tags[c];
  if (tag == 1) return __dmul_rn(Lc[j], Lc[c]);
  if (tag == 2) return __dadd_rn(__dmul_rn(Lc[j], Lc[c]), __dmul_rn(Lc[sf + j], Lc[c + 1]));
  if (tag == -1) {
    const double *L0 = Lc - sf;
    return __dadd_rn(__dmul_rn(L0[j], L0[c]), __dmul_rn(Lc[j], Lc[c]));
  }
  return 0.0;
}

// One 128 x 64 tile of C -= A B^T (lower part: i >= j, i < rmax, j < cmax)
// over K = kk pivots in order: A(i, p) = F(i, a0 + p); B(j, p) = W(j, p)
// (deferred update) or (L D)(j, a0 + p) (Schur update). 256 threads, 8 x 4
// entries each, K in chunks of 16 staged in shared memory with the next
// chunk prefetched in registers. Every entry takes one fused multiply-add
// per pivot in pivot order, a zero B(j, p) skipped, as the reference's
// GEMM loops do.
constexpr int kTM = 128, kTN = 64, kTK = 16;

struct TileSmem {
  double A[2][kTK][kTM];
  double B[2][kTK][kTN];
};

template <bool SCHUR>
__device__ __forceinline__ void tile_update(double *F, size_t sf, const double *W, int wld, const int8_t *tags,
                                            int i0, int j0, int rmax, int cmax, int a0, int kk, TileSmem &sm) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double c[8][4];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = i0 + tx + 16 * r, j = j0 + ty + 16 * q;
      c[r][q] = (i < rmax && j < cmax && i >= j) ? F[(size_t)j * sf + i] : 0.0;
    }
  double pa[8], pb[4];
  int zb = 0;  // a zero among the fetched chunk's B values (a skipped update)
  auto fetch = [&](int k0) {
    zb = 0;
    const int kc = min(kTK, kk - k0);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = threadIdx.x + 256 * u;
      const int p = t / kTM, r = t % kTM;
      pa[u] = (p < kc && i0 + r < rmax) ? F[(size_t)(a0 + k0 + p) * sf + i0 + r] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = threadIdx.x + 256 * u;
      const int p = t / kTN, r = t % kTN;
      double bv = 0.0;
      if (p < kc && j0 + r < cmax) {
        if (SCHUR) bv = ld_entry_g(F, sf, tags, a0 + k0 + p, j0 + r);
        else bv = W[(size_t)(k0 + p) * wld + j0 + r];
        zb |= bv == 0.0 ? 1 : 0;
      }
      pb[u] = bv;
    }
  };
  auto stash = [&](int buf) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = threadIdx.x + 256 * u;
      sm.A[buf][t / kTM][t % kTM] = pa[u];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = threadIdx.x + 256 * u;
      sm.B[buf][t / kTN][t % kTN] = pb[u];
    }
  };
  int buf = 0;
  fetch(0);
  __syncthreads();
  stash(0);
  // whether the chunk in sm has a zero B value: without one every update
  // applies and the loop takes no tests (the padding's zeros only reach
  // entries that are not stored)
  int anyz = __syncthreads_or(zb);
  for (int k0 = 0; k0 < kk; k0 += kTK) {
    const int kc = min(kTK, kk - k0);
    if (k0 + kTK < kk) fetch(k0 + kTK);
    if (!anyz) {
      for (int p = 0; p < kc; ++p) {
        double av[8], bv[4];
#pragma unroll
        for (int r = 0; r < 8; ++r) av[r] = sm.A[buf][p][tx + 16 * r];
#pragma unroll
        for (int q = 0; q < 4; ++q) bv[q] = sm.B[buf][p][ty + 16 * q];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int r = 0; r < 8; ++r) c[r][q] = fma(-av[r], bv[q], c[r][q]);
      }
    } else {
      for (int p = 0; p < kc; ++p) {
        double av[8], bv[4];
#pragma unroll
        for (int r = 0; r < 8; ++r) av[r] = sm.A[buf][p][tx + 16 * r];
#pragma unroll
        for (int q = 0; q < 4; ++q) bv[q] = sm.B[buf][p][ty + 16 * q];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (bv[q] != 0.0) {
#pragma unroll
            for (int r = 0; r < 8; ++r) c[r][q] = fma(-av[r], bv[q], c[r][q]);
          }
        }
      }
    }
    if (k0 + kTK < kk) {
      stash(buf ^ 1);
      anyz = __syncthreads_or(zb);
      buf ^= 1;
    }
  }
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = i0 + tx + 16 * r, j = j0 + ty + 16 * q;
      if (i < rmax && j < cmax && i >= j) F[(size_t)j * sf + i] = c[r][q];
    }
  __syncthreads();
}

// Tiles of a lower-trapezoidal region rows [r0, f) x cols [r0, c1): tile
// (ti, tj) of kTM x kTN is needed when its last row reaches its first column.
__device__ __forceinline__ int trap_tiles2(int rows, int cols) {
  const int ct = (cols + kTN - 1) / kTN;
  int n = 0;
  for (int tj = 0; tj < ct; ++tj) {
    const int first_ti = (tj * kTN) / kTM;  // tile rows from where column tile tj starts
    n += (rows + kTM - 1) / kTM - first_ti;
  }
  return n;
}

__device__ __forceinline__ void trap_tile2(int w, int rows, int cols, int &ti, int &tj) {
  const int rt = (rows + kTM - 1) / kTM;
  tj = 0;
  while (true) {
    const int first = (tj * kTN) / kTM;
    const int cnt = rt - first;
    if (w < cnt) {
      ti = first + w;
      return;
    }
    w -= cnt;
    ++tj;
  }
}

// Deferred updates of all large fronts with one pending (ldlt_kernel.cpp:705-761).
__global__ void __launch_bounds__(256) k_large_gemm(DevPlan P, DevFactor X, const int *__restrict__ large,
                                                    int nlarge, const TppState *__restrict__ tpp) {
  extern __shared__ __align__(16) double dsm_g[];
  TileSmem &sm = *reinterpret_cast<TileSmem *>(dsm_g);
  __shared__ int pref[129];
  if (X.counters[kCFlags] & kFAbort) return;
  for (int chunk = 0; chunk < nlarge; chunk += 128) {
    const int cnt = min(128, nlarge - chunk);
    __syncthreads();
    if (threadIdx.x == 0) {
      pref[0] = 0;
      for (int q = 0; q < cnt; ++q) {
        const TppState &S = tpp[chunk + q];
        int nt = 0;
        if (S.pad[0] && S.g_p1 > S.g_p0 && S.g_e > S.g_c0)
          nt = trap_tiles2(X.sn_f[large[chunk + q]] - S.g_c0, S.g_e - S.g_c0);
        pref[q + 1] = pref[q] + nt;
      }
    }
    __syncthreads();
    const int total = pref[cnt];
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
      int a = 0, b = cnt;
      while (b - a > 1) {
        const int mid = (a + b) >> 1;
        if (pref[mid] <= w) a = mid;
        else b = mid;
      }
      const int q = chunk + a;
      const int s = large[q];
      const TppState S = tpp[q];
      const int f = X.sn_f[s];
      const size_t sf = (size_t)f;
      double *F = X.arena + X.sn_off[s];
      int ti, tj;
      trap_tile2(w - pref[a], f - S.g_c0, S.g_e - S.g_c0, ti, tj);
      tile_update<false>(F, sf, F + sf * sf, f, nullptr, S.g_c0 + ti * kTM, S.g_c0 + tj * kTN, f, S.g_e,
                         S.g_p0, S.g_p1 - S.g_p0, sm);
    }
  }
}

// ---------------------------------------------------------------------------
// Deferred updates, streamed (nb <= 16): the same update as k_large_gemm,
// F[c0:f, c0:e] -= L[c0:f, p0:p1] W[:, c0:e] on the lower trapezoid, each
// element by the same chain c = fma(-l_p, w_p, c) over p in order (w_p = 0
// skipped), so the results are bitwise those of k_large_gemm. With at most
// 16 pivots an element costs 2 K flops for 16 bytes of traffic: the update
// is bound by HBM, and the kernel is shaped for that: 64 x 64 tiles (every
// front of the launch in one list), 16 elements a thread, at most 64
// registers so that four blocks share an SM and their load, update and
// store phases overlap; the L and W slices of a tile are read once into
// shared memory. Measured on one 16,000-row front (K = 16): 4.6 TB/s,
// against 3.0 TB/s for the general tiled kernel.
constexpr int kDT = 64, kDK = 32, kDFronts = 256, kDBlocksPerSM = 4;

// Tiles of a lower trapezoid rows x cols (rows >= cols) in kDT squares:
// column tile tj holds the row tiles [tj, rt).
__device__ __forceinline__ int defer_tiles(int rows, int cols) {
  const int rt = (rows + kDT - 1) / kDT, ct = (cols + kDT - 1) / kDT;
  return ct * rt - ct * (ct - 1) / 2;
}

// Tile w of that order: the largest tj with S(tj) = tj rt - tj (tj - 1) / 2
// <= w (a root of the quadratic, then corrected by exact integer steps).
__device__ __forceinline__ void defer_tile(int w, int rows, int &ti, int &tj) {
  const long long rt = (rows + kDT - 1) / kDT;
  auto S = [&](long long x) { return x * rt - x * (x - 1) / 2; };
  const double b = 2.0 * (double)rt + 1.0;
  long long t = (long long)((b - sqrt(fmax(b * b - 8.0 * (double)w, 0.0))) * 0.5);
  if (t < 0) t = 0;
  while (t > 0 && S(t) > w) --t;
  while (S(t + 1) <= w) ++t;
  tj = (int)t;
  ti = (int)(t + (w - S(t)));
}

// mode: 0 the whole update, 1 only the next step's kDK columns [c0, c0 +
// kDK), 2 only the columns past them (look-ahead). At most kDK pivots; W
// buffer pad[1] (kDK rows each).
__global__ void __launch_bounds__(256, kDBlocksPerSM) k_large_defer(DevPlan P, DevFactor X,
                                                                    const int *__restrict__ large, int nlarge,
                                                                    const TppState *__restrict__ tpp, int mode) {
  __shared__ double Ls[kDK][kDT];  // [pivot][row of the tile]
  __shared__ double Ws[kDK][kDT];  // [pivot][column of the tile]
  __shared__ int pref[kDFronts + 1];
  __shared__ int m_f[kDFronts], m_c0[kDFronts], m_e[kDFronts], m_p0[kDFronts], m_kk[kDFronts];
  __shared__ long long m_off[kDFronts];
  __shared__ int m_wo[kDFronts];
  __shared__ int wsum[8];
  if (X.counters[kCFlags] & kFAbort) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tx = tid & 15, ty = tid >> 4;
  for (int chunk = 0; chunk < nlarge; chunk += kDFronts) {
    const int cnt = min(kDFronts, nlarge - chunk);
    __syncthreads();
    int nt = 0;
    if (tid < cnt) {
      const TppState &S = tpp[chunk + tid];
      const int s = large[chunk + tid];
      const int f = X.sn_f[s];
      // the columns of this launch's share of the update
      const int split = min(S.g_e, S.g_c0 + kDK);  // the next step's 32 columns
      const int cs = mode == 2 ? split : S.g_c0, ce = mode == 1 ? split : S.g_e;
      if (S.pad[0] && S.g_p1 > S.g_p0 && ce > cs) nt = defer_tiles(f - cs, ce - cs);
      m_f[tid] = f;
      m_c0[tid] = cs;
      m_e[tid] = ce;
      m_p0[tid] = S.g_p0;
      m_kk[tid] = S.g_p1 - S.g_p0;
      // (W of the panel: the second buffer for odd look-ahead panels)
      m_off[tid] = (long long)X.sn_off[s];
      m_wo[tid] = S.pad[1];
    }
    // inclusive block scan of the tile counts
    int v = nt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    if (lane == 31) wsum[warp] = v;
    __syncthreads();
    int base = 0;
    for (int w = 0; w < warp; ++w) base += wsum[w];
    if (tid < cnt) pref[tid + 1] = base + v;
    if (tid == 0) pref[0] = 0;
    __syncthreads();
    const int total = pref[cnt];
    // diagonal rows a two-panel SPD step staged in W: into F (block q of the
    // grid takes front q; the tiles below never touch these rows)
    if (mode != 2) {
      for (int q = blockIdx.x; q < cnt; q += gridDim.x) {
        const TppState &S = tpp[chunk + q];
        const int nd = S.pad[2];
        if (!S.pad[0] || nd <= 0) continue;
        const int s = large[chunk + q];
        const int f = X.sn_f[s];
        const size_t sf = (size_t)f;
        double *F = X.arena + X.sn_off[s];
        const double *Wd = F + sf * sf + (size_t)S.pad[1] * kDK * sf;
        for (int t = tid; t < nd * nd; t += 256) {
          const int c = t / nd, r = t % nd;
          if (r >= c) F[(size_t)(S.g_p0 + c) * sf + S.g_p0 + r] = Wd[(size_t)c * f + S.g_p0 + r];
        }
      }
    }
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
      int lo = 0, hi = cnt;
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pref[mid] <= w) lo = mid;
        else hi = mid;
      }
      const int a = lo;
      int ti, tj;
      defer_tile(w - pref[a], m_f[a] - m_c0[a], ti, tj);
      const int f = m_f[a], e = m_e[a], kk = m_kk[a], p0 = m_p0[a];
      const size_t sf = (size_t)f;
      double *F = X.arena + m_off[a];
      const double *Wp = F + sf * sf + (size_t)m_wo[a] * kDK * sf;  // second W buffer: kDK rows on
      const int i0 = m_c0[a] + ti * kDT, j0 = m_c0[a] + tj * kDT;
      double c[4][4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int i = i0 + tx + 16 * r, j = j0 + ty + 16 * q;
          c[r][q] = (i < f && j < e && i >= j) ? F[(size_t)j * sf + i] : 0.0;
        }
      int zw = 0;  // a zero among the tile's w (a skipped update)
#pragma unroll
      for (int u = 0; u < kDK * kDT / 256; ++u) {
        const int t = tid + 256 * u, p = t >> 6, r = t & 63;
        Ls[p][r] = (p < kk && i0 + r < f) ? F[(size_t)(p0 + p) * sf + i0 + r] : 0.0;
        const bool real = p < kk && j0 + r < e;
        const double wv = real ? Wp[(size_t)p * sf + j0 + r] : 0.0;
        Ws[p][r] = wv;
        zw |= (real && wv == 0.0) ? 1 : 0;
      }
      if (!__syncthreads_or(zw)) {
        // no zero w: every update applies (the padding's zeros only reach
        // entries that are not stored)
        for (int p = 0; p < kk; ++p) {
          double av[4], bv[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) av[r] = Ls[p][tx + 16 * r];
#pragma unroll
          for (int q = 0; q < 4; ++q) bv[q] = Ws[p][ty + 16 * q];
#pragma unroll
          for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int r = 0; r < 4; ++r) c[r][q] = fma(-av[r], bv[q], c[r][q]);
        }
      } else {
        for (int p = 0; p < kk; ++p) {
          double av[4], bv[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) av[r] = Ls[p][tx + 16 * r];
#pragma unroll
          for (int q = 0; q < 4; ++q) bv[q] = Ws[p][ty + 16 * q];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            if (bv[q] != 0.0) {
#pragma unroll
              for (int r = 0; r < 4; ++r) c[r][q] = fma(-av[r], bv[q], c[r][q]);
            }
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int i = i0 + tx + 16 * r, j = j0 + ty + 16 * q;
          if (i < f && j < e && i >= j) F[(size_t)j * sf + i] = c[r][q];
        }
      __syncthreads();  // Ls / Ws are refilled by the next tile
    }
  }
}

// Schur updates of all large fronts of a level (schur_update,
// ldlt_kernel.cpp:820-933): F[e:f, e:f] -= L LD^T over pivots [0, k).
__global__ void __launch_bounds__(256) k_large_schur(DevPlan P, DevFactor X, const int *__restrict__ large,
                                                     int nlarge, const TppState *__restrict__ tpp) {
  extern __shared__ __align__(16) double dsm_g[];
  TileSmem &sm = *reinterpret_cast<TileSmem *>(dsm_g);
  __shared__ int pref[129];
  if (X.counters[kCFlags] & kFAbort) return;
  for (int chunk = 0; chunk < nlarge; chunk += 128) {
    const int cnt = min(128, nlarge - chunk);
    __syncthreads();
    if (threadIdx.x == 0) {
      pref[0] = 0;
      for (int q = 0; q < cnt; ++q) {
        const int s = large[chunk + q];
        // pivots [pad[3], k): an APTP front's trailing update covered its own
        const int e = X.sn_ne[s], f = X.sn_f[s], k = tpp[chunk + q].k, k0 = tpp[chunk + q].pad[3];
        // mixed fronts: the tensor-core updates covered the contribution block
        const bool fp64 = !tpp[chunk + q].mixed;
        pref[q + 1] = pref[q] + ((f > e && k > k0 && fp64) ? trap_tiles2(f - e, f - e) : 0);
      }
    }
    __syncthreads();
    const int total = pref[cnt];
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
      int a = 0, b = cnt;
      while (b - a > 1) {
        const int mid = (a + b) >> 1;
        if (pref[mid] <= w) a = mid;
        else b = mid;
      }
      const int q = chunk + a;
      const int s = large[q];
      const int f = X.sn_f[s], e = X.sn_ne[s], k0 = tpp[q].pad[3], kk = tpp[q].k - k0;
      const size_t sf = (size_t)f;
      double *F = X.arena + X.sn_off[s];
      int ti, tj;
      trap_tile2(w - pref[a], f - e, f - e, ti, tj);
      tile_update<true>(F, sf, nullptr, 0, X.tags + X.sn_roff[s], e + ti * kTM, e + tj * kTN, f, f, k0, kk, sm);
    }
  }
}

// Bookkeeping of a factored large front (one block): zero pivots at a root,
// status flags, 2x2 off-diagonals moved to their upper slots, counts, and
// the children's row maps in pivot order. The column-parallel part of the
// store (the SPD sqrt(D) fold, zeroing) is k_large_store.
template <int NT>
__global__ void __launch_bounds__(NT) k_large_finish(DevPlan P, DevFactor X, const int *__restrict__ large,
                                                     const TppState *__restrict__ tpp, PivotParams prm) {
  if (X.counters[kCFlags] & kFAbort) return;
  const int s = large[blockIdx.x];
  const TppState S = tpp[blockIdx.x];
  const FrontRef v = large_view(P, X, s);
  const int f = v.f, ne = v.ne, p = S.k;
  const size_t sf = (size_t)f;
  if (threadIdx.x == 0 && !S.mixed) {
    const double q = (double)(f - ne);
    if (q > 0 && p > S.pad[3])
      atomicAdd(reinterpret_cast<double *>(X.counters + kCGemmFlops), 2.0 * (p - S.pad[3]) * (q * (q + 1) / 2));
  }
  const bool is_root = P.sn_parent[s] < 0;
  int pstore = p;
  if (is_root && p < ne) {
    for (int c = p + threadIdx.x; c < ne; c += NT) v.tags[c] = 0;
    pstore = ne;
  }
  __syncthreads();
  if (prm.posdef) {
    if (p < ne && threadIdx.x == 0) set_flag(X.counters, kFNotPosdef);
  } else {
    bool bad = false;
    for (int c = threadIdx.x; c < pstore; c += NT) {
      double *Lc = v.F + (size_t)c * sf;
      const int8_t tag = v.tags[c];
      if (tag == 1) bad = bad || !isfinite(Lc[c]);
      else if (tag == 2) bad = bad || !isfinite(Lc[c]) || !isfinite(Lc[c + 1]) || !isfinite(Lc[sf + c + 1]);
      else if (tag == -1) Lc[c - 1] = v.F[(size_t)(c - 1) * sf + c];
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) set_flag(X.counters, kFNonfiniteD);
  }
  int *inv = X.ploc + X.rows_cap + X.sn_roff[s];
  for (int t = threadIdx.x; t < f; t += NT) inv[v.loc[t]] = t;
  __syncthreads();
  for (int t = P.child_ptr[s]; t < P.child_ptr[s + 1]; ++t) {
    const int c = P.child_idx[t];
    const int pc = X.sn_p[c];
    int *cmap = X.cbmap + X.sn_roff[c] + pc;
    for (int u = threadIdx.x; u < X.sn_f[c] - pc; u += NT) cmap[u] = inv[cmap[u]];
  }
  if (threadIdx.x == 0) {
    X.sn_p[s] = p;
    X.sn_pstore[s] = pstore;
    X.sn_dout[s] = is_root ? 0 : ne - p;
    int *st = X.sn_stat + 4 * s;
    st[0] = S.st.pos;
    st[1] = S.st.neg;
    st[2] = S.st.zero + (is_root ? ne - p : 0);
    st[3] = S.st.two_by_two;
    X.sn_flops[s] = S.st.flops;
  }
}

// Column-parallel store of the large fronts' pivot columns
// (multifrontal_serial.cpp:903-945): SPD L = L_unit sqrt(D) with the upper
// part zero; indefinite D inline (zero pivots' columns zero, the 2x2
// blocks' lower off-diagonal slot zero, the upper part zero but for the
// slot k_large_finish filled). Work items: 32 columns of one front.
__global__ void __launch_bounds__(256) k_large_store(DevPlan P, DevFactor X, const int *__restrict__ large,
                                                     int nlarge, int posdef) {
  __shared__ int pref[65];
  __shared__ double sdv[32];
  if (X.counters[kCFlags] & kFAbort) return;
  for (int chunk = 0; chunk < nlarge; chunk += 64) {
    const int cnt = min(64, nlarge - chunk);
    if (threadIdx.x == 0) {
      pref[0] = 0;
      for (int q = 0; q < cnt; ++q) pref[q + 1] = pref[q] + (X.sn_pstore[large[chunk + q]] + 31) / 32;
    }
    __syncthreads();
    const int total = pref[cnt];
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
      int a = 0, b = cnt;
      while (b - a > 1) {
        const int mid = (a + b) >> 1;
        if (pref[mid] <= w) a = mid;
        else b = mid;
      }
      const int s = large[chunk + a];
      const int f = X.sn_f[s], pstore = X.sn_pstore[s];
      const size_t sf = (size_t)f;
      double *F = X.arena + X.sn_off[s];
      const int8_t *tags = X.tags + X.sn_roff[s];
      const int c0 = (w - pref[a]) * 32, c1 = min(c0 + 32, pstore);
      if (posdef) {
        if (threadIdx.x < c1 - c0) sdv[threadIdx.x] = sqrt(F[(size_t)(c0 + threadIdx.x) * sf + c0 + threadIdx.x]);
        __syncthreads();
        // the item's columns as one run of (column, row) pairs (columns are
        // contiguous, leading dimension f), eight entries a thread in flight
        double *base = F + (size_t)c0 * sf;
        const int64_t n = (int64_t)(c1 - c0) * f;
        for (int64_t t0 = threadIdx.x; t0 < n; t0 += 8 * 256) {
          double y[8];
          int cc[8], ii[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int64_t t = t0 + 256 * u;
            cc[u] = c0 + (int)(t / f);
            ii[u] = (int)(t % f);
            y[u] = (t < n && ii[u] > cc[u]) ? base[t] : 0.0;  // the strictly lower part is read
          }
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int64_t t = t0 + 256 * u;
            if (t >= n) continue;
            if (ii[u] < cc[u]) base[t] = 0.0;
            else if (ii[u] > cc[u]) base[t] = __dmul_rn(y[u], sdv[cc[u] - c0]);
          }
        }
        __syncthreads();
        if (threadIdx.x < c1 - c0) F[(size_t)(c0 + threadIdx.x) * sf + c0 + threadIdx.x] = sdv[threadIdx.x];
      } else {
        for (int c = c0; c < c1; ++c) {
          double *Lc = F + (size_t)c * sf;
          const int8_t tag = tags[c];
          for (int i = threadIdx.x; i < f; i += 256) {
            if (tag == 0) Lc[i] = 0.0;
            else if (i < c) {
              if (!(tag == -1 && i == c - 1)) Lc[i] = 0.0;
            } else if (tag == 2 && i == c + 1) {
              Lc[i] = 0.0;
            }
          }
        }
      }
      __syncthreads();
    }
    __syncthreads();
  }
}

// Two SPD panels per launch (32 pivots, then one rank-32 deferred update:
// half the launches and half the deferred traffic of one panel at a time).
// Per entry the operations and their order are the one-panel path's: the
// second panel's columns take the first panel's update as the deferred
// update would (c = fma(-l_p, w_p, c) over its pivots in order, w_p = 0
// skipped) before the second panel's eliminations, and the columns past
// both take one chain over the 32 pivots in order. Every block factors both
// diagonal blocks itself: the first, then the first panel's pivots on the
// second panel's 16 rows (their unscaled values w and multipliers l to
// shared memory), the second block updated from them and factored. A
// failing pivot in the first panel ends the front there (as the one-panel
// path ends it).
template <int NB>
__global__ void __launch_bounds__(256) k_large_panel_spd2(DevPlan P, DevFactor X, const int *__restrict__ large,
                                                          const TppState *__restrict__ cur,
                                                          TppState *__restrict__ nxt, int iter, int w2) {
  __shared__ double T[NB][NB + 1], T2[NB][NB + 1];
  __shared__ double lm[NB][NB], lm2[NB][NB];
  __shared__ double linv[NB], linv2[NB];
  __shared__ double Wr[NB][NB], Lr[NB][NB];  // [row of panel 2][pivot of panel 1]
  __shared__ int np2_sh, zero_sh;
  if (X.counters[kCFlags] & kFAbort) return;
  const int q = blockIdx.y;
  const int s = large[q];
  const TppState S = cur[q];
  const bool lead = blockIdx.x == 0;
  if (S.phase == 2) {
    if (lead && threadIdx.x == 0) {
      TppState o = S;
      o.pad[0] = 0;
      nxt[q] = o;
    }
    return;
  }
  const int f = X.sn_f[s], ne = X.sn_ne[s];
  const int ps = S.k, pl = min(ne, ps + NB), nbp = pl - ps;
  const int ps2 = pl, pl2 = min(ne, ps2 + NB), nbp2 = pl2 - ps2;
  const int r0 = ps + blockIdx.x * 256;
  if (r0 >= f) return;
  const size_t sf = (size_t)f;
  double *F = X.arena + X.sn_off[s];
  // W: rows [0, 16) panel 1, [16, 32) panel 2; w2 (look-ahead): two such
  // buffers alternating by step
  const int wpar = w2 ? (iter & 1) : 0;
  double *W = F + sf * sf + (size_t)wpar * 2 * NB * sf;
  const double eff_small = __longlong_as_double((long long)X.counters[kCEffSmall]);
  // Every load of F this thread needs is issued here, so that their
  // latency overlaps the two diagonal factors: none of these entries is
  // written in this launch before it is read (the panels' diagonal rows are
  // staged in W, and each row below belongs to one thread, which writes
  // panel 1's columns only after reading panel 2's).
  const int i = r0 + threadIdx.x;
  static_assert(NB * NB == 256, "one entry of T and T2 per thread");
  const int tr = threadIdx.x / NB, tc = threadIdx.x % NB;
  const double t1v = (tr < nbp && tc <= tr) ? F[(size_t)(ps + tc) * sf + ps + tr] : 0.0;
  const double t2v = (tr < nbp2 && tc <= tr) ? F[(size_t)(ps2 + tc) * sf + ps2 + tr] : 0.0;
  double ra[NB], rb[NB], wa[NB];
#pragma unroll
  for (int c = 0; c < NB; ++c) {
    ra[c] = (i < f && c < nbp && ps + c <= i) ? F[(size_t)(ps + c) * sf + i] : 0.0;
    rb[c] = (i < f && c < nbp2 && ps2 + c <= i) ? F[(size_t)(ps2 + c) * sf + i] : 0.0;
    wa[c] = (threadIdx.x < nbp2 && nbp == NB) ? F[(size_t)(ps + c) * sf + ps2 + threadIdx.x] : 0.0;
  }
  // panel 1's diagonal block
  T[tr][tc] = t1v;
  if (threadIdx.x == 0) zero_sh = 0;
  const int np1 = spd_diag_factor<NB>(T, lm, linv, nbp, &zero_sh);
  const bool two = np1 == NB && nbp == NB && nbp2 > 0;
  if (two) {
    // panel 1's pivots on panel 2's rows (threads 0..15: one row each)
    if (threadIdx.x < nbp2) {
      double a[NB];
#pragma unroll
      for (int c = 0; c < NB; ++c) a[c] = wa[c];
      bool zw = false;
#pragma unroll
      for (int k = 0; k < NB; ++k) {
        const double w = a[k];
        Wr[threadIdx.x][k] = w;
        zw = zw || w == 0.0;
#pragma unroll
        for (int j = k + 1; j < NB; ++j) {
          const double l = lm[k][j];
          const double u = __dsub_rn(a[j], __dmul_rn(w, l));
          a[j] = l != 0.0 ? u : a[j];
        }
        a[k] = __dmul_rn(w, linv[k]);
        Lr[threadIdx.x][k] = a[k];
      }
      if (zw) zero_sh = 1;
    }
    // panel 2's diagonal block, panel 1's update applied as the deferred
    // update applies it
    __syncthreads();
    if (tr < nbp2 && tc <= tr) {
      double v = t2v;
#pragma unroll
      for (int p = 0; p < NB; ++p) {
        const double bw = Wr[tc][p];
        const double u = fma(-Lr[tr][p], bw, v);
        v = bw != 0.0 ? u : v;
      }
      T2[tr][tc] = v;
    } else {
      T2[tr][tc] = 0.0;
    }
    const int n2 = spd_diag_factor<NB>(T2, lm2, linv2, nbp2, &zero_sh);
    if (threadIdx.x == 0) np2_sh = n2;
  }
  __syncthreads();
  const int np2 = two ? np2_sh : 0;
  // warps whose rows all lie past the panels' diagonal blocks, with every
  // pivot taken and no zero multiplier or w: each entry takes every update
  // (no tests), the same operations in the same order
  const bool fast = zero_sh == 0 && nbp == NB && np1 == NB && (!two || (nbp2 == NB && np2 == NB)) &&
                    r0 + (int)(threadIdx.x & ~31u) >= (two ? pl2 : pl);
  if (fast && i < f) {
    double a[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) a[c] = ra[c];
#pragma unroll
    for (int k = 0; k < NB; ++k) {
      const double w = a[k];
      W[(size_t)k * f + i] = w;
#pragma unroll
      for (int j = k + 1; j < NB; ++j) a[j] = __dsub_rn(a[j], __dmul_rn(w, lm[k][j]));
      a[k] = __dmul_rn(w, linv[k]);
    }
#pragma unroll
    for (int c = 0; c < NB; ++c) F[(size_t)(ps + c) * sf + i] = a[c];
    if (two) {
      double b[NB];
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        double v = rb[c];
#pragma unroll
        for (int p = 0; p < NB; ++p) v = fma(-a[p], Wr[c][p], v);
        b[c] = v;
      }
#pragma unroll
      for (int k = 0; k < NB; ++k) {
        const double w = b[k];
        W[(size_t)(NB + k) * f + i] = w;
#pragma unroll
        for (int j = k + 1; j < NB; ++j) b[j] = __dsub_rn(b[j], __dmul_rn(w, lm2[k][j]));
        b[k] = __dmul_rn(w, linv2[k]);
      }
#pragma unroll
      for (int c = 0; c < NB; ++c) F[(size_t)(ps2 + c) * sf + i] = b[c];
    }
  } else if (r0 == ps && i < (two ? pl2 : pl)) {
    // the panels' diagonal rows (block 0's first rows): the diagonal
    // factors computed their final values by the same operations -- the
    // multipliers (lm, Lr, lm2) for the pivots taken, the rest of T and T2
    // (unscaled, their pivots' updates applied) -- so they are staged from
    // shared memory
    const int r = i - ps;
    if (r < NB) {
#pragma unroll
      for (int c = 0; c < NB; ++c)
        if (c < nbp && c <= r) W[(size_t)c * f + i] = (c < r && c < np1) ? lm[c][r] : T[r][c];
    } else {
      const int r2 = r - NB;
#pragma unroll
      for (int c = 0; c < NB; ++c) W[(size_t)c * f + i] = Lr[r2][c];
#pragma unroll
      for (int c = 0; c < NB; ++c)
        if (c < nbp2 && c <= r2) W[(size_t)(NB + c) * f + i] = (c < r2 && c < np2) ? lm2[c][r2] : T2[r2][c];
    }
  } else if (i < f) {
    double a[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) a[c] = ra[c];
#pragma unroll
    for (int k = 0; k < NB; ++k) {
      // (selects, not branches: the multipliers' loads issue ahead of the
      // chain; an entry skipped keeps its value exactly)
      const bool take = k < np1 && i > ps + k;
      const double w = a[k];
      if (take) W[(size_t)k * f + i] = w;
#pragma unroll
      for (int j = k + 1; j < NB; ++j) {
        const double l = lm[k][j];
        const double u = __dsub_rn(a[j], __dmul_rn(w, l));
        a[j] = (take && j < nbp && ps + j <= i && l != 0.0) ? u : a[j];
      }
      const double sk = __dmul_rn(w, linv[k]);
      a[k] = take ? sk : a[k];
    }
    // rows of the panels' diagonal blocks go to W (columns [ps, pend) at
    // W rows c): other blocks read their original values in this launch;
    // the deferred-update launch copies them into F
    const bool stage = i < (two ? pl2 : pl);
#pragma unroll
    for (int c = 0; c < NB; ++c)
      if (c < nbp && ps + c <= i) {
        if (stage) W[(size_t)c * f + i] = a[c];
        else F[(size_t)(ps + c) * sf + i] = a[c];
      }
    if (two && i >= ps2) {
      // the second panel's columns of this row: panel 1's update, then
      // panel 2's pivots
      double b[NB];
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        b[c] = 0.0;
        if (c < nbp2 && ps2 + c <= i) {
          double v = rb[c];
#pragma unroll
          for (int p = 0; p < NB; ++p) {
            const double bw = Wr[c][p];
            const double u = fma(-a[p], bw, v);
            v = bw != 0.0 ? u : v;
          }
          b[c] = v;
        }
      }
#pragma unroll
      for (int k = 0; k < NB; ++k) {
        const bool take = k < np2 && i > ps2 + k;
        const double w = b[k];
        if (take) W[(size_t)(NB + k) * f + i] = w;
#pragma unroll
        for (int j = k + 1; j < NB; ++j) {
          const double l = lm2[k][j];
          const double u = __dsub_rn(b[j], __dmul_rn(w, l));
          b[j] = (take && j < nbp2 && ps2 + j <= i && l != 0.0) ? u : b[j];
        }
        const double sk = __dmul_rn(w, linv2[k]);
        b[k] = take ? sk : b[k];
      }
#pragma unroll
      for (int c = 0; c < NB; ++c)
        if (c < nbp2 && ps2 + c <= i) {
          if (stage) W[(size_t)(NB + c) * f + i] = b[c];
          else F[(size_t)(ps2 + c) * sf + i] = b[c];
        }
    }
  }
  if (lead && threadIdx.x < 32) {
    // the pivots' tags, inertia and flops, a lane each (lanes 0..15 panel
    // 1, 16..31 panel 2): the counts by ballot, the flop terms (integers,
    // exact in a double, as is every partial sum of a front's) summed by
    // shuffles -- the same totals as a pivot-by-pivot loop
    const int lane = threadIdx.x;
    const bool p1 = lane < np1, p2 = lane >= NB && lane - NB < np2;
    double dv = 0.0, term = 0.0;
    if (p1 || p2) {
      const int col = p1 ? ps + lane : ps2 + lane - NB;
      X.tags[X.sn_roff[s] + col] = 1;
      dv = p1 ? T[lane][lane] : T2[lane - NB][lane - NB];
      const double rem = (double)(f - (col + 1));
      term = rem + rem * (rem + 1.0);
    }
    const bool zr = (p1 || p2) && (!isfinite(dv) || fabs(dv) < eff_small);
    const bool po = (p1 || p2) && !zr && dv > 0.0;
    const bool ng = (p1 || p2) && !zr && !(dv > 0.0);
    const int nzr = __popc(__ballot_sync(0xffffffffu, zr)), npo = __popc(__ballot_sync(0xffffffffu, po)),
              nng = __popc(__ballot_sync(0xffffffffu, ng));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) term += __shfl_xor_sync(0xffffffffu, term, o);
    if (lane != 0) return;
    TppState o = S;
    o.st.zero += nzr;
    o.st.pos += npo;
    o.st.neg += nng;
    o.st.flops += term;
    const int np = np1 + np2;
    const int pend = two ? pl2 : pl;  // the deferred update starts past the panels done
    o.k = ps + np;
    o.g_p0 = ps;
    o.g_p1 = ps + np;
    o.g_c0 = pend;
    o.g_e = tpp_upd_end(S, ne);
    o.pad[0] = np > 0 ? 1 : 0;
    o.pad[1] = wpar;       // the W buffer of this step's update
    o.pad[2] = pend - ps;  // diagonal rows [ps, pend) staged in W (copied by k_large_defer)
    if (np1 < nbp || (two && np2 < nbp2) || o.k >= ne) o.phase = 2;
    nxt[q] = o;
    if (np > 0) {
      atomicMax(X.counters + kCActive, (unsigned long long)(iter + 1));
      const long long m = tpp_upd_end(S, ne) - pend, h = f - pend;
      if (m > 0) {
        const double elems = (double)(m * h - m * (m - 1) / 2);
        atomicAdd(reinterpret_cast<double *>(X.counters + kCGemmFlops), 2.0 * (double)np * elems);
        atomicAdd(reinterpret_cast<double *>(X.counters + kCDeferBytes), 16.0 * elems);
        atomicAdd(X.counters + kCDeferUpd, 1ull);
        if (np <= 2) atomicAdd(X.counters + kCDeferSmall, 1ull);
      }
    }
  }
}

// Tensor-core updates due on a level's mixed large fronts (one thread): a
// front whose outer block is used up (k reached min(se, ne)), that asked
// for a flush, or that finished with pivots pending gets a job applying
// the pivots [tc_done, k) to its columns from min(se, ne) on (the rows and
// columns no deferred update of the block touched); its next outer block
// then starts at k. Jobs, work-item and tile prefixes go to X.tc_*.
__global__ void k_tc_jobs(DevPlan P, DevFactor X, const int *__restrict__ large, int nlarge,
                          TppState *__restrict__ tpp, int nbo, int posdef, int ke) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  tc::Job *jobs = reinterpret_cast<tc::Job *>(X.tc_jobs);
  int nj = 0, tiles = 0;
  int64_t off = 0, items = 0;
  double flops = 0.0;
  X.tc_ipref[0] = 0;
  X.tc_tpref[0] = 0;
  const bool dead = (X.counters[kCFlags] & kFAbort) != 0;
  for (int q = 0; q < nlarge && !dead; ++q) {
    TppState &S = tpp[q];
    if (!S.mixed) continue;
    const int s = large[q];
    const int f = X.sn_f[s], ne = X.sn_ne[s], k = S.k;
    const int sep = min(S.se, ne);
    const bool cb_only = S.se >= ne;  // the contribution block only (indefinite fronts)
    const bool due = cb_only ? (k - S.tc_done >= nbo) : (k >= sep);
    if (S.tc_done < k && (S.flush || due || S.phase == 2)) {
      const int n = f - sep, kc = k - S.tc_done;
      if (n > 0) {
        double *F = X.arena + X.sn_off[s];
        tc::Job J;
        J.C = F;
        J.Ls = F + (int64_t)S.tc_done * f;
        J.Ws = nullptr;
        J.tags = posdef ? nullptr : X.tags + X.sn_roff[s];
        J.ld = J.ldl = J.ldw = f;
        J.r0 = J.lr0 = J.wr0 = sep;
        J.n = n;
        J.k0 = S.tc_done;
        J.kc = kc;
        J.ntr = (n + tc::kBM - 1) / tc::kBM;
        J.nkb = (kc + ke - 1) / ke;
        J.tiles = J.ntr * (J.ntr + 1) / 2;
        J.img = off;
        off += tc::image_bytes(J.ntr, J.nkb);
        items += (int64_t)J.ntr * tc::kBM * 8 * J.nkb;
        tiles += J.tiles;
        jobs[nj++] = J;
        X.tc_ipref[nj] = items;
        X.tc_tpref[nj] = tiles;
        flops += 2.0 * kc * ((double)n * (n + 1) / 2);
      }
      S.tc_done = k;
      if (!cb_only) S.se = k + nbo;
    }
    S.flush = 0;
  }
  if (off > X.tc_img_cap) {
    set_flag(X.counters, kFTcCap);
    nj = 0;
  }
  *X.tc_njobs = nj;
  if (flops > 0.0) atomicAdd(reinterpret_cast<double *>(X.counters + kCTcFlops), flops);
}

// Graph replays run a fixed number of pivoting steps per level: a front
// still asking for an update at the last one did not finish (the host then
// factors without the graph).
__global__ void k_steps_check(unsigned long long *cnt, int steps) {
  if (threadIdx.x == 0 && cnt[kCActive] >= (unsigned long long)steps) set_flag(cnt, kFSteps);
}

// Totals over all fronts, in supernode order (deterministic).
struct FactorTotals {
  long long pos, neg, zero, two_by_two, delayed, entries;
  int max_front, pad;
  double flops;
};

__global__ void k_finish(DevPlan P, DevFactor X, FactorTotals *out) {
  __shared__ long long acc[6][32];
  __shared__ int mf[32];
  __shared__ double fl[32];
  long long a[6] = {0, 0, 0, 0, 0, 0};
  int mx = 0;
  double fsum = 0.0;
  for (int s = threadIdx.x; s < P.nsn; s += blockDim.x) {
    const int *st = X.sn_stat + 4 * s;
    a[0] += st[0];
    a[1] += st[1];
    a[2] += st[2];
    a[3] += st[3];
    a[4] += X.sn_dout[s];
    a[5] += (long long)X.sn_f[s] * X.sn_pstore[s];
    mx = max(mx, X.sn_f[s]);
    fsum += X.sn_flops[s];  // integer-valued: exact in any order
  }
  for (int o = 16; o > 0; o >>= 1) {
    for (int q = 0; q < 6; ++q) a[q] += __shfl_xor_sync(0xffffffffu, a[q], o);
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    fsum += __shfl_xor_sync(0xffffffffu, fsum, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    for (int q = 0; q < 6; ++q) acc[q][w] = a[q];
    mf[w] = mx;
    fl[w] = fsum;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    FactorTotals t{};
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      t.pos += acc[0][i];
      t.neg += acc[1][i];
      t.zero += acc[2][i];
      t.two_by_two += acc[3][i];
      t.delayed += acc[4][i];
      t.entries += acc[5][i];
      t.max_front = max(t.max_front, mf[i]);
      t.flops += fl[i];
    }
    *out = t;
  }
}

// ---------------------------------------------------------------------------
// Solves. x (new numbering, n x nrhs) and per-front work vectors w at the
// fronts' row offsets (rows_total x nrhs).
//
// The solve kernels are launched with programmatic stream serialization: a
// kernel may start while the one before it on the stream still runs. Before
// pdl_wait() it reads only what no solve kernel writes (the factor, its row
// maps and sizes), so that its loads of L overlap the kernel before it;
// pdl_wait() returns once that kernel has completed and its writes are
// visible (at once when the launch had no such dependency), and
// pdl_trigger() lets the next kernel start its own prologue.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__global__ void k_solve_gather(const double *__restrict__ b, int ldb, int nrhs, int n,
                               const int *__restrict__ perm, const double *__restrict__ scale,
                               double *__restrict__ x) {
  pdl_wait();
  pdl_trigger();
  const int64_t tot = (int64_t)n * nrhs;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(t / n), i = (int)(t % n);
    const int o = perm[i];
    double v = b[(int64_t)r * ldb + o];
    if (scale) v = __dmul_rn(v, scale[o]);
    x[t] = v;
  }
}

__global__ void k_solve_scatter(double *__restrict__ b, int ldb, int nrhs, int n,
                                const int *__restrict__ perm, const double *__restrict__ scale,
                                const double *__restrict__ x) {
  pdl_wait();
  pdl_trigger();
  const int64_t tot = (int64_t)n * nrhs;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(t / n), i = (int)(t % n);
    const int o = perm[i];
    double v = x[t];
    if (scale) v = __dmul_rn(v, scale[o]);
    b[(int64_t)r * ldb + o] = v;
  }
}

// Solves by level. Each front's work vector w (length f, at the front's row
// offset) holds its pivot rows' values and, in the forward sweep, its update
// vector for the parent (rows p..f); x (new numbering) holds the pivot
// results. Large fronts (symbolic rows >= kLargeMin) leave their L21 part
// to the multi-block kernels k_fwd_l21 / k_bwd_l21. Sums run in a fixed
// order (deterministic); solve_forward.cpp:116-293 and
// solve_backward.cpp:135-350 compute the same quantities.
constexpr int kSolveNT = 128;

// The 32 x 32 lower block L[jb:jb+nb, jb:jb+nb) staged in shared memory
// (coalesced column reads) for the warp triangle solves below.
template <int NT>
__device__ __forceinline__ void load_tri32(const double *L, size_t sf, int jb, int nb, double (*Ls)[33]) {
  __syncthreads();
  for (int t = threadIdx.x; t < 1024; t += NT) {
    const int r = t & 31, c = t >> 5;
    Ls[r][c] = (r < nb && c < nb && c <= r) ? L[(size_t)(jb + c) * sf + jb + r] : 0.0;
  }
  __syncthreads();
}

// The same triangle copied asynchronously (8-byte cp.async, zero fill
// outside the lower triangle); the caller waits with cp_async_wait_all()
// and a barrier before reading Ls.
template <int NT>
__device__ __forceinline__ void load_tri32_async(const double *L, size_t sf, int jb, int nb, double (*Ls)[33]) {
  for (int t = threadIdx.x; t < 1024; t += NT) {
    const int r = t & 31, c = t >> 5;
    const bool in = r < nb && c < nb && c <= r;
    const double *src = in ? L + (size_t)(jb + c) * sf + jb + r : L;
    const unsigned dst = (unsigned)__cvta_generic_to_shared(&Ls[r][c]);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(in ? 8 : 0) : "memory");
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// w[jb:jb+nb) <- L11^-1 w (unit, or non-unit for SPD): lane = row.
// (the lane's row of the triangle in registers and the SPD diagonal's
// reciprocal taken ahead: a step of the chain is a shuffle and an fma)
__device__ __forceinline__ void tri_fwd_warp(double *w, int jb, int nb, int posdef, const double (*Ls)[33]) {
  const int lane = threadIdx.x & 31;
  double lrow[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) lrow[j] = (j < lane && lane < nb) ? Ls[lane][j] : 0.0;
  const double rdiag = (posdef && lane < nb) ? 1.0 / Ls[lane][lane] : 1.0;
  double wi = (lane < nb) ? w[jb + lane] : 0.0;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    if (j < nb) {
      // (selects: no divergent branch in the chain; the values as the
      // branches would leave them)
      const double sc = wi * rdiag;
      wi = lane == j ? sc : wi;
      const double wj = __shfl_sync(0xffffffffu, wi, j);
      const double u = fma(-lrow[j], wj, wi);
      wi = lrow[j] != 0.0 ? u : wi;
    }
  }
  if (lane < nb) w[jb + lane] = wi;
}

// v[jb:jb+nb) <- L11^-T v: lane = row.
__device__ __forceinline__ void tri_bwd_warp(double *v, int jb, int nb, int posdef, const double (*Ls)[33]) {
  const int lane = threadIdx.x & 31;
  double lcol[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) lcol[j] = (j > lane && j < nb) ? Ls[j][lane] : 0.0;
  const double rdiag = (posdef && lane < nb) ? 1.0 / Ls[lane][lane] : 1.0;
  double vi = (lane < nb) ? v[jb + lane] : 0.0;
#pragma unroll
  for (int j = 31; j >= 0; --j) {
    if (j < nb) {
      const double sc = vi * rdiag;
      vi = lane == j ? sc : vi;
      const double xj = __shfl_sync(0xffffffffu, vi, j);
      const double u = fma(-lcol[j], xj, vi);
      vi = lcol[j] != 0.0 ? u : vi;
    }
  }
  if (lane < nb) v[jb + lane] = vi;
}

// Fronts of at most this many rows take the warp-per-front solve kernels.
constexpr int kSolveSmall = 64;

// D^-1 of the 2x2 pivot [d00 d10; d10 d11] applied to (r0, r1) by the scaled
// Cramer rule (solve_diag.cpp:49-123); zero for a singular block.
__device__ __forceinline__ void dinv2_apply(double d00, double d10, double d11, double r0, double r1, double &z0,
                                            double &z1) {
  const double s2 = max3_ref(fabs(d00), fabs(d10), fabs(d11));
  z0 = 0.0;
  z1 = 0.0;
  if (isfinite(s2) && s2 != 0.0) {
    const double a = d00 / s2, bb = d10 / s2, cc = d11 / s2;
    const double det = __dsub_rn(__dmul_rn(a, cc), __dmul_rn(bb, bb));
    if (isfinite(det) && det != 0.0) {
      if (!isfinite(r0) || !isfinite(r1)) {
        z0 = r0;
        z1 = r1;
      } else {
        const double rs = fmax(fabs(r0), fabs(r1));
        if (rs != 0.0) {
          const double q0 = r0 / rs, q1 = r1 / rs;
          const double u0 = __dsub_rn(__dmul_rn(cc, q0), __dmul_rn(bb, q1)) / det;
          const double u1 = __dadd_rn(__dmul_rn(-bb, q0), __dmul_rn(a, q1)) / det;
          const double ratio = rs / s2;
          z0 = __dmul_rn(u0, ratio);
          z1 = __dmul_rn(u1, ratio);
        }
      }
    }
  }
}

// Forward sweep of the level's fronts of at most kSolveSmall rows, a warp
// per front (no block barriers; eight fronts a block): gather, the
// children's update vectors in child order, then column by column over the
// whole front (the unit, or SPD non-unit, L11 solve and w[p:f) -= L21
// w[0:p) in one pass), the front's L columns loaded eight at a time ahead
// of their use.
__global__ void __launch_bounds__(256, 4) k_fwd_small(DevPlan P, DevFactor X, int lo, int m, int posdef, double *x,
                                                   double *wk, int64_t rows_total, int nrhs) {
  __shared__ double sw_all[8][kSolveSmall];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int item = blockIdx.x * 8 + wid;
  if (item >= m) return;
  const int s = P.lvl_sn[lo + item];
  const int f = X.sn_f[s];
  if (f > kSolveSmall || P.sn_large[s]) return;
  pdl_wait();
  pdl_trigger();
  const int p = X.sn_pstore[s];
  const int64_t roff = X.sn_roff[s];
  const int *rows = X.rows + roff;
  const double *L = X.arena + X.sn_off[s];
  double *sw = sw_all[wid];
  for (int r = 0; r < nrhs; ++r) {
    double *w = wk + (int64_t)r * rows_total + roff;
    double *xr = x + (int64_t)r * P.n;
    for (int i = lane; i < f; i += 32) sw[i] = (i < p) ? xr[rows[i]] : 0.0;
    __syncwarp();
    for (int t = P.child_ptr[s]; t < P.child_ptr[s + 1]; ++t) {
      const int c = P.child_idx[t];
      const int pc = X.sn_pstore[c], q = X.sn_f[c] - pc;
      const int *cmap = X.cbmap + X.sn_roff[c] + pc;
      const double *wc = wk + (int64_t)r * rows_total + X.sn_roff[c] + pc;
      for (int i = lane; i < q; i += 32) sw[cmap[i]] += wc[i];
      __syncwarp();
    }
    // rows lane and lane + 32
    double w0 = (lane < f) ? sw[lane] : 0.0, w1 = (lane + 32 < f) ? sw[lane + 32] : 0.0;
    for (int j0 = 0; j0 < p; j0 += 8) {
      double l0[8], l1[8], dj[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int j = j0 + u;
        const bool in = j < p;
        l0[u] = (in && lane > j && lane < f) ? __ldg(L + (size_t)j * f + lane) : 0.0;
        l1[u] = (in && lane + 32 < f) ? __ldg(L + (size_t)j * f + lane + 32) : 0.0;
        dj[u] = (in && posdef) ? __ldg(L + (size_t)j * f + j) : 1.0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int j = j0 + u;
        if (j >= p) break;
        // w_j of the row's owner lane
        double wj = __shfl_sync(0xffffffffu, j < 32 ? w0 : w1, j & 31);
        if (posdef) wj = wj / dj[u];
        if (lane == j) w0 = wj;
        if (lane + 32 == j) w1 = wj;
        if (l0[u] != 0.0) w0 = fma(-l0[u], wj, w0);
        if (l1[u] != 0.0 && lane + 32 > j) w1 = fma(-l1[u], wj, w1);
      }
    }
    if (lane < f) w[lane] = w0;
    if (lane + 32 < f) w[lane + 32] = w1;
    if (lane < p) xr[rows[lane]] = w0;
    if (lane + 32 < p) xr[rows[lane + 32]] = w1;
    __syncwarp();
  }
}

// Backward sweep of the level's fronts of at most kSolveSmall rows, a warp
// per front: D^-1 of every pivot block (2x2 blocks where the upper slot (c,
// c+1) is nonzero), v -= L21^T x_ext, then L11^-T from the last column on
// (each column's dot with the solved part a warp reduction).
__global__ void __launch_bounds__(256, 4) k_bwd_small(DevPlan P, DevFactor X, int lo, int m, int posdef, double *x,
                                                   int nrhs, int apply_d, int apply_lt) {
  __shared__ double sv_all[8][kSolveSmall];
  __shared__ double sx_all[8][kSolveSmall];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int item = blockIdx.x * 8 + wid;
  if (item >= m) return;
  const int s = P.lvl_sn[lo + item];
  const int f = X.sn_f[s];
  if (f > kSolveSmall || P.sn_large[s]) return;
  pdl_wait();
  pdl_trigger();
  const int p = X.sn_pstore[s];
  const int *rows = X.rows + X.sn_roff[s];
  const double *L = X.arena + X.sn_off[s];
  const size_t sf = (size_t)f;
  double *sv = sv_all[wid], *sx = sx_all[wid];
  for (int r = 0; r < nrhs; ++r) {
    double *xr = x + (int64_t)r * P.n;
    for (int i = lane; i < f; i += 32) sx[i] = (i >= p) ? xr[rows[i]] : 0.0;
    for (int c = lane; c < p; c += 32) {
      const bool second = apply_d && !posdef && c > 0 && L[(size_t)c * sf + c - 1] != 0.0;
      if (second) continue;
      double y0 = xr[rows[c]];
      if (!posdef && apply_d) {
        const double d00 = L[(size_t)c * sf + c];
        const double d10 = (c + 1 < p) ? L[(size_t)(c + 1) * sf + c] : 0.0;
        if (d10 != 0.0) {
          double z0, z1;
          dinv2_apply(d00, d10, L[(size_t)(c + 1) * sf + c + 1], y0, xr[rows[c + 1]], z0, z1);
          sv[c] = z0;
          sv[c + 1] = z1;
          continue;
        }
        y0 = (d00 == 0.0 || !isfinite(d00)) ? 0.0 : y0 / d00;
      }
      sv[c] = y0;
    }
    __syncwarp();
    if (apply_lt) {
      // v[c] -= L(p:f, c)^T x_ext: a lane per column
      for (int c = lane; c < p; c += 32) {
        const double *Lc = L + (size_t)c * sf;
        double acc = 0.0;
        for (int i = p; i < f; ++i) acc = fma(Lc[i], sx[i], acc);
        sv[c] -= acc;
      }
      __syncwarp();
      // L11^-T, last column first: x_j = (v_j - L(j+1:p, j)^T x) / L_jj
      for (int j = p - 1; j >= 0; --j) {
        const double *Lj = L + (size_t)j * sf;
        double acc = 0.0;
        for (int i = j + 1 + lane; i < p; i += 32) acc = fma(Lj[i], sx[i], acc);
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
          double xj = sv[j] - acc;
          if (posdef) xj = xj / Lj[j];
          sx[j] = xj;
        }
        __syncwarp();
      }
    } else {
      for (int c = lane; c < p; c += 32) sx[c] = sv[c];
      __syncwarp();
    }
    for (int c = lane; c < p; c += 32) xr[rows[c]] = sx[c];
    __syncwarp();
  }
}

// Forward sweep of one level: gather, children's update vectors in child
// order, blocked unit (indefinite) or non-unit (SPD) L11 solve, then
// w[p:f) -= L21 w[0:p) unless the front is large. Fronts of at most
// kSolveSmall rows are k_fwd_small's.
__global__ void __launch_bounds__(kSolveNT, 4) k_fwd_front(DevPlan P, DevFactor X, int lo, int posdef,
                                                        double *x, double *wk, int64_t rows_total,
                                                        int nrhs) {
  const int s = P.lvl_sn[lo + blockIdx.x];
  const int f = X.sn_f[s], p = X.sn_pstore[s];
  const int64_t roff = X.sn_roff[s];
  const int *rows = X.rows + roff;
  const double *L = X.arena + X.sn_off[s];
  const size_t sf = (size_t)f;
  const bool large = P.sn_large[s] != 0;
  if (!large && f <= kSolveSmall) return;  // k_fwd_small's
  pdl_wait();
  pdl_trigger();
  __shared__ double Ls[32][33];
  const int warp = threadIdx.x >> 5;
  // every right-hand side at once: gather, children's update vectors in
  // child order, then per 32-column strip the triangle (a warp per
  // right-hand side) and the rows below (each L entry loaded once for all)
  // (four rows a thread in flight: a large front's gather and children's
  // vectors are thousands of rows for one block)
  for (int r = 0; r < nrhs; ++r) {
    double *w = wk + (int64_t)r * rows_total + roff;
    const double *xr = x + (int64_t)r * P.n;
    for (int i0 = threadIdx.x; i0 < f; i0 += 4 * kSolveNT) {
      double v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = i0 + u * kSolveNT;
        v[u] = (i < p) ? xr[rows[i]] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (i0 + u * kSolveNT < f) w[i0 + u * kSolveNT] = v[u];
    }
  }
  __syncthreads();
  for (int t = P.child_ptr[s]; t < P.child_ptr[s + 1]; ++t) {
    const int c = P.child_idx[t];
    const int pc = X.sn_pstore[c], q = X.sn_f[c] - pc;
    const int *cmap = X.cbmap + X.sn_roff[c] + pc;
    for (int r = 0; r < nrhs; ++r) {
      double *w = wk + (int64_t)r * rows_total + roff;
      const double *wc = wk + (int64_t)r * rows_total + X.sn_roff[c] + pc;
      for (int i0 = threadIdx.x; i0 < q; i0 += 4 * kSolveNT) {
        double v[4], o[4];
        int m[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int i = i0 + u * kSolveNT;
          m[u] = (i < q) ? cmap[i] : 0;
          v[u] = (i < q) ? wc[i] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) o[u] = (i0 + u * kSolveNT < q) ? w[m[u]] : 0.0;
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (i0 + u * kSolveNT < q) w[m[u]] = o[u] + v[u];
      }
    }
    __syncthreads();
  }
  if (large) return;  // the block kernels (k_fwd_tri / k_fwd_gemv) go on
  for (int jb = 0; jb < p; jb += 32) {
    const int nb = min(32, p - jb);
    // the strip's triangle and this thread's first row below it loaded
    // before the barriers and the triangle solves (in flight meanwhile)
    double tv[1024 / kSolveNT];
#pragma unroll
    for (int u = 0; u < 1024 / kSolveNT; ++u) {
      const int t = (int)threadIdx.x + kSolveNT * u, r = t & 31, c = t >> 5;
      tv[u] = (r < nb && c < nb && c <= r) ? __ldg(L + (size_t)(jb + c) * sf + jb + r) : 0.0;
    }
    const int i1 = jb + nb + (int)threadIdx.x;
    double l[32];
#pragma unroll
    for (int u = 0; u < 32; ++u) l[u] = (i1 < f && u < nb) ? __ldg(L + (size_t)(jb + u) * sf + i1) : 0.0;
    __syncthreads();  // the previous strip's readers of Ls and the vectors are done
#pragma unroll
    for (int u = 0; u < 1024 / kSolveNT; ++u) {
      const int t = (int)threadIdx.x + kSolveNT * u;
      Ls[t & 31][t >> 5] = tv[u];
    }
    __syncthreads();
    for (int r = warp; r < nrhs; r += kSolveNT / 32) tri_fwd_warp(wk + (int64_t)r * rows_total + roff, jb, nb, posdef, Ls);
    __syncthreads();
    for (int i = i1; i < f; i += kSolveNT) {
      if (i != i1) {
        const double *li = L + (size_t)jb * sf + i;
#pragma unroll
        for (int u = 0; u < 32; ++u) l[u] = (u < nb) ? __ldg(li + (size_t)u * sf) : 0.0;
      }
      for (int r = 0; r < nrhs; ++r) {
        double *w = wk + (int64_t)r * rows_total + roff;
        double acc = 0.0;
#pragma unroll
        for (int u = 0; u < 32; ++u)
          if (u < nb) acc = fma(l[u], w[jb + u], acc);
        w[i] -= acc;
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < p * nrhs; t += kSolveNT) {
    const int r = nrhs == 1 ? 0 : t / p, i = nrhs == 1 ? t : t - r * p;
    x[(int64_t)r * P.n + rows[i]] = wk[(int64_t)r * rows_total + roff + i];
  }
}

// w[p:f) -= L21 w[0:p) of the level's large fronts, rows split over blocks.
__global__ void __launch_bounds__(256) k_fwd_l21(DevPlan P, DevFactor X, const int *__restrict__ large,
                                                 int nlarge, double *wk, int64_t rows_total, int nrhs) {
  __shared__ double ws[256];
  __shared__ int pref[65];
  for (int chunk = 0; chunk < nlarge; chunk += 64) {
    const int cnt = min(64, nlarge - chunk);
    if (threadIdx.x == 0) {
      pref[0] = 0;
      for (int q = 0; q < cnt; ++q) {
        const int s = large[chunk + q];
        pref[q + 1] = pref[q] + (X.sn_f[s] - X.sn_pstore[s] + 255) / 256 * nrhs;
      }
    }
    __syncthreads();
    const int total = pref[cnt];
    for (int wi = blockIdx.x; wi < total; wi += gridDim.x) {
      int a = 0, b = cnt;
      while (b - a > 1) {
        const int mid = (a + b) >> 1;
        if (pref[mid] <= wi) a = mid;
        else b = mid;
      }
      const int s = large[chunk + a];
      const int f = X.sn_f[s], p = X.sn_pstore[s];
      const int nchunks = (f - p + 255) / 256;
      const int item = wi - pref[a];
      const int r = item / nchunks, rc = item % nchunks;
      double *w = wk + (int64_t)r * rows_total + X.sn_roff[s];
      const double *L = X.arena + X.sn_off[s];
      const size_t sf = (size_t)f;
      const int i = p + rc * 256 + threadIdx.x;
      double acc = (i < f) ? w[i] : 0.0;
      for (int j0 = 0; j0 < p; j0 += 256) {
        const int nj = min(256, p - j0);
        __syncthreads();
        if (threadIdx.x < nj) ws[threadIdx.x] = w[j0 + threadIdx.x];
        __syncthreads();
        if (i < f)
          for (int j = 0; j < nj; ++j) acc = fma(-L[(size_t)(j0 + j) * sf + i], ws[j], acc);
      }
      if (i < f) w[i] = acc;
      __syncthreads();
    }
    __syncthreads();
  }
}

// t[0:p) = L21^T x_ext of the level's large fronts, stored at the front's
// work vector positions [0, p): a work item is kL21Cols columns of one
// front for one right-hand side. x_ext is gathered into shared memory a
// tile of rows at a time, once for all the item's columns; a warp takes
// kL21Cols / 8 columns, lane = row. Each column's sum runs over its rows as
// a warp per column would take them (lane l: rows p + l + 32m in turn),
// then a shuffle tree.
constexpr int kL21Cols = 16, kL21Tile = 1024;
__global__ void __launch_bounds__(256) k_bwd_l21(DevPlan P, DevFactor X, const int *__restrict__ large,
                                                 int nlarge, const double *x, double *wk,
                                                 int64_t rows_total, int nrhs) {
  constexpr int CW = kL21Cols / 8;  // columns a warp
  __shared__ int pref[65];
  __shared__ double xs[kL21Tile];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  pdl_wait();
  pdl_trigger();
  for (int chunk = 0; chunk < nlarge; chunk += 64) {
    const int cnt = min(64, nlarge - chunk);
    __syncthreads();
    if (threadIdx.x == 0) {
      pref[0] = 0;
      for (int q = 0; q < cnt; ++q) {
        const int s = large[chunk + q];
        pref[q + 1] = pref[q] + (X.sn_pstore[s] + kL21Cols - 1) / kL21Cols * nrhs;
      }
    }
    __syncthreads();
    const int total = pref[cnt];
    for (int wi = blockIdx.x; wi < total; wi += gridDim.x) {
      int a = 0, b = cnt;
      while (b - a > 1) {
        const int mid = (a + b) >> 1;
        if (pref[mid] <= wi) a = mid;
        else b = mid;
      }
      const int s = large[chunk + a];
      const int f = X.sn_f[s], p = X.sn_pstore[s];
      const int ncc = (p + kL21Cols - 1) / kL21Cols;
      const int item = wi - pref[a];
      const int r = item / ncc, cc = item % ncc;
      const int jw = cc * kL21Cols + warp * CW;
      const int *rows = X.rows + X.sn_roff[s] + p;
      const double *L = X.arena + X.sn_off[s] + p;
      const double *xr = x + (int64_t)r * P.n;
      double acc[CW];
#pragma unroll
      for (int c = 0; c < CW; ++c) acc[c] = 0.0;
      for (int t0 = 0; t0 < f - p; t0 += kL21Tile) {
        const int tn = min(kL21Tile, f - p - t0);
        __syncthreads();  // the tile before read
        for (int i = threadIdx.x; i < tn; i += 256) xs[i] = xr[rows[t0 + i]];
        __syncthreads();
        for (int i = lane; i < tn; i += 32) {
          const double xv = xs[i];
#pragma unroll
          for (int c = 0; c < CW; ++c)
            if (jw + c < p) acc[c] = fma(L[(size_t)(jw + c) * f + t0 + i], xv, acc[c]);
        }
      }
#pragma unroll
      for (int c = 0; c < CW; ++c) {
        double v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0 && jw + c < p) wk[(int64_t)r * rows_total + X.sn_roff[s] + jw + c] = v;
      }
    }
  }
}

// Backward sweep of one level: v = D^-1 w_piv (indefinite, apply_inline_d
// with solve_2x2_scaled's scaled Cramer rule, solve_backward.cpp:135-171,
// pivoting.cpp:30-62), v -= L21^T x_ext (here for small fronts, from
// k_bwd_l21 for large ones), then the blocked L11^-T solve.
__global__ void __launch_bounds__(kSolveNT) k_bwd_front(DevPlan P, DevFactor X, int lo, int posdef,
                                                        double *x, double *wk, int64_t rows_total,
                                                        int nrhs, int apply_d, int apply_lt) {
  const int s = P.lvl_sn[lo + blockIdx.x];
  const int f = X.sn_f[s], p = X.sn_pstore[s];
  const int64_t roff = X.sn_roff[s];
  const int *rows = X.rows + roff;
  const double *L = X.arena + X.sn_off[s];
  const size_t sf = (size_t)f;
  const bool large = P.sn_large[s] != 0;
  if (!large && f <= kSolveSmall) return;  // k_bwd_small's
  pdl_wait();
  pdl_trigger();
  __shared__ double Ls[32][33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // every right-hand side at once. D^-1 of each pivot block; 2x2 blocks
  // start where the upper slot (c, c+1) is nonzero. (large: v[0:p) holds
  // L21^T x_ext)
  for (int t = threadIdx.x; t < p * nrhs; t += kSolveNT) {
    const int r = nrhs == 1 ? 0 : t / p, c = nrhs == 1 ? t : t - r * p;
    double *v = wk + (int64_t)r * rows_total + roff;
    const double *xr = x + (int64_t)r * P.n;
    const bool second = apply_d && !posdef && (c > 0) && L[(size_t)c * sf + c - 1] != 0.0;
    if (second) continue;
    double y0 = xr[rows[c]];
    if (!posdef && apply_d) {
      const double d00 = L[(size_t)c * sf + c];
      const double d10 = (c + 1 < p) ? L[(size_t)(c + 1) * sf + c] : 0.0;
      if (d10 != 0.0) {
        const double d11 = L[(size_t)(c + 1) * sf + c + 1];
        const double r0 = y0, r1 = xr[rows[c + 1]];
        const double s2 = max3_ref(fabs(d00), fabs(d10), fabs(d11));
        double z0 = 0.0, z1 = 0.0;
        if (isfinite(s2) && s2 != 0.0) {
          const double a = d00 / s2, bb = d10 / s2, cc = d11 / s2;
          const double det = __dsub_rn(__dmul_rn(a, cc), __dmul_rn(bb, bb));
          if (isfinite(det) && det != 0.0) {
            if (!isfinite(r0) || !isfinite(r1)) {
              z0 = r0;
              z1 = r1;
            } else {
              const double rs = fmax(fabs(r0), fabs(r1));
              if (rs != 0.0) {
                const double q0 = r0 / rs, q1 = r1 / rs;
                const double u0 = __dsub_rn(__dmul_rn(cc, q0), __dmul_rn(bb, q1)) / det;
                const double u1 = __dadd_rn(__dmul_rn(-bb, q0), __dmul_rn(a, q1)) / det;
                const double ratio = rs / s2;
                z0 = __dmul_rn(u0, ratio);
                z1 = __dmul_rn(u1, ratio);
              }
            }
          }
        }
        if (apply_lt && large) {
          z0 -= v[c];
          z1 -= v[c + 1];
        }
        v[c] = z0;
        v[c + 1] = z1;
        continue;
      }
      y0 = (d00 == 0.0 || !isfinite(d00)) ? 0.0 : y0 / d00;
    }
    if (apply_lt && large) y0 -= v[c];
    v[c] = y0;
  }
  __syncthreads();
  if (!apply_lt) {
    for (int t = threadIdx.x; t < p * nrhs; t += kSolveNT) {
      const int r = nrhs == 1 ? 0 : t / p, i = nrhs == 1 ? t : t - r * p;
      x[(int64_t)r * P.n + rows[i]] = wk[(int64_t)r * rows_total + roff + i];
    }
    return;
  }
  if (large) return;  // the block kernels (k_bwd_dots / k_bwd_tri) go on
  // v -= L21^T x_ext: a warp per column, its lanes' rows loaded once for
  // every right-hand side
  for (int j = warp; j < p; j += kSolveNT / 32) {
    const double *Lj = L + (size_t)j * sf;
    for (int i0 = p; i0 < f; i0 += 32 * 4) {
      double l[4];
      int ri[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = i0 + lane + 32 * u;
        l[u] = (i < f) ? __ldg(Lj + i) : 0.0;
        ri[u] = (i < f) ? rows[i] : -1;
      }
      for (int r = 0; r < nrhs; ++r) {
        const double *xr = x + (int64_t)r * P.n;
        double acc = 0.0;
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (ri[u] >= 0) acc = fma(l[u], xr[ri[u]], acc);
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) wk[(int64_t)r * rows_total + roff + j] -= acc;
      }
    }
  }
  __syncthreads();
  // blocked L11^-T: blocks from the end; dots with the solved part, then
  // the 32 x 32 triangle (a warp per right-hand side)
  for (int je = p; je > 0; je -= 32) {
    const int jb = max(0, je - 32), nb = je - jb;
    // the strip's triangle copied to Ls first, in flight during the dots
    // (the previous strip's solves, the last readers of Ls, ended at a barrier)
    load_tri32_async<kSolveNT>(L, sf, jb, nb, Ls);
    for (int j = jb + warp; j < je; j += kSolveNT / 32) {
      const double *Lj = L + (size_t)j * sf;
      for (int i0 = je; i0 < p; i0 += 32 * 4) {
        double l[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int i = i0 + lane + 32 * u;
          l[u] = (i < p) ? __ldg(Lj + i) : 0.0;
        }
        for (int r = 0; r < nrhs; ++r) {
          double *v = wk + (int64_t)r * rows_total + roff;
          double acc = 0.0;
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int i = i0 + lane + 32 * u;
            if (i < p) acc = fma(l[u], v[i], acc);
          }
          for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
          if (lane == 0) v[j] -= acc;
        }
      }
    }
    cp_async_wait_all();
    __syncthreads();
    for (int r = warp; r < nrhs; r += kSolveNT / 32) tri_bwd_warp(wk + (int64_t)r * rows_total + roff, jb, nb, posdef, Ls);
    __syncthreads();
  }
  for (int t = threadIdx.x; t < p * nrhs; t += kSolveNT) {
    const int r = nrhs == 1 ? 0 : t / p, i = nrhs == 1 ? t : t - r * p;
    x[(int64_t)r * P.n + rows[i]] = wk[(int64_t)r * rows_total + roff + i];
  }
}

// Large fronts' L11 solves in blocks of kSB columns: one block of threads
// per front solves the block's triangle (32-column steps), then all blocks
// of the GPU update the rows below it (forward) or the dot products of the
// next block's columns with the solved rows (backward). The loops are
// latency-bound (each front's block waits for the one before it), so every
// thread keeps its loads of L in flight together: a warp takes 32 rows of
// one 32-column strip (32 loads a lane), and partial sums over strips or
// row ranges meet in shared memory in a fixed order (deterministic).
constexpr int kSB = 256;
constexpr int kTriNT = 256;  // threads of the triangle kernels

// The 256-column blocks' strips of L staged in shared memory: strip k (32
// columns, the block's rows from the strip's first on) at
// buf[k % kRing][column][row - j0], copied with cp.async ahead of its use.
// Rows are padded to kSBP doubles, so that lanes reading one row across a
// strip's 32 columns hit distinct banks.
constexpr int kSBP = kSB + 1;
constexpr int kRing = 3;
struct TriSmem {
  double buf[kRing][32][kSBP];
  double w[8][kSB];  // the block's values, per right-hand side (at most 8)
};

// Inverses of the SPD large fronts' 32 x 32 diagonal blocks of L (after
// the store: L = L_unit sqrt(D)), for the triangle solves: a warp per
// block, lane c forms column c of the inverse by forward substitution
// (x_c = 1 / l_cc, x_i = -(sum_{c <= k < i} l_ik x_k) / l_ii, the sum in k
// order), the result written column-major through shared memory.
constexpr int kInvWarps = 8;
constexpr int kInvSmem = kInvWarps * 32 * 33 * (int)sizeof(double);
__global__ void __launch_bounds__(32 * kInvWarps) k_tri_invert(DevFactor X) {
  extern __shared__ __align__(16) unsigned char inv_smem[];
  double(*S)[33] = reinterpret_cast<double(*)[33]>(inv_smem) + (threadIdx.x >> 5) * 32;
  if (X.counters[kCFlags] & kFAbort) return;
  const int lane = threadIdx.x & 31;
  const int item = blockIdx.x * kInvWarps + (threadIdx.x >> 5);
  if (item >= X.inv_nitems) return;
  const int s = X.inv_items[2 * item], blk = X.inv_items[2 * item + 1];
  const int f = X.sn_f[s], p = X.sn_pstore[s];
  const int jb = 32 * blk, nb = min(32, p - jb);
  double *out = X.tri_inv + X.sn_ioff[s] + (int64_t)blk * 1024;
  const double *L = X.arena + X.sn_off[s];
  // S[i][k] = l_ik (rows of the block, lower part)
  for (int k = 0; k < 32; ++k) S[lane][k] = (k < nb && lane < nb && lane >= k) ? L[(size_t)(jb + k) * f + jb + lane] : 0.0;
  __syncwarp();
  double x[32];
  const int c = lane;
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < i; ++k) acc = fma(S[i][k], x[k], acc);
    const double rd = (i < nb) ? 1.0 / S[i][i] : 0.0;
    x[i] = (i < nb && c < nb && i >= c) ? ((i == c) ? rd : -acc * rd) : 0.0;
  }
  __syncwarp();
#pragma unroll
  for (int i = 0; i < 32; ++i) S[c][i] = x[i];  // S[c][i] = (L^-1)_ic
  __syncwarp();
  for (int k = 0; k < 32; ++k) out[k * 32 + lane] = S[k][lane];
}

// Strip [jb, jb + nb) of the block [j0, j1) (its rows [jb, j1)) into dst by
// threads [t0, t0 + nt): a warp per column (coalesced rows), one cp.async
// group.
__device__ __forceinline__ void tri_strip_async(const double *L, size_t sf, int j0, int j1, int jb, int nb,
                                                double (*dst)[kSBP], int t0 = 0, int nt = kTriNT,
                                                const double *inv = nullptr) {
  const int rows = j1 - jb;
  const int lane = threadIdx.x & 31;
  for (int u = ((int)threadIdx.x - t0) >> 5; u < nb; u += nt / 32) {
    const double *src = L + (size_t)(jb + u) * sf + jb;
    const unsigned d = (unsigned)__cvta_generic_to_shared(&dst[u][jb - j0]);
    for (int rr = lane; rr < rows; rr += 32) {
      // the diagonal block's rows from its inverse (inv: the front's
      // blocks; jb is a multiple of 32), when there is one
      const double *sp = (inv && rr < 32) ? inv + (size_t)(jb >> 5) * 1024 + (size_t)u * 32 + rr : src + rr;
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d + 8u * (unsigned)rr), "l"(sp) : "memory");
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// Columns [c0, c1) of the block ending at j1 (each from its strip's first
// row: the strips start at multiples of 32) into L2, 128-byte lines, with
// their strips' inverse blocks when there are any: the strips past the
// first kRing are copied to shared memory later, from L2 then.
__device__ __forceinline__ void tri_prefetch_l2(const double *L, size_t sf, int j1, int c0, int c1,
                                                const double *inv) {
  constexpr int kLines = 17;  // 128-byte lines a column of at most 256 rows can touch
  for (int e = threadIdx.x; e < (c1 - c0) * kLines; e += blockDim.x) {
    const int c = c0 + e / kLines, q = e % kLines, jb = c & ~31;
    if (jb + 16 * q < j1) asm volatile("prefetch.global.L2 [%0];" ::"l"(L + (size_t)c * sf + jb + 16 * q));
  }
  if (inv) {
    const int b0 = c0 >> 5, b1 = (c1 + 31) >> 5;
    for (int e = threadIdx.x; e < (b1 - b0) * 64; e += blockDim.x)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(inv + (size_t)(b0 + e / 64) * 1024 + 16 * (e % 64)));
  }
}

// wait until at most `pending` (0..2) of this thread's cp.async groups are in flight
__device__ __forceinline__ void cp_async_wait_pending(int pending) {
  if (pending >= 2) asm volatile("cp.async.wait_group 2;" ::: "memory");
  else if (pending == 1) asm volatile("cp.async.wait_group 1;" ::: "memory");
  else asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// All threads of a subset of whole warps (n of them, from warp-aligned
// threads) meet at barrier `id` (1..15; 0 is __syncthreads).
__device__ __forceinline__ void warps_sync(int id, int n) {
  __syncwarp();
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// Strips of a forward block: strip k covers [j0 + 32k, ...).
__device__ __forceinline__ void fwd_strip(int j0, int j1, int k, int &jb, int &nb) {
  jb = j0 + 32 * k;
  nb = min(32, j1 - jb);
}
// Strips of a backward block, numbered from the last.
__device__ __forceinline__ void bwd_strip(int j0, int j1, int k, int &jb, int &nb) {
  const int nstrip = (j1 - j0 + 31) / 32;
  jb = j0 + 32 * (nstrip - 1 - k);
  nb = min(32, j1 - jb);
}

// Block [j0, j1) of a large front: its first kRing strips of L issued to
// shared memory (all threads; one cp.async group each).
__device__ __forceinline__ void fwd_block_issue(const double *L, size_t sf, int j0, int j1, TriSmem &sm,
                                                const double *inv) {
  const int nstrip = (j1 - j0 + 31) / 32;
  for (int k = 0; k < min(kRing, nstrip); ++k) {
    int jb, nb;
    fwd_strip(j0, j1, k, jb, nb);
    tri_strip_async(L, sf, j0, j1, jb, nb, sm.buf[k], 0, kTriNT, inv);
  }
}
__device__ __forceinline__ void bwd_block_issue(const double *L, size_t sf, int j0, int j1, TriSmem &sm,
                                                const double *inv) {
  const int nstrip = (j1 - j0 + 31) / 32;
  for (int k = 0; k < min(kRing, nstrip); ++k) {
    int jb, nb;
    bwd_strip(j0, j1, k, jb, nb);
    tri_strip_async(L, sf, j0, j1, jb, nb, sm.buf[k], 0, kTriNT, inv);
  }
}

// The forward 32 x 32 triangle of strip [jb, jb + nb) for one right-hand
// side (a warp; lane = row jb + lane), `pre` (the product of the strip
// before, from the look-ahead) subtracted first: w[jb + lane] <- its solved
// value, also returned. The row of the triangle is in registers and the SPD
// diagonal's reciprocal taken ahead, so a step of the chain is one shuffle
// and one fused multiply-add.
__device__ __forceinline__ double fwd_chain32(const double (*Lb)[kSBP], int j0, int jb, int nb, int posdef,
                                              double *w, double pre, bool use_inv) {
  const int lane = threadIdx.x & 31;
  if (use_inv) {
    // the strip's diagonal block holds its inverse: x = L_bb^-1 (w - pre),
    // lane i's row of the inverse against the lanes' values (four partial
    // sums, no dependent chain across the lanes)
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    const double r = (lane < nb) ? w[jb - j0 + lane] - pre : 0.0;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const double g = (j <= lane && lane < nb) ? Lb[j][jb - j0 + lane] : 0.0;
      a[j & 3] = fma(g, __shfl_sync(0xffffffffu, r, j), a[j & 3]);
    }
    const double xi = (a[0] + a[1]) + (a[2] + a[3]);
    if (lane < nb) w[jb - j0 + lane] = xi;
    return xi;
  }
  double lrow[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) lrow[j] = (j < lane && lane < nb) ? Lb[j][jb - j0 + lane] : 0.0;
  const double rdiag = (posdef && lane < nb) ? 1.0 / Lb[lane][jb - j0 + lane] : 1.0;
  double wi = (lane < nb) ? w[jb - j0 + lane] - pre : 0.0;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    if (j < nb) {
      // (selects: no divergent branch in the chain; the values as the
      // branches would leave them)
      const double sc = wi * rdiag;
      wi = lane == j ? sc : wi;
      const double wj = __shfl_sync(0xffffffffu, wi, j);
      const double u = fma(-lrow[j], wj, wi);
      wi = lrow[j] != 0.0 ? u : wi;
    }
  }
  if (lane < nb) w[jb - j0 + lane] = wi;
  return wi;
}

// The backward (transposed) 32 x 32 triangle of strip [jb, jb + nb) for one
// right-hand side (lane = column jb + lane), `pre` subtracted first.
__device__ __forceinline__ double bwd_chain32(const double (*Lb)[kSBP], int j0, int jb, int nb, int posdef,
                                              double *w, double pre, bool use_inv) {
  const int lane = threadIdx.x & 31;
  if (use_inv) {
    // x = L_bb^-T (w - pre): lane i's column of the inverse
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    const double r = (lane < nb) ? w[jb - j0 + lane] - pre : 0.0;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const double g = (j >= lane && j < nb) ? Lb[lane][jb - j0 + j] : 0.0;
      a[j & 3] = fma(g, __shfl_sync(0xffffffffu, r, j), a[j & 3]);
    }
    const double xi = (a[0] + a[1]) + (a[2] + a[3]);
    if (lane < nb) w[jb - j0 + lane] = xi;
    return xi;
  }
  double lcol[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) lcol[j] = (j > lane && j < nb) ? Lb[lane][jb - j0 + j] : 0.0;
  const double rdiag = (posdef && lane < nb) ? 1.0 / Lb[lane][jb - j0 + lane] : 1.0;
  double vi = (lane < nb) ? w[jb - j0 + lane] - pre : 0.0;
#pragma unroll
  for (int j = 31; j >= 0; --j) {
    if (j < nb) {
      const double sc = vi * rdiag;
      vi = lane == j ? sc : vi;
      const double xj = __shfl_sync(0xffffffffu, vi, j);
      const double u = fma(-lcol[j], xj, vi);
      vi = lcol[j] != 0.0 ? u : vi;
    }
  }
  if (lane < nb) w[jb - j0 + lane] = vi;
  return vi;
}

// A strip's product with one row (forward) or column (backward) is summed
// in four interleaved fused multiply-add chains (term u into chain u mod 4),
// then (c0 + c1) + (c2 + c3): the same sum wherever it is formed (the
// look-ahead, the rows or columns update, either block-solve form).
__device__ __forceinline__ double sum4(const double (&a)[4]) { return (a[0] + a[1]) + (a[2] + a[3]); }

// Look-ahead products of a solved strip (values x in the lanes of the
// warp) with the next strip. Forward: rows jn + lane of the next strip over
// the columns of this one (Lb: this strip's buffer). Backward: columns jn +
// lane of the next strip over the rows jb.. of this one (Ln: the next
// strip's buffer).
__device__ __forceinline__ double fwd_ahead32(const double (*Lb)[kSBP], int j0, int j1, int jb, double x) {
  const int i = jb + 32 + (int)(threadIdx.x & 31);
  double a[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int u = 0; u < 32; ++u) {
    const double xu = __shfl_sync(0xffffffffu, x, u);
    if (i < j1) a[u & 3] = fma(Lb[u][i - j0], xu, a[u & 3]);
  }
  return sum4(a);
}
__device__ __forceinline__ double bwd_ahead32(const double (*Ln)[kSBP], int j0, int jb, int nb, double x) {
  const int lane = threadIdx.x & 31;
  double a[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int t = 0; t < 32; ++t) {
    const double xt = __shfl_sync(0xffffffffu, x, t);
    if (t < nb) a[t & 3] = fma(Ln[lane][jb + t - j0], xt, a[t & 3]);
  }
  return sum4(a);
}

// The block's rows [r0, j1) minus a strip's products, for rhs
// 0..nrhs-1; threads [t0, t0 + nt) take rows in turn.
__device__ __forceinline__ void fwd_rows_update(const double (*Lb)[kSBP], int j0, int j1, int jb, int nb, int r0,
                                                int nrhs, TriSmem &sm, int t, int nt) {
  for (int i = r0 + t; i < j1; i += nt) {
    for (int r = 0; r < nrhs; ++r) {
      double a[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int u = 0; u < 32; ++u)
        if (u < nb) a[u & 3] = fma(Lb[u][i - j0], sm.w[r][jb - j0 + u], a[u & 3]);
      sm.w[r][i - j0] -= sum4(a);
    }
  }
}

// Columns of a backward strip (buffer L2, columns [j2, j2 + n2)) minus their
// products with the solved rows [r0, j1): a warp per column (warps w0.. of
// nw), lanes over the rows, a shuffle tree.
__device__ __forceinline__ void bwd_cols_update(const double (*L2)[kSBP], int j0, int j1, int j2, int n2, int r0,
                                                int nrhs, TriSmem &sm, int w0, int nw) {
  const int lane = threadIdx.x & 31;
  // four of the warp's columns at a time: their chains and shuffle trees
  // interleaved (each column's sum as one column alone would form it)
  for (int u0 = w0; u0 < n2; u0 += 4 * nw) {
    for (int r = 0; r < nrhs; ++r) {
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      for (int i = r0 + lane; i < j1; i += 32) {
        const double wv = sm.w[r][i - j0];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int u = u0 + q * nw;
          if (u < n2) acc[q] = fma(L2[u][i - j0], wv, acc[q]);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
      if (lane == 0)
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (u0 + q * nw < n2) sm.w[r][j2 - j0 + u0 + q * nw] -= acc[q];
    }
  }
}

// At most this many right-hand sides take the pipelined block solves (the
// first nrhs warps run the triangle chains, the others the rest of the
// block a strip behind); more take the step-by-step form, which computes
// the same sums.
constexpr int kPipeRhs = 4;

// sm.w[r][0, j1 - j0) <- L_bb^-1 sm.w[r] for each right-hand side, the
// block's first kRing strips issued by fwd_block_issue. Row i of the block
// takes each strip's product in strip order: the strips up to two before
// its own from the rows update, the one just before from the chain warp's
// look-ahead. Ends at a barrier.
__device__ void fwd_block_solve(const double *L, size_t sf, int j0, int j1, int posdef, int nrhs, TriSmem &sm,
                                const double *inv) {
  const int warp = threadIdx.x >> 5;
  const int nstrip = (j1 - j0 + 31) / 32;
  if (nrhs > kPipeRhs) {
    cp_async_wait_pending(0);
    __syncthreads();
    for (int k = 0; k < nstrip; ++k) {
      int jb, nb;
      fwd_strip(j0, j1, k, jb, nb);
      const double(*Lb)[kSBP] = sm.buf[k % kRing];
      if (k >= kRing) cp_async_wait_pending(min(kRing - 1, nstrip - 1 - k));
      __syncthreads();
      if (warp < nrhs) fwd_chain32(Lb, j0, jb, nb, posdef, sm.w[warp], 0.0, inv != nullptr);
      __syncthreads();
      fwd_rows_update(Lb, j0, j1, jb, nb, jb + nb, nrhs, sm, (int)threadIdx.x, kTriNT);
      __syncthreads();  // this strip's buffer is free
      if (k + kRing < nstrip) {
        int jb3, nb3;
        fwd_strip(j0, j1, k + kRing, jb3, nb3);
        tri_strip_async(L, sf, j0, j1, jb3, nb3, sm.buf[k % kRing], 0, kTriNT, inv);
      }
    }
    __syncthreads();
    return;
  }
  // Step k: the chain warps solve strip k and form its look-ahead product
  // with strip k + 1's rows; the other warps apply strip k - 1 to the rows
  // past strip k and then stream strip k + 2 into strip k - 1's buffer.
  const int C = nrhs, nf = kTriNT - 32 * C, ft = (int)threadIdx.x - 32 * C;
  cp_async_wait_pending(min(kRing - 1, nstrip - 1));  // strip 0 landed
  __syncthreads();
  double la = 0.0;
  for (int k = 0; k <= nstrip; ++k) {
    if (warp < C) {
      if (k < nstrip) {
        int jb, nb;
        fwd_strip(j0, j1, k, jb, nb);
        const double(*Lb)[kSBP] = sm.buf[k % kRing];
        const double x = fwd_chain32(Lb, j0, jb, nb, posdef, sm.w[warp], la, inv != nullptr);
        la = (k + 1 < nstrip) ? fwd_ahead32(Lb, j0, j1, jb, x) : 0.0;
      }
    } else {
      bool issued = false;
      if (k >= 1) {
        int jm, nm;
        fwd_strip(j0, j1, k - 1, jm, nm);
        fwd_rows_update(sm.buf[(k - 1) % kRing], j0, j1, jm, nm, jm + 64, C, sm, ft, nf);
        if (k - 1 + kRing < nstrip) {
          warps_sync(1, nf);  // every reader of strip k - 1's buffer done
          int jb3, nb3;
          fwd_strip(j0, j1, k - 1 + kRing, jb3, nb3);
          tri_strip_async(L, sf, j0, j1, jb3, nb3, sm.buf[(k - 1) % kRing], 32 * C, nf, inv);
          issued = true;
        }
      }
      // strip k + 1 (issued a step ago) landed before the chains take it
      if (k + 1 < nstrip && k + 1 >= kRing) cp_async_wait_pending(issued ? 1 : 0);
    }
    // strips 1 and 2, issued by every thread at the start
    if (k == 0 && nstrip > 1) cp_async_wait_pending(nstrip > 2 ? 1 : 0);
    if (k == 1 && nstrip > 2) cp_async_wait_pending(warp >= C && k - 1 + kRing < nstrip ? 1 : 0);
    __syncthreads();
  }
}

// Forward block b of each large front (a block of threads per front):
// w[j0:j1) <- L_bb^-1 w[j0:j1).
__global__ void __launch_bounds__(kTriNT) k_fwd_tri(DevPlan P, DevFactor X, const int *__restrict__ large,
                                                    int b, int posdef, double *x, double *wk,
                                                    int64_t rows_total, int nrhs) {
  extern __shared__ __align__(16) unsigned char tri_smem[];
  TriSmem &sm = *reinterpret_cast<TriSmem *>(tri_smem);
  const int s = large[blockIdx.x];
  const int f = X.sn_f[s], p = X.sn_pstore[s];
  const int j0 = b * kSB;
  if (j0 >= p) return;
  const int j1 = min(p, j0 + kSB);
  const int64_t roff = X.sn_roff[s];
  const int *rows = X.rows + roff;
  const double *L = X.arena + X.sn_off[s];
  const size_t sf = (size_t)f;
  // SPD: the diagonal blocks' inverses, when the factorization formed them
  const double *inv = (posdef && X.tri_inv && X.sn_ioff[s] >= 0) ? X.tri_inv + X.sn_ioff[s] : nullptr;
  fwd_block_issue(L, sf, j0, j1, sm, inv);
  tri_prefetch_l2(L, sf, j1, min(j1, j0 + 32 * kRing), j1, inv);
  pdl_wait();  // the strips of L in flight meanwhile
  pdl_trigger();
  for (int r = 0; r < nrhs; ++r)
    for (int t = threadIdx.x; t < j1 - j0; t += kTriNT) sm.w[r][t] = wk[(int64_t)r * rows_total + roff + j0 + t];
  fwd_block_solve(L, sf, j0, j1, posdef, nrhs, sm, inv);
  for (int r = 0; r < nrhs; ++r) {
    double *w = wk + (int64_t)r * rows_total + roff;
    double *xr = x + (int64_t)r * P.n;
    for (int t = threadIdx.x; t < j1 - j0; t += kTriNT) {
      w[j0 + t] = sm.w[r][t];
      xr[rows[j0 + t]] = sm.w[r][t];
    }
  }
}

// w[j1:f) -= L[j1:f, j0:j1) w[j0:j1) of each large front: a work item is 32
// rows; its 8 warps take 32-column strips of the block, lane = row, and the
// strips' partial sums are added in strip order.
__global__ void __launch_bounds__(256) k_fwd_gemv(DevPlan P, DevFactor X, const int *__restrict__ large,
                                                  int nlarge, int b, double *wk, int64_t rows_total,
                                                  int nrhs) {
  __shared__ double ws[kSB];
  __shared__ double part[8][33];
  __shared__ int pref[65];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bool waited = false;
  for (int chunk = 0; chunk < nlarge; chunk += 64) {
    const int cnt = min(64, nlarge - chunk);
    __syncthreads();
    if (threadIdx.x == 0) {
      pref[0] = 0;
      for (int q = 0; q < cnt; ++q) {
        const int s = large[chunk + q];
        const int f = X.sn_f[s], p = X.sn_pstore[s], j1 = min(p, (b + 1) * kSB);
        pref[q + 1] = pref[q] + ((b * kSB < p && f > j1) ? (f - j1 + 31) / 32 * nrhs : 0);
      }
    }
    __syncthreads();
    const int total = pref[cnt];
    for (int wi = blockIdx.x; wi < total; wi += gridDim.x) {
      int a = 0, bb = cnt;
      while (bb - a > 1) {
        const int mid = (a + bb) >> 1;
        if (pref[mid] <= wi) a = mid;
        else bb = mid;
      }
      const int s = large[chunk + a];
      const int f = X.sn_f[s], p = X.sn_pstore[s];
      const int j0 = b * kSB, j1 = min(p, j0 + kSB);
      const int nchunks = (f - j1 + 31) / 32;
      const int item = wi - pref[a];
      const int r = item / nchunks, rc = item % nchunks;
      double *w = wk + (int64_t)r * rows_total + X.sn_roff[s];
      const double *L = X.arena + X.sn_off[s];
      const size_t sf = (size_t)f;
      const int i = j1 + rc * 32 + lane;
      const int jb = j0 + warp * 32;
      const int nbw = (i < f && jb < j1) ? min(32, j1 - jb) : 0;
      // this lane's 32 entries of L in flight before the wait (the first
      // item: while the triangle kernel before this one still runs)
      double l[32];
      const double *li = L + (size_t)jb * sf + i;
#pragma unroll
      for (int u = 0; u < 32; ++u) l[u] = (u < nbw) ? __ldg(li + (size_t)u * sf) : 0.0;
      if (!waited) {
        pdl_wait();
        pdl_trigger();
        waited = true;
      }
      __syncthreads();
      for (int t = threadIdx.x; t < j1 - j0; t += 256) ws[t] = w[j0 + t];
      __syncthreads();
      double acc = 0.0;
#pragma unroll
      for (int u = 0; u < 32; ++u)
        if (u < nbw) acc = fma(l[u], ws[jb + u - j0], acc);
      part[warp][lane] = acc;
      __syncthreads();
      if (warp == 0 && i < f) {
        double sum = 0.0;
#pragma unroll
        for (int g = 0; g < 8; ++g) sum += part[g][lane];
        w[i] -= sum;
      }
    }
  }
}

// v[j] -= sum_{i in [j1, p)} L(i, j) v[i] for the columns j of block b of
// each large front: a work item is one column, its rows split over the
// block's threads (all loads of a thread in flight), partial sums added in
// thread order.
__global__ void __launch_bounds__(256) k_bwd_dots(DevPlan P, DevFactor X, const int *__restrict__ large,
                                                  int nlarge, int b, double *wk, int64_t rows_total,
                                                  int nrhs) {
  __shared__ int pref[65];
  __shared__ double red[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  pdl_wait();
  pdl_trigger();
  for (int chunk = 0; chunk < nlarge; chunk += 64) {
    const int cnt = min(64, nlarge - chunk);
    __syncthreads();
    if (threadIdx.x == 0) {
      pref[0] = 0;
      for (int q = 0; q < cnt; ++q) {
        const int s = large[chunk + q];
        const int p = X.sn_pstore[s], j0 = b * kSB, j1 = min(p, j0 + kSB);
        pref[q + 1] = pref[q] + ((j0 < p && j1 < p) ? (j1 - j0) * nrhs : 0);
      }
    }
    __syncthreads();
    const int total = pref[cnt];
    for (int wi = blockIdx.x; wi < total; wi += gridDim.x) {
      int a = 0, bb = cnt;
      while (bb - a > 1) {
        const int mid = (a + bb) >> 1;
        if (pref[mid] <= wi) a = mid;
        else bb = mid;
      }
      const int s = large[chunk + a];
      const int f = X.sn_f[s], p = X.sn_pstore[s];
      const int j0 = b * kSB, j1 = min(p, j0 + kSB);
      const int item = wi - pref[a];
      const int r = item / (j1 - j0), j = j0 + item % (j1 - j0);
      double *v = wk + (int64_t)r * rows_total + X.sn_roff[s];
      const double *Lj = X.arena + X.sn_off[s] + (size_t)j * f;
      double acc = 0.0;
      int i = j1 + (int)threadIdx.x;
      for (; i + 7 * 256 < p; i += 8 * 256) {
        double l[8], y[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          l[u] = __ldg(Lj + i + u * 256);
          y[u] = v[i + u * 256];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) acc = fma(l[u], y[u], acc);
      }
      for (; i < p; i += 256) acc = fma(Lj[i], v[i], acc);
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      __syncthreads();
      if (lane == 0) red[warp] = acc;
      __syncthreads();
      if (threadIdx.x == 0) {
        double sum = 0.0;
        for (int g = 0; g < 8; ++g) sum += red[g];
        v[j] -= sum;
      }
    }
  }
}

// sm.w[r][0, j1 - j0) <- L_bb^-T sm.w[r] (the rows past the block already
// taken), the block's first kRing strips issued by bwd_block_issue: strips
// from the last. A column of strip m takes, before its triangle, the
// product with the solved rows of the strips up to m - 2 (one shuffle-tree
// sum) and then that with strip m - 1's rows (the chain warp's look-ahead).
// Ends at a barrier.
__device__ void bwd_block_solve(const double *L, size_t sf, int j0, int j1, int posdef, int nrhs, TriSmem &sm,
                                const double *inv) {
  const int warp = threadIdx.x >> 5;
  const int nstrip = (j1 - j0 + 31) / 32;
  if (nrhs > kPipeRhs) {
    cp_async_wait_pending(0);
    __syncthreads();
    for (int k = 0; k < nstrip; ++k) {
      int jb, nb;
      bwd_strip(j0, j1, k, jb, nb);
      const double(*Lb)[kSBP] = sm.buf[k % kRing];
      if (k >= kRing) cp_async_wait_pending(min(kRing - 1, nstrip - 1 - k));
      __syncthreads();
      if (k >= 2) {
        int jm, nm;
        bwd_strip(j0, j1, k - 2, jm, nm);
        bwd_cols_update(Lb, j0, j1, jb, nb, jm, nrhs, sm, warp, kTriNT / 32);
      }
      __syncthreads();
      if (warp < nrhs) {
        double la = 0.0;
        if (k >= 1) {
          // strip k - 1's solved values in the lanes, as the chain left them
          int jp, np;
          bwd_strip(j0, j1, k - 1, jp, np);
          const int lane = threadIdx.x & 31;
          const double xp = (lane < np) ? sm.w[warp][jp - j0 + lane] : 0.0;
          la = bwd_ahead32(Lb, j0, jp, np, xp);
        }
        bwd_chain32(Lb, j0, jb, nb, posdef, sm.w[warp], la, inv != nullptr);
      }
      __syncthreads();  // this strip's buffer is free
      if (k + kRing < nstrip) {
        int jb3, nb3;
        bwd_strip(j0, j1, k + kRing, jb3, nb3);
        tri_strip_async(L, sf, j0, j1, jb3, nb3, sm.buf[k % kRing], 0, kTriNT, inv);
      }
    }
    __syncthreads();
    return;
  }
  // Step k: the chain warps solve strip k and form its look-ahead product
  // with strip k + 1's columns; the other warps stream strip k + 2 into
  // strip k - 1's buffer and apply the rows solved up to strip k - 1 to
  // strip k + 1's columns.
  const int C = nrhs, nf = kTriNT - 32 * C, fw = warp - C, nfw = nf / 32;
  cp_async_wait_pending(nstrip > 2 ? 1 : 0);  // strips 0 and 1 landed
  __syncthreads();
  double la = 0.0;
  for (int k = 0; k < nstrip; ++k) {
    if (warp < C) {
      int jb, nb;
      bwd_strip(j0, j1, k, jb, nb);
      const double x = bwd_chain32(sm.buf[k % kRing], j0, jb, nb, posdef, sm.w[warp], la, inv != nullptr);
      la = 0.0;
      if (k + 1 < nstrip) la = bwd_ahead32(sm.buf[(k + 1) % kRing], j0, jb, nb, x);
    } else {
      if (k >= 1 && k - 1 + kRing < nstrip) {
        // strip k - 1's buffer: its last readers (chain k - 1, look-ahead
        // k - 2, the columns update one step before) are done
        int jb3, nb3;
        bwd_strip(j0, j1, k - 1 + kRing, jb3, nb3);
        tri_strip_async(L, sf, j0, j1, jb3, nb3, sm.buf[(k - 1) % kRing], 32 * C, nf, inv);
      }
      if (k >= 1 && k + 1 < nstrip) {
        int jm, nm, j2, n2;
        bwd_strip(j0, j1, k - 1, jm, nm);
        bwd_strip(j0, j1, k + 1, j2, n2);
        bwd_cols_update(sm.buf[(k + 1) % kRing], j0, j1, j2, n2, jm, C, sm, fw, nfw);
      }
      // strip k + 2 landed before the next step's readers take it
      if (k + 2 < nstrip && k + 2 >= kRing) cp_async_wait_pending(0);
    }
    if (k == 0 && nstrip > 2) cp_async_wait_pending(0);  // strip 2, issued by every thread at the start
    __syncthreads();
  }
}

// Backward block b of each large front (a block of threads per front; its
// rows past the block already taken by k_bwd_dots).
__global__ void __launch_bounds__(kTriNT) k_bwd_tri(DevPlan P, DevFactor X, const int *__restrict__ large,
                                                    int b, int posdef, double *x, double *wk,
                                                    int64_t rows_total, int nrhs) {
  extern __shared__ __align__(16) unsigned char tri_smem[];
  TriSmem &sm = *reinterpret_cast<TriSmem *>(tri_smem);
  const int s = large[blockIdx.x];
  const int f = X.sn_f[s], p = X.sn_pstore[s];
  const int j0 = b * kSB;
  if (j0 >= p) return;
  const int j1 = min(p, j0 + kSB);
  const int64_t roff = X.sn_roff[s];
  const int *rows = X.rows + roff;
  const double *L = X.arena + X.sn_off[s];
  const size_t sf = (size_t)f;
  const double *inv = (posdef && X.tri_inv && X.sn_ioff[s] >= 0) ? X.tri_inv + X.sn_ioff[s] : nullptr;
  bwd_block_issue(L, sf, j0, j1, sm, inv);
  {
    int jl, nl;  // the backward strips past the first kRing: columns [j0, jl)
    bwd_strip(j0, j1, min(kRing, (j1 - j0 + 31) / 32) - 1, jl, nl);
    tri_prefetch_l2(L, sf, j1, j0, jl, inv);
  }
  pdl_wait();  // the strips of L in flight meanwhile
  pdl_trigger();
  for (int r = 0; r < nrhs; ++r)
    for (int t = threadIdx.x; t < j1 - j0; t += kTriNT) sm.w[r][t] = wk[(int64_t)r * rows_total + roff + j0 + t];
  bwd_block_solve(L, sf, j0, j1, posdef, nrhs, sm, inv);
  for (int r = 0; r < nrhs; ++r) {
    double *w = wk + (int64_t)r * rows_total + roff;
    double *xr = x + (int64_t)r * P.n;
    for (int t = threadIdx.x; t < j1 - j0; t += kTriNT) {
      w[j0 + t] = sm.w[r][t];
      xr[rows[j0 + t]] = sm.w[r][t];
    }
  }
}

// ---------------------------------------------------------------------------
// Residual r = b - A x and backward errors (refinement.cpp:39-130), on the
// full symmetric pattern, eight lanes per row, compensated dot products
// (Ogita, Rump & Oishi, "Accurate sum and dot product", SIAM J. Sci.
// Comput. 26(6), 2005: TwoProduct via fma, TwoSum) in the new numbering.
__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// kResLanes lanes per row (rows hold a few entries of the symmetric
// pattern: a warp takes 32 / kResLanes rows at a time).
constexpr int kResLanes = 8;

__global__ void k_residual(DevPlan P, const double *__restrict__ vals, const double *__restrict__ x,
                           const double *__restrict__ b, double *__restrict__ r, int n,
                           unsigned long long *mx /* [0] |r|max [1] row |A| sum max [2] |x| max [3] |b| max [4] omega */) {
  constexpr int RPW = 32 / kResLanes;
  const int lane = threadIdx.x & 31, sub = lane % kResLanes, grp = lane / kResLanes;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  double m_r = 0.0, m_a = 0.0, m_x = 0.0, m_b = 0.0, m_o = 0.0;
  for (int i0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * RPW; i0 < n; i0 += warps * RPW) {
    const int i = i0 + grp;
    double s = 0.0, c = 0.0, as = 0.0, ra = 0.0;
    if (i < n) {
      for (int k = P.sptr[i] + sub; k < P.sptr[i + 1]; k += kResLanes) {
        const double a = vals[P.sidx[k]];
        const double xj = x[P.srow[k]];
        const double pr = a * xj;
        const double pe = fma(a, xj, -pr);
        double t, e;
        two_sum(s, pr, t, e);
        s = t;
        c += e + pe;
        as = fma(fabs(a), fabs(xj), as);
        ra += fabs(a);
      }
    }
    for (int o = kResLanes / 2; o > 0; o >>= 1) {  // within the row's lanes
      const double s2 = __shfl_xor_sync(0xffffffffu, s, o);
      const double c2 = __shfl_xor_sync(0xffffffffu, c, o);
      double t, e;
      two_sum(s, s2, t, e);
      s = t;
      c += c2 + e;
      as += __shfl_xor_sync(0xffffffffu, as, o);
      ra += __shfl_xor_sync(0xffffffffu, ra, o);
    }
    if (sub == 0 && i < n) {
      const double bi = b[i];
      double t, e;
      two_sum(bi, -s, t, e);
      const double res = t + (e - c);
      r[i] = res;
      m_r = fmax(m_r, fabs(res));
      m_a = fmax(m_a, ra);
      m_x = fmax(m_x, fabs(x[i]));
      m_b = fmax(m_b, fabs(bi));
      const double den = as + fabs(bi);
      const double om = den > 0.0 ? fabs(res) / den : (res == 0.0 ? 0.0 : INFINITY);
      m_o = fmax(m_o, om);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    m_r = fmax(m_r, __shfl_xor_sync(0xffffffffu, m_r, o));
    m_a = fmax(m_a, __shfl_xor_sync(0xffffffffu, m_a, o));
    m_x = fmax(m_x, __shfl_xor_sync(0xffffffffu, m_x, o));
    m_b = fmax(m_b, __shfl_xor_sync(0xffffffffu, m_b, o));
    m_o = fmax(m_o, __shfl_xor_sync(0xffffffffu, m_o, o));
  }
  if (lane == 0) {
    atomicMax(mx + 0, (unsigned long long)__double_as_longlong(m_r));
    atomicMax(mx + 1, (unsigned long long)__double_as_longlong(m_a));
    atomicMax(mx + 2, (unsigned long long)__double_as_longlong(m_x));
    atomicMax(mx + 3, (unsigned long long)__double_as_longlong(m_b));
    atomicMax(mx + 4, (unsigned long long)__double_as_longlong(m_o));
  }
}

// Up to kResLanes right-hand sides at once: the pattern and the values read
// once for all of them, x interleaved in the new numbering (xi[i * nr + q]),
// b read and r written in the original numbering (column q at q * n). Each
// column's sums take the same operations in the same order as k_residual;
// after the row's reduction, lane sub keeps the maxima of column sub.
// Latency: a lane's next kResAhead entries have their indices, then their
// values, loaded together, the next entry's x while the current one is
// summed, and the row's b and x ahead of the entries.
constexpr int kResAhead = 4;

__global__ void __launch_bounds__(256, 2)
    k_residual_rhs(DevPlan P, const double *__restrict__ vals, const double *__restrict__ xi, int nr,
                   const double *__restrict__ b, double *__restrict__ r, int n,
                   unsigned long long *mx /* 8 per column, as k_residual */) {
  constexpr int RPW = 32 / kResLanes;
  const int lane = threadIdx.x & 31, sub = lane % kResLanes, grp = lane / kResLanes;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  double m_r = 0.0, m_a = 0.0, m_x = 0.0, m_b = 0.0, m_o = 0.0;
  for (int i0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * RPW; i0 < n; i0 += warps * RPW) {
    const int i = i0 + grp;
    double s[kResLanes], c[kResLanes], as[kResLanes], ra = 0.0;
#pragma unroll
    for (int q = 0; q < kResLanes; ++q) s[q] = c[q] = as[q] = 0.0;
    int64_t ob = 0;
    double bi = 0.0, xs = 0.0;
    if (sub < nr && i < n) {
      ob = (int64_t)sub * n + P.perm[i];
      bi = b[ob];
      xs = xi[(int64_t)i * nr + sub];
    }
    if (i < n) {
      const int ke = P.sptr[i + 1];
      for (int k0 = P.sptr[i] + sub; k0 < ke; k0 += kResLanes * kResAhead) {
        // entries past the row's end read index 0 and are not summed
        int jx[kResAhead], ix[kResAhead];
#pragma unroll
        for (int u = 0; u < kResAhead; ++u) {
          const int k = k0 + u * kResLanes;
          jx[u] = k < ke ? P.srow[k] : 0;
          ix[u] = k < ke ? P.sidx[k] : 0;
        }
        double av[kResAhead], xc[kResLanes];
#pragma unroll
        for (int u = 0; u < kResAhead; ++u) av[u] = vals[ix[u]];
#pragma unroll
        for (int q = 0; q < kResLanes; ++q) xc[q] = q < nr ? xi[(int64_t)jx[0] * nr + q] : 0.0;
#pragma unroll
        for (int u = 0; u < kResAhead; ++u) {
          double xn[kResLanes];
#pragma unroll
          for (int q = 0; q < kResLanes; ++q)
            xn[q] = (u + 1 < kResAhead && q < nr) ? xi[(int64_t)jx[u + 1 < kResAhead ? u + 1 : u] * nr + q] : 0.0;
          if (k0 + u * kResLanes < ke) {
            const double a = av[u];
#pragma unroll
            for (int q = 0; q < kResLanes; ++q) {
              if (q < nr) {
                const double xv = xc[q];
                const double pr = a * xv;
                const double pe = fma(a, xv, -pr);
                double t, e;
                two_sum(s[q], pr, t, e);
                s[q] = t;
                c[q] += e + pe;
                as[q] = fma(fabs(a), fabs(xv), as[q]);
              }
            }
            ra += fabs(a);
          }
#pragma unroll
          for (int q = 0; q < kResLanes; ++q) xc[q] = xn[q];
        }
      }
    }
    for (int o = kResLanes / 2; o > 0; o >>= 1) {  // within the row's lanes
#pragma unroll
      for (int q = 0; q < kResLanes; ++q) {
        if (q < nr) {
          const double s2 = __shfl_xor_sync(0xffffffffu, s[q], o);
          const double c2 = __shfl_xor_sync(0xffffffffu, c[q], o);
          double t, e;
          two_sum(s[q], s2, t, e);
          s[q] = t;
          c[q] += c2 + e;
          as[q] += __shfl_xor_sync(0xffffffffu, as[q], o);
        }
      }
      ra += __shfl_xor_sync(0xffffffffu, ra, o);
    }
    // the butterfly leaves the compensation term rounded differently on
    // the row's lanes: every column takes the row's first lane's values,
    // the ones k_residual uses
    double S = 0.0, C = 0.0, AS = 0.0;
    const int lead = grp * kResLanes;
#pragma unroll
    for (int q = 0; q < kResLanes; ++q) {
      if (q < nr) {
        const double s0 = __shfl_sync(0xffffffffu, s[q], lead);
        const double c0 = __shfl_sync(0xffffffffu, c[q], lead);
        const double a0 = __shfl_sync(0xffffffffu, as[q], lead);
        if (q == sub) {
          S = s0;
          C = c0;
          AS = a0;
        }
      }
    }
    if (sub < nr && i < n) {
      double t, e;
      two_sum(bi, -S, t, e);
      const double res = t + (e - C);
      r[ob] = res;
      m_r = fmax(m_r, fabs(res));
      m_a = fmax(m_a, ra);
      m_x = fmax(m_x, fabs(xs));
      m_b = fmax(m_b, fabs(bi));
      const double den = AS + fabs(bi);
      const double om = den > 0.0 ? fabs(res) / den : (res == 0.0 ? 0.0 : INFINITY);
      m_o = fmax(m_o, om);
    }
  }
  for (int o = 16; o >= kResLanes; o >>= 1) {  // across the rows, per column
    m_r = fmax(m_r, __shfl_xor_sync(0xffffffffu, m_r, o));
    m_a = fmax(m_a, __shfl_xor_sync(0xffffffffu, m_a, o));
    m_x = fmax(m_x, __shfl_xor_sync(0xffffffffu, m_x, o));
    m_b = fmax(m_b, __shfl_xor_sync(0xffffffffu, m_b, o));
    m_o = fmax(m_o, __shfl_xor_sync(0xffffffffu, m_o, o));
  }
  if (grp == 0 && sub < nr) {
    unsigned long long *m = mx + 8 * sub;
    atomicMax(m + 0, (unsigned long long)__double_as_longlong(m_r));
    atomicMax(m + 1, (unsigned long long)__double_as_longlong(m_a));
    atomicMax(m + 2, (unsigned long long)__double_as_longlong(m_x));
    atomicMax(m + 3, (unsigned long long)__double_as_longlong(m_b));
    atomicMax(m + 4, (unsigned long long)__double_as_longlong(m_o));
  }
}

// xi[i * nr + q] = x[q * n + perm[i]]: nr columns interleaved in the new
// numbering, for k_residual_rhs.
__global__ void k_gather_interleave(const double *__restrict__ x, int n, int nr, const int *__restrict__ perm,
                                    double *__restrict__ xi) {
  const int64_t tot = (int64_t)n * nr;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t / nr), q = (int)(t % nr);
    xi[t] = x[(int64_t)q * n + perm[i]];
  }
}

__global__ void k_axpy(double *__restrict__ x, const double *__restrict__ dx, int64_t len) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < len;
       t += (int64_t)gridDim.x * blockDim.x)
    x[t] += dx[t];
}

// ---------------------------------------------------------------------------
// Krylov helpers of the FGMRES refinement (refinement.cpp:451-643): dot
// products in a fixed order (per-block partials, then one block), vector
// updates whose coefficient stays in device memory, the product with A.

constexpr int kDotBlocks = 296;

__global__ void __launch_bounds__(256) k_dot_part(const double *__restrict__ a, const double *__restrict__ b,
                                                  int64_t n, double *__restrict__ part) {
  __shared__ double red[8];
  double s = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    s = fma(a[t], b[t], s);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    part[blockIdx.x] = t;
  }
}

__global__ void k_dot_fin(const double *__restrict__ part, int nparts, double *__restrict__ out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int t = threadIdx.x; t < nparts; t += blockDim.x) s += part[t];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    *out = t;
  }
}

// y -= coef[0] * x
__global__ void k_axpy_coef(double *__restrict__ y, const double *__restrict__ x, const double *__restrict__ coef,
                            int64_t n) {
  const double c = *coef;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    y[t] = fma(-c, x[t], y[t]);
}

// y = x * alpha; y may be x (in place), so neither pointer is restrict
__global__ void k_scale(double *y, const double *x, double alpha, int64_t n) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    y[t] = x[t] * alpha;
}

// xc = x0 + sum_l y[l] Z[l]
__global__ void k_lincomb(double *__restrict__ xc, const double *__restrict__ x0, const double *__restrict__ Z,
                          const double *__restrict__ y, int k, int64_t n) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    double v = x0[t];
    for (int l = 0; l < k; ++l) v = fma(y[l], Z[(int64_t)l * n + t], v);
    xc[t] = v;
  }
}

// y = A x in the new numbering (the unscaled values), a warp per row
__global__ void k_spmv(DevPlan P, const double *__restrict__ vals, const double *__restrict__ x,
                       double *__restrict__ y, int n) {
  constexpr int RPW = 32 / kResLanes;  // rows per warp, as k_residual
  const int lane = threadIdx.x & 31, sub = lane % kResLanes, grp = lane / kResLanes;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int i0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * RPW; i0 < n; i0 += warps * RPW) {
    const int i = i0 + grp;
    double s = 0.0;
    if (i < n)
      for (int k = P.sptr[i] + sub; k < P.sptr[i + 1]; k += kResLanes) s = fma(vals[P.sidx[k]], x[P.srow[k]], s);
    for (int o = kResLanes / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (sub == 0 && i < n) y[i] = s;
  }
}

}  // namespace smfg
