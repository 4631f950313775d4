// A posteriori threshold pivoting (APTP) of large indefinite fronts: the
// dense kernel smf's deterministic mode runs on every indefinite front of at
// least 512 rows (solver/src/ldlt_aptp.cpp:1-751, as 2D tile tasks in
// parallel/tile_tasks.cpp:256-351; dispatch multifrontal_serial.cpp:796-821,
// parallel/thread_plan.hpp:43-47). The fully summed columns are taken in
// block columns of 256 (Control::top_tile_nb, control.hpp:638). Per block:
//   - the diagonal tile is factored speculatively by one CTA (an inner sweep
//     of 32-column blocks, complete pivoting on each, then on what failed
//     inside the tile), the rows below it are formed by a triangular solve
//     on many CTAs and checked afterwards against 1/u; the block keeps the
//     leading pivots whose multipliers pass and restores the rest from a
//     backup, in place;
//   - the rest of the front takes a rank-nelim update with those pivots
//     (the eligible columns right of them, and the earlier failed columns)
//     as tiled FP64 GEMMs over the whole GPU.
// At the end the failed columns move behind the pivots (one gather through
// a scratch front) and the non-eligible triangle takes one deferred update.
// Every entry takes the reference's operations in the reference's order and
// rounding: the portable BLAS loops' fused multiply-add chains (a zero
// multiplier skipped), and the fused forms GCC gives ldlt_aptp.cpp's
// a*b + c*d expressions (fma(a, b, c*d), except the first output of
// row_times_d, fma(c, d, a*b)). With the same input the front's L, D, pivot
// order, tags and Schur complement are the reference's, bit for bit.
#pragma once
#include "smfg_aptp_host.h"
#include "smfg_internal.cuh"

namespace smfg {
namespace aptp {

constexpr int kTileNT = 256;

__device__ __forceinline__ size_t ix(int j, int ld) { return (size_t)j * (size_t)ld; }

__device__ __forceinline__ bool l_ok(double l, double inv_u) { return fabs(l) <= inv_u; }

// Stable inverse of the 2x2 pivot (ldlt_aptp.cpp:83-93): a*c - b*b is fused
// as GCC contracts it.
__device__ __forceinline__ void inv2(double d00, double d10, double d11, double &i00, double &i10,
                                     double &i11) {
  const double s = max3_ref(fabs(d00), fabs(d10), fabs(d11));
  const double a = d00 / s, b = d10 / s, c = d11 / s;
  const double inv = 1.0 / __dmul_rn(fma(a, c, -__dmul_rn(b, b)), s);
  i00 = __dmul_rn(c, inv);
  i10 = __dmul_rn(-b, inv);
  i11 = __dmul_rn(a, inv);
}

// (L D) of one row for the pivots [0, k) of a tile (D inline: diagonal at
// T(t, t), 2x2 off-diagonal at T(t + 1, t)) (ldlt_aptp.cpp:270-287).
__device__ __forceinline__ double ld_of(const double *T, int ld, const int8_t *tags, int t, double l0,
                                        double l1) {
  const double d00 = T[ix(t, ld) + t];
  if (tags[t] == 2) return fma(l1, T[ix(t, ld) + t + 1], __dmul_rn(l0, d00));
  if (tags[t] == -1) {  // second of a 2x2: l0 is the first column's value, l1 this one's
    return fma(l0, T[ix(t - 1, ld) + t], __dmul_rn(l1, T[ix(t, ld) + t]));
  }
  return __dmul_rn(l0, d00);
}

// ---------------------------------------------------------------------------
// CTA-level pieces of the diagonal tile's factorization (one CTA of
// kTileNT threads per tile; the tile lives in global memory / L2).

struct TileShared {
  double bk1[kNb * kIb];   // inner block backup: column t at bk1 + t * kNb (tile rows)
  double dinv1[2 * kIb];
  int q1[kNb];
  int lpc1[kIb];
  int cp_lp[kNb];
  int itmp[kNb];
  double rv[32];
  int ri[32], rj[32];
  int kind, a, b, ok, nq1, nmin, nelim;
};

// Symmetric transposition of view positions p < q (ldlt_aptp.cpp:67-80);
// tags, rows, lp and loc follow. Callers synchronize before.
static __device__ void cta_swap(double *A, int ld, int m, int p, int q, int8_t *tags, int *rows, int *lp, int *loc) {
  if (p == q) return;
  if (p > q) {
    const int t = p;
    p = q;
    q = t;
  }
  const int items = m - 1;  // p diag pair + (c < p) + (p < c < q) + (r > q)
  for (int t = threadIdx.x; t < items; t += blockDim.x) {
    size_t e1, e2;
    if (t == 0) {
      e1 = ix(p, ld) + p;
      e2 = ix(q, ld) + q;
    } else if (t <= p) {
      const int c = t - 1;
      e1 = ix(c, ld) + p;
      e2 = ix(c, ld) + q;
    } else if (t < q) {
      const int c = t;  // p < c < q
      e1 = ix(p, ld) + c;
      e2 = ix(c, ld) + q;
    } else {
      const int r = t + 1;  // r > q
      e1 = ix(p, ld) + r;
      e2 = ix(q, ld) + r;
    }
    const double x = A[e1];
    A[e1] = A[e2];
    A[e2] = x;
  }
  if (threadIdx.x == 0) {
    const int8_t tg = tags[p];
    tags[p] = tags[q];
    tags[q] = tg;
    int u = rows[p];
    rows[p] = rows[q];
    rows[q] = u;
    u = lp[p];
    lp[p] = lp[q];
    lp[q] = u;
    if (loc) {
      u = loc[p];
      loc[p] = loc[q];
      loc[q] = u;
    }
  }
  __syncthreads();
}

__device__ __forceinline__ double sym_at(const double *A, int ld, int i, int j) {
  return (i >= j) ? A[ix(j, ld) + i] : A[ix(i, ld) + j];
}

// Block-wide argmax of |A| over the lower triangle of rows / columns [k, n):
// the first maximum in column-major order, NaNs never chosen
// (ldlt_aptp.cpp:108-122).
static __device__ void cta_argmax(const double *A, int ld, int n, int k, TileShared &sh, double &amax, int &bi, int &bj) {
  double best = -1.0;
  int bii = -1, bjj = -1;
  // a warp per column, its lanes down the rows; every lane keeps its first
  // maximum in (column, row) order
  const int lane0 = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int j = k + (threadIdx.x >> 5); j < n; j += nw) {
    const double *col = A + ix(j, ld);
    for (int i = j + lane0; i < n; i += 32) {
      const double v = fabs(col[i]);
      if (v > best) {
        best = v;
        bii = i;
        bjj = j;
      }
    }
  }
  // larger value wins; equal values: the lower column, then the lower row
  auto better = [](double v1, int j1, int i1, double v2, int j2, int i2) {
    if (v1 > v2) return true;
    if (v1 < v2 || j1 < 0) return false;
    if (j2 < 0) return true;
    return j1 < j2 || (j1 == j2 && i1 < i2);
  };
  for (int o = 16; o > 0; o >>= 1) {
    const double v2 = __shfl_down_sync(0xffffffffu, best, o);
    const int i2 = __shfl_down_sync(0xffffffffu, bii, o);
    const int j2 = __shfl_down_sync(0xffffffffu, bjj, o);
    if (better(v2, j2, i2, best, bjj, bii)) {
      best = v2;
      bii = i2;
      bjj = j2;
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    sh.rv[wid] = best;
    sh.ri[wid] = bii;
    sh.rj[wid] = bjj;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double bv = sh.rv[0];
    int b_i = sh.ri[0], b_j = sh.rj[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      if (better(sh.rv[w], sh.rj[w], sh.ri[w], bv, b_j, b_i)) {
        bv = sh.rv[w];
        b_i = sh.ri[w];
        b_j = sh.rj[w];
      }
    sh.rv[0] = bv;
    sh.ri[0] = b_i;
    sh.rj[0] = b_j;
  }
  __syncthreads();
  amax = sh.rv[0];
  bi = sh.ri[0];
  bj = sh.rj[0];
  __syncthreads();
}

// Complete pivoting on an n x n view (ldlt_aptp.cpp:101-210); returns the
// pivots taken. lp: the view's permutation record.
static __device__ int cta_complete(double *A, int ld, int n, int8_t *tags, int *rows, int *lp, int *loc, double inv_u,
                            double small, TileShared &sh) {
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    lp[t] = t;
    tags[t] = 0;
  }
  __syncthreads();
  int k = 0;
  while (k < n) {
    double amax;
    int bi, bj;
    cta_argmax(A, ld, n, k, sh, amax, bi, bj);
    if (!(amax >= small) || !isfinite(amax)) break;
    if (threadIdx.x == 0) {
      int kind = 1, a = bj, b = -1;
      if (bi != bj) {
        const double amm = A[ix(bj, ld) + bj], att = A[ix(bi, ld) + bi], amt = A[ix(bj, ld) + bi];
        const double delta = fma(amm, att, -__dmul_rn(amt, amt));
        if (fabs(delta) >= __dmul_rn(__dmul_rn(0.5, amt), amt)) {
          kind = 2;
          b = bi;
        } else {
          a = (fabs(att) > fabs(amm)) ? bi : bj;
        }
      }
      sh.kind = kind;
      sh.a = a;
      sh.b = b;
    }
    __syncthreads();
    const int kind = sh.kind, a = sh.a, b = sh.b;
    // a posteriori bound inside the view
    bool bad = false;
    if (kind == 1) {
      const double lim = __dmul_rn(inv_u, fabs(A[ix(a, ld) + a]));
      for (int r = k + threadIdx.x; r < n; r += blockDim.x)
        if (r != a && !(fabs(sym_at(A, ld, r, a)) <= lim)) bad = true;
    } else {
      double i00, i10, i11;
      inv2(A[ix(a, ld) + a], A[ix(a, ld) + b], A[ix(b, ld) + b], i00, i10, i11);
      for (int r = k + threadIdx.x; r < n; r += blockDim.x) {
        if (r == a || r == b) continue;
        const double x0 = sym_at(A, ld, r, a), x1 = sym_at(A, ld, r, b);
        if (!l_ok(fma(i00, x0, __dmul_rn(i10, x1)), inv_u) || !l_ok(fma(i10, x0, __dmul_rn(i11, x1)), inv_u))
          bad = true;
      }
    }
    if (__syncthreads_or(bad)) break;
    if (kind == 1) {
      cta_swap(A, ld, n, k, a, tags, rows, lp, loc);
      const double *ck = A + ix(k, ld);
      const double inv_d = 1.0 / ck[k];
      // entries (i, j), k < j <= i < n: one fused step each (a warp per
      // column)
      for (int jj = k + 1 + (threadIdx.x >> 5); jj < n; jj += (blockDim.x >> 5)) {
        const double lj = __dmul_rn(ck[jj], inv_d);
        if (lj == 0.0) continue;
        double *cj = A + ix(jj, ld);
        for (int ii = jj + (threadIdx.x & 31); ii < n; ii += 32) cj[ii] = fma(-ck[ii], lj, cj[ii]);
      }
      __syncthreads();
      double *ckw = A + ix(k, ld);
      for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) ckw[i] = __dmul_rn(ckw[i], inv_d);
      if (threadIdx.x == 0) tags[k] = 1;
      __syncthreads();
      k += 1;
    } else {
      int partner = b;
      if (a != k) {
        cta_swap(A, ld, n, k, a, tags, rows, lp, loc);
        if (partner == k) partner = a;
      }
      if (partner != k + 1) cta_swap(A, ld, n, k + 1, partner, tags, rows, lp, loc);
      double *c0 = A + ix(k, ld), *c1 = A + ix(k + 1, ld);
      double i00, i10, i11;
      inv2(c0[k], c0[k + 1], c1[k + 1], i00, i10, i11);
      for (int jj = k + 2 + (threadIdx.x >> 5); jj < n; jj += (blockDim.x >> 5)) {
        const double a0 = c0[jj], a1 = c1[jj];
        const double l0 = fma(i00, a0, __dmul_rn(i10, a1)), l1 = fma(i10, a0, __dmul_rn(i11, a1));
        if (l0 == 0.0 && l1 == 0.0) continue;
        double *cj = A + ix(jj, ld);
        for (int ii = jj + (threadIdx.x & 31); ii < n; ii += 32)
          cj[ii] = __dsub_rn(cj[ii], fma(c0[ii], l0, __dmul_rn(c1[ii], l1)));
      }
      __syncthreads();
      for (int i = k + 2 + threadIdx.x; i < n; i += blockDim.x) {
        const double a0 = c0[i], a1 = c1[i];
        c0[i] = fma(i00, a0, __dmul_rn(i10, a1));
        c1[i] = fma(i10, a0, __dmul_rn(i11, a1));
      }
      if (threadIdx.x == 0) {
        tags[k] = 2;
        tags[k + 1] = -1;
      }
      __syncthreads();
      k += 2;
    }
  }
  __syncthreads();
  return k;
}

// Rows [r0, r0 + w) of columns [0, ncols): new row r0 + t takes old row
// r0 + perm[t] (ldlt_aptp.cpp:214-221); w <= blockDim.x.
static __device__ void cta_permute_rows(double *A, int ld, int ncols, int r0, int w, const int *perm) {
  for (int c = 0; c < ncols; ++c) {
    double v = 0.0;
    if ((int)threadIdx.x < w) v = A[ix(c, ld) + r0 + perm[threadIdx.x]];
    __syncthreads();
    if ((int)threadIdx.x < w) A[ix(c, ld) + r0 + threadIdx.x] = v;
    __syncthreads();
  }
}

static __device__ bool cta_identity(const int *perm, int w) {
  bool diff = false;
  for (int t = threadIdx.x; t < w; t += blockDim.x) diff = diff || perm[t] != t;
  return !__syncthreads_or(diff);
}

// x := x L^-T for one row (x holds its first k entries, k <= KMAX), L the
// unit lower triangle of the tile at T (2x2 off-diagonals read as zero): per
// entry one fused chain over the earlier columns in order, a zero L entry
// skipped; then the D^-1 scaling, returning the first pivot whose
// multipliers exceed 1/u, or k (ldlt_aptp.cpp:232-265, :292-304).
template <int KMAX>
__device__ __forceinline__ int row_solve_scale(double (&x)[KMAX], int k, const double *T, int ld, const int8_t *tags,
                                               const double *dinv, double inv_u) {
#pragma unroll
  for (int j = 1; j < KMAX; ++j) {
    if (j < k) {
      double xj = x[j];
#pragma unroll
      for (int p = 0; p < j; ++p) {
        const double l = (tags[p] == 2 && j == p + 1) ? 0.0 : T[ix(p, ld) + j];
        if (l != 0.0) xj = fma(-x[p], l, xj);
      }
      x[j] = xj;
    }
  }
  int fail = k;
#pragma unroll
  for (int t = 0; t < KMAX; ++t) {
    if (t < k) {
      if (tags[t] == 2) {
        const double i00 = dinv[2 * t], i10 = dinv[2 * t + 1], i11 = dinv[2 * (t + 1)];
        const double a0 = x[t], a1 = x[t + 1 < KMAX ? t + 1 : t];
        const double l0 = fma(i00, a0, __dmul_rn(i10, a1)), l1 = fma(i10, a0, __dmul_rn(i11, a1));
        x[t] = l0;
        if (t + 1 < KMAX) x[t + 1] = l1;
        if (fail == k && (!l_ok(l0, inv_u) || !l_ok(l1, inv_u))) fail = t;
      } else if (tags[t] == 1) {
        const double l = __dmul_rn(x[t], dinv[2 * t]);
        x[t] = l;
        if (fail == k && !l_ok(l, inv_u)) fail = t;
      }
    }
  }
  return fail;
}

// One inner block column [c0, c0 + w1) of the tile sweep (block ib = 32):
// backup, complete pivoting on the diagonal block, its permutation applied,
// ApplyN on the tile rows below, ApplyT on the earlier failed columns,
// restore, UpdateNN / NT / TN (ldlt_aptp.cpp:390-588 at level 1). Returns
// the accepted pivots.
static __device__ int tile_inner_block(double *T, int ld, int w, int c0, int w1, int8_t *tags, int *rows, int *lp,
                                int *loc, double inv_u, double small, TileShared &sh) {
  // 1. backup: column c0 + t, tile rows [c0 + t, w)
  for (int t = 0; t < w1; ++t)
    for (int r = c0 + t + threadIdx.x; r < w; r += blockDim.x) sh.bk1[t * kNb + r] = T[ix(c0 + t, ld) + r];
  __syncthreads();
  // 2. complete pivoting on the diagonal block
  const int ne_t = cta_complete(T + ix(c0, ld) + c0, ld, w1, tags + c0, rows + c0, sh.lpc1, loc ? loc + c0 : nullptr,
                                inv_u, small, sh);
  // 3. its permutation on the rest of the tile
  if (!cta_identity(sh.lpc1, w1)) {
    cta_permute_rows(T, ld, c0, c0, w1, sh.lpc1);
    for (int t = 0; t < w1; ++t)
      for (int r = c0 + w1 + threadIdx.x; r < w; r += blockDim.x) T[ix(c0 + t, ld) + r] = sh.bk1[sh.lpc1[t] * kNb + r];
    if ((int)threadIdx.x < w1) sh.itmp[threadIdx.x] = lp[c0 + sh.lpc1[threadIdx.x]];
    __syncthreads();
    if ((int)threadIdx.x < w1) lp[c0 + threadIdx.x] = sh.itmp[threadIdx.x];
    __syncthreads();
  }
  const double *Tb = T + ix(c0, ld) + c0;  // the block's diagonal tile
  const int8_t *tb = tags + c0;
  if (threadIdx.x == 0) {
    for (int j = 0; j < ne_t; ++j) {
      if (tb[j] == 2) {
        double i00, i10, i11;
        inv2(Tb[ix(j, ld) + j], Tb[ix(j, ld) + j + 1], Tb[ix(j + 1, ld) + j + 1], i00, i10, i11);
        sh.dinv1[2 * j] = i00;
        sh.dinv1[2 * j + 1] = i10;
        sh.dinv1[2 * (j + 1)] = i11;
        sh.dinv1[2 * (j + 1) + 1] = 0.0;
        ++j;
      } else {
        sh.dinv1[2 * j] = 1.0 / Tb[ix(j, ld) + j];
        sh.dinv1[2 * j + 1] = 0.0;
      }
    }
    sh.nmin = ne_t;
  }
  __syncthreads();
  // 4. ApplyN on the tile rows below the block and ApplyT (check pass) on
  // the earlier failed columns: the first failing pivot over all rows
  const int nq = sh.nq1;
  if (ne_t > 0) {
    const int nbelow = w - c0 - w1;
    int fail = ne_t;
    for (int t = threadIdx.x; t < nbelow + nq; t += blockDim.x) {
      double x[kIb];
      const bool below = t < nbelow;
      const int r = below ? c0 + w1 + t : 0;
      const double *src = below ? T + ix(c0, ld) + r : T + ix(sh.q1[t - nbelow], ld) + c0;
      const size_t stride = below ? (size_t)ld : 1;
#pragma unroll
      for (int u = 0; u < kIb; ++u) x[u] = (u < ne_t) ? src[u * stride] : 0.0;
      const int fl = row_solve_scale<kIb>(x, ne_t, Tb, ld, tb, sh.dinv1, inv_u);
      if (below) {
#pragma unroll
        for (int u = 0; u < kIb; ++u)
          if (u < ne_t) T[ix(c0 + u, ld) + r] = x[u];
      }
      fail = min(fail, fl);
    }
    atomicMin(&sh.nmin, fail);
  }
  __syncthreads();
  int nelim = sh.nmin;
  if (ne_t > 0 && nelim > 0 && tb[nelim - 1] == 2) --nelim;  // a 2x2 never splits
  // 5. restore the failed columns [nelim, w1) from the backup (permuted)
  if (nelim < w1) {
    for (int s2 = nelim; s2 < w1; ++s2) {
      double *col = T + ix(c0 + s2, ld);
      const int b2 = sh.lpc1[s2];
      for (int s1 = s2 + threadIdx.x; s1 < w1; s1 += blockDim.x) {
        const int a1 = sh.lpc1[s1];
        col[c0 + s1] = (a1 >= b2) ? sh.bk1[b2 * kNb + c0 + a1] : sh.bk1[a1 * kNb + c0 + b2];
      }
      for (int r = c0 + w1 + threadIdx.x; r < w; r += blockDim.x) col[r] = sh.bk1[b2 * kNb + r];
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int s2 = nelim; s2 < w1; ++s2) tags[c0 + s2] = 0;
  }
  __syncthreads();
  if (nelim > 0) {
    // ApplyT, final: the failed columns' L rows for the accepted pivots
    for (int t = threadIdx.x; t < nq; t += blockDim.x) {
      double x[kIb];
      double *src = T + ix(sh.q1[t], ld) + c0;
#pragma unroll
      for (int u = 0; u < kIb; ++u) x[u] = (u < nelim) ? src[u] : 0.0;
      row_solve_scale<kIb>(x, nelim, Tb, ld, tb, sh.dinv1, inv_u);
#pragma unroll
      for (int u = 0; u < kIb; ++u)
        if (u < nelim) src[u] = x[u];
    }
    // UpdateNN: W = (L D)^T of the columns [e0, w) into their strict upper
    // triangle rows [c0, c0 + nelim)
    const int e0 = c0 + nelim;
    for (int col = e0 + threadIdx.x; col < w; col += blockDim.x) {
      for (int t = 0; t < nelim; ++t) {
        const double l0 = T[ix(c0 + t, ld) + col];
        if (tb[t] == 2) {
          const double l1 = T[ix(c0 + t + 1, ld) + col];
          T[ix(col, ld) + c0 + t] = fma(l1, Tb[ix(t, ld) + t + 1], __dmul_rn(l0, Tb[ix(t, ld) + t]));
          T[ix(col, ld) + c0 + t + 1] = fma(l0, Tb[ix(t, ld) + t + 1], __dmul_rn(l1, Tb[ix(t + 1, ld) + t + 1]));
          ++t;
        } else {
          T[ix(col, ld) + c0 + t] = __dmul_rn(l0, Tb[ix(t, ld) + t]);
        }
      }
    }
    __syncthreads();
    for (int cj = e0 + (threadIdx.x >> 5); cj < w; cj += (blockDim.x >> 5)) {
      for (int ri = cj + (threadIdx.x & 31); ri < w; ri += 32) {
        double c = T[ix(cj, ld) + ri];
        for (int p = 0; p < nelim; ++p) {
          const double bw = T[ix(cj, ld) + c0 + p];
          if (bw != 0.0) c = fma(-T[ix(c0 + p, ld) + ri], bw, c);
        }
        T[ix(cj, ld) + ri] = c;
      }
    }
    // UpdateNT / TN: the earlier failed columns, tile rows [e0, w) and their
    // block among themselves; each entry one chain from zero, then one
    // subtraction
    for (int jq = 0; jq < nq; ++jq) {
      const int qj = sh.q1[jq];
      const double *lq = T + ix(qj, ld) + c0;  // the column's L row for the pivots
      for (int r = e0 + threadIdx.x; r < w; r += blockDim.x) {
        double acc = 0.0;
        for (int p = 0; p < nelim; ++p) {
          const double bw = (tb[p] == -1) ? ld_of(Tb, ld, tb, p, lq[p - 1], lq[p]) : ld_of(Tb, ld, tb, p, lq[p], tb[p] == 2 ? lq[p + 1] : 0.0);
          if (bw != 0.0) acc = fma(T[ix(c0 + p, ld) + r], bw, acc);
        }
        T[ix(qj, ld) + r] = __dsub_rn(T[ix(qj, ld) + r], acc);
      }
      for (int iq = jq + threadIdx.x; iq < nq; iq += blockDim.x) {
        const int qi = sh.q1[iq];
        const double *li = T + ix(qi, ld) + c0;
        double acc = 0.0;
        for (int p = 0; p < nelim; ++p) {
          const double bw = (tb[p] == -1) ? ld_of(Tb, ld, tb, p, lq[p - 1], lq[p]) : ld_of(Tb, ld, tb, p, lq[p], tb[p] == 2 ? lq[p + 1] : 0.0);
          if (bw != 0.0) acc = fma(li[p], bw, acc);
        }
        T[ix(qj, ld) + qi] = __dsub_rn(T[ix(qj, ld) + qi], acc);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int s = nelim; s < w1; ++s) sh.q1[sh.nq1++] = c0 + s;
  }
  __syncthreads();
  return nelim;
}

// Moves the failed columns behind the eliminated ones, eliminated order
// kept (ldlt_aptp.cpp:603-614), on an m x m view.
static __device__ void cta_compact(double *A, int ld, int m, int ne, int8_t *tags, int *rows, int *lp, int *loc) {
  int dst = 0;
  for (int src = 0; src < ne; ++src) {
    if (tags[src] == 0) continue;
    if (src != dst) cta_swap(A, ld, m, dst, src, tags, rows, lp, loc);
    ++dst;
  }
  __syncthreads();
}

// The diagonal tile (w x w at T): the inner sweep, then complete pivoting
// on what failed inside it (ldlt_aptp.cpp:335-350). lp: the tile's
// permutation record. Returns the tile's pivots.
static __device__ int tile_factor(double *T, int ld, int w, int8_t *tags, int *rows, int *lp, int *loc, double inv_u,
                           double small, TileShared &sh) {
  if (w <= kIb) return cta_complete(T, ld, w, tags, rows, lp, loc, inv_u, small, sh);
  for (int t = threadIdx.x; t < w; t += blockDim.x) {
    lp[t] = t;
    tags[t] = 0;
  }
  if (threadIdx.x == 0) sh.nq1 = 0;
  __syncthreads();
  int ne1 = 0;
  for (int c0 = 0; c0 < w; c0 += kIb) ne1 += tile_inner_block(T, ld, w, c0, min(kIb, w - c0), tags, rows, lp, loc,
                                                             inv_u, small, sh);
  if (ne1 < w) cta_compact(T, ld, w, w, tags, rows, lp, loc);
  if (ne1 < w) {
    const int n2 = w - ne1;
    const int ne2 = cta_complete(T + ix(ne1, ld) + ne1, ld, n2, tags + ne1, rows + ne1, sh.cp_lp,
                                 loc ? loc + ne1 : nullptr, inv_u, small, sh);
    if (!cta_identity(sh.cp_lp, n2)) {
      cta_permute_rows(T, ld, ne1, ne1, n2, sh.cp_lp);
      if ((int)threadIdx.x < n2) sh.itmp[threadIdx.x] = lp[ne1 + sh.cp_lp[threadIdx.x]];
      __syncthreads();
      if ((int)threadIdx.x < n2) lp[ne1 + threadIdx.x] = sh.itmp[threadIdx.x];
      __syncthreads();
    }
    ne1 += ne2;
  }
  return ne1;
}

}  // namespace aptp
}  // namespace smfg
