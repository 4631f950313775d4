/* Test infrastructure (the oracle). A plain-C restatement of the reference
 * smf numeric phase, written from the reference's algorithm; it is only ever
 * the checker of the CUDA engine (tests/, smoke(), bench.py's CPU-baseline
 * leg), never the thing measured or shipped.
 *
 * Every operation on a front entry follows the reference's order and
 * rounding: the pivot kernels multiply, then add or subtract (no FMA, as
 * ldlt_kernel.cpp is built with -ffp-contract=off; this file too), while the
 * GEMM steps of the deferred and Schur updates are fused multiply-adds (the
 * reference's portable BLAS loops are contracted by GCC's C++ default). For
 * the reference built with those loops (oracle/Makefile) the factor is then
 * bit for bit the reference's:
 *   process_front            solver/src/multifrontal_serial.cpp:472-1035
 *   ldlt_factor_front        solver/src/ldlt_kernel.cpp:970-1139
 *   select_pivot             solver/src/ldlt_kernel.cpp:127-275
 *   two_by_two_ok            solver/src/ldlt_kernel.cpp:97-122
 *   sym_swap                 solver/src/ldlt_kernel.cpp:333-347
 *   eliminate_1x1 / _2x2     solver/src/ldlt_kernel.cpp:352-545
 *   apply_pivot              solver/src/ldlt_kernel.cpp:666-698
 *   deferred_update          solver/src/ldlt_kernel.cpp:705-761
 *   fill_ld_column / schur   solver/src/ldlt_kernel.cpp:764-933
 *   portable GEMM loops      solver/src/dense_kernel_lapack.cpp:182-234
 *   add_inertia_2x2          solver/src/dense_indef.cpp:52-83
 *   ldlt_aptp_front          solver/src/ldlt_aptp.cpp:1-751 (deterministic
 *                            mode's kernel on indefinite fronts of >= 512 rows)
 * Not restated: static pivoting, delay budgets and the banded SPD path (tests
 * use configurations that do not reach them).
 */
#include "mf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define WEAK_PIVOT_RATIO 1e-6 /* kWeakPivotRatio, ldlt_kernel.hpp:100 */

static int is_fin(double v) { return isfinite(v); }
static double max3(double a, double b, double c) {
  double m = a;
  if (m < b) m = b;
  if (m < c) m = c;
  return m;
}
static double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */

typedef struct { int kind, a, b; } pchoice;

static double sym_at(const double *F, int ld, int i, int j) {
  return (i >= j) ? F[(size_t)j * ld + i] : F[(size_t)i * ld + j];
}

static int two_by_two_ok(const double *F, int ld, int f, int cand, int r, const double *col,
                         const double *col_r, double m2, double off1, int ext0,
                         const mfo_params *prm, double *growth) {
  const double d00 = col[cand];
  const double d10 = sym_at(F, ld, r, cand);
  const double d11 = col_r[r];
  const double s2 = max3(fabs(d00), fabs(d10), fabs(d11));
  if (!(s2 >= prm->eff_small) || !is_fin(s2)) return 0;
  const double a = d00 / s2, b = d10 / s2, c = d11 / s2;
  const double det_s = a * c - b * b;
  if (!(fabs(det_s) > prm->small_pivot)) return 0;
  double off0 = m2;
  for (int i = ext0; i < f; ++i) off0 = dmax(off0, fabs(col[i]));
  double g = 0.0;
  if (off0 > 0.0 || off1 > 0.0) {
    const double bound0 = (fabs(c) * off0 + fabs(b) * off1) / s2;
    const double bound1 = (fabs(b) * off0 + fabs(a) * off1) / s2;
    if (prm->u * dmax(bound0, bound1) > fabs(det_s)) return 0;
    g = dmax(bound0, bound1) / fabs(det_s);
  }
  *growth = g;
  return 1;
}

static pchoice select_pivot(const double *F, int ld, int f, int k, int num_elig, int limit,
                            const mfo_params *prm) {
  pchoice none = {0, -1, -1};
  if (prm->posdef) {
    const double d = F[(size_t)k * ld + k];
    if (d > 0.0 && is_fin(d)) { pchoice p1 = {1, k, -1}; return p1; }
    return none;
  }
  if (k < limit) {
    const double *col0 = F + (size_t)k * ld;
    const double a0 = fabs(col0[k]);
    if (a0 >= prm->eff_small) {
      double colmax = 0.0;
      for (int i = k + 1; i < f; ++i) {
        const double v = fabs(col0[i]);
        if (v > colmax) colmax = v;
      }
      if (!(prm->u * colmax > a0) && !(a0 < WEAK_PIVOT_RATIO * colmax)) {
        pchoice p1 = {1, k, -1};
        return p1;
      }
    }
  }
  for (int cand = k; cand < limit; ++cand) {
    const double *col = F + (size_t)cand * ld;
    const double a_cand = fabs(col[cand]);
    double m1 = 0.0, m2 = 0.0;
    int r_best = -1;
    for (int i = k; i < cand; ++i) {
      const double v = fabs(F[(size_t)i * ld + cand]);
      if (v > m1) { m2 = m1; m1 = v; r_best = i; }
      else if (v > m2) m2 = v;
    }
    for (int i = cand + 1; i < num_elig; ++i) {
      const double v = fabs(col[i]);
      if (v > m1) { m2 = m1; m1 = v; r_best = i; }
      else if (v > m2) m2 = v;
    }
    const int ext0 = num_elig > cand + 1 ? num_elig : cand + 1;
    int weak_1x1 = 0;
    double weak_growth = 0.0;
    if (a_cand >= prm->eff_small && !(prm->u * m1 > a_cand)) {
      int ok = 1;
      double colmax = m1;
      for (int i = ext0; i < f; ++i) {
        const double v = fabs(col[i]);
        if (prm->u * v > a_cand) { ok = 0; break; }
        colmax = dmax(colmax, v);
      }
      if (ok) {
        if (!(a_cand < WEAK_PIVOT_RATIO * colmax)) { pchoice p1 = {1, cand, -1}; return p1; }
        weak_1x1 = 1;
        weak_growth = colmax / a_cand;
      }
    }
    if (r_best < k || r_best >= limit || m1 <= 0.0) {
      if (weak_1x1) { pchoice p1 = {1, cand, -1}; return p1; }
      continue;
    }
    const double *col_r = F + (size_t)r_best * ld;
    double om2 = 0.0, off1 = 0.0;
    for (int i = k; i < r_best; ++i) {
      const double v = fabs(F[(size_t)i * ld + r_best]);
      om2 = dmax(om2, v);
      if (i != cand) off1 = dmax(off1, v);
    }
    for (int i = r_best + 1; i < f; ++i) {
      const double v = fabs(col_r[i]);
      om2 = dmax(om2, v);
      if (i != cand) off1 = dmax(off1, v);
    }
    double growth2 = 0.0;
    if (k + 1 < limit &&
        two_by_two_ok(F, ld, f, cand, r_best, col, col_r, m2, off1, ext0, prm, &growth2) &&
        (!weak_1x1 || growth2 < weak_growth)) {
      pchoice p2 = {2, cand, r_best};
      return p2;
    }
    if (weak_1x1) { pchoice p1 = {1, cand, -1}; return p1; }
    const double a_r = fabs(col_r[r_best]);
    if (a_r >= prm->eff_small && (om2 == 0.0 || a_r >= prm->u * om2)) {
      pchoice p1 = {1, r_best, -1};
      return p1;
    }
  }
  return none;
}

static void sym_swap(double *F, int ld, int f, int p, int q, int *rows, double *W, int w_cols) {
  if (p == q) return;
  if (p > q) { int t = p; p = q; q = t; }
  const size_t sf = (size_t)ld;
  double t;
#define SWP(x, y) (t = (x), (x) = (y), (y) = t)
  SWP(F[p * sf + p], F[q * sf + q]);
  for (int m = 0; m < p; ++m) SWP(F[m * sf + p], F[m * sf + q]);
  for (int m = p + 1; m < q; ++m) SWP(F[p * sf + m], F[m * sf + q]);
  for (int m = q + 1; m < f; ++m) SWP(F[p * sf + m], F[q * sf + m]);
  { int r = rows[p]; rows[p] = rows[q]; rows[q] = r; }
  for (int c = 0; c < w_cols; ++c) SWP(W[(size_t)c * f + p], W[(size_t)c * f + q]);
#undef SWP
}

/* eliminate_1x1: the per-entry operations of the reference (its 4-column
 * grouping and AVX lanes change no entry's operation sequence). */
static void eliminate_1x1(double *F, int f, int k, int ucol_end, double *W, int w_col) {
  const size_t sf = (size_t)f;
  double *ck = F + k * sf;
  const double inv_d = 1.0 / ck[k];
  if (W) {
    double *w = W + (size_t)w_col * sf;
    for (int i = k + 1; i < f; ++i) w[i] = ck[i];
  }
  for (int j = k + 1; j < ucol_end; ++j) {
    const double lj = ck[j] * inv_d;
    if (lj == 0.0) continue;
    double *cj = F + (size_t)j * sf;
    for (int i = j; i < f; ++i) cj[i] -= ck[i] * lj;
  }
  for (int i = k + 1; i < f; ++i) ck[i] *= inv_d;
}

static void inverse_2x2(double d00, double d10, double d11, double *i00, double *i10, double *i11) {
  const double s = max3(fabs(d00), fabs(d10), fabs(d11));
  const double a = d00 / s, b = d10 / s, c = d11 / s;
  const double inv = 1.0 / ((a * c - b * b) * s);
  *i00 = c * inv;
  *i10 = -b * inv;
  *i11 = a * inv;
}

static void eliminate_2x2(double *F, int f, int k, int ucol_end, double *W, int w_col) {
  const size_t sf = (size_t)f;
  double *c0 = F + k * sf, *c1 = F + (k + 1) * sf;
  double i00, i10, i11;
  inverse_2x2(c0[k], c0[k + 1], c1[k + 1], &i00, &i10, &i11);
  if (W) {
    double *w0 = W + (size_t)w_col * sf, *w1 = w0 + sf;
    for (int i = k + 2; i < f; ++i) { w0[i] = c0[i]; w1[i] = c1[i]; }
  }
  for (int j = k + 2; j < ucol_end; ++j) {
    const double a0 = c0[j], a1 = c1[j];
    const double l0 = i00 * a0 + i10 * a1;
    const double l1 = i10 * a0 + i11 * a1;
    if (l0 == 0.0 && l1 == 0.0) continue;
    double *d0 = F + (size_t)j * sf;
    for (int i = j; i < f; ++i) d0[i] -= c0[i] * l0 + c1[i] * l1;
  }
  for (int i = k + 2; i < f; ++i) {
    const double a0 = c0[i], a1 = c1[i];
    c0[i] = i00 * a0 + i10 * a1;
    c1[i] = i10 * a0 + i11 * a1;
  }
}

static void inertia_1x1(double d, double small, mfo_factor *o) {
  if (!is_fin(d) || fabs(d) < small) ++o->zero;
  else if (d > 0.0) ++o->pos;
  else ++o->neg;
}

static void inertia_2x2(double d00, double d10, double d11, double small, mfo_factor *o) {
  if (d10 == 0.0) {
    inertia_1x1(d00, small, o);
    inertia_1x1(d11, small, o);
    return;
  }
  const double s = max3(fabs(d00), fabs(d10), fabs(d11));
  double det_s = 0.0;
  if (is_fin(s) && s != 0.0) det_s = (d00 / s) * (d11 / s) - (d10 / s) * (d10 / s);
  if (s == 0.0 || !is_fin(det_s)) { o->zero += 2; return; }
  const double tr_s = (d00 / s) + (d11 / s);
  if (det_s < -small) { ++o->pos; ++o->neg; }
  else if (fabs(det_s) <= small) {
    ++o->zero;
    if (tr_s > small) ++o->pos;
    else if (tr_s < -small) ++o->neg;
    else ++o->zero;
  } else {
    if (tr_s > 0.0) o->pos += 2;
    else if (tr_s < 0.0) o->neg += 2;
    else o->zero += 2;
  }
}

static void apply_pivot(pchoice pc, double *F, int f, int *kp, int *rows, int8_t *tags, double *W,
                        int w_cols, int ucol_end, const mfo_params *prm, mfo_factor *o) {
  const size_t sf = (size_t)f;
  int k = *kp;
  if (pc.kind == 1) {
    sym_swap(F, f, f, k, pc.a, rows, W, w_cols);
    inertia_1x1(F[k * sf + k], prm->eff_small, o);
    tags[k] = 1;
    eliminate_1x1(F, f, k, ucol_end, W, w_cols);
    const double rem = (double)(f - (k + 1));
    o->flops += rem + rem * (rem + 1.0);
    *kp = k + 1;
    return;
  }
  int partner = pc.b;
  if (pc.a != k) {
    sym_swap(F, f, f, k, pc.a, rows, W, w_cols);
    if (partner == k) partner = pc.a;
  }
  if (partner != k + 1) sym_swap(F, f, f, k + 1, partner, rows, W, w_cols);
  inertia_2x2(F[k * sf + k], F[k * sf + k + 1], F[(k + 1) * sf + k + 1], prm->small_pivot, o);
  tags[k] = 2;
  tags[k + 1] = -1;
  eliminate_2x2(F, f, k, ucol_end, W, w_cols);
  const double rem = (double)(f - (k + 2));
  o->flops += 6.0 * rem + 2.0 * rem * (rem + 1.0);
  *kp = k + 2;
}

/* F[c0:f, c0:e] -= L[c0:f, p0:p1] W[c0:e, :]^T: per entry, pivots in order,
 * a zero W entry skipped (the portable dgemm / dgemmt loops,
 * dense_kernel_lapack.cpp:182-234). Those loops are compiled with GCC's
 * default C++ contraction, so each step is one fused multiply-add:
 * c = fma(-a, b, c). */
/* x rounded to `bits` significant bits, to nearest (ties to even). */
static double round_bits(double x, int bits) {
  if (x == 0.0 || !is_fin(x)) return x;
  int e;
  const double m = frexp(x, &e);
  return ldexp(nearbyint(ldexp(m, bits)), e - bits);
}

/* One entry of a split-product contraction: sum over t of a[t] b[t], each
 * operand split as hi + lo at `bits` bits, hi*hi + hi*lo + lo*hi summed in
 * FP32 in t order (the tensor-core accumulator). */
static double split_dot(const double *a, size_t as, const double *b, size_t bs, int n, int bits) {
  float acc = 0.0f;
  for (int t = 0; t < n; ++t) {
    const double x = a[(size_t)t * as], y = b[(size_t)t * bs];
    const double xh = round_bits(x, bits), xl = round_bits(x - xh, bits);
    const double yh = round_bits(y, bits), yl = round_bits(y - yh, bits);
    acc = acc + (float)(xh * yh);
    acc = acc + (float)(xh * yl);
    acc = acc + (float)(xl * yh);
  }
  return (double)acc;
}

static int g_mixed_bits = 0; /* set per front by ldlt_factor_front */

static void deferred_update(double *F, int f, int p0, int p1, int c0, int e, const double *W) {
  const int jb = p1 - p0;
  if (jb <= 0 || e - c0 <= 0) return;
  const size_t sf = (size_t)f;
  if (g_mixed_bits) {
    for (int j = c0; j < e; ++j)
      for (int i = j; i < f; ++i)
        F[(size_t)j * sf + i] -= split_dot(F + (size_t)p0 * sf + i, sf, W + j, sf, jb, g_mixed_bits);
    return;
  }
  for (int j = c0; j < e; ++j) {
    double *cj = F + (size_t)j * sf;
    for (int p = 0; p < jb; ++p) {
      const double b = W[(size_t)p * sf + j];
      if (b == 0.0) continue;
      const double *a = F + (size_t)(p0 + p) * sf;
      for (int i = j; i < f; ++i) cj[i] = fma(-a[i], b, cj[i]);
    }
  }
}

static double ld_entry(const double *F, int f, const int8_t *tags, int c, int i) {
  const size_t sf = (size_t)f;
  const double *Lc = F + (size_t)c * sf;
  if (tags[c] == 1) return Lc[i] * Lc[c];
  if (tags[c] == 2) return Lc[i] * Lc[c] + Lc[sf + i] * Lc[c + 1];
  if (tags[c] == -1) {
    const double *L0 = Lc - sf;
    return L0[i] * L0[c] + Lc[i] * Lc[c];
  }
  return 0.0;
}

/* F[e:f, e:f] -= L[e:f, p0:p] LD[e:f, p0:p]^T, LD = L D per fill_ld_column
 * (products rounded separately: ldlt_kernel.cpp is built without
 * contraction); the GEMM steps are fused as in deferred_update. */
static void schur_update(double *F, int f, int p0, int p, int e, const int8_t *tags, double *buf) {
  const int q = f - e;
  if (p <= p0 || q <= 0) return;
  const size_t sf = (size_t)f;
  const int kc = p - p0;
  for (int t = 0; t < kc; ++t)
    for (int i = 0; i < q; ++i) buf[(size_t)t * q + i] = ld_entry(F, f, tags, p0 + t, e + i);
  if (g_mixed_bits) {
    for (int j = 0; j < q; ++j)
      for (int i = j; i < q; ++i)
        F[(size_t)(e + j) * sf + e + i] -=
            split_dot(F + (size_t)p0 * sf + e + i, sf, buf + j, (size_t)q, kc, g_mixed_bits);
    return;
  }
  for (int j = 0; j < q; ++j) {
    double *cj = F + (size_t)(e + j) * sf + e;
    for (int t = 0; t < kc; ++t) {
      const double b = buf[(size_t)t * q + j];
      if (b == 0.0) continue;
      const double *a = F + (size_t)(p0 + t) * sf + e;
      for (int i = j; i < q; ++i) cj[i] = fma(-a[i], b, cj[i]);
    }
  }
}

/* ------------------------------------------------------------------------
 * A posteriori threshold pivoting (APTP), the dense kernel deterministic mode
 * runs on every indefinite front of at least 512 rows
 * (solver/src/ldlt_aptp.cpp:1-751; dispatch multifrontal_serial.cpp:796-821,
 * parallel/thread_plan.hpp:43-47; outer block top_tile_nb = 256,
 * control.hpp:638; inner block aptp_ib = 32, control.hpp:415). The tiled
 * variant (parallel/tile_tasks.cpp:256-351) splits the same steps into row
 * and column tiles; every entry takes the same operations in the same order,
 * so the untiled sweep is restated. ldlt_aptp.cpp is compiled with GCC's
 * default contraction: each a*b + c*d becomes fma(a, b, c*d), a*b - c*d
 * becomes fma(a, b, -(c*d)), and c -= a*b a single fma.
 * ------------------------------------------------------------------------ */
typedef struct {
  double inv_u, small;
  int nb, ib;
  double *bk[2];    /* block-column backups, per level */
  double *lt;       /* unit lower L of the tile (ld = block size) */
  double *ga, *gb, *gc;
  double *dinv;     /* 2 per pivot: inverse D, diagonal and off-diagonal */
  double *colbuf;
  int *top_lp, *q[2], *lpc[2], *cp_lp, *itmp;
} aptp_ctx;

typedef struct {
  double *A;
  int ld, m, ne, level, bs;
  int8_t *tags;
  int *rows, *lp, *Q;
  int nq, num_elim;
} aptp_sweep;

static size_t ix(int j, int ld) { return (size_t)j * (size_t)ld; }

/* symmetric transposition of view positions p and q (ldlt_aptp.cpp:67-80) */
static void ap_swap(double *A, int ld, int m, int p, int q, int8_t *tags, int *rows, int *lp) {
  if (p == q) return;
  if (p > q) { const int t = p; p = q; q = t; }
  double t;
#define SW(x, y) (t = (x), (x) = (y), (y) = t)
  SW(A[ix(p, ld) + p], A[ix(q, ld) + q]);
  for (int c = 0; c < p; ++c) SW(A[ix(c, ld) + p], A[ix(c, ld) + q]);
  for (int c = p + 1; c < q; ++c) SW(A[ix(p, ld) + c], A[ix(c, ld) + q]);
  for (int r = q + 1; r < m; ++r) SW(A[ix(p, ld) + r], A[ix(q, ld) + r]);
#undef SW
  { const int8_t u = tags[p]; tags[p] = tags[q]; tags[q] = u; }
  { const int u = rows[p]; rows[p] = rows[q]; rows[q] = u; }
  { const int u = lp[p]; lp[p] = lp[q]; lp[q] = u; }
}

/* inverse of the 2x2 pivot, scaled by its largest entry (ldlt_aptp.cpp:83-93) */
static void ap_inv2(double d00, double d10, double d11, double *i00, double *i10, double *i11) {
  const double s = max3(fabs(d00), fabs(d10), fabs(d11));
  const double a = d00 / s, b = d10 / s, c = d11 / s;
  const double inv = 1.0 / (fma(a, c, -(b * b)) * s);
  *i00 = c * inv;
  *i10 = -b * inv;
  *i11 = a * inv;
}

static double ap_sym(const double *A, int ld, int i, int j) {
  return (i >= j) ? A[ix(j, ld) + i] : A[ix(i, ld) + j];
}

static int ap_lok(double l, double inv_u) { return fabs(l) <= inv_u; }

/* complete pivoting on an n x n view (ldlt_aptp.cpp:101-210): returns the
 * pivots taken; stops at a remaining block below `small` or at a pivot that
 * would put an |l| > 1/u into the view */
static int ap_complete(double *A, int ld, int n, int8_t *tags, int *rows, int *lp,
                       const aptp_ctx *cx) {
  for (int t = 0; t < n; ++t) { lp[t] = t; tags[t] = 0; }
  int k = 0;
  while (k < n) {
    double amax = -1.0;
    int bi = -1, bj = -1;
    for (int j = k; j < n; ++j)
      for (int i = j; i < n; ++i) {
        const double v = fabs(A[ix(j, ld) + i]);
        if (v > amax) { amax = v; bi = i; bj = j; }
      }
    if (!(amax >= cx->small) || !is_fin(amax)) break;
    int kind = 1, a = bj, b = -1;
    if (bi != bj) {
      const double amm = A[ix(bj, ld) + bj], att = A[ix(bi, ld) + bi], amt = A[ix(bj, ld) + bi];
      const double delta = fma(amm, att, -(amt * amt));
      if (fabs(delta) >= 0.5 * amt * amt) { kind = 2; b = bi; }
      else a = (fabs(att) > fabs(amm)) ? bi : bj;
    }
    int ok = 1;
    if (kind == 1) {
      const double lim = cx->inv_u * fabs(A[ix(a, ld) + a]);
      for (int r = k; r < n && ok; ++r)
        if (r != a && !(fabs(ap_sym(A, ld, r, a)) <= lim)) ok = 0;
    } else {
      double i00, i10, i11;
      ap_inv2(A[ix(a, ld) + a], A[ix(a, ld) + b], A[ix(b, ld) + b], &i00, &i10, &i11);
      for (int r = k; r < n && ok; ++r) {
        if (r == a || r == b) continue;
        const double x0 = ap_sym(A, ld, r, a), x1 = ap_sym(A, ld, r, b);
        if (!ap_lok(fma(i00, x0, i10 * x1), cx->inv_u) || !ap_lok(fma(i10, x0, i11 * x1), cx->inv_u)) ok = 0;
      }
    }
    if (!ok) break;
    if (kind == 1) {
      ap_swap(A, ld, n, k, a, tags, rows, lp);
      double *ck = A + ix(k, ld);
      const double inv_d = 1.0 / ck[k];
      for (int j = k + 1; j < n; ++j) {
        const double lj = ck[j] * inv_d;
        if (lj == 0.0) continue;
        double *cj = A + ix(j, ld);
        for (int i = j; i < n; ++i) cj[i] = fma(-ck[i], lj, cj[i]);
      }
      for (int i = k + 1; i < n; ++i) ck[i] *= inv_d;
      tags[k] = 1;
      k += 1;
    } else {
      int partner = b;
      if (a != k) {
        ap_swap(A, ld, n, k, a, tags, rows, lp);
        if (partner == k) partner = a;
      }
      if (partner != k + 1) ap_swap(A, ld, n, k + 1, partner, tags, rows, lp);
      double *c0 = A + ix(k, ld), *c1 = A + ix(k + 1, ld);
      double i00, i10, i11;
      ap_inv2(c0[k], c0[k + 1], c1[k + 1], &i00, &i10, &i11);
      for (int j = k + 2; j < n; ++j) {
        const double a0 = c0[j], a1 = c1[j];
        const double l0 = fma(i00, a0, i10 * a1), l1 = fma(i10, a0, i11 * a1);
        if (l0 == 0.0 && l1 == 0.0) continue;
        double *cj = A + ix(j, ld);
        for (int i = j; i < n; ++i) cj[i] = cj[i] - fma(c0[i], l0, c1[i] * l1);
      }
      for (int i = k + 2; i < n; ++i) {
        const double a0 = c0[i], a1 = c1[i];
        c0[i] = fma(i00, a0, i10 * a1);
        c1[i] = fma(i10, a0, i11 * a1);
      }
      tags[k] = 2;
      tags[k + 1] = -1;
      k += 2;
    }
  }
  return k;
}

/* rows [r0, r0 + w) of columns [0, ncols): new row r0 + t takes old row
 * r0 + perm[t] (ldlt_aptp.cpp:214-221) */
static void ap_permute_rows(double *A, int ld, int ncols, int r0, int w, const int *perm, double *buf) {
  for (int c = 0; c < ncols; ++c) {
    double *col = A + ix(c, ld) + r0;
    for (int t = 0; t < w; ++t) buf[t] = col[perm[t]];
    memcpy(col, buf, sizeof(double) * (size_t)w);
  }
}

static int ap_identity(const int *perm, int w) {
  for (int t = 0; t < w; ++t)
    if (perm[t] != t) return 0;
  return 1;
}

/* L = X D^-1 in place, pivot by pivot; the start of the first pivot with an
 * |l| > 1/u in these rows, or k (ldlt_aptp.cpp:232-265) */
static int ap_scale_check(double *X, int nrows, int ldx, int k, const int8_t *tags, const double *dinv,
                          double inv_u) {
  for (int t = 0; t < k; ++t) {
    double *x0 = X + ix(t, ldx);
    if (tags[t] == 2) {
      double *x1 = x0 + ldx;
      const double i00 = dinv[2 * t], i10 = dinv[2 * t + 1], i11 = dinv[2 * (t + 1)];
      int ok = 1;
      for (int r = 0; r < nrows; ++r) {
        const double a0 = x0[r], a1 = x1[r];
        const double l0 = fma(i00, a0, i10 * a1), l1 = fma(i10, a0, i11 * a1);
        x0[r] = l0;
        x1[r] = l1;
        ok = ok && ap_lok(l0, inv_u) && ap_lok(l1, inv_u);
      }
      if (!ok) return t;
      ++t;
    } else {
      const double id = dinv[2 * t];
      int ok = 1;
      for (int r = 0; r < nrows; ++r) {
        const double l = x0[r] * id;
        x0[r] = l;
        ok = ok && ap_lok(l, inv_u);
      }
      if (!ok) return t;
    }
  }
  return k;
}

/* out[t] = (L D)(row, t) for the pivots [0, k) of the tile (D inline in the
 * tile) (ldlt_aptp.cpp:270-287) */
static void ap_row_times_d(const double *lrow, size_t stride, int k, const double *T, int ld,
                           const int8_t *tags, double *out, size_t ostride) {
  for (int t = 0; t < k; ++t) {
    const double d00 = T[ix(t, ld) + t];
    if (tags[t] == 2) {
      const double d10 = T[ix(t, ld) + t + 1], d11 = T[ix(t + 1, ld) + t + 1];
      const double l0 = lrow[t * stride], l1 = lrow[(t + 1) * stride];
      /* the fused forms GCC gives this function where it is inlined (found
       * by comparing against the reference bit for bit): the first output
       * fuses its second product, the second its first */
      out[t * ostride] = fma(l1, d10, l0 * d00);
      out[(t + 1) * ostride] = fma(l0, d10, l1 * d11);
      ++t;
    } else {
      out[t * ostride] = lrow[t * stride] * d00;
    }
  }
}

/* X := X L^-T for the k x k unit lower L: column by column, each entry one
 * fused chain over the earlier columns in order, a zero L entry skipped (the
 * blocked TRSM + GEMM of ldlt_aptp.cpp:292-304 over the portable loops,
 * dense_kernel_lapack.cpp:68-84 and :182-203, reduces to this chain). */
static void ap_trsm(double *X, int nrows, int k, const double *L, int ldl, int ldx) {
  for (int j = 0; j < k; ++j) {
    double *xj = X + ix(j, ldx);
    for (int p = 0; p < j; ++p) {
      const double l = L[ix(p, ldl) + j];
      if (l == 0.0) continue;
      const double *xp = X + ix(p, ldx);
      for (int i = 0; i < nrows; ++i) xj[i] = fma(-xp[i], l, xj[i]);
    }
  }
}

/* C[m x n] (ld ldc) -= A[m x k] B^T-ish product where the multiplier of
 * column p for output column j is b(j, p): the portable dgemm / dgemmt loops
 * with alpha = -1, beta = 1 (dense_kernel_lapack.cpp:159-234). lower: only
 * rows i >= j of each column. */
static void ap_gemm_sub(double *C, int m, int n, int k, const double *A, int lda, const double *B,
                        size_t bj_stride, size_t bp_stride, int ldc, int lower) {
  for (int j = 0; j < n; ++j) {
    double *cj = C + ix(j, ldc);
    for (int p = 0; p < k; ++p) {
      const double b = B[j * bj_stride + p * bp_stride];
      if (b == 0.0) continue;
      const double *ap = A + ix(p, lda);
      for (int i = lower ? j : 0; i < m; ++i) cj[i] = fma(-ap[i], b, cj[i]);
    }
  }
}

/* C = A B^T (beta 0, alpha 1): each entry a fused chain from zero over p,
 * a zero B entry skipped (smf_dgemm_nt, dense_kernel_lapack.cpp:182-203) */
static void ap_gemm_nt(double *C, int m, int n, int k, const double *A, int lda, const double *B, int ldb,
                       int ldc) {
  for (int j = 0; j < n; ++j) {
    double *cj = C + ix(j, ldc);
    for (int i = 0; i < m; ++i) cj[i] = 0.0;
    for (int p = 0; p < k; ++p) {
      const double b = B[ix(p, ldb) + j];
      if (b == 0.0) continue;
      const double *ap = A + ix(p, lda);
      for (int i = 0; i < m; ++i) cj[i] = fma(ap[i], b, cj[i]);
    }
  }
}

static int ap_factor_tile(double *A, int ld, int w, int8_t *tags, int *rows, int *lp, aptp_ctx *cx);

/* steps 1-4 of a block column (ldlt_aptp.cpp:390-449): backup, factor the
 * diagonal tile, apply its permutation, L_t and D^-1; returns the tile's
 * pivots */
static int ap_block_factor(aptp_sweep *sw, int c0, int w, aptp_ctx *cx) {
  double *A = sw->A;
  const int ld = sw->ld, m = sw->m, bs = sw->bs;
  int8_t *tags = sw->tags;
  int *lp = sw->lp;
  double *bk = cx->bk[sw->level];
  int *lpc = cx->lpc[sw->level];
  const int ldb = m - c0, rb = m - c0 - w;
  for (int t = 0; t < w; ++t)
    memcpy(bk + ix(t, ldb) + t, A + ix(c0 + t, ld) + c0 + t, sizeof(double) * (size_t)(m - c0 - t));
  double *T = A + ix(c0, ld) + c0;
  const int ne_t = sw->level == 0 ? ap_factor_tile(T, ld, w, tags + c0, sw->rows + c0, lpc, cx)
                                  : ap_complete(T, ld, w, tags + c0, sw->rows + c0, lpc, cx);
  if (!ap_identity(lpc, w)) {
    ap_permute_rows(A, ld, c0, c0, w, lpc, cx->colbuf);
    for (int t = 0; t < w; ++t)
      memcpy(A + ix(c0 + t, ld) + c0 + w, bk + ix(lpc[t], ldb) + w, sizeof(double) * (size_t)rb);
    for (int t = 0; t < w; ++t) cx->itmp[t] = lp[c0 + lpc[t]];
    memcpy(lp + c0, cx->itmp, sizeof(int) * (size_t)w);
  }
  if (ne_t > 0) {
    double *lt = cx->lt;
    for (int j = 0; j < ne_t; ++j) {
      double *lj = lt + ix(j, bs);
      lj[j] = 1.0;
      const double *tj = T + ix(j, ld);
      for (int i = j + 1; i < ne_t; ++i) lj[i] = tj[i];
    }
    for (int j = 0; j < ne_t; ++j) {
      const double *tj = T + ix(j, ld);
      if (tags[c0 + j] == 2) {
        lt[ix(j, bs) + j + 1] = 0.0;
        double i00, i10, i11;
        ap_inv2(tj[j], tj[j + 1], T[ix(j + 1, ld) + j + 1], &i00, &i10, &i11);
        cx->dinv[2 * j] = i00;
        cx->dinv[2 * j + 1] = i10;
        cx->dinv[2 * (j + 1)] = i11;
        cx->dinv[2 * (j + 1) + 1] = 0.0;
        ++j;
      } else {
        cx->dinv[2 * j] = 1.0 / tj[j];
        cx->dinv[2 * j + 1] = 0.0;
      }
    }
  }
  return ne_t;
}

/* ApplyN on rows [r0, r1) (ldlt_aptp.cpp:451-456) */
static int ap_apply_n(const aptp_sweep *sw, int c0, int ne_t, int r0, int r1, const aptp_ctx *cx) {
  if (ne_t <= 0 || r1 <= r0) return ne_t;
  double *X = sw->A + ix(c0, sw->ld) + r0;
  ap_trsm(X, r1 - r0, ne_t, cx->lt, sw->bs, sw->ld);
  return ap_scale_check(X, r1 - r0, sw->ld, ne_t, sw->tags + c0, cx->dinv, cx->inv_u);
}

/* ApplyT, restore, UpdateNN (all eligible columns), UpdateNT / TN
 * (ldlt_aptp.cpp:458-588) */
static int ap_block_finish(aptp_sweep *sw, int c0, int w, int ne_t, int nelim, aptp_ctx *cx) {
  double *A = sw->A;
  const int ld = sw->ld, m = sw->m, ne = sw->ne, bs = sw->bs;
  int8_t *tags = sw->tags;
  const int *Q = sw->Q;
  const int nq = sw->nq;
  double *bk = cx->bk[sw->level];
  const int *lpc = cx->lpc[sw->level];
  const int ldb = m - c0, rb = m - c0 - w;
  double *T = A + ix(c0, ld) + c0;
  if (ne_t > 0) {
    for (int i0 = 0; i0 < nq && nelim > 0; i0 += bs) {
      const int nc = (bs < nq - i0) ? bs : nq - i0;
      for (int t = 0; t < nelim; ++t)
        for (int ii = 0; ii < nc; ++ii) cx->ga[ix(t, bs) + ii] = A[ix(Q[i0 + ii], ld) + c0 + t];
      ap_trsm(cx->ga, nc, nelim, cx->lt, bs, bs);
      nelim = ap_scale_check(cx->ga, nc, bs, nelim, tags + c0, cx->dinv, cx->inv_u);
    }
    if (nelim > 0 && tags[c0 + nelim - 1] == 2) --nelim;
  }
  if (nelim < w) {
    for (int s2 = nelim; s2 < w; ++s2) {
      double *col = T + ix(s2, ld);
      for (int s1 = s2; s1 < w; ++s1) {
        const int a = lpc[s1], b = lpc[s2];
        col[s1] = (a >= b) ? bk[ix(b, ldb) + a] : bk[ix(a, ldb) + b];
      }
      memcpy(col + w, bk + ix(lpc[s2], ldb) + w, sizeof(double) * (size_t)rb);
      tags[c0 + s2] = 0;
    }
  }
  if (nelim > 0) {
    for (int i0 = 0; i0 < nq; i0 += bs) {
      const int nc = (bs < nq - i0) ? bs : nq - i0;
      if (nq > bs) {
        for (int t = 0; t < nelim; ++t)
          for (int ii = 0; ii < nc; ++ii) cx->ga[ix(t, bs) + ii] = A[ix(Q[i0 + ii], ld) + c0 + t];
        ap_trsm(cx->ga, nc, nelim, cx->lt, bs, bs);
        ap_scale_check(cx->ga, nc, bs, nelim, tags + c0, cx->dinv, cx->inv_u);
      }
      for (int t = 0; t < nelim; ++t)
        for (int ii = 0; ii < nc; ++ii) A[ix(Q[i0 + ii], ld) + c0 + t] = cx->ga[ix(t, bs) + ii];
    }
    /* UpdateNN: W = (L D)^T of the eligible columns [e0, ne) goes into the
     * strict upper triangle rows [c0, c0 + nelim) of those columns */
    const int e0 = c0 + nelim, msz = ne - e0;
    if (msz > 0) {
      for (int col = e0; col < ne; ++col)
        ap_row_times_d(A + ix(c0, ld) + col, (size_t)ld, nelim, T, ld, tags + c0, A + ix(col, ld) + c0, 1);
      const double *Wt = A + ix(e0, ld) + c0;
      ap_gemm_sub(A + ix(e0, ld) + e0, msz, msz, nelim, A + ix(c0, ld) + e0, ld, Wt, (size_t)ld, 1, ld, 1);
      if (m > ne)
        ap_gemm_sub(A + ix(e0, ld) + ne, m - ne, msz, nelim, A + ix(c0, ld) + ne, ld, Wt, (size_t)ld, 1, ld, 0);
    }
    /* UpdateNT / TN: the earlier failed columns, rows [e0, m) and their
     * block among themselves */
    const int mr = m - e0;
    for (int j0 = 0; j0 < nq; j0 += bs) {
      const int nj = (bs < nq - j0) ? bs : nq - j0;
      for (int jj = 0; jj < nj; ++jj)
        ap_row_times_d(A + ix(Q[j0 + jj], ld) + c0, 1, nelim, T, ld, tags + c0, cx->gb + jj, (size_t)bs);
      if (mr > 0) {
        double *Tm = bk;
        ap_gemm_nt(Tm, mr, nj, nelim, A + ix(c0, ld) + e0, ld, cx->gb, bs, mr);
        for (int jj = 0; jj < nj; ++jj) {
          double *dst = A + ix(Q[j0 + jj], ld) + e0;
          const double *src = Tm + ix(jj, mr);
          for (int r = 0; r < mr; ++r) dst[r] -= src[r];
        }
      }
      for (int i0 = j0; i0 < nq; i0 += bs) {
        const int ni = (bs < nq - i0) ? bs : nq - i0;
        for (int t = 0; t < nelim; ++t)
          for (int ii = 0; ii < ni; ++ii) cx->ga[ix(t, bs) + ii] = A[ix(Q[i0 + ii], ld) + c0 + t];
        ap_gemm_nt(cx->gc, ni, nj, nelim, cx->ga, bs, cx->gb, bs, bs);
        for (int jj = 0; jj < nj; ++jj) {
          const int qj = Q[j0 + jj];
          double *colq = A + ix(qj, ld);
          for (int ii = 0; ii < ni; ++ii) {
            const int qi = Q[i0 + ii];
            if (qi >= qj) colq[qi] -= cx->gc[ix(jj, bs) + ii];
          }
        }
      }
    }
  }
  sw->num_elim += nelim;
  for (int s = nelim; s < w; ++s) sw->Q[sw->nq++] = c0 + s;
  return nelim;
}

/* one sweep over the leading ne columns of the m x m view; level 0 the
 * front (block nb), level 1 a diagonal tile (block ib); then the failed
 * columns behind the pivots and, at the front level, the deferred update of
 * the non-eligible triangle (ldlt_aptp.cpp:317-330, :603-659) */
static int ap_sweep(double *A, int ld, int m, int ne, int level, int8_t *tags, int *rows, int *lp,
                    aptp_ctx *cx) {
  aptp_sweep sw;
  sw.A = A; sw.ld = ld; sw.m = m; sw.ne = ne; sw.level = level;
  sw.bs = level == 0 ? cx->nb : cx->ib;
  sw.tags = tags; sw.rows = rows; sw.lp = lp; sw.Q = cx->q[level];
  sw.nq = 0; sw.num_elim = 0;
  for (int t = 0; t < ne; ++t) { lp[t] = t; tags[t] = 0; }
  for (int c0 = 0; c0 < ne; c0 += sw.bs) {
    const int w = (sw.bs < ne - c0) ? sw.bs : ne - c0;
    const int ne_t = ap_block_factor(&sw, c0, w, cx);
    int nelim = ne_t;
    if (ne_t > 0 && m - c0 - w > 0) nelim = ap_apply_n(&sw, c0, ne_t, c0 + w, m, cx);
    ap_block_finish(&sw, c0, w, ne_t, nelim, cx);
  }
  if (sw.num_elim < sw.ne) {
    int dst = 0;
    for (int src = 0; src < sw.ne; ++src) {
      if (sw.tags[src] == 0) continue;
      if (src != dst) ap_swap(sw.A, sw.ld, sw.m, dst, src, sw.tags, sw.rows, sw.lp);
      ++dst;
    }
  }
  const int qn = sw.m - sw.ne, p = sw.num_elim;
  if (qn > 0 && p > 0) {
    for (int c = 0; c < p; ++c) {
      const double *Lc = A + ix(c, ld);
      if (tags[c] == 2) {
        const double *Lc1 = Lc + ld;
        const double d00 = Lc[c], d10 = Lc[c + 1], d11 = Lc1[c + 1];
        for (int i = ne; i < m; ++i) {
          A[ix(i, ld) + c] = fma(Lc[i], d00, Lc1[i] * d10);
          A[ix(i, ld) + c + 1] = fma(Lc[i], d10, Lc1[i] * d11);
        }
        ++c;
      } else {
        const double d = Lc[c];
        for (int i = ne; i < m; ++i) A[ix(i, ld) + c] = Lc[i] * d;
      }
    }
    ap_gemm_sub(A + ix(ne, ld) + ne, qn, qn, p, A + ne, ld, A + ix(ne, ld), (size_t)ld, 1, ld, 1);
  }
  return sw.num_elim;
}

/* diagonal tile of the outer sweep: the inner sweep (block ib), then
 * complete pivoting on what failed inside the tile (ldlt_aptp.cpp:335-350) */
static int ap_factor_tile(double *A, int ld, int w, int8_t *tags, int *rows, int *lp, aptp_ctx *cx) {
  if (w <= cx->ib) return ap_complete(A, ld, w, tags, rows, lp, cx);
  int ne1 = ap_sweep(A, ld, w, w, 1, tags, rows, lp, cx);
  if (ne1 < w) {
    const int n2 = w - ne1;
    int *lp2 = cx->cp_lp;
    const int ne2 = ap_complete(A + ix(ne1, ld) + ne1, ld, n2, tags + ne1, rows + ne1, lp2, cx);
    if (!ap_identity(lp2, n2)) {
      ap_permute_rows(A, ld, ne1, ne1, n2, lp2, cx->colbuf);
      for (int t = 0; t < n2; ++t) cx->itmp[t] = lp[ne1 + lp2[t]];
      memcpy(lp + ne1, cx->itmp, sizeof(int) * (size_t)n2);
    }
    ne1 += ne2;
  }
  return ne1;
}

/* ldlt_aptp_front (ldlt_aptp.cpp:728-749): returns the pivots eliminated;
 * inertia and flops added to o (front_result, :704-724: every pivot's
 * inertia against the effective small value) */
static int ldlt_aptp_front(double *F, int f, int num_elig, int *rows, const mfo_params *prm, int8_t *tags,
                           mfo_factor *o) {
  if (f <= 0 || num_elig <= 0) return 0;
  const int ne1 = num_elig > 1 ? num_elig : 1;
  int nb = prm->aptp_nb > 1 ? prm->aptp_nb : 1;
  if (nb > ne1) nb = ne1;
  int ib = prm->aptp_ib > 1 ? prm->aptp_ib : 1;
  if (ib > nb) ib = nb;
  aptp_ctx cx;
  cx.inv_u = 1.0 / prm->u;
  cx.small = prm->eff_small;
  cx.nb = nb;
  cx.ib = ib;
  const size_t sf = (size_t)f, snb = (size_t)nb, sib = (size_t)ib;
  double *mem = (double *)malloc(sizeof(double) * (sf * snb + snb * sib + 4 * snb * snb + 2 * snb + sf));
  int *imem = (int *)malloc(sizeof(int) * (2 * (size_t)ne1 + 4 * snb + sib));
  double *p = mem;
  cx.bk[0] = p; p += sf * snb;
  cx.bk[1] = p; p += snb * sib;
  cx.lt = p; p += snb * snb;
  cx.ga = p; p += snb * snb;
  cx.gb = p; p += snb * snb;
  cx.gc = p; p += snb * snb;
  cx.dinv = p; p += 2 * snb;
  cx.colbuf = p;
  int *ip = imem;
  cx.top_lp = ip; ip += ne1;
  cx.q[0] = ip; ip += ne1;
  cx.lpc[0] = ip; ip += nb;
  cx.q[1] = ip; ip += nb;
  cx.lpc[1] = ip; ip += ib;
  cx.cp_lp = ip; ip += nb;
  cx.itmp = ip;
  const int pe = ap_sweep(F, f, f, num_elig, 0, tags, rows, cx.top_lp, &cx);
  free(mem);
  free(imem);
  for (int k = 0; k < pe; ++k) {
    if (tags[k] == 2) {
      inertia_2x2(F[k * sf + k], F[k * sf + k + 1], F[(k + 1) * sf + k + 1], prm->eff_small, o);
      const double rem = (double)(f - (k + 2));
      o->flops += 6.0 * rem + 2.0 * rem * (rem + 1.0);
      ++k;
    } else {
      inertia_1x1(F[k * sf + k], prm->eff_small, o);
      const double rem = (double)(f - (k + 1));
      o->flops += rem + rem * (rem + 1.0);
    }
  }
  return pe;
}

/* ldlt_factor_front from column `first` (0, or the pivots an APTP sweep
 * took before it), no static pivoting. Returns the number of accepted pivots. */
static int ldlt_factor_front(double *F, int f, int num_elig, int *rows, const mfo_params *prm,
                             int8_t *tags, double *work, int first, mfo_factor *o) {
  int k = first;
  g_mixed_bits = (prm->mixed_bits > 0 && prm->mixed_min_front > 0 && f >= prm->mixed_min_front)
                     ? prm->mixed_bits : 0;
  if (f - first < prm->blocked_min_front || prm->nb <= 1) {
    while (k < num_elig) {
      pchoice pc = select_pivot(F, f, f, k, num_elig, num_elig, prm);
      if (pc.kind == 0) break;
      apply_pivot(pc, F, f, &k, rows, tags, NULL, 0, f, prm, o);
    }
    return k;
  }
  double *W = work; /* f x nb */
  const size_t sf = (size_t)f;
  if (!prm->posdef) {
    int live = num_elig, k_paired = -1;
    while (k < live) {
      const int ps = k;
      const int pl = (live < ps + prm->nb) ? live : ps + prm->nb;
      int stalled = 0;
      while (k < pl) {
        pchoice pc = select_pivot(F, f, f, k, num_elig, pl, prm);
        if (pc.kind == 0) { stalled = 1; break; }
        apply_pivot(pc, F, f, &k, rows, tags, W, k - ps, pl, prm, o);
      }
      deferred_update(F, f, ps, k, pl, num_elig, W);
      if (stalled && k != k_paired) {
        int order[128];
        int np = 0;
        const int max_pairs = (prm->nb / 2 < 64) ? prm->nb / 2 : 64;
        for (int pos = k; pos < pl && np / 2 < max_pairs; ++pos) {
          const double *col = F + (size_t)pos * sf;
          double in_max = 0.0;
          for (int i = k; i < pos; ++i) in_max = dmax(in_max, fabs(F[(size_t)i * sf + pos]));
          for (int i = pos + 1; i < pl; ++i) in_max = dmax(in_max, fabs(col[i]));
          double out_max = 0.0;
          int r = -1;
          for (int i = pl; i < num_elig; ++i) {
            const double v = fabs(col[i]);
            if (v > out_max) { out_max = v; r = i; }
          }
          if (r < 0 || !(out_max > in_max)) continue;
          int taken = 0;
          for (int t = 1; t < np; t += 2) taken = taken || order[t] == rows[r];
          if (taken) continue;
          order[np++] = rows[pos];
          order[np++] = rows[r];
        }
        if (np > 0) {
          for (int t = 0; t < np; ++t) {
            int qq = k + t;
            while (rows[qq] != order[t]) ++qq;
            sym_swap(F, f, f, k + t, qq, rows, NULL, 0);
          }
          live = (live > k + np) ? live : k + np;
          k_paired = k;
          continue;
        }
      }
      if (stalled) {
        const int m = pl - k;
        const int mv = (m < live - pl) ? m : live - pl;
        for (int t = 0; t < mv; ++t) sym_swap(F, f, f, k + t, live - mv + t, rows, NULL, 0);
        live -= m;
      }
    }
  }
  while (k < num_elig) {
    const int ps = k;
    const int pl = (num_elig < ps + prm->nb) ? num_elig : ps + prm->nb;
    int stalled = 0;
    while (k < pl) {
      pchoice pc = select_pivot(F, f, f, k, num_elig, pl, prm);
      if (pc.kind == 0) { stalled = 1; break; }
      apply_pivot(pc, F, f, &k, rows, tags, W, k - ps, pl, prm, o);
    }
    deferred_update(F, f, ps, k, pl, num_elig, W);
    if (stalled && k < num_elig) {
      const int ss = k;
      pchoice pc = select_pivot(F, f, f, k, num_elig, num_elig, prm);
      if (pc.kind == 0) break;
      apply_pivot(pc, F, f, &k, rows, tags, W, 0, ss, prm, o);
      deferred_update(F, f, ss, k, k, num_elig, W);
    }
  }
  schur_update(F, f, first, k, num_elig, tags, work);
  return k;
}

void mfo_factor_front(double *F, int f, int ne, int *rows, const mfo_params *prm, int8_t *tags,
                      int64_t *out) {
  mfo_factor o;
  memset(&o, 0, sizeof(o));
  double *work = (double *)malloc(sizeof(double) * ((size_t)f * (prm->nb + 2) + (size_t)f * f + 1));
  const int k = ldlt_factor_front(F, f, ne, rows, prm, tags, work, 0, &o);
  free(work);
  out[0] = o.pos;
  out[1] = o.neg;
  out[2] = o.zero;
  out[3] = k;
}

/* Test hook: the assembled front of one supernode, captured by the next
 * mfo_factorize before its kernel runs (for dense-kernel parity on real
 * fronts). */
static int g_cap_s = -1;
static double *g_cap_F = NULL;
static int64_t g_cap_cap = 0;
static int *g_cap_rows = NULL;
static int g_cap_info[2];

void mfo_capture_front(int s, double *F, int64_t cap, int *rows) {
  g_cap_s = s;
  g_cap_F = F;
  g_cap_cap = cap;
  g_cap_rows = rows;
  g_cap_info[0] = g_cap_info[1] = -1;
}

void mfo_captured_size(int *f, int *num_elig) {
  *f = g_cap_info[0];
  *num_elig = g_cap_info[1];
}

/* The APTP kernel alone on a dense front (tests): out[0..4] = eliminated,
 * failed, positive, negative, zero pivots. */
void mfo_aptp_front(double *F, int f, int ne, int *rows, const mfo_params *prm, int8_t *tags, int64_t *out) {
  mfo_factor o;
  memset(&o, 0, sizeof(o));
  const int pe = ldlt_aptp_front(F, f, ne, rows, prm, tags, &o);
  out[0] = pe;
  out[1] = ne - pe;
  out[2] = o.pos;
  out[3] = o.neg;
  out[4] = o.zero;
}

/* Deterministic mode's choice of the APTP kernel: plain threshold pivoting
 * on an indefinite front of at least aptp_min_rows realized rows, with
 * u >= kWeakPivotRatio (thread_plan.cpp:264-268, thread_plan.hpp:43-52) */
static int aptp_front(const mfo_params *prm, int f) {
  return prm->aptp_min_rows > 0 && !prm->posdef && f >= prm->aptp_min_rows && prm->u >= WEAK_PIVOT_RATIO;
}

int mfo_factorize(const mfo_analysis *a, const double *pv, const mfo_params *prm, mfo_factor *o) {
  const int n = a->n, ns = a->nsn;
  o->pos = o->neg = o->zero = o->delayed = o->two_by_two = o->max_front = o->aptp_failed = 0;
  o->flops = 0.0;
  o->status = 0;
  double **front = (double **)calloc((size_t)ns, sizeof(double *));
  int **frows = (int **)calloc((size_t)ns, sizeof(int *));
  int *fsz = (int *)calloc((size_t)ns, sizeof(int));
  int *acc = (int *)calloc((size_t)ns, sizeof(int));
  int *delayed = (int *)calloc((size_t)ns, sizeof(int));
  int *pos = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) pos[i] = -1;
  int64_t bo = 0, ro = 0, to = 0;
  for (int it = 0; it < ns && o->status == 0; ++it) {
    const int s = a->postorder[it];
    const int c0 = a->child_ptr[s], c1 = a->child_ptr[s + 1];
    const int fs = a->front_row_ptr[s + 1] - a->front_row_ptr[s];
    const int psym = a->sn_end[s] - a->sn_start[s];
    int nd = 0;
    for (int t = c0; t < c1; ++t) nd += delayed[a->child_idx[t]];
    const int f = nd + fs;
    int *rows = (int *)malloc(sizeof(int) * (size_t)(f > 0 ? f : 1));
    int ff = 0;
    for (int t = c0; t < c1; ++t) {
      const int c = a->child_idx[t];
      for (int r = 0; r < delayed[c]; ++r) {
        const int row = frows[c][acc[c] + r];
        rows[ff] = row;
        pos[row] = ff++;
      }
    }
    for (int t = 0; t < fs; ++t) {
      const int row = a->front_row_idx[a->front_row_ptr[s] + t];
      rows[ff] = row;
      pos[row] = ff++;
    }
    const int num_elig = nd + psym;
    double *F = (double *)calloc((size_t)f * f + 1, sizeof(double));
    /* original entries of the pivot columns */
    for (int j = a->sn_start[s]; j < a->sn_end[s]; ++j) {
      double *Fj = F + (size_t)pos[j] * f;
      for (int k = a->pcp[j]; k < a->pcp[j + 1]; ++k) Fj[pos[a->pri[k]]] += pv[k];
    }
    /* extend-add, children in child_idx order */
    for (int t = c0; t < c1; ++t) {
      const int c = a->child_idx[t];
      const int fc = fsz[c], pc = acc[c], q = fc - pc;
      if (q <= 0 || a->sn_parent[c] < 0) continue;
      const double *Fc = front[c];
      const int *cr = frows[c] + pc;
      for (int jj = 0; jj < q; ++jj) {
        const int lj = pos[cr[jj]];
        if (lj < 0) { o->status = 3; break; }
        for (int ii = jj; ii < q; ++ii) {
          const int li = pos[cr[ii]];
          const double v = Fc[(size_t)(pc + jj) * fc + (pc + ii)];
          if (li >= lj) F[(size_t)lj * f + li] += v;
          else F[(size_t)li * f + lj] += v;
        }
      }
    }
    if (s == g_cap_s) {
      g_cap_info[0] = f;
      g_cap_info[1] = num_elig;
      if ((int64_t)f * f <= g_cap_cap) {
        memcpy(g_cap_F, F, sizeof(double) * (size_t)f * f);
        memcpy(g_cap_rows, rows, sizeof(int) * (size_t)f);
      }
    }
    int8_t *tags = (int8_t *)calloc((size_t)(f > 0 ? f : 1), 1);
    double *work = (double *)malloc(sizeof(double) * ((size_t)f * (prm->nb + 2) + (size_t)f * f + 1));
    int p;
    if (aptp_front(prm, f)) {
      /* APTP, then the threshold kernel on the columns it failed (their
       * Schur state is current) (multifrontal_serial.cpp:796-821) */
      p = ldlt_aptp_front(F, f, num_elig, rows, prm, tags, o);
      o->aptp_failed += num_elig - p;
      if (p < num_elig) p = ldlt_factor_front(F, f, num_elig, rows, prm, tags, work, p, o);
    } else {
      p = ldlt_factor_front(F, f, num_elig, rows, prm, tags, work, 0, o);
    }
    free(work);
    if (f > o->max_front) o->max_front = f;
    const int is_root = a->sn_parent[s] < 0;
    if (prm->posdef && p < num_elig) { o->status = 1; free(tags); free(F); free(rows); break; }
    int p_store = p;
    if (is_root && p < num_elig) {
      for (int c = p; c < num_elig; ++c) tags[c] = 0;
      o->zero += num_elig - p;
      p_store = num_elig;
    }
    if (prm->posdef) {
      for (int c = 0; c < p_store; ++c) {
        double *Lc = F + (size_t)c * f;
        const double sd = sqrt(Lc[c]);
        for (int i = 0; i < c; ++i) Lc[i] = 0.0;
        Lc[c] = sd;
        for (int i = c + 1; i < f; ++i) Lc[i] *= sd;
      }
    } else {
      double d10 = 0.0;
      for (int c = 0; c < p_store; ++c) {
        double *Lc = F + (size_t)c * f;
        const int8_t tag = tags[c];
        if (tag == 0) {
          for (int i = c + 1; i < f; ++i) Lc[i] = 0.0;
          Lc[c] = 0.0;
        } else if (tag == 2) {
          ++o->two_by_two;
          if (!is_fin(Lc[c]) || !is_fin(Lc[c + 1]) || !is_fin(Lc[(size_t)f + c + 1])) o->status = 4;
          d10 = Lc[c + 1];
          Lc[c + 1] = 0.0;
        } else if (tag == 1) {
          if (!is_fin(Lc[c])) o->status = 4;
        }
        for (int i = 0; i < c; ++i) Lc[i] = 0.0;
        if (tag == -1) Lc[c - 1] = d10;
      }
    }
    o->f_out[s] = f;
    o->p_out[s] = p_store;
    o->blk_off[s] = bo;
    o->row_off[s] = ro;
    if (bo + (int64_t)f * p_store > o->blk_cap || ro + f > o->row_cap) { o->status = 3; }
    else {
      memcpy(o->blocks + bo, F, sizeof(double) * (size_t)f * p_store);
      memcpy(o->rows + ro, rows, sizeof(int) * (size_t)f);
      if (!prm->posdef && o->tags) memcpy(o->tags + to, tags, (size_t)p_store);
    }
    bo += (int64_t)f * p_store;
    ro += f;
    to += p_store;
    free(tags);
    fsz[s] = f;
    acc[s] = p;
    frows[s] = rows;
    front[s] = F;
    delayed[s] = is_root ? 0 : num_elig - p;
    o->delayed += delayed[s];
    for (int t = 0; t < f; ++t) pos[rows[t]] = -1;
    /* children's fronts are consumed */
    for (int t = c0; t < c1; ++t) {
      const int c = a->child_idx[t];
      free(front[c]);
      front[c] = NULL;
    }
  }
  if (o->status == 0 && o->zero > 0) o->status = 2;
  for (int s = 0; s < ns; ++s) { free(front[s]); free(frows[s]); }
  free(front); free(frows); free(fsz); free(acc); free(delayed); free(pos);
  return o->status;
}

/* Forward, diagonal and backward solves on the stored blocks (in place on x,
 * new numbering). solve_forward.cpp:116-293, solve_diag.cpp:49-123,
 * solve_backward.cpp:135-350 compute the same quantities. */
void mfo_solve_permuted(const mfo_analysis *a, const mfo_factor *fac, int posdef, double *x) {
  const int ns = a->nsn;
  for (int it = 0; it < ns; ++it) {
    const int s = a->postorder[it];
    const int f = fac->f_out[s], p = fac->p_out[s];
    const double *L = fac->blocks + fac->blk_off[s];
    const int *rows = fac->rows + fac->row_off[s];
    for (int j = 0; j < p; ++j) {
      const double *col = L + (size_t)j * f;
      double xj = x[rows[j]];
      if (posdef) xj /= col[j];
      x[rows[j]] = xj;
      for (int i = j + 1; i < f; ++i) x[rows[i]] -= col[i] * xj;
    }
  }
  if (!posdef) {
    for (int it = 0; it < ns; ++it) {
      const int s = a->postorder[it];
      const int f = fac->f_out[s], p = fac->p_out[s];
      const double *L = fac->blocks + fac->blk_off[s];
      const int *rows = fac->rows + fac->row_off[s];
      for (int c = 0; c < p;) {
        const double d00 = L[(size_t)c * f + c];
        if (c + 1 < p) {
          const double d10 = L[(size_t)(c + 1) * f + c];
          if (d10 != 0.0) {
            const double d11 = L[(size_t)(c + 1) * f + c + 1];
            const double s2 = max3(fabs(d00), fabs(d10), fabs(d11));
            const double aa = d00 / s2, bb = d10 / s2, cc = d11 / s2;
            const double det = aa * cc - bb * bb;
            const double r0 = x[rows[c]], r1 = x[rows[c + 1]];
            double y0 = 0.0, y1 = 0.0;
            if (s2 != 0.0 && is_fin(det) && det != 0.0) {
              y0 = ((cc * r0 - bb * r1) / det) / s2;
              y1 = ((-bb * r0 + aa * r1) / det) / s2;
            }
            x[rows[c]] = y0;
            x[rows[c + 1]] = y1;
            c += 2;
            continue;
          }
        }
        x[rows[c]] = (d00 == 0.0 || !is_fin(d00)) ? 0.0 : x[rows[c]] / d00;
        ++c;
      }
    }
  }
  for (int it = ns - 1; it >= 0; --it) {
    const int s = a->postorder[it];
    const int f = fac->f_out[s], p = fac->p_out[s];
    const double *L = fac->blocks + fac->blk_off[s];
    const int *rows = fac->rows + fac->row_off[s];
    for (int j = p - 1; j >= 0; --j) {
      const double *col = L + (size_t)j * f;
      double v = x[rows[j]];
      for (int i = j + 1; i < f; ++i) v -= col[i] * x[rows[i]];
      if (posdef) v /= col[j];
      x[rows[j]] = v;
    }
  }
}

/* r = b - A x and the backward errors of refinement.cpp:39-130 (normwise
 * eta_inf with ||A||_inf, componentwise omega), long double accumulation. */
void mfo_residual(int n, const int *cp, const int *ri, const double *v, const double *b,
                  const double *x, double *r, double *eta_inf, double *omega) {
  long double *ax = (long double *)calloc((size_t)n + 1, sizeof(long double));
  long double *aax = (long double *)calloc((size_t)n + 1, sizeof(long double));
  long double *rowabs = (long double *)calloc((size_t)n + 1, sizeof(long double));
  for (int j = 0; j < n; ++j)
    for (int k = cp[j]; k < cp[j + 1]; ++k) {
      const int i = ri[k];
      const long double val = v[k], av = fabsl(val);
      ax[i] += val * x[j];
      aax[i] += av * fabsl((long double)x[j]);
      rowabs[i] += av;
      if (i != j) {
        ax[j] += val * x[i];
        aax[j] += av * fabsl((long double)x[i]);
        rowabs[j] += av;
      }
    }
  long double na = 0, nx = 0, nb = 0, rmax = 0, om = 0;
  for (int i = 0; i < n; ++i) {
    if (rowabs[i] > na) na = rowabs[i];
    if (fabsl((long double)x[i]) > nx) nx = fabsl((long double)x[i]);
    if (fabsl((long double)b[i]) > nb) nb = fabsl((long double)b[i]);
    const long double res = (long double)b[i] - ax[i];
    r[i] = (double)res;
    if (fabsl(res) > rmax) rmax = fabsl(res);
    const long double den = aax[i] + fabsl((long double)b[i]);
    const long double oi = den > 0 ? fabsl(res) / den : (res == 0 ? 0 : 1.0L / 0.0L);
    if (oi > om) om = oi;
  }
  const long double ed = na * nx + nb;
  *eta_inf = (double)(ed > 0 ? rmax / ed : (rmax == 0 ? 0 : 1.0L / 0.0L));
  *omega = (double)om;
  free(ax);
  free(aax);
  free(rowabs);
}
