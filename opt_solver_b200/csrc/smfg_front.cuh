// Dense partial LDL^T / Cholesky of one front by one thread block, with
// smf's threshold 1x1 / 2x2 pivoting, stall handling and delayed columns.
//
// The algorithm and every per-entry operation follow the reference kernel
// ldlt_factor_front (solver/src/ldlt_kernel.cpp:970-1139); the block of
// threads shares each step:
//   - pivot search (select_pivot, ldlt_kernel.cpp:127-275; two_by_two_ok
//     :97-122) as block-wide max / top-2 reductions whose ties resolve to
//     the lowest row, i.e. the reference's first-in-scan-order rule;
//   - symmetric swaps (sym_swap :333-347): every swapped pair is disjoint,
//     so one pass of the block;
//   - eliminations (eliminate_1x1 / _2x2 :352-545): multiply, then subtract,
//     rounded separately (__dmul_rn / __dsub_rn, never contracted), as the
//     reference compiles ldlt_kernel.cpp with -ffp-contract=off;
//   - deferred and Schur updates (:705-761, :764-933): one fused
//     multiply-add per pivot and entry, pivots in order, as the reference's
//     contracted GEMM loops (dense_kernel_lapack.cpp:182-234) compute them.
// With the same inputs the front's L, D, pivot order, tags and Schur
// complement are therefore the reference's, bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace smfg {

constexpr double kWeakPivotRatio = 1e-6;  // ldlt_kernel.hpp:100

struct PivotParams {
  double u, eff_small, small_pivot;
  int nb, blocked_min_front, posdef;
  int aptp_min;  // indefinite fronts of at least this many rows take the APTP kernel (0: none)
};

struct FrontStats {
  int pos, neg, zero, two_by_two;
  double flops;
};

// Shared control block of a front kernel.
struct FrontShared {
  double red[32];
  int redi[32];
  double red2[32];
  int kind, a, b;        // pivot choice
  int k;                 // next pivot position
  int order[128];        // stall partner pairs (row ids, or assembly positions)
  int np;
  double vals[8];
  int ivals[8];
  // per-warp results of the parallel candidate tests / pairing scans
  int ckind[32], ca[32], cb[32];
  double pin[64], pout[64];
  int pr[64];
  int tr_seq;  // team reductions so far (alike in every CTA of a team)
  FrontStats st;
};

__device__ __forceinline__ double dmax_ref(double a, double b) {  // std::max(a, b)
  return (a < b) ? b : a;
}

__device__ __forceinline__ double max3_ref(double a, double b, double c) {
  double m = a;
  if (m < b) m = b;
  if (m < c) m = c;
  return m;
}

// Top-2 of a multiset of |values| with the first index of the maximum
// (the reference's "if (v > m1) {...} else if (v > m2)" scan, NaN ignored).
struct Top2 {
  double m1, m2;
  int r;
};

__device__ __forceinline__ void top2_add(Top2 &t, double v, int i) {
  if (v > t.m1) {
    t.m2 = t.m1;
    t.m1 = v;
    t.r = i;
  } else if (v > t.m2) {
    t.m2 = v;
  }
}

__device__ __forceinline__ Top2 top2_merge(Top2 a, Top2 b) {
  Top2 o;
  if (a.m1 > b.m1) {
    o.m1 = a.m1;
    o.r = a.r;
  } else if (b.m1 > a.m1) {
    o.m1 = b.m1;
    o.r = b.r;
  } else {
    o.m1 = a.m1;
    o.r = (a.r < 0) ? b.r : ((b.r < 0) ? a.r : min(a.r, b.r));
  }
  o.m2 = fmax(fmin(a.m1, b.m1), fmax(a.m2, b.m2));
  return o;
}

template <int NT>
struct Block {
  static_assert(NT % 32 == 0 && NT <= 1024, "block size");
  static constexpr int NW = NT / 32;

  // Max of non-negative values, NaN ignored (fmax).
  static __device__ double max(double v, FrontShared &sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (NW == 1) return v;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh.red[w] = v;
    __syncthreads();
    v = (l < NW) ? sh.red[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
  }

  // Two maxima at once.
  static __device__ void max2(double &a, double &b, FrontShared &sh) {
    for (int o = 16; o > 0; o >>= 1) {
      a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
      b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    if (NW == 1) return;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
      sh.red[w] = a;
      sh.red2[w] = b;
    }
    __syncthreads();
    a = (l < NW) ? sh.red[l] : 0.0;
    b = (l < NW) ? sh.red2[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
      b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
  }

  // A Top2 and two maxima in one pass (one shared-memory round).
  static __device__ void bundle(Top2 &t, double &a, double &b, FrontShared &sh) {
    for (int o = 16; o > 0; o >>= 1) {
      Top2 u;
      u.m1 = __shfl_xor_sync(0xffffffffu, t.m1, o);
      u.m2 = __shfl_xor_sync(0xffffffffu, t.m2, o);
      u.r = __shfl_xor_sync(0xffffffffu, t.r, o);
      t = top2_merge(t, u);
      a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
      b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    if (NW == 1) return;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
      sh.red[w] = t.m1;
      sh.red2[w] = t.m2;
      sh.redi[w] = t.r;
      sh.pin[w] = a;  // (the pairing scans' arrays: never in use at the same time)
      sh.pout[w] = b;
    }
    __syncthreads();
    if (l < NW) {
      t.m1 = sh.red[l];
      t.m2 = sh.red2[l];
      t.r = sh.redi[l];
      a = sh.pin[l];
      b = sh.pout[l];
    } else {
      t.m1 = 0.0;
      t.m2 = 0.0;
      t.r = -1;
      a = 0.0;
      b = 0.0;
    }
    for (int o = 16; o > 0; o >>= 1) {
      Top2 u;
      u.m1 = __shfl_xor_sync(0xffffffffu, t.m1, o);
      u.m2 = __shfl_xor_sync(0xffffffffu, t.m2, o);
      u.r = __shfl_xor_sync(0xffffffffu, t.r, o);
      t = top2_merge(t, u);
      a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
      b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
  }

  static __device__ Top2 top2(Top2 t, FrontShared &sh) {
    for (int o = 16; o > 0; o >>= 1) {
      Top2 u;
      u.m1 = __shfl_xor_sync(0xffffffffu, t.m1, o);
      u.m2 = __shfl_xor_sync(0xffffffffu, t.m2, o);
      u.r = __shfl_xor_sync(0xffffffffu, t.r, o);
      t = top2_merge(t, u);
    }
    if (NW == 1) return t;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
      sh.red[w] = t.m1;
      sh.red2[w] = t.m2;
      sh.redi[w] = t.r;
    }
    __syncthreads();
    if (l < NW) {
      t.m1 = sh.red[l];
      t.m2 = sh.red2[l];
      t.r = sh.redi[l];
    } else {
      t.m1 = 0.0;
      t.m2 = 0.0;
      t.r = -1;
    }
    for (int o = 16; o > 0; o >>= 1) {
      Top2 u;
      u.m1 = __shfl_xor_sync(0xffffffffu, t.m1, o);
      u.m2 = __shfl_xor_sync(0xffffffffu, t.m2, o);
      u.r = __shfl_xor_sync(0xffffffffu, t.r, o);
      t = top2_merge(t, u);
    }
    return t;
  }

  // First index i in [lo, hi) of the largest |col[i]| (> 0), the
  // reference's "if (v > out_max)" scan; -1 when all are zero.
  static __device__ void argmax(const double *col, int lo, int hi, double &m, int &r,
                                FrontShared &sh) {
    Top2 t{0.0, 0.0, -1};
    for (int i = lo + (int)threadIdx.x; i < hi; i += NT) top2_add(t, fabs(col[i]), i);
    t = top2(t, sh);
    m = t.m1;
    r = t.r;
  }
};

// The front: F f x f column-major with leading dimension ld (lower triangle
// used), its row ids, pivot tags, and W (f x nb, leading dimension f) for the
// blocked path's unscaled pivot columns.
// The pairing swaps' targets and their play-through on the position maps
// (moved rows -> positions, moved positions -> rows; the latest entry wins).
constexpr int kPairMax = 64;
struct PairScratch {
  int qq[kPairMax];
  int row_key[2 * kPairMax], row_pos[2 * kPairMax];
  int pos_key[2 * kPairMax], pos_row[2 * kPairMax];
};

struct FrontRef {
  double *F;
  int ld, f, ne;
  int *rows;
  int8_t *tags;
  double *W;
  int *loc;  // assembly position of the row now at each position (null: untracked)
  int *inv = nullptr;  // position of each assembly position (kept with loc; null: untracked)
  PairScratch *pair = nullptr;  // shared-memory scratch of the tracked pairing swaps
  // teams of several CTAs: the team's barrier counter, the error word a
  // timed-out barrier sets, this CTA's abort flag
  unsigned *team_bar = nullptr;  // this launch's arrival counter (monotone within the launch)
  unsigned long long *err = nullptr;
  int *abort = nullptr;
  unsigned *bar_seq = nullptr;    // this CTA's barriers so far in the launch (shared memory)
  double *team_red = nullptr;  // the team's reduction scratch: 2 buffers x C ranks x 4
};

// A team of C CTAs (a thread-block cluster; C = 1: the CTA alone) that runs
// one front's threshold pivoting: every CTA takes the same pivot decisions
// from the same data (its own block reductions, so the decisions are the
// one-CTA decisions bit for bit), and the memory-heavy updates (row and
// column swaps, eliminations of the panel) are split by rows over the team,
// each followed by a team barrier (team_sync below).
template <int C>
__device__ __forceinline__ int team_rank() {
  if constexpr (C == 1) {
    return 0;
  } else {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return (int)r;
  }
}

// Team barrier (C > 1): an arrival counter in global memory that only grows
// during a launch (the launch's own slot, reset by the previous launch): the
// i-th barrier adds 1 (acquire-release: the last arrival reads the others'
// writes through it) and waits, with acquire loads, until the counter
// reaches C (i + 1). The spin is bounded by the
// global timer (2 s): a team whose CTAs did not all arrive sets bit 128 of
// *err, and the CTA stops waiting at its later barriers (the host then
// discards the factorization and reports the timeout). The team's CTAs are
// co-scheduled (one cluster), so the wait only runs out if they took
// different paths.
template <int C>
__device__ __forceinline__ void team_sync(const FrontRef &v) {
  if constexpr (C == 1) {
    __syncthreads();
  } else {
    __syncthreads();
    if (threadIdx.x == 0 && !*v.abort) {
      const unsigned target = (unsigned)C * (*v.bar_seq + 1u);
      *v.bar_seq += 1u;
      unsigned seen;
      asm volatile("atom.add.acq_rel.gpu.u32 %0, [%1], 1;" : "=r"(seen) : "l"(v.team_bar) : "memory");
      seen += 1u;
      if (seen < target) {
        unsigned long long t0;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
        while (true) {
          asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(seen) : "l"(v.team_bar) : "memory");
          if (seen >= target) break;
          unsigned long long t;
          asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
          if (t - t0 > 2000000000ull) {
            *v.abort = 1;
            atomicOr(v.err, 128ull);
            break;
          }
        }
      }
    }
    __syncthreads();
  }
}

__device__ __forceinline__ double fat(const FrontRef &v, int i, int j) {  // element (i, j), i >= j
  return v.F[(size_t)j * v.ld + i];
}

// Returns whether it swapped (and so ended with a team barrier).
template <int NT, int C = 1>
static __device__ bool sym_swap_blk(const FrontRef &v, int p, int q, int w_cols, bool synced = false) {
  if (p == q) return false;
  if (p > q) {
    const int t = p;
    p = q;
    q = t;
  }
  // no CTA of the team writes while another still reads (C > 1); a swap
  // that follows a team barrier (the previous swap's) needs no other
  if constexpr (C > 1) {
    if (!synced) team_sync<C>(v);
  }
  const size_t sf = (size_t)v.ld;
  double *F = v.F;
  const int f = v.f;
  // Pairs: diagonal; m < p; p < m < q; m > q; rows; W rows. All disjoint.
  const int n1 = p, n2 = q - p - 1, n3 = f - q - 1;
  const int total = 1 + n1 + n2 + n3 + 1 + w_cols;
  for (int t = team_rank<C>() * NT + (int)threadIdx.x; t < total; t += C * NT) {
    if (t == 0) {
      const double x = F[p * sf + p];
      F[p * sf + p] = F[q * sf + q];
      F[q * sf + q] = x;
    } else if (t <= n1) {
      const int m = t - 1;
      const double x = F[m * sf + p];
      F[m * sf + p] = F[m * sf + q];
      F[m * sf + q] = x;
    } else if (t <= n1 + n2) {
      const int m = p + 1 + (t - 1 - n1);
      const double x = F[p * sf + m];
      F[p * sf + m] = F[m * sf + q];
      F[m * sf + q] = x;
    } else if (t <= n1 + n2 + n3) {
      const int m = q + 1 + (t - 1 - n1 - n2);
      const double x = F[p * sf + m];
      F[p * sf + m] = F[q * sf + m];
      F[q * sf + m] = x;
    } else if (t == n1 + n2 + n3 + 1) {
      const int r = v.rows[p];
      v.rows[p] = v.rows[q];
      v.rows[q] = r;
      if (v.loc) {
        const int a = v.loc[p];
        v.loc[p] = v.loc[q];
        v.loc[q] = a;
        if (v.inv) {
          v.inv[v.loc[p]] = p;
          v.inv[a] = q;
        }
      }
    } else {
      const int c = t - (n1 + n2 + n3 + 2);
      double *W = v.W + (size_t)c * f;
      const double x = W[p];
      W[p] = W[q];
      W[q] = x;
    }
  }
  team_sync<C>(v);
  return true;
}

__device__ __forceinline__ void inertia_1x1(double d, double small, FrontStats &st) {
  if (!isfinite(d) || fabs(d) < small) ++st.zero;
  else if (d > 0.0) ++st.pos;
  else ++st.neg;
}

// add_inertia_2x2 (solver/src/dense_indef.cpp:52-83).
__device__ __forceinline__ void inertia_2x2(double d00, double d10, double d11, double small,
                                            FrontStats &st) {
  if (d10 == 0.0) {
    inertia_1x1(d00, small, st);
    inertia_1x1(d11, small, st);
    return;
  }
  const double s = max3_ref(fabs(d00), fabs(d10), fabs(d11));
  double det_s = 0.0;
  if (isfinite(s) && s != 0.0)
    det_s = __dsub_rn(__dmul_rn(d00 / s, d11 / s), __dmul_rn(d10 / s, d10 / s));
  if (s == 0.0 || !isfinite(det_s)) {
    st.zero += 2;
    return;
  }
  const double tr_s = __dadd_rn(d00 / s, d11 / s);
  if (det_s < -small) {
    ++st.pos;
    ++st.neg;
  } else if (fabs(det_s) <= small) {
    ++st.zero;
    if (tr_s > small) ++st.pos;
    else if (tr_s < -small) ++st.neg;
    else ++st.zero;
  } else {
    if (tr_s > 0.0) st.pos += 2;
    else if (tr_s < 0.0) st.neg += 2;
    else st.zero += 2;
  }
}

// inverse_2x2 (ldlt_kernel.cpp:470-480).
__device__ __forceinline__ void inverse_2x2(double d00, double d10, double d11, double &i00,
                                            double &i10, double &i11) {
  const double s = max3_ref(fabs(d00), fabs(d10), fabs(d11));
  const double a = d00 / s, b = d10 / s, c = d11 / s;
  const double inv = 1.0 / __dmul_rn(__dsub_rn(__dmul_rn(a, c), __dmul_rn(b, b)), s);
  i00 = __dmul_rn(c, inv);
  i10 = __dmul_rn(-b, inv);
  i11 = __dmul_rn(a, inv);
}

// Thread layout of the block's update loops: kRB consecutive rows per pass
// (coalesced column-major accesses), NT / kRB column groups.
template <int NT>
struct Lay {
  static constexpr int RB = NT < 128 ? NT : 128;
  static constexpr int G = NT / RB;
  static __device__ __forceinline__ int r() { return threadIdx.x % RB; }
  static __device__ __forceinline__ int g() { return threadIdx.x / RB; }
};


// Panels of up to this many columns right of the pivot take the
// row-at-a-time elimination path (global-memory fronts: blocks of 512).
constexpr int kElimCols = 16;
constexpr int kElimGroup = 8;  // loads in flight per thread

template <int NT, int C = 1>
static __device__ void eliminate_1x1_blk(const FrontRef &v, int k, int ucol_end, bool useW, int w_col,
                                  bool synced = false) {
  using LY = Lay<NT>;
  const int rk = team_rank<C>();
  // (a swap that just ended with a team barrier needs no second one)
  if constexpr (C > 1) {
    if (!synced) team_sync<C>(v);
  }
  const size_t sf = (size_t)v.ld;
  const int f = v.f;
  double *ck = v.F + k * sf;
  const double inv_d = 1.0 / ck[k];
  if (useW) {
    double *w = v.W + (size_t)w_col * f;
    for (int i = k + 1 + rk * NT + (int)threadIdx.x; i < f; i += C * NT) w[i] = ck[i];
  }
  const int nj = ucol_end - (k + 1);
  if (NT >= 512 && nj <= kElimCols) {
    // a panel: the multipliers once in shared memory, then each thread
    // one row of every column at a time (all loads of the row in flight)
    __shared__ double s_l[kElimCols];
    for (int jj = threadIdx.x; jj < nj; jj += NT) s_l[jj] = __dmul_rn(ck[k + 1 + jj], inv_d);
    __syncthreads();
    for (int i = k + 1 + rk * NT + (int)threadIdx.x; i < f; i += C * NT) {
      const double cki = ck[i];
      const int jn = min(nj, i - k);  // columns j = k + 1 + jj <= i
      double *row = v.F + (size_t)(k + 1) * sf + i;
      for (int j0 = 0; j0 < jn; j0 += kElimGroup) {
        double x[kElimGroup];
#pragma unroll
        for (int u = 0; u < kElimGroup; ++u) x[u] = (j0 + u < jn) ? row[(size_t)(j0 + u) * sf] : 0.0;
#pragma unroll
        for (int u = 0; u < kElimGroup; ++u) {
          const double lj = s_l[j0 + u];
          if (j0 + u < jn && lj != 0.0) row[(size_t)(j0 + u) * sf] = __dsub_rn(x[u], __dmul_rn(cki, lj));
        }
      }
    }
  } else {
    // column j of (k, ucol_end), row i >= j: F(i, j) -= F(i, k) * l_j
    for (int i = k + 1 + rk * LY::RB + LY::r(); i < f; i += C * LY::RB) {
      const double cki = ck[i];
      const int jend = min(ucol_end, i + 1);
      for (int j = k + 1 + LY::g(); j < jend; j += LY::G) {
        const double lj = __dmul_rn(ck[j], inv_d);
        if (lj == 0.0) continue;
        double *cj = v.F + (size_t)j * sf;
        cj[i] = __dsub_rn(cj[i], __dmul_rn(cki, lj));
      }
    }
  }
  team_sync<C>(v);
  for (int i = k + 1 + rk * NT + (int)threadIdx.x; i < f; i += C * NT) ck[i] = __dmul_rn(ck[i], inv_d);
  // no barrier after the scaling for a team: the next pivot search reads
  // only later columns, and the next swap or elimination starts with one
  if constexpr (C == 1) __syncthreads();
}

template <int NT, int C = 1>
static __device__ void eliminate_2x2_blk(const FrontRef &v, int k, int ucol_end, bool useW, int w_col,
                                  bool synced = false) {
  using LY = Lay<NT>;
  const int rk = team_rank<C>();
  // (a swap that just ended with a team barrier needs no second one)
  if constexpr (C > 1) {
    if (!synced) team_sync<C>(v);
  }
  const size_t sf = (size_t)v.ld;
  const int f = v.f;
  double *c0 = v.F + k * sf;
  double *c1 = v.F + (k + 1) * sf;
  double i00, i10, i11;
  inverse_2x2(c0[k], c0[k + 1], c1[k + 1], i00, i10, i11);
  if (useW) {
    double *w0 = v.W + (size_t)w_col * f;
    double *w1 = w0 + f;
    for (int i = k + 2 + rk * NT + (int)threadIdx.x; i < f; i += C * NT) {
      w0[i] = c0[i];
      w1[i] = c1[i];
    }
  }
  const int nj = ucol_end - (k + 2);
  if (NT >= 512 && nj <= kElimCols) {
    // as eliminate_1x1_blk: multipliers in shared memory, rows in flight
    __shared__ double s_l0[kElimCols], s_l1[kElimCols];
    for (int jj = threadIdx.x; jj < nj; jj += NT) {
      const double a0 = c0[k + 2 + jj], a1 = c1[k + 2 + jj];
      s_l0[jj] = __dadd_rn(__dmul_rn(i00, a0), __dmul_rn(i10, a1));
      s_l1[jj] = __dadd_rn(__dmul_rn(i10, a0), __dmul_rn(i11, a1));
    }
    __syncthreads();
    for (int i = k + 2 + rk * NT + (int)threadIdx.x; i < f; i += C * NT) {
      const double c0i = c0[i], c1i = c1[i];
      const int jn = min(nj, i - k - 1);  // columns j = k + 2 + jj <= i
      double *row = v.F + (size_t)(k + 2) * sf + i;
      for (int j0 = 0; j0 < jn; j0 += kElimGroup) {
        double x[kElimGroup];
#pragma unroll
        for (int u = 0; u < kElimGroup; ++u) x[u] = (j0 + u < jn) ? row[(size_t)(j0 + u) * sf] : 0.0;
#pragma unroll
        for (int u = 0; u < kElimGroup; ++u) {
          const double l0 = s_l0[j0 + u], l1 = s_l1[j0 + u];
          if (j0 + u < jn && !(l0 == 0.0 && l1 == 0.0))
            row[(size_t)(j0 + u) * sf] = __dsub_rn(x[u], __dadd_rn(__dmul_rn(c0i, l0), __dmul_rn(c1i, l1)));
        }
      }
    }
  } else {
    for (int i = k + 2 + rk * LY::RB + LY::r(); i < f; i += C * LY::RB) {
      const double c0i = c0[i], c1i = c1[i];
      const int jend = min(ucol_end, i + 1);
      for (int j = k + 2 + LY::g(); j < jend; j += LY::G) {
        const double a0 = c0[j], a1 = c1[j];
        const double l0 = __dadd_rn(__dmul_rn(i00, a0), __dmul_rn(i10, a1));
        const double l1 = __dadd_rn(__dmul_rn(i10, a0), __dmul_rn(i11, a1));
        if (l0 == 0.0 && l1 == 0.0) continue;
        double *d0 = v.F + (size_t)j * sf;
        d0[i] = __dsub_rn(d0[i], __dadd_rn(__dmul_rn(c0i, l0), __dmul_rn(c1i, l1)));
      }
    }
  }
  team_sync<C>(v);
  for (int i = k + 2 + rk * NT + (int)threadIdx.x; i < f; i += C * NT) {
    const double a0 = c0[i], a1 = c1[i];
    c0[i] = __dadd_rn(__dmul_rn(i00, a0), __dmul_rn(i10, a1));
    c1[i] = __dadd_rn(__dmul_rn(i10, a0), __dmul_rn(i11, a1));
  }
  // no barrier after the scaling for a team: the next pivot search reads
  // only later columns, and the next swap or elimination starts with one
  if constexpr (C == 1) __syncthreads();
}

// two_by_two_ok (ldlt_kernel.cpp:97-122); off0 = max(m2, max_{i>=ext0} |col|).
__device__ __forceinline__ bool two_by_two_ok_s(double d00, double d10, double d11, double off0,
                                                double off1, const PivotParams &prm,
                                                double &growth) {
  const double s2 = max3_ref(fabs(d00), fabs(d10), fabs(d11));
  if (!(s2 >= prm.eff_small) || !isfinite(s2)) return false;
  const double a = d00 / s2, b = d10 / s2, c = d11 / s2;
  const double det_s = __dsub_rn(__dmul_rn(a, c), __dmul_rn(b, b));
  if (!(fabs(det_s) > prm.small_pivot)) return false;
  double g = 0.0;
  if (off0 > 0.0 || off1 > 0.0) {
    const double bound0 = __dadd_rn(__dmul_rn(fabs(c), off0), __dmul_rn(fabs(b), off1)) / s2;
    const double bound1 = __dadd_rn(__dmul_rn(fabs(b), off0), __dmul_rn(fabs(a), off1)) / s2;
    if (__dmul_rn(prm.u, dmax_ref(bound0, bound1)) > fabs(det_s)) return false;
    g = dmax_ref(bound0, bound1) / fabs(det_s);
  }
  growth = g;
  return true;
}

// select_pivot (ldlt_kernel.cpp:127-275). Result in sh.kind / sh.a / sh.b.
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ Top2 warp_top2(Top2 t) {
  for (int o = 16; o > 0; o >>= 1) {
    Top2 u;
    u.m1 = __shfl_xor_sync(0xffffffffu, t.m1, o);
    u.m2 = __shfl_xor_sync(0xffffffffu, t.m2, o);
    u.r = __shfl_xor_sync(0xffffffffu, t.r, o);
    t = top2_merge(t, u);
  }
  return t;
}

// |col[i]| for i in [lo, hi), thread tid of nth: 16-byte loads of aligned
// pairs, eight pairs in flight; each thread visits its indexes in increasing
// order (the head element before its pairs, the tail after), so fn sees a
// thread's share in scan order.
template <typename Fn>
__device__ __forceinline__ void scanv(const double *__restrict__ col, int lo, int hi, int tid, int nth, Fn fn) {
  if (lo >= hi) return;
  if (nth < 512) {  // small blocks (fronts in shared memory): one element at a time
    for (int i = lo + tid; i < hi; i += nth) fn(fabs(col[i]), i);
    return;
  }
  int a = lo;
  if (reinterpret_cast<uintptr_t>(col + a) & 15) {
    if (tid == 0) fn(fabs(col[a]), a);
    ++a;
  }
  const int npair = (hi - a) >> 1;
  const double2 *p2 = reinterpret_cast<const double2 *>(col + a);
  int m = tid;
  for (; m + 7 * nth < npair; m += 8 * nth) {
    double2 x[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) x[u] = p2[m + u * nth];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int i = a + 2 * (m + u * nth);
      fn(fabs(x[u].x), i);
      fn(fabs(x[u].y), i + 1);
    }
  }
  for (; m < npair; m += nth) {
    const double2 x = p2[m];
    fn(fabs(x.x), a + 2 * m);
    fn(fabs(x.y), a + 2 * m + 1);
  }
  if (((hi - a) & 1) && tid == npair % nth) fn(fabs(col[hi - 1]), hi - 1);
}

// Team-wide reduction of a bundle (a Top2 and two maxima): the block's
// reduction, then for a team of C > 1 CTAs each CTA's partial to the team's
// scratch, a team barrier and the C partials merged in rank order by every
// CTA (the merges are exact and order-independent, so every CTA holds the
// one-CTA result). Two buffers alternate: a buffer is rewritten only after
// the barrier of the next reduction, which every CTA reaches after reading.
template <int NT, int C>
static __device__ void team_bundle(const FrontRef &v, FrontShared &sh, Top2 &t, double &x1, double &x2) {
  Block<NT>::bundle(t, x1, x2, sh);
  if constexpr (C > 1) {
    const int buf = sh.tr_seq & 1;
    double *slot = v.team_red + (size_t)buf * C * 6;  // per rank: Top2 (4), maxima (2)
    const int rank = team_rank<C>();
    if (threadIdx.x == 0) {
      slot[rank * 4 + 0] = t.m1;
      slot[rank * 4 + 1] = t.m2;
      slot[rank * 4 + 2] = __longlong_as_double((long long)t.r);
      slot[rank * 4 + 3] = 0.0;
      slot[C * 4 + rank * 2 + 0] = x1;
      slot[C * 4 + rank * 2 + 1] = x2;
    }
    team_sync<C>(v);
    Top2 o{0.0, 0.0, -1};
    double a = 0.0, b = 0.0;
    for (int q = 0; q < C; ++q) {
      Top2 u{__ldcg(slot + q * 4 + 0), __ldcg(slot + q * 4 + 1),
             (int)__double_as_longlong(__ldcg(slot + q * 4 + 2))};
      o = top2_merge(o, u);
      a = fmax(a, __ldcg(slot + C * 4 + q * 2 + 0));
      b = fmax(b, __ldcg(slot + C * 4 + q * 2 + 1));
    }
    t = o;
    x1 = a;
    x2 = b;
    __syncthreads();
    if (threadIdx.x == 0) sh.tr_seq += 1;
    __syncthreads();
  }
}

// One candidate's test (as cand_eval_warp) by the whole team: its scans
// split by rows over every thread of every CTA, two team reductions.
template <int NT, int C>
static __device__ int cand_eval_team(const FrontRef &v, int k, int limit, int cand, const PivotParams &prm,
                              FrontShared &sh, int &pa, int &pb) {
  const int tid = team_rank<C>() * NT + (int)threadIdx.x;
  constexpr int NTT = C * NT;
  const size_t sf = (size_t)v.ld;
  const double *F = v.F;
  const int f = v.f, ne = v.ne;
  const double *col = F + (size_t)cand * sf;
  const double a_cand = fabs(col[cand]);
  Top2 t{0.0, 0.0, -1};
  for (int i = k + tid; i < cand; i += NTT) top2_add(t, fabs(F[(size_t)i * sf + cand]), i);
  // rows (cand, ne) into the top two, rows [max(ne, cand + 1), f) into ext
  double ext = 0.0, unused = 0.0;
  scanv(col, cand + 1, f, tid, NTT, [&](double x, int i) {
    if (i < ne) top2_add(t, x, i);
    else ext = fmax(ext, x);
  });
  team_bundle<NT, C>(v, sh, t, ext, unused);
  const double m1 = t.m1, m2 = t.m2;
  const int r_best = t.r;
  bool weak_1x1 = false;
  double weak_growth = 0.0;
  pa = pb = -1;
  if (a_cand >= prm.eff_small && !(__dmul_rn(prm.u, m1) > a_cand)) {
    if (!(__dmul_rn(prm.u, ext) > a_cand)) {
      const double colmax = dmax_ref(m1, ext);
      if (!(a_cand < __dmul_rn(kWeakPivotRatio, colmax))) {
        pa = cand;
        return 1;
      }
      weak_1x1 = true;
      weak_growth = colmax / a_cand;
    }
  }
  if (r_best < k || r_best >= limit || m1 <= 0.0) {
    if (weak_1x1) {
      pa = cand;
      return 1;
    }
    return 0;
  }
  const double *col_r = F + (size_t)r_best * sf;
  double om2 = 0.0, off1 = 0.0;
  for (int i = k + tid; i < r_best; i += NTT) {
    const double x = fabs(F[(size_t)i * sf + r_best]);
    om2 = fmax(om2, x);
    if (i != cand) off1 = fmax(off1, x);
  }
  scanv(col_r, r_best + 1, f, tid, NTT, [&](double x, int i) {
    om2 = fmax(om2, x);
    if (i != cand) off1 = fmax(off1, x);
  });
  Top2 none{0.0, 0.0, -1};
  team_bundle<NT, C>(v, sh, none, om2, off1);
  double growth2 = 0.0;
  const double d00 = col[cand];
  const double d10 = (r_best >= cand) ? F[(size_t)cand * sf + r_best] : F[(size_t)r_best * sf + cand];
  const double d11 = col_r[r_best];
  if (k + 1 < limit && two_by_two_ok_s(d00, d10, d11, dmax_ref(m2, ext), off1, prm, growth2) &&
      (!weak_1x1 || growth2 < weak_growth)) {
    pa = cand;
    pb = r_best;
    return 2;
  }
  if (weak_1x1) {
    pa = cand;
    return 1;
  }
  const double a_r = fabs(d11);
  if (a_r >= prm.eff_small && (om2 == 0.0 || a_r >= __dmul_rn(prm.u, om2))) {
    pa = r_best;
    return 1;
  }
  return 0;
}

// The test of one candidate column of select_pivot's search loop
// (ldlt_kernel.cpp:150-270) by one warp: 0 when the candidate gives no
// pivot, else 1 (pivot a) or 2 (pivot pair a, b). The candidates' tests are
// independent and the search takes the first candidate that gives one, so
// warps may test consecutive candidates at once; maxima are exact in any
// order, ties go to the lowest row as in the reference's scan.
static __device__ int cand_eval_warp(const FrontRef &v, int k, int limit, int cand, const PivotParams &prm, int &pa,
                              int &pb) {
  const int lane = threadIdx.x & 31;
  const size_t sf = (size_t)v.ld;
  const double *F = v.F;
  const int f = v.f, ne = v.ne;
  const double *col = F + (size_t)cand * sf;
  const double a_cand = fabs(col[cand]);
  Top2 t{0.0, 0.0, -1};
  for (int i = k + lane; i < cand; i += 32) top2_add(t, fabs(F[(size_t)i * sf + cand]), i);
#pragma unroll 4
  for (int i = cand + 1 + lane; i < ne; i += 32) top2_add(t, fabs(col[i]), i);
  t = warp_top2(t);
  const int ext0 = ne > cand + 1 ? ne : cand + 1;
  double ext = 0.0;
#pragma unroll 4
  for (int i = ext0 + lane; i < f; i += 32) ext = fmax(ext, fabs(col[i]));
  ext = warp_max(ext);
  const double m1 = t.m1, m2 = t.m2;
  const int r_best = t.r;
  bool weak_1x1 = false;
  double weak_growth = 0.0;
  pa = pb = -1;
  if (a_cand >= prm.eff_small && !(__dmul_rn(prm.u, m1) > a_cand)) {
    if (!(__dmul_rn(prm.u, ext) > a_cand)) {
      const double colmax = dmax_ref(m1, ext);
      if (!(a_cand < __dmul_rn(kWeakPivotRatio, colmax))) {
        pa = cand;
        return 1;
      }
      weak_1x1 = true;
      weak_growth = colmax / a_cand;
    }
  }
  if (r_best < k || r_best >= limit || m1 <= 0.0) {
    if (weak_1x1) {
      pa = cand;
      return 1;
    }
    return 0;
  }
  const double *col_r = F + (size_t)r_best * sf;
  double om2 = 0.0, off1 = 0.0;
  for (int i = k + lane; i < r_best; i += 32) {
    const double x = fabs(F[(size_t)i * sf + r_best]);
    om2 = fmax(om2, x);
    if (i != cand) off1 = fmax(off1, x);
  }
#pragma unroll 4
  for (int i = r_best + 1 + lane; i < f; i += 32) {
    const double x = fabs(col_r[i]);
    om2 = fmax(om2, x);
    if (i != cand) off1 = fmax(off1, x);
  }
  om2 = warp_max(om2);
  off1 = warp_max(off1);
  double growth2 = 0.0;
  const double d00 = col[cand];
  const double d10 = (r_best >= cand) ? F[(size_t)cand * sf + r_best] : F[(size_t)r_best * sf + cand];
  const double d11 = col_r[r_best];
  if (k + 1 < limit && two_by_two_ok_s(d00, d10, d11, dmax_ref(m2, ext), off1, prm, growth2) &&
      (!weak_1x1 || growth2 < weak_growth)) {
    pa = cand;
    pb = r_best;
    return 2;
  }
  if (weak_1x1) {
    pa = cand;
    return 1;
  }
  const double a_r = fabs(d11);
  if (a_r >= prm.eff_small && (om2 == 0.0 || a_r >= __dmul_rn(prm.u, om2))) {
    pa = r_best;
    return 1;
  }
  return 0;
}

template <int NT, int C = 1>
static __device__ void select_pivot_blk(const FrontRef &v, int k, int limit, const PivotParams &prm,
                                 FrontShared &sh) {
  const size_t sf = (size_t)v.ld;
  const double *F = v.F;
  const int f = v.f;
  int kind = 0, pa = -1, pb = -1;
  if (prm.posdef) {
    const double d = F[(size_t)k * sf + k];
    if (d > 0.0 && isfinite(d)) {
      kind = 1;
      pa = k;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      sh.kind = kind;
      sh.a = pa;
      sh.b = pb;
    }
    __syncthreads();
    return;
  }
  bool done = false;
  if (k < limit) {
    const double *col0 = F + (size_t)k * sf;
    const double a0 = fabs(col0[k]);
    if (a0 >= prm.eff_small) {
      double cm = 0.0;
      if constexpr (C == 1) {
        scanv(col0, k + 1, f, (int)threadIdx.x, NT, [&](double x, int) { cm = fmax(cm, x); });
        cm = Block<NT>::max(cm, sh);
      } else {
        scanv(col0, k + 1, f, team_rank<C>() * NT + (int)threadIdx.x, C * NT,
              [&](double x, int) { cm = fmax(cm, x); });
        Top2 none{0.0, 0.0, -1};
        double unused = 0.0;
        team_bundle<NT, C>(v, sh, none, cm, unused);
      }
      if (!(__dmul_rn(prm.u, cm) > a0) && !(a0 < __dmul_rn(kWeakPivotRatio, cm))) {
        kind = 1;
        pa = k;
        done = true;
      }
    }
  }
  // the search loop: long columns (and teams) one candidate at a time on
  // all threads; short ones NT / 32 candidates at a time (one warp each)
  if constexpr (C > 1) {
    // C candidates per round, one per CTA (its own block scans), then one
    // team exchange: the first candidate in order that gives a pivot wins
    const int rank = team_rank<C>();
    for (int c0 = k; c0 < limit && !done; c0 += C) {
      const int cand = c0 + rank;
      int tk = 0, ta = -1, tb = -1;
      if (cand < limit) tk = cand_eval_team<NT, 1>(v, k, limit, cand, prm, sh, ta, tb);
      double *slot = v.team_red + (size_t)(sh.tr_seq & 1) * C * 6;
      if (threadIdx.x == 0) {
        slot[rank * 4 + 0] = (double)tk;
        slot[rank * 4 + 1] = (double)ta;
        slot[rank * 4 + 2] = (double)tb;
      }
      team_sync<C>(v);
      for (int q = 0; q < C; ++q) {
        const int qk = (int)__ldcg(slot + q * 4 + 0);
        if (qk) {
          kind = qk;
          pa = (int)__ldcg(slot + q * 4 + 1);
          pb = (int)__ldcg(slot + q * 4 + 2);
          done = true;
          break;
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) sh.tr_seq += 1;
      __syncthreads();
    }
  } else if (f > 2048) {
    for (int cand = k; cand < limit && !done; ++cand) {
      int ta, tb;
      const int tk = cand_eval_team<NT, 1>(v, k, limit, cand, prm, sh, ta, tb);
      if (tk) {
        kind = tk;
        pa = ta;
        pb = tb;
        done = true;
      }
    }
  }
  constexpr int NW = NT / 32;
  const int warp = threadIdx.x >> 5;
  for (int c0 = k; c0 < limit && !done && !(C > 1 || f > 2048); c0 += NW) {
    const int cand = c0 + warp;
    int wk = 0, wa = -1, wb = -1;
    if (cand < limit) wk = cand_eval_warp(v, k, limit, cand, prm, wa, wb);
    if (NW == 1) {
      if (wk) {
        kind = wk;
        pa = wa;
        pb = wb;
        done = true;
      }
      continue;
    }
    if ((threadIdx.x & 31) == 0) {
      sh.ckind[warp] = wk;
      sh.ca[warp] = wa;
      sh.cb[warp] = wb;
    }
    __syncthreads();
    for (int w = 0; w < NW; ++w) {
      if (sh.ckind[w]) {
        kind = sh.ckind[w];
        pa = sh.ca[w];
        pb = sh.cb[w];
        done = true;
        break;
      }
    }
    __syncthreads();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    sh.kind = kind;
    sh.a = pa;
    sh.b = pb;
  }
  __syncthreads();
}

// apply_pivot (ldlt_kernel.cpp:666-698). The pivot choice is in sh.
template <int NT, int C = 1>
static __device__ void apply_pivot_blk(const FrontRef &v, int &k, bool useW, int w_cols, int ucol_end,
                                const PivotParams &prm, FrontShared &sh) {
  const size_t sf = (size_t)v.ld;
  const int f = v.f;
  const int kind = sh.kind, pa = sh.a, pb = sh.b;
  if (kind == 1) {
    const bool swapped = pa != k;
    sym_swap_blk<NT, C>(v, k, pa, useW ? w_cols : 0);
    if (threadIdx.x == 0) {
      inertia_1x1(v.F[k * sf + k], prm.eff_small, sh.st);
      v.tags[k] = 1;
      const double rem = (double)(f - (k + 1));
      sh.st.flops += rem + rem * (rem + 1.0);
    }
    eliminate_1x1_blk<NT, C>(v, k, ucol_end, useW, w_cols, swapped);
    k += 1;
    return;
  }
  int partner = pb;
  bool swapped = false;
  if (pa != k) {
    sym_swap_blk<NT, C>(v, k, pa, useW ? w_cols : 0);
    if (partner == k) partner = pa;
    swapped = true;
  }
  if (partner != k + 1) {
    sym_swap_blk<NT, C>(v, k + 1, partner, useW ? w_cols : 0, swapped);
    swapped = true;
  }
  if (threadIdx.x == 0) {
    inertia_2x2(v.F[k * sf + k], v.F[k * sf + k + 1], v.F[(k + 1) * sf + k + 1], prm.small_pivot,
                sh.st);
    v.tags[k] = 2;
    v.tags[k + 1] = -1;
    const double rem = (double)(f - (k + 2));
    sh.st.flops += 6.0 * rem + 2.0 * rem * (rem + 1.0);
    ++sh.st.two_by_two;
  }
  eliminate_2x2_blk<NT, C>(v, k, ucol_end, useW, w_cols, swapped);
  k += 2;
}

// deferred_update (ldlt_kernel.cpp:705-761): F[c0:f, c0:e] -= L[c0:f, p0:p1]
// W[c0:e, :]^T, one fused multiply-add per pivot in order, zero W skipped.
// (L D)(j, c) as fill_ld_column computes it (ldlt_kernel.cpp:764-818).
__device__ __forceinline__ double ld_entry(const FrontRef &v, int c, int j) {
  const size_t sf = (size_t)v.ld;
  const double *Lc = v.F + (size_t)c * sf;
  const int8_t tag = v.tags[c];
  if (tag == 1) return __dmul_rn(Lc[j], Lc[c]);
  if (tag == 2) return __dadd_rn(__dmul_rn(Lc[j], Lc[c]), __dmul_rn(Lc[sf + j], Lc[c + 1]));
  if (tag == -1) {
    const double *L0 = Lc - sf;
    return __dadd_rn(__dmul_rn(L0[j], L0[c]), __dmul_rn(Lc[j], Lc[c]));
  }
  return 0.0;
}

// The update F[i, j] -= sum over pivots c in [p0, p0 + kk), in order, of
// L(i, c) B(c, j) on the lower part of rows [c0, f) x columns [c0, cend),
// B = W (deferred updates) or (L D)^T (Schur), by one block of 512
// threads on a front in global memory: 64 x 64 tiles one after the other,
// 16 pivots of L and B staged in shared memory at a time (B computed once
// per tile column and chunk instead of once per entry), 8 entries a thread.
// Every entry keeps its chain c = fma(-l, b, c) over the pivots in order
// (b = 0 skipped): the loops it replaces give the same bits.
template <bool SCHUR>
static __device__ void front_update_tiles(const FrontRef &v, int c0, int cend, int p0, int kk) {
  constexpr int T = 64, KC = 16;
  __shared__ double As[KC][T], Bs[KC][T];
  const int f = v.f;
  const size_t sf = (size_t)v.ld;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;  // rows tx + 16 r, columns ty + 32 q
  const int rt = (f - c0 + T - 1) / T, ct = (cend - c0 + T - 1) / T;
  for (int tj = 0; tj < ct; ++tj) {
    for (int ti = tj; ti < rt; ++ti) {
      const int i0 = c0 + ti * T, j0 = c0 + tj * T;
      double c[4][2];
#pragma unroll
      for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int i = i0 + tx + 16 * r, j = j0 + ty + 32 * q;
          c[r][q] = (i < f && j < cend && i >= j) ? v.F[(size_t)j * sf + i] : 0.0;
        }
      for (int k0 = 0; k0 < kk; k0 += KC) {
        const int kc = min(KC, kk - k0);
        __syncthreads();  // the previous chunk's readers are done
#pragma unroll
        for (int u = 0; u < KC * T / 512; ++u) {
          const int t = tid + 512 * u, pp = t >> 6, x = t & 63;
          As[pp][x] = (pp < kc && i0 + x < f) ? v.F[(size_t)(p0 + k0 + pp) * sf + i0 + x] : 0.0;
          double bval = 0.0;
          if (pp < kc && j0 + x < cend) {
            if constexpr (SCHUR) bval = ld_entry(v, p0 + k0 + pp, j0 + x);
            else bval = v.W[(size_t)(k0 + pp) * f + j0 + x];
          }
          Bs[pp][x] = bval;
        }
        __syncthreads();
        for (int pp = 0; pp < kc; ++pp) {
          double av[4], bv[2];
#pragma unroll
          for (int r = 0; r < 4; ++r) av[r] = As[pp][tx + 16 * r];
#pragma unroll
          for (int q = 0; q < 2; ++q) bv[q] = Bs[pp][ty + 32 * q];
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            if (bv[q] != 0.0) {
#pragma unroll
              for (int r = 0; r < 4; ++r) c[r][q] = fma(-av[r], bv[q], c[r][q]);
            }
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int i = i0 + tx + 16 * r, j = j0 + ty + 32 * q;
          if (i < f && j < cend && i >= j) v.F[(size_t)j * sf + i] = c[r][q];
        }
    }
  }
  __syncthreads();
}

template <int NT>
static __device__ void deferred_update_blk(const FrontRef &v, int p0, int p1, int c0, int e) {
  using LY = Lay<NT>;
  const int jb = p1 - p0;
  if (jb <= 0 || e - c0 <= 0) return;
  if constexpr (NT == 512) {  // fronts in global memory: tiles staged in shared memory
    front_update_tiles<false>(v, c0, e, p0, jb);
    return;
  }
  const size_t sf = (size_t)v.ld;
  const int f = v.f;
  for (int i = c0 + LY::r(); i < f; i += LY::RB) {
    const int jend = min(e, i + 1);
    for (int j = c0 + LY::g(); j < jend; j += LY::G) {
      double c = v.F[(size_t)j * sf + i];
      for (int p = 0; p < jb; ++p) {
        const double b = v.W[(size_t)p * f + j];
        if (b == 0.0) continue;
        c = fma(-v.F[(size_t)(p0 + p) * sf + i], b, c);
      }
      v.F[(size_t)j * sf + i] = c;
    }
  }
  __syncthreads();
}


// schur_update (ldlt_kernel.cpp:820-933): F[e:f, e:f] -= L LD^T over the
// pivots [p0, p) in order.
template <int NT>
static __device__ void schur_update_blk(const FrontRef &v, int p0, int p, int e) {
  using LY = Lay<NT>;
  const int f = v.f;
  if (p <= p0 || f - e <= 0) return;
  if constexpr (NT == 512) {  // fronts in global memory: tiles staged in shared memory
    front_update_tiles<true>(v, e, f, p0, p - p0);
    return;
  }
  const size_t sf = (size_t)v.ld;
  for (int i = e + LY::r(); i < f; i += LY::RB) {
    for (int j = e + LY::g(); j <= i; j += LY::G) {
      double c = v.F[(size_t)j * sf + i];
      for (int cc = p0; cc < p; ++cc) {
        const double b = ld_entry(v, cc, j);
        if (b == 0.0) continue;
        c = fma(-v.F[(size_t)cc * sf + i], b, c);
      }
      v.F[(size_t)j * sf + i] = c;
    }
  }
  __syncthreads();
}

// State of the blocked path of ldlt_factor_front between its panel steps
// (ldlt_kernel.cpp:1010-1131): the first pass over the columns (phase 0,
// indefinite only), the main panel loop (phase 1), done (phase 2), or the
// unblocked loop after an APTP sweep (phase 3); `post`
// says what follows the deferred update the last step asked for. Every
// thread of the block holds the same copy (all decisions are uniform).
struct TppState {
  int phase, k, live, k_paired;
  int post, ps, pl, stalled;
  int g_p0, g_p1, g_c0, g_e;  // the deferred update asked for
  int pad[4];  // see tpp_init
  // mixed precision (outer blocks): the eligible columns [k, min(se, ne))
  // are current; every column from there on has the pivots [0, tc_done)
  // applied and waits for a tensor-core update by [tc_done, k)
  int mixed, tc_done, se, flush;
  FrontStats st;
};

__device__ __forceinline__ void tpp_init(TppState &S, int ne, bool posdef, bool mixed = false,
                                         int nbo = 0) {
  S.phase = posdef ? 1 : 0;
  S.k = 0;
  S.live = ne;
  S.k_paired = -1;
  S.post = 0;
  S.ps = S.pl = S.stalled = 0;
  S.g_p0 = S.g_p1 = S.g_c0 = S.g_e = 0;
  // pad: [0] a deferred update pending, [1] the W buffer it reads, [2] rows
  // of the panels' diagonal blocks staged in W (two-panel SPD steps)
  S.pad[0] = S.pad[1] = S.pad[2] = S.pad[3] = 0;
  S.mixed = mixed ? 1 : 0;
  S.tc_done = 0;
  // SPD: outer blocks of nbo pivots; indefinite: every eligible column
  // stays in the FP64 deferred updates (the pivot search and its swaps
  // never meet a stale column) and the tensor cores take the contribution
  // block, nbo pivots at a time
  S.se = (mixed && posdef) ? nbo : (1 << 30);
  S.flush = 0;
  S.st = FrontStats{0, 0, 0, 0, 0.0};
}

// End of the columns a deferred update may touch.
__device__ __forceinline__ int tpp_upd_end(const TppState &S, int ne) {
  return S.mixed ? min(ne, S.se) : ne;
}

// Mixed fronts: stops the step (returns true from tpp_step_blk with an
// empty update) so that the caller applies the pending tensor-core update
// before the step reads or swaps columns past the current outer block.
__device__ __forceinline__ bool tpp_request_flush(TppState &S) {
  S.flush = 1;
  S.g_p0 = S.g_p1 = S.k;
  S.g_c0 = S.g_e = S.k;
  return true;
}

// The targets of the pairing swaps (ldlt_kernel.cpp:1047-1095: the row
// order[t] goes to position k + t from the first position >= k + t that
// holds it, else from f - 1) when the front tracks positions (v.inv): the
// swaps are played on the maps, their moves kept in v.pair's override lists.
// One thread; np <= kPairMax.
__device__ __forceinline__ void pairing_targets(const FrontRef &v, int k, int f, int np, const FrontShared &sh) {
  PairScratch &ps = *v.pair;
  int nr = 0, npos = 0;
  auto pos_of = [&](int id) {
    for (int m = nr - 1; m >= 0; --m)
      if (ps.row_key[m] == id) return ps.row_pos[m];
    return v.inv[id];
  };
  auto id_at = [&](int pos) {
    for (int m = npos - 1; m >= 0; --m)
      if (ps.pos_key[m] == pos) return ps.pos_row[m];
    return v.loc[pos];
  };
  for (int t = 0; t < np; ++t) {
    const int at = pos_of(sh.order[t]);
    const int qq = (at >= k + t && at < f - 1) ? at : f - 1;
    ps.qq[t] = qq;
    if (qq != k + t) {
      const int idp = id_at(k + t), idq = id_at(qq);
      ps.row_key[nr] = idp;
      ps.row_pos[nr++] = qq;
      ps.row_key[nr] = idq;
      ps.row_pos[nr++] = k + t;
      ps.pos_key[npos] = k + t;
      ps.pos_row[npos++] = idq;
      ps.pos_key[npos] = qq;
      ps.pos_row[npos++] = idp;
    }
  }
}

// Runs the blocked algorithm up to its next deferred update, which it leaves
// in S.g_* (returns true), or to its end (returns false: the Schur update of
// the pivots [0, S.k) remains). The caller applies F[c0:f, c0:e] -=
// L[c0:f, p0:p1] W[c0:e, :]^T between two calls.
template <int NT, int C = 1>
static __device__ bool tpp_step_blk(const FrontRef &v, const PivotParams &prm, FrontShared &sh, TppState &S) {
  const int f = v.f, ne = v.ne;
  const size_t sf = (size_t)v.ld;
  if (S.phase == 3) {
    // unblocked, from the pivots an APTP sweep took (fewer than
    // blocked_min_front rows remain, ldlt_kernel.cpp:977-992): every pivot
    // updates the whole trailing triangle, no deferred or Schur update
    while (S.k < ne) {
      select_pivot_blk<NT, C>(v, S.k, ne, prm, sh);
      if (sh.kind == 0) break;
      apply_pivot_blk<NT, C>(v, S.k, false, 0, f, prm, sh);
    }
    S.pad[3] = S.k;
    S.phase = 2;
    return false;
  }
  // stale eligible columns past the outer block exist (mixed fronts)
  auto stale = [&]() { return S.mixed && S.tc_done < S.k && min(S.se, ne) < ne; };
  for (int guard = 0; guard < 4 * (ne + 8); ++guard) {
    if (S.post == 1) {  // after a first-pass panel (ldlt_kernel.cpp:1047-1095)
      if (S.stalled && stale()) return tpp_request_flush(S);
      S.post = 0;
      const int k = S.k, pl = S.pl;
      if (S.stalled && k != S.k_paired) {
        if (threadIdx.x == 0) sh.np = 0;
        __syncthreads();
        const int max_pairs = min(prm.nb / 2, 64);
        // rows named by assembly position (one to one with the row ids)
        // where the front tracks positions: the swap targets then come from
        // the position maps, not from a search
        const bool tracked = v.inv && v.pair && max_pairs <= kPairMax / 2;
        // the scans of the panel's columns are independent of the pairing
        // decisions: warps scan positions in parallel, thread 0 then takes
        // the decisions in position order
        constexpr int NWP = NT / 32;
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        for (int p0 = k; p0 < pl; p0 += 64) {
          const int pend = min(pl, p0 + 64);
          for (int pos = p0 + warp; pos < pend; pos += NWP) {
            const double *col = v.F + (size_t)pos * sf;
            double in_max = 0.0;
            for (int i = k + lane; i < pos; i += 32) in_max = fmax(in_max, fabs(v.F[(size_t)i * sf + pos]));
            for (int i = pos + 1 + lane; i < pl; i += 32) in_max = fmax(in_max, fabs(col[i]));
            in_max = warp_max(in_max);
            Top2 t{0.0, 0.0, -1};
#pragma unroll 4
            for (int i = pl + lane; i < ne; i += 32) top2_add(t, fabs(col[i]), i);
            t = warp_top2(t);
            if (lane == 0) {
              sh.pin[pos - p0] = in_max;
              sh.pout[pos - p0] = t.m1;
              sh.pr[pos - p0] = t.r;
            }
          }
          __syncthreads();
          if (threadIdx.x == 0) {
            for (int pos = p0; pos < pend; ++pos) {
              if (sh.np / 2 >= max_pairs) break;
              const int r = sh.pr[pos - p0];
              if (r >= 0 && sh.pout[pos - p0] > sh.pin[pos - p0]) {
                const int id_r = tracked ? v.loc[r] : v.rows[r];
                bool taken = false;
                for (int t = 1; t < sh.np; t += 2) taken = taken || sh.order[t] == id_r;
                if (!taken) {
                  sh.order[sh.np++] = tracked ? v.loc[pos] : v.rows[pos];
                  sh.order[sh.np++] = id_r;
                }
              }
            }
          }
          __syncthreads();
        }
        const int np = sh.np;
        if (np > 0) {
          if (tracked) {
            // positions tracked: thread 0 plays the swaps on the position
            // maps first (the maps as they stand, plus the moves so far),
            // so the swaps then run back to back
            if (threadIdx.x == 0) pairing_targets(v, k, f, np, sh);
            __syncthreads();
            bool sy = false;
            for (int t = 0; t < np; ++t) sy = sym_swap_blk<NT, C>(v, k + t, v.pair->qq[t], 0, sy) || sy;
          } else {
            for (int t = 0; t < np; ++t) {
              // the position of row id order[t] from k + t on (the first
              // match, else f - 1), searched by the whole block
              if (threadIdx.x == 0) sh.ivals[0] = f - 1;
              __syncthreads();
              const int want = sh.order[t];
              for (int i = k + t + threadIdx.x; i < f - 1; i += NT)
                if (v.rows[i] == want) atomicMin(&sh.ivals[0], i);
              __syncthreads();
              const int qq = sh.ivals[0];
              __syncthreads();
              sym_swap_blk<NT, C>(v, k + t, qq, 0);
            }
          }
          S.live = max(S.live, k + np);
          S.k_paired = k;
          continue;
        }
      }
      if (S.stalled) {
        const int m = pl - k;
        const int mv = min(m, S.live - pl);
        bool sy = false;
        for (int t = 0; t < mv; ++t) sy = sym_swap_blk<NT, C>(v, k + t, S.live - mv + t, 0, sy) || sy;
        S.live -= m;
      }
      continue;
    }
    if (S.post == 2) {  // after a main-loop panel (ldlt_kernel.cpp:1113-1127)
      if (S.stalled && S.k < ne && stale()) return tpp_request_flush(S);
      S.post = 0;
      if (S.stalled && S.k < ne) {
        const int ss = S.k;
        select_pivot_blk<NT, C>(v, S.k, ne, prm, sh);
        if (sh.kind == 0) {
          S.phase = 2;
          return false;
        }
        apply_pivot_blk<NT, C>(v, S.k, true, 0, ss, prm, sh);
        S.g_p0 = ss;
        S.g_p1 = S.k;
        S.g_c0 = S.k;
        S.g_e = tpp_upd_end(S, ne);
        S.post = 3;
        return true;
      }
      continue;
    }
    if (S.post == 3) {
      S.post = 0;
      continue;
    }
    if (S.phase == 0) {
      if (S.k < S.live) {
        if (S.mixed && S.tc_done < S.k && min(S.live, S.k + prm.nb) > min(S.se, ne))
          return tpp_request_flush(S);
        S.ps = S.k;
        S.pl = min(S.live, S.ps + prm.nb);
        S.stalled = 0;
        while (S.k < S.pl) {
          select_pivot_blk<NT, C>(v, S.k, S.pl, prm, sh);
          if (sh.kind == 0) {
            S.stalled = 1;
            break;
          }
          apply_pivot_blk<NT, C>(v, S.k, true, S.k - S.ps, S.pl, prm, sh);
        }
        S.g_p0 = S.ps;
        S.g_p1 = S.k;
        S.g_c0 = S.pl;
        S.g_e = tpp_upd_end(S, ne);
        S.post = 1;
        return true;
      }
      S.phase = 1;
    }
    if (S.phase == 1) {
      if (S.k < ne) {
        if (S.mixed && S.tc_done < S.k && min(ne, S.k + prm.nb) > min(S.se, ne))
          return tpp_request_flush(S);
        S.ps = S.k;
        S.pl = min(ne, S.ps + prm.nb);
        S.stalled = 0;
        while (S.k < S.pl) {
          select_pivot_blk<NT, C>(v, S.k, S.pl, prm, sh);
          if (sh.kind == 0) {
            S.stalled = 1;
            break;
          }
          apply_pivot_blk<NT, C>(v, S.k, true, S.k - S.ps, S.pl, prm, sh);
        }
        S.g_p0 = S.ps;
        S.g_p1 = S.k;
        S.g_c0 = S.pl;
        S.g_e = tpp_upd_end(S, ne);
        S.post = 2;
        return true;
      }
      S.phase = 2;
    }
    return false;
  }
  S.phase = 2;
  return false;
}

// ldlt_factor_front (first = 0, no static pivoting). Returns the accepted
// pivot count (uniform across the block); statistics in sh.st.
template <int NT>
static __device__ int ldlt_factor_front_blk(const FrontRef &v, const PivotParams &prm, FrontShared &sh,
                                     bool do_schur = true) {
  const int f = v.f, ne = v.ne;
  int k = 0;
  if (f < prm.blocked_min_front || prm.nb <= 1) {
    while (k < ne) {
      select_pivot_blk<NT>(v, k, ne, prm, sh);
      if (sh.kind == 0) break;
      apply_pivot_blk<NT>(v, k, false, 0, f, prm, sh);
    }
    return k;
  }
  TppState S;
  tpp_init(S, ne, prm.posdef != 0);
  while (tpp_step_blk<NT>(v, prm, sh, S)) deferred_update_blk<NT>(v, S.g_p0, S.g_p1, S.g_c0, S.g_e);
  if (do_schur) schur_update_blk<NT>(v, 0, S.k, ne);
  return S.k;
}

}  // namespace smfg
