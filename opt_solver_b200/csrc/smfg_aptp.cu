// APTP front kernel: the multi-CTA steps of each block column and the host
// side that sequences them over the APTP fronts of a tree level (see
// smfg_aptp.cuh for the algorithm and its reference).
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "../../include/smfg.h"
#include "smfg_aptp.cuh"
#include "smfg_aptp_host.h"

namespace smfg {
namespace aptp {

__device__ __forceinline__ double eff_small_of(const unsigned long long *bits) {
  return __longlong_as_double((long long)*bits);
}

// Block column k of front q: [c0, c0 + w); false when the sweep is past it.
__device__ __forceinline__ bool block_of(const Front &F, int k, int &c0, int &w) {
  c0 = k * F.nb;
  if (c0 >= F.ne) return false;
  w = min(F.nb, F.ne - c0);
  return true;
}

// 1. Backup of block column k: column c0 + t, rows [c0 + t, f) (grid.y = front).
__global__ void __launch_bounds__(256) k_backup(const Front *__restrict__ fr, int k) {
  const Front F = fr[blockIdx.y];
  int c0, w;
  if (!block_of(F, k, c0, w)) return;
  const int h = F.f - c0;
  const int64_t n = (int64_t)w * h;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(e / h), r = c0 + (int)(e % h);
    if (r >= c0 + t) F.bk[ix(t, F.f) + r] = F.A[ix(c0 + t, F.f) + r];
  }
}

// 2. The diagonal tile: one CTA per front.
__global__ void __launch_bounds__(kTileNT) k_tile(const Front *__restrict__ fr, State *__restrict__ stt, int k,
                                                  double inv_u, const unsigned long long *__restrict__ small_bits) {
  extern __shared__ __align__(16) unsigned char tile_smem[];
  TileShared &sh = *reinterpret_cast<TileShared *>(tile_smem);
  const Front F = fr[blockIdx.x];
  State &S = stt[blockIdx.x];
  int c0, w;
  if (!block_of(F, k, c0, w)) return;
  const double small = eff_small_of(small_bits);
  double *T = F.A + ix(c0, F.f) + c0;
  const int ne_t = tile_factor(T, F.f, w, F.tags + c0, F.rows + c0, S.lpc, F.loc ? F.loc + c0 : nullptr, inv_u,
                               small, sh);
  const bool ident = cta_identity(S.lpc, w);
  if (threadIdx.x == 0) {
    const int8_t *tb = F.tags + c0;
    for (int j = 0; j < ne_t; ++j) {
      if (tb[j] == 2) {
        double i00, i10, i11;
        inv2(T[ix(j, F.f) + j], T[ix(j, F.f) + j + 1], T[ix(j + 1, F.f) + j + 1], i00, i10, i11);
        S.dinv[2 * j] = i00;
        S.dinv[2 * j + 1] = i10;
        S.dinv[2 * (j + 1)] = i11;
        S.dinv[2 * (j + 1) + 1] = 0.0;
        ++j;
      } else {
        S.dinv[2 * j] = 1.0 / T[ix(j, F.f) + j];
        S.dinv[2 * j + 1] = 0.0;
      }
    }
    S.c0 = c0;
    S.w = w;
    S.ne_t = ne_t;
    S.nmin = ne_t;
    S.ident = ident ? 1 : 0;
    S.nq_old = S.nq;
  }
}

// 3. The tile's permutation on the rest of the front: rows [c0, c0 + w) of
// the columns left of the tile, and the rows below the tile from the backup
// (grid.y = front).
__global__ void __launch_bounds__(256) k_perm(const Front *__restrict__ fr, const State *__restrict__ stt, int k) {
  const Front F = fr[blockIdx.y];
  const State &S = stt[blockIdx.y];
  int c0, w;
  if (!block_of(F, k, c0, w) || S.ident) return;
  __shared__ int lpc[kNb];
  for (int t = threadIdx.x; t < w; t += blockDim.x) lpc[t] = S.lpc[t];
  __syncthreads();
  // columns [0, c0): one column per CTA iteration, the w rows gathered
  for (int c = blockIdx.x; c < c0; c += gridDim.x) {
    double v = 0.0;
    if ((int)threadIdx.x < w) v = F.A[ix(c, F.f) + c0 + lpc[threadIdx.x]];
    __syncthreads();
    if ((int)threadIdx.x < w) F.A[ix(c, F.f) + c0 + threadIdx.x] = v;
    __syncthreads();
  }
  const int h = F.f - c0 - w;
  const int64_t n = (int64_t)w * h;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(e / h), r = c0 + w + (int)(e % h);
    F.A[ix(c0 + t, F.f) + r] = F.bk[ix(lpc[t], F.f) + r];
  }
}

// 4. ApplyN (rows below the tile, in place) and ApplyT (rows of the earlier
// failed columns, into ga): x := x L_t^-T D^-1 per row, and the first pivot
// whose multipliers exceed 1/u, reduced into S.nmin. A CTA takes kRB rows,
// stages them in shared memory (coalesced), each warp solves kRB / 8 of them
// right-looking with the tile's L staged 32 columns at a time; per entry the
// chain is the same (earlier columns in order, a zero L entry skipped).
constexpr int kRB = 32;
constexpr int kRW = kRB / 8;  // rows per warp

struct ApplySmem {
  double x[kRB][kNb + 1];
  double L[32][kNb + 1];  // L_t(j, p0 + pp) at L[pp][j]
};

__global__ void __launch_bounds__(256) k_apply(const Front *__restrict__ fr, State *__restrict__ stt, int k,
                                               double inv_u) {
  extern __shared__ __align__(16) unsigned char apply_smem[];
  ApplySmem &sm = *reinterpret_cast<ApplySmem *>(apply_smem);
  const Front F = fr[blockIdx.y];
  State &S = stt[blockIdx.y];
  int c0, w;
  if (!block_of(F, k, c0, w)) return;
  const int ne_t = S.ne_t, nq = S.nq_old;
  if (ne_t <= 0) return;
  const int nbelow = F.f - c0 - w;
  const int nrb_below = (nbelow + kRB - 1) / kRB, nrb = nrb_below + (nq + kRB - 1) / kRB;
  const double *T = F.A + ix(c0, F.f) + c0;
  const int8_t *tb = F.tags + c0;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int fail = ne_t;
  for (int rb = blockIdx.x; rb < nrb; rb += gridDim.x) {
    const bool below = rb < nrb_below;
    const int r0 = below ? rb * kRB : (rb - nrb_below) * kRB;
    const int nr = min(kRB, (below ? nbelow : nq) - r0);
    __syncthreads();
    // stage the rows
    if (below) {
      for (int e = threadIdx.x; e < kRB * ne_t; e += blockDim.x) {
        const int t = e / kRB, rr = e % kRB;
        sm.x[rr][t] = rr < nr ? F.A[ix(c0 + t, F.f) + c0 + w + r0 + rr] : 0.0;
      }
    } else {
      for (int e = threadIdx.x; e < kRB * ne_t; e += blockDim.x) {
        const int rr = e / ne_t, t = e % ne_t;
        sm.x[rr][t] = rr < nr ? F.A[ix(F.Q[r0 + rr], F.f) + c0 + t] : 0.0;
      }
    }
    // the warp's rows in registers: lane l holds columns l + 32 u
    double x[kRW][8];
#pragma unroll
    for (int q = 0; q < kRW; ++q)
#pragma unroll
      for (int u = 0; u < 8; ++u) x[q][u] = 0.0;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kRW; ++q)
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int j = lane + 32 * u;
        if (j < ne_t) x[q][u] = sm.x[wid * kRW + q][j];
      }
    for (int p0 = 0; p0 < ne_t; p0 += 32) {
      __syncthreads();
      for (int e = threadIdx.x; e < 32 * ne_t; e += blockDim.x) {
        const int pp = e / ne_t, j = e % ne_t, p = p0 + pp;
        double l = 0.0;
        if (p < ne_t && j > p && !(tb[p] == 2 && j == p + 1)) l = T[ix(p, F.f) + j];
        sm.L[pp][j] = l;
      }
      __syncthreads();
      const int pend = min(32, ne_t - p0);
      for (int pp = 0; pp < pend; ++pp) {
        const int p = p0 + pp;
        const int up = p >> 5;
        double xp[kRW];
#pragma unroll
        for (int q = 0; q < kRW; ++q) {
          double v = 0.0;
#pragma unroll
          for (int u = 0; u < 8; ++u)
            if (u == up) v = x[q][u];
          xp[q] = __shfl_sync(0xffffffffu, v, p & 31);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int j = lane + 32 * u;
          if (j > p && j < ne_t) {
            const double l = sm.L[pp][j];
            if (l != 0.0) {
#pragma unroll
              for (int q = 0; q < kRW; ++q) x[q][u] = fma(-xp[q], l, x[q][u]);
            }
          }
        }
      }
    }
    // D^-1 and the check, pivot by pivot (every lane computes the values)
#pragma unroll
    for (int q = 0; q < kRW; ++q) {
      const int rr = wid * kRW + q;
      int fl = ne_t;
      for (int t = 0; t < ne_t; ++t) {
        const int8_t tg = tb[t];
        double a0 = 0.0, a1 = 0.0;
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (u == (t >> 5)) a0 = x[q][u];
        a0 = __shfl_sync(0xffffffffu, a0, t & 31);
        if (tg == 2) {
#pragma unroll
          for (int u = 0; u < 8; ++u)
            if (u == ((t + 1) >> 5)) a1 = x[q][u];
          a1 = __shfl_sync(0xffffffffu, a1, (t + 1) & 31);
          const double i00 = S.dinv[2 * t], i10 = S.dinv[2 * t + 1], i11 = S.dinv[2 * (t + 1)];
          const double l0 = fma(i00, a0, __dmul_rn(i10, a1)), l1 = fma(i10, a0, __dmul_rn(i11, a1));
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            if (lane + 32 * u == t) x[q][u] = l0;
            if (lane + 32 * u == t + 1) x[q][u] = l1;
          }
          if (fl == ne_t && (!l_ok(l0, inv_u) || !l_ok(l1, inv_u))) fl = t;
          ++t;
        } else {
          const double l = __dmul_rn(a0, S.dinv[2 * t]);
#pragma unroll
          for (int u = 0; u < 8; ++u)
            if (lane + 32 * u == t) x[q][u] = l;
          if (fl == ne_t && !l_ok(l, inv_u)) fl = t;
        }
      }
      if (rr < nr) fail = min(fail, fl);
    }
    // back to shared memory, then out (coalesced)
#pragma unroll
    for (int q = 0; q < kRW; ++q)
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int j = lane + 32 * u;
        if (j < ne_t) sm.x[wid * kRW + q][j] = x[q][u];
      }
    __syncthreads();
    if (below) {
      for (int e = threadIdx.x; e < kRB * ne_t; e += blockDim.x) {
        const int t = e / kRB, rr = e % kRB;
        if (rr < nr) F.A[ix(c0 + t, F.f) + c0 + w + r0 + rr] = sm.x[rr][t];
      }
    } else {
      for (int e = threadIdx.x; e < kRB * ne_t; e += blockDim.x) {
        const int rr = e / ne_t, t = e % ne_t;
        if (rr < nr) F.ga[ix(r0 + rr, kNb) + t] = sm.x[rr][t];
      }
    }
  }
  // the CTA's minimum, then the front's
  for (int o = 16; o > 0; o >>= 1) fail = min(fail, __shfl_down_sync(0xffffffffu, fail, o));
  if (lane == 0) atomicMin(&S.nmin, fail);
}

// 5. The block's accepted pivots (a 2x2 never splits), its failed columns
// appended to Q, counts (one thread per front).
__global__ void k_finish(const Front *__restrict__ fr, State *__restrict__ stt, int nf, int k) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nf) return;
  const Front F = fr[q];
  State &S = stt[q];
  int c0, w;
  if (!block_of(F, k, c0, w)) return;
  int nelim = S.ne_t > 0 ? S.nmin : 0;
  if (S.ne_t > 0 && nelim > 0 && F.tags[c0 + nelim - 1] == 2) --nelim;
  S.nelim = nelim;
  for (int s = nelim; s < w; ++s) F.Q[S.nq++] = c0 + s;
  S.num_elim += nelim;
}

// 6. Restore the failed columns of the block from the backup, write the
// accepted ApplyT rows back, and form W = (L D)^T of the eligible columns
// right of the pivots (into their strict upper triangle rows [c0, c0 +
// nelim)) and gb = (L D) of the earlier failed columns' rows (grid.y =
// front).
__global__ void __launch_bounds__(256) k_restore(const Front *__restrict__ fr, State *__restrict__ stt, int k) {
  const Front F = fr[blockIdx.y];
  State &S = stt[blockIdx.y];
  int c0, w;
  if (!block_of(F, k, c0, w)) return;
  const int nelim = S.nelim, nq = S.nq_old, f = F.f;
  const double *T = F.A + ix(c0, f) + c0;
  const int8_t *tb = F.tags + c0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  // restore: columns c0 + s2, s2 in [nelim, w): tile rows [s2, w) and the
  // rows below
  {
    const int nfail = w - nelim, h = f - c0;
    const int64_t n = (int64_t)nfail * h;
    for (int64_t e = tid; e < n; e += stride) {
      const int s2 = nelim + (int)(e / h), rr = (int)(e % h);
      if (rr < s2) continue;
      const int b2 = S.lpc[s2];
      double v;
      if (rr < w) {
        const int a1 = S.lpc[rr];
        v = (a1 >= b2) ? F.bk[ix(b2, f) + c0 + a1] : F.bk[ix(a1, f) + c0 + b2];
      } else {
        v = F.bk[ix(b2, f) + c0 + rr];
      }
      F.A[ix(c0 + s2, f) + c0 + rr] = v;
    }
    for (int64_t e = tid; e < nfail; e += stride) F.tags[c0 + nelim + e] = 0;
  }
  if (nelim <= 0) return;
  // ApplyT rows back, and their (L D)
  for (int64_t e = tid; e < (int64_t)nq * nelim; e += stride) {
    const int i = (int)(e / nelim), t = (int)(e % nelim);
    const double *g = F.ga + ix(i, kNb);
    F.A[ix(F.Q[i], f) + c0 + t] = g[t];
    const int8_t tg = tb[t];
    double v;
    if (tg == 2) v = ld_of(T, f, tb, t, g[t], g[t + 1]);
    else if (tg == -1) v = ld_of(T, f, tb, t, g[t - 1], g[t]);
    else v = ld_of(T, f, tb, t, g[t], 0.0);
    F.gb[ix(i, kNb) + t] = v;
  }
  // W of the eligible columns [e0, ne)
  const int e0 = c0 + nelim, ncol = F.ne - e0;
  for (int64_t e = tid; e < (int64_t)ncol * nelim; e += stride) {
    const int col = e0 + (int)(e / nelim), t = (int)(e % nelim);
    const int8_t tg = tb[t];
    double v;
    if (tg == 2) v = ld_of(T, f, tb, t, T[ix(t, f) + col - c0], T[ix(t + 1, f) + col - c0]);
    else if (tg == -1) v = ld_of(T, f, tb, t, T[ix(t - 1, f) + col - c0], T[ix(t, f) + col - c0]);
    else v = ld_of(T, f, tb, t, T[ix(t, f) + col - c0], 0.0);
    F.A[ix(col, f) + c0 + t] = v;
  }
}

// ---------------------------------------------------------------------------
// FP64 tile updates. One 128 x 64 tile of C per CTA iteration, 256 threads
// with 8 x 4 entries each, K staged 16 at a time in shared memory. Every
// entry runs its own chain over the pivots in order, a zero B entry skipped:
//   kSub:   c = fma(-a, b, c) on C (the portable dgemm / dgemmt loops);
//   kZero:  t = fma(a, b, t) from t = 0, then C = C - t (dgemm_nt into a
//           scratch, then subtracted: ldlt_aptp.cpp:558-580).
constexpr int kTM = 128, kTN = 64, kTK = 16;

struct GemmSmem {
  double A[2][kTK][kTM];
  double B[2][kTK][kTN];
};

// Tile jobs of one front (per launch): NN trapezoid, NT rectangle, TN
// trapezoid (block sweep), or the trailing trapezoid (end of the sweep).
struct Job {
  int kind;   // 0 NN, 1 NT, 2 TN, 3 trailing
  int rows, cols, ntiles;
};

__device__ __forceinline__ int trap_count(int rows, int cols) {  // tiles whose last row reaches their first column
  const int ct = (cols + kTN - 1) / kTN;
  int n = 0;
  for (int tj = 0; tj < ct; ++tj) n += (rows + kTM - 1) / kTM - (tj * kTN) / kTM;
  return n;
}

__device__ __forceinline__ void trap_at(int w, int rows, int &ti, int &tj) {
  const int rt = (rows + kTM - 1) / kTM;
  tj = 0;
  while (true) {
    const int first = (tj * kTN) / kTM, cnt = rt - first;
    if (w < cnt) {
      ti = first + w;
      return;
    }
    w -= cnt;
    ++tj;
  }
}

// The jobs of front F for this launch (mode 0: block updates, 1: trailing).
__device__ __forceinline__ int front_jobs(const Front &F, const State &S, int mode, Job *jobs) {
  int n = 0;
  if (mode == 0) {
    const int nelim = S.nelim;
    if (nelim <= 0) return 0;
    const int e0 = S.c0 + nelim;
    if (F.ne > e0) jobs[n++] = Job{0, F.f - e0, F.ne - e0, trap_count(F.f - e0, F.ne - e0)};
    const int nq = S.nq_old;
    if (nq > 0) {
      jobs[n++] = Job{1, F.f - e0, nq, ((F.f - e0 + kTM - 1) / kTM) * ((nq + kTN - 1) / kTN)};
      jobs[n++] = Job{2, nq, nq, trap_count(nq, nq)};
    }
  } else {
    const int p = S.num_elim, qn = F.f - F.ne;
    if (p > 0 && qn > 0) jobs[n++] = Job{3, qn, qn, trap_count(qn, qn)};
  }
  return n;
}

template <int KIND>
__device__ __forceinline__ void gemm_tile(const Front &F, const State &S, int i0, int j0, int rows, int cols,
                                          GemmSmem &sm) {
  const int f = F.f;
  const int c0 = (KIND == 3) ? 0 : S.c0;
  const int kk = (KIND == 3) ? S.num_elim : S.nelim;
  const int e0 = (KIND == 3) ? F.ne : S.c0 + S.nelim;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  // C(i, j): rows i < rows, columns j < cols of the job
  auto cptr = [&](int i, int j) -> double * {
    if (KIND == 0 || KIND == 3) return F.A + ix(e0 + j, f) + e0 + i;
    if (KIND == 1) return F.A + ix(F.Q[j], f) + e0 + i;
    return F.A + ix(F.Q[j], f) + F.Q[i];
  };
  auto needed = [&](int i, int j) -> bool {
    if (i >= rows || j >= cols) return false;
    if (KIND == 0) return e0 + i >= F.ne || i >= j;  // below the eligible block: every row
    if (KIND == 1) return true;
    return i >= j;  // TN: Q ascending, so Q[i] >= Q[j]; trailing: lower
  };
  double c[8][4];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = i0 + tx + 16 * r, j = j0 + ty + 16 * q;
      c[r][q] = (KIND == 1 || KIND == 2) ? 0.0 : (needed(i, j) ? *cptr(i, j) : 0.0);
    }
  double pa[8], pb[4];
  auto fetch = [&](int k0) {
    const int kc = min(kTK, kk - k0);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = threadIdx.x + 256 * u;
      const int p = t / kTM, r = t % kTM;
      double v = 0.0;
      if (p < kc && i0 + r < rows) {
        if (KIND == 2) v = F.ga[ix(i0 + r, kNb) + k0 + p];
        else v = F.A[ix(c0 + k0 + p, f) + e0 + i0 + r];
      }
      pa[u] = v;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = threadIdx.x + 256 * u;
      const int p = t / kTN, r = t % kTN;
      double v = 0.0;
      if (p < kc && j0 + r < cols) {
        if (KIND == 1 || KIND == 2) v = F.gb[ix(j0 + r, kNb) + k0 + p];
        else v = F.A[ix(e0 + j0 + r, f) + c0 + k0 + p];
      }
      pb[u] = v;
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
  stash(0);
  __syncthreads();
  for (int k0 = 0; k0 < kk; k0 += kTK) {
    const int kc = min(kTK, kk - k0);
    if (k0 + kTK < kk) fetch(k0 + kTK);
    for (int p = 0; p < kc; ++p) {
      double av[8], bv[4];
#pragma unroll
      for (int r = 0; r < 8; ++r) av[r] = sm.A[buf][p][tx + 16 * r];
#pragma unroll
      for (int q = 0; q < 4; ++q) bv[q] = sm.B[buf][p][ty + 16 * q];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (bv[q] != 0.0) {
          if (KIND == 1 || KIND == 2) {
#pragma unroll
            for (int r = 0; r < 8; ++r) c[r][q] = fma(av[r], bv[q], c[r][q]);
          } else {
#pragma unroll
            for (int r = 0; r < 8; ++r) c[r][q] = fma(-av[r], bv[q], c[r][q]);
          }
        }
      }
    }
    if (k0 + kTK < kk) {
      stash(buf ^ 1);
      __syncthreads();
      buf ^= 1;
    }
  }
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = i0 + tx + 16 * r, j = j0 + ty + 16 * q;
      if (needed(i, j)) {
        double *cp = cptr(i, j);
        if (KIND == 1 || KIND == 2) *cp = __dsub_rn(*cp, c[r][q]);
        else *cp = c[r][q];
      }
    }
  __syncthreads();
}

// 7. The block's updates (mode 0: UpdateNN, NT, TN) or the trailing update
// (mode 1) of every front, as one list of tiles.
__global__ void __launch_bounds__(256) k_update(const Front *__restrict__ fr, const State *__restrict__ stt, int nf,
                                                int k, int mode) {
  extern __shared__ __align__(16) unsigned char gemm_smem[];
  GemmSmem &sm = *reinterpret_cast<GemmSmem *>(gemm_smem);
  __shared__ int pref[3 * 64 + 1];
  __shared__ Job jobs[3 * 64];
  __shared__ int jfront[3 * 64];
  __shared__ int njobs;
  for (int chunk = 0; chunk < nf; chunk += 64) {
    const int cnt = min(64, nf - chunk);
    __syncthreads();
    if (threadIdx.x == 0) {
      int nj = 0;
      pref[0] = 0;
      for (int q = chunk; q < chunk + cnt; ++q) {
        const Front F = fr[q];
        int c0, w;
        if (mode == 0 && !block_of(F, k, c0, w)) continue;
        Job js[3];
        const int n = front_jobs(F, stt[q], mode, js);
        for (int u = 0; u < n; ++u) {
          jobs[nj] = js[u];
          jfront[nj] = q;
          pref[nj + 1] = pref[nj] + js[u].ntiles;
          ++nj;
        }
      }
      njobs = nj;
    }
    __syncthreads();
    const int nj = njobs;
    const int total = pref[nj];
    for (int wi = blockIdx.x; wi < total; wi += gridDim.x) {
      int a = 0, b = nj;
      while (b - a > 1) {
        const int mid = (a + b) >> 1;
        if (pref[mid] <= wi) a = mid;
        else b = mid;
      }
      const Job J = jobs[a];
      const Front &F = fr[jfront[a]];
      const State &S = stt[jfront[a]];
      const int local = wi - pref[a];
      int ti, tj;
      if (J.kind == 1) {
        const int rt = (J.rows + kTM - 1) / kTM;
        ti = local % rt;
        tj = local / rt;
      } else {
        trap_at(local, J.rows, ti, tj);
      }
      const int i0 = ti * kTM, j0 = tj * kTN;
      switch (J.kind) {
        case 0: gemm_tile<0>(F, S, i0, j0, J.rows, J.cols, sm); break;
        case 1: gemm_tile<1>(F, S, i0, j0, J.rows, J.cols, sm); break;
        case 2: gemm_tile<2>(F, S, i0, j0, J.rows, J.cols, sm); break;
        default: gemm_tile<3>(F, S, i0, j0, J.rows, J.cols, sm); break;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// End of the sweep.

// 8. The compaction permutation (one thread per front): the swaps that move
// the failed columns behind the pivots, eliminated order kept
// (ldlt_aptp.cpp:603-614), replayed on an index array; tags permuted on the
// way, rows and loc after.
__global__ void k_compact_perm(const Front *__restrict__ fr, const State *__restrict__ stt, int nf) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nf) return;
  const Front F = fr[q];
  const State &S = stt[q];
  if (S.num_elim >= F.ne) return;
  for (int t = 0; t < F.ne; ++t) F.pi[t] = t;
  int dst = 0;
  for (int src = 0; src < F.ne; ++src) {
    if (F.tags[src] == 0) continue;
    if (src != dst) {
      const int8_t tg = F.tags[dst];
      F.tags[dst] = F.tags[src];
      F.tags[src] = tg;
      const int u = F.pi[dst];
      F.pi[dst] = F.pi[src];
      F.pi[src] = u;
    }
    ++dst;
  }
  // rows / loc through Q (free after the sweep)
  for (int t = 0; t < F.ne; ++t) F.Q[t] = F.rows[t];
  for (int t = 0; t < F.ne; ++t) F.rows[t] = F.Q[F.pi[t]];
  if (F.loc) {
    for (int t = 0; t < F.ne; ++t) F.Q[t] = F.loc[t];
    for (int t = 0; t < F.ne; ++t) F.loc[t] = F.Q[F.pi[t]];
  }
}

// 9. The symmetric permutation of the eligible part, out of place: entry (i,
// j), j < ne, i >= j, takes the lower-stored entry of the old positions
// (pi(i), pi(j)) (pi(i) = i for i >= ne), then copied back.
__global__ void __launch_bounds__(256) k_compact_gather(const Front *__restrict__ fr, const State *__restrict__ stt,
                                                        int q, double *__restrict__ scratch, int back) {
  const Front F = fr[q];
  if (stt[q].num_elim >= F.ne) return;
  const int f = F.f, ne = F.ne;
  const int64_t n = (int64_t)ne * f;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(e / f), i = (int)(e % f);
    if (i < j) continue;
    if (back) {
      F.A[ix(j, f) + i] = scratch[e];
    } else {
      const int a = i < ne ? F.pi[i] : i, b = F.pi[j];
      scratch[e] = (a >= b) ? F.A[ix(b, f) + a] : F.A[ix(a, f) + b];
    }
  }
}

// 10. W of the trailing update: (L D)^T of the rows [ne, f) into the strict
// upper triangle rows [0, p) of those columns (ldlt_aptp.cpp:619-638).
__global__ void __launch_bounds__(256) k_trailing_w(const Front *__restrict__ fr, const State *__restrict__ stt) {
  const Front F = fr[blockIdx.y];
  const int p = stt[blockIdx.y].num_elim, f = F.f, ne = F.ne;
  const int qn = f - ne;
  if (p <= 0 || qn <= 0) return;
  const int64_t n = (int64_t)qn * p;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e / qn), i = ne + (int)(e % qn);
    const int8_t tg = F.tags[c];
    const double *Lc = F.A + ix(c, f);
    double v;
    if (tg == 2) {
      v = fma(Lc[i], Lc[c], __dmul_rn(Lc[f + i], Lc[c + 1]));
    } else if (tg == -1) {
      const double *L0 = Lc - f;
      v = fma(L0[i], L0[c], __dmul_rn(Lc[i], Lc[c]));
    } else {
      v = __dmul_rn(Lc[i], Lc[c]);
    }
    F.A[ix(i, f) + c] = v;
  }
}

// 11. Inertia and flops of the sweep's pivots (front_result,
// ldlt_aptp.cpp:704-724): every pivot against the effective small value.
__global__ void __launch_bounds__(256) k_stats(const Front *__restrict__ fr, State *__restrict__ stt,
                                               const unsigned long long *__restrict__ small_bits) {
  const Front F = fr[blockIdx.x];
  State &S = stt[blockIdx.x];
  const double small = eff_small_of(small_bits);
  const int pe = S.num_elim, f = F.f;
  FrontStats st{0, 0, 0, 0, 0.0};
  for (int k = threadIdx.x; k < pe; k += blockDim.x) {
    const int8_t tg = F.tags[k];
    if (tg == 2) {
      inertia_2x2(F.A[ix(k, f) + k], F.A[ix(k, f) + k + 1], F.A[ix(k + 1, f) + k + 1], small, st);
      const double rem = (double)(f - (k + 2));
      st.flops += __dadd_rn(__dmul_rn(6.0, rem), __dmul_rn(__dmul_rn(2.0, rem), rem + 1.0));
      ++st.two_by_two;
    } else if (tg == 1) {
      inertia_1x1(F.A[ix(k, f) + k], small, st);
      const double rem = (double)(f - (k + 1));
      st.flops += __dadd_rn(rem, __dmul_rn(rem, rem + 1.0));
    }
  }
  atomicAdd(&S.st.pos, st.pos);
  atomicAdd(&S.st.neg, st.neg);
  atomicAdd(&S.st.zero, st.zero);
  atomicAdd(&S.st.two_by_two, st.two_by_two);
  atomicAdd(&S.st.flops, st.flops);
}

__global__ void k_state_init(State *__restrict__ stt, int nf) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nf) return;
  State &S = stt[q];
  S.c0 = S.w = S.ne_t = S.nmin = S.nelim = 0;
  S.nq = S.nq_old = S.num_elim = 0;
  S.ident = 1;
  S.st = FrontStats{0, 0, 0, 0, 0.0};
}

// Front tags: zero for the eligible columns (sweep_begin).
__global__ void k_tags_init(const Front *__restrict__ fr) {
  const Front F = fr[blockIdx.x];
  for (int t = threadIdx.x; t < F.ne; t += blockDim.x) F.tags[t] = 0;
}

// ---------------------------------------------------------------------------
// Host side.

size_t tile_smem_bytes() { return sizeof(TileShared); }

void check(cudaError_t e) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("aptp: ") + cudaGetErrorString(e));
}

void set_attrs() {
  static bool done = false;
  if (done) return;
  check(cudaFuncSetAttribute(k_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TileShared)));
  check(cudaFuncSetAttribute(k_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(ApplySmem)));
  check(cudaFuncSetAttribute(k_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(GemmSmem)));
  done = true;
}

int sweep_blocks(const Front *d_fr, State *d_st, int nf, int kmax, const SweepHost &h, cudaStream_t st) {
  set_attrs();
  const int sms = h.sms;
  int launches = 0;
  k_state_init<<<(nf + 127) / 128, 128, 0, st>>>(d_st, nf);
  k_tags_init<<<nf, 256, 0, st>>>(d_fr);
  launches += 2;
  const dim3 g2(std::max(1, 2 * sms / std::max(1, nf)), nf);
  for (int k = 0; k < kmax; ++k) {
    k_backup<<<g2, 256, 0, st>>>(d_fr, k);
    k_tile<<<nf, kTileNT, sizeof(TileShared), st>>>(d_fr, d_st, k, h.inv_u, h.small_bits);
    k_perm<<<g2, 256, 0, st>>>(d_fr, d_st, k);
    k_apply<<<g2, 256, sizeof(ApplySmem), st>>>(d_fr, d_st, k, h.inv_u);
    k_finish<<<(nf + 31) / 32, 32, 0, st>>>(d_fr, d_st, nf, k);
    k_restore<<<g2, 256, 0, st>>>(d_fr, d_st, k);
    k_update<<<2 * sms, 256, sizeof(GemmSmem), st>>>(d_fr, d_st, nf, k, 0);
    launches += 7;
  }
  check(cudaGetLastError());
  return launches;
}

int sweep_finish(const Front *d_fr, State *d_st, int nf, const int *compact, int ncompact, const SweepHost &h,
                 cudaStream_t st) {
  const int sms = h.sms;
  int launches = 0;
  if (ncompact > 0) {
    k_compact_perm<<<(nf + 31) / 32, 32, 0, st>>>(d_fr, d_st, nf);
    ++launches;
    for (int u = 0; u < ncompact; ++u) {
      k_compact_gather<<<2 * sms, 256, 0, st>>>(d_fr, d_st, compact[u], h.scratch, 0);
      k_compact_gather<<<2 * sms, 256, 0, st>>>(d_fr, d_st, compact[u], h.scratch, 1);
      launches += 2;
    }
  }
  const dim3 g2(std::max(1, 2 * sms / std::max(1, nf)), nf);
  k_trailing_w<<<g2, 256, 0, st>>>(d_fr, d_st);
  k_update<<<2 * sms, 256, sizeof(GemmSmem), st>>>(d_fr, d_st, nf, 0, 1);
  k_stats<<<nf, 256, 0, st>>>(d_fr, d_st, h.small_bits);
  launches += 3;
  check(cudaGetLastError());
  return launches;
}

}  // namespace aptp
}  // namespace smfg

// ---------------------------------------------------------------------------
// The APTP kernel alone on one dense front in device memory (a self-test of
// the kernel, no reference counterpart as an entry point): the same sweep
// the engine runs on its APTP fronts.
using smfg::aptp::check;

extern "C" SMFG_API int smfg_aptp_front_dense(double *d_F, int f, int ne, int *d_rows, int8_t *d_tags, double u,
                                              double small, int64_t *out) {
  using namespace smfg::aptp;
  if (!d_F || !d_rows || !d_tags || !out || f <= 0 || ne <= 0 || ne > f || !(u > 0.0)) return SMFG_ERR_INVALID_ARG;
  std::vector<void *> mem;
  auto take = [&](size_t bytes) {
    void *p = nullptr;
    check(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
    mem.push_back(p);
    return p;
  };
  int rc = SMFG_OK;
  try {
    int dev = 0, sms = 0;
    check(cudaGetDevice(&dev));
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    Front F{};
    F.A = d_F;
    F.rows = d_rows;
    F.tags = d_tags;
    F.loc = nullptr;
    F.f = f;
    F.ne = ne;
    F.nb = std::min(kNb, ne);
    F.ib = std::min(kIb, F.nb);
    double *scr = static_cast<double *>(take(sizeof(double) * scratch_doubles(f, ne)));
    F.bk = scr;
    F.ga = scr + (int64_t)f * kNb;
    F.gb = F.ga + (int64_t)ne * kNb;
    F.Q = static_cast<int *>(take(sizeof(int) * ne));
    F.pi = static_cast<int *>(take(sizeof(int) * ne));
    Front *d_fr = static_cast<Front *>(take(sizeof(Front)));
    State *d_st = static_cast<State *>(take(sizeof(State)));
    unsigned long long *d_small = static_cast<unsigned long long *>(take(sizeof(unsigned long long)));
    double *gather = static_cast<double *>(take(sizeof(double) * (size_t)f * ne));
    unsigned long long sb;
    std::memcpy(&sb, &small, sizeof(sb));
    check(cudaMemcpy(d_small, &sb, sizeof(sb), cudaMemcpyHostToDevice));
    check(cudaMemcpy(d_fr, &F, sizeof(Front), cudaMemcpyHostToDevice));
    SweepHost h{sms, 1.0 / u, d_small, gather};
    sweep_blocks(d_fr, d_st, 1, (ne + F.nb - 1) / F.nb, h, 0);
    State S;
    check(cudaMemcpy(&S, d_st, sizeof(State), cudaMemcpyDeviceToHost));
    const int only = 0;
    sweep_finish(d_fr, d_st, 1, &only, S.num_elim < ne ? 1 : 0, h, 0);
    check(cudaMemcpy(&S, d_st, sizeof(State), cudaMemcpyDeviceToHost));
    out[0] = S.num_elim;
    out[1] = ne - S.num_elim;
    out[2] = S.st.pos;
    out[3] = S.st.neg;
    out[4] = S.st.zero;
  } catch (const std::exception &) {
    rc = SMFG_ERR_CUDA;
  }
  for (void *p : mem) cudaFree(p);
  return rc;
}
