// Tensor-core trailing updates of large fronts (the mixed-precision path):
//   C[r0 + i, r0 + j] -= sum_t L(i, t) W(j, t)    (i >= j, lower triangle)
// with W = L D, on the 5th-generation tensor cores (tcgen05.mma, accumulators
// in tensor memory). FP64 operands are split as x = hi + lo in TF32 (or
// BF16); the three products hi*hi + hi*lo + lo*hi accumulate in FP32 in
// tensor memory and the epilogue subtracts the sum from the FP64 front.
//
// Data path: k_tc_split writes each job's four operands (L hi, L lo, W hi,
// W lo) as 128-row x 128-byte blocks already in the tensor cores' canonical
// K-major shared-memory layout (8-row x 16-byte core matrices, no swizzle),
// so the GEMM kernel moves each block with one bulk copy (cp.async.bulk,
// completion counted on an mbarrier). k_tc_syrk is persistent, one CTA per
// SM: warp 0 produces (bulk copies into a 3-stage ring), warp 1 issues the
// MMAs (one elected thread) into two 128-column accumulators, warps 2..5
// drain an accumulator (tcgen05.ld) into the FP64 tile while the next tile
// accumulates into the other. Every wait is bounded by the global timer;
// a timeout sets an error flag, stops the CTA's loops and the CTA still
// drains its MMAs and copies and frees its tensor memory before returning.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace smfg {
namespace tc {

constexpr int kBM = 128;                    // tile rows = accumulator lanes
constexpr int kBN = 128;                    // tile columns = accumulator columns
constexpr int kRowBytes = 128;              // bytes of K per row of one k-block
constexpr int kBlkBytes = kBM * kRowBytes;  // one operand block: 16 KB
constexpr int kStages = 3;
constexpr int kOps = 4;                     // L hi, L lo, W hi, W lo
constexpr int kThreads = 192;               // producer, MMA, 4 epilogue warps
constexpr int kTmemCols = 2 * kBN;          // two accumulators
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s per wait

enum Kind : int { kTF32x3 = 0, kBF16x3 = 1 };

// One trailing update. L(i, t) = Ls[t * ldl + lr0 + i]; W(i, t) likewise
// from Ws, or, when Ws is null, W = L D from the front C itself: D's
// diagonal at C[(k0 + t) * ld + k0 + t] with 2x2 blocks per `tags` (null:
// 1x1 pivots only, the SPD path).
struct Job {
  double *C;
  const double *Ls, *Ws;
  const int8_t *tags;
  int64_t ld, ldl, ldw;
  int r0, lr0, wr0;  // first trailing row in C, in Ls, in Ws
  int n;             // trailing order
  int k0, kc;        // pivots
  int ntr, nkb;      // row blocks, k-blocks
  int tiles;         // ntr (ntr + 1) / 2 lower tiles
  int64_t img;       // byte offset of the job's images in the image buffer
};

struct Smem {
  uint8_t buf[kStages][kOps][kBlkBytes];
  unsigned long long full[kStages], empty[kStages], acc_full[2], acc_empty[2], drain;
  uint32_t tmem_base;
  int abort;
};

__host__ __device__ constexpr int64_t image_bytes(int ntr, int nkb) {
  return (int64_t)kOps * ntr * nkb * kBlkBytes;
}

// Elements of one 128-byte k-block row.
__host__ __device__ constexpr int kblock_elems(int kind) { return kind == kTF32x3 ? 32 : 64; }

// ---------------------------------------------------------------------------
// PTX wrappers.

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(unsigned long long *b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned long long *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false on timeout (sets *abort) or when another role aborted.
__device__ __forceinline__ bool mbar_wait(unsigned long long *b, uint32_t parity, volatile int *abort) {
  if (mbar_try(b, parity)) return true;
  const unsigned long long t0 = gtimer();
  while (!mbar_try(b, parity)) {
    if (*abort) return false;
    if (gtimer() - t0 > kWaitNs) {
      *abort = 1;
      return false;
    }
  }
  return true;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_commit(unsigned long long *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
template <int KIND>
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  if constexpr (KIND == kTF32x3) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
  } else {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
  }
}
// 32 lanes x 32 columns of 32-bit accumulators: thread = lane, 32 columns.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
      "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
      "[%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
        "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
        "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int c = 0; c < 32; ++c) v[c] = __uint_as_float(r[c]);
}

// Shared-memory matrix descriptor of one operand block for the MMA at
// 32-byte K step kk: canonical K-major layout without swizzle, core
// matrices of 8 rows x 16 bytes (128 contiguous bytes); the two core
// matrices of one K step are 128 bytes apart (leading byte offset), the
// 8-row groups 1024 bytes apart (stride byte offset); version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc(const void *blk, int kk) {
  const uint32_t a = smem_u32(blk) + 256u * (uint32_t)kk;
  uint64_t d = 0;
  d |= (uint64_t)((a >> 4) & 0x3FFFu);
  d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((1024u >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // version
  // base offset 0, leading-byte-offset mode 0, layout type 0 (no swizzle)
  return d;
}

// Instruction descriptor: FP32 accumulator, A and B of the kind's type
// (TF32 = 2 or BF16 = 1), both K-major, N = 128, M = 128.
template <int KIND>
__host__ __device__ constexpr uint32_t instr_desc() {
  return (1u << 4) | ((KIND == kTF32x3 ? 2u : 1u) << 7) | ((KIND == kTF32x3 ? 2u : 1u) << 10) |
         ((uint32_t)(kBN >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
}

// ---------------------------------------------------------------------------
// Operand split.

__device__ __forceinline__ uint32_t tf32_bits(float x) {
  // to nearest, ties away from zero, at 10 stored mantissa bits (the
  // tensor cores read the top 19 bits of each 32-bit operand)
  const uint32_t b = __float_as_uint(x);
  if ((b & 0x7F800000u) == 0x7F800000u) return b;  // inf / nan
  return (b + 0x1000u) & 0xFFFFE000u;
}

__device__ __forceinline__ double ld_value(const Job &J, int i, int t) {
  // W(i, t) = (L D)(i, t) from the front (fill_ld_column's products,
  // ldlt_kernel.cpp:779-812)
  const double *C = J.C;
  const int64_t ld = J.ld;
  const int c = J.k0 + t;
  const int64_t row = (int64_t)J.r0 + i;
  const double *Lc = C + (int64_t)c * ld;
  if (!J.tags) return Lc[row] * Lc[c];
  const int8_t tag = J.tags[c];
  if (tag == 1) return Lc[row] * Lc[c];
  if (tag == 2) return Lc[row] * Lc[c] + Lc[ld + row] * Lc[c + 1];
  if (tag == -1) {
    const double *L0 = Lc - ld;
    return L0[row] * L0[c] + Lc[row] * Lc[c];
  }
  return 0.0;
}

// Work item: one row i of one job and one 16-byte chunk of one k-block of
// each operand. Images: [op][row block][k-block][16 KB], inside a block the
// core matrix (row group g, chunk q) at (g * 8 + q) * 128 bytes, row i & 7
// at 16 (i & 7) bytes within it.
template <int KIND>
__global__ void __launch_bounds__(256) k_tc_split(const Job *__restrict__ jobs, const int *__restrict__ njobs_p,
                                                  const int64_t *__restrict__ item_pref, uint8_t *__restrict__ img) {
  constexpr int E = (KIND == kTF32x3) ? 4 : 8;  // elements per 16-byte chunk
  constexpr int KE = kRowBytes / ((KIND == kTF32x3) ? 4 : 2);  // elements per k-block row
  const int njobs = *njobs_p;
  const int64_t total = item_pref[njobs];
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < total;
       w += (int64_t)gridDim.x * blockDim.x) {
    int a = 0, b = njobs;
    while (b - a > 1) {
      const int mid = (a + b) >> 1;
      if (item_pref[mid] <= w) a = mid;
      else b = mid;
    }
    const Job J = jobs[a];
    const int64_t loc = w - item_pref[a];
    // items ordered (k-block, chunk, row) so that a warp covers 32 rows
    const int rows = J.ntr * kBM;
    const int i = (int)(loc % rows);
    const int64_t rest = loc / rows;
    const int q = (int)(rest % 8);
    const int kb = (int)(rest / 8);
    uint32_t h[4], l[4], wh[4], wl[4];
    if constexpr (KIND == kTF32x3) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int t = kb * KE + q * E + u;
        double x = 0.0, y = 0.0;
        if (i < J.n && t < J.kc) {
          x = J.Ls[(int64_t)t * J.ldl + J.lr0 + i];
          y = J.Ws ? J.Ws[(int64_t)t * J.ldw + J.wr0 + i] : ld_value(J, i, t);
        }
        const uint32_t xh = tf32_bits((float)x);
        const uint32_t yh = tf32_bits((float)y);
        h[u] = xh;
        l[u] = tf32_bits((float)(x - (double)__uint_as_float(xh)));
        wh[u] = yh;
        wl[u] = tf32_bits((float)(y - (double)__uint_as_float(yh)));
      }
    } else {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        uint32_t ph = 0, pl = 0, qh = 0, ql = 0;
#pragma unroll
        for (int v = 0; v < 2; ++v) {
          const int t = kb * KE + q * E + 2 * u + v;
          double x = 0.0, y = 0.0;
          if (i < J.n && t < J.kc) {
            x = J.Ls[(int64_t)t * J.ldl + J.lr0 + i];
            y = J.Ws ? J.Ws[(int64_t)t * J.ldw + J.wr0 + i] : ld_value(J, i, t);
          }
          const __nv_bfloat16 xh = __double2bfloat16(x);
          const __nv_bfloat16 xl = __double2bfloat16(x - (double)__bfloat162float(xh));
          const __nv_bfloat16 yh = __double2bfloat16(y);
          const __nv_bfloat16 yl = __double2bfloat16(y - (double)__bfloat162float(yh));
          ph |= (uint32_t)__bfloat16_as_ushort(xh) << (16 * v);
          pl |= (uint32_t)__bfloat16_as_ushort(xl) << (16 * v);
          qh |= (uint32_t)__bfloat16_as_ushort(yh) << (16 * v);
          ql |= (uint32_t)__bfloat16_as_ushort(yl) << (16 * v);
        }
        h[u] = ph;
        l[u] = pl;
        wh[u] = qh;
        wl[u] = ql;
      }
    }
    const int rb = i / kBM, ii = i % kBM;
    const int64_t within = (int64_t)((ii >> 3) * 8 + q) * 128 + (ii & 7) * 16;
    const int64_t opstride = (int64_t)J.ntr * J.nkb * kBlkBytes;
    uint8_t *base = img + J.img + ((int64_t)rb * J.nkb + kb) * kBlkBytes + within;
    *reinterpret_cast<uint4 *>(base) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4 *>(base + opstride) = make_uint4(l[0], l[1], l[2], l[3]);
    *reinterpret_cast<uint4 *>(base + 2 * opstride) = make_uint4(wh[0], wh[1], wh[2], wh[3]);
    *reinterpret_cast<uint4 *>(base + 3 * opstride) = make_uint4(wl[0], wl[1], wl[2], wl[3]);
  }
}

// Lower tile number w (column-major over the lower triangle of an ntr x ntr
// tile grid) -> (ti, tj), ti >= tj.
__device__ __forceinline__ void lower_tile(int w, int ntr, int &ti, int &tj) {
  tj = 0;
  int cnt = ntr;
  while (w >= cnt) {
    w -= cnt;
    ++tj;
    --cnt;
  }
  ti = tj + w;
}

__device__ __forceinline__ int find_job(const int *__restrict__ tile_pref, int njobs, int w) {
  int a = 0, b = njobs;
  while (b - a > 1) {
    const int mid = (a + b) >> 1;
    if (tile_pref[mid] <= w) a = mid;
    else b = mid;
  }
  return a;
}

template <int KIND>
__global__ void __launch_bounds__(kThreads, 1)
    k_tc_syrk(const Job *__restrict__ jobs, const int *__restrict__ njobs_p, const int *__restrict__ tile_pref,
              const uint8_t *__restrict__ img, unsigned long long *__restrict__ err, unsigned long long err_bit) {
  extern __shared__ __align__(1024) uint8_t tc_dsm[];
  Smem &sm = *reinterpret_cast<Smem *>(tc_dsm);
  const int njobs = *njobs_p;
  const int total = tile_pref[njobs];
  if ((int)blockIdx.x >= total) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int *abort = &sm.abort;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&sm.acc_full[b], 1);
      mbar_init(&sm.acc_empty[b], 4);
    }
    mbar_init(&sm.drain, 1);
    sm.abort = 0;
    mbar_fence_init();
  }
  if (warp == 1) {
    tmem_alloc(&sm.tmem_base, kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;

  if (warp == 0) {
    // producer
    if (lane == 0) {
      int g = 0;
      for (int w = blockIdx.x; w < total && !*abort; w += gridDim.x) {
        const int a = find_job(tile_pref, njobs, w);
        const Job J = jobs[a];
        int ti, tj;
        lower_tile(w - tile_pref[a], J.ntr, ti, tj);
        const int64_t opstride = (int64_t)J.ntr * J.nkb * kBlkBytes;
        const uint8_t *A = img + J.img + (int64_t)ti * J.nkb * kBlkBytes;
        const uint8_t *B = img + J.img + 2 * opstride + (int64_t)tj * J.nkb * kBlkBytes;
        for (int kb = 0; kb < J.nkb; ++kb, ++g) {
          const int s = g % kStages;
          if (g >= kStages && !mbar_wait(&sm.empty[s], ((g / kStages) - 1) & 1, abort)) break;
          mbar_expect_tx(&sm.full[s], kOps * kBlkBytes);
          bulk_g2s(sm.buf[s][0], A + (int64_t)kb * kBlkBytes, kBlkBytes, &sm.full[s]);
          bulk_g2s(sm.buf[s][1], A + opstride + (int64_t)kb * kBlkBytes, kBlkBytes, &sm.full[s]);
          bulk_g2s(sm.buf[s][2], B + (int64_t)kb * kBlkBytes, kBlkBytes, &sm.full[s]);
          bulk_g2s(sm.buf[s][3], B + opstride + (int64_t)kb * kBlkBytes, kBlkBytes, &sm.full[s]);
        }
      }
      // copies still in flight land before the CTA may exit: the last
      // kStages issued k-blocks complete on their full barriers
      if (*abort) {
        for (int h = max(0, g - kStages); h < g; ++h) {
          const unsigned long long t0 = gtimer();
          while (!mbar_try(&sm.full[h % kStages], (h / kStages) & 1) && gtimer() - t0 < kWaitNs) {
          }
        }
      }
    }
  } else if (warp == 1) {
    // MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = instr_desc<KIND>();
      int g = 0, tcount = 0;
      for (int w = blockIdx.x; w < total && !*abort; w += gridDim.x, ++tcount) {
        const int a = find_job(tile_pref, njobs, w);
        const int nkb = jobs[a].nkb;
        const int buf = tcount & 1;
        if (tcount >= 2 && !mbar_wait(&sm.acc_empty[buf], ((tcount >> 1) - 1) & 1, abort)) break;
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(buf * kBN);
        bool ok = true;
        for (int kb = 0; kb < nkb; ++kb, ++g) {
          const int s = g % kStages;
          if (!mbar_wait(&sm.full[s], (g / kStages) & 1, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int kk = 0; kk < kRowBytes / 32; ++kk) {
            const uint64_t ah = smem_desc(sm.buf[s][0], kk), al = smem_desc(sm.buf[s][1], kk);
            const uint64_t bh = smem_desc(sm.buf[s][2], kk), bl = smem_desc(sm.buf[s][3], kk);
            tc_mma<KIND>(d, ah, bh, idesc, (kb | kk) ? 1u : 0u);
            tc_mma<KIND>(d, ah, bl, idesc, 1u);
            tc_mma<KIND>(d, al, bh, idesc, 1u);
          }
          tc_commit(&sm.empty[s]);
        }
        if (!ok) break;
        tc_commit(&sm.acc_full[buf]);
      }
      // every MMA issued so far completes before tensor memory is freed
      tc_commit(&sm.drain);
      const unsigned long long t0 = gtimer();
      while (!mbar_try(&sm.drain, 0) && gtimer() - t0 < kWaitNs) {
      }
    }
  } else {
    // epilogue: warp w reads accumulator lanes 32 (w % 4) .. + 31
    const int slice = (warp & 3) * 32;
    int tcount = 0;
    for (int w = blockIdx.x; w < total; w += gridDim.x, ++tcount) {
      const int a = find_job(tile_pref, njobs, w);
      const Job J = jobs[a];
      int ti, tj;
      lower_tile(w - tile_pref[a], J.ntr, ti, tj);
      const int buf = tcount & 1;
      // warp-uniform: the tensor-memory loads below are warp-collective
      const bool ok = mbar_wait(&sm.acc_full[buf], (tcount >> 1) & 1, abort);
      if (!__all_sync(0xffffffffu, ok)) break;
      tc_fence_after();
      const int i = ti * kBM + slice + lane;
      double *Ccol = J.C + (int64_t)J.r0 * J.ld + J.r0 + i;
#pragma unroll 1
      for (int ch = 0; ch < kBN / 32; ++ch) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)slice << 16) + (uint32_t)(buf * kBN + ch * 32), v);
        const int j0 = tj * kBN + ch * 32;
        if (i < J.n) {
          // all 32 loads in flight before the stores (a warp covers 32
          // consecutive rows of each column: coalesced)
          const int jn = min(32, i - j0 + 1);  // columns j0 .. j0 + jn - 1 are <= i
          double cv[32];
#pragma unroll
          for (int c = 0; c < 32; ++c)
            cv[c] = (c < jn) ? __ldcg(Ccol + (int64_t)(j0 + c) * J.ld) : 0.0;
#pragma unroll
          for (int c = 0; c < 32; ++c)
            if (c < jn) Ccol[(int64_t)(j0 + c) * J.ld] = cv[c] - (double)v[c];
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.acc_empty[buf]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0 && sm.abort) atomicOr(err, err_bit);
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

}  // namespace tc
}  // namespace smfg
