// Host side of the B200 numeric phase: device plan from smf's analysis,
// the level-by-level factorization, solves, residual and refinement, and
// the C ABI declared in include/smfg.h.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <vector>

#include "smfg_kernels.cuh"
#include "smfg_tc.cuh"

namespace smfg {

namespace {

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t c, const char *what) : std::runtime_error(what), code(c) {}
};

#define SMFG_CUDA(call)                                                              \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) throw CudaError(e_, cudaGetErrorString(e_));             \
  } while (0)

template <class T>
T *dalloc(Plan &pl, size_t count) {
  void *p = nullptr;
  if (count == 0) count = 1;
  SMFG_CUDA(cudaMalloc(&p, count * sizeof(T)));
  pl.allocs.push_back(p);
  return static_cast<T *>(p);
}

template <class T>
T *dupload(Plan &pl, const std::vector<T> &v) {
  T *p = dalloc<T>(pl, v.size());
  if (!v.empty()) SMFG_CUDA(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, pl.stream));
  return p;
}

void dfree(Plan &pl, void *p) {
  if (!p) return;
  auto it = std::find(pl.allocs.begin(), pl.allocs.end(), p);
  if (it != pl.allocs.end()) pl.allocs.erase(it);
  cudaFree(p);
}

thread_local std::string g_last_error;

void set_last_error(const char *what) { g_last_error = what ? what : ""; }

// Clears an error left by earlier CUDA calls of the process (not sticky
// ones, which keep failing), so that it is not reported as this call's.
void clear_stale_error() { (void)cudaGetLastError(); }

int sm_count(int dev) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  return v > 0 ? v : 148;
}

// Dynamic shared memory of the in-shared-memory front kernels.
size_t front_smem_bytes(int fmax, int nb) {
  return (size_t)fmax * fmax * 8 + (size_t)fmax * nb * 8 + (size_t)fmax * 12 + (size_t)fmax + 64;
}

}  // namespace

// ---------------------------------------------------------------------------
// Plan creation (per analysis).

static void build_plan(Plan &pl, const smfg_analysis_t &a) {
  const int n = a.n, ns = a.nsn;
  pl.n = n;
  pl.nsn = ns;
  pl.nnz = a.perm_col_ptr[n];
  pl.nnz_in = a.nnz_in;
  // level = height above the leaves; postorder numbering (children first)
  std::vector<int> width(ns), fsym(ns), level(ns, 0);
  for (int s = 0; s < ns; ++s) {
    width[s] = a.sn_end[s] - a.sn_start[s];
    fsym[s] = a.front_row_ptr[s + 1] - a.front_row_ptr[s];
    if (width[s] <= 0 || fsym[s] < width[s]) throw std::invalid_argument("bad supernode");
  }
  for (int i = 0; i < ns; ++i) {
    const int s = a.postorder[i];
    int lv = 0;
    for (int t = a.child_ptr[s]; t < a.child_ptr[s + 1]; ++t) lv = std::max(lv, level[a.child_idx[t]] + 1);
    level[s] = lv;
  }
  int nl = 0;
  for (int s = 0; s < ns; ++s) nl = std::max(nl, level[s] + 1);
  pl.nlevels = nl;
  pl.lvl_ptr.assign(nl + 1, 0);
  for (int s = 0; s < ns; ++s) pl.lvl_ptr[level[s] + 1]++;
  for (int l = 0; l < nl; ++l) pl.lvl_ptr[l + 1] += pl.lvl_ptr[l];
  std::vector<int> lvl_sn(ns), fill(pl.lvl_ptr.begin(), pl.lvl_ptr.end() - 1);
  for (int i = 0; i < ns; ++i) {
    const int s = a.postorder[i];
    lvl_sn[fill[level[s]]++] = s;
  }
  // large fronts (multi-block path), by level, in the level's order
  pl.lvl_large_ptr.assign(nl + 1, 0);
  pl.lvl_large_maxw.assign(nl, 0);
  pl.lvl_large_maxf.assign(nl, 0);
  std::vector<int> lvl_large;
  for (int l = 0; l < nl; ++l) {
    for (int i = pl.lvl_ptr[l]; i < pl.lvl_ptr[l + 1]; ++i) {
      const int s = lvl_sn[i];
      if (fsym[s] >= kLargeMin) {
        lvl_large.push_back(s);
        pl.lvl_large_maxw[l] = std::max(pl.lvl_large_maxw[l], width[s]);
        pl.lvl_large_maxf[l] = std::max(pl.lvl_large_maxf[l], fsym[s]);
      }
    }
    pl.lvl_large_ptr[l + 1] = (int)lvl_large.size();
    pl.max_large = std::max(pl.max_large, pl.lvl_large_ptr[l + 1] - pl.lvl_large_ptr[l]);
  }
  pl.lvl_maxf.assign(nl, 0);
  pl.lvl_maxkids.assign(nl, 0);
  for (int s = 0; s < ns; ++s) {
    pl.lvl_maxf[level[s]] = std::max(pl.lvl_maxf[level[s]], fsym[s]);
    pl.lvl_maxkids[level[s]] = std::max(pl.lvl_maxkids[level[s]], a.child_ptr[s + 1] - a.child_ptr[s]);
  }
  // child -> parent symbolic row positions
  const int nslots = a.child_ptr[ns];
  std::vector<int> cpr_off(nslots + 1, 0), cpr_idx;
  for (int s = 0; s < ns; ++s) {
    const int *pr = a.front_row_idx + a.front_row_ptr[s];
    for (int t = a.child_ptr[s]; t < a.child_ptr[s + 1]; ++t) {
      const int c = a.child_idx[t];
      if (a.sn_parent[c] != s) throw std::invalid_argument("child list and parent links disagree");
      const int *cr = a.front_row_idx + a.front_row_ptr[c];
      for (int u = width[c]; u < fsym[c]; ++u) {
        const int *hit = std::lower_bound(pr, pr + fsym[s], cr[u]);
        if (hit == pr + fsym[s] || *hit != cr[u])
          throw std::invalid_argument("child row outside the parent's front");
        const int pos = (int)(hit - pr);
        if (!cpr_idx.empty() && u > width[c] && pos <= cpr_idx.back())
          throw std::invalid_argument("unsorted front rows");
        cpr_idx.push_back(pos);
      }
      cpr_off[t + 1] = (int)cpr_idx.size();
    }
  }
  // original entries -> symbolic row position in their supernode's front
  std::vector<int> col_sn(n, -1);
  for (int s = 0; s < ns; ++s)
    for (int j = a.sn_start[s]; j < a.sn_end[s]; ++j) col_sn[j] = s;
  std::vector<int> amap(pl.nnz), pcol(pl.nnz);
  for (int j = 0; j < n; ++j) {
    const int s = col_sn[j];
    if (s < 0) throw std::invalid_argument("column in no supernode");
    const int *pr = a.front_row_idx + a.front_row_ptr[s];
    for (int k = a.perm_col_ptr[j]; k < a.perm_col_ptr[j + 1]; ++k) {
      const int *hit = std::lower_bound(pr, pr + fsym[s], a.perm_row_idx[k]);
      if (hit == pr + fsym[s] || *hit != a.perm_row_idx[k])
        throw std::invalid_argument("entry outside its front");
      amap[k] = (int)(hit - pr);
      pcol[k] = j;
    }
  }
  // caller entry -> permuted slot (input order within a slot)
  std::vector<int> vptr(pl.nnz + 1, 0), vsrc;
  std::vector<int> slot_of(a.nnz_in, -1);
  for (int64_t k = 0; k < a.nnz_in; ++k) {
    const int c = a.orig_to_clean[k];
    if (c >= 0) {
      slot_of[k] = a.clean_to_perm[c];
      vptr[slot_of[k] + 1]++;
    }
  }
  for (int64_t s = 0; s < pl.nnz; ++s) vptr[s + 1] += vptr[s];
  vsrc.resize(vptr[pl.nnz]);
  {
    std::vector<int> pos(vptr.begin(), vptr.end() - 1);
    for (int64_t k = 0; k < a.nnz_in; ++k)
      if (slot_of[k] >= 0) vsrc[pos[slot_of[k]]++] = (int)k;
  }
  // full symmetric CSR (new numbering) for the residual
  std::vector<int> sptr(n + 1, 0);
  for (int j = 0; j < n; ++j)
    for (int k = a.perm_col_ptr[j]; k < a.perm_col_ptr[j + 1]; ++k) {
      const int i = a.perm_row_idx[k];
      sptr[i + 1]++;
      if (i != j) sptr[j + 1]++;
    }
  for (int i = 0; i < n; ++i) sptr[i + 1] += sptr[i];
  std::vector<int> scol(sptr[n]);
  std::vector<int64_t> sidx(sptr[n]);
  {
    std::vector<int> pos(sptr.begin(), sptr.end() - 1);
    for (int j = 0; j < n; ++j)
      for (int k = a.perm_col_ptr[j]; k < a.perm_col_ptr[j + 1]; ++k) {
        const int i = a.perm_row_idx[k];
        scol[pos[i]] = j;
        sidx[pos[i]++] = k;
        if (i != j) {
          scol[pos[j]] = i;
          sidx[pos[j]++] = k;
        }
      }
  }
  pl.sum_f2 = 0;
  pl.sum_f = 0;
  pl.max_fsym = 0;
  for (int s = 0; s < ns; ++s) {
    pl.sum_f2 += (int64_t)fsym[s] * fsym[s] + (int64_t)fsym[s] * pl.nb;
    pl.sum_f += fsym[s];
    pl.max_fsym = std::max(pl.max_fsym, fsym[s]);
  }
  pl.h_child_ptr.assign(a.child_ptr, a.child_ptr + ns + 1);
  pl.h_child_idx.assign(a.child_idx, a.child_idx + nslots);
  pl.h_sn_parent.assign(a.sn_parent, a.sn_parent + ns);
  pl.h_postorder.assign(a.postorder, a.postorder + ns);

  // upload
  DevPlan &d = pl.d;
  d.n = n;
  d.nsn = ns;
  d.nlevels = nl;
  d.nnz = pl.nnz;
  d.nnz_in = a.nnz_in;
  d.sn_start = dupload(pl, std::vector<int>(a.sn_start, a.sn_start + ns));
  d.sn_width = dupload(pl, width);
  d.sn_fsym = dupload(pl, fsym);
  d.sn_parent = dupload(pl, pl.h_sn_parent);
  d.child_ptr = dupload(pl, pl.h_child_ptr);
  d.child_idx = dupload(pl, pl.h_child_idx);
  d.frow_ptr = dupload(pl, std::vector<int>(a.front_row_ptr, a.front_row_ptr + ns + 1));
  d.frow_idx = dupload(pl, std::vector<int>(a.front_row_idx, a.front_row_idx + a.front_row_ptr[ns]));
  d.cpr_off = dupload(pl, cpr_off);
  d.cpr_idx = dupload(pl, cpr_idx);
  d.lvl_sn = dupload(pl, lvl_sn);
  d.lvl_large = dupload(pl, lvl_large);
  pl.h_lvl_large = lvl_large;
  d.sn_level = dupload(pl, level);
  d.pcp = dupload(pl, std::vector<int>(a.perm_col_ptr, a.perm_col_ptr + n + 1));
  d.pri = dupload(pl, std::vector<int>(a.perm_row_idx, a.perm_row_idx + pl.nnz));
  d.amap = dupload(pl, amap);
  d.vptr = dupload(pl, vptr);
  d.vsrc = dupload(pl, vsrc);
  d.perm = dupload(pl, std::vector<int>(a.perm, a.perm + n));
  d.sptr = dupload(pl, sptr);
  d.srow = dupload(pl, scol);
  d.sidx = dupload(pl, sidx);
  d.pcol = dupload(pl, pcol);

  // per-factorization state
  DevFactor &x = pl.x;
  x.pv = dalloc<double>(pl, pl.nnz);
  x.pv_raw = dalloc<double>(pl, pl.nnz);
  x.scale = dalloc<double>(pl, n);
  x.sn_nd = dalloc<int>(pl, ns);
  x.sn_f = dalloc<int>(pl, ns);
  x.sn_ne = dalloc<int>(pl, ns);
  x.sn_p = dalloc<int>(pl, ns);
  x.sn_pstore = dalloc<int>(pl, ns);
  x.sn_dout = dalloc<int>(pl, ns);
  x.sn_off = dalloc<int64_t>(pl, ns);
  x.sn_roff = dalloc<int64_t>(pl, ns);
  x.child_doff = dalloc<int>(pl, nslots);
  x.sn_stat = dalloc<int>(pl, 4 * (size_t)ns);
  x.sn_flops = dalloc<double>(pl, ns);
  x.lvl_blk = dalloc<int>(pl, (size_t)ns + nl + 1);
  x.counters = dalloc<unsigned long long>(pl, kCCount + 8);
  x.tpp = dalloc<TppState>(pl, 2 * (size_t)std::max(1, pl.max_large));  // two buffers (SPD panels)
  x.arena = nullptr;
  x.arena_cap = 0;
  x.rows = nullptr;
  x.rows_cap = 0;
}

static void ensure_arena(Plan &pl, int64_t arena_need, int64_t rows_need) {
  DevFactor &x = pl.x;
  if (x.arena_cap < arena_need) {
    dfree(pl, x.arena);
    x.arena = dalloc<double>(pl, arena_need);
    x.arena_cap = arena_need;
  }
  if (x.rows_cap < rows_need) {
    dfree(pl, x.rows);
    dfree(pl, x.tags);
    dfree(pl, x.cbmap);
    dfree(pl, x.ploc);
    x.rows = dalloc<int>(pl, rows_need);
    x.tags = dalloc<int8_t>(pl, rows_need);
    x.cbmap = dalloc<int>(pl, rows_need);
    x.ploc = dalloc<int>(pl, 2 * (size_t)rows_need);
    x.rows_cap = rows_need;
  }
}

// ---------------------------------------------------------------------------
// Factorization.

struct LaunchCount {
  int n = 0;
};

// Optional per-launch timing of the large-front GEMM kernels (events on the
// engine's stream around each launch).
struct GemmProfile {
  bool on = false;
  std::vector<cudaEvent_t> ev;
  size_t used = 0;
  void mark(cudaStream_t st) {
    if (!on) return;
    if (used == ev.size()) {
      cudaEvent_t e;
      SMFG_CUDA(cudaEventCreate(&e));
      ev.push_back(e);
    }
    SMFG_CUDA(cudaEventRecord(ev[used++], st));
  }
  double total_ms() {
    double t = 0.0;
    for (size_t i = 0; i + 1 < used; i += 2) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
      t += ms;
    }
    return t;
  }
  ~GemmProfile() {
    for (auto e : ev) cudaEventDestroy(e);
  }
};

static void enqueue_factor(Plan &pl, const double *d_values, const smfg_control_t &c, LaunchCount &lc,
                           GemmProfile &gp) {
  DevPlan &d = pl.d;
  DevFactor &x = pl.x;
  cudaStream_t st = pl.stream;
  const int sms = sm_count(pl.device);
  SMFG_CUDA(cudaMemsetAsync(x.counters, 0, sizeof(unsigned long long) * kCCount, st));
  SMFG_CUDA(cudaMemsetAsync(x.sn_dout, 0, sizeof(int) * pl.nsn, st));
  const double *scale = nullptr;
  if (c.scale) {
    SMFG_CUDA(cudaMemcpyAsync(x.scale, c.scale, sizeof(double) * pl.n, cudaMemcpyHostToDevice, st));
    scale = x.scale;
  }
  const int *pcol = d.pcol;
  const int vgrid = (int)std::max<int64_t>(1, std::min<int64_t>(4 * sms, (std::max(pl.nnz, pl.nnz_in) + 255) / 256));
  k_values<<<vgrid, 256, 0, st>>>(
      d_values, pl.nnz_in, d.vptr, d.vsrc, pcol, d.pri, d.perm, scale, pl.nnz, x.pv, x.pv_raw,
      x.counters);
  k_eff_small<<<1, 1, 0, st>>>(x.counters, c.small_pivot);
  lc.n += 2;
  PivotParams prm{c.u, c.small_pivot, c.small_pivot, c.nb, c.blocked_min_front, c.posdef};
  const size_t smem_s = front_smem_bytes(kSmallMax, c.nb);
  const size_t smem_m = front_smem_bytes(kMediumMax, c.nb);
  for (int l = 0; l < pl.nlevels; ++l) {
    const int lo = pl.lvl_ptr[l], hi = pl.lvl_ptr[l + 1], m = hi - lo;
    k_level_setup<1024><<<1, 1024, 0, st>>>(d, x, lo, hi, l, c.nb);
    k_level_rows<<<m, 128, 0, st>>>(d, x, lo, hi);
    const int asm_grid = std::max(1, std::min(4 * sms, m * 64));
    k_level_assemble<<<asm_grid, 256, 0, st>>>(d, x, lo, hi, l);
    k_factor<32, 1, kSmallMax, true><<<m, 32, smem_s, st>>>(d, x, lo, hi, prm);
    k_factor<128, kSmallMax + 1, kMediumMax, true><<<m, 128, smem_m, st>>>(d, x, lo, hi, prm);
    k_factor<512, kMediumMax + 1, 1 << 30, false><<<m, 512, 0, st>>>(d, x, lo, hi, prm);
    lc.n += 6;
    const int nL = pl.lvl_large_ptr[l + 1] - pl.lvl_large_ptr[l];
    if (nL > 0) {
      const int *lg = d.lvl_large + pl.lvl_large_ptr[l];
      k_large_init<<<nL, 256, 0, st>>>(d, x, lg, nL, c.posdef);
      SMFG_CUDA(cudaMemsetAsync(x.counters + kCActive, 0, sizeof(unsigned long long), st));
      const int ggrid = 2 * sms;
      int it = 0;
      TppState *fin = x.tpp;  // where the final state of the level's fronts ends up
      if (c.posdef && c.nb == 16) {
        // no delays, no search: one multi-block step per panel, states
        // double-buffered; the closing step leaves phase 2
        const int steps = (pl.lvl_large_maxw[l] + c.nb - 1) / c.nb + 1;
        const dim3 pgrid((pl.lvl_large_maxf[l] + 255) / 256, nL);
        for (; it < steps; ++it) {
          TppState *cur = x.tpp + (size_t)(it & 1) * pl.max_large;
          TppState *nxt = x.tpp + (size_t)((it + 1) & 1) * pl.max_large;
          k_large_panel_spd<16><<<pgrid, 256, 0, st>>>(d, x, lg, cur, nxt, it);
          gp.mark(st);
          k_large_gemm<<<ggrid, 256, sizeof(TileSmem), st>>>(d, x, lg, nL, nxt);
          gp.mark(st);
        }
        fin = x.tpp + (size_t)(steps & 1) * pl.max_large;
        lc.n += 2 * steps;
      } else if (c.posdef) {
        const int steps = (pl.lvl_large_maxw[l] + c.nb - 1) / c.nb + 1;
        for (; it < steps; ++it) {
          k_large_panel<512><<<nL, 512, 0, st>>>(d, x, lg, prm, it);
          gp.mark(st);
          k_large_gemm<<<ggrid, 256, sizeof(TileSmem), st>>>(d, x, lg, nL, x.tpp);
          gp.mark(st);
        }
        lc.n += 2 * steps;
      } else {
        // data-dependent: batches, then a look at the last step that
        // still asked for an update
        const int batch = 32;
        for (int guard = 0; guard < 1 << 20; guard += batch) {
          for (int b = 0; b < batch; ++b, ++it) {
            k_large_panel<512><<<nL, 512, 0, st>>>(d, x, lg, prm, it);
            gp.mark(st);
            k_large_gemm<<<ggrid, 256, sizeof(TileSmem), st>>>(d, x, lg, nL, x.tpp);
            gp.mark(st);
          }
          lc.n += 2 * batch;
          unsigned long long act = 0;
          SMFG_CUDA(cudaMemcpyAsync(&act, x.counters + kCActive, sizeof(act), cudaMemcpyDeviceToHost, st));
          SMFG_CUDA(cudaStreamSynchronize(st));
          if (act < (unsigned long long)it) break;
        }
      }
      gp.mark(st);
      k_large_schur<<<ggrid, 256, sizeof(TileSmem), st>>>(d, x, lg, nL, fin);
      gp.mark(st);
      k_large_finish<512><<<nL, 512, 0, st>>>(d, x, lg, fin, prm);
      k_large_store<<<ggrid, 256, 0, st>>>(d, x, lg, nL, c.posdef);
      lc.n += 4;
    }
  }
  SMFG_CUDA(cudaGetLastError());
}

static void set_kernel_attrs(int nb) {
  static int done_nb = -1;
  if (done_nb == nb) return;
  SMFG_CUDA(cudaFuncSetAttribute(k_factor<32, 1, kSmallMax, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)front_smem_bytes(kSmallMax, nb)));
  SMFG_CUDA(cudaFuncSetAttribute(k_factor<128, kSmallMax + 1, kMediumMax, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)front_smem_bytes(kMediumMax, nb)));
  SMFG_CUDA(cudaFuncSetAttribute(k_large_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TileSmem)));
  SMFG_CUDA(cudaFuncSetAttribute(k_large_schur, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TileSmem)));
  done_nb = nb;
}

static int run_factor(Plan &pl, const double *d_values, const smfg_control_t &c, smfg_info_t *info) {
  SMFG_CUDA(cudaSetDevice(pl.device));
  pl.nb = std::max(2, c.nb);
  set_kernel_attrs(pl.nb);
  // arena: exact for SPD (no delays); head-room for delays, regrown on overflow
  const int64_t base_a = pl.sum_f2, base_r = pl.sum_f;
  int64_t need_a = c.posdef ? base_a : base_a + base_a / 4 + (int64_t)pl.max_fsym * pl.max_fsym * 2 + 4096;
  int64_t need_r = c.posdef ? base_r : base_r + base_r / 2 + 4096;
  FactorTotals *d_tot = nullptr;
  unsigned long long h_cnt[kCCount];
  FactorTotals tot{};
  LaunchCount lc;
  GemmProfile gp;
  gp.on = c.reserved_i[0] != 0;
  float ms = 0.0f;
  for (int attempt = 0; attempt < 4; ++attempt) {
    ensure_arena(pl, std::max(need_a, pl.x.arena_cap), std::max(need_r, pl.x.rows_cap));
    lc = LaunchCount{};
    gp.used = 0;
    SMFG_CUDA(cudaEventRecord(pl.ev0, pl.stream));
    enqueue_factor(pl, d_values, c, lc, gp);
    if (!d_tot) d_tot = reinterpret_cast<FactorTotals *>(pl.x.counters + kCCount);
    static_assert(sizeof(FactorTotals) <= 8 * sizeof(unsigned long long), "totals slot");
    k_finish<<<1, 1024, 0, pl.stream>>>(pl.d, pl.x, d_tot);
    lc.n += 1;
    SMFG_CUDA(cudaEventRecord(pl.ev1, pl.stream));
    SMFG_CUDA(cudaMemcpyAsync(h_cnt, pl.x.counters, sizeof(h_cnt), cudaMemcpyDeviceToHost, pl.stream));
    SMFG_CUDA(cudaMemcpyAsync(&tot, d_tot, sizeof(tot), cudaMemcpyDeviceToHost, pl.stream));
    SMFG_CUDA(cudaStreamSynchronize(pl.stream));
    SMFG_CUDA(cudaEventElapsedTime(&ms, pl.ev0, pl.ev1));
    const unsigned flags = (unsigned)h_cnt[kCFlags];
    if (flags & (kFArena | kFRows)) {
      need_a = std::max<int64_t>(need_a * 2, (int64_t)h_cnt[kCArena] * 2);
      need_r = std::max<int64_t>(need_r * 2, (int64_t)h_cnt[kCRows] * 2);
      continue;
    }
    break;
  }
  const unsigned flags = (unsigned)h_cnt[kCFlags];
  // stored pivots of the large fronts by level (the solves' block counts)
  pl.lvl_large_pmax.assign(pl.nlevels, 0);
  if (!pl.h_lvl_large.empty()) {
    std::vector<int> pst(pl.nsn);
    SMFG_CUDA(cudaMemcpy(pst.data(), pl.x.sn_pstore, sizeof(int) * pl.nsn, cudaMemcpyDeviceToHost));
    for (int l = 0; l < pl.nlevels; ++l)
      for (int i = pl.lvl_large_ptr[l]; i < pl.lvl_large_ptr[l + 1]; ++i)
        pl.lvl_large_pmax[l] = std::max(pl.lvl_large_pmax[l], pst[pl.h_lvl_large[i]]);
  }
  smfg_info_t inf{};
  inf.status = SMFG_OK;
  inf.num_pos = (int)tot.pos;
  inf.num_neg = (int)tot.neg;
  inf.num_zero = (int)tot.zero;
  inf.delayed_pivots = (int)tot.delayed;
  inf.two_by_two_pivots = (int)tot.two_by_two;
  inf.max_front = tot.max_front;
  inf.factor_entries = tot.entries;
  inf.flops = tot.flops;
  std::memcpy(&inf.max_abs, &h_cnt[kCMaxAbs], sizeof(double));
  inf.factor_ms = ms;
  inf.levels = pl.nlevels;
  inf.kernel_launches = lc.n;
  // profile (ctrl.reserved_i[0]): large-front GEMM device time, launches,
  // algorithmic flops; arena bytes in use
  inf.reserved_d[0] = gp.on ? gp.total_ms() : 0.0;
  std::memcpy(&inf.reserved_d[1], &h_cnt[kCGemmFlops], sizeof(double));
  inf.reserved_d[2] = (double)h_cnt[kCArena] * 8.0;
  inf.reserved_i[0] = (int)(gp.used / 2);
  int rc = SMFG_OK;
  pl.factor_status = SMFG_FACTOR_SUCCESS;
  if (flags & (kFArena | kFRows)) rc = SMFG_ERR_ARENA;
  else if (flags & kFNonfinite) rc = SMFG_ERR_NONFINITE;
  else if (flags & (kFMap | kFInternal)) rc = SMFG_ERR_INTERNAL;
  else if (flags & kFNotPosdef) {
    rc = SMFG_ERR_SINGULAR;
    pl.factor_status = SMFG_FACTOR_NOT_POSDEF;
  } else if (flags & kFNonfiniteD) {
    rc = SMFG_ERR_NONFINITE;
    pl.factor_status = SMFG_FACTOR_SINGULAR;
  } else if (tot.zero > 0) {
    rc = SMFG_ERR_SINGULAR;
    pl.factor_status = SMFG_FACTOR_SINGULAR;
  } else if (c.max_negative_pivots >= 0 && tot.neg > c.max_negative_pivots) {
    rc = SMFG_ERR_WRONG_INERTIA;
    pl.factor_status = SMFG_FACTOR_INERTIA_EXCEEDED;
  }
  if (c.posdef && rc == SMFG_OK) {
    inf.num_pos = pl.n;
    inf.num_neg = inf.num_zero = 0;
  }
  inf.status = rc;
  inf.factor_status = pl.factor_status;
  pl.posdef = c.posdef;
  pl.factored = (rc == SMFG_OK || rc == SMFG_ERR_SINGULAR) && pl.factor_status != SMFG_FACTOR_NOT_POSDEF;
  pl.info = inf;
  if (info) *info = inf;
  return rc;
}

// ---------------------------------------------------------------------------
// Solve.

static void ensure_work(Plan &pl, int64_t need) {
  if (pl.x.work_cap < need) {
    dfree(pl, pl.x.work);
    pl.x.work = dalloc<double>(pl, need);
    pl.x.work_cap = need;
  }
}

// Upper bound of the stored pivots of level l's large fronts: their width
// (SPD: no delays), else their symbolic rows (delays may add pivots).
static int large_pmax(const Plan &pl, int l) {
  return l < (int)pl.lvl_large_pmax.size() ? pl.lvl_large_pmax[l] : pl.lvl_large_maxf[l];
}

static void enqueue_solve(Plan &pl, double *d_b, int nrhs, int ldb, int job, bool scaled, LaunchCount &lc) {
  DevPlan &d = pl.d;
  DevFactor &x = pl.x;
  cudaStream_t st = pl.stream;
  const int64_t rows_total = std::max<int64_t>(1, (int64_t)x.rows_cap);
  const int64_t xlen = (int64_t)pl.n * nrhs;
  ensure_work(pl, xlen + rows_total * nrhs + 16);
  double *xv = x.work;
  double *wk = x.work + xlen;
  const int sms = sm_count(pl.device);
  const int g = (int)std::max<int64_t>(1, std::min<int64_t>(4 * sms, (xlen + 255) / 256));
  // solve_core's jobs (solve.cpp:858-1075): the full solve takes S on both
  // sides; the forward sweep P L X = S B scales its input only, the backward
  // sweep (P L)^T S^-1 X = B its output only, the diagonal solve neither.
  const bool fwd = job == SMFG_SOLVE_FULL || job == SMFG_SOLVE_FORWARD;
  const bool use_d = job == SMFG_SOLVE_FULL || job == SMFG_SOLVE_DIAGONAL;
  const bool use_lt = job == SMFG_SOLVE_FULL || job == SMFG_SOLVE_BACKWARD;
  const double *sc_in = (scaled && fwd) ? x.scale : nullptr;
  const double *sc_out = (scaled && (job == SMFG_SOLVE_FULL || job == SMFG_SOLVE_BACKWARD)) ? x.scale : nullptr;
  k_solve_gather<<<g, 256, 0, st>>>(d_b, ldb, nrhs, pl.n, d.perm, sc_in, xv);
  lc.n++;
  const int lgrid = 2 * sms;
  if (fwd) {
    for (int l = 0; l < pl.nlevels; ++l) {
      const int lo = pl.lvl_ptr[l], m = pl.lvl_ptr[l + 1] - lo;
      k_fwd_front<<<m, kSolveNT, 0, st>>>(d, x, lo, pl.posdef, xv, wk, rows_total, nrhs);
      lc.n++;
      const int nL = pl.lvl_large_ptr[l + 1] - pl.lvl_large_ptr[l];
      if (nL > 0) {
        const int *lg = d.lvl_large + pl.lvl_large_ptr[l];
        const int nb = (large_pmax(pl, l) + kSB - 1) / kSB;
        for (int b = 0; b < nb; ++b) {
          k_fwd_tri<<<nL, kSolveNT, 0, st>>>(d, x, lg, b, pl.posdef, xv, wk, rows_total, nrhs);
          k_fwd_gemv<<<lgrid, 256, 0, st>>>(d, x, lg, nL, b, wk, rows_total, nrhs);
        }
        lc.n += 2 * nb;
      }
    }
  }
  if (use_lt || (use_d && !pl.posdef)) {
    for (int l = pl.nlevels - 1; l >= 0; --l) {
      const int lo = pl.lvl_ptr[l], m = pl.lvl_ptr[l + 1] - lo;
      const int nL = pl.lvl_large_ptr[l + 1] - pl.lvl_large_ptr[l];
      if (nL > 0 && use_lt) {
        k_bwd_l21<<<lgrid, 256, 0, st>>>(d, x, d.lvl_large + pl.lvl_large_ptr[l], nL, xv, wk, rows_total, nrhs);
        lc.n++;
      }
      k_bwd_front<<<m, kSolveNT, 0, st>>>(d, x, lo, pl.posdef, xv, wk, rows_total, nrhs,
                                          use_d ? 1 : 0, use_lt ? 1 : 0);
      lc.n++;
      if (nL > 0 && use_lt) {
        const int *lg = d.lvl_large + pl.lvl_large_ptr[l];
        const int nb = (large_pmax(pl, l) + kSB - 1) / kSB;
        for (int b = nb - 1; b >= 0; --b) {
          k_bwd_dots<<<lgrid, 256, 0, st>>>(d, x, lg, nL, b, wk, rows_total, nrhs);
          k_bwd_tri<<<nL, kSolveNT, 0, st>>>(d, x, lg, b, pl.posdef, xv, wk, rows_total, nrhs);
        }
        lc.n += 2 * nb;
      }
    }
  }
  k_solve_scatter<<<g, 256, 0, st>>>(d_b, ldb, nrhs, pl.n, d.perm, sc_out, xv);
  lc.n++;
  SMFG_CUDA(cudaGetLastError());
}

}  // namespace smfg

// ===========================================================================
// C ABI

using namespace smfg;

struct smfg_plan_s {
  Plan pl;
  bool has_scale = false;
};

extern "C" {

SMFG_API int smfg_abi_version(void) { return SMFG_ABI_VERSION; }

SMFG_API void smfg_default_control(smfg_control_t *c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->abi_version = SMFG_ABI_VERSION;
  c->posdef = 0;
  c->u = 0.01;             // Control::pivot_u
  c->small_pivot = 1e-20;  // Control::small_pivot
  c->nb = 16;              // Control::indef_panel_size
  c->blocked_min_front = 96;
  c->precision = SMFG_PREC_FP64;
  c->max_negative_pivots = -1;
  c->scale = nullptr;
}

SMFG_API const char *smfg_last_error(void) { return g_last_error.c_str(); }

SMFG_API const char *smfg_error_string(int code) {
  switch (code) {
    case SMFG_OK: return "ok";
    case SMFG_ERR_INVALID_ARG: return "invalid argument";
    case SMFG_ERR_SINGULAR: return "singular or not positive definite";
    case SMFG_ERR_INTERNAL: return "internal error";
    case SMFG_ERR_WRONG_INERTIA: return "more negative pivots than allowed";
    case SMFG_ERR_INEXACT_INERTIA: return "inexact inertia";
    case SMFG_ERR_CUDA: return "CUDA runtime error";
    case SMFG_ERR_NO_DEVICE: return "no CUDA device";
    case SMFG_ERR_NONFINITE: return "non-finite values";
    case SMFG_ERR_ARENA: return "device arena too small";
    case SMFG_ERR_TIMEOUT: return "bounded device wait gave up";
    default: return "unknown error";
  }
}

SMFG_API int smfg_plan_create(const smfg_analysis_t *a, int device, smfg_plan_t *out) {
  if (!a || !out || a->n < 0 || a->nsn < 0) return SMFG_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SMFG_ERR_NO_DEVICE;
  auto *h = new smfg_plan_s();
  try {
    if (device < 0) SMFG_CUDA(cudaGetDevice(&device));
    h->pl.device = device;
    SMFG_CUDA(cudaSetDevice(device));
    SMFG_CUDA(cudaStreamCreateWithFlags(&h->pl.stream, cudaStreamNonBlocking));
    SMFG_CUDA(cudaEventCreate(&h->pl.ev0));
    SMFG_CUDA(cudaEventCreate(&h->pl.ev1));
    h->pl.nb = 16;
    build_plan(h->pl, *a);
    SMFG_CUDA(cudaStreamSynchronize(h->pl.stream));
  } catch (const std::invalid_argument &) {
    smfg_plan_t p = h;
    smfg_plan_destroy(&p);
    return SMFG_ERR_INVALID_ARG;
  } catch (const CudaError &) {
    smfg_plan_t p = h;
    smfg_plan_destroy(&p);
    return SMFG_ERR_CUDA;
  } catch (...) {
    smfg_plan_t p = h;
    smfg_plan_destroy(&p);
    return SMFG_ERR_INTERNAL;
  }
  *out = h;
  return SMFG_OK;
}

SMFG_API void smfg_plan_destroy(smfg_plan_t *plan) {
  if (!plan || !*plan) return;
  Plan &pl = (*plan)->pl;
  cudaSetDevice(pl.device);
  if (pl.stream) cudaStreamSynchronize(pl.stream);
  for (void *p : pl.allocs) cudaFree(p);
  if (pl.ev0) cudaEventDestroy(pl.ev0);
  if (pl.ev1) cudaEventDestroy(pl.ev1);
  if (pl.stream) cudaStreamDestroy(pl.stream);
  delete *plan;
  *plan = nullptr;
}

static int factor_common(smfg_plan_t plan, const double *values, bool on_device,
                         const smfg_control_t *ctrl, smfg_info_t *info) {
  if (!plan || !values) return SMFG_ERR_INVALID_ARG;
  smfg_control_t c;
  if (ctrl) c = *ctrl;
  else smfg_default_control(&c);
  if (c.nb < 2) c.nb = 16;
  if (c.blocked_min_front <= 0) c.blocked_min_front = 96;
  Plan &pl = plan->pl;
  try {
    SMFG_CUDA(cudaSetDevice(pl.device));
    clear_stale_error();
    const double *dv = values;
    double *tmp = nullptr;
    if (!on_device) {
      tmp = pl.x.work;  // staged through the work buffer
      ensure_work(pl, std::max<int64_t>(pl.nnz_in, 1) + 16);
      tmp = pl.x.work;
      SMFG_CUDA(cudaMemcpyAsync(tmp, values, sizeof(double) * pl.nnz_in, cudaMemcpyHostToDevice, pl.stream));
      dv = tmp;
    }
    plan->has_scale = c.scale != nullptr;
    return run_factor(pl, dv, c, info);
  } catch (const CudaError &e) {
    set_last_error(e.what());
    return SMFG_ERR_CUDA;
  } catch (...) {
    return SMFG_ERR_INTERNAL;
  }
}

SMFG_API int smfg_factor(smfg_plan_t plan, const double *values, const smfg_control_t *ctrl,
                         smfg_info_t *info) {
  return factor_common(plan, values, false, ctrl, info);
}

SMFG_API int smfg_factor_device(smfg_plan_t plan, const double *d_values, const smfg_control_t *ctrl,
                                smfg_info_t *info) {
  return factor_common(plan, d_values, true, ctrl, info);
}

static int solve_common(smfg_plan_t plan, double *b, bool on_device, int nrhs, int ldb, int job,
                        smfg_info_t *info) {
  if (!plan || !b || nrhs < 1) return SMFG_ERR_INVALID_ARG;
  Plan &pl = plan->pl;
  if (ldb < pl.n || job < 0 || job > 3) return SMFG_ERR_INVALID_ARG;
  if (!pl.factored) return SMFG_ERR_SINGULAR;
  try {
    SMFG_CUDA(cudaSetDevice(pl.device));
    clear_stale_error();
    LaunchCount lc;
    double *db = b;
    double *staged = nullptr;
    const size_t bytes = sizeof(double) * ((size_t)ldb * (nrhs - 1) + pl.n);
    if (!on_device) {
      SMFG_CUDA(cudaMallocAsync((void **)&staged, bytes, pl.stream));
      SMFG_CUDA(cudaMemcpyAsync(staged, b, bytes, cudaMemcpyHostToDevice, pl.stream));
      db = staged;
    }
    SMFG_CUDA(cudaEventRecord(pl.ev0, pl.stream));
    enqueue_solve(pl, db, nrhs, ldb, job, plan->has_scale, lc);
    SMFG_CUDA(cudaEventRecord(pl.ev1, pl.stream));
    if (!on_device) {
      SMFG_CUDA(cudaMemcpyAsync(b, staged, bytes, cudaMemcpyDeviceToHost, pl.stream));
      SMFG_CUDA(cudaFreeAsync(staged, pl.stream));
    }
    SMFG_CUDA(cudaStreamSynchronize(pl.stream));
    float ms = 0.0f;
    SMFG_CUDA(cudaEventElapsedTime(&ms, pl.ev0, pl.ev1));
    pl.info.solve_ms = ms;
    if (info) {
      *info = pl.info;
      info->kernel_launches = lc.n;
    }
    return SMFG_OK;
  } catch (const CudaError &e) {
    set_last_error(e.what());
    return SMFG_ERR_CUDA;
  } catch (...) {
    return SMFG_ERR_INTERNAL;
  }
}

SMFG_API int smfg_solve(smfg_plan_t plan, double *b, int nrhs, int ldb, int job, smfg_info_t *info) {
  return solve_common(plan, b, false, nrhs, ldb, job, info);
}

SMFG_API int smfg_solve_device(smfg_plan_t plan, double *d_b, int nrhs, int ldb, int job,
                               smfg_info_t *info) {
  return solve_common(plan, d_b, true, nrhs, ldb, job, info);
}

SMFG_API int smfg_inertia(smfg_plan_t plan, int *pos, int *neg, int *zero) {
  if (!plan || !pos || !neg || !zero) return SMFG_ERR_INVALID_ARG;
  if (!plan->pl.factored) return SMFG_ERR_SINGULAR;
  *pos = plan->pl.info.num_pos;
  *neg = plan->pl.info.num_neg;
  *zero = plan->pl.info.num_zero;
  return SMFG_OK;
}

SMFG_API int smfg_front_stats(smfg_plan_t plan, int *stats) {
  if (!plan || !stats) return SMFG_ERR_INVALID_ARG;
  Plan &pl = plan->pl;
  try {
    SMFG_CUDA(cudaSetDevice(pl.device));
    std::vector<int> st(4 * (size_t)pl.nsn), dout(pl.nsn);
    SMFG_CUDA(cudaMemcpy(st.data(), pl.x.sn_stat, sizeof(int) * st.size(), cudaMemcpyDeviceToHost));
    SMFG_CUDA(cudaMemcpy(dout.data(), pl.x.sn_dout, sizeof(int) * dout.size(), cudaMemcpyDeviceToHost));
    for (int s = 0; s < pl.nsn; ++s) {
      for (int k = 0; k < 4; ++k) stats[5 * (size_t)s + k] = st[4 * (size_t)s + k];
      stats[5 * (size_t)s + 4] = dout[s];
    }
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return SMFG_ERR_CUDA;
  }
  return SMFG_OK;
}

SMFG_API int smfg_factor_sizes(smfg_plan_t plan, int64_t *block_entries, int64_t *row_entries) {
  if (!plan || !block_entries || !row_entries) return SMFG_ERR_INVALID_ARG;
  *block_entries = plan->pl.info.factor_entries;
  std::vector<int> f(plan->pl.nsn);
  try {
    SMFG_CUDA(cudaMemcpy(f.data(), plan->pl.x.sn_f, sizeof(int) * f.size(), cudaMemcpyDeviceToHost));
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return SMFG_ERR_CUDA;
  }
  int64_t r = 0;
  for (int v : f) r += v;
  *row_entries = r;
  return SMFG_OK;
}

SMFG_API int smfg_factor_export(smfg_plan_t plan, int *f, int *p, int64_t *blk_off, double *blocks,
                                int64_t *row_off, int *rows, int8_t *tags) {
  if (!plan || !f || !p || !blk_off || !blocks || !row_off || !rows) return SMFG_ERR_INVALID_ARG;
  Plan &pl = plan->pl;
  const int ns = pl.nsn;
  try {
    SMFG_CUDA(cudaSetDevice(pl.device));
    clear_stale_error();
    std::vector<int64_t> off(ns), roff(ns);
    SMFG_CUDA(cudaMemcpy(f, pl.x.sn_f, sizeof(int) * ns, cudaMemcpyDeviceToHost));
    SMFG_CUDA(cudaMemcpy(p, pl.x.sn_pstore, sizeof(int) * ns, cudaMemcpyDeviceToHost));
    SMFG_CUDA(cudaMemcpy(off.data(), pl.x.sn_off, sizeof(int64_t) * ns, cudaMemcpyDeviceToHost));
    SMFG_CUDA(cudaMemcpy(roff.data(), pl.x.sn_roff, sizeof(int64_t) * ns, cudaMemcpyDeviceToHost));
    int64_t bo = 0, ro = 0, to = 0;
    for (int s = 0; s < ns; ++s) {
      blk_off[s] = bo;
      row_off[s] = ro;
      const size_t cnt = (size_t)f[s] * p[s];
      if (cnt) SMFG_CUDA(cudaMemcpy(blocks + bo, pl.x.arena + off[s], sizeof(double) * cnt, cudaMemcpyDeviceToHost));
      SMFG_CUDA(cudaMemcpy(rows + ro, pl.x.rows + roff[s], sizeof(int) * f[s], cudaMemcpyDeviceToHost));
      if (tags && p[s]) SMFG_CUDA(cudaMemcpy(tags + to, pl.x.tags + roff[s], (size_t)p[s], cudaMemcpyDeviceToHost));
      bo += (int64_t)cnt;
      ro += f[s];
      to += p[s];
    }
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return SMFG_ERR_CUDA;
  }
  return SMFG_OK;
}

// Device residual of x for b (both n x nrhs, leading dimension n, device).
static void device_residual(Plan &pl, const double *db, const double *dx, double *dr, int nrhs,
                            double *eta, double *omega) {
  unsigned long long *mx = nullptr;
  SMFG_CUDA(cudaMallocAsync((void **)&mx, sizeof(unsigned long long) * 8, pl.stream));
  // permuted copies: the residual works in the new numbering
  double *xp = nullptr, *bp = nullptr, *rp = nullptr;
  const size_t len = (size_t)pl.n;
  SMFG_CUDA(cudaMallocAsync((void **)&xp, sizeof(double) * len * 3, pl.stream));
  bp = xp + len;
  rp = bp + len;
  const int sms = sm_count(pl.device);
  double e_max = 0.0, o_max = 0.0;
  for (int r = 0; r < nrhs; ++r) {
    SMFG_CUDA(cudaMemsetAsync(mx, 0, sizeof(unsigned long long) * 8, pl.stream));
    const int g = (int)std::max<int64_t>(1, std::min<int64_t>(4 * sms, (pl.n + 255) / 256));
    k_solve_gather<<<g, 256, 0, pl.stream>>>(dx + (size_t)r * pl.n, pl.n, 1, pl.n, pl.d.perm, nullptr, xp);
    k_solve_gather<<<g, 256, 0, pl.stream>>>(db + (size_t)r * pl.n, pl.n, 1, pl.n, pl.d.perm, nullptr, bp);
    const int rg = (int)std::max<int64_t>(1, std::min<int64_t>(8 * sms, (pl.n + 7) / 8));
    k_residual<<<rg, 256, 0, pl.stream>>>(pl.d, pl.x.pv_raw, xp, bp, rp, pl.n, mx);
    k_solve_scatter<<<g, 256, 0, pl.stream>>>(dr + (size_t)r * pl.n, pl.n, 1, pl.n, pl.d.perm, nullptr, rp);
    unsigned long long h[8];
    SMFG_CUDA(cudaMemcpyAsync(h, mx, sizeof(h), cudaMemcpyDeviceToHost, pl.stream));
    SMFG_CUDA(cudaStreamSynchronize(pl.stream));
    double v[5];
    for (int i = 0; i < 5; ++i) std::memcpy(&v[i], &h[i], 8);
    const double den = v[1] * v[2] + v[3];
    const double e = den > 0 ? v[0] / den : (v[0] == 0 ? 0.0 : INFINITY);
    e_max = std::max(e_max, e);
    o_max = std::max(o_max, v[4]);
  }
  SMFG_CUDA(cudaFreeAsync(xp, pl.stream));
  SMFG_CUDA(cudaFreeAsync(mx, pl.stream));
  *eta = e_max;
  *omega = o_max;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Residual without allocation. Its scratch (the permuted copies of x, b and
// r for one right-hand side, and the five maxima) lives in this file-scope
// device array, which every GPU that loads the library holds until the
// process exits. Host code cannot use the array's name as a device address,
// so each device's address is looked up once with cudaGetSymbolAddress and
// passed to the kernels.
namespace {

constexpr int kNoAllocMaxN = SMFG_NOALLOC_MAX_N;
constexpr size_t kNoAllocDoubles = 3 * (size_t)kNoAllocMaxN + 8;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double *g_noalloc_ptr[kMaxDevices] = {};

// The calling thread's current device must be `dev`.
double *noalloc_scratch(int dev) {
  if (dev < 0 || dev >= kMaxDevices) throw std::invalid_argument("device index");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    SMFG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_ptr[dev] = static_cast<double *>(p);
  }
  return g_noalloc_ptr[dev];
}

}  // namespace

extern "C" {

SMFG_API int smfg_residual_noalloc(smfg_plan_t plan, const double *d_b, const double *d_x, double *d_r,
                                   int nrhs, double *eta_inf, double *omega) {
  if (!plan || !d_b || !d_x || nrhs < 1) return SMFG_ERR_INVALID_ARG;
  Plan &pl = plan->pl;
  if (pl.n > kNoAllocMaxN) {
    set_last_error("smfg_residual_noalloc: matrix order exceeds SMFG_NOALLOC_MAX_N");
    return SMFG_ERR_INVALID_ARG;
  }
  try {
    SMFG_CUDA(cudaSetDevice(pl.device));
    clear_stale_error();
    double *sc = noalloc_scratch(pl.device);
    const size_t n = (size_t)pl.n;
    double *xp = sc, *bp = sc + n, *rp = sc + 2 * n;
    unsigned long long *mx = reinterpret_cast<unsigned long long *>(sc + 3 * (size_t)kNoAllocMaxN);
    const int sms = sm_count(pl.device);
    const int g = (int)std::max<int64_t>(1, std::min<int64_t>(4 * sms, ((int64_t)n + 255) / 256));
    const int rg = (int)std::max<int64_t>(1, std::min<int64_t>(8 * sms, ((int64_t)n + 7) / 8));
    double e_max = 0.0, o_max = 0.0;
    for (int r = 0; r < nrhs; ++r) {
      // the maxima start from zero on every call (the array keeps the last
      // call's contents)
      SMFG_CUDA(cudaMemsetAsync(mx, 0, sizeof(unsigned long long) * 8, pl.stream));
      k_solve_gather<<<g, 256, 0, pl.stream>>>(d_x + r * n, (int)n, 1, (int)n, pl.d.perm, nullptr, xp);
      k_solve_gather<<<g, 256, 0, pl.stream>>>(d_b + r * n, (int)n, 1, (int)n, pl.d.perm, nullptr, bp);
      k_residual<<<rg, 256, 0, pl.stream>>>(pl.d, pl.x.pv_raw, xp, bp, rp, (int)n, mx);
      if (d_r) k_solve_scatter<<<g, 256, 0, pl.stream>>>(d_r + r * n, (int)n, 1, (int)n, pl.d.perm, nullptr, rp);
      SMFG_CUDA(cudaGetLastError());
      unsigned long long h[5];
      SMFG_CUDA(cudaMemcpyAsync(h, mx, sizeof(h), cudaMemcpyDeviceToHost, pl.stream));
      SMFG_CUDA(cudaStreamSynchronize(pl.stream));
      double v[5];
      for (int i = 0; i < 5; ++i) std::memcpy(&v[i], &h[i], 8);
      const double den = v[1] * v[2] + v[3];
      e_max = std::max(e_max, den > 0 ? v[0] / den : (v[0] == 0 ? 0.0 : INFINITY));
      o_max = std::max(o_max, v[4]);
    }
    if (eta_inf) *eta_inf = e_max;
    if (omega) *omega = o_max;
    return SMFG_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return SMFG_ERR_CUDA;
  }
}

SMFG_API int smfg_residual(smfg_plan_t plan, const double *b, const double *x, int nrhs, double *r,
                           double *eta_inf, double *omega) {
  if (!plan || !b || !x || nrhs < 1) return SMFG_ERR_INVALID_ARG;
  Plan &pl = plan->pl;
  try {
    SMFG_CUDA(cudaSetDevice(pl.device));
    clear_stale_error();
    const size_t len = (size_t)pl.n * nrhs;
    double *d = nullptr;
    SMFG_CUDA(cudaMallocAsync((void **)&d, sizeof(double) * len * 3, pl.stream));
    SMFG_CUDA(cudaMemcpyAsync(d, b, sizeof(double) * len, cudaMemcpyHostToDevice, pl.stream));
    SMFG_CUDA(cudaMemcpyAsync(d + len, x, sizeof(double) * len, cudaMemcpyHostToDevice, pl.stream));
    double e = 0, o = 0;
    device_residual(pl, d, d + len, d + 2 * len, nrhs, &e, &o);
    if (r) SMFG_CUDA(cudaMemcpyAsync(r, d + 2 * len, sizeof(double) * len, cudaMemcpyDeviceToHost, pl.stream));
    SMFG_CUDA(cudaFreeAsync(d, pl.stream));
    SMFG_CUDA(cudaStreamSynchronize(pl.stream));
    if (eta_inf) *eta_inf = e;
    if (omega) *omega = o;
    return SMFG_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return SMFG_ERR_CUDA;
  }
}

SMFG_API int smfg_refine(smfg_plan_t plan, const double *b, double *x, int nrhs, int max_steps,
                         double omega_target, double *eta_inf, double *omega, int *steps) {
  if (!plan || !b || !x || nrhs < 1) return SMFG_ERR_INVALID_ARG;
  Plan &pl = plan->pl;
  if (!pl.factored) return SMFG_ERR_SINGULAR;
  try {
    SMFG_CUDA(cudaSetDevice(pl.device));
    clear_stale_error();
    const size_t len = (size_t)pl.n * nrhs;
    double *d = nullptr;
    SMFG_CUDA(cudaMallocAsync((void **)&d, sizeof(double) * len * 4, pl.stream));
    double *db = d, *dx = d + len, *dr = d + 2 * len, *dbest = d + 3 * len;
    SMFG_CUDA(cudaMemcpyAsync(db, b, sizeof(double) * len, cudaMemcpyHostToDevice, pl.stream));
    SMFG_CUDA(cudaMemcpyAsync(dx, x, sizeof(double) * len, cudaMemcpyHostToDevice, pl.stream));
    double e = 0, o = 0;
    device_residual(pl, db, dx, dr, nrhs, &e, &o);
    SMFG_CUDA(cudaMemcpyAsync(dbest, dx, sizeof(double) * len, cudaMemcpyDeviceToDevice, pl.stream));
    double be = e, bo = o;
    int it = 0;
    const int sms = sm_count(pl.device);
    const double tgt = omega_target > 0 ? omega_target : 1e-8;
    while (it < max_steps && !(be <= 1e-10 && bo <= tgt)) {
      LaunchCount lc;
      enqueue_solve(pl, dr, nrhs, pl.n, SMFG_SOLVE_FULL, plan->has_scale, lc);
      const int g = (int)std::max<int64_t>(1, std::min<int64_t>(4 * sms, ((int64_t)len + 255) / 256));
      k_axpy<<<g, 256, 0, pl.stream>>>(dx, dr, (int64_t)len);
      ++it;
      device_residual(pl, db, dx, dr, nrhs, &e, &o);
      const double sc = std::max(e / 1e-10, o / tgt), bsc = std::max(be / 1e-10, bo / tgt);
      if (sc < bsc) {
        be = e;
        bo = o;
        SMFG_CUDA(cudaMemcpyAsync(dbest, dx, sizeof(double) * len, cudaMemcpyDeviceToDevice, pl.stream));
        if (sc / bsc > 0.85 && it >= 2) break;
      } else {
        break;
      }
    }
    SMFG_CUDA(cudaMemcpyAsync(x, dbest, sizeof(double) * len, cudaMemcpyDeviceToHost, pl.stream));
    SMFG_CUDA(cudaFreeAsync(d, pl.stream));
    SMFG_CUDA(cudaStreamSynchronize(pl.stream));
    if (eta_inf) *eta_inf = be;
    if (omega) *omega = bo;
    if (steps) *steps = it;
    return SMFG_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return SMFG_ERR_CUDA;
  }
}

SMFG_API int smfg_tc_update(double *d_C, int ldc, int n, const double *d_L, int ldl, const double *d_W,
                           int ldw, int k, int kind) {
  if (!d_C || !d_L || !d_W || n < 0 || k < 0 || ldc < std::max(1, n) || ldl < std::max(1, n) ||
      ldw < std::max(1, n) || (kind != SMFG_TC_TF32X3 && kind != SMFG_TC_BF16X3))
    return SMFG_ERR_INVALID_ARG;
  if (n == 0 || k == 0) return SMFG_OK;
  try {
    clear_stale_error();
    int dev = 0;
    SMFG_CUDA(cudaGetDevice(&dev));
    const int sms = sm_count(dev);
    tc::Job J{};
    J.C = d_C;
    J.Ls = d_L;
    J.Ws = d_W;
    J.tags = nullptr;
    J.ld = ldc;
    J.ldl = ldl;
    J.ldw = ldw;
    J.r0 = J.lr0 = J.wr0 = 0;
    J.n = n;
    J.k0 = 0;
    J.kc = k;
    const int ke = kind == SMFG_TC_TF32X3 ? 32 : 64;  // elements per k-block row
    J.ntr = (n + tc::kBM - 1) / tc::kBM;
    J.nkb = (k + ke - 1) / ke;
    J.tiles = J.ntr * (J.ntr + 1) / 2;
    J.img = 0;
    const int64_t items = (int64_t)J.ntr * tc::kBM * 8 * J.nkb;
    const int64_t ipref[2] = {0, items};
    const int tpref[2] = {0, J.tiles};
    const int64_t img_bytes = tc::image_bytes(J.ntr, J.nkb);
    const size_t meta = 256 + 2 * sizeof(int64_t) + 2 * sizeof(int) + 8;
    uint8_t *buf = nullptr;
    cudaStream_t st = nullptr;
    SMFG_CUDA(cudaMalloc((void **)&buf, meta + img_bytes + 256));
    uint8_t *img = buf + ((meta + 255) / 256) * 256;
    tc::Job *dj = reinterpret_cast<tc::Job *>(buf);
    int64_t *dip = reinterpret_cast<int64_t *>(buf + sizeof(tc::Job) + 8);
    int *dtp = reinterpret_cast<int *>(dip + 2);
    unsigned long long *derr = reinterpret_cast<unsigned long long *>(dtp + 2);
    static_assert(sizeof(tc::Job) + 8 + 2 * sizeof(int64_t) + 2 * sizeof(int) + 8 <= 256 + 2 * sizeof(int64_t) + 2 * sizeof(int) + 8, "meta");
    SMFG_CUDA(cudaMemcpyAsync(dj, &J, sizeof(J), cudaMemcpyHostToDevice, st));
    SMFG_CUDA(cudaMemcpyAsync(dip, ipref, sizeof(ipref), cudaMemcpyHostToDevice, st));
    SMFG_CUDA(cudaMemcpyAsync(dtp, tpref, sizeof(tpref), cudaMemcpyHostToDevice, st));
    SMFG_CUDA(cudaMemsetAsync(derr, 0, sizeof(unsigned long long), st));
    const int sg = (int)std::max<int64_t>(1, std::min<int64_t>(8 * sms, (items + 255) / 256));
    const int gg = std::max(1, std::min(J.tiles, sms));
    const int smem = (int)sizeof(tc::Smem);
    if (kind == SMFG_TC_TF32X3) {
      SMFG_CUDA(cudaFuncSetAttribute(tc::k_tc_syrk<tc::kTF32x3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      tc::k_tc_split<tc::kTF32x3><<<sg, 256, 0, st>>>(dj, 1, dip, img);
      tc::k_tc_syrk<tc::kTF32x3><<<gg, tc::kThreads, smem, st>>>(dj, 1, dtp, img, derr);
    } else {
      SMFG_CUDA(cudaFuncSetAttribute(tc::k_tc_syrk<tc::kBF16x3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      tc::k_tc_split<tc::kBF16x3><<<sg, 256, 0, st>>>(dj, 1, dip, img);
      tc::k_tc_syrk<tc::kBF16x3><<<gg, tc::kThreads, smem, st>>>(dj, 1, dtp, img, derr);
    }
    SMFG_CUDA(cudaGetLastError());
    unsigned long long herr = 0;
    SMFG_CUDA(cudaMemcpyAsync(&herr, derr, sizeof(herr), cudaMemcpyDeviceToHost, st));
    SMFG_CUDA(cudaStreamSynchronize(st));
    SMFG_CUDA(cudaFree(buf));
    if (herr) {
      set_last_error("tensor-core update: a bounded wait gave up");
      return SMFG_ERR_TIMEOUT;
    }
    return SMFG_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return SMFG_ERR_CUDA;
  }
}

}  // extern "C"
