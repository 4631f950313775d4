// Internal types of the B200 numeric phase: the device plan built once per
// analysis and the per-factorization device state.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/smfg.h"
#include "smfg_front.cuh"

namespace smfg {

// Size classes of the front kernels (rows f after delays).
constexpr int kSmallMax = 64;    // one warp, front in shared memory
constexpr int kMediumMax = 128;  // one block, front in shared memory
constexpr int kAsmCols = 32;     // columns per assembly work item

// Device copies of the analysis-derived arrays (one per plan).
struct DevPlan {
  int n = 0, nsn = 0, nlevels = 0;
  int64_t nnz = 0;      // permuted pattern entries
  int64_t nnz_in = 0;   // caller's entries
  int *sn_start = nullptr, *sn_width = nullptr, *sn_fsym = nullptr, *sn_parent = nullptr;
  int *child_ptr = nullptr, *child_idx = nullptr;
  int *frow_ptr = nullptr, *frow_idx = nullptr;
  int *cpr_off = nullptr, *cpr_idx = nullptr;  // per child slot: parent symbolic positions
  int *lvl_sn = nullptr;                       // supernodes by level
  int *pcp = nullptr, *pri = nullptr;          // permuted lower pattern
  int *pcol = nullptr;                         // column of each permuted slot
  int *amap = nullptr;                         // entry -> symbolic row position in its front
  int *vptr = nullptr, *vsrc = nullptr;        // permuted slot -> caller entries (input order)
  int *perm = nullptr;                         // perm[new] = old
  int *srow = nullptr, *sptr = nullptr;        // full symmetric CSR (residual), new numbering
  int64_t *sidx = nullptr;                     // its entry -> permuted slot
  int *sn_level = nullptr;
  int *lvl_large = nullptr;                    // large fronts by level
  int8_t *sn_large = nullptr;                  // 1: the front takes the large-front path
};

// Device state of one factorization (sized per plan, grown on demand).
struct DevFactor {
  double *pv = nullptr;      // permuted (scaled) values
  double *pv_raw = nullptr;  // permuted unscaled values (residual)
  double *scale = nullptr;   // S (original numbering) or null
  int *sn_nd = nullptr, *sn_f = nullptr, *sn_ne = nullptr, *sn_p = nullptr, *sn_pstore = nullptr,
      *sn_dout = nullptr;
  int64_t *sn_off = nullptr, *sn_roff = nullptr;
  int *child_doff = nullptr;  // per child slot: first delayed row's position in the parent
  int *sn_stat = nullptr;     // 4 ints per supernode: pos, neg, zero, 2x2
  double *sn_flops = nullptr;
  int *lvl_blk = nullptr;     // per level entry: prefix of assembly work items (size nsn + nlevels)
  double *arena = nullptr;    // fronts (f x f) + W (f x nb)
  int64_t arena_cap = 0;
  int *rows = nullptr;        // realized row ids, per front at sn_roff
  int8_t *tags = nullptr;     // pivot tags, per front at sn_roff
  int *cbmap = nullptr;       // CB row -> parent position, at the child's sn_roff + p
  int *ploc = nullptr;        // 2 x rows_cap: pivot-order tracking of global-memory fronts
  int64_t rows_cap = 0;
  unsigned long long *counters = nullptr;  // [0] arena base, [1] rows base, [2] error flags, [3] max|A| bits, [4] blocks
  TppState *tpp = nullptr;    // per large front of a level: blocked-pivoting state
  unsigned *team_bar = nullptr;  // per large front of a level: its CTA team's barrier words
  double *team_red = nullptr;    // per large front of a level: its team's reduction scratch
  int *aptp_miss = nullptr;   // fronts that reached the APTP size outside the large-front path
  double *work = nullptr;     // solve / refinement scratch
  int64_t work_cap = 0;
  // mixed precision: fronts whose trailing updates run on the tensor cores
  int8_t *sn_mixed = nullptr;    // per supernode, 0 / 1
  void *tc_jobs = nullptr;       // tc::Job per large front of a level
  int64_t *tc_ipref = nullptr;   // split work items, prefix over jobs
  int *tc_tpref = nullptr;       // tiles, prefix over jobs
  int *tc_njobs = nullptr;
  uint8_t *tc_img = nullptr;     // operand images
  int64_t tc_img_cap = 0;
  // SPD factorizations: the inverses of the large fronts' 32 x 32 diagonal
  // blocks of L (column-major, 1024 doubles a block), for the solves
  double *tri_inv = nullptr;
  int64_t *sn_ioff = nullptr;    // per supernode: its first block's offset in tri_inv, -1 none
  int *inv_items = nullptr;      // (supernode, block) pairs, 2 ints each
  int inv_nitems = 0;
};

struct Plan {
  int device = 0;
  int n = 0, nsn = 0, nlevels = 0;
  int64_t nnz = 0, nnz_in = 0;
  std::vector<int> lvl_ptr;      // host copy: level l = lvl_sn[lvl_ptr[l] .. lvl_ptr[l+1])
  std::vector<int> lvl_maxf;     // symbolic max front per level
  std::vector<int> lvl_maxkids;
  std::vector<int> lvl_large_ptr;  // level l's large fronts: d.lvl_large[lvl_large_ptr[l] ..]
  std::vector<int> lvl_large_maxw; // widest large front per level
  std::vector<int> lvl_large_maxf; // largest symbolic front among them
  std::vector<int> lvl_large_pmax; // most stored pivots among them (last factorization)
  std::vector<int> h_lvl_large;    // host copy of the large-front lists
  std::vector<int8_t> h_large;     // per supernode: the large-front path (symbolic rows, or grown by delays)
  std::vector<int> h_lvl_sn, h_width;  // supernodes by level; pivot columns
  int max_large = 0;
  int64_t sum_f2 = 0, sum_f = 0; // symbolic
  int max_fsym = 0;
  int64_t max_factor = 0;
  DevPlan d;
  DevFactor x;
  cudaStream_t stream = nullptr;
  // the plan's own stream-ordered pool (refinement, residual and staging
  // scratch): keeps up to kPoolKeepBytes between calls instead of unmapping
  // them at each synchronization
  cudaMemPool_t pool = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ev_in = nullptr;  // orders the stream after the caller's default-stream work
  // SPD look-ahead: the deferred updates past the next panel run on stream2
  // while the next panel factors (events: a panel done, a rest update done)
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_panel = nullptr, ev_rest = nullptr;
  // last factorization
  bool factored = false;
  int posdef = 0;
  int nb = 16;
  int factor_status = -1;
  smfg_info_t info{};
  std::vector<int> h_child_ptr, h_child_idx, h_sn_parent, h_postorder;
  std::vector<int> h_fsym;             // symbolic front rows per supernode
  std::vector<int8_t> front_mask;      // caller's per-front precision choice (empty: all may)
  std::vector<int8_t> h_mixed;         // mixed fronts of the last factorization
  int mixed_count = 0;
  double refine_ms = 0.0;  // device time of the last refinement
  int panel_teams[4] = {0, 0, 0, 0};  // tuned CTAs per size bucket of a level's largest front (0: rule)
  // CUDA graph of the factorization (smfg_control_t.graph)
  cudaGraphExec_t graph_exec = nullptr;
  std::vector<unsigned char> graph_key;
  int graph_launches = 0;
  std::vector<void *> allocs;
  // APTP fronts of a level: descriptors, states, scratch, staging
  void *aptp_fr = nullptr, *aptp_st = nullptr;
  int aptp_cap = 0;
  double *aptp_buf = nullptr;
  int64_t aptp_buf_cap = 0;
  double *aptp_gather = nullptr;
  int64_t aptp_gather_cap = 0;
  int64_t *aptp_sizes = nullptr;  // device: f, ne, arena offset, row offset per large front
  int *aptp_q = nullptr;          // device: list positions of the APTP fronts
  int64_t aptp_failed = 0;        // last factorization: columns the APTP sweeps failed
  int aptp_fronts = 0;            // last factorization: fronts swept
};

}  // namespace smfg
