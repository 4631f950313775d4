// Host-visible types of the APTP front kernel (smfg_aptp.cu): the device
// descriptor of an APTP front, its per-front state, and the entry that runs
// the sweep over a set of fronts.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "smfg_front.cuh"

namespace smfg {
namespace aptp {

constexpr int kNb = 256;  // outer block (tile) width, Control::top_tile_nb
constexpr int kIb = 32;   // inner block width, Control::aptp_ib
constexpr int kMinRows = 512;  // deterministic mode tiles fronts of at least this many rows

// One APTP front (device descriptor). A is f x f column-major, leading
// dimension f; its first ne columns are eligible.
struct Front {
  double *A;
  int *rows;
  int8_t *tags;
  int *loc;     // pivot-order tracking (permuted with rows), or null
  double *bk;   // backup of the block column: column t at bk + t * f (absolute rows)
  double *ga;   // ApplyT rows of the failed columns: row i at ga + i * kNb
  double *gb;   // their (L D) rows: row i at gb + i * kNb
  int *Q;       // failed columns (positions, ascending); ne entries
  int *pi;      // compaction permutation (ne)
  int f, ne, nb, ib;
};

// Per-front state, written by the kernels.
struct State {
  int c0, w;         // the current block column
  int ne_t;          // pivots of its diagonal tile
  int nmin;          // running minimum of the first failing pivot (apply)
  int nelim;         // accepted pivots of the block
  int nq, nq_old;    // failed columns so far / before this block
  int num_elim;      // pivots of the sweep so far
  int ident;         // tile permutation is the identity
  int lpc[kNb];      // lpc[t]: tile position that moved to t
  double dinv[2 * kNb];
  FrontStats st;     // inertia, 2x2 pivots and flops of the sweep's pivots
};

// Device scratch a front needs (doubles): backup f x nb, ApplyT rows and
// their (L D) rows ne x kNb each.
inline int64_t scratch_doubles(int f, int ne) { return (int64_t)f * kNb + 2 * (int64_t)ne * kNb; }

struct SweepHost {
  int sms;
  double inv_u;                           // 1 / u
  const unsigned long long *small_bits;   // device: the effective small value's bits
  double *scratch;                        // device: max over the fronts of f * ne doubles
};

// The APTP sweep of nf fronts (d_fr, d_st device arrays) on stream st, in
// two parts: the block columns (kmax: at least the most any front needs),
// then, once the caller has read the states, the compaction of the fronts
// with failed columns (compact[0 .. ncompact), their indices; h.scratch
// holds f * ne doubles of the largest), the trailing update and the counts.
// Each returns the kernels it launched.
int sweep_blocks(const Front *d_fr, State *d_st, int nf, int kmax, const SweepHost &h, cudaStream_t st);
int sweep_finish(const Front *d_fr, State *d_st, int nf, const int *compact, int ncompact, const SweepHost &h,
                 cudaStream_t st);

}  // namespace aptp
}  // namespace smfg
