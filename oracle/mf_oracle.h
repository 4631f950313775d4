/* Test infrastructure (the oracle): a plain-C restatement of the reference
 * smf numeric phase, used only by tests/, smoke() and bench.py's CPU-baseline
 * leg as the checker of the CUDA engine. Never linked into the product.
 *
 * Input is the reference's analysis output (AnalysisKeep arrays,
 * solver/include/smf/analysis.hpp:25-144) and the values already placed in
 * the permuted lower pattern (and scaled), as multifrontal_factor_serial
 * receives them (solver/src/multifrontal_serial.cpp:1105).
 */
#ifndef MF_ORACLE_H
#define MF_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int n, nsn;
  const int *sn_start, *sn_end, *sn_parent; /* supernodes, postorder numbering */
  const int *child_ptr, *child_idx;         /* children, descending postorder */
  const int *front_row_ptr, *front_row_idx; /* symbolic front rows, sorted */
  const int *postorder;
  const int *pcp, *pri; /* permuted lower pattern (new indices) */
} mfo_analysis;

typedef struct {
  double u, eff_small, small_pivot;
  int nb, blocked_min_front, posdef;
  /* Emulation of the engine's mixed-precision updates (0 = plain FP64):
   * fronts of at least mixed_min_front rows take their deferred and Schur
   * updates as split products (each operand x = hi + lo, both rounded to
   * mixed_bits significant bits: 8 for BF16x3, 11 for TF32x3; the three
   * products hi*hi, hi*lo, lo*hi summed in FP32) subtracted from FP64. */
  int mixed_min_front, mixed_bits;
  /* Deterministic mode's APTP kernel (ldlt_aptp.cpp) on indefinite fronts of
   * at least aptp_min_rows realized rows (0: never; the reference uses 512),
   * outer block aptp_nb (256), inner block aptp_ib (32). */
  int aptp_min_rows, aptp_nb, aptp_ib;
} mfo_params;

typedef struct {
  /* outputs, sized by the caller: f_out/p_out/blk_off/row_off per supernode;
   * blocks: capacity blk_cap doubles; rows: capacity row_cap ints;
   * tags: per supernode p entries at tag_off = sum of earlier p (cap row_cap). */
  int *f_out, *p_out;
  int64_t *blk_off, *row_off;
  double *blocks;
  int64_t blk_cap;
  int *rows;
  int64_t row_cap;
  int8_t *tags;
  /* counts */
  int64_t pos, neg, zero, delayed, two_by_two, max_front;
  int64_t aptp_failed; /* columns the APTP kernel failed (Info::aptp_failed_columns) */
  double flops;
  int status; /* 0 ok, 1 not positive definite, 2 singular (zero pivots), 3 capacity, 4 non-finite D */
} mfo_factor;

int mfo_factorize(const mfo_analysis *a, const double *pvals, const mfo_params *prm, mfo_factor *out);

/* One dense front through the front kernel alone (ldlt_factor_front with
 * first = 0, solver/src/ldlt_kernel.cpp:970-1139): F f x f column-major
 * (lower triangle), the first ne columns eligible; rows, tags (f) updated in
 * place. out[0..3] = positive, negative, zero pivots, accepted pivots. For
 * the known-answer tests of the dense kernel. */
void mfo_factor_front(double *F, int f, int ne, int *rows, const mfo_params *prm, int8_t *tags,
                      int64_t *out);

/* Tests: capture supernode s's assembled front (f x f column-major, before
 * its kernel) and realized rows during the next mfo_factorize, when f * f <=
 * cap; mfo_captured_size gives its f and eligible columns (-1: not reached). */
void mfo_capture_front(int s, double *F, int64_t cap, int *rows);
void mfo_captured_size(int *f, int *num_elig);

/* The APTP kernel alone on a dense front (ldlt_aptp_front,
 * solver/src/ldlt_aptp.cpp:739): F, rows, tags (f) in place; out[0..4] =
 * eliminated, failed, positive, negative, zero pivots. */
void mfo_aptp_front(double *F, int f, int ne, int *rows, const mfo_params *prm, int8_t *tags, int64_t *out);

/* In-place full solve of A x = b on the permuted, scaled system:
 * x (n, new numbering) overwritten. */
void mfo_solve_permuted(const mfo_analysis *a, const mfo_factor *fac, int posdef, double *x);

/* r = b - A x with A given as the full lower CSC (original numbering), and
 * the normwise / componentwise backward errors (long double accumulation). */
void mfo_residual(int n, const int *cp, const int *ri, const double *v, const double *b,
                  const double *x, double *r, double *eta_inf, double *omega);

#ifdef __cplusplus
}
#endif
#endif
