// Test infrastructure, not product code: a thin extern "C" shim over the
// reference smf solver (compiled from its own sources by oracle/Makefile into
// oracle/_ref/libsmfref.so). The tests, smoke() and bench.py's CPU-baseline
// leg use it to
//   - run the reference's own symbolic analysis and export the AnalysisKeep
//     arrays the numeric phase consumes (solver/include/smf/analysis.hpp:25-144),
//   - run the reference's numeric factor (Solver::factor,
//     solver/src/solve.cpp:818-851) and export the FactorKeep per front
//     (solver/include/smf/factor_posdef.hpp:43-220): L blocks at
//     factor_col_ptr[s], solve steps, row ids, pivot tags, inertia,
//   - run the reference's solve (Solver::solve, solve.cpp:1311) and
//     refinement (refine, refinement.cpp:160) on the same factor.
// Nothing here is linked into or loaded by the product library.
#include "smf/analysis.hpp"
#include "smf/control.hpp"
#include "smf/factor_indef.hpp"
#include "smf/factor_posdef.hpp"
#include "smf/info.hpp"
#include "smf/ipm_session.hpp"
#include "smf/ldlt_aptp.hpp"
#include "parallel/tile_tasks.hpp"
#include "smf/refinement.hpp"
#include "smf/scaling_matching.hpp"
#include "smf/solver.hpp"
#include "smf/workspace.hpp"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

namespace {

struct RefHandle {
  smf::Solver solver;
  smf::Control ctrl;
  smf::Info info;
  smf::CscLower A;
  std::vector<int> user_perm;
  std::unique_ptr<smf::AnalysisKeep> ak;
  smf::FactorKeep fk;
  smf::NumericWorkspace nws;
  smf::SolveWorkspace sws;
  std::vector<double> values;  // values of the last factorization, entry order
  double factor_ms = 0.0;
  double solve_ms = 0.0;
  double analyse_ms = 0.0;
};

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" {

void *refshim_create(void) { return new RefHandle(); }

void refshim_free(void *h) { delete static_cast<RefHandle *>(h); }

// ordering: smf::OrderingMethod value. scaling: smf::ScalingMethod value.
// posdef: 1 = SPD (Cholesky path), 0 = indefinite. deterministic: Control::
// deterministic. posdef_kernel: smf::PosdefFrontKernel. Everything else keeps
// the reference's defaults (control.hpp).
void refshim_set_control(void *hp, int ordering, int nemin, int deterministic, int num_threads,
                         double u, double small, int scaling, int posdef, int posdef_kernel,
                         int top_tiles) {
  auto *h = static_cast<RefHandle *>(hp);
  h->ctrl = smf::Control{};
  h->ctrl.ordering = static_cast<smf::OrderingMethod>(ordering);
  if (nemin > 0) h->ctrl.nemin = nemin;
  h->ctrl.deterministic = deterministic != 0;
  h->ctrl.num_threads = num_threads;
  if (u >= 0.0) h->ctrl.pivot_u = u;
  if (small > 0.0) h->ctrl.small_pivot = small;
  h->ctrl.scaling = static_cast<smf::ScalingMethod>(scaling);
  h->ctrl.matrix_type = posdef ? smf::MatrixType::RealSymmetricPositiveDefinite
                               : smf::MatrixType::RealSymmetricIndefinite;
  h->ctrl.posdef_front_kernel = static_cast<smf::PosdefFrontKernel>(posdef_kernel);
  h->ctrl.top_tiles = top_tiles != 0;
}

// Lower CSC input (the caller's entry order). user_perm may be null; with
// OrderingMethod::UserSupplied it is perm[new] = old. Returns Info::status.
int refshim_analyse(void *hp, int n, const int *col_ptr, const int *row_idx, const double *values,
                    const int *user_perm) {
  auto *h = static_cast<RefHandle *>(hp);
  const int nnz = col_ptr[n];
  h->A.n = n;
  h->A.col_ptr.assign(col_ptr, col_ptr + n + 1);
  h->A.row_idx.assign(row_idx, row_idx + nnz);
  if (values) h->A.values.assign(values, values + nnz);
  else h->A.values.assign(static_cast<size_t>(nnz), 1.0);
  if (user_perm) {
    h->user_perm.assign(user_perm, user_perm + n);
    h->ctrl.user_perm = h->user_perm.data();
  }
  const auto t0 = std::chrono::steady_clock::now();
  h->info = smf::Info{};
  h->ak = h->solver.analyse(h->A, h->ctrl, h->info);
  h->analyse_ms = ms_since(t0);
  if (!h->ak) return static_cast<int>(h->info.status) == 0 ? -1 : static_cast<int>(h->info.status);
  return 0;
}

// out[0..11]: n, nsn, len(child_idx), len(front_row_idx), nnz of the permuted
// pattern (0 = identity ordering, the cleaned pattern is used), nnz of the
// original input, len(matching_scale), len(cleaned row_idx),
// len(orig_to_perm_direct), len(orig_to_clean_idx), len(orig_to_perm_idx)
void refshim_analysis_sizes(void *hp, int64_t *out) {
  auto *h = static_cast<RefHandle *>(hp);
  const smf::AnalysisKeep &k = *h->ak;
  out[0] = k.n;
  out[1] = k.num_supernodes();
  out[2] = static_cast<int64_t>(k.child_idx.size());
  out[3] = static_cast<int64_t>(k.front_row_idx.size());
  out[4] = k.perm_col_ptr.empty() ? 0 : k.perm_col_ptr.back();
  out[5] = static_cast<int64_t>(k.orig_row_idx.size());
  out[6] = static_cast<int64_t>(k.matching_scale.size());
  out[7] = static_cast<int64_t>(k.cleaned.row_idx.size());
  out[8] = static_cast<int64_t>(k.orig_to_perm_direct.size());
  out[9] = static_cast<int64_t>(k.orig_to_clean_idx.size());
  out[10] = static_cast<int64_t>(k.orig_to_perm_idx.size());
  out[11] = k.input_clean ? 1 : 0;
}

// Arrays sized by refshim_analysis_sizes. The permuted lower pattern is
// exported in full (built from the cleaned pattern when the ordering is the
// identity), with clean_to_perm[k] = slot of cleaned entry k and
// orig_to_clean[k] = cleaned slot of input entry k (-1: dropped).
void refshim_analysis_export(void *hp, int *perm, int *sn_start, int *sn_end, int *sn_parent,
                             int *child_ptr, int *child_idx, int *front_row_ptr,
                             int *front_row_idx, int *postorder, int *perm_col_ptr,
                             int *perm_row_idx, int *clean_to_perm, int *orig_to_clean,
                             int *clean_col_ptr, int *clean_row_idx, double *matching_scale) {
  auto *h = static_cast<RefHandle *>(hp);
  const smf::AnalysisKeep &k = *h->ak;
  const int n = k.n;
  const int ns = k.num_supernodes();
  for (int i = 0; i < n; ++i) perm[i] = k.perm.empty() ? i : k.perm[i];
  for (int s = 0; s < ns; ++s) {
    sn_start[s] = k.supernodes[s].col_start;
    sn_end[s] = k.supernodes[s].col_end;
    sn_parent[s] = k.supernodes[s].parent;
    postorder[s] = k.postorder[s];
  }
  std::memcpy(child_ptr, k.child_ptr.data(), sizeof(int) * (ns + 1));
  std::memcpy(child_idx, k.child_idx.data(), sizeof(int) * k.child_idx.size());
  std::memcpy(front_row_ptr, k.front_row_ptr.data(), sizeof(int) * (ns + 1));
  std::memcpy(front_row_idx, k.front_row_idx.data(), sizeof(int) * k.front_row_idx.size());
  const size_t cnnz = k.cleaned.row_idx.size();
  std::memcpy(clean_col_ptr, k.cleaned.col_ptr.data(), sizeof(int) * (n + 1));
  std::memcpy(clean_row_idx, k.cleaned.row_idx.data(), sizeof(int) * cnnz);
  if (!k.perm_col_ptr.empty()) {
    std::memcpy(perm_col_ptr, k.perm_col_ptr.data(), sizeof(int) * (n + 1));
    std::memcpy(perm_row_idx, k.perm_row_idx.data(), sizeof(int) * k.perm_row_idx.size());
    std::memcpy(clean_to_perm, k.orig_to_perm_idx.data(), sizeof(int) * cnnz);
  } else {
    std::memcpy(perm_col_ptr, k.cleaned.col_ptr.data(), sizeof(int) * (n + 1));
    std::memcpy(perm_row_idx, k.cleaned.row_idx.data(), sizeof(int) * cnnz);
    for (size_t e = 0; e < cnnz; ++e) clean_to_perm[e] = static_cast<int>(e);
  }
  const size_t nin = k.orig_row_idx.size();
  if (!k.orig_to_clean_idx.empty()) {
    std::memcpy(orig_to_clean, k.orig_to_clean_idx.data(), sizeof(int) * nin);
  } else {
    const size_t m = nin ? nin : cnnz;
    for (size_t e = 0; e < m; ++e) orig_to_clean[e] = static_cast<int>(e);
  }
  if (matching_scale && !k.matching_scale.empty())
    std::memcpy(matching_scale, k.matching_scale.data(), sizeof(double) * k.matching_scale.size());
}

double refshim_analyse_ms(void *hp) { return static_cast<RefHandle *>(hp)->analyse_ms; }

// Factor the values (input entry order). stats[0..9]: FactorStatus, pos, neg,
// zero, delayed, 2x2 pivots, max front, static pivots, factor entries used,
// Info::status. flops_ms[0] = Info::actual_flops, flops_ms[1] = factor ms.
int refshim_factor(void *hp, const double *values, int64_t *stats, double *flops_ms) {
  auto *h = static_cast<RefHandle *>(hp);
  const size_t nnz = h->A.row_idx.size();
  h->values.assign(values, values + nnz);
  smf::Info info;
  const auto t0 = std::chrono::steady_clock::now();
  const smf::FactorStatus st = h->solver.factor(*h->ak, std::span<const double>(h->values), h->ctrl,
                                                info, h->fk, h->nws);
  h->factor_ms = ms_since(t0);
  h->info = info;
  stats[0] = static_cast<int64_t>(st);
  stats[1] = info.num_positive;
  stats[2] = info.num_negative;
  stats[3] = info.num_zero;
  stats[4] = info.delayed_pivots;
  stats[5] = info.two_by_two_pivots;
  stats[6] = info.max_front_size;
  stats[7] = info.static_pivots;
  stats[8] = static_cast<int64_t>(h->fk.factor_values.used());
  stats[9] = static_cast<int64_t>(info.status);
  flops_ms[0] = info.actual_flops;
  flops_ms[1] = h->factor_ms;
  return static_cast<int>(st);
}

// The reference's dense APTP front kernel alone (ldlt_aptp.cpp:739, or the
// tile-task form deterministic mode runs, parallel/tile_tasks.cpp:256, on one
// thread): F f x f column-major (lower), the first ne columns eligible; rows
// and tags (f) updated in place. out[0..4] = eliminated, failed, positive,
// negative, zero pivots.
void refshim_aptp_front(double *F, int f, int ne, int *rows, double u, double small, int nb, int ib,
                        int tiled, int8_t *tags, int64_t *out) {
  smf::AptpParams prm;
  prm.u = u;
  prm.small = small;
  prm.nb = nb;
  prm.ib = ib;
  std::vector<double> work(smf::aptp_work_size(f, ne, prm) + 1);
  smf::TileWorkspace tws;
  const smf::AptpResult r =
      tiled ? smf::ldlt_aptp_front_tiled(F, f, ne, rows, prm, tags, work.data(), tws, 1, nullptr)
            : smf::ldlt_aptp_front(F, f, ne, rows, prm, tags, work.data());
  out[0] = r.num_eliminated;
  out[1] = r.num_failed;
  out[2] = r.inertia.positive;
  out[3] = r.inertia.negative;
  out[4] = r.inertia.zero;
}

// The reference's IpmSession (ipm_session.hpp:120-273), Feature 1 (inertia
// learning and the early abort on wrong inertia), for comparing the
// engine's session decisions step by step. Deterministic mode, one thread,
// AutoParallel ordering, automatic scaling, indefinite.
void *refshim_ipm_create(void) { return new smf::IpmSession(); }
void refshim_ipm_free(void *h) { delete static_cast<smf::IpmSession *>(h); }

int refshim_ipm_analyse(void *hp, int n, const int *col_ptr, const int *row_idx, const double *values,
                        int abort_on_wrong_inertia) {
  auto *s = static_cast<smf::IpmSession *>(hp);
  smf::CscLower A;
  A.n = n;
  A.col_ptr.assign(col_ptr, col_ptr + n + 1);
  A.row_idx.assign(row_idx, row_idx + col_ptr[n]);
  smf::Control ctrl{};
  ctrl.deterministic = true;
  ctrl.num_threads = 1;
  ctrl.matrix_type = smf::MatrixType::RealSymmetricIndefinite;
  smf::IpmControl ipm{};
  ipm.abort_on_wrong_inertia = abort_on_wrong_inertia != 0;
  const std::size_t nnz = static_cast<std::size_t>(col_ptr[n]);
  return static_cast<int>(s->analyse(A, std::span<const double>(values, nnz), ctrl, ipm));
}

// out[0..4]: IpmFactorStatus (0 Ok, 1 WrongInertia, 2 Singular, 3 Error),
// positive, negative, zero pivots, delayed pivots. expected < 0: none given.
void refshim_ipm_factor(void *hp, const double *values, int64_t nnz, int expected, int64_t *out) {
  auto *s = static_cast<smf::IpmSession *>(hp);
  std::optional<int> e;
  if (expected >= 0) e = expected;
  const smf::IpmFactorStatus st = s->factor(std::span<const double>(values, static_cast<std::size_t>(nnz)), e);
  const smf::InertiaCounts in = s->inertia();
  out[0] = static_cast<int64_t>(st);
  out[1] = in.positive;
  out[2] = in.negative;
  out[3] = in.zero;
  out[4] = s->info().delayed_pivots;
}

// Solve in place (one right-hand side); out[0..2]: the inertia afterwards
// (an aborted factor is completed first), out[3]: the learned expectation
// (-1: none).
int refshim_ipm_solve(void *hp, double *b, int n, int64_t *out) {
  auto *s = static_cast<smf::IpmSession *>(hp);
  const int rc = s->solve(b, n, 1);
  const smf::InertiaCounts in = s->inertia();
  out[0] = in.positive;
  out[1] = in.negative;
  out[2] = in.zero;
  out[3] = s->expected_negatives() ? *s->expected_negatives() : -1;
  return rc;
}

// Info::aptp_failed_columns of the last factorization: the columns the APTP
// kernel failed (then tried by the threshold kernel).
int64_t refshim_aptp_failed(void *hp) {
  return static_cast<RefHandle *>(hp)->info.aptp_failed_columns;
}

// out[0]: the last factorization's front work (Info::front_work: fully
// summed columns x rows^2 summed over the fronts,
// solver/src/multifrontal_serial.cpp:875); out[1]: the analysis' delay-free
// front work (delay_free_front_work, solver/src/factor_indef.cpp:896-903).
void refshim_front_work(void *hp, double *out) {
  auto *h = static_cast<RefHandle *>(hp);
  out[0] = h->info.front_work;
  out[1] = h->ak ? smf::delay_free_front_work(*h->ak) : 0.0;
}

// The reference's symmetric matching scaling of a lower CSC matrix
// (compute_matching_scale, solver/src/scaling_matching.cpp:1109-1118),
// n doubles into scale. Returns its ErrorCode (0: success).
int refshim_matching_scale(int n, const int *col_ptr, const int *row_idx, const double *values,
                           double *scale) {
  smf::CscLower A;
  A.n = n;
  A.col_ptr.assign(col_ptr, col_ptr + n + 1);
  A.row_idx.assign(row_idx, row_idx + col_ptr[n]);
  A.values.assign(values, values + col_ptr[n]);
  std::vector<double> s;
  const smf::ErrorCode rc = smf::compute_matching_scale(A, s, 0);
  if (rc == smf::ErrorCode::Success && s.size() == static_cast<size_t>(n))
    std::copy(s.begin(), s.end(), scale);
  return static_cast<int>(rc);
}

// out: number of solve steps, extent of factor_values, total rows of the
// solve steps, len(diag entries), is_posdef, len(scale).
void refshim_factor_sizes(void *hp, int64_t *out) {
  auto *h = static_cast<RefHandle *>(hp);
  const smf::FactorKeep &f = h->fk;
  out[0] = static_cast<int64_t>(f.solve_steps.size());
  out[1] = static_cast<int64_t>(f.factor_values.size());
  int64_t rows = 0;
  for (const auto &s : f.solve_steps) rows += s.f;
  out[2] = rows;
  out[3] = static_cast<int64_t>(f.diag().size());
  out[4] = f.is_posdef ? 1 : 0;
  out[5] = static_cast<int64_t>(f.scale.size());
}

// Per supernode s: the realized front rows f, stored pivots p (factor block
// f x p at factor_col_ptr[s], leading dimension f), its L block (copied into
// `blocks` at block_off[s], packed one after the other), its row ids (in
// pivot order, at row_off[s]) and, indefinite only, its pivot tags
// (tags at tag_off = sum of the p of earlier supernodes). Blocks, rows and
// tags are packed in supernode order; each supernode's solve step is found
// through the postorder (the serial engine's step order).
int refshim_factor_export(void *hp, int *f_out, int *p_out, int64_t *block_off, double *blocks,
                          int64_t *row_off, int *rows, int8_t *tags, double *scale) {
  auto *h = static_cast<RefHandle *>(hp);
  const smf::FactorKeep &fk = h->fk;
  const smf::AnalysisKeep &k = *h->ak;
  const int ns = k.num_supernodes();
  if (static_cast<int>(fk.solve_steps.size()) != ns) return -1;
  std::vector<int> step_of(ns, -1);
  for (int i = 0; i < ns; ++i) step_of[k.postorder[i]] = i;
  int64_t bo = 0, ro = 0, to = 0;
  for (int s = 0; s < ns; ++s) {  // supernode order
    const smf::SolveStep &st = fk.solve_steps[step_of[s]];
    if (st.factor_offset != fk.factor_col_ptr[s]) return -2;
    f_out[s] = st.f;
    p_out[s] = st.p;
    block_off[s] = bo;
    row_off[s] = ro;
    const double *src = fk.factor_values.data() + st.factor_offset;
    std::memcpy(blocks + bo, src, sizeof(double) * static_cast<size_t>(st.f) * st.p);
    std::memcpy(rows + ro, fk.solve_row_indices.data() + st.row_offset, sizeof(int) * st.f);
    if (!fk.is_posdef && tags) {
      const auto &pt = fk.pivot_types[s];
      for (size_t c = 0; c < pt.size(); ++c) tags[to + c] = pt[c];
      to += static_cast<int64_t>(pt.size());
    }
    bo += static_cast<int64_t>(st.f) * st.p;
    ro += st.f;
  }
  if (scale && !fk.scale.empty()) std::memcpy(scale, fk.scale.data(), sizeof(double) * fk.scale.size());
  return 0;
}

// Solve in place (b: n x nrhs, leading dimension ldb). job: smf::SolveJob.
int refshim_solve(void *hp, double *b, int nrhs, int ldb, int job, double *ms) {
  auto *h = static_cast<RefHandle *>(hp);
  smf::Info info;
  const int n = h->ak->n;
  const auto t0 = std::chrono::steady_clock::now();
  const int rc = h->solver.solve(h->fk, h->ctrl, info, std::span<double>(b, static_cast<size_t>(ldb) * (nrhs - 1) + n),
                                 nrhs, ldb, h->sws, static_cast<smf::SolveJob>(job));
  h->solve_ms = ms_since(t0);
  if (ms) *ms = h->solve_ms;
  return rc;
}

// Iterative refinement of x (n x nrhs, leading dimension n) against the
// factored values. res[0] = eta_inf, res[1] = omega; iters[0] = steps,
// iters[1] = status.
int refshim_refine(void *hp, const double *b, double *x, int nrhs, double *res, int *iters) {
  auto *h = static_cast<RefHandle *>(hp);
  smf::CscLower A = h->A;
  A.values = h->values;
  const int n = h->ak->n;
  const size_t len = static_cast<size_t>(n) * nrhs;
  smf::RefinementResult r = smf::refine(A, h->fk, h->ctrl, std::span<const double>(b, len),
                                        std::span<double>(x, len), nrhs, h->sws);
  res[0] = r.eta_inf;
  res[1] = r.omega;
  iters[0] = r.iterations;
  iters[1] = static_cast<int>(r.status);
  return static_cast<int>(r.status);
}

}  // extern "C"
