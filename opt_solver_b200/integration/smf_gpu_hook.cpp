// smf's own Solver on the B200 numeric phase: the reference-side binding of
// include/smfg.h, compiled against smf's headers and linked into smf's own
// objects (its solver library, its C API smf_c.cpp and its IPOPT plugin
// smf_ma97_plugin.cpp) with the linker's symbol wrapping (--wrap), so that
// no smf source changes. Every call from another smf translation unit to
//
//   smf::Solver::factor(ak, values, ctrl, info, fkeep, ws)     (solve.cpp; smf_c.cpp's smf_factor)
//   smf::Solver::factor(ak, updated, ctrl, info, fkeep, ws)    (IpmSession::run_factor, the plugin)
//   smf::Solver::solve(fkeep, ctrl, info, b, n, nrhs, job)     (smf_c.cpp's smf_solve)
//   smf::Solver::solve(fkeep, ctrl, info, b, n, nrhs, ws, job) (IpmSession::solve, the plugin)
//
// lands here and runs on the GPU: one device plan per analysis (keyed by
// the AnalysisKeep and its serial), the caller's values in their analysed
// entry order, the scaling resolved as factor_indef.cpp:422-436 and
// factor_posdef.cpp:366-368 resolve it (Auto: the analysis' matching scale
// for indefinite matrices, none for SPD ones; None; UserSupplied), the
// threshold kernel everywhere in the default one-thread mode and deterministic
// mode's APTP kernel on indefinite fronts of >= 512 rows with
// Control::deterministic, max_negative_pivots as the device-side early stop.
// The factor stays on the device; FactorKeep records its analysis, order and
// status (and one placeholder value, so that callers that test for a factor,
// IpmSession::run_factor among them, find one), and the solve reads the plan.
//
// Not carried: static pivoting, the delay budget, the quasidefinite mode,
// slack elimination, the scaling methods other than the three above, the
// realized-delay matching re-analysis and the scale-on-delay rescue inside
// Solver::factor (opt_solver_b200/delay.py restates the rescue over the
// engine). A call that asks for one of the first five returns
// ErrorCode::FeatureNotAvailable (FactorStatus::Singular), never a CPU
// factorization.
#include "smf/analysis.hpp"
#include "smf/control.hpp"
#include "smf/determinism.hpp"
#include "smf/factor_posdef.hpp"
#include "smf/info.hpp"
#include "smf/solver.hpp"
#include "smf/types.hpp"

#include <chrono>
#include <cstdint>
#include <mutex>
#include <span>
#include <unordered_map>
#include <vector>

#include "smfg.h"

namespace {

struct PlanEntry {
  std::uint64_t serial = 0;
  smfg_plan_t plan = nullptr;
  std::uint64_t generation = 0;  // factorizations on the plan so far
};
struct FactorEntry {
  const smf::AnalysisKeep *ak = nullptr;
  std::uint64_t serial = 0;
  std::uint64_t generation = 0;
  int n = 0;
  bool posdef = false;
};

std::mutex g_mu;
std::unordered_map<const smf::AnalysisKeep *, PlanEntry> g_plans;
std::unordered_map<const smf::FactorKeep *, FactorEntry> g_factors;

// smfg_analysis_t over the AnalysisKeep's arrays.
struct View {
  std::vector<int> sn, ident_perm, ident_c2p, ident_o2c;
  smfg_analysis_t a{};
};

void make_view(const smf::AnalysisKeep &k, View &v) {
  const int ns = k.num_supernodes();
  v.sn.resize(3 * static_cast<std::size_t>(ns));
  for (int s = 0; s < ns; ++s) {
    v.sn[s] = k.supernodes[s].col_start;
    v.sn[ns + s] = k.supernodes[s].col_end;
    v.sn[2 * ns + s] = k.supernodes[s].parent;
  }
  smfg_analysis_t &a = v.a;
  a.n = k.n;
  a.nsn = ns;
  if (k.perm.empty()) {
    v.ident_perm.resize(static_cast<std::size_t>(k.n));
    for (int i = 0; i < k.n; ++i) v.ident_perm[i] = i;
    a.perm = v.ident_perm.data();
  } else {
    a.perm = k.perm.data();
  }
  a.sn_start = v.sn.data();
  a.sn_end = v.sn.data() + ns;
  a.sn_parent = v.sn.data() + 2 * ns;
  a.child_ptr = k.child_ptr.data();
  a.child_idx = k.child_idx.data();
  a.front_row_ptr = k.front_row_ptr.data();
  a.front_row_idx = k.front_row_idx.data();
  a.postorder = k.postorder.data();
  const std::size_t cnnz = k.cleaned.row_idx.size();
  a.clean_col_ptr = k.cleaned.col_ptr.data();
  a.clean_row_idx = k.cleaned.row_idx.data();
  if (k.perm_col_ptr.empty()) {  // identity ordering: the cleaned pattern is the permuted one
    a.perm_col_ptr = k.cleaned.col_ptr.data();
    a.perm_row_idx = k.cleaned.row_idx.data();
    v.ident_c2p.resize(cnnz);
    for (std::size_t e = 0; e < cnnz; ++e) v.ident_c2p[e] = static_cast<int>(e);
    a.clean_to_perm = v.ident_c2p.data();
  } else {
    a.perm_col_ptr = k.perm_col_ptr.data();
    a.perm_row_idx = k.perm_row_idx.data();
    a.clean_to_perm = k.orig_to_perm_idx.data();
  }
  if (k.orig_to_clean_idx.empty()) {  // clean input: entry k is cleaned slot k
    v.ident_o2c.resize(cnnz);
    for (std::size_t e = 0; e < cnnz; ++e) v.ident_o2c[e] = static_cast<int>(e);
    a.orig_to_clean = v.ident_o2c.data();
    a.nnz_in = static_cast<int64_t>(cnnz);
  } else {
    a.orig_to_clean = k.orig_to_clean_idx.data();
    a.nnz_in = static_cast<int64_t>(k.orig_to_clean_idx.size());
  }
}

// The analysis' device plan (made on first use; remade when the address
// holds a different analysis). Called with g_mu held.
PlanEntry *plan_for(const smf::AnalysisKeep &ak) {
  auto it = g_plans.find(&ak);
  if (it != g_plans.end() && it->second.serial == ak.serial) return &it->second;
  if (it != g_plans.end()) {
    smfg_plan_destroy(&it->second.plan);
    g_plans.erase(it);
  }
  View v;
  make_view(ak, v);
  smfg_plan_t plan = nullptr;
  if (smfg_plan_create(&v.a, 0, &plan) != SMFG_OK) return nullptr;
  PlanEntry e;
  e.serial = ak.serial;
  e.plan = plan;
  return &(g_plans[&ak] = e);
}

smf::FactorStatus fail(smf::Info &info, smf::FactorKeep &fk, smf::ErrorCode code) {
  info.status = code;
  info.factor_status = smf::FactorStatus::Singular;
  fk.status = smf::FactorStatus::Singular;
  fk.factor_values.clear();
  return smf::FactorStatus::Singular;
}

smf::FactorStatus gpu_factor(const smf::AnalysisKeep &ak, const double *values, std::size_t nvals,
                             const smf::Control &ctrl, smf::Info &info, smf::FactorKeep &fk) {
  const auto t0 = std::chrono::steady_clock::now();
  const bool posdef = ctrl.matrix_type == smf::MatrixType::RealSymmetricPositiveDefinite;
  if (ctrl.pivoting != smf::Pivoting::Threshold || ctrl.static_pivot_tol > 0.0 ||
      ctrl.fallback_static_pivot_tol > 0.0 || ctrl.delay_budget >= 0 || ctrl.reg_diag_sign != nullptr ||
      ctrl.slack_elimination != smf::SlackElimination::Off)
    return fail(info, fk, smf::ErrorCode::FeatureNotAvailable);
  // the scaling, as smf resolves it before its numeric phase
  const double *scale = nullptr;
  switch (ctrl.scaling) {
    case smf::ScalingMethod::None: break;
    case smf::ScalingMethod::Auto:
      if (!posdef && !ak.matching_scale.empty()) scale = ak.matching_scale.data();
      break;
    case smf::ScalingMethod::UserSupplied: scale = ctrl.user_scale; break;
    default: return fail(info, fk, smf::ErrorCode::FeatureNotAvailable);
  }
  std::lock_guard<std::mutex> lock(g_mu);
  PlanEntry *pe = plan_for(ak);
  if (!pe) return fail(info, fk, smf::ErrorCode::AllocationError);
  int64_t nnz_in = 0;
  {
    const std::size_t o2c = ak.orig_to_clean_idx.size();
    nnz_in = static_cast<int64_t>(o2c ? o2c : ak.cleaned.row_idx.size());
  }
  if (static_cast<int64_t>(nvals) != nnz_in) return fail(info, fk, smf::ErrorCode::IllegalValue);
  smfg_control_t c;
  smfg_default_control(&c);
  c.posdef = posdef ? 1 : 0;
  c.u = ctrl.pivot_u;
  c.small_pivot = ctrl.small_pivot;
  c.nb = ctrl.indef_panel_size;
  c.max_negative_pivots = posdef ? -1 : ctrl.max_negative_pivots;
  c.scale = scale;
  // smf's one-thread default mode keeps the threshold kernel on every front;
  // its deterministic mode takes the APTP kernel on indefinite fronts of at
  // least 512 rows (the engine's default)
  if (!smf::deterministic_mode(ctrl)) c.aptp_min_rows = 0;
  smfg_info_t gi{};
  const int rc = smfg_factor(pe->plan, values, &c, &gi);
  ++pe->generation;
  if (!posdef) {  // smf's SPD path leaves the counts at zero (factor_posdef.cpp)
    info.num_positive = gi.num_pos;
    info.num_negative = gi.num_neg;
    info.num_zero = gi.num_zero;
  }
  info.delayed_pivots = gi.delayed_pivots;
  info.two_by_two_pivots = gi.two_by_two_pivots;
  info.actual_flops = gi.flops;
  info.actual_factor_entries = gi.factor_entries;
  info.max_front_size = gi.max_front;
  info.aptp_failed_columns = gi.reserved_i[4];
  info.inertia_exact = true;
  fk.n = ak.n;
  fk.analysis = &ak;
  fk.is_posdef = posdef;
  smf::FactorStatus fs = smf::FactorStatus::Success;
  switch (gi.factor_status) {
    case SMFG_FACTOR_SUCCESS: fs = smf::FactorStatus::Success; break;
    case SMFG_FACTOR_NOT_POSDEF: fs = smf::FactorStatus::NotPositiveDefinite; break;
    case SMFG_FACTOR_SINGULAR: fs = smf::FactorStatus::Singular; break;
    case SMFG_FACTOR_MAX_PIVOT_DELAYS: fs = smf::FactorStatus::MaxPivotDelays; break;
    case SMFG_FACTOR_INERTIA_EXCEEDED: fs = smf::FactorStatus::InertiaExceeded; break;
    default: fs = smf::FactorStatus::Singular; break;
  }
  if (rc == SMFG_OK) info.status = smf::ErrorCode::Success;
  else if (rc == SMFG_ERR_SINGULAR) info.status = posdef ? smf::ErrorCode::NotPositiveDefinite
                                                         : smf::ErrorCode::SingularMatrix;
  else if (rc == SMFG_ERR_WRONG_INERTIA) info.status = smf::ErrorCode::InertiaExceeded;
  else if (rc == SMFG_ERR_NONFINITE) info.status = smf::ErrorCode::IllegalValue;
  else info.status = smf::ErrorCode::InternalError;
  if (rc != SMFG_OK && rc != SMFG_ERR_SINGULAR && rc != SMFG_ERR_WRONG_INERTIA) fs = smf::FactorStatus::Singular;
  info.factor_status = fs;
  fk.status = fs;
  // a solve can use the factor (a singular one too, as smf allows)
  const bool usable = (rc == SMFG_OK || (rc == SMFG_ERR_SINGULAR && fs == smf::FactorStatus::Singular));
  if (usable) {
    fk.factor_values.assign(1, 0.0);
    FactorEntry fe;
    fe.ak = &ak;
    fe.serial = ak.serial;
    fe.generation = pe->generation;
    fe.n = ak.n;
    fe.posdef = posdef;
    g_factors[&fk] = fe;
  } else {
    fk.factor_values.clear();
    g_factors.erase(&fk);
  }
  info.factor_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return fs;
}

int gpu_solve(const smf::FactorKeep &fk, smf::Info &info, double *b, int n, int nrhs, smf::SolveJob job) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_factors.find(&fk);
  if (it == g_factors.end() || fk.factor_values.empty()) {
    info.status = smf::ErrorCode::NotInitialised;
    return static_cast<int>(smf::ErrorCode::NotInitialised);
  }
  const FactorEntry &fe = it->second;
  auto pit = g_plans.find(fe.ak);
  // the plan holds the last factorization of its analysis: a FactorKeep
  // that an older factorization filled is no longer on the device
  if (pit == g_plans.end() || pit->second.serial != fe.serial || pit->second.generation != fe.generation) {
    info.status = smf::ErrorCode::NotInitialised;
    return static_cast<int>(smf::ErrorCode::NotInitialised);
  }
  if (n != fe.n || nrhs <= 0 || !b) {
    info.status = smf::ErrorCode::IllegalValue;
    return static_cast<int>(smf::ErrorCode::IllegalValue);
  }
  const auto t0 = std::chrono::steady_clock::now();
  int jobs[2] = {SMFG_SOLVE_FULL, -1};
  switch (job) {
    case smf::SolveJob::Full: break;
    case smf::SolveJob::Forward: jobs[0] = SMFG_SOLVE_FORWARD; break;
    case smf::SolveJob::DiagOnly: jobs[0] = SMFG_SOLVE_DIAGONAL; break;
    case smf::SolveJob::Backward: jobs[0] = SMFG_SOLVE_BACKWARD; break;
    case smf::SolveJob::DiagBack: jobs[0] = SMFG_SOLVE_DIAGONAL; jobs[1] = SMFG_SOLVE_BACKWARD; break;
  }
  for (int j : jobs) {
    if (j < 0) break;
    smfg_info_t si{};
    const int rc = smfg_solve(pit->second.plan, b, nrhs, n, j, &si);
    if (rc != SMFG_OK) {
      info.status = rc == SMFG_ERR_INVALID_ARG ? smf::ErrorCode::IllegalValue : smf::ErrorCode::InternalError;
      return static_cast<int>(info.status);
    }
  }
  info.status = smf::ErrorCode::Success;
  info.solve_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return 0;
}

}  // namespace

// The wrapped symbols: member functions take `this` first (Itanium C++ ABI);
// the names are the mangled ones of smf::Solver's declarations in
// smf/solver.hpp.
extern "C" {

smf::FactorStatus
__wrap__ZNK3smf6Solver6factorERKNS_12AnalysisKeepESt4spanIKdLm18446744073709551615EERKNS_7ControlERNS_4InfoERNS_10FactorKeepERNS_16NumericWorkspaceE(
    const smf::Solver *, const smf::AnalysisKeep &ak, std::span<const double> values, const smf::Control &ctrl,
    smf::Info &info, smf::FactorKeep &fkeep, smf::NumericWorkspace &) {
  return gpu_factor(ak, values.data(), values.size(), ctrl, info, fkeep);
}

smf::FactorStatus
__wrap__ZNK3smf6Solver6factorERKNS_12AnalysisKeepERKNS_8CscLowerERKNS_7ControlERNS_4InfoERNS_10FactorKeepERNS_16NumericWorkspaceE(
    const smf::Solver *, const smf::AnalysisKeep &ak, const smf::CscLower &updated, const smf::Control &ctrl,
    smf::Info &info, smf::FactorKeep &fkeep, smf::NumericWorkspace &) {
  return gpu_factor(ak, updated.values.data(), updated.values.size(), ctrl, info, fkeep);
}

int __wrap__ZNK3smf6Solver5solveERKNS_10FactorKeepERKNS_7ControlERNS_4InfoEPdiiNS_8SolveJobE(
    const smf::Solver *, const smf::FactorKeep &fkeep, const smf::Control &, smf::Info &info, double *b, int n,
    int nrhs, smf::SolveJob job) {
  return gpu_solve(fkeep, info, b, n, nrhs, job);
}

int __wrap__ZNK3smf6Solver5solveERKNS_10FactorKeepERKNS_7ControlERNS_4InfoEPdiiRNS_14SolveWorkspaceENS_8SolveJobE(
    const smf::Solver *, const smf::FactorKeep &fkeep, const smf::Control &, smf::Info &info, double *b, int n,
    int nrhs, smf::SolveWorkspace &, smf::SolveJob job) {
  return gpu_solve(fkeep, info, b, n, nrhs, job);
}

// Tests: the device plans this binding holds, and their release.
int smf_gpu_hook_plans(void) {
  std::lock_guard<std::mutex> lock(g_mu);
  return static_cast<int>(g_plans.size());
}
void smf_gpu_hook_release(void) {
  std::lock_guard<std::mutex> lock(g_mu);
  for (auto &kv : g_plans) smfg_plan_destroy(&kv.second.plan);
  g_plans.clear();
  g_factors.clear();
}

}  // extern "C"
