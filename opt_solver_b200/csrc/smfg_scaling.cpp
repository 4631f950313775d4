// Symmetric max-product matching scaling of a sparse symmetric matrix (host
// code): the scaling smf applies before an indefinite factorization when
// matching scaling is on (solver/src/scaling_matching.cpp, its result at
// :1011-1080), restated from the published method it follows:
//
//   - costs c_ij = log(max_k |a_kj|) - log |a_ij| >= 0 over the full
//     symmetric pattern (both triangles), as its build_cost_graph (:24);
//   - a minimum-cost perfect matching (MC64 job 5, Duff & Koster, "On
//     algorithms for permuting large entries to the diagonal of a sparse
//     matrix", SIAM J. Matrix Anal. Appl. 22, 2001): row reduction, a greedy
//     pass on zero-reduced-cost edges and a second one with a one-step
//     lookahead, then one Dijkstra shortest augmenting path per free column
//     on the reduced costs c - u - v >= 0, the dual potentials u (rows) and
//     v (columns) updated after each augmentation;
//   - scale[i] = exp((u_i + v_i - log colmax_i) / 2), v re-derived on the
//     matched edge, log-scale clamped to [-340, 340] (:1015-1016): then
//     |s_i a_ij s_j| <= 1 with equality on the matched entries.
//
// A column without an augmenting path (structurally singular matrix) keeps
// its duals and stays unmatched; the count is returned.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <limits>
#include <stdexcept>
#include <vector>

#include "../../include/smfg.h"

namespace {

struct HeapItem {
  double d;
  int row;
  bool operator>(const HeapItem &o) const { return d > o.d || (d == o.d && row > o.row); }
};

int matching_scale_impl(int n, const int *cp, const int *ri, const double *val, double *scale) {
  const double inf = std::numeric_limits<double>::infinity();
  // full symmetric pattern with |a|, per column
  std::vector<int64_t> cnt(n + 1, 0);
  for (int j = 0; j < n; ++j)
    for (int64_t k = cp[j]; k < cp[j + 1]; ++k) {
      const int i = ri[k];
      if (i < 0 || i >= n) throw std::invalid_argument("row index");
      if (!std::isfinite(val[k])) throw std::domain_error("non-finite");
      if (val[k] == 0.0) continue;
      cnt[j + 1]++;
      if (i != j) cnt[i + 1]++;
    }
  for (int j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
  std::vector<int> row(cnt[n]);
  std::vector<double> cost(cnt[n]);
  std::vector<double> cmax(n, 0.0);
  {
    std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
    for (int j = 0; j < n; ++j)
      for (int64_t k = cp[j]; k < cp[j + 1]; ++k) {
        const int i = ri[k];
        const double a = std::fabs(val[k]);
        if (a == 0.0) continue;
        row[pos[j]] = i;
        cost[pos[j]++] = a;
        cmax[j] = std::max(cmax[j], a);
        if (i != j) {
          row[pos[i]] = j;
          cost[pos[i]++] = a;
          cmax[i] = std::max(cmax[i], a);
        }
      }
  }
  std::vector<double> lcmax(n, 0.0);
  for (int j = 0; j < n; ++j) {
    if (!(cmax[j] > 0.0)) throw std::runtime_error("empty column");
    lcmax[j] = std::log(cmax[j]);
    for (int64_t k = cnt[j]; k < cnt[j + 1]; ++k) cost[k] = lcmax[j] - std::log(cost[k]);
  }
  // row reduction: u_i = min over its edges; v_j = min_i (c_ij - u_i)
  std::vector<double> u(n, inf), v(n, 0.0);
  for (int j = 0; j < n; ++j)
    for (int64_t k = cnt[j]; k < cnt[j + 1]; ++k) u[row[k]] = std::min(u[row[k]], cost[k]);
  for (int j = 0; j < n; ++j) {
    double m = inf;
    for (int64_t k = cnt[j]; k < cnt[j + 1]; ++k) m = std::min(m, cost[k] - u[row[k]]);
    v[j] = m;
  }
  // greedy matching on tight edges
  std::vector<int> row_mate(n, -1), col_mate(n, -1);
  for (int j = 0; j < n; ++j)
    for (int64_t k = cnt[j]; k < cnt[j + 1]; ++k) {
      const int i = row[k];
      if (row_mate[i] < 0 && cost[k] - u[i] - v[j] <= 0.0) {
        row_mate[i] = j;
        col_mate[j] = i;
        break;
      }
    }
  // second greedy pass (the one-step lookahead of MC64's initial matching):
  // a free column takes a tight row whose column can move to another tight,
  // free row; the duals stay as they are
  for (int j = 0; j < n; ++j) {
    if (col_mate[j] >= 0) continue;
    bool found = false;
    for (int64_t k = cnt[j]; k < cnt[j + 1] && !found; ++k) {
      const int i = row[k];
      if (cost[k] - u[i] - v[j] > 0.0) continue;
      const int jj = row_mate[i];
      if (jj < 0) {
        row_mate[i] = j;
        col_mate[j] = i;
        found = true;
        break;
      }
      for (int64_t q = cnt[jj]; q < cnt[jj + 1]; ++q) {
        const int i2 = row[q];
        if (row_mate[i2] < 0 && cost[q] - u[i2] - v[jj] <= 0.0) {
          row_mate[i2] = jj;
          col_mate[jj] = i2;
          row_mate[i] = j;
          col_mate[j] = i;
          found = true;
          break;
        }
      }
    }
  }
  // shortest augmenting paths from the free columns
  std::vector<double> dist(n, inf);
  std::vector<int> pred(n, -1);     // row -> column it was reached from
  std::vector<char> done(n, 0);
  std::vector<int> touched, popped;
  std::vector<HeapItem> heap;  // a binary min-heap on (distance, row), kept across searches
  const auto later = std::greater<HeapItem>();
  int unmatched = 0;
  for (int j0 = 0; j0 < n; ++j0) {
    if (col_mate[j0] >= 0) continue;
    heap.clear();
    touched.clear();
    popped.clear();
    // The search ends when the first free row leaves the heap, so no row
    // farther than the nearest free row found so far (lsp) can leave it
    // before that: such rows are not queued. The rows that leave the heap,
    // their order and the augmenting path are those of the unbounded search.
    double lsp = inf;
    auto relax = [&](int j, double dj) {
      for (int64_t k = cnt[j]; k < cnt[j + 1]; ++k) {
        const int i = row[k];
        if (done[i]) continue;
        const double nd = dj + std::max(0.0, cost[k] - u[i] - v[j]);
        if (nd > lsp) continue;
        if (row_mate[i] < 0) lsp = nd;
        if (nd < dist[i]) {
          if (dist[i] == inf) touched.push_back(i);
          dist[i] = nd;
          pred[i] = j;
          heap.push_back({nd, i});
          std::push_heap(heap.begin(), heap.end(), later);
        }
      }
    };
    relax(j0, 0.0);
    int free_row = -1;
    double D = inf;
    while (!heap.empty()) {
      std::pop_heap(heap.begin(), heap.end(), later);
      const HeapItem it = heap.back();
      heap.pop_back();
      const int i = it.row;
      if (done[i] || it.d > dist[i]) continue;
      done[i] = 1;
      popped.push_back(i);
      if (row_mate[i] < 0) {
        free_row = i;
        D = dist[i];
        break;
      }
      relax(row_mate[i], dist[i]);
    }
    if (free_row < 0) {
      ++unmatched;
    } else {
      // duals: popped rows and the columns reached through them
      v[j0] += D;
      for (int i : popped) {
        if (i == free_row) continue;
        const double delta = D - dist[i];
        u[i] -= delta;
        v[row_mate[i]] += delta;
      }
      // augment along the predecessors
      int i = free_row;
      while (true) {
        const int j = pred[i];
        const int prev = col_mate[j];
        col_mate[j] = i;
        row_mate[i] = j;
        if (j == j0) break;
        i = prev;
      }
    }
    for (int i : touched) {
      dist[i] = inf;
      pred[i] = -1;
      done[i] = 0;
    }
  }
  // v re-derived on the matched edge, then the symmetric scale
  for (int j = 0; j < n; ++j) {
    const int r = col_mate[j];
    if (r < 0) continue;
    for (int64_t k = cnt[j]; k < cnt[j + 1]; ++k)
      if (row[k] == r) {
        v[j] = cost[k] - u[r];
        break;
      }
  }
  for (int i = 0; i < n; ++i) {
    const double ls = (col_mate[i] >= 0 || row_mate[i] >= 0) ? 0.5 * (u[i] + v[i] - lcmax[i]) : -0.5 * lcmax[i];
    scale[i] = std::exp(std::clamp(std::isfinite(ls) ? ls : 0.0, -340.0, 340.0));
  }
  return unmatched;
}

}  // namespace

extern "C" {

SMFG_API int smfg_matching_scale(int n, const int *col_ptr, const int *row_idx, const double *values,
                                 double *scale, int *unmatched) {
  if (n < 0 || !col_ptr || !scale || (n > 0 && (!row_idx || !values))) return SMFG_ERR_INVALID_ARG;
  try {
    const int u = matching_scale_impl(n, col_ptr, row_idx, values, scale);
    if (unmatched) *unmatched = u;
    return SMFG_OK;
  } catch (const std::domain_error &) {
    return SMFG_ERR_NONFINITE;
  } catch (const std::invalid_argument &) {
    return SMFG_ERR_INVALID_ARG;
  } catch (const std::runtime_error &) {
    return SMFG_ERR_SINGULAR;  // a zero row / column
  } catch (...) {
    return SMFG_ERR_INTERNAL;
  }
}

}  // extern "C"
