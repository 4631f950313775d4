// Symbolic analysis for the engine's own use (bench and examples): the
// numeric phase consumes smf's analysis output as is (AnalysisKeep,
// solver/include/smf/analysis.hpp:25-144) and this file produces arrays of
// the same contract when smf's analyse is not at hand. It is a stand-in, not
// a restatement of smf's analyse (solver/src/symbolic_analysis.cpp:434):
//   - ordering: nested dissection with breadth-first level-set separators
//     from a pseudo-peripheral vertex (George, "Nested dissection of a
//     regular finite element mesh", SIAM J. Numer. Anal. 10, 1973; George &
//     Liu 1981), leaves in their given order;
//   - elimination tree by Liu's algorithm with path compression, postorder;
//   - column counts by row-subtree marking;
//   - fundamental supernodes, then relaxed amalgamation of a supernode into
//     its parent when the columns are contiguous and both are narrower than
//     nemin (smf's nemin rule, control.hpp:14) or the merge adds few zeros;
//   - front rows by merging the children's extension rows.
// The output follows AnalysisKeep's conventions: supernodes numbered in
// postorder, children listed in descending postorder, front rows sorted
// ascending with the pivots first, the permuted lower pattern and the maps
// from the caller's entries to it.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <vector>

#include "../../include/smfg.h"

namespace {

struct Graph {
  int n = 0;
  std::vector<int> xadj, adj;
};

// Breadth-first level structure of the vertices of `part` reachable from
// `root` (mark[v] == tag means v belongs to the current subset).
int bfs_levels(const Graph &g, int root, const std::vector<int> &mark, int tag, std::vector<int> &level,
               std::vector<int> &order) {
  order.clear();
  order.push_back(root);
  level[root] = 0;
  int depth = 0;
  for (size_t h = 0; h < order.size(); ++h) {
    const int v = order[h];
    for (int k = g.xadj[v]; k < g.xadj[v + 1]; ++k) {
      const int w = g.adj[k];
      if (mark[w] == tag && level[w] < 0) {
        level[w] = level[v] + 1;
        depth = std::max(depth, level[w]);
        order.push_back(w);
      }
    }
  }
  return depth;
}

struct NestedDissection {
  const Graph &g;
  int leaf;
  std::vector<int> mark, level, perm;  // perm: new -> old, filled from the back
  int next_back;
  int tag_counter = 1;
  std::vector<int> order;

  NestedDissection(const Graph &g_, int leaf_) : g(g_), leaf(leaf_) {
    mark.assign(g.n, 0);
    level.assign(g.n, -1);
    perm.assign(g.n, -1);
    next_back = g.n;
  }

  void emit_back(const std::vector<int> &vs) {
    for (int i = (int)vs.size() - 1; i >= 0; --i) perm[--next_back] = vs[i];
  }

  // Orders `verts` (a subset) into perm[next_back - |verts| .. next_back).
  void run(std::vector<int> verts) {
    struct Task { std::vector<int> v; };
    std::vector<Task> stack;
    stack.push_back({std::move(verts)});
    while (!stack.empty()) {
      std::vector<int> vs = std::move(stack.back().v);
      stack.pop_back();
      if ((int)vs.size() <= leaf) {
        emit_back(vs);
        continue;
      }
      const int tag = ++tag_counter;
      for (int v : vs) {
        mark[v] = tag;
        level[v] = -1;
      }
      // connected component of vs[0]
      int root = vs[0];
      bfs_levels(g, root, mark, tag, level, order);
      if (order.size() < vs.size()) {
        // disconnected: split off this component, push both
        std::vector<int> comp(order.begin(), order.end()), rest;
        for (int v : vs)
          if (level[v] < 0) rest.push_back(v);
        for (int v : vs) level[v] = -1;
        stack.push_back({std::move(rest)});
        stack.push_back({std::move(comp)});
        continue;
      }
      // pseudo-peripheral root: a few sweeps to the farthest vertex
      int depth = 0;
      for (int sweep = 0; sweep < 4; ++sweep) {
        int far = order.back();
        int minDeg = 1 << 30;
        const int last_level = level[order.back()];
        for (size_t h = order.size(); h-- > 0;) {
          const int v = order[h];
          if (level[v] != last_level) break;
          const int deg = g.xadj[v + 1] - g.xadj[v];
          if (deg < minDeg) {
            minDeg = deg;
            far = v;
          }
        }
        for (int v : vs) level[v] = -1;
        const int d = bfs_levels(g, far, mark, tag, level, order);
        root = far;
        if (d <= depth) break;
        depth = d;
      }
      // level sizes
      const int nl = level[order.back()] + 1;
      if (nl < 3) {
        emit_back(vs);
        for (int v : vs) level[v] = -1;
        continue;
      }
      std::vector<int> cnt(nl, 0);
      for (int v : vs) cnt[level[v]]++;
      // separator: the smallest level with 35-65% of the vertices before it
      const int total = (int)vs.size();
      int best = -1;
      long long best_score = 0;
      int before = 0;
      for (int l = 0; l < nl; ++l) {
        const int after = total - before - cnt[l];
        if (l > 0 && l < nl - 1 && before >= total * 35 / 100 && after >= total * 35 / 100) {
          const long long score = cnt[l];
          if (best < 0 || score < best_score) {
            best = l;
            best_score = score;
          }
        }
        before += cnt[l];
      }
      if (best < 0) {  // fall back to the median level
        before = 0;
        for (int l = 0; l < nl; ++l) {
          if (before + cnt[l] >= total / 2) {
            best = std::min(std::max(l, 1), nl - 2);
            break;
          }
          before += cnt[l];
        }
      }
      std::vector<int> A, B, S;
      for (int v : vs) {
        if (level[v] < best) A.push_back(v);
        else if (level[v] > best) B.push_back(v);
        else S.push_back(v);
      }
      for (int v : vs) level[v] = -1;
      emit_back(S);
      stack.push_back({std::move(A)});
      stack.push_back({std::move(B)});
    }
  }
};

}  // namespace

struct smfg_symbolic_s {
  int n = 0, nsn = 0;
  int64_t nnz_in = 0;
  std::vector<int> perm, sn_start, sn_end, sn_parent, child_ptr, child_idx, front_row_ptr,
      front_row_idx, postorder, perm_col_ptr, perm_row_idx, orig_to_clean, clean_to_perm,
      clean_col_ptr, clean_row_idx;
  double flops = 0.0;
  int64_t factor_entries = 0;
};

namespace {

void analyse_impl(smfg_symbolic_s &S, int n, const int *cp, const int *ri, int ordering, int nemin,
                  const int *given_perm = nullptr) {
  S.n = n;
  const int64_t nin = cp[n];
  S.nnz_in = nin;
  // cleaned lower pattern: (max, min) of each entry, sorted, duplicates merged
  std::vector<int64_t> key(nin);
  for (int j = 0; j < n; ++j)
    for (int64_t k = cp[j]; k < cp[j + 1]; ++k) {
      int i = ri[k];
      if (i < 0 || i >= n) throw std::invalid_argument("row index out of range");
      const int lo = std::min(i, j), hi = std::max(i, j);
      key[k] = (int64_t)lo * n + hi;
    }
  std::vector<int64_t> uk(key);
  std::sort(uk.begin(), uk.end());
  uk.erase(std::unique(uk.begin(), uk.end()), uk.end());
  const int64_t cnnz = (int64_t)uk.size();
  S.clean_col_ptr.assign(n + 1, 0);
  S.clean_row_idx.resize(cnnz);
  for (int64_t e = 0; e < cnnz; ++e) {
    S.clean_col_ptr[uk[e] / n + 1]++;
    S.clean_row_idx[e] = (int)(uk[e] % n);
  }
  for (int j = 0; j < n; ++j) S.clean_col_ptr[j + 1] += S.clean_col_ptr[j];
  S.orig_to_clean.resize(nin);
  for (int64_t k = 0; k < nin; ++k)
    S.orig_to_clean[k] = (int)(std::lower_bound(uk.begin(), uk.end(), key[k]) - uk.begin());
  // adjacency
  Graph g;
  g.n = n;
  g.xadj.assign(n + 1, 0);
  for (int j = 0; j < n; ++j)
    for (int64_t e = S.clean_col_ptr[j]; e < S.clean_col_ptr[j + 1]; ++e) {
      const int i = S.clean_row_idx[e];
      if (i != j) {
        g.xadj[i + 1]++;
        g.xadj[j + 1]++;
      }
    }
  for (int i = 0; i < n; ++i) g.xadj[i + 1] += g.xadj[i];
  g.adj.resize(g.xadj[n]);
  {
    std::vector<int> pos(g.xadj.begin(), g.xadj.end() - 1);
    for (int j = 0; j < n; ++j)
      for (int64_t e = S.clean_col_ptr[j]; e < S.clean_col_ptr[j + 1]; ++e) {
        const int i = S.clean_row_idx[e];
        if (i != j) {
          g.adj[pos[i]++] = j;
          g.adj[pos[j]++] = i;
        }
      }
  }
  // ordering
  std::vector<int> perm(n);
  if (given_perm) {
    std::vector<char> seen(n, 0);
    for (int i = 0; i < n; ++i) {
      const int o = given_perm[i];
      if (o < 0 || o >= n || seen[o]) throw std::invalid_argument("not a permutation");
      seen[o] = 1;
      perm[i] = o;
    }
  } else if (ordering == 1) {
    std::iota(perm.begin(), perm.end(), 0);
  } else {
    NestedDissection nd(g, ordering == 2 ? 16 : 32);
    std::vector<int> all(n);
    std::iota(all.begin(), all.end(), 0);
    nd.run(std::move(all));
    perm = nd.perm;
  }
  std::vector<int> iperm(n);
  // etree of P A P^T, then a postorder, composed into the ordering
  auto etree_of = [&](const std::vector<int> &pm, std::vector<int> &parent) {
    std::vector<int> ip(n);
    for (int i = 0; i < n; ++i) ip[pm[i]] = i;
    // rows of the permuted lower triangle: for new row i, new cols j < i
    std::vector<int> rptr(n + 1, 0), rcol;
    for (int j = 0; j < n; ++j)
      for (int64_t e = S.clean_col_ptr[j]; e < S.clean_col_ptr[j + 1]; ++e) {
        const int a = ip[S.clean_row_idx[e]], b = ip[j];
        if (a != b) rptr[std::max(a, b) + 1]++;
      }
    for (int i = 0; i < n; ++i) rptr[i + 1] += rptr[i];
    rcol.resize(rptr[n]);
    std::vector<int> pos(rptr.begin(), rptr.end() - 1);
    for (int j = 0; j < n; ++j)
      for (int64_t e = S.clean_col_ptr[j]; e < S.clean_col_ptr[j + 1]; ++e) {
        const int a = ip[S.clean_row_idx[e]], b = ip[j];
        if (a != b) rcol[pos[std::max(a, b)]++] = std::min(a, b);
      }
    parent.assign(n, -1);
    std::vector<int> anc(n, -1);
    for (int i = 0; i < n; ++i) {
      for (int k = rptr[i]; k < rptr[i + 1]; ++k) {
        int r = rcol[k];
        while (r != -1 && r < i) {
          const int nx = anc[r];
          anc[r] = i;
          if (nx == -1) {
            parent[r] = i;
            break;
          }
          r = nx;
        }
      }
    }
    return std::make_pair(rptr, rcol);
  };
  std::vector<int> parent;
  etree_of(perm, parent);
  {
    // postorder (children in increasing order)
    std::vector<int> head(n, -1), nxt(n, -1), post;
    post.reserve(n);
    for (int v = n - 1; v >= 0; --v)
      if (parent[v] >= 0) {
        nxt[v] = head[parent[v]];
        head[parent[v]] = v;
      }
    std::vector<int> stack;
    for (int r = 0; r < n; ++r) {
      if (parent[r] != -1) continue;
      stack.push_back(r);
      while (!stack.empty()) {
        const int v = stack.back();
        if (head[v] != -1) {
          const int c = head[v];
          head[v] = nxt[c];
          stack.push_back(c);
        } else {
          stack.pop_back();
          post.push_back(v);
        }
      }
    }
    std::vector<int> p2(n);
    for (int k = 0; k < n; ++k) p2[k] = perm[post[k]];
    perm = p2;
  }
  auto rows = etree_of(perm, parent);
  const std::vector<int> &rptr = rows.first, &rcol = rows.second;
  for (int i = 0; i < n; ++i) iperm[perm[i]] = i;
  // column counts by row-subtree marking
  std::vector<int> cc(n, 1), mark(n, -1);
  for (int i = 0; i < n; ++i) {
    mark[i] = i;
    for (int k = rptr[i]; k < rptr[i + 1]; ++k) {
      int j = rcol[k];
      while (j != -1 && mark[j] != i) {
        cc[j]++;
        mark[j] = i;
        j = parent[j];
      }
    }
  }
  // fundamental supernodes
  std::vector<int> nchild(n, 0);
  for (int j = 0; j < n; ++j)
    if (parent[j] >= 0) nchild[parent[j]]++;
  std::vector<int> fstart;
  for (int j = 0; j < n; ++j) {
    const bool cont = j > 0 && parent[j - 1] == j && nchild[j] == 1 && cc[j - 1] == cc[j] + 1;
    if (!cont) fstart.push_back(j);
  }
  fstart.push_back(n);
  const int nf = (int)fstart.size() - 1;
  // supernode of each column, its parent supernode
  std::vector<int> col_sn(n);
  for (int s = 0; s < nf; ++s)
    for (int j = fstart[s]; j < fstart[s + 1]; ++j) col_sn[j] = s;
  // front rows bottom-up (supernodes in column order are a postorder):
  // A's rows below the pivots (both triangles: the symmetric adjacency)
  // and the children's extension rows below them.
  std::vector<int> sstart(fstart.begin(), fstart.end() - 1), send(fstart.begin() + 1, fstart.end());
  std::vector<int> sparent(nf, -1);
  for (int s = 0; s < nf; ++s) {
    const int last = send[s] - 1;
    sparent[s] = parent[last] >= 0 ? col_sn[parent[last]] : -1;
  }
  std::vector<std::vector<int>> kids(nf);
  for (int s = 0; s < nf; ++s)
    if (sparent[s] >= 0) kids[sparent[s]].push_back(s);
  std::vector<std::vector<int>> rowsets(nf);
  std::vector<int> tmp;
  for (int s = 0; s < nf; ++s) {
    tmp.clear();
    for (int j = sstart[s]; j < send[s]; ++j) {
      const int oj = perm[j];
      for (int k = g.xadj[oj]; k < g.xadj[oj + 1]; ++k) {
        const int i = iperm[g.adj[k]];
        if (i >= send[s]) tmp.push_back(i);
      }
    }
    for (int c : kids[s])
      for (int r : rowsets[c])
        if (r >= send[s]) tmp.push_back(r);
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    rowsets[s] = tmp;
  }
  // relaxed amalgamation: child c merges into its parent p when c's columns
  // end where p's begin and both are narrower than nemin, or the merge adds
  // few explicit zeros (at most 16, or 30% of the merged entries)
  std::vector<int> g_start = sstart, g_end = send, g_par(nf, -1);
  std::vector<std::vector<int>> g_rows = rowsets;
  std::vector<int> owner(nf);
  std::iota(owner.begin(), owner.end(), 0);
  auto find = [&](int s) {
    while (owner[s] != s) s = owner[s] = owner[owner[s]];
    return s;
  };
  for (int s = 0; s < nf; ++s) {
    const int rs = find(s);
    const int p = sparent[s];
    if (p < 0) continue;
    const int rp = find(p);
    if (g_end[rs] != g_start[rp]) continue;  // not contiguous
    const int wc = g_end[rs] - g_start[rs], wp = g_end[rp] - g_start[rp];
    // zeros added: the child's pivot columns get the parent's rows
    const long long fc = wc + (long long)g_rows[rs].size();
    const long long fp = wp + (long long)g_rows[rp].size();
    const long long newf = wc + fp;
    const long long zeros = (long long)wc * (newf - fc);
    const long long total_ent = (long long)wc * newf + (long long)wp * fp;
    const bool small = wc < nemin && wp < nemin;
    const bool few_zeros = zeros <= 16 || zeros * 10 <= total_ent * 3;
    // a chain of wide fronts whose patterns nest (the dense top of a poorly
    // separable graph) merges at any width when it adds under 2% zeros
    const bool nested = zeros * 50 <= total_ent;
    if (!(small || nested || (few_zeros && wc + wp <= 4 * nemin))) continue;
    // merge rs into rp
    g_start[rp] = g_start[rs];
    owner[rs] = rp;
    std::vector<int>().swap(g_rows[rs]);
  }
  // final supernodes: roots of the union-find, in increasing column order
  std::vector<int> final_id(nf, -1);
  int nsn = 0;
  std::vector<int> reps;
  for (int s = 0; s < nf; ++s)
    if (find(s) == s) reps.push_back(s);
  std::sort(reps.begin(), reps.end(), [&](int a, int b) { return g_start[a] < g_start[b]; });
  for (int r : reps) final_id[r] = nsn++;
  S.nsn = nsn;
  S.sn_start.resize(nsn);
  S.sn_end.resize(nsn);
  S.sn_parent.assign(nsn, -1);
  std::vector<int> colfinal(n);
  for (int r : reps) {
    const int id = final_id[r];
    S.sn_start[id] = g_start[r];
    S.sn_end[id] = g_end[r];
    for (int j = g_start[r]; j < g_end[r]; ++j) colfinal[j] = id;
  }
  for (int id = 0; id < nsn; ++id) {
    const int last = S.sn_end[id] - 1;
    S.sn_parent[id] = parent[last] >= 0 ? colfinal[parent[last]] : -1;
  }
  // front rows: pivots + extension rows (a merged child's extension rows
  // are contained in the parent's front: the parent's rows cover them)
  S.front_row_ptr.assign(nsn + 1, 0);
  for (int r : reps) {
    const int id = final_id[r];
    S.front_row_ptr[id + 1] = (S.sn_end[id] - S.sn_start[id]) + (int)g_rows[r].size();
  }
  for (int id = 0; id < nsn; ++id) S.front_row_ptr[id + 1] += S.front_row_ptr[id];
  S.front_row_idx.resize(S.front_row_ptr[nsn]);
  for (int r : reps) {
    const int id = final_id[r];
    int o = S.front_row_ptr[id];
    for (int j = S.sn_start[id]; j < S.sn_end[id]; ++j) S.front_row_idx[o++] = j;
    for (int x : g_rows[r]) S.front_row_idx[o++] = x;
  }
  // children in descending postorder; supernodes are numbered in postorder
  // (increasing first column is a postorder of the postordered etree)
  std::vector<int> ccount(nsn + 1, 0);
  for (int id = 0; id < nsn; ++id)
    if (S.sn_parent[id] >= 0) ccount[S.sn_parent[id] + 1]++;
  S.child_ptr.assign(nsn + 1, 0);
  for (int id = 0; id < nsn; ++id) S.child_ptr[id + 1] = S.child_ptr[id] + ccount[id + 1];
  S.child_idx.resize(S.child_ptr[nsn]);
  {
    std::vector<int> pos(S.child_ptr.begin(), S.child_ptr.end() - 1);
    for (int id = nsn - 1; id >= 0; --id)
      if (S.sn_parent[id] >= 0) S.child_idx[pos[S.sn_parent[id]]++] = id;
  }
  S.postorder.resize(nsn);
  std::iota(S.postorder.begin(), S.postorder.end(), 0);
  // permuted lower pattern and the cleaned -> permuted map
  S.perm = perm;
  S.perm_col_ptr.assign(n + 1, 0);
  std::vector<int64_t> pk(cnnz);
  for (int j = 0; j < n; ++j)
    for (int64_t e = S.clean_col_ptr[j]; e < S.clean_col_ptr[j + 1]; ++e) {
      const int a = iperm[S.clean_row_idx[e]], b = iperm[j];
      pk[e] = (int64_t)std::min(a, b) * n + std::max(a, b);
    }
  std::vector<int64_t> order(cnnz);
  std::iota(order.begin(), order.end(), 0);
  std::sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return pk[x] < pk[y]; });
  S.perm_row_idx.resize(cnnz);
  S.clean_to_perm.resize(cnnz);
  for (int64_t t = 0; t < cnnz; ++t) {
    const int64_t e = order[t];
    S.perm_col_ptr[pk[e] / n + 1]++;
    S.perm_row_idx[t] = (int)(pk[e] % n);
    S.clean_to_perm[e] = (int)t;
  }
  for (int j = 0; j < n; ++j) S.perm_col_ptr[j + 1] += S.perm_col_ptr[j];
  // delay-free flops (smf's count, ldlt_kernel.cpp:678-679) and |L|
  S.flops = 0.0;
  S.factor_entries = 0;
  for (int id = 0; id < nsn; ++id) {
    const int f = S.front_row_ptr[id + 1] - S.front_row_ptr[id];
    const int p = S.sn_end[id] - S.sn_start[id];
    S.factor_entries += (int64_t)f * p;
    for (int k = 0; k < p; ++k) {
      const double r = f - k - 1.0;
      S.flops += r + r * (r + 1.0);
    }
  }
}

}  // namespace

extern "C" {

SMFG_API int smfg_analyse(int n, const int *col_ptr, const int *row_idx, int ordering, int nemin,
                          smfg_symbolic_t *out) {
  if (!out || n < 0 || !col_ptr || (!row_idx && col_ptr[n] > 0)) return SMFG_ERR_INVALID_ARG;
  *out = nullptr;
  auto *S = new smfg_symbolic_s();
  try {
    analyse_impl(*S, n, col_ptr, row_idx, ordering, nemin > 0 ? nemin : 8);
  } catch (const std::invalid_argument &) {
    delete S;
    return SMFG_ERR_INVALID_ARG;
  } catch (...) {
    delete S;
    return SMFG_ERR_INTERNAL;
  }
  *out = S;
  return SMFG_OK;
}

SMFG_API int smfg_analyse_ordered(int n, const int *col_ptr, const int *row_idx, const int *perm,
                                  int nemin, smfg_symbolic_t *out) {
  if (!out || n < 0 || !col_ptr || !perm || (!row_idx && col_ptr[n] > 0)) return SMFG_ERR_INVALID_ARG;
  *out = nullptr;
  auto *S = new smfg_symbolic_s();
  try {
    analyse_impl(*S, n, col_ptr, row_idx, 1, nemin > 0 ? nemin : 8, perm);
  } catch (const std::invalid_argument &) {
    delete S;
    return SMFG_ERR_INVALID_ARG;
  } catch (...) {
    delete S;
    return SMFG_ERR_INTERNAL;
  }
  *out = S;
  return SMFG_OK;
}

SMFG_API int smfg_symbolic_view(smfg_symbolic_t s, smfg_analysis_t *a, double *flops,
                                int64_t *factor_entries) {
  if (!s || !a) return SMFG_ERR_INVALID_ARG;
  a->n = s->n;
  a->nsn = s->nsn;
  a->perm = s->perm.data();
  a->sn_start = s->sn_start.data();
  a->sn_end = s->sn_end.data();
  a->sn_parent = s->sn_parent.data();
  a->child_ptr = s->child_ptr.data();
  a->child_idx = s->child_idx.data();
  a->front_row_ptr = s->front_row_ptr.data();
  a->front_row_idx = s->front_row_idx.data();
  a->postorder = s->postorder.data();
  a->perm_col_ptr = s->perm_col_ptr.data();
  a->perm_row_idx = s->perm_row_idx.data();
  a->nnz_in = s->nnz_in;
  a->orig_to_clean = s->orig_to_clean.data();
  a->clean_to_perm = s->clean_to_perm.data();
  a->clean_col_ptr = s->clean_col_ptr.data();
  a->clean_row_idx = s->clean_row_idx.data();
  if (flops) *flops = s->flops;
  if (factor_entries) *factor_entries = s->factor_entries;
  return SMFG_OK;
}

SMFG_API void smfg_symbolic_free(smfg_symbolic_t *s) {
  if (!s || !*s) return;
  delete *s;
  *s = nullptr;
}

}  // extern "C"
