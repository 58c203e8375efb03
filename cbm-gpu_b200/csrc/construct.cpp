// CBM construction on the host: binary adjacency A -> (delta matrix, compression tree).
//
// Restates cbm_init_ (cbm/cbm_extensions.cpp:60-345) without MKL or arbok:
//
//  1. COO -> CSR with sorted, unique columns per row (the reference's
//     mkl_sparse_convert_csr, :70-98; duplicate (row, col) pairs are merged,
//     values are ignored: the format stores the binary pattern only).
//  2. Candidate edges of the distance graph, in the reference's order
//     (:123-151): for row = 0..N-1 the virtual edge (N -> row, nnz(row)),
//     then for every col > row with o = |A[row] & A[col]| > 0, ascending col:
//        (col -> row, h) if h < nnz(row) - alpha && h != nnz(row)
//        (row -> col, h) if h < nnz(col) - alpha && h != nnz(col)
//     with h = nnz(row) + nnz(col) - 2*o.  The reference reads o from the upper
//     triangle of syrk(A) (:101-120); here the qualifying pairs are found
//     exactly with a prefix filter, so A*A^T is never materialised.
//  3. A minimum-cost arborescence rooted at the virtual node N (the reference
//     calls arbok::TarjanPQ, :154-189).  Implemented here as Tarjan's
//     contraction algorithm with meldable (leftist) heaps and a rollback
//     union-find; ties are broken by the candidate index, so the result is
//     deterministic.  arbok's own tie-breaking is not reproduced.
//  4. Delta rows and tree edges by BFS over each non-empty branch (:191-299):
//     root children emit their row as +1 entries; each tree edge (u, v) emits
//     A[v] - A[u] by a sorted merge; branch offsets are prefix-summed.
//
// Children of a node are visited in increasing candidate index of their tree
// edge (the reference visits them in the order arbok's reconstruct returns).

#include "cbm_b200.h"

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <deque>
#include <new>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct Csr {
  int64_t n = 0;
  std::vector<int64_t> ptr;  // n + 1
  std::vector<int32_t> idx;  // sorted, unique per row
};

// ---------------------------------------------------------------------------
// 1. COO -> CSR (sorted, unique)
// ---------------------------------------------------------------------------
Csr coo_to_csr(const int32_t* row, const int32_t* col, int64_t nnz, int64_t n) {
  Csr a;
  a.n = n;
  a.ptr.assign(n + 1, 0);
  // already coalesced (sorted by row, then strictly by column): the CSR is the
  // column array itself, the row pointers are where the row id changes
  bool coalesced = true;
#pragma omp parallel for reduction(&& : coalesced) schedule(static)
  for (int64_t k = 1; k < nnz; ++k)
    if (row[k] < row[k - 1] || (row[k] == row[k - 1] && col[k] <= col[k - 1])) coalesced = false;
  if (coalesced) {
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nnz; ++k)
      if (k == nnz - 1 || row[k + 1] != row[k]) a.ptr[row[k] + 1] = k + 1;
    for (int64_t i = 0; i < n; ++i) a.ptr[i + 1] = std::max(a.ptr[i + 1], a.ptr[i]);
    a.idx.assign(col, col + nnz);
    return a;
  }
  for (int64_t k = 0; k < nnz; ++k) a.ptr[row[k] + 1]++;
  for (int64_t i = 0; i < n; ++i) a.ptr[i + 1] += a.ptr[i];
  std::vector<int32_t> tmp(nnz);
  std::vector<int64_t> fill(a.ptr.begin(), a.ptr.end() - 1);
  for (int64_t k = 0; k < nnz; ++k) tmp[fill[row[k]]++] = col[k];
  // sort + unique each row
  std::vector<int64_t> newlen(n, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < n; ++i) {
    auto b = tmp.begin() + a.ptr[i], e = tmp.begin() + a.ptr[i + 1];
    if (!std::is_sorted(b, e)) std::sort(b, e);
    newlen[i] = std::unique(b, e) - b;
  }
  std::vector<int64_t> nptr(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) nptr[i + 1] = nptr[i] + newlen[i];
  a.idx.resize(nptr[n]);
#pragma omp parallel for schedule(static, 4096)
  for (int64_t i = 0; i < n; ++i)
    std::memcpy(a.idx.data() + nptr[i], tmp.data() + a.ptr[i], sizeof(int32_t) * newlen[i]);
  a.ptr.swap(nptr);
  return a;
}

// ---------------------------------------------------------------------------
// 2. Candidate pairs
// ---------------------------------------------------------------------------
struct Pair {
  int32_t lo, hi;  // lo < hi (row, col of the syrk upper triangle)
  int32_t o;       // |A[lo] & A[hi]|
};

inline int64_t floor_div2(int64_t x) { return x >= 0 ? x / 2 : -((-x + 1) / 2); }

// Pairs {s, l} with (n_s, s) < (n_l, l) and 2*o > n_s + alpha, o >= 1.  Every
// pair that can yield a candidate in either direction satisfies this (both
// directions need 2*o > n_parent + alpha >= n_s + alpha).
//
// Prefix filter: order each row's columns by global rarity (column count,
// then id).  If o >= t then the first n_s - t + 1 columns of s in that order
// contain a column of A[l]; candidates are activated there and their exact
// overlap is completed over the remaining t - 1 columns, dropping those that
// can no longer reach t.
// Stable counting sort of 0..n-1 by key[i] (small non-negative integers): the
// order std::stable_sort by key gives, in O(n + max key).
template <typename K>
std::vector<int32_t> order_by_key(const std::vector<K>& key) {
  const int64_t n = (int64_t)key.size();
  K kmax = 0;
  for (int64_t i = 0; i < n; ++i) kmax = std::max(kmax, key[i]);
  std::vector<int64_t> start((size_t)kmax + 2, 0);
  for (int64_t i = 0; i < n; ++i) start[(size_t)key[i] + 1]++;
  for (size_t b = 0; b + 1 < start.size(); ++b) start[b + 1] += start[b];
  std::vector<int32_t> order(n);
  for (int64_t i = 0; i < n; ++i) order[start[(size_t)key[i]]++] = (int32_t)i;
  return order;
}

std::vector<Pair> candidate_pairs(const Csr& a, int64_t alpha, int n_threads) {
  const int64_t n = a.n;
  int nt = 1;
#ifdef _OPENMP
  nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#endif
  std::vector<int32_t> rowlen(n);
  for (int64_t i = 0; i < n; ++i) rowlen[i] = (int32_t)(a.ptr[i + 1] - a.ptr[i]);

  // column counts and rarity rank (column count, then id)
  std::vector<int64_t> colcnt(n, 0);
  for (int64_t k = 0; k < (int64_t)a.idx.size(); ++k) colcnt[a.idx[k]]++;
  std::vector<int32_t> by_rarity = order_by_key(colcnt);
  std::vector<int32_t> rank(n);
  for (int64_t r = 0; r < n; ++r) rank[by_rarity[r]] = (int32_t)r;

  // rows ordered by (rowlen, id): position of each row in that order
  std::vector<int32_t> by_size = order_by_key(rowlen);
  std::vector<int32_t> size_pos(n);
  for (int64_t r = 0; r < n; ++r) size_pos[by_size[r]] = (int32_t)r;

  // inverted lists: the size positions of the rows containing column c, in
  // increasing order (positions, not row ids: the searches and scans below then
  // compare plain integers; by_size maps a position back to its row).  Built in
  // parallel: thread t fills the positions of its own contiguous range of
  // positions after those of threads 0..t-1, so every list stays sorted.
  std::vector<int64_t> iptr(n + 1, 0);
  for (int64_t c = 0; c < n; ++c) iptr[c + 1] = iptr[c] + colcnt[c];
  std::vector<int32_t> inv(a.idx.size());
  {
    const int parts = std::max(1, std::min<int>(nt, (int)std::max<int64_t>(1, n / 65536)));
    std::vector<std::vector<int64_t>> fill(parts);
#pragma omp parallel for num_threads(parts) schedule(static, 1)
    for (int t = 0; t < parts; ++t) {
      fill[t].assign(n, 0);
      const int64_t r0 = n * t / parts, r1 = n * (t + 1) / parts;
      for (int64_t r = r0; r < r1; ++r) {
        const int32_t row = by_size[r];
        for (int64_t k = a.ptr[row]; k < a.ptr[row + 1]; ++k) fill[t][a.idx[k]]++;
      }
    }
    // per column: exclusive offsets of each part, starting at the column's list
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t c = 0; c < n; ++c) {
      int64_t o = iptr[c];
      for (int t = 0; t < parts; ++t) {
        const int64_t k = fill[t][c];
        fill[t][c] = o;
        o += k;
      }
    }
#pragma omp parallel for num_threads(parts) schedule(static, 1)
    for (int t = 0; t < parts; ++t) {
      const int64_t r0 = n * t / parts, r1 = n * (t + 1) / parts;
      for (int64_t r = r0; r < r1; ++r) {
        const int32_t row = by_size[r];
        for (int64_t k = a.ptr[row]; k < a.ptr[row + 1]; ++k) inv[fill[t][a.idx[k]]++] = (int32_t)r;
      }
    }
  }

  std::vector<std::vector<Pair>> out(nt);

#pragma omp parallel num_threads(nt)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    // indexed by size position; stamp and count side by side (one cache line
    // per candidate touched)
    struct Slot {
      int32_t stamp, cnt;
    };
    std::vector<Slot> slot(n, Slot{-1, 0});
    std::vector<int32_t> cand, cols;
    std::vector<Pair>& mine = out[tid];

#pragma omp for schedule(dynamic, 512)
    for (int64_t si = 0; si < n; ++si) {
      const int32_t s = (int32_t)si;
      const int64_t ns = rowlen[s];
      if (ns == 0) continue;
      const int64_t t = std::max<int64_t>(1, floor_div2(ns + alpha) + 1);
      if (t > ns) continue;  // o <= n_s < t: no pair with s as the smaller side
      const int64_t plen = ns - t + 1;
      cols.assign(a.idx.begin() + a.ptr[s], a.idx.begin() + a.ptr[s + 1]);
      std::sort(cols.begin(), cols.end(), [&](int32_t x, int32_t y) { return rank[x] < rank[y]; });
      const int32_t my_pos = size_pos[s];
      cand.clear();
      // prefix: activate (candidates are the larger rows: positions above my_pos)
      for (int64_t j = 0; j < plen; ++j) {
        const int32_t c = cols[j];
        const int32_t* lb = inv.data() + iptr[c];
        const int32_t* le = inv.data() + iptr[c + 1];
        for (const int32_t* p = std::upper_bound(lb, le, my_pos); p < le; ++p) {
          const int32_t l = *p;
          if (slot[l].stamp != s) {
            slot[l].stamp = s;
            slot[l].cnt = 1;
            cand.push_back(l);
          } else {
            slot[l].cnt++;
          }
        }
      }
      // suffix: complete the overlap of live candidates, pruning the hopeless
      int64_t live = (int64_t)cand.size();
      for (int64_t j = plen; j < ns && live > 0; ++j) {
        const int32_t c = cols[j];
        const int64_t remaining_after = ns - j - 1;
        const int32_t* lb = inv.data() + iptr[c];
        const int32_t* le = inv.data() + iptr[c + 1];
        const int32_t* st = std::upper_bound(lb, le, my_pos);
        if ((le - st) <= live * 8) {
          for (const int32_t* p = st; p < le; ++p)
            if (slot[*p].stamp == s) slot[*p].cnt++;
        } else {
          for (int64_t q = 0; q < live; ++q) {
            const int32_t l = by_size[cand[q]];
            const int32_t* rb = a.idx.data() + a.ptr[l];
            const int32_t* re = a.idx.data() + a.ptr[l + 1];
            if (std::binary_search(rb, re, c)) slot[cand[q]].cnt++;
          }
        }
        // prune
        int64_t w = 0;
        for (int64_t q = 0; q < live; ++q) {
          const int32_t l = cand[q];
          if (slot[l].cnt + remaining_after >= t) {
            cand[w++] = l;
          } else {
            slot[l].stamp = -2;  // dead for this s (stamps are row ids >= 0)
          }
        }
        live = w;
      }
      for (int64_t q = 0; q < live; ++q) {
        const int32_t lp = cand[q];
        if (slot[lp].cnt >= t) {
          const int32_t l = by_size[lp];
          Pair p;
          p.lo = std::min(s, l);
          p.hi = std::max(s, l);
          p.o = slot[lp].cnt;
          mine.push_back(p);
        }
      }
      // stamps hold row ids and each row is visited once, so no reset is needed
    }
  }

  // group by lo, order by hi: the order in which the reference meets them
  std::vector<int64_t> bptr(n + 1, 0);
  size_t total = 0;
  for (auto& v : out) {
    total += v.size();
    for (auto& p : v) bptr[p.lo + 1]++;
  }
  for (int64_t i = 0; i < n; ++i) bptr[i + 1] += bptr[i];
  std::vector<Pair> pairs(total);
  {
    std::vector<int64_t> fill(bptr.begin(), bptr.end() - 1);
    for (auto& v : out)
      for (auto& p : v) pairs[fill[p.lo]++] = p;
  }
#pragma omp parallel for schedule(dynamic, 4096) num_threads(nt)
  for (int64_t i = 0; i < n; ++i)
    std::sort(pairs.begin() + bptr[i], pairs.begin() + bptr[i + 1],
              [](const Pair& x, const Pair& y) { return x.hi < y.hi; });
  return pairs;
}

// Exhaustive variant (the reference's syrk semantics taken literally): every
// pair sharing a column.  Used to cross-check the prefix filter.
std::vector<Pair> candidate_pairs_exhaustive(const Csr& a, int64_t alpha, int n_threads) {
  const int64_t n = a.n;
  std::vector<int64_t> iptr(n + 1, 0);
  for (int64_t k = 0; k < (int64_t)a.idx.size(); ++k) iptr[a.idx[k] + 1]++;
  for (int64_t c = 0; c < n; ++c) iptr[c + 1] += iptr[c];
  std::vector<int32_t> inv(a.idx.size());
  {
    std::vector<int64_t> fill(iptr.begin(), iptr.end() - 1);
    for (int64_t r = 0; r < n; ++r)
      for (int64_t k = a.ptr[r]; k < a.ptr[r + 1]; ++k) inv[fill[a.idx[k]]++] = (int32_t)r;
  }
  int nt = 1;
#ifdef _OPENMP
  nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#endif
  std::vector<std::vector<Pair>> rows_out(n);
#pragma omp parallel num_threads(nt)
  {
    std::vector<int32_t> cnt(n, 0), touched;
#pragma omp for schedule(dynamic, 256)
    for (int64_t u = 0; u < n; ++u) {
      touched.clear();
      for (int64_t k = a.ptr[u]; k < a.ptr[u + 1]; ++k) {
        const int32_t c = a.idx[k];
        const int32_t* lb = inv.data() + iptr[c];
        const int32_t* le = inv.data() + iptr[c + 1];
        for (const int32_t* p = std::upper_bound(lb, le, (int32_t)u); p < le; ++p) {
          if (cnt[*p]++ == 0) touched.push_back(*p);
        }
      }
      std::sort(touched.begin(), touched.end());
      const int64_t nu = a.ptr[u + 1] - a.ptr[u];
      for (int32_t v : touched) {
        const int64_t nv = a.ptr[v + 1] - a.ptr[v];
        const int64_t o = cnt[v];
        cnt[v] = 0;
        if (2 * o > std::min(nu, nv) + alpha) rows_out[u].push_back(Pair{(int32_t)u, v, (int32_t)o});
      }
    }
  }
  std::vector<Pair> pairs;
  for (auto& r : rows_out) pairs.insert(pairs.end(), r.begin(), r.end());
  return pairs;
}

// ---------------------------------------------------------------------------
// 3. Minimum-cost arborescence (Tarjan contraction with leftist heaps)
// ---------------------------------------------------------------------------
struct Arb {
  // candidate edges
  std::vector<int32_t> from, to;
  std::vector<int64_t> w;
};

class LeftistPool {
 public:
  explicit LeftistPool(size_t m) : key_(m), lazy_(m, 0), l_(m, -1), r_(m, -1), rk_(m, 1) {}
  void init(int32_t e, int64_t key) { key_[e] = key; }
  int32_t meld(int32_t a, int32_t b) {
    if (a < 0) return b;
    if (b < 0) return a;
    push(a);
    push(b);
    if (less(b, a)) std::swap(a, b);
    r_[a] = meld(r_[a], b);
    if (l_[a] < 0 || (r_[a] >= 0 && rk_[l_[a]] < rk_[r_[a]])) std::swap(l_[a], r_[a]);
    rk_[a] = (r_[a] < 0 ? 0 : rk_[r_[a]]) + 1;
    return a;
  }
  int32_t pop(int32_t a) {
    push(a);
    return meld(l_[a], r_[a]);
  }
  int64_t top_key(int32_t a) {
    push(a);
    return key_[a];
  }
  void add(int32_t a, int64_t d) {
    if (a >= 0) lazy_[a] += d;
  }

 private:
  bool less(int32_t x, int32_t y) const {
    return key_[x] < key_[y] || (key_[x] == key_[y] && x < y);
  }
  void push(int32_t a) {
    if (lazy_[a] != 0) {
      key_[a] += lazy_[a];
      if (l_[a] >= 0) lazy_[l_[a]] += lazy_[a];
      if (r_[a] >= 0) lazy_[r_[a]] += lazy_[a];
      lazy_[a] = 0;
    }
  }
  std::vector<int64_t> key_, lazy_;
  std::vector<int32_t> l_, r_, rk_;
};

class RollbackDsu {
 public:
  explicit RollbackDsu(int64_t n) : p_(n, -1) {}
  int32_t find(int32_t x) const {
    while (p_[x] >= 0) x = p_[x];
    return x;
  }
  bool join(int32_t a, int32_t b) {
    a = find(a);
    b = find(b);
    if (a == b) return false;
    if (p_[a] > p_[b]) std::swap(a, b);  // a has the larger size (more negative)
    hist_.push_back({b, p_[b]});
    p_[a] += p_[b];
    p_[b] = a;
    return true;
  }
  size_t time() const { return hist_.size(); }
  void rollback(size_t t) {
    while (hist_.size() > t) {
      auto [b, old] = hist_.back();
      hist_.pop_back();
      int32_t a = p_[b];
      p_[b] = old;
      p_[a] -= old;
    }
  }

 private:
  std::vector<int32_t> p_;
  std::vector<std::pair<int32_t, int32_t>> hist_;
};

// Returns the chosen in-edge (candidate index) of every node 0..n_nodes-1
// except `root` (-1 there).  Throws if some node cannot be reached.
std::vector<int32_t> min_arborescence(const Arb& g, int32_t n_nodes, int32_t root, int64_t* total_cost) {
  const size_t m = g.from.size();
  LeftistPool heap(m);
  std::vector<int32_t> head(n_nodes, -1);
  for (size_t e = 0; e < m; ++e) {
    heap.init((int32_t)e, g.w[e]);
    head[g.to[e]] = heap.meld(head[g.to[e]], (int32_t)e);
  }
  RollbackDsu dsu(n_nodes);
  std::vector<int32_t> seen(n_nodes, -1);
  std::vector<int32_t> in(n_nodes, -1);
  seen[root] = root;
  struct Cycle {
    int32_t node;
    size_t time;
    std::vector<int32_t> edges;
  };
  std::vector<Cycle> cycles;  // in creation order
  std::vector<int32_t> path_node, path_edge;
  int64_t cost = 0;

  for (int32_t s = 0; s < n_nodes; ++s) {
    int32_t u = s;
    path_node.clear();
    path_edge.clear();
    while (seen[u] < 0) {
      int32_t e = -1;
      while (head[u] >= 0) {
        int32_t top = head[u];
        int64_t k = heap.top_key(top);
        head[u] = heap.pop(top);
        if (dsu.find(g.from[top]) == u) continue;  // edge inside a contracted node
        e = top;
        heap.add(head[u], -k);
        cost += k;
        break;
      }
      if (e < 0) throw std::runtime_error("arborescence: a node has no admissible in-edge");
      path_node.push_back(u);
      path_edge.push_back(e);
      seen[u] = s;
      u = dsu.find(g.from[e]);
      if (seen[u] == s) {
        // contract the cycle closed at u
        Cycle cyc;
        cyc.time = dsu.time();
        int32_t merged = -1;
        int32_t wnode;
        do {
          wnode = path_node.back();
          cyc.edges.push_back(path_edge.back());
          path_node.pop_back();
          path_edge.pop_back();
          merged = heap.meld(merged, head[wnode]);
          head[wnode] = -1;
        } while (dsu.join(u, wnode));
        u = dsu.find(u);
        head[u] = merged;
        seen[u] = -1;
        cyc.node = u;
        cycles.push_back(std::move(cyc));
      }
    }
    for (size_t i = 0; i < path_edge.size(); ++i) in[dsu.find(g.to[path_edge[i]])] = path_edge[i];
  }
  // expand cycles, newest first
  for (size_t ci = cycles.size(); ci-- > 0;) {
    Cycle& c = cycles[ci];
    dsu.rollback(c.time);
    const int32_t entering = in[c.node];
    for (int32_t e : c.edges) in[dsu.find(g.to[e])] = e;
    in[dsu.find(g.to[entering])] = entering;
  }
  if (total_cost) *total_cost = cost;
  in[root] = -1;
  return in;
}

}  // namespace

// ---------------------------------------------------------------------------
// 4. The structure object and the C-ABI
// ---------------------------------------------------------------------------
struct cbm_structure {
  std::vector<int32_t> delta_row, delta_col;
  std::vector<float> delta_val;
  std::vector<int32_t> branches, src, dst;
  // extras
  std::vector<int32_t> parent;  // parent per node, n for the virtual root
  std::vector<int32_t> csr_ptr, csr_col;  // delta matrix as CSR (row blocks in row order)
  std::vector<float> csr_val;
  int64_t n_candidates = 0;     // tree candidates (without the N virtual edges)
  int64_t tree_cost = 0;        // total weight of the chosen arborescence
  int64_t nnz_a = 0;            // nnz of the coalesced A
  bool symmetric = false;       // A == A^T
  std::string error;
};

namespace {

// A == A^T: every (i, j) has (j, i), found by binary search in row j's sorted
// columns (rows in parallel).
bool is_symmetric(const Csr& a) {
  bool sym = true;
#pragma omp parallel for reduction(&& : sym) schedule(dynamic, 4096)
  for (int64_t i = 0; i < a.n; ++i) {
    for (int64_t k = a.ptr[i]; k < a.ptr[i + 1] && sym; ++k) {
      const int32_t j = a.idx[k];
      const int32_t* b = a.idx.data() + a.ptr[j];
      const int32_t* e = a.idx.data() + a.ptr[j + 1];
      if (!std::binary_search(b, e, (int32_t)i)) sym = false;
    }
  }
  return sym;
}

// Entries of A[v] - A[u] (u = -1: A[v] as +1 entries) in increasing column
// order, written at out (when not null); returns their number.
int64_t delta_block(const Csr& a, int32_t u, int32_t v, int32_t* row, int32_t* col, float* val) {
  int64_t m = 0;
  auto put = [&](int32_t c, float s) {
    if (row) {
      row[m] = v;
      col[m] = c;
      val[m] = s;
    }
    ++m;
  };
  int64_t vp = a.ptr[v], ve = a.ptr[v + 1];
  if (u < 0) {
    for (; vp < ve; ++vp) put(a.idx[vp], 1.0f);
    return m;
  }
  int64_t up = a.ptr[u], ue = a.ptr[u + 1];
  while (up < ue && vp < ve) {
    const int32_t cu = a.idx[up], cv = a.idx[vp];
    if (cu == cv) {
      ++up;
      ++vp;
    } else if (cu > cv) {
      put(cv, 1.0f);
      ++vp;
    } else {
      put(cu, -1.0f);
      ++up;
    }
  }
  for (; up < ue; ++up) put(a.idx[up], -1.0f);
  for (; vp < ve; ++vp) put(a.idx[vp], 1.0f);
  return m;
}

// Delta entries and tree edges in the reference's order
// (cbm/cbm_extensions.cpp:220-294): first the root children's whole rows as
// +1 entries, then for each non-empty branch, in BFS order, every tree edge
// (u, v) and the entries of A[v] - A[u] by a sorted merge.  The block of each
// emitted row is sized first, then all blocks are written in parallel at
// their offsets, so the output equals the sequential emission.
void emit(cbm_structure& out, const Csr& a, const std::vector<std::vector<int32_t>>& children, int n_threads) {
  const int64_t n = a.n;
  const auto& roots = children[n];
  std::vector<int32_t> non_empty;
  for (int32_t v : roots)
    if (!children[v].empty()) non_empty.push_back(v);
  // blocks in output order: (u, v) with u = -1 for root children
  std::vector<int32_t> bu, bv;
  bu.reserve(n);
  bv.reserve(n);
  for (int32_t v : roots) {
    bu.push_back(-1);
    bv.push_back(v);
  }
  out.branches.assign(non_empty.size() + 1, 0);
  std::deque<int32_t> fifo;
  for (size_t b = 0; b < non_empty.size(); ++b) {
    fifo.push_back(non_empty[b]);
    while (!fifo.empty()) {
      const int32_t u = fifo.front();
      fifo.pop_front();
      for (int32_t v : children[u]) {
        fifo.push_back(v);
        out.src.push_back(u);
        out.dst.push_back(v);
        out.branches[b + 1]++;
        bu.push_back(u);
        bv.push_back(v);
      }
    }
  }
  std::partial_sum(out.branches.begin(), out.branches.end(), out.branches.begin());
  const int64_t nb = (int64_t)bu.size();
  std::vector<int64_t> off(nb + 1, 0);
  int nt = 1;
#ifdef _OPENMP
  nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#endif
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
  for (int64_t k = 0; k < nb; ++k) off[k + 1] = delta_block(a, bu[k], bv[k], nullptr, nullptr, nullptr);
  for (int64_t k = 0; k < nb; ++k) off[k + 1] += off[k];
  out.delta_row.resize(off[nb]);
  out.delta_col.resize(off[nb]);
  out.delta_val.resize(off[nb]);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
  for (int64_t k = 0; k < nb; ++k)
    delta_block(a, bu[k], bv[k], out.delta_row.data() + off[k], out.delta_col.data() + off[k],
                out.delta_val.data() + off[k]);
}

}  // namespace

extern "C" {

int cbm_build(const int32_t* row, const int32_t* col, int64_t nnz, int64_t n_rows, int64_t alpha,
              int32_t n_threads, int32_t flags, cbm_structure** out) {
  return cbm_build_clustered(row, col, nnz, n_rows, alpha, nullptr, n_threads, flags, out);
}

int cbm_build_clustered(const int32_t* row, const int32_t* col, int64_t nnz, int64_t n_rows, int64_t alpha,
                        const int32_t* cluster, int32_t n_threads, int32_t flags, cbm_structure** out) {
  nvtxRangePushA("cbm_build");
  struct Pop {
    ~Pop() { nvtxRangePop(); }
  } pop;
  if (!out) return CBM_ERR_INVALID;
  *out = nullptr;
  if (n_rows < 0 || nnz < 0 || n_rows >= INT32_MAX || (nnz > 0 && (!row || !col))) return CBM_ERR_INVALID;
  for (int64_t k = 0; k < nnz; ++k)
    if (row[k] < 0 || row[k] >= n_rows || col[k] < 0 || col[k] >= n_rows) return CBM_ERR_INDEX;
  cbm_structure* s = new (std::nothrow) cbm_structure();
  if (!s) return CBM_ERR_ALLOC;
  try {
    const int64_t n = n_rows;
    Csr a = coo_to_csr(row, col, nnz, n);
    s->nnz_a = (int64_t)a.idx.size();
    s->symmetric = is_symmetric(a);
    std::vector<Pair> pairs = (flags & CBM_BUILD_EXHAUSTIVE) ? candidate_pairs_exhaustive(a, alpha, n_threads)
                                                              : candidate_pairs(a, alpha, n_threads);
    // clustered: a row's parent may only be a row of its own cluster (the
    // per-cluster CBMs of the reference's LSH clustering, as one forest)
    if (cluster) {
      pairs.erase(std::remove_if(pairs.begin(), pairs.end(),
                                 [&](const Pair& p) { return cluster[p.lo] != cluster[p.hi]; }),
                  pairs.end());
    }
    // candidate list in the reference's order
    Arb g;
    g.from.reserve(n + 2 * pairs.size());
    g.to.reserve(n + 2 * pairs.size());
    g.w.reserve(n + 2 * pairs.size());
    size_t pi = 0;
    for (int64_t r = 0; r < n; ++r) {
      const int64_t nr = a.ptr[r + 1] - a.ptr[r];
      g.from.push_back((int32_t)n);
      g.to.push_back((int32_t)r);
      g.w.push_back(nr);
      for (; pi < pairs.size() && pairs[pi].lo == r; ++pi) {
        const int32_t c = pairs[pi].hi;
        const int64_t nc = a.ptr[c + 1] - a.ptr[c];
        const int64_t h = nr + nc - 2 * (int64_t)pairs[pi].o;
        if (h < nr - alpha && h != nr) {
          g.from.push_back(c);
          g.to.push_back((int32_t)r);
          g.w.push_back(h);
        }
        if (h < nc - alpha && h != nc) {
          g.from.push_back((int32_t)r);
          g.to.push_back(c);
          g.w.push_back(h);
        }
      }
    }
    s->n_candidates = (int64_t)g.from.size() - n;
    std::vector<int32_t> in = min_arborescence(g, (int32_t)(n + 1), (int32_t)n, &s->tree_cost);
    // children lists in increasing candidate index
    std::vector<int32_t> chosen;
    chosen.reserve(n);
    for (int64_t v = 0; v < n; ++v) chosen.push_back(in[v]);
    std::sort(chosen.begin(), chosen.end());
    std::vector<std::vector<int32_t>> children(n + 1);
    s->parent.assign(n, (int32_t)n);
    for (int32_t e : chosen) {
      children[g.from[e]].push_back(g.to[e]);
      s->parent[g.to[e]] = g.from[e];
    }
    emit(*s, a, children, n_threads);
    // Each node's delta entries are emitted as one block in increasing column
    // order, so the CSR form is a permutation of those blocks.
    // A block starts where the row id changes, so each row's first entry and
    // length are found in parallel, each row written by one k.
    const int64_t z = (int64_t)s->delta_row.size();
    const int32_t* dr = s->delta_row.data();
    int nt = 1;
#ifdef _OPENMP
    nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#endif
    s->csr_ptr.assign(n + 1, 0);
    std::vector<int64_t> first(n, -1);
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t k = 0; k < z; ++k)
      if (k == 0 || dr[k - 1] != dr[k]) first[dr[k]] = k;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t k = 0; k < z; ++k)
      if (k == z - 1 || dr[k + 1] != dr[k]) s->csr_ptr[dr[k] + 1] = (int32_t)(k + 1 - first[dr[k]]);
    for (int64_t i = 0; i < n; ++i) s->csr_ptr[i + 1] += s->csr_ptr[i];
    s->csr_col.resize(z);
    s->csr_val.resize(z);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 4096)
    for (int64_t i = 0; i < n; ++i) {
      const int64_t len = s->csr_ptr[i + 1] - s->csr_ptr[i];
      if (len == 0) continue;
      std::memcpy(&s->csr_col[s->csr_ptr[i]], &s->delta_col[first[i]], len * sizeof(int32_t));
      std::memcpy(&s->csr_val[s->csr_ptr[i]], &s->delta_val[first[i]], len * sizeof(float));
    }
  } catch (const std::bad_alloc&) {
    delete s;
    return CBM_ERR_ALLOC;
  } catch (const std::exception&) {
    delete s;
    return CBM_ERR_INTERNAL;
  }
  *out = s;
  return CBM_OK;
}

int cbm_coalesce(const int32_t* row, const int32_t* col, int64_t nnz, int64_t n, int32_t flags, int64_t* ptr,
                 int32_t* out_col, int64_t* out_nnz) {
  if (!ptr || !out_nnz || n < 0 || nnz < 0 || (nnz > 0 && (!row || !col || !out_col))) return CBM_ERR_INVALID;
  const bool sym = flags & CBM_COALESCE_SYMMETRIZE;
  const bool drop = flags & CBM_COALESCE_DROP_SELF;
  for (int64_t k = 0; k < nnz; ++k)
    if (row[k] < 0 || row[k] >= n || col[k] < 0 || col[k] >= n) return CBM_ERR_INDEX;
  try {
    std::vector<int64_t> cnt(n + 1, 0);
    for (int64_t k = 0; k < nnz; ++k) {
      if (drop && row[k] == col[k]) continue;
      cnt[row[k] + 1]++;
      if (sym && row[k] != col[k]) cnt[col[k] + 1]++;
    }
    for (int64_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
    std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
    for (int64_t k = 0; k < nnz; ++k) {
      if (drop && row[k] == col[k]) continue;
      out_col[fill[row[k]]++] = col[k];
      if (sym && row[k] != col[k]) out_col[fill[col[k]]++] = row[k];
    }
    std::vector<int64_t> len(n, 0);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < n; ++i) {
      int32_t* b = out_col + cnt[i];
      int32_t* e = out_col + cnt[i + 1];
      std::sort(b, e);
      len[i] = std::unique(b, e) - b;
    }
    // compact in place (rows move left only)
    ptr[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
      if (ptr[i] != cnt[i] && len[i] > 0) std::memmove(out_col + ptr[i], out_col + cnt[i], len[i] * sizeof(int32_t));
      ptr[i + 1] = ptr[i] + len[i];
    }
    *out_nnz = ptr[n];
  } catch (const std::bad_alloc&) {
    return CBM_ERR_ALLOC;
  }
  return CBM_OK;
}

int64_t cbm_structure_len(const cbm_structure* s, int32_t which) {
  if (!s) return -1;
  switch (which) {
    case CBM_S_DELTA_ROW: return (int64_t)s->delta_row.size();
    case CBM_S_DELTA_COL: return (int64_t)s->delta_col.size();
    case CBM_S_DELTA_VAL: return (int64_t)s->delta_val.size();
    case CBM_S_BRANCHES: return (int64_t)s->branches.size();
    case CBM_S_SRC: return (int64_t)s->src.size();
    case CBM_S_DST: return (int64_t)s->dst.size();
    case CBM_S_PARENT: return (int64_t)s->parent.size();
    case CBM_S_CSR_PTR: return (int64_t)s->csr_ptr.size();
    case CBM_S_CSR_COL: return (int64_t)s->csr_col.size();
    case CBM_S_CSR_VAL: return (int64_t)s->csr_val.size();
    case CBM_S_N_CANDIDATES: return s->n_candidates;
    case CBM_S_TREE_COST: return s->tree_cost;
    case CBM_S_NNZ_A: return s->nnz_a;
    case CBM_S_SYMMETRIC: return s->symmetric ? 1 : 0;
    default: return -1;
  }
}

int cbm_structure_copy(const cbm_structure* s, int32_t which, void* dst) {
  if (!s || !dst) return CBM_ERR_INVALID;
  auto cp = [&](const auto& v) {
    if (!v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    return CBM_OK;
  };
  switch (which) {
    case CBM_S_DELTA_ROW: return cp(s->delta_row);
    case CBM_S_DELTA_COL: return cp(s->delta_col);
    case CBM_S_DELTA_VAL: return cp(s->delta_val);
    case CBM_S_BRANCHES: return cp(s->branches);
    case CBM_S_SRC: return cp(s->src);
    case CBM_S_DST: return cp(s->dst);
    case CBM_S_PARENT: return cp(s->parent);
    case CBM_S_CSR_PTR: return cp(s->csr_ptr);
    case CBM_S_CSR_COL: return cp(s->csr_col);
    case CBM_S_CSR_VAL: return cp(s->csr_val);
    default: return CBM_ERR_INVALID;
  }
}

void cbm_structure_free(cbm_structure* s) { delete s; }

}  // extern "C"
