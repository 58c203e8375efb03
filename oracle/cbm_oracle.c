/*
 * CPU oracle for the CBM product path -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
 * file, and only as the checker or the timed CPU baseline; the product path
 * (libcbm_b200.so) never links or calls it.
 *
 * A plain-C restatement of the reference (cbm4scale/CBM-GPU):
 *   oracle_candidates     the distance-graph edge list G of cbm_init_, in its
 *                         order (cbm/cbm_extensions.cpp:123-151), computed by
 *                         brute force over all row pairs (small inputs only)
 *   oracle_arb_cost       optimum arborescence cost by the textbook
 *                         Chu-Liu/Edmonds contraction, O(V E), independent of
 *                         the product's Tarjan implementation
 *   oracle_emit           BFS emission of delta entries and tree edges from a
 *                         chosen in-edge per node (cbm/cbm_extensions.cpp:191-299)
 *   oracle_spmm_update    CSR SpMM then branch-serial Y[dst] += Y[src]
 *                         (cbm/cbm_extensions.cpp:351-444, cbm/cbm.cu:25-57)
 *   oracle_spmm_update_add
 *                         ... then Y += (1 + eps) X, the GIN form
 *                         (cbm/cbm_extensions.cpp:498-591)
 *   oracle_spmm_fused_update
 *                         ... with Y[dst] += Y[src] * m[dst] / m[src]; mode 0
 *                         evaluates it as the reference GPU kernel does
 *                         ((y*m_dst)/m_src then add, cbm/cbm.cu:88), mode 1 as
 *                         the CPU path does (fma with m_dst/m_src,
 *                         cbm/cbm_extensions.cpp:662-697)
 *   oracle_csr_spmm_f64   FP64 ground truth y = rs o (A (cs o x)), optionally
 *                         with A transposed
 *   oracle_spmm_be, oracle_spmm_t_be, oracle_update_only, oracle_axpy
 *                         the pieces of the reference's cbm_mkl_cpp products
 *                         (cbm/cbm_extensions.cpp:351-907) on MKL's four-array
 *                         CSR (begin/end row pointers): SpMM, transposed SpMM,
 *                         the branch-serial update alone, and its cblas_saxpy
 * The *_omp variants parallelise the SpMM over rows and the update over
 * branches with OpenMP (schedule(dynamic, 50) as the reference's CPU path).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- candidates ----------------------------------------------------------- */
static int64_t overlap_sorted(const int32_t* a, int64_t na, const int32_t* b, int64_t nb) {
  int64_t i = 0, j = 0, o = 0;
  while (i < na && j < nb) {
    if (a[i] == b[j]) {
      ++o;
      ++i;
      ++j;
    } else if (a[i] < b[j]) {
      ++i;
    } else {
      ++j;
    }
  }
  return o;
}

/* ptr/idx: CSR of A with sorted unique columns.  Writes up to cap edges;
 * returns the number of edges (virtual edges included), or -1 if cap is too
 * small. */
int64_t oracle_candidates(int64_t n, const int64_t* ptr, const int32_t* idx, int64_t alpha, int64_t cap,
                          int32_t* from, int32_t* to, int64_t* w) {
  int64_t m = 0;
#define PUSH(f, t, ww)          \
  do {                          \
    if (m >= cap) return -1;    \
    from[m] = (int32_t)(f);     \
    to[m] = (int32_t)(t);       \
    w[m] = (ww);                \
    ++m;                        \
  } while (0)
  for (int64_t row = 0; row < n; ++row) {
    const int64_t nr = ptr[row + 1] - ptr[row];
    PUSH(n, row, nr);
    for (int64_t col = row + 1; col < n; ++col) {
      const int64_t nc = ptr[col + 1] - ptr[col];
      const int64_t val = overlap_sorted(idx + ptr[row], nr, idx + ptr[col], nc);
      if (val == 0) continue; /* not stored in syrk(A) */
      const int64_t h = nr + nc - 2 * val;
      if ((h < (nr - alpha)) && (h != nr)) PUSH(col, row, h);
      if ((h < (nc - alpha)) && (h != nc)) PUSH(row, col, h);
    }
  }
#undef PUSH
  return m;
}

/* ---- optimum arborescence cost (Chu-Liu/Edmonds) ------------------------- */
int64_t oracle_arb_cost(int64_t n_nodes, int64_t root, int64_t m, const int32_t* from0, const int32_t* to0,
                        const int64_t* w0) {
  int32_t* from = malloc(sizeof(int32_t) * (m ? m : 1));
  int32_t* to = malloc(sizeof(int32_t) * (m ? m : 1));
  int64_t* w = malloc(sizeof(int64_t) * (m ? m : 1));
  int64_t* in_w = malloc(sizeof(int64_t) * n_nodes);
  int64_t* pre = malloc(sizeof(int64_t) * n_nodes);
  int64_t* id = malloc(sizeof(int64_t) * n_nodes);
  int64_t* vis = malloc(sizeof(int64_t) * n_nodes);
  memcpy(from, from0, sizeof(int32_t) * m);
  memcpy(to, to0, sizeof(int32_t) * m);
  memcpy(w, w0, sizeof(int64_t) * m);
  int64_t res = 0, n = n_nodes, r = root;
  for (;;) {
    for (int64_t v = 0; v < n; ++v) in_w[v] = INT64_MAX;
    for (int64_t e = 0; e < m; ++e)
      if (from[e] != to[e] && w[e] < in_w[to[e]]) {
        in_w[to[e]] = w[e];
        pre[to[e]] = from[e];
      }
    for (int64_t v = 0; v < n; ++v)
      if (v != r && in_w[v] == INT64_MAX) {
        res = -1;
        goto done;
      }
    int64_t cnt = 0;
    for (int64_t v = 0; v < n; ++v) {
      id[v] = -1;
      vis[v] = -1;
    }
    in_w[r] = 0;
    for (int64_t v = 0; v < n; ++v) {
      res += in_w[v];
      int64_t u = v;
      while (vis[u] != v && id[u] == -1 && u != r) {
        vis[u] = v;
        u = pre[u];
      }
      if (u != r && id[u] == -1) {
        for (int64_t x = pre[u]; x != u; x = pre[x]) id[x] = cnt;
        id[u] = cnt++;
      }
    }
    if (cnt == 0) break;
    for (int64_t v = 0; v < n; ++v)
      if (id[v] == -1) id[v] = cnt++;
    for (int64_t e = 0; e < m; ++e) {
      const int64_t v = to[e];
      from[e] = (int32_t)id[from[e]];
      to[e] = (int32_t)id[to[e]];
      if (from[e] != to[e]) w[e] -= in_w[v];
    }
    n = cnt;
    r = id[r];
  }
done:
  free(from);
  free(to);
  free(w);
  free(in_w);
  free(pre);
  free(id);
  free(vis);
  return res;
}

/* ---- BFS emission --------------------------------------------------------------- */
/* in_edge[v]: index (into the candidate list from/to) of v's tree in-edge.
 * Children are visited in increasing in-edge index.  Output arrays must hold
 * nnz(A) * 2 entries (delta) and n (edges) / n + 1 (branches).  Writes the
 * counts to counts[0..2] = {Z, E, B + 1}. */
static const int32_t* g_sort_key;
static int cmp_by_key(const void* a, const void* b) {
  const int32_t x = g_sort_key[*(const int32_t*)a], y = g_sort_key[*(const int32_t*)b];
  return (x > y) - (x < y);
}

int oracle_emit(int64_t n, const int64_t* ptr, const int32_t* idx, const int32_t* from, const int32_t* in_edge,
                int32_t* d_row, int32_t* d_col, float* d_val, int32_t* branches, int32_t* src, int32_t* dst,
                int64_t* counts) {
  /* children lists of every node including the virtual root n */
  int64_t* cptr = calloc(n + 2, sizeof(int64_t));
  int32_t* kids = malloc(sizeof(int32_t) * (n ? n : 1));
  int32_t* par = malloc(sizeof(int32_t) * (n ? n : 1));
  for (int64_t v = 0; v < n; ++v) {
    par[v] = from[in_edge[v]];
    cptr[par[v] + 1]++;
  }
  for (int64_t u = 0; u <= n; ++u) cptr[u + 1] += cptr[u];
  int64_t* fill = malloc(sizeof(int64_t) * (n + 1));
  memcpy(fill, cptr, sizeof(int64_t) * (n + 1));
  for (int64_t v = 0; v < n; ++v) kids[fill[par[v]]++] = (int32_t)v;
  g_sort_key = in_edge;
  for (int64_t u = 0; u <= n; ++u) qsort(kids + cptr[u], cptr[u + 1] - cptr[u], sizeof(int32_t), cmp_by_key);
  int64_t z = 0, e = 0, b = 0;
  /* root children emit their rows */
  for (int64_t k = cptr[n]; k < cptr[n + 1]; ++k) {
    const int32_t v = kids[k];
    for (int64_t q = ptr[v]; q < ptr[v + 1]; ++q) {
      d_row[z] = v;
      d_col[z] = idx[q];
      d_val[z] = 1.0f;
      ++z;
    }
  }
  int32_t* fifo = malloc(sizeof(int32_t) * (n ? n : 1));
  branches[0] = 0;
  for (int64_t k = cptr[n]; k < cptr[n + 1]; ++k) {
    const int32_t r = kids[k];
    if (cptr[r + 1] == cptr[r]) continue; /* empty branch */
    int64_t head = 0, tail = 0;
    fifo[tail++] = r;
    int64_t edges_here = 0;
    while (head < tail) {
      const int32_t u = fifo[head++];
      for (int64_t c = cptr[u]; c < cptr[u + 1]; ++c) {
        const int32_t v = kids[c];
        fifo[tail++] = v;
        src[e] = u;
        dst[e] = v;
        ++e;
        ++edges_here;
        int64_t up = ptr[u], ue = ptr[u + 1], vp = ptr[v], ve = ptr[v + 1];
        while (up < ue && vp < ve) {
          if (idx[up] == idx[vp]) {
            ++up;
            ++vp;
          } else if (idx[up] > idx[vp]) {
            d_row[z] = v; d_col[z] = idx[vp]; d_val[z] = 1.0f; ++z; ++vp;
          } else {
            d_row[z] = v; d_col[z] = idx[up]; d_val[z] = -1.0f; ++z; ++up;
          }
        }
        for (; up < ue; ++up) { d_row[z] = v; d_col[z] = idx[up]; d_val[z] = -1.0f; ++z; }
        for (; vp < ve; ++vp) { d_row[z] = v; d_col[z] = idx[vp]; d_val[z] = 1.0f; ++z; }
      }
    }
    branches[b + 1] = branches[b] + (int32_t)edges_here;
    ++b;
  }
  counts[0] = z;
  counts[1] = e;
  counts[2] = b + 1;
  free(cptr);
  free(kids);
  free(par);
  free(fill);
  free(fifo);
  return 0;
}

/* ---- products (fp32, the reference's arithmetic) -------------------------- */
/* y[n_rows, c] = A x with A in CSR (row_ptr int32 as the reference passes it) */
static void csr_spmm_f32(int64_t n_rows, int64_t c, const int32_t* rp, const int32_t* ci, const float* val,
                         const float* x, float* y, int parallel) {
  (void)parallel;
#pragma omp parallel for schedule(dynamic, 64) if (parallel)
  for (int64_t i = 0; i < n_rows; ++i) {
    float* yr = y + i * c;
    for (int64_t q = 0; q < c; ++q) yr[q] = 0.0f;
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      const float a = val[k];
      const float* xr = x + (int64_t)ci[k] * c;
      for (int64_t q = 0; q < c; ++q) yr[q] = fmaf(a, xr[q], yr[q]);
    }
  }
}

/* mode: 0 plain update; 1 ratio as the GPU kernel (cbm/cbm.cu:88);
 *       2 ratio as the CPU path (cbm/cbm_extensions.cpp:662-697) */
static void update(int64_t c, int64_t n_branches, const int32_t* br, const int32_t* src, const int32_t* dst,
                   const float* m, int mode, float* y, int parallel) {
  (void)parallel;
#pragma omp parallel for schedule(dynamic, 50) if (parallel)
  for (int64_t b = 0; b < n_branches; ++b) {
    for (int64_t e = br[b]; e < br[b + 1]; ++e) {
      const float* s = y + (int64_t)src[e] * c;
      float* d = y + (int64_t)dst[e] * c;
      if (mode == 0) {
        for (int64_t q = 0; q < c; ++q) d[q] = d[q] + s[q];
      } else if (mode == 1) {
        const float md = m[dst[e]], ms = m[src[e]];
        for (int64_t q = 0; q < c; ++q) {
          volatile float t = s[q] * md; /* no contraction */
          t = t / ms;
          d[q] = d[q] + t;
        }
      } else {
        const float r = m[dst[e]] / m[src[e]];
        for (int64_t q = 0; q < c; ++q) d[q] = fmaf(s[q], r, d[q]);
      }
    }
  }
}

void oracle_spmm_update(int64_t n_rows, int64_t c, const int32_t* rp, const int32_t* ci, const float* val,
                        const float* x, int64_t n_branches, const int32_t* br, const int32_t* src,
                        const int32_t* dst, float* y) {
  csr_spmm_f32(n_rows, c, rp, ci, val, x, y, 0);
  update(c, n_branches, br, src, dst, NULL, 0, y, 0);
}

/* s_spmm_update_add_csr_int32 (cbm/cbm_extensions.cpp:498-591): the CBM
 * product, then y += (1 + eps) x over all elements (its cblas_saxpy), taken
 * here as one fused multiply-add per element. */
void oracle_spmm_update_add(int64_t n_rows, int64_t c, const int32_t* rp, const int32_t* ci, const float* val,
                            const float* x, float eps, int64_t n_branches, const int32_t* br, const int32_t* src,
                            const int32_t* dst, float* y) {
  csr_spmm_f32(n_rows, c, rp, ci, val, x, y, 0);
  update(c, n_branches, br, src, dst, NULL, 0, y, 0);
  const float a = 1.0f + eps;
  for (int64_t i = 0; i < n_rows * c; ++i) y[i] = fmaf(a, x[i], y[i]);
}

void oracle_spmm_fused_update(int64_t n_rows, int64_t c, const int32_t* rp, const int32_t* ci, const float* val,
                              const float* x, int64_t n_branches, const int32_t* br, const int32_t* src,
                              const int32_t* dst, const float* m, int mode, float* y) {
  csr_spmm_f32(n_rows, c, rp, ci, val, x, y, 0);
  update(c, n_branches, br, src, dst, m, mode == 0 ? 1 : 2, y, 0);
}

/* OpenMP versions: the CPU baseline (all host threads) */
void oracle_spmm_update_omp(int64_t n_rows, int64_t c, const int32_t* rp, const int32_t* ci, const float* val,
                            const float* x, int64_t n_branches, const int32_t* br, const int32_t* src,
                            const int32_t* dst, float* y) {
  csr_spmm_f32(n_rows, c, rp, ci, val, x, y, 1);
  update(c, n_branches, br, src, dst, NULL, 0, y, 1);
}

void oracle_spmm_fused_update_omp(int64_t n_rows, int64_t c, const int32_t* rp, const int32_t* ci,
                                  const float* val, const float* x, int64_t n_branches, const int32_t* br,
                                  const int32_t* src, const int32_t* dst, const float* m, float* y) {
  csr_spmm_f32(n_rows, c, rp, ci, val, x, y, 1);
  update(c, n_branches, br, src, dst, m, 2, y, 1);
}

/* ---- the cbm_mkl_cpp products' pieces (cbm/cbm_extensions.cpp:351-907) ---- */
/* y[n_rows, c] = A x, row i's entries [rp_b[i], rp_e[i]) (MKL's four-array
 * CSR, mkl_sparse_s_create_csr at :365-372), one FMA per entry in order */
void oracle_spmm_be(int64_t n_rows, int64_t c, const int32_t* rp_b, const int32_t* rp_e, const int32_t* ci,
                    const float* val, const float* x, float* y) {
  for (int64_t i = 0; i < n_rows; ++i) {
    float* yr = y + i * c;
    for (int64_t q = 0; q < c; ++q) yr[q] = 0.0f;
    for (int64_t k = rp_b[i]; k < rp_e[i]; ++k) {
      const float a = val[k];
      const float* xr = x + (int64_t)ci[k] * c;
      for (int64_t q = 0; q < c; ++q) yr[q] = fmaf(a, xr[q], yr[q]);
    }
  }
}

/* y[n_cols, c] = A^T x (SPARSE_OPERATION_TRANSPOSE, :742-782): rows of A in
 * order, each entry's term added with one FMA */
void oracle_spmm_t_be(int64_t n_rows, int64_t n_cols, int64_t c, const int32_t* rp_b, const int32_t* rp_e,
                      const int32_t* ci, const float* val, const float* x, float* y) {
  memset(y, 0, sizeof(float) * n_cols * c);
  for (int64_t i = 0; i < n_rows; ++i) {
    const float* xr = x + i * c;
    for (int64_t k = rp_b[i]; k < rp_e[i]; ++k) {
      const float a = val[k];
      float* yr = y + (int64_t)ci[k] * c;
      for (int64_t q = 0; q < c; ++q) yr[q] = fmaf(a, xr[q], yr[q]);
    }
  }
}

/* the update alone, in place (:784-907): mode 0 plain, 2 the CPU fused rule */
void oracle_update_only(int64_t c, int64_t n_branches, const int32_t* br, const int32_t* src, const int32_t* dst,
                        const float* m, int mode, float* y) {
  update(c, n_branches, br, src, dst, m, mode, y, 0);
}

/* y = (a x) + y element-wise with one FMA each: the cblas_saxpy of :490, :590 */
void oracle_axpy(int64_t n, float a, const float* x, float* y) {
  for (int64_t i = 0; i < n; ++i) y[i] = fmaf(a, x[i], y[i]);
}

int oracle_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ---- FP64 ground truth ------------------------------------------------------------ */
/* y = rs o (A (cs o x)) or, transposed, y = rs o (A^T (cs o x)); rs/cs may be
 * NULL.  A: CSR (int64 row_ptr) of the binary pattern (values 1). */
void oracle_csr_spmm_f64(int64_t n_rows, int64_t n_cols, const int64_t* ptr, const int32_t* idx, int64_t c,
                         const double* x, const double* rs, const double* cs, int transpose, double* y) {
  const int64_t out_rows = transpose ? n_cols : n_rows;
  memset(y, 0, sizeof(double) * out_rows * c);
  for (int64_t i = 0; i < n_rows; ++i) {
    for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k) {
      const int64_t j = idx[k];
      const int64_t in_row = transpose ? i : j;
      const int64_t out_row = transpose ? j : i;
      const double s = cs ? cs[in_row] : 1.0;
      const double* xr = x + in_row * c;
      double* yr = y + out_row * c;
      for (int64_t q = 0; q < c; ++q) yr[q] += s * xr[q];
    }
  }
  if (rs)
    for (int64_t i = 0; i < out_rows; ++i)
      for (int64_t q = 0; q < c; ++q) y[i * c + q] *= rs[i];
}
