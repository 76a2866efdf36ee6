/*
 * sssp_oracle.c -- CPU restatement of dynG's batch-dynamic SSSP path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path of dyng_b200 is compared
 * against (tests/, __graft_entry__.smoke() and the cpu_baseline / --impl reference legs of
 * bench.py).  Nothing in the product links or calls it.
 *
 * It restates, in plain C, the algorithm of the reference's host path (file:line within the dynG
 * project):
 *   - graph construction       cpp/src/graph/apply_host.cpp:527-660  (build_rows, from_edges)
 *   - batch application        cpp/src/graph/apply_host.cpp:57-395   (apply_batch_host: Step 0,
 *                              grouping by row, first-alive-match deletes, upsert/append inserts,
 *                              CSR assembly, weight-increase classification)
 *   - transposition            cpp/src/graph/apply_host.cpp:470-518  (transpose_host)
 *   - change lists             cpp/src/algorithms/sssp/sssp.cpp:563-576 (build_changes)
 *   - Step 0 summary           cpp/src/algorithms/sssp/sssp.cpp:643-689 (prepare), :136-165
 *                              (sssp_default_delta, sssp_distances_fit, sssp_packs_parents)
 *   - the sequential engine    cpp/src/algorithms/sssp/sequential.cpp:57-381 (identify_affected
 *                              with children lists, seed/relax pull pass, round-by-round push
 *                              loop with the lexicographic (distance, parent) order, recover_parents,
 *                              count_affected, the rootless-cycle check)
 *   - CUDA packing rule        cpp/src/algorithms/sssp/kernels.cuh:80-92, cuda.cu:225-234
 *                              (make_packing / choose_packing; selected with rule = 1)
 *   - canonicalize / validate  cpp/src/algorithms/sssp/sssp.cpp:377-460 (canonicalize_tree,
 *                              validate_tree_sequential), :571-599 (normalize_imported_tree)
 *   - mosp's finalize step     cpp/src/algorithms/mosp/sequential.cpp:33-170 (combined_edge and
 *                              the combined graph), :172-232 (mospPathCosts), mosp.cpp:259-301
 *                              (preference terms and base weight); the combined graph is solved
 *                              with the compute above
 *
 * Parity of this restatement is pinned by tests/test_oracle.py against the reference's own golden
 * fixtures (cpp/tests/data/mosp_sssp: 34 cases, cpp/tests/data/mosp_graph_io: applied and
 * transposed CSR plus weight-increase masks, cpp/tests/data/mosp_combined: 9 combined-graph
 * cases), converted by tests/golden/make_golden.py.
 *
 * Threads: orc_set_threads(T > 1) runs the CSR assembly and the transposition of every apply
 * on T OpenMP threads (the reference's host path parallelises the same loops, apply_host.cpp:
 * 264-306, 417-468), and the repair of an update whose tree packs (distance, parent) into one
 * word on the threaded engine (openmp.cpp:223-583: invalidation by level, a pull seed, push
 * rounds with a compare-and-swap minimum).  Trees, invalidated and affected counts are
 * identical for every T; the schedule-dependent counters (pushes) are not.  The checker runs
 * with one thread; the CPU-baseline timings use the host's cores.
 *
 * Errors are returned as negative status codes with a message in the caller's buffer; nothing
 * aborts.  All memory is owned by the orc_graph handle or by the caller.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#else
static int omp_get_thread_num(void) { return 0; }
#endif

#define ORC_INF ((int64_t)(INT64_MAX / 4)) /* sssp_infinity, problem.hpp:340-341 */

/* Threads of the parallel loops (the reference's OpenMP host path parallelises the CSR assembly
 * and the transposition the same way, apply_host.cpp:264-306, 417-468).  1 (the default): every
 * loop runs sequentially, as the checker does; results are identical for every thread count. */
static int g_threads = 1;
void orc_set_threads(int threads) { g_threads = threads > 1 ? threads : 1; }
int orc_get_threads(void) { return g_threads; }

enum {
  ORC_OK = 0,
  ORC_INVALID_ARGUMENT = -1,
  ORC_OUT_OF_MEMORY = -2,
  ORC_NOT_CONVERGED = -3,
};

typedef struct {
  int directed;            /* graph_properties::directed */
  int sorted;              /* row_order::sorted (1) or append (0) */
  int allow_multi;         /* multi_edges::allow (1) or forbid (0) */
  int on_existing_insert;  /* 0 upsert, 1 error, 2 ignore */
  int on_missing_delete;   /* 0 ignore, 1 error */
  int on_self_loop;        /* 0 keep, 1 drop, 2 error */
  int deletions_first;     /* 1: deletions, then insertions */
  int allow_vertex_growth; /* 1: insertions may name new vertices */
} orc_props;

typedef struct {
  int64_t inserted_edges, deleted_edges, updated_edges, ignored_insertions, ignored_deletions,
      dropped_self_loops, inserted_vertices, num_vertices_after;
} orc_summary;

typedef struct {
  int64_t invalidated, affected, iterations, epochs, pushes;
  int64_t packed_parents, delta, max_weight;
} orc_stats;

typedef struct {
  int64_t n, m;
  int k;
  orc_props props;
  int64_t* row_ptr; /* n + 1 */
  int32_t* col;     /* m */
  int32_t* w;       /* k * m, objective-major */
  /* in-edges (transpose), rebuilt after every apply */
  int64_t* in_row_ptr;
  int32_t* in_col;
  int32_t* in_w;
  /* apply_delta of the last apply (graph_impl.hpp:73-87) */
  int64_t num_ins, num_del;
  int32_t *ins_src, *ins_dst, *del_src, *del_dst;
  uint8_t* weight_increased; /* num_ins * k */
} orc_graph;

static void set_err(char* err, size_t cap, const char* msg) {
  if (err && cap) {
    snprintf(err, cap, "%s", msg);
  }
}

static void* xmalloc(size_t bytes) {
  return malloc(bytes ? bytes : 1);
}

/* ---------------------------------------------------------------------------------------------
 * transpose (apply_host.cpp:470-518): inside an in-row the sources appear in out-edge order.
 * ------------------------------------------------------------------------------------------- */
static int transpose(orc_graph* g) {
  free(g->in_row_ptr);
  free(g->in_col);
  free(g->in_w);
  const int64_t n = g->n, m = g->m;
  g->in_row_ptr = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  g->in_col = (int32_t*)xmalloc((size_t)m * sizeof(int32_t));
  g->in_w = (int32_t*)xmalloc((size_t)m * (size_t)g->k * sizeof(int32_t));
  int64_t* cursor = (int64_t*)xmalloc((size_t)(n + 1) * sizeof(int64_t));
  int64_t* position = (int64_t*)xmalloc((size_t)m * sizeof(int64_t));
  if (!g->in_row_ptr || !g->in_col || !g->in_w || !cursor || !position) {
    free(cursor);
    free(position);
    return ORC_OUT_OF_MEMORY;
  }
  if (g_threads > 1) {
    /* A counting sort per thread: thread t owns the out-rows [u_t, u_t+1) (contiguous slots in
     * ascending order), counts its in-degrees privately, then writes each of its slots at
     * in_row_ptr[v] + (slots of v from threads before t) + (its own earlier slots of v): the
     * in-row order is the out-edge order, as in the sequential loop, with no atomics and no
     * sort (the reference sorts each in-row after an atomic scatter, apply_host.cpp:417-468). */
    const int T = g_threads;
    int64_t* ubound = (int64_t*)xmalloc((size_t)(T + 1) * sizeof(int64_t));
    int32_t* cnt = (int32_t*)calloc((size_t)T * (size_t)(n > 0 ? n : 1), sizeof(int32_t));
    ubound[0] = 0;
    for (int t = 1; t < T; ++t) {  /* split the slots evenly, on row boundaries */
      const int64_t target = m * t / T;
      int64_t lo = ubound[t - 1], hi = n;
      while (lo < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (g->row_ptr[mid] < target) lo = mid + 1;
        else hi = mid;
      }
      ubound[t] = lo;
    }
    ubound[T] = n;
#pragma omp parallel num_threads(T)
    {
      const int t = omp_get_thread_num();
      int32_t* c = cnt + (size_t)t * (size_t)n;
      for (int64_t e = g->row_ptr[ubound[t]]; e < g->row_ptr[ubound[t + 1]]; ++e) c[g->col[e]]++;
#pragma omp barrier
#pragma omp for schedule(static)
      for (int64_t v = 0; v < n; ++v) {  /* per vertex: threads' counts become offsets */
        int64_t sum = 0;
        for (int q = 0; q < T; ++q) {
          const int32_t x = cnt[(size_t)q * (size_t)n + (size_t)v];
          cnt[(size_t)q * (size_t)n + (size_t)v] = (int32_t)sum;
          sum += x;
        }
        g->in_row_ptr[v + 1] = sum;
      }
#pragma omp single
      for (int64_t v = 0; v < n; ++v) g->in_row_ptr[v + 1] += g->in_row_ptr[v];
      /* implicit barrier after single */
      for (int64_t u = ubound[t]; u < ubound[t + 1]; ++u) {
        for (int64_t e = g->row_ptr[u]; e < g->row_ptr[u + 1]; ++e) {
          const int32_t v = g->col[e];
          const int64_t pos = g->in_row_ptr[v] + c[v]++;
          position[e] = pos;
          g->in_col[pos] = (int32_t)u;
        }
      }
    }
    free(ubound);
    free(cnt);
  } else {
    for (int64_t e = 0; e < m; ++e) g->in_row_ptr[g->col[e] + 1]++;
    for (int64_t v = 0; v < n; ++v) g->in_row_ptr[v + 1] += g->in_row_ptr[v];
    memcpy(cursor, g->in_row_ptr, (size_t)n * sizeof(int64_t));
    for (int64_t u = 0; u < n; ++u) {
      for (int64_t e = g->row_ptr[u]; e < g->row_ptr[u + 1]; ++e) {
        const int64_t pos = cursor[g->col[e]]++;
        position[e] = pos;
        g->in_col[pos] = (int32_t)u;
      }
    }
  }
  for (int k = 0; k < g->k; ++k) {
    const int32_t* in = g->w + (size_t)k * (size_t)m;
    int32_t* out = g->in_w + (size_t)k * (size_t)m;
#pragma omp parallel for num_threads(g_threads) if (g_threads > 1) schedule(static)
    for (int64_t e = 0; e < m; ++e) out[position[e]] = in[e];
  }
  free(cursor);
  free(position);
  return ORC_OK;
}

static void free_delta(orc_graph* g) {
  free(g->ins_src);
  free(g->ins_dst);
  free(g->del_src);
  free(g->del_dst);
  free(g->weight_increased);
  g->ins_src = g->ins_dst = g->del_src = g->del_dst = NULL;
  g->weight_increased = NULL;
  g->num_ins = g->num_del = 0;
}

void orc_graph_free(orc_graph* g) {
  if (!g) return;
  free(g->row_ptr);
  free(g->col);
  free(g->w);
  free(g->in_row_ptr);
  free(g->in_col);
  free(g->in_w);
  free_delta(g);
  free(g);
}

/* ---------------------------------------------------------------------------------------------
 * construction (apply_host.cpp:527-660): counting sort by source keeping input order; under
 * forbid, a stable sort by destination merges repeats (first position kept, last weights win),
 * then append order restores the first positions; under allow + sorted, a stable sort.
 * ------------------------------------------------------------------------------------------- */
typedef struct {
  int32_t vertex;
  int64_t first; /* position of the first occurrence in row order */
  int64_t last;  /* item whose weights are used */
} row_item;

static int cmp_item_vertex(const void* a, const void* b) {
  const row_item* x = (const row_item*)a;
  const row_item* y = (const row_item*)b;
  if (x->vertex != y->vertex) return x->vertex < y->vertex ? -1 : 1;
  /* stability: ties keep their order of first appearance */
  return x->first < y->first ? -1 : (x->first > y->first);
}
static int cmp_item_first(const void* a, const void* b) {
  const row_item* x = (const row_item*)a;
  const row_item* y = (const row_item*)b;
  return x->first < y->first ? -1 : (x->first > y->first);
}

/* edges: src[i], dst[i], weights of item idx[i] at w[idx[i] * k + j] (insertion-major). */
static int build_rows(orc_graph* g, int64_t count, const int32_t* src, const int32_t* dst,
                      const int64_t* idx, const int32_t* w_items) {
  const int64_t n = g->n;
  const int k = g->k;
  int64_t* start = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  int64_t* order = (int64_t*)xmalloc((size_t)count * sizeof(int64_t));
  row_item* kept = (row_item*)xmalloc((size_t)count * sizeof(row_item));
  int64_t* cursor = (int64_t*)xmalloc((size_t)(n + 1) * sizeof(int64_t));
  if (!start || !order || !kept || !cursor) {
    free(start); free(order); free(kept); free(cursor);
    return ORC_OUT_OF_MEMORY;
  }
  for (int64_t i = 0; i < count; ++i) start[src[i] + 1]++;
  for (int64_t u = 0; u < n; ++u) start[u + 1] += start[u];
  memcpy(cursor, start, (size_t)n * sizeof(int64_t));
  for (int64_t i = 0; i < count; ++i) order[cursor[src[i]]++] = i;
  free(g->row_ptr);
  g->row_ptr = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  int64_t total = 0;
  for (int64_t u = 0; u < n; ++u) {
    row_item* row = kept + total;
    int64_t len = 0;
    for (int64_t j = start[u]; j < start[u + 1]; ++j) {
      row[len].vertex = dst[order[j]];
      row[len].first = j;
      row[len].last = order[j];
      ++len;
    }
    if (!g->props.allow_multi) {
      qsort(row, (size_t)len, sizeof(row_item), cmp_item_vertex);
      int64_t wpos = 0;
      for (int64_t r = 0; r < len; ++r) {
        if (wpos > 0 && row[wpos - 1].vertex == row[r].vertex) {
          row[wpos - 1].last = row[r].last;
        } else {
          row[wpos++] = row[r];
        }
      }
      len = wpos;
      if (!g->props.sorted) qsort(row, (size_t)len, sizeof(row_item), cmp_item_first);
    } else if (g->props.sorted) {
      qsort(row, (size_t)len, sizeof(row_item), cmp_item_vertex);
    }
    total += len;
    g->row_ptr[u + 1] = total;
  }
  g->m = total;
  free(g->col);
  free(g->w);
  g->col = (int32_t*)xmalloc((size_t)total * sizeof(int32_t));
  g->w = (int32_t*)xmalloc((size_t)total * (size_t)k * sizeof(int32_t));
  for (int64_t e = 0; e < total; ++e) {
    g->col[e] = kept[e].vertex;
    for (int j = 0; j < k; ++j) {
      g->w[(size_t)j * (size_t)total + (size_t)e] = w_items[idx[kept[e].last] * k + j];
    }
  }
  free(start); free(order); free(kept); free(cursor);
  return transpose(g);
}

orc_graph* orc_graph_from_edges(int64_t n, int64_t count, const int32_t* src, const int32_t* dst,
                                const int32_t* weights, int k, const orc_props* props, char* err,
                                size_t err_cap) {
  orc_graph* g = (orc_graph*)calloc(1, sizeof(orc_graph));
  if (!g) return NULL;
  g->n = n;
  g->k = k;
  g->props = *props;
  int32_t* s = (int32_t*)xmalloc((size_t)(2 * count) * sizeof(int32_t));
  int32_t* d = (int32_t*)xmalloc((size_t)(2 * count) * sizeof(int32_t));
  int64_t* idx = (int64_t*)xmalloc((size_t)(2 * count) * sizeof(int64_t));
  int64_t c = 0;
  for (int64_t i = 0; i < count; ++i) {
    const int32_t u = src[i], v = dst[i];
    if (u < 0 || u >= n || v < 0 || v >= n) {
      set_err(err, err_cap, "edge out of range");
      goto fail;
    }
    if (u == v && props->on_self_loop != 0) {
      if (props->on_self_loop == 2) {
        set_err(err, err_cap, "self-loop under self_loop::error");
        goto fail;
      }
      continue;
    }
    s[c] = u; d[c] = v; idx[c] = i; ++c;
    if (!props->directed && u != v) {
      s[c] = v; d[c] = u; idx[c] = i; ++c;
    }
  }
  if (build_rows(g, c, s, d, idx, weights) != ORC_OK) {
    set_err(err, err_cap, "out of memory");
    goto fail;
  }
  free(s); free(d); free(idx);
  return g;
fail:
  free(s); free(d); free(idx);
  orc_graph_free(g);
  return NULL;
}

/* from_csr: validated, then normalised as from_edges (a CSR is an edge list in row order). */
orc_graph* orc_graph_from_csr(int64_t n, const int64_t* row_ptr, const int32_t* col,
                              const int32_t* w_objective_major, int k, const orc_props* props,
                              char* err, size_t err_cap) {
  if (row_ptr[0] != 0) {
    set_err(err, err_cap, "row_ptr[0] != 0");
    return NULL;
  }
  for (int64_t u = 0; u < n; ++u) {
    if (row_ptr[u + 1] < row_ptr[u]) {
      set_err(err, err_cap, "row_ptr not monotone");
      return NULL;
    }
  }
  const int64_t m = row_ptr[n];
  int32_t* src = (int32_t*)xmalloc((size_t)m * sizeof(int32_t));
  int32_t* items = (int32_t*)xmalloc((size_t)m * (size_t)k * sizeof(int32_t));
  for (int64_t u = 0; u < n; ++u)
    for (int64_t e = row_ptr[u]; e < row_ptr[u + 1]; ++e) src[e] = (int32_t)u;
  for (int64_t e = 0; e < m; ++e)
    for (int j = 0; j < k; ++j) items[e * k + j] = w_objective_major[(size_t)j * (size_t)m + e];
  orc_graph* g = orc_graph_from_edges(n, m, src, col, items, k, props, err, err_cap);
  free(src);
  free(items);
  return g;
}

int64_t orc_graph_num_vertices(const orc_graph* g) { return g->n; }
int64_t orc_graph_num_edges(const orc_graph* g) { return g->m; }

/* Copy out the CSR (row_ptr n+1, col m, weights k*m objective-major) and the transpose. */
void orc_graph_export(const orc_graph* g, int64_t* row_ptr, int32_t* col, int32_t* w,
                      int64_t* in_row_ptr, int32_t* in_col, int32_t* in_w) {
  if (row_ptr) memcpy(row_ptr, g->row_ptr, (size_t)(g->n + 1) * sizeof(int64_t));
  if (col) memcpy(col, g->col, (size_t)g->m * sizeof(int32_t));
  if (w) memcpy(w, g->w, (size_t)g->m * (size_t)g->k * sizeof(int32_t));
  if (in_row_ptr) memcpy(in_row_ptr, g->in_row_ptr, (size_t)(g->n + 1) * sizeof(int64_t));
  if (in_col) memcpy(in_col, g->in_col, (size_t)g->m * sizeof(int32_t));
  if (in_w) memcpy(in_w, g->in_w, (size_t)g->m * (size_t)g->k * sizeof(int32_t));
}

int64_t orc_graph_num_changes(const orc_graph* g, int64_t* num_del) {
  if (num_del) *num_del = g->num_del;
  return g->num_ins;
}

/* The apply_delta of the last apply: effective insertions, deletions and the increase mask. */
void orc_graph_delta(const orc_graph* g, int32_t* ins_src, int32_t* ins_dst, int32_t* del_src,
                     int32_t* del_dst, uint8_t* weight_increased) {
  if (ins_src) memcpy(ins_src, g->ins_src, (size_t)g->num_ins * sizeof(int32_t));
  if (ins_dst) memcpy(ins_dst, g->ins_dst, (size_t)g->num_ins * sizeof(int32_t));
  if (del_src) memcpy(del_src, g->del_src, (size_t)g->num_del * sizeof(int32_t));
  if (del_dst) memcpy(del_dst, g->del_dst, (size_t)g->num_del * sizeof(int32_t));
  if (weight_increased)
    memcpy(weight_increased, g->weight_increased, (size_t)g->num_ins * (size_t)g->k);
}

/* ---------------------------------------------------------------------------------------------
 * apply (apply_host.cpp:57-395)
 * ------------------------------------------------------------------------------------------- */
typedef struct {
  int32_t vertex;
  int64_t slot; /* >= 0: original edge; < 0: effective insertion -slot-1 */
  int alive;
} row_entry;

int orc_graph_apply(orc_graph* g, int64_t num_inserts, const int32_t* ins_src,
                    const int32_t* ins_dst, const int32_t* ins_w, int64_t num_deletes,
                    const int32_t* del_src, const int32_t* del_dst, orc_summary* summary,
                    char* err, size_t err_cap) {
  const orc_props* pr = &g->props;
  const int k = g->k;
  const int64_t n = g->n;
  orc_summary sm;
  memset(&sm, 0, sizeof(sm));
  int status = ORC_OK;

  /* Step 0: effective operations */
  int32_t* ifrom = (int32_t*)xmalloc((size_t)(2 * num_inserts) * sizeof(int32_t));
  int32_t* ito = (int32_t*)xmalloc((size_t)(2 * num_inserts) * sizeof(int32_t));
  int64_t* iw = (int64_t*)xmalloc((size_t)(2 * num_inserts) * sizeof(int64_t));
  int32_t* dfrom = (int32_t*)xmalloc((size_t)(2 * num_deletes) * sizeof(int32_t));
  int32_t* dto = (int32_t*)xmalloc((size_t)(2 * num_deletes) * sizeof(int32_t));
  int64_t ni = 0, nd = 0, n_after = n;
  for (int64_t i = 0; i < num_inserts; ++i) {
    const int32_t u = ins_src[i], v = ins_dst[i];
    if (u < 0 || v < 0) {
      set_err(err, err_cap, "insertion has a negative id");
      status = ORC_INVALID_ARGUMENT;
      goto done;
    }
    if (!pr->allow_vertex_growth && (u >= n || v >= n)) {
      set_err(err, err_cap, "insertion names a vertex >= n without vertex growth");
      status = ORC_INVALID_ARGUMENT;
      goto done;
    }
    if (u == v && pr->on_self_loop != 0) {
      if (pr->on_self_loop == 2) {
        set_err(err, err_cap, "self-loop insertion under self_loop::error");
        status = ORC_INVALID_ARGUMENT;
        goto done;
      }
      sm.dropped_self_loops++;
      continue;
    }
    if ((int64_t)(u > v ? u : v) >= (int64_t)INT32_MAX) {
      set_err(err, err_cap, "insertion names the largest representable vertex id");
      status = ORC_INVALID_ARGUMENT;
      goto done;
    }
    const int64_t top = (int64_t)(u > v ? u : v) + 1;
    if (top > n_after) n_after = top;
    ifrom[ni] = u; ito[ni] = v; iw[ni] = i; ++ni;
    if (!pr->directed && u != v) {
      ifrom[ni] = v; ito[ni] = u; iw[ni] = i; ++ni;
    }
  }
  for (int64_t j = 0; j < num_deletes; ++j) {
    const int32_t u = del_src[j], v = del_dst[j];
    if (u < 0 || v < 0) {
      set_err(err, err_cap, "deletion has a negative id");
      status = ORC_INVALID_ARGUMENT;
      goto done;
    }
    if (u == v && pr->on_self_loop != 0) {
      if (pr->on_self_loop == 2) {
        set_err(err, err_cap, "self-loop deletion under self_loop::error");
        status = ORC_INVALID_ARGUMENT;
        goto done;
      }
      sm.dropped_self_loops++;
      continue;
    }
    if (u >= n_after || v >= n_after) {
      if (pr->on_missing_delete == 1) {
        set_err(err, err_cap, "deletion names a missing edge under missing_delete::error");
        status = ORC_INVALID_ARGUMENT;
        goto done;
      }
      sm.ignored_deletions += (!pr->directed && u != v) ? 2 : 1;
      continue;
    }
    dfrom[nd] = u; dto[nd] = v; ++nd;
    if (!pr->directed && u != v) {
      dfrom[nd] = v; dto[nd] = u; ++nd;
    }
  }
  {
    const int64_t rows = n_after;
    int64_t* dstart = (int64_t*)calloc((size_t)rows + 1, sizeof(int64_t));
    int64_t* istart = (int64_t*)calloc((size_t)rows + 1, sizeof(int64_t));
    int64_t* dorder = (int64_t*)xmalloc((size_t)nd * sizeof(int64_t));
    int64_t* iorder = (int64_t*)xmalloc((size_t)ni * sizeof(int64_t));
    int64_t* cursor = (int64_t*)xmalloc((size_t)(rows + 1) * sizeof(int64_t));
    for (int64_t j = 0; j < nd; ++j) dstart[dfrom[j] + 1]++;
    for (int64_t i = 0; i < ni; ++i) istart[ifrom[i] + 1]++;
    for (int64_t u = 0; u < rows; ++u) {
      dstart[u + 1] += dstart[u];
      istart[u + 1] += istart[u];
    }
    memcpy(cursor, dstart, (size_t)rows * sizeof(int64_t));
    for (int64_t j = 0; j < nd; ++j) dorder[cursor[dfrom[j]]++] = j;
    memcpy(cursor, istart, (size_t)rows * sizeof(int64_t));
    for (int64_t i = 0; i < ni; ++i) iorder[cursor[ifrom[i]]++] = i;

    /* rebuild every changed row; rows are kept as (offset, length) into one entry pool */
    int64_t* row_off = (int64_t*)xmalloc((size_t)rows * sizeof(int64_t));
    int64_t* row_len = (int64_t*)calloc((size_t)rows, sizeof(int64_t));
    int64_t pool_cap = 0;
    for (int64_t u = 0; u < rows; ++u) {
      row_off[u] = -1;
      if (dstart[u] == dstart[u + 1] && istart[u] == istart[u + 1]) continue;
      pool_cap += (u < n ? g->row_ptr[u + 1] - g->row_ptr[u] : 0) + (istart[u + 1] - istart[u]);
    }
    row_entry* pool = (row_entry*)xmalloc((size_t)pool_cap * sizeof(row_entry));
    int64_t pool_len = 0;
    for (int64_t u = 0; u < rows && status == ORC_OK; ++u) {
      if (dstart[u] == dstart[u + 1] && istart[u] == istart[u + 1]) continue;
      row_entry* row = pool + pool_len;
      int64_t len = 0;
      if (u < n) {
        for (int64_t e = g->row_ptr[u]; e < g->row_ptr[u + 1]; ++e) {
          row[len].vertex = g->col[e];
          row[len].slot = e;
          row[len].alive = 1;
          ++len;
        }
      }
      for (int pass = 0; pass < 2 && status == ORC_OK; ++pass) {
        const int deleting = (pass == 0) == (pr->deletions_first != 0);
        if (deleting) {
          for (int64_t jj = dstart[u]; jj < dstart[u + 1]; ++jj) {
            const int32_t v = dto[dorder[jj]];
            int removed = 0;
            for (int64_t r = 0; r < len; ++r) {
              if (row[r].alive && row[r].vertex == v) {
                row[r].alive = 0;
                removed = 1;
                break;
              }
            }
            if (removed) {
              sm.deleted_edges++;
            } else if (pr->on_missing_delete == 1) {
              set_err(err, err_cap, "deletion names a missing edge under missing_delete::error");
              status = ORC_INVALID_ARGUMENT;
            } else {
              sm.ignored_deletions++;
            }
          }
        } else {
          for (int64_t jj = istart[u]; jj < istart[u + 1]; ++jj) {
            const int64_t i = iorder[jj];
            const int32_t v = ito[i];
            int replaced = 0;
            for (int64_t r = 0; r < len; ++r) {
              if (row[r].alive && row[r].vertex == v) {
                if (pr->on_existing_insert == 0) {
                  row[r].slot = -i - 1;
                  sm.updated_edges++;
                } else if (pr->on_existing_insert == 2) {
                  sm.ignored_insertions++;
                } else {
                  set_err(err, err_cap, "insertion names an existing edge under existing_insert::error");
                  status = ORC_INVALID_ARGUMENT;
                }
                replaced = 1;
                break;
              }
            }
            if (!replaced) {
              row[len].vertex = v;
              row[len].slot = -i - 1;
              row[len].alive = 1;
              ++len;
              sm.inserted_edges++;
            }
          }
        }
      }
      if (pr->sorted) {
        int64_t wpos = 0;
        for (int64_t r = 0; r < len; ++r)
          if (row[r].alive) row[wpos++] = row[r];
        len = wpos;
        /* stable insertion-free sort: a merge sort would do; rows are short, use a stable
         * insertion sort for short rows and qsort on (vertex, position) otherwise */
        for (int64_t a = 1; a < len; ++a) {
          row_entry x = row[a];
          int64_t b = a - 1;
          while (b >= 0 && row[b].vertex > x.vertex) {
            row[b + 1] = row[b];
            --b;
          }
          row[b + 1] = x;
        }
      }
      row_off[u] = pool_len;
      row_len[u] = len;
      pool_len += len;
    }
    if (status == ORC_OK) {
      /* assemble the updated CSR */
      int64_t* new_row = (int64_t*)calloc((size_t)rows + 1, sizeof(int64_t));
#pragma omp parallel for num_threads(g_threads) if (g_threads > 1) schedule(static)
      for (int64_t u = 0; u < rows; ++u) {
        int64_t deg = 0;
        if (row_off[u] >= 0) {
          for (int64_t r = 0; r < row_len[u]; ++r) deg += pool[row_off[u] + r].alive ? 1 : 0;
        } else if (u < n) {
          deg = g->row_ptr[u + 1] - g->row_ptr[u];
        }
        new_row[u + 1] = deg;
      }
      for (int64_t u = 0; u < rows; ++u) new_row[u + 1] += new_row[u];
      const int64_t m_new = new_row[rows];
      int32_t* new_col = (int32_t*)xmalloc((size_t)m_new * sizeof(int32_t));
      int32_t* new_w = (int32_t*)xmalloc((size_t)m_new * (size_t)k * sizeof(int32_t));
#pragma omp parallel for num_threads(g_threads) if (g_threads > 1) schedule(dynamic, 4096)
      for (int64_t u = 0; u < rows; ++u) {
        int64_t out = new_row[u];
        if (row_off[u] < 0) {
          if (u >= n) continue;
          for (int64_t e = g->row_ptr[u]; e < g->row_ptr[u + 1]; ++e, ++out) {
            new_col[out] = g->col[e];
            for (int j = 0; j < k; ++j)
              new_w[(size_t)j * (size_t)m_new + out] = g->w[(size_t)j * (size_t)g->m + e];
          }
          continue;
        }
        for (int64_t r = 0; r < row_len[u]; ++r) {
          const row_entry* en = pool + row_off[u] + r;
          if (!en->alive) continue;
          new_col[out] = en->vertex;
          if (en->slot >= 0) {
            for (int j = 0; j < k; ++j)
              new_w[(size_t)j * (size_t)m_new + out] =
                  g->w[(size_t)j * (size_t)g->m + (size_t)en->slot];
          } else {
            const int64_t i = iw[-en->slot - 1];
            for (int j = 0; j < k; ++j)
              new_w[(size_t)j * (size_t)m_new + out] = ins_w[i * k + j];
          }
          ++out;
        }
      }
      sm.inserted_vertices = n_after - n;
      sm.num_vertices_after = n_after;

      /* classification: weight increases (first (u,v) of row u before and after) */
      free_delta(g);
      g->num_ins = ni;
      g->num_del = nd;
      g->ins_src = (int32_t*)xmalloc((size_t)ni * sizeof(int32_t));
      g->ins_dst = (int32_t*)xmalloc((size_t)ni * sizeof(int32_t));
      g->del_src = (int32_t*)xmalloc((size_t)nd * sizeof(int32_t));
      g->del_dst = (int32_t*)xmalloc((size_t)nd * sizeof(int32_t));
      g->weight_increased = (uint8_t*)calloc((size_t)ni * (size_t)k + 1, 1);
      memcpy(g->ins_src, ifrom, (size_t)ni * sizeof(int32_t));
      memcpy(g->ins_dst, ito, (size_t)ni * sizeof(int32_t));
      memcpy(g->del_src, dfrom, (size_t)nd * sizeof(int32_t));
      memcpy(g->del_dst, dto, (size_t)nd * sizeof(int32_t));
      for (int64_t i = 0; i < ni; ++i) {
        const int64_t u = ifrom[i];
        const int32_t v = ito[i];
        if (u >= n) continue;
        int64_t oe = -1, fe = -1;
        for (int64_t e = g->row_ptr[u]; e < g->row_ptr[u + 1]; ++e)
          if (g->col[e] == v) { oe = e; break; }
        if (oe < 0) continue;
        for (int64_t e = new_row[u]; e < new_row[u + 1]; ++e)
          if (new_col[e] == v) { fe = e; break; }
        if (fe < 0) continue;
        for (int j = 0; j < k; ++j) {
          if (new_w[(size_t)j * (size_t)m_new + fe] > g->w[(size_t)j * (size_t)g->m + oe])
            g->weight_increased[i * k + j] = 1;
        }
      }
      free(g->row_ptr);
      free(g->col);
      free(g->w);
      g->row_ptr = new_row;
      g->col = new_col;
      g->w = new_w;
      g->n = n_after;
      g->m = m_new;
      status = transpose(g);
    }
    free(dstart); free(istart); free(dorder); free(iorder); free(cursor);
    free(row_off); free(row_len); free(pool);
  }
done:
  free(ifrom); free(ito); free(iw); free(dfrom); free(dto);
  if (summary) *summary = sm;
  return status;
}

/* ---------------------------------------------------------------------------------------------
 * Step 0 helpers (sssp.cpp:136-165)
 * ------------------------------------------------------------------------------------------- */
int64_t orc_default_delta(int64_t m, int64_t n, int64_t weight_sum) {
  if (m <= 0 || n <= 0) return 1;
  const double avg_w = (double)weight_sum / (double)m;
  const double avg_deg = (double)m / (double)n;
  const int64_t d = (int64_t)(32.0 * avg_w / avg_deg);
  return d > 1 ? d : 1;
}

int orc_distances_fit(int64_t n, int64_t max_weight) {
  const uint64_t w = (uint64_t)(max_weight > 1 ? max_weight : 1);
  const uint64_t hops = (uint64_t)(n - 1 > 1 ? n - 1 : 1);
  const uint64_t output_max = (uint64_t)(ORC_INF / 2 - 1);
  return w <= output_max / hops;
}

static int parent_bits(int64_t n) {
  int bits = 1;
  while (((1ULL << bits) - 1) < (uint64_t)n) ++bits;
  return bits;
}

/* rule 0: the host backends' rule (bound + one more weight must fit, sssp.cpp:153-165);
 * rule 1: the CUDA engines' rule (bound must fit, kernels.cuh:80-92). */
int orc_packs_parents(int64_t n, int64_t max_weight, int rule) {
  const uint64_t w = (uint64_t)(max_weight > 1 ? max_weight : 1);
  const uint64_t hops = (uint64_t)(n - 1 > 1 ? n - 1 : 1);
  const int bits = parent_bits(n);
  const uint64_t max_distance = (~0ULL >> bits) - 1;
  if (rule == 1) return w <= max_distance / hops; /* (n-1)*w <= max_distance, no overflow */
  return w <= max_distance / hops && w * hops + w <= max_distance;
}

/* ---------------------------------------------------------------------------------------------
 * The sequential engine (sequential.cpp)
 * ------------------------------------------------------------------------------------------- */
typedef struct {
  const orc_graph* g;
  int k;
  int32_t source;
  int64_t* dist;
  int32_t* parent;
  int count_changes;
  /* save() bookkeeping */
  char* seen;
  int32_t* touched;
  int64_t* old_d;
  int32_t* old_p;
  int64_t ntouched;
  int* stamp;
  int generation;
  int32_t* affected;
  int64_t naffected;
  int32_t* next;
  orc_stats* st;
} engine;

static void save(engine* E, int32_t v) {
  if (!E->count_changes || E->seen[v]) return;
  E->seen[v] = 1;
  E->touched[E->ntouched] = v;
  E->old_d[E->ntouched] = E->dist[v];
  E->old_p[E->ntouched] = E->parent[v];
  E->ntouched++;
}

static int relax(engine* E, int32_t v) {
  const orc_graph* g = E->g;
  const int32_t* in_w = g->in_w + (size_t)E->k * (size_t)g->m;
  int32_t best_p = -1;
  int64_t best_d = ORC_INF;
  for (int64_t e = g->in_row_ptr[v]; e < g->in_row_ptr[v + 1]; ++e) {
    const int32_t u = g->in_col[e];
    if (E->dist[u] >= ORC_INF / 2) continue;
    const int64_t cd = E->dist[u] + (int64_t)in_w[e];
    if (cd < best_d || (cd == best_d && u < best_p)) {
      best_d = cd;
      best_p = u;
    }
  }
  const int better = best_d < E->dist[v] ||
                     (best_d == E->dist[v] && best_p >= 0 && best_p < E->parent[v]);
  if (!better) return 0;
  const int decreased = best_d < E->dist[v];
  save(E, v);
  E->dist[v] = best_d;
  E->parent[v] = best_p;
  return decreased;
}

static int loop(engine* E) {
  const orc_graph* g = E->g;
  const int32_t* w = g->w + (size_t)E->k * (size_t)g->m;
  while (E->naffected > 0) {
    E->st->iterations++;
    if (E->st->iterations > g->n) return ORC_NOT_CONVERGED;
    E->st->pushes += E->naffected;
    const int gen = ++E->generation;
    int64_t nn = 0;
    for (int64_t i = 0; i < E->naffected; ++i) {
      const int32_t a = E->affected[i];
      const int64_t da = E->dist[a];
      if (da >= ORC_INF / 2) continue;
      for (int64_t e = g->row_ptr[a]; e < g->row_ptr[a + 1]; ++e) {
        const int32_t x = g->col[e];
        if (x == E->source) continue;
        const int64_t offer = da + (int64_t)w[e];
        if (offer < E->dist[x] || (offer == E->dist[x] && a < E->parent[x])) {
          const int decreased = offer < E->dist[x];
          save(E, x);
          E->dist[x] = offer;
          E->parent[x] = a;
          if (decreased && E->stamp[x] != gen) {
            E->stamp[x] = gen;
            E->next[nn++] = x;
          }
        }
      }
    }
    int32_t* t = E->affected;
    E->affected = E->next;
    E->next = t;
    E->naffected = nn;
  }
  return ORC_OK;
}

static void recover_parents(engine* E) {
  const orc_graph* g = E->g;
  const int32_t* in_w = g->in_w + (size_t)E->k * (size_t)g->m;
  for (int64_t v = 0; v < g->n; ++v) {
    int32_t best = -1;
    if (v != E->source && E->dist[v] < ORC_INF / 2) {
      for (int64_t e = g->in_row_ptr[v]; e < g->in_row_ptr[v + 1]; ++e) {
        const int32_t u = g->in_col[e];
        if (E->dist[u] < ORC_INF / 2 && E->dist[u] + (int64_t)in_w[e] == E->dist[v] &&
            (best < 0 || u < best))
          best = u;
      }
    }
    if (best != E->parent[v]) {
      save(E, (int32_t)v);
      E->parent[v] = best;
    }
  }
}

static int engine_init(engine* E, const orc_graph* g, int k, int32_t source, int64_t* dist,
                       int32_t* parent, orc_stats* st) {
  memset(E, 0, sizeof(*E));
  const size_t n = (size_t)(g->n > 0 ? g->n : 1);
  E->g = g;
  E->k = k;
  E->source = source;
  E->dist = dist;
  E->parent = parent;
  E->st = st;
  E->seen = (char*)calloc(n, 1);
  E->touched = (int32_t*)xmalloc(n * sizeof(int32_t));
  E->old_d = (int64_t*)xmalloc(n * sizeof(int64_t));
  E->old_p = (int32_t*)xmalloc(n * sizeof(int32_t));
  E->stamp = (int*)calloc(n, sizeof(int));
  E->affected = (int32_t*)xmalloc(n * sizeof(int32_t));
  E->next = (int32_t*)xmalloc(n * sizeof(int32_t));
  if (!E->seen || !E->touched || !E->old_d || !E->old_p || !E->stamp || !E->affected || !E->next)
    return ORC_OUT_OF_MEMORY;
  return ORC_OK;
}

static void engine_free(engine* E) {
  free(E->seen); free(E->touched); free(E->old_d); free(E->old_p); free(E->stamp);
  free(E->affected); free(E->next);
}

static void count_affected(engine* E) {
  if (!E->count_changes) {
    int64_t reachable = 0;
    for (int64_t v = 0; v < E->g->n; ++v) reachable += E->dist[v] < ORC_INF / 2;
    E->st->affected = reachable;
    return;
  }
  int64_t a = 0;
  for (int64_t i = 0; i < E->ntouched; ++i) {
    const int32_t v = E->touched[i];
    a += (E->dist[v] != E->old_d[i] || E->parent[v] != E->old_p[i]);
  }
  E->st->affected = a;
}

static void summarize(const orc_graph* g, int k, int64_t* max_w, int64_t* sum_w, int64_t* bad) {
  const int32_t* w = g->w + (size_t)k * (size_t)g->m;
  int64_t mx = 1, s = 0, b = -1;
  for (int64_t e = 0; e < g->m; ++e) {
    if (w[e] > mx) mx = w[e];
    s += w[e];
    if (w[e] < 1 && b < 0) b = e;
  }
  *max_w = mx;
  *sum_w = s;
  *bad = b;
}

/* sssp::compute (sssp.cpp:1208-1249; sequential engine reset -> seed_static -> loop -> finalize) */
int orc_sssp_compute(const orc_graph* g, int32_t source, int k, int64_t delta_opt, int rule,
                     int64_t* dist, int32_t* parent, orc_stats* st, char* err, size_t err_cap) {
  orc_stats s;
  memset(&s, 0, sizeof(s));
  if (source < 0 || source >= g->n) {
    set_err(err, err_cap, "source out of range");
    return ORC_INVALID_ARGUMENT;
  }
  if (k < 0 || k >= g->k) {
    set_err(err, err_cap, "objective out of range");
    return ORC_INVALID_ARGUMENT;
  }
  int64_t max_w, sum_w, bad;
  summarize(g, k, &max_w, &sum_w, &bad);
  if (bad >= 0) {
    set_err(err, err_cap, "an edge weight is below 1");
    return ORC_INVALID_ARGUMENT;
  }
  if (!orc_distances_fit(g->n, max_w)) {
    set_err(err, err_cap, "distances do not fit in 62 bits");
    return ORC_INVALID_ARGUMENT;
  }
  s.delta = delta_opt > 0 ? delta_opt : orc_default_delta(g->m > 1 ? g->m : 1, g->n, sum_w);
  s.max_weight = max_w;
  engine E;
  int status = engine_init(&E, g, k, source, dist, parent, &s);
  if (status == ORC_OK) {
    for (int64_t v = 0; v < g->n; ++v) {
      dist[v] = ORC_INF;
      parent[v] = -1;
    }
    dist[source] = 0;
    E.count_changes = 0;
    E.affected[0] = source;
    E.naffected = 1;
    status = loop(&E);
    if (status == ORC_OK) {
      s.packed_parents = orc_packs_parents(g->n, max_w, rule);
      if (!s.packed_parents) recover_parents(&E);
      count_affected(&E);
    } else {
      set_err(err, err_cap, "the sequential update did not converge");
    }
  }
  engine_free(&E);
  if (st) *st = s;
  return status;
}

/* The rootless-cycle check of identify_affected (sequential.cpp:300-329). */
static int has_rootless_cycle(const orc_graph* g, const int32_t* parent, const int* stamp,
                              int gen) {
  char* color = (char*)calloc((size_t)g->n + 1, 1);
  int32_t* path = (int32_t*)xmalloc((size_t)(g->n + 1) * sizeof(int32_t));
  int cyclic = 0;
  for (int64_t v = 0; v < g->n && !cyclic; ++v) {
    int64_t len = 0;
    int32_t u = (int32_t)v;
    while (u >= 0 && color[u] == 0 && stamp[u] != gen) {
      color[u] = 1;
      path[len++] = u;
      u = parent[u];
    }
    cyclic = u >= 0 && color[u] == 1;
    for (int64_t i = 0; i < len; ++i) color[path[i]] = 2;
  }
  free(color);
  free(path);
  return cyclic;
}

/*
 * sssp::update on an oracle graph: Step 0 on G_t (sssp.cpp:643-689), the commit (apply), then
 * identify_affected -> seed -> loop -> finalize of the sequential engine on G_{t+1}.
 * dist / parent hold the old tree on entry (n_old entries) and receive the new one; their
 * capacity must cover the vertex count after growth (num_vertices_after of the summary).
 */
/* ---------------------------------------------------------------------------------------------
 * The threaded repair (openmp.cpp:223-583), used when the oracle runs on more than one thread
 * (the timed CPU baseline; the checker runs the sequential engine above).  The steps are the
 * sequential engine's, in parallel over the vertices of each step: invalidation by level over a
 * children index, a pull seed of the invalidated vertices and the insertion heads, then push
 * rounds over the vertices whose distance fell.  Every vertex's (distance, parent) lives in one
 * packed word, (distance << bits) | parent, lowered by a compare-and-swap minimum, so a word
 * only ever falls in the lexicographic (distance, parent) order and the fixed point is the
 * canonical tree the sequential engine reaches (lowest parent id among the tight in-edges).
 * ------------------------------------------------------------------------------------------- */
static int atomic_min_u64(uint64_t* p, uint64_t v, uint64_t* old) {
  uint64_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (v < cur) {
    if (__atomic_compare_exchange_n(p, &cur, v, 1, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
      *old = cur;
      return 1;
    }
  }
  return 0;
}

/* Claims v for generation gen (once per generation) and appends it to list[*count]. */
static void claim_append(int* stamp, int32_t v, int gen, int32_t* list, int64_t* count) {
  int cur = __atomic_load_n(&stamp[v], __ATOMIC_RELAXED);
  while (cur != gen) {
    if (__atomic_compare_exchange_n(&stamp[v], &cur, gen, 1, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
      list[__atomic_fetch_add(count, 1, __ATOMIC_RELAXED)] = v;
      return;
    }
  }
}

/* The best packed offer of v's in-row (pull), or ORC_PACKED_NONE.  Offers above maxd (the
 * largest distance a word holds; no shortest distance is above it) are dropped, as the device
 * kernel drops them, so no shift overflows. */
#define ORC_PACKED_NONE UINT64_MAX
static uint64_t pull_offer(const orc_graph* g, const int32_t* in_w, const uint64_t* word,
                           int bits, uint64_t maxd, int64_t v) {
  uint64_t best = ORC_PACKED_NONE;
  for (int64_t e = g->in_row_ptr[v]; e < g->in_row_ptr[v + 1]; ++e) {
    const int32_t u = g->in_col[e];
    const uint64_t wu = __atomic_load_n(&word[u], __ATOMIC_RELAXED);
    if (wu == ORC_PACKED_NONE) continue;
    const uint64_t nd = (wu >> bits) + (uint64_t)in_w[e];
    if (nd > maxd) continue;
    const uint64_t offer = (nd << bits) | (uint64_t)u;
    if (offer < best) best = offer;
  }
  return best;
}

static int update_threaded(orc_graph* g, int32_t source, int k, int64_t n_old,
                           const int32_t* cfrom, const int32_t* cto, int64_t nc, int64_t* dist,
                           int32_t* parent, orc_stats* s, char* err, size_t err_cap) {
  const int64_t n = g->n;
  const int bits = parent_bits(n);
  const uint64_t none = ((uint64_t)1 << bits) - 1;
  const uint64_t maxd = (~0ULL >> bits) - 1;
  const int32_t* w = g->w + (size_t)k * (size_t)g->m;
  const int32_t* in_w = g->in_w + (size_t)k * (size_t)g->m;
  const size_t nz = (size_t)(n > 0 ? n : 1);
  uint64_t* word = (uint64_t*)xmalloc(nz * sizeof(uint64_t));
  int64_t* old_d = (int64_t*)xmalloc(nz * sizeof(int64_t));
  int32_t* old_p = (int32_t*)xmalloc(nz * sizeof(int32_t));
  int* stamp = (int*)calloc(nz, sizeof(int));
  int32_t* list_a = (int32_t*)xmalloc((nz + 1) * sizeof(int32_t));
  int32_t* list_b = (int32_t*)xmalloc((nz + 1) * sizeof(int32_t));
  int64_t* cstart = (int64_t*)calloc(nz + 1, sizeof(int64_t));
  int32_t* children = (int32_t*)xmalloc(nz * sizeof(int32_t));
  int status = ORC_OK;
  (void)n_old;
  /* identify_affected: the roots (tree edges among the changes), checked for rootless cycles */
  const int inval = 1;
  int64_t ninv = 0;
  for (int64_t i = 0; i < nc; ++i) {
    const int32_t u = cfrom[i], v = cto[i];
    if (parent[v] == u && stamp[v] != inval) {
      stamp[v] = inval;
      list_a[ninv++] = v;
    }
  }
  if (nc > 0 && has_rootless_cycle(g, parent, stamp, inval)) {
    set_err(err, err_cap, "sssp: the input shortest-path tree has a parent cycle");
    status = ORC_INVALID_ARGUMENT;
    goto done;
  }
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t v = 0; v < n; ++v) {
    old_d[v] = dist[v];
    old_p[v] = parent[v];
  }
  if (ninv > 0) {
    /* children index: counts, a scan, then a fill (the order inside a row does not matter) */
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int64_t v = 0; v < n; ++v)
      if (v != source && parent[v] >= 0) __atomic_fetch_add(&cstart[parent[v] + 1], 1, __ATOMIC_RELAXED);
    for (int64_t v = 0; v < n; ++v) cstart[v + 1] += cstart[v];
    int64_t* fill = (int64_t*)xmalloc(nz * sizeof(int64_t));
    memcpy(fill, cstart, nz * sizeof(int64_t));
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int64_t v = 0; v < n; ++v)
      if (v != source && parent[v] >= 0)
        children[__atomic_fetch_add(&fill[parent[v]], 1, __ATOMIC_RELAXED)] = (int32_t)v;
    free(fill);
    /* the invalidated subtrees, level by level: list_a[lo, hi) is the current level */
    int64_t lo = 0, hi = ninv;
    while (lo < hi) {
      int64_t top = hi;
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 256)
      for (int64_t i = lo; i < hi; ++i) {
        const int32_t x = list_a[i];
        for (int64_t c = cstart[x]; c < cstart[x + 1]; ++c)
          claim_append(stamp, children[c], inval, list_a, &top);
      }
      lo = hi;
      hi = top;
    }
    ninv = hi;
  }
  s->invalidated = ninv;
  /* packed words: the old tree, the invalidated vertices and new vertices unreached */
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t v = 0; v < n; ++v) {
    const int dead = stamp[v] == inval || dist[v] >= ORC_INF / 2;
    word[v] = dead ? ORC_PACKED_NONE
                   : ((uint64_t)dist[v] << bits) | (parent[v] < 0 ? none : (uint64_t)parent[v]);
  }
  {
    /* seed: every invalidated vertex pulls, then every insertion head (not the source) */
    int gen = 2;
    int64_t nf = 0;
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 256)
    for (int64_t i = 0; i < ninv + g->num_ins; ++i) {
      const int32_t v = i < ninv ? list_a[i] : g->ins_dst[i - ninv];
      if (v == source) continue;
      const uint64_t best = pull_offer(g, in_w, word, bits, maxd, v);
      uint64_t prev;
      if (best != ORC_PACKED_NONE && atomic_min_u64(&word[v], best, &prev) &&
          (prev == ORC_PACKED_NONE || (best >> bits) < (prev >> bits)))
        claim_append(stamp, v, gen, list_b, &nf);
    }
    /* push rounds */
    int32_t* cur = list_b;
    int32_t* nxt = list_a;
    while (nf > 0) {
      s->iterations++;
      if (s->iterations > n) {
        set_err(err, err_cap, "the threaded update did not converge");
        status = ORC_NOT_CONVERGED;
        goto done;
      }
      s->pushes += nf;
      ++gen;
      int64_t nn = 0;
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 64)
      for (int64_t i = 0; i < nf; ++i) {
        const int32_t a = cur[i];
        const uint64_t wa = __atomic_load_n(&word[a], __ATOMIC_RELAXED);
        if (wa == ORC_PACKED_NONE) continue;
        const uint64_t da = wa >> bits;
        for (int64_t e = g->row_ptr[a]; e < g->row_ptr[a + 1]; ++e) {
          const int32_t x = g->col[e];
          const uint64_t nd = da + (uint64_t)w[e];
          if (x == source || nd > maxd) continue;
          const uint64_t offer = (nd << bits) | (uint64_t)a;
          uint64_t prev;
          if (atomic_min_u64(&word[x], offer, &prev) &&
              (prev == ORC_PACKED_NONE || (offer >> bits) < (prev >> bits)))
            claim_append(stamp, x, gen, nxt, &nn);
        }
      }
      int32_t* t = cur;
      cur = nxt;
      nxt = t;
      nf = nn;
    }
  }
  {
    int64_t affected = 0;
#pragma omp parallel for num_threads(g_threads) schedule(static) reduction(+ : affected)
    for (int64_t v = 0; v < n; ++v) {
      const uint64_t x = word[v];
      const int64_t d = x == ORC_PACKED_NONE ? ORC_INF : (int64_t)(x >> bits);
      const int32_t p = x == ORC_PACKED_NONE || (x & none) == none ? -1 : (int32_t)(x & none);
      dist[v] = d;
      parent[v] = p;
      affected += d != old_d[v] || p != old_p[v];
    }
    s->affected = affected;
  }
done:
  free(word); free(old_d); free(old_p); free(stamp); free(list_a); free(list_b); free(cstart);
  free(children);
  return status;
}

int orc_sssp_update(orc_graph* g, int32_t source, int k, int64_t delta_opt, int rule,
                    int64_t num_inserts, const int32_t* ins_src, const int32_t* ins_dst,
                    const int32_t* ins_w, int64_t num_deletes, const int32_t* del_src,
                    const int32_t* del_dst, int64_t* dist, int32_t* parent, orc_stats* st,
                    orc_summary* summary, char* err, size_t err_cap) {
  orc_stats s;
  memset(&s, 0, sizeof(s));
  const int64_t n_old = g->n;
  int64_t largest = 1, max_id = -1;
  for (int64_t i = 0; i < num_inserts; ++i) {
    const int64_t w = ins_w[i * g->k + k];
    if (w < 1) {
      set_err(err, err_cap, "an insertion weight is below 1");
      return ORC_INVALID_ARGUMENT;
    }
    if (w > largest) largest = w;
    const int64_t top = ins_src[i] > ins_dst[i] ? ins_src[i] : ins_dst[i];
    if (top > max_id) max_id = top;
  }
  int64_t col_max, col_sum, bad;
  summarize(g, k, &col_max, &col_sum, &bad);
  const int64_t max_w = largest > col_max ? largest : col_max;
  s.max_weight = max_w;
  s.delta = delta_opt > 0 ? delta_opt : orc_default_delta(g->m > 1 ? g->m : 1, g->n, col_sum);
  int64_t n_after = g->n;
  if (g->props.allow_vertex_growth && max_id + 1 > n_after) n_after = max_id + 1;
  if (!orc_distances_fit(n_after, max_w)) {
    set_err(err, err_cap, "distances do not fit in 62 bits");
    return ORC_INVALID_ARGUMENT;
  }
  int status = orc_graph_apply(g, num_inserts, ins_src, ins_dst, ins_w, num_deletes, del_src,
                               del_dst, summary, err, err_cap);
  if (status != ORC_OK) return status;
  for (int64_t v = n_old; v < g->n; ++v) {
    dist[v] = ORC_INF;
    parent[v] = -1;
  }
  /* change lists: every deletion, then every insertion that raised objective k */
  const int64_t nchanged_cap = g->num_del + g->num_ins;
  int32_t* cfrom = (int32_t*)xmalloc((size_t)nchanged_cap * sizeof(int32_t));
  int32_t* cto = (int32_t*)xmalloc((size_t)nchanged_cap * sizeof(int32_t));
  int64_t nc = 0;
  for (int64_t j = 0; j < g->num_del; ++j) {
    cfrom[nc] = g->del_src[j];
    cto[nc] = g->del_dst[j];
    ++nc;
  }
  for (int64_t i = 0; i < g->num_ins; ++i) {
    if (g->weight_increased[i * g->k + k]) {
      cfrom[nc] = g->ins_src[i];
      cto[nc] = g->ins_dst[i];
      ++nc;
    }
  }
  if (g_threads > 1 && orc_packs_parents(g->n, max_w, rule)) {
    s.packed_parents = 1;
    status = update_threaded(g, source, k, n_old, cfrom, cto, nc, dist, parent, &s, err, err_cap);
    free(cfrom);
    free(cto);
    if (st) *st = s;
    return status;
  }
  engine E;
  status = engine_init(&E, g, k, source, dist, parent, &s);
  if (status == ORC_OK) {
    E.count_changes = 1;
    const int packed = orc_packs_parents(g->n, max_w, rule);
    s.packed_parents = packed;
    /* identify_affected */
    const int inval_gen = ++E.generation;
    int32_t* inv = (int32_t*)xmalloc((size_t)(g->n + 1) * sizeof(int32_t));
    int64_t ninv = 0;
    for (int64_t i = 0; i < nc; ++i) {
      const int32_t u = cfrom[i], v = cto[i];
      if (parent[v] == u && E.stamp[v] != inval_gen) {
        E.stamp[v] = inval_gen;
        inv[ninv++] = v;
      }
    }
    if (nc > 0 && has_rootless_cycle(g, parent, E.stamp, inval_gen)) {
      set_err(err, err_cap, "sssp: the input shortest-path tree has a parent cycle");
      status = ORC_INVALID_ARGUMENT;
    }
    if (status == ORC_OK && ninv > 0) {
      const int64_t n = g->n;
      int64_t* cstart = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
      int32_t* children = (int32_t*)xmalloc((size_t)(n + 1) * sizeof(int32_t));
      int64_t* cur = (int64_t*)xmalloc((size_t)(n + 1) * sizeof(int64_t));
      for (int64_t v = 0; v < n; ++v)
        if (v != source && parent[v] >= 0) cstart[parent[v] + 1]++;
      for (int64_t v = 0; v < n; ++v) cstart[v + 1] += cstart[v];
      memcpy(cur, cstart, (size_t)n * sizeof(int64_t));
      for (int64_t v = 0; v < n; ++v)
        if (v != source && parent[v] >= 0) children[cur[parent[v]]++] = (int32_t)v;
      for (int64_t i = 0; i < ninv; ++i) {
        const int32_t x = inv[i];
        for (int64_t c = cstart[x]; c < cstart[x + 1]; ++c) {
          const int32_t ch = children[c];
          if (E.stamp[ch] != inval_gen) {
            E.stamp[ch] = inval_gen;
            inv[ninv++] = ch;
          }
        }
      }
      for (int64_t i = 0; i < ninv; ++i) {
        save(&E, inv[i]);
        dist[inv[i]] = ORC_INF;
        parent[inv[i]] = -1;
      }
      free(cstart); free(children); free(cur);
    }
    s.invalidated = ninv;
    if (status == ORC_OK) {
      /* seed: invalidated vertices, then insertion heads (not the source) */
      const int aff_gen = ++E.generation;
      E.naffected = 0;
      for (int64_t i = 0; i < ninv; ++i) {
        const int32_t v = inv[i];
        if (relax(&E, v) && E.stamp[v] != aff_gen) {
          E.stamp[v] = aff_gen;
          E.affected[E.naffected++] = v;
        }
      }
      for (int64_t i = 0; i < g->num_ins; ++i) {
        const int32_t v = g->ins_dst[i];
        if (v != source && relax(&E, v) && E.stamp[v] != aff_gen) {
          E.stamp[v] = aff_gen;
          E.affected[E.naffected++] = v;
        }
      }
      status = loop(&E);
      if (status == ORC_OK) {
        if (!packed) recover_parents(&E);
        count_affected(&E);
      } else {
        set_err(err, err_cap, "the sequential update did not converge");
      }
    }
    free(inv);
  }
  engine_free(&E);
  free(cfrom);
  free(cto);
  if (st) *st = s;
  return status;
}

/* ---------------------------------------------------------------------------------------------
 * from_arrays helpers (sssp.cpp:377-460, 571-599)
 * ------------------------------------------------------------------------------------------- */
void orc_canonicalize(const orc_graph* g, int32_t source, int k, const int64_t* dist,
                      int32_t* parent) {
  const int32_t* w = g->w + (size_t)k * (size_t)g->m;
  for (int64_t u = 0; u < g->n; ++u) {
    const int64_t du = dist[u];
    if (du >= ORC_INF / 2) continue;
    for (int64_t e = g->row_ptr[u]; e < g->row_ptr[u + 1]; ++e) {
      const int32_t v = g->col[e];
      if (v != source && u < parent[v] && du + (int64_t)w[e] == dist[v]) parent[v] = (int32_t)u;
    }
  }
}

/* Returns 0 if the tree passes the checks of validate_inputs, else a negative code and message. */
int orc_validate_tree(const orc_graph* g, int32_t source, int k, const int64_t* dist,
                      const int32_t* parent, char* err, size_t err_cap) {
  int64_t max_w, sum_w, bad;
  summarize(g, k, &max_w, &sum_w, &bad);
  const int64_t n = g->n;
  const int64_t bound = max_w * (n - 1 > 1 ? n - 1 : 1);
  if (dist[source] != 0 || parent[source] != -1) {
    set_err(err, err_cap, "the source must have distance 0 and parent -1");
    return ORC_INVALID_ARGUMENT;
  }
  for (int64_t v = 0; v < n; ++v) {
    const int64_t d = dist[v];
    const int32_t p = parent[v];
    if (p < -1 || p >= n) {
      set_err(err, err_cap, "parent outside [-1, n)");
      return ORC_INVALID_ARGUMENT;
    }
    if (d >= ORC_INF / 2) {
      if (p != -1) {
        set_err(err, err_cap, "unreachable vertex has a parent");
        return ORC_INVALID_ARGUMENT;
      }
      continue;
    }
    if (d < 0 || d > bound) {
      set_err(err, err_cap, "distance outside [0, (n - 1) * max weight]");
      return ORC_INVALID_ARGUMENT;
    }
    if (v == source) continue;
    if (p < 0 || dist[p] >= ORC_INF / 2) {
      set_err(err, err_cap, "reachable vertex without a reachable parent");
      return ORC_INVALID_ARGUMENT;
    }
  }
  char* state = (char*)calloc((size_t)n + 1, 1);
  int32_t* path = (int32_t*)xmalloc((size_t)(n + 1) * sizeof(int32_t));
  state[source] = 2;
  int cyclic = 0;
  for (int64_t v = 0; v < n && !cyclic; ++v) {
    if (state[v] != 0 || dist[v] >= ORC_INF / 2) continue;
    int64_t len = 0;
    int32_t u = (int32_t)v;
    while (state[u] == 0) {
      state[u] = 1;
      path[len++] = u;
      u = parent[u];
    }
    if (state[u] != 2) cyclic = 1;
    for (int64_t i = 0; i < len; ++i) state[path[i]] = 2;
  }
  free(state);
  free(path);
  if (cyclic) {
    set_err(err, err_cap, "the input shortest-path tree has a parent cycle");
    return ORC_INVALID_ARGUMENT;
  }
  return ORC_OK;
}

/* ---------------------------------------------------------------------------------------------
 * mosp's finalize step (cpp/src/algorithms/mosp/sequential.cpp:33-170, mosp.cpp:259-301)
 *
 * The combined graph of K trees: edge (p, v) for every distinct parent p among
 * parents[0][v] .. parents[K-1][v] (v != source), weighted
 * base - sum over the trees i with parents[i][v] == p of terms[i]; base = L * (K + 1) and
 * terms[i] = L / Pref_i.  The caller solves it with orc_sssp_compute (lowest-id ties).
 * ------------------------------------------------------------------------------------------- */
static int combined_edge(const int32_t* parents, int64_t n, int K, int64_t v, int k,
                         const int32_t* terms, int32_t base, int32_t* p_out, int32_t* w_out) {
  const int32_t p = parents[(size_t)k * (size_t)n + (size_t)v];
  if (p < 0) return 0;
  for (int j = 0; j < k; ++j)
    if (parents[(size_t)j * (size_t)n + (size_t)v] == p) return 0; /* counted once, first */
  int32_t w = base - terms[k];
  for (int j = k + 1; j < K; ++j)
    if (parents[(size_t)j * (size_t)n + (size_t)v] == p) w -= terms[j];
  *p_out = p;
  *w_out = w;
  return 1;
}

/* Writes the combined edges (src, dst, w; room for K * n) in vertex-then-objective order and
 * returns their number; *weight_sum receives the sum of their weights. */
int64_t orc_mosp_combine(int64_t n, int32_t source, int K, const int32_t* parents,
                         const int32_t* terms, int32_t base, int32_t* src, int32_t* dst,
                         int32_t* w, int64_t* weight_sum) {
  int64_t m = 0, sum = 0;
  for (int64_t v = 0; v < n; ++v) {
    if (v == source) continue;
    for (int k = 0; k < K; ++k) {
      int32_t p, wt;
      if (!combined_edge(parents, n, K, v, k, terms, base, &p, &wt)) continue;
      src[m] = p;
      dst[m] = (int32_t)v;
      w[m] = wt;
      sum += wt;
      ++m;
    }
  }
  if (weight_sum) *weight_sum = sum;
  return m;
}

/* mospPathCosts (sequential.cpp:172-232): the first `columns` objective values of the tree path
 * to every vertex; the weights of tree edge (p, v) are those of the first edge p -> v in row
 * order.  Traversal from the source over the tree's children lists; vertices it does not reach
 * keep ORC_INF.  Returns -1, or the first vertex (in traversal order) whose tree edge is not an
 * edge of the graph. */
int32_t orc_mosp_path_costs(const orc_graph* g, const int32_t* tree, int32_t source, int columns,
                            int64_t* costs) {
  const int64_t n = g->n;
  const size_t C = (size_t)columns;
  for (size_t i = 0; i < (size_t)n * C; ++i) costs[i] = ORC_INF;
  if (n == 0) return -1;
  int64_t* start = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  int64_t* cursor = (int64_t*)xmalloc(((size_t)n + 1) * sizeof(int64_t));
  int32_t* children = (int32_t*)xmalloc((size_t)n * sizeof(int32_t));
  int32_t* queue = (int32_t*)xmalloc((size_t)n * sizeof(int32_t));
  for (int64_t v = 0; v < n; ++v)
    if (v != source && tree[v] >= 0) start[tree[v] + 1]++;
  for (int64_t v = 0; v < n; ++v) start[v + 1] += start[v];
  memcpy(cursor, start, ((size_t)n + 1) * sizeof(int64_t));
  for (int64_t v = 0; v < n; ++v)
    if (v != source && tree[v] >= 0) children[cursor[tree[v]]++] = (int32_t)v;
  for (size_t j = 0; j < C; ++j) costs[(size_t)source * C + j] = 0;
  int64_t head = 0, tail = 0;
  int32_t missing = -1;
  queue[tail++] = source;
  while (head < tail && missing < 0) {
    const int32_t p = queue[head++];
    for (int64_t c = start[p]; c < start[p + 1] && missing < 0; ++c) {
      const int32_t v = children[c];
      int64_t edge = -1;
      for (int64_t e = g->row_ptr[p]; e < g->row_ptr[p + 1]; ++e)
        if (g->col[e] == v) {
          edge = e;
          break;
        }
      if (edge < 0) {
        missing = v;
        break;
      }
      for (size_t j = 0; j < C; ++j)
        costs[(size_t)v * C + j] =
            costs[(size_t)p * C + j] + (int64_t)g->w[j * (size_t)g->m + (size_t)edge];
      queue[tail++] = v;
    }
  }
  free(start);
  free(cursor);
  free(children);
  free(queue);
  return missing;
}
