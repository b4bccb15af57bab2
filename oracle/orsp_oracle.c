/*
 * ORACLE - test infrastructure only.  Nothing in the product links this file:
 * it is the CPU checker that the tests, the smoke check and the CPU baseline
 * of bench.py compare the CUDA library against.
 *
 * Plain-C restatement of the reference's CPU search path
 * (orthoroute/algorithms/manhattan/unified_pathfinder.py, "UPF"):
 *   oracle_dijkstra      SimpleDijkstra.find_path_roi            UPF:1801-1887
 *                        SimpleDijkstra.find_path_multisource_multisink
 *                                                                 UPF:1889-1989
 *   oracle_roi_bfs       ROIExtractor.extract_roi_bfs            UPF:1636-1734
 *   oracle_roi_bfs_keep  the same with portal seeds (must-keep)  UPF:1700-1731
 *   oracle_path_to_edges PathFinderRouter._path_to_edges         UPF:5463-5476
 *
 * Arithmetic: the reference adds path costs in Python float64 (UPF:1871) and
 * stores float32; this restatement adds in float32 (`alt = du + w` on floats,
 * compiled with -ffp-contract=off), which is the exact semantics the CUDA
 * kernels implement.  Both agree whenever the float64 sums are exactly
 * representable (e.g. integer costs); the golden vectors generated from the
 * reference pin that agreement.  The heap pops in (distance, ROI index) order
 * like Python's heapq on (alt, v_roi) tuples, and a parent is only replaced
 * by a strictly smaller distance, as in the reference.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  float d;
  int32_t rank;
  int32_t node;
} hitem;

typedef struct {
  hitem *a;
  int64_t n, cap;
} heap_t;

static int hless(const hitem *x, const hitem *y) {
  if (x->d < y->d) return 1;
  if (x->d > y->d) return 0;
  return x->rank < y->rank;
}

static int hpush(heap_t *h, hitem it) {
  if (h->n == h->cap) {
    int64_t nc = h->cap ? 2 * h->cap : 1024;
    hitem *na = (hitem *)realloc(h->a, (size_t)nc * sizeof(hitem));
    if (!na) return -1;
    h->a = na;
    h->cap = nc;
  }
  int64_t i = h->n++;
  h->a[i] = it;
  while (i > 0) {
    int64_t p = (i - 1) / 2;
    if (!hless(&h->a[i], &h->a[p])) break;
    hitem t = h->a[i];
    h->a[i] = h->a[p];
    h->a[p] = t;
    i = p;
  }
  return 0;
}

static hitem hpop(heap_t *h) {
  hitem top = h->a[0];
  h->a[0] = h->a[--h->n];
  int64_t i = 0;
  for (;;) {
    int64_t l = 2 * i + 1, r = l + 1, m = i;
    if (l < h->n && hless(&h->a[l], &h->a[m])) m = l;
    if (r < h->n && hless(&h->a[r], &h->a[m])) m = r;
    if (m == i) break;
    hitem t = h->a[i];
    h->a[i] = h->a[m];
    h->a[m] = t;
    i = m;
  }
  return top;
}

/*
 * Heap Dijkstra on the ROI-induced subgraph.
 *   roi_map    global_to_roi (int32[N], -1 = outside) or NULL (whole graph,
 *              rank = node id)
 *   seeds      start nodes with start costs (seed_cost NULL = 0.0); seeds are
 *              never given a parent unless a strictly shorter path reaches them
 *   dst        >= 0: stop when dst is popped (UPF:1857-1859); -1: run to the end
 *   target_mask/target_cost  multi-sink mode (dst must be -1): popped targets
 *              are not expanded (UPF:1954-1962) and the target minimising
 *              (double)d + target_cost wins, first popped on ties
 * Outputs dist (float32[N], +inf = not reached), parent (int32[N], -1), and
 * the path seed..dst (or seed..best target) in path_out; returns the path
 * length (0 = no path), -1 on allocation failure, -2 if path_cap is too small.
 */
int oracle_dijkstra(int32_t N, const int32_t *indptr, const int32_t *indices, const float *cost,
                    int32_t nseeds, const int32_t *seeds, const float *seed_cost, int32_t dst,
                    const int32_t *roi_map, const uint8_t *target_mask,
                    const double *target_cost, float *dist, int32_t *parent, int32_t *path_out,
                    int32_t path_cap, int32_t *best_target_out) {
  uint8_t *visited = (uint8_t *)calloc((size_t)N, 1);
  if (!visited) return -1;
  for (int32_t i = 0; i < N; ++i) {
    dist[i] = INFINITY;
    parent[i] = -1;
  }
  heap_t h = {0, 0, 0};
  for (int32_t i = 0; i < nseeds; ++i) {
    int32_t s = seeds[i];
    if (s < 0 || s >= N) continue;
    if (roi_map && roi_map[s] < 0) continue;
    float c = seed_cost ? seed_cost[i] : 0.0f;
    dist[s] = c;
    hitem it = {c, roi_map ? roi_map[s] : s, s};
    if (hpush(&h, it)) { free(visited); free(h.a); return -1; }
  }
  int32_t best_t = -1;
  double best_total = INFINITY;
  while (h.n > 0) {
    hitem it = hpop(&h);
    int32_t u = it.node;
    if (visited[u]) continue;
    visited[u] = 1;
    if (u == dst) break;
    if (target_mask && target_mask[u]) {
      double total = (double)it.d + target_cost[u];
      if (total < best_total) {
        best_total = total;
        best_t = u;
      }
      continue;
    }
    const float du = it.d;
    for (int32_t e = indptr[u]; e < indptr[u + 1]; ++e) {
      int32_t v = indices[e];
      if (roi_map && roi_map[v] < 0) continue;
      if (visited[v]) continue;
      float alt = du + cost[e];
      if (alt < dist[v]) {
        dist[v] = alt;
        parent[v] = u;
        hitem nv = {alt, roi_map ? roi_map[v] : v, v};
        if (hpush(&h, nv)) { free(visited); free(h.a); return -1; }
      }
    }
  }
  free(visited);
  free(h.a);
  int32_t end = dst >= 0 ? dst : best_t;
  if (best_target_out) *best_target_out = best_t;
  if (end < 0 || !(dist[end] < INFINITY)) return 0;
  int32_t len = 0;
  for (int32_t v = end; v != -1; v = parent[v]) {
    if (len >= path_cap) return -2;
    path_out[len++] = v;
  }
  for (int32_t i = 0; i < len / 2; ++i) {
    int32_t t = path_out[i];
    path_out[i] = path_out[len - 1 - i];
    path_out[len - 1 - i] = t;
  }
  return len;
}

/*
 * ROIExtractor.extract_roi_bfs (UPF:1636-1734), sequential queues exactly as
 * the reference steps them.  roi_out needs room for N ids; returns the ROI
 * size after truncation to max_nodes (-1 on allocation failure).
 */
int32_t oracle_roi_bfs_keep(int32_t N, const int32_t *indptr, const int32_t *indices, int32_t src,
                            int32_t dst, int32_t max_depth, int32_t max_nodes, const int32_t *keep,
                            int32_t nkeep, int32_t *roi_out);

int32_t oracle_roi_bfs(int32_t N, const int32_t *indptr, const int32_t *indices, int32_t src,
                       int32_t dst, int32_t max_depth, int32_t max_nodes, int32_t *roi_out) {
  return oracle_roi_bfs_keep(N, indptr, indices, src, dst, max_depth, max_nodes, 0, 0, roi_out);
}

/* The same with portal seeds (UPF:1700-1731): must_keep = [src, dst] plus
 * each keep node not yet in it; the ones not in the ROI are appended in that
 * order; on truncation, for the k-th list position (ascending) that holds a
 * must-keep node, a position >= max_nodes is swapped with position k. */
int32_t oracle_roi_bfs_keep(int32_t N, const int32_t *indptr, const int32_t *indices, int32_t src,
                            int32_t dst, int32_t max_depth, int32_t max_nodes, const int32_t *keep,
                            int32_t nkeep, int32_t *roi_out) {
  uint8_t *seen = (uint8_t *)calloc((size_t)N, 1);
  int32_t *qs = (int32_t *)malloc((size_t)N * 4), *qs2 = (int32_t *)malloc((size_t)N * 4);
  int32_t *qd = (int32_t *)malloc((size_t)N * 4), *qd2 = (int32_t *)malloc((size_t)N * 4);
  if (!seen || !qs || !qs2 || !qd || !qd2) {
    free(seen); free(qs); free(qs2); free(qd); free(qd2);
    return -1;
  }
  int32_t ns = 1, nd = 1;
  qs[0] = src;
  qd[0] = dst;
  seen[src] = 1;
  seen[dst] = 2;
  int64_t total = (src == dst) ? 1 : 2;
  int depth = 0, met = 0;
  while (depth < max_depth && (ns > 0 || nd > 0) && !met) {
    for (int wave = 0; wave < 2; ++wave) {
      if (wave == 1 && met) break;
      uint8_t mark = wave == 0 ? 1 : 2;
      int32_t *q = wave == 0 ? qs : qd, *qn = wave == 0 ? qs2 : qd2;
      int32_t n = wave == 0 ? ns : nd, nn = 0;
      int met_flag = 0;
      for (int32_t i = 0; i < n; ++i) {
        int32_t u = q[i];
        for (int32_t e = indptr[u]; e < indptr[u + 1]; ++e) {
          int32_t v = indices[e];
          if (seen[v] == 0) {
            seen[v] = mark;
            qn[nn++] = v;
          } else if (seen[v] != mark) {
            seen[v] = 3;
            met_flag = 1;
          }
        }
      }
      total += nn;
      if (met_flag) met = 1;
      if (wave == 0) {
        int32_t *t = qs; qs = qs2; qs2 = t; ns = nn;
      } else {
        int32_t *t = qd; qd = qd2; qd2 = t; nd = nn;
      }
    }
    ++depth;
    if ((double)total > (double)max_nodes * 1.5) break;
  }
  int32_t cnt = 0;
  for (int32_t v = 0; v < N; ++v)
    if (seen[v]) roi_out[cnt++] = v;
  /* must_keep = [src, dst] + keep nodes not already in it */
  int32_t *mk = (int32_t *)malloc((size_t)(nkeep + 2) * 4);
  int32_t nmk = 0;
  mk[nmk++] = src;
  mk[nmk++] = dst;
  for (int32_t i = 0; i < nkeep; ++i) {
    int dup = 0;
    for (int32_t j = 0; j < nmk; ++j) dup |= mk[j] == keep[i];
    if (!dup) mk[nmk++] = keep[i];
  }
  /* missing must-keep nodes appended in list order */
  for (int32_t j = 0; j < nmk; ++j) {
    if (seen[mk[j]]) continue;
    int dup = 0;
    for (int32_t i = 0; i < cnt; ++i) dup |= roi_out[i] == mk[j];
    if (!dup) roi_out[cnt++] = mk[j];
  }
  if (cnt > max_nodes) {
    int32_t *kept = (int32_t *)malloc((size_t)nmk * 4);
    int32_t nk = 0;
    for (int32_t i = 0; i < cnt; ++i) {
      int is_keep = 0;
      for (int32_t j = 0; j < nmk; ++j) is_keep |= roi_out[i] == mk[j];
      if (is_keep) kept[nk++] = i;
    }
    for (int32_t k = 0; k < nk; ++k) {
      if (kept[k] >= max_nodes) {
        int32_t t = roi_out[kept[k]];
        roi_out[kept[k]] = roi_out[k];
        roi_out[k] = t;
      }
    }
    free(kept);
    cnt = max_nodes;
  }
  free(mk);
  free(seen); free(qs); free(qs2); free(qd); free(qd2);
  return cnt;
}

/* PathFinderRouter._path_to_edges (UPF:5463-5476): first CSR edge per pair,
 * pairs without an edge skipped.  Returns the number of edges written. */
int32_t oracle_path_to_edges(const int32_t *indptr, const int32_t *indices, const int32_t *path,
                             int32_t len, int32_t *out) {
  int32_t n = 0;
  for (int32_t i = 0; i + 1 < len; ++i) {
    int32_t u = path[i], v = path[i + 1];
    for (int32_t e = indptr[u]; e < indptr[u + 1]; ++e) {
      if (indices[e] == v) {
        out[n++] = e;
        break;
      }
    }
  }
  return n;
}

/* Many independent single-source searches (one per net) on shared costs, each
 * inside a box ROI given as inclusive [x0,x1,y0,y1,z0,z1] on an nx*ny*nz
 * lattice, as the batched GPU search does.  Paths go to path_nodes[k*cap..],
 * lengths to path_len[k] (0 = no path).  Sequential: this is the checker. */
int oracle_batch_bbox(int32_t N, const int32_t *indptr, const int32_t *indices, const float *cost,
                      int32_t nx, int32_t ny, int32_t nz, int32_t K, const int32_t *src,
                      const int32_t *dst, const int32_t *bbox, int32_t *path_nodes,
                      int32_t path_cap, int32_t *path_len) {
  int32_t *roi = (int32_t *)malloc((size_t)N * 4);
  float *dist = (float *)malloc((size_t)N * 4);
  int32_t *parent = (int32_t *)malloc((size_t)N * 4);
  if (!roi || !dist || !parent) { free(roi); free(dist); free(parent); return -1; }
  for (int32_t i = 0; i < N; ++i) roi[i] = -1;
  const int64_t plane = (int64_t)nx * ny;
  for (int32_t k = 0; k < K; ++k) {
    const int32_t *b = bbox + 6 * (int64_t)k;
    const int32_t W = b[1] - b[0] + 1, H = b[3] - b[2] + 1;
    for (int32_t z = b[4]; z <= b[5]; ++z)
      for (int32_t y = b[2]; y <= b[3]; ++y)
        for (int32_t x = b[0]; x <= b[1]; ++x)
          roi[z * plane + (int64_t)y * nx + x] = ((z - b[4]) * H + (y - b[2])) * W + (x - b[0]);
    int32_t s = src[k];
    int rc = oracle_dijkstra(N, indptr, indices, cost, 1, &s, NULL, dst[k], roi, NULL, NULL, dist,
                             parent, path_nodes + (int64_t)k * path_cap, path_cap, NULL);
    path_len[k] = rc;
    for (int32_t z = b[4]; z <= b[5]; ++z)
      for (int32_t y = b[2]; y <= b[3]; ++y)
        for (int32_t x = b[0]; x <= b[1]; ++x) roi[z * plane + (int64_t)y * nx + x] = -1;
    (void)nz;
  }
  free(roi); free(dist); free(parent);
  return 0;
}
