// Per-iteration negotiation bookkeeping on the device: the loops the
// reference runs in Python over every committed net each iteration
// (orthoroute/algorithms/manhattan/unified_pathfinder.py, "UPF"):
//
//   orsp_node_owner        _rebuild_node_owner (UPF:2762-2837): via barrels, escape-via keepouts
//   orsp_barrel_conflicts  _detect_barrel_conflicts (UPF:5478-5569)
//   orsp_barrel_penalty    the Phase-1 penalty present[conflicts] += p (UPF:3852-3871)
//   orsp_net_scores        the per-net sums of _build_hotset (UPF:5009-5140) and
//                          _order_nets_by_difficulty (UPF:4401-4439)
//
// Nets are given in the reference's dict order as concatenated node paths or
// edge lists with offsets.  Per-net sums run one thread per net in float64 in
// list order, as Python's sum of float(over[e]) does, so they are bit-exact.
#include <algorithm>

#include "common.cuh"

namespace {

// rank[node] = max over (net position m, via step of net m covering node):
// the last net in order wins, as the reference's sequential overwrite.
__global__ void via_barrel_rank_kernel(const int32_t *__restrict__ paths, const int64_t *__restrict__ off, int32_t M,
                                       int32_t nx, int32_t ny, int32_t *__restrict__ rank) {
  const int64_t nxy = (int64_t)nx * ny;
  for (int32_t m = blockIdx.x; m < M; m += gridDim.x) {
    const int64_t a = off[m], b = off[m + 1];
    if (b - a < 2) continue;
    for (int64_t i = a + threadIdx.x; i + 1 < b; i += blockDim.x) {
      const int32_t u = paths[i], v = paths[i + 1];
      const int64_t zu = u / nxy, zv = v / nxy;
      if (u - zu * nxy != v - zv * nxy || zu == zv) continue;  // not a via step
      const int64_t col = u - zu * nxy;
      const int64_t lo = min(zu, zv), hi = max(zu, zv);
      for (int64_t z = lo; z <= hi; ++z) atomicMax(&rank[z * nxy + col], m);
    }
  }
}

__global__ void owner_from_rank_kernel(const int32_t *__restrict__ rank, const int32_t *__restrict__ net_ids,
                                       int32_t *__restrict__ owner, int64_t N) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < N; v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t r = rank[v];
    owner[v] = r >= 0 ? net_ids[r] : -1;
  }
}

// Escape-via keepouts: entry j (node, id) in dict order claims its node when
// no via barrel owns it; the first entry per node wins.
__global__ void keepout_first_kernel(const int32_t *__restrict__ nodes, int32_t K, const int32_t *__restrict__ owner,
                                     int32_t *__restrict__ first) {
  for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < K; j += gridDim.x * blockDim.x) {
    const int32_t v = nodes[j];
    if (v >= 0 && owner[v] == -1) atomicMin(&first[v], j);
  }
}

__global__ void keepout_apply_kernel(const int32_t *__restrict__ nodes, const int32_t *__restrict__ ids, int32_t K,
                                     const int32_t *__restrict__ first, int32_t *__restrict__ owner) {
  for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < K; j += gridDim.x * blockDim.x) {
    const int32_t v = nodes[j];
    if (v >= 0 && first[v] == j) owner[v] = ids[j];
  }
}

__global__ void edge_src_kernel(const int32_t *__restrict__ indptr, int32_t N, int32_t *__restrict__ esrc) {
  for (int32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x)
    for (int32_t k = indptr[u]; k < indptr[u + 1]; ++k) esrc[k] = u;
}

// Conflict: an edge of net m whose source or target is owned by another net.
__global__ void barrel_conflict_kernel(const int32_t *__restrict__ edges, const int64_t *__restrict__ off, int32_t M,
                                       const int32_t *__restrict__ net_ids, const int32_t *__restrict__ owner,
                                       const int32_t *__restrict__ esrc, const int32_t *__restrict__ indices,
                                       uint8_t *__restrict__ mask, unsigned long long *__restrict__ count) {
  unsigned long long local = 0;
  for (int32_t m = blockIdx.x; m < M; m += gridDim.x) {
    const int32_t id = net_ids[m];
    for (int64_t i = off[m] + threadIdx.x; i < off[m + 1]; i += blockDim.x) {
      const int32_t e = edges[i];
      const int32_t os = owner[esrc[e]], od = owner[indices[e]];
      if ((os != -1 && os != id) || (od != -1 && od != id)) {
        ++local;
        if (mask) mask[e] = 1;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}

// present[e] += penalty once per marked edge (numpy fancy-index add: a
// repeated index adds once).
__global__ void barrel_penalty_kernel(const uint8_t *__restrict__ mask, float *__restrict__ present, int64_t E,
                                      float penalty) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x)
    if (mask[e]) present[e] = __fadd_rn(present[e], penalty);
}

__device__ __forceinline__ float over_of(const float *present, const float *cap, int64_t e) {
  const float d = __fsub_rn(present[e], cap[e]);
  return d > 0.0f ? d : 0.0f;
}

// hot[e] = over[e] + 0.1f * hist[e] > 0.5f (float32, numpy's order); count.
__global__ void hot_count_kernel(const float *__restrict__ present, const float *__restrict__ cap,
                                 const float *__restrict__ hist, int64_t E, unsigned long long *__restrict__ count) {
  unsigned long long local = 0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    const float h = __fadd_rn(over_of(present, cap, e), __fmul_rn(0.1f, hist[e]));
    local += h > 0.5f;
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}

// One thread per net, in list order, float64 sums as Python's:
//   congestion[m] = sum(float(over[e]) for e in edges) / max(1, len(edges))
//   impact[m]     = sum(float(over[e]) for e in edges if hot(e))
//   offender[m]   = any(hot(e) for e in edges)
__global__ void net_scores_kernel(const int32_t *__restrict__ edges, const int64_t *__restrict__ off, int32_t M,
                                  const float *__restrict__ present, const float *__restrict__ cap,
                                  const float *__restrict__ hist, double *__restrict__ congestion,
                                  double *__restrict__ impact, uint8_t *__restrict__ offender) {
  for (int32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
    double s = 0.0, im = 0.0;
    bool off_m = false;
    const int64_t a = off[m], b = off[m + 1];
    for (int64_t i = a; i < b; ++i) {
      const int32_t e = edges[i];
      const float ov = over_of(present, cap, e);
      s = __dadd_rn(s, (double)ov);
      const float h = __fadd_rn(ov, __fmul_rn(0.1f, hist[e]));
      if (h > 0.5f) {
        im = __dadd_rn(im, (double)ov);
        off_m = true;
      }
    }
    const int64_t n = b - a;
    if (congestion) congestion[m] = __ddiv_rn(s, (double)(n > 1 ? n : 1));
    if (impact) impact[m] = im;
    if (offender) offender[m] = off_m ? 1 : 0;
  }
}

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

}  // namespace

using namespace orsp;

extern "C" int orsp_node_owner(orsp_graph *g, int32_t M, const int32_t *paths_d, const int64_t *off_d,
                               const int32_t *net_ids_d, int32_t K, const int32_t *keep_nodes_d,
                               const int32_t *keep_ids_d, int32_t *owner_d, uintptr_t stream) {
  if (!g || M < 0 || K < 0 || (M > 0 && (!paths_d || !off_d || !net_ids_d)) ||
      (K > 0 && (!keep_nodes_d || !keep_ids_d)) || !owner_d) {
    set_error("node_owner: bad arguments");
    return ORSP_ERR_ARG;
  }
  if (g->nx <= 0 || g->ny <= 0) { set_error("node_owner: graph has no lattice dims"); return ORSP_ERR_ARG; }
  ORSP_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_scratch(g, (size_t)g->N * 8);
  if (rc) return rc;
  int32_t *rank = (int32_t *)g->scratch;
  int32_t *first = rank + g->N;
  ORSP_CUDA(cudaMemsetAsync(rank, 0xff, (size_t)g->N * 4, st));
  if (M > 0) {
    via_barrel_rank_kernel<<<std::min(M, 148 * 8), 128, 0, st>>>(paths_d, off_d, M, g->nx, g->ny, rank);
    ORSP_CUDA(cudaGetLastError());
  }
  owner_from_rank_kernel<<<grid_for(g->N), 256, 0, st>>>(rank, net_ids_d, owner_d, g->N);
  ORSP_CUDA(cudaGetLastError());
  if (K > 0) {
    ORSP_CUDA(cudaMemsetAsync(first, 0x7f, (size_t)g->N * 4, st));  // 0x7f7f7f7f: no entry
    keepout_first_kernel<<<grid_for(K), 256, 0, st>>>(keep_nodes_d, K, owner_d, first);
    ORSP_CUDA(cudaGetLastError());
    keepout_apply_kernel<<<grid_for(K), 256, 0, st>>>(keep_nodes_d, keep_ids_d, K, first, owner_d);
    ORSP_CUDA(cudaGetLastError());
  }
  return ORSP_OK;
}

extern "C" int orsp_barrel_conflicts(orsp_graph *g, int32_t M, const int32_t *edges_d, const int64_t *off_d,
                                     const int32_t *net_ids_d, const int32_t *owner_d, uint8_t *mask_d,
                                     int64_t *count_h, uintptr_t stream) {
  if (!g || M < 0 || (M > 0 && (!edges_d || !off_d || !net_ids_d)) || !owner_d || !count_h) {
    set_error("barrel_conflicts: bad arguments");
    return ORSP_ERR_ARG;
  }
  ORSP_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = (cudaStream_t)stream;
  if (!g->edge_src) {
    ORSP_CUDA(cudaMalloc(&g->edge_src, (size_t)std::max<int64_t>(1, g->E) * 4));
    edge_src_kernel<<<grid_for(g->N), 256, 0, st>>>(g->indptr, g->N, g->edge_src);
    ORSP_CUDA(cudaGetLastError());
  }
  if (!g->route_ws) ORSP_CUDA(cudaMalloc(&g->route_ws, 256));
  unsigned long long *cnt = (unsigned long long *)((char *)g->route_ws + 64);
  ORSP_CUDA(cudaMemsetAsync(cnt, 0, 8, st));
  if (mask_d) ORSP_CUDA(cudaMemsetAsync(mask_d, 0, (size_t)g->E, st));
  if (M > 0) {
    barrel_conflict_kernel<<<std::min(M, 148 * 8), 128, 0, st>>>(edges_d, off_d, M, net_ids_d, owner_d, g->edge_src,
                                                                  g->indices, mask_d, cnt);
    ORSP_CUDA(cudaGetLastError());
  }
  unsigned long long *h = (unsigned long long *)((char *)g->pinned + 256);
  ORSP_CUDA(cudaMemcpyAsync(h, cnt, 8, cudaMemcpyDeviceToHost, st));
  ORSP_CUDA(cudaStreamSynchronize(st));
  *count_h = (int64_t)*h;
  return ORSP_OK;
}

extern "C" int orsp_barrel_penalty(int64_t E, const uint8_t *mask_d, float *present_d, float penalty,
                                   uintptr_t stream) {
  if (E < 0 || (E > 0 && (!mask_d || !present_d))) { set_error("barrel_penalty: bad arguments"); return ORSP_ERR_ARG; }
  if (E == 0) return ORSP_OK;
  barrel_penalty_kernel<<<grid_for(E), 256, 0, (cudaStream_t)stream>>>(mask_d, present_d, E, penalty);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_net_scores(orsp_graph *g, int32_t M, const int32_t *edges_d, const int64_t *off_d,
                               const float *present_d, const float *cap_d, const float *hist_d,
                               double *congestion_d, double *impact_d, uint8_t *offender_d, int64_t *hot_count_h,
                               uintptr_t stream) {
  if (!g || M < 0 || (M > 0 && (!edges_d || !off_d)) || !present_d || !cap_d || !hist_d) {
    set_error("net_scores: bad arguments");
    return ORSP_ERR_ARG;
  }
  ORSP_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = (cudaStream_t)stream;
  if (M > 0) {
    net_scores_kernel<<<std::max(1, (M + 127) / 128), 128, 0, st>>>(edges_d, off_d, M, present_d, cap_d, hist_d,
                                                                      congestion_d, impact_d, offender_d);
    ORSP_CUDA(cudaGetLastError());
  }
  if (hot_count_h) {
    if (!g->route_ws) ORSP_CUDA(cudaMalloc(&g->route_ws, 256));
    unsigned long long *cnt = (unsigned long long *)((char *)g->route_ws + 128);
    ORSP_CUDA(cudaMemsetAsync(cnt, 0, 8, st));
    hot_count_kernel<<<grid_for(g->E), 256, 0, st>>>(present_d, cap_d, hist_d, g->E, cnt);
    ORSP_CUDA(cudaGetLastError());
    unsigned long long *h = (unsigned long long *)((char *)g->pinned + 264);
    ORSP_CUDA(cudaMemcpyAsync(h, cnt, 8, cudaMemcpyDeviceToHost, st));
    ORSP_CUDA(cudaStreamSynchronize(st));
    *hot_count_h = (int64_t)*h;
  }
  return ORSP_OK;
}
