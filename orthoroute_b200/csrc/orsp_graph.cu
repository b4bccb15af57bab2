// Graph context: CSR upload, transposed CSR for the backtrace, error plumbing.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace orsp {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int cuda_fail(cudaError_t e, const char *what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  // a failed launch or call leaves its (non-sticky) error as the thread's
  // last error; clear it, so that the caller's next unrelated check does not
  // report it again
  (void)cudaGetLastError();
  return e == cudaErrorMemoryAllocation ? ORSP_ERR_NOMEM : ORSP_ERR_CUDA;
}

int dev_status_to_orsp(int dev) {
  switch (dev) {
    case DEV_OK: return ORSP_OK;
    case DEV_ERR_TIMEOUT: set_error("device wait or round limit reached"); return ORSP_ERR_TIMEOUT;
    case DEV_ERR_OVERFLOW: set_error("device work queue overflow"); return ORSP_ERR_OVERFLOW;
    case DEV_ERR_PATH_OVERFLOW: set_error("path longer than path_cap"); return ORSP_ERR_OVERFLOW;
    default: set_error("device invariant violated (no predecessor on backtrace)"); return ORSP_ERR_INTERNAL;
  }
}

int ensure_scratch(Graph *g, size_t bytes) {
  if (g->scratch_bytes >= bytes) return ORSP_OK;
  if (g->scratch) cudaFree(g->scratch);
  g->scratch = nullptr;
  g->scratch_bytes = 0;
  ORSP_CUDA(cudaMalloc(&g->scratch, bytes));
  g->scratch_bytes = bytes;
  return ORSP_OK;
}

int ensure_roi_arrays(Graph *g) {
  bool fresh = false;
  if (!g->roi_map) {
    ORSP_CUDA(cudaMalloc(&g->roi_map, (size_t)g->N * 4));
    ORSP_CUDA(cudaMemset(g->roi_map, 0xff, (size_t)g->N * 4));
    fresh = true;
  }
  if (!g->sink_mask) {
    ORSP_CUDA(cudaMalloc(&g->sink_mask, (size_t)g->N));
    ORSP_CUDA(cudaMemset(g->sink_mask, 0, (size_t)g->N));
    fresh = true;
  }
  if (!g->roi_bb) ORSP_CUDA(cudaMalloc(&g->roi_bb, 64));
  if (!g->seed_one) ORSP_CUDA(cudaMalloc(&g->seed_one, 64));
  // the memsets run on the legacy stream, which a caller's non-blocking
  // stream does not wait for
  if (fresh) ORSP_CUDA(cudaDeviceSynchronize());
  return ORSP_OK;
}

}  // namespace orsp

using namespace orsp;

extern "C" int orsp_abi_version(void) { return ORSP_ABI_VERSION; }

extern "C" const char *orsp_status_string(int s) {
  switch (s) {
    case ORSP_OK: return "ok";
    case ORSP_NO_PATH: return "no path";
    case ORSP_ERR_ARG: return "invalid argument";
    case ORSP_ERR_CUDA: return "CUDA error";
    case ORSP_ERR_TIMEOUT: return "device timeout";
    case ORSP_ERR_OVERFLOW: return "buffer overflow";
    case ORSP_ERR_NOMEM: return "out of device memory";
    case ORSP_ERR_INTERNAL: return "internal error";
    default: return "unknown status";
  }
}

extern "C" const char *orsp_last_error(void) { return g_last_error.c_str(); }

extern "C" int orsp_graph_create(int32_t N, int64_t E, const int32_t *indptr_h,
                                 const int32_t *indices_h, int32_t nx, int32_t ny,
                                 int32_t nz, int device, orsp_graph **out) {
  if (!out) { set_error("out is NULL"); return ORSP_ERR_ARG; }
  *out = nullptr;
  if (N <= 0 || E < 0 || E >= (int64_t)INT32_MAX || !indptr_h || (E > 0 && !indices_h)) {
    set_error("invalid graph sizes or NULL CSR arrays (E must fit int32)");
    return ORSP_ERR_ARG;
  }
  if (indptr_h[0] != 0 || (int64_t)indptr_h[N] != E) {
    set_error("indptr must start at 0 and end at E");
    return ORSP_ERR_ARG;
  }
  if ((nx | ny | nz) != 0 && (int64_t)nx * ny * nz != N) {
    set_error("lattice dims do not multiply to N");
    return ORSP_ERR_ARG;
  }
  // Validate the CSR on the host and build the transposed CSR (counting sort
  // by destination; within a destination, sources ascend because edges are
  // visited in CSR order, which is sorted by source).
  std::vector<int32_t> rcount(N + 1, 0);
  int32_t maxdeg = 0;
  for (int32_t u = 0; u < N; ++u) {
    int32_t b = indptr_h[u], e = indptr_h[u + 1];
    if (e < b) { set_error("indptr not monotone"); return ORSP_ERR_ARG; }
    if (e - b > maxdeg) maxdeg = e - b;
    for (int32_t k = b; k < e; ++k) {
      int32_t v = indices_h[k];
      if (v < 0 || v >= N) { set_error("indices out of range"); return ORSP_ERR_ARG; }
      rcount[v + 1]++;
    }
  }
  int32_t maxin = 0;
  for (int32_t v = 0; v < N; ++v) {
    if (rcount[v + 1] > maxin) maxin = rcount[v + 1];
    rcount[v + 1] += rcount[v];
  }
  std::vector<int32_t> rsrc(E > 0 ? E : 1), reid(E > 0 ? E : 1);
  {
    std::vector<int32_t> fill(rcount.begin(), rcount.end() - 1);
    for (int32_t u = 0; u < N; ++u) {
      for (int32_t k = indptr_h[u]; k < indptr_h[u + 1]; ++k) {
        int32_t v = indices_h[k];
        int32_t pos = fill[v]++;
        rsrc[pos] = u;
        reid[pos] = k;
      }
    }
  }

  cudaError_t ce = cudaSetDevice(device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  orsp_graph *g = new orsp_graph();
  g->device = device;
  g->N = N;
  g->E = E;
  g->nx = nx; g->ny = ny; g->nz = nz;
  g->max_degree = maxdeg;
  g->max_in_degree = maxin;
  cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, device);
  size_t eb = (size_t)(E > 0 ? E : 1) * sizeof(int32_t);
  size_t nb = (size_t)(N + 1) * sizeof(int32_t);
#define TRY(call)                                   \
  do {                                              \
    cudaError_t _e = (call);                        \
    if (_e != cudaSuccess) {                        \
      int st = cuda_fail(_e, #call);                \
      orsp_graph_destroy(g);                        \
      return st;                                    \
    }                                               \
  } while (0)
  TRY(cudaMalloc(&g->indptr, nb));
  TRY(cudaMalloc(&g->indices, eb));
  TRY(cudaMalloc(&g->rptr, nb));
  TRY(cudaMalloc(&g->rsrc, eb));
  TRY(cudaMalloc(&g->reid, eb));
  TRY(cudaMemcpy(g->indptr, indptr_h, nb, cudaMemcpyHostToDevice));
  if (E > 0) TRY(cudaMemcpy(g->indices, indices_h, (size_t)E * 4, cudaMemcpyHostToDevice));
  TRY(cudaMemcpy(g->rptr, rcount.data(), nb, cudaMemcpyHostToDevice));
  if (E > 0) {
    TRY(cudaMemcpy(g->rsrc, rsrc.data(), (size_t)E * 4, cudaMemcpyHostToDevice));
    TRY(cudaMemcpy(g->reid, reid.data(), (size_t)E * 4, cudaMemcpyHostToDevice));
  }
  TRY(cudaMallocHost(&g->pinned, 4096));
  TRY(cudaMalloc(&g->auto_delta, 2 * sizeof(float)));
#undef TRY
  if (nx > 0) {
    int rc = analyze_lattice(g, indptr_h, indices_h);
    if (rc) {
      orsp_graph_destroy(g);
      return rc;
    }
  }
  *out = g;
  return ORSP_OK;
}

extern "C" int orsp_graph_destroy(orsp_graph *g) {
  if (!g) return ORSP_OK;
  cudaSetDevice(g->device);
  cudaFree(g->indptr);
  cudaFree(g->indices);
  cudaFree(g->rptr);
  cudaFree(g->rsrc);
  cudaFree(g->reid);
  cudaFree(g->dist);
  for (int i = 0; i < 2; ++i) {
    cudaFree(g->near_q[i]);
    cudaFree(g->far_q[i]);
  }
  cudaFree(g->ctl);
  if (g->ctl_h) cudaFreeHost(g->ctl_h);
  cudaFree(g->batch_ws);
  cudaFree(g->batch_ctl);
  cudaFree(g->scratch);
  cudaFree(g->auto_delta);
  cudaFree(g->route_ws);
  cudaFree(g->batch_idx);
  cudaFree(g->blat_dist);
  cudaFree(g->blat_tab_d);
  if (g->blat_tab_h) cudaFreeHost(g->blat_tab_h);
  cudaFree(g->route_tab_d);
  if (g->route_tab_h) cudaFreeHost(g->route_tab_h);
  if (g->route_stream) cudaStreamDestroy(g->route_stream);
  cudaFree(g->route_pdist);
  cudaFree(g->route_flags);
  cudaFree(g->route_owner);
  for (cudaEvent_t e : g->route_ev)
    if (e) cudaEventDestroy(e);
  cudaFree(g->box_g2r);
  cudaFree(g->edge_src);
  cudaFree(g->roi_map);
  cudaFree(g->sink_mask);
  cudaFree(g->roi_bb);
  cudaFree(g->seed_one);
  if (g->pinned) cudaFreeHost(g->pinned);
  free_lattice(g);
  delete g;
  return ORSP_OK;
}

extern "C" int orsp_graph_csr(orsp_graph *g, const int32_t **indptr_d,
                              const int32_t **indices_d) {
  if (!g) { set_error("graph is NULL"); return ORSP_ERR_ARG; }
  if (indptr_d) *indptr_d = g->indptr;
  if (indices_d) *indices_d = g->indices;
  return ORSP_OK;
}

extern "C" int orsp_graph_max_degree(orsp_graph *g, int32_t *out) {
  if (!g || !out) { set_error("NULL argument"); return ORSP_ERR_ARG; }
  *out = g->max_degree;
  return ORSP_OK;
}

extern "C" int orsp_graph_is_lattice(orsp_graph *g, int32_t *out) {
  if (!g || !out) { set_error("NULL argument"); return ORSP_ERR_ARG; }
  *out = g->lattice_ok ? (g->cvia ? 2 : 1) : 0;
  return ORSP_OK;
}
