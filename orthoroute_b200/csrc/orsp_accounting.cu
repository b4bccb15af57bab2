// Edge accounting: cost update, present EMA, history update, overuse count,
// usage commit and path -> edge mapping.
//
// Every floating-point step is written with explicit round-to-nearest
// intrinsics (__fmul_rn / __fadd_rn / __fdiv_rn), so the compiler cannot fuse
// a multiply and an add into an FMA: each kernel reproduces, bit for bit, the
// float32 numpy expression of the reference function it replaces (numpy >= 2
// keeps Python-float scalars "weak", so every operand is rounded to float32).
#include <algorithm>

#include "accounting.cuh"

namespace {

using orsp::apply_usage;
using orsp::live_cost;

inline int grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32));
}

// EdgeAccountant.update_costs (UPF:973-1043).
__global__ void update_costs_kernel(int64_t E, const float *__restrict__ base,
                                    const float *__restrict__ ema,
                                    const float *__restrict__ cap,
                                    const float *__restrict__ hist,
                                    const uint8_t *__restrict__ layer,
                                    const uint8_t *__restrict__ kind,
                                    const float *__restrict__ lbias, float pres_fac,
                                    float hist_w, float via_mult, float base_w,
                                    int jitter, float *__restrict__ out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += stride) {
    // over = xp.maximum(0, present_ema - capacity)
    float over = __fsub_rn(ema[e], cap[e]);
    over = over > 0.0f ? over : 0.0f;
    float adjusted = __fmul_rn(__fmul_rn(base[e], via_mult), base_w);
    float present_term;
    if (lbias) {
      // per_edge_bias = where(edge_kind == 0, layer_bias[edge_layer], 1.0)
      const bool planar = kind[e] == 0;
      const float peb = planar ? lbias[layer[e]] : 1.0f;
      adjusted = __fmul_rn(adjusted, peb);
      // inverted = where(peb != 0, 1/maximum(peb, 0.5), 1); where(kind==0, inv, 1)
      float inv = 1.0f;
      if (planar && peb != 0.0f) inv = __fdiv_rn(1.0f, peb > 0.5f ? peb : 0.5f);
      present_term = __fmul_rn(__fmul_rn(pres_fac, inv), over);
    } else {
      adjusted = __fmul_rn(adjusted, 1.0f);
      present_term = __fmul_rn(pres_fac, over);
    }
    float total = __fadd_rn(__fadd_rn(adjusted, present_term), __fmul_rn(hist_w, hist[e]));
    if (jitter) {
      // xp.arange(E, dtype=float32) % 9973 * 1e-6: the index is first rounded
      // to float32 (exact below 2^24), the remainder is exact.
      const float fi = __ll2float_rn(e);
      total = __fadd_rn(total, __fmul_rn(fmodf(fi, 9973.0f), 1e-6f));
    }
    out[e] = total;
  }
}

__global__ void live_costs_kernel(int64_t n, const int32_t *__restrict__ edges, const float *__restrict__ base,
                                  const int32_t *__restrict__ usage, const float *__restrict__ cap,
                                  const float *__restrict__ hist, float pres_fac, float hist_w,
                                  float via_mult, float base_w, int jitter, float *__restrict__ out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int64_t e = edges ? (int64_t)edges[i] : i;
    if (e < 0) continue;
    out[e] = live_cost(e, base, usage, cap, hist, pres_fac, hist_w, via_mult, base_w, jitter);
  }
}

// Same over the paths of a batch (path_len[k]-1 edges of row k).
__global__ void live_costs_paths_kernel(int32_t K, const int32_t *__restrict__ pe,
                                        const int32_t *__restrict__ plen, int32_t cap_row,
                                        const float *__restrict__ base, const int32_t *__restrict__ usage,
                                        const float *__restrict__ cap, const float *__restrict__ hist,
                                        float pres_fac, float hist_w, float via_mult, float base_w,
                                        int jitter, float *__restrict__ out) {
  for (int32_t k = blockIdx.x; k < K; k += gridDim.x) {
    const int32_t len = plen[k];
    if (len < 2) continue;
    const int32_t ne = min(len - 1, cap_row);
    for (int32_t i = threadIdx.x; i < ne; i += blockDim.x) {
      const int32_t e = pe[(int64_t)k * cap_row + i];
      if (e >= 0) out[e] = live_cost(e, base, usage, cap, hist, pres_fac, hist_w, via_mult, base_w, jitter);
    }
  }
}

// EdgeAccountant.update_present_ema (UPF:963-971).
__global__ void ema_kernel(int64_t E, const float *__restrict__ present,
                           float *__restrict__ ema, float beta, float omb) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += stride)
    ema[e] = __fadd_rn(__fmul_rn(beta, present[e]), __fmul_rn(omb, ema[e]));
}

// EdgeAccountant.update_history (UPF:898-961).
__global__ void history_kernel(int64_t E, float *__restrict__ hist,
                               const float *__restrict__ present,
                               const float *__restrict__ cap,
                               const float *__restrict__ base, float gain,
                               float cap_mult, float decay) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += stride) {
    float h = __fmul_rn(hist[e], decay);
    float over = __fsub_rn(present[e], cap[e]);
    over = over > 0.0f ? over : 0.0f;
    float inc = __fmul_rn(gain, over);
    if (base) {
      const float hc = __fmul_rn(cap_mult, base[e]);
      inc = inc < hc ? inc : hc;  // xp.minimum (no NaNs here)
    }
    hist[e] = __fadd_rn(h, inc);
  }
}

// EdgeAccountant.compute_overuse (UPF:838-876), edge part.
__global__ void overuse_kernel(int64_t E, const float *__restrict__ present,
                               const float *__restrict__ cap,
                               double *__restrict__ acc_sum,
                               unsigned long long *__restrict__ acc_cnt) {
  double s = 0.0;
  unsigned long long c = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += stride) {
    float over = __fsub_rn(present[e], cap[e]);
    if (over > 0.0f) {
      s += (double)over;
      ++c;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(ORSP_FULL_MASK, s, o);
    c += __shfl_xor_sync(ORSP_FULL_MASK, c, o);
  }
  __shared__ double ss[32];
  __shared__ unsigned long long sc[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { ss[w] = s; sc[w] = c; }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    s = lane < nw ? ss[lane] : 0.0;
    c = lane < nw ? sc[lane] : 0ull;
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(ORSP_FULL_MASK, s, o);
      c += __shfl_xor_sync(ORSP_FULL_MASK, c, o);
    }
    if (lane == 0) {
      atomicAdd(acc_sum, s);
      atomicAdd(acc_cnt, c);
    }
  }
}

__global__ void overuse_finish_kernel(const double *acc_sum,
                                      const unsigned long long *acc_cnt,
                                      int64_t *out2) {
  out2[0] = (int64_t)(*acc_sum);  // int() truncation
  out2[1] = (int64_t)(*acc_cnt);
}

__global__ void present_from_usage_kernel(int64_t E, const int32_t *__restrict__ usage,
                                          float *__restrict__ present) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += stride)
    present[e] = (float)usage[e];
}


__global__ void commit_kernel(int64_t n, const int32_t *__restrict__ edges,
                              int32_t *__restrict__ usage, float *__restrict__ present,
                              int32_t sign) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int32_t e = edges[i];
    if (e >= 0) apply_usage(usage, present, e, sign);
  }
}

// Paths of a batched search: path_len[k] nodes give path_len[k]-1 edges.
__global__ void commit_batch_kernel(int32_t K, const int32_t *__restrict__ pe,
                                    const int32_t *__restrict__ plen, int32_t cap,
                                    int32_t *__restrict__ usage, float *__restrict__ present,
                                    int32_t sign) {
  for (int32_t k = blockIdx.x; k < K; k += gridDim.x) {
    const int32_t len = plen[k];
    if (len < 2) continue;
    const int32_t ne = min(len - 1, cap);
    for (int32_t i = threadIdx.x; i < ne; i += blockDim.x) {
      const int32_t e = pe[(int64_t)k * cap + i];
      if (e >= 0) apply_usage(usage, present, e, sign);
    }
  }
}

// _path_to_edges (UPF:5463-5476): first CSR edge u->v per consecutive pair;
// pairs without an edge produce -1 and are compacted away on the host side of
// the call (see orsp_path_to_edges).
__global__ void path_to_edges_kernel(const int32_t *__restrict__ indptr,
                                     const int32_t *__restrict__ indices,
                                     const int32_t *__restrict__ path, int32_t len,
                                     int32_t N, int32_t *__restrict__ out) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i + 1 < len;
       i += gridDim.x * blockDim.x) {
    const int32_t u = path[i], v = path[i + 1];
    int32_t found = -1;
    if (u >= 0 && u < N) {
      for (int32_t k = indptr[u]; k < indptr[u + 1]; ++k)
        if (indices[k] == v) { found = k; break; }
    }
    out[i] = found;
  }
}

__global__ void compact_edges_kernel(int32_t *edges, int32_t n, int32_t *count) {
  // single warp: stable in-place compaction of the >= 0 entries
  const int lane = threadIdx.x;
  int32_t w = 0;
  for (int32_t b = 0; b < n; b += 32) {
    const int32_t i = b + lane;
    const int32_t v = i < n ? edges[i] : -1;
    const unsigned m = __ballot_sync(ORSP_FULL_MASK, v >= 0);
    __syncwarp();
    if (v >= 0) edges[w + __popc(m & lanemask_lt())] = v;
    w += __popc(m);
    __syncwarp();
  }
  if (lane == 0) *count = w;
}

}  // namespace

using namespace orsp;

extern "C" int orsp_update_costs(int64_t E, const float *base, const float *ema,
                                 const float *cap, const float *hist,
                                 const uint8_t *layer, const uint8_t *kind,
                                 const float *lbias, float pres_fac, float hist_w,
                                 float via_mult, float base_w, int add_jitter,
                                 float *out, uintptr_t stream) {
  if (E < 0 || (E > 0 && (!base || !ema || !cap || !hist || !out))) {
    set_error("update_costs: NULL array");
    return ORSP_ERR_ARG;
  }
  const bool has_bias = lbias || layer || kind;
  if (has_bias && !(lbias && layer && kind)) {
    set_error("update_costs: layer_bias, edge_layer and edge_kind go together");
    return ORSP_ERR_ARG;
  }
  if (E == 0) return ORSP_OK;
  update_costs_kernel<<<grid_for(E), 256, 0, (cudaStream_t)stream>>>(
      E, base, ema, cap, hist, layer, kind, lbias, pres_fac, hist_w, via_mult,
      base_w, add_jitter, out);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_update_present_ema(int64_t E, const float *present, float *ema,
                                       float beta, float omb, uintptr_t stream) {
  if (E < 0 || (E > 0 && (!present || !ema))) { set_error("ema: NULL array"); return ORSP_ERR_ARG; }
  if (E == 0) return ORSP_OK;
  ema_kernel<<<grid_for(E), 256, 0, (cudaStream_t)stream>>>(E, present, ema, beta, omb);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_update_history(int64_t E, float *hist, const float *present,
                                   const float *cap, const float *base, float gain,
                                   float cap_mult, float decay, uintptr_t stream) {
  if (E < 0 || (E > 0 && (!hist || !present || !cap))) { set_error("history: NULL array"); return ORSP_ERR_ARG; }
  if (E == 0) return ORSP_OK;
  history_kernel<<<grid_for(E), 256, 0, (cudaStream_t)stream>>>(E, hist, present, cap, base,
                                                               gain, cap_mult, decay);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

namespace orsp {
// Overuse into a caller-visible device int64[2]; the accumulators live in a
// small per-device buffer owned by this translation unit.
int overuse_into(int64_t E, const float *present, const float *cap, int64_t *out2,
                 void *acc, cudaStream_t st) {
  ORSP_CUDA(cudaMemsetAsync(acc, 0, 16, st));
  if (E > 0) {
    overuse_kernel<<<grid_for(E), 256, 0, st>>>(E, present, cap, (double *)acc,
                                                (unsigned long long *)((char *)acc + 8));
    ORSP_CUDA(cudaGetLastError());
  }
  overuse_finish_kernel<<<1, 1, 0, st>>>((const double *)acc,
                                         (const unsigned long long *)((char *)acc + 8), out2);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}
}  // namespace orsp

extern "C" int orsp_overuse(int64_t E, const float *present, const float *cap,
                            int64_t *out2_d, int64_t *out2_h, uintptr_t stream) {
  if (E < 0 || !out2_d || (E > 0 && (!present || !cap))) { set_error("overuse: NULL array"); return ORSP_ERR_ARG; }
  static thread_local void *acc = nullptr;
  static thread_local int acc_dev = -1;
  int dev = 0;
  ORSP_CUDA(cudaGetDevice(&dev));
  if (!acc || acc_dev != dev) {
    ORSP_CUDA(cudaMalloc(&acc, 16));
    acc_dev = dev;
  }
  cudaStream_t st = (cudaStream_t)stream;
  int rc = overuse_into(E, present, cap, out2_d, acc, st);
  if (rc) return rc;
  if (out2_h) {
    ORSP_CUDA(cudaMemcpyAsync(out2_h, out2_d, 16, cudaMemcpyDeviceToHost, st));
    ORSP_CUDA(cudaStreamSynchronize(st));
  }
  return ORSP_OK;
}

extern "C" int orsp_present_from_usage(int64_t E, const int32_t *usage, float *present,
                                       uintptr_t stream) {
  if (E < 0 || (E > 0 && (!usage || !present))) { set_error("present_from_usage: NULL array"); return ORSP_ERR_ARG; }
  if (E == 0) return ORSP_OK;
  present_from_usage_kernel<<<grid_for(E), 256, 0, (cudaStream_t)stream>>>(E, usage, present);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_commit_edges(int64_t n, const int32_t *edges, int32_t *usage,
                                 float *present, int32_t sign, uintptr_t stream) {
  if (n < 0 || (n > 0 && (!edges || !usage))) { set_error("commit: NULL array"); return ORSP_ERR_ARG; }
  if (sign != 1 && sign != -1) { set_error("commit: sign must be +1 or -1"); return ORSP_ERR_ARG; }
  if (n == 0) return ORSP_OK;
  commit_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(n, edges, usage, present, sign);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_commit_batch(int32_t K, const int32_t *pe, const int32_t *plen,
                                 int32_t cap, int32_t *usage, float *present,
                                 int32_t sign, uintptr_t stream) {
  if (K < 0 || cap <= 0 || (K > 0 && (!pe || !plen || !usage))) { set_error("commit_batch: bad args"); return ORSP_ERR_ARG; }
  if (sign != 1 && sign != -1) { set_error("commit_batch: sign must be +1 or -1"); return ORSP_ERR_ARG; }
  if (K == 0) return ORSP_OK;
  commit_batch_kernel<<<std::min(K, 148 * 8), 128, 0, (cudaStream_t)stream>>>(K, pe, plen, cap,
                                                                               usage, present, sign);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_path_to_edges(orsp_graph *g, const int32_t *path, int32_t len,
                                  int32_t *edges_out, int32_t *count_h, uintptr_t stream) {
  if (!g || len < 0 || (len > 1 && (!path || !edges_out)) || !count_h) {
    set_error("path_to_edges: bad args");
    return ORSP_ERR_ARG;
  }
  *count_h = 0;
  if (len < 2) return ORSP_OK;
  ORSP_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = (cudaStream_t)stream;
  path_to_edges_kernel<<<(len + 255) / 256, 256, 0, st>>>(g->indptr, g->indices, path, len,
                                                          g->N, edges_out);
  ORSP_CUDA(cudaGetLastError());
  int32_t *cnt_d = nullptr;
  int rc = ensure_scratch(g, 64);
  if (rc) return rc;
  cnt_d = (int32_t *)g->scratch;
  compact_edges_kernel<<<1, 32, 0, st>>>(edges_out, len - 1, cnt_d);
  ORSP_CUDA(cudaGetLastError());
  ORSP_CUDA(cudaMemcpyAsync(g->pinned, cnt_d, 4, cudaMemcpyDeviceToHost, st));
  ORSP_CUDA(cudaStreamSynchronize(st));
  *count_h = *(int32_t *)g->pinned;
  return ORSP_OK;
}

extern "C" int orsp_update_costs_live(int64_t E, const int32_t *edges, int64_t n_edges,
                                      const float *base, const int32_t *usage, const float *cap,
                                      const float *hist, float pres_fac, float hist_w, float via_mult,
                                      float base_w, int add_jitter, float *out, uintptr_t stream) {
  if (E < 0 || !base || !usage || !cap || !hist || !out || (edges && n_edges < 0)) {
    set_error("update_costs_live: NULL array or bad size");
    return ORSP_ERR_ARG;
  }
  const int64_t n = edges ? n_edges : E;
  if (n == 0) return ORSP_OK;
  live_costs_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(n, edges, base, usage, cap, hist, pres_fac,
                                                                  hist_w, via_mult, base_w, add_jitter, out);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_update_costs_live_paths(int32_t K, const int32_t *pe, const int32_t *plen, int32_t cap_row,
                                            const float *base, const int32_t *usage, const float *cap,
                                            const float *hist, float pres_fac, float hist_w, float via_mult,
                                            float base_w, int add_jitter, float *out, uintptr_t stream) {
  if (K < 0 || cap_row <= 0 || (K > 0 && (!pe || !plen || !base || !usage || !cap || !hist || !out))) {
    set_error("update_costs_live_paths: bad args");
    return ORSP_ERR_ARG;
  }
  if (K == 0) return ORSP_OK;
  live_costs_paths_kernel<<<std::min(K, 148 * 8), 128, 0, (cudaStream_t)stream>>>(
      K, pe, plen, cap_row, base, usage, cap, hist, pres_fac, hist_w, via_mult, base_w, add_jitter, out);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}
