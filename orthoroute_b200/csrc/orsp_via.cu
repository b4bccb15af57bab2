// Via pooling terms of the edge costs: column / segment usage from committed
// paths, their smoothed present cost and z-prefix, the pooling penalties added
// to via-edge costs and the hard block of via edges at capacity.
//
// Restates, on the device:
//   _accumulate_via_usage_for_path   UPF:2678-2724  (usage part)
//   the via present smoothing        UPF:3622-3633  (inline in _pathfinder_negotiation)
//   _apply_via_pooling_penalties     UPF:3243-3387  (vectorised CPU path, UPF:3296-3380)
//   _block_via_edges_with_collisions UPF:3448-3546  (CPU path, UPF:3499-3546)
// (UPF = orthoroute/algorithms/manhattan/unified_pathfinder.py).  Arrays keep
// the reference's [Nx][Ny] / [Nx][Ny][segZ] C order (x-major); usage and
// capacities are int32 here (the reference uses int16 / int8).  Via edges are
// found from the CSR (source and target on different layers), with
// z_lo/z_hi clamped to the routing layers 1..Nz-2 as _build_via_edge_metadata
// does (UPF:5449-5451).  Float steps follow the numpy expressions' order with
// explicit round-to-nearest intrinsics.
#include <algorithm>

#include "common.cuh"

namespace {

inline int grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32));
}

struct Dims {
  int32_t nx, ny, nz, segz;
};

__device__ __forceinline__ void coords(const Dims &d, int32_t n, int32_t &x, int32_t &y, int32_t &z) {
  const int32_t plane = d.nx * d.ny;
  z = n / plane;
  const int32_t r = n - z * plane;
  y = r / d.nx;
  x = r - y * d.nx;
}

__device__ __forceinline__ int32_t clampi(int32_t v, int32_t lo, int32_t hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

// Paths of a batch: path_len[k] nodes in row k.
__global__ void via_usage_kernel(Dims d, int32_t K, const int32_t *__restrict__ nodes,
                                 const int32_t *__restrict__ plen, int32_t cap, int32_t *__restrict__ col_use,
                                 int32_t *__restrict__ seg_use) {
  for (int32_t k = blockIdx.x; k < K; k += gridDim.x) {
    const int32_t len = min(plen[k], cap);
    for (int32_t i = threadIdx.x; i + 1 < len; i += blockDim.x) {
      const int32_t u = nodes[(int64_t)k * cap + i], v = nodes[(int64_t)k * cap + i + 1];
      int32_t xu, yu, zu, xv, yv, zv;
      coords(d, u, xu, yu, zu);
      coords(d, v, xv, yv, zv);
      if (xu != xv || yu != yv || zu == zv) continue;
      const int64_t col = (int64_t)xu * d.ny + yu;
      if (col_use) atomicAdd(&col_use[col], 1);
      if (seg_use && d.segz > 0) {
        const int32_t zl = clampi(min(zu, zv), 1, d.nz - 2), zh = clampi(max(zu, zv), 1, d.nz - 2);
        for (int32_t z = zl; z < zh; ++z) {
          const int32_t s = z - 1;
          if (s >= 0 && s < d.segz) atomicAdd(&seg_use[col * d.segz + s], 1);
        }
      }
    }
  }
}

// pres = alpha*max(0, use - cap) + beta*pres; for segments also the running
// float32 sum along z (np.cumsum(..., axis=2)).
__global__ void via_present_kernel(int64_t ncol, int32_t segz, const int32_t *__restrict__ col_use,
                                   const int32_t *__restrict__ col_cap, float *__restrict__ col_pres,
                                   const int32_t *__restrict__ seg_use, const int32_t *__restrict__ seg_cap,
                                   float *__restrict__ seg_pres, float *__restrict__ seg_prefix, float alpha,
                                   float beta) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncol; c += stride) {
    if (col_pres) {
      const int32_t o = col_use[c] - col_cap[c];
      const float over = (float)(o > 0 ? o : 0);
      col_pres[c] = __fadd_rn(__fmul_rn(alpha, over), __fmul_rn(beta, col_pres[c]));
    }
    if (seg_pres) {
      float run = 0.0f;
      for (int32_t s = 0; s < segz; ++s) {
        const int64_t i = c * segz + s;
        const int32_t o = seg_use[i] - seg_cap[i];
        const float over = (float)(o > 0 ? o : 0);
        const float p = __fadd_rn(__fmul_rn(alpha, over), __fmul_rn(beta, seg_pres[i]));
        seg_pres[i] = p;
        run = s == 0 ? p : __fadd_rn(run, p);
        if (seg_prefix) seg_prefix[i] = run;
      }
    }
  }
}

struct PenaltyParams {
  Dims d;
  const int32_t *indptr, *indices;
  int32_t N;
  const float *col_pres, *seg_prefix;
  const double *layer_bias;  // nullptr: no discount
  int bias_f64;              // the reference's layer_bias dtype (1: float64)
  double k;                  // via_hot_layer_discount
  float col_w, seg_w, pres_fac;
  float *total;
};

__global__ void via_penalty_kernel(PenaltyParams p) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < p.N; u += stride) {
    int32_t xu, yu, zu;
    coords(p.d, (int32_t)u, xu, yu, zu);
    const int64_t col = (int64_t)xu * p.d.ny + yu;
    for (int32_t e = p.indptr[u]; e < p.indptr[u + 1]; ++e) {
      const int32_t v = p.indices[e];
      const int32_t zv = v / (p.d.nx * p.d.ny);
      if (zv == zu) continue;
      const int32_t zlo = clampi(min(zu, zv), 1, p.d.nz - 2), zhi = clampi(max(zu, zv), 1, p.d.nz - 2);
      float pen = 0.0f;
      if (p.col_pres) pen = __fadd_rn(pen, __fmul_rn(p.col_w, p.col_pres[col]));
      if (p.seg_prefix) {
        const int32_t hi = zhi - 2, lo = zlo - 2;
        const float ph = (hi >= 0 && hi < p.d.segz) ? p.seg_prefix[col * p.d.segz + hi] : 0.0f;
        const float pl = (lo >= 0 && lo < p.d.segz) ? p.seg_prefix[col * p.d.segz + lo] : 0.0f;
        const float seg = __fmul_rn(__fsub_rn(ph, pl), zhi > zlo ? 1.0f : 0.0f);
        pen = __fadd_rn(pen, __fmul_rn(p.seg_w, seg));
      }
      if (p.layer_bias) {
        const double sb = p.layer_bias[zlo], db = p.layer_bias[zhi];
        if (p.bias_f64) {
          const double disc = (1.0 - p.k * fmax(sb, 0.0)) * (1.0 + (0.5 * p.k) * fmax(db, 0.0));
          pen = __double2float_rn((double)pen * disc);
        } else {
          const float k32 = __double2float_rn(p.k), hk32 = __double2float_rn(0.5 * p.k);
          const float t1 = __fsub_rn(1.0f, __fmul_rn(k32, fmaxf((float)sb, 0.0f)));
          const float t2 = __fadd_rn(1.0f, __fmul_rn(hk32, fmaxf((float)db, 0.0f)));
          pen = __fmul_rn(pen, __fmul_rn(t1, t2));
        }
      }
      if (pen > 0.0f) p.total[e] = __fadd_rn(p.total[e], __fmul_rn(p.pres_fac, pen));
    }
  }
}

struct BlockParams {
  Dims d;
  const int32_t *indptr, *indices;
  int32_t N;
  const int32_t *col_use, *col_cap, *seg_use, *seg_cap;
  float *total;
};

__global__ void via_block_kernel(BlockParams p) {
  const float INF_F = __int_as_float(0x7f800000);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < p.N; u += stride) {
    int32_t xu, yu, zu;
    coords(p.d, (int32_t)u, xu, yu, zu);
    const int64_t col = (int64_t)xu * p.d.ny + yu;
    const bool col_blocked = p.col_use && p.col_use[col] >= p.col_cap[col];
    for (int32_t e = p.indptr[u]; e < p.indptr[u + 1]; ++e) {
      const int32_t v = p.indices[e];
      const int32_t zv = v / (p.d.nx * p.d.ny);
      if (zv == zu) continue;
      bool blocked = col_blocked;
      if (!blocked && p.seg_use) {
        const int32_t zs = clampi(min(zu, zv), 1, p.d.nz - 2), ze = clampi(max(zu, zv), 1, p.d.nz - 2);
        for (int32_t z = zs; z < ze && !blocked; ++z) {
          const int32_t s = z - 1;
          if (s >= 0 && s < p.d.segz && p.seg_use[col * p.d.segz + s] >= p.seg_cap[col * p.d.segz + s])
            blocked = true;
        }
      }
      if (blocked) p.total[e] = INF_F;
    }
  }
}

Dims dims_of(const orsp::Graph *g) {
  Dims d{g->nx, g->ny, g->nz, g->nz - 2 > 0 ? g->nz - 2 : 0};
  return d;
}

}  // namespace

using namespace orsp;

extern "C" int orsp_via_usage(orsp_graph *g, int32_t K, const int32_t *path_nodes_d, const int32_t *path_len_d,
                              int32_t path_cap, int32_t *col_use_d, int32_t *seg_use_d, uintptr_t stream) {
  if (!g || K < 0 || path_cap <= 0 || (K > 0 && (!path_nodes_d || !path_len_d))) {
    set_error("via_usage: bad args");
    return ORSP_ERR_ARG;
  }
  if (g->nx <= 0 || g->nz < 2) { set_error("via_usage: graph has no lattice dims"); return ORSP_ERR_ARG; }
  if (K == 0) return ORSP_OK;
  ORSP_CUDA(cudaSetDevice(g->device));
  via_usage_kernel<<<std::min(K, 148 * 8), 128, 0, (cudaStream_t)stream>>>(dims_of(g), K, path_nodes_d, path_len_d,
                                                                          path_cap, col_use_d, seg_use_d);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_via_present(int64_t ncol, int32_t segz, const int32_t *col_use_d, const int32_t *col_cap_d,
                                float *col_pres_d, const int32_t *seg_use_d, const int32_t *seg_cap_d,
                                float *seg_pres_d, float *seg_prefix_d, float alpha, float beta, uintptr_t stream) {
  if (ncol < 0 || segz < 0 || (col_pres_d && (!col_use_d || !col_cap_d)) ||
      (seg_pres_d && (!seg_use_d || !seg_cap_d))) {
    set_error("via_present: bad args");
    return ORSP_ERR_ARG;
  }
  if (ncol == 0) return ORSP_OK;
  via_present_kernel<<<grid_for(ncol), 256, 0, (cudaStream_t)stream>>>(ncol, segz, col_use_d, col_cap_d, col_pres_d,
                                                                      seg_use_d, seg_cap_d, seg_pres_d,
                                                                      seg_prefix_d, alpha, beta);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_via_penalties(orsp_graph *g, const float *col_pres_d, const float *seg_prefix_d,
                                  const double *layer_bias_d, int bias_f64, double hot_layer_discount,
                                  float col_weight, float seg_weight, float pres_fac, float *total_cost_d,
                                  uintptr_t stream) {
  if (!g || !total_cost_d) { set_error("via_penalties: NULL argument"); return ORSP_ERR_ARG; }
  if (g->nx <= 0 || g->nz < 2) { set_error("via_penalties: graph has no lattice dims"); return ORSP_ERR_ARG; }
  ORSP_CUDA(cudaSetDevice(g->device));
  PenaltyParams p{};
  p.d = dims_of(g);
  p.indptr = g->indptr;
  p.indices = g->indices;
  p.N = g->N;
  p.col_pres = col_pres_d;
  p.seg_prefix = p.d.segz > 0 ? seg_prefix_d : nullptr;
  p.layer_bias = layer_bias_d;
  p.bias_f64 = bias_f64;
  p.k = hot_layer_discount;
  p.col_w = col_weight;
  p.seg_w = seg_weight;
  p.pres_fac = pres_fac;
  p.total = total_cost_d;
  via_penalty_kernel<<<grid_for(g->N), 256, 0, (cudaStream_t)stream>>>(p);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_via_hard_block(orsp_graph *g, const int32_t *col_use_d, const int32_t *col_cap_d,
                                   const int32_t *seg_use_d, const int32_t *seg_cap_d, float *total_cost_d,
                                   uintptr_t stream) {
  if (!g || !total_cost_d || (col_use_d && !col_cap_d) || (seg_use_d && !seg_cap_d)) {
    set_error("via_hard_block: bad args");
    return ORSP_ERR_ARG;
  }
  if (g->nx <= 0 || g->nz < 2) { set_error("via_hard_block: graph has no lattice dims"); return ORSP_ERR_ARG; }
  ORSP_CUDA(cudaSetDevice(g->device));
  BlockParams p{};
  p.d = dims_of(g);
  p.indptr = g->indptr;
  p.indices = g->indices;
  p.N = g->N;
  p.col_use = col_use_d;
  p.col_cap = col_cap_d;
  p.seg_use = p.d.segz > 0 ? seg_use_d : nullptr;
  p.seg_cap = seg_cap_d;
  p.total = total_cost_d;
  via_block_kernel<<<grid_for(g->N), 256, 0, (cudaStream_t)stream>>>(p);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}
