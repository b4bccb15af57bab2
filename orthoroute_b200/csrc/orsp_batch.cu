// Batched box-ROI searches: one persistent launch in which every CTA takes
// searches from a shared work counter and runs each one as a block-local
// near-far delta-stepping loop (__syncthreads rounds instead of grid
// barriers), then backtraces it with one warp and maps the path to CSR edges.
//
// Replaces, for box ROIs, the per-net body of PathFinderRouter._route_all
// (UPF:4475-4800: ROI -> find_path_roi -> _path_to_edges) and the batched
// CUDADijkstra.find_paths_on_rois (CD:2014-2086).  Costs are read-only for the
// whole launch, which is what the reference guarantees inside one negotiation
// iteration (total_cost is computed once per iteration, UPF:3724-3732, and
// _route_all reads it once, UPF:4459), so every search of the batch returns
// the path the sequential loop would return for that net.
//
// Distances of boxes with at most `smem_nodes` nodes live in shared memory;
// larger boxes use a per-CTA slot in global memory (L2-resident for the
// working set).  Searches whose work queues overflow are reported with
// path_len = -2 and are re-run by the host wrapper with larger queues.
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <vector>

#include "common.cuh"
#include "fastdiv.cuh"
#include "lattice_walk.cuh"

namespace {

constexpr int BATCH_THREADS = 512;

// per-search status in path_len (< 0)
constexpr int ST_ARG = -1;
constexpr int ST_QUEUE = -2;
constexpr int ST_PATHCAP = -3;
constexpr int ST_ROUNDS = -4;
constexpr int ST_INTERNAL = -5;

struct BatchParams {
  const int32_t *indptr, *indices, *rptr, *rsrc, *reid;
  const float *cost;
  int32_t nx, ny, nz;
  FastDiv div_nx, div_plane;
  int32_t K;
  const int32_t *src, *dst, *bbox, *order;
  int range_mode;  // 1: bbox holds [lo, hi) node ranges (2 per search) instead of boxes;
                   // 2: one node-set ROI, ids through roi_map / roi_nodes
  const int32_t *roi_map;    // mode 2: global_to_roi (-1 outside)
  const int32_t *roi_nodes;  // mode 2: the ROI's nodes by ROI index
  int32_t n_roi;
  int32_t *path_nodes, *path_edges, *path_len;
  int32_t path_cap;
  char *ws;
  size_t slot_bytes;
  int64_t qcap;
  int32_t smem_nodes;
  float delta;
  const float *delta_d;  // device bucket width (overrides delta) or nullptr
  const float *delta_k;  // per-search bucket width (> 0 overrides the above) or nullptr
  unsigned *work_counter;
  unsigned long long budget_ns;
};

// A search's ROI: an inclusive lattice box (local id = row-major position in
// the box), or a node-id range [lo, lo+V) of a graph made of concatenated
// ROI-local CSRs (local id = node - lo).  Both orders follow the global id.
// Or (mapped) a node-set ROI: local id = global_to_roi[node], the ROI index,
// which is also the reference's rank.
struct Box {
  int32_t x0, y0, z0, W, H, D;
  FastDiv dw, dwh;
  int32_t V;
  int32_t lo;    // range mode: first node
  bool range;
  bool mapped;
};

__device__ __forceinline__ bool box_local(const BatchParams &p, const Box &b, int32_t gid,
                                          int32_t *lid) {
  if (b.mapped) {
    const int32_t l = __ldg(&p.roi_map[gid]);
    if (l < 0) return false;
    *lid = l;
    return true;
  }
  if (b.range) {
    if (gid < b.lo || gid - b.lo >= b.V) return false;
    *lid = gid - b.lo;
    return true;
  }
  const uint32_t z = p.div_plane.div((uint32_t)gid);
  const uint32_t rem = (uint32_t)gid - z * (uint32_t)(p.nx * p.ny);
  const uint32_t y = p.div_nx.div(rem);
  const uint32_t x = rem - y * (uint32_t)p.nx;
  const int32_t lx = (int32_t)x - b.x0, ly = (int32_t)y - b.y0, lz = (int32_t)z - b.z0;
  if (lx < 0 || ly < 0 || lz < 0 || lx >= b.W || ly >= b.H || lz >= b.D) return false;
  *lid = (lz * b.H + ly) * b.W + lx;
  return true;
}

__device__ __forceinline__ int32_t box_global(const BatchParams &p, const Box &b, int32_t lid) {
  if (b.mapped) return __ldg(&p.roi_nodes[lid]);
  if (b.range) return b.lo + lid;
  const uint32_t lz = b.dwh.div((uint32_t)lid);
  const uint32_t r = (uint32_t)lid - lz * (uint32_t)(b.W * b.H);
  const uint32_t ly = b.dw.div(r);
  const uint32_t lx = r - ly * (uint32_t)b.W;
  return ((b.z0 + (int32_t)lz) * p.ny + (b.y0 + (int32_t)ly)) * p.nx + (b.x0 + (int32_t)lx);
}

template <bool SMEM>
__device__ __forceinline__ uint32_t dist_ld(const uint32_t *d, int32_t i) {
  if (SMEM) return *(volatile const uint32_t *)&d[i];
  return __ldcg(&d[i]);
}

struct BlockCtl {
  unsigned qcnt[3];
  unsigned fcnt[4];
  unsigned fmin[4];
  int err;
};

// Block-local near-far search inside one box; same round structure as the
// grid kernel (rotating counters, far generations), with __syncthreads.
// Returns with the final distances of every node with d < d[dst] in `dist`.
template <bool SMEM>
__device__ void block_search(const BatchParams &p, const Box &b, int32_t src_l, int32_t dst_l,
                             uint32_t *dist, int2 *nq0, int2 *nq1, int2 *fq0, int2 *fq1,
                             BlockCtl *c, unsigned long long t_start, float delta) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const float INF_F = __int_as_float(0x7f800000);

  for (int32_t i = threadIdx.x; i < b.V; i += blockDim.x) dist[i] = ORSP_INF_BITS;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 0; i < 3; ++i) c->qcnt[i] = 0;
    for (int i = 0; i < 4; ++i) { c->fcnt[i] = 0; c->fmin[i] = ORSP_INF_BITS; }
    c->err = 0;
    dist[src_l] = 0u;
    fq0[0] = make_int2(src_l, 0);
    c->fcnt[0] = 1;
    c->fmin[0] = 0u;
  }
  __syncthreads();
  const unsigned max_rounds = 4u * (unsigned)b.V + 1024u;
  unsigned r = 0, g = 0;
  float T = 0.0f;
  for (;;) {
    const unsigned n_in = min((unsigned)c->qcnt[r % 3], (unsigned)p.qcap);
    if (n_in > 0) {
      const int2 *inq = ((r & 1) ? nq1 : nq0);
      int2 *outq = (((r + 1) & 1) ? nq1 : nq0);
      int2 *farq = ((g & 1) ? fq1 : fq0);
      unsigned *out_cnt = &c->qcnt[(r + 1) % 3];
      unsigned *far_cnt = &c->fcnt[g % 4];
      for (unsigned base = warp * 32; base < n_in; base += nwarps * 32) {
        const unsigned i = base + lane;
        int beg = 0, end = 0;
        unsigned dbits = 0;
        if (i < n_in) {
          const int2 it = __ldcg(&inq[i]);
          if (dist_ld<SMEM>(dist, it.x) == (unsigned)it.y) {
            const int32_t gv = box_global(p, b, it.x);
            beg = __ldg(&p.indptr[gv]);
            end = __ldg(&p.indptr[gv + 1]);
            dbits = (unsigned)it.y;
          }
        }
        const int deg = end - beg;
        const int maxdeg = __reduce_max_sync(ORSP_FULL_MASK, deg);
        const float d = bits_f(dbits);
        unsigned fmin_local = ORSP_INF_BITS;
        for (int k = 0; k < maxdeg; ++k) {
          bool pn = false, pf = false;
          int2 item = make_int2(0, 0);
          if (k < deg) {
            const int e = beg + k;
            const int32_t w = __ldg(&p.indices[e]);
            int32_t lw;
            if (box_local(p, b, w, &lw)) {
              const float nd = __fadd_rn(d, __ldg(&p.cost[e]));
              if (nd < INF_F) {
                const unsigned nb = f_bits(nd);
                if (nb < dist_ld<SMEM>(dist, lw)) {
                  const unsigned old = atomicMin(&dist[lw], nb);
                  if (nb < old) {
                    item = make_int2(lw, (int)nb);
                    if (nd < T) pn = true; else pf = true;
                  }
                }
              }
            }
          }
          warp_append(outq, out_cnt, p.qcap, pn, item, &c->err);
          warp_append(farq, far_cnt, p.qcap, pf, item, &c->err);
          if (pf && (unsigned)item.y < fmin_local) fmin_local = (unsigned)item.y;
        }
        const unsigned wm = warp_min_u32(fmin_local);
        if (lane == 0 && wm != ORSP_INF_BITS) atomicMin(&c->fmin[g % 4], wm);
      }
    } else {
      const unsigned fc = min((unsigned)c->fcnt[g % 4], (unsigned)p.qcap);
      if (fc == 0) break;
      if (bits_f(dist_ld<SMEM>(dist, dst_l)) < T) break;
      const float fm = bits_f(c->fmin[g % 4]);
      float Tn = __fadd_rn(fm, delta);
      if (!(Tn > fm)) Tn = __uint_as_float(f_bits(fm) + 1u);
      const int2 *fin = ((g & 1) ? fq1 : fq0);
      int2 *fout = (((g + 1) & 1) ? fq1 : fq0);
      int2 *outq = (((r + 1) & 1) ? nq1 : nq0);
      for (unsigned base = warp * 32; base < fc; base += nwarps * 32) {
        const unsigned i = base + lane;
        bool pn = false, pf = false;
        int2 it = make_int2(0, 0);
        if (i < fc) {
          it = __ldcg(&fin[i]);
          if (dist_ld<SMEM>(dist, it.x) == (unsigned)it.y) {
            if (bits_f((unsigned)it.y) < Tn) pn = true; else pf = true;
          }
        }
        warp_append(outq, &c->qcnt[(r + 1) % 3], p.qcap, pn, it, &c->err);
        warp_append(fout, &c->fcnt[(g + 1) % 4], p.qcap, pf, it, &c->err);
        const unsigned wm = warp_min_u32(pf ? (unsigned)it.y : ORSP_INF_BITS);
        if (lane == 0 && wm != ORSP_INF_BITS) atomicMin(&c->fmin[(g + 1) % 4], wm);
      }
      if (threadIdx.x == 0) {
        c->fcnt[(g + 2) % 4] = 0;
        c->fmin[(g + 2) % 4] = ORSP_INF_BITS;
      }
      T = Tn;
      ++g;
    }
    if (threadIdx.x == 0) {
      c->qcnt[(r + 2) % 3] = 0;
      if (r + 1 >= max_rounds || dev_globaltimer() - t_start > p.budget_ns)
        atomicCAS(&c->err, DEV_OK, DEV_ERR_TIMEOUT);
    }
    __syncthreads();
    if (c->err) break;
    ++r;
  }
  __syncthreads();
}

// One warp: parent walk with the settle-order tie-break, fused with the
// first-CSR-edge lookup of _path_to_edges.  Output in src -> dst order.
template <bool SMEM>
__device__ int block_backtrace(const BatchParams &p, const Box &b, int32_t src, int32_t dst,
                               int32_t dst_l, const uint32_t *dist, int32_t *nodes,
                               int32_t *edges) {
  const int lane = threadIdx.x & 31;
  unsigned dv = dist_ld<SMEM>(dist, dst_l);
  if (dv == ORSP_INF_BITS) return 0;
  int32_t v = dst, lv = dst_l;
  int len = 0;
  for (;;) {
    if (len >= p.path_cap) return ST_PATHCAP;
    if (lane == 0) nodes[len] = v;
    ++len;
    if (v == src) break;
    const int kb = __ldg(&p.rptr[v]), ke = __ldg(&p.rptr[v + 1]);
    unsigned long long best = ULLONG_MAX;
    int32_t bu = -1;
    for (int k0 = kb; k0 < ke; k0 += 32) {
      const int k = k0 + lane;
      if (k < ke) {
        const int32_t u = __ldg(&p.rsrc[k]);
        int32_t lu;
        if (box_local(p, b, u, &lu)) {
          const unsigned du = dist_ld<SMEM>(dist, lu);
          if (du != ORSP_INF_BITS) {
            const float s = __fadd_rn(bits_f(du), __ldg(&p.cost[__ldg(&p.reid[k])]));
            if (f_bits(s) == dv && (du < dv || (du == dv && lu < lv))) {
              const unsigned long long key = ((unsigned long long)du << 32) | (unsigned)lu;
              if (key < best) { best = key; bu = u; }
            }
          }
        }
      }
    }
    const unsigned long long wbest = warp_min_u64(best);
    if (wbest == ULLONG_MAX) return ST_INTERNAL;
    const unsigned owner = __ballot_sync(ORSP_FULL_MASK, best == wbest && bu >= 0);
    const int32_t u = __shfl_sync(ORSP_FULL_MASK, bu, __ffs(owner) - 1);
    // first CSR edge u -> v: the smallest forward edge id among in-edges from u
    int32_t emin = INT_MAX;
    for (int k0 = kb; k0 < ke; k0 += 32) {
      const int k = k0 + lane;
      if (k < ke && __ldg(&p.rsrc[k]) == u) emin = min(emin, __ldg(&p.reid[k]));
    }
    emin = __reduce_min_sync(ORSP_FULL_MASK, emin);
    if (edges && lane == 0 && len - 1 < p.path_cap) edges[len - 1] = emin;
    v = u;
    lv = (int32_t)(wbest & 0xffffffffu);
    dv = (unsigned)(wbest >> 32);
  }
  __syncwarp();
  for (int i = lane; i < len / 2; i += 32) {
    const int32_t a = nodes[i], z = nodes[len - 1 - i];
    nodes[i] = z;
    nodes[len - 1 - i] = a;
  }
  if (edges) {
    const int ne = len - 1;
    for (int i = lane; i < ne / 2; i += 32) {
      const int32_t a = edges[i], z = edges[ne - 1 - i];
      edges[i] = z;
      edges[ne - 1 - i] = a;
    }
  }
  __syncwarp();
  return len;
}

__global__ void __launch_bounds__(BATCH_THREADS) batch_bbox_kernel(BatchParams p) {
  extern __shared__ uint32_t s_dist[];
  __shared__ BlockCtl ctl;
  __shared__ int s_item;
  const unsigned long long t_start = dev_globaltimer();
  char *slot = p.ws + (size_t)blockIdx.x * p.slot_bytes;
  int2 *q = (int2 *)slot;
  int2 *nq0 = q, *nq1 = q + p.qcap, *fq0 = q + 2 * p.qcap, *fq1 = q + 3 * p.qcap;
  uint32_t *gdist = (uint32_t *)(slot + (size_t)4 * p.qcap * sizeof(int2));
  for (;;) {
    if (threadIdx.x == 0) s_item = (int)atomicAdd(p.work_counter, 1u);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= p.K) break;
    const int k = p.order ? p.order[it] : it;
    Box b;
    b.mapped = false;
    if (p.range_mode == 2) {
      b.mapped = true;
      b.range = false;
      b.lo = 0;
      b.V = p.n_roi;
      b.x0 = b.y0 = b.z0 = 0;
      b.W = b.V;
      b.H = b.D = 1;
      b.dw.init(1u);
      b.dwh.init(1u);
    } else if (p.range_mode) {
      const int32_t *rg = p.bbox + 2 * (int64_t)k;
      b.range = true;
      b.lo = rg[0];
      b.V = rg[1] - rg[0];
      b.x0 = b.y0 = b.z0 = 0;
      b.W = b.V;
      b.H = b.D = 1;
      b.dw.init(1u);
      b.dwh.init(1u);
    } else {
      const int32_t *bb = p.bbox + 6 * (int64_t)k;
      b.range = false;
      b.lo = 0;
      b.x0 = bb[0];
      b.y0 = bb[2];
      b.z0 = bb[4];
      b.W = bb[1] - bb[0] + 1;
      b.H = bb[3] - bb[2] + 1;
      b.D = bb[5] - bb[4] + 1;
      b.V = b.W * b.H * b.D;
      b.dw.init((uint32_t)b.W);
      b.dwh.init((uint32_t)(b.W * b.H));
    }
    const int32_t src = p.src[k], dst = p.dst[k];
    int32_t src_l = -1, dst_l = -1;
    int32_t *nodes = p.path_nodes + (int64_t)k * p.path_cap;
    int32_t *edges = p.path_edges ? p.path_edges + (int64_t)k * p.path_cap : nullptr;
    const bool ok = src >= 0 && dst >= 0 && box_local(p, b, src, &src_l) &&
                    box_local(p, b, dst, &dst_l);
    if (!ok) {
      if (threadIdx.x == 0) p.path_len[k] = ST_ARG;
      continue;
    }
    const bool use_smem = b.V <= p.smem_nodes;
    uint32_t *dist = use_smem ? s_dist : gdist;
    const float dk = p.delta_k ? p.delta_k[k] : 0.0f;
    const float delta = dk > 0.0f ? dk : (p.delta_d ? *p.delta_d : p.delta);
    if (use_smem)
      block_search<true>(p, b, src_l, dst_l, dist, nq0, nq1, fq0, fq1, &ctl, t_start, delta);
    else
      block_search<false>(p, b, src_l, dst_l, dist, nq0, nq1, fq0, fq1, &ctl, t_start, delta);
    int status;
    if (ctl.err == DEV_ERR_OVERFLOW) status = ST_QUEUE;
    else if (ctl.err) status = ST_ROUNDS;
    else status = 0;
    if (threadIdx.x < 32) {
      int len = status;
      if (status == 0) {
        len = use_smem ? block_backtrace<true>(p, b, src, dst, dst_l, dist, nodes, edges)
                       : block_backtrace<false>(p, b, src, dst, dst_l, dist, nodes, edges);
      }
      if (threadIdx.x == 0) p.path_len[k] = len;
    }
    __syncthreads();
  }
}

int env_int(const char *name, int dflt) {
  const char *s = getenv(name);
  if (!s || !*s) return dflt;
  return atoi(s);
}

// Backtrace of the searches done by tile sweeps with their own distance
// slices: one warp per search (block j: item[j], box boxes[j]).  The warp
// walks with lat_walk_warp (the parent rule of block_backtrace), reading distances from the box's slice (box-local row-major order,
// which is the node-id order, so the ranks agree); then the lanes reverse the
// path and map each step u -> v to the in-edge of v in u's slot (the first CSR
// edge u -> v: the lattice has no parallel edges).  Same status codes as
// block_backtrace.
struct LatBt {
  const float4 *w4;         // gathered in-edge weights (fresh inside the boxes)
  const int32_t *slot_eid;  // [4][N] in-edge id per slot
  const int32_t *vcol_eid;  // column vias: [2][nz][N] via in-edge ids by source layer (NULL: none)
  int64_t N;
  const uint32_t *dist;  // slice arena
  orsp::LatWalkGeom geom;
  const orsp::LatBox *boxes;
  const int32_t *item, *src, *dst;  // per box: search id, source, target (global ids)
  int32_t *path_nodes, *path_edges, *path_len;
  int32_t path_cap;
  const int *search_err;
};

__device__ __forceinline__ bool lat_in_box(const orsp::LatBox &B, int32_t x, int32_t y, int32_t z) {
  return x >= B.x0 && x <= B.x1 && y >= B.y0 && y <= B.y1 && z >= B.z0 && z <= B.z1;
}

__global__ void lat_batch_backtrace_kernel(LatBt p) {
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x;
  const int32_t k = p.item[j];
  const orsp::LatBox B = p.boxes[j];
  const int32_t src = p.src[j], dst = p.dst[j];
  int32_t *nodes = p.path_nodes + (int64_t)k * p.path_cap;
  int32_t *edges = p.path_edges ? p.path_edges + (int64_t)k * p.path_cap : nullptr;
  const int64_t N = (int64_t)p.geom.nx * p.geom.ny * p.geom.nz;
  int32_t sx = 0, sy = 0, sz = 0, x = 0, y = 0, z = 0;
  if (src >= 0 && src < N) orsp::lat_xyz(p.geom, src, sx, sy, sz);
  if (dst >= 0 && dst < N) orsp::lat_xyz(p.geom, dst, x, y, z);
  if (src < 0 || dst < 0 || src >= N || dst >= N || !lat_in_box(B, sx, sy, sz) || !lat_in_box(B, x, y, z)) {
    if (lane == 0) p.path_len[k] = ST_ARG;
    return;
  }
  if (*p.search_err) {
    if (lane == 0) p.path_len[k] = ST_ROUNDS;
    return;
  }
  const uint32_t *dist = p.dist + B.dbase;
  const int64_t bw = B.x1 - B.x0 + 1, bh = B.y1 - B.y0 + 1;
  const int32_t bx0 = B.x0, by0 = B.y0, bz0 = B.z0;
  auto dget = [dist, bw, bh, bx0, by0, bz0](int32_t a, int32_t b, int32_t c) {
    return __ldcg(&dist[((int64_t)(c - bz0) * bh + (b - by0)) * bw + (a - bx0)]);
  };
  unsigned dv = dget(x, y, z);
  if (dv == ORSP_INF_BITS) {
    if (lane == 0) p.path_len[k] = 0;
    return;
  }
  auto at_src = [src](int64_t v, unsigned) { return v == src; };
  int len = orsp::lat_walk_warp(p.geom, B, p.w4, dget, at_src, x, y, z, dv, nodes, p.path_cap);
  int status = 0;
  if (len == -1) status = ST_PATHCAP;
  else if (len < 0) status = ST_INTERNAL;
  __syncwarp();
  if (status) {
    if (lane == 0) p.path_len[k] = status;
    return;
  }
  for (int i = lane; i < len / 2; i += 32) {
    const int32_t a = nodes[i], zz = nodes[len - 1 - i];
    nodes[i] = zz;
    nodes[len - 1 - i] = a;
  }
  __syncwarp();
  if (edges) {
    for (int i = lane; i < len - 1; i += 32) {
      const int32_t u = nodes[i], w = nodes[i + 1];
      const int64_t plane = (int64_t)p.geom.nx * p.geom.ny;
      const int64_t zu = u / plane, zw = w / plane;
      if (p.vcol_eid && zu != zw)  // a column via: the first CSR edge u -> w (the smaller id)
        edges[i] = __ldg(&p.vcol_eid[zu * p.N + w]);
      else
        edges[i] = __ldg(&p.slot_eid[(int64_t)orsp::lat_edge_slot(p.geom, u, w) * p.N + w]);
    }
  }
  __syncwarp();
  if (lane == 0) p.path_len[k] = len;
}


}  // namespace

using namespace orsp;

namespace {


int64_t box_volume(const int32_t *b, int range_mode) {
  if (range_mode) return (int64_t)b[1] - b[0];
  return (int64_t)(b[1] - b[0] + 1) * (b[3] - b[2] + 1) * (b[5] - b[4] + 1);
}

int grow_dev(void **p, size_t *have, size_t need) {
  if (*have >= need) return ORSP_OK;
  cudaFree(*p);
  *p = nullptr;
  *have = 0;
  ORSP_CUDA(cudaMalloc(p, need));
  *have = need;
  return ORSP_OK;
}

// Searches `items` with one CTA per search (the block-local near-far kernel),
// in the order given, queue overflows re-run with 4x larger queues.
int run_batch_cta(orsp_graph *g, const float *cost_d, int32_t K, const std::vector<int32_t> &items, const int32_t *src_d,
                  const int32_t *dst_d, const int32_t *bbox_d, const std::vector<int32_t> &bb, int range_mode,
                  float delta, const std::vector<float> &delta_k, int ctas_per_sm, int32_t *path_nodes_d,
                  int32_t *path_edges_d, int32_t path_cap, int32_t *path_len_d, cudaStream_t st,
                  const int32_t *roi_map_d = nullptr, const int32_t *roi_nodes_d = nullptr) {
  const int32_t n = (int32_t)items.size();
  if (n == 0) return ORSP_OK;
  const int per = range_mode ? 2 : 6;
  int64_t vmax = 1;
  for (int32_t k : items) vmax = std::max(vmax, box_volume(&bb[(size_t)per * k], range_mode));
  // device: order (n), retry list (n), per-search widths (K, when given)
  const bool per_k = !delta_k.empty();
  int rc = grow_dev((void **)&g->batch_idx, &g->batch_idx_bytes, (size_t)n * 8 + (per_k ? (size_t)K * 4 : 0) + 256);
  if (rc) return rc;
  int32_t *order_all = g->batch_idx;
  int32_t *retry_d = g->batch_idx + n;
  float *dk_d = per_k ? (float *)(g->batch_idx + 2 * (size_t)n) : nullptr;
  ORSP_CUDA(cudaMemcpyAsync(order_all, items.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st));
  if (per_k) ORSP_CUDA(cudaMemcpyAsync(dk_d, delta_k.data(), (size_t)K * 4, cudaMemcpyHostToDevice, st));

  const int smem_nodes = std::max(0, env_int("ORSP_BATCH_SMEM_NODES", 24 * 1024));
  const size_t smem_bytes = (size_t)smem_nodes * 4;
  ORSP_CUDA(cudaFuncSetAttribute(batch_bbox_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_bytes));
  const size_t ws_budget = (size_t)std::max(1, env_int("ORSP_BATCH_WS_MB", 16384)) << 20;

  // Queue capacity: start at 2 items per node (plenty for lattice wavefronts),
  // grow to the worst case (one item per directed edge) for re-runs.
  int64_t qcap = 2 * vmax + 4096;
  const int64_t qcap_max = (int64_t)std::max(1, g->max_degree) * vmax + 4096;
  BatchParams p{};
  p.indptr = g->indptr;
  p.indices = g->indices;
  p.rptr = g->rptr;
  p.rsrc = g->rsrc;
  p.reid = g->reid;
  p.cost = cost_d;
  p.nx = g->nx;
  p.ny = g->ny;
  p.nz = g->nz;
  p.div_nx.init((uint32_t)std::max(1, g->nx));
  p.div_plane.init((uint32_t)std::max(1, g->nx * g->ny));
  p.src = src_d;
  p.dst = dst_d;
  p.bbox = bbox_d;
  p.range_mode = range_mode;
  p.roi_map = roi_map_d;
  p.roi_nodes = roi_nodes_d;
  p.n_roi = range_mode == 2 ? bb[1] - bb[0] : 0;
  p.path_nodes = path_nodes_d;
  p.path_edges = path_edges_d;
  p.path_len = path_len_d;
  p.path_cap = path_cap;
  p.smem_nodes = smem_nodes;
  p.delta = delta;
  p.delta_d = nullptr;
  p.delta_k = dk_d;
  if (delta == 0.0f) {
    rc = launch_auto_delta(cost_d, g->E, g->auto_delta + 1, st);
    if (rc) return rc;
    p.delta_d = g->auto_delta + 1;
  }
  p.budget_ns = 30ull * 1000000000ull;

  const int32_t *order = order_all;
  int32_t n_items = n;
  std::vector<int32_t> lens, retry, retry_h;
  for (int attempt = 0; attempt < 4; ++attempt) {
    const size_t slot_bytes = (((size_t)4 * qcap * sizeof(int2) + (size_t)vmax * 4) + 255) & ~(size_t)255;
    int nslots = g->num_sms * std::max(1, ctas_per_sm);
    nslots = (int)std::max<size_t>(1, std::min<size_t>((size_t)nslots, ws_budget / slot_bytes));
    nslots = std::min<int>(nslots, n_items);
    const size_t need = slot_bytes * nslots + 256;
    if (g->batch_ws_bytes < need) {
      cudaFree(g->batch_ws);
      g->batch_ws = nullptr;
      g->batch_ws_bytes = 0;
      ORSP_CUDA(cudaMalloc(&g->batch_ws, need));
      g->batch_ws_bytes = need;
    }
    if (!g->batch_ctl) ORSP_CUDA(cudaMalloc(&g->batch_ctl, 256));
    ORSP_CUDA(cudaMemsetAsync(g->batch_ctl, 0, 4, st));
    p.ws = (char *)g->batch_ws;
    p.slot_bytes = slot_bytes;
    p.qcap = qcap;
    p.work_counter = (unsigned *)g->batch_ctl;
    p.K = n_items;
    p.order = order;
    batch_bbox_kernel<<<nslots, BATCH_THREADS, smem_bytes, st>>>(p);
    ORSP_CUDA(cudaGetLastError());

    // Collect queue overflows (of this call's items) for a re-run with larger queues.
    lens.resize((size_t)K);
    ORSP_CUDA(cudaMemcpyAsync(lens.data(), path_len_d, (size_t)K * 4, cudaMemcpyDeviceToHost, st));
    ORSP_CUDA(cudaStreamSynchronize(st));
    retry.clear();
    const std::vector<int32_t> &cur = (attempt == 0) ? items : retry_h;
    for (int32_t k : cur)
      if (lens[k] == ST_QUEUE) retry.push_back(k);
    if (retry.empty() || qcap >= qcap_max) break;
    qcap = std::min(qcap_max, qcap * 4);
    ORSP_CUDA(cudaMemcpyAsync(retry_d, retry.data(), retry.size() * 4, cudaMemcpyHostToDevice, st));
    order = retry_d;
    n_items = (int32_t)retry.size();
    retry_h = retry;
  }
  return ORSP_OK;
}

// Searches `items` (box ROIs) by tile sweeps, many boxes per launch, each box
// with its own distance slice so that boxes may overlap.  Items are taken in
// chunks whose slices fit the arena (ORSP_BATCH_LAT_MB, default 4096 MB).
int run_batch_lat(orsp_graph *g, const float *cost_d, int32_t K, const std::vector<int32_t> &items,
                  const std::vector<int32_t> &bb, const std::vector<int32_t> &src_h,
                  const std::vector<int32_t> &dst_h, int tile_w, int32_t *path_nodes_d, int32_t *path_edges_d,
                  int32_t path_cap, int32_t *path_len_d, cudaStream_t st) {
  (void)K;
  const size_t n = items.size();
  if (n == 0) return ORSP_OK;
  const int64_t arena_cells = ((int64_t)std::max(64, env_int("ORSP_BATCH_LAT_MB", 4096)) << 20) / 4;
  size_t a = 0;
  while (a < n) {
    // chunk [a, b): slices within the arena (a single larger box gets its own chunk)
    size_t b = a;
    int64_t cells = 0;
    while (b < n && b - a < 65536) {
      const int64_t v = box_volume(&bb[(size_t)6 * items[b]], 0);
      if (b > a && cells + v > arena_cells) break;
      cells += v;
      ++b;
    }
    const int32_t m = (int32_t)(b - a);
    int rc = grow_dev((void **)&g->blat_dist, &g->blat_dist_bytes, (size_t)cells * 4 + 256);
    if (rc) return rc;
    // tables: boxes (LatBox), item ids, sources, targets - staged in pinned
    // memory, copied once per chunk; the chunk is synchronised before the
    // staging buffer is reused
    const size_t tab = (size_t)m * sizeof(LatBox) + (size_t)m * 12 + 256;
    if (g->blat_tab_bytes < tab) {
      cudaFree(g->blat_tab_d);
      if (g->blat_tab_h) cudaFreeHost(g->blat_tab_h);
      g->blat_tab_d = nullptr;
      g->blat_tab_h = nullptr;
      g->blat_tab_bytes = 0;
      ORSP_CUDA(cudaMalloc(&g->blat_tab_d, tab));
      ORSP_CUDA(cudaMallocHost(&g->blat_tab_h, tab));
      g->blat_tab_bytes = tab;
    }
    LatBox *hb = (LatBox *)g->blat_tab_h;
    int32_t *h_item = (int32_t *)(hb + m);
    int32_t *h_src = h_item + m;
    int32_t *h_dst = h_src + m;
    std::vector<int32_t> boxes((size_t)m * 6);
    for (int32_t j = 0; j < m; ++j) {
      const int32_t k = items[a + j];
      for (int c = 0; c < 6; ++c) boxes[(size_t)j * 6 + c] = bb[(size_t)6 * k + c];
      h_item[j] = k;
      h_src[j] = src_h[k];
      h_dst[j] = dst_h[k];
    }
    const int64_t ntiles = make_lat_boxes(boxes.data(), m, hb, tile_w);
    int64_t base = 0;
    for (int32_t j = 0; j < m; ++j) {
      hb[j].dbase = base;
      base += box_volume(&boxes[(size_t)j * 6], 0);
    }
    ORSP_CUDA(cudaMemcpyAsync(g->blat_tab_d, g->blat_tab_h, (size_t)m * sizeof(LatBox) + (size_t)m * 12,
                              cudaMemcpyHostToDevice, st));
    const LatBox *db = (const LatBox *)g->blat_tab_d;
    const int32_t *d_item = (const int32_t *)(db + m);
    const int32_t *d_src = d_item + m;
    const int32_t *d_dst = d_src + m;
    rc = reserve_lattice_ws(g, ntiles);
    if (rc) return rc;
    LatOptions opt;
    opt.tile_w = tile_w;
    opt.private_dist = true;
    opt.private_count = cells;
    opt.copy_ctl = false;
    rc = run_lattice_boxes(g, cost_d, m, d_src, nullptr, m, boxes.data(), db, g->blat_dist, st, &opt);
    if (rc) return rc;
    LatBt bt{};
    bt.w4 = (const float4 *)g->wslot;
    bt.slot_eid = g->slot_eid;
    bt.vcol_eid = g->cvia ? g->vcol_eid : nullptr;
    bt.geom.wcol = g->cvia ? g->wcol : nullptr;
    bt.geom.nzp = (g->nz + 3) & ~3;
    bt.N = g->N;
    bt.dist = g->blat_dist;
    bt.geom.nx = g->nx;
    bt.geom.ny = g->ny;
    bt.geom.nz = g->nz;
    for (int z = 0; z < 64; ++z) bt.geom.axis[z] = z < g->nz ? g->layer_axis[z] : 0;
    bt.boxes = db;
    bt.item = d_item;
    bt.src = d_src;
    bt.dst = d_dst;
    bt.path_nodes = path_nodes_d;
    bt.path_edges = path_edges_d;
    bt.path_len = path_len_d;
    bt.path_cap = path_cap;
    bt.search_err = opt.err_d;
    lat_batch_backtrace_kernel<<<m, 32, 0, st>>>(bt);
    ORSP_CUDA(cudaGetLastError());
    ORSP_CUDA(cudaStreamSynchronize(st));
    a = b;
  }
  return ORSP_OK;
}

// Bucket of a box of v nodes under the graph's plan.
int plan_bucket(const orsp::Graph *g, int64_t v) {
  for (int i = 0; i < g->plan_nb - 1; ++i)
    if (v <= g->plan_max_nodes[i]) return i;
  return g->plan_nb - 1;
}

}  // namespace

static int run_batch(orsp_graph *g, const float *cost_d, int32_t K, const int32_t *src_d,
                     const int32_t *dst_d, const int32_t *bbox_d, int range_mode,
                     const int32_t *order_d, float delta, int32_t *path_nodes_d,
                     int32_t *path_edges_d, int32_t path_cap, int32_t *path_len_d,
                     uintptr_t stream) {
  if (!g || !cost_d || K < 0 || (K > 0 && (!src_d || !dst_d || !bbox_d || !path_nodes_d ||
                                           !path_len_d)) || path_cap <= 0) {
    set_error("batch search: NULL argument or path_cap <= 0");
    return ORSP_ERR_ARG;
  }
  if (!range_mode && g->nx <= 0) { set_error("batch_bbox: graph was created without lattice dims"); return ORSP_ERR_ARG; }
  if (!(delta >= 0.0f) || !(delta < 3.0e38f)) { set_error("delta must be finite and >= 0 (0: chosen on the device)"); return ORSP_ERR_ARG; }
  if (K == 0) return ORSP_OK;
  ORSP_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = (cudaStream_t)stream;

  // ROI sizes are needed on the host to size the work.
  const int per = range_mode ? 2 : 6;
  std::vector<int32_t> bb((size_t)per * K);
  ORSP_CUDA(cudaMemcpyAsync(bb.data(), bbox_d, bb.size() * 4, cudaMemcpyDeviceToHost, st));
  std::vector<int32_t> ord(K);
  if (order_d) ORSP_CUDA(cudaMemcpyAsync(ord.data(), order_d, (size_t)K * 4, cudaMemcpyDeviceToHost, st));
  ORSP_CUDA(cudaStreamSynchronize(st));
  for (int32_t k = 0; k < K; ++k) {
    const int32_t *b = &bb[(size_t)per * k];
    if (range_mode) {
      if (b[0] < 0 || b[1] > g->N || b[1] <= b[0]) {
        set_error("batch_ranges: node range outside the graph or empty");
        return ORSP_ERR_ARG;
      }
    } else if (b[0] < 0 || b[2] < 0 || b[4] < 0 || b[1] >= g->nx || b[3] >= g->ny || b[5] >= g->nz ||
               b[1] < b[0] || b[3] < b[2] || b[5] < b[4]) {
      set_error("batch_bbox: box outside the lattice or empty");
      return ORSP_ERR_ARG;
    }
  }
  if (order_d) {
    std::vector<char> seen(K, 0);
    for (int32_t k = 0; k < K; ++k) {
      if (ord[k] < 0 || ord[k] >= K || seen[ord[k]]) {
        set_error("batch_bbox: order must be a permutation of 0..K-1");
        return ORSP_ERR_ARG;
      }
      seen[ord[k]] = 1;
    }
  } else {
    for (int32_t k = 0; k < K; ++k) ord[k] = k;
  }
  // items per bucket, in the processing order
  const bool tuned = g->plan_nb > 0 && !range_mode;
  const int nb = tuned ? g->plan_nb : 1;
  std::vector<std::vector<int32_t>> bucket(nb);
  for (int32_t i = 0; i < K; ++i) {
    const int32_t k = ord[i];
    bucket[tuned ? plan_bucket(g, box_volume(&bb[(size_t)per * k], range_mode)) : 0].push_back(k);
  }
  // Tile-sweep buckets first (one launch per tile width), then every
  // one-CTA-per-search item in a single launch, each with its bucket's width,
  // so that searches of all sizes share the GPU.
  std::vector<int32_t> src_h, dst_h;
  std::vector<int32_t> cta_items;
  std::vector<float> delta_k;
  int cta_ctas = 0;
  // a box deeper than a shared-memory tile holds goes to the CTA kernel
  auto tile_ok = [&](int32_t k, int tw) {
    if (range_mode) return true;
    const int32_t *b = &bb[(size_t)per * k];
    return lattice_tile_fits(b[5] - b[4] + 1, tw);
  };
  for (int tw : {16, 32}) {
    std::vector<int32_t> lat_items;
    for (int i = 0; i < nb; ++i)
      if (tuned && g->plan_impl[i] == 1 && g->lattice_ok && !(g->cvia && tw != 16) && g->plan_tile[i] == tw)
        for (int32_t k : bucket[i])
          if (tile_ok(k, tw)) lat_items.push_back(k);
    if (lat_items.empty()) continue;
    if (src_h.empty()) {
      src_h.resize(K);
      dst_h.resize(K);
      ORSP_CUDA(cudaMemcpyAsync(src_h.data(), src_d, (size_t)K * 4, cudaMemcpyDeviceToHost, st));
      ORSP_CUDA(cudaMemcpyAsync(dst_h.data(), dst_d, (size_t)K * 4, cudaMemcpyDeviceToHost, st));
      ORSP_CUDA(cudaStreamSynchronize(st));
    }
    int rc = run_batch_lat(g, cost_d, K, lat_items, bb, src_h, dst_h, tw, path_nodes_d, path_edges_d, path_cap,
                           path_len_d, st);
    if (rc) return rc;
  }
  for (int i = 0; i < nb; ++i) {
    std::vector<int32_t> items;
    if (tuned && g->plan_impl[i] == 1 && g->lattice_ok && !(g->cvia && g->plan_tile[i] != 16)) {
      for (int32_t k : bucket[i])
        if (!tile_ok(k, g->plan_tile[i])) items.push_back(k);
    } else {
      items = bucket[i];
    }
    if (items.empty()) continue;
    if (tuned) {
      if (delta_k.empty()) delta_k.assign(K, 0.0f);
      for (int32_t k : items) delta_k[k] = g->plan_delta[i];
      cta_ctas = std::max(cta_ctas, g->plan_ctas[i]);
    }
    cta_items.insert(cta_items.end(), items.begin(), items.end());
  }
  if (!cta_items.empty()) {
    // processing order of the caller, across buckets
    if (tuned) {
      std::vector<int32_t> pos(K);
      for (int32_t i = 0; i < K; ++i) pos[ord[i]] = i;
      std::stable_sort(cta_items.begin(), cta_items.end(), [&](int32_t x, int32_t y) { return pos[x] < pos[y]; });
    }
    const int ctas = cta_ctas > 0 ? cta_ctas : std::max(1, env_int("ORSP_BATCH_CTAS_PER_SM", 2));
    int rc = run_batch_cta(g, cost_d, K, cta_items, src_d, dst_d, bbox_d, bb, range_mode, delta, delta_k, ctas,
                           path_nodes_d, path_edges_d, path_cap, path_len_d, st);
    if (rc) return rc;
  }
  ORSP_CUDA(cudaStreamSynchronize(st));
  return ORSP_OK;
}

extern "C" int orsp_batch_set_plan(orsp_graph *g, int32_t nb, const int64_t *max_nodes, const int32_t *impl,
                                   const float *delta, const int32_t *tile_w, const int32_t *ctas_per_sm) {
  if (!g || nb < 0 || nb > 8) { set_error("batch_set_plan: 0..8 buckets"); return ORSP_ERR_ARG; }
  if (nb > 0 && (!max_nodes || !impl || !delta || !tile_w || !ctas_per_sm)) {
    set_error("batch_set_plan: NULL array");
    return ORSP_ERR_ARG;
  }
  for (int i = 0; i < nb; ++i) {
    if (i > 0 && max_nodes[i] <= max_nodes[i - 1]) { set_error("batch_set_plan: max_nodes must increase"); return ORSP_ERR_ARG; }
    if (impl[i] != 0 && impl[i] != 1) { set_error("batch_set_plan: impl must be 0 or 1"); return ORSP_ERR_ARG; }
    if (!(delta[i] >= 0.0f) || !(delta[i] < 3.0e38f)) { set_error("batch_set_plan: delta must be finite and >= 0"); return ORSP_ERR_ARG; }
    if (impl[i] == 1 && tile_w[i] != 16 && tile_w[i] != 32) { set_error("batch_set_plan: tile width must be 16 or 32"); return ORSP_ERR_ARG; }
    if (ctas_per_sm[i] < 0 || ctas_per_sm[i] > 8) { set_error("batch_set_plan: ctas_per_sm must be 0..8"); return ORSP_ERR_ARG; }
  }
  g->plan_nb = nb;
  for (int i = 0; i < nb; ++i) {
    g->plan_max_nodes[i] = max_nodes[i];
    g->plan_impl[i] = impl[i];
    g->plan_delta[i] = delta[i];
    g->plan_tile[i] = impl[i] == 1 ? tile_w[i] : 16;
    g->plan_ctas[i] = ctas_per_sm[i];
  }
  return ORSP_OK;
}

extern "C" int orsp_sssp_batch_bbox(orsp_graph *g, const float *cost_d, int32_t K,
                                    const int32_t *src_d, const int32_t *dst_d,
                                    const int32_t *bbox_d, const int32_t *order_d,
                                    float delta, int32_t *path_nodes_d,
                                    int32_t *path_edges_d, int32_t path_cap,
                                    int32_t *path_len_d, uintptr_t stream) {
  return run_batch(g, cost_d, K, src_d, dst_d, bbox_d, 0, order_d, delta, path_nodes_d, path_edges_d,
                   path_cap, path_len_d, stream);
}

extern "C" int orsp_sssp_batch_ranges(orsp_graph *g, const float *cost_d, int32_t K,
                                      const int32_t *src_d, const int32_t *dst_d,
                                      const int32_t *ranges_d, const int32_t *order_d,
                                      float delta, int32_t *path_nodes_d,
                                      int32_t *path_edges_d, int32_t path_cap,
                                      int32_t *path_len_d, uintptr_t stream) {
  return run_batch(g, cost_d, K, src_d, dst_d, ranges_d, 1, order_d, delta, path_nodes_d, path_edges_d,
                   path_cap, path_len_d, stream);
}

namespace orsp {

int run_roi_nodes_cta(Graph *gr, const float *cost_d, const int32_t *src_d, const int32_t *dst_d,
                      const int32_t *roi_map_d, const int32_t *roi_nodes_d, int64_t n_roi, int32_t *path_out_d,
                      int32_t path_cap, int32_t *path_len_d, cudaStream_t st, int32_t *len_h) {
  if (n_roi >= INT32_MAX) { set_error("sssp_roi_nodes: ROI too large"); return ORSP_ERR_ARG; }
  orsp_graph *g = static_cast<orsp_graph *>(gr);
  const std::vector<int32_t> items{0}, bb{0, (int32_t)n_roi};
  const std::vector<float> no_dk;
  int rc = run_batch_cta(g, cost_d, 1, items, src_d, dst_d, nullptr, bb, 2, 0.0f, no_dk, 1, path_out_d, nullptr,
                         path_cap, path_len_d, st, roi_map_d, roi_nodes_d);
  if (rc) return rc;
  ORSP_CUDA(cudaMemcpyAsync(len_h, path_len_d, 4, cudaMemcpyDeviceToHost, st));
  ORSP_CUDA(cudaStreamSynchronize(st));
  return ORSP_OK;
}

}  // namespace orsp

// Many whole-graph single-source searches.  On a recognised lattice, up to
// per_launch sources share one persistent launch: each source is a box
// covering the whole lattice with its own distance slice, and the slices are
// the caller's output rows, so the tile queue interleaves the wavefronts of
// all of them.  Elsewhere one grid search per source.
extern "C" int orsp_sssp_sources(orsp_graph *g, const float *cost_d, int32_t nsrc, const int32_t *src_h,
                                 float *dist_out_d, int32_t per_launch, uintptr_t stream) {
  if (!g || !cost_d || nsrc < 0 || (nsrc > 0 && (!src_h || !dist_out_d)) || per_launch < 0) {
    set_error("sssp_sources: NULL argument or negative count");
    return ORSP_ERR_ARG;
  }
  for (int32_t i = 0; i < nsrc; ++i)
    if (src_h[i] < 0 || src_h[i] >= g->N) { set_error("sssp_sources: source out of range"); return ORSP_ERR_ARG; }
  if (nsrc == 0) return ORSP_OK;
  ORSP_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = (cudaStream_t)stream;
  const char *impl = getenv("ORSP_SSSP_IMPL");
  const bool lattice = g->lattice_ok && lattice_tile_fits(g->nz) && !(impl && std::string(impl) == "generic");
  if (!lattice) {
    for (int32_t i = 0; i < nsrc; ++i) {
      int rc = grow_dev((void **)&g->batch_idx, &g->batch_idx_bytes, 256);
      if (rc) return rc;
      ORSP_CUDA(cudaMemcpyAsync(g->batch_idx, &src_h[i], 4, cudaMemcpyHostToDevice, st));
      int32_t len = 0;
      rc = orsp_sssp(g, cost_d, 1, g->batch_idx, nullptr, -1, nullptr, 0.0f, dist_out_d + (int64_t)i * g->N,
                     nullptr, 0, &len, nullptr, stream);
      if (rc != ORSP_OK && rc != ORSP_NO_PATH) return rc;
    }
    return ORSP_OK;
  }
  const int32_t per = per_launch > 0 ? std::min(per_launch, nsrc) : nsrc;
  const int32_t full[6] = {0, g->nx - 1, 0, g->ny - 1, 0, g->nz - 1};
  std::vector<int32_t> boxes((size_t)per * 6);
  for (int32_t j = 0; j < per; ++j)
    for (int c = 0; c < 6; ++c) boxes[(size_t)j * 6 + c] = full[c];
  const size_t tab = (size_t)per * sizeof(LatBox) + (size_t)per * 4 + 256;
  if (g->blat_tab_bytes < tab) {
    cudaFree(g->blat_tab_d);
    if (g->blat_tab_h) cudaFreeHost(g->blat_tab_h);
    g->blat_tab_d = nullptr;
    g->blat_tab_h = nullptr;
    g->blat_tab_bytes = 0;
    ORSP_CUDA(cudaMalloc(&g->blat_tab_d, tab));
    ORSP_CUDA(cudaMallocHost(&g->blat_tab_h, tab));
    g->blat_tab_bytes = tab;
  }
  const uint64_t decl = g->decl_cost == cost_d ? g->decl_gen : 0;
  // profiling: kernel time and counters summed over the chunks
  float ksum = 0.0f;
  int64_t csum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int32_t a = 0; a < nsrc; a += per) {
    const int32_t m = std::min(per, nsrc - a);
    LatBox *hb = (LatBox *)g->blat_tab_h;
    int32_t *h_src = (int32_t *)(hb + m);
    // the staging buffer is reused: the previous chunk was synchronised
    const int64_t ntiles = make_lat_boxes(boxes.data(), m, hb);
    for (int32_t j = 0; j < m; ++j) {
      hb[j].dbase = (int64_t)j * g->N;
      hb[j].pad = j;  // TMA staging: slice j
      h_src[j] = src_h[a + j];
    }
    ORSP_CUDA(cudaMemcpyAsync(g->blat_tab_d, g->blat_tab_h, (size_t)m * sizeof(LatBox) + (size_t)m * 4,
                              cudaMemcpyHostToDevice, st));
    const LatBox *db = (const LatBox *)g->blat_tab_d;
    const int32_t *d_src = (const int32_t *)(db + m);
    int rc = reserve_lattice_ws(g, ntiles);
    if (rc) return rc;
    LatOptions opt;
    opt.private_dist = true;
    opt.private_count = (int64_t)m * g->N;
    opt.tma_slices = m;
    // many wave fronts keep two CTAs per SM busy: one's queue handoff
    // overlaps the other's sweeps (measured 0.50 against 0.77 ms per source
    // on 1000x1000x12 at 16 sources per launch)
    opt.blocks_per_sm = 2;
    // and, for tiles of up to 12 layers (the instantiation sized for two
    // CTAs per SM), the warp-specialised schedule: its scheduler warp takes
    // the queue handoff off the workers' path (0.449 against 0.473 ms per
    // source on 1000x1000x12)
    opt.spec = g->nz <= 12 ? 1 : 0;
    // every chunk after the first reuses the gathered weights of this call
    if (decl) g->decl_cost = cost_d, g->decl_gen = decl;
    else if (a > 0) g->decl_cost = cost_d, g->decl_gen = ~0ull;
    rc = run_lattice_boxes(g, cost_d, m, d_src, nullptr, m, boxes.data(), db,
                           (uint32_t *)(dist_out_d + (int64_t)a * g->N), st, &opt);
    if (rc) return rc;
    ORSP_CUDA(cudaStreamSynchronize(st));
    rc = finish_lattice_search(g, nullptr);
    if (rc) return rc;
    for (int i = 0; i < 8; ++i) csum[i] += g_counters[i];
    if (g_timer.on && g_timer.pending) {
      float ms = 0.0f;
      ORSP_CUDA(cudaEventElapsedTime(&ms, g_timer.a, g_timer.b));
      ksum += ms;
      g_timer.pending = false;
    }
    if (!decl && a == 0) {  // the gather of this call: generation ~0 until the next undeclared search
      g->w4_gen = ~0ull;
    }
  }
  if (!decl) {  // a generation this call made up must not match a caller's later declaration
    g->w4_cost = nullptr;
    g->w4_gen = 0;
  }
  for (int i = 0; i < 8; ++i) g_counters[i] = csum[i];
  if (g_timer.on) g_timer.last_ms = ksum;
  return ORSP_OK;
}
