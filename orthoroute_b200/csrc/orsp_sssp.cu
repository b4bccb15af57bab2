// Single search over the whole graph (or a global_to_roi ROI): one persistent
// cooperative launch running near-far delta-stepping, then a one-warp
// backtrace that applies the reference's settle-order tie-break.
//
// Replaces SimpleDijkstra.find_path_roi (UPF:1801-1887),
// CUDADijkstra.find_path_roi_gpu (CD:4909) and the wavefront loop of
// _run_near_far (CD:2770-3042).  Unlike the reference wavefront (which adds
// jitter and stops a fixed number of iterations after the sink is reached,
// CD:2974-2997), the loop here runs to the exact fp32 fixpoint for every node
// with d < d[dst]: a near-far phase with threshold T settles every node whose
// final distance is < T, so the search stops after the first phase that
// leaves d[dst] < T.
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <string>

#include "common.cuh"
#include "lattice_walk.cuh"

namespace {

struct SsspCtl {
  GridBarrier bar;
  int err;
  unsigned qcnt[3];   // near-queue counts, rotating by round % 3
  unsigned fcnt[4];   // far-pile counts, rotating by far generation % 4
  unsigned fmin[4];   // min distance bits pushed into each far generation
  unsigned rounds;
  int path_len;
  int status;         // 0 = ok, 1 = no path
  int pad;
};

struct SsspParams {
  const int32_t *indptr;
  const int32_t *indices;
  const float *cost;
  const int32_t *roi_map;    // global_to_roi or nullptr
  const uint8_t *sink_mask;  // nodes that are settled but never expanded
  uint32_t *dist;            // fp32 bits
  int2 *nq0, *nq1;
  int2 *fq0, *fq1;
  int64_t qcap, fcap;
  SsspCtl *ctl;
  int32_t N;
  int32_t dst;
  float delta;
  const float *delta_d;  // device bucket width (overrides delta) or nullptr
  unsigned max_rounds;
  unsigned long long wait_ns;
  unsigned long long budget_ns;
};

// One block: twice the mean of a strided sample of the finite costs.  The
// bucket width only changes how many near-far phases a search takes, never
// its distances or paths.
__global__ void auto_delta_kernel(const float *cost, int64_t E, int64_t step, float *out) {
  __shared__ double s_sum[32];
  __shared__ long long s_cnt[32];
  double sum = 0.0;
  long long cnt = 0;
  for (int64_t i = (int64_t)threadIdx.x * step; i < E; i += (int64_t)blockDim.x * step) {
    const float c = cost[i];
    if (c >= 0.0f && c < __int_as_float(0x7f800000)) {
      sum += (double)c;
      ++cnt;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_down_sync(0xffffffffu, sum, o);
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    s_sum[w] = sum;
    s_cnt[w] = cnt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    long long n = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      t += s_sum[k];
      n += s_cnt[k];
    }
    float d = n ? (float)(2.0 * t / (double)n) : 1.0f;
    if (!(d >= 1e-6f)) d = 1e-6f;
    if (!(d < 3.0e38f)) d = 3.0e38f;
    *out = d;
  }
}

__global__ void fill_u32_kernel(uint32_t *p, int64_t n, uint32_t v) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t s = (int64_t)gridDim.x * blockDim.x;
  for (; i < n; i += s) p[i] = v;
}

// Control-block reset and seeding: every valid seed goes into far generation 0,
// so the first round is a split round that opens the first bucket at
// min(seed cost) + delta.
__global__ void seed_kernel(SsspParams p, int32_t nseeds, const int32_t *seeds,
                            const float *seed_cost) {
  SsspCtl *c = p.ctl;
  if (threadIdx.x == 0) {
    c->bar.count = 0;
    c->bar.gen = 0;
    c->err = 0;
    for (int i = 0; i < 3; ++i) c->qcnt[i] = 0;
    for (int i = 0; i < 4; ++i) {
      c->fcnt[i] = 0;
      c->fmin[i] = ORSP_INF_BITS;
    }
    c->rounds = 0;
    c->path_len = 0;
    c->status = 0;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nseeds; i += blockDim.x) {
    int s = seeds[i];
    if (s < 0 || s >= p.N) continue;
    if (p.roi_map && p.roi_map[s] < 0) continue;
    float c0 = seed_cost ? seed_cost[i] : 0.0f;
    if (!(c0 >= 0.0f) || !(c0 < __int_as_float(0x7f800000))) continue;
    unsigned b = f_bits(c0);
    atomicMin(&p.dist[s], b);
    unsigned slot = atomicAdd(&c->fcnt[0], 1u);
    if ((int64_t)slot < p.fcap) p.fq0[slot] = make_int2(s, (int)b);
    atomicMin(&c->fmin[0], b);
  }
}

__global__ void __launch_bounds__(512) sssp_grid_kernel(SsspParams p) {
  SsspCtl *ctl = p.ctl;
  const unsigned nblocks = gridDim.x;
  const int lane = threadIdx.x & 31;
  const int64_t gwarp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const bool leader = (blockIdx.x == 0 && threadIdx.x == 0);
  const unsigned long long t_start = dev_globaltimer();
  const float INF_F = __int_as_float(0x7f800000);
  const float delta = p.delta_d ? *p.delta_d : p.delta;

  unsigned r = 0, g = 0;
  float T = 0.0f;
  for (;;) {
    // ---- decisions: values read here are not modified before the barrier
    int err = (int)ld_acquire_u32((const unsigned *)&ctl->err);
    if (err) break;
    if (r >= p.max_rounds) {
      if (leader) atomicCAS(&ctl->err, DEV_OK, DEV_ERR_TIMEOUT);
      break;
    }
    unsigned n_in = ld_acquire_u32(&ctl->qcnt[r % 3]);
    if ((int64_t)n_in > p.qcap) n_in = (unsigned)p.qcap;
    if (n_in > 0) {
      // ---- relaxation round over the near queue
      const int2 *inq = ((r & 1) ? p.nq1 : p.nq0);
      int2 *outq = (((r + 1) & 1) ? p.nq1 : p.nq0);
      int2 *farq = ((g & 1) ? p.fq1 : p.fq0);
      unsigned *out_cnt = &ctl->qcnt[(r + 1) % 3];
      unsigned *far_cnt = &ctl->fcnt[g % 4];
      unsigned *far_min = &ctl->fmin[g % 4];
      for (int64_t base = gwarp * 32; base < (int64_t)n_in; base += nwarps * 32) {
        int64_t i = base + lane;
        int beg = 0, end = 0;
        unsigned dbits = 0;
        if (i < (int64_t)n_in) {
          int2 it = __ldcg(&inq[i]);
          if (__ldcg(&p.dist[it.x]) == (unsigned)it.y &&
              !(p.sink_mask && p.sink_mask[it.x])) {
            beg = __ldg(&p.indptr[it.x]);
            end = __ldg(&p.indptr[it.x + 1]);
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
            const int w = __ldg(&p.indices[e]);
            if (!p.roi_map || __ldg(&p.roi_map[w]) >= 0) {
              const float nd = __fadd_rn(d, __ldg(&p.cost[e]));
              if (nd < INF_F) {
                const unsigned nb = f_bits(nd);
                if (nb < __ldcg(&p.dist[w])) {
                  const unsigned old = atomicMin(&p.dist[w], nb);
                  if (nb < old) {
                    item = make_int2(w, (int)nb);
                    if (nd < T) pn = true; else pf = true;
                  }
                }
              }
            }
          }
          warp_append(outq, out_cnt, p.qcap, pn, item, &ctl->err);
          warp_append(farq, far_cnt, p.fcap, pf, item, &ctl->err);
          if (pf) fmin_local = fmin_local < item.y ? fmin_local : (unsigned)item.y;
        }
        const unsigned wm = warp_min_u32(fmin_local);
        if (lane == 0 && wm != ORSP_INF_BITS) atomicMin(far_min, wm);
      }
    } else {
      // ---- phase boundary: stop, or open the next bucket from the far pile
      unsigned fc = ld_acquire_u32(&ctl->fcnt[g % 4]);
      if ((int64_t)fc > p.fcap) fc = (unsigned)p.fcap;
      bool done = (fc == 0);
      if (!done && p.dst >= 0) {
        const float dd = bits_f(__ldcg(&p.dist[p.dst]));
        if (dd < T) done = true;
      }
      if (done) break;
      const float fm = bits_f(ld_acquire_u32(&ctl->fmin[g % 4]));
      float Tn = __fadd_rn(fm, delta);
      if (!(Tn > fm)) Tn = __uint_as_float(f_bits(fm) + 1u);
      const int2 *fin = ((g & 1) ? p.fq1 : p.fq0);
      int2 *fout = (((g + 1) & 1) ? p.fq1 : p.fq0);
      int2 *outq = (((r + 1) & 1) ? p.nq1 : p.nq0);
      unsigned *out_cnt = &ctl->qcnt[(r + 1) % 3];
      unsigned *fout_cnt = &ctl->fcnt[(g + 1) % 4];
      unsigned *fout_min = &ctl->fmin[(g + 1) % 4];
      for (int64_t base = gwarp * 32; base < (int64_t)fc; base += nwarps * 32) {
        int64_t i = base + lane;
        bool pn = false, pf = false;
        int2 it = make_int2(0, 0);
        if (i < (int64_t)fc) {
          it = __ldcg(&fin[i]);
          if (__ldcg(&p.dist[it.x]) == (unsigned)it.y) {
            if (bits_f((unsigned)it.y) < Tn) pn = true; else pf = true;
          }
        }
        warp_append(outq, out_cnt, p.qcap, pn, it, &ctl->err);
        warp_append(fout, fout_cnt, p.fcap, pf, it, &ctl->err);
        const unsigned wm = warp_min_u32(pf ? (unsigned)it.y : ORSP_INF_BITS);
        if (lane == 0 && wm != ORSP_INF_BITS) atomicMin(fout_min, wm);
      }
      if (leader) {
        ctl->fcnt[(g + 2) % 4] = 0;
        ctl->fmin[(g + 2) % 4] = ORSP_INF_BITS;
      }
      T = Tn;
      ++g;
    }
    if (leader) {
      ctl->qcnt[(r + 2) % 3] = 0;
      if (dev_globaltimer() - t_start > p.budget_ns) atomicCAS(&ctl->err, DEV_OK, DEV_ERR_TIMEOUT);
    }
    grid_barrier(&ctl->bar, nblocks, &ctl->err, p.wait_ns);
    ++r;
  }
  if (leader) ctl->rounds = r;
}

struct BacktraceParams {
  const float *cost;
  const int32_t *roi_map;
  const int32_t *rptr, *rsrc, *reid;
  const uint32_t *dist;
  const int32_t *seeds;
  const float *seed_cost;
  int32_t nseeds;
  int32_t dst;
  const int32_t *dst_d;  // when set, the target is read here (< 0: no path)
  int32_t *path_out;
  int32_t path_cap;
  SsspCtl *ctl;
};

// One warp walks from dst towards the seeds.  At each node v the parent is the
// in-neighbour u (inside the ROI) with fl32(d[u] + w(u,v)) == d[v] and the
// smallest (d[u], rank(u)) that is below (d[v], rank(v)); a seed whose
// distance still equals its start cost ends the walk.  (d, rank) strictly
// decreases along the walk, so it always terminates.
__global__ void backtrace_kernel(BacktraceParams p) {
  const int lane = threadIdx.x & 31;
  SsspCtl *ctl = p.ctl;
  if (ctl->err) return;
  const int32_t dst = p.dst_d ? *p.dst_d : p.dst;
  unsigned dv = dst >= 0 ? p.dist[dst] : ORSP_INF_BITS;
  if (dv == ORSP_INF_BITS) {
    if (lane == 0) { ctl->path_len = 0; ctl->status = 1; }
    return;
  }
  int v = dst;
  int len = 0;
  int err = 0;
  for (;;) {
    if (len >= p.path_cap) { err = DEV_ERR_PATH_OVERFLOW; break; }
    if (lane == 0) p.path_out[len] = v;
    ++len;
    // seed that was never improved: the walk starts here
    bool is_start = false;
    for (int i = lane; i < p.nseeds; i += 32) {
      if (p.seeds[i] == v) {
        float c0 = p.seed_cost ? p.seed_cost[i] : 0.0f;
        if (f_bits(c0) == dv) is_start = true;
      }
    }
    if (__any_sync(ORSP_FULL_MASK, is_start)) break;
    const int rv = p.roi_map ? p.roi_map[v] : v;
    const int b = p.rptr[v], e = p.rptr[v + 1];
    unsigned long long best = ULLONG_MAX;
    int bu = -1;
    for (int k0 = b; k0 < e; k0 += 32) {
      const int k = k0 + lane;
      if (k < e) {
        const int u = p.rsrc[k];
        const int ru = p.roi_map ? p.roi_map[u] : u;
        if (ru >= 0) {
          const unsigned du = p.dist[u];
          if (du != ORSP_INF_BITS) {
            const float s = __fadd_rn(bits_f(du), p.cost[p.reid[k]]);
            if (f_bits(s) == dv && (du < dv || (du == dv && ru < rv))) {
              const unsigned long long key = ((unsigned long long)du << 32) | (unsigned)ru;
              if (key < best) { best = key; bu = u; }
            }
          }
        }
      }
    }
    const unsigned long long wbest = warp_min_u64(best);
    if (wbest == ULLONG_MAX) { err = DEV_ERR_INTERNAL; break; }
    const unsigned owner = __ballot_sync(ORSP_FULL_MASK, best == wbest && bu >= 0);
    v = __shfl_sync(ORSP_FULL_MASK, bu, __ffs(owner) - 1);
    dv = (unsigned)(wbest >> 32);
  }
  __syncwarp();
  if (err) {
    if (lane == 0) atomicCAS(&ctl->err, DEV_OK, err);
    return;
  }
  for (int i = lane; i < len / 2; i += 32) {
    int a = p.path_out[i];
    int z = p.path_out[len - 1 - i];
    p.path_out[i] = z;
    p.path_out[len - 1 - i] = a;
  }
  if (lane == 0) { ctl->path_len = len; ctl->status = 0; }
}

// The same walk on a recognised H/V lattice after a tile-sweep search inside
// box B: lat_walk_warp, up to 32 nodes of a straight run per memory round
// trip (ranks are node ids, as in the tile-sweep search).
using orsp::lat_walk_warp;
using orsp::lat_xyz;
using orsp::LatBox;
using orsp::LatWalkGeom;

struct LatBacktraceParams {
  const float4 *w4;
  const uint32_t *dist;
  LatWalkGeom geom;
  LatBox box;
  const int32_t *seeds;
  const float *seed_cost;
  int32_t nseeds;
  int32_t dst;
  const int32_t *dst_d;     // when set, the target is read here (< 0: no path)
  const int32_t *rank_map;  // node-set ROI: ranks are global_to_roi (NULL: node ids)
  int32_t *path_out;
  int32_t path_cap;
  SsspCtl *ctl;
};

__global__ void lat_backtrace_kernel(LatBacktraceParams p) {
  const int lane = threadIdx.x & 31;
  SsspCtl *ctl = p.ctl;
  if (ctl->err) return;
  const LatBox &B = p.box;
  const int32_t dst = p.dst_d ? *p.dst_d : p.dst;
  if (dst < 0) {
    if (lane == 0) { ctl->path_len = 0; ctl->status = 1; }
    return;
  }
  int32_t x, y, z;
  lat_xyz(p.geom, dst, x, y, z);
  const bool in = x >= B.x0 && x <= B.x1 && y >= B.y0 && y <= B.y1 && z >= B.z0 && z <= B.z1;
  unsigned dv = in ? __ldcg(&p.dist[dst]) : ORSP_INF_BITS;
  if (dv == ORSP_INF_BITS) {
    if (lane == 0) { ctl->path_len = 0; ctl->status = 1; }
    return;
  }
  const uint32_t *dist = p.dist;
  const int32_t nx = p.geom.nx, ny = p.geom.ny;
  auto dget = [dist, nx, ny](int32_t a, int32_t b, int32_t c) {
    return __ldcg(&dist[((int64_t)c * ny + b) * nx + a]);
  };
  const int32_t *seeds = p.seeds;
  const float *seed_cost = p.seed_cost;
  const int32_t nseeds = p.nseeds;
  // a seed whose distance still equals its start cost ends the walk
  auto at_start = [seeds, seed_cost, nseeds](int64_t v, unsigned d) {
    for (int i = 0; i < nseeds; ++i)
      if (seeds[i] == v && f_bits(seed_cost ? seed_cost[i] : 0.0f) == d) return true;
    return false;
  };
  int len;
  if (p.rank_map) len = lat_walk_warp(p.geom, B, p.w4, dget, at_start, x, y, z, dv, p.path_out, p.path_cap,
                                      orsp::LatRankRoi{p.rank_map});
  else len = lat_walk_warp(p.geom, B, p.w4, dget, at_start, x, y, z, dv, p.path_out, p.path_cap);
  int err = 0;
  if (len == -1) err = DEV_ERR_PATH_OVERFLOW;
  else if (len < 0) err = DEV_ERR_INTERNAL;
  __syncwarp();
  if (err) {
    if (lane == 0) atomicCAS(&ctl->err, DEV_OK, err);
    return;
  }
  for (int i = lane; i < len / 2; i += 32) {
    const int a = p.path_out[i];
    const int zz = p.path_out[len - 1 - i];
    p.path_out[i] = zz;
    p.path_out[len - 1 - i] = a;
  }
  if (lane == 0) { ctl->path_len = len; ctl->status = 0; }
}

// Multi-sink winner, as find_path_multisource_multisink (UPF:1941-1975): the
// target with the smallest (double)d[t] + target_cost; among equal totals the
// one the heap pops first, i.e. the smallest (d[t], rank(t)).  One block.
__global__ void pick_target_kernel(const uint32_t *dist, const int32_t *roi_map, int32_t nt,
                                   const int32_t *targets, const double *tcost, int32_t N, int32_t *best) {
  __shared__ double s_tot[256];
  __shared__ unsigned long long s_key[256];
  __shared__ int s_t[256];
  double tot = __longlong_as_double(0x7ff0000000000000ll);
  unsigned long long key = ULLONG_MAX;
  int bt = -1;
  for (int i = threadIdx.x; i < nt; i += blockDim.x) {
    const int t = targets[i];
    if (t < 0 || t >= N) continue;
    const int rank = roi_map ? roi_map[t] : t;
    if (rank < 0) continue;
    const unsigned d = dist[t];
    if (d == ORSP_INF_BITS) continue;
    const double c = (double)bits_f(d) + (tcost ? tcost[i] : 0.0);
    const unsigned long long k = ((unsigned long long)d << 32) | (unsigned)rank;
    if (c < tot || (c == tot && k < key)) { tot = c; key = k; bt = t; }
  }
  s_tot[threadIdx.x] = tot;
  s_key[threadIdx.x] = key;
  s_t[threadIdx.x] = bt;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if (threadIdx.x < off) {
      const int j = threadIdx.x + off;
      if (s_tot[j] < s_tot[threadIdx.x] || (s_tot[j] == s_tot[threadIdx.x] && s_key[j] < s_key[threadIdx.x])) {
        s_tot[threadIdx.x] = s_tot[j];
        s_key[threadIdx.x] = s_key[j];
        s_t[threadIdx.x] = s_t[j];
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *best = s_t[0];
}

// global_to_roi[roi_nodes[i]] = i (a repeated node keeps its last index, as
// numpy's fancy assignment global_to_roi[roi_nodes] = arange(R) does), or,
// with clear, back to -1.
__global__ void roi_scatter_kernel(const int32_t *nodes, int64_t n, int32_t N, int32_t *map, int clear) {
  const int64_t s = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += s) {
    const int32_t v = nodes[i];
    if (v < 0 || v >= N) continue;
    if (clear) map[v] = -1;
    else atomicMax(&map[v], (int32_t)i);
  }
}

__global__ void put_i32_kernel(int32_t *p, int32_t v) { *p = v; }

__global__ void mark_kernel(uint8_t *mask, int32_t n, const int32_t *nodes, int32_t N, uint8_t v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int t = nodes[i];
    if (t >= 0 && t < N) mask[t] = v;
  }
}

unsigned long long env_u64(const char *name, unsigned long long dflt) {
  const char *s = getenv(name);
  if (!s || !*s) return dflt;
  return strtoull(s, nullptr, 10);
}

int ensure_single_ws(orsp::Graph *g, bool need_dist) {
  int64_t cap = g->E + (int64_t)g->N + 64;
  if (need_dist && !g->dist) ORSP_CUDA(cudaMalloc(&g->dist, (size_t)g->N * 4));
  if (g->qcap < cap) {
    for (int i = 0; i < 2; ++i) {
      cudaFree(g->near_q[i]);
      cudaFree(g->far_q[i]);
      g->near_q[i] = g->far_q[i] = nullptr;
    }
    g->qcap = g->fcap = 0;
    for (int i = 0; i < 2; ++i) {
      ORSP_CUDA(cudaMalloc(&g->near_q[i], (size_t)cap * sizeof(int2)));
      ORSP_CUDA(cudaMalloc(&g->far_q[i], (size_t)cap * sizeof(int2)));
    }
    g->qcap = g->fcap = cap;
  }
  if (!g->ctl) ORSP_CUDA(cudaMalloc(&g->ctl, sizeof(SsspCtl)));
  if (!g->ctl_h) ORSP_CUDA(cudaMallocHost(&g->ctl_h, sizeof(SsspCtl)));
  return ORSP_OK;
}

}  // namespace

namespace orsp {
KernelTimer g_timer;
int64_t g_counters[8] = {0, 0, 0, 0, 0, 0, 0, 0};
}  // namespace orsp

extern "C" int orsp_profile_enable(int on) {
  if (on && !orsp::g_timer.a) {
    ORSP_CUDA(cudaEventCreate(&orsp::g_timer.a));
    ORSP_CUDA(cudaEventCreate(&orsp::g_timer.b));
  }
  orsp::g_timer.on = on != 0;
  return ORSP_OK;
}

extern "C" int orsp_profile_counters(int64_t *out8) {
  if (!out8) { orsp::set_error("NULL argument"); return ORSP_ERR_ARG; }
  for (int i = 0; i < 8; ++i) out8[i] = orsp::g_counters[i];
  return ORSP_OK;
}

extern "C" int orsp_profile_last(float *kernel_ms) {
  if (!kernel_ms) { orsp::set_error("NULL argument"); return ORSP_ERR_ARG; }
  if (orsp::g_timer.pending) {
    ORSP_CUDA(cudaEventSynchronize(orsp::g_timer.b));
    ORSP_CUDA(cudaEventElapsedTime(&orsp::g_timer.last_ms, orsp::g_timer.a, orsp::g_timer.b));
    orsp::g_timer.pending = false;
  }
  *kernel_ms = orsp::g_timer.last_ms;
  return ORSP_OK;
}

namespace orsp {

// Shared by orsp_sssp and orsp_sssp_multi: seeds, runs the grid search to the
int launch_auto_delta(const float *cost_d, int64_t E, float *out_d, cudaStream_t st) {
  const int64_t step = std::max<int64_t>(1, E / 65536);
  auto_delta_kernel<<<1, 1024, 0, st>>>(cost_d, E, step, out_d);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

// exact fixpoint (dst >= 0: until d[dst] is below the open bucket) and leaves
// distances in `dist`.
int run_grid_search(Graph *g, const float *cost_d, int32_t nseeds,
                    const int32_t *seeds_d, const float *seed_cost_d,
                    int32_t dst, const int32_t *roi_map_d,
                    const uint8_t *sink_mask_d, float delta, uint32_t *dist,
                    cudaStream_t st) {
  SsspParams p{};
  p.indptr = g->indptr;
  p.indices = g->indices;
  p.cost = cost_d;
  p.roi_map = roi_map_d;
  p.sink_mask = sink_mask_d;
  p.dist = dist;
  p.nq0 = g->near_q[0];
  p.nq1 = g->near_q[1];
  p.fq0 = g->far_q[0];
  p.fq1 = g->far_q[1];
  p.qcap = g->qcap;
  p.fcap = g->fcap;
  p.ctl = (SsspCtl *)g->ctl;
  p.N = g->N;
  p.dst = dst;
  p.delta = delta;
  p.delta_d = nullptr;
  if (delta == 0.0f) {
    int rc = launch_auto_delta(cost_d, g->E, g->auto_delta, st);
    if (rc) return rc;
    p.delta_d = g->auto_delta;
  }
  p.max_rounds = (unsigned)env_u64("ORSP_MAX_ROUNDS", 4ull * g->N + 4096ull);
  p.wait_ns = env_u64("ORSP_WAIT_NS", 2000000000ull);
  p.budget_ns = env_u64("ORSP_BUDGET_NS", 20000000000ull);

  fill_u32_kernel<<<std::min<int64_t>(((int64_t)g->N + 255) / 256, 4096), 256, 0, st>>>(
      dist, g->N, ORSP_INF_BITS);
  ORSP_CUDA(cudaGetLastError());
  seed_kernel<<<1, 256, 0, st>>>(p, nseeds, seeds_d, seed_cost_d);
  ORSP_CUDA(cudaGetLastError());

  static int blocks_per_sm = -1;
  if (blocks_per_sm < 0) {
    int occ = 0;
    ORSP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, sssp_grid_kernel, 512, 0));
    int want = (int)env_u64("ORSP_GRID_BLOCKS_PER_SM", 2);
    blocks_per_sm = std::max(1, std::min(occ, want));
  }
  dim3 grid(g->num_sms * blocks_per_sm), block(512);
  void *args[] = {&p};
  if (orsp::g_timer.on) ORSP_CUDA(cudaEventRecord(orsp::g_timer.a, st));
  ORSP_CUDA(cudaLaunchCooperativeKernel((void *)sssp_grid_kernel, grid, block, args, 0, st));
  if (orsp::g_timer.on) {
    ORSP_CUDA(cudaEventRecord(orsp::g_timer.b, st));
    orsp::g_timer.pending = true;
  }
  return ORSP_OK;
}

}  // namespace orsp

using namespace orsp;

// One search over the whole graph, the ROI of roi_map_d, or the box box_h
// (at most one of the two).  Shared by orsp_sssp and orsp_sssp_box.
static int sssp_impl(orsp_graph *g, const float *cost_d, int32_t nseeds, const int32_t *seeds_d,
                     const float *seed_cost_d, int32_t dst, const int32_t *roi_map_d, const int32_t *box_h,
                     float delta, float *dist_out_d, int32_t *path_out_d, int32_t path_cap,
                     int32_t *path_len_h, int32_t *rounds_h, uintptr_t stream) {
  if (!g || !cost_d || nseeds <= 0 || !seeds_d) { set_error("NULL graph/cost/seeds"); return ORSP_ERR_ARG; }
  if (!(delta >= 0.0f) || !(delta < 3.0e38f)) { set_error("delta must be finite and >= 0 (0: chosen on the device)"); return ORSP_ERR_ARG; }
  if (dst < -1 || dst >= g->N) { set_error("dst out of range"); return ORSP_ERR_ARG; }
  if (dst >= 0 && (!path_out_d || path_cap <= 0 || !path_len_h)) {
    set_error("a destination needs path_out_d, path_cap > 0 and path_len_h");
    return ORSP_ERR_ARG;
  }
  ORSP_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_single_ws(g, dist_out_d == nullptr);
  if (rc) return rc;
  uint32_t *dist = dist_out_d ? (uint32_t *)dist_out_d : g->dist;
  // Full-graph and box searches on a recognised H/V lattice use the
  // tile-sweep search (orsp_lattice.cu); node-set ROIs and other graphs use
  // the generic near-far search, a box there becoming its ROI map.
  // ORSP_SSSP_IMPL=generic forces the latter.
  const char *impl = getenv("ORSP_SSSP_IMPL");
  // (boxes deeper than a shared-memory tile holds, about 33 layers at tile
  // width 16, also take the generic search)
  const int depth = box_h ? box_h[5] - box_h[4] + 1 : g->nz;
  const bool lattice = g->lattice_ok && lattice_tile_fits(depth) && !(impl && std::string(impl) == "generic");
  // a node-set ROI on a lattice: tile sweeps over the ROI's bounding box on
  // ROI-masked weights, ranks from the ROI map in the backtrace
  const bool lattice_roi = lattice && roi_map_d != nullptr;
  if (box_h && !lattice) {
    if (!g->box_g2r) ORSP_CUDA(cudaMalloc(&g->box_g2r, (size_t)g->N * 4));
    rc = orsp_roi_box_map(g, box_h, g->box_g2r, stream);
    if (rc) return rc;
    roi_map_d = g->box_g2r;
  }
  if (lattice_roi) {
    rc = run_lattice_roi(g, cost_d, nseeds, seeds_d, seed_cost_d, roi_map_d, nullptr, 0, nullptr, dist, st);
    if (rc) return rc;
    ORSP_CUDA(cudaMemsetAsync(g->ctl, 0, sizeof(SsspCtl), st));
  } else if (lattice) {
    LatOptions lopt;
    lopt.tma_slices = box_h ? 0 : 1;  // the whole lattice: TMA staging allowed
    rc = run_lattice_search(g, cost_d, nseeds, seeds_d, seed_cost_d, box_h, dist, st, &lopt);
    if (rc) return rc;
    ORSP_CUDA(cudaMemsetAsync(g->ctl, 0, sizeof(SsspCtl), st));
  } else {
    rc = run_grid_search(g, cost_d, nseeds, seeds_d, seed_cost_d, dst, roi_map_d,
                         nullptr, delta, dist, st);
    if (rc) return rc;
  }
  if (dst >= 0 && lattice) {
    LatBacktraceParams b{};
    b.w4 = (const float4 *)g->wslot;
    b.dist = dist;
    b.geom.nx = g->nx;
    b.geom.ny = g->ny;
    b.geom.nz = g->nz;
    for (int z = 0; z < 64; ++z) b.geom.axis[z] = z < g->nz ? g->layer_axis[z] : 0;
    b.geom.wcol = g->cvia ? g->wcol : nullptr;
    b.geom.nzp = (g->nz + 3) & ~3;
    const int32_t full[6] = {0, g->nx - 1, 0, g->ny - 1, 0, g->nz - 1};
    const int32_t *bx = (box_h && !lattice_roi) ? box_h : full;
    b.rank_map = lattice_roi ? roi_map_d : nullptr;
    b.box.x0 = bx[0];
    b.box.x1 = bx[1];
    b.box.y0 = bx[2];
    b.box.y1 = bx[3];
    b.box.z0 = bx[4];
    b.box.z1 = bx[5];
    b.box.dbase = -1;
    b.seeds = seeds_d;
    b.seed_cost = seed_cost_d;
    b.nseeds = nseeds;
    b.dst = dst;
    b.path_out = path_out_d;
    b.path_cap = path_cap;
    b.ctl = (SsspCtl *)g->ctl;
    lat_backtrace_kernel<<<1, 32, 0, st>>>(b);
    ORSP_CUDA(cudaGetLastError());
  } else if (dst >= 0) {
    BacktraceParams b{};
    b.cost = cost_d;
    b.roi_map = roi_map_d;
    b.rptr = g->rptr;
    b.rsrc = g->rsrc;
    b.reid = g->reid;
    b.dist = dist;
    b.seeds = seeds_d;
    b.seed_cost = seed_cost_d;
    b.nseeds = nseeds;
    b.dst = dst;
    b.path_out = path_out_d;
    b.path_cap = path_cap;
    b.ctl = (SsspCtl *)g->ctl;
    backtrace_kernel<<<1, 32, 0, st>>>(b);
    ORSP_CUDA(cudaGetLastError());
  }
  ORSP_CUDA(cudaMemcpyAsync(g->ctl_h, g->ctl, sizeof(SsspCtl), cudaMemcpyDeviceToHost, st));
  ORSP_CUDA(cudaStreamSynchronize(st));
  const SsspCtl *c = (const SsspCtl *)g->ctl_h;
  if (lattice) {
    rc = finish_lattice_search(g, rounds_h);
    if (rc) return rc;
  } else if (rounds_h) {
    *rounds_h = (int32_t)c->rounds;
  }
  if (c->err) return dev_status_to_orsp(c->err);
  if (dst >= 0) {
    *path_len_h = c->path_len;
    if (c->status == 1 || c->path_len < 2) {
      *path_len_h = 0;
      return ORSP_NO_PATH;
    }
  }
  return ORSP_OK;
}

// Backtrace parameters of a lattice search over the whole lattice (distances
// +inf outside the searched box).
static LatBacktraceParams lat_bt_full(orsp_graph *g, const uint32_t *dist, const int32_t *seeds_d,
                                      const float *seed_cost_d, int32_t nseeds, int32_t dst,
                                      const int32_t *dst_d, const int32_t *rank_map, int32_t *path_out_d,
                                      int32_t path_cap) {
  LatBacktraceParams b{};
  b.w4 = (const float4 *)g->wslot;
  b.dist = dist;
  b.geom.nx = g->nx;
  b.geom.ny = g->ny;
  b.geom.nz = g->nz;
  for (int z = 0; z < 64; ++z) b.geom.axis[z] = z < g->nz ? g->layer_axis[z] : 0;
  b.geom.wcol = g->cvia ? g->wcol : nullptr;
  b.geom.nzp = (g->nz + 3) & ~3;
  b.box.x0 = 0;
  b.box.x1 = g->nx - 1;
  b.box.y0 = 0;
  b.box.y1 = g->ny - 1;
  b.box.z0 = 0;
  b.box.z1 = g->nz - 1;
  b.box.dbase = -1;
  b.seeds = seeds_d;
  b.seed_cost = seed_cost_d;
  b.nseeds = nseeds;
  b.dst = dst;
  b.dst_d = dst_d;
  b.rank_map = rank_map;
  b.path_out = path_out_d;
  b.path_cap = path_cap;
  b.ctl = (SsspCtl *)g->ctl;
  return b;
}

static bool use_lattice_roi(const orsp_graph *g) {
  const char *impl = getenv("ORSP_SSSP_IMPL");
  return g->lattice_ok && lattice_tile_fits(g->nz) && !(impl && std::string(impl) == "generic");
}

// Node-list ROIs off the tile lattice: the one-CTA search (block-local
// rounds, no grid barrier, distances in shared memory) up to
// ORSP_ROI_CTA_MAX nodes (default 24 576, the shared-memory limit of the
// batch kernel), else the grid search, which is faster on larger ROIs of
// dense graphs (measured on the reference's Lattice3D shape: 10 K-node
// ROIs 1.46 against 1.68 ms per search, 49 K-node ROIs 3.63 against 2.68).
// ORSP_ROI_NODES_IMPL=grid|cta forces one.
static bool use_roi_cta(int64_t n_roi) {
  const char *impl = getenv("ORSP_ROI_NODES_IMPL");
  if (impl && std::string(impl) == "grid") return false;
  if (impl && std::string(impl) == "cta") return true;
  const char *m = getenv("ORSP_ROI_CTA_MAX");
  const int64_t lim = (m && *m) ? atoll(m) : (int64_t)24576;
  return n_roi <= lim;
}

extern "C" int orsp_sssp_roi_nodes(orsp_graph *g, const float *cost_d, int32_t src, int32_t dst,
                                   const int32_t *roi_nodes_d, int64_t n_roi, int32_t *path_out_d,
                                   int32_t path_cap, int32_t *path_len_h, uintptr_t stream) {
  if (!g || !cost_d || !roi_nodes_d || n_roi <= 0 || !path_out_d || path_cap <= 0 || !path_len_h) {
    set_error("sssp_roi_nodes: NULL argument, empty ROI or path_cap <= 0");
    return ORSP_ERR_ARG;
  }
  if (src < 0 || src >= g->N || dst < 0 || dst >= g->N) { set_error("sssp_roi_nodes: src/dst out of range"); return ORSP_ERR_ARG; }
  ORSP_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_single_ws(g, true);
  if (rc) return rc;
  rc = ensure_roi_arrays(g);
  if (rc) return rc;
  *path_len_h = 0;
  const int sblocks = (int)std::max<int64_t>(1, std::min<int64_t>((n_roi + 255) / 256, 1024));
  roi_scatter_kernel<<<sblocks, 256, 0, st>>>(roi_nodes_d, n_roi, g->N, g->roi_map, 0);
  ORSP_CUDA(cudaGetLastError());
  put_i32_kernel<<<1, 1, 0, st>>>(g->seed_one, src);
  ORSP_CUDA(cudaGetLastError());
  const bool lattice = use_lattice_roi(g);
  // a failed launch still puts the map back to -1 for the next call
  auto fail = [&](int code) {
    roi_scatter_kernel<<<sblocks, 256, 0, st>>>(roi_nodes_d, n_roi, g->N, g->roi_map, 1);
    cudaStreamSynchronize(st);
    return code;
  };
  if (lattice) {
    rc = run_lattice_roi(g, cost_d, 1, g->seed_one, nullptr, g->roi_map, roi_nodes_d, n_roi, nullptr, g->dist, st);
    if (rc) return fail(rc);
    ORSP_CUDA(cudaMemsetAsync(g->ctl, 0, sizeof(SsspCtl), st));
    LatBacktraceParams b = lat_bt_full(g, g->dist, g->seed_one, nullptr, 1, dst, nullptr, g->roi_map, path_out_d,
                                       path_cap);
    lat_backtrace_kernel<<<1, 32, 0, st>>>(b);
    ORSP_CUDA(cudaGetLastError());
  } else if (use_roi_cta(n_roi)) {
    // one CTA: block-local near-far rounds over ROI-local distances
    put_i32_kernel<<<1, 1, 0, st>>>(g->seed_one + 1, dst);
    ORSP_CUDA(cudaGetLastError());
    int32_t len = 0;
    rc = run_roi_nodes_cta(g, cost_d, g->seed_one, g->seed_one + 1, g->roi_map, roi_nodes_d, n_roi, path_out_d,
                           path_cap, g->seed_one + 2, st, &len);
    if (rc) return fail(rc);
    roi_scatter_kernel<<<sblocks, 256, 0, st>>>(roi_nodes_d, n_roi, g->N, g->roi_map, 1);
    ORSP_CUDA(cudaGetLastError());
    ORSP_CUDA(cudaStreamSynchronize(st));
    switch (len) {
      case -1: case 0: case 1: return ORSP_NO_PATH;  // endpoint outside the ROI, unreachable, src == dst
      case -2: set_error("sssp_roi_nodes: work queue overflow"); return ORSP_ERR_OVERFLOW;
      case -3: set_error("sssp_roi_nodes: path longer than path_cap"); return ORSP_ERR_OVERFLOW;
      case -4: set_error("sssp_roi_nodes: round or time limit reached"); return ORSP_ERR_TIMEOUT;
      default: break;
    }
    if (len < 0) { set_error("sssp_roi_nodes: no predecessor on the shortest-path tree"); return ORSP_ERR_INTERNAL; }
    *path_len_h = len;
    return ORSP_OK;
  } else {
    rc = run_grid_search(g, cost_d, 1, g->seed_one, nullptr, dst, g->roi_map, nullptr, 0.0f, g->dist, st);
    if (rc) return fail(rc);
    BacktraceParams b{};
    b.cost = cost_d;
    b.roi_map = g->roi_map;
    b.rptr = g->rptr;
    b.rsrc = g->rsrc;
    b.reid = g->reid;
    b.dist = g->dist;
    b.seeds = g->seed_one;
    b.seed_cost = nullptr;
    b.nseeds = 1;
    b.dst = dst;
    b.path_out = path_out_d;
    b.path_cap = path_cap;
    b.ctl = (SsspCtl *)g->ctl;
    backtrace_kernel<<<1, 32, 0, st>>>(b);
    ORSP_CUDA(cudaGetLastError());
  }
  // the map goes back to -1 for the next call
  roi_scatter_kernel<<<sblocks, 256, 0, st>>>(roi_nodes_d, n_roi, g->N, g->roi_map, 1);
  ORSP_CUDA(cudaGetLastError());
  ORSP_CUDA(cudaMemcpyAsync(g->ctl_h, g->ctl, sizeof(SsspCtl), cudaMemcpyDeviceToHost, st));
  ORSP_CUDA(cudaStreamSynchronize(st));
  const SsspCtl *c = (const SsspCtl *)g->ctl_h;
  if (lattice) {
    rc = finish_lattice_search(g, nullptr);
    if (rc) return rc;
  }
  if (c->err) return dev_status_to_orsp(c->err);
  *path_len_h = c->path_len;
  if (c->status == 1 || c->path_len < 2) {
    *path_len_h = 0;
    return ORSP_NO_PATH;
  }
  return ORSP_OK;
}

extern "C" int orsp_sssp(orsp_graph *g, const float *cost_d, int32_t nseeds,
                         const int32_t *seeds_d, const float *seed_cost_d,
                         int32_t dst, const int32_t *roi_map_d, float delta,
                         float *dist_out_d, int32_t *path_out_d, int32_t path_cap,
                         int32_t *path_len_h, int32_t *rounds_h, uintptr_t stream) {
  return sssp_impl(g, cost_d, nseeds, seeds_d, seed_cost_d, dst, roi_map_d, nullptr, delta, dist_out_d,
                   path_out_d, path_cap, path_len_h, rounds_h, stream);
}

extern "C" int orsp_sssp_box(orsp_graph *g, const float *cost_d, int32_t nseeds,
                             const int32_t *seeds_d, const float *seed_cost_d, int32_t dst,
                             const int32_t *box_h, float delta, float *dist_out_d,
                             int32_t *path_out_d, int32_t path_cap, int32_t *path_len_h,
                             int32_t *rounds_h, uintptr_t stream) {
  if (!g || !box_h) { set_error("sssp_box: NULL graph or box"); return ORSP_ERR_ARG; }
  if (g->nx <= 0) { set_error("sssp_box: graph has no lattice dims"); return ORSP_ERR_ARG; }
  const int32_t *b = box_h;
  if (b[0] < 0 || b[2] < 0 || b[4] < 0 || b[1] >= g->nx || b[3] >= g->ny || b[5] >= g->nz ||
      b[1] < b[0] || b[3] < b[2] || b[5] < b[4]) {
    set_error("sssp_box: box outside the lattice or empty");
    return ORSP_ERR_ARG;
  }
  return sssp_impl(g, cost_d, nseeds, seeds_d, seed_cost_d, dst, nullptr, box_h, delta, dist_out_d,
                   path_out_d, path_cap, path_len_h, rounds_h, stream);
}

extern "C" int orsp_sssp_multi(orsp_graph *g, const float *cost_d, int32_t nseeds, const int32_t *seeds_d,
                               const float *seed_cost_d, int32_t ntargets, const int32_t *targets_d,
                               const double *target_cost_d, const int32_t *roi_map_d, float delta,
                               int32_t *path_out_d, int32_t path_cap, int32_t *path_len_h,
                               int32_t *best_target_h, uintptr_t stream) {
  if (!g || !cost_d || nseeds <= 0 || !seeds_d || ntargets <= 0 || !targets_d || !path_out_d || path_cap <= 0 ||
      !path_len_h) {
    set_error("sssp_multi: NULL argument or empty seeds / targets");
    return ORSP_ERR_ARG;
  }
  if (!(delta >= 0.0f) || !(delta < 3.0e38f)) { set_error("delta must be finite and >= 0 (0: chosen on the device)"); return ORSP_ERR_ARG; }
  ORSP_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_single_ws(g, true);
  if (rc) return rc;
  if (use_lattice_roi(g)) {
    // tile sweeps with the targets' out-edges blocked (a target is settled
    // but never expanded, UPF:1941-1950), then the winner and the lattice walk
    rc = ensure_roi_arrays(g);
    if (rc) return rc;
    const int mblocks = std::max(1, std::min(1024, (ntargets + 255) / 256));
    mark_kernel<<<mblocks, 256, 0, st>>>(g->sink_mask, ntargets, targets_d, g->N, 1);
    ORSP_CUDA(cudaGetLastError());
    rc = run_lattice_roi(g, cost_d, nseeds, seeds_d, seed_cost_d, roi_map_d, nullptr, 0, g->sink_mask, g->dist, st);
    if (rc) {  // the sink mask goes back to 0 for the next call
      mark_kernel<<<mblocks, 256, 0, st>>>(g->sink_mask, ntargets, targets_d, g->N, 0);
      cudaStreamSynchronize(st);
      return rc;
    }
    ORSP_CUDA(cudaMemsetAsync(g->ctl, 0, sizeof(SsspCtl), st));
    int32_t *best_l = g->seed_one + 8;
    pick_target_kernel<<<1, 256, 0, st>>>(g->dist, roi_map_d, ntargets, targets_d, target_cost_d, g->N, best_l);
    ORSP_CUDA(cudaGetLastError());
    LatBacktraceParams b = lat_bt_full(g, g->dist, seeds_d, seed_cost_d, nseeds, -1, best_l, roi_map_d, path_out_d,
                                       path_cap);
    lat_backtrace_kernel<<<1, 32, 0, st>>>(b);
    ORSP_CUDA(cudaGetLastError());
    mark_kernel<<<mblocks, 256, 0, st>>>(g->sink_mask, ntargets, targets_d, g->N, 0);
    ORSP_CUDA(cudaGetLastError());
    ORSP_CUDA(cudaMemcpyAsync(g->ctl_h, g->ctl, sizeof(SsspCtl), cudaMemcpyDeviceToHost, st));
    ORSP_CUDA(cudaMemcpyAsync((char *)g->pinned + 64, best_l, 4, cudaMemcpyDeviceToHost, st));
    ORSP_CUDA(cudaStreamSynchronize(st));
    const SsspCtl *c = (const SsspCtl *)g->ctl_h;
    if (best_target_h) *best_target_h = *(const int32_t *)((const char *)g->pinned + 64);
    rc = finish_lattice_search(g, nullptr);
    if (rc) return rc;
    if (c->err) return dev_status_to_orsp(c->err);
    *path_len_h = c->path_len;
    if (c->status == 1 || c->path_len < 2) {
      *path_len_h = 0;
      return ORSP_NO_PATH;
    }
    return ORSP_OK;
  }
  // scratch: sink mask (N bytes) + the winning target
  const size_t mask_b = ((size_t)g->N + 255) & ~(size_t)255;
  rc = ensure_scratch(g, mask_b + 256);
  if (rc) return rc;
  uint8_t *sink = (uint8_t *)g->scratch;
  int32_t *best_d = (int32_t *)((char *)g->scratch + mask_b);
  ORSP_CUDA(cudaMemsetAsync(sink, 0, mask_b, st));
  mark_kernel<<<std::max(1, std::min(1024, (ntargets + 255) / 256)), 256, 0, st>>>(sink, ntargets, targets_d, g->N, 1);
  ORSP_CUDA(cudaGetLastError());
  rc = run_grid_search(g, cost_d, nseeds, seeds_d, seed_cost_d, -1, roi_map_d, sink, delta, g->dist, st);
  if (rc) return rc;
  pick_target_kernel<<<1, 256, 0, st>>>(g->dist, roi_map_d, ntargets, targets_d, target_cost_d, g->N, best_d);
  ORSP_CUDA(cudaGetLastError());
  BacktraceParams b{};
  b.cost = cost_d;
  b.roi_map = roi_map_d;
  b.rptr = g->rptr;
  b.rsrc = g->rsrc;
  b.reid = g->reid;
  b.dist = g->dist;
  b.seeds = seeds_d;
  b.seed_cost = seed_cost_d;
  b.nseeds = nseeds;
  b.dst = -1;
  b.dst_d = best_d;
  b.path_out = path_out_d;
  b.path_cap = path_cap;
  b.ctl = (SsspCtl *)g->ctl;
  backtrace_kernel<<<1, 32, 0, st>>>(b);
  ORSP_CUDA(cudaGetLastError());
  ORSP_CUDA(cudaMemcpyAsync(g->ctl_h, g->ctl, sizeof(SsspCtl), cudaMemcpyDeviceToHost, st));
  ORSP_CUDA(cudaMemcpyAsync((char *)g->pinned + 64, best_d, 4, cudaMemcpyDeviceToHost, st));
  ORSP_CUDA(cudaStreamSynchronize(st));
  const SsspCtl *c = (const SsspCtl *)g->ctl_h;
  if (best_target_h) *best_target_h = *(const int32_t *)((const char *)g->pinned + 64);
  if (c->err) return dev_status_to_orsp(c->err);
  *path_len_h = c->path_len;
  if (c->status == 1 || c->path_len < 2) {
    *path_len_h = 0;
    return ORSP_NO_PATH;
  }
  return ORSP_OK;
}

// Owner bitmap (bit v of word v/32 set = node allowed) to global_to_roi with
// rank = node id, for CUDADijkstra.find_path_fullgraph_gpu_seeds's
// allowed_bitmap (CD:5467).
__global__ void bitmap_roi_kernel(const uint32_t *bits, int32_t N, int32_t *g2r) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < N; v += (int64_t)gridDim.x * blockDim.x)
    g2r[v] = ((bits[v >> 5] >> (v & 31)) & 1u) ? (int32_t)v : -1;
}

extern "C" int orsp_roi_from_bitmap(orsp_graph *g, const uint32_t *bitmap_d, int32_t *g2r_d, uintptr_t stream) {
  if (!g || !bitmap_d || !g2r_d) { set_error("roi_from_bitmap: NULL argument"); return ORSP_ERR_ARG; }
  ORSP_CUDA(cudaSetDevice(g->device));
  bitmap_roi_kernel<<<std::min(4096, (g->N + 255) / 256), 256, 0, (cudaStream_t)stream>>>(bitmap_d, g->N, g2r_d);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}
