// Per-net routing loop on the device: the body of _route_all
// (orthoroute/algorithms/manhattan/unified_pathfinder.py:4475-4800, "UPF")
// with per-net live costs, for box ROIs on the H/V lattice.  The nets are
// taken in the given order, in groups whose boxes are pairwise disjoint (one
// net per group is the plain loop).  For each group, four steps are enqueued
// on one stream with no host synchronisation:
//   1. rip up the nets' previous paths: usage -1 on their edges (clear_path,
//      UPF:829) and the live cost of those edges recomputed;
//   2. one tile-sweep launch over the group's boxes (orsp_lattice.cu),
//      distances reset inside the boxes only;
//   3. one warp per net: backtrace inside its box (the parent rule of
//      orsp_sssp, rank = node id = box-local order), path -> edges (first CSR
//      edge u->v, UPF:5463), path and length written into the net's row;
//   4. commit: usage +1 on the new edges (commit_path, UPF:821) and their live
//      costs recomputed.
// Each step reads what the previous one wrote, in stream order.  A net's
// search reads only costs of edges inside its box, and its rip-up and commit
// touch only edges inside its box, so nets with disjoint boxes do not see
// each other: the result equals routing the same order one net at a time,
// which equals the host loop over orsp_commit_edges / orsp_update_costs_live
// / orsp_sssp_box / orsp_path_to_edges, bit for bit.  Device-side errors
// (search timeout, path overflow) are folded into one error word that the
// host reads after the last group.  The groups' launches are captured into
// CUDA graphs of kGraphGroups groups on a stream of the library's own (see
// orsp_route_nets); the launches and their order are the same either way.
#include <algorithm>
#include <cstring>
#include <climits>
#include <vector>

#include "accounting.cuh"
#include "lattice_walk.cuh"

namespace {

using orsp::apply_usage;
using orsp::lat_edge_slot;
using orsp::lat_walk_warp;
using orsp::lat_xyz;
using orsp::LatBox;
using orsp::LatWalkGeom;
using orsp::live_cost;

struct LiveParams {
  int32_t *usage;
  float *present;
  const float *base, *capa, *hist;
  float pres_fac, hist_w, via_mult, base_w;
  int jitter;
  float *cost;
};

// Steps 1 and 4 for the nets of one group: block j takes net order[j], the
// len-1 edges of its row, usage +-1 and live costs.  mode 0: both per edge
// (the edges of a shortest path are distinct and the group's boxes are
// disjoint, so each edge is handled by one thread); 1: usage only; 2: live
// costs only, launched after the usage pass of a group whose paths may share
// edges, so that every edge's cost is computed from its final usage.
// active (NULL: every net) skips net order[j] when active[j] == 0.
__global__ void route_commit_kernel(const int32_t *order, const int32_t *edges, const int32_t *lens, int32_t cap,
                                    int32_t sign, int32_t mode, const int32_t *active, LiveParams lp) {
  if (active && !active[blockIdx.x]) return;
  const int32_t k = order[blockIdx.x];
  const int32_t len = lens[k];
  if (len < 2) return;
  const int32_t ne = min(len - 1, cap);
  const int32_t *row = edges + (int64_t)k * cap;
  for (int32_t i = threadIdx.x; i < ne; i += blockDim.x) {
    const int32_t e = row[i];
    if (e < 0) continue;
    if (mode != 2) apply_usage(lp.usage, lp.present, e, sign);
    if (mode != 1)
      lp.cost[e] = live_cost(e, lp.base, lp.usage, lp.capa, lp.hist, lp.pres_fac, lp.hist_w, lp.via_mult,
                             lp.base_w, lp.jitter);
  }
}

// Snapshot groups: after a round, the nets whose new path uses an edge that
// a net earlier in the group (smaller j) of the same round also uses.  The
// three steps are separate launches: every mark lands before any test reads
// it, and every test reads before the reset.
constexpr int32_t kOwnerFree = 0x7f7f7f7f;  // byte fill of the owner array

// mark: owner[e] = the smallest j of the round's nets whose path holds e
__global__ void snap_mark_kernel(const int32_t *order, const int32_t *edges, const int32_t *lens, int32_t cap,
                                 const int32_t *active, int32_t *owner) {
  const int32_t j = blockIdx.x;
  if (active && !active[j]) return;
  const int32_t k = order[j], len = lens[k];
  if (len < 2) return;
  const int32_t ne = min(len - 1, cap);
  const int32_t *row = edges + (int64_t)k * cap;
  for (int32_t i = threadIdx.x; i < ne; i += blockDim.x) {
    const int32_t e = row[i];
    if (e >= 0) atomicMin(&owner[e], j);
  }
}

// test: next[j] = 1 (and seeds[j] = the net's source) when an edge of net j
// is held by an earlier net of the round; 0 (seeds[j] = -1) otherwise.
// searches counts the nets flagged.
__global__ void snap_test_kernel(const int32_t *order, const int32_t *edges, const int32_t *lens, int32_t cap,
                                 const int32_t *active, const int32_t *owner, const int32_t *src, int32_t *next,
                                 int32_t *seeds, unsigned long long *searches) {
  __shared__ int hit;
  const int32_t j = blockIdx.x;
  if (threadIdx.x == 0) hit = 0;
  __syncthreads();
  const bool on = !active || active[j];
  if (on) {
    const int32_t k = order[j], len = lens[k];
    const int32_t ne = len < 2 ? 0 : min(len - 1, cap);
    const int32_t *row = edges + (int64_t)k * cap;
    for (int32_t i = threadIdx.x; i < ne; i += blockDim.x) {
      const int32_t e = row[i];
      if (e >= 0 && __ldcg(&owner[e]) < j) atomicOr(&hit, 1);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int f = on && hit;
    next[j] = f;
    seeds[j] = f ? src[j] : -1;
    if (f) atomicAdd(searches, 1ull);
  }
}

// reset: the round's edges back to kOwnerFree
__global__ void snap_reset_kernel(const int32_t *order, const int32_t *edges, const int32_t *lens, int32_t cap,
                                  const int32_t *active, int32_t *owner) {
  const int32_t j = blockIdx.x;
  if (active && !active[j]) return;
  const int32_t k = order[j], len = lens[k];
  if (len < 2) return;
  const int32_t ne = min(len - 1, cap);
  const int32_t *row = edges + (int64_t)k * cap;
  for (int32_t i = threadIdx.x; i < ne; i += blockDim.x) {
    const int32_t e = row[i];
    if (e >= 0) owner[e] = kOwnerFree;
  }
}

struct RouteBt {
  const float4 *w4;         // gathered in-edge weights (fresh inside the group's boxes)
  const int32_t *slot_eid;  // [4][N] in-edge id per slot
  const int32_t *vcol_eid;  // column vias: [2][nz][N] via in-edge ids by source layer (NULL: none)
  int64_t N;
  const uint32_t *dist;
  LatWalkGeom geom;
  // the group's nets: net ids, sources (-1: source outside its box), targets, boxes
  const int32_t *order, *src, *dst;
  const LatBox *boxes;
  const int32_t *active;  // NULL: every net of the group; else nets with active[j] != 0
  int32_t *net_nodes, *net_edges, *net_lens;
  int32_t cap;
  const int *search_err;  // the group search's error word
  int *route_err;
};

// Step 3, one warp per net of the group (block j: net order[j]).  The warp
// walks from the target to the source with lat_walk_warp (the parent rule of
// orsp_sssp, rank = node id = box-local order); the source (distance 0) ends
// the walk.  The walk never leaves the box: with shared distances the nodes
// outside it hold distances of other boxes or of earlier searches, and a box
// with its own slice (dbase >= 0) has distances for its cells only.  Then the lanes reverse
// the path and map each step u -> v to its CSR edge, the in-edge of v in the
// slot that u occupies (the lattice has no parallel edges, so this is the
// first CSR edge u -> v of path_to_edges).
__global__ void route_backtrace_kernel(RouteBt p) {
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x;
  if (p.active && !p.active[j]) return;
  const int32_t k = p.order[j];
  const int32_t src = p.src[j], dst = p.dst[j];
  const LatBox B = p.boxes[j];
  int32_t *nodes = p.net_nodes + (int64_t)k * p.cap;
  int32_t *edges = p.net_edges + (int64_t)k * p.cap;
  int32_t *len_out = p.net_lens + k;
  const int serr = *p.search_err;
  if (serr) {
    if (lane == 0) {
      atomicCAS(p.route_err, DEV_OK, serr);
      *len_out = 0;
    }
    return;
  }
  int len = 0, err = 0;
  int32_t x, y, z;
  lat_xyz(p.geom, dst, x, y, z);
  const bool dst_in = x >= B.x0 && x <= B.x1 && y >= B.y0 && y <= B.y1 && z >= B.z0 && z <= B.z1;
  // distances: by node id, or box-local rows of the box's own slice
  const bool own = B.dbase >= 0;
  const uint32_t *dist = own ? p.dist + B.dbase : p.dist;
  const int32_t rx = own ? B.x1 - B.x0 + 1 : p.geom.nx, ry = own ? B.y1 - B.y0 + 1 : p.geom.ny;
  const int32_t ox = own ? B.x0 : 0, oy = own ? B.y0 : 0, oz = own ? B.z0 : 0;
  auto dget = [dist, rx, ry, ox, oy, oz](int32_t a, int32_t b, int32_t c) {
    return __ldcg(&dist[((int64_t)(c - oz) * ry + (b - oy)) * rx + (a - ox)]);
  };
  const unsigned dv = (src >= 0 && dst_in) ? dget(x, y, z) : ORSP_INF_BITS;
  if (dv != ORSP_INF_BITS && dst != src) {
    auto at_src = [src](int64_t v, unsigned d) { return v == src && d == 0u; };
    len = lat_walk_warp(p.geom, B, p.w4, dget, at_src, x, y, z, dv, nodes, p.cap);
    if (len == -1) err = DEV_ERR_PATH_OVERFLOW;
    else if (len < 0) err = DEV_ERR_INTERNAL;
    if (err) len = 0;
  }
  __syncwarp();
  if (err) {
    if (lane == 0) {
      atomicCAS(p.route_err, DEV_OK, err);
      *len_out = 0;
    }
    return;
  }
  for (int i = lane; i < len / 2; i += 32) {
    const int a = nodes[i], z = nodes[len - 1 - i];
    nodes[i] = z;
    nodes[len - 1 - i] = a;
  }
  __syncwarp();
  for (int i = lane; i < len - 1; i += 32) {
    const int32_t u = nodes[i], w = nodes[i + 1];
    const int64_t plane = (int64_t)p.geom.nx * p.geom.ny;
    const int64_t zu = u / plane, zw = w / plane;
    if (p.vcol_eid && zu != zw)  // a column via: the first CSR edge u -> w (the smaller id)
      edges[i] = __ldg(&p.vcol_eid[zu * p.N + w]);
    else
      edges[i] = __ldg(&p.slot_eid[(int64_t)lat_edge_slot(p.geom, u, w) * p.N + w]);
  }
  __syncwarp();
  if (lane == 0) *len_out = len;
}

bool box_ok(const orsp::Graph *g, const int32_t *b) {
  return b[0] >= 0 && b[2] >= 0 && b[4] >= 0 && b[1] < g->nx && b[3] < g->ny && b[5] < g->nz && b[0] <= b[1] &&
         b[2] <= b[3] && b[4] <= b[5];
}

bool boxes_meet(const int32_t *a, const int32_t *b) {
  return a[0] <= b[1] && b[0] <= a[1] && a[2] <= b[3] && b[2] <= a[3] && a[4] <= b[5] && b[4] <= a[5];
}

bool node_in(const orsp::Graph *g, int32_t u, const int32_t *b) {
  const int64_t plane = (int64_t)g->nx * g->ny;
  const int32_t z = (int32_t)(u / plane), r = (int32_t)(u - z * plane), y = r / g->nx, x = r - y * g->nx;
  return x >= b[0] && x <= b[1] && y >= b[2] && y <= b[3] && z >= b[4] && z <= b[5];
}

constexpr int32_t kMaxGroup = 1024;
constexpr int32_t kGraphGroups = 64;  // groups per captured CUDA graph

}  // namespace

using namespace orsp;

// The routing loop of orsp_route_nets (repair < 0: groups of pairwise
// disjoint boxes) and orsp_route_nets_snapshot (repair >= 0: groups whose
// boxes may overlap, searched on one cost snapshot, then `repair` rounds
// for the nets that share an edge with an earlier net of their group).
static int route_nets_impl(orsp_graph *g, int32_t M, const int32_t *src_h, const int32_t *dst_h,
                           const int32_t *box_h, int32_t K, const int32_t *order_h, int32_t G,
                           const int32_t *group_ptr_h, int32_t repair, int32_t *net_nodes_d, int32_t *net_edges_d,
                           int32_t path_cap, int32_t *net_lens_d, float *cost_d, const float *base_d,
                           int32_t *usage_d, float *present_d, const float *cap_d, const float *hist_d,
                           float pres_fac, float hist_w, float via_mult, float base_w, int32_t jitter,
                           int64_t *searches_out, uintptr_t stream) {
  const bool snap = repair >= 0;
  if (searches_out) *searches_out = 0;
  if (!g || M < 0 || K < 0 || path_cap < 2) { set_error("route_nets: bad sizes"); return ORSP_ERR_ARG; }
  if (snap && repair > 64) { set_error("route_nets: at most 64 repair rounds"); return ORSP_ERR_ARG; }
  if (K == 0) return ORSP_OK;
  if (!src_h || !dst_h || !box_h || !order_h || !net_nodes_d || !net_edges_d || !net_lens_d || !cost_d ||
      !base_d || !usage_d || !cap_d || !hist_d) {
    set_error("route_nets: NULL array");
    return ORSP_ERR_ARG;
  }
  if (!g->lattice_ok) { set_error("route_nets: needs a graph recognised as an H/V lattice"); return ORSP_ERR_ARG; }
  // groups: [group_ptr[q], group_ptr[q+1]) of the order; NULL = one net each
  std::vector<int32_t> gp;
  if (group_ptr_h) {
    if (G < 1 || group_ptr_h[0] != 0 || group_ptr_h[G] != K) {
      set_error("route_nets: group_ptr must run from 0 to K");
      return ORSP_ERR_ARG;
    }
    gp.assign(group_ptr_h, group_ptr_h + G + 1);
  } else {
    gp.resize((size_t)K + 1);
    for (int32_t i = 0; i <= K; ++i) gp[i] = i;
  }
  const int32_t ngroups = (int32_t)gp.size() - 1;
  std::vector<int32_t> seen((size_t)M, 0);
  for (int32_t i = 0; i < K; ++i) {
    const int32_t k = order_h[i];
    if (k < 0 || k >= M) { set_error("route_nets: order entry out of range"); return ORSP_ERR_ARG; }
    if (seen[k]++) { set_error("route_nets: a net appears twice in the order"); return ORSP_ERR_ARG; }
    if (src_h[k] < 0 || src_h[k] >= g->N || dst_h[k] < 0 || dst_h[k] >= g->N) {
      set_error("route_nets: src/dst out of range");
      return ORSP_ERR_ARG;
    }
    if (!box_ok(g, box_h + 6 * (int64_t)k)) {
      set_error("route_nets: box outside the lattice or empty");
      return ORSP_ERR_ARG;
    }
    if (!lattice_tile_fits(box_h[6 * (int64_t)k + 5] - box_h[6 * (int64_t)k + 4] + 1)) {
      set_error("route_nets: box deeper than a lattice tile holds (orsp_lattice_max_layers)");
      return ORSP_ERR_ARG;
    }
  }
  for (int32_t q = 0; q < ngroups; ++q) {
    const int32_t a = gp[q], b = gp[q + 1];
    if (b < a || b - a > kMaxGroup) { set_error("route_nets: group sizes must be 0..1024"); return ORSP_ERR_ARG; }
    if (snap) continue;
    for (int32_t i = a; i < b; ++i)
      for (int32_t j = a; j < i; ++j)
        if (boxes_meet(box_h + 6 * (int64_t)order_h[i], box_h + 6 * (int64_t)order_h[j])) {
          set_error("route_nets: boxes of one group must be pairwise disjoint");
          return ORSP_ERR_ARG;
        }
  }
  ORSP_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = (cudaStream_t)stream;
  if (!g->dist) ORSP_CUDA(cudaMalloc(&g->dist, (size_t)g->N * 4));
  if (!g->route_ws) ORSP_CUDA(cudaMalloc(&g->route_ws, 256));
  // per-call tables in route order: net id, source (-1 when outside its box),
  // target, box (LatBox; tile ids restart at 0 in each group).  Staged in
  // pinned memory and copied once; the call synchronises before returning,
  // so the staging buffer is free again for the next call.
  const size_t need = (size_t)K * (3 * sizeof(int32_t) + sizeof(LatBox)) + 256;
  if (g->route_tab_bytes < need) {
    cudaFree(g->route_tab_d);
    if (g->route_tab_h) cudaFreeHost(g->route_tab_h);
    g->route_tab_d = nullptr;
    g->route_tab_h = nullptr;
    g->route_tab_bytes = 0;
    ORSP_CUDA(cudaMalloc(&g->route_tab_d, need));
    ORSP_CUDA(cudaMallocHost(&g->route_tab_h, need));
    g->route_tab_bytes = need;
  }
  char *th = (char *)g->route_tab_h;
  int32_t *t_order = (int32_t *)th;
  int32_t *t_src = t_order + K;
  int32_t *t_dst = t_src + K;
  LatBox *t_box = (LatBox *)(((uintptr_t)(t_dst + K) + 63) & ~(uintptr_t)63);
  std::vector<int32_t> boxes_o((size_t)K * 6);
  for (int32_t i = 0; i < K; ++i) {
    const int32_t k = order_h[i];
    const int32_t *b = box_h + 6 * (int64_t)k;
    t_order[i] = k;
    t_src[i] = node_in(g, src_h[k], b) ? src_h[k] : -1;
    t_dst[i] = dst_h[k];
    for (int c = 0; c < 6; ++c) boxes_o[(size_t)i * 6 + c] = b[c];
  }
  int64_t max_tiles = 1;
  std::vector<int64_t> gcells((size_t)ngroups, 0);  // snapshot groups: cells of the group's own slices
  int64_t max_cells = 0;
  for (int32_t q = 0; q < ngroups; ++q) {
    const int32_t a = gp[q], b = gp[q + 1];
    max_tiles = std::max<int64_t>(max_tiles, make_lat_boxes(boxes_o.data() + (size_t)a * 6, b - a, t_box + a));
    if (snap) {
      for (int32_t i = a; i < b; ++i) {
        const int32_t *bx = boxes_o.data() + (size_t)i * 6;
        t_box[i].dbase = gcells[q];
        gcells[q] += (int64_t)(bx[1] - bx[0] + 1) * (bx[3] - bx[2] + 1) * (bx[5] - bx[4] + 1);
      }
      max_cells = std::max(max_cells, gcells[q]);
    }
  }
  const size_t off_box = (size_t)((char *)t_box - th);
  char *td = (char *)g->route_tab_d;
  const int32_t *d_order = (const int32_t *)td;
  const int32_t *d_src = d_order + K;
  const int32_t *d_dst = d_src + K;
  const LatBox *d_box = (const LatBox *)(td + off_box);
  ORSP_CUDA(cudaMemcpyAsync(td, th, off_box + (size_t)K * sizeof(LatBox), cudaMemcpyHostToDevice, st));
  int rc = reserve_lattice_ws(g, max_tiles);
  if (rc) return rc;
  int *route_err = (int *)g->route_ws;
  unsigned long long *repair_count = (unsigned long long *)((char *)g->route_ws + 8);
  ORSP_CUDA(cudaMemsetAsync(g->route_ws, 0, 16, st));
  if (snap) {
    if ((size_t)max_cells * 4 > g->route_pdist_bytes) {
      cudaFree(g->route_pdist);
      g->route_pdist = nullptr;
      g->route_pdist_bytes = 0;
      ORSP_CUDA(cudaMalloc(&g->route_pdist, (size_t)max_cells * 4));
      g->route_pdist_bytes = (size_t)max_cells * 4;
    }
    if (!g->route_flags) ORSP_CUDA(cudaMalloc(&g->route_flags, (size_t)3 * kMaxGroup * sizeof(int32_t)));
    if (!g->route_owner) {
      ORSP_CUDA(cudaMalloc(&g->route_owner, (size_t)g->E * sizeof(int32_t)));
      ORSP_CUDA(cudaMemsetAsync(g->route_owner, 0x7f, (size_t)g->E * sizeof(int32_t), st));
    }
  }

  LiveParams lp{usage_d, present_d, base_d, cap_d, hist_d, pres_fac, hist_w, via_mult, base_w, jitter, cost_d};
  LatWalkGeom geom{};
  geom.nx = g->nx;
  geom.ny = g->ny;
  geom.nz = g->nz;
  for (int z = 0; z < 64; ++z) geom.axis[z] = z < g->nz ? g->layer_axis[z] : 0;
  geom.wcol = g->cvia ? g->wcol : nullptr;
  geom.nzp = (g->nz + 3) & ~3;
  // One snapshot group, enqueued on the stream: rounds of steps 1-4 with
  // separate usage and cost passes; round 0 routes every net of the group on
  // the costs after the group's rip-ups, each later round the nets that the
  // previous round's test flagged (the others' searches have no seed and
  // their steps return at once).
  auto enqueue_snapshot = [&](int32_t q) -> int {
    const int32_t a = gp[q], n = gp[q + 1] - gp[q];
    if (n == 0) return ORSP_OK;
    int32_t *flags[2] = {g->route_flags, g->route_flags + kMaxGroup};
    int32_t *seeds = g->route_flags + 2 * kMaxGroup;
    const int32_t *act = nullptr;
    const int32_t *seed_r = d_src + a;
    for (int32_t r = 0; r <= repair; ++r) {
      route_commit_kernel<<<n, 256, 0, st>>>(d_order + a, net_edges_d, net_lens_d, path_cap, -1, 1, act, lp);
      ORSP_CUDA(cudaGetLastError());
      route_commit_kernel<<<n, 256, 0, st>>>(d_order + a, net_edges_d, net_lens_d, path_cap, -1, 2, act, lp);
      ORSP_CUDA(cudaGetLastError());
      LatOptions opt;
      opt.private_dist = true;
      opt.private_count = gcells[q];
      opt.copy_ctl = false;
      opt.active = act;  // repair rounds: only the flagged boxes are gathered and reset
      int rc = run_lattice_boxes(g, cost_d, n, seed_r, nullptr, n, boxes_o.data() + (size_t)a * 6, d_box + a,
                                 g->route_pdist, st, &opt);
      if (rc) return rc;
      RouteBt bt{};
      bt.w4 = (const float4 *)g->wslot;
      bt.slot_eid = g->slot_eid;
      bt.vcol_eid = g->cvia ? g->vcol_eid : nullptr;
      bt.N = g->N;
      bt.dist = g->route_pdist;
      bt.geom = geom;
      bt.order = d_order + a;
      bt.src = d_src + a;
      bt.dst = d_dst + a;
      bt.boxes = d_box + a;
      bt.active = act;
      bt.net_nodes = net_nodes_d;
      bt.net_edges = net_edges_d;
      bt.net_lens = net_lens_d;
      bt.cap = path_cap;
      bt.search_err = opt.err_d;
      bt.route_err = route_err;
      route_backtrace_kernel<<<n, 32, 0, st>>>(bt);
      ORSP_CUDA(cudaGetLastError());
      route_commit_kernel<<<n, 256, 0, st>>>(d_order + a, net_edges_d, net_lens_d, path_cap, 1, 1, act, lp);
      ORSP_CUDA(cudaGetLastError());
      route_commit_kernel<<<n, 256, 0, st>>>(d_order + a, net_edges_d, net_lens_d, path_cap, 1, 2, act, lp);
      ORSP_CUDA(cudaGetLastError());
      if (r == repair) break;
      int32_t *next = flags[r & 1];
      snap_mark_kernel<<<n, 256, 0, st>>>(d_order + a, net_edges_d, net_lens_d, path_cap, act, g->route_owner);
      ORSP_CUDA(cudaGetLastError());
      snap_test_kernel<<<n, 256, 0, st>>>(d_order + a, net_edges_d, net_lens_d, path_cap, act, g->route_owner,
                                          d_src + a, next, seeds, repair_count);
      ORSP_CUDA(cudaGetLastError());
      snap_reset_kernel<<<n, 256, 0, st>>>(d_order + a, net_edges_d, net_lens_d, path_cap, act, g->route_owner);
      ORSP_CUDA(cudaGetLastError());
      act = next;
      seed_r = seeds;
    }
    return ORSP_OK;
  };
  // Steps 1-4 of one group, enqueued on the stream.
  auto enqueue_group = [&](int32_t q) -> int {
    if (snap) return enqueue_snapshot(q);
    int rc = ORSP_OK;
    const int32_t a = gp[q], n = gp[q + 1] - gp[q];
    if (n == 0) return ORSP_OK;
    route_commit_kernel<<<n, 256, 0, st>>>(d_order + a, net_edges_d, net_lens_d, path_cap, -1, 0, nullptr, lp);
    ORSP_CUDA(cudaGetLastError());
    LatOptions opt;
    opt.fill_box_only = true;
    opt.copy_ctl = false;
    rc = run_lattice_boxes(g, cost_d, n, d_src + a, nullptr, n, boxes_o.data() + (size_t)a * 6, d_box + a, g->dist,
                           st, &opt);
    if (rc) return rc;
    RouteBt bt{};
    bt.w4 = (const float4 *)g->wslot;
    bt.slot_eid = g->slot_eid;
    bt.vcol_eid = g->cvia ? g->vcol_eid : nullptr;
    bt.N = g->N;
    bt.dist = g->dist;
    bt.geom = geom;
    bt.order = d_order + a;
    bt.src = d_src + a;
    bt.dst = d_dst + a;
    bt.boxes = d_box + a;
    bt.net_nodes = net_nodes_d;
    bt.net_edges = net_edges_d;
    bt.net_lens = net_lens_d;
    bt.cap = path_cap;
    bt.search_err = opt.err_d;
    bt.route_err = route_err;
    route_backtrace_kernel<<<n, 32, 0, st>>>(bt);
    ORSP_CUDA(cudaGetLastError());
    route_commit_kernel<<<n, 256, 0, st>>>(d_order + a, net_edges_d, net_lens_d, path_cap, 1, 0, nullptr, lp);
    ORSP_CUDA(cudaGetLastError());
    return rc;
  };
  // The groups are captured into CUDA graphs of up to kGraphGroups groups
  // each; a chunk's graph is launched as soon as it is instantiated, so the
  // GPU runs chunk k while the host captures chunk k + 1.  A chunk whose
  // capture or instantiation fails is enqueued directly instead (same
  // launches, same results).  ORSP_ROUTE_GRAPH=0 enqueues every group
  // directly.
  const char *ge = getenv("ORSP_ROUTE_GRAPH");
  bool use_graph = !(ge && ge[0] == '0');
  // Graphs are captured on a stream of the library's own (the caller's may be
  // the legacy default stream, which cannot be captured), ordered after the
  // caller's stream on entry and before it on exit.
  const cudaStream_t caller = st;
  if (use_graph) {
    if (!g->route_stream) ORSP_CUDA(cudaStreamCreateWithFlags(&g->route_stream, cudaStreamNonBlocking));
    for (cudaEvent_t &e : g->route_ev)
      if (!e) ORSP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ORSP_CUDA(cudaEventRecord(g->route_ev[0], caller));
    ORSP_CUDA(cudaStreamWaitEvent(g->route_stream, g->route_ev[0], 0));
    st = g->route_stream;
  }
  std::vector<cudaGraphExec_t> execs;
  int rc_loop = ORSP_OK;
  for (int32_t q0 = 0; q0 < ngroups && rc_loop == ORSP_OK; q0 += kGraphGroups) {
    const int32_t q1 = std::min(ngroups, q0 + kGraphGroups);
    bool done = false;
    bool capturing = false;
    if (use_graph) {
      capturing = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (!capturing) (void)cudaGetLastError();  // enqueue directly, with no error left pending
    }
    if (capturing) {
      int rc_c = ORSP_OK;
      for (int32_t q = q0; q < q1 && rc_c == ORSP_OK; ++q) rc_c = enqueue_group(q);
      cudaGraph_t graph = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(st, &graph);
      cudaGraphExec_t exec = nullptr;
      if (rc_c == ORSP_OK && ce == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
        if (cudaGraphLaunch(exec, st) == cudaSuccess) done = true;
        execs.push_back(exec);
      }
      if (graph) cudaGraphDestroy(graph);
      if (!done) (void)cudaGetLastError();  // clear the failed capture's error
    }
    for (int32_t q = q0; !done && q < q1 && rc_loop == ORSP_OK; ++q) rc_loop = enqueue_group(q);
  }
  if (rc_loop != ORSP_OK) {
    cudaStreamSynchronize(st);
    for (cudaGraphExec_t e : execs) cudaGraphExecDestroy(e);
    return rc_loop;
  }
  if (use_graph) {  // the caller's stream continues after the last group
    ORSP_CUDA(cudaEventRecord(g->route_ev[1], st));
    ORSP_CUDA(cudaStreamWaitEvent(caller, g->route_ev[1], 0));
    st = caller;
  }
  int *err_h = (int *)g->pinned + 32;  // [0] error word, [2..3] repair searches
  ORSP_CUDA(cudaMemcpyAsync(err_h, g->route_ws, 16, cudaMemcpyDeviceToHost, st));
  const cudaError_t se = cudaStreamSynchronize(st);
  for (cudaGraphExec_t e : execs) cudaGraphExecDestroy(e);
  ORSP_CUDA(se);
  if (searches_out) {
    unsigned long long extra = 0;
    memcpy(&extra, err_h + 2, sizeof(extra));
    *searches_out = (int64_t)K + (int64_t)extra;
  }
  if (*err_h) return dev_status_to_orsp(*err_h);
  return ORSP_OK;
}

extern "C" int orsp_route_nets(orsp_graph *g, int32_t M, const int32_t *src_h, const int32_t *dst_h,
                               const int32_t *box_h, int32_t K, const int32_t *order_h, int32_t G,
                               const int32_t *group_ptr_h, int32_t *net_nodes_d, int32_t *net_edges_d,
                               int32_t path_cap, int32_t *net_lens_d, float *cost_d, const float *base_d,
                               int32_t *usage_d, float *present_d, const float *cap_d, const float *hist_d,
                               float pres_fac, float hist_w, float via_mult, float base_w, int32_t jitter,
                               uintptr_t stream) {
  return route_nets_impl(g, M, src_h, dst_h, box_h, K, order_h, G, group_ptr_h, -1, net_nodes_d, net_edges_d,
                         path_cap, net_lens_d, cost_d, base_d, usage_d, present_d, cap_d, hist_d, pres_fac, hist_w,
                         via_mult, base_w, jitter, nullptr, stream);
}

extern "C" int orsp_route_nets_snapshot(orsp_graph *g, int32_t M, const int32_t *src_h, const int32_t *dst_h,
                                        const int32_t *box_h, int32_t K, const int32_t *order_h, int32_t G,
                                        const int32_t *group_ptr_h, int32_t repair_rounds, int32_t *net_nodes_d,
                                        int32_t *net_edges_d, int32_t path_cap, int32_t *net_lens_d, float *cost_d,
                                        const float *base_d, int32_t *usage_d, float *present_d, const float *cap_d,
                                        const float *hist_d, float pres_fac, float hist_w, float via_mult,
                                        float base_w, int32_t jitter, int64_t *searches_out, uintptr_t stream) {
  if (repair_rounds < 0) {
    set_error("route_nets_snapshot: repair_rounds must be >= 0");
    return ORSP_ERR_ARG;
  }
  return route_nets_impl(g, M, src_h, dst_h, box_h, K, order_h, G, group_ptr_h, repair_rounds, net_nodes_d,
                         net_edges_d, path_cap, net_lens_d, cost_d, base_d, usage_d, present_d, cap_d, hist_d,
                         pres_fac, hist_w, via_mult, base_w, jitter, searches_out, stream);
}
