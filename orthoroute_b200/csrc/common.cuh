// Shared device helpers for liborsp: error plumbing, bounded waits, warp
// aggregation and the graph context.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "orsp.h"

#define ORSP_INF_BITS 0x7f800000u
#define ORSP_FULL_MASK 0xffffffffu

// Device-side error codes written into a status word; mapped to ORSP_ERR_*.
#define DEV_OK 0
#define DEV_ERR_TIMEOUT 1
#define DEV_ERR_OVERFLOW 2
#define DEV_ERR_INTERNAL 3
#define DEV_ERR_PATH_OVERFLOW 4

namespace orsp {

// Thread-local message of the last failure (orsp_last_error).
void set_error(const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
int dev_status_to_orsp(int dev);

#define ORSP_CUDA(call)                                   \
  do {                                                    \
    cudaError_t _e = (call);                              \
    if (_e != cudaSuccess) return orsp::cuda_fail(_e, #call); \
  } while (0)

struct Graph {
  int device = 0;
  int32_t N = 0;
  int64_t E = 0;
  int32_t nx = 0, ny = 0, nz = 0;
  int32_t max_degree = 0;
  int32_t max_in_degree = 0;
  int num_sms = 0;
  // forward CSR (device)
  int32_t *indptr = nullptr;
  int32_t *indices = nullptr;
  // transposed CSR: for node v, in-edges k in [rptr[v], rptr[v+1]) come from
  // rsrc[k] through forward edge reid[k]; sorted by (source, edge id).
  int32_t *rptr = nullptr;
  int32_t *rsrc = nullptr;
  int32_t *reid = nullptr;
  // single-search workspace (lazily allocated)
  uint32_t *dist = nullptr;
  int2 *near_q[2] = {nullptr, nullptr};
  int2 *far_q[2] = {nullptr, nullptr};
  int64_t qcap = 0, fcap = 0;
  void *ctl = nullptr;     // device control block of the grid search
  void *ctl_h = nullptr;   // pinned host mirror
  // batched-search workspace (lazily grown)
  void *batch_ws = nullptr;
  size_t batch_ws_bytes = 0;
  void *batch_ctl = nullptr;
  // misc scratch
  void *scratch = nullptr;
  size_t scratch_bytes = 0;
  void *pinned = nullptr;  // small pinned host buffer for results
  float *auto_delta = nullptr;  // [2] device bucket widths chosen by the library (single, batch)
  int32_t *box_g2r = nullptr;   // [N] box ROI map for box searches on the generic path (lazy)
  int32_t *edge_src = nullptr;  // [E] source node of each edge (lazy, bookkeeping kernels)
  // routing loop (orsp_route.cu): error word, per-call net tables (device)
  // and their pinned staging copy
  void *route_ws = nullptr;
  // batched search: tuning plan (orsp_batch_set_plan), item lists, and the
  // distance arena and tile tables of boxes searched by tile sweeps
  int32_t plan_nb = 0;
  int64_t plan_max_nodes[8];
  int32_t plan_impl[8], plan_tile[8], plan_ctas[8];
  float plan_delta[8];
  int32_t *batch_idx = nullptr;
  size_t batch_idx_bytes = 0;
  uint32_t *blat_dist = nullptr;
  size_t blat_dist_bytes = 0;
  void *blat_tab_d = nullptr;
  void *blat_tab_h = nullptr;
  size_t blat_tab_bytes = 0;
  void *route_tab_d = nullptr;
  void *route_tab_h = nullptr;
  size_t route_tab_bytes = 0;
  cudaStream_t route_stream = nullptr;    // orsp_route_nets: stream its graphs are captured on
  cudaEvent_t route_ev[2] = {nullptr, nullptr};  // ordering with the caller's stream
  // snapshot groups (orsp_route_nets_snapshot): the boxes' own distance
  // slices, per-net round flags and seeds, and the lowest group rank per edge
  uint32_t *route_pdist = nullptr;
  size_t route_pdist_bytes = 0;
  int32_t *route_flags = nullptr;  // [3][kMaxGroup]: two rounds of flags, seeds
  int32_t *route_owner = nullptr;  // [E], 0x7f7f7f7f between uses
  // H/V lattice description, set when every CSR edge is a unit step along the
  // layer's routing axis or a via to an adjacent layer (see orsp_lattice.cu)
  bool lattice_ok = false;
  int8_t layer_axis[64] = {};     // 0: no planar edges, 1: x, 2: y
  int32_t *slot_eid = nullptr;    // [4][N] in-edge id per slot (-1 absent)
  float *wslot = nullptr;         // [N] float4: gathered in-edge weights per node, by slot
  // column vias (the reference's Lattice3D: vias between any two layers of a
  // column, up to two parallel edges each): slots 2 and 3 stay empty and
  // every via in-edge of node v from layer za is in vcol_eid[(k * nz + za) * N
  // + v] (k = 0, 1: the parallel edges, smaller id first, -1 absent); wcol
  // [nz][N] holds the gathered weight, the smaller of the parallel edges'
  bool cvia = false;
  int32_t *vcol_eid = nullptr;
  float *wcol = nullptr;
  void *lat_ws = nullptr;         // tile lists, stamps and control block
  size_t lat_ws_bytes = 0;
  void *lat_ctl_h = nullptr;      // pinned mirror of the control block
  void *lat_box_d = nullptr;      // tile table of a single-box search
  // ROI searches (orsp_sssp_roi_nodes, ROI-masked tile sweeps): a global_to_roi
  // map kept at -1 between calls (each call scatters its ROI in and clears it
  // again), a sink mask kept at 0 the same way, the ROI's bounding box as it is
  // reduced on the device, and a one-int seed slot
  int32_t *roi_map = nullptr;
  uint8_t *sink_mask = nullptr;
  int *roi_bb = nullptr;
  int32_t *seed_one = nullptr;
  // gathered-weight cache (orsp_graph_cost_generation): the cost array and
  // caller-declared generation the whole of wslot was last gathered from
  // (generation 0: not reusable), and the declaration for the next search
  const float *w4_cost = nullptr;
  uint64_t w4_gen = 0;
  const float *decl_cost = nullptr;
  uint64_t decl_gen = 0;
};

// Optional timing of a search kernel (CUDA events on the launching stream),
// enabled by orsp_profile_enable for roofline reporting.
struct KernelTimer {
  bool on = false;
  bool pending = false;
  cudaEvent_t a = nullptr, b = nullptr;
  float last_ms = 0.0f;
};
extern KernelTimer g_timer;
// rounds and tile visits of the last lattice search (orsp_profile_counters)
extern int64_t g_counters[8];

int ensure_scratch(Graph *g, size_t bytes);
// Bucket width chosen on the device when the caller passes delta == 0: twice
// the mean of a strided sample (<= 65536 entries) of the finite costs, 1.0 if
// none is finite.  Writes *out; never blocks the host.  (orsp_sssp.cu)
int launch_auto_delta(const float *cost_d, int64_t E, float *out_d, cudaStream_t st);
// orsp_lattice.cu
int analyze_lattice(Graph *g, const int32_t *indptr_h, const int32_t *indices_h);
void free_lattice(Graph *g);
// One box of a lattice search, with its tiles' place in the launch's tile
// numbering (tiles of TX x TY columns, x fastest, box after box).
struct LatBox {
  int32_t x0, x1, y0, y1, z0, z1;
  int32_t ntx, nty;  // tiles along x and y
  int32_t tile0;     // id of the box's first tile
  int32_t pad;       // the box's distance slice for the TMA staging (LatOptions::tma_slices)
  int64_t dbase;     // -1: distances indexed by node id in the shared array;
                     // >= 0: the box's own slice, box-local row-major from here
};
// Tile width of the lattice search (ORSP_LAT_TILE: 16 or 32); the height is 16.
int lattice_tile_w();
// Whether a tile of nzb layers at tile width tile_w (0: lattice_tile_w())
// fits in shared memory.
bool lattice_tile_fits(int nzb, int tile_w = 0);
// Fills out[i] for boxes_h[6i..6i+5] (tile width tile_w, 0 = lattice_tile_w(),
// shared distances) and returns the total tile count.
int64_t make_lat_boxes(const int32_t *boxes_h, int32_t nbox, LatBox *out, int tile_w = 0);
struct LatOptions {
  int tile_w = 0;              // tile width (0: lattice_tile_w()); the tables must use the same
  bool private_dist = false;   // boxes have their own slices (dbase >= 0): seed i starts box i, and
                               // `dist` is the slice arena of private_count entries, all reset
  int64_t private_count = 0;
  bool fill_box_only = false;  // reset distances inside the boxes only (the caller's backtrace checks the box)
  bool copy_ctl = true;        // copy the control block to the pinned mirror (finish_lattice_search)
  int *err_d = nullptr;        // out: device address of the launch's error word
  int blocks_per_sm = 0;       // CTAs per SM (0: one); ORSP_LAT_BLOCKS_PER_SM overrides
  int spec = 0;                // 1: the warp-specialised schedule; ORSP_LAT_SPEC overrides
  int64_t tma_slices = 0;      // > 0: every box is the whole lattice, box j's distances in slice j of N
                               // cells from `dist` (LatBox.pad = j); allows the TMA staging
  const int32_t *active = nullptr;  // private_dist, device flags: a box with active[j] == 0 has no seed, and
                                    // its weights and distances are neither gathered nor reset
};
// One box (nullptr: the whole lattice).  Stages its tile table through the
// graph's pinned buffer, so the calling entry point must synchronise before
// it returns.
int run_lattice_search(Graph *g, const float *cost_d, int32_t nseeds, const int32_t *seeds_d,
                       const float *seed_cost_d, const int32_t *box, uint32_t *dist, cudaStream_t st,
                       LatOptions *opt = nullptr);
// Several pairwise disjoint boxes searched in one launch, sharing the
// distance array: boxes_h (host, 6 ints per box) sizes the launch, lboxes_d
// (device, from make_lat_boxes) is what the kernel reads and must stay valid
// until the launch has run.  Each seed starts in the box that contains it.
int run_lattice_boxes(Graph *g, const float *cost_d, int32_t nseeds, const int32_t *seeds_d,
                      const float *seed_cost_d, int32_t nbox, const int32_t *boxes_h, const LatBox *lboxes_d,
                      uint32_t *dist, cudaStream_t st, LatOptions *opt = nullptr);
// Grows the lattice workspace for launches of up to `ntiles` tiles, so that
// later launches never reallocate it (a reallocation synchronises).
int reserve_lattice_ws(Graph *g, int64_t ntiles);
int finish_lattice_search(Graph *g, int32_t *rounds_h);
// One search on a recognised lattice restricted to a node-set ROI: nodes with
// roi_map_d[v] >= 0 (roi_map_d NULL: every node), with the out-edges of the
// nodes marked in sink_d (may be NULL) blocked.  The ROI's bounding box is
// reduced on the device, from the node list roi_nodes_d[0..n_roi) when given,
// else from roi_map_d; the in-edge weights are gathered inside that box with
// every edge that leaves the ROI, enters it from outside or leaves a sink set
// to +inf, and the tile sweeps run over the box.  `dist` is reset to +inf
// everywhere, so a backtrace may walk it with the whole lattice as its box.
// Seeds outside the ROI are ignored.  finish_lattice_search reports the status.
int run_lattice_roi(Graph *g, const float *cost_d, int32_t nseeds, const int32_t *seeds_d,
                    const float *seed_cost_d, const int32_t *roi_map_d, const int32_t *roi_nodes_d,
                    int64_t n_roi, const uint8_t *sink_d, uint32_t *dist, cudaStream_t st);
// One search over a node-list ROI whose global_to_roi map is roi_map_d (ROI
// index = rank, -1 outside), by one CTA of the batch kernel; *len_h gets the
// batch kernel's path_len (nodes, 0 = no path, < 0 a per-search status).
int run_roi_nodes_cta(Graph *g, const float *cost_d, const int32_t *src_d, const int32_t *dst_d,
                      const int32_t *roi_map_d, const int32_t *roi_nodes_d, int64_t n_roi, int32_t *path_out_d,
                      int32_t path_cap, int32_t *path_len_d, cudaStream_t st, int32_t *len_h);
// The ROI map and sink mask of orsp_sssp_roi_nodes / orsp_sssp_multi (lazily
// allocated, -1 / 0 everywhere).
int ensure_roi_arrays(Graph *g);

}  // namespace orsp

struct orsp_graph : public orsp::Graph {};

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long dev_globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned ld_cg_u32(const unsigned *p) { return __ldcg(p); }

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Grid-wide barrier for cooperative launches with a bounded wait: a block that
// waits longer than timeout_ns records DEV_ERR_TIMEOUT and stops waiting, so a
// logic error can never hang the GPU.  Every block must call it the same
// number of times (the callers make all loop decisions from values read after
// the barrier, which no block modifies until the next barrier).
struct GridBarrier {
  unsigned count;
  unsigned gen;
};

__device__ __forceinline__ void grid_barrier(GridBarrier *b, unsigned nblocks,
                                             int *err,
                                             unsigned long long timeout_ns) {
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned g = ld_acquire_u32(&b->gen);
    __threadfence();
    unsigned prev = atomicAdd(&b->count, 1u);
    if (prev == nblocks - 1) {
      atomicExch(&b->count, 0u);
      __threadfence();
      atomicAdd(&b->gen, 1u);
    } else {
      unsigned long long t0 = dev_globaltimer();
      unsigned spins = 0;
      while (ld_acquire_u32(&b->gen) == g) {
        if ((++spins & 63u) == 0 && dev_globaltimer() - t0 > timeout_ns) {
          atomicCAS(err, DEV_OK, DEV_ERR_TIMEOUT);
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// Warp-aggregated append of one int2 item per lane with `flag` set; `counter`
// may live in global or shared memory.  Must be called by all 32 lanes.
// Items that do not fit below `cap` are dropped (never written) and raise
// DEV_ERR_OVERFLOW in *err.
__device__ __forceinline__ void warp_append(int2 *buf, unsigned *counter,
                                            int64_t cap, bool flag, int2 item,
                                            int *err) {
  unsigned m = __ballot_sync(ORSP_FULL_MASK, flag);
  if (m == 0) return;
  int lane = threadIdx.x & 31;
  int leader = __ffs(m) - 1;
  unsigned base = 0;
  if (lane == leader) base = atomicAdd(counter, (unsigned)__popc(m));
  base = __shfl_sync(ORSP_FULL_MASK, base, leader);
  if (flag) {
    unsigned idx = base + __popc(m & lanemask_lt());
    if ((int64_t)idx < cap) {
      __stcg(&buf[idx], item);
    } else {
      atomicCAS(err, DEV_OK, DEV_ERR_OVERFLOW);
    }
  }
}

__device__ __forceinline__ unsigned warp_min_u32(unsigned v) {
  return __reduce_min_sync(ORSP_FULL_MASK, v);
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long t = __shfl_xor_sync(ORSP_FULL_MASK, v, o);
    v = t < v ? t : v;
  }
  return v;
}

__device__ __forceinline__ float bits_f(unsigned u) { return __uint_as_float(u); }
__device__ __forceinline__ unsigned f_bits(float f) { return __float_as_uint(f); }
