// Lattice search: single-source shortest paths on the H/V routing lattice by
// shared-memory tile sweeps.
//
// The generic grid search (orsp_sssp.cu) needs one grid-wide round per hop of
// the shortest-path tree (about 1 400 rounds on a 1000 x 1000 grid, each a
// dependent memory chain plus a grid barrier).  On the routing lattice every
// node has at most four in-edges - the two neighbours along its layer's
// routing axis (x on H layers, y on V layers) and the vias to the layers above
// and below - so a tile of TX x TY columns (all layers) can be relaxed to a
// local fixpoint in shared memory with directional sweeps:
//   x-runs on H layers, y-runs on V layers, z-runs through each via column,
// each run a forward and a backward pass (so a straight wave crosses the tile
// in one pass).  Tiles exchange only boundary improvements, once per grid
// round, so the number of grid rounds drops by about the tile width.
//
// Every update is the fp32 round-to-nearest relaxation min(d[v], d[u] + w), so
// the result is the unique fixpoint of the generic search, bit for bit, in any
// order; the backtrace (orsp_sssp.cu) is shared.  A tile that has not
// converged after MAX_CYCLES sweep cycles is simply revisited next round.
//
// Tiles in the next round's list: neighbours whose halo value improved (and
// the tile itself if it did not converge).  Each tile is in a round's list at
// most once (stamp[t] = last round it was queued for), so a tile is only ever
// processed by one CTA per round and owns its nodes' distances.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "fastdiv.cuh"

namespace {

constexpr int MAX_CYCLES = 64;

// Layer strides (floats) of a tile's shared arrays: distances with their
// halo, (TY + 2) rows of TX + 3, and the interior arrays (weights, loaded
// distances), TY rows of TX + 1, each padded to 8 (mod 16).  A warp's x- or
// y-runs cover two layers of the same kind, which are two layers apart (H
// and V layers alternate), so a layer offset of 2 x stride = 16 (mod 32)
// puts the second layer's rows on the other half of the banks.
__host__ __device__ constexpr int pad_8_mod_16(int v) { return v + ((8 - v % 16) + 16) % 16; }
__host__ __device__ constexpr int tile_ps(int TX, int TY) { return pad_8_mod_16((TY + 2) * (TX + 3)); }
__host__ __device__ constexpr int tile_wps(int TX, int TY) { return pad_8_mod_16(TY * (TX + 1)); }
// Floats of shared memory per layer of a tile (distances, four weight
// arrays, loaded distances).
__host__ __device__ constexpr int tile_floats_per_layer(int TX, int TY) { return tile_ps(TX, TY) + 5 * tile_wps(TX, TY); }

struct LatCtl {
  GridBarrier bar;
  int err;
  unsigned lcnt[3];  // tile-list counts by round % 3
  unsigned work[3];  // per-round work counters by round % 3
  unsigned rounds;
  unsigned visits;
  unsigned long long cycles;
  unsigned head, tail;  // tile queue positions (asynchronous schedule)
  int pending;          // tiles queued or being visited
  unsigned pad;
  unsigned long long ns[4];  // time in load, sweeps, write-back, scheduling (sum over visits)
};

using orsp::LatBox;

struct LatParams {
  int32_t nx, ny, nz;
  int32_t nbox;
  int32_t seed_per_box;                    // seed i starts box i (boxes with their own distances)
  const LatBox *boxes;                     // searched boxes (disjoint unless each has its own distances)
  const float4 *w4;                        // in-edge weights per node
  uint32_t *dist;
  int32_t *list0, *list1;
  unsigned *stamp;
  int32_t *qslot;  // asynchronous schedule: ring of tile ids (-1 = empty)
  int *tstate;     // 0 idle, 1 queued, 2 visiting, 3 visiting and dirty
  unsigned qcap;
  LatCtl *ctl;
  int8_t axis[64];
  unsigned max_rounds;
  unsigned long long wait_ns, budget_ns;
  int selfcont;
  int prefetch;            // warp-specialised schedule: L2 prefetch of the next tile's rows
  const int32_t *roi_map;  // node-set ROI searches: seeds outside it are ignored
  const float *wcol;       // column vias: gathered via weights [N][nzp] (Graph::wcol)
  int32_t nzp;             // nz rounded up to 4
  int64_t N;
};

__global__ void fill_kernel(uint32_t *p, int64_t n, uint32_t v) {
  const int64_t s = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += s) p[i] = v;
}

// The fill of the boxes' own distance slices [dbase, dbase + volume), box
// blockIdx.y, skipping boxes with active[j] == 0.
__global__ void fill_slices_kernel(uint32_t *p, const LatBox *__restrict__ boxes, const int32_t *__restrict__ active,
                                   uint32_t v) {
  if (active && !active[blockIdx.y]) return;
  const LatBox B = boxes[blockIdx.y];
  const int64_t count = (int64_t)(B.x1 - B.x0 + 1) * (B.y1 - B.y0 + 1) * (B.z1 - B.z0 + 1);
  uint32_t *q = p + B.dbase;
  const int64_t s = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += s) q[i] = v;
}

// The same fill over the nodes of a box (x fastest).
__global__ void fill_box_kernel(uint32_t *p, int32_t nx, int32_t ny, int32_t x0, int32_t bw, int32_t y0,
                                int32_t bh, int32_t z0, int64_t count, uint32_t v) {
  const int64_t s = (int64_t)gridDim.x * blockDim.x;
  const int64_t plane = (int64_t)bw * bh;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += s) {
    const int64_t z = i / plane;
    const int64_t r = i - z * plane;
    const int32_t y = (int32_t)(r / bw), x = (int32_t)(r - (int64_t)y * bw);
    p[((int64_t)(z0 + z) * ny + (y0 + y)) * nx + (x0 + x)] = v;
  }
}

// Cell i of a box (x fastest, then y, then z) as coordinates: multiply-high
// divisions while the box has fewer than 2^32 cells (the common case),
// 64-bit divisions otherwise.
struct BoxIndex {
  FastDiv fw, fp;
  uint32_t w;
  bool fast;
  __device__ __forceinline__ void init(int64_t bw, int64_t bh, int64_t count) {
    fast = count < ((int64_t)1 << 32) && bw * bh < ((int64_t)1 << 31);
    w = (uint32_t)bw;
    if (fast) {
      fw.init((uint32_t)bw);
      fp.init((uint32_t)(bw * bh));
    }
  }
  __device__ __forceinline__ void split(int64_t i, int64_t plane, int32_t &z, int32_t &y, int32_t &x) const {
    if (fast) {
      const uint32_t u = (uint32_t)i, zz = fp.div(u), r = u - zz * (uint32_t)plane, yy = fw.div(r);
      z = (int32_t)zz;
      y = (int32_t)yy;
      x = (int32_t)(r - yy * w);
    } else {
      const int64_t zz = i / plane, r = i - zz * plane, yy = r / w;
      z = (int32_t)zz;
      y = (int32_t)yy;
      x = (int32_t)(r - yy * w);
    }
  }
};

// In-edge weights of node v as one float4 {from lower axis neighbour, from
// upper axis neighbour, via from below, via from above}; +inf where absent.
__global__ void gather_kernel(const int32_t *__restrict__ slot_eid, const float *__restrict__ cost,
                              float4 *__restrict__ w, int64_t n) {
  const float INF_F = __int_as_float(0x7f800000);
  const int64_t s = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += s) {
    const int32_t e0 = slot_eid[v], e1 = slot_eid[n + v], e2 = slot_eid[2 * n + v], e3 = slot_eid[3 * n + v];
    w[v] = make_float4(e0 >= 0 ? __ldg(&cost[e0]) : INF_F, e1 >= 0 ? __ldg(&cost[e1]) : INF_F,
                       e2 >= 0 ? __ldg(&cost[e2]) : INF_F, e3 >= 0 ? __ldg(&cost[e3]) : INF_F);
  }
}

// The same gather for the nodes of a box only (x fastest, then y, then z).
__global__ void gather_box_kernel(const int32_t *__restrict__ slot_eid, const float *__restrict__ cost,
                                  float4 *__restrict__ w, int64_t n, int32_t nx, int32_t ny, int32_t x0,
                                  int32_t bw, int32_t y0, int32_t bh, int32_t z0, int64_t count) {
  const float INF_F = __int_as_float(0x7f800000);
  const int64_t s = (int64_t)gridDim.x * blockDim.x;
  const int64_t plane = (int64_t)bw * bh;
  BoxIndex bi;
  bi.init(bw, bh, count);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += s) {
    int32_t z, y, x;
    bi.split(i, plane, z, y, x);
    const int64_t v = ((int64_t)(z0 + z) * ny + (y0 + y)) * nx + (x0 + x);
    const int32_t e0 = slot_eid[v], e1 = slot_eid[n + v], e2 = slot_eid[2 * n + v], e3 = slot_eid[3 * n + v];
    w[v] = make_float4(e0 >= 0 ? __ldg(&cost[e0]) : INF_F, e1 >= 0 ? __ldg(&cost[e1]) : INF_F,
                       e2 >= 0 ? __ldg(&cost[e2]) : INF_F, e3 >= 0 ? __ldg(&cost[e3]) : INF_F);
  }
}

// The same gather for the nodes of several boxes in one launch: blockIdx.y
// is the box (a device LatBox table), blockIdx.x strides over its cells;
// boxes with active[j] == 0 are skipped (active NULL: none).  Cells shared by
// two boxes are written twice with the same value.
__global__ void gather_boxes_kernel(const int32_t *__restrict__ slot_eid, const float *__restrict__ cost,
                                    float4 *__restrict__ w, int64_t n, int32_t nx, int32_t ny,
                                    const LatBox *__restrict__ boxes, const int32_t *__restrict__ active) {
  if (active && !active[blockIdx.y]) return;
  const float INF_F = __int_as_float(0x7f800000);
  const LatBox B = boxes[blockIdx.y];
  const int32_t bw = B.x1 - B.x0 + 1, bh = B.y1 - B.y0 + 1;
  const int64_t plane = (int64_t)bw * bh, count = plane * (B.z1 - B.z0 + 1);
  const int64_t s = (int64_t)gridDim.x * blockDim.x;
  BoxIndex bi;
  bi.init(bw, bh, count);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += s) {
    int32_t z, y, x;
    bi.split(i, plane, z, y, x);
    const int64_t v = ((int64_t)(B.z0 + z) * ny + (B.y0 + y)) * nx + (B.x0 + x);
    const int32_t e0 = slot_eid[v], e1 = slot_eid[n + v], e2 = slot_eid[2 * n + v], e3 = slot_eid[3 * n + v];
    w[v] = make_float4(e0 >= 0 ? __ldg(&cost[e0]) : INF_F, e1 >= 0 ? __ldg(&cost[e1]) : INF_F,
                       e2 >= 0 ? __ldg(&cost[e2]) : INF_F, e3 >= 0 ? __ldg(&cost[e3]) : INF_F);
  }
}

// ---------------------------------------------------------------------------
// Node-set ROI searches (global_to_roi maps, as SimpleDijkstra.find_path_roi
// takes them, UPF:1801-1887): the tile sweeps run over the ROI's bounding box,
// on weights in which every edge that leaves or enters the ROI is +inf.

struct RoiGeom {
  int32_t nx, ny, nz;
  int8_t axis[64];
};

// Bounding box of the ROI, as running maxima bb[6] = {-x0, x1, -y0, y1, -z0,
// z1} (bb starts far below any coordinate): over the node list when given,
// else over every node v with roi_map[v] >= 0.
__global__ void roi_bbox_kernel(const int32_t *__restrict__ nodes, int64_t n, const int32_t *__restrict__ roi_map,
                                int32_t nx, int32_t ny, int64_t N, int *bb) {
  int m[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) m[k] = INT_MIN;
  const int64_t plane = (int64_t)nx * ny;
  const int64_t s = (int64_t)gridDim.x * blockDim.x;
  // node ids are int32 (N < 2^31): multiply-high divisions
  FastDiv fp, fx;
  fp.init((uint32_t)plane);
  fx.init((uint32_t)nx);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += s) {
    const int64_t v = nodes ? (int64_t)__ldg(&nodes[i]) : i;
    if (v < 0 || v >= N) continue;
    if (!nodes && __ldg(&roi_map[v]) < 0) continue;
    const uint32_t u = (uint32_t)v, zu = fp.div(u), r = u - zu * (uint32_t)plane, yu = fx.div(r);
    const int32_t z = (int32_t)zu, y = (int32_t)yu, x = (int32_t)(r - yu * (uint32_t)nx);
    m[0] = max(m[0], -x);
    m[1] = max(m[1], x);
    m[2] = max(m[2], -y);
    m[3] = max(m[3], y);
    m[4] = max(m[4], -z);
    m[5] = max(m[5], z);
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const int w = __reduce_max_sync(ORSP_FULL_MASK, m[k]);
    if ((threadIdx.x & 31) == 0 && w != INT_MIN) atomicMax(&bb[k], w);
  }
}

// The searched box from the running maxima (an empty ROI gives a box with
// no cells and no tiles).
template <int TX, int TY>
__global__ void roi_box_finish_kernel(const int *bb, LatBox *box) {
  LatBox B;
  if (bb[1] < 0) {
    B.x0 = 0; B.x1 = -1; B.y0 = 0; B.y1 = -1; B.z0 = 0; B.z1 = -1;
    B.ntx = 0;
    B.nty = 0;
  } else {
    B.x0 = -bb[0]; B.x1 = bb[1]; B.y0 = -bb[2]; B.y1 = bb[3]; B.z0 = -bb[4]; B.z1 = bb[5];
    B.ntx = (B.x1 - B.x0 + TX) / TX;
    B.nty = (B.y1 - B.y0 + TY) / TY;
  }
  B.tile0 = 0;
  B.pad = 0;
  B.dbase = -1;
  *box = B;
}

// In-edge weights of the box's nodes, as gather_kernel, with +inf on every
// edge u -> v where u or v lies outside the ROI (roi_map < 0; NULL: no
// restriction) or u is a sink (sink[u] != 0; NULL: none).  Grid-stride over
// the box read from device memory.
__global__ void gather_roi_kernel(const int32_t *__restrict__ slot_eid, const float *__restrict__ cost,
                                  float4 *__restrict__ w, int64_t n, RoiGeom G, const LatBox *__restrict__ box,
                                  const int32_t *__restrict__ roi_map, const uint8_t *__restrict__ sink) {
  const float INF_F = __int_as_float(0x7f800000);
  const LatBox B = *box;
  const int64_t bw = B.x1 - B.x0 + 1, bh = B.y1 - B.y0 + 1, bd = B.z1 - B.z0 + 1;
  if (bw <= 0 || bh <= 0 || bd <= 0) return;
  const int64_t plane = bw * bh, count = plane * bd;
  const int64_t nxy = (int64_t)G.nx * G.ny;
  const int64_t s = (int64_t)gridDim.x * blockDim.x;
  BoxIndex bi;
  bi.init(bw, bh, count);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += s) {
    int32_t zz, yy, xx;
    bi.split(i, plane, zz, yy, xx);
    const int32_t gz = B.z0 + (int32_t)zz;
    const int64_t v = (int64_t)gz * nxy + (int64_t)(B.y0 + yy) * G.nx + (B.x0 + xx);
    const bool vin = !roi_map || __ldg(&roi_map[v]) >= 0;
    const int64_t step = G.axis[gz] == 1 ? 1 : G.nx;
    const int64_t from[4] = {v - step, v + step, v - nxy, v + nxy};
    float o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int32_t e = __ldg(&slot_eid[k * n + v]);
      bool ok = e >= 0 && vin;
      if (ok) {
        const int64_t u = from[k];
        ok = (!roi_map || __ldg(&roi_map[u]) >= 0) && !(sink && __ldg(&sink[u]));
      }
      o[k] = ok ? __ldg(&cost[e]) : INF_F;
    }
    w[v] = make_float4(o[0], o[1], o[2], o[3]);
  }
}

// Column-via weights of the nodes of a box (column vias, Graph::cvia):
// wcol[v * nzp + za] (nzp = nz rounded up to 4) = the smaller cost of the (up to two) parallel vias from
// layer za of v's column into v, for every layer za of the box; +inf where
// there is none, where u or v lies outside the ROI (roi_map < 0; NULL: no
// restriction) or u is a sink (sink[u] != 0; NULL: none).  The box is read
// from device memory (bx) or given by value (bx NULL).
__global__ void gather_col_kernel(const int32_t *__restrict__ vcol_eid, const float *__restrict__ cost,
                                  float *__restrict__ wcol, int64_t n, int32_t nx, int32_t ny, int32_t nz, int32_t nzp,
                                  const LatBox *__restrict__ bx, LatBox bv, const int32_t *__restrict__ roi_map,
                                  const uint8_t *__restrict__ sink) {
  const float INF_F = __int_as_float(0x7f800000);
  const LatBox B = bx ? *bx : bv;
  const int64_t bw = B.x1 - B.x0 + 1, bh = B.y1 - B.y0 + 1, bd = B.z1 - B.z0 + 1;
  if (bw <= 0 || bh <= 0 || bd <= 0) return;
  const int64_t plane = bw * bh, cells = plane * bd, count = cells * bd;
  const int64_t nxy = (int64_t)nx * ny;
  const int64_t s = (int64_t)gridDim.x * blockDim.x;
  // cells of the box stacked bd times (one copy per source layer): the
  // "layer" coordinate of this split runs over bd * bd
  BoxIndex bi;
  bi.init(bw, bh, count);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += s) {
    int32_t zq, yy, xx;
    bi.split(i, plane, zq, yy, xx);
    const int64_t za = B.z0 + zq / (int32_t)bd;  // source layer
    const int32_t zz = zq - (int32_t)((za - B.z0) * bd);
    const int64_t col = (int64_t)(B.y0 + yy) * nx + (B.x0 + xx);
    const int64_t v = (int64_t)(B.z0 + zz) * nxy + col;
    const int32_t e0 = __ldg(&vcol_eid[za * n + v]), e1 = __ldg(&vcol_eid[((int64_t)nz + za) * n + v]);
    float w = INF_F;
    if (e0 >= 0) {
      const int64_t u = za * nxy + col;
      bool ok = !roi_map || (__ldg(&roi_map[v]) >= 0 && __ldg(&roi_map[u]) >= 0);
      ok = ok && !(sink && __ldg(&sink[u]));
      if (ok) {
        w = __ldg(&cost[e0]);
        if (e1 >= 0) w = fminf(w, __ldg(&cost[e1]));
      }
    }
    wcol[v * nzp + za] = w;
  }
}

__device__ __forceinline__ LatBox load_box(const LatParams &p, int b) {
  const int32_t *q = (const int32_t *)(p.boxes + b);
  LatBox B;
  B.x0 = __ldg(q + 0);
  B.x1 = __ldg(q + 1);
  B.y0 = __ldg(q + 2);
  B.y1 = __ldg(q + 3);
  B.z0 = __ldg(q + 4);
  B.z1 = __ldg(q + 5);
  B.ntx = __ldg(q + 6);
  B.nty = __ldg(q + 7);
  B.tile0 = __ldg(q + 8);
  B.pad = __ldg(q + 9);
  B.dbase = __ldg((const long long *)(p.boxes + b) + 5);
  return B;
}

// Index of cell (x, y, z) of box B in the distance array: the node id
// (shared distances) or the box's own slice (PRIV, B.dbase >= 0).  The search
// kernels are compiled once per mode, so the shared mode carries no slice
// arithmetic.
template <bool PRIV>
__device__ __forceinline__ int64_t dist_index(const LatParams &p, const LatBox &B, int32_t x, int32_t y, int32_t z) {
  if (!PRIV || B.dbase < 0) return ((int64_t)z * p.ny + y) * p.nx + x;
  const int64_t bw = B.x1 - B.x0 + 1, bh = B.y1 - B.y0 + 1;
  return B.dbase + ((int64_t)(z - B.z0) * bh + (y - B.y0)) * bw + (x - B.x0);
}

// Box of tile t: the last box whose first tile is <= t.
__device__ __forceinline__ int box_of_tile(const LatParams &p, int t) {
  int lo = 0, hi = p.nbox - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&p.boxes[mid].tile0) <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int TX, int TY>
__device__ __forceinline__ int tile_of(const LatBox &B, int32_t gx, int32_t gy) {
  return B.tile0 + ((gy - B.y0) / TY) * B.ntx + (gx - B.x0) / TX;
}

template <int TX, int TY>
__global__ void lattice_seed_kernel(LatParams p, int32_t nseeds, const int32_t *seeds,
                                    const float *seed_cost) {
  LatCtl *c = p.ctl;
  if (threadIdx.x == 0) {
    c->bar.count = 0;
    c->bar.gen = 0;
    c->err = 0;
    for (int i = 0; i < 3; ++i) { c->lcnt[i] = 0; c->work[i] = 0; }
    c->rounds = 0;
    c->visits = 0;
    c->cycles = 0;
    c->head = 0;
    c->tail = 0;
    c->pending = 0;
    for (int i = 0; i < 4; ++i) c->ns[i] = 0;
  }
  __syncthreads();
  const int32_t plane = p.nx * p.ny;
  for (int i = threadIdx.x; i < nseeds; i += blockDim.x) {
    const int32_t s = seeds[i];
    if (s < 0 || s >= plane * p.nz) continue;
    if (p.roi_map && __ldg(&p.roi_map[s]) < 0) continue;
    const int32_t z = s / plane, r = s - z * plane, y = r / p.nx, x = r - y * p.nx;
    int bi = -1;
    LatBox B;
    if (p.seed_per_box) {
      if (i < p.nbox) {
        B = load_box(p, i);
        if (x >= B.x0 && x <= B.x1 && y >= B.y0 && y <= B.y1 && z >= B.z0 && z <= B.z1) bi = i;
      }
    } else {
      for (int b = 0; b < p.nbox && bi < 0; ++b) {
        B = load_box(p, b);
        if (x >= B.x0 && x <= B.x1 && y >= B.y0 && y <= B.y1 && z >= B.z0 && z <= B.z1) bi = b;
      }
    }
    if (bi < 0) continue;
    const float c0 = seed_cost ? seed_cost[i] : 0.0f;
    if (!(c0 >= 0.0f) || !(c0 < __int_as_float(0x7f800000))) continue;
    atomicMin(&p.dist[p.seed_per_box ? dist_index<true>(p, B, x, y, z) : dist_index<false>(p, B, x, y, z)],
              f_bits(c0));
    // The seed's tile and its neighbours in the box: a tile visit publishes
    // only cells it improved, and a seed is set before any visit, so a seed
    // on a tile edge reaches the next tile through that tile's halo only.
    const int t = tile_of<TX, TY>(B, x, y);
    const int lt = t - B.tile0, tx = lt % B.ntx, ty = lt / B.ntx;
    const int nb[5] = {t, tx > 0 ? t - 1 : -1, tx < B.ntx - 1 ? t + 1 : -1, ty > 0 ? t - B.ntx : -1,
                       ty < B.nty - 1 ? t + B.ntx : -1};
    for (int j = 0; j < 5; ++j) {
      const int q = nb[j];
      if (q < 0) continue;
      if (p.qslot) {
        if (atomicCAS(&p.tstate[q], 0, 1) == 0) {
          atomicAdd(&c->pending, 1);
          const unsigned k = atomicAdd(&c->tail, 1u);
          atomicExch(&p.qslot[k % p.qcap], q);
        }
      } else if (atomicMax(&p.stamp[q], 1u) < 1u) {
        const unsigned k = atomicAdd(&c->lcnt[0], 1u);
        p.list0[k] = q;
      }
    }
  }
}

// One run of the sweep: cells c[1..n] at stride `ds`, with c[0] and c[n+1]
// the halo values (when `halo`; otherwise the run starts and ends at c[1] and
// c[n]).  Forward: c[i] = min(c[i], c[i-1] + wlo[i]); backward: c[i] =
// min(c[i], c[i+1] + whi[i]); each step a single fp32 round-to-nearest add
// and a min (fminf returns one of its operands; no NaN or -0 occurs here, so
// the result is that of the compare-and-replace form, without a branch).  The
// run is walked in register chunks of 4 (loads first, then the dependent
// chain), and only decreased cells are stored.  Returns whether any cell
// decreased.  Used for runs whose length is known only at run time (tiles cut
// by the box edge, z-runs).
__device__ __forceinline__ bool sweep_run(float *c, int ds, const float *wlo, const float *whi, int ws,
                                          int n, bool halo = true) {
  constexpr int K = 4;
  bool chg = false;
  float prev = halo ? c[0] : __int_as_float(0x7f800000);
  for (int b = 1; b <= n; b += K) {
    float cv[K], wv[K], nv[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (b + k <= n) { cv[k] = c[(b + k) * ds]; wv[k] = wlo[(b + k) * ws]; }
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (b + k <= n) { nv[k] = fminf(__fadd_rn(prev, wv[k]), cv[k]); prev = nv[k]; }
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (b + k <= n && nv[k] < cv[k]) { c[(b + k) * ds] = nv[k]; chg = true; }
  }
  prev = halo ? c[(n + 1) * ds] : __int_as_float(0x7f800000);
  for (int b = n; b >= 1; b -= K) {
    float cv[K], wv[K], nv[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (b - k >= 1) { cv[k] = c[(b - k) * ds]; wv[k] = whi[(b - k) * ws]; }
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (b - k >= 1) { nv[k] = fminf(__fadd_rn(prev, wv[k]), cv[k]); prev = nv[k]; }
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (b - k >= 1 && nv[k] < cv[k]) { c[(b - k) * ds] = nv[k]; chg = true; }
  }
  return chg;
}

// The same run for a full tile row or column: length N and strides known at
// compile time, so every shared-memory access is an immediate offset from one
// base, the whole run is in registers and the chain is one add and one min
// per step.
template <int N, int DS, int WS>
__device__ __forceinline__ bool sweep_run_fixed(float *c, const float *wlo, const float *whi) {
  float o[N], v[N];
#pragma unroll
  for (int i = 0; i < N; ++i) o[i] = c[(i + 1) * DS];
  float prev = c[0];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    v[i] = fminf(__fadd_rn(prev, wlo[(i + 1) * WS]), o[i]);
    prev = v[i];
  }
  prev = c[(N + 1) * DS];
#pragma unroll
  for (int i = N - 1; i >= 0; --i) {
    v[i] = fminf(__fadd_rn(prev, whi[(i + 1) * WS]), v[i]);
    prev = v[i];
  }
  bool chg = false;
#pragma unroll
  for (int i = 0; i < N; ++i)
    if (v[i] < o[i]) {
      c[(i + 1) * DS] = v[i];
      chg = true;
    }
  return chg;
}

// B consecutive cells of a z-run (stride DS, weights stride WS), forward
// (UP: from below, weights wdn) or backward (from above, weights wup), with
// the chain value carried in `prev`.
template <int B, int DS, int WS, bool UP>
__device__ __forceinline__ bool zrun_block(float *c, const float *w, float &prev) {
  float o[B], v[B];
#pragma unroll
  for (int i = 0; i < B; ++i) o[i] = c[i * DS];
#pragma unroll
  for (int k = 0; k < B; ++k) {
    const int i = UP ? k : B - 1 - k;
    v[i] = fminf(__fadd_rn(prev, w[i * WS]), o[i]);
    prev = v[i];
  }
  bool chg = false;
#pragma unroll
  for (int i = 0; i < B; ++i)
    if (v[i] < o[i]) {
      c[i * DS] = v[i];
      chg = true;
    }
  return chg;
}

// z-run of a column: cells col[z * DS] for z = 0..n-1 (no halo), forward with
// wdn, then backward with wup, in register blocks of 6.
template <int DS, int WS>
__device__ __forceinline__ bool zrun(float *col, const float *wdn, const float *wup, int n) {
  constexpr int B = 6;
  bool chg = false;
  float prev = __int_as_float(0x7f800000);
  int z = 0;
  for (; z + B <= n; z += B) chg |= zrun_block<B, DS, WS, true>(col + z * DS, wdn + z * WS, prev);
  for (; z < n; ++z) chg |= zrun_block<1, DS, WS, true>(col + z * DS, wdn + z * WS, prev);
  prev = __int_as_float(0x7f800000);
  z = n;
  for (; z >= B; z -= B) chg |= zrun_block<B, DS, WS, false>(col + (z - B) * DS, wup + (z - B) * WS, prev);
  for (; z > 0; --z) chg |= zrun_block<1, DS, WS, false>(col + (z - 1) * DS, wup + (z - 1) * WS, prev);
  return chg;
}

// Relaxes one tile (all layers of the box) to a local fixpoint and publishes
// improved values.  Called by all threads of the CTA.  Shared memory:
// distances with a one-cell halo [nzb][TY+2][TX+3], then the interior in-edge
// weights [4][nzb][TY][TX+1] and the interior distances as loaded
// [nzb][TY][TX+1], layers tile_ps / tile_wps floats apart (odd row strides:
// the row walks of the x-sweep and the column walks of the y- and z-sweeps
// are bank-conflict free within a layer; the padded layer strides keep the
// two layers of one warp apart).
// The distances and in-edge weights of one tile column (cells s0 + z * PS /
// w0 + z * WPS in shared memory) in blocks of ZB layers, each block's loads
// all issued before its stores.
template <int ZB, int PS, int WPS>
__device__ __forceinline__ void load_column_blocks_impl(const LatParams &p, int nzb, int64_t d0, int64_t dz,
                                                        int64_t n0, int64_t nxy, float *sd, float *orig, float *wlo,
                                                        float *whi, float *wdn, float *wup, int s0, int w0) {
  for (int zb = 0; zb < nzb; zb += ZB) {
    float dv[ZB];
    float4 wv[ZB];
#pragma unroll
    for (int k = 0; k < ZB; ++k)
      if (zb + k < nzb) {
        dv[k] = bits_f(__ldcg(&p.dist[d0 + (zb + k) * dz]));
        wv[k] = __ldg(&p.w4[n0 + (zb + k) * nxy]);
      }
#pragma unroll
    for (int k = 0; k < ZB; ++k)
      if (zb + k < nzb) {
        const int z = zb + k, wi = z * WPS + w0;
        sd[z * PS + s0] = dv[k];
        orig[wi] = dv[k];
        wlo[wi] = wv[k].x;
        whi[wi] = wv[k].y;
        wdn[wi] = wv[k].z;
        wup[wi] = wv[k].w;
      }
  }
}

// Barrier of the threads that visit tiles: the whole block, or (SPEC) the
// first NW threads only - named barrier 1 - while a scheduler warp runs beside
// them.
template <int NW, bool SPEC>
__device__ __forceinline__ void tile_sync() {
  if (SPEC) asm volatile("bar.sync 1, %0;" ::"r"(NW) : "memory");
  else __syncthreads();
}

// Tensor-memory-accelerator staging of a whole-lattice tile (ORSP_LAT_TMA=1):
// two cp.async.bulk.tensor loads per fresh visit, completing on one mbarrier,
// bring the tile's in-edge weights (box {4, TX, TY, nzb} of the float4 array
// seen as fp32 [nz][ny][nx][4]) and its distances with a halo (box
// {TX + 8, TY + 2, nzb} of the u32 distances [slice][nz][ny][nx], starting at
// x = X0 - 4 so that the start is 16-byte aligned) into a staging area; the
// threads then copy them into the sweep layout (odd row strides), as the
// plain loads do.  Out-of-lattice cells of the box are zero-filled by the
// copy engine and replaced by +inf (halo) or ignored (interior) in the copy.
// The tensor maps cover this GPU's memory only and no load is multicast.
struct TmaCtx {
  const CUtensorMap *tw, *td;  // the kernel's __grid_constant__ tensor maps
  uint32_t mbar;               // shared address of the CTA's mbarrier
  unsigned phase;              // parity of the next completion
  float *sw;                   // staging: weights [nzb][TY][TX] float4
  uint32_t *sdd;               // staging: distances [nzb][TY + 2][TX + 8]
};

__device__ __forceinline__ uint32_t smem_addr(const void *ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}

// Thread 0 issues the two loads of the tile at (X0, Y0) of distance slice
// `slice`; every thread then waits (bounded) for their completion.
template <int TX, int TY>
__device__ __forceinline__ void tma_stage(const LatParams &p, int32_t X0, int32_t Y0, int32_t z0, int nzb,
                                          int slice, TmaCtx &tc) {
  if (threadIdx.x == 0) {
    const uint32_t bytes = (uint32_t)nzb * (uint32_t)(TY * TX * 16 + (TY + 2) * (TX + 8) * 4);
    // distances other CTAs published (acquired through the tile state) are
    // read by the async proxy; the staging's earlier generic reads come
    // before its async-proxy writes
    asm volatile("fence.proxy.async.global;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc.mbar), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(smem_addr(tc.sw)), "l"((uint64_t)tc.tw), "r"(0), "r"(X0), "r"(Y0), "r"(z0), "r"(tc.mbar)
        : "memory");
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(smem_addr(tc.sdd)), "l"((uint64_t)tc.td), "r"(X0 - 4), "r"(Y0 - 1), "r"(z0), "r"(slice), "r"(tc.mbar)
        : "memory");
  }
  // bounded wait: past wait_ns the search is failed with a timeout, and the
  // wait goes on for one more wait_ns so that the copies are not left in
  // flight into shared memory that the next visit reuses
  const unsigned long long t0 = dev_globaltimer();
  bool timed_out = false;
  for (unsigned spins = 0;; ++spins) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred P;\n mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n selp.u32 %0, 1, 0, P;\n}"
        : "=r"(ok)
        : "r"(tc.mbar), "r"(tc.phase)
        : "memory");
    if (ok) break;
    if ((spins & 63u) == 63u) {
      const unsigned long long dt = dev_globaltimer() - t0;
      if (!timed_out && dt > p.wait_ns) {
        atomicCAS(&p.ctl->err, DEV_OK, DEV_ERR_TIMEOUT);
        timed_out = true;
      }
      if (dt > 2 * p.wait_ns) break;
    }
  }
  tc.phase ^= 1u;
}

// Via pass of one column with column vias: for each layer zb of the box in
// turn, d[zb] = min(d[zb], fl(d[za] + w(za -> zb))) over every layer za of the
// box (Gauss-Seidel, so a later layer sees an earlier one's new value), the
// in-weights read as float4 rows wcol[v * nzp ..] (+inf where no via).  col:
// the column's distances in shared memory, layer stride PS; v0: the node of
// the column's layer z0.  Returns whether any distance decreased.  The sweep
// cycles of the visit repeat it until nothing changes.
template <int PS>
__device__ __forceinline__ bool zcol_pass(float *col, const float *__restrict__ wcol, int32_t nzp, int64_t v0,
                                          int64_t nxy, int32_t z0, int32_t nzb) {
  const float INF_F = __int_as_float(0x7f800000);
  bool chg = false;
  const int q0 = z0 >> 2, q1 = (z0 + nzb - 1) >> 2;
  for (int zb = 0; zb < nzb; ++zb) {
    const float4 *wr = reinterpret_cast<const float4 *>(wcol + (v0 + (int64_t)zb * nxy) * nzp);
    float best = col[zb * PS];
    for (int q = q0; q <= q1; ++q) {
      const float4 w = __ldg(&wr[q]);
      const float wk[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int za = 4 * q + j - z0;
        if (za >= 0 && za < nzb && wk[j] < INF_F) best = fminf(best, __fadd_rn(col[za * PS], wk[j]));
      }
    }
    if (best < col[zb * PS]) {
      col[zb * PS] = best;
      chg = true;
    }
  }
  return chg;
}

// Layer lists of the box being visited: H layers (x-runs) and V layers
// (y-runs) as offsets from the box's z0.  Recomputed when a CTA moves to a
// tile of another box.
struct LayerLists {
  int hl[64], vl[64];
  int nh, nv;
  int box;
};

template <int TX, int TY, bool PRIV, bool SPEC, bool DEEP = false, bool TMA = false, bool CV = false>
__device__ __forceinline__ void process_tile(const LatParams &p, int t, float *sd, LayerLists &L, int *s_flags,
                                             int *s_act, int *s_nb = nullptr, bool warm = false,
                                             TmaCtx *tma = nullptr) {
  const int bi = box_of_tile(p, t);
  const LatBox B = load_box(p, bi);
  if (threadIdx.x == 0 && L.box != bi) {
    int nh = 0, nv = 0;
    for (int z = B.z0; z <= B.z1; ++z) {
      if (p.axis[z] == 1) L.hl[nh++] = z - B.z0;
      else if (p.axis[z] == 2) L.vl[nv++] = z - B.z0;
    }
    L.nh = nh;
    L.nv = nv;
    L.box = bi;
  }
  tile_sync<TX * TY, SPEC>();
  const int *s_hl = L.hl, *s_vl = L.vl;
  const int nh = L.nh, nv = L.nv;
  constexpr int SX = TX + 3;
  constexpr int PS = tile_ps(TX, TY);
  constexpr int WSX = TX + 1;
  constexpr int WPS = tile_wps(TX, TY);
  const float INF_F = __int_as_float(0x7f800000);
  const int lt = t - B.tile0;
  const int tx = lt % B.ntx, ty = lt / B.ntx;
  const int32_t X0 = B.x0 + tx * TX, Y0 = B.y0 + ty * TY;
  const int tw = min(TX, B.x1 - X0 + 1), th = min(TY, B.y1 - Y0 + 1);
  const int nzb = B.z1 - B.z0 + 1;
  const int64_t nxy = (int64_t)p.nx * p.ny;
  const int64_t col0 = (int64_t)Y0 * p.nx + X0;  // node of (X0, Y0, z=0)
  float *wlo = sd + nzb * PS;          // slot 0: from the lower axis neighbour
  float *whi = wlo + nzb * WPS;        // slot 1: from the upper axis neighbour
  float *wdn = whi + nzb * WPS;        // slot 2: via from below
  float *wup = wdn + nzb * WPS;        // slot 3: via from above

  float *orig = wup + nzb * WPS;        // interior distances as loaded
  unsigned long long ts0 = 0;
  if (threadIdx.x == 0) ts0 = dev_globaltimer();
  if (threadIdx.x < 5) s_act[threadIdx.x] = 0;
  if (threadIdx.x < 6) s_flags[threadIdx.x] = 0;
  if (s_nb && threadIdx.x < 4) {  // neighbour tiles in the box: left, right, down, up (-1: box edge)
    const int d = threadIdx.x;
    s_nb[d] = d == 0 ? (tx > 0 ? t - 1 : -1)
                     : d == 1 ? (tx < B.ntx - 1 ? t + 1 : -1)
                              : d == 2 ? (ty > 0 ? t - B.ntx : -1) : (ty < B.nty - 1 ? t + B.ntx : -1);
  }
  // ---- load.  Interior cells: distance and the four in-edge weights; halo
  // cells: only those the sweeps read (x-halo of H-layer rows, y-halo of
  // V-layer columns).  Distances are read through L2 (other CTAs write them);
  // weights are read-only.  A thread's first halo cells are loaded before its
  // column (one thread per column (x, y), up to 18 layers in flight at a
  // time), so their round trip overlaps the column's.
  bool staged = false;
  if constexpr (TMA) {
    if (!warm) {
      tma_stage<TX, TY>(p, X0, Y0, B.z0, nzb, PRIV ? B.pad : 0, *tma);
      constexpr int DX = TX + 8, DY = TY + 2;
      const uint32_t *sdd = tma->sdd;
      const float4 *sw4 = (const float4 *)tma->sw;
      const int c = threadIdx.x;
      if (c < th * tw) {
        const int yy = c / tw + 1, xx = c - (yy - 1) * tw + 1;
        const int s0 = yy * SX + xx, w0 = (yy - 1) * WSX + (xx - 1);
        for (int z = 0; z < nzb; ++z) {
          const float dv = __uint_as_float(sdd[(z * DY + yy) * DX + xx + 3]);
          const float4 wv = sw4[(z * TY + yy - 1) * TX + xx - 1];
          const int wi = z * WPS + w0;
          sd[z * PS + s0] = dv;
          orig[wi] = dv;
          wlo[wi] = wv.x;
          whi[wi] = wv.y;
          wdn[wi] = wv.z;
          wup[wi] = wv.w;
        }
      }
      const int nhh = 2 * nh * th, nvh = 2 * nv * tw;
      for (int i = threadIdx.x; i < nhh + nvh; i += (TX * TY)) {
        int z, xx, yy;
        if (i < nhh) {
          const int rowi = i >> 1;
          z = s_hl[rowi / th];
          yy = rowi % th + 1;
          xx = (i & 1) ? tw + 1 : 0;
        } else {
          const int coli = (i - nhh) >> 1;
          z = s_vl[coli / tw];
          xx = coli % tw + 1;
          yy = ((i - nhh) & 1) ? th + 1 : 0;
        }
        const int32_t gx = X0 + xx - 1, gy = Y0 + yy - 1;
        float v = INF_F;
        if (gx >= B.x0 && gx <= B.x1 && gy >= B.y0 && gy <= B.y1) v = __uint_as_float(sdd[(z * DY + yy) * DX + xx + 3]);
        sd[z * PS + yy * SX + xx] = v;
      }
      staged = true;
    }
  }
  if (!staged) {
    const int nhh = 2 * nh * th, nvh = 2 * nv * tw;
    constexpr int HB = 4;  // halo cells per thread in the first batch
    float hv[HB];
    int hs[HB];
#pragma unroll
    for (int k = 0; k < HB; ++k) {
      const int i = threadIdx.x + k * (TX * TY);
      hs[k] = -1;
      hv[k] = INF_F;
      if (i < nhh + nvh) {
        int z, xx, yy;
        if (i < nhh) {
          const int rowi = i >> 1;
          z = s_hl[rowi / th];
          yy = rowi % th + 1;
          xx = (i & 1) ? tw + 1 : 0;
        } else {
          const int coli = (i - nhh) >> 1;
          z = s_vl[coli / tw];
          xx = coli % tw + 1;
          yy = ((i - nhh) & 1) ? th + 1 : 0;
        }
        const int32_t gx = X0 + xx - 1, gy = Y0 + yy - 1;
        hs[k] = z * PS + yy * SX + xx;
        if (gx >= B.x0 && gx <= B.x1 && gy >= B.y0 && gy <= B.y1)
          hv[k] = bits_f(__ldcg(&p.dist[dist_index<PRIV>(p, B, gx, gy, B.z0 + z)]));
      }
    }
    // the thread's column (x, y) of the tile (th * tw <= threads)
    const int c = threadIdx.x;
    if (warm && c < th * tw) {
      // the same tile again: its interior and weights are still in shared
      // memory and equal to what the last visit published
      const int yy = c / tw + 1, xx = c - (yy - 1) * tw + 1;
      const int s0 = yy * SX + xx, w0 = (yy - 1) * WSX + (xx - 1);
      for (int z = 0; z < nzb; ++z) orig[z * WPS + w0] = sd[z * PS + s0];
    } else if (c < th * tw) {
      const int yy = c / tw + 1, xx = c - (yy - 1) * tw + 1;
      const int64_t n0 = (int64_t)B.z0 * nxy + col0 + (int64_t)(yy - 1) * p.nx + (xx - 1);
      const int64_t d0 = dist_index<PRIV>(p, B, X0 + xx - 1, Y0 + yy - 1, B.z0);
      const int64_t dz = (!PRIV || B.dbase < 0) ? nxy : (int64_t)(B.x1 - B.x0 + 1) * (B.y1 - B.y0 + 1);
      const int s0 = yy * SX + xx, w0 = (yy - 1) * WSX + (xx - 1);
      if constexpr (DEEP) {
        // boxes of more than 12 layers: blocks of 18 layers, each fully
        // unrolled and predicated, every load of a block issued before its
        // stores (one round trip for up to 18 layers)
        load_column_blocks_impl<18, PS, WPS>(p, nzb, d0, dz, n0, nxy, sd, orig, wlo, whi, wdn, wup, s0, w0);
      } else {  // twelve layers in flight
#pragma unroll 12
        for (int z = 0; z < nzb; ++z) {
          const float dv = bits_f(__ldcg(&p.dist[d0 + z * dz]));
          const float4 wv = __ldg(&p.w4[n0 + z * nxy]);
          const int wi = z * WPS + w0;
          sd[z * PS + s0] = dv;
          orig[wi] = dv;
          wlo[wi] = wv.x;
          whi[wi] = wv.y;
          wdn[wi] = wv.z;
          wup[wi] = wv.w;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < HB; ++k)
      if (hs[k] >= 0) sd[hs[k]] = hv[k];
    for (int i = threadIdx.x + HB * (TX * TY); i < nhh + nvh; i += (TX * TY)) {
      int z, xx, yy;
      if (i < nhh) {
        const int rowi = i >> 1;
        z = s_hl[rowi / th];
        yy = rowi % th + 1;
        xx = (i & 1) ? tw + 1 : 0;
      } else {
        const int coli = (i - nhh) >> 1;
        z = s_vl[coli / tw];
        xx = coli % tw + 1;
        yy = ((i - nhh) & 1) ? th + 1 : 0;
      }
      const int32_t gx = X0 + xx - 1, gy = Y0 + yy - 1;
      float v = INF_F;
      if (gx >= B.x0 && gx <= B.x1 && gy >= B.y0 && gy <= B.y1)
        v = bits_f(__ldcg(&p.dist[dist_index<PRIV>(p, B, gx, gy, B.z0 + z)]));
      sd[z * PS + yy * SX + xx] = v;
    }
  }
  tile_sync<TX * TY, SPEC>();
  unsigned long long ts1 = 0;
  if (threadIdx.x == 0) ts1 = dev_globaltimer();

  // ---- sweep cycles.  Each cycle: the planar runs (x-runs on H layers and
  // y-runs on V layers touch disjoint layers, so they run side by side), then
  // the via runs along z.  s_flags[c % 3] records a planar change in cycle c,
  // s_flags[3 + c % 3] a via change.  A pass that changes nothing leaves every
  // constraint it checks satisfied, so once a planar pass changes nothing
  // after a via pass that changed nothing, the tile is at its fixpoint and the
  // cycle's via pass is skipped.
  bool converged = false;
  int cyc = 0;
  const int nplan = nh * th + nv * tw;
  const bool full = tw == TX && th == TY;
  for (; cyc < MAX_CYCLES; ++cyc) {
    if (threadIdx.x == 0) {
      s_flags[(cyc + 1) % 3] = 0;
      s_flags[3 + (cyc + 1) % 3] = 0;
    }
    bool chg = false;
    if (full) {
      for (int rr = threadIdx.x; rr < nplan; rr += (TX * TY)) {
        if (rr < nh * TY) {  // x-run of an H-layer row
          const int z = s_hl[rr / TY], yy = rr % TY + 1;
          const int wo = z * WPS + (yy - 1) * WSX - 1;
          chg |= sweep_run_fixed<TX, 1, 1>(sd + z * PS + yy * SX, wlo + wo, whi + wo);
        } else {  // y-run of a V-layer column
          const int q = rr - nh * TY;
          const int z = s_vl[q / TX], xx = q % TX + 1;
          const int wo = z * WPS + (xx - 1) - WSX;
          chg |= sweep_run_fixed<TY, SX, WSX>(sd + z * PS + xx, wlo + wo, whi + wo);
        }
      }
    } else {
      for (int rr = threadIdx.x; rr < nplan; rr += (TX * TY)) {
        float *cell;
        int wo, ds, ws, n;
        if (rr < nh * th) {  // x-run of an H-layer row
          const int z = s_hl[rr / th], yy = rr % th + 1;
          cell = sd + z * PS + yy * SX;
          wo = z * WPS + (yy - 1) * WSX - 1;
          ds = 1;
          ws = 1;
          n = tw;
        } else {  // y-run of a V-layer column
          const int q = rr - nh * th;
          const int z = s_vl[q / tw], xx = q % tw + 1;
          cell = sd + z * PS + xx;
          wo = z * WPS + (xx - 1) - WSX;
          ds = SX;
          ws = WSX;
          n = th;
        }
        chg |= sweep_run(cell, ds, wlo + wo, whi + wo, ws, n);
      }
    }
    if (chg) s_flags[cyc % 3] = 1;
    tile_sync<TX * TY, SPEC>();
    if (cyc > 0 && !s_flags[cyc % 3] && !s_flags[3 + (cyc - 1) % 3]) { converged = true; break; }
    chg = false;
    for (int c = threadIdx.x; c < tw * th; c += (TX * TY)) {
      const int xx = c % tw + 1, yy = c / tw + 1;
      if constexpr (CV) {
        const int64_t v0 = (int64_t)B.z0 * nxy + col0 + (int64_t)(yy - 1) * p.nx + (xx - 1);
        chg |= zcol_pass<PS>(sd + yy * SX + xx, p.wcol, p.nzp, v0, nxy, B.z0, nzb);
      } else {
        const int wo = (yy - 1) * WSX + (xx - 1);
        chg |= zrun<PS, WPS>(sd + yy * SX + xx, wdn + wo, wup + wo, nzb);
      }
    }
    if (chg) s_flags[3 + cyc % 3] = 1;
    tile_sync<TX * TY, SPEC>();
    if (!s_flags[cyc % 3] && !s_flags[3 + cyc % 3]) { converged = true; break; }
  }
  unsigned long long ts2 = 0;
  if (threadIdx.x == 0) {
    ts2 = dev_globaltimer();
    atomicAdd((unsigned long long *)&p.ctl->cycles, (unsigned long long)(cyc + 1));
  }

  // ---- publish improvements; mark neighbour tiles whose halo changed
  // one thread per column (x, y) of the tile, all its layers: the layer's
  // axis decides which tile edge a changed cell activates
  const int64_t dzs = (!PRIV || B.dbase < 0) ? nxy : (int64_t)(B.x1 - B.x0 + 1) * (B.y1 - B.y0 + 1);
  for (int c = threadIdx.x; c < th * tw; c += (TX * TY)) {
    const int yy = c / tw + 1, xx = c - (yy - 1) * tw + 1;
    const int64_t d0 = dist_index<PRIV>(p, B, X0 + xx - 1, Y0 + yy - 1, B.z0);
    const int s0 = yy * SX + xx, w0 = (yy - 1) * WSX + (xx - 1);
    bool ex = false, ey = false;
    for (int z = 0; z < nzb; ++z) {
      const float v = sd[z * PS + s0];
      if (v < orig[z * WPS + w0]) {
        __stcg(&p.dist[d0 + z * dzs], f_bits(v));
        const int ax = p.axis[B.z0 + z];
        ex |= ax == 1;
        ey |= ax == 2;
      }
    }
    if (ex) {
      if (xx == 1) s_act[0] = 1;
      if (xx == tw) s_act[1] = 1;
    }
    if (ey) {
      if (yy == 1) s_act[2] = 1;
      if (yy == th) s_act[3] = 1;
    }
  }
  if (threadIdx.x == 0 && !converged) s_act[4] = 1;
  tile_sync<TX * TY, SPEC>();
  if (threadIdx.x == 0) {
    const unsigned long long ts3 = dev_globaltimer();
    atomicAdd(&p.ctl->ns[0], ts1 - ts0);
    atomicAdd(&p.ctl->ns[1], ts2 - ts1);
    atomicAdd(&p.ctl->ns[2], ts3 - ts2);
  }
}

// Tiles to revisit after a visit of tile t: the neighbours whose halo value
// improved (s_act[0..3] = left, right, down, up) and t itself if it did not
// converge (s_act[4]).  Returns the count written to nb[0..4].
__device__ __forceinline__ int revisit_list(const LatParams &p, int t, const int *s_act, int *nb) {
  const LatBox B = load_box(p, box_of_tile(p, t));
  const int lt = t - B.tile0;
  const int tx = lt % B.ntx, ty = lt / B.ntx;
  int k = 0;
  if (s_act[0] && tx > 0) nb[k++] = t - 1;
  if (s_act[1] && tx < B.ntx - 1) nb[k++] = t + 1;
  if (s_act[2] && ty > 0) nb[k++] = t - B.ntx;
  if (s_act[3] && ty < B.nty - 1) nb[k++] = t + B.ntx;
  if (s_act[4]) nb[k++] = t;
  return k;
}

template <int TX, int TY, bool PRIV>
__global__ void __launch_bounds__(TX * TY, 1) lattice_tile_kernel(LatParams p) {
  extern __shared__ float sd[];
  __shared__ LayerLists s_layers;
  __shared__ int s_flags[6];
  __shared__ int s_act[5];
  __shared__ int s_tile;
  LatCtl *ctl = p.ctl;
  const unsigned nblocks = gridDim.x;
  const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
  const unsigned long long t_start = dev_globaltimer();
  if (threadIdx.x == 0) s_layers.box = -1;
  __syncthreads();
  unsigned r = 0;
  for (;;) {
    if (ld_acquire_u32((const unsigned *)&ctl->err)) break;
    if (r >= p.max_rounds) {
      if (leader) atomicCAS(&ctl->err, DEV_OK, DEV_ERR_TIMEOUT);
      break;
    }
    const unsigned n_in = ld_acquire_u32(&ctl->lcnt[r % 3]);
    if (n_in == 0) break;  // converged
    const int32_t *inl = (r & 1) ? p.list1 : p.list0;
    int32_t *outl = (r & 1) ? p.list0 : p.list1;
    for (;;) {
      if (threadIdx.x == 0) s_tile = (int)atomicAdd(&ctl->work[r % 3], 1u);
      __syncthreads();
      const int ti = s_tile;
      __syncthreads();
      if (ti >= (int)n_in) break;
      const int t = __ldcg(&inl[ti]);
      process_tile<TX, TY, PRIV, false>(p, t, sd, s_layers, s_flags, s_act);
      if (threadIdx.x == 0) {
        int nb[5];
        const int k = revisit_list(p, t, s_act, nb);
        for (int j = 0; j < k; ++j) {
          if (atomicMax(&p.stamp[nb[j]], r + 2u) < r + 2u) {
            const unsigned idx = atomicAdd(&ctl->lcnt[(r + 1) % 3], 1u);
            __stcg(&outl[idx], nb[j]);  // idx < ntiles: each tile is queued once per round
          }
        }
        atomicAdd(&ctl->visits, 1u);
      }
    }
    if (leader) {
      ctl->lcnt[(r + 2) % 3] = 0;
      ctl->work[(r + 2) % 3] = 0;
      if (dev_globaltimer() - t_start > p.budget_ns) atomicCAS(&ctl->err, DEV_OK, DEV_ERR_TIMEOUT);
    }
    grid_barrier(&ctl->bar, nblocks, &ctl->err, p.wait_ns);
    ++r;
  }
  if (leader) ctl->rounds = r;
}


// ---------------------------------------------------------------------------
// Asynchronous schedule: no grid barrier.  Tiles wait in a ring queue; each
// CTA repeatedly takes the next tile, visits it and queues the tiles whose
// halo it improved.  A tile is in the queue at most once (state 1) and is
// visited by one CTA at a time (state 2); if its halo improves during a visit
// (state 3) the same CTA visits it again at once (or, with that switched
// off, queues it again).  Only the visiting CTA writes a tile's cells, so
// the copy in its shared memory stays exact between the two visits.  `pending` counts tiles in
// states 1-3; it is raised before a tile is queued and lowered only after the
// visiting CTA has queued everything it activated, so it reaches 0 only when
// no tile can change again - the fixpoint.
__device__ void queue_tile(const LatParams &p, int t) {
  const unsigned k = atomicAdd(&p.ctl->tail, 1u);
  atomicExch(&p.qslot[k % p.qcap], t);
}

// Returns false if the state machine could not be advanced (never expected;
// recorded as an internal error by the caller).
__device__ bool activate_tile(const LatParams &p, int t) {
  for (int tries = 0; tries < 1024; ++tries) {
    const int st = atomicCAS(&p.tstate[t], 0, 1);
    if (st == 0) {
      atomicAdd(&p.ctl->pending, 1);
      queue_tile(p, t);
      return true;
    }
    if (st == 1 || st == 3) return true;
    if (atomicCAS(&p.tstate[t], 2, 3) == 2) return true;  // visiting: mark dirty
  }
  return false;
}

// DEEP: the instantiation for tiles of more than 12 layers (the column load
// in 18-layer blocks); compiled separately so that each layer range gets its
// own register allocation.  MINB: CTAs per SM the registers are sized for
// (2 fits a 16 x 16 tile of up to 12 layers in 128 registers per thread).
//
// TMA: fresh visits stage the tile with tensor loads (TmaCtx); every box is
// the whole lattice (the tensor maps and the staging are sized for p.nz
// layers), distances in slices of N cells (LatBox.pad = slice).  tmw / tmd
// are unused otherwise.
template <int TX, int TY, bool PRIV, bool DEEP = false, int MINB = 1, bool TMA = false, bool CV = false>
__global__ void __launch_bounds__(TX * TY, MINB)
    lattice_async_kernel(LatParams p, const __grid_constant__ CUtensorMap tmw, const __grid_constant__ CUtensorMap tmd) {
  extern __shared__ __align__(128) float sd[];
  __shared__ LayerLists s_layers;
  __shared__ int s_flags[6];
  __shared__ int s_act[5];
  __shared__ int s_nb[4];
  __shared__ int s_tile;
  __shared__ __align__(8) unsigned long long s_mbar;
  LatCtl *ctl = p.ctl;
  const unsigned long long t_start = dev_globaltimer();
  TmaCtx tma{};
  if constexpr (TMA) {
    const int64_t off = ((int64_t)p.nz * tile_floats_per_layer(TX, TY) + 31) & ~(int64_t)31;
    tma.tw = &tmw;
    tma.td = &tmd;
    tma.mbar = smem_addr(&s_mbar);
    tma.phase = 0;
    tma.sw = sd + off;
    tma.sdd = (uint32_t *)(sd + off + (int64_t)p.nz * TY * TX * 4);
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tma.mbar) : "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmw) : "memory");
      asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmd) : "memory");
    }
  }
  if (threadIdx.x == 0) s_layers.box = -1;
  __syncthreads();
  unsigned visits = 0;
  unsigned long long sched_ns = 0;
  __shared__ int s_cont;
  if (threadIdx.x == 0) s_cont = -1;
  for (;;) {
    if (threadIdx.x == 0 && s_cont < 0) {
      const unsigned long long tq = dev_globaltimer();
      int t = -1;
      if (!ld_acquire_u32((const unsigned *)&ctl->err)) {
        const unsigned pos = atomicAdd(&ctl->head, 1u);
        int *slot = &p.qslot[pos % p.qcap];
        const unsigned long long t0 = dev_globaltimer();
        for (unsigned spins = 0;; ++spins) {
          const int v = (int)ld_acquire_u32((const unsigned *)slot);
          if (v >= 0) {
            atomicExch(slot, -1);
            t = v;
            break;
          }
          if (ld_acquire_u32((const unsigned *)&ctl->pending) == 0) break;  // fixpoint reached
          if (ld_acquire_u32((const unsigned *)&ctl->err)) break;
          if ((spins & 31u) == 31u) {
            const unsigned long long now = dev_globaltimer();
            if (now - t0 > p.wait_ns || now - t_start > p.budget_ns) {
              atomicCAS(&ctl->err, DEV_OK, DEV_ERR_TIMEOUT);
              break;
            }
            __nanosleep(64);
          }
        }
      }
      if (t >= 0) {
        atomicExch(&p.tstate[t], 2);
        __threadfence();
      }
      s_tile = t;
      sched_ns += dev_globaltimer() - tq;
    }
    __syncthreads();
    const bool warm = s_cont >= 0;
    const int t = warm ? s_cont : s_tile;
    __syncthreads();
    if (t < 0) break;
    process_tile<TX, TY, PRIV, false, DEEP, TMA, CV>(p, t, sd, s_layers, s_flags, s_act, s_nb, warm, &tma);
    // neighbours are activated by threads 0..3 in parallel, after this
    // tile's distances are visible
    unsigned long long ta = 0;
    if (threadIdx.x == 0) ta = dev_globaltimer();
    if (threadIdx.x < 4) {
      __threadfence();
      const int nb = s_act[threadIdx.x] ? s_nb[threadIdx.x] : -1;
      if (nb >= 0 && !activate_tile(p, nb)) atomicCAS(&ctl->err, DEV_OK, DEV_ERR_INTERNAL);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      // leave the visiting state: back to idle, or queued again when dirty
      // (halo changed meanwhile) or not converged
      s_cont = -1;
      if (s_act[4] || atomicCAS(&p.tstate[t], 2, 0) != 2) {
        if (p.selfcont) {
          // visit it again at once: the interior and weights are already in
          // shared memory, so only the halo is read again, and there is no
          // queue handoff.  Visiting again (state 2) is published before the
          // halo is read.
          atomicExch(&p.tstate[t], 2);
          __threadfence();
          s_cont = t;
        } else {
          atomicExch(&p.tstate[t], 1);
          queue_tile(p, t);
        }
      } else {
        atomicSub(&ctl->pending, 1);
      }
      ++visits;
      sched_ns += dev_globaltimer() - ta;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    atomicAdd(&ctl->visits, visits);
    atomicAdd(&ctl->ns[3], sched_ns);
  }
}

// Scheduler side of a finished visit of tile t with neighbour flags act:
// activate the neighbours whose halo improved, then leave the visiting state
// (idle, or queued again when dirty or not converged).  `pending` drops only
// after everything the visit activated is queued.
__device__ void finish_visit(const LatParams &p, int t, const int *act) {
  __threadfence();
  const LatBox B = load_box(p, box_of_tile(p, t));
  const int lt = t - B.tile0, tx = lt % B.ntx, ty = lt / B.ntx;
  const int nbs[4] = {(act[0] && tx > 0) ? t - 1 : -1, (act[1] && tx < B.ntx - 1) ? t + 1 : -1,
                      (act[2] && ty > 0) ? t - B.ntx : -1, (act[3] && ty < B.nty - 1) ? t + B.ntx : -1};
#pragma unroll
  for (int d = 0; d < 4; ++d)
    if (nbs[d] >= 0 && !activate_tile(p, nbs[d])) atomicCAS(&p.ctl->err, DEV_OK, DEV_ERR_INTERNAL);
  if (act[4] || atomicCAS(&p.tstate[t], 2, 0) != 2) {
    atomicExch(&p.tstate[t], 1);
    queue_tile(p, t);
  } else {
    atomicSub(&p.ctl->pending, 1);
  }
}

// Warp-specialised asynchronous schedule.  The block has NW = TX*TY worker
// threads that visit tiles and one scheduler warp whose lane 0 does all queue
// work, so that the chain of global atomics of a visit (pop, activation of the
// neighbours, the tile's own state transition) overlaps the workers' loads and
// sweeps instead of stalling them.
//
// Handoff protocol.  Handoff k hands tile cur_k (or -1: stop) to the workers
// through s_cur, at named barrier 2, which all NW + 32 threads pass exactly
// once per handoff (the scheduler warp passes it once per loop iteration, the
// workers once before each visit; both stop after the handoff that carries
// -1).  The workers visit cur_k with their own named barrier 1, write the
// visit's neighbour flags into s_act[k & 1] and, after a device fence, set
// s_done = k.  The scheduler finishes visit k (activations, state
// transition) once s_done == k - in its wait loop for the next tile, or just
// after the next handoff - so it never waits for work that only its own
// finished tile would create.  The flags of visit k stay intact until visit
// k + 2 starts, and the scheduler reads them before handoff k + 2.
// Prefetch into L2, by one warp, of the rows a visit of tile t loads: per
// layer of the box, each tile row's in-edge weights (16 B per node) and
// distances, with the x-halo cells and the distance rows just above and
// below the tile where the box has them (the y-halo).  Every address
// prefetched lies inside the weight array or the box's distances.
template <int TX, int TY, bool PRIV>
__device__ __forceinline__ void prefetch_tile_l2(const LatParams &p, int t, int lane) {
  const LatBox B = load_box(p, box_of_tile(p, t));
  const int lt = t - B.tile0;
  const int tx = lt % B.ntx, ty = lt / B.ntx;
  const int32_t X0 = B.x0 + tx * TX, Y0 = B.y0 + ty * TY;
  const int tw = min(TX, B.x1 - X0 + 1), th = min(TY, B.y1 - Y0 + 1);
  const int nzb = B.z1 - B.z0 + 1;
  const int64_t nxy = (int64_t)p.nx * p.ny;
  const int ya = Y0 > B.y0 ? -1 : 0, yb = Y0 + th - 1 < B.y1 ? th : th - 1;
  const int nrow = yb - ya + 1;
  for (int i = lane; i < nzb * nrow; i += 32) {
    const int zl = i / nrow, yy = ya + i % nrow;
    const int32_t z = B.z0 + zl, y = Y0 + yy;
    const uint32_t *d = &p.dist[dist_index<PRIV>(p, B, X0, y, z)];
    // the row, with its x-halo cells where the box has them
    asm volatile("prefetch.global.L2 [%0];" ::"l"(X0 > B.x0 ? d - 1 : d) : "memory");
    asm volatile("prefetch.global.L2 [%0];" ::"l"(X0 + tw - 1 < B.x1 ? d + tw : d + tw - 1) : "memory");
    if (yy >= 0 && yy < th) {
      const float4 *w = &p.w4[(int64_t)z * nxy + (int64_t)y * p.nx + X0];
      for (int c = 0; c < tw; c += 8) asm volatile("prefetch.global.L2 [%0];" ::"l"(w + c) : "memory");
      asm volatile("prefetch.global.L2 [%0];" ::"l"(w + tw - 1) : "memory");
    }
  }
}

template <int TX, int TY, bool PRIV, int MINB = 1>
__global__ void __launch_bounds__(TX * TY + 32, MINB) lattice_spec_kernel(LatParams p) {
  constexpr int NW = TX * TY;
  extern __shared__ float sd[];
  __shared__ LayerLists s_layers;
  __shared__ int s_flags[6];
  __shared__ int s_act[2][5];
  __shared__ volatile int s_cur;
  __shared__ volatile int s_done;
  LatCtl *ctl = p.ctl;
  if (threadIdx.x == 0) s_layers.box = -1;
  if (threadIdx.x == NW) s_done = 0;
  __syncthreads();
  if (threadIdx.x < NW) {
    // ---------------------------------------------------------- workers
    unsigned long long idle_ns = 0;
    for (int k = 1;; ++k) {
      unsigned long long tw = 0;
      if (threadIdx.x == 0) tw = dev_globaltimer();
      asm volatile("bar.sync 2, %0;" ::"r"(NW + 32) : "memory");
      if (threadIdx.x == 0) idle_ns += dev_globaltimer() - tw;
      const int t = s_cur;
      if (t < 0) break;
      process_tile<TX, TY, PRIV, true>(p, t, sd, s_layers, s_flags, s_act[k & 1]);
      // process_tile ended with barrier 1: every write of the visit is done
      if (threadIdx.x == 0) {
        __threadfence();
        s_done = k;
      }
    }
    if (threadIdx.x == 0) atomicAdd(&ctl->ns[3], idle_ns);
    return;
  }
  // ------------------------------------------------------------ scheduler
  const int lane = threadIdx.x & 31;
  const unsigned long long t_start = dev_globaltimer();
  int cur = -1;          // tile of the last handoff
  int k = 0;             // index of the last handoff
  bool finished = true;  // visit k finished by the scheduler (or none yet)
  unsigned visits = 0;
  for (;;) {
    int next = -1;
    if (lane == 0) {
      long long pos = -1;
      const unsigned long long t0 = dev_globaltimer();
      for (unsigned spins = 0;; ++spins) {
        if (!finished && s_done == k) {
          finish_visit(p, cur, s_act[k & 1]);
          ++visits;
          finished = true;
        }
        if (ld_acquire_u32((const unsigned *)&ctl->err)) break;
        if (pos < 0) pos = (long long)atomicAdd(&ctl->head, 1u);
        int *slot = &p.qslot[(unsigned)pos % p.qcap];
        const int v = (int)ld_acquire_u32((const unsigned *)slot);
        if (v >= 0) {
          atomicExch(slot, -1);
          atomicExch(&p.tstate[v], 2);
          __threadfence();
          next = v;
          break;
        }
        if (finished && ld_acquire_u32((const unsigned *)&ctl->pending) == 0) break;  // fixpoint reached
        if ((spins & 31u) == 31u) {
          const unsigned long long now = dev_globaltimer();
          if (now - t0 > p.wait_ns || now - t_start > p.budget_ns) {
            atomicCAS(&ctl->err, DEV_OK, DEV_ERR_TIMEOUT);
            break;
          }
          __nanosleep(64);
        }
      }
      s_cur = next;
      __threadfence_block();
    }
    next = __shfl_sync(0xffffffffu, next, 0);
    // the workers are still on visit k: bring the next tile's rows into L2
    if (next >= 0 && p.prefetch) prefetch_tile_l2<TX, TY, PRIV>(p, next, lane);
    __syncwarp();
    asm volatile("bar.sync 2, %0;" ::"r"(NW + 32) : "memory");  // handoff k + 1
    // the workers reached this barrier only after finishing visit k
    if (lane == 0 && !finished) {
      finish_visit(p, cur, s_act[k & 1]);
      ++visits;
      finished = true;
    }
    if (next < 0) break;
    cur = next;
    ++k;
    finished = false;
  }
  if (lane == 0) atomicAdd(&ctl->visits, visits);
}

unsigned long long env_u64(const char *name, unsigned long long dflt) {
  const char *s = getenv(name);
  if (!s || !*s) return dflt;
  return strtoull(s, nullptr, 10);
}

// Workspace layout for ntiles tiles: 4 tile arrays (lists, stamps, states),
// the ring queue, then the control block.
struct WsLayout {
  size_t list_b, q_b, total;
  unsigned qcap;
};
WsLayout ws_layout(const orsp::Graph *g, int64_t ntiles) {
  WsLayout w;
  w.list_b = (((size_t)ntiles * 4) + 255) & ~(size_t)255;
  w.qcap = (unsigned)(ntiles + 4 * g->num_sms * 4 + 64);
  w.q_b = (((size_t)w.qcap * 4) + 255) & ~(size_t)255;
  w.total = 4 * w.list_b + w.q_b + 256;
  return w;
}

int grow_ws(orsp::Graph *g, size_t need) {
  if (g->lat_ws_bytes < need) {
    cudaFree(g->lat_ws);
    g->lat_ws = nullptr;
    g->lat_ws_bytes = 0;
    ORSP_CUDA(cudaMalloc(&g->lat_ws, need));
    g->lat_ws_bytes = need;
  }
  if (!g->lat_ctl_h) ORSP_CUDA(cudaMallocHost(&g->lat_ctl_h, sizeof(LatCtl)));
  return ORSP_OK;
}

// Column-via weights for the nodes of a box: box_h (host, 6 ints) or box_d
// (device), with the ROI / sink masks of a node-set ROI search.
int gather_col_box(orsp::Graph *g, const float *cost_d, const int32_t *box_h, const LatBox *box_d,
                   const int32_t *roi_map_d, const uint8_t *sink_d, cudaStream_t st) {
  LatBox bv{};
  int64_t count = (int64_t)g->N * g->nz;  // upper bound when the box is on the device
  if (box_h) {
    bv.x0 = box_h[0];
    bv.x1 = box_h[1];
    bv.y0 = box_h[2];
    bv.y1 = box_h[3];
    bv.z0 = box_h[4];
    bv.z1 = box_h[5];
    const int64_t d = box_h[5] - box_h[4] + 1;
    count = (int64_t)(box_h[1] - box_h[0] + 1) * (box_h[3] - box_h[2] + 1) * d * d;
  }
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((count + 255) / 256, (int64_t)g->num_sms * 16));
  gather_col_kernel<<<blocks, 256, 0, st>>>(g->vcol_eid, cost_d, g->wcol, g->N, g->nx, g->ny, g->nz,
                                             (g->nz + 3) & ~3, box_d, bv, roi_map_d, sink_d);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); nullptr when unavailable.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  if (!tried) {
    tried = true;
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)f;
    else
      (void)cudaGetLastError();
  }
  return fn;
}

// The two tensor maps of the TMA staging: weights as fp32 [nz][ny][nx][4]
// (box {4, TX, TY, nzb}) and distances as u32 [slices][nz][ny][nx] (box
// {TX + 8, TY + 2, nzb, 1}).  False (plain loads) when a stride or base is
// not 16-byte aligned or the encoder refuses.
bool encode_lattice_maps(const orsp::Graph *g, const LatParams &p, int TX, int TY, int nzb, int64_t slices,
                         CUtensorMap *tmw, CUtensorMap *tmd) {
  const int64_t nx = g->nx, ny = g->ny, nz = g->nz, N = (int64_t)g->N;
  if (nx % 4 != 0 || ((uintptr_t)p.dist & 15) != 0 || ((uintptr_t)p.w4 & 15) != 0) return false;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint32_t es[4] = {1, 1, 1, 1};
  const cuuint64_t dw[4] = {4, (cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
  const cuuint64_t sw[3] = {16, (cuuint64_t)(16 * nx), (cuuint64_t)(16 * nx * ny)};
  const cuuint32_t bw[4] = {4, (cuuint32_t)TX, (cuuint32_t)TY, (cuuint32_t)nzb};
  if (enc(tmw, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)p.w4, dw, sw, bw, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  const cuuint64_t dd[4] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)slices};
  const cuuint64_t sdd[3] = {(cuuint64_t)(4 * nx), (cuuint64_t)(4 * nx * ny), (cuuint64_t)(4 * N)};
  const cuuint32_t bd[4] = {(cuuint32_t)(TX + 8), (cuuint32_t)(TY + 2), (cuuint32_t)nzb, 1};
  if (enc(tmd, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, (void *)p.dist, dd, sdd, bd, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  return true;
}

template <int TX, int TY>
int launch_lattice(orsp::Graph *g, LatParams &p, int64_t ntiles, int nzb, int32_t nseeds, const int32_t *seeds,
                   const float *seed_cost, cudaStream_t st, orsp::LatOptions *opt) {
  // (column vias always take the asynchronous schedule)
  const bool async = p.wcol != nullptr || env_u64("ORSP_LAT_ASYNC", 1) != 0;
  const WsLayout L = ws_layout(g, ntiles);
  const size_t list_b = L.list_b, q_b = L.q_b;
  const unsigned qcap = L.qcap;
  int rc0 = grow_ws(g, L.total);
  if (rc0) return rc0;
  char *b = (char *)g->lat_ws;
  p.list0 = (int32_t *)b;
  p.list1 = (int32_t *)(b + list_b);
  p.stamp = (unsigned *)(b + 2 * list_b);
  p.tstate = (int *)(b + 3 * list_b);
  p.qslot = async ? (int32_t *)(b + 4 * list_b) : nullptr;
  p.qcap = qcap;
  p.ctl = (LatCtl *)(b + 4 * list_b + q_b);
  if (opt) opt->err_d = &p.ctl->err;
  if (!async) ORSP_CUDA(cudaMemsetAsync(p.stamp, 0, (size_t)ntiles * 4, st));
  ORSP_CUDA(cudaMemsetAsync(p.tstate, 0, (size_t)ntiles * 4, st));
  if (async) ORSP_CUDA(cudaMemsetAsync(p.qslot, 0xff, (size_t)qcap * 4, st));
  lattice_seed_kernel<TX, TY><<<1, 256, 0, st>>>(p, nseeds, seeds, seed_cost);
  ORSP_CUDA(cudaGetLastError());
  size_t smem = (size_t)nzb * tile_floats_per_layer(TX, TY) * sizeof(float);
  if (smem > 227 * 1024) {
    orsp::set_error("lattice search: too many layers for the shared-memory tile");
    return ORSP_ERR_ARG;
  }
  const bool priv = opt && opt->private_dist;
  // ORSP_LAT_SPEC=1: the warp-specialised asynchronous schedule
  const bool spec = async && !p.wcol && env_u64("ORSP_LAT_SPEC", (opt && opt->spec) ? 1 : 0) != 0;
  // ORSP_LAT_BLOCKS_PER_SM: CTAs per SM (tiles of up to 12 layers at width
  // 16 have an instantiation sized for 2)
  const int want = (int)env_u64("ORSP_LAT_BLOCKS_PER_SM", (opt && opt->blocks_per_sm > 0) ? opt->blocks_per_sm : 1);
  // ORSP_LAT_TMA=1: tensor-load staging of fresh visits, for whole-lattice
  // boxes (opt->tma_slices: distance slices of N cells, box j in slice j)
  CUtensorMap tmw{}, tmd{};
  bool tma = false;
  if constexpr (TX == 16) {
    if (async && !spec && !p.wcol && want < 2 && nzb <= 12 && nzb == g->nz && opt && opt->tma_slices > 0 &&
        env_u64("ORSP_LAT_TMA", 0) != 0)
      tma = encode_lattice_maps(g, p, TX, TY, nzb, opt->tma_slices, &tmw, &tmd);
  }
  if (tma) {
    const size_t base = ((size_t)nzb * tile_floats_per_layer(TX, TY) + 31) & ~(size_t)31;
    smem = (base + (size_t)nzb * TY * TX * 4 + (size_t)nzb * (TY + 2) * (TX + 8)) * sizeof(float);
  }
  void *kfn;
  if (p.wcol) {
    // column vias: the asynchronous schedule with the column via pass, one
    // CTA per SM, tile width 16
    if constexpr (TX == 16) {
      kfn = nzb > 12 ? (priv ? (void *)lattice_async_kernel<TX, TY, true, true, 1, false, true>
                             : (void *)lattice_async_kernel<TX, TY, false, true, 1, false, true>)
                     : (priv ? (void *)lattice_async_kernel<TX, TY, true, false, 1, false, true>
                             : (void *)lattice_async_kernel<TX, TY, false, false, 1, false, true>);
    } else {
      orsp::set_error("lattice search: column vias need tile width 16");
      return ORSP_ERR_ARG;
    }
  } else if (spec) {
    kfn = priv ? (void *)lattice_spec_kernel<TX, TY, true> : (void *)lattice_spec_kernel<TX, TY, false>;
    if constexpr (TX == 16) {  // two CTAs per SM: the instantiation held to their register share
      if (want >= 2 && nzb <= 12)
        kfn = priv ? (void *)lattice_spec_kernel<TX, TY, true, 2> : (void *)lattice_spec_kernel<TX, TY, false, 2>;
    }
  }
  else if (async) {
    kfn = priv ? (void *)lattice_async_kernel<TX, TY, true> : (void *)lattice_async_kernel<TX, TY, false>;
    if constexpr (TX == 16) {  // deeper tiles: the instantiation with 18-layer column loads
      if (tma)
        kfn = priv ? (void *)lattice_async_kernel<TX, TY, true, false, 1, true>
                   : (void *)lattice_async_kernel<TX, TY, false, false, 1, true>;
      else if (nzb > 12)
        kfn = priv ? (void *)lattice_async_kernel<TX, TY, true, true> : (void *)lattice_async_kernel<TX, TY, false, true>;
      else if (want >= 2)
        kfn = priv ? (void *)lattice_async_kernel<TX, TY, true, false, 2>
                   : (void *)lattice_async_kernel<TX, TY, false, false, 2>;
    }
  }
  else kfn = priv ? (void *)lattice_tile_kernel<TX, TY, true> : (void *)lattice_tile_kernel<TX, TY, false>;
  const int threads = TX * TY + (spec ? 32 : 0);
  // The shared-memory cap is a per-kernel attribute: it is raised to the
  // largest tile once per (kernel, device), never lowered, so a launch with a
  // smaller tile does not invalidate a cached larger one.  The occupancy is
  // cached per (kernel, block, shared memory, device).
  struct OccEntry {
    void *fn;
    int threads, device;
    size_t smem;
    int occ;
  };
  struct CapEntry {
    void *fn;
    int device;
  };
  static OccEntry occ_cache[64];
  static int occ_n = 0;
  static CapEntry cap_set[32];
  static int cap_n = 0;
  static std::mutex occ_mu;
  int occ = -1;
  {
    std::lock_guard<std::mutex> lock(occ_mu);
    bool capped = false;
    for (int i = 0; i < cap_n; ++i) capped = capped || (cap_set[i].fn == kfn && cap_set[i].device == g->device);
    if (!capped) {
      // the opt-in maximum less the kernel's static shared memory
      cudaFuncAttributes fa{};
      ORSP_CUDA(cudaFuncGetAttributes(&fa, kfn));
      int optin = 0;
      ORSP_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, g->device));
      ORSP_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     optin - (int)fa.sharedSizeBytes));
      if (cap_n < 32) cap_set[cap_n++] = CapEntry{kfn, g->device};
    }
    for (int i = 0; i < occ_n; ++i)
      if (occ_cache[i].fn == kfn && occ_cache[i].threads == threads && occ_cache[i].smem == smem &&
          occ_cache[i].device == g->device)
        occ = occ_cache[i].occ;
    if (occ < 0) {
      ORSP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, threads, smem));
      if (occ_n < 64) occ_cache[occ_n++] = OccEntry{kfn, threads, g->device, smem, occ};
    }
  }
  if (occ < 1) {
    orsp::set_error("lattice search: kernel does not fit on an SM");
    return ORSP_ERR_ARG;
  }
  const int bps = std::max(1, std::min(occ, want));
  p.max_rounds = (unsigned)std::min<unsigned long long>(64ull * (unsigned long long)ntiles + 4096ull, 1ull << 30);
  p.wait_ns = env_u64("ORSP_WAIT_NS", 2000000000ull);
  // ORSP_LAT_SELF=0: a tile to visit again goes back to the queue instead
  p.selfcont = (int)env_u64("ORSP_LAT_SELF", 1);
  // ORSP_LAT_PREFETCH=0: no L2 prefetch of the next tile by the scheduler warp
  p.prefetch = (int)env_u64("ORSP_LAT_PREFETCH", 1);
  p.budget_ns = env_u64("ORSP_BUDGET_NS", 20000000000ull);
  void *args[] = {&p, &tmw, &tmd};  // the tile and spec kernels take p only
  if (orsp::g_timer.on) ORSP_CUDA(cudaEventRecord(orsp::g_timer.a, st));
  // Cooperative launch in both schedules: every CTA is resident, so a CTA
  // waiting for a queue slot never blocks the CTA that will fill it.
  // (launched with the cooperative attribute rather than
  // cudaLaunchCooperativeKernel, so that a stream capture keeps the
  // co-residency guarantee in the graph's kernel node)
  cudaLaunchConfig_t lc{};
  lc.gridDim = dim3(g->num_sms * bps);
  lc.blockDim = dim3(threads);
  lc.dynamicSmemBytes = smem;
  lc.stream = st;
  cudaLaunchAttribute coop[1];
  coop[0].id = cudaLaunchAttributeCooperative;
  coop[0].val.cooperative = 1;
  lc.attrs = coop;
  lc.numAttrs = 1;
  ORSP_CUDA(cudaLaunchKernelExC(&lc, kfn, args));
  if (orsp::g_timer.on) {
    ORSP_CUDA(cudaEventRecord(orsp::g_timer.b, st));
    orsp::g_timer.pending = true;
  }
  if (!opt || opt->copy_ctl)
    ORSP_CUDA(cudaMemcpyAsync(g->lat_ctl_h, p.ctl, sizeof(LatCtl), cudaMemcpyDeviceToHost, st));
  return ORSP_OK;
}

}  // namespace

namespace orsp {

// Recognises the routing lattice: every planar edge a unit step along its
// layer's single routing axis, no parallel planar edges, and vias either all
// between adjacent layers without parallel edges (slots 2 and 3) or, as in
// the reference's Lattice3D (all-pairs blind/buried vias, duplicated via
// edges, unified_pathfinder.py:1136-1172, 1264-1276), between any two layers
// of a column with at most two parallel edges each (column vias, g->cvia).
int analyze_lattice(Graph *g, const int32_t *indptr_h, const int32_t *indices_h) {
  g->lattice_ok = false;
  g->cvia = false;
  if (g->nx <= 0 || g->ny <= 0 || g->nz <= 0 || g->nz > 64) return ORSP_OK;
  const int32_t N = g->N, nx = g->nx, ny = g->ny;
  const int64_t nxy = (int64_t)nx * ny;
  std::vector<int8_t> axis(g->nz, -1);
  std::vector<int32_t> slot((size_t)4 * N, -1);
  bool adjacent_vias = true;  // every via spans one layer, no parallel vias
  for (int32_t u = 0; u < N; ++u) {
    const int32_t zu = (int32_t)(u / nxy);
    const int32_t ru = (int32_t)(u - zu * nxy);
    const int32_t yu = ru / nx, xu = ru - yu * nx;
    for (int32_t k = indptr_h[u]; k < indptr_h[u + 1]; ++k) {
      const int32_t v = indices_h[k];
      const int32_t zv = (int32_t)(v / nxy);
      const int32_t rv = (int32_t)(v - zv * nxy);
      const int32_t yv = rv / nx, xv = rv - yv * nx;
      const int dz = zv - zu, dx = xv - xu, dy = yv - yu;
      int s = -1;
      if (dz == 0) {
        int ax;
        if (dy == 0 && (dx == 1 || dx == -1)) ax = 1;
        else if (dx == 0 && (dy == 1 || dy == -1)) ax = 2;
        else return ORSP_OK;  // not a unit planar step
        if (axis[zu] == -1) axis[zu] = (int8_t)ax;
        else if (axis[zu] != ax) return ORSP_OK;  // both axes on one layer
        s = (dx + dy > 0) ? 0 : 1;  // entering v from its lower / upper neighbour
      } else if (dx == 0 && dy == 0) {
        if (dz != 1 && dz != -1) {
          adjacent_vias = false;  // a via spanning layers: column vias
          continue;
        }
        s = dz > 0 ? 2 : 3;  // via from below / from above
      } else {
        return ORSP_OK;  // diagonal: not this lattice
      }
      int32_t &slotref = slot[(size_t)s * N + v];
      if (slotref != -1) {
        if (s < 2) return ORSP_OK;  // parallel planar edges
        adjacent_vias = false;      // parallel vias: column vias
        continue;
      }
      slotref = k;
    }
  }
  std::vector<int32_t> vcol;
  if (!adjacent_vias) {
    // column vias: every via in-edge of v by source layer, two parallel
    // edges at most (edge ids ascend with u and k, so k = 0 is the smaller)
    vcol.assign((size_t)2 * g->nz * N, -1);
    for (int32_t u = 0; u < N; ++u) {
      const int32_t zu = (int32_t)(u / nxy);
      const int64_t cu = u - (int64_t)zu * nxy;
      for (int32_t k = indptr_h[u]; k < indptr_h[u + 1]; ++k) {
        const int32_t v = indices_h[k];
        const int32_t zv = (int32_t)(v / nxy);
        if (zv == zu || v - (int64_t)zv * nxy != cu) continue;  // planar (checked above)
        int32_t *e0 = &vcol[((size_t)0 * g->nz + zu) * N + v];
        int32_t *e1 = &vcol[((size_t)1 * g->nz + zu) * N + v];
        if (*e0 < 0) *e0 = k;
        else if (*e1 < 0) *e1 = k;
        else return ORSP_OK;  // three parallel vias
      }
    }
    for (int32_t v = 0; v < N; ++v) slot[(size_t)2 * N + v] = slot[(size_t)3 * N + v] = -1;
  }
  for (int z = 0; z < g->nz; ++z) g->layer_axis[z] = axis[z] < 0 ? 0 : axis[z];
  ORSP_CUDA(cudaMalloc(&g->slot_eid, slot.size() * sizeof(int32_t)));
  ORSP_CUDA(cudaMemcpy(g->slot_eid, slot.data(), slot.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  ORSP_CUDA(cudaMalloc(&g->wslot, slot.size() * sizeof(float)));
  if (!adjacent_vias) {
    ORSP_CUDA(cudaMalloc(&g->vcol_eid, vcol.size() * sizeof(int32_t)));
    ORSP_CUDA(cudaMemcpy(g->vcol_eid, vcol.data(), vcol.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    // weights of every via in-edge of a node by source layer, nz rounded up
    // to 4 so that a node's row is whole float4s; layers without a via hold
    // +inf after each gather of the box, the rest is never read
    ORSP_CUDA(cudaMalloc(&g->wcol, (size_t)((g->nz + 3) & ~3) * N * sizeof(float)));
    g->cvia = true;
  }
  g->lattice_ok = true;
  return ORSP_OK;
}

void free_lattice(Graph *g) {
  cudaFree(g->slot_eid);
  cudaFree(g->wslot);
  cudaFree(g->vcol_eid);
  cudaFree(g->wcol);
  g->vcol_eid = nullptr;
  g->wcol = nullptr;
  g->cvia = false;
  cudaFree(g->lat_ws);
  cudaFree(g->lat_box_d);
  if (g->lat_ctl_h) cudaFreeHost(g->lat_ctl_h);
  g->lat_box_d = nullptr;
  g->slot_eid = nullptr;
  g->wslot = nullptr;
  g->lat_ws = nullptr;
  g->lat_ctl_h = nullptr;
}

int lattice_tile_w() { return env_u64("ORSP_LAT_TILE", 16) == 32 ? 32 : 16; }

bool lattice_tile_fits(int nzb, int tile_w) {
  const int TX = tile_w ? tile_w : lattice_tile_w(), TY = 16;
  const size_t smem = (size_t)nzb * tile_floats_per_layer(TX, TY) * sizeof(float);
  return smem <= 227 * 1024;
}

int reserve_lattice_ws(Graph *g, int64_t ntiles) { return grow_ws(g, ws_layout(g, ntiles).total); }

int64_t make_lat_boxes(const int32_t *boxes_h, int32_t nbox, LatBox *out, int tile_w) {
  const int TX = tile_w ? tile_w : lattice_tile_w(), TY = 16;
  int64_t t0 = 0;
  for (int32_t i = 0; i < nbox; ++i) {
    const int32_t *b = boxes_h + 6 * (int64_t)i;
    LatBox &B = out[i];
    B.x0 = b[0];
    B.x1 = b[1];
    B.y0 = b[2];
    B.y1 = b[3];
    B.z0 = b[4];
    B.z1 = b[5];
    B.ntx = (b[1] - b[0] + TX) / TX;
    B.nty = (b[3] - b[2] + TY) / TY;
    B.tile0 = (int32_t)t0;
    B.pad = 0;
    B.dbase = -1;
    t0 += (int64_t)B.ntx * B.nty;
  }
  return t0;
}

// Searches pairwise disjoint boxes in one launch.  Distances are reset to
// +inf everywhere (or, with opt->fill_box_only, inside the boxes only - the
// caller's backtrace must then test box membership); only the boxes' weights
// are gathered and only their tiles are visited.  Leaves the distances in
// `dist`; finish_lattice_search reports the status after the stream sync.
int run_lattice_boxes(Graph *g, const float *cost_d, int32_t nseeds, const int32_t *seeds_d,
                      const float *seed_cost_d, int32_t nbox, const int32_t *boxes_h, const LatBox *lboxes_d,
                      uint32_t *dist, cudaStream_t st, LatOptions *opt) {
  const int64_t N = g->N;
  const int TX = (opt && opt->tile_w) ? opt->tile_w : lattice_tile_w(), TY = 16;
  if (TX != 16 && TX != 32) { set_error("lattice search: tile width must be 16 or 32"); return ORSP_ERR_ARG; }
  const bool priv = opt && opt->private_dist;
  int64_t vol_sum = 0;
  int64_t ntiles = 0;
  int nzb = 1;
  bool whole = false;
  for (int32_t i = 0; i < nbox; ++i) {
    const int32_t *b = boxes_h + 6 * (int64_t)i;
    ntiles += (int64_t)((b[1] - b[0] + TX) / TX) * ((b[3] - b[2] + TY) / TY);
    nzb = std::max(nzb, b[5] - b[4] + 1);
    vol_sum += (int64_t)(b[1] - b[0] + 1) * (b[3] - b[2] + 1) * (b[5] - b[4] + 1);
    whole = whole || (b[0] == 0 && b[1] == g->nx - 1 && b[2] == 0 && b[3] == g->ny - 1 && b[4] == 0 &&
                      b[5] == g->nz - 1);
  }
  // overlapping boxes (own distances) may hold more cells than the lattice:
  // then one gather of every node is cheaper than one per box.  A whole
  // gather is skipped when the caller declared, for this search, the same
  // cost array and generation as the last whole gather's.
  const uint64_t decl = g->decl_cost == cost_d ? g->decl_gen : 0;
  g->decl_cost = nullptr;
  g->decl_gen = 0;
  // boxes with their own slices and device activity flags: only the active
  // boxes' weights are gathered and their slices reset (one launch each)
  const bool by_flag = priv && opt->active && !g->cvia && nbox <= 65535;
  int64_t vmax = 1;
  for (int32_t i = 0; i < nbox; ++i) {
    const int32_t *b = boxes_h + 6 * (int64_t)i;
    vmax = std::max<int64_t>(vmax, (int64_t)(b[1] - b[0] + 1) * (b[3] - b[2] + 1) * (b[5] - b[4] + 1));
  }
  const unsigned per_box = (unsigned)std::max<int64_t>(1, std::min<int64_t>((vmax + 255) / 256,
                                                                            148 * 32 / std::max(1, nbox)));
  if (by_flag) {
    g->w4_cost = nullptr;  // part of wslot is rewritten
    g->w4_gen = 0;
    gather_boxes_kernel<<<dim3(per_box, (unsigned)nbox), 256, 0, st>>>(g->slot_eid, cost_d, (float4 *)g->wslot, N,
                                                                       g->nx, g->ny, lboxes_d, opt->active);
    ORSP_CUDA(cudaGetLastError());
  } else if (whole || (priv && vol_sum >= N)) {
    if (!(decl != 0 && g->w4_cost == cost_d && g->w4_gen == decl)) {
      gather_kernel<<<(int)std::min<int64_t>((N + 255) / 256, 148 * 32), 256, 0, st>>>(
          g->slot_eid, cost_d, (float4 *)g->wslot, N);
      ORSP_CUDA(cudaGetLastError());
      if (g->cvia) {
        const int32_t full[6] = {0, g->nx - 1, 0, g->ny - 1, 0, g->nz - 1};
        int rc = gather_col_box(g, cost_d, full, nullptr, nullptr, nullptr, st);
        if (rc) return rc;
      }
      g->w4_cost = cost_d;
      g->w4_gen = decl;
    }
  } else {
    g->w4_cost = nullptr;  // part of wslot is rewritten
    g->w4_gen = 0;
    if (!g->cvia && nbox > 1 && nbox <= 65535) {
      // one launch for all boxes, as many blocks per box as the largest needs
      // (within a grid of about 32 blocks per SM)
      gather_boxes_kernel<<<dim3(per_box, (unsigned)nbox), 256, 0, st>>>(g->slot_eid, cost_d, (float4 *)g->wslot,
                                                                         N, g->nx, g->ny, lboxes_d, nullptr);
      ORSP_CUDA(cudaGetLastError());
    } else {
      for (int32_t i = 0; i < nbox; ++i) {
        const int32_t *b = boxes_h + 6 * (int64_t)i;
        const int32_t bw = b[1] - b[0] + 1, bh = b[3] - b[2] + 1;
        const int64_t count = (int64_t)bw * bh * (b[5] - b[4] + 1);
        gather_box_kernel<<<(int)std::min<int64_t>((count + 255) / 256, 148 * 32), 256, 0, st>>>(
            g->slot_eid, cost_d, (float4 *)g->wslot, N, g->nx, g->ny, b[0], bw, b[2], bh, b[4], count);
        ORSP_CUDA(cudaGetLastError());
        if (g->cvia) {
          int rc = gather_col_box(g, cost_d, b, nullptr, nullptr, nullptr, st);
          if (rc) return rc;
        }
      }
    }
  }
  if (by_flag) {
    fill_slices_kernel<<<dim3(per_box, (unsigned)nbox), 256, 0, st>>>(dist, lboxes_d, opt->active, ORSP_INF_BITS);
    ORSP_CUDA(cudaGetLastError());
  } else if (priv) {
    fill_kernel<<<(int)std::min<int64_t>((opt->private_count + 255) / 256, 148 * 32), 256, 0, st>>>(
        dist, opt->private_count, ORSP_INF_BITS);
    ORSP_CUDA(cudaGetLastError());
  } else if (opt && opt->fill_box_only && !whole) {
    for (int32_t i = 0; i < nbox; ++i) {
      const int32_t *b = boxes_h + 6 * (int64_t)i;
      const int32_t bw = b[1] - b[0] + 1, bh = b[3] - b[2] + 1;
      const int64_t count = (int64_t)bw * bh * (b[5] - b[4] + 1);
      fill_box_kernel<<<(int)std::min<int64_t>((count + 255) / 256, 148 * 32), 256, 0, st>>>(
          dist, g->nx, g->ny, b[0], bw, b[2], bh, b[4], count, ORSP_INF_BITS);
      ORSP_CUDA(cudaGetLastError());
    }
  } else {
    fill_kernel<<<(int)std::min<int64_t>((N + 255) / 256, 148 * 32), 256, 0, st>>>(dist, N, ORSP_INF_BITS);
    ORSP_CUDA(cudaGetLastError());
  }
  LatParams p{};
  p.nx = g->nx;
  p.ny = g->ny;
  p.nz = g->nz;
  p.nbox = nbox;
  p.seed_per_box = priv ? 1 : 0;
  p.boxes = lboxes_d;
  p.w4 = (const float4 *)g->wslot;
  p.wcol = g->cvia ? g->wcol : nullptr;
  p.nzp = (g->nz + 3) & ~3;
  p.N = N;
  p.dist = dist;
  for (int z = 0; z < 64; ++z) p.axis[z] = z < g->nz ? g->layer_axis[z] : 0;
  if (TX == 32) return launch_lattice<32, 16>(g, p, ntiles, nzb, nseeds, seeds_d, seed_cost_d, st, opt);
  return launch_lattice<16, 16>(g, p, ntiles, nzb, nseeds, seeds_d, seed_cost_d, st, opt);
}

int run_lattice_search(Graph *g, const float *cost_d, int32_t nseeds, const int32_t *seeds_d,
                       const float *seed_cost_d, const int32_t *box, uint32_t *dist, cudaStream_t st,
                       LatOptions *opt) {
  const int32_t full[6] = {0, g->nx - 1, 0, g->ny - 1, 0, g->nz - 1};
  const int32_t *b = box ? box : full;
  if (!g->lat_box_d) ORSP_CUDA(cudaMalloc(&g->lat_box_d, sizeof(LatBox)));
  LatBox *hb = (LatBox *)((char *)g->pinned + 1024);
  make_lat_boxes(b, 1, hb);
  ORSP_CUDA(cudaMemcpyAsync(g->lat_box_d, hb, sizeof(LatBox), cudaMemcpyHostToDevice, st));
  return run_lattice_boxes(g, cost_d, nseeds, seeds_d, seed_cost_d, 1, b, (const LatBox *)g->lat_box_d, dist, st,
                           opt);
}

int run_lattice_roi(Graph *g, const float *cost_d, int32_t nseeds, const int32_t *seeds_d,
                    const float *seed_cost_d, const int32_t *roi_map_d, const int32_t *roi_nodes_d,
                    int64_t n_roi, const uint8_t *sink_d, uint32_t *dist, cudaStream_t st) {
  const int64_t N = g->N;
  const int TX = lattice_tile_w(), TY = 16;
  if (!g->lat_box_d) ORSP_CUDA(cudaMalloc(&g->lat_box_d, sizeof(LatBox)));
  int rc = ensure_roi_arrays(g);
  if (rc) return rc;
  LatBox *box_d = (LatBox *)g->lat_box_d;
  const int gblocks = g->num_sms * 8;
  if (!roi_map_d && !roi_nodes_d) {
    const int32_t full[6] = {0, g->nx - 1, 0, g->ny - 1, 0, g->nz - 1};
    LatBox *hb = (LatBox *)((char *)g->pinned + 1024);
    make_lat_boxes(full, 1, hb, TX);
    ORSP_CUDA(cudaMemcpyAsync(box_d, hb, sizeof(LatBox), cudaMemcpyHostToDevice, st));
  } else {
    // running maxima start at 0x80808080, below every coordinate
    ORSP_CUDA(cudaMemsetAsync(g->roi_bb, 0x80, 6 * sizeof(int), st));
    const int64_t n = roi_nodes_d ? n_roi : N;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, gblocks));
    roi_bbox_kernel<<<blocks, 256, 0, st>>>(roi_nodes_d, n, roi_map_d, g->nx, g->ny, N, g->roi_bb);
    ORSP_CUDA(cudaGetLastError());
    if (TX == 32) roi_box_finish_kernel<32, 16><<<1, 1, 0, st>>>(g->roi_bb, box_d);
    else roi_box_finish_kernel<16, 16><<<1, 1, 0, st>>>(g->roi_bb, box_d);
    ORSP_CUDA(cudaGetLastError());
  }
  RoiGeom G{};
  G.nx = g->nx;
  G.ny = g->ny;
  G.nz = g->nz;
  for (int z = 0; z < 64; ++z) G.axis[z] = z < g->nz ? g->layer_axis[z] : 0;
  gather_roi_kernel<<<(int)std::min<int64_t>((N + 255) / 256, gblocks), 256, 0, st>>>(
      g->slot_eid, cost_d, (float4 *)g->wslot, N, G, box_d, roi_map_d, sink_d);
  ORSP_CUDA(cudaGetLastError());
  if (g->cvia) {
    rc = gather_col_box(g, cost_d, nullptr, box_d, roi_map_d, sink_d, st);
    if (rc) return rc;
  }
  g->w4_cost = nullptr;  // masked weights: not reusable by a whole search
  g->w4_gen = 0;
  g->decl_cost = nullptr;
  g->decl_gen = 0;
  fill_kernel<<<(int)std::min<int64_t>((N + 255) / 256, 148 * 32), 256, 0, st>>>(dist, N, ORSP_INF_BITS);
  ORSP_CUDA(cudaGetLastError());
  LatParams p{};
  p.nx = g->nx;
  p.ny = g->ny;
  p.nz = g->nz;
  p.nbox = 1;
  p.seed_per_box = 0;
  p.boxes = box_d;
  p.w4 = (const float4 *)g->wslot;
  p.wcol = g->cvia ? g->wcol : nullptr;
  p.nzp = (g->nz + 3) & ~3;
  p.N = N;
  p.dist = dist;
  p.roi_map = roi_map_d;
  for (int z = 0; z < 64; ++z) p.axis[z] = z < g->nz ? g->layer_axis[z] : 0;
  // the box is known on the device only: size the tile arrays for the lattice
  const int64_t ntiles = (int64_t)((g->nx - 1 + TX) / TX) * ((g->ny - 1 + TY) / TY);
  if (TX == 32) return launch_lattice<32, 16>(g, p, ntiles, g->nz, nseeds, seeds_d, seed_cost_d, st, nullptr);
  return launch_lattice<16, 16>(g, p, ntiles, g->nz, nseeds, seeds_d, seed_cost_d, st, nullptr);
}

int finish_lattice_search(Graph *g, int32_t *rounds_h) {
  const LatCtl *c = (const LatCtl *)g->lat_ctl_h;
  if (rounds_h) *rounds_h = (int32_t)c->rounds;
  g_counters[0] = c->rounds;
  g_counters[1] = c->visits;
  g_counters[2] = (int64_t)c->cycles;
  for (int i = 0; i < 4; ++i) g_counters[4 + i] = (int64_t)c->ns[i];
  if (c->err) return dev_status_to_orsp(c->err);
  return ORSP_OK;
}

}  // namespace orsp

extern "C" int orsp_graph_cost_generation(orsp_graph *g, const float *cost_d, uint64_t generation) {
  if (!g || !cost_d) {
    orsp::set_error("cost_generation: NULL argument");
    return ORSP_ERR_ARG;
  }
  g->decl_cost = cost_d;
  g->decl_gen = generation;
  return ORSP_OK;
}

extern "C" int orsp_lattice_max_layers(int32_t tile_w, int32_t *out) {
  if (!out || (tile_w != 0 && tile_w != 16 && tile_w != 32)) {
    orsp::set_error("lattice_max_layers: tile width must be 0, 16 or 32");
    return ORSP_ERR_ARG;
  }
  int n = 0;
  while (n < 64 && orsp::lattice_tile_fits(n + 1, tile_w)) ++n;
  *out = n;
  return ORSP_OK;
}
