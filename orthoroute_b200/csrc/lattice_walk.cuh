// Predecessor walk on the H/V routing lattice.
//
// On the lattice every node v = (x, y, z) has at most four in-neighbours, one
// per slot of the gathered in-edge weights w4[v] (orsp_lattice.cu), or, with
// column vias, its two planar in-neighbours and one via from every other
// layer of its column (LatWalkGeom::wcol):
//   slot 0: the lower neighbour along the layer's axis (x-1 on H layers, y-1 on
//           V layers), slot 1: the upper one (x+1 / y+1),
//   slot 2: the via from below (z-1), slot 3: the via from above (z+1).
// So the parent of v under the settle-order rule of the heap Dijkstra
// (SimpleDijkstra.find_path_roi, unified_pathfinder.py:1846-1887: the
// in-neighbour u with fl32(d[u] + w(u,v)) == d[v] and the smallest
// (d[u], rank u) below (d[v], rank v)) needs one float4 and four distances,
// all independent loads: one memory round trip per step of the walk, where a
// walk over the transposed CSR needs three dependent ones (row pointer, source
// list, distance).  Ranks are node ids by default (box searches rank nodes in
// id order, and a box's own distance slice is laid out in that order too);
// ROI searches pass the ROI index (global_to_roi) as the rank.
#pragma once

#include "common.cuh"

namespace orsp {

struct LatWalkGeom {
  int32_t nx, ny, nz;
  int8_t axis[64];  // 1: x moves (H layer), 2: y moves (V layer), 0: none
  // column vias (the reference's Lattice3D): a node's via in-edges come from
  // every layer of its column, with weights wcol[v * nzp + za] (slots 2 and 3
  // are empty); NULL on a lattice with adjacent vias only
  const float *wcol = nullptr;
  int32_t nzp = 0;
};

// Rank of a node for the tie-break: its id.
struct LatRankId {
  __device__ __forceinline__ int64_t operator()(int64_t v) const { return v; }
};

// Rank of a node inside a node-set ROI: its index in the ROI list
// (global_to_roi[v]); nodes outside the ROI never qualify as parents, since
// their distances stay +inf.
struct LatRankRoi {
  const int32_t *g2r;
  __device__ __forceinline__ int64_t operator()(int64_t v) const { return __ldg(&g2r[v]); }
};

// Coordinates of a node id.
__device__ __forceinline__ void lat_xyz(const LatWalkGeom &G, int64_t v, int32_t &x, int32_t &y, int32_t &z) {
  const int64_t plane = (int64_t)G.nx * G.ny;
  z = (int32_t)(v / plane);
  const int64_t r = v - (int64_t)z * plane;
  y = (int32_t)(r / G.nx);
  x = (int32_t)(r - (int64_t)y * G.nx);
}

// Neighbour of (x, y, z) through slot s, or false if it leaves box B.
__device__ __forceinline__ bool lat_slot_nbr(const LatWalkGeom &G, const LatBox &B, int s, int32_t x, int32_t y,
                                             int32_t z, int32_t &ux, int32_t &uy, int32_t &uz) {
  ux = x;
  uy = y;
  uz = z;
  if (s < 2) {
    const int d = s == 0 ? -1 : 1;
    if (G.axis[z] == 1) ux += d;
    else if (G.axis[z] == 2) uy += d;
    else return false;
  } else {
    uz += s == 2 ? -1 : 1;
  }
  return ux >= B.x0 && ux <= B.x1 && uy >= B.y0 && uy <= B.y1 && uz >= B.z0 && uz <= B.z1;
}

// One step of the walk at v = (x, y, z) with distance bits dv.  DIST(x, y, z)
// gives the distance bits of a node inside the box, RANK(node) its rank.
// Returns the slot of the parent (and its coordinates and distance bits), or
// -1 when no in-neighbour qualifies.
template <class DIST, class RANK = LatRankId>
__device__ __forceinline__ int lat_parent(const LatWalkGeom &G, const LatBox &B, const float4 *__restrict__ w4,
                                          DIST dist, int32_t x, int32_t y, int32_t z, unsigned dv,
                                          int32_t &px, int32_t &py, int32_t &pz, unsigned &pdu,
                                          RANK rank = RANK()) {
  const int64_t v = ((int64_t)z * G.ny + y) * G.nx + x;
  const float4 wv = __ldcg(&w4[v]);
  const float wk[4] = {wv.x, wv.y, wv.z, wv.w};
  unsigned du[4];
  int32_t ux[4], uy[4], uz[4];
  bool ok[4];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    ok[s] = lat_slot_nbr(G, B, s, x, y, z, ux[s], uy[s], uz[s]);
    du[s] = ok[s] ? dist(ux[s], uy[s], uz[s]) : ORSP_INF_BITS;
  }
  unsigned long long best = ULLONG_MAX;
  int bs = -1;
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    if (!ok[s] || du[s] == ORSP_INF_BITS) continue;
    if (f_bits(__fadd_rn(bits_f(du[s]), wk[s])) != dv) continue;
    const int64_t ru = rank(((int64_t)uz[s] * G.ny + uy[s]) * G.nx + ux[s]);
    if (!(du[s] < dv || (du[s] == dv && ru < rank(v)))) continue;
    const unsigned long long key = ((unsigned long long)du[s] << 32) | (unsigned long long)(uint32_t)ru;
    if (key < best) {
      best = key;
      bs = s;
    }
  }
  if (G.wcol) {
    // column vias: a parent in any other layer of the box in this column
    // (slot 4 + its layer)
    const float *wr = G.wcol + v * G.nzp;
    for (int32_t za = B.z0; za <= B.z1; ++za) {
      if (za == z) continue;
      const float w = __ldg(&wr[za]);
      if (!(w < __int_as_float(0x7f800000))) continue;
      const unsigned d = dist(x, y, za);
      if (d == ORSP_INF_BITS || f_bits(__fadd_rn(bits_f(d), w)) != dv) continue;
      const int64_t ru = rank(((int64_t)za * G.ny + y) * G.nx + x);
      if (!(d < dv || (d == dv && ru < rank(v)))) continue;
      const unsigned long long key = ((unsigned long long)d << 32) | (unsigned long long)(uint32_t)ru;
      if (key < best) {
        best = key;
        bs = 4 + za;
      }
    }
    if (bs >= 4) {
      px = x;
      py = y;
      pz = bs - 4;
      pdu = (unsigned)(best >> 32);
      return bs;
    }
  }
  if (bs >= 0) {
    px = ux[bs];
    py = uy[bs];
    pz = uz[bs];
    pdu = (unsigned)(best >> 32);
  }
  return bs;
}

// Cell i steps from (x, y, z) through slot s (the direction a straight run of
// parents takes when every parent sits in slot s of its child), or false if
// it leaves box B.
__device__ __forceinline__ bool lat_run_cell(const LatWalkGeom &G, const LatBox &B, int s, int i, int32_t x,
                                             int32_t y, int32_t z, int32_t &cx, int32_t &cy, int32_t &cz) {
  cx = x;
  cy = y;
  cz = z;
  if (s < 2) {
    const int d = s == 0 ? -i : i;
    if (G.axis[z] == 1) cx += d;
    else if (G.axis[z] == 2) cy += d;
    else if (i) return false;
  } else if (s < 4) {
    cz += s == 2 ? -i : i;
  } else if (i) {
    return false;  // a column via (slot 4 + layer) is a single step
  }
  return cx >= B.x0 && cx <= B.x1 && cy >= B.y0 && cy <= B.y1 && cz >= B.z0 && cz <= B.z1;
}

// The whole walk, by one full warp, from node (x, y, z) with distance bits dv
// until STOP(node, dv) holds for the node just appended.  Nodes are appended
// to out[0..cap) from the target back to the start.  Returns the length, or
// -1 (more than cap nodes) / -2 (a node without a qualifying parent).
//
// Paths on the lattice are mostly straight runs, so each round lane i takes
// the cell i steps ahead of the current node along the direction of the last
// step and computes that cell's parent with lat_parent, all lanes at once (one
// memory round trip).  Where the parent of lane i's cell is lane i+1's cell,
// the run goes on; the first lane where it does not ends the round, and its
// parent is the next current node.  Each lane's parent is the one the
// sequential walk computes at that node (same distances, same rule), so the
// nodes are those of the one-step walk; a round advances by up to 32 nodes.
template <class DIST, class STOP, class RANK = LatRankId>
__device__ __forceinline__ int lat_walk_warp(const LatWalkGeom &G, const LatBox &B, const float4 *__restrict__ w4,
                                             DIST dist, STOP stop, int32_t x, int32_t y, int32_t z, unsigned dv,
                                             int32_t *out, int32_t cap, RANK rank = RANK()) {
  const int lane = threadIdx.x & 31;
  int len = 0;
  int s = 0;  // predicted slot: the direction of the last step
  for (;;) {
    int32_t cx, cy, cz;
    const bool valid = lat_run_cell(G, B, s, lane, x, y, z, cx, cy, cz);
    const int64_t c = ((int64_t)cz * G.ny + cy) * G.nx + cx;
    const unsigned dc = lane == 0 ? dv : (valid ? dist(cx, cy, cz) : ORSP_INF_BITS);
    const bool is_stop = valid && dc != ORSP_INF_BITS && stop(c, dc);
    int ps = -1;
    int32_t px = 0, py = 0, pz = 0;
    unsigned pdu = 0;
    if (valid && dc != ORSP_INF_BITS && !is_stop) ps = lat_parent(G, B, w4, dist, cx, cy, cz, dc, px, py, pz, pdu, rank);
    const bool cont = valid && !is_stop && ps == s && lane < 31;
    const unsigned m = __ballot_sync(ORSP_FULL_MASK, cont);
    const int last = __ffs(~m) - 1;  // lane 31 never continues
    if (lane <= last && len + lane < cap) out[len + lane] = (int32_t)c;
    if (len + last + 1 > cap) return -1;
    len += last + 1;
    if (__shfl_sync(ORSP_FULL_MASK, is_stop, last)) return len;
    s = __shfl_sync(ORSP_FULL_MASK, ps, last);
    if (s < 0) return -2;
    x = __shfl_sync(ORSP_FULL_MASK, px, last);
    y = __shfl_sync(ORSP_FULL_MASK, py, last);
    z = __shfl_sync(ORSP_FULL_MASK, pz, last);
    dv = __shfl_sync(ORSP_FULL_MASK, pdu, last);
  }
}

// Slot of the in-edge u -> v between lattice neighbours u and v (node ids).
__device__ __forceinline__ int lat_edge_slot(const LatWalkGeom &G, int64_t u, int64_t v) {
  const int64_t plane = (int64_t)G.nx * G.ny;
  const int64_t zu = u / plane, zv = v / plane;
  if (zu < zv) return 2;
  if (zu > zv) return 3;
  return u < v ? 0 : 1;
}

}  // namespace orsp
