// Geometry emission on the device: committed node paths -> straight track
// runs and vias, as PathFinderRouter._generate_geometry_from_paths
// (orthoroute/algorithms/manhattan/unified_pathfinder.py:5749-5834), one
// thread per net walking its path with the reference's rules:
//   * a planar step on the first or last layer is dropped and restarts the
//     run at its end node (the reference's outer-layer guard);
//   * a planar step that is not a unit step, or that moves across the layer's
//     axis (y on 'h' layers, x on any other), is skipped without moving on;
//   * a layer change flushes the pending run and emits a via from the
//     previous node; a change of direction flushes the run up to the turn.
// Output in node terms (run start node, run end node, layer) and (via node,
// from layer, to layer); world coordinates are an affine map done by the
// caller.
#include <algorithm>

#include "common.cuh"

namespace {

struct GeomParams {
  const int32_t *paths;
  const int64_t *off;
  int32_t M;
  int32_t nx, ny, nz;
  int32_t *tracks;  // [sum of path lengths][3]: a, b, layer (rows from off[m])
  int32_t *vias;    // [sum of path lengths][3]: node, from layer, to layer
  int32_t *ntracks, *nvias;
  int8_t axis[64];  // 1: 'h' layer (x moves only), otherwise y moves only
};

__global__ void emit_geometry_kernel(GeomParams p) {
  const int64_t plane = (int64_t)p.nx * p.ny;
  for (int32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < p.M; m += gridDim.x * blockDim.x) {
    const int64_t a = p.off[m], b = p.off[m + 1];
    int nt = 0, nv = 0;
    if (b > a) {
      int32_t *tr = p.tracks + 3 * a;
      int32_t *vi = p.vias + 3 * a;
      int32_t run_start = p.paths[a], prev = run_start;
      int prev_dir = -1;  // -1: none; else (sx + 1) * 3 + (sy + 1)
      int32_t prev_layer = (int32_t)(prev / plane);
      for (int64_t i = a + 1; i < b; ++i) {
        const int32_t node = p.paths[i];
        const int32_t z0 = (int32_t)(prev / plane), r0 = (int32_t)(prev - z0 * plane);
        const int32_t z1 = (int32_t)(node / plane), r1 = (int32_t)(node - z1 * plane);
        const int32_t y0 = r0 / p.nx, x0 = r0 - y0 * p.nx, y1 = r1 / p.nx, x1 = r1 - y1 * p.nx;
        if (z0 == z1 && (z0 == 0 || z0 == p.nz - 1)) {  // outer-layer guard
          prev = node;
          prev_layer = z1;
          run_start = node;
          continue;
        }
        const int dx = abs(x1 - x0), dy = abs(y1 - y0);
        if (z0 == z1) {
          if (dx + dy != 1) continue;
          if (p.axis[z0] == 1) {
            if (dy != 0) continue;
          } else if (dx != 0) {
            continue;
          }
        }
        if (z1 != z0) {
          if (prev != run_start) {
            tr[3 * nt + 0] = run_start;
            tr[3 * nt + 1] = prev;
            tr[3 * nt + 2] = prev_layer;
            ++nt;
          }
          vi[3 * nv + 0] = prev;
          vi[3 * nv + 1] = z0;
          vi[3 * nv + 2] = z1;
          ++nv;
          run_start = node;
          prev_dir = -1;
        } else {
          const int dir = ((x1 > x0) - (x1 < x0) + 1) * 3 + ((y1 > y0) - (y1 < y0) + 1);
          if (prev_dir != -1 && dir != prev_dir) {
            tr[3 * nt + 0] = run_start;
            tr[3 * nt + 1] = prev;
            tr[3 * nt + 2] = prev_layer;
            ++nt;
            run_start = prev;
          }
          prev_dir = dir;
        }
        prev = node;
        prev_layer = z1;
      }
      if (prev != run_start) {
        tr[3 * nt + 0] = run_start;
        tr[3 * nt + 1] = prev;
        tr[3 * nt + 2] = prev_layer;
        ++nt;
      }
    }
    p.ntracks[m] = nt;
    p.nvias[m] = nv;
  }
}

}  // namespace

using namespace orsp;

extern "C" int orsp_emit_geometry(orsp_graph *g, int32_t M, const int32_t *paths_d, const int64_t *off_d,
                                  const int8_t *layer_axis_h, int32_t *tracks_d, int32_t *vias_d,
                                  int32_t *ntracks_d, int32_t *nvias_d, uintptr_t stream) {
  if (!g || M < 0 || (M > 0 && (!paths_d || !off_d || !tracks_d || !vias_d || !ntracks_d || !nvias_d)) ||
      !layer_axis_h) {
    set_error("emit_geometry: bad arguments");
    return ORSP_ERR_ARG;
  }
  if (g->nx <= 0 || g->nz <= 0 || g->nz > 64) { set_error("emit_geometry: needs lattice dims (nz <= 64)"); return ORSP_ERR_ARG; }
  if (M == 0) return ORSP_OK;
  ORSP_CUDA(cudaSetDevice(g->device));
  GeomParams p{};
  p.paths = paths_d;
  p.off = off_d;
  p.M = M;
  p.nx = g->nx;
  p.ny = g->ny;
  p.nz = g->nz;
  p.tracks = tracks_d;
  p.vias = vias_d;
  p.ntracks = ntracks_d;
  p.nvias = nvias_d;
  for (int z = 0; z < 64; ++z) p.axis[z] = z < g->nz ? layer_axis_h[z] : 0;
  emit_geometry_kernel<<<std::max(1, (M + 127) / 128), 128, 0, (cudaStream_t)stream>>>(p);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}
