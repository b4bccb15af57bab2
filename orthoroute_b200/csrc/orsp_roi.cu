// ROI extraction: bidirectional level-synchronous BFS, as
// ROIExtractor.extract_roi_bfs (UPF:1636-1734).
//
// Marks live in one byte per node (0 unseen, 1 src wave, 2 dst wave, 3 both)
// and are updated with a 32-bit atomicOr on the containing word: OR-ing the
// wave's mark reproduces the reference's three cases exactly (unseen -> mark;
// other wave or both -> 3, which ends the expansion; own mark -> unchanged),
// and the set of marked nodes after each step does not depend on the order in
// which the frontier is processed.  The ROI is then the marked nodes in
// ascending id order (np.where), produced by an order-preserving compaction.
#include <algorithm>
#include <mutex>
#include <string>

#include "common.cuh"

namespace {

constexpr int BFS_THREADS = 1024;

__device__ __forceinline__ unsigned or_mark(uint8_t *seen, int v, unsigned mark) {
  unsigned *word = (unsigned *)(seen + (v & ~3));
  const int sh = (v & 3) * 8;
  const unsigned old = atomicOr(word, mark << sh);
  return (old >> sh) & 0xffu;
}

struct BfsCtl {
  int total;   // marked nodes
  int depth;
  int met;
  int err;
};

// One CTA runs the whole expansion (depth <= 150 in the reference).
__global__ void __launch_bounds__(BFS_THREADS) roi_bfs_kernel(
    const int32_t *__restrict__ indptr, const int32_t *__restrict__ indices, int32_t N,
    int32_t src, int32_t dst, int32_t max_depth, int32_t max_nodes, uint8_t *seen,
    int32_t *qs0, int32_t *qs1, int32_t *qd0, int32_t *qd1, BfsCtl *ctl) {
  __shared__ int s_next;
  __shared__ int s_met;
  __shared__ int s_err;
  int n_src = 1, n_dst = 1;
  int32_t *qs = qs0, *qs_next = qs1, *qd = qd0, *qd_next = qd1;
  int total;
  if (threadIdx.x == 0) {
    seen[src] = 1;
    seen[dst] = 2;  // src == dst leaves mark 2, as the reference does
    qs[0] = src;
    qd[0] = dst;
    s_met = 0;
    s_err = 0;
  }
  total = (src == dst) ? 1 : 2;
  __syncthreads();
  int depth = 0;
  bool met = false;
  const double limit = (double)max_nodes * 1.5;
  while (depth < max_depth && (n_src > 0 || n_dst > 0) && !met) {
    for (int wave = 0; wave < 2; ++wave) {
      if (wave == 1 && met) break;
      const unsigned mark = wave == 0 ? 1u : 2u;
      const int n = wave == 0 ? n_src : n_dst;
      const int32_t *q = wave == 0 ? qs : qd;
      int32_t *qn = wave == 0 ? qs_next : qd_next;
      if (threadIdx.x == 0) s_next = 0;
      __syncthreads();
      bool met_local = false;
      for (int base = 0; base < n; base += BFS_THREADS) {
        const int i = base + threadIdx.x;
        int beg = 0, end = 0;
        if (i < n) {
          const int u = q[i];
          beg = indptr[u];
          end = indptr[u + 1];
        }
        const int deg = end - beg;
        const int maxdeg = __reduce_max_sync(ORSP_FULL_MASK, deg);
        for (int k = 0; k < maxdeg; ++k) {
          bool push = false;
          int v = 0;
          if (k < deg) {
            v = indices[beg + k];
            const unsigned old = or_mark(seen, v, mark);
            if (old == 0) push = true;
            else if (old != mark) met_local = true;
          }
          const unsigned m = __ballot_sync(ORSP_FULL_MASK, push);
          if (m) {
            const int lane = threadIdx.x & 31;
            const int leader = __ffs(m) - 1;
            int basei = 0;
            if (lane == leader) basei = atomicAdd(&s_next, __popc(m));
            basei = __shfl_sync(ORSP_FULL_MASK, basei, leader);
            if (push) {
              const int idx = basei + __popc(m & lanemask_lt());
              if (idx < N) qn[idx] = v; else s_err = 1;
            }
          }
        }
      }
      if (met_local) s_met = 1;
      __syncthreads();
      const int nn = s_next;
      total += nn;
      met = s_met != 0;
      if (wave == 0) {
        n_src = nn;
        int32_t *t = qs; qs = qs_next; qs_next = t;
      } else {
        n_dst = nn;
        int32_t *t = qd; qd = qd_next; qd_next = t;
      }
      __syncthreads();  // s_next is reset by the next wave
    }
    ++depth;
    if ((double)total > limit) break;
  }
  if (threadIdx.x == 0) {
    ctl->total = total;
    ctl->depth = depth;
    ctl->met = met ? 1 : 0;
    ctl->err = s_err;
  }
}

constexpr int CMP_THREADS = 512;
constexpr int CMP_ITEMS = 16;  // nodes per thread per tile
constexpr int CMP_TILE = CMP_THREADS * CMP_ITEMS;

__device__ __forceinline__ int block_excl_scan(int v, int *smem_warp, int *total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(ORSP_FULL_MASK, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem_warp[w] = x;
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    int s = lane < nw ? smem_warp[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(ORSP_FULL_MASK, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) smem_warp[lane] = s;
  }
  __syncthreads();
  const int warp_off = w > 0 ? smem_warp[w - 1] : 0;
  *total = smem_warp[(blockDim.x >> 5) - 1];
  const int r = warp_off + x - v;
  __syncthreads();
  return r;
}

// Pass 1: marked-node count per tile.
__global__ void __launch_bounds__(CMP_THREADS) count_tiles_kernel(const uint8_t *seen, int32_t N,
                                                                  int32_t *tile_cnt) {
  __shared__ int sw[32];
  const int64_t t0 = (int64_t)blockIdx.x * CMP_TILE;
  int c = 0;
  for (int j = 0; j < CMP_ITEMS; ++j) {
    const int64_t v = t0 + (int64_t)j * CMP_THREADS + threadIdx.x;
    if (v < N && seen[v]) ++c;
  }
  int tot;
  block_excl_scan(c, sw, &tot);
  if (threadIdx.x == 0) tile_cnt[blockIdx.x] = tot;
}

// Pass 2: exclusive scan of tile counts (one block, serial over chunks).
__global__ void __launch_bounds__(1024) scan_tiles_kernel(int32_t *tile_cnt, int32_t ntiles,
                                                          int32_t *total_out) {
  __shared__ int sw[32];
  int carry = 0;
  for (int base = 0; base < ntiles; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int v = i < ntiles ? tile_cnt[i] : 0;
    int tot;
    const int ex = block_excl_scan(v, sw, &tot);
    if (i < ntiles) tile_cnt[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) *total_out = carry;
}

// Pass 3: write marked ids in ascending order.  Within a tile, node
// t0 + j*THREADS + tid is visited in (j, tid) order, which is ascending.
__global__ void __launch_bounds__(CMP_THREADS) write_tiles_kernel(const uint8_t *seen, int32_t N,
                                                                  const int32_t *tile_off,
                                                                  int32_t *out) {
  __shared__ int sw[32];
  const int64_t t0 = (int64_t)blockIdx.x * CMP_TILE;
  int base = tile_off[blockIdx.x];
  for (int j = 0; j < CMP_ITEMS; ++j) {
    const int64_t v = t0 + (int64_t)j * CMP_THREADS + threadIdx.x;
    const int f = (v < N && seen[v]) ? 1 : 0;
    int tot;
    const int ex = block_excl_scan(f, sw, &tot);
    if (f) out[base + ex] = (int32_t)v;
    base += tot;
  }
}

// Truncation to max_nodes with the reference's must-keep swap (UPF:1705-1722):
// for the k-th kept node (in list order) at position p >= max_nodes, swap it
// with position k; then keep the first max_nodes entries.
__global__ void truncate_kernel(int32_t *roi, const int32_t *count_in, int32_t max_nodes,
                                int32_t src, int32_t dst, int32_t *count_out) {
  if (threadIdx.x != 0) return;
  const int n = *count_in;
  int cnt = n;
  if (n > max_nodes) {
    // positions of must-keep nodes in list order
    int kept[2];
    int nk = 0;
    for (int i = 0; i < n && nk < 2; ++i) {
      const int v = roi[i];
      if (v == src || v == dst) kept[nk++] = i;
    }
    for (int k = 0; k < nk; ++k) {
      const int p = kept[k];
      if (p >= max_nodes) {
        const int t = roi[p];
        roi[p] = roi[k];
        roi[k] = t;
      }
    }
    cnt = max_nodes;
  }
  *count_out = cnt;
}

// The same truncation with a general must-keep list, as extract_roi_bfs does
// with portal seeds (UPF:1700-1731): must_keep = [src, dst] followed by the
// keep nodes not already in it (list order); the ones missing from the ROI
// are appended after the ascending part in that order; then, if the list is
// longer than max_nodes, the k-th must-keep position (ascending) at or past
// max_nodes is swapped with position k and the list is cut to max_nodes.
// One thread; the ascending part is binary-searched.  MAX_KEEP bounds the
// list (checked on the host).
constexpr int MAX_KEEP = 256;
__global__ void keep_truncate_kernel(int32_t *roi, const int32_t *count_in, int32_t max_nodes, int32_t src,
                                     int32_t dst, const int32_t *keep, int32_t nkeep, int32_t *count_out) {
  if (threadIdx.x != 0) return;
  int32_t mk[MAX_KEEP + 2];
  int nmk = 0;
  mk[nmk++] = src;
  if (dst != src) mk[nmk++] = dst;
  for (int i = 0; i < nkeep; ++i) {
    const int32_t v = keep[i];
    bool dup = false;
    for (int j = 0; j < nmk; ++j) dup |= mk[j] == v;
    if (!dup) mk[nmk++] = v;
  }
  const int n0 = *count_in;
  int n = n0;
  int32_t pos[MAX_KEEP + 2];
  for (int j = 0; j < nmk; ++j) {
    int lo = 0, hi = n0;  // first position with roi[p] >= mk[j]
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (roi[mid] < mk[j]) lo = mid + 1;
      else hi = mid;
    }
    if (lo < n0 && roi[lo] == mk[j]) {
      pos[j] = lo;
    } else {
      roi[n] = mk[j];
      pos[j] = n++;
    }
  }
  int cnt = n;
  if (n > max_nodes) {
    // positions in ascending order (insertion sort of a short list)
    for (int a = 1; a < nmk; ++a) {
      const int32_t t = pos[a];
      int b = a - 1;
      while (b >= 0 && pos[b] > t) {
        pos[b + 1] = pos[b];
        --b;
      }
      pos[b + 1] = t;
    }
    for (int k = 0; k < nmk; ++k) {
      const int p = pos[k];
      if (p >= max_nodes) {
        const int32_t t = roi[p];
        roi[p] = roi[k];
        roi[k] = t;
      }
    }
    cnt = max_nodes;
  }
  *count_out = cnt;
}

__global__ void fill_i32_kernel(int32_t *p, int64_t n, int32_t v) {
  const int64_t s = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += s) p[i] = v;
}

__global__ void scatter_g2r_kernel(const int32_t *roi, const int32_t *count, int32_t *g2r) {
  const int n = *count;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    g2r[roi[i]] = i;
}

// global_to_roi for an inclusive box: -1 everywhere, local id inside
// (local ids ascend with global ids, so ROI rank = global order).
__global__ void box_map_kernel(int32_t *g2r, int64_t N, int32_t nx, int32_t ny, int32_t x0,
                               int32_t x1, int32_t y0, int32_t y1, int32_t z0, int32_t z1) {
  const int64_t plane = (int64_t)nx * ny;
  const int32_t W = x1 - x0 + 1, H = y1 - y0 + 1;
  const int64_t s = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < N; v += s) {
    const int32_t z = (int32_t)(v / plane);
    const int64_t r = v - (int64_t)z * plane;
    const int32_t y = (int32_t)(r / nx), x = (int32_t)(r - (int64_t)y * nx);
    int32_t id = -1;
    if (x >= x0 && x <= x1 && y >= y0 && y <= y1 && z >= z0 && z <= z1)
      id = ((z - z0) * H + (y - y0)) * W + (x - x0);
    g2r[v] = id;
  }
}

}  // namespace

using namespace orsp;

extern "C" int orsp_roi_box_map(orsp_graph *g, const int32_t *box_h, int32_t *g2r_d,
                                uintptr_t stream) {
  if (!g || !box_h || !g2r_d) { set_error("roi_box_map: NULL argument"); return ORSP_ERR_ARG; }
  if (g->nx <= 0) { set_error("roi_box_map: graph has no lattice dims"); return ORSP_ERR_ARG; }
  const int32_t *b = box_h;
  if (b[0] < 0 || b[2] < 0 || b[4] < 0 || b[1] >= g->nx || b[3] >= g->ny || b[5] >= g->nz ||
      b[1] < b[0] || b[3] < b[2] || b[5] < b[4]) {
    set_error("roi_box_map: box outside the lattice or empty");
    return ORSP_ERR_ARG;
  }
  ORSP_CUDA(cudaSetDevice(g->device));
  const int64_t N = g->N;
  box_map_kernel<<<(int)std::min<int64_t>((N + 255) / 256, 148 * 16), 256, 0, (cudaStream_t)stream>>>(
      g2r_d, N, g->nx, g->ny, b[0], b[1], b[2], b[3], b[4], b[5]);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

static int roi_bfs_impl(orsp_graph *g, int32_t src, int32_t dst, int32_t max_depth, int32_t max_nodes,
                        const int32_t *keep_d, int32_t nkeep, int32_t *roi_nodes_d, int32_t *g2r_d,
                        int32_t *roi_count_h, uintptr_t stream);

extern "C" int orsp_roi_bfs(orsp_graph *g, int32_t src, int32_t dst, int32_t max_depth,
                            int32_t max_nodes, int32_t *roi_nodes_d, int32_t *g2r_d,
                            int32_t *roi_count_h, uintptr_t stream) {
  return roi_bfs_impl(g, src, dst, max_depth, max_nodes, nullptr, 0, roi_nodes_d, g2r_d, roi_count_h, stream);
}

extern "C" int orsp_roi_bfs_keep(orsp_graph *g, int32_t src, int32_t dst, int32_t max_depth,
                                 int32_t max_nodes, const int32_t *keep_d, int32_t nkeep,
                                 int32_t *roi_nodes_d, int32_t *g2r_d, int32_t *roi_count_h,
                                 uintptr_t stream) {
  if (nkeep < 0 || nkeep > MAX_KEEP || (nkeep > 0 && !keep_d)) {
    set_error("roi_bfs_keep: nkeep must be 0.." + std::to_string(MAX_KEEP) + " with a keep list");
    return ORSP_ERR_ARG;
  }
  return roi_bfs_impl(g, src, dst, max_depth, max_nodes, keep_d, nkeep, roi_nodes_d, g2r_d, roi_count_h, stream);
}

static int roi_bfs_impl(orsp_graph *g, int32_t src, int32_t dst, int32_t max_depth, int32_t max_nodes,
                        const int32_t *keep_d, int32_t nkeep, int32_t *roi_nodes_d, int32_t *g2r_d,
                        int32_t *roi_count_h, uintptr_t stream) {
  if (!g || !roi_nodes_d || !roi_count_h) { set_error("roi_bfs: NULL argument"); return ORSP_ERR_ARG; }
  if (src < 0 || src >= g->N || dst < 0 || dst >= g->N) { set_error("roi_bfs: src/dst out of range"); return ORSP_ERR_ARG; }
  if (max_nodes <= 0) { set_error("roi_bfs: max_nodes must be > 0"); return ORSP_ERR_ARG; }
  ORSP_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t N = g->N;
  const int ntiles = (int)((N + CMP_TILE - 1) / CMP_TILE);
  // scratch: seen (N bytes, rounded to 16) | 4 queues of N | tiles | ctl
  const size_t seen_b = ((size_t)N + 15) & ~(size_t)15;
  const size_t q_b = (size_t)N * 4;
  const size_t tiles_b = ((size_t)ntiles * 4 + 15) & ~(size_t)15;
  const size_t total_b = seen_b + 4 * q_b + tiles_b + 64;
  int rc = ensure_scratch(g, total_b);
  if (rc) return rc;
  char *base = (char *)g->scratch;
  uint8_t *seen = (uint8_t *)base;
  int32_t *q[4];
  for (int i = 0; i < 4; ++i) q[i] = (int32_t *)(base + seen_b + i * q_b);
  int32_t *tiles = (int32_t *)(base + seen_b + 4 * q_b);
  int32_t *misc = (int32_t *)(base + seen_b + 4 * q_b + tiles_b);  // [0..3] BfsCtl, [4] total, [5] count
  BfsCtl *ctl = (BfsCtl *)misc;

  ORSP_CUDA(cudaMemsetAsync(seen, 0, seen_b, st));
  roi_bfs_kernel<<<1, BFS_THREADS, 0, st>>>(g->indptr, g->indices, g->N, src, dst, max_depth,
                                            max_nodes, seen, q[0], q[1], q[2], q[3], ctl);
  ORSP_CUDA(cudaGetLastError());
  count_tiles_kernel<<<ntiles, CMP_THREADS, 0, st>>>(seen, g->N, tiles);
  ORSP_CUDA(cudaGetLastError());
  scan_tiles_kernel<<<1, 1024, 0, st>>>(tiles, ntiles, misc + 4);
  ORSP_CUDA(cudaGetLastError());
  write_tiles_kernel<<<ntiles, CMP_THREADS, 0, st>>>(seen, g->N, tiles, roi_nodes_d);
  ORSP_CUDA(cudaGetLastError());
  if (nkeep > 0)
    keep_truncate_kernel<<<1, 32, 0, st>>>(roi_nodes_d, misc + 4, max_nodes, src, dst, keep_d, nkeep, misc + 5);
  else
    truncate_kernel<<<1, 32, 0, st>>>(roi_nodes_d, misc + 4, max_nodes, src, dst, misc + 5);
  ORSP_CUDA(cudaGetLastError());
  if (g2r_d) {
    fill_i32_kernel<<<std::min<int64_t>((N + 255) / 256, 4096), 256, 0, st>>>(g2r_d, N, -1);
    scatter_g2r_kernel<<<std::min<int64_t>((N + 255) / 256, 1024), 256, 0, st>>>(roi_nodes_d,
                                                                                 misc + 5, g2r_d);
    ORSP_CUDA(cudaGetLastError());
  }
  ORSP_CUDA(cudaMemcpyAsync(g->pinned, misc, 24, cudaMemcpyDeviceToHost, st));
  ORSP_CUDA(cudaStreamSynchronize(st));
  const int32_t *h = (const int32_t *)g->pinned;
  if (h[3]) { set_error("roi_bfs: queue overflow"); return ORSP_ERR_OVERFLOW; }
  *roi_count_h = h[5];
  return ORSP_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free ROI extraction.
//
// orsp_roi_bfs keeps its work buffers (visit marks, the four wave queues and
// the compaction tiles) in device memory that the library allocates with
// cudaMalloc on first use.  Some callers cannot allow that: a host
// application whose own caching allocator has reserved the GPU's memory up
// front and forbids any other cudaMalloc / cudaFree on the routing path
// (a cudaFree there also synchronises the whole device).
// orsp_roi_bfs_noalloc gives them the same extraction with its work buffers
// in one file-scope device array, so the call itself allocates nothing.  The
// array is sized for graphs of at most ORSP_ROI_BFS_NOALLOC_MAX_NODES nodes
// and every GPU that loads the library holds it (about 8.5 MB) until the
// process exits.
namespace {

constexpr size_t kNaSeenBytes = ((size_t)ORSP_ROI_BFS_NOALLOC_MAX_NODES + 15) & ~(size_t)15;
constexpr size_t kNaQueueBytes = (size_t)ORSP_ROI_BFS_NOALLOC_MAX_NODES * 4;
constexpr size_t kNaTileBytes =
    (((size_t)ORSP_ROI_BFS_NOALLOC_MAX_NODES + CMP_TILE - 1) / CMP_TILE * 4 + 15) & ~(size_t)15;
constexpr size_t kNaBytes = kNaSeenBytes + 4 * kNaQueueBytes + kNaTileBytes + 64;

// Shared by every call on a device; see orsp_roi_bfs_noalloc for the rules.
static __device__ __align__(256) unsigned char g_roi_noalloc_scratch[kNaBytes];

constexpr int kNaMaxDevices = 64;
std::mutex g_na_mutex;
void *g_na_ptr[kNaMaxDevices] = {};

// Device address of the array on `device` (which must be current).  Looked up
// once per device, by the first call on it: in host code the symbol is only a
// host-side stand-in, not a device address.  The address is cached by device
// ordinal, so the call assumes the device's primary context (the runtime
// API's default); a caller that switches driver-API contexts on one device
// would get an address from another context.
int noalloc_scratch(int device, unsigned char **out) {
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (device < 0 || device >= kNaMaxDevices) {
    set_error("roi_bfs_noalloc: device ordinal out of range");
    return ORSP_ERR_ARG;
  }
  if (!g_na_ptr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_roi_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_roi_noalloc_scratch)");
    g_na_ptr[device] = p;
  }
  *out = (unsigned char *)g_na_ptr[device];
  return ORSP_OK;
}

}  // namespace

extern "C" int orsp_roi_bfs_noalloc(orsp_graph *g, int32_t src, int32_t dst, int32_t max_depth,
                                    int32_t max_nodes, int32_t *roi_nodes_d, int32_t *g2r_d,
                                    int32_t *roi_count_h, uintptr_t stream) {
  if (!g || !roi_nodes_d || !roi_count_h) { set_error("roi_bfs_noalloc: NULL argument"); return ORSP_ERR_ARG; }
  if (g->N > ORSP_ROI_BFS_NOALLOC_MAX_NODES) {
    set_error("roi_bfs_noalloc: graph has " + std::to_string(g->N) + " nodes, more than the " +
              std::to_string(ORSP_ROI_BFS_NOALLOC_MAX_NODES) +
              " its fixed work array holds; use orsp_roi_bfs");
    return ORSP_ERR_ARG;
  }
  if (src < 0 || src >= g->N || dst < 0 || dst >= g->N) { set_error("roi_bfs_noalloc: src/dst out of range"); return ORSP_ERR_ARG; }
  if (max_nodes <= 0) { set_error("roi_bfs_noalloc: max_nodes must be > 0"); return ORSP_ERR_ARG; }
  ORSP_CUDA(cudaSetDevice(g->device));
  unsigned char *base = nullptr;
  int rc = noalloc_scratch(g->device, &base);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t N = g->N;
  const int ntiles = (int)((N + CMP_TILE - 1) / CMP_TILE);
  uint8_t *seen = base;
  int32_t *q[4];
  for (int i = 0; i < 4; ++i) q[i] = (int32_t *)(base + kNaSeenBytes + i * kNaQueueBytes);
  int32_t *tiles = (int32_t *)(base + kNaSeenBytes + 4 * kNaQueueBytes);
  int32_t *misc = (int32_t *)(base + kNaSeenBytes + 4 * kNaQueueBytes + kNaTileBytes);
  BfsCtl *ctl = (BfsCtl *)misc;

  // The array keeps the previous call's contents: the visit marks must start
  // at zero; the queues, tile counts and counters are written before read.
  ORSP_CUDA(cudaMemsetAsync(seen, 0, ((size_t)N + 15) & ~(size_t)15, st));
  roi_bfs_kernel<<<1, BFS_THREADS, 0, st>>>(g->indptr, g->indices, g->N, src, dst, max_depth,
                                            max_nodes, seen, q[0], q[1], q[2], q[3], ctl);
  ORSP_CUDA(cudaGetLastError());
  count_tiles_kernel<<<ntiles, CMP_THREADS, 0, st>>>(seen, g->N, tiles);
  ORSP_CUDA(cudaGetLastError());
  scan_tiles_kernel<<<1, 1024, 0, st>>>(tiles, ntiles, misc + 4);
  ORSP_CUDA(cudaGetLastError());
  write_tiles_kernel<<<ntiles, CMP_THREADS, 0, st>>>(seen, g->N, tiles, roi_nodes_d);
  ORSP_CUDA(cudaGetLastError());
  truncate_kernel<<<1, 32, 0, st>>>(roi_nodes_d, misc + 4, max_nodes, src, dst, misc + 5);
  ORSP_CUDA(cudaGetLastError());
  if (g2r_d) {
    fill_i32_kernel<<<std::min<int64_t>((N + 255) / 256, 4096), 256, 0, st>>>(g2r_d, N, -1);
    scatter_g2r_kernel<<<std::min<int64_t>((N + 255) / 256, 1024), 256, 0, st>>>(roi_nodes_d,
                                                                                 misc + 5, g2r_d);
    ORSP_CUDA(cudaGetLastError());
  }
  // g->pinned was allocated when the graph was created, not here; it is one
  // buffer per graph, so overlapping calls on one graph race on it too.
  ORSP_CUDA(cudaMemcpyAsync(g->pinned, misc, 24, cudaMemcpyDeviceToHost, st));
  ORSP_CUDA(cudaStreamSynchronize(st));
  const int32_t *h = (const int32_t *)g->pinned;
  if (h[3]) { set_error("roi_bfs_noalloc: queue overflow"); return ORSP_ERR_OVERFLOW; }
  *roi_count_h = h[5];
  return ORSP_OK;
}
