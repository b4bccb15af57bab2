/*
 * orsp.h — C ABI of the B200-native PathFinder search library (liborsp.so).
 *
 * The library replaces the hot path of OrthoRoute's Manhattan PathFinder:
 * per-net single-source shortest path on the lattice CSR, edge-cost update,
 * ROI extraction, predecessor backtrace, path -> edge mapping, overuse count
 * and history update.  Each entry point names the reference function it
 * replaces (paths are relative to the OrthoRoute project root;
 * UPF = orthoroute/algorithms/manhattan/unified_pathfinder.py,
 * CD  = orthoroute/algorithms/manhattan/pathfinder/cuda_dijkstra.py).
 *
 * Conventions
 *  - Plain C types only.  Pointers with the suffix `_d` are CUDA device
 *    pointers on the device the graph was created on; `_h` are host pointers.
 *  - `stream` is a cudaStream_t passed as uintptr_t (0 = legacy default stream).
 *  - Every call returns an int status: ORSP_OK (0), ORSP_NO_PATH (1, not an
 *    error: the reference returns None), or a negative error code.
 *    orsp_last_error() returns a thread-local message for the last failure.
 *  - Distances are IEEE fp32 computed with round-to-nearest additions
 *    d[v] = min_u fl32(d[u] + w(u,v)); the fixpoint is unique, so results are
 *    bit-identical to a sequential fp32 Dijkstra.  Costs must be >= 0
 *    (+inf = blocked edge; NaN edges are never relaxed).
 *  - Path tie-break: among predecessors u with fl32(d[u] + w(u,v)) == d[v]
 *    and (d[u], rank(u)) < (d[v], rank(v)), the parent is the one with the
 *    smallest (d[u], rank(u)), where rank is the ROI index (the position in
 *    roi_nodes, i.e. global_to_roi[u]) or the global node id for full-graph
 *    searches.  This is the order in which the reference heap Dijkstra
 *    (UPF:1846-1878) settles nodes and keeps the first strictly better parent.
 */
#ifndef ORSP_H
#define ORSP_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define ORSP_API __attribute__((visibility("default")))
#else
#define ORSP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define ORSP_OK 0
#define ORSP_NO_PATH 1          /* search finished, destination unreachable  */
#define ORSP_ERR_ARG (-1)       /* invalid argument (checked on the host)    */
#define ORSP_ERR_CUDA (-2)      /* a CUDA runtime call failed                */
#define ORSP_ERR_TIMEOUT (-3)   /* device round / wait limit reached         */
#define ORSP_ERR_OVERFLOW (-4)  /* a work queue or path buffer was too small */
#define ORSP_ERR_NOMEM (-5)     /* device allocation failed                  */
#define ORSP_ERR_INTERNAL (-6)  /* invariant broken (e.g. no predecessor)    */

/* Version of this ABI; bumped on any signature change.  This function, the
 * status names and the last-error message have no counterpart in the
 * reference, which signals failures with Python exceptions or None. */
#define ORSP_ABI_VERSION 1
ORSP_API int orsp_abi_version(void);
ORSP_API const char *orsp_status_string(int status);
ORSP_API const char *orsp_last_error(void);

/* Profiling hook: when enabled, the search kernel of orsp_sssp (the
 * persistent grid launch alone, without its init kernels) is bracketed by CUDA
 * events on the caller's stream; orsp_profile_last returns the duration of
 * the most recent one in milliseconds.  No counterpart in the reference. */
ORSP_API int orsp_profile_enable(int on);
ORSP_API int orsp_profile_last(float *kernel_ms);
/* Work counters of the last lattice search: {grid rounds, tile visits,
 * sweep cycles, 0, ns loading tiles, ns sweeping, ns writing back,
 * ns scheduling} (times summed over tile visits). */
ORSP_API int orsp_profile_counters(int64_t *out8);

/* ---- graph ------------------------------------------------------------- */
typedef struct orsp_graph orsp_graph;

/* Uploads the CSR (host arrays) to `device` and builds the device-side
 * transposed CSR used by the backtrace.  Replaces the graph ownership of
 * CUDADijkstra.__init__ (CD:110-121) and CSRGraph (UPF:647-792).
 * Nx, Ny, Nz describe the lattice (node = z*Nx*Ny + y*Nx + x, as
 * KiCadGeometry.node_index, pathfinder/kicad_geometry.py:63-66); pass
 * 0,0,0 for a graph that is not a lattice (bbox searches are then refused). */
ORSP_API int orsp_graph_create(int32_t num_nodes, int64_t num_edges,
                      const int32_t *indptr_h, const int32_t *indices_h,
                      int32_t nx, int32_t ny, int32_t nz, int device,
                      orsp_graph **out);
ORSP_API int orsp_graph_destroy(orsp_graph *g);
/* Device pointers of the uploaded CSR (indptr[N+1], indices[E]) and its
 * largest out-degree, for callers that share them; no counterpart in the
 * reference, which keeps its CSR on the host (CD:119-121). */
ORSP_API int orsp_graph_csr(orsp_graph *g, const int32_t **indptr_d,
                   const int32_t **indices_d);
ORSP_API int orsp_graph_max_degree(orsp_graph *g, int32_t *out);
/* 1 when the graph was recognised as an H/V routing lattice (every edge a
 * unit step along its layer's axis or a via between adjacent layers, no
 * parallel edges): full-graph, box and ROI searches then use the tile sweeps
 * and orsp_route_nets is available.  2 for the same planar structure with
 * column vias, as the reference's Lattice3D builds them (vias between any
 * two layers of a column, up to two parallel edges each,
 * unified_pathfinder.py:1136-1172, 1264-1276): single, ROI, multi-target and
 * many-source and batched box searches and orsp_route_nets use the tile
 * sweeps with a per-column via pass (tile width 16; batched plans at width
 * 32 take the one-CTA kernel).  0 otherwise.  (No reference counterpart: the reference has one
 * search path for every graph.) */
ORSP_API int orsp_graph_is_lattice(orsp_graph *g, int32_t *out);
/* Deepest box (layers) that one shared-memory tile of the lattice search holds
 * at tile width tile_w (16 or 32; 0: the library's width).  Single and
 * batched box searches deeper than this take the generic search; the device
 * routing loop (orsp_route_nets) rejects them.  (No reference counterpart.) */
ORSP_API int orsp_lattice_max_layers(int32_t tile_w, int32_t *out);

/* Declares, for the next search on this graph only, that the contents of
 * cost_d are identified by `generation` (non-zero; the caller changes it
 * whenever it writes the array).  A whole-lattice tile search first gathers
 * the costs into per-node in-edge weights (16 B per node); it skips that
 * gather when the declaration names the same array and generation as the
 * last whole gather (e.g. many sources searched on one fixed cost array, as
 * the reference routes every net of an iteration on one total_cost,
 * UPF:3724-3732, 4463).  Without a declaration every search gathers.  No
 * counterpart in the reference. */
ORSP_API int orsp_graph_cost_generation(orsp_graph *g, const float *cost_d, uint64_t generation);

/* ---- single search ----------------------------------------------------- */
/* Single-source (or multi-seed) shortest path over the whole graph or over
 * the ROI given by roi_map_d (global_to_roi, int32[N], -1 = outside).  On a
 * recognised H/V lattice it runs the tile-sweep search: over the whole
 * lattice, or, with a ROI, over the ROI's bounding box (reduced on the
 * device) with every edge into or out of the ROI at +inf, ties ranked by
 * global_to_roi.  Other graphs run one persistent cooperative launch of
 * near-far delta-stepping with a bounded grid barrier.  Replaces SimpleDijkstra.find_path_roi (UPF:1801-1887) and
 * CUDADijkstra.find_path_roi_gpu (CD:4909-4996).
 *   seeds_d[nseeds]       start nodes (global ids); seed_cost_d may be NULL
 *                          (all seeds start at 0.0) or give fp32 start costs.
 *   dst                    target node, or -1 for a full search (no path).
 *   delta                  near-far bucket width (> 0), or 0 to let the
 *                          library choose it on the device (twice the mean
 *                          of a strided sample of the finite costs).  It
 *                          changes the work, never the distances or path.
 *   dist_out_d             optional fp32[N]; receives distances (nodes not
 *                          settled before an early exit hold upper bounds).
 *   path_out_d/path_cap    receives the node path seed..dst (global ids).
 *   path_len_h             receives the path length (0 when no path).
 *   rounds_h               optional: device rounds executed (for tuning).  */
ORSP_API int orsp_sssp(orsp_graph *g, const float *cost_d, int32_t nseeds,
              const int32_t *seeds_d, const float *seed_cost_d, int32_t dst,
              const int32_t *roi_map_d, float delta, float *dist_out_d,
              int32_t *path_out_d, int32_t path_cap, int32_t *path_len_h,
              int32_t *rounds_h, uintptr_t stream);

/* nsrc whole-graph single-source searches (no target): row i of
 * dist_out_d (fp32[nsrc][N], device) receives the distances from src_h[i]
 * (host), bit for bit those of orsp_sssp with that source.  On a recognised
 * lattice up to per_launch sources (0: all) share one persistent launch, each
 * a whole-lattice box with its own distance row, so the tile queue
 * interleaves their wavefronts and the launch is bound by tile visits rather
 * than by one wave's hop latency.  Other graphs run orsp_sssp per source.
 * The batched counterpart of SimpleDijkstra.find_path_roi over the full
 * graph (UPF:1801-1887) for many sources, as CUDADijkstra.find_paths_on_rois
 * (CD:2014-2086) batches ROI searches.  A cost-generation declaration covers
 * the whole call; orsp_profile_last / orsp_profile_counters report the sum
 * over the call's launches. */
ORSP_API int orsp_sssp_sources(orsp_graph *g, const float *cost_d, int32_t nsrc, const int32_t *src_h,
                               float *dist_out_d, int32_t per_launch, uintptr_t stream);

/* One search from src to dst over the ROI given as its node list (the
 * roi_nodes array SimpleDijkstra.find_path_roi, UPF:1801-1887, and
 * CUDADijkstra.find_path_roi_gpu, CD:4909-4996, take, int32[n_roi], device):
 * the ROI index of roi_nodes_d[i] is i (a repeated node keeps its last
 * index, as the reference's global_to_roi[roi_nodes] = arange(R) does), and
 * ties between equal distances go to the smaller ROI index.  The call builds
 * its global_to_roi on the device from the list, in a map the graph keeps at
 * -1 between calls, so a caller passes O(R) data per search instead of an
 * int32[N] map.  Path (global ids, src..dst) as orsp_sssp; ORSP_NO_PATH when
 * src or dst is outside the ROI or unreachable. */
ORSP_API int orsp_sssp_roi_nodes(orsp_graph *g, const float *cost_d, int32_t src, int32_t dst,
                        const int32_t *roi_nodes_d, int64_t n_roi, int32_t *path_out_d,
                        int32_t path_cap, int32_t *path_len_h, uintptr_t stream);

/* The same search inside an axis-aligned box ROI (inclusive bounds
 * x0,x1,y0,y1,z0,z1 in the host array box_h[6]): identical, bit for bit, to
 * orsp_sssp with roi_map_d = the orsp_roi_box_map of the box (the bounding
 * box + margin ROI of the benchmark router, searched by
 * SimpleDijkstra.find_path_roi, UPF:1801-1887; the box-local index order is
 * the node-id order).  On a recognised H/V lattice only the box's tiles are
 * gathered and swept; dist_out_d (optional) is +inf outside the box. */
ORSP_API int orsp_sssp_box(orsp_graph *g, const float *cost_d, int32_t nseeds,
                  const int32_t *seeds_d, const float *seed_cost_d, int32_t dst,
                  const int32_t *box_h, float delta, float *dist_out_d,
                  int32_t *path_out_d, int32_t path_cap, int32_t *path_len_h,
                  int32_t *rounds_h, uintptr_t stream);

/* Multi-seed / multi-target search with portal costs, as
 * SimpleDijkstra.find_path_multisource_multisink (UPF:1889-1989): seeds start
 * at seed_cost (NULL = 0.0), the search runs to completion inside the ROI,
 * targets are settled but never expanded, and the target with the smallest
 * (double)d[t] + target_cost[t] wins (equal totals: the one settled first,
 * i.e. smallest (d[t], rank)).  Targets must be distinct.  The path runs from
 * a seed to the winning target (best_target_h, optional).  Also serves
 * CUDADijkstra.find_path_fullgraph_gpu_seeds (CD:5467-5751) with zero costs;
 * unlike that wavefront (which stops at the first target it reaches) the
 * answer is the exact shortest one.  On a recognised H/V lattice it runs the
 * tile-sweep search over the ROI's bounding box with the targets' out-edges
 * at +inf. */
ORSP_API int orsp_sssp_multi(orsp_graph *g, const float *cost_d, int32_t nseeds,
                    const int32_t *seeds_d, const float *seed_cost_d,
                    int32_t ntargets, const int32_t *targets_d,
                    const double *target_cost_d, const int32_t *roi_map_d,
                    float delta, int32_t *path_out_d, int32_t path_cap,
                    int32_t *path_len_h, int32_t *best_target_h, uintptr_t stream);

/* global_to_roi from an allowed-node bitmap (uint32 words, bit v%32 of word
 * v/32 set = allowed), rank = node id: the allowed_bitmap of
 * find_path_fullgraph_gpu_seeds (CD:5467) as a roi_map. */
ORSP_API int orsp_roi_from_bitmap(orsp_graph *g, const uint32_t *bitmap_d, int32_t *g2r_d,
                         uintptr_t stream);

/* ---- batched searches (one launch, one CTA per search) ----------------- */
/* K independent searches on shared fp32 costs, each inside an axis-aligned
 * box ROI (inclusive bounds x0,x1,y0,y1,z0,z1 per search in bbox_d[6*K]).
 * One persistent launch; each CTA runs a block-local near-far search per
 * work item, backtraces it and maps the path to CSR edges.
 * Replaces CUDADijkstra.find_paths_on_rois (CD:2014-2086) for box ROIs and
 * the per-net loop body of _route_all (UPF:4475-4800) under fixed costs.
 *   order_d               optional int32[K] processing order, a permutation
 *                          of 0..K-1 (e.g. largest box first); NULL = 0..K-1.
 *   delta                  bucket width as for orsp_sssp (0: device choice).
 *   path_nodes_d/edges_d  int32[K*path_cap] outputs (edges_d may be NULL).
 *   path_len_d            int32[K]: path length, 0 = no path, <0 = error. */
ORSP_API int orsp_sssp_batch_bbox(orsp_graph *g, const float *cost_d, int32_t K,
                         const int32_t *src_d, const int32_t *dst_d,
                         const int32_t *bbox_d, const int32_t *order_d,
                         float delta, int32_t *path_nodes_d,
                         int32_t *path_edges_d, int32_t path_cap,
                         int32_t *path_len_d, uintptr_t stream);

/* The same batched search with node-range ROIs: search k stays inside nodes
 * [ranges[2k], ranges[2k+1]) and ranks nodes by id - ranges[2k].  Built for
 * graphs made of concatenated ROI-local CSRs - the 13-tuple batch of
 * CUDADijkstra.find_paths_on_rois (CD:2014-2086, tuple format CD:55-91),
 * where every ROI is its own block of node ids and the local order is the
 * ROI index order.  src/dst and the returned paths are global ids of the
 * concatenated graph. */
ORSP_API int orsp_sssp_batch_ranges(orsp_graph *g, const float *cost_d, int32_t K,
                           const int32_t *src_d, const int32_t *dst_d,
                           const int32_t *ranges_d, const int32_t *order_d,
                           float delta, int32_t *path_nodes_d,
                           int32_t *path_edges_d, int32_t path_cap,
                           int32_t *path_len_d, uintptr_t stream);

/* Tuning plan for orsp_sssp_batch_bbox (no counterpart in the reference,
 * whose batch search has one fixed configuration).  Boxes are put into
 * buckets by node count: bucket i takes the boxes with
 * max_nodes[i-1] < V <= max_nodes[i] (the last bucket takes every larger box
 * too).  Per bucket:
 *   impl 0   one CTA per search (block-local near-far) with bucket width
 *            delta[i] (0: the call's); all impl-0 searches of a call share
 *            one launch of the largest ctas_per_sm of their buckets CTAs per
 *            SM (0: default 2);
 *   impl 1   tile sweeps over many boxes per launch, each box with its own
 *            distance slice, tile width tile_w[i] (16 or 32); used on graphs
 *            recognised as H/V lattices, impl 0 otherwise.
 * nb = 0 restores the default (impl 0 for every box).  Every plan gives the
 * same paths, bit for bit; the plan only changes the time.  No counterpart in
 * the reference. */
ORSP_API int orsp_batch_set_plan(orsp_graph *g, int32_t nb, const int64_t *max_nodes, const int32_t *impl,
                        const float *delta, const int32_t *tile_w, const int32_t *ctas_per_sm);

/* ---- routing loop ------------------------------------------------------ */
/* Routes nets with per-net live costs, as the per-net body of _route_all
 * (UPF:4475-4800) with the live-usage cost refresh of orsp_update_costs_live.
 * For each net k = order_h[i] (i < K, each net at most once): rip up its
 * previous path (row k of net_edges_d, net_lens_d[k] nodes; usage -1 and live
 * costs of those edges), search src_h[k] -> dst_h[k] inside its box
 * (box_h[6k..6k+5], as orsp_sssp_box) on the costs as they are now, write the
 * node path, its edges (first CSR edge per pair, UPF:5463) and its length
 * (0 = no path; also when src lies outside the box) into row k, then commit
 * it (usage +1, live costs).
 *   group_ptr_h[G+1]   optional: the order is cut into groups
 *                      [group_ptr[q], group_ptr[q+1]) of at most 1024 nets with
 *                      pairwise disjoint boxes (checked); a group's nets are
 *                      ripped up, searched in one tile-sweep launch and
 *                      committed together.  NULL: one net per group.
 * With every net's previous path inside its box (boxes that never shrink),
 * nets of one group read and write disjoint edges, so the result is bit for
 * bit the one-net-at-a-time result in the same order (the host loop over
 * orsp_commit_edges / orsp_update_costs_live / orsp_sssp_box /
 * orsp_path_to_edges).  Everything is enqueued without host synchronisation
 * (one sync at the end).  Rows are path_cap wide; src_h, dst_h and box_h are
 * host arrays over all M nets.  Needs a graph recognised as an H/V lattice.
 * usage_d/present_d/cost_d are updated in place. */
ORSP_API int orsp_route_nets(orsp_graph *g, int32_t M, const int32_t *src_h, const int32_t *dst_h,
                    const int32_t *box_h, int32_t K, const int32_t *order_h, int32_t G,
                    const int32_t *group_ptr_h, int32_t *net_nodes_d, int32_t *net_edges_d,
                    int32_t path_cap, int32_t *net_lens_d, float *cost_d, const float *base_d,
                    int32_t *usage_d, float *present_d, const float *cap_d, const float *hist_d,
                    float pres_fac, float hist_w, float via_mult, float base_w, int32_t jitter,
                    uintptr_t stream);
/* The same loop with snapshot groups: the boxes of a group may overlap.  A
 * group's nets are ripped up together, searched in one tile-sweep launch on
 * the costs after those rip-ups (each box on distances of its own), and
 * committed together: within a group no net sees another, as the
 * reference's batched GPU mode routes a batch of ROIs on one cost array
 * (CUDADijkstra.find_paths_on_rois, CD:2014).  Usage is applied for the
 * whole group before any live cost is recomputed, so every cost is computed
 * from the final usage and the result does not depend on thread order.  Then
 * up to repair_rounds rounds: the nets whose new path uses an edge that a
 * net earlier in the group also uses (in the same round) are ripped up,
 * searched again on the live costs (which hold every path of the group) and
 * committed again; a round that flags no net ends the group's repair early
 * (its launches find no work).  Of two nets of a round that share an edge,
 * the later one in the order is routed again and then sees the earlier one's
 * path, as it would one net at a time.
 * *searches_out (optional) receives the searches made: K plus the repair
 * searches.  A group of one net is the plain loop.  Other arguments as
 * orsp_route_nets; repair_rounds is 0..64.  No reference counterpart for the
 * repair rounds. */
ORSP_API int orsp_route_nets_snapshot(orsp_graph *g, int32_t M, const int32_t *src_h, const int32_t *dst_h,
                    const int32_t *box_h, int32_t K, const int32_t *order_h, int32_t G,
                    const int32_t *group_ptr_h, int32_t repair_rounds, int32_t *net_nodes_d,
                    int32_t *net_edges_d, int32_t path_cap, int32_t *net_lens_d, float *cost_d,
                    const float *base_d, int32_t *usage_d, float *present_d, const float *cap_d,
                    const float *hist_d, float pres_fac, float hist_w, float via_mult, float base_w,
                    int32_t jitter, int64_t *searches_out, uintptr_t stream);

/* ---- negotiation bookkeeping ------------------------------------------- */
/* The per-iteration loops the reference runs in Python over all committed
 * nets.  Nets come in the router's dict order as concatenated node paths or
 * edge lists with int64 offsets off_d[M+1]; net_ids_d[m] is net m's integer
 * id (PathFinderRouter._get_net_id). */

/* Node ownership, _rebuild_node_owner (UPF:2762-2837).  First the committed
 * via barrels: every node of every via step (same x, y; different z) of net
 * m, over the whole z span, gets net m's id; where several nets cover a node
 * the last one in order wins, as the reference's sequential overwrite.  Then
 * the escape-via keepouts keep_nodes_d[K] / keep_ids_d[K] (the
 * _via_keepouts_map entries with z > 0, in dict order): an entry claims its
 * node if no barrel owns it, the first entry per node winning.  owner_d
 * int32[N], -1 = free. */
ORSP_API int orsp_node_owner(orsp_graph *g, int32_t M, const int32_t *paths_d, const int64_t *off_d,
                    const int32_t *net_ids_d, int32_t K, const int32_t *keep_nodes_d,
                    const int32_t *keep_ids_d, int32_t *owner_d, uintptr_t stream);

/* Via barrel conflicts, _detect_barrel_conflicts (UPF:5478-5569): an edge of
 * net m whose source or target node is owned by another net.  count_h
 * receives the number of conflicting (net, edge) entries, duplicates
 * included, as the reference's count; mask_d (uint8[E], optional) marks the
 * conflicting edges. */
ORSP_API int orsp_barrel_conflicts(orsp_graph *g, int32_t M, const int32_t *edges_d, const int64_t *off_d,
                          const int32_t *net_ids_d, const int32_t *owner_d, uint8_t *mask_d,
                          int64_t *count_h, uintptr_t stream);

/* The Phase-1 barrel penalty of _pathfinder_negotiation (UPF:3852-3871):
 * present[e] += penalty once for every marked edge (numpy fancy-index add). */
ORSP_API int orsp_barrel_penalty(int64_t E, const uint8_t *mask_d, float *present_d, float penalty,
                        uintptr_t stream);

/* Per-net scores of _order_nets_by_difficulty (UPF:4401-4439) and
 * _build_hotset (UPF:5009-5140), with over = max(0, present - cap) and
 * hot(e) = over + 0.1 * history > 0.5 in float32:
 *   congestion_d[m] = sum over net m's edges of over / max(1, count)  (float64)
 *   impact_d[m]     = sum over net m's hot edges of over               (float64)
 *   offender_d[m]   = 1 if net m has a hot edge
 * Sums run in list order in float64, as Python's sum of float(over[e]).
 * hot_count_h (optional) receives the number of hot edges in the graph.
 * Each output pointer may be NULL. */
ORSP_API int orsp_net_scores(orsp_graph *g, int32_t M, const int32_t *edges_d, const int64_t *off_d,
                    const float *present_d, const float *cap_d, const float *hist_d, double *congestion_d,
                    double *impact_d, uint8_t *offender_d, int64_t *hot_count_h, uintptr_t stream);

/* Geometry emission, PathFinderRouter._generate_geometry_from_paths
 * (UPF:5749-5834): net m's node path paths_d[off_d[m] .. off_d[m+1]) becomes
 * straight track runs and vias with the reference's rules (outer-layer
 * planar steps dropped, non-unit or off-axis planar steps skipped, runs
 * flushed at vias and turns).  Net m writes rows starting at off_d[m] of
 * tracks_d (int32 [.][3]: run start node, run end node, layer) and vias_d
 * (int32 [.][3]: node, from layer, to layer), and its counts to
 * ntracks_d[m] / nvias_d[m].  layer_axis_h[z] (host, nz entries): 1 for 'h'
 * layers (x moves only), anything else for layers checked as 'v'. */
ORSP_API int orsp_emit_geometry(orsp_graph *g, int32_t M, const int32_t *paths_d, const int64_t *off_d,
                       const int8_t *layer_axis_h, int32_t *tracks_d, int32_t *vias_d, int32_t *ntracks_d,
                       int32_t *nvias_d, uintptr_t stream);

/* ---- ROI extraction ---------------------------------------------------- */
/* Bidirectional level-synchronous BFS ROI, as ROIExtractor.extract_roi_bfs
 * (UPF:1636-1734): waves from src (mark 1) and dst (mark 2) alternate, a node
 * reached by the other wave is marked 3 and ends the expansion; depth is
 * limited to max_depth and the expansion stops early once more than
 * 1.5*max_nodes nodes are marked.  The ROI is the marked nodes in ascending
 * order, truncated to max_nodes with src/dst moved to the front exactly as
 * the reference does.  roi_nodes_d needs room for N entries; g2r_d (int32[N],
 * may be NULL) receives global_to_roi. */
ORSP_API int orsp_roi_bfs(orsp_graph *g, int32_t src, int32_t dst, int32_t max_depth,
                 int32_t max_nodes, int32_t *roi_nodes_d, int32_t *g2r_d,
                 int32_t *roi_count_h, uintptr_t stream);

/* orsp_roi_bfs with extra must-keep nodes, as extract_roi_bfs with
 * portal_seeds (UPF:1700-1731): the must-keep list is src, dst and then the
 * keep_d[0..nkeep) nodes not already listed (device array, nkeep <= 256);
 * those missing from the BFS are appended after the ascending part in that
 * order, and the truncation to max_nodes moves every must-keep node that
 * lies at or past max_nodes to the front, as the reference swaps them. */
ORSP_API int orsp_roi_bfs_keep(orsp_graph *g, int32_t src, int32_t dst, int32_t max_depth,
                      int32_t max_nodes, const int32_t *keep_d, int32_t nkeep,
                      int32_t *roi_nodes_d, int32_t *g2r_d, int32_t *roi_count_h,
                      uintptr_t stream);

/* Allocation-free variant of orsp_roi_bfs (no counterpart in the reference).
 * For callers that cannot allocate device memory while routing: a host
 * application whose own caching allocator reserves the GPU's memory up front
 * and allows no other cudaMalloc / cudaFree on the routing path.  This call
 * allocates nothing: its work buffers live in one fixed device array inside
 * liborsp.so (about 8.5 MB, held on every GPU that loads the library until
 * exit).  Same arguments, semantics and results as orsp_roi_bfs, for graphs
 * of at most ORSP_ROI_BFS_NOALLOC_MAX_NODES nodes; larger graphs get
 * ORSP_ERR_ARG.  The first call on a device looks up the array's device
 * address (once per device, in the device's primary context); make that
 * first call before any stream capture.  All calls on a device share the
 * array, and all calls on one graph share its small pinned result buffer, so
 * calls that overlap on the GPU (other streams, other threads) race and must
 * be serialised by the caller. */
#define ORSP_ROI_BFS_NOALLOC_MAX_NODES 524288
ORSP_API int orsp_roi_bfs_noalloc(orsp_graph *g, int32_t src, int32_t dst, int32_t max_depth,
                         int32_t max_nodes, int32_t *roi_nodes_d, int32_t *g2r_d,
                         int32_t *roi_count_h, uintptr_t stream);

/* global_to_roi (int32[N]) of an inclusive box [x0,x1,y0,y1,z0,z1] (host
 * array box_h[6]): -1 outside, row-major local id inside.  The box ROI of the
 * benchmark router (bounding box of the pins plus a margin), in the
 * global_to_roi format that SimpleDijkstra.find_path_roi (UPF:1801) takes. */
ORSP_API int orsp_roi_box_map(orsp_graph *g, const int32_t *box_h, int32_t *g2r_d,
                     uintptr_t stream);

/* ---- path -> edges ----------------------------------------------------- */
/* For consecutive (u, v) of a node path, the first CSR edge u->v, as
 * PathFinderRouter._path_to_edges (UPF:5463-5476).  Pairs without an edge are
 * skipped like the reference does; edge_count_h receives the count. */
ORSP_API int orsp_path_to_edges(orsp_graph *g, const int32_t *path_d, int32_t len,
                       int32_t *edges_out_d, int32_t *edge_count_h,
                       uintptr_t stream);

/* ---- edge accounting (EdgeAccountant, UPF:799-1068) -------------------- */
/* total = ((base*via_mult)*base_w)*bias + (pres_fac*inv_bias)*over
 *         + hist_w*history [+ fmodf((float)e, 9973)*1e-6]
 * with over = max(0, present_ema - cap), bias = layer_bias[edge_layer[e]] on
 * planar edges (1 on vias) and inv_bias = 1/max(bias, 0.5); every operation
 * rounds to fp32 in the numpy order of EdgeAccountant.update_costs
 * (UPF:973-1043).  layer_bias_d/edge_layer_d/edge_kind_d may all be NULL
 * (no layer bias, as when the reference passes None). */
ORSP_API int orsp_update_costs(int64_t E, const float *base_d, const float *present_ema_d,
                      const float *cap_d, const float *history_d,
                      const uint8_t *edge_layer_d, const uint8_t *edge_kind_d,
                      const float *layer_bias_d, float pres_fac, float hist_w,
                      float via_mult, float base_w, int add_jitter,
                      float *total_out_d, uintptr_t stream);

/* Live-usage costs for negotiation with a cost refresh after every net
 * (classic PathFinder; the refresh the reference's
 * EdgeAccountant.update_present_cost_only, UPF:1045-1068, is meant for):
 *   total = ((base*via_mult)*base_w) + pres_fac*max(0, (usage+1) - cap)
 *           + hist_w*history [+ fmodf((float)e, 9973)*1e-6]
 * in the float32 order of update_costs, with present_ema replaced by the
 * prospective usage.  edges_d == NULL refreshes all E edges; otherwise the
 * n_edges listed ids (negative ids skipped). */
ORSP_API int orsp_update_costs_live(int64_t E, const int32_t *edges_d, int64_t n_edges,
                           const float *base_d, const int32_t *usage_d,
                           const float *cap_d, const float *history_d, float pres_fac,
                           float hist_w, float via_mult, float base_w, int add_jitter,
                           float *total_out_d, uintptr_t stream);
/* The same refresh (update_present_cost_only, UPF:1045-1068) over the path
 * edges of a batch (rows of orsp_sssp_batch_bbox). */
ORSP_API int orsp_update_costs_live_paths(int32_t K, const int32_t *path_edges_d,
                                 const int32_t *path_len_d, int32_t path_cap,
                                 const float *base_d, const int32_t *usage_d,
                                 const float *cap_d, const float *history_d,
                                 float pres_fac, float hist_w, float via_mult,
                                 float base_w, int add_jitter, float *total_out_d,
                                 uintptr_t stream);

/* ---- via pooling (column / segment capacity of via barrels) ------------ */
/* Arrays use the reference's C order [Nx][Ny] and [Nx][Ny][segZ] with
 * segZ = Nz - 2 (segment z -> z+1 at index z-1); usage and capacities are
 * int32 (int16 / int8 in the reference).  Via edges are the CSR edges whose
 * endpoints lie on different layers; their z range is clamped to 1..Nz-2
 * (_build_via_edge_metadata, UPF:5389-5461). */

/* Adds the via usage of the batch paths (path_len[k] nodes in row k) to
 * col_use / seg_use (either may be NULL), as _accumulate_via_usage_for_path
 * (UPF:2678-2724) does for every committed path in
 * _rebuild_via_usage_from_committed (UPF:2726-2762).  The caller zeroes the
 * arrays first. */
ORSP_API int orsp_via_usage(orsp_graph *g, int32_t K, const int32_t *path_nodes_d,
                   const int32_t *path_len_d, int32_t path_cap, int32_t *col_use_d,
                   int32_t *seg_use_d, uintptr_t stream);
/* pres = alpha*max(0, use-cap) + beta*pres for columns and segments, and the
 * float32 running sum of seg_pres along z into seg_prefix (UPF:3622-3633;
 * alpha 0.6, beta 0.4 by default).  A NULL pres array skips that part. */
ORSP_API int orsp_via_present(int64_t ncol, int32_t segz, const int32_t *col_use_d,
                     const int32_t *col_cap_d, float *col_pres_d,
                     const int32_t *seg_use_d, const int32_t *seg_cap_d,
                     float *seg_pres_d, float *seg_prefix_d, float alpha, float beta,
                     uintptr_t stream);
/* total[e] += pres_fac*penalty(e) on via edges with penalty > 0, penalty =
 * (col_weight*col_pres[x][y] + seg_weight*(prefix[z_hi-2] - prefix[z_lo-2]))
 * times the leave-hot-layer factor (1 - k*bias[z_lo])*(1 + 0.5*k*bias[z_hi])
 * when layer_bias_d is given; bias_f64 selects the float32 or float64
 * arithmetic the reference uses for that factor (its layer_bias array starts
 * as float32 and becomes float64 after the first bias update).  As
 * _apply_via_pooling_penalties (UPF:3243-3387). */
ORSP_API int orsp_via_penalties(orsp_graph *g, const float *col_pres_d,
                       const float *seg_prefix_d, const double *layer_bias_d,
                       int bias_f64, double hot_layer_discount, float col_weight,
                       float seg_weight, float pres_fac, float *total_cost_d,
                       uintptr_t stream);
/* total[e] = +inf on via edges whose column is at capacity or any of whose
 * spanned segments is at capacity (_block_via_edges_with_collisions,
 * UPF:3448-3546). */
ORSP_API int orsp_via_hard_block(orsp_graph *g, const int32_t *col_use_d,
                        const int32_t *col_cap_d, const int32_t *seg_use_d,
                        const int32_t *seg_cap_d, float *total_cost_d,
                        uintptr_t stream);

/* ema = beta*present + (1-beta)*ema  (EdgeAccountant.update_present_ema,
 * UPF:963-971); one_minus_beta is passed rounded as the caller computes it. */
ORSP_API int orsp_update_present_ema(int64_t E, const float *present_d, float *ema_d,
                            float beta, float one_minus_beta, uintptr_t stream);

/* history = history*decay + min(gain*max(0, present - cap), cap_mult*base)
 * (EdgeAccountant.update_history, UPF:898-961; base_d NULL = no clamp). */
ORSP_API int orsp_update_history(int64_t E, float *history_d, const float *present_d,
                        const float *cap_d, const float *base_d, float gain,
                        float cap_mult, float decay, uintptr_t stream);

/* (sum of max(0, present - cap), count of edges with present > cap), as
 * EdgeAccountant.compute_overuse (UPF:838-876) without the via terms.  The
 * sum is accumulated in fp64 and truncated like int(); out2_d is
 * int64[2] on the device; out2_h (optional) receives a synchronous copy. */
ORSP_API int orsp_overuse(int64_t E, const float *present_d, const float *cap_d,
                 int64_t *out2_d, int64_t *out2_h, uintptr_t stream);

/* present[e] = (float)usage[e] (refresh_from_canonical, UPF:814-819). */
ORSP_API int orsp_present_from_usage(int64_t E, const int32_t *usage_d,
                            float *present_d, uintptr_t stream);

/* usage[edges[i]] += sign for i < n (EdgeAccountant.commit_path /
 * clear_path, UPF:821-836).  present_d (optional) is kept in sync the way the
 * reference does it: present += 1 on commit, present = max(0, present - 1) on
 * clear; the usage count never drops below 0. */
ORSP_API int orsp_commit_edges(int64_t n, const int32_t *edges_d, int32_t *usage_d,
                      float *present_d, int32_t sign, uintptr_t stream);

/* commit_path / clear_path (UPF:821-836) for every path of a batch produced
 * by orsp_sssp_batch_bbox (path_len[k] nodes give path_len[k]-1 edges;
 * entries with path_len < 2 are skipped). */
ORSP_API int orsp_commit_batch(int32_t K, const int32_t *path_edges_d,
                      const int32_t *path_len_d, int32_t path_cap,
                      int32_t *usage_d, float *present_d, int32_t sign,
                      uintptr_t stream);

#ifdef __cplusplus
}
#endif
#endif /* ORSP_H */
