// Device helpers shared by the accounting kernels and the routing loop.
#pragma once
#include "common.cuh"

namespace orsp {

// commit_path / clear_path on one edge (UPF:821-836): usage +-1 (never below
// 0) and present kept equal to it; atomic, so paths of a batch may share edges.
__device__ __forceinline__ void apply_usage(int32_t *usage, float *present, int32_t e,
                                            int32_t sign) {
  if (sign >= 0) {
    atomicAdd(&usage[e], sign);
    if (present) atomicAdd(&present[e], 1.0f);
  } else {
    // clear_path: canonical count drops (never below 0) and
    // present = max(0, present - 1)
    int32_t old = __ldcg(&usage[e]);
    for (;;) {
      const int32_t nv = old > 0 ? old - 1 : 0;
      const int32_t prev = atomicCAS(&usage[e], old, nv);
      if (prev == old) break;
      old = prev;
    }
    if (present) {
      unsigned *pp = (unsigned *)&present[e];
      unsigned ob = __ldcg(pp);
      for (;;) {
        float nv = __fsub_rn(__uint_as_float(ob), 1.0f);
        nv = nv > 0.0f ? nv : 0.0f;
        const unsigned prev = atomicCAS(pp, ob, __float_as_uint(nv));
        if (prev == ob) break;
        ob = prev;
      }
    }
  }
}

// Live-usage cost (classic PathFinder, the per-net refresh the reference's
// EdgeAccountant.update_present_cost_only (UPF:1045-1068) is meant for):
//   total = ((base*via_mult)*base_w) + pres_fac*max(0, (usage+1) - cap)
//           + hist_w*history [+ jitter]
// i.e. update_costs with present_ema replaced by the prospective usage if the
// net being routed takes the edge.  Applied to every edge (edges == nullptr)
// or to a list of edge ids (negative ids skipped; repeats are harmless).
__device__ __forceinline__ float live_cost(int64_t e, const float *base, const int32_t *usage,
                                           const float *cap, const float *hist, float pres_fac,
                                           float hist_w, float via_mult, float base_w, int jitter) {
  float over = __fsub_rn(__fadd_rn((float)usage[e], 1.0f), cap[e]);
  over = over > 0.0f ? over : 0.0f;
  const float adjusted = __fmul_rn(__fmul_rn(base[e], via_mult), base_w);
  float total = __fadd_rn(__fadd_rn(adjusted, __fmul_rn(pres_fac, over)), __fmul_rn(hist_w, hist[e]));
  if (jitter) total = __fadd_rn(total, __fmul_rn(fmodf(__ll2float_rn(e), 9973.0f), 1e-6f));
  return total;
}

}  // namespace orsp
