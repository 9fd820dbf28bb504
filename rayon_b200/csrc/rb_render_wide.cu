// The per-pixel kernel's instances for scenes traversed on the 4-wide copy of
// their BVH (compiled apart from the binary-tree instances in rb_render.cu).
#include "rb_render_kernel.cuh"

namespace rb {

int k_render_dispatch_wide(bool launch, bool nee, int ms, int minb, dim3 grd, dim3 blk, size_t sm, cudaStream_t st,
                           const SceneView &S, const Globals &G, const FrameF &P, float4 *acc, float4 *comp,
                           float4 *part, int *counts, unsigned long long *counters, int *fetch, int nslices) {
  return k_render_dispatch<RB_NODES_WIDE>(launch, nee, ms, minb, grd, blk, sm, st, S, G, P, acc, comp, part, counts,
                                          counters, fetch, nslices);
}

}  // namespace rb
