// Device helpers shared by the FP64 and the tensor-core plane-wave kernels.
#pragma once
#include <cuda_runtime.h>

namespace bfgt {

// Fixed-order reduction of the per-chunk partial expansions into the cutoff
// boxes' expansions, done by the form kernels themselves.  Chunks of a cutoff
// box are grouped by 32.  Called by every thread of a form CTA after it has
// written its partial Mpart(chunk, 0:nd-1, :): the last CTA of a group sums the
// group's partials in chunk order (into M directly when the box has one group,
// else into G(group)); the last group of a box sums the box's groups in order
// into M.  Counters are re-armed for the next transform.  This completes the
// merge to the cutoff level of boxfgt.f:764-783.  A group expects groups[g].w
// arrivals: one per CTA that writes partials of its chunks (a chunk's
// densities may be split over several CTAs).
struct ReduceArgs {
  const double2 *Mpart;
  double2 *G;
  double2 *M;
  int *gcnt, *bcnt;
  const int *chunk_group;   // chunk -> group
  const int4 *groups;       // {chunk begin, chunk end, icut, arrivals}
  const int *box_groups;    // icut -> first group (ncut + 1 entries)
};

#ifdef __CUDACC__
__device__ __forceinline__ void sum_partials(const double2 *src, size_t per, int c0, int c1, double2 *dst) {
  for (size_t e = threadIdx.x; e < per; e += blockDim.x) {
    double2 s = make_double2(0, 0);
    for (int c = c0; c < c1; c++) {
      const double2 v = __ldcg(&src[(size_t)c * per + e]);
      s.x += v.x;
      s.y += v.y;
    }
    dst[e] = s;
  }
}

__device__ __forceinline__ void finish_cutoff_box(const ReduceArgs &r, int chunk, int nd, int nexp, int *s_flag) {
  const size_t per = (size_t)nd * nexp;
  const int g = r.chunk_group[chunk];
  const int4 gi = r.groups[g];
  const int icut = gi.z;
  const int bg0 = r.box_groups[icut], bg1 = r.box_groups[icut + 1];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) *s_flag = (atomicAdd(&r.gcnt[g], 1) == gi.w - 1) ? 1 : 0;
  __syncthreads();
  if (!*s_flag) return;
  __threadfence();
  if (bg1 - bg0 == 1) {
    sum_partials(r.Mpart, per, gi.x, gi.y, r.M + (size_t)icut * per);
    if (threadIdx.x == 0) r.gcnt[g] = 0;
    return;
  }
  sum_partials(r.Mpart, per, gi.x, gi.y, r.G + (size_t)g * per);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    r.gcnt[g] = 0;
    *s_flag = (atomicAdd(&r.bcnt[icut], 1) == bg1 - bg0 - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!*s_flag) return;
  __threadfence();
  sum_partials(r.G, per, bg0, bg1, r.M + (size_t)icut * per);
  if (threadIdx.x == 0) r.bcnt[icut] = 0;
}

#endif  // __CUDACC__

}  // namespace bfgt
