// otg_internal.cuh -- shared definitions of the libotg CUDA sources.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/otg.h"

namespace otg {

// Kernel-launch counter (reported by otg_kernel_launches()).
void count_launch();

// Per-net workspace of the block path, in bytes from the slice base.  The
// slice is shared memory for nets that fit, a per-CTA slice of the caller's
// workspace otherwise.  Three regions:
//   I  (whole net)  pre[n] (by local id), nap[n] (preorder -> local id),
//                   size[n] (subtree size by preorder), nas[n] (BFS slot ->
//                   local id), tour[2m] (adjacency, then Euler tour codes)
//   A  (topology)   posin[2m], lr[2m] (int2: next, rank; also the radix
//                   ping-pong), es[m], et[m], start[n+1], depth[n],
//                   parent[n], pedge[n], slot[n], hist[256*W]
//   B  (Elmore)     pres[n], cap[n] f4, X[n] f4, Y[n] f4, L[n] f4,
//                   Bh[c] f4, Bl[c] f4 (c = chunks of 4 preorder slots)
// B overlays A once the topology outputs are written; pres (first in B)
// only overlaps posin, which is dead by then.
struct RcLayout {
  uint32_t pre, nap, size, nas, tour;
  uint32_t posin, lr, es, et, start, depth, parent, pedge, slot, hist;
  uint32_t pres, cap, X, Y, L, Bh, Bl;
  uint32_t total;
};

__host__ __device__ inline RcLayout rc_layout(int n, int T) {
  RcLayout l;
  const uint32_t N = (uint32_t)n, M = n > 0 ? (uint32_t)(n - 1) : 0u, A = 2u * M;
  const uint32_t W = (uint32_t)T / 32u, NCH = (N + 3u) / 4u + 1u;
  uint32_t o = 0;
#define OTG_TAKE(f, bytes)             \
  do {                                 \
    l.f = o;                           \
    o = (o + (bytes) + 15u) & ~15u;    \
  } while (0)
  OTG_TAKE(pre, 4u * N);
  OTG_TAKE(nap, 4u * N);
  OTG_TAKE(size, 4u * N);
  OTG_TAKE(nas, 4u * N);
  OTG_TAKE(tour, 4u * A);
  const uint32_t r0 = o;
  OTG_TAKE(posin, 4u * A);
  OTG_TAKE(lr, 8u * A);
  OTG_TAKE(es, 4u * M);
  OTG_TAKE(et, 4u * M);
  OTG_TAKE(start, 4u * (N + 1u));
  OTG_TAKE(depth, 4u * N);
  OTG_TAKE(parent, 4u * N);
  OTG_TAKE(pedge, 4u * N);
  OTG_TAKE(slot, 4u * N);
  OTG_TAKE(hist, 4u * 256u * W);
  const uint32_t endA = o;
  o = r0;
  OTG_TAKE(pres, 4u * N);
  OTG_TAKE(cap, 16u * N);
  OTG_TAKE(X, 16u * N);
  OTG_TAKE(Y, 16u * N);
  OTG_TAKE(L, 16u * N);
  OTG_TAKE(Bh, 16u * NCH);
  OTG_TAKE(Bl, 16u * NCH);
#undef OTG_TAKE
  l.total = endA > o ? endA : o;
  return l;
}

// Net-size classes: class c takes nets with nmax[c-1] < n <= nmax[c].
struct RcClasses {
  static constexpr int kMax = 7;
  int num;
  int nmax[kMax];
};

RcClasses rc_classes(int smem_budget);
int rc_smem_nmax(int T, int smem_budget);

}  // namespace otg
