// otg_internal.cuh -- shared definitions of the libotg CUDA sources.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/otg.h"

namespace otg {

// Kernel-launch counter (reported by otg_kernel_launches()).
void count_launch();

// ---- bounded grid barrier of the cooperative kernels (levelization,
// propagation).  Every wait gives up after kGridWaitNs of %globaltimer,
// raises `abort` (which every other wait watches) and records
// OTG_ERR_TIMEOUT, so a stuck launch returns instead of hanging.
constexpr unsigned long long kGridWaitNs = 2000000000ull;  // 2 s per barrier wait

struct GridCtl {
  unsigned count;  // barrier arrivals
  unsigned gen;    // barrier generation
  int abort;       // set by a wait that timed out
  int status;      // OTG_* status of the launch
};

__device__ __forceinline__ unsigned long long gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Returns false if the barrier was abandoned (timeout somewhere).
__device__ inline bool grid_barrier(GridCtl* c) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile GridCtl* vc = c;
    int ok = 1;
    const unsigned gen = vc->gen;
    __threadfence();
    const unsigned arrived = atomicAdd(&c->count, 1u);
    if (arrived == gridDim.x - 1) {
      c->count = 0;
      __threadfence();
      atomicAdd(&c->gen, 1u);
    } else {
      // each poll is one L2 round trip: the abort flag and the clock are
      // read on every 8th poll only, and no poll sleeps (a sleeping thread
      // sees the release only after it wakes)
      const unsigned long long t0 = gtime();
      for (int k = 0; vc->gen == gen; ++k) {
        if ((k & 7) == 7) {
          if (vc->abort) { ok = 0; break; }
          if (gtime() - t0 > kGridWaitNs) {
            atomicExch(&c->abort, 1);
            atomicCAS(&c->status, 0, (int)OTG_ERR_TIMEOUT);
            ok = 0;
            break;
          }
        }
      }
    }
    __threadfence();
    if (vc->abort) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Per-net workspace of the block path, in bytes from the slice base.  The
// slice is shared memory for nets that fit (16-bit indices), a per-CTA
// slice of the caller's workspace otherwise (32-bit indices).  Regions:
//   I  (whole net)  pre[n] (by local id), nap[n] (preorder -> local id),
//                   size[n] (subtree size by preorder), nas[n] (BFS slot ->
//                   local id), tour[2m] (adjacency, then the Euler tour,
//                   then signed tour codes), pres[n] f32 (by preorder)
//   A  (topology)   es[m], et[m], then one of
//                     A-a  ends[n] i32, posin[2m]
//                     A-b  sub[2m], off[2m], spl[2m], splarc[S], sl[S] u64
//                     A-c  depth[n], parent[n], pedge[n], slot[n]
//                   then succ[2m] / radix buffers 2n, hist[bins*W] i32
//   B  (Elmore, one corner pair at a time; overlays A)
//                   X[n] f2 (load, then ldelay), Y[n] f2 (delay),
//                   Ip[n] 2 x i64 (fixed-point inclusive prefix of an
//                   up-sweep; then the impulse, f2)
struct RcLayout {
  uint32_t pre, nap, size, nas, tour, pres;
  uint32_t es, et, ends, posin, sub, off, spl, splarc, sl, depth, parent, pedge, slot;
  uint32_t r2, hist;
  uint32_t X, Y, Ip;
  uint32_t total;
  uint32_t ns_cap;  // capacity of the splitter arrays
};

// Sublist splitters of the Euler-tour ranking: about one arc in kSplit
// (a power of two; OTG_KSPLIT overrides it at build time).
#ifndef OTG_KSPLIT
#define OTG_KSPLIT 8
#endif
constexpr int kSplit = OTG_KSPLIT;

// Radix digit of the block sort: 8 bits, 7 for 1024-thread CTAs (whose
// 32 per-warp histograms would otherwise take 32 KB of shared memory).
__host__ __device__ constexpr int rc_radix_bits(int T) { return T >= 1024 ? 7 : 8; }

__host__ __device__ inline uint32_t rc_max3(uint32_t a, uint32_t b, uint32_t c) {
  return a > b ? (a > c ? a : c) : (b > c ? b : c);
}

__host__ __device__ inline RcLayout rc_layout(int n, int T, int K, int ib, int S = 1) {
  RcLayout l;
  const uint32_t N = (uint32_t)n, M = n > 0 ? (uint32_t)(n - 1) : 0u, A = 2u * M;
  const uint32_t W = (uint32_t)(S * T) / 32u;  // warps of the group (S CTAs of T threads)
  (void)K;
  const uint32_t I = (uint32_t)ib;
  l.ns_cap = 2u * (A / (uint32_t)kSplit) + 64u;
  uint32_t o = 0;
#define OTG_AL(x) (((x) + 15u) & ~15u)
#define OTG_TAKE(f, bytes)      \
  do {                          \
    l.f = o;                    \
    o = OTG_AL(o + (bytes));    \
  } while (0)
  OTG_TAKE(pre, I * N);
  OTG_TAKE(nap, I * N);
  OTG_TAKE(size, I * N);
  OTG_TAKE(nas, I * N);
  OTG_TAKE(tour, I * A);
  OTG_TAKE(pres, 4u * N);
  const uint32_t rA = o;
  OTG_TAKE(es, I * M);
  OTG_TAKE(et, I * M);
  const uint32_t r1 = o;
  // A-a
  OTG_TAKE(ends, 4u * N);
  OTG_TAKE(posin, I * A);
  const uint32_t end_a = o;
  // A-b
  o = r1;
  OTG_TAKE(sub, I * A);
  OTG_TAKE(off, I * A);
  OTG_TAKE(spl, I * A);
  OTG_TAKE(splarc, I * l.ns_cap);
  OTG_TAKE(sl, 8u * l.ns_cap);
  const uint32_t end_b = o;
  // A-c
  o = r1;
  OTG_TAKE(depth, I * N);
  OTG_TAKE(parent, I * N);
  OTG_TAKE(pedge, I * N);
  OTG_TAKE(slot, I * N);
  const uint32_t end_c = o;
  o = rc_max3(end_a, end_b, end_c);
  OTG_TAKE(r2, I * (A > 2u * N ? A : 2u * N));
  OTG_TAKE(hist, 4u * (1u << rc_radix_bits(T)) * W);
  const uint32_t endA = o;
  o = rA;
  OTG_TAKE(X, 8u * (N + N / 4u + 1u));  // padded slots, see rc_pad8
  OTG_TAKE(Y, 8u * (N + N / 4u + 1u));
  OTG_TAKE(Ip, 16u * (N + N / 8u + 1u));  // rc_pad16
#undef OTG_TAKE
#undef OTG_AL
  l.total = endA > o ? endA : o;
  return l;
}

// Padded slot indices of the Elmore arrays.  The scans give each thread K
// consecutive slots, so for a given k a warp's lanes touch elements K
// apart, several to a shared-memory bank; one spare element per 4 (8-byte
// X, Y) and per 8 (16-byte Ip) spreads them over the banks.
__host__ __device__ __forceinline__ int rc_pad8(int i) { return i + (i >> 2); }
__host__ __device__ __forceinline__ int rc_pad16(int i) { return i + (i >> 3); }

// Net-size classes: class c takes nets with nmax[c-1] < n <= nmax[c].
struct RcClasses {
  static constexpr int kMax = 8;
  int num;
  int nmax[kMax];
};



// Entry of the fused RC pass with an explicit workspace (otg_rc.cu); the
// public otg_rc_timing wraps it.
otg_status rc_launch(const otg_rc_forest* f, int max_net_nodes, void* workspace,
                     size_t workspace_bytes, cudaStream_t stream);

// Multi-forest form (used by the design server): `forests` is a device
// array of per-forest kernel arguments (rc_args_bytes() each, filled on the
// host with rc_args_fill and copied up), `items` a device list of
// (forest, net) pairs whose length is read from *num_dev (at most cap).
// `fork` (optional): side streams the size-class launches are spread
// over, joined back into `stream` before the call returns (also under
// stream capture, where they become parallel graph branches).
struct RcFork {
  static constexpr int kMax = 4;
  int n = 0;
  cudaStream_t side[kMax] = {};
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[kMax] = {};
};
cudaError_t rc_fork_create(RcFork* f, int n);
void rc_fork_destroy(RcFork* f);
struct RcArgsOpaque;
otg_status rc_launch_items(const RcArgsOpaque* forests, const int2* items, const int* num_dev,
                           int cap, int max_net_nodes, void* workspace, size_t workspace_bytes,
                           cudaStream_t stream, const RcFork* fork = nullptr);
size_t rc_args_bytes();
void rc_args_fill(const otg_rc_forest* f, int* status, void* out);
}  // namespace otg
