// otg_levelize.cu -- timing-graph levelization (frontier Kahn) on B200.
//
// Replaces toposort_advance + toposort_compute_cuda (ot/cuda/toposort.cu:4-72)
// which launch one kernel per level and copy the frontier size back to the
// host after each one.  Here every level runs inside ONE cooperative launch:
//
//   level 0      = the caller's seed (pins without candidate fanout)
//   expand(k)    every pin of level k decrements the fanout counter of each
//                of its fanins, edge-parallel: a block scan over the pins'
//                fanin counts hands one edge to each thread, so all of a
//                chunk's decrements are in flight at once (warp-aggregated
//                atomics: lanes that hit the same pin combine into one
//                atomicSub); the pin whose counter reaches zero sets its bit
//                in the "ready" bitmap
//   compact(k+1) the ready bitmap is split into per-CTA word ranges of C
//                words.  The expansion that sets a pin's bit also counts it
//                for its range, so after ONE grid barrier every CTA knows its
//                offset (the counts of the ranges before it), writes its pins
//                in ascending index order there -- every level after the seed
//                comes out sorted by pin index, deterministically -- and
//                expands them into the other bitmap.  The range counts rotate
//                through three buffers: read in level k, filled for k+1,
//                cleared for k+2.
//
// One grid barrier per level.  The barrier is a sense-counting barrier on
// global memory whose waits are bounded by %globaltimer: a wait that runs
// past the limit raises an abort flag that every other wait also watches,
// so the kernel always returns and the host sees OTG_ERR_TIMEOUT.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <climits>

#include "../../include/otg.h"
#include "otg_internal.cuh"

namespace otg {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int LT = 512;                              // threads per CTA
using LvCtl = GridCtl;

// One fanin edge per lane (target v, ok = a valid pin): decrement v's
// fanout counter; the pin whose counter reaches zero sets its bit in `bm`
// and counts for its range.  Lanes of a warp that target the same pin
// combine into one atomicSub.  Every lane of the warp must call it.  A
// seed pin's counter starts at INT_MAX, so a seed is never emitted twice,
// even if the caller's out_deg disagrees with the fanin lists, and no
// other read is needed on this chain.
__device__ __forceinline__ void decrement(int v, bool ok, int* cnt, unsigned* bm, int* rcount,
                                          int C) {
  const int lane = threadIdx.x & 31;
  const unsigned peers = __match_any_sync(FULL, ok ? v : -2 - lane);
  if (ok && (__ffs(peers) - 1 == lane)) {
    const int k = __popc(peers);
    const int old = atomicSub(&cnt[v], k);
    if (old > 0 && old - k <= 0) {
      atomicOr(&bm[v >> 5], 1u << (v & 31));
      atomicAdd(&rcount[(v >> 5) / C], 1);
    }
  }
}

// Decrement the fanout counters of u's fanins, one edge per lane per step
// (the seed level).
__device__ __forceinline__ void expand_pin(int u, bool active, const int* fanin_start,
                                           const int* fanin, int* cnt, unsigned* bm, int n,
                                           int* rcount, int C) {
  int e = active ? fanin_start[u] : 0;
  const int e1 = active ? fanin_start[u + 1] : 0;
  while (__any_sync(FULL, e < e1)) {
    const bool has = e < e1;
    const int v = has ? fanin[e] : -1;
    decrement(v, has && (unsigned)v < (unsigned)n, cnt, bm, rcount, C);
    e += has ? 1 : 0;
  }
}

__global__ void __launch_bounds__(LT) levelize_kernel(int n, const int* fanin_start,
                                                      const int* fanin, const int* out_deg,
                                                      const int* frontier0, int first_size,
                                                      int* order, int* level, int* level_ends,
                                                      int* counts, LvCtl* ctl, int* cnt,
                                                      unsigned* bm0, unsigned* bm1, int* blk) {
  // blk: three rotating [G] buffers of per-range ready counts
  __shared__ int wsum[LT / 32];
  __shared__ int red_t[LT / 32], red_b[LT / 32];
  __shared__ int s_estart[LT], s_e0[LT];
  __shared__ int s_total, s_off;
  const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
  const int gtid = b * LT + tid, gstride = G * LT;
  const int nw = (n + 31) >> 5;
  const int lane = tid & 31, w = tid >> 5;

  for (int v = gtid; v < n; v += gstride) {
    cnt[v] = out_deg[v];
    level[v] = -1;
  }
  for (int i = gtid; i < nw; i += gstride) bm0[i] = bm1[i] = 0u;
  for (int i = gtid; i < 3 * G; i += gstride) blk[i] = 0;
  const int C = max(1, (nw + G - 1) / G);  // bitmap words per CTA range
  if (!grid_barrier(ctl)) return;
  for (int k = gtid; k < first_size; k += gstride) {
    const int v = frontier0[k];
    order[k] = v;
    if ((unsigned)v < (unsigned)n) {
      level[v] = 0;
      cnt[v] = INT_MAX;  // after the counters' fill (grid barrier above)
    } else {
      atomicCAS(&ctl->status, 0, (int)OTG_ERR_INVALID);
    }
  }
  if (gtid == 0) {
    level_ends[0] = 0;
    if (first_size > 0) level_ends[1] = first_size;
  }
  if (first_size == 0) {
    if (gtid == 0) { counts[0] = 0; counts[1] = 0; }
    return;
  }
  if (!grid_barrier(ctl)) return;
  // expand the seed
  for (int k0 = b * LT; k0 < first_size; k0 += gstride) {
    const int k = k0 + tid;
    const bool act = k < first_size && (unsigned)order[k] < (unsigned)n;
    expand_pin(act ? order[k] : 0, act, fanin_start, fanin, cnt, bm0, n, blk + G, C);
  }
  unsigned* cur = bm0;
  unsigned* nxt = bm1;
  int emitted = first_size;
  int L = 1;
  const int w0 = min(nw, b * C), w1 = min(nw, (b + 1) * C);
  while (true) {
    if (!grid_barrier(ctl)) return;
    int* rc_now = blk + (L % 3) * G;         // counts of this level's ranges
    int* rc_next = blk + ((L + 1) % 3) * G;  // filled by this level's expansion
    if (tid == 0) blk[((L + 2) % 3) * G + b] = 0;  // read a level ago, filled next level
    // the first tile's bitmap words load while the counts are summed
    unsigned word0[2];
#pragma unroll
    for (int j = 0; j < 2; ++j)
      word0[j] = w0 + 2 * tid + j < w1 ? __ldcg(cur + w0 + 2 * tid + j) : 0u;
    // offset of this CTA and level total: every thread reads at most a few
    // counts (independent loads), then a block reduction
    {
      int before = 0, total = 0;
      for (int i = tid; i < G; i += LT) {
        const int x = __ldcg(rc_now + i);
        total += x;
        if (i < b) before += x;
      }
      for (int d = 16; d >= 1; d >>= 1) {
        total += __shfl_xor_sync(FULL, total, d);
        before += __shfl_xor_sync(FULL, before, d);
      }
      if (lane == 0) { red_t[w] = total; red_b[w] = before; }
      __syncthreads();
      if (tid == 0) {
        int t = 0, o = 0;
        for (int k = 0; k < LT / 32; ++k) { t += red_t[k]; o += red_b[k]; }
        s_total = t;
        s_off = o;
      }
      __syncthreads();
    }
    const int total = s_total;
    if (total == 0) break;
    int run = emitted + s_off;
    // write own pins in ascending order, tile by tile (two bitmap words per
    // thread), and expand them
    for (int t0 = w0; t0 < w1; t0 += 2 * LT) {
      const int i = t0 + 2 * tid;
      unsigned wd[2];
#pragma unroll
      for (int j = 0; j < 2; ++j)
        wd[j] = t0 == w0 ? word0[j] : (i + j < w1 ? __ldcg(cur + i + j) : 0u);
      const int pc = __popc(wd[0]) + __popc(wd[1]);
      // block exclusive scan of pc
      int x = pc;
      for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(FULL, x, d);
        if (lane >= d) x += y;
      }
      if (lane == 31) wsum[w] = x;
      __syncthreads();
      int wb = 0, tt = 0;
      for (int u = 0; u < LT / 32; ++u) {
        if (u < w) wb += wsum[u];
        tt += wsum[u];
      }
      __syncthreads();
      int pos = run + wb + x - pc;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        unsigned bits = wd[j];
        while (bits) {
          const int bit = __ffs(bits) - 1;
          bits &= bits - 1;
          const int v = ((i + j) << 5) + bit;
          if (pos < n) {
            order[pos] = v;
          } else {
            atomicCAS(&ctl->status, 0, (int)OTG_ERR_INVALID);  // duplicate seeds
          }
          ++pos;
          level[v] = L;
        }
        if (i + j < w1) cur[i + j] = 0u;  // ready for reuse two levels on
      }
      __syncthreads();  // the tile's slice of `order` is visible to the CTA
      // expand the tile's pins edge-parallel: LT pins at a time, their fanin
      // edges spread one per thread, so every decrement of a chunk is in
      // flight at once instead of one edge after another per pin
      const int tn = min(tt, n - run);
      for (int c0 = 0; c0 < tn; c0 += LT) {
        const int k = c0 + tid;
        int e0 = 0, deg = 0;
        if (k < tn) {
          const int u = order[run + k];
          if ((unsigned)u < (unsigned)n) {
            e0 = fanin_start[u];
            deg = fanin_start[u + 1] - e0;
          }
        }
        // block exclusive scan of the degrees
        int y = deg;
        for (int d = 1; d < 32; d <<= 1) {
          const int z = __shfl_up_sync(FULL, y, d);
          if (lane >= d) y += z;
        }
        if (lane == 31) wsum[w] = y;
        __syncthreads();
        int eb = 0, etot = 0;
        for (int u = 0; u < LT / 32; ++u) {
          if (u < w) eb += wsum[u];
          etot += wsum[u];
        }
        s_estart[tid] = eb + y - deg;
        s_e0[tid] = e0;
        __syncthreads();
        const int np = min(LT, tn - c0);
        for (int q0 = 0; q0 < etot; q0 += LT) {
          const int q = q0 + tid;
          int v = -1;
          if (q < etot) {
            // the pin owning edge q: the last one whose start is <= q
            int lo = 0, hi = np - 1;
            while (lo < hi) {
              const int mid = (lo + hi + 1) >> 1;
              if (s_estart[mid] <= q) lo = mid; else hi = mid - 1;
            }
            v = fanin[s_e0[lo] + (q - s_estart[lo])];
          }
          decrement(v, (unsigned)v < (unsigned)n, cnt, nxt, rc_next, C);
        }
        __syncthreads();  // s_estart / s_e0 / wsum are reused
      }
      run += tt;
    }
    emitted += total;
    if (emitted > n) {  // only reachable with duplicate seeds; stop cleanly
      if (gtid == 0) atomicCAS(&ctl->status, 0, (int)OTG_ERR_INVALID);
      emitted = n;
      break;
    }
    if (gtid == 0) level_ends[L + 1] = emitted;
    ++L;
    unsigned* t = cur;
    cur = nxt;
    nxt = t;
  }
  if (gtid == 0) {
    counts[0] = L;
    counts[1] = emitted;
  }
}

struct LvDev {
  int sms = 0;
  int occ = 0;
  bool init = false;
};
LvDev g_lv[64];

LvDev& lv_dev() {
  int d = 0;
  cudaGetDevice(&d);
  LvDev& x = g_lv[d & 63];
  if (!x.init) {
    cudaDeviceGetAttribute(&x.sms, cudaDevAttrMultiProcessorCount, d);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&x.occ, levelize_kernel, LT, 0);
    x.occ = std::max(1, std::min(x.occ, 2));
    x.init = true;
  }
  return x;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct LvWs {
  size_t ctl, cnt, bm0, bm1, blk, total;
};
LvWs lv_ws(int n, int G) {
  LvWs l;
  size_t o = 0;
  l.ctl = o; o = align256(o + sizeof(LvCtl));
  l.cnt = o; o = align256(o + 4 * (size_t)std::max(n, 1));
  const size_t nw = ((size_t)n + 31) / 32 + 1;
  l.bm0 = o; o = align256(o + 4 * nw);
  l.bm1 = o; o = align256(o + 4 * nw);
  l.blk = o; o = align256(o + 12 * (size_t)G);  // three rotating [G] count buffers
  l.total = o;
  return l;
}

}  // namespace
}  // namespace otg

extern "C" {

otg_status otg_levelize_workspace_size(int32_t n, int32_t num_edges, size_t* bytes) {
  (void)num_edges;
  if (!bytes || n < 0) return OTG_ERR_INVALID;
  otg::LvDev& d = otg::lv_dev();
  if (d.sms <= 0) return OTG_ERR_CUDA;
  *bytes = otg::lv_ws(n, d.sms * d.occ).total;
  return OTG_OK;
}

otg_status otg_levelize(int32_t n, int32_t num_edges, const int32_t* fanin_start,
                        const int32_t* fanin, const int32_t* out_deg, const int32_t* frontier0,
                        int32_t first_size, int32_t* order, int32_t* level, int32_t* level_ends,
                        int32_t* counts, void* workspace, size_t workspace_bytes,
                        otg_stream_t stream) {
  if (n < 0 || num_edges < 0 || first_size < 0 || first_size > n || !workspace || !counts ||
      !level_ends)
    return OTG_ERR_INVALID;
  if (n > 0 && (!fanin_start || !out_deg || !order || !level || (first_size && !frontier0) ||
                (num_edges && !fanin)))
    return OTG_ERR_INVALID;
  otg::LvDev& d = otg::lv_dev();
  int G = d.sms * d.occ;
  const otg::LvWs l = otg::lv_ws(n, G);
  if (workspace_bytes < l.total) return OTG_ERR_WORKSPACE;
  const int nw = (n + 31) / 32;
  // Small graphs take fewer CTAs: a range of at least kWordsPerCta bitmap
  // words each, so that fewer CTAs meet at every level's grid barrier.  On a
  // 165k-pin, 600-level graph, 81 CTAs took 4.16 ms where 296 took 4.50
  // (6 and 21 CTAs: 4.32 and 4.42); graphs of 5M pins keep every CTA.
  constexpr int kWordsPerCta = 64;
  G = std::max(1, std::min(G, (nw + kWordsPerCta - 1) / kWordsPerCta));
  char* ws = (char*)workspace;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(ws + l.ctl, 0, sizeof(otg::LvCtl), s) != cudaSuccess) return OTG_ERR_CUDA;
  otg::LvCtl* ctl = (otg::LvCtl*)(ws + l.ctl);
  int* cnt = (int*)(ws + l.cnt);
  unsigned* bm0 = (unsigned*)(ws + l.bm0);
  unsigned* bm1 = (unsigned*)(ws + l.bm1);
  int* blk = (int*)(ws + l.blk);
  void* args[] = {&n,     (void*)&fanin_start, (void*)&fanin, (void*)&out_deg, (void*)&frontier0,
                  &first_size, &order, &level, &level_ends, &counts, &ctl, &cnt, &bm0, &bm1, &blk};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)otg::levelize_kernel, dim3(G),
                                              dim3(otg::LT), args, 0, s);
  otg::count_launch();
  return e == cudaSuccess ? OTG_OK : OTG_ERR_CUDA;
}

otg_status otg_levelize_status(const void* workspace, otg_stream_t stream) {
  if (!workspace) return OTG_ERR_INVALID;
  otg::LvCtl h;
  if (cudaMemcpyAsync(&h, workspace, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream) !=
          cudaSuccess ||
      cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
    return OTG_ERR_CUDA;
  return (otg_status)h.status;
}

}  // extern "C"
