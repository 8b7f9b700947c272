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
//
// Graphs of up to about a million pins run instead in ONE thread-block
// cluster (levelize_cluster_kernel below):
// the same rule and the same outputs, with the ready bitmaps and counts in
// distributed shared memory, the hardware cluster barrier between levels,
// and the next level's fanin ranges gathered while the counters are
// decremented.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <climits>
#include <cstdlib>

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

// ---- the cluster path --------------------------------------------------
//
// Graphs whose two ready bitmaps fit in the shared memory of one thread-
// block cluster (up to 16 CTAs, 8 or fewer where the device cannot place
// 16) run the same frontier rule inside one cluster: CTA r owns the bitmap
// words [r*C, (r+1)*C) of both levels in its own shared memory, and a pin
// whose fanout counter reaches zero sets its bit and bumps its owner's
// count through distributed shared memory.  A level ends at the hardware
// cluster barrier (barrier.cluster, release/acquire) instead of the global
// barrier, and the counts and bitmaps never leave the SMs.  Where the
// ranges' fanout counters fit beside them (32 ints per bitmap word), the
// counters live in their owner's shared memory too, and a level costs the
// dependent global loads of its expansion (the fanin entry; the fanin
// range, loaded speculatively beside the decrement) plus on-chip work.
// The emission rule is the one
// above (seed order, then ascending pin index per level, CTA ranges in rank
// order), so both paths give identical outputs.
//
// No wait in this path polls memory: the cluster barrier is hardware, and
// every CTA takes the same number of barriers (the loop ends on the level
// total, which every CTA computes from the same counts).

// CTA widths of the cluster path: a level of a narrow graph has a few pins
// per CTA, and every warp of the CTA takes part in each of its scans and
// barriers, so narrow graphs run narrow CTAs.
constexpr int kCtMax = 1024;

// Optional per-segment cycle accounting of the level loop (build with
// -DOTG_PHASE_TIMING): thread 0 of CTA 0 sums the clock64() deltas of each
// segment and stores them after the counts, in counts[2..9] (the caller
// then passes a counts array of 10).
#ifdef OTG_PHASE_TIMING
#define LV_PHASE_BEGIN() long long _ph_t = clock64(), _ph[8] = {0, 0, 0, 0, 0, 0, 0, 0}
#define LV_PHASE(k)                        \
  do {                                     \
    if (gtid == 0) {                       \
      const long long _t = clock64();      \
      _ph[k] += _t - _ph_t;                \
      _ph_t = _t;                          \
    }                                      \
  } while (0)
#define LV_PHASE_END(c)                                                   \
  do {                                                                    \
    if (gtid == 0)                                                        \
      for (int _k = 0; _k < 8; ++_k) (c)[2 + _k] = (int)(_ph[_k] >> 10); \
  } while (0)
#else
#define LV_PHASE_BEGIN() \
  do {                   \
  } while (0)
#define LV_PHASE(k) \
  do {              \
  } while (0)
#define LV_PHASE_END(c) \
  do {                  \
  } while (0)
#endif

namespace cg = cooperative_groups;

// Where a pin that becomes ready goes: its owner's bitmap word and count
// (distributed shared memory), and the list of fanin ranges that one CTA,
// chosen by a hash of the pin, expands next level.  (Hashing keeps the
// lists even: a CTA that readied a whole level -- a buffer tree readies
// its levels from one place -- would otherwise expand the next one alone.)
struct ClNext {
  unsigned* bm;  // next level's bitmap (this CTA's address; mapped to the owner)
  int* scnt;     // the fanin counters of the CTA's range (mapped to the owner), or null:
                 // the counters are the global cnt[]
  int cshift;    // log2 of the words per CTA range: the owner of word w is w >> cshift
  int sshift;    // log2 of the cluster size
  int* rc;       // next level's per-owner counts [16] (every CTA keeps a copy)
  int2* lst;     // next level's list of (fanin start, fanin count) (mapped to the target)
  int* lcnt;     // its length (likewise)
  int* ovf;      // next level's overflow flag (set in every CTA)
  int cap;       // list capacity
};

// One fanin edge per lane (as decrement above).  The leader lane of each
// distinct pin v also loads v's fanin range, in flight with the decrement,
// so a pin that becomes ready is expanded next level without another
// global round trip; a full list raises the next level's overflow flag in
// every CTA, and that level then expands from the bitmaps instead.  The
// counter lives in the owner's shared memory where the ranges fit there
// (a distributed-shared-memory atomic instead of an L2 round trip on every
// level's critical path).  The warp's pins that became ready add to the
// per-owner counts of every CTA once per owner.
__device__ __forceinline__ void decrement_cl(int v, bool ok, const int* fanin_start, int* cnt,
                                             const ClNext& nx, const cg::cluster_group& cl) {
  const int lane = threadIdx.x & 31;
  const unsigned peers = __match_any_sync(FULL, ok ? v : -2 - lane);
  bool ready = false;
  int owner = 0;
  if (ok && (__ffs(peers) - 1 == lane)) {
    const int k = __popc(peers);
    const int s0 = __ldg(fanin_start + v), s1 = __ldg(fanin_start + v + 1);
    const int w = v >> 5;
    owner = w >> nx.cshift;
    int* c = nx.scnt ? cl.map_shared_rank(nx.scnt + (v - (owner << (nx.cshift + 5))), owner)
                     : cnt + v;
    const int old = atomicSub(c, k);
    if (old > 0 && old - k <= 0) {
      ready = true;
      atomicOr(cl.map_shared_rank(nx.bm, owner) + (w - (owner << nx.cshift)), 1u << (v & 31));
      const int t = nx.sshift ? (int)(((unsigned)v * 0x9E3779B1u) >> (32 - nx.sshift)) : 0;
      const int slot = atomicAdd(cl.map_shared_rank(nx.lcnt, t), 1);
      if (slot < nx.cap) {
        *cl.map_shared_rank(nx.lst + slot, t) = make_int2(s0, s1 - s0);
      } else {
        for (int i = 0; i < (int)cl.num_blocks(); ++i) *cl.map_shared_rank(nx.ovf, i) = 1;
      }
    }
  }
  const unsigned grp = __match_any_sync(FULL, ready ? owner : -1 - lane);
  if (ready && (__ffs(grp) - 1 == lane)) {
    const int k = __popc(grp), S = (int)cl.num_blocks();
    for (int i = 0; i < S; ++i) atomicAdd(cl.map_shared_rank(nx.rc + owner, i), k);
  }
}

template <int CT>
__global__ void __launch_bounds__(CT, 1) levelize_cluster_kernel(
    int n, const int* fanin_start, const int* fanin, const int* out_deg, const int* frontier0,
    int first_size, int* order, int* level, int* level_ends, int* counts, LvCtl* ctl, int* cnt,
    int cshift, int lst_cap, int scnt_on) {
  const int C = 1 << cshift;  // bitmap words per CTA range
  extern __shared__ unsigned lv_sm[];
  unsigned* const bm0 = lv_sm;  // level L's ready pins: bm0 for even L, bm1 for odd
  unsigned* const bm1 = lv_sm + C;
  // with scnt_on: the fanin counters of the range's 32*C pins
  int* const scnt = scnt_on ? (int*)(lv_sm + 2 * C) : nullptr;
  // fanin ranges to expand at even / odd levels
  int2* const lst0 = (int2*)(lv_sm + 2 * C + (scnt_on ? 32 * C : 0));
  int2* const lst1 = lst0 + lst_cap;
  // per-level scalars in three rotating slots (this level, the next, the
  // one after): a slot is cleared a level before anything adds to it, so
  // no block barrier orders the clear
  __shared__ int rc[3][16];  // ready pins of every CTA's range (each CTA keeps a copy)
  __shared__ int lcnt[3];  // length of the list of fanin ranges
  __shared__ int ovf[3];   // some CTA's list overflowed
  __shared__ int wsum[2][2 * (CT / 32)];  // warp totals of the level's scans, by level parity
  __shared__ int s_excl[CT], s_e0[CT];    // list entries: warp-exclusive edge start, fanin start
  const cg::cluster_group cl = cg::this_cluster();
  const int S = (int)cl.num_blocks(), r = (int)cl.block_rank(), tid = threadIdx.x;
  const int sshift = 31 - __clz(S);  // cluster sizes are powers of two
  const int gtid = r * CT + tid, gstride = S * CT;
  const int nw = (n + 31) >> 5;
  const int lane = tid & 31, w = tid >> 5;

  for (int v = gtid; v < n; v += gstride) {
    if (!scnt) cnt[v] = out_deg[v];
    level[v] = -1;
  }
  if (scnt)
    for (int j = tid; j < 32 * C; j += CT) {
      const int v = (r << (cshift + 5)) + j;
      scnt[j] = v < n ? out_deg[v] : 0;
    }
  for (int i = tid; i < 2 * C; i += CT) lv_sm[i] = 0u;
  if (tid < 48) rc[tid / 16][tid % 16] = 0;
  if (tid < 3) { lcnt[tid] = 0; ovf[tid] = 0; }
  cl.sync();
  for (int k = gtid; k < first_size; k += gstride) {
    const int v = frontier0[k];
    order[k] = v;
    if ((unsigned)v < (unsigned)n) {
      level[v] = 0;
      // after the counters' fill (cluster barrier above)
      if (scnt) {
        const int owner = v >> (cshift + 5);
        *cl.map_shared_rank(scnt + (v - (owner << (cshift + 5))), owner) = INT_MAX;
      } else {
        cnt[v] = INT_MAX;
      }
    } else {
      atomicCAS(&ctl->status, 0, (int)OTG_ERR_INVALID);
    }
  }
  if (gtid == 0) {
    level_ends[0] = 0;
    if (first_size > 0) level_ends[1] = first_size;
  }
  if (first_size == 0) {  // uniform: no CTA has touched another's memory
    if (gtid == 0) { counts[0] = 0; counts[1] = 0; }
    return;
  }
  cl.sync();
  // expand the seed into level 1 (bm1, slot 1, lst1)
  {
    const ClNext nx{bm1, scnt, cshift, sshift, rc[1], lst1, &lcnt[1], &ovf[1], lst_cap};
    for (int k0 = r * CT; k0 < first_size; k0 += gstride) {
      const int k = k0 + tid;
      const bool act = k < first_size && (unsigned)order[k] < (unsigned)n;
      const int u = act ? order[k] : 0;
      int e = act ? fanin_start[u] : 0;
      const int e1 = act ? fanin_start[u + 1] : 0;
      while (__any_sync(FULL, e < e1)) {
        const bool has = e < e1;
        const int v = has ? fanin[e] : -1;
        decrement_cl(v, has && (unsigned)v < (unsigned)n, fanin_start, cnt, nx, cl);
        e += has ? 1 : 0;
      }
    }
  }
  int emitted = first_size;
  int L = 1;
  const int w0 = min(nw, r * C), w1 = min(nw, (r + 1) * C);
  // this thread's words of the range: KW consecutive ones
  const int KW = max(1, (w1 - w0 + CT - 1) / CT);
  const int i0 = min(w1, w0 + tid * KW), i1 = min(w1, i0 + KW);
  int q_now = 1, q_next = 2, q_free = 0;
  LV_PHASE_BEGIN();
  while (true) {
    cl.sync();
    LV_PHASE(0);
    const int par = L & 1;
    unsigned* cur = par ? bm1 : bm0;
    int2* lcur = par ? lst1 : lst0;
    const ClNext nx{par ? bm0 : bm1,   scnt,          cshift,       sshift, rc[q_next],
                    par ? lst0 : lst1, &lcnt[q_next], &ovf[q_next], lst_cap};
    if (tid < 16) rc[q_free][tid] = 0;  // read a level ago; added to from the next level on
    if (tid == 0) {
      lcnt[q_free] = 0;
      ovf[q_free] = 0;
    }
    // every warp: the level total and this CTA's offset from the counts
    const int x = lane < S ? rc[q_now][lane] : 0;
    const int before = __reduce_add_sync(FULL, lane < r ? x : 0);
    const int total = __reduce_add_sync(FULL, x);
    if (total == 0) break;  // uniform: every CTA read the same counts
    const int run = emitted + before;
    const int m = lcnt[q_now];          // appended before the cluster barrier
    const bool over = ovf[q_now] != 0;  // likewise; the same in every CTA
#ifdef OTG_PHASE_TIMING
    if (tid == 0 && L < 4096) counts[16 + L * 16 + r] = m;
    const long long _lt0 = clock64();
#endif
    LV_PHASE(3);
    // the emission writes the range's pins in ascending order into `order`
    // with their level and clears the words for reuse two levels on
    auto emit = [&](int pos) {
      for (int i = i0; i < i1; ++i) {
        unsigned bits = cur[i - r * C];
        while (bits) {
          const int bit = __ffs(bits) - 1;
          bits &= bits - 1;
          const int v = (i << 5) + bit;
          if (pos < n) order[pos] = v;
          else atomicCAS(&ctl->status, 0, (int)OTG_ERR_INVALID);  // duplicate seeds
          ++pos;
          level[v] = L;
        }
        cur[i - r * C] = 0u;
      }
    };
    int pc = 0;
    for (int i = i0; i < i1; ++i) pc += __popc(cur[i - r * C]);
    constexpr int W = CT / 32;
    // Expansion of fanin ranges range(k), k < mm, CT at a time: ONE block
    // scan per chunk hands one edge to each thread -- an edge q finds its
    // warp by a shuffle search over the warps' edge totals, then its range
    // by a binary search over that warp's exclusive starts.  With `emit_on`
    // the first chunk's scan also gives the emission offsets (popcounts),
    // and the emission runs while the first fanin loads are in flight.
    auto expand = [&](int mm, auto range, bool emit_on) {
      bool pending = emit_on;
      int c0 = 0;
      do {
        const int k = c0 + tid;
        const int2 en = k < mm ? range(k) : make_int2(0, 0);
        int y1 = en.y, y2 = (emit_on && c0 == 0) ? pc : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const int z1 = __shfl_up_sync(FULL, y1, d), z2 = __shfl_up_sync(FULL, y2, d);
          if (lane >= d) {
            y1 += z1;
            y2 += z2;
          }
        }
        s_excl[tid] = y1 - en.y;
        s_e0[tid] = en.x;
        if (lane == 31) {
          wsum[par][w] = y1;
          wsum[par][W + w] = y2;
        }
        __syncthreads();
        const int tE = lane < W ? wsum[par][lane] : 0;
        const int tP = lane < W ? wsum[par][W + lane] : 0;
        const int epos = run + __reduce_add_sync(FULL, lane < w ? tP : 0) + y2 - pc;
        int inclE = tE;  // lane u: edges of warps 0..u
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const int z = __shfl_up_sync(FULL, inclE, d);
          if (lane >= d) inclE += z;
        }
        const int etot = __shfl_sync(FULL, inclE, 31);
        for (int q0 = 0; q0 < etot; q0 += CT) {
          const int q = q0 + tid;
          const int qc = min(q, etot - 1);  // every lane searches (the shuffles are warp-wide)
          int u = 0;                        // warps whose edges all lie before qc
#pragma unroll
          for (int step = 16; step >= 1; step >>= 1) {
            const int ic = __shfl_sync(FULL, inclE, (u + step - 1) & 31);
            if (ic <= qc) u += step;
          }
          const int base = __shfl_sync(FULL, inclE, (u - 1) & 31);
          const int ql = qc - (u > 0 ? base : 0);
          const int* xs = s_excl + u * 32;
          int j = 0;  // the last range of warp u whose start is <= ql
#pragma unroll
          for (int step = 16; step >= 1; step >>= 1)
            if (xs[j + step] <= ql) j += step;
          const int v = q < etot ? fanin[s_e0[u * 32 + j] + (ql - xs[j])] : -1;
          if (pending) {
            emit(epos);
            pending = false;
          }
          decrement_cl(v, (unsigned)v < (unsigned)n, fanin_start, cnt, nx, cl);
        }
        if (pending) {
          emit(epos);
          pending = false;
        }
        c0 += CT;
        if (c0 < mm) __syncthreads();  // the next chunk reuses s_excl, s_e0 and wsum
      } while (c0 < mm);
    };
    if (!over) {
      // the fanin ranges this CTA collected last level
      expand(m, [&](int k) { return lcur[k]; }, true);
      LV_PHASE(1);
    } else {
      // a list overflowed last level: every CTA emits its own range's pins
      // of this level and expands them, read back from `order`, their
      // fanin ranges from global memory
      int y2 = pc;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int z2 = __shfl_up_sync(FULL, y2, d);
        if (lane >= d) y2 += z2;
      }
      if (lane == 31) wsum[par][W + w] = y2;
      __syncthreads();
      const int tP = lane < W ? wsum[par][W + lane] : 0;
      const int wbP = __reduce_add_sync(FULL, lane < w ? tP : 0);
      const int tt = min(__reduce_add_sync(FULL, tP), n - run);
      emit(run + wbP + y2 - pc);
      __syncthreads();  // this range's slice of `order` is written; wsum is reused
      expand(
          tt,
          [&](int k) {
            const int u = __ldcg(order + run + k);
            const int e0 = fanin_start[u];
            return make_int2(e0, fanin_start[u + 1] - e0);
          },
          false);
    }
    emitted += total;
    if (emitted > n) {  // only reachable with duplicate seeds; stop cleanly
      if (gtid == 0) atomicCAS(&ctl->status, 0, (int)OTG_ERR_INVALID);
      emitted = n;
      break;
    }
    if (gtid == 0) level_ends[L + 1] = emitted;
#ifdef OTG_PHASE_TIMING
    if (tid == 0 && L < 4096) counts[16 + 65536 + L * 16 + r] = (int)(clock64() - _lt0);
#endif
    ++L;
    const int q = q_free;
    q_free = q_now;
    q_now = q_next;
    q_next = q;
    LV_PHASE(2);
  }
  if (gtid == 0) {
    counts[0] = L;
    counts[1] = emitted;
  }
  LV_PHASE_END(counts);
  cl.sync();  // no CTA leaves while another may still read its counts
}

// Dynamic shared memory of the cluster path: both bitmaps (C words each),
// optionally the range's fanin counters (32*C ints), and two lists of at
// least kLstMin fanin ranges (8 bytes each); the lists take what is left of
// kClusterSmemMax.
constexpr size_t kClusterSmemMax = 200 * 1024;
constexpr int kLstMin = kCtMax;
size_t lv_cluster_smem(int C, bool scnt) {
  return (size_t)(2 * C + (scnt ? 32 * C : 0) + 4 * kLstMin) * 4;
}
int lv_lst_cap(int C, bool scnt) {
  return ((int)(kClusterSmemMax / 4) - 2 * C - (scnt ? 32 * C : 0)) / 4;
}

constexpr int kWidths[4] = {128, 256, 512, 1024};
const void* cluster_fn(int wi) {
  switch (wi) {
    case 0: return (const void*)levelize_cluster_kernel<128>;
    case 1: return (const void*)levelize_cluster_kernel<256>;
    case 2: return (const void*)levelize_cluster_kernel<512>;
    default: return (const void*)levelize_cluster_kernel<1024>;
  }
}

struct LvDev {
  int sms = 0;
  int occ = 0;
  bool init = false;
  int max_cluster[4] = {0, 0, 0, 0};  // per CTA width: largest cluster (power of two <= 16) placed
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
    // the cluster path: allow its largest shared memory and 16-CTA clusters,
    // then keep, per CTA width, the largest cluster size the device places
    for (int wi = 0; wi < 4; ++wi) {
      const void* fn = cluster_fn(wi);
      if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kClusterSmemMax) != cudaSuccess ||
          cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
              cudaSuccess)
        continue;
      for (int s = 16; s >= 1 && !x.max_cluster[wi]; s >>= 1) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)s;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(s);
        cfg.blockDim = dim3(kWidths[wi]);
        cfg.dynamicSmemBytes = kClusterSmemMax;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int nc = 0;
        if (cudaOccupancyMaxActiveClusters(&nc, fn, &cfg) == cudaSuccess && nc >= 1)
          x.max_cluster[wi] = s;
      }
    }
    cudaGetLastError();  // a refused attribute or query leaves no sticky error
    x.init = true;
  }
  return x;
}

// The cluster path's shape for an n-pin graph: S CTAs of kWidths[wi]
// threads, each owning 2^cshift bitmap words.  S = 0: the cooperative path.
struct ClPlan {
  int S = 0, wi = 0, cshift = 0;
  bool scnt = false;  // the fanin counters in shared memory
};
// Default: the largest cluster the device places (16 CTAs on B200) of 256
// threads each, for graphs whose ranges then hold at most kClusterMaxWords
// words (about a million pins); larger graphs take the cooperative path,
// which spreads a level over every SM.  OTG_LEVELIZE_CLUSTER=0 turns the
// cluster path off, =1|2|4|8|16 asks for that size; OTG_LEVELIZE_CT=
// 128|256|512|1024 asks for that width (both only where the graph fits and
// the device places the cluster).
constexpr int kClusterMaxWords = 2048;
ClPlan lv_cluster_plan(int n, const LvDev& d) {
  ClPlan p;
  const int nw = std::max(1, (n + 31) / 32);
  p.wi = 1;
  if (const char* e = std::getenv("OTG_LEVELIZE_CT")) {
    const int want = std::atoi(e);
    for (int wi = 0; wi < 4; ++wi)
      if (kWidths[wi] == want) p.wi = wi;
  }
  const int maxc = d.max_cluster[p.wi];
  if (maxc < 1) return ClPlan{};
  int s = maxc;
  if (const char* e = std::getenv("OTG_LEVELIZE_CLUSTER")) {
    const int want = std::atoi(e);
    if (want <= 0) return ClPlan{};
    s = 1;
    while (s < want && s < maxc) s <<= 1;
  } else if ((nw + s - 1) / s > kClusterMaxWords) {
    return ClPlan{};  // large graphs: the whole GPU (the cooperative path)
  }
  int cs = 0;
  while ((1 << cs) * s < nw) ++cs;
  if (lv_cluster_smem(1 << cs, false) > kClusterSmemMax) return ClPlan{};
  p.S = s;
  p.cshift = cs;
  // the counters go on chip where they fit (ranges of up to 32k pins:
  // graphs of about half a million pins); OTG_LEVELIZE_SCNT=0 keeps them in
  // global memory
  p.scnt = lv_cluster_smem(1 << cs, true) <= kClusterSmemMax;
  if (const char* e = std::getenv("OTG_LEVELIZE_SCNT"))
    if (std::atoi(e) == 0) p.scnt = false;
  return p;
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
  const otg::ClPlan pl = otg::lv_cluster_plan(n, d);
  if (pl.S > 0) {
    char* ws = (char*)workspace;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(ws + l.ctl, 0, sizeof(otg::LvCtl), s) != cudaSuccess) return OTG_ERR_CUDA;
    otg::LvCtl* ctl = (otg::LvCtl*)(ws + l.ctl);
    int* cnt = (int*)(ws + l.cnt);
    int cshift = pl.cshift;
    int lst_cap = otg::lv_lst_cap(1 << pl.cshift, pl.scnt);
    int scnt_on = pl.scnt ? 1 : 0;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)pl.S;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(pl.S);
    cfg.blockDim = dim3(otg::kWidths[pl.wi]);
    cfg.dynamicSmemBytes = otg::kClusterSmemMax;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    void* args[] = {&n,          (void*)&fanin_start, (void*)&fanin, (void*)&out_deg,
                    (void*)&frontier0, &first_size, &order, &level, &level_ends, &counts,
                    &ctl,        &cnt,        &cshift,       &lst_cap,  &scnt_on};
    const cudaError_t e = cudaLaunchKernelExC(&cfg, otg::cluster_fn(pl.wi), args);
    otg::count_launch();
    return e == cudaSuccess ? OTG_OK : OTG_ERR_CUDA;
  }
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
