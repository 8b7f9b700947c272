// otg_rc.cu -- RC-net timing on B200: BFS flattening of each net's RC tree
// plus Elmore load / delay / ldelay / impulse for 2 splits x 2 transitions,
// fused into one pass over HBM.
//
// Replaces, from the OpenTimer reference:
//   compute_net_bfs + block_couting_sort   ot/cuda/rct.cu:120-245, ot/cuda/sort.cuh:15-142
//   prepare_res_cap                        ot/cuda/rct.cu:314-359
//   compute_net_timing                     ot/cuda/rct.cu:11-59
//   Rct::update_rc_timing (CPU twin)       ot/timer/net.cpp:101-193
//
// Work is bucketed by net size; every bucket is one persistent launch whose
// CTAs pull nets from a device-side queue (no host round trip, graph
// capturable):
//   * nets of <= 32 nodes: one warp per net, one lane per node, all in
//     registers and shuffles;
//   * larger nets: one CTA per net, staged in shared memory (or, for nets
//     beyond the shared-memory budget, in a per-CTA slice of the caller's
//     workspace, which stays L2-resident).  The tree is processed with
//     log-depth parallel algorithms so that deep chains cost the same as
//     bushy trees: a stable radix sort builds the adjacency, pointer
//     jumping ranks the Euler tour, one scan over the tour yields parent,
//     depth, DFS preorder and subtree sizes, a stable radix sort by depth
//     yields the reference's BFS slots, and Elmore runs as two compensated
//     (float-float) segmented scans up the preorder (subtree sums: load,
//     ldelay) and two down the Euler tour (path sums: delay, beta).
//
// BFS order is bit-exact with the reference: (distance asc, local id desc).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <cstring>

#include "../../include/otg.h"
#include "otg_internal.cuh"

namespace otg {

namespace {

constexpr int NC = 4;
constexpr unsigned FULL = 0xffffffffu;
constexpr int END = -1;

// ------------------------------------------------------------------ args

struct RcArgs {
  int num_nets;
  const int* nodes_start;
  int2* edges;
  const int* roots;
  const float* res;
  const float4* cap;
  int* node2bfs;
  int* pid;
  float4* load;
  float4* delay;
  float4* ldelay;
  float4* impulse;
  const int* sinks_start;
  const int* sink_nodes;
  const float4* driver_slew;
  float4* sink_slew;
  int* status;  // [0] first error code, [1] its net
};

__device__ __forceinline__ void report(const RcArgs& a, int code, int net) {
  if (atomicCAS(a.status, 0, code) == 0) a.status[1] = net;
}

// ------------------------------------------------------- float-float math
// Knuth TwoSum; x += y on (hi, lo) pairs.  No multiplies, so FMA
// contraction cannot change these.
__device__ __forceinline__ void ffadd(float& ah, float& al, float bh, float bl) {
  float s = ah + bh;
  float bb = s - ah;
  float e = (ah - (s - bb)) + (bh - bb);
  e += al + bl;
  ah = s + e;
  al = e - (ah - s);
}

__device__ __forceinline__ float f4get(const float4& v, int j) {
  return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w;
}
__device__ __forceinline__ void f4set(float4& v, int j, float x) {
  if (j == 0) v.x = x; else if (j == 1) v.y = x; else if (j == 2) v.z = x; else v.w = x;
}
__device__ __forceinline__ float4 f4add(float4 a, float4 b) {
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__device__ __forceinline__ float4 f4mul(float4 a, float4 b) {
  return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w);
}
__device__ __forceinline__ float4 f4scale(float4 a, float s) {
  return make_float4(a.x * s, a.y * s, a.z * s, a.w * s);
}
__device__ __forceinline__ float4 shfl4(float4 v, int src) {
  return make_float4(__shfl_sync(FULL, v.x, src), __shfl_sync(FULL, v.y, src),
                     __shfl_sync(FULL, v.z, src), __shfl_sync(FULL, v.w, src));
}

// =====================================================================
// Warp path: nets of <= 32 nodes.  Lane v holds node v and edge v.
// =====================================================================
__device__ void rc_net_warp(const RcArgs& a, int net, int* s_par, int* s_pe) {
  const int lane = threadIdx.x & 31;
  const int b = a.nodes_start[net];
  const int n = a.nodes_start[net + 1] - b;
  const int m = n - 1;
  const int eb = b - net;
  const int root = a.roots[net];
  const bool isnode = lane < n;
  const bool isedge = lane < m;

  int es = 0, et = 0;
  float r = 0.0f;
  if (isedge) {
    int2 e = a.edges[eb + lane];
    es = e.x;
    et = e.y;
    r = a.res[eb + lane];
  }
  float4 cap = isnode ? a.cap[b + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
  const bool bad = (isedge && ((unsigned)es >= (unsigned)n || (unsigned)et >= (unsigned)n)) ||
                   (unsigned)root >= (unsigned)n;
  if (__any_sync(FULL, bad)) {
    if (lane == 0) report(a, OTG_ERR_INVALID, net);
    return;
  }

  // Level-synchronous BFS from the root (depth <= 31).
  constexpr int INF = 1 << 20;
  int dist = (lane == root) ? 0 : INF;
  int my_par = -1, my_child = -1;
  s_par[lane] = -1;
  s_pe[lane] = -1;
  __syncwarp();
  for (int level = 0; level < n; ++level) {
    int ds = __shfl_sync(FULL, dist, es);
    int dt = __shfl_sync(FULL, dist, et);
    int child = -1, par = -1;
    if (isedge) {
      if (ds == level && dt == INF) { child = et; par = es; }
      else if (dt == level && ds == INF) { child = es; par = et; }
    }
    unsigned D = __reduce_or_sync(FULL, child >= 0 ? (1u << child) : 0u);
    if (child >= 0) {
      s_par[child] = par;
      s_pe[child] = lane;
      my_par = par;
      my_child = child;
    }
    if ((D >> lane) & 1u) dist = level + 1;
    if (D == 0u) break;
  }
  __syncwarp();
  const unsigned reached = __ballot_sync(FULL, isnode && dist < INF);
  const unsigned want = (n == 32) ? FULL : ((1u << n) - 1u);
  if (reached != want) {
    if (lane == 0) report(a, OTG_ERR_NOT_TREE, net);
    return;
  }
  int parent = s_par[lane];
  if (lane == root || !isnode) parent = lane;

  // BFS slot: (dist asc, local id desc) -- ot/cuda/sort.cuh:102-121.
  int slot = 0;
  for (int u = 0; u < n; ++u) {
    int du = __shfl_sync(FULL, dist, u);
    slot += (du < dist) || (du == dist && u > lane);
  }
  const int pslot = __shfl_sync(FULL, slot, parent);
  if (isnode) {
    a.node2bfs[b + lane] = slot;
    a.pid[b + slot] = slot - pslot;  // root: 0
  }
  if (isedge) a.edges[eb + lane] = make_int2(my_par, my_child);

  // Ancestor-or-self masks by pointer doubling.
  unsigned M = isnode ? ((1u << lane) | (1u << parent)) : 0u;
  int anc = parent;
  for (int k = 0; k < 5; ++k) {
    unsigned Ma = __shfl_sync(FULL, M, anc);
    int aa = __shfl_sync(FULL, anc, anc);
    M |= Ma;
    anc = aa;
  }
  // pres of node v = resistance of the edge to its parent
  float pres = 0.0f;
  {
    int pe = (isnode && lane != root) ? s_pe[lane] : 0;
    float rr = __shfl_sync(FULL, r, pe);
    pres = (isnode && lane != root) ? rr : 0.0f;
  }
  // load: sum of cap over the subtree (descendants u have bit v in M[u])
  float4 load = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int u = 0; u < n; ++u) {
    unsigned Mu = __shfl_sync(FULL, M, u);
    float4 c = shfl4(cap, u);
    if ((Mu >> lane) & 1u) load = f4add(load, c);
  }
  // delay: sum of pres*load over ancestors-or-self
  float4 w = f4scale(load, pres);
  float4 delay = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int u = 0; u < n; ++u) {
    float4 wu = shfl4(w, u);
    if ((M >> u) & 1u) delay = f4add(delay, wu);
  }
  float4 x = f4mul(cap, delay);
  float4 ldelay = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int u = 0; u < n; ++u) {
    unsigned Mu = __shfl_sync(FULL, M, u);
    float4 c = shfl4(x, u);
    if ((Mu >> lane) & 1u) ldelay = f4add(ldelay, c);
  }
  w = f4scale(ldelay, pres);
  float4 beta = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int u = 0; u < n; ++u) {
    float4 wu = shfl4(w, u);
    if ((M >> u) & 1u) beta = f4add(beta, wu);
  }
  float4 imp = make_float4(fmaf(-delay.x, delay.x, 2.0f * beta.x),
                           fmaf(-delay.y, delay.y, 2.0f * beta.y),
                           fmaf(-delay.z, delay.z, 2.0f * beta.z),
                           fmaf(-delay.w, delay.w, 2.0f * beta.w));
  if (isnode) {
    a.load[b + slot] = load;
    a.delay[b + slot] = delay;
    a.ldelay[b + slot] = ldelay;
    a.impulse[b + slot] = imp;
  }
  if (a.sinks_start) {
    const int s0 = a.sinks_start[net], s1 = a.sinks_start[net + 1];
    const float4 si = a.driver_slew[net];
    for (int k0 = s0; k0 < s1; k0 += 32) {
      int k = k0 + lane;
      int v = k < s1 ? a.sink_nodes[k] : 0;
      bool ok = k < s1 && (unsigned)v < (unsigned)n;
      float4 iv = shfl4(imp, ok ? v : 0);
      if (ok) {
        float4 o;
        o.x = copysignf(sqrtf(si.x * si.x + iv.x), si.x);
        o.y = copysignf(sqrtf(si.y * si.y + iv.y), si.y);
        o.z = copysignf(sqrtf(si.z * si.z + iv.z), si.z);
        o.w = copysignf(sqrtf(si.w * si.w + iv.w), si.w);
        a.sink_slew[k] = o;
      } else if (k < s1) {
        report(a, OTG_ERR_INVALID, net);
      }
    }
  }
}

__global__ void __launch_bounds__(256) rc_warp_kernel(RcArgs a, const int* list,
                                                       const int* count, int* work) {
  __shared__ int s_par[8][32];
  __shared__ int s_pe[8][32];
  const int w = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int cnt = *count;
  while (true) {
    int item = 0;
    if (lane == 0) item = atomicAdd(work, 1);
    item = __shfl_sync(FULL, item, 0);
    if (item >= cnt) break;
    rc_net_warp(a, list[item], s_par[w], s_pe[w]);
    __syncwarp();
  }
}

// =====================================================================
// Block path.
// =====================================================================

// Block-wide exclusive scan of one int per thread.
template <int T>
__device__ __forceinline__ int block_excl_scan(int v, int& total, int* wsum) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  constexpr int W = T / 32;
  int x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int y = __shfl_up_sync(FULL, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < W ? wsum[lane] : 0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      int y = __shfl_up_sync(FULL, s, d);
      if (lane >= d) s += y;
    }
    if (lane < W) wsum[lane] = s;
  }
  __syncthreads();
  const int base = w ? wsum[w - 1] : 0;
  total = wsum[W - 1];
  __syncthreads();
  return base + x - v;
}

// Exclusive scan over `count` items: val(i) gives item i, out(i, prefix, v)
// receives it.  K consecutive items per thread per tile.
template <int T, int K, class ValF, class OutF>
__device__ int block_scan_items(int count, ValF val, OutF out, int* wsum) {
  int carry = 0;
  for (int base = 0; base < count; base += T * K) {
    int v[K];
    int local = 0;
    const int i0 = base + threadIdx.x * K;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      v[k] = (i0 + k < count) ? val(i0 + k) : 0;
      local += v[k];
    }
    int tot;
    int run = carry + block_excl_scan<T>(local, tot, wsum);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (i0 + k < count) out(i0 + k, run, v[k]);
      run += v[k];
    }
    carry += tot;
  }
  return carry;
}

// Stable LSD radix sort of the items 0..N-1 by key(i) (nbits bits, 8 bits
// per pass).  The final order lands in `out` (out[rank] = item); b0/b1 are
// ping-pong buffers of N ints; hist has 256*(T/32) ints.  Each warp owns a
// contiguous range of the current sequence, so ranks inside a warp follow
// sequence order (match_any + popc) and the digit-major scan of per-warp
// counts keeps the sort stable.
template <int T, class KeyF>
__device__ void block_radix_sort(int N, int nbits, KeyF key, int* b0, int* b1, int* out,
                                 int* hist, int* wsum) {
  constexpr int W = T / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int per = ((N + W - 1) / W + 31) & ~31;
  const int passes = nbits <= 0 ? 1 : (nbits + 7) / 8;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    const int* src = (p == 0) ? nullptr : ((p - 1) % 2 == 0 ? b0 : b1);
    int* dst = (p == passes - 1) ? out : (p % 2 == 0 ? b0 : b1);
    for (int i = threadIdx.x; i < 256 * W; i += T) hist[i] = 0;
    __syncthreads();
    // sweep 1: per-warp digit counts
    for (int j = 0; j < per; j += 32) {
      const int idx = w * per + j + lane;
      const bool valid = idx < N;
      const int item = valid ? (src ? src[idx] : idx) : 0;
      const int d = valid ? ((key(item) >> shift) & 255) : (256 + lane);
      const unsigned peers = __match_any_sync(FULL, d);
      const bool leader = valid && (__ffs(peers) - 1 == lane);
      if (leader) hist[d * W + w] += __popc(peers);
      __syncwarp();
    }
    __syncthreads();
    // digit-major exclusive scan of the per-warp counts
    block_scan_items<T, 4>(
        256 * W, [&](int i) { return hist[i]; }, [&](int i, int pre, int) { hist[i] = pre; },
        wsum);
    __syncthreads();
    // sweep 2: place
    for (int j = 0; j < per; j += 32) {
      const int idx = w * per + j + lane;
      const bool valid = idx < N;
      const int item = valid ? (src ? src[idx] : idx) : 0;
      const int d = valid ? ((key(item) >> shift) & 255) : (256 + lane);
      const unsigned peers = __match_any_sync(FULL, d);
      int base = valid ? hist[d * W + w] : 0;
      __syncwarp();
      if (valid) {
        dst[base + __popc(peers & lt)] = item;
        if (__ffs(peers) - 1 == lane) hist[d * W + w] = base + __popc(peers);
      }
      __syncwarp();
    }
    __syncthreads();
  }
}

// Compensated up-sweep over the preorder: x(i) -> L (fp32 inclusive prefix
// inside each thread's 4-position chunk) and Bh/Bl (float-float exclusive
// prefix of the chunks).  The inclusive prefix is I(p) = Bh[p/4] + Bl[p/4]
// + L[p].  Keeping the uncompensated part to <= 4 terms matters: every
// subtree on a long path shares the right end I(n-1), so an error there
// would repeat in every load of the path and add up along its delays.
template <int T, class XF>
__device__ void up_scan(int n, XF x, float4* L, float4* Bh, float4* Bl, float* sm) {
  constexpr int W = T / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  float ch[NC] = {0.f, 0.f, 0.f, 0.f}, cl[NC] = {0.f, 0.f, 0.f, 0.f};  // carry
  float* swh = sm;           // [W][4]
  float* swl = sm + W * NC;  // [W][4]
  for (int base = 0; base < n; base += T * 4) {
    const int q0 = base + threadIdx.x * 4;
    float4 v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = (q0 + k < n) ? x(q0 + k) : make_float4(0.f, 0.f, 0.f, 0.f);
    float eh[NC], el[NC];  // warp-exclusive ff prefix of this thread's chunk
#pragma unroll
    for (int j = 0; j < NC; ++j) {
      float acc = 0.f, h = 0.f, l = 0.f;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float e = f4get(v[k], j);
        acc += e;
        ffadd(h, l, e, 0.f);
        f4set(v[k], j, acc);
      }
      float ih = h, il = l;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const float yh = __shfl_up_sync(FULL, ih, d), yl = __shfl_up_sync(FULL, il, d);
        if (lane >= d) {
          float sh = yh, sl = yl;
          ffadd(sh, sl, ih, il);
          ih = sh;
          il = sl;
        }
      }
      const float xh = __shfl_up_sync(FULL, ih, 1), xl = __shfl_up_sync(FULL, il, 1);
      eh[j] = lane ? xh : 0.f;
      el[j] = lane ? xl : 0.f;
      if (lane == 31) { swh[w * NC + j] = ih; swl[w * NC + j] = il; }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (q0 + k < n) L[q0 + k] = v[k];
    __syncthreads();
    float bh[NC], bl[NC];
#pragma unroll
    for (int j = 0; j < NC; ++j) { bh[j] = ch[j]; bl[j] = cl[j]; }
    for (int u = 0; u < w; ++u)
#pragma unroll
      for (int j = 0; j < NC; ++j) ffadd(bh[j], bl[j], swh[u * NC + j], swl[u * NC + j]);
#pragma unroll
    for (int j = 0; j < NC; ++j) ffadd(bh[j], bl[j], eh[j], el[j]);
    if (q0 < n) {
      Bh[q0 >> 2] = make_float4(bh[0], bh[1], bh[2], bh[3]);
      Bl[q0 >> 2] = make_float4(bl[0], bl[1], bl[2], bl[3]);
    }
    for (int u = 0; u < W; ++u)
#pragma unroll
      for (int j = 0; j < NC; ++j) ffadd(ch[j], cl[j], swh[u * NC + j], swl[u * NC + j]);
    __syncthreads();
  }
}

// Compensated inclusive down-sweep over the Euler tour: x(p) gives the
// signed contribution of tour position p; emit(p, value) receives the
// rounded inclusive prefix at every position.
template <int T, class XF, class EmitF>
__device__ void down_scan(int A, XF x, EmitF emit, float* sm) {
  constexpr int W = T / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  float ch[NC] = {0.f, 0.f, 0.f, 0.f}, cl[NC] = {0.f, 0.f, 0.f, 0.f};
  float* swh = sm;
  float* swl = sm + W * NC;
  for (int base = 0; base < A; base += T * 4) {
    const int q0 = base + threadIdx.x * 4;
    float4 v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = (q0 + k < A) ? x(q0 + k) : make_float4(0.f, 0.f, 0.f, 0.f);
    float ph[4][NC], pl[4][NC];  // thread-local inclusive prefixes
    float eh[NC], el[NC];        // warp-exclusive prefix of the thread
#pragma unroll
    for (int j = 0; j < NC; ++j) {
      float h = 0.f, l = 0.f;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        ffadd(h, l, f4get(v[k], j), 0.f);
        ph[k][j] = h;
        pl[k][j] = l;
      }
      float ih = h, il = l;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        float yh = __shfl_up_sync(FULL, ih, d), yl = __shfl_up_sync(FULL, il, d);
        if (lane >= d) {
          // prefix of earlier lanes goes first
          float sh = yh, sl = yl;
          ffadd(sh, sl, ih, il);
          ih = sh;
          il = sl;
        }
      }
      // exclusive = inclusive - own total: recompute as shuffle of neighbour
      float xh = __shfl_up_sync(FULL, ih, 1), xl = __shfl_up_sync(FULL, il, 1);
      eh[j] = lane ? xh : 0.f;
      el[j] = lane ? xl : 0.f;
      if (lane == 31) { swh[w * NC + j] = ih; swl[w * NC + j] = il; }
    }
    __syncthreads();
    float bh[NC], bl[NC];
#pragma unroll
    for (int j = 0; j < NC; ++j) { bh[j] = ch[j]; bl[j] = cl[j]; }
    for (int u = 0; u < w; ++u)
#pragma unroll
      for (int j = 0; j < NC; ++j) ffadd(bh[j], bl[j], swh[u * NC + j], swl[u * NC + j]);
#pragma unroll
    for (int j = 0; j < NC; ++j) ffadd(bh[j], bl[j], eh[j], el[j]);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (q0 + k < A) {
        float4 o;
#pragma unroll
        for (int j = 0; j < NC; ++j) {
          float h = bh[j], l = bl[j];
          ffadd(h, l, ph[k][j], pl[k][j]);
          f4set(o, j, h + l);
        }
        emit(q0 + k, o);
      }
    }
    for (int u = 0; u < W; ++u)
#pragma unroll
      for (int j = 0; j < NC; ++j) ffadd(ch[j], cl[j], swh[u * NC + j], swl[u * NC + j]);
    __syncthreads();
  }
}

// Range sums of an up_scan.
struct UpPrefix {
  const float4* L;
  const float4* Bh;
  const float4* Bl;
  // range sum over preorder [lo, hi] (inclusive), compensated
  __device__ __forceinline__ float4 range(int lo, int hi) const {
    const int cb = hi >> 2;
    float4 hb = Bh[cb], lb = Bl[cb], Lb = L[hi];
    float4 ha, la, La;
    if (lo > 0) {
      const int ca = (lo - 1) >> 2;
      ha = Bh[ca];
      la = Bl[ca];
      La = L[lo - 1];
    } else {
      ha = la = La = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    float4 o;
#pragma unroll
    for (int j = 0; j < NC; ++j) {
      float h = f4get(hb, j), l = f4get(lb, j);
      ffadd(h, l, -f4get(ha, j), -f4get(la, j));
      ffadd(h, l, f4get(Lb, j) - f4get(La, j), 0.f);
      f4set(o, j, h + l);
    }
    return o;
  }
};

__device__ __forceinline__ unsigned long long lr_pack(int next, int rank) {
  return ((unsigned long long)(unsigned)rank << 32) | (unsigned)next;
}
__device__ __forceinline__ int lr_next(unsigned long long p) { return (int)(unsigned)p; }
__device__ __forceinline__ int lr_rank(unsigned long long p) { return (int)(p >> 32); }

// Block-path per-net workspace layout (see rc_layout_host for the phases).
template <int T>
__device__ void rc_net_block(const RcArgs& a, int net, char* ws, int n, int* sh) {
  const int tid = threadIdx.x;
  const int b = a.nodes_start[net];
  const int m = n - 1, A = 2 * m, eb = b - net;
  const RcLayout lay = rc_layout(n, T);
  int* pre = (int*)(ws + lay.pre);
  int* nap = (int*)(ws + lay.nap);
  int* size = (int*)(ws + lay.size);
  int* nas = (int*)(ws + lay.nas);
  int* tour = (int*)(ws + lay.tour);  // adjacency first, then the tour
  int* posin = (int*)(ws + lay.posin);
  // (next, rank) pairs for list ranking, one 64-bit word each so a pair is
  // always read and written whole (volatile: relaxed, single-copy atomic)
  volatile unsigned long long* lr = (volatile unsigned long long*)(ws + lay.lr);
  int* rb0 = (int*)(ws + lay.lr);  // radix ping-pong, aliases lr
  int* rb1 = rb0 + A;
  int* es = (int*)(ws + lay.es);
  int* et = (int*)(ws + lay.et);
  int* start = (int*)(ws + lay.start);
  int* depth = (int*)(ws + lay.depth);
  int* parent = (int*)(ws + lay.parent);
  int* pedge = (int*)(ws + lay.pedge);
  int* slot = (int*)(ws + lay.slot);
  int* hist = (int*)(ws + lay.hist);
  float* pres = (float*)(ws + lay.pres);
  float4* capp = (float4*)(ws + lay.cap);
  float4* X = (float4*)(ws + lay.X);
  float4* Y = (float4*)(ws + lay.Y);
  float4* L = (float4*)(ws + lay.L);
  float4* Bh = (float4*)(ws + lay.Bh);
  float4* Bl = (float4*)(ws + lay.Bl);
  int* wsum = sh;                  // [W]
  int* s_flag = sh + 32;           // error flag
  int* s_maxd = sh + 33;           // max depth
  float* sm = (float*)(sh + 64);   // [2][W][4] floats
  const int root = a.roots[net];

  // ---- A1: edges, validation, degrees
  if (tid == 0) { *s_flag = ((unsigned)root >= (unsigned)n) ? OTG_ERR_INVALID : 0; *s_maxd = 0; }
  for (int v = tid; v <= n; v += T) start[v] = 0;
  __syncthreads();
  for (int e = tid; e < m; e += T) {
    int2 ed = a.edges[eb + e];
    if ((unsigned)ed.x >= (unsigned)n || (unsigned)ed.y >= (unsigned)n) {
      *s_flag = OTG_ERR_INVALID;
      ed = make_int2(0, 0);
    }
    es[e] = ed.x;
    et[e] = ed.y;
    atomicAdd(&start[ed.x], 1);
    atomicAdd(&start[ed.y], 1);
  }
  __syncthreads();
  if (*s_flag) { if (tid == 0) report(a, *s_flag, net); return; }
  // degree -> offsets; a node without an edge cannot be in a spanning tree
  block_scan_items<T, 4>(
      n + 1, [&](int v) { return v < n ? start[v] : 0; },
      [&](int v, int p, int d) {
        start[v] = p;
        if (v < n && d == 0) *s_flag = OTG_ERR_NOT_TREE;
      },
      wsum);
  __syncthreads();
  if (*s_flag) { if (tid == 0) report(a, *s_flag, net); return; }

  // ---- A3: adjacency = arcs stably sorted by source (arc 2e: s->t, 2e+1: t->s)
  int nbits = 32 - __clz(n - 1);
  block_radix_sort<T>(
      A, nbits, [&](int arc) { return (arc & 1) ? et[arc >> 1] : es[arc >> 1]; }, rb0, rb1,
      tour, hist, wsum);
  for (int j = tid; j < A; j += T) posin[tour[j]] = j;
  __syncthreads();

  // ---- A4: Euler-tour successor; the tour starts at the root's first arc
  for (int arc = tid; arc < A; arc += T) {
    const int v = (arc & 1) ? es[arc >> 1] : et[arc >> 1];  // head
    int k = posin[arc ^ 1] + 1;
    if (k == start[v + 1]) k = start[v];
    int nx = tour[k];
    if (nx == tour[start[root]]) nx = END;  // the arc that closes the tour
    lr[arc] = lr_pack(nx, nx == END ? 0 : 1);
  }
  __syncthreads();

  // ---- A5: list ranking by pointer jumping ((next, rank) read as one pair)
  int rounds = 2;
  while ((1 << rounds) < A) ++rounds;
  for (int r = 0; r < rounds + 1; ++r) {
    for (int arc = tid; arc < A; arc += T) {
      const unsigned long long p = lr[arc];
      if (lr_next(p) != END) {
        const unsigned long long q = lr[lr_next(p)];
        lr[arc] = lr_pack(lr_next(q), lr_rank(p) + lr_rank(q));
      }
    }
    __syncthreads();
  }
  for (int arc = tid; arc < A; arc += T)
    if (lr_next(lr[arc]) != END) *s_flag = OTG_ERR_NOT_TREE;
  for (int v = tid; v < n; v += T) pre[v] = -1;
  __syncthreads();
  if (*s_flag) { if (tid == 0) report(a, *s_flag, net); return; }
  // position in the tour = A-1-rank
  for (int arc = tid; arc < A; arc += T) tour[A - 1 - lr_rank(lr[arc])] = arc;
  __syncthreads();

  // ---- A7: scan of down arcs -> preorder, depth, parent, subtree size
  if (tid == 0) {
    pre[root] = 0;
    nap[0] = root;
    size[0] = n;
    depth[root] = 0;
    parent[root] = root;
    pedge[root] = -1;
  }
  block_scan_items<T, 4>(
      A,
      [&](int p) {
        const int arc = tour[p];
        return (p < A - 1 - lr_rank(lr[arc ^ 1])) ? 1 : 0;
      },
      [&](int p, int ex, int down) {
        if (!down) return;
        const int arc = tour[p];
        const int u = (arc & 1) ? et[arc >> 1] : es[arc >> 1];
        const int v = (arc & 1) ? es[arc >> 1] : et[arc >> 1];
        const int pv = ex + 1;
        if (atomicCAS(&pre[v], -1, pv) != -1 || v == root) { *s_flag = OTG_ERR_NOT_TREE; return; }
        const int d = 2 * pv - p - 1;
        depth[v] = d;
        parent[v] = u;
        pedge[v] = arc >> 1;
        nap[pv] = v;
        size[pv] = ((A - 1 - lr_rank(lr[arc ^ 1])) - p + 1) >> 1;
        atomicMax(s_maxd, d);
      },
      wsum);
  __syncthreads();
  for (int v = tid; v < n; v += T)
    if (pre[v] < 0) *s_flag = OTG_ERR_NOT_TREE;
  __syncthreads();
  if (*s_flag) { if (tid == 0) report(a, *s_flag, net); return; }
  // tour codes for the down-sweeps: +(pre+1) entering a node, -(pre+1) leaving it
  for (int p = tid; p < A; p += T) {
    const int arc = tour[p];
    const bool down = p < A - 1 - lr_rank(lr[arc ^ 1]);
    const int v = down ? ((arc & 1) ? es[arc >> 1] : et[arc >> 1])
                       : ((arc & 1) ? et[arc >> 1] : es[arc >> 1]);
    tour[p] = down ? (pre[v] + 1) : -(pre[v] + 1);
  }
  __syncthreads();

  // ---- A8: BFS slots: stable sort by depth of ids in DESCENDING order
  const int maxd = *s_maxd;
  block_radix_sort<T>(
      n, 32 - __clz(maxd), [&](int j) { return depth[n - 1 - j]; }, rb0, rb1, nas, hist, wsum);
  for (int r = tid; r < n; r += T) {
    const int v = n - 1 - nas[r];
    nas[r] = v;
    slot[v] = r;
  }
  __syncthreads();

  // ---- A9: topology outputs
  for (int v = tid; v < n; v += T) a.node2bfs[b + v] = slot[v];
  for (int r = tid; r < n; r += T) {
    const int v = nas[r];
    a.pid[b + r] = r == 0 ? 0 : r - slot[parent[v]];
  }
  for (int e = tid; e < m; e += T) {
    const int s = es[e], t = et[e];
    a.edges[eb + e] = (pedge[t] == e) ? make_int2(s, t) : make_int2(t, s);
  }
  // ---- A10: resistance to the parent, by preorder
  for (int i = tid; i < n; i += T) pres[i] = i == 0 ? 0.0f : a.res[eb + pedge[nap[i]]];
  __syncthreads();

  // ---- B: Elmore.  cap by preorder.
  for (int i = tid; i < n; i += T) capp[i] = a.cap[b + nap[i]];
  __syncthreads();
  const UpPrefix up{L, Bh, Bl};
  // load (up)
  up_scan<T>(n, [&](int i) { return capp[i]; }, L, Bh, Bl, sm);
  __syncthreads();
  for (int i = tid; i < n; i += T) X[i] = up.range(i, i + size[i] - 1);
  __syncthreads();
  for (int r = tid; r < n; r += T) a.load[b + r] = X[pre[nas[r]]];
  // delay (down): +pres*load entering, - leaving
  if (tid == 0) Y[0] = make_float4(0.f, 0.f, 0.f, 0.f);
  down_scan<T>(
      A,
      [&](int p) {
        const int c = tour[p];
        const int i = (c > 0 ? c : -c) - 1;
        const float s = c > 0 ? pres[i] : -pres[i];
        return f4scale(X[i], s);
      },
      [&](int p, float4 v) {
        const int c = tour[p];
        if (c > 0) Y[c - 1] = v;
      },
      sm);
  __syncthreads();
  for (int r = tid; r < n; r += T) a.delay[b + r] = Y[pre[nas[r]]];
  // ldelay (up): cap*delay over the subtree
  up_scan<T>(n, [&](int i) { return f4mul(capp[i], Y[i]); }, L, Bh, Bl, sm);
  __syncthreads();
  for (int i = tid; i < n; i += T) X[i] = up.range(i, i + size[i] - 1);
  __syncthreads();
  for (int r = tid; r < n; r += T) a.ldelay[b + r] = X[pre[nas[r]]];
  // beta (down) -> impulse = 2*beta - delay^2, kept in L
  if (tid == 0) L[0] = make_float4(0.f, 0.f, 0.f, 0.f);
  down_scan<T>(
      A,
      [&](int p) {
        const int c = tour[p];
        const int i = (c > 0 ? c : -c) - 1;
        const float s = c > 0 ? pres[i] : -pres[i];
        return f4scale(X[i], s);
      },
      [&](int p, float4 v) {
        const int c = tour[p];
        if (c > 0) {
          const float4 d = Y[c - 1];
          L[c - 1] = make_float4(fmaf(-d.x, d.x, 2.0f * v.x), fmaf(-d.y, d.y, 2.0f * v.y),
                                 fmaf(-d.z, d.z, 2.0f * v.z), fmaf(-d.w, d.w, 2.0f * v.w));
        }
      },
      sm);
  __syncthreads();
  for (int r = tid; r < n; r += T) a.impulse[b + r] = L[pre[nas[r]]];
  if (a.sinks_start) {
    const int s0 = a.sinks_start[net], s1 = a.sinks_start[net + 1];
    const float4 si = a.driver_slew[net];
    for (int k = s0 + tid; k < s1; k += T) {
      const int v = a.sink_nodes[k];
      if ((unsigned)v >= (unsigned)n) { report(a, OTG_ERR_INVALID, net); continue; }
      const float4 iv = L[pre[v]];
      float4 o;
      o.x = copysignf(sqrtf(si.x * si.x + iv.x), si.x);
      o.y = copysignf(sqrtf(si.y * si.y + iv.y), si.y);
      o.z = copysignf(sqrtf(si.z * si.z + iv.z), si.z);
      o.w = copysignf(sqrtf(si.w * si.w + iv.w), si.w);
      a.sink_slew[k] = o;
    }
  }
  __syncthreads();
}

template <int T, bool SMEM>
__global__ void __launch_bounds__(T) rc_block_kernel(RcArgs a, const int* list, const int* count,
                                                     int* work, char* gws, size_t ws_stride) {
  extern __shared__ __align__(16) char dsm[];
  __shared__ int sh[64 + 2 * (T / 32) * NC];
  __shared__ int s_item;
  char* ws = SMEM ? dsm : gws + (size_t)blockIdx.x * ws_stride;
  const int cnt = *count;
  while (true) {
    if (threadIdx.x == 0) s_item = atomicAdd(work, 1);
    __syncthreads();
    const int item = s_item;
    __syncthreads();
    if (item >= cnt) break;
    const int net = list[item];
    const int n = a.nodes_start[net + 1] - a.nodes_start[net];
    rc_net_block<T>(a, net, ws, n, sh);
    __syncthreads();
  }
}

// ------------------------------------------------------------ bucketing
__global__ void rc_classify_kernel(int num_nets, const int* nodes_start, int max_net_nodes,
                                   RcClasses cls, int* lists, int* counts, int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  int c = -1;
  if (i < num_nets) {
    const int n = nodes_start[i + 1] - nodes_start[i];
    if (n < 1 || n > max_net_nodes) {
      if (atomicCAS(status, 0, n < 1 ? OTG_ERR_INVALID : OTG_ERR_TOO_LARGE) == 0) status[1] = i;
    } else {
      c = 0;
      while (c < cls.num - 1 && n > cls.nmax[c]) ++c;
    }
  }
  // warp-aggregated append
  const unsigned active = __ballot_sync(FULL, c >= 0);
  const unsigned peers = __match_any_sync(FULL, c);
  if (c >= 0) {
    const int leader = __ffs(peers & active) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&counts[c], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    lists[(size_t)c * num_nets + base + __popc(peers & ((1u << lane) - 1u))] = i;
  }
}

// ------------------------------------------------------------ host side

struct DevInfo {
  int sms = 0;
  int smem_optin = 0;
  bool init = false;
};
DevInfo g_dev[64];

DevInfo& dev_info() {
  int d = 0;
  cudaGetDevice(&d);
  DevInfo& di = g_dev[d & 63];
  if (!di.init) {
    cudaDeviceGetAttribute(&di.sms, cudaDevAttrMultiProcessorCount, d);
    cudaDeviceGetAttribute(&di.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, d);
    di.init = true;
  }
  return di;
}

// Opt-in shared memory left for the static __shared__ arrays of the block
// kernel (sh[], s_item: under 1 KB).
constexpr int kStaticSmemReserve = 2048;

// Size classes: warp path, then block paths in shared memory, then the
// global-workspace path.  T per class is fixed at compile time.
constexpr int kClassT[RcClasses::kMax] = {32, 128, 128, 256, 256, 512, 512};

}  // namespace

// Largest n of the last shared-memory class for a given opt-in budget.
int rc_smem_nmax(int T, int smem_budget) {
  int lo = 33, hi = 1 << 16;
  if (rc_layout(lo, T).total > (uint32_t)smem_budget) return 32;
  while (lo < hi) {
    int mid = (lo + hi + 1) / 2;
    if (rc_layout(mid, T).total <= (uint32_t)smem_budget) lo = mid; else hi = mid - 1;
  }
  return lo;
}

RcClasses rc_classes(int smem_budget) {
  RcClasses c;
  c.num = 7;
  c.nmax[0] = 32;
  c.nmax[1] = 128;
  c.nmax[2] = 256;
  c.nmax[3] = 512;
  c.nmax[4] = 1024;
  c.nmax[5] = std::max(1025, rc_smem_nmax(512, smem_budget));
  c.nmax[6] = 1 << 30;  // global workspace
  return c;
}

// Workspace: [status 64 B][counters 64 B][lists C x N ints][huge slices]
static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// CTAs of the global-workspace path: two per SM, fewer when a slice is so
// large that the slices would exceed 4 GiB.
static int huge_ctas(int sms, size_t stride) {
  const size_t cap = ((size_t)4 << 30) / std::max<size_t>(stride, 1);
  return (int)std::max<size_t>(1, std::min<size_t>((size_t)sms * 2, cap));
}

size_t rc_workspace_bytes(int num_nets, int max_net_nodes, int sms, int smem_budget,
                          size_t* off_lists, size_t* off_huge, size_t* huge_stride) {
  RcClasses c = rc_classes(smem_budget);
  size_t o = 128;
  *off_lists = o;
  o = align256(o + (size_t)c.num * (size_t)std::max(num_nets, 1) * 4);
  *off_huge = o;
  *huge_stride = 0;
  if (max_net_nodes > c.nmax[5]) {
    *huge_stride = align256(rc_layout(max_net_nodes, 512).total);
    o += *huge_stride * (size_t)huge_ctas(sms, *huge_stride);
  }
  return o;
}

otg_status rc_launch(const otg_rc_forest* f, int max_net_nodes, void* workspace,
                     size_t workspace_bytes, cudaStream_t stream) {
  if (!f || !workspace || f->num_nets < 0 || max_net_nodes < 1) return OTG_ERR_INVALID;
  if (f->num_nets == 0) return OTG_OK;
  if (!f->nodes_start || !f->edges || !f->roots || !f->edges_res || !f->nodes_cap ||
      !f->node2bfs || !f->pid || !f->load || !f->delay || !f->ldelay || !f->impulse)
    return OTG_ERR_INVALID;
  const bool sinks = f->sinks_start != nullptr;
  if (sinks && (!f->sink_nodes || !f->driver_slew || !f->sink_slew)) return OTG_ERR_INVALID;
  DevInfo& di = dev_info();
  const int budget = di.smem_optin - kStaticSmemReserve;
  size_t off_lists, off_huge, stride;
  const size_t need = rc_workspace_bytes(f->num_nets, max_net_nodes, di.sms, budget, &off_lists,
                                         &off_huge, &stride);
  if (workspace_bytes < need) return OTG_ERR_WORKSPACE;
  char* ws = (char*)workspace;
  int* status = (int*)ws;
  int* counters = (int*)(ws + 64);  // [0..7] counts, [8..15] work
  int* lists = (int*)(ws + off_lists);
  const RcClasses cls = rc_classes(budget);

  if (cudaMemsetAsync(ws, 0, 128, stream) != cudaSuccess) return OTG_ERR_CUDA;
  RcArgs a;
  a.num_nets = f->num_nets;
  a.nodes_start = f->nodes_start;
  a.edges = (int2*)f->edges;
  a.roots = f->roots;
  a.res = f->edges_res;
  a.cap = (const float4*)f->nodes_cap;
  a.node2bfs = f->node2bfs;
  a.pid = f->pid;
  a.load = (float4*)f->load;
  a.delay = (float4*)f->delay;
  a.ldelay = (float4*)f->ldelay;
  a.impulse = (float4*)f->impulse;
  a.sinks_start = sinks ? f->sinks_start : nullptr;
  a.sink_nodes = f->sink_nodes;
  a.driver_slew = (const float4*)f->driver_slew;
  a.sink_slew = (float4*)f->sink_slew;
  a.status = status;

  rc_classify_kernel<<<(f->num_nets + 255) / 256, 256, 0, stream>>>(
      f->num_nets, f->nodes_start, max_net_nodes, cls, lists, counters, status);
  count_launch();
  const int N = f->num_nets;
  // Largest nets first so the long tail overlaps the small ones.
  auto L = [&](int c) { return lists + (size_t)c * N; };
  int* work = counters + 8;
  // huge (global workspace)
  if (max_net_nodes > cls.nmax[5]) {
    rc_block_kernel<512, false><<<huge_ctas(di.sms, stride), 512, 0, stream>>>(
        a, L(6), counters + 6, work + 6, ws + off_huge, stride);
    count_launch();
  }
  // shared-memory classes, big to small
  struct K { int c; int T; };
  const int cmax[7] = {32, 128, 256, 512, 1024, cls.nmax[5], 0};
  for (int c = 5; c >= 1; --c) {
    if (max_net_nodes <= cmax[c - 1]) continue;
    const int nmax = std::min(cmax[c], max_net_nodes);
    const int T = kClassT[c];
    const size_t smem = rc_layout(nmax, T).total;
    int occ = 1;
    cudaError_t err = cudaSuccess;
#define LAUNCH_BLOCK(TT)                                                                     \
  do {                                                                                       \
    auto kern = rc_block_kernel<TT, true>;                                                   \
    err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
    if (err == cudaSuccess)                                                                  \
      err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, TT, smem);             \
    if (err == cudaSuccess) {                                                                \
      occ = std::max(occ, 1);                                                                \
      kern<<<di.sms * occ, TT, smem, stream>>>(a, L(c), counters + c, work + c, nullptr, 0); \
      count_launch();                                                                        \
    }                                                                                        \
  } while (0)
    if (T == 128) LAUNCH_BLOCK(128);
    else if (T == 256) LAUNCH_BLOCK(256);
    else LAUNCH_BLOCK(512);
#undef LAUNCH_BLOCK
    if (err != cudaSuccess) {
      cudaGetLastError();  // do not leave the error for the caller's next call
      return OTG_ERR_CUDA;
    }
  }
  rc_warp_kernel<<<di.sms * 8, 256, 0, stream>>>(a, L(0), counters + 0, work + 0);
  count_launch();
  if (cudaGetLastError() != cudaSuccess) return OTG_ERR_CUDA;
  return OTG_OK;
}

}  // namespace otg

extern "C" {

otg_status otg_rc_workspace_size(int32_t num_nets, int32_t max_net_nodes, size_t* bytes) {
  if (!bytes || num_nets < 0 || max_net_nodes < 1) return OTG_ERR_INVALID;
  otg::DevInfo& di = otg::dev_info();
  if (di.sms <= 0) return OTG_ERR_CUDA;
  size_t a, b, c;
  *bytes = otg::rc_workspace_bytes(num_nets, max_net_nodes, di.sms,
                                   di.smem_optin - otg::kStaticSmemReserve, &a, &b, &c);
  return OTG_OK;
}

otg_status otg_rc_timing(const otg_rc_forest* forest, int32_t max_net_nodes, void* workspace,
                         size_t workspace_bytes, otg_stream_t stream) {
  return otg::rc_launch(forest, max_net_nodes, workspace, workspace_bytes, (cudaStream_t)stream);
}

otg_status otg_rc_status(const void* workspace, otg_stream_t stream, int32_t* bad_net) {
  if (!workspace) return OTG_ERR_INVALID;
  int h[2] = {0, -1};
  if (cudaMemcpyAsync(h, workspace, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream) !=
          cudaSuccess ||
      cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
    return OTG_ERR_CUDA;
  if (bad_net) *bad_net = h[0] ? h[1] : -1;
  return (otg_status)h[0];
}

}  // extern "C"
