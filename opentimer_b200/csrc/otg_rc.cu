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
//     yields the reference's BFS slots, and Elmore runs as two exact int64
//     fixed-point scans up the preorder (subtree sums: load, ldelay) and two
//     down the Euler tour (path sums: delay, beta).
//
// BFS order is bit-exact with the reference: (distance asc, local id desc).
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "../../include/otg.h"
#include "otg_internal.cuh"

namespace otg {

namespace {

constexpr unsigned FULL = 0xffffffffu;
namespace cg = cooperative_groups;

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

// One launch's work: all nets of forest a0 (nets == items == null), a
// device list of nets of a0 (nets), or a device list of (forest, net)
// pairs over the device array `forests` (items).  The list lengths come
// from device memory so one captured graph serves every batch.
struct RcJob {
  RcArgs a0;
  const RcArgs* forests;
  const int* nets;
  const int2* items;
  const int* num_dev;  // device count for nets/items
  int num;             // count when neither list is given
};

__device__ __forceinline__ int job_count(const RcJob& j) {
  return (j.nets || j.items) ? *j.num_dev : j.num;
}
__device__ __forceinline__ void job_item(const RcJob& j, int k, int& f, int& net) {
  if (j.items) {
    const int2 it = j.items[k];
    f = it.x;
    net = it.y;
  } else {
    f = 0;
    net = j.nets ? j.nets[k] : k;
  }
}
__device__ __forceinline__ const RcArgs& job_forest(const RcJob& j, int f) {
  return j.items ? j.forests[f] : j.a0;
}

// ------------------------------------------------------------ float4 math
// Sink slew sign(si) * sqrt(si^2 + impulse) (ot/timer/net.cpp:280-283).
// The square and the sum are rounded separately, as in the reference's
// host code; explicit intrinsics keep the compiler from fusing them into an
// FMA in some kernels and not in others, so every path and tile shape
// gives the same bits.
__device__ __forceinline__ float sink_slew1(float si, float imp) {
  const float r = sqrtf(__fadd_rn(__fmul_rn(si, si), imp));
  return si < 0.0f ? -r : r;
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
        o.x = sink_slew1(si.x, iv.x);
        o.y = sink_slew1(si.y, iv.y);
        o.z = sink_slew1(si.z, iv.z);
        o.w = sink_slew1(si.w, iv.w);
        a.sink_slew[k] = o;
      } else if (k < s1) {
        report(a, OTG_ERR_INVALID, net);
      }
    }
  }
}

__global__ void __launch_bounds__(256) rc_warp_kernel(RcJob job, const int* list,
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
    int f, net;
    job_item(job, list[item], f, net);
    rc_net_warp(job_forest(job, f), net, s_par[w], s_pe[w]);
    __syncwarp();
  }
}

// Optional per-phase cycle accounting (build with -DOTG_PHASE_TIMING; the
// product build compiles it out).  Thread 0 of each CTA adds the clock64()
// delta of every phase of the block path into otg_phase_cycles[].
#ifdef OTG_PHASE_TIMING
}  // namespace
__device__ unsigned long long otg_phase_cycles[32];
namespace {
#define PHASE_BEGIN() long long _ph_t = clock64()
#define PHASE(k)                                                              \
  do {                                                                        \
    if (threadIdx.x == 0) {                                                   \
      const long long _t = clock64();                                         \
      atomicAdd(&otg_phase_cycles[k], (unsigned long long)(_t - _ph_t));      \
      _ph_t = _t;                                                             \
    }                                                                         \
  } while (0)
#else
#define PHASE_BEGIN() \
  do {                \
  } while (0)
#define PHASE(k) \
  do {           \
  } while (0)
#endif

// =====================================================================
// Block path: one CTA per net, 16-bit indices in shared memory (32-bit in
// the global-workspace slices).  Phases:
//   A1-A2  edges -> degrees -> adjacency offsets (validates ids, degrees)
//   A3     adjacency: atomic fill, then each list sorted by arc id so the
//          Euler tour is deterministic (a stable radix sort by source
//          replaces this when some node has degree > 32)
//   A4     Euler-tour successor of every arc; the tour starts at the
//          root's first arc
//   A5     tour ranking: hashed splitter arcs cut the tour into short
//          sublists, one thread walks each sublist, pointer jumping ranks
//          the splitters; every arc lands at its tour position
//   A6     one scan over the tour: down arcs give preorder, depth,
//          parent, parent edge and subtree size of every node
//   A7     BFS slots: stable radix sort by depth of the ids in descending
//          order (the reference's (dist asc, id desc) rule)
//   A8     topology outputs (node2bfs, pid, directed edges) and the
//          parent resistance by preorder
//   B      Elmore, one corner pair at a time: load and ldelay as exact
//          int64 fixed-point range sums over the preorder, delay and beta
//          as exact int64 fixed-point prefix sums over the signed tour.
// =====================================================================

template <class Ix> struct IxT;
template <> struct IxT<uint16_t> {
  using S = int16_t;
  static constexpr unsigned NONE = 0xFFFFu;
};
template <> struct IxT<int> {
  using S = int;
  static constexpr unsigned NONE = 0xFFFFFFFFu;
};

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

// Warp-inclusive int64 scan of two values; ex gets the warp-exclusive prefix.
__device__ __forceinline__ void warp_i64_scan2(long long (&v)[2], long long (&ex)[2]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const long long y = __shfl_up_sync(FULL, v[j], d);
      if (lane >= d) v[j] += y;
    }
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const long long t = __shfl_up_sync(FULL, v[j], 1);
    ex[j] = lane ? t : 0;
  }
}

// Block part of a tile scan: per-warp exclusive bases and the tile total
// from the warps' inclusive totals (held by lane 31).  shl holds 4*W+2
// int64.  Ends after the second barrier; the caller syncs before reuse.
template <int T>
__device__ __forceinline__ void tile_i64_bases(const long long (&v)[2], long long (&wb)[2],
                                               long long (&tt)[2], long long* shl) {
  constexpr int W = T / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 31) { shl[2 * w] = v[0]; shl[2 * w + 1] = v[1]; }
  __syncthreads();
  if (w == 0) {
    long long x[2], ex[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) x[j] = lane < W ? shl[2 * lane + j] : 0;
    warp_i64_scan2(x, ex);
    if (lane < W) { shl[2 * W + 2 * lane] = ex[0]; shl[2 * W + 2 * lane + 1] = ex[1]; }
    if (lane == W - 1) { shl[4 * W] = x[0]; shl[4 * W + 1] = x[1]; }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    wb[j] = shl[2 * W + 2 * w + j];
    tt[j] = shl[4 * W + j];
  }
}

// ---- thread groups of the block path.  A net of the block path is run by
// a group of threads: one CTA (CtaGroup), or -- for nets above the shared-
// memory classes -- a thread-block cluster of S CTAs acting as one virtual
// block over the net's global-memory workspace slice (ClusterGroup).  The
// group gives each thread its rank, its barrier and an exclusive scan; the
// net's shared scalars (error flag, maximum depth, sweep maxima) live in
// the shared memory of the group's first CTA.
template <int T>
struct CtaGroup {
  int* flag = nullptr;
  int* maxd = nullptr;
  unsigned* smx = nullptr;
  __device__ static constexpr int vt() { return T; }
  __device__ int rank() const { return (int)threadIdx.x; }
  __device__ void sync() const { __syncthreads(); }
  __device__ int excl_scan(int v, int& total, int* wsum) const {
    return block_excl_scan<T>(v, total, wsum);
  }
  __device__ void i64_bases(const long long (&v)[2], long long (&wb)[2], long long (&tt)[2],
                            long long* shl) const {
    tile_i64_bases<T>(v, wb, tt, shl);
  }
};

template <int T>
struct ClusterGroup {
  int S = 1, r = 0;         // CTAs in the cluster, this CTA's rank
  int* flag = nullptr;      // in rank 0's shared memory
  int* maxd = nullptr;
  unsigned* smx = nullptr;
  long long* xch = nullptr;  // this CTA's exchange slot [2] (its own shared memory)
  __device__ int vt() const { return S * T; }
  __device__ int rank() const { return r * T + (int)threadIdx.x; }
  // The cluster barrier orders the workspace writes of every CTA (release
  // at arrive, acquire at wait); the fence after it also keeps each SM from
  // serving a later read of the workspace from a line it cached before.
  __device__ void sync() const {
    cg::this_cluster().sync();
    __threadfence();
  }
  // the CTAs' totals of a pair of values: this CTA's exclusive base and the
  // group total (two cluster barriers: publish, then free the slot again)
  __device__ void cta_bases(long long t0, long long t1, long long (&base)[2],
                            long long (&tot)[2]) const {
    const cg::cluster_group cl = cg::this_cluster();
    if (threadIdx.x == 0) {
      xch[0] = t0;
      xch[1] = t1;
    }
    cl.sync();
    const int lane = threadIdx.x & 31;
    long long x0 = 0, x1 = 0;
    if (lane < S) {
      const long long* o = cl.map_shared_rank(xch, lane);
      x0 = o[0];
      x1 = o[1];
    }
    long long b0 = lane < r ? x0 : 0, b1 = lane < r ? x1 : 0;
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
      x0 += __shfl_xor_sync(FULL, x0, d);
      x1 += __shfl_xor_sync(FULL, x1, d);
      b0 += __shfl_xor_sync(FULL, b0, d);
      b1 += __shfl_xor_sync(FULL, b1, d);
    }
    base[0] = b0;
    base[1] = b1;
    tot[0] = x0;
    tot[1] = x1;
    cl.sync();
  }
  __device__ int excl_scan(int v, int& total, int* wsum) const {
    int t_cta;
    const int e = block_excl_scan<T>(v, t_cta, wsum);
    long long base[2], tot[2];
    cta_bases(t_cta, 0, base, tot);
    total = (int)tot[0];
    return (int)base[0] + e;
  }
  __device__ void i64_bases(const long long (&v)[2], long long (&wb)[2], long long (&tt)[2],
                            long long* shl) const {
    long long cw[2], ct[2];
    tile_i64_bases<T>(v, cw, ct, shl);
    __syncthreads();  // shl is reused by the next tile only after every warp read it
    long long base[2], tot[2];
    cta_bases(ct[0], ct[1], base, tot);
    wb[0] = base[0] + cw[0];
    wb[1] = base[1] + cw[1];
    tt[0] = tot[0];
    tt[1] = tot[1];
  }
};

// Exclusive scan over `count` items: val(i) gives item i, out(i, prefix, v)
// receives it.  K consecutive items per thread per tile.  Returns the total.
template <int K, class G, class ValF, class OutF>
__device__ int group_scan_items(const G& g, int count, ValF val, OutF out, int* wsum) {
  int carry = 0;
  const int VT = g.vt();
  for (int base = 0; base < count; base += VT * K) {
    int v[K];
    int local = 0;
    const int i0 = base + g.rank() * K;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      v[k] = (i0 + k < count) ? val(i0 + k) : 0;
      local += v[k];
    }
    int tot;
    int run = carry + g.excl_scan(local, tot, wsum);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (i0 + k < count) out(i0 + k, run, v[k]);
      run += v[k];
    }
    carry += tot;
  }
  return carry;
}
template <int T, int K, class ValF, class OutF>
__device__ int block_scan_items(int count, ValF val, OutF out, int* wsum) {
  return group_scan_items<K>(CtaGroup<T>{}, count, val, out, wsum);
}

// Stable LSD radix sort of the items 0..N-1 by key(i) (nbits bits,
// rc_radix_bits(T) bits per pass) over the group's threads.  The final
// order lands in `out` (out[rank] = item); b0/b1 are ping-pong buffers of N
// entries; hist holds (1 << rc_radix_bits(T)) * (the group's warps) ints.
// Each warp owns a contiguous range of the current sequence, so ranks
// inside a warp follow sequence order (match_any + popc) and the
// digit-major scan of the per-warp counts keeps the sort stable.
template <int T, class G, class Ix, class KeyF>
__device__ void group_radix_sort(const G& g, int N, int nbits, KeyF key, Ix* b0, Ix* b1, Ix* out,
                                 int* hist, int* wsum) {
  const int VT = g.vt(), W = VT / 32;
  const int lane = threadIdx.x & 31, w = g.rank() >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int per = ((N + W - 1) / W + 31) & ~31;
  constexpr int DB = rc_radix_bits(T);
  if (nbits < 1) nbits = 1;
  const int passes = (nbits + DB - 1) / DB;
  for (int p = 0; p < passes; ++p) {
    const int shift = DB * p;
    const int db = min(DB, nbits - shift);
    const int nb = 1 << db;
    const unsigned mask = (unsigned)nb - 1u;
    const Ix* src = (p == 0) ? nullptr : ((p - 1) % 2 == 0 ? b0 : b1);
    Ix* dst = (p == passes - 1) ? out : (p % 2 == 0 ? b0 : b1);
    for (int i = g.rank(); i < nb * W; i += VT) hist[i] = 0;
    g.sync();
    for (int j = 0; j < per; j += 32) {
      const int idx = w * per + j + lane;
      const bool valid = idx < N;
      const int item = valid ? (src ? (int)src[idx] : idx) : 0;
      const int d = valid ? (int)(((unsigned)key(item) >> shift) & mask) : (256 + lane);
      const unsigned peers = __match_any_sync(FULL, d);
      if (valid && (__ffs(peers) - 1 == lane)) hist[d * W + w] += __popc(peers);
      __syncwarp();
    }
    g.sync();
    group_scan_items<4>(
        g, nb * W, [&](int i) { return hist[i]; }, [&](int i, int pre, int) { hist[i] = pre; },
        wsum);
    g.sync();
    for (int j = 0; j < per; j += 32) {
      const int idx = w * per + j + lane;
      const bool valid = idx < N;
      const int item = valid ? (src ? (int)src[idx] : idx) : 0;
      const int d = valid ? (int)(((unsigned)key(item) >> shift) & mask) : (256 + lane);
      const unsigned peers = __match_any_sync(FULL, d);
      const int base = valid ? hist[d * W + w] : 0;
      __syncwarp();
      if (valid) {
        dst[base + __popc(peers & lt)] = (Ix)item;
        if (__ffs(peers) - 1 == lane) hist[d * W + w] = base + __popc(peers);
      }
      __syncwarp();
    }
    g.sync();
  }
}
template <int T, class Ix, class KeyF>
__device__ void block_radix_sort(int N, int nbits, KeyF key, Ix* b0, Ix* b1, Ix* out, int* hist,
                                 int* wsum) {
  group_radix_sort<T>(CtaGroup<T>{}, N, nbits, key, b0, b1, out, hist, wsum);
}

__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return make_float2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ float2 f2scale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// ------------------------------------------------ exact fixed-point sums
// Every fp32 term x of a sweep is mapped to the integer rint(x * 2^s), with
// one power of two per net, corner and sweep chosen from n * max|x| so that
// no partial sum reaches 2^62.  int64 sums of those integers are exact, so
// a subtree sum taken as a difference of two prefixes has no cancellation
// error and no result depends on the order of the terms -- the tour may
// visit children in any order and every output is still bit-reproducible.
// Each term is rounded once to a grid of 2^-s (relative to n * max|x| that
// is 2^-61), each result once back to fp32.

__device__ __forceinline__ float pow2f(int e) { return __int_as_float((e + 127) << 23); }

// 2^s and 2^-s for terms with |x| <= mx over n positions.
__device__ __forceinline__ void fx_scale(float mx, int n, float& up, float& dn) {
  const float bound = mx * (float)n;
  int s = 0;
  if (bound > 0.f) {
    // bound < 2^e with e from the exponent field; s leaves one bit of margin
    const int e = ((__float_as_int(bound) >> 23) & 0xff) - 126;
    s = min(max(61 - e, -126), 126);
  }
  up = pow2f(s);
  dn = pow2f(-s);
}
__device__ __forceinline__ long long to_fx(float x, float up) { return __float2ll_rn(x * up); }
__device__ __forceinline__ float from_fx(long long v, float dn) { return __ll2float_rn(v) * dn; }

// Up-sweep over n preorder slots for one corner pair: Ip[p] = exact
// fixed-point inclusive prefix of x(0..p).  K slots per thread per tile.
template <int K, class G, class XF>
__device__ void up_scan_fx(const G& g, int n, XF x, const float (&up)[2], longlong2* Ip,
                           long long* shl) {
  long long carry[2] = {0, 0};
  const int VT = g.vt();
  for (int base = 0; base < n; base += VT * K) {
    const int q0 = base + g.rank() * K;
    long long loc[K][2];
    long long acc[2] = {0, 0};
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (q0 + k < n) {
        const float2 v = x(q0 + k);
        acc[0] += to_fx(v.x, up[0]);
        acc[1] += to_fx(v.y, up[1]);
      }
      loc[k][0] = acc[0];
      loc[k][1] = acc[1];
    }
    long long ex[2], wb[2], tt[2];
    warp_i64_scan2(acc, ex);
    g.i64_bases(acc, wb, tt, shl);
    const long long b0 = carry[0] + wb[0] + ex[0], b1 = carry[1] + wb[1] + ex[1];
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (q0 + k < n) Ip[rc_pad16(q0 + k)] = make_longlong2(b0 + loc[k][0], b1 + loc[k][1]);
    carry[0] += tt[0];
    carry[1] += tt[1];
    g.sync();
  }
}

// Sum over preorder slots [lo, hi] of an up_scan_fx, back in fp32.
__device__ __forceinline__ float2 up_range_fx(const longlong2* Ip, int lo, int hi,
                                              const float (&dn)[2]) {
  longlong2 h = Ip[rc_pad16(hi)];
  if (lo > 0) {
    const longlong2 l = Ip[rc_pad16(lo - 1)];
    h.x -= l.x;
    h.y -= l.y;
  }
  return make_float2(from_fx(h.x, dn[0]), from_fx(h.y, dn[1]));
}

// Inclusive prefix over A tour slots for one corner pair: x(p) is the
// signed term of slot p; emit(p, v0, v1) receives the exact fixed-point
// prefix (converted by the callee only where it is used).
template <int K, class G, class XF, class EmitF>
__device__ void down_scan_fx(const G& g, int A, XF x, const float (&up)[2], EmitF emit,
                             long long* shl) {
  long long carry[2] = {0, 0};
  const int VT = g.vt();
  for (int base = 0; base < A; base += VT * K) {
    const int q0 = base + g.rank() * K;
    long long loc[K][2];
    long long acc[2] = {0, 0};
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (q0 + k < A) {
        const float2 v = x(q0 + k);
        acc[0] += to_fx(v.x, up[0]);
        acc[1] += to_fx(v.y, up[1]);
      }
      loc[k][0] = acc[0];
      loc[k][1] = acc[1];
    }
    long long ex[2], wb[2], tt[2];
    warp_i64_scan2(acc, ex);
    g.i64_bases(acc, wb, tt, shl);
    const long long b0 = carry[0] + wb[0] + ex[0], b1 = carry[1] + wb[1] + ex[1];
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (q0 + k < A) emit(q0 + k, b0 + loc[k][0], b1 + loc[k][1]);
    carry[0] += tt[0];
    carry[1] += tt[1];
    g.sync();
  }
}

// Per-corner maxima of non-negative terms, gathered into smx[0..1] (float
// bits, which order like unsigned ints for non-negative floats).
__device__ __forceinline__ void max2_accumulate(float2 v, float (&m)[2]) {
  m[0] = fmaxf(m[0], fabsf(v.x));
  m[1] = fmaxf(m[1], fabsf(v.y));
}
__device__ __forceinline__ void max2_commit(const float (&m)[2], unsigned* smx) {
  const unsigned a = __reduce_max_sync(FULL, __float_as_uint(m[0]));
  const unsigned c = __reduce_max_sync(FULL, __float_as_uint(m[1]));
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&smx[0], a);
    atomicMax(&smx[1], c);
  }
}

__device__ __forceinline__ unsigned long long sl_pack(unsigned next, unsigned acc) {
  return ((unsigned long long)acc << 32) | next;
}
__device__ __forceinline__ unsigned sl_next(unsigned long long p) { return (unsigned)p; }
__device__ __forceinline__ unsigned sl_acc(unsigned long long p) { return (unsigned)(p >> 32); }

// Splitter arcs of the tour ranking: the first arc and ~1 in kSplit<<sel
// others, chosen by a hash of the arc id so that runs of the tour (for
// example the up arcs of a long path, which have consecutive odd ids)
// cannot avoid them.
__device__ __forceinline__ bool is_splitter(int arc, int sel, int first) {
  unsigned h = (unsigned)arc * 0x9E3779B1u;
  h ^= h >> 15;
  h *= 0x85EBCA77u;
  h ^= h >> 13;
  return arc == first || (h & (((unsigned)kSplit << sel) - 1u)) == 0u;
}

template <int T, int K, class Ix, class G>
__device__ void rc_net_block(const RcArgs& a, int net, char* ws, int n, int* sh, long long* shl,
                             const G& g) {
  using S = typename IxT<Ix>::S;
  constexpr unsigned NONE = IxT<Ix>::NONE;
  const int tid = g.rank();
  const int VT = g.vt();
  const int b = a.nodes_start[net];
  const int m = n - 1, A = 2 * m, eb = b - net;
  const RcLayout lay = rc_layout(n, T, K, (int)sizeof(Ix));
  Ix* pre = (Ix*)(ws + lay.pre);
  Ix* nap = (Ix*)(ws + lay.nap);
  Ix* size = (Ix*)(ws + lay.size);
  Ix* nas = (Ix*)(ws + lay.nas);
  Ix* tour = (Ix*)(ws + lay.tour);  // adjacency, then the tour
  S* code = (S*)(ws + lay.tour);    // then the signed tour codes
  float* pres = (float*)(ws + lay.pres);
  Ix* es = (Ix*)(ws + lay.es);
  Ix* et = (Ix*)(ws + lay.et);
  int* ends = (int*)(ws + lay.ends);
  Ix* posin = (Ix*)(ws + lay.posin);
  Ix* sub = (Ix*)(ws + lay.sub);
  Ix* off = (Ix*)(ws + lay.off);
  Ix* spl = (Ix*)(ws + lay.spl);
  Ix* splarc = (Ix*)(ws + lay.splarc);
  volatile unsigned long long* sl = (volatile unsigned long long*)(ws + lay.sl);
  Ix* depth = (Ix*)(ws + lay.depth);
  Ix* parent = (Ix*)(ws + lay.parent);
  Ix* pedge = (Ix*)(ws + lay.pedge);
  Ix* slot = (Ix*)(ws + lay.slot);
  Ix* r2 = (Ix*)(ws + lay.r2);  // succ, then subtree size by tour slot, then radix buffers
  int* hist = (int*)(ws + lay.hist);
  float2* X = (float2*)(ws + lay.X);
  float2* Y = (float2*)(ws + lay.Y);
  longlong2* Ip = (longlong2*)(ws + lay.Ip);
  int* wsum = sh;          // [W] this CTA's warp totals
  int* s_flag = g.flag;    // error code
  int* s_maxd = g.maxd;    // max depth
  unsigned* smx = g.smx;   // [8] per-sweep maxima (float bits)
  const int root = a.roots[net];
  auto src = [&](int arc) -> int { return (arc & 1) ? (int)et[arc >> 1] : (int)es[arc >> 1]; };
  auto dst = [&](int arc) -> int { return (arc & 1) ? (int)es[arc >> 1] : (int)et[arc >> 1]; };
  auto fail = [&]() -> bool {
    g.sync();
    const int f = *s_flag;
    if (f && tid == 0) report(a, f, net);
    return f != 0;
  };
  PHASE_BEGIN();

  // ---- A1: edges, validation, degrees
  if (tid == 0) {
    *s_flag = ((unsigned)root >= (unsigned)n) ? OTG_ERR_INVALID : 0;
    *s_maxd = 0;
  }
  for (int v = tid; v < n; v += VT) ends[v] = 0;
  g.sync();
  for (int e = tid; e < m; e += VT) {
    int2 ed = a.edges[eb + e];
    if ((unsigned)ed.x >= (unsigned)n || (unsigned)ed.y >= (unsigned)n) {
      *s_flag = OTG_ERR_INVALID;
      ed = make_int2(0, 0);
    }
    es[e] = (Ix)ed.x;
    et[e] = (Ix)ed.y;
    atomicAdd(&ends[ed.x], 1);
    atomicAdd(&ends[ed.y], 1);
  }
  if (fail()) return;
  PHASE(0);
  // ---- A2: degree -> begin offsets; a node without an edge is no tree node
  group_scan_items<K>(
        g,
      n, [&](int v) { return ends[v]; },
      [&](int v, int p, int d) {
        ends[v] = p;
        if (d == 0) *s_flag = OTG_ERR_NOT_TREE;
      },
      wsum);
  if (fail()) return;
  PHASE(1);
  // ---- A3: adjacency lists by atomic fill.  The order inside a list only
  // decides the tour's child order, which no output depends on (the BFS
  // slots follow (depth, id), the Elmore sums are exact).  After this, node
  // v's arcs are tour[begin(v) .. ends[v]).
  for (int arc = tid; arc < A; arc += VT) tour[atomicAdd(&ends[src(arc)], 1)] = (Ix)arc;
  g.sync();
  PHASE(2);
  // ---- A4: Euler-tour successor: after (u->v) comes v's next arc after (v->u)
  for (int j = tid; j < A; j += VT) posin[tour[j]] = (Ix)j;
  g.sync();
  const int first = (int)tour[root ? ends[root - 1] : 0];
  for (int arc = tid; arc < A; arc += VT) {
    const int v = dst(arc);
    int k = (int)posin[arc ^ 1] + 1;
    if (k == ends[v]) k = v ? ends[v - 1] : 0;
    const int nx = (int)tour[k];
    r2[arc] = nx == first ? (Ix)NONE : (Ix)nx;
  }
  g.sync();
  PHASE(3);
  // ---- A5: tour ranking by sublists
  int sel = 0, ns = 0;
  while (true) {
    ns = group_scan_items<K>(
        g,
        A, [&](int arc) { return is_splitter(arc, sel, first) ? 1 : 0; },
        [&](int arc, int p, int f) {
          sub[arc] = (Ix)NONE;
          if (f) {
            spl[arc] = (Ix)p;
            if (p < (int)lay.ns_cap) splarc[p] = (Ix)arc;
          }
        },
        wsum);
    if (ns <= (int)lay.ns_cap) break;
    ++sel;  // uniform: every thread saw the same total
  }
  g.sync();
  for (int s = tid; s < ns; s += VT) {
    int cur = (int)splarc[s];
    unsigned o = 0, next = 0xFFFFFFFFu;
    for (int step = 0; step < A; ++step) {
      sub[cur] = (Ix)s;
      off[cur] = (Ix)o;
      ++o;
      const unsigned nx = (unsigned)r2[cur];
      if (nx == NONE) break;
      if (is_splitter((int)nx, sel, first)) { next = (unsigned)spl[nx]; break; }
      cur = (int)nx;
    }
    sl[s] = sl_pack(next, o);
  }
  g.sync();
  {
    int rounds = 1;
    while ((1 << rounds) < ns) ++rounds;
    for (int r = 0; r <= rounds; ++r) {
      for (int s = tid; s < ns; s += VT) {
        const unsigned long long p = sl[s];
        if (sl_next(p) != 0xFFFFFFFFu) {
          const unsigned long long q = sl[sl_next(p)];
          sl[s] = sl_pack(sl_next(q), sl_acc(p) + sl_acc(q));
        }
      }
      g.sync();
    }
  }
  for (int s = tid; s < ns; s += VT)
    if (sl_next(sl[s]) != 0xFFFFFFFFu) *s_flag = OTG_ERR_NOT_TREE;
  for (int arc = tid; arc < A; arc += VT)
    if ((unsigned)sub[arc] == NONE) *s_flag = OTG_ERR_NOT_TREE;
  if (tid == 0 && sl_acc(sl[spl[first]]) != (unsigned)A) *s_flag = OTG_ERR_NOT_TREE;
  if (fail()) return;
  // place every arc; remember each down arc's subtree size by tour slot
  for (int arc = tid; arc < A; arc += VT) {
    const int p = A - (int)sl_acc(sl[sub[arc]]) + (int)off[arc];
    const int q = A - (int)sl_acc(sl[sub[arc ^ 1]]) + (int)off[arc ^ 1];
    if ((unsigned)p >= (unsigned)A) { *s_flag = OTG_ERR_NOT_TREE; continue; }
    tour[p] = (Ix)arc;
    r2[p] = (Ix)(p < q ? (q - p + 1) >> 1 : 0);
  }
  if (fail()) return;
  PHASE(4);
  // ---- A6: preorder, depth, parent, subtree size from the down arcs
  for (int v = tid; v < n; v += VT) pre[v] = (Ix)NONE;
  g.sync();
  if (tid == 0) {
    pre[root] = 0;
    nap[0] = (Ix)root;
    size[0] = (Ix)n;
    depth[root] = 0;
    parent[root] = (Ix)root;
    pedge[root] = (Ix)NONE;
  }
  g.sync();
  group_scan_items<K>(
        g,
      A, [&](int p) { return r2[p] != 0 ? 1 : 0; },
      [&](int p, int ex, int down) {
        if (!down) return;
        const int arc = (int)tour[p];
        const int v = dst(arc), pv = ex + 1;
        const int d = 2 * pv - p - 1;
        pre[v] = (Ix)pv;
        depth[v] = (Ix)d;
        parent[v] = (Ix)src(arc);
        pedge[v] = (Ix)(arc >> 1);
        nap[pv] = (Ix)v;
        size[pv] = r2[p];
        atomicMax(s_maxd, d);
      },
      wsum);
  g.sync();
  for (int v = tid; v < n; v += VT) {
    const unsigned pv = (unsigned)pre[v];
    if (pv == NONE || (int)nap[pv] != v) *s_flag = OTG_ERR_NOT_TREE;
  }
  if (fail()) return;
  for (int p = tid; p < A; p += VT) {
    const int arc = (int)tour[p];
    const bool down = r2[p] != 0;
    const int v = down ? dst(arc) : src(arc);
    code[p] = (S)(down ? (int)pre[v] + 1 : -((int)pre[v] + 1));
  }
  g.sync();
  PHASE(5);
  // ---- A7: BFS slots: stable sort by depth of the ids in DESCENDING order
  {
    Ix* rs0 = r2;
    Ix* rs1 = r2 + n;
    group_radix_sort<T>(
        g,
        n, 32 - __clz(max(*s_maxd, 1)), [&](int j) { return (int)depth[n - 1 - j]; }, rs0, rs1,
        nas, hist, wsum);
    for (int r = tid; r < n; r += VT) {
      const int v = n - 1 - (int)nas[r];
      nas[r] = (Ix)v;
      slot[v] = (Ix)r;
    }
    g.sync();
  }
  PHASE(6);
  // ---- A8: topology outputs, parent resistance by preorder (read in edge
  // order, coalesced, and placed at the child's preorder slot).  From here
  // on nas[r] holds the preorder slot of BFS slot r (bpre).
  Ix* bpre = nas;
  for (int v = tid; v < n; v += VT) a.node2bfs[b + v] = (int)slot[v];
  for (int r = tid; r < n; r += VT) {
    const int v = (int)nas[r];
    a.pid[b + r] = r == 0 ? 0 : r - (int)slot[parent[v]];
    bpre[r] = pre[v];
  }
  if (tid == 0) pres[0] = 0.0f;
  for (int e = tid; e < m; e += VT) {
    const int s = (int)es[e], t = (int)et[e];
    const bool down = (int)pedge[t] == e;  // t is the child of edge e
    a.edges[eb + e] = down ? make_int2(s, t) : make_int2(t, s);
    pres[(int)pre[down ? t : s]] = a.res[eb + e];
  }
  g.sync();
  PHASE(7);

  // ---- B: Elmore, one corner pair at a time (corners 2cp, 2cp+1), with
  // exact fixed-point sums (see fx_scale).  The maximum term of every sweep
  // is gathered in the loop before it (smx) to set its scale.  The pair's
  // caps are read from HBM once, in id order, into Y by preorder; after the
  // load sweep they move to the unused half of each Ip slot, where the
  // ldelay sweep reads them last (and overwrites them in place).
  const float2* cap2 = (const float2*)a.cap;
  float2* capI = (float2*)Ip;  // cap of preorder slot i at capI[2 * rc_pad16(i)]
  for (int cp = 0; cp < 2; ++cp) {
    float2* out;
    float up[2], dn[2], m[2];
    auto scale = [&](int k) {
      fx_scale(__uint_as_float(smx[2 * k]), n, up[0], dn[0]);
      fx_scale(__uint_as_float(smx[2 * k + 1]), n, up[1], dn[1]);
    };
    if (tid < 8) smx[tid] = 0u;
    g.sync();
    m[0] = m[1] = 0.f;
    for (int j = tid; j < n; j += VT) {
      const float2 c = cap2[2 * (size_t)(b + j) + cp];
      Y[rc_pad8((int)pre[j])] = c;
      max2_accumulate(c, m);
    }
    max2_commit(m, smx + 0);
    g.sync();
    // load (up): cap summed over the subtree
    scale(0);
    up_scan_fx<K>(g, n, [&](int i) { return Y[rc_pad8(i)]; }, up, Ip, shl);
    m[0] = m[1] = 0.f;
    for (int i = tid; i < n; i += VT) {
      const float2 v = up_range_fx(Ip, i, i + (int)size[i] - 1, dn);
      X[rc_pad8(i)] = v;
      max2_accumulate(f2scale(v, pres[i]), m);
    }
    max2_commit(m, smx + 2);
    g.sync();
    out = (float2*)a.load;
    for (int r = tid; r < n; r += VT) out[2 * (size_t)(b + r) + cp] = X[rc_pad8(bpre[r])];
    for (int i = tid; i < n; i += VT) capI[2 * rc_pad16(i)] = Y[rc_pad8(i)];  // Ip is free until the ldelay sweep
    g.sync();
    PHASE(8);
    // delay (down): +pres*load entering a node, - leaving it
    scale(1);
    if (tid == 0) Y[rc_pad8(0)] = make_float2(0.f, 0.f);
    down_scan_fx<K>(
        g,
        A,
        [&](int p) {
          const int c = (int)code[p];
          const int i = (c > 0 ? c : -c) - 1;
          return f2scale(X[rc_pad8(i)], c > 0 ? pres[i] : -pres[i]);
        },
        up,
        [&](int p, long long v0, long long v1) {
          const int c = (int)code[p];
          if (c > 0) Y[rc_pad8(c - 1)] = make_float2(from_fx(v0, dn[0]), from_fx(v1, dn[1]));
        },
        shl);
    m[0] = m[1] = 0.f;
    out = (float2*)a.delay;
    for (int r = tid; r < n; r += VT) {
      const int i = (int)bpre[r];
      const float2 d = Y[rc_pad8(i)];
      out[2 * (size_t)(b + r) + cp] = d;
      max2_accumulate(f2mul(capI[2 * rc_pad16(i)], d), m);
    }
    max2_commit(m, smx + 4);
    g.sync();
    PHASE(9);
    // ldelay (up): cap*delay over the subtree
    scale(2);
    // each thread reads its own slots' caps before it writes their sums
    up_scan_fx<K>(g, n, [&](int i) { return f2mul(capI[2 * rc_pad16(i)], Y[rc_pad8(i)]); }, up, Ip, shl);
    m[0] = m[1] = 0.f;
    for (int i = tid; i < n; i += VT) {
      const float2 v = up_range_fx(Ip, i, i + (int)size[i] - 1, dn);
      X[rc_pad8(i)] = v;
      max2_accumulate(f2scale(v, pres[i]), m);
    }
    max2_commit(m, smx + 6);
    g.sync();
    out = (float2*)a.ldelay;
    for (int r = tid; r < n; r += VT) out[2 * (size_t)(b + r) + cp] = X[rc_pad8(bpre[r])];
    PHASE(10);
    // beta (down) -> impulse = 2*beta - delay^2, kept where Ip was
    scale(3);
    float2* imp = (float2*)Ip;
    if (tid == 0) imp[2 * rc_pad16(0)] = make_float2(0.f, 0.f);
    down_scan_fx<K>(
        g,
        A,
        [&](int p) {
          const int c = (int)code[p];
          const int i = (c > 0 ? c : -c) - 1;
          return f2scale(X[rc_pad8(i)], c > 0 ? pres[i] : -pres[i]);
        },
        up,
        [&](int p, long long v0, long long v1) {
          const int c = (int)code[p];
          if (c > 0) {
            const float2 d = Y[rc_pad8(c - 1)];
            imp[2 * rc_pad16(c - 1)] = make_float2(fmaf(-d.x, d.x, 2.0f * from_fx(v0, dn[0])),
                                     fmaf(-d.y, d.y, 2.0f * from_fx(v1, dn[1])));
          }
        },
        shl);
    out = (float2*)a.impulse;
    for (int r = tid; r < n; r += VT) out[2 * (size_t)(b + r) + cp] = imp[2 * rc_pad16(bpre[r])];
    if (a.sinks_start) {
      const int s0 = a.sinks_start[net], s1 = a.sinks_start[net + 1];
      const float2 si = ((const float2*)a.driver_slew)[2 * (size_t)net + cp];
      float2* so = (float2*)a.sink_slew;
      for (int k = s0 + tid; k < s1; k += VT) {
        const int v = a.sink_nodes[k];
        if ((unsigned)v >= (unsigned)n) { report(a, OTG_ERR_INVALID, net); continue; }
        const float2 iv = imp[2 * rc_pad16(pre[v])];
        so[2 * (size_t)k + cp] = make_float2(sink_slew1(si.x, iv.x), sink_slew1(si.y, iv.y));
      }
    }
    g.sync();
    PHASE(11);
  }
}

#include "otg_rc_tile.cuh"

// Shared-memory bytes of a block-class net of n nodes with T threads.
__host__ __device__ inline uint32_t rc_smem_bytes(int n, int T, int K, bool tile) {
  return tile ? rc_tile_layout(n, T).total : rc_layout(n, T, K, 2).total;
}

// `few`: a class of at most this many items is left to the cluster kernel
// (the huge-net class; 0 elsewhere).
template <int T, int K, class Ix, bool SMEM, bool TILE = false>
__global__ void __launch_bounds__(T) rc_block_kernel(RcJob job, const int* list, const int* count,
                                                     int* work, char* gws, size_t ws_stride,
                                                     int few) {
  extern __shared__ __align__(16) char dsm[];
  __shared__ int sh[96];
  __shared__ long long shl[4 * (T / 32) + 4];
  __shared__ int s_item[2];
  __shared__ RcArgs s_args;  // the current net's forest
  char* ws = SMEM ? dsm : gws + (size_t)blockIdx.x * ws_stride;
  const int cnt = *count;
  if (cnt <= few) return;
  while (true) {
    if (threadIdx.x == 0) {
      const int item = atomicAdd(work, 1);
      s_item[0] = item;
      if (item < cnt) {
        int f, net;
        job_item(job, list[item], f, net);
        s_item[1] = net;
        s_args = job_forest(job, f);
      }
    }
    __syncthreads();
    const int item = s_item[0], net = s_item[1];
    __syncthreads();
    if (item >= cnt) break;
    const int n = s_args.nodes_start[net + 1] - s_args.nodes_start[net];
    if constexpr (TILE) rc_net_tile<T>(s_args, net, ws, n, sh, shl);
    else rc_net_block<T, K, Ix>(s_args, net, ws, n, sh, shl,
                                CtaGroup<T>{sh + 32, sh + 33, (unsigned*)(sh + 40)});
    __syncthreads();
  }
}

// Nets above the shared-memory classes, one thread-block cluster per net:
// the cluster's S CTAs run rc_net_block as ONE virtual block of S*T
// threads over the cluster's workspace slice (32-bit indices), with the
// cluster barrier between phases and the CTAs' scan totals exchanged
// through distributed shared memory.  Items go to the clusters in turn
// (cluster c takes items c, c + C, c + 2C, ...), so every CTA of a cluster
// walks the same items without a shared fetch.  A class of more than
// `few` items is left to the one-CTA-per-net kernel (many huge nets keep
// every SM busy on their own; a few finish sooner on clusters).
template <int T, int K>
__global__ void __launch_bounds__(T) rc_cluster_kernel(RcJob job, const int* list,
                                                       const int* count, char* gws,
                                                       size_t ws_stride, int few) {
  __shared__ int sh[96];
  __shared__ long long shl[4 * (T / 32) + 4];
  __shared__ long long xch[2];
  __shared__ RcArgs s_args;  // the current net's forest
  const cg::cluster_group cl = cg::this_cluster();
  const int S = (int)cl.num_blocks();
  const int cid = (int)blockIdx.x / S, ncl = (int)gridDim.x / S;
  char* ws = gws + (size_t)cid * ws_stride;
  ClusterGroup<T> g;
  g.S = S;
  g.r = (int)cl.block_rank();
  g.flag = cl.map_shared_rank(sh + 32, 0);
  g.maxd = cl.map_shared_rank(sh + 33, 0);
  g.smx = (unsigned*)cl.map_shared_rank(sh + 40, 0);
  g.xch = xch;
  const int cnt = *count;
  if (cnt > few) return;  // uniform: no CTA has touched another's memory
  for (int item = cid; item < cnt; item += ncl) {
    if (threadIdx.x == 0) {
      int f, net;
      job_item(job, list[item], f, net);
      s_args = job_forest(job, f);
      sh[34] = net;
    }
    __syncthreads();
    const int net = sh[34];
    const int n = s_args.nodes_start[net + 1] - s_args.nodes_start[net];
    rc_net_block<T, K, int>(s_args, net, ws, n, sh, shl, g);
    g.sync();  // the slice, s_args and rank 0's scalars are reused by the next item
  }
}

// ------------------------------------------------------------ bucketing
__global__ void rc_classify_kernel(RcJob job, int cap, int max_net_nodes, RcClasses cls,
                                   int* lists, int* counts, int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int num = min(job_count(job), cap);
  int c = -1;
  if (i < num) {
    int f, net;
    job_item(job, i, f, net);
    const RcArgs& a = job_forest(job, f);
    const int n = (unsigned)net < (unsigned)a.num_nets
                      ? a.nodes_start[net + 1] - a.nodes_start[net] : 0;
    if (n < 1 || n > max_net_nodes) {
      if (atomicCAS(status, 0, n < 1 ? OTG_ERR_INVALID : OTG_ERR_TOO_LARGE) == 0) status[1] = i;
    } else {
      c = 0;
      while (c < cls.num - 1 && n > cls.nmax[c]) ++c;
    }
  }
  if (i == 0 && job_count(job) > cap && atomicCAS(status, 0, OTG_ERR_WORKSPACE) == 0)
    status[1] = -1;
  // warp-aggregated append of the item index
  const unsigned active = __ballot_sync(FULL, c >= 0);
  const unsigned peers = __match_any_sync(FULL, c);
  if (c >= 0) {
    const int leader = __ffs(peers & active) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&counts[c], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    lists[(size_t)c * cap + base + __popc(peers & ((1u << lane) - 1u))] = i;
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

// Size classes.  Class 0: the warp path (nets of <= 32 nodes; its
// lane-per-node scheme fixes that bound).  Classes 1..6: one CTA per net in
// shared memory (16-bit indices); their upper bounds and tile shapes (T
// threads, K scan items per thread) come from the device's tuning.
// Class 7: nets beyond the last block class, in per-CTA slices of the
// workspace (32-bit indices, 512 x 8).
struct Shape {
  int T, K;
};
// The compiled block-class shapes (launch_shape dispatches on the index).
constexpr Shape kShapeSet[] = {{64, 4},  {64, 8},  {128, 4}, {128, 8}, {256, 2},  {256, 4},
                               {256, 8}, {512, 2}, {512, 4}, {512, 8}, {1024, 2}, {1024, 4}};
constexpr int kNumShapes = (int)(sizeof(kShapeSet) / sizeof(kShapeSet[0]));
constexpr int kBlockClasses = 6;

int shape_index(int T, int K) {
  for (int s = 0; s < kNumShapes; ++s)
    if (kShapeSet[s].T == T && kShapeSet[s].K == K) return s;
  return -1;
}

}  // namespace

// The block path in use: the edge-wise tile kernel (otg_rc_tile.cuh), or
// with OTG_RC_LEGACY set in the environment the earlier adjacency-list
// kernel (kept for comparison while the tile kernel is measured).
bool rc_use_tile() {
  static const bool tile = std::getenv("OTG_RC_LEGACY") == nullptr;
  return tile;
}

// Largest n whose 16-bit block layout fits the shared-memory budget.
int rc_smem_nmax(int T, int K, int smem_budget) {
  const bool tile = rc_use_tile();
  int lo = 33, hi = 32767;
  if (rc_smem_bytes(lo, T, K, tile) > (uint32_t)smem_budget) return 32;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (rc_smem_bytes(mid, T, K, tile) <= (uint32_t)smem_budget) lo = mid; else hi = mid - 1;
  }
  return lo;
}

namespace {

// Block-class tuning of one device: `num` classes, ascending upper bounds,
// a kShapeSet index each.  Every tuning gives the same outputs (the sums
// are exact, the BFS order is fixed); only the speed differs.
struct RcTune {
  int num = 0;
  int nmax[kBlockClasses] = {};
  int shape[kBlockClasses] = {};
};

RcTune default_tune(int smem_budget) {
  RcTune t;
  const int bounds[kBlockClasses - 1] = {128, 256, 512, 1024, 2048};
  const Shape shapes[kBlockClasses] = {{64, 4}, {64, 8}, {128, 8}, {256, 4}, {256, 8}, {1024, 4}};
  t.num = kBlockClasses;
  for (int c = 0; c < kBlockClasses; ++c) {
    t.shape[c] = shape_index(shapes[c].T, shapes[c].K);
    t.nmax[c] = c < kBlockClasses - 1 ? bounds[c] : 0;
  }
  t.nmax[kBlockClasses - 1] =
      std::max(bounds[kBlockClasses - 2] + 1, rc_smem_nmax(shapes[kBlockClasses - 1].T,
                                                           shapes[kBlockClasses - 1].K, smem_budget));
  return t;
}

bool tune_ok(const RcTune& t, int smem_budget) {
  if (t.num < 1 || t.num > kBlockClasses) return false;
  int prev = 32;
  for (int c = 0; c < t.num; ++c) {
    if (t.shape[c] < 0 || t.shape[c] >= kNumShapes || t.nmax[c] <= prev) return false;
    const Shape sh = kShapeSet[t.shape[c]];
    if (rc_smem_bytes(t.nmax[c], sh.T, sh.K, rc_use_tile()) > (uint32_t)smem_budget) return false;
    prev = t.nmax[c];
  }
  return true;
}

// Device-visible class bounds of a tuning: class c takes nets with
// nmax[c-1] < n <= nmax[c]; unused block classes are empty ranges.
RcClasses classes_of(const RcTune& t) {
  RcClasses c;
  c.num = RcClasses::kMax;
  c.nmax[0] = 32;
  for (int k = 1; k <= kBlockClasses; ++k) c.nmax[k] = t.nmax[std::min(k, t.num) - 1];
  c.nmax[RcClasses::kMax - 1] = 1 << 30;
  return c;
}

std::mutex g_tune_mu;
RcTune g_tune[64];
bool g_tune_set[64] = {};

RcTune current_tune(int smem_budget) {
  int d = 0;
  cudaGetDevice(&d);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (!g_tune_set[d & 63]) {
    g_tune[d & 63] = default_tune(smem_budget);
    g_tune_set[d & 63] = true;
  }
  return g_tune[d & 63];
}

void set_tune(const RcTune& t) {
  int d = 0;
  cudaGetDevice(&d);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[d & 63] = t;
  g_tune_set[d & 63] = true;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// CTAs of the global-workspace path: two per SM, fewer when a slice is so
// large that the slices would exceed 4 GiB.
int huge_ctas(int sms, size_t stride) {
  const size_t cap = ((size_t)4 << 30) / std::max<size_t>(stride, 1);
  return (int)std::max<size_t>(1, std::min<size_t>((size_t)sms * 2, cap));
}

// The huge-net path: one CTA per net, and clusters of S CTAs of 512
// threads per net.  Both are launched; the device-side count of huge nets
// picks one: clusters for at most kClusterNetsPerCluster nets per cluster,
// one CTA per net for more.  S defaults to 8 (the portable cluster size),
// capped by what the device places; OTG_RC_HUGE_CLUSTER=2|4|8|16 asks for
// another size, =1 turns the clusters off.
constexpr int kHugeT = 512, kHugeK = 8;
constexpr int kClusterNetsPerCluster = 2;
struct HugePlan {
  int S = 1;            // CTAs per cluster (1: no cluster launch)
  int clusters = 0;     // clusters launched, one workspace slice each
  size_t stride_c = 0;  // bytes per cluster slice
  int ctas = 0;         // CTAs of the one-CTA-per-net launch, one slice each
  size_t stride = 0;    // bytes per slice of that launch
  size_t bytes() const { return stride * (size_t)ctas + stride_c * (size_t)clusters; }
};

int max_clusters(int S) {  // clusters of S CTAs the device holds at once (0: none)
  static std::mutex mu;
  static int cache[64][5];
  static bool done[64][5];
  int d = 0;
  cudaGetDevice(&d);
  int si = 0;
  while ((1 << si) < S && si < 4) ++si;
  std::lock_guard<std::mutex> lk(mu);
  if (!done[d & 63][si]) {
    auto kern = rc_cluster_kernel<kHugeT, kHugeK>;
    int nc = 0;
    if (S > 8) cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)S;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(S);
    cfg.blockDim = dim3(kHugeT);
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (cudaOccupancyMaxActiveClusters(&nc, (const void*)kern, &cfg) != cudaSuccess) nc = 0;
    cudaGetLastError();
    cache[d & 63][si] = nc;
    done[d & 63][si] = true;
  }
  return cache[d & 63][si];
}

HugePlan huge_plan(int max_net_nodes, int sms) {
  HugePlan h;
  h.stride = align256(rc_layout(max_net_nodes, kHugeT, kHugeK, 4).total);
  h.ctas = huge_ctas(sms, h.stride);
  int S = 8;
  if (const char* e = std::getenv("OTG_RC_HUGE_CLUSTER")) S = std::atoi(e);
  int s2 = 1;
  while (s2 * 2 <= std::min(std::max(S, 1), 16)) s2 *= 2;
  S = s2;
  int ncl = 0;
  while (S > 1 && (ncl = max_clusters(S)) < 1) S /= 2;
  if (S > 1) {
    h.S = S;
    h.stride_c = align256(rc_layout(max_net_nodes, kHugeT, kHugeK, 4, S).total);
    const size_t cap = ((size_t)4 << 30) / std::max<size_t>(h.stride_c, 1);
    h.clusters = (int)std::max<size_t>(1, std::min<size_t>((size_t)ncl, cap));
  }
  return h;
}

}  // namespace

// Workspace: [status 64 B][counters 64 B][lists C x N ints][huge slices]
// (the slices only when some net may exceed the tuning's last block class)
size_t rc_workspace_bytes_for(const RcTune& t, int num_nets, int max_net_nodes, int sms,
                              size_t* off_lists, size_t* off_huge, size_t* huge_stride) {
  const RcClasses c = classes_of(t);
  size_t o = 128;
  *off_lists = o;
  o = align256(o + (size_t)c.num * (size_t)std::max(num_nets, 1) * 4);
  *off_huge = o;
  *huge_stride = 0;
  if (max_net_nodes > c.nmax[6]) {
    const HugePlan h = huge_plan(max_net_nodes, sms);
    *huge_stride = h.stride;
    o += h.bytes();
  }
  return o;
}

size_t rc_workspace_bytes(int num_nets, int max_net_nodes, int sms, int smem_budget,
                          size_t* off_lists, size_t* off_huge, size_t* huge_stride) {
  return rc_workspace_bytes_for(current_tune(smem_budget), num_nets, max_net_nodes, sms,
                                off_lists, off_huge, huge_stride);
}

namespace {

template <int T, int K>
cudaError_t launch_smem_class(const RcJob& job, const int* list, int* count, int* work, int nmax,
                              int sms, cudaStream_t stream) {
  const bool tile = rc_use_tile();
  auto kern = tile ? rc_block_kernel<T, K, uint16_t, true, true> : rc_block_kernel<T, K, uint16_t, true>;
  const size_t smem = rc_smem_bytes(nmax, T, K, tile);
  // The attribute is always set to the same (largest) value, so threads
  // launching with different nmax never lower it under one another.
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         dev_info().smem_optin - kStaticSmemReserve);
  int occ = 1;
  if (err == cudaSuccess) err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, T, smem);
  if (err != cudaSuccess) return err;
  occ = std::max(occ, 1);
  kern<<<sms * occ, T, smem, stream>>>(job, list, count, work, nullptr, 0, 0);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_shape(int s, const RcJob& job, const int* list, int* count, int* work,
                         int nmax, int sms, cudaStream_t st) {
  switch (s) {
    case 0: return launch_smem_class<64, 4>(job, list, count, work, nmax, sms, st);
    case 1: return launch_smem_class<64, 8>(job, list, count, work, nmax, sms, st);
    case 2: return launch_smem_class<128, 4>(job, list, count, work, nmax, sms, st);
    case 3: return launch_smem_class<128, 8>(job, list, count, work, nmax, sms, st);
    case 4: return launch_smem_class<256, 2>(job, list, count, work, nmax, sms, st);
    case 5: return launch_smem_class<256, 4>(job, list, count, work, nmax, sms, st);
    case 6: return launch_smem_class<256, 8>(job, list, count, work, nmax, sms, st);
    case 7: return launch_smem_class<512, 2>(job, list, count, work, nmax, sms, st);
    case 8: return launch_smem_class<512, 4>(job, list, count, work, nmax, sms, st);
    case 9: return launch_smem_class<512, 8>(job, list, count, work, nmax, sms, st);
    case 10: return launch_smem_class<1024, 2>(job, list, count, work, nmax, sms, st);
    case 11: return launch_smem_class<1024, 4>(job, list, count, work, nmax, sms, st);
    default: return cudaErrorInvalidValue;
  }
}
static_assert(kNumShapes == 12, "launch_shape covers every kShapeSet entry");

RcArgs make_args(const otg_rc_forest* f, int* status) {
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
  a.sinks_start = f->sinks_start;
  a.sink_nodes = f->sink_nodes;
  a.driver_slew = (const float4*)f->driver_slew;
  a.sink_slew = (float4*)f->sink_slew;
  a.status = status;
  return a;
}

bool forest_ok(const otg_rc_forest* f) {
  if (!f || f->num_nets < 0) return false;
  if (f->num_nets == 0) return true;
  if (!f->nodes_start || !f->edges || !f->roots || !f->edges_res || !f->nodes_cap ||
      !f->node2bfs || !f->pid || !f->load || !f->delay || !f->ldelay || !f->impulse)
    return false;
  if (f->sinks_start && (!f->sink_nodes || !f->driver_slew || !f->sink_slew)) return false;
  return true;
}

}  // namespace

// Launches the fused pass over the items of `job` (at most `cap` of them).
// The workspace starts with [status 64 B][counters 64 B]; its status word is
// where a.status should point for single-forest jobs.
// `tune` (optional) overrides the device's tuning.
otg_status rc_launch_job(RcJob job, int cap, int max_net_nodes, void* workspace,
                         size_t workspace_bytes, cudaStream_t stream, const RcFork* fork = nullptr,
                         const RcTune* tune = nullptr) {
  if (!workspace || cap < 0 || max_net_nodes < 1) return OTG_ERR_INVALID;
  DevInfo& di = dev_info();
  const int budget = di.smem_optin - kStaticSmemReserve;
  const RcTune tn = tune ? *tune : current_tune(budget);
  size_t off_lists, off_huge, stride;
  const size_t need = rc_workspace_bytes_for(tn, std::max(cap, 1), max_net_nodes, di.sms,
                                             &off_lists, &off_huge, &stride);
  if (workspace_bytes < need) return OTG_ERR_WORKSPACE;
  char* ws = (char*)workspace;
  int* status = (int*)ws;
  int* counters = (int*)(ws + 64);  // [0..7] counts, [8..15] work
  int* lists = (int*)(ws + off_lists);
  const RcClasses cls = classes_of(tn);
  if (cudaMemsetAsync(ws, 0, 128, stream) != cudaSuccess) {
    cudaGetLastError();
    return OTG_ERR_CUDA;
  }
  if (cap == 0) return OTG_OK;
  rc_classify_kernel<<<(cap + 255) / 256, 256, 0, stream>>>(job, cap, max_net_nodes, cls, lists,
                                                            counters, status);
  count_launch();
  auto L = [&](int c) { return lists + (size_t)c * cap; };
  int* work = counters + 8;
  cudaError_t err = cudaGetLastError();
  // With a fork, the class launches go round-robin over the caller's
  // stream and the side streams (joined back below), so the classes run
  // side by side instead of one after another.
  const int nside = fork ? std::min(fork->n, RcFork::kMax) : 0;
  int nth = 0;
  auto next_stream = [&]() -> cudaStream_t {
    const int k = nth++ % (nside + 1);
    return k == 0 ? stream : fork->side[k - 1];
  };
  if (nside > 0 && err == cudaSuccess) {
    err = cudaEventRecord(fork->fork, stream);
    for (int i = 0; i < nside && err == cudaSuccess; ++i)
      err = cudaStreamWaitEvent(fork->side[i], fork->fork, 0);
  }
  // Largest nets first so the long tail overlaps the small ones.
  if (err == cudaSuccess && max_net_nodes > cls.nmax[6]) {
    const HugePlan h = huge_plan(max_net_nodes, di.sms);
    const int few = h.S > 1 ? kClusterNetsPerCluster * h.clusters : 0;
    cudaStream_t hs = next_stream();
    rc_block_kernel<kHugeT, kHugeK, int, false><<<h.ctas, kHugeT, 0, hs>>>(
        job, L(7), counters + 7, work + 7, ws + off_huge, stride, few);
    count_launch();
    err = cudaGetLastError();
    if (err == cudaSuccess && h.S > 1) {
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = (unsigned)h.S;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3(h.clusters * h.S);
      cfg.blockDim = dim3(kHugeT);
      cfg.stream = hs;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      err = cudaLaunchKernelEx(&cfg, rc_cluster_kernel<kHugeT, kHugeK>, job, (const int*)L(7),
                               (const int*)(counters + 7), ws + off_huge + stride * (size_t)h.ctas,
                               h.stride_c, few);
      count_launch();
    }
  }
  for (int c = tn.num; c >= 1 && err == cudaSuccess; --c) {
    if (max_net_nodes <= cls.nmax[c - 1]) continue;
    const int nmax = std::min(cls.nmax[c], max_net_nodes);
    err = launch_shape(tn.shape[c - 1], job, L(c), counters + c, work + c, nmax, di.sms,
                       next_stream());
  }
  if (err == cudaSuccess) {
    rc_warp_kernel<<<di.sms * 8, 256, 0, next_stream()>>>(job, L(0), counters + 0, work + 0);
    count_launch();
    err = cudaGetLastError();
  }
  // join (also after a failed launch, so a capture is never left unjoined)
  for (int i = 0; i < nside; ++i) {
    cudaError_t e = cudaEventRecord(fork->join[i], fork->side[i]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, fork->join[i], 0);
    if (err == cudaSuccess) err = e;
  }
  if (err != cudaSuccess) {
    cudaGetLastError();  // do not leave the error for the caller's next call
    return OTG_ERR_CUDA;
  }
  return OTG_OK;
}

otg_status rc_launch(const otg_rc_forest* f, int max_net_nodes, void* workspace,
                     size_t workspace_bytes, cudaStream_t stream) {
  if (!forest_ok(f) || !workspace || max_net_nodes < 1) return OTG_ERR_INVALID;
  if (f->num_nets == 0) return OTG_OK;
  RcJob job{};
  job.a0 = make_args(f, (int*)workspace);
  job.num = f->num_nets;
  return rc_launch_job(job, f->num_nets, max_net_nodes, workspace, workspace_bytes, stream);
}

otg_status rc_launch_subset(const otg_rc_forest* f, int max_net_nodes, const int* nets,
                            const int* num_dev, int cap, void* workspace, size_t workspace_bytes,
                            cudaStream_t stream) {
  if (!forest_ok(f) || !workspace || !nets || !num_dev || cap < 0 || max_net_nodes < 1)
    return OTG_ERR_INVALID;
  RcJob job{};
  job.a0 = make_args(f, (int*)workspace);
  job.nets = nets;
  job.num_dev = num_dev;
  return rc_launch_job(job, cap, max_net_nodes, workspace, workspace_bytes, stream);
}

otg_status rc_launch_items(const RcArgsOpaque* forests, const int2* items, const int* num_dev,
                           int cap, int max_net_nodes, void* workspace, size_t workspace_bytes,
                           cudaStream_t stream, const RcFork* fork) {
  if (!forests || !items || !num_dev || cap < 0) return OTG_ERR_INVALID;
  RcJob job{};
  job.forests = (const RcArgs*)forests;
  job.items = items;
  job.num_dev = num_dev;
  return rc_launch_job(job, cap, max_net_nodes, workspace, workspace_bytes, stream, fork);
}

size_t rc_args_bytes() { return sizeof(RcArgs); }

namespace {

// Autotuner: coordinate descent over the tuning on a sample forest (device
// pointers), timing whole passes with CUDA events (best of 3 after one
// checked pass).  Two rounds of: a shape per class, scaled class bounds
// (lowering the last bound moves nets to the global-workspace path), and
// merging a class into the next.  Every candidate gives the same outputs.
otg_status rc_autotune(const otg_rc_forest* f, int max_net_nodes, cudaStream_t st, RcTune* out) {
  if (!forest_ok(f) || f->num_nets < 1 || max_net_nodes < 1) return OTG_ERR_INVALID;
  DevInfo& di = dev_info();
  const int budget = di.smem_optin - kStaticSmemReserve;
  RcTune widest;  // sends every block net to the global path: the largest workspace
  widest.num = 1;
  widest.nmax[0] = 33;
  widest.shape[0] = 0;
  size_t a0, a1, a2;
  const size_t bytes =
      rc_workspace_bytes_for(widest, f->num_nets, max_net_nodes, di.sms, &a0, &a1, &a2);
  void* ws = nullptr;
  if (cudaMalloc(&ws, bytes) != cudaSuccess) {
    cudaGetLastError();
    return OTG_ERR_OOM;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  RcJob job{};
  job.a0 = make_args(f, (int*)ws);
  job.num = f->num_nets;
  otg_status err = OTG_OK;
  auto time_of = [&](const RcTune& t) -> float {
    if (rc_launch_job(job, f->num_nets, max_net_nodes, ws, bytes, st, nullptr, &t) != OTG_OK)
      return 1e30f;
    int code = 0;
    if (cudaMemcpyAsync(&code, ws, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      cudaGetLastError();
      err = OTG_ERR_CUDA;
      return 1e30f;
    }
    if (code != 0) {
      err = (otg_status)code;  // the sample itself is bad
      return 1e30f;
    }
    float best = 1e30f;
    for (int r = 0; r < 3; ++r) {
      cudaEventRecord(e0, st);
      rc_launch_job(job, f->num_nets, max_net_nodes, ws, bytes, st, nullptr, &t);
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      best = std::min(best, ms);
    }
    return best;
  };
  RcTune best = current_tune(budget);
  float tb = time_of(best);
  auto consider = [&](const RcTune& t) {
    if (err != OTG_OK || !tune_ok(t, budget)) return;
    const float x = time_of(t);
    if (x < tb) {
      tb = x;
      best = t;
    }
  };
  for (int round = 0; round < 2 && err == OTG_OK; ++round) {
    for (int c = 0; c < best.num; ++c)
      for (int sh = 0; sh < kNumShapes; ++sh) {
        if (sh == best.shape[c]) continue;
        RcTune t = best;
        t.shape[c] = sh;
        consider(t);
      }
    for (int c = 0; c < best.num; ++c)
      for (float fct : {0.5f, 0.7f, 1.4f, 2.0f}) {
        RcTune t = best;
        t.nmax[c] = (int)(best.nmax[c] * fct);
        consider(t);
      }
    for (int c = 0; c + 1 < best.num; ++c) {  // merge class c into c+1
      RcTune t = best;
      for (int k = c; k + 1 < t.num; ++k) {
        t.nmax[k] = t.nmax[k + 1];
        t.shape[k] = t.shape[k + 1];
      }
      --t.num;
      consider(t);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(ws);
  if (err != OTG_OK) return err;
  set_tune(best);
  *out = best;
  return OTG_OK;
}

void to_c(const RcTune& t, otg_rc_tuning* o) {
  std::memset(o, 0, sizeof(*o));
  o->num_classes = t.num;
  for (int c = 0; c < t.num; ++c) {
    o->class_max[c] = t.nmax[c];
    o->class_threads[c] = kShapeSet[t.shape[c]].T;
    o->class_items[c] = kShapeSet[t.shape[c]].K;
  }
}

bool from_c(const otg_rc_tuning* o, RcTune* t) {
  if (o->num_classes < 1 || o->num_classes > kBlockClasses) return false;
  t->num = o->num_classes;
  for (int c = 0; c < t->num; ++c) {
    t->nmax[c] = o->class_max[c];
    t->shape[c] = shape_index(o->class_threads[c], o->class_items[c]);
    if (t->shape[c] < 0) return false;
  }
  return true;
}

}  // namespace

cudaError_t rc_fork_create(RcFork* f, int n) {
  *f = RcFork{};
  f->n = std::min(std::max(n, 0), (int)RcFork::kMax);
  cudaError_t e = cudaEventCreateWithFlags(&f->fork, cudaEventDisableTiming);
  for (int i = 0; i < f->n && e == cudaSuccess; ++i) {
    e = cudaStreamCreateWithFlags(&f->side[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f->join[i], cudaEventDisableTiming);
  }
  return e;
}

void rc_fork_destroy(RcFork* f) {
  for (int i = 0; i < RcFork::kMax; ++i) {
    if (f->side[i]) cudaStreamDestroy(f->side[i]);
    if (f->join[i]) cudaEventDestroy(f->join[i]);
  }
  if (f->fork) cudaEventDestroy(f->fork);
  *f = RcFork{};
}

void rc_args_fill(const otg_rc_forest* f, int* status, void* out) {
  const RcArgs a = make_args(f, status);
  std::memcpy(out, &a, sizeof(a));
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

otg_status otg_rc_get_tuning(otg_rc_tuning* out) {
  if (!out) return OTG_ERR_INVALID;
  otg::DevInfo& di = otg::dev_info();
  if (di.sms <= 0) return OTG_ERR_CUDA;
  otg::to_c(otg::current_tune(di.smem_optin - otg::kStaticSmemReserve), out);
  return OTG_OK;
}

otg_status otg_rc_set_tuning(const otg_rc_tuning* t) {
  otg::DevInfo& di = otg::dev_info();
  if (di.sms <= 0) return OTG_ERR_CUDA;
  const int budget = di.smem_optin - otg::kStaticSmemReserve;
  otg::RcTune tn = otg::default_tune(budget);
  if (t && (!otg::from_c(t, &tn) || !otg::tune_ok(tn, budget))) return OTG_ERR_INVALID;
  otg::set_tune(tn);
  return OTG_OK;
}

otg_status otg_rc_autotune(const otg_rc_forest* sample, int32_t max_net_nodes,
                           otg_stream_t stream, otg_rc_tuning* out) {
  otg::RcTune t;
  const otg_status st = otg::rc_autotune(sample, max_net_nodes, (cudaStream_t)stream, &t);
  if (st == OTG_OK && out) otg::to_c(t, out);
  return st;
}

otg_status otg_rc_timing(const otg_rc_forest* forest, int32_t max_net_nodes, void* workspace,
                         size_t workspace_bytes, otg_stream_t stream) {
  return otg::rc_launch(forest, max_net_nodes, workspace, workspace_bytes, (cudaStream_t)stream);
}

#ifdef OTG_PHASE_TIMING
// Instrumented builds only: copies (and clears) the per-phase cycle totals.
int otg_debug_phase_cycles(unsigned long long* out, int n) {
  if (n > 32) n = 32;
  if (cudaMemcpyFromSymbol(out, otg::otg_phase_cycles, sizeof(unsigned long long) * n) !=
      cudaSuccess)
    return -1;
  unsigned long long z[32] = {0};
  cudaMemcpyToSymbol(otg::otg_phase_cycles, z, sizeof(z));
  return n;
}
#endif

otg_status otg_rc_timing_subset(const otg_rc_forest* forest, int32_t max_net_nodes,
                                const int32_t* net_list, const int32_t* num_listed,
                                int32_t max_listed, void* workspace, size_t workspace_bytes,
                                otg_stream_t stream) {
  return otg::rc_launch_subset(forest, max_net_nodes, net_list, num_listed, max_listed, workspace,
                               workspace_bytes, (cudaStream_t)stream);
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
