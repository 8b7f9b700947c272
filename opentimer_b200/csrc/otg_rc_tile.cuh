// otg_rc_tile.cuh -- the block path of the fused RC pass: one CTA per net,
// the whole net staged in shared memory with 16-bit indices.  Included by
// otg_rc.cu inside its anonymous namespace (it uses RcArgs, report(),
// block_radix_sort, the fixed-point helpers and the splitter hash there).
//
// Replaces, per net, compute_net_bfs + block_couting_sort
// (ot/cuda/rct.cu:120-245, ot/cuda/sort.cuh:63-142), prepare_res_cap
// (rct.cu:314-359) and compute_net_timing (rct.cu:11-59).
//
// Topology (T1-T7) works edge by edge and needs no adjacency list:
//   T1  edges in (validated), packed 16-bit degree counters by atomics;
//   T2  degree scan -> each node's arc range [off(v), off(v+1));
//   T3  one atomic per arc end places the arc in its node's range, and
//       since the twin's place is known in the same step, the Euler-tour
//       successor follows at once: after (x->y) comes y's next arc after
//       (y->x), cyclically; the arc before the root's first arc is cut;
//   T4  tour ranking: hashed splitter arcs cut the tour into short
//       sublists, one thread walks each, pointer jumping ranks them;
//   T5  per edge, the arc of lower rank is the down arc: parent, child,
//       the child's tour entry and exit; the directed edge goes out;
//   T6  a bitmap of down-arc positions and its popcount prefix give each
//       child's preorder number (down arcs up to its entry) and depth
//       (downs - ups up to it); subtree size is half the entry/exit span;
//   T7  BFS slots: stable radix sort by depth of the ids in descending
//       order, the reference's (distance asc, local id desc) rule
//       (sort.cuh:102-121); node2bfs, pid.
// Elmore (E1-E9), one corner pair at a time, with exact int64 fixed-point
// sums (fx_scale): load and ldelay are subtree sums, taken as differences
// of an exclusive prefix over the preorder; delay and beta are path sums,
// taken as a prefix over the signed Euler tour of per-node int64 terms
// that are converted once per node, so the tour scans only add integers.
// Every scan is one tile: thread t owns an odd number KE of consecutive
// items (odd, so strided 8- and 16-byte accesses spread over the banks),
// sums them, and the block-wide base comes from the warp totals after a
// single barrier; a second pass over its items emits the prefixes.

// ---- layout -------------------------------------------------------------
struct RcTileLayout {
  // persistent
  uint32_t pre, psz, bpre, code, pres;
  // topology scratch (T1-T7)
  uint32_t E, PX, deg, off, succ, sidx, subrk, spos, sl, db, dbp, depth, par, slot, rbuf, hist;
  // Elmore (E1-E9), overlaying the topology scratch
  uint32_t X, Y, Ip;
  uint32_t total, ns_cap;
};

__host__ __device__ inline RcTileLayout rc_tile_layout(int n, int T) {
  RcTileLayout l;
  const uint32_t N = (uint32_t)n, M = n > 0 ? (uint32_t)(n - 1) : 0u, A = 2u * M;
  const uint32_t W = (uint32_t)T / 32u;
  l.ns_cap = 2u * (A / (uint32_t)kSplit) + 64u;
  uint32_t o = 0;
#define OTG_AL(x) (((x) + 15u) & ~15u)
#define OTG_TAKE(f, bytes)   \
  do {                       \
    l.f = o;                 \
    o = OTG_AL(o + (bytes)); \
  } while (0)
  OTG_TAKE(pre, 2u * N);
  OTG_TAKE(psz, 2u * N);
  OTG_TAKE(bpre, 2u * N);
  OTG_TAKE(code, 2u * A);
  OTG_TAKE(pres, 4u * N);
  const uint32_t scratch = o;
  // topology
  OTG_TAKE(E, 4u * M);
  OTG_TAKE(PX, 4u * M);
  OTG_TAKE(deg, 4u * ((N + 1u) / 2u));
  OTG_TAKE(off, 2u * (N + 1u));
  OTG_TAKE(succ, 2u * A);  // then the tour rank of every arc
  const uint32_t r1 = o;
  OTG_TAKE(sidx, 2u * A);
  OTG_TAKE(subrk, 4u * A);
  OTG_TAKE(spos, 2u * l.ns_cap);
  OTG_TAKE(sl, 8u * l.ns_cap);
  const uint32_t end_rank = o;
  o = r1;  // after the ranking: bitmap, depth, parent, BFS sort
  OTG_TAKE(db, 4u * ((A + 31u) / 32u));
  OTG_TAKE(dbp, 4u * ((A + 31u) / 32u));
  OTG_TAKE(depth, 2u * N);
  OTG_TAKE(par, 2u * N);
  OTG_TAKE(slot, 2u * N);
  OTG_TAKE(rbuf, 2u * 2u * N);
  OTG_TAKE(hist, 4u * (1u << rc_radix_bits(T)) * W);
  const uint32_t end_topo = o > end_rank ? o : end_rank;
  // Elmore
  o = scratch;
  OTG_TAKE(X, 8u * N);
  OTG_TAKE(Y, 8u * N);
  OTG_TAKE(Ip, 16u * (N + 1u));
#undef OTG_TAKE
#undef OTG_AL
  l.total = end_topo > o ? end_topo : o;
  return l;
}

// ---- scans --------------------------------------------------------------

// Items per thread for a one-tile scan of C items: odd, so that consecutive
// threads' strided accesses of 8- and 16-byte elements fall in different
// banks.
__device__ __forceinline__ int tile_items(int C, int T) {
  const int k = (C + T - 1) / T;
  return k | 1;
}

// Block-wide exclusive scan of one int per thread with a single barrier:
// wt[] (T/32 ints) holds the warps' totals; the caller alternates between
// two wt buffers so that consecutive scans need no barrier in between.
template <int T>
__device__ __forceinline__ int tile_excl_i32(int v, int* wt, int* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  constexpr int W = T / 32;
  int x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int y = __shfl_up_sync(FULL, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) wt[w] = x;
  __syncthreads();
  const int t = lane < W ? wt[lane] : 0;
  const int before = __reduce_add_sync(FULL, lane < w ? t : 0);
  if (total) *total = __reduce_add_sync(FULL, t);
  return before + x - v;
}

__device__ __forceinline__ long long shfl_up_ll(long long v, int d) {
  return __shfl_up_sync(FULL, v, d);
}
__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) v += __shfl_xor_sync(FULL, v, d);
  return v;
}

// Exclusive block base of a pair of int64 values (one pair per thread),
// one barrier.  wt holds 2*(T/32) int64.
template <int T>
__device__ __forceinline__ void tile_excl_i64x2(long long a0, long long a1, long long* wt,
                                                long long& e0, long long& e1) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  constexpr int W = T / 32;
  long long x0 = a0, x1 = a1;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const long long y0 = shfl_up_ll(x0, d), y1 = shfl_up_ll(x1, d);
    if (lane >= d) {
      x0 += y0;
      x1 += y1;
    }
  }
  if (lane == 31) {
    wt[2 * w] = x0;
    wt[2 * w + 1] = x1;
  }
  __syncthreads();
  long long b0 = 0, b1 = 0;
  if (lane < w && lane < W) {
    b0 = wt[2 * lane];
    b1 = wt[2 * lane + 1];
  }
  e0 = warp_sum_ll(b0) + x0 - a0;
  e1 = warp_sum_ll(b1) + x1 - a1;
}

// Exclusive fixed-point scan of a corner pair over C items: term(i) gives
// item i's two int64 terms, emit(i, e0, e1, t) receives the exclusive
// prefix before item i and the item's terms.  Thread t owns items
// [t*KE, t*KE+KE); the terms are evaluated twice (sum, then emit), which
// keeps no per-item state in registers.
template <int T, class TermF, class EmitF>
__device__ __forceinline__ void scan_pair(int C, TermF term, EmitF emit, long long* wt) {
  const int KE = tile_items(C, T);
  const int i0 = threadIdx.x * KE;
  const int i1 = min(i0 + KE, C);
  long long s0 = 0, s1 = 0;
#pragma unroll 3
  for (int i = i0; i < i1; ++i) {
    const longlong2 t = term(i);
    s0 += t.x;
    s1 += t.y;
  }
  long long e0, e1;
  tile_excl_i64x2<T>(s0, s1, wt, e0, e1);
#pragma unroll 3
  for (int i = i0; i < i1; ++i) {
    const longlong2 t = term(i);
    emit(i, e0, e1, t);
    e0 += t.x;
    e1 += t.y;
  }
}

__device__ __forceinline__ unsigned u16_half(unsigned word, int hi) {
  return hi ? (word >> 16) : (word & 0xFFFFu);
}

// Per-warp max of |v| for non-negative float bit patterns, committed to
// a shared max word.
__device__ __forceinline__ void commit_max(float m, unsigned* dst) {
  const unsigned x = __reduce_max_sync(FULL, __float_as_uint(fabsf(m)));
  if ((threadIdx.x & 31) == 0 && x) atomicMax(dst, x);
}

// ---- the net --------------------------------------------------------------
template <int T>
__device__ void rc_net_tile(const RcArgs& a, int net, char* ws, int n, int* sh, long long* shl) {
  using Ix = uint16_t;
  constexpr unsigned NONE = 0xFFFFu;
  constexpr int W = T / 32;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int b = a.nodes_start[net];
  const int m = n - 1, A = 2 * m, eb = b - net;
  const RcTileLayout L = rc_tile_layout(n, T);
  Ix* pre = (Ix*)(ws + L.pre);
  Ix* psz = (Ix*)(ws + L.psz);
  Ix* bpre = (Ix*)(ws + L.bpre);
  int16_t* code = (int16_t*)(ws + L.code);
  float* pres = (float*)(ws + L.pres);
  unsigned* E = (unsigned*)(ws + L.E);
  unsigned* PX = (unsigned*)(ws + L.PX);
  unsigned* deg = (unsigned*)(ws + L.deg);
  Ix* off = (Ix*)(ws + L.off);
  Ix* succ = (Ix*)(ws + L.succ);
  Ix* rank = succ;
  Ix* sidx = (Ix*)(ws + L.sidx);
  unsigned* subrk = (unsigned*)(ws + L.subrk);
  Ix* spos = (Ix*)(ws + L.spos);
  volatile unsigned long long* sl = (volatile unsigned long long*)(ws + L.sl);
  unsigned* db = (unsigned*)(ws + L.db);
  unsigned* dbp = (unsigned*)(ws + L.dbp);
  Ix* depth = (Ix*)(ws + L.depth);
  Ix* par = (Ix*)(ws + L.par);
  Ix* slot = (Ix*)(ws + L.slot);
  Ix* rbuf = (Ix*)(ws + L.rbuf);
  int* hist = (int*)(ws + L.hist);
  float2* X = (float2*)(ws + L.X);
  float2* Y = (float2*)(ws + L.Y);
  longlong2* Ip = (longlong2*)(ws + L.Ip);
  int* wt0 = sh;        // [32] warp totals, ping
  int* wt1 = sh + 32;   // [32] pong
  int* s_flag = sh + 64;
  int* s_ns = sh + 65;
  int* s_maxd = sh + 66;
  int* s_sel = sh + 67;
  unsigned* smx = (unsigned*)(sh + 72);  // [16] float maxima
  const int root = a.roots[net];
  // the forest's pointers in registers (a lives in shared memory)
  int2* __restrict__ g_edges = a.edges;
  const float* __restrict__ g_res = a.res;
  const float2* __restrict__ cap2 = (const float2*)a.cap;

  auto fail = [&]() -> bool {
    __syncthreads();
    const int f = *s_flag;
    if (f && tid == 0) report(a, f, net);
    return f != 0;
  };

  PHASE_BEGIN();
  // ---- T1: edges and degrees
  if (tid == 0) {
    *s_flag = ((unsigned)root >= (unsigned)n) ? OTG_ERR_INVALID : 0;
    *s_ns = 0;
    *s_maxd = 0;
    *s_sel = 0;
  }
  if (tid < 16) smx[tid] = 0u;
  const int NW = (n + 1) >> 1;
  for (int w = tid; w < NW; w += T) deg[w] = 0u;
  __syncthreads();
  for (int e = tid; e < m; e += T) {
    int2 ed = g_edges[eb + e];
    if ((unsigned)ed.x >= (unsigned)n || (unsigned)ed.y >= (unsigned)n) {
      *s_flag = OTG_ERR_INVALID;
      ed = make_int2(0, 0);
    }
    E[e] = (unsigned)ed.x | ((unsigned)ed.y << 16);
    atomicAdd(&deg[ed.x >> 1], 1u << ((ed.x & 1) << 4));
    atomicAdd(&deg[ed.y >> 1], 1u << ((ed.y & 1) << 4));
  }
  if (fail()) return;

  PHASE(0);
  // ---- T2: arc ranges; the counters become placement cursors
  {
    const int KW = tile_items(NW, T);
    const int w0 = tid * KW, w1 = min(w0 + KW, NW);
    int local = 0;
    bool zero = false;
    for (int w = w0; w < w1; ++w) {
      const unsigned d = deg[w];
      const int d0 = (int)(d & 0xFFFFu), d1 = 2 * w + 1 < n ? (int)(d >> 16) : 1;
      zero |= d0 == 0 || d1 == 0;
      local += d0 + (2 * w + 1 < n ? d1 : 0);
    }
    if (zero) *s_flag = OTG_ERR_NOT_TREE;  // a node without an edge
    int run = tile_excl_i32<T>(local, wt0, nullptr);
    for (int w = w0; w < w1; ++w) {
      const unsigned d = deg[w];
      const int o0 = run, o1 = run + (int)(d & 0xFFFFu);
      run = o1 + (2 * w + 1 < n ? (int)(d >> 16) : 0);
      off[2 * w] = (Ix)o0;
      if (2 * w + 1 < n) off[2 * w + 1] = (Ix)o1;
      deg[w] = (unsigned)o0 | ((unsigned)o1 << 16);
    }
    if (tid == 0) off[n] = (Ix)A;
  }
  if (fail()) return;

  PHASE(1);
  // ---- T3: place arcs, Euler-tour successors
  const int head = (int)off[root];
  for (int e = tid; e < m; e += T) {
    const unsigned xy = E[e];
    const int x = (int)(xy & 0xFFFFu), y = (int)(xy >> 16);
    const int px = (int)u16_half(atomicAdd(&deg[x >> 1], 1u << ((x & 1) << 4)), x & 1);
    const int py = (int)u16_half(atomicAdd(&deg[y >> 1], 1u << ((y & 1) << 4)), y & 1);
    int sy = py + 1;
    if (sy == (int)off[y + 1]) sy = (int)off[y];
    int sx = px + 1;
    if (sx == (int)off[x + 1]) sx = (int)off[x];
    succ[px] = (Ix)(sy == head ? (int)NONE : sy);  // after x->y: y's next arc
    succ[py] = (Ix)(sx == head ? (int)NONE : sx);
    PX[e] = (unsigned)px | ((unsigned)py << 16);
  }
  // ---- T4: tour ranking.  Number the splitters (warp-aggregated), walk
  // the sublists, rank the sublists by pointer jumping.
  int ns = 0, sel = 0;
  for (;;) {
    __syncthreads();
    for (int p0 = (tid & ~31); p0 < A; p0 += T) {
      const int p = p0 + lane;
      const bool s = p < A && is_splitter(p, sel, head);
      const unsigned bal = __ballot_sync(FULL, s);
      int base = 0;
      if (lane == 0 && bal) base = atomicAdd(s_ns, __popc(bal));
      base = __shfl_sync(FULL, base, 0);
      if (s) {
        const int id = base + __popc(bal & ((1u << lane) - 1u));
        if (id < (int)L.ns_cap) {
          sidx[p] = (Ix)id;
          spos[id] = (Ix)p;
        }
      }
    }
    __syncthreads();
    ns = *s_ns;
    if (ns <= (int)L.ns_cap) break;
    __syncthreads();
    if (tid == 0) *s_ns = 0;
    ++sel;  // uniform: every thread read the same count
  }
  PHASE(2);
  for (int s = tid; s < ns; s += T) {
    int cur = (int)spos[s];
    unsigned o = 0, next = 0xFFFFFFFFu;
    for (int step = 0; step < A; ++step) {
      subrk[cur] = (unsigned)s | (o << 16);
      ++o;
      const int nx = (int)succ[cur];
      if (nx == (int)NONE) break;
      if (is_splitter(nx, sel, head)) {
        next = (unsigned)sidx[nx];
        break;
      }
      cur = nx;
    }
    sl[s] = sl_pack(next, o);
  }
  __syncthreads();
  PHASE(3);
  {
    int rounds = 1;
    while ((1 << rounds) < ns) ++rounds;
    for (int r = 0; r <= rounds; ++r) {
      for (int s = tid; s < ns; s += T) {
        const unsigned long long p = sl[s];
        if (sl_next(p) != 0xFFFFFFFFu) {
          const unsigned long long q = sl[sl_next(p)];
          sl[s] = sl_pack(sl_next(q), sl_acc(p) + sl_acc(q));
        }
      }
      __syncthreads();
    }
  }
  PHASE(4);
  // the head's chain must be the whole tour (else: a cycle or a second
  // component, i.e. not a tree)
  if (tid == 0) {
    const unsigned long long h = sl[sidx[head]];
    if (sl_next(h) != 0xFFFFFFFFu || sl_acc(h) != (unsigned)A) *s_flag = OTG_ERR_NOT_TREE;
  }
  if (fail()) return;
  for (int p = tid; p < A; p += T) {
    const unsigned sr = subrk[p];
    rank[p] = (Ix)(A - (int)sl_acc(sl[sr & 0xFFFFu]) + (int)(sr >> 16));
  }
  const int NDW = (A + 31) >> 5;
  __syncthreads();
  for (int w = tid; w < NDW; w += T) db[w] = 0u;
  __syncthreads();

  PHASE(5);
  // ---- T5: per edge: down arc, parent/child, entry/exit; directed edge out
  for (int e = tid; e < m; e += T) {
    const unsigned pp = PX[e], xy = E[e];
    const int rx = (int)rank[pp & 0xFFFFu], ry = (int)rank[pp >> 16];
    const int x = (int)(xy & 0xFFFFu), y = (int)(xy >> 16);
    const bool xdown = rx < ry;  // x->y entered y first: x is the parent
    const int par_ = xdown ? x : y, ch = xdown ? y : x;
    const int en = xdown ? rx : ry, ex = xdown ? ry : rx;
    atomicOr(&db[en >> 5], 1u << (en & 31));
    PX[e] = (unsigned)en | ((unsigned)ex << 16);
    E[e] = (unsigned)par_ | ((unsigned)ch << 16);
    g_edges[eb + e] = make_int2(par_, ch);
  }
  __syncthreads();
  PHASE(6);
  // ---- T6: preorder and depth from the down-arc bitmap
  {
    const int KW = tile_items(NDW, T);
    const int w0 = tid * KW, w1 = min(w0 + KW, NDW);
    int local = 0;
    for (int w = w0; w < w1; ++w) local += __popc(db[w]);
    int run = tile_excl_i32<T>(local, wt1, nullptr);
    for (int w = w0; w < w1; ++w) {
      dbp[w] = (unsigned)run;
      run += __popc(db[w]);
    }
  }
  if (tid == 0) {
    pre[root] = 0;
    psz[0] = (Ix)n;
    pres[0] = 0.0f;
    depth[root] = 0;
    par[root] = (Ix)root;
  }
  __syncthreads();
  {
    int dmax = 0;
    for (int e = tid; e < m; e += T) {
      const unsigned pp = PX[e], pc = E[e];
      const int en = (int)(pp & 0xFFFFu), ex = (int)(pp >> 16);
      const int ch = (int)(pc >> 16);
      const int downs = (int)dbp[en >> 5] + __popc(db[en >> 5] & (0xFFFFFFFFu >> (31 - (en & 31))));
      const int pv = downs;  // the root is preorder 0
      const int d = 2 * downs - en - 1;
      pre[ch] = (Ix)pv;
      depth[ch] = (Ix)d;
      par[ch] = (Ix)(pc & 0xFFFFu);
      psz[pv] = (Ix)((ex - en + 1) >> 1);
      pres[pv] = g_res[eb + e];
      code[en] = (int16_t)(pv + 1);
      code[ex] = (int16_t)(-(pv + 1));
      dmax = max(dmax, d);
    }
    dmax = __reduce_max_sync(FULL, dmax);
    if (lane == 0 && dmax) atomicMax(s_maxd, dmax);
  }
  __syncthreads();
  PHASE(7);
  // ---- T7: BFS slots, the rank under (depth asc, local id desc)
  {
    Ix* nas = bpre;  // BFS slot -> id, then BFS slot -> preorder
    const int maxd = *s_maxd;
    const int NWB = (n + 31) >> 5;  // bitmap words per depth
    const int words = (maxd + 1) * NWB;
    const int region = (int)(L.hist - L.rbuf) + 4 * (1 << rc_radix_bits(T)) * W;
    if (words * 6 <= region) {
      // shallow trees: one bitmap of ids per depth; a node's slot is the
      // number of set bits before it in (depth asc, word desc, bit desc)
      // order: a prefix count per word plus the bits above it in its word
      unsigned* bm = (unsigned*)rbuf;
      Ix* wp = (Ix*)(bm + words);
      for (int k = tid; k < words; k += T) bm[k] = 0u;
      __syncthreads();
      for (int v = tid; v < n; v += T)
        atomicOr(&bm[(int)depth[v] * NWB + (v >> 5)], 1u << (v & 31));
      __syncthreads();
      // flattened order f = d * NWB + (NWB - 1 - w)
      const int KW = tile_items(words, T);
      const int f0 = tid * KW, f1 = min(f0 + KW, words);
      auto word_of = [&](int f) { const int d = f / NWB; return d * NWB + (NWB - 1 - (f - d * NWB)); };
      int local = 0;
      for (int f = f0; f < f1; ++f) local += __popc(bm[word_of(f)]);
      int run = tile_excl_i32<T>(local, wt0, nullptr);
      for (int f = f0; f < f1; ++f) {
        const int k = word_of(f);
        wp[k] = (Ix)run;
        run += __popc(bm[k]);
      }
      __syncthreads();
      for (int v = tid; v < n; v += T) {
        const int k = (int)depth[v] * NWB + (v >> 5);
        const int r = (int)wp[k] + __popc(bm[k] >> (v & 31) >> 1);
        slot[v] = (Ix)r;
        nas[r] = (Ix)v;
      }
    } else {
      // deep trees: stable radix sort by depth of the ids in descending order
      // (the reference's (distance asc, local id desc) rule, sort.cuh:102-121)
      block_radix_sort<T>(
          n, 32 - __clz(max(maxd, 1)), [&](int j) { return (int)depth[n - 1 - j]; }, rbuf,
          rbuf + n, nas, hist, wt0);
      for (int r = tid; r < n; r += T) {
        const int v = n - 1 - (int)nas[r];
        nas[r] = (Ix)v;
        slot[v] = (Ix)r;
      }
    }
    __syncthreads();
    for (int v = tid; v < n; v += T) a.node2bfs[b + v] = (int)slot[v];
    for (int r = tid; r < n; r += T) {
      const int v = (int)nas[r];
      a.pid[b + r] = r == 0 ? 0 : r - (int)slot[par[v]];
      bpre[r] = pre[v];
    }
    __syncthreads();
  }

  PHASE(8);
  // ---- E: Elmore per corner pair
  for (int cp = 0; cp < 2; ++cp) {
    long long* wtl0 = shl;
    long long* wtl1 = shl + 2 * W;
    if (tid < 4) smx[4 + tid] = 0u;  // the pair's sweep maxima (w, delay, w2)
    // E0: the pair's caps, read once in id order (coalesced), staged by
    // preorder in Y (free until the delay sweep), and their maxima
    {
      float m0 = 0.f, m1 = 0.f;
      for (int v = tid; v < n; v += T) {
        const float2 c = cap2[2 * (size_t)(b + v) + cp];
        Y[pre[v]] = c;
        m0 = fmaxf(m0, fabsf(c.x));
        m1 = fmaxf(m1, fabsf(c.y));
      }
      commit_max(m0, smx + 2 * cp);
      commit_max(m1, smx + 2 * cp + 1);
    }
    __syncthreads();
    float upc[2], dnc[2];
    fx_scale(__uint_as_float(smx[2 * cp]), n, upc[0], dnc[0]);
    fx_scale(__uint_as_float(smx[2 * cp + 1]), n, upc[1], dnc[1]);
    // E1: load scan over the preorder: Ip[i] = exclusive prefix of cap
    scan_pair<T>(
        n,
        [&](int i) {
          const float2 c = Y[i];
          return make_longlong2(to_fx(c.x, upc[0]), to_fx(c.y, upc[1]));
        },
        [&](int i, long long e0, long long e1, longlong2 t) {
          Ip[i] = make_longlong2(e0, e1);
          if (i == n - 1) Ip[n] = make_longlong2(e0 + t.x, e1 + t.y);  // the total
        },
        wtl0);
    __syncthreads();
    PHASE(10);
    // E2: load = prefix difference over the subtree's preorder range
    {
      const int KE = tile_items(n, T);
      const int i0 = tid * KE, i1 = min(i0 + KE, n);
      float mw0 = 0.f, mw1 = 0.f;
      for (int i = i0; i < i1; ++i) {
        const longlong2 lo = Ip[i], hi = Ip[i + (int)psz[i]];
        const float2 v = make_float2(from_fx(hi.x - lo.x, dnc[0]), from_fx(hi.y - lo.y, dnc[1]));
        X[i] = v;
        const float r = pres[i];
        mw0 = fmaxf(mw0, fabsf(v.x * r));
        mw1 = fmaxf(mw1, fabsf(v.y * r));
      }
      commit_max(mw0, smx + 4);
      commit_max(mw1, smx + 5);
    }
    __syncthreads();
    PHASE(11);
    // E3: delay terms W = fx(R * load) into Ip; load out in BFS order
    float upw[2], dnw[2];
    fx_scale(__uint_as_float(smx[4]), n, upw[0], dnw[0]);
    fx_scale(__uint_as_float(smx[5]), n, upw[1], dnw[1]);
    {
      const int KE = tile_items(n, T);
      const int i0 = tid * KE, i1 = min(i0 + KE, n);
      for (int i = i0; i < i1; ++i) {
        const float2 v = X[i];
        const float r = pres[i];
        Ip[i] = make_longlong2(to_fx(v.x * r, upw[0]), to_fx(v.y * r, upw[1]));
      }
      float2* out = (float2*)a.load;
      for (int r = tid; r < n; r += T) out[2 * (size_t)(b + r) + cp] = X[bpre[r]];
    }
    if (tid < 2) smx[6 + tid] = 0u;
    __syncthreads();
    PHASE(12);
    // E4: delay = prefix over the signed tour of W; emitted at down arcs.
    // First the caps move from Y to X (free since the load went out); the
    // scan's barrier lies between this copy and the first delay written to Y.
    {
      const int KE = tile_items(n, T);
      const int i0 = tid * KE, i1 = min(i0 + KE, n);
      for (int i = i0; i < i1; ++i) X[i] = Y[i];
    }
    {
      float md0 = 0.f, md1 = 0.f;
      scan_pair<T>(
          A,
          [&](int p) {
            const int c = (int)code[p];
            const longlong2 w = Ip[(c > 0 ? c : -c) - 1];
            return c > 0 ? w : make_longlong2(-w.x, -w.y);
          },
          [&](int p, long long e0, long long e1, longlong2 t) {
            const int c = (int)code[p];
            if (c > 0) {
              const float2 d = make_float2(from_fx(e0 + t.x, dnw[0]), from_fx(e1 + t.y, dnw[1]));
              Y[c - 1] = d;
              md0 = fmaxf(md0, fabsf(d.x));
              md1 = fmaxf(md1, fabsf(d.y));
            }
          },
          wtl1);
      commit_max(md0, smx + 6);
      commit_max(md1, smx + 7);
      if (tid == 0) Y[0] = make_float2(0.f, 0.f);
    }
    __syncthreads();
    PHASE(13);
    // E5: ldelay scan over the preorder of cap * delay (scale from the
    // bound max|cap| * max|delay|); delay out in BFS order
    float upd[2], dnd[2];
    fx_scale(__uint_as_float(smx[2 * cp]) * __uint_as_float(smx[6]), n, upd[0], dnd[0]);
    fx_scale(__uint_as_float(smx[2 * cp + 1]) * __uint_as_float(smx[7]), n, upd[1], dnd[1]);
    {
      float2* out = (float2*)a.delay;
      for (int r = tid; r < n; r += T) out[2 * (size_t)(b + r) + cp] = Y[bpre[r]];
    }
    scan_pair<T>(
        n,
        [&](int i) {
          const float2 c = X[i];
          const float2 d = Y[i];
          return make_longlong2(to_fx(c.x * d.x, upd[0]), to_fx(c.y * d.y, upd[1]));
        },
        [&](int i, long long e0, long long e1, longlong2 t) {
          Ip[i] = make_longlong2(e0, e1);
          if (i == n - 1) Ip[n] = make_longlong2(e0 + t.x, e1 + t.y);
        },
        wtl0);
    if (tid < 2) smx[8 + tid] = 0u;
    __syncthreads();
    PHASE(14);
    // E6: ldelay = prefix difference over the subtree range
    {
      const int KE = tile_items(n, T);
      const int i0 = tid * KE, i1 = min(i0 + KE, n);
      float mw0 = 0.f, mw1 = 0.f;
      for (int i = i0; i < i1; ++i) {
        const longlong2 lo = Ip[i], hi = Ip[i + (int)psz[i]];
        const float2 v = make_float2(from_fx(hi.x - lo.x, dnd[0]), from_fx(hi.y - lo.y, dnd[1]));
        X[i] = v;
        const float r = pres[i];
        mw0 = fmaxf(mw0, fabsf(v.x * r));
        mw1 = fmaxf(mw1, fabsf(v.y * r));
      }
      commit_max(mw0, smx + 8);
      commit_max(mw1, smx + 9);
    }
    __syncthreads();
    PHASE(15);
    // E7: beta terms into Ip; ldelay out
    fx_scale(__uint_as_float(smx[8]), n, upw[0], dnw[0]);
    fx_scale(__uint_as_float(smx[9]), n, upw[1], dnw[1]);
    {
      const int KE = tile_items(n, T);
      const int i0 = tid * KE, i1 = min(i0 + KE, n);
      for (int i = i0; i < i1; ++i) {
        const float2 v = X[i];
        const float r = pres[i];
        Ip[i] = make_longlong2(to_fx(v.x * r, upw[0]), to_fx(v.y * r, upw[1]));
      }
      float2* out = (float2*)a.ldelay;
      for (int r = tid; r < n; r += T) out[2 * (size_t)(b + r) + cp] = X[bpre[r]];
    }
    __syncthreads();
    PHASE(16);
    // E8: beta over the signed tour -> impulse = 2 beta - delay^2 (into X)
    scan_pair<T>(
        A,
        [&](int p) {
          const int c = (int)code[p];
          const longlong2 w = Ip[(c > 0 ? c : -c) - 1];
          return c > 0 ? w : make_longlong2(-w.x, -w.y);
        },
        [&](int p, long long e0, long long e1, longlong2 t) {
          const int c = (int)code[p];
          if (c > 0) {
            const float2 d = Y[c - 1];
            X[c - 1] = make_float2(fmaf(-d.x, d.x, 2.0f * from_fx(e0 + t.x, dnw[0])),
                                   fmaf(-d.y, d.y, 2.0f * from_fx(e1 + t.y, dnw[1])));
          }
        },
        wtl1);
    if (tid == 0) X[0] = make_float2(0.f, 0.f);
    __syncthreads();
    PHASE(17);
    // E9: impulse out; sink slews
    {
      float2* out = (float2*)a.impulse;
      for (int r = tid; r < n; r += T) out[2 * (size_t)(b + r) + cp] = X[bpre[r]];
      if (a.sinks_start) {
        const int s0 = a.sinks_start[net], s1 = a.sinks_start[net + 1];
        const float2 si = ((const float2*)a.driver_slew)[2 * (size_t)net + cp];
        float2* so = (float2*)a.sink_slew;
        for (int k = s0 + tid; k < s1; k += T) {
          const int v = a.sink_nodes[k];
          if ((unsigned)v >= (unsigned)n) {
            report(a, OTG_ERR_INVALID, net);
            continue;
          }
          const float2 iv = X[pre[v]];
          so[2 * (size_t)k + cp] = make_float2(sink_slew1(si.x, iv.x), sink_slew1(si.y, iv.y));
        }
      }
    }
    __syncthreads();
    PHASE(18);
  }
}
