// otg_prop.cu -- levelized timing propagation on the GPU, the consumer of
// the RC pass: slew, arc delay, arrival time and timing-test RAT forward,
// required time and slack backward, two splits x two transitions.
//
// Semantics follow the reference Timer's per-pin tasks: Timer::_fprop_slew,
// _fprop_delay, _fprop_at, _fprop_test, _bprop_rat (ot/timer/timer.cpp:733-
// 832), Arc::_fprop_slew/_fprop_delay/_fprop_at/_bprop_rat (arc.cpp:82-
// 205), Pin::_relax_slew/_relax_at/_relax_rat (pin.cpp:324-380), Test::
// _fprop_rat (test.cpp:88-135), Timing::delay/slew/constraint and
// is_transition_defined (ot/liberty/timing.cpp:198-230, 411-628), and the
// look-up interpolation Lut::operator() (ot/liberty/lut.cpp:166-245).  Net
// arcs read the RC pass's outputs: the driver's load at BFS slot 0, the
// Elmore delay and sign(si)*sqrt(si^2 + impulse) at the sink's slot
// (net.cpp:626-699, FlatRct accessors).  A value the reference keeps as an
// empty std::optional is NaN here.  Every add and multiply is an explicit
// rounding intrinsic, so no compiler fusion changes a bit.
//
// Schedule: one cooperative launch, a warp per pin, dataflow instead of
// level barriers.  Pins are numbered in level order (otg_levelize: every
// pin after all of its fanouts); the forward pass takes them last level
// first, warp w the items w, w+W, w+2W, ...  A pin waits (bounded) until
// the values it reads from its fanins are there, computes, and stores its
// own.  Because a pin depends only on lower-numbered items and each warp
// works through its items in order, the lowest unfinished item always has
// every input ready: the schedule cannot deadlock while all CTAs are
// resident, which the cooperative launch guarantees.  One grid barrier
// separates the forward pass from the backward pass, which runs the same
// way first level first.
//
// Readiness is carried by the values themselves: a fill kernel sets every
// arrival time and slew to kPending, a NaN payload that no stored value
// carries (an empty value is stored as the canonical NaN), and the forward
// pass does the same to each pin's required time before the barrier.  A
// reader polls exactly the words it needs with relaxed loads, each word is
// written once, so no fence or flag sits on the critical path.
//
// Inside a warp the lanes split a pin's (arc, split, from-transition,
// to-transition) combinations and reduce with shuffles; min/max reductions
// are order-free, so the lane split does not change a value.  Values that
// other warps wrote after the barrier are read with __ldcg (L2); the graph
// and the library are read-only for the launch and go through __ldg.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/otg.h"
#include "otg_internal.cuh"

namespace otg {
namespace {

constexpr int MIN_ = 0, MAX_ = 1, RISE_ = 0, FALL_ = 1;

__device__ __forceinline__ bool none(float x) { return isnan(x); }

// Lut::operator(): clamped segment search by lower_bound, then linear
// inter/extrapolation per axis (boundary values returned as they are).
__device__ float interpolate(float x, float x1, float x2, float y1, float y2) {
  if (x >= 3.402823466e+38f || x <= -3.402823466e+38f) return x;
  const float slope = __fdiv_rn(__fsub_rn(y2, y1), __fsub_rn(x2, x1));
  if (x < x1) return __fsub_rn(y1, __fmul_rn(__fsub_rn(x1, x), slope));
  if (x > x2) return __fadd_rn(y2, __fmul_rn(__fsub_rn(x, x2), slope));
  if (x == x1) return y1;
  if (x == x2) return y2;
  return __fadd_rn(y1, __fmul_rn(__fsub_rn(x, x1), slope));
}

// Table reads go through a generic pointer: shared memory when the
// library is staged on chip, else global memory (cached in L1).
__device__ int lower_bound(const float* a, int n, float v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

struct G {
  otg_prop_graph g;
  otg_prop_rc rc;
};

constexpr unsigned FULL = 0xffffffffu;

// A table chosen before the query values are known: lut_meta's (n1, n2,
// offset, variable order), n1 = -1 for "no table".
struct Lut {
  int n1, n2, off, var;
};

__device__ __forceinline__ Lut no_lut() { return Lut{-1, 0, 0, 0}; }

// Lut::operator() on (v1, v2) in the table's own axis order.
__device__ float lut_eval(const Lut& m, const float* data, float v1, float v2) {
  const int n1 = m.n1, n2 = m.n2;
  const float* i1 = data + m.off;
  const float* i2 = i1 + n1;
  const float* tb = i2 + n2;
  if (n1 < 1 || n2 < 1) return nanf("");
  if (n1 == 1 && n2 == 1) return tb[0];
  const int a1 = max(1, min(lower_bound(i1, n1, v1), n1 - 1));
  const int a2 = max(1, min(lower_bound(i2, n2, v2), n2 - 1));
  if (n1 == 1) return interpolate(v2, i2[a2 - 1], i2[a2], tb[a2 - 1], tb[a2]);
  const float x1 = i1[a1 - 1], x2 = i1[a1];
  if (n2 == 1) return interpolate(v1, x1, x2, tb[(a1 - 1) * n2], tb[a1 * n2]);
  const float lo = interpolate(v1, x1, x2, tb[(a1 - 1) * n2 + a2 - 1], tb[a1 * n2 + a2 - 1]);
  const float hi = interpolate(v1, x1, x2, tb[(a1 - 1) * n2 + a2], tb[a1 * n2 + a2]);
  return interpolate(v2, i2[a2 - 1], i2[a2], lo, hi);
}

// timing record: [sense, edge, constraint, lut x6]
__device__ bool transition_defined(const int* tr, int irf, int orf) {
  const int edge = __ldg(tr + 1), sense = __ldg(tr);
  if (edge == 1 && irf != RISE_) return false;
  if (edge == 2 && irf != FALL_) return false;
  if (sense == 0 && irf != orf) return false;  // positive unate
  if (sense == 1 && irf == orf) return false;  // negative unate
  return true;
}

// The table a Timing::delay/slew/constraint query of record t reads:
// which = 0 delay, 1 slew, 2 constraint.
__device__ Lut timing_lut(const G& G_, int t, int which, int irf, int orf) {
  if (t < 0) return no_lut();
  const int* tr = G_.g.timing + 9 * t;
  if (!transition_defined(tr, irf, orf)) return no_lut();
  const int lut = __ldg(tr + 3 + 2 * which + orf);
  if (lut < 0) return no_lut();
  const int4 m = __ldg(reinterpret_cast<const int4*>(G_.g.lut_meta) + lut);
  return Lut{m.x, m.y, m.z, m.w};
}

// The query itself; (a, b) = (slew, load) for delay and slew, (related
// slew, constrained slew) for constraint.
// Where the tables are read: the staged copy (floats [0, n)) for a table
// that lies inside it, global memory otherwise.
struct LutSrc {
  const float* smem;
  int n;
  const float* gmem;
};

__device__ float timing_value(const LutSrc& src, const Lut& m, float a, float b) {
  if (m.n1 < 0) return nanf("");
  const bool staged = m.off >= 0 && m.off + m.n1 + m.n2 + m.n1 * m.n2 <= src.n;
  const float* lutd = staged ? src.smem : src.gmem;
  if (m.var < 0) {  // no template: a scalar only
    if (m.n1 == 1 && m.n2 == 1) return lutd[m.off + 2];
    return nanf("");
  }
  // var 0: (slew | related) first; var 1: (load | constrained) first
  return m.var == 0 ? lut_eval(m, lutd, a, b) : lut_eval(m, lutd, b, a);
}

// RC node of a net arc's sink (arc_node: its local id in the net) as a
// global BFS slot (-1: none)
__device__ __forceinline__ int rc_slot(const G& G_, int arc) {
  const int node = __ldg(G_.g.arc_node + arc);
  if (node < 0) return -1;
  const int b = __ldg(G_.rc.nodes_start + __ldg(G_.g.arc_net + arc));
  return b + __ldg(G_.rc.node2bfs + b + node);
}

constexpr unsigned kPending = 0x7fbadbadu;  // "not yet computed"
constexpr unsigned kEmpty = 0x7fffffffu;    // the stored empty value

__device__ __forceinline__ float canon(float x) { return none(x) ? __uint_as_float(kEmpty) : x; }

__device__ __forceinline__ float ld_relaxed(const float* p) {
  float v;
  asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed4(float* p, float a, float b, float c, float d) {
  asm volatile("st.relaxed.gpu.global.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b),
               "f"(c), "f"(d)
               : "memory");
}

// Bounded wait until *p holds a computed value, returned in out; false
// when this or another wait gave up.  Each poll is one L2 round trip: the
// abort flag and the clock are read on every 8th poll only, and no poll
// sleeps, since a sleeping warp sees a new value only after it wakes.
__device__ bool wait_value(const float* p, float& out, GridCtl* c) {
  out = ld_relaxed(p);
  if (__float_as_uint(out) != kPending) return true;
  const unsigned long long t0 = gtime();
  for (int k = 0;; ++k) {
    out = ld_relaxed(p);
    if (__float_as_uint(out) != kPending) return true;
    if ((k & 7) != 7) continue;
    if (*(volatile int*)&c->abort) return false;
    if (gtime() - t0 > kGridWaitNs) {
      atomicExch(&c->abort, 1);
      atomicCAS(&c->status, 0, (int)OTG_ERR_TIMEOUT);
      return false;
    }
  }
}

// wait_value for two words at once: both loads in flight per poll.
__device__ bool wait_values(const float* p, const float* q, float& x, float& y, GridCtl* c) {
  x = ld_relaxed(p);
  y = ld_relaxed(q);
  if (__float_as_uint(x) != kPending && __float_as_uint(y) != kPending) return true;
  const unsigned long long t0 = gtime();
  for (int k = 0;; ++k) {
    if (__float_as_uint(x) == kPending) x = ld_relaxed(p);
    if (__float_as_uint(y) == kPending) y = ld_relaxed(q);
    if (__float_as_uint(x) != kPending && __float_as_uint(y) != kPending) return true;
    if ((k & 7) != 7) continue;
    if (*(volatile int*)&c->abort) return false;
    if (gtime() - t0 > kGridWaitNs) {
      atomicExch(&c->abort, 1);
      atomicCAS(&c->status, 0, (int)OTG_ERR_TIMEOUT);
      return false;
    }
  }
}

// Order-free relax of Pin::_relax_slew/_relax_at (MIN keeps the smallest,
// MAX the largest) and Pin::_relax_rat (the other way round); NaN is the
// empty value and loses to any number.
__device__ __forceinline__ float relax_fwd(int el, float cur, float v) {
  return el == MIN_ ? fminf(cur, v) : fmaxf(cur, v);
}
__device__ __forceinline__ float relax_bwd(int el, float cur, float v) {
  return el == MIN_ ? fmaxf(cur, v) : fminf(cur, v);
}

// Forward at pin v (one warp): Timer::_fprop_slew, _fprop_delay, _fprop_at
// and _fprop_test.  Lane j of a pass takes fanin arc j/8 and the combination
// (el, frf, trf) = bits (2, 1, 0) of j; its slew and arrival candidates go to
// output corner (el, trf).  Returns false if a wait gave up.
__device__ bool fprop_warp(const G& G_, const LutSrc& lutd, int v, int lane, float* at,
                           float* slew, float* rat, float* arc_delay, float* test_rat,
                           GridCtl* ctl) {
  const otg_prop_graph& g = G_.g;
  const int el = (lane >> 2) & 1, frf = (lane >> 1) & 1, trf = lane & 1;
  const int c_out = 2 * el + trf;
  const int f0 = __ldg(g.fanin_start + v), nitems = 8 * (__ldg(g.fanin_start + v + 1) - f0);
  // a primary input's assertions (NaN: none) seed the lanes with frf 0 of
  // the first pass, one per output corner
  float sl = nanf(""), a = nanf("");
  if (lane < 8 && frf == 0) {
    sl = __ldg(g.pi_slew + 4 * v + c_out);
    a = __ldg(g.pi_at + 4 * v + c_out);
  }
  bool ok = true;
  for (int j = lane; j < nitems; j += 32) {
    const int arc = __ldg(g.fanin + f0 + (j >> 3));
    const int u = __ldg(g.arc_from + arc);
    const int kind = __ldg(g.arc_kind + arc);
    float d = nanf(""), so = nanf(""), imp = nanf("");
    Lut ls = no_lut(), ld = no_lut();
    float load = 0.0f;
    int s = -1;
    if (kind == 0) {
      s = frf == trf ? rc_slot(G_, arc) : -1;
      if (s >= 0) {
        imp = __ldg(G_.rc.impulse + 4 * (size_t)s + c_out);
        d = __ldg(G_.rc.delay + 4 * (size_t)s + c_out);
      }
    }
    // A cell arc out of a pin whose only fanin is a net arc (a gate's input
    // pin) reads through it: the lane waits on the net's driver and derives
    // the input pin's slew and arrival time at (el, frf) exactly as that
    // pin's own warp does (one candidate relaxed against the assertion).
    // The input pin still stores its own values; this only shortens the
    // chain of waits.
    int src = u;
    bool thru = false;
    float t_imp = 0.0f, t_d = nanf(""), t_psl = nanf(""), t_pat = nanf("");
    int t_s = -1;
    if (kind != 0) {
      const int t = __ldg(g.arc_timing + 2 * arc + el);
      ls = timing_lut(G_, t, 1, frf, trf);
      ld = timing_lut(G_, t, 0, frf, trf);
      const int net = __ldg(g.arc_net + arc);
      if (net >= 0 && t >= 0)
        load = __ldg(G_.rc.load + 4 * (size_t)__ldg(G_.rc.nodes_start + net) + c_out);
      const int uf0 = __ldg(g.fanin_start + u);
      if (__ldg(g.fanin_start + u + 1) - uf0 == 1) {
        const int a0 = __ldg(g.fanin + uf0);
        if (__ldg(g.arc_kind + a0) == 0) {
          const int c_in = 2 * el + frf;
          thru = true;
          src = __ldg(g.arc_from + a0);
          t_s = rc_slot(G_, a0);
          if (t_s >= 0) {
            t_imp = __ldg(G_.rc.impulse + 4 * (size_t)t_s + c_in);
            t_d = __ldg(G_.rc.delay + 4 * (size_t)t_s + c_in);
          }
          t_psl = __ldg(g.pi_slew + 4 * u + c_in);
          t_pat = __ldg(g.pi_at + 4 * u + c_in);
        }
      }
    }
    float si, fa;
    if (!wait_values(slew + 4 * src + 2 * el + frf, at + 4 * src + 2 * el + frf, si, fa, ctl)) {
      ok = false;
      break;
    }
    if (thru) {
      float so_u = nanf(""), at_u = nanf("");
      if (t_s >= 0 && !none(si)) {
        const float r = sqrtf(__fadd_rn(__fmul_rn(si, si), t_imp));
        so_u = si < 0.0f ? -r : r;
      }
      if (!none(fa) && !none(t_d)) at_u = __fadd_rn(t_d, fa);
      si = relax_fwd(el, t_psl, so_u);
      fa = relax_fwd(el, t_pat, at_u);
    }
    if (kind == 0) {
      // sign(si) * sqrt(si^2 + impulse) at the sink (FlatRct::slew)
      if (s >= 0 && !none(si)) {
        const float r = sqrtf(__fadd_rn(__fmul_rn(si, si), imp));
        so = si < 0.0f ? -r : r;
      }
    } else if (!none(si)) {
      so = timing_value(lutd, ls, si, load);
      d = timing_value(lutd, ld, si, load);
    } else {
      d = nanf("");
    }
    arc_delay[8 * (size_t)arc + (j & 7)] = d;
    sl = relax_fwd(el, sl, so);
    if (!none(fa) && !none(d)) a = relax_fwd(el, a, __fadd_rn(d, fa));
  }
  ok = __all_sync(FULL, ok);
  if (!ok) return false;
  // lanes sharing (el, trf) differ in bits 1, 3 and 4
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int m = k == 0 ? 2 : (k == 1 ? 8 : 16);
    sl = relax_fwd(el, sl, __shfl_xor_sync(FULL, sl, m));
    a = relax_fwd(el, a, __shfl_xor_sync(FULL, a, m));
  }
  // corner c's result sits in lane 4 * (c >> 1) + (c & 1); lane 0 stores
  // the pin's slew and arrival time, which releases its readers, and marks
  // its required time pending for the backward pass (the arc delays and
  // test RATs are read only after the grid barrier)
  float slc[4], atc[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    slc[c] = canon(__shfl_sync(FULL, sl, 4 * (c >> 1) + (c & 1)));
    atc[c] = canon(__shfl_sync(FULL, a, 4 * (c >> 1) + (c & 1)));
  }
  if (lane == 0) {
    st_relaxed4(slew + 4 * v, slc[0], slc[1], slc[2], slc[3]);
    st_relaxed4(at + 4 * v, atc[0], atc[1], atc[2], atc[3]);
    const float p = __uint_as_float(kPending);
    reinterpret_cast<float4*>(rat)[v] = make_float4(p, p, p, p);
  }
  // timing tests constrained at v (Test::_fprop_rat): lane j of a pass takes
  // test j/4 and output corner j%4
  const int t0 = __ldg(g.test_start + v), ntest = 4 * (__ldg(g.test_start + v + 1) - t0);
  for (int j = lane; j < ntest; j += 32) {
    const int test = __ldg(g.test_of_pin + t0 + (j >> 2));
    const int arc = __ldg(g.test_arc + test), u = __ldg(g.arc_from + arc);
    const int tel = (j >> 1) & 1, rf = j & 1;
    const int t = __ldg(g.arc_timing + 2 * arc + tel);
    float val = nanf("");
    if (!none(g.period) && t >= 0) {
      const int edge = __ldg(g.timing + 9 * t + 1);
      const int fel = tel == MIN_ ? MAX_ : MIN_;
      const int rrf = edge == 1 ? RISE_ : FALL_;
      const float csl = slc[2 * tel + rf];
      if (!(rrf == FALL_ && edge != 2) && !none(csl)) {
        const Lut lc = timing_lut(G_, t, 2, rrf, rf);
        float rat_at, rsl;
        if (!wait_values(at + 4 * u + 2 * fel + rrf, slew + 4 * u + 2 * fel + rrf, rat_at, rsl,
                         ctl)) {
          ok = false;
          break;
        }
        if (!none(rat_at) && !none(rsl)) {
          const float related = tel == MIN_ ? rat_at : __fadd_rn(rat_at, g.period);
          const float cons = timing_value(lutd, lc, rsl, csl);
          if (!none(cons))
            val = tel == MIN_ ? __fadd_rn(cons, related) : __fsub_rn(related, cons);
        }
      }
    }
    test_rat[4 * (size_t)test + (j & 3)] = val;
  }
  return __all_sync(FULL, ok);
}

// Backward at pin v (one warp): Timer::_bprop_rat and the slack.  Lanes
// first take the tests constrained at v (4 corners each), then the fanout
// arcs (8 combinations each); every candidate lands in a 4-corner register
// set reduced over the whole warp.
__device__ bool bprop_warp(const G& G_, int v, int lane, const float* at, float* rat, float* slack,
                           const float* arc_delay, const float* test_rat, GridCtl* ctl) {
  const otg_prop_graph& g = G_.g;
  float r[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) r[c] = lane == 0 ? __ldg(g.po_rat + 4 * v + c) : nanf("");
  const int t0 = __ldg(g.test_start + v), ntest = 4 * (__ldg(g.test_start + v + 1) - t0);
  const int o0 = __ldg(g.fanout_start + v), nitems = ntest + 8 * (__ldg(g.fanout_start + v + 1) - o0);
  bool ok = true;
  for (int j = lane; j < nitems; j += 32) {
    int tc = 0;  // target corner
    float cand = nanf("");
    if (j < ntest) {
      tc = j & 3;
      cand = __ldcg(test_rat + 4 * (size_t)__ldg(g.test_of_pin + t0 + (j >> 2)) + tc);
    } else {
      const int jj = j - ntest;
      const int arc = __ldg(g.fanout + o0 + (jj >> 3)), w = __ldg(g.arc_to + arc);
      const int el = (jj >> 2) & 1, frf = (jj >> 1) & 1, trf = jj & 1;
      const int kind = __ldg(g.arc_kind + arc);
      const float* d = arc_delay + 8 * (size_t)arc;
      int mode = 0;  // 0 none, 1 propagation, 2 MIN constraint, 3 MAX constraint
      if (kind == 0) {
        mode = frf == trf ? 1 : 0;
      } else {
        const int t = __ldg(g.arc_timing + 2 * arc + el);
        if (t >= 0) {
          const int* tr = g.timing + 9 * t;
          if (!__ldg(tr + 2)) mode = 1;
          else if (transition_defined(tr, frf, trf)) mode = el == MIN_ ? 2 : 3;
        }
      }
      if (mode != 0) {
        // the fanout's required time this combination reads
        const int wc = mode == 1 ? 2 * el + trf : (mode == 2 ? trf : 2 + trf);
        // arc delays and arrival times are final since the forward pass, so
        // they are loaded before the wait and arrive during it
        float dl = nanf(""), a = nanf(""), wa = nanf("");
        if (mode == 1) {
          dl = __ldcg(d + 4 * el + 2 * frf + trf);
        } else {
          const int ael = mode == 2 ? MAX_ : MIN_, wel = mode == 2 ? MIN_ : MAX_;
          a = __ldcg(at + 4 * v + 2 * ael + frf);
          wa = __ldcg(at + 4 * w + 2 * wel + trf);
        }
        float wr;
        if (!wait_value(rat + 4 * w + wc, wr, ctl)) {
          ok = false;
          break;
        }
        if (mode == 1) {
          tc = 2 * el + frf;
          if (!none(wr) && !none(dl)) cand = __fsub_rn(wr, dl);
        } else if (mode == 2) {  // hold-like: w's MIN slack moves v's MAX rat
          tc = 2 * MAX_ + frf;
          if (!none(a) && !none(wa) && !none(wr)) cand = __fadd_rn(a, __fsub_rn(wa, wr));
        } else {  // setup-like: w's MAX slack moves v's MIN rat
          tc = 2 * MIN_ + frf;
          if (!none(a) && !none(wa) && !none(wr)) cand = __fsub_rn(a, __fsub_rn(wr, wa));
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (c == tc) r[c] = relax_bwd(c >> 1, r[c], cand);
  }
  ok = __all_sync(FULL, ok);
  if (!ok) return false;
#pragma unroll
  for (int c = 0; c < 4; ++c)
#pragma unroll
    for (int m = 1; m < 32; m <<= 1) r[c] = relax_bwd(c >> 1, r[c], __shfl_xor_sync(FULL, r[c], m));
  if (lane == 0) {
    st_relaxed4(rat + 4 * v, canon(r[0]), canon(r[1]), canon(r[2]), canon(r[3]));
    const float4 a4 = __ldcg(reinterpret_cast<const float4*>(at) + v);
    const float a[4] = {a4.x, a4.y, a4.z, a4.w};
    float sk[4];
#pragma unroll
    for (int c = 0; c < 4; ++c)
      sk[c] = (none(a[c]) || none(r[c])) ? __uint_as_float(kEmpty)
              : (c < 2 ? __fsub_rn(a[c], r[c]) : __fsub_rn(r[c], a[c]));
    reinterpret_cast<float4*>(slack)[v] = make_float4(sk[0], sk[1], sk[2], sk[3]);
  }
  return true;
}

// Marks every arrival time and slew pending and clears the control block.
// (pin_group: only the pins whose group is active, see otg_propagate_groups.)
__device__ __forceinline__ bool pin_on(const int32_t* pin_group, const uint8_t* group_active,
                                       int v) {
  return !pin_group || group_active[__ldg(pin_group + v)];
}

// (items: only the listed pins, see otg_propagate_items; num_pins is then
// the list's length.)
__global__ void prop_init_kernel(float4* at, float4* slew, int num_pins, GridCtl* ctl,
                                 const int32_t* pin_group, const uint8_t* group_active,
                                 const int32_t* items, int all_pins) {
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (i0 == 0 && !items) *ctl = GridCtl{0u, 0u, 0, 0};
  const float p = __uint_as_float(kPending);
  for (int k = i0; k < num_pins; k += gridDim.x * blockDim.x) {
    const int i = items ? __ldg(items + k) : k;
    if (items && (unsigned)i >= (unsigned)all_pins) {
      atomicCAS(&ctl->status, 0, (int)OTG_ERR_INVALID);  // reported; the passes skip it
      continue;
    }
    if (!pin_on(pin_group, group_active, i)) continue;
    at[i] = make_float4(p, p, p, p);
    slew[i] = make_float4(p, p, p, p);
  }
}

// The whole propagation in one cooperative launch; warp w of W takes items
// w, w + W, ... of each pass.
__global__ void __launch_bounds__(256) prop_kernel(G G_, const int* order, const int* fwd_order,
                                                   int num_pins,
                                                   float* at, float* slew, float* rat,
                                                   float* slack, float* arc_delay,
                                                   float* test_rat, GridCtl* ctl, int lut_smem,
                                                   const int32_t* pin_group,
                                                   const uint8_t* group_active) {
  // the library's tables, staged on chip when the caller gave their size
  // and they fit (lut_smem floats)
  extern __shared__ float s_lut[];
  for (int i = threadIdx.x; i < lut_smem; i += blockDim.x) s_lut[i] = __ldg(G_.g.lut_data + i);
  __syncthreads();
  const LutSrc lutd{s_lut, lut_smem, G_.g.lut_data};
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int W = (gridDim.x * blockDim.x) >> 5;
  bool ok = true;
  for (int j = warp; ok && j < num_pins; j += W) {
    const int v = fwd_order ? __ldg(fwd_order + j) : __ldg(order + num_pins - 1 - j);
    if ((unsigned)v >= (unsigned)G_.g.num_pins) continue;  // a bad item (reported by the fill)
    if (!pin_on(pin_group, group_active, v)) continue;
    ok = fprop_warp(G_, lutd, v, lane, at, slew, rat, arc_delay, test_rat, ctl);
  }
  // the barrier also lets every CTA leave together when a wait gave up
  if (!grid_barrier(ctl) || !ok) return;
  for (int j = warp; ok && j < num_pins; j += W) {
    const int v = __ldg(order + j);
    if ((unsigned)v >= (unsigned)G_.g.num_pins) continue;
    if (!pin_on(pin_group, group_active, v)) continue;
    ok = bprop_warp(G_, v, lane, at, rat, slack, arc_delay, test_rat, ctl);
  }
}

size_t align256p(size_t x) { return (x + 255) & ~(size_t)255; }

// Tables up to this many floats are staged in shared memory (40 KB per
// CTA keeps five 256-thread CTAs per SM; a library with three drive
// strengths of its combinational cells takes about 33 KB).
constexpr int kLutSmemFloats = 10240;

struct PropDev {
  int sms = 0;
  int occ[2] = {0, 0};  // CTAs per SM without / with the staged tables
  bool init = false;
};
PropDev g_pdev[64];

}  // namespace
}  // namespace otg

extern "C" {

otg_status otg_prop_workspace_size(int32_t num_pins, int32_t num_arcs, int32_t num_tests,
                                   size_t* bytes) {
  if (!bytes || num_pins < 0 || num_arcs < 0 || num_tests < 0) return OTG_ERR_INVALID;
  *bytes = 256 + otg::align256p(32 * (size_t)num_arcs) + otg::align256p(16 * (size_t)num_tests);
  return OTG_OK;
}

// items (with num_items): propagate only the listed pins, `order` and
// fwd_order unused (see otg_propagate_items).
static otg_status propagate_impl(const otg_prop_graph* g, const otg_prop_rc* rc,
                                 const int32_t* order, const int32_t* fwd_order,
                                 const int32_t* pin_group, const uint8_t* group_active, float* at,
                                 float* slew, float* rat, float* slack, void* workspace,
                                 size_t workspace_bytes, otg_stream_t stream,
                                 const int32_t* items = nullptr, int num_items = 0) {
  if (items) {
    if (num_items < 0) return OTG_ERR_INVALID;
    order = items;
    fwd_order = nullptr;
  }
  if (!g || !rc || !order || !at || !slew || !rat || !slack || !workspace || g->num_pins < 0)
    return OTG_ERR_INVALID;
  // lut_meta rows and the per-pin [4] rows are read and written as 16-byte vectors
  if ((((uintptr_t)g->lut_meta | (uintptr_t)at | (uintptr_t)slew | (uintptr_t)rat |
        (uintptr_t)slack) & 15) != 0 || ((uintptr_t)workspace & 255) != 0)
    return OTG_ERR_INVALID;
  size_t need = 0;
  otg_prop_workspace_size(g->num_pins, g->num_arcs, g->num_tests, &need);
  if (workspace_bytes < need) return OTG_ERR_WORKSPACE;
  const int P = items ? num_items : g->num_pins;  // the items the two passes take
  char* ws = (char*)workspace;
  otg::GridCtl* ctl = (otg::GridCtl*)ws;
  float* arc_delay = (float*)(ws + 256);
  float* test_rat = (float*)(ws + 256 + otg::align256p(32 * (size_t)g->num_arcs));
  cudaStream_t st = (cudaStream_t)stream;
  // with items, the fill may record a bad item, so the control block is
  // cleared before it (without items the fill clears it itself)
  if (items && cudaMemsetAsync(ctl, 0, sizeof(otg::GridCtl), st) != cudaSuccess) return OTG_ERR_CUDA;
  otg::prop_init_kernel<<<std::max(1, std::min(1184, (P + 255) / 256)), 256, 0, st>>>(
      (float4*)at, (float4*)slew, P, ctl, pin_group, group_active, items, g->num_pins);
  otg::count_launch();
  if (cudaGetLastError() != cudaSuccess) return OTG_ERR_CUDA;
  if (P == 0) return OTG_OK;
  int dev = 0;
  cudaGetDevice(&dev);
  otg::PropDev& d = otg::g_pdev[dev & 63];
  if (!d.init) {
    cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(otg::prop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         4 * otg::kLutSmemFloats);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ[0], otg::prop_kernel, 256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ[1], otg::prop_kernel, 256,
                                                  4 * otg::kLutSmemFloats);
    d.init = true;
  }
  int lut_smem = g->num_lut_data > 0 && g->num_lut_data <= otg::kLutSmemFloats ? g->num_lut_data : 0;
  const int occ = lut_smem ? d.occ[1] : d.occ[0];
  // every CTA resident (the schedule and the barrier rely on it), no more
  // warps than pins
  const int grid = std::max(1, std::min(d.sms * std::max(occ, 1), (P + 7) / 8));
  otg::G G_{*g, *rc};
  int num_pins = P;
  void* args[] = {&G_,       (void*)&order, (void*)&fwd_order, &num_pins,
                  &at,       &slew,         &rat,              &slack,
                  &arc_delay, &test_rat,    &ctl,              &lut_smem,
                  (void*)&pin_group, (void*)&group_active};
  const cudaError_t e = cudaLaunchCooperativeKernel(
      (const void*)otg::prop_kernel, dim3(grid), dim3(256), args, 4 * (size_t)lut_smem, st);
  otg::count_launch();
  if (e != cudaSuccess) {
    cudaGetLastError();
    return OTG_ERR_CUDA;
  }
  return OTG_OK;
}

otg_status otg_propagate(const otg_prop_graph* g, const otg_prop_rc* rc, const int32_t* order,
                         const int32_t* fwd_order, float* at, float* slew, float* rat,
                         float* slack, void* workspace, size_t workspace_bytes,
                         otg_stream_t stream) {
  return propagate_impl(g, rc, order, fwd_order, nullptr, nullptr, at, slew, rat, slack,
                        workspace, workspace_bytes, stream);
}

otg_status otg_propagate_groups(const otg_prop_graph* g, const otg_prop_rc* rc,
                                const int32_t* order, const int32_t* fwd_order,
                                const int32_t* pin_group, const uint8_t* group_active,
                                float* at, float* slew, float* rat, float* slack,
                                void* workspace, size_t workspace_bytes, otg_stream_t stream) {
  if (!pin_group || !group_active) return OTG_ERR_INVALID;
  return propagate_impl(g, rc, order, fwd_order, pin_group, group_active, at, slew, rat, slack,
                        workspace, workspace_bytes, stream);
}

otg_status otg_propagate_items(const otg_prop_graph* g, const otg_prop_rc* rc,
                               const int32_t* items, int32_t num_items, float* at, float* slew,
                               float* rat, float* slack, void* workspace, size_t workspace_bytes,
                               otg_stream_t stream) {
  if (!items && num_items > 0) return OTG_ERR_INVALID;
  if (num_items <= 0) {  // nothing to propagate; the status word still reads OK
    if (num_items < 0 || !workspace) return OTG_ERR_INVALID;
    return cudaMemsetAsync(workspace, 0, sizeof(otg::GridCtl), (cudaStream_t)stream) ==
                   cudaSuccess
               ? OTG_OK
               : OTG_ERR_CUDA;
  }
  return propagate_impl(g, rc, nullptr, nullptr, nullptr, nullptr, at, slew, rat, slack,
                        workspace, workspace_bytes, stream, items, num_items);
}

otg_status otg_prop_arc_delays(const void* workspace, size_t workspace_bytes, int32_t num_arcs,
                               const float** arc_delay) {
  if (!workspace || !arc_delay || num_arcs < 0) return OTG_ERR_INVALID;
  if (workspace_bytes < 256 + 32 * (size_t)num_arcs) return OTG_ERR_WORKSPACE;
  *arc_delay = (const float*)((const char*)workspace + 256);
  return OTG_OK;
}

otg_status otg_prop_status(const void* workspace, otg_stream_t stream) {
  if (!workspace) return OTG_ERR_INVALID;
  otg::GridCtl h;
  if (cudaMemcpyAsync(&h, workspace, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream) !=
          cudaSuccess ||
      cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) {
    cudaGetLastError();
    return OTG_ERR_CUDA;
  }
  return (otg_status)h.status;
}

}  // extern "C"
