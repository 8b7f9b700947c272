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
// Order: one launch per level, a thread per pin; the levels come from
// otg_levelize over the same graph (a pin's fanins sit on higher levels,
// its fanouts on lower ones), forward from the last level to the first,
// backward from the first to the last.
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

__device__ int lower_bound(const float* a, int n, float v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// meta: n1, n2, offset, variable order (unused here)
__device__ float lut_eval(const int* meta, const float* data, float v1, float v2) {
  const int n1 = meta[0], n2 = meta[1];
  const float* i1 = data + meta[2];
  const float* i2 = i1 + n1;
  const float* tb = i2 + n2;
  if (n1 < 1 || n2 < 1) return nanf("");
  if (n1 == 1 && n2 == 1) return tb[0];
  const int a1 = max(1, min(lower_bound(i1, n1, v1), n1 - 1));
  const int a2 = max(1, min(lower_bound(i2, n2, v2), n2 - 1));
  if (n1 == 1) return interpolate(v2, i2[a2 - 1], i2[a2], tb[a2 - 1], tb[a2]);
  if (n2 == 1) return interpolate(v1, i1[a1 - 1], i1[a1], tb[(a1 - 1) * n2], tb[a1 * n2]);
  const float lo = interpolate(v1, i1[a1 - 1], i1[a1], tb[(a1 - 1) * n2 + a2 - 1],
                               tb[a1 * n2 + a2 - 1]);
  const float hi = interpolate(v1, i1[a1 - 1], i1[a1], tb[(a1 - 1) * n2 + a2], tb[a1 * n2 + a2]);
  return interpolate(v2, i2[a2 - 1], i2[a2], lo, hi);
}

struct G {
  otg_prop_graph g;
  otg_prop_rc rc;
};

// timing record: [sense, edge, constraint, lut x6]
__device__ bool transition_defined(const int* tr, int irf, int orf) {
  const int edge = tr[1];
  if (edge == 1 && irf != RISE_) return false;
  if (edge == 2 && irf != FALL_) return false;
  if (tr[0] == 0 && irf != orf) return false;  // positive unate
  if (tr[0] == 1 && irf == orf) return false;  // negative unate
  return true;
}

// which = 0 delay, 1 slew, 2 constraint; (a, b) = (slew, load) for delay and
// slew, (related slew, constrained slew) for constraint
__device__ float timing_query(const G& G_, int t, int which, int irf, int orf, float a, float b) {
  const int* tr = G_.g.timing + 9 * t;
  if (!transition_defined(tr, irf, orf)) return nanf("");
  const int lut = tr[3 + 2 * which + orf];
  if (lut < 0) return nanf("");
  const int* meta = G_.g.lut_meta + 4 * lut;
  const int var = meta[3];
  if (var < 0) {  // no template: a scalar only
    if (meta[0] == 1 && meta[1] == 1) return G_.g.lut_data[meta[2] + 2];
    return nanf("");
  }
  // var 0: (slew | related) first; var 1: (load | constrained) first
  return var == 0 ? lut_eval(meta, G_.g.lut_data, a, b) : lut_eval(meta, G_.g.lut_data, b, a);
}

__device__ __forceinline__ float rc_load(const G& G_, int net, int el, int trf) {
  if (net < 0) return 0.0f;
  return G_.rc.load[4 * (size_t)G_.rc.nodes_start[net] + 2 * el + trf];
}

// RC node of a net arc's sink: global BFS slot (-1: none)
__device__ __forceinline__ int rc_slot(const G& G_, int arc) {
  const int node = G_.g.arc_node[arc];
  if (node < 0) return -1;
  const int net = G_.g.arc_net[arc];
  return G_.rc.nodes_start[net] + G_.rc.node2bfs[node];
}

__device__ __forceinline__ void relax_min(float& cur, float v) {
  if (none(cur) || v < cur) cur = v;
}
__device__ __forceinline__ void relax_max(float& cur, float v) {
  if (none(cur) || v > cur) cur = v;
}

__global__ void fprop_kernel(G G_, const int* order, int lo, int hi, float* at, float* slew,
                             float* arc_delay, float* test_rat) {
  const otg_prop_graph& g = G_.g;
  for (int idx = lo + blockIdx.x * blockDim.x + threadIdx.x; idx < hi;
       idx += gridDim.x * blockDim.x) {
    const int v = order[idx];
    float sl[4], a[4];
    for (int c = 0; c < 4; ++c) {
      sl[c] = g.pi_slew[4 * v + c];  // a primary input's assertion (NaN: none)
      a[c] = g.pi_at[4 * v + c];
    }
    const int f0 = g.fanin_start[v], f1 = g.fanin_start[v + 1];
    // slew
    for (int k = f0; k < f1; ++k) {
      const int arc = g.fanin[k], u = g.arc_from[arc];
      if (g.arc_kind[arc] == 0) {
        const int s = rc_slot(G_, arc);
        for (int c = 0; c < 4; ++c) {
          const float si = slew[4 * u + c];
          if (none(si) || s < 0) continue;
          const float imp = G_.rc.impulse[4 * (size_t)s + c];
          const float r = sqrtf(__fadd_rn(__fmul_rn(si, si), imp));
          const float so = si < 0.0f ? -r : r;
          if (c < 2) relax_min(sl[c], so); else relax_max(sl[c], so);
        }
      } else {
        for (int el = 0; el < 2; ++el) {
          const int t = g.arc_timing[2 * arc + el];
          if (t < 0) continue;
          for (int frf = 0; frf < 2; ++frf) {
            const float si = slew[4 * u + 2 * el + frf];
            if (none(si)) continue;
            for (int trf = 0; trf < 2; ++trf) {
              const float so = timing_query(G_, t, 1, frf, trf, si,
                                            rc_load(G_, g.arc_net[arc], el, trf));
              if (none(so)) continue;
              if (el == MIN_) relax_min(sl[2 * el + trf], so);
              else relax_max(sl[2 * el + trf], so);
            }
          }
        }
      }
    }
    for (int c = 0; c < 4; ++c) slew[4 * v + c] = sl[c];
    // arc delays and arrival times
    for (int k = f0; k < f1; ++k) {
      const int arc = g.fanin[k], u = g.arc_from[arc];
      float* d = arc_delay + 8 * (size_t)arc;  // [el][frf][trf]
      for (int j = 0; j < 8; ++j) d[j] = nanf("");
      if (g.arc_kind[arc] == 0) {
        const int s = rc_slot(G_, arc);
        for (int el = 0; el < 2; ++el)
          for (int rf = 0; rf < 2; ++rf)
            d[4 * el + 2 * rf + rf] = s < 0 ? nanf("") : G_.rc.delay[4 * (size_t)s + 2 * el + rf];
      } else {
        for (int el = 0; el < 2; ++el) {
          const int t = g.arc_timing[2 * arc + el];
          if (t < 0) continue;
          for (int frf = 0; frf < 2; ++frf) {
            const float si = slew[4 * u + 2 * el + frf];
            if (none(si)) continue;
            for (int trf = 0; trf < 2; ++trf)
              d[4 * el + 2 * frf + trf] =
                  timing_query(G_, t, 0, frf, trf, si, rc_load(G_, g.arc_net[arc], el, trf));
          }
        }
      }
      for (int el = 0; el < 2; ++el)
        for (int frf = 0; frf < 2; ++frf) {
          const float fa = at[4 * u + 2 * el + frf];
          if (none(fa)) continue;
          for (int trf = 0; trf < 2; ++trf) {
            const float dl = d[4 * el + 2 * frf + trf];
            if (none(dl)) continue;
            const float val = __fadd_rn(dl, fa);
            if (el == MIN_) relax_min(a[2 * el + trf], val);
            else relax_max(a[2 * el + trf], val);
          }
        }
    }
    for (int c = 0; c < 4; ++c) at[4 * v + c] = a[c];
    // timing tests constrained at v (Test::_fprop_rat)
    for (int k = g.test_start[v]; k < g.test_start[v + 1]; ++k) {
      const int test = g.test_of_pin[k], arc = g.test_arc[test], u = g.arc_from[arc];
      float* tr = test_rat + 4 * (size_t)test;
      for (int c = 0; c < 4; ++c) tr[c] = nanf("");
      if (none(g.period)) continue;
      for (int el = 0; el < 2; ++el) {
        const int t = g.arc_timing[2 * arc + el];
        if (t < 0) continue;
        const int edge = g.timing[9 * t + 1];
        const int fel = el == MIN_ ? MAX_ : MIN_;
        const int frf = edge == 1 ? RISE_ : FALL_;
        if (frf == FALL_ && edge != 2) continue;
        for (int rf = 0; rf < 2; ++rf) {
          if (none(sl[2 * el + rf])) continue;
          const float rat_at = at[4 * u + 2 * fel + frf], rsl = slew[4 * u + 2 * fel + frf];
          if (none(rat_at) || none(rsl)) continue;
          const float related = el == MIN_ ? rat_at : __fadd_rn(rat_at, g.period);
          const float cons = timing_query(G_, t, 2, frf, rf, rsl, sl[2 * el + rf]);
          if (none(cons)) continue;
          tr[2 * el + rf] = el == MIN_ ? __fadd_rn(cons, related) : __fsub_rn(related, cons);
        }
      }
    }
  }
}

__global__ void bprop_kernel(G G_, const int* order, int lo, int hi, const float* at,
                             float* rat, float* slack, const float* arc_delay,
                             const float* test_rat) {
  const otg_prop_graph& g = G_.g;
  for (int idx = lo + blockIdx.x * blockDim.x + threadIdx.x; idx < hi;
       idx += gridDim.x * blockDim.x) {
    const int v = order[idx];
    float r[4];
    for (int c = 0; c < 4; ++c) r[c] = g.po_rat[4 * v + c];  // a primary output's assertion
    // Pin::_relax_rat: the MIN split keeps the largest, MAX the smallest
    auto relax = [&](int el, int rf, float val) {
      if (el == MIN_) relax_max(r[2 * el + rf], val);
      else relax_min(r[2 * el + rf], val);
    };
    for (int k = g.test_start[v]; k < g.test_start[v + 1]; ++k) {
      const float* tr = test_rat + 4 * (size_t)g.test_of_pin[k];
      for (int c = 0; c < 4; ++c)
        if (!none(tr[c])) relax(c >> 1, c & 1, tr[c]);
    }
    for (int k = g.fanout_start[v]; k < g.fanout_start[v + 1]; ++k) {
      const int arc = g.fanout[k], w = g.arc_to[arc];
      const float* d = arc_delay + 8 * (size_t)arc;
      if (g.arc_kind[arc] == 0) {
        for (int el = 0; el < 2; ++el)
          for (int rf = 0; rf < 2; ++rf) {
            const float wr = rat[4 * w + 2 * el + rf], dl = d[4 * el + 2 * rf + rf];
            if (!none(wr) && !none(dl)) relax(el, rf, __fsub_rn(wr, dl));
          }
        continue;
      }
      for (int el = 0; el < 2; ++el) {
        const int t = g.arc_timing[2 * arc + el];
        if (t < 0) continue;
        const int* tr = g.timing + 9 * t;
        for (int frf = 0; frf < 2; ++frf)
          for (int trf = 0; trf < 2; ++trf) {
            if (!tr[2]) {  // a propagation arc
              const float wr = rat[4 * w + 2 * el + trf], dl = d[4 * el + 2 * frf + trf];
              if (!none(wr) && !none(dl)) relax(el, frf, __fsub_rn(wr, dl));
              continue;
            }
            if (!transition_defined(tr, frf, trf)) continue;  // a constraint arc
            if (el == MIN_) {
              const float a = at[4 * v + 2 * MAX_ + frf];
              const float wa = at[4 * w + trf], wr = rat[4 * w + trf];  // w's MIN slack
              if (!none(a) && !none(wa) && !none(wr))
                relax(MAX_, frf, __fadd_rn(a, __fsub_rn(wa, wr)));
            } else {
              const float a = at[4 * v + 2 * MIN_ + frf];
              const float wa = at[4 * w + 2 + trf], wr = rat[4 * w + 2 + trf];  // w's MAX slack
              if (!none(a) && !none(wa) && !none(wr))
                relax(MIN_, frf, __fsub_rn(a, __fsub_rn(wr, wa)));
            }
          }
      }
    }
    for (int c = 0; c < 4; ++c) {
      rat[4 * v + c] = r[c];
      const float a = at[4 * v + c];
      slack[4 * v + c] = (none(a) || none(r[c])) ? nanf("")
                         : (c < 2 ? __fsub_rn(a, r[c]) : __fsub_rn(r[c], a));
    }
  }
}

size_t align256p(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace
}  // namespace otg

extern "C" {

otg_status otg_prop_workspace_size(int32_t num_arcs, int32_t num_tests, size_t* bytes) {
  if (!bytes || num_arcs < 0 || num_tests < 0) return OTG_ERR_INVALID;
  *bytes = otg::align256p(32 * (size_t)num_arcs) + otg::align256p(16 * (size_t)num_tests) + 256;
  return OTG_OK;
}

otg_status otg_propagate(const otg_prop_graph* g, const otg_prop_rc* rc, const int32_t* order,
                         const int32_t* level_ends, int32_t num_levels, float* at, float* slew,
                         float* rat, float* slack, void* workspace, size_t workspace_bytes,
                         otg_stream_t stream) {
  if (!g || !rc || !order || !level_ends || num_levels < 0 || !at || !slew || !rat || !slack ||
      !workspace)
    return OTG_ERR_INVALID;
  size_t need = 0;
  otg_prop_workspace_size(g->num_arcs, g->num_tests, &need);
  if (workspace_bytes < need) return OTG_ERR_WORKSPACE;
  float* arc_delay = (float*)workspace;
  float* test_rat = (float*)((char*)workspace + otg::align256p(32 * (size_t)g->num_arcs));
  cudaStream_t st = (cudaStream_t)stream;
  otg::G G_{*g, *rc};
  // at and slew start as "none": pins are written as their level runs, and
  // a pin only reads pins of higher levels
  auto grid = [](int n) { return std::max(1, std::min(1184, (n + 127) / 128)); };
  for (int L = num_levels - 1; L >= 0; --L) {
    const int lo = level_ends[L], hi = level_ends[L + 1];
    if (hi <= lo) continue;
    otg::fprop_kernel<<<grid(hi - lo), 128, 0, st>>>(G_, order, lo, hi, at, slew, arc_delay,
                                                      test_rat);
    otg::count_launch();
  }
  for (int L = 0; L < num_levels; ++L) {
    const int lo = level_ends[L], hi = level_ends[L + 1];
    if (hi <= lo) continue;
    otg::bprop_kernel<<<grid(hi - lo), 128, 0, st>>>(G_, order, lo, hi, at, rat, slack,
                                                      arc_delay, test_rat);
    otg::count_launch();
  }
  if (cudaGetLastError() != cudaSuccess) return OTG_ERR_CUDA;
  return OTG_OK;
}

}  // extern "C"
