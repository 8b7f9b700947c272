// otg_paths.cpp -- the K worst data paths of a propagated timing graph, as
// Timer::report_timing gives them (ot/timer/path.cpp:365-537, sfxt.cpp:
// 52-246, pfxt.cpp:67-149, endpoint.cpp:33-127), on the host over the
// device's results (arrival / required times, slacks, and every arc's
// delay per (split, from transition, to transition), otg_prop_arc_delays).
//
// Nodes are (pin, transition), encoded 2 * pin + transition; S is the
// super source.
//   endpoints   per (split, transition) the endpoint pins whose slack is
//               defined, sorted by slack (stable in pin order); K of them
//               by taking the smallest head, ties to the first list in the
//               order (MIN,RISE), (MIN,FALL), (MAX,RISE), (MAX,FALL);
//   suffix tree of endpoint T at split el: the fanin cone's depth-first
//               post-order from T, stopping at data-path sources; dist(T) =
//               +rat (late) / -rat (early); in reverse post-order, every
//               arc u -> v relaxes dist(u) with dist(v) + w, w = -delay
//               (late) / +delay (early), first minimum kept (strict <);
//               then S from every source s with dist(s) + (-at / +at);
//   K == 1      the worst endpoint's tree path with the endpoint's slack;
//   K > 1       per endpoint a min-heap of prefix-tree nodes (slack, from,
//               to, arc, parent): the sources first, then per popped path
//               every arc leaving it into the cone other than the tree's,
//               at dist(v) + w - dist(u) + slack; negative slacks only; the
//               K smallest over all endpoints, ascending;
//   points      (pin, transition, arrival): the source's arrival, then the
//               previous point's plus each arc's delay.
// Arithmetic in float32, in the reference's order of operations.
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <queue>
#include <vector>

#include "../../include/otg.h"

namespace {

constexpr int kS = -1;  // the super source

struct Link {
  int arc, frf, trf;
};

struct PfxNode {
  float slack;
  int from, to, arc, parent;  // parent: index into the endpoint's node list, -1 none
};

struct Search {
  const otg_path_graph& g;
  std::vector<int> fin_start, fin, fout_start, fout;
  // per-endpoint state, indexed by node; stamp marks the current endpoint
  std::vector<int> stamp, tree;
  std::vector<float> dist;
  std::vector<Link> link;
  int cur = 0;
  // the super source's state
  bool s_has = false;
  float s_dist = 0.0f;
  int s_tree = -1;

  explicit Search(const otg_path_graph& graph) : g(graph) {
    const int P = g.num_pins, A = g.num_arcs;
    fin_start.assign(P + 1, 0);
    fout_start.assign(P + 1, 0);
    for (int a = 0; a < A; ++a)
      if (!g.arc_is_test[a]) {
        ++fin_start[g.arc_to[a] + 1];
        ++fout_start[g.arc_from[a] + 1];
      }
    for (int p = 0; p < P; ++p) {
      fin_start[p + 1] += fin_start[p];
      fout_start[p + 1] += fout_start[p];
    }
    fin.resize(fin_start[P]);
    fout.resize(fout_start[P]);
    std::vector<int> ci(fin_start.begin(), fin_start.end() - 1);
    std::vector<int> co(fout_start.begin(), fout_start.end() - 1);
    for (int a = 0; a < A; ++a)  // arc order within a pin
      if (!g.arc_is_test[a]) {
        fin[ci[g.arc_to[a]]++] = a;
        fout[co[g.arc_from[a]]++] = a;
      }
    stamp.assign(2 * (size_t)P, 0);
    tree.assign(2 * (size_t)P, -1);
    dist.assign(2 * (size_t)P, 0.0f);
    link.assign(2 * (size_t)P, Link{-1, 0, 0});
  }

  float delay(int arc, int el, int frf, int trf) const {
    return g.arc_delay[8 * (size_t)arc + (el << 2) + (frf << 1) + trf];
  }
  float pin_value(const float* x, int pin, int c) const { return x[4 * (size_t)pin + c]; }
  bool has(int u) const { return u == kS ? s_has : stamp[u] == cur; }
  float get(int u) const { return u == kS ? s_dist : dist[u]; }

  void relax(int u, int v, Link l, float d) {
    if (u == kS) {
      if (!s_has || d < s_dist) {
        s_has = true;
        s_dist = d;
        s_tree = v;
      }
      return;
    }
    if (stamp[u] != cur || d < dist[u]) {
      stamp[u] = cur;
      dist[u] = d;
      tree[u] = v;
      link[u] = l;
    }
  }

  // Suffix tree of endpoint node t at split el; srcs receives the sources
  // in the order they are met with their offsets (NaN: no arrival).
  void sfxt(int t, int el, std::vector<std::pair<int, float>>& srcs) {
    ++cur;
    s_has = false;
    s_tree = -1;
    srcs.clear();
    // depth-first post-order over the cone (Timer::_topologize), with the
    // visit marks cleared afterwards
    std::vector<int> post;
    std::vector<char>& seen = seen_;
    if (seen.size() != stamp.size()) seen.assign(stamp.size(), 0);
    std::vector<int> touched;
    struct Frame {
      int v, k, rf;  // node, next fanin arc index, next from transition
    };
    std::vector<Frame> st;
    auto mark = [&](int v) {
      seen[v] = 1;
      touched.push_back(v);
      st.push_back(Frame{v, fin_start[v >> 1], 0});
    };
    mark(t);
    while (!st.empty()) {
      Frame& f = st.back();
      const int pin = f.v >> 1, vrf = f.v & 1;
      bool pushed = false;
      if (!g.pin_is_source[pin]) {
        while (f.k < fin_start[pin + 1]) {
          const int a = fin[f.k];
          const int urf = f.rf;
          if (++f.rf == 2) {
            f.rf = 0;
            ++f.k;
          }
          if (std::isnan(delay(a, el, urf, vrf))) continue;
          const int u = 2 * g.arc_from[a] + urf;
          if (!seen[u]) {
            mark(u);
            pushed = true;
            break;
          }
        }
      }
      if (!pushed) {
        post.push_back(st.back().v);
        st.pop_back();
      }
    }
    for (int v : touched) seen[v] = 0;
    const int T = t >> 1, rf = t & 1;
    const float rat = pin_value(g.rat, T, 2 * el + rf);
    stamp[t] = cur;
    dist[t] = el == 0 ? -rat : rat;
    tree[t] = -1;
    for (auto it = post.rbegin(); it != post.rend(); ++it) {
      const int v = *it, pin = v >> 1, vrf = v & 1;
      if (g.pin_is_source[pin]) {
        const float at = pin_value(g.at, pin, 2 * el + vrf);
        srcs.emplace_back(v, std::isnan(at) ? at : (el == 0 ? at : -at));
        continue;
      }
      const float dv = dist[v];
      for (int k = fin_start[pin]; k < fin_start[pin + 1]; ++k) {
        const int a = fin[k];
        for (int urf = 0; urf < 2; ++urf) {
          const float d = delay(a, el, urf, vrf);
          if (std::isnan(d)) continue;
          relax(2 * g.arc_from[a] + urf, v, Link{a, urf, vrf}, dv + (el == 0 ? d : -d));
        }
      }
    }
    for (const auto& [s, off] : srcs)
      if (!std::isnan(off)) relax(kS, s, Link{-1, 0, 0}, dist[s] + off);
  }

  std::vector<char> seen_;
};

struct OutPath {
  float slack;
  int pin, el, rf;
  std::vector<int> pins, trans;
  std::vector<float> ats;
};

void follow(const Search& s, int el, int u, int v, OutPath& p) {
  while (u != v) {
    const Link l = s.link[u];
    u = s.tree[u];
    p.pins.push_back(u >> 1);
    p.trans.push_back(u & 1);
    p.ats.push_back(p.ats.back() + s.delay(l.arc, el, l.frf, l.trf));
  }
}

void source_point(const Search& s, int el, int u, OutPath& p) {
  p.pins.push_back(u >> 1);
  p.trans.push_back(u & 1);
  p.ats.push_back(s.pin_value(s.g.at, u >> 1, 2 * el + (u & 1)));
}

}  // namespace

extern "C" otg_status otg_report_paths(const otg_path_graph* g, int32_t K, int32_t split,
                                       int32_t tran, int32_t* num_paths, float* path_slack,
                                       int32_t* path_endpoint, int32_t* path_start,
                                       int32_t max_points, int32_t* point_pin,
                                       int32_t* point_tran, float* point_at,
                                       int32_t* points_needed) {
  if (!g || K < 0 || !num_paths || split < -1 || split > 1 || tran < -1 || tran > 1 ||
      g->num_pins < 0 || g->num_arcs < 0 || g->num_endpoints < 0)
    return OTG_ERR_INVALID;
  if (K > 0 && (!path_slack || !path_endpoint || !path_start || !points_needed))
    return OTG_ERR_INVALID;
  if (g->num_pins > 0 && (!g->at || !g->rat || !g->slack || !g->pin_is_source))
    return OTG_ERR_INVALID;
  if (g->num_arcs > 0 && (!g->arc_from || !g->arc_to || !g->arc_is_test || !g->arc_delay))
    return OTG_ERR_INVALID;
  if (g->num_endpoints > 0 && !g->endpoints) return OTG_ERR_INVALID;
  for (int a = 0; a < g->num_arcs; ++a)
    if ((unsigned)g->arc_from[a] >= (unsigned)g->num_pins ||
        (unsigned)g->arc_to[a] >= (unsigned)g->num_pins)
      return OTG_ERR_INVALID;
  for (int e = 0; e < g->num_endpoints; ++e)
    if ((unsigned)g->endpoints[e] >= (unsigned)g->num_pins) return OTG_ERR_INVALID;
  *num_paths = 0;
  if (points_needed) *points_needed = 0;
  if (K == 0) return OTG_OK;

  // ---- the worst endpoints
  std::vector<std::pair<float, int>> lists[4];
  for (int el = 0; el < 2; ++el)
    for (int rf = 0; rf < 2; ++rf) {
      if ((split >= 0 && split != el) || (tran >= 0 && tran != rf)) continue;
      auto& L = lists[2 * el + rf];
      for (int e = 0; e < g->num_endpoints; ++e) {
        const float sl = g->slack[4 * (size_t)g->endpoints[e] + 2 * el + rf];
        if (!std::isnan(sl)) L.emplace_back(sl, g->endpoints[e]);
      }
      std::stable_sort(L.begin(), L.end(),
                       [](const auto& x, const auto& y) { return x.first < y.first; });
    }
  struct Ept {
    int pin, el, rf;
  };
  std::vector<Ept> epts;
  size_t head[4] = {0, 0, 0, 0};
  for (int k = 0; k < K; ++k) {
    int best = -1;
    for (int c = 0; c < 4; ++c)
      if (head[c] < lists[c].size() &&
          (best < 0 || lists[c][head[c]].first < lists[best][head[best]].first))
        best = c;
    if (best < 0) break;
    epts.push_back(Ept{lists[best][head[best]].second, best >> 1, best & 1});
    ++head[best];
  }
  if (epts.empty()) return OTG_OK;

  Search s(*g);
  std::vector<std::pair<int, float>> srcs;
  std::vector<OutPath> out;
  if (K == 1) {
    const Ept e = epts[0];
    s.sfxt(2 * e.pin + e.rf, e.el, srcs);
    OutPath p{s.pin_value(g->slack, e.pin, 2 * e.el + e.rf), e.pin, e.el, e.rf, {}, {}, {}};
    if (s.s_has) {
      source_point(s, e.el, s.s_tree, p);
      follow(s, e.el, s.s_tree, 2 * e.pin + e.rf, p);
    }
    out.push_back(std::move(p));
  } else {
    // the K best so far: a max-heap by slack; of equal slacks the one found
    // first is on top (evicted first)
    auto worse = [](const std::pair<float, int>& a, const std::pair<float, int>& b) {
      return a.first < b.first || (a.first == b.first && a.second > b.second);
    };
    std::priority_queue<std::pair<float, int>, std::vector<std::pair<float, int>>,
                        decltype(worse)>
        best(worse);
    std::vector<OutPath> kept;
    int seq = 0;
    for (const Ept& e : epts) {
      const int t = 2 * e.pin + e.rf;
      s.sfxt(t, e.el, srcs);
      std::vector<PfxNode> nodes;
      auto cmp = [&nodes](int a, int b) {  // min-heap by slack, ties by creation
        return nodes[a].slack > nodes[b].slack ||
               (nodes[a].slack == nodes[b].slack && a > b);
      };
      std::priority_queue<int, std::vector<int>, decltype(cmp)> pf(cmp);
      for (const auto& [src, off] : srcs) {
        if (std::isnan(off)) continue;
        const float sl = s.dist[src] + off;
        if (sl < 0.0f) {
          nodes.push_back(PfxNode{sl, kS, src, -1, -1});
          pf.push((int)nodes.size() - 1);
        }
      }
      for (int k = 0; k < K && !pf.empty(); ++k) {
        const int ni = pf.top();
        pf.pop();
        const PfxNode nd = nodes[ni];
        if ((int)best.size() >= K && best.top().first <= nd.slack) break;
        // the path: its chain of deviations from the source on
        OutPath p{nd.slack, e.pin, e.el, e.rf, {}, {}, {}};
        std::vector<int> chain;
        for (int c = ni; c >= 0; c = nodes[c].parent) chain.push_back(c);
        for (int c = (int)chain.size() - 1; c >= 0; --c) {
          const PfxNode& x = nodes[chain[c]];
          const int end = c > 0 ? nodes[chain[c - 1]].from : t;
          if (x.from == kS) {
            source_point(s, e.el, x.to, p);
          } else {
            p.pins.push_back(x.to >> 1);
            p.trans.push_back(x.to & 1);
            p.ats.push_back(p.ats.back() + s.delay(x.arc, e.el, p.trans[p.trans.size() - 2],
                                                   x.to & 1));
          }
          follow(s, e.el, x.to, end, p);
        }
        kept.push_back(std::move(p));
        best.push({nd.slack, seq++});
        if ((int)best.size() > K) best.pop();
        // spur: deviations along the popped path's tree part
        for (int u = nd.to; u != t; u = s.tree[u]) {
          const int pin = u >> 1, urf = u & 1;
          const float du = s.dist[u];
          for (int q = s.fout_start[pin]; q < s.fout_start[pin + 1]; ++q) {
            const int a = s.fout[q];
            for (int vrf = 0; vrf < 2; ++vrf) {
              const float d = s.delay(a, e.el, urf, vrf);
              if (std::isnan(d)) continue;
              const int v = 2 * g->arc_to[a] + vrf;
              if (!s.has(v)) continue;
              const Link l = s.link[u];
              if (l.arc == a && l.frf == urf && l.trf == vrf) continue;
              const float w = e.el == 0 ? d : -d;
              const float sl = s.dist[v] + w - du + nd.slack;
              if (sl < 0.0f) {
                nodes.push_back(PfxNode{sl, u, v, a, ni});
                pf.push((int)nodes.size() - 1);
              }
            }
          }
        }
      }
    }
    // the kept paths still in the heap, ascending by slack (ties: found first)
    std::vector<int> ids;
    while (!best.empty()) {
      ids.push_back(best.top().second);
      best.pop();
    }
    std::sort(ids.begin(), ids.end(), [&kept](int a, int b) {
      return kept[a].slack < kept[b].slack || (kept[a].slack == kept[b].slack && a < b);
    });
    for (int i : ids) out.push_back(std::move(kept[i]));
  }

  // ---- outputs
  int need = 0;
  for (const OutPath& p : out) need += (int)p.pins.size();
  *points_needed = need;
  *num_paths = (int)out.size();
  int o = 0;
  for (size_t i = 0; i < out.size(); ++i) {
    const OutPath& p = out[i];
    path_slack[i] = p.slack;
    path_endpoint[3 * i] = p.pin;
    path_endpoint[3 * i + 1] = p.el;
    path_endpoint[3 * i + 2] = p.rf;
    path_start[i] = o;
    for (size_t k = 0; k < p.pins.size(); ++k, ++o)
      if (o < max_points) {
        point_pin[o] = p.pins[k];
        point_tran[o] = p.trans[k];
        point_at[o] = p.ats[k];
      }
  }
  path_start[out.size()] = o;
  return need > max_points ? OTG_ERR_WORKSPACE : OTG_OK;
}
