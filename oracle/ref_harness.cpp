// ref_harness.cpp -- C entry points around the OpenTimer reference code,
// compiled together with the reference's own sources (see oracle/Makefile)
// into oracle/_ref/libotref.so.  TEST INFRASTRUCTURE ONLY: loaded by tests/,
// the fixture scripts and bench.py's reference/CPU-baseline legs, never by
// the product library.
//
// What runs here is the reference's code:
//   * ot::Rct::insert_node / insert_segment / update_rc_timing
//     (ot/timer/net.cpp:72-193) -- the CPU Elmore path, driven by the
//     reference's vendored Cpp-Taskflow parallel_for with chunk 32, as
//     Timer::_build_rc_timing_tasks does (ot/timer/timer.cpp:972-976);
//   * rct_bfs_and_compute_cuda (ot/cuda/rct.cu:361-397), built for sm_100a
//     (the levelization kernel is driven from ref_toposort.cu);
//   * spef::Spef::read / expand_name (ot/parser-spef/parser-spef.hpp:1177-1290).
//
// The private members of Rct/RctNode are reached with `#define private
// public`; the harness only reads results and sets per-corner node caps.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#define private public
#define protected public
#include <ot/timer/net.hpp>
#include <ot/timer/pin.hpp>
#undef private
#undef protected
#include <ot/cuda/rct.cuh>

// The Rct code path references two Pin members; RC nodes built here never
// carry a pin (their pin capacitance is folded into the per-corner node cap,
// which is what RctNode::cap sums, net.cpp:25-27), so these are unreachable.
namespace ot {
bool Pin::is_rct_root() const { return false; }
float Pin::cap(Split, Tran) const { return 0.0f; }
}  // namespace ot

namespace {

constexpr int NC = 4;

struct NetNames {
  std::vector<std::string> names;
};

// One net through the reference CPU path: build the Rct the way
// Net::_make_rct does (ground caps, then one insert_segment per RES line in
// order, net.cpp:318-343), bind the root, run update_rc_timing and read the
// per-node results back in local-id order.
void run_one_net(int net, const int* nodes_start, const int* edges, const int* roots,
                 const float* res, const float* cap, const std::vector<std::string>& names,
                 float* load, float* delay, float* ldelay, float* impulse) {
  const int b = nodes_start[net], n = nodes_start[net + 1] - b, eb = b - net;
  ot::Rct rct;
  for (int v = 0; v < n; ++v) {
    rct.insert_node(names[v], cap[(size_t)(b + v) * NC]);
  }
  for (int e = 0; e < n - 1; ++e) {
    rct.insert_segment(names[edges[2 * (eb + e)]], names[edges[2 * (eb + e) + 1]], res[eb + e]);
  }
  for (int v = 0; v < n; ++v) {
    ot::RctNode* node = rct._node(names[v]);
    for (int c = 0; c < NC; ++c) {
      node->_ncap[c >> 1][c & 1] = cap[(size_t)(b + v) * NC + c];
    }
  }
  rct._root = rct._node(names[roots[net]]);
  rct.update_rc_timing();
  if (!load) return;
  for (int v = 0; v < n; ++v) {
    const ot::RctNode* node = rct.node(names[v]);
    for (int c = 0; c < NC; ++c) {
      const size_t k = (size_t)(b + v) * NC + c;
      load[k] = node->_load[c >> 1][c & 1];
      delay[k] = node->_delay[c >> 1][c & 1];
      ldelay[k] = node->_ldelay[c >> 1][c & 1];
      impulse[k] = node->_impulse[c >> 1][c & 1];
    }
  }
}

}  // namespace

extern "C" {

// Node names are precomputed (outside any timed region) like the strings of
// a parsed SPEF; `max_nodes` bounds the largest net.
static std::vector<std::string> make_names(int max_nodes) {
  std::vector<std::string> names((size_t)max_nodes);
  for (int v = 0; v < max_nodes; ++v) names[v] = "n:" + std::to_string(v);
  return names;
}

// Reference CPU Elmore over a flat forest (local ids, undirected edges in
// RES order, per-corner caps [V][4]).  Outputs [V][4] by local id; pass
// load == nullptr to skip the read-back.  num_threads <= 0 uses the
// reference executor's default (hardware_concurrency).  Returns 0, or -1 if
// the reference threw (e.g. a missing root).
int otref_rct_update(int num_nets, const int* nodes_start, const int* edges, const int* roots,
                     const float* res, const float* cap, float* load, float* delay,
                     float* ldelay, float* impulse, int num_threads) {
  int mx = 1;
  for (int i = 0; i < num_nets; ++i) mx = std::max(mx, nodes_start[i + 1] - nodes_start[i]);
  const std::vector<std::string> names = make_names(mx);
  std::vector<int> ids((size_t)num_nets);
  for (int i = 0; i < num_nets; ++i) ids[i] = i;
  std::atomic<int> failed{0};
  tf::Taskflow taskflow;
  taskflow.parallel_for(
      ids.begin(), ids.end(),
      [&](int net) {
        try {
          run_one_net(net, nodes_start, edges, roots, res, cap, names, load, delay, ldelay,
                      impulse);
        } catch (...) {
          failed = 1;
        }
      },
      32);
  if (num_threads > 0) {
    tf::Executor executor((unsigned)num_threads);
    executor.run(taskflow).wait();
  } else {
    tf::Executor executor;
    executor.run(taskflow).wait();
  }
  return failed ? -1 : 0;
}

// The reference GPU path: rct_bfs_and_compute_cuda on host arrays exactly as
// FlatRctStorage::_update_timing_cuda hands them over (net.cpp:239-276).
// edges is rewritten to (parent, child); outputs are in BFS order.
void otref_rct_bfs_and_compute_cuda(int num_nets, int total_nodes, int* nodes_start, int* edges,
                                    int* roots, float* res, float* cap, int* node2bfs, int* pid,
                                    float* load, float* delay, float* ldelay, float* impulse) {
  RctEdgeArrayCUDA a;
  a.num_nets = num_nets;
  a.total_num_nodes = total_nodes;
  a.total_num_edges = total_nodes - num_nets;
  a.rct_nodes_start = nodes_start;
  a.rct_edges = reinterpret_cast<RctEdgeCUDA*>(edges);
  a.rct_roots = roots;
  a.rct_edges_res = res;
  a.rct_nodes_cap = cap;
  a.rct_node2bfs_order = node2bfs;
  a.rct_pid = pid;
  a.load = load;
  a.delay = delay;
  a.ldelay = ldelay;
  a.impulse = impulse;
  rct_bfs_and_compute_cuda(a);
}

// ---------------------------------------------------------------------------
// SPEF -> flat forest, with the reference parser.  Local ids follow
// Net::_make_flat_rct: first appearance while scanning *RES lines (node1
// then node2, net.cpp:392-410); cap = the ground cap of each *CAP line
// (net.cpp:425-431); root = the net's driver, i.e. the *CONN entry that is an
// input port (*P ... I) or an output cell pin (*I ... O) -- Pin::is_rct_root
// (pin.cpp:156-168).  Nets without RES lines are skipped, as
// Net::_init_flat_rct skips nets without a SPEF tree (net.cpp:347-367).
// Two calls: the first (bufs null) reports sizes, the second fills.
struct SpefFlat {
  std::vector<int> nodes_start, edges, roots;
  std::vector<float> res, cap;
  std::vector<std::string> net_names;
};
static SpefFlat g_spef;

int otref_spef_load(const char* path, int* num_nets, int* total_nodes) {
  spef::Spef spef;
  if (!spef.read(path) || spef.error) return -1;
  spef.expand_name();
  g_spef = SpefFlat{};
  g_spef.nodes_start.push_back(0);
  for (auto& net : spef.nets) {
    if (net.ress.empty()) continue;
    std::unordered_map<std::string, int> id;
    auto get = [&](const std::string& s) {
      auto it = id.find(s);
      if (it != id.end()) return it->second;
      int k = (int)id.size();
      id.emplace(s, k);
      return k;
    };
    for (auto& [n1, n2, r] : net.ress) {
      g_spef.edges.push_back(get(n1));
      g_spef.edges.push_back(get(n2));
      g_spef.res.push_back(r);
    }
    int n = (int)net.ress.size() + 1;
    if ((int)id.size() != n) return -2;  // not a tree: ids != |RES| + 1
    int root = -1;
    for (auto& c : net.connections) {
      bool drv = (c.type == spef::ConnectionType::EXTERNAL &&
                  c.direction == spef::ConnectionDirection::INPUT) ||
                 (c.type == spef::ConnectionType::INTERNAL &&
                  c.direction == spef::ConnectionDirection::OUTPUT);
      if (drv) {
        auto it = id.find(c.name);
        if (it != id.end()) { root = it->second; break; }
      }
    }
    if (root < 0) return -3;
    size_t base = g_spef.cap.size();
    g_spef.cap.resize(base + (size_t)n * NC, 0.0f);
    for (auto& [n1, n2, cv] : net.caps) {
      auto it = id.find(n1);
      if (it == id.end()) return -4;
      for (int c = 0; c < NC; ++c) g_spef.cap[base + (size_t)it->second * NC + c] = cv;
    }
    g_spef.roots.push_back(root);
    g_spef.net_names.push_back(net.name);
    g_spef.nodes_start.push_back(g_spef.nodes_start.back() + n);
  }
  *num_nets = (int)g_spef.roots.size();
  *total_nodes = g_spef.nodes_start.back();
  return 0;
}

void otref_spef_fetch(int* nodes_start, int* edges, int* roots, float* res, float* cap) {
  std::memcpy(nodes_start, g_spef.nodes_start.data(), g_spef.nodes_start.size() * sizeof(int));
  std::memcpy(edges, g_spef.edges.data(), g_spef.edges.size() * sizeof(int));
  std::memcpy(roots, g_spef.roots.data(), g_spef.roots.size() * sizeof(int));
  std::memcpy(res, g_spef.res.data(), g_spef.res.size() * sizeof(float));
  std::memcpy(cap, g_spef.cap.data(), g_spef.cap.size() * sizeof(float));
}

}  // extern "C"
