// ot_run.cpp -- runs the reference OpenTimer Timer on a design directory and
// dumps its results.  TEST INFRASTRUCTURE ONLY (the full-update parity check).
//
//   ot_run <dir> cpu|cuda <out.txt> [graph.txt] [change=<spef>]...
//          [repower=<ops> [dump_every=<k>]] [paths=<K>]
//
// graph.txt (optional) is the Timer's timing graph, for the GPU propagation
// check: pins, arcs (net arcs with their net, cell arcs with one timing
// record per split; each with the delays of the last update), the
// data-path sources, timing records (sense, edge, constraint flag, six
// LUT ids), LUTs (variable order, indices, values), timing tests, the clock
// period and the primary-input/-output assertions, all by pin index.
// <dir> holds early.lib, late.lib, design.v, design.spef, design.timing.
// repower=<ops>: after the first update, a sequence of gate resizes, one
// "<gate> <cell>" per line, steps separated by lines holding "=": each step
// is Timer::repower_gate for its lines, then update_timing (the dirty nets
// and the affected cone only, as the Timer does).  The Timer clears all of
// its state bits, CUDA_ENABLED among them, at the end of every update
// (_remove_state() in Timer::_update_timing, ot/timer/timer.cpp), so in
// "cuda" mode each step calls cuda(true) again before its update_timing;
// otherwise every step after the first would run the CPU path.  The
// seconds of every step go to stdout ("repower_step_s <k> <s>"); with
// dump_every=<k> the pins (P lines) after every k-th step go to
// <out>.step<k>.
// paths=<K>[,<split>[,<tran>]]: after the updates, Timer::report_timing(K)
// (or its split / split-and-transition forms; split -1 with a transition
// is the transition-only form), the K worst paths, to the output (T and Q
// lines).
// The same Timer sources are linked twice (oracle/Makefile): with the
// reference's own CUDA module (ot_run_ref) and with libotg in its place
// (ot_run_otg), so "cuda" runs either the reference kernels or ours behind
// the unchanged Timer.  Output lines (all values %.9g, corners in the order
// MIN-RISE, MIN-FALL, MAX-RISE, MAX-FALL; nan where the Timer has none):
//   P <pin> at[4] slew[4] rat[4] slack[4]
//   R <net> <node> load[4] delay[4] ldelay[4] impulse[4]   (per RC node)
//   B <net> <node> <bfs slot> <pid of that slot>            (cuda only)
//   K <pin> cap[4]                                          (pin caps)
//   L <net> report_load[4]
//   N <split> <tran> report_wns report_tns                   (per corner)
//   T <k> <slack> <split> <points>                           (paths=K: path k,
//   Q <k> <pin> <tran> <at>                                   then its points)
//   S <net> <num nodes> <root id>                           (cuda only:
//   E <net> <edge k> <s> <t> <res>                           the flat
//   C <net> <id> cap[4]                                      storage)
// The per-node values are read from Rct::_nodes (cpu) or from the
// FlatRctStorage arrays in BFS order (cuda), the node's local id being
// rebuilt with the flat path's first-appearance rule over the SPEF RES
// lines (ot/timer/net.cpp:388-410).
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <string>
#include <unordered_map>
#include <vector>

#define private public
#define protected public
#include <ot/timer/timer.hpp>
#undef private
#undef protected

// FlatRct keeps its offsets in the implicit private section of a class
// (ot/timer/net.hpp:172-178), which the access macro cannot open; this view
// has the same members in the same order.
struct FlatRctView {
  ot::FlatRctStorage* stor;
  size_t num_nodes;
  int arr_start;
  int edge_start;
  int net_id;
};
static_assert(sizeof(FlatRctView) == sizeof(ot::FlatRct), "FlatRct layout changed");

static void put(FILE* f, std::optional<float> v) {
  if (v) std::fprintf(f, " %.9g", *v);
  else std::fprintf(f, " nan");
}

// ---- graph export
static void opt4(FILE* f, const ot::TimingData<std::optional<float>, ot::MAX_SPLIT, ot::MAX_TRAN>& d) {
  for (int el = 0; el < 2; ++el)
    for (int rf = 0; rf < 2; ++rf) {
      if (d[el][rf]) std::fprintf(f, " %.9g", *d[el][rf]);
      else std::fprintf(f, " nan");
    }
}

static void dump_graph(ot::Timer& timer, const char* path) {
  FILE* f = std::fopen(path, "w");
  if (!f) return;
  std::unordered_map<const ot::Timing*, int> tid;
  std::unordered_map<const ot::Lut*, int> lid;
  std::vector<const ot::Timing*> timings;
  std::vector<const ot::Lut*> luts;
  auto lut_id = [&](const std::optional<ot::Lut>& l) -> int {
    if (!l) return -1;
    auto it = lid.find(&*l);
    if (it != lid.end()) return it->second;
    lid[&*l] = (int)luts.size();
    luts.push_back(&*l);
    return (int)luts.size() - 1;
  };
  auto timing_id = [&](const ot::Timing* t) -> int {
    if (!t) return -1;
    auto it = tid.find(t);
    if (it != tid.end()) return it->second;
    tid[t] = (int)timings.size();
    timings.push_back(t);
    return (int)timings.size() - 1;
  };
  // pins by index
  std::vector<const ot::Pin*> pins(timer._pins.size(), nullptr);
  for (auto& [name, pin] : timer._pins)
    if (pin._idx < pins.size()) pins[pin._idx] = &pin;
  for (size_t i = 0; i < pins.size(); ++i) {
    const ot::Pin* p = pins[i];
    if (!p) continue;
    std::fprintf(f, "p %zu %s %s", i, p->name().c_str(), p->_net ? p->_net->name().c_str() : "-");
    ot::TimingData<std::optional<float>, ot::MAX_SPLIT, ot::MAX_TRAN> none{};
    opt4(f, p->primary_input() ? p->primary_input()->_at : none);
    opt4(f, p->primary_input() ? p->primary_input()->_slew : none);
    opt4(f, p->primary_output() ? p->primary_output()->_rat : none);
    std::fprintf(f, "\n");
  }
  // arcs
  std::unordered_map<const ot::Arc*, int> aid;
  int k = 0;
  for (auto& arc : timer._arcs) {
    aid[&arc] = k;
    std::fprintf(f, "a %d %zu %zu %d", k, arc._from._idx, arc._to._idx, arc._state);
    if (auto net = std::get_if<ot::Net*>(&arc._handle)) {
      std::fprintf(f, " net %s -1 -1\n", (*net)->name().c_str());
    } else {
      auto tv = std::get<ot::TimingView>(arc._handle);
      std::fprintf(f, " cell - %d %d\n", timing_id(tv[ot::MIN]), timing_id(tv[ot::MAX]));
    }
    // the delays the last update left on the arc, (split, from, to transition)
    std::fprintf(f, "d %d", k);
    for (int el = 0; el < 2; ++el)
      for (int fr = 0; fr < 2; ++fr)
        for (int tr = 0; tr < 2; ++tr) put(f, arc._delay[el][fr][tr]);
    std::fprintf(f, "\n");
    ++k;
  }
  for (size_t i = 0; i < pins.size(); ++i)  // data-path sources of the path search
    if (pins[i] && pins[i]->is_datapath_source()) std::fprintf(f, "z %zu\n", i);
  for (auto& [name, pin] : timer._pins)
    for (auto* test : pin._tests) std::fprintf(f, "s %d\n", aid[&test->_arc]);
  for (size_t i = 0; i < timings.size(); ++i) {
    const ot::Timing* t = timings[i];
    const int sense = !t->sense ? 2 : (*t->sense == ot::TimingSense::POSITIVE_UNATE ? 0
                                      : *t->sense == ot::TimingSense::NEGATIVE_UNATE ? 1 : 2);
    const int edge = t->is_rising_edge_triggered() ? 1 : (t->is_falling_edge_triggered() ? 2 : 0);
    const int l[6] = {lut_id(t->cell_rise), lut_id(t->cell_fall), lut_id(t->rise_transition),
                      lut_id(t->fall_transition), lut_id(t->rise_constraint),
                      lut_id(t->fall_constraint)};
    std::fprintf(f, "t %zu %d %d %d %d %d %d %d %d %d\n", i, sense, edge, t->is_constraint() ? 1 : 0,
                 l[0], l[1], l[2], l[3], l[4], l[5]);
  }
  for (size_t i = 0; i < luts.size(); ++i) {
    const ot::Lut* l = luts[i];
    // variable order: 0 = (slew | related, ...), 1 = (load | constrained, ...), -1 = no template
    int var = -1;
    if (l->lut_template && l->lut_template->variable1) {
      const auto v = *l->lut_template->variable1;
      var = (v == ot::LutVar::TOTAL_OUTPUT_NET_CAPACITANCE ||
             v == ot::LutVar::CONSTRAINED_PIN_TRANSITION) ? 1 : 0;
    }
    std::fprintf(f, "l %zu %d %zu %zu", i, var, l->indices1.size(), l->indices2.size());
    for (float x : l->indices1) std::fprintf(f, " %.9g", x);
    for (float x : l->indices2) std::fprintf(f, " %.9g", x);
    for (float x : l->table) std::fprintf(f, " %.9g", x);
    std::fprintf(f, "\n");
  }
  if (!timer._clocks.empty()) std::fprintf(f, "c %.9g\n", timer._clocks.begin()->second._period);
  std::fclose(f);
}

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s <dir> cpu|cuda <out> [graph] [change=<spef>]...\n",
                 argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  const bool cuda = std::string(argv[2]) == "cuda";
  // optional: a graph dump path, and change SPEFs applied after the first
  // update (read_spef + update_timing, as the TAU15 ops files do)
  const char* graph_path = nullptr;
  std::vector<std::string> changes;
  std::string repower;
  int dump_every = 0;
  int num_paths = 0, path_el = -1, path_rf = -1;
  for (int a = 4; a < argc; ++a) {
    const std::string s = argv[a];
    if (s.rfind("change=", 0) == 0) changes.push_back(s.substr(7));
    else if (s.rfind("repower=", 0) == 0) repower = s.substr(8);
    else if (s.rfind("dump_every=", 0) == 0) dump_every = std::atoi(s.c_str() + 11);
    else if (s.rfind("paths=", 0) == 0) {
      num_paths = std::atoi(s.c_str() + 6);
      const size_t c1 = s.find(',');
      if (c1 != std::string::npos) {
        path_el = std::atoi(s.c_str() + c1 + 1);
        const size_t c2 = s.find(',', c1 + 1);
        if (c2 != std::string::npos) path_rf = std::atoi(s.c_str() + c2 + 1);
      }
    }
    else graph_path = argv[a];
  }
  ot::Timer timer;
  timer.read_celllib(dir + "/early.lib", ot::MIN)
      .read_celllib(dir + "/late.lib", ot::MAX)
      .read_verilog(dir + "/design.v")
      .read_spef(dir + "/design.spef")
      .read_timing(dir + "/design.timing");
  timer.cuda(cuda);
  const auto t0 = std::chrono::steady_clock::now();
  timer.update_timing();
  const double secs =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::printf("update_timing_s %.6f\n", secs);
  if (!changes.empty()) {
    const auto t1 = std::chrono::steady_clock::now();
    for (const auto& c : changes) timer.read_spef(c);
    timer.update_timing();
    const double s2 =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
    std::printf("incremental_update_timing_s %.6f\n", s2);
  }

  const ot::Split splits[2] = {ot::MIN, ot::MAX};
  const ot::Tran trans[2] = {ot::RISE, ot::FALL};
  auto dump_pins = [&](FILE* f) {
    for (auto& [name, pin] : timer._pins) {
      (void)pin;
      std::fprintf(f, "P %s", name.c_str());
      for (auto el : splits)
        for (auto rf : trans) put(f, timer.report_at(name, el, rf));
      for (auto el : splits)
        for (auto rf : trans) put(f, timer.report_slew(name, el, rf));
      for (auto el : splits)
        for (auto rf : trans) put(f, timer.report_rat(name, el, rf));
      for (auto el : splits)
        for (auto rf : trans) put(f, timer.report_slack(name, el, rf));
      std::fprintf(f, "\n");
    }
  };
  if (!repower.empty()) {
    FILE* ops = std::fopen(repower.c_str(), "r");
    if (!ops) return 4;
    char gate[256], cell[256];
    int step = 0, pending = 0;
    double total = 0.0;
    auto finish_step = [&]() {
      if (cuda) timer.cuda(true);  // the previous update cleared the flag
      const auto t1 = std::chrono::steady_clock::now();
      timer.update_timing();
      const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
      total += s;
      ++step;
      std::printf("repower_step_s %d %.6f %d\n", step, s, pending);
      if (dump_every > 0 && step % dump_every == 0) {
        const std::string path = std::string(argv[3]) + ".step" + std::to_string(step);
        if (FILE* g = std::fopen(path.c_str(), "w")) {
          dump_pins(g);
          std::fclose(g);
        }
      }
      pending = 0;
    };
    char line[600];
    const auto t0r = std::chrono::steady_clock::now();
    double repower_calls = 0.0;
    while (std::fgets(line, sizeof(line), ops)) {
      if (line[0] == '=') {
        finish_step();
        continue;
      }
      if (std::sscanf(line, "%255s %255s", gate, cell) == 2) {
        const auto t1 = std::chrono::steady_clock::now();
        timer.repower_gate(gate, cell);
        repower_calls += std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
        ++pending;
      }
    }
    if (pending) finish_step();
    std::fclose(ops);
    const double wall =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0r).count();
    std::printf("repower_total_s %.6f %d %.6f %.6f\n", total + repower_calls, step, wall,
                repower_calls);
  }

  FILE* f = std::fopen(argv[3], "w");
  if (!f) return 3;
  for (auto& [name, pin] : timer._pins) {
    std::fprintf(f, "P %s", name.c_str());
    for (auto el : splits)
      for (auto rf : trans) put(f, timer.report_at(name, el, rf));
    for (auto el : splits)
      for (auto rf : trans) put(f, timer.report_slew(name, el, rf));
    for (auto el : splits)
      for (auto rf : trans) put(f, timer.report_rat(name, el, rf));
    for (auto el : splits)
      for (auto rf : trans) put(f, timer.report_slack(name, el, rf));
    std::fprintf(f, "\n");
    std::fprintf(f, "K %s", name.c_str());
    for (auto el : splits)
      for (auto rf : trans) std::fprintf(f, " %.9g", pin.cap(el, rf));
    std::fprintf(f, "\n");
  }
  for (auto& [nname, net] : timer._nets) {
    (void)net;
    std::fprintf(f, "L %s", nname.c_str());
    for (auto el : splits)
      for (auto rf : trans) put(f, timer.report_load(nname, el, rf));
    std::fprintf(f, "\n");
  }
  for (auto el : splits)
    for (auto rf : trans) {
      std::fprintf(f, "N %d %d", (int)el, (int)rf);
      put(f, timer.report_wns(el, rf));
      put(f, timer.report_tns(el, rf));
      std::fprintf(f, "\n");
    }
  for (auto& [nname, net] : timer._nets) {
    if (const ot::Rct* rct = std::get_if<ot::Rct>(&net._rct)) {
      for (auto& [node, rn] : rct->_nodes) {
        std::fprintf(f, "R %s %s", nname.c_str(), node.c_str());
        for (auto el : splits)
          for (auto rf : trans) std::fprintf(f, " %.9g", rn._load[el][rf]);
        for (auto el : splits)
          for (auto rf : trans) std::fprintf(f, " %.9g", rn._delay[el][rf]);
        for (auto el : splits)
          for (auto rf : trans) std::fprintf(f, " %.9g", rn._ldelay[el][rf]);
        for (auto el : splits)
          for (auto rf : trans) std::fprintf(f, " %.9g", rn._impulse[el][rf]);
        std::fprintf(f, "\n");
      }
    } else if (const ot::FlatRct* fr = std::get_if<ot::FlatRct>(&net._rct)) {
      if (!net._spef_net || !timer._flat_rct_stor) continue;
      const ot::FlatRctStorage& st = *timer._flat_rct_stor;
      std::unordered_map<std::string, int> id;
      std::vector<std::string> names;
      for (const auto& [a, b, r] : net._spef_net->ress) {
        (void)r;
        for (const std::string* s : {&a, &b})
          if (id.emplace(*s, (int)names.size()).second) names.push_back(*s);
      }
      const FlatRctView* view = reinterpret_cast<const FlatRctView*>(fr);
      const int base = view->arr_start;
      std::fprintf(f, "S %s %zu %d\n", nname.c_str(), view->num_nodes, st.rct_roots[view->net_id]);
      for (size_t k = 0; k + 1 < view->num_nodes; ++k) {
        const auto& e = st.rct_edges[view->edge_start + k];
        std::fprintf(f, "E %s %zu %d %d %.9g\n", nname.c_str(), k, e.s, e.t,
                     st.rct_edges_res[view->edge_start + k]);
      }
      for (size_t k = 0; k < view->num_nodes; ++k) {
        std::fprintf(f, "C %s %zu", nname.c_str(), k);
        for (int c = 0; c < 4; ++c) std::fprintf(f, " %.9g", st.rct_nodes_cap[(base + k) * 4 + c]);
        std::fprintf(f, "\n");
      }
      for (size_t k = 0; k < names.size(); ++k) {
        const int slot = st.rct_node2bfs_order[base + k];
        const size_t at = (size_t)(base + slot) * 4;
        std::fprintf(f, "R %s %s", nname.c_str(), names[k].c_str());
        for (const std::vector<float>* q : {&st.load, &st.delay, &st.ldelay, &st.impulse})
          for (int c = 0; c < 4; ++c) std::fprintf(f, " %.9g", (*q)[at + c]);
        std::fprintf(f, "\n");
        std::fprintf(f, "B %s %s %d %d\n", nname.c_str(), names[k].c_str(), slot,
                     slot == 0 ? 0 : st.rct_pid[base + slot]);
      }
    }
  }
  if (num_paths > 0) {
    const size_t K = (size_t)num_paths;
    const ot::Split el = path_el == 1 ? ot::MAX : ot::MIN;
    const ot::Tran rf = path_rf == 1 ? ot::FALL : ot::RISE;
    const std::vector<ot::Path> paths =
        path_el >= 0 && path_rf >= 0 ? timer.report_timing(K, el, rf)
        : path_el >= 0              ? timer.report_timing(K, el)
        : path_rf >= 0              ? timer.report_timing(K, rf)
                                    : timer.report_timing(K);
    for (size_t k = 0; k < paths.size(); ++k) {
      const ot::Path& p = paths[k];
      std::fprintf(f, "T %zu %.9g %d %zu\n", k, p.slack, (int)p.endpoint->_el, p.size());
      for (const ot::Point& pt : p)
        std::fprintf(f, "Q %zu %s %d %.9g\n", k, pt.pin.name().c_str(), (int)pt.transition,
                     pt.at);
    }
  }
  std::fclose(f);
  if (graph_path) dump_graph(timer, graph_path);
  return 0;
}
