// otg_spef_write.cpp -- RC nets out as SPEF text, in parallel on the host.
//
// The subset of IEEE 1481 SPEF that the reference's parser
// (ot/parser-spef/parser-spef.hpp) and otg_spef_read take: a header with
// units (ns, fF, ohm), then per net
//   *D_NET <net> <total cap>
//   *CONN    the driver (*P <port> I, or *I <inst:pin> O) and the sinks
//            (*P <port> O, or *I <inst:pin> I)
//   *CAP     "<k> <node> <cap>" per node, in the given node order
//   *RES     "<k> <node a> <node b> <res>" per edge, in the given order
//   *END
// A net's nodes are its pins (by name) and internal nodes "<net>:<k>".
// Nets are formatted by several threads into their own buffers, which are
// then written in net order, so the file does not depend on the thread
// count.  Values are printed with four decimals.
#include <algorithm>
#include <charconv>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <string_view>
#include <thread>
#include <vector>

#include "../../include/otg.h"

namespace {

struct Out {
  std::string s;
  void put(std::string_view v) { s.append(v.data(), v.size()); }
  void put(char c) { s.push_back(c); }
  void num(long long v) {
    char b[24];
    auto r = std::to_chars(b, b + sizeof(b), v);
    s.append(b, r.ptr);
  }
  void fix4(double v) {
    char b[64];
    auto r = std::to_chars(b, b + sizeof(b), v, std::chars_format::fixed, 4);
    s.append(b, r.ptr);
  }
};

struct Args {
  const char* blob;
  const int64_t* name_off;
  const int32_t* net_name;
  const int32_t* pins_start;
  const int32_t* pin_name;
  const int8_t* pin_port;
  const int32_t* nodes_start;
  const int32_t* node_code;
  const float* node_cap;
  const int32_t* edges;
  const float* res;
};

std::string_view name_of(const Args& a, int id) {
  const int64_t b = a.name_off[id], e = a.name_off[id + 1];
  return std::string_view(a.blob + b, (size_t)(e - b - 1));  // without the '\0'
}

void node_name(const Args& a, Out& o, int net, int local) {
  const int c = a.node_code[a.nodes_start[net] + local];
  if (c >= 0) {
    o.put(name_of(a, a.pin_name[a.pins_start[net] + c]));
  } else {
    o.put(name_of(a, a.net_name[net]));
    o.put(':');
    o.num(-(long long)c);
  }
}

void format_net(const Args& a, int i, Out& o) {
  const int b = a.nodes_start[i], n = a.nodes_start[i + 1] - b, eb = b - i;
  double total = 0.0;
  for (int k = 0; k < n; ++k) total += (double)a.node_cap[b + k];
  o.put("*D_NET ");
  o.put(name_of(a, a.net_name[i]));
  o.put(' ');
  o.fix4(total);
  o.put("\n*CONN\n");
  const int p0 = a.pins_start[i], p1 = a.pins_start[i + 1];
  for (int p = p0; p < p1; ++p) {
    const bool port = a.pin_port[p] != 0, driver = p == p0;
    o.put(port ? "*P " : "*I ");
    o.put(name_of(a, a.pin_name[p]));
    // a driving port is an input of the design, a driving cell pin an output
    o.put(driver == port ? " I\n" : " O\n");
  }
  o.put("*CAP\n");
  for (int k = 0; k < n; ++k) {
    o.num(k + 1);
    o.put(' ');
    node_name(a, o, i, k);
    o.put(' ');
    o.fix4((double)a.node_cap[b + k]);
    o.put('\n');
  }
  o.put("*RES\n");
  for (int k = 0; k < n - 1; ++k) {
    o.num(k + 1);
    o.put(' ');
    node_name(a, o, i, a.edges[2 * (eb + k)]);
    o.put(' ');
    node_name(a, o, i, a.edges[2 * (eb + k) + 1]);
    o.put(' ');
    o.fix4((double)a.res[eb + k]);
    o.put('\n');
  }
  o.put("*END\n\n");
}

}  // namespace

extern "C" otg_status otg_spef_write(const char* path, int32_t num_nets, const char* names_blob,
                                     const int64_t* name_off, const int32_t* net_name,
                                     const int32_t* pins_start, const int32_t* pin_name,
                                     const int8_t* pin_port, const int32_t* nodes_start,
                                     const int32_t* node_code, const float* node_cap,
                                     const int32_t* edges, const float* res, int32_t threads) {
  if (!path || num_nets < 0) return OTG_ERR_INVALID;
  if (num_nets > 0 && (!names_blob || !name_off || !net_name || !pins_start || !pin_name ||
                       !pin_port || !nodes_start || !node_code || !node_cap || !res))
    return OTG_ERR_INVALID;
  for (int i = 0; i < num_nets; ++i) {
    const int n = nodes_start[i + 1] - nodes_start[i], np_ = pins_start[i + 1] - pins_start[i];
    if (n < 1 || np_ < 1 || (n > 1 && !edges)) return OTG_ERR_INVALID;
  }
  const Args a{names_blob, name_off, net_name,  pins_start, pin_name, pin_port,
               nodes_start, node_code, node_cap, edges,      res};
  std::FILE* f = std::fopen(path, "wb");
  if (!f) return OTG_ERR_INVALID;
  const char* header =
      "*SPEF \"IEEE 1481-1998\"\n*DESIGN \"top\"\n*DATE \"0\"\n*VENDOR \"otg\"\n"
      "*PROGRAM \"opentimer_b200\"\n*VERSION \"0\"\n*DESIGN_FLOW \"NETLIST_TYPE_VERILOG\"\n"
      "*DIVIDER /\n*DELIMITER :\n*BUS_DELIMITER [ ]\n*T_UNIT 1 NS\n*C_UNIT 1 FF\n"
      "*R_UNIT 1 OHM\n*L_UNIT 1 HENRY\n\n";
  bool ok = std::fputs(header, f) >= 0;
  int T = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
  T = std::min(T, 64);
  // chunks of nets, formatted T at a time, written in order
  const int chunk = 2048;
  for (int c0 = 0; c0 < num_nets && ok; c0 += chunk * T) {
    std::vector<Out> bufs((size_t)T);
    std::vector<std::thread> pool;
    for (int t = 0; t < T; ++t) {
      const int n0 = c0 + t * chunk, n1 = std::min(num_nets, n0 + chunk);
      if (n0 >= n1) break;
      pool.emplace_back([&, t, n0, n1]() {
        for (int i = n0; i < n1; ++i) format_net(a, i, bufs[(size_t)t]);
      });
    }
    for (auto& th : pool) th.join();
    for (auto& b : bufs)
      if (!b.s.empty() && std::fwrite(b.s.data(), 1, b.s.size(), f) != b.s.size()) ok = false;
  }
  if (std::fclose(f) != 0) ok = false;
  return ok ? OTG_OK : OTG_ERR_INVALID;
}
