// otg_spef.cpp -- SPEF to the flat RC layout, in parallel on the host.
//
// The reference reads SPEF with a PEGTL grammar into per-net string tuples
// (ot/parser-spef/parser-spef.hpp), expands *NAME_MAP references
// (parser-spef.hpp:1215-1290), rebases units with a float scale per value
// (Timer::_rebase_unit, ot/timer/unit.cpp:328-360), and then, per net,
// hashes every node name again to build the flat layout
// (Net::_make_flat_rct, ot/timer/net.cpp:370-461).  This reader goes from
// the file to that layout in one pass per net, nets in parallel:
//   * local ids in order of first appearance over the *RES lines (node1,
//     then node2 of each line); edges and res in *RES order;
//   * the root is the net's driver: the *CONN entry that is an instance
//     pin of direction O or a port of direction I;
//   * cap[id][c] = the value of each *CAP line of the node, in file order
//     (a coupling line assigns its value to its first node, as the flat
//     path does, net.cpp:425-431), the same in all four corners; the
//     caller adds pin caps (which need its cell library);
//   * values are parsed with float rounding (as std::strtof) and then
//     multiplied by r_scale / c_scale in float, as a Timer rebases units.
// Nets without *RES lines carry no RC tree and are left out.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cctype>
#include <charconv>
#include <cstdint>
#include <cstring>
#include <deque>
#include <string>
#include <string_view>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/otg.h"

namespace {

using sv = std::string_view;

struct Edge {
  int32_t s, t;
};

struct Pin {
  std::string name;
  int32_t node;  // local id, -1 when the pin is not in the RC tree
  int8_t dir;    // 0 I, 1 O, 2 B
  int8_t port;   // 1 for *P (a port), 0 for *I (an instance pin)
};

struct Net {
  std::string name;
  int32_t n = 0, root = -1;
  uint8_t flags = 0;
  std::vector<Edge> edges;
  std::vector<float> res, cap;
  std::vector<Pin> pins;
};

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// Splits one line into whitespace-separated tokens.
int tokens(sv line, sv* t, int max) {
  int k = 0;
  size_t i = 0;
  while (i < line.size() && k < max) {
    while (i < line.size() && is_space(line[i])) ++i;
    size_t j = i;
    while (j < line.size() && !is_space(line[j])) ++j;
    if (j > i) t[k++] = line.substr(i, j - i);
    i = j;
  }
  return k;
}

bool parse_float(sv s, float* out) {
  const char* b = s.data();
  const char* e = b + s.size();
  if (b < e && *b == '+') ++b;
  auto r = std::from_chars(b, e, *out, std::chars_format::general);
  return r.ec == std::errc();
}

// *NAME_MAP expansion: every "*<digits>" in a name, scanned from the end,
// is replaced by its mapped name when the map has that key.
std::string expand(sv s, const std::unordered_map<uint64_t, std::string>& map) {
  std::string str(s);
  if (map.empty()) return str;
  size_t beg = str.size();
  while (beg > 0) {
    const size_t last = beg;
    --beg;
    beg = str.find_last_of('*', beg);
    if (beg == std::string::npos) break;
    size_t end = beg + 1;
    while (end < last && std::isdigit((unsigned char)str[end])) ++end;
    uint64_t key = 0;
    for (size_t i = beg + 1; i < end; ++i) key = key * 10 + (uint64_t)(str[i] - '0');
    auto it = map.find(key);
    if (end > beg + 1 && it != map.end()) str.replace(beg, end - beg, it->second);
  }
  return str;
}

// Open-addressing name -> local id table, reused net after net.
struct IdTable {
  std::vector<uint64_t> hash;
  std::vector<int32_t> id;
  std::vector<sv> key;
  size_t mask = 0;
  void reset(size_t n) {
    size_t cap = 16;
    while (cap < 2 * n + 2) cap <<= 1;
    if (hash.size() < cap) {
      hash.assign(cap, 0);
      id.assign(cap, -1);
      key.assign(cap, sv());
    } else {
      std::fill(id.begin(), id.begin() + cap, -1);
    }
    mask = cap - 1;
  }
  static uint64_t h(sv s) {
    uint64_t x = 1469598103934665603ull;
    for (unsigned char c : s) x = (x ^ c) * 1099511628211ull;
    return x | 1;
  }
  // returns the id of s, inserting `fresh` when absent
  int32_t get(sv s, int32_t fresh, bool* inserted) {
    const uint64_t hv = h(s);
    for (size_t i = hv & mask;; i = (i + 1) & mask) {
      if (id[i] < 0) {
        hash[i] = hv;
        id[i] = fresh;
        key[i] = s;
        *inserted = true;
        return fresh;
      }
      if (hash[i] == hv && key[i] == s) {
        *inserted = false;
        return id[i];
      }
    }
  }
  int32_t find(sv s) const {
    const uint64_t hv = h(s);
    for (size_t i = hv & mask;; i = (i + 1) & mask) {
      if (id[i] < 0) return -1;
      if (hash[i] == hv && key[i] == s) return id[i];
    }
  }
};

constexpr uint8_t kNoDriver = 1, kNotTree = 2, kCapNode = 4, kSyntax = 8;

// Parses one *D_NET block (from "*D_NET" up to the next one).
bool parse_net(sv block, const std::unordered_map<uint64_t, std::string>& map, float r_scale,
               float c_scale, IdTable& tab, Net* net) {
  enum { NONE, CONN, CAP, RES, OTHER } sec = NONE;
  // Node names are views into the file; with a name map, into expanded
  // copies kept in `store` (a deque: its elements never move).
  std::deque<std::string> store;
  auto name = [&](sv s) -> sv {
    if (map.empty()) return s;
    store.push_back(expand(s, map));
    return store.back();
  };
  std::vector<std::pair<sv, float>> caps;
  std::vector<std::pair<sv, sv>> ress;
  std::vector<float> resv;
  sv t[8];
  size_t p = 0;
  bool first = true;
  while (p < block.size()) {
    size_t q = block.find('\n', p);
    if (q == sv::npos) q = block.size();
    const sv line = block.substr(p, q - p);
    p = q + 1;
    const int k = tokens(line, t, 8);
    if (k == 0) continue;
    if (first) {
      if (k < 2 || t[0] != "*D_NET") return false;
      net->name = expand(t[1], map);
      first = false;
      continue;
    }
    if (t[0][0] == '*') {
      if (t[0] == "*CONN") { sec = CONN; continue; }
      if (t[0] == "*CAP") { sec = CAP; continue; }
      if (t[0] == "*RES") { sec = RES; continue; }
      if (t[0] == "*END") break;
      if (sec == CONN && (t[0] == "*P" || t[0] == "*I") && k >= 3) {
        Pin pin;
        pin.name = expand(t[1], map);
        pin.port = t[0] == "*P";
        pin.dir = t[2] == "O" ? 1 : (t[2] == "B" ? 2 : 0);
        pin.node = -1;
        net->pins.push_back(std::move(pin));
        continue;
      }
      if (sec == CONN) continue;  // *N coordinates and other attributes
      sec = OTHER;                // *INDUC and sections this layout ignores
      continue;
    }
    float v = 0.f;
    if (sec == CAP) {
      if (k == 3 && parse_float(t[2], &v)) caps.emplace_back(name(t[1]), v);
      else if (k >= 4 && parse_float(t[3], &v)) caps.emplace_back(name(t[1]), v);
      else net->flags |= kSyntax;
    } else if (sec == RES) {
      if (k >= 4 && parse_float(t[3], &v)) {
        ress.emplace_back(name(t[1]), name(t[2]));
        resv.push_back(v);
      } else {
        net->flags |= kSyntax;
      }
    }
  }
  if (ress.empty()) return true;  // no RC tree
  // ids by first appearance over the RES lines
  tab.reset(2 * ress.size() + 2);
  int32_t count = 0;
  net->edges.resize(ress.size());
  net->res.resize(ress.size());
  for (size_t e = 0; e < ress.size(); ++e) {
    int32_t ids[2];
    const sv nm[2] = {ress[e].first, ress[e].second};
    for (int j = 0; j < 2; ++j) {
      bool ins = false;
      ids[j] = tab.get(nm[j], count, &ins);
      if (ins) ++count;
    }
    net->edges[e] = Edge{ids[0], ids[1]};
    net->res[e] = resv[e] * r_scale;
  }
  net->n = count;
  if ((size_t)net->n != ress.size() + 1) net->flags |= kNotTree;
  for (auto& pin : net->pins) {
    pin.node = tab.find(pin.name);
    if (net->root < 0 && pin.node >= 0 && (pin.port ? pin.dir == 0 : pin.dir == 1))
      net->root = pin.node;
  }
  if (net->root < 0) net->flags |= kNoDriver;
  net->cap.assign((size_t)net->n, 0.0f);
  for (auto& [nm, v] : caps) {
    const int32_t i = tab.find(nm);
    if (i < 0) net->flags |= kCapNode;
    else net->cap[i] = v * c_scale;
  }
  return true;
}

}  // namespace

struct otg_spef {
  std::vector<Net> nets;  // with RC trees, in file order
  double units[3] = {1.0, 1.0, 1.0};  // ohm, farad, second per file unit
  int64_t total_nodes = 0, total_pins = 0;
};

namespace {

double unit_scale(sv num, sv unit, char kind) {
  float v = 1.f;
  parse_float(num, &v);
  std::string u(unit);
  for (auto& c : u) c = (char)std::toupper((unsigned char)c);
  double m = 1.0;
  if (u.size() >= 2) {
    switch (u[0]) {
      case 'K': m = 1e3; break;
      case 'M': m = (kind == 'R') ? 1e6 : 1e-3; break;
      case 'U': m = 1e-6; break;
      case 'N': m = 1e-9; break;
      case 'P': m = 1e-12; break;
      case 'F': m = 1e-15; break;
      default: m = 1.0;
    }
  }
  return v * m;
}

}  // namespace

extern "C" {

otg_status otg_spef_read(const char* path, int32_t threads, float r_scale, float c_scale,
                         otg_spef** out) {
  if (!path || !out) return OTG_ERR_INVALID;
  const int fd = open(path, O_RDONLY);
  if (fd < 0) return OTG_ERR_INVALID;
  struct stat st;
  if (fstat(fd, &st) != 0 || st.st_size <= 0) {
    close(fd);
    return OTG_ERR_INVALID;
  }
  const size_t size = (size_t)st.st_size;
  void* mem = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
  close(fd);
  if (mem == MAP_FAILED) return OTG_ERR_OOM;
  const sv text((const char*)mem, size);
  auto* S = new (std::nothrow) otg_spef();
  if (!S) {
    munmap(mem, size);
    return OTG_ERR_OOM;
  }
  const int T = threads > 0 ? threads : std::max(1u, std::thread::hardware_concurrency());
  // header: units and the name map, up to the first *D_NET
  size_t first = text.find("*D_NET");
  if (first == sv::npos) first = size;
  std::unordered_map<uint64_t, std::string> map;
  {
    const sv head = text.substr(0, first);
    bool in_map = false;
    sv t[8];
    size_t p = 0;
    while (p < head.size()) {
      size_t q = head.find('\n', p);
      if (q == sv::npos) q = head.size();
      const int k = tokens(head.substr(p, q - p), t, 8);
      p = q + 1;
      if (k == 0) continue;
      if (t[0] == "*R_UNIT" && k >= 3) S->units[0] = unit_scale(t[1], t[2], 'R');
      else if (t[0] == "*C_UNIT" && k >= 3) S->units[1] = unit_scale(t[1], t[2], 'C');
      else if (t[0] == "*T_UNIT" && k >= 3) S->units[2] = unit_scale(t[1], t[2], 'T');
      else if (t[0] == "*NAME_MAP") in_map = true;
      else if (t[0] == "*PORTS") in_map = false;
      else if (in_map && k >= 2 && t[0].size() > 1 && t[0][0] == '*') {
        uint64_t key = 0;
        bool ok = true;
        for (size_t i = 1; i < t[0].size(); ++i) {
          if (!std::isdigit((unsigned char)t[0][i])) { ok = false; break; }
          key = key * 10 + (uint64_t)(t[0][i] - '0');
        }
        if (ok) map[key] = std::string(t[1]);
      }
    }
  }
  // block starts: "*D_NET" at a line start, found by T threads in slices
  std::vector<std::vector<size_t>> found(T);
  {
    std::vector<std::thread> pool;
    const size_t span = (size - first + T - 1) / T;
    for (int w = 0; w < T; ++w)
      pool.emplace_back([&, w] {
        const size_t a = first + (size_t)w * span, b = std::min(size, a + span);
        for (size_t i = a; i < b;) {
          const size_t hit = text.find("*D_NET", i);
          if (hit == sv::npos || hit >= b) break;
          if (hit == 0 || text[hit - 1] == '\n') found[w].push_back(hit);
          i = hit + 6;
        }
      });
    for (auto& th : pool) th.join();
  }
  std::vector<size_t> starts;
  for (auto& f : found) starts.insert(starts.end(), f.begin(), f.end());
  const size_t nb = starts.size();
  std::vector<Net> nets(nb);
  std::vector<char> keep(nb, 0);
  std::atomic<size_t> next{0};
  std::atomic<int> bad{0};
  {
    std::vector<std::thread> pool;
    for (int w = 0; w < T; ++w)
      pool.emplace_back([&] {
        IdTable tab;
        for (;;) {
          const size_t b = next.fetch_add(16);
          if (b >= nb) break;
          for (size_t i = b; i < std::min(nb, b + 16); ++i) {
            const size_t end = i + 1 < nb ? starts[i + 1] : size;
            if (!parse_net(text.substr(starts[i], end - starts[i]), map, r_scale, c_scale, tab,
                           &nets[i]))
              bad.fetch_add(1);
            keep[i] = nets[i].n > 0;
          }
        }
      });
    for (auto& th : pool) th.join();
  }
  munmap(mem, size);
  if (bad.load()) {
    delete S;
    return OTG_ERR_INVALID;
  }
  for (size_t i = 0; i < nb; ++i)
    if (keep[i]) {
      S->total_nodes += nets[i].n;
      S->total_pins += (int64_t)nets[i].pins.size();
      S->nets.push_back(std::move(nets[i]));
    }
  if (S->total_nodes >= ((int64_t)1 << 31)) {
    delete S;
    return OTG_ERR_TOO_LARGE;
  }
  *out = S;
  return OTG_OK;
}

otg_status otg_spef_sizes(const otg_spef* s, int32_t* num_nets, int32_t* total_nodes,
                          int32_t* total_pins, double* units) {
  if (!s) return OTG_ERR_INVALID;
  if (num_nets) *num_nets = (int32_t)s->nets.size();
  if (total_nodes) *total_nodes = (int32_t)s->total_nodes;
  if (total_pins) *total_pins = (int32_t)s->total_pins;
  if (units)
    for (int i = 0; i < 3; ++i) units[i] = s->units[i];
  return OTG_OK;
}

otg_status otg_spef_fill(const otg_spef* s, int32_t* nodes_start, otg_rc_edge* edges,
                         int32_t* roots, float* res, float* cap, uint8_t* net_flags) {
  if (!s || !nodes_start || !edges || !roots || !res || !cap) return OTG_ERR_INVALID;
  const size_t N = s->nets.size();
  nodes_start[0] = 0;
  for (size_t i = 0; i < N; ++i) nodes_start[i + 1] = nodes_start[i] + s->nets[i].n;
  const int T = (int)std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), 64);
  std::vector<std::thread> pool;
  for (int w = 0; w < T; ++w)
    pool.emplace_back([&, w] {
      for (size_t i = (size_t)w; i < N; i += (size_t)T) {
        const Net& n = s->nets[i];
        const int32_t b = nodes_start[i], eb = b - (int32_t)i;
        for (size_t e = 0; e < n.edges.size(); ++e) {
          edges[eb + e].s = n.edges[e].s;
          edges[eb + e].t = n.edges[e].t;
          res[eb + e] = n.res[e];
        }
        roots[i] = n.root;
        for (int32_t v = 0; v < n.n; ++v)
          for (int c = 0; c < 4; ++c) cap[4 * (size_t)(b + v) + c] = n.cap[v];
        if (net_flags) net_flags[i] = n.flags;
      }
    });
  for (auto& th : pool) th.join();
  return OTG_OK;
}

otg_status otg_spef_pins(const otg_spef* s, int32_t* pins_start, int32_t* pin_node,
                         int8_t* pin_dir, int8_t* pin_port) {
  if (!s || !pins_start) return OTG_ERR_INVALID;
  pins_start[0] = 0;
  for (size_t i = 0; i < s->nets.size(); ++i) {
    const Net& n = s->nets[i];
    int32_t at = pins_start[i];
    for (const Pin& p : n.pins) {
      if (pin_node) pin_node[at] = p.node;
      if (pin_dir) pin_dir[at] = p.dir;
      if (pin_port) pin_port[at] = p.port;
      ++at;
    }
    pins_start[i + 1] = at;
  }
  return OTG_OK;
}

const char* otg_spef_net_name(const otg_spef* s, int32_t net) {
  if (!s || net < 0 || (size_t)net >= s->nets.size()) return nullptr;
  return s->nets[net].name.c_str();
}

const char* otg_spef_pin_name(const otg_spef* s, int32_t net, int32_t k) {
  if (!s || net < 0 || (size_t)net >= s->nets.size()) return nullptr;
  const auto& p = s->nets[net].pins;
  if (k < 0 || (size_t)k >= p.size()) return nullptr;
  return p[k].name.c_str();
}

otg_status otg_spef_names(const otg_spef* s, char* buf, size_t* bytes) {
  if (!s || !bytes) return OTG_ERR_INVALID;
  size_t need = 0;
  for (const auto& n : s->nets) {
    need += n.name.size() + 1;
    for (const auto& p : n.pins) need += p.name.size() + 1;
  }
  if (!buf) {
    *bytes = need;
    return OTG_OK;
  }
  if (*bytes < need) return OTG_ERR_WORKSPACE;
  char* o = buf;
  auto put = [&](const std::string& x) {
    std::memcpy(o, x.data(), x.size());
    o += x.size();
    *o++ = '\0';
  };
  for (const auto& n : s->nets) put(n.name);
  for (const auto& n : s->nets)
    for (const auto& p : n.pins) put(p.name);
  *bytes = need;
  return OTG_OK;
}

void otg_spef_free(otg_spef* s) { delete s; }

}  // extern "C"
