// otg_host.cu -- host-buffer entry points of libotg: a per-device context
// with cached device buffers, the chunked end-to-end RC pipeline, the
// levelization host path, and the drop-in C++ symbols of OpenTimer's CUDA
// module (see include/otg_compat.hpp).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/otg.h"
#include "../../include/otg_compat.hpp"
#include "otg_internal.cuh"

namespace otg {

static std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

namespace {

// Grow-only device buffer.
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  bool ensure(size_t need) {
    if (need <= bytes) return true;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t b = std::max<size_t>(need + need / 8, 256);
    if (cudaMalloc(&p, b) != cudaSuccess) { cudaGetLastError(); return false; }
    bytes = b;
    return true;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T* as() const { return (T*)p; }
};

struct RcChunkBufs {
  DBuf ns, edges, roots, res, cap, n2b, pid, load, delay, ldelay, imp, ss, sn, dslew, sslew, ws,
      status;
};

struct Ctx {
  int device = -1;
  bool ok = false;
  cudaStream_t st[2] = {nullptr, nullptr};
  RcChunkBufs rc[2];
  DBuf lv_fs, lv_fi, lv_out, lv_f0, lv_order, lv_level, lv_ends, lv_counts, lv_ws;
  std::mutex mu;
};

Ctx g_ctx[64];

Ctx* ctx_get() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) return nullptr;
  Ctx& c = g_ctx[d & 63];
  if (!c.ok) {
    c.device = d;
    if (cudaStreamCreateWithFlags(&c.st[0], cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c.st[1], cudaStreamNonBlocking) != cudaSuccess)
      return nullptr;
    c.ok = true;
  }
  return &c;
}

__global__ void rebase_kernel(int* a, int count, int base) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) a[i] -= base;
}

#define CK(x)                                 \
  do {                                        \
    if ((x) != cudaSuccess) {                 \
      cudaGetLastError();                     \
      return OTG_ERR_CUDA;                    \
    }                                         \
  } while (0)

// Target nodes per chunk: large enough that launch overhead vanishes,
// small enough that two chunks in flight overlap their copies.
constexpr int64_t kChunkNodes = 1 << 25;

otg_status rc_host(const otg_rc_forest* h) {
  if (!h || h->num_nets < 0) return OTG_ERR_INVALID;
  if (h->num_nets == 0) return OTG_OK;
  if (!h->nodes_start || !h->edges || !h->roots || !h->edges_res || !h->nodes_cap ||
      !h->node2bfs || !h->pid || !h->load || !h->delay || !h->ldelay || !h->impulse)
    return OTG_ERR_INVALID;
  const bool sinks = h->sinks_start != nullptr;
  if (sinks && (!h->sink_nodes || !h->driver_slew || !h->sink_slew)) return OTG_ERR_INVALID;
  const int N = h->num_nets;
  const int* ns = h->nodes_start;
  int max_n = 1;
  for (int i = 0; i < N; ++i) {
    const int n = ns[i + 1] - ns[i];
    if (n < 1) return OTG_ERR_INVALID;
    max_n = std::max(max_n, n);
  }
  Ctx* c = ctx_get();
  if (!c) return OTG_ERR_CUDA;
  std::lock_guard<std::mutex> lock(c->mu);
  // chunk plan
  std::vector<int> cut{0};
  while (cut.back() < N) {
    int i = cut.back();
    const int64_t b0 = ns[i];
    while (i < N && (i == cut.back() || (int64_t)ns[i + 1] - b0 <= kChunkNodes)) ++i;
    cut.push_back(i);
  }
  int64_t cap_nodes = 0, cap_nets = 0, cap_sinks = 1;
  for (size_t k = 0; k + 1 < cut.size(); ++k) {
    cap_nodes = std::max<int64_t>(cap_nodes, ns[cut[k + 1]] - ns[cut[k]]);
    cap_nets = std::max<int64_t>(cap_nets, cut[k + 1] - cut[k]);
    if (sinks)
      cap_sinks = std::max<int64_t>(cap_sinks,
                                    h->sinks_start[cut[k + 1]] - h->sinks_start[cut[k]]);
  }
  size_t wsb = 0;
  if (otg_rc_workspace_size((int)cap_nets, max_n, &wsb) != OTG_OK) return OTG_ERR_CUDA;
  const int nbuf = cut.size() > 2 ? 2 : 1;
  for (int k = 0; k < nbuf; ++k) {
    RcChunkBufs& B = c->rc[k];
    const size_t V = (size_t)cap_nodes, M = (size_t)cap_nodes, Nn = (size_t)cap_nets;
    bool ok = B.ns.ensure(4 * (Nn + 1)) && B.edges.ensure(8 * M) && B.roots.ensure(4 * Nn) &&
              B.res.ensure(4 * M) && B.cap.ensure(16 * V) && B.n2b.ensure(4 * V) &&
              B.pid.ensure(4 * V) && B.load.ensure(16 * V) && B.delay.ensure(16 * V) &&
              B.ldelay.ensure(16 * V) && B.imp.ensure(16 * V) && B.ws.ensure(wsb) &&
              B.status.ensure(256);
    if (ok && sinks)
      ok = B.ss.ensure(4 * (Nn + 1)) && B.sn.ensure(4 * (size_t)cap_sinks) &&
           B.dslew.ensure(16 * Nn) && B.sslew.ensure(16 * (size_t)cap_sinks);
    if (!ok) return OTG_ERR_OOM;
  }
  std::vector<int> status((cut.size() - 1) * 2, 0);
  for (size_t k = 0; k + 1 < cut.size(); ++k) {
    RcChunkBufs& B = c->rc[k % nbuf];
    cudaStream_t s = c->st[k % nbuf];
    const int n0 = cut[k], n1 = cut[k + 1], nn = n1 - n0;
    const int v0 = ns[n0], vn = ns[n1] - v0;
    const int e0 = v0 - n0, en = vn - nn;
    CK(cudaMemcpyAsync(B.ns.p, ns + n0, 4 * (size_t)(nn + 1), cudaMemcpyHostToDevice, s));
    rebase_kernel<<<(nn + 1 + 255) / 256, 256, 0, s>>>(B.ns.as<int>(), nn + 1, v0);
    count_launch();
    CK(cudaMemcpyAsync(B.edges.p, h->edges + e0, 8 * (size_t)en, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(B.roots.p, h->roots + n0, 4 * (size_t)nn, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(B.res.p, h->edges_res + e0, 4 * (size_t)en, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(B.cap.p, h->nodes_cap + 4 * (size_t)v0, 16 * (size_t)vn,
                       cudaMemcpyHostToDevice, s));
    otg_rc_forest f{};
    f.num_nets = nn;
    f.total_nodes = vn;
    f.nodes_start = B.ns.as<int>();
    f.edges = B.edges.as<otg_rc_edge>();
    f.roots = B.roots.as<int>();
    f.edges_res = B.res.as<float>();
    f.nodes_cap = B.cap.as<float>();
    f.node2bfs = B.n2b.as<int>();
    f.pid = B.pid.as<int>();
    f.load = B.load.as<float>();
    f.delay = B.delay.as<float>();
    f.ldelay = B.ldelay.as<float>();
    f.impulse = B.imp.as<float>();
    int s0 = 0, sn = 0;
    if (sinks) {
      s0 = h->sinks_start[n0];
      sn = h->sinks_start[n1] - s0;
      CK(cudaMemcpyAsync(B.ss.p, h->sinks_start + n0, 4 * (size_t)(nn + 1),
                         cudaMemcpyHostToDevice, s));
      rebase_kernel<<<(nn + 1 + 255) / 256, 256, 0, s>>>(B.ss.as<int>(), nn + 1, s0);
      count_launch();
      if (sn) CK(cudaMemcpyAsync(B.sn.p, h->sink_nodes + s0, 4 * (size_t)sn,
                                 cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(B.dslew.p, h->driver_slew + 4 * (size_t)n0, 16 * (size_t)nn,
                         cudaMemcpyHostToDevice, s));
      f.sinks_start = B.ss.as<int>();
      f.sink_nodes = B.sn.as<int>();
      f.driver_slew = B.dslew.as<float>();
      f.sink_slew = B.sslew.as<float>();
    }
    otg_status st = otg_rc_timing(&f, max_n, B.ws.p, B.ws.bytes, (otg_stream_t)s);
    if (st != OTG_OK) return st;
    CK(cudaMemcpyAsync(&status[2 * k], B.ws.p, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h->edges + e0, B.edges.p, 8 * (size_t)en, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h->node2bfs + v0, B.n2b.p, 4 * (size_t)vn, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h->pid + v0, B.pid.p, 4 * (size_t)vn, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h->load + 4 * (size_t)v0, B.load.p, 16 * (size_t)vn,
                       cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h->delay + 4 * (size_t)v0, B.delay.p, 16 * (size_t)vn,
                       cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h->ldelay + 4 * (size_t)v0, B.ldelay.p, 16 * (size_t)vn,
                       cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h->impulse + 4 * (size_t)v0, B.imp.p, 16 * (size_t)vn,
                       cudaMemcpyDeviceToHost, s));
    if (sinks && sn)
      CK(cudaMemcpyAsync(h->sink_slew + 4 * (size_t)s0, B.sslew.p, 16 * (size_t)sn,
                         cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(c->st[0]));
  CK(cudaStreamSynchronize(c->st[1]));
  for (size_t k = 0; k + 1 < cut.size(); ++k)
    if (status[2 * k]) return (otg_status)status[2 * k];
  return OTG_OK;
}

otg_status lv_host(int n, int num_edges, const int* fanin_start, const int* fanin,
                   const int* out_deg, const int* frontier0, int first_size, int* order,
                   int* level, int* level_ends, int* counts) {
  if (n < 0 || num_edges < 0 || first_size < 0 || first_size > n || !counts || !level_ends)
    return OTG_ERR_INVALID;
  if (n > 0 && (!fanin_start || !out_deg || !order || !level || (first_size && !frontier0) ||
                (num_edges && !fanin)))
    return OTG_ERR_INVALID;
  Ctx* c = ctx_get();
  if (!c) return OTG_ERR_CUDA;
  std::lock_guard<std::mutex> lock(c->mu);
  size_t wsb = 0;
  otg_status st = otg_levelize_workspace_size(n, num_edges, &wsb);
  if (st != OTG_OK) return st;
  const size_t N = (size_t)std::max(n, 1);
  if (!(c->lv_fs.ensure(4 * (N + 1)) && c->lv_fi.ensure(4 * (size_t)std::max(num_edges, 1)) &&
        c->lv_out.ensure(4 * N) && c->lv_f0.ensure(4 * N) && c->lv_order.ensure(4 * N) &&
        c->lv_level.ensure(4 * N) && c->lv_ends.ensure(4 * (N + 2)) && c->lv_counts.ensure(64) &&
        c->lv_ws.ensure(wsb)))
    return OTG_ERR_OOM;
  cudaStream_t s = c->st[0];
  CK(cudaMemcpyAsync(c->lv_fs.p, fanin_start, 4 * (size_t)(n + 1), cudaMemcpyHostToDevice, s));
  if (num_edges)
    CK(cudaMemcpyAsync(c->lv_fi.p, fanin, 4 * (size_t)num_edges, cudaMemcpyHostToDevice, s));
  if (n) CK(cudaMemcpyAsync(c->lv_out.p, out_deg, 4 * (size_t)n, cudaMemcpyHostToDevice, s));
  if (first_size)
    CK(cudaMemcpyAsync(c->lv_f0.p, frontier0, 4 * (size_t)first_size, cudaMemcpyHostToDevice, s));
  st = otg_levelize(n, num_edges, c->lv_fs.as<int>(), c->lv_fi.as<int>(), c->lv_out.as<int>(),
                    c->lv_f0.as<int>(), first_size, c->lv_order.as<int>(), c->lv_level.as<int>(),
                    c->lv_ends.as<int>(), c->lv_counts.as<int>(), c->lv_ws.p, c->lv_ws.bytes,
                    (otg_stream_t)s);
  if (st != OTG_OK) return st;
  int hc[2] = {0, 0};
  CK(cudaMemcpyAsync(hc, c->lv_counts.p, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  st = otg_levelize_status(c->lv_ws.p, (otg_stream_t)s);
  if (st != OTG_OK) return st;
  counts[0] = hc[0];
  counts[1] = hc[1];
  if (hc[1]) CK(cudaMemcpyAsync(order, c->lv_order.p, 4 * (size_t)hc[1], cudaMemcpyDeviceToHost, s));
  if (n) CK(cudaMemcpyAsync(level, c->lv_level.p, 4 * (size_t)n, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(level_ends, c->lv_ends.p, 4 * (size_t)(hc[0] + 1), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return OTG_OK;
}

}  // namespace
}  // namespace otg

extern "C" {

otg_status otg_rc_timing_host(const otg_rc_forest* host_forest) {
  return otg::rc_host(host_forest);
}

otg_status otg_levelize_host(int32_t n, int32_t num_edges, const int32_t* fanin_start,
                             const int32_t* fanin, const int32_t* out_deg,
                             const int32_t* frontier0, int32_t first_size, int32_t* order,
                             int32_t* level, int32_t* level_ends, int32_t* counts) {
  return otg::lv_host(n, num_edges, fanin_start, fanin, out_deg, frontier0, first_size, order,
                      level, level_ends, counts);
}

void otg_release_host_context(void) {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) return;
  otg::Ctx& c = otg::g_ctx[d & 63];
  std::lock_guard<std::mutex> lock(c.mu);
  for (auto& B : c.rc) {
    for (otg::DBuf* b : {&B.ns, &B.edges, &B.roots, &B.res, &B.cap, &B.n2b, &B.pid, &B.load,
                         &B.delay, &B.ldelay, &B.imp, &B.ss, &B.sn, &B.dslew, &B.sslew, &B.ws,
                         &B.status})
      b->release();
  }
  for (otg::DBuf* b : {&c.lv_fs, &c.lv_fi, &c.lv_out, &c.lv_f0, &c.lv_order, &c.lv_level,
                       &c.lv_ends, &c.lv_counts, &c.lv_ws})
    b->release();
}

const char* otg_status_string(otg_status s) {
  switch (s) {
    case OTG_OK: return "ok";
    case OTG_ERR_INVALID: return "invalid argument or id out of range";
    case OTG_ERR_CUDA: return "CUDA runtime error";
    case OTG_ERR_OOM: return "out of memory";
    case OTG_ERR_NOT_TREE: return "RC net is not a spanning tree";
    case OTG_ERR_CYCLE: return "timing graph has a cycle";
    case OTG_ERR_TIMEOUT: return "bounded device wait timed out";
    case OTG_ERR_TOO_LARGE: return "net larger than the workspace was sized for";
    case OTG_ERR_WORKSPACE: return "workspace too small";
    case OTG_ERR_ADMISSION: return "request exceeds the device memory budget";
  }
  return "unknown status";
}

uint64_t otg_kernel_launches(void) { return otg::g_launches.load(); }

}  // extern "C"

// ------------------------------------------------- reference drop-in symbols

void rct_bfs_and_compute_cuda(RctEdgeArrayCUDA d) {
  otg_rc_forest f{};
  f.num_nets = d.num_nets;
  f.total_nodes = d.total_num_nodes;
  f.nodes_start = d.rct_nodes_start;
  f.edges = reinterpret_cast<otg_rc_edge*>(d.rct_edges);
  f.roots = d.rct_roots;
  f.edges_res = d.rct_edges_res;
  f.nodes_cap = d.rct_nodes_cap;
  f.node2bfs = d.rct_node2bfs_order;
  f.pid = d.rct_pid;
  f.load = d.load;
  f.delay = d.delay;
  f.ldelay = d.ldelay;
  f.impulse = d.impulse;
  const otg_status st = otg_rc_timing_host(&f);
  if (st != OTG_OK) std::fprintf(stderr, "rct_bfs_and_compute_cuda: %s\n", otg_status_string(st));
}

void rct_compute_cuda(RctCUDA d) {
  // The tree arrives BFS-ordered (parent of i is i - pid[i]); rebuild it as
  // an edge list with slot ids, run the fused path and map the results back
  // to the caller's order.
  const int N = d.num_nets, V = d.total_num_nodes;
  std::vector<otg_rc_edge> edges((size_t)std::max(V - N, 0));
  std::vector<float> res(edges.size());
  std::vector<int> roots((size_t)N, 0), n2b((size_t)V), pid((size_t)V);
  std::vector<float> out[4];
  for (auto& o : out) o.resize(4 * (size_t)V);
  for (int net = 0; net < N; ++net) {
    const int b = d.rct_nodes_start[net], e = d.rct_nodes_start[net + 1];
    for (int i = b + 1; i < e; ++i) {
      const size_t k = (size_t)(i - net - 1);
      edges[k] = otg_rc_edge{i - b - d.rct_pid[i], i - b};
      res[k] = d.pres[i];
    }
  }
  otg_rc_forest f{};
  f.num_nets = N;
  f.total_nodes = V;
  f.nodes_start = d.rct_nodes_start;
  f.edges = edges.data();
  f.roots = roots.data();
  f.edges_res = res.data();
  f.nodes_cap = d.cap;
  f.node2bfs = n2b.data();
  f.pid = pid.data();
  f.load = out[0].data();
  f.delay = out[1].data();
  f.ldelay = out[2].data();
  f.impulse = out[3].data();
  const otg_status st = otg_rc_timing_host(&f);
  if (st != OTG_OK) {
    std::fprintf(stderr, "rct_compute_cuda: %s\n", otg_status_string(st));
    return;
  }
  float* dst[4] = {d.load, d.delay, d.ldelay, d.impulse};
  for (int net = 0; net < N; ++net) {
    const int b = d.rct_nodes_start[net], e = d.rct_nodes_start[net + 1];
    for (int i = b; i < e; ++i)
      for (int q = 0; q < 4; ++q)
        std::memcpy(dst[q] + 4 * (size_t)i, out[q].data() + 4 * (size_t)(b + n2b[i]),
                    4 * sizeof(float));
  }
}

void toposort_compute_cuda(int n, int num_edges, int first_size, int* edgelist_start,
                           int* edgelist, int* out, int* frontiers,
                           std::vector<int>& frontiers_ends) {
  std::vector<int> order((size_t)std::max(n, 1)), level((size_t)std::max(n, 1)),
      ends((size_t)n + 2);
  int counts[2] = {0, 0};
  const otg_status st = otg_levelize_host(n, num_edges, edgelist_start, edgelist, out, frontiers,
                                          first_size, order.data(), level.data(), ends.data(),
                                          counts);
  if (st != OTG_OK) {
    std::fprintf(stderr, "toposort_compute_cuda: %s\n", otg_status_string(st));
    return;
  }
  std::memcpy(frontiers, order.data(), sizeof(int) * (size_t)counts[1]);
  for (int k = 2; k <= counts[0]; ++k) frontiers_ends.push_back(ends[k]);
}
