// otg_serve.cu -- device-resident designs and the incremental timing server.
//
// The reference re-times dirty nets on the CPU (Net::_update_rc_timing skips
// clean nets, ot/timer/net.cpp:536-540) and its GPU path re-flattens every
// net per update (timer.cpp:929-970).  Here a design's RC state stays on the
// device, and a request (node-cap and driver-slew updates, i.e. gate
// resizes) re-times only its dirty nets.
//
// Batching: a dispatcher thread takes pending requests of idle designs --
// one request per design per batch, so every request sees exactly the
// state its predecessors left (the same result alone or in a mix) -- into
// one of `slots` batch slots.  A slot replays a CUDA graph captured once:
//   clear counters -> apply_kernel (writes the updates, marks dirty nets,
//   lists distinct (design, net) items) -> the fused RC pass over the items
//   of all designs (rc_launch_items) -> result_kernel (per-request worst
//   |sink slew| and sink delay over its dirty nets) -> publish_kernel.
// Request data and results travel through pinned, mapped host buffers, so
// the graph has no size-dependent copies.  Slots run on their own streams
// and overlap on the device; requests that arrive meanwhile are batched as
// soon as a slot and their design are free (continuous batching).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/otg.h"
#include "otg_internal.cuh"

namespace otg {
namespace {

constexpr int kMaxDesigns = 256;

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// What the apply/result kernels need of a design.
struct DesignDev {
  int num_nets;
  const int* nodes_start;
  float4* cap;
  float4* driver_slew;
  const int* sinks_start;
  const int* sink_nodes;
  const int* node2bfs;
  const float4* delay;
  const float4* sink_slew;
  int* marks;   // batch stamp of the last batch that dirtied each net
  int* status;  // [0] first device-side error of the design, [1] its net
};

// A batch as the device sees it (mapped host memory).
struct BatchHdr {
  int num_req, num_cap, num_slew, stamp;
};
struct BatchView {
  BatchHdr* hdr;
  int* req_design;
  int* cap_req;
  int* cap_net;
  int* cap_node;
  float4* cap_val;
  int* slew_req;
  int* slew_net;
  float4* slew_val;
};
struct ResultDev {
  unsigned slew[4], delay[4];
  int status, dirty;
};

__global__ void apply_kernel(BatchView b, const DesignDev* dz, int2* items, int* num_items,
                             int cap_items, ResultDev* res) {
  const BatchHdr h = *b.hdr;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  for (int r = tid; r < h.num_req; r += stride) {
    const int d = b.req_design[r];
    dz[d].status[0] = 0;
    dz[d].status[1] = -1;
  }
  for (int u = tid; u < h.num_cap + h.num_slew; u += stride) {
    const bool is_cap = u < h.num_cap;
    const int k = is_cap ? u : u - h.num_cap;
    const int r = is_cap ? b.cap_req[k] : b.slew_req[k];
    const int d = b.req_design[r];
    const DesignDev D = dz[d];
    const int net = is_cap ? b.cap_net[k] : b.slew_net[k];
    if ((unsigned)net >= (unsigned)D.num_nets) {
      atomicCAS(&res[r].status, 0, (int)OTG_ERR_INVALID);
      continue;
    }
    if (is_cap) {
      const int base = D.nodes_start[net], n = D.nodes_start[net + 1] - base;
      const int node = b.cap_node[k];
      if ((unsigned)node >= (unsigned)n) {
        atomicCAS(&res[r].status, 0, (int)OTG_ERR_INVALID);
        continue;
      }
      D.cap[base + node] = b.cap_val[k];
    } else {
      D.driver_slew[net] = b.slew_val[k];
    }
    if (atomicExch(&D.marks[net], h.stamp) != h.stamp) {
      const int pos = atomicAdd(num_items, 1);
      if (pos < cap_items) items[pos] = make_int2(d, net);
      else atomicCAS(&res[r].status, 0, (int)OTG_ERR_WORKSPACE);
      atomicAdd(&res[r].dirty, 1);
    }
  }
}

__device__ __forceinline__ void amax(unsigned* p, float v) { atomicMax(p, __float_as_uint(v)); }

__global__ void result_kernel(BatchView b, const DesignDev* dz, ResultDev* res) {
  const BatchHdr h = *b.hdr;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  for (int u = tid; u < h.num_cap + h.num_slew; u += stride) {
    const bool is_cap = u < h.num_cap;
    const int k = is_cap ? u : u - h.num_cap;
    const int r = is_cap ? b.cap_req[k] : b.slew_req[k];
    const DesignDev D = dz[b.req_design[r]];
    const int net = is_cap ? b.cap_net[k] : b.slew_net[k];
    if ((unsigned)net >= (unsigned)D.num_nets || !D.sinks_start) continue;
    const int base = D.nodes_start[net];
    for (int s = D.sinks_start[net]; s < D.sinks_start[net + 1]; ++s) {
      const float4 sl = D.sink_slew[s];
      const int v = D.sink_nodes[s];
      const float4 dl = D.delay[base + D.node2bfs[base + v]];
      amax(&res[r].slew[0], fabsf(sl.x));
      amax(&res[r].slew[1], fabsf(sl.y));
      amax(&res[r].slew[2], fabsf(sl.z));
      amax(&res[r].slew[3], fabsf(sl.w));
      amax(&res[r].delay[0], fabsf(dl.x));
      amax(&res[r].delay[1], fabsf(dl.y));
      amax(&res[r].delay[2], fabsf(dl.z));
      amax(&res[r].delay[3], fabsf(dl.w));
    }
  }
}

__global__ void publish_kernel(BatchView b, const DesignDev* dz, const ResultDev* res,
                               otg_result* out) {
  const int nreq = b.hdr->num_req;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nreq; r += gridDim.x * blockDim.x) {
    const ResultDev x = res[r];
    otg_result o;
    for (int c = 0; c < 4; ++c) {
      o.worst_slew[c] = __uint_as_float(x.slew[c]);
      o.worst_delay[c] = __uint_as_float(x.delay[c]);
    }
    const int ds = dz[b.req_design[r]].status[0];
    o.status = x.status ? x.status : ds;
    o.dirty_nets = x.dirty;
    o.t_submit_ns = 0;
    o.t_done_ns = 0;
    out[r] = o;
  }
}

struct Request {
  int64_t ticket;
  int design;
  std::vector<int> cap_net, cap_node, slew_net;
  std::vector<float4> cap_val, slew_val;
  int64_t t_submit;
};

struct Design {
  bool live = false;
  int num_nets = 0, total_nodes = 0, num_sinks = 0, max_n = 1;
  size_t footprint = 0;
  std::vector<void*> allocs;
  int *ns = nullptr, *roots = nullptr, *n2b = nullptr, *pid = nullptr, *ss = nullptr, *sn = nullptr,
      *marks = nullptr, *status = nullptr;
  int2* edges = nullptr;
  float *res = nullptr, *cap = nullptr, *load = nullptr, *delay = nullptr, *ldelay = nullptr,
        *imp = nullptr, *dslew = nullptr, *sslew = nullptr;
  bool busy = false;
};

struct Slot {
  cudaStream_t st = nullptr;
  cudaEvent_t ev = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_gen = -1;
  char* hbuf = nullptr;       // pinned, mapped
  BatchView hv{}, dv{};       // host and device views of hbuf
  otg_result* hres = nullptr;  // pinned, mapped
  otg_result* dres_out = nullptr;
  ResultDev* dres = nullptr;
  int2* items = nullptr;
  int* num_items = nullptr;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  int ws_max_n = 0;
  bool busy = false;
  std::vector<int64_t> tickets;
  std::vector<int> designs;
};

}  // namespace

struct Server {
  size_t budget = 0, used = 0;
  int R = 0, U = 0;
  std::vector<Design> designs;
  char* forests_dev = nullptr;  // kMaxDesigns x rc_args_bytes()
  DesignDev* dz_dev = nullptr;
  int max_n = 1;
  int gen = 0;  // bumps when max_n grows (graphs must be recaptured)
  int stamp = 0;
  std::vector<Slot> slots;
  Slot sync_slot;
  std::mutex mu;
  std::mutex sync_mu;  // serializes otg_server_update_sync callers (one sync slot)
  std::condition_variable cv_disp, cv_done;
  std::deque<Request> pending;
  std::unordered_map<int64_t, otg_result> done;
  int64_t next_ticket = 1;
  bool stop = false;
  std::thread disp;
  int device = 0;

  ~Server();
  otg_status init_slot(Slot& s);
  otg_status ensure_ws(Slot& s);
  otg_status launch_batch(Slot& s, bool graph);
  otg_status capture(Slot& s);
  void fill(Slot& s, const std::vector<Request*>& reqs);
  void dispatcher();
};

namespace {

size_t batch_bytes(int R, int U) {
  size_t o = 0;
  auto take = [&](size_t b) { size_t r = o; o = (o + b + 15) & ~(size_t)15; return r; };
  take(sizeof(BatchHdr));
  take(4 * (size_t)R);
  take(4 * (size_t)U * 3);
  take(16 * (size_t)U);
  take(4 * (size_t)U * 2);
  take(16 * (size_t)U);
  return o;
}

BatchView batch_view(char* base, int R, int U) {
  BatchView v;
  size_t o = 0;
  auto take = [&](size_t b) { char* p = base + o; o = (o + b + 15) & ~(size_t)15; return p; };
  v.hdr = (BatchHdr*)take(sizeof(BatchHdr));
  v.req_design = (int*)take(4 * (size_t)R);
  char* c3 = take(4 * (size_t)U * 3);
  v.cap_req = (int*)c3;
  v.cap_net = v.cap_req + U;
  v.cap_node = v.cap_net + U;
  v.cap_val = (float4*)take(16 * (size_t)U);
  char* s2 = take(4 * (size_t)U * 2);
  v.slew_req = (int*)s2;
  v.slew_net = v.slew_req + U;
  v.slew_val = (float4*)take(16 * (size_t)U);
  return v;
}

#define SCK(x)                  \
  do {                          \
    if ((x) != cudaSuccess) {   \
      cudaGetLastError();       \
      return OTG_ERR_CUDA;      \
    }                           \
  } while (0)

}  // namespace

otg_status Server::init_slot(Slot& s) {
  SCK(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
  SCK(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
  SCK(cudaHostAlloc((void**)&s.hbuf, batch_bytes(R, U), cudaHostAllocMapped));
  char* dbuf = nullptr;
  SCK(cudaHostGetDevicePointer((void**)&dbuf, s.hbuf, 0));
  s.hv = batch_view(s.hbuf, R, U);
  s.dv = batch_view(dbuf, R, U);
  SCK(cudaHostAlloc((void**)&s.hres, sizeof(otg_result) * (size_t)R, cudaHostAllocMapped));
  SCK(cudaHostGetDevicePointer((void**)&s.dres_out, s.hres, 0));
  SCK(cudaMalloc(&s.dres, sizeof(ResultDev) * (size_t)R));
  SCK(cudaMalloc(&s.items, sizeof(int2) * (size_t)U));
  SCK(cudaMalloc(&s.num_items, 64));
  return OTG_OK;
}

otg_status Server::ensure_ws(Slot& s) {
  if (s.ws && s.ws_max_n >= max_n) return OTG_OK;
  size_t need = 0;
  otg_status st = otg_rc_workspace_size(U, max_n, &need);
  if (st != OTG_OK) return st;
  if (s.ws) cudaFree(s.ws);
  s.ws = nullptr;
  SCK(cudaMalloc(&s.ws, need));
  s.ws_bytes = need;
  s.ws_max_n = max_n;
  return OTG_OK;
}

// Enqueues one batch on the slot's stream (graph = false: direct launches).
otg_status Server::launch_batch(Slot& s, bool graph) {
  if (graph) {
    SCK(cudaGraphLaunch(s.exec, s.st));
    count_launch();
    return OTG_OK;
  }
  SCK(cudaMemsetAsync(s.num_items, 0, 64, s.st));
  SCK(cudaMemsetAsync(s.dres, 0, sizeof(ResultDev) * (size_t)R, s.st));
  const int blocks = std::max(1, std::min(1024, (U + 255) / 256));
  apply_kernel<<<blocks, 256, 0, s.st>>>(s.dv, dz_dev, s.items, s.num_items, U, s.dres);
  count_launch();
  otg_status st = rc_launch_items((const RcArgsOpaque*)forests_dev, s.items, s.num_items, U,
                                  s.ws_max_n, s.ws, s.ws_bytes, s.st);
  if (st != OTG_OK) return st;
  result_kernel<<<blocks, 256, 0, s.st>>>(s.dv, dz_dev, s.dres);
  count_launch();
  publish_kernel<<<std::max(1, std::min(64, (R + 255) / 256)), 256, 0, s.st>>>(s.dv, dz_dev, s.dres,
                                                                              s.dres_out);
  count_launch();
  SCK(cudaGetLastError());
  return OTG_OK;
}

otg_status Server::capture(Slot& s) {
  otg_status st = ensure_ws(s);
  if (st != OTG_OK) return st;
  if (s.exec) {
    cudaGraphExecDestroy(s.exec);
    s.exec = nullptr;
  }
  // one direct batch of zero requests first: sets kernel attributes outside
  // the capture
  s.hv.hdr->num_req = s.hv.hdr->num_cap = s.hv.hdr->num_slew = 0;
  st = launch_batch(s, false);
  if (st != OTG_OK) return st;
  SCK(cudaStreamSynchronize(s.st));
  cudaGraph_t g = nullptr;
  SCK(cudaStreamBeginCapture(s.st, cudaStreamCaptureModeThreadLocal));
  st = launch_batch(s, false);
  cudaError_t e = cudaStreamEndCapture(s.st, &g);
  if (st != OTG_OK || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return st != OTG_OK ? st : OTG_ERR_CUDA;
  }
  e = cudaGraphInstantiate(&s.exec, g, 0);
  cudaGraphDestroy(g);
  SCK(e);
  s.graph_gen = gen;
  return OTG_OK;
}

void Server::fill(Slot& s, const std::vector<Request*>& reqs) {
  BatchView& v = s.hv;
  int nc = 0, nsl = 0;
  for (size_t r = 0; r < reqs.size(); ++r) {
    const Request& q = *reqs[r];
    v.req_design[r] = q.design;
    for (size_t k = 0; k < q.cap_net.size(); ++k, ++nc) {
      v.cap_req[nc] = (int)r;
      v.cap_net[nc] = q.cap_net[k];
      v.cap_node[nc] = q.cap_node[k];
      v.cap_val[nc] = q.cap_val[k];
    }
    for (size_t k = 0; k < q.slew_net.size(); ++k, ++nsl) {
      v.slew_req[nsl] = (int)r;
      v.slew_net[nsl] = q.slew_net[k];
      v.slew_val[nsl] = q.slew_val[k];
    }
  }
  v.hdr->num_req = (int)reqs.size();
  v.hdr->num_cap = nc;
  v.hdr->num_slew = nsl;
  v.hdr->stamp = ++stamp;
}

void Server::dispatcher() {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> lk(mu);
  while (true) {
    // completions
    bool any_busy = false;
    for (auto& s : slots) {
      if (!s.busy) continue;
      if (cudaEventQuery(s.ev) == cudaSuccess) {
        const int64_t t = now_ns();
        for (size_t r = 0; r < s.tickets.size(); ++r) {
          otg_result o = s.hres[r];
          o.t_done_ns = t;
          auto it = done.find(s.tickets[r]);
          if (it != done.end()) {
            o.t_submit_ns = it->second.t_submit_ns;
            it->second = o;
          }
        }
        for (int d : s.designs) designs[d].busy = false;
        s.tickets.clear();
        s.designs.clear();
        s.busy = false;
        cv_done.notify_all();
      } else {
        any_busy = true;
      }
    }
    if (stop && !any_busy) break;
    // new batches
    for (auto& s : slots) {
      if (s.busy || pending.empty() || stop) continue;
      std::vector<Request*> take;
      std::vector<bool> seen(designs.size(), false);
      size_t nu = 0;
      for (auto& q : pending) {
        if ((int)take.size() >= R) break;
        // The first pending request of a design decides for the design:
        // a later one never overtakes it.
        if (seen[q.design]) continue;
        seen[q.design] = true;
        const size_t qu = q.cap_net.size() + q.slew_net.size();
        if (designs[q.design].busy || nu + qu > (size_t)U) continue;
        nu += qu;
        take.push_back(&q);
      }
      if (take.empty()) break;
      if (s.graph_gen != gen) {
        if (capture(s) != OTG_OK) {
          // cannot run: fail the requests
          for (Request* q : take) {
            auto it = done.find(q->ticket);
            if (it != done.end()) {
              it->second.status = OTG_ERR_CUDA;
              it->second.t_done_ns = now_ns();
            }
            q->ticket = -1;
          }
          pending.erase(std::remove_if(pending.begin(), pending.end(),
                                       [](const Request& q) { return q.ticket < 0; }),
                        pending.end());
          cv_done.notify_all();
          continue;
        }
      }
      fill(s, take);
      for (Request* q : take) {
        s.tickets.push_back(q->ticket);
        s.designs.push_back(q->design);
        designs[q->design].busy = true;
        q->ticket = -q->ticket - 1;  // taken
      }
      pending.erase(std::remove_if(pending.begin(), pending.end(),
                                   [](const Request& q) { return q.ticket < 0; }),
                    pending.end());
      s.busy = true;
      if (launch_batch(s, true) != OTG_OK || cudaEventRecord(s.ev, s.st) != cudaSuccess) {
        cudaGetLastError();
        for (size_t r = 0; r < s.tickets.size(); ++r) {
          auto it = done.find(s.tickets[r]);
          if (it != done.end()) {
            it->second.status = OTG_ERR_CUDA;
            it->second.t_done_ns = now_ns();
          }
        }
        for (int d : s.designs) designs[d].busy = false;
        s.tickets.clear();
        s.designs.clear();
        s.busy = false;
        cv_done.notify_all();
      }
    }
    bool busy_now = false;
    for (auto& s : slots) busy_now |= s.busy;
    if (busy_now) {
      lk.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(5));
      lk.lock();
    } else {
      cv_disp.wait(lk, [&] { return stop || !pending.empty(); });
    }
  }
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu);
    stop = true;
  }
  cv_disp.notify_all();
  if (disp.joinable()) disp.join();
  cudaSetDevice(device);
  auto free_slot = [](Slot& s) {
    if (s.exec) cudaGraphExecDestroy(s.exec);
    if (s.st) cudaStreamSynchronize(s.st);
    if (s.ev) cudaEventDestroy(s.ev);
    if (s.st) cudaStreamDestroy(s.st);
    if (s.hbuf) cudaFreeHost(s.hbuf);
    if (s.hres) cudaFreeHost(s.hres);
    cudaFree(s.dres);
    cudaFree(s.items);
    cudaFree(s.num_items);
    cudaFree(s.ws);
  };
  for (auto& s : slots) free_slot(s);
  free_slot(sync_slot);
  for (auto& d : designs)
    for (void* p : d.allocs) cudaFree(p);
  cudaFree(forests_dev);
  cudaFree(dz_dev);
}

}  // namespace otg

using otg::Server;

struct otg_server : public otg::Server {};

namespace otg {
otg_status make_request(otg_server* s, int32_t d, int32_t num_cap, const int32_t* cap_net,
                               const int32_t* cap_node, const float* cap_val, int32_t num_slew,
                               const int32_t* slew_net, const float* slew_val,
                               otg::Request* q) {
  if (!s || d < 0 || d >= otg::kMaxDesigns || !s->designs[d].live || num_cap < 0 || num_slew < 0 ||
      num_cap + num_slew > s->U || (num_cap && (!cap_net || !cap_node || !cap_val)) ||
      (num_slew && (!slew_net || !slew_val)))
    return OTG_ERR_INVALID;
  q->design = d;
  // A node (net) updated twice in one request keeps its last value: only
  // the last occurrence is kept, so the parallel apply is deterministic.
  std::unordered_set<uint64_t> seen;
  q->cap_net.clear();
  q->cap_node.clear();
  q->cap_val.clear();
  for (int k = num_cap - 1; k >= 0; --k) {
    const uint64_t key = ((uint64_t)(uint32_t)cap_net[k] << 32) | (uint32_t)cap_node[k];
    if (num_cap > 1 && !seen.insert(key).second) continue;
    q->cap_net.push_back(cap_net[k]);
    q->cap_node.push_back(cap_node[k]);
    q->cap_val.push_back(make_float4(cap_val[4 * k], cap_val[4 * k + 1], cap_val[4 * k + 2],
                                     cap_val[4 * k + 3]));
  }
  seen.clear();
  q->slew_net.clear();
  q->slew_val.clear();
  for (int k = num_slew - 1; k >= 0; --k) {
    if (num_slew > 1 && !seen.insert((uint32_t)slew_net[k]).second) continue;
    q->slew_net.push_back(slew_net[k]);
    q->slew_val.push_back(make_float4(slew_val[4 * k], slew_val[4 * k + 1], slew_val[4 * k + 2],
                                      slew_val[4 * k + 3]));
  }
  q->t_submit = otg::now_ns();
  return OTG_OK;
}
}  // namespace otg

extern "C" {

otg_status otg_server_create(size_t budget_bytes, int32_t slots, int32_t max_requests,
                             int32_t max_updates, otg_server** out) {
  if (!out || slots < 1 || max_requests < 1 || max_updates < 1) return OTG_ERR_INVALID;
  otg_server* s = new (std::nothrow) otg_server();
  if (!s) return OTG_ERR_OOM;
  cudaGetDevice(&s->device);
  s->budget = budget_bytes;
  s->R = max_requests;
  s->U = max_updates;
  s->designs.resize(otg::kMaxDesigns);
  otg_status st = OTG_OK;
  if (cudaMalloc((void**)&s->forests_dev, otg::rc_args_bytes() * otg::kMaxDesigns) != cudaSuccess ||
      cudaMalloc((void**)&s->dz_dev, sizeof(otg::DesignDev) * otg::kMaxDesigns) != cudaSuccess)
    st = OTG_ERR_OOM;
  s->slots.resize(slots);
  for (auto& sl : s->slots)
    if (st == OTG_OK) st = s->init_slot(sl);
  if (st == OTG_OK) st = s->init_slot(s->sync_slot);
  if (st != OTG_OK) {
    cudaGetLastError();
    delete s;
    return st;
  }
  s->disp = std::thread([s] { s->dispatcher(); });
  *out = s;
  return OTG_OK;
}

void otg_server_destroy(otg_server* s) { delete s; }

otg_status otg_server_add_design(otg_server* s, const otg_rc_forest* h, int32_t* design_id,
                                 size_t* footprint_bytes) {
  if (!s || !h || !design_id || h->num_nets < 1 || !h->nodes_start || !h->edges || !h->roots ||
      !h->edges_res || !h->nodes_cap || !h->sinks_start || !h->sink_nodes || !h->driver_slew)
    return OTG_ERR_INVALID;
  const int N = h->num_nets, V = h->nodes_start[N], E = V - N, S = h->sinks_start[N];
  int max_n = 1;
  for (int i = 0; i < N; ++i) max_n = std::max(max_n, h->nodes_start[i + 1] - h->nodes_start[i]);
  const size_t fp = 4 * (size_t)(N + 1) * 2 + 8 * (size_t)E + 4 * (size_t)N + 4 * (size_t)E +
                    16 * (size_t)V * 5 + 4 * (size_t)V * 2 + 4 * (size_t)S + 16 * (size_t)S +
                    16 * (size_t)N + 4 * (size_t)N + 64;
  // Admission: reserve the footprint and an id under the lock; upload and
  // time the design without it, so batches of other designs keep flowing.
  int d = -1;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->budget && s->used + fp > s->budget) return OTG_ERR_ADMISSION;
    for (int i = 0; i < otg::kMaxDesigns; ++i)
      if (!s->designs[i].live && !s->designs[i].busy) { d = i; break; }
    if (d < 0) return OTG_ERR_ADMISSION;
    s->designs[d].busy = true;  // reserved
    s->used += fp;
  }
  otg::Design D;
  auto dalloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    D.allocs.push_back(p);
    return p;
  };
  D.ns = (int*)dalloc(4 * (size_t)(N + 1));
  D.edges = (int2*)dalloc(8 * (size_t)E);
  D.roots = (int*)dalloc(4 * (size_t)N);
  D.res = (float*)dalloc(4 * (size_t)E);
  D.cap = (float*)dalloc(16 * (size_t)V);
  D.n2b = (int*)dalloc(4 * (size_t)V);
  D.pid = (int*)dalloc(4 * (size_t)V);
  D.load = (float*)dalloc(16 * (size_t)V);
  D.delay = (float*)dalloc(16 * (size_t)V);
  D.ldelay = (float*)dalloc(16 * (size_t)V);
  D.imp = (float*)dalloc(16 * (size_t)V);
  D.ss = (int*)dalloc(4 * (size_t)(N + 1));
  D.sn = (int*)dalloc(4 * (size_t)S);
  D.dslew = (float*)dalloc(16 * (size_t)N);
  D.sslew = (float*)dalloc(16 * (size_t)S);
  D.marks = (int*)dalloc(4 * (size_t)N);
  D.status = (int*)dalloc(64);
  bool ok = true;
  for (void* p : D.allocs) ok &= p != nullptr;
  auto cp = [&](void* dst, const void* src, size_t b) {
    if (ok && b) ok = cudaMemcpy(dst, src, b, cudaMemcpyHostToDevice) == cudaSuccess;
  };
  cp(D.ns, h->nodes_start, 4 * (size_t)(N + 1));
  cp(D.edges, h->edges, 8 * (size_t)E);
  cp(D.roots, h->roots, 4 * (size_t)N);
  cp(D.res, h->edges_res, 4 * (size_t)E);
  cp(D.cap, h->nodes_cap, 16 * (size_t)V);
  cp(D.ss, h->sinks_start, 4 * (size_t)(N + 1));
  cp(D.sn, h->sink_nodes, 4 * (size_t)S);
  cp(D.dslew, h->driver_slew, 16 * (size_t)N);
  if (ok) ok = cudaMemset(D.marks, 0, 4 * (size_t)N) == cudaSuccess &&
               cudaMemset(D.status, 0, 64) == cudaSuccess;
  otg_rc_forest f{};
  f.num_nets = N;
  f.total_nodes = V;
  f.nodes_start = D.ns;
  f.edges = (otg_rc_edge*)D.edges;
  f.roots = D.roots;
  f.edges_res = D.res;
  f.nodes_cap = D.cap;
  f.node2bfs = D.n2b;
  f.pid = D.pid;
  f.load = D.load;
  f.delay = D.delay;
  f.ldelay = D.ldelay;
  f.impulse = D.imp;
  f.sinks_start = D.ss;
  f.sink_nodes = D.sn;
  f.driver_slew = D.dslew;
  f.sink_slew = D.sslew;
  // the first full pass, with a temporary workspace
  otg_status st = ok ? OTG_OK : OTG_ERR_OOM;
  void* ws = nullptr;
  size_t wsb = 0;
  if (st == OTG_OK) st = otg_rc_workspace_size(N, max_n, &wsb);
  if (st == OTG_OK && cudaMalloc(&ws, wsb) != cudaSuccess) {
    cudaGetLastError();
    st = OTG_ERR_OOM;
  }
  if (st == OTG_OK) st = otg_rc_timing(&f, max_n, ws, wsb, nullptr);
  if (st == OTG_OK) st = otg_rc_status(ws, nullptr, nullptr);
  if (ws) cudaFree(ws);
  std::vector<char> blob(otg::rc_args_bytes());
  if (st == OTG_OK) {
    otg::rc_args_fill(&f, D.status, blob.data());
    otg::DesignDev dd{N, D.ns, (float4*)D.cap, (float4*)D.dslew, D.ss, D.sn, D.n2b,
                      (const float4*)D.delay, (const float4*)D.sslew, D.marks, D.status};
    if (cudaMemcpy(s->forests_dev + (size_t)d * blob.size(), blob.data(), blob.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->dz_dev + d, &dd, sizeof(dd), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      st = OTG_ERR_CUDA;
    }
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (st != OTG_OK) {
    for (void* p : D.allocs) cudaFree(p);
    s->designs[d].busy = false;
    s->used -= fp;
    return st;
  }
  D.live = true;
  D.num_nets = N;
  D.total_nodes = V;
  D.num_sinks = S;
  D.max_n = max_n;
  D.footprint = fp;
  D.busy = false;
  s->designs[d] = D;
  if (max_n > s->max_n) {
    s->max_n = max_n;
    s->gen++;
  }
  *design_id = d;
  if (footprint_bytes) *footprint_bytes = fp;
  return OTG_OK;
}

otg_status otg_server_remove_design(otg_server* s, int32_t d) {
  if (!s || d < 0 || d >= otg::kMaxDesigns) return OTG_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  otg::Design& D = s->designs[d];
  if (!D.live) return OTG_ERR_INVALID;
  s->cv_done.wait(lk, [&] {
    if (D.busy) return false;
    for (auto& q : s->pending)
      if (q.design == d) return false;
    return true;
  });
  for (void* p : D.allocs) cudaFree(p);
  s->used -= D.footprint;
  D = otg::Design{};
  return OTG_OK;
}


otg_status otg_server_submit(otg_server* s, int32_t d, int32_t num_cap, const int32_t* cap_net,
                             const int32_t* cap_node, const float* cap_val, int32_t num_slew,
                             const int32_t* slew_net, const float* slew_val, int64_t* ticket) {
  if (!s || !ticket) return OTG_ERR_INVALID;
  otg::Request q;
  otg_status st;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    st = otg::make_request(s, d, num_cap, cap_net, cap_node, cap_val, num_slew, slew_net, slew_val, &q);
    if (st != OTG_OK) return st;
    q.ticket = s->next_ticket++;
    otg_result r{};
    r.status = -1;  // pending
    r.t_submit_ns = q.t_submit;
    s->done[q.ticket] = r;
    *ticket = q.ticket;
    s->pending.push_back(std::move(q));
  }
  s->cv_disp.notify_one();
  return OTG_OK;
}

otg_status otg_server_wait(otg_server* s, int64_t ticket, int32_t timeout_ms, otg_result* out) {
  if (!s || !out) return OTG_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->done.find(ticket);
  if (it == s->done.end()) return OTG_ERR_INVALID;
  auto ready = [&] { return s->done[ticket].t_done_ns != 0; };
  if (timeout_ms < 0) {
    s->cv_done.wait(lk, ready);
  } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    return OTG_ERR_TIMEOUT;
  }
  *out = s->done[ticket];
  s->done.erase(ticket);
  return OTG_OK;
}

otg_status otg_server_update_sync(otg_server* s, int32_t d, int32_t num_cap,
                                  const int32_t* cap_net, const int32_t* cap_node,
                                  const float* cap_val, int32_t num_slew, const int32_t* slew_net,
                                  const float* slew_val, otg_result* out) {
  if (!out) return OTG_ERR_INVALID;
  if (!s) return OTG_ERR_INVALID;
  otg::Request q;
  std::lock_guard<std::mutex> sync_lk(s->sync_mu);
  std::unique_lock<std::mutex> lk(s->mu);
  otg_status st =
      otg::make_request(s, d, num_cap, cap_net, cap_node, cap_val, num_slew, slew_net, slew_val, &q);
  if (st != OTG_OK) return st;
  s->cv_done.wait(lk, [&] { return !s->designs[d].busy; });
  s->designs[d].busy = true;
  otg::Slot& sl = s->sync_slot;
  st = s->ensure_ws(sl);
  std::vector<otg::Request*> one{&q};
  if (st == OTG_OK) {
    s->fill(sl, one);
    lk.unlock();
    st = s->launch_batch(sl, false);
    if (st == OTG_OK && cudaStreamSynchronize(sl.st) != cudaSuccess) {
      cudaGetLastError();
      st = OTG_ERR_CUDA;
    }
    lk.lock();
  }
  s->designs[d].busy = false;
  s->cv_done.notify_all();
  if (st != OTG_OK) return st;
  *out = sl.hres[0];
  out->t_submit_ns = q.t_submit;
  out->t_done_ns = otg::now_ns();
  return OTG_OK;
}

otg_status otg_server_replay(otg_server* s, int32_t num_req, const int64_t* arrival_ns,
                             const int32_t* design, const int32_t* cap_start,
                             const int32_t* cap_net, const int32_t* cap_node,
                             const float* cap_val, const int32_t* slew_start,
                             const int32_t* slew_net, const float* slew_val, int32_t plain,
                             int64_t* latency_ns, int64_t* makespan_ns) {
  if (!s || num_req < 0 || !arrival_ns || !design || !cap_start || !slew_start || !latency_ns ||
      !makespan_ns)
    return OTG_ERR_INVALID;
  const int64_t t0 = otg::now_ns();
  auto until = [&](int64_t t) {
    // sleep to within ~50 us of the arrival, then spin
    int64_t now = otg::now_ns();
    if (t - now > 60000) std::this_thread::sleep_for(std::chrono::nanoseconds(t - now - 50000));
    while (otg::now_ns() < t) {
    }
  };
  auto args = [&](int r, otg::Request* q) {
    const int c0 = cap_start[r], c1 = cap_start[r + 1], s0 = slew_start[r], s1 = slew_start[r + 1];
    return otg::make_request(s, design[r], c1 - c0, cap_net + c0, cap_node + c0, cap_val + 4 * c0,
                             s1 - s0, slew_net + s0, slew_val + 4 * s0, q);
  };
  otg_status st = OTG_OK;
  int64_t last = t0;
  if (plain) {
    for (int r = 0; r < num_req && st == OTG_OK; ++r) {
      const int c0 = cap_start[r], s0 = slew_start[r];
      until(t0 + arrival_ns[r]);
      otg_result o{};
      st = otg_server_update_sync(s, design[r], cap_start[r + 1] - c0, cap_net + c0,
                                  cap_node + c0, cap_val + 4 * c0, slew_start[r + 1] - s0,
                                  slew_net + s0, slew_val + 4 * s0, &o);
      if (st == OTG_OK && o.status != OTG_OK) st = (otg_status)o.status;
      latency_ns[r] = o.t_done_ns - (t0 + arrival_ns[r]);
      last = std::max(last, o.t_done_ns);
    }
    *makespan_ns = last - t0;
    return st;
  }
  std::vector<int64_t> tickets(num_req, 0);
  std::atomic<int> submitted{0};
  std::atomic<int> sub_err{OTG_OK};
  std::thread submitter([&] {
    for (int r = 0; r < num_req; ++r) {
      until(t0 + arrival_ns[r]);
      otg::Request q;
      otg_status e;
      {
        std::lock_guard<std::mutex> lk(s->mu);
        e = args(r, &q);
        if (e == OTG_OK) {
          q.t_submit = t0 + arrival_ns[r];
          q.ticket = s->next_ticket++;
          otg_result pend{};
          pend.status = -1;
          pend.t_submit_ns = q.t_submit;
          s->done[q.ticket] = pend;
          tickets[r] = q.ticket;
          s->pending.push_back(std::move(q));
        }
      }
      if (e != OTG_OK) {
        sub_err = e;
        submitted.store(num_req + 1);
        s->cv_done.notify_all();
        return;
      }
      s->cv_disp.notify_one();
      submitted.store(r + 1);
      s->cv_done.notify_all();
    }
  });
  for (int r = 0; r < num_req; ++r) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_done.wait(lk, [&] { return submitted.load() > r; });
    }
    if (submitted.load() > num_req) break;
    otg_result o{};
    otg_status e = otg_server_wait(s, tickets[r], -1, &o);
    if (e == OTG_OK && o.status != OTG_OK) e = (otg_status)o.status;
    if (e != OTG_OK && st == OTG_OK) st = e;
    latency_ns[r] = o.t_done_ns - o.t_submit_ns;
    last = std::max(last, o.t_done_ns);
  }
  submitter.join();
  if (st == OTG_OK) st = (otg_status)sub_err.load();
  *makespan_ns = last - t0;
  return st;
}

otg_status otg_server_read(otg_server* s, int32_t d, int32_t* node2bfs, float* load,
                           float* delay, float* ldelay, float* impulse, float* sink_slew) {
  if (!s || d < 0 || d >= otg::kMaxDesigns) return OTG_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  otg::Design& D = s->designs[d];
  if (!D.live) return OTG_ERR_INVALID;
  s->cv_done.wait(lk, [&] { return !D.busy; });
  const size_t V = (size_t)D.total_nodes;
  bool ok = true;
  auto cp = [&](void* dst, const void* src, size_t b) {
    if (dst && ok) ok = cudaMemcpy(dst, src, b, cudaMemcpyDeviceToHost) == cudaSuccess;
  };
  cp(node2bfs, D.n2b, 4 * V);
  cp(load, D.load, 16 * V);
  cp(delay, D.delay, 16 * V);
  cp(ldelay, D.ldelay, 16 * V);
  cp(impulse, D.imp, 16 * V);
  cp(sink_slew, D.sslew, 16 * (size_t)D.num_sinks);
  if (!ok) {
    cudaGetLastError();
    return OTG_ERR_CUDA;
  }
  return OTG_OK;
}

}  // extern "C"
