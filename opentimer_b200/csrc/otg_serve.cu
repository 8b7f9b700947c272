// otg_serve.cu -- device-resident designs and the incremental timing server.
//
// The reference re-times dirty nets on the CPU (Net::_update_rc_timing skips
// clean nets, ot/timer/net.cpp:536-540) and its GPU path re-flattens every
// net per update (timer.cpp:929-970).  Here a design's RC state stays on the
// device, and a request (node-cap and driver-slew updates, i.e. gate
// resizes) re-times only its dirty nets.
//
// Batching: a dispatcher thread takes pending requests in arrival order
// into one of `slots` batch slots.  A design is in at most one batch in
// flight, and a batch takes several requests of a design only while their
// net sets are disjoint (the first one that overlaps ends that design's
// share of the batch), so every request sees exactly the state its
// predecessors left: its result is the same alone or in a mix.  A slot replays a CUDA graph captured once:
//   clear counters -> apply_kernel (writes the updates, marks dirty nets,
//   lists distinct (design, net) items) -> the fused RC pass over the items
//   of all designs (rc_launch_items, size classes on parallel branches) ->
//   result_kernel (per-request worst |sink slew| and sink delay over its
//   dirty nets, published by the last CTA).
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
#include <list>
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
                // (sticky: topology is validated when the design is added,
                // so a later pass has nothing left to report)
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

// Writes the updates, marks dirty nets and lists each distinct (design,
// net) once.  upd[u] keeps (request, net) of update u for result_kernel
// (net -1 when the update was refused), so the batch in mapped host memory
// is read only once.
__global__ void apply_kernel(BatchView b, const DesignDev* dz, int2* items, int* num_items,
                             int cap_items, ResultDev* res, int2* upd) {
  const BatchHdr h = *b.hdr;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  for (int u = tid; u < h.num_cap + h.num_slew; u += stride) {
    const bool is_cap = u < h.num_cap;
    const int k = is_cap ? u : u - h.num_cap;
    const int r = is_cap ? b.cap_req[k] : b.slew_req[k];
    const int net = is_cap ? b.cap_net[k] : b.slew_net[k];
    const int node = is_cap ? b.cap_node[k] : 0;
    const float4 val = is_cap ? b.cap_val[k] : b.slew_val[k];
    const int d = b.req_design[r];
    const DesignDev D = dz[d];
    upd[u] = make_int2(r, -1);
    if ((unsigned)net >= (unsigned)D.num_nets) {
      atomicCAS(&res[r].status, 0, (int)OTG_ERR_INVALID);
      continue;
    }
    if (is_cap) {
      const int base = D.nodes_start[net], n = D.nodes_start[net + 1] - base;
      if ((unsigned)node >= (unsigned)n) {
        atomicCAS(&res[r].status, 0, (int)OTG_ERR_INVALID);
        continue;
      }
      D.cap[base + node] = val;
    } else {
      D.driver_slew[net] = val;
    }
    upd[u] = make_int2(r, net);
    if (atomicExch(&D.marks[net], h.stamp) != h.stamp) {
      const int pos = atomicAdd(num_items, 1);
      if (pos < cap_items) items[pos] = make_int2(d, net);
      else atomicCAS(&res[r].status, 0, (int)OTG_ERR_WORKSPACE);
      atomicAdd(&res[r].dirty, 1);
    }
  }
}

__device__ __forceinline__ unsigned fbits(float v) { return __float_as_uint(fabsf(v)); }

// Per-request worst |sink slew| and sink delay over the nets its updates
// touched, then (last CTA to finish) the results into mapped host memory.
// One warp per update: the lanes stride over the net's sinks and reduce.
// A warp keeps a running maximum while consecutive updates belong to the
// same request and flushes it with atomics when the request changes.
// Maxima are taken on the bit patterns of non-negative floats, whose
// order is the float order.
__global__ void result_kernel(BatchView b, const DesignDev* dz, ResultDev* res, const int2* upd,
                              int* blocks_done, otg_result* out) {
  const BatchHdr h = *b.hdr;
  const int nu = h.num_cap + h.num_slew;
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  int cur = -1;
  unsigned m[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  auto flush = [&]() {
    if (cur >= 0 && lane == 0) {
      for (int c = 0; c < 4; ++c) {
        if (m[c]) atomicMax(&res[cur].slew[c], m[c]);
        if (m[4 + c]) atomicMax(&res[cur].delay[c], m[4 + c]);
      }
    }
    for (int c = 0; c < 8; ++c) m[c] = 0;
  };
  for (int u = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); u < nu; u += warps) {
    const int2 x = upd[u];
    if (x.x != cur) {
      flush();
      cur = x.x;
    }
    const int net = x.y;
    if (net < 0) continue;
    const DesignDev D = dz[b.req_design[cur]];
    if (!D.sinks_start) continue;
    const int nb = D.nodes_start[net];
    const int s1 = D.sinks_start[net + 1];
    for (int s = D.sinks_start[net] + lane; s < s1; s += 32) {
      const float4 sl = D.sink_slew[s];
      const float4 dl = D.delay[nb + D.node2bfs[nb + D.sink_nodes[s]]];
      m[0] = max(m[0], fbits(sl.x));
      m[1] = max(m[1], fbits(sl.y));
      m[2] = max(m[2], fbits(sl.z));
      m[3] = max(m[3], fbits(sl.w));
      m[4] = max(m[4], fbits(dl.x));
      m[5] = max(m[5], fbits(dl.y));
      m[6] = max(m[6], fbits(dl.z));
      m[7] = max(m[7], fbits(dl.w));
    }
    for (int c = 0; c < 8; ++c) m[c] = __reduce_max_sync(0xffffffffu, m[c]);
  }
  flush();
  // last CTA out publishes
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(blocks_done, 1) == (int)gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int r = threadIdx.x; r < h.num_req; r += blockDim.x) {
    const volatile ResultDev* x = res + r;
    otg_result o;
    for (int c = 0; c < 4; ++c) {
      o.worst_slew[c] = __uint_as_float(x->slew[c]);
      o.worst_delay[c] = __uint_as_float(x->delay[c]);
    }
    const int ds = dz[b.req_design[r]].status[0];
    o.status = x->status ? x->status : ds;
    o.dirty_nets = x->dirty;
    o.t_submit_ns = 0;
    o.t_done_ns = 0;
    out[r] = o;
  }
}

struct Request {
  int64_t ticket = 0;
  int design = 0;
  std::vector<int> cap_net, cap_node, slew_net;
  std::vector<float4> cap_val, slew_val;
  std::vector<int> nets;  // distinct nets the request touches, ascending
  int64_t t_submit = 0;
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
  bool busy = false;   // held by add (reservation), update_sync, read or remove
  int inflight = 0;    // batches in flight that touch the design
  std::vector<int> nodes_start;   // host copy, to validate requests
  std::vector<int> net_inflight;  // per net: in-flight requests touching it
  std::vector<int> net_taken;     // per net: last batch formation that took it
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
  int2* upd = nullptr;
  int* num_items = nullptr;  // [0] items, [1] result CTAs done
  RcFork fork;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  int ws_max_n = 0;
  bool busy = false;
  std::vector<Request> reqs;  // the batch in flight
};

// Builds a request from the caller's arrays (no server state touched).  A
// node (net) updated twice in one request keeps its last value: only the
// last occurrence is kept, so the parallel apply is deterministic.
otg_status build_request(int max_updates, int32_t d, int32_t num_cap, const int32_t* cap_net,
                         const int32_t* cap_node, const float* cap_val, int32_t num_slew,
                         const int32_t* slew_net, const float* slew_val, Request* q) {
  if (d < 0 || d >= kMaxDesigns || num_cap < 0 || num_slew < 0 ||
      (int64_t)num_cap + num_slew > max_updates || (num_cap && (!cap_net || !cap_node || !cap_val)) ||
      (num_slew && (!slew_net || !slew_val)))
    return OTG_ERR_INVALID;
  q->design = d;
  auto last_of_each = [](int n, auto key) {
    std::vector<std::pair<uint64_t, int>> k(n);
    for (int i = 0; i < n; ++i) k[i] = {key(i), -i};
    std::sort(k.begin(), k.end());
    std::vector<int> keep;
    keep.reserve(n);
    for (int i = 0; i < n; ++i)
      if (i == 0 || k[i].first != k[i - 1].first) keep.push_back(-k[i].second);
    std::sort(keep.begin(), keep.end());
    return keep;
  };
  const std::vector<int> kc = last_of_each(num_cap, [&](int i) {
    return ((uint64_t)(uint32_t)cap_net[i] << 32) | (uint32_t)cap_node[i];
  });
  const std::vector<int> ks = last_of_each(num_slew, [&](int i) { return (uint64_t)(uint32_t)slew_net[i]; });
  q->cap_net.resize(kc.size());
  q->cap_node.resize(kc.size());
  q->cap_val.resize(kc.size());
  for (size_t j = 0; j < kc.size(); ++j) {
    const int k = kc[j];
    q->cap_net[j] = cap_net[k];
    q->cap_node[j] = cap_node[k];
    q->cap_val[j] = make_float4(cap_val[4 * k], cap_val[4 * k + 1], cap_val[4 * k + 2], cap_val[4 * k + 3]);
  }
  q->slew_net.resize(ks.size());
  q->slew_val.resize(ks.size());
  for (size_t j = 0; j < ks.size(); ++j) {
    const int k = ks[j];
    q->slew_net[j] = slew_net[k];
    q->slew_val[j] = make_float4(slew_val[4 * k], slew_val[4 * k + 1], slew_val[4 * k + 2], slew_val[4 * k + 3]);
  }
  q->nets = q->cap_net;
  q->nets.insert(q->nets.end(), q->slew_net.begin(), q->slew_net.end());
  std::sort(q->nets.begin(), q->nets.end());
  q->nets.erase(std::unique(q->nets.begin(), q->nets.end()), q->nets.end());
  q->t_submit = now_ns();
  return OTG_OK;
}

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
  std::list<Request> pending;  // arrival order; taken entries erased in O(1)
  std::unordered_map<int64_t, otg_result> done;
  int64_t next_ticket = 1;
  bool stop = false;
  std::thread disp;
  int device = 0;
  int dev_sms = 148;
  int64_t n_batches = 0, n_batched = 0;
  int form = 0;  // batch-formation counter (net_taken stamps)
  // bumped (under mu) whenever a waiting request may have become
  // dispatchable: a new request, or a design released by a caller
  std::atomic<uint64_t> kick_gen{0};
  std::atomic<bool> stopping{false};
  void kick_locked() { kick_gen.fetch_add(1); }

  ~Server();
  otg_status init_slot(Slot& s);
  otg_status ensure_ws(Slot& s, int need_n);
  otg_status launch_batch(Slot& s, bool graph);
  otg_status capture(Slot& s, int need_n);
  void fill(Slot& s, int stamp_value);
  void dispatcher();
  void form_batches(std::unique_lock<std::mutex>& lk);
  void release(Slot& s, const otg_result* res, int status);
  void release_slot(Slot& s, int status);
  bool idle(int d) const { return !designs[d].busy && designs[d].inflight == 0; }
  // a live design, and every net and node of the request inside it
  bool valid(const Request& q) const {
    const Design& D = designs[q.design];
    if (!D.live) return false;
    for (int net : q.nets)
      if ((unsigned)net >= (unsigned)D.num_nets) return false;
    for (size_t k = 0; k < q.cap_net.size(); ++k) {
      const int net = q.cap_net[k];
      if ((unsigned)q.cap_node[k] >= (unsigned)(D.nodes_start[net + 1] - D.nodes_start[net]))
        return false;
    }
    return true;
  }
  otg_status enqueue(Request&& q, int64_t* ticket);
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
  SCK(cudaMalloc(&s.upd, sizeof(int2) * (size_t)U));
  SCK(cudaMalloc(&s.num_items, 64));
  SCK(rc_fork_create(&s.fork, 3));
  return OTG_OK;
}

otg_status Server::ensure_ws(Slot& s, int need_n) {
  if (s.ws && s.ws_max_n >= need_n) return OTG_OK;
  size_t need = 0;
  otg_status st = otg_rc_workspace_size(U, need_n, &need);
  if (st != OTG_OK) return st;
  if (s.ws) cudaFree(s.ws);
  s.ws = nullptr;
  SCK(cudaMalloc(&s.ws, need));
  s.ws_bytes = need;
  s.ws_max_n = need_n;
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
  // result_kernel: a warp per update, up to 8 resident CTAs per SM
  const int rblocks = std::max(1, std::min(dev_sms * 8, (U + 7) / 8));
  apply_kernel<<<blocks, 256, 0, s.st>>>(s.dv, dz_dev, s.items, s.num_items, U, s.dres, s.upd);
  count_launch();
  otg_status st = rc_launch_items((const RcArgsOpaque*)forests_dev, s.items, s.num_items, U,
                                  s.ws_max_n, s.ws, s.ws_bytes, s.st, &s.fork);
  if (st != OTG_OK) return st;
  result_kernel<<<rblocks, 256, 0, s.st>>>(s.dv, dz_dev, s.dres, s.upd, s.num_items + 1,
                                           s.dres_out);
  count_launch();
  SCK(cudaGetLastError());
  return OTG_OK;
}

otg_status Server::capture(Slot& s, int need_n) {
  otg_status st = ensure_ws(s, need_n);
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
  return OTG_OK;
}

// Writes the slot's requests into its mapped batch buffer.
void Server::fill(Slot& s, int stamp_value) {
  BatchView& v = s.hv;
  int nc = 0, nsl = 0;
  for (size_t r = 0; r < s.reqs.size(); ++r) {
    const Request& q = s.reqs[r];
    v.req_design[r] = q.design;
    const size_t kc = q.cap_net.size(), ks = q.slew_net.size();
    for (size_t k = 0; k < kc; ++k) v.cap_req[nc + k] = (int)r;
    std::memcpy(v.cap_net + nc, q.cap_net.data(), 4 * kc);
    std::memcpy(v.cap_node + nc, q.cap_node.data(), 4 * kc);
    std::memcpy(v.cap_val + nc, q.cap_val.data(), 16 * kc);
    for (size_t k = 0; k < ks; ++k) v.slew_req[nsl + k] = (int)r;
    std::memcpy(v.slew_net + nsl, q.slew_net.data(), 4 * ks);
    std::memcpy(v.slew_val + nsl, q.slew_val.data(), 16 * ks);
    nc += (int)kc;
    nsl += (int)ks;
  }
  v.hdr->num_req = (int)s.reqs.size();
  v.hdr->num_cap = nc;
  v.hdr->num_slew = nsl;
  v.hdr->stamp = stamp_value;
}

// Completes a slot's batch: results to the waiters, in-flight nets freed.
void Server::release(Slot& s, const otg_result* res, int status) {
  const int64_t t = now_ns();
  for (size_t r = 0; r < s.reqs.size(); ++r) {
    const Request& q = s.reqs[r];
    auto it = done.find(q.ticket);
    if (it != done.end()) {
      otg_result o = res ? res[r] : otg_result{};
      if (!res) o.status = status;
      o.t_submit_ns = it->second.t_submit_ns;
      o.t_done_ns = t;
      it->second = o;
    }
    Design& D = designs[q.design];
    for (int net : q.nets) D.net_inflight[net]--;
  }
  std::vector<int> ds;
  for (const Request& q : s.reqs) ds.push_back(q.design);
  std::sort(ds.begin(), ds.end());
  ds.erase(std::unique(ds.begin(), ds.end()), ds.end());
  for (int d : ds) designs[d].inflight--;
  s.reqs.clear();
  s.busy = false;
  cv_done.notify_all();
}

void Server::release_slot(Slot& s, int status) { release(s, nullptr, status); }

void Server::dispatcher() {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> lk(mu);
  lk.unlock();
  uint64_t seen = ~(uint64_t)0;
  std::vector<Slot*> finished;
  while (true) {
    // completions: the slots belong to this thread, so polling needs no lock
    finished.clear();
    bool any_busy = false, any_free = false;
    for (auto& s : slots) {
      if (!s.busy) any_free = true;
      else if (cudaEventQuery(s.ev) == cudaSuccess) finished.push_back(&s);
      else any_busy = true;
    }
    const bool stop_now = stopping.load();
    if (!finished.empty() || stop_now || (any_free && kick_gen.load() != seen)) {
      lk.lock();
      for (Slot* f : finished) release(*f, f->hres, 0);
      if (stop && !any_busy) break;
      seen = kick_gen.load();
      form_batches(lk);
      lk.unlock();
    }
    bool busy_now = false;
    for (auto& s : slots) busy_now |= s.busy;
    if (busy_now) {
      // poll the slots' events (a sleep would add the scheduler's timer
      // slack, tens of microseconds, to every batch)
      std::this_thread::yield();
    } else {
      lk.lock();
      cv_disp.wait(lk, [&] { return stop || kick_gen.load() != seen; });
      lk.unlock();
    }
  }
}

// Forms and launches batches for the free slots (called with lk held; lk
// is released around the fill and launch of each batch).  Requests are
// taken in arrival order.  A request joins when its design is not held,
// its nets are disjoint from the nets of the design's requests in flight
// and of the requests already in this batch, and it fits; a request that
// cannot join holds back its design's later requests.
void Server::form_batches(std::unique_lock<std::mutex>& lk) {
  for (auto& s : slots) {
    if (s.busy || pending.empty() || stop) continue;
    const int fstamp = ++form;
    std::vector<std::list<Request>::iterator> take;
    std::vector<char> blocked(designs.size(), 0);
    int nblocked = 0, nlive = 0;
    for (auto& d : designs) nlive += d.live;
    size_t nu = 0;
    for (auto it = pending.begin(); it != pending.end(); ++it) {
      if ((int)take.size() >= R || nblocked >= nlive) break;
      const Request& q = *it;
      const int d = q.design;
      if (blocked[d]) continue;
      const size_t qu = q.cap_net.size() + q.slew_net.size();
      Design& D = designs[d];
      bool ok = !D.busy && nu + qu <= (size_t)U;
      for (size_t i = 0; ok && i < q.nets.size(); ++i) {
        const int net = q.nets[i];
        ok = D.net_inflight[net] == 0 && D.net_taken[net] != fstamp;
      }
      if (!ok) {
        blocked[d] = 1;
        ++nblocked;
        continue;
      }
      for (int net : q.nets) D.net_taken[net] = fstamp;
      nu += qu;
      take.push_back(it);
    }
    if (take.empty()) break;
    for (auto it : take) {
      s.reqs.push_back(std::move(*it));
      pending.erase(it);
    }
    std::vector<int> ds;
    for (const Request& q : s.reqs) {
      Design& D = designs[q.design];
      for (int net : q.nets) D.net_inflight[net]++;
      ds.push_back(q.design);
    }
    std::sort(ds.begin(), ds.end());
    ds.erase(std::unique(ds.begin(), ds.end()), ds.end());
    for (int d : ds) designs[d].inflight++;
    s.busy = true;
    n_batches++;
    n_batched += (int64_t)s.reqs.size();
    const int st_value = ++stamp;
    otg_status st = OTG_OK;
    if (s.graph_gen != gen) {
      st = capture(s, max_n);  // rare: under the lock (reads max_n)
      if (st == OTG_OK) s.graph_gen = gen;
    }
    if (st == OTG_OK) {
      // the slot belongs to this thread until it is released
      lk.unlock();
      fill(s, st_value);
      st = launch_batch(s, true);
      if (st == OTG_OK && cudaEventRecord(s.ev, s.st) != cudaSuccess) st = OTG_ERR_CUDA;
      lk.lock();
    }
    if (st != OTG_OK) {
      cudaGetLastError();
      if (s.exec) cudaStreamSynchronize(s.st);
      release_slot(s, st);
    }
  }
}

otg_status Server::enqueue(Request&& q, int64_t* ticket) {
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!valid(q)) return OTG_ERR_INVALID;
    q.ticket = next_ticket++;
    otg_result r{};
    r.status = -1;  // pending
    r.t_submit_ns = q.t_submit;
    done[q.ticket] = r;
    *ticket = q.ticket;
    pending.push_back(std::move(q));
    kick_locked();
  }
  cv_disp.notify_one();
  return OTG_OK;
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu);
    stop = true;
    stopping = true;
  }
  cv_disp.notify_all();
  if (disp.joinable()) disp.join();
  cudaSetDevice(device);
  auto free_slot = [](Slot& s) {
    if (s.st) cudaStreamSynchronize(s.st);
    if (s.exec) cudaGraphExecDestroy(s.exec);
    if (s.ev) cudaEventDestroy(s.ev);
    if (s.st) cudaStreamDestroy(s.st);
    if (s.hbuf) cudaFreeHost(s.hbuf);
    if (s.hres) cudaFreeHost(s.hres);
    cudaFree(s.dres);
    cudaFree(s.items);
    cudaFree(s.upd);
    cudaFree(s.num_items);
    rc_fork_destroy(&s.fork);
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

struct otg_server : public otg::Server {};

extern "C" {

otg_status otg_server_create(size_t budget_bytes, int32_t slots, int32_t max_requests,
                             int32_t max_updates, otg_server** out) {
  if (!out || slots < 1 || max_requests < 1 || max_updates < 1) return OTG_ERR_INVALID;
  otg_server* s = new (std::nothrow) otg_server();
  if (!s) return OTG_ERR_OOM;
  cudaGetDevice(&s->device);
  cudaDeviceGetAttribute(&s->dev_sms, cudaDevAttrMultiProcessorCount, s->device);
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
  // the first full pass, with a temporary workspace; its status check
  // also validates the topology (every later pass re-times the same trees)
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
  D.nodes_start.assign(h->nodes_start, h->nodes_start + N + 1);
  D.net_inflight.assign(N, 0);
  D.net_taken.assign(N, 0);
  s->designs[d] = std::move(D);
  s->kick_locked();
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
    if (!s->idle(d)) return false;
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
  otg_status st = otg::build_request(s->U, d, num_cap, cap_net, cap_node, cap_val, num_slew,
                                     slew_net, slew_val, &q);
  if (st != OTG_OK) return st;
  return s->enqueue(std::move(q), ticket);
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
  if (!s || !out) return OTG_ERR_INVALID;
  otg::Request q;
  otg_status st = otg::build_request(s->U, d, num_cap, cap_net, cap_node, cap_val, num_slew,
                                     slew_net, slew_val, &q);
  if (st != OTG_OK) return st;
  std::lock_guard<std::mutex> sync_lk(s->sync_mu);
  std::unique_lock<std::mutex> lk(s->mu);
  if (!s->valid(q)) return OTG_ERR_INVALID;
  s->cv_done.wait(lk, [&] { return s->idle(d); });
  s->designs[d].busy = true;
  otg::Slot& sl = s->sync_slot;
  st = s->ensure_ws(sl, s->max_n);
  const int st_value = ++s->stamp;
  lk.unlock();
  if (st == OTG_OK) {
    sl.reqs.clear();
    sl.reqs.push_back(std::move(q));
    s->fill(sl, st_value);
    st = s->launch_batch(sl, false);
    if (st == OTG_OK && cudaStreamSynchronize(sl.st) != cudaSuccess) {
      cudaGetLastError();
      st = OTG_ERR_CUDA;
    }
  }
  const int64_t t_done = otg::now_ns();
  lk.lock();
  s->designs[d].busy = false;
  s->kick_locked();
  s->cv_done.notify_all();
  s->cv_disp.notify_one();
  if (st != OTG_OK) return st;
  *out = sl.hres[0];
  out->t_submit_ns = sl.reqs[0].t_submit;
  out->t_done_ns = t_done;
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
  // batched: a submitter thread issues the requests on schedule, this
  // thread collects them in order
  std::vector<int64_t> tickets(num_req, 0);
  std::atomic<int> submitted{0};
  std::atomic<int> sub_err{OTG_OK};
  std::mutex tmu;
  std::condition_variable tcv;
  std::thread submitter([&] {
    for (int r = 0; r < num_req; ++r) {
      until(t0 + arrival_ns[r]);
      const int c0 = cap_start[r], c1 = cap_start[r + 1], s0 = slew_start[r], s1 = slew_start[r + 1];
      otg::Request q;
      otg_status e = otg::build_request(s->U, design[r], c1 - c0, cap_net + c0, cap_node + c0,
                                        cap_val + 4 * c0, s1 - s0, slew_net + s0,
                                        slew_val + 4 * s0, &q);
      if (e == OTG_OK) {
        q.t_submit = t0 + arrival_ns[r];  // latency counts from the scheduled arrival
        e = s->enqueue(std::move(q), &tickets[r]);
      }
      {
        std::lock_guard<std::mutex> lk(tmu);
        if (e != OTG_OK) {
          sub_err = e;
          submitted.store(num_req + 1);
        } else {
          submitted.store(r + 1);
        }
      }
      tcv.notify_one();
      if (e != OTG_OK) return;
    }
  });
  for (int r = 0; r < num_req; ++r) {
    {
      std::unique_lock<std::mutex> lk(tmu);
      tcv.wait(lk, [&] { return submitted.load() > r; });
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

otg_status otg_server_stats(otg_server* s, int64_t* batches, int64_t* requests) {
  if (!s || !batches || !requests) return OTG_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  *batches = s->n_batches;
  *requests = s->n_batched;
  return OTG_OK;
}

otg_status otg_server_read(otg_server* s, int32_t d, int32_t* node2bfs, float* load,
                           float* delay, float* ldelay, float* impulse, float* sink_slew) {
  if (!s || d < 0 || d >= otg::kMaxDesigns) return OTG_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  otg::Design& D = s->designs[d];
  if (!D.live) return OTG_ERR_INVALID;
  s->cv_done.wait(lk, [&] { return s->idle(d); });
  D.busy = true;
  lk.unlock();
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
  lk.lock();
  D.busy = false;
  s->kick_locked();
  s->cv_done.notify_all();
  s->cv_disp.notify_one();
  if (!ok) {
    cudaGetLastError();
    return OTG_ERR_CUDA;
  }
  return OTG_OK;
}

}  // extern "C"
