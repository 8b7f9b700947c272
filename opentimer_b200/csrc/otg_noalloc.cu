// otg_noalloc.cu -- the fused RC pass for callers that cannot allocate
// device memory.
//
// Some programs that call RC timing may not allocate device memory at that
// point: a host that has given all device memory to its own pool allocator
// and forbids allocations outside it, or a latency-bound loop that cannot
// afford cudaMalloc's implicit synchronization of the whole device.
// otg_rc_timing (otg_rc.cu) needs a workspace from its caller;
// otg_rc_timing_noalloc runs the same pass with a workspace that is compiled
// into this library instead: the fixed array below, 16 MiB of device memory
// that every GPU which loads it holds until the process exits.
//
// How it behaves:
//   * The CUDA runtime loads this file's device code, and with it the
//     16 MiB array, lazily: on the first call on each device, which looks
//     up the array's device address (cudaGetSymbolAddress -- the array's
//     name in host code only stands in for it).  A host whose pool takes
//     all device memory at start-up should make that first call before the
//     pool does; a call with an empty forest (num_nets == 0) does only this
//     set-up.  Make the first call before any stream capture, too.
//   * Every call reuses the same array.  The call clears the parts that must
//     start at zero (status word and work counters) before it launches, and
//     everything else is written before it is read.  Two calls that overlap
//     on the GPU (different streams, or different host threads) race on the
//     array: serialize them.
//   * The call synchronizes `stream` and returns the device-side status of
//     this call (an empty call returns OTG_OK without reading the array).
//   * It never calls cudaMalloc, cudaFree or any other allocating routine.
//   * Limit: the workspace of the batch must fit 16 MiB, i.e. at most
//     524,284 nets per call, and every net within the shared-memory classes
//     of the device's tuning (4,265 nodes on a B200 with the default
//     tuning; otg_rc_set_tuning moves the bound); anything larger returns
//     OTG_ERR_WORKSPACE before launching.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/otg.h"
#include "otg_internal.cuh"

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

void* g_scratch_addr[64];
bool g_scratch_ready[64];
std::mutex g_scratch_mu;

// Device address of g_noalloc_scratch on the current device.
otg_status scratch_address(void** out) {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) {
    cudaGetLastError();
    return OTG_ERR_CUDA;
  }
  if (d < 0 || d >= 64) return OTG_ERR_INVALID;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ready[d]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return OTG_ERR_CUDA;
    }
    g_scratch_addr[d] = p;
    g_scratch_ready[d] = true;
  }
  *out = g_scratch_addr[d];
  return OTG_OK;
}

}  // namespace

extern "C" otg_status otg_rc_timing_noalloc(const otg_rc_forest* forest, int32_t max_net_nodes,
                                            otg_stream_t stream) {
  if (!forest || forest->num_nets < 0 || max_net_nodes < 1) return OTG_ERR_INVALID;
  size_t need = 0;
  otg_status st = otg_rc_workspace_size(forest->num_nets, max_net_nodes, &need);
  if (st != OTG_OK) return st;
  if (need > kNoAllocScratchBytes) return OTG_ERR_WORKSPACE;
  void* ws = nullptr;
  st = scratch_address(&ws);
  if (st != OTG_OK) return st;
  // An empty batch launches nothing and clears nothing: the status word may
  // still hold an earlier call's error, so do not read it.
  if (forest->num_nets == 0) return OTG_OK;
  st = otg::rc_launch(forest, max_net_nodes, ws, kNoAllocScratchBytes, (cudaStream_t)stream);
  if (st != OTG_OK) return st;
  return otg_rc_status(ws, stream, nullptr);
}
