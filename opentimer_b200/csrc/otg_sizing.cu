// otg_sizing.cu -- the device side of an incremental gate resize.
//
// Timer::repower_gate (ot/timer/timer.cpp:57-118) swaps a gate's cell for
// another drive strength of the same function: every pin of the gate is
// remapped to the new cell's pin (Pin::_remap_cellpin, ot/timer/pin.cpp:
// 382-399), which changes the capacitance an input pin adds to its net's RC
// tree and marks that net for RC re-timing, and the gate's timing arcs are
// rebuilt on the new cell's timing groups.  The next update_timing re-times
// the marked nets and propagates over the affected cone
// (ot/timer/timer.cpp:888-923, 1245-1334).
//
// Here a design's RC forest and timing graph stay on the device; a resize
// batch arrives as a list of node-cap updates (the input pins' RC nodes,
// new ground + pin capacitance) and a list of arc-timing updates (a cell
// arc and split, the new cell's timing record).  otg_apply_updates writes
// both in one launch; the caller then re-times the dirty nets
// (otg_rc_timing_subset) and propagates (otg_propagate).
// otg_worst_slack reduces the propagated slack to its per-corner minimum.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/otg.h"
#include "otg_internal.cuh"

namespace otg {
namespace {

__global__ void apply_updates_kernel(int num_cap, const int32_t* __restrict__ cap_row,
                                     const float4* __restrict__ cap_val, float4* nodes_cap,
                                     int num_rows, int num_arc,
                                     const int32_t* __restrict__ arc_slot,
                                     const int32_t* __restrict__ arc_rec, int32_t* arc_timing,
                                     int num_slots, int* status) {
  const int stride = gridDim.x * blockDim.x;
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < num_cap + num_arc; u += stride) {
    if (u < num_cap) {
      const int r = cap_row[u];
      if ((unsigned)r < (unsigned)num_rows) nodes_cap[r] = cap_val[u];
      else atomicCAS(status, 0, (int)OTG_ERR_INVALID);
    } else {
      const int k = u - num_cap;
      const int s = arc_slot[k];
      if ((unsigned)s < (unsigned)num_slots) arc_timing[s] = arc_rec[k];
      else atomicCAS(status, 0, (int)OTG_ERR_INVALID);
    }
  }
}

// Minimum of the finite values per corner over [P][4]; one CTA-wide
// reduction per block, then float-ordered atomics on the result (slack
// can be negative: the bits are mapped to an order-preserving unsigned).
__device__ __forceinline__ unsigned f2ord(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

__global__ void worst_slack_kernel(const float4* __restrict__ slack, int P, unsigned* out) {
  unsigned m[4] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    const float4 s = slack[p];
    const float v[4] = {s.x, s.y, s.z, s.w};
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (isfinite(v[c])) m[c] = min(m[c], f2ord(v[c]));
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const unsigned w = __reduce_min_sync(0xFFFFFFFFu, m[c]);
    if ((threadIdx.x & 31) == 0 && w != 0xFFFFFFFFu) atomicMin(&out[c], w);
  }
}

__global__ void worst_slack_init(unsigned* out, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = 0xFFFFFFFFu;
}

__global__ void worst_slack_finish(const unsigned* in, float* out, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned u = in[i];
    out[i] = u == 0xFFFFFFFFu ? __uint_as_float(0x7FC00000u) : ord2f(u);
  }
}

// Per group: pins with an active group reduce into their group's row.
// Pins of a group are mostly contiguous, so a warp reduces runs of equal
// groups before it touches the result row.
__global__ void worst_slack_groups_kernel(const float4* __restrict__ slack, int P,
                                          const int32_t* __restrict__ pin_group,
                                          const uint8_t* __restrict__ group_active,
                                          unsigned* out) {
  for (int p0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; p0 < P;
       p0 += gridDim.x * blockDim.x) {
    const int p = p0 + (threadIdx.x & 31);
    const int g = p < P ? pin_group[p] : -1;
    const bool on = g >= 0 && group_active[g];
    unsigned m[4] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};
    if (on) {
      const float4 s = slack[p];
      const float v[4] = {s.x, s.y, s.z, s.w};
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (isfinite(v[c])) m[c] = f2ord(v[c]);
    }
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, on ? g : -1);
    if (peers == 0xFFFFFFFFu) {  // the whole warp in one group (the common case)
#pragma unroll
      for (int c = 0; c < 4; ++c) m[c] = __reduce_min_sync(0xFFFFFFFFu, m[c]);
    } else {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        unsigned x = m[c];
        for (int k = 0; k < 32; ++k) {  // min over the lanes of the same group
          const unsigned y = __shfl_sync(0xFFFFFFFFu, x, k);
          if ((peers >> k) & 1u) x = min(x, y);
        }
        m[c] = x;
      }
    }
    if (on && (__ffs(peers) - 1) == (threadIdx.x & 31))
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (m[c] != 0xFFFFFFFFu) atomicMin(&out[4 * g + c], m[c]);
  }
}

}  // namespace
}  // namespace otg

extern "C" {

otg_status otg_apply_updates(int32_t num_cap, const int32_t* cap_row, const float* cap_val,
                             float* nodes_cap, int32_t total_nodes, int32_t num_arc,
                             const int32_t* arc_slot, const int32_t* arc_rec,
                             int32_t* arc_timing, int32_t num_arcs, int32_t* status,
                             otg_stream_t stream) {
  if (num_cap < 0 || num_arc < 0 || total_nodes < 0 || num_arcs < 0 || !status)
    return OTG_ERR_INVALID;
  if ((num_cap && (!cap_row || !cap_val || !nodes_cap)) ||
      (num_arc && (!arc_slot || !arc_rec || !arc_timing)))
    return OTG_ERR_INVALID;
  if (((uintptr_t)cap_val | (uintptr_t)nodes_cap) & 15) return OTG_ERR_INVALID;
  const int n = num_cap + num_arc;
  if (n == 0) return OTG_OK;
  const int blocks = (n + 255) / 256 < 592 ? (n + 255) / 256 : 592;
  otg::apply_updates_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(
      num_cap, cap_row, (const float4*)cap_val, (float4*)nodes_cap, total_nodes, num_arc,
      arc_slot, arc_rec, arc_timing, 2 * num_arcs, status);
  otg::count_launch();
  return cudaGetLastError() == cudaSuccess ? OTG_OK : OTG_ERR_CUDA;
}

otg_status otg_worst_slack(const float* slack, int32_t num_pins, uint32_t* scratch4,
                           float* out4, otg_stream_t stream) {
  if (!slack || num_pins < 0 || !scratch4 || !out4) return OTG_ERR_INVALID;
  if ((uintptr_t)slack & 15) return OTG_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  otg::worst_slack_init<<<1, 32, 0, st>>>(scratch4, 4);
  otg::count_launch();
  if (num_pins > 0) {
    const int blocks = (num_pins + 255) / 256 < 296 ? (num_pins + 255) / 256 : 296;
    otg::worst_slack_kernel<<<blocks, 256, 0, st>>>((const float4*)slack, num_pins, scratch4);
    otg::count_launch();
  }
  otg::worst_slack_finish<<<1, 32, 0, st>>>(scratch4, out4, 4);
  otg::count_launch();
  return cudaGetLastError() == cudaSuccess ? OTG_OK : OTG_ERR_CUDA;
}

otg_status otg_worst_slack_groups(const float* slack, int32_t num_pins, const int32_t* pin_group,
                                  const uint8_t* group_active, int32_t num_groups,
                                  uint32_t* scratch, float* out, otg_stream_t stream) {
  if (!slack || num_pins < 0 || num_groups < 0 || !pin_group || !group_active || !scratch ||
      !out)
    return OTG_ERR_INVALID;
  if ((uintptr_t)slack & 15) return OTG_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  const int n = 4 * num_groups;
  const int gb = (n + 255) / 256 < 64 ? (n + 255) / 256 : 64;
  otg::worst_slack_init<<<gb > 0 ? gb : 1, 256, 0, st>>>(scratch, n);
  otg::count_launch();
  if (num_pins > 0) {
    const int blocks = (num_pins + 255) / 256 < 592 ? (num_pins + 255) / 256 : 592;
    otg::worst_slack_groups_kernel<<<blocks, 256, 0, st>>>((const float4*)slack, num_pins,
                                                           pin_group, group_active, scratch);
    otg::count_launch();
  }
  otg::worst_slack_finish<<<gb > 0 ? gb : 1, 256, 0, st>>>(scratch, out, n);
  otg::count_launch();
  return cudaGetLastError() == cudaSuccess ? OTG_OK : OTG_ERR_CUDA;
}

}  // extern "C"
