// otg_move.cu -- moving whole nets between two RC forest layouts on the
// device: the relayout step of incremental SPEF ingestion.
//
// The reference re-attaches the parasitics of every net named in a change
// SPEF (Timer::_read_spef, ot/timer/spef.cpp:40-53; Net::_attach,
// net.cpp:310-341), marks it dirty, and its next update_timing re-flattens
// and re-times (on its CUDA path: every net, net.cpp:239-276).  Here the
// forest stays on the device: a new layout is allocated with the changed
// nets' new sizes, the unchanged nets are moved into it with their inputs
// AND their results (a net's values depend on that net alone, so they
// stay valid), the changed nets' inputs are moved in from a staging
// forest, and only those nets are re-timed (otg_rc_timing_subset).
//
// A net's ids, BFS slots and pids are net-relative, so a move is a plain
// copy of its node range [nodes_start[j], nodes_start[j+1]) and of its
// edge range (the same range shifted down by the net index).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/otg.h"
#include "otg_internal.cuh"

namespace otg {
namespace {

struct MoveSide {
  const int* nodes_start;
  int num_nets;
  otg_rc_edge* edges;
  int* roots;
  float* res;
  float4* cap;
  int* node2bfs;
  int* pid;
  float4* load;
  float4* delay;
  float4* ldelay;
  float4* impulse;
};

// A warp per destination net; lanes stride over the net's nodes and edges.
__global__ void move_nets_kernel(MoveSide s, MoveSide d, const int* src_net, int copy_outputs,
                                 int* status) {
  const int lane = threadIdx.x & 31;
  const int W = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < d.num_nets; i += W) {
    const int j = src_net[i];
    if (j < 0) continue;
    if (j >= s.num_nets) {
      if (lane == 0) atomicCAS(status, 0, (int)OTG_ERR_INVALID);
      continue;
    }
    const int sb = s.nodes_start[j], n = s.nodes_start[j + 1] - sb;
    const int db = d.nodes_start[i];
    if (d.nodes_start[i + 1] - db != n || n < 1) {
      if (lane == 0) atomicCAS(status, 0, (int)OTG_ERR_INVALID);
      continue;
    }
    if (lane == 0) d.roots[i] = s.roots[j];
    const int se = sb - j, de = db - i;  // edge ranges: one edge fewer than nodes per net
    for (int k = lane; k < n - 1; k += 32) {
      d.edges[de + k] = s.edges[se + k];
      d.res[de + k] = s.res[se + k];
    }
    for (int k = lane; k < n; k += 32) d.cap[db + k] = s.cap[sb + k];
    if (!copy_outputs) continue;
    for (int k = lane; k < n; k += 32) {
      d.node2bfs[db + k] = s.node2bfs[sb + k];
      d.pid[db + k] = s.pid[sb + k];
      d.load[db + k] = s.load[sb + k];
      d.delay[db + k] = s.delay[sb + k];
      d.ldelay[db + k] = s.ldelay[sb + k];
      d.impulse[db + k] = s.impulse[sb + k];
    }
  }
}

// The forest struct declares the pass's inputs const (the pass only reads
// them); the destination of a move is written, so they are cast here.
MoveSide side(const otg_rc_forest* f) {
  return MoveSide{f->nodes_start,
                  f->num_nets,
                  f->edges,
                  const_cast<int*>(f->roots),
                  const_cast<float*>(f->edges_res),
                  (float4*)const_cast<float*>(f->nodes_cap),
                  f->node2bfs,
                  f->pid,
                  (float4*)f->load,
                  (float4*)f->delay,
                  (float4*)f->ldelay,
                  (float4*)f->impulse};
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

}  // namespace
}  // namespace otg

extern "C" otg_status otg_rc_move_nets(const otg_rc_forest* src, const otg_rc_forest* dst,
                                       const int32_t* src_net, int32_t copy_outputs,
                                       int32_t* status, otg_stream_t stream) {
  if (!src || !dst || !src_net || !status || src->num_nets < 0 || dst->num_nets < 0)
    return OTG_ERR_INVALID;
  if (dst->num_nets == 0) return OTG_OK;
  for (const otg_rc_forest* f : {src, dst})
    if (!f->nodes_start || !f->edges || !f->roots || !f->edges_res || !f->nodes_cap ||
        !otg::aligned16(f->nodes_cap))
      return OTG_ERR_INVALID;
  if (copy_outputs)
    for (const otg_rc_forest* f : {src, dst})
      if (!f->node2bfs || !f->pid || !f->load || !f->delay || !f->ldelay || !f->impulse ||
          !otg::aligned16(f->load) || !otg::aligned16(f->delay) || !otg::aligned16(f->ldelay) ||
          !otg::aligned16(f->impulse))
        return OTG_ERR_INVALID;
  const int warps = std::min(dst->num_nets, 148 * 64);
  const int grid = (warps * 32 + 255) / 256;
  otg::move_nets_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(
      otg::side(src), otg::side(dst), src_net, copy_outputs ? 1 : 0, status);
  otg::count_launch();
  return cudaGetLastError() == cudaSuccess ? OTG_OK : OTG_ERR_CUDA;
}
