// otg_synth.cu -- seeded synthetic RC forests for the batched-Elmore
// workload, generated on the device (so a 1M-net, 5e8-node batch is built
// in HBM in milliseconds) or on the host with bit-identical results: the
// generator uses only integer hashing and correctly rounded fmaf.
//
// Per net (node count from nodes_start):
//   * 30% chains with side branches: a spine of 80% of the nodes, the rest
//     hung on uniformly chosen spine nodes; 70% random recursive trees
//     (parent of canonical node i uniform in [0, i));
//   * the edge list is shuffled (Fisher-Yates) and each edge randomly
//     oriented, then local ids are assigned by first appearance while
//     scanning the edges -- the id rule of Net::_make_flat_rct
//     (ot/timer/net.cpp:392-410); the root is canonical node 0;
//   * R ~ U(0.1, 50) per edge, ground C ~ U(0.05, 5) per node, plus a
//     per-corner pin cap U(0.5, 2) on every leaf so the four corners differ;
//   * driver slew per corner U(5, 200).
#include <cuda_runtime.h>
#include <stdint.h>

#include <new>

#include "../../include/otg.h"
#include "otg_internal.cuh"

namespace otg {
namespace {

struct Rng {
  uint64_t s;
  __host__ __device__ uint64_t next() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  // uniform in [0, 1) with 24 random bits (exact in fp32)
  __host__ __device__ float unif() { return (float)(next() >> 40) * (1.0f / 16777216.0f); }
  __host__ __device__ float unif(float lo, float hi) { return fmaf(unif(), hi - lo, lo); }
  // uniform integer in [0, k)
  __host__ __device__ uint32_t below(uint32_t k) {
    return (uint32_t)(((next() >> 32) * (uint64_t)k) >> 32);
  }
};

constexpr int kLeafBit = 1 << 30;

__host__ __device__ void synth_net(uint64_t seed, int net, const int* nodes_start, int2* edges,
                                   int* roots, float* res, float4* cap, float4* slew,
                                   int* sink_count, int* scratch) {
  const int b = nodes_start[net];
  const int n = nodes_start[net + 1] - b;
  const int m = n - 1;
  const int eb = b - net;
  int2* E = edges + eb;
  int* S = scratch + b;
  Rng g{seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(net + 1))};
  const bool chain = g.unif() < 0.3f;
  const int spine = (n * 4) / 5 > 0 ? (n * 4) / 5 : 1;
  for (int v = 0; v < n; ++v) S[v] = 0;
  for (int i = 1; i < n; ++i) {
    int p;
    if (chain) p = (i < spine) ? i - 1 : (int)g.below((uint32_t)spine);
    else p = (int)g.below((uint32_t)i);
    E[i - 1] = make_int2(p, i);
    S[p] += 1;
  }
  int leaves = 0;
  for (int v = 0; v < n; ++v) {
    const bool leaf = v != 0 && S[v] == 0;
    S[v] = leaf ? kLeafBit : 0;
    leaves += leaf;
  }
  // shuffle + random orientation
  for (int i = m - 1; i > 0; --i) {
    const int j = (int)g.below((uint32_t)(i + 1));
    const int2 t = E[i];
    E[i] = E[j];
    E[j] = t;
  }
  for (int i = 0; i < m; ++i)
    if (g.next() & 1ull) E[i] = make_int2(E[i].y, E[i].x);
  // local ids by first appearance
  int cnt = 0;
  for (int i = 0; i < m; ++i) {
    int x = E[i].x, y = E[i].y;
    if ((S[x] & (kLeafBit - 1)) == 0) S[x] |= ++cnt;
    if ((S[y] & (kLeafBit - 1)) == 0) S[y] |= ++cnt;
    E[i] = make_int2((S[x] & (kLeafBit - 1)) - 1, (S[y] & (kLeafBit - 1)) - 1);
  }
  if (n == 1) S[0] |= ++cnt;
  roots[net] = (S[0] & (kLeafBit - 1)) - 1;
  for (int i = 0; i < m; ++i) res[eb + i] = g.unif(0.1f, 50.0f);
  for (int v = 0; v < n; ++v) {
    const int l = (S[v] & (kLeafBit - 1)) - 1;
    const float c = g.unif(0.05f, 5.0f);
    float4 o = make_float4(c, c, c, c);
    if (S[v] & kLeafBit) {
      o.x += g.unif(0.5f, 2.0f);
      o.y += g.unif(0.5f, 2.0f);
      o.z += g.unif(0.5f, 2.0f);
      o.w += g.unif(0.5f, 2.0f);
    }
    cap[b + l] = o;
  }
  // one draw per statement: argument evaluation order differs between the
  // host and device compilers
  float4 sl;
  sl.x = g.unif(5.0f, 200.0f);
  sl.y = g.unif(5.0f, 200.0f);
  sl.z = g.unif(5.0f, 200.0f);
  sl.w = g.unif(5.0f, 200.0f);
  slew[net] = sl;
  sink_count[net] = leaves;
}

// Degree-1 non-root nodes of each net in ascending local id.
__host__ __device__ void synth_sinks(int net, const int* nodes_start, const int2* edges,
                                     const int* roots, const int* sinks_start, int* sink_nodes,
                                     int* scratch) {
  const int b = nodes_start[net];
  const int n = nodes_start[net + 1] - b;
  const int eb = b - net;
  int* S = scratch + b;
  for (int v = 0; v < n; ++v) S[v] = 0;
  for (int i = 0; i < n - 1; ++i) {
    S[edges[eb + i].x] += 1;
    S[edges[eb + i].y] += 1;
  }
  int k = sinks_start[net];
  for (int v = 0; v < n; ++v)
    if (S[v] == 1 && v != roots[net]) sink_nodes[k++] = v;
}

__global__ void synth_kernel(uint64_t seed, int num_nets, const int* nodes_start, int2* edges,
                             int* roots, float* res, float4* cap, float4* slew, int* sink_count,
                             int* scratch) {
  for (int net = blockIdx.x * blockDim.x + threadIdx.x; net < num_nets;
       net += gridDim.x * blockDim.x)
    synth_net(seed, net, nodes_start, edges, roots, res, cap, slew, sink_count, scratch);
}

__global__ void synth_sinks_kernel(int num_nets, const int* nodes_start, const int2* edges,
                                   const int* roots, const int* sinks_start, int* sink_nodes,
                                   int* scratch) {
  for (int net = blockIdx.x * blockDim.x + threadIdx.x; net < num_nets;
       net += gridDim.x * blockDim.x)
    synth_sinks(net, nodes_start, edges, roots, sinks_start, sink_nodes, scratch);
}

}  // namespace
}  // namespace otg

extern "C" {

otg_status otg_synth_rc_forest(uint64_t seed, int32_t num_nets, const int32_t* nodes_start,
                               otg_rc_edge* edges, int32_t* roots, float* res, float* cap,
                               float* driver_slew, int32_t* sink_count, int32_t* scratch,
                               otg_stream_t stream) {
  if (num_nets < 0 || !nodes_start || !edges || !roots || !res || !cap || !driver_slew ||
      !sink_count || !scratch)
    return OTG_ERR_INVALID;
  if (num_nets == 0) return OTG_OK;
  // one thread per net; small blocks spread the long nets over the SMs
  otg::synth_kernel<<<(num_nets + 63) / 64, 64, 0, (cudaStream_t)stream>>>(
      seed, num_nets, nodes_start, (int2*)edges, roots, res, (float4*)cap, (float4*)driver_slew,
      sink_count, scratch);
  otg::count_launch();
  return cudaGetLastError() == cudaSuccess ? OTG_OK : OTG_ERR_CUDA;
}

otg_status otg_synth_rc_sinks(int32_t num_nets, const int32_t* nodes_start,
                              const otg_rc_edge* edges, const int32_t* roots,
                              const int32_t* sinks_start, int32_t* sink_nodes, int32_t* scratch,
                              otg_stream_t stream) {
  if (num_nets < 0 || !nodes_start || !edges || !roots || !sinks_start || !sink_nodes || !scratch)
    return OTG_ERR_INVALID;
  if (num_nets == 0) return OTG_OK;
  otg::synth_sinks_kernel<<<(num_nets + 63) / 64, 64, 0, (cudaStream_t)stream>>>(
      num_nets, nodes_start, (const int2*)edges, roots, sinks_start, sink_nodes, scratch);
  otg::count_launch();
  return cudaGetLastError() == cudaSuccess ? OTG_OK : OTG_ERR_CUDA;
}

otg_status otg_synth_rc_forest_host(uint64_t seed, int32_t num_nets, const int32_t* nodes_start,
                                    otg_rc_edge* edges, int32_t* roots, float* res, float* cap,
                                    float* driver_slew, int32_t* sink_count) {
  if (num_nets < 0 || !nodes_start || !edges || !roots || !res || !cap || !driver_slew ||
      !sink_count)
    return OTG_ERR_INVALID;
  if (num_nets == 0) return OTG_OK;
  const int V = nodes_start[num_nets];
  int* scratch = new (std::nothrow) int[V > 0 ? V : 1];
  if (!scratch) return OTG_ERR_OOM;
  for (int net = 0; net < num_nets; ++net)
    otg::synth_net(seed, net, nodes_start, (int2*)edges, roots, res, (float4*)cap,
                   (float4*)driver_slew, sink_count, scratch);
  delete[] scratch;
  return OTG_OK;
}

}  // extern "C"
