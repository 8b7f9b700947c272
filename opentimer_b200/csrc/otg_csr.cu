// otg_csr.cu -- the levelization input of a timing update built on the
// device: the fanin CSR of the propagation candidates, their fanout counts
// and the seed frontier.
//
// Replaces Timer::_build_prop_tasks_cuda steps 1-2 (ot/timer/timer.cpp:
// 996-1061), which count each candidate pin's fanin and fanout arcs in a
// taskflow parallel_for, take a serial prefix sum, fill the edge list in a
// second parallel_for and collect the candidates without fanout as the
// first frontier.  An arc counts when it is not a loop breaker and both of
// its pins are candidates.  Here:
//   count    one thread per arc: atomics on the fanin and fanout counters;
//   scan     exclusive scan of the fanin counts (block sums, a scan of the
//            block sums, block-local scans);
//   fill     one thread per arc places its index at its pin's cursor;
//   order    one thread per pin sorts its (short) fanin list by arc index,
//            so the list is in the graph's arc order, as a pin's _fanin list
//            is in its insertion order; then arc -> source pin;
//   seed     the candidates without fanout, in the caller's candidate
//            order (a flag scan and a scatter).
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/otg.h"
#include "otg_internal.cuh"

namespace otg {
namespace {

constexpr int kScanT = 512, kScanK = 8, kScanTile = kScanT * kScanK;

__global__ void csr_zero(int32_t* a, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = 0;
}

__device__ __forceinline__ bool kept(int a, const int32_t* from, const int32_t* to,
                                     const uint8_t* skip, const uint8_t* cand, int n,
                                     int* status) {
  const int f = from[a], t = to[a];
  if ((unsigned)f >= (unsigned)n || (unsigned)t >= (unsigned)n) {
    atomicCAS(status, 0, (int)OTG_ERR_INVALID);
    return false;
  }
  if (skip && skip[a]) return false;
  return !cand || (cand[f] && cand[t]);
}

__global__ void csr_count(int num_arcs, const int32_t* from, const int32_t* to,
                          const uint8_t* skip, const uint8_t* cand, int n, int32_t* fanin_cnt,
                          int32_t* out_deg, int* status) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < num_arcs; a += gridDim.x * blockDim.x)
    if (kept(a, from, to, skip, cand, n, status)) {
      atomicAdd(&fanin_cnt[to[a]], 1);
      atomicAdd(&out_deg[from[a]], 1);
    }
}

// Block-wide inclusive scan of one int per thread (kScanT threads).
__device__ __forceinline__ int block_incl(int v, int* wsum) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int y = __shfl_up_sync(0xFFFFFFFFu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < kScanT / 32 ? wsum[lane] : 0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int y = __shfl_up_sync(0xFFFFFFFFu, s, d);
      if (lane >= d) s += y;
    }
    if (lane < kScanT / 32) wsum[lane] = s;
  }
  __syncthreads();
  const int r = x + (w ? wsum[w - 1] : 0);
  __syncthreads();
  return r;
}

// Scan pass 1: the sum of each tile of kScanTile values (val(i) = src[i] or
// the flag of item i).
template <class ValF>
__device__ void tile_sums(int count, ValF val, int32_t* sums) {
  __shared__ int wsum[32];
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanK;
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanK; ++k)
    if (base + k < count) s += val(base + k);
  const int tot = block_incl(s, wsum);
  if (threadIdx.x == kScanT - 1) sums[blockIdx.x] = tot;
}

// Scan pass 2: exclusive scan of the tile sums in place (one block; any
// number of tiles, in chunks of kScanT); *total gets their sum.
__global__ void scan_sums(int32_t* sums, int tiles, int32_t* total) {
  __shared__ int wsum[32];
  __shared__ int s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int c = 0; c < tiles; c += kScanT) {
    const int i = c + threadIdx.x;
    const int v = i < tiles ? sums[i] : 0;
    const int inc = block_incl(v, wsum);
    const int carry = s_carry;
    if (i < tiles) sums[i] = carry + inc - v;
    __syncthreads();
    if (threadIdx.x == kScanT - 1) s_carry = carry + inc;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = s_carry;
}

// fanin_start[0..n]: exclusive scan of the counts (counts in fanin_start[0..n-1]).
__global__ void csr_sums(const int32_t* cnt, int n, int32_t* sums) {
  tile_sums(n, [&](int i) { return cnt[i]; }, sums);
}
__global__ void csr_scan(int32_t* start, int n, const int32_t* sums, int32_t* cursor) {
  __shared__ int wsum[32];
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanK;
  int v[kScanK], s = 0;
#pragma unroll
  for (int k = 0; k < kScanK; ++k) {
    v[k] = base + k < n ? start[base + k] : 0;
    s += v[k];
  }
  int run = block_incl(s, wsum) - s + sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanK; ++k)
    if (base + k < n) {
      start[base + k] = run;
      cursor[base + k] = run;
      run += v[k];
    }
}
__global__ void csr_last(int32_t* start, int n, const int32_t* total) { start[n] = *total; }

__global__ void csr_fill(int num_arcs, const int32_t* from, const int32_t* to,
                         const uint8_t* skip, const uint8_t* cand, int n, int32_t* cursor,
                         int32_t* fanin, int* status) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < num_arcs; a += gridDim.x * blockDim.x)
    if (kept(a, from, to, skip, cand, n, status)) fanin[atomicAdd(&cursor[to[a]], 1)] = a;
}

// Each pin's fanin arcs in arc order, then (from != null) arc -> source pin.
__global__ void csr_order(int n, const int32_t* start, int32_t* fanin, const int32_t* from) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const int b = start[v], e = start[v + 1];
    for (int i = b + 1; i < e; ++i) {
      const int x = fanin[i];
      int j = i - 1;
      while (j >= b && fanin[j] > x) {
        fanin[j + 1] = fanin[j];
        --j;
      }
      fanin[j + 1] = x;
    }
    if (from)
      for (int i = b; i < e; ++i) fanin[i] = from[fanin[i]];
  }
}

__global__ void seed_sums(int num_cands, const int32_t* cand_order, const int32_t* out_deg,
                          int n, int32_t* sums) {
  tile_sums(num_cands, [&](int i) {
    const int c = cand_order[i];
    return ((unsigned)c < (unsigned)n && out_deg[c] == 0) ? 1 : 0;
  }, sums);
}
__global__ void seed_put(int num_cands, const int32_t* cand_order, const int32_t* out_deg, int n,
                         const int32_t* sums, int32_t* frontier0, int* status) {
  __shared__ int wsum[32];
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanK;
  int f[kScanK], s = 0;
#pragma unroll
  for (int k = 0; k < kScanK; ++k) {
    f[k] = 0;
    if (base + k < num_cands) {
      const int c = cand_order[base + k];
      if ((unsigned)c >= (unsigned)n) atomicCAS(status, 0, (int)OTG_ERR_INVALID);
      else f[k] = out_deg[c] == 0;
    }
    s += f[k];
  }
  int run = block_incl(s, wsum) - s + sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanK; ++k)
    if (f[k]) frontier0[run++] = cand_order[base + k];
}

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace
}  // namespace otg

extern "C" {

otg_status otg_fanin_csr_workspace_size(int32_t n, int32_t num_arcs, int32_t num_cands,
                                        size_t* bytes) {
  if (!bytes || n < 0 || num_arcs < 0 || num_cands < 0) return OTG_ERR_INVALID;
  const size_t t1 = (size_t)(n + otg::kScanTile) / otg::kScanTile + 1;
  const size_t t2 = (size_t)(num_cands + otg::kScanTile) / otg::kScanTile + 1;
  *bytes = 256 + otg::al256(4 * (size_t)(n + 1)) + otg::al256(4 * (t1 > t2 ? t1 : t2));
  return OTG_OK;
}

otg_status otg_fanin_csr(int32_t n, int32_t num_arcs, const int32_t* from, const int32_t* to,
                         const uint8_t* arc_skip, const uint8_t* pin_cand, int32_t num_cands,
                         const int32_t* cand_order, int32_t fanin_as_arcs, int32_t* fanin_start,
                         int32_t* fanin, int32_t* out_deg, int32_t* frontier0, int32_t* counts,
                         void* workspace, size_t workspace_bytes, otg_stream_t stream) {
  if (n < 0 || num_arcs < 0 || num_cands < 0 || !fanin_start || !out_deg || !counts ||
      !workspace)
    return OTG_ERR_INVALID;
  if ((num_arcs && (!from || !to || !fanin)) || (num_cands && (!cand_order || !frontier0)))
    return OTG_ERR_INVALID;
  size_t need = 0;
  otg_fanin_csr_workspace_size(n, num_arcs, num_cands, &need);
  if (workspace_bytes < need) return OTG_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)workspace;
  int* status = (int*)ws;  // [0] status, [1] seed count scratch
  int32_t* cursor = (int32_t*)(ws + 256);
  int32_t* sums = (int32_t*)(ws + 256 + otg::al256(4 * (size_t)(n + 1)));
  int launches = 0;
  auto grid = [](long long items) {
    const long long b = (items + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 592 ? 592 : b));
  };
  otg::csr_zero<<<1, 32, 0, st>>>(status, 2); ++launches;
  otg::csr_zero<<<grid(n + 1), 256, 0, st>>>(fanin_start, n + 1); ++launches;
  otg::csr_zero<<<grid(n), 256, 0, st>>>(out_deg, n); ++launches;
  otg::csr_count<<<grid(num_arcs), 256, 0, st>>>(num_arcs, from, to, arc_skip, pin_cand, n,
                                                 fanin_start, out_deg, status); ++launches;
  const int tiles = (n + otg::kScanTile - 1) / otg::kScanTile;
  if (tiles > 0) {
    otg::csr_sums<<<tiles, otg::kScanT, 0, st>>>(fanin_start, n, sums); ++launches;
    otg::scan_sums<<<1, otg::kScanT, 0, st>>>(sums, tiles, counts + 1); ++launches;
    otg::csr_scan<<<tiles, otg::kScanT, 0, st>>>(fanin_start, n, sums, cursor); ++launches;
  } else {
    otg::csr_zero<<<1, 32, 0, st>>>(counts + 1, 1); ++launches;
  }
  otg::csr_last<<<1, 1, 0, st>>>(fanin_start, n, counts + 1); ++launches;
  otg::csr_fill<<<grid(num_arcs), 256, 0, st>>>(num_arcs, from, to, arc_skip, pin_cand, n,
                                                cursor, fanin, status); ++launches;
  otg::csr_order<<<grid(n), 256, 0, st>>>(n, fanin_start, fanin,
                                          fanin_as_arcs ? nullptr : from); ++launches;
  const int ctiles = (num_cands + otg::kScanTile - 1) / otg::kScanTile;
  if (ctiles > 0) {
    otg::seed_sums<<<ctiles, otg::kScanT, 0, st>>>(num_cands, cand_order, out_deg, n, sums); ++launches;
    otg::scan_sums<<<1, otg::kScanT, 0, st>>>(sums, ctiles, counts); ++launches;
    otg::seed_put<<<ctiles, otg::kScanT, 0, st>>>(num_cands, cand_order, out_deg, n, sums,
                                                 frontier0, status); ++launches;
  } else {
    otg::csr_zero<<<1, 32, 0, st>>>(counts, 1); ++launches;
  }
  for (int i = 0; i < launches; ++i) otg::count_launch();
  return cudaGetLastError() == cudaSuccess ? OTG_OK : OTG_ERR_CUDA;
}

otg_status otg_fanin_csr_status(const void* workspace, otg_stream_t stream) {
  if (!workspace) return OTG_ERR_INVALID;
  int h = 0;
  if (cudaMemcpyAsync(&h, workspace, 4, cudaMemcpyDeviceToHost, (cudaStream_t)stream) !=
          cudaSuccess ||
      cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
    return OTG_ERR_CUDA;
  return (otg_status)h;
}

}  // extern "C"
