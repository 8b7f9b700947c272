// ref_toposort.cu -- drives the reference's own toposort_advance kernel
// (ot/cuda/toposort.cu:4-21, compiled from the reference source into the
// same library) with a restatement of the host loop of toposort_compute_cuda
// (ot/cuda/toposort.cu:25-72).  TEST INFRASTRUCTURE ONLY.
//
// The reference loop itself is not called: it allocates its frontier
// counter with cudaMalloc and never clears it (toposort.cu:36-38, read back
// at :50 after the first launch), so a non-zero leftover value would make
// toposort_advance write past the frontier array.  This loop is the same
// except that the counter starts at zero; the kernel is the reference's.
#include <cuda_runtime.h>

#include <vector>

__global__ void toposort_advance(int* edgelist_start, int* edgelist, int* out, int* frontiers,
                                 int last_size, int* new_size);

extern "C" int otref_toposort_levels_cuda(int n, int num_edges, int first_size,
                                          const int* edgelist_start, const int* edgelist,
                                          const int* out, int* frontiers, int* ends_out,
                                          int max_ends) {
  if (first_size <= 0 || n <= 0) return -1;
  int *d_es = nullptr, *d_el = nullptr, *d_out = nullptr, *d_fr = nullptr, *d_ns = nullptr;
  bool ok = cudaMalloc(&d_es, sizeof(int) * (n + 1)) == cudaSuccess &&
            cudaMalloc(&d_el, sizeof(int) * (num_edges > 0 ? num_edges : 1)) == cudaSuccess &&
            cudaMalloc(&d_out, sizeof(int) * n) == cudaSuccess &&
            cudaMalloc(&d_fr, sizeof(int) * n) == cudaSuccess &&
            cudaMalloc(&d_ns, sizeof(int)) == cudaSuccess;
  int k = 0;
  if (ok) {
    cudaMemcpy(d_es, edgelist_start, sizeof(int) * (n + 1), cudaMemcpyHostToDevice);
    if (num_edges > 0) cudaMemcpy(d_el, edgelist, sizeof(int) * num_edges, cudaMemcpyHostToDevice);
    cudaMemcpy(d_out, out, sizeof(int) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_fr, frontiers, sizeof(int) * n, cudaMemcpyHostToDevice);
    cudaMemset(d_ns, 0, sizeof(int));
    std::vector<int> ends{0, first_size};
    int total_wo_last = 0, last = first_size;
    while (true) {
      toposort_advance<<<(last + 127) / 128, 128>>>(d_es, d_el, d_out, d_fr + total_wo_last,
                                                   last, d_ns);
      int cur = 0;
      cudaMemcpy(&cur, d_ns, sizeof(int), cudaMemcpyDeviceToHost);
      if (!cur) break;
      total_wo_last += last;
      last = cur;
      ends.push_back(total_wo_last + cur);
      cudaMemset(d_ns, 0, sizeof(int));
    }
    cudaMemcpy(frontiers, d_fr, sizeof(int) * n, cudaMemcpyDeviceToHost);
    for (; k < (int)ends.size() && k < max_ends; ++k) ends_out[k] = ends[k];
  }
  cudaFree(d_es);
  cudaFree(d_el);
  cudaFree(d_out);
  cudaFree(d_fr);
  cudaFree(d_ns);
  return ok && cudaGetLastError() == cudaSuccess ? k : -1;
}
