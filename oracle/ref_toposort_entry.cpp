// ref_toposort_entry.cpp -- toposort_compute_cuda for the reference Timer
// build that runs the reference's own CUDA kernels.  TEST INFRASTRUCTURE.
//
// The reference's host loop (ot/cuda/toposort.cu:25-72) reads a frontier
// counter it never clears, so it is not run (see ref_toposort.cu).  In the
// ot_run_ref link its symbol is made weak (objcopy -W) and this definition,
// with the reference's signature (ot/cuda/toposort.cuh:3-6), takes its
// place: the same levels from the reference's toposort_advance kernel,
// driven by otref_toposort_levels_cuda with the counter zeroed.
#include <cstdio>
#include <vector>

extern "C" int otref_toposort_levels_cuda(int n, int num_edges, int first_size,
                                          const int* edgelist_start, const int* edgelist,
                                          const int* out, int* frontiers, int* ends_out,
                                          int max_ends);

void toposort_compute_cuda(int n, int num_edges, int first_size, int* edgelist_start,
                           int* edgelist, int* out, int* frontiers,
                           std::vector<int>& frontiers_ends) {
  std::vector<int> ends(n + 2);
  const int k = otref_toposort_levels_cuda(n, num_edges, first_size, edgelist_start, edgelist,
                                           out, frontiers, ends.data(), (int)ends.size());
  if (k < 2) {
    std::fprintf(stderr, "ref toposort failed (%d)\n", k);
    return;
  }
  // the reference appends the level boundaries after {0, first_size}
  frontiers_ends.assign(ends.begin(), ends.begin() + k);
}
