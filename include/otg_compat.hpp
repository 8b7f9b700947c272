// otg_compat.hpp -- drop-in replacements for the C++ entry points of
// OpenTimer's CUDA module (ot/cuda/rct.cuh, ot/cuda/toposort.cuh), exported
// by libotg.so with the same mangled names so a reference build links them
// in place of its OpenTimerCUDA library.
//
// The three structs repeat the reference's member order exactly
// (ot/cuda/rct.cuh:7-42): they are the binary interface the reference's
// FlatRctStorage::_update_timing_cuda (ot/timer/net.cpp:239-276) fills in.
#ifndef OTG_COMPAT_HPP_
#define OTG_COMPAT_HPP_

#include <vector>

struct RctCUDA {
  int num_nets;
  int total_num_nodes;
  int* rct_nodes_start;
  int* rct_pid;
  float *pres, *cap, *load, *delay, *ldelay, *impulse;
};

struct RctEdgeCUDA {
  int s;
  int t;
};

struct RctEdgeArrayCUDA {
  int num_nets;
  int total_num_nodes;
  int total_num_edges;
  int* rct_nodes_start = nullptr;
  RctEdgeCUDA* rct_edges = nullptr;
  int* rct_roots = nullptr;
  float* rct_edges_res = nullptr;
  float* rct_nodes_cap = nullptr;
  int* rct_distances = nullptr;    // unused here (kept for layout)
  int* rct_sort_counts = nullptr;  // unused here (kept for layout)
  float* pres = nullptr;           // unused here (kept for layout)
  float* cap = nullptr;            // unused here (kept for layout)
  int* rct_node2bfs_order = nullptr;
  int* rct_pid = nullptr;
  float* load = nullptr;
  float* delay = nullptr;
  float* ldelay = nullptr;
  float* impulse = nullptr;
};

// Replaces rct_bfs_and_compute_cuda (ot/cuda/rct.cuh:45, ot/cuda/rct.cu:361-397).
// Host arrays in, host arrays out (edges rewritten to parent->child,
// node2bfs, pid, load/delay/ldelay/impulse in BFS order).  Errors are logged
// to stderr (the reference asserts); the copies back are queued before the
// status is read, so after an error the output arrays hold undefined values.
void rct_bfs_and_compute_cuda(RctEdgeArrayCUDA data_cpu);

// Replaces the never-called rct_compute_cuda (ot/cuda/rct.cuh:44,
// ot/cuda/rct.cu:102-118): the four Elmore sweeps on already BFS-ordered
// pid/pres/cap host arrays.
void rct_compute_cuda(RctCUDA data_cpu);

// Replaces toposort_compute_cuda (ot/cuda/toposort.cuh:3-6,
// ot/cuda/toposort.cu:25-72).  frontiers[0..first_size) holds the seed and
// frontiers_ends arrives as {0, first_size}; on return frontiers holds every
// level (later levels in ascending pin index) and frontiers_ends one entry
// per level boundary, as the reference appends them.
void toposort_compute_cuda(int n, int num_edges, int first_size, int* edgelist_start,
                           int* edgelist, int* out, int* frontiers,
                           std::vector<int>& frontiers_ends);

#endif  // OTG_COMPAT_HPP_
