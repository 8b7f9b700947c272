// ref_launch_timer.cpp -- CUDA-event timing of the kernels that the
// reference's own host code launches.  TEST / BENCHMARK INFRASTRUCTURE ONLY,
// linked into oracle/_ref/libotref.so with -Wl,--wrap=cudaLaunchKernel, so
// every <<<...>>> launch compiled into that library (the reference's
// ot/cuda/rct.cu among them) goes through __wrap_cudaLaunchKernel below.
//
// rct_bfs_and_compute_cuda (ot/cuda/rct.cu:361-397) allocates, copies,
// launches compute_net_bfs, prepare_res_cap and compute_net_timing, copies
// back and frees, all inside one call.  To report its kernel time apart
// from its copies, the wrapper records an event pair around each launch on
// the launch's stream while timing is on; otref_launch_timing_end sums the
// pairs after the call (the reference synchronizes the device itself).
// With timing off the wrapper only forwards the launch.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

extern "C" cudaError_t __real_cudaLaunchKernel(const void* func, dim3 grid, dim3 block,
                                               void** args, size_t smem, cudaStream_t stream);

namespace {
std::mutex g_mu;
bool g_on = false;
std::vector<cudaEvent_t> g_ev;  // pairs: before, after
}  // namespace

extern "C" {

cudaError_t __wrap_cudaLaunchKernel(const void* func, dim3 grid, dim3 block, void** args,
                                    size_t smem, cudaStream_t stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_on) return __real_cudaLaunchKernel(func, grid, block, args, smem, stream);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const bool ok = cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
  if (ok) cudaEventRecord(e0, stream);
  const cudaError_t r = __real_cudaLaunchKernel(func, grid, block, args, smem, stream);
  if (ok) {
    cudaEventRecord(e1, stream);
    g_ev.push_back(e0);
    g_ev.push_back(e1);
  }
  return r;
}

// Starts recording event pairs around every launch.
void otref_launch_timing_begin() {
  std::lock_guard<std::mutex> lk(g_mu);
  for (cudaEvent_t e : g_ev) cudaEventDestroy(e);
  g_ev.clear();
  g_on = true;
}

// Stops recording; returns the number of launches seen and their summed
// device time in milliseconds (-1 when an event could not be read).
int otref_launch_timing_end(double* total_ms) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_on = false;
  double sum = 0.0;
  bool bad = false;
  for (size_t i = 0; i + 1 < g_ev.size(); i += 2) {
    float ms = 0.f;
    if (cudaEventSynchronize(g_ev[i + 1]) != cudaSuccess ||
        cudaEventElapsedTime(&ms, g_ev[i], g_ev[i + 1]) != cudaSuccess)
      bad = true;
    sum += ms;
  }
  const int n = (int)(g_ev.size() / 2);
  for (cudaEvent_t e : g_ev) cudaEventDestroy(e);
  g_ev.clear();
  if (total_ms) *total_ms = bad ? -1.0 : sum;
  return n;
}

}  // extern "C"
