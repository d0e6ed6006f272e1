// bench_probe.cu -- measurement probe of bench.py (bench_probe.so, built by
// bench.build_probe): the L2 reduction rate of this GPU for binary64 adds
// (the default deposit) and for 64-bit integer adds (the deterministic
// deposit's fixed-point words), the ceiling of an atomic-bound deposit.  Not
// part of the PIC library.
#include <cuda_runtime.h>

namespace {

// Every lane adds to its own 32-byte sector; neighbouring lanes use
// neighbouring sectors and the window is small enough to stay in L2, as the
// cell-sorted deposit's reductions do.  Each block walks its own slice of the
// window so blocks do not contend on one sector.
template <class T>
__global__ void red_probe_kernel(T* window, unsigned sectors, int rounds) {
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned stride = gridDim.x * blockDim.x;
  for (int r = 0; r < rounds; ++r) {
    const unsigned sector = (t + (unsigned)r * stride) % sectors;
    atomicAdd(&window[4u * sector], T(1));
  }
}

template <class T>
int reduction_rate(int window_mb, int repeats, double* reductions_per_second) {
  const size_t bytes = (size_t)window_mb << 20;
  const unsigned sectors = (unsigned)(bytes / 32);
  T* window = nullptr;
  if (cudaMalloc(&window, bytes) != cudaSuccess) return 1;
  cudaMemset(window, 0, bytes);
  int device = 0, sms = 0;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const dim3 grid(sms * 8), block(256);
  const int rounds = 256;
  cudaEvent_t start, stop;
  cudaEventCreate(&start);
  cudaEventCreate(&stop);
  red_probe_kernel<T><<<grid, block>>>(window, sectors, rounds);
  float best = 0.f;
  for (int i = 0; i < repeats; ++i) {
    cudaEventRecord(start);
    red_probe_kernel<T><<<grid, block>>>(window, sectors, rounds);
    cudaEventRecord(stop);
    cudaEventSynchronize(stop);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, start, stop);
    if (i == 0 || ms < best) best = ms;
  }
  const cudaError_t status = cudaGetLastError();
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  cudaFree(window);
  if (status != cudaSuccess || best <= 0.f) return 2;
  *reductions_per_second = (double)grid.x * block.x * rounds / (best * 1e-3);
  return 0;
}

}  // namespace

extern "C" {

// L2 reductions per second (best of `repeats` timed launches after one
// warm-up) into a `window_mb` MB array: binary64 adds, and 64-bit integer adds.
int aprl_probe_reduction_rate(int window_mb, int repeats, double* reductions_per_second) {
  return reduction_rate<double>(window_mb, repeats, reductions_per_second);
}
int aprl_probe_integer_reduction_rate(int window_mb, int repeats, double* reductions_per_second) {
  return reduction_rate<unsigned long long>(window_mb, repeats, reductions_per_second);
}

}  // extern "C"
