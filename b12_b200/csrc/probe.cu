// Measurement helpers: a kernel-launch counter and an FP64 FMA throughput probe.
//
// The probe gives the FP64 roofline denominator for the box-image kernels: every
// thread runs 8 independent chains of dependent fused multiply-adds, enough
// independent work to keep the FP64 pipes of all SMs busy.
#include <atomic>

#include "tree.h"

namespace b12g {

std::atomic<unsigned long long> g_launches{0};

void count_launches(unsigned long long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

namespace {

__global__ void __launch_bounds__(256) fp64_fma_probe_kernel(double* out, int iters, double a, double b)
{
  double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-9, x2 = x0 + 2e-9, x3 = x0 + 3e-9;
  double x4 = x0 + 4e-9, x5 = x0 + 5e-9, x6 = x0 + 6e-9, x7 = x0 + 7e-9;
#pragma unroll 1
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = __fma_rn(x0, a, b); x1 = __fma_rn(x1, a, b); x2 = __fma_rn(x2, a, b); x3 = __fma_rn(x3, a, b);
      x4 = __fma_rn(x4, a, b); x5 = __fma_rn(x5, a, b); x6 = __fma_rn(x6, a, b); x7 = __fma_rn(x7, a, b);
    }
  }
  const double s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == 12345.678) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keep the chains alive
}

}  // namespace
}  // namespace b12g

using namespace b12g;
using namespace b12g::host;

extern "C" {

b12g_status b12g_launch_count(uint64_t* launches)
{
  if (!launches) return fail(B12G_ERR_INVALID, "NULL argument");
  *launches = g_launches.load();
  return B12G_OK;
}

b12g_status b12g_probe_fp64_fma(double seconds_hint, double* tflops, double* sm_seconds)
{
  if (!tflops) return fail(B12G_ERR_INVALID, "NULL argument");
  int dev = 0, sms = 0, bps = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fp64_fma_probe_kernel, 256, 0));
  const int blocks = sms * (bps > 0 ? bps : 1);
  double* out = nullptr;
  CK(cudaMalloc(&out, size_t(blocks) * 256 * sizeof(double)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int iters = 256;
  float ms = 0.f;
  // warm up, then grow the loop until one launch takes about `seconds_hint`
  for (int round = 0; round < 12; ++round) {
    cudaEventRecord(e0);
    fp64_fma_probe_kernel<<<blocks, 256>>>(out, iters, 0.999999999, 1e-12);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms > 1000.0 * seconds_hint || round == 11) break;
    iters *= 2;
  }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (e != cudaSuccess) return cuda_fail(e, "fp64 probe");
  const double flops = 2.0 * 8.0 * 16.0 * double(iters) * double(blocks) * 256.0;
  *tflops = flops / (ms * 1e-3) / 1e12;
  if (sm_seconds) *sm_seconds = ms * 1e-3;
  return B12G_OK;
}

}  // extern "C"
