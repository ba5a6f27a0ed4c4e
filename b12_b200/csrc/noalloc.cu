// Allocation-free invariant measure.
//
// Some callers of this library cannot let it allocate device memory: processes that
// have handed all free HBM to their own memory pool (a serving process whose caching
// allocator owns the device), and latency-critical loops where cudaMalloc/cudaFree
// would synchronize the whole device and stall every other stream.  For them,
// b12g_invariant_measure_noalloc runs the same power-iteration kernel as
// b12g_invariant_measure with its scratch (two iterates, per-block partial sums and the
// grid-barrier words) in one file-scope __device__ array of fixed size, so the call
// itself allocates nothing; the caller passes the matrix and the output.
//
// Limits and sharing: at most kMaxRows boxes (the array is 4.03 MiB and every GPU that
// loads the library holds it until the process exits).  All calls share the array, so
// calls that overlap on the GPU (different streams, or different host threads at the
// same time) race with each other; the barrier words that must start at zero are
// cleared by every call.  Before the power iteration a check kernel reads the row
// pointers and sources once; a matrix whose sources are not all below n is refused
// with B12G_ERR_INVALID before any iterate is read.
#include <mutex>

#include "csr.h"
#include "tree.h"

namespace {

constexpr uint32_t kMaxRows = 1u << 18;          // 262,144 boxes
constexpr uint32_t kPartialSlots = 4096;         // 2 x the largest grid of the launch
constexpr size_t kScratchBytes = 2 * size_t(kMaxRows) * sizeof(double) + kPartialSlots * sizeof(double) + 512;

static __device__ __align__(256) unsigned char g_measure_scratch[kScratchBytes];

std::mutex g_scratch_mu;
unsigned char* g_scratch_addr[64] = {};          // device address of the array, per device

// The host-side name of a __device__ array is only a stand-in; its device address is
// looked up once per device, with that device current.
b12g_status scratch_address(unsigned char** out)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return b12g::host::cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return b12g::host::fail(B12G_ERR_INVALID, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_measure_scratch);
    if (e != cudaSuccess) return b12g::host::cuda_fail(e, "cudaGetSymbolAddress(measure scratch)");
    g_scratch_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_addr[dev];
  return B12G_OK;
}

// The caller's P^T must index only its own n boxes: the iterates in the scratch array
// are read at every source index, so a source >= n would read past them.  One pass
// over the row pointers and sources sets bit 0 of *bad on the first violation
// (tptr[0] != 0, a decreasing row pointer, a source >= n).
__global__ void check_transpose_kernel(const uint32_t* tptr, const uint32_t* trows, uint32_t n, unsigned* bad)
{
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  if (tid == 0 && tptr[0] != 0u) atomicOr(bad, 1u);
  for (uint32_t j = tid; j < n; j += nthreads)
    if (tptr[j] > tptr[j + 1]) atomicOr(bad, 1u);
  const uint32_t nnz = tptr[n];
  for (uint32_t k = tid; k < nnz; k += nthreads)
    if (trows[k] >= n) atomicOr(bad, 1u);
}

}  // namespace

using namespace b12g::host;

extern "C" b12g_status b12g_invariant_measure_noalloc(const uint32_t* tptr, const uint32_t* trows,
                                                      const double* tvals, uint32_t n, uint32_t iters, double* v,
                                                      void* stream)
{
  if (!tptr || !trows || !tvals || !v) return fail(B12G_ERR_INVALID, "NULL argument");
  if (n > kMaxRows)
    return fail(B12G_ERR_CAPACITY, "invariant_measure_noalloc handles at most %u boxes (got %u)", kMaxRows, n);
  if (n == 0) return B12G_OK;
  unsigned char* base = nullptr;
  ST(scratch_address(&base));
  double* w0 = reinterpret_cast<double*>(base);
  double* w1 = w0 + kMaxRows;
  double* partial = w1 + kMaxRows;
  unsigned* sync_words = reinterpret_cast<unsigned*>(partial + kPartialSlots);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // word 96 of the barrier block (past the 65 words the kernel uses): the check's result
  unsigned* bad = sync_words + 96;
  unsigned err = 0;
  CK(cudaMemsetAsync(bad, 0, sizeof(unsigned), s));
  check_transpose_kernel<<<b12g::device_sm_count() * 4, 256, 0, s>>>(tptr, trows, n, bad);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(&err, bad, sizeof err, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (err) return fail(B12G_ERR_INVALID, "invariant_measure_noalloc: tptr/trows do not describe a matrix of %u boxes", n);
  CK(b12g::invariant_measure(tptr, trows, tvals, nullptr, 0, nullptr, 0, n, iters, w0, w1, partial, kPartialSlots, v,
                             sync_words, s));
  b12g::count_launches(2);
  CK(cudaMemcpyAsync(&err, sync_words + 64, sizeof err, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (err & 2u) return fail(B12G_ERR_TIMEOUT, "invariant_measure_noalloc: grid barrier gave up");
  return B12G_OK;
}
