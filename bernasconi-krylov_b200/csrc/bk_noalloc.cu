// Measurement of a caller-owned statevector without any device allocation.
//
// Some callers cannot let a library allocate device memory: a host framework
// that owns all of the GPU's memory through its own caching allocator or a
// fixed arena (where a foreign cudaMalloc would fragment or exceed the budget),
// or a latency-critical loop where an allocation's implicit synchronisation is
// not allowed. bk_measure_noalloc serves them: the caller passes the statevector
// and the output buffer, and the only scratch — the per-block partial sums and
// the finishing ticket of the reduction — lives in the file-scope array below,
// which every GPU that loads this library holds until the process exits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "bk_device.cuh"
#include "bk_engine.h"

namespace {

// Scratch layout: [ticket: 4 B, padded to 256 B][kNoAllocSlots x 3 doubles].
constexpr int kNoAllocSlots = 1024;
constexpr size_t kTicketBytes = 256;
constexpr size_t kScratchBytes = kTicketBytes + (size_t)kNoAllocSlots * 3 * sizeof(double);  // 24.25 KiB
static __device__ __align__(256) unsigned char bk_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};  // device address of the array, per device
unsigned long long g_scratch_ctx[kMaxDevices] = {};  // id of the context that address belongs to

// Unique id of the calling thread's current context (cuCtxGetId never reuses an
// id within a process), or 0 when the driver entry points are unavailable. A
// cudaDeviceReset destroys the primary context and with it the array's
// address; the next call sees a new id and resolves the address again.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
    looked_up = true;
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

template <class A>
__global__ void __launch_bounds__(bk::kThreads) measure_noalloc_kernel(const A* __restrict__ psi, int n, int e0,
                                                                       uint32_t s0, unsigned char* scratch,
                                                                       double* out) {
  unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch);
  double* partials = reinterpret_cast<double*>(scratch + kTicketBytes);
  bk::MeasureAcc acc;
  const uint32_t count = 1u << n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    acc.add(bk::norm2d(psi[i]), bk::labs_energy(i, n) < e0, __popc(i ^ s0));
  // out[0] = P_<, out[1] = <d_H>, out[2] = |psi|^2 (row 0 of the results layout)
  bk::block_reduce_and_finalize(acc, partials, ticket, out, 0, (int)gridDim.x);
}

}  // namespace

extern "C" int bk_measure_noalloc(int n, int precision, const void* d_state, int64_t e0, uint64_t s0,
                                  double* d_out, void* stream) {
  if (n < 1 || n > 30) return BK_ERR_TOO_LARGE;
  if (!d_state || !d_out || (precision != BK_C64 && precision != BK_C128)) return BK_ERR_INVALID;
  // the kernel reads float2 / double2 amplitudes and writes doubles: a pointer
  // off that alignment would fault on the device, so it is refused here
  const uintptr_t state_align = precision == BK_C64 ? sizeof(float2) : sizeof(double2);
  if (reinterpret_cast<uintptr_t>(d_state) % state_align != 0 || reinterpret_cast<uintptr_t>(d_out) % sizeof(double) != 0)
    return BK_ERR_INVALID;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return BK_ERR_CUDA;
  unsigned char* scratch = nullptr;
  {
    // first call on this device (or in a new context of it): resolve the
    // array's device address, the host symbol being only a stand-in; make this
    // first call before any stream capture
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    const unsigned long long ctx_id = current_context_id();
    if (!g_scratch_ptr[dev] || ctx_id != g_scratch_ctx[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, bk_noalloc_scratch) != cudaSuccess || !p) return BK_ERR_CUDA;
      g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
      // the lookup has made the device's context current if it was not yet
      g_scratch_ctx[dev] = current_context_id();
    }
    scratch = g_scratch_ptr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the ticket must start at zero; calls that overlap on the GPU share this array and race
  if (cudaMemsetAsync(scratch, 0, sizeof(unsigned int), s) != cudaSuccess) return BK_ERR_CUDA;
  const uint32_t count = 1u << n;
  const unsigned blocks = (unsigned)((count + bk::kThreads * 8u - 1) / (bk::kThreads * 8u));
  const unsigned grid = blocks < (unsigned)kNoAllocSlots ? (blocks > 0 ? blocks : 1u) : (unsigned)kNoAllocSlots;
  const uint32_t s0m = (uint32_t)(s0 & (((uint64_t)1 << n) - 1u));
  if (e0 < 0) {  // threshold = E(s0)
    e0 = 0;
    for (int k = 1; k < n; ++k) {
      const int64_t ck = (int64_t)(n - k) - 2 * (int64_t)__builtin_popcount((s0m ^ (s0m >> k)) & ((1u << (n - k)) - 1u));
      e0 += ck * ck;
    }
  }
  const int e = (int)(e0 > (1 << 20) ? (1 << 20) : e0);
  if (precision == BK_C64)
    measure_noalloc_kernel<float2><<<grid, bk::kThreads, 0, s>>>(static_cast<const float2*>(d_state), n, e,
                                                                   s0m, scratch, d_out);
  else
    measure_noalloc_kernel<double2><<<grid, bk::kThreads, 0, s>>>(static_cast<const double2*>(d_state), n, e,
                                                                    s0m, scratch, d_out);
  return cudaGetLastError() == cudaSuccess ? BK_OK : BK_ERR_CUDA;
}
