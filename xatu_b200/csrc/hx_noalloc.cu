// y = H x for the mixed-precision BSE matrix without any device allocation.
//
// Who needs it: callers that cannot call cudaMalloc.  Two kinds use this
// library that way:
//   * host codes that reserve (nearly) all of the GPU's memory up front in
//     their own pool and hand out pieces of it; a cudaMalloc behind their back
//     fails or fragments that pool, so they pass in every buffer themselves;
//   * iterative eigensolvers written by the caller (reverse-communication
//     Lanczos / Davidson loops) that request the product thousands of times; a
//     cudaMalloc / cudaFree pair per request would add a device-wide
//     synchronisation to every iteration.
// The caller owns the inputs (the two BF16 planes and the FP64 diagonal of a
// mixed build, and x) and the output y, all in device memory.  The scratch the
// tensor-core product needs -- the BF16 operand planes built from x, the FP32
// accumulator and a status word -- lives in one file-scope __device__ array of
// fixed size (8 MB + 256 B), which every GPU that loads this library holds
// until the process exits.
#include <cuda.h>

#include <cstdio>
#include <mutex>

#include "engine.h"

// Largest problem the static scratch is sized for.
#define XATU_NOALLOC_MAX_N 16384
#define XATU_NOALLOC_MAX_NVEC 16

namespace {

constexpr long long kMaxLdb = 2LL * XATU_NOALLOC_MAX_N;          // bf16 per Bt operand row (multiple of 8)
constexpr long long kMaxLdu = XATU_NOALLOC_MAX_N;                // bf16 per Bu operand row (multiple of 8)
constexpr int kMaxRows = 2 * XATU_NOALLOC_MAX_NVEC;             // operand rows: Re block + Im block
constexpr size_t kPlaneBytes = (size_t)kMaxRows * kMaxLdb * 2;  // 2 MB per Bt plane
constexpr size_t kUPlaneBytes = (size_t)kMaxRows * kMaxLdu * 2; // 1 MB per Bu plane
constexpr size_t kAccBytes = (size_t)XATU_NOALLOC_MAX_N * kMaxRows * sizeof(float);  // 2 MB
constexpr size_t kScratchBytes = 2 * kPlaneBytes + 2 * kUPlaneBytes + kAccBytes + 256;
static_assert(XATU_NOALLOC_MAX_NVEC <= XATU_HX_TC_MAXB, "one tensor-core product per call");

}  // namespace

// The scratch.  In host code `g_hx_noalloc_scratch` is only a host-side stand-in
// for the symbol; its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_hx_noalloc_scratch[kScratchBytes];

namespace {

// The driver's handle of the current context, looked up through the runtime's entry-point table so that the
// library does not link libcuda directly.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrentFn>(p);
  }
  return fn;
}

std::mutex g_setup_mu;
void* g_scratch_addr[64] = {};
CUcontext g_scratch_ctx[64] = {};
int g_num_sms[64] = {};

// Once per device and context, with that device current: the device address of the scratch.  The address
// is looked up again when the device's context changed since the last call (after cudaDeviceReset or a
// released and recreated primary context, the module and its array are loaded anew).
xatu_status noalloc_setup(int dev, unsigned char** base, int* sms) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (dev < 0 || dev >= 64) {
    fprintf(stderr, "xatu_hx_noalloc: device ordinal %d out of range\n", dev);
    return XATU_ERR_UNSUPPORTED;
  }
  CUcontext cur = nullptr;
  CtxGetCurrentFn get = ctx_get_current();
  if (!get || get(&cur) != CUDA_SUCCESS) {
    fprintf(stderr, "xatu_hx_noalloc: cannot query the current CUDA context\n");
    return XATU_ERR_CUDA;
  }
  if (!g_scratch_addr[dev] || g_scratch_ctx[dev] != cur) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_hx_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      fprintf(stderr, "xatu_hx_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev, cudaGetErrorString(e));
      return XATU_ERR_CUDA;
    }
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    if (get(&cur) != CUDA_SUCCESS) return XATU_ERR_CUDA;   // the lookup may have created the primary context
    g_scratch_addr[dev] = p;
    g_scratch_ctx[dev] = cur;
    g_num_sms[dev] = n;
  }
  *base = static_cast<unsigned char*>(g_scratch_addr[dev]);
  *sms = g_num_sms[dev];
  return XATU_OK;
}

}  // namespace

// y[:, s] = acc (row i: Re in column s, Im in column bp + s) + diag .* x[:, s], in FP64.
__global__ void hx_noalloc_finish_kernel(const float* __restrict__ acc, const double* __restrict__ diag,
                                         const cd* __restrict__ x, long long n, int nvec, int bp, cd* __restrict__ y) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n * nvec) return;
  const int s = (int)(t / n);
  const long long i = t - (long long)s * n;
  const cd v = x[t];
  const float* a = acc + i * 2 * bp;
  y[t] = mk((double)a[s] + diag[i] * v.x, (double)a[bp + s] + diag[i] * v.y);
}

extern "C" xatu_status xatu_hx_noalloc(const void* k_hi, const void* k_lo, const double* diag, int64_t n, int64_t ldk,
                                       int nvec, const double* x, double* y, void* stream) {
  if (!k_hi || !k_lo || !diag || !x || !y) {
    fprintf(stderr, "xatu_hx_noalloc: null device pointer\n");
    return XATU_ERR_INVALID;
  }
  if (n < 1 || n > XATU_NOALLOC_MAX_N) {
    fprintf(stderr, "xatu_hx_noalloc: n = %lld outside [1, %d], the size its static scratch is built for\n",
            (long long)n, XATU_NOALLOC_MAX_N);
    return XATU_ERR_UNSUPPORTED;
  }
  if (nvec < 1 || nvec > XATU_NOALLOC_MAX_NVEC) {
    fprintf(stderr, "xatu_hx_noalloc: nvec = %d outside [1, %d], the size its static scratch is built for\n", nvec,
            XATU_NOALLOC_MAX_NVEC);
    return XATU_ERR_UNSUPPORTED;
  }
  if (ldk < n || (ldk % 4) != 0) {
    fprintf(stderr, "xatu_hx_noalloc: ldk = %lld must be >= n and a multiple of 4\n", (long long)ldk);
    return XATU_ERR_INVALID;
  }
  if ((reinterpret_cast<uintptr_t>(k_hi) | reinterpret_cast<uintptr_t>(k_lo) | reinterpret_cast<uintptr_t>(x) |
       reinterpret_cast<uintptr_t>(y)) & 15) {
    fprintf(stderr, "xatu_hx_noalloc: device pointers must be 16-byte aligned\n");
    return XATU_ERR_INVALID;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  {
    // the call reads its status word back and waits for the stream, which a stream capture does not allow
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) return XATU_ERR_CUDA;
    if (cs != cudaStreamCaptureStatusNone) {
      fprintf(stderr, "xatu_hx_noalloc: the stream is being captured; the call waits for its stream and cannot "
                      "run inside a capture\n");
      return XATU_ERR_STATE;
    }
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return XATU_ERR_CUDA;
  unsigned char* base = nullptr;
  int sms = 0;
  xatu_status st = noalloc_setup(dev, &base, &sms);
  if (st != XATU_OK) return st;
  __nv_bfloat16* op_hi = reinterpret_cast<__nv_bfloat16*>(base);
  __nv_bfloat16* op_lo = reinterpret_cast<__nv_bfloat16*>(base + kPlaneBytes);
  __nv_bfloat16* ou_hi = reinterpret_cast<__nv_bfloat16*>(base + 2 * kPlaneBytes);
  __nv_bfloat16* ou_lo = reinterpret_cast<__nv_bfloat16*>(base + 2 * kPlaneBytes + kUPlaneBytes);
  float* acc = reinterpret_cast<float*>(base + 2 * kPlaneBytes + 2 * kUPlaneBytes);
  int* status = reinterpret_cast<int*>(base + 2 * kPlaneBytes + 2 * kUPlaneBytes + kAccBytes);
  const int bp = (nvec + 7) / 8 * 8;
  const int ng = 2 * bp;
  const long long ldb = (2 * n + 7) / 8 * 8, ldu = (n + 7) / 8 * 8;
  // the status word keeps the last call's value: clear it
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), s);
  if (e != cudaSuccess) goto cuda_error;
  {
    // every operand row (padding rows included) is rewritten from x: nothing of an earlier call is read
    if ((e = xatu_launch_hx_operands(reinterpret_cast<const cd*>(x), n, n, nvec, bp, op_hi, op_lo, ldb, ou_hi, ou_lo,
                                     ldu, s)) != cudaSuccess)
      goto cuda_error;
    // the product zeroes the accumulator before it adds into it
    if ((e = xatu_launch_hx_tc(k_hi, k_lo, n, ldk, op_hi, op_lo, ldb, ou_hi, ou_lo, ldu, ng, acc, status, sms, s)) !=
        cudaSuccess)
      goto cuda_error;
    const long long t2 = n * nvec;
    hx_noalloc_finish_kernel<<<(unsigned)((t2 + 255) / 256), 256, 0, s>>>(acc, diag, reinterpret_cast<const cd*>(x), n,
                                                                          nvec, bp, reinterpret_cast<cd*>(y));
    if ((e = cudaGetLastError()) != cudaSuccess) goto cuda_error;
    int h_status = 0;
    if ((e = cudaMemcpyAsync(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) goto cuda_error;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) goto cuda_error;
    if (h_status & XATU_DEVERR_INDEX) {
      // a CTA's row range spans more accumulators than the kernel holds: a launch-geometry fault of the library
      fprintf(stderr, "xatu_hx_noalloc: internal error, tile range outside the kernel's accumulators (status %d)\n",
              h_status);
      return XATU_ERR_INVALID;
    }
    if (h_status != 0) {
      fprintf(stderr, "xatu_hx_noalloc: a tensor-core pipeline wait timed out (status %d)\n", h_status);
      return XATU_ERR_NOT_CONVERGED;
    }
  }
  return XATU_OK;
cuda_error:
  fprintf(stderr, "xatu_hx_noalloc: %s\n", cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? XATU_ERR_ALLOC : XATU_ERR_CUDA;
}
