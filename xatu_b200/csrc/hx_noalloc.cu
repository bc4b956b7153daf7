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
// fixed size (6 MB + 256 B), which every GPU that loads this library holds
// until the process exits.
#include <cstdio>
#include <mutex>

#include "engine.h"

// Largest problem the static scratch is sized for.
#define XATU_NOALLOC_MAX_N 16384
#define XATU_NOALLOC_MAX_NVEC 16

namespace {

constexpr long long kMaxLdb = 2LL * XATU_NOALLOC_MAX_N;          // bf16 per operand row (multiple of 8)
constexpr int kMaxRows = 2 * XATU_NOALLOC_MAX_NVEC;             // operand rows: Re block + Im block
constexpr size_t kPlaneBytes = (size_t)kMaxRows * kMaxLdb * 2;  // 2 MB per BF16 plane
constexpr size_t kAccBytes = (size_t)XATU_NOALLOC_MAX_N * kMaxRows * sizeof(float);  // 2 MB
constexpr size_t kScratchBytes = 2 * kPlaneBytes + kAccBytes + 256;

}  // namespace

// The scratch.  In host code `g_hx_noalloc_scratch` is only a host-side stand-in
// for the symbol; its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_hx_noalloc_scratch[kScratchBytes];

namespace {

std::mutex g_setup_mu;
void* g_scratch_addr[64] = {};
int g_num_sms[64] = {};

// Once per device, with that device current: the device address of the scratch.
xatu_status noalloc_setup(int dev, unsigned char** base, int* sms) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (dev < 0 || dev >= 64) {
    fprintf(stderr, "xatu_hx_noalloc: device ordinal %d out of range\n", dev);
    return XATU_ERR_UNSUPPORTED;
  }
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_hx_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      fprintf(stderr, "xatu_hx_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev, cudaGetErrorString(e));
      return XATU_ERR_CUDA;
    }
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    g_scratch_addr[dev] = p;
    g_num_sms[dev] = n;
  }
  *base = static_cast<unsigned char*>(g_scratch_addr[dev]);
  *sms = g_num_sms[dev];
  return XATU_OK;
}

}  // namespace

// Operand planes from x (column-major n x nvec complex): row s (< bp) holds
// (Re x_js, -Im x_js) at columns (2j, 2j+1), row bp + s holds (Im x_js, Re x_js);
// rows of padding vectors are zero.  BF16 hi + lo split.
__global__ void hx_noalloc_operand_kernel(const cd* __restrict__ x, long long n, int nvec, int bp, long long ldb,
                                          __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n * bp) return;
  const int s = (int)(t / n);
  const long long j = t - (long long)s * n;
  float re = 0.f, im = 0.f;
  if (s < nvec) {
    const cd v = x[(long long)s * n + j];
    re = (float)v.x;
    im = (float)v.y;
  }
  const float vals[4] = {re, -im, im, re};
  const long long off[4] = {(long long)s * ldb + 2 * j, (long long)s * ldb + 2 * j + 1,
                            (long long)(bp + s) * ldb + 2 * j, (long long)(bp + s) * ldb + 2 * j + 1};
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const __nv_bfloat16 h = __float2bfloat16_rn(vals[q]);
    hi[off[q]] = h;
    lo[off[q]] = __float2bfloat16_rn(vals[q] - __bfloat162float(h));
  }
}

// y[:, s] = acc (Re rows s, Im rows bp + s) + diag .* x[:, s], in FP64.
__global__ void hx_noalloc_finish_kernel(const float* __restrict__ acc, const double* __restrict__ diag,
                                         const cd* __restrict__ x, long long n, int nvec, int bp, cd* __restrict__ y) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n * nvec) return;
  const int s = (int)(t / n);
  const long long i = t - (long long)s * n;
  const cd v = x[t];
  y[t] = mk((double)acc[(long long)s * n + i] + diag[i] * v.x, (double)acc[(long long)(bp + s) * n + i] + diag[i] * v.y);
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
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return XATU_ERR_CUDA;
  unsigned char* base = nullptr;
  int sms = 0;
  xatu_status st = noalloc_setup(dev, &base, &sms);
  if (st != XATU_OK) return st;
  __nv_bfloat16* op_hi = reinterpret_cast<__nv_bfloat16*>(base);
  __nv_bfloat16* op_lo = reinterpret_cast<__nv_bfloat16*>(base + kPlaneBytes);
  float* acc = reinterpret_cast<float*>(base + 2 * kPlaneBytes);
  int* status = reinterpret_cast<int*>(base + 2 * kPlaneBytes + kAccBytes);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int bp = (nvec + 7) / 8 * 8;
  const int ng = 2 * bp;
  const long long ldb = (2 * n + 7) / 8 * 8;
  // the status word keeps the last call's value: clear it
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), s);
  if (e != cudaSuccess) goto cuda_error;
  {
    const long long t1 = n * bp;
    hx_noalloc_operand_kernel<<<(unsigned)((t1 + 255) / 256), 256, 0, s>>>(reinterpret_cast<const cd*>(x), n, nvec,
                                                                           bp, ldb, op_hi, op_lo);
    if ((e = cudaGetLastError()) != cudaSuccess) goto cuda_error;
    // the product zeroes the accumulator before it adds into it
    if ((e = xatu_launch_hx_tc(k_hi, k_lo, n, ldk, op_hi, op_lo, ldb, ng, acc, status, sms, s)) != cudaSuccess)
      goto cuda_error;
    const long long t2 = n * nvec;
    hx_noalloc_finish_kernel<<<(unsigned)((t2 + 255) / 256), 256, 0, s>>>(acc, diag, reinterpret_cast<const cd*>(x), n,
                                                                          nvec, bp, reinterpret_cast<cd*>(y));
    if ((e = cudaGetLastError()) != cudaSuccess) goto cuda_error;
    int h_status = 0;
    if ((e = cudaMemcpyAsync(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) goto cuda_error;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) goto cuda_error;
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
