// Y = K X for the mixed-precision kernel K = K_hi + K_lo (two BF16 planes,
// complex, row-major N x ldk, upper block triangle stored: xatu_kstored) and a
// block X of b complex FP32 vectors (row-major N x b).  CUDA-core version:
// 64-row x 32-column tiles of K are combined (hi + lo) into FP32 in shared
// memory and reused by every vector of the block; elements below the stored
// block triangle are read as the conjugate of their mirror; FP32 accumulation.
#include "engine.h"

#define HX_ROWS 64
#define HX_COLS 32
#define HX_THREADS 256
#define HX_MAXB 32

__global__ void __launch_bounds__(HX_THREADS)
hx_cuda_core_kernel(const __nv_bfloat162* __restrict__ Khi, const __nv_bfloat162* __restrict__ Klo,
                    long long ldk, const float2* __restrict__ X, float2* __restrict__ Y, long long N, int b) {
  __shared__ float2 sK[HX_ROWS][HX_COLS + 1];
  __shared__ float2 sX[HX_COLS][HX_MAXB];
  const long long row0 = (long long)blockIdx.x * HX_ROWS;
  const int tid = threadIdx.x;
  const int r = tid >> 2;         // 0..63
  const int sg = tid & 3;         // vector group
  const int per = (b + 3) / 4;    // vectors per thread (<= 8)
  float2 acc[HX_MAXB / 4];
#pragma unroll
  for (int s = 0; s < HX_MAXB / 4; s++) acc[s] = make_float2(0.f, 0.f);
  for (long long c0 = 0; c0 < N; c0 += HX_COLS) {
    for (int t = tid; t < HX_ROWS * HX_COLS; t += HX_THREADS) {
      const int rr = t / HX_COLS, cc = t % HX_COLS;
      const long long gr = row0 + rr, gc = c0 + cc;
      float2 v = make_float2(0.f, 0.f);
      if (gr < N && gc < N) {
        const bool st = xatu_kstored(gr, gc);
        const long long o = st ? gr * ldk + gc : gc * ldk + gr;
        const __nv_bfloat162 h = Khi[o], l = Klo[o];
        v.x = __bfloat162float(h.x) + __bfloat162float(l.x);
        v.y = __bfloat162float(h.y) + __bfloat162float(l.y);
        if (!st) v.y = -v.y;
      }
      sK[rr][cc] = v;
    }
    for (int t = tid; t < HX_COLS * b; t += HX_THREADS) {
      const int cc = t / b, s = t % b;
      const long long gc = c0 + cc;
      sX[cc][s] = (gc < N) ? X[gc * b + s] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int j = 0; j < HX_COLS; j++) {
      const float2 k = sK[r][j];
#pragma unroll
      for (int u = 0; u < HX_MAXB / 4; u++) {
        const int s = sg * per + u;
        if (u < per && s < b) {
          const float2 x = sX[j][s];
          acc[u].x = fmaf(k.x, x.x, acc[u].x);
          acc[u].x = fmaf(-k.y, x.y, acc[u].x);
          acc[u].y = fmaf(k.x, x.y, acc[u].y);
          acc[u].y = fmaf(k.y, x.x, acc[u].y);
        }
      }
    }
    __syncthreads();
  }
  const long long gr = row0 + r;
  if (gr < N) {
#pragma unroll
    for (int u = 0; u < HX_MAXB / 4; u++) {
      const int s = sg * per + u;
      if (u < per && s < b) Y[gr * b + s] = acc[u];
    }
  }
}

cudaError_t xatu_launch_hx_cuda_core(const __nv_bfloat162* Khi, const __nv_bfloat162* Klo, long long ldk, const float2* X,
                                     float2* Y, long long N, int b, cudaStream_t s) {
  if (b > HX_MAXB) return cudaErrorInvalidValue;
  const unsigned grid = (unsigned)((N + HX_ROWS - 1) / HX_ROWS);
  hx_cuda_core_kernel<<<grid, HX_THREADS, 0, s>>>(Khi, Klo, ldk, X, Y, N, b);
  return cudaGetLastError();
}
