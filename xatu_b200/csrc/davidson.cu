// Block Davidson for the lowest exciton states of the BSE matrix, kept on
// the device (replaces davidson_method, davidson.cpp:5-60, and the dense
// eigensolve when only a few states are wanted).
//
// Design (not the reference's algorithm; it converges to the same lowest
// eigenpairs):
//   * start vectors: unit vectors at the smallest diagonal entries of H
//     (the reference starts from the first identity columns, davidson.cpp:19);
//   * H.V: mixed build -> diag(E) V in FP64 plus K V with K = K_hi + K_lo
//     (split BF16, FP32 accumulation); FP64 build -> ZGEMM on the FP64 matrix;
//   * Rayleigh-Ritz in FP64: T = V^H (H V) grown by the new columns only, the
//     lowest block of its eigenpairs by a one-CTA Householder / multisection /
//     inverse-iteration solver (eigh_small.cuh);
//   * residuals r = H u - theta u in FP64, per-row diagonal preconditioner
//     t = r / (theta - H_ii) (the reference divides by H_jj of the state
//     index j, davidson.cpp:36-40);
//   * FP64 orthogonalisation: two passes of block classical Gram-Schmidt
//     against the basis, then pivoted Cholesky-QR (twice) inside the block;
//   * thick restart on the lowest `block` Ritz vectors when the basis is full;
//   * caps on iterations and wall time -> XATU_ERR_NOT_CONVERGED.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "engine.h"
#include "dav_tall.cuh"
#include "eigh_small.cuh"

#define DAV_MAX_BASIS 112

// Chained launch (xatu_launch_chained) on the context's stream, counted and checked.
#define XATU_CHAIN(kernel, grid, block, smem, ...)                                                        \
  do {                                                                                                   \
    const cudaError_t e__ = xatu_launch_chained(kernel, dim3(grid), dim3(block), (size_t)(smem), ctx->stream, \
                                                __VA_ARGS__);                                            \
    ctx->launches++;                                                                                     \
    if (e__ != cudaSuccess) return xatu_cuda_fail(ctx, e__, "launch of " #kernel);                      \
  } while (0)

// ---------------------------------------------------------------- kernels
__global__ void dav_diag_mixed_kernel(const __nv_bfloat162* __restrict__ Khi, const __nv_bfloat162* __restrict__ Klo,
                                      const double* __restrict__ d, long long N, long long ldk, double* __restrict__ out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  out[i] = d[i] + (double)__bfloat162float(Khi[i * ldk + i].x) + (double)__bfloat162float(Klo[i * ldk + i].x);
}

__global__ void dav_diag_fp64_kernel(const cd* __restrict__ H, long long N, double* __restrict__ out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  out[i] = H[i * N + i].x;
}

// V[:, col0 + s] = e_{idx[s]}
// Start block: column s = e_idx[s] + noise * xi_s, xi_s a fixed pseudo-random vector (splitmix64 of (i, s),
// entries uniform in [-1, 1)).  The reference starts from unit vectors (davidson.cpp:16).  Unit vectors alone can leave a symmetry sector of H without a start vector
// for every copy of a degenerate level (spin-degenerate models: H is block diagonal, the unit vectors of
// the lowest diagonal entries fall unevenly in the blocks), and no correction ever leaves its block; the
// noise gives every column a component in every sector.
__device__ __forceinline__ double dav_noise(unsigned long long i, unsigned long long s) {
  unsigned long long z = i * 0x9E3779B97F4A7C15ull + (s + 1) * 0xD1B54A32D192ED03ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// The nsel lowest entries of d, ties resolved by the lower index, in ascending order into idx (the start
// columns of the Davidson basis), and *kept = nsel.  One CTA: every thread keeps the lowest untaken entry of its
// strided share; each round a block-wide arg-min picks the winner, whose owner marks it taken in the scratch copy
// w and rescans its share.
#define DAV_SEL_THREADS 1024
__device__ __forceinline__ bool dav_sel_less(double a, long long ia, double b, long long ib) {
  return a < b || (a == b && ia < ib);
}
#define DAV_SEL_SMEM_ROWS 24576   // diagonals up to this length are worked on in shared memory (192 KB)
__global__ void __launch_bounds__(DAV_SEL_THREADS)
dav_select_lowest_kernel(const double* __restrict__ d, long long N, int nsel, double* __restrict__ wg,
                         int* __restrict__ idx, int* __restrict__ kept) {
  extern __shared__ double ws[];
  __shared__ double sv[DAV_SEL_THREADS / 32];
  __shared__ long long si[DAV_SEL_THREADS / 32];
  __shared__ long long win;
  double* w = N <= DAV_SEL_SMEM_ROWS ? ws : wg;   // working copy of the diagonal (winners set to +inf)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double best = INFINITY;
  long long bi = N;
  for (long long i = tid; i < N; i += DAV_SEL_THREADS) {
    const double v = d[i];
    w[i] = v;
    if (dav_sel_less(v, i, best, bi)) {
      best = v;
      bi = i;
    }
  }
  for (int r = 0; r < nsel; r++) {
    double b = best;
    long long ib = bi;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, b, o);
      const long long oi = __shfl_xor_sync(0xffffffffu, ib, o);
      if (dav_sel_less(ob, oi, b, ib)) {
        b = ob;
        ib = oi;
      }
    }
    if (lane == 0) {
      sv[warp] = b;
      si[warp] = ib;
    }
    __syncthreads();
    if (warp == 0) {
      b = lane < DAV_SEL_THREADS / 32 ? sv[lane] : INFINITY;
      ib = lane < DAV_SEL_THREADS / 32 ? si[lane] : N;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, b, o);
        const long long oi = __shfl_xor_sync(0xffffffffu, ib, o);
        if (dav_sel_less(ob, oi, b, ib)) {
          b = ob;
          ib = oi;
        }
      }
      if (lane == 0) {
        win = ib;
        idx[r] = (int)(ib < N ? ib : r);   // fewer than nsel finite entries: any column
      }
    }
    __syncthreads();
    const long long wi = win;
    if (wi < N && wi % DAV_SEL_THREADS == tid) {
      w[wi] = INFINITY;
      best = INFINITY;
      bi = N;
      for (long long i = tid; i < N; i += DAV_SEL_THREADS) {
        const double v = w[i];
        if (dav_sel_less(v, i, best, bi)) {
          best = v;
          bi = i;
        }
      }
    }
  }
  if (tid == 0) *kept = nsel;
}

__global__ void dav_start_vectors_kernel(cd* V, long long N, int col0, const int* idx, int nvec, double noise) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= N * nvec) return;
  const int s = (int)(t / N);
  const long long i = t - (long long)s * N;
  V[(long long)(col0 + s) * N + i] = mk((i == idx[s] ? 1.0 : 0.0) + noise * dav_noise(i, s), 0.0);
}

// X (row-major N x nv, complex float) <- V[:, col0 : col0 + nv]
__global__ void dav_gather_f32_kernel(const cd* __restrict__ V, long long N, int col0, int nv, float2* __restrict__ X) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= N * nv) return;
  const long long i = t / nv;
  const int s = (int)(t - i * nv);
  const cd v = V[(long long)(col0 + s) * N + i];
  X[t] = make_float2((float)v.x, (float)v.y);
}

// W[:, col0 + s] = Y[:, s] + d .* V[:, col0 + s]   (the FP64 band-energy diagonal)
__global__ void dav_finish_w_kernel(const float2* __restrict__ Y, const double* __restrict__ d,
                                    const cd* __restrict__ V, long long N, int col0, int nv, cd* __restrict__ W) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= N * nv) return;
  const long long i = t / nv;
  const int s = (int)(t - i * nv);
  const float2 y = Y[t];
  const long long o = (long long)(col0 + s) * N + i;
  const cd v = V[o];
  W[o] = mk((double)y.x + d[i] * v.x, (double)y.y + d[i] * v.y);
}

// T (column-major, ld) : fill T[m0:m, 0:m0] = conj(T[0:m0, m0:m])^T and make the new block Hermitian.
// Columns of the new block that the orthonormalisation dropped are exact zero vectors (and so are their
// W = H V columns): their rows and columns of T are zero.  Their diagonal is set above a Gershgorin bound of
// the kept part, so they stay decoupled and never enter the lowest Ritz pairs (their Ritz coefficients
// multiply zero columns).  The kept count is copied next to the Ritz values for the host's read-back.
__global__ void dav_dead_kernel(cd* T, int ld, int m, int m0, const int* __restrict__ kept, double* kept_out) {
  xatu_grid_chain();
  const int nnew = m - m0;
  const int kc = min(max(*kept, 0), nnew);
  if (threadIdx.x == 0) *kept_out = (double)kc;
  if (kc >= nnew) return;   // uniform over the CTA
  const int live = m0 + kc;
  __shared__ double red[32];
  double bnd = -INFINITY;
  for (int r = threadIdx.x; r < live; r += blockDim.x) {
    double sum = T[r + (long long)r * ld].x;
    for (int c = 0; c < live; c++)
      if (c != r) {
        const cd v = T[r + (long long)c * ld];
        sum += sqrt(v.x * v.x + v.y * v.y);
      }
    bnd = fmax(bnd, sum);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) bnd = fmax(bnd, __shfl_xor_sync(0xffffffffu, bnd, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = bnd;
  __syncthreads();
  double b = -INFINITY;
  for (int w = 0; w < (int)(blockDim.x >> 5); w++) b = fmax(b, red[w]);
  if (!(b > -INFINITY)) b = 0.0;
  const double shift = b + fmax(1.0, fabs(b));
  for (int j = live + threadIdx.x; j < m; j += blockDim.x) T[j + (long long)j * ld] = mk(shift, 0.0);
}

__global__ void dav_hermitize_kernel(cd* T, int ld, int m, int m0) {
  xatu_grid_chain();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nnew = m - m0;
  if (t >= nnew * m) return;
  const int c = m0 + t / m;   // column in the new block
  const int r = t % m;        // row
  if (r < m0) {
    const cd v = T[r + (long long)c * ld];
    T[c + (long long)r * ld] = conj(v);
  } else if (r < c) {
    const cd a = T[r + (long long)c * ld], b = T[c + (long long)r * ld];
    const cd h = mk(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
    T[r + (long long)c * ld] = h;
    T[c + (long long)r * ld] = conj(h);
  } else if (r == c) {
    T[r + (long long)c * ld].y = 0.0;
  }
}

// T = diag(theta[0:k])
__global__ void dav_set_diag_kernel(cd* T, int ld, int k, const double* theta) {
  xatu_grid_chain();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= k * k) return;
  const int r = t % k, c = t / k;
  T[r + (long long)c * ld] = mk(r == c ? theta[r] : 0.0, 0.0);
}

// Rayleigh-Ritz eigensolve: lowest k eigenpairs of T (m x m, column-major ldt), one CTA (eigh_small.cuh).
__global__ void __launch_bounds__(HEEV_THREADS)
dav_heev_kernel(const cd* __restrict__ T, int ldt, int m, int k, double* __restrict__ theta, cd* __restrict__ Y,
                int ldy, cd* __restrict__ refl, int* __restrict__ status, long long* __restrict__ prof) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  xatu_grid_chain();
  heev_lowest(T, ldt, m, k, theta, Y, ldy, refl, smem_raw, status, prof);
}

// Bt operand of the tensor-core product (hx_tc.cu) from V[:, col0 : col0 + b]:
//   rows [0, bp):   Re X at 2j, -Im X at 2j+1;   rows [bp, 2bp): Im X at 2j, Re X at 2j+1
// (bp = b rounded up to 8; padding rows are zero), split into BF16 hi + lo.
// W[:, col0 + s] = (Y[:, s], Y[:, bp + s]) + d .* V[:, col0 + s]; Y row-major N x 2bp.
__global__ void dav_finish_w_tc_kernel(const float* __restrict__ Y, const double* __restrict__ d,
                                       const cd* __restrict__ V, long long N, int col0, int b, int bp,
                                       cd* __restrict__ W) {
  xatu_grid_chain();
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= N * b) return;
  const int s = (int)(t / N);
  const long long i = t - (long long)s * N;
  const long long o = (long long)(col0 + s) * N + i;
  const cd v = V[o];
  const float* y = Y + i * 2 * bp;
  W[o] = mk((double)y[s] + d[i] * v.x, (double)y[bp + s] + d[i] * v.y);
}

static bool tc_usable(const xatu_ctx* ctx) {
  if (ctx->hx_backend == 1) return false;
  return (ctx->ldk % 4) == 0;
}

xatu_status xatu_apply_h(xatu_ctx* ctx, long long N, int col0, int nv) {
  cd* V = ctx->dv_V.as<cd>();
  cd* W = ctx->dv_W.as<cd>();
  const int threads = 256;
  if (ctx->built_prec == XATU_PREC_FP64) {
    static const cuDoubleComplex one = {1.0, 0.0}, zero = {0.0, 0.0};
    cublasStatus_t bs = cublasZgemm(ctx->blas, CUBLAS_OP_T, CUBLAS_OP_N, (int)N, nv, (int)N, &one,
                                    ctx->d_H.as<cuDoubleComplex>(), (int)N,
                                    reinterpret_cast<cuDoubleComplex*>(V + (long long)col0 * N), (int)N, &zero,
                                    reinterpret_cast<cuDoubleComplex*>(W + (long long)col0 * N), (int)N);
    if (bs != CUBLAS_STATUS_SUCCESS) return xatu_fail(ctx, XATU_ERR_CUDA, "cublasZgemm (H.V) failed");
    return XATU_OK;
  }
  if (tc_usable(ctx)) {
    const long long ldb = (2 * N + 7) / 8 * 8, ldu = (N + 7) / 8 * 8;
    constexpr int MAXB = XATU_HX_TC_MAXB;
    for (int c = 0; c < nv; c += MAXB) {
      const int b = std::min(MAXB, nv - c);
      const int bp = (b + 7) / 8 * 8;
      const int ng = 2 * bp;
      XATU_CK(ctx->dv_Bop.ensure((size_t)2 * MAXB * ldb * sizeof(__nv_bfloat16)));
      XATU_CK(ctx->dv_Blo.ensure((size_t)2 * MAXB * ldb * sizeof(__nv_bfloat16)));
      XATU_CK(ctx->dv_Uhi.ensure((size_t)2 * MAXB * ldu * sizeof(__nv_bfloat16)));
      XATU_CK(ctx->dv_Ulo.ensure((size_t)2 * MAXB * ldu * sizeof(__nv_bfloat16)));
      XATU_CK(ctx->dv_Yf.ensure((size_t)N * 2 * MAXB * sizeof(float)));
      XATU_CK(xatu_launch_hx_operands(V + (long long)(col0 + c) * N, N, N, b, bp, ctx->dv_Bop.p, ctx->dv_Blo.p, ldb,
                                      ctx->dv_Uhi.p, ctx->dv_Ulo.p, ldu, ctx->stream));
      ctx->launches++;
      if (c == 0) XATU_CK(cudaEventRecord(ctx->ev[8], ctx->stream));
      XATU_CK(xatu_launch_hx_tc(ctx->d_Khi.p, ctx->d_Klo.p, N, ctx->ldk, ctx->dv_Bop.p, ctx->dv_Blo.p, ldb,
                                ctx->dv_Uhi.p, ctx->dv_Ulo.p, ldu, ng, ctx->dv_Yf.as<float>(), ctx->d_status.as<int>(),
                                ctx->num_sms, ctx->stream));
      if (c + MAXB >= nv) XATU_CK(cudaEventRecord(ctx->ev[9], ctx->stream));
      ctx->hx_pending = true;
      ctx->hx_calls++;
      ctx->hx_last_path = 2;
      ctx->launches++;
      const long long tw = N * b;
      XATU_CHAIN(dav_finish_w_tc_kernel, (int)((tw + threads - 1) / threads), threads, 0, ctx->dv_Yf.as<float>(),
                 ctx->d_diag.as<double>(), V, N, col0 + c, b, bp, W);
    }
    return XATU_OK;
  }
  XATU_CK(ctx->dv_X.ensure((size_t)N * 32 * sizeof(float2)));
  XATU_CK(ctx->dv_Yf.ensure((size_t)N * 64 * sizeof(float)));
  for (int c = 0; c < nv; c += 32) {
    const int b = std::min(32, nv - c);
    const long long tot = N * b;
    const int blocks = (int)((tot + threads - 1) / threads);
    dav_gather_f32_kernel<<<blocks, threads, 0, ctx->stream>>>(V, N, col0 + c, b, ctx->dv_X.as<float2>());
    ctx->launches++;
    if (c == 0) XATU_CK(cudaEventRecord(ctx->ev[8], ctx->stream));
    XATU_CK(xatu_launch_hx_cuda_core(ctx->d_Khi.as<__nv_bfloat162>(), ctx->d_Klo.as<__nv_bfloat162>(), ctx->ldk,
                                     ctx->dv_X.as<float2>(), ctx->dv_Yf.as<float2>(), N, b, ctx->stream));
    if (c + 32 >= nv) XATU_CK(cudaEventRecord(ctx->ev[9], ctx->stream));
    ctx->hx_pending = true;
    ctx->hx_calls++;
    ctx->hx_last_path = 1;
    ctx->launches++;
    dav_finish_w_kernel<<<blocks, threads, 0, ctx->stream>>>(ctx->dv_Yf.as<float2>(), ctx->d_diag.as<double>(), V, N,
                                                             col0 + c, b, W);
    ctx->launches++;
    XATU_CK(cudaGetLastError());
  }
  return XATU_OK;
}

void xatu_hx_collect(xatu_ctx* ctx) {
  if (!ctx->hx_pending) return;
  float ms = 0;
  if (cudaEventElapsedTime(&ms, ctx->ev[8], ctx->ev[9]) == cudaSuccess) ctx->hx_ms += ms;
  ctx->hx_pending = false;
}

#define XATU_TRY(x)                  \
  do {                               \
    xatu_status s__ = (x);           \
    if (s__ != XATU_OK) return s__;  \
  } while (0)

// Row-tile height for a kernel whose shared memory is smem(TR): 64 rows while that fits in 100 KB, else the
// largest of 32 / 16 (min_tr at least) within 200 KB.
template <typename F>
static int ts_pick_tile(F smem, int min_tr) {
  if (smem(64) <= 100 * 1024) return 64;
  if (smem(32) <= 200 * 1024 || min_tr >= 32) return 32;
  return 16;
}

static xatu_status ts_part_ensure(xatu_ctx* ctx, size_t bytes) {
  if (ctx->dv_part.bytes < bytes) XATU_CK(ctx->dv_part.ensure(bytes));
  return XATU_OK;
}

// Z[0:a, 0:b] (leading dimension ldz) = A[:, 0:a]^H B[:, 0:b] over N rows: per-tile partials, then their
// ordered sum.  status_out (may be NULL) gets a copy of the device status word.
static xatu_status ts_proj(xatu_ctx* ctx, const cd* A, int a, const cd* B, int b, long long N, cd* Z, int ldz,
                           double* status_out = nullptr) {
  if (a <= 0 || b <= 0) return XATU_OK;
  const int TR = ts_pick_tile([&](int tr) { return ts_proj_smem(a, b, tr); }, 16);
  const int G = (int)((N + TR - 1) / TR);
  const int ab = a * b;
  XATU_TRY(ts_part_ensure(ctx, (size_t)G * ab * sizeof(cd)));
  XATU_CHAIN(ts_proj_kernel, G, TS_THREADS, ts_proj_smem(a, b, TR), A, a, B, b, N, TR, ctx->dv_part.as<cd>());
  XATU_CHAIN(ts_sum_kernel, (ab + 31) / 32, TS_SUM_THREADS, 0, ctx->dv_part.as<cd>(), G, ab, a, Z, ldz,
             ctx->d_status.as<int>(), status_out);
  return XATU_OK;
}

// Out[:, 0:b] = (In[:, 0:b] - A[:, 0:a] C) S over N rows (A NULL: no projection; S NULL: identity).
static xatu_status ts_update(xatu_ctx* ctx, const cd* In, int b, const cd* A, int a, const cd* C, int ldc,
                             const cd* S, cd* Out, long long N) {
  const int TR = ts_pick_tile([&](int tr) { return ts_update_smem(a, b, tr); }, 16);
  const int G = (int)((N + TR - 1) / TR);
  XATU_CHAIN(ts_update_kernel, G, TS_THREADS, ts_update_smem(a, b, TR), In, b, A, a, C, ldc, S, Out, N, TR);
  return XATU_OK;
}

// Out = (In - A C) S (ts_update), then Z[0 : pa + b, 0 : b] = [A[:, 0:pa], Out]^H Out from the same row tiles.
static xatu_status ts_update_proj(xatu_ctx* ctx, const cd* In, int b, const cd* A, int a, const cd* C, int ldc,
                                  const cd* S, cd* Out, long long N, int pa, cd* Z, int ldz) {
  const int TR = ts_pick_tile([&](int tr) { return ts_update_smem(a, b, tr); }, 16);
  const int G = (int)((N + TR - 1) / TR);
  const int ab = (pa + b) * b;
  XATU_TRY(ts_part_ensure(ctx, (size_t)G * ab * sizeof(cd)));
  XATU_CHAIN(ts_update_proj_kernel, G, TS_THREADS, ts_update_smem(a, b, TR), In, b, A, a, C, ldc, S, Out, N, TR, pa,
             ctx->dv_part.as<cd>());
  XATU_CHAIN(ts_sum_kernel, (ab + 31) / 32, TS_SUM_THREADS, 0, ctx->dv_part.as<cd>(), G, ab, pa + b, Z, ldz,
             ctx->d_status.as<int>(), static_cast<double*>(nullptr));
  return XATU_OK;
}

// Orthonormalise the block t = V[:, m : m + nsel] against V[:, 0 : m] and within itself:
//   t <- t - V (V^H t);
//   Z = [V t]^H t: C = V^H t, G = t^H t - C^H C; Cholesky of G with dropping -> S;  X = (t - V C) S;
//   G = X^H X -> S (second Cholesky pass, absolute threshold);  t <- X S.
// The kept directions end in V[:, m : m + kept] and the rest of the block is zero; kept stays on the device
// (dav_dead_kernel of the next step parks the zero columns and hands the count to the host's read-back).
static xatu_status orthonormalize_block(xatu_ctx* ctx, long long N, int m, int nsel) {
  cd* V = ctx->dv_V.as<cd>();
  cd* t = V + (long long)m * N;
  cd* X = ctx->dv_tmp.as<cd>();
  cd* Z = ctx->dv_G.as<cd>();
  const int ldZ = DAV_MAX_BASIS;
  cd* S = Z + (size_t)DAV_MAX_BASIS * DAV_MAX_BASIS / 2;   // nsel x nsel (nsel <= DAV_MAX_BASIS / 2)
  int* dkept = reinterpret_cast<int*>(ctx->dv_norm.as<double>() + 1024);
  if (m > 0) {
    // t <- t - V (V^H t), and Z = [V t]^H t from the updated row tiles
    XATU_TRY(ts_proj(ctx, V, m, t, nsel, N, Z, ldZ));
    XATU_TRY(ts_update_proj(ctx, t, nsel, V, m, Z, ldZ, nullptr, t, N, m, Z, ldZ));
  } else {
    XATU_TRY(ts_proj(ctx, t, nsel, t, nsel, N, Z, ldZ));
  }
  XATU_CHAIN(ts_gram_orth_kernel, 1, 32, ts_gram_orth_smem(m, nsel), Z, ldZ, m, nsel, 1e-20, S, dkept);
  // X = (t - V Z[0:m]) S, and Z = X^H X from the same row tiles
  XATU_TRY(ts_update_proj(ctx, t, nsel, m > 0 ? V : nullptr, m, Z, ldZ, S, X, N, 0, Z, ldZ));
  XATU_CHAIN(ts_gram_orth_kernel, 1, 32, ts_gram_orth_smem(0, nsel), Z, ldZ, 0, nsel, 1e-24, S, dkept);
  XATU_TRY(ts_update(ctx, X, nsel, nullptr, 0, nullptr, 0, S, t, N));
  return XATU_OK;
}

xatu_status xatu_davidson_solve(xatu_ctx* ctx, int nstates, double* eigval, double* eigvec) {
  const long long N = ctx->N;
  if (!ctx->blas) {
    if (cublasCreate(&ctx->blas) != CUBLAS_STATUS_SUCCESS) return xatu_fail(ctx, XATU_ERR_CUDA, "cublasCreate failed");
  }
  cublasSetStream(ctx->blas, ctx->stream);
  cublasSetPointerMode(ctx->blas, CUBLAS_POINTER_MODE_HOST);
  const bool mixed = ctx->built_prec == XATU_PREC_MIXED;
  // block = nstates plus guard vectors (two, or an eighth of the states when more), so that a state of a dense
  // spectrum cannot drop out of the block unnoticed while every residual of the block looks converged; only
  // the first nstates must converge.  The basis holds at most 4 blocks.
  int bsz = ctx->dav_block > 0 ? ctx->dav_block : std::max(8, nstates + std::max(2, (nstates + 7) / 8));
  bsz = std::max(bsz, nstates);
  bsz = (int)std::min<long long>(bsz, N);
  int mmax = (int)std::min<long long>(N, std::min(DAV_MAX_BASIS, 4 * bsz));
  if (mmax < bsz + 1 && N > bsz) mmax = std::min<long long>(N, bsz + 1);
  if (bsz > DAV_MAX_BASIS / 2 && N > DAV_MAX_BASIS)
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "Davidson block too large (nstates > 56)");
  const double tol = ctx->dav_tol > 0 ? ctx->dav_tol : (mixed ? 1e-4 : 1e-6);
  const size_t vbytes = (size_t)N * mmax * sizeof(cd);
  XATU_CK(ctx->dv_V.ensure(vbytes));
  XATU_CK(ctx->dv_W.ensure(vbytes));
  XATU_CK(ctx->dv_R.ensure((size_t)N * bsz * sizeof(cd)));
  if (!ctx->h_small) XATU_CK(cudaMallocHost(&ctx->h_small, 8192));
  XATU_CK(ctx->dv_U.ensure((size_t)2 * N * bsz * sizeof(cd)));
  XATU_CK(ctx->dv_tmp.ensure((size_t)N * mmax * sizeof(cd)));
  XATU_CK(ctx->dv_T.ensure((size_t)DAV_MAX_BASIS * DAV_MAX_BASIS * sizeof(cd) * 3 + 4096));
  XATU_CK(ctx->dv_G.ensure((size_t)DAV_MAX_BASIS * DAV_MAX_BASIS * sizeof(cd)));
  XATU_CK(ctx->dv_diagH.ensure((size_t)N * sizeof(double)));
  XATU_CK(ctx->dv_norm.ensure(4096 * sizeof(double)));
  cd* V = ctx->dv_V.as<cd>();
  cd* W = ctx->dv_W.as<cd>();
  cd* P = ctx->dv_R.as<cd>();                           // preconditioned residuals (N x bsz)
  cd* U = ctx->dv_U.as<cd>();                           // Ritz vectors V Y (N x bsz)
  cd* WU = U + (size_t)N * bsz;                         // W Y
  const int ldT = DAV_MAX_BASIS;
  cd* T = ctx->dv_T.as<cd>();                           // projected matrix V^H H V (ldT x ldT)
  cd* Yr = T + (size_t)ldT * ldT;                       // Ritz coefficients (ldT x bsz)
  cd* refl = Yr + (size_t)ldT * ldT;                    // reflectors of the small eigensolver
  double* theta = ctx->dv_norm.as<double>();            // [0, 256)
  double* norms = theta + 256;                          // [256, 512)
  int* sel_dev = reinterpret_cast<int*>(theta + 512);   // ints
  int* dkept = reinterpret_cast<int*>(theta + 1024);    // kept columns of the newest block (ts_gram_orth_kernel)
  double* diagH = ctx->dv_diagH.as<double>();
  const int threads = 256;
  // diagonal of H
  {
    const int blocks = (int)((N + threads - 1) / threads);
    if (mixed)
      dav_diag_mixed_kernel<<<blocks, threads, 0, ctx->stream>>>(ctx->d_Khi.as<__nv_bfloat162>(),
                                                                 ctx->d_Klo.as<__nv_bfloat162>(),
                                                                 ctx->d_diag.as<double>(), N, ctx->ldk, diagH);
    else
      dav_diag_fp64_kernel<<<blocks, threads, 0, ctx->stream>>>(ctx->d_H.as<cd>(), N, diagH);
    ctx->launches++;
    XATU_CK(cudaGetLastError());
  }
  // start columns: the bsz lowest diagonal entries, chosen on the device (no host round trip)
  {
    const size_t sel_smem = N <= DAV_SEL_SMEM_ROWS ? (size_t)N * sizeof(double) : 0;
    XATU_CK(xatu_raise_smem_limit((const void*)dav_select_lowest_kernel, DAV_SEL_SMEM_ROWS * sizeof(double)));
    dav_select_lowest_kernel<<<1, DAV_SEL_THREADS, sel_smem, ctx->stream>>>(
        diagH, N, bsz, reinterpret_cast<double*>(ctx->dv_tmp.p), sel_dev, dkept);
  }
  ctx->launches++;
  XATU_CK(cudaGetLastError());
  {
    // unit vectors of the lowest diagonal entries plus noise of norm ~1e-3 per column, orthonormalised below
    // (enough to seed every symmetry sector; larger noise costs Davidson steps to remove again)
    const long long tot = N * bsz;
    const double noise = N > bsz ? 1e-3 * std::sqrt(3.0 / (double)N) : 0.0;
    dav_start_vectors_kernel<<<(int)((tot + threads - 1) / threads), threads, 0, ctx->stream>>>(V, N, 0, sel_dev, bsz,
                                                                                                noise);
    ctx->launches++;
    XATU_CK(cudaGetLastError());
  }
  XATU_CK(xatu_raise_smem_limit((const void*)dav_heev_kernel, heev_smem_bytes(DAV_MAX_BASIS, DAV_MAX_BASIS / 2)));
  {
    const int bmax = DAV_MAX_BASIS / 2;
    XATU_CK(xatu_raise_smem_limit((const void*)ts_proj_kernel, 224 * 1024));
    XATU_CK(xatu_raise_smem_limit((const void*)ts_update_kernel, 224 * 1024));
    XATU_CK(xatu_raise_smem_limit((const void*)ts_update_proj_kernel, 224 * 1024));
    XATU_CK(xatu_raise_smem_limit((const void*)ts_ritz_kernel, 224 * 1024));
    XATU_CK(xatu_raise_smem_limit((const void*)ts_gram_orth_kernel, ts_gram_orth_smem(DAV_MAX_BASIS - bmax, bmax)));
  }
  if (N > bsz) XATU_TRY(orthonormalize_block(ctx, N, 0, bsz));

  // Thick-restart block Davidson on the basis V (W = H V):
  //   T[:, new] = V^H W[:, new] (the old block of T is kept);  lowest nritz Ritz pairs of T;
  //   U = V Y, WU = W Y, residuals WU - U theta;  corrections appended after orthonormalisation;
  //   restart: V <- U, W <- WU, T <- diag(theta).
  int m0 = 0, m = bsz;
  int dead = 0;   // zero columns in V[:, 0 : m] (directions the orthonormalisation dropped)
  int it = 0;
  bool converged = false;
  std::vector<double> h_theta(ldT), h_norm(bsz);
  const auto t_start = std::chrono::steady_clock::now();
  const double wall_cap_s = 300.0;
  ctx->dav_iters = 0;
  ctx->dav_maxres = 0;
  ctx->hx_calls = 0;
  ctx->hx_ms = 0;
  ctx->hx_pending = false;
  for (it = 0; it < ctx->dav_max_iter; it++) {
    const int nnew = m - m0;
    // 1. W for the new columns
    XATU_TRY(xatu_apply_h(ctx, N, m0, nnew));
    // 2. new columns of T = V^H W
    XATU_TRY(ts_proj(ctx, V, m, W + (long long)m0 * N, nnew, N, T + (long long)m0 * ldT, ldT));
    {
      const int tot = nnew * m;
      XATU_CHAIN(dav_hermitize_kernel, (tot + 127) / 128, 128, 0, T, ldT, m, m0);
      XATU_CHAIN(dav_dead_kernel, 1, 128, 0, T, ldT, m, m0, dkept, theta + 769);
    }
    // 3. Rayleigh-Ritz: the lowest nritz eigenpairs of T
    const int nritz = std::min(bsz, m);
    XATU_CHAIN(dav_heev_kernel, 1, HEEV_THREADS, heev_smem_bytes(m, nritz), T, ldT, m, nritz, theta, Yr, ldT, refl,
               ctx->d_status.as<int>(), nullptr);
    // 4. Ritz vectors and residuals
    {
      const int TR = ts_ritz_smem(m, nritz, 64) <= 100 * 1024 ? 64 : 32;
      const int G = (int)((N + TR - 1) / TR);
      XATU_TRY(ts_part_ensure(ctx, (size_t)G * nritz * sizeof(cd)));
      XATU_CHAIN(ts_ritz_kernel, G, TS_THREADS, ts_ritz_smem(m, nritz, TR), V, W, m, Yr, ldT, nritz, theta, diagH, N,
                 TR, U, WU, P, ctx->dv_part.as<cd>());
      // squared residual norms as complex pairs at [256, 256 + 2 nritz), the status word at 768
      XATU_CHAIN(ts_sum_kernel, (nritz + 31) / 32, TS_SUM_THREADS, 0, ctx->dv_part.as<cd>(), G, nritz, nritz,
                 reinterpret_cast<cd*>(norms), 1, ctx->d_status.as<int>(), theta + 768);
    }
    // one read-back: theta [0, 256), residual norms [256, 512), status word at 768, kept columns of the
    // newest block at 769
    XATU_CK(cudaMemcpyAsync(ctx->h_small, theta, 770 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    XATU_CK(cudaStreamSynchronize(ctx->stream));
    xatu_hx_collect(ctx);
    {
      const double* hb = reinterpret_cast<const double*>(ctx->h_small);
      std::copy(hb, hb + nritz, h_theta.begin());
      for (int c = 0; c < nritz; c++) h_norm[c] = std::sqrt(hb[256 + 2 * c]);
    }
    const int st = (int)reinterpret_cast<const double*>(ctx->h_small)[768];
    const int kept_new = (int)reinterpret_cast<const double*>(ctx->h_small)[769];
    dead += (m - m0) - kept_new;   // zero columns of the newest block
    if (st) {
      cudaMemsetAsync(ctx->d_status.p, 0, sizeof(int), ctx->stream);
      return xatu_fail(ctx, XATU_ERR_NOT_CONVERGED, "Davidson: Rayleigh-Ritz or K.X stage reported an error");
    }
    double maxres = 0;
    for (int s = 0; s < nstates; s++) maxres = std::max(maxres, h_norm[s]);
    for (int s = 0; s < nritz; s++)
      if (!std::isfinite(h_norm[s]) || !std::isfinite(h_theta[s]))
        return xatu_fail(ctx, XATU_ERR_NUMERIC, "Davidson: non-finite Ritz value or residual");
    ctx->dav_iters = it + 1;
    ctx->dav_maxres = maxres;
    if (maxres < tol || m - dead >= N) {
      converged = true;
      break;
    }
    if (it > 0 && kept_new == 0) break;   // the last corrections added no direction
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    if (el > wall_cap_s) break;
    // 5. correction targets: unconverged among the lowest Ritz pairs
    std::vector<int> sel;
    for (int s = 0; s < nritz; s++)
      if (h_norm[s] >= tol) sel.push_back(s);
    int nsel = (int)sel.size();
    // 6. thick restart on the Ritz vectors
    if (m + nsel > mmax) {
      XATU_CK(cudaMemcpyAsync(V, U, sizeof(cd) * (size_t)N * nritz, cudaMemcpyDeviceToDevice, ctx->stream));
      XATU_CK(cudaMemcpyAsync(W, WU, sizeof(cd) * (size_t)N * nritz, cudaMemcpyDeviceToDevice, ctx->stream));
      XATU_CHAIN(dav_set_diag_kernel, (nritz * nritz + 127) / 128, 128, 0, T, ldT, nritz, theta);
      m = nritz;
      dead = 0;
      if (m + nsel > mmax) nsel = mmax - m;
    }
    if (nsel <= 0) break;
    XATU_CK(cudaMemcpyAsync(sel_dev, sel.data(), nsel * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    {
      const long long tot = N * nsel;
      XATU_CHAIN(ts_gather_kernel, (int)((tot + threads - 1) / threads), threads, 0, P, sel_dev, nsel, N,
                 V + (long long)m * N);
    }
    XATU_TRY(orthonormalize_block(ctx, N, m, nsel));
    m0 = m;
    m += nsel;   // dropped directions stay as zero columns, parked by dav_dead_kernel
  }
  // results: the Ritz vectors of the last Rayleigh-Ritz step
  std::copy(h_theta.begin(), h_theta.begin() + nstates, eigval);
  if (eigvec)
    XATU_CK(cudaMemcpyAsync(eigvec, U, sizeof(cd) * (size_t)N * nstates, cudaMemcpyDeviceToHost, ctx->stream));
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  if (!converged) {
    char buf[160];
    snprintf(buf, sizeof(buf), "Davidson: not converged after %d iterations (max residual %.3e, tol %.1e)",
             ctx->dav_iters, ctx->dav_maxres, tol);
    return xatu_fail(ctx, XATU_ERR_NOT_CONVERGED, buf);
  }
  return XATU_OK;
}

// Lowest k eigenpairs of a Hermitian matrix given on the host (column-major, m x m) through the device
// solver of the Rayleigh-Ritz step.  Self-test of that solver; allocates and frees its own buffers.
extern "C" xatu_status xatu_selftest_small_eigh(int device, int m, int k, const double* T, double* theta,
                                                double* Y, int64_t* cycles) {
  if (m < 1 || m > HEEV_MAXM || k < 1 || k > m || !T || !theta || !Y) return XATU_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return XATU_ERR_CUDA;
  cd *dT = nullptr, *dY = nullptr, *dR = nullptr;
  double* dth = nullptr;
  int* dst = nullptr;
  long long* dprof = nullptr;
  xatu_status out = XATU_OK;
  const size_t mm = (size_t)m * m * sizeof(cd);
  int hst = 0;
  if (cudaMalloc(&dT, mm) != cudaSuccess || cudaMalloc(&dY, mm) != cudaSuccess || cudaMalloc(&dR, mm) != cudaSuccess ||
      cudaMalloc(&dth, (size_t)m * sizeof(double)) != cudaSuccess || cudaMalloc(&dst, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&dprof, 8 * sizeof(long long)) != cudaSuccess) {
    out = XATU_ERR_CUDA;
  } else {
    const size_t smem = heev_smem_bytes(m, k);
    bool ok = cudaMemcpy(dT, T, mm, cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemset(dst, 0, sizeof(int)) == cudaSuccess &&
              xatu_raise_smem_limit((const void*)dav_heev_kernel, smem) == cudaSuccess;
    if (ok) {
      dav_heev_kernel<<<1, HEEV_THREADS, smem>>>(dT, m, m, k, dth, dY, m, dR, dst, cycles ? dprof : nullptr);
      ok = cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess &&
           cudaMemcpy(theta, dth, (size_t)k * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess &&
           cudaMemcpy(Y, dY, (size_t)m * k * sizeof(cd), cudaMemcpyDeviceToHost) == cudaSuccess &&
           cudaMemcpy(&hst, dst, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess &&
           (!cycles || cudaMemcpy(cycles, dprof, 8 * sizeof(long long), cudaMemcpyDeviceToHost) == cudaSuccess);
    }
    if (!ok) out = XATU_ERR_CUDA;
    else if (hst) out = XATU_ERR_NUMERIC;
  }
  cudaFree(dT);
  cudaFree(dY);
  cudaFree(dR);
  cudaFree(dth);
  cudaFree(dst);
  cudaFree(dprof);
  return out;
}
