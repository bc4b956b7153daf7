// Tall-skinny kernels of the single-system Davidson solver: blocks of N-row
// vectors (column-major, leading dimension N, FP64 complex) against small
// matrices.  Each CTA owns a tile of TS_TILE (or TS_TILE / 2) consecutive rows,
// staged into shared memory with 16-byte cp.async copies that are all in
// flight at once (the blocks are L2-resident; the kernels are bound by load
// latency, not bandwidth).  Reductions over the N rows are deterministic:
// per-tile partial sums, then ts_sum_kernel adds them in tile order.  Every
// kernel starts with xatu_grid_chain(), so that it can be launched chained to
// its predecessor (xatu_launch_chained).
#pragma once
#include "common.cuh"

#define TS_THREADS 256
#define TS_TILE 64          // rows per CTA

// 16-byte asynchronous global -> shared copy; src_bytes = 0 fills zeros (src is then not read).
__device__ __forceinline__ void ts_cp16(void* dst, const void* src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void ts_cp_wait() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Stage rows [row0, row0 + TR) of columns [0, ncols) of X (leading dimension N) into s (row x, column c at
// s[x * lds + c]); rows past N are zero.
__device__ __forceinline__ void ts_stage(cd* s, int lds, const cd* __restrict__ X, int ncols, long long N,
                                         long long row0, int TR) {
  for (int t = threadIdx.x; t < TR * ncols; t += blockDim.x) {
    const int x = t % TR, c = t / TR;
    const bool ok = row0 + x < N;
    ts_cp16(s + x * lds + c, ok ? (const void*)(X + (long long)c * N + row0 + x) : (const void*)X, ok ? 16 : 0);
  }
}

__host__ __device__ inline size_t ts_proj_smem(int a, int b, int TR) { return (size_t)TR * (a + 1 + b + 1) * sizeof(cd); }

// Partial projections of one row tile: part[blockIdx.x][o] = sum over the tile's rows of conj(A[x, r]) B[x, c],
// o = r + c * a (r < a, c < b).  A and B may be the same block.
__global__ void __launch_bounds__(TS_THREADS)
ts_proj_kernel(const cd* __restrict__ A, int a, const cd* __restrict__ B, int b, long long N, int TR,
               cd* __restrict__ part) {
  xatu_grid_chain();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd* sA = reinterpret_cast<cd*>(smem_raw);   // TR x (a + 1)
  cd* sB = sA + TR * (a + 1);                 // TR x (b + 1)
  const long long row0 = (long long)blockIdx.x * TR;
  ts_stage(sA, a + 1, A, a, N, row0, TR);
  ts_stage(sB, b + 1, B, b, N, row0, TR);
  ts_cp_wait();
  __syncthreads();
  const int ab = a * b;
  cd* mine = part + (size_t)blockIdx.x * ab;
  for (int o = threadIdx.x; o < ab; o += TS_THREADS) {
    const int r = o % a, c = o / a;
    double sx0 = 0.0, sy0 = 0.0, sx1 = 0.0, sy1 = 0.0;
#pragma unroll 4
    for (int x = 0; x < TR; x += 2) {
      const cd u0 = sA[x * (a + 1) + r], v0 = sB[x * (b + 1) + c];
      const cd u1 = sA[(x + 1) * (a + 1) + r], v1 = sB[(x + 1) * (b + 1) + c];
      sx0 = fma(u0.x, v0.x, fma(u0.y, v0.y, sx0));
      sy0 = fma(u0.x, v0.y, fma(-u0.y, v0.x, sy0));
      sx1 = fma(u1.x, v1.x, fma(u1.y, v1.y, sx1));
      sy1 = fma(u1.x, v1.y, fma(-u1.y, v1.x, sy1));
    }
    mine[o] = mk(sx0 + sx1, sy0 + sy1);
  }
}

// Z[r + c * ldz] = sum_g part[g][r + c * a] for o = r + c * a < n, the tiles g added in order.  One CTA per
// 32 outputs per CTA of TS_SUM_THREADS: the 32 warps split the tiles g (warp w takes g = w, w + 32, ...; every
// load of a thread is in flight at once), then a fixed-order sum over the warps (deterministic).
// status_out (may be NULL) receives a copy of the device status word, for a single read-back.
#define TS_SUM_THREADS 1024
__global__ void __launch_bounds__(TS_SUM_THREADS)
ts_sum_kernel(const cd* __restrict__ part, int G, int n, int a, cd* __restrict__ Z, int ldz,
              const int* __restrict__ status_in, double* __restrict__ status_out) {
  constexpr int NWS = TS_SUM_THREADS / 32;
  __shared__ double red[NWS][32][2];
  xatu_grid_chain();
  if (status_out && blockIdx.x == 0 && threadIdx.x == 0) *status_out = (double)*status_in;
  const int ol = threadIdx.x & 31, gl = threadIdx.x >> 5;
  const int o = blockIdx.x * 32 + ol;
  double sx = 0.0, sy = 0.0;
  if (o < n) {
    int g = gl;
    for (; g + 7 * NWS < G; g += 8 * NWS) {
      double2 p[8];
#pragma unroll
      for (int u = 0; u < 8; u++) p[u] = __ldcg(reinterpret_cast<const double2*>(part + (size_t)(g + NWS * u) * n + o));
#pragma unroll
      for (int u = 0; u < 8; u++) {
        sx += p[u].x;
        sy += p[u].y;
      }
    }
    for (; g < G; g += NWS) {
      const double2 p = __ldcg(reinterpret_cast<const double2*>(part + (size_t)g * n + o));
      sx += p.x;
      sy += p.y;
    }
  }
  red[gl][ol][0] = sx;
  red[gl][ol][1] = sy;
  __syncthreads();
  if (gl == 0 && o < n) {
    double tx = 0.0, ty = 0.0;
#pragma unroll 8
    for (int q = 0; q < NWS; q++) {
      tx += red[q][ol][0];
      ty += red[q][ol][1];
    }
    Z[(o % a) + (size_t)(o / a) * ldz] = mk(tx, ty);
  }
}

// Out[:, 0:b] = (In[:, 0:b] - A[:, 0:a] C) S  per row tile.  A may be NULL (a = 0: no projection), S may be
// NULL (identity).  C: a x b (leading dimension ldc), S: b x b (leading dimension b).  Out may be In.
__global__ void __launch_bounds__(TS_THREADS)
ts_update_kernel(const cd* In, int b, const cd* __restrict__ A, int a, const cd* __restrict__ C, int ldc,
                 const cd* __restrict__ S, cd* Out, long long N, int TR) {
  xatu_grid_chain();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd* sI = reinterpret_cast<cd*>(smem_raw);   // TR x (b + 1)
  cd* sO = sI + TR * (b + 1);                 // TR x (b + 1): In - A C
  cd* sA = sO + TR * (b + 1);                 // TR x (a + 1)
  cd* sC = sA + TR * (a + 1);                 // a x b row-major
  cd* sS = sC + a * b;                        // b x b row-major
  const long long row0 = (long long)blockIdx.x * TR;
  ts_stage(sI, b + 1, In, b, N, row0, TR);
  if (a > 0) ts_stage(sA, a + 1, A, a, N, row0, TR);
  for (int t = threadIdx.x; t < a * b; t += TS_THREADS) {
    const int r = t / b, c = t - r * b;
    sC[t] = C[r + (size_t)c * ldc];
  }
  if (S)
    for (int t = threadIdx.x; t < b * b; t += TS_THREADS) {
      const int r = t / b, c = t - r * b;
      sS[t] = S[r + (size_t)c * b];
    }
  ts_cp_wait();
  __syncthreads();
  const cd* src = sI;
  if (a > 0) {
    for (int t = threadIdx.x; t < TR * b; t += TS_THREADS) {
      const int x = t % TR, c = t / TR;
      cd s = sI[x * (b + 1) + c];
#pragma unroll 4
      for (int r = 0; r < a; r++) s = s - sA[x * (a + 1) + r] * sC[r * b + c];
      sO[x * (b + 1) + c] = s;
    }
    __syncthreads();
    src = sO;
  }
  for (int t = threadIdx.x; t < TR * b; t += TS_THREADS) {
    const int x = t % TR, c = t / TR;
    const long long i = row0 + x;
    if (i >= N) continue;
    cd v;
    if (S) {
      v = mk(0, 0);
#pragma unroll 4
      for (int r = 0; r < b; r++) v = v + src[x * (b + 1) + r] * sS[r * b + c];
    } else {
      v = src[x * (b + 1) + c];
    }
    Out[(long long)c * N + i] = v;
  }
}

__host__ __device__ inline size_t ts_update_smem(int a, int b, int TR) {
  return ((size_t)2 * TR * (b + 1) + (size_t)TR * (a + 1) + (size_t)a * b + (size_t)b * b) * sizeof(cd);
}

// ts_update_kernel fused with the projection that follows it in the orthonormalisation: Out = (In - A C) S per row
// tile as above, then the tile's partial of [A[:, 0:pa], Out]^H Out from the rows still in shared memory
// (pa = a or 0): part[tile][r + c (pa + b)], r < pa + b, c < b (added in tile order by ts_sum_kernel).
// Shared memory: ts_update_smem(a, b, TR).
__global__ void __launch_bounds__(TS_THREADS)
ts_update_proj_kernel(const cd* In, int b, const cd* __restrict__ A, int a, const cd* __restrict__ C, int ldc,
                      const cd* __restrict__ S, cd* Out, long long N, int TR, int pa, cd* __restrict__ part) {
  xatu_grid_chain();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd* sI = reinterpret_cast<cd*>(smem_raw);   // TR x (b + 1)
  cd* sO = sI + TR * (b + 1);                 // TR x (b + 1): In - A C
  cd* sA = sO + TR * (b + 1);                 // TR x (a + 1)
  cd* sC = sA + TR * (a + 1);                 // a x b row-major
  cd* sS = sC + a * b;                        // b x b row-major
  const long long row0 = (long long)blockIdx.x * TR;
  ts_stage(sI, b + 1, In, b, N, row0, TR);
  if (a > 0) ts_stage(sA, a + 1, A, a, N, row0, TR);
  for (int t = threadIdx.x; t < a * b; t += TS_THREADS) {
    const int r = t / b, c = t - r * b;
    sC[t] = C[r + (size_t)c * ldc];
  }
  if (S)
    for (int t = threadIdx.x; t < b * b; t += TS_THREADS) {
      const int r = t / b, c = t - r * b;
      sS[t] = S[r + (size_t)c * b];
    }
  ts_cp_wait();
  __syncthreads();
  const cd* src = sI;
  if (a > 0) {
    for (int t = threadIdx.x; t < TR * b; t += TS_THREADS) {
      const int x = t % TR, c = t / TR;
      cd s = sI[x * (b + 1) + c];
#pragma unroll 4
      for (int r = 0; r < a; r++) s = s - sA[x * (a + 1) + r] * sC[r * b + c];
      sO[x * (b + 1) + c] = s;
    }
    __syncthreads();
    src = sO;
  }
  cd* sF = a > 0 ? sI : sO;   // the tile of Out (rows past N are zero, as the staged rows are)
  for (int t = threadIdx.x; t < TR * b; t += TS_THREADS) {
    const int x = t % TR, c = t / TR;
    const long long i = row0 + x;
    cd v;
    if (S) {
      v = mk(0, 0);
#pragma unroll 4
      for (int r = 0; r < b; r++) v = v + src[x * (b + 1) + r] * sS[r * b + c];
    } else {
      v = src[x * (b + 1) + c];
    }
    sF[x * (b + 1) + c] = v;
    if (i < N) Out[(long long)c * N + i] = v;
  }
  __syncthreads();
  const int na = pa + b, ab = na * b;
  cd* mine = part + (size_t)blockIdx.x * ab;
  for (int o = threadIdx.x; o < ab; o += TS_THREADS) {
    const int r = o % na, c = o / na;
    const cd* u = r < pa ? sA + r : sF + (r - pa);
    const int us = r < pa ? a + 1 : b + 1;
    double sx0 = 0.0, sy0 = 0.0, sx1 = 0.0, sy1 = 0.0;
#pragma unroll 4
    for (int x = 0; x < TR; x += 2) {
      const cd u0 = u[x * us], v0 = sF[x * (b + 1) + c];
      const cd u1 = u[(x + 1) * us], v1 = sF[(x + 1) * (b + 1) + c];
      sx0 = fma(u0.x, v0.x, fma(u0.y, v0.y, sx0));
      sy0 = fma(u0.x, v0.y, fma(-u0.y, v0.x, sy0));
      sx1 = fma(u1.x, v1.x, fma(u1.y, v1.y, sx1));
      sy1 = fma(u1.x, v1.y, fma(-u1.y, v1.x, sy1));
    }
    mine[o] = mk(sx0 + sx1, sy0 + sy1);
  }
}

// Ritz vectors and preconditioned residuals of the lowest k Ritz pairs, per row tile (TR a multiple of 32):
//   U = V Y, WU = W Y (V, W: N x m; Y: m x k, leading dimension ldy),
//   r_c = WU_c - theta_c U_c,  P_c = r_c / (theta_c - H_ii)  (|denominator| >= 1e-8),
//   part[blockIdx.x][c] = sum over the tile's rows of |r_c|^2 (as the real part of a complex partial).
__global__ void __launch_bounds__(TS_THREADS)
ts_ritz_kernel(const cd* __restrict__ V, const cd* __restrict__ W, int m, const cd* __restrict__ Y, int ldy, int k,
               const double* __restrict__ theta, const double* __restrict__ diagH, long long N, int TR,
               cd* __restrict__ U, cd* __restrict__ WU, cd* __restrict__ P, cd* __restrict__ part) {
  xatu_grid_chain();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd* sV = reinterpret_cast<cd*>(smem_raw);   // TR x (m + 1)
  cd* sW = sV + TR * (m + 1);                 // TR x (m + 1)
  cd* sY = sW + TR * (m + 1);                 // m x k row-major
  const int rgroups = TR / 32;                // warps per column
  double* red = reinterpret_cast<double*>(sY + m * k);   // k x rgroups
  const long long row0 = (long long)blockIdx.x * TR;
  ts_stage(sV, m + 1, V, m, N, row0, TR);
  ts_stage(sW, m + 1, W, m, N, row0, TR);
  for (int t = threadIdx.x; t < m * k; t += TS_THREADS) {
    const int r = t / k, c = t - r * k;
    sY[t] = Y[r + (size_t)c * ldy];
  }
  ts_cp_wait();
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int cw = warp; cw < rgroups * k; cw += TS_THREADS / 32) {
    const int c = cw / rgroups, g = cw - c * rgroups, x = g * 32 + lane;
    const long long i = row0 + x;
    cd u = mk(0, 0), w = mk(0, 0);
#pragma unroll 4
    for (int r = 0; r < m; r++) {
      const cd y = sY[r * k + c];
      u = u + sV[x * (m + 1) + r] * y;
      w = w + sW[x * (m + 1) + r] * y;
    }
    double n2 = 0.0;
    if (i < N) {
      const double th = theta[c];
      const cd rr = mk(w.x - th * u.x, w.y - th * u.y);
      n2 = nrm2(rr);
      double den = th - diagH[i];
      if (fabs(den) < 1e-8) den = (den < 0 ? -1e-8 : 1e-8);
      const double rd = 1.0 / den;
      U[(long long)c * N + i] = u;
      WU[(long long)c * N + i] = w;
      P[(long long)c * N + i] = mk(rr.x * rd, rr.y * rd);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n2 += __shfl_xor_sync(0xffffffffu, n2, o);
    if (lane == 0) red[c * rgroups + g] = n2;
  }
  __syncthreads();
  for (int c = threadIdx.x; c < k; c += TS_THREADS) {
    double s = 0.0;
    for (int g = 0; g < rgroups; g++) s += red[c * rgroups + g];
    part[(size_t)blockIdx.x * k + c] = mk(s, 0.0);
  }
}

__host__ __device__ inline size_t ts_ritz_smem(int m, int k, int TR) {
  return ((size_t)2 * TR * (m + 1) + (size_t)m * k) * sizeof(cd) + (size_t)k * (TR / 32) * sizeof(double);
}

// Dst[:, j] = Src[:, sel[j]], j < nsel.
__global__ void ts_gather_kernel(const cd* __restrict__ Src, const int* __restrict__ sel, int nsel, long long N,
                                 cd* __restrict__ Dst) {
  xatu_grid_chain();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= N * nsel) return;
  const int j = (int)(t / N);
  const long long i = t - (long long)j * N;
  Dst[t] = Src[(long long)sel[j] * N + i];
}

// Orthonormaliser of a block t from its Gram matrix.  Z (leading dimension ldz) holds [C; Gt] with
// C = V^H t (rows 0 .. m-1, m may be 0) and Gt = t^H t (rows m .. m+b-1); G = Gt - C^H C is the Gram matrix
// of t - V C.  Cholesky G = L L^H without pivoting, a column dropped (left out of L) when its remaining pivot
// is <= drop * max_i G_ii: Gram-Schmidt of the columns in order, keeping a column when its component
// orthogonal to the kept ones is large enough.  With L_k the factor of the kept columns, S = P L_k^{-H}
// (P places the kept rows), so (t - V C) S has orthonormal columns: the kept directions in S's first
// columns, zero columns after them; *kept = their number.  One warp.
__global__ void __launch_bounds__(32)
ts_gram_orth_kernel(const cd* __restrict__ Z, int ldz, int m, int b, double drop, cd* __restrict__ S,
                    int* __restrict__ kept) {
  xatu_grid_chain();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd* A = reinterpret_cast<cd*>(smem_raw);        // b x b row-major, lower triangle -> L
  cd* M = A + b * b;                              // L_k^{-1}, row-major
  cd* Zs = M + b * b;                             // Z[0 : m + b, 0 : b], column-major (ld m + b)
  double* rdg = reinterpret_cast<double*>(Zs + (size_t)(m + b) * b);   // 1 / L_ii of the kept columns
  int* idx = reinterpret_cast<int*>(rdg + b);                            // kept column indices
  const int lane = threadIdx.x;
  const int mz = m + b;
  // stage the block of Z (coalesced along each column), eight loads per lane in flight before their stores so
  // that the warp waits for L2 once per batch, then G = Z[m:, :] - Z[:m, :]^H Z[:m, :] from shared memory
  const int tot = mz * b;
  for (int t0 = 0; t0 < tot; t0 += 8 * 32) {
    cd v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int t = t0 + u * 32 + lane;
      if (t < tot) v[u] = Z[t % mz + (size_t)(t / mz) * ldz];
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int t = t0 + u * 32 + lane;
      if (t < tot) Zs[t] = v[u];
    }
  }
  __syncwarp();
  for (int t = lane; t < b * b; t += 32) {
    const int r = t / b, c = t - r * b;
    cd g = Zs[(m + r) + c * mz];
    const cd* zr = Zs + r * mz;
    const cd* zc = Zs + c * mz;
    for (int q = 0; q < m; q++) g = g - cmulc(zr[q], zc[q]);
    A[t] = g;
  }
  __syncwarp();
  double maxd = 0.0;
  for (int r = lane; r < b; r += 32) maxd = fmax(maxd, A[r * b + r].x);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) maxd = fmax(maxd, __shfl_xor_sync(0xffffffffu, maxd, o));
  const double thr = drop * maxd;
  int nk = 0;
  for (int c = 0; c < b; c++) {
    const double piv = A[c * b + c].x;
    const bool keep = piv > thr && piv > 0.0;
    if (keep) {
      const double lc = sqrt(piv), rl = 1.0 / lc;
      for (int r = c + 1 + lane; r < b; r += 32) A[r * b + c] = rl * A[r * b + c];
      __syncwarp();
      const int w = b - c - 1;
      for (int t = lane; t < w * w; t += 32) {
        const int r = c + 1 + t / w, q = c + 1 + t % w;
        if (q <= r) A[r * b + q] = A[r * b + q] - A[r * b + c] * conj(A[q * b + c]);
      }
      if (lane == 0) {
        A[c * b + c] = mk(lc, 0.0);
        idx[nk] = c;
      }
      nk++;
    }
    __syncwarp();
  }
  // M = L_k^{-1} (lower triangular, nk x nk): lane j solves column j by forward substitution, with the
  // reciprocal pivots formed once per kept column instead of once per (row, column) pair
  for (int i = lane; i < nk; i += 32) rdg[i] = 1.0 / A[idx[i] * b + idx[i]].x;
  __syncwarp();
  for (int j = lane; j < nk; j += 32) {
    for (int i = 0; i < nk; i++) M[i * b + j] = mk(0, 0);
    M[j * b + j] = mk(rdg[j], 0.0);
    for (int i = j + 1; i < nk; i++) {
      cd sum = mk(0, 0);
      for (int l = j; l < i; l++) sum = sum + A[idx[i] * b + idx[l]] * M[l * b + j];
      const double rd = rdg[i];
      M[i * b + j] = mk(-sum.x * rd, -sum.y * rd);
    }
  }
  __syncwarp();
  // S[idx[i], c] = conj(M[c][i]) for c >= i (S = P L_k^{-H}); everything else zero
  for (int t = lane; t < b * b; t += 32) {
    const int r = t % b, c = t / b;
    cd v = mk(0, 0);
    if (c < nk) {
      for (int i = 0; i <= c; i++)
        if (idx[i] == r) v = conj(M[c * b + i]);
    }
    S[t] = v;
  }
  if (lane == 0) *kept = nk;
}

__host__ __device__ inline size_t ts_gram_orth_smem(int m, int b) {
  return (size_t)(2 * b * b + (m + b) * b) * sizeof(cd) + (size_t)b * (sizeof(double) + sizeof(int));
}
