// Batched build + solve of many BSE instances of uneven size (k grids, band
// windows, dielectric parameters) on one GPU.
//
// Members are ordinary contexts (system, exciton parameters, device buffers);
// the batch runs their stages back to back on one stream and records them in
// two CUDA graphs:
//   * the build graph: per-system band solves and interaction tables, then ONE
//     persistent assembly launch per band-window class (nv, nc, natoms) over a
//     device work list of (system, tile) items taken through an atomic
//     counter, largest systems first; the tile size of each class is chosen by
//     the autotuner (timed candidates on the batch's own data, first run);
//   * the solve graph: a conditional WHILE node whose body is one step of a
//     block Davidson run in lockstep for all systems, with every decision taken
//     on the device (Rayleigh-Ritz, restart, convergence, orthonormalisation);
//     a one-thread kernel at the end of the body counts the step and sets the
//     loop condition (systems still active, iteration cap), so the whole solve
//     is one graph launch with no host round trip per step.  Converged systems
//     skip their work, the tcgen05 K.X product included.
//
// Davidson step of one system (basis V, W = H V, projected matrix T = V^H W
// grown by the new columns only; block P of at most BD_MAXB new directions):
//   W_P = H P (split-BF16 K on tcgen05 + FP64 band diagonal);  append P, W_P;
//   T[:, new] = V^H W_P;  lowest block of Ritz pairs of T (eigh_small.cuh);
//   U = V Y, WU = W Y (block columns only);
//   r_j = WU_j - theta_j U_j,  P_j = r_j / (theta_j - H_jj)  (j < block);
//   converged when max_{j < nstates} |r_j| < tol;
//   restart (basis full): V <- U, W <- WU, T <- diag(theta);
//   P orthonormalised (eigen-decomposition of its Gram matrix), projected out of
//   V twice (classical Gram-Schmidt), orthonormalised again; directions whose
//   norm falls below the threshold are dropped.
// The reference solves one system at a time (davidson.cpp:5-60, ExcitonTB.cpp:930-959).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "eigh_small.cuh"
#include "engine.h"
#include "jacobi.cuh"
#include "kernels.h"

#define BD_ROWS 64            // rows per chunk of the row kernels (one thread per row)
#define BD_RED_ROWS 512       // rows per chunk of the reduction kernels
#define BD_SUB 16             // rows staged per pass of a reduction
#define BD_MAXB 16            // largest Davidson block
#define BD_BASIS_BLOCKS 6     // basis limit in blocks (restart beyond it)
#define BD_MMAX (BD_BASIS_BLOCKS * BD_MAXB)   // largest basis
#define BD_EIGH_THREADS 256
#define BD_RR_THREADS HEEV_THREADS

struct BDav {
  long long N, ldk, ldb, ldu;
  const __nv_bfloat162* Khi;
  const __nv_bfloat162* Klo;
  const double* diag;       // FP64 band-energy diagonal
  double* diagH;            // diagonal of H
  cd* V;                    // N x mmax, column-major
  cd* W;
  cd* P;                    // N x BD_MAXB
  cd* U;                    // N x BD_MAXB: Ritz vectors of the block
  cd* WU;                   // N x BD_MAXB: W Y
  cd* T;                    // mmax x mmax (ld BD_MMAX), both triangles
  cd* Y;                    // mmax x BD_MAXB (ld BD_MMAX): Ritz coefficients
  cd* R;                    // mmax x mmax: reflector scratch of the Rayleigh-Ritz eigensolver
  cd* C1;                   // BD_MMAX x BD_MAXB (ld BD_MMAX)
  cd* C2;
  cd* G1;                   // BD_MAXB x BD_MAXB (ld BD_MAXB)
  cd* G2;
  cd* S;                    // BD_MAXB x BD_MAXB
  double* theta;            // BD_MMAX
  double* norms;            // BD_MAXB
  float* Yf;                // N x 2 bp, row-major (tcgen05 output)
  __nv_bfloat16* Bhi;       // 2 bp x ldb: operand along the interleaved columns of K
  __nv_bfloat16* Blo;
  __nv_bfloat16* Uhi;       // 2 bp x ldu: operand along the rows of K
  __nv_bfloat16* Ulo;
  int m, k, active, iters, stalled, kmask, restart;
};

struct BDGlobal {
  int nmem;
  int bsz;                  // block size
  int bp;                   // bsz rounded up to 8
  int mmax;
  int nstates;
  int max_iter;
  double tol;
};

__device__ __forceinline__ int bd_member(const int* __restrict__ off, int nmem, int chunk) {
  int lo = 0, hi = nmem - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= chunk) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// ------------------------------------------------------------------ row kernels (one thread per row)
__global__ void __launch_bounds__(BD_ROWS) bd_diag_kernel(BDGlobal g, BDav* D, const int* __restrict__ off) {
  const int mem = bd_member(off, g.nmem, blockIdx.x);
  const BDav& d = D[mem];
  const long long i = (long long)(blockIdx.x - off[mem]) * BD_ROWS + threadIdx.x;
  if (i >= d.N) return;
  d.diagH[i] = d.diag[i] + (double)__bfloat162float(d.Khi[i * d.ldk + i].x) +
               (double)__bfloat162float(d.Klo[i * d.ldk + i].x);
}

// Bt operand of the tensor-core product from P (as dav_build_bt_kernel).
__global__ void __launch_bounds__(BD_ROWS) bd_build_bt_kernel(BDGlobal g, BDav* D, const int* __restrict__ off) {
  const int mem = bd_member(off, g.nmem, blockIdx.x);
  const BDav& d = D[mem];
  if (!d.active) return;
  const long long j = (long long)(blockIdx.x - off[mem]) * BD_ROWS + threadIdx.x;
  if (j >= d.N) return;
  for (int s = 0; s < g.bp; s++) {
    float re = 0.f, im = 0.f;
    if (s < g.bsz) {
      const cd v = d.P[(long long)s * d.N + j];
      re = (float)v.x;
      im = (float)v.y;
    }
    // the operand layouts of the tcgen05 product (hx_tc.cu): Bt along the interleaved columns, Bu along rows
    const float vals[6] = {re, -im, im, re, re, im};
    const long long o[6] = {(long long)s * d.ldb + 2 * j, (long long)s * d.ldb + 2 * j + 1,
                            (long long)(g.bp + s) * d.ldb + 2 * j, (long long)(g.bp + s) * d.ldb + 2 * j + 1,
                            (long long)s * d.ldu + j, (long long)(g.bp + s) * d.ldu + j};
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const __nv_bfloat16 h = __float2bfloat16_rn(vals[q]);
      const __nv_bfloat16 l = __float2bfloat16_rn(vals[q] - __bfloat162float(h));
      if (q < 4) {
        d.Bhi[o[q]] = h;
        d.Blo[o[q]] = l;
      } else {
        d.Uhi[o[q]] = h;
        d.Ulo[o[q]] = l;
      }
    }
  }
}

// W_P = Y + diag .* P, then append P and W_P to the basis at column m.
__global__ void __launch_bounds__(BD_ROWS) bd_finish_append_kernel(BDGlobal g, BDav* D, const int* __restrict__ off) {
  const int mem = bd_member(off, g.nmem, blockIdx.x);
  const BDav& d = D[mem];
  if (!d.active) return;
  const long long i = (long long)(blockIdx.x - off[mem]) * BD_ROWS + threadIdx.x;
  if (i >= d.N) return;
  const double di = d.diag[i];
  for (int s = 0; s < d.k; s++) {
    const cd p = d.P[(long long)s * d.N + i];
    const float* y = d.Yf + i * 2 * g.bp;
    const cd w = mk((double)y[s] + di * p.x, (double)y[g.bp + s] + di * p.y);
    d.V[(long long)(d.m + s) * d.N + i] = p;
    d.W[(long long)(d.m + s) * d.N + i] = w;
  }
}

// Residuals and preconditioned corrections of the lowest block: norms^2 accumulated.
__global__ void __launch_bounds__(BD_ROWS) bd_residual_kernel(BDGlobal g, BDav* D, const int* __restrict__ off) {
  const int mem = bd_member(off, g.nmem, blockIdx.x);
  BDav& d = D[mem];
  if (!d.active) return;
  const long long i = (long long)(blockIdx.x - off[mem]) * BD_ROWS + threadIdx.x;
  __shared__ double red[BD_MAXB][BD_ROWS / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int j = 0; j < g.bsz; j++) {
    double n2 = 0.0;
    if (i < d.N) {
      const double th = d.theta[j];
      const cd u = d.U[(long long)j * d.N + i], wv = d.WU[(long long)j * d.N + i];
      const cd r = mk(wv.x - th * u.x, wv.y - th * u.y);
      n2 = nrm2(r);
      double den = th - d.diagH[i];
      if (fabs(den) < 1e-8) den = (den < 0 ? -1e-8 : 1e-8);
      d.P[(long long)j * d.N + i] = mk(r.x / den, r.y / den);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n2 += __shfl_xor_sync(0xffffffffu, n2, o);
    if (lane == 0) red[j][w] = n2;
  }
  __syncthreads();
  if (threadIdx.x < g.bsz) {
    double s = 0.0;
    for (int q = 0; q < BD_ROWS / 32; q++) s += red[threadIdx.x][q];
    atomicAdd(&d.norms[threadIdx.x], s);
  }
}

// P[:, 0:kk] = P[:, 0:bsz] S, remaining columns zero.
__global__ void __launch_bounds__(BD_ROWS) bd_apply_s_kernel(BDGlobal g, BDav* D, const int* __restrict__ off) {
  const int mem = bd_member(off, g.nmem, blockIdx.x);
  const BDav& d = D[mem];
  if (!d.active) return;
  __shared__ cd sS[BD_MAXB * BD_MAXB];
  for (int t = threadIdx.x; t < g.bsz * BD_MAXB; t += blockDim.x) sS[t] = d.S[t];
  __syncthreads();
  const long long i = (long long)(blockIdx.x - off[mem]) * BD_ROWS + threadIdx.x;
  if (i >= d.N) return;
  cd x[BD_MAXB];
#pragma unroll
  for (int s = 0; s < BD_MAXB; s++) x[s] = s < g.bsz ? d.P[(long long)s * d.N + i] : mk(0, 0);
  for (int c = 0; c < g.bsz; c++) {
    cd v = mk(0, 0);
    if (c < d.k) {
#pragma unroll
      for (int s = 0; s < BD_MAXB; s++) v = v + x[s] * sS[s + c * BD_MAXB];
    }
    d.P[(long long)c * d.N + i] = v;
  }
}

// P -= V[:, 0:m] C  (C: m x bsz, ld BD_MMAX).
__global__ void __launch_bounds__(BD_ROWS) bd_cgs_update_kernel(BDGlobal g, BDav* D, const int* __restrict__ off,
                                                                 int pass) {
  const int mem = bd_member(off, g.nmem, blockIdx.x);
  const BDav& d = D[mem];
  if (!d.active) return;
  __shared__ cd sC[BD_MMAX * BD_MAXB];
  const cd* C = pass == 0 ? d.C1 : d.C2;
  const int m = d.m;
  for (int t = threadIdx.x; t < m * g.bsz; t += blockDim.x) {
    const int r = t % m, c = t / m;
    sC[r + c * BD_MMAX] = C[r + c * BD_MMAX];
  }
  __syncthreads();
  const long long i = (long long)(blockIdx.x - off[mem]) * BD_ROWS + threadIdx.x;
  if (i >= d.N) return;
  cd acc[BD_MAXB];
#pragma unroll
  for (int s = 0; s < BD_MAXB; s++) acc[s] = mk(0, 0);
  for (int j = 0; j < m; j++) {
    const cd v = d.V[(long long)j * d.N + i];
#pragma unroll
    for (int s = 0; s < BD_MAXB; s++)
      if (s < g.bsz) acc[s] = acc[s] + v * sC[j + s * BD_MMAX];
  }
#pragma unroll
  for (int s = 0; s < BD_MAXB; s++)
    if (s < g.bsz) d.P[(long long)s * d.N + i] = d.P[(long long)s * d.N + i] - acc[s];
}

// U = V[:, 0:m] Y, WU = W[:, 0:m] Y for the bsz block columns: one thread per row, Y in shared memory
// (broadcast reads), V and W read once per row in coalesced column order.
__global__ void __launch_bounds__(BD_ROWS) bd_ritz_kernel(BDGlobal g, BDav* D, const int* __restrict__ off) {
  const int mem = bd_member(off, g.nmem, blockIdx.x);
  const BDav& d = D[mem];
  if (!d.active) return;
  __shared__ cd sY[BD_MMAX * BD_MAXB];
  const int m = d.m;
  for (int t = threadIdx.x; t < m * g.bsz; t += blockDim.x) {
    const int r = t % m, c = t / m;
    sY[r * BD_MAXB + c] = d.Y[r + c * BD_MMAX];
  }
  __syncthreads();
  const long long i = (long long)(blockIdx.x - off[mem]) * BD_ROWS + threadIdx.x;
  if (i >= d.N) return;
  cd au[BD_MAXB], aw[BD_MAXB];
#pragma unroll
  for (int s = 0; s < BD_MAXB; s++) au[s] = aw[s] = mk(0, 0);
  for (int j = 0; j < m; j++) {
    const cd v = d.V[(long long)j * d.N + i], w = d.W[(long long)j * d.N + i];
#pragma unroll
    for (int s = 0; s < BD_MAXB; s++)
      if (s < g.bsz) {
        const cd y = sY[j * BD_MAXB + s];
        au[s] = au[s] + v * y;
        aw[s] = aw[s] + w * y;
      }
  }
#pragma unroll
  for (int s = 0; s < BD_MAXB; s++)
    if (s < g.bsz) {
      d.U[(long long)s * d.N + i] = au[s];
      d.WU[(long long)s * d.N + i] = aw[s];
    }
}

// Thick restart of the members that decided one: V[:, 0:bsz] = U, W[:, 0:bsz] = WU.
__global__ void __launch_bounds__(BD_ROWS) bd_restart_kernel(BDGlobal g, BDav* D, const int* __restrict__ off) {
  const int mem = bd_member(off, g.nmem, blockIdx.x);
  const BDav& d = D[mem];
  if (!d.active || !d.restart) return;
  const long long i = (long long)(blockIdx.x - off[mem]) * BD_ROWS + threadIdx.x;
  if (i >= d.N) return;
  for (int s = 0; s < g.bsz; s++) {
    d.V[(long long)s * d.N + i] = d.U[(long long)s * d.N + i];
    d.W[(long long)s * d.N + i] = d.WU[(long long)s * d.N + i];
  }
}

// ------------------------------------------------------------------ reductions  Z += A^H B
// mode 0: T[:, m:m+k] += V[:, 0:m+k]^H W[:, m:m+k]     (projection; m = basis before the append)
// mode 1/2: C1/C2 += V[:, 0:m]^H P[:, 0:bsz]           (Gram-Schmidt coefficients)
// mode 3/4: G1/G2 += P^H P                              (Gram matrices)
__global__ void __launch_bounds__(256) bd_gemm_h_kernel(BDGlobal g, BDav* D, const int* __restrict__ off, int mode) {
  const int mem = bd_member(off, g.nmem, blockIdx.x);
  const BDav& d = D[mem];
  if (!d.active) return;
  const cd *A, *B;
  cd* Z;
  int ma, nb, b0 = 0, ldz;
  if (mode == 0) {
    A = d.V; ma = d.m + d.k; B = d.W; b0 = d.m; nb = d.k; Z = d.T + (long long)d.m * BD_MMAX; ldz = BD_MMAX;
  } else if (mode <= 2) {
    A = d.V; ma = d.m; B = d.P; nb = g.bsz; Z = mode == 1 ? d.C1 : d.C2; ldz = BD_MMAX;
  } else {
    A = d.P; ma = g.bsz; B = d.P; nb = g.bsz; Z = mode == 3 ? d.G1 : d.G2; ldz = BD_MAXB;
  }
  if (ma <= 0 || nb <= 0) return;
  __shared__ cd sA[BD_SUB][BD_MMAX + 1];
  __shared__ cd sB[BD_SUB][BD_MAXB + 1];
  constexpr int PER = (BD_MMAX * BD_MAXB + 255) / 256;
  cd acc[PER];
#pragma unroll
  for (int q = 0; q < PER; q++) acc[q] = mk(0, 0);
  const long long row0 = (long long)(blockIdx.x - off[mem]) * BD_RED_ROWS;
  const long long row1 = min(row0 + BD_RED_ROWS, d.N);
  for (long long r0 = row0; r0 < row1; r0 += BD_SUB) {
    for (int t = threadIdx.x; t < BD_SUB * ma; t += blockDim.x) {
      const int q = t % BD_SUB, c = t / BD_SUB;
      sA[q][c] = (r0 + q < row1) ? A[(long long)c * d.N + r0 + q] : mk(0, 0);
    }
    for (int t = threadIdx.x; t < BD_SUB * nb; t += blockDim.x) {
      const int q = t % BD_SUB, c = t / BD_SUB;
      sB[q][c] = (r0 + q < row1) ? B[(long long)(b0 + c) * d.N + r0 + q] : mk(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PER; q++) {
      const int o = threadIdx.x + q * 256;
      if (o < ma * nb) {
        const int r = o % ma, c = o / ma;
        cd s = acc[q];
        for (int x = 0; x < BD_SUB; x++) s = s + cmulc(sA[x][r], sB[x][c]);
        acc[q] = s;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < PER; q++) {
    const int o = threadIdx.x + q * 256;
    if (o < ma * nb) {
      const int r = o % ma, c = o / ma;
      atomicAdd(&Z[r + (long long)c * ldz].x, acc[q].x);
      atomicAdd(&Z[r + (long long)c * ldz].y, acc[q].y);
    }
  }
}

// ------------------------------------------------------------------ per-system kernels (one CTA each)
// Start vectors: unit vectors at the bsz smallest diagonal entries.
__global__ void __launch_bounds__(256) bd_init_kernel(BDGlobal g, BDav* D) {
  BDav& d = D[blockIdx.x];
  __shared__ long long sel[BD_MAXB];
  __shared__ double rv[8];
  __shared__ long long ri[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int j = 0; j < g.bsz; j++) {
    double best = INFINITY;
    long long bi = d.N;
    for (long long i = threadIdx.x; i < d.N; i += blockDim.x) {
      bool taken = false;
      for (int q = 0; q < j; q++) taken |= (sel[q] == i);
      const double v = d.diagH[i];
      if (!taken && (v < best || (v == best && i < bi))) {
        best = v;
        bi = i;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, best, o);
      const long long oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov < best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
      }
    }
    if (lane == 0) {
      rv[w] = best;
      ri[w] = bi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double b = rv[0];
      long long i0 = ri[0];
      for (int q = 1; q < (int)(blockDim.x >> 5); q++)
        if (rv[q] < b || (rv[q] == b && ri[q] < i0)) {
          b = rv[q];
          i0 = ri[q];
        }
      sel[j] = i0;
    }
    __syncthreads();
  }
  for (long long t = threadIdx.x; t < d.N * BD_MAXB; t += blockDim.x) d.P[t] = mk(0, 0);
  for (int t = threadIdx.x; t < BD_MMAX * BD_MMAX; t += blockDim.x) d.T[t] = mk(0, 0);
  __syncthreads();
  if (threadIdx.x < g.bsz) d.P[(long long)threadIdx.x * d.N + sel[threadIdx.x]] = mk(1.0, 0.0);
  if (threadIdx.x == 0) {
    d.m = 0;
    d.k = g.bsz;
    d.active = 1;
    d.iters = 0;
    d.stalled = 0;
    d.kmask = 0;
  }
}

// Zero the new columns of T before the projection.
__global__ void bd_prep_kernel(BDGlobal g, BDav* D) {
  BDav& d = D[blockIdx.x];
  if (!d.active) return;
  const int m1 = d.m + d.k;
  for (int t = threadIdx.x; t < m1 * d.k; t += blockDim.x) {
    const int r = t % m1, c = d.m + t / m1;
    d.T[r + (long long)c * BD_MMAX] = mk(0, 0);
  }
}

// Make the new columns of T exactly Hermitian (new x new block: the average of both triangles; the rows of
// the new columns in the old columns by conjugation), then the lowest bsz Ritz pairs of T; m <- m + k.
__global__ void __launch_bounds__(BD_RR_THREADS) bd_rr_kernel(BDGlobal g, BDav* D, int* status) {
  BDav& d = D[blockIdx.x];
  if (!d.active) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int m0 = d.m, m = d.m + d.k;
  cd* T = d.T;
  const int nn = d.k;
  for (int t = threadIdx.x; t < m * nn; t += blockDim.x) {
    const int r = t % m, c = m0 + t / m;
    if (r < m0) {
      T[c + (long long)r * BD_MMAX] = conj(T[r + (long long)c * BD_MMAX]);
    } else if (r >= c) {
      const cd a = T[r + (long long)c * BD_MMAX], bb = T[c + (long long)r * BD_MMAX];
      const cd v = (r == c) ? mk(a.x, 0.0) : mk(0.5 * (a.x + bb.x), 0.5 * (a.y - bb.y));
      T[r + (long long)c * BD_MMAX] = v;
      T[c + (long long)r * BD_MMAX] = conj(v);
    }
  }
  __syncthreads();
  const int nr = min(g.bsz, m);
  heev_lowest(T, BD_MMAX, m, nr, d.theta, d.Y, BD_MMAX, d.R, smem_raw, status);
  for (int c = threadIdx.x; c < BD_MAXB; c += blockDim.x) d.norms[c] = 0.0;
  __syncthreads();
  if (threadIdx.x == 0) d.m = m;
}

// Convergence, restart decision (T <- diag(theta) on restart), next targets; zero the reduction targets.
__global__ void bd_control_kernel(BDGlobal g, BDav* D) {
  BDav& d = D[blockIdx.x];
  if (!d.active) return;
  __shared__ int s_restart;
  if (threadIdx.x == 0) {
    d.iters++;
    double maxres = 0.0;
    int mask = 0;
    for (int j = 0; j < g.bsz; j++) {
      const double nj = sqrt(d.norms[j]);
      d.norms[j] = nj;
      if (j < g.nstates) maxres = fmax(maxres, (nj == nj) ? nj : INFINITY);
      if (nj >= g.tol) mask |= 1 << j;
    }
    d.kmask = mask;
    if (maxres < g.tol) {
      d.active = 0;
    } else if (d.iters >= g.max_iter) {
      d.active = 0;
      d.stalled = 1;
    }
    s_restart = (d.active && d.m + g.bsz > g.mmax) ? 1 : 0;
    d.restart = s_restart;
    if (s_restart) d.m = g.bsz;
  }
  __syncthreads();
  if (!d.active) return;
  if (s_restart) {
    const int m = d.m;
    for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
      const int r = t % m, c = t / m;
      d.T[r + (long long)c * BD_MMAX] = mk(r == c ? d.theta[r] : 0.0, 0.0);
    }
  }
  for (int t = threadIdx.x; t < BD_MMAX * BD_MAXB; t += blockDim.x) {
    d.C1[t] = mk(0, 0);
    d.C2[t] = mk(0, 0);
  }
  for (int t = threadIdx.x; t < BD_MAXB * BD_MAXB; t += blockDim.x) {
    d.G1[t] = mk(0, 0);
    d.G2[t] = mk(0, 0);
  }
}

// Orthonormaliser of P from its Gram matrix: S = U_kept diag(lambda^-1/2); k <- kept.
// pass 0: columns outside the correction mask are dropped, relative threshold;
// pass 1: absolute threshold (the columns had unit norm before the projection).
__global__ void __launch_bounds__(BD_EIGH_THREADS) bd_orth_kernel(BDGlobal g, BDav* D, int pass, int* status) {
  BDav& d = D[blockIdx.x];
  if (!d.active) return;
  const int n = g.bsz, lda = BD_MAXB + 1;
  __shared__ cd A[BD_MAXB * (BD_MAXB + 1)];
  __shared__ cd Vs[BD_MAXB * BD_MAXB];
  __shared__ JacobiRot rot[BD_MAXB / 2 + 2];
  __shared__ double scratch[64];
  __shared__ int perm[BD_MAXB + 1];
  const cd* G = pass == 0 ? d.G1 : d.G2;
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
    const int r = t % n, c = t / n;
    cd v = G[r + c * BD_MAXB];
    if (pass == 0 && (!((d.kmask >> r) & 1) || !((d.kmask >> c) & 1))) v = mk(0, 0);
    if (pass == 1 && (r >= d.k || c >= d.k)) v = mk(0, 0);
    A[r * lda + c] = v;
  }
  __syncthreads();
  BlockGroup grp;
  const int sweeps = jacobi_eigh(grp, A, lda, Vs, n, n, rot, scratch, 60, 1e-15);
  if (sweeps > 60 && threadIdx.x == 0) atomicOr(status, XATU_DEVERR_NOCONV);
  jacobi_sort(grp, A, lda, n, perm);
  __shared__ int s_kept;
  if (threadIdx.x == 0) {
    const double lmax = A[perm[n - 1] * lda + perm[n - 1]].x;
    const double thr = pass == 0 ? fmax(1e-14 * lmax, 1e-300) : 1e-12;
    int kept = 0;
    for (int q = n - 1; q >= 0; q--)
      if (A[perm[q] * lda + perm[q]].x > thr) kept++;
    s_kept = kept;
  }
  __syncthreads();
  const int kept = s_kept;
  // S[:, c] = u_{perm[n-1-c]} / sqrt(lambda), c < kept (largest first)
  for (int t = threadIdx.x; t < n * BD_MAXB; t += blockDim.x) {
    const int r = t % BD_MAXB, c = t / BD_MAXB;
    cd v = mk(0, 0);
    if (r < n && c < kept) {
      const int e = perm[n - 1 - c];
      const double f = 1.0 / sqrt(A[e * lda + e].x);
      v = f * Vs[r * n + e];
    }
    d.S[r + c * BD_MAXB] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    d.k = kept;
    if (kept == 0) {
      d.active = 0;
      d.stalled = 1;
    }
  }
}

__global__ void bd_count_kernel(BDGlobal g, const BDav* D, int* count) {
  int c = 0;
  for (int i = threadIdx.x; i < g.nmem; i += blockDim.x) c += D[i].active;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if (threadIdx.x == 0) *count = c;
}

// Loop control of the solve graph (body of its conditional WHILE node): counts the finished lockstep iteration
// and keeps the loop running while a member is still active and the iteration cap is not reached.
__global__ void bd_loop_kernel(cudaGraphConditionalHandle h, const int* __restrict__ count, int* __restrict__ iters,
                               int max_iter) {
  const int it = ++*iters;
  cudaGraphSetConditional(h, (*count > 0 && it < max_iter) ? 1u : 0u);
}

// ------------------------------------------------------------------ host side
struct BatchClass {
  int nv, nc, na, tk;
  std::vector<int> members;      // member indices, largest first
  DBuf d_members, d_work, d_counter;
  int nwork = 0;
  size_t smem = 0;
  float tuned_ms[2] = {-1, -1};  // tk = 8, 16
};

struct xatu_batch {
  int device = 0;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  std::string err;
  std::vector<xatu_ctx*> members;
  std::vector<BatchClass> classes;
  bool prepared = false;
  int num_sms = 148;
  int nstates = 0, bsz = 0, max_iter = 200;
  double tol = 1e-4;
  BDGlobal g{};
  BDGlobal chosen{};
  std::vector<BDav> hdesc;
  DBuf d_desc, d_row_off, d_red_off, d_count, d_iters, d_status, d_arena;
  int nrow = 0, nred = 0;
  int* h_count = nullptr;        // pinned
  cudaGraphExec_t build_exec = nullptr, iter_exec = nullptr;
  cudaEvent_t ev[4] = {};
  float build_ms = 0, solve_ms = 0;
  int iterations = 0;
  long long launches_per_iter = 0, launches_build = 0;
  std::string tuning;
};

static xatu_status bfail(xatu_batch* b, xatu_status code, const std::string& msg) {
  if (b) b->err = msg;
  return code;
}

#define BCK(call)                                                                         \
  do {                                                                                    \
    cudaError_t e__ = (call);                                                             \
    if (e__ != cudaSuccess)                                                               \
      return bfail(b, e__ == cudaErrorMemoryAllocation ? XATU_ERR_ALLOC : XATU_ERR_CUDA,  \
                   std::string("CUDA error in ") + #call + ": " + cudaGetErrorString(e__)); \
  } while (0)

#define BTRY(x)                                                                   \
  do {                                                                            \
    xatu_status s__ = (x);                                                        \
    if (s__ != XATU_OK) return s__;                                               \
  } while (0)

static xatu_status member_fail(xatu_batch* b, int i, xatu_status st) {
  return bfail(b, st, "system " + std::to_string(i) + ": " + std::string(xatu_last_error(b->members[i])));
}

// class launch with the member table for tile size tk
static xatu_status class_setup(xatu_batch* b, BatchClass& c, int tk) {
  std::vector<AsmBatchMember> hm(c.members.size());
  std::vector<int2> work;
  int norb_max = 0, exch = 0;
  for (size_t q = 0; q < c.members.size(); q++) {
    xatu_ctx* ctx = b->members[c.members[q]];
    memset(&hm[q], 0, sizeof(AsmBatchMember));
    xatu_assembly_setup(ctx, nullptr, &hm[q].p, &hm[q].in, &hm[q].out);
    const int nblk = (ctx->nk + tk - 1) / tk;
    hm[q].nblk = nblk;
    const int ntiles = nblk * (nblk + 1) / 2;
    for (int t = 0; t < ntiles; t++) work.push_back(make_int2((int)q, t));
    norb_max = std::max(norb_max, ctx->norb);
    exch |= ctx->exchange;
  }
  c.smem = xatu_assembly_batch_smem(c.nv, c.nc, c.na, tk, norb_max, exch);
  if (c.smem > 227 * 1024) return bfail(b, XATU_ERR_UNSUPPORTED, "assembly tile does not fit in shared memory");
  BCK(c.d_members.ensure(hm.size() * sizeof(AsmBatchMember)));
  BCK(cudaMemcpyAsync(c.d_members.p, hm.data(), hm.size() * sizeof(AsmBatchMember), cudaMemcpyHostToDevice,
                      b->stream));
  BCK(c.d_work.ensure(work.size() * sizeof(int2)));
  BCK(cudaMemcpyAsync(c.d_work.p, work.data(), work.size() * sizeof(int2), cudaMemcpyHostToDevice, b->stream));
  BCK(c.d_counter.ensure(sizeof(int)));
  BCK(cudaStreamSynchronize(b->stream));
  c.nwork = (int)work.size();
  c.tk = tk;
  return XATU_OK;
}

static xatu_status class_launch(xatu_batch* b, BatchClass& c, bool set_attr) {
  BCK(cudaMemsetAsync(c.d_counter.p, 0, sizeof(int), b->stream));
  BCK(xatu_launch_assembly_batch(c.nv, c.nc, c.na, c.tk, c.d_members.as<AsmBatchMember>(), c.d_work.as<int2>(),
                                 c.nwork, c.d_counter.as<int>(), c.smem, b->num_sms, set_attr, b->stream));
  return XATU_OK;
}

// Autotuner: every candidate tile size of every class, timed twice on the batch's own data.
static xatu_status autotune(xatu_batch* b) {
  b->tuning = "[";
  for (size_t ci = 0; ci < b->classes.size(); ci++) {
    BatchClass& c = b->classes[ci];
    int best_tk = -1;
    float best = 1e30f;
    const int cands[2] = {8, 16};
    for (int q = 0; q < 2; q++) {
      const int tk = cands[q];
      xatu_status st = class_setup(b, c, tk);
      if (st != XATU_OK) {
        b->err.clear();
        continue;
      }
      float ms = 1e30f;
      for (int rep = 0; rep < 2; rep++) {
        BCK(cudaEventRecord(b->ev[0], b->stream));
        BTRY(class_launch(b, c, true));
        BCK(cudaEventRecord(b->ev[1], b->stream));
        BCK(cudaEventSynchronize(b->ev[1]));
        float t = 0;
        cudaEventElapsedTime(&t, b->ev[0], b->ev[1]);
        ms = std::min(ms, t);
      }
      c.tuned_ms[q] = ms;
      if (ms < best) {
        best = ms;
        best_tk = tk;
      }
    }
    if (best_tk < 0) return bfail(b, XATU_ERR_UNSUPPORTED, "no assembly tile fits this band-window class");
    BTRY(class_setup(b, c, best_tk));
    char buf[256];
    snprintf(buf, sizeof(buf), "%s{\"nv\": %d, \"nc\": %d, \"natoms\": %d, \"systems\": %zu, \"tk8_ms\": %.4f, "
             "\"tk16_ms\": %.4f, \"chosen_tk\": %d}", ci ? ", " : "", c.nv, c.nc, c.na, c.members.size(),
             c.tuned_ms[0], c.tuned_ms[1], best_tk);
    b->tuning += buf;
  }
  b->tuning += "]";
  return XATU_OK;
}

// Build stage of every member (bands, tables, exchange factors) and the class assemblies, then the
// Davidson start; used eagerly once and then recorded into the build graph.
static xatu_status enqueue_build(xatu_batch* b, bool with_assembly, bool with_init) {
  for (size_t i = 0; i < b->members.size(); i++) {
    xatu_ctx* ctx = b->members[i];
    xatu_status st = xatu_bands_enqueue(ctx);
    if (st != XATU_OK) return member_fail(b, (int)i, st);
    st = xatu_tables_enqueue(ctx);
    if (st != XATU_OK) return member_fail(b, (int)i, st);
    if (ctx->exchange) {
      const long long N = ctx->N;
      exchange_vectors_kernel<<<(int)((N + 127) / 128), 128, 0, b->stream>>>(
          (int)N, ctx->nv, ctx->nc, ctx->nb, ctx->norb, ctx->natoms, ctx->d_orboff.as<int>(), ctx->d_eigvec.as<cd>(),
          ctx->d_eigvecQ.as<cd>(), ctx->d_VX.as<cd>(), nullptr, ctx->d_exL.as<cd>(), ctx->d_exR.as<cd>());
      BCK(cudaGetLastError());
    }
  }
  if (with_assembly)
    for (BatchClass& c : b->classes) BTRY(class_launch(b, c, false));
  if (with_init) {
    bd_diag_kernel<<<b->nrow, BD_ROWS, 0, b->stream>>>(b->g, b->d_desc.as<BDav>(), b->d_row_off.as<int>());
    BCK(cudaGetLastError());
    bd_init_kernel<<<b->g.nmem, 256, 0, b->stream>>>(b->g, b->d_desc.as<BDav>());
    BCK(cudaGetLastError());
  }
  return XATU_OK;
}

static size_t rr_smem() { return heev_smem_bytes(BD_MMAX, BD_MAXB); }

// One Davidson step for every active member; to_host: the number of active members is also copied to the host.
static xatu_status enqueue_iteration(xatu_batch* b, bool to_host) {
  const BDGlobal g = b->g;
  BDav* D = b->d_desc.as<BDav>();
  const int* ro = b->d_row_off.as<int>();
  const int* rd = b->d_red_off.as<int>();
  int* status = b->d_status.as<int>();
  bd_build_bt_kernel<<<b->nrow, BD_ROWS, 0, b->stream>>>(g, D, ro);
  BCK(cudaGetLastError());
  for (size_t i = 0; i < b->members.size(); i++) {
    const BDav& h = b->hdesc[i];
    const int ng = 2 * g.bp;
    BCK(xatu_launch_hx_tc(h.Khi, h.Klo, h.N, h.ldk, h.Bhi, h.Blo, h.ldb, h.Uhi, h.Ulo, h.ldu, ng, h.Yf, status,
                          b->num_sms, b->stream, &D[i].active));
  }
  bd_finish_append_kernel<<<b->nrow, BD_ROWS, 0, b->stream>>>(g, D, ro);
  bd_prep_kernel<<<g.nmem, 256, 0, b->stream>>>(g, D);
  bd_gemm_h_kernel<<<b->nred, 256, 0, b->stream>>>(g, D, rd, 0);
  bd_rr_kernel<<<g.nmem, BD_RR_THREADS, rr_smem(), b->stream>>>(g, D, status);
  bd_ritz_kernel<<<b->nrow, BD_ROWS, 0, b->stream>>>(g, D, ro);
  bd_residual_kernel<<<b->nrow, BD_ROWS, 0, b->stream>>>(g, D, ro);
  bd_control_kernel<<<g.nmem, 256, 0, b->stream>>>(g, D);
  bd_restart_kernel<<<b->nrow, BD_ROWS, 0, b->stream>>>(g, D, ro);
  bd_gemm_h_kernel<<<b->nred, 256, 0, b->stream>>>(g, D, rd, 3);
  bd_orth_kernel<<<g.nmem, BD_EIGH_THREADS, 0, b->stream>>>(g, D, 0, status);
  bd_apply_s_kernel<<<b->nrow, BD_ROWS, 0, b->stream>>>(g, D, ro);
  for (int pass = 0; pass < 2; pass++) {
    bd_gemm_h_kernel<<<b->nred, 256, 0, b->stream>>>(g, D, rd, 1 + pass);
    bd_cgs_update_kernel<<<b->nrow, BD_ROWS, 0, b->stream>>>(g, D, ro, pass);
  }
  bd_gemm_h_kernel<<<b->nred, 256, 0, b->stream>>>(g, D, rd, 4);
  bd_orth_kernel<<<g.nmem, BD_EIGH_THREADS, 0, b->stream>>>(g, D, 1, status);
  bd_apply_s_kernel<<<b->nrow, BD_ROWS, 0, b->stream>>>(g, D, ro);
  bd_count_kernel<<<1, 32, 0, b->stream>>>(g, D, b->d_count.as<int>());
  BCK(cudaGetLastError());
  if (to_host) BCK(cudaMemcpyAsync(b->h_count, b->d_count.p, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  return XATU_OK;
}

// Build graph, then the solve graph (the lockstep iterations under a conditional WHILE node: the loop runs on the
// device until no system is active or the iteration cap is reached, without a host round trip per iteration);
// device ms of the whole solve.
static xatu_status run_graphs(xatu_batch* b, cudaGraphExec_t build, cudaGraphExec_t solve, int* iters, float* ms) {
  BCK(cudaMemsetAsync(b->d_iters.p, 0, sizeof(int), b->stream));
  BCK(cudaEventRecord(b->ev[0], b->stream));
  BCK(cudaGraphLaunch(build, b->stream));
  BCK(cudaEventRecord(b->ev[1], b->stream));
  BCK(cudaGraphLaunch(solve, b->stream));
  BCK(cudaEventRecord(b->ev[2], b->stream));
  int h_it = 0;
  BCK(cudaMemcpyAsync(b->h_count, b->d_count.p, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaMemcpyAsync(&h_it, b->d_iters.p, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  cudaEventElapsedTime(&b->build_ms, b->ev[0], b->ev[1]);
  cudaEventElapsedTime(&b->solve_ms, b->ev[1], b->ev[2]);
  b->iterations = h_it;
  if (ms) *ms = b->build_ms + b->solve_ms;
  if (iters) *iters = h_it;
  return XATU_OK;
}

// The solve graph: one conditional WHILE node (condition set to 1 at every launch) whose body is one lockstep
// iteration followed by bd_loop_kernel.
static xatu_status capture_solve(xatu_batch* b, cudaGraphExec_t* exec) {
  cudaGraph_t graph = nullptr;
  BCK(cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle h;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault);
  cudaGraphNodeParams cp = {};
  cudaGraphNode_t node = nullptr;
  if (e == cudaSuccess) {
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    e = cudaGraphAddNode(&node, graph, nullptr, 0, &cp);
  }
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    BCK(e);
  }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  e = cudaStreamBeginCaptureToGraph(b->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    BCK(e);
  }
  xatu_status st = enqueue_iteration(b, false);
  if (st == XATU_OK) {
    bd_loop_kernel<<<1, 1, 0, b->stream>>>(h, b->d_count.as<int>(), b->d_iters.as<int>(), b->max_iter);
    if ((e = cudaGetLastError()) != cudaSuccess) st = bfail(b, XATU_ERR_CUDA, cudaGetErrorString(e));
  }
  cudaGraph_t captured = nullptr;
  e = cudaStreamEndCapture(b->stream, &captured);
  if (st != XATU_OK) {
    cudaGraphDestroy(graph);
    return st;
  }
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    BCK(e);
  }
  e = cudaGraphInstantiate(exec, graph, 0);
  cudaGraphDestroy(graph);
  BCK(e);
  return XATU_OK;
}

static xatu_status capture(xatu_batch* b, bool build, cudaGraphExec_t* exec) {
  cudaGraph_t graph = nullptr;
  BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
  xatu_status st = build ? enqueue_build(b, true, true) : enqueue_iteration(b, true);   // (the solve: capture_solve)
  cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
  if (st != XATU_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  BCK(e);
  e = cudaGraphInstantiate(exec, graph, 0);
  cudaGraphDestroy(graph);
  BCK(e);
  return XATU_OK;
}

// Allocations, start offsets, tuning and graphs (first run only).
static xatu_status prepare(xatu_batch* b, int nstates, double tol) {
  const int nmem = (int)b->members.size();
  if (nmem == 0) return bfail(b, XATU_ERR_STATE, "empty batch");
  b->nstates = nstates;
  // block candidates: nstates plus guard vectors, and the same rounded up to the 8-column granule of the
  // tensor-core operand (no extra pass over K; a larger basis per iteration).  The buffers are sized for
  // the largest; the autotuner keeps the faster.
  const int b0 = std::max(8, nstates + std::max(4, (nstates + 3) / 4));
  if (b0 > BD_MAXB || b0 < nstates)
    return bfail(b, XATU_ERR_UNSUPPORTED, "batched Davidson supports at most 12 states (block of 16)");
  std::vector<int> blocks = {b0};
  if ((b0 + 7) / 8 * 8 != b0 && (b0 + 7) / 8 * 8 <= BD_MAXB) blocks.push_back((b0 + 7) / 8 * 8);
  b->bsz = blocks.back();
  const int mmax = BD_MMAX;
  auto basis_of = [](int bs) { return std::min(BD_MMAX, BD_BASIS_BLOCKS * bs); };
  // per-member buffers
  for (int i = 0; i < nmem; i++) {
    xatu_ctx* ctx = b->members[i];
    const long long N = ctx->N;
    if (N < basis_of(b0))
      return bfail(b, XATU_ERR_UNSUPPORTED, "system " + std::to_string(i) + " is smaller than the basis");
    if (N < basis_of(blocks.back())) blocks.resize(1);   // the larger block's basis would not fit this system
    if (!xatu_assembly_batch_supported(ctx->nv, ctx->nc, ctx->natoms))
      return bfail(b, XATU_ERR_UNSUPPORTED, "system " + std::to_string(i) +
                                                ": batched assembly supports 1-3 valence/conduction bands, 2-3 atoms");
    BCK(ctx->d_Khi.ensure((size_t)N * ctx->ldk * sizeof(__nv_bfloat162)));
    BCK(ctx->d_Klo.ensure((size_t)N * ctx->ldk * sizeof(__nv_bfloat162)));
    BCK(ctx->d_diag.ensure((size_t)N * sizeof(double)));
    if (ctx->exchange) {
      BCK(ctx->d_exL.ensure((size_t)N * ctx->natoms * sizeof(cd)));
      BCK(ctx->d_exR.ensure((size_t)N * ctx->natoms * sizeof(cd)));
    }
  }
  // classes, largest systems first
  b->classes.clear();
  std::vector<int> order(nmem);
  for (int i = 0; i < nmem; i++) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int x, int y) { return b->members[x]->N > b->members[y]->N; });
  for (int i : order) {
    xatu_ctx* ctx = b->members[i];
    BatchClass* c = nullptr;
    for (auto& cc : b->classes)
      if (cc.nv == ctx->nv && cc.nc == ctx->nc && cc.na == ctx->natoms) c = &cc;
    if (!c) {
      b->classes.emplace_back();
      c = &b->classes.back();
      c->nv = ctx->nv;
      c->nc = ctx->nc;
      c->na = ctx->natoms;
    }
    c->members.push_back(i);
  }
  // eager build (allocates the stage buffers), then the tile autotuner on the real data
  BTRY(enqueue_build(b, false, false));
  BCK(cudaStreamSynchronize(b->stream));
  BTRY(autotune(b));
  // Davidson arena
  b->g.nmem = nmem;
  b->g.bsz = b->bsz;
  b->g.bp = BD_MAXB;                 // allocation: the largest operand
  b->g.mmax = mmax;
  b->g.nstates = nstates;
  b->g.max_iter = b->max_iter;
  b->g.tol = tol;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  std::vector<size_t> offs(nmem);
  size_t total = 0;
  for (int i = 0; i < nmem; i++) {
    const long long N = b->members[i]->N;
    const long long ldb = (2 * N + 7) / 8 * 8, ldu = (N + 7) / 8 * 8;
    offs[i] = total;
    total += al(N * sizeof(double)) + 2 * al((size_t)N * mmax * sizeof(cd)) + 3 * al((size_t)N * BD_MAXB * sizeof(cd)) +
             3 * al((size_t)BD_MMAX * BD_MMAX * sizeof(cd)) + 2 * al((size_t)BD_MMAX * BD_MAXB * sizeof(cd)) +
             3 * al((size_t)BD_MAXB * BD_MAXB * sizeof(cd)) + al(BD_MMAX * sizeof(double)) +
             al(BD_MAXB * sizeof(double)) + al((size_t)N * 2 * b->g.bp * sizeof(float)) +
             2 * al((size_t)2 * b->g.bp * ldb * sizeof(__nv_bfloat16)) +
             2 * al((size_t)2 * b->g.bp * ldu * sizeof(__nv_bfloat16));
  }
  BCK(b->d_arena.ensure(total));
  BCK(cudaMemsetAsync(b->d_arena.p, 0, total, b->stream));
  b->hdesc.assign(nmem, BDav{});
  for (int i = 0; i < nmem; i++) {
    xatu_ctx* ctx = b->members[i];
    BDav& d = b->hdesc[i];
    const long long N = ctx->N;
    unsigned char* p = b->d_arena.as<unsigned char>() + offs[i];
    auto take = [&](size_t bytes) {
      unsigned char* q = p;
      p += al(bytes);
      return q;
    };
    d.N = N;
    d.ldk = ctx->ldk;
    d.ldb = (2 * N + 7) / 8 * 8;
    d.ldu = (N + 7) / 8 * 8;
    d.Khi = ctx->d_Khi.as<__nv_bfloat162>();
    d.Klo = ctx->d_Klo.as<__nv_bfloat162>();
    d.diag = ctx->d_diag.as<double>();
    d.diagH = reinterpret_cast<double*>(take(N * sizeof(double)));
    d.V = reinterpret_cast<cd*>(take((size_t)N * mmax * sizeof(cd)));
    d.W = reinterpret_cast<cd*>(take((size_t)N * mmax * sizeof(cd)));
    d.P = reinterpret_cast<cd*>(take((size_t)N * BD_MAXB * sizeof(cd)));
    d.U = reinterpret_cast<cd*>(take((size_t)N * BD_MAXB * sizeof(cd)));
    d.WU = reinterpret_cast<cd*>(take((size_t)N * BD_MAXB * sizeof(cd)));
    d.T = reinterpret_cast<cd*>(take((size_t)BD_MMAX * BD_MMAX * sizeof(cd)));
    d.Y = reinterpret_cast<cd*>(take((size_t)BD_MMAX * BD_MMAX * sizeof(cd)));
    d.R = reinterpret_cast<cd*>(take((size_t)BD_MMAX * BD_MMAX * sizeof(cd)));
    d.C1 = reinterpret_cast<cd*>(take((size_t)BD_MMAX * BD_MAXB * sizeof(cd)));
    d.C2 = reinterpret_cast<cd*>(take((size_t)BD_MMAX * BD_MAXB * sizeof(cd)));
    d.G1 = reinterpret_cast<cd*>(take((size_t)BD_MAXB * BD_MAXB * sizeof(cd)));
    d.G2 = reinterpret_cast<cd*>(take((size_t)BD_MAXB * BD_MAXB * sizeof(cd)));
    d.S = reinterpret_cast<cd*>(take((size_t)BD_MAXB * BD_MAXB * sizeof(cd)));
    d.theta = reinterpret_cast<double*>(take(BD_MMAX * sizeof(double)));
    d.norms = reinterpret_cast<double*>(take(BD_MAXB * sizeof(double)));
    d.Yf = reinterpret_cast<float*>(take((size_t)N * 2 * b->g.bp * sizeof(float)));
    d.Bhi = reinterpret_cast<__nv_bfloat16*>(take((size_t)2 * b->g.bp * d.ldb * sizeof(__nv_bfloat16)));
    d.Blo = reinterpret_cast<__nv_bfloat16*>(take((size_t)2 * b->g.bp * d.ldb * sizeof(__nv_bfloat16)));
    d.Uhi = reinterpret_cast<__nv_bfloat16*>(take((size_t)2 * b->g.bp * d.ldu * sizeof(__nv_bfloat16)));
    d.Ulo = reinterpret_cast<__nv_bfloat16*>(take((size_t)2 * b->g.bp * d.ldu * sizeof(__nv_bfloat16)));
  }
  BCK(b->d_desc.ensure(nmem * sizeof(BDav)));
  BCK(cudaMemcpyAsync(b->d_desc.p, b->hdesc.data(), nmem * sizeof(BDav), cudaMemcpyHostToDevice, b->stream));
  // chunk offsets
  std::vector<int> ro(nmem + 1), rd(nmem + 1);
  ro[0] = rd[0] = 0;
  for (int i = 0; i < nmem; i++) {
    const long long N = b->members[i]->N;
    ro[i + 1] = ro[i] + (int)((N + BD_ROWS - 1) / BD_ROWS);
    rd[i + 1] = rd[i] + (int)((N + BD_RED_ROWS - 1) / BD_RED_ROWS);
  }
  b->nrow = ro[nmem];
  b->nred = rd[nmem];
  BCK(b->d_row_off.ensure((nmem + 1) * sizeof(int)));
  BCK(b->d_red_off.ensure((nmem + 1) * sizeof(int)));
  BCK(cudaMemcpyAsync(b->d_row_off.p, ro.data(), ro.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  BCK(cudaMemcpyAsync(b->d_red_off.p, rd.data(), rd.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  BCK(b->d_count.ensure(sizeof(int)));
  BCK(b->d_iters.ensure(sizeof(int)));
  BCK(b->d_status.ensure(sizeof(int)));
  BCK(cudaMemsetAsync(b->d_status.p, 0, sizeof(int), b->stream));
  if (!b->h_count) BCK(cudaMallocHost(&b->h_count, sizeof(int)));
  BCK(xatu_raise_smem_limit((const void*)bd_rr_kernel, rr_smem()));
  BCK(cudaStreamSynchronize(b->stream));
  // graphs of every block candidate, each timed on a full solve; the fastest is kept
  std::string dav = "";
  float best = 1e30f;
  for (size_t q = 0; q < blocks.size(); q++) {
    const int bs = blocks[q];
    b->bsz = bs;
    b->g.bsz = bs;
    b->g.bp = (bs + 7) / 8 * 8;
    b->g.mmax = basis_of(bs);
    cudaGraphExec_t be = nullptr, ie = nullptr;
    BTRY(capture(b, true, &be));
    BTRY(capture_solve(b, &ie));
    int it = 0;
    float ms = 0;
    const xatu_status st = run_graphs(b, be, ie, &it, &ms);
    char buf[160];
    snprintf(buf, sizeof(buf), "%s{\"davidson_block\": %d, \"solve_ms\": %.3f, \"iterations\": %d}", q ? ", " : "", bs,
             ms, it);
    dav += buf;
    if (st == XATU_OK && ms < best) {
      best = ms;
      if (b->build_exec) cudaGraphExecDestroy(b->build_exec);
      if (b->iter_exec) cudaGraphExecDestroy(b->iter_exec);
      b->build_exec = be;
      b->iter_exec = ie;
      b->chosen = b->g;
    } else {
      cudaGraphExecDestroy(be);
      cudaGraphExecDestroy(ie);
    }
  }
  if (!b->build_exec) return bfail(b, XATU_ERR_NOT_CONVERGED, "no Davidson block candidate converged");
  b->g = b->chosen;
  b->bsz = b->g.bsz;
  b->tuning = "{\"assembly\": " + b->tuning + ", \"davidson\": [" + dav + "]}";
  b->prepared = true;
  return XATU_OK;
}

extern "C" {

xatu_status xatu_batch_create(xatu_batch** out, int device) {
  if (!out) return XATU_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return XATU_ERR_CUDA;
  if (device < 0 || device >= ndev) return XATU_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return XATU_ERR_CUDA;
  xatu_batch* b = new xatu_batch();
  b->device = device;
  if (cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return XATU_ERR_CUDA;
  }
  b->stream = b->own_stream;
  cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device);
  for (auto& e : b->ev) cudaEventCreate(&e);
  *out = b;
  return XATU_OK;
}

xatu_status xatu_batch_destroy(xatu_batch* b) {
  if (!b) return XATU_OK;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  if (b->build_exec) cudaGraphExecDestroy(b->build_exec);
  if (b->iter_exec) cudaGraphExecDestroy(b->iter_exec);
  for (auto& c : b->classes) {
    c.d_members.release();
    c.d_work.release();
    c.d_counter.release();
  }
  for (DBuf* d : {&b->d_desc, &b->d_row_off, &b->d_red_off, &b->d_count, &b->d_iters, &b->d_status, &b->d_arena})
    d->release();
  if (b->h_count) cudaFreeHost(b->h_count);
  for (xatu_ctx* c : b->members) xatu_ctx_destroy(c);
  for (auto& e : b->ev)
    if (e) cudaEventDestroy(e);
  if (b->own_stream) cudaStreamDestroy(b->own_stream);
  delete b;
  return XATU_OK;
}

const char* xatu_batch_last_error(const xatu_batch* b) { return b ? b->err.c_str() : "null batch"; }

xatu_status xatu_batch_set_stream(xatu_batch* b, void* stream) {
  if (!b) return XATU_ERR_INVALID;
  if (b->prepared) return bfail(b, XATU_ERR_STATE, "the stream must be set before the first run");
  b->stream = stream ? static_cast<cudaStream_t>(stream) : b->own_stream;
  for (xatu_ctx* c : b->members) xatu_ctx_set_stream(c, b->stream);
  return XATU_OK;
}

xatu_status xatu_batch_add(xatu_batch* b, const xatu_system_desc* sys, const xatu_exciton_desc* exc, int* index) {
  if (!b || !sys || !exc) return XATU_ERR_INVALID;
  if (b->prepared) return bfail(b, XATU_ERR_STATE, "systems must be added before the first run");
  cudaSetDevice(b->device);
  xatu_ctx* ctx = nullptr;
  xatu_status st = xatu_ctx_create(&ctx, b->device);
  if (st != XATU_OK) return bfail(b, st, "context creation failed");
  xatu_ctx_set_stream(ctx, b->stream);
  if ((st = xatu_system_upload(ctx, sys)) != XATU_OK || (st = xatu_exciton_set(ctx, exc)) != XATU_OK) {
    b->err = "system " + std::to_string(b->members.size()) + ": " + xatu_last_error(ctx);
    xatu_ctx_destroy(ctx);
    return st;
  }
  if (index) *index = (int)b->members.size();
  b->members.push_back(ctx);
  return XATU_OK;
}

xatu_status xatu_batch_run(xatu_batch* b, int nstates, double tol, int max_iter) {
  if (!b || nstates < 1) return XATU_ERR_INVALID;
  cudaSetDevice(b->device);
  if (!b->prepared) {
    if (max_iter > 0) b->max_iter = max_iter;
    BTRY(prepare(b, nstates, tol > 0 ? tol : 1e-4));
  } else if (nstates != b->nstates || (tol > 0 && tol != b->g.tol) || (max_iter > 0 && max_iter != b->max_iter)) {
    return bfail(b, XATU_ERR_STATE, "nstates, tol and max_iter are fixed at the first run of a batch");
  }
  BTRY(run_graphs(b, b->build_exec, b->iter_exec, nullptr, nullptr));
  // device error words: the batch's own and every member's
  int st = 0;
  BCK(cudaMemcpy(&st, b->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
  for (xatu_ctx* c : b->members) {
    int s2 = 0;
    BCK(cudaMemcpy(&s2, c->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
    st |= s2;
  }
  if (st) {
    cudaMemsetAsync(b->d_status.p, 0, sizeof(int), b->stream);
    for (xatu_ctx* c : b->members) cudaMemsetAsync(c->d_status.p, 0, sizeof(int), b->stream);
    cudaStreamSynchronize(b->stream);
    return bfail(b, (st & (XATU_DEVERR_NAN | XATU_DEVERR_OVERLAP)) ? XATU_ERR_NUMERIC : XATU_ERR_NOT_CONVERGED,
                 "a device stage of the batch reported an error (flags " + std::to_string(st) + ")");
  }
  BCK(cudaMemcpy(b->hdesc.data(), b->d_desc.p, b->hdesc.size() * sizeof(BDav), cudaMemcpyDeviceToHost));
  int bad = 0;
  for (const BDav& d : b->hdesc) bad += (d.active || d.stalled) ? 1 : 0;
  if (bad)
    return bfail(b, XATU_ERR_NOT_CONVERGED, std::to_string(bad) + " systems of the batch did not converge");
  return XATU_OK;
}

xatu_status xatu_batch_result(xatu_batch* b, int index, double* eigval, double* eigvec) {
  if (!b || index < 0 || index >= (int)b->members.size()) return XATU_ERR_INVALID;
  if (!b->prepared) return bfail(b, XATU_ERR_STATE, "run the batch first");
  const BDav& d = b->hdesc[index];
  if (eigval) BCK(cudaMemcpy(eigval, d.theta, b->nstates * sizeof(double), cudaMemcpyDeviceToHost));
  if (eigvec) BCK(cudaMemcpy(eigvec, d.U, (size_t)d.N * b->nstates * sizeof(cd), cudaMemcpyDeviceToHost));
  return XATU_OK;
}

xatu_status xatu_batch_dim(const xatu_batch* b, int index, int64_t* n) {
  if (!b || !n || index < 0 || index >= (int)b->members.size()) return XATU_ERR_INVALID;
  *n = b->members[index]->N;
  return XATU_OK;
}

xatu_status xatu_batch_stats(const xatu_batch* b, double* build_ms, double* solve_ms, int* iterations,
                             int* converged_iters, char* tuning, size_t tuning_len) {
  if (!b) return XATU_ERR_INVALID;
  if (build_ms) *build_ms = b->build_ms;
  if (solve_ms) *solve_ms = b->solve_ms;
  if (iterations) *iterations = b->iterations;
  if (converged_iters)
    for (size_t i = 0; i < b->hdesc.size(); i++) converged_iters[i] = b->hdesc[i].iters;
  if (tuning && tuning_len) {
    strncpy(tuning, b->tuning.c_str(), tuning_len - 1);
    tuning[tuning_len - 1] = 0;
  }
  return XATU_OK;
}

}  // extern "C"
