// Single-particle band solve on the device (ExcitonTB::initializeResultsH0,
// ExcitonTB.cpp:737-758): for every k of the exciton basis (and k + Q),
//   H(k) = sum_R H(R) e^{i k.R}           (SystemTB::hamiltonian, SystemTB.cpp:60-75,
//                                          triangular storage symmetrised as :69-72)
//   H(k) C = C diag(E), E ascending        (SystemTB::solveBands, SystemTB.cpp:113-125)
//   column sums of C made real positive    (ExcitonTB::fixGlobalPhase, ExcitonTB.cpp:673-683)
//   keep the columns of the band list      (ExcitonTB.cpp:741-742)
// With overlap matrices the basis is orthogonalised first (Loewdin,
// SystemTB::orthogonalize_hamiltonian, SystemTB.cpp:136-156):
//   S(k) = sum_R S(R) e^{i k.R},  S = U diag(l) U^H,  X = U diag(l^-1/2) U^H,
//   h <- X h X  (h scaled by 27.2 first when the model is in Hartree),
// and the eigenvectors of X h X are kept as they are, as in the reference.
// One warp per k point, the matrices in shared memory, FP64 Jacobi.
#include "jacobi.cuh"
#include "params.h"

// Odd row pitch (in 16-byte elements) keeps the lane-per-row passes bank-conflict free.
__host__ __device__ __forceinline__ int band_lda(int n) { return (n % 2 == 0) ? n + 1 : n + 2; }

// Bloch sum of a [R][row][col] stack into M (row stride ld), with the
// triangular-storage symmetrisation of SystemTB::hamiltonian (SystemTB.cpp:69-72);
// W is scratch of the same shape.
__device__ void bloch_sum(const WarpGroup& g, const cd* __restrict__ MR, const cd* ph, int nR, int n, int ld,
                          int triangular, double scale, cd* M, cd* W) {
  const int lane = g.rank();
  for (int t = lane; t < n * n; t += 32) {
    const int i = t / n, j = t - i * n;
    cd h = mk(0, 0);
    for (int r = 0; r < nR; r++) h = h + MR[(int64_t)r * n * n + t] * ph[r];
    M[i * ld + j] = scale * h;
  }
  g.sync();
  if (triangular) {
    // h.diag() -= h.diag()/2; h += h^dagger
    for (int t = lane; t < n * n; t += 32) {
      const int i = t / n, j = t - i * n;
      if (i == j) {
        const cd d = M[i * ld + i];
        const cd dh = mk(d.x - d.x / 2, d.y - d.y / 2);
        W[i * ld + j] = dh + conj(dh);
      } else {
        W[i * ld + j] = M[i * ld + j] + conj(M[j * ld + i]);
      }
    }
    g.sync();
    for (int t = lane; t < n * n; t += 32) {
      const int i = t / n, j = t - i * n;
      M[i * ld + j] = W[i * ld + j];
    }
    g.sync();
  }
}

// C = A B (n x n, row stride ld), one warp.
__device__ void warp_matmul(const WarpGroup& g, const cd* A, const cd* B, cd* C, int n, int ld) {
  for (int t = g.rank(); t < n * n; t += 32) {
    const int i = t / n, j = t - i * n;
    cd s = mk(0, 0);
    for (int m = 0; m < n; m++) s = s + A[i * ld + m] * B[m * ld + j];
    C[i * ld + j] = s;
  }
  g.sync();
}

extern "C" __global__ void band_solve_kernel(BandParams bp, const double* __restrict__ kpoints,
                                             const double* __restrict__ cellsR, const cd* __restrict__ HR,
                                             const cd* __restrict__ SR, double* __restrict__ eigval,
                                             cd* __restrict__ eigvec, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = bp.norb, lda = band_lda(n);
  const int warps = blockDim.x >> 5;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nmat = bp.has_overlap ? 3 : 2;
  // per-warp shared layout
  const size_t matsz = (size_t)n * lda;
  const size_t per_warp = nmat * matsz * sizeof(cd) + (size_t)(n / 2 + 2) * sizeof(JacobiRot) +
                          (size_t)bp.nR * sizeof(cd) + (size_t)(n + 1) * sizeof(int);
  const size_t per_warp_al = (per_warp + 15) & ~(size_t)15;
  unsigned char* base = smem_raw + per_warp_al * w;
  cd* A = reinterpret_cast<cd*>(base);
  cd* V = A + matsz;
  cd* B = V + (nmat == 3 ? matsz : 0);          // third matrix (overlap only)
  JacobiRot* rot = reinterpret_cast<JacobiRot*>(A + nmat * matsz);
  cd* ph = reinterpret_cast<cd*>(rot + (n / 2 + 2));
  int* perm = reinterpret_cast<int*>(ph + bp.nR);

  const int k = blockIdx.x * warps + w;
  if (k >= bp.nk) return;  // whole warp exits together
  WarpGroup g;
  const double kx = kpoints[3 * k] + bp.shift[0];
  const double ky = kpoints[3 * k + 1] + bp.shift[1];
  const double kz = kpoints[3 * k + 2] + bp.shift[2];
  for (int r = lane; r < bp.nR; r += 32) {
    double s, c;
    sincos(kx * cellsR[3 * r] + ky * cellsR[3 * r + 1] + kz * cellsR[3 * r + 2], &s, &c);
    ph[r] = mk(c, s);
  }
  g.sync();
  if (bp.has_overlap) {
    // B = h (scaled), A = S(k); Jacobi of S into (A, V); A = X = V diag(l^-1/2) V^H; h' = X h X -> A
    bloch_sum(g, HR, ph, bp.nR, n, lda, bp.triangular, bp.is_au ? 27.2 : 1.0, B, V);
    bloch_sum(g, SR, ph, bp.nR, n, lda, bp.triangular, 1.0, A, V);
    const int sw = jacobi_eigh_warp(A, lda, V, lda, n, rot, bp.max_sweeps, 1e-15);
    if (sw > bp.max_sweeps && lane == 0) atomicOr(status, XATU_DEVERR_NOCONV);
    bool nonpos = false;
    for (int i = lane; i < n; i += 32) nonpos |= !(A[i * lda + i].x > 0.0);
    if (__any_sync(0xffffffffu, nonpos)) {
      if (lane == 0) atomicOr(status, XATU_DEVERR_OVERLAP);
      return;
    }
    // l^-1/2 into scratch (the rotation array is free between the two solves)
    double* lis = reinterpret_cast<double*>(rot);
    for (int i = lane; i < n; i += 32) lis[i] = 1.0 / sqrt(A[i * lda + i].x);
    g.sync();
    // A = X = V diag(l^-1/2) V^H
    for (int t = lane; t < n * n; t += 32) {
      const int i = t / n, j = t - i * n;
      cd sum = mk(0, 0);
      for (int m = 0; m < n; m++) sum = sum + lis[m] * (V[i * lda + m] * conj(V[j * lda + m]));
      A[i * lda + j] = sum;
    }
    g.sync();
    warp_matmul(g, A, B, V, n, lda);   // V = X h
    warp_matmul(g, V, A, B, n, lda);   // B = X h X
    for (int t = lane; t < n * n; t += 32) {
      const int i = t / n, j = t - i * n;
      A[i * lda + j] = B[i * lda + j];
    }
    g.sync();
  } else {
    bloch_sum(g, HR, ph, bp.nR, n, lda, bp.triangular, 1.0, A, V);
  }
  // NaN guard on the input matrix
  bool bad = false;
  for (int t = lane; t < n * n; t += 32) {
    const int i = t / n, j = t - i * n;
    const cd a = A[i * lda + j];
    if (!(isfinite(a.x) && isfinite(a.y))) bad = true;
  }
  if (__any_sync(0xffffffffu, bad)) {
    if (lane == 0) atomicOr(status, XATU_DEVERR_NAN);
    return;
  }
  const int sweeps = jacobi_eigh_warp(A, lda, V, lda, n, rot, bp.max_sweeps, 1e-15);
  if (sweeps > bp.max_sweeps && lane == 0) atomicOr(status, XATU_DEVERR_NOCONV);
  jacobi_sort(g, A, lda, n, perm);
  for (int b = 0; b < bp.nb; b++) {
    const int col = perm[bp.band_list[b]];
    // fixGlobalPhase: multiply the column by e^{-i arg(sum_o C_o)}
    double sr = 0.0, si = 0.0;
    for (int o = lane; o < n; o += 32) { sr += V[o * lda + col].x; si += V[o * lda + col].y; }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, off);
      si += __shfl_xor_sync(0xffffffffu, si, off);
    }
    const double ang = atan2(si, sr);
    double s, c;
    sincos(-ang, &s, &c);
    const cd f = mk(c, s);
    cd* out = eigvec + ((int64_t)k * bp.nb + b) * n;
    for (int o = lane; o < n; o += 32) out[o] = V[o * lda + col] * f;
    if (lane == 0) eigval[(int64_t)k * bp.nb + b] = A[col * lda + col].x;
  }
}

extern "C" size_t band_solve_smem_per_warp(int norb, int nR, int has_overlap) {
  const int n = norb, lda = band_lda(n);
  const size_t matsz = (size_t)n * lda;
  const size_t per_warp = (has_overlap ? 3 : 2) * matsz * sizeof(cd) + (size_t)(n / 2 + 2) * sizeof(JacobiRot) +
                          (size_t)nR * sizeof(cd) + (size_t)(n + 1) * sizeof(int);
  return (per_warp + 15) & ~(size_t)15;
}
