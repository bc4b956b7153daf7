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
// One CTA of BAND_THREADS threads per k point, the matrices in shared memory,
// FP64 two-phase Jacobi (jacobi.cuh).
#include "jacobi.cuh"
#include "params.h"

#define BAND_THREADS 128

// Odd row pitch (in 16-byte elements) spreads the 2x2-block accesses over the banks.
__host__ __device__ __forceinline__ int band_lda(int n) { return (n % 2 == 0) ? n + 1 : n + 2; }

// Bloch sum of a [R][row][col] stack into M (row stride ld), with the
// triangular-storage symmetrisation of SystemTB::hamiltonian (SystemTB.cpp:69-72);
// W is scratch of the same shape.
__device__ void bloch_sum(const BlockGroup& g, const cd* __restrict__ MR, const cd* ph, int nR, int n, int ld,
                          int triangular, double scale, cd* M, cd* W) {
  for (int t = g.rank(); t < n * n; t += g.size()) {
    const int i = t / n, j = t - i * n;
    cd h = mk(0, 0);
    for (int r = 0; r < nR; r++) h = h + MR[(int64_t)r * n * n + t] * ph[r];
    M[i * ld + j] = scale * h;
  }
  g.sync();
  if (triangular) {
    // h.diag() -= h.diag()/2; h += h^dagger
    for (int t = g.rank(); t < n * n; t += g.size()) {
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
    for (int t = g.rank(); t < n * n; t += g.size()) {
      const int i = t / n, j = t - i * n;
      M[i * ld + j] = W[i * ld + j];
    }
    g.sync();
  }
}

// C = A B (n x n, row stride ld).
__device__ void group_matmul(const BlockGroup& g, const cd* A, const cd* B, cd* C, int n, int ld) {
  for (int t = g.rank(); t < n * n; t += g.size()) {
    const int i = t / n, j = t - i * n;
    cd s = mk(0, 0);
    for (int m = 0; m < n; m++) s = s + A[i * ld + m] * B[m * ld + j];
    C[i * ld + j] = s;
  }
  g.sync();
}

extern "C" __global__ void __launch_bounds__(BAND_THREADS)
band_solve_kernel(BandParams bp, const double* __restrict__ kpoints, const double* __restrict__ cellsR,
                  const cd* __restrict__ HR, const cd* __restrict__ SR, double* __restrict__ eigval,
                  cd* __restrict__ eigvec, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = bp.norb, lda = band_lda(n);
  const int nmat = bp.has_overlap ? 3 : 2;
  const size_t matsz = (size_t)n * lda;
  cd* A = reinterpret_cast<cd*>(smem_raw);
  cd* V = A + matsz;
  cd* B = V + (nmat == 3 ? matsz : 0);          // third matrix (overlap only)
  JacobiRot* rot = reinterpret_cast<JacobiRot*>(A + nmat * matsz);
  cd* ph = reinterpret_cast<cd*>(rot + (n / 2 + 2));
  double* scratch = reinterpret_cast<double*>(ph + bp.nR);       // 64 doubles
  int* perm = reinterpret_cast<int*>(scratch + 64);
  __shared__ int s_flag;

  const int k = blockIdx.x;
  BlockGroup g;
  const int tid = threadIdx.x;
  const double kx = kpoints[3 * k] + bp.shift[0];
  const double ky = kpoints[3 * k + 1] + bp.shift[1];
  const double kz = kpoints[3 * k + 2] + bp.shift[2];
  for (int r = tid; r < bp.nR; r += BAND_THREADS) {
    double s, c;
    sincos(kx * cellsR[3 * r] + ky * cellsR[3 * r + 1] + kz * cellsR[3 * r + 2], &s, &c);
    ph[r] = mk(c, s);
  }
  if (tid == 0) s_flag = 0;
  g.sync();
  if (bp.has_overlap) {
    // B = h (scaled), A = S(k); Jacobi of S into (A, V); A = X = V diag(l^-1/2) V^H; h' = X h X -> A
    bloch_sum(g, HR, ph, bp.nR, n, lda, bp.triangular, bp.is_au ? 27.2 : 1.0, B, V);
    bloch_sum(g, SR, ph, bp.nR, n, lda, bp.triangular, 1.0, A, V);
    const int sw = jacobi_eigh(g, A, lda, V, lda, n, rot, scratch, bp.max_sweeps, 1e-15);
    if (sw > bp.max_sweeps && tid == 0) atomicOr(status, XATU_DEVERR_NOCONV);
    for (int i = tid; i < n; i += BAND_THREADS)
      if (!(A[i * lda + i].x > 0.0)) s_flag = 1;
    g.sync();
    if (s_flag) {
      if (tid == 0) atomicOr(status, XATU_DEVERR_OVERLAP);
      return;
    }
    // l^-1/2 into scratch (the rotation array is free between the two solves)
    double* lis = reinterpret_cast<double*>(rot);
    for (int i = tid; i < n; i += BAND_THREADS) lis[i] = 1.0 / sqrt(A[i * lda + i].x);
    g.sync();
    // A = X = V diag(l^-1/2) V^H
    for (int t = tid; t < n * n; t += BAND_THREADS) {
      const int i = t / n, j = t - i * n;
      cd sum = mk(0, 0);
      for (int m = 0; m < n; m++) sum = sum + lis[m] * (V[i * lda + m] * conj(V[j * lda + m]));
      A[i * lda + j] = sum;
    }
    g.sync();
    group_matmul(g, A, B, V, n, lda);   // V = X h
    group_matmul(g, V, A, B, n, lda);   // B = X h X
    for (int t = tid; t < n * n; t += BAND_THREADS) {
      const int i = t / n, j = t - i * n;
      A[i * lda + j] = B[i * lda + j];
    }
    g.sync();
  } else {
    bloch_sum(g, HR, ph, bp.nR, n, lda, bp.triangular, 1.0, A, V);
  }
  // NaN guard on the input matrix
  for (int t = tid; t < n * n; t += BAND_THREADS) {
    const int i = t / n, j = t - i * n;
    const cd a = A[i * lda + j];
    if (!(isfinite(a.x) && isfinite(a.y))) s_flag = 1;
  }
  g.sync();
  if (s_flag) {
    if (tid == 0) atomicOr(status, XATU_DEVERR_NAN);
    return;
  }
  const int sweeps = jacobi_eigh(g, A, lda, V, lda, n, rot, scratch, bp.max_sweeps, 1e-15);
  if (sweeps > bp.max_sweeps && tid == 0) atomicOr(status, XATU_DEVERR_NOCONV);
  jacobi_sort(g, A, lda, n, perm);
  // fixGlobalPhase on the selected columns: one warp per band
  const int warp = tid >> 5, lane = tid & 31;
  for (int b = warp; b < bp.nb; b += BAND_THREADS / 32) {
    const int col = perm[bp.band_list[b]];
    double sr = 0.0, si = 0.0;
    for (int o = lane; o < n; o += 32) {
      sr += V[o * lda + col].x;
      si += V[o * lda + col].y;
    }
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

extern "C" size_t band_solve_smem(int norb, int nR, int has_overlap) {
  const int n = norb, lda = band_lda(n);
  const size_t matsz = (size_t)n * lda;
  return (has_overlap ? 3 : 2) * matsz * sizeof(cd) + (size_t)(n / 2 + 2) * sizeof(JacobiRot) +
         (size_t)nR * sizeof(cd) + 64 * sizeof(double) + (size_t)(n + 1) * sizeof(int);
}
