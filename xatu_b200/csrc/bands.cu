// Single-particle band solve on the device (ExcitonTB::initializeResultsH0,
// ExcitonTB.cpp:737-758): for every k of the exciton basis (and k + Q),
//   H(k) = sum_R H(R) e^{i k.R}           (SystemTB::hamiltonian, SystemTB.cpp:60-75,
//                                          triangular storage symmetrised as :69-72)
//   H(k) C = C diag(E), E ascending        (SystemTB::solveBands, SystemTB.cpp:113-125)
//   column sums of C made real positive    (ExcitonTB::fixGlobalPhase, ExcitonTB.cpp:673-683)
//   keep the columns of the band list      (ExcitonTB.cpp:741-742)
// One warp per k point, the matrix in shared memory, FP64 Jacobi.
#include "jacobi.cuh"
#include "params.h"

__device__ __forceinline__ int band_lda(int n) { return n + 1; }

extern "C" __global__ void band_solve_kernel(BandParams bp, const double* __restrict__ kpoints,
                                             const double* __restrict__ cellsR, const cd* __restrict__ HR,
                                             double* __restrict__ eigval, cd* __restrict__ eigvec,
                                             int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = bp.norb, lda = band_lda(n);
  const int warps = blockDim.x >> 5;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // per-warp shared layout
  const size_t matsz = (size_t)n * lda;
  const size_t per_warp = 2 * matsz * sizeof(cd) + (size_t)(n / 2 + 2) * sizeof(JacobiRot) +
                          (size_t)bp.nR * sizeof(cd) + (size_t)(n + 1) * sizeof(int);
  const size_t per_warp_al = (per_warp + 15) & ~(size_t)15;
  unsigned char* base = smem_raw + per_warp_al * w;
  cd* A = reinterpret_cast<cd*>(base);
  cd* V = A + matsz;
  JacobiRot* rot = reinterpret_cast<JacobiRot*>(V + matsz);
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
  for (int t = lane; t < n * n; t += 32) {
    const int i = t / n, j = t - i * n;
    cd h = mk(0, 0);
    for (int r = 0; r < bp.nR; r++) h = h + HR[(int64_t)r * n * n + t] * ph[r];
    A[i * lda + j] = h;
  }
  g.sync();
  if (bp.triangular) {
    // h.diag() -= h.diag()/2; h += h^dagger  (V is free scratch until the solve)
    for (int t = lane; t < n * n; t += 32) {
      const int i = t / n, j = t - i * n;
      if (i == j) {
        const cd d = A[i * lda + i];
        const cd dh = mk(d.x - d.x / 2, d.y - d.y / 2);
        V[i * lda + j] = dh + conj(dh);
      } else {
        V[i * lda + j] = A[i * lda + j] + conj(A[j * lda + i]);
      }
    }
    g.sync();
    for (int t = lane; t < n * n; t += 32) {
      const int i = t / n, j = t - i * n;
      A[i * lda + j] = V[i * lda + j];
    }
    g.sync();
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
  const int sweeps = jacobi_eigh(g, A, lda, V, lda, n, rot, nullptr, bp.max_sweeps, 1e-15);
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

extern "C" size_t band_solve_smem_per_warp(int norb, int nR) {
  const int n = norb, lda = n + 1;
  const size_t matsz = (size_t)n * lda;
  const size_t per_warp = 2 * matsz * sizeof(cd) + (size_t)(n / 2 + 2) * sizeof(JacobiRot) +
                          (size_t)nR * sizeof(cd) + (size_t)(n + 1) * sizeof(int);
  return (per_warp + 15) & ~(size_t)15;
}
