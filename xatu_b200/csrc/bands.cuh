// Device-side band eigensystem of one k point, shared by the band solve
// (bands.cu) and the adjoint of the band solve (adjoint.cu).
//
//   H(k) = sum_R H(R) e^{i k.R}           (SystemTB::hamiltonian, SystemTB.cpp:60-75,
//                                          triangular storage symmetrised as :69-72)
//   H(k) C = C diag(E)                     (SystemTB::solveBands, SystemTB.cpp:113-125)
// With overlap matrices the basis is orthogonalised first (Loewdin,
// SystemTB::orthogonalize_hamiltonian, SystemTB.cpp:136-156):
//   S(k) = sum_R S(R) e^{i k.R},  S = U diag(l) U^H,  X = U diag(l^-1/2) U^H,
//   h <- X h X  (h scaled by 27.2 first when the model is in Hartree).
// One CTA per k point, matrices in shared memory, FP64 two-phase Jacobi.
#pragma once
#include "jacobi.cuh"
#include "params.h"

// Odd row pitch (in 16-byte elements) spreads the 2x2-block accesses over the banks.
__host__ __device__ __forceinline__ int band_lda(int n) { return (n % 2 == 0) ? n + 1 : n + 2; }

// Shared-memory layout of one k point: A, V (and B with overlap) n x lda,
// the rotation table, the Bloch phases, a reduction scratch and the sort
// permutation.
struct BandSmem {
  cd* A;
  cd* V;
  cd* B;
  JacobiRot* rot;
  cd* ph;
  double* scratch;   // 64 doubles
  int* perm;         // n + 1
  int lda;
  size_t matsz;
};

__host__ __device__ inline size_t band_smem_bytes(int n, int nR, int has_overlap) {
  const size_t matsz = (size_t)n * band_lda(n);
  return (has_overlap ? 3 : 2) * matsz * sizeof(cd) + (size_t)(n / 2 + 2) * sizeof(JacobiRot) +
         (size_t)nR * sizeof(cd) + 64 * sizeof(double) + (size_t)(n + 1) * sizeof(int);
}

__device__ inline BandSmem band_smem_layout(unsigned char* raw, int n, int nR, int has_overlap) {
  BandSmem s;
  s.lda = band_lda(n);
  s.matsz = (size_t)n * s.lda;
  s.A = reinterpret_cast<cd*>(raw);
  s.V = s.A + s.matsz;
  s.B = has_overlap ? s.V + s.matsz : nullptr;
  s.rot = reinterpret_cast<JacobiRot*>(s.A + (has_overlap ? 3 : 2) * s.matsz);
  s.ph = reinterpret_cast<cd*>(s.rot + (n / 2 + 2));
  s.scratch = reinterpret_cast<double*>(s.ph + nR);
  s.perm = reinterpret_cast<int*>(s.scratch + 64);
  return s;
}

// Bloch sum of a [R][row][col] stack into M (row stride ld), with the
// triangular-storage symmetrisation of SystemTB::hamiltonian (SystemTB.cpp:69-72);
// W is scratch of the same shape.
__device__ inline void bloch_sum(const BlockGroup& g, const cd* __restrict__ MR, const cd* ph, int nR, int n, int ld,
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
__device__ inline void group_matmul(const BlockGroup& g, const cd* A, const cd* B, cd* C, int n, int ld) {
  for (int t = g.rank(); t < n * n; t += g.size()) {
    const int i = t / n, j = t - i * n;
    cd s = mk(0, 0);
    for (int m = 0; m < n; m++) s = s + A[i * ld + m] * B[m * ld + j];
    C[i * ld + j] = s;
  }
  g.sync();
}

// Eigensystem of the Bloch Hamiltonian at k + bp.shift.  On success returns
// the matrix whose diagonal holds the eigenvalues (in Jacobi order); V holds
// the eigenvectors as columns and perm[rank] the column of the rank-th
// smallest eigenvalue.  With overlap, A holds X = S^{-1/2} on return.
// Returns nullptr (status flags set) on a non-positive overlap eigenvalue or a
// non-finite matrix.  s_flag: a shared int.
__device__ inline cd* band_eigensystem(const BlockGroup& g, const BandParams& bp, int k,
                                       const double* __restrict__ kpoints, const double* __restrict__ cellsR,
                                       const cd* __restrict__ HR, const cd* __restrict__ SR, const BandSmem& s,
                                       int* __restrict__ status, int* s_flag) {
  const int n = bp.norb, lda = s.lda;
  const int tid = g.rank(), nt = g.size();
  const double kx = kpoints[3 * k] + bp.shift[0];
  const double ky = kpoints[3 * k + 1] + bp.shift[1];
  const double kz = kpoints[3 * k + 2] + bp.shift[2];
  for (int r = tid; r < bp.nR; r += nt) {
    double sn, cs;
    sincos(kx * cellsR[3 * r] + ky * cellsR[3 * r + 1] + kz * cellsR[3 * r + 2], &sn, &cs);
    s.ph[r] = mk(cs, sn);
  }
  if (tid == 0) *s_flag = 0;
  g.sync();
  cd* M = s.A;   // the matrix diagonalised
  if (bp.has_overlap) {
    // B = h (scaled), A = S(k); Jacobi of S into (A, V); A = X = V diag(l^-1/2) V^H; B = X h X
    bloch_sum(g, HR, s.ph, bp.nR, n, lda, bp.triangular, bp.is_au ? 27.2 : 1.0, s.B, s.V);
    bloch_sum(g, SR, s.ph, bp.nR, n, lda, bp.triangular, 1.0, s.A, s.V);
    const int sw = jacobi_eigh(g, s.A, lda, s.V, lda, n, s.rot, s.scratch, bp.max_sweeps, 1e-15);
    if (sw > bp.max_sweeps && tid == 0) atomicOr(status, XATU_DEVERR_NOCONV);
    for (int i = tid; i < n; i += nt)
      if (!(s.A[i * lda + i].x > 0.0)) *s_flag = 1;
    g.sync();
    if (*s_flag) {
      if (tid == 0) atomicOr(status, XATU_DEVERR_OVERLAP);
      return nullptr;
    }
    // l^-1/2 into the rotation table (free between the two solves)
    double* lis = reinterpret_cast<double*>(s.rot);
    for (int i = tid; i < n; i += nt) lis[i] = 1.0 / sqrt(s.A[i * lda + i].x);
    g.sync();
    for (int t = tid; t < n * n; t += nt) {
      const int i = t / n, j = t - i * n;
      cd sum = mk(0, 0);
      for (int m = 0; m < n; m++) sum = sum + lis[m] * (s.V[i * lda + m] * conj(s.V[j * lda + m]));
      s.A[i * lda + j] = sum;
    }
    g.sync();
    group_matmul(g, s.A, s.B, s.V, n, lda);   // V = X h
    group_matmul(g, s.V, s.A, s.B, n, lda);   // B = X h X
    M = s.B;
  } else {
    bloch_sum(g, HR, s.ph, bp.nR, n, lda, bp.triangular, 1.0, s.A, s.V);
  }
  for (int t = tid; t < n * n; t += nt) {
    const int i = t / n, j = t - i * n;
    const cd a = M[i * lda + j];
    if (!(isfinite(a.x) && isfinite(a.y))) *s_flag = 1;
  }
  g.sync();
  if (*s_flag) {
    if (tid == 0) atomicOr(status, XATU_DEVERR_NAN);
    return nullptr;
  }
  const int sweeps = jacobi_eigh(g, M, lda, s.V, lda, n, s.rot, s.scratch, bp.max_sweeps, 1e-15);
  if (sweeps > bp.max_sweeps && tid == 0) atomicOr(status, XATU_DEVERR_NOCONV);
  jacobi_sort(g, M, lda, n, s.perm);
  return M;
}
