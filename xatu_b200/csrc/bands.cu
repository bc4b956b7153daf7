// Single-particle band solve on the device (ExcitonTB::initializeResultsH0,
// ExcitonTB.cpp:737-758): for every k of the exciton basis (and k + Q) the
// Bloch Hamiltonian is diagonalised (bands.cuh), then
//   column sums of C made real positive    (ExcitonTB::fixGlobalPhase, ExcitonTB.cpp:673-683)
//   keep the columns of the band list      (ExcitonTB.cpp:741-742)
// With overlap the eigenvectors of X h X are kept as they are, as in the reference.
// One CTA of BAND_THREADS threads per k point.
#include "bands.cuh"

#define BAND_THREADS 128

extern "C" __global__ void __launch_bounds__(BAND_THREADS)
band_solve_kernel(BandParams bp, const double* __restrict__ kpoints, const double* __restrict__ cellsR,
                  const cd* __restrict__ HR, const cd* __restrict__ SR, double* __restrict__ eigval,
                  cd* __restrict__ eigvec, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_flag;
  const int n = bp.norb;
  const BandSmem s = band_smem_layout(smem_raw, n, bp.nR, bp.has_overlap);
  const int lda = s.lda;
  const int k = blockIdx.x;
  BlockGroup g;
  const cd* M = band_eigensystem(g, bp, k, kpoints, cellsR, HR, SR, s, status, &s_flag);
  if (!M) return;
  // fixGlobalPhase on the selected columns: one warp per band
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int b = warp; b < bp.nb; b += BAND_THREADS / 32) {
    const int col = s.perm[bp.band_list[b]];
    double sr = 0.0, si = 0.0;
    for (int o = lane; o < n; o += 32) {
      sr += s.V[o * lda + col].x;
      si += s.V[o * lda + col].y;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, off);
      si += __shfl_xor_sync(0xffffffffu, si, off);
    }
    const double ang = atan2(si, sr);
    double sn, cs;
    sincos(-ang, &sn, &cs);
    const cd f = mk(cs, sn);
    cd* out = eigvec + ((int64_t)k * bp.nb + b) * n;
    for (int o = lane; o < n; o += 32) out[o] = s.V[o * lda + col] * f;
    if (lane == 0) eigval[(int64_t)k * bp.nb + b] = M[col * lda + col].x;
  }
}

extern "C" size_t band_solve_smem(int norb, int nR, int has_overlap) {
  return band_smem_bytes(norb, nR, has_overlap);
}
