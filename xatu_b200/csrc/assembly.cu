// BSE matrix assembly (ExcitonTB::BShamiltonian, ExcitonTB.cpp:840-921).
//
// For e-h states i = (k, c, v) and j = (k', c', v') (row order of
// Exciton::createBasis, Exciton.tpp:128-147: i = k*nc*nv + c*nv + v):
//
//   rho1_a(c, c') = sum_{o in a} conj(CQ_k[c]_o)  CQ_k'[c']_o
//   rho2_b(v', v) = sum_{o in b} conj(C_k'[v']_o) C_k[v]_o
//   D_ij = sum_ab rho1_a V_ab rho2_b
//     V = motif FT at the mesh point equivalent to k' - k     (real space, :893-895)
//     V = G-summed kernel W(k - k')                           (reciprocal space, :903)
//   X_ij = sum_a L_a(i) R_a(j)                                (exchange, :897 / :905)
//   H_ij = -(D - X) (i < j),  H_ji = conj(H_ij),
//   H_ii = 2 Re[(scissor + E_c - E_v)/2 - (D - X)/2]          (:909-919)
//
// Fast path (assembly_tile.cuh): one thread per (k, k') pair of a tile of k points; the
// rho1 / rho2 factors are formed once per pair (not once per element as in
// the reference) from band coefficients staged in shared memory
// ([band][orbital][k] layout so the k' threads of a warp read consecutive
// words).  Only tiles with kblock <= kblock' are launched; the mirror block is
// written as the conjugate transpose, so H is exactly Hermitian.
//
// Precision: T = double writes the complex128 matrix (parity mode).  T = float
// writes the mixed-precision form used by the tensor-core solver: the band
// energies scissor + E_c - E_v as an FP64 diagonal, and the interaction
// kernel K = H - diag in two BF16 planes, K ~= K_hi + K_lo.
#include "assembly_tile.cuh"
#include "kernels.h"

// Generic fallback: one thread per element (i, j), i <= j, any band window.
template <typename T, bool MIXED>
__global__ void bse_assemble_generic_kernel(AsmParams p, AsmInputs in, AsmOutputs out) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (int64_t i = blockIdx.y; i < p.N; i += gridDim.y) {
  if (j >= p.N || j < i) continue;
  int k, c, v, k2, c2, v2;
  if (in.basis) {
    // caller-given basis rows (ExcitonTB::BShamiltonian(const arma::imat&), ExcitonTB.cpp:840-849)
    k = in.basis[3 * i]; v = in.basis[3 * i + 1]; c = in.basis[3 * i + 2];
    k2 = in.basis[3 * j]; v2 = in.basis[3 * j + 1]; c2 = in.basis[3 * j + 2];
  } else {
    const int ncv = p.nc * p.nv;
    k = (int)(i / ncv);
    k2 = (int)(j / ncv);
    c = (int)((i - (int64_t)k * ncv) / p.nv);
    v = (int)(i - (int64_t)k * ncv - c * p.nv);
    c2 = (int)((j - (int64_t)k2 * ncv) / p.nv);
    v2 = (int)(j - (int64_t)k2 * ncv - c2 * p.nv);
  }
  const cd* Vt = interaction_ptr(p, in, k, k2);
  const cd* Cc = in.eigvecQ + ((int64_t)k * p.nb + p.nv + c) * p.norb;
  const cd* Cc2 = in.eigvecQ + ((int64_t)k2 * p.nb + p.nv + c2) * p.norb;
  const cd* Cv = in.eigvec + ((int64_t)k * p.nb + v) * p.norb;
  const cd* Cv2 = in.eigvec + ((int64_t)k2 * p.nb + v2) * p.norb;
  cd rho2[XATU_MAX_ATOMS];
  for (int b = 0; b < p.na; b++) {
    cd s = mk(0, 0);
    for (int o = p.orb_off[b]; o < p.orb_off[b + 1]; o++) s = s + cmulc(Cv2[o], Cv[o]);
    rho2[b] = s;
  }
  cd d = mk(0, 0);
  for (int a = 0; a < p.na; a++) {
    cd r1 = mk(0, 0);
    for (int o = p.orb_off[a]; o < p.orb_off[a + 1]; o++) r1 = r1 + cmulc(Cc[o], Cc2[o]);
    cd t = mk(0, 0);
    for (int b = 0; b < p.na; b++) t = t + Vt[a * p.na + b] * rho2[b];
    d = d + r1 * t;
  }
  if (p.exchange) {
    for (int a = 0; a < p.na; a++) d = d - in.exL[i * p.na + a] * in.exR[j * p.na + a];
  }
  const double ec = in.eigvalQ[(int64_t)k * p.nb + p.nv + c];
  const double ev = in.eigval[(int64_t)k * p.nb + v];
  cplx<T> dmx = {(T)d.x, (T)d.y};
  write_element<T, MIXED>(p, out, i, j, dmx, ec, ev);
  }
}

// ----------------------------------------------------------------- launchers
template <typename T, bool MIXED>
static cudaError_t launch_generic(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out, cudaStream_t s) {
  dim3 block(128);
  dim3 grid((unsigned)((p.N + 127) / 128), (unsigned)(p.N < 65535 ? p.N : 65535));
  bse_assemble_generic_kernel<T, MIXED><<<grid, block, 0, s>>>(p, in, out);
  return cudaGetLastError();
}

// *path: 0 tile kernel (CUDA cores), 1 generic kernel, 2 tile kernel with the band overlaps on tcgen05, 3 row-panel
// kernel with the band overlaps on tcgen05.
cudaError_t xatu_launch_assembly(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out, bool mixed,
                                 bool force_generic, cudaStream_t s, int* path) {
  if (!force_generic && in.basis == nullptr) {
    bool launched = false, tc = false, panel = false;
    cudaError_t e = mixed ? xatu_dispatch_tile_f32(p, in, out, s, &launched, &tc, &panel)
                          : xatu_dispatch_tile_f64(p, in, out, s, &launched);
    if (e == cudaErrorNotSupported) {
      cudaGetLastError();
      launched = false;
    } else if (e != cudaSuccess) {
      return e;
    }
    if (launched) {
      *path = panel ? 3 : tc ? 2 : 0;
      return cudaSuccess;
    }
  }
  *path = 1;
  return mixed ? launch_generic<float, true>(p, in, out, s) : launch_generic<double, false>(p, in, out, s);
}
