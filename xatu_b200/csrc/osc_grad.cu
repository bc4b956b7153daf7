// Gradient of the summed oscillator strength of the excitons in an energy window,
//   F = sum_{n in W} sum_{j = x, y, z} |vme_ex_j(n)|^2,   vme_ex_j(n) = sum_i X_in v_j(i)
// (ResultTB::excitonOscillatorStrength, ResultTB.cpp:242-298, skubo_w.f90:175-330, summed over the
// window W = {n : e_lo <= E_n <= e_hi}), with respect to r0, eps_m and eps_s.  The reference has no
// derivative code.
//
// The velocity matrix elements v do not depend on the potential, so only the eigenvectors move:
//   dX_n = sum_{m != n} X_m (X_m^H dH X_n) / (E_n - E_m).
// Rotations inside W leave F unchanged (F = sum_j v_j^T P_W conj(v_j)), so only m outside W count:
//   dF = sum_{n in W} 2 Re(lambda_n^H dH X_n),
//   lambda_n = sum_{m not in W} X_m (X_m^H b_n) / (E_n - E_m),   b_n = sum_j vme_ex_j(n) conj(v_j).
// Everything is FP64 on the device: all eigenpairs by the dense solver, the tall products by ZGEMM
// (library GEMMs), dH/dtheta assembled by the BSE assembly kernel from derivative tables with the band
// energies set to zero.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.h"
#include "kernels.h"

__global__ void og_conj_kernel(cd* v, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    v[t].y = -v[t].y;
}

// C[m, n] *= 1 / (E[n0 + n] - E[m]) for m outside [n0, n0 + nw), 0 inside; near-degenerate pairs flagged.
__global__ void og_scale_kernel(cd* C, long long N, int n0, int nw, const double* __restrict__ E, int* status) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N * nw;
       t += (long long)gridDim.x * blockDim.x) {
    const int n = (int)(t / N);
    const long long m = t - (long long)n * N;
    if (m >= n0 && m < n0 + nw) {
      C[t] = mk(0, 0);
      continue;
    }
    const double d = E[n0 + n] - E[m];
    if (fabs(d) < 1e-12) {
      atomicOr(status, XATU_DEVERR_DEGEN);
      C[t] = mk(0, 0);
      continue;
    }
    C[t] = (1.0 / d) * C[t];
  }
}

static xatu_status og_zgemm(xatu_ctx* ctx, cublasOperation_t ta, cublasOperation_t tb, long long m, long long n,
                            long long k, const cd* A, long long lda, const cd* B, long long ldb, cd* C, long long ldc,
                            bool accumulate = false) {
  static const cuDoubleComplex one = {1.0, 0.0}, zero = {0.0, 0.0};
  cublasStatus_t s = cublasZgemm(ctx->blas, ta, tb, (int)m, (int)n, (int)k, &one,
                                 reinterpret_cast<const cuDoubleComplex*>(A), (int)lda,
                                 reinterpret_cast<const cuDoubleComplex*>(B), (int)ldb, accumulate ? &one : &zero,
                                 reinterpret_cast<cuDoubleComplex*>(C), (int)ldc);
  if (s != CUBLAS_STATUS_SUCCESS) return xatu_fail(ctx, XATU_ERR_CUDA, "cublasZgemm failed");
  return XATU_OK;
}

#define OG_TRY(x)                 \
  do {                            \
    xatu_status s__ = (x);        \
    if (s__ != XATU_OK) return s__; \
  } while (0)

// dH/dtheta (FP64, row-major N x N, band energies zero) into out.
static xatu_status og_build_derivative(xatu_ctx* ctx, int which, cd* out) {
  OG_TRY(xatu_derivative_tables(ctx, which));
  const long long N = ctx->N;
  const int na = ctx->natoms;
  AsmParams p;
  AsmInputs in;
  AsmOutputs o;
  xatu_assembly_setup(ctx, nullptr, &p, &in, &o);
  p.scissor = 0.0;
  XATU_CK(ctx->dv_tmp.ensure((size_t)ctx->nk * ctx->nb * sizeof(double)));
  XATU_CK(cudaMemsetAsync(ctx->dv_tmp.p, 0, (size_t)ctx->nk * ctx->nb * sizeof(double), ctx->stream));
  in.eigval = ctx->dv_tmp.as<double>();
  in.eigvalQ = ctx->dv_tmp.as<double>();
  in.table = ctx->d_adjdtable.as<cd>();
  if (ctx->exchange) {
    XATU_CK(ctx->d_exL.ensure((size_t)N * na * sizeof(cd)));
    XATU_CK(ctx->d_exR.ensure((size_t)N * na * sizeof(cd)));
    exchange_vectors_kernel<<<(int)((N + 127) / 128), 128, 0, ctx->stream>>>(
        (int)N, ctx->nv, ctx->nc, ctx->nb, ctx->norb, na, ctx->d_orboff.as<int>(), ctx->d_eigvec.as<cd>(),
        ctx->d_eigvecQ.as<cd>(), ctx->d_adjdVX.as<cd>(), nullptr, ctx->d_exL.as<cd>(), ctx->d_exR.as<cd>());
    ctx->launches++;
    XATU_CK_LAUNCH("exchange_vectors_kernel (derivative)");
  }
  o.H = out;
  int path = -1;
  XATU_CK(xatu_launch_assembly(p, in, o, false, false, ctx->stream, &path));
  ctx->launches++;
  return XATU_OK;
}

extern "C" xatu_status xatu_oscillator_window_gradient(xatu_ctx* ctx, double e_lo, double e_hi, int* nwindow,
                                                       double* F, double* grad_params, double* grad_hamiltonian) {
  if (!ctx || !F) return xatu_fail(ctx, XATU_ERR_INVALID, "bad argument");
  cudaSetDevice(ctx->device);
  if (ctx->built_prec != XATU_PREC_FP64) return xatu_fail(ctx, XATU_ERR_STATE, "needs an FP64 build (xatu_bse_build)");
  if (ctx->custom_basis) return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "needs the full e-h basis");
  if (!(e_hi >= e_lo)) return xatu_fail(ctx, XATU_ERR_INVALID, "empty energy window");
  if (grad_hamiltonian && (!ctx->bands_from_model || ctx->qnonzero || ctx->triangular))
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED,
                     "hopping gradient of the oscillator strength needs bands from the model, Q = 0 and full storage");
  const long long N = ctx->N;
  cudaStream_t st = ctx->stream;
  if (!ctx->blas) {
    if (cublasCreate(&ctx->blas) != CUBLAS_STATUS_SUCCESS) return xatu_fail(ctx, XATU_ERR_CUDA, "cublasCreate failed");
  }
  cublasSetStream(ctx->blas, st);
  cublasSetPointerMode(ctx->blas, CUBLAS_POINTER_MODE_HOST);
  // all eigenpairs (eigenvectors recomputed here, columns of dv_V)
  OG_TRY(xatu_dense_eig_device(ctx, true));
  std::vector<double> E(N);
  XATU_CK(cudaMemcpyAsync(E.data(), ctx->dv_diagH.p, N * sizeof(double), cudaMemcpyDeviceToHost, st));
  XATU_CK(cudaStreamSynchronize(st));
  int n0 = 0;
  while (n0 < N && E[n0] < e_lo) n0++;
  int n1 = n0;
  while (n1 < N && E[n1] <= e_hi) n1++;
  const int nw = n1 - n0;
  if (nwindow) *nwindow = nw;
  *F = 0.0;
  if (grad_params)
    for (int q = 0; q < 3; q++) grad_params[q] = 0.0;
  if (grad_hamiltonian) memset(grad_hamiltonian, 0, 2 * sizeof(double) * (size_t)ctx->nR * ctx->norb * ctx->norb);
  if (nw == 0) return XATU_OK;
  const cd* X = ctx->dv_V.as<cd>();
  const cd* XW = X + (long long)n0 * N;
  // v (3 x N row-major = N x 3 column-major), Z = X_W^T v (nw x 3): Z[n, j] = vme_ex_j(n)
  const size_t need = (size_t)3 * N + (size_t)nw * 3 + 3 * (size_t)N * nw;
  XATU_CK(ctx->dv_R.ensure(need * sizeof(cd)));
  cd* v = ctx->dv_R.as<cd>();
  cd* Z = v + 3 * N;
  cd* B = Z + (size_t)nw * 3;          // N x nw
  cd* C = B + (size_t)N * nw;          // N x nw
  cd* Lam = C + (size_t)N * nw;        // N x nw
  OG_TRY(xatu_vme_enqueue(ctx, v));
  OG_TRY(og_zgemm(ctx, CUBLAS_OP_T, CUBLAS_OP_N, nw, 3, N, XW, N, v, N, Z, nw));
  std::vector<cd> Zh((size_t)nw * 3);
  XATU_CK(cudaMemcpyAsync(Zh.data(), Z, Zh.size() * sizeof(cd), cudaMemcpyDeviceToHost, st));
  XATU_CK(cudaStreamSynchronize(st));
  double f = 0.0;
  for (const cd& z : Zh) f += nrm2(z);
  *F = f;
  if (!grad_params && !grad_hamiltonian) return XATU_OK;
  // b_n = sum_j vme_ex_j(n) conj(v_j): B = conj(v Z^H)
  OG_TRY(og_zgemm(ctx, CUBLAS_OP_N, CUBLAS_OP_C, N, nw, 3, v, N, Z, nw, B, N));
  og_conj_kernel<<<592, 256, 0, st>>>(B, N * nw);
  ctx->launches++;
  XATU_CK_LAUNCH("og_conj_kernel");
  // lambda = X diag-scaled (X^H B)
  OG_TRY(og_zgemm(ctx, CUBLAS_OP_C, CUBLAS_OP_N, N, nw, N, X, N, B, N, C, N));
  XATU_CK(cudaMemsetAsync(ctx->d_status.p, 0, sizeof(int), st));
  og_scale_kernel<<<592, 256, 0, st>>>(C, N, n0, nw, ctx->dv_diagH.as<double>(), ctx->d_status.as<int>());
  ctx->launches++;
  XATU_CK_LAUNCH("og_scale_kernel");
  OG_TRY(og_zgemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, N, nw, N, X, N, C, N, Lam, N));
  {
    xatu_status s0 = xatu_check_device_status(ctx, "oscillator window gradient");
    if (s0 != XATU_OK) return s0;
  }
  // dF/dtheta = 2 Re <lambda, dH X_W> for theta = r0, eps (= eps_m = eps_s)
  XATU_CK(ctx->dv_W.ensure((size_t)N * N * sizeof(cd)));
  cd* dH = ctx->dv_W.as<cd>();
  if (grad_params) {
    for (int which = 0; which < 2; which++) {
      OG_TRY(og_build_derivative(ctx, which, dH));
      // G = dH X_W; dH is row-major, i.e. the column-major buffer holds dH^T
      OG_TRY(og_zgemm(ctx, CUBLAS_OP_T, CUBLAS_OP_N, N, nw, N, dH, N, XW, N, C, N));
      cuDoubleComplex dot;
      if (cublasZdotc(ctx->blas, (int)(N * nw), reinterpret_cast<const cuDoubleComplex*>(Lam), 1,
                      reinterpret_cast<const cuDoubleComplex*>(C), 1, &dot) != CUBLAS_STATUS_SUCCESS)
        return xatu_fail(ctx, XATU_ERR_CUDA, "cublasZdotc failed");
      const double g = 2.0 * dot.x;
      if (which == 0) {
        grad_params[0] = g;
      } else {
        grad_params[1] = g;
        grad_params[2] = g;
      }
    }
    XATU_CK(cudaStreamSynchronize(st));
    OG_TRY(xatu_check_device_status(ctx, "oscillator window gradient (derivative assembly)"));
  }
  if (!grad_hamiltonian) return XATU_OK;
  // hopping matrices.  (1) through the eigenvectors: dF = sum_ij Y_ij dH_ij with the Hermitian weight
  // Y = conj(Lambda) X_W^T + conj(X_W) Lambda^T, stored row-major (= the column-major X_W Lambda^H + Lambda X_W^H)
  cd* Yr = dH;
  OG_TRY(og_zgemm(ctx, CUBLAS_OP_N, CUBLAS_OP_C, N, N, nw, XW, N, Lam, N, Yr, N));
  OG_TRY(og_zgemm(ctx, CUBLAS_OP_N, CUBLAS_OP_C, N, N, nw, Lam, N, XW, N, Yr, N, true));
  const int na = ctx->natoms, nk = ctx->nk, nb = ctx->nb, norb = ctx->norb;
  cd* Zc = nullptr;
  cd* Zv = nullptr;
  XATU_CK(ctx->dv_tmp.ensure((size_t)2 * N * na * sizeof(cd) + (size_t)N * 3 * sizeof(cd) + 64));
  if (ctx->exchange) {
    XATU_CK(ctx->d_exL.ensure((size_t)N * na * sizeof(cd)));
    XATU_CK(ctx->d_exR.ensure((size_t)N * na * sizeof(cd)));
    exchange_vectors_kernel<<<(int)((N + 127) / 128), 128, 0, st>>>(
        (int)N, ctx->nv, ctx->nc, nb, norb, na, ctx->d_orboff.as<int>(), ctx->d_eigvec.as<cd>(), ctx->d_eigvecQ.as<cd>(),
        ctx->d_VX.as<cd>(), nullptr, ctx->d_exL.as<cd>(), ctx->d_exR.as<cd>());
    ctx->launches++;
    XATU_CK_LAUNCH("exchange_vectors_kernel");
    // L[i * na + a] is the column-major na x N matrix M; Zc = Y M^H = Yt^T M^H, Zv = Y^T M^T = Yt M^T
    Zc = ctx->dv_tmp.as<cd>();
    Zv = Zc + (size_t)N * na;
    OG_TRY(og_zgemm(ctx, CUBLAS_OP_T, CUBLAS_OP_C, N, na, N, Yr, N, ctx->d_exL.as<cd>(), na, Zc, N));
    OG_TRY(og_zgemm(ctx, CUBLAS_OP_N, CUBLAS_OP_T, N, na, N, Yr, N, ctx->d_exL.as<cd>(), na, Zv, N));
  }
  XATU_CK(ctx->d_adjCbar.ensure((size_t)nk * nb * norb * sizeof(cd)));
  XATU_CK(ctx->d_adjEbar.ensure((size_t)nk * nb * sizeof(double)));
  cd* cbar = ctx->d_adjCbar.as<cd>();
  double* ebar = ctx->d_adjEbar.as<double>();
  OG_TRY(xatu_adjoint_weighted(ctx, Yr, Zc, Zv, cbar, ebar));
  // (2) through the velocity matrix elements: vbar = dF/dconj(v) = conj(X_W conj(Z))
  cd* vbar = ctx->dv_tmp.as<cd>() + (size_t)2 * N * na;
  {
    std::vector<cd> Zcj(Zh.size());
    for (size_t q = 0; q < Zh.size(); q++) Zcj[q] = conj(Zh[q]);
    XATU_CK(cudaMemcpyAsync(Z, Zcj.data(), Zcj.size() * sizeof(cd), cudaMemcpyHostToDevice, st));
    OG_TRY(og_zgemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, N, 3, nw, XW, N, Z, nw, vbar, N));
    og_conj_kernel<<<592, 256, 0, st>>>(vbar, N * 3);
    ctx->launches++;
    XATU_CK_LAUNCH("og_conj_kernel");
    XATU_CK(cudaStreamSynchronize(st));   // Zcj leaves scope
  }
  XATU_CK(ctx->d_oscG.ensure((size_t)2 * nk * norb * norb * sizeof(cd)));
  OG_TRY(xatu_vme_adjoint_enqueue(ctx, vbar, cbar, ebar, ctx->d_oscG.as<cd>(), nullptr));
  // bands -> G(R), then the direct H(R) part of the velocity matrix elements
  OG_TRY(xatu_adjoint_bands_to_hoppings(ctx, 1, cbar, ebar));
  OG_TRY(xatu_vme_hop_enqueue(ctx, ctx->d_oscG.as<cd>(), ctx->d_adjG.as<cd>()));
  XATU_CK(cudaMemcpyAsync(grad_hamiltonian, ctx->d_adjG.p, (size_t)ctx->nR * norb * norb * sizeof(cd),
                          cudaMemcpyDeviceToHost, st));
  XATU_CK(cudaStreamSynchronize(st));
  return xatu_check_device_status(ctx, "oscillator window gradient (hopping matrices)");
}
