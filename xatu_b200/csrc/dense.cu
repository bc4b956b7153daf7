// Dense FP64 eigensolve of the assembled BSE matrix: the reference's "diag"
// method (arma::eig_sym = LAPACK zheevd, ExcitonTB.cpp:942) on the device,
// via cuSOLVER's divide-and-conquer Hermitian eigensolver (library call; the
// plain FP64 path the mixed-precision Davidson is measured against).
//
// H is stored row-major.  Read column-major the same buffer is H^T = conj(H)
// (H is Hermitian), which has the same eigenvalues and conjugated
// eigenvectors; the eigenvectors are conjugated back on the way out.
#include <string>
#include <vector>

#include "engine.h"

__global__ void conj_columns_kernel(cd* v, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    v[t].y = -v[t].y;
}

// All eigenpairs of the FP64 build on the device: eigenvalues ascending in dv_diagH, eigenvectors as the
// columns of dv_V (column-major N x N; conjugated back when `vectors`).
xatu_status xatu_dense_eig_device(xatu_ctx* ctx, bool vectors) {
  const long long N = ctx->N;
  if (!ctx->solver) {
    if (cusolverDnCreate(&ctx->solver) != CUSOLVER_STATUS_SUCCESS)
      return xatu_fail(ctx, XATU_ERR_CUDA, "cusolverDnCreate failed");
  }
  cusolverDnSetStream(ctx->solver, ctx->stream);
  // work copy of H (the solver overwrites it with eigenvectors)
  const size_t hbytes = (size_t)N * N * sizeof(cd);
  XATU_CK(ctx->dv_V.ensure(hbytes));
  XATU_CK(ctx->dv_diagH.ensure((size_t)N * sizeof(double)));
  XATU_CK(ctx->dv_small.ensure(sizeof(int)));
  XATU_CK(cudaMemcpyAsync(ctx->dv_V.p, ctx->d_H.p, hbytes, cudaMemcpyDeviceToDevice, ctx->stream));
  cusolverDnParams_t params;
  if (cusolverDnCreateParams(&params) != CUSOLVER_STATUS_SUCCESS)
    return xatu_fail(ctx, XATU_ERR_CUDA, "cusolverDnCreateParams failed");
  size_t dev_ws = 0, host_ws = 0;
  const cusolverEigMode_t jobz = vectors ? CUSOLVER_EIG_MODE_VECTOR : CUSOLVER_EIG_MODE_NOVECTOR;
  cusolverStatus_t cs = cusolverDnXsyevd_bufferSize(ctx->solver, params, jobz, CUBLAS_FILL_MODE_LOWER, N, CUDA_C_64F,
                                                     ctx->dv_V.p, N, CUDA_R_64F, ctx->dv_diagH.p, CUDA_C_64F, &dev_ws,
                                                     &host_ws);
  if (cs != CUSOLVER_STATUS_SUCCESS) {
    cusolverDnDestroyParams(params);
    return xatu_fail(ctx, vectors ? XATU_ERR_UNSUPPORTED : XATU_ERR_CUDA,
                     std::string("cusolverDnXsyevd_bufferSize failed (status ") + std::to_string((int)cs) +
                         ") for N = " + std::to_string(N) +
                         (vectors ? " with eigenvectors (request eigenvalues only, or use the Davidson solver)" : ""));
  }
  cudaError_t e = ctx->dv_W.ensure(dev_ws + 16);
  if (e != cudaSuccess) {
    cusolverDnDestroyParams(params);
    return xatu_cuda_fail(ctx, e, "solver workspace");
  }
  std::vector<char> hws(host_ws + 16);
  cs = cusolverDnXsyevd(ctx->solver, params, jobz, CUBLAS_FILL_MODE_LOWER, N, CUDA_C_64F, ctx->dv_V.p, N, CUDA_R_64F,
                        ctx->dv_diagH.p, CUDA_C_64F, ctx->dv_W.p, dev_ws, hws.data(), host_ws,
                        ctx->dv_small.as<int>());
  cusolverDnDestroyParams(params);
  if (cs != CUSOLVER_STATUS_SUCCESS)
    return xatu_fail(ctx, XATU_ERR_CUDA, std::string("cusolverDnXsyevd failed (status ") + std::to_string((int)cs) + ")");
  int info = 0;
  XATU_CK(cudaMemcpyAsync(&info, ctx->dv_small.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  if (info != 0) return xatu_fail(ctx, XATU_ERR_NOT_CONVERGED, "cusolverDnXsyevd reported info != 0");
  if (vectors) {
    conj_columns_kernel<<<592, 256, 0, ctx->stream>>>(ctx->dv_V.as<cd>(), N * N);
    ctx->launches++;
    XATU_CK(cudaGetLastError());
  }
  return XATU_OK;
}

xatu_status xatu_dense_solve(xatu_ctx* ctx, int nstates, double* eigval, double* eigvec) {
  const long long N = ctx->N;
  xatu_status st = xatu_dense_eig_device(ctx, eigvec != nullptr);
  if (st != XATU_OK) return st;
  const long long ns = (nstates <= 0) ? N : nstates;
  XATU_CK(cudaMemcpyAsync(eigval, ctx->dv_diagH.p, (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (eigvec)
    XATU_CK(cudaMemcpyAsync(eigvec, ctx->dv_V.p, (size_t)ns * N * sizeof(cd), cudaMemcpyDeviceToHost, ctx->stream));
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  return XATU_OK;
}
