// Internal state of an engine context and the launchers shared between the
// translation units of libxatu_bse.so.  Not part of the public ABI.
#pragma once
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <string>
#include <vector>

#include "../../include/xatu_bse.h"
#include "common.cuh"

// A device allocation that only grows.
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t n) {
    if (n <= bytes && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&p, n);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename T> T* as() const { return reinterpret_cast<T*>(p); }
};

struct xatu_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  std::string err;
  long long launches = 0;
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t solver = nullptr;
  cudaEvent_t ev[12] = {};
  float stage_ms[4] = {0, 0, 0, 0};

  // ---------------- system
  bool has_system = false;
  int ndim = 0, natoms = 0, norb = 0, nR = 0, filling = 0;
  bool triangular = false, is_au = false, has_overlap = false;
  std::vector<double> bravais, recip, motif, cellsR, inv_gram;
  std::vector<int> orb_off;
  double a1 = 0, b1 = 0, area = 0;
  DBuf d_motif, d_orboff, d_cellsR, d_HR, d_SR;

  // ---------------- exciton
  bool has_exciton = false;
  int ncell = 0, factor = 1, n_eff = 0, nk = 0, nmesh = 0, nv = 0, nc = 0, nb = 0;
  long long N = 0;
  long long N_full = 0;        // nk * nv * nc
  bool custom_basis = false;   // last build used a caller-given basis
  long long ldk = 0;          // row pitch of the mixed planes (N rounded up to 4)
  std::vector<int> band_list;
  double eps_m = 1, eps_s = 1, r0 = 1, regularization = 0, cutoff = 0, scissor = 0;
  double Q[3] = {0, 0, 0};
  bool qnonzero = false;
  int exchange = 0, mode = 0, n_recip = 1, potential = 0, exchange_potential = 0, gauge = 0;
  double total_cells = 1;
  std::vector<double> kpoints, mesh, cells, G;
  std::vector<int> kgrid;
  bool kgrid_ok = false;
  // integer coordinates of the mesh (units b_d / n_eff) and of the cells (units a_d, reduced mod n_eff) when
  // both are commensurate; the motif FT then takes its phases from a table of roots of unity
  std::vector<int> mesh_int, cells_int;
  bool ft_roots = false;
  DBuf d_mesh_int, d_cells_int;
  int rt_len[3] = {1, 1, 1}, rt_span[3] = {0, 0, 0};
  long long rt_entries = 1;
  DBuf d_kpoints, d_mesh, d_cells, d_G, d_kgrid, d_basis, d_Q;

  // ---------------- derived device data
  bool bands_ok = false, tables_ok = false;
  int built_prec = -1;
  DBuf d_eigval, d_eigvec, d_eigvalQ, d_eigvecQ;
  DBuf d_pairs, d_vtab, d_vtabX, d_table, d_VX, d_exL, d_exR;
  DBuf d_H, d_Khi, d_Klo, d_diag, d_status;
  DBuf d_asmops;   // operand images of the tensor-core assembly tile
  DBuf d_work;       // solver scratch
  int last_assembly_path = -1;

  // ---------------- Davidson
  double dav_tol = 0.0;      // 0: default per precision
  int dav_max_iter = 1000;
  int dav_block = 0;
  int hx_backend = 0;         // 0 auto, 1 CUDA cores, 2 tensor cores (tcgen05)
  int band_backend = 0;       // 0 auto, 1 full band solve (Jacobi), 2 band window only
  int band_last_path = -1;    // path of the last band solve (1 full, 2 window)
  long long hx_calls = 0;     // K.X launches of the last solve
  double hx_ms = 0;           // their summed device time
  int hx_last_path = -1;      // 1 CUDA cores, 2 tcgen05
  bool hx_pending = false;    // ev[8]..ev[9] bracket K.X launches not yet added to hx_ms
  int num_sms = 148;
  int dav_iters = 0;
  double dav_maxres = 0;
  DBuf dv_V, dv_W, dv_T, dv_Y, dv_U, dv_R, dv_X, dv_Yf, dv_G, dv_tmp, dv_diagH, dv_small, dv_norm, dv_Bop, dv_Blo, dv_Uhi, dv_Ulo;
  DBuf dv_part;                // per-tile partial sums of the Davidson reductions
  void* h_small = nullptr;     // pinned host staging for small read-backs (4 KB)
  void* h_stage = nullptr;     // pinned host staging of the exciton set-up's uploads
  size_t h_stage_bytes = 0;

  // ---------------- adjoint
  bool bands_from_model = false;   // bands came from xatu_bands_compute (not uploaded)
  float adjoint_ms = 0;            // last xatu_adjoint call, first to last launch
  float adj_pair_ms = 0;           // its pair kernel
  DBuf d_oscG;

  // ---------------- post-processing (postproc.cu)
  DBuf d_pp_X, d_pp_A, d_pp_B, d_pp_C, d_pp_D, d_pp_P, d_pp_E;
  DBuf d_adjX, d_adjdvtab, d_adjdtable, d_adjdVX, d_adjAlpha, d_adjExUW, d_adjCbar, d_adjEbar, d_adjEpart, d_adjGk,
      d_adjG;
};

// Stage helpers without host synchronisation (api.cu); the batch records them into CUDA graphs.
extern "C" {
xatu_status xatu_bands_enqueue(xatu_ctx* ctx);
xatu_status xatu_tables_enqueue(xatu_ctx* ctx);
void xatu_assembly_setup(const xatu_ctx* ctx, const int* basis, struct AsmParams* p, struct AsmInputs* in,
                         struct AsmOutputs* out);
}

// Raises (never lowers) a kernel's dynamic shared-memory limit on the current device.  The limit is a
// per-kernel, process-wide setting: lowering it for a small launch would invalidate larger launches of
// the same kernel already recorded in CUDA graphs or issued by other contexts.
cudaError_t xatu_raise_smem_limit(const void* kernel, size_t bytes);

// status helpers
xatu_status xatu_fail(xatu_ctx* ctx, xatu_status code, const std::string& msg);
xatu_status xatu_cuda_fail(xatu_ctx* ctx, cudaError_t e, const char* where);
// Reads and clears the device error word; maps its flags to a status and message.
xatu_status xatu_check_device_status(xatu_ctx* ctx, const char* stage);

// launchers implemented in the .cu files
struct AsmParams;
struct AsmInputs;
struct AsmOutputs;

// Davidson (davidson.cu): lowest nstates of H = diag + K (mixed) or H (FP64).
xatu_status xatu_davidson_solve(xatu_ctx* ctx, int nstates, double* eigval, double* eigvec);
// Dense FP64 (dense.cu): all eigenpairs with cuSOLVER.
xatu_status xatu_dense_solve(xatu_ctx* ctx, int nstates, double* eigval, double* eigvec);
// The same, left on the device: eigenvalues in dv_diagH, eigenvectors as columns of dv_V (N x N).
xatu_status xatu_dense_eig_device(xatu_ctx* ctx, bool vectors);
// Velocity matrix elements of every e-h state into out (3 x N, row-major) (oscillator.cu).
xatu_status xatu_vme_enqueue(xatu_ctx* ctx, cd* out);
// vme_ex (3 x ns, column-major) = sum_i X(i, s) v_j(i) for the 3 x N elements v of xatu_vme_enqueue (oscillator.cu).
xatu_status xatu_exciton_vme_enqueue(xatu_ctx* ctx, const cd* v, const cd* X, long long N, int ns, cd* out);
// Adjoint of the velocity matrix elements (oscillator.cu): vbar (N x 3, column-major) -> added to cbar/ebar
// and, for the direct dependence on H(R), to G (nR x norb x norb); gvme: scratch of 2 x nk x norb^2.
// G = NULL: only cbar/ebar and gvme; xatu_vme_hop_enqueue then adds the direct part to G.
xatu_status xatu_vme_adjoint_enqueue(xatu_ctx* ctx, const cd* vbar, cd* cbar, double* ebar, cd* gvme, cd* G);
xatu_status xatu_vme_hop_enqueue(xatu_ctx* ctx, const cd* gvme, cd* G);
// Derivative interaction tables (adjoint.cu): which = 0: d/dr0, 1: d/deps_m (= d/deps_s), into
// d_adjdtable (same layout as d_table) and d_adjdVX (as d_VX).
xatu_status xatu_derivative_tables(xatu_ctx* ctx, int which);
// Band-level back-propagation (adjoint.cu): cbar/ebar of ns objectives -> G(R) in d_adjG.
xatu_status xatu_adjoint_bands_to_hoppings(xatu_ctx* ctx, int ns, const cd* cbar, const double* ebar);
// cbar/ebar of sum_ij Y_ij H_ij for a Hermitian row-major weight matrix Y (adjoint.cu); Zc = Y conj(L),
// Zv = Y^T L with the exchange vectors L (NULL without exchange).
xatu_status xatu_adjoint_weighted(xatu_ctx* ctx, const cd* Y, const cd* Zc, const cd* Zv, cd* cbar, double* ebar);

// K.X products (hx.cu).  Y[N x b] = (Khi + Klo) X, all row-major complex float.
cudaError_t xatu_launch_hx_cuda_core(const __nv_bfloat162* Khi, const __nv_bfloat162* Klo, long long ldk, const float2* X,
                                     float2* Y, long long N, int b, cudaStream_t s);
// tcgen05 version (hx_tc.cu) over the upper block triangle of K: operands Bt (ng x ldb bf16, hi/lo) and
// Bu (ng x ldu bf16, hi/lo) from xatu_launch_hx_operands, ng in {16, 32, 48}; Y row-major N x ng FP32
// (columns s < ng/2 the real parts, ng/2 + s the imaginary parts), zeroed here.
// active: NULL, or a device word read by the kernel; 0 skips the product (Y is still zeroed).
cudaError_t xatu_launch_hx_tc(const void* Khi, const void* Klo, long long N, long long ldk, const void* Bhi,
                              const void* Blo, long long ldb, const void* Uhi, const void* Ulo, long long ldu, int ng,
                              float* Y, int* status, int num_sms, cudaStream_t s, const int* active = nullptr);
// Operand planes of the tcgen05 product from b columns of X (complex FP64, column stride ldx), padded to bp:
// ldb >= 2N and ldu >= N, both multiples of 8.
cudaError_t xatu_launch_hx_operands(const cd* X, long long ldx, long long N, int b, int bp, void* Bhi, void* Blo,
                                    long long ldb, void* Uhi, void* Ulo, long long ldu, cudaStream_t s);
size_t xatu_hx_tc_smem(int ng);
// Widest block of vectors one tcgen05 product takes (ng = 2 * 24 = 48).
#define XATU_HX_TC_MAXB 24
// W[:, col0 : col0 + nv] = H V[:, col0 : col0 + nv] with the current build (davidson.cu).
xatu_status xatu_apply_h(xatu_ctx* ctx, long long N, int col0, int nv);
// Adds the bracketed K.X device time of the last xatu_apply_h to hx_ms (call after a stream synchronisation).
void xatu_hx_collect(xatu_ctx* ctx);

// After a kernel launch: the launch's own error, labelled with the kernel.
// Launch of a kernel that begins with xatu_grid_chain(): programmatic stream serialisation, so that the
// kernel is scheduled while its predecessor on the stream finishes (the launch latency of the short
// Davidson kernels overlaps the tail of the previous one).
template <typename... KArgs, typename... Args>
inline cudaError_t xatu_launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                       cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

#define XATU_CK_LAUNCH(name)                                                       \
  do {                                                                             \
    cudaError_t e__ = cudaGetLastError();                                          \
    if (e__ != cudaSuccess) return xatu_cuda_fail(ctx, e__, "launch of " name);     \
  } while (0)

#define XATU_CK(call)                                              \
  do {                                                             \
    cudaError_t e__ = (call);                                      \
    if (e__ != cudaSuccess) return xatu_cuda_fail(ctx, e__, #call); \
  } while (0)
