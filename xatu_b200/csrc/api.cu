// C ABI of the engine (include/xatu_bse.h): context, inputs, stage
// orchestration on the context's stream, and the host geometry helpers.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "engine.h"
#include "geometry.h"

#include "kernels.h"

// ------------------------------------------------------------------ status
xatu_status xatu_fail(xatu_ctx* ctx, xatu_status code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

xatu_status xatu_cuda_fail(xatu_ctx* ctx, cudaError_t e, const char* where) {
  std::string m = std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e);
  return xatu_fail(ctx, e == cudaErrorMemoryAllocation ? XATU_ERR_ALLOC : XATU_ERR_CUDA, m);
}

xatu_status xatu_check_device_status(xatu_ctx* ctx, const char* stage) {
  int st = 0;
  XATU_CK(cudaMemcpyAsync(&st, ctx->d_status.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  if (st == 0) return XATU_OK;
  XATU_CK(cudaMemsetAsync(ctx->d_status.p, 0, sizeof(int), ctx->stream));
  std::string m = std::string(stage) + ":";
  if (st & XATU_DEVERR_NAN) m += " non-finite input;";
  if (st & XATU_DEVERR_INDEX) m += " table index out of range;";
  if (st & XATU_DEVERR_NOCONV) m += " Jacobi sweep cap reached;";
  if (st & XATU_DEVERR_OVERLAP) m += " Zero or negative overlap eigenvalues found;";
  if (st & XATU_DEVERR_DEGEN)
    m += " degenerate bands (or a zero coefficient sum) at a k point: the band eigenvector derivative is undefined;";
  return xatu_fail(ctx, (st & (XATU_DEVERR_NAN | XATU_DEVERR_OVERLAP | XATU_DEVERR_DEGEN)) ? XATU_ERR_NUMERIC
                                                                                           : XATU_ERR_NOT_CONVERGED,
                   m);
}

cudaError_t xatu_raise_smem_limit(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> limits;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  size_t& cur = limits[std::make_pair(dev, kernel)];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

template <typename T>
static cudaError_t upload(DBuf& b, const T* src, size_t n, cudaStream_t s) {
  cudaError_t e = b.ensure(std::max<size_t>(n * sizeof(T), 16));
  if (e != cudaSuccess) return e;
  if (n) return cudaMemcpyAsync(b.p, src, n * sizeof(T), cudaMemcpyHostToDevice, s);
  return cudaSuccess;
}

// Nearest integer, halves away from zero (std::round) for the grid coordinates of the set-up (|x| < 2^52), by
// truncating conversions that compile inline: these loops run over every k point and cell of every call.
static inline double round_coord(double x) {
  return x >= 0 ? (double)(long long)(x + 0.5) : -(double)(long long)(0.5 - x);
}

// Integer coordinates of points p (n x 3) in units of b_d / n_eff: red = n_eff inv(B B^T) B p, rounded; relative
// to the first point when relative.  out: n x 3 (unused dimensions 0), lo / hi: the range per dimension.
// Returns whether every point lies within 1e-6 of the grid.  Local copies of the small matrices keep the loop
// free of reloads through the context.
static bool grid_coords(const double* p, long n, int nd, const double* recip_in, const double* inv_in, int n_eff,
                        bool relative, int* out, int* lo, int* hi) {
  double rc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, iv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 3 * nd; i++) rc[i] = recip_in[i];
  for (int i = 0; i < nd * nd; i++) iv[i] = inv_in[i];
  double r0v[3] = {0, 0, 0};
  bool ok = true;
  for (int a = 0; a < 3; a++) lo[a] = hi[a] = 0;
  for (long i = 0; i < n && ok; i++) {
    const double* k = p + 3 * i;
    double ind[3] = {0, 0, 0}, red[3] = {0, 0, 0};
    for (int a = 0; a < nd; a++) ind[a] = rc[3 * a] * k[0] + rc[3 * a + 1] * k[1] + rc[3 * a + 2] * k[2];
    for (int a = 0; a < nd; a++) {
      for (int b = 0; b < nd; b++) red[a] += iv[a * nd + b] * ind[b];
      red[a] *= n_eff;
    }
    if (i == 0 && relative)
      for (int a = 0; a < nd; a++) r0v[a] = red[a];
    for (int a = 0; a < nd; a++) {
      const double d = red[a] - r0v[a];
      const double u = round_coord(d);
      if (std::fabs(d - u) > 1e-6) ok = false;
      const int v = (int)u;
      out[3 * i + a] = v;
      if (i == 0 || v < lo[a]) lo[a] = v;
      if (i == 0 || v > hi[a]) hi[a] = v;
    }
  }
  return ok;
}

// Lattice coordinates n_d = b_d.R / 2 pi of cells R (n x 3), reduced to [0, n_eff); whether all are integers.
static bool cell_coords(const double* R, long n, int nd, const double* recip_in, int n_eff, int* out) {
  double rc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 3 * nd; i++) rc[i] = recip_in[i];
  for (long i = 0; i < n; i++) {
    const double* r = R + 3 * i;
    for (int a = 0; a < nd; a++) {
      const double f = (rc[3 * a] * r[0] + rc[3 * a + 1] * r[1] + rc[3 * a + 2] * r[2]) / (2.0 * XATU_PI);
      const double u = round_coord(f);
      if (std::fabs(f - u) > 1e-6) return false;
      long long v = (long long)u % n_eff;
      if (v < 0) v += n_eff;
      out[3 * i + a] = (int)v;
    }
  }
  return true;
}

// Host-to-device copies of one call through the context's pinned staging buffer: a pageable source makes the
// driver stage it copy by copy; here each source is copied into the pinned buffer on the host and sent with an
// asynchronous copy.  The caller synchronises the stream before the buffer is written again.
struct Stager {
  xatu_ctx* ctx;
  size_t off = 0;
  template <typename V>
  static size_t size(const V& v) {
    return (v.size() * sizeof(typename V::value_type) + 15) / 16 * 16;
  }
  cudaError_t begin(size_t bytes) {
    if (ctx->h_stage_bytes < bytes) {
      if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
      ctx->h_stage = nullptr;
      ctx->h_stage_bytes = 0;
      const cudaError_t e = cudaMallocHost(&ctx->h_stage, bytes);
      if (e != cudaSuccess) return e;
      ctx->h_stage_bytes = bytes;
    }
    off = 0;
    return cudaSuccess;
  }
  template <typename T>
  cudaError_t put(DBuf& b, const T* src, size_t n) {
    const cudaError_t e = b.ensure(std::max<size_t>(n * sizeof(T), 16));
    if (e != cudaSuccess || !n) return e;
    const size_t bytes = n * sizeof(T);
    if (off + bytes > ctx->h_stage_bytes) return cudaErrorInvalidValue;
    unsigned char* dst = static_cast<unsigned char*>(ctx->h_stage) + off;
    memcpy(dst, src, bytes);
    off += (bytes + 15) / 16 * 16;
    return cudaMemcpyAsync(b.p, dst, bytes, cudaMemcpyHostToDevice, ctx->stream);
  }
};

extern "C" {

int xatu_abi_version(void) { return 1; }

xatu_status xatu_ctx_create(xatu_ctx** out, int device) {
  if (!out) return XATU_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return XATU_ERR_CUDA;
  if (device < 0 || device >= ndev) return XATU_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return XATU_ERR_CUDA;
  xatu_ctx* ctx = new xatu_ctx();
  ctx->device = device;
  if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return XATU_ERR_CUDA;
  }
  ctx->stream = ctx->own_stream;
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  for (auto& e : ctx->ev) cudaEventCreate(&e);
  if (ctx->d_status.ensure(sizeof(int)) != cudaSuccess) {
    delete ctx;
    return XATU_ERR_ALLOC;
  }
  cudaMemset(ctx->d_status.p, 0, sizeof(int));
  *out = ctx;
  return XATU_OK;
}

xatu_status xatu_ctx_destroy(xatu_ctx* ctx) {
  if (!ctx) return XATU_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  DBuf* bufs[] = {&ctx->d_motif, &ctx->d_orboff, &ctx->d_basis, &ctx->d_cellsR, &ctx->d_HR, &ctx->d_SR, &ctx->d_kpoints, &ctx->d_mesh,
                  &ctx->d_cells, &ctx->d_G, &ctx->d_kgrid, &ctx->d_Q, &ctx->d_eigval, &ctx->d_eigvec, &ctx->d_eigvalQ,
                  &ctx->d_eigvecQ, &ctx->d_pairs, &ctx->d_vtab, &ctx->d_vtabX, &ctx->d_table, &ctx->d_VX,
                  &ctx->d_exL, &ctx->d_exR, &ctx->d_H, &ctx->d_Khi, &ctx->d_Klo, &ctx->d_diag, &ctx->d_status, &ctx->d_asmops,
                  &ctx->d_work, &ctx->dv_V, &ctx->dv_W, &ctx->dv_T, &ctx->dv_Y, &ctx->dv_U, &ctx->dv_R,
                  &ctx->dv_X, &ctx->dv_Yf, &ctx->dv_G, &ctx->dv_tmp, &ctx->dv_diagH, &ctx->dv_small,
                  &ctx->dv_norm, &ctx->dv_Bop, &ctx->dv_Blo, &ctx->dv_Uhi, &ctx->dv_Ulo, &ctx->d_adjX, &ctx->d_adjdvtab,
                  &ctx->d_adjdtable, &ctx->d_adjdVX, &ctx->d_adjAlpha, &ctx->d_adjExUW, &ctx->d_adjCbar,
                  &ctx->d_adjEbar, &ctx->d_adjEpart, &ctx->d_adjGk, &ctx->d_adjG, &ctx->d_oscG,
                  &ctx->dv_part, &ctx->d_pp_X, &ctx->d_pp_A, &ctx->d_pp_B, &ctx->d_pp_C, &ctx->d_pp_D,
                  &ctx->d_pp_P, &ctx->d_pp_E, &ctx->d_mesh_int, &ctx->d_cells_int};
  for (DBuf* b : bufs) b->release();
  if (ctx->h_small) cudaFreeHost(ctx->h_small);
  if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
  if (ctx->blas) cublasDestroy(ctx->blas);
  if (ctx->solver) cusolverDnDestroy(ctx->solver);
  for (auto& e : ctx->ev)
    if (e) cudaEventDestroy(e);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return XATU_OK;
}

const char* xatu_last_error(const xatu_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

xatu_status xatu_ctx_set_stream(xatu_ctx* ctx, void* stream) {
  if (!ctx) return XATU_ERR_INVALID;
  ctx->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : ctx->own_stream;
  if (ctx->blas) cublasSetStream(ctx->blas, ctx->stream);
  if (ctx->solver) cusolverDnSetStream(ctx->solver, ctx->stream);
  return XATU_OK;
}

// ------------------------------------------------------------------ system
xatu_status xatu_system_upload(xatu_ctx* ctx, const xatu_system_desc* s) {
  if (!ctx || !s) return xatu_fail(ctx, XATU_ERR_INVALID, "null argument");
  cudaSetDevice(ctx->device);
  if (s->ndim < 1 || s->ndim > 3) return xatu_fail(ctx, XATU_ERR_INVALID, "ndim must be 1, 2 or 3");
  if (!s->bravais || !s->motif || !s->norbitals || !s->cells || !s->hamiltonian)
    return xatu_fail(ctx, XATU_ERR_INVALID, "missing system array");
  if (s->natoms < 1 || s->nspecies < 1 || s->ncells < 1)
    return xatu_fail(ctx, XATU_ERR_INVALID, "natoms, nspecies and ncells must be positive");
  if (s->natoms > XATU_MAX_ATOMS)
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "more atoms in the motif than this build supports (16)");
  std::vector<int> off(s->natoms + 1, 0);
  for (int a = 0; a < s->natoms; a++) {
    const double sp = s->motif[4 * a + 3];
    const int isp = (int)sp;
    if (isp < 0 || isp >= s->nspecies || (double)isp != sp)
      return xatu_fail(ctx, XATU_ERR_INVALID, "motif species index out of range");
    if (s->norbitals[isp] < 1) return xatu_fail(ctx, XATU_ERR_INVALID, "species with no orbitals");
    off[a + 1] = off[a] + s->norbitals[isp];
  }
  const int norb = off[s->natoms];
  if (norb > XATU_MAX_ORB)
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "more orbitals per cell than this build supports (64)");
  std::vector<double> recip(9, 0.0), inv(9, 0.0);
  if (!xatu_geo::reciprocal_lattice(s->ndim, s->bravais, recip.data()))
    return xatu_fail(ctx, XATU_ERR_INVALID, "Failed to obtain reciprocal lattice vectors");
  if (!xatu_geo::inverse_gram(s->ndim, recip.data(), inv.data()))
    return xatu_fail(ctx, XATU_ERR_INVALID, "Unable to compute inverse reciprocal coefficients");
  const size_t nn = (size_t)norb * norb;
  for (size_t i = 0; i < 2 * nn * s->ncells; i++)
    if (!std::isfinite(s->hamiltonian[i])) return xatu_fail(ctx, XATU_ERR_NUMERIC, "non-finite hamiltonian entry");
  ctx->has_system = false;
  ctx->has_exciton = false;
  ctx->bands_ok = ctx->tables_ok = false;
  ctx->built_prec = -1;
  ctx->ndim = s->ndim;
  ctx->natoms = s->natoms;
  ctx->norb = norb;
  ctx->nR = s->ncells;
  ctx->filling = s->filling;
  ctx->bravais.assign(s->bravais, s->bravais + 3 * s->ndim);
  ctx->recip.assign(recip.begin(), recip.begin() + 3 * s->ndim);
  ctx->inv_gram.assign(inv.begin(), inv.begin() + s->ndim * s->ndim);
  ctx->motif.assign(s->motif, s->motif + 4 * s->natoms);
  ctx->cellsR.assign(s->cells, s->cells + 3 * s->ncells);
  ctx->orb_off = off;
  ctx->a1 = xatu_geo::norm3(s->bravais);
  ctx->b1 = xatu_geo::norm3(recip.data());
  ctx->area = xatu_geo::unit_cell_area(s->ndim, s->bravais);
  ctx->is_au = s->is_au != 0;
  ctx->has_overlap = s->overlap != nullptr;
  if (s->is_triangular >= 0) {
    ctx->triangular = s->is_triangular != 0;
  } else {
    // checkIfTriangular (utils.cpp:176-178) on the first matrix: upper XOR lower
    const double* h = s->hamiltonian;
    bool upper = true, lower = true;
    for (int r = 0; r < norb; r++)
      for (int c = 0; c < norb; c++) {
        const double re = h[2 * ((size_t)r * norb + c)], im = h[2 * ((size_t)r * norb + c) + 1];
        const bool z = (re == 0.0 && im == 0.0);
        if (r > c && !z) upper = false;
        if (r < c && !z) lower = false;
      }
    ctx->triangular = (upper != lower);
  }
  XATU_CK(upload(ctx->d_motif, ctx->motif.data(), ctx->motif.size(), ctx->stream));
  XATU_CK(upload(ctx->d_orboff, ctx->orb_off.data(), ctx->orb_off.size(), ctx->stream));
  XATU_CK(upload(ctx->d_cellsR, ctx->cellsR.data(), ctx->cellsR.size(), ctx->stream));
  XATU_CK(upload(ctx->d_HR, s->hamiltonian, 2 * nn * s->ncells, ctx->stream));
  if (s->overlap) XATU_CK(upload(ctx->d_SR, s->overlap, 2 * nn * s->ncells, ctx->stream));
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  ctx->has_system = true;
  return XATU_OK;
}

// ------------------------------------------------------------------ exciton
xatu_status xatu_exciton_set(xatu_ctx* ctx, const xatu_exciton_desc* e) {
  if (!ctx || !e) return xatu_fail(ctx, XATU_ERR_INVALID, "null argument");
  cudaSetDevice(ctx->device);
  if (!ctx->has_system) return xatu_fail(ctx, XATU_ERR_STATE, "system must be uploaded first");
  if (e->nvalence + e->nconduction == 0)
    return xatu_fail(ctx, XATU_ERR_INVALID, "Error: Exciton object must have some bands");
  if (e->nvalence < 1 || e->nconduction < 1)
    return xatu_fail(ctx, XATU_ERR_INVALID, "need at least one valence and one conduction band");
  if (e->nvalence > XATU_MAX_BANDS || e->nconduction > XATU_MAX_BANDS)
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "more than 8 valence or conduction bands");
  if (e->nk <= 0 || !e->kpoints) return xatu_fail(ctx, XATU_ERR_INVALID, "Error: BZ mesh must be initialized first");
  if (e->ncell <= 0) return xatu_fail(ctx, XATU_ERR_INVALID, "'ncell' must be a positive number");
  if (e->factor < 1) return xatu_fail(ctx, XATU_ERR_INVALID, "mesh factor must be >= 1");
  if (e->r0 == 0) return xatu_fail(ctx, XATU_ERR_INVALID, "Error: r0 must be non-zero");
  if (e->mode != XATU_MODE_REALSPACE && e->mode != XATU_MODE_RECIPROCAL)
    return xatu_fail(ctx, XATU_ERR_INVALID, "mode must be either realspace or reciprocalspace");
  if (e->n_reciprocal < 0) return xatu_fail(ctx, XATU_ERR_INVALID, "setReciprocalVectors(): given number must be positive");
  if (e->potential < 0 || e->potential > 1 || e->exchange_potential < 0 || e->exchange_potential > 1)
    return xatu_fail(ctx, XATU_ERR_INVALID, "potential must be either 'keldysh' or 'coulomb'");
  if (e->gauge != XATU_GAUGE_LATTICE && e->gauge != XATU_GAUGE_ATOMIC)
    return xatu_fail(ctx, XATU_ERR_INVALID, "gauge must be either lattice or atomic");
  if (e->gauge == XATU_GAUGE_ATOMIC)
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "atomic gauge is not supported by this build");
  std::vector<int> bl;
  for (int i = 0; i < e->nvalence; i++) bl.push_back(e->valence_bands[i]);
  for (int i = 0; i < e->nconduction; i++) bl.push_back(e->conduction_bands[i]);
  for (int b : bl)
    if (b < 0 || b >= ctx->norb) return xatu_fail(ctx, XATU_ERR_INVALID, "band index outside the model's bands");
  for (int i = 0; i < 3 * e->nk; i++)
    if (!std::isfinite(e->kpoints[i])) return xatu_fail(ctx, XATU_ERR_NUMERIC, "non-finite k point");
  const int n_eff = e->ncell * e->factor;
  long long nmesh = 1;
  for (int d = 0; d < ctx->ndim; d++) nmesh *= n_eff;
  if (e->mesh && e->nmesh != nmesh)
    return xatu_fail(ctx, XATU_ERR_INVALID, "mesh must have (ncell*factor)^ndim rows");
  ctx->has_exciton = false;
  ctx->bands_ok = ctx->tables_ok = false;
  ctx->built_prec = -1;
  ctx->ncell = e->ncell;
  ctx->factor = e->factor;
  ctx->n_eff = n_eff;
  ctx->nk = e->nk;
  ctx->nmesh = (int)nmesh;
  ctx->nv = e->nvalence;
  ctx->nc = e->nconduction;
  ctx->nb = ctx->nv + ctx->nc;
  ctx->N = (long long)e->nk * ctx->nv * ctx->nc;
  ctx->N_full = ctx->N;
  ctx->custom_basis = false;
  ctx->ldk = (ctx->N + 3) / 4 * 4;
  ctx->band_list = bl;
  ctx->eps_m = e->eps_m;
  ctx->eps_s = e->eps_s;
  ctx->r0 = e->r0;
  ctx->regularization = (e->regularization < 1E-10) ? ctx->a1 : e->regularization;
  ctx->cutoff = (e->cutoff > 0) ? e->cutoff : e->ncell / 2.5;
  ctx->scissor = e->scissor;
  for (int i = 0; i < 3; i++) ctx->Q[i] = e->Q[i];
  ctx->qnonzero = xatu_geo::norm3(e->Q) != 0;
  ctx->exchange = e->exchange != 0;
  ctx->mode = e->mode;
  ctx->n_recip = e->n_reciprocal;
  ctx->potential = e->potential;
  ctx->exchange_potential = e->exchange_potential;
  ctx->gauge = e->gauge;
  ctx->total_cells = std::pow((double)n_eff, ctx->ndim);
  ctx->kpoints.assign(e->kpoints, e->kpoints + 3 * e->nk);
  if (e->mesh) ctx->mesh.assign(e->mesh, e->mesh + 3 * nmesh);
  else ctx->mesh = xatu_geo::mp_mesh(ctx->ndim, ctx->recip.data(), n_eff);
  // cells within |a1| * cutoff (ExcitonTB.cpp:710-711)
  ctx->cells = xatu_geo::truncate_supercell(ctx->ndim, ctx->bravais.data(), e->ncell, ctx->a1 * ctx->cutoff);
  if (ctx->cells.empty()) ctx->cells.assign(3, 0.0);
  // reciprocal vectors within cutoff * |b1| (ExcitonTB.cpp:574-575)
  if (ctx->mode == XATU_MODE_RECIPROCAL)
    ctx->G = xatu_geo::truncate_supercell(ctx->ndim, ctx->recip.data(), e->n_reciprocal, ctx->cutoff * ctx->b1);
  else
    ctx->G.clear();
  // integer grid offsets of the k points in units of b_d / n_eff (reciprocal-mode table)
  ctx->kgrid.assign(3 * (size_t)e->nk, 0);
  {
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    ctx->kgrid_ok = grid_coords(e->kpoints, e->nk, ctx->ndim, ctx->recip.data(), ctx->inv_gram.data(), n_eff, true,
                                ctx->kgrid.data(), lo, hi);
    ctx->rt_entries = 1;
    for (int a = 0; a < 3; a++) {
      ctx->rt_span[a] = (a < ctx->ndim) ? (hi[a] - lo[a]) : 0;
      ctx->rt_len[a] = 2 * ctx->rt_span[a] + 1;
      if (a < ctx->ndim) ctx->rt_entries *= ctx->rt_len[a];
    }
  }
  if (ctx->mode == XATU_MODE_RECIPROCAL && !ctx->kgrid_ok)
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED,
                     "reciprocal-space mode needs k points on a regular grid of the (ncell*factor) mesh");
  // integer coordinates of the BZ mesh (q = sum_d m_d / n_eff b_d) and of the cells (R = sum_d n_d a_d,
  // n_d = b_d.R / 2 pi), for the root-of-unity phases of the motif FT
  ctx->ft_roots = ctx->mode == XATU_MODE_REALSPACE && n_eff <= XATU_FT_MAXDEN;
  if (ctx->ft_roots) {
    int lo[3], hi[3];
    ctx->mesh_int.assign(3 * (size_t)nmesh, 0);
    ctx->ft_roots = grid_coords(ctx->mesh.data(), nmesh, ctx->ndim, ctx->recip.data(), ctx->inv_gram.data(), n_eff,
                                false, ctx->mesh_int.data(), lo, hi);
  }
  if (ctx->ft_roots) {
    const size_t ncl = ctx->cells.size() / 3;
    ctx->cells_int.assign(3 * ncl, 0);
    ctx->ft_roots = cell_coords(ctx->cells.data(), (long)ncl, ctx->ndim, ctx->recip.data(), n_eff,
                                ctx->cells_int.data());
  }
  {
    std::vector<int2> pairs;
    for (int a = 0; a < ctx->natoms; a++)
      for (int b = a; b < ctx->natoms; b++) pairs.push_back(make_int2(a, b));
    // every array of the call goes through the pinned staging buffer (one host copy each, then asynchronous
    // transfers; the synchronisation below frees the buffer for the next call)
    Stager st{ctx};
    const size_t need = st.size(ctx->kpoints) + st.size(ctx->mesh) + st.size(ctx->cells) + st.size(ctx->mesh_int) +
                        st.size(ctx->cells_int) + st.size(ctx->G) + st.size(ctx->kgrid) + st.size(pairs) + 3 * 16;
    XATU_CK(st.begin(need));
    XATU_CK(st.put(ctx->d_kpoints, ctx->kpoints.data(), ctx->kpoints.size()));
    XATU_CK(st.put(ctx->d_mesh, ctx->mesh.data(), ctx->mesh.size()));
    XATU_CK(st.put(ctx->d_cells, ctx->cells.data(), ctx->cells.size()));
    if (ctx->ft_roots) {
      XATU_CK(st.put(ctx->d_mesh_int, ctx->mesh_int.data(), ctx->mesh_int.size()));
      XATU_CK(st.put(ctx->d_cells_int, ctx->cells_int.data(), ctx->cells_int.size()));
    }
    XATU_CK(st.put(ctx->d_G, ctx->G.data(), ctx->G.size()));
    XATU_CK(st.put(ctx->d_kgrid, ctx->kgrid.data(), ctx->kgrid.size()));
    XATU_CK(st.put(ctx->d_pairs, pairs.data(), pairs.size()));
    XATU_CK(st.put(ctx->d_Q, ctx->Q, 3));
  }
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  ctx->has_exciton = true;
  return XATU_OK;
}

// ------------------------------------------------------------------ bands
// Band-solve kernels on the context's stream: no host synchronisation and no
// host copies (so that the sequence can be recorded into a CUDA graph once the
// buffers exist).
xatu_status xatu_bands_enqueue(xatu_ctx* ctx) {
  {
    const cudaError_t pending = cudaGetLastError();
    if (pending != cudaSuccess) return xatu_cuda_fail(ctx, pending, "an earlier call (pending before the band solve)");
  }
  const size_t nk = ctx->nk, nb = ctx->nb, norb = ctx->norb;
  XATU_CK(ctx->d_eigval.ensure(nk * nb * sizeof(double)));
  XATU_CK(ctx->d_eigvec.ensure(nk * nb * norb * sizeof(cd)));
  XATU_CK(ctx->d_eigvalQ.ensure(nk * nb * sizeof(double)));
  XATU_CK(ctx->d_eigvecQ.ensure(nk * nb * norb * sizeof(cd)));
  BandParams bp;
  memset(&bp, 0, sizeof(bp));
  bp.nk = ctx->nk;
  bp.norb = ctx->norb;
  bp.nR = ctx->nR;
  bp.triangular = ctx->triangular;
  bp.nb = ctx->nb;
  for (int i = 0; i < ctx->nb; i++) bp.band_list[i] = ctx->band_list[i];
  bp.max_sweeps = 40;
  bp.has_overlap = ctx->has_overlap ? 1 : 0;
  bp.is_au = ctx->is_au ? 1 : 0;
  const bool window = ctx->band_backend != 1 && xatu_band_select_supported(bp.norb, bp.nb, bp.has_overlap);
  if (ctx->band_backend == 2 && !window)
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "band-window solve: needs no overlap, norb <= 64, <= 16 bands");
  ctx->band_last_path = window ? 2 : 1;
  if (window) {
    cudaError_t e = xatu_launch_band_select(bp, ctx->d_kpoints.as<double>(), ctx->d_cellsR.as<double>(),
                                            ctx->d_HR.as<cd>(), ctx->d_eigval.as<double>(), ctx->d_eigvec.as<cd>(),
                                            ctx->d_status.as<int>(), ctx->stream);
    if (e != cudaSuccess) return xatu_cuda_fail(ctx, e, "launch of band_select_kernel");
    ctx->launches++;
    if (ctx->qnonzero) {
      for (int i = 0; i < 3; i++) bp.shift[i] = ctx->Q[i];
      e = xatu_launch_band_select(bp, ctx->d_kpoints.as<double>(), ctx->d_cellsR.as<double>(), ctx->d_HR.as<cd>(),
                                  ctx->d_eigvalQ.as<double>(), ctx->d_eigvecQ.as<cd>(), ctx->d_status.as<int>(),
                                  ctx->stream);
      if (e != cudaSuccess) return xatu_cuda_fail(ctx, e, "launch of band_select_kernel (k+Q)");
      ctx->launches++;
    } else {
      XATU_CK(cudaMemcpyAsync(ctx->d_eigvalQ.p, ctx->d_eigval.p, nk * nb * sizeof(double), cudaMemcpyDeviceToDevice,
                              ctx->stream));
      XATU_CK(cudaMemcpyAsync(ctx->d_eigvecQ.p, ctx->d_eigvec.p, nk * nb * norb * sizeof(cd),
                              cudaMemcpyDeviceToDevice, ctx->stream));
    }
    return XATU_OK;
  }
  const size_t smem = band_solve_smem(ctx->norb, ctx->nR, bp.has_overlap);
  XATU_CK(xatu_raise_smem_limit((const void*)band_solve_kernel, smem));
  const int grid = ctx->nk, threads = 128;
  const cd* SR = ctx->has_overlap ? ctx->d_SR.as<cd>() : nullptr;
  band_solve_kernel<<<grid, threads, smem, ctx->stream>>>(bp, ctx->d_kpoints.as<double>(),
                                                             ctx->d_cellsR.as<double>(), ctx->d_HR.as<cd>(), SR,
                                                             ctx->d_eigval.as<double>(), ctx->d_eigvec.as<cd>(),
                                                             ctx->d_status.as<int>());
  ctx->launches++;
  XATU_CK_LAUNCH("band_solve_kernel");
  if (ctx->qnonzero) {
    for (int i = 0; i < 3; i++) bp.shift[i] = ctx->Q[i];
    band_solve_kernel<<<grid, threads, smem, ctx->stream>>>(bp, ctx->d_kpoints.as<double>(),
                                                               ctx->d_cellsR.as<double>(), ctx->d_HR.as<cd>(), SR,
                                                               ctx->d_eigvalQ.as<double>(), ctx->d_eigvecQ.as<cd>(),
                                                               ctx->d_status.as<int>());
    ctx->launches++;
    XATU_CK_LAUNCH("band_solve_kernel (k+Q)");
  } else {
    XATU_CK(cudaMemcpyAsync(ctx->d_eigvalQ.p, ctx->d_eigval.p, nk * nb * sizeof(double), cudaMemcpyDeviceToDevice,
                            ctx->stream));
    XATU_CK(cudaMemcpyAsync(ctx->d_eigvecQ.p, ctx->d_eigvec.p, nk * nb * norb * sizeof(cd), cudaMemcpyDeviceToDevice,
                            ctx->stream));
  }
  return XATU_OK;
}

xatu_status xatu_bands_compute(xatu_ctx* ctx) {
  if (!ctx) return XATU_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (!ctx->has_exciton) return xatu_fail(ctx, XATU_ERR_STATE, "exciton parameters must be set first");
  XATU_CK(cudaEventRecord(ctx->ev[0], ctx->stream));
  xatu_status st = xatu_bands_enqueue(ctx);
  if (st != XATU_OK) return st;
  XATU_CK(cudaEventRecord(ctx->ev[1], ctx->stream));
  st = xatu_check_device_status(ctx, "band solve");
  if (st != XATU_OK) return st;
  cudaEventElapsedTime(&ctx->stage_ms[0], ctx->ev[0], ctx->ev[1]);
  ctx->bands_ok = true;
  ctx->bands_from_model = true;
  ctx->built_prec = -1;
  return XATU_OK;
}

xatu_status xatu_bands_upload(xatu_ctx* ctx, const double* eigval, const double* eigvec, const double* eigvalQ,
                              const double* eigvecQ) {
  if (!ctx || !eigval || !eigvec) return xatu_fail(ctx, XATU_ERR_INVALID, "null argument");
  cudaSetDevice(ctx->device);
  if (!ctx->has_exciton) return xatu_fail(ctx, XATU_ERR_STATE, "exciton parameters must be set first");
  if (ctx->qnonzero && (!eigvalQ || !eigvecQ))
    return xatu_fail(ctx, XATU_ERR_INVALID, "k+Q band stacks are required when Q != 0");
  const size_t nk = ctx->nk, nb = ctx->nb, norb = ctx->norb;
  XATU_CK(upload(ctx->d_eigval, eigval, nk * nb, ctx->stream));
  XATU_CK(upload(ctx->d_eigvec, eigvec, 2 * nk * nb * norb, ctx->stream));
  XATU_CK(upload(ctx->d_eigvalQ, eigvalQ ? eigvalQ : eigval, nk * nb, ctx->stream));
  XATU_CK(upload(ctx->d_eigvecQ, eigvecQ ? eigvecQ : eigvec, 2 * nk * nb * norb, ctx->stream));
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  ctx->bands_ok = true;
  ctx->bands_from_model = false;
  ctx->built_prec = -1;
  return XATU_OK;
}

xatu_status xatu_bands_download(xatu_ctx* ctx, double* eigval, double* eigvec, double* eigvalQ, double* eigvecQ) {
  if (!ctx) return XATU_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (!ctx->bands_ok) return xatu_fail(ctx, XATU_ERR_STATE, "bands are not computed");
  const size_t nk = ctx->nk, nb = ctx->nb, norb = ctx->norb;
  if (eigval) XATU_CK(cudaMemcpyAsync(eigval, ctx->d_eigval.p, nk * nb * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (eigvec) XATU_CK(cudaMemcpyAsync(eigvec, ctx->d_eigvec.p, nk * nb * norb * 16, cudaMemcpyDeviceToHost, ctx->stream));
  if (eigvalQ) XATU_CK(cudaMemcpyAsync(eigvalQ, ctx->d_eigvalQ.p, nk * nb * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (eigvecQ)
    XATU_CK(cudaMemcpyAsync(eigvecQ, ctx->d_eigvecQ.p, nk * nb * norb * 16, cudaMemcpyDeviceToHost, ctx->stream));
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  return XATU_OK;
}

// ------------------------------------------------------------------ interaction tables
static PotParams pot_params(const xatu_ctx* ctx) {
  PotParams p;
  p.a1norm = ctx->a1;
  p.b1norm = ctx->b1;
  p.area = ctx->area;
  p.eps_m = ctx->eps_m;
  p.eps_s = ctx->eps_s;
  p.r0 = ctx->r0;
  p.regularization = ctx->regularization;
  p.cutoff = ctx->cutoff;
  p.total_cells = ctx->total_cells;
  return p;
}

static RecipTable recip_table(const xatu_ctx* ctx, bool single_q) {
  RecipTable t;
  memset(&t, 0, sizeof(t));
  t.ndim = ctx->ndim;
  t.n_eff = ctx->n_eff;
  for (int a = 0; a < 3; a++) {
    t.span[a] = single_q ? 0 : ctx->rt_span[a];
    t.len[a] = single_q ? 1 : ctx->rt_len[a];
  }
  for (int i = 0; i < 3 * ctx->ndim; i++) t.b[i] = ctx->recip[i];
  t.nG = (int)(ctx->G.size() / 3);
  if (single_q)
    for (int i = 0; i < 3; i++) t.q0[i] = ctx->Q[i];
  return t;
}

// Interaction-table kernels on the context's stream (no synchronisation, no host copies).
xatu_status xatu_tables_enqueue(xatu_ctx* ctx) {
  const int na = ctx->natoms;
  const PotParams pp = pot_params(ctx);
  const int npairs = na * (na + 1) / 2;
  const int ncells = (int)(ctx->cells.size() / 3);
  XATU_CK(ctx->d_VX.ensure((size_t)na * na * sizeof(cd)));
  XATU_CK(cudaMemsetAsync(ctx->d_VX.p, 0, (size_t)na * na * sizeof(cd), ctx->stream));
  if (ctx->mode == XATU_MODE_REALSPACE) {
    XATU_CK(ctx->d_vtab.ensure((size_t)npairs * ncells * sizeof(double)));
    XATU_CK(ctx->d_table.ensure((size_t)ctx->nmesh * na * na * sizeof(cd)));
    const long long tot = (long long)npairs * ncells;
    int grid = (int)std::min<long long>((tot + 255) / 256, 148 * 16);
    pair_potential_kernel<<<grid, 256, 0, ctx->stream>>>(pp, ctx->potential, 0, na, ctx->d_motif.as<double>(), ncells,
                                                         ctx->d_cells.as<double>(), npairs, ctx->d_pairs.as<int2>(),
                                                         ctx->d_vtab.as<double>());
    ctx->launches++;
    XATU_CK_LAUNCH("pair_potential_kernel");
    dim3 g2(ctx->nmesh, (npairs + 7) / 8);
    if (ctx->ft_roots) {
      const dim3 gr((ctx->nmesh + XATU_MOTIF_QB - 1) / XATU_MOTIF_QB, (npairs + 7) / 8);
      motif_ft_roots_kernel<<<gr, 256, motif_roots_smem(ctx->n_eff), ctx->stream>>>(
          ctx->nmesh, ctx->d_mesh_int.as<int>(), ctx->n_eff, ncells, ctx->d_cells_int.as<int>(), npairs,
          ctx->d_pairs.as<int2>(), ctx->d_vtab.as<double>(), 1.0 / ctx->total_cells, na, ctx->d_table.as<cd>());
      ctx->launches++;
      XATU_CK_LAUNCH("motif_ft_roots_kernel");
    } else {
      motif_ft_kernel<<<g2, 256, 0, ctx->stream>>>(ctx->nmesh, ctx->d_mesh.as<double>(), ncells,
                                                   ctx->d_cells.as<double>(), npairs, ctx->d_pairs.as<int2>(),
                                                   ctx->d_vtab.as<double>(), 1.0 / ctx->total_cells, na,
                                                   ctx->d_table.as<cd>());
      ctx->launches++;
      XATU_CK_LAUNCH("motif_ft_kernel");
    }
    if (ctx->exchange) {
      const double* vt = ctx->d_vtab.as<double>();
      if (ctx->exchange_potential != ctx->potential) {
        XATU_CK(ctx->d_vtabX.ensure((size_t)npairs * ncells * sizeof(double)));
        pair_potential_kernel<<<grid, 256, 0, ctx->stream>>>(pp, ctx->exchange_potential, 0, na,
                                                             ctx->d_motif.as<double>(), ncells,
                                                             ctx->d_cells.as<double>(), npairs,
                                                             ctx->d_pairs.as<int2>(), ctx->d_vtabX.as<double>());
        ctx->launches++;
        XATU_CK(cudaGetLastError());
        vt = ctx->d_vtabX.as<double>();
      }
      dim3 g3(1, (npairs + 7) / 8);
      motif_ft_kernel<<<g3, 256, 0, ctx->stream>>>(1, ctx->d_Q.as<double>(), ncells, ctx->d_cells.as<double>(),
                                                   npairs, ctx->d_pairs.as<int2>(), vt, 1.0 / ctx->total_cells, na,
                                                   ctx->d_VX.as<cd>());
      ctx->launches++;
      XATU_CK(cudaGetLastError());
    }
  } else {
    const RecipTable t = recip_table(ctx, false);
    XATU_CK(ctx->d_table.ensure((size_t)ctx->rt_entries * na * na * sizeof(cd)));
    const long long tot = ctx->rt_entries * na;
    int grid = (int)std::min<long long>((tot + 127) / 128, 148 * 32);
    recip_table_kernel<<<grid, 128, 0, ctx->stream>>>(pp, t, 0, (int)ctx->rt_entries, ctx->d_G.as<double>(), na,
                                                      ctx->d_motif.as<double>(), ctx->d_table.as<cd>());
    ctx->launches++;
    XATU_CK(cudaGetLastError());
    if (ctx->exchange) {
      const RecipTable tx = recip_table(ctx, true);
      recip_table_kernel<<<1, 128, 0, ctx->stream>>>(pp, tx, 0, 1, ctx->d_G.as<double>(), na, ctx->d_motif.as<double>(),
                                                     ctx->d_VX.as<cd>());
      ctx->launches++;
      XATU_CK(cudaGetLastError());
    }
  }
  return XATU_OK;
}

xatu_status xatu_interaction_build(xatu_ctx* ctx) {
  if (!ctx) return XATU_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (!ctx->has_exciton) return xatu_fail(ctx, XATU_ERR_STATE, "exciton parameters must be set first");
  XATU_CK(cudaEventRecord(ctx->ev[2], ctx->stream));
  xatu_status st = xatu_tables_enqueue(ctx);
  if (st != XATU_OK) return st;
  XATU_CK(cudaEventRecord(ctx->ev[3], ctx->stream));
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  cudaEventElapsedTime(&ctx->stage_ms[1], ctx->ev[2], ctx->ev[3]);
  ctx->tables_ok = true;
  ctx->built_prec = -1;
  return XATU_OK;
}

xatu_status xatu_motif_ft_download(xatu_ctx* ctx, double* ft_stack, double* ft_Q) {
  if (!ctx) return XATU_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (!ctx->tables_ok) return xatu_fail(ctx, XATU_ERR_STATE, "interaction tables are not built");
  const size_t na2 = (size_t)ctx->natoms * ctx->natoms;
  const size_t rows = ctx->mode == XATU_MODE_REALSPACE ? (size_t)ctx->nmesh : (size_t)ctx->rt_entries;
  if (ft_stack)
    XATU_CK(cudaMemcpyAsync(ft_stack, ctx->d_table.p, rows * na2 * sizeof(cd), cudaMemcpyDeviceToHost, ctx->stream));
  if (ft_Q) XATU_CK(cudaMemcpyAsync(ft_Q, ctx->d_VX.p, na2 * sizeof(cd), cudaMemcpyDeviceToHost, ctx->stream));
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  return XATU_OK;
}

// ------------------------------------------------------------------ assembly
static xatu_status build_impl(xatu_ctx* ctx, int precision, const int* basis);

xatu_status xatu_bse_build(xatu_ctx* ctx, int precision) {
  if (!ctx) return XATU_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (!ctx->has_exciton) return xatu_fail(ctx, XATU_ERR_STATE, "exciton parameters must be set first");
  ctx->N = ctx->N_full;
  ctx->ldk = (ctx->N + 3) / 4 * 4;
  ctx->custom_basis = false;
  return build_impl(ctx, precision, nullptr);
}

xatu_status xatu_bse_build_basis(xatu_ctx* ctx, int precision, int64_t nbasis, const int* basis) {
  if (!ctx || !basis || nbasis < 1) return xatu_fail(ctx, XATU_ERR_INVALID, "bad argument");
  cudaSetDevice(ctx->device);
  if (!ctx->has_exciton) return xatu_fail(ctx, XATU_ERR_STATE, "exciton parameters must be set first");
  // absolute band numbers -> stack columns (Exciton::generateBandDictionary, Exciton.tpp:191-199)
  std::vector<int> rows(3 * (size_t)nbasis);
  for (int64_t i = 0; i < nbasis; i++) {
    const int vb = basis[3 * i], cb = basis[3 * i + 1], k = basis[3 * i + 2];
    int vcol = -1, crel = -1;
    for (int b = 0; b < ctx->nv; b++)
      if (ctx->band_list[b] == vb) vcol = b;
    for (int b = 0; b < ctx->nc; b++)
      if (ctx->band_list[ctx->nv + b] == cb) crel = b;
    if (vcol < 0 || crel < 0 || k < 0 || k >= ctx->nk)
      return xatu_fail(ctx, XATU_ERR_INVALID, "basis row outside the exciton's bands or k points");
    rows[3 * i] = k;
    rows[3 * i + 1] = vcol;
    rows[3 * i + 2] = crel;
  }
  XATU_CK(upload(ctx->d_basis, rows.data(), rows.size(), ctx->stream));
  ctx->N = nbasis;
  ctx->ldk = (ctx->N + 3) / 4 * 4;
  ctx->custom_basis = true;
  return build_impl(ctx, precision, ctx->d_basis.as<int>());
}

void xatu_assembly_setup(const xatu_ctx* ctx, const int* basis, AsmParams* pp, AsmInputs* inp, AsmOutputs* outp) {
  AsmParams& p = *pp;
  AsmInputs& in = *inp;
  AsmOutputs& out = *outp;
  const int na = ctx->natoms;
  memset(&p, 0, sizeof(p));
  p.nk = ctx->nk;
  p.nv = ctx->nv;
  p.nc = ctx->nc;
  p.nb = ctx->nb;
  p.norb = ctx->norb;
  p.na = na;
  p.N = ctx->N;
  p.mode = ctx->mode;
  p.exchange = ctx->exchange;
  p.scissor = ctx->scissor;
  p.emap.ndim = ctx->ndim;
  p.emap.n = ctx->n_eff;
  for (int i = 0; i < 3 * ctx->ndim; i++) p.emap.B[i] = ctx->recip[i];
  for (int i = 0; i < ctx->ndim * ctx->ndim; i++) p.emap.inv[i] = ctx->inv_gram[i];
  p.rt_ndim = ctx->ndim;
  for (int a = 0; a < 3; a++) {
    p.rt_len[a] = ctx->rt_len[a];
    p.rt_span[a] = ctx->rt_span[a];
  }
  for (int a = 0; a <= na; a++) p.orb_off[a] = ctx->orb_off[a];
  p.nentries = ctx->mode == XATU_MODE_REALSPACE ? ctx->nmesh : ctx->rt_entries;
  p.ldk = ctx->ldk;
  memset(&in, 0, sizeof(in));
  in.kpoints = ctx->d_kpoints.as<double>();
  in.kgrid = ctx->d_kgrid.as<int>();
  in.eigval = ctx->d_eigval.as<double>();
  in.eigvalQ = ctx->d_eigvalQ.as<double>();
  in.eigvec = ctx->d_eigvec.as<cd>();
  in.eigvecQ = ctx->d_eigvecQ.as<cd>();
  in.table = ctx->d_table.as<cd>();
  in.exL = ctx->d_exL.as<cd>();
  in.exR = ctx->d_exR.as<cd>();
  in.status = ctx->d_status.as<int>();
  in.basis = basis;
  in.tc_ops = nullptr;
  in.tc_ops_bytes = 0;
  memset(&out, 0, sizeof(out));
  out.H = ctx->d_H.as<cd>();
  out.Khi = ctx->d_Khi.as<__nv_bfloat162>();
  out.Klo = ctx->d_Klo.as<__nv_bfloat162>();
  out.diag = ctx->d_diag.as<double>();
}

static xatu_status build_impl(xatu_ctx* ctx, int precision, const int* basis) {
  if (!ctx->has_exciton) return xatu_fail(ctx, XATU_ERR_STATE, "exciton parameters must be set first");
  if (precision != XATU_PREC_FP64 && precision != XATU_PREC_MIXED)
    return xatu_fail(ctx, XATU_ERR_INVALID, "precision must be XATU_PREC_FP64 or XATU_PREC_MIXED");
  xatu_status st;
  if (!ctx->bands_ok && (st = xatu_bands_compute(ctx)) != XATU_OK) return st;
  if (!ctx->tables_ok && (st = xatu_interaction_build(ctx)) != XATU_OK) return st;
  const long long N = ctx->N;
  const int na = ctx->natoms;
  if (ctx->exchange) {
    XATU_CK(ctx->d_exL.ensure((size_t)N * na * sizeof(cd)));
    XATU_CK(ctx->d_exR.ensure((size_t)N * na * sizeof(cd)));
  }
  const bool mixed = precision == XATU_PREC_MIXED;
  if (mixed) {
    XATU_CK(ctx->d_Khi.ensure((size_t)N * ctx->ldk * sizeof(__nv_bfloat162)));
    XATU_CK(ctx->d_Klo.ensure((size_t)N * ctx->ldk * sizeof(__nv_bfloat162)));
    XATU_CK(ctx->d_diag.ensure((size_t)N * sizeof(double)));
  } else {
    XATU_CK(ctx->d_H.ensure((size_t)N * N * sizeof(cd)));
  }
  AsmParams p;
  AsmInputs in;
  AsmOutputs out;
  xatu_assembly_setup(ctx, basis, &p, &in, &out);
  if (mixed && basis == nullptr) {
    // scratch for the operand images of the tensor-core tile (none when the band window does not take it)
    const size_t ops = xatu_assembly_tc_scratch_bytes(p);
    if (ops) {
      XATU_CK(ctx->d_asmops.ensure(ops));
      in.tc_ops = ctx->d_asmops.as<unsigned char>();
      in.tc_ops_bytes = ops;
    }
  }
  XATU_CK(cudaEventRecord(ctx->ev[4], ctx->stream));
  if (ctx->exchange) {
    const int blocks = (int)((N + 127) / 128);
    exchange_vectors_kernel<<<blocks, 128, 0, ctx->stream>>>((int)N, ctx->nv, ctx->nc, ctx->nb, ctx->norb, na,
                                                             ctx->d_orboff.as<int>(), ctx->d_eigvec.as<cd>(),
                                                             ctx->d_eigvecQ.as<cd>(), ctx->d_VX.as<cd>(), basis,
                                                             ctx->d_exL.as<cd>(), ctx->d_exR.as<cd>());
    ctx->launches++;
    XATU_CK(cudaGetLastError());
  }
  int path = -1;
  const char* force = getenv("XATU_FORCE_GENERIC_ASSEMBLY");
  XATU_CK(xatu_launch_assembly(p, in, out, mixed, (force && force[0] == '1') || basis != nullptr, ctx->stream, &path));
  ctx->launches++;
  ctx->last_assembly_path = path;
  XATU_CK(cudaEventRecord(ctx->ev[5], ctx->stream));
  st = xatu_check_device_status(ctx, "BSE assembly");
  if (st != XATU_OK) return st;
  cudaEventElapsedTime(&ctx->stage_ms[2], ctx->ev[4], ctx->ev[5]);
  ctx->built_prec = precision;
  return XATU_OK;
}

xatu_status xatu_bse_dim(const xatu_ctx* ctx, int64_t* n) {
  if (!ctx || !n) return XATU_ERR_INVALID;
  if (!ctx->has_exciton) return XATU_ERR_STATE;
  *n = ctx->N;
  return XATU_OK;
}

__global__ void expand_mixed_kernel(const __nv_bfloat162* __restrict__ hi, const __nv_bfloat162* __restrict__ lo,
                                    const double* __restrict__ diag, long long N, long long ldk, long long row0,
                                    long long rows, cd* __restrict__ out) {
  const long long total = rows * N;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long r = row0 + t / N, c = t % N;
    // the kernel planes hold the upper block triangle; the rest is the conjugate of its mirror
    const bool st = xatu_kstored(r, c);
    const long long o = st ? r * ldk + c : c * ldk + r;
    const __nv_bfloat162 h = hi[o], l = lo[o];
    double re = (double)__bfloat162float(h.x) + (double)__bfloat162float(l.x);
    double im = (double)__bfloat162float(h.y) + (double)__bfloat162float(l.y);
    if (!st) im = -im;
    if (r == c) re += diag[r];
    out[t] = mk(re, im);
  }
}

xatu_status xatu_bse_copy_to_host(xatu_ctx* ctx, double* H) {
  if (!ctx || !H) return xatu_fail(ctx, XATU_ERR_INVALID, "null argument");
  cudaSetDevice(ctx->device);
  if (ctx->built_prec < 0) return xatu_fail(ctx, XATU_ERR_STATE, "BSE Hamiltonian is not initialized");
  const long long N = ctx->N;
  if (ctx->built_prec == XATU_PREC_FP64) {
    XATU_CK(cudaMemcpyAsync(H, ctx->d_H.p, (size_t)N * N * sizeof(cd), cudaMemcpyDeviceToHost, ctx->stream));
    XATU_CK(cudaStreamSynchronize(ctx->stream));
    return XATU_OK;
  }
  long long rows = std::max<long long>(1, (256ll << 20) / (N * (long long)sizeof(cd)));
  rows = std::min(rows, N);
  XATU_CK(ctx->d_work.ensure((size_t)rows * N * sizeof(cd)));
  for (long long r0 = 0; r0 < N; r0 += rows) {
    const long long nr = std::min(rows, N - r0);
    expand_mixed_kernel<<<1184, 256, 0, ctx->stream>>>(ctx->d_Khi.as<__nv_bfloat162>(), ctx->d_Klo.as<__nv_bfloat162>(),
                                                       ctx->d_diag.as<double>(), N, ctx->ldk, r0, nr,
                                                       ctx->d_work.as<cd>());
    ctx->launches++;
    XATU_CK(cudaGetLastError());
    XATU_CK(cudaMemcpyAsync(H + 2 * r0 * N, ctx->d_work.p, (size_t)nr * N * sizeof(cd), cudaMemcpyDeviceToHost,
                            ctx->stream));
    XATU_CK(cudaStreamSynchronize(ctx->stream));
  }
  return XATU_OK;
}

xatu_status xatu_bse_device_buffers(xatu_ctx* ctx, void** h_or_hi, void** lo, void** diag) {
  if (!ctx) return XATU_ERR_INVALID;
  if (ctx->built_prec < 0) return xatu_fail(ctx, XATU_ERR_STATE, "BSE Hamiltonian is not initialized");
  if (ctx->built_prec == XATU_PREC_FP64) {
    if (h_or_hi) *h_or_hi = ctx->d_H.p;
    if (lo) *lo = nullptr;
    if (diag) *diag = nullptr;
  } else {
    if (h_or_hi) *h_or_hi = ctx->d_Khi.p;
    if (lo) *lo = ctx->d_Klo.p;
    if (diag) *diag = ctx->d_diag.p;
  }
  return XATU_OK;
}

// ------------------------------------------------------------------ solve
xatu_status xatu_bse_solve(xatu_ctx* ctx, int solver, int nstates, double* eigval, double* eigvec) {
  if (!ctx || !eigval) return xatu_fail(ctx, XATU_ERR_INVALID, "null argument");
  cudaSetDevice(ctx->device);
  if (ctx->built_prec < 0) return xatu_fail(ctx, XATU_ERR_STATE, "diagonalizeRaw(): BSE Hamiltonian is not initialized.");
  if (nstates > ctx->N) return xatu_fail(ctx, XATU_ERR_INVALID, "nstates larger than the BSE dimension");
  xatu_status st;
  XATU_CK(cudaEventRecord(ctx->ev[6], ctx->stream));
  if (solver == XATU_SOLVER_DENSE_FP64) {
    if (ctx->built_prec != XATU_PREC_FP64)
      return xatu_fail(ctx, XATU_ERR_STATE, "the dense FP64 solver needs an FP64 build");
    st = xatu_dense_solve(ctx, nstates, eigval, eigvec);
  } else if (solver == XATU_SOLVER_DAVIDSON) {
    if (nstates < 1) return xatu_fail(ctx, XATU_ERR_INVALID, "Davidson needs nstates >= 1");
    st = xatu_davidson_solve(ctx, nstates, eigval, eigvec);
  } else {
    return xatu_fail(ctx, XATU_ERR_INVALID, "unknown solver");
  }
  cudaEventRecord(ctx->ev[7], ctx->stream);
  cudaEventSynchronize(ctx->ev[7]);
  cudaEventElapsedTime(&ctx->stage_ms[3], ctx->ev[6], ctx->ev[7]);
  return st;
}

xatu_status xatu_davidson_config(xatu_ctx* ctx, double tol, int max_iter, int block) {
  if (!ctx) return XATU_ERR_INVALID;
  if (tol < 0 || max_iter < 0 || block < 0) return xatu_fail(ctx, XATU_ERR_INVALID, "negative Davidson setting");
  ctx->dav_tol = tol;
  ctx->dav_max_iter = max_iter > 0 ? max_iter : 1000;
  ctx->dav_block = block;
  return XATU_OK;
}

xatu_status xatu_bands_backend(xatu_ctx* ctx, int backend) {
  if (!ctx) return XATU_ERR_INVALID;
  if (backend < 0 || backend > 2) return xatu_fail(ctx, XATU_ERR_INVALID, "backend must be 0, 1 or 2");
  ctx->band_backend = backend;
  return XATU_OK;
}

xatu_status xatu_hx_backend(xatu_ctx* ctx, int backend) {
  if (!ctx) return XATU_ERR_INVALID;
  if (backend < 0 || backend > 2) return xatu_fail(ctx, XATU_ERR_INVALID, "backend must be 0, 1 or 2");
  ctx->hx_backend = backend;
  return XATU_OK;
}

xatu_status xatu_kernel_matvec(xatu_ctx* ctx, int nvec, const double* X, double* Y) {
  if (!ctx || !X || !Y || nvec < 1) return xatu_fail(ctx, XATU_ERR_INVALID, "bad argument");
  cudaSetDevice(ctx->device);
  if (ctx->built_prec < 0) return xatu_fail(ctx, XATU_ERR_STATE, "BSE Hamiltonian is not initialized");
  if (!ctx->blas) {
    if (cublasCreate(&ctx->blas) != CUBLAS_STATUS_SUCCESS) return xatu_fail(ctx, XATU_ERR_CUDA, "cublasCreate failed");
  }
  cublasSetStream(ctx->blas, ctx->stream);
  const long long N = ctx->N;
  const size_t bytes = (size_t)N * nvec * sizeof(cd);
  if (ctx->dv_V.bytes < bytes) XATU_CK(ctx->dv_V.ensure(bytes));
  if (ctx->dv_W.bytes < bytes) XATU_CK(ctx->dv_W.ensure(bytes));
  XATU_CK(cudaMemcpyAsync(ctx->dv_V.p, X, bytes, cudaMemcpyHostToDevice, ctx->stream));
  xatu_status st = xatu_apply_h(ctx, N, 0, nvec);
  if (st != XATU_OK) return st;
  XATU_CK(cudaMemcpyAsync(Y, ctx->dv_W.p, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  xatu_hx_collect(ctx);
  int dst = 0;
  XATU_CK(cudaMemcpy(&dst, ctx->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (dst) {
    cudaMemset(ctx->d_status.p, 0, sizeof(int));
    return xatu_fail(ctx, XATU_ERR_NOT_CONVERGED, "tensor-core product: a pipeline wait timed out");
  }
  return XATU_OK;
}

xatu_status xatu_davidson_stats(const xatu_ctx* ctx, int* iterations, double* max_residual) {
  if (!ctx) return XATU_ERR_INVALID;
  if (iterations) *iterations = ctx->dav_iters;
  if (max_residual) *max_residual = ctx->dav_maxres;
  return XATU_OK;
}

xatu_status xatu_stage_times(const xatu_ctx* ctx, float* ms4) {
  if (!ctx || !ms4) return XATU_ERR_INVALID;
  for (int i = 0; i < 4; i++) ms4[i] = ctx->stage_ms[i];
  return XATU_OK;
}

xatu_status xatu_kernel_stats(const xatu_ctx* ctx, int which, int64_t* launches, double* total_ms, int* path) {
  if (!ctx || !launches || !total_ms || !path) return XATU_ERR_INVALID;
  if (which == 0) {
    *launches = ctx->built_prec >= 0 ? 1 : 0;
    *total_ms = ctx->stage_ms[2];
    *path = ctx->last_assembly_path;
  } else if (which == 1) {
    *launches = ctx->hx_calls;
    *total_ms = ctx->hx_ms;
    *path = ctx->hx_last_path;
  } else if (which == 2) {
    *launches = ctx->adjoint_ms > 0 ? 1 : 0;
    *total_ms = ctx->adjoint_ms;
    *path = 0;
  } else if (which == 3) {
    *launches = ctx->adj_pair_ms > 0 ? 1 : 0;
    *total_ms = ctx->adj_pair_ms;
    *path = 0;
  } else {
    return XATU_ERR_INVALID;
  }
  return XATU_OK;
}

xatu_status xatu_kernel_launches(const xatu_ctx* ctx, int64_t* count) {
  if (!ctx || !count) return XATU_ERR_INVALID;
  *count = ctx->launches;
  return XATU_OK;
}

// ------------------------------------------------------------------ geometry helpers
xatu_status xatu_reciprocal_lattice(int ndim, const double* bravais, double* recip) {
  if (ndim < 1 || ndim > 3 || !bravais || !recip) return XATU_ERR_INVALID;
  double r[9];
  if (!xatu_geo::reciprocal_lattice(ndim, bravais, r)) return XATU_ERR_INVALID;
  std::memcpy(recip, r, sizeof(double) * 3 * ndim);
  return XATU_OK;
}

xatu_status xatu_mesh_mp(int ndim, const double* recip, int n, double* kpoints) {
  if (ndim < 1 || ndim > 3 || !recip || !kpoints || n < 1) return XATU_ERR_INVALID;
  std::vector<double> k = xatu_geo::mp_mesh(ndim, recip, n);
  std::memcpy(kpoints, k.data(), k.size() * sizeof(double));
  return XATU_OK;
}

xatu_status xatu_mesh_reduced(int ndim, const double* recip, int n, int factor, double* kpoints) {
  if (ndim < 1 || ndim > 3 || !recip || !kpoints || n < 1 || factor < 1) return XATU_ERR_INVALID;
  std::vector<double> k = xatu_geo::reduced_mesh(ndim, recip, n, factor);
  std::memcpy(kpoints, k.data(), k.size() * sizeof(double));
  return XATU_OK;
}

xatu_status xatu_equivalent_points(int ndim, const double* recip, int n_eff, int npts, const double* k, int* index) {
  if (ndim < 1 || ndim > 3 || !recip || !k || !index || n_eff < 1 || npts < 0) return XATU_ERR_INVALID;
  double inv[9];
  if (!xatu_geo::inverse_gram(ndim, recip, inv)) return XATU_ERR_INVALID;
  for (int i = 0; i < npts; i++) index[i] = xatu_geo::equivalent_point(ndim, recip, inv, n_eff, k + 3 * i);
  return XATU_OK;
}

xatu_status xatu_truncate_supercell(int ndim, const double* bravais, int ncell, double radius, int* count,
                                    double* cells) {
  if (ndim < 1 || ndim > 3 || !bravais || !count || ncell < 1) return XATU_ERR_INVALID;
  std::vector<double> c = xatu_geo::truncate_supercell(ndim, bravais, ncell, radius);
  *count = (int)(c.size() / 3);
  if (cells) std::memcpy(cells, c.data(), c.size() * sizeof(double));
  return XATU_OK;
}

}  // extern "C"
