/*
 * xatu_bse.h -- C ABI of the B200 BSE engine.
 *
 * The engine replaces the hot path of Xatu's ExcitonTB:
 *
 *   ExcitonTB::initializeHamiltonian()         include/xatu/ExcitonTB.hpp:140
 *   ExcitonTB::BShamiltonian() / (basis)       include/xatu/ExcitonTB.hpp:141-142
 *   ExcitonTB::diagonalize(method, nstates)    include/xatu/ExcitonTB.hpp:143
 *
 * together with the pure virtuals they implement (include/xatu/Exciton.hpp:117,125-126).
 * Plain pointers and sizes only; no C++ or torch types cross this boundary.
 *
 * Conventions
 *   - Complex numbers are interleaved (re, im) doubles.
 *   - Matrices are row-major unless stated otherwise.  The tight-binding
 *     matrices H(R) are given per cell as [R][row][col] (an Armadillo cube
 *     slice is column-major; a caller holding one passes each slice
 *     transposed).
 *   - Units: Angstrom and eV, as in the reference.
 *   - Every call returns a status; xatu_last_error() gives the message of the
 *     last failing call on that context.  No call throws, exits or spins
 *     without bound.
 *   - A context owns one CUDA stream on the device it was created on and all
 *     device buffers (band stacks, interaction tables, the BSE matrix).  One
 *     context per host thread.
 */
#ifndef XATU_BSE_H
#define XATU_BSE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct xatu_ctx xatu_ctx;
typedef int xatu_status;

enum {
  XATU_OK = 0,
  XATU_ERR_INVALID = 1,        /* bad argument or inconsistent sizes (reference: std::invalid_argument) */
  XATU_ERR_CUDA = 2,           /* a CUDA / cuSOLVER / cuBLAS call failed */
  XATU_ERR_NOT_CONVERGED = 3,  /* an iterative solver hit its iteration or time cap */
  XATU_ERR_STATE = 4,          /* call out of order (e.g. solve before build) */
  XATU_ERR_ALLOC = 5,          /* device or host allocation failed */
  XATU_ERR_UNSUPPORTED = 6,    /* valid input outside what this build supports */
  XATU_ERR_NUMERIC = 7         /* NaN/Inf found in inputs or results */
};

enum { XATU_MODE_REALSPACE = 0, XATU_MODE_RECIPROCAL = 1 };          /* ExcitonTB::setMode */
enum { XATU_POT_KELDYSH = 0, XATU_POT_COULOMB = 1 };                  /* ExcitonTB::selectPotential */
enum { XATU_GAUGE_LATTICE = 0, XATU_GAUGE_ATOMIC = 1 };               /* ExcitonTB::setGauge */

/* Storage/arithmetic of the assembled BSE matrix. */
enum {
  XATU_PREC_FP64 = 0,   /* complex128 H, FP64 arithmetic (parity mode; the reference's HBS_) */
  XATU_PREC_MIXED = 1   /* FP64 band-energy diagonal + interaction kernel in split BF16 (hi + lo),
                           FP32 arithmetic; the tensor-core solve path */
};

/* Solvers for xatu_bse_solve (ExcitonTB::diagonalizeRaw, ExcitonTB.cpp:930-959). */
enum {
  XATU_SOLVER_DENSE_FP64 = 0,  /* all eigenpairs, FP64 (the reference's "diag"); needs XATU_PREC_FP64 */
  XATU_SOLVER_DAVIDSON = 1     /* lowest nstates; block Davidson, FP64 orthogonalisation and Rayleigh-Ritz,
                                  H.X on tcgen05 tensor cores from the split-BF16 kernel (XATU_PREC_MIXED)
                                  or FP64 CUDA cores (XATU_PREC_FP64) */
};

/* SystemTB inputs (System.hpp:20-40, Lattice.hpp:21-63, SystemConfiguration.hpp:13-36). */
typedef struct {
  int ndim;                    /* 1, 2 or 3 */
  const double *bravais;       /* ndim x 3 */
  int natoms;
  const double *motif;         /* natoms x 4: x, y, z, species index */
  int nspecies;
  const int *norbitals;        /* orbitals per species */
  int ncells;                  /* number of H(R) matrices */
  const double *cells;         /* ncells x 3, R vectors */
  const double *hamiltonian;   /* ncells x norb x norb complex, [R][row][col] */
  const double *overlap;       /* NULL, or like hamiltonian (non-orthogonal basis, Loewdin) */
  int filling;                 /* electrons; Fermi level band = filling - 1 */
  int is_triangular;           /* -1: detect from H(R_0) like checkIfTriangular (utils.cpp:176-178) */
  int is_au;                   /* energies in Hartree (scaled by 27.2 in solveBands, SystemTB.cpp:117-120) */
} xatu_system_desc;

/* ExcitonTB parameters (ExcitonTB.hpp:30-45, Exciton.hpp:29-48). */
typedef struct {
  int ncell;                   /* k points per axis of the full mesh (before the submesh factor) */
  int factor;                  /* reduced-mesh factor (Lattice::reducedBrillouinZoneMesh), 1 = full mesh */
  int nk;                      /* rows of kpoints */
  const double *kpoints;       /* nk x 3: the exciton basis k points (Lattice::kpoints) */
  int nmesh;                   /* rows of mesh ((ncell*factor)^ndim) */
  const double *mesh;          /* nmesh x 3: full BZ mesh (Lattice::meshBZ); NULL = kpoints */
  int nvalence, nconduction;
  const int *valence_bands;    /* absolute band indices (ExcitonTB::valenceBands) */
  const int *conduction_bands; /* absolute band indices (ExcitonTB::conductionBands) */
  double eps_m, eps_s, r0;
  double regularization;       /* < 1e-10 -> |a1| (ExcitonTB.cpp:803-805) */
  double cutoff;               /* ExcitonTB::cutoff_ in units of |a1|; <= 0 -> ncell / 2.5 */
  double Q[3];                 /* exciton centre-of-mass momentum */
  double scissor;
  int exchange;                /* 0 / 1 */
  int mode;                    /* XATU_MODE_* */
  int n_reciprocal;            /* reciprocal vectors per axis (ExcitonTB::nReciprocalVectors) */
  int potential;               /* XATU_POT_* for the direct term (real space) */
  int exchange_potential;      /* XATU_POT_* for the exchange term (real space) */
  int gauge;                   /* XATU_GAUGE_* */
} xatu_exciton_desc;

/* ------------------------------------------------------------------ context */
xatu_status xatu_ctx_create(xatu_ctx **ctx, int device);
xatu_status xatu_ctx_destroy(xatu_ctx *ctx);
const char *xatu_last_error(const xatu_ctx *ctx);
/* Run the context's work on an external stream (cudaStream_t passed as void*; NULL = own stream). */
xatu_status xatu_ctx_set_stream(xatu_ctx *ctx, void *stream);
int xatu_abi_version(void);

/* ------------------------------------------------------------------ inputs */
/* Copies the SystemTB arrays (the constructor SystemTB(SystemConfiguration), SystemTB.cpp:29-31). */
xatu_status xatu_system_upload(xatu_ctx *ctx, const xatu_system_desc *sys);
/* Copies the exciton parameters, builds the e-h basis (Exciton::createBasis, Exciton.tpp:128-147), the
   real-space cell list (Lattice::truncateSupercell, Lattice.cpp:320-341) and the reciprocal-vector list
   (Lattice::truncateReciprocalSupercell, Lattice.cpp:349-370).  ExcitonTB::initializeHamiltonian's guards
   (ExcitonTB.cpp:794-815) apply. */
xatu_status xatu_exciton_set(xatu_ctx *ctx, const xatu_exciton_desc *exc);

/* ------------------------------------------------------------------ initializeResultsH0 (ExcitonTB.cpp:707-787) */
/* Band solve at every k (and k+Q) on the device: Bloch H(k) (SystemTB.cpp:60-75), Hermitian eigensolve
   (SystemTB.cpp:113-125), fixGlobalPhase (ExcitonTB.cpp:673-683), band selection. */
xatu_status xatu_bands_compute(xatu_ctx *ctx);
/* Alternative: caller-supplied band stacks (gauge-controlled parity).  eigval: nk x nb,
   eigvec: nk x nb x norb complex (band b of k at [k][b][:]); nb = nvalence + nconduction, valence first.
   eigvalQ/eigvecQ may be NULL when Q = 0. */
xatu_status xatu_bands_upload(xatu_ctx *ctx, const double *eigval, const double *eigvec,
                              const double *eigvalQ, const double *eigvecQ);
xatu_status xatu_bands_download(xatu_ctx *ctx, double *eigval, double *eigvec, double *eigvalQ,
                                double *eigvecQ);
/* Interaction tables: motif lattice Fourier transform V_ab(q) over the mesh (ExcitonTB.cpp:438-476, :761-786)
   or, in reciprocal mode, the G-summed kernel (ExcitonTB.cpp:410-426, :562-621). */
xatu_status xatu_interaction_build(xatu_ctx *ctx);
/* nmesh x na x na complex, and na x na complex (exchange at Q). */
xatu_status xatu_motif_ft_download(xatu_ctx *ctx, double *ft_stack, double *ft_Q);

/* ------------------------------------------------------------------ BShamiltonian (ExcitonTB.cpp:840-921) */
/* Runs the band solve and interaction tables if they are not current, then assembles H on the device. */
xatu_status xatu_bse_build(xatu_ctx *ctx, int precision);
/* ExcitonTB::BShamiltonian(const arma::imat& basis) (ExcitonTB.cpp:840-849): assemble H over a caller-given
   subset of e-h states; basis: nbasis rows {valence band, conduction band, k index} with absolute band numbers
   (the reference's basisStates layout).  The following solve works on this nbasis x nbasis matrix; a plain
   xatu_bse_build returns to the full basis. */
xatu_status xatu_bse_build_basis(xatu_ctx *ctx, int precision, int64_t nbasis, const int *basis);
xatu_status xatu_bse_dim(const xatu_ctx *ctx, int64_t *n);
/* Full Hermitian H, row-major N x N complex (FP64 build), or the mixed build expanded to complex128
   (diagonal band term + split-BF16 kernel). */
xatu_status xatu_bse_copy_to_host(xatu_ctx *ctx, double *H);
/* Device pointer and layout of the assembled matrix (row-major complex128 for FP64; for MIXED the two
   split-BF16 planes hi and lo, each N x ldk complex bf16 with ldk = N rounded up to a multiple of 4, and the
   FP64 diagonal).  The MIXED planes hold the Hermitian kernel's upper block triangle only: with blocks of
   128 x 128 elements, element (r, c) is stored when c / 128 >= r / 128 (the diagonal blocks in full); any
   other element is the conjugate of its mirror (c, r). */
xatu_status xatu_bse_device_buffers(xatu_ctx *ctx, void **h_or_hi, void **lo, void **diag);

/* ------------------------------------------------------------------ diagonalize (ExcitonTB.cpp:930-972) */
/* DAVIDSON: eigval receives nstates doubles (ascending).  DENSE_FP64: eigval receives all N eigenvalues
   (ascending), like arma::eig_sym.  eigvec: NULL, or the eigenvectors of the lowest nstates states
   (all N when nstates <= 0 with DENSE_FP64) as N x nstates complex, column s = state s, column-major
   (Armadillo layout). */
xatu_status xatu_bse_solve(xatu_ctx *ctx, int solver, int nstates, double *eigval, double *eigvec);
/* Davidson controls: residual tolerance (eV), iteration cap, block size (0 = automatic). */
xatu_status xatu_davidson_config(xatu_ctx *ctx, double tol, int max_iter, int block);
/* Iterations used by the last Davidson solve. */
xatu_status xatu_davidson_stats(const xatu_ctx *ctx, int *iterations, double *max_residual);
/* Kernel of H.X for the mixed build: 0 automatic (tcgen05 tensor cores when the layout allows), 1 CUDA cores,
   2 tensor cores.  No reference counterpart (the reference multiplies dense Armadillo matrices, davidson.cpp:31-37). */
xatu_status xatu_hx_backend(xatu_ctx *ctx, int backend);
/* Band-solve algorithm (no counterpart in the reference, which diagonalises every H(k) in full with
   Armadillo, SystemTB.cpp:113-125): 0 auto (band window when supported), 1 full Jacobi eigensolve of every
   H(k), 2 eigenpairs of the band list only (Householder tridiagonalisation, Sturm multisection, inverse
   iteration; models without overlap matrices, norb <= 64, at most 16 bands; XATU_ERR_UNSUPPORTED
   otherwise).  Same results to rounding for bands that are not degenerate. */
xatu_status xatu_bands_backend(xatu_ctx *ctx, int backend);
/* Y = H X for nvec host vectors with the current build (X, Y: N x nvec complex, column-major); the product the
   Davidson iterations use. */
xatu_status xatu_kernel_matvec(xatu_ctx *ctx, int nvec, const double *X, double *Y);

/* ------------------------------------------------------------------ oscillator strengths */
/* ResultTB::excitonOscillatorStrength (ResultTB.cpp:242-298; skubo_w.f90:175-330, 445-628): velocity matrix
   elements of the excitons given by `eigvec` (host, N x nstates complex, column-major), in atomic units.
   vme_ex receives 3 x nstates complex, column-major (the reference's 3 x N matrix restricted to these states).
   Uses the band stacks of the context (bands computed or uploaded).  Unlike the reference, no argument is
   modified in place. */
xatu_status xatu_oscillator_strength(xatu_ctx *ctx, int nstates, const double *eigvec, double *vme_ex);

/* ------------------------------------------------------------------ post-processing of exciton states */
/* The observables and writers of Result / ResultTB evaluated on the device for a batch of states.  eigvec is
   host, N x nstates complex, column-major, in the full e-h basis of the context (row k*nc*nv + c*nv + v); the
   band stacks are the context's (computed or uploaded).  XATU_ERR_UNSUPPORTED when the last build used a
   caller-given basis subset. */

/* Per-state reductions, each output optional (NULL skips it):
     kinetic[s]       Result::kineticEnergy (Result.tpp:25-40): sum |A|^2 (E^Q_c(k) - E_v(k)), no scissor;
     kweight[s*nk+k]  sum_{c,v} |A(k,c,v)|^2, the numerator of writeReciprocalAmplitude / ftExcitonEnvelope
                      (Result.tpp:101-128, :160-226);
     peak[s]          Result::findExcitonPeak (Result.tpp:478-484): k index of the first largest |A|;
     spin[6*s ..]     ResultTB::spinX (ResultTB.cpp:21-98) as three complex numbers {total, hole, electron};
                      XATU_ERR_INVALID when an atom has an odd number of orbitals (the reference throws). */
xatu_status xatu_state_observables(xatu_ctx *ctx, int nstates, const double *eigvec, double *kinetic,
                                   double *kweight, int64_t *peak, double *spin);

/* ResultTB::realSpaceWavefunction (ResultTB.cpp:310-357) for every state, electron cell and electron atom:
   out[(s*ncells + cell)*natoms + atom] = sum over the orbitals a of `atom` and b of atom hole_index of
   |sum_{k,c,v} C^Q_{k,c}[a] conj(C_{k,v}[b]) A_s(k,c,v) exp(i k.(cells[cell] - hole_cell))|^2 -- the loop of
   writeRealspaceAmplitude (ResultTB.cpp:370-408).  cells: ncells x 3 (Angstrom); hole_cell: 3. */
xatu_status xatu_realspace_amplitude(xatu_ctx *ctx, int nstates, const double *eigvec, int hole_index,
                                     const double *hole_cell, int ncells, const double *cells, double *out);

/* Result::ftExcitonEnvelope (Result.tpp:101-128) at npoints separations d = r_e - r_h (npoints x 3):
   out[s*npoints + p] = Re sum_k kweight_s(k) exp(-i k.d_p). */
xatu_status xatu_envelope_ft(xatu_ctx *ctx, int nstates, const double *eigvec, int npoints, const double *points,
                             double *out);

/* Broadening of the exciton peaks in skubo_w's broad_vector (skubo_w.f90:684-720); any other value keeps the
   reference's default weight 1. */
enum {
  XATU_BROAD_OTHER = 0,
  XATU_BROAD_LORENTZIAN = 1,
  XATU_BROAD_GAUSSIAN = 2,
  XATU_BROAD_EXPONENTIAL = 3
};
/* ResultTB::writeAbsorptionSpectrum -> skubo_w (ResultTB.cpp:412-461, skubo_w.f90:2-173) without the file
   I/O: frequencies w_i = (w0 + wrange/nw * i) eV, i < nw, broadening eta (eV) -- the kubo_w.in parameters.
     sigma_sp  nw x 9 complex: the single-particle Kubo conductivity sigma_ij(w) over every (k, c, v) with
               the Gaussian delta of get_kubo_intens (skubo_w.f90:630-681); the file holds -Re.
     sigma_ex  nw x 9 real: sum_n Re(pi/(nk vcell) conj(V_i,n) V_j,n / E_n) broadening(w - E_n), i, j < 2
               (the other entries 0, as in the reference), over the nstates given states.
     vme_ex    optional, 3 x nstates complex column-major: their velocity matrix elements (atomic units).
   eigval: nstates exciton energies (eV).  nstates = 0 computes the single-particle part only.  vcell is
   |a1 x a2| in bohr^2 as in skubo_w.f90:69-71; it is zero for a one-dimensional lattice, where the reference
   divides by it and so does this entry (infinite or NaN values). */
xatu_status xatu_absorption(xatu_ctx *ctx, int nstates, const double *eigval, const double *eigvec, double w0,
                            double wrange, int nw, double eta, int broadening, double *sigma_sp, double *sigma_ex,
                            double *vme_ex);

/* ------------------------------------------------------------------ adjoint gradients */
#define XATU_ADJOINT_MAX_STATES 8
/* Hellmann-Feynman gradients dE_n/dtheta = x_n^H (dH/dtheta) x_n of exciton energies through the whole path
   (band solve, fixGlobalPhase, interaction tables, BShamiltonian).  No reference counterpart: the reference has
   no derivative code; this differentiates what ExcitonTB::initializeHamiltonian / BShamiltonian compute
   (ExcitonTB.cpp:673-683, 707-921; SystemTB.cpp:60-156).
   eigvec: host, N x nstates complex, column-major, normalised eigenvectors of the current build (for example
   those returned by xatu_bse_solve); nstates <= XATU_ADJOINT_MAX_STATES.  The band eigenvectors are
   recomputed on the device, not stored.
   grad_hamiltonian (or NULL): nstates x nR x norb x norb complex, G_n(R)_ab = dE_n/dRe H(R)_ab + i dE_n/dIm H(R)_ab
   for perturbations that keep H(k) Hermitian (with full storage, perturb H(R)_ab and H(-R)_ba = conj together;
   the first-order change is dE = Re sum conj(G) dH).  Needs bands from xatu_bands_compute; undefined (and
   XATU_ERR_NUMERIC) where a selected band is degenerate with another band.
   grad_params (or NULL): nstates x 3 doubles, dE_n/dr0, dE_n/deps_m, dE_n/deps_s.
   Supported: full e-h basis, at most 2 valence and 2 conduction bands, at most 4 atoms, both modes,
   exchange, Q, overlap. */
xatu_status xatu_adjoint(xatu_ctx *ctx, int nstates, const double *eigvec, double *grad_hamiltonian,
                         double *grad_params);

/* Summed oscillator strength F = sum_{n: e_lo <= E_n <= e_hi} sum_j |vme_ex_j(n)|^2 of the excitons in an
   energy window (ResultTB::excitonOscillatorStrength, ResultTB.cpp:242-298, summed over the window) and its
   gradients: dF/d(r0, eps_m, eps_s) through the eigenvectors (grad_params, 3 doubles) and dF/dH(R)
   (grad_hamiltonian, nR x norb x norb complex, same convention as xatu_adjoint) through the eigenvectors, the
   bands and the velocity matrix elements; either may be NULL.  Needs an FP64 build; computes all eigenpairs
   on the device (dense solver).  *nwindow = number of states in the window.  The hopping gradient needs bands
   from the model, Q = 0 and full (non-triangular) storage.  No reference counterpart for the gradient. */
xatu_status xatu_oscillator_window_gradient(xatu_ctx *ctx, double e_lo, double e_hi, int *nwindow, double *F,
                                            double *grad_params, double *grad_hamiltonian);

/* ------------------------------------------------------------------ batches of systems */
/* Many BSE instances of uneven size (k grids, band windows, dielectric parameters) built and solved together
   on one GPU.  No reference counterpart (the reference handles one ExcitonTB at a time); each member follows
   initializeHamiltonian + BShamiltonian(mixed) + diagonalize("davidson") of one system.  The first
   xatu_batch_run tunes the assembly tile of each band-window class on the batch's own data and records the
   build (band solves, tables, one persistent assembly launch per class) and one step of a lockstep block
   Davidson into CUDA graphs; later runs replay them.  Supported members: 1-3 valence and 1-3 conduction bands,
   2-3 atoms, BSE dimension >= 64, lowest nstates <= 12 (block of at most 16 vectors). */
typedef struct xatu_batch xatu_batch;
xatu_status xatu_batch_create(xatu_batch **batch, int device);
xatu_status xatu_batch_destroy(xatu_batch *batch);
const char *xatu_batch_last_error(const xatu_batch *batch);
/* cudaStream_t as void*, NULL = the batch's own stream; before the first run. */
xatu_status xatu_batch_set_stream(xatu_batch *batch, void *stream);
/* Adds one system (copies the descriptors' arrays, as xatu_system_upload + xatu_exciton_set); *index = its slot. */
xatu_status xatu_batch_add(xatu_batch *batch, const xatu_system_desc *sys, const xatu_exciton_desc *exc, int *index);
/* Builds and solves every member: lowest nstates, residual tolerance tol (<= 0: 1e-4), at most max_iter
   Davidson steps (<= 0: 200).  nstates, tol and max_iter are fixed by the first run. */
xatu_status xatu_batch_run(xatu_batch *batch, int nstates, double tol, int max_iter);
xatu_status xatu_batch_dim(const xatu_batch *batch, int index, int64_t *n);
/* eigval: nstates; eigvec: N x nstates complex, column-major (either may be NULL). */
xatu_status xatu_batch_result(xatu_batch *batch, int index, double *eigval, double *eigvec);
/* Device ms of the last run's build graph and Davidson iterations, the number of lockstep iterations, the
   iterations each member needed (array of the batch size, or NULL) and the autotuner's choices as JSON text. */
xatu_status xatu_batch_stats(const xatu_batch *batch, double *build_ms, double *solve_ms, int *iterations,
                             int *member_iterations, char *tuning, size_t tuning_len);

/* ------------------------------------------------------------------ instrumentation */
/* Device milliseconds of the last run of each stage: [0] bands, [1] interaction tables, [2] assembly,
   [3] solve.  Measured with CUDA events on the context's stream. */
xatu_status xatu_stage_times(const xatu_ctx *ctx, float *ms4);
/* Device time of one kernel family measured with CUDA events on the context's stream: which = 0 the BSE
   assembly (last build), 1 the K.X products of the last Davidson solve, 2 the last xatu_adjoint call (first
   to last launch), 3 its pair kernel.  *path: for the K.X products 1 CUDA cores, 2 tcgen05; for the assembly
   0 tile kernel on CUDA cores, 1 element-wise kernel, 2 tile kernel with the band overlaps on tcgen05, 3 row-panel
   kernel with the band overlaps on tcgen05; 0 where it does not apply. */
xatu_status xatu_kernel_stats(const xatu_ctx *ctx, int which, int64_t *launches, double *total_ms, int *path);
/* Number of engine kernels launched on this context since creation. */
xatu_status xatu_kernel_launches(const xatu_ctx *ctx, int64_t *count);
/* Self-test of the device eigensolver of the Davidson Rayleigh-Ritz step (no counterpart in the reference,
   whose Davidson calls Armadillo's eig_sym on the projected matrix, davidson.cpp:30): the lowest k
   eigenpairs of the Hermitian m x m matrix T (host, column-major complex128), m <= 112, k <= m.  Outputs
   theta[k] ascending and Y (host, m x k column-major complex128); cycles (may be NULL): 8 SM clock stamps
   at the solver's phase boundaries.  Allocates and frees its own device buffers; XATU_ERR_NUMERIC when the
   solver flagged a breakdown. */
xatu_status xatu_selftest_small_eigh(int device, int m, int k, const double *T, double *theta, double *Y,
                                     int64_t *cycles);

/* ------------------------------------------------------------------ allocation-free product */
/* y = H x for a mixed build (FP64 diagonal + split-BF16 kernel planes), without any device allocation.
   No counterpart in the reference: it exists for callers that cannot call cudaMalloc -- codes that keep
   (nearly) all of the GPU's memory in their own pool, and caller-written iterative eigensolvers that request
   the product thousands of times and cannot afford a cudaMalloc/cudaFree (device-wide synchronisation) per
   request.  All arguments are device pointers owned by the caller: k_hi, k_lo, diag as returned by
   xatu_bse_device_buffers for XATU_PREC_MIXED (n x ldk complex bf16 planes, ldk a multiple of 4, upper block
   triangle stored), x and y n x nvec complex128, column-major, 16-byte aligned.  Limits: n <= 16384,
   nvec <= 16; larger sizes return XATU_ERR_UNSUPPORTED with a message on stderr.  Scratch is one static 8 MB
   device array per GPU that loads
   the library, held until the process exits; the first call on a device (and the first after that device's
   context was recreated) looks up its address (do that first call before any stream capture).  Every call
   shares that array and leaves its contents behind, so calls that overlap on the GPU (other streams, other
   host threads) race.  Runs on `stream` (cudaStream_t, NULL = legacy default stream) and waits for it before
   returning, to read its status word: on a stream that is being captured it does nothing and returns
   XATU_ERR_STATE.  A tensor-core pipeline wait that timed out returns XATU_ERR_NOT_CONVERGED. */
xatu_status xatu_hx_noalloc(const void *k_hi, const void *k_lo, const double *diag, int64_t n, int64_t ldk, int nvec,
                            const double *x, double *y, void *stream);

/* ------------------------------------------------------------------ geometry helpers (host, no device work) */
/* Lattice::calculateReciprocalLattice (Lattice.cpp:56-80): out ndim x 3. */
xatu_status xatu_reciprocal_lattice(int ndim, const double *bravais, double *recip);
/* Lattice::brillouinZoneMesh (Lattice.cpp:140-162): out n^ndim x 3. */
xatu_status xatu_mesh_mp(int ndim, const double *recip, int n, double *kpoints);
/* Lattice::reducedBrillouinZoneMesh (Lattice.cpp:172-197): submesh n^ndim x 3 (mesh: xatu_mesh_mp(n*factor)). */
xatu_status xatu_mesh_reduced(int ndim, const double *recip, int n, int factor, double *kpoints);
/* Lattice::findEquivalentPointBZ (Lattice.cpp:251-279) for a batch of points: index into the n_eff mesh. */
xatu_status xatu_equivalent_points(int ndim, const double *recip, int n_eff, int npts, const double *k,
                                   int *index);
/* Lattice::truncateSupercell (Lattice.cpp:320-341): count only when cells == NULL. */
xatu_status xatu_truncate_supercell(int ndim, const double *bravais, int ncell, double radius, int *count,
                                    double *cells);

#ifdef __cplusplus
}
#endif

#endif /* XATU_BSE_H */
