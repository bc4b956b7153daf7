// Declarations of the engine's kernels and launchers (internal).
#pragma once
#include "params.h"

extern "C" __global__ void pair_potential_kernel(PotParams p, int kind, int deriv, int na, const double* motif,
                                                 int ncells, const double* cells, int npairs, const int2* pairs,
                                                 double* vtab);
extern "C" __global__ void motif_ft_kernel(int nq, const double* q, int ncells, const double* cells, int npairs,
                                           const int2* pairs, const double* vtab, double inv_total, int na, cd* out);
extern "C" __global__ void motif_ft_roots_kernel(int nq, const int* mi, int den, int ncells, const int* ni,
                                                 int npairs, const int2* pairs, const double* vtab, double inv_total,
                                                 int na, cd* out);
#define XATU_FT_MAXDEN 1536   // largest mesh denominator of the root-of-unity table (24 KB of shared memory)
#define XATU_MOTIF_QB 8       // mesh points per CTA of motif_ft_roots_kernel (a warp per point)
extern "C" size_t motif_roots_smem(int den);
extern "C" __global__ void recip_table_kernel(PotParams p, RecipTable t, int deriv, int nentries, const double* G,
                                              int na, const double* motif, cd* W);
extern "C" __global__ void exchange_vectors_kernel(int N, int nv, int nc, int nb, int norb, int na, const int* orb_off,
                                                   const cd* eigvec, const cd* eigvecQ, const cd* VX, const int* basis,
                                                   cd* L, cd* R);
extern "C" __global__ void band_solve_kernel(BandParams bp, const double* kpoints, const double* cellsR, const cd* HR,
                                             const cd* SR, double* eigval, cd* eigvec, int* status);
extern "C" size_t band_solve_smem(int norb, int nR, int has_overlap);
// Band-window solve (bands_select.cu): eigenpairs of the band list only, models without overlap.
extern "C" bool xatu_band_select_supported(int norb, int nb, int has_overlap);
extern "C" cudaError_t xatu_launch_band_select(const BandParams& bp, const double* kpoints, const double* cellsR,
                                               const cd* HR, double* eigval, cd* eigvec, int* status,
                                               cudaStream_t s);
cudaError_t xatu_launch_assembly(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out, bool mixed,
                                 bool force_generic, cudaStream_t s, int* path);

// Single-system tile kernels (assembly_f32.cu / assembly_f64.cu).
// Bytes of operand-image scratch (AsmInputs::tc_ops) the tensor-core kernels of p's class need (row panels or
// tiles, whichever needs more); 0 when the class takes neither.
size_t xatu_assembly_tc_scratch_bytes(const AsmParams& p);
// *tensor_cores: the band overlaps ran on tcgen05; *panel: in the row-panel kernel (assembly_panel.cuh).
cudaError_t xatu_dispatch_tile_f32(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out, cudaStream_t s,
                                   bool* launched, bool* tensor_cores, bool* panel);
cudaError_t xatu_dispatch_tile_f64(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out, cudaStream_t s,
                                   bool* launched);
// Batched persistent assembly (assembly_batch.cu), mixed precision, one band-window class per launch.
bool xatu_assembly_batch_supported(int nv, int nc, int na);
size_t xatu_assembly_batch_smem(int nv, int nc, int na, int tk, int norb, int exchange);
cudaError_t xatu_launch_assembly_batch(int nv, int nc, int na, int tk, const AsmBatchMember* members,
                                       const int2* work, int nwork, int* counter, size_t smem, int num_sms,
                                       bool set_attr, cudaStream_t s);
