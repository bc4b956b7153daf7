// Launch-parameter structs shared by the host orchestration (api.cu) and
// the kernels.  Passed by value as kernel arguments.
#pragma once
#include "common.cuh"

// Raises (never lowers) a kernel's dynamic shared-memory limit on the current device (api.cu).
cudaError_t xatu_raise_smem_limit(const void* kernel, size_t bytes);

// Reciprocal-space kernel table: entry e is the k - k' difference with
// integer grid offsets (e / stride_d) % len_d - span_d along each reciprocal
// axis, q = q0 + sum_d off_d b_d / n_eff.
struct RecipTable {
  int ndim;
  int n_eff;
  int span[3];
  int len[3];
  double b[9];            // reciprocal vectors (ndim x 3)
  int nG;
  double q0[3];
};

struct BandParams {
  int nk;
  int norb;
  int nR;
  int triangular;
  int nb;                 // selected bands
  int band_list[2 * XATU_MAX_BANDS];
  double shift[3];        // k -> k + shift (Q)
  int max_sweeps;
  int has_overlap;        // Loewdin orthogonalisation with S(k) (SystemTB.cpp:113-156)
  int is_au;              // H in Hartree: scaled by 27.2 before the orthogonalisation (SystemTB.cpp:117-120)
};

struct AsmParams {
  int nk, nv, nc, nb, norb, na;
  int64_t N;
  int mode;          // 0 real space, 1 reciprocal space
  int exchange;
  double scissor;
  EquivMap emap;
  int rt_ndim;
  int rt_len[3];
  int rt_span[3];
  int orb_off[XATU_MAX_ATOMS + 1];
  int64_t nentries;  // rows of the interaction table
  int64_t ldk;       // row pitch (complex elements) of the mixed-precision planes
};

struct AsmInputs {
  const double* kpoints;   // nk x 3
  const int* kgrid;        // nk x 3 integer grid offsets (reciprocal mode)
  const double* eigval;    // nk x nb
  const double* eigvalQ;
  const cd* eigvec;        // nk x nb x norb
  const cd* eigvecQ;
  const cd* table;         // entries x na x na
  const cd* exL;           // N x na
  const cd* exR;           // N x na
  int* status;             // device error word
  const int* basis;        // NULL, or N x 3 (k, valence column, conduction index) of a caller-given basis
  unsigned char* tc_ops;   // NULL, or scratch for the tensor-core tile's operand images (assembly_tc.cuh)
  size_t tc_ops_bytes;
};

struct AsmOutputs {
  cd* H;                   // FP64: N x N
  __nv_bfloat162* Khi;     // MIXED: N x ldk, upper block triangle (xatu_kstored)
  __nv_bfloat162* Klo;
  double* diag;            // MIXED: N
};

// One system of a batched (mixed-precision) assembly launch.
struct AsmBatchMember {
  AsmParams p;
  AsmInputs in;
  AsmOutputs out;
  int nblk;                // k blocks of the tile size in use
  int pad;
};


// Row of the interaction table for the pair (k, k2) of exciton k points:
// real space: the mesh point equivalent to k2 - k (findEquivalentPointBZ);
// reciprocal space: the integer grid offset k - k2.  P needs the members
// mode, emap, rt_ndim, rt_len, rt_span and nentries.  Returns -1 when the entry
// falls outside the table.
template <class P>
__device__ __forceinline__ int64_t interaction_entry(const P& p, const double* __restrict__ kpoints,
                                                     const int* __restrict__ kgrid, int k, int k2) {
  int64_t e;
  if (p.mode == 0) {
    const double dx = kpoints[3 * k2] - kpoints[3 * k];
    const double dy = kpoints[3 * k2 + 1] - kpoints[3 * k + 1];
    const double dz = kpoints[3 * k2 + 2] - kpoints[3 * k + 2];
    e = equivalent_index(p.emap, dx, dy, dz);
  } else {
    e = 0;
    int64_t stride = 1;
    for (int d = 0; d < p.rt_ndim; d++) {
      const int off = kgrid[3 * k + d] - kgrid[3 * k2 + d];
      e += (int64_t)(off + p.rt_span[d]) * stride;
      stride *= p.rt_len[d];
    }
  }
  return (e < 0 || e >= p.nentries) ? -1 : e;
}
