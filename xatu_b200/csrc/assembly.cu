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
// Fast path: one thread per (k, k') pair of a 16 x 16 tile of k points; the
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
#include "params.h"

#define ASM_TK 16

__device__ __forceinline__ void split_store(__nv_bfloat162* hi, __nv_bfloat162* lo, int64_t idx, float re, float im) {
  const __nv_bfloat16 hr = __float2bfloat16_rn(re), hi_ = __float2bfloat16_rn(im);
  const __nv_bfloat16 lr = __float2bfloat16_rn(re - __bfloat162float(hr));
  const __nv_bfloat16 li = __float2bfloat16_rn(im - __bfloat162float(hi_));
  __nv_bfloat162 h; h.x = hr; h.y = hi_;
  __nv_bfloat162 l; l.x = lr; l.y = li;
  hi[idx] = h;
  lo[idx] = l;
}

__device__ __forceinline__ const cd* interaction_ptr(const AsmParams& p, const AsmInputs& in, int k, int k2) {
  int64_t e = interaction_entry(p, in.kpoints, in.kgrid, k, k2);
  if (e < 0) {
    atomicOr(in.status, XATU_DEVERR_INDEX);
    e = 0;
  }
  return in.table + e * p.na * p.na;
}

// Writes element (i, j) (and its mirror when i != j) given D - X.
template <typename T, bool MIXED>
__device__ __forceinline__ void write_element(const AsmParams& p, const AsmOutputs& out, int64_t i, int64_t j,
                                              cplx<T> dmx, double ec, double ev) {
  if (i == j) {
    if (MIXED) {
      split_store(out.Khi, out.Klo, i * p.ldk + i, (float)(-dmx.x), 0.0f);
      out.diag[i] = p.scissor + ec - ev;
    } else {
      const double hr = (p.scissor + ec - ev) / 2. - (double)dmx.x / 2.;
      const double hi = -(double)dmx.y / 2.;
      out.H[i * p.N + i] = mk(hr + hr, hi - hi);
    }
  } else {
    if (MIXED) {
      split_store(out.Khi, out.Klo, i * p.ldk + j, (float)(-dmx.x), (float)(-dmx.y));
      split_store(out.Khi, out.Klo, j * p.ldk + i, (float)(-dmx.x), (float)(dmx.y));
    } else {
      out.H[i * p.N + j] = mk(-(double)dmx.x, -(double)dmx.y);
      out.H[j * p.N + i] = mk(-(double)dmx.x, (double)dmx.y);
    }
  }
}

// Tiles: blockIdx.x enumerates the upper-triangular k-block pairs (kb <= kb2).
__device__ __forceinline__ void tile_of(int t, int nblk, int& kb, int& kb2) {
  // row kb holds nblk - kb tiles
  int r = 0, rem = t;
  while (rem >= nblk - r) { rem -= nblk - r; r++; }
  kb = r;
  kb2 = r + rem;
}

// Fast-path kernel.  CTA = a TK x TK tile of (k, k') pairs (TK = 16), one thread
// per pair.
//   phase 1: band coefficients of both k blocks (and the exchange factors of the
//            tile's rows and columns) are staged in shared memory;
//   phase 2: each thread forms T_a(v', v) = sum_b V_ab rho2_b(v', v), then for
//            every (c, c') the conduction factors rho1_a(c, c'), and writes the
//            final matrix values of its NC*NV x NC*NV block into a shared-memory
//            staging tile (the V table row is read on demand through L1);
//   phase 3: the tile and, off the diagonal, its conjugate transpose are written
//            to HBM row by row with coalesced stores (16-byte vectors for the
//            split-BF16 planes).
template <typename T, int NV, int NC, int NA, bool MIXED, int TK>
__device__ __forceinline__ void assemble_tile(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out,
                                              int nblk, int tile) {
  constexpr int NB = NV + NC;
  constexpr int NCV = NV * NC;
  constexpr int TR = TK * NCV;     // rows (and columns) of the staging tile
  constexpr int LDT = TR + 1;      // padded row pitch
  using E = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int kb, kb2;
  tile_of(tile, nblk, kb, kb2);
  const int norb = p.norb;
  const int side_sz = NB * norb * TK;
  E* sC = reinterpret_cast<E*>(smem_raw);                  // [2][NB][norb][TK]
  E* sTile = sC + 2 * side_sz;                             // [TR][LDT]
  E* sL = sTile + TR * LDT;                                // [TR][NA] exchange rows
  E* sR = sL + TR * NA;                                    // [TR][NA] exchange columns
  const int tid = threadIdx.x;
  const int kk = tid / TK, kk2 = tid % TK;
  const int k = kb * TK + kk, k2 = kb2 * TK + kk2;
  const bool active = (k < p.nk) && (k2 < p.nk) && !(kb == kb2 && k > k2);
  // FP32 path: the pair's interaction-table row goes to registers before the
  // staging barrier, so its L2 latency overlaps the coefficient staging.
  constexpr bool kPrefetchV = sizeof(T) == 4;
  E Vr[kPrefetchV ? NA : 1][kPrefetchV ? NA : 1];
  const cd* Vt = nullptr;
  if (active) {
    Vt = interaction_ptr(p, in, k, k2);
    if (kPrefetchV) {
#pragma unroll
      for (int a = 0; a < (kPrefetchV ? NA : 1); a++)
#pragma unroll
        for (int b = 0; b < (kPrefetchV ? NA : 1); b++) {
          const cd v = Vt[a * NA + b];
          Vr[a][b] = {(T)v.x, (T)v.y};
        }
    }
  }
#pragma unroll 4
  for (int t = tid; t < 2 * side_sz; t += blockDim.x) {
    const int side = t / side_sz;
    const int r = t - side * side_sz;
    const int band = r / (norb * TK);
    const int r2 = r - band * norb * TK;
    const int o = r2 / TK;
    const int kk = r2 - o * TK;
    const int k = (side == 0 ? kb : kb2) * TK + kk;
    E v = {T(0), T(0)};
    if (k < p.nk) {
      // valence bands from the k stack, conduction bands from the k+Q stack
      const cd c = (band < NV) ? in.eigvec[((int64_t)k * p.nb + band) * norb + o]
                               : in.eigvecQ[((int64_t)k * p.nb + band) * norb + o];
      v.x = (T)c.x;
      v.y = (T)c.y;
    }
    sC[t] = v;
  }
  const int64_t row0 = (int64_t)kb * TR, col0 = (int64_t)kb2 * TR;
  if (p.exchange) {
    for (int t = tid; t < TR * NA; t += blockDim.x) {
      const int r = t / NA, a = t - r * NA;
      E l = {T(0), T(0)}, rr = {T(0), T(0)};
      if (row0 + r < p.N) {
        const cd x = in.exL[(row0 + r) * NA + a];
        l.x = (T)x.x;
        l.y = (T)x.y;
      }
      if (col0 + r < p.N) {
        const cd x = in.exR[(col0 + r) * NA + a];
        rr.x = (T)x.x;
        rr.y = (T)x.y;
      }
      sL[t] = l;
      sR[t] = rr;
    }
  }
  __syncthreads();
  if (active) {
    const E* C1 = sC;
    const E* C2 = sC + side_sz;
#define SCO(S, band, o, q) (S)[((band) * norb + (o)) * TK + (q)]
    // T_a(v', v) = sum_b V_ab rho2_b(v', v)
    E Tm[NA][NV][NV];
#pragma unroll
    for (int a = 0; a < NA; a++)
#pragma unroll
      for (int v2 = 0; v2 < NV; v2++)
#pragma unroll
        for (int v = 0; v < NV; v++) Tm[a][v2][v] = {T(0), T(0)};
#pragma unroll
    for (int b = 0; b < NA; b++) {
      E rho2[NV][NV];
#pragma unroll
      for (int v2 = 0; v2 < NV; v2++)
#pragma unroll
        for (int v = 0; v < NV; v++) rho2[v2][v] = {T(0), T(0)};
      for (int o = p.orb_off[b]; o < p.orb_off[b + 1]; o++) {
        E cv[NV], cv2[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) {
          cv[v] = SCO(C1, v, o, kk);
          cv2[v] = SCO(C2, v, o, kk2);
        }
#pragma unroll
        for (int v2 = 0; v2 < NV; v2++)
#pragma unroll
          for (int v = 0; v < NV; v++) cfmac(rho2[v2][v], cv2[v2], cv[v]);
      }
#pragma unroll
      for (int a = 0; a < NA; a++) {
        E V;
        if (kPrefetchV) {
          V = Vr[kPrefetchV ? a : 0][kPrefetchV ? b : 0];
        } else {
          const cd vab = Vt[a * NA + b];
          V = {(T)vab.x, (T)vab.y};
        }
#pragma unroll
        for (int v2 = 0; v2 < NV; v2++)
#pragma unroll
          for (int v = 0; v < NV; v++) cfma(Tm[a][v2][v], V, rho2[v2][v]);
      }
    }
#pragma unroll
    for (int c = 0; c < NC; c++) {
#pragma unroll
      for (int c2 = 0; c2 < NC; c2++) {
        E rho1[NA];
#pragma unroll
        for (int a = 0; a < NA; a++) {
          E acc = {T(0), T(0)};
          for (int o = p.orb_off[a]; o < p.orb_off[a + 1]; o++)
            cfmac(acc, SCO(C1, NV + c, o, kk), SCO(C2, NV + c2, o, kk2));
          rho1[a] = acc;
        }
#pragma unroll
        for (int v = 0; v < NV; v++) {
#pragma unroll
          for (int v2 = 0; v2 < NV; v2++) {
            const int pi = c * NV + v, pj = c2 * NV + v2;
            if (k == k2 && pj < pi) continue;
            E d = {T(0), T(0)};
#pragma unroll
            for (int a = 0; a < NA; a++) cfma(d, rho1[a], Tm[a][v2][v]);
            const int r = kk * NCV + pi, cc = kk2 * NCV + pj;
            if (p.exchange) {
#pragma unroll
              for (int a = 0; a < NA; a++) {
                const E l = sL[r * NA + a], rr = sR[cc * NA + a];
                d.x -= l.x * rr.x - l.y * rr.y;
                d.y -= l.x * rr.y + l.y * rr.x;
              }
            }
            E val;
            if (k == k2 && pi == pj) {
              const double ec = in.eigvalQ[(int64_t)k * p.nb + NV + c];
              const double ev = in.eigval[(int64_t)k * p.nb + v];
              if (MIXED) {
                val.x = -d.x;
                val.y = T(0);
                out.diag[row0 + r] = p.scissor + ec - ev;
              } else {
                // H_ii = z + conj(z), z = (scissor + Ec - Ev)/2 - (D - X)/2
                const double hr = (p.scissor + ec - ev) / 2. - (double)d.x / 2.;
                val.x = (T)(hr + hr);
                val.y = T(0);
              }
            } else {
              val.x = -d.x;
              val.y = -d.y;
            }
            sTile[r * LDT + cc] = val;
          }
        }
      }
    }
#undef SCO
  }
  __syncthreads();
  const int rows = (int)min((int64_t)TR, p.N - row0);
  const int cols = (int)min((int64_t)TR, p.N - col0);
  if (kb == kb2) {
    // lower triangle of a diagonal tile = conjugate of its upper triangle
    for (int t = tid; t < TR * TR; t += blockDim.x) {
      const int r = t / TR, c = t - r * TR;
      if (r > c && r < rows) {
        const E u = sTile[c * LDT + r];
        sTile[r * LDT + c] = E{u.x, -u.y};
      }
    }
    __syncthreads();
  }
  if (MIXED) {
    constexpr int VEC = 4;                  // complex elements per 16-byte store
    constexpr int CV = (TR + VEC - 1) / VEC;
    // direct block: rows row0 + r, columns col0 + c
    for (int t = tid; t < TR * CV; t += blockDim.x) {
      const int r = t / CV, c = (t - r * CV) * VEC;
      if (r >= rows || c >= cols) continue;
      const int64_t o = (row0 + r) * p.ldk + col0 + c;
      if (c + VEC <= cols && (o & 3) == 0) {
        __align__(16) __nv_bfloat162 h[VEC], l[VEC];
#pragma unroll
        for (int q = 0; q < VEC; q++) {
          const E v = sTile[r * LDT + c + q];
          const float re = (float)v.x, im = (float)v.y;
          const __nv_bfloat16 hr = __float2bfloat16_rn(re), hi_ = __float2bfloat16_rn(im);
          h[q].x = hr;
          h[q].y = hi_;
          l[q].x = __float2bfloat16_rn(re - __bfloat162float(hr));
          l[q].y = __float2bfloat16_rn(im - __bfloat162float(hi_));
        }
        *reinterpret_cast<uint4*>(out.Khi + o) = *reinterpret_cast<const uint4*>(h);
        *reinterpret_cast<uint4*>(out.Klo + o) = *reinterpret_cast<const uint4*>(l);
      } else {
        for (int q = 0; q < VEC && c + q < cols; q++) {
          const E v = sTile[r * LDT + c + q];
          split_store(out.Khi, out.Klo, o + q, (float)v.x, (float)v.y);
        }
      }
    }
    if (kb != kb2) {
      // mirror block: rows col0 + c, columns row0 + r, conjugate transpose
      constexpr int RV = (TR + VEC - 1) / VEC;
      for (int t = tid; t < TR * RV; t += blockDim.x) {
        const int c = t / RV, r = (t - c * RV) * VEC;
        if (c >= cols || r >= rows) continue;
        const int64_t o = (col0 + c) * p.ldk + row0 + r;
        if (r + VEC <= rows && (o & 3) == 0) {
          __align__(16) __nv_bfloat162 h[VEC], l[VEC];
#pragma unroll
          for (int q = 0; q < VEC; q++) {
            const E v = sTile[(r + q) * LDT + c];
            const float re = (float)v.x, im = -(float)v.y;
            const __nv_bfloat16 hr = __float2bfloat16_rn(re), hi_ = __float2bfloat16_rn(im);
            h[q].x = hr;
            h[q].y = hi_;
            l[q].x = __float2bfloat16_rn(re - __bfloat162float(hr));
            l[q].y = __float2bfloat16_rn(im - __bfloat162float(hi_));
          }
          *reinterpret_cast<uint4*>(out.Khi + o) = *reinterpret_cast<const uint4*>(h);
          *reinterpret_cast<uint4*>(out.Klo + o) = *reinterpret_cast<const uint4*>(l);
        } else {
          for (int q = 0; q < VEC && r + q < rows; q++) {
            const E v = sTile[(r + q) * LDT + c];
            split_store(out.Khi, out.Klo, o + q, (float)v.x, -(float)v.y);
          }
        }
      }
    }
  } else {
    for (int t = tid; t < TR * TR; t += blockDim.x) {
      const int r = t / TR, c = t - r * TR;
      if (r >= rows || c >= cols) continue;
      const E v = sTile[r * LDT + c];
      out.H[(row0 + r) * p.N + col0 + c] = mk((double)v.x, (double)v.y);
    }
    if (kb != kb2) {
      for (int t = tid; t < TR * TR; t += blockDim.x) {
        const int c = t / TR, r = t - c * TR;
        if (r >= rows || c >= cols) continue;
        const E v = sTile[r * LDT + c];
        out.H[(col0 + c) * p.N + row0 + r] = mk((double)v.x, -(double)v.y);
      }
    }
  }
}

template <typename T, int NV, int NC, int NA, bool MIXED>
__global__ void __launch_bounds__(ASM_TK * ASM_TK)
bse_assemble_tile_kernel(AsmParams p, AsmInputs in, AsmOutputs out, int nblk) {
  assemble_tile<T, NV, NC, NA, MIXED, ASM_TK>(p, in, out, nblk, blockIdx.x);
}

// Persistent batched assembly (mixed precision) over the tiles of many systems
// of one band-window class: each CTA takes (system, tile) items from a device
// work list through an atomic counter until the list is exhausted; the
// system's parameters are copied to shared memory once per item.
template <int NV, int NC, int NA, int TK>
__global__ void __launch_bounds__(TK * TK)
bse_assemble_batch_kernel(const AsmBatchMember* __restrict__ members, const int2* __restrict__ work, int nwork,
                          int* __restrict__ counter) {
  __shared__ AsmBatchMember sm;
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= nwork) break;
    const int2 w = work[it];
    {
      const int* src = reinterpret_cast<const int*>(members + w.x);
      int* dst = reinterpret_cast<int*>(&sm);
      for (int q = threadIdx.x; q < (int)(sizeof(AsmBatchMember) / sizeof(int)); q += blockDim.x) dst[q] = src[q];
    }
    __syncthreads();
    assemble_tile<float, NV, NC, NA, true, TK>(sm.p, sm.in, sm.out, sm.nblk, w.y);
    __syncthreads();
  }
}

size_t xatu_assembly_batch_smem(int nv, int nc, int na, int tk, int norb, int exchange) {
  const int tr = tk * nv * nc;
  return (2 * (size_t)(nv + nc) * norb * tk + (size_t)tr * (tr + 1) + (exchange ? 2 * (size_t)tr * na : 0)) *
         sizeof(cplx<float>);
}

template <int NV, int NC, int NA, int TK>
static cudaError_t launch_batch_t(const AsmBatchMember* members, const int2* work, int nwork, int* counter,
                                  size_t smem, int num_sms, bool set_attr, cudaStream_t s) {
  auto kern = bse_assemble_batch_kernel<NV, NC, NA, TK>;
  if (set_attr) {
    cudaError_t e = xatu_raise_smem_limit((const void*)kern, smem);
    if (e != cudaSuccess) return e;
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TK * TK, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int grid = std::max(1, std::min(nwork, per_sm * num_sms));
  kern<<<grid, TK * TK, smem, s>>>(members, work, nwork, counter);
  return cudaGetLastError();
}

template <int NV, int NC, int NA>
static cudaError_t launch_batch_tk(int tk, const AsmBatchMember* members, const int2* work, int nwork, int* counter,
                                   size_t smem, int num_sms, bool set_attr, cudaStream_t s) {
  if (tk == 8) return launch_batch_t<NV, NC, NA, 8>(members, work, nwork, counter, smem, num_sms, set_attr, s);
  if (tk == 16) return launch_batch_t<NV, NC, NA, 16>(members, work, nwork, counter, smem, num_sms, set_attr, s);
  return cudaErrorInvalidValue;
}

template <int NV, int NC>
static cudaError_t launch_batch_na(int na, int tk, const AsmBatchMember* members, const int2* work, int nwork,
                                   int* counter, size_t smem, int num_sms, bool set_attr, cudaStream_t s) {
  if (na == 2) return launch_batch_tk<NV, NC, 2>(tk, members, work, nwork, counter, smem, num_sms, set_attr, s);
  if (na == 3) return launch_batch_tk<NV, NC, 3>(tk, members, work, nwork, counter, smem, num_sms, set_attr, s);
  return cudaErrorInvalidValue;
}

bool xatu_assembly_batch_supported(int nv, int nc, int na) {
  return nv >= 1 && nv <= 3 && nc >= 1 && nc <= 3 && (na == 2 || na == 3);
}

cudaError_t xatu_launch_assembly_batch(int nv, int nc, int na, int tk, const AsmBatchMember* members,
                                       const int2* work, int nwork, int* counter, size_t smem, int num_sms,
                                       bool set_attr, cudaStream_t s) {
#define XATU_BCASE(NVv, NCv) \
  if (nv == NVv && nc == NCv) return launch_batch_na<NVv, NCv>(na, tk, members, work, nwork, counter, smem, num_sms, set_attr, s);
  XATU_BCASE(1, 1)
  XATU_BCASE(1, 2)
  XATU_BCASE(1, 3)
  XATU_BCASE(2, 1)
  XATU_BCASE(2, 2)
  XATU_BCASE(2, 3)
  XATU_BCASE(3, 1)
  XATU_BCASE(3, 2)
  XATU_BCASE(3, 3)
#undef XATU_BCASE
  return cudaErrorInvalidValue;
}

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
template <typename T, int NV, int NC, int NA, bool MIXED>
static cudaError_t launch_tile(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out, cudaStream_t s) {
  const int nblk = (p.nk + ASM_TK - 1) / ASM_TK;
  const int ntiles = nblk * (nblk + 1) / 2;
  constexpr int TR = ASM_TK * NV * NC;
  const size_t smem = (2 * (size_t)(NV + NC) * p.norb * ASM_TK + (size_t)TR * (TR + 1) +
                       (p.exchange ? 2 * (size_t)TR * NA : 0)) *
                      sizeof(cplx<T>);
  auto kern = bse_assemble_tile_kernel<T, NV, NC, NA, MIXED>;
  cudaError_t e = xatu_raise_smem_limit((const void*)kern, smem);
  if (e != cudaSuccess) return e;
  kern<<<ntiles, ASM_TK * ASM_TK, smem, s>>>(p, in, out, nblk);
  return cudaGetLastError();
}

template <typename T, bool MIXED>
static cudaError_t dispatch_tile(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out, cudaStream_t s,
                                 bool& launched) {
  launched = true;
#define XATU_CASE(NVv, NCv)                                                 \
  if (p.nv == NVv && p.nc == NCv) {                                         \
    if (p.na == 1) return launch_tile<T, NVv, NCv, 1, MIXED>(p, in, out, s); \
    if (p.na == 2) return launch_tile<T, NVv, NCv, 2, MIXED>(p, in, out, s); \
    if (p.na == 3) return launch_tile<T, NVv, NCv, 3, MIXED>(p, in, out, s); \
    if (p.na == 4) return launch_tile<T, NVv, NCv, 4, MIXED>(p, in, out, s); \
  }
  XATU_CASE(1, 1)
  XATU_CASE(1, 2)
  XATU_CASE(2, 1)
  XATU_CASE(2, 2)
#undef XATU_CASE
  launched = false;
  return cudaSuccess;
}

template <typename T, bool MIXED>
static cudaError_t launch_generic(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out, cudaStream_t s) {
  dim3 block(128);
  dim3 grid((unsigned)((p.N + 127) / 128), (unsigned)(p.N < 65535 ? p.N : 65535));
  bse_assemble_generic_kernel<T, MIXED><<<grid, block, 0, s>>>(p, in, out);
  return cudaGetLastError();
}

// Returns the kernel name used (for instrumentation) through *path: 0 pair, 1 generic.
cudaError_t xatu_launch_assembly(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out, bool mixed,
                                 bool force_generic, cudaStream_t s, int* path) {
  const int tr = ASM_TK * p.nv * p.nc;
  const size_t smem_f64 = (2 * (size_t)(p.nv + p.nc) * p.norb * ASM_TK + (size_t)tr * (tr + 1) + 2 * (size_t)tr * 4) *
                          sizeof(cd);
  const bool pair_ok = !force_generic && in.basis == nullptr && smem_f64 <= 200 * 1024;
  cudaError_t e = cudaSuccess;
  bool launched = false;
  if (pair_ok) {
    e = mixed ? dispatch_tile<float, true>(p, in, out, s, launched)
              : dispatch_tile<double, false>(p, in, out, s, launched);
    if (e != cudaSuccess) return e;
  }
  if (launched) { *path = 0; return cudaSuccess; }
  *path = 1;
  return mixed ? launch_generic<float, true>(p, in, out, s) : launch_generic<double, false>(p, in, out, s);
}
