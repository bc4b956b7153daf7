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
// written as the conjugate transpose, so H is exactly Hermitian.  The mixed
// build stores only the upper block triangle of K (blocks of XATU_KBLOCK, see
// xatu_kstored): there the mirror block is written only where it reaches that
// triangle, next to the diagonal.
//
// Precision: T = double writes the complex128 matrix (parity mode).  T = float
// writes the mixed-precision form used by the tensor-core solver: the band
// energies scissor + E_c - E_v as an FP64 diagonal, and the interaction
// kernel K = H - diag in two BF16 planes, K ~= K_hi + K_lo.
#pragma once
#include "params.h"

__device__ __forceinline__ void split_store(__nv_bfloat162* hi, __nv_bfloat162* lo, int64_t idx, float re, float im) {
  const __nv_bfloat16 hr = __float2bfloat16_rn(re), hi_ = __float2bfloat16_rn(im);
  const __nv_bfloat16 lr = __float2bfloat16_rn(re - __bfloat162float(hr));
  const __nv_bfloat16 li = __float2bfloat16_rn(im - __bfloat162float(hi_));
  __nv_bfloat162 h; h.x = hr; h.y = hi_;
  __nv_bfloat162 l; l.x = lr; l.y = li;
  hi[idx] = h;
  lo[idx] = l;
}

// Split-BF16 pair of one complex value packed as two 32-bit words: (hi.re, hi.im) and (lo.re, lo.im).  The split
// commutes with negation (hi and lo of -x are -hi and -lo), so the conjugate of a packed value is the same words
// with the sign bits of the imaginary halves flipped (bit 31 of each word).
__device__ __forceinline__ uint2 split_pack(float re, float im) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(re, im);   // one paired conversion, re in the low half
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(re - hf.x, im - hf.y);
  return make_uint2(*reinterpret_cast<const unsigned*>(&h), *reinterpret_cast<const unsigned*>(&l));
}

__device__ __forceinline__ uint2 split_conj(uint2 u) { return make_uint2(u.x ^ 0x80000000u, u.y ^ 0x80000000u); }

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
// Row r of the enumeration starts at S(r) = r nblk - r (r - 1) / 2: r from the quadratic formula, then an
// exact correction.
__device__ __forceinline__ void tile_of(int t, int nblk, int& kb, int& kb2) {
  const double b = 2.0 * nblk + 1.0;
  int r = (int)floor(0.5 * (b - sqrt(fmax(b * b - 8.0 * t, 0.0))));
  r = max(0, min(r, nblk - 1));
  auto S = [nblk](int q) { return q * nblk - q * (q - 1) / 2; };
  while (r > 0 && S(r) > t) r--;
  while (r + 1 < nblk && S(r + 1) <= t) r++;
  kb = r;
  kb2 = r + (t - S(r));
}

// Fast-path kernel.  CTA = a TK x TK tile of (k, k') pairs (TK = 16), one thread
// per pair.
//   phase 1: band coefficients of both k blocks (read as contiguous per-k rows,
//            stored transposed with padded rows) and the exchange factors of the
//            tile's rows and columns are staged in shared memory;
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
  // staging tile: with TR a multiple of 16 the columns are XOR-swizzled by (row / 4) mod 16, so that the
  // column-wise reads of the mirror block are free of bank conflicts; otherwise rows are padded by one
  constexpr bool SWZ = (TR % 16) == 0;
  constexpr int LDT = SWZ ? TR : TR + 1;   // row pitch
#define TIDX(r, c) ((r) * LDT + (SWZ ? ((c) ^ (((r) >> 2) & 15)) : (c)))
  using E = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int kb, kb2;
  tile_of(tile, nblk, kb, kb2);
  const int norb = p.norb;
  constexpr int TKP = TK + 1;      // padded coefficient row (bank-conflict-free transposed stores)
  const int side_sz = NB * norb * TKP;
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
  // coefficients: the TK k rows [band][orbital] of a side are one contiguous block in global memory
  // (valence part from the k stack, conduction part from the k+Q stack, same layout), so consecutive
  // threads read consecutive elements; each thread issues its loads in batches of 8 before storing them,
  // transposed, to [side][band][orbital][kq] with padded rows
  {
    const int nbo = NB * norb;
    const int per_side = TK * nbo;
    const int total = 2 * per_side;
    constexpr int BATCH = 8;
    for (int t0 = tid; t0 < total; t0 += BATCH * blockDim.x) {
      cd cv[BATCH];
#pragma unroll
      for (int q = 0; q < BATCH; q++) {
        const int t = t0 + q * blockDim.x;
        cv[q] = mk(0, 0);
        if (t < total) {
          const int side = t >= per_side ? 1 : 0;
          const int r = t - side * per_side;
          const int kq = r / nbo, e = r - kq * nbo;
          const int k = (side ? kb2 : kb) * TK + kq;
          if (k < p.nk) cv[q] = (e < NV * norb ? in.eigvec : in.eigvecQ)[(int64_t)k * p.nb * norb + e];
        }
      }
#pragma unroll
      for (int q = 0; q < BATCH; q++) {
        const int t = t0 + q * blockDim.x;
        if (t < total) {
          const int side = t >= per_side ? 1 : 0;
          const int r = t - side * per_side;
          const int kq = r / nbo, e = r - kq * nbo;
          sC[side * side_sz + e * TKP + kq] = E{(T)cv[q].x, (T)cv[q].y};
        }
      }
    }
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
#define SCO(S, band, o, q) (S)[((band) * norb + (o)) * TKP + (q)]
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
    // rho1_a(c, c') = sum_{o in a} conj(CQ_k[c]_o) CQ_k'[c']_o, each coefficient loaded once
    E rho1a[NA][NC][NC];
#pragma unroll
    for (int a = 0; a < NA; a++) {
#pragma unroll
      for (int c = 0; c < NC; c++)
#pragma unroll
        for (int c2 = 0; c2 < NC; c2++) rho1a[a][c][c2] = {T(0), T(0)};
      for (int o = p.orb_off[a]; o < p.orb_off[a + 1]; o++) {
        E cq[NC], cq2[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) {
          cq[c] = SCO(C1, NV + c, o, kk);
          cq2[c] = SCO(C2, NV + c, o, kk2);
        }
#pragma unroll
        for (int c = 0; c < NC; c++)
#pragma unroll
          for (int c2 = 0; c2 < NC; c2++) cfmac(rho1a[a][c][c2], cq[c], cq2[c2]);
      }
    }
#pragma unroll
    for (int c = 0; c < NC; c++) {
#pragma unroll
      for (int c2 = 0; c2 < NC; c2++) {
        E rho1[NA];
#pragma unroll
        for (int a = 0; a < NA; a++) rho1[a] = rho1a[a][c][c2];
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
            if constexpr (MIXED)
              reinterpret_cast<uint2*>(sTile)[TIDX(r, cc)] = split_pack((float)val.x, (float)val.y);
            else
              sTile[TIDX(r, cc)] = val;
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
        if constexpr (MIXED) {
          uint2* sT2 = reinterpret_cast<uint2*>(sTile);
          sT2[TIDX(r, c)] = split_conj(sT2[TIDX(c, r)]);
        } else {
          const E u = sTile[TIDX(c, r)];
          sTile[TIDX(r, c)] = E{u.x, -u.y};
        }
      }
    }
    __syncthreads();
  }
  if constexpr (MIXED) {
    // the tile holds the packed split-BF16 words: the planes are written without further conversion
    const uint2* sT2 = reinterpret_cast<const uint2*>(sTile);
    unsigned* Kh = reinterpret_cast<unsigned*>(out.Khi);
    unsigned* Kl = reinterpret_cast<unsigned*>(out.Klo);
    constexpr int VEC = 4;                  // complex elements per 16-byte store
    constexpr int CV = (TR + VEC - 1) / VEC;
    // direct block: rows row0 + r, columns col0 + c
    for (int t = tid; t < TR * CV; t += blockDim.x) {
      const int r = t / CV, c = (t - r * CV) * VEC;
      if (r >= rows || c >= cols) continue;
      const int64_t o = (row0 + r) * p.ldk + col0 + c;
      if (c + VEC <= cols && (o & 3) == 0) {
        uint2 u[VEC];
#pragma unroll
        for (int q = 0; q < VEC; q++) u[q] = sT2[TIDX(r, c + q)];
        *reinterpret_cast<uint4*>(Kh + o) = make_uint4(u[0].x, u[1].x, u[2].x, u[3].x);
        *reinterpret_cast<uint4*>(Kl + o) = make_uint4(u[0].y, u[1].y, u[2].y, u[3].y);
      } else {
        for (int q = 0; q < VEC && c + q < cols; q++) {
          const uint2 u = sT2[TIDX(r, c + q)];
          Kh[o + q] = u.x;
          Kl[o + q] = u.y;
        }
      }
    }
    // mirror block (rows col0 + c, columns row0 + r, conjugate transpose): only where it reaches the stored
    // upper block triangle of the kernel planes (xatu_kstored), i.e. near the diagonal
    if (kb != kb2 && (row0 + rows - 1) / XATU_KBLOCK >= col0 / XATU_KBLOCK) {
      constexpr int RV = (TR + VEC - 1) / VEC;
      for (int t = tid; t < TR * RV; t += blockDim.x) {
        const int c = t / RV, r = (t - c * RV) * VEC;
        if (c >= cols || r >= rows) continue;
        const int64_t o = (col0 + c) * p.ldk + row0 + r;
        if (r + VEC <= rows && (o & 3) == 0) {
          uint2 u[VEC];
#pragma unroll
          for (int q = 0; q < VEC; q++) u[q] = split_conj(sT2[TIDX(r + q, c)]);
          *reinterpret_cast<uint4*>(Kh + o) = make_uint4(u[0].x, u[1].x, u[2].x, u[3].x);
          *reinterpret_cast<uint4*>(Kl + o) = make_uint4(u[0].y, u[1].y, u[2].y, u[3].y);
        } else {
          for (int q = 0; q < VEC && r + q < rows; q++) {
            const uint2 u = split_conj(sT2[TIDX(r + q, c)]);
            Kh[o + q] = u.x;
            Kl[o + q] = u.y;
          }
        }
      }
    }
  } else {
    for (int t = tid; t < TR * TR; t += blockDim.x) {
      const int r = t / TR, c = t - r * TR;
      if (r >= rows || c >= cols) continue;
      const E v = sTile[TIDX(r, c)];
      out.H[(row0 + r) * p.N + col0 + c] = mk((double)v.x, (double)v.y);
    }
    if (kb != kb2) {
      for (int t = tid; t < TR * TR; t += blockDim.x) {
        const int c = t / TR, r = t - c * TR;
        if (r >= rows || c >= cols) continue;
        const E v = sTile[TIDX(r, c)];
        out.H[(col0 + c) * p.N + row0 + r] = mk((double)v.x, -(double)v.y);
      }
    }
  }
#undef TIDX
}

