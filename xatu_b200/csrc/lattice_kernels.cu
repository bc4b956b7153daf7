// Interaction tables of the BSE kernel.
//
//  * pair_potential_kernel   V(|R + tau_a - tau_b|) for every atom pair a <= b and
//                            cell R: the Struve/Bessel evaluation, hoisted out of
//                            the q loop (the reference re-evaluates it for every q,
//                            ExcitonTB.cpp:438-454 inside the loop at :765-779).
//  * motif_ft_kernel         V_ab(q) = (1/T) sum_R V(|R + tau_a - tau_b|) e^{i q.R}
//                            for every q of the BZ mesh, lower triangle by
//                            conjugation (motifFTMatrix, ExcitonTB.cpp:462-476).
//                            One CTA per (q, chunk of pairs); the phase e^{iq.R}
//                            is computed once per cell and reused by every pair;
//                            warp-shuffle + shared-memory reduction.
//                            motif_ft_roots_kernel: the same sum when the mesh
//                            and the cells are commensurate (a Monkhorst-Pack
//                            mesh and lattice cells), the phase a table lookup.
//  * recip_table_kernel      W_ab(q) = sum_G Vt(q + G) e^{i (q+G).(tau_a - tau_b)}
//                            over the table of k - k' differences of a grid of k
//                            points.  It carries the reciprocal-space interaction
//                            (reciprocalInteractionTerm + blochCoherenceFactor,
//                            ExcitonTB.cpp:562-621) with the per-element G sum
//                            factored out: D = rho1^T W(k - k') rho2.
//  * exchange_vectors_kernel per e-h state i: L_a(i) and R_a(i) = sum_b VX_ab rho2x_b(i)
//                            so that the exchange term is X_ij = sum_a L_a(i) R_a(j)
//                            (realSpaceInteractionTerm with (c_k, v'_k', v_k, c'_k'),
//                            ExcitonTB.cpp:897, and its reciprocal form :905).
#include "kernels.h"

#define MOTIF_PAIR_CHUNK 8
#define MOTIF_THREADS 256

// deriv = 0: V itself; deriv = 1: dV/dr0 (zero for the Coulomb potential).
extern "C" __global__ void pair_potential_kernel(PotParams p, int kind, int deriv, int na,
                                                 const double* __restrict__ motif, int ncells,
                                                 const double* __restrict__ cells, int npairs,
                                                 const int2* __restrict__ pairs, double* __restrict__ vtab) {
  const int64_t total = (int64_t)npairs * ncells;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int pr = (int)(t / ncells);
    const int n = (int)(t - (int64_t)pr * ncells);
    const int2 ab = pairs[pr];
    const double* ta = motif + 4 * ab.x;
    const double* tb = motif + 4 * ab.y;
    const double* c = cells + 3 * n;
    const double d0 = c[0] + ta[0] - tb[0];
    const double d1 = c[1] + ta[1] - tb[1];
    const double d2 = c[2] + ta[2] - tb[2];
    const double r = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    if (deriv)
      vtab[t] = (kind == 1) ? 0.0 : keldysh_potential_dr0(p, r);
    else
      vtab[t] = (kind == 1) ? coulomb_potential(p, r) : keldysh_potential(p, r);
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// grid: (nq, ceil(npairs / MOTIF_PAIR_CHUNK)); block MOTIF_THREADS.
extern "C" __global__ void __launch_bounds__(MOTIF_THREADS)
motif_ft_kernel(int nq, const double* __restrict__ q, int ncells, const double* __restrict__ cells, int npairs,
                const int2* __restrict__ pairs, const double* __restrict__ vtab, double inv_total, int na,
                cd* __restrict__ out) {
  const int iq = blockIdx.x;
  const int p0 = blockIdx.y * MOTIF_PAIR_CHUNK;
  const int np = min(MOTIF_PAIR_CHUNK, npairs - p0);
  const double qx = q[3 * iq], qy = q[3 * iq + 1], qz = q[3 * iq + 2];
  double accr[MOTIF_PAIR_CHUNK], acci[MOTIF_PAIR_CHUNK];
#pragma unroll
  for (int j = 0; j < MOTIF_PAIR_CHUNK; j++) { accr[j] = 0.0; acci[j] = 0.0; }
  for (int n = threadIdx.x; n < ncells; n += blockDim.x) {
    const double cx = cells[3 * n], cy = cells[3 * n + 1], cz = cells[3 * n + 2];
    double s, c;
    sincos(qx * cx + qy * cy + qz * cz, &s, &c);
#pragma unroll
    for (int j = 0; j < MOTIF_PAIR_CHUNK; j++) {
      if (j < np) {
        const double v = vtab[(int64_t)(p0 + j) * ncells + n];
        accr[j] = fma(v, c, accr[j]);
        acci[j] = fma(v, s, acci[j]);
      }
    }
  }
  __shared__ double red[2][MOTIF_PAIR_CHUNK][MOTIF_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < MOTIF_PAIR_CHUNK; j++) {
    const double r = warp_sum(accr[j]);
    const double i = warp_sum(acci[j]);
    if (lane == 0) { red[0][j][warp] = r; red[1][j][warp] = i; }
  }
  __syncthreads();
  if (threadIdx.x < np) {
    const int j = threadIdx.x;
    double r = 0.0, i = 0.0;
    for (int w = 0; w < MOTIF_THREADS / 32; w++) { r += red[0][j][w]; i += red[1][j][w]; }
    r *= inv_total;
    i *= inv_total;
    const int2 ab = pairs[p0 + j];
    cd* o = out + (int64_t)iq * na * na;
    o[ab.x * na + ab.y] = mk(r, i);
    o[ab.y * na + ab.x] = mk(r, -i);
  }
}

// motif_ft_kernel for a mesh and cells that are commensurate: q = sum_d (m_d / den) b_d and R = sum_d n_d a_d
// with integers m, n, so that e^{i q.R} = e^{2 pi i (m.n mod den) / den} comes from a table of the den roots of
// unity (sincospi of exact fractions) instead of one sincos per (q, cell).  One CTA per MOTIF_QB mesh points
// (MOTIF_THREADS / MOTIF_QB threads each) and chunk of pairs: the potentials of a chunk of cells are staged in shared memory once and
// used by all of the CTA's points.  mi: nq x 3, ni: ncells x 3, every n_d reduced to [0, den).
// Dynamic shared memory: motif_roots_smem(den).
#define MOTIF_QB XATU_MOTIF_QB
extern "C" __global__ void __launch_bounds__(MOTIF_THREADS)
motif_ft_roots_kernel(int nq, const int* __restrict__ mi, int den, int ncells, const int* __restrict__ ni, int npairs,
                      const int2* __restrict__ pairs, const double* __restrict__ vtab, double inv_total, int na,
                      cd* __restrict__ out) {
  constexpr int TPQ = MOTIF_THREADS / MOTIF_QB;
  extern __shared__ double2 roots[];                                                    // den
  double* vst = reinterpret_cast<double*>(roots + den);                                 // [pair][cell of chunk]
  int* nst = reinterpret_cast<int*>(vst + MOTIF_PAIR_CHUNK * MOTIF_THREADS);             // [cell of chunk][3]
  const int ql = threadIdx.x / TPQ, sub = threadIdx.x - ql * TPQ;
  const int iq = blockIdx.x * MOTIF_QB + ql;
  const bool qv = iq < nq;
  const int p0 = blockIdx.y * MOTIF_PAIR_CHUNK;
  const int np = min(MOTIF_PAIR_CHUNK, npairs - p0);
  for (int t = threadIdx.x; t < den; t += blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)t / (double)den, &s, &c);
    roots[t] = make_double2(c, s);
  }
  int m0 = qv ? mi[3 * iq] % den : 0, m1 = qv ? mi[3 * iq + 1] % den : 0, m2 = qv ? mi[3 * iq + 2] % den : 0;
  m0 += m0 < 0 ? den : 0;
  m1 += m1 < 0 ? den : 0;
  m2 += m2 < 0 ? den : 0;
  double accr[MOTIF_PAIR_CHUNK], acci[MOTIF_PAIR_CHUNK];
#pragma unroll
  for (int j = 0; j < MOTIF_PAIR_CHUNK; j++) { accr[j] = 0.0; acci[j] = 0.0; }
  for (int c0 = 0; c0 < ncells; c0 += MOTIF_THREADS) {
    const int nc = min(MOTIF_THREADS, ncells - c0);
    __syncthreads();   // the previous chunk is consumed (and the table is written)
    if (threadIdx.x < nc) {
      for (int j = 0; j < np; j++) vst[j * MOTIF_THREADS + threadIdx.x] = vtab[(int64_t)(p0 + j) * ncells + c0 + threadIdx.x];
      nst[3 * threadIdx.x] = ni[3 * (c0 + threadIdx.x)];
      nst[3 * threadIdx.x + 1] = ni[3 * (c0 + threadIdx.x) + 1];
      nst[3 * threadIdx.x + 2] = ni[3 * (c0 + threadIdx.x) + 2];
    }
    __syncthreads();
    for (int t = sub; t < nc; t += TPQ) {
      const int e = (m0 * nst[3 * t] + m1 * nst[3 * t + 1] + m2 * nst[3 * t + 2]) % den;
      const double2 ph = roots[e];
#pragma unroll
      for (int j = 0; j < MOTIF_PAIR_CHUNK; j++) {
        if (j < np) {
          const double v = vst[j * MOTIF_THREADS + t];
          accr[j] = fma(v, ph.x, accr[j]);
          acci[j] = fma(v, ph.y, acci[j]);
        }
      }
    }
  }
  // sum over the TPQ threads of each point (a fixed shuffle tree inside the half warp)
#pragma unroll
  for (int j = 0; j < MOTIF_PAIR_CHUNK; j++)
#pragma unroll
    for (int o = TPQ / 2; o > 0; o >>= 1) {
      accr[j] += __shfl_xor_sync(0xffffffffu, accr[j], o);
      acci[j] += __shfl_xor_sync(0xffffffffu, acci[j], o);
    }
  if (sub == 0 && qv) {
    cd* o = out + (int64_t)iq * na * na;
#pragma unroll
    for (int j = 0; j < MOTIF_PAIR_CHUNK; j++) {
      if (j < np) {
        const int2 ab = pairs[p0 + j];
        const double r = accr[j] * inv_total, i = acci[j] * inv_total;
        o[ab.x * na + ab.y] = mk(r, i);
        o[ab.y * na + ab.x] = mk(r, -i);
      }
    }
  }
}

extern "C" size_t motif_roots_smem(int den) {
  return (size_t)den * sizeof(double2) + (size_t)MOTIF_PAIR_CHUNK * MOTIF_THREADS * sizeof(double) +
         (size_t)3 * MOTIF_THREADS * sizeof(int);
}

// deriv = 0: W itself; deriv = 1: dW/dr0.
extern "C" __global__ void recip_table_kernel(PotParams p, RecipTable t, int deriv, int nentries,
                                              const double* __restrict__ G, int na, const double* __restrict__ motif,
                                              cd* __restrict__ W) {
  const int64_t total = (int64_t)nentries * na;
  for (int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id < total;
       id += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(id / na);
    const int a = (int)(id - (int64_t)e * na);
    double qx = t.q0[0], qy = t.q0[1], qz = t.q0[2];
    int rem = e;
    for (int d = 0; d < t.ndim; d++) {
      const int off = rem % t.len[d] - t.span[d];
      rem /= t.len[d];
      const double f = (double)off / t.n_eff;
      qx += f * t.b[3 * d];
      qy += f * t.b[3 * d + 1];
      qz += f * t.b[3 * d + 2];
    }
    cd acc[XATU_MAX_ATOMS];
    for (int b = 0; b < na; b++) acc[b] = mk(0, 0);
    const double tax = motif[4 * a], tay = motif[4 * a + 1], taz = motif[4 * a + 2];
    for (int g = 0; g < t.nG; g++) {
      const double gx = qx + G[3 * g], gy = qy + G[3 * g + 1], gz = qz + G[3 * g + 2];
      const double v = deriv ? keldysh_ft_dr0(p, gx, gy, gz) : keldysh_ft(p, gx, gy, gz);
      if (v == 0.0) continue;
      for (int b = 0; b < na; b++) {
        const double ph = gx * (tax - motif[4 * b]) + gy * (tay - motif[4 * b + 1]) + gz * (taz - motif[4 * b + 2]);
        double s, c;
        sincos(ph, &s, &c);
        acc[b].x = fma(v, c, acc[b].x);
        acc[b].y = fma(v, s, acc[b].y);
      }
    }
    cd* o = W + (int64_t)e * na * na + a * na;
    for (int b = 0; b < na; b++) o[b] = acc[b];
  }
}

// Exchange factors.  State i = (k, c, v) with stack columns (v, nv + c).
//   L_a(i)   = sum_{o in a} conj(CQ_k[c]_o) C_k[v]_o
//   rho_b(i) = sum_{o in b} conj(C_k[v]_o)  CQ_k[c]_o
//   R_a(i)   = sum_b VX_ab rho_b(i)
extern "C" __global__ void exchange_vectors_kernel(int N, int nv, int nc, int nb, int norb, int na,
                                                   const int* __restrict__ orb_off, const cd* __restrict__ eigvec,
                                                   const cd* __restrict__ eigvecQ, const cd* __restrict__ VX,
                                                   const int* __restrict__ basis, cd* __restrict__ L,
                                                   cd* __restrict__ R) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int k, c, v;
  if (basis) {
    k = basis[3 * i];
    v = basis[3 * i + 1];
    c = basis[3 * i + 2];
  } else {
    const int ncv = nc * nv;
    k = i / ncv;
    c = (i - k * ncv) / nv;
    v = i - k * ncv - c * nv;
  }
  const cd* cv = eigvec + ((int64_t)k * nb + v) * norb;
  const cd* cc = eigvecQ + ((int64_t)k * nb + nv + c) * norb;
  cd rho[XATU_MAX_ATOMS];
  for (int a = 0; a < na; a++) {
    cd l = mk(0, 0), r = mk(0, 0);
    for (int o = orb_off[a]; o < orb_off[a + 1]; o++) {
      l = l + cmulc(cc[o], cv[o]);
      r = r + cmulc(cv[o], cc[o]);
    }
    L[(int64_t)i * na + a] = l;
    rho[a] = r;
  }
  for (int a = 0; a < na; a++) {
    cd s = mk(0, 0);
    for (int b = 0; b < na; b++) s = s + VX[a * na + b] * rho[b];
    R[(int64_t)i * na + a] = s;
  }
}
