// Adjoint (Hellmann-Feynman) gradients of exciton energies.
//
// The reference has no derivative code; this is the derivative of the path it
// computes (band solve -> fixGlobalPhase -> BShamiltonian, ExcitonTB.cpp:673-683,
// 707-921, SystemTB.cpp:60-156) for a normalised eigenvector x of the BSE
// matrix H:  dE/dtheta = x^H (dH/dtheta) x.
//
// With i = (k, c, v), j = (k', c', v') and the factors of the assembly
//   P_a(c, c')  = sum_{o in a} conj(CQ_k[c]_o) CQ_k'[c']_o
//   R_b(v', v)  = sum_{o in b} conj(C_k'[v']_o) C_k[v]_o
//   D_ij = sum_ab P_a V_ab(k, k') R_b,    X_ij = sum_ab L_a(i) VX_ab conj(L_b(j))
// the energy is (D and X are Hermitian in (i, j), so the full double sum equals
// the reference's upper-triangle construction)
//   E = sum_i |x_i|^2 (s + E_c - E_v) - sum_ij conj(x_i) x_j D_ij + sum_ij conj(x_i) x_j X_ij.
//
// adj_pair_kernel (one CTA per k, the partners k' in chunks of ADJ_THREADS) forms
//   * the band-coefficient adjoint  cbar = dE/d conj(C)  of row k:
//       conduction c:  -sum_{k', c'} wc[c][a(o)][c'] CQ_k'[c']_o,
//                      wc[c][a][c'] = sum_v conj(x_kcv) sum_v' x_k'c'v' sum_b V_ab R_b(v', v)
//       valence v (from the conjugate form of the same sum):
//                      -sum_{k', v'} wv[v][b(o)][v'] C_k'[v']_o,
//                      wv[v][b][v'] = conj(sum_c conj(x_kcv) sum_a V_ab sum_c' P_a(c, c') x_k'c'v')
//   * the band-energy adjoint  dE/dE_c = sum_v |x_kcv|^2,  dE/dE_v = -sum_c |x_kcv|^2
//   * the interaction sums  sum Gamma_ab V_ab  and  sum Gamma_ab dV_ab/dr0
//     (Gamma_ab(k, k') = sum conj(x_i) x_j P_a R_b), from which the potential
//     parameters follow:  dE/dr0 = -sum Gamma dV/dr0 + (exchange),
//     dE/deps_m = dE/deps_s = sum Gamma V / (2 eps_bar) - E_X / (2 eps_bar)
//     (the Keldysh potential and its Fourier transform scale as 1 / eps_bar).
// The exchange part is rank one: alpha_a = sum_i conj(x_i) L_a(i),
// E_X = alpha^T VX conj(alpha).
//
// adj_band_kernel (one CTA per k) recomputes the band eigensystem and pulls
// cbar / ebar back to the Bloch Hamiltonian:
//   fixGlobalPhase: C = zeta u, zeta = conj(s)/|s|, s = sum_o u_o
//     ubar = conj(zeta) cbar + i beta s / |s|^2,   beta = Im(cbar^H C)
//   Hermitian eigenproblem (first-order perturbation theory):
//     Gamma(k) = A + A^H,  A = sum_b u_b [ ebar_b / 2 u_b^H + sum_{m != b} (ubar_b^H u_m) / (l_b - l_m) u_m^H ]
//   Loewdin: Gamma_h = f X Gamma X (f = 27.2 for Hartree models).
// adj_hop_kernel sums Gamma over k:  G(R) = sum_k Gamma(k) e^{-i k.R}, so that
// for a perturbation of the hopping matrices that keeps H(k) Hermitian
//   dE = Re sum_{R,a,b} conj(G(R)_ab) dH(R)_ab
// (triangular storage: G doubled off the diagonal, as H(k) = h' + h'^H).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bands.cuh"
#include "engine.h"
#include "kernels.h"

#define ADJ_THREADS 128
#define ADJ_WS (ADJ_THREADS + 1)   // row pitch of the per-partner weight buffer (padded against bank conflicts)
#define ADJ_BAND_THREADS 128

struct AdjParams {
  int nk, nv, nc, nb, norb, na, ns;
  int64_t N;
  int mode;
  EquivMap emap;
  int rt_ndim;
  int rt_len[3];
  int rt_span[3];
  int64_t nentries;
  int orb_off[XATU_MAX_ATOMS + 1];
};

struct AdjInputs {
  const double* kpoints;
  const int* kgrid;
  const cd* eigvec;    // nk x nb x norb, bands at k
  const cd* eigvecQ;   // bands at k + Q
  const cd* table;     // interaction table V
  const cd* dtable;    // dV/dr0
  const cd* x;         // N x ns, column-major
  const cd* exu;       // ns x na: (VX conj(alpha))_a, or NULL without exchange
  const cd* exw;       // ns x na: (VX^T alpha)_b
  int* status;
};

struct AdjOutputs {
  cd* cbar;            // ns x nk x nb x norb
  double* ebar;        // ns x nk x nb
  double* epart;       // nk x ns x 2: sum Re(Gamma V), sum Re(Gamma dV)
};

__device__ __forceinline__ double adj_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// cbar, ebar and the interaction sums of row k.  Dynamic shared memory: see adj_pair_smem.
template <int NV, int NC, int NA>
__global__ void __launch_bounds__(ADJ_THREADS) adj_pair_kernel(AdjParams p, AdjInputs in, AdjOutputs out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NB = NV + NC;
  constexpr int WC = NC * NA * NC;   // wc elements per partner (wv: NV * NA * NV follow)
  const int norb = p.norb, ns = p.ns, k = blockIdx.x, tid = threadIdx.x;
  cd* Ck = reinterpret_cast<cd*>(smem_raw);    // NB x norb (valence rows from the k stack, conduction from k + Q)
  cd* xa = Ck + NB * norb;                     // ns x NC*NV
  cd* acc = xa + ns * NC * NV;                 // ns x NB x norb
  cd* w = acc + ns * NB * norb;                // WN x ADJ_WS (element-major, padded rows)
  __shared__ double eacc[8][2];
  __shared__ int atom_of[XATU_MAX_ORB];

  for (int t = tid; t < NB * norb; t += ADJ_THREADS) {
    const int b = t / norb;
    Ck[t] = (b < NV ? in.eigvec : in.eigvecQ)[(int64_t)k * p.nb * norb + t];
  }
  for (int t = tid; t < ns * NC * NV; t += ADJ_THREADS) {
    const int s = t / (NC * NV), e = t - s * (NC * NV);
    xa[t] = in.x[(int64_t)s * p.N + (int64_t)k * (NC * NV) + e];
  }
  for (int t = tid; t < ns * NB * norb; t += ADJ_THREADS) acc[t] = mk(0, 0);
  if (tid < 16) eacc[tid >> 1][tid & 1] = 0.0;
  for (int o = tid; o < norb; o += ADJ_THREADS) {
    int a = 0;
    while (a + 1 < NA && o >= p.orb_off[a + 1]) a++;
    atom_of[o] = a;
  }
  __syncthreads();

  for (int base = 0; base < p.nk; base += ADJ_THREADS) {
    const int k2 = base + tid;
    const int nq = min(ADJ_THREADS, p.nk - base);
    const bool valid = k2 < p.nk;
    cd P[NA][NC][NC], R[NA][NV][NV];
    const cd* Vt = nullptr;
    const cd* dVt = nullptr;
    if (valid) {
      const cd* c2 = in.eigvec + (int64_t)k2 * p.nb * norb;
      const cd* c2q = in.eigvecQ + (int64_t)k2 * p.nb * norb;
#pragma unroll
      for (int a = 0; a < NA; a++) {
#pragma unroll
        for (int c = 0; c < NC; c++)
#pragma unroll
          for (int c2i = 0; c2i < NC; c2i++) P[a][c][c2i] = mk(0, 0);
#pragma unroll
        for (int v = 0; v < NV; v++)
#pragma unroll
          for (int v2 = 0; v2 < NV; v2++) R[a][v][v2] = mk(0, 0);
        for (int o = p.orb_off[a]; o < p.orb_off[a + 1]; o++) {
          cd cq[NC], vv[NV];
#pragma unroll
          for (int c2i = 0; c2i < NC; c2i++) cq[c2i] = c2q[(NV + c2i) * norb + o];
#pragma unroll
          for (int v2 = 0; v2 < NV; v2++) vv[v2] = c2[v2 * norb + o];
#pragma unroll
          for (int c = 0; c < NC; c++) {
            const cd ck = Ck[(NV + c) * norb + o];
#pragma unroll
            for (int c2i = 0; c2i < NC; c2i++) P[a][c][c2i] = P[a][c][c2i] + cmulc(ck, cq[c2i]);
          }
#pragma unroll
          for (int v = 0; v < NV; v++) {
            const cd vk = Ck[v * norb + o];
#pragma unroll
            for (int v2 = 0; v2 < NV; v2++) R[a][v2][v] = R[a][v2][v] + cmulc(vv[v2], vk);
          }
        }
      }
      int64_t e = interaction_entry(p, in.kpoints, in.kgrid, k, k2);
      if (e < 0) {
        atomicOr(in.status, XATU_DEVERR_INDEX);
        e = 0;
      }
      Vt = in.table + e * NA * NA;
      dVt = in.dtable + e * NA * NA;
    }
    for (int s = 0; s < ns; s++) {
      double eV = 0.0, eR = 0.0;
      if (valid) {
        const cd* xs = xa + s * (NC * NV);
        cd* wt = w + tid;   // element e of this partner at wt[e * ADJ_WS]
        cd xb[NC][NV];
#pragma unroll
        for (int c2i = 0; c2i < NC; c2i++)
#pragma unroll
          for (int v2 = 0; v2 < NV; v2++)
            xb[c2i][v2] = in.x[(int64_t)s * p.N + (int64_t)k2 * (NC * NV) + c2i * NV + v2];
        // valence side: Px_a(c, v') = sum_c' P_a(c, c') x_k'c'v';  wv[v][b][v'] = conj(sum_c conj(x_kcv) sum_a V_ab Px_a(c, v'))
        {
          cd Px[NA][NC][NV];
#pragma unroll
          for (int a = 0; a < NA; a++)
#pragma unroll
            for (int c = 0; c < NC; c++)
#pragma unroll
              for (int v2 = 0; v2 < NV; v2++) {
                cd t = mk(0, 0);
#pragma unroll
                for (int c2i = 0; c2i < NC; c2i++) t = t + P[a][c][c2i] * xb[c2i][v2];
                Px[a][c][v2] = t;
              }
#pragma unroll
          for (int b = 0; b < NA; b++) {
            cd PV[NC][NV];
#pragma unroll
            for (int c = 0; c < NC; c++)
#pragma unroll
              for (int v2 = 0; v2 < NV; v2++) {
                cd t = mk(0, 0);
#pragma unroll
                for (int a = 0; a < NA; a++) t = t + Vt[a * NA + b] * Px[a][c][v2];
                PV[c][v2] = t;
              }
#pragma unroll
            for (int v = 0; v < NV; v++)
#pragma unroll
              for (int v2 = 0; v2 < NV; v2++) {
                cd t = mk(0, 0);
#pragma unroll
                for (int c = 0; c < NC; c++) t = t + cmulc(xs[c * NV + v], PV[c][v2]);
                wt[(WC + (v * NA + b) * NV + v2) * ADJ_WS] = mk(-t.x, t.y);   // -conj(t)
              }
          }
        }
        // conduction side: Rx_b(c', v) = sum_v' x_k'c'v' R_b(v', v);  B_a = sum_b V_ab Rx_b
        {
          cd Rx[NA][NC][NV];
#pragma unroll
          for (int b = 0; b < NA; b++)
#pragma unroll
            for (int c2i = 0; c2i < NC; c2i++)
#pragma unroll
              for (int v = 0; v < NV; v++) {
                cd t = mk(0, 0);
#pragma unroll
                for (int v2 = 0; v2 < NV; v2++) t = t + xb[c2i][v2] * R[b][v2][v];
                Rx[b][c2i][v] = t;
              }
#pragma unroll
          for (int a = 0; a < NA; a++) {
            cd B[NC][NV], dB[NC][NV];
#pragma unroll
            for (int c2i = 0; c2i < NC; c2i++)
#pragma unroll
              for (int v = 0; v < NV; v++) {
                cd t = mk(0, 0), u = mk(0, 0);
#pragma unroll
                for (int b = 0; b < NA; b++) {
                  t = t + Vt[a * NA + b] * Rx[b][c2i][v];
                  u = u + dVt[a * NA + b] * Rx[b][c2i][v];
                }
                B[c2i][v] = t;
                dB[c2i][v] = u;
              }
#pragma unroll
            for (int c = 0; c < NC; c++) {
#pragma unroll
              for (int c2i = 0; c2i < NC; c2i++) {
                cd t = mk(0, 0), u = mk(0, 0);
#pragma unroll
                for (int v = 0; v < NV; v++) {
                  t = t + cmulc(xs[c * NV + v], B[c2i][v]);
                  u = u + cmulc(xs[c * NV + v], dB[c2i][v]);
                }
                wt[((c * NA + a) * NC + c2i) * ADJ_WS] = mk(-t.x, -t.y);
                // Gamma-weighted sums: sum_c' P_a(c, c') (.)
                const cd pt = P[a][c][c2i] * t, pu = P[a][c][c2i] * u;
                eV += pt.x;
                eR += pu.x;
              }
            }
          }
        }
      }
      eV = adj_warp_sum(eV);
      eR = adj_warp_sum(eR);
      if ((tid & 31) == 0) {
        atomicAdd(&eacc[s][0], eV);
        atomicAdd(&eacc[s][1], eR);
      }
      __syncthreads();
      // cbar_k += sum over the chunk's partners
      for (int t = tid; t < NB * norb; t += ADJ_THREADS) {
        const int b = t / norb, o = t - b * norb, a = atom_of[o];
        cd sum = mk(0, 0);
        if (b >= NV) {
          const int c = b - NV;
          for (int q = 0; q < nq; q++) {
            const cd* ww = w + (c * NA + a) * NC * ADJ_WS + q;
            const cd* cq = in.eigvecQ + ((int64_t)(base + q) * p.nb + NV) * norb + o;
#pragma unroll
            for (int c2i = 0; c2i < NC; c2i++) sum = sum + ww[c2i * ADJ_WS] * cq[c2i * norb];
          }
        } else {
          for (int q = 0; q < nq; q++) {
            const cd* ww = w + (WC + (b * NA + a) * NV) * ADJ_WS + q;
            const cd* cv = in.eigvec + (int64_t)(base + q) * p.nb * norb + o;
#pragma unroll
            for (int v2 = 0; v2 < NV; v2++) sum = sum + ww[v2 * ADJ_WS] * cv[v2 * norb];
          }
        }
        acc[(s * NB + b) * norb + o] = acc[(s * NB + b) * norb + o] + sum;
      }
      __syncthreads();
    }
  }

  // exchange terms (rank one) and the outputs of row k
  for (int t = tid; t < ns * NB * norb; t += ADJ_THREADS) {
    const int s = t / (NB * norb), r = t - s * (NB * norb);
    const int b = r / norb, o = r - b * norb, a = atom_of[o];
    cd v = acc[t];
    if (in.exu) {
      const cd* xs = xa + s * (NC * NV);
      if (b >= NV) {
        // + sum_v conj(x_kcv) C_k[v]_o u_a
        const int c = b - NV;
        cd t2 = mk(0, 0);
#pragma unroll
        for (int vv = 0; vv < NV; vv++) t2 = t2 + cmulc(xs[c * NV + vv], Ck[vv * norb + o]);
        v = v + t2 * in.exu[s * p.na + a];
      } else {
        // + sum_c x_kcv CQ_k[c]_o w_b
        cd t2 = mk(0, 0);
#pragma unroll
        for (int c = 0; c < NC; c++) t2 = t2 + xs[c * NV + b] * Ck[(NV + c) * norb + o];
        v = v + t2 * in.exw[s * p.na + a];
      }
    }
    out.cbar[(((int64_t)s * p.nk + k) * NB + b) * norb + o] = v;
  }
  for (int t = tid; t < ns * NB; t += ADJ_THREADS) {
    const int s = t / NB, b = t - s * NB;
    const cd* xs = xa + s * (NC * NV);
    double e = 0.0;
    if (b >= NV) {
      for (int vv = 0; vv < NV; vv++) e += nrm2(xs[(b - NV) * NV + vv]);
    } else {
      for (int c = 0; c < NC; c++) e -= nrm2(xs[c * NV + b]);
    }
    out.ebar[((int64_t)s * p.nk + k) * NB + b] = e;
  }
  if (tid < ns) {
    out.epart[((int64_t)k * ns + tid) * 2] = eacc[tid][0];
    out.epart[((int64_t)k * ns + tid) * 2 + 1] = eacc[tid][1];
  }
}

static size_t adj_pair_smem(int nv, int nc, int na, int norb, int ns) {
  const int nb = nv + nc;
  const int wn = nc * na * nc + nv * na * nv;
  return ((size_t)nb * norb + (size_t)ns * nc * nv + (size_t)ns * nb * norb + (size_t)ADJ_WS * wn) * sizeof(cd);
}

// alpha_a = sum_i conj(x_i) L_a(i); grid (ns, na).
extern "C" __global__ void adj_alpha_kernel(int64_t N, int na, const cd* __restrict__ x, const cd* __restrict__ L,
                                            cd* __restrict__ alpha) {
  const int s = blockIdx.x, a = blockIdx.y;
  double sr = 0.0, si = 0.0;
  for (int64_t i = threadIdx.x; i < N; i += blockDim.x) {
    const cd t = cmulc(x[(int64_t)s * N + i], L[i * na + a]);
    sr += t.x;
    si += t.y;
  }
  __shared__ double red[2][32];
  sr = adj_warp_sum(sr);
  si = adj_warp_sum(si);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = sr;
    red[1][threadIdx.x >> 5] = si;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a0 = 0.0, a1 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      a0 += red[0][w];
      a1 += red[1][w];
    }
    alpha[s * na + a] = mk(a0, a1);
  }
}

// Gamma(k) of the band-list rows [row0, row1) of one stack (shift bp.shift).
extern "C" __global__ void __launch_bounds__(ADJ_BAND_THREADS)
adj_band_kernel(BandParams bp, int ns, int row0, int row1, const double* __restrict__ kpoints,
                const double* __restrict__ cellsR, const cd* __restrict__ HR, const cd* __restrict__ SR,
                const cd* __restrict__ cbar, const double* __restrict__ ebar, cd* __restrict__ gk,
                int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_band[];
  __shared__ int s_flag;
  const int n = bp.norb, nsel = row1 - row0, k = blockIdx.x, tid = threadIdx.x;
  const int nt = ADJ_BAND_THREADS;
  const BandSmem s = band_smem_layout(smem_band, n, bp.nR, bp.has_overlap);
  const int lda = s.lda;
  double* lam = reinterpret_cast<double*>(smem_band + ((band_smem_bytes(n, bp.nR, bp.has_overlap) + 15) & ~(size_t)15));
  cd* ub = reinterpret_cast<cd*>(lam + n + (n & 1));   // nsel x n
  cd* Mc = ub + nsel * n;                               // nsel x n
  cd* Z = Mc + nsel * n;                                // nsel x n
  cd* XU = Z + nsel * n;                                // n x nsel
  cd* ssum = XU + n * nsel;                             // nsel
  double* beta = reinterpret_cast<double*>(ssum + nsel);  // nsel
  int* cols = reinterpret_cast<int*>(beta + nsel);         // nsel
  BlockGroup g;
  const cd* M = band_eigensystem(g, bp, k, kpoints, cellsR, HR, SR, s, status, &s_flag);
  if (!M) return;
  for (int i = tid; i < n; i += nt) lam[i] = M[i * lda + i].x;
  for (int b = tid; b < nsel; b += nt) cols[b] = s.perm[bp.band_list[row0 + b]];
  g.sync();
  // column sums (fixGlobalPhase) and XU = X U_sel
  const int warp = tid >> 5, lane = tid & 31;
  for (int b = warp; b < nsel; b += nt / 32) {
    double sr = 0.0, si = 0.0;
    for (int o = lane; o < n; o += 32) {
      sr += s.V[o * lda + cols[b]].x;
      si += s.V[o * lda + cols[b]].y;
    }
    sr = adj_warp_sum(sr);
    si = adj_warp_sum(si);
    if (lane == 0) {
      ssum[b] = mk(sr, si);
      if (!(sr * sr + si * si > 1e-200)) atomicOr(status, XATU_DEVERR_DEGEN);
    }
  }
  for (int t = tid; t < n * nsel; t += nt) {
    const int i = t / nsel, b = t - i * nsel;
    cd v;
    if (bp.has_overlap) {
      v = mk(0, 0);
      for (int m = 0; m < n; m++) v = v + s.A[i * lda + m] * s.V[m * lda + cols[b]];
    } else {
      v = s.V[i * lda + cols[b]];
    }
    XU[t] = v;
  }
  g.sync();
  const double f = (bp.has_overlap && bp.is_au) ? 27.2 : 1.0;
  for (int st = 0; st < ns; st++) {
    const cd* cb = cbar + ((int64_t)st * bp.nk + k) * bp.nb * n;
    const double* eb = ebar + ((int64_t)st * bp.nk + k) * bp.nb;
    // beta_b = Im(cbar^H C), C = zeta u
    for (int b = warp; b < nsel; b += nt / 32) {
      const cd sb = ssum[b];
      const double as = sqrt(nrm2(sb));
      const cd zeta = mk(sb.x / as, -sb.y / as);
      double bi = 0.0;
      for (int o = lane; o < n; o += 32) bi += cmulc(cb[(row0 + b) * n + o], zeta * s.V[o * lda + cols[b]]).y;
      bi = adj_warp_sum(bi);
      if (lane == 0) beta[b] = bi;
    }
    g.sync();
    // ubar = conj(zeta) cbar + i beta s / |s|^2
    for (int t = tid; t < nsel * n; t += nt) {
      const int b = t / n, o = t - b * n;
      const cd sb = ssum[b];
      const double s2 = nrm2(sb), as = sqrt(s2);
      const cd zc = mk(sb.x / as, sb.y / as);
      const cd ib = mk(-beta[b] * sb.y / s2, beta[b] * sb.x / s2);
      ub[t] = zc * cb[(row0 + b) * n + o] + ib;
    }
    g.sync();
    // Mc[b][m] = (ubar_b^H u_m) / (l_b - l_m),  Mc[b][col_b] = ebar_b / 2
    for (int t = tid; t < nsel * n; t += nt) {
      const int b = t / n, m = t - b * n;
      const int col = cols[b];
      cd v;
      if (m == col) {
        v = mk(0.5 * eb[row0 + b], 0.0);
      } else {
        const double d = lam[col] - lam[m];
        if (fabs(d) < 1e-10) {
          atomicOr(status, XATU_DEVERR_DEGEN);
          v = mk(0, 0);
        } else {
          cd t2 = mk(0, 0);
          for (int o = 0; o < n; o++) t2 = t2 + cmulc(ub[b * n + o], s.V[o * lda + m]);
          v = (1.0 / d) * t2;
        }
      }
      Mc[t] = v;
    }
    g.sync();
    // Z[b][j] = sum_m Mc[b][m] conj(u_m[j])
    for (int t = tid; t < nsel * n; t += nt) {
      const int b = t / n, j = t - b * n;
      cd v = mk(0, 0);
      for (int m = 0; m < n; m++) v = v + Mc[b * n + m] * conj(s.V[j * lda + m]);
      Z[t] = v;
    }
    g.sync();
    const cd* ZZ = Z;
    if (bp.has_overlap) {
      // Mc <- Z X
      for (int t = tid; t < nsel * n; t += nt) {
        const int b = t / n, j = t - b * n;
        cd v = mk(0, 0);
        for (int m = 0; m < n; m++) v = v + Z[b * n + m] * s.A[m * lda + j];
        Mc[t] = v;
      }
      g.sync();
      ZZ = Mc;
    }
    // Gamma_ij = f ((XU ZZ)_ij + conj((XU ZZ)_ji))
    cd* go = gk + ((int64_t)st * bp.nk + k) * n * n;
    for (int t = tid; t < n * n; t += nt) {
      const int i = t / n, j = t - i * n;
      cd a = mk(0, 0), h = mk(0, 0);
      for (int b = 0; b < nsel; b++) {
        a = a + XU[i * nsel + b] * ZZ[b * n + j];
        h = h + XU[j * nsel + b] * ZZ[b * n + i];
      }
      go[t] = f * (a + conj(h));
    }
    g.sync();
  }
}

static size_t adj_band_smem(int norb, int nR, int has_overlap, int nsel) {
  const int n = norb;
  return ((band_smem_bytes(n, nR, has_overlap) + 15) & ~(size_t)15) + (size_t)(n + (n & 1)) * sizeof(double) +
         (4 * (size_t)nsel * n + nsel) * sizeof(cd) + (size_t)nsel * sizeof(double) + (size_t)nsel * sizeof(int);
}

// G[s][R][a][b] = fac_ab (sum_k Gamma0[s][k] e^{-i k.R} + sum_k GammaQ[s][k] e^{-i (k+Q).R});
// grid (nR, ceil(norb^2 / 256), ns), block 256.
extern "C" __global__ void __launch_bounds__(256)
adj_hop_kernel(int nk, int norb, int triangular, const double* __restrict__ kpoints,
               const double* __restrict__ cellsR, const cd* __restrict__ g0, const cd* __restrict__ gQ, double qx,
               double qy, double qz, cd* __restrict__ G, int nR) {
  const int r = blockIdx.x, st = blockIdx.z;
  const int n2 = norb * norb;
  const int ab = blockIdx.y * blockDim.x + threadIdx.x;
  __shared__ cd ph[256], phq[256];
  const double Rx = cellsR[3 * r], Ry = cellsR[3 * r + 1], Rz = cellsR[3 * r + 2];
  double ar = 0.0, ai = 0.0;
  for (int base = 0; base < nk; base += 256) {
    const int kk = base + threadIdx.x;
    if (kk < nk) {
      const double kr = kpoints[3 * kk] * Rx + kpoints[3 * kk + 1] * Ry + kpoints[3 * kk + 2] * Rz;
      double sn, cs;
      sincos(kr, &sn, &cs);
      ph[threadIdx.x] = mk(cs, -sn);
      if (gQ) {
        sincos(kr + qx * Rx + qy * Ry + qz * Rz, &sn, &cs);
        phq[threadIdx.x] = mk(cs, -sn);
      }
    }
    __syncthreads();
    if (ab < n2) {
      const int m = min(256, nk - base);
      for (int q = 0; q < m; q++) {
        const cd gv = g0[((int64_t)st * nk + base + q) * n2 + ab];
        const cd t = gv * ph[q];
        ar += t.x;
        ai += t.y;
        if (gQ) {
          const cd u = gQ[((int64_t)st * nk + base + q) * n2 + ab] * phq[q];
          ar += u.x;
          ai += u.y;
        }
      }
    }
    __syncthreads();
  }
  if (ab < n2) {
    const int a = ab / norb, b = ab - a * norb;
    const double fac = (triangular && a != b) ? 2.0 : 1.0;
    G[((int64_t)st * nR + r) * n2 + ab] = mk(fac * ar, fac * ai);
  }
}

template <int NV, int NC, int NA>
static cudaError_t launch_pair(const AdjParams& p, const AdjInputs& in, const AdjOutputs& out, cudaStream_t st) {
  const size_t smem = adj_pair_smem(NV, NC, NA, p.norb, p.ns);
  cudaError_t e = xatu_raise_smem_limit((const void*)adj_pair_kernel<NV, NC, NA>, smem);
  if (e != cudaSuccess) return e;
  adj_pair_kernel<NV, NC, NA><<<p.nk, ADJ_THREADS, smem, st>>>(p, in, out);
  return cudaGetLastError();
}

template <int NV, int NC>
static cudaError_t launch_pair_na(const AdjParams& p, const AdjInputs& in, const AdjOutputs& out, cudaStream_t st) {
  switch (p.na) {
    case 1: return launch_pair<NV, NC, 1>(p, in, out, st);
    case 2: return launch_pair<NV, NC, 2>(p, in, out, st);
    case 3: return launch_pair<NV, NC, 3>(p, in, out, st);
    case 4: return launch_pair<NV, NC, 4>(p, in, out, st);
  }
  return cudaErrorInvalidValue;
}

static cudaError_t launch_pair_any(const AdjParams& p, const AdjInputs& in, const AdjOutputs& out, cudaStream_t st) {
  if (p.nv == 1 && p.nc == 1) return launch_pair_na<1, 1>(p, in, out, st);
  if (p.nv == 1 && p.nc == 2) return launch_pair_na<1, 2>(p, in, out, st);
  if (p.nv == 2 && p.nc == 1) return launch_pair_na<2, 1>(p, in, out, st);
  if (p.nv == 2 && p.nc == 2) return launch_pair_na<2, 2>(p, in, out, st);
  return cudaErrorInvalidValue;
}

__global__ void adj_scale_copy_kernel(const cd* __restrict__ in, cd* __restrict__ out, long long n, double f) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    out[t] = f * in[t];
}

// Derivative interaction tables into d_adjdtable / d_adjdVX (layouts of d_table / d_VX):
//   which = 0: d/dr0 (pair potentials or keldyshFT in derivative mode, then the same transforms);
//   which = 1: d/deps_m = d/deps_s = -V / (2 eps_bar) for the Keldysh potential and its Fourier
//              transform (scaled copies of the built tables), 0 for the Coulomb potential.
xatu_status xatu_derivative_tables(xatu_ctx* ctx, int which) {
  cudaStream_t st = ctx->stream;
  const int na = ctx->natoms;
  const int npairs = na * (na + 1) / 2;
  const int ncells = (int)(ctx->cells.size() / 3);
  const long long nentries = ctx->mode == XATU_MODE_REALSPACE ? (long long)ctx->nmesh : ctx->rt_entries;
  XATU_CK(ctx->d_adjdtable.ensure((size_t)nentries * na * na * sizeof(cd)));
  XATU_CK(ctx->d_adjdVX.ensure((size_t)na * na * sizeof(cd)));
  XATU_CK(cudaMemsetAsync(ctx->d_adjdVX.p, 0, (size_t)na * na * sizeof(cd), st));
  if (which == 1) {
    const double eps_bar = (ctx->eps_m + ctx->eps_s) / 2;
    const bool dkel = ctx->mode != XATU_MODE_REALSPACE || ctx->potential == XATU_POT_KELDYSH;
    const bool xkel = ctx->mode != XATU_MODE_REALSPACE || ctx->exchange_potential == XATU_POT_KELDYSH;
    const long long n = nentries * na * na;
    adj_scale_copy_kernel<<<(int)std::min<long long>((n + 255) / 256, 4096), 256, 0, st>>>(
        ctx->d_table.as<cd>(), ctx->d_adjdtable.as<cd>(), n, dkel ? -1.0 / (2 * eps_bar) : 0.0);
    ctx->launches++;
    XATU_CK_LAUNCH("adj_scale_copy_kernel");
    if (ctx->exchange) {
      adj_scale_copy_kernel<<<1, 256, 0, st>>>(ctx->d_VX.as<cd>(), ctx->d_adjdVX.as<cd>(), (long long)na * na,
                                               xkel ? -1.0 / (2 * eps_bar) : 0.0);
      ctx->launches++;
      XATU_CK_LAUNCH("adj_scale_copy_kernel");
    }
    return XATU_OK;
  }
  PotParams pp;
  pp.a1norm = ctx->a1;
  pp.b1norm = ctx->b1;
  pp.area = ctx->area;
  pp.eps_m = ctx->eps_m;
  pp.eps_s = ctx->eps_s;
  pp.r0 = ctx->r0;
  pp.regularization = ctx->regularization;
  pp.cutoff = ctx->cutoff;
  pp.total_cells = ctx->total_cells;
  if (ctx->mode == XATU_MODE_REALSPACE) {
    XATU_CK(ctx->d_adjdvtab.ensure((size_t)npairs * ncells * sizeof(double)));
    const long long tot = (long long)npairs * ncells;
    const int grid = (int)std::min<long long>((tot + 255) / 256, 148 * 16);
    pair_potential_kernel<<<grid, 256, 0, st>>>(pp, ctx->potential, 1, na, ctx->d_motif.as<double>(), ncells,
                                                ctx->d_cells.as<double>(), npairs, ctx->d_pairs.as<int2>(),
                                                ctx->d_adjdvtab.as<double>());
    ctx->launches++;
    XATU_CK_LAUNCH("pair_potential_kernel (d/dr0)");
    dim3 g2(ctx->nmesh, (npairs + 7) / 8);
    motif_ft_kernel<<<g2, 256, 0, st>>>(ctx->nmesh, ctx->d_mesh.as<double>(), ncells, ctx->d_cells.as<double>(), npairs,
                                        ctx->d_pairs.as<int2>(), ctx->d_adjdvtab.as<double>(), 1.0 / ctx->total_cells,
                                        na, ctx->d_adjdtable.as<cd>());
    ctx->launches++;
    XATU_CK_LAUNCH("motif_ft_kernel (d/dr0)");
    if (ctx->exchange) {
      pair_potential_kernel<<<grid, 256, 0, st>>>(pp, ctx->exchange_potential, 1, na, ctx->d_motif.as<double>(),
                                                  ncells, ctx->d_cells.as<double>(), npairs, ctx->d_pairs.as<int2>(),
                                                  ctx->d_adjdvtab.as<double>());
      ctx->launches++;
      XATU_CK_LAUNCH("pair_potential_kernel (exchange, d/dr0)");
      dim3 g3(1, (npairs + 7) / 8);
      motif_ft_kernel<<<g3, 256, 0, st>>>(1, ctx->d_Q.as<double>(), ncells, ctx->d_cells.as<double>(), npairs,
                                          ctx->d_pairs.as<int2>(), ctx->d_adjdvtab.as<double>(),
                                          1.0 / ctx->total_cells, na, ctx->d_adjdVX.as<cd>());
      ctx->launches++;
      XATU_CK_LAUNCH("motif_ft_kernel (exchange, d/dr0)");
    }
  } else {
    RecipTable t;
    memset(&t, 0, sizeof(t));
    t.ndim = ctx->ndim;
    t.n_eff = ctx->n_eff;
    for (int a = 0; a < 3; a++) {
      t.span[a] = ctx->rt_span[a];
      t.len[a] = ctx->rt_len[a];
    }
    for (int i = 0; i < 3 * ctx->ndim; i++) t.b[i] = ctx->recip[i];
    t.nG = (int)(ctx->G.size() / 3);
    const long long tot = nentries * na;
    const int grid = (int)std::min<long long>((tot + 127) / 128, 148 * 32);
    recip_table_kernel<<<grid, 128, 0, st>>>(pp, t, 1, (int)nentries, ctx->d_G.as<double>(), na,
                                             ctx->d_motif.as<double>(), ctx->d_adjdtable.as<cd>());
    ctx->launches++;
    XATU_CK_LAUNCH("recip_table_kernel (d/dr0)");
    if (ctx->exchange) {
      RecipTable tx = t;
      for (int a = 0; a < 3; a++) {
        tx.span[a] = 0;
        tx.len[a] = 1;
        tx.q0[a] = ctx->Q[a];
      }
      recip_table_kernel<<<1, 128, 0, st>>>(pp, tx, 1, 1, ctx->d_G.as<double>(), na, ctx->d_motif.as<double>(),
                                            ctx->d_adjdVX.as<cd>());
      ctx->launches++;
      XATU_CK_LAUNCH("recip_table_kernel (exchange, d/dr0)");
    }
  }
  return XATU_OK;
}

// cbar / ebar (ns x nk x nb x norb, ns x nk x nb) -> G(R) in d_adjG (ns x nR x norb x norb): the band
// eigensystems are recomputed and the adjoint pulled back through fixGlobalPhase and the eigenproblem.
xatu_status xatu_adjoint_bands_to_hoppings(xatu_ctx* ctx, int ns, const cd* cbar, const double* ebar) {
  cudaStream_t st = ctx->stream;
  const int nk = ctx->nk, norb = ctx->norb, nb = ctx->nb;
  BandParams bp;
  memset(&bp, 0, sizeof(bp));
  bp.nk = nk;
  bp.norb = norb;
  bp.nR = ctx->nR;
  bp.triangular = ctx->triangular;
  bp.nb = nb;
  for (int i = 0; i < nb; i++) bp.band_list[i] = ctx->band_list[i];
  bp.max_sweeps = 40;
  bp.has_overlap = ctx->has_overlap ? 1 : 0;
  bp.is_au = ctx->is_au ? 1 : 0;
  const size_t n2 = (size_t)norb * norb;
  XATU_CK(ctx->d_adjGk.ensure((ctx->qnonzero ? 2 : 1) * (size_t)ns * nk * n2 * sizeof(cd)));
  const cd* SR = ctx->has_overlap ? ctx->d_SR.as<cd>() : nullptr;
  cd* g0 = ctx->d_adjGk.as<cd>();
  cd* gQ = ctx->qnonzero ? g0 + (size_t)ns * nk * n2 : nullptr;
  const int r1 = ctx->qnonzero ? ctx->nv : nb;
  const size_t smem = adj_band_smem(norb, ctx->nR, bp.has_overlap, r1);
  const size_t smemQ = ctx->qnonzero ? adj_band_smem(norb, ctx->nR, bp.has_overlap, nb - ctx->nv) : 0;
  if (std::max(smem, smemQ) > 227 * 1024)
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "adjoint band kernel: orbital basis too large for shared memory");
  XATU_CK(xatu_raise_smem_limit((const void*)adj_band_kernel, std::max(smem, smemQ)));
  adj_band_kernel<<<nk, ADJ_BAND_THREADS, smem, st>>>(bp, ns, 0, r1, ctx->d_kpoints.as<double>(),
                                                      ctx->d_cellsR.as<double>(), ctx->d_HR.as<cd>(), SR, cbar, ebar, g0,
                                                      ctx->d_status.as<int>());
  ctx->launches++;
  XATU_CK_LAUNCH("adj_band_kernel");
  if (ctx->qnonzero) {
    for (int i = 0; i < 3; i++) bp.shift[i] = ctx->Q[i];
    adj_band_kernel<<<nk, ADJ_BAND_THREADS, smemQ, st>>>(bp, ns, ctx->nv, nb, ctx->d_kpoints.as<double>(),
                                                        ctx->d_cellsR.as<double>(), ctx->d_HR.as<cd>(), SR, cbar,
                                                        ebar, gQ, ctx->d_status.as<int>());
    ctx->launches++;
    XATU_CK_LAUNCH("adj_band_kernel (k+Q)");
  }
  XATU_CK(ctx->d_adjG.ensure((size_t)ns * ctx->nR * n2 * sizeof(cd)));
  dim3 gh(ctx->nR, (unsigned)((n2 + 255) / 256), ns);
  adj_hop_kernel<<<gh, 256, 0, st>>>(nk, norb, ctx->triangular ? 1 : 0, ctx->d_kpoints.as<double>(),
                                     ctx->d_cellsR.as<double>(), g0, gQ, ctx->Q[0], ctx->Q[1], ctx->Q[2],
                                     ctx->d_adjG.as<cd>(), ctx->nR);
  ctx->launches++;
  XATU_CK_LAUNCH("adj_hop_kernel");
  return XATU_OK;
}

// ------------------------------------------------------------------ weight-matrix form
// The same back-propagation for a general Hermitian weight matrix Y (row-major N x N): the derivative of
// sum_ij Y_ij H_ij, i.e. of sum_t 2 Re(a_t^H H b_t) when Y = sum_t (conj(a_t) b_t^T + conj(b_t) a_t^T).
// Exchange factors: Zc = Y conj(L), Zv = Y^T L (N x na, column-major) with the exchange vectors L.
struct AdjWeightInputs {
  const cd* Y;        // row-major N x N
  const cd* Zc;       // N x na, or NULL without exchange
  const cd* Zv;
  const cd* VX;       // na x na
};

template <int NV, int NC, int NA>
__global__ void __launch_bounds__(ADJ_THREADS) adj_pair_weight_kernel(AdjParams p, AdjInputs in, AdjWeightInputs wi,
                                                                       cd* __restrict__ cbar, double* __restrict__ ebar) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NB = NV + NC, NCV = NC * NV;
  constexpr int WC = NC * NA * NC;
  const int norb = p.norb, k = blockIdx.x, tid = threadIdx.x;
  cd* Ck = reinterpret_cast<cd*>(smem_raw);    // NB x norb
  cd* acc = Ck + NB * norb;                    // NB x norb
  cd* w = acc + NB * norb;                     // (WC + NV NA NV) x ADJ_WS
  __shared__ int atom_of[XATU_MAX_ORB];
  for (int t = tid; t < NB * norb; t += ADJ_THREADS) {
    const int b = t / norb;
    Ck[t] = (b < NV ? in.eigvec : in.eigvecQ)[(int64_t)k * p.nb * norb + t];
    acc[t] = mk(0, 0);
  }
  for (int o = tid; o < norb; o += ADJ_THREADS) {
    int a = 0;
    while (a + 1 < NA && o >= p.orb_off[a + 1]) a++;
    atom_of[o] = a;
  }
  __syncthreads();
  for (int base = 0; base < p.nk; base += ADJ_THREADS) {
    const int k2 = base + tid;
    const int nq = min(ADJ_THREADS, p.nk - base);
    if (k2 < p.nk) {
      cd P[NA][NC][NC], R[NA][NV][NV];
      const cd* c2 = in.eigvec + (int64_t)k2 * p.nb * norb;
      const cd* c2q = in.eigvecQ + (int64_t)k2 * p.nb * norb;
#pragma unroll
      for (int a = 0; a < NA; a++) {
#pragma unroll
        for (int c = 0; c < NC; c++)
#pragma unroll
          for (int c2i = 0; c2i < NC; c2i++) P[a][c][c2i] = mk(0, 0);
#pragma unroll
        for (int v = 0; v < NV; v++)
#pragma unroll
          for (int v2 = 0; v2 < NV; v2++) R[a][v][v2] = mk(0, 0);
        for (int o = p.orb_off[a]; o < p.orb_off[a + 1]; o++) {
          cd cq[NC], vv[NV];
#pragma unroll
          for (int c2i = 0; c2i < NC; c2i++) cq[c2i] = c2q[(NV + c2i) * norb + o];
#pragma unroll
          for (int v2 = 0; v2 < NV; v2++) vv[v2] = c2[v2 * norb + o];
#pragma unroll
          for (int c = 0; c < NC; c++) {
            const cd ck = Ck[(NV + c) * norb + o];
#pragma unroll
            for (int c2i = 0; c2i < NC; c2i++) P[a][c][c2i] = P[a][c][c2i] + cmulc(ck, cq[c2i]);
          }
#pragma unroll
          for (int v = 0; v < NV; v++) {
            const cd vk = Ck[v * norb + o];
#pragma unroll
            for (int v2 = 0; v2 < NV; v2++) R[a][v2][v] = R[a][v2][v] + cmulc(vv[v2], vk);
          }
        }
      }
      int64_t e = interaction_entry(p, in.kpoints, in.kgrid, k, k2);
      if (e < 0) {
        atomicOr(in.status, XATU_DEVERR_INDEX);
        e = 0;
      }
      const cd* Vt = in.table + e * NA * NA;
      cd Yb[NCV][NCV];
#pragma unroll
      for (int r = 0; r < NCV; r++)
#pragma unroll
        for (int c = 0; c < NCV; c++) Yb[r][c] = wi.Y[((int64_t)k * NCV + r) * p.N + (int64_t)k2 * NCV + c];
      cd* wt = w + tid;
      // wc[c][a][c'] = -sum_{v,v'} Y[cv][c'v'] sum_b V_ab R_b(v', v)
#pragma unroll
      for (int a = 0; a < NA; a++) {
        cd VR[NV][NV];
#pragma unroll
        for (int v2 = 0; v2 < NV; v2++)
#pragma unroll
          for (int v = 0; v < NV; v++) {
            cd t = mk(0, 0);
#pragma unroll
            for (int b = 0; b < NA; b++) t = t + Vt[a * NA + b] * R[b][v2][v];
            VR[v2][v] = t;
          }
#pragma unroll
        for (int c = 0; c < NC; c++)
#pragma unroll
          for (int c2i = 0; c2i < NC; c2i++) {
            cd t = mk(0, 0);
#pragma unroll
            for (int v = 0; v < NV; v++)
#pragma unroll
              for (int v2 = 0; v2 < NV; v2++) t = t + Yb[c * NV + v][c2i * NV + v2] * VR[v2][v];
            wt[((c * NA + a) * NC + c2i) * ADJ_WS] = mk(-t.x, -t.y);
          }
      }
      // wv[v][b][v'] = -sum_{c,c'} conj(Y[cv][c'v']) conj(sum_a P_a(c, c') V_ab)
#pragma unroll
      for (int b = 0; b < NA; b++) {
        cd PV[NC][NC];
#pragma unroll
        for (int c = 0; c < NC; c++)
#pragma unroll
          for (int c2i = 0; c2i < NC; c2i++) {
            cd t = mk(0, 0);
#pragma unroll
            for (int a = 0; a < NA; a++) t = t + P[a][c][c2i] * Vt[a * NA + b];
            PV[c][c2i] = t;
          }
#pragma unroll
        for (int v = 0; v < NV; v++)
#pragma unroll
          for (int v2 = 0; v2 < NV; v2++) {
            cd t = mk(0, 0);
#pragma unroll
            for (int c = 0; c < NC; c++)
#pragma unroll
              for (int c2i = 0; c2i < NC; c2i++) t = t + Yb[c * NV + v][c2i * NV + v2] * PV[c][c2i];
            wt[(WC + (v * NA + b) * NV + v2) * ADJ_WS] = mk(-t.x, t.y);   // -conj(t)
          }
      }
    }
    __syncthreads();
    for (int t = tid; t < NB * norb; t += ADJ_THREADS) {
      const int b = t / norb, o = t - b * norb, a = atom_of[o];
      cd sum = mk(0, 0);
      if (b >= NV) {
        const int c = b - NV;
        for (int q = 0; q < nq; q++) {
          const cd* ww = w + (c * NA + a) * NC * ADJ_WS + q;
          const cd* cq = in.eigvecQ + ((int64_t)(base + q) * p.nb + NV) * norb + o;
#pragma unroll
          for (int c2i = 0; c2i < NC; c2i++) sum = sum + ww[c2i * ADJ_WS] * cq[c2i * norb];
        }
      } else {
        for (int q = 0; q < nq; q++) {
          const cd* ww = w + (WC + (b * NA + a) * NV) * ADJ_WS + q;
          const cd* cv = in.eigvec + (int64_t)(base + q) * p.nb * norb + o;
#pragma unroll
          for (int v2 = 0; v2 < NV; v2++) sum = sum + ww[v2 * ADJ_WS] * cv[v2 * norb];
        }
      }
      acc[t] = acc[t] + sum;
    }
    __syncthreads();
  }
  // exchange (per state i of row k: u(i) = VX Zc(i), w(i) = VX^T Zv(i)) and outputs
  for (int t = tid; t < NB * norb; t += ADJ_THREADS) {
    const int b = t / norb, o = t - b * norb, a = atom_of[o];
    cd v = acc[t];
    if (wi.Zc) {
      if (b >= NV) {
        const int c = b - NV;
        for (int vv = 0; vv < NV; vv++) {
          const int64_t i = (int64_t)k * NCV + c * NV + vv;
          cd u = mk(0, 0);
          for (int b2 = 0; b2 < NA; b2++) u = u + wi.VX[a * NA + b2] * wi.Zc[(int64_t)b2 * p.N + i];
          v = v + Ck[vv * norb + o] * u;
        }
      } else {
        for (int c = 0; c < NC; c++) {
          const int64_t i = (int64_t)k * NCV + c * NV + b;
          cd u = mk(0, 0);
          for (int a2 = 0; a2 < NA; a2++) u = u + wi.VX[a2 * NA + a] * wi.Zv[(int64_t)a2 * p.N + i];
          v = v + Ck[(NV + c) * norb + o] * u;
        }
      }
    }
    cbar[((int64_t)k * NB + b) * norb + o] = v;
  }
  for (int b = tid; b < NB; b += ADJ_THREADS) {
    double e = 0.0;
    if (b >= NV) {
      for (int vv = 0; vv < NV; vv++) {
        const int64_t i = (int64_t)k * NCV + (b - NV) * NV + vv;
        e += wi.Y[i * p.N + i].x;
      }
    } else {
      for (int c = 0; c < NC; c++) {
        const int64_t i = (int64_t)k * NCV + c * NV + b;
        e -= wi.Y[i * p.N + i].x;
      }
    }
    ebar[(int64_t)k * NB + b] = e;
  }
}

template <int NV, int NC, int NA>
static cudaError_t launch_weight(const AdjParams& p, const AdjInputs& in, const AdjWeightInputs& wi, cd* cbar,
                                 double* ebar, cudaStream_t st) {
  const int nb = NV + NC;
  const int wn = NC * NA * NC + NV * NA * NV;
  const size_t smem = ((size_t)2 * nb * p.norb + (size_t)ADJ_WS * wn) * sizeof(cd);
  cudaError_t e = xatu_raise_smem_limit((const void*)adj_pair_weight_kernel<NV, NC, NA>, smem);
  if (e != cudaSuccess) return e;
  adj_pair_weight_kernel<NV, NC, NA><<<p.nk, ADJ_THREADS, smem, st>>>(p, in, wi, cbar, ebar);
  return cudaGetLastError();
}

template <int NV, int NC>
static cudaError_t launch_weight_na(const AdjParams& p, const AdjInputs& in, const AdjWeightInputs& wi, cd* cbar,
                                    double* ebar, cudaStream_t st) {
  switch (p.na) {
    case 1: return launch_weight<NV, NC, 1>(p, in, wi, cbar, ebar, st);
    case 2: return launch_weight<NV, NC, 2>(p, in, wi, cbar, ebar, st);
    case 3: return launch_weight<NV, NC, 3>(p, in, wi, cbar, ebar, st);
    case 4: return launch_weight<NV, NC, 4>(p, in, wi, cbar, ebar, st);
  }
  return cudaErrorInvalidValue;
}

static AdjParams adj_params(const xatu_ctx* ctx, int ns) {
  AdjParams p;
  memset(&p, 0, sizeof(p));
  p.nk = ctx->nk;
  p.nv = ctx->nv;
  p.nc = ctx->nc;
  p.nb = ctx->nb;
  p.norb = ctx->norb;
  p.na = ctx->natoms;
  p.ns = ns;
  p.N = ctx->N_full;
  p.mode = ctx->mode == XATU_MODE_REALSPACE ? 0 : 1;
  p.emap.ndim = ctx->ndim;
  p.emap.n = ctx->n_eff;
  for (int i = 0; i < 3 * ctx->ndim; i++) p.emap.B[i] = ctx->recip[i];
  for (int i = 0; i < ctx->ndim * ctx->ndim; i++) p.emap.inv[i] = ctx->inv_gram[i];
  p.rt_ndim = ctx->ndim;
  for (int a = 0; a < 3; a++) {
    p.rt_len[a] = ctx->rt_len[a];
    p.rt_span[a] = ctx->rt_span[a];
  }
  p.nentries = ctx->mode == XATU_MODE_REALSPACE ? (long long)ctx->nmesh : ctx->rt_entries;
  for (int a = 0; a <= ctx->natoms; a++) p.orb_off[a] = ctx->orb_off[a];
  return p;
}

// Weighted back-propagation through the assembly: cbar (nk x nb x norb), ebar (nk x nb) of
// sum_ij Y_ij H_ij for the row-major weight matrix Y on the device.
xatu_status xatu_adjoint_weighted(xatu_ctx* ctx, const cd* Y, const cd* Zc, const cd* Zv, cd* cbar, double* ebar) {
  if (ctx->nv > 2 || ctx->nc > 2 || ctx->natoms > 4)
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "adjoint supports at most 2 valence, 2 conduction bands and 4 atoms");
  const AdjParams p = adj_params(ctx, 1);
  AdjInputs in;
  memset(&in, 0, sizeof(in));
  in.kpoints = ctx->d_kpoints.as<double>();
  in.kgrid = ctx->d_kgrid.as<int>();
  in.eigvec = ctx->d_eigvec.as<cd>();
  in.eigvecQ = ctx->d_eigvecQ.as<cd>();
  in.table = ctx->d_table.as<cd>();
  in.status = ctx->d_status.as<int>();
  AdjWeightInputs wi;
  wi.Y = Y;
  wi.Zc = Zc;
  wi.Zv = Zv;
  wi.VX = ctx->d_VX.as<cd>();
  cudaError_t e = cudaErrorInvalidValue;
  if (p.nv == 1 && p.nc == 1) e = launch_weight_na<1, 1>(p, in, wi, cbar, ebar, ctx->stream);
  if (p.nv == 1 && p.nc == 2) e = launch_weight_na<1, 2>(p, in, wi, cbar, ebar, ctx->stream);
  if (p.nv == 2 && p.nc == 1) e = launch_weight_na<2, 1>(p, in, wi, cbar, ebar, ctx->stream);
  if (p.nv == 2 && p.nc == 2) e = launch_weight_na<2, 2>(p, in, wi, cbar, ebar, ctx->stream);
  ctx->launches++;
  XATU_CK(e);
  return XATU_OK;
}

extern "C" xatu_status xatu_adjoint(xatu_ctx* ctx, int nstates, const double* eigvec, double* grad_hamiltonian,
                                    double* grad_params) {
  if (!ctx || !eigvec || nstates < 1) return xatu_fail(ctx, XATU_ERR_INVALID, "bad argument");
  cudaSetDevice(ctx->device);
  if (!ctx->bands_ok || !ctx->tables_ok) return xatu_fail(ctx, XATU_ERR_STATE, "bands and tables must be built first");
  if (nstates > XATU_ADJOINT_MAX_STATES)
    return xatu_fail(ctx, XATU_ERR_INVALID, "at most 8 eigenvectors per call");
  if (ctx->custom_basis) return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "adjoint needs the full e-h basis");
  if (ctx->nv > 2 || ctx->nc > 2 || ctx->natoms > 4)
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "adjoint supports at most 2 valence, 2 conduction bands and 4 atoms");
  if (grad_hamiltonian && !ctx->bands_from_model)
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED,
                     "hopping gradients need bands computed from the model (xatu_bands_compute), not uploaded ones");
  const int ns = nstates, na = ctx->natoms, norb = ctx->norb, nk = ctx->nk, nb = ctx->nb;
  const long long N = ctx->N_full;
  if (ctx->N != N) return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "adjoint needs the full e-h basis");
  cudaStream_t st = ctx->stream;
  XATU_CK(cudaEventRecord(ctx->ev[10], st));

  // eigenvectors, derivative tables
  XATU_CK(ctx->d_adjX.ensure((size_t)N * ns * sizeof(cd)));
  XATU_CK(cudaMemcpyAsync(ctx->d_adjX.p, eigvec, (size_t)N * ns * sizeof(cd), cudaMemcpyHostToDevice, st));
  {
    xatu_status s0 = xatu_derivative_tables(ctx, 0);
    if (s0 != XATU_OK) return s0;
  }
  const long long nentries = ctx->mode == XATU_MODE_REALSPACE ? (long long)ctx->nmesh : ctx->rt_entries;
  // exchange: alpha, u = VX conj(alpha), w = VX^T alpha (host, na x na)
  std::vector<cd> alpha((size_t)ns * na, mk(0, 0)), VX((size_t)na * na, mk(0, 0)), dVX((size_t)na * na, mk(0, 0));
  std::vector<cd> exu((size_t)ns * na), exw((size_t)ns * na);
  if (ctx->exchange) {
    XATU_CK(ctx->d_exL.ensure((size_t)N * na * sizeof(cd)));
    XATU_CK(ctx->d_exR.ensure((size_t)N * na * sizeof(cd)));
    exchange_vectors_kernel<<<(unsigned)((N + 127) / 128), 128, 0, st>>>(
        (int)N, ctx->nv, ctx->nc, nb, norb, na, ctx->d_orboff.as<int>(), ctx->d_eigvec.as<cd>(),
        ctx->d_eigvecQ.as<cd>(), ctx->d_VX.as<cd>(), nullptr, ctx->d_exL.as<cd>(), ctx->d_exR.as<cd>());
    ctx->launches++;
    XATU_CK(cudaGetLastError());
    XATU_CK(ctx->d_adjAlpha.ensure((size_t)ns * na * sizeof(cd)));
    adj_alpha_kernel<<<dim3(ns, na), 256, 0, st>>>(N, na, ctx->d_adjX.as<cd>(), ctx->d_exL.as<cd>(),
                                                   ctx->d_adjAlpha.as<cd>());
    ctx->launches++;
    XATU_CK(cudaGetLastError());
    XATU_CK(cudaMemcpyAsync(alpha.data(), ctx->d_adjAlpha.p, alpha.size() * sizeof(cd), cudaMemcpyDeviceToHost, st));
    XATU_CK(cudaMemcpyAsync(VX.data(), ctx->d_VX.p, VX.size() * sizeof(cd), cudaMemcpyDeviceToHost, st));
    XATU_CK(cudaMemcpyAsync(dVX.data(), ctx->d_adjdVX.p, dVX.size() * sizeof(cd), cudaMemcpyDeviceToHost, st));
    XATU_CK(cudaStreamSynchronize(st));
    for (int s = 0; s < ns; s++)
      for (int a = 0; a < na; a++) {
        cd u = mk(0, 0), w = mk(0, 0);
        for (int b = 0; b < na; b++) {
          u = u + VX[a * na + b] * conj(alpha[s * na + b]);
          w = w + alpha[s * na + b] * VX[b * na + a];
        }
        exu[s * na + a] = u;
        exw[s * na + a] = w;
      }
    XATU_CK(ctx->d_adjExUW.ensure((size_t)2 * ns * na * sizeof(cd)));
    XATU_CK(cudaMemcpyAsync(ctx->d_adjExUW.p, exu.data(), exu.size() * sizeof(cd), cudaMemcpyHostToDevice, st));
    XATU_CK(cudaMemcpyAsync(ctx->d_adjExUW.as<cd>() + ns * na, exw.data(), exw.size() * sizeof(cd),
                            cudaMemcpyHostToDevice, st));
  }

  // pair kernel
  AdjParams p;
  memset(&p, 0, sizeof(p));
  p.nk = nk;
  p.nv = ctx->nv;
  p.nc = ctx->nc;
  p.nb = nb;
  p.norb = norb;
  p.na = na;
  p.ns = ns;
  p.N = N;
  p.mode = ctx->mode == XATU_MODE_REALSPACE ? 0 : 1;
  p.emap.ndim = ctx->ndim;
  p.emap.n = ctx->n_eff;
  for (int i = 0; i < 3 * ctx->ndim; i++) p.emap.B[i] = ctx->recip[i];
  for (int i = 0; i < ctx->ndim * ctx->ndim; i++) p.emap.inv[i] = ctx->inv_gram[i];
  p.rt_ndim = ctx->ndim;
  for (int a = 0; a < 3; a++) {
    p.rt_len[a] = ctx->rt_len[a];
    p.rt_span[a] = ctx->rt_span[a];
  }
  p.nentries = nentries;
  for (int a = 0; a <= na; a++) p.orb_off[a] = ctx->orb_off[a];
  XATU_CK(ctx->d_adjCbar.ensure((size_t)ns * nk * nb * norb * sizeof(cd)));
  XATU_CK(ctx->d_adjEbar.ensure((size_t)ns * nk * nb * sizeof(double)));
  XATU_CK(ctx->d_adjEpart.ensure((size_t)nk * ns * 2 * sizeof(double)));
  AdjInputs in;
  in.kpoints = ctx->d_kpoints.as<double>();
  in.kgrid = ctx->d_kgrid.as<int>();
  in.eigvec = ctx->d_eigvec.as<cd>();
  in.eigvecQ = ctx->d_eigvecQ.as<cd>();
  in.table = ctx->d_table.as<cd>();
  in.dtable = ctx->d_adjdtable.as<cd>();
  in.x = ctx->d_adjX.as<cd>();
  in.exu = ctx->exchange ? ctx->d_adjExUW.as<cd>() : nullptr;
  in.exw = ctx->exchange ? ctx->d_adjExUW.as<cd>() + ns * na : nullptr;
  in.status = ctx->d_status.as<int>();
  AdjOutputs out;
  out.cbar = ctx->d_adjCbar.as<cd>();
  out.ebar = ctx->d_adjEbar.as<double>();
  out.epart = ctx->d_adjEpart.as<double>();
  XATU_CK(cudaEventRecord(ctx->ev[8], st));
  XATU_CK(launch_pair_any(p, in, out, st));
  ctx->launches++;
  XATU_CK(cudaEventRecord(ctx->ev[9], st));

  // potential parameters
  std::vector<double> epart((size_t)nk * ns * 2);
  XATU_CK(cudaMemcpyAsync(epart.data(), out.epart, epart.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  XATU_CK(cudaStreamSynchronize(st));
  cudaEventElapsedTime(&ctx->adj_pair_ms, ctx->ev[8], ctx->ev[9]);
  {
    xatu_status s0 = xatu_check_device_status(ctx, "adjoint pair sums");
    if (s0 != XATU_OK) return s0;
  }
  if (grad_params) {
    const double eps_bar = (ctx->eps_m + ctx->eps_s) / 2;
    const bool dkel = ctx->mode != XATU_MODE_REALSPACE || ctx->potential == XATU_POT_KELDYSH;
    const bool xkel = ctx->mode != XATU_MODE_REALSPACE || ctx->exchange_potential == XATU_POT_KELDYSH;
    for (int s = 0; s < ns; s++) {
      double eV = 0.0, eR = 0.0;
      for (int k = 0; k < nk; k++) {
        eV += epart[((size_t)k * ns + s) * 2];
        eR += epart[((size_t)k * ns + s) * 2 + 1];
      }
      double xV = 0.0, xR = 0.0;
      if (ctx->exchange)
        for (int a = 0; a < na; a++)
          for (int b = 0; b < na; b++) {
            xV += (alpha[s * na + a] * VX[a * na + b] * conj(alpha[s * na + b])).x;
            xR += (alpha[s * na + a] * dVX[a * na + b] * conj(alpha[s * na + b])).x;
          }
      const double deps = (dkel ? eV : 0.0) / (2 * eps_bar) - (xkel ? xV : 0.0) / (2 * eps_bar);
      grad_params[3 * s] = -eR + xR;
      grad_params[3 * s + 1] = deps;
      grad_params[3 * s + 2] = deps;
    }
  }

  // hopping matrices
  if (grad_hamiltonian) {
    xatu_status sb = xatu_adjoint_bands_to_hoppings(ctx, ns, out.cbar, out.ebar);
    if (sb != XATU_OK) return sb;
    const size_t n2 = (size_t)norb * norb;
    XATU_CK(cudaMemcpyAsync(grad_hamiltonian, ctx->d_adjG.p, (size_t)ns * ctx->nR * n2 * sizeof(cd),
                            cudaMemcpyDeviceToHost, st));
    XATU_CK(cudaStreamSynchronize(st));
    xatu_status s1 = xatu_check_device_status(ctx, "adjoint band solve");
    if (s1 != XATU_OK) return s1;
  }
  XATU_CK(cudaEventRecord(ctx->ev[11], st));
  XATU_CK(cudaEventSynchronize(ctx->ev[11]));
  cudaEventElapsedTime(&ctx->adjoint_ms, ctx->ev[10], ctx->ev[11]);
  return XATU_OK;
}
