// Exciton post-processing on the device: the observables and writers of Result / ResultTB that consume the
// eigen-pairs of the BSE (Result.tpp:25-484, ResultTB.cpp:21-98, :310-481) and the Kubo absorption of
// skubo_w (skubo_w.f90:2-173, :630-720).
//
// Coefficients X (N x ns, column-major) use the e-h basis of the build, row = k*nc*nv + c*nv + v; band stacks
// are the context's (nk x nb x norb, valence columns first).
//
// pp_state_obs_kernel   one warp per (k, state): sum_cv |A|^2 (reciprocal amplitude), the kinetic energy
//                       sum |A|^2 (E^Q_c - E_v), the first largest |A| of the k block and, on request, the
//                       spin of hole and electron through the nv x nv / nc x nc band spin matrices.
// pp_state_reduce_kernel  one CTA per state: ordered sums of those per-k partials.
// pp_rs_pair_kernel     F_s[k][a][b] = sum_cv A_s(k,c,v) C^Q_{k,c}[a] conj(C_{k,v}[hole orbital b]).
// pp_kdft_kernel        G[point][p] = sum_k exp(+-i k.d_point) F[k][p] over a k range (split-k partials):
//                       a point tile x pair tile per CTA, the phase tile computed once in shared memory and
//                       shared by all pairs, pairs on lanes, the k range of a stage spread over the spare lanes.
// pp_rs_finish_kernel   |G|^2 summed over the orbitals of each electron atom and the hole orbitals.
// pp_absorption_kernel  one CTA per frequency: the single-particle Kubo sum over every (k, c, v) with the
//                       Gaussian delta of get_kubo_intens and the broadened exciton oscillator strengths.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>

#include "engine.h"

#define PP_HARTREE 27.211385
#define PP_BOHR 0.52917721067121
#define PP_PI 3.141592653589793

// ------------------------------------------------------------------ per-state reductions

struct ObsParams {
  int nk, nv, nc, nb, norb, ns;
  long long N;
  int spin;
};

#define OBS_PARTS 6   // kinetic, hole (re, im), electron (re, im), largest |A|^2

__device__ __forceinline__ void pp_argmax_merge(double& mx, long long& mi, double m2, long long i2) {
  if (m2 > mx || (m2 == mx && i2 < mi)) {
    mx = m2;
    mi = i2;
  }
}

extern "C" __global__ void __launch_bounds__(256) pp_state_obs_kernel(ObsParams p, const cd* __restrict__ X,
                                                                      const double* __restrict__ eval,
                                                                      const double* __restrict__ evalQ,
                                                                      const cd* __restrict__ evec,
                                                                      const cd* __restrict__ evecQ,
                                                                      const double* __restrict__ sz,
                                                                      double* __restrict__ kweight,
                                                                      double* __restrict__ part,
                                                                      long long* __restrict__ pidx) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k = blockIdx.x * (blockDim.x >> 5) + warp;
  const int s = blockIdx.y;
  if (k >= p.nk) return;   // whole warp
  const int nv = p.nv, nc = p.nc, nb = p.nb, norb = p.norb, nvc = nv * nc;
  const cd* A = X + (long long)s * p.N + (long long)k * nvc;
  double w = 0, kin = 0, mx = -1.0;
  long long mi = LLONG_MAX;
  for (int e = lane; e < nvc; e += 32) {
    const cd a = A[e];
    const int c = e / nv, v = e - c * nv;
    const double m2 = nrm2(a);
    w += m2;
    kin += m2 * (evalQ[(long long)k * nb + nv + c] - eval[(long long)k * nb + v]);
    if (m2 > mx) {   // lanes walk e upwards: the first largest is kept
      mx = m2;
      mi = e;
    }
  }
  cd hole = mk(0, 0), elec = mk(0, 0);
  if (p.spin) {
    const cd* Ck = evec + (long long)k * nb * norb;
    const cd* CQk = evecQ + (long long)k * nb * norb;
    // hole: -sum_c sum_ij conj(A[c,i]) Sh(i,j) A[c,j],  Sh(i,j) = sum_a conj(C_vj[a]) C_vi[a] sz[a]
    for (int t = lane; t < nv * nv; t += 32) {
      const int i = t / nv, j = t - i * nv;
      cd sh = mk(0, 0), th = mk(0, 0);
      for (int a = 0; a < norb; a++) sh = sh + sz[a] * cmulc(Ck[j * norb + a], Ck[i * norb + a]);
      for (int c = 0; c < nc; c++) th = th + cmulc(A[c * nv + i], A[c * nv + j]);
      hole = hole + sh * th;
    }
    // electron: sum_v sum_ij conj(A[i,v]) Se(i,j) A[j,v],  Se(i,j) = sum_a conj(CQ_ci[a]) CQ_cj[a] sz[a]
    for (int t = lane; t < nc * nc; t += 32) {
      const int i = t / nc, j = t - i * nc;
      cd se = mk(0, 0), te = mk(0, 0);
      for (int a = 0; a < norb; a++) se = se + sz[a] * cmulc(CQk[(nv + i) * norb + a], CQk[(nv + j) * norb + a]);
      for (int v = 0; v < nv; v++) te = te + cmulc(A[i * nv + v], A[j * nv + v]);
      elec = elec + se * te;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    w += __shfl_xor_sync(0xffffffffu, w, o);
    kin += __shfl_xor_sync(0xffffffffu, kin, o);
    hole.x += __shfl_xor_sync(0xffffffffu, hole.x, o);
    hole.y += __shfl_xor_sync(0xffffffffu, hole.y, o);
    elec.x += __shfl_xor_sync(0xffffffffu, elec.x, o);
    elec.y += __shfl_xor_sync(0xffffffffu, elec.y, o);
    const double m2 = __shfl_xor_sync(0xffffffffu, mx, o);
    const long long i2 = __shfl_xor_sync(0xffffffffu, mi, o);
    pp_argmax_merge(mx, mi, m2, i2);
  }
  if (lane == 0) {
    const long long r = (long long)s * p.nk + k;
    kweight[r] = w;
    double* q = part + r * OBS_PARTS;
    q[0] = kin;
    q[1] = -hole.x;
    q[2] = -hole.y;
    q[3] = elec.x;
    q[4] = elec.y;
    q[5] = mx;
    pidx[r] = (mi == LLONG_MAX) ? LLONG_MAX : (long long)k * nvc + mi;
  }
}

// One CTA (256 threads) per state: kinetic[s], spin[s] = {total, 0, hole re, im, electron re, im}, peak[s] = k
// index of the first largest |A|.
extern "C" __global__ void __launch_bounds__(256) pp_state_reduce_kernel(int nk, int nvc, const double* __restrict__ part,
                                                                         const long long* __restrict__ pidx,
                                                                         double* __restrict__ out /* ns x 8 */) {
  const int s = blockIdx.x;
  double acc[5] = {0, 0, 0, 0, 0};
  double mx = -1.0;
  long long mi = LLONG_MAX;
  for (int k = threadIdx.x; k < nk; k += blockDim.x) {
    const double* q = part + ((long long)s * nk + k) * OBS_PARTS;
#pragma unroll
    for (int t = 0; t < 5; t++) acc[t] += q[t];
    pp_argmax_merge(mx, mi, q[5], pidx[(long long)s * nk + k]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int t = 0; t < 5; t++) acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], o);
    const double m2 = __shfl_xor_sync(0xffffffffu, mx, o);
    const long long i2 = __shfl_xor_sync(0xffffffffu, mi, o);
    pp_argmax_merge(mx, mi, m2, i2);
  }
  __shared__ double sacc[8][5], smx[8];
  __shared__ long long smi[8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
#pragma unroll
    for (int t = 0; t < 5; t++) sacc[warp][t] = acc[t];
    smx[warp] = mx;
    smi[warp] = mi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot[5] = {0, 0, 0, 0, 0};
    double m = -1.0;
    long long i = LLONG_MAX;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      for (int t = 0; t < 5; t++) tot[t] += sacc[w][t];
      pp_argmax_merge(m, i, smx[w], smi[w]);
    }
    double* o = out + (long long)s * 8;
    o[0] = tot[0];
    o[1] = tot[1] + tot[3];   // real(hole + electron)
    o[2] = tot[1];
    o[3] = tot[2];
    o[4] = tot[3];
    o[5] = tot[4];
    o[6] = (i == LLONG_MAX) ? -1.0 : (double)(i / nvc);   // -1: no finite coefficient
    o[7] = 0;
  }
}

// ------------------------------------------------------------------ real-space amplitude

// F[k][p], p = (s * norb + a) * nho + b.
extern "C" __global__ void pp_rs_pair_kernel(int nk, int nv, int nc, int nb, int norb, int hoff, int nho, int ns,
                                             long long N, const cd* __restrict__ X, const cd* __restrict__ evec,
                                             const cd* __restrict__ evecQ, cd* __restrict__ F) {
  const long long P = (long long)ns * norb * nho;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)nk * P) return;
  const int k = (int)(idx / P);
  const int pp = (int)(idx - (long long)k * P);
  const int b = pp % nho, a = (pp / nho) % norb, s = pp / (nho * norb);
  const int nvc = nv * nc;
  const cd* A = X + (long long)s * N + (long long)k * nvc;
  cd acc = mk(0, 0);
  for (int c = 0; c < nc; c++) {
    const cd cq = evecQ[((long long)k * nb + nv + c) * norb + a];
    for (int v = 0; v < nv; v++) {
      const cd hv = evec[((long long)k * nb + v) * norb + hoff + b];
      acc = acc + cmulc(hv, A[c * nv + v] * cq);   // A C^Q conj(C)
    }
  }
  F[idx] = acc;
}

// Complex weights F[k][s] = kweight[s][k] (the envelope transform).
extern "C" __global__ void pp_weights_to_f_kernel(int nk, int ns, const double* __restrict__ kweight,
                                                  cd* __restrict__ F) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)nk * ns) return;
  const int k = (int)(idx / ns), s = (int)(idx - (long long)k * ns);
  F[idx] = mk(kweight[(long long)s * nk + k], 0.0);
}

// E[pt][k] = exp(i sign k.d_pt) for npts points (the phase factors of the GEMM form of the transform).
extern "C" __global__ void pp_phase_kernel(int nk, int npts, const double* __restrict__ kpts,
                                           const double* __restrict__ pts, double sign, cd* __restrict__ E) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)nk * npts) return;
  const int pt = (int)(idx / nk), k = (int)(idx - (long long)pt * nk);
  const double x = kpts[3 * k] * pts[3 * pt] + kpts[3 * k + 1] * pts[3 * pt + 1] + kpts[3 * k + 2] * pts[3 * pt + 2];
  double sn, cs;
  sincos(x, &sn, &cs);
  E[idx] = mk(cs, sign * sn);
}

#define DFT_TK 16    // k points per shared-memory stage

// part[z][pt][p] = sum_{k in split z} exp(i sign k.d_pt) F[k][p].  A CTA covers 8*CPW points x PT*NPL pairs:
// the phase tile (8*CPW points x 16 k) is evaluated once per stage in shared memory and shared by all pairs of
// the CTA; lane l holds pairs l % PT + j*PT (j < NPL) for the CPW points of its warp, so each phase read feeds
// NPL complex products and each F read feeds CPW.  With PT < 32 the 32 / PT lane groups take interleaved k of
// each stage and are summed by a fixed butterfly at the end (deterministic for a given launch shape).
template <int PT, int NPL, int CPW>
constexpr size_t pp_kdft_smem() {
  return sizeof(double2) * ((size_t)8 * CPW * (DFT_TK + 1) + (size_t)DFT_TK * PT * NPL) +
         sizeof(double) * 3 * (8 * CPW + DFT_TK);
}

template <int PT, int NPL, int CPW>
__global__ void __launch_bounds__(256, 2) pp_kdft_kernel(int nk, int P, const double* __restrict__ kpts,
                                                         const cd* __restrict__ F, int npts,
                                                         const double* __restrict__ pts, double sign, int kchunk,
                                                         cd* __restrict__ part) {
  constexpr int PW = PT * NPL;   // pairs per CTA
  constexpr int TC = 8 * CPW;    // points per CTA
  extern __shared__ __align__(16) unsigned char pp_smem[];
  auto ph = reinterpret_cast<double2(*)[DFT_TK + 1]>(pp_smem);                                   // [TC][TK + 1]
  auto fs = reinterpret_cast<double2(*)[PW]>(pp_smem + sizeof(double2) * TC * (DFT_TK + 1));        // [TK][PW]
  auto dp = reinterpret_cast<double(*)[3]>(pp_smem + sizeof(double2) * (TC * (DFT_TK + 1) + DFT_TK * PW));
  auto kp = dp + TC;                                                                             // [TK][3]
  constexpr int KS = 32 / PT;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int pl = lane % PT, ks = lane / PT;
  const int pt0 = blockIdx.x * TC, p0 = blockIdx.y * PW;
  const int kbeg = blockIdx.z * kchunk, kend = min(nk, kbeg + kchunk);
  for (int t = tid; t < TC * 3; t += blockDim.x) {
    const int c = t / 3, d = t - c * 3;
    dp[c][d] = (pt0 + c < npts) ? pts[(long long)(pt0 + c) * 3 + d] : 0.0;
  }
  double2 acc[CPW][NPL];
#pragma unroll
  for (int c = 0; c < CPW; c++)
#pragma unroll
    for (int j = 0; j < NPL; j++) acc[c][j] = make_double2(0.0, 0.0);
  for (int k0 = kbeg; k0 < kend; k0 += DFT_TK) {
    __syncthreads();   // the previous stage is consumed (and dp is visible on the first pass)
    if (tid < DFT_TK * 3) {
      const int kk = tid / 3, d = tid - kk * 3;
      kp[kk][d] = (k0 + kk < kend) ? kpts[(long long)(k0 + kk) * 3 + d] : 0.0;
    }
    for (int t = tid; t < DFT_TK * PW; t += blockDim.x) {
      const int kk = t / PW, q = t - kk * PW;
      cd f = mk(0, 0);
      if (k0 + kk < kend && p0 + q < P) f = F[(long long)(k0 + kk) * P + p0 + q];
      fs[kk][q] = make_double2(f.x, f.y);
    }
    __syncthreads();
    for (int t = tid; t < TC * DFT_TK; t += blockDim.x) {
      const int c = t / DFT_TK, kk = t - c * DFT_TK;
      const double x = kp[kk][0] * dp[c][0] + kp[kk][1] * dp[c][1] + kp[kk][2] * dp[c][2];
      double sn, cs;
      sincos(x, &sn, &cs);
      ph[c][kk] = make_double2(cs, sign * sn);
    }
    __syncthreads();
    for (int kk = ks; kk < DFT_TK; kk += KS) {
      double2 f[NPL];
#pragma unroll
      for (int j = 0; j < NPL; j++) f[j] = fs[kk][pl + j * PT];
#pragma unroll
      for (int c = 0; c < CPW; c++) {
        const double2 e = ph[warp * CPW + c][kk];
#pragma unroll
        for (int j = 0; j < NPL; j++) {
          acc[c][j].x = fma(e.x, f[j].x, fma(-e.y, f[j].y, acc[c][j].x));
          acc[c][j].y = fma(e.x, f[j].y, fma(e.y, f[j].x, acc[c][j].y));
        }
      }
    }
  }
#pragma unroll
  for (int o = PT; o < 32; o <<= 1) {
#pragma unroll
    for (int c = 0; c < CPW; c++)
#pragma unroll
      for (int j = 0; j < NPL; j++) {
        acc[c][j].x += __shfl_xor_sync(0xffffffffu, acc[c][j].x, o);
        acc[c][j].y += __shfl_xor_sync(0xffffffffu, acc[c][j].y, o);
      }
  }
  if (ks == 0) {
#pragma unroll
    for (int j = 0; j < NPL; j++) {
      const int p = p0 + pl + j * PT;
      if (p >= P) continue;
#pragma unroll
      for (int c = 0; c < CPW; c++) {
        const int pt = pt0 + warp * CPW + c;
        if (pt < npts) part[((long long)blockIdx.z * npts + pt) * P + p] = mk(acc[c][j].x, acc[c][j].y);
      }
    }
  }
}

// out[s][pt][atom] = sum_{a in atom} sum_b |sum_z part[z][pt][(s * norb + a) * nho + b]|^2.
extern "C" __global__ void pp_rs_finish_kernel(int npts, int P, int nsplit, int ns, int natoms,
                                               const int* __restrict__ orboff, int norb, int nho,
                                               const cd* __restrict__ part, double* __restrict__ out) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)ns * npts * natoms) return;
  const int atom = (int)(idx % natoms);
  const int pt = (int)((idx / natoms) % npts);
  const int s = (int)(idx / ((long long)natoms * npts));
  double total = 0;
  for (int a = orboff[atom]; a < orboff[atom + 1]; a++) {
    for (int b = 0; b < nho; b++) {
      const int p = (s * norb + a) * nho + b;
      cd g = mk(0, 0);
      for (int z = 0; z < nsplit; z++) g = g + part[((long long)z * npts + pt) * P + p];
      total += nrm2(g);
    }
  }
  out[idx] = total;
}

// out[s][pt] = Re sum_z part[z][pt][s].
extern "C" __global__ void pp_env_finish_kernel(int npts, int ns, int nsplit, const cd* __restrict__ part,
                                                double* __restrict__ out) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)ns * npts) return;
  const int s = (int)(idx / npts), pt = (int)(idx - (long long)s * npts);
  double g = 0;
  for (int z = 0; z < nsplit; z++) g += part[((long long)z * npts + pt) * ns + s].x;
  out[idx] = g;
}

// ------------------------------------------------------------------ absorption

struct AbsParams {
  int nk, nv, nc, nb, ns, nw, broad;
  long long N;
  double w0, wrange, eta, pref;   // eta in Hartree, pref = pi / (nk vcell)
};

__device__ __forceinline__ double pp_broadening(int kind, double x, double eta) {
  if (kind == XATU_BROAD_LORENTZIAN) return 1.0 / PP_PI * (eta / (x * x + eta * eta));
  if (kind == XATU_BROAD_GAUSSIAN) return 1.0 / eta * 1.0 / sqrt(2.0 * PP_PI) * exp(-0.5 / (eta * eta) * (x * x));
  if (kind == XATU_BROAD_EXPONENTIAL) return 0.5 / eta * exp(-fabs(x) / eta);
  return 1.0;
}

// sig_sp[iw][i][j] = sum_{k,c,v} pref f [vme_i(c,v) vme_j(v,c) g(w - e_c + e_v) + vme_i(v,c) vme_j(c,v) g(w - e_v + e_c)]
// with f = -1/(e_c - e_v) and vme(v,c) = conj(vme(c,v)) = u (vme_kernel's output); sig_ex[iw][i][j], i, j < 2:
// sum_n Re(pref conj(V_i,n) V_j,n / E_n) broadening(w - E_n).
extern "C" __global__ void __launch_bounds__(256) pp_absorption_kernel(AbsParams p, const double* __restrict__ eval,
                                                                       const cd* __restrict__ vme,
                                                                       const double* __restrict__ exen,
                                                                       const cd* __restrict__ vex,
                                                                       cd* __restrict__ sig_sp,
                                                                       double* __restrict__ sig_ex) {
  const int iw = blockIdx.x;
  const double w = (p.w0 + p.wrange / (double)p.nw * (double)iw) / PP_HARTREE;
  const double eta = p.eta;
  const int nv = p.nv, nvc = p.nv * p.nc;
  cd acc[9];
#pragma unroll
  for (int t = 0; t < 9; t++) acc[t] = mk(0, 0);
  for (long long j = threadIdx.x; j < p.N; j += blockDim.x) {
    const int k = (int)(j / nvc);
    const int r = (int)(j - (long long)k * nvc);
    const int c = r / nv, v = r - c * nv;
    const double ec = eval[(long long)k * p.nb + nv + c] / PP_HARTREE;
    const double ev = eval[(long long)k * p.nb + v] / PP_HARTREE;
    const double f1 = p.pref * (-1.0 / (ec - ev));   // (n, n') = (c, v)
    const double f2 = p.pref * (1.0 / (ev - ec));    // (n, n') = (v, c)
    const double x1 = (w - ec) + ev, x2 = (w - ev) + ec;
    const double g1 = 1.0 / eta * 1.0 / sqrt(2.0 * PP_PI) * exp(-0.5 / (eta * eta) * (x1 * x1));
    const double g2 = 1.0 / eta * 1.0 / sqrt(2.0 * PP_PI) * exp(-0.5 / (eta * eta) * (x2 * x2));
    cd u[3];
#pragma unroll
    for (int i = 0; i < 3; i++) u[i] = vme[(long long)i * p.N + j];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const cd t1 = f1 * cmulc(u[i], u[q]);          // conj(u_i) u_q
        const cd t2 = f2 * cmulc(u[q], u[i]);          // u_i conj(u_q)
        acc[i * 3 + q] = acc[i * 3 + q] + g1 * t1 + g2 * t2;
      }
  }
  double ax[4] = {0, 0, 0, 0};
  for (int n = threadIdx.x; n < p.ns; n += blockDim.x) {
    const double en = exen[n] / PP_HARTREE;
    const double rb = pp_broadening(p.broad, w - en, eta);
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const cd t = (p.pref * conj(vex[(long long)n * 3 + i])) * vex[(long long)n * 3 + q];
        ax[i * 2 + q] += (t.x / en) * rb;
      }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int t = 0; t < 9; t++) {
      acc[t].x += __shfl_xor_sync(0xffffffffu, acc[t].x, o);
      acc[t].y += __shfl_xor_sync(0xffffffffu, acc[t].y, o);
    }
#pragma unroll
    for (int t = 0; t < 4; t++) ax[t] += __shfl_xor_sync(0xffffffffu, ax[t], o);
  }
  __shared__ cd sacc[8][9];
  __shared__ double sax[8][4];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
#pragma unroll
    for (int t = 0; t < 9; t++) sacc[warp][t] = acc[t];
#pragma unroll
    for (int t = 0; t < 4; t++) sax[warp][t] = ax[t];
  }
  __syncthreads();
  if (threadIdx.x < 9) {
    cd tsum = mk(0, 0);
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) tsum = tsum + sacc[q][threadIdx.x];
    sig_sp[(long long)iw * 9 + threadIdx.x] = tsum;
    const int i = threadIdx.x / 3, q = threadIdx.x % 3;
    double e = 0;
    if (i < 2 && q < 2)
      for (int wq = 0; wq < (int)(blockDim.x >> 5); wq++) e += sax[wq][i * 2 + q];
    sig_ex[(long long)iw * 9 + threadIdx.x] = e;
  }
}

// ------------------------------------------------------------------ host entries

static xatu_status pp_check(xatu_ctx* ctx, int ns, const double* eigvec) {
  if (!ctx) return XATU_ERR_INVALID;
  if (ns < 1 || !eigvec) return xatu_fail(ctx, XATU_ERR_INVALID, "bad argument");
  cudaSetDevice(ctx->device);
  if (!ctx->bands_ok) return xatu_fail(ctx, XATU_ERR_STATE, "bands are not computed");
  if (ctx->custom_basis)
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "post-processing needs the full e-h basis (last build used a subset)");
  return XATU_OK;
}

static long long pp_dim(const xatu_ctx* ctx) { return (long long)ctx->nk * ctx->nv * ctx->nc; }

// Buffers of the entries below (all sized before an entry's first launch):
//   d_pp_X  coefficients (N x ns)          d_pp_A  pair table F / velocity matrix elements
//   d_pp_B  per-k weights, points, output  d_pp_C  per-k partials of the state reductions
//   d_pp_D  state summaries / absorption   d_pp_P  split-k partials of the k-space transforms
//   d_pp_E  phase matrix of the GEMM form of the transform

static size_t pp_obs_bytes_c(const xatu_ctx* ctx, int ns) {
  return (size_t)ns * ctx->nk * (OBS_PARTS + 1) * sizeof(double) + (size_t)ctx->norb * sizeof(double);
}

// Uploads X and runs the per-state reductions: kweight (ns x nk) into d_pp_B, and with reduce the ns x 8
// summaries into d_pp_D.  The caller has sized d_pp_X, d_pp_B (ns * nk doubles), d_pp_C and d_pp_D.
static xatu_status pp_state_obs(xatu_ctx* ctx, int ns, const double* eigvec, bool spin, bool reduce) {
  const long long N = pp_dim(ctx);
  const int nk = ctx->nk;
  double* part = ctx->d_pp_C.as<double>();
  long long* pidx = reinterpret_cast<long long*>(part + (size_t)ns * nk * OBS_PARTS);
  double* sz = reinterpret_cast<double*>(pidx + (size_t)ns * nk);
  if (spin) {
    std::vector<double> h(ctx->norb, 0.0);
    for (int a = 0; a < ctx->natoms; a++) {
      const int n = ctx->orb_off[a + 1] - ctx->orb_off[a];
      if (n % 2) return xatu_fail(ctx, XATU_ERR_INVALID, "spinX needs an even number of orbitals on every atom");
      for (int o = 0; o < n; o++) h[ctx->orb_off[a] + o] = (o % 2) ? -0.5 : 0.5;
    }
    XATU_CK(cudaMemcpyAsync(sz, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    XATU_CK(cudaStreamSynchronize(ctx->stream));   // h is a local
  }
  XATU_CK(cudaMemcpyAsync(ctx->d_pp_X.p, eigvec, (size_t)N * ns * sizeof(cd), cudaMemcpyHostToDevice, ctx->stream));
  ObsParams p;
  p.nk = nk;
  p.nv = ctx->nv;
  p.nc = ctx->nc;
  p.nb = ctx->nb;
  p.norb = ctx->norb;
  p.ns = ns;
  p.N = N;
  p.spin = spin ? 1 : 0;
  dim3 g((unsigned)((nk + 7) / 8), (unsigned)ns);
  pp_state_obs_kernel<<<g, 256, 0, ctx->stream>>>(p, ctx->d_pp_X.as<cd>(), ctx->d_eigval.as<double>(),
                                                  ctx->d_eigvalQ.as<double>(), ctx->d_eigvec.as<cd>(),
                                                  ctx->d_eigvecQ.as<cd>(), sz, ctx->d_pp_B.as<double>(), part, pidx);
  ctx->launches++;
  XATU_CK_LAUNCH("pp_state_obs_kernel");
  if (!reduce) return XATU_OK;
  pp_state_reduce_kernel<<<ns, 256, 0, ctx->stream>>>(nk, ctx->nv * ctx->nc, part, pidx, ctx->d_pp_D.as<double>());
  ctx->launches++;
  XATU_CK_LAUNCH("pp_state_reduce_kernel");
  return XATU_OK;
}

extern "C" xatu_status xatu_state_observables(xatu_ctx* ctx, int nstates, const double* eigvec, double* kinetic,
                                              double* kweight, int64_t* peak, double* spin) {
  xatu_status st = pp_check(ctx, nstates, eigvec);
  if (st != XATU_OK) return st;
  const long long N = pp_dim(ctx);
  XATU_CK(ctx->d_pp_X.ensure((size_t)N * nstates * sizeof(cd)));
  XATU_CK(ctx->d_pp_B.ensure((size_t)nstates * ctx->nk * sizeof(double)));
  XATU_CK(ctx->d_pp_C.ensure(pp_obs_bytes_c(ctx, nstates)));
  XATU_CK(ctx->d_pp_D.ensure((size_t)nstates * 8 * sizeof(double)));
  st = pp_state_obs(ctx, nstates, eigvec, spin != nullptr, true);
  if (st != XATU_OK) return st;
  std::vector<double> summary((size_t)nstates * 8);
  XATU_CK(cudaMemcpyAsync(summary.data(), ctx->d_pp_D.p, summary.size() * sizeof(double), cudaMemcpyDeviceToHost,
                          ctx->stream));
  if (kweight)
    XATU_CK(cudaMemcpyAsync(kweight, ctx->d_pp_B.p, (size_t)nstates * ctx->nk * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->stream));
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  for (int s = 0; s < nstates; s++) {
    const double* o = summary.data() + (size_t)s * 8;
    if (kinetic) kinetic[s] = o[0];
    if (peak) peak[s] = (int64_t)o[6];
    if (spin) {
      double* q = spin + (size_t)s * 6;
      q[0] = o[1];
      q[1] = 0.0;
      q[2] = o[2];
      q[3] = o[3];
      q[4] = o[4];
      q[5] = o[5];
    }
  }
  return XATU_OK;
}

// Launch shape of pp_kdft_kernel: lanes per pair tile (PT), pairs per lane (NPL; 4 pairs with 4 points per
// warp, otherwise 8 points per warp), k splits and the k range of a split.  The split count fills the GPU and,
// among up to 8 splits, keeps the last wave of CTAs fullest.
struct KdftPlan {
  int PT, NPL, CPW, nsplit, kchunk;
  dim3 grid;
  int gemm;    // 1: phase matrix E (chunks of `chunk` points) times F with cuBLAS ZGEMM
  int chunk;
};

// From this many pairs on, the transform is a plain complex GEMM G = E F: the phase matrix of a chunk of
// points is formed once (pp_phase_kernel) and multiplied by cuBLAS ZGEMM (FP64 tensor cores), which sustains
// a higher FP64 rate than the fused kernel; the chunk keeps E under the byte bound.
#define PP_GEMM_MIN_PAIRS 64
#define PP_E_BUDGET (256ull << 20)

#define PP_KDFT_VARIANTS(X) \
  X(1, 1, 8) X(2, 1, 8) X(4, 1, 8) X(8, 1, 8) X(16, 1, 8) X(32, 1, 8) X(32, 2, 8) X(32, 4, 4)

static const void* pp_kdft_fn(int PT, int NPL, int CPW) {
#define PP_FN(A, B, C) \
  if (PT == A && NPL == B && CPW == C) return (const void*)pp_kdft_kernel<A, B, C>;
  PP_KDFT_VARIANTS(PP_FN)
#undef PP_FN
  return nullptr;
}

static size_t pp_kdft_smem_of(int PT, int NPL, int CPW) {
#define PP_SM(A, B, C) \
  if (PT == A && NPL == B && CPW == C) return pp_kdft_smem<A, B, C>();
  PP_KDFT_VARIANTS(PP_SM)
#undef PP_SM
  return 0;
}

static KdftPlan pp_kdft_plan(const xatu_ctx* ctx, int P, int npts) {
  KdftPlan pl;
  const int nk = ctx->nk;
  pl.gemm = 0;
  pl.chunk = 0;
  if (P >= PP_GEMM_MIN_PAIRS) {
    pl.gemm = 1;
    pl.PT = pl.NPL = pl.CPW = 0;
    pl.nsplit = 1;
    pl.kchunk = nk;
    pl.chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)npts, PP_E_BUDGET / ((size_t)nk * sizeof(cd))));
    pl.grid = dim3(1, 1, 1);
    return pl;
  }
  pl.PT = 1;
  while (pl.PT < 32 && pl.PT < P) pl.PT <<= 1;
  pl.NPL = (P >= 128) ? 4 : (P > 32) ? 2 : 1;
  pl.CPW = (pl.NPL == 4) ? 4 : 8;
  const int PW = pl.PT * pl.NPL, TC = 8 * pl.CPW;
  const long long tiles = (long long)((npts + TC - 1) / TC) * ((P + PW - 1) / PW);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pp_kdft_fn(pl.PT, pl.NPL, pl.CPW), 256,
                                                    pp_kdft_smem_of(pl.PT, pl.NPL, pl.CPW)) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const long long slots = (long long)per_sm * ctx->num_sms;
  const int max_split = std::max(1, (nk + 4 * DFT_TK - 1) / (4 * DFT_TK));
  int nsplit = 1;
  if (tiles < slots) {
    nsplit = (int)std::min<long long>((slots + tiles - 1) / tiles, max_split);
  } else {
    double best = -1.0;
    for (int z = 1; z <= std::min(8, max_split); z++) {
      const double waves = (double)(tiles * z) / (double)slots;
      const double eff = waves / std::ceil(waves);
      if (eff > best + 0.02) {
        best = eff;
        nsplit = z;
      }
    }
  }
  int kchunk = (nk + nsplit - 1) / nsplit;
  kchunk = (kchunk + DFT_TK - 1) / DFT_TK * DFT_TK;
  pl.nsplit = (nk + kchunk - 1) / kchunk;
  pl.kchunk = kchunk;
  pl.grid = dim3((unsigned)((npts + TC - 1) / TC), (unsigned)((P + PW - 1) / PW), (unsigned)pl.nsplit);
  return pl;
}

static size_t pp_kdft_bytes(const KdftPlan& pl, int P, int npts) { return (size_t)pl.nsplit * npts * P * sizeof(cd); }
static size_t pp_kdft_ebytes(const xatu_ctx* ctx, const KdftPlan& pl) {
  return pl.gemm ? (size_t)pl.chunk * ctx->nk * sizeof(cd) : 0;
}

// d_pp_P[z][pt][p] = sum_{k in split z} exp(i sign k.d_pt) F[k][p] (d_pp_P sized by the caller).
static xatu_status pp_kdft(xatu_ctx* ctx, const KdftPlan& pl, const cd* F, int P, int npts, const double* dpts,
                           double sign) {
  const int nk = ctx->nk;
  const double* kp = ctx->d_kpoints.as<double>();
  cd* part = ctx->d_pp_P.as<cd>();
  if (pl.gemm) {
    // column-major view: G (P x npts, ld P) = F (P x nk, ld P) E (nk x npts, ld nk)
    if (!ctx->blas && cublasCreate(&ctx->blas) != CUBLAS_STATUS_SUCCESS)
      return xatu_fail(ctx, XATU_ERR_CUDA, "cublasCreate failed");
    if (cublasSetStream(ctx->blas, ctx->stream) != CUBLAS_STATUS_SUCCESS)
      return xatu_fail(ctx, XATU_ERR_CUDA, "cublasSetStream failed");
    cd* E = ctx->d_pp_E.as<cd>();
    const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
    for (int c0 = 0; c0 < npts; c0 += pl.chunk) {
      const int nc = std::min(pl.chunk, npts - c0);
      const long long tot = (long long)nk * nc;
      pp_phase_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(nk, nc, kp, dpts + 3 * (size_t)c0, sign,
                                                                              E);
      ctx->launches++;
      XATU_CK_LAUNCH("pp_phase_kernel");
      if (cublasZgemm(ctx->blas, CUBLAS_OP_N, CUBLAS_OP_N, P, nc, nk, &one,
                      reinterpret_cast<const cuDoubleComplex*>(F), P, reinterpret_cast<const cuDoubleComplex*>(E), nk,
                      &zero, reinterpret_cast<cuDoubleComplex*>(part + (size_t)c0 * P), P) != CUBLAS_STATUS_SUCCESS)
        return xatu_fail(ctx, XATU_ERR_CUDA, "cublasZgemm (k-space transform) failed");
    }
    return XATU_OK;
  }
  const dim3 g = pl.grid;
  const int kc = pl.kchunk;
  const size_t sm = pp_kdft_smem_of(pl.PT, pl.NPL, pl.CPW);
  XATU_CK(xatu_raise_smem_limit(pp_kdft_fn(pl.PT, pl.NPL, pl.CPW), sm));
#define PP_LAUNCH(A, B, C)                                                                                 \
  if (pl.PT == A && pl.NPL == B && pl.CPW == C)                                                            \
    pp_kdft_kernel<A, B, C><<<g, 256, sm, ctx->stream>>>(nk, P, kp, F, npts, dpts, sign, kc, part);
  PP_KDFT_VARIANTS(PP_LAUNCH)
#undef PP_LAUNCH
  ctx->launches++;
  XATU_CK_LAUNCH("pp_kdft_kernel");
  return XATU_OK;
}

// Bytes of the pair table F per group of states, and pairs per group: the groups keep both under these bounds.
#define PP_F_BUDGET (512ull << 20)
#define PP_MAX_PAIRS 2000000

extern "C" xatu_status xatu_realspace_amplitude(xatu_ctx* ctx, int nstates, const double* eigvec, int hole_index,
                                                const double* hole_cell, int ncells, const double* cells,
                                                double* out) {
  xatu_status st = pp_check(ctx, nstates, eigvec);
  if (st != XATU_OK) return st;
  if (hole_index < 0 || hole_index >= ctx->natoms || !hole_cell || ncells < 0 || (ncells > 0 && (!cells || !out)))
    return xatu_fail(ctx, XATU_ERR_INVALID, "bad argument");
  if (ncells == 0) return XATU_OK;
  const long long N = pp_dim(ctx);
  const int nk = ctx->nk, norb = ctx->norb, natoms = ctx->natoms;
  const int hoff = ctx->orb_off[hole_index], nho = ctx->orb_off[hole_index + 1] - hoff;
  // electron minus hole cell, as the reference forms eCell - hCell
  std::vector<double> d((size_t)ncells * 3);
  for (int c = 0; c < ncells; c++)
    for (int q = 0; q < 3; q++) d[(size_t)c * 3 + q] = cells[(size_t)c * 3 + q] - hole_cell[q];
  const size_t per_state = (size_t)nk * norb * nho * sizeof(cd);
  size_t group = std::min<size_t>((size_t)nstates, PP_F_BUDGET / per_state);
  group = std::min<size_t>(group, (size_t)PP_MAX_PAIRS / ((size_t)norb * nho));
  group = std::max<size_t>(group, 1);
  const int P0 = (int)group * norb * nho;
  const KdftPlan pl0 = pp_kdft_plan(ctx, P0, ncells);
  XATU_CK(ctx->d_pp_X.ensure((size_t)N * group * sizeof(cd)));
  XATU_CK(ctx->d_pp_A.ensure(per_state * group));
  XATU_CK(ctx->d_pp_B.ensure((size_t)ncells * 3 * sizeof(double) + group * ncells * natoms * sizeof(double)));
  // later (smaller) groups need no more partials (nor phase matrix) than the first
  XATU_CK(ctx->d_pp_P.ensure(pp_kdft_bytes(pl0, P0, ncells)));
  XATU_CK(ctx->d_pp_E.ensure(pp_kdft_ebytes(ctx, pl0)));
  double* dpts = ctx->d_pp_B.as<double>();
  double* dout = dpts + (size_t)ncells * 3;
  XATU_CK(cudaMemcpyAsync(dpts, d.data(), d.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  for (int s0 = 0; s0 < nstates; s0 += (int)group) {
    const int ns = std::min((int)group, nstates - s0);
    const int P = ns * norb * nho;
    const KdftPlan pl = pp_kdft_plan(ctx, P, ncells);
    if (pp_kdft_bytes(pl, P, ncells) > ctx->d_pp_P.bytes || pp_kdft_ebytes(ctx, pl) > ctx->d_pp_E.bytes)
      return xatu_fail(ctx, XATU_ERR_INVALID, "internal: k-space transform partials exceed their buffer");
    XATU_CK(cudaMemcpyAsync(ctx->d_pp_X.p, eigvec + (size_t)2 * N * s0, (size_t)N * ns * sizeof(cd),
                            cudaMemcpyHostToDevice, ctx->stream));
    const long long total = (long long)nk * P;
    pp_rs_pair_kernel<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(
        nk, ctx->nv, ctx->nc, ctx->nb, norb, hoff, nho, ns, N, ctx->d_pp_X.as<cd>(), ctx->d_eigvec.as<cd>(),
        ctx->d_eigvecQ.as<cd>(), ctx->d_pp_A.as<cd>());
    ctx->launches++;
    XATU_CK_LAUNCH("pp_rs_pair_kernel");
    st = pp_kdft(ctx, pl, ctx->d_pp_A.as<cd>(), P, ncells, dpts, 1.0);
    if (st != XATU_OK) return st;
    const long long nout = (long long)ns * ncells * natoms;
    pp_rs_finish_kernel<<<(unsigned)((nout + 255) / 256), 256, 0, ctx->stream>>>(
        ncells, P, pl.nsplit, ns, natoms, ctx->d_orboff.as<int>(), norb, nho, ctx->d_pp_P.as<cd>(), dout);
    ctx->launches++;
    XATU_CK_LAUNCH("pp_rs_finish_kernel");
    XATU_CK(cudaMemcpyAsync(out + (size_t)s0 * ncells * natoms, dout, (size_t)nout * sizeof(double),
                            cudaMemcpyDeviceToHost, ctx->stream));
    // the next group overwrites X, F and the output block
    XATU_CK(cudaStreamSynchronize(ctx->stream));
  }
  return XATU_OK;
}

extern "C" xatu_status xatu_envelope_ft(xatu_ctx* ctx, int nstates, const double* eigvec, int npoints,
                                        const double* points, double* out) {
  xatu_status st = pp_check(ctx, nstates, eigvec);
  if (st != XATU_OK) return st;
  if (npoints < 0 || (npoints > 0 && (!points || !out))) return xatu_fail(ctx, XATU_ERR_INVALID, "bad argument");
  if (npoints == 0) return XATU_OK;
  const long long N = pp_dim(ctx);
  const int nk = ctx->nk;
  const KdftPlan pl = pp_kdft_plan(ctx, nstates, npoints);
  XATU_CK(ctx->d_pp_X.ensure((size_t)N * nstates * sizeof(cd)));
  XATU_CK(ctx->d_pp_B.ensure((size_t)nstates * nk * sizeof(double)));
  XATU_CK(ctx->d_pp_C.ensure(pp_obs_bytes_c(ctx, nstates)));
  XATU_CK(ctx->d_pp_A.ensure((size_t)nk * nstates * sizeof(cd)));
  XATU_CK(ctx->d_pp_D.ensure((size_t)npoints * 3 * sizeof(double) + (size_t)nstates * npoints * sizeof(double)));
  XATU_CK(ctx->d_pp_P.ensure(pp_kdft_bytes(pl, nstates, npoints)));
  XATU_CK(ctx->d_pp_E.ensure(pp_kdft_ebytes(ctx, pl)));
  double* dpts = ctx->d_pp_D.as<double>();
  double* dout = dpts + (size_t)npoints * 3;
  st = pp_state_obs(ctx, nstates, eigvec, false, false);
  if (st != XATU_OK) return st;
  XATU_CK(cudaMemcpyAsync(dpts, points, (size_t)npoints * 3 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  const long long total = (long long)nk * nstates;
  pp_weights_to_f_kernel<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(nk, nstates, ctx->d_pp_B.as<double>(),
                                                                                   ctx->d_pp_A.as<cd>());
  ctx->launches++;
  XATU_CK_LAUNCH("pp_weights_to_f_kernel");
  st = pp_kdft(ctx, pl, ctx->d_pp_A.as<cd>(), nstates, npoints, dpts, -1.0);
  if (st != XATU_OK) return st;
  const long long nout = (long long)nstates * npoints;
  pp_env_finish_kernel<<<(unsigned)((nout + 255) / 256), 256, 0, ctx->stream>>>(npoints, nstates, pl.nsplit,
                                                                                ctx->d_pp_P.as<cd>(), dout);
  ctx->launches++;
  XATU_CK_LAUNCH("pp_env_finish_kernel");
  XATU_CK(cudaMemcpyAsync(out, dout, (size_t)nout * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  return XATU_OK;
}

extern "C" xatu_status xatu_absorption(xatu_ctx* ctx, int nstates, const double* eigval, const double* eigvec,
                                       double w0, double wrange, int nw, double eta, int broadening,
                                       double* sigma_sp, double* sigma_ex, double* vme_ex) {
  if (!ctx) return XATU_ERR_INVALID;
  if (nstates < 0 || nw < 1 || !sigma_sp || !sigma_ex || (nstates > 0 && (!eigval || !eigvec)))
    return xatu_fail(ctx, XATU_ERR_INVALID, "bad argument");
  cudaSetDevice(ctx->device);
  if (!ctx->bands_ok) return xatu_fail(ctx, XATU_ERR_STATE, "bands are not computed");
  if (ctx->custom_basis)
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "absorption needs the full e-h basis (last build used a subset)");
  const long long N = pp_dim(ctx);
  // vcell (skubo_w.f90:69-71): |a1 x a2| in bohr^2, the lattice padded to three rows
  double R[2][3] = {{0, 0, 0}, {0, 0, 0}};
  for (int i = 0; i < 2 && i < ctx->ndim; i++)
    for (int q = 0; q < 3; q++) R[i][q] = ctx->bravais[3 * i + q] / PP_BOHR;
  const double cx = R[0][1] * R[1][2] - R[0][2] * R[1][1];
  const double cy = R[0][2] * R[1][0] - R[0][0] * R[1][2];
  const double cz = R[0][0] * R[1][1] - R[0][1] * R[1][0];
  const double vcell = sqrt(cx * cx + cy * cy + cz * cz);
  XATU_CK(ctx->d_pp_A.ensure((size_t)3 * N * sizeof(cd)));
  if (nstates > 0) XATU_CK(ctx->d_pp_X.ensure((size_t)N * nstates * sizeof(cd)));
  XATU_CK(ctx->d_pp_D.ensure((size_t)nw * 9 * (sizeof(cd) + sizeof(double)) + (size_t)nstates * (sizeof(double) + 3 * sizeof(cd))));
  // complex blocks first, so every block starts on a 16-byte boundary
  cd* dsp = ctx->d_pp_D.as<cd>();
  cd* dvex = dsp + (size_t)nw * 9;
  double* dex = reinterpret_cast<double*>(dvex + (size_t)3 * nstates);
  double* den = dex + (size_t)nw * 9;
  xatu_status st = xatu_vme_enqueue(ctx, ctx->d_pp_A.as<cd>());
  if (st != XATU_OK) return st;
  if (nstates > 0) {
    XATU_CK(cudaMemcpyAsync(ctx->d_pp_X.p, eigvec, (size_t)N * nstates * sizeof(cd), cudaMemcpyHostToDevice,
                            ctx->stream));
    XATU_CK(cudaMemcpyAsync(den, eigval, (size_t)nstates * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    st = xatu_exciton_vme_enqueue(ctx, ctx->d_pp_A.as<cd>(), ctx->d_pp_X.as<cd>(), N, nstates, dvex);
    if (st != XATU_OK) return st;
  }
  AbsParams p;
  p.nk = ctx->nk;
  p.nv = ctx->nv;
  p.nc = ctx->nc;
  p.nb = ctx->nb;
  p.ns = nstates;
  p.nw = nw;
  p.broad = broadening;
  p.N = N;
  p.w0 = w0;
  p.wrange = wrange;
  p.eta = eta / PP_HARTREE;
  p.pref = PP_PI / ((double)ctx->nk * vcell);
  pp_absorption_kernel<<<nw, 256, 0, ctx->stream>>>(p, ctx->d_eigval.as<double>(), ctx->d_pp_A.as<cd>(), den, dvex, dsp,
                                                    dex);
  ctx->launches++;
  XATU_CK_LAUNCH("pp_absorption_kernel");
  XATU_CK(cudaMemcpyAsync(sigma_sp, dsp, (size_t)nw * 9 * sizeof(cd), cudaMemcpyDeviceToHost, ctx->stream));
  XATU_CK(cudaMemcpyAsync(sigma_ex, dex, (size_t)nw * 9 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (vme_ex && nstates > 0)
    XATU_CK(cudaMemcpyAsync(vme_ex, dvex, (size_t)3 * nstates * sizeof(cd), cudaMemcpyDeviceToHost, ctx->stream));
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  return XATU_OK;
}
