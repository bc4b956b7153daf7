// Exciton oscillator strengths (ResultTB::excitonOscillatorStrength,
// ResultTB.cpp:242-298, with exciton_oscillator_strength / get_vme_kernels /
// get_eigen_vme of skubo_w.f90:175-330, 445-628), in atomic units as the
// reference returns them.
//
// vme_kernel: one CTA per k.  For each Cartesian direction it builds in shared
// memory the Bloch kernels of the hopping derivative and of the position
// ("A") operator -- summing only the lower triangle over R (R_z = 0) and filling
// the upper triangle by conjugation, the A kernel as conj(A) + i conj(S'), which
// also replaces its diagonal, exactly as the reference does -- and contracts
// them with the stored band coefficients:
//   vme(n, n') = sum_{a,a'} conj(C_a n) C_a' n' [ H'_aa' + i (e_n A_aa' - e_n' conj(A_a'a)) ]
// for n = conduction, n' = valence; the element the exciton sum uses is
// vme(v, c) = conj(vme(c, v)).
// exciton_vme_kernel: vme_ex(j, s) = sum_i X_is v_j(i), one CTA per (j, s).
#include <cstring>

#include "engine.h"

#define OSC_BOHR 0.52917721067121
#define OSC_HARTREE 27.211385

struct OscParams {
  int nk, norb, nR, nb, nv, nc, natoms;
  int has_overlap;
  int orb_off[XATU_MAX_ATOMS + 1];
  double pos[3 * XATU_MAX_ATOMS];   // atom positions (Angstrom)
};

// Hd (hopping derivative) and A (position) kernels of direction nj at the k whose Bloch phases are in ph:
// lower triangle summed over R (R_z = 0), upper triangle by conjugation, the A kernel's upper triangle as
// conj(A) + i conj(S'), which also replaces its diagonal (skubo_w.f90:445-530).
__device__ void vme_build_kernels(const OscParams& p, int nj, const double* __restrict__ cellsR,
                                  const cd* __restrict__ HR, const cd* __restrict__ SR, const cd* ph, cd* Hd, cd* Ak) {
  const int n = p.norb;
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
    const int a = t / n, a2 = t - a * n;
    if (a2 > a) continue;
    cd hd = mk(0, 0), sd = mk(0, 0);
    if (nj < 2) {
      for (int r = 0; r < p.nR; r++) {
        const double Rc = cellsR[3 * r + nj] / OSC_BOHR;
        const cd f = mk(-Rc * ph[r].y, Rc * ph[r].x);   // i R e^{ik.R}
        hd = hd + f * ((1.0 / OSC_HARTREE) * HR[(int64_t)r * n * n + a * n + a2]);
        const cd sv = p.has_overlap ? mk(SR[(int64_t)r * n * n + a * n + a2].x, 0.0) : mk(a == a2 ? 1.0 : 0.0, 0.0);
        sd = sd + f * sv;
      }
    }
    // A = sum_R e^{ikR} (r_hop + i S'_hop); r_hop holds the orbital position on R index 0 only
    cd ak = mk(-sd.y, sd.x);
    if (a == a2) {
      int atom = 0;
      while (atom + 1 < p.natoms && a >= p.orb_off[atom + 1]) atom++;
      ak = ak + (p.pos[3 * atom + nj] / OSC_BOHR) * ph[0];
    }
    const cd isdc = mk(sd.y, sd.x);   // i conj(S')
    if (a == a2) {
      Hd[a * n + a] = conj(hd);
      Ak[a * n + a] = conj(ak) + isdc;
    } else {
      Hd[a * n + a2] = hd;
      Hd[a2 * n + a] = conj(hd);
      Ak[a * n + a2] = ak;
      Ak[a2 * n + a] = conj(ak) + isdc;
    }
  }
}

extern "C" __global__ void vme_kernel(OscParams p, const double* __restrict__ kpoints, const double* __restrict__ cellsR,
                                      const cd* __restrict__ HR, const cd* __restrict__ SR,
                                      const double* __restrict__ eigval, const cd* __restrict__ eigvec,
                                      cd* __restrict__ vout /* 3 x N, row-major */) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = p.norb;
  const int k = blockIdx.x;
  cd* Hd = reinterpret_cast<cd*>(smem_raw);   // n x n
  cd* Ak = Hd + n * n;                        // n x n
  cd* ph = Ak + n * n;                        // nR
  cd* C = ph + p.nR;                          // nb x n
  double* e = reinterpret_cast<double*>(C + p.nb * n);   // nb
  const double kx = kpoints[3 * k] * OSC_BOHR, ky = kpoints[3 * k + 1] * OSC_BOHR;
  for (int r = threadIdx.x; r < p.nR; r += blockDim.x) {
    double s, c;
    sincos(kx * (cellsR[3 * r] / OSC_BOHR) + ky * (cellsR[3 * r + 1] / OSC_BOHR), &s, &c);
    ph[r] = mk(c, s);
  }
  for (int t = threadIdx.x; t < p.nb * n; t += blockDim.x) C[t] = eigvec[(int64_t)k * p.nb * n + t];
  for (int b = threadIdx.x; b < p.nb; b += blockDim.x) e[b] = eigval[(int64_t)k * p.nb + b] / OSC_HARTREE;
  __syncthreads();
  const int N = p.nk * p.nv * p.nc;
  for (int nj = 0; nj < 3; nj++) {
    vme_build_kernels(p, nj, cellsR, HR, SR, ph, Hd, Ak);
    __syncthreads();
    // one warp per (valence, conduction) pair
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int pr = warp; pr < p.nv * p.nc; pr += nw) {
      const int ic = pr / p.nv, iv = pr - ic * p.nv;
      const int nn = p.nv + ic, nnp = iv;
      const double en = e[nn], enp = e[nnp];
      cd acc = mk(0, 0);
      for (int t = lane; t < n * n; t += 32) {
        const int a = t / n, a2 = t - a * n;
        const cd w = cmulc(C[nn * n + a], C[nnp * n + a2]);   // conj(C_a n) C_a' n'
        const cd A1 = Ak[a * n + a2], A2c = conj(Ak[a2 * n + a]);
        const cd bterm = mk(en * A1.x - enp * A2c.x, en * A1.y - enp * A2c.y);
        const cd term = Hd[a * n + a2] + mk(-bterm.y, bterm.x);
        acc = acc + w * term;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
      }
      if (lane == 0) {
        const int j = k * p.nc * p.nv + ic * p.nv + iv;
        vout[(int64_t)nj * N + j] = conj(acc);
      }
    }
    __syncthreads();
  }
}

// Adjoint of vme_kernel.  With v_j(i) = sum_{a,a'} C_c,a conj(C_v,a') conj(T_aa'),
// T = Hd + i (e_c A - e_v conj(A^T)) (energies in Hartree) and vbar_j(i) = dF/dconj(v_j(i)):
//   cbar_c,a  += sum_a' vbar C_v,a' T_aa'          cbar_v,a' += sum_a conj(vbar) C_c,a conj(T_aa')
//   ebar_c    += 2/Ha Re sum conj(vbar) C_c,a conj(C_v,a') (-i conj(A_aa'))
//   ebar_v    += 2/Ha Re sum conj(vbar) C_c,a conj(C_v,a') ( i A_a'a)
// (added to cbar / ebar of row k), and, for the direct dependence on H(R) through Hd (directions x, y),
//   Om_j(a, a') = sum_states vbar_j conj(C_c,a) C_v,a'
//   gvme[j][k][a][a2] = Om(a, a2) + conj(Om(a2, a)) (a2 < a),  conj(Om(a, a)) (a2 = a),  0 (a2 > a).
extern "C" __global__ void vme_adjoint_kernel(OscParams p, const double* __restrict__ kpoints,
                                              const double* __restrict__ cellsR, const cd* __restrict__ HR,
                                              const cd* __restrict__ SR, const double* __restrict__ eigval,
                                              const cd* __restrict__ eigvec, const cd* __restrict__ vbar,
                                              cd* __restrict__ cbar, double* __restrict__ ebar, cd* __restrict__ gvme) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = p.norb, k = blockIdx.x, nb = p.nb;
  cd* Hd = reinterpret_cast<cd*>(smem_raw);
  cd* Ak = Hd + n * n;
  cd* Om = Ak + n * n;
  cd* ph = Om + n * n;
  cd* C = ph + p.nR;                                  // nb x n
  cd* cacc = C + nb * n;                              // nb x n
  double* e = reinterpret_cast<double*>(cacc + nb * n);
  double* eacc = e + nb;
  __shared__ double red[2][32];
  const double kx = kpoints[3 * k] * OSC_BOHR, ky = kpoints[3 * k + 1] * OSC_BOHR;
  for (int r = threadIdx.x; r < p.nR; r += blockDim.x) {
    double s, c;
    sincos(kx * (cellsR[3 * r] / OSC_BOHR) + ky * (cellsR[3 * r + 1] / OSC_BOHR), &s, &c);
    ph[r] = mk(c, s);
  }
  for (int t = threadIdx.x; t < nb * n; t += blockDim.x) {
    C[t] = eigvec[(int64_t)k * nb * n + t];
    cacc[t] = mk(0, 0);
  }
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    e[b] = eigval[(int64_t)k * nb + b] / OSC_HARTREE;
    eacc[b] = 0.0;
  }
  __syncthreads();
  const int N = p.nk * p.nv * p.nc;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int nj = 0; nj < 3; nj++) {
    vme_build_kernels(p, nj, cellsR, HR, SR, ph, Hd, Ak);
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) Om[t] = mk(0, 0);
    __syncthreads();
    for (int pr = 0; pr < p.nv * p.nc; pr++) {
      const int ic = pr / p.nv, iv = pr - ic * p.nv;
      const int cc = p.nv + ic;
      const double ec = e[cc], ev = e[iv];
      const cd vb = vbar[(int64_t)nj * N + (int64_t)k * p.nc * p.nv + ic * p.nv + iv];
      // T_aa' on the fly
      for (int a = threadIdx.x; a < n; a += blockDim.x) {
        cd sc = mk(0, 0), sv = mk(0, 0);
        for (int a2 = 0; a2 < n; a2++) {
          const cd A1 = Ak[a * n + a2], A2c = conj(Ak[a2 * n + a]);
          const cd bt = mk(ec * A1.x - ev * A2c.x, ec * A1.y - ev * A2c.y);
          const cd T = Hd[a * n + a2] + mk(-bt.y, bt.x);
          sc = sc + C[iv * n + a2] * T;                          // row a of cbar_c
          // column a of cbar_v: sum_a'' conj(vb) C_c,a'' conj(T_a'' a)
          const cd B1 = Ak[a2 * n + a], B2c = conj(Ak[a * n + a2]);
          const cd bt2 = mk(ec * B1.x - ev * B2c.x, ec * B1.y - ev * B2c.y);
          const cd T2 = Hd[a2 * n + a] + mk(-bt2.y, bt2.x);
          sv = sv + C[cc * n + a2] * conj(T2);
        }
        cacc[cc * n + a] = cacc[cc * n + a] + vb * sc;
        cacc[iv * n + a] = cacc[iv * n + a] + conj(vb) * sv;
      }
      double sce = 0.0, sve = 0.0;
      for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
        const int a = t / n, a2 = t - a * n;
        const cd w = C[cc * n + a] * conj(C[iv * n + a2]);      // C_c,a conj(C_v,a')
        const cd q = conj(vb) * w;
        const cd A = Ak[a * n + a2], At = Ak[a2 * n + a];
        // (-i conj(A)) and (i A^T)
        const cd mc = mk(-A.y, -A.x);
        const cd mv = mk(-At.y, At.x);
        sce += (q * mc).x;
        sve += (q * mv).x;
        Om[t] = Om[t] + vb * cmulc(C[cc * n + a], C[iv * n + a2]);  // vbar conj(C_c,a) C_v,a'
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        sce += __shfl_xor_sync(0xffffffffu, sce, o);
        sve += __shfl_xor_sync(0xffffffffu, sve, o);
      }
      if (lane == 0) {
        red[0][warp] = sce;
        red[1][warp] = sve;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double a0 = 0.0, a1 = 0.0;
        for (int q = 0; q < nwarps; q++) {
          a0 += red[0][q];
          a1 += red[1][q];
        }
        eacc[cc] += 2.0 / OSC_HARTREE * a0;
        eacc[iv] += 2.0 / OSC_HARTREE * a1;
      }
      __syncthreads();
    }
    if (nj < 2) {
      for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
        const int a = t / n, a2 = t - a * n;
        cd gv = mk(0, 0);
        if (a2 < a) gv = Om[a * n + a2] + conj(Om[a2 * n + a]);
        else if (a2 == a) gv = conj(Om[a * n + a]);
        gvme[((int64_t)nj * p.nk + k) * n * n + t] = gv;
      }
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < nb * n; t += blockDim.x) cbar[(int64_t)k * nb * n + t] = cbar[(int64_t)k * nb * n + t] + cacc[t];
  for (int b = threadIdx.x; b < nb; b += blockDim.x) ebar[(int64_t)k * nb + b] += eacc[b];
}

// Direct H(R) part: G(R)_{a,a2} += sum_{j = x, y} (-2 i R_j / Ha) sum_k conj(gvme[j][k][a][a2]) e^{-i k.R}
// (R in Bohr).  grid (nR, ceil(norb^2 / 256)).
extern "C" __global__ void vme_hop_kernel(int nk, int norb, const double* __restrict__ kpoints,
                                          const double* __restrict__ cellsR, const cd* __restrict__ gvme,
                                          cd* __restrict__ G) {
  const int r = blockIdx.x, n2 = norb * norb;
  const int ab = blockIdx.y * blockDim.x + threadIdx.x;
  __shared__ cd ph[256];
  const double Rx = cellsR[3 * r], Ry = cellsR[3 * r + 1], Rz = cellsR[3 * r + 2];
  cd s0 = mk(0, 0), s1 = mk(0, 0);
  for (int base = 0; base < nk; base += 256) {
    const int kk = base + threadIdx.x;
    if (kk < nk) {
      double sn, cs;
      sincos(kpoints[3 * kk] * Rx + kpoints[3 * kk + 1] * Ry + kpoints[3 * kk + 2] * Rz, &sn, &cs);
      ph[threadIdx.x] = mk(cs, -sn);
    }
    __syncthreads();
    if (ab < n2) {
      const int m = min(256, nk - base);
      for (int q = 0; q < m; q++) {
        s0 = s0 + conj(gvme[((int64_t)0 * nk + base + q) * n2 + ab]) * ph[q];
        s1 = s1 + conj(gvme[((int64_t)1 * nk + base + q) * n2 + ab]) * ph[q];
      }
    }
    __syncthreads();
  }
  if (ab < n2) {
    const double f0 = -2.0 * (Rx / OSC_BOHR) / OSC_HARTREE, f1 = -2.0 * (Ry / OSC_BOHR) / OSC_HARTREE;
    // (-2 i R_j / Ha) z = (2 R_j / Ha) (z.y, -z.x) with f = -2 R_j / Ha: f * (-z.y, z.x)
    const cd add = mk(f0 * (-s0.y) + f1 * (-s1.y), f0 * s0.x + f1 * s1.x);
    G[(int64_t)r * n2 + ab] = G[(int64_t)r * n2 + ab] + add;
  }
}

extern "C" __global__ void exciton_vme_kernel(const cd* __restrict__ v, const cd* __restrict__ X, int N, int ns,
                                              cd* __restrict__ out /* 3 x ns, column-major */) {
  const int nj = blockIdx.x % 3, s = blockIdx.x / 3;
  cd acc = mk(0, 0);
  for (int i = threadIdx.x; i < N; i += blockDim.x) acc = acc + X[(int64_t)s * N + i] * v[(int64_t)nj * N + i];
  __shared__ double rr[32], ri[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
  }
  if ((threadIdx.x & 31) == 0) {
    rr[threadIdx.x >> 5] = acc.x;
    ri[threadIdx.x >> 5] = acc.y;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      a += rr[w];
      b += ri[w];
    }
    out[(int64_t)s * 3 + nj] = mk(a, b);
  }
}

static OscParams osc_params(const xatu_ctx* ctx) {
  OscParams p;
  memset(&p, 0, sizeof(p));
  p.nk = ctx->nk;
  p.norb = ctx->norb;
  p.nR = ctx->nR;
  p.nb = ctx->nb;
  p.nv = ctx->nv;
  p.nc = ctx->nc;
  p.natoms = ctx->natoms;
  p.has_overlap = ctx->has_overlap ? 1 : 0;
  for (int a = 0; a <= ctx->natoms; a++) p.orb_off[a] = ctx->orb_off[a];
  for (int a = 0; a < ctx->natoms; a++)
    for (int d = 0; d < 3; d++) p.pos[3 * a + d] = ctx->motif[4 * a + d];
  return p;
}

xatu_status xatu_exciton_vme_enqueue(xatu_ctx* ctx, const cd* v, const cd* X, long long N, int ns, cd* out) {
  exciton_vme_kernel<<<3 * ns, 256, 0, ctx->stream>>>(v, X, (int)N, ns, out);
  ctx->launches++;
  XATU_CK_LAUNCH("exciton_vme_kernel");
  return XATU_OK;
}

// Velocity matrix elements of every e-h state of the full basis into out (3 x N, row-major).
xatu_status xatu_vme_enqueue(xatu_ctx* ctx, cd* out) {
  const OscParams p = osc_params(ctx);
  const size_t smem = (2 * (size_t)p.norb * p.norb + p.nR + (size_t)p.nb * p.norb) * sizeof(cd) + p.nb * sizeof(double);
  XATU_CK(xatu_raise_smem_limit((const void*)vme_kernel, smem));
  vme_kernel<<<ctx->nk, 256, smem, ctx->stream>>>(p, ctx->d_kpoints.as<double>(), ctx->d_cellsR.as<double>(),
                                                  ctx->d_HR.as<cd>(), ctx->has_overlap ? ctx->d_SR.as<cd>() : nullptr,
                                                  ctx->d_eigval.as<double>(), ctx->d_eigvec.as<cd>(), out);
  ctx->launches++;
  XATU_CK_LAUNCH("vme_kernel");
  return XATU_OK;
}

// Adds the VME adjoint of vbar (N x 3, column-major) to cbar / ebar (nk x nb x norb / nk x nb) and its
// direct H(R) part to G (nR x norb x norb); gvme: scratch of 2 x nk x norb^2.
xatu_status xatu_vme_adjoint_enqueue(xatu_ctx* ctx, const cd* vbar, cd* cbar, double* ebar, cd* gvme, cd* G) {
  const OscParams p = osc_params(ctx);
  const int n = p.norb;
  const size_t smem = (3 * (size_t)n * n + p.nR + 2 * (size_t)p.nb * n) * sizeof(cd) + 2 * p.nb * sizeof(double);
  XATU_CK(xatu_raise_smem_limit((const void*)vme_adjoint_kernel, smem));
  vme_adjoint_kernel<<<ctx->nk, 256, smem, ctx->stream>>>(p, ctx->d_kpoints.as<double>(), ctx->d_cellsR.as<double>(),
                                                          ctx->d_HR.as<cd>(),
                                                          ctx->has_overlap ? ctx->d_SR.as<cd>() : nullptr,
                                                          ctx->d_eigval.as<double>(), ctx->d_eigvec.as<cd>(), vbar,
                                                          cbar, ebar, gvme);
  ctx->launches++;
  XATU_CK_LAUNCH("vme_adjoint_kernel");
  if (!G) return XATU_OK;
  return xatu_vme_hop_enqueue(ctx, gvme, G);
}

// G (nR x norb x norb) += the direct H(R) part of the VME adjoint from gvme (vme_adjoint_kernel).
xatu_status xatu_vme_hop_enqueue(xatu_ctx* ctx, const cd* gvme, cd* G) {
  const int n = ctx->norb;
  dim3 g(ctx->nR, (unsigned)((n * n + 255) / 256));
  vme_hop_kernel<<<g, 256, 0, ctx->stream>>>(ctx->nk, n, ctx->d_kpoints.as<double>(), ctx->d_cellsR.as<double>(), gvme,
                                             G);
  ctx->launches++;
  XATU_CK_LAUNCH("vme_hop_kernel");
  return XATU_OK;
}

extern "C" xatu_status xatu_oscillator_strength(xatu_ctx* ctx, int nstates, const double* eigvec, double* vme_ex) {
  if (!ctx || !eigvec || !vme_ex || nstates < 1) return xatu_fail(ctx, XATU_ERR_INVALID, "bad argument");
  cudaSetDevice(ctx->device);
  if (!ctx->bands_ok) return xatu_fail(ctx, XATU_ERR_STATE, "bands are not computed");
  if (ctx->custom_basis)
    return xatu_fail(ctx, XATU_ERR_UNSUPPORTED, "oscillator strengths need the full e-h basis (last build used a subset)");
  if (nstates > ctx->N) return xatu_fail(ctx, XATU_ERR_INVALID, "nstates larger than the BSE dimension");
  const long long N = ctx->N;
  const size_t vbytes = (size_t)3 * N * sizeof(cd);
  const size_t xbytes = (size_t)N * nstates * sizeof(cd);
  XATU_CK(ctx->dv_R.ensure(vbytes));
  XATU_CK(ctx->dv_tmp.ensure(xbytes + 64 * (size_t)nstates));
  XATU_CK(ctx->dv_small.ensure((size_t)3 * nstates * sizeof(cd)));
  xatu_status st = xatu_vme_enqueue(ctx, ctx->dv_R.as<cd>());
  if (st != XATU_OK) return st;
  XATU_CK(cudaMemcpyAsync(ctx->dv_tmp.p, eigvec, xbytes, cudaMemcpyHostToDevice, ctx->stream));
  st = xatu_exciton_vme_enqueue(ctx, ctx->dv_R.as<cd>(), ctx->dv_tmp.as<cd>(), N, nstates, ctx->dv_small.as<cd>());
  if (st != XATU_OK) return st;
  XATU_CK(cudaMemcpyAsync(vme_ex, ctx->dv_small.p, (size_t)3 * nstates * sizeof(cd), cudaMemcpyDeviceToHost,
                          ctx->stream));
  XATU_CK(cudaStreamSynchronize(ctx->stream));
  return XATU_OK;
}
