// Band solve for the band window only (ExcitonTB::initializeResultsH0,
// ExcitonTB.cpp:737-758, without overlap matrices): for every k of the
// exciton basis the Bloch Hamiltonian H(k) = sum_R H(R) e^{i k.R} (triangular
// storage symmetrised as SystemTB::hamiltonian, SystemTB.cpp:69-72) is
// diagonalised for the eigenpairs of the band list only (ranks band_list[b]
// in ascending order of energy, ExcitonTB.cpp:741-742), and each eigenvector
// gets its global phase fixed (column sum real positive, ExcitonTB::fixGlobalPhase,
// ExcitonTB.cpp:673-683).
//
// One warp per k point: the H(R) blocks are staged once per CTA (cp.async,
// double-buffered) and accumulated by every warp with its own Bloch phases
// into the packed lower triangle of H(k) (row r at r(r+1)/2; 4 KB per warp at
// 22 orbitals, so that up to 25 warps fit one SM and a mesh of 3600 k points
// runs in one wave); then Householder reduction to real tridiagonal form in
// the warp (one row of the lower triangle per lane), Sturm-sequence multisection for the wanted
// ranks (a group of lanes per eigenvalue), inverse iteration with cluster
// orthonormalisation for the eigenvectors (one lane per eigenvector), and the
// back-transformation by the stored reflectors.  The algorithms are those of
// eigh_small.cuh at warp scale.  Models with overlap matrices use the full
// band solve (bands.cu), which orthogonalises with all eigenpairs of S(k).
#include "bands.cuh"
#include "eigh_small.cuh"

// Largest warps per CTA of each instantiation: 25 for the 4-band window (72 registers; 3600 k points fill
// 148 SMs in one wave), 8 for the wider windows (128 and 255 registers).
template <int NBS>
struct BsMaxW {
  static constexpr int value = NBS == 4 ? 25 : 8;
};

// Packed lower triangle: element (r, c), c <= r.
__device__ __forceinline__ int bs_tri(int r, int c) { return ((r * (r + 1)) >> 1) + c; }

__device__ __forceinline__ void ts_cp16_bs(cd* dst, const cd* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

// Per-warp shared memory.  Arrays live in phases and share space where their phases do not overlap:
// the Bloch phases (H(k) sum) with the inverse-iteration factors, the reflector v and p (reduction) with
// the tridiagonal eigenvectors Z, e^2 (multisection) with the cluster Gram matrix (inverse iteration).
struct BsLayout {
  size_t stage;      // two staged H(R) blocks
  size_t per_warp;
  size_t oR1, oU2, oTau, oD, oE, oU3, oLam, oPM, oInt;   // offsets from the warp's base; A at 0
};

__host__ __device__ inline size_t bs_max(size_t a, size_t b) { return a > b ? a : b; }

__host__ __device__ inline BsLayout bs_layout(int n, int nR, int nbs) {
  BsLayout L;
  L.stage = (size_t)2 * n * n * sizeof(cd);
  size_t w = (size_t)n * (n + 1) / 2 * sizeof(cd);                                    // A, packed lower triangle
  L.oR1 = w;
  w += bs_max((size_t)nR * sizeof(cd), (size_t)4 * n * nbs * sizeof(double));         // phases | LU factors
  L.oU2 = w;
  w += bs_max((size_t)2 * n * sizeof(cd), (size_t)n * nbs * sizeof(double));         // v, p | Z
  L.oTau = w;
  w += (size_t)n * sizeof(cd);                                                        // tau
  L.oD = w;
  w += (size_t)n * sizeof(double);                                                    // d
  L.oE = w;
  w += (size_t)n * sizeof(double);                                                    // e
  L.oU3 = w;
  w += bs_max((size_t)n * sizeof(double), (size_t)nbs * nbs * sizeof(double));        // e^2 | Gram
  L.oLam = w;
  w += (size_t)nbs * sizeof(double);                                                  // lam
  L.oPM = w;
  w += (size_t)n * sizeof(unsigned);                                                  // row-swap masks
  w = (w + 15) / 16 * 16;
  L.oInt = w;
  w += (size_t)3 * nbs * sizeof(int) + 16;                                            // order, clusters, flags
  L.per_warp = (w + 15) / 16 * 16;
  return L;
}

template <int NBS>
__global__ void __launch_bounds__(BsMaxW<NBS>::value * 32)
band_select_kernel(BandParams bp, const double* __restrict__ kpoints, const double* __restrict__ cellsR,
                   const cd* __restrict__ HR, double* __restrict__ eigval, cd* __restrict__ eigvec,
                   int* __restrict__ status, int wpc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = bp.norb, nR = bp.nR, nb = bp.nb, nn = n * n;
  const BsLayout Ly = bs_layout(n, nR, NBS);
  const int np = n * (n + 1) / 2;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k = blockIdx.x * wpc + warp;
  const bool kval = k < bp.nk;
  cd* HRs = reinterpret_cast<cd*>(smem_raw);   // [2][n * n]
  unsigned char* wb = smem_raw + Ly.stage + (size_t)warp * Ly.per_warp;
  cd* A = reinterpret_cast<cd*>(wb);                           // packed lower triangle (bs_tri)
  cd* ph = reinterpret_cast<cd*>(wb + Ly.oR1);                 // Bloch phases (H(k) sum only)
  double* RI = reinterpret_cast<double*>(wb + Ly.oR1);         // [n][NBS] LU factors (inverse iteration only)
  double* DU = RI + n * NBS;
  double* DU2 = DU + n * NBS;
  double* FM = DU2 + n * NBS;
  cd* sv = reinterpret_cast<cd*>(wb + Ly.oU2);                 // reflector v, p (reduction only)
  cd* sp = sv + n;
  double* Z = reinterpret_cast<double*>(wb + Ly.oU2);          // n x NBS (after the multisection)
  cd* stau = reinterpret_cast<cd*>(wb + Ly.oTau);
  double* sd = reinterpret_cast<double*>(wb + Ly.oD);
  double* se = reinterpret_cast<double*>(wb + Ly.oE);
  double* se2 = reinterpret_cast<double*>(wb + Ly.oU3);        // multisection only
  double* G = reinterpret_cast<double*>(wb + Ly.oU3);          // NBS x NBS (inverse iteration only)
  double* lam = reinterpret_cast<double*>(wb + Ly.oLam);
  unsigned* PM = reinterpret_cast<unsigned*>(wb + Ly.oPM);
  int* ord = reinterpret_cast<int*>(wb + Ly.oInt);   // slots in ascending rank
  int* cl = ord + NBS;
  int* flg = cl + NBS;
  const double eps = 2.220446049250313e-16;

  // ---- Bloch phases and H(k) = sum_R H(R) e^{i k.R}, H(R) staged per CTA
  const double kx = kval ? kpoints[3 * k] + bp.shift[0] : 0.0;
  const double ky = kval ? kpoints[3 * k + 1] + bp.shift[1] : 0.0;
  const double kz = kval ? kpoints[3 * k + 2] + bp.shift[2] : 0.0;
  for (int r = lane; r < nR; r += 32) {
    double sn, cs;
    sincos(kx * cellsR[3 * r] + ky * cellsR[3 * r + 1] + kz * cellsR[3 * r + 2], &sn, &cs);
    ph[r] = mk(cs, sn);
  }
  for (int t = lane; t < np; t += 32) A[t] = mk(0, 0);
  // (row, column) of this lane's first packed entry; the lane then steps 32 entries at a time
  int r0 = (int)((sqrt(8.0 * lane + 1.0) - 1.0) * 0.5);
  while ((r0 + 1) * (r0 + 2) / 2 <= lane) r0++;
  while (r0 * (r0 + 1) / 2 > lane) r0--;
  const int c0 = lane - r0 * (r0 + 1) / 2;
  const bool tri = bp.triangular;
  for (int t = threadIdx.x; t < nn; t += blockDim.x) ts_cp16_bs(HRs + t, HR + t);
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  for (int r = 0; r < nR; r++) {
    cd* cur = HRs + (r & 1) * nn;
    if (r + 1 < nR) {
      cd* nxt = HRs + ((r + 1) & 1) * nn;
      for (int t = threadIdx.x; t < nn; t += blockDim.x) ts_cp16_bs(nxt + t, HR + (size_t)(r + 1) * nn + t);
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 1;\n" ::: "memory");
    __syncthreads();
    const cd f = ph[r];
    // lower triangle of H(k); in triangular storage H(k) = h + h^H (h the lower-triangular sum with half its
    // diagonal): entry (i, j) takes h_ij + conj(h_ji), the diagonal the real part of h_ii
    int i = r0, j = c0;
    for (int t = lane; t < np; t += 32) {
      const cd a = cur[i * n + j] * f;
      cd add;
      if (!tri) add = a;
      else if (i == j) add = mk(a.x, 0.0);
      else add = a + conj(cur[j * n + i] * f);
      A[t] = A[t] + add;
      j += 32;
      while (j > i) {
        j -= i + 1;
        i++;
      }
    }
    __syncthreads();
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  if (!kval) return;   // no CTA-wide barrier below this point
  __syncwarp();
  if (!tri)
    for (int i = lane; i < n; i += 32) A[bs_tri(i, i)].y = 0.0;
  __syncwarp();
  {
    bool fin = true;
    for (int t = lane; t < np; t += 32) fin = fin && isfinite(A[t].x) && isfinite(A[t].y);
    if (!__all_sync(0xffffffffu, fin)) {
      if (lane == 0) atomicOr(status, XATU_DEVERR_NAN);
      return;
    }
  }

  // ---- Householder reduction (lower triangle; reflector j kept in column j below row j+1)
  for (int j = 0; j < n - 1; j++) {
    const int L = n - j - 1;
    double s = 0.0;
    for (int i = 1 + lane; i < L; i += 32) s += nrm2(A[bs_tri(j + 1 + i, j)]);
    s = heev_wsum(s);
    const cd al = A[bs_tri(j + 1, j)];
    cd tau = mk(0, 0), scal = mk(0, 0);
    double beta = al.x;
    const bool on = (s > 0.0 || al.y != 0.0);
    if (on) {
      beta = -copysign(sqrt(nrm2(al) + s), al.x);
      const double rb = 1.0 / beta;
      tau = mk((beta - al.x) * rb, -al.y * rb);
      const cd den = mk(al.x - beta, al.y);
      const double rdn = 1.0 / nrm2(den);
      scal = mk(den.x * rdn, -den.y * rdn);
    }
    for (int i = lane; i < L; i += 32) {
      cd vi = (i == 0) ? mk(1.0, 0.0) : (on ? A[bs_tri(j + 1 + i, j)] * scal : mk(0, 0));
      sv[i] = vi;
      if (i >= 1) A[bs_tri(j + 1 + i, j)] = vi;
    }
    if (lane == 0) {
      stau[j] = tau;
      se[j] = beta;
      sd[j] = A[bs_tri(j, j)].x;
    }
    __syncwarp();
    if (!on) continue;
    for (int i = lane; i < L; i += 32) {
      const int gr = j + 1 + i;
      cd acc0 = mk(0, 0), acc1 = mk(0, 0);
      int l = 0;
      for (; l + 1 < L; l += 2) {
        const int g0 = j + 1 + l, g1 = g0 + 1;
        cd a0 = A[l <= i ? bs_tri(gr, g0) : bs_tri(g0, gr)];
        if (l > i) a0.y = -a0.y;
        cd a1 = A[l + 1 <= i ? bs_tri(gr, g1) : bs_tri(g1, gr)];
        if (l + 1 > i) a1.y = -a1.y;
        acc0 = acc0 + a0 * sv[l];
        acc1 = acc1 + a1 * sv[l + 1];
      }
      if (l < L) {
        const int g0 = j + 1 + l;
        cd a0 = A[l <= i ? bs_tri(gr, g0) : bs_tri(g0, gr)];
        if (l > i) a0.y = -a0.y;
        acc0 = acc0 + a0 * sv[l];
      }
      sp[i] = tau * (acc0 + acc1);
    }
    __syncwarp();
    double sx = 0.0, sy = 0.0;
    for (int i = lane; i < L; i += 32) {
      const cd t = cmulc(sv[i], sp[i]);
      sx += t.x;
      sy += t.y;
    }
    sx = heev_wsum(sx);
    sy = heev_wsum(sy);
    const double K = 0.5 * (tau.x * sx + tau.y * sy);
    for (int i = lane; i < L; i += 32) {
      const cd vi = sv[i], wi = sp[i] - K * vi;
      cd* Ar = A + bs_tri(j + 1 + i, j + 1);
      for (int l = 0; l <= i; l++) {
        const cd vl = sv[l], wl = sp[l] - K * vl;
        Ar[l] = Ar[l] - (vi * conj(wl) + wi * conj(vl));
      }
    }
    __syncwarp();
  }
  if (lane == 0) {
    sd[n - 1] = A[bs_tri(n - 1, n - 1)].x;
    se[n - 1] = 0.0;
  }
  __syncwarp();
  double lo = INFINITY, hi = -INFINITY, e2max = 0.0;
  for (int i = lane; i < n; i += 32) {
    se2[i] = se[i] * se[i];
    const double r = (i > 0 ? fabs(se[i - 1]) : 0.0) + fabs(se[i]);
    lo = fmin(lo, sd[i] - r);
    hi = fmax(hi, sd[i] + r);
    e2max = fmax(e2max, se[i] * se[i]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    e2max = fmax(e2max, __shfl_xor_sync(0xffffffffu, e2max, o));
  }
  __syncwarp();
  const double tnorm = fmax(fmax(fabs(lo), fabs(hi)), 1e-100);
  const double pivmin = 1e-290 * fmax(1.0, e2max);
  const double fudge = 4.0 * (n + 1) * eps * tnorm + 4.0 * pivmin;
  const double gl = lo - fudge, gu = hi + fudge;

  // ---- multisection: group of GS lanes per selected rank, two shifts per lane
  constexpr int GS = 32 / NBS;
  {
    const int grp = lane / GS, gln = lane % GS;
    const int b = grp;
    const int rank = b < nb ? bp.band_list[b] : 0;
    double a = gl, bb = gu;
    bool done = b >= nb;
    for (int it = 0; it < 96; it++) {
      const double w = bb - a;
      if (!(w > fmax(2.0 * eps * fmax(fabs(a), fabs(bb)), fmax(0.5 * eps * tnorm, pivmin)))) done = true;
      if (__all_sync(0xffffffffu, done)) break;
      const double den = 1.0 / (2 * GS + 1);
      const double s0 = a + w * (double)(gln + 1) * den, s1 = a + w * (double)(gln + 1 + GS) * den;
      int c0, c1;
      heev_sturm2(sd, se2, n, s0, s1, pivmin, c0, c1);
      double na = (c1 <= rank) ? s1 : ((c0 <= rank) ? s0 : -INFINITY);
      double nbv = (c0 > rank) ? s0 : ((c1 > rank) ? s1 : INFINITY);
#pragma unroll
      for (int o = GS / 2; o > 0; o >>= 1) {
        na = fmax(na, __shfl_xor_sync(0xffffffffu, na, o));
        nbv = fmin(nbv, __shfl_xor_sync(0xffffffffu, nbv, o));
      }
      if (!done) {
        const double a2 = fmax(a, na), b2 = fmin(bb, nbv);
        if (!(a2 < b2)) {
          a = bb = 0.5 * (a + bb);
          done = true;
        } else if (a2 == a && b2 == bb) {
          done = true;
        } else {
          a = a2;
          bb = b2;
        }
      }
    }
    if (gln == 0 && b < nb) lam[b] = 0.5 * (a + bb);
  }
  __syncwarp();
  // slots in ascending rank, clusters of close eigenvalues
  if (lane == 0) {
    for (int b = 0; b < nb; b++) ord[b] = b;
    for (int b = 1; b < nb; b++) {
      const int x = ord[b];
      int q = b - 1;
      while (q >= 0 && bp.band_list[ord[q]] > bp.band_list[x]) {
        ord[q + 1] = ord[q];
        q--;
      }
      ord[q + 1] = x;
    }
    const double ortol = 1e-3 * tnorm;
    int multi = 0;
    for (int q = 0; q < nb; q++) {
      cl[q] = (q > 0 && lam[ord[q]] - lam[ord[q - 1]] <= ortol) ? cl[q - 1] : q;
      multi |= cl[q] != q;
    }
    flg[0] = multi;
  }
  for (int t = lane; t < n * NBS; t += 32) Z[t] = heev_start(t / NBS, t % NBS);
  __syncwarp();

  // ---- inverse iteration (lane q < nb: the q-th slot in rank order), Z columns in rank order
  const double tiny = eps * tnorm;
  for (int iter = 0; iter < 3; iter++) {
    const int q = lane;
    const bool act = q < nb;
    if (iter == 0) {
      const double lj = act ? lam[ord[q]] : lam[ord[0]];
      double cur_d = sd[0] - lj, cur_u = (n > 1) ? se[0] : 0.0;
      for (int i = 0; i < n - 1; i++) {
        const double sub = se[i];
        double nd = sd[i + 1] - lj, nu = (i < n - 2) ? se[i + 1] : 0.0;
        double piv, up, u2 = 0.0, f, rp;
        const bool sw = fabs(cur_d) < fabs(sub);
        if (!sw) {
          piv = cur_d;
          if (fabs(piv) < tiny) piv = (piv < 0.0) ? -tiny : tiny;
          rp = 1.0 / piv;
          f = sub * rp;
          nd -= f * cur_u;
          up = cur_u;
        } else {
          piv = sub;
          rp = 1.0 / piv;
          f = cur_d * rp;
          const double tmp = nd;
          nd = cur_u - f * tmp;
          if (i < n - 2) {
            u2 = nu;
            nu = -f * u2;
          }
          up = tmp;
        }
        const unsigned msk = __ballot_sync(0xffffffffu, sw);
        if (act) {
          RI[i * NBS + q] = rp;
          DU[i * NBS + q] = up;
          DU2[i * NBS + q] = u2;
          FM[i * NBS + q] = f;
        }
        if (lane == 0) PM[i] = msk;
        cur_d = nd;
        cur_u = nu;
      }
      if (fabs(cur_d) < tiny) cur_d = (cur_d < 0.0) ? -tiny : tiny;
      if (act) RI[(n - 1) * NBS + q] = 1.0 / cur_d;
      __syncwarp();
    }
    if (act) {
      double nn2 = 0.0;
      for (int i = 0; i < n; i++) nn2 += Z[i * NBS + q] * Z[i * NBS + q];
      const double f0 = nn2 > 0.0 ? 1.0 / sqrt(nn2) : 1.0;
      double xi = Z[q] * f0;
      for (int i = 0; i < n - 1; i++) {
        double xn = Z[(i + 1) * NBS + q] * f0;
        const double f = FM[i * NBS + q];
        if ((PM[i] >> lane) & 1u) {
          const double t = xi;
          xi = xn;
          xn = t - f * xn;
        } else {
          xn -= f * xi;
        }
        Z[i * NBS + q] = xi;
        xi = xn;
      }
      double x2 = 0.0, x1 = xi * RI[(n - 1) * NBS + q];
      Z[(n - 1) * NBS + q] = x1;
      nn2 = x1 * x1;
      for (int i = n - 2; i >= 0; i--) {
        const double x0 = (Z[i * NBS + q] - DU[i * NBS + q] * x1 - DU2[i * NBS + q] * x2) * RI[i * NBS + q];
        Z[i * NBS + q] = x0;
        nn2 += x0 * x0;
        x2 = x1;
        x1 = x0;
      }
      const double f1 = 1.0 / sqrt(nn2);
      for (int i = 0; i < n; i++) Z[i * NBS + q] *= f1;
    }
    __syncwarp();
    if (!flg[0]) continue;
    // Cholesky QR of each cluster (lane 0; nb <= NBS is small)
    for (int t = lane; t < nb * nb; t += 32) {
      const int r = t / nb, c = t % nb;
      if (c <= r && cl[r] == cl[c]) {
        double g = 0.0;
        for (int i = 0; i < n; i++) g += Z[i * NBS + r] * Z[i * NBS + c];
        G[r * NBS + c] = g;
      }
    }
    __syncwarp();
    if (lane == 0) {
      for (int c = 0; c < nb; c++) {
        double pv = G[c * NBS + c];
        for (int l = cl[c]; l < c; l++) pv -= G[c * NBS + l] * G[c * NBS + l];
        if (!(pv > 1e-24)) {
          atomicOr(status, XATU_DEVERR_NOCONV);
          pv = 1e-24;
        }
        const double lc = sqrt(pv);
        G[c * NBS + c] = lc;
        for (int r = c + 1; r < nb; r++) {
          if (cl[r] != cl[c]) continue;
          double v = G[r * NBS + c];
          for (int l = cl[c]; l < c; l++) v -= G[r * NBS + l] * G[c * NBS + l];
          G[r * NBS + c] = v / lc;
        }
      }
    }
    __syncwarp();
    for (int i = lane; i < n; i += 32) {
      double* zr = Z + i * NBS;
      for (int c = 0; c < nb; c++) {
        double v = zr[c];
        for (int l = cl[c]; l < c; l++) v -= zr[l] * G[c * NBS + l];
        zr[c] = v / G[c * NBS + c];
      }
    }
    __syncwarp();
  }

  // ---- back-transformation y = H_0 ... H_{n-2} z, then the global phase, for every selected slot
  constexpr int PER = XATU_MAX_ORB / 32;
  cd y[PER][NBS];
#pragma unroll
  for (int pq = 0; pq < PER; pq++)
#pragma unroll
    for (int q = 0; q < NBS; q++) {
      const int row = lane + 32 * pq;
      y[pq][q] = mk((row < n && q < nb) ? Z[row * NBS + q] : 0.0, 0.0);
    }
  for (int r = n - 2; r >= 0; r--) {
    const cd tau = stau[r];
    if (tau.x == 0.0 && tau.y == 0.0) continue;
    cd vr[PER];
#pragma unroll
    for (int pq = 0; pq < PER; pq++) {
      const int row = lane + 32 * pq;
      vr[pq] = (row < n && row > r) ? (row == r + 1 ? mk(1.0, 0.0) : A[bs_tri(row, r)]) : mk(0, 0);
    }
    double sx[NBS], sy[NBS];
#pragma unroll
    for (int q = 0; q < NBS; q++) {
      sx[q] = 0.0;
      sy[q] = 0.0;
#pragma unroll
      for (int pq = 0; pq < PER; pq++) {
        const cd t = cmulc(vr[pq], y[pq][q]);
        sx[q] += t.x;
        sy[q] += t.y;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int q = 0; q < NBS; q++) {
        sx[q] += __shfl_xor_sync(0xffffffffu, sx[q], o);
        sy[q] += __shfl_xor_sync(0xffffffffu, sy[q], o);
      }
#pragma unroll
    for (int q = 0; q < NBS; q++) {
      const cd ts = tau * mk(sx[q], sy[q]);
#pragma unroll
      for (int pq = 0; pq < PER; pq++) y[pq][q] = y[pq][q] - ts * vr[pq];
    }
  }
#pragma unroll
  for (int q = 0; q < NBS; q++) {
    if (q >= nb) continue;
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int pq = 0; pq < PER; pq++) {
      sr += y[pq][q].x;
      si += y[pq][q].y;
    }
    sr = heev_wsum(sr);
    si = heev_wsum(si);
    double sn, cs;
    sincos(-atan2(si, sr), &sn, &cs);
    const cd f = mk(cs, sn);
    const int b = ord[q];
    cd* out = eigvec + ((int64_t)k * nb + b) * n;
#pragma unroll
    for (int pq = 0; pq < PER; pq++) {
      const int row = lane + 32 * pq;
      if (row < n) out[row] = y[pq][q] * f;
    }
    if (lane == 0) eigval[(int64_t)k * nb + b] = lam[b];
  }
}

// The fast path covers models without overlap matrices, norb <= XATU_MAX_ORB and at most 16 bands.
extern "C" bool xatu_band_select_supported(int norb, int nb, int has_overlap) {
  return !has_overlap && norb >= 2 && norb <= XATU_MAX_ORB && nb >= 1 && nb <= 16;
}

extern "C" cudaError_t xatu_launch_band_select(const BandParams& bp, const double* kpoints, const double* cellsR,
                                               const cd* HR, double* eigval, cd* eigvec, int* status,
                                               cudaStream_t s) {
  const int nbs = bp.nb <= 4 ? 4 : (bp.nb <= 8 ? 8 : 16);
  const BsLayout Ly = bs_layout(bp.norb, bp.nR, nbs);
  const void* fn = nbs == 4 ? (const void*)band_select_kernel<4>
                            : (nbs == 8 ? (const void*)band_select_kernel<8> : (const void*)band_select_kernel<16>);
  // warps per CTA: the fewest waves of one-warp-per-k work over the GPU (resident CTAs from the occupancy
  // calculator for each candidate), then the most warps per CTA (the staged H(R) blocks are shared by them)
  const size_t max_smem = 227 * 1024;
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  int wmax = 1;
  const int maxw = nbs == 4 ? BsMaxW<4>::value : (nbs == 8 ? BsMaxW<8>::value : BsMaxW<16>::value);
  while (wmax < maxw && Ly.stage + (size_t)(wmax + 1) * Ly.per_warp <= max_smem) wmax++;
  cudaError_t e = xatu_raise_smem_limit(fn, Ly.stage + (size_t)wmax * Ly.per_warp);
  if (e != cudaSuccess) return e;
  int wpc = 1;
  long long best_waves = -1;
  for (int w = 1; w <= wmax; w++) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, w * 32, Ly.stage + (size_t)w * Ly.per_warp) !=
            cudaSuccess ||
        per_sm < 1)
      continue;
    const long long slots = (long long)per_sm * w * sms;
    const long long waves = (bp.nk + slots - 1) / slots;
    if (best_waves < 0 || waves <= best_waves) {
      best_waves = waves;
      wpc = w;
    }
  }
  (void)cudaGetLastError();   // a failed occupancy query only removes its candidate
  const size_t smem = Ly.stage + (size_t)wpc * Ly.per_warp;
  const int grid = (bp.nk + wpc - 1) / wpc;
  const int threads = wpc * 32;
  if (nbs == 4)
    band_select_kernel<4><<<grid, threads, smem, s>>>(bp, kpoints, cellsR, HR, eigval, eigvec, status, wpc);
  else if (nbs == 8)
    band_select_kernel<8><<<grid, threads, smem, s>>>(bp, kpoints, cellsR, HR, eigval, eigvec, status, wpc);
  else
    band_select_kernel<16><<<grid, threads, smem, s>>>(bp, kpoints, cellsR, HR, eigval, eigvec, status, wpc);
  return cudaGetLastError();
}
