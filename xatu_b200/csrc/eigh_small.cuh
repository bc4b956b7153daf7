// Lowest k eigenpairs of a small dense Hermitian matrix (m <= HEEV_MAXM), one
// CTA of HEEV_THREADS threads, FP64 throughout.  Used for the Rayleigh-Ritz
// step of the Davidson solvers, where only the lowest block of Ritz pairs of
// the projected matrix is wanted.
//
//   1. Householder reduction to real symmetric tridiagonal form,
//        A = Q T Q^H,  Q = H_0 H_1 ... H_{m-2},  H_j = I - tau_j v_j v_j^H
//      (reflectors chosen so that H_j^H x = beta e_1 with beta real, the
//      convention of LAPACK's ZLARFG; the trailing block is updated as
//        A <- A - v w^H - w v^H,  p = tau A v,  w = p - (1/2) Re(conj(tau) v^H p) v;
//      Golub & Van Loan, Matrix Computations, 8.3.1).  The reflectors are
//      parked in global scratch and brought back for step 4.
//   2. Eigenvalues k = 0 .. k-1 of T by Sturm-sequence multisection: one warp
//      per eigenvalue, 32 shifts per step (the interval shrinks 33-fold),
//      count(s) = #{q_i < 0}, q_i = d_i - s - e_{i-1}^2 / q_{i-1} (Wilkinson;
//      Barth, Martin & Wilkinson 1967), tiny pivots replaced by -pivmin.
//   3. Eigenvectors of T by inverse iteration (three steps from a fixed
//      pseudo-random start), one lane per eigenvector, tridiagonal Gaussian
//      elimination with partial pivoting; after every step the vectors of
//      each cluster (neighbours closer than 1e-3 |T|) are orthonormalised
//      together by a Cholesky QR of their Gram matrix (the clustering rule of
//      LAPACK's DSTEIN, with block instead of sequential Gram-Schmidt).
//   4. Back-transformation y = Q z, one warp per eigenvector.
#pragma once
#include "common.cuh"

#define HEEV_THREADS 512
#define HEEV_MAXM 112   // the m x m matrix is held whole in shared memory

__host__ __device__ inline int heev_lda(int m) { return (m % 2 == 0) ? m + 1 : m + 2; }

struct HeevLayout {
  size_t r0;        // the matrix, later Z + U factors + Gram, later Z + reflectors
  size_t zb, gb, ub, rb;
  size_t total;
};

__host__ __device__ inline HeevLayout heev_layout(int m, int k) {
  HeevLayout L;
  const size_t sq = (size_t)m * heev_lda(m) * 16;
  L.zb = ((size_t)m * k * 8 + 15) / 16 * 16;
  L.gb = ((size_t)k * k * 8 + 15) / 16 * 16;
  L.ub = (size_t)3 * m * 32 * 8;
  L.rb = m >= 2 ? (size_t)(m - 1) * (m - 2) / 2 * 16 : 0;
  size_t r0 = sq;
  if (L.zb + L.gb + L.ub > r0) r0 = L.zb + L.gb + L.ub;
  if (L.zb + L.rb > r0) r0 = L.zb + L.rb;
  L.r0 = (r0 + 15) / 16 * 16;
  // + d, e, e^2 (m doubles each), lam (k), red (64), tau, v, p (m complex each), cluster ids (k ints)
  L.total = L.r0 + (size_t)3 * m * 8 + (size_t)k * 8 + 64 * 8 + (size_t)3 * m * 16 + ((size_t)k * 4 + 15) / 16 * 16;
  return L;
}

__host__ __device__ inline size_t heev_smem_bytes(int m, int k) { return heev_layout(m, k).total; }

__device__ __forceinline__ double heev_wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Number of eigenvalues of the tridiagonal (d, e) below s.
__device__ __forceinline__ int heev_sturm(const double* d, const double* e2, int m, double s, double pivmin) {
  double q = d[0] - s;
  if (fabs(q) < pivmin) q = -pivmin;
  int c = q < 0.0;
  for (int i = 1; i < m; i++) {
    q = d[i] - s - e2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    c += q < 0.0;
  }
  return c;
}

// Fixed pseudo-random start vector of inverse iteration (entries in (-1, 1)).
__device__ __forceinline__ double heev_start(int i, int j) {
  unsigned h = (unsigned)(i + 1) * 2654435761u ^ (unsigned)(j + 7) * 2246822519u;
  h ^= h >> 15;
  h *= 2654435761u;
  h ^= h >> 13;
  return ((double)(h & 0xffffff) + 0.5) / 8388608.0 - 1.0;
}

// T: m x m Hermitian, column-major (leading dimension ldt; the lower triangle
// is read).  Outputs theta[0:k] ascending and Y (column-major, ldy) with the
// eigenvectors.  refl: global scratch of m * m complex.  prof (may be NULL):
// clock64() at the 8 phase boundaries.  Every thread of the CTA calls this
// (blockDim.x == HEEV_THREADS).
__device__ void heev_lowest(const cd* __restrict__ Tg, int ldt, int m, int k, double* __restrict__ theta,
                            cd* __restrict__ Yg, int ldy, cd* __restrict__ refl, unsigned char* smem,
                            int* __restrict__ status, long long* __restrict__ prof = nullptr) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#define HEEV_MARK(i) \
  if (prof && tid == 0) prof[i] = clock64();
  HEEV_MARK(0)
  constexpr int NW = HEEV_THREADS / 32;
  const HeevLayout Ly = heev_layout(m, k);
  const int lda = heev_lda(m);
  cd* A = reinterpret_cast<cd*>(smem);
  double* Z = reinterpret_cast<double*>(smem);                   // m x k, row-major (after step 1)
  double* G = reinterpret_cast<double*>(smem + Ly.zb);           // k x k
  double* U3 = reinterpret_cast<double*>(smem + Ly.zb + Ly.gb);  // [3][m][32]
  cd* P = reinterpret_cast<cd*>(smem + Ly.zb);                   // packed reflectors (step 4)
  double* sd = reinterpret_cast<double*>(smem + Ly.r0);
  double* se = sd + m;
  double* se2 = se + m;
  double* lam = se2 + m;
  double* red = lam + k;
  cd* stau = reinterpret_cast<cd*>(red + 64);
  cd* sv = stau + m;
  cd* sp = sv + m;
  int* cl = reinterpret_cast<int*>(sp + m);
  const double eps = 2.220446049250313e-16;

  // ---- load (lower triangle authoritative, exact Hermitian copy)
  for (int t = tid; t < m * m; t += HEEV_THREADS) {
    const int r = t % m, c = t / m;
    if (r >= c) {
      const cd a = Tg[r + (size_t)c * ldt];
      if (r == c) {
        A[r * lda + r] = mk(a.x, 0.0);
      } else {
        A[r * lda + c] = a;
        A[c * lda + r] = conj(a);
      }
    }
  }
  __syncthreads();
  HEEV_MARK(1)

  // ---- 1. tridiagonal reduction
  for (int j = 0; j < m - 1; j++) {
    const int L = m - j - 1;
    if (warp == 0) {
      double s = 0.0;
      for (int i = 1 + lane; i < L; i += 32) s += nrm2(A[(j + 1 + i) * lda + j]);
      s = heev_wsum(s);
      const cd al = A[(j + 1) * lda + j];
      cd tau = mk(0, 0), scal = mk(0, 0);
      double beta = al.x;
      const bool refl_on = (s > 0.0 || al.y != 0.0);
      if (refl_on) {
        beta = -copysign(sqrt(nrm2(al) + s), al.x);
        tau = mk((beta - al.x) / beta, -al.y / beta);
        const cd den = mk(al.x - beta, al.y);
        const double dn = nrm2(den);
        scal = mk(den.x / dn, -den.y / dn);
      }
      for (int i = lane; i < L; i += 32) {
        cd vi = (i == 0) ? mk(1.0, 0.0) : (refl_on ? A[(j + 1 + i) * lda + j] * scal : mk(0, 0));
        sv[i] = vi;
        if (i >= 1) refl[(size_t)j * m + (j + 1 + i)] = vi;
      }
      if (lane == 0) {
        stau[j] = tau;
        se[j] = beta;
        sd[j] = A[j * lda + j].x;
      }
    }
    __syncthreads();
    const cd tau = stau[j];
    if (tau.x == 0.0 && tau.y == 0.0) continue;
    {
      const int tpr = (L <= 64) ? 8 : 4;
      const int row = tid / tpr, sub = tid % tpr;
      cd acc = mk(0, 0);
      if (row < L) {
        const cd* Ar = A + (j + 1 + row) * lda + (j + 1);
        for (int l = sub; l < L; l += tpr) acc = acc + Ar[l] * sv[l];
      }
      for (int o = tpr >> 1; o > 0; o >>= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
      }
      if (row < L && sub == 0) sp[row] = tau * acc;
    }
    __syncthreads();
    double K;
    {
      double sx = 0.0, sy = 0.0;
      for (int i = lane; i < L; i += 32) {
        const cd t = cmulc(sv[i], sp[i]);
        sx += t.x;
        sy += t.y;
      }
      sx = heev_wsum(sx);
      sy = heev_wsum(sy);
      K = 0.5 * (tau.x * sx + tau.y * sy);   // (1/2) Re(conj(tau) v^H p)
    }
    for (int t = tid; t < L * L; t += HEEV_THREADS) {
      const int i = t / L, l = t - i * L;
      const cd vi = sv[i], vl = sv[l];
      const cd wi = sp[i] - K * vi, wl = sp[l] - K * vl;
      cd& a = A[(j + 1 + i) * lda + (j + 1 + l)];
      a = a - (vi * conj(wl) + wi * conj(vl));
    }
    __syncthreads();
  }
  if (tid == 0) {
    sd[m - 1] = A[(m - 1) * lda + (m - 1)].x;
    if (m >= 1) se[m - 1] = 0.0;
  }
  __syncthreads();
  HEEV_MARK(2)
  for (int i = tid; i < m; i += HEEV_THREADS) se2[i] = se[i] * se[i];
  // Gershgorin interval, |T|, pivmin
  if (warp == 0) {
    double lo = INFINITY, hi = -INFINITY, e2max = 0.0;
    bool finite = true;
    for (int i = lane; i < m; i += 32) {
      const double r = (i > 0 ? fabs(se[i - 1]) : 0.0) + (i < m - 1 ? fabs(se[i]) : 0.0);
      lo = fmin(lo, sd[i] - r);
      hi = fmax(hi, sd[i] + r);
      if (i < m - 1) e2max = fmax(e2max, se[i] * se[i]);
      finite = finite && isfinite(sd[i]) && isfinite(se[i]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
      e2max = fmax(e2max, __shfl_xor_sync(0xffffffffu, e2max, o));
    }
    finite = __all_sync(0xffffffffu, finite);
    if (lane == 0) {
      const double tn = fmax(fmax(fabs(lo), fabs(hi)), 1e-100);
      const double pivmin = 1e-290 * fmax(1.0, e2max);
      const double fudge = 4.0 * (m + 1) * eps * tn + 4.0 * pivmin;
      red[0] = lo - fudge;
      red[1] = hi + fudge;
      red[2] = tn;
      red[3] = pivmin;
      red[4] = finite ? 0.0 : 1.0;
      if (!finite) atomicOr(status, XATU_DEVERR_NAN);
    }
  }
  __syncthreads();
  const double gl = red[0], gu = red[1], tnorm = red[2], pivmin = red[3];
  if (red[4] != 0.0) {
    for (int t = tid; t < k; t += HEEV_THREADS) theta[t] = NAN;
    return;
  }

  HEEV_MARK(3)
  // ---- 2. multisection, one warp per eigenvalue
  for (int i = warp; i < k; i += NW) {
    double a = gl, b = gu;
    for (int it = 0; it < 64; it++) {
      const double w = b - a;
      if (!(w > fmax(2.0 * eps * fmax(fabs(a), fabs(b)), fmax(0.5 * eps * tnorm, pivmin)))) break;
      const double s = a + w * (double)(lane + 1) / 33.0;
      const int c = heev_sturm(sd, se2, m, s, pivmin);
      double na = (c <= i) ? s : -INFINITY, nb = (c > i) ? s : INFINITY;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        na = fmax(na, __shfl_xor_sync(0xffffffffu, na, o));
        nb = fmin(nb, __shfl_xor_sync(0xffffffffu, nb, o));
      }
      const double a2 = fmax(a, na), b2 = fmin(b, nb);
      if (!(a2 < b2)) {   // inconsistent counts: stop at the current bracket
        a = b = 0.5 * (a + b);
        break;
      }
      if (a2 == a && b2 == b) break;
      a = a2;
      b = b2;
    }
    if (lane == 0) lam[i] = 0.5 * (a + b);
  }
  __syncthreads();
  if (tid == 0) {
    const double ortol = 1e-3 * tnorm;
    for (int j = 0; j < k; j++) cl[j] = (j > 0 && lam[j] - lam[j - 1] <= ortol) ? cl[j - 1] : j;
  }
  for (int t = tid; t < m * k; t += HEEV_THREADS) Z[t] = heev_start(t / k, t % k);
  __syncthreads();
  HEEV_MARK(4)

  // ---- 3. inverse iteration + cluster orthonormalisation
  const double tiny = eps * tnorm;
  for (int iter = 0; iter < 3; iter++) {
    if (warp == 0) {
      for (int c0 = 0; c0 < k; c0 += 32) {
        const int j = c0 + lane;
        if (j < k) {
          const double lj = lam[j];
          double* DD = U3;
          double* DU = U3 + (size_t)m * 32;
          double* DU2 = U3 + (size_t)2 * m * 32;
          // normalise the right-hand side
          double nn = 0.0;
          for (int i = 0; i < m; i++) nn += Z[i * k + j] * Z[i * k + j];
          const double f0 = nn > 0.0 ? 1.0 / sqrt(nn) : 1.0;
          double cur_d = sd[0] - lj, cur_u = (m > 1) ? se[0] : 0.0, xi = Z[j] * f0;
          for (int i = 0; i < m - 1; i++) {
            const double sub = se[i];
            double nd = sd[i + 1] - lj, nu = (i < m - 2) ? se[i + 1] : 0.0;
            double xn = Z[(i + 1) * k + j] * f0;
            double piv, up, u2 = 0.0;
            if (fabs(cur_d) >= fabs(sub)) {
              piv = cur_d;
              if (fabs(piv) < tiny) piv = (piv < 0.0) ? -tiny : tiny;
              const double f = sub / piv;
              nd -= f * cur_u;
              xn -= f * xi;
              up = cur_u;
            } else {
              const double f = cur_d / sub;
              piv = sub;
              const double tmp = nd;
              nd = cur_u - f * tmp;
              if (i < m - 2) {
                u2 = nu;
                nu = -f * u2;
              }
              up = tmp;
              const double xs = xi;
              xi = xn;
              xn = xs - f * xn;
            }
            DD[i * 32 + lane] = piv;
            DU[i * 32 + lane] = up;
            DU2[i * 32 + lane] = u2;
            Z[i * k + j] = xi;
            cur_d = nd;
            cur_u = nu;
            xi = xn;
          }
          if (fabs(cur_d) < tiny) cur_d = (cur_d < 0.0) ? -tiny : tiny;
          // back substitution
          double x2 = 0.0, x1 = xi / cur_d;
          Z[(m - 1) * k + j] = x1;
          nn = x1 * x1;
          for (int i = m - 2; i >= 0; i--) {
            const double x0 = (Z[i * k + j] - DU[i * 32 + lane] * x1 - DU2[i * 32 + lane] * x2) / DD[i * 32 + lane];
            Z[i * k + j] = x0;
            nn += x0 * x0;
            x2 = x1;
            x1 = x0;
          }
          const double f1 = 1.0 / sqrt(nn);
          for (int i = 0; i < m; i++) Z[i * k + j] *= f1;
        }
        __syncwarp();
      }
    }
    __syncthreads();
    // Gram matrix of each cluster (lower triangle)
    for (int t = tid; t < k * k; t += HEEV_THREADS) {
      const int r = t / k, c = t - r * k;
      if (c <= r && cl[r] == cl[c]) {
        double g = 0.0;
        for (int i = 0; i < m; i++) g += Z[i * k + r] * Z[i * k + c];
        G[r * k + c] = g;
      }
    }
    __syncthreads();
    // Cholesky (one warp; columns of different clusters never meet)
    if (warp == 0) {
      for (int c = 0; c < k; c++) {
        if (lane == 0) {
          double pv = G[c * k + c];
          if (!(pv > 1e-24)) {
            atomicOr(status, XATU_DEVERR_NOCONV);
            pv = 1e-24;
          }
          G[c * k + c] = sqrt(pv);
        }
        __syncwarp();
        const double lc = G[c * k + c];
        for (int r = c + 1 + lane; r < k; r += 32)
          if (cl[r] == cl[c]) G[r * k + c] /= lc;
        __syncwarp();
        // trailing update of the cluster block
        for (int r = c + 1 + lane; r < k; r += 32) {
          if (cl[r] != cl[c]) continue;
          const double grc = G[r * k + c];
          for (int s = c + 1; s <= r; s++) G[r * k + s] -= grc * G[s * k + c];
        }
        __syncwarp();
      }
    }
    __syncthreads();
    // Z <- Z L^{-T}, one thread per row
    for (int i = tid; i < m; i += HEEV_THREADS) {
      double* zr = Z + (size_t)i * k;
      for (int c = 0; c < k; c++) {
        double v = zr[c];
        for (int l = cl[c]; l < c; l++) v -= zr[l] * G[c * k + l];
        zr[c] = v / G[c * k + c];
      }
    }
    __syncthreads();
  }

  HEEV_MARK(5)
  // ---- 4. back-transformation y = H_0 ... H_{m-2} z
  for (int r = warp; r < m - 1; r += NW) {
    const int L = m - r - 1;
    const size_t off = (size_t)r * (m - 2) - (size_t)r * (r - 1) / 2;
    for (int i = 1 + lane; i < L; i += 32) P[off + i - 1] = refl[(size_t)r * m + (r + 1 + i)];
  }
  __syncthreads();
  HEEV_MARK(6)
  constexpr int PER = (HEEV_MAXM + 31) / 32;
  for (int j = warp; j < k; j += NW) {
    cd y[PER];
#pragma unroll
    for (int q = 0; q < PER; q++) {
      const int p = lane + 32 * q;
      y[q] = mk(p < m ? Z[p * k + j] : 0.0, 0.0);
    }
    for (int r = m - 2; r >= 0; r--) {
      const cd tau = stau[r];
      if (tau.x == 0.0 && tau.y == 0.0) continue;
      const size_t off = (size_t)r * (m - 2) - (size_t)r * (r - 1) / 2;
      double sx = 0.0, sy = 0.0;
      cd vq[PER];
#pragma unroll
      for (int q = 0; q < PER; q++) {
        const int p = lane + 32 * q;
        const int i = p - r - 1;
        vq[q] = (p < m && i >= 0) ? (i == 0 ? mk(1.0, 0.0) : P[off + i - 1]) : mk(0, 0);
        const cd t = cmulc(vq[q], y[q]);
        sx += t.x;
        sy += t.y;
      }
      sx = heev_wsum(sx);
      sy = heev_wsum(sy);
      const cd ts = tau * mk(sx, sy);
#pragma unroll
      for (int q = 0; q < PER; q++) y[q] = y[q] - ts * vq[q];
    }
#pragma unroll
    for (int q = 0; q < PER; q++) {
      const int p = lane + 32 * q;
      if (p < m) Yg[p + (size_t)j * ldy] = y[q];
    }
    if (lane == 0) theta[j] = lam[j];
  }
  if (prof) {
    __syncthreads();
    HEEV_MARK(7)
  }
#undef HEEV_MARK
}
