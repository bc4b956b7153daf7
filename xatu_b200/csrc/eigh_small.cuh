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
//      Golub & Van Loan, Matrix Computations, 8.3.1), on the lower triangle
//      only, by HEEV_RW warps with two named barriers per column: warp 0
//      updates the next column itself and forms the next reflector while the
//      other warps finish the trailing update.  The
//      reflectors are parked in global scratch and brought back for step 4.
//   2. Eigenvalues 0 .. k-1 of T by Sturm-sequence multisection: one warp
//      per eigenvalue, 64 shifts per step (the interval shrinks 65-fold).
//      The count of negative pivots q_i = d_i - s - e_{i-1}^2 / q_{i-1}
//      (Barth, Martin & Wilkinson 1967) is taken from the equivalent
//      three-term recurrence of the leading minors p_i = (d_i - s) p_{i-1} -
//      e_{i-1}^2 p_{i-2} (a negative pivot is a sign change p_{i-1} -> p_i),
//      renormalised every step by an exact power of two (integer arithmetic
//      on the exponent), so that the chain has no division; tiny pivots are
//      replaced by -pivmin as in the ratio form.
//   3. Eigenvectors of T by inverse iteration (three steps from a fixed
//      pseudo-random start), one lane per eigenvector, tridiagonal Gaussian
//      elimination with partial pivoting (factored once per eigenvalue, the
//      solves multiply by stored reciprocal pivots); after every step the
//      vectors of each cluster (neighbours closer than 1e-3 |T|) are
//      orthonormalised together by a Cholesky QR of their Gram matrix (the
//      clustering rule of LAPACK's DSTEIN, with a block Gram-Schmidt).
//   4. Back-transformation y = Q z, one warp per eigenvector, the reflectors
//      applied four at a time in compact WY form H_r..H_{r+3} = I - V T V^H
//      (Schreiber & Van Loan 1989; T by the recurrence of LAPACK's ZLARFT).
#pragma once
#include "common.cuh"

#define HEEV_THREADS 512
#define HEEV_MAXM 112   // the m x m matrix is held whole in shared memory
#define HEEV_WY 4       // reflectors per compact-WY block
#define HEEV_RW 4       // warps that run the tridiagonal reduction (named barrier 1)

__host__ __device__ inline int heev_lda(int m) { return (m % 2 == 0) ? m + 1 : m + 2; }

struct HeevLayout {
  size_t r0;        // the matrix; then Z + Gram + factors; then Z + reflectors + WY factors
  size_t zb, gb, fb, rb, tb;
  size_t total;
};

__host__ __device__ inline HeevLayout heev_layout(int m, int k) {
  HeevLayout L;
  const size_t sq = (size_t)m * heev_lda(m) * 16;
  const int nblk = (m - 1 + HEEV_WY - 1) / HEEV_WY;
  L.zb = ((size_t)m * k * 8 + 15) / 16 * 16;
  L.gb = ((size_t)k * k * 8 + 15) / 16 * 16;
  L.fb = (size_t)4 * m * 32 * 8 + ((size_t)m * 4 + 15) / 16 * 16;
  L.rb = (size_t)m * (m - 1) / 2 * 16;
  L.tb = (size_t)(nblk > 0 ? nblk : 0) * HEEV_WY * HEEV_WY * 16;
  size_t r0 = sq;
  if (L.zb + L.gb + L.fb > r0) r0 = L.zb + L.gb + L.fb;
  if (L.zb + L.rb + L.tb > r0) r0 = L.zb + L.rb + L.tb;
  L.r0 = (r0 + 15) / 16 * 16;
  // + d, e, e^2 (m doubles each), lam (k), red (64), tau (m), v (2 m), p (m) complex, cluster ids (k ints)
  L.total = L.r0 + (size_t)3 * m * 8 + (size_t)k * 8 + 64 * 8 + (size_t)4 * m * 16 + ((size_t)k * 4 + 15) / 16 * 16;
  return L;
}

__host__ __device__ inline size_t heev_smem_bytes(int m, int k) { return heev_layout(m, k).total; }

__device__ __forceinline__ double heev_wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Named barrier of the reduction warps.
__device__ __forceinline__ void heev_bar() { asm volatile("bar.sync 1, %0;" ::"n"(HEEV_RW * 32) : "memory"); }

// Bring |b| into [1, 2) and scale a by the same power of two, by integer arithmetic on the exponent
// fields.  Requires b normal and a with |a| in [1, 2) or 1 (the previous b), so that no field leaves
// the normal range for matrices with |T| < 1e150.
__device__ __forceinline__ void heev_rescale(double& a, double& b) {
  const int hb = __double2hiint(b);
  const int sh = (((hb >> 20) & 0x7ff) - 1023) << 20;
  b = __hiloint2double(hb - sh, __double2loint(b));
  a = __hiloint2double(__double2hiint(a) - sh, __double2loint(a));
}

// Numbers of eigenvalues of the tridiagonal (d, e) below s0 and below s1 (two independent chains, no
// division in either).  After each step |p_{i-1}| is in [1, 2), so the ratio-form guard |q_i| < pivmin
// becomes |p_i| < pivmin, and the replacement q_i = -pivmin becomes p_i = -pivmin sign(p_{i-1}).
__device__ __forceinline__ void heev_sturm2(const double* d, const double* e2, int m, double s0, double s1,
                                            double pivmin, int& c0, int& c1) {
  double p0 = 1.0, p1 = d[0] - s0, q0 = 1.0, q1 = d[0] - s1;
  if (fabs(p1) < pivmin) p1 = -pivmin;
  if (fabs(q1) < pivmin) q1 = -pivmin;
  c0 = p1 < 0.0;
  c1 = q1 < 0.0;
  heev_rescale(p0, p1);
  heev_rescale(q0, q1);
#pragma unroll 2
  for (int i = 1; i < m; i++) {
    const double di = d[i], ei = e2[i - 1];
    double p2 = fma(di - s0, p1, -ei * p0);
    double q2 = fma(di - s1, q1, -ei * q0);
    if (fabs(p2) < pivmin) p2 = copysign(pivmin, -p1);
    if (fabs(q2) < pivmin) q2 = copysign(pivmin, -q1);
    c0 += (p2 < 0.0) != (p1 < 0.0);
    c1 += (q2 < 0.0) != (q1 < 0.0);
    p0 = p1;
    p1 = p2;
    q0 = q1;
    q1 = q2;
    heev_rescale(p0, p1);
    heev_rescale(q0, q1);
  }
}

// Fixed pseudo-random start vector of inverse iteration (entries in (-1, 1)).
__device__ __forceinline__ double heev_start(int i, int j) {
  unsigned h = (unsigned)(i + 1) * 2654435761u ^ (unsigned)(j + 7) * 2246822519u;
  h ^= h >> 15;
  h *= 2654435761u;
  h ^= h >> 13;
  return ((double)(h & 0xffffff) + 0.5) / 8388608.0 - 1.0;
}

// Offset of reflector r in the packed store (entries v_r[0 .. L_r - 1], L_r = m - r - 1, v_r[0] = 1).
__device__ __forceinline__ int heev_poff(int r, int m) { return r * (m - 1) - r * (r - 1) / 2; }

// T: m x m Hermitian, column-major (leading dimension ldt; the lower triangle
// is read).  Outputs theta[0:k] ascending and Y (column-major, ldy) with the
// eigenvectors.  refl: global scratch of m * m complex.  prof (may be NULL):
// clock64() at the 8 phase boundaries.  Every thread of the CTA calls this
// (blockDim.x == HEEV_THREADS).
static __device__ void heev_lowest(const cd* __restrict__ Tg, int ldt, int m, int k, double* __restrict__ theta,
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
  double* FR = reinterpret_cast<double*>(smem + Ly.zb + Ly.gb);  // [4][m][32]: 1/pivot, u1, u2, multiplier
  unsigned* PM = reinterpret_cast<unsigned*>(FR + (size_t)4 * m * 32);   // [m] row-swap masks (bit = lane)
  cd* P = reinterpret_cast<cd*>(smem + Ly.zb);                   // packed reflectors (step 4)
  cd* TW = reinterpret_cast<cd*>(smem + Ly.zb + Ly.rb);          // WY factors (step 4)
  double* sd = reinterpret_cast<double*>(smem + Ly.r0);
  double* se = sd + m;
  double* se2 = se + m;
  double* lam = se2 + m;
  double* red = lam + k;
  cd* stau = reinterpret_cast<cd*>(red + 64);
  cd* sv = stau + m;   // two buffers of m
  cd* sp = sv + 2 * m;
  int* cl = reinterpret_cast<int*>(sp + m);
  const double eps = 2.220446049250313e-16;

  // ---- load (the lower triangle; the reduction keeps only the lower triangle)
  for (int t = tid; t < m * m; t += HEEV_THREADS) {
    const int r = t % m, c = t / m;
    if (r >= c) {
      const cd a = Tg[r + (size_t)c * ldt];
      A[r * lda + c] = (r == c) ? mk(a.x, 0.0) : a;
    }
  }
  __syncthreads();
  HEEV_MARK(1)

  // ---- 1. tridiagonal reduction (warps 0 .. HEEV_RW-1; the others wait at the next CTA barrier)
  if (warp < HEEV_RW) {
    constexpr int RT = HEEV_RW * 32;
    for (int j = 0; j < m - 1; j++) {
      const int L = m - j - 1;
      cd* v = sv + (j & 1) * m;
      if (warp == 0) {
        // reflector j from column j (updated by this warp in the previous step)
        double s = 0.0;
        for (int i = 1 + lane; i < L; i += 32) s += nrm2(A[(j + 1 + i) * lda + j]);
        s = heev_wsum(s);
        const cd al = A[(j + 1) * lda + j];
        cd tau = mk(0, 0), scal = mk(0, 0);
        double beta = al.x;
        const bool refl_on = (s > 0.0 || al.y != 0.0);
        if (refl_on) {
          beta = -copysign(sqrt(nrm2(al) + s), al.x);
          const double rb = 1.0 / beta;
          tau = mk((beta - al.x) * rb, -al.y * rb);
          const cd den = mk(al.x - beta, al.y);
          const double rdn = 1.0 / nrm2(den);
          scal = mk(den.x * rdn, -den.y * rdn);
        }
        for (int i = lane; i < L; i += 32) {
          cd vi = (i == 0) ? mk(1.0, 0.0) : (refl_on ? A[(j + 1 + i) * lda + j] * scal : mk(0, 0));
          v[i] = vi;
          refl[(size_t)j * m + (j + 1 + i)] = vi;
        }
        if (lane == 0) {
          stau[j] = tau;
          se[j] = beta;
          sd[j] = A[j * lda + j].x;
        }
      }
      heev_bar();
      const cd tau = stau[j];
      if (tau.x == 0.0 && tau.y == 0.0) continue;
      // p = tau A22 v, four threads per row (only the lower triangle is kept: A[r][c] = conj(A[c][r]))
      for (int r0 = 0; r0 < L; r0 += RT / 4) {
        const int row = r0 + (tid >> 2), sub = tid & 3;
        cd acc = mk(0, 0);
        if (row < L) {
          const int gr = j + 1 + row;
#pragma unroll 4
          for (int l = sub; l < L; l += 4) {
            const int gc = j + 1 + l;
            const bool lo = l <= row;
            cd a = A[lo ? gr * lda + gc : gc * lda + gr];
            if (!lo) a.y = -a.y;
            acc = acc + a * v[l];
          }
        }
#pragma unroll
        for (int o = 2; o > 0; o >>= 1) {
          acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
          acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
        }
        if (row < L && sub == 0) sp[row] = tau * acc;
      }
      heev_bar();
      double K;
      {
        double sx = 0.0, sy = 0.0;
        for (int i = lane; i < L; i += 32) {
          const cd t = cmulc(v[i], sp[i]);
          sx += t.x;
          sy += t.y;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          sx += __shfl_xor_sync(0xffffffffu, sx, o);
          sy += __shfl_xor_sync(0xffffffffu, sy, o);
        }
        K = 0.5 * (tau.x * sx + tau.y * sy);   // (1/2) Re(conj(tau) v^H p)
      }
      if (warp == 0) {
        // column 0 of the trailing block (the next reflector's column)
        const cd v0 = v[0], w0 = sp[0] - K * v0;
        for (int i = lane; i < L; i += 32) {
          const cd vi = v[i], wi = sp[i] - K * vi;
          cd& a = A[(j + 1 + i) * lda + (j + 1)];
          a = a - (vi * conj(w0) + wi * conj(v0));
        }
        __syncwarp();
      } else {
        // lower triangle, columns 1 .. i of row i: one warp per row
        for (int i = warp; i < L; i += HEEV_RW - 1) {
          const cd vi = v[i], wi = sp[i] - K * vi;
          cd* Ar = A + (j + 1 + i) * lda + (j + 1);
          for (int l = 1 + lane; l <= i; l += 32) {
            const cd vl = v[l], wl = sp[l] - K * vl;
            Ar[l] = Ar[l] - (vi * conj(wl) + wi * conj(vl));
          }
        }
      }
    }
  }
  __syncthreads();
  if (tid == 0) {
    sd[m - 1] = A[(m - 1) * lda + (m - 1)].x;
    se[m - 1] = 0.0;
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
      const double s0 = a + w * (double)(lane + 1) * (1.0 / 65.0);
      const double s1 = a + w * (double)(lane + 33) * (1.0 / 65.0);
      int c0, c1;
      heev_sturm2(sd, se2, m, s0, s1, pivmin, c0, c1);
      double na = (c1 <= i) ? s1 : ((c0 <= i) ? s0 : -INFINITY);
      double nb = (c0 > i) ? s0 : ((c1 > i) ? s1 : INFINITY);
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
    int multi = 0;
    for (int j = 0; j < k; j++) {
      cl[j] = (j > 0 && lam[j] - lam[j - 1] <= ortol) ? cl[j - 1] : j;
      multi |= cl[j] != j;
    }
    red[5] = multi ? 1.0 : 0.0;
  }
  for (int t = tid; t < m * k; t += HEEV_THREADS) Z[t] = heev_start(t / k, t % k);
  __syncthreads();
  HEEV_MARK(4)

  // ---- 3. inverse iteration + cluster orthonormalisation
  const double tiny = eps * tnorm;
  const bool keep_factors = k <= 32;
  double* RI = FR;
  double* DU = FR + (size_t)m * 32;
  double* DU2 = FR + (size_t)2 * m * 32;
  double* FM = FR + (size_t)3 * m * 32;
  for (int iter = 0; iter < 3; iter++) {
    if (warp == 0) {
      for (int c0 = 0; c0 < k; c0 += 32) {
        const int j = c0 + lane;
        const bool act = j < k;
        if (iter == 0 || !keep_factors) {
          // LU of T - lam_j I with partial pivoting (all lanes run it; idle lanes on lam[k-1])
          const double lj = lam[act ? j : k - 1];
          double cur_d = sd[0] - lj, cur_u = (m > 1) ? se[0] : 0.0;
          for (int i = 0; i < m - 1; i++) {
            const double sub = se[i];
            double nd = sd[i + 1] - lj, nu = (i < m - 2) ? se[i + 1] : 0.0;
            double piv, up, u2 = 0.0, f;
            const bool sw = fabs(cur_d) < fabs(sub);
            double rp;
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
              if (i < m - 2) {
                u2 = nu;
                nu = -f * u2;
              }
              up = tmp;
            }
            RI[i * 32 + lane] = rp;
            DU[i * 32 + lane] = up;
            DU2[i * 32 + lane] = u2;
            FM[i * 32 + lane] = f;
            const unsigned msk = __ballot_sync(0xffffffffu, sw);
            if (lane == 0) PM[i] = msk;
            cur_d = nd;
            cur_u = nu;
          }
          if (fabs(cur_d) < tiny) cur_d = (cur_d < 0.0) ? -tiny : tiny;
          RI[(m - 1) * 32 + lane] = 1.0 / cur_d;
          __syncwarp();
        }
        if (act) {
          double nn = 0.0;
          for (int i = 0; i < m; i++) nn += Z[i * k + j] * Z[i * k + j];
          const double f0 = nn > 0.0 ? 1.0 / sqrt(nn) : 1.0;
          // forward elimination of the right-hand side
          double xi = Z[j] * f0;
#pragma unroll 4
          for (int i = 0; i < m - 1; i++) {
            double xn = Z[(i + 1) * k + j] * f0;
            const double f = FM[i * 32 + lane];
            if ((PM[i] >> lane) & 1u) {
              const double t = xi;
              xi = xn;
              xn = t - f * xn;
            } else {
              xn -= f * xi;
            }
            Z[i * k + j] = xi;
            xi = xn;
          }
          // back substitution
          double x2 = 0.0, x1 = xi * RI[(m - 1) * 32 + lane];
          Z[(m - 1) * k + j] = x1;
          nn = x1 * x1;
#pragma unroll 4
          for (int i = m - 2; i >= 0; i--) {
            const double x0 = (Z[i * k + j] - DU[i * 32 + lane] * x1 - DU2[i * 32 + lane] * x2) * RI[i * 32 + lane];
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
    if (red[5] == 0.0) continue;   // every cluster is a single vector (normalised above)
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
        const double lc = 1.0 / G[c * k + c];
        for (int r = c + 1 + lane; r < k; r += 32)
          if (cl[r] == cl[c]) G[r * k + c] *= lc;
        __syncwarp();
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

  // ---- 4. back-transformation y = H_0 ... H_{m-2} z in compact WY blocks
  const int nr = m - 1;
  const int nblk = (nr + HEEV_WY - 1) / HEEV_WY;
  for (int r = warp; r < nr; r += NW) {
    const int L = m - r - 1;
    const int off = heev_poff(r, m);
    for (int i = lane; i < L; i += 32) P[off + i] = (i == 0) ? mk(1.0, 0.0) : refl[(size_t)r * m + (r + 1 + i)];
  }
  __syncthreads();
  // T factor of each block: T_ii = tau_i, T(0:i, i) = -tau_i T(0:i, 0:i) (V(:, 0:i)^H v_i)
  for (int q = warp; q < nblk; q += NW) {
    const int r0 = q * HEEV_WY, nb = min(HEEV_WY, nr - r0);
    cd g[HEEV_WY][HEEV_WY];
#pragma unroll
    for (int a = 0; a < HEEV_WY; a++)
#pragma unroll
      for (int b = 0; b < HEEV_WY; b++) g[a][b] = mk(0, 0);
#pragma unroll
    for (int a = 0; a < HEEV_WY; a++)
#pragma unroll
      for (int b = a + 1; b < HEEV_WY; b++) {
        if (b >= nb) continue;
        double sx = 0.0, sy = 0.0;
        const cd* va = P + heev_poff(r0 + a, m) - (r0 + a + 1);   // va[row], row > r0 + a
        const cd* vb = P + heev_poff(r0 + b, m) - (r0 + b + 1);
        for (int row = r0 + b + 1 + lane; row < m; row += 32) {
          const cd t = cmulc(va[row], vb[row]);
          sx += t.x;
          sy += t.y;
        }
        g[a][b] = mk(heev_wsum(sx), heev_wsum(sy));
      }
    if (lane == 0) {
      cd Tq[HEEV_WY][HEEV_WY];
#pragma unroll
      for (int a = 0; a < HEEV_WY; a++)
#pragma unroll
        for (int b = 0; b < HEEV_WY; b++) Tq[a][b] = mk(0, 0);
#pragma unroll
      for (int i = 0; i < HEEV_WY; i++) {
        if (i >= nb) continue;
        const cd ti = stau[r0 + i];
#pragma unroll
        for (int a = 0; a < HEEV_WY; a++) {
          if (a >= i) continue;
          cd s = mk(0, 0);
#pragma unroll
          for (int c = 0; c < HEEV_WY; c++)
            if (c >= a && c < i) s = s + Tq[a][c] * g[c][i];
          const cd t = ti * s;
          Tq[a][i] = mk(-t.x, -t.y);
        }
        Tq[i][i] = ti;
      }
#pragma unroll
      for (int a = 0; a < HEEV_WY; a++)
#pragma unroll
        for (int b = 0; b < HEEV_WY; b++) TW[(q * HEEV_WY + a) * HEEV_WY + b] = Tq[a][b];
    }
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
    for (int qb = nblk - 1; qb >= 0; qb--) {
      const int r0 = qb * HEEV_WY, nb = min(HEEV_WY, nr - r0);
      cd vv[HEEV_WY][PER];
      double wx[HEEV_WY], wy[HEEV_WY];
#pragma unroll
      for (int a = 0; a < HEEV_WY; a++) {
        wx[a] = 0.0;
        wy[a] = 0.0;
        const int ra = r0 + a;
        const cd* va = P + heev_poff(ra, m) - (ra + 1);   // va[row], row > ra
#pragma unroll
        for (int q = 0; q < PER; q++) {
          const int p = lane + 32 * q;
          vv[a][q] = (a < nb && p > ra && p < m) ? va[p] : mk(0, 0);
          const cd t = cmulc(vv[a][q], y[q]);
          wx[a] += t.x;
          wy[a] += t.y;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int a = 0; a < HEEV_WY; a++) {
          wx[a] += __shfl_xor_sync(0xffffffffu, wx[a], o);
          wy[a] += __shfl_xor_sync(0xffffffffu, wy[a], o);
        }
      // u = T w (T upper triangular)
      cd u[HEEV_WY];
#pragma unroll
      for (int a = 0; a < HEEV_WY; a++) {
        cd s = mk(0, 0);
#pragma unroll
        for (int b = 0; b < HEEV_WY; b++)
          if (b >= a) s = s + TW[(qb * HEEV_WY + a) * HEEV_WY + b] * mk(wx[b], wy[b]);
        u[a] = s;
      }
#pragma unroll
      for (int q = 0; q < PER; q++)
#pragma unroll
        for (int a = 0; a < HEEV_WY; a++) y[q] = y[q] - vv[a][q] * u[a];
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
