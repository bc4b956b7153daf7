// Two-sided cyclic Jacobi eigensolver for complex Hermitian matrices held in
// shared memory, FP64, run cooperatively by a thread group (one warp or one
// CTA).  Parallel ordering: round-robin tournament, n/2 disjoint rotations per
// round.  Each round has two phases separated by a group barrier:
//   (1) one thread per pair computes its rotation from the current 2x2 block;
//   (2) every 2x2 block A[P x R] of row pair P and column pair R is replaced
//       by J_P^H A[P x R] J_R (blocks are disjoint, so all are updated at
//       once), the diagonal blocks get their exact diagonal form, and the
//       eigenvector rows are rotated, V[row, R] <- V[row, R] J_R.
// Quadratic convergence; the sweep count is capped.
//
// Rotation for the pair (p, q), c = A_pq = |c| e^{i phi}:
//   tau = (A_qq - A_pp) / (2|c|),  t = sgn(tau) / (|tau| + sqrt(1 + tau^2)),
//   cs = 1/sqrt(1 + t^2),  sn = t cs,
//   J = [[cs, sn e^{i phi}], [-sn e^{-i phi}, cs]],   A <- J^H A J,  V <- V J.
// The real case is the classical Jacobi rotation (Golub & Van Loan 8.5); the
// phase e^{i phi} first makes the pivot real.
#pragma once
#include "common.cuh"

struct WarpGroup {
  __device__ __forceinline__ int rank() const { return threadIdx.x & 31; }
  __device__ __forceinline__ int size() const { return 32; }
  __device__ __forceinline__ void sync() const { __syncwarp(); }
  // Sum over the group; every thread gets the result.
  __device__ __forceinline__ double sum(double v, double* /*scratch*/) const {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
  }
};

struct BlockGroup {
  __device__ __forceinline__ int rank() const { return threadIdx.x; }
  __device__ __forceinline__ int size() const { return blockDim.x; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
  // scratch: at least blockDim.x/32 + 1 doubles of shared memory.
  __device__ __forceinline__ double sum(double v, double* scratch) const {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) scratch[w] = v;
    __syncthreads();
    double s = 0.0;
    for (int i = 0; i < nw; i++) s += scratch[i];
    __syncthreads();
    return s;
  }
};

struct JacobiRot {
  double cs;
  cd se;        // sn * e^{i phi}
  double app, aqq;
  int p, q;     // q >= n: dummy pair (odd n); rot == 0: identity
  int rot;
};

// x J restricted to one row: (x_p, x_q) -> (cs x_p - conj(se) x_q, se x_p + cs x_q)
__device__ __forceinline__ void rot_right(const JacobiRot& R, cd& xp, cd& xq) {
  const cd a = xp, b = xq;
  xp = mk(R.cs * a.x - (b.x * R.se.x + b.y * R.se.y), R.cs * a.y - (b.y * R.se.x - b.x * R.se.y));
  xq = a * R.se + R.cs * b;
}
// J^H applied from the left to one column: (y_p, y_q) -> (cs y_p - se y_q, conj(se) y_p + cs y_q)
__device__ __forceinline__ void rot_left(const JacobiRot& R, cd& yp, cd& yq) {
  const cd a = yp, b = yq;
  yp = R.cs * a - R.se * b;
  yq = mk(R.se.x * a.x + R.se.y * a.y + R.cs * b.x, R.se.x * a.y - R.se.y * a.x + R.cs * b.y);
}

// A: n x n (row stride lda), V: n x n (row stride ldv) initialised here to the
// identity.  rot: scratch for n/2 + 1 rotations, scratch: reduction scratch.
// Returns the number of sweeps used (> max_sweeps: not converged).
template <class G>
__device__ int jacobi_eigh(const G& g, cd* A, int lda, cd* V, int ldv, int n, JacobiRot* rot, double* scratch,
                           int max_sweeps, double rel_tol) {
  const int tid = g.rank(), nt = g.size();
  for (int r = 0; r < n; r++)
    for (int c = tid; c < n; c += nt) V[r * ldv + c] = mk(r == c ? 1.0 : 0.0, 0.0);
  for (int i = tid; i < n; i += nt) A[i * lda + i].y = 0.0;
  g.sync();
  if (n <= 1) return 0;
  const int n2 = n + (n & 1);
  const int m = n2 - 1;
  const int np = n2 / 2;
  int sweep = 0;
  for (; sweep <= max_sweeps; sweep++) {
    double off = 0.0, tot = 0.0;
    for (int r = 0; r < n; r++)
      for (int c = tid; c < n; c += nt) {
        const double a2 = nrm2(A[r * lda + c]);
        tot += a2;
        if (r != c) off += a2;
      }
    off = g.sum(off, scratch);
    tot = g.sum(tot, scratch);
    if (off <= rel_tol * rel_tol * tot || off == 0.0) break;
    if (sweep == max_sweeps) {
      sweep++;
      break;
    }
    for (int r = 0; r < m; r++) {
      // ---- phase 1: rotations
      for (int i = tid; i < np; i += nt) {
        int a, b;
        if (i == 0) {
          a = r;
          b = m;
        } else {
          a = r + i;
          if (a >= m) a -= m;
          b = r - i;
          if (b < 0) b += m;
        }
        JacobiRot R;
        R.p = min(a, b);
        R.q = max(a, b);
        R.rot = 0;
        R.cs = 1.0;
        R.se = mk(0, 0);
        if (R.q < n) {
          const cd c = A[R.p * lda + R.q];
          const double ac = sqrt(nrm2(c));
          const double app = A[R.p * lda + R.p].x, aqq = A[R.q * lda + R.q].x;
          R.app = app;
          R.aqq = aqq;
          if (ac > 1e-300) {
            const double tau = (aqq - app) / (2.0 * ac);
            const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            const double cs = 1.0 / sqrt(1.0 + t * t);
            const double sn = t * cs;
            R.cs = cs;
            R.se = mk(sn * c.x / ac, sn * c.y / ac);
            R.app = app - t * ac;
            R.aqq = aqq + t * ac;
            R.rot = 1;
          }
        }
        rot[i] = R;
      }
      g.sync();
      // ---- phase 2: all 2x2 blocks J_P^H A[P x R] J_R, and V rows
      const int nblk = np * np;
      for (int t = tid; t < nblk + n * np; t += nt) {
        if (t < nblk) {
          const int P = t / np, Q = t - P * np;
          const JacobiRot RP = rot[P], RQ = rot[Q];
          if (!RP.rot && !RQ.rot) continue;
          const bool hasq = RP.q < n, hass = RQ.q < n;
          if (P == Q) {
            if (RP.rot) {
              A[RP.p * lda + RP.p] = mk(RP.app, 0);
              A[RP.q * lda + RP.q] = mk(RP.aqq, 0);
              A[RP.p * lda + RP.q] = mk(0, 0);
              A[RP.q * lda + RP.p] = mk(0, 0);
            }
            continue;
          }
          cd b00 = A[RP.p * lda + RQ.p];
          cd b01 = hass ? A[RP.p * lda + RQ.q] : mk(0, 0);
          cd b10 = hasq ? A[RP.q * lda + RQ.p] : mk(0, 0);
          cd b11 = (hasq && hass) ? A[RP.q * lda + RQ.q] : mk(0, 0);
          if (RQ.rot) {
            rot_right(RQ, b00, b01);
            rot_right(RQ, b10, b11);
          }
          if (RP.rot) {
            rot_left(RP, b00, b10);
            rot_left(RP, b01, b11);
          }
          A[RP.p * lda + RQ.p] = b00;
          if (hass) A[RP.p * lda + RQ.q] = b01;
          if (hasq) A[RP.q * lda + RQ.p] = b10;
          if (hasq && hass) A[RP.q * lda + RQ.q] = b11;
        } else {
          const int u = t - nblk;
          const int row = u / np, Q = u - row * np;
          const JacobiRot RQ = rot[Q];
          if (!RQ.rot) continue;
          cd x = V[row * ldv + RQ.p], y = V[row * ldv + RQ.q];
          rot_right(RQ, x, y);
          V[row * ldv + RQ.p] = x;
          V[row * ldv + RQ.q] = y;
        }
      }
      g.sync();
    }
  }
  return sweep;
}

// Ascending order of the eigenvalues (diagonal of A): perm[rank] = index.
template <class G>
__device__ void jacobi_sort(const G& g, const cd* A, int lda, int n, int* perm) {
  for (int i = g.rank(); i < n; i += g.size()) {
    const double li = A[i * lda + i].x;
    int rank = 0;
    for (int j = 0; j < n; j++) {
      const double lj = A[j * lda + j].x;
      rank += (lj < li) || (lj == li && j < i);
    }
    perm[rank] = i;
  }
  g.sync();
}
