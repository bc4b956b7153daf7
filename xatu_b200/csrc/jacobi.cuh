// Two-sided cyclic Jacobi eigensolver for complex Hermitian matrices held in
// shared memory, FP64, run cooperatively by a thread group (one warp or one
// CTA).  Parallel ordering: round-robin tournament, n/2 disjoint rotations
// per round; each round applies all column rotations, then all row
// rotations (they commute because the pairs are disjoint), then writes the
// exact 2x2 results.  Quadratic convergence; the sweep count is capped.
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
  int p, q;     // q < 0: no rotation
};

// A: n x n (row stride lda), V: n x n (row stride ldv) initialised here to the
// identity.  rot: scratch for n/2 + 1 rotations, scratch: reduction scratch.
// Returns the number of sweeps used (> max_sweeps: not converged).
template <class G>
__device__ int jacobi_eigh(const G& g, cd* A, int lda, cd* V, int ldv, int n, JacobiRot* rot, double* scratch,
                           int max_sweeps, double rel_tol) {
  const int tid = g.rank(), nt = g.size();
  for (int t = tid; t < n * n; t += nt) {
    const int r = t / n, c = t - r * n;
    V[r * ldv + c] = mk(r == c ? 1.0 : 0.0, 0.0);
  }
  for (int i = tid; i < n; i += nt) A[i * lda + i].y = 0.0;
  g.sync();
  if (n <= 1) return 0;
  const int n2 = n + (n & 1);
  const int m = n2 - 1;
  const int np = n2 / 2;
  int sweep = 0;
  for (; sweep <= max_sweeps; sweep++) {
    double off = 0.0, tot = 0.0;
    for (int t = tid; t < n * n; t += nt) {
      const int r = t / n, c = t - r * n;
      const double a2 = nrm2(A[r * lda + c]);
      tot += a2;
      if (r != c) off += a2;
    }
    off = g.sum(off, scratch);
    tot = g.sum(tot, scratch);
    if (off <= rel_tol * rel_tol * tot || off == 0.0) break;
    if (sweep == max_sweeps) { sweep++; break; }
    for (int r = 0; r < m; r++) {
      for (int i = tid; i < np; i += nt) {
        int a, b;
        if (i == 0) { a = r; b = m; }
        else { a = (r + i) % m; b = (r - i + m) % m; }
        const int p = min(a, b), q = max(a, b);
        JacobiRot R;
        R.p = p; R.q = -1;
        if (q < n) {
          const cd c = A[p * lda + q];
          const double ac = sqrt(nrm2(c));
          const double app = A[p * lda + p].x, aqq = A[q * lda + q].x;
          if (ac > 1e-300) {
            const double tau = (aqq - app) / (2.0 * ac);
            const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            const double cs = 1.0 / sqrt(1.0 + t * t);
            const double sn = t * cs;
            R.cs = cs;
            R.se = mk(sn * c.x / ac, sn * c.y / ac);
            R.app = app - t * ac;
            R.aqq = aqq + t * ac;
            R.q = q;
          }
        }
        rot[i] = R;
      }
      g.sync();
      // A <- A J and V <- V J (columns p, q)
      for (int t = tid; t < np * n; t += nt) {
        const int i = t / n, row = t - i * n;
        const JacobiRot R = rot[i];
        if (R.q < 0) continue;
        const cd x = A[row * lda + R.p], y = A[row * lda + R.q];
        // x cs - y sn e^{-i phi} ;  x sn e^{i phi} + y cs
        A[row * lda + R.p] = mk(R.cs * x.x - (y.x * R.se.x + y.y * R.se.y), R.cs * x.y - (y.y * R.se.x - y.x * R.se.y));
        A[row * lda + R.q] = x * R.se + R.cs * y;
        const cd vx = V[row * ldv + R.p], vy = V[row * ldv + R.q];
        V[row * ldv + R.p] = mk(R.cs * vx.x - (vy.x * R.se.x + vy.y * R.se.y), R.cs * vx.y - (vy.y * R.se.x - vy.x * R.se.y));
        V[row * ldv + R.q] = vx * R.se + R.cs * vy;
      }
      g.sync();
      // A <- J^H A (rows p, q)
      for (int t = tid; t < np * n; t += nt) {
        const int i = t / n, col = t - i * n;
        const JacobiRot R = rot[i];
        if (R.q < 0) continue;
        const cd x = A[R.p * lda + col], y = A[R.q * lda + col];
        // cs x - sn e^{i phi} y ;  sn e^{-i phi} x + cs y
        A[R.p * lda + col] = R.cs * x - R.se * y;
        A[R.q * lda + col] = mk(R.se.x * x.x + R.se.y * x.y + R.cs * y.x, R.se.x * x.y - R.se.y * x.x + R.cs * y.y);
      }
      g.sync();
      for (int i = tid; i < np; i += nt) {
        const JacobiRot R = rot[i];
        if (R.q < 0) continue;
        A[R.p * lda + R.q] = mk(0, 0);
        A[R.q * lda + R.p] = mk(0, 0);
        A[R.p * lda + R.p] = mk(R.app, 0);
        A[R.q * lda + R.q] = mk(R.aqq, 0);
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
