// Shared definitions of the B200 BSE engine: complex helpers, physical
// constants, the device-side potentials and the launch-parameter structs.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#define XATU_PI 3.141592653589793
#define XATU_EC 1.6021766E-19
#define XATU_EPS0 8.8541878E-12

// Upper bounds of the fast kernels (checked on the host before launch).
#define XATU_MAX_ATOMS 16
#define XATU_MAX_ORB 64
#define XATU_MAX_BANDS 8   // per side (valence or conduction)

// ------------------------------------------------ programmatic dependent launch
// A kernel launched with programmatic stream serialisation (xatu_launch_chained) may start while its
// predecessor on the stream is still running: xatu_grid_wait() returns once the predecessor grid has
// completed and its writes are visible, so every kernel of such a chain calls it before its first access to
// global memory.  xatu_grid_release() then lets the next kernel of the chain be scheduled (its blocks wait in
// their own xatu_grid_wait()).  Outside a chained launch both are no-ops.
__device__ __forceinline__ void xatu_grid_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void xatu_grid_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void xatu_grid_chain() {
  xatu_grid_wait();
  xatu_grid_release();
}

// ----------------------------------------------------------------- complex
struct cd { double x, y; };
struct cf { float x, y; };

__host__ __device__ __forceinline__ cd mk(double a, double b) { return cd{a, b}; }
__host__ __device__ __forceinline__ cd operator+(cd a, cd b) { return cd{a.x + b.x, a.y + b.y}; }
__host__ __device__ __forceinline__ cd operator-(cd a, cd b) { return cd{a.x - b.x, a.y - b.y}; }
__host__ __device__ __forceinline__ cd operator*(cd a, cd b) { return cd{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__host__ __device__ __forceinline__ cd operator*(double s, cd a) { return cd{s * a.x, s * a.y}; }
__host__ __device__ __forceinline__ cd conj(cd a) { return cd{a.x, -a.y}; }
// conj(a) * b
__host__ __device__ __forceinline__ cd cmulc(cd a, cd b) { return cd{a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x}; }
__host__ __device__ __forceinline__ double nrm2(cd a) { return a.x * a.x + a.y * a.y; }

// Scalar-type generic complex (T = double or float) used by the assembly.
template <typename T> struct cplx { T x, y; };
template <typename T> __device__ __forceinline__ cplx<T> cadd(cplx<T> a, cplx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T> __device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// acc += a * b
template <typename T> __device__ __forceinline__ void cfma(cplx<T>& acc, cplx<T> a, cplx<T> b) {
  acc.x = fma(a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y); acc.y = fma(a.y, b.x, acc.y);
}
// acc += conj(a) * b
template <typename T> __device__ __forceinline__ void cfmac(cplx<T>& acc, cplx<T> a, cplx<T> b) {
  acc.x = fma(a.x, b.x, acc.x); acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y); acc.y = fma(-a.y, b.x, acc.y);
}

// ----------------------------------------------------------------- potentials
struct PotParams {
  double a1norm;          // |a_1|
  double b1norm;          // |b_1|
  double area;            // unit-cell area
  double eps_m, eps_s, r0;
  double regularization;
  double cutoff;          // in units of |a_1|
  double total_cells;     // (ncell * factor)^ndim
};

// Struve H0(x) for x >= 0 by the method of Zhang & Jin, "Computation of
// Special Functions" (1996), routine STVH0: power series up to x = 20 (60
// terms at most, relative stop 1e-12), then the asymptotic series of
// H0 - Y0 together with Zhang & Jin's rational approximation of Y0.  The
// reference uses the same method (ExcitonTB.cpp:306-337), so the engine
// reproduces its values to rounding.
__host__ __device__ inline double struve_h0(double x) {
  double s = 1.0, r = 1.0;
  if (x <= 20.0) {
    const double a0 = 2.0 * x / XATU_PI;
    for (int k = 1; k < 61; k++) {
      const double d = 2.0 * k + 1.0;
      r = -r * x / d * x / d;
      s += r;
      if (fabs(r) < fabs(s) * 1.0e-12) break;
    }
    return a0 * s;
  }
  int km = (int)(0.5 * (x + 1.0));
  if (x >= 50.0) km = 25;
  for (int k = 1; k <= km; k++) {
    const double u = (2.0 * k - 1.0) / x;
    r = -r * (u * u);
    s += r;
    if (fabs(r) < fabs(s) * 1.0e-12) break;
  }
  const double t = 4.0 / x, t2 = t * t;
  const double p0 = ((((-.37043e-5 * t2 + .173565e-4) * t2 - .487613e-4) * t2 + .17343e-3) * t2 - 0.1753062e-2) * t2 +
                    .3989422793;
  const double q0 =
      t * (((((.32312e-5 * t2 - 0.142078e-4) * t2 + 0.342468e-4) * t2 - 0.869791e-4) * t2 + 0.4564324e-3) * t2 -
           0.0124669441);
  const double ta0 = x - 0.25 * XATU_PI;
  const double by0 = 2.0 / sqrt(x) * (p0 * sin(ta0) + q0 * cos(ta0));
  return 2.0 / (XATU_PI * x) * s + by0;
}

// Derivative d/dx of struve_h0: the exact derivative of the same truncated
// approximation (same branch, same number of series terms), so that it is
// consistent with finite differences of struve_h0 itself.
//   x <= 20:  H0 = (2/pi) sum_k r_k x,    r_k ~ x^{2k}   ->  H0' = (2/pi) sum_k (2k+1) r_k
//   x  > 20:  A  = (2/pi) sum_k r_k / x,  r_k ~ x^{-2k}  ->  A'  = -(2/pi) sum_k (2k+1) r_k / x^2
//             by0 = 2 x^{-1/2} (p0 sin th + q0 cos th), th = x - pi/4, p0 = P(t^2),
//             q0 = t Qp(t^2), t = 4/x, differentiated term by term.
__host__ __device__ inline double struve_h0_dx(double x) {
  double s = 1.0, r = 1.0, sk = 0.0;   // sk = sum_k k r_k
  if (x <= 20.0) {
    for (int k = 1; k < 61; k++) {
      const double d = 2.0 * k + 1.0;
      r = -r * x / d * x / d;
      s += r;
      sk += k * r;
      if (fabs(r) < fabs(s) * 1.0e-12) break;
    }
    return (2.0 / XATU_PI) * (s + 2.0 * sk);
  }
  int km = (int)(0.5 * (x + 1.0));
  if (x >= 50.0) km = 25;
  for (int k = 1; k <= km; k++) {
    const double u = (2.0 * k - 1.0) / x;
    r = -r * (u * u);
    s += r;
    sk += k * r;
    if (fabs(r) < fabs(s) * 1.0e-12) break;
  }
  const double dA = -(2.0 / (XATU_PI * x * x)) * (s + 2.0 * sk);
  const double t = 4.0 / x, t2 = t * t;
  const double P = ((((-.37043e-5 * t2 + .173565e-4) * t2 - .487613e-4) * t2 + .17343e-3) * t2 - 0.1753062e-2) * t2 +
                   .3989422793;
  const double dP = (((5.0 * -.37043e-5 * t2 + 4.0 * .173565e-4) * t2 - 3.0 * .487613e-4) * t2 + 2.0 * .17343e-3) * t2 -
                    0.1753062e-2;
  const double Qp = ((((.32312e-5 * t2 - 0.142078e-4) * t2 + 0.342468e-4) * t2 - 0.869791e-4) * t2 + 0.4564324e-3) * t2 -
                    0.0124669441;
  const double dQp = (((5.0 * .32312e-5 * t2 - 4.0 * 0.142078e-4) * t2 + 3.0 * 0.342468e-4) * t2 - 2.0 * 0.869791e-4) *
                         t2 +
                     0.4564324e-3;
  const double dt2 = -2.0 * t2 / x;   // d(t^2)/dx
  const double q0 = t * Qp;
  const double dp0 = dP * dt2;
  const double dq0 = (-t / x) * Qp + t * dQp * dt2;
  const double th = x - 0.25 * XATU_PI;
  const double sn = sin(th), cs = cos(th);
  const double g = P * sn + q0 * cs;
  const double dg = dp0 * sn + P * cs + dq0 * cs - q0 * sn;
  const double rs = 1.0 / sqrt(x);
  const double dby0 = -rs / x * g + 2.0 * rs * dg;
  return dA + dby0;
}

// Keldysh potential V(r) in eV (ExcitonTB::keldysh semantics, ExcitonTB.cpp:347-366):
// r = 0 uses the regularisation distance, r beyond |a1| * cutoff + 1e-5 is zero.
__device__ inline double keldysh_potential(const PotParams& p, double r) {
  const double eps_bar = (p.eps_m + p.eps_s) / 2;
  const double rc = p.a1norm * p.cutoff + 1E-5;
  const double pref = XATU_EC / (8E-10 * XATU_EPS0 * eps_bar * p.r0);
  if (r == 0) {
    const double x = p.regularization / p.r0;
    return pref * (struve_h0(x) - y0(x));
  }
  if (r > rc) return 0.0;
  const double x = fabs(r) / p.r0;
  return pref * (struve_h0(x) - y0(x));
}

// dV/dr0 of keldysh_potential.  With P = ec / (8e-10 eps0 eps_bar), rho = r (or
// the regularisation distance at r = 0) and x = rho / r0:
//   V = P / r0 f(x),  f = H0 - Y0,  f' = H0' + Y1
//   dV/dr0 = -P / r0^2 (f(x) + x f'(x)).
// (dV/deps_m = dV/deps_s = -V / (2 eps_bar) needs no table.)
__device__ inline double keldysh_potential_dr0(const PotParams& p, double r) {
  const double eps_bar = (p.eps_m + p.eps_s) / 2;
  const double rc = p.a1norm * p.cutoff + 1E-5;
  const double pref = XATU_EC / (8E-10 * XATU_EPS0 * eps_bar * p.r0 * p.r0);
  double x;
  if (r == 0) {
    x = p.regularization / p.r0;
  } else {
    if (r > rc) return 0.0;
    x = fabs(r) / p.r0;
  }
  const double f = struve_h0(x) - y0(x);
  const double df = struve_h0_dx(x) + y1(x);
  return -pref * (f + x * df);
}

// Coulomb potential in eV (ExcitonTB::coulomb semantics, ExcitonTB.cpp:374-381).
__device__ inline double coulomb_potential(const PotParams& p, double r) {
  const double rc = p.a1norm * p.cutoff + 1E-5;
  r = fabs(r);
  if (r > rc) return 0.0;
  return (r != 0) ? XATU_EC / (4E-10 * XATU_PI * XATU_EPS0 * r)
                  : XATU_EC * 1E10 / (4 * XATU_PI * XATU_EPS0 * p.regularization);
}

// Fourier transform of the Keldysh potential (ExcitonTB::keldyshFT semantics, ExcitonTB.cpp:410-426).
__device__ inline double keldysh_ft(const PotParams& p, double qx, double qy, double qz) {
  const double eps_bar = (p.eps_m + p.eps_s) / 2;
  const double eps = p.b1norm / p.total_cells;
  const double qn = sqrt(qx * qx + qy * qy + qz * qz);
  const double v = (qn < eps) ? 0.0 : 1 / (qn * (1 + p.r0 * qn));
  return v * XATU_EC * 1E10 / (2 * XATU_EPS0 * eps_bar * p.area * p.total_cells);
}

// dVt/dr0 of keldysh_ft: Vt ~ 1 / (|q| (1 + r0 |q|))  ->  dVt/dr0 = -Vt |q| / (1 + r0 |q|).
__device__ inline double keldysh_ft_dr0(const PotParams& p, double qx, double qy, double qz) {
  const double eps_bar = (p.eps_m + p.eps_s) / 2;
  const double eps = p.b1norm / p.total_cells;
  const double qn = sqrt(qx * qx + qy * qy + qz * qz);
  if (qn < eps) return 0.0;
  const double d = 1 + p.r0 * qn;
  return -1.0 / (d * d) * XATU_EC * 1E10 / (2 * XATU_EPS0 * eps_bar * p.area * p.total_cells);
}

// ----------------------------------------------------------------- k-difference -> mesh index
// Lattice::findEquivalentPointBZ semantics (Lattice.cpp:251-279) for the
// difference k2 - k1: reduced coordinates inv(B B^T) (B dk) scaled by 2n,
// odd-n shift, rounding half away from zero, wrap into [-n, n), (c + n) / 2.
struct EquivMap {
  int ndim;
  int n;            // ncell * factor
  double B[9];      // reciprocal vectors, ndim x 3
  double inv[9];    // inv(B B^T), ndim x ndim
};

__device__ __forceinline__ int equivalent_index(const EquivMap& m, double dx, double dy, double dz) {
  double ind[3];
  for (int i = 0; i < m.ndim; i++) ind[i] = m.B[3 * i] * dx + m.B[3 * i + 1] * dy + m.B[3 * i + 2] * dz;
  double acc = 0.0;
  double stride = 1.0;
  for (int i = 0; i < m.ndim; i++) {
    double c = 0.0;
    for (int j = 0; j < m.ndim; j++) c += m.inv[i * m.ndim + j] * ind[j];
    c *= 2 * m.n;
    if (m.n & 1) c -= 1;
    c = round(c);
    if (c >= m.n) c -= 2 * m.n;
    else if (c < -m.n) c += 2 * m.n;
    c += m.n;
    c /= 2;
    acc += c * stride;
    stride *= m.n;
  }
  return (int)acc;
}

// ----------------------------------------------------------------- Hermitian block storage of the mixed kernel
// The split-BF16 interaction kernel K of a mixed build keeps only its upper block triangle: with blocks of
// XATU_KBLOCK x XATU_KBLOCK elements, block (I, J) is stored for J >= I (the diagonal blocks in full); the
// rest of the N x ldk planes is never written or read.  K_rc for any (r, c) is K[r][c] where stored, else
// conj(K[c][r]).
#define XATU_KBLOCK 128
__host__ __device__ __forceinline__ bool xatu_kstored(long long r, long long c) {
  return (c / XATU_KBLOCK) >= (r / XATU_KBLOCK);
}

// ----------------------------------------------------------------- error flag
// Kernels never trap: out-of-contract indices are recorded in a device word the
// host reads after the stage.
enum {
  XATU_DEVERR_NONE = 0,
  XATU_DEVERR_INDEX = 1,
  XATU_DEVERR_NAN = 2,
  XATU_DEVERR_NOCONV = 4,
  XATU_DEVERR_OVERLAP = 8,
  XATU_DEVERR_DEGEN = 16   // degenerate band pair where an eigenvector derivative is needed
};
