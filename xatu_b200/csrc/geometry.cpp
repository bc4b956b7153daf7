#include "geometry.h"

#include <cmath>

namespace xatu_geo {

static const double kPi = 3.141592653589793;

double norm3(const double* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

// Solve the small dense system A x = b (n <= 3) by Gaussian elimination with
// partial pivoting.  A is row-major n x n.
static bool solve_small(int n, const double* A, const double* b, double* x) {
  double M[3][4];
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < n; j++) M[i][j] = A[i * n + j];
    M[i][n] = b[i];
  }
  for (int c = 0; c < n; c++) {
    int piv = c;
    for (int r = c + 1; r < n; r++)
      if (std::fabs(M[r][c]) > std::fabs(M[piv][c])) piv = r;
    if (std::fabs(M[piv][c]) < 1e-300) return false;
    if (piv != c)
      for (int j = 0; j <= n; j++) std::swap(M[c][j], M[piv][j]);
    for (int r = c + 1; r < n; r++) {
      const double f = M[r][c] / M[c][c];
      for (int j = c; j <= n; j++) M[r][j] -= f * M[c][j];
    }
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = M[i][n];
    for (int j = i + 1; j < n; j++) s -= M[i][j] * x[j];
    x[i] = s / M[i][i];
  }
  return true;
}

bool reciprocal_lattice(int ndim, const double* bravais, double* recip) {
  for (int i = 0; i < 3 * ndim; i++) recip[i] = 0.0;
  if (ndim == 1) {
    const double n2 = bravais[0] * bravais[0] + bravais[1] * bravais[1] + bravais[2] * bravais[2];
    if (n2 == 0) return false;
    for (int j = 0; j < 3; j++) recip[j] = 2. * kPi * bravais[j] / n2;
    return true;
  }
  // a_i . b_j = 2 pi delta_ij using the first ndim Cartesian components
  double A[9];
  for (int i = 0; i < ndim; i++)
    for (int j = 0; j < ndim; j++) A[i * ndim + j] = bravais[3 * i + j];
  for (int i = 0; i < ndim; i++) {
    double rhs[3] = {0, 0, 0}, x[3] = {0, 0, 0};
    rhs[i] = 2 * kPi;
    if (!solve_small(ndim, A, rhs, x)) return false;
    for (int j = 0; j < ndim; j++) recip[3 * i + j] = x[j];
  }
  return true;
}

double unit_cell_area(int ndim, const double* b) {
  if (ndim == 1) return norm3(b);
  const double c[3] = {b[1] * b[5] - b[2] * b[4], b[2] * b[3] - b[0] * b[5], b[0] * b[4] - b[1] * b[3]};
  if (ndim == 2) return norm3(c);
  return c[0] * b[6] + c[1] * b[7] + c[2] * b[8];
}

std::vector<double> combinations(int n, int ndim, bool centered) {
  const int shift = centered ? n / 2 : 0;
  long total = 1;
  for (int d = 0; d < ndim; d++) total *= n;
  std::vector<double> out((size_t)total * ndim);
  for (long i = 0; i < total; i++) {
    long rem = i;
    for (int d = 0; d < ndim; d++) {
      out[(size_t)i * ndim + d] = (double)(rem % n) - shift;
      rem /= n;
    }
  }
  return out;
}

// Digits of the combinations in the order combinations() lists them (dimension 0 fastest), kept as a counter
// that the caller advances, so that no list is built and no division is done per combination.
struct CombinationCounter {
  int n, ndim, shift, dig[3] = {0, 0, 0};
  CombinationCounter(int n_, int ndim_, int shift_) : n(n_), ndim(ndim_), shift(shift_) {}
  void get(double* c) const {
    for (int d = 0; d < ndim; d++) c[d] = (double)dig[d] - shift;
  }
  void next() {
    for (int d = 0; d < ndim; d++) {
      if (++dig[d] < n) return;
      dig[d] = 0;
    }
  }
};

std::vector<double> mp_mesh(int ndim, const double* recip, int n) {
  long nk = 1;
  for (int d = 0; d < ndim; d++) nk *= n;
  std::vector<double> k((size_t)nk * 3, 0.0);
  CombinationCounter cnt(n, ndim, 0);
  for (long i = 0; i < nk; i++, cnt.next()) {
    double cc[3];
    cnt.get(cc);
    for (int j = 0; j < ndim; j++) {
      double c = cc[j];
      if (n % 2 == 1) c += 1. / 2;
      const double f = (2 * c - n) / (2 * n);
      for (int x = 0; x < 3; x++) k[(size_t)i * 3 + x] += f * recip[3 * j + x];
    }
  }
  return k;
}

std::vector<double> reduced_mesh(int ndim, const double* recip, int n, int factor) {
  long nk = 1;
  for (int d = 0; d < ndim; d++) nk *= n;
  std::vector<double> k((size_t)nk * 3, 0.0);
  CombinationCounter cnt(n, ndim, 0);
  for (long i = 0; i < nk; i++, cnt.next()) {
    double cc[3];
    cnt.get(cc);
    for (int j = 0; j < ndim; j++) {
      double c = cc[j];
      if (n % 2 == 1) c += 1. / 2;
      const double f = (2 * c - n) / (2 * n * factor);
      for (int x = 0; x < 3; x++) k[(size_t)i * 3 + x] += f * recip[3 * j + x];
    }
  }
  return k;
}

std::vector<double> truncate_supercell(int ndim, const double* basis, int ncell, double radius) {
  long nc = 1;
  for (int d = 0; d < ndim; d++) nc *= ncell;
  std::vector<double> cells;
  cells.reserve((size_t)nc * 3);
  CombinationCounter cnt(ncell, ndim, ncell / 2);
  for (long i = 0; i < nc; i++, cnt.next()) {
    double cc[3];
    cnt.get(cc);
    double v[3] = {0, 0, 0};
    for (int j = 0; j < ndim; j++)
      for (int x = 0; x < 3; x++) v[x] += cc[j] * basis[3 * j + x];
    if (norm3(v) < radius + 1E-5) {
      cells.push_back(v[0]);
      cells.push_back(v[1]);
      cells.push_back(v[2]);
    }
  }
  return cells;
}

bool inverse_gram(int ndim, const double* recip, double* inv) {
  double G[9];
  for (int i = 0; i < ndim; i++)
    for (int j = 0; j < ndim; j++)
      G[i * ndim + j] = recip[3 * i] * recip[3 * j] + recip[3 * i + 1] * recip[3 * j + 1] + recip[3 * i + 2] * recip[3 * j + 2];
  for (int c = 0; c < ndim; c++) {
    double e[3] = {0, 0, 0}, x[3] = {0, 0, 0};
    e[c] = 1.0;
    if (!solve_small(ndim, G, e, x)) return false;
    for (int r = 0; r < ndim; r++) inv[r * ndim + c] = x[r];
  }
  return true;
}

int equivalent_point(int ndim, const double* recip, const double* inv, int n, const double* k) {
  double ind[3] = {0, 0, 0};
  for (int i = 0; i < ndim; i++) ind[i] = recip[3 * i] * k[0] + recip[3 * i + 1] * k[1] + recip[3 * i + 2] * k[2];
  double acc = 0.0, stride = 1.0;
  for (int i = 0; i < ndim; i++) {
    double c = 0.0;
    for (int j = 0; j < ndim; j++) c += inv[i * ndim + j] * ind[j];
    c *= 2 * n;
    if (n % 2 == 1) c -= 1;
    c = std::round(c);
    if (c >= n) c -= 2 * n;
    else if (c < -n) c += 2 * n;
    c += n;
    c /= 2;
    acc += c * stride;
    stride *= n;
  }
  return (int)acc;
}

}  // namespace xatu_geo
