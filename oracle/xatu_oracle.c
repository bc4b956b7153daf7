/*
 * CPU oracle for the BSE build path -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain C (FP64, OpenMP) restatement of the reference algorithm for the
 * Bethe-Salpeter kernel assembly of Xatu v1.3.1.  Only the test-suite, the
 * smoke check and the CPU-baseline leg of the benchmark load this file's
 * shared object; the product library never links or calls it.
 *
 * Every routine cites the reference function it restates (file:line within
 * the xatu project).  Loop order and arithmetic follow the reference so that
 * the oracle reproduces the reference's numbers to rounding; storage is flat
 * (no Armadillo), and the per-element heap copies of the reference are gone.
 *
 * Layouts (all row-major / C order):
 *   complex numbers      interleaved (re, im) doubles
 *   motif                natoms x 4   (x, y, z, species)
 *   orbital offsets      natoms + 1   (first orbital of each atom)
 *   eigvec stacks        nk x nb x norb complex  (band b of k = row [k][b])
 *   eigval stacks        nk x nb
 *   motif FT stacks      nq x na x na complex
 *   BSE matrix           N x N complex, full Hermitian
 */
#define _GNU_SOURCE 1
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.141592653589793
#define ORC_EC 1.6021766E-19
#define ORC_EPS0 8.8541878E-12

typedef struct {
  int ndim;
  int natoms;
  int norb;
  const double *motif;       /* natoms x 4 */
  const int *orb_offset;     /* natoms + 1 */
  double a1norm;             /* |a_1| (Lattice::a) */
  double b1norm;             /* |b_1| */
  double unit_cell_area;
  double eps_m, eps_s, r0;
  double regularization;
  double cutoff;             /* ExcitonTB::cutoff_, in units of |a_1| */
  double total_cells;        /* (ncell * factor)^ndim */
} orc_params;

/* Struve function H0(x), x >= 0.  Restates ExcitonTB::STVH0
 * (ExcitonTB.cpp:306-337), which is routine STVH0 of Zhang & Jin,
 * "Computation of Special Functions" (Wiley 1996): power series for x <= 20
 * (at most 60 terms, relative stop 1e-12), otherwise the asymptotic series of
 * H0 - Y0 plus the Zhang-Jin rational approximation of Y0 for large x. */
double orc_stvh0(double x) {
  double s = 1.0, r = 1.0;
  if (x <= 20.0) {
    double a0 = 2.0 * x / ORC_PI;
    for (int k = 1; k < 61; k++) {
      r = -r * x / (2.0 * k + 1.0) * x / (2.0 * k + 1.0);
      s = s + r;
      if (fabs(r) < fabs(s) * 1.0e-12) break;
    }
    return a0 * s;
  }
  int km = (int)(0.5 * (x + 1.0));
  if (x >= 50.0) km = 25;
  for (int k = 1; k <= km; k++) {
    r = -r * pow((2.0 * k - 1.0) / x, 2);
    s = s + r;
    if (fabs(r) < fabs(s) * 1.0e-12) break;
  }
  double t = 4.0 / x;
  double t2 = t * t;
  double p0 = ((((-.37043e-5 * t2 + .173565e-4) * t2 - .487613e-4) * t2 + .17343e-3) * t2 -
               0.1753062e-2) * t2 + .3989422793;
  double q0 = t * (((((.32312e-5 * t2 - 0.142078e-4) * t2 + 0.342468e-4) * t2 - 0.869791e-4) * t2 +
                    0.4564324e-3) * t2 - 0.0124669441);
  double ta0 = x - 0.25 * ORC_PI;
  double by0 = 2.0 / sqrt(x) * (p0 * sin(ta0) + q0 * cos(ta0));
  return 2.0 / (ORC_PI * x) * s + by0;
}

/* Keldysh potential in eV.  Restates ExcitonTB::keldysh (ExcitonTB.cpp:347-366). */
double orc_keldysh(const orc_params *p, double r) {
  double eps_bar = (p->eps_m + p->eps_s) / 2;
  double cutoff = p->a1norm * p->cutoff + 1E-5;
  double R = fabs(r) / p->r0;
  if (r == 0) {
    double sh0 = orc_stvh0(p->regularization / p->r0);
    return ORC_EC / (8E-10 * ORC_EPS0 * eps_bar * p->r0) * (sh0 - y0(p->regularization / p->r0));
  } else if (r > cutoff) {
    return 0.0;
  }
  double sh0 = orc_stvh0(R);
  return ORC_EC / (8E-10 * ORC_EPS0 * eps_bar * p->r0) * (sh0 - y0(R));
}

/* Coulomb potential in eV.  Restates ExcitonTB::coulomb (ExcitonTB.cpp:374-381). */
double orc_coulomb(const orc_params *p, double r) {
  double cutoff = p->a1norm * p->cutoff + 1E-5;
  r = fabs(r);
  if (r > cutoff) return 0.0;
  return (r != 0) ? ORC_EC / (4E-10 * ORC_PI * ORC_EPS0 * r)
                  : ORC_EC * 1E10 / (4 * ORC_PI * ORC_EPS0 * p->regularization);
}

static double orc_potential(const orc_params *p, int kind, double r) {
  return kind == 1 ? orc_coulomb(p, r) : orc_keldysh(p, r);
}

/* Fourier transform of the Keldysh potential.  Restates ExcitonTB::keldyshFT
 * (ExcitonTB.cpp:410-426). */
double orc_keldysh_ft(const orc_params *p, const double q[3]) {
  double eps_bar = (p->eps_m + p->eps_s) / 2;
  double eps = p->b1norm / p->total_cells;
  double qnorm = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
  double potential = (qnorm < eps) ? 0.0 : 1 / (qnorm * (1 + p->r0 * qnorm));
  return potential * ORC_EC * 1E10 / (2 * ORC_EPS0 * eps_bar * p->unit_cell_area * p->total_cells);
}

/* Motif lattice Fourier transform matrix at q.  Restates
 * ExcitonTB::motifFourierTransform / motifFTMatrix (ExcitonTB.cpp:438-476):
 * upper triangle summed cell by cell, lower triangle = conjugate. */
static void orc_motif_ft_matrix(const orc_params *p, int kind, const double *q, int ncells,
                                const double *cells, double *out /* na x na complex */) {
  int na = p->natoms;
  for (int fa = 0; fa < na; fa++) {
    for (int sa = fa; sa < na; sa++) {
      const double *t1 = p->motif + 4 * fa;
      const double *t2 = p->motif + 4 * sa;
      double vr = 0.0, vi = 0.0;
      for (int n = 0; n < ncells; n++) {
        const double *c = cells + 3 * n;
        double d0 = c[0] + t1[0] - t2[0];
        double d1 = c[1] + t1[1] - t2[1];
        double d2 = c[2] + t1[2] - t2[2];
        double module = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        double v = orc_potential(p, kind, module);
        double ph = q[0] * c[0] + q[1] * c[1] + q[2] * c[2];
        vr += v * cos(ph);
        vi += v * sin(ph);
      }
      vr /= p->total_cells;
      vi /= p->total_cells;
      out[2 * (fa * na + sa)] = vr;
      out[2 * (fa * na + sa) + 1] = vi;
      out[2 * (sa * na + fa)] = vr;
      out[2 * (sa * na + fa) + 1] = -vi;
    }
  }
}

/* ftMotifStack over all q of the mesh (ExcitonTB.cpp:761-781, OpenMP over q
 * exactly like the reference) or a single matrix (ftMotifQ, :783-786). */
void orc_motif_ft_stack(const orc_params *p, int kind, int nq, const double *q, int ncells,
                        const double *cells, double *out) {
  int na = p->natoms;
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < nq; i++)
    orc_motif_ft_matrix(p, kind, q + 3 * i, ncells, cells, out + 2 * (size_t)i * na * na);
}

/* Lattice::findEquivalentPointBZ (Lattice.cpp:251-279).  recip: ndim x 3
 * reciprocal vectors, inv: ndim x ndim inverse of recip*recip^T, n: ncell*factor. */
int orc_find_equivalent(int ndim, const double *recip, const double *inv, int n, const double *k) {
  double ind[3] = {0, 0, 0}, coefs[3] = {0, 0, 0};
  for (int i = 0; i < ndim; i++)
    ind[i] = recip[3 * i] * k[0] + recip[3 * i + 1] * k[1] + recip[3 * i + 2] * k[2];
  for (int i = 0; i < ndim; i++) {
    double s = 0.0;
    for (int j = 0; j < ndim; j++) s += inv[i * ndim + j] * ind[j];
    coefs[i] = s * 2 * n;
  }
  int index = 0;
  int cells_array[3] = {1, n, n * n};
  double acc = 0.0;
  for (int i = 0; i < ndim; i++) {
    double c = (n % 2 == 1) ? coefs[i] - 1 : coefs[i];
    c = round(c);
    if (c >= n)
      c -= 2 * n;
    else if (c < -n)
      c += 2 * n;
    c += n;
    c /= 2;
    acc += c * cells_array[i];
  }
  index = (int)acc;
  return index;
}

/* realSpaceInteractionTerm (ExcitonTB.cpp:520-548):
 *   rho1(a) = sum_{o in a} conj(C1_o) C3_o,  rho2(a) = sum_{o in a} conj(C2_o) C4_o,
 *   term = rho1^T V rho2 (arma::dot: no conjugation). */
static void orc_realspace_term(const orc_params *p, const double *c1, const double *c2, const double *c3,
                               const double *c4, const double *V, double *tr, double *ti) {
  int na = p->natoms;
  double r1r[64], r1i[64], r2r[64], r2i[64];
  for (int a = 0; a < na; a++) {
    double ar = 0, ai = 0, br = 0, bi = 0;
    for (int o = p->orb_offset[a]; o < p->orb_offset[a + 1]; o++) {
      /* conj(c1) * c3 */
      ar += c1[2 * o] * c3[2 * o] + c1[2 * o + 1] * c3[2 * o + 1];
      ai += c1[2 * o] * c3[2 * o + 1] - c1[2 * o + 1] * c3[2 * o];
      /* conj(c2) * c4 */
      br += c2[2 * o] * c4[2 * o] + c2[2 * o + 1] * c4[2 * o + 1];
      bi += c2[2 * o] * c4[2 * o + 1] - c2[2 * o + 1] * c4[2 * o];
    }
    r1r[a] = ar; r1i[a] = ai; r2r[a] = br; r2i[a] = bi;
  }
  double sr = 0, si = 0;
  for (int a = 0; a < na; a++) {
    double mr = 0, mi = 0; /* (V rho2)(a) */
    for (int b = 0; b < na; b++) {
      double vr = V[2 * (a * na + b)], vi = V[2 * (a * na + b) + 1];
      mr += vr * r2r[b] - vi * r2i[b];
      mi += vr * r2i[b] + vi * r2r[b];
    }
    sr += r1r[a] * mr - r1i[a] * mi;
    si += r1r[a] * mi + r1i[a] * mr;
  }
  *tr = sr;
  *ti = si;
}

/* blochCoherenceFactor (ExcitonTB.cpp:598-621):
 *   I = sum_o conj(c1_o) c2_o exp(i (k1 - k2 + G) . tau_atom(o)). */
static void orc_bloch_factor(const orc_params *p, const double *c1, const double *c2, const double *k1,
                             const double *k2, const double *G, double *fr, double *fi) {
  double sr = 0, si = 0;
  for (int a = 0; a < p->natoms; a++) {
    const double *tau = p->motif + 4 * a;
    double ph = (k1[0] - k2[0] + G[0]) * tau[0] + (k1[1] - k2[1] + G[1]) * tau[1] +
                (k1[2] - k2[2] + G[2]) * tau[2];
    double cr = cos(ph), ci = sin(ph);
    for (int o = p->orb_offset[a]; o < p->orb_offset[a + 1]; o++) {
      double xr = c1[2 * o] * c2[2 * o] + c1[2 * o + 1] * c2[2 * o + 1];
      double xi = c1[2 * o] * c2[2 * o + 1] - c1[2 * o + 1] * c2[2 * o];
      sr += xr * cr - xi * ci;
      si += xr * ci + xi * cr;
    }
  }
  *fr = sr;
  *fi = si;
}

/* reciprocalInteractionTerm (ExcitonTB.cpp:562-587):
 *   term = sum_G Ic conj(Iv) keldyshFT(k - k2 + G). */
static void orc_reciprocal_term(const orc_params *p, const double *cK, const double *cK2, const double *cKQ,
                                const double *cK2Q, const double *k, const double *k2, const double *kQ,
                                const double *k2Q, int nG, const double *G, double *tr, double *ti) {
  double sr = 0, si = 0;
  for (int g = 0; g < nG; g++) {
    const double *Gv = G + 3 * g;
    double icr, ici, ivr, ivi;
    orc_bloch_factor(p, cKQ, cK2Q, kQ, k2Q, Gv, &icr, &ici);
    orc_bloch_factor(p, cK, cK2, k, k2, Gv, &ivr, &ivi);
    double q[3] = {k[0] - k2[0] + Gv[0], k[1] - k2[1] + Gv[1], k[2] - k2[2] + Gv[2]};
    double v = orc_keldysh_ft(p, q);
    /* Ic * conj(Iv) * v */
    double pr = icr * ivr + ici * ivi;
    double pi = ici * ivr - icr * ivi;
    sr += pr * v;
    si += pi * v;
  }
  *tr = sr;
  *ti = si;
}

typedef struct {
  int N;                 /* BSE dimension */
  const int *basis_v;    /* N: stack column of the valence band */
  const int *basis_c;    /* N: stack column of the conduction band */
  const int *basis_k;    /* N: k index */
  int nk, nb;
  const double *kpoints; /* nk x 3 */
  const double *eigvec;  /* nk x nb x norb complex, bands at k */
  const double *eigvecQ; /* bands at k + Q */
  const double *eigval;  /* nk x nb */
  const double *eigvalQ;
  double scissor;
  int exchange;
  int mode;              /* 0 realspace, 1 reciprocalspace */
  /* realspace */
  const double *ft_stack; /* nmesh x na x na complex */
  const double *ft_Q;     /* na x na complex */
  const double *recip;    /* ndim x 3 */
  const double *inv_recip;/* ndim x ndim */
  int n_eff;              /* ncell * factor */
  /* reciprocal */
  int nG;
  const double *G;        /* nG x 3 */
  double Q[3];
} orc_bse_input;

/* BShamiltonian (ExcitonTB.cpp:840-921): upper triangle element by element,
 * H_ii = (scissor + Ec - Ev)/2 - (D - X)/2, H_ij = -(D - X), then
 * H = H + H^dagger.  OpenMP over rows (the reference runs the packed triangle
 * with one OpenMP loop; the element arithmetic is identical). */
void orc_bse_build(const orc_params *p, const orc_bse_input *in, double *H) {
  int N = in->N;
  int norb = p->norb, nb = in->nb;
#pragma omp parallel for schedule(dynamic, 8)
  for (int i = 0; i < N; i++) {
    int ki = in->basis_k[i], v = in->basis_v[i], c = in->basis_c[i];
    const double *coefsK = in->eigvec + 2 * ((size_t)ki * nb + v) * norb;
    const double *coefsKQ = in->eigvecQ + 2 * ((size_t)ki * nb + c) * norb;
    for (int j = i; j < N; j++) {
      int kj = in->basis_k[j], v2 = in->basis_v[j], c2 = in->basis_c[j];
      const double *coefsK2 = in->eigvec + 2 * ((size_t)kj * nb + v2) * norb;
      const double *coefsK2Q = in->eigvecQ + 2 * ((size_t)kj * nb + c2) * norb;
      double Dr = 0, Di = 0, Xr = 0, Xi = 0;
      if (in->mode == 0) {
        const double *k1 = in->kpoints + 3 * ki, *k2 = in->kpoints + 3 * kj;
        double dk[3] = {k2[0] - k1[0], k2[1] - k1[1], k2[2] - k1[2]};
        int eff = orc_find_equivalent(p->ndim, in->recip, in->inv_recip, in->n_eff, dk);
        const double *V = in->ft_stack + 2 * (size_t)eff * p->natoms * p->natoms;
        orc_realspace_term(p, coefsKQ, coefsK2, coefsK2Q, coefsK, V, &Dr, &Di);
        if (in->exchange) orc_realspace_term(p, coefsKQ, coefsK2, coefsK, coefsK2Q, in->ft_Q, &Xr, &Xi);
      } else {
        const double *k = in->kpoints + 3 * ki, *k2 = in->kpoints + 3 * kj;
        orc_reciprocal_term(p, coefsK, coefsK2, coefsKQ, coefsK2Q, k, k2, k, k2, in->nG, in->G, &Dr, &Di);
        if (in->exchange) {
          double k2Q[3] = {k2[0] + in->Q[0], k2[1] + in->Q[1], k2[2] + in->Q[2]};
          double kQ[3] = {k[0] + in->Q[0], k[1] + in->Q[1], k[2] + in->Q[2]};
          orc_reciprocal_term(p, coefsK2Q, coefsK2, coefsKQ, coefsK, k2Q, k2, kQ, k, in->nG, in->G, &Xr, &Xi);
        }
      }
      double hr, hi;
      if (i == j) {
        double ec_ = in->eigvalQ[(size_t)ki * nb + c], ev_ = in->eigval[(size_t)ki * nb + v];
        hr = (in->scissor + ec_ - ev_) / 2. - (Dr - Xr) / 2.;
        hi = -(Di - Xi) / 2.;
        H[2 * ((size_t)i * N + i)] = hr + hr;
        H[2 * ((size_t)i * N + i) + 1] = hi - hi;
      } else {
        hr = -(Dr - Xr);
        hi = -(Di - Xi);
        H[2 * ((size_t)i * N + j)] = hr;
        H[2 * ((size_t)i * N + j) + 1] = hi;
        H[2 * ((size_t)j * N + i)] = hr;
        H[2 * ((size_t)j * N + i) + 1] = -hi;
      }
    }
  }
}

/* Rows [row0, row1) of the upper triangle only (bounded CPU-baseline sample:
 * same per-element work as orc_bse_build, no mirror write). */
void orc_bse_build_rows(const orc_params *p, const orc_bse_input *in, int row0, int row1, double *rows) {
  int N = in->N;
  int norb = p->norb, nb = in->nb;
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = row0; i < row1; i++) {
    int ki = in->basis_k[i], v = in->basis_v[i], c = in->basis_c[i];
    const double *coefsK = in->eigvec + 2 * ((size_t)ki * nb + v) * norb;
    const double *coefsKQ = in->eigvecQ + 2 * ((size_t)ki * nb + c) * norb;
    double *out = rows + 2 * (size_t)(i - row0) * N;
    for (int j = i; j < N; j++) {
      int kj = in->basis_k[j], v2 = in->basis_v[j], c2 = in->basis_c[j];
      const double *coefsK2 = in->eigvec + 2 * ((size_t)kj * nb + v2) * norb;
      const double *coefsK2Q = in->eigvecQ + 2 * ((size_t)kj * nb + c2) * norb;
      double Dr = 0, Di = 0, Xr = 0, Xi = 0;
      if (in->mode == 0) {
        const double *k1 = in->kpoints + 3 * ki, *k2 = in->kpoints + 3 * kj;
        double dk[3] = {k2[0] - k1[0], k2[1] - k1[1], k2[2] - k1[2]};
        int eff = orc_find_equivalent(p->ndim, in->recip, in->inv_recip, in->n_eff, dk);
        const double *V = in->ft_stack + 2 * (size_t)eff * p->natoms * p->natoms;
        orc_realspace_term(p, coefsKQ, coefsK2, coefsK2Q, coefsK, V, &Dr, &Di);
        if (in->exchange) orc_realspace_term(p, coefsKQ, coefsK2, coefsK, coefsK2Q, in->ft_Q, &Xr, &Xi);
      } else {
        const double *k = in->kpoints + 3 * ki, *k2 = in->kpoints + 3 * kj;
        orc_reciprocal_term(p, coefsK, coefsK2, coefsKQ, coefsK2Q, k, k2, k, k2, in->nG, in->G, &Dr, &Di);
        if (in->exchange) {
          double k2Q[3] = {k2[0] + in->Q[0], k2[1] + in->Q[1], k2[2] + in->Q[2]};
          double kQ[3] = {k[0] + in->Q[0], k[1] + in->Q[1], k[2] + in->Q[2]};
          orc_reciprocal_term(p, coefsK2Q, coefsK2, coefsKQ, coefsK, k2Q, k2, kQ, k, in->nG, in->G, &Xr, &Xi);
        }
      }
      out[2 * j] = -(Dr - Xr);
      out[2 * j + 1] = -(Di - Xi);
    }
  }
}

int orc_abi_version(void) { return 1; }
