// ref_harness.cpp -- flat-array C entry points over PHCpack's own host code.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together
// with the reference's host sources (read in place from the reference
// tree, never copied) into oracle/_ref/libphcref.so.  It serves two
// purposes: pinning the oracle restatement (oracle_core.hpp) against the
// reference itself, and generating the golden fixtures under tests/golden.
//
// The harness converts between this project's limb-interleaved flat arrays
// and the reference's separate-limb double*, double** and double*** arrays.
// The composition code below is this project's; every arithmetic routine
// it calls is the reference's.
#include <vector>
#include <cstring>
#include <cstdlib>
#include "double_double_functions.h"
#include "quad_double_functions.h"
#include "octo_double_functions.h"
#include "dbl2_convolutions_host.h"
#include "dbl2_monomials_host.h"
#include "dbl4_convolutions_host.h"
#include "dbl4_monomials_host.h"
#include "dbl2_factorizations.h"
#include "dbl4_factorizations.h"
#include "dbl2_baqr_host.h"
#include "dbl4_baqr_host.h"
#include "dbl2_tabs_host.h"
#include "dbl4_tabs_host.h"
#include "dbl2_bals_host.h"
#include "dbl4_bals_host.h"

namespace {

// C = number of component arrays (limbs x (1 + complex)); component c of
// element i sits at flat[i*C + c].
struct Vec {
  int C;
  long n;
  std::vector<std::vector<double> > d;
  double *p[8];
  Vec(int C_, long n_) : C(C_), n(n_), d(C_, std::vector<double>(n_ > 0 ? n_ : 1, 0.0)) {
    for (int c = 0; c < C; ++c) p[c] = d[c].data();
  }
  void in(const double *f) {
    for (long i = 0; i < n; ++i)
      for (int c = 0; c < C; ++c) d[c][i] = f[i * C + c];
  }
  void out(double *f) const {
    for (long i = 0; i < n; ++i)
      for (int c = 0; c < C; ++c) f[i * C + c] = d[c][i];
  }
};
struct Mat {
  int C;
  long r, k;
  std::vector<std::vector<double> > d;
  std::vector<std::vector<double *> > rows;
  double **p[8];
  Mat(int C_, long r_, long k_) : C(C_), r(r_), k(k_), d(C_, std::vector<double>(r_ * k_, 0.0)), rows(C_) {
    for (int c = 0; c < C; ++c) {
      rows[c].resize(r);
      for (long i = 0; i < r; ++i) rows[c][i] = d[c].data() + i * k;
      p[c] = rows[c].data();
    }
  }
  void in(const double *f) {
    for (long i = 0; i < r * k; ++i)
      for (int c = 0; c < C; ++c) d[c][i] = f[i * C + c];
  }
  void out(double *f) const {
    for (long i = 0; i < r * k; ++i)
      for (int c = 0; c < C; ++c) f[i * C + c] = d[c][i];
  }
};
struct Mat3 {
  int C;
  long s;
  std::vector<Mat *> m;
  std::vector<std::vector<double **> > lay;
  double ***p[8];
  Mat3(int C_, long s_, long r, long k) : C(C_), s(s_), lay(C_) {
    for (long i = 0; i < s; ++i) m.push_back(new Mat(C, r, k));
    for (int c = 0; c < C; ++c) {
      lay[c].resize(s);
      for (long i = 0; i < s; ++i) lay[c][i] = m[i]->p[c];
      p[c] = lay[c].data();
    }
  }
  ~Mat3() {
    for (auto q : m) delete q;
  }
  void in(const double *f) {
    const long blk = m[0]->r * m[0]->k * C;
    for (long i = 0; i < s; ++i) m[i]->in(f + i * blk);
  }
};

#define E2(a) a[0], a[1]
#define E4(a) a[0], a[1], a[2], a[3]
#define E8(a) a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7]

void product(int prec, int cplx, int deg, double **x, double **y, double **z) {
  if (prec == 2 && !cplx) CPU_dbl2_product(deg, E2(x), E2(y), E2(z));
  if (prec == 2 && cplx) CPU_cmplx2_product(deg, E4(x), E4(y), E4(z));
  if (prec == 4 && !cplx) CPU_dbl4_product(deg, E4(x), E4(y), E4(z));
  if (prec == 4 && cplx) CPU_cmplx4_product(deg, E8(x), E8(y), E8(z));
}
void evaldiff(int prec, int cplx, int dim, int nvr, int deg, int *idx, double **cff, double ***in, double ***out) {
  if (prec == 2 && !cplx) CPU_dbl2_evaldiff(dim, nvr, deg, idx, E2(cff), E2(in), E2(out));
  if (prec == 2 && cplx) CPU_cmplx2_evaldiff(dim, nvr, deg, idx, E4(cff), E4(in), E4(out));
  if (prec == 4 && !cplx) CPU_dbl4_evaldiff(dim, nvr, deg, idx, E4(cff), E4(in), E4(out));
  if (prec == 4 && cplx) CPU_cmplx4_evaldiff(dim, nvr, deg, idx, E8(cff), E8(in), E8(out));
}
// a <- factor * a on every real limb group (re and im scaled alike), with
// ddf_mul_d_dd / qdf_mul_qd_d as in Newton/dbl2_systems_host.cpp:88-110
void scale(int prec, int cplx, double f, double **a, int i) {
  const int parts = cplx ? 2 : 1;
  for (int q = 0; q < parts; ++q) {
    double **c = a + q * prec;
    if (prec == 2) {
      double h, l;
      ddf_mul_d_dd(f, c[0][i], c[1][i], &h, &l);
      c[0][i] = h; c[1][i] = l;
    } else {
      double r0, r1, r2, r3;
      qdf_mul_qd_d(c[0][i], c[1][i], c[2][i], c[3][i], f, &r0, &r1, &r2, &r3);
      c[0][i] = r0; c[1][i] = r1; c[2][i] = r2; c[3][i] = r3;
    }
  }
}
// a <- a + b on all real limb groups, ddf_inc / qdf_inc
void inc(int prec, int cplx, double **a, int i, double **b, int j) {
  const int parts = cplx ? 2 : 1;
  for (int q = 0; q < parts; ++q) {
    double **x = a + q * prec, **y = b + q * prec;
    if (prec == 2)
      ddf_inc(&x[0][i], &x[1][i], y[0][j], y[1][j]);
    else
      qdf_inc(&x[0][i], &x[1][i], &x[2][i], &x[3][i], y[0][j], y[1][j], y[2][j], y[3][j]);
  }
}

}  // namespace

extern "C" {

// Batch of systems, same conventions as orc_system_evaldiff.  Per monomial:
// common factors by CPU_dbl2_product, CPU_dbl2_evaldiff, derivative scaling
// by the exponent, accumulation by ddf_inc (the reference's common-factor
// method, Newton/dbl2_systems_host.cpp:18-110, applied per monomial).
int ref_system_evaldiff(int prec, int cplx, int nsys, int dim, int deg, int maxvar, const int *mon_off,
                        const int *nvr, const int *idx, const int *exps, const double *cst, const double *cff,
                        const double *input, double *output) {
  if (prec != 2 && prec != 4) return -1;
  const int C = prec * (cplx ? 2 : 1);
  const long n1 = deg + 1;
  for (int s = 0; s < nsys; ++s) {
    Mat X(C, dim, n1);
    X.in(input + (long)s * dim * n1 * C);
    double **xin[8];
    for (int c = 0; c < C; ++c) xin[c] = X.p[c];
    for (int p = 0; p < dim; ++p) {
      const long sp = (long)s * dim + p;
      Mat O(C, dim + 1, n1);     // polynomial output
      Mat M(C, dim + 1, n1);     // one monomial's output
      Vec c(C, n1), acc(C, n1);
      Vec cs(C, n1);
      cs.in(cst + sp * n1 * C);
      for (long i = 0; i < n1; ++i)
        for (int q = 0; q < C; ++q) O.d[q][dim * n1 + i] = cs.d[q][i];
      double **opp[8], **mpp[8];
      for (int q = 0; q < C; ++q) { opp[q] = O.p[q]; mpp[q] = M.p[q]; }
      for (int m = mon_off[sp]; m < mon_off[sp + 1]; ++m) {
        c.in(cff + (long)m * n1 * C);
        int ix[64];
        const int k = nvr[m];
        for (int v = 0; v < k; ++v) ix[v] = idx[(long)m * maxvar + v];
        bool common = false;
        for (int v = 0; v < k; ++v)
          for (int e = 1; e < exps[(long)m * maxvar + v]; ++e) {
            double *xv[8];
            for (int q = 0; q < C; ++q) xv[q] = X.p[q][ix[v]];
            product(prec, cplx, deg, xv, c.p, acc.p);
            for (int q = 0; q < C; ++q) c.d[q] = acc.d[q];
            common = true;
          }
        evaldiff(prec, cplx, dim, k, deg, ix, c.p, xin, mpp);
        if (common)
          for (int v = 0; v < k; ++v) {
            double *row[8];
            for (int q = 0; q < C; ++q) row[q] = M.p[q][ix[v]];
            for (long i = 0; i < n1; ++i) scale(prec, cplx, (double)exps[(long)m * maxvar + v], row, (int)i);
          }
        {
          double *a[8], *b[8];
          for (int q = 0; q < C; ++q) { a[q] = O.p[q][dim]; b[q] = M.p[q][dim]; }
          for (long i = 0; i < n1; ++i) inc(prec, cplx, a, (int)i, b, (int)i);
        }
        for (int v = 0; v < k; ++v) {
          double *a[8], *b[8];
          for (int q = 0; q < C; ++q) { a[q] = O.p[q][ix[v]]; b[q] = M.p[q][ix[v]]; }
          for (long i = 0; i < n1; ++i) inc(prec, cplx, a, (int)i, b, (int)i);
        }
      }
      O.out(output + sp * (dim + 1) * n1 * C);
    }
  }
  return 0;
}

int ref_blocked_houseqr(int prec, int cplx, int nrows, int ncols, int szt, int nbt, const double *A, double *Q,
                        double *R) {
  const int C = prec * (cplx ? 2 : 1);
  Mat Am(C, nrows, ncols), Qm(C, nrows, nrows), Rm(C, nrows, ncols);
  Am.in(A);
  double lap;
  if (prec == 2 && !cplx) CPU_dbl2_blocked_houseqr(nrows, ncols, szt, nbt, E2(Am.p), E2(Qm.p), E2(Rm.p), &lap, false);
  else if (prec == 2 && cplx) CPU_cmplx2_blocked_houseqr(nrows, ncols, szt, nbt, E4(Am.p), E4(Qm.p), E4(Rm.p), &lap, false);
  else if (prec == 4 && !cplx) CPU_dbl4_blocked_houseqr(nrows, ncols, szt, nbt, E4(Am.p), E4(Qm.p), E4(Rm.p), &lap, false);
  else if (prec == 4 && cplx) CPU_cmplx4_blocked_houseqr(nrows, ncols, szt, nbt, E8(Am.p), E8(Qm.p), E8(Rm.p), &lap, false);
  else return -1;
  Qm.out(Q);
  Rm.out(R);
  return 0;
}

int ref_upper_tiled_solver(int prec, int cplx, int dim, int szt, int nbt, double *U, double *b, double *x) {
  const int C = prec * (cplx ? 2 : 1);
  Mat Um(C, dim, dim);
  Vec bv(C, dim), xv(C, dim);
  Um.in(U);
  bv.in(b);
  double lap;
  if (prec == 2 && !cplx) CPU_dbl2_upper_tiled_solver(dim, szt, nbt, E2(Um.p), E2(bv.p), E2(xv.p), &lap);
  else if (prec == 2 && cplx) CPU_cmplx2_upper_tiled_solver(dim, szt, nbt, E4(Um.p), E4(bv.p), E4(xv.p), &lap);
  else if (prec == 4 && !cplx) CPU_dbl4_upper_tiled_solver(dim, szt, nbt, E4(Um.p), E4(bv.p), E4(xv.p), &lap);
  else if (prec == 4 && cplx) CPU_cmplx4_upper_tiled_solver(dim, szt, nbt, E8(Um.p), E8(bv.p), E8(xv.p), &lap);
  else return -1;
  Um.out(U);
  bv.out(b);
  xv.out(x);
  return 0;
}

// flags: zeroQ, noqr, upidx, bsidx, newtail (in/out), as orc_bals_solve
int ref_bals_solve(int prec, int cplx, int dim, int degp1, int tailidx, const double *mat, double *rhs,
                   double *sol, double *Q, double *R, int *flags) {
  const int C = prec * (cplx ? 2 : 1);
  Mat3 M(C, degp1, dim, dim);
  M.in(mat);
  Mat B(C, degp1, dim), X(C, degp1, dim), Qm(C, dim, dim), Rm(C, dim, dim);
  B.in(rhs);
  X.in(sol);
  Qm.in(Q);
  Rm.in(R);
  Vec w(C, dim);
  bool zeroQ = flags[0] != 0, noqr = flags[1] != 0;
  int up = 0, bs = 0, nt = flags[4];
  if (prec == 2 && !cplx)
    CPU_dbl2_qrbs_solve(dim, degp1, tailidx, E2(M.p), E2(B.p), E2(X.p), E2(Qm.p), E2(Rm.p), E2(w.p), &zeroQ, &noqr, &up, &bs, &nt, 0);
  else if (prec == 2 && cplx)
    CPU_cmplx2_qrbs_solve(dim, degp1, tailidx, E4(M.p), E4(B.p), E4(X.p), E4(Qm.p), E4(Rm.p), E4(w.p), &zeroQ, &noqr, &up, &bs, &nt, 0);
  else if (prec == 4 && !cplx)
    CPU_dbl4_qrbs_solve(dim, degp1, tailidx, E4(M.p), E4(B.p), E4(X.p), E4(Qm.p), E4(Rm.p), E4(w.p), &zeroQ, &noqr, &up, &bs, &nt, 0);
  else if (prec == 4 && cplx)
    CPU_cmplx4_qrbs_solve(dim, degp1, tailidx, E8(M.p), E8(B.p), E8(X.p), E8(Qm.p), E8(Rm.p), E8(w.p), &zeroQ, &noqr, &up, &bs, &nt, 0);
  else
    return -1;
  B.out(rhs);
  X.out(sol);
  Qm.out(Q);
  Rm.out(R);
  flags[0] = zeroQ; flags[1] = noqr; flags[2] = up; flags[3] = bs; flags[4] = nt;
  return 0;
}

// The residual of the linearised system by the reference's host code
// (Newton/dbl2_bals_host.cpp:548 CPU_dbl2_linear_residue and its cmplx2,
// dbl4, cmplx4 twins): res rows tailidx..degp1-1, resmax prec doubles.
int ref_linear_residue(int prec, int cplx, int dim, int degp1, int tailidx, const double *mat, const double *rhs,
                       const double *sol, double *res, double *resmax) {
  const int C = prec * (cplx ? 2 : 1);
  Mat3 M(C, degp1, dim, dim);
  M.in(mat);
  Mat B(C, degp1, dim), X(C, degp1, dim), Rv(C, degp1, dim);
  B.in(rhs);
  X.in(sol);
  Rv.in(res);
  double mx[4] = {0.0, 0.0, 0.0, 0.0};
  if (prec == 2 && !cplx)
    CPU_dbl2_linear_residue(dim, degp1, tailidx, E2(M.p), E2(B.p), E2(X.p), E2(Rv.p), &mx[0], &mx[1], 0);
  else if (prec == 2 && cplx)
    CPU_cmplx2_linear_residue(dim, degp1, tailidx, E4(M.p), E4(B.p), E4(X.p), E4(Rv.p), &mx[0], &mx[1], 0);
  else if (prec == 4 && !cplx)
    CPU_dbl4_linear_residue(dim, degp1, tailidx, E4(M.p), E4(B.p), E4(X.p), E4(Rv.p), &mx[0], &mx[1], &mx[2],
                            &mx[3], 0);
  else if (prec == 4 && cplx)
    CPU_cmplx4_linear_residue(dim, degp1, tailidx, E8(M.p), E8(B.p), E8(X.p), E8(Rv.p), &mx[0], &mx[1], &mx[2],
                              &mx[3], 0);
  else
    return -1;
  Rv.out(res);
  for (int l = 0; l < prec; ++l) resmax[l] = mx[l];
  return 0;
}

// Octo-double arithmetic of the reference (Norms/octo_double_functions.cpp):
// op 0 add, 1 mul, 2 div, 3 multiply by the double b[0]; n numbers of eight
// limbs each in a, b, out.
int ref_od_binop(int op, int n, const double *a, const double *b, double *out) {
  for (int k = 0; k < n; ++k) {
    const double *x = a + 8 * k, *y = b + 8 * k;
    double *z = out + 8 * k;
    if (op == 0)
      odf_add(x[0], x[1], x[2], x[3], x[4], x[5], x[6], x[7], y[0], y[1], y[2], y[3], y[4], y[5], y[6], y[7], &z[0],
              &z[1], &z[2], &z[3], &z[4], &z[5], &z[6], &z[7]);
    else if (op == 1)
      odf_mul(x[0], x[1], x[2], x[3], x[4], x[5], x[6], x[7], y[0], y[1], y[2], y[3], y[4], y[5], y[6], y[7], &z[0],
              &z[1], &z[2], &z[3], &z[4], &z[5], &z[6], &z[7]);
    else if (op == 2)
      odf_div(x[0], x[1], x[2], x[3], x[4], x[5], x[6], x[7], y[0], y[1], y[2], y[3], y[4], y[5], y[6], y[7], &z[0],
              &z[1], &z[2], &z[3], &z[4], &z[5], &z[6], &z[7]);
    else if (op == 3)
      odf_mul_od_d(x[0], x[1], x[2], x[3], x[4], x[5], x[6], x[7], y[0], &z[0], &z[1], &z[2], &z[3], &z[4], &z[5],
                   &z[6], &z[7]);
    else
      return -1;
  }
  return 0;
}

}  // extern "C"
