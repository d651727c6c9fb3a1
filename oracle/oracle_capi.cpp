// oracle_capi.cpp -- flat C entry points of the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, by the smoke check and by the
// CPU-baseline leg of bench.py, always as the checker.  Never part of the
// product path.
//
// prec selects the limb count (1 double, 2 double-double, 4 quad-double),
// cplx selects complex numbers (re limbs then im limbs).  Every array is
// flat, row-major and limb-interleaved.
#include <vector>
#include <cstdlib>
#include "oracle_core.hpp"

using namespace orc;

#define ORC_DISPATCH(prec, cplx, CALL)              \
  do {                                              \
    if (!(cplx)) {                                  \
      if ((prec) == 1) { typedef double T; CALL; }  \
      else if ((prec) == 2) { typedef dd T; CALL; } \
      else if ((prec) == 4) { typedef qd T; CALL; } \
      else return -1;                               \
    } else {                                        \
      if ((prec) == 1) { typedef cx<double> T; CALL; } \
      else if ((prec) == 2) { typedef cx<dd> T; CALL; } \
      else if ((prec) == 4) { typedef cx<qd> T; CALL; } \
      else return -1;                               \
    }                                               \
  } while (0)

template <class T> static std::vector<T> unpack(const double *p, long n) {
  std::vector<T> v(n);
  for (long i = 0; i < n; ++i) v[i] = ld<T>(p, i);
  return v;
}
template <class T> static void pack(double *p, const std::vector<T> &v) {
  for (long i = 0; i < (long)v.size(); ++i) st<T>(p, i, v[i]);
}

template <class T> static int conv_t(int deg, const double *x, const double *y, double *z) {
  auto X = unpack<T>(x, deg + 1), Y = unpack<T>(y, deg + 1);
  std::vector<T> Z(deg + 1);
  conv(deg, X.data(), Y.data(), Z.data());
  pack(z, Z);
  return 0;
}

// batch of nsys systems of dim polynomials; polynomial (s,p) owns the
// monomials mon_off[s*dim+p] .. mon_off[s*dim+p+1]-1.
template <class T>
static int system_t(int nsys, int dim, int deg, int maxvar, const int *mon_off, const int *nvr,
                    const int *idx, const int *exps, const double *cst, const double *cff,
                    const double *input, double *output) {
  const long n1 = deg + 1;
  const int W = limbs<T>::n;
  for (int s = 0; s < nsys; ++s) {
    auto X = unpack<T>(input + (long)s * dim * n1 * W, dim * n1);
    std::vector<T> out((dim + 1) * n1);
    for (int p = 0; p < dim; ++p) {
      const long sp = (long)s * dim + p;
      const int m0 = mon_off[sp], nb = mon_off[sp + 1] - m0;
      auto C = unpack<T>(cst + sp * n1 * W, n1);
      auto F = unpack<T>(cff + (long)m0 * n1 * W, (long)nb * n1);
      poly_evaldiff(dim, deg, nb, nvr + m0, idx + (long)m0 * maxvar, exps + (long)m0 * maxvar, maxvar,
                    C.data(), F.data(), X.data(), out.data());
      pack(output + sp * (dim + 1) * n1 * W, out);
    }
  }
  return 0;
}

template <class T>
static int baqr_t(int nrows, int ncols, int szt, int nbt, const double *A, double *Q, double *R) {
  auto Av = unpack<T>(A, (long)nrows * ncols);
  std::vector<T> Qv((long)nrows * nrows), Rv((long)nrows * ncols);
  blocked_houseqr(nrows, ncols, szt, nbt, Av.data(), Qv.data(), Rv.data());
  pack(Q, Qv);
  pack(R, Rv);
  return 0;
}

template <class T>
static int houseqr_t(int nrows, int ncols, const double *A, double *Q, double *R) {
  auto Av = unpack<T>(A, (long)nrows * ncols);
  std::vector<T> Qv((long)nrows * nrows), Rv((long)nrows * ncols);
  houseqr(nrows, ncols, Av.data(), Qv.data(), Rv.data());
  pack(Q, Qv);
  pack(R, Rv);
  return 0;
}

template <class T> static int tabs_t(int dim, int szt, int nbt, double *U, double *b, double *x) {
  auto Uv = unpack<T>(U, (long)dim * dim);
  auto bv = unpack<T>(b, dim);
  std::vector<T> xv(dim);
  upper_tiled_solver(dim, szt, nbt, Uv.data(), bv.data(), xv.data());
  pack(U, Uv);
  pack(b, bv);
  pack(x, xv);
  return 0;
}

template <class T>
static int bals_t(int dim, int degp1, int tailidx, const double *mat, double *rhs, double *sol, double *Q,
                  double *R, int *flags) {
  auto M = unpack<T>(mat, (long)degp1 * dim * dim);
  auto B = unpack<T>(rhs, (long)degp1 * dim);
  auto X = unpack<T>(sol, (long)degp1 * dim);
  auto Qv = unpack<T>(Q, (long)dim * dim);
  auto Rv = unpack<T>(R, (long)dim * dim);
  bals_state st{flags[0], flags[1], flags[2], flags[3], flags[4]};
  bals_solve(dim, degp1, tailidx, M.data(), B.data(), X.data(), Qv.data(), Rv.data(), &st);
  pack(rhs, B);
  pack(sol, X);
  pack(Q, Qv);
  pack(R, Rv);
  flags[0] = st.zeroQ; flags[1] = st.noqr; flags[2] = st.upidx; flags[3] = st.bsidx; flags[4] = st.newtail;
  return 0;
}

// One Newton step on a single system at working degree deg (row form):
// Newton/dbl2_newton_method.cpp:429 (dbl2_row_newton_qrstep, host mode)
// and :134 (dbl2_update_newton_qrstep): evaluate, map to funval/jacval
// (Newton/dbl2_systems_host.cpp:709), rhs = -funval, solve, then
// x[i][j] += dx[j][i] for j >= newtail-1 (dbl2_newton_testers.cpp:116).
// series: dim x (maxdeg+1); flags: zeroQ, noqr, upidx, bsidx, tailidx.
template <class T>
static int newton_t(int dim, int deg, int maxdeg, int maxvar, const int *mon_off, const int *nvr,
                    const int *idx, const int *exps, const double *cst, const double *cff, double *series,
                    double *Qd, double *Rd, int *flags) {
  const int W = limbs<T>::n;
  const long n1 = deg + 1, nmax = maxdeg + 1;
  std::vector<T> X((long)dim * n1);
  for (int i = 0; i < dim; ++i)
    for (int k = 0; k < n1; ++k) X[i * n1 + k] = ld<T>(series, i * nmax + k);
  std::vector<T> out((dim + 1) * n1), jac(n1 * dim * dim), rhs(n1 * dim), sol(n1 * dim);
  for (int p = 0; p < dim; ++p) {
    const int m0 = mon_off[p], nb = mon_off[p + 1] - m0;
    std::vector<T> C(n1), F((long)nb * n1);
    for (int k = 0; k < n1; ++k) C[k] = ld<T>(cst, p * nmax + k);
    for (int m = 0; m < nb; ++m)
      for (int k = 0; k < n1; ++k) F[m * n1 + k] = ld<T>(cff, (long)(m0 + m) * nmax + k);
    poly_evaldiff(dim, deg, nb, nvr + m0, idx + (long)m0 * maxvar, exps + (long)m0 * maxvar, maxvar, C.data(),
                  F.data(), X.data(), out.data());
    for (int k = 0; k < n1; ++k) {
      rhs[k * dim + p] = -out[dim * n1 + k];
      for (int j = 0; j < dim; ++j) jac[(k * dim + p) * dim + j] = out[j * n1 + k];
    }
  }
  auto Qv = unpack<T>(Qd, (long)dim * dim);
  auto Rv = unpack<T>(Rd, (long)dim * dim);
  bals_state bs{flags[0], flags[1], 0, 0, flags[4]};
  bals_solve(dim, (int)n1, flags[4], jac.data(), rhs.data(), sol.data(), Qv.data(), Rv.data(), &bs);
  for (int j = bs.newtail - 1; j < n1; ++j)
    for (int i = 0; i < dim; ++i) X[i * n1 + j] = X[i * n1 + j] + sol[j * dim + i];
  for (int i = 0; i < dim; ++i)
    for (int k = 0; k < n1; ++k) st<T>(series, i * nmax + k, X[i * n1 + k]);
  pack(Qd, Qv);
  pack(Rd, Rv);
  flags[0] = bs.zeroQ; flags[1] = bs.noqr; flags[2] = bs.upidx; flags[3] = bs.bsidx; flags[4] = bs.newtail;
  (void)W;
  return 0;
}

extern "C" {

int orc_conv(int prec, int cplx, int deg, const double *x, const double *y, double *z) {
  ORC_DISPATCH(prec, cplx, return conv_t<T>(deg, x, y, z));
  return -1;
}

int orc_system_evaldiff(int prec, int cplx, int nsys, int dim, int deg, int maxvar, const int *mon_off,
                        const int *nvr, const int *idx, const int *exps, const double *cst, const double *cff,
                        const double *input, double *output) {
  ORC_DISPATCH(prec, cplx,
               return system_t<T>(nsys, dim, deg, maxvar, mon_off, nvr, idx, exps, cst, cff, input, output));
  return -1;
}

int orc_blocked_houseqr(int prec, int cplx, int nrows, int ncols, int szt, int nbt, const double *A, double *Q,
                        double *R) {
  ORC_DISPATCH(prec, cplx, return baqr_t<T>(nrows, ncols, szt, nbt, A, Q, R));
  return -1;
}

int orc_houseqr(int prec, int cplx, int nrows, int ncols, const double *A, double *Q, double *R) {
  ORC_DISPATCH(prec, cplx, return houseqr_t<T>(nrows, ncols, A, Q, R));
  return -1;
}

int orc_upper_tiled_solver(int prec, int cplx, int dim, int szt, int nbt, double *U, double *b, double *x) {
  ORC_DISPATCH(prec, cplx, return tabs_t<T>(dim, szt, nbt, U, b, x));
  return -1;
}

int orc_bals_solve(int prec, int cplx, int dim, int degp1, int tailidx, const double *mat, double *rhs,
                   double *sol, double *Q, double *R, int *flags) {
  ORC_DISPATCH(prec, cplx, return bals_t<T>(dim, degp1, tailidx, mat, rhs, sol, Q, R, flags));
  return -1;
}

int orc_newton_step(int prec, int cplx, int dim, int deg, int maxdeg, int maxvar, const int *mon_off,
                    const int *nvr, const int *idx, const int *exps, const double *cst, const double *cff,
                    double *series, double *Q, double *R, int *flags) {
  ORC_DISPATCH(prec, cplx,
               return newton_t<T>(dim, deg, maxdeg, maxvar, mon_off, nvr, idx, exps, cst, cff, series, Q, R,
                                  flags));
  return -1;
}

// Octo-double arithmetic of this oracle: op 0 add, 1 mul, 2 div, 3 multiply
// by the double b[8k]; n numbers of eight limbs each.
int orc_od_binop(int op, int n, const double *a, const double *b, double *out) {
  for (int k = 0; k < n; ++k) {
    od x, y, z;
    load(a + 8 * k, x);
    load(b + 8 * k, y);
    if (op == 0) z = x + y;
    else if (op == 1) z = x * y;
    else if (op == 2) z = x / y;
    else if (op == 3) z = mul_d(x, y.x[0]);
    else return -1;
    store(out + 8 * k, z);
  }
  return 0;
}

}  // extern "C"
