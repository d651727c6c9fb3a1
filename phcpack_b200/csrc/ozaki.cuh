// ozaki.cuh -- multiple-double matrix products on FP64 tensor cores by
// error-free splitting (Ozaki's scheme), CTA level.
//
// C = A B with A (M x K) and B (K x N) in double-double or quad-double:
//  1. every row i of A gets an exponent E_i with |A_ik| < 2^E_i, every
//     column j of B an exponent F_j;
//  2. A is cut into s slices A = sum_p A^(p), A^(p)_ik a multiple of
//     u_p(i) = 2^(E_i - (p+1) beta) with |A^(p)_ik| <= (2^beta + 1) u_p(i),
//     by rounding the running remainder's leading limb to the grid u_p with
//     the add-and-subtract trick (x + sigma) - sigma, sigma = 1.5 2^52 u_p;
//     likewise B column by column;
//  3. for each order r = p + q < s the products A^(p) B^(q) are summed on
//     the FP64 tensor cores (mma.sync m8n8k4 f64).  All of them are integer
//     multiples of 2^(E_i + F_j - (r+2) beta) below (r+1) K (2^beta+1)^2
//     times that unit; with beta = 21, K <= 64 and s <= 11 this stays below
//     2^53, so every partial sum is exact;
//  4. the s exact order sums are added into the multiple-double result.
// The slices cover s*beta bits below the row / column maximum (231 bits for
// quad-double with s = 11, 126 for double-double with s = 6), so the product
// is accurate to the working precision relative to the row and column
// scales.  The reference has host-only splitting of this kind
// (TensorCore/splitting_doubles.h:22-110, vectored_double_doubles.h:43-340)
// and no GPU split GEMM.
#pragma once
#include "md.cuh"

namespace phc {

static const int kOzakiBeta = 21;

template <class R> struct ozaki_slices;
template <> struct ozaki_slices<double> { static const int s = 3; };
template <> struct ozaki_slices<md::dd> { static const int s = 6; };
template <> struct ozaki_slices<md::qd> { static const int s = 11; };

__device__ __forceinline__ void dmma_m8n8k4(double a, double b, double &c0, double &c1) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// limbs of a real number as an array
__device__ __forceinline__ void limbs_of(double a, double *x) { x[0] = a; }
__device__ __forceinline__ void limbs_of(const md::dd &a, double *x) { x[0] = a.hi; x[1] = a.lo; }
__device__ __forceinline__ void limbs_of(const md::qd &a, double *x) {
  for (int i = 0; i < 4; ++i) x[i] = a.x[i];
}

__device__ __forceinline__ int grid_exponent(double m) {
  // smallest E with m < 2^E (m > 0)
  return ilogb(m) + 1;
}

// Slice planes of an M x K operand (rows = the dimension with the common
// exponent): planes[p*Mp*Kp + i*Kp + k].  rows_are_M: true for A (exponent
// per row i), false for B stored as planes[p*Kp*Np + k*Np + j] with the
// exponent per column j.  get(i, k) returns the element as R.
template <class R, class Get>
__device__ void ozaki_split(int rows, int cols, int prow, int pcol, bool by_row, Get get, double *planes,
                            int *expo) {
  const int L = md::real_traits<R>::limbs;
  const int S = ozaki_slices<R>::s;
  // exponent per row (by_row) or per column
  const int nx = by_row ? rows : cols;
  for (int a = threadIdx.x; a < nx; a += blockDim.x) {
    double m = 0.0;
    const int ny = by_row ? cols : rows;
    for (int b = 0; b < ny; ++b) {
      double x[4];
      limbs_of(by_row ? get(a, b) : get(b, a), x);
      m = fmax(m, fabs(x[0]));
    }
    expo[a] = (m > 0.0) ? grid_exponent(m) : -1000000;
  }
  __syncthreads();
  const long plane = (long)prow * pcol;
  for (int t = threadIdx.x; t < prow * pcol; t += blockDim.x) {
    const int i = t / pcol, k = t % pcol;
    // (i, k) indexes the padded plane: rows of A / rows (k) of B
    double x[4] = {0.0, 0.0, 0.0, 0.0};
    int E = -1000000;
    bool inside;
    if (by_row) {
      inside = i < rows && k < cols;
      if (inside) { limbs_of(get(i, k), x); E = expo[i]; }
    } else {
      inside = i < rows && k < cols;
      if (inside) { limbs_of(get(i, k), x); E = expo[k]; }
    }
    for (int p = 0; p < S; ++p) {
      double sl = 0.0;
      if (inside && E > -1000000) {
        const double sigma = 1.5 * ldexp(1.0, E - (p + 1) * kOzakiBeta + 52);
        sl = md::sub(md::add(x[0], sigma), sigma);
        x[0] = md::sub(x[0], sl);  // exact: both on the grid of ulp(x[0])
        // renormalise the remainder so that x[0] leads again
        double e, s = x[L - 1];
        for (int l = L - 2; l >= 0; --l) {
          s = md::two_sum(x[l], s, e);
          x[l + 1] = e;
        }
        x[0] = s;
      }
      planes[p * plane + t] = sl;
    }
  }
  __syncthreads();
}

// out(i, j) = [out(i, j) +] (A B)(i, j) from the slice planes of A (Mp x Kp,
// exponent per row) and B (Kp x Np, exponent per column); one warp per 8x8
// output tile.  put(i, j, value) receives the multiple-double product.
template <class R, class Put>
__device__ void ozaki_mma(int M, int N, int Mp, int Kp, int Np, const double *Ap, const double *Bp, Put put) {
  typedef md::num<R, false> RN;
  const int S = ozaki_slices<R>::s;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int g = lane >> 2, tg = lane & 3;
  const long pa = (long)Mp * Kp, pb = (long)Kp * Np;
  const int tiles_n = Np / 8;
  for (int tile = warp; tile < (Mp / 8) * tiles_n; tile += nw) {
    const int i0 = (tile / tiles_n) * 8, j0 = (tile % tiles_n) * 8;
    R res0 = RN::zero(), res1 = RN::zero();
    for (int r = 0; r < S; ++r) {
      double c0 = 0.0, c1 = 0.0;
      for (int p = 0; p <= r; ++p) {
        const int q = r - p;
        const double *A = Ap + p * pa + (long)(i0 + g) * Kp;
        const double *B = Bp + q * pb + j0 + g;
        for (int k0 = 0; k0 < Kp; k0 += 4) dmma_m8n8k4(A[k0 + tg], B[(long)(k0 + tg) * Np], c0, c1);
      }
      res0 = RN::add(res0, RN::from(c0));
      res1 = RN::add(res1, RN::from(c1));
    }
    const int i = i0 + g, j = j0 + 2 * tg;
    if (i < M && j < N) put(i, j, res0);
    if (i < M && j + 1 < N) put(i, j + 1, res1);
  }
  __syncthreads();
}

__host__ __device__ inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

// Workspace (doubles) of one product with dimensions up to n
__host__ __device__ inline long ozaki_work_doubles(int n, int s) {
  const long np = round_up(n, 8);
  return (long)s * 2 * np * np + 2 * np;
}

// C = A B, the whole pipeline; get_a(i, k), get_b(k, j) read the operands,
// put(i, j, v) writes (or accumulates) the product.
template <class R, class GA, class GB, class Put>
__device__ void ozaki_gemm(int M, int N, int K, GA get_a, GB get_b, Put put, double *work) {
  const int S = ozaki_slices<R>::s;
  const int Mp = round_up(M, 8), Np = round_up(N, 8), Kp = round_up(K, 4);
  double *Ap = work;
  double *Bp = Ap + (long)S * Mp * Kp;
  int *ea = reinterpret_cast<int *>(Bp + (long)S * Kp * Np);
  int *eb = ea + Mp;
  ozaki_split<R>(M, K, Mp, Kp, true, get_a, Ap, ea);
  ozaki_split<R>(K, N, Kp, Np, false, get_b, Bp, eb);
  ozaki_mma<R>(M, N, Mp, Kp, Np, Ap, Bp, put);
}

}  // namespace phc
