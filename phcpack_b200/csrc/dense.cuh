// dense.cuh -- CTA-level multiple-double dense linear algebra: blocked
// Householder QR in WY form, inversion of the diagonal tiles of R and tiled
// back substitution, Q^H b, and the block lower-triangular Toeplitz solve of
// the power-series Newton step.
//
// One CTA owns one instance.  Matrices are row-major, limb-interleaved, in
// global memory (one instance's Q, R and WY panels stay resident in L2);
// shared memory holds the Householder vector, the reflector coefficients,
// the current solution vector and the reduction buffers.  Norms and dot
// products are warp-shuffle reductions followed by a shared-memory pass
// across warps.
#pragma once
#include "md.cuh"
#include "ozaki.cuh"

namespace phc {

template <class N>
__device__ __forceinline__ typename N::T ldn_at(const double *p, long i) {
  typename N::T a;
  md::ldn(p + i * N::width, a);
  return a;
}
template <class N>
__device__ __forceinline__ void stn_at(double *p, long i, const typename N::T &a) {
  md::stn(p + i * N::width, a);
}

template <class N>
__device__ __forceinline__ typename N::T warp_sum(typename N::T a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a = N::add(a, md::shfl_xor(a, o));
  return a;
}

__device__ __forceinline__ double warp_max(double a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
  return a;
}

// Block-wide sum, every thread gets the result.  red: shared scratch of
// (blockDim/32) numbers of width N::width.
template <class N>
__device__ typename N::T block_sum(typename N::T a, double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  a = warp_sum<N>(a);
  __syncthreads();
  if (lane == 0) stn_at<N>(red, warp, a);
  __syncthreads();
  typename N::T s = N::zero();
  for (int w = 0; w < nw; ++w) s = N::add(s, ldn_at<N>(red, w));
  __syncthreads();
  return s;
}

__device__ __forceinline__ double block_max(double a, double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  a = warp_max(a);
  __syncthreads();
  if (lane == 0) red[warp] = a;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < nw; ++w) s = fmax(s, red[w]);
  __syncthreads();
  return s;
}

// Block-wide minimum of one double per thread (any sign).
__device__ __forceinline__ double block_min(double a, double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a = fmin(a, __shfl_xor_sync(0xffffffffu, a, o));
  __syncthreads();
  if (lane == 0) red[warp] = a;
  __syncthreads();
  double s = red[0];
  for (int w = 1; w < nw; ++w) s = fmin(s, red[w]);
  __syncthreads();
  return s;
}

// max_i |leading limb| of v (complex: |re| + |im|): the "1-norm" of the
// reference's skip rules, Newton/dbl_onenorms_host.cpp:9,20
template <class N>
__device__ double block_maxnorm(int n, const double *v, double *red) {
  double a = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) a = fmax(a, N::lead(ldn_at<N>(v, i)));
  return block_max(a, red);
}

// Skip thresholds of the reference's least-squares solvers per precision:
// Newton/dbl_bals_host.cpp:36,199 (double: |b_0| + 1 == 1 in the head,
// 1e-15 in the tail), dbl2_bals_host.cpp:43,254 (1e-28),
// dbl4_bals_host.cpp:51,335 (1e-56).
template <class N>
__device__ __forceinline__ double skip_tol() {
  return N::tr::limbs == 1 ? 1.0e-15 : (N::tr::limbs == 2 ? 1.0e-28 : 1.0e-56);
}
template <class N>
__device__ __forceinline__ bool head_tiny(double nrm) {
  return N::tr::limbs == 1 ? (__dadd_rn(nrm, 1.0) == 1.0) : (nrm < skip_tol<N>());
}

// Shared-memory layout of one CTA (in doubles), sized by dense_smem_doubles.
struct dense_smem {
  double *v;     // Householder vector, n numbers
  double *w;     // n numbers: reflector products / right hand side
  double *x;     // n numbers: solution of one stage
  double *beta;  // szt reals (as numbers of width N::width)
  double *red;   // reduction scratch, 32 numbers
  double *misc;  // 8 numbers
};

template <class N>
__device__ dense_smem carve(double *sm, int n, int szt) {
  const int W = N::width;
  dense_smem s;
  s.v = sm;
  s.w = s.v + n * W;
  s.x = s.w + n * W;
  s.beta = s.x + n * W;
  s.red = s.beta + szt * W;
  s.misc = s.red + 32 * W;
  return s;
}
__host__ __device__ inline long dense_smem_doubles(int n, int szt, int W) { return (long)(3 * n + szt + 40) * W; }
// with the WY panels (Y, W, P, T) and the current column panel of R staged
// in shared memory as well
__host__ __device__ inline long dense_smem_doubles_staged(int n, int szt, int W) {
  return dense_smem_doubles(n, szt, W) + 5L * n * szt * W;
}

// Workspace in global memory per instance (numbers): Y, W, P (szt x n each),
// T (n x szt) and the inverted diagonal tiles of R (n x szt).
__host__ __device__ inline long dense_work_numbers(int n, int szt) { return 5L * n * szt; }

// Dot products shared by aligned groups of four lanes: output o of a pass
// is computed by the four lanes 4(o mod 8) .. +3 of warp o / 8, each summing
// every fourth term, then two xor shuffles add the four partial sums (the
// chains of dependent multiple-double operations are a quarter as long as
// with one thread per output).  All lanes of a warp take part in every pass.
template <class N>
__device__ __forceinline__ typename N::T group4_sum(typename N::T a) {
  a = N::add(a, md::shfl_xor(a, 1));
  return N::add(a, md::shfl_xor(a, 2));
}

// ------------------------------------------------------------- Householder
// Reflector of x = R[c.., c], m = n - c entries, in PHCpack's convention
// (Matrices/dbl2_factorizations.cpp:374 real, :436 complex): v[0] = 1,
// beta = 2|v0|^2/(sigma + |v0|^2); the real case takes v0 = x0 - mu or
// -sigma/(x0 + mu), the complex case v0 = x0 - mu x0/|x0|.
// Leaves v in S.v (m numbers) and beta in S.misc[0] (real part of a number).
template <class N>
__device__ void block_house(int m, const double *col, long ld, dense_smem &S) {
  typedef typename N::T T;
  typedef typename N::real R;
  typedef md::num<R, false> RN;
  R sig = RN::zero();
  for (int i = 1 + threadIdx.x; i < m; i += blockDim.x) {
    const T xi = ldn_at<N>(col, (long)i * ld);
    sig = RN::add(sig, N::norm2(xi));
    stn_at<N>(S.v, i, xi);
  }
  const R sigma = block_sum<RN>(sig, S.red);
  if (threadIdx.x == 0) {
    const T x0 = ldn_at<N>(col, 0);
    R beta = RN::zero();
    T inv = N::one();
    if (!md::is_zero(sigma)) {
      T v0;
      if constexpr (N::is_complex) {
        const R sq0 = N::norm2(x0);
        const R rad0 = RN::tr::sqrt(sq0);
        R mu = RN::tr::sqrt(RN::add(sq0, sigma));
        if (md::is_zero(rad0)) {
          v0 = N::mkc(RN::neg(mu), RN::zero());
        } else {
          mu = RN::tr::div(mu, rad0);
          v0 = N::mkc(RN::sub(x0.re, RN::mul(mu, x0.re)), RN::sub(x0.im, RN::mul(mu, x0.im)));
        }
      } else {
        const R mu = RN::tr::sqrt(RN::add(RN::mul(x0, x0), sigma));
        if (md::lead(x0) <= 0.0)
          v0 = RN::sub(x0, mu);
        else
          v0 = RN::neg(RN::tr::div(sigma, RN::add(x0, mu)));
      }
      const R v0sq = N::norm2(v0);
      beta = md::mul_d(RN::tr::div(v0sq, RN::add(sigma, v0sq)), 2.0);
      if constexpr (N::is_complex) {
        inv = N::mkc(RN::tr::div(v0.re, v0sq), RN::neg(RN::tr::div(v0.im, v0sq)));
      } else {
        inv = v0;  // the real case divides by v0
      }
    }
    stn_at<RN>(S.misc, 0, beta);
    stn_at<N>(S.misc + 2 * N::width, 0, inv);
  }
  __syncthreads();
  const R beta = ldn_at<RN>(S.misc, 0);
  const T inv = ldn_at<N>(S.misc + 2 * N::width, 0);
  if (!md::is_zero(beta)) {
    for (int i = 1 + threadIdx.x; i < m; i += blockDim.x) {
      const T vi = ldn_at<N>(S.v, i);
      if constexpr (N::is_complex)
        stn_at<N>(S.v, i, N::mul(vi, inv));
      else
        stn_at<N>(S.v, i, N::div(vi, inv));
    }
  }
  if (threadIdx.x == 0) stn_at<N>(S.v, 0, N::one());
  __syncthreads();
}

// R[c.., c..e) <- (I - beta v v^H) R[c.., c..e): w_j = beta sum_i conj(R_ij) v_i,
// R_ij -= v_i conj(w_j)   (Matrices/dbl2_factorizations.cpp:534/:567).
// Entry (i, j) of R sits at Rm[(i - r0) * ld + (j - c0)]: the whole matrix
// (r0 = c0 = 0, ld = ncols) or a panel of it staged in shared memory.
template <class N>
__device__ void block_apply_reflector(int n, long ld, int c, int e, double *Rm, dense_smem &S, int r0 = 0,
                                      int c0 = 0) {
  typedef typename N::T T;
  typedef typename N::real R;
  typedef md::num<R, false> RN;
  const int grp = threadIdx.x >> 2, part = threadIdx.x & 3, ngrp = blockDim.x >> 2;
  const R beta = ldn_at<RN>(S.misc, 0);
  if (md::is_zero(beta)) return;
  for (int base = c; base < e; base += ngrp) {  // four lanes per column
    const int j = base + grp;
    T acc = N::zero();
    if (j < e)
      for (int i = c + part; i < n; i += 4)
        acc = N::add(acc, N::mul(N::conj(ldn_at<N>(Rm, (long)(i - r0) * ld + (j - c0))), ldn_at<N>(S.v, i - c)));
    acc = group4_sum<N>(acc);
    if (j < e && part == 0) stn_at<N>(S.w, j - c, N::scale(acc, beta));
  }
  __syncthreads();
  const int nc = e - c;
  for (int t = threadIdx.x; t < (n - c) * nc; t += blockDim.x) {
    const int i = c + t / nc, j = c + t % nc;
    const long o = (long)(i - r0) * ld + (j - c0);
    stn_at<N>(Rm, o, N::sub(ldn_at<N>(Rm, o), N::mul(ldn_at<N>(S.v, i - c), N::conj(ldn_at<N>(S.w, j - c)))));
  }
  __syncthreads();
}

// ------------------------------------------------------------- blocked QR
// A = Q R with Q n x n and R n x ncols (row-major), ncols = szt*nbt <= n.
// Matrices/dbl2_baqr_host.cpp:728 and dbl2_baqr_kernels.cu:3520: per tile
// the szt reflectors are applied to the panel column by column, then
// W = -B (I + W Y^H) Y column by column (:13), the trailing columns get
// R <- R + Y (W^H R) and Q <- Q + (Q W) Y^H.  R must hold A on entry.
// work: the WY panels Y, W, the product P and T (4 n szt numbers), in
// shared memory when the kernel staged them there, else in the instance's
// global workspace; panel: shared memory for the current column panel of R
// (n szt numbers: rows rowoff.., the tile's szt columns), or nullptr to
// factor the panel in place in global memory.  With OZ (real numbers only)
// the four trailing products run as Ozaki-split products on the FP64 tensor
// cores (ozaki.cuh) with the scratch oz (ozaki_work_doubles, global);
// complex numbers keep the CUDA-core products.
template <class N, bool OZ = false>
__device__ void block_houseqr(int n, int ncols, int szt, double *Q, double *Rm, double *work, double *oz,
                              dense_smem &S, double *panel = nullptr) {
  typedef typename N::T T;
  typedef typename N::real R;
  typedef md::num<R, false> RN;
  const int W = N::width;
  double *Y = work;                         // szt x n
  double *Wm = Y + (long)szt * n * W;       // szt x n
  double *P = Wm + (long)szt * n * W;       // szt x n
  double *Tm = P + (long)szt * n * W;       // n x szt
  const int nbt = ncols / szt;
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
    const int i = t / n, j = t % n;
    stn_at<N>(Q, t, (i == j) ? N::one() : N::zero());
  }
  __syncthreads();
  for (int k = 0; k < nbt; ++k) {
    const int rowoff = k * szt;
    const int m = n - rowoff;
    const int endcol = (k + 1) * szt;
    if (panel) {  // the tile's columns, rows rowoff.., into shared memory
      for (int t = threadIdx.x; t < m * szt; t += blockDim.x)
        stn_at<N>(panel, t, ldn_at<N>(Rm, (long)(rowoff + t / szt) * ncols + rowoff + t % szt));
      __syncthreads();
    }
    for (int L = 0; L < szt; ++L) {
      const int c = rowoff + L;
      if (panel) {
        block_house<N>(n - c, panel + ((long)L * szt + L) * W, szt, S);
        block_apply_reflector<N>(n, szt, c, endcol, panel, S, rowoff, rowoff);
      } else {
        block_house<N>(n - c, Rm + (long)c * ncols * W + (long)c * W, ncols, S);
        block_apply_reflector<N>(n, ncols, c, endcol, Rm, S);
      }
      if (threadIdx.x == 0) stn_at<RN>(S.beta, L, ldn_at<RN>(S.misc, 0));
      for (int i = threadIdx.x; i < m; i += blockDim.x)
        stn_at<N>(Y, (long)L * m + i, (i < L) ? N::zero() : ldn_at<N>(S.v, i - L));
      __syncthreads();
    }
    if (panel) {
      for (int t = threadIdx.x; t < m * szt; t += blockDim.x)
        stn_at<N>(Rm, (long)(rowoff + t / szt) * ncols + rowoff + t % szt, ldn_at<N>(panel, t));
      __syncthreads();
    }
    // W from the betas and Y (Matrices/dbl2_baqr_host.cpp:13)
    {
      const R b0 = ldn_at<RN>(S.beta, 0);
      for (int i = threadIdx.x; i < m; i += blockDim.x)
        stn_at<N>(Wm, i, N::neg(N::scale(ldn_at<N>(Y, i), b0)));
      __syncthreads();
      const int grp = threadIdx.x >> 2, part = threadIdx.x & 3, ngrp = blockDim.x >> 2;
      for (int j = 1; j < szt; ++j) {
        for (int base = 0; base < j; base += ngrp) {  // four lanes per inner product
          const int kk = base + grp;
          T acc = N::zero();
          if (kk < j)
            for (int i = part; i < m; i += 4)
              acc = N::add(acc, N::mul(N::conj(ldn_at<N>(Y, (long)kk * m + i)), ldn_at<N>(Y, (long)j * m + i)));
          acc = group4_sum<N>(acc);
          if (kk < j && part == 0) stn_at<N>(S.w, kk, acc);
        }
        __syncthreads();
        const R bj = ldn_at<RN>(S.beta, j);
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
          T z = N::zero();
          for (int kk = 0; kk < j; ++kk) z = N::add(z, N::mul(ldn_at<N>(Wm, (long)kk * m + i), ldn_at<N>(S.w, kk)));
          z = N::add(z, ldn_at<N>(Y, (long)j * m + i));
          stn_at<N>(Wm, (long)j * m + i, N::neg(N::scale(z, bj)));
        }
        __syncthreads();
      }
    }
    if constexpr (OZ && !N::is_complex) {
      if (k < nbt - 1) {
        const int nc = ncols - endcol;
        // P = W^T C, then C += Y^T P
        ozaki_gemm<R>(szt, nc, m, [&](int a, int b) { return ldn_at<N>(Wm, (long)a * m + b); },
                      [&](int a, int b) { return ldn_at<N>(Rm, (long)(rowoff + a) * ncols + endcol + b); },
                      [&](int a, int b, const R &v) { stn_at<N>(P, (long)a * nc + b, v); }, oz);
        ozaki_gemm<R>(m, nc, szt, [&](int a, int b) { return ldn_at<N>(Y, (long)b * m + a); },
                      [&](int a, int b) { return ldn_at<N>(P, (long)a * nc + b); },
                      [&](int a, int b, const R &v) {
                        const long o = (long)(rowoff + a) * ncols + endcol + b;
                        stn_at<N>(Rm, o, N::add(ldn_at<N>(Rm, o), v));
                      }, oz);
      }
      // T = Q[:, rowoff..] W^T, then Q[:, rowoff..] += T Y
      ozaki_gemm<R>(n, szt, m, [&](int a, int b) { return ldn_at<N>(Q, (long)a * n + rowoff + b); },
                    [&](int a, int b) { return ldn_at<N>(Wm, (long)b * m + a); },
                    [&](int a, int b, const R &v) { stn_at<N>(Tm, (long)a * szt + b, v); }, oz);
      ozaki_gemm<R>(n, m, szt, [&](int a, int b) { return ldn_at<N>(Tm, (long)a * szt + b); },
                    [&](int a, int b) { return ldn_at<N>(Y, (long)a * m + b); },
                    [&](int a, int b, const R &v) {
                      const long o = (long)a * n + rowoff + b;
                      stn_at<N>(Q, o, N::add(ldn_at<N>(Q, o), v));
                    }, oz);
      continue;
    }
    if (k < nbt - 1) {
      // R[rowoff.., endcol..] += Y (W^H C)
      const int nc = ncols - endcol;
      for (int t = threadIdx.x; t < szt * nc; t += blockDim.x) {
        const int kk = t / nc, j = t % nc;
        T acc = N::zero();
        for (int i = 0; i < m; ++i)
          acc = N::add(acc, N::mul(N::conj(ldn_at<N>(Wm, (long)kk * m + i)),
                                   ldn_at<N>(Rm, (long)(rowoff + i) * ncols + endcol + j)));
        stn_at<N>(P, (long)kk * nc + j, acc);
      }
      __syncthreads();
      for (int t = threadIdx.x; t < m * nc; t += blockDim.x) {
        const int i = t / nc, j = t % nc;
        T acc = N::zero();
        for (int kk = 0; kk < szt; ++kk)
          acc = N::add(acc, N::mul(ldn_at<N>(Y, (long)kk * m + i), ldn_at<N>(P, (long)kk * nc + j)));
        const long o = (long)(rowoff + i) * ncols + endcol + j;
        stn_at<N>(Rm, o, N::add(ldn_at<N>(Rm, o), acc));
      }
      __syncthreads();
    }
    // Q[:, rowoff..] += (Q[:, rowoff..] W) Y^H
    for (int t = threadIdx.x; t < n * szt; t += blockDim.x) {
      const int i = t / szt, kk = t % szt;
      T acc = N::zero();
      for (int l = 0; l < m; ++l)
        acc = N::add(acc, N::mul(ldn_at<N>(Q, (long)i * n + rowoff + l), ldn_at<N>(Wm, (long)kk * m + l)));
      stn_at<N>(Tm, (long)i * szt + kk, acc);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n * m; t += blockDim.x) {
      const int i = t / m, j = t % m;
      T acc = N::zero();
      for (int kk = 0; kk < szt; ++kk)
        acc = N::add(acc, N::mul(ldn_at<N>(Tm, (long)i * szt + kk), N::conj(ldn_at<N>(Y, (long)kk * m + j))));
      const long o = (long)i * n + rowoff + j;
      stn_at<N>(Q, o, N::add(ldn_at<N>(Q, o), acc));
    }
    __syncthreads();
  }
}

// ------------------------------------------------------ tiled back substitution
// Inverse of every szt x szt diagonal tile of the upper triangular U (dim x dim,
// leading dimension ldu) into Tinv (nbt tiles of szt x szt), one thread per
// (tile, column): column j of the inverse solves T x = e_j by back
// substitution (Matrices/dbl2_tabs_host.cpp:31 CPU_dbl2_upper_inverse,
// dbl2_tabs_kernels.cu:397 dbl2_invert_tiles).
template <class N>
__device__ void block_invert_tiles(int dim, int szt, const double *U, int ldu, double *Tinv) {
  typedef typename N::T T;
  const int nbt = dim / szt;
  for (int t = threadIdx.x; t < nbt * szt; t += blockDim.x) {
    const int tile = t / szt, j = t % szt;
    const int off = tile * szt;
    double *inv = Tinv + (long)tile * szt * szt * N::width;
    for (int i = szt - 1; i > j; --i) stn_at<N>(inv, (long)i * szt + j, N::zero());
    for (int i = j; i >= 0; --i) {
      T acc = (i == j) ? N::one() : N::zero();
      for (int l = j; l > i; --l)
        acc = N::sub(acc, N::mul(ldn_at<N>(U, (long)(off + i) * ldu + off + l), ldn_at<N>(inv, (long)l * szt + j)));
      stn_at<N>(inv, (long)i * szt + j, N::div(acc, ldn_at<N>(U, (long)(off + i) * ldu + off + i)));
    }
  }
  __syncthreads();
}

// x = U^{-1} b with the inverted diagonal tiles: for k = nbt-1..0,
// x_k = Tinv_k b_k, then b_j -= U_jk x_k for j < k
// (Matrices/dbl2_tabs_host.cpp:147).  b (shared or global) is overwritten.
template <class N>
__device__ void block_tiled_backsub(int dim, int szt, const double *U, int ldu, const double *Tinv, double *b,
                                    double *x) {
  typedef typename N::T T;
  const int nbt = dim / szt;
  const int grp = threadIdx.x >> 2, part = threadIdx.x & 3, ngrp = blockDim.x >> 2;
  for (int k = nbt - 1; k >= 0; --k) {
    const int off = k * szt;
    const double *inv = Tinv + (long)k * szt * szt * N::width;
    for (int base = 0; base < szt; base += ngrp) {
      const int i = base + grp;
      T acc = N::zero();
      if (i < szt)
        for (int j = part; j < szt; j += 4)
          acc = N::add(acc, N::mul(ldn_at<N>(inv, (long)i * szt + j), ldn_at<N>(b, off + j)));
      acc = group4_sum<N>(acc);
      if (i < szt && part == 0) stn_at<N>(x, off + i, acc);
    }
    __syncthreads();
    for (int base = 0; base < off; base += ngrp) {
      const int r = base + grp;
      T acc = N::zero();
      if (r < off)
        for (int j = part; j < szt; j += 4)
          acc = N::add(acc, N::mul(ldn_at<N>(U, (long)r * ldu + off + j), ldn_at<N>(x, off + j)));
      acc = group4_sum<N>(acc);
      if (r < off && part == 0) stn_at<N>(b, r, N::sub(ldn_at<N>(b, r), acc));
    }
    __syncthreads();
  }
}

// w = Q^H b (Newton/dbl2_bals_kernels.cu:22 dbl2_bals_qtb), four lanes per
// output
template <class N>
__device__ void block_qhb(int n, const double *Q, const double *b, double *w) {
  typedef typename N::T T;
  const int grp = threadIdx.x >> 2, part = threadIdx.x & 3, ngrp = blockDim.x >> 2;
  for (int base = 0; base < n; base += ngrp) {
    const int i = base + grp;
    T acc = N::zero();
    if (i < n)
      for (int j = part; j < n; j += 4)
        acc = N::add(acc, N::mul(N::conj(ldn_at<N>(Q, (long)j * n + i)), ldn_at<N>(b, j)));
    acc = group4_sum<N>(acc);
    if (i < n && part == 0) stn_at<N>(w, i, acc);
  }
  __syncthreads();
}

// b_j -= A_{j-i+1} x for j = i..degp1-1 (Newton/dbl2_tail_kernels.cu:19
// dbl2_bals_tail, all right hand sides of one stage at once): one thread per
// row of the stacked matrices A_1 .. A_{degp1-i}, the row's dot product with
// x (shared memory) in two interleaved partial sums.  The stage is a chain
// of dependent multiple-double operations per row; a thread per row keeps
// every thread of the CTA on its own chain instead of reducing each row
// across a warp.
template <class N>
__device__ void block_tail_update(int n, int degp1, int i, const double *mat, double *rhs, const double *x) {
  typedef typename N::T T;
  const long nn = (long)n * n;
  const int rows = (degp1 - i) * n;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    const int j = i + r / n, row = r % n;
    const double *A = mat + (long)(j - i + 1) * nn * N::width + (long)row * n * N::width;
    T a0 = N::zero(), a1 = N::zero();
    int l = 0;
    for (; l + 1 < n; l += 2) {
      a0 = N::add(a0, N::mul(ldn_at<N>(A, l), ldn_at<N>(x, l)));
      a1 = N::add(a1, N::mul(ldn_at<N>(A, l + 1), ldn_at<N>(x, l + 1)));
    }
    if (l < n) a0 = N::add(a0, N::mul(ldn_at<N>(A, l), ldn_at<N>(x, l)));
    double *bj = rhs + ((long)j * n + row) * N::width;
    T v;
    md::ldn(bj, v);
    md::stn(bj, N::sub(v, N::add(a0, a1)));
  }
  __syncthreads();
}

}  // namespace phc
