// In-shared-memory FP64 FFT engine for sm_100a.
//
// Transforms are mixed-radix Cooley-Tukey, done IN PLACE in shared memory:
//   forward  = decimation in frequency (natural input -> digit-reversed output)
//   inverse  = decimation in time      (digit-reversed input -> natural output)
// Each butterfly reads and writes the same R slots, so a stage needs no
// register staging across a barrier and no second buffer; one
// __syncthreads() separates stages.  Spectra therefore live in digit-reversed
// order along every transformed axis; the k-space stages look frequencies up
// through position tables instead of permuting data.
//
// The forward transform is the unnormalised DFT  X_k = sum_j x_j w^{jk},
// w = exp(-2 pi i / n); the inverse uses w^{-jk}, also unnormalised.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define CMM_MAX_STAGES 16

#define CMM_MAX_SMALL_RADIX 16   // larger radices run as two-phase direct DFT stages

struct FftAxis {
  int n;                         // transform length
  int nstage;                    // number of radix stages
  int big;                       // 1 when a radix exceeds CMM_MAX_SMALL_RADIX (needs scratch)
  int radix[CMM_MAX_STAGES];     // radix of stage s (forward order)
  int span[CMM_MAX_STAGES];      // block length L_s at stage s (L_0 = n)
};

// ------------------------------------------------------------ complex ----
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ double2 rot_mi(double2 a) {
  return INV ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// ---------------------------------------------------------- butterflies ---
// In-register R-point DFT, forward (w = e^{-2 pi i/R}) or inverse (conj).
template <bool INV>
__device__ __forceinline__ void dft2(double2* v) {
  double2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <bool INV>
__device__ __forceinline__ void dft4(double2* v) {
  double2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
  double2 c = cadd(v[1], v[3]), d = rot_mi<INV>(csub(v[1], v[3]));
  v[0] = cadd(a, c);
  v[2] = csub(a, c);
  v[1] = cadd(b, d);
  v[3] = csub(b, d);
}

template <bool INV>
__device__ __forceinline__ void dft8(double2* v) {
  const double h = 0.70710678118654752440;  // sqrt(1/2)
  // radix-2 first: pairs (r, r+4)
  double2 a[4], b[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    a[r] = cadd(v[r], v[r + 4]);
    b[r] = csub(v[r], v[r + 4]);
  }
  // twiddle b[r] by w8^r
  b[1] = INV ? make_double2(h * (b[1].x - b[1].y), h * (b[1].x + b[1].y))
             : make_double2(h * (b[1].x + b[1].y), h * (b[1].y - b[1].x));
  b[2] = rot_mi<INV>(b[2]);
  b[3] = INV ? make_double2(-h * (b[3].x + b[3].y), h * (b[3].x - b[3].y))
             : make_double2(h * (b[3].y - b[3].x), -h * (b[3].x + b[3].y));
  dft4<INV>(a);
  dft4<INV>(b);
  // outputs: even k from a, odd k from b
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    v[2 * r] = a[r];
    v[2 * r + 1] = b[r];
  }
}

template <bool INV>
__device__ __forceinline__ void dft3(double2* v) {
  const double s3 = 0.86602540378443864676;  // sqrt(3)/2
  double2 t = cadd(v[1], v[2]);
  double2 u = make_double2(v[0].x - 0.5 * t.x, v[0].y - 0.5 * t.y);
  double2 d = csub(v[1], v[2]);
  // -i * s3 * d (forward) / +i * s3 * d (inverse)
  double2 w = rot_mi<INV>(cscale(d, s3));
  v[0] = cadd(v[0], t);
  v[1] = cadd(u, w);
  v[2] = csub(u, w);
}

template <bool INV>
__device__ __forceinline__ void dft5(double2* v) {
  const double c1 = 0.30901699437494742410;   // cos(2pi/5)
  const double c2 = -0.80901699437494742410;  // cos(4pi/5)
  const double s1 = 0.95105651629515357212;   // sin(2pi/5)
  const double s2 = 0.58778525229247312917;   // sin(4pi/5)
  double2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
  double2 d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
  double2 a1 = make_double2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
  double2 a2 = make_double2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
  // b = -i*(s1*d1 + s2*d2) etc. (forward sign)
  double2 b1 = rot_mi<INV>(make_double2(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y));
  double2 b2 = rot_mi<INV>(make_double2(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y));
  v[0] = cadd(v[0], cadd(t1, t2));
  v[1] = cadd(a1, b1);
  v[4] = csub(a1, b1);
  v[2] = cadd(a2, b2);
  v[3] = csub(a2, b2);
}

// Generic odd radix (primes > 5): direct DFT through the axis twiddle table.
// tw holds w_n^t for the axis length n (table length twn); w_R = w_n^{n/R}.
template <bool INV>
__device__ __forceinline__ void dft_generic(double2* v, int R, const double2* tw, int twn) {
  double2 out[16];
  int step = twn / R;
  for (int q = 0; q < R; ++q) {
    double2 acc = v[0];
    for (int r = 1; r < R; ++r) {
      double2 w = tw[((r * q) % R) * step];
      acc = cadd(acc, INV ? cmulc(v[r], w) : cmul(v[r], w));
    }
    out[q] = acc;
  }
  for (int q = 0; q < R; ++q) v[q] = out[q];
}

template <int R, bool INV>
__device__ __forceinline__ void dftR(double2* v, const double2* tw, int twn) {
  if (R == 2) dft2<INV>(v);
  else if (R == 4) dft4<INV>(v);
  else if (R == 8) dft8<INV>(v);
  else if (R == 3) dft3<INV>(v);
  else if (R == 5) dft5<INV>(v);
}

// One butterfly of a stage.  Forward (DIF): y = DFT_R(x); y_q *= w_L^{jj q}.
// Inverse (DIT, transposed): y_q *= conj(w_L^{jj q}); x = IDFT_R(y).
// `tb` = jj * (twn / L): index of w_L^{jj} in the table; jj*q*tstep < twn.
template <int R, bool INV>
__device__ __forceinline__ void butterfly(double2* b, int es, const double2* tw, int twn, int tb) {
  double2 v[R];
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = b[r * es];
  if (INV) {
    if (tb) {
#pragma unroll
      for (int q = 1; q < R; ++q) v[q] = cmulc(v[q], tw[tb * q]);
    }
    dftR<R, true>(v, tw, twn);
  } else {
    dftR<R, false>(v, tw, twn);
    if (tb) {
#pragma unroll
      for (int q = 1; q < R; ++q) v[q] = cmul(v[q], tw[tb * q]);
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) b[r * es] = v[r];
}

template <bool INV>
__device__ __forceinline__ void butterfly_generic(double2* b, int R, int es, const double2* tw, int twn, int tb) {
  double2 v[16];
  for (int r = 0; r < R; ++r) v[r] = b[r * es];
  if (INV) {
    if (tb)
      for (int q = 1; q < R; ++q) v[q] = cmulc(v[q], tw[tb * q]);
    dft_generic<true>(v, R, tw, twn);
  } else {
    dft_generic<false>(v, R, tw, twn);
    if (tb)
      for (int q = 1; q < R; ++q) v[q] = cmul(v[q], tw[tb * q]);
  }
  for (int r = 0; r < R; ++r) b[r * es] = v[r];
}

// Pencil geometry inside shared memory:
//   base(p) = (p / ppg) * gstride + (p % ppg) * pstride;  element j at base + j*estride
struct PencilSet {
  int npencil, ppg, gstride, pstride, estride;
  bool pencil_fast;  // consecutive threads take consecutive pencils (else consecutive butterflies)
};

// A stage of a large (prime) radix R: every output element is a direct
// length-R DFT of its butterfly's inputs, written to `tmp` (ps.npencil * n
// elements, pencil fastest) and copied back after a barrier.  Same twiddle
// conventions as butterfly(): forward (DIF) y_q = (sum_r x_r w_R^{rq}) w_L^{jj q};
// inverse (DIT) y_q = sum_r (x_r conj w_L^{jj r}) conj w_R^{rq}.
template <bool INV>
__device__ void big_stage(double2* s, int n, int R, int L, const double2* tw, int twn, const PencilSet& ps,
                          double2* tmp) {
  // One thread per output pair (q, R - q) of a butterfly: both sums run over
  // the same inputs with conjugate twiddles w^{rq} and w^{-rq}, so the four
  // products a c, b s, a s, b c of x = a + ib and w = c + is serve both.
  // Twiddle indices advance by addition (no division inside the sum).
  const int sR = L / R;
  const int rstep = twn / R, lstep = twn / L;
  const int nq = R / 2 + 1;                 // q = 0 .. R/2; q pairs with R - q
  const int nb = n / R;
  const int total = ps.npencil * nb * nq;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int p = t % ps.npencil, u = t / ps.npencil;
    const int q = u % nq, bj = u / nq;
    const int blk = bj / sR, jj = bj - blk * sR;
    const double2* b = s + (p / ps.ppg) * ps.gstride + (p % ps.ppg) * ps.pstride + (blk * L + jj) * ps.estride;
    const int es = sR * ps.estride;
    const int wstep = q * rstep, xstep = jj * lstep;
    double2 a1 = make_double2(0.0, 0.0), a2 = make_double2(0.0, 0.0);
    int wi = 0, xi = 0;
    for (int r = 0; r < R; ++r) {
      double2 x = b[r * es];
      if (INV && jj) x = cmulc(x, tw[xi]);
      const double2 w = tw[wi];
      const double ac = x.x * w.x, bs = x.y * w.y, as = x.x * w.y, bc = x.y * w.x;
      if (INV) {   // sum x conj(w) for q, sum x w for R - q
        a1.x += ac + bs; a1.y += bc - as;
        a2.x += ac - bs; a2.y += as + bc;
      } else {     // sum x w for q, sum x conj(w) for R - q
        a1.x += ac - bs; a1.y += as + bc;
        a2.x += ac + bs; a2.y += bc - as;
      }
      wi += wstep;
      if (wi >= twn) wi -= twn;
      xi += xstep;
    }
    const int q2 = R - q;
    if (!INV && jj) {
      a1 = cmul(a1, tw[jj * q * lstep]);
      a2 = cmul(a2, tw[jj * q2 * lstep]);
    }
    const int e1 = blk * L + q * sR + jj;
    tmp[p + ps.npencil * e1] = a1;
    if (q != 0 && 2 * q != R) tmp[p + ps.npencil * (blk * L + q2 * sR + jj)] = a2;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < ps.npencil * n; t += blockDim.x) {
    const int p = t % ps.npencil, e = t / ps.npencil;
    s[(p / ps.ppg) * ps.gstride + (p % ps.ppg) * ps.pstride + e * ps.estride] = tmp[t];
  }
  __syncthreads();
}

// Transform every pencil of `ps` (length ax.n) in place.  `tw` is the twiddle
// table w_{twn}^t in shared memory with twn = ax.n * twmul (twmul = 2 when the
// table of the full real length is reused for a half-length complex FFT).
// `tmp` (ps.npencil * ax.n elements) is needed when ax.big.
// Ends with __syncthreads().
template <bool INV>
__device__ void fft_pencils(double2* s, const FftAxis& ax, const double2* tw, int twmul, const PencilSet& ps,
                           double2* tmp = nullptr) {
  const int n = ax.n;
  const int twn = n * twmul;
  for (int k = 0; k < ax.nstage; ++k) {
    const int st = INV ? (ax.nstage - 1 - k) : k;
    const int R = ax.radix[st];
    const int L = ax.span[st];
    if (R > CMM_MAX_SMALL_RADIX) {
      big_stage<INV>(s, n, R, L, tw, twn, ps, tmp);
      continue;
    }
    const int sR = L / R;
    const int nb = n / R;
    const int tstep = (n / L) * twmul;
    const int total = ps.npencil * nb;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      int p, j;
      if (ps.pencil_fast) {
        p = t % ps.npencil;
        j = t / ps.npencil;
      } else {
        j = t % nb;
        p = t / nb;
      }
      const int blk = j / sR;
      const int jj = j - blk * sR;
      double2* b = s + (p / ps.ppg) * ps.gstride + (p % ps.ppg) * ps.pstride + (blk * L + jj) * ps.estride;
      const int es = sR * ps.estride;
      const int tb = jj * tstep;
      switch (R) {
        case 8: butterfly<8, INV>(b, es, tw, twn, tb); break;
        case 4: butterfly<4, INV>(b, es, tw, twn, tb); break;
        case 2: butterfly<2, INV>(b, es, tw, twn, tb); break;
        case 3: butterfly<3, INV>(b, es, tw, twn, tb); break;
        case 5: butterfly<5, INV>(b, es, tw, twn, tb); break;
        default: butterfly_generic<INV>(b, R, es, tw, twn, tb); break;
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------
// Uniform pencil sets: pencil p starts at s + p * pstride, element j at
// + j * estride.  Threads take consecutive pencils at the same butterfly
// index (conflict-free for unit-stride pencils and for the odd row strides
// used here; every thread of a warp reads the same twiddle).
// ------------------------------------------------------------------------

// Radix plan of a power of two N: 8-stages, then one 4 or 2 stage.
template <int N>
struct Pow2Plan {
  static constexpr int log2n = (N >= 2 ? 1 : 0) + (N >= 4 ? 1 : 0) + (N >= 8 ? 1 : 0) + (N >= 16 ? 1 : 0) +
                               (N >= 32 ? 1 : 0) + (N >= 64 ? 1 : 0) + (N >= 128 ? 1 : 0) + (N >= 256 ? 1 : 0) +
                               (N >= 512 ? 1 : 0) + (N >= 1024 ? 1 : 0);
  static constexpr int n8 = log2n / 3;
  static constexpr int tail = 1 << (log2n - 3 * n8);   // 1, 2 or 4
  static constexpr int nstage = n8 + (tail > 1 ? 1 : 0);
  __host__ __device__ static constexpr int radix(int s) { return s < n8 ? 8 : tail; }
  __host__ __device__ static constexpr int span(int s) {
    int L = N;
    for (int i = 0; i < s; ++i) L /= (i < n8 ? 8 : tail);
    return L;
  }
};

template <bool INV, int R, int L, int N>
__device__ __forceinline__ void stage_ct(double2* s, const double2* tw, int twmul, int npencil, int pstride,
                                         int estride) {
  constexpr int sR = L / R;
  constexpr int nb = N / R;
  const int tstep = (N / L) * twmul;
  const int total = npencil * nb;
  const int es = sR * estride;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int j = t / npencil;            // one division per task (npencil runtime)
    const int p = t - j * npencil;
    const int blk = j / sR;               // compile-time power of two
    const int jj = j - blk * sR;
    double2* b = s + p * pstride + (blk * L + jj) * estride;
    butterfly<R, INV>(b, es, tw, N * twmul, jj * tstep);
  }
}

template <bool INV, int N, int S>
__device__ __forceinline__ void stage_dispatch(double2* s, const double2* tw, int twmul, int npencil, int pstride,
                                               int estride) {
  if constexpr (S >= 0 && S < Pow2Plan<N>::nstage) {
    constexpr int R = Pow2Plan<N>::radix(S);
    constexpr int L = Pow2Plan<N>::span(S);
    stage_ct<INV, R, L, N>(s, tw, twmul, npencil, pstride, estride);
    __syncthreads();
  }
}

// Compile-time-length transform of npencil uniform pencils (N a power of two <= 512).
template <bool INV, int N>
__device__ __forceinline__ void fft_ct(double2* s, const double2* tw, int twmul, int npencil, int pstride,
                                       int estride) {
  constexpr int ns = Pow2Plan<N>::nstage;
  if constexpr (!INV) {
    stage_dispatch<false, N, 0>(s, tw, twmul, npencil, pstride, estride);
    stage_dispatch<false, N, 1>(s, tw, twmul, npencil, pstride, estride);
    stage_dispatch<false, N, 2>(s, tw, twmul, npencil, pstride, estride);
    stage_dispatch<false, N, 3>(s, tw, twmul, npencil, pstride, estride);
  } else {
    stage_dispatch<true, N, ns - 1>(s, tw, twmul, npencil, pstride, estride);
    stage_dispatch<true, N, ns - 2>(s, tw, twmul, npencil, pstride, estride);
    stage_dispatch<true, N, ns - 3>(s, tw, twmul, npencil, pstride, estride);
    stage_dispatch<true, N, ns - 4>(s, tw, twmul, npencil, pstride, estride);
  }
  static_assert(ns <= 4, "fft_ct handles up to 4 stages (N <= 4096)");
}

// Runtime-length transform of uniform pencils (any factorisation of ax.n);
// tmp: npencil * ax.n elements of scratch when ax.big.
template <bool INV>
__device__ void fft_rt(double2* s, const FftAxis& ax, const double2* tw, int twmul, int npencil, int pstride,
                       int estride, double2* tmp = nullptr) {
  PencilSet ps = {npencil, npencil, 0, pstride, estride, true};
  fft_pencils<INV>(s, ax, tw, twmul, ps, tmp);
}
