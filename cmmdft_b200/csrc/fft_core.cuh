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

#define CMM_MAX_SMALL_RADIX 16   // larger (prime) radices run as Rader or direct-DFT stages

struct RaderTab;

struct FftAxis {
  int n;                         // transform length
  int nstage;                    // number of radix stages
  int big;                       // 1 when a radix exceeds CMM_MAX_SMALL_RADIX (needs scratch)
  int radix[CMM_MAX_STAGES];     // radix of stage s (forward order)
  int span[CMM_MAX_STAGES];      // block length L_s at stage s (L_0 = n)
  const RaderTab* rader;         // device array indexed by stage (null: every big stage is a direct DFT)
};

// Rader's algorithm (C. M. Rader, Proc. IEEE 56, 1107 (1968)) for a prime
// radix R whose M = R - 1 factors into radices <= 16.  With g a primitive
// root mod R the outputs q = g^k, k < M, are
//   y_{g^k} = x_0 + sum_m x_{g^-m} w_R^{g^(k-m)},
// a length-M cyclic convolution: forward FFT of the permuted inputs, product
// with the transformed kernel, inverse FFT.  y_0 = x_0 + sum_{r>0} x_r is the
// DC bin of the forward transform.
struct RaderTab {
  FftAxis axm;          // plan of the length-M transforms (no big radix)
  int M;                // 0: the stage keeps the direct DFT
  const double2* twm;   // w_M^t, t < M
  const double2* kf;    // DFT_M of b_j = w_R^{g^j}, divided by M, at the DIF output positions (forward stage)
  const double2* ki;    // the same for b_j = conj(w_R^{g^j}) (inverse stage)
  const int* gin;       // gin[m] = g^-m mod R
  const int* gout;      // gout[k] = g^k mod R
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

template <int R, bool INV>
__device__ __forceinline__ void dftR(double2* v, const double2* tw, int twn) {
  if constexpr (R == 2) dft2<INV>(v);
  else if constexpr (R == 4) dft4<INV>(v);
  else if constexpr (R == 8) dft8<INV>(v);
  else if constexpr (R == 3) dft3<INV>(v);
  else if constexpr (R == 5) dft5<INV>(v);
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

// Butterfly of an odd prime radix R (7, 11, 13).  The output pairs
// (q, R - q) share the sums and differences of the input pairs (r, R - r):
//   y_q, y_{R-q} = x_0 + sum_r (x_r + x_{R-r}) cos(2 pi rq/R)
//                  -/+ i sum_r (x_r - x_{R-r}) sin(2 pi rq/R)
// (forward signs; the inverse swaps them).  Only the pair sums and
// differences and the R - 1 cos/sin values stay in registers; each output
// pair is written back as soon as it is formed.  Twiddles as in butterfly().
// Not inlined: its registers would otherwise raise the allocation of every
// kernel that holds an FFT loop.
template <int R, bool INV>
__device__ __noinline__ void butterfly_odd(double2* b, int es, const double2* tw, int twn, int tb) {
  constexpr int h = (R - 1) / 2;
  const int step = twn / R;
  double c[h + 1], sn[h + 1];
#pragma unroll
  for (int k = 1; k <= h; ++k) {
    const double2 w = tw[k * step];
    c[k] = w.x;
    sn[k] = -w.y;
  }
  const double2 x0 = b[0];
  double2 sp[h + 1], dm[h + 1];
  double2 y0 = x0;
#pragma unroll
  for (int r = 1; r <= h; ++r) {
    double2 u = b[r * es], w = b[(R - r) * es];
    if (INV && tb) {
      u = cmulc(u, tw[tb * r]);
      w = cmulc(w, tw[tb * (R - r)]);
    }
    sp[r] = cadd(u, w);
    dm[r] = csub(u, w);
    y0 = cadd(y0, sp[r]);
  }
  b[0] = y0;
#pragma unroll
  for (int q = 1; q <= h; ++q) {
    double2 A = x0, B = make_double2(0.0, 0.0);
#pragma unroll
    for (int r = 1; r <= h; ++r) {
      const int m = (r * q) % R;
      const int k = m <= h ? m : R - m;
      A.x += sp[r].x * c[k];
      A.y += sp[r].y * c[k];
      if (m <= h) {
        B.x += dm[r].x * sn[k];
        B.y += dm[r].y * sn[k];
      } else {
        B.x -= dm[r].x * sn[k];
        B.y -= dm[r].y * sn[k];
      }
    }
    const double2 iB = rot_mi<INV>(B);
    double2 yq = cadd(A, iB), ym = csub(A, iB);
    if (!INV && tb) {
      yq = cmul(yq, tw[tb * q]);
      ym = cmul(ym, tw[tb * (R - q)]);
    }
    b[q * es] = yq;
    b[(R - q) * es] = ym;
  }
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

// Start of butterfly u (pencil fastest) of a stage with span L and sR = L / R.
__device__ __forceinline__ int bfly_base(const PencilSet& ps, int u, int sR, int L, int& jj) {
  const int p = u % ps.npencil, bj = u / ps.npencil;
  const int blk = bj / sR;
  jj = bj - blk * sR;
  return (p / ps.ppg) * ps.gstride + (p % ps.ppg) * ps.pstride + (blk * L + jj) * ps.estride;
}

// Calls f(t, e, base, jj) for slot e < R of every butterfly u < nbt, t = u + nbt e.
// When the butterflies fit in the block each thread keeps one butterfly and
// computes its base once.
template <class F>
__device__ __forceinline__ void for_bfly_slots(const PencilSet& ps, int nbt, int R, int sR, int L, F f) {
  if (nbt <= (int)blockDim.x) {
    const int per = blockDim.x / nbt;
    const int u = threadIdx.x % nbt, e0 = threadIdx.x / nbt;
    if (e0 >= per) return;
    int jj;
    const int base = bfly_base(ps, u, sR, L, jj);
    for (int e = e0; e < R; e += per) f(u + nbt * e, e, base, jj);
  } else {
    for (int t = threadIdx.x; t < nbt * R; t += blockDim.x) {
      const int u = t % nbt, e = t / nbt;
      int jj;
      const int base = bfly_base(ps, u, sR, L, jj);
      f(t, e, base, jj);
    }
  }
}

// One stage of radix R <= 16 over every pencil of `ps`; ends with __syncthreads().
// EX compiles the odd radices 7, 11, 13 in (kept out of the kernels of
// other grids, whose register allocation they would raise); LEAN (the Rader
// convolutions, whose plans have no radix 8) leaves out the radix-8
// butterfly, the register peak of the stage loop.
template <bool INV, bool EX, bool LEAN = false>
__device__ __forceinline__ void small_stage(double2* s, int n, int R, int L, const double2* tw, int twmul,
                                            const PencilSet& ps) {
  const int twn = n * twmul;
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
      case 8: if constexpr (!LEAN) butterfly<8, INV>(b, es, tw, twn, tb); break;
      case 4: butterfly<4, INV>(b, es, tw, twn, tb); break;
      case 2: butterfly<2, INV>(b, es, tw, twn, tb); break;
      case 3: butterfly<3, INV>(b, es, tw, twn, tb); break;
      case 5: butterfly<5, INV>(b, es, tw, twn, tb); break;
      case 7: if constexpr (EX) butterfly_odd<7, INV>(b, es, tw, twn, tb); break;
      case 11: if constexpr (EX) butterfly_odd<11, INV>(b, es, tw, twn, tb); break;
      case 13: if constexpr (EX) butterfly_odd<13, INV>(b, es, tw, twn, tb); break;
    }
  }
  __syncthreads();
}

// Every stage of a Rader convolution plan (radices 4, 2 and odd primes <= 13).
template <bool INV>
__device__ void small_stages(double2* s, const FftAxis& ax, const double2* tw, int twmul, const PencilSet& ps) {
  for (int k = 0; k < ax.nstage; ++k) {
    const int st = INV ? (ax.nstage - 1 - k) : k;
    small_stage<INV, true, true>(s, ax.n, ax.radix[st], ax.span[st], tw, twmul, ps);
  }
}

// A stage of prime radix R by Rader's algorithm, same input/output
// conventions as big_stage.  Scratch (ps.npencil * n elements) holds, for
// butterfly u, slot m < M = R - 1 at tmp[u + nbt m] and x_0 at slot M:
//   gather   a_m = x_{g^-m} (inverse stages first apply conj w_L^{jj r}),
//   forward length-M FFT (digit-reversed output),
//   product with the kernel spectrum (1/M included); the DC bin also takes
//            x_0 (so the inverse adds x_0 to every output) and slot M
//            becomes y_0 = x_0 + A_0,
//   inverse length-M FFT (natural output: slot k holds y_{g^k}),
//   scatter  (forward stages apply w_L^{jj q}).
template <bool INV>
__device__ __noinline__ void rader_stage(double2* s, int n, int R, int L, const double2* tw, int twn, const PencilSet& ps,
                            double2* tmp, const RaderTab& rt) {
  const int sR = L / R, lstep = twn / L, M = R - 1;
  const int nbt = ps.npencil * (n / R);
  const int es = sR * ps.estride;
  const int* gin = rt.gin;
  for_bfly_slots(ps, nbt, R, sR, L, [&](int t, int e, int base, int jj) {
    const int r = (e < M) ? __ldg(gin + e) : 0;
    double2 x = s[base + r * es];
    if (INV && jj && r) x = cmulc(x, tw[jj * r * lstep]);
    tmp[t] = x;
  });
  __syncthreads();
  const PencilSet cs = {nbt, nbt, 0, 1, nbt, true};
  small_stages<false>(tmp, rt.axm, rt.twm, 1, cs);
  const double2* kt = INV ? rt.ki : rt.kf;
  for (int t = threadIdx.x; t < nbt * M; t += blockDim.x) {
    const int pos = t / nbt;
    const double2 a = tmp[t];
    double2 c = cmul(a, __ldg(kt + pos));
    if (pos == 0) {
      const double2 x0 = tmp[t + nbt * M];
      c = cadd(c, x0);
      tmp[t + nbt * M] = cadd(x0, a);
    }
    tmp[t] = c;
  }
  __syncthreads();
  small_stages<true>(tmp, rt.axm, rt.twm, 1, cs);
  const int* gout = rt.gout;
  for_bfly_slots(ps, nbt, R, sR, L, [&](int t, int e, int base, int jj) {
    const int q = (e < M) ? __ldg(gout + e) : 0;
    double2 y = tmp[t];
    if (!INV && jj && q) y = cmul(y, tw[jj * q * lstep]);
    s[base + q * es] = y;
  });
  __syncthreads();
}

// Transform every pencil of `ps` (length ax.n) in place.  `tw` is the twiddle
// table w_{twn}^t in shared memory with twn = ax.n * twmul (twmul = 2 when the
// table of the full real length is reused for a half-length complex FFT).
// `tmp` (ps.npencil * ax.n elements) is needed when ax.big.  Without EX the
// radices 2, 3, 4, 5, 8 and direct-DFT stages are compiled; EX adds 7, 11,
// 13 and Rader stages (the host launches EX kernels for plans that use
// them).  Ends with __syncthreads().
template <bool INV, bool EX>
__device__ void fft_pencils(double2* s, const FftAxis& ax, const double2* tw, int twmul, const PencilSet& ps,
                           double2* tmp = nullptr) {
  const int n = ax.n;
  const int twn = n * twmul;
  for (int k = 0; k < ax.nstage; ++k) {
    const int st = INV ? (ax.nstage - 1 - k) : k;
    const int R = ax.radix[st];
    const int L = ax.span[st];
    if (R > CMM_MAX_SMALL_RADIX) {
      if constexpr (EX) {
        if (ax.rader && ax.rader[st].M) {
          rader_stage<INV>(s, n, R, L, tw, twn, ps, tmp, ax.rader[st]);
          continue;
        }
      }
      big_stage<INV>(s, n, R, L, tw, twn, ps, tmp);
      continue;
    }
    small_stage<INV, EX>(s, n, R, L, tw, twmul, ps);
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
template <bool INV, bool EX>
__device__ void fft_rt(double2* s, const FftAxis& ax, const double2* tw, int twmul, int npencil, int pstride,
                       int estride, double2* tmp = nullptr) {
  PencilSet ps = {npencil, npencil, 0, pstride, estride, true};
  fft_pencils<INV, EX>(s, ax, tw, twmul, ps, tmp);
}
