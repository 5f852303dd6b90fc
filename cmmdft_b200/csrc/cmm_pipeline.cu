// Fused FP64 grid-solve kernels for sm_100a.
//
// Per fixed-point iteration the solve runs four passes over HBM:
//   plane  (one CTA per x-plane): inverse y/z of the C1 spectrum, the update
//          (Picard / residual / mix), forward z (R2C) + y of the new density
//   column (one CTA per tile of (y,z) columns): forward x, the analytic FMT
//          weights, inverse x of the 5 weighted-density spectra
//   plane  : inverse y/z of 5 fields, White-Bear dPhi/dn, forward z/y of 5
//   column : forward x of 5 dPhi spectra and rho_hat, back-convolution with the
//          weights plus the MFA kernel, inverse x of the C1 spectrum
// All transforms are in place in shared memory (fft_core.cuh).
#include <cmath>
#include <cstdio>
#include <cstring>

#include <map>
#include <mutex>
#include <utility>

#include <cooperative_groups.h>

#include "cmm_common.cuh"
#include "cmm_dual.cuh"

// --------------------------------------------------------- shared tables --
// Plane layout in shared memory: nslot fields interleaved by row,
//   slots[(r * nslot + f) * h3 + c]   (y row r, field f, stored z frequency c)
// so y pencils (p = f*h3 + c) and z rows (p = r*nslot + f) are both uniform
// pencil sets (base = p * pstride).  A real row of N3 doubles occupies the
// first N3/2 double2 of its row.
struct PlaneSmem {
  double2* slots;   // n2 * nslot * h3
  double2* tw2;     // n2
  double2* tw3;     // n3
  int* zpos;        // m3
  double2* tmp;     // z rows only: direct-DFT stage scratch (z transforms with a prime factor > 16)
};

__host__ __device__ inline size_t plane_smem_bytes(int n2, int n3, int nslot) {
  int h3 = n3 / 2 + 1, m3 = n3 / 2;
  size_t b = sizeof(double2) * ((size_t)nslot * n2 * h3 + n2 + n3);
  b += sizeof(int) * m3;
  return (b + 15) & ~(size_t)15;
}

// Compile-time shape of a plane pass: N2C = y length, M3C = z half length
// (0 = take them from the plan at run time, radices 2, 3, 4, 5, 8 and
// direct-DFT stages; -1 = from the plan, also radices 7, 11, 13 and Rader
// stages).
template <int N2C, int M3C>
struct PlaneShape {
  int n2, m3, h3, n3;
  __device__ PlaneShape(const GridDev& g)
      : n2(N2C > 0 ? N2C : g.n2), m3(M3C > 0 ? M3C : g.m3), h3((M3C > 0 ? M3C : g.m3) + 1), n3(2 * (M3C > 0 ? M3C : g.m3)) {}
};

template <int N2C, int M3C>
__device__ inline PlaneSmem plane_smem_setup(const GridDev& g, int nslot) {
  extern __shared__ double2 smem_d2[];
  const PlaneShape<N2C, M3C> sh(g);
  PlaneSmem s;
  s.tmp = nullptr;
  s.slots = smem_d2;
  s.tw2 = s.slots + (size_t)nslot * sh.n2 * sh.h3;
  s.tw3 = s.tw2 + sh.n2;
  s.zpos = (int*)(s.tw3 + sh.n3);
  for (int i = threadIdx.x; i < sh.n2; i += blockDim.x) s.tw2[i] = g.tw2[i];
  for (int i = threadIdx.x; i < sh.n3; i += blockDim.x) s.tw3[i] = g.tw3[i];
  for (int i = threadIdx.x; i < sh.m3; i += blockDim.x) s.zpos[i] = g.zpos[i];
  return s;
}

template <bool INV, int NC>
__device__ __forceinline__ void axis_fft(double2* base, const FftAxis& ax, const double2* tw, int twmul,
                                         int npencil, int pstride, int estride, double2* tmp = nullptr) {
  if constexpr (NC > 0) fft_ct<INV, NC>(base, tw, twmul, npencil, pstride, estride);
  else fft_rt<INV, (NC < 0)>(base, ax, tw, twmul, npencil, pstride, estride, tmp);
}

// R2C twist on `nrow` rows: pairs (k, m3-k), k = 0..m3/2, rows fastest.
template <int M3C>
__device__ void r2c_twist_rows(const GridDev& g, const PlaneSmem& s, int nrow) {
  const int m3 = M3C > 0 ? M3C : g.m3, h3 = m3 + 1;
  const int total = nrow * (m3 / 2 + 1);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int k = t / nrow, row = t - k * nrow;
    double2* rp = s.slots + (size_t)row * h3;
    if (k == 0) {
      double2 z0 = rp[0];
      rp[0] = make_double2(z0.x + z0.y, 0.0);
      rp[m3] = make_double2(z0.x - z0.y, 0.0);
    } else {
      const int pk = s.zpos[k], pm = s.zpos[m3 - k];
      double2 zk = rp[pk], zm = rp[pm];
      // E = (zk + conj zm)/2 ; O = -i (zk - conj zm)/2 ; X[k] = E + W O ; X[m-k] = conj(E - W O)
      double2 E = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
      double2 O = make_double2(0.5 * (zk.y + zm.y), -0.5 * (zk.x - zm.x));
      double2 WO = cmul(s.tw3[k], O);
      rp[pk] = cadd(E, WO);
      if (pm != pk) rp[pm] = cconj(csub(E, WO));
    }
  }
  __syncthreads();
}

// C2R twist: Zin[k] = (X[k] + conj X[m-k]) + i (X[k] - conj X[m-k]) e^{2 pi i k / N3}.
template <int M3C>
__device__ void c2r_twist_rows(const GridDev& g, const PlaneSmem& s, int nrow) {
  const int m3 = M3C > 0 ? M3C : g.m3, h3 = m3 + 1;
  const int total = nrow * (m3 / 2 + 1);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int k = t / nrow, row = t - k * nrow;
    double2* rp = s.slots + (size_t)row * h3;
    if (k == 0) {
      // real parts of the DC and Nyquist bins (Grid.ifft keeps .real)
      double x0 = rp[0].x, xm = rp[m3].x;
      rp[0] = make_double2(x0 + xm, x0 - xm);
    } else {
      const int pk = s.zpos[k], pm = s.zpos[m3 - k];
      double2 xk = rp[pk], xm = rp[pm];
      double2 e = make_double2(xk.x + xm.x, xk.y - xm.y);
      double2 o = cmulc(make_double2(xk.x - xm.x, xk.y + xm.y), s.tw3[k]);
      rp[pk] = make_double2(e.x - o.y, e.y + o.x);
      if (pm != pk) rp[pm] = make_double2(e.x + o.y, -e.y + o.x);
    }
  }
  __syncthreads();
}

// z rows only: real rows (natural z) -> DIF z + R2C twist, and back.
template <int M3C>
__device__ void row_forward(const GridDev& g, const PlaneSmem& s, int nrow) {
  const int h3 = (M3C > 0 ? M3C : g.m3) + 1;
  axis_fft<false, M3C>(s.slots, g.ax3, s.tw3, 2, nrow, h3, 1);
  r2c_twist_rows<M3C>(g, s, nrow);
}

template <int M3C>
__device__ void row_inverse(const GridDev& g, const PlaneSmem& s, int nrow) {
  const int h3 = (M3C > 0 ? M3C : g.m3) + 1;
  c2r_twist_rows<M3C>(g, s, nrow);
  axis_fft<true, M3C>(s.slots, g.ax3, s.tw3, 2, nrow, h3, 1);
}

// Forward: real rows (natural z) in each slot -> DIF z, R2C twist, DIF y.
template <int N2C, int M3C>
__device__ void plane_forward(const GridDev& g, const PlaneSmem& s, int nslot) {
  const PlaneShape<N2C, M3C> sh(g);
  row_forward<M3C>(g, s, nslot * sh.n2);
  axis_fft<false, N2C>(s.slots, g.ax2, s.tw2, 1, nslot * sh.h3, 1, nslot * sh.h3);
}

// Inverse: spectrum slots -> DIT y, C2R twist, DIT z -> real rows (unnormalised).
template <int N2C, int M3C>
__device__ void plane_inverse(const GridDev& g, const PlaneSmem& s, int nslot) {
  const PlaneShape<N2C, M3C> sh(g);
  axis_fft<true, N2C>(s.slots, g.ax2, s.tw2, 1, nslot * sh.h3, 1, nslot * sh.h3);
  row_inverse<M3C>(g, s, nslot * sh.n2);
}

// Real element (y=r, z=j) of field f.
template <int N2C, int M3C>
__device__ __forceinline__ double& rel(const PlaneSmem& s, const PlaneShape<N2C, M3C>& sh, int nslot, int f, int r,
                                       int j) {
  return ((double*)(s.slots + ((size_t)r * nslot + f) * sh.h3))[j];
}

// Copy nslot spectrum planes (global: field f at src + f*fs + plane_off, [n2][h3]) into smem.
// Every element is an asynchronous 16-byte global-to-shared copy
// (cp.async.cg: through L2, no register staging), so all of a thread's
// copies are in flight at once and the plane's load latency is paid once;
// the thread waits for its own copies, and the caller's __syncthreads()
// makes the whole plane visible.
template <int N2C, int M3C>
__device__ inline void load_spec_planes(const GridDev& g, const PlaneSmem& s, int nslot, const double2* src,
                                        size_t plane_off, size_t fs) {
  const PlaneShape<N2C, M3C> sh(g);
  const int h3 = sh.h3, cnt = sh.n2 * h3;
  for (int f = 0; f < nslot; ++f) {
    const double2* p = src + f * fs + plane_off;
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      const int r = i / h3, c = i - r * h3;
      const unsigned dst = (unsigned)__cvta_generic_to_shared(s.slots + ((size_t)r * nslot + f) * h3 + c);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(p + i) : "memory");
    }
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

template <int N2C, int M3C>
__device__ inline void store_spec_planes(const GridDev& g, const PlaneSmem& s, int nslot, double2* dst,
                                         size_t plane_off, size_t fs) {
  const PlaneShape<N2C, M3C> sh(g);
  const int h3 = sh.h3, cnt = sh.n2 * h3;
  for (int f = 0; f < nslot; ++f) {
    double2* p = dst + f * fs + plane_off;
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      const int r = i / h3, c = i - r * h3;
      p[i] = s.slots[((size_t)r * nslot + f) * h3 + c];
    }
  }
}

// ---------------------------------------------------- block reductions --
__device__ inline double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = (l < nw) ? red[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  return r;  // valid in thread 0
}

__device__ inline double block_max(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double r = -INFINITY;
  if (threadIdx.x < 32) {
    r = (l < nw) ? red[l] : -INFINITY;
    for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
  }
  return r;
}

__device__ inline void put_part(double* part, int b, int q, int nslot, int slot, double v) {
  if (threadIdx.x == 0) part[((size_t)b * NQ + q) * nslot + slot] = v;
}

// ================================================ 3D FFT (setup / tests) ==
template <int N2C, int M3C>
__global__ void __launch_bounds__(CMM_PLANE_THREADS, CMM_PLANE_MINB_FOR(N2C))
k_plane_r2c(GridDev g, const int* __restrict__ active, const double* __restrict__ in, double2* __restrict__ out) {
  const int i1 = blockIdx.x, b = blockIdx.y;
  if (active && !active[b]) return;
  PlaneSmem s = plane_smem_setup<N2C, M3C>(g, 1);
  const PlaneShape<N2C, M3C> sh(g);
  const size_t roff = ((size_t)b * g.n1 + i1) * sh.n2 * sh.n3;
  for (int i = threadIdx.x; i < sh.n2 * sh.n3; i += blockDim.x) {
    const int r = i / sh.n3, j = i - r * sh.n3;
    rel(s, sh, 1, 0, r, j) = __ldg(in + roff + i);
  }
  __syncthreads();
  plane_forward<N2C, M3C>(g, s, 1);
  store_spec_planes<N2C, M3C>(g, s, 1, out, ((size_t)b * g.n1 + i1) * sh.n2 * sh.h3, 0);
}

template <int N2C, int M3C>
__global__ void __launch_bounds__(CMM_PLANE_THREADS, CMM_PLANE_MINB_FOR(N2C))
k_plane_c2r(GridDev g, const double2* __restrict__ in, double* __restrict__ out) {
  const int i1 = blockIdx.x, b = blockIdx.y;
  PlaneSmem s = plane_smem_setup<N2C, M3C>(g, 1);
  const PlaneShape<N2C, M3C> sh(g);
  load_spec_planes<N2C, M3C>(g, s, 1, in, ((size_t)b * g.n1 + i1) * sh.n2 * sh.h3, 0);
  __syncthreads();
  plane_inverse<N2C, M3C>(g, s, 1);
  const size_t roff = ((size_t)b * g.n1 + i1) * sh.n2 * sh.n3;
  for (int i = threadIdx.x; i < sh.n2 * sh.n3; i += blockDim.x) {
    const int r = i / sh.n3, j = i - r * sh.n3;
    out[roff + i] = rel(s, sh, 1, 0, r, j);
  }
}

// Column tile: TC consecutive (y,z) columns of one instance, all N1 x rows.
// Shared layout [n1][nslot][tc]: element (f, x=p1, c) at (p1*nslot + f)*tc + c,
// so the x pencils (p = f*tc + c) are uniform with estride nslot*tc.
struct ColSmem {
  double2* slots;
  double2* tw1;
  double2* tmp;   // direct-DFT stage scratch (x axes with a prime factor > 16)
};

__host__ __device__ inline size_t col_smem_bytes(int n1, int tc, int nslot, int big) {
  return sizeof(double2) * ((size_t)nslot * n1 * tc * (big ? 2 : 1) + n1);
}

template <int N1C, int TCC>
struct ColShape {
  int n1, tc;
  __device__ ColShape(const GridDev& g, int tc_rt) : n1(N1C > 0 ? N1C : g.n1), tc(TCC ? TCC : tc_rt) {}
};

template <int N1C, int TCC>
__device__ inline ColSmem col_smem_setup(const GridDev& g, const ColShape<N1C, TCC>& sh, int nslot) {
  extern __shared__ double2 smem_d2[];
  ColSmem s;
  s.slots = smem_d2;
  s.tw1 = s.slots + (size_t)nslot * sh.n1 * sh.tc;
  s.tmp = g.ax1.big ? s.tw1 + sh.n1 : nullptr;
  for (int i = threadIdx.x; i < sh.n1; i += blockDim.x) s.tw1[i] = g.tw1[i];
  return s;
}

template <int N1C, int TCC>
__device__ __forceinline__ double2& cel(const ColSmem& s, const ColShape<N1C, TCC>& sh, int nslot, int f, int p1,
                                        int c) {
  return s.slots[((size_t)p1 * nslot + f) * sh.tc + c];
}

// Load a tile [n1][tc] of one field (instance b) into slot f; zero past the last column.
template <int N1C, int TCC>
__device__ inline void load_col_tile(const GridDev& g, const ColSmem& s, const ColShape<N1C, TCC>& sh, int nslot,
                                     int f, const double2* src, int b, int c0, const int* rowmap) {
  const int nc = g.n2 * g.h3;
  const size_t base = (size_t)b * sh.n1 * nc;
  for (int i = threadIdx.x; i < sh.n1 * sh.tc; i += blockDim.x) {
    const int p1 = i / sh.tc, c = i - p1 * sh.tc;
    const int col = c0 + c;
    const int r = rowmap ? rowmap[p1] : p1;
    cel(s, sh, nslot, f, p1, c) = (col < nc) ? src[base + (size_t)r * nc + col] : make_double2(0.0, 0.0);
  }
}

template <int N1C, int TCC>
__device__ inline void store_col_tile(const GridDev& g, const ColSmem& s, const ColShape<N1C, TCC>& sh, int nslot,
                                      int f, double2* dst, int b, int c0, const int* rowmap) {
  const int nc = g.n2 * g.h3;
  const size_t base = (size_t)b * sh.n1 * nc;
  for (int i = threadIdx.x; i < sh.n1 * sh.tc; i += blockDim.x) {
    const int p1 = i / sh.tc, c = i - p1 * sh.tc;
    const int col = c0 + c;
    const int r = rowmap ? rowmap[p1] : p1;
    if (col < nc) dst[base + (size_t)r * nc + col] = cel(s, sh, nslot, f, p1, c);
  }
}

// x transform of `nfield` fields starting at field f0 of an nslot tile.
template <bool INV, int N1C, int TCC>
__device__ inline void col_fft(const GridDev& g, const ColSmem& s, const ColShape<N1C, TCC>& sh, int nslot, int f0,
                               int nfield) {
  axis_fft<INV, N1C>(s.slots + (size_t)f0 * sh.tc, g.ax1, s.tw1, 1, nfield * sh.tc, 1, nslot * sh.tc, s.tmp);
}

// Plain x transform of a tile (setup / tests).  HBM spectra keep x natural:
// forward loads natural rows, runs DIF and stores row k1pos[p]; inverse loads
// row k1pos[p] into position p, runs DIT and stores natural rows.
template <int N1C, int TCC>
__global__ void __launch_bounds__(CMM_COL_THREADS, CMM_COL_MINB)
k_col_fft(GridDev g, const double2* in, double2* out, int tc, int inv) {
  const int b = blockIdx.y, c0 = blockIdx.x * (TCC ? TCC : tc);
  const ColShape<N1C, TCC> sh(g, tc);
  ColSmem s = col_smem_setup(g, sh, 1);
  load_col_tile(g, s, sh, 1, 0, in, b, c0, inv ? g.k1pos : nullptr);
  __syncthreads();
  if (inv) col_fft<true>(g, s, sh, 1, 0, 1);
  else col_fft<false>(g, s, sh, 1, 0, 1);
  store_col_tile(g, s, sh, 1, 0, out, b, c0, inv ? nullptr : g.k1pos);
}

// ================================================ FMT weights ===========
// Weights of HardSphereFunctional._init_weight_functions
// (cmmdft/functionals.py:421-455) at one stored frequency.  Vector weights
// are replaced by their Hermitian part: zero on their own axis' Nyquist plane
// (what Grid.ifft's .real keeps of a purely imaginary self-conjugate bin).
struct Weights {
  double w0;      // kw0 = j0(kR) sigma_L
  double w3;      // kw3 = (4 pi R^3 / 3) * 3 (sin x - x cos x) / x^3 * sigma_L
  double v[3];    // kwv2 = -i * kw3 * k  -> stored as the real factor of -i
};

__device__ __forceinline__ double2 fmt_scalar_weights(double kx, double ky, double kz, double sl, double R) {
  const double kk = sqrt(kx * kx + ky * ky + kz * kz);
  const double om = kk * R;
  if (fabs(om) <= 1e-8)  // np.isclose(omega, 0)
    return make_double2(sl, (4.0 * M_PI * R * R * R / 3.0) * sl);
  double sn, cs;
  sincos(om, &sn, &cs);
  const double y = M_PI * (om / M_PI);
  const double j0 = sin(y) / y;  // np.sinc(omega / pi)
  const double j2 = 3.0 * (sn - om * cs) / (om * om * om);
  return make_double2(j0 * sl, (4.0 * M_PI * R * R * R / 3.0) * (j2 * sl));
}

// Weights at (x position p1, column col); from the table when given.
__device__ __forceinline__ Weights fmt_weights_at(const GridDev& g, const double2* __restrict__ wtab, int p1,
                                                  int col, double R) {
  const int p2 = col / g.h3, p3 = col - p2 * g.h3;
  const double kx = g.kp1[p1], ky = g.kp2[p2], kz = g.kp3[p3];
  double2 ws;
  if (wtab) {
    ws = __ldg(wtab + (size_t)p1 * g.n2 * g.h3 + col);
  } else {
    const double sl = (g.sl1[p1] * g.sl2[p2]) * g.sl3[p3];
    ws = fmt_scalar_weights(kx, ky, kz, sl, R);
  }
  Weights w;
  w.w0 = ws.x;
  w.w3 = ws.y;
  const bool zero = (kx == 0.0 && ky == 0.0 && kz == 0.0);
  w.v[0] = (zero || g.nq1[p1]) ? 0.0 : w.w3 * kx;
  w.v[1] = (zero || g.nq2[p2]) ? 0.0 : w.w3 * ky;
  w.v[2] = (zero || g.nq3[p3]) ? 0.0 : w.w3 * kz;
  return w;
}

// Tensor weights B (k_i k_j / k^2 - delta_ij / 3), B = -4 pi R^2 (j2 - j0) sigma_L
// (functionals.py:457-487), in the order xx, xy, xz, yy, yz, zz, from the scalar
// weights w0 = j0 sigma_L and w3 = (4 pi R^3 / 3) j2 sigma_L.  All vanish at k = 0.
// Under k -> -k an off-diagonal weight k_i k_j changes sign once for every
// one of its two components that is not on its axis' Nyquist plane (the
// Nyquist frequency maps to itself).  Its Hermitian part (what Grid.ifft's
// .real keeps) is therefore zero where exactly one of the two is at Nyquist,
// and the weight itself elsewhere.
__device__ __forceinline__ void tensor_weights_at(const GridDev& g, int p1, int col, double w0, double w3,
                                                  double R, double* tw) {
  const int p2 = col / g.h3, p3 = col - p2 * g.h3;
  const double kx = g.kp1[p1], ky = g.kp2[p2], kz = g.kp3[p3];
  const double K = sqrt(kx * kx + ky * ky + kz * kz);
  if (!(K > 0.0)) {
    for (int c = 0; c < 6; ++c) tw[c] = 0.0;
    return;
  }
  const double K2 = K * K;
  const double B = -4 * M_PI * (R * R) * (w3 / (4.0 * M_PI * R * R * R / 3.0) - w0);
  const int q1 = g.nq1[p1], q2 = g.nq2[p2], q3 = g.nq3[p3];
  tw[0] = B * ((kx * kx) / K2 - 1.0 / 3);
  tw[1] = (q1 != q2) ? 0.0 : B * ((kx * ky) / K2);
  tw[2] = (q1 != q3) ? 0.0 : B * ((kx * kz) / K2);
  tw[3] = B * ((ky * ky) / K2 - 1.0 / 3);
  tw[4] = (q2 != q3) ? 0.0 : B * ((ky * kz) / K2);
  tw[5] = B * ((kz * kz) / K2 - 1.0 / 3);
}

// WDA weight (WDAVFunctional._init_weight_function, cmmdft/functionals.py:1139-1155):
// 3 (sin x - x cos x) / x^3 sigma_L at x = |k| D, 1 sigma_L at k = 0.
// D < 0 selects the LDA part (LDAFunctional, cmmdft/functionals.py:1085-1114):
// weight 1 at every frequency, without the Lanczos factor, so that the
// "weighted density" is the density itself up to the transforms' rounding.
__device__ __forceinline__ double wda_weight_at(const GridDev& g, int p1, int col, double D) {
  if (D < 0) return 1.0;
  const int p2 = col / g.h3, p3 = col - p2 * g.h3;
  const double kx = g.kp1[p1], ky = g.kp2[p2], kz = g.kp3[p3];
  const double sl = (g.sl1[p1] * g.sl2[p2]) * g.sl3[p3];
  const double om = sqrt(kx * kx + ky * ky + kz * kz) * D;
  if (fabs(om) <= 1e-8) return sl;
  double sn, cs;
  sincos(om, &sn, &cs);
  return (3.0 * (sn - om * cs) / (om * om * om)) * sl;
}

// SumOfEOS(MBWR, CS, MFA) excess free energy per volume and its density
// derivative at one weighted density (cmmdft/eos.py:226-265, 295-546).  A
// template on the scalar type: double for the functional, Dual for the
// second derivative in the Hessian-vector product.
template <class S>
__device__ __forceinline__ void wda_eos(const cmm_wda_eos& e, S rho, S& fv, S& dfv) {
  // MBWR (eos.py:368-422)
  const S rr = rho * e.sigma3;
  S A = 0.0, dA = 0.0, p = 1.0;  // p = rr^i
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    dA += e.a[i] * p * e.sigma3;
    p *= rr;
    A += e.a[i] / (i + 1) * p;
  }
  const S rr2 = rr * rr;
  const S F = exp(-e.gamma * rr2);
  const double ig = 1.0 / (2 * e.gamma);
  S G = ig * (1 - F), q = 1.0, podd = rr;  // q = rr^(2(n-1)), podd = rr^(2t+1)
  A += e.b[0] * G;
  dA += e.b[0] * e.sigma3 * podd * F;
#pragma unroll
  for (int n = 2; n <= 6; ++n) {
    q *= rr2;
    G = -ig * (F * q - 2 * (n - 1) * G);
    A += e.b[n - 1] * G;
    podd *= rr2;
    dA += e.b[n - 1] * e.sigma3 * podd * F;
  }
  const S fp_m = A * e.epsilon, dfp_m = dA * e.epsilon;
  // Carnahan-Starling (eos.py:503-509)
  const S er = e.eta * rho, om = 1 - er;
  const S fp_c = e.kT * (4 * e.eta * rho - 3 * er * er) / (om * om);
  const S dfp_c = 2 * e.kT * e.eta * (2 - er) / (om * om * om);
  // mean-field EOS (eos.py:536-540)
  const S fp_a = e.a_mfa * rho;
  const double dfp_a = e.a_mfa;
  S d_m = rho * dfp_m; d_m += fp_m;
  S d_c = rho * dfp_c; d_c += fp_c;
  S d_a = rho * dfp_a; d_a += fp_a;
  dfv = 0.0;
  dfv += e.factors[0] * d_m;
  dfv += e.factors[1] * d_c;
  dfv += e.factors[2] * d_a;
  fv = 0.0;
  fv += e.factors[0] * (rho * fp_m);
  fv += e.factors[1] * (rho * fp_c);
  fv += e.factors[2] * (rho * fp_a);
}

// Weight table (w0, w3) in the column-pass layout [x DIF position][column].
__global__ void k_fmt_weights(GridDev g, double R, double2* __restrict__ wtab) {
  const int nc = g.n2 * g.h3;
  const long long tot = (long long)g.n1 * nc;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= tot) return;
  const int p1 = (int)(idx / nc), col = (int)(idx - (long long)p1 * nc);
  const int p2 = col / g.h3, p3 = col - p2 * g.h3;
  const double sl = (g.sl1[p1] * g.sl2[p2]) * g.sl3[p3];
  wtab[idx] = fmt_scalar_weights(g.kp1[p1], g.kp2[p2], g.kp3[p3], sl, R);
}

// ================================== column pass 1: rho_hat -> 5 fields ==
// Outputs (field stride fsw): 0 = n0 (w0), 1 = n3 (w3), 2..4 = nv2 (x, y, z).
// The WDA field is a template parameter, as in the plane pass, so that the
// plain kernels keep their register budget.
// LS (hybrid line search): the input is the spectrum of a residual r; the
// spectrum of the current density rho (rho_ref) is forwarded alongside so
// that the MFA energy of rho + a r can be assembled from sum |r|^2 K and the
// cross term sum Re(conj(rho) r) K (into ls_part, CMM_LS_MFA_RR / _XR).
template <int N1C, int TCC, bool WDA, bool TEN, bool LS>
__device__ __forceinline__ void col_weights_body(GridDev g, const int* __restrict__ active, double R,
                                                 double inv_npts, const double2* __restrict__ rhohat,
                                                 double2* __restrict__ wout, size_t fsw,
                                                 const double2* __restrict__ kst, const double2* __restrict__ wtab,
                                                 double* __restrict__ part, int nslot_part, int want_value, int tc,
                                                 double wda_D, const double2* __restrict__ rho_ref,
                                                 double* __restrict__ ls_part) {
  const int b = blockIdx.y, tile = blockIdx.x;
  if (active && !active[b]) return;
  const ColShape<N1C, TCC> sh(g, tc);
  const int c0 = tile * sh.tc;
  const int tb = WDA ? 6 : 5;           // first tensor field
  const int nw = tb + (TEN ? 6 : 0);    // n0, n3, nv2 x/y/z, WDA, then the tensor densities
  const int ns = nw + (LS ? 1 : 0);     // slots: the weighted densities (+ rho_ref)
  ColSmem s = col_smem_setup(g, sh, ns);
  load_col_tile(g, s, sh, ns, 0, rhohat, b, c0, nullptr);
  if constexpr (LS) load_col_tile(g, s, sh, ns, nw, rho_ref, b, c0, nullptr);
  __syncthreads();
  col_fft<false>(g, s, sh, ns, 0, 1);
  if constexpr (LS) col_fft<false>(g, s, sh, ns, nw, 1);
  const int nc = g.n2 * g.h3;
  double mfa = 0.0, mxr = 0.0;
  for (int i = threadIdx.x; i < sh.n1 * sh.tc; i += blockDim.x) {
    const int p1 = i / sh.tc, c = i - p1 * sh.tc;
    const int col = c0 + c;
    if (col >= nc) continue;
    double2 F = cel(s, sh, ns, 0, p1, c);
    const Weights w = fmt_weights_at(g, wtab, p1, col, R);
    if (want_value || LS) {
      const double2 K = __ldg(kst + (size_t)p1 * nc + col);
      const double w3 = g.wt3[col - (col / g.h3) * g.h3];
      mfa += w3 * (F.x * F.x + F.y * F.y) * K.x;
      if constexpr (LS) {
        const double2 P = cel(s, sh, ns, nw, p1, c);
        mxr += w3 * (P.x * F.x + P.y * F.y) * K.x;
      }
    }
    F = cscale(F, inv_npts);
    if (WDA) cel(s, sh, ns, 5, p1, c) = cscale(F, wda_weight_at(g, p1, col, wda_D));
    cel(s, sh, ns, 1, p1, c) = cscale(F, w.w3);
    // -i * v * F
    cel(s, sh, ns, 2, p1, c) = make_double2(F.y * w.v[0], -F.x * w.v[0]);
    cel(s, sh, ns, 3, p1, c) = make_double2(F.y * w.v[1], -F.x * w.v[1]);
    cel(s, sh, ns, 4, p1, c) = make_double2(F.y * w.v[2], -F.x * w.v[2]);
    if constexpr (TEN) {
      double tw[6];
      tensor_weights_at(g, p1, col, w.w0, w.w3, R, tw);
      for (int q = 0; q < 6; ++q) cel(s, sh, ns, tb + q, p1, c) = cscale(F, tw[q]);
    }
    cel(s, sh, ns, 0, p1, c) = cscale(F, w.w0);
  }
  __syncthreads();
  col_fft<true>(g, s, sh, ns, 0, nw);
  for (int f = 0; f < nw; ++f) store_col_tile(g, s, sh, ns, f, wout + f * fsw, b, c0, nullptr);
  __shared__ double red[32];
  if (want_value && !LS) {
    double t = block_sum(mfa, red);
    put_part(part, b, CMM_STAT_MFA, nslot_part, tile, t);
  }
  if constexpr (LS) {
    double t = block_sum(mfa, red);
    if (threadIdx.x == 0) ls_part[((size_t)b * CMM_NLS + CMM_LS_MFA_RR) * nslot_part + tile] = t;
    t = block_sum(mxr, red);
    if (threadIdx.x == 0) ls_part[((size_t)b * CMM_NLS + CMM_LS_MFA_XR) * nslot_part + tile] = t;
  }
}

#define COL_WEIGHTS_ARGS                                                                                   \
  GridDev g, const int *__restrict__ active, double R, double inv_npts, const double2 *__restrict__ rhohat, \
      double2 *__restrict__ wout, size_t fsw, const double2 *__restrict__ kst,                             \
      const double2 *__restrict__ wtab, double *__restrict__ part, int nslot_part, int want_value, int tc,  \
      double wda_D, const double2 *__restrict__ rho_ref, double *__restrict__ ls_part
#define COL_WEIGHTS_KERNEL(name, wda, ten, ls)                                                          \
  template <int N1C, int TCC>                                                                            \
  __global__ void __launch_bounds__(CMM_COL_THREADS, CMM_COL_MINB_FOR(N1C)) name(COL_WEIGHTS_ARGS) {                  \
    col_weights_body<N1C, TCC, wda, ten, ls>(g, active, R, inv_npts, rhohat, wout, fsw, kst, wtab, part, \
                                             nslot_part, want_value, tc, wda_D, rho_ref, ls_part);       \
  }
COL_WEIGHTS_KERNEL(k_col_weights, false, false, false)
COL_WEIGHTS_KERNEL(k_col_weights_wda, true, false, false)
COL_WEIGHTS_KERNEL(k_col_weights_t, false, true, false)
COL_WEIGHTS_KERNEL(k_col_weights_wda_t, true, true, false)
COL_WEIGHTS_KERNEL(k_col_weights_ls, false, false, true)
COL_WEIGHTS_KERNEL(k_col_weights_ls_wda, true, false, true)
COL_WEIGHTS_KERNEL(k_col_weights_ls_t, false, true, true)
COL_WEIGHTS_KERNEL(k_col_weights_ls_wda_t, true, true, true)

// ======================== column pass 2: dPhi spectra -> C1 spectrum ====
// Inputs: 5 dPhi spectra (field stride fsg): g_s (pairs with w0), g3 (w3),
// gv (x,y,z, pairs with kwv2); rho_hat for the MFA term.  gin == NULL: MFA only.
template <int N1C, int TCC, bool WDA, bool TEN>
__device__ __forceinline__ void col_backconv_body(GridDev g, const int* __restrict__ active, double R,
                                                  double scale, const double2* __restrict__ gin, size_t fsg,
                                                  const double2* __restrict__ rhohat,
                                                  const double2* __restrict__ kst, const double2* __restrict__ wtab,
                                                  double2* __restrict__ chat, int tc, double wda_D,
                                                  double inv_npts) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  const ColShape<N1C, TCC> sh(g, tc);
  const int c0 = blockIdx.x * sh.tc;
  const int tb = WDA ? 6 : 5;           // first tensor field
  const int nin = tb + (TEN ? 6 : 0);
  const int ns = nin + 1;    // 5 dPhi (+1 WDA, +6 tensor) fields, then rho_hat
  const int fr = nin;        // slot of rho_hat
  ColSmem s = col_smem_setup(g, sh, ns);
  const bool hs = (gin != nullptr);
  if (hs)
    for (int f = 0; f < nin; ++f) load_col_tile(g, s, sh, ns, f, gin + f * fsg, b, c0, nullptr);
  load_col_tile(g, s, sh, ns, fr, rhohat, b, c0, nullptr);
  __syncthreads();
  if (hs) col_fft<false>(g, s, sh, ns, 0, ns);
  else col_fft<false>(g, s, sh, ns, fr, 1);
  const int nc = g.n2 * g.h3;
  for (int i = threadIdx.x; i < sh.n1 * sh.tc; i += blockDim.x) {
    const int p1 = i / sh.tc, c = i - p1 * sh.tc;
    const int col = c0 + c;
    if (col >= nc) continue;
    double2 acc = make_double2(0.0, 0.0);
    if (hs) {
      const Weights w = fmt_weights_at(g, wtab, p1, col, R);
      acc = cadd(cscale(cel(s, sh, ns, 0, p1, c), w.w0), cscale(cel(s, sh, ns, 1, p1, c), w.w3));
      // - sum_j G_j * (-i v_j) = + i * sum_j v_j G_j
      double2 gv = make_double2(0.0, 0.0);
      for (int a = 0; a < 3; ++a) gv = cadd(gv, cscale(cel(s, sh, ns, 2 + a, p1, c), w.v[a]));
      acc = cadd(acc, make_double2(-gv.y, gv.x));
      if constexpr (TEN) {  // + sum_ij fft(dPhi/dn_ij) w_ij (functionals.py:602-605)
        double tw[6];
        tensor_weights_at(g, p1, col, w.w0, w.w3, R, tw);
        for (int q = 0; q < 6; ++q) acc = cadd(acc, cscale(cel(s, sh, ns, tb + q, p1, c), tw[q]));
      }
      acc = cscale(acc, scale);
      // WDA: ifft(fft(dphi) kw), no 1/beta (the EOS derivative is an energy)
      if (WDA) acc = cadd(acc, cscale(cel(s, sh, ns, 5, p1, c), wda_weight_at(g, p1, col, wda_D) * inv_npts));
    }
    const double2 K = __ldg(kst + (size_t)p1 * nc + col);
    acc = cadd(acc, cmul(cel(s, sh, ns, fr, p1, c), K));
    cel(s, sh, ns, 0, p1, c) = acc;
  }
  __syncthreads();
  col_fft<true>(g, s, sh, ns, 0, 1);
  store_col_tile(g, s, sh, ns, 0, chat, b, c0, nullptr);
}

#define COL_BACKCONV_ARGS                                                                                  \
  GridDev g, const int *__restrict__ active, double R, double scale, const double2 *__restrict__ gin,      \
      size_t fsg, const double2 *__restrict__ rhohat, const double2 *__restrict__ kst,                     \
      const double2 *__restrict__ wtab, double2 *__restrict__ chat, int tc, double wda_D, double inv_npts
#define COL_BACKCONV_KERNEL(name, wda, ten)                                                             \
  template <int N1C, int TCC>                                                                            \
  __global__ void __launch_bounds__(CMM_COL_THREADS, CMM_COL_MINB_FOR(N1C)) name(COL_BACKCONV_ARGS) {                          \
    col_backconv_body<N1C, TCC, wda, ten>(g, active, R, scale, gin, fsg, rhohat, kst, wtab, chat, tc,    \
                                          wda_D, inv_npts);                                              \
  }
COL_BACKCONV_KERNEL(k_col_backconv, false, false)
COL_BACKCONV_KERNEL(k_col_backconv_wda, true, false)
COL_BACKCONV_KERNEL(k_col_backconv_t, false, true)
COL_BACKCONV_KERNEL(k_col_backconv_wda_t, true, true)

// ===================================== plane pass: dPhi/dn (White-Bear) ==
// Arithmetic of _phi*, _dphi*, get_phi and _get_dphi_* (cmmdft/functionals.py:620-767).
// The pointwise functions are templates on the scalar type: double for the
// functional, Dual (cmm_dual.cuh) for its directional derivative in the
// Hessian-vector product.
template <class S>
struct PhiOutT { S gs, g3, gv[3], phi; };
using PhiOut = PhiOutT<double>;

template <class S>
__device__ __forceinline__ void phi_funcs(S n3, S ln, S n32, S n33, int base, S& p2, S& dp2, S& p3, S& dp3) {
  const S q = (1 - 2 * n3 + n32);
  const S c = (1 - 3 * n3 + 3 * n32 - n33);
  if (base == CMM_FMT) {
    p2 = 1 / (1.0 - n3);
    dp2 = 1 / q;
    p3 = 1 / (24 * M_PI * q);
    dp3 = 1 / (12 * M_PI * c);
  } else if (base == CMM_MFMT) {
    p2 = 1 / (1.0 - n3);
    dp2 = 1 / q;
    if (n3 <= 1e-8) {
      p3 = (1.0 - 2 * n3 / 9 - n32 / 18) / (24 * M_PI * q);
      dp3 = (8.0 / 3 - 0.5 * n3 - 0.1 * n32) / (36 * M_PI * c);
    } else {
      p3 = (n3 + q * ln) / (36 * M_PI * n32 * q);
      dp3 = -(2 * n3 - 5 * n32 + n33 + 2 * c * ln) / (36 * M_PI * n33 * c);
    }
  } else {  // WBII
    if (n3 <= 1e-8) {
      p2 = (1 + n32 / 9) / (1 - n3);
      dp2 = (1 + 2 * n3 / 9 + n32 / 18) / q;
      p3 = (1 - 4 * n3 / 9 + n32 / 18) / (24 * M_PI * q);
      dp3 = (7.0 / 3 - n3 / 2 + n32 / 10) / (36 * M_PI * c);
    } else {
      p2 = (5 * n3 - n32 + 2 * (1 - n3) * ln) / (3 * (n3 - n32));
      dp2 = -2 * (n3 - 3 * n32 + q * ln) / (3 * n32 * q);
      p3 = -2 * (n3 - 3 * n32 + n33 + ln * q) / ((3 * n32) * 24 * M_PI * q);
      dp3 = (2 * n3 - 5 * n32 + 6 * n33 - n32 * n32 + 2 * c * ln) / (36 * M_PI * n33 * c);
    }
  }
}

// Prefactor of phi3 (functionals.py:629-639): n2^3 (1 - xi)^3 ('a') or
// n2^3 - 3 n2 |nv2|^2, plus the tensor terms 9/2 (nv2 T nv2 - tr T^3) ('t').
template <bool TEN, class S>
__device__ __forceinline__ S fmt_pref3(S n2, S vx, S vy, S vz, S vv, const S* T, bool anti, S& xi) {
  S pref3;
  xi = 0.0;
  if (anti) {
    xi = vv / (n2 * n2 + 1e-16);
    xi = fmin(fmax(xi, 0.0), 1.0);
    const S om = 1 - xi;
    pref3 = (n2 * n2 * n2) * (om * om * om);
  } else {
    pref3 = n2 * n2 * n2 - 3.0 * n2 * vv;
  }
  if constexpr (TEN) {
    const S xx = T[0], xy = T[1], xz = T[2], yy = T[3], yz = T[4], zz = T[5];
    const S quad = xx * (vx * vx) + yy * (vy * vy) + zz * (vz * vz) + 2 * xy * vx * vy + 2 * xz * vx * vz +
                   2 * yz * vy * vz;
    const S tr3 = (xx * xx * xx + yy * yy * yy + zz * zz * zz) +
                       3 * (xx * xy * xy + xx * xz * xz + yy * xy * xy + yy * yz * yz + zz * xz * xz + zz * yz * yz) +
                       6 * xy * xz * yz;
    pref3 += 4.5 * quad;
    pref3 -= 4.5 * tr3;
  }
  return pref3;
}

// phi2 and phi3 alone (the values of phi_funcs).
__device__ __forceinline__ void phi_values(double n3, double ln, double n32, double n33, int base, double& p2,
                                           double& p3) {
  const double q = (1 - 2 * n3 + n32);
  if (base == CMM_FMT) {
    p2 = 1 / (1.0 - n3);
    p3 = 1 / (24 * M_PI * q);
  } else if (base == CMM_MFMT) {
    p2 = 1 / (1.0 - n3);
    p3 = (n3 <= 1e-8) ? (1.0 - 2 * n3 / 9 - n32 / 18) / (24 * M_PI * q) : (n3 + q * ln) / (36 * M_PI * n32 * q);
  } else if (n3 <= 1e-8) {
    p2 = (1 + n32 / 9) / (1 - n3);
    p3 = (1 - 4 * n3 / 9 + n32 / 18) / (24 * M_PI * q);
  } else {
    p2 = (5 * n3 - n32 + 2 * (1 - n3) * ln) / (3 * (n3 - n32));
    p3 = -2 * (n3 - 3 * n32 + n33 + ln * q) / ((3 * n32) * 24 * M_PI * q);
  }
}

// Phi alone at one point (get_phi, functionals.py:620-641).
template <bool TEN>
__device__ __forceinline__ double fmt_phi(double n0, double n3raw, double vx, double vy, double vz, const double* T,
                                          double R, int version) {
  const double n1 = R * n0;
  const double n2 = (4.0 * M_PI * R * R) * n0;
  const double i4r = 1.0 / (4 * M_PI * R);
  const double n3 = fmin(fmax(n3raw, 1e-30), 0.99);
  const double ln = log(1 - n3);
  const double n32 = n3 * n3, n33 = n32 * n3;
  double p2, p3, xi;
  phi_values(n3, ln, n32, n33, version & 3, p2, p3);
  const double vv = vx * vx + vy * vy + vz * vz;
  const double uv = (vx * i4r) * vx + (vy * i4r) * vy + (vz * i4r) * vz;
  const double pref3 = fmt_pref3<TEN, double>(n2, vx, vy, vz, vv, T, (version & CMM_ANTISYM) != 0, xi);
  const double s12 = n1 * n2 - uv;
  return n0 * (-ln) + s12 * p2 + pref3 * p3;
}

// With TEN, T holds the tensor densities (xx, xy, xz, yy, yz, zz) and gT
// receives dPhi/dn_T (functionals.py:634-639, 669-674, 692-717).
template <bool TEN, class S>
__device__ __forceinline__ PhiOutT<S> fmt_point(S n0, S n3raw, S vx, S vy, S vz, const S* T, S* gT, double R,
                                                int version) {
  const S n1 = R * n0;
  const S n2 = (4.0 * M_PI * R * R) * n0;
  const double i4r = 1.0 / (4 * M_PI * R);
  const S ux = vx * i4r, uy = vy * i4r, uz = vz * i4r;  // nv1
  const S n3 = fmin(fmax(n3raw, 1e-30), 0.99);
  const S ln = log(1 - n3);
  const S n32 = n3 * n3, n33 = n32 * n3;
  const int base = version & 3;
  const bool anti = (version & CMM_ANTISYM) != 0;
  S p2, dp2, p3, dp3;
  phi_funcs(n3, ln, n32, n33, base, p2, dp2, p3, dp3);
  const S p1 = -ln, dp1 = 1.0 / (1.0 - n3);
  const S vv = vx * vx + vy * vy + vz * vz;
  const S uv = ux * vx + uy * vy + uz * vz;
  S xi;
  const S pref3 = fmt_pref3<TEN, S>(n2, vx, vy, vz, vv, T, anti, xi);
  const S s12 = n1 * n2 - uv;
  PhiOutT<S> o;
  o.phi = n0 * p1 + s12 * p2 + pref3 * p3;
  const S d0 = p1;
  const S d1 = n2 * p2;
  S d2 = n1 * p2;
  if (anti) d2 += (3 * (n2 * n2) * (1 + xi) * ((1 - xi) * (1 - xi))) * p3;
  else d2 += 3 * (n2 * n2 - vv) * p3;
  const S d3 = n0 * dp1 + s12 * dp2 + pref3 * dp3;
  const S f3 = anti ? (-6 * n2 * ((1 - xi) * (1 - xi)) * p3) : (-6 * n2 * p3);
  // dPhi/dnv1 = -nv2 p2 ; dPhi/dnv2 = -nv1 p2 + nv2 f3
  o.gs = d0 + R * d1 + (4.0 * M_PI * R * R) * d2;
  o.g3 = d3;
  const S v[3] = {vx, vy, vz}, u[3] = {ux, uy, uz};
  S tv[3] = {0.0, 0.0, 0.0};  // 2 T v, the gradient of the quadratic form
  if constexpr (TEN) {
    tv[0] = 2 * (T[0] * vx + T[1] * vy + T[2] * vz);
    tv[1] = 2 * (T[1] * vx + T[3] * vy + T[4] * vz);
    tv[2] = 2 * (T[2] * vx + T[4] * vy + T[5] * vz);
  }
  for (int a = 0; a < 3; ++a) {
    const S dv1 = -v[a] * p2;
    S dv2 = -u[a] * p2 + v[a] * f3;
    if constexpr (TEN) dv2 += 4.5 * tv[a] * p3;
    o.gv[a] = dv1 * i4r + dv2;
  }
  if constexpr (TEN) {
    const S xx = T[0], xy = T[1], xz = T[2], yy = T[3], yz = T[4], zz = T[5];
    gT[0] = 4.5 * (vx * vx - 3 * (xx * xx + xy * xy + xz * xz)) * p3;
    gT[1] = 4.5 * ((vx * vy - 3 * (xx * xy + yy * xy + xz * yz)) * 2) * p3;
    gT[2] = 4.5 * ((vx * vz - 3 * (xx * xz + zz * xz + xy * yz)) * 2) * p3;
    gT[3] = 4.5 * (vy * vy - 3 * (yy * yy + xy * xy + yz * yz)) * p3;
    gT[4] = 4.5 * ((vy * vz - 3 * (yy * yz + zz * yz + xy * xz)) * 2) * p3;
    gT[5] = 4.5 * (vz * vz - 3 * (zz * zz + xz * xz + yz * yz)) * p3;
  }
  return o;
}

// The WDA branch is a template parameter: its EOS code, compiled into the
// plain kernel, pushes that kernel past the 64 registers a 1024-thread block
// allows and makes it spill.
template <int N2C, int M3C, bool has_wda>
__device__ __forceinline__ void plane_fmt_body(GridDev g, const int* __restrict__ active, double R, int version,
                                               const cmm_wda_eos& wda, const double2* __restrict__ win,
                                               size_t fsw, double2* __restrict__ gout, size_t fsg,
                                               double* __restrict__ part, int nslot_part, int want,
                                               double* __restrict__ wd, size_t fsr) {
  const int i1 = blockIdx.x, b = blockIdx.y;
  if (active && !active[b]) return;
  const int ns = has_wda ? 6 : 5;
  PlaneSmem s = plane_smem_setup<N2C, M3C>(g, ns);
  const PlaneShape<N2C, M3C> sh(g);
  const size_t poff = ((size_t)b * g.n1 + i1) * sh.n2 * sh.h3;
  load_spec_planes<N2C, M3C>(g, s, ns, win, poff, fsw);
  __syncthreads();
  plane_inverse<N2C, M3C>(g, s, ns);
  double phi = 0.0, n3max = -INFINITY, fwda = 0.0;
  const bool do_c1 = (want & 1) != 0, do_phi = (want & 3) != 0;
  const size_t roff = ((size_t)b * g.n1 + i1) * sh.n2 * sh.n3;
  for (int i = threadIdx.x; i < sh.n2 * sh.n3; i += blockDim.x) {
    const int r = i / sh.n3, j = i - r * sh.n3;
    double& a0 = rel(s, sh, ns, 0, r, j);
    double& a3 = rel(s, sh, ns, 1, r, j);
    double& ax = rel(s, sh, ns, 2, r, j);
    double& ay = rel(s, sh, ns, 3, r, j);
    double& az = rel(s, sh, ns, 4, r, j);
    n3max = fmax(n3max, a3);
    if (want & 8)  // the weighted densities themselves (hybrid line search)
      for (int f = 0; f < ns; ++f) wd[f * fsr + roff + i] = rel(s, sh, ns, f, r, j);
    if (do_phi) {
      PhiOut o = fmt_point<false, double>(a0, a3, ax, ay, az, nullptr, nullptr, R, version);
      phi += o.phi;
      if (do_c1) {
        a0 = o.gs; a3 = o.g3; ax = o.gv[0]; ay = o.gv[1]; az = o.gv[2];
      }
      if (has_wda) {
        double& aw = rel(s, sh, ns, 5, r, j);
        double fv, dfv;
        wda_eos(wda, aw, fv, dfv);
        fwda += fv;
        if (do_c1) aw = dfv;
      }
    }
  }
  __syncthreads();
  __shared__ double red[32];
  if (want & 2) {
    double t = block_sum(phi, red);
    put_part(part, b, CMM_STAT_PHI, nslot_part, i1, t);
    if (has_wda) {
      t = block_sum(fwda, red);
      put_part(part, b, CMM_STAT_WDA, nslot_part, i1, t);
    }
  }
  if (want & 4) {
    double t = block_max(n3max, red);
    put_part(part, b, CMM_STAT_N3MAX, nslot_part, i1, t);
  }
  if (!do_c1) return;
  __syncthreads();
  plane_forward<N2C, M3C>(g, s, ns);
  store_spec_planes<N2C, M3C>(g, s, ns, gout, poff, fsg);
}

template <int N2C, int M3C>
__global__ void __launch_bounds__(CMM_FMT_THREADS)
k_plane_fmt(GridDev g, const int* __restrict__ active, double R, int version, cmm_wda_eos wda,
            const double2* __restrict__ win, size_t fsw, double2* __restrict__ gout, size_t fsg,
            double* __restrict__ part, int nslot_part, int want, double* __restrict__ wd, size_t fsr) {
  plane_fmt_body<N2C, M3C, false>(g, active, R, version, wda, win, fsw, gout, fsg, part, nslot_part, want, wd,
                                  fsr);
}

template <int N2C, int M3C>
__global__ void __launch_bounds__(CMM_FMT_THREADS)
k_plane_fmt_wda(GridDev g, const int* __restrict__ active, double R, int version, cmm_wda_eos wda,
                const double2* __restrict__ win, size_t fsw, double2* __restrict__ gout, size_t fsg,
                double* __restrict__ part, int nslot_part, int want, double* __restrict__ wd, size_t fsr) {
  plane_fmt_body<N2C, M3C, true>(g, active, R, version, wda, win, fsw, gout, fsg, part, nslot_part, want, wd,
                                 fsr);
}

// ---------------------------------------- plane pass split over 2 CTAs ---
// The same plane pass with the plane's fields split between the two CTAs of
// a cluster (fields [0, nA) on rank 0, [nA, ns) on rank 1; nA = ceil(ns/2)),
// so that a CTA holds ~100 KB instead of ~170 KB of shared memory and two
// CTAs (of different planes) share an SM: one block's memory phases overlap
// the other's FP64 phases.  Each CTA transforms its own fields; the
// pointwise step reads and writes every field through distributed shared
// memory.  The results are bit for bit those of plane_fmt_body: CTA rank r,
// thread t plays thread v = r * T + t of the one-CTA pass (T = half its
// block) and visits the same points in the same order, and the block
// reductions combine the same 32-lane warp partials in the same tree.
#define CMM_FMT2_THREADS (CMM_FMT_THREADS / 2)

template <int N2C, int M3C, bool has_wda>
__device__ __forceinline__ void plane_fmt_body_c2(GridDev g, const int* __restrict__ active, double R, int version,
                                                  const cmm_wda_eos& wda, const double2* __restrict__ win,
                                                  size_t fsw, double2* __restrict__ gout, size_t fsg,
                                                  double* __restrict__ part, int nslot_part, int want,
                                                  double* __restrict__ wd, size_t fsr) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const unsigned rank = cl.block_rank();
  const int i1 = blockIdx.x >> 1, b = blockIdx.y;
  if (active && !active[b]) return;  // the same for both CTAs of the cluster
  constexpr int ns = has_wda ? 6 : 5, nA = (ns + 1) / 2, nB = ns - nA;
  const int f0 = rank ? nA : 0, nloc = rank ? nB : nA;
  PlaneSmem s = plane_smem_setup<N2C, M3C>(g, nloc);
  const PlaneShape<N2C, M3C> sh(g);
  const size_t poff = ((size_t)b * g.n1 + i1) * sh.n2 * sh.h3;
  load_spec_planes<N2C, M3C>(g, s, nloc, win + (size_t)f0 * fsw, poff, fsw);
  __syncthreads();
  plane_inverse<N2C, M3C>(g, s, nloc);
  cl.sync();  // both halves of the plane in real space
  double2* peer = cl.map_shared_rank(s.slots, rank ^ 1u);
  double* bA = (double*)(rank == 0 ? s.slots : peer);
  double* bB = (double*)(rank == 1 ? s.slots : peer);
  const size_t rowA = (size_t)nA * sh.h3 * 2, rowB = (size_t)nB * sh.h3 * 2;  // doubles per y row
  auto fld = [&](int f, int r, int j) -> double& {
    return f < nA ? bA[r * rowA + (size_t)f * sh.h3 * 2 + j] : bB[r * rowB + (size_t)(f - nA) * sh.h3 * 2 + j];
  };
  double phi = 0.0, n3max = -INFINITY, fwda = 0.0;
  const bool do_c1 = (want & 1) != 0, do_phi = (want & 3) != 0;
  const size_t roff = ((size_t)b * g.n1 + i1) * sh.n2 * sh.n3;
  const int vstride = 2 * blockDim.x;
  for (int i = (int)(rank * blockDim.x + threadIdx.x); i < sh.n2 * sh.n3; i += vstride) {
    const int r = i / sh.n3, j = i - r * sh.n3;
    double& a0 = fld(0, r, j);
    double& a3 = fld(1, r, j);
    double& ax = fld(2, r, j);
    double& ay = fld(3, r, j);
    double& az = fld(4, r, j);
    n3max = fmax(n3max, a3);
    if (want & 8)
      for (int f = 0; f < ns; ++f) wd[f * fsr + roff + i] = fld(f, r, j);
    if (do_phi) {
      PhiOut o = fmt_point<false, double>(a0, a3, ax, ay, az, nullptr, nullptr, R, version);
      phi += o.phi;
      if (do_c1) {
        a0 = o.gs; a3 = o.g3; ax = o.gv[0]; ay = o.gv[1]; az = o.gv[2];
      }
      if (has_wda) {
        double& aw = fld(5, r, j);
        double fv, dfv;
        wda_eos(wda, aw, fv, dfv);
        fwda += fv;
        if (do_c1) aw = dfv;
      }
    }
  }
  // warp partials of the one-CTA pass's virtual warps, gathered on rank 0
  __shared__ double red[3][32];
  for (int o = 16; o > 0; o >>= 1) {
    phi += __shfl_xor_sync(0xffffffffu, phi, o);
    fwda += __shfl_xor_sync(0xffffffffu, fwda, o);
    n3max = fmax(n3max, __shfl_xor_sync(0xffffffffu, n3max, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (l == 0) {
    double* dst = cl.map_shared_rank(&red[0][0], 0u);
    const int vw = (int)rank * nw + w;
    dst[vw] = phi;
    dst[32 + vw] = fwda;
    dst[64 + vw] = n3max;
  }
  cl.sync();  // dPhi of every point and the warp partials in place; no remote access after this
  if (rank == 0 && threadIdx.x < 32) {
    double t0 = (l < 2 * nw) ? red[0][l] : 0.0, t1 = (l < 2 * nw) ? red[1][l] : 0.0;
    double t2 = (l < 2 * nw) ? red[2][l] : -INFINITY;
    for (int o = 16; o > 0; o >>= 1) {
      t0 += __shfl_xor_sync(0xffffffffu, t0, o);
      t1 += __shfl_xor_sync(0xffffffffu, t1, o);
      t2 = fmax(t2, __shfl_xor_sync(0xffffffffu, t2, o));
    }
    if (want & 2) {
      put_part(part, b, CMM_STAT_PHI, nslot_part, i1, t0);
      if (has_wda) put_part(part, b, CMM_STAT_WDA, nslot_part, i1, t1);
    }
    if (want & 4) put_part(part, b, CMM_STAT_N3MAX, nslot_part, i1, t2);
  }
  if (!do_c1) return;
  plane_forward<N2C, M3C>(g, s, nloc);
  store_spec_planes<N2C, M3C>(g, s, nloc, gout + (size_t)f0 * fsg, poff, fsg);
}

template <int N2C, int M3C>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(CMM_FMT2_THREADS, 2)
k_plane_fmt_c2(GridDev g, const int* __restrict__ active, double R, int version, cmm_wda_eos wda,
               const double2* __restrict__ win, size_t fsw, double2* __restrict__ gout, size_t fsg,
               double* __restrict__ part, int nslot_part, int want, double* __restrict__ wd, size_t fsr) {
  plane_fmt_body_c2<N2C, M3C, false>(g, active, R, version, wda, win, fsw, gout, fsg, part, nslot_part, want, wd,
                                     fsr);
}

template <int N2C, int M3C>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(CMM_FMT2_THREADS, 2)
k_plane_fmt_wda_c2(GridDev g, const int* __restrict__ active, double R, int version, cmm_wda_eos wda,
                   const double2* __restrict__ win, size_t fsw, double2* __restrict__ gout, size_t fsg,
                   double* __restrict__ part, int nslot_part, int want, double* __restrict__ wd, size_t fsr) {
  plane_fmt_body_c2<N2C, M3C, true>(g, active, R, version, wda, win, fsw, gout, fsg, part, nslot_part, want, wd,
                                    fsr);
}

// ================================================ staged plane passes ==
// For planes whose fields do not fit in one SM's shared memory (and for the
// tensor variants), the plane pass runs as a y pass over HBM followed by a
// z-row pass with the pointwise step; the y pass of the results follows.

// y transform of one field of one x-plane, a tile of tc stored z frequencies
// at a time: [n2][tc] in shared memory, pencils along y.  Fields f of the
// launch are at src/dst + f * fs; blockIdx.z = b * nfield + f.
template <int N2C>
__global__ void __launch_bounds__(CMM_COL_THREADS, (N2C >= 0 ? 4 : CMM_COL_MINB))
k_ypass(GridDev g, const int* __restrict__ active, const double2* src, double2* dst, size_t fs, int nfield,
        int tc, int inv) {
  const int i1 = blockIdx.y;
  const int b = blockIdx.z / nfield, f = blockIdx.z - b * nfield;
  if (active && !active[b]) return;
  const int n2 = N2C > 0 ? N2C : g.n2, h3 = g.h3;
  extern __shared__ double2 smem_d2[];
  double2* t = smem_d2;       // [n2][tc]
  double2* tw = t + (size_t)n2 * tc;
  double2* tmp = g.ax2.big ? tw + n2 : nullptr;   // direct-DFT stage scratch [n2 * tc]
  for (int i = threadIdx.x; i < n2; i += blockDim.x) tw[i] = g.tw2[i];
  const int c0 = blockIdx.x * tc;
  const size_t base = (size_t)f * fs + ((size_t)b * g.n1 + i1) * n2 * h3;
  for (int i = threadIdx.x; i < n2 * tc; i += blockDim.x) {
    const int r = i / tc, c = i - r * tc;
    const int col = c0 + c;
    t[i] = (col < h3) ? src[base + (size_t)r * h3 + col] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  if (inv) axis_fft<true, N2C>(t, g.ax2, tw, 1, tc, 1, tc, tmp);
  else axis_fft<false, N2C>(t, g.ax2, tw, 1, tc, 1, tc, tmp);
  for (int i = threadIdx.x; i < n2 * tc; i += blockDim.x) {
    const int r = i / tc, c = i - r * tc;
    const int col = c0 + c;
    if (col < h3) dst[base + (size_t)r * h3 + col] = t[i];
  }
}


// z rows in shared memory: nrow rows of rs slots (rs = h3, or n3 for odd N3)
// | z twiddles (n3) | direct-DFT scratch (nrow * z length, when needed) | z
// position table.
__host__ __device__ inline size_t zrow_smem_bytes(int rs, int n3, int zlen, int nz, int big, int nrow) {
  size_t b = sizeof(double2) * ((size_t)nrow * rs + n3 + (big ? (size_t)nrow * zlen : 0)) + sizeof(int) * nz;
  return (b + 15) & ~(size_t)15;
}

static inline size_t zrow_smem_bytes_g(const cmm_grid* g, int nrow) {
  const int full = g->dev.zfull;
  return zrow_smem_bytes(full ? g->n3 : g->h3, g->n3, g->ax3.n, full ? g->n3 : g->m3, g->ax3.big, nrow);
}

template <int M3C>
__device__ inline PlaneSmem zrow_smem_setup(const GridDev& g, int nrow) {
  extern __shared__ double2 smem_d2[];
  const bool full = (M3C <= 0) && g.zfull;
  const int m3 = M3C > 0 ? M3C : g.m3;
  const int rs = full ? g.n3 : m3 + 1, n3 = full ? g.n3 : 2 * m3, nz = full ? g.n3 : m3;
  PlaneSmem s;
  s.slots = smem_d2;
  s.tw2 = nullptr;
  s.tw3 = s.slots + (size_t)nrow * rs;
  s.tmp = g.ax3.big ? s.tw3 + n3 : nullptr;
  s.zpos = (int*)(g.ax3.big ? s.tmp + (size_t)nrow * g.ax3.n : s.tw3 + n3);
  for (int i = threadIdx.x; i < n3; i += blockDim.x) s.tw3[i] = g.tw3[i];
  for (int i = threadIdx.x; i < nz; i += blockDim.x) s.zpos[i] = g.zpos[i];
  __syncthreads();  // zrow_load (odd N3) reads zpos right away
  return s;
}

// Load nr stored-spectrum rows of field f (src: nr * h3 elements) into slot
// rows r * nf + f.  Odd N3: frequency k goes to its DIF position and its
// Hermitian partner n3 - k gets the conjugate; the k = 0 bin keeps its real
// part (Grid.ifft's .real of a self-conjugate bin).
template <int M3C>
__device__ inline void zrow_load(const GridDev& g, const PlaneSmem& s, int nf, int f, int nr,
                                 const double2* __restrict__ src) {
  const bool full = (M3C <= 0) && g.zfull;
  const int h3 = M3C > 0 ? M3C + 1 : g.h3;
  const int rs = full ? g.n3 : h3;
  for (int i = threadIdx.x; i < nr * h3; i += blockDim.x) {
    const int r = i / h3, c = i - r * h3;
    const double2 X = __ldg(src + i);
    double2* row = s.slots + ((size_t)r * nf + f) * rs;
    if (!full) {
      row[c] = X;
    } else if (c == 0) {
      row[s.zpos[0]] = make_double2(X.x, 0.0);
    } else {
      row[s.zpos[c]] = X;
      row[s.zpos[g.n3 - c]] = cconj(X);
    }
  }
}

template <int M3C>
__device__ inline void zrow_store(const GridDev& g, const PlaneSmem& s, int nf, int f, int nr,
                                  double2* __restrict__ dst) {
  const bool full = (M3C <= 0) && g.zfull;
  const int h3 = M3C > 0 ? M3C + 1 : g.h3;
  const int rs = full ? g.n3 : h3;
  for (int i = threadIdx.x; i < nr * h3; i += blockDim.x) {
    const int r = i / h3, c = i - r * h3;
    const double2* row = s.slots + ((size_t)r * nf + f) * rs;
    dst[i] = full ? row[s.zpos[c]] : row[c];
  }
}

// Real element j of slot row r * nf + f (after zrow_inverse).
template <int M3C>
__device__ __forceinline__ double& zrow_rel(const GridDev& g, const PlaneSmem& s, int nf, int f, int r, int j) {
  if constexpr (M3C <= 0) {
    if (g.zfull) return s.slots[((size_t)r * nf + f) * g.n3 + j].x;
  }
  return ((double*)(s.slots + ((size_t)r * nf + f) * (M3C > 0 ? M3C + 1 : g.h3)))[j];
}

template <int M3C>
__device__ void zrow_inverse(const GridDev& g, const PlaneSmem& s, int nrow) {
  if constexpr (M3C <= 0) {
    if (g.zfull) {
      axis_fft<true, M3C>(s.slots, g.ax3, s.tw3, 1, nrow, g.n3, 1, s.tmp);
      return;
    }
  }
  const int h3 = (M3C > 0 ? M3C : g.m3) + 1;
  c2r_twist_rows<M3C>(g, s, nrow);
  axis_fft<true, M3C>(s.slots, g.ax3, s.tw3, 2, nrow, h3, 1, s.tmp);
}

template <int M3C>
__device__ void zrow_forward(const GridDev& g, const PlaneSmem& s, int nrow) {
  if constexpr (M3C <= 0) {
    if (g.zfull) {
      for (int i = threadIdx.x; i < nrow * g.n3; i += blockDim.x) s.slots[i].y = 0.0;
      __syncthreads();
      axis_fft<false, M3C>(s.slots, g.ax3, s.tw3, 1, nrow, g.n3, 1, s.tmp);
      return;
    }
  }
  const int h3 = (M3C > 0 ? M3C : g.m3) + 1;
  axis_fft<false, M3C>(s.slots, g.ax3, s.tw3, 2, nrow, h3, 1, s.tmp);
  r2c_twist_rows<M3C>(g, s, nrow);
}

// z rows of the dPhi/dn step: one block per x-plane, `chunk` y rows of all
// fields at a time (rows interleaved by field as in the plane layout).  The
// input fields (w, y already inverted) are read, the dPhi fields written to
// gout (z forward; their y forward follows).  Same pointwise arithmetic and
// reductions as k_plane_fmt.
template <int M3C, bool WDA, bool TEN>
__global__ void __launch_bounds__(CMM_ZFMT_THREADS)
k_zrow_fmt(GridDev g, const int* __restrict__ active, double R, int version, cmm_wda_eos wda,
           const double2* __restrict__ win, size_t fs, double2* __restrict__ gout, int chunk,
           double* __restrict__ part, int nslot_part, int want, double* __restrict__ wd, size_t fsr) {
  const int i1 = blockIdx.x, b = blockIdx.y;
  if (active && !active[b]) return;
  constexpr int tb = WDA ? 6 : 5;
  constexpr int nf = tb + (TEN ? 6 : 0);
  const int h3 = M3C > 0 ? M3C + 1 : g.h3, n3 = g.n3, n2 = g.n2;
  PlaneSmem s = zrow_smem_setup<M3C>(g, nf * chunk);
  const size_t poff = ((size_t)b * g.n1 + i1) * n2 * h3;
  const bool do_c1 = (want & 1) != 0, do_phi = (want & 3) != 0;
  const size_t roff = ((size_t)b * g.n1 + i1) * n2 * n3;
  double phi = 0.0, n3max = -INFINITY, fwda = 0.0;
  for (int r0 = 0; r0 < n2; r0 += chunk) {
    const int nr = min(chunk, n2 - r0);
    for (int f = 0; f < nf; ++f) zrow_load<M3C>(g, s, nf, f, nr, win + f * fs + poff + (size_t)r0 * h3);
    __syncthreads();
    zrow_inverse<M3C>(g, s, nf * nr);
    for (int i = threadIdx.x; i < nr * n3; i += blockDim.x) {
      const int r = i / n3, j = i - r * n3;
      double& a0 = zrow_rel<M3C>(g, s, nf, 0, r, j);
      double& a3 = zrow_rel<M3C>(g, s, nf, 1, r, j);
      double& ax = zrow_rel<M3C>(g, s, nf, 2, r, j);
      double& ay = zrow_rel<M3C>(g, s, nf, 3, r, j);
      double& az = zrow_rel<M3C>(g, s, nf, 4, r, j);
      n3max = fmax(n3max, a3);
      if (want & 8)
        for (int f = 0; f < nf; ++f) wd[f * fsr + roff + (size_t)(r0 + r) * n3 + j] = zrow_rel<M3C>(g, s, nf, f, r, j);
      if (!do_phi) continue;
      double T[6], gT[6];
      if constexpr (TEN)
        for (int q = 0; q < 6; ++q) T[q] = zrow_rel<M3C>(g, s, nf, tb + q, r, j);
      PhiOut o = fmt_point<TEN, double>(a0, a3, ax, ay, az, T, gT, R, version);
      phi += o.phi;
      if (do_c1) {
        a0 = o.gs; a3 = o.g3; ax = o.gv[0]; ay = o.gv[1]; az = o.gv[2];
        if constexpr (TEN)
          for (int q = 0; q < 6; ++q) zrow_rel<M3C>(g, s, nf, tb + q, r, j) = gT[q];
      }
      if constexpr (WDA) {
        double& aw = zrow_rel<M3C>(g, s, nf, 5, r, j);
        double fv, dfv;
        wda_eos(wda, aw, fv, dfv);
        fwda += fv;
        if (do_c1) aw = dfv;
      }
    }
    __syncthreads();
    if (do_c1) {
      zrow_forward<M3C>(g, s, nf * nr);
      for (int f = 0; f < nf; ++f) zrow_store<M3C>(g, s, nf, f, nr, gout + f * fs + poff + (size_t)r0 * h3);
    }
    __syncthreads();
  }
  __shared__ double red[32];
  if (want & 2) {
    double t = block_sum(phi, red);
    put_part(part, b, CMM_STAT_PHI, nslot_part, i1, t);
    if constexpr (WDA) {
      t = block_sum(fwda, red);
      put_part(part, b, CMM_STAT_WDA, nslot_part, i1, t);
    }
  }
  if (want & 4) {
    double t = block_max(n3max, red);
    put_part(part, b, CMM_STAT_N3MAX, nslot_part, i1, t);
  }
}

// ========================================== plane pass: solver updates ==
struct PlaneStats {
  double n, iue, nonfin, fid, fext;
};

__device__ __forceinline__ void stats_point(PlaneStats& st, double rho, double ref, double V,
                                            double lambda3) {
  st.n += rho;
  st.iue += fabs(rho - ref);
  st.nonfin += cmm_isfinite(rho) ? 0.0 : 1.0;
  const double rr = (rho < 1e-12) ? 1e-30 : rho;  // Solver._clip_density
  st.fid += rr * (log(lambda3 * rr) - 1.0);
  st.fext += rho * V;
}

__device__ inline void stats_store(const PlaneStats& st, double* part, int b, int nslot, int slot) {
  __shared__ double red[32];
  double t;
  t = block_sum(st.n, red);      put_part(part, b, CMM_STAT_N, nslot, slot, t);
  t = block_sum(st.iue, red);    put_part(part, b, CMM_STAT_IUE, nslot, slot, t);
  t = block_sum(st.nonfin, red); put_part(part, b, CMM_STAT_NONFIN, nslot, slot, t);
  t = block_sum(st.fid, red);    put_part(part, b, CMM_STAT_FID, nslot, slot, t);
  t = block_sum(st.fext, red);   put_part(part, b, CMM_STAT_FEXT, nslot, slot, t);
}

// One term of the DER criterion (Solver._check_convergence, cmmdft/solver.py:200-205):
// (|rho| beta dOmega / (a_tol + r_tol |rho|))^2 with dOmega = ln(L^3 rho_reg)/beta + C1 - mu,
// skipped where np.isclose(rho, 0) (|rho| <= 1e-8).
__device__ __forceinline__ double der_term(double rho, double C1, double mu, double beta, double lambda3,
                                           double a_tol, double r_tol) {
  if (fabs(rho) <= 1e-8) return 0.0;
  const double rr = (rho < 1e-12) ? 1e-30 : rho;
  const double dO = log(lambda3 * rr) / beta + C1 - mu;
  const double t = fabs(rho) * beta * dO / (a_tol + r_tol * fabs(rho));
  return t * t;
}

// Static Picard step fused with the C1 inverse and the forward of rho'.
template <int N2C, int M3C>
__global__ void __launch_bounds__(CMM_PLANE_THREADS, CMM_PLANE_MINB_FOR(N2C))
k_plane_picard(GridDev g, const int* __restrict__ active, const double* __restrict__ params,
               double beta, double lambda3, double thr, double a_tol, double r_tol,
               const double2* __restrict__ chat,
               const double* __restrict__ rho, const double* __restrict__ V, long long vstride,
               double* __restrict__ rho_out, double2* __restrict__ rhohat_out,
               double* __restrict__ part, int nslot_part) {
  const int i1 = blockIdx.x, b = blockIdx.y;
  if (active && !active[b]) return;
  PlaneSmem s = plane_smem_setup<N2C, M3C>(g, 1);
  const PlaneShape<N2C, M3C> sh(g);
  const size_t poff = ((size_t)b * g.n1 + i1) * sh.n2 * sh.h3;
  const size_t roff = ((size_t)b * g.n1 + i1) * sh.n2 * sh.n3;
  const double* Vp = V + b * vstride + (size_t)i1 * sh.n2 * sh.n3;
  const size_t pbytes = sizeof(double) * sh.n2 * sh.n3;
  if (threadIdx.x == 0) cmm_prefetch_l2(Vp, pbytes);
  if (threadIdx.x == 32) cmm_prefetch_l2(rho + roff, pbytes);
  load_spec_planes<N2C, M3C>(g, s, 1, chat, poff, 0);
  __syncthreads();
  plane_inverse<N2C, M3C>(g, s, 1);
  const double fug = params[b * 4 + 0], a = params[b * 4 + 1], mu = params[b * 4 + 2];
  PlaneStats st = {0, 0, 0, 0, 0};
  double res2 = 0.0, gnf = 0.0, der = 0.0;
  for (int i = threadIdx.x; i < sh.n2 * sh.n3; i += blockDim.x) {
    const int r = i / sh.n3, j = i - r * sh.n3;
    double& cell = rel(s, sh, 1, 0, r, j);
    const double v = __ldg(Vp + i);
    const double C1 = cell + v;
    const double G = beta * exp(-beta * C1) * fug;
    const double x = __ldg(rho + roff + i);
    res2 += (G - x) * (G - x);
    gnf += cmm_isfinite(G) ? 0.0 : 1.0;
    der += der_term(x, C1, mu, beta, lambda3, a_tol, r_tol);
    double xn = (1.0 - a) * x + a * G;
    if (xn < thr) xn = 0.0;
    rho_out[roff + i] = xn;
    stats_point(st, xn, x, v, lambda3);
    cell = xn;
  }
  {
    __shared__ double red2[32];
    double t = block_sum(res2, red2);
    put_part(part, b, CMM_STAT_RES2, nslot_part, i1, t);
    t = block_sum(gnf, red2);
    put_part(part, b, CMM_STAT_GNONFIN, nslot_part, i1, t);
    t = block_sum(der, red2);
    put_part(part, b, CMM_STAT_DER, nslot_part, i1, t);
  }
  stats_store(st, part, b, nslot_part, i1);
  __syncthreads();
  plane_forward<N2C, M3C>(g, s, 1);
  store_spec_planes<N2C, M3C>(g, s, 1, rhohat_out, poff, 0);
}

struct HistPtrs { const double* p[CMM_MAX_HIST]; };

// Residual r = G(C1) - rho with the Gram row against stored residuals.
template <int N2C, int M3C>
__global__ void __launch_bounds__(CMM_PLANE_THREADS, CMM_PLANE_MINB_FOR(N2C))
k_plane_residual(GridDev g, const int* __restrict__ active, const double* __restrict__ params,
                 double beta, double lambda3, double a_tol, double r_tol, const double2* __restrict__ chat,
                 const double* __restrict__ rho,
                 const double* __restrict__ V, long long vstride, double* __restrict__ r_out,
                 HistPtrs hist, int nhist, long long hstride, double* __restrict__ part,
                 int nslot_part) {
  const int i1 = blockIdx.x, b = blockIdx.y;
  if (active && !active[b]) return;
  PlaneSmem s = plane_smem_setup<N2C, M3C>(g, 1);
  const PlaneShape<N2C, M3C> sh(g);
  const size_t poff = ((size_t)b * g.n1 + i1) * sh.n2 * sh.h3;
  const size_t roff = ((size_t)b * g.n1 + i1) * sh.n2 * sh.n3;
  const size_t hoff = (size_t)b * hstride + (size_t)i1 * sh.n2 * sh.n3;
  const double* Vp = V + b * vstride + (size_t)i1 * sh.n2 * sh.n3;
  {
    const size_t pbytes = sizeof(double) * sh.n2 * sh.n3;
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
      if (w == 0) cmm_prefetch_l2(Vp, pbytes);
      else if (w == 1) cmm_prefetch_l2(rho + roff, pbytes);
#pragma unroll
      for (int h = 0; h < CMM_MAX_HIST; ++h)   // static indices: the pointer table stays in parameter space
        if (w == h + 2 && h < nhist) cmm_prefetch_l2(hist.p[h] + hoff, pbytes);
    }
  }
  load_spec_planes<N2C, M3C>(g, s, 1, chat, poff, 0);
  __syncthreads();
  plane_inverse<N2C, M3C>(g, s, 1);
  const double fug = params[b * 4 + 0], mu = params[b * 4 + 2];
  double res2 = 0.0, gnf = 0.0, der = 0.0;
  double gram[CMM_MAX_HIST];
#pragma unroll
  for (int j = 0; j < CMM_MAX_HIST; ++j) gram[j] = 0.0;
  for (int i = threadIdx.x; i < sh.n2 * sh.n3; i += blockDim.x) {
    const int r = i / sh.n3, j = i - r * sh.n3;
    const double C1 = rel(s, sh, 1, 0, r, j) + __ldg(Vp + i);
    const double G = beta * exp(-beta * C1) * fug;
    const double x = __ldg(rho + roff + i);
    const double rr = G - x;
    res2 += rr * rr;
    gnf += cmm_isfinite(G) ? 0.0 : 1.0;
    der += der_term(x, C1, mu, beta, lambda3, a_tol, r_tol);
    r_out[roff + i] = rr;
#pragma unroll
    for (int h = 0; h < CMM_MAX_HIST; ++h)
      if (h < nhist) gram[h] += rr * __ldg(hist.p[h] + hoff + i);
  }
  __shared__ double red[32];
  double t = block_sum(res2, red);
  put_part(part, b, CMM_STAT_RES2, nslot_part, i1, t);
  t = block_sum(gnf, red);
  put_part(part, b, CMM_STAT_GNONFIN, nslot_part, i1, t);
  t = block_sum(der, red);
  put_part(part, b, CMM_STAT_DER, nslot_part, i1, t);
  for (int h = 0; h < nhist; ++h) {
    t = block_sum(gram[h], red);
    put_part(part, b, CMM_STAT_GRAM0 + h, nslot_part, i1, t);
  }
}

struct FieldPtrs { const double* p[CMM_MAX_FIELDS]; long long stride[CMM_MAX_FIELDS]; };

// rho' = sum_j c_j field_j, clipped, with stats and the forward transform.
template <int N2C, int M3C>
__global__ void __launch_bounds__(CMM_PLANE_THREADS, CMM_PLANE_MINB_FOR(N2C))
k_plane_mix(GridDev g, const int* __restrict__ active, const double* __restrict__ coef,
            FieldPtrs fields, int nfield, int clip, double thr, double lambda3, const double* __restrict__ ref,
            long long refstride, const double* __restrict__ V, long long vstride,
            double* __restrict__ rho_out, double2* __restrict__ rhohat_out,
            double* __restrict__ part, int nslot_part) {
  const int i1 = blockIdx.x, b = blockIdx.y;
  if (active && !active[b]) return;
  PlaneSmem s = plane_smem_setup<N2C, M3C>(g, 1);
  const PlaneShape<N2C, M3C> sh(g);
  const size_t plane = (size_t)i1 * sh.n2 * sh.n3;
  const size_t roff = (size_t)b * g.n1 * sh.n2 * sh.n3 + plane;
  const double* Vp = V + b * vstride + plane;
  const double* Rp = ref + b * refstride + plane;
  double c[CMM_MAX_FIELDS];
#pragma unroll
  for (int j = 0; j < CMM_MAX_FIELDS; ++j) c[j] = (j < nfield) ? coef[b * CMM_MAX_FIELDS + j] : 0.0;
  {
    const size_t pbytes = sizeof(double) * sh.n2 * sh.n3;
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
      if (w == 0) cmm_prefetch_l2(Vp, pbytes);
      else if (w == 1) cmm_prefetch_l2(Rp, pbytes);
#pragma unroll
      for (int f = 0; f < CMM_MAX_FIELDS; ++f)
        if (w == f + 2 && f < nfield && c[f] != 0.0)
          cmm_prefetch_l2(fields.p[f] + b * fields.stride[f] + plane, pbytes);
    }
  }
  PlaneStats st = {0, 0, 0, 0, 0};
  for (int i = threadIdx.x; i < sh.n2 * sh.n3; i += blockDim.x) {
    const int r = i / sh.n3, j = i - r * sh.n3;
    double x = 0.0;
#pragma unroll
    for (int f = 0; f < CMM_MAX_FIELDS; ++f)
      if (f < nfield && c[f] != 0.0) x += c[f] * __ldg(fields.p[f] + b * fields.stride[f] + plane + i);
    if (clip == CMM_CLIP_DENSITY) x = (x < 1e-12) ? 1e-30 : x;
    else if (clip == CMM_CLIP_PICARD && x < thr) x = 0.0;
    rho_out[roff + i] = x;
    stats_point(st, x, __ldg(Rp + i), __ldg(Vp + i), lambda3);
    rel(s, sh, 1, 0, r, j) = x;
  }
  stats_store(st, part, b, nslot_part, i1);
  __syncthreads();
  plane_forward<N2C, M3C>(g, s, 1);
  store_spec_planes<N2C, M3C>(g, s, 1, rhohat_out, ((size_t)b * g.n1 + i1) * sh.n2 * sh.h3, 0);
}

// ===================================== staged single-field plane passes ==
// The solver updates and the plain transforms as z-row passes (after / before
// a y pass over HBM): one block per x-plane, `chunk` y rows at a time.  An op
// supplies the pointwise step (point) and the reductions (finish); kIn loads
// and inverts a spectrum, kOut forwards and stores the rows.  The arithmetic
// per point is that of the fused plane kernels above.
template <int M3C, class Op>
__global__ void __launch_bounds__(CMM_ROW_THREADS)
k_zrow_op(GridDev g, const int* __restrict__ active, Op op, const double2* __restrict__ spec_in,
          double2* __restrict__ spec_out, int chunk, double* __restrict__ part, int nslot_part) {
  const int i1 = blockIdx.x, b = blockIdx.y;
  if (active && !active[b]) return;
  const int h3 = M3C > 0 ? M3C + 1 : g.h3, n3 = g.n3, n2 = g.n2;
  PlaneSmem s = zrow_smem_setup<M3C>(g, chunk);
  const size_t poff = ((size_t)b * g.n1 + i1) * n2 * h3;
  const size_t plane = (size_t)i1 * n2 * n3;
  const size_t inst = (size_t)b * g.n1 * n2 * n3;
  typename Op::Acc acc;
  op.init(acc, b);
  for (int r0 = 0; r0 < n2; r0 += chunk) {
    const int nr = min(chunk, n2 - r0);
    if constexpr (Op::kIn) {
      zrow_load<M3C>(g, s, 1, 0, nr, spec_in + poff + (size_t)r0 * h3);
      __syncthreads();
      zrow_inverse<M3C>(g, s, nr);
    }
    for (int i = threadIdx.x; i < nr * n3; i += blockDim.x) {
      const int r = i / n3, j = i - r * n3;
      const size_t pi = plane + (size_t)(r0 + r) * n3 + j;   // index within the instance
      op.point(acc, b, inst + pi, pi, zrow_rel<M3C>(g, s, 1, 0, r, j));
    }
    __syncthreads();
    if constexpr (Op::kOut) {
      zrow_forward<M3C>(g, s, nr);
      zrow_store<M3C>(g, s, 1, 0, nr, spec_out + poff + (size_t)r0 * h3);
    }
    __syncthreads();
  }
  op.finish(acc, part, b, nslot_part, i1);
}

struct OpR2C {   // real rows -> spectrum (cmm_rfft_yz)
  static constexpr bool kIn = false, kOut = true;
  const double* in;
  struct Acc {};
  __device__ void init(Acc&, int) const {}
  __device__ void point(Acc&, int, size_t gi, size_t, double& cell) const { cell = __ldg(in + gi); }
  __device__ void finish(Acc&, double*, int, int, int) const {}
};

struct OpC2R {   // spectrum -> real rows (cmm_irfft_yz)
  static constexpr bool kIn = true, kOut = false;
  double* out;
  struct Acc {};
  __device__ void init(Acc&, int) const {}
  __device__ void point(Acc&, int, size_t gi, size_t, double& cell) const { out[gi] = cell; }
  __device__ void finish(Acc&, double*, int, int, int) const {}
};

struct OpPicard {   // k_plane_picard
  static constexpr bool kIn = true, kOut = true;
  const double* params;
  double beta, lambda3, thr, a_tol, r_tol;
  const double* rho;
  const double* V;
  long long vstride;
  double* rho_out;
  struct Acc { double fug, a, mu; PlaneStats st; double res2, gnf, der; };
  __device__ void init(Acc& c, int b) const {
    c.fug = params[b * 4 + 0]; c.a = params[b * 4 + 1]; c.mu = params[b * 4 + 2];
    c.st = {0, 0, 0, 0, 0}; c.res2 = c.gnf = c.der = 0.0;
  }
  __device__ void point(Acc& c, int b, size_t gi, size_t pi, double& cell) const {
    const double v = __ldg(V + b * vstride + pi);
    const double C1 = cell + v;
    const double G = beta * exp(-beta * C1) * c.fug;
    const double x = __ldg(rho + gi);
    c.res2 += (G - x) * (G - x);
    c.gnf += cmm_isfinite(G) ? 0.0 : 1.0;
    c.der += der_term(x, C1, c.mu, beta, lambda3, a_tol, r_tol);
    double xn = (1.0 - c.a) * x + c.a * G;
    if (xn < thr) xn = 0.0;
    rho_out[gi] = xn;
    stats_point(c.st, xn, x, v, lambda3);
    cell = xn;
  }
  __device__ void finish(Acc& c, double* part, int b, int nslot, int slot) const {
    __shared__ double red2[32];
    double t = block_sum(c.res2, red2);
    put_part(part, b, CMM_STAT_RES2, nslot, slot, t);
    t = block_sum(c.gnf, red2);
    put_part(part, b, CMM_STAT_GNONFIN, nslot, slot, t);
    t = block_sum(c.der, red2);
    put_part(part, b, CMM_STAT_DER, nslot, slot, t);
    stats_store(c.st, part, b, nslot, slot);
  }
};

struct OpResidual {   // k_plane_residual
  static constexpr bool kIn = true, kOut = false;
  const double* params;
  double beta, lambda3, a_tol, r_tol;
  const double* rho;
  const double* V;
  long long vstride;
  double* r_out;
  HistPtrs hist;
  int nhist;
  long long hstride;
  struct Acc { double fug, mu, res2, gnf, der, gram[CMM_MAX_HIST]; };
  __device__ void init(Acc& c, int b) const {
    c.fug = params[b * 4 + 0]; c.mu = params[b * 4 + 2];
    c.res2 = c.gnf = c.der = 0.0;
#pragma unroll
    for (int h = 0; h < CMM_MAX_HIST; ++h) c.gram[h] = 0.0;
  }
  __device__ void point(Acc& c, int b, size_t gi, size_t pi, double& cell) const {
    const double C1 = cell + __ldg(V + b * vstride + pi);
    const double G = beta * exp(-beta * C1) * c.fug;
    const double x = __ldg(rho + gi);
    const double rr = G - x;
    c.res2 += rr * rr;
    c.gnf += cmm_isfinite(G) ? 0.0 : 1.0;
    c.der += der_term(x, C1, c.mu, beta, lambda3, a_tol, r_tol);
    r_out[gi] = rr;
#pragma unroll
    for (int h = 0; h < CMM_MAX_HIST; ++h)
      if (h < nhist) c.gram[h] += rr * __ldg(hist.p[h] + b * hstride + pi);
  }
  __device__ void finish(Acc& c, double* part, int b, int nslot, int slot) const {
    __shared__ double red[32];
    double t = block_sum(c.res2, red);
    put_part(part, b, CMM_STAT_RES2, nslot, slot, t);
    t = block_sum(c.gnf, red);
    put_part(part, b, CMM_STAT_GNONFIN, nslot, slot, t);
    t = block_sum(c.der, red);
    put_part(part, b, CMM_STAT_DER, nslot, slot, t);
    for (int h = 0; h < nhist; ++h) {
      t = block_sum(c.gram[h], red);
      put_part(part, b, CMM_STAT_GRAM0 + h, nslot, slot, t);
    }
  }
};

struct OpMix {   // k_plane_mix
  static constexpr bool kIn = false, kOut = true;
  const double* coef;
  FieldPtrs fields;
  int nfield, clip;
  double thr, lambda3;
  const double* ref;
  long long refstride;
  const double* V;
  long long vstride;
  double* rho_out;
  struct Acc { double c[CMM_MAX_FIELDS]; PlaneStats st; };
  __device__ void init(Acc& a, int b) const {
#pragma unroll
    for (int j = 0; j < CMM_MAX_FIELDS; ++j) a.c[j] = (j < nfield) ? coef[b * CMM_MAX_FIELDS + j] : 0.0;
    a.st = {0, 0, 0, 0, 0};
  }
  __device__ void point(Acc& a, int b, size_t gi, size_t pi, double& cell) const {
    double x = 0.0;
#pragma unroll
    for (int f = 0; f < CMM_MAX_FIELDS; ++f)
      if (f < nfield && a.c[f] != 0.0) x += a.c[f] * __ldg(fields.p[f] + b * fields.stride[f] + pi);
    if (clip == CMM_CLIP_DENSITY) x = (x < 1e-12) ? 1e-30 : x;
    else if (clip == CMM_CLIP_PICARD && x < thr) x = 0.0;
    rho_out[gi] = x;
    stats_point(a.st, x, __ldg(ref + b * refstride + pi), __ldg(V + b * vstride + pi), lambda3);
    cell = x;
  }
  __device__ void finish(Acc& a, double* part, int b, int nslot, int slot) const {
    stats_store(a.st, part, b, nslot, slot);
  }
};

// ================================================= hybrid line search ==
// max over each plane of n3(rho) + n3(r) (field 1 of the stored weighted densities).
__global__ void __launch_bounds__(256)
k_ls_n3max(GridDev g, const int* __restrict__ active, const double* __restrict__ wd_rho,
           const double* __restrict__ wd_r, size_t fsr, double* __restrict__ ls_part, int nslot) {
  const int i1 = blockIdx.x, b = blockIdx.y;
  if (active && !active[b]) return;
  const size_t plane = (size_t)g.n2 * g.n3;
  const size_t off = fsr + ((size_t)b * g.n1 + i1) * plane;
  double m = -INFINITY;
  for (size_t i = threadIdx.x; i < plane; i += blockDim.x) m = fmax(m, __ldg(wd_rho + off + i) + __ldg(wd_r + off + i));
  __shared__ double red[32];
  m = block_max(m, red);
  if (threadIdx.x == 0) ls_part[((size_t)b * CMM_NLS + CMM_LS_N3MAX_G) * nslot + i1] = m;
}

// Omega ingredients of rho + alpha_i r for three alphas, one plane per block.
// FP64-issue bound: three 256-thread blocks per SM (85 registers a thread)
// keep 24 warps in flight.
#define CMM_LS_THREADS 256
template <bool WDA, bool TEN>
__global__ void __launch_bounds__(CMM_LS_THREADS, 3)
k_ls_omega(GridDev g, const int* __restrict__ active, const double* __restrict__ n3a, long long n3a_stride, double c0, double c1,
           double c2, double R, double lambda3, int version, cmm_wda_eos wda, const double* __restrict__ rho,
           const double* __restrict__ r, const double* __restrict__ V, long long vstride,
           const double* __restrict__ wd_rho, const double* __restrict__ wd_r, size_t fsr,
           double* __restrict__ ls_part, int nslot, double* __restrict__ alpha_out) {
  const int i1 = blockIdx.x, b = blockIdx.y;
  if (active && !active[b]) return;
  constexpr int tb = WDA ? 6 : 5;
  constexpr int nf = tb + (TEN ? 6 : 0);
  __shared__ double s_alpha[3];
  if (threadIdx.x < 32) {  // alpha_max of this instance (every block reduces the same partials)
    const double* pm = ls_part + ((size_t)b * CMM_NLS + CMM_LS_N3MAX_G) * nslot;
    double gmax = -INFINITY;
    for (int k = threadIdx.x; k < nslot; k += 32) gmax = fmax(gmax, pm[k]);
    for (int o = 16; o > 0; o >>= 1) gmax = fmax(gmax, __shfl_xor_sync(0xffffffffu, gmax, o));
    if (threadIdx.x == 0) {
      const double a = n3a[(size_t)b * n3a_stride];
      const double q = fabs((1 - a) / ((gmax - a) + 1e-16));
      const double amax = (q != q) ? q : fmin(q, 1.0);   // np.min([q, 1]) (propagates NaN)
      s_alpha[0] = c0 * amax; s_alpha[1] = c1 * amax; s_alpha[2] = c2 * amax;
      if (i1 == 0) alpha_out[b] = amax;
    }
  }
  __syncthreads();
  const double al[3] = {s_alpha[0], s_alpha[1], s_alpha[2]};
  const size_t plane = (size_t)g.n2 * g.n3;
  const size_t pbase = (size_t)i1 * plane;
  const size_t gbase = (size_t)b * g.n1 * plane + pbase;
  double sr = 0.0, srv = 0.0, fid[3] = {0, 0, 0}, phi[3] = {0, 0, 0}, fw[3] = {0, 0, 0};
  for (size_t i = threadIdx.x; i < plane; i += blockDim.x) {
    const size_t gi = gbase + i;
    const double x0 = __ldg(rho + gi), rr = __ldg(r + gi), v = __ldg(V + b * vstride + pbase + i);
    sr += rr;
    srv += rr * v;
    // one alpha at a time (the weighted densities are re-read from L1/L2):
    // fewer live registers, two blocks per SM without spills
#pragma unroll 1
    for (int k = 0; k < 3; ++k) {
      const double a = (k == 0) ? al[0] : (k == 1 ? al[1] : al[2]);
      double x = x0 + a * rr;
      x = (x < 1e-12) ? 1e-30 : x;  // Solver._clip_density
      const double fk = x * (log(lambda3 * x) - 1.0);
      double n[nf];
#pragma unroll
      for (int f = 0; f < nf; ++f) n[f] = __ldg(wd_rho + f * fsr + gi) + a * __ldg(wd_r + f * fsr + gi);
      const double pk = fmt_phi<TEN>(n[0], n[1], n[2], n[3], n[4], TEN ? n + tb : nullptr, R, version);
      double wk = 0.0;
      if constexpr (WDA) {
        double dfv;
        wda_eos(wda, n[5], wk, dfv);
      }
      if (k == 0) { fid[0] += fk; phi[0] += pk; fw[0] += wk; }
      else if (k == 1) { fid[1] += fk; phi[1] += pk; fw[1] += wk; }
      else { fid[2] += fk; phi[2] += pk; fw[2] += wk; }
    }
  }
  __shared__ double red[32];
  double* out = ls_part + (size_t)b * CMM_NLS * nslot + i1;
  double t = block_sum(sr, red);
  if (threadIdx.x == 0) out[CMM_LS_SUM_R * nslot] = t;
  t = block_sum(srv, red);
  if (threadIdx.x == 0) out[CMM_LS_SUM_RV * nslot] = t;
  for (int k = 0; k < 3; ++k) {
    t = block_sum(fid[k], red);
    if (threadIdx.x == 0) out[(CMM_LS_FID + k) * nslot] = t;
    t = block_sum(phi[k], red);
    if (threadIdx.x == 0) out[(CMM_LS_PHI + k) * nslot] = t;
    if constexpr (WDA) {
      t = block_sum(fw[k], red);
      if (threadIdx.x == 0) out[(CMM_LS_WDA + k) * nslot] = t;
    }
  }
}

__global__ void k_ls_finalize(const int* __restrict__ active, const double* __restrict__ part, int nslot,
                              double* __restrict__ ls) {
  const int b = blockIdx.x, q = threadIdx.y;
  if (q >= CMM_NLS) return;
  if (active && !active[b]) return;
  const double* p = part + ((size_t)b * CMM_NLS + q) * nslot;
  const bool mx = (q == CMM_LS_N3MAX_G);
  double acc = mx ? -INFINITY : 0.0;
  for (int i = threadIdx.x; i < nslot; i += 32) acc = mx ? fmax(acc, p[i]) : acc + p[i];
  for (int o = 16; o > 0; o >>= 1) {
    double v = __shfl_xor_sync(0xffffffffu, acc, o);
    acc = mx ? fmax(acc, v) : acc + v;
  }
  if (threadIdx.x == 0) ls[(size_t)b * CMM_NLS + q] = acc;
}

// ============================================================ finalize ==
__global__ void k_stats_finalize(const int* __restrict__ active, const double* __restrict__ part,
                                 int nslot, unsigned mask, double* __restrict__ stats) {
  const int b = blockIdx.x, q = threadIdx.y;
  if (q >= NQ || !((mask >> q) & 1u)) return;
  if (active && !active[b]) return;
  const double* p = part + ((size_t)b * NQ + q) * nslot;
  const bool mx = (q == CMM_STAT_N3MAX);
  double acc = mx ? -INFINITY : 0.0;
  for (int i = threadIdx.x; i < nslot; i += 32) acc = mx ? fmax(acc, p[i]) : acc + p[i];
  for (int o = 16; o > 0; o >>= 1) {
    double v = __shfl_xor_sync(0xffffffffu, acc, o);
    acc = mx ? fmax(acc, v) : acc + v;
  }
  if (threadIdx.x == 0) stats[(size_t)b * NQ + q] = acc;
}

// ============================================================ host side ==
static int last_err() { return (cudaPeekAtLastError() == cudaSuccess) ? CMM_OK : CMM_ERR_CUDA; }

// The dynamic shared-memory limit is an attribute of the kernel function,
// shared by every caller: solves of different grids on concurrent host
// threads launch the same generic kernel with different sizes.  The limit
// therefore only grows (under a lock, per device and kernel), so no thread
// lowers it below a launch another thread is about to make.
static int set_smem(const void* fn, size_t bytes) {
  if (bytes > 232448) return CMM_ERR_SMEM;  // the B200 per-block opt-in limit
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> limits;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return CMM_ERR_CUDA;
  std::lock_guard<std::mutex> lock(mu);
  size_t& cur = limits[std::make_pair(dev, fn)];
  if (bytes <= cur) return CMM_OK;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
    return CMM_ERR_CUDA;
  cur = bytes;
  return CMM_OK;
}

// Shape specialisations compiled with compile-time transform lengths; the
// run-time-length kernels come in two instantiations, 0 (radices 2, 3, 4, 5,
// 8 and direct-DFT stages) and -1 (also 7, 11, 13 and Rader stages).
static int plane_kind(const cmm_grid* g) {
  if (!g->generic && g->n2 == 64 && g->m3 == 32) return 1;
  if (!g->generic && g->n2 == 32 && g->m3 == 16) return 2;
  return g->exotic ? -1 : 0;
}
static int col_kind(const cmm_grid* g) {
  if (!g->generic && g->n1 == 64) return 1;
  if (!g->generic && g->n1 == 32) return 2;
  return g->exotic ? -1 : 0;
}

#define LAUNCH_PLANE(kind, kern, grd, smem, st, ...)                                      \
  do {                                                                                   \
    int rc_;                                                                             \
    if ((kind) == 1) {                                                                   \
      if ((rc_ = set_smem((const void*)kern<64, 32>, smem))) return rc_;                \
      kern<64, 32><<<grd, CMM_PLANE_THREADS, smem, st>>>(__VA_ARGS__);                   \
    } else if ((kind) == 2) {                                                            \
      if ((rc_ = set_smem((const void*)kern<32, 16>, smem))) return rc_;                \
      kern<32, 16><<<grd, CMM_PLANE_THREADS, smem, st>>>(__VA_ARGS__);                   \
    } else if ((kind) == -1) {                                                           \
      if ((rc_ = set_smem((const void*)kern<-1, -1>, smem))) return rc_;                \
      kern<-1, -1><<<grd, CMM_PLANE_THREADS, smem, st>>>(__VA_ARGS__);                 \
    } else {                                                                             \
      if ((rc_ = set_smem((const void*)kern<0, 0>, smem))) return rc_;                  \
      kern<0, 0><<<grd, CMM_PLANE_THREADS, smem, st>>>(__VA_ARGS__);                     \
    }                                                                                    \
  } while (0)

#define LAUNCH_PLANE_T(kind, kern, grd, nthr, smem, st, ...)                              \
  do {                                                                                   \
    int rc_;                                                                             \
    if ((kind) == 1) {                                                                   \
      if ((rc_ = set_smem((const void*)kern<64, 32>, smem))) return rc_;                \
      kern<64, 32><<<grd, nthr, smem, st>>>(__VA_ARGS__);                                \
    } else if ((kind) == 2) {                                                            \
      if ((rc_ = set_smem((const void*)kern<32, 16>, smem))) return rc_;                \
      kern<32, 16><<<grd, nthr, smem, st>>>(__VA_ARGS__);                                \
    } else if ((kind) == -1) {                                                           \
      if ((rc_ = set_smem((const void*)kern<-1, -1>, smem))) return rc_;                \
      kern<-1, -1><<<grd, nthr, smem, st>>>(__VA_ARGS__);                              \
    } else {                                                                             \
      if ((rc_ = set_smem((const void*)kern<0, 0>, smem))) return rc_;                  \
      kern<0, 0><<<grd, nthr, smem, st>>>(__VA_ARGS__);                                  \
    }                                                                                    \
  } while (0)

#define LAUNCH_COL(kind, kern, grd, smem, st, ...)                                        \
  do {                                                                                   \
    int rc_;                                                                             \
    if ((kind) == 1) {                                                                   \
      if ((rc_ = set_smem((const void*)kern<64, 8>, smem))) return rc_;                \
      kern<64, 8><<<grd, CMM_COL_THREADS, smem, st>>>(__VA_ARGS__);                     \
    } else if ((kind) == 2) {                                                            \
      if ((rc_ = set_smem((const void*)kern<32, 8>, smem))) return rc_;                \
      kern<32, 8><<<grd, CMM_COL_THREADS, smem, st>>>(__VA_ARGS__);                     \
    } else if ((kind) == -1) {                                                           \
      if ((rc_ = set_smem((const void*)kern<-1, 0>, smem))) return rc_;                 \
      kern<-1, 0><<<grd, CMM_COL_THREADS, smem, st>>>(__VA_ARGS__);                      \
    } else {                                                                             \
      if ((rc_ = set_smem((const void*)kern<0, 0>, smem))) return rc_;                  \
      kern<0, 0><<<grd, CMM_COL_THREADS, smem, st>>>(__VA_ARGS__);                       \
    }                                                                                    \
  } while (0)

// Column tile width: 8 columns (128 B rows) for the specialised kernels, up to
// 16 when it fits otherwise.
static int col_tile(const cmm_grid* g, int nslot) {
  if (col_kind(g) > 0) return 8;
  int tc = g->col_tile > 0 ? g->col_tile : 16;   // the plan's schedule may fix it
  while (tc > 1 && col_smem_bytes(g->n1, tc, nslot, g->ax1.big) > 200 * 1024) tc /= 2;
  return tc;
}

// ---------------------------------------------------- staged plane path --
#define CMM_SMEM_MAX 232448

// y pass over nfield fields (in place when src == dst): tiles of at most 16
// stored z frequencies, spread evenly over the h3 columns.
static int ypass(const cmm_grid* g, int batch, const int* act, const double2* src, double2* dst, size_t fs,
                 int nfield, int inv, cudaStream_t st) {
  const int ntile = cmm_div_up(g->h3, 16);
  const int tc = cmm_div_up(g->h3, ntile);
  if ((long long)batch * nfield > 65535 || g->n1 > 65535) return CMM_ERR_SHAPE;
  const size_t sb = sizeof(double2) * ((size_t)g->n2 * tc * (g->ax2.big ? 2 : 1) + g->n2);
  const dim3 grd(ntile, g->n1, batch * nfield);
  int rc;
  if (!g->generic && g->n2 == 64) {
    if ((rc = set_smem((const void*)k_ypass<64>, sb))) return rc;
    k_ypass<64><<<grd, CMM_COL_THREADS, sb, st>>>(g->dev, act, src, dst, fs, nfield, tc, inv);
  } else if (!g->generic && g->n2 == 32) {
    if ((rc = set_smem((const void*)k_ypass<32>, sb))) return rc;
    k_ypass<32><<<grd, CMM_COL_THREADS, sb, st>>>(g->dev, act, src, dst, fs, nfield, tc, inv);
  } else if (g->exotic) {
    if ((rc = set_smem((const void*)k_ypass<-1>, sb))) return rc;
    k_ypass<-1><<<grd, CMM_COL_THREADS, sb, st>>>(g->dev, act, src, dst, fs, nfield, tc, inv);
  } else {
    if ((rc = set_smem((const void*)k_ypass<0>, sb))) return rc;
    k_ypass<0><<<grd, CMM_COL_THREADS, sb, st>>>(g->dev, act, src, dst, fs, nfield, tc, inv);
  }
  return last_err();
}

// Staged plane passes when the plane of nf fields does not fit in shared
// memory, the y or z transform has a prime factor > 16 (direct-DFT stages
// need scratch), N3 is odd (full-length z transform) or staging is forced.
static bool plane_staged(const cmm_grid* g, int nf) {
  return g->staging == 1 || g->dev.zfull || g->ax2.big || g->ax3.big ||
         plane_smem_bytes(g->n2, g->n3, nf) > CMM_SMEM_MAX;
}

// Compile-time z half length of the z-row kernels (0: from the plan).
static int zrow_m3(const cmm_grid* g) {
  if (!g->generic && !g->dev.zfull && g->m3 == 32) return 32;
  if (!g->generic && !g->dev.zfull && g->m3 == 16) return 16;
  return g->exotic ? -1 : 0;
}

// y rows per z-row chunk so that nf fields fit in the shared-memory budget (0: none fit).
static int zrow_chunk(const cmm_grid* g, int nf) {
  const size_t fixed = zrow_smem_bytes_g(g, 0) + 16;
  const size_t per = zrow_smem_bytes_g(g, nf) - zrow_smem_bytes_g(g, 0) + 16;
  if (fixed + per > CMM_SMEM_MAX) return 0;
  size_t c = (CMM_SMEM_MAX - fixed) / per;
  return (int)(c > (size_t)g->n2 ? g->n2 : c);
}

template <int M3C, class Op>
static int zrow_op_m3(const cmm_grid* g, int batch, const int* act, const Op& op, const double2* in,
                      double2* out, int chunk, double* part, int nslot, cudaStream_t st) {
  const size_t sb = zrow_smem_bytes_g(g, chunk);
  int rc;
  if ((rc = set_smem((const void*)k_zrow_op<M3C, Op>, sb))) return rc;
  k_zrow_op<M3C, Op><<<dim3(g->n1, batch), CMM_ROW_THREADS, sb, st>>>(g->dev, act, op, in, out, chunk, part, nslot);
  return last_err();
}

// One single-field z-row pass (in: y-inverted spectrum rows; out: z-forward rows).
template <class Op>
static int zrow_op(const cmm_grid* g, int batch, const int* act, const Op& op, const double2* in, double2* out,
                   double* part, int nslot, cudaStream_t st) {
  const int chunk = zrow_chunk(g, 1);
  if (chunk < 1) return CMM_ERR_SMEM;
  switch (zrow_m3(g)) {
    case 32: return zrow_op_m3<32>(g, batch, act, op, in, out, chunk, part, nslot, st);
    case 16: return zrow_op_m3<16>(g, batch, act, op, in, out, chunk, part, nslot, st);
    case -1: return zrow_op_m3<-1>(g, batch, act, op, in, out, chunk, part, nslot, st);
    default: return zrow_op_m3<0>(g, batch, act, op, in, out, chunk, part, nslot, st);
  }
}

template <int M3C, bool WDA, bool TEN>
static int zrow_fmt_one(const cmm_grid* g, int batch, const int* act, double R, int version,
                        const cmm_wda_eos& we, const double2* win, size_t fs, double2* gout, int chunk,
                        double* part, int nslot, int want, double* wd, cudaStream_t st) {
  constexpr int nf = (WDA ? 6 : 5) + (TEN ? 6 : 0);
  const size_t sb = zrow_smem_bytes_g(g, nf * chunk);
  int rc;
  if ((rc = set_smem((const void*)k_zrow_fmt<M3C, WDA, TEN>, sb))) return rc;
  k_zrow_fmt<M3C, WDA, TEN><<<dim3(g->n1, batch), CMM_ZFMT_THREADS, sb, st>>>(
      g->dev, act, R, version, we, win, fs, gout, chunk, part, nslot, want, wd,
      (size_t)batch * g->n1 * g->n2 * g->n3);
  return last_err();
}

template <int M3C>
static int zrow_fmt_m3(const cmm_grid* g, int batch, const int* act, double R, int version, const cmm_wda_eos& we,
                       const double2* win, size_t fs, double2* gout, int chunk, double* part, int nslot, int want,
                       double* wd, cudaStream_t st) {
  const bool wda = (version & CMM_WDA) != 0, ten = (version & CMM_TENSOR) != 0;
  if (wda && ten)
    return zrow_fmt_one<M3C, true, true>(g, batch, act, R, version, we, win, fs, gout, chunk, part, nslot, want, wd, st);
  if (wda)
    return zrow_fmt_one<M3C, true, false>(g, batch, act, R, version, we, win, fs, gout, chunk, part, nslot, want, wd, st);
  if (ten)
    return zrow_fmt_one<M3C, false, true>(g, batch, act, R, version, we, win, fs, gout, chunk, part, nslot, want, wd, st);
  return zrow_fmt_one<M3C, false, false>(g, batch, act, R, version, we, win, fs, gout, chunk, part, nslot, want, wd, st);
}

static int zrow_fmt(const cmm_grid* g, int batch, const int* act, double R, int version, const cmm_wda_eos& we,
                    const double2* win, size_t fs, double2* gout, int nf, double* part, int nslot, int want,
                    double* wd, cudaStream_t st) {
  const int chunk = zrow_chunk(g, nf);
  if (chunk < 1) return CMM_ERR_SMEM;
  switch (zrow_m3(g)) {
    case 32: return zrow_fmt_m3<32>(g, batch, act, R, version, we, win, fs, gout, chunk, part, nslot, want, wd, st);
    case 16: return zrow_fmt_m3<16>(g, batch, act, R, version, we, win, fs, gout, chunk, part, nslot, want, wd, st);
    case -1: return zrow_fmt_m3<-1>(g, batch, act, R, version, we, win, fs, gout, chunk, part, nslot, want, wd, st);
    default: return zrow_fmt_m3<0>(g, batch, act, R, version, we, win, fs, gout, chunk, part, nslot, want, wd, st);
  }
}

// ============================================ Hessian-vector product ==
// z rows of the second-derivative step: the weighted densities of v (y
// already inverted) arrive in the slots, those of rho are read from wdrho
// (stored by the functional pass, want bit 3); the pointwise step is the
// directional derivative of dPhi/dn at n(rho) along n(v), fmt_point
// evaluated in Dual arithmetic.  Its fields go out z-forward (y forward
// follows), in the layout of the dPhi spectra of k_zrow_fmt.
// TR: the transposed pointwise Jacobian.  It equals the Jacobian except
// where n3 is clipped (n3 < 1e-30 or > 0.99): there dPhi/dn3 is still taken
// at the clipped value, so it depends on the other densities while nothing
// depends on n3; the transpose passes the tangent of n3 through the clip
// into the other outputs and returns no dPhi/dn3 tangent.
// WDA: the weighted density of the WDA part follows the five FMT densities
// (before the tensor ones); its output is f''_EOS(wd) times the tangent.
template <int M3C, bool TEN, bool TR, bool WDA>
__global__ void __launch_bounds__(CMM_ROW_THREADS)
k_zrow_hvp(GridDev g, const int* __restrict__ active, double R, int version, cmm_wda_eos wda,
           const double2* __restrict__ win, size_t fs, double2* __restrict__ gout, int chunk,
           const double* __restrict__ wdrho, size_t fsr) {
  const int i1 = blockIdx.x, b = blockIdx.y;
  if (active && !active[b]) return;
  constexpr int tb = WDA ? 6 : 5;
  constexpr int nf = tb + (TEN ? 6 : 0);
  const int h3 = M3C > 0 ? M3C + 1 : g.h3, n3 = g.n3, n2 = g.n2;
  PlaneSmem s = zrow_smem_setup<M3C>(g, nf * chunk);
  const size_t poff = ((size_t)b * g.n1 + i1) * n2 * h3;
  const size_t roff = ((size_t)b * g.n1 + i1) * n2 * n3;
  for (int r0 = 0; r0 < n2; r0 += chunk) {
    const int nr = min(chunk, n2 - r0);
    for (int f = 0; f < nf; ++f) zrow_load<M3C>(g, s, nf, f, nr, win + f * fs + poff + (size_t)r0 * h3);
    __syncthreads();
    zrow_inverse<M3C>(g, s, nf * nr);
    for (int i = threadIdx.x; i < nr * n3; i += blockDim.x) {
      const int r = i / n3, j = i - r * n3;
      const size_t q = roff + (size_t)(r0 + r) * n3 + j;
      Dual n[nf], gT[6];
      for (int f = 0; f < nf; ++f) n[f] = Dual(__ldg(wdrho + f * fsr + q), zrow_rel<M3C>(g, s, nf, f, r, j));
      bool clipped = false;
      if constexpr (TR) {
        clipped = !(n[1].v >= 1e-30) || !(n[1].v <= 0.99);
        if (clipped) n[1].v = fmin(fmax(n[1].v, 1e-30), 0.99);
      }
      const PhiOutT<Dual> o = fmt_point<TEN, Dual>(n[0], n[1], n[2], n[3], n[4], TEN ? n + tb : nullptr, gT, R,
                                                   version);
      zrow_rel<M3C>(g, s, nf, 0, r, j) = o.gs.d;
      zrow_rel<M3C>(g, s, nf, 1, r, j) = clipped ? 0.0 : o.g3.d;
      zrow_rel<M3C>(g, s, nf, 2, r, j) = o.gv[0].d;
      zrow_rel<M3C>(g, s, nf, 3, r, j) = o.gv[1].d;
      zrow_rel<M3C>(g, s, nf, 4, r, j) = o.gv[2].d;
      if constexpr (WDA) {
        Dual fv, dfv;
        wda_eos<Dual>(wda, n[5], fv, dfv);
        zrow_rel<M3C>(g, s, nf, 5, r, j) = dfv.d;
      }
      if constexpr (TEN)
        for (int t = 0; t < 6; ++t) zrow_rel<M3C>(g, s, nf, tb + t, r, j) = gT[t].d;
    }
    __syncthreads();
    zrow_forward<M3C>(g, s, nf * nr);
    for (int f = 0; f < nf; ++f) zrow_store<M3C>(g, s, nf, f, nr, gout + f * fs + poff + (size_t)r0 * h3);
    __syncthreads();
  }
}

template <int M3C, bool TEN, bool TR, bool WDA>
static int zrow_hvp_one(const cmm_grid* g, int batch, const int* act, double R, int version,
                        const cmm_wda_eos& wda, const double2* win, size_t fs, double2* gout, int chunk,
                        const double* wdrho, cudaStream_t st) {
  constexpr int nf = (WDA ? 6 : 5) + (TEN ? 6 : 0);
  const size_t sb = zrow_smem_bytes_g(g, nf * chunk);
  int rc;
  if ((rc = set_smem((const void*)k_zrow_hvp<M3C, TEN, TR, WDA>, sb))) return rc;
  k_zrow_hvp<M3C, TEN, TR, WDA><<<dim3(g->n1, batch), CMM_ROW_THREADS, sb, st>>>(
      g->dev, act, R, version, wda, win, fs, gout, chunk, wdrho, (size_t)batch * g->n1 * g->n2 * g->n3);
  return last_err();
}

template <int M3C, bool WDA>
static int zrow_hvp_w(const cmm_grid* g, int batch, const int* act, double R, int version, const cmm_wda_eos& wda,
                      int tr, const double2* win, size_t fs, double2* gout, int chunk, const double* wdrho,
                      cudaStream_t st) {
  if (version & CMM_TENSOR)
    return tr ? zrow_hvp_one<M3C, true, true, WDA>(g, batch, act, R, version, wda, win, fs, gout, chunk, wdrho, st)
              : zrow_hvp_one<M3C, true, false, WDA>(g, batch, act, R, version, wda, win, fs, gout, chunk, wdrho, st);
  return tr ? zrow_hvp_one<M3C, false, true, WDA>(g, batch, act, R, version, wda, win, fs, gout, chunk, wdrho, st)
            : zrow_hvp_one<M3C, false, false, WDA>(g, batch, act, R, version, wda, win, fs, gout, chunk, wdrho, st);
}

template <int M3C>
static int zrow_hvp_m3(const cmm_grid* g, int batch, const int* act, double R, int version,
                       const cmm_wda_eos& wda, int tr, const double2* win, size_t fs, double2* gout, int chunk,
                       const double* wdrho, cudaStream_t st) {
  if (version & CMM_WDA)
    return zrow_hvp_w<M3C, true>(g, batch, act, R, version, wda, tr, win, fs, gout, chunk, wdrho, st);
  return zrow_hvp_w<M3C, false>(g, batch, act, R, version, wda, tr, win, fs, gout, chunk, wdrho, st);
}

// Spectrum of A v = d C1 / d rho . v (Hartree per density unit), A the
// Hessian of the excess free energy per grid volume: hard-sphere part
// through the second derivatives of Phi at the stored weighted densities of
// rho, plus the MFA convolution K v (the external potential does not depend
// on rho).  transpose: A^T v (the caller passes the conjugate MFA spectrum).
// The y/z steps run in the staged form for every grid shape.
extern "C" int cmm_fmt_hvp(const cmm_grid* g, int batch, const int* d_active, double R, double beta, int version,
                           const cmm_wda_eos* wda, int transpose, const double* d_kst, const double* d_wtab,
                           const double* d_wd_rho, const double* d_vhat, double* d_out_hat, double* d_work,
                           void* stream) {
  if (!g || batch < 1 || !d_kst || !d_vhat || !d_out_hat || !d_work) return CMM_ERR_ARG;
  const bool has_wda = (version & CMM_WDA) != 0 && !(version & CMM_NOHS);
  if (has_wda && !wda) return CMM_ERR_ARG;
  cmm_wda_eos we;
  memset(&we, 0, sizeof(we));
  if (has_wda) we = *wda;
  const bool ten = (version & CMM_TENSOR) != 0;
  const int nf = (has_wda ? 6 : 5) + (ten ? 6 : 0);
  cudaStream_t st = (cudaStream_t)stream;
  const size_t fs = (size_t)batch * g->n1 * g->n2 * g->h3;
  double2* wbuf = (double2*)d_work;
  double2* gbuf = wbuf + (ten ? 12 : 6) * fs;
  const double npts = (double)g->n1 * g->n2 * g->n3;
  const int tc = col_tile(g, nf + 1);
  const int ntile = cmm_div_up((long long)g->n2 * g->h3, tc);
  const double2* wt = (const double2*)d_wtab;
  const int ck = col_kind(g);
  if (version & CMM_NOHS) {
    LAUNCH_COL(ck, k_col_backconv, dim3(ntile, batch), col_smem_bytes(g->n1, tc, 6, g->ax1.big), st, g->dev,
               d_active, R, 1.0 / (beta * npts), (const double2*)nullptr, fs, (const double2*)d_vhat,
               (const double2*)d_kst, wt, (double2*)d_out_hat, tc, 0.0, 1.0 / npts);
    return last_err();
  }
  if (!d_wd_rho) return CMM_ERR_ARG;
  const size_t csw = col_smem_bytes(g->n1, tc, nf, g->ax1.big), csb = col_smem_bytes(g->n1, tc, nf + 1, g->ax1.big);
#define LAUNCH_WEIGHTS(kern)                                                                                   \
  LAUNCH_COL(ck, kern, dim3(ntile, batch), csw, st, g->dev, d_active, R, 1.0 / npts, (const double2*)d_vhat,      \
             wbuf, fs, (const double2*)d_kst, wt, (double*)nullptr, 0, 0, tc, we.D, (const double2*)nullptr,   \
             (double*)nullptr)
  if (has_wda && ten) LAUNCH_WEIGHTS(k_col_weights_wda_t);
  else if (has_wda) LAUNCH_WEIGHTS(k_col_weights_wda);
  else if (ten) LAUNCH_WEIGHTS(k_col_weights_t);
  else LAUNCH_WEIGHTS(k_col_weights);
#undef LAUNCH_WEIGHTS
  int rc = last_err();
  if (rc) return rc;
  if ((rc = ypass(g, batch, d_active, wbuf, wbuf, fs, nf, 1, st))) return rc;
  const int chunk = zrow_chunk(g, nf);
  if (chunk < 1) return CMM_ERR_SMEM;
  switch (zrow_m3(g)) {
    case 32: rc = zrow_hvp_m3<32>(g, batch, d_active, R, version, we, transpose, wbuf, fs, gbuf, chunk, d_wd_rho, st); break;
    case 16: rc = zrow_hvp_m3<16>(g, batch, d_active, R, version, we, transpose, wbuf, fs, gbuf, chunk, d_wd_rho, st); break;
    case -1: rc = zrow_hvp_m3<-1>(g, batch, d_active, R, version, we, transpose, wbuf, fs, gbuf, chunk, d_wd_rho, st); break;
    default: rc = zrow_hvp_m3<0>(g, batch, d_active, R, version, we, transpose, wbuf, fs, gbuf, chunk, d_wd_rho, st);
  }
  if (rc) return rc;
  if ((rc = ypass(g, batch, d_active, gbuf, gbuf, fs, nf, 0, st))) return rc;
#define LAUNCH_BACKCONV(kern)                                                                                   \
  LAUNCH_COL(ck, kern, dim3(ntile, batch), csb, st, g->dev, d_active, R, 1.0 / (beta * npts), (const double2*)gbuf, \
             fs, (const double2*)d_vhat, (const double2*)d_kst, wt, (double2*)d_out_hat, tc, we.D, 1.0 / npts)
  if (has_wda && ten) LAUNCH_BACKCONV(k_col_backconv_wda_t);
  else if (has_wda) LAUNCH_BACKCONV(k_col_backconv_wda);
  else if (ten) LAUNCH_BACKCONV(k_col_backconv_t);
  else LAUNCH_BACKCONV(k_col_backconv);
#undef LAUNCH_BACKCONV
  return last_err();
}

// Partial-sum slots any pass writes per instance: one per x-plane, or one
// per column tile of the narrowest column pass (13 fields + rho_hat).
extern "C" int cmm_part_slots(const cmm_grid* g) {
  if (!g) return 0;
  const int tc = col_tile(g, 14);
  const int ntile = cmm_div_up((long long)g->n2 * g->h3, tc);
  return g->n1 > ntile ? g->n1 : ntile;
}

extern "C" int cmm_plane_smem_bytes(const cmm_grid* g, int nslot, size_t* bytes) {
  if (!g || !bytes) return CMM_ERR_ARG;
  *bytes = plane_smem_bytes(g->n2, g->n3, nslot);
  return CMM_OK;
}

static int col_fft_3d(const cmm_grid* g, int batch, const double2* in, double2* out, int inv, cudaStream_t st) {
  const int tc = col_tile(g, 1);
  const size_t cs = col_smem_bytes(g->n1, tc, 1, g->ax1.big);
  const int ntile = cmm_div_up((long long)g->n2 * g->h3, tc);
  LAUNCH_COL(col_kind(g), k_col_fft, dim3(ntile, batch), cs, st, g->dev, in, out, tc, inv);
  return last_err();
}

// Real fields -> yz-spectra (y and z forward) of every plane.
static int plane_r2c(const cmm_grid* g, int batch, const double* in, double2* spec, cudaStream_t st,
                     const int* act = nullptr) {
  if (plane_staged(g, 1)) {
    int rc = zrow_op(g, batch, act, OpR2C{in}, nullptr, spec, nullptr, 0, st);
    if (rc) return rc;
    return ypass(g, batch, act, spec, spec, 0, 1, 0, st);
  }
  const size_t ps = plane_smem_bytes(g->n2, g->n3, 1);
  LAUNCH_PLANE(plane_kind(g), k_plane_r2c, dim3(g->n1, batch), ps, st, g->dev, act, in, spec);
  return last_err();
}

// yz-spectra -> real fields; the staged form inverts y in place (spec is consumed).
static int plane_c2r_consume(const cmm_grid* g, int batch, double2* spec, double* out, cudaStream_t st) {
  if (plane_staged(g, 1)) {
    int rc = ypass(g, batch, nullptr, spec, spec, 0, 1, 1, st);
    if (rc) return rc;
    return zrow_op(g, batch, nullptr, OpC2R{out}, spec, nullptr, nullptr, 0, st);
  }
  const size_t ps = plane_smem_bytes(g->n2, g->n3, 1);
  LAUNCH_PLANE(plane_kind(g), k_plane_c2r, dim3(g->n1, batch), ps, st, g->dev, (const double2*)spec, out);
  return last_err();
}

// Stream-ordered scratch of `bytes` for the staged passes whose input is read-only.
static int scratch_alloc(void** p, size_t bytes, cudaStream_t st) {
  return (cudaMallocAsync(p, bytes, st) == cudaSuccess) ? CMM_OK : CMM_ERR_NOMEM;
}

extern "C" int cmm_rfft3d(const cmm_grid* g, int batch, const double* d_in, double* d_spec, void* stream) {
  if (!g || !d_in || !d_spec || batch < 1) return CMM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = plane_r2c(g, batch, d_in, (double2*)d_spec, st);
  if (rc) return rc;
  return col_fft_3d(g, batch, (const double2*)d_spec, (double2*)d_spec, 0, st);
}

extern "C" int cmm_irfft3d(const cmm_grid* g, int batch, double* d_spec, double* d_out, void* stream) {
  if (!g || !d_spec || !d_out || batch < 1) return CMM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = col_fft_3d(g, batch, (const double2*)d_spec, (double2*)d_spec, 1, st);  // in place (consumed)
  if (rc) return rc;
  return plane_c2r_consume(g, batch, (double2*)d_spec, d_out, st);
}

extern "C" int cmm_rfft_yz(const cmm_grid* g, int batch, const double* d_in, double* d_spec, void* stream) {
  if (!g || !d_in || !d_spec || batch < 1) return CMM_ERR_ARG;
  return plane_r2c(g, batch, d_in, (double2*)d_spec, (cudaStream_t)stream);
}

extern "C" int cmm_irfft_yz(const cmm_grid* g, int batch, const double* d_spec, double* d_out, void* stream) {
  if (!g || !d_spec || !d_out || batch < 1) return CMM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (plane_staged(g, 1)) {
    void* tmp = nullptr;
    const size_t bytes = sizeof(double2) * (size_t)batch * g->n1 * g->n2 * g->h3;
    int rc = scratch_alloc(&tmp, bytes, st);
    if (rc) return rc;
    rc = ypass(g, batch, nullptr, (const double2*)d_spec, (double2*)tmp, 0, 1, 1, st);
    if (!rc) rc = zrow_op(g, batch, nullptr, OpC2R{d_out}, (const double2*)tmp, nullptr, nullptr, 0, st);
    cudaFreeAsync(tmp, st);
    return rc;
  }
  const size_t ps = plane_smem_bytes(g->n2, g->n3, 1);
  LAUNCH_PLANE(plane_kind(g), k_plane_c2r, dim3(g->n1, batch), ps, st, g->dev, (const double2*)d_spec, d_out);
  return last_err();
}

extern "C" int cmm_fmt_weights(const cmm_grid* g, double R, double* d_wtab, void* stream) {
  if (!g || !d_wtab) return CMM_ERR_ARG;
  const long long tot = (long long)g->n1 * g->n2 * g->h3;
  k_fmt_weights<<<(int)((tot + 255) / 256), 256, 0, (cudaStream_t)stream>>>(g->dev, R, (double2*)d_wtab);
  return last_err();
}

// Plane pass of the functional pipeline over nf weighted-density spectra
// (wbuf, field stride fs): fused where the plane fits, else staged (y pass,
// z rows with the pointwise step, y pass of the results).  want as
// cmm_fmt_c1; dPhi spectra into gbuf when want & 1.
static int fmt_plane_pass(const cmm_grid* g, int batch, const int* act, double R, int version,
                          const cmm_wda_eos& we, double2* wbuf, double2* gbuf, size_t fs, int nf, double* part,
                          int nslot, int want, double* wd, cudaStream_t st) {
  const bool ten = (version & CMM_TENSOR) != 0, has_wda = (version & CMM_WDA) != 0;
  const size_t fsr = (size_t)batch * g->n1 * g->n2 * g->n3;  // real field stride of wd
  const size_t ps = plane_smem_bytes(g->n2, g->n3, nf);
  if (!ten && !plane_staged(g, nf) && g->staging == 0) {  // fused, the plane split over a CTA pair
    const size_t ps2 = plane_smem_bytes(g->n2, g->n3, (nf + 1) / 2);
    if (has_wda)
      LAUNCH_PLANE_T(plane_kind(g), k_plane_fmt_wda_c2, dim3(2 * g->n1, batch), CMM_FMT2_THREADS, ps2, st, g->dev,
                     act, R, version, we, (const double2*)wbuf, fs, gbuf, fs, part, nslot, want, wd, fsr);
    else
      LAUNCH_PLANE_T(plane_kind(g), k_plane_fmt_c2, dim3(2 * g->n1, batch), CMM_FMT2_THREADS, ps2, st, g->dev, act,
                     R, version, we, (const double2*)wbuf, fs, gbuf, fs, part, nslot, want, wd, fsr);
    return last_err();
  }
  if (!ten && !plane_staged(g, nf)) {  // fused plane pass
    if (has_wda)
      LAUNCH_PLANE_T(plane_kind(g), k_plane_fmt_wda, dim3(g->n1, batch), CMM_FMT_THREADS, ps, st, g->dev, act, R,
                     version, we, (const double2*)wbuf, fs, gbuf, fs, part, nslot, want, wd, fsr);
    else
      LAUNCH_PLANE_T(plane_kind(g), k_plane_fmt, dim3(g->n1, batch), CMM_FMT_THREADS, ps, st, g->dev, act, R,
                     version, we, (const double2*)wbuf, fs, gbuf, fs, part, nslot, want, wd, fsr);
    return last_err();
  }
  int rc = ypass(g, batch, act, wbuf, wbuf, fs, nf, 1, st);
  if (rc) return rc;
  rc = zrow_fmt(g, batch, act, R, version, we, wbuf, fs, gbuf, nf, part, nslot, want, wd, st);
  if (rc) return rc;
  if (want & 1) rc = ypass(g, batch, act, gbuf, gbuf, fs, nf, 0, st);
  return rc;
}

extern "C" int cmm_fmt_c1(const cmm_grid* g, int batch, const int* d_active, double R, double beta,
                          int version, const cmm_wda_eos* wda, const double* d_kst, const double* d_wtab,
                          const double* d_rhohat, double* d_chat, double* d_work, double* d_part, int nslot,
                          int want, double* d_wd, void* stream) {
  if (!g || batch < 1 || !d_kst || !d_rhohat || !d_work || !d_part) return CMM_ERR_ARG;
  if ((want & 1) && !d_chat) return CMM_ERR_ARG;
  if ((want & 8) && !d_wd) return CMM_ERR_ARG;
  const bool has_wda = (version & CMM_WDA) != 0;
  const bool ten = (version & CMM_TENSOR) != 0;
  if (has_wda && !wda) return CMM_ERR_ARG;
  cmm_wda_eos we;
  memset(&we, 0, sizeof(we));
  if (has_wda) we = *wda;
  const int nf = (has_wda ? 6 : 5) + (ten ? 6 : 0);  // weighted densities (and dPhi fields)
  cudaStream_t st = (cudaStream_t)stream;
  const size_t fs = (size_t)batch * g->n1 * g->n2 * g->h3;  // field stride (double2)
  double2* wbuf = (double2*)d_work;               // weighted-density spectra (up to 6, 12 with tensors)
  double2* gbuf = wbuf + (ten ? 12 : 6) * fs;     // dPhi spectra
  const double npts = (double)g->n1 * g->n2 * g->n3;
  const int tc = col_tile(g, nf + 1);
  const int ntile = cmm_div_up((long long)g->n2 * g->h3, tc);
  if (nslot < g->n1 || nslot < ntile) return CMM_ERR_WORKSPACE;
  const size_t csw = col_smem_bytes(g->n1, tc, nf, g->ax1.big), csb = col_smem_bytes(g->n1, tc, nf + 1, g->ax1.big);
  const double2* wt = (const double2*)d_wtab;
  const int ck = col_kind(g);
  if (version & CMM_NOHS) {  // MFA term alone: one column pass, the C1 spectrum only
    if (want != 1) return CMM_ERR_ARG;
    LAUNCH_COL(ck, k_col_backconv, dim3(ntile, batch), col_smem_bytes(g->n1, tc, 6, g->ax1.big), st, g->dev, d_active, R,
               1.0 / (beta * npts), (const double2*)nullptr, fs, (const double2*)d_rhohat, (const double2*)d_kst,
               wt, (double2*)d_chat, tc, 0.0, 1.0 / npts);
    return last_err();
  }
#define LAUNCH_WEIGHTS(kern)                                                                             \
  LAUNCH_COL(ck, kern, dim3(ntile, batch), csw, st, g->dev, d_active, R, 1.0 / npts, (const double2*)d_rhohat, \
             wbuf, fs, (const double2*)d_kst, wt, d_part, nslot, (want & 2) ? 1 : 0, tc, we.D,             \
             (const double2*)nullptr, (double*)nullptr)
  if (has_wda && ten) LAUNCH_WEIGHTS(k_col_weights_wda_t);
  else if (has_wda) LAUNCH_WEIGHTS(k_col_weights_wda);
  else if (ten) LAUNCH_WEIGHTS(k_col_weights_t);
  else LAUNCH_WEIGHTS(k_col_weights);
#undef LAUNCH_WEIGHTS
  int rc = fmt_plane_pass(g, batch, d_active, R, version, we, wbuf, gbuf, fs, nf, d_part, nslot, want, d_wd, st);
  if (rc) return rc;
  if (want & 1) {
#define LAUNCH_BACKCONV(kern)                                                                            \
  LAUNCH_COL(ck, kern, dim3(ntile, batch), csb, st, g->dev, d_active, R, 1.0 / (beta * npts),               \
             (const double2*)gbuf, fs, (const double2*)d_rhohat, (const double2*)d_kst, wt, (double2*)d_chat, \
             tc, we.D, 1.0 / npts)
    if (has_wda && ten) LAUNCH_BACKCONV(k_col_backconv_wda_t);
    else if (has_wda) LAUNCH_BACKCONV(k_col_backconv_wda);
    else if (ten) LAUNCH_BACKCONV(k_col_backconv_t);
    else LAUNCH_BACKCONV(k_col_backconv);
#undef LAUNCH_BACKCONV
  }
  return last_err();
}

extern "C" int cmm_picard_static_step(const cmm_grid* g, int batch, const int* d_active,
                                      const double* d_params, double beta, double lambda3, double thr,
                                      double a_tol, double r_tol, const double* d_chat, const double* d_rho, const double* d_V,
                                      long long vstride, double* d_rho_out, double* d_rhohat_out,
                                      double* d_part, int nslot, void* stream) {
  if (!g || batch < 1 || !d_params || !d_chat || !d_rho || !d_V || !d_rho_out || !d_rhohat_out || !d_part)
    return CMM_ERR_ARG;
  if (!(a_tol >= 0) || !(r_tol >= 0)) return CMM_ERR_ARG;
  if (nslot < g->n1) return CMM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (plane_staged(g, 1)) {  // y inverse of C1 into the output spectrum, z rows in place, y forward
    double2* out = (double2*)d_rhohat_out;
    int rc = ypass(g, batch, d_active, (const double2*)d_chat, out, 0, 1, 1, st);
    if (rc) return rc;
    OpPicard op{d_params, beta, lambda3, thr, a_tol, r_tol, d_rho, d_V, vstride, d_rho_out};
    rc = zrow_op(g, batch, d_active, op, out, out, d_part, nslot, st);
    if (rc) return rc;
    return ypass(g, batch, d_active, out, out, 0, 1, 0, st);
  }
  const size_t ps = plane_smem_bytes(g->n2, g->n3, 1);
  LAUNCH_PLANE(plane_kind(g), k_plane_picard, dim3(g->n1, batch), ps, (cudaStream_t)stream, g->dev, d_active,
               d_params, beta, lambda3, thr, a_tol, r_tol, (const double2*)d_chat, d_rho, d_V, vstride,
               d_rho_out,
               (double2*)d_rhohat_out, d_part, nslot);
  return last_err();
}

extern "C" int cmm_residual_step(const cmm_grid* g, int batch, const int* d_active, const double* d_params,
                                 double beta, double lambda3, double a_tol, double r_tol, const double* d_chat,
                                 const double* d_rho,
                                 const double* d_V,
                                 long long vstride, double* d_r_out, const double* const* d_hist, int nhist,
                                 long long hstride, double* d_part, int nslot, void* stream) {
  if (!g || batch < 1 || !d_params || !d_chat || !d_rho || !d_V || !d_r_out || !d_part) return CMM_ERR_ARG;
  if (nhist < 0 || nhist > CMM_MAX_HIST || (nhist && !d_hist)) return CMM_ERR_ARG;
  if (!(a_tol >= 0) || !(r_tol >= 0)) return CMM_ERR_ARG;
  if (nslot < g->n1) return CMM_ERR_WORKSPACE;
  HistPtrs hp;
  for (int j = 0; j < CMM_MAX_HIST; ++j) hp.p[j] = (j < nhist) ? d_hist[j] : nullptr;
  cudaStream_t st = (cudaStream_t)stream;
  if (plane_staged(g, 1)) {  // y inverse of C1 into stream-ordered scratch, then z rows
    void* tmp = nullptr;
    int rc = scratch_alloc(&tmp, sizeof(double2) * (size_t)batch * g->n1 * g->n2 * g->h3, st);
    if (rc) return rc;
    rc = ypass(g, batch, d_active, (const double2*)d_chat, (double2*)tmp, 0, 1, 1, st);
    OpResidual op{d_params, beta, lambda3, a_tol, r_tol, d_rho, d_V, vstride, d_r_out, hp, nhist, hstride};
    if (!rc) rc = zrow_op(g, batch, d_active, op, (const double2*)tmp, nullptr, d_part, nslot, st);
    cudaFreeAsync(tmp, st);
    return rc;
  }
  const size_t ps = plane_smem_bytes(g->n2, g->n3, 1);
  LAUNCH_PLANE(plane_kind(g), k_plane_residual, dim3(g->n1, batch), ps, (cudaStream_t)stream, g->dev, d_active,
               d_params, beta, lambda3, a_tol, r_tol, (const double2*)d_chat, d_rho, d_V, vstride, d_r_out,
               hp, nhist, hstride, d_part, nslot);
  return last_err();
}

extern "C" int cmm_mix_step(const cmm_grid* g, int batch, const int* d_active, const double* d_coef,
                            const double* const* d_fields, const long long* fstride, int nfield, int clip,
                            double thr, double lambda3, const double* d_ref, long long refstride, const double* d_V,
                            long long vstride, double* d_rho_out, double* d_rhohat_out, double* d_part,
                            int nslot, void* stream) {
  if (!g || batch < 1 || !d_coef || !d_fields || !fstride || !d_ref || !d_V || !d_rho_out || !d_rhohat_out)
    return CMM_ERR_ARG;
  if (nfield < 1 || nfield > CMM_MAX_FIELDS) return CMM_ERR_ARG;
  if (nslot < g->n1) return CMM_ERR_WORKSPACE;
  FieldPtrs fp;
  for (int j = 0; j < CMM_MAX_FIELDS; ++j) {
    fp.p[j] = (j < nfield) ? d_fields[j] : nullptr;
    fp.stride[j] = (j < nfield) ? fstride[j] : 0;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (plane_staged(g, 1)) {  // z rows (mix, forward) into the output spectrum, then y forward
    OpMix op{d_coef, fp, nfield, clip, thr, lambda3, d_ref, refstride, d_V, vstride, d_rho_out};
    int rc = zrow_op(g, batch, d_active, op, nullptr, (double2*)d_rhohat_out, d_part, nslot, st);
    if (rc) return rc;
    return ypass(g, batch, d_active, (double2*)d_rhohat_out, (double2*)d_rhohat_out, 0, 1, 0, st);
  }
  const size_t ps = plane_smem_bytes(g->n2, g->n3, 1);
  LAUNCH_PLANE(plane_kind(g), k_plane_mix, dim3(g->n1, batch), ps, (cudaStream_t)stream, g->dev, d_active, d_coef,
               fp, nfield, clip, thr, lambda3, d_ref, refstride, d_V, vstride, d_rho_out, (double2*)d_rhohat_out,
               d_part, nslot);
  return last_err();
}

extern "C" int cmm_ls_prepare(const cmm_grid* g, int batch, const int* d_active, double R, int version,
                              const cmm_wda_eos* wda, const double* d_kst, const double* d_wtab, const double* d_r,
                              const double* d_rhohat, const double* d_wd_rho, double* d_rhat, double* d_work,
                              double* d_wd_r, double* d_ls_part, int nslot, void* stream) {
  if (!g || batch < 1 || !d_kst || !d_r || !d_rhohat || !d_wd_rho || !d_rhat || !d_work || !d_wd_r || !d_ls_part)
    return CMM_ERR_ARG;
  if (version & CMM_NOHS) return CMM_ERR_ARG;
  const bool has_wda = (version & CMM_WDA) != 0, ten = (version & CMM_TENSOR) != 0;
  if (has_wda && !wda) return CMM_ERR_ARG;
  cmm_wda_eos we;
  memset(&we, 0, sizeof(we));
  if (has_wda) we = *wda;
  const int nw = (has_wda ? 6 : 5) + (ten ? 6 : 0);
  cudaStream_t st = (cudaStream_t)stream;
  const size_t fs = (size_t)batch * g->n1 * g->n2 * g->h3;
  const double npts = (double)g->n1 * g->n2 * g->n3;
  const int tc = col_tile(g, nw + 1);
  const int ntile = cmm_div_up((long long)g->n2 * g->h3, tc);
  if (nslot < g->n1 || nslot < ntile) return CMM_ERR_WORKSPACE;
  double2* rhat = (double2*)d_rhat;
  int rc = plane_r2c(g, batch, d_r, rhat, st, d_active);  // yz-spectrum of r
  if (rc) return rc;
  double2* wbuf = (double2*)d_work;
  const size_t csw = col_smem_bytes(g->n1, tc, nw + 1, g->ax1.big);
  const double2* wt = (const double2*)d_wtab;
  const int ck = col_kind(g);
#define LAUNCH_WEIGHTS_LS(kern)                                                                          \
  LAUNCH_COL(ck, kern, dim3(ntile, batch), csw, st, g->dev, d_active, R, 1.0 / npts, (const double2*)rhat,   \
             wbuf, fs, (const double2*)d_kst, wt, (double*)nullptr, nslot, 0, tc, we.D,                     \
             (const double2*)d_rhohat, d_ls_part)
  if (has_wda && ten) LAUNCH_WEIGHTS_LS(k_col_weights_ls_wda_t);
  else if (has_wda) LAUNCH_WEIGHTS_LS(k_col_weights_ls_wda);
  else if (ten) LAUNCH_WEIGHTS_LS(k_col_weights_ls_t);
  else LAUNCH_WEIGHTS_LS(k_col_weights_ls);
#undef LAUNCH_WEIGHTS_LS
  // inverse y/z of the weighted densities of r, stored in real space
  rc = fmt_plane_pass(g, batch, d_active, R, version, we, wbuf, wbuf, fs, nw, d_ls_part, nslot, 8, d_wd_r, st);
  if (rc) return rc;
  const size_t fsr = (size_t)batch * g->n1 * g->n2 * g->n3;
  k_ls_n3max<<<dim3(g->n1, batch), 256, 0, st>>>(g->dev, d_active, d_wd_rho, d_wd_r, fsr, d_ls_part, nslot);
  return last_err();
}

template <bool WDA, bool TEN>
static int ls_omega_one(const cmm_grid* g, int batch, const int* act, const double* n3a, long long n3s, double c0, double c1,
                        double c2, double R, double lambda3, int version, const cmm_wda_eos& we, const double* rho,
                        const double* r, const double* V, long long vstride, const double* wd_rho,
                        const double* wd_r, double* ls_part, int nslot, double* alpha, cudaStream_t st) {
  const size_t fsr = (size_t)batch * g->n1 * g->n2 * g->n3;
  k_ls_omega<WDA, TEN><<<dim3(g->n1, batch), CMM_LS_THREADS, 0, st>>>(
      g->dev, act, n3a, n3s, c0, c1, c2, R, lambda3, version, we, rho, r, V, vstride, wd_rho, wd_r, fsr, ls_part,
      nslot, alpha);
  return last_err();
}

extern "C" int cmm_ls_omega(const cmm_grid* g, int batch, const int* d_active, const double* d_n3a,
                            long long n3a_stride, double c0, double c1, double c2, double R, double lambda3, int version,
                            const cmm_wda_eos* wda, const double* d_rho, const double* d_r, const double* d_V,
                            long long vstride, const double* d_wd_rho, const double* d_wd_r, double* d_ls_part,
                            int nslot, double* d_alpha, void* stream) {
  if (!g || batch < 1 || !d_n3a || !d_rho || !d_r || !d_V || !d_wd_rho || !d_wd_r || !d_ls_part || !d_alpha)
    return CMM_ERR_ARG;
  if (nslot < g->n1) return CMM_ERR_WORKSPACE;
  const bool has_wda = (version & CMM_WDA) != 0, ten = (version & CMM_TENSOR) != 0;
  if (has_wda && !wda) return CMM_ERR_ARG;
  cmm_wda_eos we;
  memset(&we, 0, sizeof(we));
  if (has_wda) we = *wda;
  cudaStream_t st = (cudaStream_t)stream;
#define LS_OMEGA(w, t)                                                                                     \
  ls_omega_one<w, t>(g, batch, d_active, d_n3a, n3a_stride, c0, c1, c2, R, lambda3, version, we, d_rho, d_r, d_V, vstride, \
                     d_wd_rho, d_wd_r, d_ls_part, nslot, d_alpha, st)
  if (has_wda && ten) return LS_OMEGA(true, true);
  if (has_wda) return LS_OMEGA(true, false);
  if (ten) return LS_OMEGA(false, true);
  return LS_OMEGA(false, false);
#undef LS_OMEGA
}

extern "C" int cmm_ls_finalize(int batch, const int* d_active, const double* d_ls_part, int nslot, double* d_ls,
                               void* stream) {
  if (batch < 1 || !d_ls_part || !d_ls || nslot < 1) return CMM_ERR_ARG;
  k_ls_finalize<<<batch, dim3(32, CMM_NLS), 0, (cudaStream_t)stream>>>(d_active, d_ls_part, nslot, d_ls);
  return last_err();
}

extern "C" int cmm_stats_finalize(int batch, const int* d_active, const double* d_part, int nslot,
                                  unsigned mask, double* d_stats, void* stream) {
  if (batch < 1 || !d_part || !d_stats || nslot < 1) return CMM_ERR_ARG;
  k_stats_finalize<<<batch, dim3(32, NQ), 0, (cudaStream_t)stream>>>(d_active, d_part, nslot, mask, d_stats);
  return last_err();
}
