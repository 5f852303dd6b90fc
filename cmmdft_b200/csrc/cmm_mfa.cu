// Mean-field-attraction kernel spectrum.
//
// MFAFunctional (cmmdft/functionals.py:770-939) samples the cut-and-shifted
// LJ pair potential U(r) on the centred grid (or on the rep x rep x rep
// supercell with tail corrections), transforms it with the reference's phase
// convention and multiplies by the Lanczos factor:
//   kpotential = fftn(U) * exp(i pi scalprod) / Npts_big * sigma_L
// and derive(krho) = ifft(krho * kpotential[::rep, ::rep, ::rep]) * V_big.
// Unlike the FMT weights, this phase does not cancel: the effective kernel
// is  K(k) = fftn(U)(rep k) sigma_L(rep k) exp(i pi scalprod(rep k)) V_big /
// (Npts_big Npts_small), of which Grid.ifft's .real keeps the Hermitian part
//   K_h(k) = F(K) sigma_L(K) [exp(i pi s(K)) + exp(-i pi s(-K))] / 2 * scale.
// This file builds K_h on the device in the column-pass layout.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cmm_common.cuh"

// U(r) on the (super)cell grid, generate_potential_lj (functionals.py:878-910).
__global__ void k_mfa_potential(double rv0, double rv1, double rv2, double rv3, double rv4, double rv5,
                                double rv6, double rv7, double rv8, int n1, int n2, int n3, double sigma,
                                double epsilon, double cutoff, int has_cut, double rmin, double limit,
                                double* __restrict__ U) {
  const long long npts = (long long)n1 * n2 * n3;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= npts) return;
  const int k = (int)(idx % n3);
  const int j = (int)((idx / n3) % n2);
  const int i = (int)(idx / ((long long)n3 * n2));
  const double g0 = __dadd_rn(__dmul_rn((double)i, 1.0 / (double)n1), -0.5);
  const double g1 = __dadd_rn(__dmul_rn((double)j, 1.0 / (double)n2), -0.5);
  const double g2 = __dadd_rn(__dmul_rn((double)k, 1.0 / (double)n3), -0.5);
  const double rv[9] = {rv0, rv1, rv2, rv3, rv4, rv5, rv6, rv7, rv8};
  double p[3];
  for (int b = 0; b < 3; ++b)
    p[b] = __dadd_rn(__dadd_rn(__dmul_rn(rv[b], g0), __dmul_rn(rv[3 + b], g1)), __dmul_rn(rv[6 + b], g2));
  const double r = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(p[0], p[0]), __dmul_rn(p[1], p[1])), __dmul_rn(p[2], p[2])));
  double pot = limit;
  if (r > rmin) {
    const double x = __ddiv_rn(sigma, r);
    const double x2 = __dmul_rn(x, x);
    const double x6 = __dmul_rn(__dmul_rn(x2, x2), x2);
    const double x12 = __dmul_rn(x6, x6);
    pot = __dmul_rn(4.0 * epsilon, __dsub_rn(x12, x6));
  }
  if (has_cut) {
    if (r <= cutoff) {
      const double q = sigma / cutoff;
      const double q2 = q * q;
      const double rc6 = q2 * q2 * q2;
      pot = __dsub_rn(pot, __dmul_rn(4.0 * epsilon, __dsub_rn(__dmul_rn(rc6, rc6), rc6)));
    } else {
      pot = 0.0;
    }
  }
  U[idx] = pot;
}

struct MfaTables {
  const int* P1;     // big-spectrum x index (natural) at small DIF-x position
  const int* P2;     // big-spectrum y position at small y position
  const int* P3;     // big-spectrum z position at small z position
  const double* sA[3];  // scalprod term at K
  const double* sB[3];  // scalprod term at -K
  const double* sl[3];  // big-grid Lanczos factor at K
};

__global__ void k_mfa_gather(int n1, int n2, int h3, int nb2, int hb3, MfaTables t, double scale,
                             const double2* __restrict__ big, double2* __restrict__ kst) {
  const long long tot = (long long)n1 * n2 * h3;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= tot) return;
  const int p3 = (int)(idx % h3);
  const int p2 = (int)((idx / h3) % n2);
  const int p1 = (int)(idx / ((long long)h3 * n2));
  const double2 F = big[((size_t)t.P1[p1] * nb2 + t.P2[p2]) * hb3 + t.P3[p3]];
  const double sa = (t.sA[0][p1] + t.sA[1][p2]) + t.sA[2][p3];
  const double sb = (t.sB[0][p1] + t.sB[1][p2]) + t.sB[2][p3];
  double sna, csa, snb, csb;
  sincos(M_PI * sa, &sna, &csa);
  sincos(M_PI * sb, &snb, &csb);
  // (exp(i pi sa) + exp(-i pi sb)) / 2
  const double2 ph = make_double2(0.5 * (csa + csb), 0.5 * (sna - snb));
  const double sl = (t.sl[0][p1] * t.sl[1][p2]) * t.sl[2][p3];
  const double2 K = cscale(cmul(F, ph), sl * scale);
  kst[idx] = K;
}

__global__ void k_sum(const double* __restrict__ x, long long n, double* __restrict__ out) {
  __shared__ double red[32];
  double acc = 0.0;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) acc += x[i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    acc = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (threadIdx.x == 0) *out = acc;
  }
}

static int signed_freq_h(int k, int n) {
  int half = (n - 1) / 2 + 1;
  return (k < half) ? k : k - n;
}

static double np_sinc_h(double x) {
  volatile double y = M_PI * (x == 0.0 ? 1.0e-20 : x);
  return sin(y) / y;
}

extern "C" int cmm_mfa_kernel(const cmm_grid* g, double sigma, double epsilon, double cutoff, double rmin,
                              double limit, int rep, double* d_kst, double* d_work, size_t* work_bytes,
                              double* vdw_a, void* stream) {
  if (!g || rep < 1 || rep > 4) return CMM_ERR_ARG;
  const int nb[3] = {rep * g->n1, rep * g->n2, rep * g->n3};
  const int hb3 = nb[2] / 2 + 1;
  const long long nptb = (long long)nb[0] * nb[1] * nb[2];
  const long long nspb = (long long)nb[0] * nb[1] * hb3;
  const int ns[3] = {g->n1, g->n2, g->h3};
  // work: U (nptb doubles) | big spectrum (nspb double2) | tables | sum
  size_t off_U = 0;
  size_t off_S = (off_U + sizeof(double) * nptb + 255) & ~(size_t)255;
  size_t off_T = (off_S + sizeof(double2) * nspb + 255) & ~(size_t)255;
  size_t tbytes = sizeof(int) * (ns[0] + ns[1] + ns[2]) + sizeof(double) * 3 * (ns[0] + ns[1] + ns[2]) + 64;
  size_t off_sum = (off_T + tbytes + 255) & ~(size_t)255;
  size_t need = off_sum + 256;
  if (!d_kst) {
    if (!work_bytes) return CMM_ERR_ARG;
    *work_bytes = need;
    return CMM_OK;
  }
  if (!d_work || !work_bytes || *work_bytes < need) return CMM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  double rvb[9];
  for (int i = 0; i < 9; ++i) rvb[i] = g->rvecs[i] * rep;  // rvecs * repetitions (rows)
  cmm_grid* big = nullptr;
  int rc = (rep == 1) ? CMM_OK : cmm_grid_create(nb[0], nb[1], nb[2], rvb, &big);
  if (rc) return rc;
  const cmm_grid* gb = (rep == 1) ? g : big;
  char* w = (char*)d_work;
  double* U = (double*)(w + off_U);
  double* S = (double*)(w + off_S);
  const int has_cut = cutoff > 0.0 ? 1 : 0;
  {
    int nblk = (int)((nptb + 255) / 256);
    k_mfa_potential<<<nblk, 256, 0, st>>>(rvb[0], rvb[1], rvb[2], rvb[3], rvb[4], rvb[5], rvb[6], rvb[7], rvb[8],
                                          nb[0], nb[1], nb[2], sigma, epsilon, cutoff, has_cut, rmin, limit, U);
  }
  double* dsum = (double*)(w + off_sum);
  k_sum<<<1, 1024, 0, st>>>(U, nptb, dsum);
  rc = cmm_rfft3d(gb, 1, U, S, st);
  if (rc) { if (big) cmm_grid_destroy(big); return rc; }

  // host tables for the gather
  std::vector<int> P[3];
  std::vector<double> sA[3], sB[3], sl[3];
  // inverse position maps of the big plan (y, z)
  std::vector<int> bpos2(nb[1]), bpos3(hb3);
  for (int p = 0; p < nb[1]; ++p) bpos2[gb->hpos_k2[p]] = p;
  for (int p = 0; p < hb3; ++p) bpos3[gb->hpos_k3[p]] = p;
  const int* kof[3] = {g->hpos_k1, g->hpos_k2, g->hpos_k3};
  for (int a = 0; a < 3; ++a) {
    P[a].resize(ns[a]); sA[a].resize(ns[a]); sB[a].resize(ns[a]); sl[a].resize(ns[a]);
    const double d = gb->spacing[a];
    const double val = 1.0 / (nb[a] * d);
    const double kcut = 2.0 * M_PI / d;
    for (int p = 0; p < ns[a]; ++p) {
      const int K = (rep * kof[a][p]) % nb[a];
      const int Kn = (nb[a] - K) % nb[a];
      if (a == 0) P[a][p] = K;
      else if (a == 1) P[a][p] = bpos2[K];
      else P[a][p] = bpos3[K];
      volatile double fa = (double)signed_freq_h(K, nb[a]) * val;
      volatile double ka = (2.0 * M_PI) * fa;
      volatile double fb = (double)signed_freq_h(Kn, nb[a]) * val;
      volatile double kb = (2.0 * M_PI) * fb;
      volatile double ta = ka * d;
      volatile double tb = kb * d;
      sA[a][p] = ta * nb[a];
      sB[a][p] = tb * nb[a];
      sl[a][p] = np_sinc_h(ka / kcut);
    }
  }
  std::vector<char> host(tbytes, 0);
  size_t o = 0;
  const int* dP[3];
  const double *dA[3], *dB[3], *dL[3];
  char* dT = w + off_T;
  for (int a = 0; a < 3; ++a) {
    memcpy(&host[o], P[a].data(), sizeof(int) * ns[a]);
    dP[a] = (const int*)(dT + o);
    o += sizeof(int) * ns[a];
  }
  o = (o + 7) & ~(size_t)7;
  for (int a = 0; a < 3; ++a) {
    memcpy(&host[o], sA[a].data(), sizeof(double) * ns[a]); dA[a] = (const double*)(dT + o); o += sizeof(double) * ns[a];
    memcpy(&host[o], sB[a].data(), sizeof(double) * ns[a]); dB[a] = (const double*)(dT + o); o += sizeof(double) * ns[a];
    memcpy(&host[o], sl[a].data(), sizeof(double) * ns[a]); dL[a] = (const double*)(dT + o); o += sizeof(double) * ns[a];
  }
  if (cudaMemcpyAsync(dT, host.data(), o, cudaMemcpyHostToDevice, st) != cudaSuccess) {
    if (big) cmm_grid_destroy(big);
    return CMM_ERR_CUDA;
  }
  MfaTables t;
  t.P1 = dP[0]; t.P2 = dP[1]; t.P3 = dP[2];
  for (int a = 0; a < 3; ++a) { t.sA[a] = dA[a]; t.sB[a] = dB[a]; t.sl[a] = dL[a]; }
  const double vol_big = gb->volume;
  const double npts_small = (double)g->n1 * g->n2 * g->n3;
  const double scale = vol_big / ((double)nptb * npts_small);
  const long long tot = (long long)g->n1 * g->n2 * g->h3;
  k_mfa_gather<<<(int)((tot + 255) / 256), 256, 0, st>>>(g->n1, g->n2, g->h3, nb[1], hb3, t, scale,
                                                         (const double2*)S, (double2*)d_kst);
  rc = (cudaPeekAtLastError() == cudaSuccess) ? CMM_OK : CMM_ERR_CUDA;
  if (vdw_a && rc == CMM_OK) {
    double hsum = 0.0;
    if (cudaMemcpyAsync(&hsum, dsum, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      rc = CMM_ERR_CUDA;
    *vdw_a = 0.5 * (hsum * (vol_big / (double)nptb));
  }
  cudaStreamSynchronize(st);  // tables in d_work and the temporary big plan are released below
  if (big) cmm_grid_destroy(big);
  return rc;
}
