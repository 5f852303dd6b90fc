// Grid plans: radix factorisation, twiddle tables, digit-reversal position
// tables and per-position k-space tables.
//
// Reference: the k-grid, scalprod and Lanczos tables of Grid.__init__
// (cmmdft/system.py:232-295).  The k component of axis a at signed
// frequency m is computed the way numpy does it there:
//   k = (2 pi) * (m * (1 / (N * d)))   with d = |rvecs[:, a]| / N  (column norm)
// and the Lanczos factor per axis is np.sinc(k / kcut), kcut = 2 pi / d.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <vector>

#include "cmm_common.cuh"

static const char* kStatusText[] = {
    "ok", "bad argument", "unsupported grid shape", "CUDA runtime error",
    "plane or tile does not fit in shared memory", "out of memory",
    "workspace too small", "unsupported option"};

extern "C" int cmm_version(void) { return 100; }

extern "C" const char* cmm_status_string(int s) {
  if (s < 0 || s > 7) return "unknown status";
  return kStatusText[s];
}

// Radix orders of a length-n axis (the stages run in this order forward):
//   CMM_ORDER_DEFAULT  8s, 4s, 2s, then odd primes ascending
//   CMM_ORDER_NO8      4s, 2s (no radix 8), then odd primes ascending
//   CMM_ORDER_ODDFIRST odd primes descending, then 8s, 4s, 2s
//   CMM_ORDER_ODDDESC  8s, 4s, 2s, then odd primes descending
// (primes > 16 run as Rader or direct-DFT stages).
static bool factorise(int n, FftAxis* ax, int order = CMM_ORDER_DEFAULT) {
  ax->n = n;
  ax->nstage = 0;
  ax->rader = nullptr;
  int m = n;
  std::vector<int> pow2, odd, r;
  while (order != CMM_ORDER_NO8 && m % 8 == 0) { pow2.push_back(8); m /= 8; }
  while (m % 4 == 0) { pow2.push_back(4); m /= 4; }
  while (m % 2 == 0) { pow2.push_back(2); m /= 2; }
  for (int p = 3; m > 1; p += 2)
    while (m % p == 0) { odd.push_back(p); m /= p; }
  if (order == CMM_ORDER_ODDFIRST || order == CMM_ORDER_ODDDESC) std::reverse(odd.begin(), odd.end());
  if (order == CMM_ORDER_ODDFIRST) {
    r = odd;
    r.insert(r.end(), pow2.begin(), pow2.end());
  } else {
    r = pow2;
    r.insert(r.end(), odd.begin(), odd.end());
  }
  if ((int)r.size() > CMM_MAX_STAGES) return false;
  ax->big = 0;
  for (int x : r) if (x > CMM_MAX_SMALL_RADIX) ax->big = 1;
  if (r.empty()) r.push_back(1);
  int L = n;
  for (size_t s = 0; s < r.size(); ++s) {
    ax->radix[s] = r[s];
    ax->span[s] = L;
    L /= r[s];
  }
  ax->nstage = (int)r.size();
  if (n == 1) ax->nstage = 0;
  return true;
}

// Frequency index stored at each DIF output position: position
// p = q0*s0 + q1*s1 + ... holds k = q0 + R0*(q1 + R1*(q2 + ...)).
static void dif_positions(const FftAxis& ax, int* k_of_pos) {
  const int n = ax.n;
  for (int p = 0; p < n; ++p) {
    int rem = p, k = 0, mul = 1;
    for (int s = 0; s < ax.nstage; ++s) {
      int stride = ax.span[s] / ax.radix[s];
      int q = rem / stride;
      rem -= q * stride;
      k += q * mul;
      mul *= ax.radix[s];
    }
    k_of_pos[p] = (ax.nstage == 0) ? 0 : k;
  }
}

static void twiddles(int n, std::vector<double>& out) {
  out.resize(2 * (size_t)n);
  for (int t = 0; t < n; ++t) {
    long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)t / (long double)n;
    out[2 * t] = (double)cosl(a);
    out[2 * t + 1] = (double)sinl(a);
  }
}

// Host tables of one Rader stage (prime radix R, M = R - 1 smooth).
struct RaderHost {
  FftAxis axm;
  std::vector<double> twm, kf, ki;   // interleaved re, im
  std::vector<int> gin, gout;
};

static long long powmod(long long b, long long e, long long m) {
  long long r = 1;
  b %= m;
  while (e) {
    if (e & 1) r = r * b % m;
    b = b * b % m;
    e >>= 1;
  }
  return r;
}

// Smallest prime run by Rader's algorithm: below it the paired direct DFT
// (R/2 + 1 sums of R terms per butterfly, no extra barrier) is cheaper than
// the Rader stage's gather, two length R - 1 transforms, product and scatter
// (measured on B200: a 41 stage slower with Rader, 97 and above faster).
#define CMM_RADER_MIN 67

// false when R < CMM_RADER_MIN or R - 1 has a prime factor above
// CMM_MAX_SMALL_RADIX (the stage then stays a direct DFT).
static bool rader_plan(int R, RaderHost& h) {
  const int M = R - 1;
  if (R < CMM_RADER_MIN) return false;
  if (!factorise(M, &h.axm, CMM_ORDER_NO8) || h.axm.big) return false;
  std::vector<int> pf;
  for (int m = M, p = 2; m > 1; ++p)
    if (m % p == 0) {
      pf.push_back(p);
      while (m % p == 0) m /= p;
    }
  int g = 0;
  for (int c = 2; c < R && !g; ++c) {
    bool ok = true;
    for (int f : pf) ok = ok && powmod(c, M / f, R) != 1;
    if (ok) g = c;
  }
  if (!g) return false;
  const int ginv = (int)powmod(g, R - 2, R);
  h.gin.resize(M);
  h.gout.resize(M);
  for (int k = 0, a = 1, b = 1; k < M; ++k) {
    h.gout[k] = a;
    h.gin[k] = b;
    a = (int)((long long)a * g % R);
    b = (int)((long long)b * ginv % R);
  }
  twiddles(M, h.twm);
  // B_f = sum_j b_j w_M^{jf} with b_j = w_R^{g^j} (w = e^{-2 pi i/.}); the
  // inverse stage's kernel conj(b_j) has spectrum conj(B_{-f}).
  const long double pi = 3.141592653589793238462643383279502884L;
  std::vector<long double> cr(R), sr(R), cm(M), sm(M);
  for (int t = 0; t < R; ++t) { cr[t] = cosl(-2 * pi * t / R); sr[t] = sinl(-2 * pi * t / R); }
  for (int t = 0; t < M; ++t) { cm[t] = cosl(-2 * pi * t / M); sm[t] = sinl(-2 * pi * t / M); }
  std::vector<long double> Br(M), Bi(M);
  for (int f = 0; f < M; ++f) {
    long double re = 0, im = 0;
    for (int j = 0; j < M; ++j) {
      const int a = h.gout[j], w = (int)((long long)j * f % M);
      re += cr[a] * cm[w] - sr[a] * sm[w];
      im += cr[a] * sm[w] + sr[a] * cm[w];
    }
    Br[f] = re / M;
    Bi[f] = im / M;
  }
  std::vector<int> kpos(M);
  dif_positions(h.axm, kpos.data());
  h.kf.resize(2 * (size_t)M);
  h.ki.resize(2 * (size_t)M);
  for (int p = 0; p < M; ++p) {
    const int f = kpos[p], fm = (M - f) % M;
    h.kf[2 * p] = (double)Br[f];
    h.kf[2 * p + 1] = (double)Bi[f];
    h.ki[2 * p] = (double)Br[fm];
    h.ki[2 * p + 1] = -(double)Bi[fm];
  }
  return true;
}

static int signed_freq(int k, int n) {
  // numpy.fft.fftfreq ordering: [0, 1, ..., (n-1)/2, -(n/2), ..., -1]
  int half = (n - 1) / 2 + 1;  // number of non-negative entries
  return (k < half) ? k : k - n;
}

static double np_sinc(double x) {
  // numpy.sinc: y = pi * (x == 0 ? 1e-20 : x); sin(y) / y
  volatile double y = M_PI * (x == 0.0 ? 1.0e-20 : x);
  return sin(y) / y;
}

extern "C" int cmm_grid_create(int n1, int n2, int n3, const double* rvecs, cmm_grid** out) {
  return cmm_grid_create_sched(n1, n2, n3, rvecs, nullptr, out);
}

extern "C" int cmm_grid_create_sched(int n1, int n2, int n3, const double* rvecs, const int* sched,
                                     cmm_grid** out) {
  if (!out || !rvecs || n1 < 1 || n2 < 1 || n3 < 2) return CMM_ERR_ARG;
  int order[3] = {CMM_ORDER_DEFAULT, CMM_ORDER_DEFAULT, CMM_ORDER_DEFAULT};
  int staging = 0, tile = 0;
  if (sched) {
    for (int a = 0; a < 3; ++a) {
      if (sched[a] < -1 || sched[a] > CMM_ORDER_ODDDESC) return CMM_ERR_ARG;
      if (sched[a] >= 0) order[a] = sched[a];
    }
    if (sched[3] < -1 || sched[3] > 2) return CMM_ERR_ARG;
    staging = sched[3] > 0 ? sched[3] : 0;
    if (sched[4] < 0 || sched[4] > 16 || (sched[4] & (sched[4] - 1))) return CMM_ERR_ARG;
    tile = sched[4];
  }
  if (n1 > CMM_MAX_N || n2 > CMM_MAX_N || n3 > CMM_MAX_N) return CMM_ERR_SHAPE;
  // Even N3: the z axis is a half-length complex FFT plus the R2C/C2R twist.
  // Odd N3: a full-length complex FFT of the real rows (z rows kernels only).
  const int zfull = n3 % 2;
  cmm_grid* g = (cmm_grid*)calloc(1, sizeof(cmm_grid));
  if (!g) return CMM_ERR_NOMEM;
  g->n1 = n1; g->n2 = n2; g->n3 = n3; g->m3 = n3 / 2; g->h3 = n3 / 2 + 1;
  memcpy(g->rvecs, rvecs, 9 * sizeof(double));
  int N[3] = {n1, n2, n3};
  for (int a = 0; a < 3; ++a) {
    double c0 = rvecs[0 * 3 + a], c1 = rvecs[1 * 3 + a], c2 = rvecs[2 * 3 + a];
    g->spacing[a] = sqrt(c0 * c0 + c1 * c1 + c2 * c2) / N[a];  // column norms (system.py:262-266)
  }
  {
    const double* r = rvecs;
    double det = r[0] * (r[4] * r[8] - r[5] * r[7]) - r[1] * (r[3] * r[8] - r[5] * r[6]) +
                 r[2] * (r[3] * r[7] - r[4] * r[6]);
    g->volume = fabs(det);
  }
  if (!factorise(n1, &g->ax1, order[0]) || !factorise(n2, &g->ax2, order[1]) ||
      !factorise(zfull ? n3 : g->m3, &g->ax3, order[2])) {
    free(g);
    return CMM_ERR_SHAPE;
  }
  for (int a = 0; a < 3; ++a) g->order[a] = order[a];
  // the compile-time-length kernels (x 32 / 64, plane 32x16 / 64x32) fix
  // their own radix order: any other order takes the run-time kernels
  g->generic = (order[0] | order[1] | order[2]) != CMM_ORDER_DEFAULT;
  g->staging = staging;
  g->col_tile = tile;
  const int m3 = g->m3, h3 = g->h3;
  g->hpos_k1 = (int*)malloc(sizeof(int) * n1);
  g->hpos_k2 = (int*)malloc(sizeof(int) * n2);
  g->hpos_k3 = (int*)malloc(sizeof(int) * h3);
  // zpos: position of frequency k in the z transform's DIF output (k < m3
  // for even N3; k < N3 for odd N3, whose h3 stored frequencies are kept in
  // natural order: position p holds k = p).
  const int nz = zfull ? n3 : m3;
  std::vector<int> zdif(nz), zpos(nz);
  dif_positions(g->ax1, g->hpos_k1);
  dif_positions(g->ax2, g->hpos_k2);
  dif_positions(g->ax3, zdif.data());
  for (int p = 0; p < nz; ++p) zpos[zdif[p]] = p;
  if (zfull) {
    for (int p = 0; p < h3; ++p) g->hpos_k3[p] = p;
  } else {
    for (int p = 0; p < m3; ++p) g->hpos_k3[p] = zdif[p];
    g->hpos_k3[m3] = m3;
  }

  std::vector<double> tw1, tw2, tw3;
  twiddles(n1, tw1); twiddles(n2, tw2); twiddles(n3, tw3);

  // per-position k tables
  std::vector<double> kp[3], sl[3], wt3(h3);
  std::vector<int> nq[3];
  const int* kof[3] = {g->hpos_k1, g->hpos_k2, g->hpos_k3};
  int npos[3] = {n1, n2, h3};
  for (int a = 0; a < 3; ++a) {
    kp[a].resize(npos[a]); sl[a].resize(npos[a]); nq[a].resize(npos[a]);
    const double d = g->spacing[a];
    const double val = 1.0 / (N[a] * d);
    const double twopi = 2.0 * M_PI;
    const double kcut = 2.0 * M_PI / d;
    for (int p = 0; p < npos[a]; ++p) {
      int k = kof[a][p];
      int m = signed_freq(k, N[a]);
      volatile double f = (double)m * val;
      volatile double kk = twopi * f;
      kp[a][p] = kk;
      sl[a][p] = np_sinc(kk / kcut);
      nq[a][p] = (N[a] % 2 == 0 && k == N[a] / 2) ? 1 : 0;
    }
  }
  for (int p = 0; p < h3; ++p) {
    int k = g->hpos_k3[p];
    wt3[p] = (k == 0 || (!zfull && k == m3)) ? 1.0 : 2.0;  // Parseval weight of a stored frequency
  }

  // one device block for everything
  size_t off = 0;
  auto bump = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~(size_t)255; return o; };
  size_t o_tw1 = bump(sizeof(double) * tw1.size()), o_tw2 = bump(sizeof(double) * tw2.size()),
         o_tw3 = bump(sizeof(double) * tw3.size()), o_zpos = bump(sizeof(int) * nz),
         o_k1 = bump(sizeof(int) * n1);
  size_t o_kp[3], o_sl[3], o_nq[3];
  for (int a = 0; a < 3; ++a) {
    o_kp[a] = bump(sizeof(double) * npos[a]);
    o_sl[a] = bump(sizeof(double) * npos[a]);
    o_nq[a] = bump(sizeof(int) * npos[a]);
  }
  size_t o_wt3 = bump(sizeof(double) * h3);
  // Rader tables: per axis an array of nstage RaderTab (M = 0 for other
  // stages) followed by the tables of each Rader stage.
  FftAxis* axes[3] = {&g->ax1, &g->ax2, &g->ax3};
  std::vector<RaderHost> rh[3];
  size_t o_rt[3] = {0, 0, 0};
  std::vector<std::vector<size_t>> o_rs(3);
  for (int a = 0; a < 3; ++a) {
    const FftAxis& ax = *axes[a];
    rh[a].resize(ax.nstage);
    bool any = false;
    std::vector<bool> use(ax.nstage, false);
    for (int st = 0; st < ax.nstage; ++st)
      if (ax.radix[st] > CMM_MAX_SMALL_RADIX && rader_plan(ax.radix[st], rh[a][st])) use[st] = any = true;
    if (!any) continue;
    o_rt[a] = bump(sizeof(RaderTab) * ax.nstage);
    o_rs[a].assign(ax.nstage, 0);
    for (int st = 0; st < ax.nstage; ++st)
      if (use[st]) {
        const size_t M = ax.radix[st] - 1;
        o_rs[a][st] = bump(3 * sizeof(double2) * M + 2 * sizeof(int) * M);
      }
  }
  // kernels instantiated with -1 (odd radices 7, 11, 13 and Rader stages)
  g->exotic = 0;
  for (int a = 0; a < 3; ++a)
    for (int st = 0; st < axes[a]->nstage; ++st) {
      const int r = axes[a]->radix[st];
      if (r == 7 || r == 11 || r == 13 || (!o_rs[a].empty() && o_rs[a][st])) g->exotic = 1;
    }
  std::vector<char> host(off);
  memcpy(&host[o_tw1], tw1.data(), sizeof(double) * tw1.size());
  memcpy(&host[o_tw2], tw2.data(), sizeof(double) * tw2.size());
  memcpy(&host[o_tw3], tw3.data(), sizeof(double) * tw3.size());
  memcpy(&host[o_zpos], zpos.data(), sizeof(int) * nz);
  memcpy(&host[o_k1], g->hpos_k1, sizeof(int) * n1);
  for (int a = 0; a < 3; ++a) {
    memcpy(&host[o_kp[a]], kp[a].data(), sizeof(double) * npos[a]);
    memcpy(&host[o_sl[a]], sl[a].data(), sizeof(double) * npos[a]);
    memcpy(&host[o_nq[a]], nq[a].data(), sizeof(int) * npos[a]);
  }
  memcpy(&host[o_wt3], wt3.data(), sizeof(double) * h3);
  if (cudaMalloc(&g->dmem, off) != cudaSuccess) {
    free(g->hpos_k1); free(g->hpos_k2); free(g->hpos_k3); free(g);
    return CMM_ERR_NOMEM;
  }
  for (int a = 0; a < 3; ++a) {
    if (o_rs[a].empty()) continue;
    FftAxis& ax = *axes[a];
    char* dbase = (char*)g->dmem;
    for (int st = 0; st < ax.nstage; ++st) {
      RaderTab rt;
      memset(&rt, 0, sizeof(rt));
      if (o_rs[a][st]) {
        const RaderHost& h = rh[a][st];
        const size_t M = ax.radix[st] - 1, o = o_rs[a][st];
        rt.axm = h.axm;
        rt.M = (int)M;
        const size_t o_twm = o, o_kf = o + sizeof(double2) * M, o_ki = o + 2 * sizeof(double2) * M,
                     o_gin = o + 3 * sizeof(double2) * M, o_gout = o_gin + sizeof(int) * M;
        memcpy(&host[o_twm], h.twm.data(), sizeof(double2) * M);
        memcpy(&host[o_kf], h.kf.data(), sizeof(double2) * M);
        memcpy(&host[o_ki], h.ki.data(), sizeof(double2) * M);
        memcpy(&host[o_gin], h.gin.data(), sizeof(int) * M);
        memcpy(&host[o_gout], h.gout.data(), sizeof(int) * M);
        rt.twm = (const double2*)(dbase + o_twm);
        rt.kf = (const double2*)(dbase + o_kf);
        rt.ki = (const double2*)(dbase + o_ki);
        rt.gin = (const int*)(dbase + o_gin);
        rt.gout = (const int*)(dbase + o_gout);
      }
      memcpy(&host[o_rt[a] + sizeof(RaderTab) * st], &rt, sizeof(rt));
    }
    ax.rader = (const RaderTab*)(dbase + o_rt[a]);
  }
  if (cudaMemcpy(g->dmem, host.data(), off, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(g->dmem);
    free(g->hpos_k1); free(g->hpos_k2); free(g->hpos_k3); free(g);
    return CMM_ERR_CUDA;
  }
  char* b = (char*)g->dmem;
  GridDev& d = g->dev;
  d.n1 = n1; d.n2 = n2; d.n3 = n3; d.h3 = h3; d.m3 = m3;
  d.zfull = zfull;
  d.ax1 = g->ax1; d.ax2 = g->ax2; d.ax3 = g->ax3;
  d.tw1 = (const double2*)(b + o_tw1);
  d.tw2 = (const double2*)(b + o_tw2);
  d.tw3 = (const double2*)(b + o_tw3);
  d.zpos = (const int*)(b + o_zpos);
  d.k1pos = (const int*)(b + o_k1);
  d.kp1 = (const double*)(b + o_kp[0]); d.kp2 = (const double*)(b + o_kp[1]); d.kp3 = (const double*)(b + o_kp[2]);
  d.sl1 = (const double*)(b + o_sl[0]); d.sl2 = (const double*)(b + o_sl[1]); d.sl3 = (const double*)(b + o_sl[2]);
  d.nq1 = (const int*)(b + o_nq[0]); d.nq2 = (const int*)(b + o_nq[1]); d.nq3 = (const int*)(b + o_nq[2]);
  d.wt3 = (const double*)(b + o_wt3);
  *out = g;
  return CMM_OK;
}

extern "C" int cmm_grid_destroy(cmm_grid* g) {
  if (!g) return CMM_OK;
  if (g->dmem) cudaFree(g->dmem);
  free(g->hpos_k1); free(g->hpos_k2); free(g->hpos_k3);
  free(g);
  return CMM_OK;
}

extern "C" int cmm_grid_set_staging(cmm_grid* g, int mode) {
  if (!g || mode < 0 || mode > 2) return CMM_ERR_ARG;
  g->staging = mode;
  return CMM_OK;
}

extern "C" int cmm_grid_schedule(const cmm_grid* g, int* sched, int* radices) {
  if (!g || !sched) return CMM_ERR_ARG;
  for (int a = 0; a < 3; ++a) sched[a] = g->order[a];
  sched[3] = g->staging;
  sched[4] = g->col_tile;
  if (radices) {
    const FftAxis* ax[3] = {&g->ax1, &g->ax2, &g->ax3};
    for (int a = 0; a < 3; ++a)
      for (int st = 0; st < CMM_MAX_STAGES; ++st) radices[a * CMM_MAX_STAGES + st] = st < ax[a]->nstage ? ax[a]->radix[st] : 0;
  }
  return CMM_OK;
}

extern "C" int cmm_grid_spectrum_size(const cmm_grid* g, long long* nspec, int* h3) {
  if (!g) return CMM_ERR_ARG;
  if (nspec) *nspec = (long long)g->n1 * g->n2 * g->h3;
  if (h3) *h3 = g->h3;
  return CMM_OK;
}

extern "C" int cmm_spectrum_index(const cmm_grid* g, int* k1, int* k2, int* k3) {
  if (!g || !k1 || !k2 || !k3) return CMM_ERR_ARG;
  // spectra in HBM keep x natural (the column passes undo their own x order)
  for (int i = 0; i < g->n1; ++i) k1[i] = i;
  memcpy(k2, g->hpos_k2, sizeof(int) * g->n2);
  memcpy(k3, g->hpos_k3, sizeof(int) * g->h3);
  return CMM_OK;
}
