// Native batched solve: the control flow of Solver._solve with the Picard
// hybrid and (hybrid-)Anderson updates (cmmdft/solver.py:236-345, 403-457,
// 515-604) for a batch of chemical potentials on one functional.
//
// The GPU work is the same sequence of C-ABI calls the Python driver
// (cmmdft_b200/batch.py, BatchSolve) issues; the per-instance decisions
// between read-backs (Anderson coefficients, line-search fit, convergence)
// are evaluated here in C++ with the same arithmetic, so that a decision
// point costs microseconds of host time instead of an interpreter round.
// Host arithmetic follows the Python expressions operation by operation
// (IEEE double, no contraction on the host).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include <math_constants.h>

#include "cmm_common.cuh"

// SLSQP mixing coefficients (cmm_anderson.cu)
int anderson_slsqp(const double* G, int n, double* x, int* nit_out);

namespace {

constexpr int NST = CMM_NSTAT;
constexpr int NLS = CMM_NLS;
constexpr int MAXF = CMM_MAX_FIELDS;
constexpr int NSTAGE = 32;   // pinned upload slots (several uploads between two read-backs)
constexpr int CLIP_NONE = CMM_CLIP_NONE, CLIP_DENSITY = CMM_CLIP_DENSITY;
constexpr double LS_COEF[3] = {0.45, 0.9, 0.225};   // trial alphas / alpha_max (solver.py:414-423)
constexpr int GRID_N = 10000;                       // np.linspace(-max/4, max, 10000) (solver.py:426)

size_t stage_slot_bytes(int B) {
  size_t b = sizeof(int) * (size_t)B + sizeof(double) * (size_t)B * (MAXF + 4);
  return (b + 255) & ~(size_t)255;
}

// a_i >= 0, sum a_i = 1 minimiser of a^T M a over all supports of n <= 8
// variables (batch.simplex_qp_batched for one Gram matrix): the bordered
// system [M_SS 1; 1^T 0][a; lam] = [0; 1] per support (partial-pivot LU;
// singular systems fall back to least squares through the normal equations
// of the bordered matrix), lowest objective, ties within 1e-14 to the first
// support in enumeration order (bit k of the support index = variable k).
void simplex_qp(const double* M, int n, double* best) {
  double scale = 0.0;
  for (int i = 0; i < n; ++i) scale = std::fmax(scale, std::fabs(M[i * n + i]));
  scale = std::fmax(scale, 1e-300);
  double Ms[64];
  for (int i = 0; i < n * n; ++i) Ms[i] = M[i] / scale;
  const int K = (1 << n) - 1, N = n + 1;
  std::vector<double> vals(K), as((size_t)K * n);
  std::vector<char> ok(K);
  for (int k = 0; k < K; ++k) {
    const unsigned S = (unsigned)(k + 1);
    double A[81], x[9];
    for (int i = 0; i < N * N; ++i) A[i] = 0.0;
    for (int i = 0; i < n; ++i) {
      const bool si = (S >> i) & 1u;
      for (int j = 0; j < n; ++j) {
        const bool sj = (S >> j) & 1u;
        A[i * N + j] = (si && sj) ? Ms[i * n + j] : 0.0;
      }
      if (!si) A[i * N + i] = 1.0;
      A[i * N + n] = si ? 1.0 : 0.0;
      A[n * N + i] = si ? 1.0 : 0.0;
    }
    for (int i = 0; i < N; ++i) x[i] = (i == n) ? 1.0 : 0.0;
    // Gaussian elimination with partial pivoting (LAPACK getrf/getrs order)
    double LU[81];
    std::memcpy(LU, A, sizeof(double) * N * N);
    int piv[9];
    bool singular = false;
    for (int c = 0; c < N; ++c) {
      int p = c;
      double mx = std::fabs(LU[c * N + c]);
      for (int r = c + 1; r < N; ++r)
        if (std::fabs(LU[r * N + c]) > mx) { mx = std::fabs(LU[r * N + c]); p = r; }
      piv[c] = p;
      if (mx == 0.0) { singular = true; break; }
      if (p != c)
        for (int j = 0; j < N; ++j) std::swap(LU[c * N + j], LU[p * N + j]);
      for (int r = c + 1; r < N; ++r) {
        const double f = LU[r * N + c] / LU[c * N + c];
        LU[r * N + c] = f;
        for (int j = c + 1; j < N; ++j) LU[r * N + j] -= f * LU[c * N + j];
      }
    }
    if (!singular) {
      for (int c = 0; c < N; ++c)
        if (piv[c] != c) std::swap(x[c], x[piv[c]]);
      for (int r = 1; r < N; ++r)
        for (int j = 0; j < r; ++j) x[r] -= LU[r * N + j] * x[j];
      for (int r = N - 1; r >= 0; --r) {
        for (int j = r + 1; j < N; ++j) x[r] -= LU[r * N + j] * x[j];
        x[r] /= LU[r * N + r];
      }
    } else {
      // minimum-norm least squares through A^T A (+ tiny ridge) for a singular support
      double AtA[81], Atb[9];
      for (int i = 0; i < N; ++i) {
        Atb[i] = A[n * N + i];   // b = e_n
        for (int j = 0; j < N; ++j) {
          double s = 0.0;
          for (int r = 0; r < N; ++r) s += A[r * N + i] * A[r * N + j];
          AtA[i * N + j] = s + (i == j ? 1e-14 : 0.0);
        }
      }
      // Cholesky
      bool fail = false;
      for (int i = 0; i < N && !fail; ++i)
        for (int j = 0; j <= i; ++j) {
          double s = AtA[i * N + j];
          for (int q = 0; q < j; ++q) s -= AtA[i * N + q] * AtA[j * N + q];
          if (i == j) {
            if (!(s > 0.0)) { fail = true; break; }
            AtA[i * N + i] = std::sqrt(s);
          } else {
            AtA[i * N + j] = s / AtA[j * N + j];
          }
        }
      if (fail) {
        for (int i = 0; i < N; ++i) x[i] = NAN;
      } else {
        for (int i = 0; i < N; ++i) {
          double s = Atb[i];
          for (int q = 0; q < i; ++q) s -= AtA[i * N + q] * x[q];
          x[i] = s / AtA[i * N + i];
        }
        for (int i = N - 1; i >= 0; --i) {
          double s = x[i];
          for (int q = i + 1; q < N; ++q) s -= AtA[q * N + i] * x[q];
          x[i] = s / AtA[i * N + i];
        }
      }
    }
    double* a = &as[(size_t)k * n];
    bool good = true;
    double sum = 0.0;
    for (int i = 0; i < n; ++i) {
      a[i] = ((S >> i) & 1u) ? x[i] : 0.0;
      if (!std::isfinite(a[i])) good = false;
      if (a[i] < -1e-12) good = false;
    }
    for (int i = 0; i < n; ++i) {
      double v = std::isfinite(a[i]) ? a[i] : (std::isnan(a[i]) ? 0.0 : (a[i] > 0 ? 1.7976931348623157e308 : -1.7976931348623157e308));
      a[i] = v < 0.0 ? 0.0 : v;
      sum += a[i];
    }
    const double d = std::fmax(sum, 1e-300);
    for (int i = 0; i < n; ++i) a[i] /= d;
    double val = 0.0;
    for (int i = 0; i < n; ++i) {
      double t = 0.0;
      for (int j = 0; j < n; ++j) t += Ms[i * n + j] * a[j];
      val += a[i] * t;
    }
    ok[k] = good;
    vals[k] = good ? val : INFINITY;
  }
  double vmin = INFINITY;
  for (int k = 0; k < K; ++k) vmin = std::fmin(vmin, vals[k]);
  if (!std::isfinite(vmin)) {
    for (int i = 0; i < n; ++i) best[i] = 1.0 / n;
    return;
  }
  for (int k = 0; k < K; ++k)
    if (vals[k] <= vmin + 1e-14) {
      for (int i = 0; i < n; ++i) best[i] = as[(size_t)k * n + i];
      return;
    }
}

// np.argmin over the grid points js (the first NaN, if any, else the first
// minimum) and np.max (NaN if any value is NaN).
void grid_eval(double a0, double b, double c, double lo, double step, double hi, const long long* js, int nj,
               double* aopt, double* mn, double* mx) {
  auto alpha = [&](long long j) { return (j == GRID_N - 1) ? hi : (double)j * step + lo; };
  int best = -1, firstnan = -1;
  double bv = 0.0, vmax = -INFINITY;
  for (int q = 0; q < nj; ++q) {
    const double al = alpha(js[q]);
    const double om = a0 + b * al + c * (al * al);
    if (std::isnan(om)) {
      if (firstnan < 0) firstnan = q;
      continue;
    }
    if (best < 0 || om < bv) { best = q; bv = om; }
    vmax = std::fmax(vmax, om);
  }
  if (firstnan >= 0) {
    *aopt = alpha(js[firstnan]);
    *mn = NAN;
    *mx = NAN;
    return;
  }
  *aopt = alpha(js[best]);
  *mn = bv;
  *mx = vmax;
}

// batch.grid_parabola for one row: exact against evaluating all GRID_N points.
void grid_parabola(double c, double b, double a0, double hi, double* aopt, double* mn, double* mx) {
  const int n = GRID_N;
  const double lo = -hi / 4;
  const double step = (hi - lo) / (n - 1);
  const double eps = 2.220446049250313e-16;
  const double vert = -b / (2 * c);
  const double scale = std::fmax(std::fabs(a0), std::fabs(a0 + b * vert + c * vert * vert));
  const double W = std::ceil(std::sqrt(64 * eps * scale / c) / step) + 2;
  const bool fast = (c > 0) && std::isfinite(W) && (W < n / 4) && (step > 0) && std::isfinite(vert);
  std::vector<long long> js;
  if (fast) {
    double jv = std::floor((vert - lo) / step);
    jv = std::fmin(std::fmax(jv, 0.0), (double)(n - 1));
    const long long w = (long long)W;
    js.push_back(0);
    for (long long o = -w; o <= w; ++o) {
      long long j = (long long)jv + o;
      j = j < 0 ? 0 : (j > n - 1 ? n - 1 : j);
      js.push_back(j);
    }
    js.push_back(n - 1);
    std::sort(js.begin(), js.end());
  } else {
    js.resize(n);
    for (int j = 0; j < n; ++j) js[j] = j;
  }
  grid_eval(a0, b, c, lo, step, hi, js.data(), (int)js.size(), aopt, mn, mx);
}

bool isclose0(double a) { return std::fabs(a) <= 1e-8; }   // np.isclose(a, 0)

// A few host threads for per-instance work between two read-backs (the
// Anderson coefficients of every instance are independent).  run(n, f) calls
// f(i) for i < n on the workers and the calling thread and returns when all
// workers have checked in; items are claimed from one atomic counter.
// ------------------------------------------------ device-side static loop --
// Static Picard with the per-instance decisions on the device: one step is a
// fixed launch sequence (the Picard pass of each ring parity, the stats
// reduction, k_static_decide, the C1 pipeline) that a CUDA graph replays; the
// host reads one counter every few steps.  k_static_decide is the
// convergence / divergence / retry logic of Driver::loop_static evaluated per
// instance with the same operations in the same order (explicitly rounded,
// no contraction), so the trajectory and every reported number are those of
// the host loop.
struct StaticDev {
  int* live;       // [B] stepping
  int* act;        // [2][B] instances whose current density is in ring slot 0 / 1
  int* cur;        // [B] ring slot of the current density
  int* retry;      // [B] non-finite density: restart with a halved correction factor
  int* fin;        // [B] finished (converged, step limit or diverging)
  int* steps;      // [B]
  int* conv;       // [B]
  int* divg;       // [B]
  int* ctr;        // [0] step, [1] instances still stepping
  double* prev;    // [B][NST] the previous step's stats
  double* N;       // [B] loading at finish
  double* omega0;  // [B]
  double* res_hist;   // [B][nsteps + 2]
  double* history;    // [B][nsteps + 2][CMM_HISTORY_COLS] or null
};

struct StaticParams {
  int B, nsteps, ncrit, guard;
  int crit[3];
  double thr[3];
  double dr, npts;
};

__device__ bool dev_diverging(const double* r, int k, int guard) {
  if (!guard || k < 8) return false;
  const double last_r = r[k];
  if (!isfinite(last_r)) return true;
  double best = CUDART_NAN;
  for (int j = 1; j <= k; ++j)
    if (!isnan(r[j])) best = isnan(best) ? r[j] : fmin(best, r[j]);
  bool rising = true;
  for (int j = k - 4; j <= k; ++j) rising = rising && (__dsub_rn(r[j], r[j - 1]) >= 0);
  return last_r > __dmul_rn(1e6, best) && rising;
}

__global__ void k_static_decide(StaticParams P, const double* __restrict__ stats, StaticDev D) {
  const int step = D.ctr[0] + 1;
  __shared__ int nlive;
  if (threadIdx.x == 0) nlive = 0;
  __syncthreads();
  for (int b = threadIdx.x; b < P.B; b += blockDim.x) {
    const double* s = stats + (size_t)b * NST;
    double* pv = D.prev + (size_t)b * NST;
    if (D.live[b]) {
      bool done = false;
      if (step > 1) {
        const int k = step - 1;
        const double N = __dmul_rn(pv[CMM_STAT_N], P.dr);
        const double res = __ddiv_rn(__ddiv_rn(__dsqrt_rn(s[CMM_STAT_RES2]), __dsqrt_rn(N)), __dsqrt_rn(P.npts));
        const double iue = __dmul_rn(pv[CMM_STAT_IUE], P.dr);
        const double der = __ddiv_rn(__dsqrt_rn(s[CMM_STAT_DER]), __dsqrt_rn(P.npts));
        D.steps[b] = k;
        const double riue = (N > 0) ? __ddiv_rn(iue, N) : CUDART_NAN;
        bool ok = true;
        for (int c = 0; c < P.ncrit; ++c) {
          const double v = P.crit[c] == CMM_CRIT_RES ? res : (P.crit[c] == CMM_CRIT_RIUE ? riue : der);
          ok = ok && (v < P.thr[c]);
        }
        if (D.history && k <= P.nsteps + 1) {
          double* h = D.history + ((size_t)b * (P.nsteps + 2) + k) * CMM_HISTORY_COLS;
          h[0] = N; h[1] = res; h[2] = riue; h[3] = D.omega0[b]; h[4] = der;
        }
        if (iue == 0 && isnan(riue)) ok = true;
        double* rh = D.res_hist + (size_t)b * (P.nsteps + 2);
        if (k <= P.nsteps + 1) rh[k] = res;
        if (ok || k >= P.nsteps || dev_diverging(rh, k, P.guard)) {
          if (!ok) D.divg[b] = k < P.nsteps ? 1 : 0;
          D.conv[b] = ok ? 1 : 0;
          D.N[b] = N;
          D.fin[b] = 1;
          D.live[b] = 0;
          done = true;
        }
      }
      if (!done && s[CMM_STAT_NONFIN] > 0) {
        D.retry[b] = 1;
        D.live[b] = 0;
        done = true;
      }
      if (!done) {
        D.cur[b] = 1 - D.cur[b];
        atomicAdd(&nlive, 1);
      }
    }
    D.act[b] = D.live[b] && D.cur[b] == 0;
    D.act[P.B + b] = D.live[b] && D.cur[b] == 1;
    for (int q = 0; q < NST; ++q) pv[q] = s[q];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    D.ctr[0] = step;
    D.ctr[1] = nlive;
  }
}

class HostPool {
 public:
  explicit HostPool(int nthreads) {
    try {
      for (int i = 0; i < nthreads; ++i) th_.emplace_back([this] { worker(); });
    } catch (...) {
      shutdown();   // threads already started are joined before the error propagates
      throw;
    }
  }
  ~HostPool() { shutdown(); }
  void shutdown() {
    {
      std::lock_guard<std::mutex> l(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_)
      if (t.joinable()) t.join();
  }
  void run(int n, const std::function<void(int)>& f) {
    if (th_.empty() || n < 4) {
      for (int i = 0; i < n; ++i) f(i);
      return;
    }
    {
      std::lock_guard<std::mutex> l(m_);
      job_ = &f;
      n_ = n;
      next_.store(0);
      pending_ = (int)th_.size();
      ++gen_;
    }
    cv_.notify_all();
    for (int i; (i = next_.fetch_add(1)) < n;) f(i);
    std::unique_lock<std::mutex> l(m_);
    done_.wait(l, [this] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  void worker() {
    long seen = 0;
    for (;;) {
      const std::function<void(int)>* job;
      int n;
      {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
        job = job_;
        n = n_;
      }
      for (int i; (i = next_.fetch_add(1)) < n;) (*job)(i);
      std::lock_guard<std::mutex> l(m_);
      if (--pending_ == 0) done_.notify_one();
    }
  }
  std::vector<std::thread> th_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  const std::function<void(int)>* job_ = nullptr;
  int n_ = 0, pending_ = 0;
  long gen_ = 0;
  bool stop_ = false;
  std::atomic<int> next_{0};
};

struct Driver {
  const cmm_functional_desc* fn;
  const cmm_solve_opts* o;
  int B;
  const cmm_solve_ws* w;
  cmm_solve_out* out;
  cmm_fallback_fn fb;
  void* fbctx;
  cudaStream_t st;
  const cmm_grid* g;
  size_t npts, S;
  int nwd, m;
  double dr, beta;
  bool wda, anderson, pure, statik = false;
  const double *mu, *fug;
  std::vector<double> cf;
  std::vector<char> failed, And_true;
  std::vector<int> ls_slot;
  std::vector<double> omega0, n3max, Ncur, last, gram, rnorm2, it_eps0, damping, ls_host, alpha_host, res_hist;
  std::vector<double> stats_h, ls_h, alpha_h;
  size_t slot_bytes;
  int stage_i = 0;
  int rc = CMM_OK;
  cudaStream_t copy_st = nullptr;        // side stream of the host copies of finished densities
  std::vector<cudaEvent_t> copy_ev;
  std::vector<char> wd_ok;               // [B][m]: weighted densities of ring slot s stored
  struct PipeRec { cudaEvent_t a, b; int want, nact; };
  std::vector<PipeRec> pipe;             // timed full pipeline launches (out->pipe_log)
  std::vector<char> act_now;             // the active mask last uploaded
  std::unique_ptr<HostPool> pool;        // SLSQP coefficients of several instances at once

  double* ring(int s) const { return w->ring + (size_t)s * B * npts; }
  double* rres(int s) const { return w->rres + (size_t)s * B * npts; }
  double* spec_ring(int s) const { return w->spec_ring + (size_t)s * B * S; }
  double* wd_ring(int s) const { return w->wd_ring + (size_t)s * nwd * B * npts; }

  char* stage() {
    char* p = (char*)w->h_stage + (size_t)stage_i * slot_bytes;
    stage_i = (stage_i + 1) % NSTAGE;
    return p;
  }
  bool check(int r) {
    if (r != CMM_OK && rc == CMM_OK) rc = r;
    return rc == CMM_OK;
  }
  bool cuda(cudaError_t e) { return check(e == cudaSuccess ? CMM_OK : CMM_ERR_CUDA); }

  void set_active(const std::vector<char>& mask) {
    act_now = mask;
    int* h = (int*)stage();
    for (int b = 0; b < B; ++b) h[b] = mask[b] ? 1 : 0;
    cuda(cudaMemcpyAsync(w->active, h, sizeof(int) * B, cudaMemcpyHostToDevice, st));
  }
  // params[b] = (fugacity, Picard mixing a, mu, max n3 of the current density)
  void set_params(const double* n3, const double* a = nullptr) {
    double* h = (double*)stage();
    for (int b = 0; b < B; ++b) {
      h[b * 4 + 0] = fug[b];
      h[b * 4 + 1] = a ? a[b] : 0.0;
      h[b * 4 + 2] = mu[b];
      h[b * 4 + 3] = n3 ? n3[b] : 0.0;
    }
    cuda(cudaMemcpyAsync(w->params, h, sizeof(double) * B * 4, cudaMemcpyHostToDevice, st));
  }
  void mix(const std::vector<double>& coefs /*B x MAXF*/, const std::vector<const double*>& fields, int clip,
           const double* ref, double* dst, double* spec_out) {
    double* h = (double*)stage();
    std::memcpy(h, coefs.data(), sizeof(double) * B * MAXF);
    cuda(cudaMemcpyAsync(w->coef, h, sizeof(double) * B * MAXF, cudaMemcpyHostToDevice, st));
    long long fstride[MAXF];
    for (int j = 0; j < MAXF; ++j) fstride[j] = (long long)npts;
    check(cmm_mix_step(g, B, w->active, w->coef, fields.data(), fstride, (int)fields.size(), clip, 0.0, fn->lambda3,
                       ref, (long long)npts, fn->d_V, 0, dst, spec_out, w->part, w->nslot, st));
    out->launches += 1;
  }
  void c1(const double* spec, double* chat, int want, double* wd) {
    PipeRec r{nullptr, nullptr, want, 0};
    const bool timed = out->pipe_log && (want & 1) && (int)pipe.size() < out->pipe_cap;
    if (timed) {
      cuda(cudaEventCreate(&r.a));
      cuda(cudaEventCreate(&r.b));
      cuda(cudaEventRecord(r.a, st));
      for (int b = 0; b < B; ++b) r.nact += act_now.size() == (size_t)B && act_now[b] ? 1 : 0;
    }
    check(cmm_fmt_c1(g, B, w->active, fn->R, fn->beta, fn->version, fn->wda, fn->d_kst, fn->d_wtab, spec, chat,
                     w->work, w->part, w->nslot, want, wd, st));
    if (timed) {
      cuda(cudaEventRecord(r.b, st));
      pipe.push_back(r);
    }
    out->launches += (want & 1) ? 3 : 2;
  }
  void residual(const double* chat, const double* rho, double* r_out, const std::vector<int>& hist) {
    const double* hp[CMM_MAX_HIST];
    for (size_t h = 0; h < hist.size(); ++h) hp[h] = rres(hist[h]);
    check(cmm_residual_step(g, B, w->active, w->params, beta, fn->lambda3, o->a_tol, o->r_tol, chat, rho, fn->d_V, 0,
                            r_out, hist.empty() ? nullptr : hp, (int)hist.size(), (long long)npts, w->part, w->nslot,
                            st));
    out->launches += 1;
  }
  void finalize() {
    check(cmm_stats_finalize(B, w->active, w->part, w->nslot, (1u << NST) - 1u, w->stats, st));
    out->launches += 1;
  }
  void launch_ls(const std::vector<char>& mask, int s, const double* n3a, long long n3s) {
    set_active(mask);
    check(cmm_ls_prepare(g, B, w->active, fn->R, fn->version, fn->wda, fn->d_kst, fn->d_wtab, rres(s), spec_ring(s),
                         wd_ring(s), w->rhat, w->work, w->wd_r, w->ls_part, w->nslot, st));
    check(cmm_ls_omega(g, B, w->active, n3a, n3s, LS_COEF[0], LS_COEF[1], LS_COEF[2], fn->R, fn->lambda3,
                       fn->version, fn->wda, ring(s), rres(s), fn->d_V, 0, wd_ring(s), w->wd_r, w->ls_part, w->nslot,
                       w->ls_alpha, st));
    check(cmm_ls_finalize(B, w->active, w->ls_part, w->nslot, w->ls, st));
    out->launches += 6;
  }
  // one read-back: the finalized stats and/or the line-search sums
  void read(bool stats, bool ls) {
    if (stats) cuda(cudaMemcpyAsync(w->h_stats, w->stats, sizeof(double) * B * NST, cudaMemcpyDeviceToHost, st));
    if (ls) {
      cuda(cudaMemcpyAsync(w->h_ls, w->ls, sizeof(double) * B * NLS, cudaMemcpyDeviceToHost, st));
      cuda(cudaMemcpyAsync(w->h_alpha, w->ls_alpha, sizeof(double) * B, cudaMemcpyDeviceToHost, st));
    }
    cuda(cudaStreamSynchronize(st));
    if (stats) std::memcpy(stats_h.data(), w->h_stats, sizeof(double) * B * NST);
    if (ls) {
      std::memcpy(ls_h.data(), w->h_ls, sizeof(double) * B * NLS);
      std::memcpy(alpha_h.data(), w->h_alpha, sizeof(double) * B);
    }
  }
  void keep_ls(const std::vector<char>& mask, int s) {
    for (int b = 0; b < B; ++b)
      if (mask[b]) {
        std::memcpy(&ls_host[(size_t)b * NLS], &ls_h[(size_t)b * NLS], sizeof(double) * NLS);
        alpha_host[b] = alpha_h[b];
        ls_slot[b] = s;
      }
  }

  // _omega (batch.py): grand potential from a stats row
  double omega(const double* s, int b) const {
    const double N = s[CMM_STAT_N] * dr;
    double G = (s[CMM_STAT_FID] * dr) / beta - mu[b] * N;
    G += (s[CMM_STAT_PHI] * dr) / beta;
    G += 0.5 * (s[CMM_STAT_MFA] * dr);
    G += s[CMM_STAT_FEXT] * dr;
    if (wda) G += s[CMM_STAT_WDA] * dr;
    return G;
  }
  // _ls_omega_rows: Omega(rho + alpha r) from the line-search sums
  double ls_omega(int b, int i, double alpha) const {
    const double* s = &last[(size_t)b * NST];
    const double* l = &ls_host[(size_t)b * NLS];
    const double N = (s[CMM_STAT_N] + alpha * l[CMM_LS_SUM_R]) * dr;
    double G = (l[CMM_LS_FID + i] * dr) / beta - mu[b] * N;
    G += (l[CMM_LS_PHI + i] * dr) / beta;
    G += 0.5 * ((s[CMM_STAT_MFA] + 2 * alpha * l[CMM_LS_MFA_XR] + alpha * alpha * l[CMM_LS_MFA_RR]) * dr);
    G += (s[CMM_STAT_FEXT] + alpha * l[CMM_LS_SUM_RV]) * dr;
    if (wda) G += l[CMM_LS_WDA + i] * dr;
    return G;
  }

  std::vector<int> valid_hist(int k_new) const {
    std::vector<int> h;
    for (int j = std::max(0, k_new - m + 1); j < k_new; ++j) h.push_back(j % m);
    return h;
  }

  // C1, Omega ingredients and residual of the density in ring slot s_new.
  // The weighted densities are stored while an instance of `mask` can still
  // take a hybrid step; later they are regenerated only if needed.
  std::vector<int> post_update(const std::vector<char>& mask, int k, int s_new, const std::vector<char>* ahead) {
    bool need = false;
    for (int b = 0; b < B; ++b) need = need || (mask[b] && !And_true[b]);
    c1(spec_ring(s_new), w->chat2, 1 | 2 | 4 | (need ? 8 : 0), need ? wd_ring(s_new) : nullptr);
    for (int b = 0; b < B; ++b)
      if (mask[b]) wd_ok[(size_t)b * m + s_new] = need ? 1 : 0;
    std::vector<int> hist = valid_hist(k);
    residual(w->chat2, ring(s_new), rres(s_new), hist);
    finalize();
    bool any = false;
    if (ahead)
      for (int b = 0; b < B; ++b) any |= (*ahead)[b] != 0;
    if (any) {
      launch_ls(*ahead, s_new, w->stats + CMM_STAT_N3MAX, NST);
      read(true, true);
      keep_ls(*ahead, s_new);
    } else {
      read(true, false);
    }
    return hist;
  }

  void commit(const std::vector<char>& mask, int s_new, const std::vector<int>& hist) {
    for (int b = 0; b < B; ++b) {
      if (!mask[b]) continue;
      const double* s = &stats_h[(size_t)b * NST];
      double* G = &gram[(size_t)b * m * m];
      rnorm2[(size_t)b * m + s_new] = s[CMM_STAT_RES2];
      G[s_new * m + s_new] = s[CMM_STAT_RES2];
      for (size_t h = 0; h < hist.size(); ++h) {
        const double v = s[CMM_STAT_GRAM0 + h];
        G[s_new * m + hist[h]] = v;
        G[hist[h] * m + s_new] = v;
      }
      n3max[b] = s[CMM_STAT_N3MAX];
      std::memcpy(&last[(size_t)b * NST], s, sizeof(double) * NST);
    }
  }

  void init_state(const std::vector<char>& todo) {
    set_active(todo);
    std::vector<double> coefs((size_t)B * MAXF, 0.0);
    for (int b = 0; b < B; ++b) coefs[(size_t)b * MAXF] = 1.0;
    if (statik) {  // the density's spectrum lives in `that`; no line search
      mix(coefs, {w->rho0}, CLIP_NONE, w->rho0, ring(0), w->that);
      c1(w->that, w->chat2, 1 | 2 | 4, nullptr);
    } else {
      mix(coefs, {w->rho0}, CLIP_NONE, w->rho0, ring(0), spec_ring(0));
      c1(spec_ring(0), w->chat2, 1 | 2 | 4 | 8, wd_ring(0));
    }
    finalize();
    read(true, false);
    cuda(cudaMemcpyAsync(w->chat, w->chat2, sizeof(double) * B * S, cudaMemcpyDeviceToDevice, st));
    for (int b = 0; b < B; ++b) {
      const double* s = &stats_h[(size_t)b * NST];
      omega0[b] = omega(s, b);
      n3max[b] = s[CMM_STAT_N3MAX];
      Ncur[b] = s[CMM_STAT_N] * dr;
      std::memcpy(&last[(size_t)b * NST], s, sizeof(double) * NST);
    }
    std::fill(wd_ok.begin(), wd_ok.end(), 0);
    for (int b = 0; b < B; ++b) wd_ok[(size_t)b * m] = todo[b];
  }

  void finish(int b, int s, double N, int k, bool conv) {
    cuda(cudaMemcpyAsync(w->result + (size_t)b * npts, ring(s) + (size_t)b * npts, sizeof(double) * npts,
                         cudaMemcpyDeviceToDevice, st));
    if (w->h_result && copy_st) {  // to the host while the other instances iterate
      cudaEvent_t ev;
      if (cuda(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming))) {
        copy_ev.push_back(ev);
        cuda(cudaEventRecord(ev, st));
        cuda(cudaStreamWaitEvent(copy_st, ev, 0));
        cuda(cudaMemcpyAsync(w->h_result + (size_t)b * npts, w->result + (size_t)b * npts, sizeof(double) * npts,
                             cudaMemcpyDeviceToHost, copy_st));
      }
    }
    out->N[b] = N;
    out->converged[b] = conv ? 1 : 0;
    out->steps[b] = k;
    out->omega[b] = omega0[b];
  }

  bool anderson_candidate(std::vector<char>& mask, int k, int s_prev, int s_new, std::vector<char>& ok) {
    const int mk = std::min(k, m);
    std::vector<int> slots;
    for (int j = k - mk; j < k; ++j) slots.push_back(j % m);
    std::vector<double> coefs((size_t)B * MAXF, 0.0);
    std::vector<int> todo;
    for (int b = 0; b < B; ++b)
      if (mask[b]) todo.push_back(b);
    std::vector<double> als((size_t)B * 8);
    auto coef_of = [&](int t) {
      const int b = todo[t];
      const double* G = &gram[(size_t)b * m * m];
      double Msub[64];
      for (int i = 0; i < mk; ++i)
        for (int j = 0; j < mk; ++j) Msub[i * mk + j] = G[slots[i] * m + slots[j]];
      double* al = &als[(size_t)b * 8];
      if (o->coefs == CMM_COEF_EXACT) simplex_qp(Msub, mk, al);
      else anderson_slsqp(Msub, mk, al, nullptr);   // update_rho_Anderson's SLSQP (solver.py:585-591)
    };
    if (pool) pool->run((int)todo.size(), coef_of);
    else for (int t = 0; t < (int)todo.size(); ++t) coef_of(t);
    for (int b : todo) {
      const double* al = &als[(size_t)b * 8];
      if (o->adaptive_damping) {  // _get_damping_coefficient (solver.py:537-544)
        const double r = std::sqrt(rnorm2[(size_t)b * m + s_prev]);
        const double p = (k >= 2) ? std::sqrt(rnorm2[(size_t)b * m + (k - 2) % m]) : 0.0;
        const double dm = damping[b];
        damping[b] = (r < p) ? std::fmin(dm * o->damping_up, o->damping_max)
                             : std::fmax(dm * o->damping_down, o->damping_min);
      }
      const double d = cf[b] * damping[b];
      for (int i = 0; i < mk; ++i) {
        coefs[(size_t)b * MAXF + i] = al[i];
        coefs[(size_t)b * MAXF + mk + i] = d * al[i];
      }
    }
    std::vector<const double*> fields;
    for (int s : slots) fields.push_back(ring(s));
    for (int s : slots) fields.push_back(rres(s));
    set_active(mask);
    for (int b = 0; b < B; ++b)
      if (mask[b] && ls_slot[b] == s_new) ls_slot[b] = -1;
    mix(coefs, fields, CLIP_DENSITY, ring(s_prev), ring(s_new), spec_ring(s_new));
    std::vector<int> hist = post_update(mask, k, s_new, nullptr);
    for (int b = 0; b < B; ++b) {
      ok[b] = 0;
      if (!mask[b]) continue;
      const double* s = &stats_h[(size_t)b * NST];
      if (s[CMM_STAT_GNONFIN] > 0) continue;
      const double om = omega(s, b);
      const double prev = omega0[b];
      omega0[b] = om;  // _get_Omega stores omega0 even when rejected
      out->omega_evals += 1;
      if (!(om > prev * 0.8)) ok[b] = 1;
    }
    commit(ok, s_new, hist);
    return rc == CMM_OK;
  }

  bool hybrid_step(const std::vector<char>& mask, int k, int s_prev, int s_new) {
    std::vector<double> prev(omega0);
    std::vector<char> fresh(B, 0);
    bool anyfresh = false;
    for (int b = 0; b < B; ++b) {
      fresh[b] = mask[b] && ls_slot[b] != s_prev;
      anyfresh |= fresh[b] != 0;
    }
    if (anyfresh) {
      std::vector<char> regen(B, 0);
      bool anyregen = false;
      for (int b = 0; b < B; ++b) {
        regen[b] = fresh[b] && !wd_ok[(size_t)b * m + s_prev];
        anyregen = anyregen || regen[b];
      }
      if (anyregen) {  // weighted densities of rho from its stored spectrum
        set_active(regen);
        c1(spec_ring(s_prev), nullptr, 8, wd_ring(s_prev));
        for (int b = 0; b < B; ++b)
          if (regen[b]) wd_ok[(size_t)b * m + s_prev] = 1;
      }
      set_params(n3max.data());
      launch_ls(fresh, s_prev, w->params + 3, 4);
      read(false, true);
      keep_ls(fresh, s_prev);
    }
    if (rc) return false;
    std::vector<double> aopt(B, 0.0), mn(B, 0.0), mx(B, 0.0), amax(B, 0.0);
    for (int b = 0; b < B; ++b) {
      if (!mask[b]) continue;
      amax[b] = alpha_host[b];
      if (isclose0(amax[b])) continue;
      const double a1 = 0.45 * amax[b];
      const double o1 = ls_omega(b, 0, a1);
      const bool first = o1 <= prev[b];
      const double a2 = first ? 0.9 * amax[b] : 0.225 * amax[b];
      const double o2 = ls_omega(b, first ? 1 : 2, a2);
      out->omega_evals += 2;
      // parabola through (0, prev), (a1, o1), (a2, o2) (batch.parabola3)
      const double y0 = prev[b];
      const double d1 = (o1 - y0) / a1;
      const double d2 = (o2 - y0) / a2;
      const double c2 = (d2 - d1) / (a2 - a1);
      const double cc1 = d1 - c2 * a1;
      grid_parabola(c2, cc1, y0, std::fmax(a1, a2), &aopt[b], &mn[b], &mx[b]);
      mn[b] /= o->kjmol;
      mx[b] /= o->kjmol;
      omega0[b] = o2;
    }
    for (int b = 0; b < B; ++b) {
      if (!mask[b]) continue;
      if (aopt[b] <= 0) {
        if ((mx[b] - mn[b]) > o->ls_thresh) {  // SLSQP on full evaluations (rare), by the caller
          double al = 0.0, om = omega0[b];
          if (!fb || fb(fbctx, b, s_prev, amax[b], &al, &om) != 0) {
            check(CMM_ERR_UNSUPPORTED);
            return false;
          }
          aopt[b] = al;
          omega0[b] = om;
        } else {
          aopt[b] = o->alpha_mix * amax[b];
        }
      }
      if (aopt[b] <= 0 || isclose0(aopt[b])) aopt[b] = o->alpha_mix * amax[b];
    }
    std::vector<double> coefs((size_t)B * MAXF, 0.0);
    for (int b = 0; b < B; ++b) {
      coefs[(size_t)b * MAXF] = 1.0;
      coefs[(size_t)b * MAXF + 1] = aopt[b] * cf[b];
    }
    set_active(mask);
    for (int b = 0; b < B; ++b)
      if (mask[b] && ls_slot[b] == s_new) ls_slot[b] = -1;
    mix(coefs, {ring(s_prev), rres(s_prev)}, CLIP_DENSITY, ring(s_prev), ring(s_new), spec_ring(s_new));
    // the next step is a hybrid one for every instance while k + 1 <= 4 (solver.py:561)
    std::vector<char> ahead(B, 0);
    if (k + 1 <= 4)
      for (int b = 0; b < B; ++b) ahead[b] = mask[b] && !And_true[b];
    std::vector<int> hist = post_update(mask, k, s_new, &ahead);
    for (int b = 0; b < B; ++b)
      if (mask[b]) {
        omega0[b] = omega(&stats_h[(size_t)b * NST], b);
        out->omega_evals += 1;
      }
    commit(mask, s_new, hist);
    return rc == CMM_OK;
  }

  bool diverging(int b, int k) const {
    if (!o->divergence_guard || k < 8) return false;
    const double* r = &res_hist[(size_t)b * (o->nsteps + 2)];
    const double last_r = r[k];
    if (!std::isfinite(last_r)) return true;
    double best = NAN;
    for (int j = 1; j <= k; ++j)
      if (!std::isnan(r[j])) best = std::isnan(best) ? r[j] : std::fmin(best, r[j]);
    bool rising = true;
    for (int j = k - 4; j <= k; ++j) rising = rising && (r[j] - r[j - 1] >= 0);
    return last_r > 1e6 * best && rising;
  }

  bool converged(int b, double N, double res, double iue, double der, int k) {
    const double riue = (N > 0) ? iue / N : NAN;
    bool ok = true;
    for (int c = 0; c < o->ncrit; ++c) {
      const double v = o->crit[c] == CMM_CRIT_RES ? res : (o->crit[c] == CMM_CRIT_RIUE ? riue : der);
      ok = ok && (v < o->thr[c]);
    }
    if (out->history && k <= o->nsteps + 1) {
      double* h = out->history + ((size_t)b * (o->nsteps + 2) + k) * CMM_HISTORY_COLS;
      h[0] = N; h[1] = res; h[2] = riue; h[3] = omega0[b]; h[4] = der;
    }
    if (iue == 0 && std::isnan(riue)) ok = true;
    return ok;
  }

  // _loop_static (batch.py): static Picard (Picard.update_rho_static,
  // solver.py:392-401).  One fused plane pass per step takes C1 of the
  // current density (ring slot cur[b]) to the mixed density in the other
  // slot and its spectrum; the residual that pass measures belongs to the
  // current density, so the convergence test of a step's density is read
  // one step later, as the Python driver does.
  void loop_static(std::vector<char>& live, std::vector<char>& retry) {
    std::vector<int> cur(B, 0);
    std::vector<double> prev((size_t)B * NST, 0.0), a(B);
    std::fill(res_hist.begin(), res_hist.end(), NAN);
    int step = 0;
    set_active(live);
    while (rc == CMM_OK) {
      bool any = false;
      for (int b = 0; b < B; ++b) any |= live[b] != 0;
      if (!any) break;
      step += 1;
      for (int b = 0; b < B; ++b) a[b] = o->alpha_mix * cf[b];
      set_params(nullptr, a.data());
      for (int par = 0; par < 2; ++par) {
        std::vector<char> grp(B, 0);
        bool anyg = false;
        for (int b = 0; b < B; ++b) {
          grp[b] = live[b] && cur[b] == par;
          anyg |= grp[b] != 0;
        }
        if (!anyg) continue;
        set_active(grp);
        check(cmm_picard_static_step(g, B, w->active, w->params, beta, fn->lambda3, o->picard_thr, o->a_tol,
                                     o->r_tol, w->chat, ring(par), fn->d_V, 0, ring(1 - par), w->that, w->part,
                                     w->nslot, st));
        out->launches += 1;
      }
      set_active(live);
      finalize();
      read(true, false);
      if (rc != CMM_OK) return;
      for (int b = 0; b < B; ++b) {
        if (!live[b]) continue;
        const double* s = &stats_h[(size_t)b * NST];
        if (step > 1) {
          const double* p = &prev[(size_t)b * NST];
          const int k = step - 1;
          const double N = p[CMM_STAT_N] * dr;
          const double res = std::sqrt(s[CMM_STAT_RES2]) / std::sqrt(N) / std::sqrt((double)npts);
          const double iue = p[CMM_STAT_IUE] * dr;
          const double der = std::sqrt(s[CMM_STAT_DER]) / std::sqrt((double)npts);
          out->steps[b] = k;
          const bool conv = converged(b, N, res, iue, der, k);
          if (k <= o->nsteps + 1) res_hist[(size_t)b * (o->nsteps + 2) + k] = res;
          if (conv || k >= o->nsteps || diverging(b, k)) {
            if (!conv) out->diverged[b] = k < o->nsteps ? 1 : 0;
            finish(b, cur[b], N, k, conv);
            live[b] = 0;
            continue;
          }
        }
        if (s[CMM_STAT_NONFIN] > 0) {
          retry[b] = 1;
          live[b] = 0;
          continue;
        }
        cur[b] = 1 - cur[b];
      }
      any = false;
      for (int b = 0; b < B; ++b) any |= live[b] != 0;
      if (!any) break;
      set_active(live);
      c1(w->that, w->chat, 1, nullptr);
      prev = stats_h;
    }
  }

  // loop_static with the decisions on the device (k_static_decide) and the
  // step replayed as a CUDA graph; the host reads the count of instances
  // still stepping every STATIC_CHECK steps.  Same trajectory and outputs as
  // loop_static.
  static constexpr int STATIC_CHECK = 4;
  void static_step(const StaticParams& P, const StaticDev& D, cudaStream_t s) {
    for (int par = 0; par < 2; ++par)
      check(cmm_picard_static_step(g, B, D.act + par * B, w->params, beta, fn->lambda3, o->picard_thr, o->a_tol,
                                   o->r_tol, w->chat, ring(par), fn->d_V, 0, ring(1 - par), w->that, w->part,
                                   w->nslot, s));
    check(cmm_stats_finalize(B, D.live, w->part, w->nslot, (1u << NST) - 1u, w->stats, s));
    k_static_decide<<<1, 256, 0, s>>>(P, w->stats, D);
    cuda(cudaPeekAtLastError());
    check(cmm_fmt_c1(g, B, D.live, fn->R, fn->beta, fn->version, fn->wda, fn->d_kst, fn->d_wtab, w->that,
                     w->chat, w->work, w->part, w->nslot, 1, nullptr, s));
    out->launches += 7;
  }

  void loop_static_device(std::vector<char>& live, std::vector<char>& retry) {
    const int H = o->nsteps + 2;
    const size_t ni = (size_t)B, nd_hist = out->history ? (size_t)B * H * CMM_HISTORY_COLS : 0;
    const size_t ibytes = sizeof(int) * (ni * 9 + 2);
    const size_t dbytes = sizeof(double) * (ni * NST + 2 * ni + ni * H + nd_hist);
    void* mem = nullptr;
    const size_t ioff = (ibytes + 15) & ~(size_t)15;
    if (!cuda(cudaMalloc(&mem, ioff + dbytes))) return;
    StaticDev D;
    int* ip = (int*)mem;
    D.live = ip; D.act = ip + ni; D.cur = ip + 3 * ni; D.retry = ip + 4 * ni; D.fin = ip + 5 * ni;
    D.steps = ip + 6 * ni; D.conv = ip + 7 * ni; D.divg = ip + 8 * ni; D.ctr = ip + 9 * ni;
    double* dp = (double*)((char*)mem + ioff);
    D.prev = dp; D.N = dp + ni * NST; D.omega0 = D.N + ni; D.res_hist = D.omega0 + ni;
    D.history = out->history ? D.res_hist + ni * H : nullptr;
    // initial state, as loop_static starts
    std::vector<int> hi(ni * 9 + 2, 0);
    int nl = 0;
    for (int b = 0; b < B; ++b) {
      hi[b] = live[b] ? 1 : 0;          // live
      hi[ni + b] = live[b] ? 1 : 0;     // act[0]: every current density in slot 0
      nl += live[b] ? 1 : 0;
    }
    hi[ni * 9 + 1] = nl;
    std::vector<double> hd(ni * NST + 2 * ni + ni * H + nd_hist, 0.0);
    for (int b = 0; b < B; ++b) hd[ni * NST + ni + b] = omega0[b];
    for (size_t q = 0; q < ni * H; ++q) hd[ni * NST + 2 * ni + q] = NAN;
    if (nd_hist) std::memcpy(&hd[ni * NST + 2 * ni + ni * H], out->history, sizeof(double) * nd_hist);
    cuda(cudaMemcpyAsync(D.live, hi.data(), sizeof(int) * hi.size(), cudaMemcpyHostToDevice, st));
    cuda(cudaMemcpyAsync(D.prev, hd.data(), sizeof(double) * hd.size(), cudaMemcpyHostToDevice, st));
    std::vector<double> a(B);
    for (int b = 0; b < B; ++b) a[b] = o->alpha_mix * cf[b];
    set_params(nullptr, a.data());
    StaticParams P;
    P.B = B; P.nsteps = o->nsteps; P.ncrit = o->ncrit; P.guard = o->divergence_guard;
    for (int c = 0; c < 3; ++c) { P.crit[c] = o->crit[c]; P.thr[c] = o->thr[c]; }
    P.dr = dr; P.npts = (double)npts;
    // the first step eagerly (it also raises the kernels' shared-memory
    // limits outside any capture), then the step captured on a private
    // stream (the caller's may be the legacy default stream, which cannot
    // be captured) and replayed on the caller's stream
    static_step(P, D, st);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cs = nullptr;
    if (rc == CMM_OK && cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess) {
      if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const long long l0 = out->launches;
        static_step(P, D, cs);
        out->launches = l0;
        const bool ok = cudaStreamEndCapture(cs, &graph) == cudaSuccess && rc == CMM_OK &&
                        cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
        if (!ok) {
          if (exec) cudaGraphExecDestroy(exec);
          exec = nullptr;
          rc = CMM_OK;          // no graph: the same step sequence is launched eagerly
        }
      }
    }
    cudaGetLastError();         // a refused capture leaves only a non-sticky error behind
    int* hc = (int*)stage();
    int steps_run = 1;
    while (rc == CMM_OK) {
      cuda(cudaMemcpyAsync(hc, D.ctr, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
      cuda(cudaStreamSynchronize(st));
      if (hc[1] == 0 || steps_run > o->nsteps + 2) break;
      for (int i = 0; i < STATIC_CHECK && rc == CMM_OK; ++i, ++steps_run) {
        if (exec) {
          cuda(cudaGraphLaunch(exec, st));
          out->launches += 7;
        } else {
          static_step(P, D, st);
        }
      }
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (cs) cudaStreamDestroy(cs);
    if (rc == CMM_OK) {
      cuda(cudaMemcpyAsync(hi.data(), D.live, sizeof(int) * hi.size(), cudaMemcpyDeviceToHost, st));
      cuda(cudaMemcpyAsync(hd.data(), D.prev, sizeof(double) * hd.size(), cudaMemcpyDeviceToHost, st));
      cuda(cudaStreamSynchronize(st));
    }
    if (rc == CMM_OK) {
      if (nd_hist) std::memcpy(out->history, &hd[ni * NST + 2 * ni + ni * H], sizeof(double) * nd_hist);
      for (int b = 0; b < B; ++b) {
        if (!live[b]) continue;
        const int k = hi[6 * ni + b];
        if (k > 0) out->steps[b] = k;
        if (hi[5 * ni + b]) {           // finished
          if (!hi[7 * ni + b]) out->diverged[b] = hi[8 * ni + b];
          finish(b, hi[3 * ni + b], hd[ni * NST + b], k, hi[7 * ni + b] != 0);
          live[b] = 0;
        } else if (hi[4 * ni + b]) {    // non-finite: retried by the caller
          retry[b] = 1;
          live[b] = 0;
        }
      }
    }
    cudaStreamSynchronize(st);
    cudaFree(mem);
  }

  // _loop_general (batch.py)
  void loop_general(std::vector<char>& live, std::vector<char>& retry) {
    std::fill(gram.begin(), gram.end(), 0.0);
    std::fill(rnorm2.begin(), rnorm2.end(), 0.0);
    std::fill(And_true.begin(), And_true.end(), 0);
    std::fill(it_eps0.begin(), it_eps0.end(), NAN);
    std::fill(damping.begin(), damping.end(), o->damping);
    std::fill(res_hist.begin(), res_hist.end(), NAN);
    std::fill(ls_slot.begin(), ls_slot.end(), -1);
    // r_0 and the first line search
    set_active(live);
    residual(w->chat, ring(0), rres(0), {});
    finalize();
    launch_ls(live, 0, w->stats + CMM_STAT_N3MAX, NST);
    read(true, true);
    keep_ls(live, 0);
    for (int b = 0; b < B; ++b) {
      rnorm2[(size_t)b * m] = stats_h[(size_t)b * NST + CMM_STAT_RES2];
      gram[(size_t)b * m * m] = stats_h[(size_t)b * NST + CMM_STAT_RES2];
    }
    int k = 0;
    std::vector<char> cond(B), hyb(B), ok(B);
    while (rc == CMM_OK) {
      bool any = false;
      for (int b = 0; b < B; ++b) any |= live[b] != 0;
      if (!any) break;
      k += 1;
      const int s_prev = (k - 1) % m, s_new = k % m;
      for (int b = 0; b < B; ++b) {
        const double it_eps = std::sqrt(rnorm2[(size_t)b * m + s_prev]) / Ncur[b];
        if (k < 3 && live[b]) it_eps0[b] = it_eps;
        cond[b] = anderson ? (pure || ((it_eps <= it_eps0[b] * o->delta) && k > 4) || And_true[b]) : 0;
        cond[b] = cond[b] && live[b];
        hyb[b] = live[b] && !cond[b];
      }
      bool anyc = false, anyh = false;
      for (int b = 0; b < B; ++b) anyc |= cond[b] != 0;
      if (anyc) {
        if (!anderson_candidate(cond, k, s_prev, s_new, ok)) return;
        for (int b = 0; b < B; ++b) {
          And_true[b] = And_true[b] || cond[b];
          hyb[b] = hyb[b] || (cond[b] && !ok[b]);
        }
      }
      for (int b = 0; b < B; ++b) anyh |= hyb[b] != 0;
      if (anyh && !hybrid_step(hyb, k, s_prev, s_new)) return;
      // after the update: non-finite check, N, convergence (solver.py:286-305)
      for (int b = 0; b < B; ++b) {
        if (!live[b]) continue;
        out->steps[b] = k;
        const double* s = &last[(size_t)b * NST];
        if (s[CMM_STAT_NONFIN] > 0) {
          retry[b] = 1;
          live[b] = 0;
          continue;
        }
        const double N = s[CMM_STAT_N] * dr;
        const double res = std::sqrt(rnorm2[(size_t)b * m + s_new]) / std::sqrt(N) / std::sqrt((double)npts);
        const double iue = s[CMM_STAT_IUE] * dr;
        const double der = std::sqrt(s[CMM_STAT_DER]) / std::sqrt((double)npts);
        Ncur[b] = N;
        const bool conv = converged(b, N, res, iue, der, k);
        if (k <= o->nsteps + 1) res_hist[(size_t)b * (o->nsteps + 2) + k] = res;
        if (conv || k >= o->nsteps || diverging(b, k)) {
          if (!conv) out->diverged[b] = k < o->nsteps ? 1 : 0;
          finish(b, s_new, N, k, conv);
          live[b] = 0;
        }
      }
    }
  }

  int run(const double* cf0) {
    npts = (size_t)g->n1 * g->n2 * g->n3;
    S = (size_t)2 * g->n1 * g->n2 * g->h3;
    nwd = 5 + ((fn->version & CMM_WDA) ? 1 : 0) + ((fn->version & CMM_TENSOR) ? 6 : 0);
    wda = (fn->version & CMM_WDA) != 0;
    m = std::max(o->m, 2);
    if (m > CMM_MAX_HIST || 2 * m > MAXF) return CMM_ERR_ARG;
    anderson = o->method == CMM_SOLVE_ANDERSON || o->method == CMM_SOLVE_HYBRIDANDERSON;
    pure = o->method == CMM_SOLVE_ANDERSON;
    statik = o->method == CMM_SOLVE_STATIC;
    if (!anderson) m = 2;
    if (anderson && o->coefs == CMM_COEF_SLSQP && B >= 8) {
      const unsigned hw = std::thread::hardware_concurrency();
      const int nt = (int)std::min(3u, hw > 1 ? hw - 1 : 0u);
      try {
        if (nt > 0) pool.reset(new HostPool(nt));
      } catch (const std::exception&) {
        pool.reset();   // no threads: the coefficients are computed inline
      }
    }
    dr = g->volume / (double)npts;
    beta = fn->beta;
    slot_bytes = stage_slot_bytes(B);
    cf.assign(cf0, cf0 + B);
    failed.assign(B, 0);
    And_true.assign(B, 0);
    ls_slot.assign(B, -1);
    omega0.assign(B, 0.0); n3max.assign(B, 0.0); Ncur.assign(B, 0.0);
    last.assign((size_t)B * NST, 0.0);
    gram.assign((size_t)B * m * m, 0.0); rnorm2.assign((size_t)B * m, 0.0);
    it_eps0.assign(B, NAN); damping.assign(B, o->damping);
    ls_host.assign((size_t)B * NLS, 0.0); alpha_host.assign(B, 0.0);
    res_hist.assign((size_t)B * (o->nsteps + 2), NAN);
    stats_h.assign((size_t)B * NST, 0.0); ls_h.assign((size_t)B * NLS, 0.0); alpha_h.assign(B, 0.0);
    wd_ok.assign((size_t)B * m, 0);
    for (int b = 0; b < B; ++b) {
      out->N[b] = NAN; out->converged[b] = 0; out->steps[b] = 0; out->diverged[b] = 0; out->failed[b] = 0;
      out->omega[b] = NAN;
    }
    if (out->history)
      for (size_t i = 0; i < (size_t)B * (o->nsteps + 2) * CMM_HISTORY_COLS; ++i) out->history[i] = NAN;
    if (w->h_result) cuda(cudaStreamCreateWithFlags(&copy_st, cudaStreamNonBlocking));
    set_params(nullptr);
    std::vector<char> todo(B, 1);
    while (rc == CMM_OK) {
      bool any = false;
      for (int b = 0; b < B; ++b) any |= todo[b] != 0;
      if (!any) break;
      std::vector<char> live(todo), retry(B, 0);
      init_state(todo);
      if (rc) break;
      if (statik && o->device_loop) loop_static_device(live, retry);
      else if (statik) loop_static(live, retry);
      else loop_general(live, retry);
      // non-finite -> halve the correction factor and restart (solver.py:335-345)
      for (int b = 0; b < B; ++b) {
        if (retry[b]) {
          cf[b] /= 2;
          if (cf[b] < 0.25) {
            failed[b] = 1;
            retry[b] = 0;
          }
        }
        todo[b] = retry[b];
      }
    }
    for (int b = 0; b < B; ++b) out->failed[b] = failed[b];
    if (out->cf)
      for (int b = 0; b < B; ++b) out->cf[b] = cf[b];
    cuda(cudaStreamSynchronize(st));
    if (copy_st) {
      cuda(cudaStreamSynchronize(copy_st));
      cudaStreamDestroy(copy_st);
    }
    for (cudaEvent_t ev : copy_ev) cudaEventDestroy(ev);
    out->pipe_n = 0;
    for (const PipeRec& r : pipe) {
      float ms = 0.0f;
      if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess && out->pipe_n < out->pipe_cap) {
        double* q = out->pipe_log + (size_t)out->pipe_n * 3;
        q[0] = r.want; q[1] = r.nact; q[2] = ms;
        out->pipe_n += 1;
      }
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
    return rc;
  }
};

}  // namespace

extern "C" size_t cmm_solve_stage_bytes(int batch) {
  return batch < 1 ? 0 : stage_slot_bytes(batch) * NSTAGE;
}

extern "C" int cmm_solve_batched(const cmm_functional_desc* fn, const cmm_solve_opts* opt, int batch,
                                 const double* mu, const double* fug, const double* cf0, const cmm_solve_ws* ws,
                                 cmm_solve_out* out, cmm_fallback_fn fallback, void* fallback_ctx, void* stream) {
  if (!fn || !fn->grid || !opt || batch < 1 || !mu || !fug || !cf0 || !ws || !out) return CMM_ERR_ARG;
  if (!out->N || !out->omega || !out->converged || !out->steps || !out->diverged || !out->failed) return CMM_ERR_ARG;
  if (opt->method != CMM_SOLVE_HYBRID && opt->method != CMM_SOLVE_ANDERSON && opt->method != CMM_SOLVE_HYBRIDANDERSON &&
      opt->method != CMM_SOLVE_STATIC)
    return CMM_ERR_UNSUPPORTED;
  if (opt->method == CMM_SOLVE_STATIC ? (!ws->ring || !ws->that || !ws->chat || !ws->chat2)
                                      : (!ws->spec_ring || !ws->wd_ring || !ws->wd_r || !ws->rhat || !ws->ls_part))
    return CMM_ERR_ARG;
  if (opt->ncrit < 1 || opt->ncrit > 3 || opt->nsteps < 1) return CMM_ERR_ARG;
  if (opt->coefs != CMM_COEF_SLSQP && opt->coefs != CMM_COEF_EXACT) return CMM_ERR_ARG;
  if (!ws->h_stats || !ws->h_ls || !ws->h_alpha || !ws->h_stage) return CMM_ERR_ARG;
  Driver d;
  d.fn = fn; d.o = opt; d.B = batch; d.w = ws; d.out = out; d.fb = fallback; d.fbctx = fallback_ctx;
  d.st = (cudaStream_t)stream; d.g = fn->grid; d.mu = mu; d.fug = fug;
  out->launches = 0;
  out->omega_evals = 0;
  return d.run(cf0);
}
