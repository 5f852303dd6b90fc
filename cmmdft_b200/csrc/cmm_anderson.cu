// Anderson mixing coefficients as the reference computes them
// (Anderson.update_rho_Anderson, cmmdft/solver.py:581-591):
//
//     alphas = scipy.optimize.minimize(sum_res, full(mk, 1/mk), method='SLSQP',
//                                      tol=1e-10, bounds=Bounds(0, 1),
//                                      constraints=LinearConstraint(ones(mk), 1, 1)).x
//
// with sum_res(a) = ||sum_i a_i r_i||_2.  SLSQP stops early when the residuals
// are small (its tests are absolute, acc = 1e-10), so its result is not the
// minimiser and the solver's trajectory depends on every detail of the
// method.  This file restates it for this problem class from the published
// algorithm -- D. Kraft, "A software package for sequential quadratic
// programming", DFVLR-FB 88-28 (1988): SQP with an L1 merit line search,
// damped BFGS on LDL^T factors updated by the Fletcher-Powell composite
// t-method (Math. Comp. 28 (1974) 1067-1087) -- together with the finite
// differences scipy's minimize supplies when no gradient is given (2-point,
// absolute step 2^-26, step reversed where it would leave the bounds).
// The objective is evaluated from the Gram matrix G_ij = <r_i, r_j> as
// sqrt(a^T G a), so no residual field is read on the host.
//
// The QP subproblem (min 1/2 s^T B s + g^T s, sum s = -c, -x <= s <= 1-x) is
// strictly convex, so its solution does not depend on the method; it is
// solved exactly on the support of x + s that satisfies the KKT conditions
// (the upper bounds are implied by x + s >= 0 and sum (x + s) = 1).
#include <cmath>
#include <cstring>

#include "cmm_common.cuh"

namespace {

constexpr int NMAX = 8;
constexpr double FD_STEP = 1.4901161193847656e-08;   // 2^-26: sqrt of the double epsilon

struct Gram {
  const double* G;
  int n;
  double operator()(const double* a) const {
    double q = 0.0;
    for (int i = 0; i < n; ++i) {
      double t = 0.0;
      for (int j = 0; j < n; ++j) t += G[i * n + j] * a[j];
      q += a[i] * t;
    }
    return std::sqrt(q > 0.0 ? q : 0.0);
  }
};

// forward differences with the step reversed where x + h leaves [0, 1]
void fd_gradient(const Gram& f, const double* x, double f0, double* g) {
  const int n = f.n;
  double x1[NMAX];
  for (int i = 0; i < n; ++i) {
    double h = FD_STEP;
    const double xh = x[i] + h;
    if ((xh < 0.0 || xh > 1.0) && h <= std::fmax(x[i], 1.0 - x[i])) h = -h;
    std::memcpy(x1, x, sizeof(double) * n);
    x1[i] = x[i] + h;
    const double dx = (x[i] + h) - x[i];
    g[i] = (f(x1) - f0) / dx;
  }
}

// dense solve of a small system by Gaussian elimination with partial pivoting;
// returns false for a singular matrix
bool dense_solve(double* A, double* b, int N) {
  for (int c = 0; c < N; ++c) {
    int p = c;
    double mx = std::fabs(A[c * N + c]);
    for (int r = c + 1; r < N; ++r)
      if (std::fabs(A[r * N + c]) > mx) { mx = std::fabs(A[r * N + c]); p = r; }
    if (mx == 0.0) return false;
    if (p != c) {
      for (int j = 0; j < N; ++j) { const double t = A[c * N + j]; A[c * N + j] = A[p * N + j]; A[p * N + j] = t; }
      const double t = b[c]; b[c] = b[p]; b[p] = t;
    }
    for (int r = c + 1; r < N; ++r) {
      const double q = A[r * N + c] / A[c * N + c];
      for (int j = c; j < N; ++j) A[r * N + j] -= q * A[c * N + j];
      b[r] -= q * b[c];
    }
  }
  for (int r = N - 1; r >= 0; --r) {
    double s = b[r];
    for (int j = r + 1; j < N; ++j) s -= A[r * N + j] * b[j];
    b[r] = s / A[r * N + r];
  }
  return true;
}

// Equality-constrained minimiser of the QP on support S (variables outside S
// at their lower bound s_i = -x_i): the bordered system
// [B_SS -1; 1^T 0][s_S; lam] = [-(g_S + B_SN s_N); sig + sum_N x_i].
// Returns false for a singular system; *primal: s_S >= -x_S; *dual: the
// multipliers (B s + g)_i - lam of the bounds outside S are >= 0.
bool support_solve(const double* B, const double* g, const double* x, double sig, int n, unsigned S,
                   double* sv, double* lam, bool* primal, bool* dual, int* drop, int* add) {
  int idx[NMAX], k = 0;
  double rest = 0.0;
  for (int i = 0; i < n; ++i) {
    if ((S >> i) & 1u) idx[k++] = i;
    else { sv[i] = -x[i]; rest += x[i]; }
  }
  const int N = k + 1;
  double A[(NMAX + 1) * (NMAX + 1)], r[NMAX + 1];
  for (int a = 0; a < k; ++a) {
    const int i = idx[a];
    double t = g[i];
    for (int j = 0; j < n; ++j)
      if (!((S >> j) & 1u)) t += B[i * n + j] * sv[j];
    r[a] = -t;
    for (int b = 0; b < k; ++b) A[a * N + b] = B[i * n + idx[b]];
    A[a * N + k] = -1.0;
    A[k * N + a] = 1.0;
  }
  A[k * N + k] = 0.0;
  r[k] = sig + rest;
  if (!dense_solve(A, r, N)) return false;
  *primal = true;
  double worst = 0.0;
  for (int a = 0; a < k; ++a) {
    sv[idx[a]] = r[a];
    const double viol = -x[idx[a]] - r[a];
    if (!(r[a] >= -x[idx[a]] - 1e-14)) {
      if (*primal || viol > worst) { worst = viol; *drop = idx[a]; }
      *primal = false;
    }
  }
  *lam = r[k];
  double gmax = std::fabs(r[k]);
  for (int i = 0; i < n; ++i) gmax = std::fmax(gmax, std::fabs(g[i]));
  *dual = true;
  double most = 0.0;
  for (int i = 0; i < n; ++i) {
    if ((S >> i) & 1u) continue;
    double t = g[i];
    for (int j = 0; j < n; ++j) t += B[i * n + j] * sv[j];
    const double mult = t - r[k];
    if (mult < -1e-12 * gmax) {
      if (*dual || mult < most) { most = mult; *add = i; }
      *dual = false;
    }
  }
  return true;
}

double qp_objective(const double* B, const double* g, const double* sv, int n) {
  double obj = 0.0;
  for (int i = 0; i < n; ++i) {
    double t = 0.0;
    for (int j = 0; j < n; ++j) t += B[i * n + j] * sv[j];
    obj += sv[i] * (0.5 * t + g[i]);
  }
  return obj;
}

// min 1/2 s^T B s + g^T s  s.t.  sum s = sig, s >= -x (the unique minimiser
// of a strictly convex QP).  The support that satisfies the KKT conditions
// is searched from *hint (the previous subproblem's support): a variable
// below its bound leaves the support, else the bound with the most negative
// multiplier is released, for at most 2n trials; when that does not settle
// (or rounding leaves no support passing both tests) every support is tried
// and the first passing both, else the lowest objective over the
// primal-feasible ones, is taken.  s and the equality multiplier lam.
bool qp_subproblem(const double* B, const double* g, const double* x, double sig, int n, double* s, double* lam,
                   unsigned* hint) {
  const unsigned K = 1u << n;
  double sv[NMAX], lv;
  bool primal, dual, done = false;
  int drop = -1, add = -1;
  unsigned S = (*hint > 0 && *hint < K) ? *hint : K - 1;
  for (int trial = 0; trial < 2 * n && S > 0; ++trial) {
    if (!support_solve(B, g, x, sig, n, S, sv, &lv, &primal, &dual, &drop, &add)) break;
    if (primal && dual) { done = true; break; }
    S = primal ? (S | (1u << add)) : (S & ~(1u << drop));
  }
  if (done) {
    std::memcpy(s, sv, sizeof(double) * n);
    *lam = lv;
    *hint = S;
  } else {
    bool found = false, kkt = false;
    double best = 0.0;
    for (unsigned T = 1; T < K && !kkt; ++T) {
      if (!support_solve(B, g, x, sig, n, T, sv, &lv, &primal, &dual, &drop, &add) || !primal) continue;
      const double obj = qp_objective(B, g, sv, n);
      if (dual || !found || obj < best) {
        found = true;
        kkt = dual;
        best = obj;
        std::memcpy(s, sv, sizeof(double) * n);
        *lam = lv;
        *hint = T;
      }
    }
    if (!found) return false;
  }
  for (int i = 0; i < n; ++i) s[i] = std::fmin(std::fmax(s[i], -x[i]), 1.0 - x[i]);
  return true;
}

// packed LDL^T (lower triangle by columns, D on the diagonal positions)
void ldl_reset(double* L, int n) {
  std::memset(L, 0, sizeof(double) * n * (n + 1) / 2);
  for (int i = 0, j = 0; i < n; ++i) { L[j] = 1.0; j += n - i; }
}

void ldl_dense(const double* L, int n, double* B) {
  double Lm[NMAX * NMAX] = {0.0}, D[NMAX];
  for (int i = 0, ij = 0; i < n; ++i) {
    D[i] = L[ij];
    Lm[i * n + i] = 1.0;
    for (int j = i + 1; j < n; ++j) Lm[j * n + i] = L[++ij];
    ++ij;
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double t = 0.0;
      for (int q = 0; q < n; ++q) t += Lm[i * n + q] * D[q] * Lm[j * n + q];
      B[i * n + j] = t;
    }
}

// L D L^T + sigma z z^T, composite t-method; z is overwritten, w is work
void ldl_update(double* L, int n, double* z, double sigma, double* w) {
  constexpr double EPMACH = 2.22e-16;
  if (sigma == 0.0) return;
  int ij = 0;
  double t = 1.0 / sigma;
  if (sigma < 0.0) {
    for (int i = 0; i < n; ++i) w[i] = z[i];
    for (int i = 0; i < n; ++i) {
      const double v = w[i];
      t += v * v / L[ij];
      for (int j = i + 1; j < n; ++j) { ++ij; w[j] -= v * L[ij]; }
      ++ij;
    }
    if (t >= 0.0) t = EPMACH / sigma;
    for (int i = 0; i < n; ++i) {
      const int j = n - 1 - i;
      ij -= i + 1;
      const double u = w[j];
      w[j] = t;
      t -= u * u / L[ij];
    }
  }
  for (int i = 0; i < n; ++i) {
    const double v = z[i];
    const double delta = v / L[ij];
    const double tp = (sigma < 0.0) ? w[i] : t + delta * v;
    const double alpha = tp / t;
    L[ij] = alpha * L[ij];
    if (i == n - 1) return;
    const double beta = delta / tp;
    if (alpha > 4.0) {
      const double gamma = t / tp;
      for (int j = i + 1; j < n; ++j) {
        ++ij;
        const double u = L[ij];
        L[ij] = gamma * u + beta * z[j];
        z[j] -= v * u;
      }
    } else {
      for (int j = i + 1; j < n; ++j) {
        ++ij;
        z[j] -= v * L[ij];
        L[ij] += beta * z[j];
      }
    }
    ++ij;
    t = tp;
  }
}

double sum_minus_one(const double* x, int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += x[i];
  return s - 1.0;
}

double norm2(const double* v, int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += v[i] * v[i];
  return std::sqrt(s);
}

}  // namespace

// Exit modes as scipy reports them: 0 converged, 8 positive directional
// derivative in the line search, 9 iteration limit; -2 for an unsupported
// size or a QP subproblem without a solution.
int anderson_slsqp(const double* G, int n, double* x, int* nit_out) {
  constexpr double ACC = 1e-10, TOL = 10.0 * ACC;
  constexpr int MAXITER = 100;
  if (n < 1 || n > NMAX) return -2;
  const Gram f{G, n};
  double g[NMAX], s[NMAX] = {0.0}, x0[NMAX], vg[NMAX], u[NMAX], v[NMAX], w[NMAX];
  double L[NMAX * (NMAX + 1) / 2], B[NMAX * NMAX];
  for (int i = 0; i < n; ++i) x[i] = 1.0 / n;
  double fx = f(x);
  fd_gradient(f, x, fx, g);
  double c = sum_minus_one(x, n);
  double mu = 0.0, f0 = fx;
  int it = 0, ireset = 1, mode = 9;
  unsigned support = (1u << n) - 1;   // x = 1/n: every variable free
  ldl_reset(L, n);
  auto relaxed = [&]() {
    return ((std::fabs(fx - f0) < TOL || norm2(s, n) < TOL) && std::fabs(c) < TOL) ? 0 : 8;
  };
  for (;;) {
    if (++it > MAXITER) { mode = 9; break; }
    ldl_dense(L, n, B);
    double r;
    if (!qp_subproblem(B, g, x, -c, n, s, &r, &support)) { mode = -2; break; }
    for (int i = 0; i < n; ++i) vg[i] = g[i] - r;
    f0 = fx;
    std::memcpy(x0, x, sizeof(double) * n);
    double gs = 0.0;
    for (int i = 0; i < n; ++i) gs += g[i] * s[i];
    double h1 = std::fabs(gs) + std::fabs(r) * std::fabs(c);
    const double h2 = std::fabs(c);
    mu = std::fmax(std::fabs(r), (mu + std::fabs(r)) / 2.0);
    if (h1 < ACC && h2 < ACC) { mode = 0; break; }
    const double t0 = fx + mu * std::fabs(c);
    double h3 = gs - mu * std::fabs(c);
    if (h3 >= 0.0) {   // not a descent direction: restart from the identity
      if (++ireset > 5) { mode = relaxed(); break; }
      ldl_reset(L, n);
      continue;
    }
    double alpha = 1.0;
    for (int line = 1;; ++line) {   // L1 merit line search
      h3 *= alpha;
      for (int i = 0; i < n; ++i) {
        s[i] *= alpha;
        x[i] = std::fmin(std::fmax(x0[i] + s[i], 0.0), 1.0);
      }
      fx = f(x);
      c = sum_minus_one(x, n);
      h1 = fx + mu * std::fabs(c) - t0;
      if (h1 <= h3 / 10.0 || line > 10) break;
      alpha = std::fmax(h3 / (2.0 * (h3 - h1)), 0.1);
    }
    if ((std::fabs(fx - f0) < ACC || norm2(s, n) < ACC) && std::fabs(c) < ACC) { mode = 0; break; }
    fd_gradient(f, x, fx, g);
    // damped BFGS on the Lagrangian gradient difference (the multiplier
    // terms cancel: the constraint is linear); B still holds L D L^T
    double sv = 0.0, sBs = 0.0;
    for (int i = 0; i < n; ++i) {
      u[i] = g[i] - r - vg[i];
      double t = 0.0;
      for (int j = 0; j < n; ++j) t += B[i * n + j] * s[j];
      v[i] = t;
    }
    for (int i = 0; i < n; ++i) { sv += s[i] * u[i]; sBs += s[i] * v[i]; }
    double hu = sv;
    const double h3b = 0.2 * sBs;
    if (hu < h3b) {
      const double h4 = (sBs - h3b) / (sBs - hu);
      hu = h3b;
      for (int i = 0; i < n; ++i) u[i] = h4 * u[i] + (1.0 - h4) * v[i];
    }
    if (hu == 0.0 || sBs == 0.0) {
      if (++ireset > 5) { mode = relaxed(); break; }
      ldl_reset(L, n);
      continue;
    }
    ldl_update(L, n, u, 1.0 / hu, w);
    ldl_update(L, n, v, -1.0 / sBs, w);
  }
  if (nit_out) *nit_out = it;
  return mode;
}

extern "C" int cmm_anderson_slsqp(const double* gram, int n, double* alpha, int* mode, int* nit) {
  if (!gram || !alpha || n < 1 || n > NMAX) return CMM_ERR_ARG;
  const int md = anderson_slsqp(gram, n, alpha, nit);
  if (mode) *mode = md;
  return CMM_OK;
}
