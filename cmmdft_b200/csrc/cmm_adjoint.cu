// Implicit-adjoint pieces at a converged density: the parameter derivatives
// of the capped Lennard-Jones external potential, weighted contractions of
// fields, and the vector steps of a batched BiCGSTAB solve of the adjoint
// system (I + beta S A^T S) y = c, S = diag(sqrt(rho)) (the scaled Jacobian
// of the Euler-Lagrange residual ln(Lambda^3 rho) + beta (C1 - mu)).
//
// The BiCGSTAB scalars live on the device ([B][CMM_BICG_NS] doubles), so an
// iteration needs no host round trip; the host reads the residual norms only
// to decide when to stop.
#include <cmath>
#include <vector>

#include "cmm_common.cuh"

#define ADJ_THREADS 256
#define ADJ_MAX_TYPES 8

namespace {

// ---------------------------------------- LJ parameter derivatives ----
struct AtomG { double x, y, z, sm, fe, shift, dshift; int t; };

struct GradArgs {
  double rv[9];
  double L[3];
  int n1, n2, n3;
  int natom, ntype;
  double cutoff, vcap;
  double geps;              // guest epsilon
  double teps[ADJ_MAX_TYPES];
};

__device__ __forceinline__ double lin_coord(int i, int n) {
  const double step = 1.0 / (double)n;
  return __dadd_rn(__dmul_rn((double)i, step), -0.5);
}

__device__ __forceinline__ double min_image(double r, double L, double invL) {
  double q = r * invL;
  double f = fabs(q - trunc(q));
  if (fabs(f - 0.5) < 1e-9) q = __ddiv_rn(r, L);
  return __dsub_rn(r, __dmul_rn(L, rint(q)));
}

// dV/d(theta) at every grid point for theta = (guest eps, guest sigma,
// eps_t for each host type, sigma_t for each host type), rows of dV.  The
// pair sum repeats cmm_extpot_lj's arithmetic and order, so the capping
// decision (V not finite or V > vcap: derivative 0) is the same.  With
// Lorentz-Berthelot mixing, per pair v = 4 e_m ((s_m/R)^12 - (s_m/R)^6) - shift:
//   dv/de_t = v / (2 e_t), dv/de_g = v / (2 e_g),
//   dv/ds_t = dv/ds_g = (1/2) dv/ds_m,
//   dv/ds_m = (4 e_m / s_m) (12 q^12 - 6 q^6) - dshift/ds_m,  q = s_m / R.
__global__ void __launch_bounds__(ADJ_THREADS)
k_extpot_grad(GradArgs a, const AtomG* __restrict__ atoms, double* __restrict__ dV, long long ldv) {
  __shared__ AtomG tile[ADJ_THREADS];
  const long long npts = (long long)a.n1 * a.n2 * a.n3;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = idx < npts;
  double p[3] = {0, 0, 0};
  if (live) {
    const int k = (int)(idx % a.n3);
    const int j = (int)((idx / a.n3) % a.n2);
    const int i = (int)(idx / ((long long)a.n3 * a.n2));
    const double g0 = lin_coord(i, a.n1), g1 = lin_coord(j, a.n2), g2 = lin_coord(k, a.n3);
#pragma unroll
    for (int b = 0; b < 3; ++b)
      p[b] = __dadd_rn(__dadd_rn(__dmul_rn(a.rv[0 * 3 + b], g0), __dmul_rn(a.rv[1 * 3 + b], g1)),
                       __dmul_rn(a.rv[2 * 3 + b], g2));
  }
  const double invL0 = 1.0 / a.L[0], invL1 = 1.0 / a.L[1], invL2 = 1.0 / a.L[2];
  double acc = 0.0;
  double E[ADJ_MAX_TYPES], Sg[ADJ_MAX_TYPES];
  for (int t = 0; t < ADJ_MAX_TYPES; ++t) { E[t] = 0.0; Sg[t] = 0.0; }
  for (int base = 0; base < a.natom; base += ADJ_THREADS) {
    __syncthreads();
    if (base + threadIdx.x < a.natom) tile[threadIdx.x] = atoms[base + threadIdx.x];
    __syncthreads();
    const int cnt = min(ADJ_THREADS, a.natom - base);
    if (!live) continue;
    for (int t = 0; t < cnt; ++t) {
      const AtomG at = tile[t];
      const double rx = min_image(__dsub_rn(p[0], at.x), a.L[0], invL0);
      const double ry = min_image(__dsub_rn(p[1], at.y), a.L[1], invL1);
      const double rz = min_image(__dsub_rn(p[2], at.z), a.L[2], invL2);
      const double r2 = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz)), 1e-16);
      const double R = sqrt(r2);
      if (R < a.cutoff) {
        const double q = __ddiv_rn(at.sm, R);
        const double q2 = __dmul_rn(q, q);
        const double r6 = __dmul_rn(__dmul_rn(q2, q2), q2);
        const double r12 = __dmul_rn(r6, r6);
        const double v = __dsub_rn(__dmul_rn(at.fe, __dsub_rn(r12, r6)), at.shift);
        acc = __dadd_rn(acc, v);
#pragma unroll
        for (int ty = 0; ty < ADJ_MAX_TYPES; ++ty)
          if (ty == at.t) {
            E[ty] += v;
            Sg[ty] += at.fe / at.sm * (12.0 * r12 - 6.0 * r6) - at.dshift;
          }
      }
    }
  }
  if (!live) return;
  const bool capped = !isfinite(acc) || acc > a.vcap;
  double eg = 0.0, sg = 0.0;
  for (int t = 0; t < a.ntype; ++t) {
    dV[(2 + t) * ldv + idx] = capped ? 0.0 : E[t] / (2.0 * a.teps[t]);
    dV[(2 + a.ntype + t) * ldv + idx] = capped ? 0.0 : 0.5 * Sg[t];
    eg += E[t];
    sg += Sg[t];
  }
  dV[0 * ldv + idx] = capped ? 0.0 : eg / (2.0 * a.geps);
  dV[1 * ldv + idx] = capped ? 0.0 : 0.5 * sg;
}

// ------------------------------------------------------ reductions ----
__device__ inline double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  v = 0.0;
  if (w == 0) {
    if (l < (int)(blockDim.x >> 5)) v = red[l];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// part[(w * K + k) * nchunk + chunk] = sum over the chunk's points of W_w * D_k
__global__ void __launch_bounds__(ADJ_THREADS)
k_contract(const double* __restrict__ W, long long ldw, const double* __restrict__ D, long long ldd, int K,
           long long n, double* __restrict__ part, int nchunk) {
  __shared__ double red[32];
  const int chunk = blockIdx.x, w = blockIdx.y;
  const long long per = (n + nchunk - 1) / nchunk;
  const long long lo = (long long)chunk * per, hi = min(n, lo + per);
  const double* wr = W + (long long)w * ldw;
  for (int k = 0; k < K; ++k) {
    const double* dr = D + (long long)k * ldd;
    double acc = 0.0;
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) acc += wr[i] * dr[i];
    const double t = block_sum(acc, red);
    if (threadIdx.x == 0) part[((long long)w * K + k) * nchunk + chunk] = t;
  }
}

// --------------------------------------------------- BiCGSTAB steps ----
enum { S_RHO = 0, S_ALPHA, S_OMEGA, S_BETA, S_D0, S_D1, S_RR, S_FIRST, NS };

__device__ __forceinline__ double sqrt_rho(const double* rho, size_t i) {
  const double r = rho[i];
  return r > 0.0 ? sqrt(r) : 0.0;
}

struct VecArgs {
  int op;
  long long npts;
  const int* active;
  const double* rho;
  const double* sc;
  double c;
  const double *x, *y, *a;
  double *out, *out2;
  const double* rhat;
  double* part;
  int nblk;
};

// the ops of cmm_bicg_vec (include/cmmdft_b200.h)
__global__ void __launch_bounds__(ADJ_THREADS) k_bicg_vec(VecArgs g) {
  __shared__ double red[32];
  const int b = blockIdx.y;
  if (g.active && !g.active[b]) return;
  const size_t off = (size_t)b * g.npts;
  const double* s = g.sc ? g.sc + (size_t)b * NS : nullptr;
  double d0 = 0.0, d1 = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.npts;
       i += (long long)gridDim.x * blockDim.x) {
    const size_t q = off + i;
    switch (g.op) {
      case 0: g.out[q] = sqrt_rho(g.rho, q) * g.x[q]; break;
      case 1: {
        const double o = g.x[q] + g.c * sqrt_rho(g.rho, q) * g.y[q];
        g.out[q] = o;
        d0 += o * g.a[q];
        d1 += o * o;
        break;
      }
      case 2: g.out[q] = g.x[q] + s[S_BETA] * (g.out[q] - s[S_OMEGA] * g.y[q]); break;
      case 3: g.out[q] = g.x[q] - s[S_ALPHA] * g.y[q]; break;
      case 4: {
        g.out[q] += s[S_ALPHA] * g.x[q] + s[S_OMEGA] * g.y[q];
        const double r = g.y[q] - s[S_OMEGA] * g.a[q];
        g.out2[q] = r;
        d0 += g.rhat[q] * r;
        d1 += r * r;
        break;
      }
    }
  }
  if (g.op == 1 || g.op == 4) {
    double t = block_sum(d0, red);
    if (threadIdx.x == 0) g.part[((size_t)b * 2 + 0) * g.nblk + blockIdx.x] = t;
    t = block_sum(d1, red);
    if (threadIdx.x == 0) g.part[((size_t)b * 2 + 1) * g.nblk + blockIdx.x] = t;
  }
}

// Reduce the two dot products of instance b (fixed order) and advance its
// scalars: stage 0 after op 4 (rho_new, rr -> beta), stage 1 after the
// product of p (rhat . v -> alpha), stage 2 after the product of s
// (t . s, t . t -> omega).  A zero denominator freezes the instance's step
// at zero instead of producing NaN.
__global__ void k_bicg_scalars(int B, const int* __restrict__ active, const double* __restrict__ part, int nblk,
                               double* __restrict__ sc, int stage) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B || (active && !active[b])) return;
  double d0 = 0.0, d1 = 0.0;
  for (int i = 0; i < nblk; ++i) {
    d0 += part[((size_t)b * 2 + 0) * nblk + i];
    d1 += part[((size_t)b * 2 + 1) * nblk + i];
  }
  double* s = sc + (size_t)b * NS;
  s[S_D0] = d0;
  s[S_D1] = d1;
  if (stage == 0) {
    s[S_RR] = d1;
    if (s[S_FIRST] != 0.0) {
      s[S_BETA] = 0.0;
      s[S_FIRST] = 0.0;
    } else {
      const double den = s[S_RHO] * s[S_OMEGA];
      s[S_BETA] = (den != 0.0) ? (d0 / s[S_RHO]) * (s[S_ALPHA] / s[S_OMEGA]) : 0.0;
    }
    s[S_RHO] = d0;
  } else if (stage == 1) {
    s[S_ALPHA] = (d0 != 0.0) ? s[S_RHO] / d0 : 0.0;
  } else {
    s[S_OMEGA] = (d1 != 0.0) ? d0 / d1 : 0.0;
  }
}

}  // namespace

extern "C" int cmm_extpot_lj_grad(const cmm_grid* g, const double* d_pos, const int* d_type, int natom,
                                  const double* d_type_sig, const double* d_type_eps, int ntype, double guest_sig,
                                  double guest_eps, double cutoff, double v_cap, double* d_dV, void* stream) {
  if (!g || !d_dV || natom < 0 || ntype < 1 || ntype > ADJ_MAX_TYPES ||
      (natom > 0 && (!d_pos || !d_type || !d_type_sig || !d_type_eps)))
    return CMM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  GradArgs a;
  for (int i = 0; i < 9; ++i) a.rv[i] = g->rvecs[i];
  for (int r = 0; r < 3; ++r) {
    const double* v = g->rvecs + 3 * r;
    a.L[r] = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  }
  a.n1 = g->n1; a.n2 = g->n2; a.n3 = g->n3;
  a.natom = natom;
  a.ntype = ntype;
  a.cutoff = cutoff;
  a.vcap = v_cap;
  a.geps = guest_eps;
  std::vector<double> hpos(3 * (size_t)natom), hs(ntype), he(ntype);
  std::vector<int> htyp(natom);
  std::vector<AtomG> h(natom);
  if (natom > 0) {
    bool ok = cudaMemcpyAsync(hpos.data(), d_pos, sizeof(double) * 3 * natom, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(htyp.data(), d_type, sizeof(int) * natom, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(hs.data(), d_type_sig, sizeof(double) * ntype, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(he.data(), d_type_eps, sizeof(double) * ntype, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) return CMM_ERR_CUDA;
  }
  for (int t = 0; t < ntype; ++t) a.teps[t] = he[t];
  for (int i = 0; i < natom; ++i) {
    const int t = htyp[i];
    if (t < 0 || t >= ntype) return CMM_ERR_ARG;
    // mixed parameters formed as cmm_extpot_lj forms them
    volatile double sm = 0.5 * (hs[t] + guest_sig);
    volatile double em = sqrt(he[t] * guest_eps);
    volatile double q = sm / cutoff;
    volatile double q2 = q * q;
    volatile double rc6 = q2 * q2 * q2;
    volatile double fe = 4.0 * em;
    volatile double sq = rc6 * rc6;
    volatile double df = sq - rc6;
    h[i].x = hpos[3 * i]; h[i].y = hpos[3 * i + 1]; h[i].z = hpos[3 * i + 2];
    h[i].sm = sm;
    h[i].fe = fe;
    h[i].shift = fe * df;
    h[i].dshift = fe / sm * (12.0 * sq - 6.0 * rc6);
    h[i].t = t;
  }
  AtomG* d = nullptr;
  if (natom > 0) {
    if (cudaMallocAsync((void**)&d, sizeof(AtomG) * natom, st) != cudaSuccess) return CMM_ERR_NOMEM;
    if (cudaMemcpyAsync(d, h.data(), sizeof(AtomG) * natom, cudaMemcpyHostToDevice, st) != cudaSuccess) {
      cudaFreeAsync(d, st);
      return CMM_ERR_CUDA;
    }
  }
  const long long npts = (long long)g->n1 * g->n2 * g->n3;
  const int nblk = (int)((npts + ADJ_THREADS - 1) / ADJ_THREADS);
  k_extpot_grad<<<nblk, ADJ_THREADS, 0, st>>>(a, d, d_dV, npts);
  int rc = (cudaPeekAtLastError() == cudaSuccess) ? CMM_OK : CMM_ERR_CUDA;
  if (d) {
    cudaFreeAsync(d, st);
    // the host staging vectors are released on return: wait for the upload
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = CMM_ERR_CUDA;
  }
  return rc;
}

extern "C" int cmm_contract(const double* d_W, long long ldw, int nw, const double* d_D, long long ldd, int K,
                            long long n, double* d_part, int nchunk, void* stream) {
  if (!d_W || !d_D || !d_part || nw < 1 || K < 1 || n < 1 || nchunk < 1 || nchunk > 65535 || nw > 65535)
    return CMM_ERR_ARG;
  k_contract<<<dim3(nchunk, nw), ADJ_THREADS, 0, (cudaStream_t)stream>>>(d_W, ldw, d_D, ldd, K, n, d_part, nchunk);
  return cudaPeekAtLastError() == cudaSuccess ? CMM_OK : CMM_ERR_CUDA;
}

extern "C" int cmm_bicg_vec(int op, long long npts, int batch, const int* d_active, const double* d_rho,
                            const double* d_sc, double c, const double* d_x, const double* d_y, const double* d_a,
                            double* d_out, double* d_out2, const double* d_rhat, double* d_part, int nblk,
                            void* stream) {
  if (op < 0 || op > 4 || npts < 1 || batch < 1 || batch > 65535 || nblk < 1 || nblk > 65535 || !d_out || !d_x)
    return CMM_ERR_ARG;
  if ((op == 0 || op == 1) && !d_rho) return CMM_ERR_ARG;
  if (op == 1 && (!d_y || !d_a || !d_part)) return CMM_ERR_ARG;
  if (op >= 2 && (!d_sc || !d_y)) return CMM_ERR_ARG;
  if (op == 4 && (!d_a || !d_out2 || !d_rhat || !d_part)) return CMM_ERR_ARG;
  VecArgs g{op, npts, d_active, d_rho, d_sc, c, d_x, d_y, d_a, d_out, d_out2, d_rhat, d_part, nblk};
  k_bicg_vec<<<dim3(nblk, batch), ADJ_THREADS, 0, (cudaStream_t)stream>>>(g);
  return cudaPeekAtLastError() == cudaSuccess ? CMM_OK : CMM_ERR_CUDA;
}

extern "C" int cmm_bicg_scalars(int batch, const int* d_active, const double* d_part, int nblk, double* d_sc,
                                int stage, void* stream) {
  if (batch < 1 || !d_part || !d_sc || nblk < 1 || stage < 0 || stage > 2) return CMM_ERR_ARG;
  k_bicg_scalars<<<(batch + 127) / 128, 128, 0, (cudaStream_t)stream>>>(batch, d_active, d_part, nblk, d_sc, stage);
  return cudaPeekAtLastError() == cudaSuccess ? CMM_OK : CMM_ERR_CUDA;
}
