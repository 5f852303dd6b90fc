// Lennard-Jones external potential on the grid.
//
// Arithmetic of get_external_potential / lennard_jones
// (cmmdft/extpot_calculator.py:156-222): for every host atom in file order,
// Lorentz-Berthelot mixed sigma/epsilon, per-axis minimum image
// r -= L * round(r / L), R = sqrt(rx^2 + ry^2 + rz^2 + 1e-16), cut-and-shifted
// 12-6 potential for R < cutoff, accumulated in atom order.  Then the capping
// of FreeEnergy.add_external_potential (cmmdft/functionals.py:247-251).
//
// One thread per grid point; atoms are staged through shared memory in tiles
// with their mixed parameters precomputed.  Products and sums that numpy
// rounds separately use explicit _rn intrinsics so the compiler does not
// contract them into FMAs.
#include <cmath>

#include "cmm_common.cuh"

#define EXT_THREADS 256

struct AtomLJ { double x, y, z, sm, fe, shift; };

// Grid coordinate of index i on an axis of n points:
// numpy.linspace(-0.5, 0.5, n, endpoint=False)[i] = i * (1/n) + (-0.5).
__device__ __forceinline__ double lin_coord(int i, int n) {
  const double step = 1.0 / (double)n;
  return __dadd_rn(__dmul_rn((double)i, step), -0.5);
}

// Cartesian point of grid index (i,j,k): sum_a rvecs[a][b] * g_a (Grid.points).
__device__ __forceinline__ void grid_point(const double* rv, int i, int j, int k, int n1, int n2, int n3,
                                           double* p) {
  const double g0 = lin_coord(i, n1), g1 = lin_coord(j, n2), g2 = lin_coord(k, n3);
#pragma unroll
  for (int b = 0; b < 3; ++b)
    p[b] = __dadd_rn(__dadd_rn(__dmul_rn(rv[0 * 3 + b], g0), __dmul_rn(rv[1 * 3 + b], g1)),
                     __dmul_rn(rv[2 * 3 + b], g2));
}

__device__ __forceinline__ double min_image(double r, double L, double invL) {
  double q = r * invL;
  double f = fabs(q - trunc(q));
  if (fabs(f - 0.5) < 1e-9) q = __ddiv_rn(r, L);  // exact rounding near the half-way case
  return __dsub_rn(r, __dmul_rn(L, rint(q)));
}

struct ExtArgs {
  double rv[9];
  double L[3];
  int n1, n2, n3;
  int natom;
  double cutoff, vcap;
};

__global__ void __launch_bounds__(EXT_THREADS)
k_extpot(ExtArgs a, const AtomLJ* __restrict__ atoms, double* __restrict__ V) {
  __shared__ AtomLJ tile[EXT_THREADS];
  const long long npts = (long long)a.n1 * a.n2 * a.n3;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = idx < npts;
  double p[3] = {0, 0, 0};
  if (live) {
    const int k = (int)(idx % a.n3);
    const int j = (int)((idx / a.n3) % a.n2);
    const int i = (int)(idx / ((long long)a.n3 * a.n2));
    grid_point(a.rv, i, j, k, a.n1, a.n2, a.n3, p);
  }
  const double invL0 = 1.0 / a.L[0], invL1 = 1.0 / a.L[1], invL2 = 1.0 / a.L[2];
  double acc = 0.0;
  for (int base = 0; base < a.natom; base += EXT_THREADS) {
    __syncthreads();
    if (base + threadIdx.x < a.natom) tile[threadIdx.x] = atoms[base + threadIdx.x];
    __syncthreads();
    const int cnt = min(EXT_THREADS, a.natom - base);
    if (!live) continue;
    for (int t = 0; t < cnt; ++t) {
      const AtomLJ at = tile[t];
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
      }
    }
  }
  if (live) {
    double v = acc;
    if (!isfinite(v)) v = a.vcap;
    if (v > a.vcap) v = a.vcap;
    V[idx] = v;
  }
}

extern "C" int cmm_extpot_lj(const cmm_grid* g, const double* d_pos, const int* d_type, int natom,
                             const double* d_type_sig, const double* d_type_eps, int ntype,
                             double guest_sig, double guest_eps, double cutoff, double v_cap,
                             double* d_V, void* stream) {
  if (!g || !d_V || natom < 0 || ntype < 1 || (natom > 0 && (!d_pos || !d_type || !d_type_sig || !d_type_eps)))
    return CMM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  ExtArgs a;
  for (int i = 0; i < 9; ++i) a.rv[i] = g->rvecs[i];
  for (int r = 0; r < 3; ++r) {  // row norms (extpot_calculator.py:202)
    const double* v = g->rvecs + 3 * r;
    a.L[r] = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  }
  a.n1 = g->n1; a.n2 = g->n2; a.n3 = g->n3;
  a.natom = natom;
  a.cutoff = cutoff;
  a.vcap = v_cap;
  // Mixed per-atom parameters, built on the host from the (small) device tables.
  AtomLJ* h = nullptr;
  AtomLJ* d = nullptr;
  if (natom > 0) {
    double* hpos = (double*)malloc(sizeof(double) * 3 * natom);
    int* htyp = (int*)malloc(sizeof(int) * natom);
    double* hs = (double*)malloc(sizeof(double) * ntype);
    double* he = (double*)malloc(sizeof(double) * ntype);
    h = (AtomLJ*)malloc(sizeof(AtomLJ) * natom);
    bool ok = hpos && htyp && hs && he && h;
    ok = ok && cudaMemcpyAsync(hpos, d_pos, sizeof(double) * 3 * natom, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(htyp, d_type, sizeof(int) * natom, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(hs, d_type_sig, sizeof(double) * ntype, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(he, d_type_eps, sizeof(double) * ntype, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
    int rc = ok ? CMM_OK : CMM_ERR_CUDA;
    for (int i = 0; ok && i < natom; ++i) {
      int t = htyp[i];
      if (t < 0 || t >= ntype) { rc = CMM_ERR_ARG; break; }
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
    }
    free(hpos); free(htyp); free(hs); free(he);
    if (rc == CMM_OK && cudaMalloc(&d, sizeof(AtomLJ) * natom) != cudaSuccess) rc = CMM_ERR_NOMEM;
    if (rc == CMM_OK && cudaMemcpyAsync(d, h, sizeof(AtomLJ) * natom, cudaMemcpyHostToDevice, st) != cudaSuccess)
      rc = CMM_ERR_CUDA;
    if (rc != CMM_OK) {
      free(h);
      if (d) cudaFree(d);
      return rc;
    }
  }
  const long long npts = (long long)g->n1 * g->n2 * g->n3;
  const int nblk = (int)((npts + EXT_THREADS - 1) / EXT_THREADS);
  k_extpot<<<nblk, EXT_THREADS, 0, st>>>(a, d, d_V);
  int rc = (cudaPeekAtLastError() == cudaSuccess) ? CMM_OK : CMM_ERR_CUDA;
  if (d) {
    cudaStreamSynchronize(st);
    cudaFree(d);
  }
  free(h);
  return rc;
}
