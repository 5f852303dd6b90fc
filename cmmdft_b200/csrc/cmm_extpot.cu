// Lennard-Jones external potential on the grid.
//
// Arithmetic of get_external_potential / lennard_jones
// (cmmdft/extpot_calculator.py:156-222): for every host atom in file order,
// Lorentz-Berthelot mixed sigma/epsilon, per-axis minimum image
// r -= L * round(r / L), R = sqrt(rx^2 + ry^2 + rz^2 + 1e-16), cut-and-shifted
// 12-6 potential for R < cutoff, accumulated in atom order.  Then the capping
// of FreeEnergy.add_external_potential (cmmdft/functionals.py:247-251).
//
// All-atom form: one thread per grid point; atoms are staged through shared
// memory in tiles with their mixed parameters precomputed.  Products and sums
// that numpy rounds separately use explicit _rn intrinsics so the compiler
// does not contract them into FMAs.  The cell-list form below serves large
// orthorhombic cells.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

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

// ------------------------------------------------ cell-list form ------
// For an orthorhombic cell much larger than the cutoff (the 64 A host at
// 256^3: 16.8 M points x 14,700 atoms, ~3% of the pairs inside 12 A) most
// pairs of the all-atom loop are wasted.  The cell-list form gives every
// block one tile of XT_TX x XT_TY x XT_TZ grid points and stages in shared
// memory only the host atoms that can reach the tile: the atoms are binned
// on the host (bins of edge >= cutoff / 2, stably sorted so each bin keeps
// file order), the block walks the bins that overlap the tile box grown by
// the cutoff, keeps the atoms whose per-axis minimum-image distance from
// the box is below the cutoff (a conservative bound: every atom that the
// exact per-point test accepts passes), and then runs the same per-pair
// arithmetic as k_extpot over that list.  Candidates are compacted with a
// block-wide scan in bin order, so the summation order, and with it every
// bit of the result, is the same from run to run; it differs from the
// reference's file order only by the rounding of the sum.
#define XT_TX 4
#define XT_TY 8
#define XT_TZ 8
#define XT_THREADS (XT_TX * XT_TY * XT_TZ)
#define XT_CAND 768     // staged candidates per round (48 B each)
#define XT_MAXV 1024    // visited bins per tile (a multiple of XT_THREADS)

struct CellArgs {
  ExtArgs a;
  int nb[3];            // bins per axis
  double binw[3];       // bin edge L / nb
  double cut_bound;     // cutoff with a relative margin for the box bound
  int ntile[3];         // tiles per axis
};

// Per-axis minimum-image distance from coordinate x to the interval
// [c - h, c + h] (0 inside), on a circle of length L.
__device__ __forceinline__ double box_axis_dist(double x, double c, double h, double L, double invL) {
  double d = x - c;
  d -= L * rint(d * invL);
  return fmax(fabs(d) - h, 0.0);
}

__global__ void __launch_bounds__(XT_THREADS)
k_extpot_cells(CellArgs c, const AtomLJ* __restrict__ atoms, const int* __restrict__ bin_start, double* __restrict__ V) {
  __shared__ AtomLJ cand[XT_CAND];
  __shared__ int vb_beg[XT_MAXV], vb_off[XT_MAXV];
  __shared__ int wsum[XT_THREADS / 32];
  __shared__ int total_s;
  const ExtArgs& a = c.a;
  const int tid = threadIdx.x;
  // tile and point of this thread
  int t = blockIdx.x;
  const int t3 = t % c.ntile[2]; t /= c.ntile[2];
  const int t2 = t % c.ntile[1];
  const int t1 = t / c.ntile[1];
  const int tz = tid % XT_TZ, ty = (tid / XT_TZ) % XT_TY, tx = tid / (XT_TZ * XT_TY);
  const int i = t1 * XT_TX + tx, j = t2 * XT_TY + ty, k = t3 * XT_TZ + tz;
  const bool live = i < a.n1 && j < a.n2 && k < a.n3;
  double p[3] = {0, 0, 0};
  if (live) grid_point(a.rv, i, j, k, a.n1, a.n2, a.n3, p);
  const double invL[3] = {1.0 / a.L[0], 1.0 / a.L[1], 1.0 / a.L[2]};
  // tile box per axis (orthorhombic: coordinate a of point index q is L_a lin(q))
  const int first[3] = {t1 * XT_TX, t2 * XT_TY, t3 * XT_TZ};
  const int nax[3] = {a.n1, a.n2, a.n3};
  const int ext[3] = {XT_TX, XT_TY, XT_TZ};
  double bc[3], bh[3];
  int blo[3], bcnt[3];
  for (int d = 0; d < 3; ++d) {
    const int last = min(first[d] + ext[d], nax[d]) - 1;
    const double lo = a.rv[d * 3 + d] * lin_coord(first[d], nax[d]);
    const double hi = a.rv[d * 3 + d] * lin_coord(last, nax[d]);
    bc[d] = 0.5 * (lo + hi);
    bh[d] = 0.5 * (hi - lo);
    // bins that overlap [lo - cut, hi + cut] on the circle, one spare on each side
    const double ulo = lo - c.cut_bound + 0.5 * a.L[d], uhi = hi + c.cut_bound + 0.5 * a.L[d];
    int b0 = (int)floor(ulo / c.binw[d]) - 1, b1 = (int)floor(uhi / c.binw[d]) + 1;
    if (b1 - b0 + 1 >= c.nb[d]) { b0 = 0; b1 = c.nb[d] - 1; }
    blo[d] = b0;
    bcnt[d] = b1 - b0 + 1;
  }
  // visited bins in (x, y, z) order: start and atom count, then the running
  // offsets by a block-wide scan (XT_MAXV / XT_THREADS bins per thread)
  const int nvis = bcnt[0] * bcnt[1] * bcnt[2];   // <= XT_MAXV (host check)
  constexpr int PER = XT_MAXV / XT_THREADS;
  int mycnt[PER];
  int mysum = 0;
  for (int q = 0; q < PER; ++q) {
    const int v = tid * PER + q;
    mycnt[q] = 0;
    if (v < nvis) {
      const int z = v % bcnt[2], y = (v / bcnt[2]) % bcnt[1], x = v / (bcnt[2] * bcnt[1]);
      const int bx = ((blo[0] + x) % c.nb[0] + c.nb[0]) % c.nb[0];
      const int by = ((blo[1] + y) % c.nb[1] + c.nb[1]) % c.nb[1];
      const int bz = ((blo[2] + z) % c.nb[2] + c.nb[2]) % c.nb[2];
      const int bin = (bx * c.nb[1] + by) * c.nb[2] + bz;
      vb_beg[v] = bin_start[bin];
      mycnt[q] = bin_start[bin + 1] - bin_start[bin];
    }
    mysum += mycnt[q];
  }
  {
    const int lane = tid & 31, w = tid >> 5;
    int incl = mysum;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    int before = 0, tot = 0;
    for (int q = 0; q < XT_THREADS / 32; ++q) {
      before += (q < w) ? wsum[q] : 0;
      tot += wsum[q];
    }
    int off = before + incl - mysum;
    for (int q = 0; q < PER; ++q) {
      const int v = tid * PER + q;
      if (v < nvis) vb_off[v] = off;
      off += mycnt[q];
    }
    if (tid == 0) total_s = tot;
    __syncthreads();
  }
  const int total = total_s;
  const double cb2 = c.cut_bound * c.cut_bound;
  double acc = 0.0;
  int ncand = 0;
  for (int base = 0; base < total; base += XT_THREADS) {
    const int v = base + tid;
    bool take = false;
    AtomLJ at;
    if (v < total) {
      int lo = 0, hi = nvis - 1;   // last visited bin with vb_off <= v
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (vb_off[mid] <= v) lo = mid; else hi = mid - 1;
      }
      at = atoms[vb_beg[lo] + (v - vb_off[lo])];
      const double dx = box_axis_dist(at.x, bc[0], bh[0], a.L[0], invL[0]);
      const double dy = box_axis_dist(at.y, bc[1], bh[1], a.L[1], invL[1]);
      const double dz = box_axis_dist(at.z, bc[2], bh[2], a.L[2], invL[2]);
      take = dx * dx + dy * dy + dz * dz < cb2;
    }
    // block-wide exclusive scan of `take`, in thread order
    const unsigned bal = __ballot_sync(0xffffffffu, take);
    const int lane = tid & 31, w = tid >> 5;
    if (lane == 0) wsum[w] = __popc(bal);   // (read by every thread before the last barrier)
    __syncthreads();
    int before = 0, sum = 0;
    for (int q = 0; q < XT_THREADS / 32; ++q) {
      before += (q < w) ? wsum[q] : 0;
      sum += wsum[q];
    }
    const int pos = ncand + before + __popc(bal & ((1u << lane) - 1u));
    if (take) cand[pos] = at;
    ncand += sum;
    __syncthreads();
    const bool flush = (ncand > XT_CAND - XT_THREADS) || (base + XT_THREADS >= total);
    if (flush) {
      if (live) {
        for (int q = 0; q < ncand; ++q) {
          const AtomLJ atq = cand[q];
          const double rx = min_image(__dsub_rn(p[0], atq.x), a.L[0], invL[0]);
          const double ry = min_image(__dsub_rn(p[1], atq.y), a.L[1], invL[1]);
          const double rz = min_image(__dsub_rn(p[2], atq.z), a.L[2], invL[2]);
          const double r2 =
              __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz)), 1e-16);
          const double R = sqrt(r2);
          if (R < a.cutoff) {
            const double qq = __ddiv_rn(atq.sm, R);
            const double q2 = __dmul_rn(qq, qq);
            const double r6 = __dmul_rn(__dmul_rn(q2, q2), q2);
            const double r12 = __dmul_rn(r6, r6);
            const double vv = __dsub_rn(__dmul_rn(atq.fe, __dsub_rn(r12, r6)), atq.shift);
            acc = __dadd_rn(acc, vv);
          }
        }
      }
      ncand = 0;
      __syncthreads();
    }
  }
  if (live) {
    double vv = acc;
    if (!isfinite(vv)) vv = a.vcap;
    if (vv > a.vcap) vv = a.vcap;
    V[((size_t)i * a.n2 + j) * a.n3 + k] = vv;
  }
}

// Bins of the cell-list form, or 0 when the all-atom form is the better
// choice: the cell must be orthorhombic, every axis at least 3 bins of edge
// >= cutoff / 2, the visited bins of one tile within XT_MAXV, and the staged
// atoms a small share of all (mode 1 forces the cell list where legal).
static int extpot_cell_bins(const cmm_grid* g, const ExtArgs& a, int natom, int mode, int nb[3]) {
  const double* rv = g->rvecs;
  if (rv[1] != 0 || rv[2] != 0 || rv[3] != 0 || rv[5] != 0 || rv[6] != 0 || rv[7] != 0) return 0;
  if (!(a.cutoff > 0) || natom < 1) return 0;
  const int nax[3] = {a.n1, a.n2, a.n3};
  const int ext[3] = {XT_TX, XT_TY, XT_TZ};
  double frac = 1.0;
  long long vis = 1;
  for (int d = 0; d < 3; ++d) {
    nb[d] = (int)floor(a.L[d] / (0.5 * a.cutoff));
    if (nb[d] < 3) return 0;
    if (nb[d] > 256) nb[d] = 256;
    const double binw = a.L[d] / nb[d];
    const double box = a.L[d] * ext[d] / nax[d];
    // the kernel visits floor(uhi/w) - floor(ulo/w) + 3 <= (uhi - ulo)/w + 4 bins
    const int cnt = std::min(nb[d], (int)ceil((box + 2 * a.cutoff) / binw) + 4);
    vis *= cnt;
    frac *= std::min(1.0, ((box + 2 * a.cutoff) / binw + 3) / nb[d]);   // expected share of the atoms
  }
  if (vis > XT_MAXV) return 0;
  if (mode == 1) return 1;
  return (natom >= 1024 && frac < 0.5) ? 1 : 0;
}

static int g_extpot_mode = 0;   // 0 by size, 1 cell list where legal, 2 all atoms

extern "C" int cmm_extpot_set_mode(int mode) {
  if (mode < 0 || mode > 2) return CMM_ERR_ARG;
  g_extpot_mode = mode;
  return CMM_OK;
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
    if (rc != CMM_OK) {
      free(h);
      return rc;
    }
  }
  int nb[3] = {0, 0, 0};
  const bool cells = natom > 0 && g_extpot_mode != 2 && extpot_cell_bins(g, a, natom, g_extpot_mode, nb);
  std::vector<int> bin_start;
  if (cells) {  // stable sort of the table by bin: each bin keeps file order
    const int nbin = nb[0] * nb[1] * nb[2];
    std::vector<int> bin_of(natom), cnt(nbin + 1, 0);
    for (int q = 0; q < natom; ++q) {
      const double x[3] = {h[q].x, h[q].y, h[q].z};
      int bi[3];
      for (int ax = 0; ax < 3; ++ax) {
        double w = x[ax] - a.L[ax] * rint(x[ax] / a.L[ax]);      // [-L/2, L/2]
        int b = (int)floor((w + 0.5 * a.L[ax]) / (a.L[ax] / nb[ax]));
        bi[ax] = b < 0 ? 0 : (b >= nb[ax] ? nb[ax] - 1 : b);
      }
      bin_of[q] = (bi[0] * nb[1] + bi[1]) * nb[2] + bi[2];
      cnt[bin_of[q] + 1] += 1;
    }
    for (int b = 0; b < nbin; ++b) cnt[b + 1] += cnt[b];
    bin_start = cnt;
    std::vector<AtomLJ> sorted(natom);
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int q = 0; q < natom; ++q) sorted[fill[bin_of[q]]++] = h[q];
    std::memcpy(h, sorted.data(), sizeof(AtomLJ) * natom);
  }
  int* d_bins = nullptr;
  int rc = CMM_OK;
  if (natom > 0) {
    const size_t abytes = sizeof(AtomLJ) * natom, bbytes = sizeof(int) * bin_start.size();
    if (cudaMalloc(&d, abytes + bbytes) != cudaSuccess) rc = CMM_ERR_NOMEM;
    if (rc == CMM_OK && cudaMemcpyAsync(d, h, abytes, cudaMemcpyHostToDevice, st) != cudaSuccess) rc = CMM_ERR_CUDA;
    if (rc == CMM_OK && cells) {
      d_bins = (int*)((char*)d + abytes);
      if (cudaMemcpyAsync(d_bins, bin_start.data(), bbytes, cudaMemcpyHostToDevice, st) != cudaSuccess)
        rc = CMM_ERR_CUDA;
    }
  }
  if (rc == CMM_OK) {
    if (cells) {
      CellArgs c;
      c.a = a;
      for (int ax = 0; ax < 3; ++ax) {
        c.nb[ax] = nb[ax];
        c.binw[ax] = a.L[ax] / nb[ax];
      }
      c.cut_bound = cutoff * (1.0 + 1e-9) + 1e-9;
      c.ntile[0] = cmm_div_up(g->n1, XT_TX);
      c.ntile[1] = cmm_div_up(g->n2, XT_TY);
      c.ntile[2] = cmm_div_up(g->n3, XT_TZ);
      const long long nt = (long long)c.ntile[0] * c.ntile[1] * c.ntile[2];
      k_extpot_cells<<<(unsigned)nt, XT_THREADS, 0, st>>>(c, d, d_bins, d_V);
    } else {
      const long long npts = (long long)g->n1 * g->n2 * g->n3;
      const int nblk = (int)((npts + EXT_THREADS - 1) / EXT_THREADS);
      k_extpot<<<nblk, EXT_THREADS, 0, st>>>(a, d, d_V);
    }
    rc = (cudaPeekAtLastError() == cudaSuccess) ? CMM_OK : CMM_ERR_CUDA;
  }
  if (d) {
    cudaStreamSynchronize(st);
    cudaFree(d);
  }
  free(h);
  return rc;
}

// ------------------------------------------- orientational average ------
// Effective potential of a rigid multi-site guest at every grid point p
// (effective_potential_vectorized, cmmdft/extpot_calculator.py:569-613,
// as generate_effective_potential calls it, :616-655):
//   neutral_k = pos_k + p, COM = sum_k m_k neutral_k / M, rel_k = neutral_k - COM,
//   site k of rotation r at R_r rel_k + COM,
//   V_k,r = the LJ sum of that site over the host atoms with the mixed
//           parameters of the site's type (the arithmetic of k_extpot),
//   pot_r = sum_k V_k,r,   a_r = -beta pot_r,
//   V_eff(p) = -logsumexp(a, b=w) / beta, NaN -> v_limit.
// The reference stores V_k,r in float32 and sums and scales there (a
// float32 array times a Python float stays float32); the kernel rounds to
// float32 at the same points.  The log-sum-exp follows scipy's form: the
// largest a_r is taken out, m = the summed weights of the entries equal to
// it, s = sum of the others' w exp(a - a_max) / m, result log1p(s) + log(m)
// + a_max, and the direct log(sum w exp(a)) where that is not finite.
// One block per grid point; the block's threads take the rotations; host
// atoms are staged in shared memory tiles; a_r lives in dynamic shared
// memory between the potential pass and the reductions.
#define ROT_THREADS 256
#define ROT_MAX_SITES 8
#define ROT_MAX_PAIRTYPES 128
#define ROT_MAX_ROT 6144          // 48 KB of a_r in shared memory

struct RotArgs {
  ExtArgs a;
  int nsite, nhtype, nrot;
  double beta, vlimit, mtot;
  double pos[ROT_MAX_SITES][3];   // guest atoms in the guest's own frame
  double mass[ROT_MAX_SITES];
};
struct MixLJ { double sm, fe, shift; };
struct HostAtom { double x, y, z; int t; int pad; };

__device__ __forceinline__ double lj_pair(const double* q, const HostAtom& at, const MixLJ& mx, const ExtArgs& a,
                                          const double* invL) {
  const double rx = min_image(__dsub_rn(q[0], at.x), a.L[0], invL[0]);
  const double ry = min_image(__dsub_rn(q[1], at.y), a.L[1], invL[1]);
  const double rz = min_image(__dsub_rn(q[2], at.z), a.L[2], invL[2]);
  const double r2 = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz)), 1e-16);
  const double R = sqrt(r2);
  if (!(R < a.cutoff)) return 0.0;
  const double qq = __ddiv_rn(mx.sm, R);
  const double q2 = __dmul_rn(qq, qq);
  const double r6 = __dmul_rn(__dmul_rn(q2, q2), q2);
  const double r12 = __dmul_rn(r6, r6);
  return __dsub_rn(__dmul_rn(mx.fe, __dsub_rn(r12, r6)), mx.shift);
}

// Block-wide reduction of one double (op 0: max, 1: sum) into every thread.
__device__ __forceinline__ double block_reduce(double v, int op, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    const double u = __shfl_xor_sync(0xffffffffu, v, o);
    v = op ? v + u : fmax(v, u);
  }
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double r = red[0];
  for (int q = 1; q < nw; ++q) r = op ? r + red[q] : fmax(r, red[q]);
  return r;
}

// The guest at grid point (i,j,k) in its centre-of-mass frame: frame[s] =
// pos_s + p - COM, frame[ROT_MAX_SITES] = COM (threads 0-2, one axis each).
__device__ __forceinline__ void rot_frame(const RotArgs& c, int i, int j, int k, double (*frame)[3]) {
  if (threadIdx.x >= 3) return;
  const ExtArgs& a = c.a;
  const int d = threadIdx.x;
  double p[3];
  grid_point(a.rv, i, j, k, a.n1, a.n2, a.n3, p);
  double acc = 0.0;
  for (int s = 0; s < c.nsite; ++s) acc = __dadd_rn(acc, __dmul_rn(__dadd_rn(c.pos[s][d], p[d]), c.mass[s]));
  const double com = __ddiv_rn(acc, c.mtot);
  for (int s = 0; s < c.nsite; ++s) frame[s][d] = __dsub_rn(__dadd_rn(c.pos[s][d], p[d]), com);
  frame[ROT_MAX_SITES][d] = com;
}

// Site s turned by R about the centre of mass: R rel_s + COM.
__device__ __forceinline__ void rot_site(const double* R, const double (*frame)[3], int s, double* q) {
#pragma unroll
  for (int d = 0; d < 3; ++d)
    q[d] = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(R[3 * d], frame[s][0]), __dmul_rn(R[3 * d + 1], frame[s][1])),
                               __dmul_rn(R[3 * d + 2], frame[s][2])), frame[ROT_MAX_SITES][d]);
}

// -logsumexp(a, b=w) / beta over the block's a_r (scipy's form), NaN -> v_limit.
__device__ void rot_finish(const RotArgs& c, const double* s_a, const double* __restrict__ w, double* red,
                           double* out_v) {
  double amax = -INFINITY;
  for (int r = threadIdx.x; r < c.nrot; r += blockDim.x) amax = fmax(amax, s_a[r]);
  amax = block_reduce(amax, 0, red);
  double m = 0.0, sm = 0.0, direct = 0.0;
  for (int r = threadIdx.x; r < c.nrot; r += blockDim.x) {
    const double ar = s_a[r];
    direct += w[r] * exp(ar);
    if (ar == amax) m += w[r];
    else sm += w[r] * exp(ar - amax);
  }
  m = block_reduce(m, 1, red);
  sm = block_reduce(sm, 1, red);
  direct = block_reduce(direct, 1, red);
  if (threadIdx.x == 0) {
    if (sm != 0.0) sm = sm / m;
    double out = log1p(sm) + log(m) + amax;
    if (!isfinite(out)) out = log(direct);
    double res = -out / c.beta;
    if (res != res) res = c.vlimit;
    *out_v = res;
  }
}

// The direct kernel runs 128 threads a block: 342 or 550 rotations fill 89 %
// or 86 % of its thread rounds (67 % and 72 % with 256).  NS: the sites a
// thread holds in registers (3 covers rigid CO2 and N2, 90 registers, 5
// blocks per SM; 8 any guest).
#define ROT_DIRECT_THREADS 128

template <int NS>
__global__ void __launch_bounds__(ROT_DIRECT_THREADS, NS <= 3 ? 5 : 4)
k_extpot_rot(RotArgs c, const HostAtom* __restrict__ atoms, const MixLJ* __restrict__ mix,
             const double* __restrict__ rot, const double* __restrict__ w, double* __restrict__ V,
             long long idx0, double* __restrict__ scratch) {
  __shared__ HostAtom tile[ROT_DIRECT_THREADS];
  __shared__ MixLJ smix[ROT_MAX_PAIRTYPES];
  __shared__ double frame[ROT_MAX_SITES + 1][3];   // rel_k, then COM
  __shared__ double red[32];
  extern __shared__ double s_dyn[];
  // a_r, r < nrot: in shared memory, or this block's row of a global scratch
  double* s_a = scratch ? scratch + (size_t)blockIdx.x * c.nrot : s_dyn;
  const ExtArgs& a = c.a;
  const long long idx = idx0 + blockIdx.x;
  const int k = (int)(idx % a.n3), j = (int)((idx / a.n3) % a.n2), i = (int)(idx / ((long long)a.n3 * a.n2));
  for (int t = threadIdx.x; t < c.nsite * c.nhtype; t += blockDim.x) smix[t] = mix[t];
  rot_frame(c, i, j, k, frame);
  __syncthreads();
  const double invL[3] = {1.0 / a.L[0], 1.0 / a.L[1], 1.0 / a.L[2]};
  const float fnb = __double2float_rn(-c.beta);
  for (int r0 = 0; r0 < c.nrot; r0 += blockDim.x) {
    const int r = r0 + threadIdx.x;
    double q[NS][3];
    double v[NS];
    if (r < c.nrot) {
      const double* R = rot + (size_t)r * 9;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        v[s] = 0.0;
        if (s < c.nsite) rot_site(R, frame, s, q[s]);
      }
    }
    for (int base = 0; base < a.natom; base += ROT_DIRECT_THREADS) {
      __syncthreads();
      if (base + threadIdx.x < a.natom) tile[threadIdx.x] = atoms[base + threadIdx.x];
      __syncthreads();
      const int cnt = min(ROT_DIRECT_THREADS, a.natom - base);
      if (r >= c.nrot) continue;
      for (int t = 0; t < cnt; ++t) {
        const HostAtom at = tile[t];
#pragma unroll
        for (int s = 0; s < NS; ++s)
          if (s < c.nsite) v[s] = __dadd_rn(v[s], lj_pair(q[s], at, smix[s * c.nhtype + at.t], a, invL));
      }
    }
    if (r < c.nrot) {
      float pot = 0.0f;
#pragma unroll
      for (int s = 0; s < NS; ++s)
        if (s < c.nsite) pot = __fadd_rn(pot, __double2float_rn(v[s]));
      s_a[r] = (double)__fmul_rn(fnb, pot);
    }
  }
  __syncthreads();
  rot_finish(c, s_a, w, red, V + idx);
}

// Launch a rotation-average kernel over npts grid points: a_r in dynamic
// shared memory when nrot fits (ROT_MAX_ROT), else in a global scratch of
// one row per block, the points taken in chunks that keep it under 1 GiB
// but never below 8 blocks per SM (7.3 GB at the largest Lebedev set).
template <class Launch>
static int rot_launch(long long npts, int nrot, const void* kern, cudaStream_t st, Launch launch) {
  if (npts <= 0) return CMM_OK;
  if (nrot <= ROT_MAX_ROT) {
    const size_t dyn = sizeof(double) * (size_t)nrot;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn) != cudaSuccess)
      return CMM_ERR_CUDA;
    for (long long p0 = 0; p0 < npts; p0 += 0x7fffffffLL)
      launch((unsigned)std::min(npts - p0, 0x7fffffffLL), dyn, p0, (double*)nullptr);
    return (cudaPeekAtLastError() == cudaSuccess) ? CMM_OK : CMM_ERR_CUDA;
  }
  const long long chunk = std::min(npts, std::max(148LL * 8, (1LL << 30) / (8LL * nrot)));
  double* scr = nullptr;
  if (cudaMallocAsync((void**)&scr, sizeof(double) * (size_t)chunk * nrot, st) != cudaSuccess) return CMM_ERR_NOMEM;
  for (long long p0 = 0; p0 < npts; p0 += chunk) launch((unsigned)std::min(chunk, npts - p0), 0, p0, scr);
  const int rc = (cudaPeekAtLastError() == cudaSuccess) ? CMM_OK : CMM_ERR_CUDA;
  cudaFreeAsync(scr, st);
  return rc;
}

extern "C" int cmm_extpot_rot(const cmm_grid* g, const double* d_pos, const int* d_type, int natom,
                              const double* d_type_sig, const double* d_type_eps, int ntype, const double* guest_pos,
                              const double* guest_mass, const double* guest_sig, const double* guest_eps, int nsite,
                              const double* d_rot, const double* d_w, int nrot, double cutoff, double beta,
                              double v_limit, double* d_V, void* stream) {
  if (!g || !d_V || !d_rot || !d_w || !guest_pos || !guest_mass || !guest_sig || !guest_eps) return CMM_ERR_ARG;
  if (natom < 0 || ntype < 1 || nsite < 1 || nrot < 1 || !(beta > 0) ||
      (natom > 0 && (!d_pos || !d_type || !d_type_sig || !d_type_eps)))
    return CMM_ERR_ARG;
  if (nsite > ROT_MAX_SITES || nsite * ntype > ROT_MAX_PAIRTYPES) return CMM_ERR_UNSUPPORTED;
  cudaStream_t st = (cudaStream_t)stream;
  RotArgs c;
  memset(&c, 0, sizeof(c));
  for (int q = 0; q < 9; ++q) c.a.rv[q] = g->rvecs[q];
  for (int r = 0; r < 3; ++r) {
    const double* v = g->rvecs + 3 * r;
    c.a.L[r] = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  }
  c.a.n1 = g->n1; c.a.n2 = g->n2; c.a.n3 = g->n3;
  c.a.natom = natom;
  c.a.cutoff = cutoff;
  c.nsite = nsite; c.nhtype = ntype; c.nrot = nrot;
  c.beta = beta; c.vlimit = v_limit;
  double mt = 0.0;
  for (int q = 0; q < nsite; ++q) {
    for (int d = 0; d < 3; ++d) c.pos[q][d] = guest_pos[3 * q + d];
    c.mass[q] = guest_mass[q];
    mt += guest_mass[q];
  }
  if (!(mt > 0)) return CMM_ERR_ARG;
  c.mtot = mt;
  std::vector<HostAtom> h(natom > 0 ? natom : 1);
  std::vector<MixLJ> mx((size_t)nsite * ntype);
  if (natom > 0) {
    std::vector<double> hpos(3 * (size_t)natom), hs(ntype), he(ntype);
    std::vector<int> htyp(natom);
    bool ok = cudaMemcpyAsync(hpos.data(), d_pos, sizeof(double) * 3 * natom, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(htyp.data(), d_type, sizeof(int) * natom, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(hs.data(), d_type_sig, sizeof(double) * ntype, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(he.data(), d_type_eps, sizeof(double) * ntype, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) return CMM_ERR_CUDA;
    for (int q = 0; q < natom; ++q) {
      if (htyp[q] < 0 || htyp[q] >= ntype) return CMM_ERR_ARG;
      h[q].x = hpos[3 * q]; h[q].y = hpos[3 * q + 1]; h[q].z = hpos[3 * q + 2];
      h[q].t = htyp[q]; h[q].pad = 0;
    }
    // mixed parameters per (site, host type), formed as cmm_extpot_lj forms them
    for (int sI = 0; sI < nsite; ++sI)
      for (int t = 0; t < ntype; ++t) {
        volatile double sm = 0.5 * (hs[t] + guest_sig[sI]);
        volatile double em = sqrt(he[t] * guest_eps[sI]);
        volatile double qq = sm / cutoff;
        volatile double q2 = qq * qq;
        volatile double rc6 = q2 * q2 * q2;
        volatile double fe = 4.0 * em;
        volatile double sq = rc6 * rc6;
        volatile double df = sq - rc6;
        mx[(size_t)sI * ntype + t] = MixLJ{sm, fe, fe * df};
      }
  }
  const long long npts = (long long)g->n1 * g->n2 * g->n3;
  void* d = nullptr;
  const size_t ab = sizeof(HostAtom) * h.size(), mb = sizeof(MixLJ) * mx.size();
  if (cudaMalloc(&d, ab + mb) != cudaSuccess) return CMM_ERR_NOMEM;
  HostAtom* da = (HostAtom*)d;
  MixLJ* dm = (MixLJ*)((char*)d + ab);
  int rc = CMM_OK;
  if (cudaMemcpyAsync(da, h.data(), ab, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(dm, mx.data(), mb, cudaMemcpyHostToDevice, st) != cudaSuccess)
    rc = CMM_ERR_CUDA;
  if (rc == CMM_OK)
    rc = (nsite <= 3)
             ? rot_launch(npts, nrot, (const void*)k_extpot_rot<3>, st,
                          [&](unsigned nb, size_t dyn, long long p0, double* scr) {
                            k_extpot_rot<3><<<nb, ROT_DIRECT_THREADS, dyn, st>>>(c, da, dm, d_rot, d_w, d_V, p0, scr);
                          })
             : rot_launch(npts, nrot, (const void*)k_extpot_rot<ROT_MAX_SITES>, st,
                          [&](unsigned nb, size_t dyn, long long p0, double* scr) {
                            k_extpot_rot<ROT_MAX_SITES><<<nb, ROT_DIRECT_THREADS, dyn, st>>>(c, da, dm, d_rot, d_w,
                                                                                            d_V, p0, scr);
                          });
  if (cudaStreamSynchronize(st) != cudaSuccess) rc = CMM_ERR_CUDA;
  cudaFree(d);
  return rc;
}

// ------------------------------------- tricubic-interpolated average ------
// ExternalPotential.generate_potential(interpolate=True)
// (cmmdft/functionals.py:1032-1055): per guest atom type, the LJ potential
// and its derivatives on a fine grid (get_external_potential_derivatives,
// cmmdft/extpot_calculator.py:264-338), then the orientational average with
// each site potential interpolated tricubically from its type's grid
// (Interpolator.tricubic_interpolation, :391-549).

// Eight channels at every point of an n1 x n2 x n3 grid over the cell: V,
// dV/dx, dV/dy, dV/dz, d2V/dxdy, d2V/dxdz, d2V/dydz, d3V/dxdydz, summed over
// host atoms with the radial factors of lennard_jones(derivative=True):
//   dV = 24 eps (r6 - 2 r12) / R^2, ddV = 96 eps (7 r12 - 2 r6) / R^4,
//   dddV = 384 eps (5 r6 - 28 r12) / R^6   (r6 = (sigma/R)^6),
// dV/dx += dV rx, d2V/dxdy += ddV rx ry, d3V/dxdydz += dddV rx ry rz; then
// V and the first derivatives clipped to +-1e6 kJ/mol, the cross
// derivatives zeroed where V exceeded it, and every derivative scaled to the
// unit cube (times the spacings of its axes).  Output [8][n1][n2][n3].
struct DerivArgs {
  double rv[9];
  double L[3];
  double sp[3];
  int n1, n2, n3, natom;
  double cutoff, vmax;
};
struct AtomLJD { double x, y, z, sm, fe, shift, e24; };

__global__ void __launch_bounds__(EXT_THREADS)
k_extpot_deriv(DerivArgs a, const AtomLJD* __restrict__ atoms, double* __restrict__ out) {
  __shared__ AtomLJD tile[EXT_THREADS];
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
  const double invL[3] = {1.0 / a.L[0], 1.0 / a.L[1], 1.0 / a.L[2]};
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int base = 0; base < a.natom; base += EXT_THREADS) {
    __syncthreads();
    if (base + threadIdx.x < a.natom) tile[threadIdx.x] = atoms[base + threadIdx.x];
    __syncthreads();
    const int cnt = min(EXT_THREADS, a.natom - base);
    if (!live) continue;
    for (int t = 0; t < cnt; ++t) {
      const AtomLJD at = tile[t];
      const double rx = min_image(__dsub_rn(p[0], at.x), a.L[0], invL[0]);
      const double ry = min_image(__dsub_rn(p[1], at.y), a.L[1], invL[1]);
      const double rz = min_image(__dsub_rn(p[2], at.z), a.L[2], invL[2]);
      const double r2 = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz)), 1e-16);
      const double R = sqrt(r2);
      if (!(R < a.cutoff)) continue;
      const double q = __ddiv_rn(at.sm, R);
      const double q2 = __dmul_rn(q, q);
      const double r6 = __dmul_rn(__dmul_rn(q2, q2), q2);
      const double r12 = __dmul_rn(r6, r6);
      const double RR = __dmul_rn(R, R), R4 = __dmul_rn(RR, RR), R6 = __dmul_rn(R4, RR);
      const double v = __dsub_rn(__dmul_rn(at.fe, __dsub_rn(r12, r6)), at.shift);
      const double dv = __ddiv_rn(__dmul_rn(at.e24, __dsub_rn(r6, __dmul_rn(2.0, r12))), RR);
      const double ddv = __ddiv_rn(__dmul_rn(__dmul_rn(4.0, at.e24), __dsub_rn(__dmul_rn(7.0, r12), __dmul_rn(2.0, r6))), R4);
      const double dddv = __ddiv_rn(__dmul_rn(__dmul_rn(16.0, at.e24), __dsub_rn(__dmul_rn(5.0, r6), __dmul_rn(28.0, r12))), R6);
      acc[0] = __dadd_rn(acc[0], v);
      acc[1] = __dadd_rn(acc[1], __dmul_rn(dv, rx));
      acc[2] = __dadd_rn(acc[2], __dmul_rn(dv, ry));
      acc[3] = __dadd_rn(acc[3], __dmul_rn(dv, rz));
      acc[4] = __dadd_rn(acc[4], __dmul_rn(__dmul_rn(ddv, rx), ry));
      acc[5] = __dadd_rn(acc[5], __dmul_rn(__dmul_rn(ddv, rx), rz));
      acc[6] = __dadd_rn(acc[6], __dmul_rn(__dmul_rn(ddv, ry), rz));
      acc[7] = __dadd_rn(acc[7], __dmul_rn(__dmul_rn(__dmul_rn(dddv, rx), ry), rz));
    }
  }
  if (!live) return;
  const bool big = acc[0] > a.vmax;
#pragma unroll
  for (int c = 0; c < 4; ++c) {       // np.clip keeps NaN
    double x = acc[c];
    if (x > a.vmax) x = a.vmax;
    else if (x < -a.vmax) x = -a.vmax;
    acc[c] = x;
  }
  if (big) acc[4] = acc[5] = acc[6] = acc[7] = 0.0;
  const double f[8] = {1.0, a.sp[0], a.sp[1], a.sp[2], __dmul_rn(a.sp[0], a.sp[1]), __dmul_rn(a.sp[0], a.sp[2]),
                       __dmul_rn(a.sp[1], a.sp[2]), __dmul_rn(__dmul_rn(a.sp[0], a.sp[1]), a.sp[2])};
#pragma unroll
  for (int c = 0; c < 8; ++c) out[(size_t)c * npts + idx] = (c == 0) ? acc[0] : __dmul_rn(acc[c], f[c]);
}

extern "C" int cmm_extpot_lj_deriv(const double* rvecs, int n1, int n2, int n3, const double* spacings,
                                   const double* d_pos, const int* d_type, int natom, const double* d_type_sig,
                                   const double* d_type_eps, int ntype, double guest_sig, double guest_eps,
                                   double cutoff, double v_max, double* d_out, void* stream) {
  if (!rvecs || !spacings || !d_out || n1 < 1 || n2 < 1 || n3 < 1 || natom < 0 || ntype < 1) return CMM_ERR_ARG;
  if (natom > 0 && (!d_pos || !d_type || !d_type_sig || !d_type_eps)) return CMM_ERR_ARG;
  const long long npts = (long long)n1 * n2 * n3;
  if (npts > ((long long)1 << 40)) return CMM_ERR_SHAPE;
  cudaStream_t st = (cudaStream_t)stream;
  DerivArgs a;
  memset(&a, 0, sizeof(a));
  for (int q = 0; q < 9; ++q) a.rv[q] = rvecs[q];
  for (int r = 0; r < 3; ++r) {
    const double* v = rvecs + 3 * r;
    a.L[r] = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    a.sp[r] = spacings[r];
  }
  a.n1 = n1; a.n2 = n2; a.n3 = n3; a.natom = natom;
  a.cutoff = cutoff; a.vmax = v_max;
  std::vector<AtomLJD> h(natom > 0 ? natom : 1);
  if (natom > 0) {
    std::vector<double> hpos(3 * (size_t)natom), hs(ntype), he(ntype);
    std::vector<int> htyp(natom);
    bool ok = cudaMemcpyAsync(hpos.data(), d_pos, sizeof(double) * 3 * natom, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(htyp.data(), d_type, sizeof(int) * natom, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(hs.data(), d_type_sig, sizeof(double) * ntype, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(he.data(), d_type_eps, sizeof(double) * ntype, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) return CMM_ERR_CUDA;
    for (int q = 0; q < natom; ++q) {
      const int t = htyp[q];
      if (t < 0 || t >= ntype) return CMM_ERR_ARG;
      volatile double sm = 0.5 * (hs[t] + guest_sig);
      volatile double em = sqrt(he[t] * guest_eps);
      volatile double qq = sm / cutoff;
      volatile double q2 = qq * qq;
      volatile double rc6 = q2 * q2 * q2;
      volatile double fe = 4.0 * em;
      volatile double sq = rc6 * rc6;
      volatile double df = sq - rc6;
      volatile double e24 = 24.0 * em;
      h[q] = AtomLJD{hpos[3 * q], hpos[3 * q + 1], hpos[3 * q + 2], sm, fe, fe * df, e24};
    }
  }
  void* d = nullptr;
  const size_t ab = sizeof(AtomLJD) * h.size();
  if (cudaMalloc(&d, ab) != cudaSuccess) return CMM_ERR_NOMEM;
  int rc = CMM_OK;
  if (cudaMemcpyAsync(d, h.data(), ab, cudaMemcpyHostToDevice, st) != cudaSuccess) rc = CMM_ERR_CUDA;
  if (rc == CMM_OK) {
    k_extpot_deriv<<<cmm_div_up(npts, EXT_THREADS), EXT_THREADS, 0, st>>>(a, (const AtomLJD*)d, d_out);
    rc = (cudaPeekAtLastError() == cudaSuccess) ? CMM_OK : CMM_ERR_CUDA;
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) rc = CMM_ERR_CUDA;
  cudaFree(d);
  return rc;
}

// Tricubic interpolation of one channel set (Interpolator.
// tricubic_interpolation): the cell of q by floor((q - origin) / spacing),
// the 8 corners wrapped periodically, and the tricubic polynomial fixed by
// the 64 corner values -- the tensor product of cubic Hermite interpolants
// on [0, 1] (exactly what the reference's 64 x 64 coefficient matrix
// encodes), evaluated as sum over corners and channels of value x basis.
struct InterpArgs {
  int f[3];                       // fine-grid points per axis
  double origin[3], spacing[3];   // the interpolator's origin and spacing
  int site_tab[ROT_MAX_SITES];    // channel table of each site
};

__device__ __forceinline__ void hermite4(double t, double* h) {
  const double u = 1.0 - t;
  h[0] = u * u * (1.0 + 2.0 * t);   // value at 0
  h[1] = t * u * u;                 // slope at 0
  h[2] = t * t * (3.0 - 2.0 * t);   // value at 1
  h[3] = t * t * (t - 1.0);         // slope at 1
}

__device__ double tricubic_at(const double* __restrict__ tab, long long npts, const InterpArgs& ia,
                              const double* q) {
  double hx[4], hy[4], hz[4], r[3];
  long long i0[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double s = __ddiv_rn(__dsub_rn(q[d], ia.origin[d]), ia.spacing[d]);
    const double fl = floor(s);
    r[d] = __dsub_rn(s, fl);
    i0[d] = (long long)fl;
  }
  hermite4(r[0], hx);
  hermite4(r[1], hy);
  hermite4(r[2], hz);
  // channel d has derivative orders (ox, oy, oz): V, x, y, z, xy, xz, yz, xyz
  const int ox[8] = {0, 1, 0, 0, 1, 1, 0, 1}, oy[8] = {0, 0, 1, 0, 1, 0, 1, 1}, oz[8] = {0, 0, 0, 1, 0, 1, 1, 1};
  double res = 0.0;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int cx = c & 1, cy = (c >> 1) & 1, cz = (c >> 2) & 1;
    long long ix = (i0[0] + cx) % ia.f[0], iy = (i0[1] + cy) % ia.f[1], iz = (i0[2] + cz) % ia.f[2];
    if (ix < 0) ix += ia.f[0];
    if (iy < 0) iy += ia.f[1];
    if (iz < 0) iz += ia.f[2];
    const long long base = (ix * ia.f[1] + iy) * ia.f[2] + iz;
#pragma unroll
    for (int d = 0; d < 8; ++d)
      res += __ldg(tab + (size_t)d * npts + base) * (hx[2 * cx + ox[d]] * hy[2 * cy + oy[d]] * hz[2 * cz + oz[d]]);
  }
  return res;
}

__global__ void __launch_bounds__(ROT_THREADS)
k_extpot_rot_interp(RotArgs c, InterpArgs ia, const double* __restrict__ tab, const double* __restrict__ rot,
                    const double* __restrict__ w, double* __restrict__ V, long long idx0,
                    double* __restrict__ scratch) {
  __shared__ double frame[ROT_MAX_SITES + 1][3];
  __shared__ double red[32];
  extern __shared__ double s_dyn[];
  double* s_a = scratch ? scratch + (size_t)blockIdx.x * c.nrot : s_dyn;
  const ExtArgs& a = c.a;
  const long long idx = idx0 + blockIdx.x;
  const int k = (int)(idx % a.n3), j = (int)((idx / a.n3) % a.n2), i = (int)(idx / ((long long)a.n3 * a.n2));
  rot_frame(c, i, j, k, frame);
  __syncthreads();
  const long long fpts = (long long)ia.f[0] * ia.f[1] * ia.f[2];
  const float fnb = __double2float_rn(-c.beta);
  for (int r = threadIdx.x; r < c.nrot; r += blockDim.x) {
    const double* R = rot + (size_t)r * 9;
    float pot = 0.0f;
    for (int s = 0; s < c.nsite; ++s) {
      double q[3];
      rot_site(R, frame, s, q);
      const double v = tricubic_at(tab + (size_t)ia.site_tab[s] * 8 * fpts, fpts, ia, q);
      pot = __fadd_rn(pot, __double2float_rn(v));
    }
    s_a[r] = (double)__fmul_rn(fnb, pot);
  }
  __syncthreads();
  rot_finish(c, s_a, w, red, V + idx);
}

extern "C" int cmm_extpot_rot_interp(const cmm_grid* g, const double* d_tab, int ntab, const int* fine_n,
                                     const double* origin, const double* spacing, const double* guest_pos,
                                     const double* guest_mass, const int* site_tab, int nsite, const double* d_rot,
                                     const double* d_w, int nrot, double beta, double v_limit, double* d_V,
                                     void* stream) {
  if (!g || !d_tab || !fine_n || !origin || !spacing || !guest_pos || !guest_mass || !site_tab || !d_rot || !d_w ||
      !d_V || ntab < 1 || nsite < 1 || nrot < 1 || !(beta > 0))
    return CMM_ERR_ARG;
  if (nsite > ROT_MAX_SITES) return CMM_ERR_UNSUPPORTED;
  RotArgs c;
  memset(&c, 0, sizeof(c));
  InterpArgs ia;
  memset(&ia, 0, sizeof(ia));
  for (int q = 0; q < 9; ++q) c.a.rv[q] = g->rvecs[q];
  c.a.n1 = g->n1; c.a.n2 = g->n2; c.a.n3 = g->n3;
  c.nsite = nsite; c.nrot = nrot; c.beta = beta; c.vlimit = v_limit;
  double mt = 0.0;
  for (int d = 0; d < 3; ++d) {
    if (fine_n[d] < 1 || !(spacing[d] > 0)) return CMM_ERR_ARG;
    ia.f[d] = fine_n[d];
    ia.origin[d] = origin[d];
    ia.spacing[d] = spacing[d];
  }
  for (int q = 0; q < nsite; ++q) {
    if (site_tab[q] < 0 || site_tab[q] >= ntab) return CMM_ERR_ARG;
    ia.site_tab[q] = site_tab[q];
    for (int d = 0; d < 3; ++d) c.pos[q][d] = guest_pos[3 * q + d];
    c.mass[q] = guest_mass[q];
    mt += guest_mass[q];
  }
  if (!(mt > 0)) return CMM_ERR_ARG;
  c.mtot = mt;
  const long long npts = (long long)g->n1 * g->n2 * g->n3;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = rot_launch(npts, nrot, (const void*)k_extpot_rot_interp, st,
                      [&](unsigned nb, size_t dyn, long long p0, double* scr) {
                        k_extpot_rot_interp<<<nb, ROT_THREADS, dyn, st>>>(c, ia, d_tab, d_rot, d_w, d_V, p0, scr);
                      });
  if (cudaStreamSynchronize(st) != cudaSuccess) rc = CMM_ERR_CUDA;
  return rc;
}
