// Shared definitions for the cmmdft_b200 CUDA sources.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "fft_core.cuh"
#include "../../include/cmmdft_b200.h"

#define CMM_MAX_N 1024        // longest axis a grid plan accepts
#define CMM_MAX_FIELDS 12     // fields a mix launch combines
#define CMM_PLANE_THREADS 512
#define CMM_COL_THREADS 256
#define CMM_FMT_THREADS 768    // the 5-field plane pass (one block per SM; 768 balances its radix-8 rounds)
// Resident blocks per SM the compiler must allow for (register budget) in the
// single-field plane passes and the column passes.  The weights and
// back-convolution column passes of the specialised x lengths (32, 64) run
// five 256-thread blocks per SM (48 registers, a few spilled bytes): 5% faster
// C1 pipeline at 64^3 than four blocks with 64 registers, measured; the
// run-time-length instantiation without radix 7/11/13 and Rader stages (0)
// runs four blocks (64 registers; C1 5-7 % faster on 80x96x72 and
// 160x144x160, with the y pass of the staged plane passes likewise); the one
// with them (-1) keeps its full register budget.
#ifndef CMM_PLANE_MINB
#define CMM_PLANE_MINB 1
#endif
#ifndef CMM_COL_MINB
#define CMM_COL_MINB 1
#endif
#define CMM_COL_MINB_FOR(n1c) ((n1c) > 0 ? 5 : ((n1c) == 0 ? 4 : CMM_COL_MINB))
// The single-field plane passes (transforms, Picard, residual, mix) run two
// 512-thread blocks per SM (64 registers, no spills) except in the
// instantiation with radix 7/11/13 and Rader stages (-1), whose stage code
// needs more registers: residual 0.235 -> 0.156 ms, mix 0.225 -> 0.179 ms,
// Picard 0.185 -> 0.125 ms for 24 instances at 64^3 against one block per SM.
#define CMM_PLANE_MINB_FOR(n2c) ((n2c) >= 0 ? 2 : CMM_PLANE_MINB)
#define CMM_ROW_THREADS 512    // staged z-row passes
#define CMM_ZFMT_THREADS 768   // the staged z-row pass of dPhi/dn (768 measured faster than 256-512 and 1024)

// Per-instance reduction slots (see cmm_stat_* in the public header).
#define NQ CMM_NSTAT

// Device-side description of one grid plan.  Every table is indexed by the
// POSITION at which a frequency is stored (digit-reversed layout), so the
// k-space stages never permute data.
struct GridDev {
  int n1, n2, n3, h3, m3;      // h3 = n3/2+1 stored z frequencies, m3 = n3/2
  int zfull;                   // odd N3: ax3 is the full-length z transform, stored z in natural order
  FftAxis ax1, ax2, ax3;       // ax3: the half-length complex z transform (length m3) for even N3
  const double2* tw1;          // w_{n1}^t, t < n1
  const double2* tw2;          // w_{n2}^t
  const double2* tw3;          // w_{n3}^t (the z transform and the R2C twist)
  const int* zpos;             // z DIF position of frequency k (k < m3; k < n3 when zfull)
  const int* k1pos;            // x frequency at DIF position p (column passes)
  const double* kp1;           // signed k component (bohr^-1) at x position
  const double* kp2;
  const double* kp3;           // at z position p3 <= m3
  const double* sl1;           // Lanczos sinc factor at x position
  const double* sl2;
  const double* sl3;
  const int* nq1;              // 1 where the x position holds the Nyquist frequency of an even axis
  const int* nq2;
  const int* nq3;
  const double* wt3;           // Parseval weight at z position (1 for k3 = 0 and k3 = n3/2, else 2)
};

struct cmm_grid {
  int n1, n2, n3, h3, m3;
  double rvecs[9];
  double spacing[3];
  double volume;
  FftAxis ax1, ax2, ax3;
  // host copies of the position tables
  int* hpos_k1;                // k index at x position (DIF output order)
  int* hpos_k2;
  int* hpos_k3;                // k index at z position (p < m3 -> DIF; p == m3 -> m3)
  // one device allocation holding every table
  void* dmem;
  GridDev dev;
  int staging;                 // 0: by size, 1: staged plane passes always
  int exotic;                  // 1: radix 7, 11 or 13 or a Rader stage on some axis (kernels instantiated with -1)
  int order[3];                // radix order per axis (CMM_ORDER_*)
  int generic;                 // 1: a non-default radix order, so no compile-time-length kernels
  int col_tile;                // column-pass tile width of the run-time kernels (0: by size)
};

static inline int cmm_div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

__device__ __forceinline__ bool cmm_isfinite(double x) { return isfinite(x); }

// A hint: bring [p, p + bytes) into L2 by bulk prefetches of at most 16 KB
// (cp.async.bulk.prefetch.L2).  Issued by one thread; skipped unless p and
// bytes are multiples of 16 bytes.  Plane passes call it for the real-space
// planes their pointwise step reads, so that those reads hit L2 instead of
// waiting on HBM one loop iteration at a time.
__device__ __forceinline__ void cmm_prefetch_l2(const void* p, size_t bytes) {
  if ((((uintptr_t)p) & 15) || (bytes & 15)) return;
  const char* c = (const char*)p;
  for (size_t o = 0; o < bytes; o += 16384) {
    const unsigned n = (unsigned)((bytes - o) < 16384 ? (bytes - o) : 16384);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(c + o), "r"(n) : "memory");
  }
}
