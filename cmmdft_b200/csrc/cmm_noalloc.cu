// Allocation-free variant of the functional pipeline (cmm_fmt_c1).
//
// Some callers cannot allocate device memory at the point where they need a
// functional evaluation: plugin hosts that forbid allocation inside a solve
// callback, integrations that run under a fixed device-memory budget
// reserved up front, and bindings from languages whose runtime cannot own
// the lifetime of a CUDA allocation.  For them, cmm_fmt_c1_noalloc keeps its
// scratch (the twelve intermediate spectra and the per-block partial sums) in
// one file-scope device array of fixed size, CMM_NOALLOC_SCRATCH_BYTES, that
// every GPU loading this library holds until the process exits.
//
// The array's device address is looked up once per device, with that device
// current, on the first call made on it; make that first call before any
// stream capture.  The address is cached per device index for the life of
// the process: after a cudaDeviceReset (or any other re-creation of the
// device's primary context) it is stale, and the entry point must not be
// called on that device again.  All calls share the array and it keeps the contents of
// the last call, so calls that overlap on the GPU (other streams, other host
// threads) race and must be serialised by the caller.
#include <mutex>

#include "cmm_common.cuh"

#define CMM_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_noalloc_scratch[CMM_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mutex;
static void* g_noalloc_addr[CMM_NOALLOC_MAX_DEVICES];

// Device address of the scratch array on the current device (looked up once).
static int noalloc_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return CMM_ERR_CUDA;
  if (dev < 0 || dev >= CMM_NOALLOC_MAX_DEVICES) return CMM_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return CMM_ERR_CUDA;
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return CMM_OK;
}

// Partial sums start at 0 (sums) or -inf (the n3 maximum) on every call.
__global__ void k_noalloc_clear_part(double* part, int batch, int nslot) {
  const long long n = (long long)batch * CMM_NSTAT * nslot;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int q = (int)((i / nslot) % CMM_NSTAT);
    part[i] = (q == CMM_STAT_N3MAX) ? -INFINITY : 0.0;
  }
}

#define NOALLOC_NSPEC 12   // intermediate spectra per instance (6 weighted densities, 6 dPhi)

extern "C" size_t cmm_fmt_c1_noalloc_capacity(const cmm_grid* g) {
  if (!g) return 0;
  const size_t spec = (size_t)g->n1 * g->n2 * g->h3 * sizeof(double2);
  const size_t nslot = (size_t)((g->n1 > g->n2 * g->h3) ? g->n1 : g->n2 * g->h3);
  const size_t per = NOALLOC_NSPEC * spec + (size_t)CMM_NSTAT * nslot * sizeof(double);
  return per ? (size_t)CMM_NOALLOC_SCRATCH_BYTES / per : 0;
}

extern "C" int cmm_fmt_c1_noalloc(const cmm_grid* g, int batch, const int* d_active, double R, double beta,
                                  int version, const cmm_wda_eos* wda, const double* d_kst, const double* d_wtab,
                                  const double* d_rhohat, double* d_chat, double* d_stats, int want, void* stream) {
  if (!g || batch < 1 || !d_kst || !d_rhohat) return CMM_ERR_ARG;
  if (version & CMM_TENSOR) return CMM_ERR_UNSUPPORTED;  // 24 spectra: beyond the sizing below
  if ((want & 1) && !d_chat) return CMM_ERR_ARG;
  if ((want & 6) && !d_stats) return CMM_ERR_ARG;
  if ((version & CMM_NOHS) && want != 1) return CMM_ERR_ARG;  // as cmm_fmt_c1: C1 only
  if ((size_t)batch > cmm_fmt_c1_noalloc_capacity(g)) return CMM_ERR_WORKSPACE;  // beyond the fixed scratch
  void* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  const size_t spec = (size_t)g->n1 * g->n2 * g->h3 * sizeof(double2);
  const int nslot = (g->n1 > g->n2 * g->h3) ? g->n1 : g->n2 * g->h3;
  double* work = (double*)base;
  double* part = (double*)((unsigned char*)base + NOALLOC_NSPEC * spec * (size_t)batch);
  cudaStream_t st = (cudaStream_t)stream;
  k_noalloc_clear_part<<<148, 256, 0, st>>>(part, batch, nslot);
  if (cudaPeekAtLastError() != cudaSuccess) return CMM_ERR_CUDA;
  rc = cmm_fmt_c1(g, batch, d_active, R, beta, version, wda, d_kst, d_wtab, d_rhohat, d_chat, work, part, nslot,
                  want & 7, nullptr, stream);
  if (rc) return rc;
  if (want & 6) {
    unsigned mask = 0;
    if (want & 2) mask |= (1u << CMM_STAT_PHI) | (1u << CMM_STAT_MFA) | (1u << CMM_STAT_WDA);
    if (want & 4) mask |= (1u << CMM_STAT_N3MAX);
    rc = cmm_stats_finalize(batch, d_active, part, nslot, mask, d_stats, stream);
  }
  return rc;
}
