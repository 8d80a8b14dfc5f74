// noalloc.cu -- sparc_ke_norm_noalloc: the kinetic-energy norm of a handle's
// current state (norm() of all_modules.f90:684-706 as driver.f90:161 uses
// it), computed without allocating any memory.  It equals the ke_norm of
// sparc_diagnostics when called right after an iteration's stages, before
// that iteration's filter or a sparc_set_state replaces the state.
//
// For a handle in a batch the batch owns the buffer roles and rotates them
// on the device every step; the kernel then reads the live role from the
// member's device slot instead of the handle's (stale) host copy.
//
// The reduction is a variant of the last-block-done diagnostics reduction
// of the stage kernels.  Its scratch is the file-scope static device array
// below instead of handle-owned device memory:
//   bytes [0, 8)        completion counter (unsigned); MUST be zero when a
//                       call starts.  It is zero-initialised at module load
//                       and the last block of every call resets it.
//   bytes [8, 16)       the result (double), written by the last block
//   bytes [256, ...)    one partial sum per block, at most kMaxBlocks
// Each block reduces kBlockPoints consecutive grid points, so a call needs
// ceil(N / kBlockPoints) blocks; grids above kMaxBlocks * kBlockPoints
// points are rejected.  All calls on a device share this scratch: calls
// that overlap in time (other host threads, other streams) race on it and
// must be serialised by the caller.
//
// Setup: the first call on a device looks up the scratch's device address
// with cudaGetSymbolAddress (that device current) and caches it; the first
// call on each device should therefore happen before any stream capture.
// The cached address belongs to the device's primary context as it was at
// that first call: after cudaDeviceReset (which tears that context down)
// the cache is stale, so do not use this entry point after a reset.

#include <mutex>

#include "internal.h"

namespace sparc {

constexpr int kNoallocThreads = 256;
constexpr int kBlockPoints = 16384;     // 64 points per thread
constexpr int kMaxBlocks = 4096;        // => at most 67,108,864 grid points
constexpr int kScratchBytes = 256 + kMaxBlocks * 8;  // 33,024 bytes
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

static std::mutex g_noalloc_mu;
static unsigned char *g_noalloc_ptr[kMaxDevices] = {};

// m = (rho0 + rho) |v|^2 / 2 at point n, from the FP64 state or from the
// FP32 state with its carry and depth scales
struct KeSrc {
  long long N, NXY;
  int nz, bg1d;
  const double *a;                       // FP64 form
  const float *fa, *carry, *isc, *frho0; // FP32 form
  const double *rho0;
  const Slot32 *slot;                    // batch member: live roles (or null)
};

__device__ __forceinline__ double ke_density(const KeSrc &S, const float *fa, long long n) {
  const int k = (int)(n / S.NXY);
  double r, v1, v2, v3, r0;
  if (S.a) {
    r = S.a[n];
    v1 = S.a[S.N + n];
    v2 = S.a[2 * S.N + n];
    v3 = S.a[3 * S.N + n];
    r0 = S.rho0[n];
  } else {
    auto ph = [&](int l) {
      const long long q = l * S.N + n;
      return ((double)fa[q] - (double)S.carry[q]) * (double)S.isc[l * S.nz + k];
    };
    r = ph(0);
    v1 = ph(1);
    v2 = ph(2);
    v3 = ph(3);
    r0 = (double)S.frho0[S.bg1d ? k : n];
  }
  return (r0 + r) * (v1 * v1 + v2 * v2 + v3 * v3) / 2.0;
}

__global__ void __launch_bounds__(kNoallocThreads)
    k_ke_norm_noalloc(KeSrc S, unsigned char *scratch, double scale) {
  __shared__ double red[kNoallocThreads / 32];
  __shared__ int am_last;
  unsigned *counter = (unsigned *)scratch;
  double *result = (double *)(scratch + 8);
  double *partials = (double *)(scratch + 256);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long p0 = (long long)blockIdx.x * kBlockPoints;
  const long long p1 = min(S.N, p0 + kBlockPoints);
  // a batch member's state is the buffer of its slot's current role 0
  const float *fa = S.slot ? S.slot->buf[S.slot->role[0]] : S.fa;
  double s = 0.0;
  for (long long n = p0 + tid; n < p1; n += kNoallocThreads) {
    const double m = ke_density(S, fa, n);
    s += m * m;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) red[warp] = s;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < kNoallocThreads / 32; ++w) t += red[w];
    partials[blockIdx.x] = t;
    __threadfence();
    am_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  s = 0.0;
  for (int b = tid; b < (int)gridDim.x; b += kNoallocThreads) s += __ldcg(partials + b);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __syncthreads();
  if (lane == 0) red[warp] = s;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < kNoallocThreads / 32; ++w) t += red[w];
    *result = sqrt(t / (double)S.N) * scale;
    *counter = 0u;  // ready for the next call
  }
}

// device address of the scratch on the current device (cached per device)
static int scratch_for(int device, unsigned char **out, std::string &err) {
  if (device < 0 || device >= kMaxDevices) {
    err = "device index beyond the no-allocation path's table";
    return SPARC_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      err = std::string("cudaGetSymbolAddress of the reduction scratch: ") +
            cudaGetErrorString(e);
      cudaGetLastError();
      return SPARC_ERR_CUDA;
    }
    g_noalloc_ptr[device] = (unsigned char *)p;
  }
  *out = g_noalloc_ptr[device];
  return SPARC_OK;
}

}  // namespace sparc

using namespace sparc;

extern "C" int sparc_ke_norm_noalloc(sparc_handle *hh, double *ke_norm) {
  if (!hh || !ke_norm) return SPARC_ERR_INVALID;
  Handle *h = reinterpret_cast<Handle *>(hh);
  const long long limit = (long long)kMaxBlocks * kBlockPoints;
  if (h->N > limit) {
    h->err = "grid of " + std::to_string(h->N) + " points exceeds the " +
             std::to_string(limit) + "-point limit of the no-allocation reduction (" +
             std::to_string(kMaxBlocks) + " blocks of static scratch)";
    return SPARC_ERR_INVALID;
  }
  if (!h->bg_ready) {
    h->err = "set the background first";
    return SPARC_ERR_ORDER;
  }
  if (cudaSetDevice(h->device) != cudaSuccess) return SPARC_ERR_CUDA;
  unsigned char *scratch = nullptr;
  int r = scratch_for(h->device, &scratch, h->err);
  if (r) return r;
  KeSrc S{};
  S.N = h->N;
  S.NXY = (long long)h->nx * h->ny;
  S.nz = h->nz;
  if (h->batch) {
    // the batch owns the roles: read the live one from the member's device
    // slot (until the batch's first upload the handle's roles are current)
    r = batch_member_slot(h, &S.slot);
    if (r) {
      h->err = "handle's batch does not list it";
      return r;
    }
  }
  if (h->fp32) {
    S.fa = h->fbuf[h->ra];
    S.carry = h->f_carry;
    S.isc = h->f_isc;
    S.frho0 = h->f_bg[FB_RHO0];
    S.bg1d = h->bg1d ? 1 : 0;
  } else {
    S.a = h->buf[h->ra];
    S.rho0 = h->rho0;
  }
  cudaStream_t st = h->batch ? h->batch_stream : h->stream;
  const unsigned blocks = (unsigned)((h->N + kBlockPoints - 1) / kBlockPoints);
  k_ke_norm_noalloc<<<blocks, kNoallocThreads, 0, st>>>(S, scratch,
                                                        (h->dimc * h->dimc) * h->dimrho);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ke_norm, scratch + 8, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    h->err = std::string("no-allocation reduction: ") + cudaGetErrorString(e);
    return SPARC_ERR_CUDA;
  }
  ++h->launches;
  return SPARC_OK;
}
