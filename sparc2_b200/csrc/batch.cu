// batch.cu -- host side of the batched engine (precision form): the C ABI
// sparc_batch_* of include/sparc_gpu.h.  A batch holds simulation handles
// created with SPARC_FP32; each step of all of them is one CUDA-graph launch
// (work counters reset, step begin, PULSE = 2 forcing, five persistent RK
// stage launches over the (sim, tile, z-chunk) work-list, three filter
// passes).  The work-list, the slot table and the per-simulation buffer
// roles live in device memory, so the captured graph stays valid while
// simulations are added and removed; only a larger work-list re-captures.
//
// The reference has no counterpart: it runs one simulation per MPI job.

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "filter_body.cuh"
#include "internal.h"

namespace sparc {

struct Batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  int cap = 0;
  std::vector<Slot32> slots;            // host image of the slot table
  std::vector<Handle *> members;        // nullptr: free slot
  std::vector<char> on_device;          // slot image uploaded (device owns roles)
  Slot32 *d_slots = nullptr;
  int4 *d_items = nullptr, *d_fitems = nullptr, *d_pitems = nullptr, *d_zitems = nullptr,
       *d_xyitems = nullptr;
  size_t items_cap = 0, fitems_cap = 0, pitems_cap = 0, zitems_cap = 0, xyitems_cap = 0;
  size_t partials_cap = 0;
  int *d_counts = nullptr;
  unsigned *d_wctr = nullptr;
  double *d_partials = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool dirty = true;                    // work-list or slot table to upload
  bool recapture = true;                // device arrays moved
  int zchunk_mhd = 32, zchunk_quiet = 48;
  int fchunk = 1 << 16;
  int grid = 148;
  size_t psr_smem = 0;
  int nkernels = 0;
  long long launches = 0;
  std::string err;
};

}  // namespace sparc

using namespace sparc;

struct sparc_batch : Batch {};

namespace {

int bfail(Batch *b, int code, const std::string &m) {
  if (b) b->err = m;
  return code;
}

bool bok(Batch *b, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  b->err = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

#define BCK(b, x)                                          \
  do {                                                     \
    if (!bok((b), (x), #x)) return SPARC_ERR_CUDA;         \
  } while (0)

template <class T>
int grow(Batch *b, T *&p, size_t &cap, size_t need) {
  if (need <= cap && p) return SPARC_OK;
  size_t n = std::max<size_t>(need, cap * 2);
  n = std::max<size_t>(n, 64);
  if (p) cudaFree(p);
  p = nullptr;
  if (!bok(b, cudaMalloc(&p, n * sizeof(T)), "cudaMalloc")) return SPARC_ERR_NOMEM;
  cap = n;
  b->recapture = true;
  return SPARC_OK;
}

// Rebuild the work-lists from the occupied slots and upload them with the
// slot table (the batch stream is idle when this runs).
int rebuild(Batch *b) {
  std::vector<int4> items, fitems, pitems, zitems, xyitems;
  size_t npart = 0;
  size_t maxp = 0;
  // pass 0: interior MHD tiles (the list's prefix, run by the branch-free
  // kernel); pass 1: MHD tiles at edges / CPML slabs; pass 2: quiet tiles.
  // Costlier items first, dynamic scheduling then fills in.
  int n_int = 0;
  for (int pass = 0; pass < 3; ++pass) {
    for (int q = 0; q < b->cap; ++q) {
      Handle *h = b->members[q];
      if (!h || (pass < 2) != h->magnetic) continue;
      Slot32 &L = b->slots[q];
      const int TY = h->magnetic ? 8 : 16;
      const int zc = std::max(11, h->magnetic ? b->zchunk_mhd : b->zchunk_quiet);
      const int first = (int)items.size();
      for (int k0 = 0; k0 < h->nz; k0 += zc) {
        const int k1 = std::min(h->nz, k0 + zc);
        for (int y0 = 0; y0 < h->ny; y0 += TY)
          for (int x0 = 0; x0 < h->nx; x0 += 32) {
            bool in = false;
            if (h->magnetic) {  // the kernels' interior test
              const FaceT<float> *F = h->f_faces;
              const int xm = std::max(5, F[2].on ? F[2].np : 0);
              const int xM = std::max(5, F[3].on ? F[3].np : 0);
              const int ym = std::max(5, F[4].on ? F[4].np : 0);
              const int yM = std::max(5, F[5].on ? F[5].np : 0);
              in = x0 >= xm && x0 + 32 <= h->nx - xM && y0 >= ym && y0 + TY <= h->ny - yM;
            }
            if (in == (pass == 0)) items.push_back(make_int4(q, x0, y0, k0 | (k1 << 16)));
          }
      }
      if (pass == 0) {
        L.first_item = first;
        L.n_items = (int)items.size() - first;
      } else {
        L.first_item2 = first;
        L.n_items2 = (int)items.size() - first;
      }
      L.partials = nullptr;  // set below
    }
    if (pass == 0) n_int = (int)items.size();
  }
  for (int q = 0; q < b->cap; ++q)
    if (b->members[q] && !b->members[q]->magnetic) b->slots[q].first_item = b->slots[q].n_items = 0;
  npart = items.size();
  for (int q = 0; q < b->cap; ++q) {
    Handle *h = b->members[q];
    if (!h) continue;
    Slot32 &L = b->slots[q];
    const long long tot = (long long)h->V * h->N;
    L.f_first = (int)fitems.size();
    for (long long t = 0; t < tot; t += b->fchunk)
      fitems.push_back(make_int4(q, (int)t, (int)std::min<long long>(b->fchunk, tot - t), 0));
    L.f_items = (int)fitems.size() - L.f_first;
    // z pass: (slot, field, slab of 32 x 4 columns, chunk of 32 layers), the
    // chunks of a slab adjacent (their shared margins come from L2)
    const int nxb = (h->nx + fb::ZX - 1) / fb::ZX, nyb = (h->ny + fb::ZY - 1) / fb::ZY;
    const int nzc = (h->nz + fb::ZC - 1) / fb::ZC;
    const size_t z0 = zitems.size();
    for (int l = 0; l < h->V; ++l)
      for (int sl = 0; sl < nxb * nyb; ++sl)
        for (int c = 0; c < nzc; ++c) zitems.push_back(make_int4(q, l, sl, c));
    L.z_items = (int)(zitems.size() - z0);
    // xy pass: (slot, field, group of LPB layers, 32 x 32 tile)
    const int ntx = (h->nx + fb::TX - 1) / fb::TX, nty = (h->ny + fb::TR - 1) / fb::TR;
    const int nlg = (h->nz + fb::LPB - 1) / fb::LPB;
    const size_t xy0 = xyitems.size();
    for (int l = 0; l < h->V; ++l)
      for (int g = 0; g < nlg; ++g)
        for (int t = 0; t < ntx * nty; ++t) xyitems.push_back(make_int4(q, l, g, t));
    L.xy_items = (int)(xyitems.size() - xy0);
    if (L.has_psr) {
      for (int k = h->psr_klo; k < h->psr_khi; ++k) pitems.push_back(make_int4(q, k, 0, 0));
      maxp = std::max(maxp, h->pulses.size());
    }
  }
  int r = SPARC_OK;
  r |= grow(b, b->d_items, b->items_cap, items.size());
  r |= grow(b, b->d_fitems, b->fitems_cap, fitems.size());
  r |= grow(b, b->d_pitems, b->pitems_cap, pitems.size());
  r |= grow(b, b->d_zitems, b->zitems_cap, zitems.size());
  r |= grow(b, b->d_xyitems, b->xyitems_cap, xyitems.size());
  r |= grow(b, b->d_partials, b->partials_cap, 3 * npart);
  if (r) return r;
  for (int q = 0; q < b->cap; ++q)
    if (b->members[q]) b->slots[q].partials = b->d_partials;
  const size_t smem = std::max<size_t>(maxp, 1) * (sizeof(float) + sizeof(int));
  if (smem != b->psr_smem) {
    b->psr_smem = smem;
    b->recapture = true;
  }
  const int counts[6] = {(int)items.size(), (int)fitems.size(), (int)pitems.size(), n_int,
                         (int)zitems.size(), (int)xyitems.size()};
  BCK(b, cudaStreamSynchronize(b->stream));
  // ordered on the batch stream (its kernels read these), finished before
  // the host arrays go
  if (!items.empty())
    BCK(b, cudaMemcpyAsync(b->d_items, items.data(), items.size() * sizeof(int4),
                           cudaMemcpyHostToDevice, b->stream));
  if (!fitems.empty())
    BCK(b, cudaMemcpyAsync(b->d_fitems, fitems.data(), fitems.size() * sizeof(int4),
                           cudaMemcpyHostToDevice, b->stream));
  if (!pitems.empty())
    BCK(b, cudaMemcpyAsync(b->d_pitems, pitems.data(), pitems.size() * sizeof(int4),
                           cudaMemcpyHostToDevice, b->stream));
  if (!zitems.empty())
    BCK(b, cudaMemcpyAsync(b->d_zitems, zitems.data(), zitems.size() * sizeof(int4),
                           cudaMemcpyHostToDevice, b->stream));
  if (!xyitems.empty())
    BCK(b, cudaMemcpyAsync(b->d_xyitems, xyitems.data(), xyitems.size() * sizeof(int4),
                           cudaMemcpyHostToDevice, b->stream));
  BCK(b, cudaMemcpyAsync(b->d_counts, counts, sizeof(counts), cudaMemcpyHostToDevice,
                         b->stream));
  BCK(b, cudaMemcpyAsync(b->d_slots, b->slots.data(), b->cap * sizeof(Slot32),
                         cudaMemcpyHostToDevice, b->stream));
  BCK(b, cudaStreamSynchronize(b->stream));
  for (int q = 0; q < b->cap; ++q) b->on_device[q] = b->members[q] != nullptr;
  b->dirty = false;
  return SPARC_OK;
}

int capture(Batch *b) {
  if (b->exec && !b->recapture) return SPARC_OK;
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  BatchLaunch L;
  L.slots = b->d_slots;
  L.nslots = b->cap;
  L.items = b->d_items;
  L.fitems = b->d_fitems;
  L.pitems = b->d_pitems;
  L.zitems = b->d_zitems;
  L.xyitems = b->d_xyitems;
  L.counts = b->d_counts;
  L.wctr = b->d_wctr;
  L.grid = b->grid;
  L.zmax = std::max(11, std::max(b->zchunk_mhd, b->zchunk_quiet));
  L.psr_smem = b->psr_smem;
  cudaGraph_t g;
  BCK(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int nk = 0;
  int r = launch_batch_step(L, b->stream, &nk);
  cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (r) return bfail(b, SPARC_ERR_CUDA, "batched step launch failed");
  BCK(b, e);
  cudaError_t ie = cudaGraphInstantiate(&b->exec, g, 0);
  cudaGraphDestroy(g);
  BCK(b, ie);
  b->nkernels = nk;
  b->recapture = false;
  return SPARC_OK;
}

// Bring the device-owned part of the slot table (roles, steps left) of the
// uploaded members back into the host image; slots added since the last
// upload keep their host image.
int pull_all(Batch *b) {
  std::vector<Slot32> t(b->cap);
  BCK(b, cudaStreamSynchronize(b->stream));
  BCK(b, cudaMemcpy(t.data(), b->d_slots, b->cap * sizeof(Slot32), cudaMemcpyDeviceToHost));
  for (int q = 0; q < b->cap; ++q)
    if (b->members[q] && b->on_device[q]) b->slots[q] = t[q];
  return SPARC_OK;
}

}  // namespace

namespace sparc {

// The slot of batch member h: its device slot when the slot table holding
// it has been uploaded (the device then owns its buffer roles), else null
// (the handle's own roles are still current).
int batch_member_slot(const Handle *h, const Slot32 **dslot) {
  *dslot = nullptr;
  const Batch *b = static_cast<const Batch *>(h->batch);
  if (!b) return SPARC_ERR_INVALID;
  for (int q = 0; q < b->cap; ++q)
    if (b->members[q] == h) {
      if (b->on_device[q]) *dslot = b->d_slots + q;
      return SPARC_OK;
    }
  return SPARC_ERR_INVALID;
}

}  // namespace sparc

extern "C" {

int sparc_batch_create(int device, int capacity, sparc_batch **out) {
  if (!out || capacity < 1 || capacity > 4096) return SPARC_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return SPARC_ERR_NODEVICE;
  }
  if (cudaSetDevice(device) != cudaSuccess) return SPARC_ERR_CUDA;
  sparc_batch *b = new (std::nothrow) sparc_batch();
  if (!b) return SPARC_ERR_NOMEM;
  b->device = device;
  b->cap = capacity;
  b->slots.assign(capacity, Slot32{});
  b->members.assign(capacity, nullptr);
  b->on_device.assign(capacity, 0);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  b->grid = sms;
  bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&b->d_slots, capacity * sizeof(Slot32)) == cudaSuccess &&
            cudaMalloc(&b->d_counts, 6 * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&b->d_wctr, 14 * sizeof(unsigned)) == cudaSuccess &&
            cudaMemsetAsync(b->d_slots, 0, capacity * sizeof(Slot32), b->stream) == cudaSuccess &&
            cudaMemsetAsync(b->d_counts, 0, 6 * sizeof(int), b->stream) == cudaSuccess &&
            cudaStreamSynchronize(b->stream) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    sparc_batch_destroy(b);
    return SPARC_ERR_NOMEM;
  }
  *out = b;
  return SPARC_OK;
}

int sparc_batch_destroy(sparc_batch *b) {
  if (!b) return SPARC_ERR_INVALID;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (int q = 0; q < b->cap; ++q)
    if (b->members[q]) sparc_batch_remove(b, q);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  cudaFree(b->d_slots);
  cudaFree(b->d_items);
  cudaFree(b->d_fitems);
  cudaFree(b->d_pitems);
  cudaFree(b->d_zitems);
  cudaFree(b->d_xyitems);
  cudaFree(b->d_counts);
  cudaFree(b->d_wctr);
  cudaFree(b->d_partials);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return SPARC_OK;
}

int sparc_batch_add(sparc_batch *b, sparc_handle *hh, int64_t first, int64_t count,
                    int *slot) {
  if (!b || !hh || count < 0) return SPARC_ERR_INVALID;
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h->fp32) return bfail(b, SPARC_ERR_INVALID, "batched simulations use SPARC_FP32");
  if (!h->bg_ready) return bfail(b, SPARC_ERR_ORDER, "set the background first");
  if (h->batch) return bfail(b, SPARC_ERR_ORDER, "handle is already in a batch");
  if (h->device != b->device) return bfail(b, SPARC_ERR_INVALID, "handle on another device");
  int q = 0;
  while (q < b->cap && b->members[q]) ++q;
  if (q == b->cap) return bfail(b, SPARC_ERR_NOMEM, "batch is full");
  cudaSetDevice(b->device);
  BCK(b, cudaStreamSynchronize(h->stream));
  BCK(b, cudaMemcpyAsync(h->d_iter, &first, 8, cudaMemcpyHostToDevice, h->stream));
  BCK(b, cudaStreamSynchronize(h->stream));
  Slot32 L{};
  L.S = make_sim32(h);
  L.has_psr = h->src.kind == SPARC_SRC_PSR && h->psr_khi > h->psr_klo;
  if (L.has_psr) L.psr = make_psr32(h);
  L.has_rnd = h->src.kind == SPARC_SRC_RANDOM;
  if (L.has_rnd) {  // the member's own forcing plane, rebuilt every step
    L.rnd.series = h->d_series;
    L.rnd.damp = h->f_sd;
    L.rnd.out = h->f_f2d;
    L.rnd.nxy = h->nx * h->ny;
    L.rnd.ns = h->src.nseries;
    L.rnd.timestep = h->P.timestep;
    L.rnd.cad = h->src.cadforcing;
  }
  for (int i = 0; i < 3; ++i) L.buf[i] = h->fbuf[i];
  L.role[0] = h->ra;
  L.role[1] = h->rf1;
  L.role[2] = h->rf2;
  for (int i = 0; i < 5; ++i) L.betas[i] = h->betas[i];
  L.remaining = count;
  L.gxy = h->gxy;
  L.gz = h->gz;
  L.xyfreq = h->xyfreq;
  L.zfreq = h->zfreq;
  L.s_xy = (float)h->P.s_xy;
  L.s_z = (float)h->P.s_z;
  b->slots[q] = L;
  b->members[q] = h;
  b->on_device[q] = 0;
  h->batch = b;
  h->batch_stream = b->stream;
  b->dirty = true;
  if (slot) *slot = q;
  return SPARC_OK;
}

int sparc_batch_remove(sparc_batch *b, int q) {
  if (!b || q < 0 || q >= b->cap || !b->members[q]) return SPARC_ERR_INVALID;
  cudaSetDevice(b->device);
  int r = pull_all(b);
  if (r) return r;
  Handle *h = b->members[q];
  const Slot32 &L = b->slots[q];
  h->ra = L.role[0];
  h->rf1 = L.role[1];
  h->rf2 = L.role[2];
  h->batch = nullptr;
  h->batch_stream = nullptr;
  b->members[q] = nullptr;
  b->on_device[q] = 0;
  b->slots[q] = Slot32{};
  b->dirty = true;
  return SPARC_OK;
}

int sparc_batch_run(sparc_batch *b, int64_t steps) {
  if (!b || steps < 0) return SPARC_ERR_INVALID;
  cudaSetDevice(b->device);
  int r;
  if (b->dirty) {
    // device-side roles and steps left of the current members survive
    if ((r = pull_all(b))) return r;
    if ((r = rebuild(b))) return r;
  }
  if ((r = capture(b))) return r;
  for (int64_t s = 0; s < steps; ++s) {
    BCK(b, cudaGraphLaunch(b->exec, b->stream));
    b->launches += b->nkernels;
  }
  return SPARC_OK;
}

int sparc_batch_remaining(sparc_batch *b, int64_t *remaining) {
  if (!b || !remaining) return SPARC_ERR_INVALID;
  cudaSetDevice(b->device);
  int r = pull_all(b);
  if (r) return r;
  for (int q = 0; q < b->cap; ++q) remaining[q] = b->members[q] ? b->slots[q].remaining : -1;
  return SPARC_OK;
}

int sparc_batch_set_tiles(sparc_batch *b, int zchunk_mhd, int zchunk_quiet) {
  if (!b || zchunk_mhd < 11 || zchunk_quiet < 11 || zchunk_mhd > 65535 ||
      zchunk_quiet > 65535)
    return SPARC_ERR_INVALID;
  if (zchunk_mhd == b->zchunk_mhd && zchunk_quiet == b->zchunk_quiet) return SPARC_OK;
  cudaSetDevice(b->device);
  int r = pull_all(b);
  if (r) return r;
  b->zchunk_mhd = zchunk_mhd;
  b->zchunk_quiet = zchunk_quiet;
  b->dirty = true;
  b->recapture = true;  // the stage launches' shared memory depends on it
  return SPARC_OK;
}

int sparc_batch_get_tiles(const sparc_batch *b, int *zchunk_mhd, int *zchunk_quiet) {
  if (!b) return SPARC_ERR_INVALID;
  if (zchunk_mhd) *zchunk_mhd = b->zchunk_mhd;
  if (zchunk_quiet) *zchunk_quiet = b->zchunk_quiet;
  return SPARC_OK;
}

int sparc_batch_synchronize(sparc_batch *b) {
  if (!b) return SPARC_ERR_INVALID;
  cudaSetDevice(b->device);
  BCK(b, cudaStreamSynchronize(b->stream));
  return SPARC_OK;
}

int sparc_batch_stream(sparc_batch *b, void **stream) {
  if (!b || !stream) return SPARC_ERR_INVALID;
  *stream = (void *)b->stream;
  return SPARC_OK;
}

int sparc_batch_launch_count(const sparc_batch *b, int64_t *count) {
  if (!b || !count) return SPARC_ERR_INVALID;
  *count = b->launches;
  return SPARC_OK;
}

// Autotuner: picks the z extent of the MHD and of the quiet work items (the
// work items' third tile dimension; their 32 x 8 and 32 x 16 column shapes
// are fixed by the kernels' thread layout) by timing batched steps (CUDA
// events on the batch stream) over a candidate list, one axis at a time.
// The trial steps are real steps of the members.
int sparc_batch_tune(sparc_batch *b, int steps_per_trial, int *best_mhd, int *best_quiet) {
  if (!b || steps_per_trial < 1) return SPARC_ERR_INVALID;
  cudaSetDevice(b->device);
  static const int cand[] = {16, 24, 32, 48, 64, 96, 150};
  cudaEvent_t e0, e1;
  BCK(b, cudaEventCreate(&e0));
  BCK(b, cudaEventCreate(&e1));
  auto trial = [&](int zm, int zq, float *ms) -> int {
    int r = sparc_batch_set_tiles(b, zm, zq);
    if (!r) r = sparc_batch_run(b, 1);  // upload, capture, warm
    if (r) return r;
    if (!bok(b, cudaEventRecord(e0, b->stream), "cudaEventRecord")) return SPARC_ERR_CUDA;
    if ((r = sparc_batch_run(b, steps_per_trial))) return r;
    if (!bok(b, cudaEventRecord(e1, b->stream), "cudaEventRecord") ||
        !bok(b, cudaEventSynchronize(e1), "cudaEventSynchronize") ||
        !bok(b, cudaEventElapsedTime(ms, e0, e1), "cudaEventElapsedTime"))
      return SPARC_ERR_CUDA;
    return SPARC_OK;
  };
  int bm = b->zchunk_mhd, bq = b->zchunk_quiet, r = SPARC_OK;
  float best = 1e30f, ms = 0.f;
  bool any_mhd = false, any_quiet = false;
  for (int q = 0; q < b->cap; ++q)
    if (b->members[q]) (b->members[q]->magnetic ? any_mhd : any_quiet) = true;
  for (int axis = 0; axis < 2 && !r; ++axis) {
    if ((axis == 0 && !any_mhd) || (axis == 1 && !any_quiet)) continue;
    for (int c : cand) {
      const int zm = axis == 0 ? c : bm, zq = axis == 1 ? c : bq;
      if ((r = trial(zm, zq, &ms))) break;
      if (ms < best) {
        best = ms;
        bm = zm;
        bq = zq;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (r) return r;
  r = sparc_batch_set_tiles(b, bm, bq);
  if (best_mhd) *best_mhd = bm;
  if (best_quiet) *best_quiet = bq;
  return r;
}

const char *sparc_batch_last_error(const sparc_batch *b) {
  return b ? b->err.c_str() : "";
}

}  // extern "C"
