// api.cu -- the C ABI of include/sparc_gpu.h: handle lifecycle, state I/O,
// the driver-loop orchestration (stage kernels, filter passes, CUDA graphs)
// and the unit entry points.

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace sparc {

static std::string g_create_error;

bool cuda_ok(Handle *h, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  if (h) h->err = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

void *dev_alloc(Handle *h, size_t bytes) {
  void *p = nullptr;
  if (bytes == 0) bytes = 8;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    h->err = "cudaMalloc of " + std::to_string(bytes) + " bytes failed";
    cudaGetLastError();
    return nullptr;
  }
  h->allocs.push_back(p);
  return p;
}

void dev_free(Handle *h, const void *p) {
  for (size_t n = 0; n < h->allocs.size(); ++n)
    if (h->allocs[n] == p) {
      cudaFree(h->allocs[n]);
      h->allocs.erase(h->allocs.begin() + n);
      return;
    }
}

static int fail(Handle *h, int code, const std::string &msg) {
  if (h) h->err = msg;
  return code;
}

// a handle in a batch is advanced by the batch only
#define NOT_IN_BATCH(h)                                                       \
  do {                                                                        \
    if ((h)->batch) return fail((h), SPARC_ERR_ORDER, "handle is in a batch"); \
  } while (0)

static void block_partition(int n, int B, std::vector<int> &start,
                            std::vector<int> &len) {
  // rank extents, initialize.f90:77-120 (remainder to the low ranks)
  start.assign(B, 0);
  len.assign(B, n / B);
  int rem = n - (n / B) * B;
  for (int i = 0; i < rem; ++i) len[i] += 1;
  for (int b = 1; b < B; ++b) start[b] = start[b - 1] + len[b - 1];
}

static std::string validate(const sparc_params &P) {
  if (P.nx < 22 || P.ny < 22 || P.nz < 22) return "grid must be at least 22 per axis";
  if (P.magnetic < 0 || P.magnetic > 2) return "magnetic must be 0, 1 or 2";
  if (P.block_x < 1 || P.block_y < 1 || P.block_z < 2)
    return "block counts must be >= 1 (x, y) and >= 2 (z)";
  const bool hp = P.use_hpml != 0;
  if (P.periodic && hp) return "PERIODIC and USE_HPML are exclusive";
  if (!P.periodic && (P.block_x < 2 || P.block_y < 2))
    return "non-periodic runs need >= 2 blocks along x and y";
  if (P.filter_mode_xy != 1 && P.filter_mode_xy != 2) return "filter_mode_xy";
  if (P.filter_mode_z != 1 && P.filter_mode_z != 2) return "filter_mode_z";
  if (!(P.timestep > 0)) return "timestep must be positive";
  if (P.precision != SPARC_FP64 && P.precision != SPARC_FP32)
    return "precision must be SPARC_FP64 or SPARC_FP32";
  if (P.damping != 0 && P.damping != 1) return "damping must be 0 or 1";
  if (P.damping && P.precision == SPARC_FP32)
    return "DAMPING runs in the FP64 plain form only";
  if (P.precision == SPARC_FP32 && (long long)P.nx * P.ny * P.nz * 8 >= (1LL << 31))
    return "the precision form takes grids below 2^28 points";
  if (P.magnetic == 2 && (long long)P.nx * P.ny * P.nz * 8 >= (1LL << 31))
    return "MHD grids are limited to 2^28 points (32-bit indexing of 8 fields)";
  std::vector<int> s, l;
  const int dims[3] = {P.nx, P.ny, P.nz}, B[3] = {P.block_x, P.block_y, P.block_z};
  for (int a = 0; a < 3; ++a) {
    block_partition(dims[a], B[a], s, l);
    for (int b = 0; b < B[a]; ++b)
      if (l[b] < 11) return "every rank block needs >= 11 points per axis";
  }
  const bool pml = P.use_pml != 0 || hp;
  if (pml) {
    block_partition(P.nz, P.block_z, s, l);
    if (P.npml_zb < 2 || P.npml_zt < 2) return "z PML needs >= 2 points";
    if (P.npml_zb > l[0] || P.npml_zt > l[P.block_z - 1])
      return "z PML thicker than the boundary block";
  }
  if (hp) {
    if (P.npml_xb < 2 || P.npml_xt < 2 || P.npml_yb < 2 || P.npml_yt < 2)
      return "x/y PML needs >= 2 points";
    block_partition(P.nx, P.block_x, s, l);
    if (P.npml_xb > l[0] || P.npml_xt > l[P.block_x - 1]) return "x PML thicker than the boundary block";
    block_partition(P.ny, P.block_y, s, l);
    if (P.npml_yb > l[0] || P.npml_yt > l[P.block_y - 1]) return "y PML thicker than the boundary block";
  }
  return "";
}

#define CK(h, x)                                        \
  do {                                                  \
    if (!cuda_ok((h), (x), #x)) return SPARC_ERR_CUDA;  \
  } while (0)

static int alloc_face(Handle *h, int f, int n0, int n1, int n2, int np) {
  FaceDev &F = h->faces[f];
  F.on = 1;
  F.n0 = n0; F.n1 = n1; F.n2 = n2; F.np = np; F.P = h->Pp;
  F.uniform = 0;
  F.cnt = (long long)n0 * n1 * n2;
  if (h->fp32) {  // FP32 auxiliary fields; FP64 face keeps the geometry
    FaceT<float> &G = h->f_faces[f];
    G.on = 1;
    G.n0 = n0; G.n1 = n1; G.n2 = n2; G.np = np; G.P = F.P;
    G.uniform = 0;
    G.cnt = F.cnt;
    G.vars = (float *)dev_alloc(h, G.cnt * G.P * 4);
    G.scr = (float *)dev_alloc(h, G.cnt * G.P * 4);
    if (!G.vars || !G.scr) return SPARC_ERR_NOMEM;
    return SPARC_OK;
  }
  F.vars = (double *)dev_alloc(h, F.cnt * F.P * 8);
  F.scr = (double *)dev_alloc(h, F.cnt * F.P * 8);
  if (!F.vars || !F.scr) return SPARC_ERR_NOMEM;
  CK(h, cudaMemset(F.vars, 0, F.cnt * F.P * 8));
  CK(h, cudaMemset(F.scr, 0, F.cnt * F.P * 8));
  return SPARC_OK;
}

static int zero_state(Handle *h) {
  if (h->fp32) {
    for (int b = 0; b < 3; ++b)
      CK(h, cudaMemsetAsync(h->fbuf[b], 0, (size_t)h->V * h->N * 4, h->stream));
    CK(h, cudaMemsetAsync(h->f_carry, 0, (size_t)h->V * h->N * 4, h->stream));
    for (auto &F : h->f_faces)
      if (F.on) {
        CK(h, cudaMemsetAsync(F.vars, 0, F.cnt * F.P * 4, h->stream));
        CK(h, cudaMemsetAsync(F.scr, 0, F.cnt * F.P * 4, h->stream));
      }
    return SPARC_OK;
  }
  for (int b = 0; b < 3; ++b)
    CK(h, cudaMemsetAsync(h->buf[b], 0, (size_t)h->V * h->N * 8, h->stream));
  for (auto &F : h->faces)
    if (F.on) {
      CK(h, cudaMemsetAsync(F.vars, 0, F.cnt * F.P * 8, h->stream));
      CK(h, cudaMemsetAsync(F.scr, 0, F.cnt * F.P * 8, h->stream));
    }
  return SPARC_OK;
}

static void drop_graphs(Handle *h) {
  for (auto &g : h->graphs) cudaGraphExecDestroy(g.exec);
  h->graphs.clear();
}

// ------------------------------------------------------------- one step
static void rotate(Handle *h) {
  int a = h->ra;
  h->ra = h->rf1;
  h->rf1 = h->rf2;
  h->rf2 = a;
}

// precision form of enqueue_step: FP32 buffers, same roles
static int enqueue_step32(Handle *h, cudaStream_t s, int *nk) {
  SimT<float> S = make_sim32(h);
  float *a = h->fbuf[h->ra], *f1 = h->fbuf[h->rf1], *f2 = h->fbuf[h->rf2];
  int r = SPARC_OK;
  const long long l0 = h->launches;
  if (h->src.kind == SPARC_SRC_PSR && h->psr_khi > h->psr_klo) r |= launch_psr32(h, s);
  if (h->src.kind == SPARC_SRC_RANDOM) r |= launch_random_forcing(h, s);
  r |= launch_stage32(h, S, 1, a, a, f1, s);
  r |= launch_stage32(h, S, 2, a, f1, f2, s);
  r |= launch_stage32(h, S, 3, a, f2, f1, s);
  r |= launch_stage32(h, S, 4, a, f1, f2, s);
  r |= launch_stage32(h, S, 5, a, f2, f1, s);
  *nk += (int)(h->launches - l0);
  rotate(h);
  return r ? SPARC_ERR_CUDA : SPARC_OK;
}

// forcing + five stages (step.f90:26-61); a_new lands in buf[rf1]
static int enqueue_step(Handle *h, cudaStream_t s, int *nk) {
  if (h->fp32) return enqueue_step32(h, s, nk);
  SimDev S = make_simdev(h);
  double *a = h->buf[h->ra], *f1 = h->buf[h->rf1], *f2 = h->buf[h->rf2];
  int r = SPARC_OK;
  const long long l0 = h->launches;
  if (h->src.kind == SPARC_SRC_PSR && h->psr_khi > h->psr_klo) r |= launch_psr_forcing(h, S, s);
  if (h->src.kind == SPARC_SRC_RANDOM) r |= launch_random_forcing(h, s);
  // the persistent MHD stages' work counters
  if (h->d_wctr64 && cudaMemsetAsync(h->d_wctr64, 0, 5 * sizeof(unsigned), s) != cudaSuccess)
    r |= SPARC_ERR_CUDA;
  // stage k reads temp_k and writes temp_{k+1}; stage 5 writes a_new.
  // DAMPING: the velocity damping terms of each stage's input first
  const double *tins[5] = {a, f1, f2, f1, f2};
  double *sos[5] = {f1, f2, f1, f2, f1};
  for (int st = 0; st < 5; ++st) {
    if (h->damping) r |= damping_enqueue(h, tins[st], s);
    r |= launch_stage(h, S, st + 1, a, tins[st], sos[st], s);
  }
  *nk += (int)(h->launches - l0);
  rotate(h);
  return r ? SPARC_ERR_CUDA : SPARC_OK;
}

// filter kind after iteration nn: bit 0 xy, bit 1 z (driver.f90:200,
// derivatives.f90:669, 690)
static int filter_kind(Handle *h, long long nn) {
  if (nn == 0) return 0;
  int fk = 0;
  if (nn % h->xyfreq == 0) fk |= 1;
  if (nn % h->zfreq == 0) fk |= 2;
  return fk;
}

// precision form: the first pass of an event filters the compensated
// value stored - carry; the filtered state starts a new compensated sum
// (its carry is cleared after the passes)
static int enqueue_filter32(Handle *h, int fk, cudaStream_t s, int *nk) {
  int r = SPARC_OK;
  if (fk & 1) {  // y then x, fused
    r |= launch_filter_event32(h, true, h->fbuf[h->ra], h->f_carry, h->fbuf[h->rf1], s);
    rotate(h);
    ++*nk;
  }
  if (fk & 2) {
    r |= launch_filter_event32(h, false, h->fbuf[h->ra], (fk & 1) ? nullptr : h->f_carry,
                               h->fbuf[h->rf1], s);
    rotate(h);
    ++*nk;
  }
  if (fk && cudaMemsetAsync(h->f_carry, 0, (size_t)h->V * h->N * 4, s) != cudaSuccess)
    r = SPARC_ERR_CUDA;
  return r ? SPARC_ERR_CUDA : SPARC_OK;
}

static int enqueue_filter(Handle *h, int fk, cudaStream_t s, int *nk) {
  if (h->fp32) return enqueue_filter32(h, fk, s, nk);
  int r = SPARC_OK;
  if (fk & 1) {  // y then x, fused
    r |= launch_filter_event(h, true, h->buf[h->ra], h->buf[h->rf1], s);
    rotate(h);
    ++*nk;
  }
  if (fk & 2) {
    r |= launch_filter_event(h, false, h->buf[h->ra], h->buf[h->rf1], s);
    rotate(h);
    ++*nk;
  }
  return r ? SPARC_ERR_CUDA : SPARC_OK;
}

// The driver iteration lives in device memory so that captured graphs
// replay without parameter updates; it is set by a one-thread kernel whose
// argument is captured at launch (a pinned staging word could be rewritten
// by the host before an earlier asynchronous copy from it has run).
__global__ void k_set_iter(long long *d, long long nn) { *d = nn; }

static int set_iter(Handle *h, long long nn) {
  k_set_iter<<<1, 1, 0, h->stream>>>(h->d_iter, nn);
  ++h->launches;
  CK(h, cudaGetLastError());
  return SPARC_OK;
}

static Handle::GraphEntry *graph_for(Handle *h, int fk) {
  for (auto &g : h->graphs)
    if (g.ra == h->ra && g.rf1 == h->rf1 && g.rf2 == h->rf2 && g.fk == fk)
      return &g;
  Handle::GraphEntry e{h->ra, h->rf1, h->rf2, fk, nullptr, 0, 0, 0, 0};
  const int ra = h->ra, rf1 = h->rf1, rf2 = h->rf2;
  const long long launches = h->launches;
  cudaGraph_t graph;
  if (!cuda_ok(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal),
               "cudaStreamBeginCapture"))
    return nullptr;
  int nk = 0;
  int r = enqueue_step(h, h->stream, &nk);
  r |= enqueue_filter(h, fk, h->stream, &nk);
  cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
  // the roles the iteration leaves (as many rotations as its launches made)
  e.out_ra = h->ra; e.out_rf1 = h->rf1; e.out_rf2 = h->rf2;
  h->ra = ra; h->rf1 = rf1; h->rf2 = rf2;  // capture does not execute
  h->launches = launches;
  if (r || !cuda_ok(h, ce, "cudaStreamEndCapture")) return nullptr;
  if (!cuda_ok(h, cudaGraphInstantiate(&e.exec, graph, 0), "cudaGraphInstantiate")) {
    cudaGraphDestroy(graph);
    return nullptr;
  }
  cudaGraphDestroy(graph);
  e.nkernels = nk;
  h->graphs.push_back(e);
  return &h->graphs.back();
}

// f(i) for i in [0, n) on the host's cores (state conversion of the
// precision form: one (field, layer) plane per index)
template <class F>
static void parallel_for(long long n, F f) {
  const long long nt = std::max<long long>(
      1, std::min<long long>(n, std::min(16u, std::max(1u, std::thread::hardware_concurrency()))));
  std::vector<std::thread> th;
  for (long long w = 0; w < nt; ++w)
    th.emplace_back([=, &f] {
      for (long long i = w; i < n; i += nt) f(i);
    });
  for (auto &t : th) t.join();
}

// Failure injection: one thread waits on an mbarrier that expects one
// arrival which never comes; the bounded wait gives up after `polls` polls
// or 10 ms of the global timer, whichever comes first, and raises the error
// flag, as a stage kernel's gave-up wait does.
__global__ void k_wait_probe(int *err, long long polls) {
  __shared__ unsigned long long bar;
  if (threadIdx.x != 0) return;
  const unsigned a = (unsigned)__cvta_generic_to_shared(&bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  unsigned long long t0, t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (long long n = 0; n < polls; ++n) {
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 > 10000000ull) break;
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(0u)
        : "memory");
    if (ok) return;
  }
  atomicExch(err, 1);
}

}  // namespace sparc

using namespace sparc;

struct sparc_handle : Handle {};

extern "C" {

int sparc_create(const sparc_params *p, int device, sparc_handle **out) {
  if (!p || !out) return SPARC_ERR_INVALID;
  *out = nullptr;
  std::string e = validate(*p);
  if (!e.empty()) {
    g_create_error = e;
    return SPARC_ERR_INVALID;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    g_create_error = "no CUDA device";
    return SPARC_ERR_NODEVICE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
    g_create_error = "the kernels are built for sm_100a only";
    return SPARC_ERR_NODEVICE;
  }
  sparc_handle *h = new (std::nothrow) sparc_handle();
  if (!h) return SPARC_ERR_NOMEM;
  h->P = *p;
  h->device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete h;
    return SPARC_ERR_CUDA;
  }
  h->nx = p->nx; h->ny = p->ny; h->nz = p->nz;
  h->N = (long long)h->nx * h->ny * h->nz;
  h->magnetic = p->magnetic == 2;
  h->quiet = p->magnetic == 0;
  h->periodic = p->periodic != 0;
  h->use_hpml = p->use_hpml != 0;
  h->use_pml = p->use_pml != 0 || h->use_hpml;
  h->V = h->magnetic ? 8 : 5;
  h->fp32 = p->precision == SPARC_FP32;
  h->damping = p->damping != 0;
  h->Pp = h->magnetic ? 6 : 2;
  h->gxy = p->filter_mode_xy == 1 ? 5 : 3;
  h->gz = p->filter_mode_z == 1 ? 5 : 3;
  const double tz = std::max(p->t_z, p->timestep), txy = std::max(p->t_xy, p->timestep);
  h->zfreq = (int)std::floor(tz / p->timestep + 1.0e-5);  // initialize.f90:1911-1912
  h->xyfreq = (int)std::floor(txy / p->timestep + 1.0e-5);
  // axes and horizontal metrics, initialize.f90:468-517
  h->xaxis.resize(h->nx);
  h->yaxis.resize(h->ny);
  for (int i = 0; i < h->nx; ++i)
    h->xaxis[i] = h->periodic ? (double)i / (double)h->nx : (double)i / (double)(h->nx - 1);
  for (int j = 0; j < h->ny; ++j)
    h->yaxis[j] = h->periodic ? (double)j / (double)h->ny : (double)j / (double)(h->ny - 1);
  h->stretchx = h->periodic ? RSUN / p->xlength * h->nx : RSUN / p->xlength * (h->nx - 1);
  h->stretchy = h->periodic ? RSUN / p->ylength * h->ny : RSUN / p->ylength * (h->ny - 1);
  block_partition(h->nx, p->block_x, h->bxs, h->bxl);
  block_partition(h->ny, p->block_y, h->bys, h->byl);
  block_partition(h->nz, p->block_z, h->bzs, h->bzl);
  h->nblocks = p->block_x * p->block_y * p->block_z;
  std::vector<int> cols(h->nx + h->ny + h->nz);
  for (int i = 0; i < h->nx; ++i) {
    int b = 0;
    while (b + 1 < p->block_x && i >= h->bxs[b + 1]) ++b;
    cols[i] = b;
  }
  for (int j = 0; j < h->ny; ++j) {
    int b = 0;
    while (b + 1 < p->block_y && j >= h->bys[b + 1]) ++b;
    cols[h->nx + j] = b;
  }
  for (int k = 0; k < h->nz; ++k) {
    int b = 0;
    while (b + 1 < p->block_z && k >= h->bzs[b + 1]) ++b;
    cols[h->nx + h->ny + k] = b;
  }
  if (const char *kv = std::getenv("SPARC_TMA32"))  // A/B timing only
    h->allow_tma32 = std::atoi(kv) != 0;
  if (const char *kv = std::getenv("SPARC_TMA64"))  // A/B timing only
    h->allow_tma64 = std::atoi(kv) != 0;
  int r = SPARC_OK;
  // A handle's streams take the device's greatest priority: when a handle
  // is set up beside a running batch (serving), its set-up kernels are
  // scheduled ahead of the batch launches queued at the same time.
  int prio_least = 0, prio_greatest = 0;
  if (cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest) != cudaSuccess) {
    cudaGetLastError();
    prio_greatest = 0;
  }
  if (!cuda_ok(h, cudaStreamCreateWithPriority(&h->stream, cudaStreamNonBlocking, prio_greatest),
               "stream") ||
      !cuda_ok(h, cudaStreamCreateWithPriority(&h->aux, cudaStreamNonBlocking, prio_greatest),
               "stream") ||
      !cuda_ok(h, cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming), "event") ||
      !cuda_ok(h, cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming), "event")) {
    r = SPARC_ERR_CUDA;
  }
  if (!r && (setup_constants() || step_constants() || filter_constants() ||
             step32_constants()))
    r = fail(h, SPARC_ERR_CUDA, "constant upload failed");
  if (!r && stage_geometry(h))
    r = fail(h, SPARC_ERR_INVALID, "no tile shape fits this grid");
  if (!r) {
    h->d_colx = (int *)dev_alloc(h, cols.size() * sizeof(int));
    if (!h->d_colx) r = SPARC_ERR_NOMEM;
    else {
      h->d_coly = h->d_colx + h->nx;
      if (cudaMemcpyAsync(h->d_colx, cols.data(), cols.size() * sizeof(int),
                          cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
        r = SPARC_ERR_CUDA;
    }
  }
  for (int b = 0; !r && b < 3; ++b) {
    if (h->fp32) {
      h->fbuf[b] = (float *)dev_alloc(h, (size_t)h->V * h->N * 4);
      if (!h->fbuf[b]) r = SPARC_ERR_NOMEM;
    } else {
      h->buf[b] = (double *)dev_alloc(h, (size_t)h->V * h->N * 8);
      if (!h->buf[b]) r = SPARC_ERR_NOMEM;
    }
  }
  if (!r && h->fp32) {
    h->f_carry = (float *)dev_alloc(h, (size_t)h->V * h->N * 4);
    if (!h->f_carry) r = SPARC_ERR_NOMEM;
  }
  if (!r && h->use_pml) {
    r |= alloc_face(h, 0, h->nx, h->ny, p->npml_zb, p->npml_zb);
    r |= alloc_face(h, 1, h->nx, h->ny, p->npml_zt, p->npml_zt);
  }
  if (!r && h->use_hpml) {
    r |= alloc_face(h, 2, p->npml_xb, h->ny, h->nz, p->npml_xb);
    r |= alloc_face(h, 3, p->npml_xt, h->ny, h->nz, p->npml_xt);
    r |= alloc_face(h, 4, h->nx, p->npml_yb, h->nz, p->npml_yb);
    r |= alloc_face(h, 5, h->nx, p->npml_yt, h->nz, p->npml_yt);
  }
  if (!r) {
    h->d_err = (int *)dev_alloc(h, 4);
    if (!h->d_err || cudaMemset(h->d_err, 0, 4) != cudaSuccess) r = SPARC_ERR_NOMEM;
  }
  if (!r) {
    h->d_iter = (long long *)dev_alloc(h, 8);
    h->d_fail = (long long *)dev_alloc(h, 8);
    h->d_partials = (double *)dev_alloc(h, (size_t)h->partials_blocks * 3 * 8);
    h->d_diag = (double *)dev_alloc(h, 4 * 8);
    h->d_counter = (unsigned int *)dev_alloc(h, 4);
    if (!h->d_iter || !h->d_fail || !h->d_partials || !h->d_diag || !h->d_counter)
      r = SPARC_ERR_NOMEM;
  }
  if (!r) {
    long long m1 = -1;
    double d4[4] = {0, 0, 0, -1};
    // ordered on the handle's stream; synchronised before m1 and d4 go
    if (cudaMemcpyAsync(h->d_fail, &m1, 8, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        cudaMemcpyAsync(h->d_iter, &m1, 8, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        cudaMemcpyAsync(h->d_diag, d4, 32, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        cudaMemsetAsync(h->d_counter, 0, 4, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
      r = SPARC_ERR_CUDA;
  }
  if (!r) r = zero_state(h);
  if (r) {
    g_create_error = h->err.empty() ? "allocation failed" : h->err;
    sparc_destroy(h);
    return r;
  }
  h->src.kind = SPARC_SRC_NONE;
  *out = h;
  return SPARC_OK;
}

int sparc_destroy(sparc_handle *h) {
  if (!h) return SPARC_ERR_INVALID;
  NOT_IN_BATCH(h);
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  drop_graphs(h);
  damping_destroy(h);
  for (void *p : h->allocs) cudaFree(p);
  if (h->aux) cudaStreamSynchronize(h->aux);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  if (h->aux) cudaStreamDestroy(h->aux);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return SPARC_OK;
}

int sparc_set_background(sparc_handle *h, const double *rho0,
                         const double *pre0, const double *cs0,
                         const double *bx0, const double *by0,
                         const double *bz0, const double *zaxis_mm,
                         const double *grav) {
  if (!h || !rho0 || !pre0 || !cs0 || !zaxis_mm || !grav)
    return fail(h, SPARC_ERR_INVALID, "missing background array");
  if (h->magnetic && (!bx0 || !by0 || !bz0))
    return fail(h, SPARC_ERR_INVALID, "MHD needs bx0, by0, bz0");
  if (h->bg_ready) return fail(h, SPARC_ERR_ORDER, "background already set");
  cudaSetDevice(h->device);
  int r = setup_background(h, rho0, pre0, cs0, bx0, by0, bz0, zaxis_mm, grav);
  if (r) return r;
  if (h->damping && (r = damping_setup(h))) return r == SPARC_ERR_CUDA ? fail(h, r, h->err) : r;
  if ((r = mhd64_plan(h))) return fail(h, r, "MHD stage plan");
  if (h->fp32) {
    r = setup32(h);
    if (r) return r;
    h->h_scale.resize((size_t)2 * h->V * h->nz);
    CK(h, cudaMemcpy(h->h_scale.data(), h->f_sc, h->h_scale.size() * 4,
                     cudaMemcpyDeviceToHost));
  } else {
    r = encode_tensor_maps(h);
    if (r) return r;
  }
  r = zero_state(h);
  if (r) return r;
  h->bg_ready = true;
  return cudaStreamSynchronize(h->stream) == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

// psr rank-block culling, all_modules.f90:594-598 (global form per block)
static bool psr_in_block(const Handle *h, const sparc_pulse &q, int b) {
  const int BX = h->P.block_x, BY = h->P.block_y;
  int bxi = b % BX, byi = (b / BX) % BY, bzi = b / (BX * BY);
  const auto &xa = h->xaxis, &ya = h->yaxis, &za = h->zaxis;
  double x1 = xa[h->bxs[bxi]], xN = xa[h->bxs[bxi] + h->bxl[bxi] - 1];
  double y1 = ya[h->bys[byi]], yN = ya[h->bys[byi] + h->byl[byi] - 1];
  double z1 = za[h->bzs[bzi]], zN = za[h->bzs[bzi] + h->bzl[bzi] - 1];
  auto mod1 = [](double v) { return v - std::floor(v); };
  bool cx = ((mod1(q.px + 3.0 * q.sr) >= x1) || (q.px + 3.0 * q.sr >= xa[h->nx - 1])) &&
            ((mod1(q.px - 3.0 * q.sr) <= xN) || (q.px - 3.0 * q.sr <= xa[0]));
  bool cy = ((mod1(q.py + 3.0 * q.sr) >= y1) || (q.py + 3.0 * q.sr >= ya[h->ny - 1])) &&
            ((mod1(q.py - 3.0 * q.sr) <= yN) || (q.py - 3.0 * q.sr <= ya[0]));
  bool cz = (q.pz + 3.0 * q.sz >= z1) && (q.pz - 3.0 * q.sz <= zN);
  return cx && cy && cz;
}

int sparc_set_source(sparc_handle *h, const sparc_source *s) {
  if (!h || !s) return SPARC_ERR_INVALID;
  NOT_IN_BATCH(h);
  if (!h->bg_ready) return fail(h, SPARC_ERR_ORDER, "set the background first");
  if (s->kind < SPARC_SRC_NONE || s->kind > SPARC_SRC_RANDOM)
    return fail(h, SPARC_ERR_INVALID, "unknown source kind");
  if (s->kind != SPARC_SRC_NONE && s->kind != SPARC_SRC_RANDOM && (s->dir < 1 || s->dir > 3))
    return fail(h, SPARC_ERR_INVALID, "pulse_dir must be 1, 2 or 3");
  if (s->kind == SPARC_SRC_RANDOM && (s->nseries < 1 || !s->series || !(s->cadforcing > 0.0)))
    return fail(h, SPARC_ERR_INVALID, "forcing series (nseries >= 1, cadforcing > 0)");
  if (s->kind == SPARC_SRC_PSR && (s->npulses < 0 || (s->npulses > 0 && !s->pulses)))
    return fail(h, SPARC_ERR_INVALID, "pulse table");
  cudaSetDevice(h->device);
  CK(h, cudaStreamSynchronize(h->stream));
  drop_graphs(h);
  h->src = *s;
  h->src.pulses = nullptr;
  h->src.series = nullptr;
  const int nx = h->nx, ny = h->ny, nz = h->nz;
  const double diml = h->diml;
  if (s->kind == SPARC_SRC_RANDOM) {
    // driver.f90:80: vr = (randomexciteampl/dimc)*vr; the forcing acts on v_z
    h->src.dir = 3;
    const double f = s->rnd_ampl / h->dimc;
    const size_t n = (size_t)nx * ny * s->nseries;
    std::vector<double> vr(n);
    for (size_t q = 0; q < n; ++q) vr[q] = f * s->series[q];
    // e_rad and source_dep (all_modules.f90:289-301)
    const double temp2 = 1.0 + s->rnd_depth / RSUN;
    double temp = 1.0;
    int e_rad = 0;
    for (int k = 0; k < nz; ++k)
      if (std::fabs(h->zaxis[k] - temp2) <= temp) {
        temp = std::fabs(h->zaxis[k] - temp2);
        e_rad = k;
      }
    std::vector<double> dep(nz);
    const double sg = s->rnd_sigma / RSUN;
    for (int k = 0; k < nz; ++k) {
      const double d = h->zaxis[k] - h->zaxis[e_rad];
      dep[k] = std::exp(-0.5 * (d * d) / 2.0 / (sg * sg));
    }
    dev_free(h, h->d_series);
    h->d_series = (double *)dev_alloc(h, n * 8);
    if (!h->d_sdep) h->d_sdep = (double *)dev_alloc(h, (size_t)nz * 8);
    if (!h->d_f2d) h->d_f2d = (double *)dev_alloc(h, (size_t)nx * ny * 8);
    if (!h->d_series || !h->d_sdep || !h->d_f2d) return SPARC_ERR_NOMEM;
    CK(h, cudaMemcpyAsync(h->d_series, vr.data(), n * 8, cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaMemcpyAsync(h->d_sdep, dep.data(), (size_t)nz * 8, cudaMemcpyHostToDevice,
                          h->stream));
  }
  if (s->kind == SPARC_SRC_PULSE) {
    // driver.f90:140-145, split into x, y, z factors
    std::vector<double> t(nx + ny + nz);
    const double sr = s->sr / diml, sz = s->sz / diml;
    for (int i = 0; i < nx; ++i) {
      double a = h->xaxis[i] * h->P.xlength / RSUN - s->px / diml;
      t[i] = std::exp(-1.0 * (a * a) / (2.0 * (sr * sr)));
    }
    for (int j = 0; j < ny; ++j) {
      double a = h->yaxis[j] * h->P.ylength / RSUN - s->py / diml;
      t[nx + j] = std::exp(-1.0 * (a * a) / (2.0 * (sr * sr)));
    }
    for (int k = 0; k < nz; ++k) {
      double a = h->zaxis[k] - (s->pz / diml + 1.0);
      t[nx + ny + k] = std::exp(-1.0 * (a * a) / (2.0 * (sz * sz)));
    }
    if (!h->d_fx) {
      h->d_fx = (double *)dev_alloc(h, t.size() * 8);
      if (!h->d_fx) return SPARC_ERR_NOMEM;
      h->d_fy = h->d_fx + nx;
      h->d_fz = h->d_fx + nx + ny;
    }
    CK(h, cudaMemcpyAsync(h->d_fx, t.data(), t.size() * 8, cudaMemcpyHostToDevice, h->stream));
  } else if (s->kind == SPARC_SRC_PSR) {
    const int np = s->npulses;
    h->pulses.assign(s->pulses, s->pulses + np);
    // separable factors of all_modules.f90:602-607
    std::vector<double> px((size_t)np * nx), py((size_t)np * ny), pt(3 * (size_t)np);
    std::vector<unsigned char> mask((size_t)np * h->nblocks);
    for (int n = 0; n < np; ++n) {
      const sparc_pulse &q = h->pulses[n];
      for (int i = 0; i < nx; ++i) {
        double x = h->xaxis[i];
        double m = std::min(std::min((x - q.px) * (x - q.px), (x - 1.0 - q.px) * (x - 1.0 - q.px)),
                            (x + 1.0 - q.px) * (x + 1.0 - q.px));
        px[(size_t)n * nx + i] = std::exp(-m / (2.0 * (q.sr * q.sr)));
      }
      for (int j = 0; j < ny; ++j) {
        double y = h->yaxis[j];
        double m = std::min(std::min((y - q.py) * (y - q.py), (y - 1.0 - q.py) * (y - 1.0 - q.py)),
                            (y + 1.0 - q.py) * (y + 1.0 - q.py));
        py[(size_t)n * ny + j] = std::exp(-m / (2.0 * (q.sr * q.sr)));
      }
      pt[3 * n] = q.amp; pt[3 * n + 1] = q.t0; pt[3 * n + 2] = q.t1;
      for (int b = 0; b < h->nblocks; ++b)
        mask[(size_t)n * h->nblocks + b] = psr_in_block(h, q, b);
    }
    // per-layer pulse lists; a pulse leaves a layer where its depth factor
    // is below 1e-40 (far below FP64 resolution of any nearby sum)
    std::vector<int> off(nz + 1, 0), idx;
    std::vector<double> zv;
    int klo = nz, khi = 0;
    for (int k = 0; k < nz; ++k) {
      off[k] = (int)idx.size();
      for (int n = 0; n < np; ++n) {
        const sparc_pulse &q = h->pulses[n];
        double d = h->zaxis[k] - q.pz;
        double ez = std::exp(-(d * d) / (2.0 * (q.sz * q.sz)));
        if (ez < 1e-40) continue;
        idx.push_back(n);
        zv.push_back(h->invrho0q[k] * ez);
        klo = std::min(klo, k);
        khi = std::max(khi, k + 1);
      }
    }
    off[nz] = (int)idx.size();
    if (khi <= klo) { klo = 0; khi = 0; }
    h->psr_klo = klo;
    h->psr_khi = khi;
    // a later call replaces the tables of an earlier one
    for (const void *p : {(const void *)h->d_px, (const void *)h->d_py, (const void *)h->d_ptime,
                          (const void *)h->d_pmask, (const void *)h->d_plane_off,
                          (const void *)h->d_plane_idx, (const void *)h->d_plane_z,
                          (const void *)h->d_psr})
      dev_free(h, p);
    auto upd = [&](void *&dst, const void *src, size_t bytes) -> int {
      dst = dev_alloc(h, bytes);
      if (!dst) return SPARC_ERR_NOMEM;
      if (bytes && cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream) !=
                       cudaSuccess)
        return SPARC_ERR_CUDA;
      return SPARC_OK;
    };
    int r = 0;
    void *v;
    r |= upd(v, px.data(), px.size() * 8); h->d_px = (double *)v;
    r |= upd(v, py.data(), py.size() * 8); h->d_py = (double *)v;
    r |= upd(v, pt.data(), pt.size() * 8); h->d_ptime = (double *)v;
    r |= upd(v, mask.data(), mask.size()); h->d_pmask = (unsigned char *)v;
    r |= upd(v, off.data(), off.size() * 4); h->d_plane_off = (int *)v;
    r |= upd(v, idx.data(), idx.size() * 4); h->d_plane_idx = (int *)v;
    r |= upd(v, zv.data(), zv.size() * 8); h->d_plane_z = (double *)v;
    h->d_psr = (double *)dev_alloc(h, std::max<size_t>(8, (size_t)(khi - klo) * nx * ny * 8));
    if (r || !h->d_psr) return r ? r : SPARC_ERR_NOMEM;
  }
  // the uploads above are ordered on the handle's stream
  if (h->fp32) return source32(h);
  CK(h, cudaStreamSynchronize(h->stream));
  return SPARC_OK;
}

int sparc_sizes(const sparc_handle *h, int64_t *ns, int64_t *np) {
  if (!h) return SPARC_ERR_INVALID;
  if (ns) *ns = (int64_t)h->V * h->N;
  int64_t t = 0;
  for (const auto &F : h->faces)
    if (F.on) t += F.cnt * F.P;
  if (np) *np = t;
  return SPARC_OK;
}

// precision form: stored = float(sc * a), carry 0; a = (stored - carry)/sc
static int set_state32(Handle *h, const double *a, const double *psi) {
  const long long N = h->N;
  const int nz = h->nz;
  const long long NXY = (long long)h->nx * h->ny;
  if (a && h->h_scale.empty()) return fail(h, SPARC_ERR_ORDER, "set the background first");
  if (a) {
    std::vector<float> t((size_t)h->V * N);
    parallel_for((long long)h->V * nz, [&](long long lk) {
      const double sc = h->h_scale[(size_t)lk];  // field l = lk / nz, layer lk % nz
      const size_t o = (size_t)lk * NXY;
      for (long long n = 0; n < NXY; ++n) t[o + n] = (float)(sc * a[o + n]);
    });
    // ordered on the handle's (non-blocking) stream, done before t goes
    CK(h, cudaMemcpyAsync(h->fbuf[h->ra], t.data(), t.size() * 4, cudaMemcpyHostToDevice,
                          h->stream));
    CK(h, cudaMemsetAsync(h->f_carry, 0, t.size() * 4, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
  }
  if (psi) {
    size_t off = 0;
    for (auto &F : h->f_faces)
      if (F.on) {
        std::vector<float> t(F.cnt * F.P);
        for (size_t n = 0; n < t.size(); ++n) t[n] = (float)psi[off + n];
        CK(h, cudaMemcpyAsync(F.vars, t.data(), t.size() * 4, cudaMemcpyHostToDevice,
                              h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        off += t.size();
      }
  }
  return SPARC_OK;
}

static int get_state32(Handle *h, double *a, double *psi) {
  const long long N = h->N;
  const int nz = h->nz, V = h->V;
  const long long NXY = (long long)h->nx * h->ny;
  CK(h, cudaStreamSynchronize(h->stream));
  if (a) {
    if (h->h_scale.empty()) return fail(h, SPARC_ERR_ORDER, "set the background first");
    std::vector<float> t((size_t)V * N), c((size_t)V * N);
    CK(h, cudaMemcpy(t.data(), h->fbuf[h->ra], t.size() * 4, cudaMemcpyDeviceToHost));
    CK(h, cudaMemcpy(c.data(), h->f_carry, c.size() * 4, cudaMemcpyDeviceToHost));
    parallel_for((long long)V * nz, [&](long long lk) {
      const double isc = h->h_scale[(size_t)V * nz + (size_t)lk];
      const size_t o = (size_t)lk * NXY;
      for (long long n = 0; n < NXY; ++n) a[o + n] = ((double)t[o + n] - (double)c[o + n]) * isc;
    });
  }
  if (psi) {
    size_t off = 0;
    for (auto &F : h->f_faces)
      if (F.on) {
        std::vector<float> t(F.cnt * F.P);
        CK(h, cudaMemcpy(t.data(), F.vars, t.size() * 4, cudaMemcpyDeviceToHost));
        for (size_t n = 0; n < t.size(); ++n) psi[off + n] = t[n];
        off += t.size();
      }
  }
  return SPARC_OK;
}

int sparc_set_state(sparc_handle *h, const double *a, const double *psi) {
  if (!h) return SPARC_ERR_INVALID;
  NOT_IN_BATCH(h);
  cudaSetDevice(h->device);
  // a restart from saved state clears the device error flag
  if (h->fp32) {
    CK(h, cudaStreamSynchronize(h->stream));
    const int r = set_state32(h, a, psi);
    if (r != SPARC_OK) return r;
    CK(h, cudaMemsetAsync(h->d_err, 0, 4, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return SPARC_OK;
  }
  if (a)
    CK(h, cudaMemcpyAsync(h->buf[h->ra], a, (size_t)h->V * h->N * 8,
                          cudaMemcpyHostToDevice, h->stream));
  if (psi) {
    size_t off = 0;
    for (auto &F : h->faces)
      if (F.on) {
        CK(h, cudaMemcpyAsync(F.vars, psi + off, F.cnt * F.P * 8,
                              cudaMemcpyHostToDevice, h->stream));
        off += F.cnt * F.P;
      }
  }
  CK(h, cudaMemsetAsync(h->d_err, 0, 4, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return SPARC_OK;
}

int sparc_inject_wait_timeout(sparc_handle *h, int64_t polls) {
  if (!h) return SPARC_ERR_INVALID;
  NOT_IN_BATCH(h);
  if (polls < 1 || polls > (1LL << 20))
    return fail(h, SPARC_ERR_INVALID, "polls must be in [1, 2^20]");
  cudaSetDevice(h->device);
  k_wait_probe<<<1, 32, 0, h->stream>>>(h->d_err, (long long)polls);
  ++h->launches;
  CK(h, cudaGetLastError());
  return SPARC_OK;
}

int sparc_get_state(sparc_handle *h, double *a, double *psi) {
  if (!h) return SPARC_ERR_INVALID;
  NOT_IN_BATCH(h);
  cudaSetDevice(h->device);
  if (h->fp32) return get_state32(h, a, psi);
  if (a)
    CK(h, cudaMemcpyAsync(a, h->buf[h->ra], (size_t)h->V * h->N * 8,
                          cudaMemcpyDeviceToHost, h->stream));
  if (psi) {
    size_t off = 0;
    for (auto &F : h->faces)
      if (F.on) {
        CK(h, cudaMemcpyAsync(psi + off, F.vars, F.cnt * F.P * 8,
                              cudaMemcpyDeviceToHost, h->stream));
        off += F.cnt * F.P;
      }
  }
  CK(h, cudaStreamSynchronize(h->stream));
  return SPARC_OK;
}

int sparc_step(sparc_handle *h, int64_t nn) {
  if (!h) return SPARC_ERR_INVALID;
  NOT_IN_BATCH(h);
  if (!h->bg_ready) return fail(h, SPARC_ERR_ORDER, "set the background first");
  cudaSetDevice(h->device);
  int r = set_iter(h, nn);
  if (r) return r;
  int nk = 0;
  r = enqueue_step(h, h->stream, &nk);
  return r;
}

int sparc_filter_vars(sparc_handle *h, int64_t nn) {
  if (!h) return SPARC_ERR_INVALID;
  NOT_IN_BATCH(h);
  if (!h->bg_ready) return fail(h, SPARC_ERR_ORDER, "set the background first");
  cudaSetDevice(h->device);
  int nk = 0;
  return enqueue_filter(h, filter_kind(h, nn), h->stream, &nk);
}

int sparc_run(sparc_handle *h, int64_t first, int64_t count) {
  if (!h || count < 0) return SPARC_ERR_INVALID;
  NOT_IN_BATCH(h);
  if (!h->bg_ready) return fail(h, SPARC_ERR_ORDER, "set the background first");
  cudaSetDevice(h->device);
  int r = set_iter(h, first);
  if (r) return r;
  for (int64_t nn = first; nn < first + count; ++nn) {
    const int fk = filter_kind(h, nn);
    Handle::GraphEntry *g = graph_for(h, fk);
    if (!g) return SPARC_ERR_CUDA;
    CK(h, cudaGraphLaunch(g->exec, h->stream));
    h->launches += g->nkernels;
    // roles after the step and the filter passes, as recorded at capture
    h->ra = g->out_ra;
    h->rf1 = g->out_rf1;
    h->rf2 = g->out_rf2;
  }
  return SPARC_OK;
}

// z extent of the stage kernels' work items; the captured graphs hold the
// old launch shapes and are dropped
static int set_zchunk(Handle *h, int zc) {
  zc = std::min(zc, h->nz);
  const long long per = (long long)h->max_stage_blocks / ((h->nz + h->zchunk - 1) / h->zchunk);
  const long long blocks = per * ((h->nz + zc - 1) / zc);
  if (blocks > h->partials_blocks) return SPARC_ERR_INVALID;
  if (zc != h->zchunk) drop_graphs(h);
  h->zchunk = zc;
  h->max_stage_blocks = (int)blocks;
  return SPARC_OK;
}

int sparc_set_zchunk(sparc_handle *h, int zchunk) {
  if (!h || zchunk < 11) return SPARC_ERR_INVALID;
  NOT_IN_BATCH(h);
  cudaSetDevice(h->device);
  CK(h, cudaStreamSynchronize(h->stream));  // graphs in flight finish first
  return set_zchunk(h, zchunk) ? fail(h, SPARC_ERR_INVALID, "z chunk out of range") : SPARC_OK;
}

int sparc_get_zchunk(const sparc_handle *h, int *zchunk) {
  if (!h || !zchunk) return SPARC_ERR_INVALID;
  *zchunk = h->zchunk;
  return SPARC_OK;
}

// Autotuner of the z extent: iterations first, first+1, ... of the driver
// loop run as in sparc_run; each candidate extent gets one untimed
// iteration (new launch shapes), then `steps_per_trial` iterations off the
// filter cadence are timed with CUDA events on the handle's stream (the
// filter iterations between them run untimed, so every candidate is timed
// on the same kind of iteration).  The fastest extent is kept.  Results do
// not depend on the extent.
int sparc_tune(sparc_handle *h, int64_t first, int steps_per_trial, int64_t *next,
               int *best) {
  if (!h || first < 0 || steps_per_trial < 1 || steps_per_trial > 1000)
    return SPARC_ERR_INVALID;
  NOT_IN_BATCH(h);
  if (!h->bg_ready) return fail(h, SPARC_ERR_ORDER, "set the background first");
  cudaSetDevice(h->device);
  static const int cand[] = {16, 24, 32, 40, 48, 64, 80, 100, 150};
  std::vector<int> cs;
  for (int c : cand) {
    const int z = std::min(c, h->nz);
    if (std::find(cs.begin(), cs.end(), z) == cs.end()) cs.push_back(z);
  }
  int r = set_iter(h, first);
  if (r) return r;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(h, cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail(h, SPARC_ERR_CUDA, "cudaEventCreate");
  }
  int64_t nn = first;
  auto one = [&](int64_t it) -> int {
    Handle::GraphEntry *g = graph_for(h, filter_kind(h, it));
    if (!g) return SPARC_ERR_CUDA;
    if (!cuda_ok(h, cudaGraphLaunch(g->exec, h->stream), "cudaGraphLaunch"))
      return SPARC_ERR_CUDA;
    h->launches += g->nkernels;
    h->ra = g->out_ra;
    h->rf1 = g->out_rf1;
    h->rf2 = g->out_rf2;
    return SPARC_OK;
  };
  float best_ms = 3.4e38f;
  int bz = h->zchunk;
  for (int c : cs) {
    if (set_zchunk(h, c)) continue;  // more blocks than the partials hold
    // the off-cadence graph is captured before anything is timed
    if (!graph_for(h, 0)) { r = SPARC_ERR_CUDA; break; }
    if ((r = one(nn++))) break;
    float tot = 0.f;
    for (int timed = 0; timed < steps_per_trial && !r; ++nn) {
      if (filter_kind(h, nn) != 0) {
        r = one(nn);
        continue;
      }
      float ms = 0.f;
      if (!cuda_ok(h, cudaEventRecord(e0, h->stream), "cudaEventRecord") || (r = one(nn)) ||
          !cuda_ok(h, cudaEventRecord(e1, h->stream), "cudaEventRecord") ||
          !cuda_ok(h, cudaEventSynchronize(e1), "cudaEventSynchronize") ||
          !cuda_ok(h, cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime")) {
        if (!r) r = SPARC_ERR_CUDA;
        break;
      }
      tot += ms;
      ++timed;
    }
    if (r) break;
    if (tot < best_ms) {
      best_ms = tot;
      bz = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (r) return r;
  if (set_zchunk(h, bz)) return fail(h, SPARC_ERR_INVALID, "z chunk out of range");
  if (next) *next = nn;
  if (best) *best = bz;
  return SPARC_OK;
}

int sparc_diagnostics(sparc_handle *h, sparc_diag *out) {
  if (!h || !out) return SPARC_ERR_INVALID;
  cudaSetDevice(h->device);
  double d[4];
  long long f;
  int e = 0;
  // in a batch, the batch stream orders the writes of these values
  cudaStream_t st = h->batch ? h->batch_stream : h->stream;
  CK(h, cudaMemcpyAsync(d, h->d_diag, 32, cudaMemcpyDeviceToHost, st));
  CK(h, cudaMemcpyAsync(&f, h->d_fail, 8, cudaMemcpyDeviceToHost, st));
  CK(h, cudaMemcpyAsync(&e, h->d_err, 4, cudaMemcpyDeviceToHost, st));
  CK(h, cudaStreamSynchronize(st));
  if (e) return fail(h, SPARC_ERR_TIMEOUT, "a bounded device wait gave up");
  out->ke_norm = d[0];
  out->min_rho = d[1];
  out->min_p = d[2];
  out->iteration = (int64_t)d[3];
  out->fail_iteration = f;
  return f >= 0 ? SPARC_ERR_UNSTABLE : SPARC_OK;
}

int sparc_synchronize(sparc_handle *h) {
  if (!h) return SPARC_ERR_INVALID;
  cudaSetDevice(h->device);
  CK(h, cudaStreamSynchronize(h->stream));
  return SPARC_OK;
}

int sparc_stream(sparc_handle *h, void **stream) {
  if (!h || !stream) return SPARC_ERR_INVALID;
  *stream = (void *)h->stream;
  return SPARC_OK;
}

int sparc_launch_count(const sparc_handle *h, int64_t *count) {
  if (!h || !count) return SPARC_ERR_INVALID;
  *count = h->launches;
  return SPARC_OK;
}

int sparc_derivative(sparc_handle *h, int dir, int bc, const double *in,
                     double *out) {
  if (!h || !in || !out || dir < 0 || dir > 2 || (bc != 1 && bc != 5))
    return SPARC_ERR_INVALID;
  if (h->fp32) return fail(h, SPARC_ERR_INVALID, "unit entry points need the FP64 form");
  if (!h->bg_ready) return fail(h, SPARC_ERR_ORDER, "set the background first");
  cudaSetDevice(h->device);
  double *dev_in = h->buf[h->rf1], *dev_out = h->buf[h->rf2];
  CK(h, cudaMemcpyAsync(dev_in, in, h->N * 8, cudaMemcpyHostToDevice, h->stream));
  int r = launch_derivative(h, dir, bc, dev_in, dev_out, h->stream);
  if (r) return r;
  CK(h, cudaMemcpyAsync(out, dev_out, h->N * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return SPARC_OK;
}

int sparc_filter_field(sparc_handle *h, int dir, const double *in, double *out) {
  if (!h || !in || !out || dir < 0 || dir > 2) return SPARC_ERR_INVALID;
  if (h->fp32) return fail(h, SPARC_ERR_INVALID, "unit entry points need the FP64 form");
  cudaSetDevice(h->device);
  double *dev_in = h->buf[h->rf1], *dev_out = h->buf[h->rf2];
  CK(h, cudaMemcpyAsync(dev_in, in, h->N * 8, cudaMemcpyHostToDevice, h->stream));
  int r = launch_filter_raw(h, dir, dev_in, dev_out, h->stream);
  if (r) return r;
  CK(h, cudaMemcpyAsync(out, dev_out, h->N * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return SPARC_OK;
}

int sparc_get_coeff(sparc_handle *h, const char *name, double *out,
                    int64_t *count) {
  if (!h || !name || !count) return SPARC_ERR_INVALID;
  if (!h->bg_ready) return fail(h, SPARC_ERR_ORDER, "set the background first");
  cudaSetDevice(h->device);
  std::string s(name);
  if (h->fp32 && s != "stretch" && s != "zaxis" && s != "xaxis" && s != "yaxis" && s != "g" &&
      s != "gblk" && s != "invrho0q" && s != "cq")
    return fail(h, SPARC_ERR_INVALID, "FP64 coefficients are released in the precision form");
  const double *dsrc = nullptr;
  const std::vector<double> *hsrc = nullptr;
  long long n = h->N;
  if (s == "rho0") dsrc = h->rho0;
  else if (s == "p0") dsrc = h->p0;
  else if (s == "c2") dsrc = h->c2;
  else if (s == "rhoinv") dsrc = h->rhoinv;
  else if (s == "c2rho0") dsrc = h->c2rho0;
  else if (s == "gradrho0_z") dsrc = h->grz;
  else if (s == "gradp0_z") dsrc = h->gpz;
  else if (s == "gradrho0_x") dsrc = h->grx;
  else if (s == "gradrho0_y") dsrc = h->gry;
  else if (s == "gradp0_x") dsrc = h->gpx;
  else if (s == "gradp0_y") dsrc = h->gpy;
  else if (s == "spongexyz") dsrc = h->sponge;
  else if (s == "box") dsrc = h->box;
  else if (s == "boy") dsrc = h->boy;
  else if (s == "boz") dsrc = h->boz;
  else if (s == "curlbox") dsrc = h->cbx;
  else if (s == "curlboy") dsrc = h->cby;
  else if (s == "curlboz") dsrc = h->cbz;
  else if (s == "reduction") dsrc = h->red;
  else if (s == "source_damp") dsrc = h->source_damp;
  else if (s == "src_scale_beta") dsrc = h->ssb;
  else if (s == "stretch") hsrc = &h->stretch;
  else if (s == "zaxis") hsrc = &h->zaxis;
  else if (s == "xaxis") hsrc = &h->xaxis;
  else if (s == "yaxis") hsrc = &h->yaxis;
  else if (s == "g") hsrc = &h->g;
  else if (s == "gblk") hsrc = &h->g_blk;
  else if (s == "invrho0q") hsrc = &h->invrho0q;
  else if (s == "cq") hsrc = &h->cq;
  else {
    static const char *fn[6] = {"z_bot", "z_top", "x_bot", "x_top", "y_bot", "y_top"};
    for (int f = 0; f < 6 && !dsrc; ++f) {
      const FaceDev &F = h->faces[f];
      const double *arr = nullptr;
      if (s == std::string("a_") + fn[f]) arr = F.pa;
      else if (s == std::string("b_") + fn[f]) arr = F.pb;
      else if (s == std::string("kappa_") + fn[f]) arr = F.pk;
      else continue;
      if (!F.on) return fail(h, SPARC_ERR_INVALID, "face not in use");
      *count = F.cnt;
      if (!out) return SPARC_OK;
      if (F.uniform) {  // layer profile: expand to the face layout
        std::vector<double> lay(F.np);
        CK(h, cudaMemcpy(lay.data(), arr, F.np * 8, cudaMemcpyDeviceToHost));
        const long long per = (long long)F.n0 * F.n1;
        for (long long t = 0; t < F.cnt; ++t) out[t] = lay[t / per];
      } else {
        CK(h, cudaMemcpy(out, arr, F.cnt * 8, cudaMemcpyDeviceToHost));
      }
      return SPARC_OK;
    }
    if (!dsrc) return fail(h, SPARC_ERR_INVALID, "unknown coefficient " + s);
  }
  if (hsrc) {
    *count = (int64_t)hsrc->size();
    if (out) std::memcpy(out, hsrc->data(), hsrc->size() * 8);
    return SPARC_OK;
  }
  if (!dsrc) return fail(h, SPARC_ERR_INVALID, "coefficient not used in this mode");
  *count = n;
  if (out) CK(h, cudaMemcpy(out, dsrc, n * 8, cudaMemcpyDeviceToHost));
  return SPARC_OK;
}

int sparc_get_scalars(sparc_handle *h, double *o) {
  if (!h || !o) return SPARC_ERR_INVALID;
  double s[12] = {h->dimc, h->dimrho, h->diml, h->dimb, h->deltat, h->stretchx,
                  h->stretchy, h->betas[0], h->betas[1], h->betas[2], h->betas[3],
                  h->betas[4]};
  std::memcpy(o, s, sizeof(s));
  return SPARC_OK;
}

const char *sparc_last_error(const sparc_handle *h) {
  return h ? h->err.c_str() : g_create_error.c_str();
}

}  // extern "C"
