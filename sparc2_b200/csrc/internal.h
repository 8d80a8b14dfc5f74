// internal.h -- device-side data layout shared by the translation units of
// libsparc_gpu.so (setup.cu, step.cu, api.cu).  Host C++ only; kernels get
// the POD structs below by value.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/sparc_gpu.h"

namespace sparc {

constexpr double RSUN = 69598946770.0;   // all_modules.f90:56
constexpr double PI = 3.14159265358979;  // all_modules.f90:56 (truncated pi)

// One CPML face on the device.  Auxiliary fields are stored in the
// reference's layout (n0 fastest, P slots); profiles a, b, kappa are either
// per point of the slab or, when `uniform`, one value per PML layer.
// R is the storage type: double (plain form) or float (precision form).
template <class R>
struct FaceT {
  int on;
  int n0, n1, n2, np, P;
  int uniform;          // profiles depend on the layer index only
  long long cnt;        // n0*n1*n2
  R *vars;              // RK state (zpmlvars...), cnt*P
  R *scr;               // stage right-hand side (scrzpml...), cnt*P
  const R *pa, *pb, *pk;
  const R *pki;         // 1/kappa (precision form)
};
using FaceDev = FaceT<double>;

// Forcing description consumed by the stage kernels.
template <class R>
struct ForcingT {
  int kind;             // SPARC_SRC_*
  int dir;              // 1..3
  long long init;
  // PULSE = 1: f = T(t) * fz[k] * fy[j] * fx[i], T on the device
  const R *fx, *fy, *fz;
  double amp_c, t0, t1, st, timestep;  // amp_c = pulse_amp/0.56458272/dimc
  // PULSE = 2: precomputed per iteration for layers [klo, khi)
  const R *psr;          // (khi-klo)*nx*ny
  int klo, khi;
  // PULSE = 0: f = f2d[j*nx + i] * sdep[k], f2d rebuilt per iteration
  const R *f2d, *sdep;
};
using ForcingDev = ForcingT<double>;

// Everything the fused stage kernels read.  Background arrays are either
// 3-D (N) or, for the horizontally uniform quiet background, 1-D (nz).
// In the precision form (R = float) the state is stored scaled by depth
// profiles: stored = sc[l*nz + k] * physical (isc = 1/sc), and the final
// RK update carries a compensated-sum term per state value.
template <class R>
struct SimT {
  int nx, ny, nz;
  long long N;
  int periodic, magnetic, bg1d;
  int sponge_slabs;            // the sponge vanishes outside the CPML slabs
  int V;
  double stretchx, stretchy;
  const R *stretch;            // nz
  double deltat;
  double dimc2rho;             // dimc^2*dimrho for the KE norm
  // background (code units)
  const R *rho0, *p0, *rhoinv, *c2rho0, *grz, *gpz, *sponge;
  const R *box, *boy, *boz, *cbx, *cby, *cbz;
  const R *grx, *gry, *gpx, *gpy, *red;
  const R *gblk;               // (block_x*block_y) * nz gravity
  const int *colx, *coly;      // block index of each x / y
  int bxdim;
  FaceT<R> zb, zt, xb, xt, yb, yt;
  ForcingT<R> frc;
  const R *sc, *isc;           // V x nz depth scales (precision form)
  R *carry;                    // V x N compensated-sum carry (precision form)
  const R *term;               // 3 x N velocity damping terms (DAMPING), or null
  // iteration bookkeeping and diagnostics (device)
  long long *iter;             // current driver iteration
  int *err;                    // device error flag (bounded waits)
  double *partials;            // 3 per block of the last stage
  unsigned int *counter;
  double *diag;                // ke, min_rho, min_p, iteration(double)
  long long *fail_iter;
};
using SimDev = SimT<double>;

// z chunk boundaries of a persistent stage launch: chunk c covers layers
// [b[c], b[c+1])
struct ZSched {
  static constexpr int MAX = 32;
  int n;
  int b[MAX + 1];
};

// PULSE = 2 forcing of the precision form: the per-layer pulse lists and
// separable factors the forcing kernels read (all_modules.f90:521-663).
struct Psr32 {
  int nx, ny, klo, khi, nblocks, bx, bxy;
  long long init;
  double timestep, st;
  const int *off, *idx, *colx, *coly, *colz;
  const double *zv, *ptime;
  const float *px, *py, *sd, *ssb;
  const unsigned char *mask;
  float *out;
  const long long *iter;
};

// PULSE = 0 forcing of a batch member: the series, source_damp(:,:,1) and
// the member's forcing plane, rebuilt at the start of each batched step.
struct Rnd32 {
  const double *series;        // nxy * ns, times randomexciteampl / dimc
  const float *damp;           // nxy
  float *out;                  // nxy (the plane the stage kernels read)
  int nxy, ns;
  double timestep, cad;
};

// One simulation of a batch, as the batched kernels read it.  Buffer roles,
// the steps left and the completion counter live here and are advanced on
// the device, so a captured step stays valid while simulations come and go.
struct Slot32 {
  SimT<float> S;
  Psr32 psr;
  float *buf[3];
  int role[3];                 // a, free1, free2
  double betas[5];
  long long remaining;         // driver iterations left
  int active;                  // set at the start of each step
  int has_psr;
  int has_rnd;
  Rnd32 rnd;
  int first_item, n_items;     // stage items of the interior part (MHD only)
  int first_item2, n_items2;   // stage items of the general part
  int f_first, f_items;        // carry-clear work-list range
  int xy_items;                // xy-pass items (field, 8-layer group, 32x32 tile)
  int z_items;                 // z-pass items (field, 32x4 column slab, 32-layer chunk)
  int gxy, gz, xyfreq, zfreq;
  float s_xy, s_z;
  unsigned counter;            // items done in the current launch
  double *partials;            // 3 per stage item of the work-list (last stage)
};

// Device work-lists and launch shape of one batched step.
struct BatchLaunch {
  Slot32 *slots;
  int nslots;
  const int4 *items, *fitems, *pitems;  // stage, filter, forcing items
  const int4 *xyitems, *zitems;         // xy- and z-pass filter items
  const int *counts;                    // [6] stage, carry-clear, forcing
                                        // items, interior stage items (a
                                        // prefix), z-pass, xy-pass items
  unsigned *wctr;                       // [14] work counters, zeroed per step
  int grid;                             // persistent CTAs
  int zmax;                             // largest z extent of a stage item
  size_t psr_smem;
};

// Background arrays of the precision form (FP32 copies of the FP64 setup).
enum {
  FB_RHO0, FB_P0, FB_RHOINV, FB_C2R, FB_GRZ, FB_GPZ, FB_SPONGE, FB_BOX, FB_BOY,
  FB_BOZ, FB_CBX, FB_CBY, FB_CBZ, FB_GRX, FB_GRY, FB_GPX, FB_GPY, FB_RED, FB_COUNT
};

struct Handle {
  sparc_params P{};
  int device = 0;
  int nx = 0, ny = 0, nz = 0, V = 0, Pp = 0;
  long long N = 0;
  bool magnetic = false, quiet = false, periodic = false;
  bool use_pml = false, use_hpml = false;
  int gxy = 5, gz = 5, xyfreq = 1, zfreq = 1;
  bool bg_ready = false;
  cudaStream_t stream = nullptr;
  // MHD stages: the edge/CPML launch runs on `aux`, forked from and joined
  // back to `stream` by the two events, beside the interior launch
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  std::string err;
  long long launches = 0;

  // host-side 1-D setup
  std::vector<double> xaxis, yaxis, zaxis, g, stretch, cq, invrho0q;
  std::vector<int> colx, coly, bxs, bys, bzs, bxl, byl, bzl;
  double stretchx = 0, stretchy = 0, dimc = 0, dimrho = 0, diml = 0,
         dimb = 0, deltat = 0, betas[5] = {0, 0, 0, 0, 0};

  // device memory (all owned)
  std::vector<void *> allocs;
  double *buf[3] = {nullptr, nullptr, nullptr};  // rotating state buffers
  int ra = 0, rf1 = 1, rf2 = 2;                  // roles: a, free1, free2
  // 3-D FP64 setup arrays (code units)
  double *rho0 = nullptr, *p0 = nullptr, *c2 = nullptr, *rhoinv = nullptr,
         *c2rho0 = nullptr, *grz = nullptr, *gpz = nullptr, *sponge = nullptr,
         *box = nullptr, *boy = nullptr, *boz = nullptr, *cbx = nullptr,
         *cby = nullptr, *cbz = nullptr, *grx = nullptr, *gry = nullptr,
         *gpx = nullptr, *gpy = nullptr, *red = nullptr,
         *source_damp = nullptr, *ssb = nullptr;
  // 1-D profiles for the uniform quiet background
  double *rho0_1 = nullptr, *p0_1 = nullptr, *rhoinv_1 = nullptr,
         *c2rho0_1 = nullptr, *grz_1 = nullptr, *gpz_1 = nullptr,
         *sponge_1 = nullptr;
  double *d_stretch = nullptr, *d_gblk = nullptr;
  int *d_colx = nullptr, *d_coly = nullptr;
  FaceDev faces[6]{};  // z_bot, z_top, x_bot, x_top, y_bot, y_top
  std::vector<double> g_blk;  // host copy of the gravity table
  bool bg1d = false;
  // the sponge is zero outside the CPML slabs (the base sponges of
  // initialize.f90:899-947 all vanish): stage kernels skip its loads there
  bool sponge_slabs = false;

  // DAMPING (damping.cu): cuFFT plans over the nz layers, the rates of the
  // half spectrum, the spectrum and the three velocity terms
  bool damping = false, fft_plans = false;
  int fft_fwd = 0, fft_inv = 0;  // cufftHandle
  double *d_damp = nullptr, *d_term = nullptr;
  double2 *d_spec = nullptr;

  // forcing
  sparc_source src{};
  std::vector<sparc_pulse> pulses;
  double *d_fx = nullptr, *d_fy = nullptr, *d_fz = nullptr;
  double *d_psr = nullptr;          // forcing buffer for PULSE = 2
  int psr_klo = 0, psr_khi = 0;
  // PULSE = 2 tables
  double *d_px = nullptr, *d_py = nullptr;  // npulses*nx, npulses*ny
  int *d_plane_off = nullptr, *d_plane_idx = nullptr;
  double *d_plane_z = nullptr;              // Z_n(k) per CSR entry
  unsigned char *d_pmask = nullptr;         // npulses * nblocks
  double *d_ptime = nullptr;                // amp, t0, t1 per pulse
  // PULSE = 0: the scaled forcing series (nx*ny*nseries), source_dep and
  // the per-iteration forcing plane
  double *d_series = nullptr, *d_sdep = nullptr, *d_f2d = nullptr;
  float *f_f2d = nullptr, *f_sdep = nullptr;
  int nblocks = 1;

  // TMA tensor maps (32x8x1 boxes) of the MHD own-point arrays: [0..2] the
  // state buffers (nx, ny, nz*V), [3..17] the background arrays per layer
  bool tma = false;
  CUtensorMap tmaps_ty[24];
  // FILTER_VARS xy pass (non-periodic FP64 grids, nx even): the state
  // buffers in 44x44x1 boxes
  bool ftma = false;
  CUtensorMap fmaps[3];
  // FILTER_VARS z pass (FP64, nx even): the state buffers as (nx, ny, nz, V)
  // in 32x4x44x1 boxes
  bool ztma = false;
  CUtensorMap zmaps[3];
  // device bookkeeping
  int *d_err = nullptr;
  long long *d_iter = nullptr, *d_fail = nullptr;
  double *d_partials = nullptr, *d_diag = nullptr;
  unsigned int *d_counter = nullptr;
  int max_stage_blocks = 0;
  // FP64 MHD stages as one persistent launch (step.cu:mhd64_plan): the
  // edge/CPML tiles (tile coordinates), the interior rectangle, a work
  // counter per stage, CTAs per launch
  int2 *d_gen = nullptr;
  int ngen = 0, gix0 = 0, giy0 = 0, gnix = 0, gniy = 0, pgrid = 0;
  unsigned *d_wctr64 = nullptr;
  int partials_blocks = 0;  // blocks the partials hold: any z chunk >= 11

  // stage launch geometry (quiet tiles tx x ty; MHD tiles 32 x 8)
  int tx = 32, ty = 8, zchunk = 32;

  // precision form (SPARC_FP32): FP32 state in fbuf (roles ra/rf1/rf2 as
  // for buf), the compensated-sum carry of the state, depth scales
  // (stored = f_sc[l*nz+k] * physical), FP32 background and CPML faces.
  // The FP64 setup arrays are released once converted.
  bool fp32 = false;
  float *fbuf[3] = {nullptr, nullptr, nullptr};
  float *f_carry = nullptr;
  float *f_sc = nullptr, *f_isc = nullptr;  // V x nz
  std::vector<float> h_scale;               // host copy: sc then isc
  float *f_bg[FB_COUNT] = {};
  float *f_stretch = nullptr, *f_gblk = nullptr;
  FaceT<float> f_faces[6]{};
  float *f_fx = nullptr, *f_fy = nullptr, *f_fz = nullptr;
  float *f_psr = nullptr, *f_px = nullptr, *f_py = nullptr;
  float *f_sd = nullptr, *f_ssb = nullptr;
  bool tma32 = false;
  bool allow_tma32 = true;   // FP32 MHD own-point loads by TMA (nx % 4 == 0)
  bool allow_tma64 = true;   // FP64 MHD own-point loads by TMA (nx even)
  CUtensorMap tmaps32[18];

  // member of a batch (sparc_batch_add): the batch owns the buffer roles,
  // the iteration and the stream order until sparc_batch_remove
  void *batch = nullptr;
  cudaStream_t batch_stream = nullptr;

  // captured graphs keyed by (ra, rf1, rf2, filter kind)
  struct GraphEntry {
    int ra, rf1, rf2, fk;
    cudaGraphExec_t exec;
    int nkernels;
    int out_ra, out_rf1, out_rf2;  // buffer roles after the captured iteration
  };
  std::vector<GraphEntry> graphs;
};

// setup.cu: published coefficient tables (initialize.f90:1929-2031)
extern const double kDerivRows[6][11];
extern const double kFilter11[11];
extern const double kFilter7[7];
int setup_background(Handle *h, const double *rho0, const double *pre0,
                     const double *cs0, const double *bx0, const double *by0,
                     const double *bz0, const double *zaxis_mm,
                     const double *grav);
int setup_constants();
int launch_derivative(Handle *h, int dir, int bc, const double *in,
                      double *out, cudaStream_t s);
int launch_filter_raw(Handle *h, int dir, const double *in, double *out,
                      cudaStream_t s);

// step.cu
int step_constants();
int filter_constants();
SimDev make_simdev(Handle *h);
int launch_stage(Handle *h, const SimDev &S, int stage, const double *a,
                 const double *tin, double *tout, cudaStream_t s);
int launch_psr_forcing(Handle *h, const SimDev &S, cudaStream_t s);
int launch_random_forcing(Handle *h, cudaStream_t s);
int launch_filter_event(Handle *h, bool xy, const double *in, double *out, cudaStream_t s);
int stage_geometry(Handle *h);
int encode_tensor_maps(Handle *h);

// step32.cu (precision form)
int step32_constants();
SimT<float> make_sim32(Handle *h);
int launch_stage32(Handle *h, const SimT<float> &S, int stage, const float *a,
                   const float *tin, float *so, cudaStream_t s);
int launch_psr32(Handle *h, cudaStream_t s);
Psr32 make_psr32(Handle *h);
int launch_batch_step(const BatchLaunch &B, cudaStream_t s, int *nkernels);
size_t batch_stage_smem();
int launch_filter_event32(Handle *h, bool xy, const float *in, const float *carry, float *out,
                          cudaStream_t s);
int encode_tensor_maps32(Handle *h);
int setup32(Handle *h);
int damping_setup(Handle *h);
int mhd64_plan(Handle *h);
int damping_enqueue(Handle *h, const double *tin, cudaStream_t s);
void damping_destroy(Handle *h);
int source32(Handle *h);

// batch.cu: the device slot of batch member h (null while the slot table
// holding it has not been uploaded)
int batch_member_slot(const Handle *h, const Slot32 **dslot);

// api.cu
void *dev_alloc(Handle *h, size_t bytes);
void dev_free(Handle *h, const void *p);
bool cuda_ok(Handle *h, cudaError_t e, const char *what);

}  // namespace sparc
