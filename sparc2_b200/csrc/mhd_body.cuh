// mhd_body.cuh -- the fused MP_MHD_3D stage body (RHS.f90:363-668 with the
// CPML of RHS.f90:424-546 and one RK stage of step.f90:26-61), shared by the
// plain form (R = double, step.cu) and the precision form (R = float,
// step32.cu, with depth-scaled state and a compensated final update).
//
// Two roles per column (threadIdx.z): role 0 computes the momentum
// equations (z windows vz, p, bx), role 1 continuity, pressure and
// induction (z windows flux1, flux2, by); d(vz)/dz and d(by)/dz cross over
// through shared memory.  A CTA owns a 32x8 column tile and marches a chunk
// of z layers; the layer's halo planes and own-point arrays are copied into
// a double-buffered shared tile one layer ahead.
//
// Each translation unit that includes this header defines
// dcoef<R>(row, m): its constant table of the derivative rows
// (initialize.f90:1959-2031).
#pragma once

#include "internal.h"
#include "tma_util.cuh"
#include "tmem_window.cuh"

namespace sparc {

enum { F_FIRST = 0, F_MID = 1, F_LAST = 2 };

template <class R>
__device__ __forceinline__ R dcoef(int r, int m);

// geometry of the MHD stage tile (precision independent)
namespace mg {
constexpr int TX = 32, TY = 8, NC = TX * TY, NT = 2 * NC;
constexpr int HX = TX + 10, HY = TY + 10, HS = HX * HY;
constexpr int NH = 10, NO = 24;
constexpr long long WAIT_LIMIT = kMbarWaitLimit;
// own-point slots: stage rho, a[0..7], 14 background arrays, p0
constexpr int O_RHO = 0, O_A = 1, O_BG = 9, O_P0 = 23;
enum { B_RED, B_SPONGE, B_RHO0, B_GRX, B_GRY, B_GRZ, B_C2R, B_GPX, B_GPY,
       B_GPZ, B_RHOINV, B_CBX, B_CBY, B_CBZ };
}  // namespace mg

// shared-memory buffers of one layer (in R words, 128-byte multiple), the
// exchange area and the dynamic size.  TH: the halo planes arrive as TMA
// boxes (interior tiles of the plain form): a plane is 44 x 18 starting at
// x0 - 6 (a 16-byte aligned start), each plane 128-byte aligned; otherwise
// 42 x 18 copied by cp.async.  Exchange area:
// d(vz)/dz and d(by)/dz in R, |v_new|^2 in FP64 (in the d(by)/dz slot in
// the plain form, after its reader).
template <class R, bool TH = false, bool HV = false>
struct MhdBuf {
  static constexpr int ALIGN = 128 / (int)sizeof(R);
  static_assert(!TH || sizeof(R) == 8, "TMA halo boxes in the plain form only");
  static_assert(!HV || sizeof(R) == 4, "16-byte halo vectors in the precision form only");
  // HV: halo rows of 48 values from x0 - 8 (a 16-byte aligned start), copied
  // as 4-value vectors
  static constexpr int HXL = TH ? 44 : (HV ? 48 : mg::HX);
  static constexpr int XOFF = TH ? 1 : (HV ? 3 : 0);
  static constexpr int HSL =
      (TH || HV) ? (HXL * mg::HY + ALIGN - 1) / ALIGN * ALIGN : mg::HS;
  static constexpr int BUF = ((mg::NO * mg::NC + mg::NH * HSL) + ALIGN - 1) / ALIGN * ALIGN;
  static constexpr int XCH = sizeof(R) == 4 ? 4 * mg::NC : 2 * mg::NC;
  static constexpr size_t SMEM = (2 * (size_t)BUF + XCH) * sizeof(R) + 128;
  // plain form, general tiles: the per-lane and per-row coefficient tables
  // follow the exchange area (dynamic, so one kernel can hold both bodies)
  static constexpr size_t TABLES =
      (size_t)(mg::TX + mg::TY) * 11 * sizeof(R) + (mg::TX + mg::TY) * sizeof(int);
  static constexpr size_t SMEM_GEN = SMEM + (sizeof(R) == 8 ? TABLES : 0);
  // precision form: the depth scales (8 inverse, 8 forward per layer) of a
  // chunk of at most zext layers follow the exchange area
  static constexpr size_t smem_bytes(int zext) {
    return SMEM + (sizeof(R) == 4 ? (size_t)(zext + 16) * 16 * sizeof(R) : 0);
  }
};

// tensor maps: [0..2] the state buffers (nx, ny, nz*V) and [3..17] the
// background arrays in 32x8x1 boxes (own points); plain form: [18..20] the
// state buffers and [21..23] B0 x, y, z in 44x18x1 halo boxes
struct TmaSet {
  CUtensorMap m[24];
};

template <class R>
__device__ __forceinline__ void cp_r(R *dst, const R *src) {
  if constexpr (sizeof(R) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sm_addr_t(dst)), "l"(src)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sm_addr_t(dst)), "l"(src)
                 : "memory");
}
// one 16-byte cp.async (both addresses 16-byte aligned)
template <class R>
__device__ __forceinline__ void cp16_t(R *dst, const R *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sm_addr_t(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_commit_t() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// brings the line holding p into L2 (no register, no wait)
__device__ __forceinline__ void pf_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
// brings the line holding p into L1
__device__ __forceinline__ void pf_l1(const void *p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// named barrier of two warps (64 threads)
__device__ __forceinline__ void bar_pair_t(int id) {
  asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory");
}

__device__ __forceinline__ int wrap_t(int q, int n) {
  q = q < 0 ? q + n : q;
  return q >= n ? q - n : q;
}
// first halo column/row of a tile; on a non-periodic axis the last tile
// moves down so that the one-sided window f(n-11..n-1) lies in the tile
__device__ __forceinline__ int origin_t(int t0, int T, int n, bool per) {
  int o = t0 - 5;
  if (!per && t0 + T >= n) o = min(o, n - 11);
  return o;
}

template <class R>
__device__ __forceinline__ void shift_t(R (&w)[11], R v) {
#pragma unroll
  for (int m = 0; m < 10; ++m) w[m] = w[m + 1];
  w[10] = v;
}

// Centred 11-point sum at p[5*st]: the centred row is antisymmetric
// (c[5+m] = -c[5-m], c[5] = 0), so it is sum_m c[5+m] (f[+m] - f[-m]),
// evaluated as two short independent chains.
template <class R>
__device__ __forceinline__ R csum_t(const R *p, int st) {
  const R d1 = p[6 * st] - p[4 * st], d2 = p[7 * st] - p[3 * st], d3 = p[8 * st] - p[2 * st],
          d4 = p[9 * st] - p[st], d5 = p[10 * st] - p[0];
  const R a = dcoef<R>(5, 8) * d3 + (dcoef<R>(5, 10) * d5 + dcoef<R>(5, 6) * d1);
  const R b = dcoef<R>(5, 9) * d4 + dcoef<R>(5, 7) * d2;
  return a + b;
}

// ddz on the register window w = f(k-5..k+5) (derivatives.f90:451-562): the
// centred stencil (zero ghosts below the bottom), one-sided rows in the top
// five layers on the frozen window f(nz-11..nz-1)
template <class R>
__device__ __forceinline__ R dz_t(const R (&w)[11], int k, int nz, R sc) {
  if (k < nz - 5) {
    const R d1 = w[6] - w[4], d2 = w[7] - w[3], d3 = w[8] - w[2], d4 = w[9] - w[1],
            d5 = w[10] - w[0];
    const R a = dcoef<R>(5, 8) * d3 + (dcoef<R>(5, 10) * d5 + dcoef<R>(5, 6) * d1);
    const R b = dcoef<R>(5, 9) * d4 + dcoef<R>(5, 7) * d2;
    return sc * (a + b);
  }
  const int row = nz - 1 - k;
  R s = R(0);
#pragma unroll
  for (int m = 0; m < 11; ++m) s += w[10 - m] * dcoef<R>(row, m);
  return -sc * s;
}

// The z derivative of a window held as a ring: slot (RR + m) % 11 holds
// logical value m (layer L + m); with sh the new head h replaces logical
// value 10 (its slot still holds the layer it overwrites).  RR is a
// template parameter, so the rotation is a renaming of registers.
template <int RR, class R>
__device__ __forceinline__ R dz_rot(const R (&v)[11], R h, bool sh, int k, int nz, R sc) {
  R w[11];
#pragma unroll
  for (int m = 0; m < 11; ++m) w[m] = v[(RR + m) % 11];
  if (sh) w[10] = h;
  return dz_t(w, k, nz, sc);
}
template <class R>
__device__ __forceinline__ R dz_ring(const R (&v)[11], R h, bool sh, int rr, int k, int nz,
                                     R sc) {
  switch (rr) {
    case 0: return dz_rot<0>(v, h, sh, k, nz, sc);
    case 1: return dz_rot<1>(v, h, sh, k, nz, sc);
    case 2: return dz_rot<2>(v, h, sh, k, nz, sc);
    case 3: return dz_rot<3>(v, h, sh, k, nz, sc);
    case 4: return dz_rot<4>(v, h, sh, k, nz, sc);
    case 5: return dz_rot<5>(v, h, sh, k, nz, sc);
    case 6: return dz_rot<6>(v, h, sh, k, nz, sc);
    case 7: return dz_rot<7>(v, h, sh, k, nz, sc);
    case 8: return dz_rot<8>(v, h, sh, k, nz, sc);
    case 9: return dz_rot<9>(v, h, sh, k, nz, sc);
    default: return dz_rot<10>(v, h, sh, k, nz, sc);
  }
}

// Compensated (Kahan) update a + inc with the running carry c.
__device__ __forceinline__ float kahan(float a, float inc, float &c) {
  const float y = inc - c;
  const float t = a + y;
  c = (t - a) - y;
  return t;
}

// Three CPML fields of one face at one point (RHS.f90:50-93, 424-546:
// RHSpsi = a d + b psi, then d = d/kappa + psi with the stored 1/kappa).
// Every load is issued before any store, and the profile once.
template <class R, int MODE>
__device__ __forceinline__ void cpml3_t(const FaceT<R> &F, long long f, int layer, int s0, int s1,
                                        int s2, R beta, R dt, R &d0, R &d1, R &d2) {
  const long long pf = F.uniform ? (long long)layer : f;
  const R pa = __ldg(F.pa + pf), pb = __ldg(F.pb + pf), pki = __ldg(F.pki + pf);
  const long long o0 = (long long)s0 * F.cnt + f, o1 = (long long)s1 * F.cnt + f,
                  o2 = (long long)s2 * F.cnt + f;
  const R v0 = F.vars[o0], v1 = F.vars[o1], v2 = F.vars[o2];
  R p0 = v0, p1 = v1, p2 = v2;
  if (MODE != F_FIRST) {
    const R c0 = F.scr[o0], c1 = F.scr[o1], c2 = F.scr[o2];
    p0 = v0 + beta * c0;
    p1 = v1 + beta * c1;
    p2 = v2 + beta * c2;
  }
  const R r0 = pa * d0 + pb * p0, r1 = pa * d1 + pb * p1, r2 = pa * d2 + pb * p2;
  d0 = d0 * pki + p0;
  d1 = d1 * pki + p1;
  d2 = d2 * pki + p2;
  if (MODE == F_LAST) {
    F.vars[o0] = v0 + dt * r0;
    F.vars[o1] = v1 + dt * r1;
    F.vars[o2] = v2 + dt * r2;
  } else {
    F.scr[o0] = r0;
    F.scr[o1] = r1;
    F.scr[o2] = r2;
  }
}

// PULSE = 1 time factor (driver.f90:140-145), FP64, at iteration it
template <class R>
__device__ __forceinline__ R pulse_time_t(const SimT<R> &S, long long it) {
  const ForcingT<R> &F = S.frc;
  if (F.kind != SPARC_SRC_PULSE) return R(0);
  const double t = (double)it * F.timestep;
  double T = F.amp_c * sin(2.0 * PI * (t - F.t1 + 2.0 * F.t0) / F.t0);
  return (R)(T * exp(-1.0 * ((t - F.t1) * (t - F.t1)) / (2.0 * (F.st * F.st))));
}

// forcing of driver.f90:137-153 at point (i, j, k)
template <class R>
__device__ __forceinline__ R forcing_t(const SimT<R> &S, R T, int i, int j, int k) {
  const ForcingT<R> &F = S.frc;
  if (F.kind == SPARC_SRC_PULSE) return T * __ldg(F.fz + k) * (__ldg(F.fy + j) * __ldg(F.fx + i));
  if (F.kind == SPARC_SRC_PSR && k >= F.klo && k < F.khi)
    return F.psr[((long long)(k - F.klo) * S.ny + j) * S.nx + i];
  if (F.kind == SPARC_SRC_RANDOM) return F.f2d[(long long)j * S.nx + i] * __ldg(F.sdep + k);
  return R(0);
}

// Block partial of the KE norm and minima (FP64); the last block of the
// logical grid (bid/nb: a stage split over several launches shares one) to
// finish reduces all partials and applies the fail criterion of
// driver.f90:175-183, then advances the device iteration.
template <class R>
__device__ void diag_reduce_t(const SimT<R> &S, double ke, double mr, double mp, long long bid,
                              long long nb) {
  __shared__ double r[3][32];
  __shared__ int am_last;
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const int tid = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5, nw = (nt + 31) >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    ke += __shfl_down_sync(0xffffffffu, ke, o);
    mr = fmin(mr, __shfl_down_sync(0xffffffffu, mr, o));
    mp = fmin(mp, __shfl_down_sync(0xffffffffu, mp, o));
  }
  if (lane == 0) { r[0][warp] = ke; r[1][warp] = mr; r[2][warp] = mp; }
  __syncthreads();
  if (warp == 0) {
    ke = lane < nw ? r[0][lane] : 0.0;
    mr = lane < nw ? r[1][lane] : 1e300;
    mp = lane < nw ? r[2][lane] : 1e300;
    for (int o = 16; o > 0; o >>= 1) {
      ke += __shfl_down_sync(0xffffffffu, ke, o);
      mr = fmin(mr, __shfl_down_sync(0xffffffffu, mr, o));
      mp = fmin(mp, __shfl_down_sync(0xffffffffu, mp, o));
    }
    if (lane == 0) {
      S.partials[3 * bid] = ke;
      S.partials[3 * bid + 1] = mr;
      S.partials[3 * bid + 2] = mp;
      __threadfence();
      unsigned t = atomicAdd(S.counter, 1u);
      am_last = (t == (unsigned)(nb - 1));
    }
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  ke = 0.0; mr = 1e300; mp = 1e300;
  for (long long b = tid; b < nb; b += nt) {
    ke += __ldcg(S.partials + 3 * b);
    mr = fmin(mr, __ldcg(S.partials + 3 * b + 1));
    mp = fmin(mp, __ldcg(S.partials + 3 * b + 2));
  }
  for (int o = 16; o > 0; o >>= 1) {
    ke += __shfl_down_sync(0xffffffffu, ke, o);
    mr = fmin(mr, __shfl_down_sync(0xffffffffu, mr, o));
    mp = fmin(mp, __shfl_down_sync(0xffffffffu, mp, o));
  }
  __syncthreads();
  if (lane == 0) { r[0][warp] = ke; r[1][warp] = mr; r[2][warp] = mp; }
  __syncthreads();
  if (tid == 0) {
    ke = 0.0; mr = 1e300; mp = 1e300;
    for (int w = 0; w < nw; ++w) {
      ke += r[0][w]; mr = fmin(mr, r[1][w]); mp = fmin(mp, r[2][w]);
    }
    const long long it = *S.iter;
    double nrm = sqrt(ke / ((double)S.nx * (double)S.ny * (double)S.nz));
    double kev = nrm * S.dimc2rho;
    S.diag[0] = kev;
    S.diag[1] = mr;
    S.diag[2] = mp;
    S.diag[3] = (double)it;
    bool fail = !(kev <= 1000.0) || !(mr > 0.0) || !(mp > 0.0);
    if (fail && *S.fail_iter < 0) *S.fail_iter = it;
    *S.iter = it + 1;
    *S.counter = 0u;
  }
}

// Tiles away from every edge, CPML slab and periodic wrap: their x/y
// derivatives are the centred stencil with no branch.
template <class R>
__device__ __forceinline__ bool mhd_interior(const SimT<R> &S, int x0, int y0) {
  const int xm = max(5, S.xb.on ? S.xb.np : 0), xM = max(5, S.xt.on ? S.xt.np : 0);
  const int ym = max(5, S.yb.on ? S.yb.np : 0), yM = max(5, S.yt.on ? S.yt.np : 0);
  return x0 >= xm && x0 + mg::TX <= S.nx - xM && y0 >= ym && y0 + mg::TY <= S.ny - yM;
}

// Host side: the rectangle of interior tiles [ix0, ix1) x [iy0, iy1) (tile
// units) of a grid whose x/y CPML widths are np[0..3] (0 if off); empty if
// ix1 <= ix0 or iy1 <= iy0.
inline void mhd_interior_rect(int nx, int ny, const int np[4], int &ix0, int &ix1, int &iy0,
                              int &iy1) {
  const int xm = np[0] > 5 ? np[0] : 5, xM = np[1] > 5 ? np[1] : 5;
  const int ym = np[2] > 5 ? np[2] : 5, yM = np[3] > 5 ? np[3] : 5;
  ix0 = (xm + mg::TX - 1) / mg::TX;
  iy0 = (ym + mg::TY - 1) / mg::TY;
  ix1 = nx - xM - mg::TX >= 0 ? (nx - xM - mg::TX) / mg::TX + 1 : 0;
  iy1 = ny - yM - mg::TY >= 0 ? (ny - yM - mg::TY) / mg::TY + 1 : 0;
}

// The body covers the tile (x0, y0) over layers [k0, k1) with a block of
// 32 x 8 x 2 threads (threadIdx.z is the role); smem is the 128-byte aligned
// dynamic buffer.  TMA = false: the own-point arrays are fetched by
// cp.async too (any nx).  INT: the tile's stencil footprint touches no
// non-periodic edge, no x/y CPML slab and needs no periodic wrap, so its
// x/y derivatives are the centred stencil with no branch.  Returns false
// when a bounded wait gave up.
//
// Per layer: every thread waits for its own halo copies, turns the B0 halo
// values it copied into the fluxes v x B0 in place, then one barrier makes
// the layer visible; the copies of the next layer are issued after that
// barrier (the buffer they overwrite was last read before it).  A named
// barrier of the two warps that share rows ty (role 0 warp ty, role 1 warp
// 8 + ty) exchanges d(vz)/dz and d(by)/dz: nothing else crosses warps
// until the next layer's barrier.
//
// TW (FP64): the z windows live in tensor memory between layers
// (tmem_window.cuh; tw is this warp's window address, the caller allocates
// and frees): each layer loads them, shifts in the new head, stores them
// back and forms the z derivatives, so they hold registers only then.
template <class R, int MODE, bool TMA, bool INT, bool TW = false>
__device__ __forceinline__ bool mhd_body(const SimT<R> &S, const TmaSet *T, R *smem,
                                         const R *__restrict__ a,
                                         const R *__restrict__ tin,
                                         R *__restrict__ so, R beta, R bnext,
                                         int x0, int y0, int k0, int k1, int mt, int ma,
                                         double &ke, double &mr, double &mp, uint32_t tw = 0) {
  static_assert(!TW || sizeof(R) == 8, "TMEM windows of FP64 values");
  using namespace mg;
  // halo planes by TMA in the plain form's interior kernel (measured: 4 %
  // faster in FP64; in FP32 the 48-wide boxes cost more than the cp.async
  // copies they replace)
  constexpr bool TH = TMA && INT && sizeof(R) == 8;
  // precision form, interior tiles of a grid whose rows are 16-byte
  // multiples (the TMA own-point condition): halo rows of 48 values from
  // x0 - 8 copied as 16-byte vectors, 216 of them per plane, one per role-1
  // thread, in place of one 4-byte copy per halo position
  constexpr bool HV = TMA && INT && sizeof(R) == 4;
  using MB = MhdBuf<R, TH, HV>;
  constexpr int BUF = MB::BUF, HXL = MB::HXL, XOFF = MB::XOFF, HSL = MB::HSL;
  constexpr bool SCALED = sizeof(R) == 4;
  __shared__ unsigned long long bar[2];
  const int tx = threadIdx.x, ty = threadIdx.y, role = threadIdx.z;
  const int tid = (role * TY + ty) * TX + tx, cid = ty * TX + tx;
  const int nx = S.nx, ny = S.ny, nz = S.nz;
  const int N = (int)S.N, NXY = nx * ny;
  const int i = x0 + tx, j = y0 + ty;
  const bool act = INT || (i < nx && j < ny);
  const bool per = S.periodic;
  const int col = j * nx + i;
  const int xo = INT ? x0 - 5 : origin_t(x0, TX, nx, per);
  const int yo = INT ? y0 - 5 : origin_t(y0, TY, ny, per);
  const int ry = y0 - yo + ty, rx = x0 - xo + tx;
  const int own = ry * HXL + rx + XOFF;
  const R *isc = S.isc, *sc = S.sc;
  // depth scales of the precision form, staged in shared memory for the
  // layers this chunk touches; 1 (folded away) in the plain form
  R *ZT = smem + 2 * BUF + MB::XCH;
  const int zb = max(0, min(k0 - 5, nz - 11));
  if constexpr (SCALED) {
    const int ze = min(nz, max(k1 + 5, zb + 11));
    for (int t = tid; t < (ze - zb) * 16; t += NT) {
      const int kk = zb + (t >> 4), l = t & 15;
      ZT[t] = l < 8 ? isc[l * nz + kk] : sc[(l - 8) * nz + kk];
    }
  }
  auto IS = [&](int l, int kk) -> R {
    if constexpr (SCALED) return ZT[(kk - zb) * 16 + l];
    else return R(1);
  };
  auto SS = [&](int l, int kk) -> R {
    if constexpr (SCALED) return ZT[(kk - zb) * 16 + 8 + l];
    else return R(1);
  };
  // General tiles: each lane (x) and row (y) gets its own 11 coefficients and
  // window start in the tile, so every x/y derivative is one branch-free
  // sum: the centred row; one-sided row q at the low edge (q = i); at the
  // high edge -row q reversed over f(n-11..n-1) (derivatives.f90:72, 98).
  // CTA-uniform: every lane's (row's) stencil is the centred one (periodic
  // axis, or no lane within 5 points of an edge); then the centred sum
  // from the window start cxo (cyo) of lane (row) 0 serves
  const bool cen_x = per || (x0 >= 5 && x0 + TX <= nx - 5);
  const bool cen_y = per || (y0 >= 5 && y0 + TY <= ny - 5);
  const int cxo = x0 - 5 - xo, cyo = y0 - 5 - yo;
  // the tables: FP64 in the dynamic buffer after the exchange area
  // (MhdBuf::SMEM_GEN), FP32 static (its depth scales follow the exchange
  // area)
  constexpr bool DYN_T = !INT && !SCALED;
  __shared__ R cxs_s[INT || DYN_T ? 1 : TX * 11], cys_s[INT || DYN_T ? 1 : TY * 11];
  __shared__ int cxb_s[INT || DYN_T ? 1 : TX], cyb_s[INT || DYN_T ? 1 : TY];
  R *cxs = cxs_s, *cys = cys_s;
  int *cxb = cxb_s, *cyb = cyb_s;
  if constexpr (DYN_T) {
    cxs = smem + 2 * BUF + MB::XCH;
    cys = cxs + TX * 11;
    cxb = reinterpret_cast<int *>(cys + TY * 11);
    cyb = cxb + TX;
  }
  if (!INT && tid < TX + TY) {
    const bool isx = tid < TX;
    const int q0 = isx ? tid : tid - TX;                 // lane or row
    const int g = isx ? x0 + q0 : y0 + q0, n = isx ? nx : ny, o = isx ? xo : yo;
    R *c = isx ? cxs + q0 * 11 : cys + q0 * 11;
    int base;
    if (per || (g >= 5 && g < n - 5) || g >= n) {
      for (int m = 0; m < 11; ++m) c[m] = dcoef<R>(5, m);
      base = g - 5 - o;
    } else if (g < 5) {
      for (int m = 0; m < 11; ++m) c[m] = dcoef<R>(g, m);
      base = -o;
    } else {
      const int q = n - 1 - g;
      for (int m = 0; m < 11; ++m) c[m] = -dcoef<R>(q, 10 - m);
      base = n - 11 - o;
    }
    if (isx) cxb[q0] = base;
    else cyb[q0] = base;
  }
  if (TMA && tid == 0) {
    mbar_init_t(&bar[0]);
    mbar_init_t(&bar[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto O = [&](int b, int slot) -> R { return smem[b * BUF + slot * NC + cid]; };
  auto Hp = [&](int b, int slot) -> R * { return smem + b * BUF + NO * NC + slot * HSL; };
  R *X = smem + 2 * BUF;
  int hs0 = -1, hs1 = -1, ho0 = 0, ho1 = 0;
  {
    const int cx0 = x0 - xo, cy0 = y0 - yo;
    auto pos = [&](int t, int &hs, int &ho) {
      if constexpr (HV) {  // vector t of 216: row t / 12, values 4 (t % 12) ..
        if (t >= HY * (HXL / 4)) return;
        const int ly = t / (HXL / 4), lx = (t - ly * (HXL / 4)) * 4;
        const int gx = x0 - 8 + lx, gy = yo + ly;
        // inside the grid by the interior test (x0 >= 32, x0 + 40 <= nx
        // with nx a multiple of 4); checked so that no copy can leave it
        if (gx < 0 || gx + 3 >= nx || gy < 0 || gy >= ny) return;
        hs = ly * HXL + lx;
        ho = gy * nx + gx;
        return;
      }
      if (t >= HS) return;
      const int ly = t / HX, lx = t - ly * HX;
      const bool inx = lx >= cx0 && lx < cx0 + TX, iny = ly >= cy0 && ly < cy0 + TY;
      if (!inx && !iny) return;
      if (TH) {  // in the domain by the interior test; no global offset
        hs = ly * HXL + lx + XOFF;
        return;
      }
      int gx = xo + lx, gy = yo + ly;
      if (per) {
        gx = wrap_t(gx, nx);
        gy = wrap_t(gy, ny);
      } else if (gx < 0 || gx >= nx || gy < 0 || gy >= ny) {
        return;
      }
      hs = t;
      ho = gy * nx + gx;
    };
    // halo positions 0..511 one per thread, 512..755 on role 1 (role 0
    // carries the TMA issue and the heavier momentum update); HV: the
    // vectors on role 1
    if constexpr (HV) {
      if (role == 1) pos(tid - NC, hs0, ho0);
    } else {
      pos(tid, hs0, ho0);
      if (role == 1) pos(tid + NC, hs1, ho1);
    }
  }
  // Own-point arrays not read: where the sponge vanishes outside the CPML
  // slabs, the sponge of layers whose points lie in no slab (a CTA-uniform
  // test per layer).  rhoinv is read, not formed as 1/rho0 in the kernel:
  // the FP64 division measured 0.7 % slower than the load (FP64 kernels
  // with TMEM windows), and more in the precision form.
  const bool slab_xy = !INT && ((S.xb.on && (x0 < S.xb.np || x0 + TX > nx - S.xt.np)) ||
                                (S.yb.on && (y0 < S.yb.np || y0 + TY > ny - S.yt.np)));
  auto sponge_at = [&](int k) -> bool {
    return !S.sponge_slabs || slab_xy || (S.zb.on && (k < S.zb.np || k >= nz - S.zt.np));
  };
  auto skip_own = [&](int c, int k) -> bool {
    return (MODE == F_FIRST && c >= O_A && c < O_BG) || (MODE != F_LAST && c == O_P0) ||
           (c == O_BG + B_SPONGE && !sponge_at(k));
  };
  auto own_bytes = [&](int k) -> unsigned {
    return ((MODE == F_FIRST ? 15u : (MODE == F_MID ? 23u : 24u)) -
            (sponge_at(k) ? 0u : 1u)) *
               NC * (unsigned)sizeof(R) +
           (TH ? (unsigned)(NH * HXL * HY * sizeof(R)) : 0u);
  };
  auto issue = [&](int k, int b) {
    const int kb = k * NXY;
    if (HV && hs0 >= 0) {
      R *h = Hp(b, 0) + hs0;
      const int id = kb + ho0;
#pragma unroll
      for (int sl = 0; sl < 7; ++sl) cp16_t(h + sl * HSL, tin + (sl + 1) * N + id);
      cp16_t(h + 7 * HSL, S.box + id);
      cp16_t(h + 8 * HSL, S.boy + id);
      cp16_t(h + 9 * HSL, S.boz + id);
    }
    if (!TH && !HV && hs0 >= 0) {
      R *h = Hp(b, 0) + hs0;
      const int id = kb + ho0;
#pragma unroll
      for (int sl = 0; sl < 7; ++sl) cp_r(h + sl * HSL, tin + (sl + 1) * N + id);
      cp_r(h + 7 * HSL, S.box + id);
      cp_r(h + 8 * HSL, S.boy + id);
      cp_r(h + 9 * HSL, S.boz + id);
    }
    if (!TH && hs1 >= 0) {
      R *h = Hp(b, 0) + hs1;
      const int id = kb + ho1;
#pragma unroll
      for (int sl = 0; sl < 7; ++sl) cp_r(h + sl * HSL, tin + (sl + 1) * N + id);
      cp_r(h + 7 * HSL, S.box + id);
      cp_r(h + 8 * HSL, S.boy + id);
      cp_r(h + 9 * HSL, S.boz + id);
    }
    if (!TMA && act) {
      R *ob = smem + b * BUF + cid;
      const int id = kb + col;
      if (role == 0) {
        cp_r(ob + O_RHO * NC, tin + id);
        if (MODE != F_FIRST)
#pragma unroll
          for (int l = 0; l < 8; ++l) cp_r(ob + (O_A + l) * NC, a + l * N + id);
      } else {
        const R *bg[14] = {S.red, S.sponge, S.rho0, S.grx, S.gry, S.grz,
                               S.c2rho0, S.gpx, S.gpy, S.gpz, S.rhoinv, S.cbx, S.cby, S.cbz};
        const bool spg = sponge_at(k);
#pragma unroll
        for (int n = 0; n < 14; ++n)
          if (n != B_SPONGE || spg)
            cp_r(ob + (O_BG + n) * NC, bg[n] + id);
        if (MODE == F_LAST) cp_r(ob + O_P0 * NC, S.p0 + id);
      }
    }
    cp_commit_t();
    // TMA copies of the layer, spread over warp 0 (lane l issues copies l
    // and l + 32): copy c < 24 is own slot c (stage rho, a[0..7], 14
    // background arrays, p0); with TH, copy 24 + s is halo plane s (state
    // fields 1..7, then B0 x, y, z)
    if (TMA && tid < 32) {
      if (tid == 0) mbar_tx_t(&bar[b], own_bytes(k));
      __syncwarp();
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      R *ob = smem + b * BUF;
      for (int c = tid; c < (TH ? NO + NH : NO); c += 32) {
        if (skip_own(c, k)) continue;
        int map = mt, xx = x0, yy = y0, z = k;
        R *dst = ob + c * NC;
        if (c >= O_A && c < O_BG) {
          map = ma;
          z = (c - O_A) * nz + k;
        } else if (c >= O_BG && c <= O_P0) {
          map = 3 + (c - O_BG);
        } else if (c >= NO) {
          const int sl = c - NO;
          dst = Hp(b, sl);
          xx = x0 - 5 - XOFF;
          yy = y0 - 5;
          if (sl < 7) {
            map = 18 + mt;
            z = (sl + 1) * nz + k;
          } else {
            map = 21 + (sl - 7);
          }
        }
        tma3d_t(dst, &T->m[map], xx, yy, z, &bar[b]);
      }
    }
  };
  // fluxes v x B0 (stored velocity units) in place of the B0 halo values,
  // at the halo positions this thread copied
  auto flux = [&](int b, int t) {
    R *H = Hp(b, 0) + t;
    const R vx_ = H[0], vy_ = H[HSL], vz_ = H[2 * HSL];
    const R bx0 = H[7 * HSL], by0 = H[8 * HSL], bz0 = H[9 * HSL];
    H[7 * HSL] = -vz_ * by0 + vy_ * bz0;
    H[8 * HSL] = -vx_ * bz0 + vz_ * bx0;
    H[9 * HSL] = -vy_ * bx0 + vx_ * by0;
  };
  R w0[11], w1[11], w2[11];  // physical values
  auto head = [&](int kk, R &v0, R &v1, R &v2) {
    const int id = kk * NXY + col;
    if (role == 0) {
      v0 = __ldg(tin + 3 * N + id) * IS(3, kk);
      v1 = __ldg(tin + 4 * N + id) * IS(4, kk);
      v2 = __ldg(tin + 5 * N + id) * IS(5, kk);
    } else {
      const R iv = IS(1, kk);
      const R vx_ = __ldg(tin + N + id) * iv, vy_ = __ldg(tin + 2 * N + id) * iv,
                  vz_ = __ldg(tin + 3 * N + id) * iv;
      const R ox = __ldg(S.box + id), oy = __ldg(S.boy + id), oz = __ldg(S.boz + id);
      v0 = -vz_ * oy + vy_ * oz;
      v1 = -vx_ * oz + vz_ * ox;
      v2 = __ldg(tin + 6 * N + id) * IS(6, kk);
    }
  };
  // the z-window head of layer kk is read from DRAM a layer before it is
  // needed; an L2 prefetch two layers earlier takes that latency off the
  // layer loop
  auto prefetch = [&](int kk) {
    if (!act || kk >= nz) return;
    const int id = kk * NXY + col;
    if (role == 0) {
      pf_l2(tin + 3 * N + id);
      pf_l2(tin + 4 * N + id);
      pf_l2(tin + 5 * N + id);
    } else {
      pf_l2(tin + N + id);
      pf_l2(tin + 2 * N + id);
      pf_l2(tin + 6 * N + id);
      pf_l2(S.box + id);
      pf_l2(S.boy + id);
      pf_l2(S.boz + id);
    }
  };
  issue(k0, 0);
  prefetch(k0 + 6);
  {
    const int b0 = min(k0 - 5, nz - 11);
#pragma unroll
    for (int m = 0; m < 11; ++m) {
      const int kk = b0 + m;
      if (act && kk >= 0) head(kk, w0[m], w1[m], w2[m]);
      else w0[m] = w1[m] = w2[m] = R(0);
    }
    if constexpr (TW) {
      __syncwarp();
      tm_wait_st();  // a previous work item's stores to these columns
      tm_st_window(tm_window(tw, 0), w0);
      tm_st_window(tm_window(tw, 1), w1);
      tm_st_window(tm_window(tw, 2), w2);
    }
  }
  unsigned phase = 0;
  int rr = 0;  // TW: ring position of the windows (logical value 0 in slot rr)
  bool ok = true;
  const R dt = (R)S.deltat;
  const R sx = (R)S.stretchx, sy = (R)S.stretchy;
  const R *gcol = S.gblk + (act ? S.colx[i] + S.bxdim * S.coly[j] : 0) * nz;
  // PULSE = 1 time factor: the iteration is fixed during a stage
  const R Tp = S.frc.kind == SPARC_SRC_PULSE ? pulse_time_t(S, *S.iter) : R(0);
  // |v_new|^2 of the last stage (role 0 writes, role 1 reads after a barrier)
  double *VSQ = (double *)(SCALED ? X + 2 * NC : X + NC);

  for (int k = k0; k < k1; ++k) {
    const int b = (k - k0) & 1;
    const int id = k * NXY + col;
    R h0 = 0, h1 = 0, h2 = 0;
    const bool sh = k > k0 && k <= nz - 6;
    if (sh && act) head(k + 5, h0, h1, h2);
    prefetch(k + 7);
    // precision form, last stage: the compensation carries of layer k + 2
    // into L2 (they are read just before their use)
    if (SCALED && MODE == F_LAST && act && k + 2 < k1) {
      const int id2 = (k + 2) * NXY + col;
      if (role == 0) {
        pf_l2(S.carry + N + id2);
        pf_l2(S.carry + 2 * N + id2);
        pf_l2(S.carry + 3 * N + id2);
      } else {
        pf_l2(S.carry + id2);
        pf_l2(S.carry + 4 * N + id2);
        pf_l2(S.carry + 5 * N + id2);
        pf_l2(S.carry + 6 * N + id2);
        pf_l2(S.carry + 7 * N + id2);
      }
    }
    // momentum role: own-point B0 (its halo slots will hold the fluxes),
    // gravity and forcing, prefetched into L1 here and loaded after the
    // exchange barrier (not live across the derivatives: fewer registers)
    R ox = 0, oy = 0, oz = 0, gk = 0, frc = 0;
    auto own_loads = [&] {
      ox = __ldg(S.box + id);
      oy = __ldg(S.boy + id);
      oz = __ldg(S.boz + id);
      gk = __ldg(gcol + k);
      if (S.frc.kind != SPARC_SRC_NONE) frc = forcing_t(S, Tp, i, j, k);
    };
    if (role == 0 && act) {
      pf_l1(S.box + id);
      pf_l1(S.boy + id);
      pf_l1(S.boz + id);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    const R szk = __ldg(S.stretch + k);
    // TW: the z derivatives of the three windows, formed by the whole warp
    // (the TMEM accesses are warp-collective); they read no shared memory,
    // so they are formed before the wait for the layer's copies and the
    // layer barrier, overlapping both (0.6 % per iteration, A/B on one box)
    R wz0 = R(0), wz1 = R(0), wz2 = R(0);
    if constexpr (TW) {
      __syncwarp();
      tm_wait_st();  // the previous layer's store of these columns
      // the windows are rings: each layer with a new head stores only the
      // head, into the slot of the layer it replaces, (rr + 10) % 11
      if (sh) rr = rr == 10 ? 0 : rr + 1;
      const uint32_t hslot = 2u * (uint32_t)(rr == 0 ? 10 : rr - 1);
      auto zwin = [&](int f, R h) -> R {
        R v[11];
        tm_ld_window(tm_window(tw, f), v);
        if (sh) tm_st_one(tm_window(tw, f) + hslot, h);
        return dz_ring(v, h, sh, rr, k, nz, szk);
      };
      wz0 = zwin(0, h0);
      wz1 = zwin(1, h1);
      wz2 = zwin(2, h2);
    }
    bool mine = true;
    // TH: every thread waits for the layer's TMA copies (its flux positions
    // arrive that way); otherwise thread 0 alone, before the barrier
    if (TH) mine = mbar_wait_t(&bar[b], (phase >> b) & 1u, S.err);
    if constexpr (HV) {
      if (mine && hs0 >= 0)
#pragma unroll
        for (int q = 0; q < 4; ++q) flux(b, hs0 + q);
    } else {
      if (mine && hs0 >= 0) flux(b, hs0);
      if (mine && hs1 >= 0) flux(b, hs1);
    }
    if (TMA && !TH && tid == 0) mine = mbar_wait_t(&bar[b], (phase >> b) & 1u, S.err);
    phase ^= 1u << b;
    if (!__syncthreads_and(mine)) { ok = false; break; }
    if (k + 1 < k1) issue(k + 1, b ^ 1);
    if constexpr (!TW) {
      if (sh) { shift_t(w0, h0); shift_t(w1, h1); shift_t(w2, h2); }
    }
    auto DZ = [&](int f) -> R {
      if constexpr (TW) {
        return f == 0 ? wz0 : (f == 1 ? wz1 : wz2);
      } else {
        if (f == 0) return dz_t(w0, k, nz, szk);
        if (f == 1) return dz_t(w1, k, nz, szk);
        return dz_t(w2, k, nz, szk);
      }
    };
    auto DX = [&](int slot) {
      const R *row = Hp(b, slot) + ry * HXL + XOFF;
      if (INT) return sx * csum_t(row + tx, 1);
      if (cen_x) return sx * csum_t(row + cxo + tx, 1);
      const R *r = row + cxb[tx], *c = cxs + tx * 11;
      R sum = R(0);
#pragma unroll
      for (int m = 0; m < 11; ++m) sum += r[m] * c[m];
      return sx * sum;
    };
    auto DY = [&](int slot) {
      const R *colp = Hp(b, slot) + rx + XOFF;
      if (INT) return sy * csum_t(colp + ty * HXL, HXL);
      if (cen_y) return sy * csum_t(colp + (cyo + ty) * HXL, HXL);
      const R *r = colp + cyb[ty] * HXL, *c = cys + ty * 11;
      R sum = R(0);
#pragma unroll
      for (int m = 0; m < 11; ++m) sum += r[m * HXL] * c[m];
      return sy * sum;
    };
    const bool zpml = S.zb.on && (k < S.zb.np || k >= nz - S.zt.np);
    const bool xpml = !INT && S.xb.on && act && (i < S.xb.np || i >= nx - S.xt.np);
    const bool ypml = !INT && S.yb.on && act && (j < S.yb.np || j >= ny - S.yt.np);
    auto pz = [&](int s0, int s1, int s2, R &da, R &db, R &dc) {
      const bool bot = k < S.zb.np;
      const FaceT<R> &F = bot ? S.zb : S.zt;
      const int kl = bot ? k : k - (nz - S.zt.np);
      cpml3_t<R, MODE>(F, (long long)kl * NXY + col, kl, s0, s1, s2, beta, dt, da, db, dc);
    };
    auto px = [&](int s0, int s1, int s2, R &da, R &db, R &dc) {
      const bool bot = i < S.xb.np;
      const FaceT<R> &F = bot ? S.xb : S.xt;
      const int il = bot ? i : i - (nx - S.xt.np);
      cpml3_t<R, MODE>(F, il + (long long)F.np * (j + (long long)ny * k), il, s0, s1, s2, beta,
                     dt, da, db, dc);
    };
    auto py = [&](int s0, int s1, int s2, R &da, R &db, R &dc) {
      const bool bot = j < S.yb.np;
      const FaceT<R> &F = bot ? S.yb : S.yt;
      const int jl = bot ? j : j - (ny - S.yt.np);
      cpml3_t<R, MODE>(F, i + (long long)nx * (jl + (long long)F.np * k), jl, s0, s1, s2, beta,
                     dt, da, db, dc);
    };
    auto Hv = [&](int slot) { return Hp(b, slot)[own]; };
    const R iv = IS(1, k);  // velocity (and flux) scale of this layer
    R d0 = 0, d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0, d6 = 0, d7 = 0, d8 = 0;
    if (act) {
      const R ip = IS(4, k), ib = IS(5, k);
      if (role == 0) {
        d0 = ip * DX(3); d5 = ib * DX(6); d7 = ib * DX(5);
        d1 = ip * DY(3); d4 = ib * DY(6); d8 = ib * DY(4);
        d3 = DZ(0); d2 = DZ(1); d6 = DZ(2);
        if (zpml) pz(1, 0, 2, d2, d3, d6);
        if (xpml) px(1, 3, 2, d0, d5, d7);
        if (ypml) py(1, 3, 2, d1, d4, d8);
        X[cid] = d3;
        // curl b: y and z components now, x after the exchange (fewer live
        // registers across the barrier; the same arithmetic)
        d5 = -d5 + d6;
        d7 = d7 - d8;
      } else {
        d0 = iv * DX(0); d2 = iv * DX(9); d3 = iv * DX(8);
        d1 = iv * DY(1); d4 = iv * DY(9); d5 = iv * DY(7);
        d6 = DZ(0); d7 = DZ(1); d8 = DZ(2);
        if (zpml) pz(4, 5, 3, d7, d6, d8);
        if (xpml) px(0, 4, 5, d0, d2, d3);
        if (ypml) py(0, 4, 5, d1, d4, d5);
        X[NC + cid] = d8;
        // curl(v x B0) and d(vx)/dx + d(vy)/dy now (fewer live registers
        // across the barrier; the same arithmetic)
        d4 = d4 - d7;
        d6 = d6 - d2;
        d3 = d3 - d5;
        d0 = d0 + d1;
      }
    }
    // the exchange involves only the role-0 and role-1 warps of rows ty
    bar_pair_t(1 + ty);
    double an_rho = 0.0;
    if (act) {
      const bool zero = k == 0 || k == nz - 1 ||
                        (!INT && !per && (i == 0 || i == nx - 1 || j == 0 || j == ny - 1));
      const R fac = MODE == F_LAST ? dt : bnext;
      const R rho = O(b, O_RHO) * IS(0, k), vx = Hv(0) * iv, vy = Hv(1) * iv,
                  vz = Hv(2) * iv;
      const R red = O(b, O_BG + B_RED);
      const R sg = sponge_at(k) ? O(b, O_BG + B_SPONGE) : R(0);
      if (role == 0) {
        own_loads();
        const R ib = IS(5, k);
        const R dzby = X[NC + cid];
        const R cbx = d4 - dzby, cby = d5, cbz = d7;
        const R c1 = cby * oz - cbz * oy, c2 = ox * cbz - cbx * oz, c3 = cbx * oy - cby * ox;
        const R ri = O(b, O_BG + B_RHOINV);
        R vxr = -ri * (d0 - (c1 * red)) - sg * vx;
        R vyr = -ri * (d1 - (c2 * red)) - sg * vy;
        R vzr = -ri * (d2 - (c3 * red)) - sg * vz;
        const R bx = Hv(4) * ib, by = Hv(5) * ib, bz = Hv(6) * ib;
        const R qx = O(b, O_BG + B_CBX), qy = O(b, O_BG + B_CBY), qz = O(b, O_BG + B_CBZ);
        const R e1 = qy * bz - qz * by, e2 = bx * qz - qx * bz, e3 = qx * by - qy * bx;
        vxr = vxr + ri * e1 * red;
        vyr = vyr + ri * e2 * red;
        vzr = vzr + ri * e3 * red;
        vzr = vzr - ri * rho * gk;
        if (S.frc.kind != SPARC_SRC_NONE) {
          if (S.frc.dir == 1) vxr = vxr + frc;
          else if (S.frc.dir == 2) vyr = vyr + frc;
          else vzr = vzr + frc;
        }
        const R sv = SS(1, k);
        R Rv[3] = {vxr, vyr, vzr};
        // DAMPING (plain form): the velocity RHS minus the damping term,
        // after the boundary zeroing, so the boundary planes move by -term
        // (RHS.f90:166-172, 659-665)
        bool zv = zero;
        if constexpr (!SCALED) {
          if (S.term) {
#pragma unroll
            for (int l = 0; l < 3; ++l)
              Rv[l] = (zero ? R(0) : Rv[l]) - __ldg(S.term + (long long)l * N + id);
            zv = false;
          }
        }
        double vsq = 0.0;
#pragma unroll
        for (int l = 1; l < 4; ++l) {
          const R av = MODE == F_FIRST ? Hv(l - 1) : O(b, O_A + l);
          R an;
          if (MODE == F_LAST) {
            if constexpr (SCALED) {
              R c = S.carry[l * N + id];
              an = zero ? av : kahan(av, fac * (sv * Rv[l - 1]), c);
              S.carry[l * N + id] = c;
              const double ph = ((double)an - (double)c) * (double)iv;
              vsq += ph * ph;
            } else {
              an = zv ? av : av + fac * Rv[l - 1];
              vsq += (double)an * (double)an;
            }
          } else {
            an = zv ? av : av + fac * (sv * Rv[l - 1]);
          }
          so[l * N + id] = an;
        }
        if (MODE == F_LAST) VSQ[cid] = vsq;
      } else {
        const R p = Hv(3) * IS(4, k);
        const R dvzdz = X[cid];
        const R div = d0 + dvzdz;
        const R r0 = O(b, O_BG + B_RHO0);
        const R Rr = -O(b, O_BG + B_GRX) * vx - O(b, O_BG + B_GRY) * vy -
                         O(b, O_BG + B_GRZ) * vz - r0 * div - sg * rho;
        const R Rp = -O(b, O_BG + B_C2R) * div - vx * O(b, O_BG + B_GPX) -
                         vy * O(b, O_BG + B_GPY) - vz * O(b, O_BG + B_GPZ) - sg * p;
        const R Rb[3] = {red * d4, red * d6, red * d3};
        const R Rs[5] = {Rr, Rp, Rb[0], Rb[1], Rb[2]};
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          const int l = q == 0 ? 0 : (q == 1 ? 4 : q + 3);
          const R av = MODE == F_FIRST ? (l == 0 ? O(b, O_RHO) : Hv(l - 1)) : O(b, O_A + l);
          const R s = SS(l, k);
          R an;
          if (MODE == F_LAST) {
            if constexpr (SCALED) {
              R c = S.carry[l * N + id];
              an = zero ? av : kahan(av, fac * (s * Rs[q]), c);
              S.carry[l * N + id] = c;
              if (q == 0) an_rho = ((double)an - (double)c) * (double)IS(0, k);
            } else {
              an = zero ? av : av + fac * Rs[q];
              if (q == 0) an_rho = an;
            }
          } else {
            an = zero ? av : av + fac * (s * Rs[q]);
          }
          so[l * N + id] = an;
        }
        if (MODE == F_LAST) {
          mr = fmin(mr, (double)rho + (double)r0);
          mp = fmin(mp, (double)p + (double)O(b, O_P0));
        }
      }
    }
    if (MODE == F_LAST) {
      bar_pair_t(1 + ty);
      if (act && role == 1) {
        const double m = ((double)O(b, O_BG + B_RHO0) + an_rho) * VSQ[cid] / 2.0;
        ke += m * m;
      }
    }
  }
  if (!ok) {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (TMA && tid == 0) {
      mbar_wait_t(&bar[0], phase & 1u, S.err);
      mbar_wait_t(&bar[1], (phase >> 1) & 1u, S.err);
    }
    return false;
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  return true;
}



}  // namespace sparc
