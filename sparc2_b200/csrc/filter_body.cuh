// filter_body.cuh -- FILTER_VARS (derivatives.f90:659-703) as two kernels
// per filter event, shared by the plain form (R = double, step.cu) and the
// precision form (R = float, step32.cu).
//
//   * xy (nn % xyfreq == 0): one fused pass per layer tile.  A CTA loads a
//     (32+12) x (32+12) tile of one field's layer into shared memory (in
//     FP64 on non-periodic grids as one TMA tensor copy per layer), forms
//     the y pre-average of the non-periodic edge rows (derivatives.f90:671-
//     675), the y filter of filty (derivatives.f90:345-447) with its edge
//     rows (copy-through for the 11-point filter, zero for the 7-point one)
//     and the mode-2 combination a - s*filt, then the x pre-average
//     (derivatives.f90:680-684), the x filter and its combination, and
//     writes the tile once.  The reference's y-then-x order is kept.
//   * z (nn % zfreq == 0): a CTA loads a slab of 32 x 4 columns of one field
//     over 32 layers and their 6-layer margins into shared memory (44 KB in
//     FP64, so that five CTAs share an SM), every load in flight at once
//     (in FP64 one 4-D TMA tensor copy);
//     each thread then runs a 13-deep register window of raw values down
//     its column for 16 layers (the pre-average of derivatives.f90:690-693
//     needs the neighbours of the 11 taps).  The z chunks of a slab are
//     adjacent in the launch order, so their shared margins come from L2.
//     filtz's edge layers are copied through (derivatives.f90:610-633).
//
// The filter width (11 or 7 points) and the carry are template parameters,
// so a kernel carries no per-element branch on them.  No 64-bit division
// or modulo per element: tile and column coordinates come from the launch
// geometry.  In the precision form the stored state
// is depth-scaled and carries a compensation term: within a layer the scale
// is one number, so the xy pass filters stored values; the z pass filters
// physical values (stored * isc(k)) and stores back times sc(k).  The first
// pass of an event reads stored - carry (the compensated value) and the
// caller clears the carry after the event.
//
// Each translation unit defines fcoef<R>(g, m): its constant table of the
// filter stencils (initialize.f90:1929-1957), [0] the 11-point, [1] the
// 7-point one.
#pragma once

#include "internal.h"
#include "tma_util.cuh"

namespace sparc {

template <class R>
__device__ __forceinline__ R fcoef(int table, int m);

// dynamic shared memory of the z pass (one slab)
template <class R>
constexpr size_t filt_z_smem();

template <class R>
struct FiltArgs {
  int nx, ny, nz, V;
  long long N;
  int periodic;
  R s;                // a - s*filt (7-point filter)
  const R *in;
  R *out;
  const R *carry;     // compensation subtracted on load (first pass), or null
  const R *sc, *isc;  // depth scales V x nz (precision form z pass), or null
  int *err;           // device error flag (bounded waits of the TMA copies)
};

namespace fb {
// xy pass: a 32 x 32 tile per CTA of 32 x 8 threads; the y pass gives 176
// of them 8 rows of one of the 44 loaded columns
constexpr int TX = 32, TY = 8, NT = TX * TY;
constexpr int TR = 32, YG = 8;            // tile rows, rows per y-pass item
constexpr int RX = TX + 12, RY = TR + 12;
constexpr int NYI = RX * (TR / YG);       // y-pass items
constexpr int LPB = 8;                    // layers per xy CTA (pipelined)
static_assert(NYI <= NT, "one y-pass item per thread at most");
constexpr int ZX = 32, ZY = 4, ZC = 32;   // z pass: 32 x 4 columns x 32 layers
constexpr int ZH = ZC + 12;               // layers loaded per z slab
constexpr int ZL = ZC / 2;                // layers per thread
}  // namespace fb

template <class R>
constexpr size_t filt_z_smem() {
  return (size_t)fb::ZH * fb::ZY * fb::ZX * sizeof(R);
}

// q wrapped into [0, n) (q within a few periods of the range)
__device__ __forceinline__ int wrap_idx(int q, int n) {
  while (q < 0) q += n;
  while (q >= n) q -= n;
  return q;
}

// the 2G+1 taps of the filter at centre p of a strided row: G = 5 the
// 11-point table, G = 3 the 7-point one
template <class R, int G>
__device__ __forceinline__ R ftaps(const R *p, int st) {
  R s = R(0);
#pragma unroll
  for (int m = 0; m <= 2 * G; ++m) s += p[(m - G) * st] * fcoef<R>(G == 5 ? 0 : 1, m);
  return s;
}

// Pre-average in place (derivatives.f90:671-675, 680-684): the rows (DIM = 0)
// or columns (DIM = 1) q = 1..G-1 and n-G..n-2 of a shared array with row
// pitch RX, whose index 0 sits at grid coordinate o, and whose rows or
// columns [1, lim) may be read; each becomes the mean of its two neighbours.
// ext: the extent along the other axis.  All values are formed before any
// is stored (the reference averages the unaveraged array).
template <class R, int G, int DIM>
__device__ __forceinline__ void pre_average(R *a, int o, int n, int lim, int ext, int tid) {
  constexpr int NE = 2 * (G - 1);
  constexpr int PER = (NE * 44 + fb::NT - 1) / fb::NT;
  R v[PER];
  int at[PER];
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    at[u] = -1;
    const int t = tid + u * fb::NT;
    if (t >= NE * ext) continue;
    const int e = t / ext, x = t - e * ext;
    const int q = e < G - 1 ? 1 + e : n - G + (e - (G - 1));
    const int l = q - o;
    if (q < 1 || q > n - 2 || l < 1 || l >= lim) continue;
    const int p = DIM == 0 ? l * fb::RX + x : x * fb::RX + l;
    const int st = DIM == 0 ? fb::RX : 1;
    v[u] = (a[p + st] + a[p - st]) / R(2);
    at[u] = p;
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < PER; ++u)
    if (at[u] >= 0) a[at[u]] = v[u];
  __syncthreads();
}

// The fused y-then-x pass over the 32 x 32 tile (x0, y0) of layer k of
// field l; block (TX, TY) threads.  G: the filter half-width (5: the
// 11-point filter, result filt; 3: the 7-point one, result a - s*filt).
// CARRY: the first pass of a precision-form event (stored - carry).
template <class R, int G, bool CARRY>
__device__ __forceinline__ void filt_xy_tile(const FiltArgs<R> &F, int l, int k, int x0,
                                             int y0) {
  using namespace fb;
  constexpr bool M2 = G == 3;
  static_assert(RX == 44, "pre_average's item count");
  __shared__ R raw[RY][RX];  // rows y0-6 .., columns x0-6 ..
  __shared__ R fy[TR][RX];   // after the y pass, rows y0 .., columns x0-6 ..
  const int tid = threadIdx.y * TX + threadIdx.x;
  const int nx = F.nx, ny = F.ny;
  const bool per = F.periodic;
  const R fs = F.s;
  const long long base = (long long)l * F.N + (long long)k * nx * ny;
  const R *in = F.in + base;
  const R *cin = CARRY ? F.carry + base : nullptr;
  // the (32+12) x (32+12) neighbourhood, one flat index over it
  for (int t = tid; t < RY * RX; t += NT) {
    const int ry = t / RX, rx = t - ry * RX;
    int gy = y0 - 6 + ry, gx = x0 - 6 + rx;
    bool ok = true;
    if (per) {
      gy = wrap_idx(gy, ny);
      gx = wrap_idx(gx, nx);
    } else {
      ok = gy >= 0 && gy < ny && gx >= 0 && gx < nx;
    }
    R v = R(0);
    if (ok) {
      const int id = gy * nx + gx;
      v = in[id];
      if (CARRY) v = v - cin[id];
    }
    raw[ry][rx] = v;
  }
  __syncthreads();
  // y pre-average of rows 1..G-1 and ny-G..ny-2 (non-periodic) on the tiles
  // whose y window reaches such a row (rows 1 .. RY-2 are read below)
  if (!per && (y0 - 5 <= G - 1 || y0 + TR + 4 >= ny - G))
    pre_average<R, G, 0>(&raw[0][0], y0 - 6, ny, RY - 1, RX, tid);
  // the y pass: column rx, rows r0 .. r0+7 from one read of the 8 + 2G
  // values around them (the centre of row r0 + j is v[j + 5])
  if (tid < NYI) {
    const int grp = tid / RX, rx = tid - grp * RX, r0 = grp * YG;
    const R *sb = &raw[r0 + 1][rx];
    R v[YG + 10];
#pragma unroll
    for (int q = 5 - G; q < YG + 5 + G; ++q) v[q] = sb[q * RX];
#pragma unroll
    for (int j = 0; j < YG; ++j) {
      const int gyo = y0 + r0 + j;
      const R pq = v[j + 5];
      R filt;
      if (!per && (gyo < G || gyo >= ny - G)) {
        filt = M2 ? R(0) : pq;
      } else {
        R s = R(0);
#pragma unroll
        for (int m = 0; m <= 2 * G; ++m) s += v[j + 5 - G + m] * fcoef<R>(G == 5 ? 0 : 1, m);
        filt = s;
      }
      fy[r0 + j][rx] = M2 ? pq - fs * filt : filt;
    }
  }
  __syncthreads();
  // x pre-average of columns 1..G-1 and nx-G..nx-2 on the tiles whose x
  // window reaches such a column
  if (!per && (x0 - 5 <= G - 1 || x0 + TX + 4 >= nx - G))
    pre_average<R, G, 1>(&fy[0][0], x0 - 6, nx, RX - 1, TR, tid);
  // the x pass at the tile's own columns, a warp per row
  R *out = F.out + base;
#pragma unroll
  for (int u = 0; u < TR * TX / NT; ++u) {
    const int t = tid + u * NT;
    const int r = t / TX, tx = t - r * TX;
    const int gxo = x0 + tx, gyo = y0 + r;
    if (gxo >= nx || gyo >= ny) continue;
    const R *c = &fy[r][tx + 6];
    const R pq = *c;
    const R filt = (!per && (gxo < G || gxo >= nx - G)) ? (M2 ? R(0) : pq) : ftaps<R, G>(c, 1);
    out[gyo * nx + gxo] = M2 ? pq - fs * filt : filt;
  }
}

// 4- or 8-byte cp.async of one value; ok = false fills the slot with zero
// (no byte is read)
template <class R>
__device__ __forceinline__ void filt_cp(R *dst, const R *src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const unsigned n = ok ? (unsigned)sizeof(R) : 0u;
  if constexpr (sizeof(R) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(n)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n)
                 : "memory");
}

// The fused y-then-x pass over layers k0 .. k0+nk-1 of the 32 x 32 tile
// (x0, y0) of field l (no carry): the neighbourhood of the next layer is
// copied into the second buffer while a layer is filtered, so the loads of
// one layer overlap the arithmetic of the previous one.  The arithmetic is
// filt_xy_tile's.  TMA (non-periodic grids, rows a multiple of 16 bytes):
// the neighbourhood is one 44 x 44 x 1 tile of `map` (the input buffer as
// nx x ny x (V nz)) from (x0 - 6, y0 - 6), issued by one thread; the tensor
// copy reads zero outside the grid, as the edge rule wants, and x0 - 6 is
// even, so the start is 16-byte aligned.  Otherwise every thread copies
// its share by cp.async (zero fill outside the grid, wrap on periodic
// axes).
template <class R, int G, bool TMA = false>
__device__ __forceinline__ void filt_xy_layers(const FiltArgs<R> &F, int l, int k0, int nk,
                                               int x0, int y0,
                                               const CUtensorMap *map = nullptr) {
  using namespace fb;
  constexpr bool M2 = G == 3;
  static_assert(RX == 44, "pre_average's item count");
  static_assert(RY * RX * sizeof(R) % 128 == 0, "each layer buffer 128-byte aligned");
  __shared__ __align__(128) R raw2[2][RY][RX];  // two layers' rows y0-6 .., columns x0-6 ..
  __shared__ R fy[TR][RX];       // after the y pass, rows y0 .., columns x0-6 ..
  __shared__ unsigned long long fbar[2];
  const int tid = threadIdx.y * TX + threadIdx.x;
  const int nx = F.nx, ny = F.ny;
  const bool per = F.periodic;
  const R fs = F.s;
  const long long NXY = (long long)nx * ny;
  const R *inl = F.in + (long long)l * F.N;
  R *outl = F.out + (long long)l * F.N;
  if constexpr (TMA) {
    if (tid == 0) {
      mbar_init_t(&fbar[0]);
      mbar_init_t(&fbar[1]);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
  }
  auto issue = [&](int k, int b) {
    if constexpr (TMA) {
      if (tid == 0) {
        // orders the generic reads and writes of this buffer (two layers
        // back, before a barrier) before the tensor copy's writes
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_tx_t(&fbar[b], (unsigned)(RY * RX * sizeof(R)));
        tma3d_t(&raw2[b][0][0], map, x0 - 6, y0 - 6, l * F.nz + k, &fbar[b]);
      }
    } else {
      const R *in = inl + (long long)k * NXY;
#pragma unroll 1
      for (int t = tid; t < RY * RX; t += NT) {
        const int ry = t / RX, rx = t - ry * RX;
        int gy = y0 - 6 + ry, gx = x0 - 6 + rx;
        bool ok = true;
        if (per) {
          gy = wrap_idx(gy, ny);
          gx = wrap_idx(gx, nx);
        } else {
          ok = gy >= 0 && gy < ny && gx >= 0 && gx < nx;
        }
        filt_cp(&raw2[b][ry][rx], ok ? in + gy * nx + gx : in, ok);
      }
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
  };
  const bool ypre = !per && (y0 - 5 <= G - 1 || y0 + TR + 4 >= ny - G);
  const bool xpre = !per && (x0 - 5 <= G - 1 || x0 + TX + 4 >= nx - G);
  issue(k0, 0);
  for (int kk = 0; kk < nk; ++kk) {
    const int b = kk & 1;
    // the buffer being refilled was last read before the previous layer's
    // post-y-pass barrier
    if (kk + 1 < nk) issue(k0 + kk + 1, b ^ 1);
    if constexpr (TMA) {
      // every thread sees the tensor copy complete (buffer b's (kk/2)-th fill)
      const bool ok = mbar_wait_t(&fbar[b], (unsigned)(kk >> 1) & 1u, F.err);
      if (!__syncthreads_and(ok)) {
        // gave up (error flag raised): wait, again bounded, for the copies
        // still in flight into this CTA's buffers, then leave
        if (tid == 0) {
          mbar_wait_t(&fbar[b], (unsigned)(kk >> 1) & 1u, F.err);
          if (kk + 1 < nk) mbar_wait_t(&fbar[b ^ 1], (unsigned)((kk + 1) >> 1) & 1u, F.err);
        }
        return;
      }
    } else {
      if (kk + 1 < nk) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
      else asm volatile("cp.async.wait_group 0;\n" ::: "memory");
      __syncthreads();  // this layer's values visible; the previous x pass done
    }
    R(*raw)[RX] = raw2[b];
    if (ypre) pre_average<R, G, 0>(&raw[0][0], y0 - 6, ny, RY - 1, RX, tid);
    if (tid < NYI) {
      const int grp = tid / RX, rx = tid - grp * RX, r0 = grp * YG;
      const R *sb = &raw[r0 + 1][rx];
      R v[YG + 10];
#pragma unroll
      for (int q = 5 - G; q < YG + 5 + G; ++q) v[q] = sb[q * RX];
#pragma unroll
      for (int j = 0; j < YG; ++j) {
        const int gyo = y0 + r0 + j;
        const R pq = v[j + 5];
        R filt;
        if (!per && (gyo < G || gyo >= ny - G)) {
          filt = M2 ? R(0) : pq;
        } else {
          R sm = R(0);
#pragma unroll
          for (int m = 0; m <= 2 * G; ++m) sm += v[j + 5 - G + m] * fcoef<R>(G == 5 ? 0 : 1, m);
          filt = sm;
        }
        fy[r0 + j][rx] = M2 ? pq - fs * filt : filt;
      }
    }
    __syncthreads();
    if (xpre) pre_average<R, G, 1>(&fy[0][0], x0 - 6, nx, RX - 1, TR, tid);
    R *out = outl + (long long)(k0 + kk) * NXY;
#pragma unroll
    for (int u = 0; u < TR * TX / NT; ++u) {
      const int t = tid + u * NT;
      const int r = t / TX, tx = t - r * TX;
      const int gxo = x0 + tx, gyo = y0 + r;
      if (gxo >= nx || gyo >= ny) continue;
      const R *c = &fy[r][tx + 6];
      const R pq = *c;
      const R filt =
          (!per && (gxo < G || gxo >= nx - G)) ? (M2 ? R(0) : pq) : ftaps<R, G>(c, 1);
      out[gyo * nx + gxo] = M2 ? pq - fs * filt : filt;
    }
  }
}

// The z pass of a slab of 32 x 4 columns and ZC layers from k0 of field l:
// the slab and its 6-layer margins are loaded into shared memory in one go
// (every load in flight at once), then each thread filters ZL consecutive
// layers of its column.  Block (32, 4, 2) threads; sl is the CTA's dynamic
// shared memory, ZH x ZY x ZX values (layers k0-6 ..).  G and CARRY as for
// the xy pass; SC: the precision form (filters physical values, stored *
// isc(k), and stores them times sc(k)).  TMA (no carry, no scaling; rows a
// multiple of 16 bytes): the slab is one 32 x 4 x 44 x 1 tile of `map`
// (the input buffer as nx x ny x nz x V) from (x0, y0, k0 - 6, l), whose
// layout in shared memory is the slab's; it reads zero outside the grid,
// as the per-thread loads do, and x0 is a multiple of 32; sl must be
// 128-byte aligned and have 8 more bytes (the mbarrier).
template <class R, int G, bool CARRY, bool SC, bool TMA = false>
__device__ __forceinline__ void filt_z_slab(const FiltArgs<R> &F, int l, int x0, int y0,
                                            int k0, R *sl, const CUtensorMap *map = nullptr) {
  using namespace fb;
  constexpr bool M2 = G == 3;
  static_assert(!TMA || (!CARRY && !SC), "the tensor copy moves stored values only");
  const int tx = threadIdx.x, ty = threadIdx.y, tz = threadIdx.z;
  const int nx = F.nx, ny = F.ny, nz = F.nz;
  const long long NXY = (long long)nx * ny;
  const int gx = x0 + tx, gy = y0 + ty;
  const bool colok = gx < nx && gy < ny;
  // this thread's column; each thread loads layers q = tz, tz + 2, ...
  const R *icol = F.in + (long long)l * F.N + (colok ? (long long)gy * nx + gx : 0);
  if constexpr (TMA) {
    // the mbarrier follows the slab in the dynamic buffer (a static one
    // would cost a kilobyte of the CTA's shared allocation)
    unsigned long long &zbar = *(unsigned long long *)(sl + ZH * ZY * ZX);
    const bool lead = tx == 0 && ty == 0 && tz == 0;
    if (lead) {
      mbar_init_t(&zbar);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (lead) {
      mbar_tx_t(&zbar, (unsigned)(ZH * ZY * ZX * sizeof(R)));
      tma4d_t(sl, map, x0, y0, k0 - 6, l, &zbar);
    }
    const bool ok = mbar_wait_t(&zbar, 0u, F.err);
    if (!__syncthreads_and(ok)) {
      // gave up (error flag raised): wait, again bounded, for the copy
      // still in flight into this CTA's buffer, then leave
      if (lead) mbar_wait_t(&zbar, 0u, F.err);
      return;
    }
  } else {
    const R *ccol = CARRY ? F.carry + (icol - F.in) : nullptr;
    const R *isc = SC ? F.isc + l * nz : nullptr;
    for (int q = tz; q < ZH; q += 2) {
      const int gz = k0 - 6 + q;
      R v = R(0);
      if (colok && gz >= 0 && gz < nz) {
        v = icol[gz * NXY];
        if (CARRY) v = v - ccol[gz * NXY];
        if (SC) v = v * isc[gz];
      }
      sl[(q * ZY + ty) * ZX + tx] = v;
    }
    __syncthreads();
  }
  if (!colok) return;
  R *ocol = F.out + (icol - F.in);
  const R fs = F.s;
  const R *sc = SC ? F.sc + l * nz : nullptr;
  // this thread's layers [ka, kb); layer L sits at slab index L - (k0 - 6)
  const int ka = k0 + tz * ZL, kb = min(nz, ka + ZL);
  const R *wl = sl + ((ka - k0) * ZY + ty) * ZX + tx;  // raw(ka - 6) ..
  if (kb - ka == ZL && ka - 6 >= G && kb + 5 <= nz - G - 1) {
    // every layer away from the edges: no pre-average, no edge rule; the
    // window is unrolled, so its values are named registers
    R w[ZL + 12];
#pragma unroll
    for (int m = 6 - G; m < ZL + 6 + G; ++m) w[m] = wl[m * ZY * ZX];
#pragma unroll
    for (int j = 0; j < ZL; ++j) {
      R s = R(0);
#pragma unroll
      for (int m = 0; m <= 2 * G; ++m) s += w[j + 6 - G + m] * fcoef<R>(G == 5 ? 0 : 1, m);
      R r = M2 ? w[j + 6] - fs * s : s;
      if (SC) r = r * sc[ka + j];
      ocol[(ka + j) * NXY] = r;
    }
    return;
  }
  auto in_avg = [&](int q) { return (q >= 1 && q <= G - 1) || (q >= nz - G && q <= nz - 2); };
  R w[13];  // w[m] = raw(k - 6 + m)
#pragma unroll
  for (int m = 0; m < 13; ++m) w[m] = wl[m * ZY * ZX];
  for (int k = ka; k < kb; ++k) {
    auto pre = [&](int m) -> R {
      return in_avg(k - 6 + m) ? (w[m + 1] + w[m - 1]) / R(2) : w[m];
    };
    const R pq = pre(6);
    R filt;
    if (k < G || k >= nz - G) {
      filt = pq;
    } else if (k - 6 >= G && k + 6 <= nz - G - 1) {
      R s = R(0);
#pragma unroll
      for (int m = 0; m <= 2 * G; ++m) s += w[6 - G + m] * fcoef<R>(G == 5 ? 0 : 1, m);
      filt = s;
    } else {
      R s = R(0);
#pragma unroll
      for (int m = 0; m <= 2 * G; ++m) s += pre(6 - G + m) * fcoef<R>(G == 5 ? 0 : 1, m);
      filt = s;
    }
    R r = M2 ? pq - fs * filt : filt;
    if (SC) r = r * sc[k];
    ocol[k * NXY] = r;
#pragma unroll
    for (int m = 0; m < 12; ++m) w[m] = w[m + 1];
    if (k + 1 < kb) w[12] = wl[(k + 13 - ka) * ZY * ZX];  // raw(k + 7)
  }
}

}  // namespace sparc
