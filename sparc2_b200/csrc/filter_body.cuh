// filter_body.cuh -- FILTER_VARS (derivatives.f90:659-703) as two kernels
// per filter event, shared by the plain form (R = double, step.cu) and the
// precision form (R = float, step32.cu).
//
//   * xy (nn % xyfreq == 0): one fused pass per layer tile.  A CTA loads a
//     (32+12) x (32+12) tile of one field's layer into shared memory, forms
//     the y pre-average of the non-periodic edge rows (derivatives.f90:671-
//     675), the y filter of filty (derivatives.f90:345-447) with its edge
//     rows (copy-through for the 11-point filter, zero for the 7-point one)
//     and the mode-2 combination a - s*filt, then the x pre-average
//     (derivatives.f90:680-684), the x filter and its combination, and
//     writes the tile once.  The reference's y-then-x order is kept.
//   * z (nn % zfreq == 0): a CTA loads a slab of 32 x 4 columns of one field
//     over 64 layers and their 6-layer margins into shared memory, every
//     load in flight at once; each thread then runs a 13-deep register
//     window of raw values down its column for 32 layers (the pre-average of
//     derivatives.f90:690-693 needs the neighbours of the 11 taps).
//     filtz's edge layers are copied through (derivatives.f90:610-633).
//
// No 64-bit division or modulo per element: tile and column coordinates
// come from the launch geometry.  In the precision form the stored state
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

namespace sparc {

template <class R>
__device__ __forceinline__ R fcoef(int table, int m);

// dynamic shared memory of the z pass (one slab)
template <class R>
constexpr size_t filt_z_smem() {
  return (size_t)(64 + 12) * 4 * 32 * sizeof(R);
}

template <class R>
struct FiltArgs {
  int nx, ny, nz, V;
  long long N;
  int periodic;
  int g;          // half-width of the event's filter (5: 11-point, 3: 7-point)
  int mode2;      // a - s*filt (7-point) instead of filt
  R s;
  const R *in;
  R *out;
  const R *carry;  // compensation subtracted on load (first pass), or null
  const R *sc, *isc;  // depth scales V x nz (precision form z pass), or null
};

namespace fb {
constexpr int TX = 32, TY = 8;           // threads of the xy pass (32 x 8)
constexpr int TR = 32;                    // rows of an xy tile (4 per thread)
constexpr int RX = TX + 12, RY = TR + 12, PY = TR + 10;
constexpr int ZX = 32, ZY = 4, ZC = 64;   // z pass: 32 x 4 columns x 64 layers
constexpr int ZH = ZC + 12;               // layers loaded per z slab
}  // namespace fb

__device__ __forceinline__ int fmod_idx(int q, int n) {
  q %= n;
  return q < 0 ? q + n : q;
}

// 11 or 7 taps of the filter at centre p of a strided row
template <class R>
__device__ __forceinline__ R ftaps(const R *p, int st, int g) {
  R s = R(0);
  if (g == 5) {
#pragma unroll
    for (int m = 0; m < 11; ++m) s += p[(m - 5) * st] * fcoef<R>(0, m);
  } else {
#pragma unroll
    for (int m = 0; m < 7; ++m) s += p[(m - 3) * st] * fcoef<R>(1, m);
  }
  return s;
}

// The fused y-then-x pass over the 32 x 32 tile (x0, y0) of layer k of
// field l; block (TX, TY) threads, each serving rows ty, ty + 8, ...
template <class R>
__device__ __forceinline__ void filt_xy_tile(const FiltArgs<R> &F, int l, int k, int x0,
                                             int y0) {
  using namespace fb;
  __shared__ R raw[RY][RX];  // rows y0-6 .., columns x0-6 ..
  __shared__ R pre[PY][RX];  // y pre-averaged rows y0-5 .. (edge tiles only)
  __shared__ R fy[TR][RX];   // after the y pass, rows y0 .., columns x0-6 ..
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int nx = F.nx, ny = F.ny, g = F.g;
  const bool per = F.periodic;
  const long long base = (long long)l * F.N + (long long)k * nx * ny;
  // rows in groups of RX columns: lanes walk a row, warps the rows
  for (int ry = ty; ry < RY; ry += TY) {
    int gy = y0 - 6 + ry;
    bool oky = true;
    if (per) gy = fmod_idx(gy, ny);
    else oky = gy >= 0 && gy < ny;
    for (int rx = tx; rx < RX; rx += TX) {
      int gx = x0 - 6 + rx;
      bool ok = oky;
      if (per) gx = fmod_idx(gx, nx);
      else ok = ok && gx >= 0 && gx < nx;
      R v = R(0);
      if (ok) {
        const long long id = base + (long long)gy * nx + gx;
        v = F.in[id];
        if (F.carry) v = v - F.carry[id];
      }
      raw[ry][rx] = v;
    }
  }
  __syncthreads();
  // y pre-average of rows 1..g-1 and ny-g..ny-2 (non-periodic), only on
  // tiles whose y window reaches such a row
  const bool ypre = !per && (y0 - 5 <= g - 1 || y0 + TR + 4 >= ny - g);
  if (ypre) {
    for (int py = ty; py < PY; py += TY) {
      const int gy = y0 - 5 + py;
      const bool avg = (gy >= 1 && gy <= g - 1) || (gy >= ny - g && gy <= ny - 2);
      for (int rx = tx; rx < RX; rx += TX)
        pre[py][rx] = avg ? (raw[py + 2][rx] + raw[py][rx]) / R(2) : raw[py + 1][rx];
    }
    __syncthreads();
  }
  // the y pass of the tile's rows over every loaded column
  for (int r = ty; r < TR; r += TY) {
    const int gyo = y0 + r;
    const bool yedge = !per && (gyo < g || gyo >= ny - g);
    for (int rx = tx; rx < RX; rx += TX) {
      const R *c = ypre ? &pre[r + 5][rx] : &raw[r + 6][rx];
      const R pq = *c;
      const R filt = yedge ? (g == 3 ? R(0) : pq) : ftaps(c, RX, g);
      fy[r][rx] = F.mode2 ? pq - F.s * filt : filt;
    }
  }
  __syncthreads();
  // the x pre-average (on the fly) and the x pass at the tile's own columns
  const int gxo = x0 + tx;
  if (gxo >= nx) return;
  const bool xpre = !per && (x0 - 5 <= g - 1 || x0 + TX + 4 >= nx - g);
  const bool xedge = !per && (gxo < g || gxo >= nx - g);
  const int c0 = tx + 6;
  for (int r = ty; r < TR; r += TY) {
    const int gyo = y0 + r;
    if (gyo >= ny) break;
    auto px = [&](int c) -> R {  // x pre-averaged value at loaded column c
      const int gx = x0 - 6 + c;
      if ((gx >= 1 && gx <= g - 1) || (gx >= nx - g && gx <= nx - 2))
        return (fy[r][c + 1] + fy[r][c - 1]) / R(2);
      return fy[r][c];
    };
    R pq, filt;
    if (!xpre) {
      pq = fy[r][c0];
      filt = ftaps(&fy[r][c0], 1, g);
    } else {
      pq = px(c0);
      if (xedge) {
        filt = g == 3 ? R(0) : pq;
      } else {
        R s = R(0);
        if (g == 5) {
#pragma unroll
          for (int m = 0; m < 11; ++m) s += px(c0 - 5 + m) * fcoef<R>(0, m);
        } else {
#pragma unroll
          for (int m = 0; m < 7; ++m) s += px(c0 - 3 + m) * fcoef<R>(1, m);
        }
        filt = s;
      }
    }
    F.out[base + (long long)gyo * nx + gxo] = F.mode2 ? pq - F.s * filt : filt;
  }
}

// The z pass of a slab of 32 x 4 columns and ZC layers from k0 of field l:
// the slab and its 6-layer margins are loaded into shared memory in one go
// (every load in flight at once), then each thread runs a register window
// down its column for half of the layers.  Block (32, 4, 2) threads; sl is
// the CTA's dynamic shared memory, ZH x ZY x ZX values (layers k0-6 ..).
template <class R>
__device__ __forceinline__ void filt_z_slab(const FiltArgs<R> &F, int l, int x0, int y0,
                                            int k0, R *sl) {
  using namespace fb;
  const int tx = threadIdx.x, ty = threadIdx.y, tz = threadIdx.z;
  const int tid = (tz * ZY + ty) * ZX + tx;
  const int nx = F.nx, ny = F.ny, nz = F.nz, g = F.g;
  const long long NXY = (long long)nx * ny;
  const long long fb0 = (long long)l * F.N;
  const bool sc = F.isc != nullptr;
  for (int t = tid; t < ZH * ZY * ZX; t += 2 * ZY * ZX) {
    const int x = t % ZX, y = (t / ZX) % ZY, q = t / (ZX * ZY);
    const int gx = x0 + x, gy = y0 + y, gz = k0 - 6 + q;
    R v = R(0);
    if (gx < nx && gy < ny && gz >= 0 && gz < nz) {
      const long long id = fb0 + gz * NXY + (long long)gy * nx + gx;
      v = F.in[id];
      if (F.carry) v = v - F.carry[id];
      if (sc) v = v * F.isc[l * nz + gz];
    }
    sl[(q * ZY + y) * ZX + x] = v;
  }
  __syncthreads();
  const int gx = x0 + tx, gy = y0 + ty;
  if (gx >= nx || gy >= ny) return;
  const long long col = fb0 + (long long)gy * nx + gx;
  // this thread's layers [ka, kb)
  const int ka = k0 + tz * (ZC / 2), kb = min(nz, ka + ZC / 2);
  auto in_avg = [&](int q) { return (q >= 1 && q <= g - 1) || (q >= nz - g && q <= nz - 2); };
  // layer L sits at slab index L - (k0 - 6)
  R w[13];  // w[m] = raw(k - 6 + m)
#pragma unroll
  for (int m = 0; m < 13; ++m) w[m] = sl[((ka - k0 + m) * ZY + ty) * ZX + tx];
  for (int k = ka; k < kb; ++k) {
    auto pre = [&](int m) -> R {
      return in_avg(k - 6 + m) ? (w[m + 1] + w[m - 1]) / R(2) : w[m];
    };
    const R pq = pre(6);
    R filt;
    if (k < g || k >= nz - g) {
      filt = pq;
    } else if (k - 6 >= g && k + 6 <= nz - g - 1) {
      R s = R(0);
      if (g == 5) {
#pragma unroll
        for (int m = 0; m < 11; ++m) s += w[1 + m] * fcoef<R>(0, m);
      } else {
#pragma unroll
        for (int m = 0; m < 7; ++m) s += w[3 + m] * fcoef<R>(1, m);
      }
      filt = s;
    } else {
      R s = R(0);
      if (g == 5) {
#pragma unroll
        for (int m = 0; m < 11; ++m) s += pre(1 + m) * fcoef<R>(0, m);
      } else {
#pragma unroll
        for (int m = 0; m < 7; ++m) s += pre(3 + m) * fcoef<R>(1, m);
      }
      filt = s;
    }
    R r = F.mode2 ? pq - F.s * filt : filt;
    if (sc) r = r * F.sc[l * nz + k];
    F.out[col + k * NXY] = r;
#pragma unroll
    for (int m = 0; m < 12; ++m) w[m] = w[m + 1];
    if (k + 1 < kb) w[12] = sl[((k + 13 - k0) * ZY + ty) * ZX + tx];  // raw(k + 7)
  }
}

}  // namespace sparc
