// filter_body.cuh -- FILTER_VARS (derivatives.f90:659-703) as two kernels
// per filter event, shared by the plain form (R = double, step.cu) and the
// precision form (R = float, step32.cu).
//
//   * xy (nn % xyfreq == 0): one fused pass per layer tile.  A CTA loads a
//     (TX+12) x (TY+12) tile of one field's layer into shared memory, forms
//     the y pre-average of the non-periodic edge rows (derivatives.f90:671-
//     675), the y filter of filty (derivatives.f90:345-447) with its edge
//     rows (copy-through for the 11-point filter, zero for the 7-point one)
//     and the mode-2 combination a - s*filt, then the x pre-average
//     (derivatives.f90:680-684), the x filter and its combination, and
//     writes the tile once.  The reference's y-then-x order is kept.
//   * z (nn % zfreq == 0): each thread marches one (x, y) column of one
//     field up the whole depth with a 13-deep register window of raw values
//     (the pre-average of derivatives.f90:690-693 needs the neighbours of
//     the 11 taps); loads are issued a block of ZB layers ahead so that
//     ZB loads per thread are in flight.  filtz's edge layers are copied
//     through (derivatives.f90:610-633).
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
constexpr int TX = 32, TY = 8, RX = TX + 12, RY = TY + 12, PY = TY + 10;
constexpr int ZB = 8;  // z pass: layers per load block
}  // namespace fb

__device__ __forceinline__ int fmod_idx(int q, int n) {
  q %= n;
  return q < 0 ? q + n : q;
}

// 11 or 7 taps of the filter at centre index c of a strided row p
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

// The fused y-then-x pass over the TX x TY tile (x0, y0) of layer k of
// field l; block (TX, TY) threads.
template <class R>
__device__ __forceinline__ void filt_xy_tile(const FiltArgs<R> &F, int l, int k, int x0,
                                             int y0) {
  using namespace fb;
  __shared__ R raw[RY][RX];  // rows y0-6 .., columns x0-6 ..
  __shared__ R pre[PY][RX];  // y pre-averaged rows y0-5 ..
  __shared__ R fy[TY][RX];   // after the y pass, rows y0 .., columns x0-6 ..
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int nx = F.nx, ny = F.ny, g = F.g;
  const bool per = F.periodic;
  const long long base = (long long)l * F.N + (long long)k * nx * ny;
  for (int t = tid; t < RY * RX; t += TX * TY) {
    const int ry = t / RX, rx = t - ry * RX;
    int gx = x0 - 6 + rx, gy = y0 - 6 + ry;
    bool ok = true;
    if (per) {
      gx = fmod_idx(gx, nx);
      gy = fmod_idx(gy, ny);
    } else {
      ok = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
    }
    R v = R(0);
    if (ok) {
      const long long id = base + (long long)gy * nx + gx;
      v = F.in[id];
      if (F.carry) v = v - F.carry[id];
    }
    raw[ry][rx] = v;
  }
  __syncthreads();
  // y pre-average of rows 1..g-1 and ny-g..ny-2 (non-periodic)
  for (int t = tid; t < PY * RX; t += TX * TY) {
    const int py = t / RX, rx = t - py * RX;
    const int gy = y0 - 5 + py;
    R v = raw[py + 1][rx];
    if (!per && ((gy >= 1 && gy <= g - 1) || (gy >= ny - g && gy <= ny - 2)))
      v = (raw[py + 2][rx] + raw[py][rx]) / R(2);
    pre[py][rx] = v;
  }
  __syncthreads();
  // y filter of the tile's rows over every loaded column
  const int gyo = y0 + ty;
  const bool yedge = !per && (gyo < g || gyo >= ny - g);
  for (int rx = tx; rx < RX; rx += TX) {
    const R pq = pre[ty + 5][rx];
    const R filt = yedge ? (g == 3 ? R(0) : pq) : ftaps(&pre[ty + 5][rx], RX, g);
    fy[ty][rx] = F.mode2 ? pq - F.s * filt : filt;
  }
  __syncthreads();
  // x pre-average and x filter at the tile's own columns
  const int gxo = x0 + tx;
  if (gxo >= nx || gyo >= ny) return;
  auto px = [&](int c) -> R {  // x pre-averaged value at loaded column c
    const int gx = x0 - 6 + c;
    if (!per && ((gx >= 1 && gx <= g - 1) || (gx >= nx - g && gx <= nx - 2)))
      return (fy[ty][c + 1] + fy[ty][c - 1]) / R(2);
    return fy[ty][c];
  };
  const int c0 = tx + 6;
  const R pq = px(c0);
  R filt;
  if (!per && (gxo < g || gxo >= nx - g)) {
    filt = g == 3 ? R(0) : pq;
  } else if (per || (x0 - 6 >= g && x0 + TX + 6 <= nx - g)) {
    filt = ftaps(&fy[ty][c0], 1, g);  // no pre-averaged column in reach
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
  F.out[base + (long long)gyo * nx + gxo] = F.mode2 ? pq - F.s * filt : filt;
}

// The z pass of column (i, j) of field l: every layer, marching up with a
// register window raw(k-6 .. k+6) and the next ZB layers loaded a block
// ahead.
template <class R>
__device__ __forceinline__ void filt_z_column(const FiltArgs<R> &F, int l, int i, int j) {
  using namespace fb;
  const int nz = F.nz, g = F.g;
  const long long NXY = (long long)F.nx * F.ny;
  const long long col = (long long)l * F.N + (long long)j * F.nx + i;
  const bool sc = F.isc != nullptr;
  auto load = [&](int q) -> R {  // physical raw value at layer q (0 outside)
    if (q < 0 || q >= nz) return R(0);
    const long long id = col + q * NXY;
    R v = __ldg(F.in + id);
    if (F.carry) v = v - __ldg(F.carry + id);
    return sc ? v * __ldg(F.isc + l * nz + q) : v;
  };
  R w[13];
#pragma unroll
  for (int m = 0; m < 13; ++m) w[m] = load(m - 6);
  R nxt[ZB];
#pragma unroll
  for (int u = 0; u < ZB; ++u) nxt[u] = load(7 + u);
  auto in_avg = [&](int q) { return (q >= 1 && q <= g - 1) || (q >= nz - g && q <= nz - 2); };
  for (int kb = 0; kb < nz; kb += ZB) {
    R cur[ZB];
#pragma unroll
    for (int u = 0; u < ZB; ++u) cur[u] = nxt[u];
#pragma unroll
    for (int u = 0; u < ZB; ++u) nxt[u] = load(kb + ZB + 7 + u);  // next block, in flight
#pragma unroll
    for (int u = 0; u < ZB; ++u) {
      const int k = kb + u;
      if (k >= nz) break;
      // w[m] = raw(k - 6 + m)
      auto pre = [&](int m) -> R {  // pre-averaged value at layer k - 6 + m
        const int q = k - 6 + m;
        return in_avg(q) ? (w[m + 1] + w[m - 1]) / R(2) : w[m];
      };
      const R pq = pre(6);
      R filt;
      if (k < g || k >= nz - g) {
        filt = pq;
      } else if (k - 6 >= g && k + 6 <= nz - g - 1) {
        // no pre-averaged layer among the taps
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
      if (sc) r = r * __ldg(F.sc + l * nz + k);
      F.out[col + k * NXY] = r;
#pragma unroll
      for (int m = 0; m < 12; ++m) w[m] = w[m + 1];
      w[12] = cur[u];
    }
  }
}

}  // namespace sparc
