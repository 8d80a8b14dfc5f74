// step32.cu -- the precision form of the time step: FP32 state, coefficients
// and arithmetic (FP32 accumulation), FP64 only for the setup (setup.cu),
// the CPML profiles (computed in FP64, stored in FP32) and the energy
// diagnostics.
//
// Depth scaling.  The state is stored as sc_l(z) * physical value with
//   rho: 1/rho0(z), v: sqrt(rho0(z)), p: 1/(rho0 c0^2)(z), b: 1,
// profiles of the background column (1,1,:), so that wave amplitudes keep
// the same magnitude across the ~1e6 density stratification.  Kernels turn
// stored values into physical ones on load (x/y derivatives of a layer are
// scaled once after the stencil; z windows hold physical values) and scale
// the right-hand side back on store.
//
// Compensated update.  The final RK update a + deltat*F (step.f90:58) keeps
// a per-value FP32 carry (Kahan summation), so the slow accumulation of
// small increments onto the state does not lose the low-order digits.
//
// The stencils, CPML, RHS algebra, boundary zeroing and diagnostics follow
// the same reference lines as the FP64 kernels of step.cu.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "filter_body.cuh"
#include "mhd_body.cuh"
#include "random_forcing.cuh"

namespace sparc {

__constant__ float f_dp[6][11];
__constant__ float f_df[2][11];


// Derivative rows and both filter stencils ([0] 11-point, [1] 7-point) in
// FP32; a filter pass picks its table by half-width.
int step32_constants() {
  float t[6][11];
  for (int r = 0; r < 6; ++r)
    for (int m = 0; m < 11; ++m) t[r][m] = (float)kDerivRows[r][m];
  if (cudaMemcpyToSymbol(f_dp, t, sizeof(t)) != cudaSuccess) return SPARC_ERR_CUDA;
  float f[2][11] = {};
  for (int m = 0; m < 11; ++m) f[0][m] = (float)kFilter11[m];
  for (int m = 0; m < 7; ++m) f[1][m] = (float)kFilter7[m];
  return cudaMemcpyToSymbol(f_df, f, sizeof(f)) == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

template <>
__device__ __forceinline__ float dcoef<float>(int r, int m) {
  return f_dp[r][m];
}
template <>
__device__ __forceinline__ float fcoef<float>(int t, int m) {
  return f_df[t][m];
}

using Sim32 = SimT<float>;
using Face32 = FaceT<float>;

// ------------------------------------------------------------- helpers
__device__ __forceinline__ int wrap32(int q, int n) {
  q = q < 0 ? q + n : q;
  return q >= n ? q - n : q;
}
__device__ __forceinline__ int origin32(int t0, int T, int n, bool per) {
  int o = t0 - 5;
  if (!per && t0 + T >= n) o = min(o, n - 11);
  return o;
}

template <int MODE>
__device__ __forceinline__ void cpml32(const Face32 &F, long long f, int layer, int slot,
                                       float beta, float dt, float &d) {
  const long long pf = F.uniform ? (long long)layer : f;
  const float pa = __ldg(F.pa + pf), pb = __ldg(F.pb + pf), pki = __ldg(F.pki + pf);
  const long long o = (long long)slot * F.cnt + f;
  const float v = F.vars[o];
  float psi = v;
  if (MODE != F_FIRST) psi = v + beta * F.scr[o];
  const float rhs = pa * d + pb * psi;
  d = d * pki + psi;
  if (MODE == F_LAST) F.vars[o] = v + dt * rhs;
  else F.scr[o] = rhs;
}

__device__ __forceinline__ float pulse_time32(const Sim32 &S, long long it) {
  const ForcingT<float> &F = S.frc;
  if (F.kind != SPARC_SRC_PULSE) return 0.f;
  const double t = (double)it * F.timestep;
  double T = F.amp_c * sin(2.0 * PI * (t - F.t1 + 2.0 * F.t0) / F.t0);
  return (float)(T * exp(-1.0 * ((t - F.t1) * (t - F.t1)) / (2.0 * (F.st * F.st))));
}

__device__ __forceinline__ float forcing32(const Sim32 &S, float T, int i, int j, int k) {
  const ForcingT<float> &F = S.frc;
  if (F.kind == SPARC_SRC_PULSE)
    return T * __ldg(F.fz + k) * (__ldg(F.fy + j) * __ldg(F.fx + i));
  if (F.kind == SPARC_SRC_PSR && k >= F.klo && k < F.khi)
    return F.psr[((long long)(k - F.klo) * S.ny + j) * S.nx + i];
  if (F.kind == SPARC_SRC_RANDOM) return F.f2d[(long long)j * S.nx + i] * __ldg(F.sdep + k);
  return 0.f;
}

template <class Get>
__device__ __forceinline__ float dxy32(int q, int n, bool per, float sc, Get t) {
  float s = 0.f;
  if (per || (q >= 5 && q < n - 5)) {
#pragma unroll
    for (int m = 0; m < 11; ++m) s += t(q - 5 + m) * f_dp[5][m];
    return sc * s;
  }
  if (q < 5) {
#pragma unroll
    for (int m = 0; m < 11; ++m) s += t(m) * f_dp[q][m];
    return sc * s;
  }
  const int row = n - 1 - q;
#pragma unroll
  for (int m = 0; m < 11; ++m) s += t(n - 1 - m) * f_dp[row][m];
  return -sc * s;
}

__device__ __forceinline__ float dz32(const float (&w)[11], int k, int nz, float sc) {
  float s = 0.f;
  if (k < nz - 5) {
    const float d1 = w[6] - w[4], d2 = w[7] - w[3], d3 = w[8] - w[2], d4 = w[9] - w[1],
                d5 = w[10] - w[0];
    const float a = fmaf(f_dp[5][8], d3, fmaf(f_dp[5][10], d5, f_dp[5][6] * d1));
    const float b = fmaf(f_dp[5][9], d4, f_dp[5][7] * d2);
    return sc * (a + b);
  }
  const int row = nz - 1 - k;
#pragma unroll
  for (int m = 0; m < 11; ++m) s += w[10 - m] * f_dp[row][m];
  return -sc * s;
}

__device__ __forceinline__ void shift32(float (&w)[11], float v) {
#pragma unroll
  for (int m = 0; m < 10; ++m) w[m] = w[m + 1];
  w[10] = v;
}

// Per-CTA partial of the KE norm and minima (FP64) and the last-CTA
// reduction with the fail criterion of driver.f90:175-183.
// bid/nb: this block's index and the block count of the logical grid (a
// stage split over several launches shares one logical grid).
__device__ void diag_reduce32(const Sim32 &S, double ke, double mr, double mp, long long bid,
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

// ------------------------------------------ MP_QUIET_3D, precision form
// RHS.f90:18-175 fused with one RK stage (as k_stage_quiet of step.cu),
// FP32 with depth-scaled state.  Field scales: l = 0 rho, 1-3 v, 4 p.
// The body covers the tile (x0, y0) of TX x TY columns over layers
// [k0, k1); (tx, ty) is the calling thread's column in the tile.  Every
// thread of the block calls it.  Diagnostics of the last stage accumulate
// into ke, mr, mp.
template <int TX, int TY, int MODE, bool BG1D>
__device__ __forceinline__ void quiet_body(const Sim32 &S, const float *__restrict__ a,
                                           const float *__restrict__ tin,
                                           float *__restrict__ so, float beta, float bnext,
                                           int x0, int y0, int k0, int k1, int tx, int ty,
                                           float *zt, double &ke, double &mr, double &mp) {
  constexpr int HX = TX + 10, HY = TY + 10;
  __shared__ float t_vx[HY][HX], t_vy[HY][HX], t_p[HY][HX];
  const int tid = ty * TX + tx;
  const int nx = S.nx, ny = S.ny, nz = S.nz;
  const long long N = S.N, NXY = (long long)nx * ny;
  const int i = x0 + tx, j = y0 + ty;
  const bool act = i < nx && j < ny;
  const bool per = S.periodic;
  const long long col = (long long)j * nx + i;
  const long long it = *S.iter;
  const float Tp = pulse_time32(S, it);
  const float dt = (float)S.deltat;
  const int gc = act ? S.colx[i] + S.bxdim * S.coly[j] : 0;
  const int xo = origin32(x0, TX, nx, per), yo = origin32(y0, TY, ny, per);
  const int cx0 = x0 - xo, cy0 = y0 - yo;
  // depth scales of the layers this chunk touches, staged in shared memory
  // (zt: 16 floats per layer, 1/sc of the 5 fields then sc)
  const int zb = max(0, min(k0 - 5, nz - 11));
  {
    const int ze = min(nz, max(k1 + 5, zb + 11));
    for (int t = tid; t < (ze - zb) * 16; t += TX * TY) {
      const int kk = zb + (t >> 4), l = t & 15;
      zt[t] = l < 5 ? S.isc[l * nz + kk] : (l >= 8 && l < 13 ? S.sc[(l - 8) * nz + kk] : 0.f);
    }
  }
  __syncthreads();
  auto isc_ = [&](int l, int kk) { return zt[(kk - zb) * 16 + l]; };
  auto sc_ = [&](int l, int kk) { return zt[(kk - zb) * 16 + 8 + l]; };

  float wvz[11], wp[11];  // physical values
  const int b0 = min(k0 - 5, nz - 11);
#pragma unroll
  for (int m = 0; m < 11; ++m) {
    const int kk = b0 + m;
    const bool ok = act && kk >= 0;
    const long long id = (long long)kk * NXY + col;
    wvz[m] = ok ? __ldg(tin + 3 * N + id) * isc_(3, kk) : 0.f;
    wp[m] = ok ? __ldg(tin + 4 * N + id) * isc_(4, kk) : 0.f;
  }

  for (int k = k0; k < k1; ++k) {
    if (k > k0 && k <= nz - 6) {
      const long long id = (long long)(k + 5) * NXY + col;
      shift32(wvz, act ? __ldg(tin + 3 * N + id) * isc_(3, k + 5) : 0.f);
      shift32(wp, act ? __ldg(tin + 4 * N + id) * isc_(4, k + 5) : 0.f);
    }
    const long long kb = (long long)k * NXY;
    __syncthreads();
    for (int t = tid; t < HY * HX; t += TX * TY) {
      const int ly = t / HX, lx = t - ly * HX;
      const bool inx = lx >= cx0 && lx < cx0 + TX, iny = ly >= cy0 && ly < cy0 + TY;
      if (!inx && !iny) continue;
      int gx = xo + lx, gy = yo + ly;
      bool ok;
      if (per) {
        gx = wrap32(gx, nx);
        gy = wrap32(gy, ny);
        ok = true;
      } else {
        ok = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
      }
      const long long id = kb + (long long)gy * nx + gx;
      if (iny) t_vx[ly][lx] = ok ? __ldg(tin + N + id) : 0.f;
      if (inx) t_vy[ly][lx] = ok ? __ldg(tin + 2 * N + id) : 0.f;
      t_p[ly][lx] = ok ? __ldg(tin + 4 * N + id) : 0.f;
    }
    __syncthreads();
    if (!act) continue;
    const long long id = kb + col;
    float isv[5], scv[5];
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      isv[l] = isc_(l, k);
      scv[l] = sc_(l, k);
    }
    float av[5], tv[5];
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      const float st = __ldg(tin + l * N + id);
      av[l] = MODE == F_FIRST ? st : __ldg(a + l * N + id);
      tv[l] = st * isv[l];
    }
    const float rho = tv[0], vx = tv[1], vy = tv[2], vz = tv[3], p = tv[4];
    const int ry = cy0 + ty, rx = cx0 + tx;
    const float sx = (float)S.stretchx, sy = (float)S.stretchy;
    float dvxdx = isv[1] * dxy32(i, nx, per, sx, [&](int g) { return t_vx[ry][g - xo]; });
    float gpx = isv[4] * dxy32(i, nx, per, sx, [&](int g) { return t_p[ry][g - xo]; });
    float dvydy = isv[2] * dxy32(j, ny, per, sy, [&](int g) { return t_vy[g - yo][rx]; });
    float gpy = isv[4] * dxy32(j, ny, per, sy, [&](int g) { return t_p[g - yo][rx]; });
    const float szk = __ldg(S.stretch + k);
    float dvzdz = dz32(wvz, k, nz, szk);
    float gpz = dz32(wp, k, nz, szk);
    if (k < S.zb.np) {
      const long long f = kb + col;
      cpml32<MODE>(S.zb, f, k, 1, beta, dt, gpz);
      cpml32<MODE>(S.zb, f, k, 0, beta, dt, dvzdz);
    } else if (S.zt.on && k >= nz - S.zt.np) {
      const int kl = k - (nz - S.zt.np);
      const long long f = (long long)kl * NXY + col;
      cpml32<MODE>(S.zt, f, kl, 1, beta, dt, gpz);
      cpml32<MODE>(S.zt, f, kl, 0, beta, dt, dvzdz);
    }
    if (S.xb.on) {
      if (i < S.xb.np) {
        const long long f = i + (long long)S.xb.np * (j + (long long)ny * k);
        cpml32<MODE>(S.xb, f, i, 1, beta, dt, gpx);
        cpml32<MODE>(S.xb, f, i, 0, beta, dt, dvxdx);
      } else if (i >= nx - S.xt.np) {
        const int il = i - (nx - S.xt.np);
        const long long f = il + (long long)S.xt.np * (j + (long long)ny * k);
        cpml32<MODE>(S.xt, f, il, 1, beta, dt, gpx);
        cpml32<MODE>(S.xt, f, il, 0, beta, dt, dvxdx);
      }
      if (j < S.yb.np) {
        const long long f = i + (long long)nx * (j + (long long)S.yb.np * k);
        cpml32<MODE>(S.yb, f, j, 1, beta, dt, gpy);
        cpml32<MODE>(S.yb, f, j, 0, beta, dt, dvydy);
      } else if (j >= ny - S.yt.np) {
        const int jl = j - (ny - S.yt.np);
        const long long f = i + (long long)nx * (jl + (long long)S.yt.np * k);
        cpml32<MODE>(S.yt, f, jl, 1, beta, dt, gpy);
        cpml32<MODE>(S.yt, f, jl, 0, beta, dt, dvydy);
      }
    }
    const long long bi = BG1D ? (long long)k : id;
    const float r0 = __ldg(S.rho0 + bi), ri = __ldg(S.rhoinv + bi),
                c2r = __ldg(S.c2rho0 + bi), grz = __ldg(S.grz + bi),
                gp0 = __ldg(S.gpz + bi), sg = __ldg(S.sponge + bi);
    const float gk = __ldg(S.gblk + (long long)gc * nz + k);
    const float div = dvxdx + dvydy + dvzdz;
    float R[5];
    R[0] = -grz * vz - r0 * div - sg * rho;
    R[1] = -ri * gpx - sg * vx;
    R[2] = -ri * gpy - sg * vy;
    R[3] = -ri * (gpz + rho * gk) - vz * sg;
    if (S.frc.kind != SPARC_SRC_NONE) {
      const float frc = forcing32(S, Tp, i, j, k);
      if (S.frc.dir == 1) R[1] = R[1] + frc;
      else if (S.frc.dir == 2) R[2] = R[2] + frc;
      else R[3] = R[3] + frc;
    }
    R[4] = -c2r * div - vz * gp0 - sg * p;
    const bool zero = k == 0 || k == nz - 1 ||
                      (!per && (i == 0 || i == nx - 1 || j == 0 || j == ny - 1));
    if (MODE == F_LAST) {
      double an[5];
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        float c = S.carry[l * N + id];
        const float t = zero ? av[l] : kahan(av[l], dt * (scv[l] * R[l]), c);
        so[l * N + id] = t;
        S.carry[l * N + id] = c;
        an[l] = ((double)t - (double)c) * (double)isv[l];
      }
      const double p0v = __ldg(S.p0 + bi);
      double m = ((double)r0 + an[0]) * (an[1] * an[1] + an[2] * an[2] + an[3] * an[3]) / 2.0;
      ke += m * m;
      mr = fmin(mr, (double)rho + (double)r0);
      mp = fmin(mp, (double)p + p0v);
    } else {
#pragma unroll
      for (int l = 0; l < 5; ++l)
        so[l * N + id] = zero ? av[l] : av[l] + bnext * (scv[l] * R[l]);
    }
  }
}

template <int TX, int TY, int MODE, bool BG1D>
__global__ void __launch_bounds__(TX *TY)
    k_quiet32(const Sim32 S, const float *__restrict__ a, const float *__restrict__ tin,
              float *__restrict__ so, float beta, float bnext, int zchunk) {
  extern __shared__ __align__(1024) float smem_raw32[];  // the depth-scale table
  double ke = 0.0, mr = 1e300, mp = 1e300;
  const int k0 = blockIdx.z * zchunk;
  quiet_body<TX, TY, MODE, BG1D>(S, a, tin, so, beta, bnext, blockIdx.x * TX, blockIdx.y * TY,
                                 k0, min(S.nz, k0 + zchunk), threadIdx.x, threadIdx.y, smem_raw32,
                                 ke, mr, mp);
  if (MODE == F_LAST)
    diag_reduce32(S, ke, mr, mp,
                  blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z),
                  (long long)gridDim.x * gridDim.y * gridDim.z);
}

// -------------------------------------------- MP_MHD_3D, precision form
// The two-role body of mhd_body.cuh in FP32 with depth scaling (field
// scales: 0 rho, 1-3 v, 4 p, 5-7 b), one row of columns per thread: a CTA
// of 512 threads owns a 32 x 8 column tile.  Own-point arrays of a layer
// arrive by TMA (32x8 FP32 boxes), halos by cp.async; one CTA per SM.  (Two
// rows per thread measured 30 % slower on the 256x256x300 flux tube: the
// register spills of the doubled windows land in L2, the shared-memory
// carve-out leaving little L1.)

namespace t32 {
using namespace mg;
constexpr int TYT = TY;  // tile rows
using MB = MhdBuf<float, false>;
}  // namespace t32

// One RK stage of the MHD equations.  A stage is two launches over one
// logical grid of (x tile, y tile, z chunk) blocks: INT = true covers the
// interior tile rectangle [ix0, ix0 + gridDim.x) x [iy0, iy0 + gridDim.y)
// with the branch-free body; INT = false covers the whole grid and returns at
// once on interior tiles.  Each kernel is compiled with one body only, so
// neither pays the other's registers.
template <int MODE, bool TMA, bool INT>
__global__ void __launch_bounds__(t32::NT, 1)
    k_mhd32(const Sim32 S, const __grid_constant__ TmaSet T,
            const float *__restrict__ a, const float *__restrict__ tin,
            float *__restrict__ so, float beta, float bnext, int zchunk, int mt,
            int ma, int ix0, int iy0, int gx, int gy) {
  extern __shared__ __align__(1024) float smem_raw32[];
  float *smem = (float *)(((size_t)smem_raw32 + 127) & ~(size_t)127);
  const int tx_ = INT ? blockIdx.x + ix0 : blockIdx.x;
  const int ty_ = INT ? blockIdx.y + iy0 : blockIdx.y;
  const int x0 = tx_ * t32::TX, y0 = ty_ * t32::TYT;
  if (!INT && mhd_interior(S, x0, y0)) return;
  if (sm_addr_t(smem) & 127u) {
    if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) atomicExch(S.err, 2);
    return;
  }
  double ke = 0.0, mr = 1e300, mp = 1e300;
  const int k0 = blockIdx.z * zchunk;
  if (!mhd_body<float, MODE, TMA, INT>(S, &T, smem, a, tin, so, beta, bnext, x0, y0, k0,
                                       min(S.nz, k0 + zchunk), mt, ma, ke, mr, mp))
    return;
  if (MODE == F_LAST)
    diag_reduce_t(S, ke, mr, mp, tx_ + (long long)gx * (ty_ + (long long)gy * blockIdx.z),
                  (long long)gx * gy * gridDim.z);
}

// ---------------------------------------------- FILTER_VARS, precision form
// FILTER_VARS of a filter event in the precision form (filter_body.cuh):
// the fused y-then-x pass over stored values (one depth scale per layer)
// and the z pass over physical values; `carry` (the first pass of an event)
// is subtracted on load, so the filter acts on the compensated value.
template <int G, bool CARRY>
__global__ void __launch_bounds__(fb::TX *fb::TY) k_filt_xy32(FiltArgs<float> F) {
  const int l = blockIdx.z / F.nz, k = blockIdx.z - l * F.nz;
  filt_xy_tile<float, G, CARRY>(F, l, k, blockIdx.x * fb::TX, blockIdx.y * fb::TR);
}
// the z pass: blockIdx.x is the z chunk, blockIdx.y the slab, blockIdx.z
// the field
template <int G, bool CARRY>
__global__ void __launch_bounds__(2 * fb::ZX * fb::ZY) k_filt_z32(FiltArgs<float> F) {
  extern __shared__ __align__(16) float zsl32[];
  const int nxb = (F.nx + fb::ZX - 1) / fb::ZX;
  const int yb = blockIdx.y / nxb, xb = blockIdx.y - yb * nxb;
  filt_z_slab<float, G, CARRY, true>(F, blockIdx.z, xb * fb::ZX, yb * fb::ZY, blockIdx.x * fb::ZC,
                               zsl32);
}

template <int G, bool CARRY>
static void filt_launch32(bool xy, const FiltArgs<float> &F, const dim3 &grid, size_t zs,
                          cudaStream_t s) {
  if (xy) {
    k_filt_xy32<G, CARRY><<<grid, dim3(fb::TX, fb::TY), 0, s>>>(F);
  } else {
    cudaFuncSetAttribute(k_filt_z32<G, CARRY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)zs);
    k_filt_z32<G, CARRY><<<grid, dim3(fb::ZX, fb::ZY, 2), zs, s>>>(F);
  }
}

int launch_filter_event32(Handle *h, bool xy, const float *in, const float *carry, float *out,
                          cudaStream_t s) {
  FiltArgs<float> F{};
  F.nx = h->nx; F.ny = h->ny; F.nz = h->nz; F.V = h->V; F.N = h->N;
  F.periodic = h->periodic ? 1 : 0;
  F.s = (float)(xy ? h->P.s_xy : h->P.s_z);
  F.in = in;
  F.out = out;
  F.carry = carry;
  const int g = xy ? h->gxy : h->gz;
  dim3 grid;
  size_t zs = 0;
  if (xy) {
    grid = dim3((h->nx + fb::TX - 1) / fb::TX, (h->ny + fb::TR - 1) / fb::TR, h->V * h->nz);
  } else {
    F.sc = h->f_sc;
    F.isc = h->f_isc;
    zs = filt_z_smem<float>();
    const long long slabs = (long long)((h->nx + fb::ZX - 1) / fb::ZX) *
                            ((h->ny + fb::ZY - 1) / fb::ZY);
    if (slabs > 65535) return SPARC_ERR_INVALID;
    grid = dim3((h->nz + fb::ZC - 1) / fb::ZC, (unsigned)slabs, h->V);
  }
  if (g == 5) {
    if (carry) filt_launch32<5, true>(xy, F, grid, zs, s);
    else filt_launch32<5, false>(xy, F, grid, zs, s);
  } else {
    if (carry) filt_launch32<3, true>(xy, F, grid, zs, s);
    else filt_launch32<3, false>(xy, F, grid, zs, s);
  }
  ++h->launches;
  return cudaGetLastError() == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

// ------------------------------------------------ PULSE = 2, precision form
// As k_psr of step.cu with an FP32 forcing buffer (the sum over pulses is
// accumulated in FP32).
__global__ void k_psr32(Psr32 D) {
  extern __shared__ float shf[];
  const int k = D.klo + blockIdx.z;
  const int e0 = D.off[k], e1 = D.off[k + 1], ne = e1 - e0;
  float *sT = shf;
  int *sN = (int *)(shf + ne);
  const long long it = *D.iter;
  const double t = (double)it * D.timestep;
  const double passes = (it == D.init) ? 2.0 : 1.0;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  for (int e = tid; e < ne; e += blockDim.x * blockDim.y) {
    const int n = D.idx[e0 + e];
    const double amp = D.ptime[3 * n], t0 = D.ptime[3 * n + 1], t1 = D.ptime[3 * n + 2];
    double v = amp * sin(2.0 * PI * (t - t1) / t0);
    v = v * exp(-((t - t1) * (t - t1)) / (2.0 * (D.st * D.st)));
    sT[e] = (float)(v * D.zv[e0 + e] * passes);
    sN[e] = n;
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= D.nx || j >= D.ny) return;
  const int blk = D.colx[i] + D.bx * D.coly[j] + D.bxy * D.colz[k];
  float f = 0.f;
  for (int e = 0; e < ne; ++e) {
    const int n = sN[e];
    if (!D.mask[(long long)n * D.nblocks + blk]) continue;
    f = f + sT[e] * (D.px[(long long)n * D.nx + i] * D.py[(long long)n * D.ny + j]);
  }
  const long long g = ((long long)k * D.ny + j) * D.nx + i;
  D.out[((long long)blockIdx.z * D.ny + j) * D.nx + i] = f * D.sd[g] * D.ssb[g];
}

Psr32 make_psr32(Handle *h) {
  Psr32 D{};
  D.nx = h->nx; D.ny = h->ny;
  D.klo = h->psr_klo;
  D.khi = h->psr_khi;
  D.nblocks = h->nblocks;
  D.bx = h->P.block_x;
  D.bxy = h->P.block_x * h->P.block_y;
  D.init = h->src.init;
  D.timestep = h->P.timestep;
  D.st = h->src.psr_st;
  D.off = h->d_plane_off;
  D.idx = h->d_plane_idx;
  D.colx = h->d_colx;
  D.coly = h->d_coly;
  D.colz = h->d_colx + h->nx + h->ny;
  D.zv = h->d_plane_z;
  D.ptime = h->d_ptime;
  D.px = h->f_px;
  D.py = h->f_py;
  D.sd = h->f_sd;
  D.ssb = h->f_ssb;
  D.mask = h->d_pmask;
  D.out = h->f_psr;
  D.iter = h->d_iter;
  return D;
}

int launch_psr32(Handle *h, cudaStream_t s) {
  if (h->src.kind != SPARC_SRC_PSR || h->psr_khi <= h->psr_klo) return SPARC_OK;
  Psr32 D = make_psr32(h);
  dim3 blk(32, 8);
  dim3 grd((h->nx + 31) / 32, (h->ny + 7) / 8, h->psr_khi - h->psr_klo);
  size_t smem = h->pulses.size() * (sizeof(float) + sizeof(int));
  k_psr32<<<grd, blk, smem, s>>>(D);
  ++h->launches;
  return cudaGetLastError() == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

// ------------------------------------------------------ FP64 -> FP32 copy
__global__ void k_d2f(long long n, const double *in, float *out) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    out[t] = (float)in[t];
}

__global__ void k_d2f_inv(long long n, const double *in, float *out) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    out[t] = (float)(1.0 / in[t]);
}

// 1/x in FP64, stored FP32 (the CPML 1/kappa profile)
int to_float_inv(const double *in, float *out, long long n, cudaStream_t s) {
  if (n <= 0) return SPARC_OK;
  unsigned nb = (unsigned)std::min<long long>((n + 255) / 256, 148 * 32);
  k_d2f_inv<<<nb, 256, 0, s>>>(n, in, out);
  return cudaGetLastError() == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

int to_float(const double *in, float *out, long long n, cudaStream_t s) {
  if (n <= 0) return SPARC_OK;
  unsigned nb = (unsigned)std::min<long long>((n + 255) / 256, 148 * 32);
  k_d2f<<<nb, 256, 0, s>>>(n, in, out);
  return cudaGetLastError() == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

// ------------------------------------------------------------- launchers
Sim32 make_sim32(Handle *h) {
  Sim32 S{};
  S.nx = h->nx; S.ny = h->ny; S.nz = h->nz; S.N = h->N;
  S.periodic = h->periodic ? 1 : 0;
  S.magnetic = h->magnetic ? 1 : 0;
  S.bg1d = h->bg1d ? 1 : 0;
  S.sponge_slabs = h->sponge_slabs ? 1 : 0;
  S.V = h->V;
  S.stretchx = h->stretchx;
  S.stretchy = h->stretchy;
  S.stretch = h->f_stretch;
  S.deltat = h->deltat;
  S.dimc2rho = (h->dimc * h->dimc) * h->dimrho;
  const float *const *b = h->f_bg;
  S.rho0 = b[FB_RHO0]; S.p0 = b[FB_P0]; S.rhoinv = b[FB_RHOINV];
  S.c2rho0 = b[FB_C2R]; S.grz = b[FB_GRZ]; S.gpz = b[FB_GPZ]; S.sponge = b[FB_SPONGE];
  S.box = b[FB_BOX]; S.boy = b[FB_BOY]; S.boz = b[FB_BOZ];
  S.cbx = b[FB_CBX]; S.cby = b[FB_CBY]; S.cbz = b[FB_CBZ];
  S.grx = b[FB_GRX]; S.gry = b[FB_GRY]; S.gpx = b[FB_GPX]; S.gpy = b[FB_GPY];
  S.red = b[FB_RED];
  S.gblk = h->f_gblk;
  S.colx = h->d_colx;
  S.coly = h->d_coly;
  S.bxdim = h->P.block_x;
  S.zb = h->f_faces[0]; S.zt = h->f_faces[1];
  S.xb = h->f_faces[2]; S.xt = h->f_faces[3];
  S.yb = h->f_faces[4]; S.yt = h->f_faces[5];
  ForcingT<float> &F = S.frc;
  F.kind = h->src.kind;
  F.dir = h->src.dir;
  F.init = h->src.init;
  F.fx = h->f_fx; F.fy = h->f_fy; F.fz = h->f_fz;
  F.amp_c = h->src.amp / 0.56458272 / h->dimc;
  F.t0 = h->src.t0; F.t1 = h->src.t1; F.st = h->src.st;
  F.timestep = h->P.timestep;
  F.psr = h->f_psr;
  F.klo = h->psr_klo;
  F.khi = h->psr_khi;
  F.f2d = h->f_f2d;
  F.sdep = h->f_sdep;
  S.sc = h->f_sc;
  S.isc = h->f_isc;
  S.carry = h->f_carry;
  S.iter = h->d_iter;
  S.err = h->d_err;
  S.partials = h->d_partials;
  S.counter = h->d_counter;
  S.diag = h->d_diag;
  S.fail_iter = h->d_fail;
  return S;
}

template <int TX, int TY>
static void launch_quiet32(Handle *h, const Sim32 &S, int mode, const float *a,
                           const float *tin, float *so, float beta, float bnext,
                           cudaStream_t s) {
  dim3 blk(TX, TY);
  dim3 grd((h->nx + TX - 1) / TX, (h->ny + TY - 1) / TY, (h->nz + h->zchunk - 1) / h->zchunk);
  const int zsm = (h->zchunk + 16) * 16 * (int)sizeof(float);
#define QL32(M, B)                                                                     \
  do {                                                                                 \
    cudaFuncSetAttribute(k_quiet32<TX, TY, M, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, zsm); \
    k_quiet32<TX, TY, M, B><<<grd, blk, zsm, s>>>(S, a, tin, so, beta, bnext, h->zchunk); \
  } while (0)
  if (S.bg1d) {
    if (mode == F_FIRST) QL32(F_FIRST, true);
    else if (mode == F_MID) QL32(F_MID, true);
    else QL32(F_LAST, true);
  } else {
    if (mode == F_FIRST) QL32(F_FIRST, false);
    else if (mode == F_MID) QL32(F_MID, false);
    else QL32(F_LAST, false);
  }
#undef QL32
}

int launch_stage32(Handle *h, const Sim32 &S, int stage, const float *a,
                   const float *tin, float *so, cudaStream_t s) {
  const float beta = (float)h->betas[stage - 1];
  const float bnext = (float)(stage < 5 ? h->betas[stage] : h->deltat);
  const int mode = stage == 1 ? F_FIRST : (stage == 5 ? F_LAST : F_MID);
  if (h->magnetic) {
    using namespace t32;
    int mt = -1, ma = -1;
    for (int b = 0; b < 3; ++b) {
      if (h->fbuf[b] == tin) mt = b;
      if (h->fbuf[b] == a) ma = b;
    }
    if (mt < 0 || ma < 0) return SPARC_ERR_INVALID;
    TmaSet T;
    std::memset(&T, 0, sizeof(T));  // [18..23]: the plain form's halo maps
    if (h->tma32)
      for (int n = 0; n < 18; ++n) T.m[n] = h->tmaps32[n];
    dim3 blk(TX, TY, 2);
    dim3 grd((h->nx + TX - 1) / TX, (h->ny + TYT - 1) / TYT, (h->nz + h->zchunk - 1) / h->zchunk);
    // interior tile rectangle (see mhd_interior), in tile units
    const int gx = (h->nx + TX - 1) / TX, gy = (h->ny + TYT - 1) / TYT;
    const FaceT<float> *F = h->f_faces;
    const int xm = std::max(5, F[2].on ? F[2].np : 0), xM = std::max(5, F[3].on ? F[3].np : 0);
    const int ym = std::max(5, F[4].on ? F[4].np : 0), yM = std::max(5, F[5].on ? F[5].np : 0);
    const int ix0 = (xm + TX - 1) / TX, ix1 = (h->nx - xM - TX) / TX + 1;
    const int iy0 = (ym + TYT - 1) / TYT, iy1 = (h->ny - yM - TYT) / TYT + 1;
    const bool has_int = h->nx - xM - TX >= 0 && h->ny - yM - TYT >= 0 && ix1 > ix0 && iy1 > iy0;
    dim3 gint(has_int ? ix1 - ix0 : 1, has_int ? iy1 - iy0 : 1, grd.z);
    const int smz = (int)MB::smem_bytes(h->zchunk);
    // the interior kernel's layout holds 48-wide halo rows with TMA own points
    const int smi = h->tma32 ? (int)MhdBuf<float, false, true>::smem_bytes(h->zchunk) : smz;
#define ML32(M, U)                                                                          \
  do {                                                                                      \
    cudaFuncSetAttribute(k_mhd32<M, U, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smi); \
    cudaFuncSetAttribute(k_mhd32<M, U, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smz); \
    if (has_int) {                                                                          \
      cudaEventRecord(h->ev_fork, s);                                                       \
      cudaStreamWaitEvent(h->aux, h->ev_fork, 0);                                           \
      k_mhd32<M, U, false><<<grd, blk, smz, h->aux>>>(S, T, a, tin, so, beta, bnext,       \
                                                       h->zchunk, mt, ma, 0, 0, gx, gy);    \
      cudaEventRecord(h->ev_join, h->aux);                                                  \
      k_mhd32<M, U, true><<<gint, blk, smi, s>>>(S, T, a, tin, so, beta, bnext, h->zchunk, \
                                                  mt, ma, ix0, iy0, gx, gy);                \
      cudaStreamWaitEvent(s, h->ev_join, 0);                                                \
    } else {                                                                                \
      k_mhd32<M, U, false><<<grd, blk, smz, s>>>(S, T, a, tin, so, beta, bnext, h->zchunk, \
                                                  mt, ma, 0, 0, gx, gy);                    \
    }                                                                                       \
  } while (0)
    if (has_int) ++h->launches;  // the interior launch (counted below: the other)
    if (h->tma32) {
      if (mode == F_FIRST) ML32(F_FIRST, true);
      else if (mode == F_MID) ML32(F_MID, true);
      else ML32(F_LAST, true);
    } else {
      if (mode == F_FIRST) ML32(F_FIRST, false);
      else if (mode == F_MID) ML32(F_MID, false);
      else ML32(F_LAST, false);
    }
#undef ML32
  } else {
    if (h->tx == 32) launch_quiet32<32, 8>(h, S, mode, a, tin, so, beta, bnext, s);
    else launch_quiet32<16, 8>(h, S, mode, a, tin, so, beta, bnext, s);
  }
  ++h->launches;
  return cudaGetLastError() == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

// FP32 tensor maps (32 x TYT x 1 boxes) of the own-point arrays of the MHD kernel
// (needs 16-byte row strides: nx a multiple of 4).
int encode_tensor_maps32(Handle *h) {
  h->tma32 = false;
  if (!h->magnetic || (h->nx & 3) || !h->allow_tma32) return SPARC_OK;
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
          cudaSuccess || !fn || q != cudaDriverEntryPointSuccess) {
    cudaGetLastError();
    return SPARC_OK;
  }
  auto enc = (CUresult(*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                          const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                          const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                          CUtensorMapL2promotion, CUtensorMapFloatOOBfill))fn;
  auto one = [&](CUtensorMap *m, const float *base, unsigned long long depth) {
    cuuint64_t dims[3] = {(cuuint64_t)h->nx, (cuuint64_t)h->ny, (cuuint64_t)depth};
    cuuint64_t strides[2] = {(cuuint64_t)h->nx * 4, (cuuint64_t)h->nx * h->ny * 4};
    cuuint32_t box[3] = {32, (cuuint32_t)t32::TYT, 1};
    cuuint32_t es[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)base, dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  bool ok = true;
  for (int b = 0; b < 3; ++b)
    ok = ok && one(&h->tmaps32[b], h->fbuf[b], (unsigned long long)h->nz * h->V);
  const int order[15] = {FB_RED, FB_SPONGE, FB_RHO0, FB_GRX, FB_GRY, FB_GRZ, FB_C2R,
                         FB_GPX, FB_GPY, FB_GPZ, FB_RHOINV, FB_CBX, FB_CBY, FB_CBZ, FB_P0};
  for (int n = 0; n < 15; ++n)
    ok = ok && h->f_bg[order[n]] && one(&h->tmaps32[3 + n], h->f_bg[order[n]], h->nz);
  h->tma32 = ok;
  return SPARC_OK;
}

// ------------------------------------------------------------ batched engine
// Many simulations advance together: each RK stage is one persistent launch
// whose blocks pull (sim, tile, z-chunk) items from a device work-list
// (dynamic scheduling by an atomic counter).  MHD items are 32x8-column
// tiles of the two-role body; quiet items are 32x16 tiles of the quiet body
// on the same 512 threads.  The last item of a simulation to finish the
// last stage reduces its diagnostics, advances its iteration, decrements
// its steps left and rotates its buffer roles; filter passes check their
// cadence per simulation on the device.

constexpr int BT = t32::NT;  // threads of a batched block

// block-wide sum / min / min of (ke, mr, mp); the result is valid in tid 0
__device__ __forceinline__ void block_reduce3(double &ke, double &mr, double &mp, int tid) {
  __shared__ double r[3][32];
  const int lane = tid & 31, warp = tid >> 5, nw = BT / 32;
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
  }
}

__device__ __forceinline__ void rotate_roles(Slot32 &L) {
  const int a = L.role[0];
  L.role[0] = L.role[1];
  L.role[1] = L.role[2];
  L.role[2] = a;
}

// Item w (of slot L) finished the last stage: store its partial; the last
// item of the slot ends the step (driver.f90:161-183 diagnostics).
__device__ void batch_finish_step(Slot32 &L, const Sim32 &S, int w, double ke, double mr,
                                  double mp, int tid) {
  __shared__ int am_last;
  block_reduce3(ke, mr, mp, tid);
  if (tid == 0) {
    L.partials[3 * w] = ke;
    L.partials[3 * w + 1] = mr;
    L.partials[3 * w + 2] = mp;
    __threadfence();
    const unsigned t = atomicAdd(&L.counter, 1u);
    am_last = (t == (unsigned)(L.n_items + L.n_items2 - 1));
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  ke = 0.0; mr = 1e300; mp = 1e300;
  for (int q = tid; q < L.n_items + L.n_items2; q += BT) {
    const int b = q < L.n_items ? L.first_item + q : L.first_item2 + (q - L.n_items);
    ke += __ldcg(L.partials + 3 * b);
    mr = fmin(mr, __ldcg(L.partials + 3 * b + 1));
    mp = fmin(mp, __ldcg(L.partials + 3 * b + 2));
  }
  block_reduce3(ke, mr, mp, tid);
  if (tid == 0) {
    const long long it = *S.iter;
    const double kev = sqrt(ke / ((double)S.nx * (double)S.ny * (double)S.nz)) * S.dimc2rho;
    S.diag[0] = kev;
    S.diag[1] = mr;
    S.diag[2] = mp;
    S.diag[3] = (double)it;
    const bool fail = !(kev <= 1000.0) || !(mr > 0.0) || !(mp > 0.0);
    if (fail && *S.fail_iter < 0) *S.fail_iter = it;
    *S.iter = it + 1;
    L.remaining -= 1;
    rotate_roles(L);
    L.counter = 0u;
  }
}

__global__ void k_batch_begin(Slot32 *slots, int n) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
    slots[q].active = slots[q].remaining > 0 ? 1 : 0;
}

// PART 0: the interior MHD items (a prefix of the list, branch-free body);
// PART 1: the rest (MHD tiles at edges/CPML, quiet tiles); PART 2: the whole
// list in one launch (interior items first, then the rest, so no launch
// boundary separates the two parts).
template <int MODE, int PART>
__global__ void __launch_bounds__(BT, 1)
    k_batch_stage(Slot32 *__restrict__ slots, const int4 *__restrict__ items,
                  const int *__restrict__ counts, unsigned *wctr, int stage) {
  using MB = t32::MB;
  extern __shared__ __align__(1024) float smem_raw32[];
  __shared__ __align__(16) unsigned long long sS_raw[(sizeof(Sim32) + 7) / 8];
  __shared__ int s_w;
  float *smem = (float *)(((size_t)smem_raw32 + 127) & ~(size_t)127);
  float *qzt = smem + 2 * MB::BUF + MB::XCH;  // quiet items' scale table
  Sim32 &sS = *reinterpret_cast<Sim32 *>(sS_raw);
  const int tid = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
  const int lo = PART == 1 ? counts[3] : 0, hi = PART == 0 ? counts[3] : counts[0];
  int cur = -1;
  for (;;) {
    if (tid == 0) s_w = lo + (int)atomicAdd(wctr, 1u);
    __syncthreads();
    const int w = s_w;
    if (w >= hi) break;
    const int4 it = items[w];
    Slot32 &L = slots[it.x];
    if (!L.active) {
      __syncthreads();
      continue;
    }
    if (it.x != cur) {
      const unsigned long long *src = reinterpret_cast<const unsigned long long *>(&L.S);
      for (int q = tid; q < (int)(sizeof(Sim32) / 8); q += BT) sS_raw[q] = src[q];
      cur = it.x;
      __syncthreads();
    }
    const int ra = L.role[0], r1 = L.role[1], r2 = L.role[2];
    const float *a = L.buf[ra];
    const float *tin = stage == 1 ? a : L.buf[(stage == 2 || stage == 4) ? r1 : r2];
    float *so = L.buf[(stage & 1) ? r1 : r2];
    const float beta = (float)L.betas[stage - 1];
    const float bnext = (float)(stage < 5 ? L.betas[stage] : sS.deltat);
    const int x0 = it.y, y0 = it.z, k0 = it.w & 0xffff, k1 = it.w >> 16;
    double ke = 0.0, mr = 1e300, mp = 1e300;
    if (PART == 0 || (PART == 2 && w < counts[3]))
      mhd_body<float, MODE, false, true>(sS, nullptr, smem, a, tin, so, beta, bnext, x0, y0,
                                         k0, k1, 0, 0, ke, mr, mp);
    else if (sS.magnetic)
      mhd_body<float, MODE, false, false>(sS, nullptr, smem, a, tin, so, beta, bnext, x0, y0,
                                          k0, k1, 0, 0, ke, mr, mp);
    else if (sS.bg1d)
      quiet_body<32, 16, MODE, true>(sS, a, tin, so, beta, bnext, x0, y0, k0, k1, threadIdx.x,
                                     threadIdx.y + 8 * threadIdx.z, qzt, ke, mr, mp);
    else
      quiet_body<32, 16, MODE, false>(sS, a, tin, so, beta, bnext, x0, y0, k0, k1, threadIdx.x,
                                      threadIdx.y + 8 * threadIdx.z, qzt, ke, mr, mp);
    if (MODE == F_LAST) batch_finish_step(L, sS, w, ke, mr, mp, tid);
    __syncthreads();
  }
}

// PULSE = 0 forcing planes of the random-source members, at each member's
// iteration (random_forcing.cuh); every block strides over every such
// member's plane.
__global__ void __launch_bounds__(BT)
    k_batch_random(Slot32 *__restrict__ slots, int nslots) {
  for (int q = 0; q < nslots; ++q) {
    const Slot32 &L = slots[q];
    if (!L.active || !L.has_rnd) continue;
    const Rnd32 &D = L.rnd;
    const RndStencil R = rnd_stencil(*L.S.iter, D.timestep, D.cad, D.ns);
    for (int p = blockIdx.x * BT + threadIdx.x; p < D.nxy; p += gridDim.x * BT)
      D.out[p] = (float)rnd_column(R, D.series, D.nxy, p, D.damp[p]);
  }
}

// PULSE = 2 forcing of one layer of one simulation per item.
__global__ void __launch_bounds__(BT)
    k_batch_psr(Slot32 *__restrict__ slots, const int4 *__restrict__ items,
                const int *__restrict__ counts, unsigned *wctr) {
  extern __shared__ float shf[];
  __shared__ int s_w;
  const int tid = threadIdx.x;
  const int total = counts[2];
  for (;;) {
    if (tid == 0) s_w = (int)atomicAdd(wctr, 1u);
    __syncthreads();
    const int w = s_w;
    if (w >= total) break;
    const int4 it = items[w];
    const Slot32 &L = slots[it.x];
    if (!L.active) {
      __syncthreads();
      continue;
    }
    const Psr32 &D = L.psr;
    const int k = it.y;
    const int e0 = D.off[k], e1 = D.off[k + 1], ne = e1 - e0;
    float *sT = shf;
    int *sN = (int *)(shf + ne);
    const long long itn = *D.iter;
    const double t = (double)itn * D.timestep;
    const double passes = (itn == D.init) ? 2.0 : 1.0;
    for (int e = tid; e < ne; e += BT) {
      const int n = D.idx[e0 + e];
      const double amp = D.ptime[3 * n], t0 = D.ptime[3 * n + 1], t1 = D.ptime[3 * n + 2];
      double v = amp * sin(2.0 * PI * (t - t1) / t0);
      v = v * exp(-((t - t1) * (t - t1)) / (2.0 * (D.st * D.st)));
      sT[e] = (float)(v * D.zv[e0 + e] * passes);
      sN[e] = n;
    }
    __syncthreads();
    const int nx = D.nx, ny = D.ny;
    const int bz = D.bxy * D.colz[k];
    for (int q = tid; q < nx * ny; q += BT) {
      const int j = q / nx, i = q - j * nx;
      const int blk = D.colx[i] + D.bx * D.coly[j] + bz;
      float f = 0.f;
      for (int e = 0; e < ne; ++e) {
        const int n = sN[e];
        if (!D.mask[(long long)n * D.nblocks + blk]) continue;
        f = f + sT[e] * (D.px[(long long)n * nx + i] * D.py[(long long)n * ny + j]);
      }
      const long long g = (long long)k * nx * ny + q;
      D.out[(long long)(k - D.klo) * nx * ny + q] = f * D.sd[g] * D.ssb[g];
    }
    __syncthreads();
  }
}

// The fused y-then-x pass of FILTER_VARS for the members whose xy cadence
// asks for it after the iteration just stepped (always the first pass of
// the event: stored - carry): work items (member, field, group of LPB
// layers, 32 x 32 tile) of the single path's tile kernel (filter_body.cuh,
// filt_xy_tile, stored values: one depth scale per layer).  Block (32, 8).
// The last item of a member rotates its buffer roles.
__global__ void __launch_bounds__(fb::NT)
    k_batch_filter_xy(Slot32 *__restrict__ slots, const int4 *__restrict__ xyitems,
                      const int *__restrict__ counts, unsigned *wctr) {
  __shared__ int s_w;
  const int tid = threadIdx.y * fb::TX + threadIdx.x;
  const int total = counts[5];
  for (;;) {
    if (tid == 0) s_w = (int)atomicAdd(wctr, 1u);
    __syncthreads();
    const int w = s_w;
    if (w >= total) break;
    const int4 it = xyitems[w];
    Slot32 &L = slots[it.x];
    bool need_xy = false;
    if (L.active) {
      const long long nn = *L.S.iter - 1;
      need_xy = nn != 0 && nn % L.xyfreq == 0;
    }
    if (!need_xy) {
      __syncthreads();
      continue;
    }
    FiltArgs<float> F{};
    F.nx = L.S.nx; F.ny = L.S.ny; F.nz = L.S.nz; F.V = L.S.V; F.N = L.S.N;
    F.periodic = L.S.periodic;
    F.s = L.s_xy;
    F.in = L.buf[L.role[0]];
    F.out = L.buf[L.role[1]];
    F.carry = L.S.carry;
    const int ntx = (F.nx + fb::TX - 1) / fb::TX;
    const int ty = it.w / ntx, tx = it.w - ty * ntx;
    const int k0 = it.z * fb::LPB, k1 = min(F.nz, k0 + fb::LPB);
    // consecutive calls: each one's first barrier follows the previous
    // one's last shared reads
    for (int k = k0; k < k1; ++k) {
      if (L.gxy == 5) filt_xy_tile<float, 5, true>(F, it.y, k, tx * fb::TX, ty * fb::TR);
      else filt_xy_tile<float, 3, true>(F, it.y, k, tx * fb::TX, ty * fb::TR);
    }
    __syncthreads();
    if (tid == 0) {
      const unsigned c = atomicAdd(&L.counter, 1u);
      if (c == (unsigned)(L.xy_items - 1)) {
        rotate_roles(L);
        L.counter = 0u;
      }
    }
  }
}

// The z direction of FILTER_VARS for the members whose z cadence asks for
// it: each work item is one (member, field, 32 x 4 column slab, 32-layer
// chunk), filtered by the single path's slab kernel (filter_body.cuh,
// filt_z_slab: physical values, stored back scaled; stored - carry when the
// event has no xy part, as the first pass of the event).  Block (32, 4, 2).
__global__ void __launch_bounds__(2 * fb::ZX * fb::ZY)
    k_batch_filter_z(Slot32 *__restrict__ slots, const int4 *__restrict__ zitems,
                     const int *__restrict__ counts, unsigned *wctr) {
  extern __shared__ __align__(16) float zsl_b[];
  __shared__ int s_w;
  const int tid = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
  const int total = counts[4];
  for (;;) {
    if (tid == 0) s_w = (int)atomicAdd(wctr, 1u);
    __syncthreads();
    const int w = s_w;
    if (w >= total) break;
    const int4 it = zitems[w];
    Slot32 &L = slots[it.x];
    bool need_z = false, need_xy = false;
    if (L.active) {
      const long long nn = *L.S.iter - 1;
      need_xy = nn != 0 && nn % L.xyfreq == 0;
      need_z = nn != 0 && nn % L.zfreq == 0;
    }
    if (!need_z) {
      __syncthreads();
      continue;
    }
    FiltArgs<float> F{};
    F.nx = L.S.nx; F.ny = L.S.ny; F.nz = L.S.nz; F.V = L.S.V; F.N = L.S.N;
    F.periodic = L.S.periodic;
    F.s = L.s_z;
    F.in = L.buf[L.role[0]];
    F.out = L.buf[L.role[1]];
    F.sc = L.S.sc;
    F.isc = L.S.isc;
    const bool first = !need_xy;
    F.carry = first ? L.S.carry : nullptr;
    const int nxb = (F.nx + fb::ZX - 1) / fb::ZX;
    const int yb = it.z / nxb, xb = it.z - yb * nxb;
    const int x0 = xb * fb::ZX, y0 = yb * fb::ZY, k0 = it.w * fb::ZC;
    if (L.gz == 5) {
      if (first) filt_z_slab<float, 5, true, true>(F, it.y, x0, y0, k0, zsl_b);
      else filt_z_slab<float, 5, false, true>(F, it.y, x0, y0, k0, zsl_b);
    } else {
      if (first) filt_z_slab<float, 3, true, true>(F, it.y, x0, y0, k0, zsl_b);
      else filt_z_slab<float, 3, false, true>(F, it.y, x0, y0, k0, zsl_b);
    }
    __syncthreads();
    if (tid == 0) {
      const unsigned c = atomicAdd(&L.counter, 1u);
      if (c == (unsigned)(L.z_items - 1)) {
        rotate_roles(L);
        L.counter = 0u;
      }
    }
  }
}

// After a member's filter event its filtered state starts a new compensated
// sum: zero its carry over the filter items' ranges.
__global__ void __launch_bounds__(BT)
    k_batch_carry_clear(Slot32 *__restrict__ slots, const int4 *__restrict__ items,
                        const int *__restrict__ counts, unsigned *wctr) {
  __shared__ int s_w;
  const int total = counts[1];
  for (;;) {
    if (threadIdx.x == 0) s_w = (int)atomicAdd(wctr, 1u);
    __syncthreads();
    const int w = s_w;
    __syncthreads();
    if (w >= total) break;
    const int4 it = items[w];
    const Slot32 &L = slots[it.x];
    if (!L.active) continue;
    const long long nn = *L.S.iter - 1;
    if (nn == 0 || (nn % L.xyfreq != 0 && nn % L.zfreq != 0)) continue;
    for (long long t = it.y + threadIdx.x; t < (long long)it.y + it.z; t += BT) L.S.carry[t] = 0.f;
  }
}

size_t batch_stage_smem() { return t32::MB::SMEM; }

// One persistent launch per RK stage over the whole work-list (MHD items of
// 32 x 8 columns).
static void launch_batch_stages(const BatchLaunch &B, cudaStream_t s) {
  const int sm = (int)t32::MB::smem_bytes(B.zmax);
  cudaFuncSetAttribute(k_batch_stage<F_FIRST, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  cudaFuncSetAttribute(k_batch_stage<F_MID, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  cudaFuncSetAttribute(k_batch_stage<F_LAST, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  const dim3 blk(t32::TX, t32::TY, 2);
  for (int st = 1; st <= 5; ++st) {
    unsigned *c = B.wctr + st;  // work counter of stage st
    if (st == 1)
      k_batch_stage<F_FIRST, 2><<<B.grid, blk, (size_t)sm, s>>>(B.slots, B.items, B.counts, c, st);
    else if (st < 5)
      k_batch_stage<F_MID, 2><<<B.grid, blk, (size_t)sm, s>>>(B.slots, B.items, B.counts, c, st);
    else
      k_batch_stage<F_LAST, 2><<<B.grid, blk, (size_t)sm, s>>>(B.slots, B.items, B.counts, c, st);
  }
}

int launch_batch_step(const BatchLaunch &B, cudaStream_t s, int *nkernels) {
  if (cudaMemsetAsync(B.wctr, 0, 14 * sizeof(unsigned), s) != cudaSuccess) return SPARC_ERR_CUDA;
  k_batch_begin<<<(B.nslots + 255) / 256, 256, 0, s>>>(B.slots, B.nslots);
  k_batch_psr<<<B.grid, BT, B.psr_smem, s>>>(B.slots, B.pitems, B.counts, B.wctr + 0);
  k_batch_random<<<B.grid, BT, 0, s>>>(B.slots, B.nslots);
  launch_batch_stages(B, s);
  k_batch_filter_xy<<<B.grid * 6, dim3(fb::TX, fb::TY), 0, s>>>(B.slots, B.xyitems, B.counts,
                                                                 B.wctr + 6);
  k_batch_filter_z<<<B.grid * 6, dim3(fb::ZX, fb::ZY, 2), filt_z_smem<float>(), s>>>(
      B.slots, B.zitems, B.counts, B.wctr + 8);
  k_batch_carry_clear<<<B.grid * 2, BT, 0, s>>>(B.slots, B.fitems, B.counts, B.wctr + 9);
  *nkernels = 11;
  return cudaGetLastError() == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

// ------------------------------------------------------ precision-form setup
// Runs after the FP64 setup (setup.cu): derives the depth scales from the
// background column (1,1,:), converts the coefficients, CPML profiles and
// tables to FP32 and releases the FP64 arrays that the FP32 path does not
// read.
static float *f_up(Handle *h, const double *src, long long n, cudaStream_t s) {
  float *d = (float *)dev_alloc(h, (size_t)std::max<long long>(n, 1) * sizeof(float));
  if (!d) return nullptr;
  if (src && n > 0 && to_float(src, d, n, s)) return nullptr;
  return d;
}

int setup32(Handle *h) {
  cudaStream_t s = h->stream;
  const int nz = h->nz, V = h->V;
  const long long N = h->N, NXY = (long long)h->nx * h->ny;
  // depth scales: rho 1/rho0, v sqrt(rho0), p 1/(rho0 c0^2), b 1
  std::vector<double> r0(nz), c2r(nz);
  if (cudaMemcpy2D(r0.data(), 8, h->rho0, NXY * 8, 8, nz, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy2D(c2r.data(), 8, h->c2rho0, NXY * 8, 8, nz, cudaMemcpyDeviceToHost) !=
          cudaSuccess)
    return SPARC_ERR_CUDA;
  std::vector<float> sc((size_t)2 * V * nz);
  for (int l = 0; l < V; ++l)
    for (int k = 0; k < nz; ++k) {
      double v = 1.0;
      if (l == 0) v = 1.0 / r0[k];
      else if (l <= 3) v = std::sqrt(r0[k]);
      else if (l == 4) v = 1.0 / c2r[k];
      sc[(size_t)l * nz + k] = (float)v;
      sc[(size_t)(V + l) * nz + k] = (float)(1.0 / v);
    }
  h->f_sc = (float *)dev_alloc(h, sc.size() * sizeof(float));
  if (!h->f_sc) return SPARC_ERR_NOMEM;
  h->f_isc = h->f_sc + (size_t)V * nz;
  if (cudaMemcpyAsync(h->f_sc, sc.data(), sc.size() * sizeof(float), cudaMemcpyHostToDevice,
                      s) != cudaSuccess)
    return SPARC_ERR_CUDA;
  // background
  struct Src {
    int fb;
    double *d3, *d1;
  } srcs[FB_COUNT] = {
      {FB_RHO0, h->rho0, h->rho0_1},     {FB_P0, h->p0, h->p0_1},
      {FB_RHOINV, h->rhoinv, h->rhoinv_1}, {FB_C2R, h->c2rho0, h->c2rho0_1},
      {FB_GRZ, h->grz, h->grz_1},        {FB_GPZ, h->gpz, h->gpz_1},
      {FB_SPONGE, h->sponge, h->sponge_1}, {FB_BOX, h->box, nullptr},
      {FB_BOY, h->boy, nullptr},         {FB_BOZ, h->boz, nullptr},
      {FB_CBX, h->cbx, nullptr},         {FB_CBY, h->cby, nullptr},
      {FB_CBZ, h->cbz, nullptr},         {FB_GRX, h->grx, nullptr},
      {FB_GRY, h->gry, nullptr},         {FB_GPX, h->gpx, nullptr},
      {FB_GPY, h->gpy, nullptr},         {FB_RED, h->red, nullptr}};
  for (const Src &q : srcs) {
    const bool one = h->bg1d && q.d1;
    const double *src = one ? q.d1 : q.d3;
    if (!src) continue;
    h->f_bg[q.fb] = f_up(h, src, one ? nz : N, s);
    if (!h->f_bg[q.fb]) return SPARC_ERR_NOMEM;
  }
  h->f_stretch = f_up(h, h->d_stretch, nz, s);
  h->f_gblk = f_up(h, h->d_gblk, (long long)h->g_blk.size(), s);
  h->f_sd = f_up(h, h->source_damp, N, s);
  h->f_ssb = f_up(h, h->ssb, N, s);
  if (!h->f_stretch || !h->f_gblk || !h->f_sd || !h->f_ssb) return SPARC_ERR_NOMEM;
  // CPML profiles (FP64 setup, FP32 storage)
  for (int f = 0; f < 6; ++f) {
    const FaceDev &D = h->faces[f];
    FaceT<float> &F = h->f_faces[f];
    if (!D.on) continue;
    const long long n = D.uniform ? D.np : D.cnt;
    float *pa = f_up(h, D.pa, n, s), *pb = f_up(h, D.pb, n, s), *pk = f_up(h, D.pk, n, s);
    float *pki = f_up(h, nullptr, n, s);
    if (!pa || !pb || !pk || !pki) return SPARC_ERR_NOMEM;
    if (to_float_inv(D.pk, pki, n, s)) return SPARC_ERR_CUDA;
    F.pa = pa; F.pb = pb; F.pk = pk; F.pki = pki;
    F.uniform = D.uniform;
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return SPARC_ERR_CUDA;
  // release the FP64 arrays (geometry of the faces is kept)
  double *rel[] = {h->rho0, h->p0, h->c2, h->rhoinv, h->c2rho0, h->grz, h->gpz,
                   h->sponge, h->box, h->boy, h->boz, h->cbx, h->cby, h->cbz,
                   h->grx, h->gry, h->gpx, h->gpy, h->red, h->source_damp, h->ssb,
                   h->rho0_1, h->p0_1, h->rhoinv_1, h->c2rho0_1, h->grz_1, h->gpz_1,
                   h->sponge_1};
  for (double *p : rel)
    if (p) dev_free(h, p);
  h->rho0 = h->p0 = h->c2 = h->rhoinv = h->c2rho0 = h->grz = h->gpz = h->sponge = nullptr;
  h->box = h->boy = h->boz = h->cbx = h->cby = h->cbz = nullptr;
  h->grx = h->gry = h->gpx = h->gpy = h->red = h->source_damp = h->ssb = nullptr;
  h->rho0_1 = h->p0_1 = h->rhoinv_1 = h->c2rho0_1 = h->grz_1 = h->gpz_1 = h->sponge_1 = nullptr;
  for (int f = 0; f < 6; ++f) {
    FaceDev &D = h->faces[f];
    if (!D.on) continue;
    dev_free(h, D.pa);
    dev_free(h, D.pb);
    dev_free(h, D.pk);
    dev_free(h, D.pki);
    D.pa = D.pb = D.pk = D.pki = nullptr;
  }
  return encode_tensor_maps32(h);
}

// FP32 copies of the forcing tables built by sparc_set_source.
int source32(Handle *h) {
  cudaStream_t s = h->stream;
  if (h->src.kind == SPARC_SRC_PULSE) {
    if (!h->f_fx) {
      h->f_fx = f_up(h, nullptr, h->nx + h->ny + h->nz, s);
      if (!h->f_fx) return SPARC_ERR_NOMEM;
      h->f_fy = h->f_fx + h->nx;
      h->f_fz = h->f_fy + h->ny;
    }
    if (to_float(h->d_fx, h->f_fx, h->nx + h->ny + h->nz, s)) return SPARC_ERR_CUDA;
  } else if (h->src.kind == SPARC_SRC_PSR) {
    const long long np = (long long)h->pulses.size();
    dev_free(h, h->f_px);  // a later call replaces the tables of an earlier one
    dev_free(h, h->f_py);
    dev_free(h, h->f_psr);
    h->f_px = f_up(h, h->d_px, np * h->nx, s);
    h->f_py = f_up(h, h->d_py, np * h->ny, s);
    h->f_psr = f_up(h, nullptr,
                    std::max<long long>(1, (long long)(h->psr_khi - h->psr_klo) * h->nx * h->ny), s);
    if (!h->f_px || !h->f_py || !h->f_psr) return SPARC_ERR_NOMEM;
  } else if (h->src.kind == SPARC_SRC_RANDOM) {
    dev_free(h, h->f_sdep);
    dev_free(h, h->f_f2d);
    h->f_sdep = f_up(h, h->d_sdep, h->nz, s);
    h->f_f2d = f_up(h, nullptr, (long long)h->nx * h->ny, s);
    if (!h->f_sdep || !h->f_f2d) return SPARC_ERR_NOMEM;
  }
  return cudaStreamSynchronize(s) == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

}  // namespace sparc
