// step.cu -- the time step on the device: one fused kernel per RK stage
// (stage values, 11-point derivatives, CPML, RHS, boundary zeroing, stage or
// final update, diagnostics), the PULSE = 2 forcing of an iteration, and
// the FILTER_VARS passes.
//
// Stage kernel layout: a CTA owns a TX x TY tile of (x, y) columns and
// marches up a chunk of z layers.  z derivatives come from an 11-deep
// register window per z-differentiated field (the thread's own column);
// x and y derivatives from a shared-memory layer tile with a 5-point halo.
// Stage values are forwarded: stage k writes temp_{k+1} = a + beta_{k+1}*F_k
// (step.f90:33) instead of F_k, so every halo and window load of the next
// stage reads one array; stage 5 writes a + deltat*F_5 (step.f90:58).  The
// HBM traffic is that of the reference's scheme (14 V words per point and
// step) and the values are bitwise those of forming a + beta*F on load.

#include <cmath>
#include <cstdlib>
#include <cstring>

#include "filter_body.cuh"
#include "mhd_body.cuh"
#include "random_forcing.cuh"

namespace sparc {

__constant__ double c_dp[6][11];   // derivative rows, initialize.f90:1959-2031
__constant__ double c_df[2][11];   // filter stencils: [0] 11-point, [1] 7-point

enum { FIRST = 0, MID = 1, LAST = 2 };

template <>
__device__ __forceinline__ double dcoef<double>(int r, int m) {
  return c_dp[r][m];
}
template <>
__device__ __forceinline__ double fcoef<double>(int t, int m) {
  return c_df[t][m];
}

int step_constants() {
  if (cudaMemcpyToSymbol(c_dp, kDerivRows, sizeof(double) * 66) != cudaSuccess)
    return SPARC_ERR_CUDA;
  return SPARC_OK;
}


// CPML correction of one derivative (RHS.f90:50-93, 424-546):
// RHSpsi = a*d + b*psi ; d = d/kappa + psi.  LAST applies the final RK
// update of the auxiliary field in place (step.f90:59-61).
template <int MODE>
__device__ __forceinline__ void cpml(const FaceDev &F, long long f, int layer,
                                     int slot, double beta, double dt,
                                     double &d) {
  const long long pf = F.uniform ? (long long)layer : f;
  const double pa = __ldg(F.pa + pf), pb = __ldg(F.pb + pf),
               pk = __ldg(F.pk + pf);
  const long long o = (long long)slot * F.cnt + f;
  const double v = F.vars[o];
  double psi = v;
  if (MODE != FIRST) psi = v + beta * F.scr[o];
  const double rhs = pa * d + pb * psi;
  d = d / pk + psi;
  if (MODE == LAST) F.vars[o] = v + dt * rhs;
  else F.scr[o] = rhs;
}

// Forcing of driver.f90:137-153 at point (i, j, k) of iteration `it`.
__device__ __forceinline__ double forcing_at(const SimDev &S, long long it,
                                             double T, int i, int j, int k) {
  const ForcingDev &F = S.frc;
  if (F.kind == SPARC_SRC_PULSE)
    return T * __ldg(F.fz + k) * (__ldg(F.fy + j) * __ldg(F.fx + i));
  if (F.kind == SPARC_SRC_PSR && k >= F.klo && k < F.khi)
    return F.psr[((long long)(k - F.klo) * S.ny + j) * S.nx + i];
  if (F.kind == SPARC_SRC_RANDOM) return F.f2d[(long long)j * S.nx + i] * __ldg(F.sdep + k);
  return 0.0;
}

__device__ __forceinline__ double pulse_time(const SimDev &S, long long it) {
  const ForcingDev &F = S.frc;
  if (F.kind != SPARC_SRC_PULSE) return 0.0;
  const double t = (double)it * F.timestep;
  double T = F.amp_c * sin(2.0 * PI * (t - F.t1 + 2.0 * F.t0) / F.t0);
  return T * exp(-1.0 * ((t - F.t1) * (t - F.t1)) / (2.0 * (F.st * F.st)));
}

// ------------------------------------------------------------ diagnostics
// Block partial of the KE norm and the two minima, then the last CTA to
// finish reduces all partials (no waiting: it is simply the last to arrive)
// and applies the fail criterion of driver.f90:175-183.
__device__ void diag_reduce(const SimDev &S, double ke, double mr, double mp) {
  __shared__ double r[3][32];
  __shared__ int am_last;
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const int tid = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5, nw = (nt + 31) >> 5;
  const long long nb = (long long)gridDim.x * gridDim.y * gridDim.z;
  const long long bid = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
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
    // norm(): sqrt(sum/(nx*ny*nz)) (all_modules.f90:703), times dimc^2*dimrho
    double nrm = sqrt(ke / ((double)S.nx * (double)S.ny * (double)S.nz));
    double kev = nrm * S.dimc2rho;
    S.diag[0] = kev;
    S.diag[1] = mr;
    S.diag[2] = mp;
    S.diag[3] = (double)it;
    // driver.f90:175-183; a NaN norm also counts as a failure
    bool fail = !(kev <= 1000.0) || !(mr > 0.0) || !(mp > 0.0);
    if (fail && *S.fail_iter < 0) *S.fail_iter = it;
    *S.iter = it + 1;
    *S.counter = 0u;
  }
}

// ------------------------------------------------------------ helpers
__device__ __forceinline__ int wrapi(int q, int n) {
  q = q < 0 ? q + n : q;
  return q >= n ? q - n : q;
}

// Global index of local tile position 0 along one axis.  Normally t0 - 5;
// on a non-periodic axis the last tile may start closer than 6 points to
// the edge, and its origin then moves down to n - 11 so that the one-sided
// window f(n-11 .. n-1) is in the tile (interior points still see +-5).
__device__ __forceinline__ int tile_origin(int t0, int T, int n, bool per) {
  int o = t0 - 5;
  if (!per && t0 + T >= n) o = min(o, n - 11);
  return o;
}

// x or y derivative at local tile position from a row/column of shared
// memory: `t(m)` returns the tile value at global index g0 + m.  Periodic
// axes and interior points use the centred row (RHS bh = 5 / interior),
// non-periodic edges the one-sided rows (derivatives.f90:72, 98).
template <class Get>
__device__ __forceinline__ double dxy(int q, int n, bool per, double sc,
                                      Get t) {
  double s = 0.0;
  if (per || (q >= 5 && q < n - 5)) {
#pragma unroll
    for (int m = 0; m < 11; ++m) s += t(q - 5 + m) * c_dp[5][m];
    return sc * s;
  }
  if (q < 5) {
#pragma unroll
    for (int m = 0; m < 11; ++m) s += t(m) * c_dp[q][m];
    return sc * s;
  }
  const int row = n - 1 - q;
#pragma unroll
  for (int m = 0; m < 11; ++m) s += t(n - 1 - m) * c_dp[row][m];
  return -sc * s;
}

// z derivative from the 11-deep window w (w[m] = f(base + m)), with the
// bottom zero ghosts already in the window and the top one-sided rows
// (derivatives.f90:509-545).
__device__ __forceinline__ double dz(const double (&w)[11], int k, int nz,
                                     double sc) {
  double s = 0.0;
  if (k < nz - 5) {
#pragma unroll
    for (int m = 0; m < 11; ++m) s += w[m] * c_dp[5][m];
    return sc * s;
  }
  const int row = nz - 1 - k;
#pragma unroll
  for (int m = 0; m < 11; ++m) s += w[10 - m] * c_dp[row][m];
  return -sc * s;
}

__device__ __forceinline__ void shift(double (&w)[11], double v) {
#pragma unroll
  for (int m = 0; m < 10; ++m) w[m] = w[m + 1];
  w[10] = v;
}

// ------------------------------------------------ MP_QUIET_3D stage kernel
// RHS.f90:18-175 fused with one RK stage of step.f90:26-61.
template <int TX, int TY, int MODE, bool BG1D>
__global__ void __launch_bounds__(TX *TY)
    k_stage_quiet(const SimDev S, const double *__restrict__ a,
                  const double *__restrict__ tin, double *__restrict__ so,
                  double beta, double bnext, int zchunk) {
  constexpr int HX = TX + 10, HY = TY + 10;
  __shared__ double t_vx[HY][HX], t_vy[HY][HX], t_p[HY][HX];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int nx = S.nx, ny = S.ny, nz = S.nz;
  const long long N = S.N, NXY = (long long)nx * ny;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int i = x0 + tx, j = y0 + ty;
  const bool act = i < nx && j < ny;
  const bool per = S.periodic;
  const int k0 = blockIdx.z * zchunk, k1 = min(nz, k0 + zchunk);
  const long long col = (long long)j * nx + i;
  const long long it = *S.iter;
  const double Tp = pulse_time(S, it);
  const double dt = S.deltat;
  const int gc = act ? S.colx[i] + S.bxdim * S.coly[j] : 0;
  const int xo = tile_origin(x0, TX, nx, per), yo = tile_origin(y0, TY, ny, per);
  const int cx0 = x0 - xo, cy0 = y0 - yo;  // interior offset in the tile

  double wvz[11], wp[11];
  const int b0 = min(k0 - 5, nz - 11);
#pragma unroll
  for (int m = 0; m < 11; ++m) {
    const int kk = b0 + m;
    const bool ok = act && kk >= 0;
    const long long id = (long long)kk * NXY + col;
    wvz[m] = ok ? __ldg(tin + 3 * N + id) : 0.0;
    wp[m] = ok ? __ldg(tin + 4 * N + id) : 0.0;
  }
  double ke = 0.0, mr = 1e300, mp = 1e300;

  for (int k = k0; k < k1; ++k) {
    if (k > k0 && k <= nz - 6) {
      const long long id = (long long)(k + 5) * NXY + col;
      shift(wvz, act ? __ldg(tin + 3 * N + id) : 0.0);
      shift(wp, act ? __ldg(tin + 4 * N + id) : 0.0);
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
        gx = wrapi(gx, nx);
        gy = wrapi(gy, ny);
        ok = true;
      } else {
        ok = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
      }
      const long long id = kb + (long long)gy * nx + gx;
      if (iny) t_vx[ly][lx] = ok ? __ldg(tin + N + id) : 0.0;
      if (inx) t_vy[ly][lx] = ok ? __ldg(tin + 2 * N + id) : 0.0;
      t_p[ly][lx] = ok ? __ldg(tin + 4 * N + id) : 0.0;
    }
    __syncthreads();
    if (!act) continue;
    const long long id = kb + col;
    double av[5], tv[5];
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      tv[l] = __ldg(tin + l * N + id);
      av[l] = MODE == FIRST ? tv[l] : __ldg(a + l * N + id);
    }
    const double rho = tv[0], vx = tv[1], vy = tv[2], vz = tv[3], p = tv[4];
    // derivatives (RHS.f90:42-48)
    const int ry = cy0 + ty, rx = cx0 + tx;  // own tile row / column
    double dvxdx = dxy(i, nx, per, S.stretchx, [&](int g) { return t_vx[ry][g - xo]; });
    double gpx = dxy(i, nx, per, S.stretchx, [&](int g) { return t_p[ry][g - xo]; });
    double dvydy = dxy(j, ny, per, S.stretchy, [&](int g) { return t_vy[g - yo][rx]; });
    double gpy = dxy(j, ny, per, S.stretchy, [&](int g) { return t_p[g - yo][rx]; });
    const double szk = __ldg(S.stretch + k);
    double dvzdz = dz(wvz, k, nz, szk);
    double gpz = dz(wp, k, nz, szk);
    // CPML (RHS.f90:50-93); psi slots: 0 vz/vx/vy, 1 p
    if (k < S.zb.np) {
      const long long f = kb + col;
      cpml<MODE>(S.zb, f, k, 1, beta, dt, gpz);
      cpml<MODE>(S.zb, f, k, 0, beta, dt, dvzdz);
    } else if (S.zt.on && k >= nz - S.zt.np) {
      const int kl = k - (nz - S.zt.np);
      const long long f = (long long)kl * NXY + col;
      cpml<MODE>(S.zt, f, kl, 1, beta, dt, gpz);
      cpml<MODE>(S.zt, f, kl, 0, beta, dt, dvzdz);
    }
    if (S.xb.on) {
      if (i < S.xb.np) {
        const long long f = i + (long long)S.xb.np * (j + (long long)ny * k);
        cpml<MODE>(S.xb, f, i, 1, beta, dt, gpx);
        cpml<MODE>(S.xb, f, i, 0, beta, dt, dvxdx);
      } else if (i >= nx - S.xt.np) {
        const int il = i - (nx - S.xt.np);
        const long long f = il + (long long)S.xt.np * (j + (long long)ny * k);
        cpml<MODE>(S.xt, f, il, 1, beta, dt, gpx);
        cpml<MODE>(S.xt, f, il, 0, beta, dt, dvxdx);
      }
      if (j < S.yb.np) {
        const long long f = i + (long long)nx * (j + (long long)S.yb.np * k);
        cpml<MODE>(S.yb, f, j, 1, beta, dt, gpy);
        cpml<MODE>(S.yb, f, j, 0, beta, dt, dvydy);
      } else if (j >= ny - S.yt.np) {
        const int jl = j - (ny - S.yt.np);
        const long long f = i + (long long)nx * (jl + (long long)S.yt.np * k);
        cpml<MODE>(S.yt, f, jl, 1, beta, dt, gpy);
        cpml<MODE>(S.yt, f, jl, 0, beta, dt, dvydy);
      }
    }
    // RHS algebra (RHS.f90:95-152)
    const long long bi = BG1D ? (long long)k : id;
    const double r0 = __ldg(S.rho0 + bi), ri = __ldg(S.rhoinv + bi),
                 c2r = __ldg(S.c2rho0 + bi), grz = __ldg(S.grz + bi),
                 gp0 = __ldg(S.gpz + bi), sg = __ldg(S.sponge + bi);
    const double gk = __ldg(S.gblk + (long long)gc * nz + k);
    const double div = dvxdx + dvydy + dvzdz;
    double R[5];
    R[0] = -grz * vz - r0 * div - sg * rho;
    R[1] = -ri * gpx - sg * vx;
    R[2] = -ri * gpy - sg * vy;
    R[3] = -ri * (gpz + rho * gk) - vz * sg;
    if (S.frc.kind != SPARC_SRC_NONE) {
      const double frc = forcing_at(S, it, Tp, i, j, k);
      if (S.frc.dir == 1) R[1] = R[1] + frc;
      else if (S.frc.dir == 2) R[2] = R[2] + frc;
      else R[3] = R[3] + frc;
    }
    R[4] = -c2r * div - vz * gp0 - sg * p;
    // boundary planes (RHS.f90:154-164)
    const bool zero = k == 0 || k == nz - 1 ||
                      (!per && (i == 0 || i == nx - 1 || j == 0 || j == ny - 1));
    // DAMPING: the velocity RHS minus the damping term after the boundary
    // zeroing (RHS.f90:166-172), so the boundary planes move by -term
    bool zl[5] = {zero, zero, zero, zero, zero};
    if (S.term) {
#pragma unroll
      for (int l = 1; l < 4; ++l) {
        R[l] = (zero ? 0.0 : R[l]) - __ldg(S.term + (long long)(l - 1) * N + id);
        zl[l] = false;
      }
    }
    if (MODE == LAST) {
      double an[5];
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        an[l] = zl[l] ? av[l] : av[l] + dt * R[l];
        so[l * N + id] = an[l];
      }
      const double p0v = __ldg(S.p0 + bi);
      double m = (r0 + an[0]) * (an[1] * an[1] + an[2] * an[2] + an[3] * an[3]) / 2.0;
      ke += m * m;
      mr = fmin(mr, rho + r0);
      mp = fmin(mp, p + p0v);
    } else {
#pragma unroll
      for (int l = 0; l < 5; ++l) so[l * N + id] = zl[l] ? av[l] : av[l] + bnext * R[l];
    }
  }
  if (MODE == LAST) diag_reduce(S, ke, mr, mp);
}

int stage_geometry(Handle *h) {
  // tile shape: (32, 8); the quiet kernel drops to (16, 8) on grids too
  // small to fill the GPU.  The MHD kernels always use (32, 8).
  h->tx = 32;
  h->ty = 8;
  long long tiles = (long long)((h->nx + h->tx - 1) / h->tx) *
                    ((h->ny + h->ty - 1) / h->ty);
  if (tiles < 64 && !h->magnetic) {
    h->tx = 16;
    tiles = (long long)((h->nx + 15) / 16) * ((h->ny + 7) / 8);
  }
  // z chunk: about seven CTAs per SM on 148 SMs (one MHD CTA is resident per
  // SM: shorter tails; each chunk pays 10 window warm-up layers)
  const long long chunks = std::max<long long>(1, (148LL * 7 + tiles - 1) / tiles);
  int zc = (int)std::max<long long>(16, (h->nz + chunks - 1) / chunks);
  // MHD: at most 40 layers (swept 30..60 on the 256x256x300 flux tube in
  // both precisions: 40 best, 60 1.5-2 % slower, 30 1-3 % slower)
  if (h->magnetic) zc = std::min(zc, 40);
  zc = std::min(zc, h->nz);
  if (const char *kv = std::getenv("SPARC_ZCHUNK")) {  // A/B timing only
    const int v = std::atoi(kv);
    if (v >= 11) zc = std::min(v, h->nz);
  }
  h->zchunk = zc;
  h->max_stage_blocks = (int)(tiles * ((h->nz + zc - 1) / zc));
  h->partials_blocks = (int)(tiles * ((h->nz + 10) / 11));
  return SPARC_OK;
}

template <int TX, int TY>
static int launch_quiet(Handle *h, const SimDev &S, int stage,
                        const double *a, const double *tin, double *so,
                        cudaStream_t s) {
  dim3 blk(TX, TY);
  dim3 grd((h->nx + TX - 1) / TX, (h->ny + TY - 1) / TY,
           (h->nz + h->zchunk - 1) / h->zchunk);
  const double beta = h->betas[stage - 1];
  const double bnext = stage < 5 ? h->betas[stage] : h->deltat;
  const int mode = stage == 1 ? FIRST : (stage == 5 ? LAST : MID);
#define QL(M, B) k_stage_quiet<TX, TY, M, B><<<grd, blk, 0, s>>>(S, a, tin, so, beta, bnext, h->zchunk)
  if (S.bg1d) {
    if (mode == FIRST) QL(FIRST, true);
    else if (mode == MID) QL(MID, true);
    else QL(LAST, true);
  } else {
    if (mode == FIRST) QL(FIRST, false);
    else if (mode == MID) QL(MID, false);
    else QL(LAST, false);
  }
#undef QL
  return SPARC_OK;
}

int encode_tensor_maps(Handle *h) {
  h->tma = false;
  h->ftma = false;
  // rows of a multiple of 16 bytes; the filter's tiles read zero outside
  // the grid, so its maps serve non-periodic grids only
  const bool want_f = !h->periodic && !(h->nx & 1);
  const bool want_m = h->magnetic && !(h->nx & 1);
  h->ztma = false;
  const bool want_z = !(h->nx & 1);
  if (!want_f && !want_m && !want_z) return SPARC_OK;
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
          cudaSuccess || !fn || q != cudaDriverEntryPointSuccess) {
    cudaGetLastError();
    return SPARC_OK;  // the cp.async kernel serves instead
  }
  auto enc = (CUresult(*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                          const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                          const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                          CUtensorMapL2promotion, CUtensorMapFloatOOBfill))fn;
  auto boxed = [&](CUtensorMap *m, const double *base, unsigned long long depth, int bx,
                   int by) {
    cuuint64_t dims[3] = {(cuuint64_t)h->nx, (cuuint64_t)h->ny, (cuuint64_t)depth};
    cuuint64_t strides[2] = {(cuuint64_t)h->nx * 8, (cuuint64_t)h->nx * h->ny * 8};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    cuuint32_t es[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)base, dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  auto one = [&](CUtensorMap *m, const double *base, unsigned long long depth, bool halo = false) {
    return boxed(m, base, depth, halo ? MhdBuf<double, true>::HXL : mg::TX,
                 halo ? mg::HY : mg::TY);
  };
  if (want_f) {
    // FILTER_VARS xy pass: the 44 x 44 neighbourhood of a 32 x 32 tile
    bool fok = true;
    for (int b = 0; b < 3; ++b)
      fok = fok && boxed(&h->fmaps[b], h->buf[b], (unsigned long long)h->nz * h->V, fb::RX,
                         fb::RY);
    h->ftma = fok;
  }
  if (want_z) {
    // FILTER_VARS z pass: a slab of 32 x 4 columns over 44 layers of one
    // field, in a 4-D view (nx, ny, nz, V), so layers outside [0, nz) read
    // zero instead of the neighbouring field
    bool zok = true;
    for (int b = 0; b < 3 && zok; ++b) {
      cuuint64_t dims[4] = {(cuuint64_t)h->nx, (cuuint64_t)h->ny, (cuuint64_t)h->nz,
                            (cuuint64_t)h->V};
      cuuint64_t strides[3] = {(cuuint64_t)h->nx * 8, (cuuint64_t)h->nx * h->ny * 8,
                               (cuuint64_t)h->nx * h->ny * h->nz * 8};
      cuuint32_t box[4] = {(cuuint32_t)fb::ZX, (cuuint32_t)fb::ZY, (cuuint32_t)fb::ZH, 1};
      cuuint32_t es[4] = {1, 1, 1, 1};
      zok = enc(&h->zmaps[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void *)h->buf[b], dims,
                strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    }
    h->ztma = zok;
  }
  if (!want_m) return SPARC_OK;
  bool ok = true;
  for (int b = 0; b < 3; ++b) ok = ok && one(&h->tmaps_ty[b], h->buf[b], (unsigned long long)h->nz * h->V);
  const double *bg[15] = {h->red, h->sponge, h->rho0, h->grx, h->gry, h->grz, h->c2rho0,
                          h->gpx, h->gpy, h->gpz, h->rhoinv, h->cbx, h->cby, h->cbz, h->p0};
  for (int n = 0; n < 15; ++n) ok = ok && bg[n] && one(&h->tmaps_ty[3 + n], bg[n], h->nz);
  for (int b = 0; b < 3; ++b)
    ok = ok && one(&h->tmaps_ty[18 + b], h->buf[b], (unsigned long long)h->nz * h->V, true);
  const double *b0[3] = {h->box, h->boy, h->boz};
  for (int n = 0; n < 3; ++n) ok = ok && b0[n] && one(&h->tmaps_ty[21 + n], b0[n], h->nz, true);
  h->tma = ok;
  return SPARC_OK;
}

// ------------------------- MP_MHD_3D, shared-body stage kernel

// z chunk boundaries of the persistent launch: chunks of zchunk layers
// (decreasing chunk sizes, so that the last items to start are short,
// measured 1-3 % slower on the flux tube than equal chunks)
static ZSched zsched(const Handle *h) {
  ZSched Z{};
  int n = 0;
  for (int k = 0; k < h->nz && n < ZSched::MAX; k += h->zchunk) Z.b[n++] = k;
  Z.b[n] = h->nz;
  Z.n = n;
  return Z;
}

// One FP64 MHD RK stage as a single persistent launch: each CTA (one per
// SM) allocates its tensor memory once and pulls work items (32x8 tile, z
// chunk) from a device counter until the list is done.  The edge/CPML
// tiles' items come first (they are the slower ones, so the last items to
// start are short), each list chunk-major so that neighbouring tiles of a
// chunk run together; interior tiles take the branch-free body with TMA
// halo planes, the others the general body.  The diagnostics partials are
// per work item (the last stage reduces each item in the CTA and the item
// that finishes last sums them in item order), so the norm does not depend
// on which CTA took which item.
template <int MODE, bool TMA>
__global__ void __launch_bounds__(mg::NT, 1)
    k_mhd64p(const SimDev S, const __grid_constant__ TmaSet T, const double *__restrict__ a,
             const double *__restrict__ tin, double *__restrict__ so, double beta,
             double bnext, const ZSched Z, int mt, int ma, int ix0, int iy0, int nix, int nint,
             int ngen, const int2 *__restrict__ gen, unsigned *ctr) {
  const int nch = Z.n;
  extern __shared__ __align__(1024) double smem_raw64[];
  double *smem = (double *)(((size_t)smem_raw64 + 127) & ~(size_t)127);
  __shared__ uint32_t s_tmem;
  __shared__ int s_w;
  const int tid = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
  const int warp = tid / 32;
  if (warp == 0) tm_alloc_all(&s_tmem);
  tm_fence_before();
  __syncthreads();
  tm_fence_after();
  const uint32_t tbase = s_tmem, tw = tm_warp_addr(tbase, warp);
  const int ngi = ngen * nch, total = (ngen + nint) * nch;
  bool ok = true;
  for (;;) {
    if (tid == 0) s_w = (int)atomicAdd(ctr, 1u);
    __syncthreads();
    const int w = s_w;
    if (w >= total) break;
    int x0, y0, c;
    const bool in = w >= ngi;
    if (!in) {
      c = w / ngen;
      const int2 g = gen[w - c * ngen];
      x0 = g.x * mg::TX;
      y0 = g.y * mg::TY;
    } else {
      const int w2 = w - ngi;
      c = w2 / nint;
      const int t = w2 - c * nint;
      const int ty = t / nix;
      x0 = (ix0 + t - ty * nix) * mg::TX;
      y0 = (iy0 + ty) * mg::TY;
    }
    const int k0 = Z.b[c], k1 = Z.b[c + 1];
    // the body's first barrier orders every thread's read of s_w before
    // thread 0 takes the next item
    double ke = 0.0, mr = 1e300, mp = 1e300;
    if (in)
      ok = mhd_body<double, MODE, TMA, true, true>(S, &T, smem, a, tin, so, beta, bnext, x0, y0,
                                                   k0, k1, mt, ma, ke, mr, mp, tw);
    else
      ok = mhd_body<double, MODE, TMA, false, true>(S, &T, smem, a, tin, so, beta, bnext, x0,
                                                    y0, k0, k1, mt, ma, ke, mr, mp, tw);
    if (!ok) break;
    if (MODE == F_LAST) diag_reduce_t(S, ke, mr, mp, w, total);
  }
  __syncwarp();
  tm_wait_st();
  tm_fence_before();
  __syncthreads();
  tm_fence_after();
  if (warp == 0) tm_free_all(tbase);
}

// The persistent launch's plan: the edge/CPML tiles (all tiles outside the
// interior rectangle), a work counter per stage (cleared at the start of
// each step), one CTA per SM.
int mhd64_plan(Handle *h) {
  if (!h->magnetic || h->fp32) return SPARC_OK;
  const int np[4] = {h->faces[2].on ? h->faces[2].np : 0, h->faces[3].on ? h->faces[3].np : 0,
                     h->faces[4].on ? h->faces[4].np : 0, h->faces[5].on ? h->faces[5].np : 0};
  int ix0, ix1, iy0, iy1;
  mhd_interior_rect(h->nx, h->ny, np, ix0, ix1, iy0, iy1);
  const int gx = (h->nx + mg::TX - 1) / mg::TX, gy = (h->ny + mg::TY - 1) / mg::TY;
  const bool has_int = ix1 > ix0 && iy1 > iy0;
  std::vector<int2> gen;
  for (int ty = 0; ty < gy; ++ty)
    for (int tx = 0; tx < gx; ++tx)
      if (!(has_int && tx >= ix0 && tx < ix1 && ty >= iy0 && ty < iy1))
        gen.push_back(make_int2(tx, ty));
  h->gix0 = has_int ? ix0 : 0;
  h->giy0 = has_int ? iy0 : 0;
  h->gnix = has_int ? ix1 - ix0 : 0;
  h->gniy = has_int ? iy1 - iy0 : 0;
  h->ngen = (int)gen.size();
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
  h->pgrid = sms;
  h->d_wctr64 = (unsigned *)dev_alloc(h, 8 * sizeof(unsigned));
  if (!h->d_wctr64) return SPARC_ERR_NOMEM;
  if (!gen.empty()) {
    h->d_gen = (int2 *)dev_alloc(h, gen.size() * sizeof(int2));
    if (!h->d_gen) return SPARC_ERR_NOMEM;
    if (cudaMemcpy(h->d_gen, gen.data(), gen.size() * sizeof(int2), cudaMemcpyHostToDevice) !=
        cudaSuccess)
      return SPARC_ERR_CUDA;
  }
  return cudaMemset(h->d_wctr64, 0, 8 * sizeof(unsigned)) == cudaSuccess ? SPARC_OK
                                                                        : SPARC_ERR_CUDA;
}

static int launch_mhd64p(Handle *h, const SimDev &S, int stage, const double *a,
                         const double *tin, double *so, cudaStream_t s) {
  const double beta = h->betas[stage - 1];
  const double bnext = stage < 5 ? h->betas[stage] : h->deltat;
  const int mode = stage == 1 ? FIRST : (stage == 5 ? LAST : MID);
  const bool tma = h->tma && h->allow_tma64;
  const size_t sm = std::max(MhdBuf<double>::SMEM_GEN,
                             tma ? MhdBuf<double, true>::SMEM : MhdBuf<double>::SMEM_GEN);
  int mt = -1, ma = -1;
  for (int b = 0; b < 3; ++b) {
    if (h->buf[b] == tin) mt = b;
    if (h->buf[b] == a) ma = b;
  }
  if (mt < 0 || ma < 0 || !h->d_wctr64) return SPARC_ERR_INVALID;
  TmaSet T;
  if (tma)
    for (int n = 0; n < 24; ++n) T.m[n] = h->tmaps_ty[n];
  else
    std::memset(&T, 0, sizeof(T));
  const ZSched Z = zsched(h);
  const int nch = Z.n;
  const int nint = h->gnix * h->gniy;
  const long long total = (long long)(h->ngen + nint) * nch;
  const int grid = (int)std::min<long long>(h->pgrid, total);
  unsigned *ctr = h->d_wctr64 + (stage - 1);
  const dim3 blk(mg::TX, mg::TY, 2);
#define MP64(M, U)                                                                           \
  do {                                                                                       \
    cudaFuncSetAttribute(k_mhd64p<M, U>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
    k_mhd64p<M, U><<<grid, blk, sm, s>>>(S, T, a, tin, so, beta, bnext, Z, mt, ma, h->gix0,   \
                                        h->giy0, h->gnix, nint, h->ngen, h->d_gen, ctr);     \
  } while (0)
  if (tma) {
    if (mode == FIRST) MP64(F_FIRST, true);
    else if (mode == MID) MP64(F_MID, true);
    else MP64(F_LAST, true);
  } else {
    if (mode == FIRST) MP64(F_FIRST, false);
    else if (mode == MID) MP64(F_MID, false);
    else MP64(F_LAST, false);
  }
#undef MP64
  return SPARC_OK;
}

int launch_stage(Handle *h, const SimDev &S, int stage, const double *a,
                 const double *tin, double *so, cudaStream_t s) {
  int r = SPARC_ERR_INVALID;
  if (h->magnetic) {
    if (h->tx != 32 || h->ty != 8) return SPARC_ERR_INVALID;
    r = launch_mhd64p(h, S, stage, a, tin, so, s);
    ++h->launches;
    if (r == SPARC_OK && cudaGetLastError() != cudaSuccess) r = SPARC_ERR_CUDA;
    return r;
  }
  const int key = h->tx * 100 + h->ty;
#define DISPATCH(FN)                                            \
  switch (key) {                                                \
    case 3208: r = FN<32, 8>(h, S, stage, a, tin, so, s); break; \
    case 1608: r = FN<16, 8>(h, S, stage, a, tin, so, s); break; \
    default: r = SPARC_ERR_INVALID;                             \
  }
  DISPATCH(launch_quiet)
#undef DISPATCH
  ++h->launches;
  if (r == SPARC_OK && cudaGetLastError() != cudaSuccess) r = SPARC_ERR_CUDA;
  return r;
}

// ------------------------------------------------------- PULSE = 2 forcing
// all_modules.f90:592-611 / 644-660 and driver.f90:153 for the layers that
// carry any pulse: sum over the layer's pulses of
// T_n(t) * Z_n(k) * X_n(i) * Y_n(j), culled per reference rank block, twice
// at the run's first iteration, times source_damp * src_scale_beta.
struct PsrDev {
  int nx, ny, nz, klo, npulses, nblocks;
  long long init;
  double timestep, st;
  const int *off, *idx;
  const double *zv, *px, *py, *ptime, *sd, *ssb;
  const unsigned char *mask;
  const int *colx, *coly, *colz;
  int bx, bxy;
  double *out;
  const long long *iter;
};

__global__ void k_psr(PsrDev D) {
  extern __shared__ double sh[];
  const int k = D.klo + blockIdx.z;
  const int e0 = D.off[k], e1 = D.off[k + 1], ne = e1 - e0;
  double *sT = sh;
  int *sN = (int *)(sh + ne);
  const long long it = *D.iter;
  const double t = (double)it * D.timestep;
  const double passes = (it == D.init) ? 2.0 : 1.0;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  for (int e = tid; e < ne; e += blockDim.x * blockDim.y) {
    const int n = D.idx[e0 + e];
    const double amp = D.ptime[3 * n], t0 = D.ptime[3 * n + 1],
                 t1 = D.ptime[3 * n + 2];
    double v = amp * sin(2.0 * PI * (t - t1) / t0);
    v = v * exp(-((t - t1) * (t - t1)) / (2.0 * (D.st * D.st)));
    sT[e] = v * D.zv[e0 + e] * passes;
    sN[e] = n;
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= D.nx || j >= D.ny) return;
  const int blk = D.colx[i] + D.bx * D.coly[j] + D.bxy * D.colz[k];
  double f = 0.0;
  for (int e = 0; e < ne; ++e) {
    const int n = sN[e];
    if (!D.mask[(long long)n * D.nblocks + blk]) continue;
    f = f + sT[e] * (D.px[(long long)n * D.nx + i] * D.py[(long long)n * D.ny + j]);
  }
  const long long g = ((long long)k * D.ny + j) * D.nx + i;
  D.out[((long long)blockIdx.z * D.ny + j) * D.nx + i] = f * D.sd[g] * D.ssb[g];
}

int launch_psr_forcing(Handle *h, const SimDev &S, cudaStream_t s);

// ------------------------------------------------------ FILTER_VARS
// FILTER_VARS of a filter event (filter_body.cuh): the fused y-then-x pass
// (blockIdx.z: field and a group of LPB layers, pipelined)
template <int G, bool TMA>
__global__ void __launch_bounds__(fb::NT, 4)
    k_filt_xy64(FiltArgs<double> F, const __grid_constant__ CUtensorMap map) {
  const int nzc = (F.nz + fb::LPB - 1) / fb::LPB;
  const int l = blockIdx.z / nzc, k0 = (blockIdx.z - l * nzc) * fb::LPB;
  filt_xy_layers<double, G, TMA>(F, l, k0, min(fb::LPB, F.nz - k0), blockIdx.x * fb::TX,
                                 blockIdx.y * fb::TR, &map);
}
// the z pass: blockIdx.x is the z chunk (the chunks of a slab run
// together), blockIdx.y the slab of the layer, blockIdx.z the field
// (the launch gives 128 bytes of slack for a 128-byte aligned slab and 16
// for the mbarrier after it)
template <int G, bool TMA>
__global__ void __launch_bounds__(2 * fb::ZX * fb::ZY)
    k_filt_z64(FiltArgs<double> F, const __grid_constant__ CUtensorMap map) {
  extern __shared__ __align__(128) unsigned char zraw64[];
  double *zsl = (double *)(zraw64 + ((128u - (sm_addr_t(zraw64) & 127u)) & 127u));
  const int nxb = (F.nx + fb::ZX - 1) / fb::ZX;
  const int yb = blockIdx.y / nxb, xb = blockIdx.y - yb * nxb;
  filt_z_slab<double, G, false, false, TMA>(F, blockIdx.z, xb * fb::ZX, yb * fb::ZY,
                                            blockIdx.x * fb::ZC, zsl, &map);
}

// xy: the y and x passes fused; z: the z pass (in -> out, never in place)
int launch_filter_event(Handle *h, bool xy, const double *in, double *out, cudaStream_t s) {
  FiltArgs<double> F{};
  F.nx = h->nx; F.ny = h->ny; F.nz = h->nz; F.V = h->V; F.N = h->N;
  F.periodic = h->periodic ? 1 : 0;
  F.s = xy ? h->P.s_xy : h->P.s_z;
  F.in = in;
  F.out = out;
  F.err = h->d_err;
  const int g = xy ? h->gxy : h->gz;
  if (xy) {
    const dim3 grid((h->nx + fb::TX - 1) / fb::TX, (h->ny + fb::TR - 1) / fb::TR,
                    h->V * ((h->nz + fb::LPB - 1) / fb::LPB));
    // the tensor map of the input buffer (neighbourhoods by TMA), if any
    int mb = -1;
    if (h->ftma)
      for (int b = 0; b < 3; ++b)
        if (h->buf[b] == in) mb = b;
    CUtensorMap map;
    if (mb >= 0) map = h->fmaps[mb];
    else std::memset(&map, 0, sizeof(map));
    const dim3 blk(fb::TX, fb::TY);
    if (mb >= 0) {
      if (g == 5) k_filt_xy64<5, true><<<grid, blk, 0, s>>>(F, map);
      else k_filt_xy64<3, true><<<grid, blk, 0, s>>>(F, map);
    } else {
      if (g == 5) k_filt_xy64<5, false><<<grid, blk, 0, s>>>(F, map);
      else k_filt_xy64<3, false><<<grid, blk, 0, s>>>(F, map);
    }
  } else {
    const size_t zs = filt_z_smem<double>() + 128 + 16;
    const long long slabs = (long long)((h->nx + fb::ZX - 1) / fb::ZX) *
                            ((h->ny + fb::ZY - 1) / fb::ZY);
    if (slabs > 65535) return SPARC_ERR_INVALID;
    const dim3 grid((h->nz + fb::ZC - 1) / fb::ZC, (unsigned)slabs, h->V);
    // the tensor map of the input buffer (slabs by TMA), if any
    int mb = -1;
    if (h->ztma)
      for (int b = 0; b < 3; ++b)
        if (h->buf[b] == in) mb = b;
    CUtensorMap map;
    if (mb >= 0) map = h->zmaps[mb];
    else std::memset(&map, 0, sizeof(map));
    const dim3 blk(fb::ZX, fb::ZY, 2);
#define ZP(GG, TT)                                                                          \
  do {                                                                                      \
    cudaFuncSetAttribute(k_filt_z64<GG, TT>, cudaFuncAttributeMaxDynamicSharedMemorySize,   \
                         (int)zs);                                                          \
    k_filt_z64<GG, TT><<<grid, blk, zs, s>>>(F, map);                                       \
  } while (0)
    if (mb >= 0) {
      if (g == 5) ZP(5, true);
      else ZP(3, true);
    } else {
      if (g == 5) ZP(5, false);
      else ZP(3, false);
    }
#undef ZP
  }
  ++h->launches;
  return cudaGetLastError() == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

// Both stencils stay resident, so handles with different filter modes can
// coexist; a pass picks its table by half-width.
int filter_constants() {
  double t[2][11] = {};
  for (int m = 0; m < 11; ++m) t[0][m] = kFilter11[m];
  for (int m = 0; m < 7; ++m) t[1][m] = kFilter7[m];
  return cudaMemcpyToSymbol(c_df, t, sizeof(t)) == cudaSuccess ? SPARC_OK
                                                               : SPARC_ERR_CUDA;
}

// PULSE = 0: the forcing plane of the device's iteration
// (random_forcing.cuh), one value per column.
template <class D, class T>
__global__ void k_random(const double *__restrict__ vr, const D *__restrict__ damp, int nxy,
                         int ns, double timestep, double cad, const long long *iter,
                         T *__restrict__ out) {
  const RndStencil R = rnd_stencil(*iter, timestep, cad, ns);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nxy; q += gridDim.x * blockDim.x)
    out[q] = (T)rnd_column(R, vr, nxy, q, damp[q]);
}

int launch_random_forcing(Handle *h, cudaStream_t s) {
  if (h->src.kind != SPARC_SRC_RANDOM) return SPARC_OK;
  const int nxy = h->nx * h->ny;
  const int grid = std::min((nxy + 255) / 256, 4 * 148);
  if (h->fp32)
    k_random<float, float><<<grid, 256, 0, s>>>(h->d_series, h->f_sd, nxy, h->src.nseries,
                                               h->P.timestep, h->src.cadforcing, h->d_iter,
                                               h->f_f2d);
  else
    k_random<double, double><<<grid, 256, 0, s>>>(h->d_series, h->source_damp, nxy,
                                                 h->src.nseries, h->P.timestep,
                                                 h->src.cadforcing, h->d_iter, h->d_f2d);
  ++h->launches;
  return cudaGetLastError() == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

int launch_psr_forcing(Handle *h, const SimDev &S, cudaStream_t s) {
  (void)S;
  if (h->src.kind != SPARC_SRC_PSR || h->psr_khi <= h->psr_klo) return SPARC_OK;
  PsrDev D;
  D.nx = h->nx; D.ny = h->ny; D.nz = h->nz;
  D.klo = h->psr_klo;
  D.npulses = (int)h->pulses.size();
  D.nblocks = h->nblocks;
  D.init = h->src.init;
  D.timestep = h->P.timestep;
  D.st = h->src.psr_st;
  D.off = h->d_plane_off;
  D.idx = h->d_plane_idx;
  D.zv = h->d_plane_z;
  D.px = h->d_px;
  D.py = h->d_py;
  D.ptime = h->d_ptime;
  D.sd = h->source_damp;
  D.ssb = h->ssb;
  D.mask = h->d_pmask;
  D.colx = h->d_colx;
  D.coly = h->d_coly;
  D.colz = h->d_colx + h->nx + h->ny;  // packed after colx, coly
  D.bx = h->P.block_x;
  D.bxy = h->P.block_x * h->P.block_y;
  D.out = h->d_psr;
  D.iter = h->d_iter;
  dim3 blk(32, 8);
  dim3 grd((h->nx + 31) / 32, (h->ny + 7) / 8, h->psr_khi - h->psr_klo);
  size_t smem = (size_t)D.npulses * (sizeof(double) + sizeof(int));
  k_psr<<<grd, blk, smem, s>>>(D);
  ++h->launches;
  return cudaGetLastError() == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

SimDev make_simdev(Handle *h) {
  SimDev S{};
  S.nx = h->nx; S.ny = h->ny; S.nz = h->nz; S.N = h->N;
  S.periodic = h->periodic ? 1 : 0;
  S.magnetic = h->magnetic ? 1 : 0;
  S.bg1d = h->bg1d ? 1 : 0;
  S.sponge_slabs = h->sponge_slabs ? 1 : 0;
  S.V = h->V;
  S.stretchx = h->stretchx;
  S.stretchy = h->stretchy;
  S.stretch = h->d_stretch;
  S.deltat = h->deltat;
  S.dimc2rho = (h->dimc * h->dimc) * h->dimrho;
  S.term = h->damping ? h->d_term : nullptr;
  if (h->bg1d) {
    S.rho0 = h->rho0_1; S.p0 = h->p0_1; S.rhoinv = h->rhoinv_1;
    S.c2rho0 = h->c2rho0_1; S.grz = h->grz_1; S.gpz = h->gpz_1;
    S.sponge = h->sponge_1;
  } else {
    S.rho0 = h->rho0; S.p0 = h->p0; S.rhoinv = h->rhoinv;
    S.c2rho0 = h->c2rho0; S.grz = h->grz; S.gpz = h->gpz;
    S.sponge = h->sponge;
  }
  S.box = h->box; S.boy = h->boy; S.boz = h->boz;
  S.cbx = h->cbx; S.cby = h->cby; S.cbz = h->cbz;
  S.grx = h->grx; S.gry = h->gry; S.gpx = h->gpx; S.gpy = h->gpy;
  S.red = h->red;
  S.gblk = h->d_gblk;
  S.colx = h->d_colx;
  S.coly = h->d_coly;
  S.bxdim = h->P.block_x;
  S.zb = h->faces[0]; S.zt = h->faces[1];
  S.xb = h->faces[2]; S.xt = h->faces[3];
  S.yb = h->faces[4]; S.yt = h->faces[5];
  ForcingDev &F = S.frc;
  F.kind = h->src.kind;
  F.dir = h->src.dir;
  F.init = h->src.init;
  F.fx = h->d_fx; F.fy = h->d_fy; F.fz = h->d_fz;
  F.amp_c = h->src.amp / 0.56458272 / h->dimc;
  F.t0 = h->src.t0; F.t1 = h->src.t1; F.st = h->src.st;
  F.timestep = h->P.timestep;
  F.psr = h->d_psr;
  F.klo = h->psr_klo;
  F.khi = h->psr_khi;
  F.f2d = h->d_f2d;
  F.sdep = h->d_sdep;
  S.iter = h->d_iter;
  S.err = h->d_err;
  S.partials = h->d_partials;
  S.counter = h->d_counter;
  S.diag = h->d_diag;
  S.fail_iter = h->d_fail;
  return S;
}

}  // namespace sparc
