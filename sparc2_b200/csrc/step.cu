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

#include "mhd_body.cuh"

namespace sparc {

__constant__ double c_dp[6][11];   // derivative rows, initialize.f90:1959-2031
__constant__ double c_df[2][11];   // filter stencils: [0] 11-point, [1] 7-point

enum { FIRST = 0, MID = 1, LAST = 2 };

template <>
__device__ __forceinline__ double dcoef<double>(int r, int m) {
  return c_dp[r][m];
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

// value of layer k held in a window whose base is b
__device__ __forceinline__ double wsel(const double (&w)[11], int off) {
  double v = w[5];
#pragma unroll
  for (int m = 0; m < 11; ++m)
    if (m == off) v = w[m];
  return v;
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
    if (MODE == LAST) {
      double an[5];
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        an[l] = zero ? av[l] : av[l] + dt * R[l];
        so[l * N + id] = an[l];
      }
      const double p0v = __ldg(S.p0 + bi);
      double m = (r0 + an[0]) * (an[1] * an[1] + an[2] * an[2] + an[3] * an[3]) / 2.0;
      ke += m * m;
      mr = fmin(mr, rho + r0);
      mp = fmin(mp, p + p0v);
    } else {
#pragma unroll
      for (int l = 0; l < 5; ++l) so[l * N + id] = zero ? av[l] : av[l] + bnext * R[l];
    }
  }
  if (MODE == LAST) diag_reduce(S, ke, mr, mp);
}

// ------------------------------------ MP_MHD_3D, pipelined stage kernel
// Shared-memory layout of the pipelined MHD kernels: every
// array a layer needs is copied into shared memory with cp.async one layer
// ahead (double buffer), so the loads of layer k+1 stream while layer k is
// computed.  Per buffer: 10 halo slots over the cross-shaped tile (stage
// fields vx vy vz p bx by bz and B0; the B0 slots become flux1..3 in place
// once the layer has landed) and 24 own-point slots (stage rho, a[0..7],
// 14 background arrays, p0).
namespace pipe {
// own slots
constexpr int O_RHO = 0, O_A = 1, O_BG = 9, O_P0 = 23;
// background order in the own slots (O_BG + n)
enum { B_RED, B_SPONGE, B_RHO0, B_GRX, B_GRY, B_GRZ, B_C2R, B_GPX, B_GPY,
       B_GPZ, B_RHOINV, B_CBX, B_CBY, B_CBZ, NBG };
}  // namespace pipe

__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async16(double *dst, const double *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_wait1() {
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

// ------------------------- MP_MHD_3D, two-role pipelined stage kernel
// The pipelined layer tiles of k_stage_mhd_pipe, with each column served by
// two warps-groups (threadIdx.z = role) so that a thread holds only three
// z windows (66 FP64 registers) and the CTA keeps 16 warps resident:
//   role 0: momentum (RHS.f90:570-580, 630-645); windows vz, p, bx;
//           derivatives gpx gpy gpz dvzdz dybz dxbz dzbx dxby dybx
//   role 1: continuity, pressure, induction (RHS.f90:548-568); windows
//           flux1, flux2, by; derivatives dvxdx dvydy dxflux3 dxflux2
//           dyflux3 dyflux1 dzflux1 dzflux2 dzby
// dvzdz and dzby cross over through shared memory after their CPML
// corrections.  Arithmetic and summation order follow RHS.f90 as in the
// oracle (11-tap sums from the first tap, operand order of each term).
namespace duo {
constexpr int TX = 32, TY = 8, NC = TX * TY, NT = 2 * NC;
constexpr int HX = TX + 10, HY = TY + 10, HS = HX * HY;
constexpr int NH = 10, NO = 24;
constexpr int BUF = NH * HS + NO * NC;
constexpr int XCH = 3 * NC;                       // exchange slots
constexpr size_t SMEM = (2 * BUF + XCH) * sizeof(double);
}  // namespace duo

template <int MODE>
__global__ void __launch_bounds__(duo::NT, 1)
    k_stage_mhd_duo(const SimDev S, const double *__restrict__ a,
                    const double *__restrict__ tin, double *__restrict__ so,
                    double beta, double bnext, int zchunk) {
  using namespace duo;
  using pipe::O_RHO;
  using pipe::O_A;
  using pipe::O_BG;
  using pipe::O_P0;
  extern __shared__ double smem[];
  __shared__ const double *optr[NO];
  const int tx = threadIdx.x, ty = threadIdx.y, role = threadIdx.z;
  const int tid = (role * TY + ty) * TX + tx, cid = ty * TX + tx;
  const int nx = S.nx, ny = S.ny, nz = S.nz;
  const long long N = S.N, NXY = (long long)nx * ny;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int i = x0 + tx, j = y0 + ty;
  const bool act = i < nx && j < ny;
  const bool per = S.periodic;
  const int k0 = blockIdx.z * zchunk, k1 = min(nz, k0 + zchunk);
  const long long col = (long long)j * nx + i;
  const long long it = *S.iter;
  const double dt = S.deltat;
  const int xo = tile_origin(x0, TX, nx, per), yo = tile_origin(y0, TY, ny, per);
  const int cx0 = x0 - xo, cy0 = y0 - yo;
  const int ry = cy0 + ty, rx = cx0 + tx;
  const bool vec2 = (nx & 1) == 0;
  if (tid == 0) {
    optr[O_RHO] = tin;
    for (int l = 0; l < 8; ++l) optr[O_A + l] = a + l * N;
    optr[O_BG + pipe::B_RED] = S.red;    optr[O_BG + pipe::B_SPONGE] = S.sponge;
    optr[O_BG + pipe::B_RHO0] = S.rho0;  optr[O_BG + pipe::B_GRX] = S.grx;
    optr[O_BG + pipe::B_GRY] = S.gry;    optr[O_BG + pipe::B_GRZ] = S.grz;
    optr[O_BG + pipe::B_C2R] = S.c2rho0; optr[O_BG + pipe::B_GPX] = S.gpx;
    optr[O_BG + pipe::B_GPY] = S.gpy;    optr[O_BG + pipe::B_GPZ] = S.gpz;
    optr[O_BG + pipe::B_RHOINV] = S.rhoinv;
    optr[O_BG + pipe::B_CBX] = S.cbx;    optr[O_BG + pipe::B_CBY] = S.cby;
    optr[O_BG + pipe::B_CBZ] = S.cbz;
    optr[O_P0] = S.p0;
  }
  __syncthreads();
  auto H = [&](int b, int slot, int ly, int lx) -> double & {
    return smem[b * BUF + (slot * HY + ly) * HX + lx];
  };
  auto O = [&](int b, int slot) -> double & {
    return smem[b * BUF + NH * HS + slot * NC + cid];
  };
  double *X = smem + 2 * BUF;  // [0] dvzdz, [1] dzby, [2] |v_new|^2
  auto own_active = [&](int slot) -> bool {
    if (slot >= O_A && slot < O_BG) return MODE != FIRST;
    if (slot == O_P0) return MODE == LAST;
    return true;
  };
  auto issue = [&](int k, int b) {
    const long long kb = (long long)k * NXY;
    for (int t = tid; t < HS; t += NT) {
      const int ly = t / HX, lx = t - ly * HX;
      const bool inx = lx >= cx0 && lx < cx0 + TX, iny = ly >= cy0 && ly < cy0 + TY;
      if (!inx && !iny) continue;
      int gx = xo + lx, gy = yo + ly;
      if (per) {
        gx = wrapi(gx, nx);
        gy = wrapi(gy, ny);
      } else if (gx < 0 || gx >= nx || gy < 0 || gy >= ny) {
        continue;
      }
      const long long id = kb + (long long)gy * nx + gx;
#pragma unroll
      for (int sl = 0; sl < 7; ++sl) cp_async8(&H(b, sl, ly, lx), tin + (sl + 1) * N + id);
      cp_async8(&H(b, 7, ly, lx), S.box + id);
      cp_async8(&H(b, 8, ly, lx), S.boy + id);
      cp_async8(&H(b, 9, ly, lx), S.boz + id);
    }
    double *ob = smem + b * BUF + NH * HS;
    if (vec2) {
      constexpr int PAIRS = NC / 2;
      for (int t = tid; t < NO * PAIRS; t += NT) {
        const int slot = t / PAIRS, rem = t - slot * PAIRS;
        if (!own_active(slot)) continue;
        const int r = rem / (TX / 2), c = 2 * (rem - r * (TX / 2));
        const int gx = x0 + c, gy = y0 + r;
        if (gx >= nx || gy >= ny) continue;
        cp_async16(ob + slot * NC + r * TX + c, optr[slot] + kb + (long long)gy * nx + gx);
      }
    } else {
      for (int t = tid; t < NO * NC; t += NT) {
        const int slot = t / NC, rem = t - slot * NC;
        if (!own_active(slot)) continue;
        const int r = rem / TX, c = rem - r * TX;
        const int gx = x0 + c, gy = y0 + r;
        if (gx >= nx || gy >= ny) continue;
        cp_async8(ob + slot * NC + r * TX + c, optr[slot] + kb + (long long)gy * nx + gx);
      }
    }
    cp_commit();
  };

  // role 0 windows: vz, p, bx ; role 1 windows: flux1, flux2, by
  double w0[11], w1[11], w2[11];
  auto head = [&](int kk, double &v0, double &v1, double &v2) {
    const long long id = (long long)kk * NXY + col;
    if (role == 0) {
      v0 = __ldg(tin + 3 * N + id);
      v1 = __ldg(tin + 4 * N + id);
      v2 = __ldg(tin + 5 * N + id);
    } else {
      const double vx_ = __ldg(tin + N + id), vy_ = __ldg(tin + 2 * N + id),
                   vz_ = __ldg(tin + 3 * N + id);
      const double ox = __ldg(S.box + id), oy = __ldg(S.boy + id),
                   oz = __ldg(S.boz + id);
      v0 = -vz_ * oy + vy_ * oz;       // flux1
      v1 = -vx_ * oz + vz_ * ox;       // flux2
      v2 = __ldg(tin + 6 * N + id);    // by
    }
  };
  issue(k0, 0);
  const int b0 = min(k0 - 5, nz - 11);
#pragma unroll
  for (int m = 0; m < 11; ++m) {
    const int kk = b0 + m;
    if (act && kk >= 0) head(kk, w0[m], w1[m], w2[m]);
    else w0[m] = w1[m] = w2[m] = 0.0;
  }
  double h0 = 0, h1 = 0, h2 = 0;
  double ke = 0.0, mr = 1e300, mp = 1e300;

  for (int k = k0; k < k1; ++k) {
    const int b = (k - k0) & 1;
    if (k > k0 && k <= nz - 6) {
      shift(w0, h0); shift(w1, h1); shift(w2, h2);
    }
    if (k + 1 < k1) issue(k + 1, b ^ 1);
    else cp_commit();
    cp_wait1();
    __syncthreads();
    const double ox = H(b, 7, ry, rx), oy = H(b, 8, ry, rx), oz = H(b, 9, ry, rx);
    __syncthreads();
    for (int t = tid; t < HS; t += NT) {
      const int ly = t / HX, lx = t - ly * HX;
      const bool inx = lx >= cx0 && lx < cx0 + TX, iny = ly >= cy0 && ly < cy0 + TY;
      if (!inx && !iny) continue;
      const double vx_ = H(b, 0, ly, lx), vy_ = H(b, 1, ly, lx), vz_ = H(b, 2, ly, lx);
      const double bx0 = H(b, 7, ly, lx), by0 = H(b, 8, ly, lx), bz0 = H(b, 9, ly, lx);
      H(b, 7, ly, lx) = -vz_ * by0 + vy_ * bz0;
      H(b, 8, ly, lx) = -vx_ * bz0 + vz_ * bx0;
      H(b, 9, ly, lx) = -vy_ * bx0 + vx_ * by0;
    }
    __syncthreads();
    const long long id = (long long)k * NXY + col;
    const double szk = __ldg(S.stretch + k);
    auto DX = [&](int slot) {
      return dxy(i, nx, per, S.stretchx, [&](int g) { return H(b, slot, ry, g - xo); });
    };
    auto DY = [&](int slot) {
      return dxy(j, ny, per, S.stretchy, [&](int g) { return H(b, slot, g - yo, rx); });
    };
    const bool zpml = S.zb.on && (k < S.zb.np || k >= nz - S.zt.np);
    const bool zbot = k < S.zb.np;
    const FaceDev &FZ = zbot ? S.zb : S.zt;
    const int kl = zbot ? k : k - (nz - S.zt.np);
    const long long fz = (long long)kl * NXY + col;
    const bool xpml = S.xb.on && act && (i < S.xb.np || i >= nx - S.xt.np);
    const bool xbot = i < S.xb.np;
    const FaceDev &FX = xbot ? S.xb : S.xt;
    const int il = xbot ? i : i - (nx - S.xt.np);
    const long long fx = il + (long long)FX.np * (j + (long long)ny * k);
    const bool ypml = S.xb.on && act && (j < S.yb.np || j >= ny - S.yt.np);
    const bool ybot = j < S.yb.np;
    const FaceDev &FY = ybot ? S.yb : S.yt;
    const int jl = ybot ? j : j - (ny - S.yt.np);
    const long long fy = i + (long long)nx * (jl + (long long)FY.np * k);
    const bool zero = k == 0 || k == nz - 1 ||
                      (!per && (i == 0 || i == nx - 1 || j == 0 || j == ny - 1));
    // halo slots: 0 vx, 1 vy, 2 vz, 3 p, 4 bx, 5 by, 6 bz, 7-9 flux1..3
    // phase A: the role's nine derivatives with their CPML corrections.
    // role 0: d0 gpx d1 gpy d2 gpz d3 dvzdz d4 dybz d5 dxbz d6 dzbx d7 dxby d8 dybx
    // role 1: d0 dvxdx d1 dvydy d2 dxflux3 d3 dxflux2 d4 dyflux3 d5 dyflux1
    //         d6 dzflux1 d7 dzflux2 d8 dzby
    double d0 = 0, d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0, d6 = 0, d7 = 0, d8 = 0;
    if (act) {
      if (role == 0) {
        d0 = DX(3); d5 = DX(6); d7 = DX(5);
        d1 = DY(3); d4 = DY(6); d8 = DY(4);
        d3 = dz(w0, k, nz, szk); d2 = dz(w1, k, nz, szk); d6 = dz(w2, k, nz, szk);
        if (zpml) {
          cpml<MODE>(FZ, fz, kl, 1, beta, dt, d2);
          cpml<MODE>(FZ, fz, kl, 0, beta, dt, d3);
          cpml<MODE>(FZ, fz, kl, 2, beta, dt, d6);
        }
        if (xpml) {
          cpml<MODE>(FX, fx, il, 1, beta, dt, d0);
          cpml<MODE>(FX, fx, il, 3, beta, dt, d5);
          cpml<MODE>(FX, fx, il, 2, beta, dt, d7);
        }
        if (ypml) {
          cpml<MODE>(FY, fy, jl, 1, beta, dt, d1);
          cpml<MODE>(FY, fy, jl, 3, beta, dt, d4);
          cpml<MODE>(FY, fy, jl, 2, beta, dt, d8);
        }
        X[cid] = d3;          // dvzdz for role 1
      } else {
        d0 = DX(0); d2 = DX(9); d3 = DX(8);
        d1 = DY(1); d4 = DY(9); d5 = DY(7);
        d6 = dz(w0, k, nz, szk); d7 = dz(w1, k, nz, szk); d8 = dz(w2, k, nz, szk);
        if (zpml) {
          cpml<MODE>(FZ, fz, kl, 4, beta, dt, d7);
          cpml<MODE>(FZ, fz, kl, 5, beta, dt, d6);
          cpml<MODE>(FZ, fz, kl, 3, beta, dt, d8);
        }
        if (xpml) {
          cpml<MODE>(FX, fx, il, 0, beta, dt, d0);
          cpml<MODE>(FX, fx, il, 4, beta, dt, d2);
          cpml<MODE>(FX, fx, il, 5, beta, dt, d3);
        }
        if (ypml) {
          cpml<MODE>(FY, fy, jl, 0, beta, dt, d1);
          cpml<MODE>(FY, fy, jl, 4, beta, dt, d4);
          cpml<MODE>(FY, fy, jl, 5, beta, dt, d5);
        }
        X[NC + cid] = d8;     // dzby for role 0
      }
    }
    __syncthreads();
    // phase B: right-hand sides and the stage (or final) update
    double an_rho = 0.0;
    if (act) {
      const double rho = O(b, O_RHO), vx = H(b, 0, ry, rx), vy = H(b, 1, ry, rx),
                   vz = H(b, 2, ry, rx);
      const double red = O(b, O_BG + pipe::B_RED), sg = O(b, O_BG + pipe::B_SPONGE);
      if (role == 0) {
        const double bx = H(b, 4, ry, rx), by = H(b, 5, ry, rx), bz = H(b, 6, ry, rx);
        const double dzby = X[NC + cid];
        const double cbx = d4 - dzby, cby = -d5 + d6, cbz = d7 - d8;
        const double c1 = cby * oz - cbz * oy, c2 = ox * cbz - cbx * oz,
                     c3 = cbx * oy - cby * ox;
        const double ri = O(b, O_BG + pipe::B_RHOINV);
        double vxr = -ri * (d0 - (c1 * red)) - sg * vx;
        double vyr = -ri * (d1 - (c2 * red)) - sg * vy;
        double vzr = -ri * (d2 - (c3 * red)) - sg * vz;
        const double qx = O(b, O_BG + pipe::B_CBX), qy = O(b, O_BG + pipe::B_CBY),
                     qz = O(b, O_BG + pipe::B_CBZ);
        const double e1 = qy * bz - qz * by, e2 = bx * qz - qx * bz,
                     e3 = qx * by - qy * bx;
        vxr = vxr + ri * e1 * red;
        vyr = vyr + ri * e2 * red;
        vzr = vzr + ri * e3 * red;
        const int gc = S.colx[i] + S.bxdim * S.coly[j];
        vzr = vzr - ri * rho * __ldg(S.gblk + (long long)gc * nz + k);
        if (S.frc.kind != SPARC_SRC_NONE) {
          const double frc = forcing_at(S, it, pulse_time(S, it), i, j, k);
          if (S.frc.dir == 1) vxr = vxr + frc;
          else if (S.frc.dir == 2) vyr = vyr + frc;
          else vzr = vzr + frc;
        }
        const double R[3] = {vxr, vyr, vzr};
        double vsq = 0.0;
#pragma unroll
        for (int l = 1; l < 4; ++l) {
          const double av = MODE == FIRST ? H(b, l - 1, ry, rx) : O(b, O_A + l);
          const double an = zero ? av : av + (MODE == LAST ? dt : bnext) * R[l - 1];
          so[l * N + id] = an;
          vsq = l == 1 ? an * an : vsq + an * an;
        }
        if (MODE == LAST) X[2 * NC + cid] = vsq;
      } else {
        const double p = H(b, 3, ry, rx);
        const double dvzdz = X[cid];
        double R[5];  // rho, p, bx, by, bz
        R[2] = red * (d4 - d7);
        R[3] = red * (d6 - d2);
        R[4] = red * (d3 - d5);
        const double div = d0 + d1 + dvzdz;
        const double r0 = O(b, O_BG + pipe::B_RHO0);
        R[0] = -O(b, O_BG + pipe::B_GRX) * vx - O(b, O_BG + pipe::B_GRY) * vy -
               O(b, O_BG + pipe::B_GRZ) * vz - r0 * div - sg * rho;
        R[1] = -O(b, O_BG + pipe::B_C2R) * div - vx * O(b, O_BG + pipe::B_GPX) -
               vy * O(b, O_BG + pipe::B_GPY) - vz * O(b, O_BG + pipe::B_GPZ) - sg * p;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          const int l = q == 0 ? 0 : q + 3;   // fields rho, p(4), bx(5), by(6), bz(7)
          const int ls = q == 1 ? 4 : l;
          const double av = MODE == FIRST ? (ls == 0 ? rho : H(b, ls - 1, ry, rx))
                                          : O(b, O_A + ls);
          const double an = zero ? av : av + (MODE == LAST ? dt : bnext) * R[q];
          so[ls * N + id] = an;
          if (q == 0) an_rho = an;
        }
        if (MODE == LAST) {
          mr = fmin(mr, rho + r0);
          mp = fmin(mp, p + O(b, O_P0));
        }
      }
    }
    if (MODE == LAST) {
      __syncthreads();
      if (act && role == 1) {  // KE density of driver.f90:161 on a_new
        const double r0 = O(b, O_BG + pipe::B_RHO0);
        const double m = (r0 + an_rho) * X[2 * NC + cid] / 2.0;
        ke += m * m;
      }
    }
    if (act && k + 1 < k1 && k + 1 <= nz - 6) head(k + 6, h0, h1, h2);
    __syncthreads();
  }
  if (MODE == LAST) diag_reduce(S, ke, mr, mp);
}

// --------------------- MP_MHD_3D, two-role stage kernel with TMA loads
// k_stage_mhd_duo with the 24 own-point arrays of a layer fetched by TMA
// (one elected thread, 3-D tensor maps, 32x8 boxes, one mbarrier per
// buffer) instead of per-thread copies, halo copy addresses computed once
// per CTA, and branch-free centred x/y stencils for interior columns.
// Shared memory per buffer: 24 own slots (2 KB each, 128-B aligned) then
// the 10 halo slots.  Needs an even nx (16-B row strides).
struct TmaSet {
  CUtensorMap m[18];
};

namespace tmak {
constexpr long long WAIT_LIMIT = 1LL << 26;
}  // namespace tmak
// geometry of the TMA kernel for a tile height TY (tile 32 x TY columns,
// two roles -> 64*TY threads)
template <int TY_>
struct TmaGeo {
  static constexpr int TX = 32, TY = TY_, NC = TX * TY, NT = 2 * NC;
  static constexpr int HX = TX + 10, HY = TY + 10, HS = HX * HY;
  static constexpr int NH = 10, NO = 24;
  static constexpr int BUF = ((NO * NC + NH * HS) + 15) / 16 * 16;  // 128-B multiple
  static constexpr int XCH = 3 * NC;
  static constexpr size_t SMEM = (2 * (size_t)BUF + XCH) * sizeof(double) + 128;
};

__device__ __forceinline__ unsigned sm_addr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sm_addr(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sm_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_load_3d(double *dst, const CUtensorMap *map, int x,
                                            int y, int z, unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(sm_addr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(sm_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(sm_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: false (and the error flag set) if the copies never land
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity,
                                          int *err) {
  for (long long n = 0; n < tmak::WAIT_LIMIT; ++n)
    if (mbar_try_wait(bar, parity)) return true;
  atomicExch(err, 1);
  return false;
}

// centred 11-point sum along a shared-memory line with element stride st
__device__ __forceinline__ double csum(const double *p, int st) {
  double s = 0.0;
#pragma unroll
  for (int m = 0; m < 11; ++m) s += p[m * st] * c_dp[5][m];
  return s;
}

template <int MODE, int TYV>
__global__ void __launch_bounds__(TmaGeo<TYV>::NT, 1)
    k_stage_mhd_tma(const SimDev S, const __grid_constant__ TmaSet T,
                    const double *__restrict__ a, const double *__restrict__ tin,
                    double *__restrict__ so, double beta, double bnext,
                    int zchunk, int mt, int ma) {
  // 32-bit indexing throughout (the launcher checks V*N < 2^31)
  using G = TmaGeo<TYV>;
  constexpr int TX = G::TX, TY = G::TY, NC = G::NC, NT = G::NT, HX = G::HX,
                HS = G::HS, NO = G::NO, BUF = G::BUF;
  using pipe::O_RHO;
  using pipe::O_A;
  using pipe::O_BG;
  using pipe::O_P0;
  extern __shared__ __align__(1024) double smem_raw[];
  __shared__ unsigned long long bar[2];
  const int tx = threadIdx.x, ty = threadIdx.y, role = threadIdx.z;
  const int tid = (role * TY + ty) * TX + tx, cid = ty * TX + tx;
  double *smem = (double *)(((size_t)smem_raw + 127) & ~(size_t)127);
  if (sm_addr(smem) & 127u) {
    if (tid == 0) atomicExch(S.err, 2);
    return;
  }
  const int nx = S.nx, ny = S.ny, nz = S.nz;
  const int N = (int)S.N, NXY = nx * ny;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int i = x0 + tx, j = y0 + ty;
  const bool act = i < nx && j < ny;
  const bool per = S.periodic;
  const int k0 = blockIdx.z * zchunk, k1 = min(nz, k0 + zchunk);
  const int col = j * nx + i;
  const int xo = tile_origin(x0, TX, nx, per), yo = tile_origin(y0, TY, ny, per);
  const int ry = y0 - yo + ty, rx = x0 - xo + tx;
  const int own = ry * HX + rx;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto O = [&](int b, int slot) -> double { return smem[b * BUF + slot * NC + cid]; };
  auto Hp = [&](int b, int slot) -> double * { return smem + b * BUF + NO * NC + slot * HS; };
  double *X = smem + 2 * BUF;
  // this thread's halo positions (smem index, global xy offset), or -1
  int hs0 = -1, hs1 = -1, ho0 = 0, ho1 = 0;
  {
    const int cx0 = x0 - xo, cy0 = y0 - yo;
    auto pos = [&](int t, int &hs, int &ho) {
      if (t >= HS) return;
      const int ly = t / HX, lx = t - ly * HX;
      const bool inx = lx >= cx0 && lx < cx0 + TX, iny = ly >= cy0 && ly < cy0 + TY;
      if (!inx && !iny) return;
      int gx = xo + lx, gy = yo + ly;
      if (per) {
        gx = wrapi(gx, nx);
        gy = wrapi(gy, ny);
      } else if (gx < 0 || gx >= nx || gy < 0 || gy >= ny) {
        return;
      }
      hs = t;
      ho = gy * nx + gx;
    };
    pos(tid, hs0, ho0);
    pos(tid + NT, hs1, ho1);
  }
  const unsigned own_bytes =
      (MODE == FIRST ? 15u : (MODE == MID ? 23u : 24u)) * NC * (unsigned)sizeof(double);
  auto issue = [&](int k, int b) {
    const int kb = k * NXY;
    if (hs0 >= 0) {
      double *h = Hp(b, 0) + hs0;
      const int id = kb + ho0;
#pragma unroll
      for (int sl = 0; sl < 7; ++sl) cp_async8(h + sl * HS, tin + (sl + 1) * N + id);
      cp_async8(h + 7 * HS, S.box + id);
      cp_async8(h + 8 * HS, S.boy + id);
      cp_async8(h + 9 * HS, S.boz + id);
    }
    if (hs1 >= 0) {
      double *h = Hp(b, 0) + hs1;
      const int id = kb + ho1;
#pragma unroll
      for (int sl = 0; sl < 7; ++sl) cp_async8(h + sl * HS, tin + (sl + 1) * N + id);
      cp_async8(h + 7 * HS, S.box + id);
      cp_async8(h + 8 * HS, S.boy + id);
      cp_async8(h + 9 * HS, S.boz + id);
    }
    cp_commit();
    if (tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&bar[b], own_bytes);
      double *ob = smem + b * BUF;
      tma_load_3d(ob + O_RHO * NC, &T.m[mt], x0, y0, k, &bar[b]);
      if (MODE != FIRST)
        for (int l = 0; l < 8; ++l)
          tma_load_3d(ob + (O_A + l) * NC, &T.m[ma], x0, y0, l * nz + k, &bar[b]);
      for (int n = 0; n < 14; ++n)
        tma_load_3d(ob + (O_BG + n) * NC, &T.m[3 + n], x0, y0, k, &bar[b]);
      if (MODE == LAST) tma_load_3d(ob + O_P0 * NC, &T.m[17], x0, y0, k, &bar[b]);
    }
  };
  // role 0 windows vz, p, bx; role 1 windows flux1, flux2, by
  double w0[11], w1[11], w2[11];
  auto head = [&](int kk, double &v0, double &v1, double &v2) {
    const int id = kk * NXY + col;
    if (role == 0) {
      v0 = __ldg(tin + 3 * N + id);
      v1 = __ldg(tin + 4 * N + id);
      v2 = __ldg(tin + 5 * N + id);
    } else {
      const double vx_ = __ldg(tin + N + id), vy_ = __ldg(tin + 2 * N + id),
                   vz_ = __ldg(tin + 3 * N + id);
      const double ox = __ldg(S.box + id), oy = __ldg(S.boy + id),
                   oz = __ldg(S.boz + id);
      v0 = -vz_ * oy + vy_ * oz;
      v1 = -vx_ * oz + vz_ * ox;
      v2 = __ldg(tin + 6 * N + id);
    }
  };
  issue(k0, 0);
  {
    const int b0 = min(k0 - 5, nz - 11);
#pragma unroll
    for (int m = 0; m < 11; ++m) {
      const int kk = b0 + m;
      if (act && kk >= 0) head(kk, w0[m], w1[m], w2[m]);
      else w0[m] = w1[m] = w2[m] = 0.0;
    }
  }
  double ke = 0.0, mr = 1e300, mp = 1e300;
  unsigned phase = 0;
  bool ok = true;

  for (int k = k0; k < k1; ++k) {
    const int b = (k - k0) & 1;
    double h0 = 0, h1 = 0, h2 = 0;
    const bool sh = k > k0 && k <= nz - 6;
    if (sh && act) head(k + 5, h0, h1, h2);   // in flight during the waits
    if (k + 1 < k1) issue(k + 1, b ^ 1);
    else cp_commit();
    cp_wait1();
    ok = mbar_wait(&bar[b], (phase >> b) & 1u, S.err);
    phase ^= 1u << b;
    if (!__syncthreads_and(ok)) { ok = false; break; }
    if (sh) { shift(w0, h0); shift(w1, h1); shift(w2, h2); }
    double *H7 = Hp(b, 7), *H8 = Hp(b, 8), *H9 = Hp(b, 9);
    const double ox = H7[own], oy = H8[own], oz = H9[own];
    __syncthreads();
    {
      const double *H0 = Hp(b, 0), *H1 = Hp(b, 1), *H2 = Hp(b, 2);
      const int cx0 = x0 - xo, cy0 = y0 - yo;
      for (int t = tid; t < HS; t += NT) {
        const int ly = t / HX, lx = t - ly * HX;
        const bool inx = lx >= cx0 && lx < cx0 + TX, iny = ly >= cy0 && ly < cy0 + TY;
        if (!inx && !iny) continue;
        const double vx_ = H0[t], vy_ = H1[t], vz_ = H2[t];
        const double bx0 = H7[t], by0 = H8[t], bz0 = H9[t];
        H7[t] = -vz_ * by0 + vy_ * bz0;
        H8[t] = -vx_ * bz0 + vz_ * bx0;
        H9[t] = -vy_ * bx0 + vx_ * by0;
      }
    }
    __syncthreads();
    const int id = k * NXY + col;
    const double szk = __ldg(S.stretch + k);
    const double dt = S.deltat;
    auto DX = [&](int slot) {
      const double *row = Hp(b, slot) + ry * HX;
      if (per || (i >= 5 && i < nx - 5)) return S.stretchx * csum(row + (i - 5 - xo), 1);
      return dxy(i, nx, per, S.stretchx, [&](int g) { return row[g - xo]; });
    };
    auto DY = [&](int slot) {
      const double *colp = Hp(b, slot) + rx;
      if (per || (j >= 5 && j < ny - 5)) return S.stretchy * csum(colp + (j - 5 - yo) * HX, HX);
      return dxy(j, ny, per, S.stretchy, [&](int g) { return colp[(g - yo) * HX]; });
    };
    const bool zpml = S.zb.on && (k < S.zb.np || k >= nz - S.zt.np);
    const bool xpml = S.xb.on && act && (i < S.xb.np || i >= nx - S.xt.np);
    const bool ypml = S.xb.on && act && (j < S.yb.np || j >= ny - S.yt.np);
    // CPML correction of derivative d with auxiliary slot `slot` on the
    // z, x or y face this point lies in (RHS.f90:424-546)
    auto pz = [&](int slot, double &d) {
      const bool bot = k < S.zb.np;
      const FaceDev &F = bot ? S.zb : S.zt;
      const int kl = bot ? k : k - (nz - S.zt.np);
      cpml<MODE>(F, (long long)kl * NXY + col, kl, slot, beta, dt, d);
    };
    auto px = [&](int slot, double &d) {
      const bool bot = i < S.xb.np;
      const FaceDev &F = bot ? S.xb : S.xt;
      const int il = bot ? i : i - (nx - S.xt.np);
      cpml<MODE>(F, il + (long long)F.np * (j + (long long)ny * k), il, slot, beta, dt, d);
    };
    auto py = [&](int slot, double &d) {
      const bool bot = j < S.yb.np;
      const FaceDev &F = bot ? S.yb : S.yt;
      const int jl = bot ? j : j - (ny - S.yt.np);
      cpml<MODE>(F, i + (long long)nx * (jl + (long long)F.np * k), jl, slot, beta, dt, d);
    };
    auto Hv = [&](int slot) { return Hp(b, slot)[own]; };
    double d0 = 0, d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0, d6 = 0, d7 = 0, d8 = 0;
    if (act) {
      if (role == 0) {
        d0 = DX(3); d5 = DX(6); d7 = DX(5);
        d1 = DY(3); d4 = DY(6); d8 = DY(4);
        d3 = dz(w0, k, nz, szk); d2 = dz(w1, k, nz, szk); d6 = dz(w2, k, nz, szk);
        if (zpml) { pz(1, d2); pz(0, d3); pz(2, d6); }
        if (xpml) { px(1, d0); px(3, d5); px(2, d7); }
        if (ypml) { py(1, d1); py(3, d4); py(2, d8); }
        X[cid] = d3;
      } else {
        d0 = DX(0); d2 = DX(9); d3 = DX(8);
        d1 = DY(1); d4 = DY(9); d5 = DY(7);
        d6 = dz(w0, k, nz, szk); d7 = dz(w1, k, nz, szk); d8 = dz(w2, k, nz, szk);
        if (zpml) { pz(4, d7); pz(5, d6); pz(3, d8); }
        if (xpml) { px(0, d0); px(4, d2); px(5, d3); }
        if (ypml) { py(0, d1); py(4, d4); py(5, d5); }
        X[NC + cid] = d8;
      }
    }
    __syncthreads();
    double an_rho = 0.0;
    if (act) {
      const bool zero = k == 0 || k == nz - 1 ||
                        (!per && (i == 0 || i == nx - 1 || j == 0 || j == ny - 1));
      const double fac = MODE == LAST ? dt : bnext;
      const double rho = O(b, O_RHO), vx = Hv(0), vy = Hv(1), vz = Hv(2);
      const double red = O(b, O_BG + pipe::B_RED), sg = O(b, O_BG + pipe::B_SPONGE);
      if (role == 0) {
        const double dzby = X[NC + cid];
        const double cbx = d4 - dzby, cby = -d5 + d6, cbz = d7 - d8;
        const double c1 = cby * oz - cbz * oy, c2 = ox * cbz - cbx * oz,
                     c3 = cbx * oy - cby * ox;
        const double ri = O(b, O_BG + pipe::B_RHOINV);
        double vxr = -ri * (d0 - (c1 * red)) - sg * vx;
        double vyr = -ri * (d1 - (c2 * red)) - sg * vy;
        double vzr = -ri * (d2 - (c3 * red)) - sg * vz;
        const double bx = Hv(4), by = Hv(5), bz = Hv(6);
        const double qx = O(b, O_BG + pipe::B_CBX), qy = O(b, O_BG + pipe::B_CBY),
                     qz = O(b, O_BG + pipe::B_CBZ);
        const double e1 = qy * bz - qz * by, e2 = bx * qz - qx * bz,
                     e3 = qx * by - qy * bx;
        vxr = vxr + ri * e1 * red;
        vyr = vyr + ri * e2 * red;
        vzr = vzr + ri * e3 * red;
        const int gc = S.colx[i] + S.bxdim * S.coly[j];
        vzr = vzr - ri * rho * __ldg(S.gblk + gc * nz + k);
        if (S.frc.kind != SPARC_SRC_NONE) {
          const long long it = *S.iter;
          const double frc = forcing_at(S, it, pulse_time(S, it), i, j, k);
          if (S.frc.dir == 1) vxr = vxr + frc;
          else if (S.frc.dir == 2) vyr = vyr + frc;
          else vzr = vzr + frc;
        }
        const double a1 = MODE == FIRST ? vx : O(b, O_A + 1);
        const double a2 = MODE == FIRST ? vy : O(b, O_A + 2);
        const double a3 = MODE == FIRST ? vz : O(b, O_A + 3);
        const double n1 = zero ? a1 : a1 + fac * vxr;
        const double n2 = zero ? a2 : a2 + fac * vyr;
        const double n3 = zero ? a3 : a3 + fac * vzr;
        so[N + id] = n1;
        so[2 * N + id] = n2;
        so[3 * N + id] = n3;
        if (MODE == LAST) X[2 * NC + cid] = n1 * n1 + n2 * n2 + n3 * n3;
      } else {
        const double p = Hv(3);
        const double dvzdz = X[cid];
        const double div = d0 + d1 + dvzdz;
        const double r0 = O(b, O_BG + pipe::B_RHO0);
        const double Rr = -O(b, O_BG + pipe::B_GRX) * vx - O(b, O_BG + pipe::B_GRY) * vy -
                          O(b, O_BG + pipe::B_GRZ) * vz - r0 * div - sg * rho;
        const double Rp = -O(b, O_BG + pipe::B_C2R) * div - vx * O(b, O_BG + pipe::B_GPX) -
                          vy * O(b, O_BG + pipe::B_GPY) - vz * O(b, O_BG + pipe::B_GPZ) -
                          sg * p;
        const double Rbx = red * (d4 - d7), Rby = red * (d6 - d2), Rbz = red * (d3 - d5);
        const double ar = MODE == FIRST ? rho : O(b, O_A + 0);
        const double ap = MODE == FIRST ? p : O(b, O_A + 4);
        const double abx = MODE == FIRST ? Hv(4) : O(b, O_A + 5);
        const double aby = MODE == FIRST ? Hv(5) : O(b, O_A + 6);
        const double abz = MODE == FIRST ? Hv(6) : O(b, O_A + 7);
        an_rho = zero ? ar : ar + fac * Rr;
        so[id] = an_rho;
        so[4 * N + id] = zero ? ap : ap + fac * Rp;
        so[5 * N + id] = zero ? abx : abx + fac * Rbx;
        so[6 * N + id] = zero ? aby : aby + fac * Rby;
        so[7 * N + id] = zero ? abz : abz + fac * Rbz;
        if (MODE == LAST) {
          mr = fmin(mr, rho + r0);
          mp = fmin(mp, p + O(b, O_P0));
        }
      }
    }
    if (MODE == LAST) {
      __syncthreads();
      if (act && role == 1) {  // KE density of driver.f90:161 on a_new
        const double m = (O(b, O_BG + pipe::B_RHO0) + an_rho) * X[2 * NC + cid] / 2.0;
        ke += m * m;
      }
    }
    __syncthreads();
  }
  if (!ok) {
    // a bounded wait gave up: drain (again bounded) what this CTA issued
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (tid == 0) {
      mbar_wait(&bar[0], phase & 1u, S.err);
      mbar_wait(&bar[1], (phase >> 1) & 1u, S.err);
    }
    return;
  }
  if (MODE == LAST) diag_reduce(S, ke, mr, mp);
}

// ------------------------------------------------------- stage dispatch
int stage_geometry(Handle *h) {
  // tile shape: (32, 8); the quiet kernel drops to (16, 8) on grids too
  // small to fill the GPU.  The MHD kernels always use (32, 8).
  h->tx = 32;
  h->ty = 8;
  if (h->magnetic && !h->fp32 && h->mhd_kernel == 4 && (h->nx % 2) == 0)
    h->ty = h->tma_ty;  // TMA tiles: 32 x tma_ty
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
  zc = std::min(zc, h->nz);
  if (const char *kv = std::getenv("SPARC_ZCHUNK")) {  // A/B timing only
    const int v = std::atoi(kv);
    if (v >= 11) zc = std::min(v, h->nz);
  }
  h->zchunk = zc;
  h->max_stage_blocks = (int)(tiles * ((h->nz + zc - 1) / zc));
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

static int launch_mhd_duo(Handle *h, const SimDev &S, int stage,
                          const double *a, const double *tin, double *so,
                          cudaStream_t s) {
  using namespace duo;
  dim3 blk(TX, TY, 2);
  dim3 grd((h->nx + TX - 1) / TX, (h->ny + TY - 1) / TY,
           (h->nz + h->zchunk - 1) / h->zchunk);
  const double beta = h->betas[stage - 1];
  const double bnext = stage < 5 ? h->betas[stage] : h->deltat;
  const int mode = stage == 1 ? FIRST : (stage == 5 ? LAST : MID);
  if (mode == FIRST) {
    cudaFuncSetAttribute(k_stage_mhd_duo<FIRST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    k_stage_mhd_duo<FIRST><<<grd, blk, SMEM, s>>>(S, a, tin, so, beta, bnext, h->zchunk);
  } else if (mode == MID) {
    cudaFuncSetAttribute(k_stage_mhd_duo<MID>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    k_stage_mhd_duo<MID><<<grd, blk, SMEM, s>>>(S, a, tin, so, beta, bnext, h->zchunk);
  } else {
    cudaFuncSetAttribute(k_stage_mhd_duo<LAST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    k_stage_mhd_duo<LAST><<<grd, blk, SMEM, s>>>(S, a, tin, so, beta, bnext, h->zchunk);
  }
  return SPARC_OK;
}

template <int TYV>
static int launch_mhd_tma_ty(Handle *h, const SimDev &S, int stage, const double *a,
                             const double *tin, double *so, cudaStream_t s, int mt,
                             int ma) {
  using G = TmaGeo<TYV>;
  TmaSet T;
  for (int n = 0; n < 18; ++n) T.m[n] = h->tmaps_ty[n];
  dim3 blk(G::TX, G::TY, 2);
  dim3 grd((h->nx + G::TX - 1) / G::TX, (h->ny + G::TY - 1) / G::TY,
           (h->nz + h->zchunk - 1) / h->zchunk);
  const double beta = h->betas[stage - 1];
  const double bnext = stage < 5 ? h->betas[stage] : h->deltat;
  const int mode = stage == 1 ? FIRST : (stage == 5 ? LAST : MID);
  const int sm = (int)G::SMEM;
  if (mode == FIRST) {
    cudaFuncSetAttribute(k_stage_mhd_tma<FIRST, TYV>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    k_stage_mhd_tma<FIRST, TYV><<<grd, blk, G::SMEM, s>>>(S, T, a, tin, so, beta, bnext, h->zchunk, mt, ma);
  } else if (mode == MID) {
    cudaFuncSetAttribute(k_stage_mhd_tma<MID, TYV>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    k_stage_mhd_tma<MID, TYV><<<grd, blk, G::SMEM, s>>>(S, T, a, tin, so, beta, bnext, h->zchunk, mt, ma);
  } else {
    cudaFuncSetAttribute(k_stage_mhd_tma<LAST, TYV>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    k_stage_mhd_tma<LAST, TYV><<<grd, blk, G::SMEM, s>>>(S, T, a, tin, so, beta, bnext, h->zchunk, mt, ma);
  }
  return SPARC_OK;
}

static int launch_mhd_tma(Handle *h, const SimDev &S, int stage,
                          const double *a, const double *tin, double *so,
                          cudaStream_t s) {
  int mt = -1, ma = -1;
  for (int b = 0; b < 3; ++b) {
    if (h->buf[b] == tin) mt = b;
    if (h->buf[b] == a) ma = b;
  }
  if (mt < 0 || ma < 0) return SPARC_ERR_INVALID;
  if ((long long)h->V * h->N >= (1LL << 31)) return SPARC_ERR_INVALID;
  if (h->tma_ty == 6) return launch_mhd_tma_ty<6>(h, S, stage, a, tin, so, s, mt, ma);
  return launch_mhd_tma_ty<8>(h, S, stage, a, tin, so, s, mt, ma);
}

// Tensor maps (3-D, FP64, 32x8x1 boxes) of the arrays the TMA kernel loads
// per layer; needs 16-byte row strides, i.e. an even nx.
int encode_tensor_maps(Handle *h) {
  h->tma = false;
  if (!h->magnetic || (h->nx & 1)) return SPARC_OK;
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
  auto one = [&](CUtensorMap *m, const double *base, unsigned long long depth) {
    cuuint64_t dims[3] = {(cuuint64_t)h->nx, (cuuint64_t)h->ny, (cuuint64_t)depth};
    cuuint64_t strides[2] = {(cuuint64_t)h->nx * 8, (cuuint64_t)h->nx * h->ny * 8};
    cuuint32_t box[3] = {32, (cuuint32_t)h->tma_ty, 1};
    cuuint32_t es[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)base, dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  bool ok = true;
  for (int b = 0; b < 3; ++b) ok = ok && one(&h->tmaps_ty[b], h->buf[b], (unsigned long long)h->nz * h->V);
  const double *bg[15] = {h->red, h->sponge, h->rho0, h->grx, h->gry, h->grz, h->c2rho0,
                          h->gpx, h->gpy, h->gpz, h->rhoinv, h->cbx, h->cby, h->cbz, h->p0};
  for (int n = 0; n < 15; ++n) ok = ok && bg[n] && one(&h->tmaps_ty[3 + n], bg[n], h->nz);
  h->tma = ok;
  return SPARC_OK;
}

// ------------------------- MP_MHD_3D, shared-body stage kernels (default)
// One RK stage as two launches over one logical grid of (x tile, y tile, z
// chunk) blocks: INT = true over the interior tile rectangle with the
// branch-free body of mhd_body.cuh, INT = false over the whole grid,
// returning at once on interior tiles (edge and CPML tiles).
// TMA: the 24 own-point arrays of a layer arrive as 32x8x1 TMA boxes.
template <int MODE, bool TMA, bool INT>
__global__ void __launch_bounds__(mg::NT, 1)
    k_mhd64(const SimDev S, const __grid_constant__ TmaSet32 T, const double *__restrict__ a,
            const double *__restrict__ tin, double *__restrict__ so, double beta, double bnext,
            int zchunk, int mt, int ma, int ix0, int iy0, int gx, int gy) {
  extern __shared__ __align__(1024) double smem_raw64[];
  double *smem = (double *)(((size_t)smem_raw64 + 127) & ~(size_t)127);
  const int tx_ = INT ? blockIdx.x + ix0 : blockIdx.x;
  const int ty_ = INT ? blockIdx.y + iy0 : blockIdx.y;
  const int x0 = tx_ * mg::TX, y0 = ty_ * mg::TY;
  if (!INT && mhd_interior(S, x0, y0)) return;
  double ke = 0.0, mr = 1e300, mp = 1e300;
  const int k0 = blockIdx.z * zchunk;
  if (!mhd_body<double, MODE, TMA, INT>(S, &T, smem, a, tin, so, beta, bnext, x0, y0, k0,
                                         min(S.nz, k0 + zchunk), mt, ma, ke, mr, mp))
    return;
  if (MODE == F_LAST)
    diag_reduce_t(S, ke, mr, mp, tx_ + (long long)gx * (ty_ + (long long)gy * blockIdx.z),
                  (long long)gx * gy * gridDim.z);
}

static int launch_mhd64(Handle *h, const SimDev &S, int stage, const double *a,
                        const double *tin, double *so, cudaStream_t s) {
  const double beta = h->betas[stage - 1];
  const double bnext = stage < 5 ? h->betas[stage] : h->deltat;
  const int mode = stage == 1 ? FIRST : (stage == 5 ? LAST : MID);
  dim3 blk(mg::TX, mg::TY, 2);
  dim3 grd((h->nx + mg::TX - 1) / mg::TX, (h->ny + mg::TY - 1) / mg::TY,
           (h->nz + h->zchunk - 1) / h->zchunk);
  const int np[4] = {h->faces[2].on ? h->faces[2].np : 0, h->faces[3].on ? h->faces[3].np : 0,
                     h->faces[4].on ? h->faces[4].np : 0, h->faces[5].on ? h->faces[5].np : 0};
  int ix0, ix1, iy0, iy1;
  mhd_interior_rect(h->nx, h->ny, np, ix0, ix1, iy0, iy1);
  const bool has_int = ix1 > ix0 && iy1 > iy0;
  dim3 gint(has_int ? ix1 - ix0 : 1, has_int ? iy1 - iy0 : 1, grd.z);
  const size_t sm = MhdBuf<double>::SMEM;
  const bool tma = h->tma && h->tma_ty == mg::TY && h->allow_tma64;
  int mt = -1, ma = -1;
  for (int b = 0; b < 3; ++b) {
    if (h->buf[b] == tin) mt = b;
    if (h->buf[b] == a) ma = b;
  }
  if (mt < 0 || ma < 0) return SPARC_ERR_INVALID;
  TmaSet32 T;
  if (tma)
    for (int n = 0; n < 18; ++n) T.m[n] = h->tmaps_ty[n];
  else
    std::memset(&T, 0, sizeof(T));
#define ML64(M, U)                                                                            \
  do {                                                                                        \
    cudaFuncSetAttribute(k_mhd64<M, U, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
    cudaFuncSetAttribute(k_mhd64<M, U, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
    if (has_int) {                                                                            \
      cudaEventRecord(h->ev_fork, s);                                                         \
      cudaStreamWaitEvent(h->aux, h->ev_fork, 0);                                             \
      k_mhd64<M, U, false><<<grd, blk, sm, h->aux>>>(S, T, a, tin, so, beta, bnext, h->zchunk, \
                                                     mt, ma, 0, 0, grd.x, grd.y);             \
      cudaEventRecord(h->ev_join, h->aux);                                                    \
      k_mhd64<M, U, true><<<gint, blk, sm, s>>>(S, T, a, tin, so, beta, bnext, h->zchunk, mt,  \
                                                ma, ix0, iy0, grd.x, grd.y);                  \
      cudaStreamWaitEvent(s, h->ev_join, 0);                                                  \
    } else {                                                                                  \
      k_mhd64<M, U, false><<<grd, blk, sm, s>>>(S, T, a, tin, so, beta, bnext, h->zchunk, mt,  \
                                                ma, 0, 0, grd.x, grd.y);                      \
    }                                                                                         \
  } while (0)
  if (has_int) ++h->launches;  // the interior launch (launch_stage counts the other)
  if (tma) {
    if (mode == FIRST) ML64(F_FIRST, true);
    else if (mode == MID) ML64(F_MID, true);
    else ML64(F_LAST, true);
  } else {
    if (mode == FIRST) ML64(F_FIRST, false);
    else if (mode == MID) ML64(F_MID, false);
    else ML64(F_LAST, false);
  }
#undef ML64
  return SPARC_OK;
}

int launch_stage(Handle *h, const SimDev &S, int stage, const double *a,
                 const double *tin, double *so, cudaStream_t s) {
  int r = SPARC_ERR_INVALID;
  if (h->magnetic && h->mhd_kernel == 5) {
    if (h->tx != 32 || h->ty != 8) return SPARC_ERR_INVALID;
    r = launch_mhd64(h, S, stage, a, tin, so, s);
    ++h->launches;
    if (r == SPARC_OK && cudaGetLastError() != cudaSuccess) r = SPARC_ERR_CUDA;
    return r;
  }
  if (h->magnetic && h->mhd_kernel == 4 && h->tma && h->tx == 32 &&
      (long long)h->V * h->N < (1LL << 31)) {
    r = launch_mhd_tma(h, S, stage, a, tin, so, s);
    ++h->launches;
    if (r == SPARC_OK && cudaGetLastError() != cudaSuccess) r = SPARC_ERR_CUDA;
    return r;
  }
  if (h->magnetic) {
    if (h->tx != 32 || h->ty != 8) return SPARC_ERR_INVALID;
    r = launch_mhd_duo(h, S, stage, a, tin, so, s);
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

// ------------------------------------------------------ FILTER_VARS pass
// One direction of FILTER_VARS (derivatives.f90:659-703) over all fields:
// out = filt(pre(in)) (mode 1) or pre(in) - s*filt(pre(in)) (mode 2), where
// pre() is the edge pre-averaging of :672-693 applied on the fly from the
// unmodified input.
struct FiltDev {
  int nx, ny, nz, periodic, g, mode2, V;
  long long N;
  double s;
};

template <int DIR>
__global__ void k_filter_pass(FiltDev F, const double *__restrict__ in,
                              double *__restrict__ out) {
  const long long total = F.N * F.V;
  const int n = DIR == 0 ? F.nx : (DIR == 1 ? F.ny : F.nz);
  const long long st = DIR == 0 ? 1 : (DIR == 1 ? F.nx : (long long)F.nx * F.ny);
  const bool per = DIR != 2 && F.periodic;
  const bool avg = DIR == 2 || !F.periodic;
  const int g = F.g;
  const double *c = c_df[g == 5 ? 0 : 1];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long pnt = t % F.N;
    int q;
    if (DIR == 0) q = (int)(pnt % F.nx);
    else if (DIR == 1) q = (int)((pnt / F.nx) % F.ny);
    else q = (int)(pnt / ((long long)F.nx * F.ny));
    const long long base = t - (long long)q * st;
    auto pre = [&](int qq) -> double {
      const long long id = base + (long long)qq * st;
      if (avg && ((qq >= 1 && qq <= g - 1) || (qq >= n - g && qq <= n - 2)))
        return (__ldg(in + id + st) + __ldg(in + id - st)) / 2.0;
      return __ldg(in + id);
    };
    const double pq = pre(q);
    double filt;
    if (!per && (q < g || q >= n - g)) {
      filt = (DIR != 2 && g == 3) ? 0.0 : pq;
    } else {
      double s = 0.0;
      for (int m = 0; m < 2 * g + 1; ++m) {
        int qq = q - g + m;
        if (per) qq = wrapi(qq, n);
        s += pre(qq) * c[m];
      }
      filt = s;
    }
    out[t] = F.mode2 ? pq - F.s * filt : filt;
  }
}

int launch_filter_pass(Handle *h, int dir, const double *in, double *out,
                       cudaStream_t s) {
  FiltDev F;
  F.nx = h->nx; F.ny = h->ny; F.nz = h->nz;
  F.periodic = h->periodic ? 1 : 0;
  F.g = dir == 2 ? h->gz : h->gxy;
  F.mode2 = F.g == 3;
  F.V = h->V;
  F.N = h->N;
  F.s = dir == 2 ? h->P.s_z : h->P.s_xy;
  long long total = F.N * F.V;
  unsigned nb = (unsigned)std::min<long long>((total + 255) / 256, 148 * 32);
  if (dir == 0) k_filter_pass<0><<<nb, 256, 0, s>>>(F, in, out);
  else if (dir == 1) k_filter_pass<1><<<nb, 256, 0, s>>>(F, in, out);
  else k_filter_pass<2><<<nb, 256, 0, s>>>(F, in, out);
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
  S.V = h->V;
  S.stretchx = h->stretchx;
  S.stretchy = h->stretchy;
  S.stretch = h->d_stretch;
  S.deltat = h->deltat;
  S.dimc2rho = (h->dimc * h->dimc) * h->dimrho;
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
  S.iter = h->d_iter;
  S.err = h->d_err;
  S.partials = h->d_partials;
  S.counter = h->d_counter;
  S.diag = h->d_diag;
  S.fail_iter = h->d_fail;
  return S;
}

}  // namespace sparc
