// setup.cu -- FP64 background and coefficient setup on the device, plus the
// generic (unfused) derivative and filter kernels used by the setup and by
// the unit entry points.
//
// This translation unit is compiled with -fmad=false: every product feeding
// a sum is rounded on its own, as in the reference's Fortran, so the
// coefficient arrays reproduce a plain IEEE evaluation of the reference's
// expressions (operand order kept, see the file:line cited at each step).
// One-dimensional quantities (axes, z metric, CPML layer factors, RK
// coefficients) are computed on the host; every 3-D array on the device.

#include <algorithm>
#include <cmath>
#include <cstring>

#include "internal.h"

namespace sparc {

__constant__ double k_dp[6][11];   // derivative rows, initialize.f90:1959-2031
__constant__ double k_df[2][11];   // filters: [0] xy, [1] z

// Published Bogey-Bailly optimized 11-point first-derivative coefficients
// (centred row 6 and the one-sided rows 1-5 with the reference's hand
// perturbations), initialize.f90:1959-2029.
const double kDerivRows[6][11] = {
    {-2.391602219538, 5.832490322294, -7.650218001182 + 0.000000000001,
     7.907810563576, -5.922599052629, 3.071037015445, -1.014956769726,
     0.170022256519, 0.002819958377, -0.004791009708, -0.000013063429},
    {-0.180022054228, -1.237550583044, 2.484731692990, -1.810320814061,
     1.112990048440, -0.481086916514, 0.126598690230, -0.015510730165,
     0.000024609059 - 0.000003, 0.000156447571 - 0.000000000001,
     -0.000007390277},
    {0.057982271137, -0.536135360383, -0.264089548967 + 0.000000000002,
     0.917445877606 - 0.000000000002, -0.169688364841, -0.029716326170,
     0.029681617641, -0.005222483773, -0.000118806260, -0.000118806260,
     -0.000020069730},
    {-0.013277273810, 0.115976072920, -0.617479187931,
     -0.274113948206 + 0.000000000002, 1.086208764655 - 0.000000000002,
     -0.402951626982, 0.131066986242, -0.028154858354, 0.002596328316,
     0.000128743150, 0.0},
    {0.016756572303, -0.117478455239, 0.411034935097, -1.130286765151,
     0.341435872100 - 0.000000000001, 0.556396830543, -0.082525734207,
     0.003565834658, 0.001173034777, -0.000071772671 + 0.000000000064,
     -0.000000352273},
    {-0.002484594688, 0.020779405824, -0.090320001280, 0.286511173973,
     -0.872756993962, 0.0, 0.872756993962, -0.286511173973, 0.090320001280,
     -0.020779405824, 0.002484594688}};

// Filter stencils, initialize.f90:1931-1951: 11-point low pass (mode 1)
// and 7-point high pass (mode 2).
const double kFilter11[11] = {
    0.5 * 0.00195312500000, -0.5 * 0.01953125000000, 0.5 * 0.08789062500000,
    -0.5 * 0.23437500000000, 0.5 * 0.41015625000000, 0.75390625000000,
    0.5 * 0.41015625000000, -0.5 * 0.23437500000000, 0.5 * 0.08789062500000,
    -0.5 * 0.01953125000000, 0.5 * 0.00195312500000};
const double kFilter7[7] = {-0.015625000, 0.093750000, -0.234375000,
                            0.312500000, -0.234375000, 0.093750000,
                            -0.015625000};

int setup_constants() {
  if (cudaMemcpyToSymbol(k_dp, kDerivRows, sizeof(kDerivRows)) != cudaSuccess)
    return SPARC_ERR_CUDA;
  return SPARC_OK;
}

static void filter_table(int g, double *out) {
  for (int m = 0; m < 11; ++m) out[m] = 0.0;
  if (g == 5)
    for (int m = 0; m < 11; ++m) out[m] = kFilter11[m];
  else
    for (int m = 0; m < 7; ++m) out[m] = kFilter7[m];
}

// ------------------------------------------------------------ helpers
template <class F>
__global__ void k_each(long long n, F f) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    f(t);
}

template <class F>
static void each(long long n, cudaStream_t s, F f) {
  if (n <= 0) return;
  long long nb = (n + 255) / 256;
  if (nb > 148 * 32) nb = 148 * 32;
  k_each<<<(unsigned)nb, 256, 0, s>>>(n, f);
}

struct Geo {
  int nx, ny, nz, periodic;
  double stretchx, stretchy;
  const double *stretch;
};

// ddx/ddy/ddz on the global domain (derivatives.f90:10-116, 226-341,
// 451-562): centred 11-point stencil; x/y periodic -> wrapped halo; x/y
// non-periodic with bc 1 -> one-sided rows at both edges; z with bc 1 ->
// zero ghosts at the bottom and one-sided rows at the top; bc 5 on a
// non-periodic axis -> zero ghosts.
__global__ void k_deriv(Geo G, int dir, int bc, const double *__restrict__ in,
                        double *__restrict__ out) {
  const long long N = (long long)G.nx * G.ny * G.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
       t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % G.nx);
    int j = (int)((t / G.nx) % G.ny);
    int k = (int)(t / ((long long)G.nx * G.ny));
    int q, n;
    long long st;
    double sc;
    bool per;
    if (dir == 0) { q = i; n = G.nx; st = 1; sc = G.stretchx; per = G.periodic; }
    else if (dir == 1) { q = j; n = G.ny; st = G.nx; sc = G.stretchy; per = G.periodic; }
    else { q = k; n = G.nz; st = (long long)G.nx * G.ny; sc = G.stretch[k]; per = false; }
    const long long base = t - (long long)q * st;
    double s = 0.0;
    if (per) {
      for (int m = 0; m < 11; ++m) {
        int qq = q - 5 + m;
        qq = (qq % n + n) % n;
        s += in[base + qq * st] * k_dp[5][m];
      }
      out[t] = sc * s;
    } else if (bc == 1 && dir != 2 && q < 5) {
      for (int m = 0; m < 11; ++m) s += in[base + m * st] * k_dp[q][m];
      out[t] = sc * s;
    } else if (bc == 1 && q >= n - 5) {
      int row = n - 1 - q;
      for (int m = 0; m < 11; ++m)
        s += in[base + (long long)(n - 1 - m) * st] * k_dp[row][m];
      out[t] = -sc * s;
    } else {
      for (int m = 0; m < 11; ++m) {
        int qq = q - 5 + m;
        double v = (qq >= 0 && qq < n) ? in[base + qq * st] : 0.0;
        s += v * k_dp[5][m];
      }
      out[t] = sc * s;
    }
  }
}

// filtx/filty/filtz output (derivatives.f90:119-223, 345-447, 565-642)
// without FILTER_VARS's edge pre-averaging.
__global__ void k_filter_raw(Geo G, int dir, int g, double c0, double c1,
                             double c2, double c3, double c4, double c5,
                             double c6, double c7, double c8, double c9,
                             double c10, const double *__restrict__ in,
                             double *__restrict__ out) {
  const double c[11] = {c0, c1, c2, c3, c4, c5, c6, c7, c8, c9, c10};
  const long long N = (long long)G.nx * G.ny * G.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
       t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % G.nx);
    int j = (int)((t / G.nx) % G.ny);
    int k = (int)(t / ((long long)G.nx * G.ny));
    int q = dir == 0 ? i : (dir == 1 ? j : k);
    int n = dir == 0 ? G.nx : (dir == 1 ? G.ny : G.nz);
    long long st = dir == 0 ? 1 : (dir == 1 ? G.nx : (long long)G.nx * G.ny);
    bool per = dir != 2 && G.periodic;
    const long long base = t - (long long)q * st;
    if (!per && (q < g || q >= n - g)) {
      out[t] = (dir != 2 && g == 3) ? 0.0 : in[t];
      continue;
    }
    double s = 0.0;
    for (int m = 0; m < 2 * g + 1; ++m) {
      int qq = q - g + m;
      qq = (qq % n + n) % n;
      s += in[base + qq * st] * c[m];
    }
    out[t] = s;
  }
}

static Geo geo(Handle *h) {
  return Geo{h->nx, h->ny, h->nz, h->periodic ? 1 : 0, h->stretchx,
             h->stretchy, h->d_stretch};
}

static unsigned grid_for(long long n) {
  long long nb = (n + 255) / 256;
  return (unsigned)std::min<long long>(nb, 148 * 32);
}

int launch_derivative(Handle *h, int dir, int bc, const double *in,
                      double *out, cudaStream_t s) {
  k_deriv<<<grid_for(h->N), 256, 0, s>>>(geo(h), dir, bc, in, out);
  ++h->launches;
  return cudaGetLastError() == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

int launch_filter_raw(Handle *h, int dir, const double *in, double *out,
                      cudaStream_t s) {
  int g = dir == 2 ? h->gz : h->gxy;
  double c[11];
  filter_table(g, c);
  k_filter_raw<<<grid_for(h->N), 256, 0, s>>>(geo(h), dir, g, c[0], c[1],
                                               c[2], c[3], c[4], c[5], c[6],
                                               c[7], c[8], c[9], c[10], in,
                                               out);
  ++h->launches;
  return cudaGetLastError() == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

// atomic max of non-negative doubles through their bit patterns
__device__ inline void atomic_max_pos(unsigned long long *addr, double v) {
  atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

__global__ void k_vamax(long long N, double T, double dimb2, double den0,
                        const double *box, const double *boy,
                        const double *boz, const double *red,
                        const double *rho0, unsigned long long *out) {
  double m = 0.0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N;
       n += (long long)gridDim.x * blockDim.x) {
    double b2 = box[n] * box[n] + boy[n] * boy[n] + boz[n] * boz[n];
    // initialize.f90:974
    double v = sqrt(dimb2 * T / (T + red[n]) * b2 / (den0 * rho0[n]));
    m = fmax(m, v);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomic_max_pos(out, m);
}

// The Alfven-speed maximum of initialize.f90:974 for up to kVaCand limiter
// candidates T[c] at once: out[c] = max over points of the square of
// v(T[c]) (sqrt is monotone and correctly rounded, so sqrt(max v^2) equals
// the maximum of the square roots the reference takes).
constexpr int kVaCand = 12;
struct VaCand {
  double T[kVaCand];
  int n;
};
__global__ void k_vamax_multi(long long N, VaCand C, double dimb2, double den0,
                              const double *box, const double *boy, const double *boz,
                              const double *red, const double *rho0, unsigned long long *out) {
  double m[kVaCand];
#pragma unroll
  for (int c = 0; c < kVaCand; ++c) m[c] = 0.0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N;
       n += (long long)gridDim.x * blockDim.x) {
    const double b2 = box[n] * box[n] + boy[n] * boy[n] + boz[n] * boz[n];
    const double r = red[n], q = den0 * rho0[n];
#pragma unroll
    for (int c = 0; c < kVaCand; ++c)
      if (c < C.n) m[c] = fmax(m[c], dimb2 * C.T[c] / (C.T[c] + r) * b2 / q);
  }
#pragma unroll
  for (int c = 0; c < kVaCand; ++c) {
    double v = m[c];
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0 && c < C.n) atomic_max_pos(out + c, v);
  }
}

__global__ void k_max(long long N, const double *x, unsigned long long *out) {
  double m = 0.0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N;
       n += (long long)gridDim.x * blockDim.x)
    m = fmax(m, x[n]);
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomic_max_pos(out, m);
}

#define CK(x)                                          \
  do {                                                 \
    if (!cuda_ok(h, (x), #x)) return SPARC_ERR_CUDA;   \
  } while (0)

// Device copy of n host doubles, ordered on the handle's stream (the set-up
// kernels run there); a pageable source may be released on return.
static double *up(Handle *h, const double *src, size_t n) {
  double *d = (double *)dev_alloc(h, n * sizeof(double));
  if (d && src)
    if (!cuda_ok(h, cudaMemcpyAsync(d, src, n * sizeof(double), cudaMemcpyHostToDevice,
                                    h->stream), "upload"))
      return nullptr;
  return d;
}

// Per-layer CPML factors of one face, computed on the host exactly as the
// reference writes them (initialize.f90:1054-1069 and the analogous blocks).
struct Layers {
  std::vector<double> rn, rn1, alpha, kap;
};

int setup_background(Handle *h, const double *rho0_in, const double *pre0_in,
                     const double *cs0_in, const double *bx0,
                     const double *by0, const double *bz0,
                     const double *zaxis_mm, const double *grav) {
  const int nx = h->nx, ny = h->ny, nz = h->nz;
  const long long N = h->N;
  const sparc_params &P = h->P;
  cudaStream_t s = h->stream;
  auto I = [&](int i, int j, int k) {
    return (long long)i + (long long)nx * ((long long)j + (long long)ny * k);
  };

  // ------------------------------------------------ host 1-D setup
  // scales, all_modules.f90:284-308, 401-405
  h->zaxis.resize(nz);
  for (int k = 0; k < nz; ++k) h->zaxis[k] = 1.0 + zaxis_mm[k] * 1.0e8 / RSUN;
  h->dimc = cs0_in[0];
  h->dimrho = rho0_in[0];
  h->diml = RSUN;
  h->dimb = std::sqrt(4.0 * PI * (h->dimc * h->dimc) * h->dimrho);
  const double dimc = h->dimc, dimrho = h->dimrho, diml = h->diml,
               dimb = h->dimb;
  h->cq.resize(nz);
  h->invrho0q.resize(nz);
  for (int k = 0; k < nz; ++k) {
    h->cq[k] = cs0_in[I(0, 0, k)];
    h->invrho0q[k] = 2.5440390e-7 / rho0_in[I(0, 0, k)];
  }
  h->g.assign(grav, grav + nz);
  for (int k = 0; k < nz; ++k) h->g[k] = h->g[k] * diml / (dimc * dimc);
  for (int k = 0; k < nz; ++k) h->cq[k] = h->cq[k] / dimc;
  // z metric, initialize.f90:674-730
  h->stretch.resize(nz);
  const double(*dp)[11] = kDerivRows;
  const std::vector<double> &z = h->zaxis;
  for (int k = 0; k < nz; ++k) {
    double u;
    if (k < 5) {
      u = 0.0;
      for (int m = 0; m < 11; ++m) u += z[m] * dp[k][m];
      u = u * (nz - 1);
    } else if (k >= nz - 5) {
      int row = nz - 1 - k;
      u = 0.0;
      for (int m = 0; m < 11; ++m) u = u + z[nz - 1 - m] * dp[row][m];
      u = -u * (nz - 1);
    } else {
      u = ((-z[k - 5] + z[k + 5]) * dp[5][10] + (-z[k - 4] + z[k + 4]) * dp[5][9] +
           (-z[k - 3] + z[k + 3]) * dp[5][8] + (-z[k - 2] + z[k + 2]) * dp[5][7] +
           (-z[k - 1] + z[k + 1]) * dp[5][6]) * (nz - 1);
    }
    h->stretch[k] = (nz - 1) * 1.0 / u;
  }
  h->deltat = P.timestep * dimc / diml;  // initialize.f90:733
  {  // INITIALIZE_STEP, initialize.f90:1366-1381
    double o[5] = {1.0, 0.5, 0.1665579725791151184, 0.03950410250586729987,
                   0.007810706393337838236};
    double b5 = o[1], b4 = o[2] / b5, b3 = o[3] / (b5 * b4),
           b2 = o[4] / (b5 * b4 * b3);
    h->betas[0] = 0.0 * h->deltat;
    h->betas[1] = b2 * h->deltat;
    h->betas[2] = b3 * h->deltat;
    h->betas[3] = b4 * h->deltat;
    h->betas[4] = b5 * h->deltat;
  }
  h->d_stretch = up(h, h->stretch.data(), nz);
  if (!h->d_stretch) return SPARC_ERR_NOMEM;

  // ------------------------------------------------ 3-D arrays (FP64)
  double *rho0 = h->rho0 = up(h, nullptr, N);
  double *p0 = h->p0 = up(h, nullptr, N);
  double *c2 = h->c2 = up(h, nullptr, N);
  double *cs = up(h, nullptr, N);
  if (!rho0 || !p0 || !c2 || !cs) return SPARC_ERR_NOMEM;
  if (h->quiet) {  // column (1,1,:) replicated, all_modules.f90:353-384
    std::vector<double> col(3 * nz);
    for (int k = 0; k < nz; ++k) {
      col[k] = rho0_in[I(0, 0, k)];
      col[nz + k] = pre0_in[I(0, 0, k)];
      col[2 * nz + k] = cs0_in[I(0, 0, k)];
    }
    double *dcol = up(h, col.data(), col.size());
    if (!dcol) return SPARC_ERR_NOMEM;
    const long long NXY = (long long)nx * ny;
    each(N, s, [=] __device__(long long n) {
      int k = (int)(n / NXY);
      rho0[n] = dcol[k];
      p0[n] = dcol[nz + k];
      cs[n] = dcol[2 * nz + k];
    });
  } else {
    CK(cudaMemcpyAsync(rho0, rho0_in, N * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(p0, pre0_in, N * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(cs, cs0_in, N * 8, cudaMemcpyHostToDevice, s));
  }
  double *ssb = h->ssb = up(h, nullptr, N);
  if (!ssb) return SPARC_ERR_NOMEM;
  double *box = nullptr, *boy = nullptr, *boz = nullptr;
  if (h->magnetic) {
    box = h->box = up(h, nullptr, N);
    boy = h->boy = up(h, nullptr, N);
    boz = h->boz = up(h, nullptr, N);
    if (!box || !boy || !boz) return SPARC_ERR_NOMEM;
    CK(cudaMemcpyAsync(box, bx0, N * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(boy, by0, N * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(boz, bz0, N * 8, cudaMemcpyHostToDevice, s));
    // all_modules.f90:388-396; 0.01*8.0 is a single-precision product
    const double k8 = (double)(0.01f * 8.0f);
    each(N, s, [=] __device__(long long n) {
      double b2 = box[n] * box[n] + boy[n] * boy[n] + boz[n] * boz[n];
      double v = k8 * PI * p0[n] / fmax(b2, 1.0e-20);
      ssb[n] = fmin(v, 1.0);
    });
  } else {
    each(N, s, [=] __device__(long long n) { ssb[n] = 1.0; });
  }
  // nondimensionalisation, all_modules.f90:401-412
  {
    const bool mag = h->magnetic;
    each(N, s, [=] __device__(long long n) {
      p0[n] = p0[n] / (dimrho * (dimc * dimc));
      rho0[n] = rho0[n] / dimrho;
      double c = cs[n] / dimc;
      if (mag) {
        box[n] = box[n] / dimb;
        boy[n] = boy[n] / dimb;
        boz[n] = boz[n] / dimb;
      }
      c2[n] = c * c;
    });
  }

  // ------------------------------------------------ INITIALISE_RHS
  const int bc = h->periodic ? 5 : 1;
  {  // sponges, initialize.f90:899-947
    std::vector<double> sz(nz, 0.0), sx(nx, 0.0), sy(ny, 0.0);
    if (!h->use_pml)
      for (int k = 0; k < nz; ++k)
        sz[k] = 400.0 / (1.0 + std::exp((1.002 - z[k]) / 0.0001)) +
                40.0 / (1.0 + std::exp((z[k] - (z[0] + 0.005)) / 0.0005));
    const double s0 = P.sp_length / P.xlength, s1 = 1.0 - P.sp_length / P.xlength;
    if (!h->periodic && !h->use_hpml) {
      for (int i = 0; i < nx; ++i)
        sx[i] = P.sp_str * (1.0 - 1.0 / ((1.0 + std::exp((s0 - h->xaxis[i]) / P.sp_decay)) *
                                         (1.0 + std::exp((h->xaxis[i] - s1) / P.sp_decay))));
      for (int j = 0; j < ny; ++j)
        sy[j] = P.sp_str * (1.0 - 1.0 / ((1.0 + std::exp((s0 - h->yaxis[j]) / P.sp_decay)) *
                                         (1.0 + std::exp((h->yaxis[j] - s1) / P.sp_decay))));
    }
    h->sponge_slabs = true;
    for (double v : sz) h->sponge_slabs = h->sponge_slabs && v == 0.0;
    for (double v : sx) h->sponge_slabs = h->sponge_slabs && v == 0.0;
    for (double v : sy) h->sponge_slabs = h->sponge_slabs && v == 0.0;
    std::vector<double> all(nz + nx + ny);
    std::copy(sz.begin(), sz.end(), all.begin());
    std::copy(sx.begin(), sx.end(), all.begin() + nz);
    std::copy(sy.begin(), sy.end(), all.begin() + nz + nx);
    double *d = up(h, all.data(), all.size());
    double *sponge = h->sponge = up(h, nullptr, N);
    if (!d || !sponge) return SPARC_ERR_NOMEM;
    const bool per = h->periodic;
    each(N, s, [=] __device__(long long n) {
      int i = (int)(n % nx), j = (int)((n / nx) % ny),
          k = (int)(n / ((long long)nx * ny));
      sponge[n] = per ? d[k] : d[nz + i] + d[nz + nx + j] + d[k];
    });
  }
  double *tmp = up(h, nullptr, N);
  if (!tmp) return SPARC_ERR_NOMEM;
  if (h->magnetic) {
    // Alfven limiter, initialize.f90:962-991
    double *red = h->red = up(h, nullptr, N);
    double *dcq = up(h, h->cq.data(), nz);
    unsigned long long *dmax = (unsigned long long *)dev_alloc(h, 8 * kVaCand);
    if (!red || !dcq || !dmax) return SPARC_ERR_NOMEM;
    const long long NXY = (long long)nx * ny;
    each(N, s, [=] __device__(long long n) {
      int k = (int)(n / NXY);
      red[n] = (boz[n] * boz[n] + box[n] * box[n] + boy[n] * boy[n]) /
               (rho0[n] * (dcq[k] * dcq[k]));
    });
    auto devmax = [&](bool va, double T, double *out) -> int {
      CK(cudaMemsetAsync(dmax, 0, 8, s));
      if (va)
        k_vamax<<<grid_for(N), 256, 0, s>>>(N, T, dimb * dimb,
                                            4.0 * PI * dimrho, box, boy, boz,
                                            red, rho0, dmax);
      else
        k_max<<<grid_for(N), 256, 0, s>>>(N, red, dmax);
      unsigned long long bits;
      CK(cudaMemcpyAsync(&bits, dmax, 8, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      std::memcpy(out, &bits, 8);
      return SPARC_OK;
    };
    // The decade search of initialize.f90:966-975: the inner loop steps T
    // by dtemp until the maximum Alfven speed reaches maxva.  The steps of
    // one pass are formed on the host by the same repeated additions and
    // their maxima evaluated together (one synchronisation per pass instead
    // of one per step); the loop then stops at the same step.
    auto vamax_steps = [&](double T0, double d, double *Tstop, double *vastop) -> int {
      double Tc = T0;
      for (;;) {
        VaCand C{};
        C.n = 0;
        while (C.n < kVaCand) {
          Tc = Tc + d;
          C.T[C.n++] = Tc;
          if (!(Tc < 1.0e10)) break;  // the loop tests T < 1e10 before a step
        }
        CK(cudaMemsetAsync(dmax, 0, 8 * kVaCand, s));
        k_vamax_multi<<<grid_for(N), 256, 0, s>>>(N, C, dimb * dimb, 4.0 * PI * dimrho, box,
                                                  boy, boz, red, rho0, dmax);
        unsigned long long bits[kVaCand];
        CK(cudaMemcpyAsync(bits, dmax, 8 * kVaCand, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (int c = 0; c < C.n; ++c) {
          double v2;
          std::memcpy(&v2, &bits[c], 8);
          const double v = sqrt(v2);
          if (!(v < P.maxva) || !(C.T[c] < 1.0e10)) {
            *Tstop = C.T[c];
            *vastop = v;
            return SPARC_OK;
          }
        }
      }
    };
    double va = 0.0, dtemp = 1.0e9, T = -dtemp, mx = 0.0;
    if (devmax(false, 0.0, &mx)) return SPARC_ERR_CUDA;
    if (mx > 0.0) {
      while (dtemp > 1.0e-5 && T < 1.0e10 - 1.1) {
        if (va < P.maxva && T < 1.0e10)
          if (vamax_steps(T, dtemp, &T, &va)) return SPARC_ERR_CUDA;
        T = T - dtemp;
        dtemp = dtemp / 10.0;
        va = 0.0;
      }
    } else {
      T = 1.0e10;
    }
    each(N, s, [=] __device__(long long n) { red[n] = T / (T + red[n]); });
    // curl B0, initialize.f90:993-1006
    double *cbx = h->cbx = up(h, nullptr, N);
    double *cby = h->cby = up(h, nullptr, N);
    double *cbz = h->cbz = up(h, nullptr, N);
    if (!cbx || !cby || !cbz) return SPARC_ERR_NOMEM;
    int r = 0;
    r |= launch_derivative(h, 0, bc, boy, cbz, s);
    r |= launch_derivative(h, 1, bc, box, tmp, s);
    each(N, s, [=] __device__(long long n) { cbz[n] = cbz[n] - tmp[n]; });
    r |= launch_derivative(h, 1, bc, boz, tmp, s);
    r |= launch_derivative(h, 2, 1, boy, cbx, s);
    each(N, s, [=] __device__(long long n) { cbx[n] = tmp[n] - cbx[n]; });
    r |= launch_derivative(h, 2, 1, box, cby, s);
    r |= launch_derivative(h, 0, bc, boz, tmp, s);
    each(N, s, [=] __device__(long long n) { cby[n] = cby[n] - tmp[n]; });
    if (r) return SPARC_ERR_CUDA;
  }
  // initialize.f90:1012-1034
  double *rhoinv = h->rhoinv = up(h, nullptr, N);
  double *c2rho0 = h->c2rho0 = up(h, nullptr, N);
  double *grz = h->grz = up(h, nullptr, N);
  double *gpz = h->gpz = up(h, nullptr, N);
  if (!rhoinv || !c2rho0 || !grz || !gpz) return SPARC_ERR_NOMEM;
  each(N, s, [=] __device__(long long n) {
    rhoinv[n] = 1.0 / rho0[n];
    c2rho0[n] = c2[n] * rho0[n];
  });
  if (launch_derivative(h, 2, 1, rho0, grz, s) ||
      launch_derivative(h, 2, 1, p0, gpz, s))
    return SPARC_ERR_CUDA;
  if (P.stabilise) {
    double *dz = up(h, z.data(), nz);
    double *dg = up(h, h->g.data(), nz);
    if (!dz || !dg) return SPARC_ERR_NOMEM;
    const double lo = (double)0.9998f, hi = (double)1.0001f;
    const double add = 1.e-4 * RSUN / (dimrho * (dimc * dimc));
    const long long NXY = (long long)nx * ny;
    each(N, s, [=] __device__(long long n) {
      int k = (int)(n / NXY);
      double zk = dz[k];
      if (zk > lo && zk < 1.0)
        gpz[n] = fmax(c2[n] * grz[n] + add, -rho0[n] * dg[k]);
      else if (zk <= lo)
        gpz[n] = fmax(c2[n] * grz[n], -rho0[n] * dg[k]);
      else if (zk >= hi)
        gpz[n] = fmax(c2[n] * grz[n], -rho0[n] * dg[k]);
    });
  }

  // ------------------------------------------------ CPML, initialize.f90:1036-1216
  const int BXY = P.block_x * P.block_y;
  h->g_blk.assign((size_t)BXY * nz, 0.0);
  for (int b = 0; b < BXY; ++b)
    for (int k = 0; k < nz; ++k) h->g_blk[(size_t)b * nz + k] = h->g[k];
  double *sd = h->source_damp = up(h, nullptr, N);
  if (!sd) return SPARC_ERR_NOMEM;
  CK(cudaMemsetAsync(sd, 0, N * 8, s));
  const int mag = h->magnetic ? 1 : 0;
  double *sponge = h->sponge;
  double *redp = h->red;
  if (h->use_pml) {
    double *tempin = tmp;
    each(N, s, [=] __device__(long long n) {
      if (mag)
        tempin[n] = sqrt(c2[n] + redp[n] * (box[n] * box[n] + boy[n] * boy[n] +
                                            boz[n] * boz[n]) / rho0[n]);
      else
        tempin[n] = sqrt(c2[n]);
    });
    const double pml_f0 = PI * 0.005 * diml / dimc;
    std::vector<double> sdx(nx, 0.0), sdy(ny, 0.0);
    // face order: z_bot, z_top, x_bot, x_top, y_bot, y_top
    for (int f = 0; f < 6; ++f) {
      FaceDev &F = h->faces[f];
      if (!F.on) continue;
      // face order z_bot, z_top, x_bot, x_top, y_bot, y_top; axis 0 x, 1 y, 2 z
      const int axis = f < 2 ? 2 : (f < 4 ? 0 : 1);
      const bool top = f & 1;
      {  // the slab's normal extent must be the PML width (guards the kernel)
        const int ext = axis == 0 ? F.n0 : (axis == 1 ? F.n1 : F.n2);
        const int o1 = axis == 0 ? F.n1 : F.n0, o2 = axis == 2 ? F.n1 : F.n2;
        const int w1 = axis == 0 ? ny : nx, w2 = axis == 2 ? ny : nz;
        if (ext != F.np || o1 != w1 || o2 != w2) {
          h->err = "CPML face layout mismatch";
          return SPARC_ERR_INVALID;
        }
      }
      const double *q = axis == 0 ? (top ? P.pml_xt : P.pml_xb)
                                  : axis == 1 ? (top ? P.pml_yt : P.pml_yb)
                                              : (top ? P.pml_zt : P.pml_zb);
      const int np = F.np;
      const int n = axis == 0 ? nx : (axis == 1 ? ny : nz);
      const std::vector<double> &ax =
          axis == 0 ? h->xaxis : (axis == 1 ? h->yaxis : h->zaxis);
      const double L = top ? ax[n - 1] - ax[n - np] : ax[np - 1] - ax[0];
      Layers Ly;
      Ly.rn.resize(np); Ly.rn1.resize(np); Ly.alpha.resize(np); Ly.kap.resize(np);
      for (int kk = 0; kk < np; ++kk) {
        int gq = top ? n - np + kk : kk;
        double ratio = top ? (-(ax[n - np] - ax[gq])) / L : (ax[np - 1] - ax[gq]) / L;
        Ly.rn[kk] = std::pow(ratio, q[1]);
        Ly.rn1[kk] = std::pow(ratio, q[1] + 1.0);
        Ly.alpha[kk] = top ? pml_f0 * (ax[n - 1] - ax[gq]) / L
                           : pml_f0 * (ax[gq] - ax[0]) / L;
        Ly.kap[kk] = 1.0 + (q[2] - 1.0) * Ly.rn[kk];
        if (axis == 0) sdx[gq] = Ly.rn[kk];
        if (axis == 1) sdy[gq] = Ly.rn[kk];
      }
      std::vector<double> lay(4 * np);
      for (int kk = 0; kk < np; ++kk) {
        lay[kk] = Ly.rn[kk];
        lay[np + kk] = Ly.rn1[kk];
        lay[2 * np + kk] = Ly.alpha[kk];
        lay[3 * np + kk] = Ly.kap[kk];
      }
      double *dl = up(h, lay.data(), lay.size());
      double *pa = up(h, nullptr, F.cnt), *pb = up(h, nullptr, F.cnt),
             *pk = up(h, nullptr, F.cnt);
      if (!dl || !pa || !pb || !pk) return SPARC_ERR_NOMEM;
      F.pa = pa; F.pb = pb; F.pk = pk;
      const double q0 = q[0], q1 = q[1], q3 = q[3];
      const int n0 = F.n0, n1 = F.n1;
      const int inner = top ? n - np : np - 1;  // plane of tempin
      each(F.cnt, s, [=] __device__(long long t) {
        int a0 = (int)(t % n0), a1 = (int)((t / n0) % n1),
            a2 = (int)(t / ((long long)n0 * n1));
        int kk = axis == 0 ? a0 : (axis == 1 ? a1 : a2);
        int gi = a0, gj = a1, gk = a2;
        if (axis == 0 && top) gi = nx - np + a0;
        if (axis == 1 && top) gj = ny - np + a1;
        if (axis == 2 && top) gk = nz - np + a2;
        int ti = axis == 0 ? inner : gi, tj = axis == 1 ? inner : gj,
            tk = axis == 2 ? inner : gk;
        long long gidx = (long long)gi + (long long)nx * ((long long)gj + (long long)ny * gk);
        double tin = tempin[(long long)ti + (long long)nx * ((long long)tj + (long long)ny * tk)];
        double rn = dl[kk], rn1 = dl[np + kk], alpha = dl[2 * np + kk],
               kap = dl[3 * np + kk];
        double damp = q0 * tin * (q1 + 1.0) / (2.0 * L) * rn;
        pk[t] = kap;
        pb[t] = -alpha - damp / kap;
        pa[t] = -damp / (kap * kap);
        if (axis == 2) {
          grz[gidx] = grz[gidx] * alpha / kap / (damp / kap + alpha);
          gpz[gidx] = gpz[gidx] * alpha / kap / (damp / kap + alpha);
        }
        sponge[gidx] = sponge[gidx] + q3 * tin * rn1;
      });
      if (axis == 2) {  // gravity of each ZBOT/ZTOP rank: its local (1,1)
        // the inner-plane value of each block column's first point, read
        // back in one synchronisation (a set-up that shares the device with
        // a running batch pays for every synchronisation)
        std::vector<double> tins(BXY);
        for (int b = 0; b < BXY; ++b) {
          int i0 = h->bxs[b % P.block_x], j0 = h->bys[b / P.block_x];
          CK(cudaMemcpyAsync(&tins[b], tempin + I(i0, j0, inner), 8, cudaMemcpyDeviceToHost, s));
        }
        CK(cudaStreamSynchronize(s));
        for (int b = 0; b < BXY; ++b) {
          for (int kk = 0; kk < np; ++kk) {
            int gk = top ? nz - np + kk : kk;
            const double tin = tins[b];
            double damp = q0 * tin * (q1 + 1.0) / (2.0 * L) * Ly.rn[kk];
            double kap = Ly.kap[kk], alpha = Ly.alpha[kk];
            double &gg = h->g_blk[(size_t)b * nz + gk];
            gg = gg * alpha / kap / (damp / kap + alpha);
          }
        }
      }
    }
    std::vector<double> sdxy(nx + ny);
    std::copy(sdx.begin(), sdx.end(), sdxy.begin());
    std::copy(sdy.begin(), sdy.end(), sdxy.begin() + nx);
    double *dsd = up(h, sdxy.data(), sdxy.size());
    if (!dsd) return SPARC_ERR_NOMEM;
    each(N, s, [=] __device__(long long n) {
      int i = (int)(n % nx), j = (int)((n / nx) % ny);
      sd[n] = fmax(dsd[i], dsd[nx + j]);
    });
  }
  {
    const bool per = h->periodic;
    each(N, s, [=] __device__(long long n) { sd[n] = per ? 1.0 : 1.0 - sd[n]; });
  }
  if (h->magnetic) {  // initialize.f90:1219-1228
    h->grx = up(h, nullptr, N); h->gpx = up(h, nullptr, N);
    h->gry = up(h, nullptr, N); h->gpy = up(h, nullptr, N);
    if (!h->grx || !h->gpx || !h->gry || !h->gpy) return SPARC_ERR_NOMEM;
    if (launch_derivative(h, 0, bc, rho0, h->grx, s) ||
        launch_derivative(h, 0, bc, p0, h->gpx, s) ||
        launch_derivative(h, 1, bc, rho0, h->gry, s) ||
        launch_derivative(h, 1, bc, p0, h->gpy, s))
      return SPARC_ERR_CUDA;
  }
  h->d_gblk = up(h, h->g_blk.data(), h->g_blk.size());
  if (!h->d_gblk) return SPARC_ERR_NOMEM;

  // 1-D profiles of the horizontally uniform quiet background
  h->bg1d = h->quiet && h->periodic;
  if (h->bg1d) {
    const long long NXY = (long long)nx * ny;
    double **dst[7] = {&h->rho0_1, &h->p0_1, &h->rhoinv_1, &h->c2rho0_1,
                       &h->grz_1, &h->gpz_1, &h->sponge_1};
    const double *srcs[7] = {rho0, p0, rhoinv, c2rho0, grz, gpz, sponge};
    for (int a = 0; a < 7; ++a) {
      double *d = up(h, nullptr, nz);
      if (!d) return SPARC_ERR_NOMEM;
      *dst[a] = d;
      CK(cudaMemcpy2DAsync(d, 8, srcs[a], NXY * 8, 8, nz,
                           cudaMemcpyDeviceToDevice, s));
    }
  }
  // layer-only profiles for the z faces of the quiet background
  for (int f = 0; f < 2; ++f) {
    FaceDev &F = h->faces[f];
    if (!F.on || !h->quiet) continue;
    const long long NXY = (long long)F.n0 * F.n1;
    const double **pp[3] = {&F.pa, &F.pb, &F.pk};
    for (int a = 0; a < 3; ++a) {
      double *d = up(h, nullptr, F.np);
      if (!d) return SPARC_ERR_NOMEM;
      CK(cudaMemcpy2DAsync(d, 8, *pp[a], NXY * 8, 8, F.np,
                           cudaMemcpyDeviceToDevice, s));
      *pp[a] = d;
    }
    F.uniform = 1;
  }
  // 1/kappa of every face (the stage kernels multiply by it)
  for (int f = 0; f < 6; ++f) {
    FaceDev &F = h->faces[f];
    if (!F.on) continue;
    const long long n = F.uniform ? F.np : F.cnt;
    double *ki = up(h, nullptr, n);
    if (!ki) return SPARC_ERR_NOMEM;
    const double *pk = F.pk;
    each(n, s, [=] __device__(long long t) { ki[t] = 1.0 / pk[t]; });
    F.pki = ki;
  }
  CK(cudaStreamSynchronize(s));
  return SPARC_OK;
}

}  // namespace sparc
