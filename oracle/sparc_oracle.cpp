// sparc_oracle.cpp -- TEST INFRASTRUCTURE (the oracle), not the product.
//
// Parity unpinned by the reference itself: the reference has no tests or
// golden vectors and cannot be built here (Fortran, MPI, parallel HDF5
// absent); this restatement is pinned by analytic known-answer tests and
// by committed golden fixtures of its own output (sparc_oracle.h).
//
// CPU FP64 restatement of the reference SPARC linear wave time step over the
// global domain (see sparc_oracle.h).  Array layout is the reference's:
// Fortran order, x fastest; indices here are 0-based.  Expressions keep the
// reference's operand order so that the restatement rounds like the Fortran
// (left-to-right evaluation, SUM accumulated from the first tap).  Built with
// -ffp-contract=off so no FMA is introduced.
//
// The reference runs as MPI ranks on a block_x x block_y x block_z grid.
// Where a result depends on the rank layout (the z-PML gravity factor uses
// the rank-local (1,1) column, initialize.f90:1067/1095; PSR pulses are
// culled per rank, all_modules.f90:594-598/644-648) the layout is an explicit
// parameter.  Derivative and filter edges follow the rules of a run with at
// least two ranks along every non-periodic axis (initialize.f90:541-557
// aborts otherwise when CPML is on).

#include "sparc_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double RSUN = 69598946770.0;     // all_modules.f90:56
const double PI = 3.14159265358979;    // all_modules.f90:56 (truncated pi)

// Default-real (single precision) Fortran literals, promoted to double.
inline double sp(float f) { return (double)f; }

struct Blocks {  // rank extents along one axis, initialize.f90:77-120
  std::vector<int> start, len;
  void init(int n, int B) {
    start.assign(B, 0);
    len.assign(B, n / B);
    int rem = n - (n / B) * B;
    for (int i = 0; i < rem; ++i) len[i] += 1;
    for (int b = 1; b < B; ++b) start[b] = start[b - 1] + len[b - 1];
  }
  int of(int i) const {
    int b = 0;
    while (b + 1 < (int)start.size() && i >= start[b + 1]) ++b;
    return b;
  }
};

struct Face {  // one CPML face: RK state, stage value, RHS, profiles
  bool on = false;
  int n0 = 0, n1 = 0, n2 = 0, np = 0, P = 0;
  std::vector<double> vars, psi, scr;  // n0*n1*n2*P
  std::vector<double> a, b, kappa;     // n0*n1*n2
  size_t cnt() const { return (size_t)n0 * n1 * n2; }
  size_t id(int i, int j, int k) const {
    return (size_t)i + (size_t)n0 * ((size_t)j + (size_t)n1 * k);
  }
};

}  // namespace

struct orc_handle {
  sparc_params P;
  int nx, ny, nz, V, Pp;
  size_t N;
  bool magnetic, quiet, periodic, use_pml, use_hpml;
  int gxy, gz, xyfreq, zfreq;
  Blocks bx, by, bz;
  double dp[6][11];
  double dfxy[11], dfz[11];
  std::vector<double> xaxis, yaxis, zaxis, g, stretch, gblk;
  double stretchx, stretchy, dimc, dimrho, diml, dimb, deltat, betas[5];
  std::vector<double> rho0, p0, c_speed, c2, rhoinv, c2rho0, gradrho0_z,
      gradp0_z, spongexyz, box, boy, boz, curlbox, curlboy, curlboz,
      gradrho0_x, gradrho0_y, gradp0_x, gradp0_y, reduction, source_damp,
      src_scale_beta, cq, invrho0q, spongez;
  Face zb, zt, xb, xt, yb, yt;
  std::vector<double> a, temp, scr, forcing;
  std::vector<double> w[16];
  sparc_source src;
  std::vector<double> vr;          // PULSE = 0: the scaled forcing series
  std::vector<double> source_dep;  // PULSE = 0: depth profile (all_modules.f90:300)
  std::vector<sparc_pulse> pulses;
  std::vector<unsigned char> pulse_in_block;  // npulses * nblocks
  int64_t forcing_iter = -1;
  sparc_diag diag;

  size_t I(int i, int j, int k) const {
    return (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
  }
  int gcol(int i, int j) const {  // block column of a point
    return bx.of(i) + P.block_x * by.of(j);
  }

  // ---------------------------------------------------------- derivatives
  // ddx, derivatives.f90:10-116.  bc 1 on a non-periodic axis: one-sided rows
  // dpxy(1..5,:) at the low edge (:72) and -dpxy on the reversed field at the
  // high edge (:98); periodic: halo from the wrapped neighbour; bc 5 on a
  // non-periodic axis: centred with zero ghosts.  A periodic axis wraps
  // whatever bc is.  The reference would take the one-sided rows on its
  // XBOT/XTOP ranks for bc 1 even in a periodic communicator
  // (derivatives.f90:62-76, initialize.f90:66-67); its step passes bc 5
  // whenever the axis is periodic, so that branch is never reached on the
  // step's path, and the restatement leaves it out.
  void ddx(const double *in, double *out, int bc) const {
    const double *c = dp[5];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        const double *r = in + I(0, j, k);
        double *o = out + I(0, j, k);
        for (int i = 0; i < nx; ++i) {
          double s = 0.0;
          if (periodic) {
            for (int m = 0; m < 11; ++m) {
              int ii = i - 5 + m;
              ii = (ii % nx + nx) % nx;
              s += r[ii] * c[m];
            }
            o[i] = stretchx * s;
          } else if (bc == 1 && i < 5) {
            for (int m = 0; m < 11; ++m) s += r[m] * dp[i][m];
            o[i] = stretchx * s;
          } else if (bc == 1 && i >= nx - 5) {
            int row = nx - 1 - i;
            for (int m = 0; m < 11; ++m) s += r[nx - 1 - m] * dp[row][m];
            o[i] = -stretchx * s;
          } else {
            for (int m = 0; m < 11; ++m) {
              int ii = i - 5 + m;
              double v = (ii >= 0 && ii < nx) ? r[ii] : 0.0;
              s += v * c[m];
            }
            o[i] = stretchx * s;
          }
        }
      }
  }

  // ddy, derivatives.f90:226-341 (same edge rules as ddx along y).
  void ddy(const double *in, double *out, int bc) const {
    const double *c = dp[5];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        double *o = out + I(0, j, k);
        for (int i = 0; i < nx; ++i) {
          double s = 0.0;
          if (periodic) {
            for (int m = 0; m < 11; ++m) {
              int jj = j - 5 + m;
              jj = (jj % ny + ny) % ny;
              s += in[I(i, jj, k)] * c[m];
            }
            o[i] = stretchy * s;
          } else if (bc == 1 && j < 5) {
            for (int m = 0; m < 11; ++m) s += in[I(i, m, k)] * dp[j][m];
            o[i] = stretchy * s;
          } else if (bc == 1 && j >= ny - 5) {
            int row = ny - 1 - j;
            for (int m = 0; m < 11; ++m)
              s += in[I(i, ny - 1 - m, k)] * dp[row][m];
            o[i] = -stretchy * s;
          } else {
            for (int m = 0; m < 11; ++m) {
              int jj = j - 5 + m;
              double v = (jj >= 0 && jj < ny) ? in[I(i, jj, k)] : 0.0;
              s += v * c[m];
            }
            o[i] = stretchy * s;
          }
        }
      }
  }

  // ddz, derivatives.f90:451-562.  z is never periodic.  bc 1: the bottom
  // (ZBOT) keeps the centred stencil with zero ghosts (:509-518), the top
  // (ZTOP) uses -dpz(kk,:) on the reversed column (:536-545).
  void ddz(const double *in, double *out, int bc) const {
    const double *c = dp[5];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        double *o = out + I(0, j, k);
        for (int i = 0; i < nx; ++i) {
          double s = 0.0;
          if (bc == 1 && k >= nz - 5) {
            int row = nz - 1 - k;
            for (int m = 0; m < 11; ++m)
              s += in[I(i, j, nz - 1 - m)] * dp[row][m];
            o[i] = -stretch[k] * s;
          } else {
            for (int m = 0; m < 11; ++m) {
              int kk = k - 5 + m;
              double v = (kk >= 0 && kk < nz) ? in[I(i, j, kk)] : 0.0;
              s += v * c[m];
            }
            o[i] = stretch[k] * s;
          }
        }
      }
  }

  void deriv(int dir, const double *in, double *out, int bc) const {
    if (dir == 0) ddx(in, out, bc);
    else if (dir == 1) ddy(in, out, bc);
    else ddz(in, out, bc);
  }

  // ------------------------------------------------------------- filters
  // filtx/filty, derivatives.f90:119-223, 345-447: periodic -> wrapped
  // centred filter everywhere; otherwise the g_xy_filt edge points are
  // copied (g = 5) or zeroed (g = 3).
  void filt_xy(int dir, const double *in, double *out) const {
    const int g = gxy, n = dir == 0 ? nx : ny;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          int q = dir == 0 ? i : j;
          double s = 0.0;
          if (!periodic && (q < g || q >= n - g)) {
            out[I(i, j, k)] = (g == 3) ? 0.0 : in[I(i, j, k)];
            continue;
          }
          for (int m = 0; m < 2 * g + 1; ++m) {
            int qq = q - g + m;
            qq = (qq % n + n) % n;
            double v = dir == 0 ? in[I(qq, j, k)] : in[I(i, qq, k)];
            s += v * dfxy[m];
          }
          out[I(i, j, k)] = s;
        }
  }

  // filtz, derivatives.f90:565-642: the g_z_filt points at each end are
  // copied unfiltered (:624, :635) for both filter widths.
  void filt_z(const double *in, double *out) const {
    const int g = gz;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          if (k < g || k >= nz - g) {
            out[I(i, j, k)] = in[I(i, j, k)];
            continue;
          }
          double s = 0.0;
          for (int m = 0; m < 2 * g + 1; ++m)
            s += in[I(i, j, k - g + m)] * dfz[m];
          out[I(i, j, k)] = s;
        }
  }

  void filt(int dir, const double *in, double *out) const {
    if (dir == 2) filt_z(in, out);
    else filt_xy(dir, in, out);
  }

  // FILTER_VARS, derivatives.f90:659-703.
  void filter_vars(int64_t time) {
    double *f = w[0].data();
    double *t = w[1].data();
    for (int l = 0; l < V; ++l) {
      double *al = a.data() + (size_t)l * N;
      if (time % xyfreq == 0) {
        for (int dir = 1; dir >= 0; --dir) {  // y first, then x
          if (!periodic) edge_average(dir, gxy, al, t);
          filt_xy(dir, al, f);
          apply_filter(al, f, gxy, P.s_xy);
        }
      }
      if (time % zfreq == 0) {
        edge_average(2, gz, al, t);
        filt_z(al, f);
        apply_filter(al, f, gz, P.s_z);
      }
    }
  }

  void apply_filter(double *al, const double *f, int g, double s) const {
#pragma omp parallel for schedule(static)
    for (size_t n = 0; n < N; ++n)
      al[n] = (g == 3) ? al[n] - s * f[n] : f[n];
  }

  // Edge pre-averaging of FILTER_VARS (derivatives.f90:672-674, 681-683,
  // 691-693): points 2..g and n-g+1..n-1 become the mean of their old
  // neighbours (array-assignment semantics: all right-hand sides first).
  void edge_average(int dir, int g, double *al, double *tmp) const {
    std::memcpy(tmp, al, N * sizeof(double));
    const int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          int q = dir == 0 ? i : (dir == 1 ? j : k);
          bool top = (q >= n - g && q <= n - 2);
          bool bot = (q >= 1 && q <= g - 1);
          if (!top && !bot) continue;
          size_t st = dir == 0 ? 1 : (dir == 1 ? (size_t)nx : (size_t)nx * ny);
          size_t id = I(i, j, k);
          al[id] = (tmp[id + st] + tmp[id - st]) / 2.0;
        }
  }


  // ------------------------------------------------------------- sources
  // PULSE = 1, driver.f90:137-148 (operand order kept).
  void forcing_pulse(int64_t nn) {
    const double t = (double)nn * P.timestep;
    const double amp = src.amp, t0 = src.t0, t1 = src.t1, st = src.st;
    const double Lx = P.xlength, Ly = P.ylength;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          double f = amp / 0.56458272 / dimc;
          f = f * std::sin(2.0 * PI * (t - t1 + 2.0 * t0) / t0);
          f = f * std::exp(-1.0 * ((t - t1) * (t - t1)) / (2.0 * (st * st)));
          double ax = xaxis[i] * Lx / RSUN - src.px / diml;
          double ay = yaxis[j] * Ly / RSUN - src.py / diml;
          double sr = src.sr / diml;
          f = f * std::exp(-1.0 * (ax * ax + ay * ay) / (2.0 * (sr * sr)));
          double az = zaxis[k] - (src.pz / diml + 1.0);
          double sz = src.sz / diml;
          f = f * std::exp(-1.0 * (az * az) / (2.0 * (sz * sz)));
          forcing[I(i, j, k)] = f;
        }
  }

  // RUN_PSR_PULSE, all_modules.f90:592-611 and 644-660: every pulse whose
  // 3-sigma box reaches a rank's block is added over that whole block.
  bool psr_in_block(const sparc_pulse &q, int b) const {
    int bxi = b % P.block_x, byi = (b / P.block_x) % P.block_y,
        bzi = b / (P.block_x * P.block_y);
    double x1 = xaxis[bx.start[bxi]], xN = xaxis[bx.start[bxi] + bx.len[bxi] - 1];
    double y1 = yaxis[by.start[byi]], yN = yaxis[by.start[byi] + by.len[byi] - 1];
    double z1 = zaxis[bz.start[bzi]], zN = zaxis[bz.start[bzi] + bz.len[bzi] - 1];
    auto mod1 = [](double v) { return v - std::floor(v); };
    bool cx = ((mod1(q.px + 3.0 * q.sr) >= x1) || (q.px + 3.0 * q.sr >= xaxis[nx - 1])) &&
              ((mod1(q.px - 3.0 * q.sr) <= xN) || (q.px - 3.0 * q.sr <= xaxis[0]));
    bool cy = ((mod1(q.py + 3.0 * q.sr) >= y1) || (q.py + 3.0 * q.sr >= yaxis[ny - 1])) &&
              ((mod1(q.py - 3.0 * q.sr) <= yN) || (q.py - 3.0 * q.sr <= yaxis[0]));
    bool cz = (q.pz + 3.0 * q.sz >= z1) && (q.pz - 3.0 * q.sz <= zN);
    return cx && cy && cz;
  }

  void forcing_psr(int64_t nn) {
    const double t = (double)nn * P.timestep;
    const double st = src.psr_st;
    const int nb = P.block_x * P.block_y * P.block_z;
    const int passes = (nn == src.init) ? 2 : 1;  // all_modules.f90:560, 614
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        for (int i = 0; i < nx; ++i) {
          int blk = gcol(i, j) + P.block_x * P.block_y * bz.of(k);
          double f = 0.0;
          for (int pass = 0; pass < passes; ++pass)
            for (size_t n = 0; n < pulses.size(); ++n) {
              if (!pulse_in_block[n * nb + blk]) continue;
              const sparc_pulse &q = pulses[n];
              double x = xaxis[i], y = yaxis[j];
              double mx = std::min(std::min((x - q.px) * (x - q.px),
                                            (x - 1.0 - q.px) * (x - 1.0 - q.px)),
                                   (x + 1.0 - q.px) * (x + 1.0 - q.px));
              double my = std::min(std::min((y - q.py) * (y - q.py),
                                            (y - 1.0 - q.py) * (y - 1.0 - q.py)),
                                   (y + 1.0 - q.py) * (y + 1.0 - q.py));
              double v = invrho0q[k] * q.amp;
              v = v * std::sin(2.0 * PI * (t - q.t1) / q.t0);
              v = v * std::exp(-((t - q.t1) * (t - q.t1)) / (2.0 * (st * st)));
              v = v * std::exp(-(mx + my) / (2.0 * (q.sr * q.sr)));
              double dz = zaxis[k] - q.pz;
              v = v * std::exp(-(dz * dz) / (2.0 * (q.sz * q.sz)));
              f = f + v;
            }
          size_t id = I(i, j, k);
          forcing[id] = f * source_damp[id] * src_scale_beta[id];  // driver.f90:153
        }
      }
  }

  // PULSE = 0, LAGRANGE_INTERP (all_modules.f90:1892-1950) then
  // forcing * source_damp(:,:,1) (driver.f90:131-132), spread over the
  // layers by source_dep (RHS.f90:147, 641).  Samples the reference would
  // read past the end of the series count as absent (zero weight).
  void forcing_random(int64_t nn) {
    const double cad = src.cadforcing;
    const int ns = src.nseries;
    double xt = (double)nn * P.timestep / cad;
    const long long time1 = (long long)std::floor(xt) + 1;
    xt = (double)nn * P.timestep;
    double x[7];
    for (int j = 0; j < 7; ++j) x[j] = (double)(time1 - 4 + j) * cad;
    bool use[7];
    for (int j = 0; j < 4; ++j) use[j] = x[j] >= 0.0;
    use[4] = true;
    use[5] = time1 < ns;
    use[6] = time1 < ns - 1;
    for (int j = 0; j < 7; ++j) {
      const long long m = time1 - 4 + j;  // 0-based sample of vr(:,:,time1-3+j)
      use[j] = use[j] && m >= 0 && m < ns;
    }
    double den[7];  // (x_j - x_a) * (x_j - x_b) ... left to right
    for (int j = 0; j < 7; ++j) {
      double d = 1.0;
      bool first = true;
      for (int m = 0; m < 7; ++m) {
        if (m == j) continue;
        d = first ? x[j] - x[m] : d * (x[j] - x[m]);
        first = false;
      }
      den[j] = d;
    }
    const size_t NXY = (size_t)nx * ny;
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < NXY; ++q) {
      double f = 0.0;
      for (int j = 0; j < 7; ++j) {
        double lc = use[j] ? vr[q + NXY * (size_t)(time1 - 4 + j)] / den[j] : 0.0;
        // LC_j * (xt - x_a) * (xt - x_b) ... left to right, as the reference
        double t = lc;
        for (int m = 0; m < 7; ++m)
          if (m != j) t = t * (xt - x[m]);
        f = j == 0 ? t : f + t;
      }
      f = f * source_damp[q];  // source_damp(:,:,1)
      for (int k = 0; k < nz; ++k) forcing[q + NXY * (size_t)k] = f * source_dep[k];
    }
  }

  void build_forcing(int64_t nn) {
    if (forcing_iter == nn) return;
    if (src.kind == SPARC_SRC_PULSE) forcing_pulse(nn);
    else if (src.kind == SPARC_SRC_PSR) forcing_psr(nn);
    else if (src.kind == SPARC_SRC_RANDOM) forcing_random(nn);
    else std::fill(forcing.begin(), forcing.end(), 0.0);
    forcing_iter = nn;
  }

  // ----------------------------------------------------------------- RHS
  // CPML correction of one derivative on one face (RHS.f90:50-93, 424-546):
  //   RHSpsi = a*f' + b*psi ;  f' = f'/kappa + psi
  void pml_face(Face &F, int slot, double *d, int axis, bool top) {
    if (!F.on) return;
    const size_t cnt = F.cnt();
    const double *psi = F.psi.data() + (size_t)slot * cnt;
    double *rhs = F.scr.data() + (size_t)slot * cnt;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < F.n2; ++k)
      for (int j = 0; j < F.n1; ++j)
        for (int i = 0; i < F.n0; ++i) {
          size_t f = F.id(i, j, k);
          int gi = i, gj = j, gk = k;
          if (axis == 0 && top) gi = nx - F.np + i;
          if (axis == 1 && top) gj = ny - F.np + j;
          if (axis == 2 && top) gk = nz - F.np + k;
          size_t id = I(gi, gj, gk);
          rhs[f] = F.a[f] * d[id] + F.b[f] * psi[f];
          d[id] = d[id] / F.kappa[f] + psi[f];
        }
  }

  double grav(int i, int j, int k) const {
    return gblk[(size_t)gcol(i, j) * nz + k];
  }

  void add_forcing(double *RVx, double *RVy, double *RVz) const {
    if (src.kind == SPARC_SRC_NONE) return;
    const int dir = src.kind == SPARC_SRC_RANDOM ? 3 : src.dir;
    double *R = dir == 1 ? RVx : (dir == 2 ? RVy : RVz);
#pragma omp parallel for schedule(static)
    for (size_t n = 0; n < N; ++n) R[n] = R[n] + forcing[n];
  }

  // INIT_DAMPING, initialize.f90:1276-1340 (3-D): the rates of the half
  // spectrum, kx = 0..nx/2 fastest, then ky (the negative frequencies of y
  // from ny/2+1 on), kay2d in units of 1/Rsun, in the reference's order.
  std::vector<double> damp_rates;
  void init_damping() {
    const int nh = nx / 2 + 1;
    const double constx = 2.0 * PI * RSUN / P.xlength;
    const double consty = 2.0 * PI * RSUN / P.ylength;
    const double kayref = 902.0;
    damp_rates.assign((size_t)nh * ny, 0.0);
    for (int j = 0; j < ny; ++j) {
      const double ky = j <= ny / 2 ? (double)j : (double)(ny - j);
      for (int i = 0; i < nh; ++i) {
        const double kay = std::pow(
            constx * constx * ((double)i * (double)i) + consty * consty * (ky * ky), 0.5);
        damp_rates[(size_t)j * nh + i] = diml / dimc / nx / ny * 1.0e-6 *
                                         (500.0 * std::pow(kay / kayref, 2.2)) * 20.0;
      }
    }
  }

  // damp_velocity, all_modules.f90:1803-1888, applied as RHS.f90:166-172:
  // RHSv -= term, term(:,:,k) = c2r(r2c(v(:,:,k)) * rates) with FFTW's
  // unnormalised transforms (the 1/(nx*ny) is in the rates).  Restated as
  // direct sums: r2c along x (kx = 0..nx/2), a complex transform along y,
  // the product, its inverse along y, and c2r along x, which takes the
  // real parts of the kx = 0 and (even nx) kx = nx/2 bins and twice the
  // real part of the others, as a half-spectrum inverse does.
  void damp_velocity(const double *T, double *S) {
    const int nh = nx / 2 + 1;
    std::vector<double> cx((size_t)nx), sx((size_t)nx), cy((size_t)ny), sy((size_t)ny);
    for (int q = 0; q < nx; ++q) {
      cx[q] = std::cos(2.0 * M_PI * q / nx);
      sx[q] = std::sin(2.0 * M_PI * q / nx);
    }
    for (int q = 0; q < ny; ++q) {
      cy[q] = std::cos(2.0 * M_PI * q / ny);
      sy[q] = std::sin(2.0 * M_PI * q / ny);
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int l = 1; l < 4; ++l)
      for (int k = 0; k < nz; ++k) {
        const double *v = T + (size_t)l * N + (size_t)k * nx * ny;
        double *R = S + (size_t)l * N + (size_t)k * nx * ny;
        std::vector<double> ar((size_t)ny * nh), ai((size_t)ny * nh), br((size_t)ny * nh),
            bi((size_t)ny * nh);
        for (int j = 0; j < ny; ++j)  // r2c along x
          for (int m = 0; m < nh; ++m) {
            double re = 0.0, im = 0.0;
            for (int i = 0; i < nx; ++i) {
              const int q = (int)(((long long)m * i) % nx);
              re += v[(size_t)j * nx + i] * cx[q];
              im -= v[(size_t)j * nx + i] * sx[q];
            }
            ar[(size_t)j * nh + m] = re;
            ai[(size_t)j * nh + m] = im;
          }
        for (int p = 0; p < ny; ++p)  // along y, times the rates
          for (int m = 0; m < nh; ++m) {
            double re = 0.0, im = 0.0;
            for (int j = 0; j < ny; ++j) {
              const int q = (int)(((long long)p * j) % ny);
              const double xr = ar[(size_t)j * nh + m], xi = ai[(size_t)j * nh + m];
              re += xr * cy[q] + xi * sy[q];
              im += xi * cy[q] - xr * sy[q];
            }
            const double d = damp_rates[(size_t)p * nh + m];
            br[(size_t)p * nh + m] = re * d;
            bi[(size_t)p * nh + m] = im * d;
          }
        for (int j = 0; j < ny; ++j)  // inverse along y
          for (int m = 0; m < nh; ++m) {
            double re = 0.0, im = 0.0;
            for (int p = 0; p < ny; ++p) {
              const int q = (int)(((long long)p * j) % ny);
              const double xr = br[(size_t)p * nh + m], xi = bi[(size_t)p * nh + m];
              re += xr * cy[q] - xi * sy[q];
              im += xi * cy[q] + xr * sy[q];
            }
            ar[(size_t)j * nh + m] = re;
            ai[(size_t)j * nh + m] = im;
          }
        for (int j = 0; j < ny; ++j)  // c2r along x, subtracted from RHSv
          for (int i = 0; i < nx; ++i) {
            double t = ar[(size_t)j * nh];
            for (int m = 1; m < nh; ++m) {
              const int q = (int)(((long long)m * i) % nx);
              const double c = ar[(size_t)j * nh + m] * cx[q] - ai[(size_t)j * nh + m] * sx[q];
              t += (2 * m == nx) ? c : 2.0 * c;
            }
            R[(size_t)j * nx + i] -= t;
          }
      }
  }

  // scr zeroed on the global boundary planes (RHS.f90:154-164, 647-657).
  void zero_boundaries(double *S) const {
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          bool z = (k == 0 || k == nz - 1);
          bool xy = !periodic && (i == 0 || i == nx - 1 || j == 0 || j == ny - 1);
          if (z || xy)
            for (int l = 0; l < V; ++l) S[(size_t)l * N + I(i, j, k)] = 0.0;
        }
  }

  // MP_QUIET_3D, RHS.f90:18-175 (FLOWS and DAMPING off).
  void rhs_quiet(const double *T, double *S) {
    const double *rho = T, *vx = T + N, *vy = T + 2 * N, *vz = T + 3 * N,
                 *p = T + 4 * N;
    double *dvxdx = w[0].data(), *dvydy = w[1].data(), *dvzdz = w[2].data(),
           *gpx = w[3].data(), *gpy = w[4].data(), *gpz = w[5].data();
    const int bh = periodic ? 5 : 1;
    ddx(vx, dvxdx, bh);
    ddy(vy, dvydy, bh);
    ddz(vz, dvzdz, 1);
    ddx(p, gpx, bh);
    ddy(p, gpy, bh);
    ddz(p, gpz, 1);
    if (use_pml) {  // psi slots: 0 vz, 1 p (initialize.f90:742-746)
      pml_face(zb, 1, gpz, 2, false);
      pml_face(zb, 0, dvzdz, 2, false);
      pml_face(zt, 1, gpz, 2, true);
      pml_face(zt, 0, dvzdz, 2, true);
    }
    if (use_hpml) {
      pml_face(xb, 1, gpx, 0, false);
      pml_face(xb, 0, dvxdx, 0, false);
      pml_face(xt, 1, gpx, 0, true);
      pml_face(xt, 0, dvxdx, 0, true);
      pml_face(yb, 1, gpy, 1, false);
      pml_face(yb, 0, dvydy, 1, false);
      pml_face(yt, 1, gpy, 1, true);
      pml_face(yt, 0, dvydy, 1, true);
    }
    double *Rc = S, *Rx = S + N, *Ry = S + 2 * N, *Rz = S + 3 * N,
           *Rp = S + 4 * N;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          size_t n = I(i, j, k);
          double div = dvxdx[n] + dvydy[n] + dvzdz[n];
          double sg = spongexyz[n];
          Rc[n] = -gradrho0_z[n] * vz[n] - rho0[n] * div - sg * rho[n];
          Rx[n] = -rhoinv[n] * gpx[n] - sg * vx[n];
          Ry[n] = -rhoinv[n] * gpy[n] - sg * vy[n];
          Rz[n] = -rhoinv[n] * (gpz[n] + rho[n] * grav(i, j, k)) - vz[n] * sg;
          Rp[n] = -c2rho0[n] * div - vz[n] * gradp0_z[n] - sg * p[n];
        }
    // the forcing joins RHSv between the v_z line and RHSp (RHS.f90:134-152)
    add_forcing(Rx, Ry, Rz);
    zero_boundaries(S);
    if (P.damping) damp_velocity(T, S);  // RHS.f90:166-172
  }

  // MP_MHD_3D, RHS.f90:363-668 (FLOWS and DAMPING off).
  void rhs_mhd(const double *T, double *S) {
    const double *rho = T, *vx = T + N, *vy = T + 2 * N, *vz = T + 3 * N,
                 *p = T + 4 * N, *bxv = T + 5 * N, *byv = T + 6 * N,
                 *bzv = T + 7 * N;
    double *f1 = w[15].data(), *f2 = w[14].data(), *f3 = w[13].data();
#pragma omp parallel for schedule(static)
    for (size_t n = 0; n < N; ++n) {  // RHS.f90:394-396
      f1[n] = -vz[n] * boy[n] + vy[n] * boz[n];
      f2[n] = -vx[n] * boz[n] + vz[n] * box[n];
      f3[n] = -vy[n] * box[n] + vx[n] * boy[n];
    }
    double *dvxdx = w[0].data(), *dvydy = w[1].data(), *dvzdz = w[2].data(),
           *dxflux3 = w[3].data(), *gpy = w[4].data(), *dzflux1 = w[5].data(),
           *gpx = w[6].data(), *dyflux3 = w[7].data(), *dzflux2 = w[8].data(),
           *dxflux2 = w[9].data(), *dybz = w[10].data(), *dzbx = w[11].data(),
           *dxby = w[12].data();
    std::vector<double> &e0 = extra[0], &e1 = extra[1], &e2 = extra[2],
                        &e3 = extra[3], &e4 = extra[4];
    double *dybx = e0.data(), *gpz = e1.data(), *dxbz = e2.data(),
           *dyflux1 = e3.data(), *dzby = e4.data();
    const int bh = periodic ? 5 : 1;
    ddx(vx, dvxdx, bh);   ddy(vy, dvydy, bh);   ddz(vz, dvzdz, 1);
    ddx(f3, dxflux3, bh); ddy(p, gpy, bh);      ddz(f1, dzflux1, 1);
    ddx(p, gpx, bh);      ddy(f3, dyflux3, bh); ddz(f2, dzflux2, 1);
    ddx(f2, dxflux2, bh); ddy(bzv, dybz, bh);   ddz(bxv, dzbx, 1);
    ddx(byv, dxby, bh);   ddy(bxv, dybx, bh);   ddz(p, gpz, 1);
    ddx(bzv, dxbz, bh);   ddy(f1, dyflux1, bh); ddz(byv, dzby, 1);
    // psi slots (initialize.f90:742-871): z: 0 vz, 1 p, 2 dzbx, 3 dzby,
    // 4 inductionbx (dzflux2), 5 inductionby (dzflux1); x: 0 vx, 1 p,
    // 2 dxby, 3 dxbz, 4 inductionby (dxflux3), 5 inductionbz (dxflux2);
    // y: 0 vy, 1 p, 2 dybx, 3 dybz, 4 inductionbx (dyflux3),
    // 5 inductionbz (dyflux1)
    if (use_pml)
      for (int t = 0; t < 2; ++t) {
        Face &F = t ? zt : zb;
        pml_face(F, 1, gpz, 2, t);
        pml_face(F, 0, dvzdz, 2, t);
      }
    if (use_hpml)
      for (int t = 0; t < 2; ++t) {
        Face &X = t ? xt : xb, &Y = t ? yt : yb;
        pml_face(X, 1, gpx, 0, t);
        pml_face(X, 0, dvxdx, 0, t);
        pml_face(Y, 1, gpy, 1, t);
        pml_face(Y, 0, dvydy, 1, t);
      }
    if (use_pml)
      for (int t = 0; t < 2; ++t) {
        Face &F = t ? zt : zb;
        pml_face(F, 4, dzflux2, 2, t);
        pml_face(F, 5, dzflux1, 2, t);
        pml_face(F, 2, dzbx, 2, t);
        pml_face(F, 3, dzby, 2, t);
      }
    if (use_hpml)
      for (int t = 0; t < 2; ++t) {
        Face &X = t ? xt : xb, &Y = t ? yt : yb;
        pml_face(X, 4, dxflux3, 0, t);
        pml_face(X, 5, dxflux2, 0, t);
        pml_face(X, 2, dxby, 0, t);
        pml_face(X, 3, dxbz, 0, t);
        pml_face(Y, 4, dyflux3, 1, t);
        pml_face(Y, 5, dyflux1, 1, t);
        pml_face(Y, 2, dybx, 1, t);
        pml_face(Y, 3, dybz, 1, t);
      }
    double *Rc = S, *Rx = S + N, *Ry = S + 2 * N, *Rz = S + 3 * N,
           *Rp = S + 4 * N, *Rbx = S + 5 * N, *Rby = S + 6 * N,
           *Rbz = S + 7 * N;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          size_t n = I(i, j, k);
          double red = reduction[n];
          Rbx[n] = red * (dyflux3[n] - dzflux2[n]);
          Rby[n] = red * (dzflux1[n] - dxflux3[n]);
          Rbz[n] = red * (dxflux2[n] - dyflux1[n]);
          double div = dvxdx[n] + dvydy[n] + dvzdz[n];
          double cbx = dybz[n] - dzby[n];
          double cby = -dxbz[n] + dzbx[n];
          double cbz = dxby[n] - dybx[n];
          double sg = spongexyz[n];
          Rc[n] = -gradrho0_x[n] * vx[n] - gradrho0_y[n] * vy[n] -
                  gradrho0_z[n] * vz[n] - rho0[n] * div - sg * rho[n];
          Rp[n] = -c2rho0[n] * div - vx[n] * gradp0_x[n] -
                  vy[n] * gradp0_y[n] - vz[n] * gradp0_z[n] - sg * p[n];
          // CROSS (derivatives.f90:646-655) of curl b with B0
          double c1 = cby * boz[n] - cbz * boy[n];
          double c2v = box[n] * cbz - cbx * boz[n];
          double c3 = cbx * boy[n] - cby * box[n];
          double ri = rhoinv[n];
          double vxr = -ri * (gpx[n] - (c1 * red)) - sg * vx[n];
          double vyr = -ri * (gpy[n] - (c2v * red)) - sg * vy[n];
          double vzr = -ri * (gpz[n] - (c3 * red)) - sg * vz[n];
          // CROSS of curl B0 with b
          double d1 = curlboy[n] * bzv[n] - curlboz[n] * byv[n];
          double d2 = bxv[n] * curlboz[n] - curlbox[n] * bzv[n];
          double d3 = curlbox[n] * byv[n] - curlboy[n] * bxv[n];
          vxr = vxr + ri * d1 * red;
          vyr = vyr + ri * d2 * red;
          vzr = vzr + ri * d3 * red;
          vzr = vzr - ri * rho[n] * grav(i, j, k);  // RHS.f90:630
          Rx[n] = vxr;
          Ry[n] = vyr;
          Rz[n] = vzr;
        }
    add_forcing(Rx, Ry, Rz);
    zero_boundaries(S);
    if (P.damping) damp_velocity(T, S);  // RHS.f90:659-665
  }
  std::vector<double> extra[5];

  void rhs(const double *T, double *S) {
    if (magnetic) rhs_mhd(T, S);
    else rhs_quiet(T, S);
  }

  // ---------------------------------------------------------------- STEP
  Face *faces[6] = {&zb, &zt, &xb, &xt, &yb, &yt};

  // step.f90:20-63 (5-stage low-storage RK, same update for the CPML fields)
  void step() {
    for (int rk = 1; rk <= 5; ++rk) {
      const double beta = betas[rk - 1];
      if (rk == 1) {
        std::memcpy(temp.data(), a.data(), a.size() * sizeof(double));
        for (Face *F : faces)
          if (F->on) F->psi = F->vars;
      } else {
#pragma omp parallel for schedule(static)
        for (size_t n = 0; n < a.size(); ++n) temp[n] = a[n] + beta * scr[n];
        for (Face *F : faces)
          if (F->on)
            for (size_t n = 0; n < F->vars.size(); ++n)
              F->psi[n] = F->vars[n] + beta * F->scr[n];
      }
      rhs(temp.data(), scr.data());
    }
#pragma omp parallel for schedule(static)
    for (size_t n = 0; n < a.size(); ++n) a[n] = a[n] + deltat * scr[n];
    for (Face *F : faces)
      if (F->on)
        for (size_t n = 0; n < F->vars.size(); ++n)
          F->vars[n] = F->vars[n] + deltat * F->scr[n];
  }

  // norm() of all_modules.f90:684-706 on the kinetic-energy density of
  // driver.f90:161, and the fail criterion of driver.f90:175-183 (which
  // reads rho and p through the stage pointers, i.e. the stage-5 fields).
  void diagnostics(int64_t nn) {
    double sum = 0.0, mr = 1e300, mp = 1e300;
#pragma omp parallel for reduction(+ : sum) reduction(min : mr, mp) schedule(static)
    for (size_t n = 0; n < N; ++n) {
      double m = (rho0[n] + a[n]) *
                 (a[N + n] * a[N + n] + a[2 * N + n] * a[2 * N + n] +
                  a[3 * N + n] * a[3 * N + n]) / 2.0;
      sum += m * m;
      mr = std::min(mr, temp[n] + rho0[n]);
      mp = std::min(mp, temp[4 * N + n] + p0[n]);
    }
    double nrm = std::sqrt(sum / ((double)nx * (double)ny * (double)nz));
    diag.ke_norm = nrm * (dimc * dimc) * dimrho;
    diag.min_rho = mr;
    diag.min_p = mp;
    diag.iteration = nn;
    bool fail = (diag.ke_norm > 1000.0) || (mr <= 0.0) || (mp <= 0.0);
    if (fail && diag.fail_iteration < 0) diag.fail_iteration = nn;
  }

  int iterate_step(int64_t nn) {
    build_forcing(nn);
    step();
    diagnostics(nn);
    return 0;
  }

  void filter_after(int64_t nn) {
    if (nn != 0) filter_vars(nn);  // driver.f90:200
  }

  // ---------------------------------------------------------------- setup
  std::string setup(const sparc_params *p, const double *rho0_in,
                    const double *pre0_in, const double *cs0_in,
                    const double *bx0, const double *by0, const double *bz0,
                    const double *zaxis_mm, const double *grav_in);
  void init_coeffs();
  void init_pml();
};

// initexplicitders, initialize.f90:1927-2034 (published Bogey-Bailly
// optimized 11-point coefficients and the two filter stencils).
void orc_handle::init_coeffs() {
  static const double c7[7] = {-0.015625000, 0.093750000, -0.234375000,
                               0.312500000, -0.234375000, 0.093750000,
                               -0.015625000};
  const double c11[11] = {
      0.5 * 0.00195312500000, -0.5 * 0.01953125000000,
      0.5 * 0.08789062500000, -0.5 * 0.23437500000000,
      0.5 * 0.41015625000000, 0.75390625000000,
      0.5 * 0.41015625000000, -0.5 * 0.23437500000000,
      0.5 * 0.08789062500000, -0.5 * 0.01953125000000,
      0.5 * 0.00195312500000};
  for (int m = 0; m < 11; ++m) {
    dfxy[m] = gxy == 5 ? c11[m] : (m < 7 ? c7[m] : 0.0);
    dfz[m] = gz == 5 ? c11[m] : (m < 7 ? c7[m] : 0.0);
  }
  const double D[6][11] = {
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
      {-0.002484594688, +0.020779405824, -0.090320001280, +0.286511173973,
       -0.872756993962, 0.0, +0.872756993962, -0.286511173973,
       +0.090320001280, -0.020779405824, +0.002484594688}};
  std::memcpy(dp, D, sizeof(D));
}

static void alloc_face(Face &F, int n0, int n1, int n2, int np, int P) {
  F.on = true;
  F.n0 = n0; F.n1 = n1; F.n2 = n2; F.np = np; F.P = P;
  size_t c = F.cnt();
  F.vars.assign(c * P, 0.0);
  F.psi.assign(c * P, 0.0);
  F.scr.assign(c * P, 0.0);
  F.a.assign(c, 0.0);
  F.b.assign(c, 0.0);
  F.kappa.assign(c, 1.0);
}

// CPML profiles, damped background gradients/gravity and PML sponge,
// initialize.f90:1036-1216.
void orc_handle::init_pml() {
  std::vector<double> tempin(N);
  for (size_t n = 0; n < N; ++n) {
    if (magnetic)
      tempin[n] = std::sqrt(c2[n] + reduction[n] *
                                        (box[n] * box[n] + boy[n] * boy[n] +
                                         boz[n] * boz[n]) / rho0[n]);
    else
      tempin[n] = std::sqrt(c2[n]);
  }
  std::vector<double> sdx(nx, 0.0), sdy(ny, 0.0);
  const double pml_f0 = PI * 0.005 * diml / dimc;
  const int BXY = P.block_x * P.block_y;
  if (use_pml) {
    // bottom (ZBOT), initialize.f90:1048-1074
    {
      const int np = P.npml_zb;
      const double *q = P.pml_zb;
      const double L = zaxis[np - 1] - zaxis[0];
      for (int kk = 0; kk < np; ++kk) {
        double ratio = (zaxis[np - 1] - zaxis[kk]) / L;
        double rn = std::pow(ratio, q[1]);
        double alpha = pml_f0 * (zaxis[kk] - zaxis[0]) / L;
        double kap = 1.0 + (q[2] - 1.0) * rn;
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i) {
            size_t f = zb.id(i, j, kk), n = I(i, j, kk);
            double damp = q[0] * tempin[I(i, j, np - 1)] * (q[1] + 1.0) /
                          (2.0 * L) * rn;
            zb.kappa[f] = kap;
            zb.b[f] = -alpha - damp / kap;
            zb.a[f] = -damp / (kap * kap);
            gradrho0_z[n] = gradrho0_z[n] * alpha / kap / (damp / kap + alpha);
            gradp0_z[n] = gradp0_z[n] * alpha / kap / (damp / kap + alpha);
            spongexyz[n] = spongexyz[n] + q[3] * tempin[I(i, j, np - 1)] *
                                              std::pow(ratio, q[1] + 1.0);
          }
        for (int b = 0; b < BXY; ++b) {  // damp(1,1,kk) of each ZBOT rank
          int i0 = bx.start[b % P.block_x], j0 = by.start[b / P.block_x];
          double damp = q[0] * tempin[I(i0, j0, np - 1)] * (q[1] + 1.0) /
                        (2.0 * L) * rn;
          double &gg = gblk[(size_t)b * nz + kk];
          gg = gg * alpha / kap / (damp / kap + alpha);
        }
      }
    }
    // top (ZTOP), initialize.f90:1075-1104
    {
      const int np = P.npml_zt;
      const double *q = P.pml_zt;
      const double L = zaxis[nz - 1] - zaxis[nz - np];
      for (int kk = 0; kk < np; ++kk) {
        int kg = nz - np + kk;
        double ratio = (-(zaxis[nz - np] - zaxis[kg])) / L;
        double rn = std::pow(ratio, q[1]);
        double alpha = pml_f0 * (zaxis[nz - 1] - zaxis[kg]) / L;
        double kap = 1.0 + (q[2] - 1.0) * rn;
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i) {
            size_t f = zt.id(i, j, kk), n = I(i, j, kg);
            double damp = q[0] * tempin[I(i, j, nz - np)] * (q[1] + 1.0) /
                          (2.0 * L) * rn;
            zt.kappa[f] = kap;
            zt.b[f] = -alpha - damp / kap;
            zt.a[f] = -damp / (kap * kap);
            gradrho0_z[n] = gradrho0_z[n] * alpha / kap / (damp / kap + alpha);
            gradp0_z[n] = gradp0_z[n] * alpha / kap / (damp / kap + alpha);
            spongexyz[n] = spongexyz[n] + q[3] * tempin[I(i, j, nz - np)] *
                                              std::pow(ratio, q[1] + 1.0);
          }
        for (int b = 0; b < BXY; ++b) {
          int i0 = bx.start[b % P.block_x], j0 = by.start[b / P.block_x];
          double damp = q[0] * tempin[I(i0, j0, nz - np)] * (q[1] + 1.0) /
                        (2.0 * L) * rn;
          double &gg = gblk[(size_t)b * nz + kg];
          gg = gg * alpha / kap / (damp / kap + alpha);
        }
      }
    }
    if (use_hpml) {
      // x bottom, initialize.f90:1108-1129
      {
        const int np = P.npml_xb;
        const double *q = P.pml_xb;
        const double L = xaxis[np - 1] - xaxis[0];
        for (int ii = 0; ii < np; ++ii) {
          double ratio = (xaxis[np - 1] - xaxis[ii]) / L;
          double rn = std::pow(ratio, q[1]);
          double alpha = pml_f0 * (xaxis[ii] - xaxis[0]) / L;
          double kap = 1.0 + (q[2] - 1.0) * rn;
          sdx[ii] = rn;
          for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j) {
              size_t f = xb.id(ii, j, k), n = I(ii, j, k);
              double tin = tempin[I(np - 1, j, k)];
              double damp = q[0] * tin * (q[1] + 1.0) / (2.0 * L) * rn;
              xb.kappa[f] = kap;
              xb.b[f] = -alpha - damp / kap;
              xb.a[f] = -damp / (kap * kap);
              spongexyz[n] = spongexyz[n] + q[3] * tin * std::pow(ratio, q[1] + 1.0);
            }
        }
      }
      // x top, initialize.f90:1130-1152
      {
        const int np = P.npml_xt;
        const double *q = P.pml_xt;
        const double L = xaxis[nx - 1] - xaxis[nx - np];
        for (int ii = 0; ii < np; ++ii) {
          int ig = nx - np + ii;
          double ratio = (-(xaxis[nx - np] - xaxis[ig])) / L;
          double rn = std::pow(ratio, q[1]);
          double alpha = pml_f0 * (xaxis[nx - 1] - xaxis[ig]) / L;
          double kap = 1.0 + (q[2] - 1.0) * rn;
          sdx[ig] = rn;
          for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j) {
              size_t f = xt.id(ii, j, k), n = I(ig, j, k);
              double tin = tempin[I(nx - np, j, k)];
              double damp = q[0] * tin * (q[1] + 1.0) / (2.0 * L) * rn;
              xt.kappa[f] = kap;
              xt.b[f] = -alpha - damp / kap;
              xt.a[f] = -damp / (kap * kap);
              spongexyz[n] = spongexyz[n] + q[3] * tin * std::pow(ratio, q[1] + 1.0);
            }
        }
      }
      // y bottom, initialize.f90:1154-1176
      {
        const int np = P.npml_yb;
        const double *q = P.pml_yb;
        const double L = yaxis[np - 1] - yaxis[0];
        for (int jj = 0; jj < np; ++jj) {
          double ratio = (yaxis[np - 1] - yaxis[jj]) / L;
          double rn = std::pow(ratio, q[1]);
          double alpha = pml_f0 * (yaxis[jj] - yaxis[0]) / L;
          double kap = 1.0 + (q[2] - 1.0) * rn;
          sdy[jj] = rn;
          for (int k = 0; k < nz; ++k)
            for (int i = 0; i < nx; ++i) {
              size_t f = yb.id(i, jj, k), n = I(i, jj, k);
              double tin = tempin[I(i, np - 1, k)];
              double damp = q[0] * tin * (q[1] + 1.0) / (2.0 * L) * rn;
              yb.kappa[f] = kap;
              yb.b[f] = -alpha - damp / kap;
              yb.a[f] = -damp / (kap * kap);
              spongexyz[n] = spongexyz[n] + q[3] * tin * std::pow(ratio, q[1] + 1.0);
            }
        }
      }
      // y top, initialize.f90:1177-1199
      {
        const int np = P.npml_yt;
        const double *q = P.pml_yt;
        const double L = yaxis[ny - 1] - yaxis[ny - np];
        for (int jj = 0; jj < np; ++jj) {
          int jg = ny - np + jj;
          double ratio = (-(yaxis[ny - np] - yaxis[jg])) / L;
          double rn = std::pow(ratio, q[1]);
          double alpha = pml_f0 * (yaxis[ny - 1] - yaxis[jg]) / L;
          double kap = 1.0 + (q[2] - 1.0) * rn;
          sdy[jg] = rn;
          for (int k = 0; k < nz; ++k)
            for (int i = 0; i < nx; ++i) {
              size_t f = yt.id(i, jj, k), n = I(i, jg, k);
              double tin = tempin[I(i, ny - np, k)];
              double damp = q[0] * tin * (q[1] + 1.0) / (2.0 * L) * rn;
              yt.kappa[f] = kap;
              yt.b[f] = -alpha - damp / kap;
              yt.a[f] = -damp / (kap * kap);
              spongexyz[n] = spongexyz[n] + q[3] * tin * std::pow(ratio, q[1] + 1.0);
            }
        }
      }
    }
    for (int k = 0; k < nz; ++k)  // initialize.f90:1203-1207
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i)
          source_damp[I(i, j, k)] = std::max(sdx[i], sdy[j]);
  }
  for (size_t n = 0; n < N; ++n)  // initialize.f90:1212-1216
    source_damp[n] = periodic ? 1.0 : 1.0 - source_damp[n];
}

std::string orc_handle::setup(const sparc_params *pin, const double *rho0_in,
                              const double *pre0_in, const double *cs0_in,
                              const double *bx0, const double *by0,
                              const double *bz0, const double *zaxis_mm,
                              const double *grav_in) {
  P = *pin;
  nx = P.nx; ny = P.ny; nz = P.nz;
  if (nx < 22 || ny < 22 || nz < 22) return "grid must be at least 22 per axis";
  if (P.magnetic < 0 || P.magnetic > 2) return "magnetic must be 0, 1 or 2";
  if (P.block_x < 1 || P.block_y < 1 || P.block_z < 2)
    return "block counts must be >= 1 (x, y) and >= 2 (z)";
  periodic = P.periodic != 0;
  use_hpml = P.use_hpml != 0;
  use_pml = P.use_pml != 0 || use_hpml;
  if (periodic && use_hpml) return "PERIODIC and USE_HPML are exclusive";
  if (!periodic && (P.block_x < 2 || P.block_y < 2))
    return "non-periodic runs need >= 2 blocks along x and y";
  if (P.filter_mode_xy != 1 && P.filter_mode_xy != 2) return "filter_mode_xy";
  if (P.filter_mode_z != 1 && P.filter_mode_z != 2) return "filter_mode_z";
  if (P.damping != 0 && P.damping != 1) return "damping must be 0 or 1";
  magnetic = P.magnetic == 2;
  quiet = P.magnetic == 0;
  V = magnetic ? 8 : 5;
  Pp = magnetic ? 6 : 2;
  gxy = P.filter_mode_xy == 1 ? 5 : 3;
  gz = P.filter_mode_z == 1 ? 5 : 3;
  N = (size_t)nx * ny * nz;
  bx.init(nx, P.block_x);
  by.init(ny, P.block_y);
  bz.init(nz, P.block_z);
  if (use_pml) {
    if (P.npml_zb < 2 || P.npml_zt < 2) return "z PML needs >= 2 points";
    if (P.npml_zb > bz.len[0] || P.npml_zt > bz.len[P.block_z - 1])
      return "z PML thicker than the boundary block";
  }
  if (use_hpml) {
    if (P.npml_xb < 2 || P.npml_xt < 2 || P.npml_yb < 2 || P.npml_yt < 2)
      return "x/y PML needs >= 2 points";
    if (P.npml_xb > bx.len[0] || P.npml_xt > bx.len[P.block_x - 1] ||
        P.npml_yb > by.len[0] || P.npml_yt > by.len[P.block_y - 1])
      return "x/y PML thicker than the boundary block";
  }
  double tz = std::max(P.t_z, P.timestep), txy = std::max(P.t_xy, P.timestep);
  zfreq = (int)std::floor(tz / P.timestep + 1.0e-5);   // initialize.f90:1911-1912
  xyfreq = (int)std::floor(txy / P.timestep + 1.0e-5);

  // INITANDALLOCATE axes and metrics, initialize.f90:468-517
  xaxis.resize(nx); yaxis.resize(ny);
  for (int i = 0; i < nx; ++i)
    xaxis[i] = periodic ? (double)i / (double)nx : (double)i / (double)(nx - 1);
  for (int j = 0; j < ny; ++j)
    yaxis[j] = periodic ? (double)j / (double)ny : (double)j / (double)(ny - 1);
  stretchx = periodic ? RSUN / P.xlength * nx : RSUN / P.xlength * (nx - 1);
  stretchy = periodic ? RSUN / P.ylength * ny : RSUN / P.ylength * (ny - 1);

  // READ_IN_HDF5 post-processing, all_modules.f90:284-412
  rho0.assign(rho0_in, rho0_in + N);
  p0.assign(pre0_in, pre0_in + N);
  c_speed.assign(cs0_in, cs0_in + N);
  if (magnetic) {
    if (!bx0 || !by0 || !bz0) return "MHD needs bx0, by0, bz0";
    box.assign(bx0, bx0 + N);
    boy.assign(by0, by0 + N);
    boz.assign(bz0, bz0 + N);
  }
  g.assign(grav_in, grav_in + nz);
  zaxis.resize(nz);
  for (int k = 0; k < nz; ++k) zaxis[k] = 1.0 + zaxis_mm[k] * 1.0e8 / RSUN;
  dimc = c_speed[0];
  dimrho = rho0[0];
  diml = RSUN;
  dimb = std::sqrt(4.0 * PI * (dimc * dimc) * dimrho);
  if (P.damping) init_damping();
  cq.resize(nz);
  invrho0q.resize(nz);
  for (int k = 0; k < nz; ++k) {
    cq[k] = c_speed[I(0, 0, k)];
    invrho0q[k] = 2.5440390e-7 / rho0[I(0, 0, k)];
  }
  if (quiet)  // column (1,1,:) replicated, all_modules.f90:353-384
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          p0[I(i, j, k)] = p0[I(0, 0, k)];
          rho0[I(i, j, k)] = rho0[I(0, 0, k)];
          c_speed[I(i, j, k)] = c_speed[I(0, 0, k)];
        }
  src_scale_beta.assign(N, 1.0);
  if (magnetic) {  // all_modules.f90:388-396 (0.01*8.0 in single precision)
    const double k8 = sp(0.01f * 8.0f);
    for (size_t n = 0; n < N; ++n) {
      double b2 = box[n] * box[n] + boy[n] * boy[n] + boz[n] * boz[n];
      double v = k8 * PI * p0[n] / std::max(b2, 1.0e-20);
      src_scale_beta[n] = std::min(v, 1.0);
    }
  }
  for (int k = 0; k < nz; ++k) g[k] = g[k] * diml / (dimc * dimc);
  for (int k = 0; k < nz; ++k) cq[k] = cq[k] / dimc;
  c2.resize(N);
  for (size_t n = 0; n < N; ++n) {
    p0[n] = p0[n] / (dimrho * (dimc * dimc));
    rho0[n] = rho0[n] / dimrho;
    c_speed[n] = c_speed[n] / dimc;
    if (magnetic) {
      box[n] = box[n] / dimb;
      boy[n] = boy[n] / dimb;
      boz[n] = boz[n] / dimb;
    }
    c2[n] = c_speed[n] * c_speed[n];
  }

  init_coeffs();

  // z metric, initialize.f90:674-730
  stretch.resize(nz);
  for (int k = 0; k < nz; ++k) {
    double u;
    if (k < 5) {
      u = 0.0;
      for (int m = 0; m < 11; ++m) u += zaxis[m] * dp[k][m];
      u = u * (nz - 1);
    } else if (k >= nz - 5) {
      int row = nz - 1 - k;
      u = 0.0;
      for (int m = 0; m < 11; ++m) u = u + zaxis[nz - 1 - m] * dp[row][m];
      u = -u * (nz - 1);
    } else {
      u = ((-zaxis[k - 5] + zaxis[k + 5]) * dp[5][10] +
           (-zaxis[k - 4] + zaxis[k + 4]) * dp[5][9] +
           (-zaxis[k - 3] + zaxis[k + 3]) * dp[5][8] +
           (-zaxis[k - 2] + zaxis[k + 2]) * dp[5][7] +
           (-zaxis[k - 1] + zaxis[k + 1]) * dp[5][6]) * (nz - 1);
    }
    stretch[k] = (nz - 1) * 1.0 / u;
  }
  deltat = P.timestep * dimc / diml;  // initialize.f90:733

  // state
  a.assign((size_t)V * N, 0.0);
  temp.assign((size_t)V * N, 0.0);
  scr.assign((size_t)V * N, 0.0);
  forcing.assign(N, 0.0);
  for (auto &v : w) v.assign(N, 0.0);
  if (magnetic)
    for (auto &v : extra) v.assign(N, 0.0);
  if (use_pml) {
    alloc_face(zb, nx, ny, P.npml_zb, P.npml_zb, Pp);
    alloc_face(zt, nx, ny, P.npml_zt, P.npml_zt, Pp);
  }
  if (use_hpml) {
    alloc_face(xb, P.npml_xb, ny, nz, P.npml_xb, Pp);
    alloc_face(xt, P.npml_xt, ny, nz, P.npml_xt, Pp);
    alloc_face(yb, nx, P.npml_yb, nz, P.npml_yb, Pp);
    alloc_face(yt, nx, P.npml_yt, nz, P.npml_yt, Pp);
  }

  // INITIALISE_RHS, initialize.f90:883-1228
  const int bc = periodic ? 5 : 1;
  spongez.assign(nz, 0.0);  // left unset by the reference when USE_PML
  if (!use_pml)
    for (int k = 0; k < nz; ++k)
      spongez[k] = 400.0 / (1.0 + std::exp((1.002 - zaxis[k]) / 0.0001)) +
                   40.0 / (1.0 + std::exp((zaxis[k] - (zaxis[0] + 0.005)) / 0.0005));
  spongexyz.assign(N, 0.0);
  {
    std::vector<double> spx(nx, 0.0), spy(ny, 0.0);
    double s0 = P.sp_length / P.xlength, s1 = 1.0 - P.sp_length / P.xlength;
    if (!periodic && !use_hpml) {
      for (int i = 0; i < nx; ++i)
        spx[i] = P.sp_str * (1.0 - 1.0 / ((1.0 + std::exp((s0 - xaxis[i]) / P.sp_decay)) *
                                          (1.0 + std::exp((xaxis[i] - s1) / P.sp_decay))));
      for (int j = 0; j < ny; ++j)
        spy[j] = P.sp_str * (1.0 - 1.0 / ((1.0 + std::exp((s0 - yaxis[j]) / P.sp_decay)) *
                                          (1.0 + std::exp((yaxis[j] - s1) / P.sp_decay))));
    }
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i)
          spongexyz[I(i, j, k)] = periodic ? spongez[k] : spx[i] + spy[j] + spongez[k];
  }
  if (magnetic) {
    // Alfven limiter, initialize.f90:962-991 (decade search for T)
    reduction.resize(N);
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          size_t n = I(i, j, k);
          reduction[n] = (boz[n] * boz[n] + box[n] * box[n] + boy[n] * boy[n]) /
                         (rho0[n] * (cq[k] * cq[k]));
        }
    double va = 0.0, dtemp = 1.0e9, T = -dtemp;
    double mx = *std::max_element(reduction.begin(), reduction.end());
    if (mx > 0.0) {
      while (dtemp > 1.0e-5 && T < 1.0e10 - 1.1) {
        while (va < P.maxva && T < 1.0e10) {
          T = T + dtemp;
          double m = 0.0;
#pragma omp parallel for reduction(max : m) schedule(static)
          for (size_t n = 0; n < N; ++n) {
            double b2 = box[n] * box[n] + boy[n] * boy[n] + boz[n] * boz[n];
            double v = std::sqrt((dimb * dimb) * T / (T + reduction[n]) * b2 /
                                 (4.0 * PI * dimrho * rho0[n]));
            m = std::max(m, v);
          }
          va = m;
        }
        T = T - dtemp;
        dtemp = dtemp / 10.0;
        va = 0.0;
      }
    } else {
      T = 1.0e10;
    }
    for (size_t n = 0; n < N; ++n) reduction[n] = T / (T + reduction[n]);
    // curl B0, initialize.f90:993-1006
    curlbox.assign(N, 0.0); curlboy.assign(N, 0.0); curlboz.assign(N, 0.0);
    std::vector<double> ct(N, 0.0);
    ddx(boy.data(), curlboz.data(), bc);
    ddy(box.data(), ct.data(), bc);
    for (size_t n = 0; n < N; ++n) curlboz[n] = curlboz[n] - ct[n];
    ddy(boz.data(), ct.data(), bc);
    ddz(boy.data(), curlbox.data(), 1);
    for (size_t n = 0; n < N; ++n) curlbox[n] = ct[n] - curlbox[n];
    ddz(box.data(), curlboy.data(), 1);
    ddx(boz.data(), ct.data(), bc);
    for (size_t n = 0; n < N; ++n) curlboy[n] = curlboy[n] - ct[n];
  }
  rhoinv.resize(N);
  c2rho0.resize(N);
  for (size_t n = 0; n < N; ++n) {  // initialize.f90:1012-1013
    rhoinv[n] = 1.0 / rho0[n];
    c2rho0[n] = c2[n] * rho0[n];
  }
  gradrho0_z.assign(N, 0.0);
  gradp0_z.assign(N, 0.0);
  ddz(rho0.data(), gradrho0_z.data(), 1);
  ddz(p0.data(), gradp0_z.data(), 1);
  if (P.stabilise) {  // initialize.f90:1018-1034 (single-precision bounds)
    const double lo = sp(0.9998f), hi = sp(1.0001f);
    const double add = 1.e-4 * RSUN / (dimrho * (dimc * dimc));
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          size_t n = I(i, j, k);
          double zk = zaxis[k];
          if (zk > lo && zk < 1.0)
            gradp0_z[n] = std::max(c2[n] * gradrho0_z[n] + add, -rho0[n] * g[k]);
          else if (zk <= lo)
            gradp0_z[n] = std::max(c2[n] * gradrho0_z[n], -rho0[n] * g[k]);
          else if (zk >= hi)
            gradp0_z[n] = std::max(c2[n] * gradrho0_z[n], -rho0[n] * g[k]);
        }
  }
  gblk.resize((size_t)P.block_x * P.block_y * nz);
  for (int b = 0; b < P.block_x * P.block_y; ++b)
    for (int k = 0; k < nz; ++k) gblk[(size_t)b * nz + k] = g[k];
  source_damp.assign(N, 0.0);
  init_pml();
  if (magnetic) {  // initialize.f90:1219-1228
    gradrho0_x.assign(N, 0.0); gradrho0_y.assign(N, 0.0);
    gradp0_x.assign(N, 0.0); gradp0_y.assign(N, 0.0);
    ddx(rho0.data(), gradrho0_x.data(), bc);
    ddx(p0.data(), gradp0_x.data(), bc);
    ddy(rho0.data(), gradrho0_y.data(), bc);
    ddy(p0.data(), gradp0_y.data(), bc);
  }
  // INITIALIZE_STEP, initialize.f90:1366-1381
  {
    double o[5] = {1.0, 0.5, 0.1665579725791151184, 0.03950410250586729987,
                   0.007810706393337838236};
    double b5 = o[1];
    double b4 = o[2] / b5;
    double b3 = o[3] / (b5 * b4);
    double b2 = o[4] / (b5 * b4 * b3);
    betas[0] = 0.0 * deltat;
    betas[1] = b2 * deltat;
    betas[2] = b3 * deltat;
    betas[3] = b4 * deltat;
    betas[4] = b5 * deltat;
  }
  src = sparc_source{};
  src.kind = SPARC_SRC_NONE;
  diag = sparc_diag{0.0, 0.0, 0.0, -1, -1};
  return "";
}

// ------------------------------------------------------------------ C API
extern "C" {

orc_handle *orc_create(const sparc_params *p, const double *rho0,
                       const double *pre0, const double *cs0,
                       const double *bx0, const double *by0,
                       const double *bz0, const double *zaxis_mm,
                       const double *grav, char *err, int errlen) {
  orc_handle *h = new orc_handle();
  std::string e = h->setup(p, rho0, pre0, cs0, bx0, by0, bz0, zaxis_mm, grav);
  if (!e.empty()) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.c_str());
    delete h;
    return nullptr;
  }
  return h;
}

void orc_destroy(orc_handle *h) { delete h; }

int orc_set_source(orc_handle *h, const sparc_source *s) {
  if (!s) return SPARC_ERR_INVALID;
  if (s->kind < SPARC_SRC_NONE || s->kind > SPARC_SRC_RANDOM) return SPARC_ERR_INVALID;
  if (s->kind != SPARC_SRC_NONE && s->kind != SPARC_SRC_RANDOM && (s->dir < 1 || s->dir > 3))
    return SPARC_ERR_INVALID;
  if (s->kind == SPARC_SRC_RANDOM && (s->nseries < 1 || !s->series || !(s->cadforcing > 0.0)))
    return SPARC_ERR_INVALID;
  h->src = *s;
  h->pulses.clear();
  h->pulse_in_block.clear();
  h->vr.clear();
  h->source_dep.clear();
  if (s->kind == SPARC_SRC_RANDOM) {
    // driver.f90:80: vr = (randomexciteampl/dimc)*vr
    const double f = s->rnd_ampl / h->dimc;
    const size_t n = (size_t)h->nx * h->ny * s->nseries;
    h->vr.resize(n);
    for (size_t q = 0; q < n; ++q) h->vr[q] = f * s->series[q];
    // e_rad and source_dep (all_modules.f90:289-301)
    const double temp2 = 1.0 + s->rnd_depth / RSUN;
    double temp = 1.0;
    int e_rad = 0;
    for (int k = 0; k < h->nz; ++k)
      if (std::fabs(h->zaxis[k] - temp2) <= temp) {
        temp = std::fabs(h->zaxis[k] - temp2);
        e_rad = k;
      }
    h->source_dep.resize(h->nz);
    const double sg = s->rnd_sigma / RSUN;
    for (int k = 0; k < h->nz; ++k) {
      const double d = h->zaxis[k] - h->zaxis[e_rad];
      h->source_dep[k] = std::exp(-0.5 * (d * d) / 2.0 / (sg * sg));
    }
  }
  h->src.series = nullptr;
  if (s->kind == SPARC_SRC_PSR) {
    if (s->npulses < 0 || (s->npulses > 0 && !s->pulses)) return SPARC_ERR_INVALID;
    h->pulses.assign(s->pulses, s->pulses + s->npulses);
    int nb = h->P.block_x * h->P.block_y * h->P.block_z;
    h->pulse_in_block.assign((size_t)s->npulses * nb, 0);
    for (int n = 0; n < s->npulses; ++n)
      for (int b = 0; b < nb; ++b)
        h->pulse_in_block[(size_t)n * nb + b] = h->psr_in_block(h->pulses[n], b);
  }
  h->src.pulses = nullptr;
  h->forcing_iter = -1;
  return SPARC_OK;
}

int orc_sizes(orc_handle *h, int64_t *ns, int64_t *np) {
  if (ns) *ns = (int64_t)h->a.size();
  int64_t t = 0;
  for (Face *F : h->faces)
    if (F->on) t += (int64_t)F->vars.size();
  if (np) *np = t;
  return SPARC_OK;
}

int orc_set_state(orc_handle *h, const double *a, const double *psi) {
  if (a) std::memcpy(h->a.data(), a, h->a.size() * sizeof(double));
  if (psi) {
    size_t off = 0;
    for (Face *F : h->faces)
      if (F->on) {
        std::memcpy(F->vars.data(), psi + off, F->vars.size() * sizeof(double));
        off += F->vars.size();
      }
  }
  return SPARC_OK;
}

int orc_get_state(orc_handle *h, double *a, double *psi) {
  if (a) std::memcpy(a, h->a.data(), h->a.size() * sizeof(double));
  if (psi) {
    size_t off = 0;
    for (Face *F : h->faces)
      if (F->on) {
        std::memcpy(psi + off, F->vars.data(), F->vars.size() * sizeof(double));
        off += F->vars.size();
      }
  }
  return SPARC_OK;
}

int orc_step(orc_handle *h, int64_t nn) { return h->iterate_step(nn); }

int orc_filter_vars(orc_handle *h, int64_t nn) {
  h->filter_after(nn);
  return SPARC_OK;
}

int orc_run(orc_handle *h, int64_t first, int64_t count) {
  for (int64_t nn = first; nn < first + count; ++nn) {
    h->iterate_step(nn);
    h->filter_after(nn);
  }
  return h->diag.fail_iteration >= 0 ? SPARC_ERR_UNSTABLE : SPARC_OK;
}

int orc_diagnostics(orc_handle *h, sparc_diag *out) {
  *out = h->diag;
  return h->diag.fail_iteration >= 0 ? SPARC_ERR_UNSTABLE : SPARC_OK;
}

int orc_derivative(orc_handle *h, int dir, int bc, const double *in, double *out) {
  if (dir < 0 || dir > 2 || (bc != 1 && bc != 5)) return SPARC_ERR_INVALID;
  h->deriv(dir, in, out, bc);
  return SPARC_OK;
}

int orc_filter_field(orc_handle *h, int dir, const double *in, double *out) {
  if (dir < 0 || dir > 2) return SPARC_ERR_INVALID;
  h->filt(dir, in, out);
  return SPARC_OK;
}

int orc_get_coeff(orc_handle *h, const char *name, double *out, int64_t *count) {
  std::string s(name);
  const std::vector<double> *v = nullptr;
  std::vector<double> tmp;
  if (s == "rho0") v = &h->rho0;
  else if (s == "p0") v = &h->p0;
  else if (s == "c2") v = &h->c2;
  else if (s == "rhoinv") v = &h->rhoinv;
  else if (s == "c2rho0") v = &h->c2rho0;
  else if (s == "gradrho0_z") v = &h->gradrho0_z;
  else if (s == "gradp0_z") v = &h->gradp0_z;
  else if (s == "gradrho0_x") v = &h->gradrho0_x;
  else if (s == "gradrho0_y") v = &h->gradrho0_y;
  else if (s == "gradp0_x") v = &h->gradp0_x;
  else if (s == "gradp0_y") v = &h->gradp0_y;
  else if (s == "spongexyz") v = &h->spongexyz;
  else if (s == "box") v = &h->box;
  else if (s == "boy") v = &h->boy;
  else if (s == "boz") v = &h->boz;
  else if (s == "curlbox") v = &h->curlbox;
  else if (s == "curlboy") v = &h->curlboy;
  else if (s == "curlboz") v = &h->curlboz;
  else if (s == "reduction") v = &h->reduction;
  else if (s == "source_damp") v = &h->source_damp;
  else if (s == "src_scale_beta") v = &h->src_scale_beta;
  else if (s == "stretch") v = &h->stretch;
  else if (s == "zaxis") v = &h->zaxis;
  else if (s == "xaxis") v = &h->xaxis;
  else if (s == "yaxis") v = &h->yaxis;
  else if (s == "g") v = &h->g;
  else if (s == "gblk") v = &h->gblk;
  else if (s == "invrho0q") v = &h->invrho0q;
  else if (s == "cq") v = &h->cq;
  else if (s == "source_dep") v = &h->source_dep;
  else {
    static const char *fn[6] = {"z_bot", "z_top", "x_bot", "x_top", "y_bot", "y_top"};
    for (int f = 0; f < 6; ++f) {
      Face *F = h->faces[f];
      if (s == std::string("a_") + fn[f]) v = &F->a;
      else if (s == std::string("b_") + fn[f]) v = &F->b;
      else if (s == std::string("kappa_") + fn[f]) v = &F->kappa;
    }
  }
  if (!v) return SPARC_ERR_INVALID;
  if (count) *count = (int64_t)v->size();
  if (out) std::memcpy(out, v->data(), v->size() * sizeof(double));
  return SPARC_OK;
}

int orc_get_scalars(orc_handle *h, double *o) {
  double s[12] = {h->dimc, h->dimrho, h->diml, h->dimb, h->deltat, h->stretchx,
                  h->stretchy, h->betas[0], h->betas[1], h->betas[2], h->betas[3],
                  h->betas[4]};
  std::memcpy(o, s, sizeof(s));
  return SPARC_OK;
}

int orc_forcing(orc_handle *h, int64_t nn, double *out) {
  h->forcing_iter = -1;
  h->build_forcing(nn);
  std::memcpy(out, h->forcing.data(), h->N * sizeof(double));
  return SPARC_OK;
}

int orc_rhs(orc_handle *h, int64_t nn, const double *temp, const double *psi,
            double *scr, double *scr_psi) {
  h->build_forcing(nn);
  size_t off = 0;
  for (Face *F : h->faces)
    if (F->on) {
      if (psi) std::memcpy(F->psi.data(), psi + off, F->psi.size() * sizeof(double));
      else std::fill(F->psi.begin(), F->psi.end(), 0.0);
      off += F->psi.size();
    }
  std::vector<double> S((size_t)h->V * h->N);
  h->rhs(temp, S.data());
  std::memcpy(scr, S.data(), S.size() * sizeof(double));
  if (scr_psi) {
    off = 0;
    for (Face *F : h->faces)
      if (F->on) {
        std::memcpy(scr_psi + off, F->scr.data(), F->scr.size() * sizeof(double));
        off += F->scr.size();
      }
  }
  return SPARC_OK;
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
