// random_forcing.cuh -- PULSE = 0 forcing plane: LAGRANGE_INTERP
// (all_modules.f90:1892-1950) of the forcing series at one driver
// iteration, times source_damp(:,:,1) (driver.f90:131-132), one value per
// column; the stage kernels add f2d(i,j) * source_dep(k) to RHSv_z
// (RHS.f90:147, 641).  FP64 in the reference's operation order, without
// contraction; samples the reference would read past the end of the series
// count as absent.  Shared by the single-simulation kernel (step.cu) and the
// batched engine (step32.cu).
#pragma once

namespace sparc {

// The seven-point stencil of one iteration: sample times, denominators and
// which samples take part.
struct RndStencil {
  long long time1;
  double xt, x[7], den[7];
  bool use[7];
};

__device__ __forceinline__ RndStencil rnd_stencil(long long nn, double timestep, double cad,
                                                  int ns) {
  RndStencil R;
  double xt = __ddiv_rn(__dmul_rn((double)nn, timestep), cad);
  R.time1 = (long long)floor(xt) + 1;
  R.xt = __dmul_rn((double)nn, timestep);
#pragma unroll
  for (int j = 0; j < 7; ++j) R.x[j] = __dmul_rn((double)(R.time1 - 4 + j), cad);
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    const long long m = R.time1 - 4 + j;
    R.use[j] = (j < 4 ? R.x[j] >= 0.0
                      : (j == 4 ? true : (j == 5 ? R.time1 < ns : R.time1 < ns - 1))) &&
               m >= 0 && m < ns;
    double d = 0.0;
    bool first = true;
#pragma unroll
    for (int q = 0; q < 7; ++q) {
      if (q == j) continue;
      const double e = __dsub_rn(R.x[j], R.x[q]);
      d = first ? e : __dmul_rn(d, e);
      first = false;
    }
    R.den[j] = d;
  }
  return R;
}

// The forcing of column q (series vr: nxy values per sample) times damp.
template <class D>
__device__ __forceinline__ double rnd_column(const RndStencil &R, const double *__restrict__ vr,
                                             int nxy, int q, D damp) {
  double f = 0.0;
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    double t = R.use[j] ? __ddiv_rn(vr[q + (long long)nxy * (R.time1 - 4 + j)], R.den[j]) : 0.0;
#pragma unroll
    for (int m = 0; m < 7; ++m)
      if (m != j) t = __dmul_rn(t, __dsub_rn(R.xt, R.x[m]));
    f = j == 0 ? t : __dadd_rn(f, t);
  }
  return __dmul_rn(f, (double)damp);
}

}  // namespace sparc
