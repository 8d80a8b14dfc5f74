// damping.cu -- DAMPING: the FFT horizontal damping of the velocities
// (all_modules.f90:1803-1888 damp_velocity; rates of initialize.f90:
// 1276-1340 INIT_DAMPING), in the FP64 plain form.
//
// At the end of every RHS evaluation the reference subtracts, from each
// velocity's RHS, the field's damping term (RHS.f90:166-172, 659-665):
// per layer, the unnormalised 2-D real-to-complex transform of v(:,:,k),
// times the real rates damping_rates(kx, ky), transformed back (complex to
// real, unnormalised: the 1/(nx*ny) is folded into the rates).  The MPI
// transposes of the reference only gather whole layers on ranks; the
// result is the per-layer transform.  Here the transforms are cuFFT plans
// batched over the nz layers (library FFTs on the handle's stream,
// capturable in the iteration graph), the rate product is k_damp_mul, and
// the stage kernels read the three terms where the reference subtracts
// them (after the boundary zeroing, so the boundary planes get -term).
#include <cufft.h>

#include <cmath>
#include <vector>

#include "internal.h"

namespace sparc {

// spec(k, j, i) *= rates(j, i) over the half spectrum of nz layers
__global__ void k_damp_mul(double2 *__restrict__ spec, const double *__restrict__ rates,
                           long long nh, long long total) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const double r = __ldg(rates + t % nh);
    double2 c = spec[t];
    c.x = c.x * r;
    c.y = c.y * r;
    spec[t] = c;
  }
}

static bool fft_ok(Handle *h, cufftResult r, const char *what) {
  if (r == CUFFT_SUCCESS) return true;
  h->err = std::string(what) + " failed (cufftResult " + std::to_string((int)r) + ")";
  return false;
}

// The damping rates (initialize.f90:1287-1312, FP64 on the host, in the
// reference's operation order) and the batched plans.  kay2d is the
// horizontal wavenumber in units of 1/Rsun: kx = i (i = 0..nx/2), ky = j
// for j <= ny/2 and ny - j above (the negative frequencies).
int damping_setup(Handle *h) {
  const int nx = h->nx, ny = h->ny, nz = h->nz, nh = nx / 2 + 1;
  const double constx = 2.0 * PI * RSUN / h->P.xlength;
  const double consty = 2.0 * PI * RSUN / h->P.ylength;
  const double kayref = 902.0;
  std::vector<double> rates((size_t)nh * ny);
  for (int j = 0; j < ny; ++j) {
    const double ky = j <= ny / 2 ? (double)j : (double)(ny - j);
    for (int i = 0; i < nh; ++i) {
      const double kay = std::pow(constx * constx * ((double)i * (double)i) +
                                      consty * consty * (ky * ky),
                                  0.5);
      rates[(size_t)j * nh + i] = h->diml / h->dimc / nx / ny * 1.0e-6 *
                                  (500.0 * std::pow(kay / kayref, 2.2)) * 20.0;
    }
  }
  h->d_damp = (double *)dev_alloc(h, rates.size() * 8);
  h->d_spec = (double2 *)dev_alloc(h, (size_t)nh * ny * nz * sizeof(double2));
  h->d_term = (double *)dev_alloc(h, (size_t)3 * h->N * 8);
  if (!h->d_damp || !h->d_spec || !h->d_term) return SPARC_ERR_NOMEM;
  if (cudaMemcpyAsync(h->d_damp, rates.data(), rates.size() * 8, cudaMemcpyHostToDevice,
                      h->stream) != cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess)
    return SPARC_ERR_CUDA;
  int n[2] = {ny, nx}, real_e[2] = {ny, nx}, half_e[2] = {ny, nh};
  if (!fft_ok(h, cufftPlanMany(&h->fft_fwd, 2, n, real_e, 1, nx * ny, half_e, 1, nh * ny,
                               CUFFT_D2Z, nz),
              "cufftPlanMany (forward)") ||
      !fft_ok(h, cufftPlanMany(&h->fft_inv, 2, n, half_e, 1, nh * ny, real_e, 1, nx * ny,
                               CUFFT_Z2D, nz),
              "cufftPlanMany (inverse)"))
    return SPARC_ERR_CUDA;
  h->fft_plans = true;
  return SPARC_OK;
}

// The three damping terms of the velocities of state tin (fields 1..3)
// into h->d_term, on stream s.
int damping_enqueue(Handle *h, const double *tin, cudaStream_t s) {
  const long long nh = (long long)(h->nx / 2 + 1) * h->ny, total = nh * h->nz;
  const unsigned blocks = (unsigned)std::min<long long>((total + 255) / 256, 148LL * 16);
  if (!fft_ok(h, cufftSetStream(h->fft_fwd, s), "cufftSetStream") ||
      !fft_ok(h, cufftSetStream(h->fft_inv, s), "cufftSetStream"))
    return SPARC_ERR_CUDA;
  for (int l = 0; l < 3; ++l) {
    // the forward transform does not write its input (out of place)
    double *in = const_cast<double *>(tin) + (size_t)(l + 1) * h->N;
    if (!fft_ok(h, cufftExecD2Z(h->fft_fwd, in, (cufftDoubleComplex *)h->d_spec),
                "cufftExecD2Z"))
      return SPARC_ERR_CUDA;
    k_damp_mul<<<blocks, 256, 0, s>>>(h->d_spec, h->d_damp, nh, total);
    ++h->launches;
    if (!fft_ok(h, cufftExecZ2D(h->fft_inv, (cufftDoubleComplex *)h->d_spec,
                                h->d_term + (size_t)l * h->N),
                "cufftExecZ2D"))
      return SPARC_ERR_CUDA;
  }
  return cudaGetLastError() == cudaSuccess ? SPARC_OK : SPARC_ERR_CUDA;
}

void damping_destroy(Handle *h) {
  if (!h->fft_plans) return;
  cufftDestroy(h->fft_fwd);
  cufftDestroy(h->fft_inv);
  h->fft_plans = false;
}

}  // namespace sparc
