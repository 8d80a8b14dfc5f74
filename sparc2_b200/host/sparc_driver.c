/* sparc_driver.c -- the reference's time loop (driver.f90:123-202) as a C
 * caller of the library: create (INITANDALLOCATE), background
 * (READ_IN_HDF5 + INITIALISE_RHS), source, then per iteration nn the step
 * (driver.f90:157), the norm and fail test (driver.f90:161-183) and
 * FILTER_VARS (driver.f90:200, skipped at nn = 0).
 *
 * The inputs are raw little-endian files in one directory, standing in for
 * the reference's .trol parameters and HDF5 background:
 *   params.bin  one sparc_params            source.bin  one sparc_source
 *   rho0.bin pre0.bin cs0.bin               nx*ny*nz doubles each
 *   bx0.bin by0.bin bz0.bin                 (MAGNETIC = 2 only)
 *   zaxis.bin (Mm) grav.bin (cm/s^2)        nz doubles each
 *   pulses.bin  npulses sparc_pulse         (source.bin kind PULSE = 2)
 *   series.bin  nx*ny*nseries doubles       (source.bin kind PULSE = 0)
 * source.bin is optional; its pointer fields are replaced by the tables.
 * With --trol FILE the parameters and the source come from the reference's
 * .trol control file instead of params.bin and source.bin (sparc_read_trol,
 * READ_SPARC_PARAMETERS); the background files and the PULSE = 2 table /
 * PULSE = 0 series still come from DIR (the .trol names an HDF5 background,
 * a FITS forcing cube and a clock-seeded pulse draw, none of which this
 * caller reads).  FIRST and COUNT may then be "-": the .trol's own run,
 * iterations init .. maxtime (driver.f90:64-69, 123).
 *
 * Output: one line per iteration, "nn ke_norm min_rho min_p status".
 * Exit status: 0 done, 1 bad input, 2 library error, 3 no usable device,
 * 4 the fail criterion was met (the reference dumps and stops there).
 *
 * Build: cc -O2 -I include sparc2_b200/host/sparc_driver.c \
 *           -L sparc2_b200/_lib -lsparc_gpu -Wl,-rpath,sparc2_b200/_lib
 * Run:   sparc_driver DIR FIRST COUNT [DEVICE | --dry-run] [--trol FILE]
 * --dry-run reads and checks the inputs, prints one summary line and exits
 * without touching a device.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "sparc_gpu.h"
#include "sparc_trol.h"

static void *slurp(const char *dir, const char *name, size_t *bytes) {
  char path[4096];
  snprintf(path, sizeof path, "%s/%s", dir, name);
  FILE *f = fopen(path, "rb");
  if (!f) return NULL;
  fseek(f, 0, SEEK_END);
  long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  void *p = n > 0 ? malloc((size_t)n) : NULL;
  if (p && fread(p, 1, (size_t)n, f) != (size_t)n) {
    free(p);
    p = NULL;
  }
  fclose(f);
  if (bytes) *bytes = p ? (size_t)n : 0;
  return p;
}

static double *field(const char *dir, const char *name, size_t count) {
  size_t n = 0;
  double *p = (double *)slurp(dir, name, &n);
  if (p && n != count * sizeof(double)) {
    fprintf(stderr, "%s: %zu bytes, want %zu\n", name, n, count * sizeof(double));
    free(p);
    return NULL;
  }
  return p;
}

int main(int argc, char **argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s DIR FIRST COUNT [DEVICE | --dry-run] [--trol FILE]\n", argv[0]);
    return 1;
  }
  const char *dir = argv[1];
  const char *trol_path = NULL;
  int dry = 0, device = 0;
  for (int q = 4; q < argc; ++q) {
    if (strcmp(argv[q], "--dry-run") == 0) dry = 1;
    else if (strcmp(argv[q], "--trol") == 0 && q + 1 < argc) trol_path = argv[++q];
    else device = atoi(argv[q]);
  }
  size_t n = 0;
  sparc_params *p = NULL;
  sparc_source *src = NULL;
  sparc_trol trol;
  if (trol_path) {
    char err[256];
    if (sparc_read_trol(trol_path, &trol, err, sizeof err) != SPARC_OK) {
      fprintf(stderr, "%s: %s\n", trol_path, err);
      return 1;
    }
    if (trol.stopped_line)
      fprintf(stderr, "%s: reading stopped at line %d (a value failed to read), as the "
              "reference's does\n", trol_path, trol.stopped_line);
    if (trol.twod || trol.displ || trol.flows) {
      fprintf(stderr, "%s: TWOD, MODE = 1 and FLOWS are not supported\n", trol_path);
      return 1;
    }
    p = (sparc_params *)malloc(sizeof *p);
    src = (sparc_source *)malloc(sizeof *src);
    if (!p || !src) return 1;
    *p = trol.params;
    *src = trol.source;
  } else {
    p = (sparc_params *)slurp(dir, "params.bin", &n);
    if (!p || n != sizeof *p) {
      fprintf(stderr, "params.bin: want %zu bytes\n", sizeof *p);
      return 1;
    }
  }
  const int whole = trol_path && (strcmp(argv[2], "-") == 0 || strcmp(argv[3], "-") == 0);
  const long long first = whole ? trol.init : atoll(argv[2]);
  const long long count = whole ? trol.maxtime - trol.init + 1 : atoll(argv[3]);
  const size_t N = (size_t)p->nx * p->ny * p->nz;
  double *rho0 = field(dir, "rho0.bin", N), *pre0 = field(dir, "pre0.bin", N),
         *cs0 = field(dir, "cs0.bin", N), *zaxis = field(dir, "zaxis.bin", p->nz),
         *grav = field(dir, "grav.bin", p->nz);
  double *bx0 = NULL, *by0 = NULL, *bz0 = NULL;
  if (p->magnetic == 2) {
    bx0 = field(dir, "bx0.bin", N);
    by0 = field(dir, "by0.bin", N);
    bz0 = field(dir, "bz0.bin", N);
  }
  if (!rho0 || !pre0 || !cs0 || !zaxis || !grav ||
      (p->magnetic == 2 && (!bx0 || !by0 || !bz0))) {
    fprintf(stderr, "missing background files\n");
    return 1;
  }
  if (!trol_path) {
    src = (sparc_source *)slurp(dir, "source.bin", &n);
    if (src && n != sizeof *src) {
      fprintf(stderr, "source.bin: want %zu bytes\n", sizeof *src);
      return 1;
    }
  }
  sparc_pulse *pulses = NULL;
  double *series = NULL;
  if (src) {
    src->pulses = NULL;
    src->series = NULL;
    if (src->kind == SPARC_SRC_PSR) {
      pulses = (sparc_pulse *)slurp(dir, "pulses.bin", &n);
      if (!pulses || n % sizeof(sparc_pulse) != 0) {
        fprintf(stderr, "pulses.bin: whole sparc_pulse records wanted\n");
        return 1;
      }
      src->npulses = (int32_t)(n / sizeof(sparc_pulse));
      src->pulses = pulses;
    } else if (src->kind == SPARC_SRC_RANDOM) {
      if (src->nseries < 1) {
        fprintf(stderr, "source.bin: nseries must be >= 1\n");
        return 1;
      }
      series = field(dir, "series.bin", (size_t)p->nx * p->ny * (size_t)src->nseries);
      if (!series) {
        fprintf(stderr, "series.bin missing or of the wrong size\n");
        return 1;
      }
      src->series = series;
    } else {
      src->npulses = 0;
    }
  }
  if (dry) {
    double ssum = 0.0;
    if (series)
      for (size_t q = 0; q < (size_t)p->nx * p->ny * (size_t)src->nseries; ++q) ssum += series[q];
    printf("inputs ok: %d x %d x %d, magnetic %d, source %d, pulses %d, series %d (sum %.17g)"
           ", iterations %lld..%lld\n",
           p->nx, p->ny, p->nz, p->magnetic, src ? src->kind : -1,
           src && src->kind == SPARC_SRC_PSR ? src->npulses : 0,
           src && src->kind == SPARC_SRC_RANDOM ? src->nseries : 0, ssum, first,
           first + count - 1);
    return 0;
  }

  sparc_handle *h = NULL;
  int r = sparc_create(p, device, &h);
  if (r != SPARC_OK) {
    fprintf(stderr, "sparc_create: %d (%s)\n", r, sparc_last_error(h));
    return r == SPARC_ERR_NODEVICE ? 3 : 2;
  }
  r = sparc_set_background(h, rho0, pre0, cs0, bx0, by0, bz0, zaxis, grav);
  if (r == SPARC_OK && src) r = sparc_set_source(h, src);
  int status = 0;
  for (long long nn = first; r == SPARC_OK && nn < first + count; ++nn) {
    r = sparc_step(h, nn);
    if (r != SPARC_OK) break;
    sparc_diag d;
    const int rd = sparc_diagnostics(h, &d);
    printf("%lld %.17g %.17g %.17g %d\n", nn, d.ke_norm, d.min_rho, d.min_p, rd);
    if (rd == SPARC_ERR_UNSTABLE) {
      status = 4;
      break;
    }
    if (rd != SPARC_OK) {
      r = rd;
      break;
    }
    if (nn != 0) r = sparc_filter_vars(h, nn);
  }
  if (r != SPARC_OK) {
    fprintf(stderr, "library error %d (%s)\n", r, sparc_last_error(h));
    status = 2;
  }
  sparc_destroy(h);
  free(p);
  free(src);
  free(pulses);
  free(series);
  free(rho0); free(pre0); free(cs0); free(zaxis); free(grav);
  free(bx0); free(by0); free(bz0);
  return status;
}
