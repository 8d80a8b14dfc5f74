/*
 * sparc_trol.h -- reader of SPARC's `.trol` parameter file, so a caller of
 * libsparc_gpu.so can start from the same control file as the reference.
 *
 * Replaces READ_SPARC_PARAMETERS (initialize.f90:1385-1924) and the run
 * quantities driver.f90 derives from it (driver.f90:38-39, 64-69).  The
 * rules are the reference's:
 *   - a line is split at its first '='; the name is the text before it with
 *     trailing blanks removed (leading blanks are kept, so an indented key
 *     matches nothing) and cut to 30 characters; names match exactly
 *     (case-sensitive); lines without '=' and unknown names are ignored;
 *   - the value is read list-directed: the first item of the text after the
 *     '=' (blank or comma separated; 'd'/'D' exponents as in 200.0d8;
 *     strings quoted or up to the first blank/comma);
 *   - a value that fails to read ends the file there, as the reference's
 *     iostat does (the rest of the file is not read; stopped_line says where);
 *   - order-sensitive keys: USE_HPML = 0 turns USE_PML on; PERIODIC = 1 is
 *     dropped when USE_HPML is already on; the x/y PML widths are zeroed
 *     unless USE_HPML is already on, the z widths unless USE_PML is; the
 *     pulse_* keys are read only when PULSE (1 or 2) is already set, else
 *     they take 1.0 (pulse_amp 0.0, pulse_dir 1); t_xy and t_z below the
 *     timestep already read become the timestep; wall_time is in hours;
 *   - keys the file does not set keep zero (the reference leaves module
 *     variables uninitialised; filter_mode_* has no default there).
 * Derived: maxtime = floor(solartime*3600/timestep) made even
 * (initialize.f90:1880-1881), the filter and output cadences
 * floor(t/timestep + 1e-5) (initialize.f90:1883-1897), num_steps of the
 * random forcing series as driver.f90:38-39 recomputes it, and the first
 * iteration (driver.f90:64-69: time0*fulloutputsteps + 1 on a restart,
 * else 0).  The driver loop runs iterations init .. maxtime.
 *
 * The reader allocates nothing and touches no device.
 */
#ifndef SPARC_TROL_H
#define SPARC_TROL_H

#include <stdint.h>

#include "sparc_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sparc_trol {
    sparc_params params;  /* the keys the time step reads (precision FP64)   */
    sparc_source source;  /* kind from PULSE; pulse_* or random-source keys;
                             pulses/series NULL: the PSR table and the
                             forcing cube are not in the .trol             */
    int32_t pulse;        /* PULSE as written: 0 random, 1 pulse, 2 PSR      */
    int32_t psr_npulses;  /* pulses the reference draws for PULSE = 2
                             (driver.f90:50-54: 100 in 2-D, else 500)       */
    int32_t restart, time0;
    int32_t twod, twop5d, displ, flows;  /* unsupported when set             */
    int32_t damping;      /* DAMPING as written (also params.damping)        */
    int32_t timestamp_size;
    int32_t xcb, xct, ycb, yct, zcb, zct;         /* chunk output box        */
    int32_t fullout, chunkout;                    /* output enabled          */
    double  solartime;        /* hours of solar time                         */
    double  wall_time;        /* seconds (the file gives hours)              */
    double  fulloutputcad, chunkoutputcad, minsavtime;
    int64_t maxtime;          /* last driver iteration                       */
    int64_t init;             /* first driver iteration                      */
    int64_t xyfreq, zfreq;    /* filter cadences in iterations               */
    int64_t fulloutputsteps, chunkoutputsteps;
    int64_t num_steps;        /* samples of the PULSE = 0 forcing series     */
    int32_t lines_read;       /* lines consumed                              */
    int32_t stopped_line;     /* 0, or the 1-based line whose value failed  */
    char    dir_bkg[200], dir_out[200], simname[240], forcingfunc[200];
} sparc_trol;

/* Reads the .trol file at `path` into *out.  Returns SPARC_OK, or
 * SPARC_ERR_INVALID when the file cannot be opened or a required key is
 * missing (nx, ny, nz, timestep); the message goes to err (errlen bytes,
 * may be NULL). */
int sparc_read_trol(const char *path, sparc_trol *out, char *err, int errlen);

/* The same from the file's text in memory (NUL-terminated). */
int sparc_parse_trol(const char *text, sparc_trol *out, char *err, int errlen);

#ifdef __cplusplus
}
#endif

#endif
