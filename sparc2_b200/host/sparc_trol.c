/* sparc_trol.c -- the .trol parameter-file reader of include/sparc_trol.h,
 * a restatement of READ_SPARC_PARAMETERS (initialize.f90:1385-1924) and of
 * the run quantities driver.f90:38-39 and 64-69 derive from it.  Host C
 * only; compiled into libsparc_gpu.so beside the device code. */
#include <ctype.h>
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "sparc_trol.h"

#define LINE_MAX_CHARS 200 /* CHARACTER(LEN=200) :: linebuffer */
#define NAME_MAX_CHARS 30  /* CHARACTER(LEN=30)  :: linename   */

static void set_err(char *err, int errlen, const char *msg) {
  if (err && errlen > 0) {
    strncpy(err, msg, (size_t)errlen - 1);
    err[errlen - 1] = '\0';
  }
}

/* ------------------------------------------- list-directed value reading
 * A cursor over the value text.  next_item() yields the next item of a
 * list-directed record: items are separated by a comma or blanks (a comma
 * between blanks is one separator); an empty item between two commas is a
 * null value (the variable keeps its value); '/' ends the list. */
typedef struct {
  const char *p;
  int ended; /* a '/' was met */
} cursor;

/* 1: item in buf; 0: null value; -1: end of record (the read fails) */
static int next_item(cursor *c, char *buf, size_t cap, int want_string) {
  if (c->ended) return 0;
  while (*c->p == ' ' || *c->p == '\t') ++c->p;
  if (*c->p == '\0') return -1;
  if (*c->p == '/') {
    c->ended = 1;
    return 0;
  }
  if (*c->p == ',') {  /* null value */
    ++c->p;
    return 0;
  }
  size_t n = 0;
  if (want_string && (*c->p == '"' || *c->p == '\'')) {
    const char q = *c->p++;
    for (;;) {
      if (*c->p == '\0') break; /* unterminated: the rest of the line */
      if (*c->p == q) {
        if (c->p[1] == q) { /* doubled quote: a literal quote */
          if (n + 1 < cap) buf[n++] = q;
          c->p += 2;
          continue;
        }
        ++c->p;
        break;
      }
      if (n + 1 < cap) buf[n++] = *c->p;
      ++c->p;
    }
  } else {
    while (*c->p && *c->p != ' ' && *c->p != '\t' && *c->p != ',' && *c->p != '/') {
      if (n + 1 < cap) buf[n++] = *c->p;
      ++c->p;
    }
  }
  buf[n] = '\0';
  /* the separator after the item */
  while (*c->p == ' ' || *c->p == '\t') ++c->p;
  if (*c->p == ',') ++c->p;
  return 1;
}

static int parse_real(const char *s, double *v) {
  char t[96];
  size_t n = strlen(s);
  if (n == 0 || n >= sizeof t) return 0;
  for (size_t i = 0; i <= n; ++i) t[i] = (s[i] == 'd' || s[i] == 'D') ? 'e' : s[i];
  char *end = NULL;
  errno = 0;
  const double x = strtod(t, &end);
  if (end == t || *end != '\0' || errno == ERANGE) return 0;
  *v = x;
  return 1;
}

static int parse_int(const char *s, long long *v) {
  const char *p = s;
  if (*p == '+' || *p == '-') ++p;
  if (!isdigit((unsigned char)*p)) return 0;
  for (const char *q = p; *q; ++q)
    if (!isdigit((unsigned char)*q)) return 0;
  *v = strtoll(s, NULL, 10);
  return 1;
}

/* Reads one item of the given kind; 1 ok (or null: unchanged), 0 failed */
static int read_real(cursor *c, double *v) {
  char b[96];
  const int r = next_item(c, b, sizeof b, 0);
  if (r < 0) return 0;
  return r == 0 ? 1 : parse_real(b, v);
}
static int read_int(cursor *c, long long *v) {
  char b[96];
  const int r = next_item(c, b, sizeof b, 0);
  if (r < 0) return 0;
  return r == 0 ? 1 : parse_int(b, v);
}
static int read_str(cursor *c, char *dst, size_t cap) {
  char b[LINE_MAX_CHARS + 1];
  const int r = next_item(c, b, sizeof b, 1);
  if (r < 0) return 0;
  if (r == 1) {
    strncpy(dst, b, cap - 1);
    dst[cap - 1] = '\0';
  }
  return 1;
}

/* ---------------------------------------------------------------- parse */
typedef struct {
  /* the reference's module variables the keys set (zero = unset) */
  long long nx, ny, nz, time0, xcb, xct, ycb, yct, zcb, zct, timestamp_size;
  long long nxb, nxt, nyb, nyt, nzb, nzt, pulse_dir, twop5d, blk[3];
  double xlength, ylength, timestep, wall_time, solartime, chunkoutputcad,
      fulloutputcad, minsavtime, maxva, sp_str, sp_length, sp_decay, cadforcing,
      rdepth, rsigma, rampl, t0, t1, st, px, py, pz, sr, sz, amp, s_xy, s_z, t_xy,
      t_z;
  double xpb[4], xpt[4], ypb[4], ypt[4], zpb[4], zpt[4];
  int restart, stabilise, damping, displ, flows, pulse, psr, gxy, gz, magnetic,
      quiet, twod, use_pml, use_hpml, periodic, pulse_kind;
  char dir_out[200], dir_bkg[200], simname[240], forcingfunc[200];
} vars;

/* 1: read (or not a key), 0: the value failed to read */
static int apply(vars *v, const char *name, const char *value) {
  cursor c = {value, 0};
  long long sw = 0;
#define KEY(s) (strcmp(name, s) == 0)
#define RI(x) read_int(&c, &(x))
#define RR(x) read_real(&c, &(x))
  if (KEY("dir_out")) return read_str(&c, v->dir_out, sizeof v->dir_out);
  if (KEY("dir_bkg")) return read_str(&c, v->dir_bkg, sizeof v->dir_bkg);
  if (KEY("simname")) return read_str(&c, v->simname, sizeof v->simname);
  if (KEY("forcingfunc")) return read_str(&c, v->forcingfunc, sizeof v->forcingfunc);
  if (KEY("nx")) return RI(v->nx);
  if (KEY("ny")) return RI(v->ny);
  if (KEY("nz")) return RI(v->nz);
  if (KEY("xlength")) return RR(v->xlength);
  if (KEY("ylength")) return RR(v->ylength);
  if (KEY("restart")) {
    if (!RI(sw)) return 0;
    v->restart = sw != 0;
    return 1;
  }
  if (KEY("time0")) return RI(v->time0);
  if (KEY("timestep")) return RR(v->timestep);
  if (KEY("wall_time")) {
    if (!RR(v->wall_time)) return 0;
    v->wall_time = v->wall_time * 3600;
    return 1;
  }
  if (KEY("solartime")) return RR(v->solartime);
  if (KEY("chunkoutputcad")) return RR(v->chunkoutputcad);
  if (KEY("xcb")) return RI(v->xcb);
  if (KEY("xct")) return RI(v->xct);
  if (KEY("ycb")) return RI(v->ycb);
  if (KEY("yct")) return RI(v->yct);
  if (KEY("zcb")) return RI(v->zcb);
  if (KEY("zct")) return RI(v->zct);
  if (KEY("fulloutputcad")) return RR(v->fulloutputcad);
  if (KEY("minsavtime")) return RR(v->minsavtime);
  if (KEY("timestamp_size")) return RI(v->timestamp_size);
  if (KEY("STABILISE") || KEY("DAMPING") || KEY("MODE") || KEY("FLOWS") || KEY("TWOD") ||
      KEY("USE_PML")) {
    if (!RI(sw)) return 0;
    int *dst = KEY("STABILISE") ? &v->stabilise
               : KEY("DAMPING") ? &v->damping
               : KEY("MODE")    ? &v->displ
               : KEY("FLOWS")   ? &v->flows
               : KEY("TWOD")    ? &v->twod
                                : &v->use_pml;
    *dst = sw != 0;
    return 1;
  }
  if (KEY("PULSE")) {
    if (!RI(sw)) return 0;
    v->pulse = sw != 0;
    if (sw == 2) v->psr = 1;
    v->pulse_kind = (int)sw;
    return 1;
  }
  if (KEY("filter_mode_xy") || KEY("filter_mode_z")) {
    if (!RI(sw)) return 0;
    int *g = KEY("filter_mode_xy") ? &v->gxy : &v->gz;
    if (sw == 1) *g = 5;
    else if (sw == 2) *g = 3;
    return 1;
  }
  if (KEY("MAGNETIC")) {
    if (!RI(sw)) return 0;
    if (sw == 0) { v->magnetic = 0; v->quiet = 1; }
    else if (sw == 1) { v->magnetic = 0; v->quiet = 0; }
    else if (sw == 2) { v->magnetic = 1; v->quiet = 0; }
    return 1;
  }
  if (KEY("maxva")) return RR(v->maxva);
  if (KEY("TWOP5D")) return RI(v->twop5d);
  if (KEY("USE_HPML")) {
    if (!RI(sw)) return 0;
    if (sw == 0) {
      v->use_pml = 1; /* HPMLs need USE_PML; the reference turns it on */
      v->use_hpml = 0;
    } else {
      v->use_hpml = 1;
    }
    return 1;
  }
  if (KEY("PERIODIC")) {
    if (!RI(sw)) return 0;
    v->periodic = sw == 0 ? 0 : (v->use_hpml ? 0 : 1);
    return 1;
  }
  {
    static const char *pk[6] = {"xpmlt", "xpmlb", "ypmlt", "ypmlb", "zpmlt", "zpmlb"};
    for (int f = 0; f < 6; ++f) {
      if (!KEY(pk[f])) continue;
      long long *np = f == 0 ? &v->nxt : f == 1 ? &v->nxb : f == 2 ? &v->nyt
                    : f == 3 ? &v->nyb : f == 4 ? &v->nzt : &v->nzb;
      double *pp = f == 0 ? v->xpt : f == 1 ? v->xpb : f == 2 ? v->ypt
                 : f == 3 ? v->ypb : f == 4 ? v->zpt : v->zpb;
      if (!RI(*np)) return 0;
      for (int q = 0; q < 4; ++q)
        if (!RR(pp[q])) return 0;
      if (f < 4 ? !v->use_hpml : !v->use_pml) *np = 0;
      return 1;
    }
  }
  if (KEY("sp_str")) return RR(v->sp_str);
  if (KEY("sp_length")) return RR(v->sp_length);
  if (KEY("sp_decay")) return RR(v->sp_decay);
  if (KEY("cadforcing")) return RR(v->cadforcing);
  if (KEY("randomexcitedepth")) return RR(v->rdepth);
  if (KEY("randomexcitesigma")) return RR(v->rsigma);
  if (KEY("randomexciteampl")) return RR(v->rampl);
  if (KEY("pulse_dir")) {
    if (v->pulse) return RI(v->pulse_dir);
    v->pulse_dir = 1;
    return 1;
  }
  {
    static const char *pk[8] = {"pulse_t0", "pulse_t1", "pulse_st", "pulse_px",
                                "pulse_py", "pulse_pz", "pulse_sr", "pulse_sz"};
    double *dst[8] = {&v->t0, &v->t1, &v->st, &v->px, &v->py, &v->pz, &v->sr, &v->sz};
    for (int q = 0; q < 8; ++q) {
      if (!KEY(pk[q])) continue;
      if (v->pulse) return RR(*dst[q]);
      *dst[q] = 1.0;
      return 1;
    }
  }
  if (KEY("pulse_amp")) {
    if (v->pulse) return RR(v->amp);
    v->amp = 0.0;
    return 1;
  }
  if (KEY("s_xy")) return RR(v->s_xy);
  if (KEY("s_z")) return RR(v->s_z);
  if (KEY("t_xy") || KEY("t_z")) {
    double *t = KEY("t_xy") ? &v->t_xy : &v->t_z;
    if (!RR(*t)) return 0;
    if (*t < v->timestep) *t = v->timestep;
    return 1;
  }
  if (KEY("block_x")) return RI(v->blk[0]);
  if (KEY("block_y")) return RI(v->blk[1]);
  if (KEY("block_z")) return RI(v->blk[2]);
  return 1; /* unknown name: ignored */
#undef KEY
#undef RI
#undef RR
}

static void finish(const vars *v, sparc_trol *o) {
  sparc_params *p = &o->params;
  memset(o, 0, sizeof *o);
  long long nx = v->nx, ny = v->ny, nz = v->nz;
  long long nyb = v->nyb, nyt = v->nyt;
  double ylength = v->ylength, py = v->py;
  if (v->twod) { /* initialize.f90:1791-1797, 1830-1836 */
    ylength = 0.0;
    ny = 1;
    nyb = nyt = 0;
    py = 0.0;
  }
  p->nx = (int32_t)nx;
  p->ny = (int32_t)ny;
  p->nz = (int32_t)nz;
  p->magnetic = v->magnetic ? 2 : (v->quiet ? 0 : 1);
  p->periodic = v->periodic;
  p->use_pml = v->use_pml;
  p->use_hpml = v->use_hpml;
  p->stabilise = v->stabilise;
  p->filter_mode_xy = v->gxy == 5 ? 1 : (v->gxy == 3 ? 2 : 0);
  p->filter_mode_z = v->gz == 5 ? 1 : (v->gz == 3 ? 2 : 0);
  p->block_x = (int32_t)v->blk[0];
  p->block_y = (int32_t)v->blk[1];
  p->block_z = (int32_t)v->blk[2];
  p->npml_xb = (int32_t)v->nxb;
  p->npml_xt = (int32_t)v->nxt;
  p->npml_yb = (int32_t)nyb;
  p->npml_yt = (int32_t)nyt;
  p->npml_zb = (int32_t)v->nzb;
  p->npml_zt = (int32_t)v->nzt;
  memcpy(p->pml_xb, v->xpb, sizeof p->pml_xb);
  memcpy(p->pml_xt, v->xpt, sizeof p->pml_xt);
  memcpy(p->pml_yb, v->ypb, sizeof p->pml_yb);
  memcpy(p->pml_yt, v->ypt, sizeof p->pml_yt);
  memcpy(p->pml_zb, v->zpb, sizeof p->pml_zb);
  memcpy(p->pml_zt, v->zpt, sizeof p->pml_zt);
  p->xlength = v->xlength;
  p->ylength = ylength;
  p->timestep = v->timestep;
  p->s_xy = v->s_xy;
  p->s_z = v->s_z;
  p->t_xy = v->t_xy;
  p->t_z = v->t_z;
  p->maxva = v->maxva;
  p->sp_str = v->sp_str;
  p->sp_length = v->sp_length;
  p->sp_decay = v->sp_decay;
  p->precision = SPARC_FP64;

  /* initialize.f90:1880-1900 */
  const double ts = v->timestep;
  long long maxtime = ts > 0 ? (long long)floor(v->solartime * 3600.0 / ts) : 0;
  maxtime = 2 * (maxtime / 2);
  long long full = ts > 0 ? (long long)floor(v->fulloutputcad / ts + 1.0e-5) : 0;
  long long chunk = ts > 0 ? (long long)floor(v->chunkoutputcad / ts + 1.0e-5) : 0;
  o->fullout = o->chunkout = 1;
  if (chunk == 0) { o->chunkout = 0; chunk = 1; }
  if (full == 0) { o->fullout = 0; full = 1; }
  o->maxtime = maxtime;
  o->fulloutputsteps = full;
  o->chunkoutputsteps = chunk;
  o->xyfreq = ts > 0 ? (long long)floor(v->t_xy / ts + 1.0e-5) : 0;
  o->zfreq = ts > 0 ? (long long)floor(v->t_z / ts + 1.0e-5) : 0;
  /* driver.f90:38-39 (the value the run uses) */
  long long ns = v->cadforcing > 0 ? (long long)floor((double)maxtime * ts / v->cadforcing) + 2 : 2;
  o->num_steps = 2 * (ns / 2) + 2;
  /* driver.f90:64-69 */
  o->init = v->restart ? v->time0 * full + 1 : 0;

  o->pulse = v->pulse_kind;
  o->psr_npulses = v->twod ? 100 : 500;
  o->restart = v->restart;
  o->time0 = (int32_t)v->time0;
  o->twod = v->twod;
  o->twop5d = (int32_t)v->twop5d;
  o->displ = v->displ;
  o->flows = v->flows;
  o->damping = v->damping;
  o->params.damping = v->damping ? 1 : 0;
  o->timestamp_size = (int32_t)v->timestamp_size;
  o->xcb = (int32_t)v->xcb; o->xct = (int32_t)v->xct;
  o->ycb = (int32_t)v->ycb; o->yct = (int32_t)v->yct;
  o->zcb = (int32_t)v->zcb; o->zct = (int32_t)v->zct;
  o->solartime = v->solartime;
  o->wall_time = v->wall_time;
  o->fulloutputcad = v->fulloutputcad;
  o->chunkoutputcad = v->chunkoutputcad;
  o->minsavtime = v->minsavtime;
  snprintf(o->dir_bkg, sizeof o->dir_bkg, "%s", v->dir_bkg);
  snprintf(o->dir_out, sizeof o->dir_out, "%s", v->dir_out);
  snprintf(o->forcingfunc, sizeof o->forcingfunc, "%s", v->forcingfunc);
  /* simname suffixes, initialize.f90:1799-1824 */
  char sfx[16];
  snprintf(sfx, sizeof sfx, "%s%s%s%s_", v->twod ? "_2D" : "_3D", v->displ ? "_d" : "_v",
           v->magnetic ? "m" : (v->quiet ? "q" : "t"), v->flows ? "f" : "");
  size_t n = strlen(v->simname);
  while (n > 0 && v->simname[n - 1] == ' ') --n;
  snprintf(o->simname, sizeof o->simname, "%.*s%s", (int)n, v->simname, sfx);

  /* the source the driver loop uses (driver.f90:130-155) */
  sparc_source *s = &o->source;
  s->init = o->init;
  s->dir = (int32_t)v->pulse_dir;
  if (!v->pulse) {
    s->kind = SPARC_SRC_RANDOM;
    s->dir = 3;
    s->cadforcing = v->cadforcing;
    s->rnd_ampl = v->rampl;
    s->rnd_depth = v->rdepth;
    s->rnd_sigma = v->rsigma;
    s->nseries = (int32_t)o->num_steps;
  } else if (v->psr) {
    s->kind = SPARC_SRC_PSR;
    s->psr_st = 120.0; /* all_modules.f90:590 */
  } else {
    s->kind = SPARC_SRC_PULSE;
    s->amp = v->amp;
    s->t0 = v->t0;
    s->t1 = v->t1;
    s->st = v->st;
    s->px = v->px;
    s->py = py;
    s->pz = v->pz;
    s->sr = v->sr;
    s->sz = v->sz;
  }
}

int sparc_parse_trol(const char *text, sparc_trol *out, char *err, int errlen) {
  if (!text || !out) {
    set_err(err, errlen, "null argument");
    return SPARC_ERR_INVALID;
  }
  vars v;
  memset(&v, 0, sizeof v);
  int lines = 0, stopped = 0;
  const char *p = text;
  while (*p) {
    /* one record, cut to the 200-character buffer */
    const char *e = strchr(p, '\n');
    const size_t len = e ? (size_t)(e - p) : strlen(p);
    char line[LINE_MAX_CHARS + 1];
    size_t n = len < LINE_MAX_CHARS ? len : LINE_MAX_CHARS;
    memcpy(line, p, n);
    line[n] = '\0';
    if (n > 0 && line[n - 1] == '\r') line[--n] = '\0';
    ++lines;
    p = e ? e + 1 : p + len;
    char *eq = strchr(line, '=');
    if (!eq) continue;
    /* name: text before the first '=', trailing blanks removed, 30 chars */
    size_t m = (size_t)(eq - line);
    while (m > 0 && line[m - 1] == ' ') --m;
    if (m > NAME_MAX_CHARS) m = NAME_MAX_CHARS;
    char name[NAME_MAX_CHARS + 1];
    memcpy(name, line, m);
    name[m] = '\0';
    /* a 30-character cut may leave trailing blanks, which compare equal */
    while (m > 0 && name[m - 1] == ' ') name[--m] = '\0';
    if (!apply(&v, name, eq + 1)) {
      stopped = lines; /* the reference's iostat ends the read loop here */
      break;
    }
  }
  finish(&v, out);
  out->lines_read = lines;
  out->stopped_line = stopped;
  if (v.nx <= 0 || v.nz <= 0 || (v.ny <= 0 && !v.twod) || !(v.timestep > 0)) {
    set_err(err, errlen,
            stopped ? "a value failed to read before nx, ny, nz and timestep were all set"
                    : "nx, ny, nz and timestep must be set");
    return SPARC_ERR_INVALID;
  }
  set_err(err, errlen, "");
  return SPARC_OK;
}

int sparc_read_trol(const char *path, sparc_trol *out, char *err, int errlen) {
  if (!path || !out) {
    set_err(err, errlen, "null argument");
    return SPARC_ERR_INVALID;
  }
  FILE *f = fopen(path, "rb");
  if (!f) {
    set_err(err, errlen, "cannot open the parameter file");
    return SPARC_ERR_INVALID;
  }
  fseek(f, 0, SEEK_END);
  const long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  if (n < 0 || n > (1L << 24)) {
    fclose(f);
    set_err(err, errlen, "parameter file too large");
    return SPARC_ERR_INVALID;
  }
  char *text = (char *)malloc((size_t)n + 1);
  if (!text) {
    fclose(f);
    set_err(err, errlen, "out of host memory");
    return SPARC_ERR_NOMEM;
  }
  const size_t got = fread(text, 1, (size_t)n, f);
  fclose(f);
  text[got] = '\0';
  const int r = sparc_parse_trol(text, out, err, errlen);
  free(text);
  return r;
}
