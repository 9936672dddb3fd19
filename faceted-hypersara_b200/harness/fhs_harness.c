/*
 * fhs_harness -- standalone C driver of the libfhs_b200 C ABI.
 *
 * Plays the part of the reference's imaging/imaging.m for a seeded synthetic
 * problem: reads a JSON configuration in the layout of
 * imaging/default_parameters.json (solver parameters "reweighting", "pdfb",
 * "proj", "noise_estimation"; model parameters "nufft", "preconditioning",
 * "sara"; "aux_global" flags) plus a "harness" section describing the
 * synthetic problem, builds the measurement operator (optionally the
 * preconditioner of imaging.m:436-438 or the visibility-gridding operator of
 * util_load_data_gen_dr_measurement_operator.m), computes the operator norms
 * (imaging.m:701-768), the noise levels and regularisation parameters
 * (compute_noise_level.m:49-89, imaging.m:798-860), runs the solver
 * (imaging.m:896-947) and prints one JSON line with the result.
 *
 *   fhs_harness [config.json] [key=value ...] [--dry-run]
 *
 * key=value pairs override "harness" fields (Ny=256 L=8 algo=hs precond=1
 * dr=1 ...; dr defaults to aux_global.measop_flag_visibility_gridding).
 * --dry-run prints the resolved configuration and exits without touching a
 * GPU.  Exit status: 0 on success, 1 on a configuration error, 2 on a
 * library error (its message is printed).
 *
 * The synthetic problem follows the reference's generators in spirit
 * (util_gen_measurements_snr_new.m, util_gen_sampling_pattern.m): a
 * nonnegative sky of Gaussian blobs and point sources with power-law spectra
 * over 1-2 GHz, Gaussian uv coverage N(0, (pi/4)^2) scaled by nu_l / nu_max,
 * complex Gaussian noise at the requested input SNR, whitened data and
 * chi-square l2 bounds.  Its random numbers are its own (SplitMix64 +
 * Box-Muller), not those of the Python generators.
 */
#include <ctype.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "fhs_b200.h"

static const double kPi = 3.14159265358979323846;

/* ------------------------------------------------------------------ JSON */
typedef enum { J_NULL, J_BOOL, J_NUM, J_STR, J_ARR, J_OBJ } jtype;

typedef struct jnode {
  jtype t;
  double num;
  char* str;              /* J_STR value */
  struct jnode** items;   /* J_ARR / J_OBJ children */
  char** keys;            /* J_OBJ keys */
  int n;
} jnode;

typedef struct {
  const char* s;
  size_t i, len;
  const char* err;
} jparser;

static void jskip(jparser* p) {
  while (p->i < p->len && isspace((unsigned char)p->s[p->i])) ++p->i;
}

static jnode* jnew(jtype t) {
  jnode* n = (jnode*)calloc(1, sizeof(jnode));
  if (n) n->t = t;
  return n;
}

static void jfree(jnode* n) {
  if (!n) return;
  for (int k = 0; k < n->n; ++k) {
    jfree(n->items[k]);
    if (n->keys) free(n->keys[k]);
  }
  free(n->items);
  free(n->keys);
  free(n->str);
  free(n);
}

static jnode* jvalue(jparser* p);

static char* jstring(jparser* p) {
  if (p->s[p->i] != '"') {
    p->err = "expected a string";
    return NULL;
  }
  ++p->i;
  size_t cap = 16, n = 0;
  char* out = (char*)malloc(cap);
  while (p->i < p->len && p->s[p->i] != '"') {
    char c = p->s[p->i++];
    if (c == '\\' && p->i < p->len) {
      char e = p->s[p->i++];
      switch (e) {
        case 'n': c = '\n'; break;
        case 't': c = '\t'; break;
        case 'r': c = '\r'; break;
        case 'b': c = '\b'; break;
        case 'f': c = '\f'; break;
        case 'u': /* keep the escape as '?', the configuration needs no code points */
          p->i += 4;
          c = '?';
          break;
        default: c = e; break;
      }
    }
    if (n + 2 > cap) out = (char*)realloc(out, cap *= 2);
    out[n++] = c;
  }
  if (p->i >= p->len) {
    p->err = "unterminated string";
    free(out);
    return NULL;
  }
  ++p->i;
  out[n] = 0;
  return out;
}

static int jappend(jnode* node, jnode* item, char* key) {
  jnode** it = (jnode**)realloc(node->items, sizeof(jnode*) * (node->n + 1));
  if (!it) return 0;
  node->items = it;
  if (node->t == J_OBJ) {
    char** ks = (char**)realloc(node->keys, sizeof(char*) * (node->n + 1));
    if (!ks) return 0;
    node->keys = ks;
    node->keys[node->n] = key;
  }
  node->items[node->n++] = item;
  return 1;
}

static jnode* jvalue(jparser* p) {
  jskip(p);
  if (p->i >= p->len) {
    p->err = "unexpected end of input";
    return NULL;
  }
  const char c = p->s[p->i];
  if (c == '{' || c == '[') {
    const int obj = c == '{';
    jnode* node = jnew(obj ? J_OBJ : J_ARR);
    ++p->i;
    jskip(p);
    if (p->i < p->len && p->s[p->i] == (obj ? '}' : ']')) {
      ++p->i;
      return node;
    }
    for (;;) {
      char* key = NULL;
      if (obj) {
        jskip(p);
        key = jstring(p);
        if (!key) break;
        jskip(p);
        if (p->i >= p->len || p->s[p->i] != ':') {
          p->err = "expected ':'";
          free(key);
          break;
        }
        ++p->i;
      }
      jnode* v = jvalue(p);
      if (!v || !jappend(node, v, key)) {
        free(key);
        jfree(v);
        break;
      }
      jskip(p);
      if (p->i < p->len && p->s[p->i] == ',') {
        ++p->i;
        continue;
      }
      if (p->i < p->len && p->s[p->i] == (obj ? '}' : ']')) {
        ++p->i;
        return node;
      }
      p->err = obj ? "expected ',' or '}'" : "expected ',' or ']'";
      break;
    }
    jfree(node);
    return NULL;
  }
  if (c == '"') {
    jnode* node = jnew(J_STR);
    node->str = jstring(p);
    if (!node->str) {
      jfree(node);
      return NULL;
    }
    return node;
  }
  if (!strncmp(p->s + p->i, "true", 4) || !strncmp(p->s + p->i, "false", 5)) {
    jnode* node = jnew(J_BOOL);
    node->num = p->s[p->i] == 't';
    p->i += node->num ? 4 : 5;
    return node;
  }
  if (!strncmp(p->s + p->i, "null", 4)) {
    p->i += 4;
    return jnew(J_NULL);
  }
  char* end = NULL;
  const double v = strtod(p->s + p->i, &end);
  if (end == p->s + p->i) {
    p->err = "unexpected character";
    return NULL;
  }
  p->i = (size_t)(end - p->s);
  jnode* node = jnew(J_NUM);
  node->num = v;
  return node;
}

static jnode* jget(const jnode* obj, const char* key) {
  if (!obj || obj->t != J_OBJ) return NULL;
  for (int k = 0; k < obj->n; ++k)
    if (!strcmp(obj->keys[k], key)) return obj->items[k];
  return NULL;
}

/* section.key over the configuration: the root object or every object of a
 * root array (the layout of imaging/default_parameters.json) */
static const jnode* cfg_find(const jnode* root, const char* section, const char* key) {
  if (!root) return NULL;
  if (root->t == J_OBJ) return jget(jget(root, section), key);
  if (root->t == J_ARR)
    for (int k = 0; k < root->n; ++k) {
      const jnode* v = jget(jget(root->items[k], section), key);
      if (v) return v;
    }
  return NULL;
}

static double cfg_num(const jnode* root, const char* section, const char* key, double dflt) {
  const jnode* v = cfg_find(root, section, key);
  return v && (v->t == J_NUM || v->t == J_BOOL) ? v->num : dflt;
}

/* ---------------------------------------------------------------- random */
static uint64_t g_rng;

static uint64_t splitmix64(void) {
  uint64_t z = (g_rng += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

static double urand(void) { return (double)(splitmix64() >> 11) * (1.0 / 9007199254740992.0); }

static double nrand(void) {
  double u1 = urand();
  while (u1 <= 0.0) u1 = urand();
  return sqrt(-2.0 * log(u1)) * cos(2.0 * kPi * urand());
}

/* -------------------------------------------------------------- problem */
typedef struct {
  char algo[8];
  int Ny, Nx, L, Qy, Qx, n_blocks, seed, max_iter, device, precond, dr, opnorm_iter;
  double overlap_fraction, vis_fraction, snr_db;
  char output[512];
} problem_cfg;

static void set_field(problem_cfg* c, const char* key, const char* val) {
  if (!strcmp(key, "algo")) {
    snprintf(c->algo, sizeof c->algo, "%s", val);
  } else if (!strcmp(key, "output")) {
    snprintf(c->output, sizeof c->output, "%s", val);
  } else {
    const double v = atof(val);
    if (!strcmp(key, "Ny")) c->Ny = (int)v;
    else if (!strcmp(key, "Nx")) c->Nx = (int)v;
    else if (!strcmp(key, "L")) c->L = (int)v;
    else if (!strcmp(key, "Qy")) c->Qy = (int)v;
    else if (!strcmp(key, "Qx")) c->Qx = (int)v;
    else if (!strcmp(key, "n_blocks")) c->n_blocks = (int)v;
    else if (!strcmp(key, "seed")) c->seed = (int)v;
    else if (!strcmp(key, "max_iter")) c->max_iter = (int)v;
    else if (!strcmp(key, "device")) c->device = (int)v;
    else if (!strcmp(key, "precond")) c->precond = (int)v;
    else if (!strcmp(key, "dr")) c->dr = (int)v;
    else if (!strcmp(key, "opnorm_iter")) c->opnorm_iter = (int)v;
    else if (!strcmp(key, "overlap_fraction")) c->overlap_fraction = v;
    else if (!strcmp(key, "vis_fraction")) c->vis_fraction = v;
    else if (!strcmp(key, "snr_db")) c->snr_db = v;
    else fprintf(stderr, "fhs_harness: unknown harness field '%s' ignored\n", key);
  }
}

static void load_problem(problem_cfg* c, const jnode* root) {
  memset(c, 0, sizeof *c);
  snprintf(c->algo, sizeof c->algo, "fhs");
  c->Ny = c->Nx = 128;
  c->L = 4;
  c->Qy = c->Qx = 2;
  c->n_blocks = 2;
  c->seed = 1;
  c->max_iter = 200;
  c->opnorm_iter = 200;
  c->overlap_fraction = 0.1;
  c->vis_fraction = 0.5;
  c->snr_db = 40.0;
  c->dr = (int)cfg_num(root, "aux_global", "measop_flag_visibility_gridding", 0);
  /* the "harness" section of any object of the configuration */
  const jnode* secs[8];
  int ns = 0;
  if (root && root->t == J_OBJ) secs[ns++] = jget(root, "harness");
  if (root && root->t == J_ARR)
    for (int k = 0; k < root->n && ns < 8; ++k) secs[ns++] = jget(root->items[k], "harness");
  for (int s = 0; s < ns; ++s) {
    const jnode* h = secs[s];
    if (!h || h->t != J_OBJ) continue;
    for (int k = 0; k < h->n; ++k) {
      char buf[64];
      const jnode* v = h->items[k];
      if (v->t == J_STR) set_field(c, h->keys[k], v->str);
      else if (v->t == J_NUM || v->t == J_BOOL) {
        snprintf(buf, sizeof buf, "%.17g", v->num);
        set_field(c, h->keys[k], buf);
      }
    }
  }
}

/* reference split_range: nearly equal contiguous chunks */
static void split_range(int q, int n, int* s) {
  for (int k = 0; k <= q; ++k) s[k] = (int)floor((double)n * k / q + 0.5);
}

/* one nonnegative image of Gaussian blobs and point sources */
static void sky_image(int Ny, int Nx, double* img) {
  memset(img, 0, sizeof(double) * Ny * Nx);
  for (int b = 0; b < 30; ++b) {
    const double cy = urand() * Ny, cx = urand() * Nx, sg = 2.0 + 10.0 * urand(), a = -log(1.0 - urand());
    const int r = (int)(4 * sg);
    for (int ix = (int)cx - r; ix <= (int)cx + r; ++ix)
      for (int iy = (int)cy - r; iy <= (int)cy + r; ++iy) {
        if (ix < 0 || ix >= Nx || iy < 0 || iy >= Ny) continue;
        const double d2 = (iy - cy) * (iy - cy) + (ix - cx) * (ix - cx);
        img[(size_t)ix * Ny + iy] += a * exp(-d2 / (2 * sg * sg));
      }
  }
  for (int p = 0; p < 200; ++p) {
    const int iy = (int)(urand() * Ny), ix = (int)(urand() * Nx);
    img[(size_t)ix * Ny + iy] += pow(10.0, -3.0 * urand());
  }
}

static int fail(const char* what) {
  fprintf(stderr, "fhs_harness: %s failed: %s\n", what, fhs_last_error());
  return 2;
}

#define CHECK(call)                  \
  do {                               \
    if ((call) != FHS_OK) {          \
      rc = fail(#call);              \
      goto done;                     \
    }                                \
  } while (0)

static double now_s(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec + 1e-9 * t.tv_nsec;
}

int main(int argc, char** argv) {
  const char* cfg_path = NULL;
  int dry = 0;
  for (int a = 1; a < argc; ++a) {
    if (!strcmp(argv[a], "--dry-run")) dry = 1;
    else if (!strcmp(argv[a], "--help") || !strcmp(argv[a], "-h")) {
      printf("usage: fhs_harness [config.json] [key=value ...] [--dry-run]\n");
      return 0;
    } else if (!strchr(argv[a], '=')) cfg_path = argv[a];
  }
  jnode* root = NULL;
  if (cfg_path) {
    FILE* f = fopen(cfg_path, "rb");
    if (!f) {
      fprintf(stderr, "fhs_harness: cannot open %s\n", cfg_path);
      return 1;
    }
    fseek(f, 0, SEEK_END);
    const long len = ftell(f);
    fseek(f, 0, SEEK_SET);
    char* buf = (char*)malloc((size_t)len + 1);
    const size_t got = fread(buf, 1, (size_t)len, f);
    fclose(f);
    buf[got] = 0;
    jparser p = {buf, 0, got, NULL};
    root = jvalue(&p);
    if (!root) {
      fprintf(stderr, "fhs_harness: %s: %s at byte %zu\n", cfg_path, p.err ? p.err : "parse error", p.i);
      free(buf);
      return 1;
    }
    free(buf);
  }
  problem_cfg pc;
  load_problem(&pc, root);
  for (int a = 1; a < argc; ++a) {
    char* eq = strchr(argv[a], '=');
    if (!eq) continue;
    char key[64];
    snprintf(key, sizeof key, "%.*s", (int)(eq - argv[a]), argv[a]);
    set_field(&pc, key, eq + 1);
  }
  const int algo = !strcmp(pc.algo, "sara") ? FHS_ALGO_SARA : !strcmp(pc.algo, "hs") ? FHS_ALGO_HS : FHS_ALGO_FHS;
  if (algo == FHS_ALGO_SARA) pc.L = 1;
  if (algo != FHS_ALGO_FHS) pc.Qy = pc.Qx = 1;
  const int oy = (int)cfg_num(root, "nufft", "oy", 2), ox = (int)cfg_num(root, "nufft", "ox", 2);
  const int J = (int)cfg_num(root, "nufft", "Ky", 7);
  const int nlevel = (int)cfg_num(root, "sara", "nlevel", 4);
  const int sub_pixels = (int)cfg_num(root, "preconditioning", "uniform_weight_sub_pixels", 1);
  const int adjust = (int)cfg_num(root, "aux_global", "adjust_flag_noise", 0);
  const int reweight = (int)cfg_num(root, "aux_global", "reg_flag_reweighting", 1);
  if (pc.Ny <= 0 || pc.Nx <= 0 || pc.L <= 0 || pc.Qy <= 0 || pc.Qx <= 0 || pc.n_blocks <= 0 ||
      pc.n_blocks > 16 || pc.vis_fraction <= 0 || (pc.dr && pc.precond)) {
    fprintf(stderr, "fhs_harness: invalid problem configuration\n");
    jfree(root);
    return 1;
  }
  if (dry) {
    printf("{\"algo\": \"%s\", \"Ny\": %d, \"Nx\": %d, \"L\": %d, \"Qy\": %d, \"Qx\": %d, \"n_blocks\": %d, "
           "\"vis_fraction\": %g, \"snr_db\": %g, \"seed\": %d, \"max_iter\": %d, \"precond\": %d, \"dr\": %d, "
           "\"oy\": %d, \"ox\": %d, \"J\": %d, \"nlevel\": %d, \"reweighting\": %d, \"adjust_flag_noise\": %d, "
           "\"pdfb_max_iter\": %g, \"pdfb_min_iter\": %g, \"reweighting_max_iter\": %g, \"elipse_proj_max_iter\": %g}\n",
           pc.algo, pc.Ny, pc.Nx, pc.L, pc.Qy, pc.Qx, pc.n_blocks, pc.vis_fraction, pc.snr_db, pc.seed,
           pc.max_iter, pc.precond, pc.dr, oy, ox, J, nlevel, reweight, adjust,
           cfg_num(root, "pdfb", "max_iter", 2000), cfg_num(root, "pdfb", "min_iter", 10),
           cfg_num(root, "reweighting", "max_iter", 20), cfg_num(root, "proj", "max_iter", 20));
    jfree(root);
    return 0;
  }

  int rc = 0;
  const int Ny = pc.Ny, Nx = pc.Nx, L = pc.L, Q = pc.Qy * pc.Qx;
  const int64_t N = (int64_t)Ny * Nx, M = (int64_t)(pc.vis_fraction * N);
  if (M < (int64_t)pc.n_blocks) {
    fprintf(stderr, "fhs_harness: vis_fraction gives fewer visibilities than blocks\n");
    jfree(root);
    return 1;
  }
  g_rng = 0x5EEDULL + (uint64_t)pc.seed;
  double *x_true = NULL, *om_y = NULL, *om_x = NULL, *y = NULL, *y0 = NULL, *eps = NULL, *sig = NULL,
         *nu2 = NULL, *xs = NULL, *pu = NULL, *gridv = NULL, *lam = NULL, *noise = NULL;
  double* ydr = NULL;
  int64_t* blocks = NULL;
  int64_t* cells = NULL;
  fhs_measop *op = NULL, *dr = NULL, *use = NULL;
  fhs_solver* solver = NULL;
  double* ydata = NULL;
  int nblk = pc.n_blocks;
  x_true = (double*)malloc(sizeof(double) * N * L);
  om_y = (double*)malloc(sizeof(double) * M * L);
  om_x = (double*)malloc(sizeof(double) * M * L);
  y = (double*)malloc(sizeof(double) * 2 * M * L);
  y0 = (double*)malloc(sizeof(double) * 2 * M * L);
  sig = (double*)malloc(sizeof(double) * L);
  nu2 = (double*)malloc(sizeof(double) * L);
  blocks = (int64_t*)malloc(sizeof(int64_t) * pc.n_blocks);
  if (!x_true || !om_y || !om_x || !y || !y0 || !sig || !nu2 || !blocks) {
    fprintf(stderr, "fhs_harness: host allocation failed\n");
    rc = 2;
    goto done;
  }
  /* sky: reference image with per-pixel power-law spectra over 1-2 GHz */
  {
    double* ref = (double*)malloc(sizeof(double) * N);
    sky_image(Ny, Nx, ref);
    for (int64_t p = 0; p < N; ++p) {
      const double alpha = -0.7 + 0.2 * nrand();
      for (int l = 0; l < L; ++l) {
        const double nu = L > 1 ? 1.0 + (double)l / (L - 1) : 1.0;
        x_true[(size_t)l * N + p] = ref[p] * pow(nu, alpha);
      }
    }
    free(ref);
  }
  /* uv: base coverage N(0, (pi/4)^2) inside [-pi, pi), scaled by nu_l / nu_max */
  for (int64_t m = 0; m < M; ++m) {
    double v, u;
    do v = kPi / 4 * nrand(); while (fabs(v) >= kPi);
    do u = kPi / 4 * nrand(); while (fabs(u) >= kPi);
    for (int l = 0; l < L; ++l) {
      const double s = L > 1 ? (1.0 + (double)l / (L - 1)) / 2.0 : 1.0;
      om_y[(size_t)l * M + m] = v * s;
      om_x[(size_t)l * M + m] = u * s;
    }
  }
  for (int b = 0; b < pc.n_blocks; ++b) blocks[b] = M / pc.n_blocks + (b < M % pc.n_blocks ? 1 : 0);
  /* noiseless data, then whitening by the channel noise level */
  CHECK(fhs_measop_create(pc.device, Ny, Nx, oy, ox, J, J, L, &op));
  for (int l = 0; l < L; ++l)
    CHECK(fhs_measop_set_channel(op, l, M, om_y + (size_t)l * M, om_x + (size_t)l * M, NULL, pc.n_blocks, blocks));
  CHECK(fhs_measop_commit(op));
  CHECK(fhs_forward_operator(op, x_true, y0));
  fhs_measop_destroy(op);
  op = NULL;
  {
    double* w = (double*)malloc(sizeof(double) * M);
    CHECK(fhs_measop_create(pc.device, Ny, Nx, oy, ox, J, J, L, &op));
    for (int l = 0; l < L; ++l) {
      double e2 = 0.0;
      for (int64_t m = 0; m < 2 * M; ++m) e2 += y0[2 * (size_t)l * M + m] * y0[2 * (size_t)l * M + m];
      /* util_gen_measurements_snr_new.m: sigma = 10^(-snr/20) ||y0|| / sqrt(M) */
      sig[l] = pow(10.0, -pc.snr_db / 20.0) * sqrt(e2 / M);
      for (int64_t m = 0; m < M; ++m) {
        w[m] = 1.0 / sig[l];
        for (int c = 0; c < 2; ++c) {
          const size_t i = 2 * ((size_t)l * M + m) + c;
          y[i] = y0[i] / sig[l] + nrand() / sqrt(2.0);
        }
      }
      if (fhs_measop_set_channel(op, l, M, om_y + (size_t)l * M, om_x + (size_t)l * M, w, pc.n_blocks, blocks) !=
          FHS_OK) {
        free(w);
        rc = fail("fhs_measop_set_channel");
        goto done;
      }
    }
    free(w);
    CHECK(fhs_measop_commit(op));
  }
  eps = (double*)malloc(sizeof(double) * L * nblk);
  for (int l = 0; l < L; ++l)
    for (int b = 0; b < nblk; ++b) /* util_gen_data_fidelity_bounds2.m: chi-square bound, whitened */
      eps[l * nblk + b] = sqrt((double)blocks[b] + 2.0 * sqrt((double)blocks[b]));
  if (pc.precond) {
    pu = (double*)malloc(sizeof(double) * M);
    for (int l = 0; l < L; ++l) {
      CHECK(fhs_gen_preconditioning_matrix(M, om_y + (size_t)l * M, om_x + (size_t)l * M, oy * Ny, ox * Nx,
                                           sub_pixels, pu));
      CHECK(fhs_measop_set_preconditioner(op, l, pu));
    }
  }
  use = op;
  ydata = y;
  if (pc.dr) {
    /* util_load_data_gen_dr_measurement_operator.m: H = G'G, gridded data
     * Lambda .* (G'y)(W), l2 bounds from gridded unit-variance noise */
    CHECK(fhs_measop_create_dr(op, &dr));
    const int64_t No = fhs_measop_grid_size(op);
    int64_t ntot = 0;
    for (int l = 0; l < L; ++l) ntot += fhs_measop_n_vis(dr, l);
    ydr = (double*)malloc(sizeof(double) * 2 * (ntot > 0 ? ntot : 1));
    gridv = (double*)malloc(sizeof(double) * 2 * No);
    noise = (double*)malloc(sizeof(double) * 2 * M);
    int64_t pos = 0;
    for (int l = 0; l < L; ++l) {
      const int64_t n = fhs_measop_n_vis(dr, l);
      cells = (int64_t*)realloc(cells, sizeof(int64_t) * (n > 0 ? n : 1));
      lam = (double*)realloc(lam, sizeof(double) * (n > 0 ? n : 1));
      CHECK(fhs_measop_dr_cells(dr, l, cells));
      CHECK(fhs_measop_dr_lambda(dr, l, lam));
      CHECK(fhs_apply_adjoint_operator(op, l, y + 2 * (size_t)l * M, gridv));
      for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < 2; ++c) ydr[2 * (pos + i) + c] = lam[i] * gridv[2 * cells[i] + c];
      for (int64_t m = 0; m < 2 * M; ++m) noise[m] = nrand() / sqrt(2.0);
      CHECK(fhs_apply_adjoint_operator(op, l, noise, gridv));
      double e2 = 0.0;
      for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < 2; ++c) {
          const double v = lam[i] * gridv[2 * cells[i] + c];
          e2 += v * v;
        }
      eps[l] = sqrt(e2);
      pos += n;
    }
    nblk = 1;
    use = dr;
    ydata = ydr;
  }
  if (pc.precond)
    CHECK(fhs_operator_norm_precond(use, pc.opnorm_iter, 1e-6, nu2));
  else
    CHECK(fhs_operator_norm(use, pc.opnorm_iter, 1e-6, nu2));
  {
    /* compute_noise_level.m:49-89 with unit (whitened) noise per channel */
    double ssum = 0.0;
    for (int l = 0; l < L; ++l) ssum += 1.0 / nu2[l];
    const double mu_chi = sqrt(2.0) * exp(lgamma((L + 1) / 2.0) - lgamma(L / 2.0));
    const double sig_chi = sqrt(fmax(L - mu_chi * mu_chi, 0.0));
    double gamma = algo == FHS_ALGO_SARA ? sqrt(1.0 / nu2[0]) : sqrt(ssum / L) * (mu_chi + sig_chi);
    int sy[65], sx[65];
    split_range(pc.Qy, Ny, sy);
    split_range(pc.Qx, Nx, sx);
    const int ovl = algo == FHS_ALGO_FHS
                        ? (int)floor(pc.overlap_fraction * fmin((double)Ny / pc.Qy, (double)Nx / pc.Qx) + 0.5)
                        : 0;
    double* gamma0 = (double*)malloc(sizeof(double) * Q);
    for (int qx = 0; qx < pc.Qx; ++qx)
      for (int qy = 0; qy < pc.Qy; ++qy) {
        const int y0p = qy > 0 ? (sy[qy] - ovl > 0 ? sy[qy] - ovl : 0) : 0;
        const int x0p = qx > 0 ? (sx[qx] - ovl > 0 ? sx[qx] - ovl : 0) : 0;
        const double P = (double)(sy[qy + 1] - y0p) * (double)(sx[qx + 1] - x0p);
        gamma0[qx * pc.Qy + qy] = sqrt(P * ssum / fmin(P, (double)L));
      }
    fhs_solver_config cfg;
    memset(&cfg, 0, sizeof cfg);
    cfg.algo = algo;
    cfg.nlevel = nlevel;
    cfg.n_groups = 1;
    cfg.Qy = pc.Qy;
    cfg.Qx = pc.Qx;
    cfg.splits_y = sy;
    cfg.splits_x = sx;
    cfg.overlap_y = cfg.overlap_x = ovl;
    cfg.window = algo == FHS_ALGO_FHS ? FHS_WINDOW_TRIANGULAR : FHS_WINDOW_NONE;
    if (fhs_solver_create(use, &cfg, &solver) != FHS_OK) {
      free(gamma0);
      rc = fail("fhs_solver_create");
      goto done;
    }
    fhs_solver_params prm;
    memset(&prm, 0, sizeof prm);
    prm.nu0 = prm.nu1 = 1.0;
    prm.nu2 = nu2;
    prm.gamma = &gamma;
    prm.gamma0 = gamma0;
    prm.reweighting_sig = &gamma;
    prm.reweighting_sig_bar = gamma0;
    prm.reweighting_alpha = cfg_num(root, "reweighting", "alpha", 1.0);
    prm.reweighting_flag = reweight;
    prm.reweighting_min_iter = (int)cfg_num(root, "reweighting", "min_iter", 1);
    prm.reweighting_max_iter = (int)cfg_num(root, "reweighting", "max_iter", 20);
    prm.reweighting_rel_var = cfg_num(root, "reweighting", "rel_var", 1e-4);
    prm.pdfb_min_iter = (int)cfg_num(root, "pdfb", "min_iter", 10);
    prm.pdfb_max_iter = (int)cfg_num(root, "pdfb", "max_iter", 2000);
    prm.pdfb_rel_var = cfg_num(root, "pdfb", "rel_var", 5e-5);
    prm.pdfb_fidelity_tolerance = cfg_num(root, "pdfb", "fidelity_tolerance", 1.01);
    prm.pdfb_rel_var_low = cfg_num(root, "pdfb", "rel_var_low", 5e-6);
    prm.elipse_proj_max_iter = (int)cfg_num(root, "proj", "max_iter", 20);
    prm.elipse_proj_min_iter = (int)cfg_num(root, "proj", "min_iter", 1);
    prm.elipse_proj_eps = cfg_num(root, "proj", "eps", 1e-8);
    prm.adjust_flag_noise = adjust;
    prm.adjust_noise_min_iter = (int)cfg_num(root, "noise_estimation", "min_iter", 100);
    prm.adjust_noise_rel_var = cfg_num(root, "noise_estimation", "rel_var", 1e-3);
    prm.adjust_noise_start_iter = (int)cfg_num(root, "noise_estimation", "start_iter", 2000);
    prm.adjust_noise_change_percentage = cfg_num(root, "noise_estimation", "change_percentage", 0.5);
    prm.alph = prm.alph_bar = 1.0;
    const fhs_status st = fhs_solver_set_params(solver, &prm);
    free(gamma0);
    if (st != FHS_OK) {
      rc = fail("fhs_solver_set_params");
      goto done;
    }
  }
  CHECK(fhs_solver_set_data(solver, ydata, eps));
  CHECK(fhs_solver_init(solver, NULL));
  {
    fhs_run_info ri;
    const double t0 = now_s();
    CHECK(fhs_solver_run(solver, pc.max_iter, &ri));
    const double secs = now_s() - t0;
    xs = (double*)malloc(sizeof(double) * N * L);
    CHECK(fhs_solver_get_x(solver, xs));
    double e = 0.0, r = 0.0;
    for (int64_t i = 0; i < N * L; ++i) {
      r += x_true[i] * x_true[i];
      e += (x_true[i] - xs[i]) * (x_true[i] - xs[i]);
    }
    double sara_prior = 0.0, nuc = 0.0;
    CHECK(fhs_compute_sara_prior(pc.device, Ny, Nx, L, nlevel, xs, &sara_prior));
    if (L > 1) CHECK(fhs_nuclear_norm(pc.device, N, L, xs, &nuc));
    printf("{\"algo\": \"%s\", \"Ny\": %d, \"Nx\": %d, \"L\": %d, \"Q\": %d, \"visibilities\": %lld, "
           "\"precond\": %d, \"dr\": %d, \"n_iter\": %d, \"n_reweights\": %d, \"n_noise_adjustments\": %d, "
           "\"converged\": %d, \"seconds\": %.6f, \"iter_per_s\": %.3f, \"snr_db\": %.4f, \"residual\": %.6g, "
           "\"epsilon\": %.6g, \"sara_prior\": %.8g, \"nuclear_norm\": %.8g}\n",
           pc.algo, Ny, Nx, L, Q, (long long)(M * L), pc.precond, pc.dr, ri.n_iter, ri.n_reweights,
           ri.n_noise_adjustments, ri.converged, secs, ri.n_iter / (secs > 0 ? secs : 1e-300),
           10.0 * log10(r / (e > 0 ? e : 1e-300)), ri.residual, ri.epsilon, sara_prior, nuc);
    if (pc.output[0]) {
      FILE* f = fopen(pc.output, "wb");
      if (!f || fwrite(xs, sizeof(double), (size_t)(N * L), f) != (size_t)(N * L)) {
        fprintf(stderr, "fhs_harness: cannot write %s\n", pc.output);
        rc = 1;
      }
      if (f) fclose(f);
    }
  }
done:
  if (solver) fhs_solver_destroy(solver);
  if (dr) fhs_measop_destroy(dr);
  if (op) fhs_measop_destroy(op);
  free(x_true);
  free(om_y);
  free(om_x);
  free(y);
  free(y0);
  free(eps);
  free(sig);
  free(nu2);
  free(xs);
  free(pu);
  free(gridv);
  free(lam);
  free(noise);
  free(blocks);
  free(cells);
  free(ydr);
  jfree(root);
  return rc;
}
