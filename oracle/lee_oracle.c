/*
 * lee_oracle.c -- CPU restatement of the camille reference's LEE time-advance
 * path, in plain C. TEST INFRASTRUCTURE ONLY: the parity tests, smoke() and
 * bench.py's CPU-baseline leg load it as the checker; the product never links,
 * loads or calls it.
 *
 * It exports the ABI of include/lee_b200.h with the prefix orc_ instead of lee_,
 * so a test drives the oracle and the CUDA library with identical calls. Every
 * function follows the reference's arithmetic step by step, in the reference's
 * order of summation, so that on one rank it reproduces the reference to the
 * last bits or close to them. It is pinned against the compiled reference
 * (oracle/_ref/camille_ref) by tests/test_oracle_pin.py.
 *
 * Citations are files of the camille reference, relative to its root.
 */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/lee_b200.h"

/* The point loops of the time advance run on all host threads (OpenMP): every point, and
 * every line of a directional pass, is computed by the same operations in the same order
 * whichever thread takes it, so the results are the same bits as a serial run. */
#define PAR_FOR _Pragma("omp parallel for schedule(static)")

#define NOTBLANKED 0
#define BLANKED 1
#define INTERPOLATED (-1)
#define MAXB 8
#define MAXBND 64
#define MAXSC 8          /* passive scalars (PHYSICAL_MODEL = LEE_SCALAR) */
#define MAXV (5 + MAXSC) /* state slots: s', u', v', w', p', then the scalars Z_k' */

/* One directional operator: interior stencil c[l+h] for l = -h..h, boundary rows
 * B[row][s] for row < nb, s < S, and the right-boundary sign (-1 for the
 * antisymmetric difference, +1 for the symmetric filter), as the classes of
 * src/solver/spatial_discretization.h:49-132 hold them. */
typedef struct {
  int h, nb, S;
  double c[11];
  double B[5][9];
  double mfac;
} op_t;

typedef struct {
  int kind, dir, end, lo[3], hi[3];
  double *sigma; /* sponge strengths over the box, i fastest */
} bnd_t;

typedef struct {
  int set, nx, ny, nz, N;
  double *xyz[3];
  int *iblank;
  double *met[9];  /* metrics[l][i] at l*3+i */
  double *minv[9]; /* metricsInverse[i][l] at i*3+l */
  double *jac, *invjac;
  double *mean[MAXV];
  double *grad[3 * MAXV]; /* d mean_v / dx_j at v*ndim + j */
  double *aux[4];   /* rho', rho_bar, T', T_bar (IAUX_*, src/core/param.h:77-80) */
  double *sol[MAXV];
  int nbnd;
  bnd_t bnd[MAXBND];
} blk_t;

/* Overset donor maps as overset::initialize_donor / initialize_receiver hold them
 * (src/overset/overset.cpp:88-554): per receiver its block and linear index, the donor
 * block and the linear index of the stencil's lower-left corner, and the weights
 * normalised by their sum (:516-526), zeta outermost, xi innermost. */
typedef struct {
  int n;
  int *rb, *db;
  long long *rl, *dl;
  int w[3], W;
  double *wt;
  double *buf; /* n x MAXV interpolants */
} ovs_t;

struct orc_ctx {
  lee_config cfg;
  op_t fd, flt;
  int nsc, nv; /* passive scalars (UserInput::num_scalar, src/core/input.cpp:113-119) and state slots */
  int nblk;
  blk_t blk[MAXB];
  int src_kind;
  double src[7];
  int bsrc_mode[MAXB];     /* per block: 0 the context's source, 1 its own monopole, 2 none */
  double bsrc[MAXB][7];
  double *dsrc;  /* distributed source parameters */
  int ndsrc;
  double *dsrc_g; /* its prolonged field on block dsrc[0] (full grid, zero outside the lattice) */
  int mic_block, nmic; /* objective: p' at microphones */
  long long *mic;
  double mic_weight;
  int prepared, step;
  double time;
  ovs_t ovs;
  /* time-harmonic wave (UserInput::harmonicWave_*, src/core/input.cpp:219-231) */
  int wave_type, wave_form, wave_dir;
  double wave_amp, wave_len, wave_hw;
  int axisym; /* UserInput::axisym (src/core/input.cpp:105-108) */
  double *scr[3]; /* work fields of the right-hand side, scrn points each */
  int finite_every; /* steps between non-finite checks (0: end of each advance, -1: none) */
  size_t scrn;
  char err[512];
};
typedef struct orc_ctx orc_ctx;

static char g_err[512];

static int fail(orc_ctx *c, int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(c ? c->err : g_err, 512, fmt, ap);
  va_end(ap);
  return code;
}

static double *dalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

/* ---------------------------------------------------------------------------
 * Coefficient tables: StandardCentral::initialize (:28-109), StandardCentralFilter
 * ::initialize (:113-224), OptimizedCentralExplicit::initialize (:228-344),
 * OptimizedCentralFilterExplicit::initialize (:348-492) of
 * src/solver/spatial_discretization.cpp. The numbers are the published tables
 * (Lele 1992; Bogey & Bailly 2004; Berland et al. 2007) and must be identical. */
static int make_fd(op_t *o, int scheme, int order) {
  memset(o, 0, sizeof *o);
  o->mfac = -1.0;
  if (scheme == LEE_FD_STANDARD_CENTRAL && order == 4) {
    o->h = 2; o->nb = 2; o->S = 3;
    o->c[2 + 0] = 0.0; o->c[2 + 1] = 8.0 / 12.0; o->c[2 + 2] = -1.0 / 12.0;
    o->B[0][0] = -3.0 / 2.0; o->B[0][1] = 4.0 / 2.0; o->B[0][2] = -1.0 / 2.0;
    o->B[1][0] = -1.0 / 2.0; o->B[1][1] = 0.0; o->B[1][2] = 1.0 / 2.0;
  } else if (scheme == LEE_FD_FDO11P) {
    o->h = 5; o->nb = 5; o->S = 9;
    o->c[5 + 0] = 0.0; o->c[5 + 1] = 0.872756993962; o->c[5 + 2] = -0.286511173973;
    o->c[5 + 3] = 0.090320001280; o->c[5 + 4] = -0.020779405824; o->c[5 + 5] = 0.002484594688;
    double r0[7] = {-2.225833963270, 4.827779580575, -5.001388453836, 3.911103941646,
                    -2.115267458633, 0.718882784412, -0.115276430894};
    double r1[7] = {-0.212932721951, -1.060320390770, 2.078926116439, -1.287179452384,
                    0.685176395471, -0.245320613994, 0.041650667189};
    double r2[5] = {1.0 / 12.0, -8.0 / 12.0, 0.0, 8.0 / 12.0, -1.0 / 12.0};
    double r3[7] = {-0.02625099337517627, 0.18833730683403838, -0.797921633542548, 0.0,
                    0.797921633542548, -0.18833730683403838, 0.02625099337517627};
    double r4[9] = {0.007650904064, -0.059463584768, 0.244678631765, -0.841570125482, 0.0,
                    0.841570125482, -0.244678631765, 0.059463584768, -0.007650904064};
    for (int s = 0; s < 7; ++s) { o->B[0][s] = r0[s]; o->B[1][s] = r1[s]; o->B[3][s] = r3[s]; }
    for (int s = 0; s < 5; ++s) o->B[2][s] = r2[s];
    for (int s = 0; s < 9; ++s) o->B[4][s] = r4[s];
  } else {
    return 0;
  }
  for (int k = 1; k <= o->h; ++k) o->c[o->h - k] = -o->c[o->h + k];
  return 1;
}

static int make_filter(op_t *o, int scheme, int order, double strength) {
  memset(o, 0, sizeof *o);
  o->mfac = 1.0;
  double r2[5] = {(-1.0 / 8.0) / 2.0, (1.0 / 2.0) / 2.0, 5.0 / 8.0, (1.0 / 2.0) / 2.0, (-1.0 / 8.0) / 2.0};
  double r3[7] = {(1.0 / 32.0) / 2.0, (-3.0 / 16.0) / 2.0, (15.0 / 32.0) / 2.0, 11.0 / 16.0,
                  (15.0 / 32.0) / 2.0, (-3.0 / 16.0) / 2.0, (1.0 / 32.0) / 2.0};
  if (scheme == LEE_FILTER_STANDARD_CENTRAL && order == 4) {
    o->h = 2; o->nb = 2; o->S = 3;
    o->c[2] = 5.0 / 8.0; o->c[3] = (1.0 / 2.0) / 2.0; o->c[4] = (-1.0 / 8.0) / 2.0;
    o->B[0][0] = 1.0; o->B[1][1] = 1.0;
  } else if (scheme == LEE_FILTER_STANDARD_CENTRAL && order == 8) {
    o->h = 4; o->nb = 4; o->S = 7;
    o->c[4] = 35.0 / 128.0; o->c[5] = -7.0 / 32.0; o->c[6] = 7.0 / 64.0; o->c[7] = -1.0 / 32.0;
    o->c[8] = 1.0 / 256.0;
    o->c[4] = 1.0 - strength * o->c[4];
    for (int k = 1; k <= 4; ++k) o->c[4 + k] *= -strength;
    o->B[0][0] = 1.0; o->B[1][1] = 1.0;
    for (int s = 0; s < 5; ++s) o->B[2][s] = r2[s];
    for (int s = 0; s < 7; ++s) o->B[3][s] = r3[s];
  } else if (scheme == LEE_FILTER_SFO11P) {
    o->h = 5; o->nb = 5; o->S = 9;
    double d[6] = {0.215044884112, -0.187772883589, 0.123755948787, -0.059227575576, 0.018721609157,
                   -0.002999540835};
    for (int k = 0; k <= 5; ++k) o->c[5 + k] = d[k];
    o->c[5] = 1.0 - strength * o->c[5];
    for (int k = 1; k <= 5; ++k) o->c[5 + k] *= -strength;
    o->B[0][0] = 1.0; o->B[1][1] = 1.0;
    for (int s = 0; s < 5; ++s) o->B[2][s] = r2[s];
    for (int s = 0; s < 7; ++s) o->B[3][s] = r3[s];
    double r4[9] = {0.008228661760, -0.045211119360, 0.120007591680, -0.204788880640, 0.243527493120,
                    -0.204788880640, 0.120007591680, -0.045211119360, 0.008228661760};
    for (int s = 0; s < 9; ++s) o->B[4][s] = (s == 4) ? 1.0 - strength * r4[s] : r4[s] * -strength;
  } else {
    return 0;
  }
  for (int k = 1; k <= o->h; ++k) o->c[o->h - k] = o->c[o->h + k];
  return 1;
}

/* One line of apply_dir: the line at (b1, b2) across the operator's direction. Returns -1
 * where the reference's fluid-support assert would fire. */
static int apply_line(const op_t *o, const int *iblank, const double *f, double *out, int b1, int b2, int st1,
                      int st2, int nd, int sd, int h, int nb, int S) {
  int base = b1 * st1 + b2 * st2;
  for (int i = 0; i < nd; ++i) out[base + i * sd] = 0.0;
  for (int i = h; i <= nd - 1 - h; ++i) {
    int l0 = base + i * sd;
    double acc = out[l0];
    for (int l = -h; l <= h; ++l) acc += o->c[l + h] * f[l0 + l * sd];
    out[l0] = acc;
  }
  for (int i = 0; i < h; ++i) { /* left boundary rows anchored at the first point */
    int l0 = base + i * sd;
    double acc = out[l0];
    for (int s = 0; s < S; ++s) acc += o->B[i][s] * f[base + s * sd];
    out[l0] = acc;
  }
  for (int i = nd - 1; i > nd - 1 - h; --i) { /* right rows mirrored from the last point */
    int r = nd - 1 - i;
    int l0 = base + i * sd, le = base + (nd - 1) * sd;
    double acc = out[l0];
    for (int s = 0; s < S; ++s) acc += o->mfac * o->B[r][s] * f[le - s * sd];
    out[l0] = acc;
  }
  if (!iblank) return 0;
  int last = iblank[base];
  for (int i = 0; i < nd; ++i) {
    int l0 = base + i * sd;
    int my = iblank[l0];
    if (my == BLANKED) {
      if (last == BLANKED) {
        out[l0] = 0.0;
      } else if (last / BLANKED) { /* `last_iblank /= BLANKED` (:1391): true only after an INTERPOLATED point */
        if (i > 0) {
          for (int ib = 0; ib < nb; ++ib) {
            int p = i - 1 - ib;
            if (p < 0) return -1;
            if (iblank[base + p * sd] > 0) return -1;
          }
          if (i - 1 - (S - 1) < 0) return -1; /* the rows would read outside the line */
          int lref = base + (i - 1) * sd;
          for (int ib = 0; ib < nb; ++ib) {
            int p = i - 1 - ib;
            if (p >= 0 && p <= nd - 1) {
              int l1 = base + p * sd;
              out[l1] = 0.0;
              for (int s = 0; s < S; ++s) out[l1] += o->mfac * o->B[ib][s] * f[lref - s * sd];
            }
          }
        }
      }
    } else {
      if (last == BLANKED && i <= nd - 1) {
        for (int ib = 0; ib < nb; ++ib) {
          int p = i + ib;
          if (p > nd - 1) return -1;
          if (iblank[base + p * sd] > 0) return -1;
        }
        if (i + S - 1 > nd - 1) return -1; /* the rows would read outside the line */
        for (int ib = 0; ib < nb; ++ib) {
          int p = i + ib;
          if (p >= 0 && p <= nd - 1) {
            int l1 = base + p * sd;
            out[l1] = 0.0;
            for (int s = 0; s < S; ++s) out[l1] += o->B[ib][s] * f[l0 + s * sd];
          }
        }
      }
    }
    last = my;
  }
  return 0;
}

/* ---------------------------------------------------------------------------
 * One directional application of an operator to f, written to out:
 * StandardCentral::apply_spatial_discretization (src/solver/spatial_discretization.cpp:1078-1290)
 * on a single rank (no ghost cells: is = iso = 0, ie = ieo = n-1, and the stencil
 * ranges of src/geometry/geometry.cpp:931-1001), followed by
 * StandardCentral::iblank_correction (:1356-1652) with the right/left hole
 * closures of :1656-1745. iblank may be NULL (all fluid). Returns 0, or -1 when
 * the reference's fluid-support assert (:1749-1798) would fire. */
static int apply_dir(const op_t *o, const blk_t *bk, const int *iblank, const double *f, double *out, int d) {
  int n[3] = {bk->nx, bk->ny, bk->nz};
  int st[3] = {1, bk->nx, bk->nx * bk->ny};
  int nd = n[d], sd = st[d];
  int o1 = (d == 0) ? 1 : 0, o2 = (d == 2) ? 1 : 2;
  int h = o->h, nb = o->nb, S = o->S;
  int nlines = n[o1] * n[o2], bad = 0;
  PAR_FOR
  for (int line = 0; line < nlines; ++line) {
    if (apply_line(o, iblank, f, out, line % n[o1], line / n[o1], st[o1], st[o2], nd, sd, h, nb, S)) {
#pragma omp atomic write
      bad = 1;
    }
  }
  return bad ? -1 : 0;
}

/* take_derivative_xi_eta_zeta (:1322-1336): dflux <- 0, then the operator; a
 * one-cell direction leaves zero (:1080-1081). */
static int d_xi(orc_ctx *c, const blk_t *bk, const int *ib, const double *f, double *out, int d) {
  int n[3] = {bk->nx, bk->ny, bk->nz};
  if (n[d] == 1) {
    memset(out, 0, sizeof(double) * (size_t)bk->N);
    return 0;
  }
  if (apply_dir(&c->fd, bk, ib, f, out, d)) return fail(c, LEE_ERR_ARG, "hole closure lacks fluid support");
  return 0;
}

/* take_derivative_xyz (:1802-1826): dflux = J * sum_l metrics[l][i] * d/dxi_l f. */
static int d_x(orc_ctx *c, const blk_t *bk, const double *f, double *out, int i, double *work, double *sum) {
  int nd = c->cfg.num_dim, N = bk->N;
  PAR_FOR
  for (int p = 0; p < N; ++p) sum[p] = 0.0;
  for (int l = 0; l < nd; ++l) {
    int rc = d_xi(c, bk, bk->iblank, f, work, l);
    if (rc) return rc;
    const double *m = bk->met[l * 3 + i];
    PAR_FOR
    for (int p = 0; p < N; ++p) sum[p] += m[p] * work[p];
  }
  PAR_FOR
  for (int p = 0; p < N; ++p) out[p] = sum[p] * bk->jac[p];
  return 0;
}

/* Three work fields of at least n points, kept by the context between calls. */
static double **scratch(orc_ctx *c, size_t n) {
  if (c->scrn < n) {
    for (int k = 0; k < 3; ++k) {
      free(c->scr[k]);
      c->scr[k] = dalloc(n);
    }
    c->scrn = n;
  }
  return c->scr;
}

/* ---------------------------------------------------------------------------
 * Metrics: metrics::compute (src/metrics/metrics.cpp:9-44) with Thomas-Lombard
 * products (:107-251), the Jacobian (:255-328, with oracle patch P1 in 3-D: the
 * determinant formula kept as comments at :297-307) and the inverse (:355-426).
 * The reference computes metrics before the overset iblank exists
 * (src/core/simulation.cpp:207 vs :214), so no hole closures apply here. */
static int compute_metrics(orc_ctx *c, blk_t *bk) {
  int nd = c->cfg.num_dim, N = bk->N;
  double *xx[3][3] = {{0}};
  double *func = dalloc((size_t)N), *tmp = dalloc((size_t)N);
  for (int k = 0; k < 9; ++k) {
    bk->met[k] = dalloc((size_t)N);
    bk->minv[k] = dalloc((size_t)N);
  }
  bk->jac = dalloc((size_t)N);
  bk->invjac = dalloc((size_t)N);
  for (int ip = 0; ip < nd; ++ip)
    for (int ic = 0; ic < nd; ++ic) {
      xx[ip][ic] = dalloc((size_t)N);
      if (d_xi(c, bk, NULL, bk->xyz[ip], xx[ip][ic], ic)) return LEE_ERR_ARG;
    }
  double **m = bk->met;
#define M(l, i) m[(l) * 3 + (i)]
  if (nd == 2) {
    for (int p = 0; p < N; ++p) {
      M(0, 0)[p] = xx[1][1][p];
      M(0, 1)[p] = -xx[0][1][p];
      M(1, 0)[p] = -xx[1][0][p];
      M(1, 1)[p] = xx[0][0][p];
    }
  } else {
    double **z = bk->xyz;
    /* xi_x and zeta_x from (y_eta z) */
    for (int p = 0; p < N; ++p) func[p] = xx[1][1][p] * z[2][p];
    d_xi(c, bk, NULL, func, tmp, 2); for (int p = 0; p < N; ++p) M(0, 0)[p] = tmp[p];
    d_xi(c, bk, NULL, func, tmp, 0); for (int p = 0; p < N; ++p) M(2, 0)[p] = -tmp[p];
    for (int p = 0; p < N; ++p) func[p] = xx[0][1][p] * z[2][p];
    d_xi(c, bk, NULL, func, tmp, 2); for (int p = 0; p < N; ++p) M(0, 1)[p] = -tmp[p];
    d_xi(c, bk, NULL, func, tmp, 0); for (int p = 0; p < N; ++p) M(2, 1)[p] = tmp[p];
    for (int p = 0; p < N; ++p) func[p] = xx[0][1][p] * z[1][p];
    d_xi(c, bk, NULL, func, tmp, 2); for (int p = 0; p < N; ++p) M(0, 2)[p] = tmp[p];
    d_xi(c, bk, NULL, func, tmp, 0); for (int p = 0; p < N; ++p) M(2, 2)[p] = -tmp[p];
    for (int p = 0; p < N; ++p) func[p] = xx[1][0][p] * z[2][p];
    d_xi(c, bk, NULL, func, tmp, 2); for (int p = 0; p < N; ++p) M(1, 0)[p] = -tmp[p];
    d_xi(c, bk, NULL, func, tmp, 1); for (int p = 0; p < N; ++p) M(2, 0)[p] += tmp[p];
    for (int p = 0; p < N; ++p) func[p] = xx[0][0][p] * z[2][p];
    d_xi(c, bk, NULL, func, tmp, 2); for (int p = 0; p < N; ++p) M(1, 1)[p] = tmp[p];
    d_xi(c, bk, NULL, func, tmp, 1); for (int p = 0; p < N; ++p) M(2, 1)[p] -= tmp[p];
    for (int p = 0; p < N; ++p) func[p] = xx[0][0][p] * z[1][p];
    d_xi(c, bk, NULL, func, tmp, 2); for (int p = 0; p < N; ++p) M(1, 2)[p] = -tmp[p];
    d_xi(c, bk, NULL, func, tmp, 1); for (int p = 0; p < N; ++p) M(2, 2)[p] += tmp[p];
    for (int p = 0; p < N; ++p) func[p] = xx[1][2][p] * z[2][p];
    d_xi(c, bk, NULL, func, tmp, 1); for (int p = 0; p < N; ++p) M(0, 0)[p] -= tmp[p];
    d_xi(c, bk, NULL, func, tmp, 0); for (int p = 0; p < N; ++p) M(1, 0)[p] += tmp[p];
    for (int p = 0; p < N; ++p) func[p] = xx[0][2][p] * z[2][p];
    d_xi(c, bk, NULL, func, tmp, 1); for (int p = 0; p < N; ++p) M(0, 1)[p] += tmp[p];
    d_xi(c, bk, NULL, func, tmp, 0); for (int p = 0; p < N; ++p) M(1, 1)[p] -= tmp[p];
    for (int p = 0; p < N; ++p) func[p] = xx[0][2][p] * z[1][p];
    d_xi(c, bk, NULL, func, tmp, 1); for (int p = 0; p < N; ++p) M(0, 2)[p] -= tmp[p];
    d_xi(c, bk, NULL, func, tmp, 0); for (int p = 0; p < N; ++p) M(1, 2)[p] += tmp[p];
  }
  for (int p = 0; p < N; ++p) {
    if (nd == 2) {
      bk->invjac[p] = xx[0][0][p] * xx[1][1][p] - xx[0][1][p] * xx[1][0][p];
    } else {
      bk->invjac[p] = xx[0][0][p] * (xx[1][1][p] * xx[2][2][p] - xx[1][2][p] * xx[2][1][p])
                    - xx[0][1][p] * (xx[1][0][p] * xx[2][2][p] - xx[1][2][p] * xx[2][0][p])
                    + xx[0][2][p] * (xx[1][0][p] * xx[2][1][p] - xx[1][1][p] * xx[2][0][p]);
    }
    bk->jac[p] = 1.0 / bk->invjac[p];
  }
  double **mi = bk->minv;
#define MI(i, l) mi[(i) * 3 + (l)]
  for (int p = 0; p < N; ++p) {
    if (nd == 2) {
      MI(0, 0)[p] = M(1, 1)[p];
      MI(0, 1)[p] = -M(0, 1)[p];
      MI(1, 0)[p] = -M(1, 0)[p];
      MI(1, 1)[p] = M(0, 0)[p];
    } else {
      MI(0, 0)[p] = M(1, 1)[p] * M(2, 2)[p] - M(1, 2)[p] * M(2, 1)[p];
      MI(0, 1)[p] = M(0, 2)[p] * M(2, 1)[p] - M(0, 1)[p] * M(2, 2)[p];
      MI(0, 2)[p] = M(0, 1)[p] * M(1, 2)[p] - M(0, 2)[p] * M(1, 1)[p];
      MI(1, 0)[p] = M(1, 2)[p] * M(2, 0)[p] - M(1, 0)[p] * M(2, 2)[p];
      MI(1, 1)[p] = M(0, 0)[p] * M(2, 2)[p] - M(0, 2)[p] * M(2, 0)[p];
      MI(1, 2)[p] = M(0, 2)[p] * M(1, 0)[p] - M(0, 0)[p] * M(1, 2)[p];
      MI(2, 0)[p] = M(1, 0)[p] * M(2, 1)[p] - M(1, 1)[p] * M(2, 0)[p];
      MI(2, 1)[p] = M(0, 1)[p] * M(2, 0)[p] - M(0, 0)[p] * M(2, 1)[p];
      MI(2, 2)[p] = M(0, 0)[p] * M(1, 1)[p] - M(0, 1)[p] * M(1, 0)[p];
    }
  }
#undef M
#undef MI
  for (int ip = 0; ip < 3; ++ip)
    for (int ic = 0; ic < 3; ++ic) free(xx[ip][ic]);
  free(func);
  free(tmp);
  return 0;
}

/* State::compute_auxiliary_variables_linear_Euler (src/core/state.cpp:701-736). */
static void compute_aux(orc_ctx *c, blk_t *bk, double *const *y) {
  double g = c->cfg.gamma, gi = 1.0 / g, gg = g / (g - 1.0);
  PAR_FOR
  for (int p = 0; p < bk->N; ++p) {
    double sbar = bk->mean[0][p], pbar = bk->mean[4][p];
    double pbi = 1.0 / pbar;
    double rhobar = pow(g * pbar, gi) * exp(-sbar);
    double rbi = 1.0 / rhobar;
    double Tbar = pbar * gg * rbi;
    bk->aux[1][p] = rhobar;
    bk->aux[0][p] = y[4][p] * gi * pbi - y[0][p];
    bk->aux[0][p] *= rhobar;
    bk->aux[3][p] = Tbar;
    bk->aux[2][p] = y[4][p] * pbi - bk->aux[0][p] * rbi;
    bk->aux[2][p] *= Tbar;
  }
}

/* Sponge strength: Geometry::additionalInit_bufferZones (src/geometry/geometry.cpp:1028-1142)
 * with the zone's IN/OUT faces of StructuredBufferZone::set_parameters_4bufferZone (:715-743). */
static void compute_sigma(orc_ctx *c, blk_t *bk, bnd_t *z) {
  int bn[3], face[2][2];
  for (int d = 0; d < 3; ++d) bn[d] = z->hi[d] - z->lo[d] + 1;
  int nb = bn[0] * bn[1] * bn[2];
  z->sigma = dalloc((size_t)nb);
  int d = z->dir;
  /* [side][0] = index of the face in direction d; side 0 = IN, 1 = OUT */
  if (z->end == 0) { face[0][0] = z->hi[d]; face[1][0] = z->lo[d]; }
  else { face[0][0] = z->lo[d]; face[1][0] = z->hi[d]; }
  for (int k = z->lo[2]; k <= z->hi[2]; ++k)
    for (int j = z->lo[1]; j <= z->hi[1]; ++j)
      for (int i = z->lo[0]; i <= z->hi[0]; ++i) {
        int l0 = i + bk->nx * (j + bk->ny * k);
        double xb[3] = {bk->xyz[0][l0], bk->xyz[1][l0], bk->xyz[2][l0]};
        double dist[2];
        for (int side = 0; side < 2; ++side) {
          double dmin = 1000000000.0; /* abs(DUMMY_DOUBLE) through int abs (:1110) */
          int flo[3] = {z->lo[0], z->lo[1], z->lo[2]}, fhi[3] = {z->hi[0], z->hi[1], z->hi[2]};
          flo[d] = fhi[d] = face[side][0];
          for (int kk = flo[2]; kk <= fhi[2]; ++kk)
            for (int jj = flo[1]; jj <= fhi[1]; ++jj)
              for (int ii = flo[0]; ii <= fhi[0]; ++ii) {
                int lf = ii + bk->nx * (jj + bk->ny * kk);
                double s = 0.0;
                for (int q = 0; q < 3; ++q) s += pow(xb[q] - bk->xyz[q][lf], 2);
                if (s < dmin) dmin = s;
              }
          dist[side] = sqrt(dmin);
        }
        double rel = dist[0] / (dist[0] + dist[1]);
        int lb = (i - z->lo[0]) + bn[0] * ((j - z->lo[1]) + bn[1] * (k - z->lo[2]));
        z->sigma[lb] = c->cfg.sponge_constant * pow(rel, c->cfg.sponge_order);
      }
}

/* ---------------------------------------------------------------------------
 * Right-hand side: spatial::compute_RHS (src/solver/spatial_discretization.cpp:1963-1990),
 * compute_RHS_linearized_Euler (:2053-2130) and source::add_RHSSourceTerms
 * (src/solver/source.cpp:10-18): physical source, then Freund sponges (:174-201). */
/* The wave of bc::bc_dirichlet_harmonicwave (src/solver/boundary_condition.cpp:232-344) at
 * point l0 and the given time, into the five LEE slots (entropy 0, velocity 1 + dir, pressure
 * 4; every other slot 0), for a point that is not a hole. */
static const int dir_other[3][2] = {{1, 2}, {0, 2}, {0, 1}}; /* src/core/param.h:133 */
static void wave_at(const orc_ctx *c, const blk_t *bk, int l0, double time, double out[5]) {
  double rho_0 = 1.0, p_0 = 1.0 / c->cfg.gamma, c_0 = 1.0;
  double wavenumber = (2.0 * acos(-1.0)) / c->wave_len;
  int idir = c->wave_dir;
  double loc = bk->xyz[idir][l0];
  double t1 = bk->xyz[dir_other[idir][0]][l0], t2 = bk->xyz[dir_other[idir][1]][l0];
  double pf = 0.0, vf = 0.0, sf = 0.0;
  if (c->wave_form == LEE_WAVEFORM_PLANE) {
    pf = c->wave_amp * p_0 * sin(wavenumber * (loc - c_0 * time));
    vf = pf;
  } else if (c->wave_form == LEE_WAVEFORM_HOMOGENEOUS && c->wave_type == LEE_WAVE_ACOUSTIC) {
    pf = c->wave_amp * p_0 * sin(wavenumber * c_0 * time);
    vf = pf;
  } else {
    sf = c->wave_amp * (1.0 + sin(wavenumber * c_0 * time));
    if (c->wave_form == LEE_WAVEFORM_GAUSSIAN_ROUNDJET) {
      double fac = -log(2.0) / pow(c->wave_hw, 2);
      sf *= exp(fac * (pow(t1, 2) + pow(t2, 2)));
    }
  }
  for (int v = 0; v < 5; ++v) out[v] = 0.0;
  out[0] = sf;
  out[1 + idir] = vf / (rho_0 * c_0);
  out[4] = pf;
}

static int rhs_block(orc_ctx *c, blk_t *bk, double *const *y, double **rhs, double time) {
  int nd = c->cfg.num_dim, N = bk->N;
  double g = c->cfg.gamma;
  double **scr = scratch(c, (size_t)N);
  double *df = scr[0], *work = scr[1], *sum = scr[2];
  int rc = 0;
  for (int v = 0; v < c->nv; ++v) memset(rhs[v], 0, sizeof(double) * (size_t)N);
  for (int j = 0; j < nd && !rc; ++j) { /* entropy */
    rc = d_x(c, bk, y[0], df, j, work, sum);
    PAR_FOR
    for (int p = 0; p < N; ++p) rhs[0][p] -= bk->mean[1 + j][p] * df[p];
    PAR_FOR
    for (int p = 0; p < N; ++p) rhs[0][p] -= y[1 + j][p] * bk->grad[0 * nd + j][p];
  }
  for (int i = 0; i < nd && !rc; ++i) { /* velocity */
    for (int j = 0; j < nd && !rc; ++j) {
      rc = d_x(c, bk, y[1 + i], df, j, work, sum);
      PAR_FOR
      for (int p = 0; p < N; ++p) rhs[1 + i][p] -= bk->mean[1 + j][p] * df[p];
      PAR_FOR
      for (int p = 0; p < N; ++p)
        rhs[1 + i][p] -= (y[1 + j][p] + bk->aux[0][p] / bk->aux[1][p] * bk->mean[1 + j][p]) *
                         bk->grad[(1 + i) * nd + j][p];
    }
    if (!rc) rc = d_x(c, bk, y[4], df, i, work, sum);
    PAR_FOR
    for (int p = 0; p < N; ++p) rhs[1 + i][p] -= df[p] / bk->aux[1][p];
  }
  for (int j = 0; j < nd && !rc; ++j) { /* pressure */
    rc = d_x(c, bk, y[4], df, j, work, sum);
    PAR_FOR
    for (int p = 0; p < N; ++p) rhs[4][p] -= bk->mean[1 + j][p] * df[p];
    PAR_FOR
    for (int p = 0; p < N; ++p) rhs[4][p] -= y[1 + j][p] * bk->grad[4 * nd + j][p];
    if (!rc) rc = d_x(c, bk, y[1 + j], df, j, work, sum);
    PAR_FOR
    for (int p = 0; p < N; ++p) rhs[4][p] -= g * bk->mean[4][p] * df[p];
    PAR_FOR
    for (int p = 0; p < N; ++p) rhs[4][p] -= g * y[4][p] * bk->grad[(1 + j) * nd + j][p];
  }
  if (rc) return rc;
  if (c->axisym) /* additional terms due to axisymmetry (:2118-2126), IVAR_UR = 2, RDIR = 1 */
    PAR_FOR
    for (int p = 0; p < N; ++p)
      rhs[4][p] -= g * (bk->mean[4][p] * y[2][p] + y[4][p] * bk->mean[2][p]) / (bk->xyz[1][p] + 1e-99);
  /* compute_RHS_linearized_Euler_scalar (:2134-2158): dZ'/dt = -u_bar . grad Z' - u' . grad Z_bar */
  for (int k = 0; k < c->nsc && !rc; ++k) {
    int v = 5 + k;
    for (int j = 0; j < nd && !rc; ++j) {
      rc = d_x(c, bk, y[v], df, j, work, sum);
      PAR_FOR
      for (int p = 0; p < N; ++p) rhs[v][p] -= bk->mean[1 + j][p] * df[p];
      PAR_FOR
      for (int p = 0; p < N; ++p) rhs[v][p] -= y[1 + j][p] * bk->grad[v * nd + j][p];
    }
  }
  if (rc) return rc;
  if (c->src_kind == LEE_SOURCE_DISTRIBUTED && bk == &c->blk[(int)c->dsrc[0]] && c->dsrc_g) {
    double fac = (g - 1.0) * sin(c->dsrc[1] * time);
    PAR_FOR
    for (int p = 0; p < N; ++p) rhs[4][p] += fac * c->dsrc_g[p];
  }
  int bix = (int)(bk - &c->blk[0]);
  if (c->src_kind == LEE_SOURCE_JET2D_HARMONIC && c->bsrc_mode[bix] == 0) { /* source.cpp:27-58 */
    double twopi = 2.0 * acos(-1.0), inverse_twopi = 1.0 / twopi;
    double amplitude = 0.001, frequency = 76.0, Bx = 0.04 * log(2.0), By = 0.32 * log(2.0);
    double b = 1.3, R = 287.0, rhoinfty = 1.184, Tinfty = 300.0;
    double cinfty = sqrt(g * R * Tinfty);
    amplitude /= rhoinfty * pow(cinfty, 2) / (b / cinfty);
    frequency *= inverse_twopi * (b / cinfty);
    Bx *= pow(b, 2);
    By *= pow(b, 2);
    double angular_frequency = frequency * twopi;
    double amp_cos_wt = amplitude * cos(angular_frequency * time);
    PAR_FOR
    for (int p = 0; p < N; ++p) {
      double xloc = bk->xyz[0][p], yloc = bk->xyz[1][p];
      rhs[4][p] += exp(-(Bx * xloc * xloc + By * yloc * yloc)) * amp_cos_wt;
    }
  }
  const double *mp = c->bsrc_mode[bix] == 1 ? c->bsrc[bix]
                   : (c->bsrc_mode[bix] == 0 && c->src_kind == LEE_SOURCE_MONOPOLE && c->src[5] > 0.0) ? c->src
                   : NULL;
  if (mp) { /* oracle patch P2 (oracle/ref_patch_source.cpp) */
    double x0 = mp[0], y0 = mp[1], z0 = mp[2], amp = mp[3], om = mp[4];
    double b = mp[5], T = mp[6];
    double ramp = 1.0;
    if (T > 0.0 && time < T) {
      double s = sin(0.5 * M_PI * time / T);
      ramp = s * s;
    }
    double fac = amp * (g - 1.0) * ramp * sin(om * time);
    double ef = -log(2.0) / (b * b);
    PAR_FOR
    for (int p = 0; p < N; ++p) {
      double dx = bk->xyz[0][p] - x0, dy = bk->xyz[1][p] - y0, dz = bk->xyz[2][p] - z0;
      rhs[4][p] += fac * exp(ef * (dx * dx + dy * dy + dz * dz));
    }
  }
  for (int zi = 0; zi < bk->nbnd; ++zi) {
    bnd_t *z = &bk->bnd[zi];
    int wave = z->kind == LEE_SPONGE_FREUND_HARMONICWAVE; /* apply_bufferZone_Freund_harmonicWave (:264-320) */
    if (z->kind != LEE_SPONGE_FREUND_AMBIENT && !wave) continue;
    int bn0 = z->hi[0] - z->lo[0] + 1, bn1 = z->hi[1] - z->lo[1] + 1;
    for (int k = z->lo[2]; k <= z->hi[2]; ++k)
      for (int j = z->lo[1]; j <= z->hi[1]; ++j)
        for (int i = z->lo[0]; i <= z->hi[0]; ++i) {
          int lb = (i - z->lo[0]) + bn0 * ((j - z->lo[1]) + bn1 * (k - z->lo[2]));
          int l0 = i + bk->nx * (j + bk->ny * k);
          double sg = z->sigma[lb];
          double ref[MAXV] = {0.0};
          if (wave && !(bk->iblank && bk->iblank[l0] == BLANKED)) wave_at(c, bk, l0, time, ref);
          for (int v = 0; v < c->nv; ++v) { /* the scalars relax to zero (sol_ref, src/core/state.cpp:361-363) */
            double relax = -sg * (y[v][l0] - ref[v]);
            rhs[v][l0] += relax;
          }
        }
  }
  return 0;
}

/* ---------------------------------------------------------------------------
 * Boundary conditions: bc::apply_BC (src/solver/boundary_condition.cpp:46-209) with
 * bc_dirichlet_allzero (:213-228), bc_dirichlet_harmonicwave (:232-344), bc_neumann
 * (:348-444), bc_wall_slip_kinematic (:448-494) and bc_centerline (:498-574) at the given
 * time. The boundary is the box's end face in its direction (src/geometry/geometry.cpp:583-645). */
static void apply_bc(orc_ctx *c, blk_t *bk, double **y, double time) {
  int nd = c->cfg.num_dim;
  int st[3] = {1, bk->nx, bk->nx * bk->ny};
  const op_t *o = &c->fd;
  for (int zi = 0; zi < bk->nbnd; ++zi) {
    bnd_t *z = &bk->bnd[zi];
    int centerline = z->kind >= LEE_BC_CENTERLINE_CART_NORM2X && z->kind <= LEE_BC_CENTERLINE_AXISYM;
    int dirichlet = z->kind == LEE_BC_DIRICHLET_ALLZERO || z->kind == LEE_BC_DIRICHLET_HARMONICWAVE;
    if (z->kind != LEE_BC_NEUMANN && z->kind != LEE_BC_WALL_SLIP_KINEMATIC && !centerline && !dirichlet) continue;
    int lo[3] = {z->lo[0], z->lo[1], z->lo[2]}, hi[3] = {z->hi[0], z->hi[1], z->hi[2]};
    lo[z->dir] = hi[z->dir] = (z->end == 0) ? z->lo[z->dir] : z->hi[z->dir];
    int sd = st[z->dir];
    int nbx = hi[0] - lo[0] + 1, nby = hi[1] - lo[1] + 1, nbz = hi[2] - lo[2] + 1;
    int nbp = nbx * nby * nbz;
    int nv = c->nv;
    double *data[MAXV];
    for (int v = 0; v < nv; ++v) data[v] = dalloc((size_t)nbp);
    int vars_neu[MAXV], nneu = 0;
    if (z->kind == LEE_BC_NEUMANN || centerline) {
      for (int v = 0; v < nv; ++v) vars_neu[nneu++] = v;
    } else if (z->kind == LEE_BC_WALL_SLIP_KINEMATIC) {
      /* every non-velocity slot, the scalars included (:122-133) */
      vars_neu[nneu++] = 0;
      vars_neu[nneu++] = 4;
      for (int v = 5; v < nv; ++v) vars_neu[nneu++] = v;
    }
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          int lb = (i - lo[0]) + nbx * ((j - lo[1]) + nby * (k - lo[2]));
          int l0 = i + bk->nx * (j + bk->ny * k);
          int hole = bk->iblank && bk->iblank[l0] == BLANKED;
          if (dirichlet) {
            for (int v = 0; v < nv; ++v) data[v][lb] = 0.0;
            if (z->kind == LEE_BC_DIRICHLET_HARMONICWAVE && !hole) {
              double w[5];
              wave_at(c, bk, l0, time, w);
              for (int v = 0; v < 5; ++v) data[v][lb] = w[v];
            }
          }
          if (!hole) {
            for (int q = 0; q < nneu; ++q) {
              int v = vars_neu[q];
              data[v][lb] = 0.0;
              if (z->end == 0) {
                for (int s = 1; s < o->S; ++s) data[v][lb] -= o->B[0][s] * y[v][l0 + sd * s];
                data[v][lb] /= o->B[0][0];
              } else {
                for (int s = 1; s < o->S; ++s) data[v][lb] += o->B[0][s] * y[v][l0 - sd * s];
                data[v][lb] /= -o->B[0][0];
              }
            }
          }
          if (z->kind == LEE_BC_WALL_SLIP_KINEMATIC) {
            double vc[3] = {0, 0, 0}, vel[3] = {0, 0, 0};
            if (!hole) {
              for (int q = 0; q < 3; ++q) vel[q] = y[1 + q][l0];
              for (int l = 0; l < nd; ++l) {
                vc[l] = 0.0;
                for (int q = 0; q < nd; ++q) vc[l] += bk->met[l * 3 + q][l0] * vel[q];
              }
              vc[z->dir] = 0.0;
              for (int q = 0; q < nd; ++q) {
                vel[q] = 0.0;
                for (int l = 0; l < nd; ++l) vel[q] += bk->minv[q * 3 + l][l0] * vc[l];
                vel[q] *= bk->jac[l0];
              }
            }
            for (int q = 0; q < 3; ++q) data[1 + q][lb] = vel[q];
          }
          if (centerline && !hole) /* IVAR_UX + which_dir, or IVAR_UR on the axis */
            data[z->kind == LEE_BC_CENTERLINE_AXISYM ? 2 : 1 + (z->kind - LEE_BC_CENTERLINE_CART_NORM2X)][lb] = 0.0;
        }
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          int lb = (i - lo[0]) + nbx * ((j - lo[1]) + nby * (k - lo[2]));
          int l0 = i + bk->nx * (j + bk->ny * k);
          if (bk->iblank && bk->iblank[l0] == BLANKED) continue;
          for (int v = 0; v < nv; ++v) y[v][l0] = data[v][lb];
        }
    for (int v = 0; v < nv; ++v) free(data[v]);
  }
}

/* spatial::apply_filter (src/solver/spatial_discretization.cpp:2191-2246) for one block. */
static int filter_block(orc_ctx *c, blk_t *bk, double **y) {
  int N = bk->N, n[3] = {bk->nx, bk->ny, bk->nz};
  double *func0 = dalloc((size_t)N), *func = dalloc((size_t)N), *out = dalloc((size_t)N);
  double blend = c->cfg.filter_blend, rem = 1.0 - blend;
  for (int v = 0; v < c->nv; ++v) {
    memcpy(func0, y[v], sizeof(double) * (size_t)N);
    memcpy(func, func0, sizeof(double) * (size_t)N);
    for (int d = 0; d < c->cfg.num_dim; ++d) {
      if (n[d] == 1) continue; /* dflux = func: a one-cell direction is left alone */
      if (apply_dir(&c->flt, bk, bk->iblank, func, out, d)) {
        free(func0); free(func); free(out);
        return fail(c, LEE_ERR_ARG, "filter hole closure lacks fluid support");
      }
      memcpy(func, out, sizeof(double) * (size_t)N);
    }
    PAR_FOR
    for (int p = 0; p < N; ++p) y[v][p] = rem * func0[p] + blend * func[p];
  }
  free(func0); free(func); free(out);
  return 0;
}

/* overset::interpolate (src/overset/overset.cpp:820-845) in its OVERTURE form: every
 * receiver's weighted sum over its donor stencil, for all five variables
 * (compute_weighted_sum :886-974), all of them before any receiver is overwritten
 * (update_each_grid :1241-1278). y[b] is the stage output of block b. */
static void interpolate(orc_ctx *c, double **y[MAXB]) {
  ovs_t *o = &c->ovs;
  for (int r = 0; r < o->n; ++r) {
    blk_t *dk = &c->blk[o->db[r]];
    double acc[MAXV] = {0.0};
    const double *cf = o->wt + (size_t)r * o->W;
    int st = 0;
    for (int w3 = 0; w3 < o->w[2]; ++w3)
      for (int w2 = 0; w2 < o->w[1]; ++w2)
        for (int w1 = 0; w1 < o->w[0]; ++w1) {
          long long l1 = o->dl[r] + (w1 + w2 * dk->nx + (long long)w3 * dk->nx * dk->ny);
          for (int v = 0; v < c->nv; ++v) acc[v] += cf[st] * y[o->db[r]][v][l1];
          st++;
        }
    for (int v = 0; v < c->nv; ++v) o->buf[(size_t)r * MAXV + v] = acc[v];
  }
  for (int r = 0; r < o->n; ++r)
    for (int v = 0; v < c->nv; ++v) y[o->rb[r]][v][o->rl[r]] = o->buf[(size_t)r * MAXV + v];
}

/* ---------------------------------------------------------------------------
 * Exported ABI (orc_ prefix). */
int orc_create(const lee_config *cfg, orc_ctx **out) {
  if (!cfg || !out) return fail(NULL, LEE_ERR_ARG, "null argument");
  if (cfg->num_dim != 2 && cfg->num_dim != 3) return fail(NULL, LEE_ERR_ARG, "num_dim must be 2 or 3");
  if (cfg->num_blocks < 1 || cfg->num_blocks > MAXB) return fail(NULL, LEE_ERR_ARG, "bad num_blocks");
  orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
  c->cfg = *cfg;
  if (!make_fd(&c->fd, cfg->fd_scheme, cfg->fd_order)) {
    free(c);
    return fail(NULL, LEE_ERR_UNSUPPORTED, "unsupported spatial scheme");
  }
  if (cfg->filter_scheme != LEE_FILTER_NONE) {
    double s = cfg->filter_scheme == LEE_FILTER_STANDARD_CENTRAL ? 1.0 : cfg->filter_strength;
    if (!make_filter(&c->flt, cfg->filter_scheme, cfg->filter_order, s)) {
      free(c);
      return fail(NULL, LEE_ERR_UNSUPPORTED, "unsupported filter");
    }
  }
  c->nblk = cfg->num_blocks;
  c->nv = 5;
  *out = c;
  return LEE_OK;
}

void orc_destroy(orc_ctx *c) {
  if (!c) return;
  for (int b = 0; b < c->nblk; ++b) {
    blk_t *bk = &c->blk[b];
    for (int q = 0; q < 3; ++q) free(bk->xyz[q]);
    free(bk->iblank);
    for (int q = 0; q < 9; ++q) { free(bk->met[q]); free(bk->minv[q]); }
    free(bk->jac); free(bk->invjac);
    for (int q = 0; q < MAXV; ++q) { free(bk->mean[q]); free(bk->sol[q]); }
    for (int q = 0; q < 3 * MAXV; ++q) free(bk->grad[q]);
    for (int q = 0; q < 4; ++q) free(bk->aux[q]);
    for (int q = 0; q < bk->nbnd; ++q) free(bk->bnd[q].sigma);
  }
  for (int k = 0; k < 3; ++k) free(c->scr[k]);
  free(c->ovs.rb); free(c->ovs.db); free(c->ovs.rl); free(c->ovs.dl); free(c->ovs.wt); free(c->ovs.buf);
  free(c->dsrc); free(c->dsrc_g); free(c->mic);
  free(c);
}

const char *orc_last_error(const orc_ctx *c) { return c ? c->err : g_err; }

int orc_set_block(orc_ctx *c, int b, int nx, int ny, int nz, const double *x, const double *y,
                  const double *z, const int *iblank) {
  if (b < 0 || b >= c->nblk) return fail(c, LEE_ERR_ARG, "block index");
  blk_t *bk = &c->blk[b];
  bk->nx = nx; bk->ny = ny; bk->nz = nz;
  bk->N = nx * ny * nz;
  const double *src[3] = {x, y, z};
  for (int q = 0; q < 3; ++q) {
    bk->xyz[q] = dalloc((size_t)bk->N);
    memcpy(bk->xyz[q], src[q], sizeof(double) * (size_t)bk->N);
  }
  if (iblank) {
    bk->iblank = (int *)malloc(sizeof(int) * (size_t)bk->N);
    memcpy(bk->iblank, iblank, sizeof(int) * (size_t)bk->N);
  }
  for (int q = 0; q < c->nv; ++q) { bk->mean[q] = dalloc((size_t)bk->N); bk->sol[q] = dalloc((size_t)bk->N); }
  for (int q = 0; q < 4; ++q) bk->aux[q] = dalloc((size_t)bk->N);
  bk->set = 1;
  return LEE_OK;
}

int orc_set_mean(orc_ctx *c, int b, const double *const mean[5]) {
  if (b < 0 || b >= c->nblk || !c->blk[b].set) return fail(c, LEE_ERR_STATE, "set_block first");
  for (int q = 0; q < 5; ++q) memcpy(c->blk[b].mean[q], mean[q], sizeof(double) * (size_t)c->blk[b].N);
  return LEE_OK;
}

int orc_add_boundary(orc_ctx *c, int b, int kind, int dir, int end, const int lo[3], const int hi[3],
                     const double *sigma) {
  if (b < 0 || b >= c->nblk || !c->blk[b].set) return fail(c, LEE_ERR_STATE, "set_block first");
  blk_t *bk = &c->blk[b];
  if (bk->nbnd >= MAXBND) return fail(c, LEE_ERR_ARG, "too many boundaries");
  bnd_t *z = &bk->bnd[bk->nbnd++];
  z->kind = kind; z->dir = dir; z->end = end;
  for (int d = 0; d < 3; ++d) { z->lo[d] = lo[d]; z->hi[d] = hi[d]; }
  z->sigma = NULL;
  if ((kind == LEE_SPONGE_FREUND_AMBIENT || kind == LEE_SPONGE_FREUND_HARMONICWAVE) && sigma) {
    int nb = (hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
    z->sigma = dalloc((size_t)nb);
    memcpy(z->sigma, sigma, sizeof(double) * (size_t)nb);
  }
  return LEE_OK;
}

/* The HARMONIC_WAVE deck line (src/core/input.cpp:219-231) with check_consistency_wave's
 * amplitude range (:650-652); the forms each type has a formula for
 * (src/solver/boundary_condition.cpp:263-307). */
int orc_set_harmonic_wave(orc_ctx *c, int type, int form, int dir, double amplitude, double wavelength,
                          double halfwidth) {
  if (type == LEE_WAVE_NONE) {
    c->wave_type = LEE_WAVE_NONE;
    return LEE_OK;
  }
  int ok = (type == LEE_WAVE_ACOUSTIC && (form == LEE_WAVEFORM_PLANE || form == LEE_WAVEFORM_HOMOGENEOUS)) ||
           (type == LEE_WAVE_ENTROPY && (form == LEE_WAVEFORM_HOMOGENEOUS || form == LEE_WAVEFORM_GAUSSIAN_ROUNDJET));
  if (!ok) return fail(c, LEE_ERR_ARG, "unknown type of wave for this wave form");
  if (dir < 0 || dir > 2) return fail(c, LEE_ERR_ARG, "wave direction");
  if (amplitude < 0.0 || amplitude > 1.0) return fail(c, LEE_ERR_ARG, "the wave amplitude should be between 0 and 1");
  if (!(wavelength > 0.0)) return fail(c, LEE_ERR_ARG, "wavelength");
  if (form == LEE_WAVEFORM_GAUSSIAN_ROUNDJET && !(halfwidth > 0.0)) return fail(c, LEE_ERR_ARG, "halfwidth");
  c->wave_type = type;
  c->wave_form = form;
  c->wave_dir = dir;
  c->wave_amp = amplitude;
  c->wave_len = wavelength;
  c->wave_hw = halfwidth;
  return LEE_OK;
}

/* AXISYMMETRY (src/core/input.cpp:105-108) with check_consistency_dimension (:519-535). */
int orc_set_axisymmetric(orc_ctx *c, int on, int axis) {
  if (!on) {
    c->axisym = 0;
    return LEE_OK;
  }
  if (c->cfg.num_dim != 2) return fail(c, LEE_ERR_ARG, "Axisymmetry requires 2-D.");
  if (axis != 0) return fail(c, LEE_ERR_ARG, "The axis of symmetry should be x by definition of the coordinate system.");
  c->axisym = 1;
  return LEE_OK;
}

int orc_set_source(orc_ctx *c, int kind, const double *params, int np) {
  c->src_kind = kind;
  if (kind == LEE_SOURCE_DISTRIBUTED) {
    free(c->dsrc);
    c->dsrc = dalloc((size_t)np);
    memcpy(c->dsrc, params, sizeof(double) * (size_t)np);
    c->ndsrc = np;
    return LEE_OK;
  }
  for (int i = 0; i < 7 && i < np; ++i) c->src[i] = params[i];
  return LEE_OK;
}

int orc_set_block_source(orc_ctx *c, int b, int kind, const double *params, int np) {
  if (b < 0 || b >= c->nblk) return fail(c, LEE_ERR_ARG, "block index");
  if (kind == LEE_SOURCE_NONE) {
    c->bsrc_mode[b] = 2;
    return LEE_OK;
  }
  if (kind != LEE_SOURCE_MONOPOLE || np != 7) return fail(c, LEE_ERR_ARG, "monopole takes 7 params");
  c->bsrc_mode[b] = 1;
  for (int i = 0; i < 7; ++i) c->bsrc[b][i] = params[i];
  if (c->src_kind == LEE_SOURCE_NONE) c->src_kind = LEE_SOURCE_MONOPOLE;
  return LEE_OK;
}

/* Blocks advance in lockstep with one clock here, so every dt must be the same. */
int orc_advance_blocks(orc_ctx *c, int nsteps, const double *dt) {
  for (int b = 1; b < c->nblk; ++b)
    if (dt[b] != dt[0]) return fail(c, LEE_ERR_UNSUPPORTED, "the oracle advances blocks with one time step");
  return orc_advance(c, nsteps, dt[0]);
}

/* The distributed source's lattice weights and trilinear prolongation (the same arithmetic
 * as the CUDA library's host setup): node (p,q,r) at grid index (o + p h) per direction. */
static void lattice_weights(double i, double o, double h, int cn, int *p0, double *f) {
  double u = (i - o) / h;
  int q = (int)floor(u);
  if (q > cn - 2) q = cn - 2;
  if (q < 0) q = 0;
  *p0 = q;
  *f = u - q;
}

static void prolong_distributed(orc_ctx *c, blk_t *bk) {
  const double *p = c->dsrc, *A = c->dsrc + 11;
  int dim = c->cfg.num_dim, cx = (int)p[2], cy = (int)p[3];
  int n[3] = {bk->nx, bk->ny, bk->nz}, lo[3], hi[3];
  c->dsrc_g = dalloc((size_t)bk->N);
  for (int d = 0; d < 3; ++d) {
    if (d >= dim) { lo[d] = hi[d] = 0; continue; }
    lo[d] = (int)ceil(p[5 + d]);
    if (lo[d] < 0) lo[d] = 0;
    hi[d] = (int)floor(p[5 + d] + ((int)p[2 + d] - 1) * p[8 + d]);
    if (hi[d] > n[d] - 1) hi[d] = n[d] - 1;
  }
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[0]; i <= hi[0]; ++i) {
        int q[3] = {0, 0, 0};
        double f[3] = {0.0, 0.0, 0.0};
        lattice_weights(i, p[5], p[8], cx, &q[0], &f[0]);
        lattice_weights(j, p[6], p[9], cy, &q[1], &f[1]);
        if (dim == 3) lattice_weights(k, p[7], p[10], (int)p[4], &q[2], &f[2]);
        double sum = 0.0;
        for (int c2 = 0; c2 < (dim == 3 ? 2 : 1); ++c2)
          for (int c1 = 0; c1 < 2; ++c1)
            for (int c0 = 0; c0 < 2; ++c0) {
              double w = (c0 ? f[0] : 1.0 - f[0]) * (c1 ? f[1] : 1.0 - f[1]) *
                         (dim == 3 ? (c2 ? f[2] : 1.0 - f[2]) : 1.0);
              sum += w * A[(q[0] + c0) + (size_t)cx * ((q[1] + c1) + (size_t)cy * (q[2] + c2))];
            }
        c->dsrc_g[i + (size_t)bk->nx * (j + (size_t)bk->ny * k)] = sum;
      }
}

/* overset::initialize_overset (src/overset/overset.cpp:56-84): the maps of the
 * Overture file (src/io/overture.cpp:473-680), weights normalised as initialize_donor
 * does (:516-526), then holes BLANKED (:683-751) and receivers INTERPOLATED (:755-790). */
int orc_set_overset(orc_ctx *c, int n, const int *recv_block, const int *recv_ijk, const int *donor_block,
                    const int *donor_ijk, const int width[3], const double *weights, int num_holes,
                    const int *hole_block, const int *hole_ijk) {
  if (c->prepared) return fail(c, LEE_ERR_STATE, "set_overset after prepare");
  if (n < 0 || num_holes < 0) return fail(c, LEE_ERR_ARG, "negative count");
  int W = width[0] * width[1] * width[2];
  ovs_t *o = &c->ovs;
  free(o->rb); free(o->db); free(o->rl); free(o->dl); free(o->wt); free(o->buf);
  memset(o, 0, sizeof *o);
  o->rb = (int *)malloc(sizeof(int) * (size_t)(n ? n : 1));
  o->db = (int *)malloc(sizeof(int) * (size_t)(n ? n : 1));
  o->rl = (long long *)malloc(sizeof(long long) * (size_t)(n ? n : 1));
  o->dl = (long long *)malloc(sizeof(long long) * (size_t)(n ? n : 1));
  o->wt = dalloc((size_t)n * (size_t)W);
  o->buf = dalloc((size_t)n * MAXV);
  for (int d = 0; d < 3; ++d) o->w[d] = width[d];
  o->W = W;
  for (int q = 0; q < num_holes; ++q) {
    int b = hole_block[q];
    if (b < 0 || b >= c->nblk || !c->blk[b].set) return fail(c, LEE_ERR_ARG, "hole block");
    blk_t *bk = &c->blk[b];
    const int *ijk = hole_ijk + 3 * q;
    if (ijk[0] < 0 || ijk[0] >= bk->nx || ijk[1] < 0 || ijk[1] >= bk->ny || ijk[2] < 0 || ijk[2] >= bk->nz)
      return fail(c, LEE_ERR_ARG, "hole outside block");
    if (!bk->iblank) bk->iblank = (int *)calloc((size_t)bk->N, sizeof(int));
    bk->iblank[ijk[0] + bk->nx * (ijk[1] + bk->ny * ijk[2])] = BLANKED;
  }
  for (int r = 0; r < n; ++r) {
    int rb = recv_block[r], db = donor_block[r];
    if (rb < 0 || rb >= c->nblk || db < 0 || db >= c->nblk || !c->blk[rb].set || !c->blk[db].set)
      return fail(c, LEE_ERR_ARG, "receiver or donor block");
    blk_t *rk = &c->blk[rb], *dk = &c->blk[db];
    const int *ri = recv_ijk + 3 * r, *di = donor_ijk + 3 * r;
    int dn[3] = {dk->nx, dk->ny, dk->nz}, rn[3] = {rk->nx, rk->ny, rk->nz};
    for (int d = 0; d < 3; ++d) {
      if (ri[d] < 0 || ri[d] >= rn[d]) return fail(c, LEE_ERR_ARG, "receiver outside block");
      if (di[d] < 0 || di[d] + width[d] - 1 >= dn[d]) return fail(c, LEE_ERR_ARG, "donor stencil outside block");
    }
    o->rb[r] = rb;
    o->db[r] = db;
    o->rl[r] = ri[0] + (long long)rk->nx * (ri[1] + (long long)rk->ny * ri[2]);
    o->dl[r] = di[0] + (long long)dk->nx * (di[1] + (long long)dk->ny * di[2]);
    double sum = 0.0;
    for (int q = 0; q < W; ++q) sum += weights[(size_t)r * W + q];
    sum = 1.0 / sum;
    for (int q = 0; q < W; ++q) o->wt[(size_t)r * W + q] = weights[(size_t)r * W + q] * sum;
  }
  for (int r = 0; r < n; ++r) {
    blk_t *rk = &c->blk[o->rb[r]];
    if (!rk->iblank) rk->iblank = (int *)calloc((size_t)rk->N, sizeof(int));
    rk->iblank[o->rl[r]] = INTERPOLATED;
  }
  o->n = n;
  return LEE_OK;
}

/* read_overset_at_headrank (src/io/overture.cpp:473-680), then orc_set_overset. */
int orc_read_overset_file(orc_ctx *c, const char *path, int order_accuracy) {
  FILE *f = fopen(path, "rb");
  if (!f) return fail(c, LEE_ERR_ARG, "cannot open %s", path);
  int rc = LEE_OK, nd = 0, nb = 0, R = 0, H = 0;
  int *cnt = NULL, *rb = NULL, *rijk = NULL, *db = NULL, *dijk = NULL, *hc = NULL, *hb = NULL, *hijk = NULL;
  double *wt = NULL;
  int width[3] = {1, 1, 1};
#define RD(p, sz, n) do { if (fread((p), (sz), (size_t)(n), f) != (size_t)(n)) { rc = fail(c, LEE_ERR_ARG, "short overset file"); goto done; } } while (0)
  RD(&nd, 4, 1);
  RD(&nb, 4, 1);
  if (nd != c->cfg.num_dim || nb != c->nblk) { rc = fail(c, LEE_ERR_ARG, "overset file dimension/blocks"); goto done; }
  cnt = (int *)calloc((size_t)nb, sizeof(int));
  for (int b = 0; b < nb; ++b) {
    int np;
    RD(&np, 4, 1);
    if (np != c->blk[b].N) { rc = fail(c, LEE_ERR_ARG, "overset file points of block %d", b); goto done; }
  }
  RD(cnt, 4, nb);
  for (int b = 0; b < nb; ++b) R += cnt[b];
  rb = (int *)calloc((size_t)R + 1, sizeof(int));
  db = (int *)calloc((size_t)R + 1, sizeof(int));
  rijk = (int *)calloc(3 * (size_t)R + 3, sizeof(int));
  dijk = (int *)calloc(3 * (size_t)R + 3, sizeof(int));
  RD(rb, 4, R);
  for (int r = 0; r < R; ++r) RD(rijk + 3 * r, 4, nd);
  RD(db, 4, R);
  for (int r = 0; r < R; ++r) RD(dijk + 3 * r, 4, nd);
  {
    int base = 0;
    for (int b = 0; b < nb; ++b) {
      RD(width, 4, 3);
      for (int d = 0; d < nd; ++d)
        if (width[d] - 1 != order_accuracy) { rc = fail(c, LEE_ERR_ARG, "stencil width vs order"); goto done; }
      int W = width[0] * width[1] * width[2];
      if (!wt) wt = dalloc((size_t)R * W + 1);
      RD(wt + (size_t)base * W, 8, (size_t)cnt[b] * W);
      base += cnt[b];
    }
  }
  hc = (int *)calloc((size_t)nb, sizeof(int));
  RD(hc, 4, nb);
  for (int b = 0; b < nb; ++b) H += hc[b];
  hb = (int *)calloc((size_t)H + 1, sizeof(int));
  hijk = (int *)calloc(3 * (size_t)H + 3, sizeof(int));
  RD(hijk, 4, 3 * (size_t)H);
  {
    int q = 0;
    for (int b = 0; b < nb; ++b)
      for (int h = 0; h < hc[b]; ++h) hb[q++] = b;
  }
  rc = orc_set_overset(c, R, rb, rijk, db, dijk, width, wt, H, hb, hijk);
#undef RD
done:
  fclose(f);
  free(cnt); free(rb); free(rijk); free(db); free(dijk); free(hc); free(hb); free(hijk); free(wt);
  return rc;
}

int orc_get_overset(orc_ctx *c, int *recv_block, long long *recv_l0, int *donor_block, long long *donor_l0,
                    double *weights) {
  ovs_t *o = &c->ovs;
  for (int r = 0; r < o->n; ++r) {
    if (recv_block) recv_block[r] = o->rb[r];
    if (recv_l0) recv_l0[r] = o->rl[r];
    if (donor_block) donor_block[r] = o->db[r];
    if (donor_l0) donor_l0[r] = o->dl[r];
  }
  if (weights) memcpy(weights, o->wt, sizeof(double) * (size_t)o->n * (size_t)o->W);
  return LEE_OK;
}

int orc_prepare(orc_ctx *c) {
  for (int b = 0; b < c->nblk; ++b)
    for (int zi = 0; zi < c->blk[b].nbnd; ++zi) {
      int k = c->blk[b].bnd[zi].kind;
      if ((k == LEE_BC_DIRICHLET_HARMONICWAVE || k == LEE_SPONGE_FREUND_HARMONICWAVE) && c->wave_type == LEE_WAVE_NONE)
        return fail(c, LEE_ERR_STATE, "a harmonic-wave boundary needs a harmonic wave");
    }
  for (int b = 0; b < c->nblk; ++b) {
    blk_t *bk = &c->blk[b];
    if (!bk->set) return fail(c, LEE_ERR_STATE, "block %d not set", b);
    int rc = compute_metrics(c, bk);
    if (rc) return rc;
    for (int zi = 0; zi < bk->nbnd; ++zi)
      if ((bk->bnd[zi].kind == LEE_SPONGE_FREUND_AMBIENT || bk->bnd[zi].kind == LEE_SPONGE_FREUND_HARMONICWAVE) &&
          !bk->bnd[zi].sigma)
        compute_sigma(c, bk, &bk->bnd[zi]);
    /* mean gradients: spatial::precompute_something (:2250-2271), with hole closures */
    int nd = c->cfg.num_dim;
    double *work = dalloc((size_t)bk->N), *sum = dalloc((size_t)bk->N);
    for (int v = 0; v < c->nv; ++v)
      for (int j = 0; j < nd; ++j) {
        bk->grad[v * nd + j] = dalloc((size_t)bk->N);
        rc = d_x(c, bk, bk->mean[v], bk->grad[v * nd + j], j, work, sum);
        if (rc) { free(work); free(sum); return rc; }
      }
    free(work);
    free(sum);
    compute_aux(c, bk, bk->sol);
    if (c->src_kind == LEE_SOURCE_DISTRIBUTED && b == (int)c->dsrc[0]) prolong_distributed(c, bk);
  }
  c->prepared = 1;
  return LEE_OK;
}

int orc_upload_state(orc_ctx *c, int b, const double *const sol[5], int step, double time) {
  if (b < 0 || b >= c->nblk || !c->blk[b].set) return fail(c, LEE_ERR_STATE, "set_block first");
  blk_t *bk = &c->blk[b];
  for (int q = 0; q < 5; ++q) memcpy(bk->sol[q], sol[q], sizeof(double) * (size_t)bk->N);
  c->step = step;
  c->time = time;
  if (c->prepared) compute_aux(c, bk, bk->sol);
  return LEE_OK;
}

int orc_download_state(orc_ctx *c, int b, double *const sol[5], int *step, double *time) {
  if (b < 0 || b >= c->nblk || !c->blk[b].set) return fail(c, LEE_ERR_STATE, "set_block first");
  blk_t *bk = &c->blk[b];
  for (int q = 0; q < 5; ++q) memcpy(sol[q], bk->sol[q], sizeof(double) * (size_t)bk->N);
  if (step) *step = c->step;
  if (time) *time = c->time;
  return LEE_OK;
}

/* Passive scalars: n slots Z_k' after p' (PHYSICAL_MODEL = LEE_SCALAR, NUMBER_SCALAR = n;
 * src/core/input.cpp:113-119, :768-773), before any block is set. */
int orc_set_scalars(orc_ctx *c, int n) {
  if (n < 0 || n > MAXSC) return fail(c, LEE_ERR_ARG, "0 <= n <= %d scalars", MAXSC);
  for (int b = 0; b < c->nblk; ++b)
    if (c->blk[b].set) return fail(c, LEE_ERR_STATE, "lee_set_scalars before lee_set_block");
  c->nsc = n;
  c->nv = 5 + n;
  return LEE_OK;
}

int orc_set_mean_scalars(orc_ctx *c, int b, const double *const *zbar) {
  if (b < 0 || b >= c->nblk || !c->blk[b].set) return fail(c, LEE_ERR_STATE, "set_block first");
  if (!c->nsc || !zbar) return fail(c, LEE_ERR_ARG, "no scalars");
  for (int k = 0; k < c->nsc; ++k) memcpy(c->blk[b].mean[5 + k], zbar[k], sizeof(double) * (size_t)c->blk[b].N);
  return LEE_OK;
}

int orc_upload_scalars(orc_ctx *c, int b, const double *const *z) {
  if (b < 0 || b >= c->nblk || !c->blk[b].set) return fail(c, LEE_ERR_STATE, "set_block first");
  if (!c->nsc || !z) return fail(c, LEE_ERR_ARG, "no scalars");
  for (int k = 0; k < c->nsc; ++k) memcpy(c->blk[b].sol[5 + k], z[k], sizeof(double) * (size_t)c->blk[b].N);
  return LEE_OK;
}

int orc_download_scalars(orc_ctx *c, int b, double *const *z) {
  if (b < 0 || b >= c->nblk || !c->blk[b].set) return fail(c, LEE_ERR_STATE, "set_block first");
  if (!c->nsc || !z) return fail(c, LEE_ERR_ARG, "no scalars");
  for (int k = 0; k < c->nsc; ++k) memcpy(z[k], c->blk[b].sol[5 + k], sizeof(double) * (size_t)c->blk[b].N);
  return LEE_OK;
}

/* temporal::compute_CFL (src/solver/temporal_discretization.cpp:397-450) at time step dt;
 * orc_compute_dt applies it at the reference's dummy initial dt of 1e-6
 * (src/core/input.cpp:131) with the FIX_CFL rescale of solver::solve (src/solver/solver.cpp:58-64). */
static double cfl_at(orc_ctx *c, double dt) {
  int nd = c->cfg.num_dim;
  double cmax = -1e99, gm1 = c->cfg.gamma - 1.0;
  for (int b = 0; b < c->nblk; ++b) {
    blk_t *bk = &c->blk[b];
    for (int p = 0; p < bk->N; ++p) {
      if (bk->iblank && bk->iblank[p] != NOTBLANKED) continue;
      double vcart[3] = {bk->mean[1][p], bk->mean[2][p], bk->mean[3][p]}, vc[3];
      for (int q = nd; q < 3; ++q) vcart[q] = 0.0;
      for (int l = 0; l < nd; ++l) {
        vc[l] = 0.0;
        for (int q = 0; q < nd; ++q) vc[l] += bk->met[l * 3 + q][p] * vcart[q];
      }
      double cfl = 0.0;
      for (int l = 0; l < nd; ++l)
        for (int q = 0; q < nd; ++q) cfl += abs((int)(vc[l] * bk->met[l * 3 + q][p]));
      double fac = 0.0;
      for (int l = 0; l < nd; ++l)
        for (int q = 0; q < nd; ++q) fac += bk->met[l * 3 + q][p] * bk->met[l * 3 + q][p];
      double sos = sqrt(gm1 * bk->aux[3][p]);
      cfl += sos * sqrt(fac);
      cfl *= dt * bk->jac[p];
      if (cfl > cmax) cmax = cfl;
    }
  }
  return cmax;
}

int orc_compute_dt(orc_ctx *c, double cfl_target, double *dt_out) {
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "prepare first");
  double dt = 1e-6;
  double ratio = cfl_target / cfl_at(c, dt);
  dt *= ratio;
  *dt_out = dt;
  return LEE_OK;
}

int orc_compute_cfl(orc_ctx *c, double dt, double *cfl) {
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "prepare first");
  if (!(dt > 0.0)) return fail(c, LEE_ERR_ARG, "dt must be positive");
  *cfl = cfl_at(c, dt);
  return LEE_OK;
}

/* ReportSolution::minmax (src/io/io.cpp:440-499) over every point of every block. */
int orc_state_minmax(orc_ctx *c, double *mn, double *mx) {
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "prepare first");
  for (int q = 0; q < 5; ++q) {
    mn[q] = 1e300;
    mx[q] = -1e300;
    for (int b = 0; b < c->nblk; ++b)
      for (int p = 0; p < c->blk[b].N; ++p) {
        double v = c->blk[b].sol[q][p];
        mn[q] = v < mn[q] ? v : mn[q];
        mx[q] = v > mx[q] ? v : mx[q];
      }
  }
  return LEE_OK;
}

int orc_compute_dt_blocks(orc_ctx *c, double cfl_target, double *dt_out) {
  int n = c->nblk;
  for (int b = 0; b < n; ++b) {
    c->nblk = 1;
    blk_t save = c->blk[0];
    c->blk[0] = c->blk[b];
    int rc = orc_compute_dt(c, cfl_target, &dt_out[b]);
    c->blk[0] = save;
    c->nblk = n;
    if (rc) return rc;
  }
  return LEE_OK;
}

/* RungeKutta::integrate (src/solver/temporal_discretization.cpp:177-252) and
 * temporal::time_advance (:334-374) for every block. Blocks advance in lockstep
 * stage by stage, as the reference's ranks do between barriers. */
int orc_advance(orc_ctx *c, int nsteps, double dt) {
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "prepare first");
  double bi[4], ci[4], aij[4];
  int ns;
  if (c->cfg.rk_scheme == LEE_RK4) {
    ns = 4;
    bi[0] = 1.0 / 6.0; bi[1] = 1.0 / 3.0; bi[2] = 1.0 / 3.0; bi[3] = 1.0 / 6.0;
    ci[0] = 0.0; ci[1] = 1.0 / 2.0; ci[2] = 1.0 / 2.0; ci[3] = 1.0;
    aij[0] = 1.0 / 2.0; aij[1] = 1.0 / 2.0; aij[2] = 1.0; aij[3] = 0.0;
  } else if (c->cfg.rk_scheme == LEE_RK2) {
    ns = 2;
    bi[0] = 1.0 / 2.0; bi[1] = 1.0 / 2.0;
    ci[0] = 0.0; ci[1] = 1.0;
    aij[0] = 1.0; aij[1] = 0.0;
  } else {
    return fail(c, LEE_ERR_UNSUPPORTED, "rk scheme");
  }
  int nb = c->nblk;
  int nv = c->nv;
  double *yn[MAXB][MAXV], *ynext[MAXB][MAXV], *zi[MAXB][MAXV], *rhs[MAXB][MAXV];
  for (int b = 0; b < nb; ++b)
    for (int v = 0; v < nv; ++v) {
      size_t N = (size_t)c->blk[b].N;
      yn[b][v] = dalloc(N); ynext[b][v] = dalloc(N); zi[b][v] = dalloc(N); rhs[b][v] = dalloc(N);
    }
  int rc = 0;
  for (int it = 0; it < nsteps && !rc; ++it) {
    c->time += dt; /* solver::solve increments the time before time_advance (src/solver/solver.cpp:72) */
    c->step += 1;
    double tn = c->time, h = dt;
    for (int b = 0; b < nb; ++b)
      for (int v = 0; v < nv; ++v) {
        size_t N = (size_t)c->blk[b].N;
        memcpy(yn[b][v], c->blk[b].sol[v], N * sizeof(double));
        memcpy(ynext[b][v], yn[b][v], N * sizeof(double));
        memcpy(zi[b][v], yn[b][v], N * sizeof(double));
      }
    for (int s = 0; s < ns && !rc; ++s) {
      for (int b = 0; b < nb && !rc; ++b) {
        blk_t *bk = &c->blk[b];
        rc = rhs_block(c, bk, zi[b], rhs[b], tn + ci[s] * h);
        PAR_FOR
        for (int p = 0; p < bk->N; ++p) {
          if (!(bk->iblank && bk->iblank[p] == BLANKED)) {
            for (int v = 0; v < nv; ++v) {
              rhs[b][v][p] *= h;
              ynext[b][v][p] += bi[s] * rhs[b][v][p];
              if (s < ns - 1) zi[b][v][p] = yn[b][v][p] + aij[s] * rhs[b][v][p];
            }
          } else {
            for (int v = 0; v < nv; ++v) {
              rhs[b][v][p] = 0.0;
              ynext[b][v][p] = 0.0;
              zi[b][v][p] = 0.0;
            }
          }
        }
      }
      double **tgts[MAXB];
      /* spatial::update_boundary (:2162-2187) at tn + c_{min(i+1, last)} h
       * (src/solver/temporal_discretization.cpp:232-244), then aux */
      int sb = (s + 1 < ns - 1) ? s + 1 : ns - 1;
      for (int b = 0; b < nb; ++b) {
        tgts[b] = (s < ns - 1) ? zi[b] : ynext[b];
        apply_bc(c, &c->blk[b], tgts[b], tn + ci[sb] * h);
      }
      if (c->ovs.n > 0) interpolate(c, tgts);
      for (int b = 0; b < nb; ++b) compute_aux(c, &c->blk[b], (s < ns - 1) ? zi[b] : ynext[b]);
    }
    for (int b = 0; b < nb && !rc; ++b) {
      blk_t *bk = &c->blk[b];
      if (c->cfg.filter_scheme != LEE_FILTER_NONE) rc = filter_block(c, bk, ynext[b]);
      for (int p = 0; p < bk->N; ++p) /* temporal::iblank_correction (:380-393) */
        if (bk->iblank && bk->iblank[p] == BLANKED)
          for (int v = 0; v < nv; ++v) ynext[b][v][p] = 0.0;
      for (int v = 0; v < nv; ++v) memcpy(bk->sol[v], ynext[b][v], sizeof(double) * (size_t)bk->N);
    }
    /* the non-finite sentinel of lee_set_finite_check (the reference has none) */
    int last = it == nsteps - 1;
    if (!rc && c->finite_every >= 0 && (last || (c->finite_every > 0 && (it + 1) % c->finite_every == 0)))
      for (int b = 0; b < nb && !rc; ++b)
        for (int v = 0; v < nv && !rc; ++v)
          for (int p = 0; p < c->blk[b].N; ++p)
            if (!isfinite(c->blk[b].sol[v][p])) {
              rc = fail(c, LEE_ERR_NONFINITE, "the state holds a non-finite value after step %d", c->step);
              break;
            }
  }
  for (int b = 0; b < nb; ++b)
    for (int v = 0; v < nv; ++v) { free(yn[b][v]); free(ynext[b][v]); free(zi[b][v]); free(rhs[b][v]); }
  return rc;
}

int orc_eval_rhs(orc_ctx *c, int b, double time, double *const rhs[5]) {
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "prepare first");
  blk_t *bk = &c->blk[b];
  double *r[MAXV];
  for (int v = 0; v < 5; ++v) r[v] = rhs[v];
  for (int v = 5; v < c->nv; ++v) r[v] = dalloc((size_t)bk->N); /* the scalars' right-hand sides are dropped */
  int rc = rhs_block(c, bk, bk->sol, r, time);
  for (int v = 5; v < c->nv; ++v) free(r[v]);
  return rc;
}

int orc_apply_filter(orc_ctx *c) {
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "prepare first");
  if (c->cfg.filter_scheme == LEE_FILTER_NONE) return LEE_OK;
  for (int b = 0; b < c->nblk; ++b) {
    int rc = filter_block(c, &c->blk[b], c->blk[b].sol);
    if (rc) return rc;
  }
  return LEE_OK;
}

int orc_get_setup(orc_ctx *c, int b, int what, double *out) {
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "prepare first");
  blk_t *bk = &c->blk[b];
  size_t N = (size_t)bk->N;
  int nd = c->cfg.num_dim;
  if (what == LEE_SETUP_METRICS) {
    for (int q = 0; q < 9; ++q) memcpy(out + q * N, bk->met[q], N * sizeof(double));
  } else if (what == LEE_SETUP_JACOBIAN) {
    memcpy(out, bk->jac, N * sizeof(double));
  } else if (what == LEE_SETUP_MEAN_GRADIENT) {
    for (int q = 0; q < 5 * nd; ++q) memcpy(out + q * N, bk->grad[q], N * sizeof(double));
  } else if (what == LEE_SETUP_SPONGE) {
    memset(out, 0, N * sizeof(double));
    for (int zi = 0; zi < bk->nbnd; ++zi) {
      bnd_t *z = &bk->bnd[zi];
      if (z->kind != LEE_SPONGE_FREUND_AMBIENT && z->kind != LEE_SPONGE_FREUND_HARMONICWAVE) continue;
      int bn0 = z->hi[0] - z->lo[0] + 1, bn1 = z->hi[1] - z->lo[1] + 1;
      for (int k = z->lo[2]; k <= z->hi[2]; ++k)
        for (int j = z->lo[1]; j <= z->hi[1]; ++j)
          for (int i = z->lo[0]; i <= z->hi[0]; ++i)
            out[i + bk->nx * (j + bk->ny * k)] +=
                z->sigma[(i - z->lo[0]) + bn0 * ((j - z->lo[1]) + bn1 * (k - z->lo[2]))];
    }
  } else {
    return fail(c, LEE_ERR_ARG, "unknown setup selector");
  }
  return LEE_OK;
}

/* Sizes of the oracle context (the oracle has no device and no timers). */
int orc_get_info(orc_ctx *c, lee_info *info) {
  memset(info, 0, sizeof *info);
  for (int b = 0; b < c->nblk; ++b) info->points += c->blk[b].N;
  info->state_vars = c->cfg.num_dim + 2;
  info->bytes_per_value = 8;
  return LEE_OK;
}

int orc_set_timing(orc_ctx *c, int on) {
  (void)c;
  (void)on;
  return LEE_OK;
}

/* The microphone objective J = weight * sum_n sum_m p'_n(l_m)^2 (the same definition as the
 * CUDA library's), evaluated on the oracle's own steps. */
int orc_set_objective(orc_ctx *c, int b, int n, const long long *l, double weight) {
  if (b < 0 || b >= c->nblk || n < 1) return fail(c, LEE_ERR_ARG, "objective");
  free(c->mic);
  c->mic = (long long *)malloc(sizeof(long long) * (size_t)n);
  memcpy(c->mic, l, sizeof(long long) * (size_t)n);
  c->nmic = n;
  c->mic_block = b;
  c->mic_weight = weight;
  return LEE_OK;
}

int orc_eval_objective(orc_ctx *c, int nsteps, double dt, double *J) {
  double acc = 0.0;
  for (int n = 0; n < nsteps; ++n) {
    int rc = orc_advance(c, 1, dt);
    if (rc) return rc;
    for (int m = 0; m < c->nmic; ++m) {
      double p = c->blk[c->mic_block].sol[4][c->mic[m]];
      acc += p * p;
    }
  }
  *J = c->mic_weight * acc;
  return LEE_OK;
}

/* The adjoint is not restated on the CPU: it is checked against the CUDA forward map
 * (dot-product test) and against oracle objectives (finite differences). */
int orc_apply_adjoint(orc_ctx *c, int nsteps, double dt) {
  (void)nsteps; (void)dt;
  return fail(c, LEE_ERR_UNSUPPORTED, "the oracle has no adjoint");
}

int orc_adjoint_gradient(orc_ctx *c, int nsteps, double dt, int k, int recompute, double *J, double *grad,
                         long long *mism) {
  (void)nsteps; (void)dt; (void)k; (void)recompute; (void)J; (void)grad; (void)mism;
  return fail(c, LEE_ERR_UNSUPPORTED, "the oracle has no adjoint");
}

int orc_set_batch_shapes(orc_ctx *c, int stage_shape, int filter_shape) {
  (void)stage_shape; (void)filter_shape;
  return fail(c, LEE_ERR_STATE, "the oracle has no batched kernels");
}

int orc_set_batch_persistent(orc_ctx *c, int shape) {
  (void)shape;
  return fail(c, LEE_ERR_STATE, "the oracle has no batched kernels");
}

int orc_set_stage_kernel(orc_ctx *c, int kind) {
  (void)c;
  (void)kind;
  return LEE_OK; /* one stage path */
}

int orc_set_filter_kernel(orc_ctx *c, int kind) {
  (void)c;
  (void)kind;
  return LEE_OK; /* one filter path */
}

int orc_set_filter_form(orc_ctx *c, int form) {
  (void)c;
  (void)form;
  return LEE_OK; /* one filter path */
}

int orc_set_graphs(orc_ctx *c, int on) {
  (void)c; (void)on;
  return LEE_OK;
}

/* The oracle runs its blocks one after the other: both switches are accepted and change nothing. */
int orc_set_block_streams(orc_ctx *c, int on) {
  (void)c; (void)on;
  return LEE_OK;
}

int orc_set_increment_step(orc_ctx *c, int on) {
  (void)c; (void)on;
  return LEE_OK;
}

int orc_set_batching(orc_ctx *c, int on) {
  (void)c; (void)on;
  return LEE_OK;
}

int orc_set_finite_check(orc_ctx *c, int every) {
  if (every < -1) return fail(c, LEE_ERR_ARG, "finite-check interval %d", every);
  c->finite_every = every;
  return LEE_OK;
}

/* The oracle stages nothing and waits on nothing: the limit is accepted and has no effect. */
int orc_set_wait_limit(orc_ctx *c, double seconds) {
  if (!(seconds <= 10.0)) return fail(c, LEE_ERR_ARG, "wait limit %g s: at most 10 s", seconds);
  return LEE_OK;
}

int orc_get_stats(orc_ctx *c, lee_stats *st) {
  (void)c;
  memset(st, 0, sizeof *st);
  return LEE_OK;
}
