/*
 * lcs_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement, in plain C, of the LCS.jl time step (the reference is Julia
 * and cannot run in this environment).  It is the parity checker for the CUDA
 * library and the timed CPU baseline; nothing in the product links it.  Only
 * tests/, __graft_entry__.smoke() and bench.py (its CPU-baseline leg) load it.
 *
 * It implements the same C ABI (include/lcs_b200.h) so a test can drive both
 * libraries with identical calls.  Arithmetic follows the Julia source term by
 * term and in the same evaluation order (left-to-right folds, the same
 * constants), compiled with -ffp-contract=off, so every element-wise stage is
 * a bit-exact restatement.  Reductions (`sum`/`mean`) are sequential
 * column-major left folds, the order Julia's `mapfoldl` uses for a Cartesian
 * view; the reference's GPU path reduces in a tree, so the last bits of
 * means are not pinned by any reference artefact.
 *
 * Pinning: the reference's golden vectors (test/references/flows.jld2, particles.jld2) are git-LFS
 * stubs and its inputs come from Julia's Xoshiro stream, so the field stages
 * are "parity unpinned" against reference outputs.  What is pinned is listed
 * in tests/test_oracle_known_answers.py (box-mean exactness, kset/kcount,
 * enespe on a constant spectrum, sirdft vs masked inverse DFT, drag
 * coefficients, colouring masks, periodic halo invariant, particle wrap).
 *
 * Layout: haloed arrays (n+2h)^3, x fastest, logical index i in 1-h..n+h.
 */
#include "../include/lcs_b200.h"

#include <math.h>
#include <quadmath.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#else
#include <time.h>
static double omp_get_wtime(void) { /* the serial build's wall clock */
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
#endif

#define DOMAIN_LENGTH (2.0 * 3.14159265358979323846) /* src/LCS.jl:17 */
#define DOMAIN_ORIGIN 0.0                            /* src/LCS.jl:16 */
#define PI_F64 3.14159265358979323846                /* Float64(pi) */

typedef struct {
  int n[3];  /* interior cells per axis */
  int h;     /* halo */
  int s[3];  /* storage per axis = n + 2h */
} grid_t;

typedef struct {
  int64_t n;
  double* p[LCS_NPROP];
  int64_t* ids;
  int64_t *ci_hashes, *ci_starts, *ci_stops; /* the last cell index (makeindex.jl:29-67) */
  int64_t ci_H;
} species_t;

struct lcs_handle {
  lcs_config cfg;
  grid_t g;
  size_t hsz, isz;                 /* haloed / interior element counts */
  double *U, *V, *W, *U2, *V2, *W2, *P;
  double *dU, *dV, *dW;            /* interior */
  double* J[6];                    /* Jx1 Jy1 Jz1 Jx3 Jy3 Jz3 scratches (rhs.jl:36) */
  double* Div2;                    /* scratches[1] (hsmac.jl:64) */
  double* S1;                      /* U2 / Power scratch (lf.jl:20, rcf.jl:11) */
  double* Ui[3];                   /* U_interp.. (flows/timestep.jl:31) */
  species_t sp[LCS_MAX_SPECIES];
  int64_t step;
  double t;
  int32_t async_n;                 /* steps of a pending lcs_step_begin (run at begin) */
  int32_t sort_interval, sort_ratio; /* lcs_set_particle_sort */
  int32_t async_rc;
  lcs_log* async_logs;
  char err[512];
};

static _Thread_local char g_err[512]; /* per thread, as in the CUDA library */

static int fail(lcs_handle* h, int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(h ? h->err : g_err, 512, fmt, ap);
  va_end(ap);
  return code;
}

/* ---- indexing (lib/offsets/src/Offsets.jl:70-73) ---------------------- */
static inline size_t IX(const grid_t* g, int i, int j, int k) {
  return ((size_t)(k + g->h - 1) * g->s[1] + (size_t)(j + g->h - 1)) * g->s[0] + (size_t)(i + g->h - 1);
}
static inline size_t IN(const grid_t* g, int i, int j, int k) {
  return ((size_t)(k - 1) * g->n[1] + (size_t)(j - 1)) * g->n[0] + (size_t)(i - 1);
}

static double spacing(const grid_t* g, int a) { return DOMAIN_LENGTH / g->n[a]; } /* src/config.jl:89 */
/* Base.max / Base.min of Julia on floats: NaN if either operand is NaN, and
 * max(-0.0, 0.0) = 0.0, min(-0.0, 0.0) = -0.0 (C's fmax/fmin drop a NaN).
 * `maximum`, `minimum` and `min(cands...)` reduce with them. */
static inline double jl_max(double a, double b) {
  if (isnan(a)) return a;
  if (isnan(b)) return b;
  return (a > b || (a == b && !signbit(a))) ? a : b;
}
static inline double jl_min(double a, double b) {
  if (isnan(a)) return a;
  if (isnan(b)) return b;
  return (a < b || (a == b && signbit(a))) ? a : b;
}
static double Re_of(const lcs_config* c) { return c->U0 * c->L0 / c->NU; }      /* flows/config.jl:18 */

/* ---- stencil primitives (src/diff.jl:1-39) ----------------------------- */
static inline double interp_o2_at_half(double a, double b) { return (1.0 / 2.0) * (a + b); }
static inline double interp_o4_at_half(double a, double b, double c, double d) {
  return (1.0 / 16.0) * (-a + 9.0 * b + 9.0 * c - d);
}
static inline double diff1_o2_at_half(double a, double b) { return (-a + b); }
static inline double diff2_o4_at_node(double a, double b, double c, double d, double e) {
  return (1.0 / 12.0) * (-a + 16.0 * b - 30.0 * c + 16.0 * d - e);
}
static inline double sum_flux_o4(double j1a, double j1b, double j3a, double j3b) {
  return (9.0 / 8.0) * (-j1a + j1b) - ((1.0 / 8.0) * (1.0 / 3.0)) * (-j3a + j3b);
}

/* ---- single-process halo fill (lib/topologies/src/halo.jl:138-159, 298-347) */
static int wrap1(int i, int n) { /* mod1 onto 1..n */
  int r = (i - 1) % n;
  if (r < 0) r += n;
  return r + 1;
}
static void synchalo(const grid_t* g, double* A, int r, int full) {
  const int nx = g->n[0], ny = g->n[1], nz = g->n[2];
#pragma omp parallel for schedule(static)
  for (int k = 1 - r; k <= nz + r; k++)
    for (int j = 1 - r; j <= ny + r; j++)
      for (int i = 1 - r; i <= nx + r; i++) {
        int ox = (i < 1 || i > nx), oy = (j < 1 || j > ny), oz = (k < 1 || k > nz);
        int nout = ox + oy + oz;
        if (nout == 0) continue;
        if (!full && nout != 1) continue; /* FaceHalo: DIRECTIONS[1:6] only */
        A[IX(g, i, j, k)] = A[IX(g, wrap1(i, nx), wrap1(j, ny), wrap1(k, nz))];
      }
}

/* ---- sequential reductions (Topologies.allmean etc., operators.jl:1-99) -- */
typedef struct { int lo[3], hi[3]; } box_t;
static box_t box3(int lo, int hiplus, const grid_t* g) { /* lo:(n+hiplus) per axis */
  box_t b;
  for (int a = 0; a < 3; a++) { b.lo[a] = lo; b.hi[a] = g->n[a] + hiplus; }
  return b;
}
static double box_count(box_t b) {
  return (double)((int64_t)(b.hi[0] - b.lo[0] + 1) * (b.hi[1] - b.lo[1] + 1) * (b.hi[2] - b.lo[2] + 1));
}
static double mean_haloed(const grid_t* g, const double* A, box_t b) {
  double s = 0.0;
  int first = 1;
  for (int k = b.lo[2]; k <= b.hi[2]; k++)
    for (int j = b.lo[1]; j <= b.hi[1]; j++)
      for (int i = b.lo[0]; i <= b.hi[0]; i++) {
        double v = A[IX(g, i, j, k)];
        if (first) { s = v; first = 0; } else s = s + v;
      }
  return s / box_count(b);
}

/* ---- rhs (src/flows/rhs.jl:20-252) ------------------------------------- */
static void rhs_component(lcs_handle* h, int comp, const double* U, const double* V, const double* W, double* dUdt) {
  const grid_t* g = &h->g;
  const double dxi = 1.0 / spacing(g, 0), dyi = 1.0 / spacing(g, 1), dzi = 1.0 / spacing(g, 2);
  const double Rei = 1.0 / Re_of(&h->cfg);
  const double* P = h->P;
  double **J = h->J;
  const double* A = comp == 0 ? U : comp == 1 ? V : W; /* the transported component */
  const int nx = g->n[0], ny = g->n[1], nz = g->n[2];
  const size_t sx = 1, sy = (size_t)g->s[0], sz = (size_t)g->s[0] * g->s[1];
  const size_t sc = comp == 0 ? sx : comp == 1 ? sy : sz; /* stride along the component axis */
  const double dci = comp == 0 ? dxi : comp == 1 ? dyi : dzi;
  /* pass 1 over domain1 = -1:n+1 (rhs.jl:65-100) */
#pragma omp parallel for schedule(static)
  for (int k = -1; k <= nz + 1; k++)
    for (int j = -1; j <= ny + 1; j++)
      for (int i = -1; i <= nx + 1; i++) {
        size_t c = IX(g, i, j, k);
        double uc = interp_o4_at_half(U[c - sc], U[c], U[c + sc], U[c + 2 * sc]);
        double vc = interp_o4_at_half(V[c - sc], V[c], V[c + sc], V[c + 2 * sc]);
        double wc = interp_o4_at_half(W[c - sc], W[c], W[c + sc], W[c + 2 * sc]);
        double ax1 = interp_o2_at_half(A[c], A[c + sx]);
        double ay1 = interp_o2_at_half(A[c], A[c + sy]);
        double az1 = interp_o2_at_half(A[c], A[c + sz]);
        double ax3 = interp_o2_at_half(A[c - sx], A[c + 2 * sx]);
        double ay3 = interp_o2_at_half(A[c - sy], A[c + 2 * sy]);
        double az3 = interp_o2_at_half(A[c - sz], A[c + 2 * sz]);
        if (i >= 1 && i <= nx && j >= 1 && j <= ny && k >= 1 && k <= nz) {
          double diff = (dxi * dxi * diff2_o4_at_node(A[c - 2 * sx], A[c - sx], A[c], A[c + sx], A[c + 2 * sx]) +
                         dyi * dyi * diff2_o4_at_node(A[c - 2 * sy], A[c - sy], A[c], A[c + sy], A[c + 2 * sy]) +
                         dzi * dzi * diff2_o4_at_node(A[c - 2 * sz], A[c - sz], A[c], A[c + sz], A[c + 2 * sz])) *
                        Rei;
          double pres = dci * diff1_o2_at_half(P[c], P[c + sc]);
          dUdt[IN(g, i, j, k)] = diff - pres;
        }
        J[0][c] = uc * ax1;
        J[1][c] = vc * ay1;
        J[2][c] = wc * az1;
        J[3][c] = uc * ax3;
        J[4][c] = vc * ay3;
        J[5][c] = wc * az3;
      }
  /* pass 2 over domain2 = 1:n (rhs.jl:102-111) */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        size_t c = IX(g, i, j, k);
        double advect = dxi * sum_flux_o4(J[0][c - sx], J[0][c], J[3][c - 2 * sx], J[3][c + sx]) +
                        dyi * sum_flux_o4(J[1][c - sy], J[1][c], J[4][c - 2 * sy], J[4][c + sy]) +
                        dzi * sum_flux_o4(J[2][c - sz], J[2][c], J[5][c - 2 * sz], J[5][c + sz]);
        size_t o = IN(g, i, j, k);
        dUdt[o] = dUdt[o] - advect;
      }
}

static void get_Us(lcs_handle* h, int set, double** U, double** V, double** W) {
  if (set == 0) { *U = h->U; *V = h->V; *W = h->W; }
  else { *U = h->U2; *V = h->V2; *W = h->W2; }
}

static void flow_rhs(lcs_handle* h, int stage) { /* Us_rhs: stage1 -> Us, stage2 -> Us2 (rhs.jl:1-2) */
  double *U, *V, *W;
  get_Us(h, stage == 1 ? 0 : 1, &U, &V, &W);
  rhs_component(h, 0, U, V, W, h->dU);
  rhs_component(h, 1, U, V, W, h->dV);
  rhs_component(h, 2, U, V, W, h->dW);
}

/* update! (src/flows/update.jl:1-54): stage1 Us2 = Us + dU*dt; stage2 Us = Us + dU*dt */
static void flow_update(lcs_handle* h, int stage, double dt) {
  const grid_t* g = &h->g;
  double *U, *V, *W, *U0, *V0, *W0;
  get_Us(h, stage == 1 ? 1 : 0, &U, &V, &W);
  get_Us(h, 0, &U0, &V0, &W0);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= g->n[2]; k++)
    for (int j = 1; j <= g->n[1]; j++)
      for (int i = 1; i <= g->n[0]; i++) {
        size_t o = IN(g, i, j, k), c = IX(g, i, j, k);
        double du = h->dU[o] * dt, dv = h->dV[o] * dt, dw = h->dW[o] * dt;
        double u = U0[c], v = V0[c], w = W0[c];
        U[c] = u + du;
        V[c] = v + dv;
        W[c] = w + dw;
      }
}

/* ---- HSMAC (src/flows/couples/hsmac.jl) -------------------------------- */
typedef struct {
  double *U, *V, *W, *P, *Div2;
  double dti, dxi, dyi, dzi, dl, omega;
} hsmac_t;

static inline void hsmac_cellwise(const grid_t* g, const hsmac_t* s, int i, int j, int k) { /* hsmac.jl:1-35 */
  const size_t sy = (size_t)g->s[0], sz = (size_t)g->s[0] * g->s[1];
  size_t c = IX(g, i, j, k);
  double dudx = s->dxi * diff1_o2_at_half(s->U[c - 1], s->U[c]);
  double dvdy = s->dyi * diff1_o2_at_half(s->V[c - sy], s->V[c]);
  double dwdz = s->dzi * diff1_o2_at_half(s->W[c - sz], s->W[c]);
  double div = dudx + dvdy + dwdz;
  double dp = -s->omega * div * s->dl;
  s->Div2[c] = div * div;
  s->P[c] = s->P[c] + dp * s->dti;
  s->U[c - 1] = s->U[c - 1] - dp * s->dxi;
  s->U[c] = s->U[c] + dp * s->dxi;
  s->V[c - sy] = s->V[c - sy] - dp * s->dyi;
  s->V[c] = s->V[c] + dp * s->dyi;
  s->W[c - sz] = s->W[c - sz] - dp * s->dzi;
  s->W[c] = s->W[c] + dp * s->dzi;
}

/* colour predicate of one cell (lib/parallel/src/foraxes.jl:82-107) */
static inline int in_color(int coloring, int i, int j, int k, int color) {
  int sum = i + j + k;
  if (coloring == LCS_COLORING_RED_BLACK) return (sum % 2) == color; /* Julia rem: negative odd sums match neither */
  return (sum & 1) == color;                                          /* RedBlackFast: true parity */
}

/* foraxes(backend, box; coloring) with f = hsmac_cellwise */
static void sweep_box(lcs_handle* h, const hsmac_t* s, box_t b) {
  const grid_t* g = &h->g;
  const int coloring = h->cfg.coloring;
  if (b.lo[0] > b.hi[0] || b.lo[1] > b.hi[1] || b.lo[2] > b.hi[2]) return;
  if (coloring == LCS_COLORING_NO) { /* sequential lexicographic order (foraxes.jl:16-18) */
    for (int k = b.lo[2]; k <= b.hi[2]; k++)
      for (int j = b.lo[1]; j <= b.hi[1]; j++)
        for (int i = b.lo[0]; i <= b.hi[0]; i++) hsmac_cellwise(g, s, i, j, k);
    return;
  }
  if (coloring == LCS_COLORING_RED_BLACK_BLOCK) { /* foraxes.jl:114-136 */
    const int bs = h->cfg.coloring_block;
    int nb[3];
    for (int a = 0; a < 3; a++) { int len = b.hi[a] - b.lo[a] + 1; nb[a] = (len + bs - 1) / bs; }
    for (int color = 0; color <= 1; color++) {
#pragma omp parallel for schedule(static)
      for (int bk = 1; bk <= nb[2]; bk++)
        for (int bj = 1; bj <= nb[1]; bj++)
          for (int bi = 1; bi <= nb[0]; bi++) {
            if ((bi + bj + bk) % 2 != color) continue;
            for (int lk = 1; lk <= bs; lk++)
              for (int lj = 1; lj <= bs; lj++)
                for (int li = 1; li <= bs; li++) {
                  int i = b.lo[0] + bs * (bi - 1) + li - 1;
                  int j = b.lo[1] + bs * (bj - 1) + lj - 1;
                  int k = b.lo[2] + bs * (bk - 1) + lk - 1;
                  if (i <= b.hi[0] && j <= b.hi[1] && k <= b.hi[2]) hsmac_cellwise(g, s, i, j, k);
                }
          }
    }
    return;
  }
  for (int color = 0; color <= 1; color++) {
#pragma omp parallel for schedule(static)
    for (int k = b.lo[2]; k <= b.hi[2]; k++)
      for (int j = b.lo[1]; j <= b.hi[1]; j++)
        for (int i = b.lo[0]; i <= b.hi[0]; i++)
          if (in_color(coloring, i, j, k, color)) hsmac_cellwise(g, s, i, j, k);
  }
}

/* Topologies.faces(domain, core) (lib/topologies/src/halo.jl:349-366) */
static void faces_of(box_t d, box_t c, box_t out[6]) {
  for (int f = 0; f < 6; f++) out[f] = d;
  out[0].hi[2] = c.lo[2] - 1;                           /* z- */
  out[1].lo[2] = c.hi[2] + 1;                           /* z+ */
  out[2].hi[1] = c.lo[1] - 1; out[2].lo[2] = c.lo[2]; out[2].hi[2] = c.hi[2]; /* y- */
  out[3].lo[1] = c.hi[1] + 1; out[3].lo[2] = c.lo[2]; out[3].hi[2] = c.hi[2]; /* y+ */
  out[4].hi[0] = c.lo[0] - 1; out[4].lo[1] = c.lo[1]; out[4].hi[1] = c.hi[1];
  out[4].lo[2] = c.lo[2]; out[4].hi[2] = c.hi[2];        /* x- */
  out[5].lo[0] = c.hi[0] + 1; out[5].lo[1] = c.lo[1]; out[5].hi[1] = c.hi[1];
  out[5].lo[2] = c.lo[2]; out[5].hi[2] = c.hi[2];        /* x+ */
}

static double residual(lcs_handle* h) { /* sqrt(allmean(Div2[1:n+1]^3)) (hsmac.jl:120,177) */
  return sqrt(mean_haloed(&h->g, h->Div2, box3(1, 1, &h->g)));
}

static int couple(lcs_handle* h, int stage, double dt, lcs_couple_log* log) {
  const grid_t* g = &h->g;
  const lcs_config* c = &h->cfg;
  hsmac_t s;
  double *U, *V, *W;
  get_Us(h, stage == 1 ? 1 : 0, &U, &V, &W); /* Us_couple (couple.jl:1-2) */
  s.U = U; s.V = V; s.W = W; s.P = h->P; s.Div2 = h->Div2;
  s.dxi = 1.0 / spacing(g, 0); s.dyi = 1.0 / spacing(g, 1); s.dzi = 1.0 / spacing(g, 2);
  s.dl = 1.0 / (2.0 * (s.dxi * s.dxi + s.dyi * s.dyi + s.dzi * s.dzi));
  s.omega = c->omega;
  s.dti = 1.0 / dt;
  double dxmin = spacing(g, 0);
  for (int a = 1; a < 3; a++) dxmin = fmin(dxmin, spacing(g, a));

  int itr = 0, sweeps = 0;
  double div = 0.0;
  box_t dom3 = box3(1, 1, g);
  if (c->time_blocking) { /* _couple_time_blocking! (hsmac.jl:131-201) */
    box_t d1 = box3(-1, 3, g), d2 = box3(0, 2, g), core = box3(2, 0, g);
    box_t doms[3] = {d1, d2, dom3};
    while (itr < c->itrmax) {
      if (!c->overlap) { synchalo(g, U, g->h, 1); synchalo(g, V, g->h, 1); synchalo(g, W, g->h, 1); }
      for (int d = 0; d < 3; d++) {
        if (c->overlap && d == 0) {
          synchalo(g, U, g->h, 1); synchalo(g, V, g->h, 1); synchalo(g, W, g->h, 1);
          sweep_box(h, &s, core);
          box_t f[6];
          faces_of(d1, core, f);
          for (int q = 0; q < 6; q++) sweep_box(h, &s, f[q]);
        } else {
          sweep_box(h, &s, doms[d]);
        }
        sweeps++;
        div = residual(h);
        if (!isfinite(div)) return fail(h, LCS_ENONFINITE, "HSMAC residual is not finite at itr %d", itr);
        if (div * dxmin < c->epsp && c->itrmin <= itr) goto done;
        itr += 1;
      }
    }
  } else { /* _couple_naive! (hsmac.jl:77-129) */
    box_t core = box3(2, 0, g);
    while (itr < c->itrmax) {
      if (c->overlap) {
        synchalo(g, U, 1, 1); synchalo(g, V, 1, 1); synchalo(g, W, 1, 1);
        sweep_box(h, &s, core);
        box_t f[6];
        faces_of(dom3, core, f);
        for (int q = 0; q < 6; q++) sweep_box(h, &s, f[q]);
      } else {
        synchalo(g, U, 1, 1); synchalo(g, V, 1, 1); synchalo(g, W, 1, 1); synchalo(g, h->P, 1, 1);
        sweep_box(h, &s, dom3);
      }
      sweeps++;
      div = residual(h);
      if (!isfinite(div)) return fail(h, LCS_ENONFINITE, "HSMAC residual is not finite at itr %d", itr);
      if (div * dxmin < c->epsp && c->itrmin <= itr) break;
      itr += 1;
    }
  }
done:
  if (log) { log->itr = itr; log->sweeps = sweeps; log->div = div; }
  return LCS_OK;
}

/* ---- timestep (src/flows/timestep.jl:18-65, src/timestep.jl:14-27) ----- */
static double flow_timestep(lcs_handle* h) {
  const grid_t* g = &h->g;
  const lcs_config* c = &h->cfg;
  synchalo(g, h->U, g->h, 0); synchalo(g, h->V, g->h, 0); synchalo(g, h->W, g->h, 0);
  const size_t sy = (size_t)g->s[0], sz = (size_t)g->s[0] * g->s[1];
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= g->n[2]; k++)
    for (int j = 1; j <= g->n[1]; j++)
      for (int i = 1; i <= g->n[0]; i++) {
        size_t q = IX(g, i, j, k);
        h->Ui[0][q] = interp_o4_at_half(h->U[q - 2], h->U[q - 1], h->U[q], h->U[q + 1]);
        h->Ui[1][q] = interp_o4_at_half(h->V[q - 2 * sy], h->V[q - sy], h->V[q], h->V[q + sy]);
        h->Ui[2][q] = interp_o4_at_half(h->W[q - 2 * sz], h->W[q - sz], h->W[q], h->W[q + sz]);
      }
  double mx[3] = {0, 0, 0};
  for (int a = 0; a < 3; a++) {
    int first = 1;
    for (int k = 1; k <= g->n[2]; k++)
      for (int j = 1; j <= g->n[1]; j++)
        for (int i = 1; i <= g->n[0]; i++) {
          double v = fabs(h->Ui[a][IX(g, i, j, k)]);
          mx[a] = first ? v : jl_max(mx[a], v);  /* maximum(abs, ...): NaN propagates */
          first = 0;
        }
    mx[a] = mx[a] + 1e-10;
  }
  double dx = spacing(g, 0), dy = spacing(g, 1), dz = spacing(g, 2);
  double Re = Re_of(c);
  double cands[5] = {c->dtmax, c->cfl * dx / mx[0], c->cfl * dy / mx[1], c->cfl * dz / mx[2],
                     0.5 * ((dx / 2.0) * (dx / 2.0)) / (1.0 / Re)};
  double m = cands[0];
  for (int q = 1; q < 5; q++) m = jl_min(m, cands[q]);
  return m;
}

static double taup(const lcs_config* c, const lcs_species* s, double diam) { /* particles/config.jl:41 */
  return 1.0 / 18.0 * s->density_ratio * Re_of(c) * (diam * diam);
}

static double particles_timestep(lcs_handle* h) { /* src/particles/timestep.jl:6-25 */
  const lcs_config* c = &h->cfg;
  if (c->mode != LCS_MODE_FLOW_PARTICLE || c->n_species == 0) return c->dtmax;
  double m = INFINITY;
  for (int s = 0; s < c->n_species; s++) {
    double dmax = 0.0;
    for (int64_t p = 0; p < h->sp[s].n; p++) dmax = jl_max(dmax, h->sp[s].p[LCS_PROP_DIAM][p]);
    double tp = taup(c, &c->species[s], dmax);
    m = jl_min(m, jl_min(0.5 * tp, c->dtmax));
  }
  return m;
}

/* ---- forcing: linear-power (src/flows/forcings/lf.jl:27-106) ----------- */
static double forcing_lf(lcs_handle* h, double dt) {
  const grid_t* g = &h->g;
  const double p0 = h->cfg.power;
  double *U = h->U, *V = h->V, *W = h->W, *U2 = h->S1;
  synchalo(g, U, g->h, 1); synchalo(g, V, g->h, 1); synchalo(g, W, g->h, 1);
  const size_t sy = (size_t)g->s[0], sz = (size_t)g->s[0] * g->s[1];
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= g->n[2]; k++)
    for (int j = 1; j <= g->n[1]; j++)
      for (int i = 1; i <= g->n[0]; i++) {
        size_t q = IX(g, i, j, k);
        double u = interp_o2_at_half(U[q - 1], U[q]);
        double v = interp_o2_at_half(V[q - sy], V[q]);
        double w = interp_o2_at_half(W[q - sz], W[q]);
        U2[q] = u * u + v * v + w * w;
      }
  box_t dom = box3(1, 0, g);
  double u2 = mean_haloed(g, U2, dom), um = mean_haloed(g, U, dom), vm = mean_haloed(g, V, dom),
         wm = mean_haloed(g, W, dom);
  double e = 0.5 * (u2 - um * um - vm * vm - wm * wm);
  double A = p0 / (2.0 * e);
  double* Power = U2;
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= g->n[2]; k++)
    for (int j = 1; j <= g->n[1]; j++)
      for (int i = 1; i <= g->n[0]; i++) {
        size_t q = IX(g, i, j, k);
        double usrc = A * (U[q] - um), vsrc = A * (V[q] - vm), wsrc = A * (W[q] - wm);
        double u = U[q], v = V[q], w = W[q];
        double p = u * usrc + v * vsrc + w * wsrc;
        U[q] = u + usrc * dt;
        V[q] = v + vsrc * dt;
        W[q] = w + wsrc * dt;
        Power[q] = p;
      }
  return mean_haloed(g, Power, dom);
}

/* ---- forcing: rc-energy (src/flows/forcings/rcf.jl, lib/fouriertools) --- */
typedef struct { double re, im; } cplx;
static inline cplx cmul(cplx a, cplx b) { /* Julia *(::Complex, ::Complex) */
  cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return r;
}
static inline cplx cconj(cplx a) { cplx r = {a.re, -a.im}; return r; }

/* sin(pi x), cos(pi x) with exact argument reduction (Julia's cispi). */
static void sincospi_host(double x, double* s, double* c) {
  double r = fmod(x, 2.0); /* exact */
  if (r < 0) r += 2.0;
  int neg_s = 0, neg_c = 0;
  if (r >= 1.0) { r -= 1.0; neg_s = 1; neg_c = 1; } /* sin(pi(r+1)) = -sin(pi r) */
  if (r > 0.5) { r = 1.0 - r; neg_c = !neg_c; }      /* sin(pi(1-r)) = sin(pi r), cos -> -cos */
  double ss, cc;
  if (r == 0.0) { ss = 0.0; cc = 1.0; }
  else if (r == 0.5) { ss = 1.0; cc = 0.0; }
  else if (r <= 0.25) { ss = sin(3.14159265358979323846 * r); cc = cos(3.14159265358979323846 * r); }
  else { double t = 0.5 - r; ss = cos(3.14159265358979323846 * t); cc = sin(3.14159265358979323846 * t); }
  *s = neg_s ? -ss : ss;
  *c = neg_c ? -cc : cc;
}

static int kcount(int k0) { /* FourierTools.jl:87-96 */
  int c = 0;
  for (int kz = -k0; kz <= k0; kz++)
    for (int ky = -k0; ky <= k0; ky++)
      for (int kx = -k0; kx <= k0; kx++) {
        int r2 = kx * kx + ky * ky + kz * kz;
        if ((k0 - 0.5) * (k0 - 0.5) <= r2 && r2 < (k0 + 0.5) * (k0 + 0.5)) c++;
      }
  return c;
}

/* kset(k0) in generation order (FourierTools.jl:59-80); returns count. */
static int kset(int k0, int out[][3], int cap) {
  int n = 0;
  for (int kz = -k0; kz <= k0; kz++)
    for (int ky = -k0; ky <= k0; ky++)
      for (int kx = 0; kx <= k0; kx++) {
        int r2 = kx * kx + ky * ky + kz * kz;
        if (!((k0 - 0.5) * (k0 - 0.5) <= r2 && r2 < (k0 + 0.5) * (k0 + 0.5))) continue;
        int k[3] = {kx, ky, kz}, sgn = 1;
        for (int a = 0; a < 3; a++) {
          if (k[a] > 0) { sgn = 1; break; }
          if (k[a] < 0) { sgn = -1; break; }
        }
        int cc[3] = {sgn * kx, sgn * ky, sgn * kz}, seen = 0;
        for (int q = 0; q < n; q++)
          if (out[q][0] == cc[0] && out[q][1] == cc[1] && out[q][2] == cc[2]) seen = 1;
        if (!seen && n < cap) { out[n][0] = cc[0]; out[n][1] = cc[1]; out[n][2] = cc[2]; n++; }
      }
  return n;
}

static double enespe0(int k0, double e10) { /* rcf.jl:187-191 */
  double c1 = (double)kcount(1), ck = (double)kcount(k0);
  double a = k0 + 0.5, b = k0 - 0.5;
  return e10 * pow((double)k0, -5.0 / 3.0) * (1.5 * 1.5 * 1.5 - 0.5 * 0.5 * 0.5) / (a * a * a - b * b * b) * ck / c1;
}

/* fftindex(k, n) = k >= 0 ? k + 1 : n + k + 1 (FourierTools.jl:9): the cropped spectrum below is stored
 * offset by kmax instead, which addresses the same coefficients. */

/* powi: x^n as right-nested products, conj for n < 0 (FourierTools.jl:159-163) */
static int powi(cplx x, int n, cplx* out) { /* returns 0 when the factor is the Int 1 */
  if (n == 0) return 0;
  int m = n < 0 ? -n : n;
  cplx p = x;
  for (int q = 2; q <= m; q++) p = cmul(x, p);
  *out = n < 0 ? cconj(p) : p;
  return 1;
}

/* enespe(U_hat, V_hat, W_hat, k0) (FourierTools.jl:103-120) on the cropped
 * coefficient layout hat[a][kz+kmax][ky+kmax][kx] (re, im), normalised by norm. */
static double enespe_cropped(const cplx* hat, int kmax, int k0, double norm) {
  const int KX = kmax + 1, KY = 2 * kmax + 1, nm = KX * KY * KY;
  double lo = (k0 - 0.5) * (k0 - 0.5), hi = (k0 + 0.5) * (k0 + 0.5);
  double e = 0.0;
  for (int kz = -k0; kz <= k0; kz++)
    for (int ky = -k0; ky <= k0; ky++)
      for (int kx = 0; kx <= k0; kx++) {
        int r2 = kx * kx + ky * ky + kz * kz;
        if (lo <= r2 && r2 < hi) {
          double wgt = kx == 0 ? 1.0 : 2.0, acc = 0.0;
          for (int a = 0; a < 3; a++) {
            cplx z = hat[(size_t)a * nm + ((kz + kmax) * KY + (ky + kmax)) * KX + kx];
            double zr = z.re / norm, zi = z.im / norm;
            double ab = zr * zr + zi * zi;
            acc = a == 0 ? ab : acc + ab;
          }
          e += wgt * acc;
        }
      }
  return e / 2.0;
}

static double forcing_rcf(lcs_handle* h, double dt, double* e10_out) {
  const grid_t* g = &h->g;
  const lcs_config* c = &h->cfg;
  const int cs = c->coarse_size, kmin = c->kmin, kmax = c->kmax;
  const int fx = g->n[0] / cs, fy = g->n[1] / cs, fz = g->n[2] / cs; /* filter_dims */
  const double dti = 1.0 / dt;
  const double phi = (double)(g->n[0] / cs) / 2.0;                   /* phase_shift (flows/config.jl:149) */
  const double e10 = c->energy;
  double* Us[3] = {h->U, h->V, h->W};
  const int ncs = cs * cs * cs;
  double* coarse = (double*)malloc(sizeof(double) * 3 * ncs);
  /* boxmean_l! (ext/AMDGPUExt.jl:25-40 loop order) */
  for (int a = 0; a < 3; a++) {
    const double w = 1.0 / (double)(fx * fy * fz);
    for (int kc = 1; kc <= cs; kc++)
      for (int jc = 1; jc <= cs; jc++)
        for (int ic = 1; ic <= cs; ic++) {
          double s = 0.0;
          for (int dk = 1; dk <= fz; dk++)
            for (int dj = 1; dj <= fy; dj++)
              for (int di = 1; di <= fx; di++)
                s += Us[a][IX(g, (ic - 1) * fx + di, (jc - 1) * fy + dj, (kc - 1) * fz + dk)];
          coarse[(size_t)a * ncs + ((kc - 1) * cs + (jc - 1)) * cs + (ic - 1)] = s * w;
        }
  }
  /* rfft coefficients of the modes |k_a| <= kmax, kx >= 0, by direct DFT
   * (FFTW in the reference, rcf.jl:45-47): hat[kz][ky][kx] over (2kmax+1)^2 x (kmax+1) */
  const int KX = kmax + 1, KY = 2 * kmax + 1, KZ = 2 * kmax + 1;
  const int nm = KX * KY * KZ;
  cplx* hat = (cplx*)calloc((size_t)3 * nm, sizeof(cplx));
  cplx* tw = (cplx*)malloc(sizeof(cplx) * cs);
  for (int x = 0; x < cs; x++) { double s, co; sincospi_host(-2.0 * x / cs, &s, &co); tw[x].re = co; tw[x].im = s; }
  for (int a = 0; a < 3; a++)
    for (int kz = -kmax; kz <= kmax; kz++)
      for (int ky = -kmax; ky <= kmax; ky++)
        for (int kx = 0; kx <= kmax; kx++) {
          double sre = 0.0, sim = 0.0;
          for (int z = 0; z < cs; z++)
            for (int y = 0; y < cs; y++)
              for (int x = 0; x < cs; x++) {
                int ph = (((kx * x + ky * y + kz * z) % cs) + cs) % cs;
                double v = coarse[(size_t)a * ncs + (z * cs + y) * cs + x];
                sre += v * tw[ph].re;
                sim += v * tw[ph].im;
              }
          cplx* o = &hat[(size_t)a * nm + ((kz + kmax) * KY + (ky + kmax)) * KX + kx];
          o->re = sre;
          o->im = sim;
        }
  /* rfftcoeff normalises by prod((2*size(A_hat,1)-2, size(A_hat)[2:end]...)) (FourierTools.jl:31-41) */
  const double norm = (double)(2 * (cs / 2 + 1) - 2) * cs * cs;
#define HAT(a, kx, ky, kz) hat[(size_t)(a) * nm + (((kz) + kmax) * KY + ((ky) + kmax)) * KX + (kx)]
  for (int k0 = kmin; k0 <= kmax; k0++) {
    double lo = (k0 - 0.5) * (k0 - 0.5), hi = (k0 + 0.5) * (k0 + 0.5);
    double en = enespe_cropped(hat, kmax, k0, norm);
    double en0 = enespe0(k0, e10);
    double r = sqrt(en0 / jl_max(en, 1e-8)) - 1.0;
    for (int kz = -kmax; kz <= kmax; kz++)
      for (int ky = -kmax; ky <= kmax; ky++)
        for (int kx = 0; kx <= kmax; kx++) {
          int r2 = kx * kx + ky * ky + kz * kz;
          if (lo <= r2 && r2 < hi)
            for (int a = 0; a < 3; a++) { HAT(a, kx, ky, kz).re *= r; HAT(a, kx, ky, kz).im *= r; }
        }
  }
  /* crop (FourierTools.jl:142-157): Ac[a][kz][ky][kx] = hat / N^3 */
  cplx* Ac = (cplx*)malloc(sizeof(cplx) * 3 * nm);
  for (int a = 0; a < 3; a++)
    for (int q = 0; q < nm; q++) {
      Ac[(size_t)a * nm + q].re = hat[(size_t)a * nm + q].re / norm;
      Ac[(size_t)a * nm + q].im = hat[(size_t)a * nm + q].im / norm;
    }
#undef HAT
  /* phase tables cispi(2 (i_g - phi) / n) (rcf.jl:78-80) */
  cplx* ph[3];
  for (int a = 0; a < 3; a++) {
    ph[a] = (cplx*)malloc(sizeof(cplx) * (g->n[a] + 1));
    for (int i = 1; i <= g->n[a]; i++) {
      double s, co;
      sincospi_host(2.0 * (i - phi) * (1.0 / g->n[a]), &s, &co);
      ph[a][i].re = co;
      ph[a][i].im = s;
    }
  }
  int ks[256][3], kofs[16], nk = 0; /* kset(1..4) hold 9 + 31 + 49 + 105 vectors */
  for (int K = kmin; K <= kmax; K++) { kofs[K - kmin] = nk; nk += kset(K, ks + nk, 256 - nk); }
  kofs[kmax - kmin + 1] = nk;
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= g->n[2]; k++)
    for (int j = 1; j <= g->n[1]; j++)
      for (int i = 1; i <= g->n[0]; i++) {
        cplx ei = ph[0][i], ej = ph[1][j], ek = ph[2][k];
        double src[3];
        for (int a = 0; a < 3; a++) {
          double tot = 0.0;
          for (int K = kmin; K <= kmax; K++) {
            double acc = 0.0; /* sirdft(Val(K)) (FourierTools.jl:165-180) */
            for (int q = kofs[K - kmin]; q < kofs[K - kmin + 1]; q++) {
              int kx = ks[q][0], ky = ks[q][1], kz = ks[q][2];
              cplx fxv, fyv, fzv, prod;
              int hx = powi(ei, kx, &fxv), hy = powi(ej, ky, &fyv), hz = powi(ek, kz, &fzv);
              int have = 0;
              if (hx) { prod = fxv; have = 1; }
              if (hy) { prod = have ? cmul(prod, fyv) : fyv; have = 1; }
              if (hz) { prod = have ? cmul(prod, fzv) : fzv; have = 1; }
              if (!have) { prod.re = 1.0; prod.im = 0.0; }
              cplx A = Ac[(size_t)a * nm + ((kz + kmax) * KY + (ky + kmax)) * KX + kx];
              acc += 2.0 * (A.re * prod.re - A.im * prod.im);
            }
            tot += acc;
          }
          src[a] = tot;
        }
        size_t q = IX(g, i, j, k);
        double u = h->U[q], v = h->V[q], w = h->W[q];
        double p = (u * src[0] + v * src[1] + w * src[2]) * dti;
        h->U[q] += src[0];
        h->V[q] += src[1];
        h->W[q] += src[2];
        h->S1[q] = p;
      }
  double pm = mean_haloed(g, h->S1, box3(1, 0, g));
  for (int a = 0; a < 3; a++) free(ph[a]);
  free(Ac); free(tw); free(hat); free(coarse);
  if (e10_out) *e10_out = e10;
  return pm;
}

/* ---- particles (src/particles/{boundary,interp,motion,update}.jl) ------ */
typedef struct { int i, j, k; double r1, r2, r3; } mapping_t;
static inline int unsafe_floor(double x) { return (int)floor(x); } /* Utils.unsafe_floor (fast.jl:49-52) */
static inline mapping_t xmapping(double x, double y, double z, double dx, double dy, double dz) {
  mapping_t m;
  m.i = unsafe_floor(x / dx); m.j = unsafe_floor(y / dy + 0.5); m.k = unsafe_floor(z / dz + 0.5);
  m.r1 = x / dx - m.i; m.r2 = y / dy - m.j + 0.5; m.r3 = z / dz - m.k + 0.5;
  return m;
}
static inline mapping_t ymapping(double x, double y, double z, double dx, double dy, double dz) {
  mapping_t m;
  m.j = unsafe_floor(y / dy); m.k = unsafe_floor(z / dz + 0.5); m.i = unsafe_floor(x / dx + 0.5);
  m.r2 = y / dy - m.j; m.r3 = z / dz - m.k + 0.5; m.r1 = x / dx - m.i + 0.5;
  return m;
}
static inline mapping_t zmapping(double x, double y, double z, double dx, double dy, double dz) {
  mapping_t m;
  m.k = unsafe_floor(z / dz); m.i = unsafe_floor(x / dx + 0.5); m.j = unsafe_floor(y / dy + 0.5);
  m.r3 = z / dz - m.k; m.r2 = y / dy - m.j + 0.5; m.r1 = x / dx - m.i + 0.5;
  return m;
}
static inline double interp(const grid_t* g, const double* U, mapping_t m) { /* interp.jl:62-90 */
  int i = m.i, j = m.j, k = m.k;
  double r1 = m.r1, r2 = m.r2, r3 = m.r3;
  double c0 = U[IX(g, i, j, k)], c1 = U[IX(g, i + 1, j, k)], c2 = U[IX(g, i + 1, j + 1, k)],
         c3 = U[IX(g, i, j + 1, k)], c4 = U[IX(g, i, j, k + 1)], c5 = U[IX(g, i + 1, j, k + 1)],
         c6 = U[IX(g, i + 1, j + 1, k + 1)], c7 = U[IX(g, i, j + 1, k + 1)];
  return (1 - r1) * (1 - r2) * (1 - r3) * c0 + r1 * (1 - r2) * (1 - r3) * c1 + r1 * r2 * (1 - r3) * c2 +
         (1 - r1) * r2 * (1 - r3) * c3 + (1 - r1) * (1 - r2) * r3 * c4 + r1 * (1 - r2) * r3 * c5 +
         r1 * r2 * r3 * c6 + (1 - r1) * r2 * r3 * c7;
}

static void particles_boundary(lcs_handle* h, int s, int stage) { /* boundary.jl:81-120 */
  species_t* sp = &h->sp[s];
  int a0 = stage == 1 ? LCS_PROP_X : LCS_PROP_X2, b0 = stage == 1 ? LCS_PROP_X2 : LCS_PROP_X;
  const double L = DOMAIN_LENGTH, O = DOMAIN_ORIGIN;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < sp->n; p++)
    for (int a = 0; a < 3; a++) {
      double* X = sp->p[a0 + a];
      double* X2 = sp->p[b0 + a];
      double x = X[p], x2 = X2[p];
      if (x < O) { X[p] = x + L; X2[p] = x2 + L; }
      if (x >= O + L) { X[p] = x - L; X2[p] = x2 - L; }
    }
}

static void particles_motion(lcs_handle* h, int s, int stage) { /* motion.jl:38-84 */
  species_t* sp = &h->sp[s];
  const grid_t* g = &h->g;
  const lcs_config* c = &h->cfg;
  const lcs_species* ps = &c->species[s];
  double *U, *V, *W;
  get_Us(h, stage == 1 ? 0 : 1, &U, &V, &W);
  int xo = stage == 1 ? LCS_PROP_X : LCS_PROP_X2, uo = stage == 1 ? LCS_PROP_U : LCS_PROP_U2;
  const double dx = spacing(g, 0), dy = spacing(g, 1), dz = spacing(g, 2);
  const double Re = Re_of(c), gr = ps->gravity;
  const double ox = 0.0, oy = 0.0, oz = 0.0; /* origins_l on one process */
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < sp->n; p++) {
    double xp = sp->p[xo][p], yp = sp->p[xo + 1][p], zp = sp->p[xo + 2][p];
    double up = sp->p[uo][p], vp = sp->p[uo + 1][p], wp = sp->p[uo + 2][p];
    double diam = sp->p[LCS_PROP_DIAM][p];
    double uf = interp(g, U, xmapping(xp - ox, yp - oy, zp - oz, dx, dy, dz));
    double vf = interp(g, V, ymapping(xp - ox, yp - oy, zp - oz, dx, dy, dz));
    double wf = interp(g, W, zmapping(xp - ox, yp - oy, zp - oz, dx, dy, dz));
    double f = 1.0;
    if (ps->drag == LCS_DRAG_NONLINEAR) {
      double a = uf - up, b = vf - vp, cc = wf - wp;
      double vrel = sqrt(a * a + b * b + cc * cc);
      double Rep = diam * vrel * Re;
      f = 1.0 + 0.15 * pow(Rep, 0.687);
    }
    double taui = 1.0 / taup(c, ps, diam);
    sp->p[LCS_PROP_DUDT][p] = f * (uf - up) * taui - gr;
    sp->p[LCS_PROP_DVDT][p] = f * (vf - vp) * taui;
    sp->p[LCS_PROP_DWDT][p] = f * (wf - wp) * taui;
  }
}

static void particles_update(lcs_handle* h, int s, int stage, double dt) { /* update.jl:1-65 */
  species_t* sp = &h->sp[s];
  int xo = stage == 1 ? LCS_PROP_X2 : LCS_PROP_X, uo = stage == 1 ? LCS_PROP_U2 : LCS_PROP_U;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < sp->n; p++)
    for (int a = 0; a < 3; a++) {
      double x0 = sp->p[LCS_PROP_X + a][p], u0 = sp->p[LCS_PROP_U + a][p];
      double dudt = sp->p[LCS_PROP_DUDT + a][p];
      sp->p[xo + a][p] = x0 + dt * u0;
      sp->p[uo + a][p] = u0 + dt * dudt;
    }
}

/* ---- evolve! (src/evolve.jl:15-146) ------------------------------------ */
static int evolve(lcs_handle* h, double dt, lcs_log* log) {
  const grid_t* g = &h->g;
  const lcs_config* c = &h->cfg;
  int particles = c->mode == LCS_MODE_FLOW_PARTICLE;
  lcs_log L;
  memset(&L, 0, sizeof L);
  L.forcing_p = NAN;
  L.forcing_e10 = NAN;
  int rc;
  for (int stage = 1; stage <= 2; stage++) {
    double dtrk = stage == 1 ? 0.5 * dt : dt; /* state.jl:37-38 */
    double *U, *V, *W;
    get_Us(h, stage == 1 ? 0 : 1, &U, &V, &W);
    synchalo(g, U, g->h, 1); synchalo(g, V, g->h, 1); synchalo(g, W, g->h, 1); synchalo(g, h->P, g->h, 1);
    if (particles) {
      for (int s = 0; s < c->n_species; s++) particles_boundary(h, s, stage);
      for (int s = 0; s < c->n_species; s++) particles_motion(h, s, stage);
      for (int s = 0; s < c->n_species; s++) particles_update(h, s, stage, dtrk);
    }
    flow_rhs(h, stage);
    flow_update(h, stage, dtrk);
    if (stage == 2) {
      if (c->forcing == LCS_FORCING_LINEAR_POWER) L.forcing_p = forcing_lf(h, dtrk);
      else if (c->forcing == LCS_FORCING_RC_ENERGY) L.forcing_p = forcing_rcf(h, dtrk, &L.forcing_e10);
    }
    rc = couple(h, stage, dtrk, stage == 1 ? &L.couple1 : &L.couple2);
    if (rc) return rc;
  }
  h->step += 1; /* evolve.jl:10-13 */
  h->t += dt;
  L.dt = dt;
  L.t = h->t;
  L.step = h->step;
  if (log) *log = L;
  return LCS_OK;
}

/* ---- C ABI ------------------------------------------------------------- */
static double* zalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

int lcs_footprint(const lcs_config* cfg, int64_t* bytes) {
  if (!cfg || !bytes) return LCS_EINVAL;
  int64_t s = 1, n = 1;
  for (int a = 0; a < 3; a++) { s *= cfg->dims[a] + 2 * cfg->halo_size; n *= cfg->dims[a]; }
  int64_t b = (7 + 6 + 1 + 1 + 3) * s * 8 + 3 * n * 8;
  for (int q = 0; q < cfg->n_species; q++) b += cfg->species[q].nvalid * (LCS_NPROP * 8 + 8);
  *bytes = b;
  return LCS_OK;
}

int lcs_create(const lcs_config* cfg, lcs_handle** out) {
  if (!cfg || !out) return fail(NULL, LCS_EINVAL, "null argument");
  if (cfg->abi_version != LCS_ABI_VERSION) return fail(NULL, LCS_EINVAL, "abi_version mismatch");
  for (int a = 0; a < 3; a++)
    if (cfg->dims[a] < 4 || cfg->dims[a] % 2) return fail(NULL, LCS_EINVAL, "dims must be even and >= 4");
  if (cfg->halo_size < 3) return fail(NULL, LCS_EINVAL, "halo_size must be >= 3");
  if (cfg->n_species < 0 || cfg->n_species > LCS_MAX_SPECIES) return fail(NULL, LCS_EINVAL, "bad n_species");
  /* maximum(diams) over an empty species throws in the reference (src/particles/timestep.jl:22) */
  for (int s = 0; cfg->mode == LCS_MODE_FLOW_PARTICLE && s < cfg->n_species; s++)
    if (cfg->species[s].nvalid < 1) return fail(NULL, LCS_EINVAL, "every particle species needs at least one particle");
  if (cfg->coloring == LCS_COLORING_RED_BLACK_BLOCK && cfg->coloring_block < 1)
    return fail(NULL, LCS_EINVAL, "red-black-block needs size >= 1");
  if (cfg->forcing == LCS_FORCING_RC_ENERGY) {
    if (cfg->kmin < 1 || cfg->kmax < cfg->kmin || cfg->kmax > 4)
      return fail(NULL, LCS_EINVAL, "rc-energy needs 1 <= kmin <= kmax <= 4");
    /* fftindex into the rfft of the coarse grid stays in bounds only for kmax <= coarse_size/2 */
    if (2 * cfg->kmax > cfg->coarse_size || cfg->dims[0] % cfg->coarse_size || cfg->dims[1] % cfg->coarse_size ||
        cfg->dims[2] % cfg->coarse_size)
      return fail(NULL, LCS_EINVAL, "rc-energy coarse_size must divide dims and be >= 2*kmax");
  }
  lcs_handle* h = (lcs_handle*)calloc(1, sizeof(lcs_handle));
  h->cfg = *cfg;
  for (int a = 0; a < 3; a++) { h->g.n[a] = cfg->dims[a]; h->g.s[a] = cfg->dims[a] + 2 * cfg->halo_size; }
  h->g.h = cfg->halo_size;
  h->hsz = (size_t)h->g.s[0] * h->g.s[1] * h->g.s[2];
  h->isz = (size_t)h->g.n[0] * h->g.n[1] * h->g.n[2];
  h->U = zalloc(h->hsz); h->V = zalloc(h->hsz); h->W = zalloc(h->hsz);
  h->U2 = zalloc(h->hsz); h->V2 = zalloc(h->hsz); h->W2 = zalloc(h->hsz); h->P = zalloc(h->hsz);
  h->dU = zalloc(h->isz); h->dV = zalloc(h->isz); h->dW = zalloc(h->isz);
  for (int q = 0; q < 6; q++) h->J[q] = zalloc(h->hsz);
  h->Div2 = zalloc(h->hsz);
  h->S1 = zalloc(h->hsz);
  for (int q = 0; q < 3; q++) h->Ui[q] = zalloc(h->hsz);
  for (int s = 0; s < cfg->n_species; s++) {
    h->sp[s].n = cfg->species[s].nvalid;
    for (int q = 0; q < LCS_NPROP; q++) h->sp[s].p[q] = zalloc((size_t)h->sp[s].n);
    h->sp[s].ids = (int64_t*)calloc((size_t)h->sp[s].n + 1, sizeof(int64_t));
  }
  *out = h;
  return LCS_OK;
}

void lcs_destroy(lcs_handle* h) {
  if (!h) return;
  double* all[] = {h->U, h->V, h->W, h->U2, h->V2, h->W2, h->P, h->dU, h->dV, h->dW, h->Div2, h->S1};
  for (size_t q = 0; q < sizeof all / sizeof *all; q++) free(all[q]);
  for (int q = 0; q < 6; q++) free(h->J[q]);
  for (int q = 0; q < 3; q++) free(h->Ui[q]);
  for (int s = 0; s < h->cfg.n_species; s++) {
    for (int q = 0; q < LCS_NPROP; q++) free(h->sp[s].p[q]);
    free(h->sp[s].ids);
    free(h->sp[s].ci_hashes);
    free(h->sp[s].ci_starts);
    free(h->sp[s].ci_stops);
  }
  free(h->async_logs);
  free(h);
}

const char* lcs_last_error(const lcs_handle* h) { return h ? h->err : g_err; }

/* The oracle has no device waits: the test hook only checks its argument. */
int lcs_debug_unreachable_waits(lcs_handle* h, int32_t kind) {
  if (!h) return LCS_EINVAL;
  if (kind < 0 || kind > 2) return fail(h, LCS_EINVAL, "debug wait kind must be 0, 1 or 2");
  return LCS_OK;
}
static int wrapi(int i, int n);
int lcs_flow_divergence(lcs_handle* h, double* rms, double* maxabs) {
  if (!h) return LCS_EINVAL;
  const grid_t* g = &h->g;
  const int nx = g->n[0], ny = g->n[1], nz = g->n[2];
  const double dxi = 1.0 / spacing(g, 0), dyi = 1.0 / spacing(g, 1), dzi = 1.0 / spacing(g, 2);
  double s2 = 0.0, mx = 0.0;
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        const double dudx = dxi * (-h->U[IX(g, wrapi(i - 1, nx), j, k)] + h->U[IX(g, i, j, k)]);
        const double dvdy = dyi * (-h->V[IX(g, i, wrapi(j - 1, ny), k)] + h->V[IX(g, i, j, k)]);
        const double dwdz = dzi * (-h->W[IX(g, i, j, wrapi(k - 1, nz))] + h->W[IX(g, i, j, k)]);
        const double div = dudx + dvdy + dwdz;
        s2 += div * div;
        mx = jl_max(mx, fabs(div));
      }
  if (rms) *rms = sqrt(s2 / ((double)nx * ny * nz));
  if (maxabs) *maxabs = mx;
  return LCS_OK;
}

int lcs_measure_fp64_peak(int32_t device, double* tflops) {
  (void)device;
  (void)tflops;
  return fail(NULL, LCS_EINVAL, "the CPU oracle has no device");
}

int lcs_get_config(const lcs_handle* h, lcs_config* out) {
  if (!h || !out) return LCS_EINVAL;
  *out = h->cfg;
  return LCS_OK;
}

static double* field_ptr(lcs_handle* h, int f) {
  switch (f) {
    case LCS_FIELD_U: return h->U;
    case LCS_FIELD_V: return h->V;
    case LCS_FIELD_W: return h->W;
    case LCS_FIELD_U2: return h->U2;
    case LCS_FIELD_V2: return h->V2;
    case LCS_FIELD_W2: return h->W2;
    case LCS_FIELD_P: return h->P;
    case LCS_FIELD_DUDT: return h->dU;
    case LCS_FIELD_DVDT: return h->dV;
    case LCS_FIELD_DWDT: return h->dW;
  }
  return NULL;
}

int lcs_field_set(lcs_handle* h, int32_t f, const double* data, int32_t haloed) {
  if (!h || !data) return LCS_EINVAL;
  double* A = field_ptr(h, f);
  if (!A) return fail(h, LCS_EINVAL, "bad field %d", f);
  const grid_t* g = &h->g;
  if (f >= LCS_FIELD_DUDT) { memcpy(A, data, h->isz * sizeof(double)); return LCS_OK; }
  if (haloed) { memcpy(A, data, h->hsz * sizeof(double)); return LCS_OK; }
  for (int k = 1; k <= g->n[2]; k++)
    for (int j = 1; j <= g->n[1]; j++)
      for (int i = 1; i <= g->n[0]; i++) A[IX(g, i, j, k)] = data[IN(g, i, j, k)];
  return LCS_OK;
}

int lcs_field_get(lcs_handle* h, int32_t f, double* data, int32_t haloed) {
  if (!h || !data) return LCS_EINVAL;
  double* A = field_ptr(h, f);
  if (!A) return fail(h, LCS_EINVAL, "bad field %d", f);
  const grid_t* g = &h->g;
  if (f >= LCS_FIELD_DUDT) { memcpy(data, A, h->isz * sizeof(double)); return LCS_OK; }
  if (haloed) { memcpy(data, A, h->hsz * sizeof(double)); return LCS_OK; }
  for (int k = 1; k <= g->n[2]; k++)
    for (int j = 1; j <= g->n[1]; j++)
      for (int i = 1; i <= g->n[0]; i++) data[IN(g, i, j, k)] = A[IX(g, i, j, k)];
  return LCS_OK;
}

int lcs_upload_flow(lcs_handle* h, const double* U, const double* V, const double* W, const double* P) {
  int rc = 0;
  rc |= lcs_field_set(h, LCS_FIELD_U, U, 0);
  rc |= lcs_field_set(h, LCS_FIELD_V, V, 0);
  rc |= lcs_field_set(h, LCS_FIELD_W, W, 0);
  rc |= lcs_field_set(h, LCS_FIELD_P, P, 0);
  return rc ? LCS_EINVAL : LCS_OK;
}

/* load_coarse_flow_fields! (src/LCSIO/upsample.jl:1-45): the coarse interior
 * in a (m+2)^3 array with a periodic one-cell halo (the FullHalo(1) synchalo!
 * on one rank), then trilinear_upsample2x! (upsample.jl:47-91) into the fine
 * interior, term by term. */
int lcs_upload_flow_coarse(lcs_handle* h, const double* U, const double* V, const double* W, const double* P) {
  if (!h || !U || !V || !W || !P) return LCS_EINVAL;
  const grid_t* g = &h->g;
  if (g->n[0] % 2 || g->n[1] % 2 || g->n[2] % 2) return fail(h, LCS_EINVAL, "upsampling needs even dims");
  const int mx = g->n[0] / 2, my = g->n[1] / 2, mz = g->n[2] / 2;
  const int sx = mx + 2, sy = my + 2, sz = mz + 2;
  double* Ac = (double*)malloc((size_t)sx * sy * sz * sizeof(double));
  const double* src[4] = {U, V, W, P};
  double* dst[4] = {h->U, h->V, h->W, h->P};
#define AC(i, j, k) Ac[(i) + (size_t)sx * ((j) + (size_t)sy * (k))] /* logical 0..m+1 */
  for (int q = 0; q < 4; q++) {
    for (int k = 0; k <= mz + 1; k++)
      for (int j = 0; j <= my + 1; j++)
        for (int i = 0; i <= mx + 1; i++) {
          const int ii = (i + mx - 1) % mx, jj = (j + my - 1) % my, kk = (k + mz - 1) % mz; /* periodic */
          AC(i, j, k) = src[q][ii + (size_t)mx * (jj + (size_t)my * kk)];
        }
    double* F = dst[q];
    for (int k = 1; k <= mz; k++)
      for (int j = 1; j <= my; j++)
        for (int i = 1; i <= mx; i++) {
          const int a = 2 * i - 1, b = 2 * j - 1, c = 2 * k - 1;
          F[IX(g, a, b, c)] = AC(i, j, k);
          F[IX(g, a + 1, b, c)] = (1.0 / 2) * (AC(i, j, k) + AC(i + 1, j, k));
          F[IX(g, a, b + 1, c)] = (1.0 / 2) * (AC(i, j, k) + AC(i, j + 1, k));
          F[IX(g, a, b, c + 1)] = (1.0 / 2) * (AC(i, j, k) + AC(i, j, k + 1));
          F[IX(g, a + 1, b + 1, c)] = (1.0 / 4) * (AC(i, j, k) + AC(i + 1, j, k) + AC(i, j + 1, k) + AC(i + 1, j + 1, k));
          F[IX(g, a + 1, b, c + 1)] = (1.0 / 4) * (AC(i, j, k) + AC(i + 1, j, k) + AC(i, j, k + 1) + AC(i + 1, j, k + 1));
          F[IX(g, a, b + 1, c + 1)] = (1.0 / 4) * (AC(i, j, k) + AC(i, j + 1, k) + AC(i, j, k + 1) + AC(i, j + 1, k + 1));
          F[IX(g, a + 1, b + 1, c + 1)] =
              (1.0 / 8) * (AC(i, j, k) + AC(i + 1, j, k) + AC(i, j + 1, k) + AC(i, j, k + 1) + AC(i + 1, j + 1, k) +
                           AC(i + 1, j, k + 1) + AC(i, j + 1, k + 1) + AC(i + 1, j + 1, k + 1));
        }
  }
#undef AC
  free(Ac);
  return LCS_OK;
}

/* Groups (no reference counterpart): on the CPU a group's step is its members'
 * steps one after another. */
struct lcs_group {
  int32_t m;
  lcs_handle** h;
};
int lcs_group_create(lcs_handle* const* members, int32_t m, lcs_group** out) {
  if (!out) return fail(NULL, LCS_EINVAL, "null output");
  *out = NULL;
  if (!members || m < 2 || m > 64) return fail(NULL, LCS_EINVAL, "a group has 2..64 members");
  for (int32_t q = 0; q < m; q++) {
    if (!members[q]) return fail(NULL, LCS_EINVAL, "null group member");
    const lcs_config *a = &members[0]->cfg, *b = &members[q]->cfg;
    if (a->dims[0] != b->dims[0] || a->dims[1] != b->dims[1] || a->dims[2] != b->dims[2] ||
        a->halo_size != b->halo_size || a->precision != b->precision || a->itrmax != b->itrmax)
      return fail(NULL, LCS_EINVAL, "group members differ in shape or HSMAC settings");
  }
  lcs_group* g = (lcs_group*)calloc(1, sizeof *g);
  g->m = m;
  g->h = (lcs_handle**)calloc((size_t)m, sizeof *g->h);
  memcpy(g->h, members, (size_t)m * sizeof *g->h);
  *out = g;
  return LCS_OK;
}
int lcs_group_step_begin(lcs_group* g, int32_t nsteps) {
  if (!g) return fail(NULL, LCS_EINVAL, "null group");
  for (int32_t q = 0; q < g->m; q++) {
    const int rc = lcs_step_begin(g->h[q], nsteps);
    if (rc) return fail(NULL, rc, "group member %d: %s", q, g->h[q]->err);
  }
  return LCS_OK;
}
void lcs_group_destroy(lcs_group* g) {
  if (!g) return;
  free(g->h);
  free(g);
}

int lcs_download_flow(lcs_handle* h, double* U, double* V, double* W, double* P) {
  int rc = 0;
  if (U) rc |= lcs_field_get(h, LCS_FIELD_U, U, 0);
  if (V) rc |= lcs_field_get(h, LCS_FIELD_V, V, 0);
  if (W) rc |= lcs_field_get(h, LCS_FIELD_W, W, 0);
  if (P) rc |= lcs_field_get(h, LCS_FIELD_P, P, 0);
  return rc ? LCS_EINVAL : LCS_OK;
}

static int check_species(lcs_handle* h, int s) {
  if (!h) return LCS_EINVAL;
  if (s < 0 || s >= h->cfg.n_species) return fail(h, LCS_EINVAL, "bad species %d", s);
  return LCS_OK;
}

int lcs_upload_particles(lcs_handle* h, int32_t s, int64_t n, const int64_t* ids, const double* diam, const double* x,
                         const double* y, const double* z, const double* u, const double* v, const double* w) {
  int rc = check_species(h, s);
  if (rc) return rc;
  species_t* sp = &h->sp[s];
  if (n != sp->n) return fail(h, LCS_EINVAL, "species %d holds %lld particles, got %lld", s, (long long)sp->n, (long long)n);
  const double* src[7] = {diam, x, y, z, u, v, w};
  int dst[7] = {LCS_PROP_DIAM, LCS_PROP_X, LCS_PROP_Y, LCS_PROP_Z, LCS_PROP_U, LCS_PROP_V, LCS_PROP_W};
  for (int q = 0; q < 7; q++)
    if (src[q]) memcpy(sp->p[dst[q]], src[q], (size_t)n * sizeof(double));
  if (ids) memcpy(sp->ids, ids, (size_t)n * sizeof(int64_t));
  return LCS_OK;
}

int lcs_download_particles(lcs_handle* h, int32_t s, int64_t* ids, double* diam, double* x, double* y, double* z,
                           double* u, double* v, double* w) {
  int rc = check_species(h, s);
  if (rc) return rc;
  species_t* sp = &h->sp[s];
  double* dst[7] = {diam, x, y, z, u, v, w};
  int src[7] = {LCS_PROP_DIAM, LCS_PROP_X, LCS_PROP_Y, LCS_PROP_Z, LCS_PROP_U, LCS_PROP_V, LCS_PROP_W};
  for (int q = 0; q < 7; q++)
    if (dst[q]) memcpy(dst[q], sp->p[src[q]], (size_t)sp->n * sizeof(double));
  if (ids) memcpy(ids, sp->ids, (size_t)sp->n * sizeof(int64_t));
  return LCS_OK;
}

int lcs_prop_set(lcs_handle* h, int32_t s, int32_t prop, const double* data) {
  int rc = check_species(h, s);
  if (rc) return rc;
  if (prop < 0 || prop >= LCS_NPROP || !data) return fail(h, LCS_EINVAL, "bad prop");
  memcpy(h->sp[s].p[prop], data, (size_t)h->sp[s].n * sizeof(double));
  return LCS_OK;
}

int lcs_prop_get(lcs_handle* h, int32_t s, int32_t prop, double* data) {
  int rc = check_species(h, s);
  if (rc) return rc;
  if (prop < 0 || prop >= LCS_NPROP || !data) return fail(h, LCS_EINVAL, "bad prop");
  memcpy(data, h->sp[s].p[prop], (size_t)h->sp[s].n * sizeof(double));
  return LCS_OK;
}

int lcs_set_state(lcs_handle* h, int64_t step, double t) {
  if (!h) return LCS_EINVAL;
  h->step = step;
  h->t = t;
  return LCS_OK;
}
int lcs_get_state(lcs_handle* h, int64_t* step, double* t) {
  if (!h) return LCS_EINVAL;
  if (step) *step = h->step;
  if (t) *t = h->t;
  return LCS_OK;
}

int lcs_flow_timestep(lcs_handle* h, double* dt) {
  if (!h || !dt) return LCS_EINVAL;
  *dt = flow_timestep(h);
  return LCS_OK;
}
int lcs_particles_timestep(lcs_handle* h, double* dt) {
  if (!h || !dt) return LCS_EINVAL;
  *dt = particles_timestep(h);
  return LCS_OK;
}
int lcs_timestep(lcs_handle* h, double* dt) {
  if (!h || !dt) return LCS_EINVAL;
  double f = flow_timestep(h);
  if (h->cfg.mode == LCS_MODE_FLOW_PARTICLE) f = jl_min(f, particles_timestep(h));
  if (!isfinite(f) || f <= 0) return fail(h, LCS_ENONFINITE, "dt is not finite/positive: %g", f);
  *dt = f;
  return LCS_OK;
}
int lcs_evolve(lcs_handle* h, double dt, lcs_log* log) {
  if (!h) return LCS_EINVAL;
  return evolve(h, dt, log);
}
int lcs_step(lcs_handle* h, int32_t nsteps, lcs_log* logs) {
  if (!h || nsteps < 0) return LCS_EINVAL;
  for (int q = 0; q < nsteps; q++) {
    double dt;
    int rc = lcs_timestep(h, &dt);
    if (rc) return rc;
    rc = evolve(h, dt, logs ? &logs[q] : NULL);
    if (rc) return rc;
    if (h->sort_interval > 0 && h->step % h->sort_interval == 0)
      for (int s = 0; s < h->cfg.n_species; s++) {
        rc = lcs_particles_makeindex(h, s, 1, h->sort_ratio);
        if (rc) return rc;
      }
  }
  return LCS_OK;
}

/* The particle sort of the CUDA library: makeindex! of every species after
 * each step of lcs_step that brings the counter to a multiple of interval. */
int lcs_set_particle_sort(lcs_handle* h, int32_t interval, int32_t ratio) {
  if (!h) return LCS_EINVAL;
  if (interval < 0) return fail(h, LCS_EINVAL, "interval < 0");
  if (interval > 0) {
    if (h->cfg.mode != LCS_MODE_FLOW_PARTICLE || h->cfg.n_species < 1)
      return fail(h, LCS_EINVAL, "the particle sort needs the flow-particle mode");
    const grid_t* g = &h->g;
    if (ratio < 1 || g->n[0] % ratio || g->n[1] % ratio || g->n[2] % ratio)
      return fail(h, LCS_EINVAL, "grid_ratio must be positive and divide the grid dims");
  }
  h->sort_interval = interval;
  h->sort_ratio = ratio;
  return LCS_OK;
}

int lcs_step_timed(lcs_handle* h, int32_t nsteps, lcs_log* logs, double* ms) {
  double t0 = omp_get_wtime();
  int rc = lcs_step(h, nsteps, logs);
  if (ms) *ms = (omp_get_wtime() - t0) * 1e3;
  return rc;
}
/* Asynchronous steps on the CPU: the steps run inside lcs_step_begin, poll
 * reports them done, finish returns their logs. */
int lcs_step_begin(lcs_handle* h, int32_t nsteps) {
  if (!h) return LCS_EINVAL;
  if (h->async_n) return fail(h, LCS_ESTATE, "steps are already in flight on this handle");
  if (nsteps < 1 || nsteps > LCS_MAX_ASYNC_STEPS) return fail(h, LCS_EINVAL, "nsteps must be in 1..%d", LCS_MAX_ASYNC_STEPS);
  free(h->async_logs);
  h->async_logs = (lcs_log*)calloc((size_t)nsteps, sizeof(lcs_log));
  if (!h->async_logs) return fail(h, LCS_ENOMEM, "host allocation failed");
  h->async_rc = lcs_step(h, nsteps, h->async_logs);
  h->async_n = nsteps;
  return LCS_OK;
}
int lcs_step_poll(lcs_handle* h, int32_t* done) {
  if (!h || !done) return LCS_EINVAL;
  if (!h->async_n) return fail(h, LCS_ESTATE, "no steps in flight on this handle");
  *done = 1;
  return LCS_OK;
}
int lcs_step_finish(lcs_handle* h, lcs_log* logs) {
  if (!h) return LCS_EINVAL;
  if (!h->async_n) return fail(h, LCS_ESTATE, "no steps in flight on this handle");
  const int32_t n = h->async_n;
  h->async_n = 0;
  if (h->async_rc) return h->async_rc;
  if (logs) memcpy(logs, h->async_logs, (size_t)n * sizeof(lcs_log));
  return LCS_OK;
}
/* `Flows.stat` (src/flows/stat.jl:66-153): per-cell squared speed, strain
 * invariant and du/dx moments with the o4 half-point derivative (src/diff.jl),
 * halo reads by periodic wrapping; sums in the order i, j, k. */
static double d1o4(double a, double b, double c, double d) { return (1.0 / 24.0) * (a - 27.0 * b + 27.0 * c - d); }
static int wrapi(int i, int n) { int r = (i - 1) % n; return (r < 0 ? r + n : r) + 1; }
int lcs_flow_stat(lcs_handle* h, lcs_flow_stats* o) {
  if (!h || !o) return LCS_EINVAL;
  const grid_t* g = &h->g;
  const int nx = g->n[0], ny = g->n[1], nz = g->n[2];
  const double dxi = 1.0 / spacing(g, 0), dyi = 1.0 / spacing(g, 1), dzi = 1.0 / spacing(g, 2);
  const double *U = h->U, *V = h->V, *W = h->W;
#define A(F, a, b, c) F[IX(g, wrapi(a, nx), wrapi(b, ny), wrapi(c, nz))]
  double su2 = 0, ss2 = 0, sd2 = 0, sd3 = 0, sd4 = 0, su = 0, sv = 0, sw = 0;
  double mxu = -INFINITY, mxv = -INFINITY, mxw = -INFINITY, mnu = INFINITY, mnv = INFINITY, mnw = INFINITY;
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        const double u = A(U, i, j, k), v = A(V, i, j, k), w = A(W, i, j, k);
        const double dudx = dxi * d1o4(A(U, i - 2, j, k), A(U, i - 1, j, k), u, A(U, i + 1, j, k));
        const double dvdy = dyi * d1o4(A(V, i, j - 2, k), A(V, i, j - 1, k), v, A(V, i, j + 1, k));
        const double dwdz = dzi * d1o4(A(W, i, j, k - 2), A(W, i, j, k - 1), w, A(W, i, j, k + 1));
        const double dudy = dyi * d1o4(A(U, i, j - 2, k), A(U, i, j - 1, k), u, A(U, i, j + 1, k));
        const double dvdx = dxi * d1o4(A(V, i - 1, j - 1, k), A(V, i, j - 1, k), A(V, i + 1, j - 1, k), A(V, i + 2, j - 1, k));
        const double dvdz = dzi * d1o4(A(V, i, j - 1, k - 1), A(V, i, j - 1, k), A(V, i, j - 1, k + 1), A(V, i, j - 1, k + 2));
        const double dwdy = dyi * d1o4(A(W, i, j - 2, k), A(W, i, j - 1, k), w, A(W, i, j + 1, k));
        const double dwdx = dxi * d1o4(A(W, i - 1, j, k - 1), A(W, i, j, k - 1), A(W, i + 1, j, k - 1), A(W, i + 2, j, k - 1));
        const double dudz = dzi * d1o4(A(U, i, j, k - 2), A(U, i, j, k - 1), u, A(U, i, j, k + 1));
        const double s11 = 0.5 * (dudx + dudx), s22 = 0.5 * (dvdy + dvdy), s33 = 0.5 * (dwdz + dwdz);
        const double s12 = 0.5 * (dudy + dvdx), s13 = 0.5 * (dudz + dwdx), s23 = 0.5 * (dvdz + dwdy);
        ss2 += 2.0 * (s11 * s11 + s22 * s22 + s33 * s33 + 2.0 * (s12 * s12 + s13 * s13 + s23 * s23));
        su2 += u * u + v * v + w * w;
        const double d2 = dudx * dudx;
        sd2 += d2; sd3 += d2 * dudx; sd4 += d2 * d2;
        su += u; sv += v; sw += w;
        mxu = jl_max(mxu, u); mxv = jl_max(mxv, v); mxw = jl_max(mxw, w);
        mnu = jl_min(mnu, u); mnv = jl_min(mnv, v); mnw = jl_min(mnw, w);
      }
#undef A
  const double N = (double)nx * ny * nz;
  o->u_mean = su / N; o->v_mean = sv / N; o->w_mean = sw / N;
  o->u_max = mxu; o->v_max = mxv; o->w_max = mxw; o->u_min = mnu; o->v_min = mnv; o->w_min = mnw;
  const double u2 = su2 / N, s2 = ss2 / N, d2 = sd2 / N, d3 = sd3 / N, d4 = sd4 / N;
  const double Re = h->cfg.U0 * h->cfg.L0 / h->cfg.NU;
  o->urms = sqrt(u2 / 3.0);
  o->k = 0.5 * (u2 - o->u_mean * o->u_mean - o->v_mean * o->v_mean - o->w_mean * o->w_mean);
  o->epsilon = s2 / Re;
  o->tau_eta = sqrt(1.0 / o->epsilon / Re);
  o->l_mu = sqrt(15.0 * o->urms * o->urms / o->epsilon / Re);
  o->l_eta = pow(1.0 / o->epsilon / (Re * Re * Re), 0.25);
  o->Re_lambda = o->l_mu * o->urms * Re;
  const int nmin = nx < ny ? (nx < nz ? nx : nz) : (ny < nz ? ny : nz);
  o->k_eta = (nmin / 2.0) * o->l_eta;
  o->skewness = -d3 / pow(d2, 1.5);
  o->flatness = d4 / (d2 * d2);
  o->L = 0.0;
  o->C_epsilon = 0.0;
  return LCS_OK;
}

/* Launch shapes do not exist on the CPU: checked and ignored. */
int lcs_set_tuning(lcs_handle* h, int32_t rw_rows, int32_t zchunk, double share) {
  if (!h) return LCS_EINVAL;
  if ((rw_rows != 0 && rw_rows != 13 && rw_rows != 8 && rw_rows != 5) || zchunk < 0 || !(share > 0.0 && share <= 1.0))
    return fail(h, LCS_EINVAL, "bad tuning");
  return LCS_OK;
}
int lcs_device_bytes(lcs_handle* h, int64_t* bytes) {
  if (!h || !bytes) return LCS_EINVAL;
  return lcs_footprint(&h->cfg, bytes);
}

int lcs_transfer_stats(lcs_handle* h, int64_t* a, int64_t* b) {
  if (!h) return LCS_EINVAL;
  if (a) *a = 0;
  if (b) *b = 0;
  return LCS_OK;
}

int lcs_synchalo(lcs_handle* h, int32_t mask, int32_t r, int32_t full) {
  if (!h || r < 0 || r > h->g.h) return LCS_EINVAL;
  for (int f = 0; f <= LCS_FIELD_P; f++)
    if (mask & (1 << f)) synchalo(&h->g, field_ptr(h, f), r, full);
  return LCS_OK;
}
int lcs_flow_rhs(lcs_handle* h, int32_t stage) {
  if (!h || (stage != 1 && stage != 2)) return LCS_EINVAL;
  flow_rhs(h, stage);
  return LCS_OK;
}
int lcs_flow_update(lcs_handle* h, int32_t stage, double dtrk) {
  if (!h || (stage != 1 && stage != 2)) return LCS_EINVAL;
  flow_update(h, stage, dtrk);
  return LCS_OK;
}
int lcs_flow_rhs_update(lcs_handle* h, int32_t stage, double dtrk) {
  if (!h || (stage != 1 && stage != 2)) return LCS_EINVAL;
  flow_rhs(h, stage);
  flow_update(h, stage, dtrk);
  return LCS_OK;
}
int lcs_flow_couple(lcs_handle* h, int32_t stage, double dtrk, lcs_couple_log* log) {
  if (!h || (stage != 1 && stage != 2)) return LCS_EINVAL;
  return couple(h, stage, dtrk, log);
}
int lcs_flow_forcing(lcs_handle* h, double dtrk, double* p, double* e10) {
  if (!h) return LCS_EINVAL;
  double pp = NAN, ee = NAN;
  if (h->cfg.forcing == LCS_FORCING_LINEAR_POWER) pp = forcing_lf(h, dtrk);
  else if (h->cfg.forcing == LCS_FORCING_RC_ENERGY) pp = forcing_rcf(h, dtrk, &ee);
  if (p) *p = pp;
  if (e10) *e10 = ee;
  return LCS_OK;
}
/* `Particles.makeindex!` (src/particles/makeindex.jl:29-67).  Cell index
 * ci = unsafe_floor(Int32, (x - x0) / dxc) + 1 with dxc = spacing * grid_ratio
 * (particles/config.jl:60), hash = Utils.sub2ind over the axes 0:nc+1
 * (src/utils/hasher.jl:15-38), a stable sort of the particles by hash
 * (makeindex.jl:54-58: sortperm! then sortbyperm! of hashes and every
 * property), then the binary searches of src/utils/fast.jl:8-40 for starts and
 * stops of every hash 1..(nc+2)^3 (makeindex.jl:60-66). */
/* Utils.encode / sub2ind over axes of lengths len[] starting at 0 (hasher.jl:15-38) */
static int64_t encode_cell(const int64_t len[3], const int ci[3]) {
  int64_t hash = 1, stride = 1;
  for (int a = 0; a < 3; a++) {
    hash += (int64_t)ci[a] * stride; /* offset from the axis start 0 */
    stride *= len[a];
  }
  return hash;
}
typedef struct { int64_t h, i; } hash_idx;
static int cmp_hash_idx(const void* a, const void* b) {
  const hash_idx *x = (const hash_idx*)a, *y = (const hash_idx*)b;
  if (x->h != y->h) return x->h < y->h ? -1 : 1;
  return x->i < y->i ? -1 : (x->i > y->i);  /* equal hashes keep their order: stable */
}
static int64_t sorted_first(const int64_t* a, int64_t n, int64_t x) { /* fast.jl:8-24 */
  int64_t lo = 1, len = n;
  while (len != 0) {
    int64_t half = len >> 1, m = lo + half;
    if (a[m - 1] < x) { lo = m + 1; len -= half + 1; }
    else len = half;
  }
  return lo;
}
static int64_t sorted_last(const int64_t* a, int64_t n, int64_t x) { /* fast.jl:26-40 */
  int64_t lo = 0, hi = n + 1;
  while (lo < hi - 1) {
    int64_t m = lo + ((hi - lo) >> 1);
    if (x < a[m - 1]) hi = m;
    else lo = m;
  }
  return lo;
}
int lcs_particles_makeindex(lcs_handle* h, int32_t s, int32_t stage, int32_t ratio) {
  int rc = check_species(h, s);
  if (rc) return rc;
  if (stage != 1 && stage != 2) return fail(h, LCS_EINVAL, "stage must be 1 or 2");
  const grid_t* g = &h->g;
  if (ratio < 1 || g->n[0] % ratio || g->n[1] % ratio || g->n[2] % ratio)
    return fail(h, LCS_EINVAL, "grid_ratio must be positive and divide the grid dims");
  species_t* sp = &h->sp[s];
  const int64_t n = sp->n;
  int nc[3];
  double dxc[3];
  int64_t H = 1;
  for (int a = 0; a < 3; a++) {
    nc[a] = g->n[a] / ratio;
    dxc[a] = spacing(g, a) * ratio;
    H *= nc[a] + 2;
  }
  if (H > (int64_t)UINT32_MAX) return fail(h, LCS_EINVAL, "cell index too large");
  const int pos = stage == 1 ? LCS_PROP_X : LCS_PROP_X2;
  hash_idx* hi = (hash_idx*)malloc((size_t)n * sizeof *hi);
  double* tmp = (double*)malloc((size_t)n * sizeof *tmp);
  free(sp->ci_hashes);
  free(sp->ci_starts);
  free(sp->ci_stops);
  sp->ci_hashes = (int64_t*)malloc((size_t)n * sizeof(int64_t));
  sp->ci_starts = (int64_t*)malloc((size_t)H * sizeof(int64_t));
  sp->ci_stops = (int64_t*)malloc((size_t)H * sizeof(int64_t));
  sp->ci_H = H;
  for (int64_t i = 0; i < n; i++) {
    int ci[3];
    const int64_t len[3] = {nc[0] + 2, nc[1] + 2, nc[2] + 2};
    for (int a = 0; a < 3; a++) ci[a] = (int)floor((sp->p[pos + a][i] - DOMAIN_ORIGIN) / dxc[a]) + 1;
    hi[i].h = encode_cell(len, ci);
    hi[i].i = i;
  }
  qsort(hi, (size_t)n, sizeof *hi, cmp_hash_idx);
  for (int q = 0; q < LCS_NPROP; q++) {
    for (int64_t i = 0; i < n; i++) tmp[i] = sp->p[q][hi[i].i];
    memcpy(sp->p[q], tmp, (size_t)n * sizeof(double));
  }
  int64_t* itmp = (int64_t*)tmp;
  for (int64_t i = 0; i < n; i++) itmp[i] = sp->ids[hi[i].i];
  memcpy(sp->ids, itmp, (size_t)n * sizeof(int64_t));
  for (int64_t i = 0; i < n; i++) sp->ci_hashes[i] = hi[i].h;
  for (int64_t x = 1; x <= H; x++) {
    sp->ci_starts[x - 1] = sorted_first(sp->ci_hashes, n, x);
    sp->ci_stops[x - 1] = sorted_last(sp->ci_hashes, n, x);
  }
  free(hi);
  free(tmp);
  return LCS_OK;
}
int lcs_particles_cellindex(lcs_handle* h, int32_t s, int64_t* hashes, int64_t* starts, int64_t* stops) {
  int rc = check_species(h, s);
  if (rc) return rc;
  const species_t* sp = &h->sp[s];
  if (!sp->ci_hashes) return fail(h, LCS_ESTATE, "no cell index built for species %d", s);
  if (hashes) memcpy(hashes, sp->ci_hashes, (size_t)sp->n * sizeof(int64_t));
  if (starts) memcpy(starts, sp->ci_starts, (size_t)sp->ci_H * sizeof(int64_t));
  if (stops) memcpy(stops, sp->ci_stops, (size_t)sp->ci_H * sizeof(int64_t));
  return LCS_OK;
}
/* ---- particle statistics (src/particles/stat.jl:113-215, rdf.jl, spectrum.jl) */
/* logrange(a, b, len) (Julia Base.LogRange): endpoints exact, the interior
 * exp((len - i) log a + (i - 1) log b) / (len - 1)) evaluated in binary128. */
static void oracle_logrange(double a, double b, int len, double* out) {
  out[0] = a;
  for (int i = 2; i < len; i++) {
    __float128 x = ((__float128)(len - i) * logq((__float128)a) + (__float128)(i - 1) * logq((__float128)b)) /
                   (__float128)(len - 1);
    out[i - 1] = (double)expq(x);
  }
  out[len - 1] = b;
}
static const int WAVENUMBERS[19] = {1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768};
/* Utils.decode (src/utils/hasher.jl:40-59): 0-based offsets from the axis start 0 */
static void decode_cell(int64_t hash, const int nc[3], int c[3]) {
  int64_t lin = hash - 1;
  for (int a = 0; a < 3; a++) {
    c[a] = (int)(lin % (nc[a] + 2));
    lin /= nc[a] + 2;
  }
}
static double norm3(double a, double b, double c) { return sqrt(a * a + b * b + c * c); } /* fast.jl:43-47 */
int lcs_particles_stat(lcs_handle* h, int32_t s, const lcs_particle_stat_config* pc, double tau_eta,
                       lcs_particle_stats* out) {
  int rc = check_species(h, s);
  if (rc) return rc;
  if (!pc || !out) return fail(h, LCS_EINVAL, "null config or output");
  const int nbins = pc->bin_size, ns = pc->nsamples;
  if (nbins < 1 || nbins > LCS_RDF_MAX_BINS) return fail(h, LCS_EINVAL, "bad bin_size");
  if (ns < 2 || ns > LCS_SPECTRUM_MAX_SAMPLES) return fail(h, LCS_EINVAL, "bad nsamples");
  if (pc->search_cell_size < 0 || pc->search_cell_size > 64) return fail(h, LCS_EINVAL, "bad search_cell_size");
  if (!(pc->min_radius > 0.0)) return fail(h, LCS_EINVAL, "bad min_radius");
  species_t* sp = &h->sp[s];
  const int64_t n = sp->n;
  /* Summary (src/stat.jl:20-22): mean = sum / n, sequential sum */
  const int props[7] = {LCS_PROP_X, LCS_PROP_Y, LCS_PROP_Z, LCS_PROP_U, LCS_PROP_V, LCS_PROP_W, LCS_PROP_DIAM};
  lcs_summary* S[7] = {&out->x, &out->y, &out->z, &out->u, &out->v, &out->w, &out->diam};
  for (int q = 0; q < 7; q++) {
    const double* a = sp->p[props[q]];
    double sum = 0.0, mx = -INFINITY, mn = INFINITY;
    for (int64_t i = 0; i < n; i++) {
      sum += a[i];
      mx = jl_max(mx, a[i]);
      mn = jl_min(mn, a[i]);
    }
    S[q]->mean = sum / (double)n;
    S[q]->max = mx;
    S[q]->min = mn;
  }
  const lcs_config* c = &h->cfg;
  const double Re = c->U0 * c->L0 / c->NU;
  const double dm = out->diam.mean;
  out->taup = 1.0 / 18.0 * c->species[s].density_ratio * Re * (dm * dm); /* config.jl:41 */
  out->St = out->taup / tau_eta;
  rc = lcs_particles_makeindex(h, s, 1, pc->grid_ratio);
  if (rc) return rc;
  /* rdf_assume_ci (rdf.jl:1-103) */
  const grid_t* g = &h->g;
  int nc[3];
  for (int a = 0; a < 3; a++) nc[a] = g->n[a] / pc->grid_ratio;
  const double hmin = fmin(spacing(g, 0), fmin(spacing(g, 1), spacing(g, 2)));
  const double rmax = pc->search_cell_size * hmin;
  out->nbins = nbins;
  oracle_logrange(pc->min_radius, rmax, nbins + 1, out->edges);
  int64_t cnt[LCS_RDF_MAX_BINS] = {0}, contact = 0;
  const double *X = sp->p[LCS_PROP_X], *Y = sp->p[LCS_PROP_Y], *Z = sp->p[LCS_PROP_Z];
  const int ncell = pc->search_cell_size;
  for (int64_t i1 = 0; i1 < n; i1++) {
    int c1[3];
    decode_cell(sp->ci_hashes[i1], nc, c1);
    if (c1[0] < 1 || c1[0] > nc[0] || c1[1] < 1 || c1[1] > nc[1] || c1[2] < 1 || c1[2] > nc[2]) continue;
    for (int di = -ncell; di <= ncell; di++)
      for (int dj = -ncell; dj <= ncell; dj++)
        for (int dk = -ncell; dk <= ncell; dk++) {
          const int a = c1[0] + di, b = c1[1] + dj, cc = c1[2] + dk;
          if (a < 0 || a > nc[0] + 1 || b < 0 || b > nc[1] + 1 || cc < 0 || cc > nc[2] + 1) continue;
          const int64_t h2 = 1 + a + (int64_t)b * (nc[0] + 2) + (int64_t)cc * (nc[0] + 2) * (nc[1] + 2);
          for (int64_t i2 = sp->ci_starts[h2 - 1]; i2 <= sp->ci_stops[h2 - 1]; i2++) {
            if (!(sp->ids[i1] < sp->ids[i2 - 1])) continue;
            const double d = norm3(X[i1] - X[i2 - 1], Y[i1] - Y[i2 - 1], Z[i1] - Z[i2 - 1]);
            int k = 0; /* searchsortedfirst(edges, d) - 1, by a linear scan */
            while (k < nbins + 1 && out->edges[k] < d) k++;
            if (k >= 1 && k <= nbins) cnt[k - 1]++;
            if (fabs(d / dm - 1.0) < pc->contact_tolerance) contact++;
          }
        }
  }
  const double L = DOMAIN_LENGTH;
  const double rho0 = (double)(n * (n - 1) / 2) / (L * L * L); /* binomial(n, 2) / volume_g() */
  for (int k = 0; k < nbins; k++) {
    const double e0 = out->edges[k], e1 = out->edges[k + 1];
    const double vol_shell = (4.0 / 3.0) * PI_F64 * (e1 * e1 * e1 - e0 * e0 * e0);
    out->npairs[k] = cnt[k];
    out->gr[k] = ((double)cnt[k] / vol_shell) / rho0;
  }
  out->npairs_contact = contact;
  out->gr_contact = ((double)contact / ((4.0 / 3.0) * PI_F64 * (dm * dm * dm) * 6.0 * pc->contact_tolerance)) / rho0;
  /* spectrum (spectrum.jl:11-78): sequential sums over the particles */
  int nshells = 0;
  while (nshells < 19 && WAVENUMBERS[nshells] <= pc->max_wavenumber) nshells++;
  out->nshells = nshells;
  const double phi0 = PI_F64 * (3.0 - sqrt(5.0));
  for (int b = 0; b < nshells; b++) {
    const double kk = WAVENUMBERS[b];
    out->wavenumbers[b] = kk;
    double phi = 0.0;
    for (int i = 0; i < ns; i++) {
      const double y = 1.0 - ((double)i / (double)(ns - 1)) * 2.0;
      const double radius = sqrt(1.0 - y * y);
      const double theta = phi0 * i;
      const double kx = kk * (cos(theta) * radius), ky = kk * y, kz = kk * (sin(theta) * radius);
      double cs = 0.0, sn = 0.0;
      for (int64_t p = 0; p < n; p++) {
        const double kd = kx * X[p] + ky * Y[p] + kz * Z[p];
        cs += cos(kd);
        sn += sin(kd);
      }
      phi += (cs * cs + sn * sn) / (double)(n * n) - 1.0 / (double)n;
    }
    out->Enp[b] = phi / ns * 4.0 * PI_F64 * (kk * kk);
  }
  return LCS_OK;
}
/* `Particles.density` (stat.jl:176-215) */
int lcs_particles_density(lcs_handle* h, int32_t s, int32_t ratio, double* rho_out) {
  int rc = lcs_particles_makeindex(h, s, 1, ratio);
  if (rc) return rc;
  if (!rho_out) return fail(h, LCS_EINVAL, "null output");
  const species_t* sp = &h->sp[s];
  const grid_t* g = &h->g;
  int nc[3];
  for (int a = 0; a < 3; a++) nc[a] = g->n[a] / ratio;
  const double hh = fmin(spacing(g, 0), fmin(spacing(g, 1), spacing(g, 2)));
  const double factor = 1.0 / (PI_F64 * (hh * hh * hh));
  const double *X = sp->p[LCS_PROP_X], *Y = sp->p[LCS_PROP_Y], *Z = sp->p[LCS_PROP_Z];
  for (int64_t i1 = 0; i1 < sp->n; i1++) {
    int c1[3];
    decode_cell(sp->ci_hashes[i1], nc, c1);
    double rho = 0.0;
    if (c1[0] >= 1 && c1[0] <= nc[0] && c1[1] >= 1 && c1[1] <= nc[1] && c1[2] >= 1 && c1[2] <= nc[2]) {
      for (int di = -1; di <= 1; di++)
        for (int dj = -1; dj <= 1; dj++)
          for (int dk = -1; dk <= 1; dk++) {
            const int64_t h2 = 1 + (c1[0] + di) + (int64_t)(c1[1] + dj) * (nc[0] + 2) +
                               (int64_t)(c1[2] + dk) * (nc[0] + 2) * (nc[1] + 2);
            for (int64_t i2 = sp->ci_starts[h2 - 1]; i2 <= sp->ci_stops[h2 - 1]; i2++) {
              const double d = norm3(X[i1] - X[i2 - 1], Y[i1] - Y[i2 - 1], Z[i1] - Z[i2 - 1]);
              if (d < 2 * hh) {
                /* cubic_spline_kernel (stat.jl:217-227) */
                const double q = d / hh;
                double w;
                if (q < 1) w = factor * (1 - 1.5 * (q * q) + 0.75 * (q * q * q));
                else if (q < 2) w = factor * 0.25 * ((2 - q) * (2 - q) * (2 - q));
                else w = 0.0;
                rho += w;
              }
            }
          }
    }
    rho_out[i1] = rho;
  }
  return LCS_OK;
}
int lcs_particles_boundary(lcs_handle* h, int32_t s, int32_t stage) {
  int rc = check_species(h, s);
  if (rc) return rc;
  particles_boundary(h, s, stage);
  return LCS_OK;
}
int lcs_particles_motion(lcs_handle* h, int32_t s, int32_t stage) {
  int rc = check_species(h, s);
  if (rc) return rc;
  particles_motion(h, s, stage);
  return LCS_OK;
}
int lcs_particles_update(lcs_handle* h, int32_t s, int32_t stage, double dtrk) {
  int rc = check_species(h, s);
  if (rc) return rc;
  particles_update(h, s, stage, dtrk);
  return LCS_OK;
}
int lcs_init_particle_velocity(lcs_handle* h, int32_t s) {
  int rc = check_species(h, s);
  if (rc) return rc;
  const grid_t* g = &h->g;
  synchalo(g, h->U, g->h, 1); synchalo(g, h->V, g->h, 1); synchalo(g, h->W, g->h, 1);
  species_t* sp = &h->sp[s];
  const double dx = spacing(g, 0), dy = spacing(g, 1), dz = spacing(g, 2);
  for (int64_t p = 0; p < sp->n; p++) {
    double x = sp->p[LCS_PROP_X][p], y = sp->p[LCS_PROP_Y][p], z = sp->p[LCS_PROP_Z][p];
    sp->p[LCS_PROP_U][p] = interp(g, h->U, xmapping(x, y, z, dx, dy, dz));
    sp->p[LCS_PROP_V][p] = interp(g, h->V, ymapping(x, y, z, dx, dy, dz));
    sp->p[LCS_PROP_W][p] = interp(g, h->W, zmapping(x, y, z, dx, dy, dz));
  }
  return LCS_OK;
}

/* profiling is a device concept; the oracle reports nothing */
int lcs_profile_enable(lcs_handle* h, int32_t on) { (void)on; return h ? LCS_OK : LCS_EINVAL; }
int lcs_profile_reset(lcs_handle* h) { return h ? LCS_OK : LCS_EINVAL; }
int lcs_profile_count(lcs_handle* h, int32_t* n) { if (!h || !n) return LCS_EINVAL; *n = 0; return LCS_OK; }
int lcs_profile_entry(lcs_handle* h, int32_t i, char* name, int32_t cap, double* ms, int64_t* launches) {
  (void)i; (void)name; (void)cap; (void)ms; (void)launches;
  return h ? LCS_EINVAL : LCS_EINVAL;
}
int lcs_launch_count(lcs_handle* h, int64_t* n) { if (!h || !n) return LCS_EINVAL; *n = 0; return LCS_OK; }
int lcs_synchronize(lcs_handle* h) { return h ? LCS_OK : LCS_EINVAL; }

/* ---- oracle-only helpers for the known-answer tests -------------------- */
int lcs_oracle_kcount(int k0) { return kcount(k0); }
/* test hooks of the cell index: the binary searches and the hasher */
void lcs_oracle_searchsorted(const int64_t* v, int64_t n, int64_t x, int64_t* first, int64_t* last) {
  *first = sorted_first(v, n, x);
  *last = sorted_last(v, n, x);
}
int64_t lcs_oracle_cell_encode(const int64_t len[3], const int32_t ci[3]) {
  const int c[3] = {ci[0], ci[1], ci[2]};
  return encode_cell(len, c);
}
void lcs_oracle_cell_decode(const int64_t len[3], int64_t hash, int32_t ci[3]) {
  const int nc[3] = {(int)len[0] - 2, (int)len[1] - 2, (int)len[2] - 2};
  int c[3];
  decode_cell(hash, nc, c);
  for (int a = 0; a < 3; a++) ci[a] = c[a];
}
int lcs_oracle_kset(int k0, int32_t* out, int cap) {
  int tmp[256][3];
  int n = kset(k0, tmp, cap < 256 ? cap : 256);
  for (int q = 0; q < n; q++) { out[3 * q] = tmp[q][0]; out[3 * q + 1] = tmp[q][1]; out[3 * q + 2] = tmp[q][2]; }
  return n;
}
double lcs_oracle_enespe0(int k0, double e10) { return enespe0(k0, e10); }
/* boxmean_l! on a haloed array (n+2h)^3 into coarse c^3 */
void lcs_oracle_boxmean(const double* A, int n, int h, int c, double* out) {
  grid_t g;
  for (int a = 0; a < 3; a++) { g.n[a] = n; g.s[a] = n + 2 * h; }
  g.h = h;
  int f = n / c;
  double w = 1.0 / (double)(f * f * f);
  for (int kc = 1; kc <= c; kc++)
    for (int jc = 1; jc <= c; jc++)
      for (int ic = 1; ic <= c; ic++) {
        double s = 0.0;
        for (int dk = 1; dk <= f; dk++)
          for (int dj = 1; dj <= f; dj++)
            for (int di = 1; di <= f; di++) s += A[IX(&g, (ic - 1) * f + di, (jc - 1) * f + dj, (kc - 1) * f + dk)];
        out[((kc - 1) * c + (jc - 1)) * c + (ic - 1)] = s * w;
      }
}
/* sirdft of a cropped spectrum Ac[kz][ky][kx] (sizes 2kmax+1, 2kmax+1, kmax+1) at phases ei,ej,ek */
double lcs_oracle_sirdft(const double* Ac_reim, int kmin, int kmax, double eir, double eii, double ejr, double eji,
                         double ekr, double eki) {
  int ks[256][3];
  const int KX = kmax + 1, KY = 2 * kmax + 1;
  cplx ei = {eir, eii}, ej = {ejr, eji}, ek = {ekr, eki};
  double tot = 0.0;
  for (int K = kmin; K <= kmax; K++) {
    int n = kset(K, ks, 256);
    double acc = 0.0;
    for (int q = 0; q < n; q++) {
      int kx = ks[q][0], ky = ks[q][1], kz = ks[q][2];
      cplx fx, fy, fz, prod;
      int hx = powi(ei, kx, &fx), hy = powi(ej, ky, &fy), hz = powi(ek, kz, &fz), have = 0;
      if (hx) { prod = fx; have = 1; }
      if (hy) { prod = have ? cmul(prod, fy) : fy; have = 1; }
      if (hz) { prod = have ? cmul(prod, fz) : fz; have = 1; }
      if (!have) { prod.re = 1.0; prod.im = 0.0; }
      size_t idx = ((size_t)(kz + kmax) * KY + (ky + kmax)) * KX + kx;
      acc += 2.0 * (Ac_reim[2 * idx] * prod.re - Ac_reim[2 * idx + 1] * prod.im);
    }
    tot += acc;
  }
  return tot;
}
void lcs_oracle_sincospi(double x, double* s, double* c) { sincospi_host(x, s, c); }
int lcs_oracle_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
/* Cells a colour phase of foraxes visits on the box lo..hi (dense, x fastest). */
int lcs_oracle_color_mask(int coloring, int block, const int32_t* lo, const int32_t* hi, int color, int32_t* out) {
  const int lx = hi[0] - lo[0] + 1, ly = hi[1] - lo[1] + 1, lz = hi[2] - lo[2] + 1;
  memset(out, 0, sizeof(int32_t) * (size_t)lx * ly * lz);
  if (coloring == LCS_COLORING_RED_BLACK_BLOCK) {
    const int nb[3] = {(lx + block - 1) / block, (ly + block - 1) / block, (lz + block - 1) / block};
    for (int bk = 1; bk <= nb[2]; bk++)
      for (int bj = 1; bj <= nb[1]; bj++)
        for (int bi = 1; bi <= nb[0]; bi++) {
          if ((bi + bj + bk) % 2 != color) continue;
          for (int lk = 1; lk <= block; lk++)
            for (int lj = 1; lj <= block; lj++)
              for (int li = 1; li <= block; li++) {
                int i = lo[0] + block * (bi - 1) + li - 1, j = lo[1] + block * (bj - 1) + lj - 1,
                    k = lo[2] + block * (bk - 1) + lk - 1;
                if (i <= hi[0] && j <= hi[1] && k <= hi[2])
                  out[((size_t)(k - lo[2]) * ly + (j - lo[1])) * lx + (i - lo[0])] = 1;
              }
        }
    return 0;
  }
  for (int k = lo[2]; k <= hi[2]; k++)
    for (int j = lo[1]; j <= hi[1]; j++)
      for (int i = lo[0]; i <= hi[0]; i++)
        if (coloring == LCS_COLORING_NO || in_color(coloring, i, j, k, color))
          out[((size_t)(k - lo[2]) * ly + (j - lo[1])) * lx + (i - lo[0])] = 1;
  return 0;
}
double lcs_oracle_enespe(const double* hat_reim, int kmax, int k0, double norm) {
  return enespe_cropped((const cplx*)hat_reim, kmax, k0, norm);
}
double lcs_oracle_phase_shift(int n, int coarse_size) { return (double)(n / coarse_size) / 2.0; }

/* The same dt as lcs_flow_timestep, on caller-owned (here: host) arrays in the
 * reference's haloed layout, reading the interior with periodic wrapping. */
int lcs_flow_timestep_noalloc(const double* U, const double* V, const double* W, const int32_t dims[3],
                              int32_t halo, double cfl, double dtmax, double Re, double* dt_out, void* stream) {
  (void)stream;
  if (!U || !V || !W || !dims || !dt_out) return fail(NULL, LCS_EINVAL, "null argument");
  if (dims[2] > LCS_NOALLOC_MAX_PLANES) return fail(NULL, LCS_EINVAL, "dims[2] exceeds LCS_NOALLOC_MAX_PLANES");
  grid_t g;
  for (int a = 0; a < 3; a++) { g.n[a] = dims[a]; g.s[a] = dims[a] + 2 * halo; }
  g.h = halo;
  double mx[3] = {0, 0, 0};
  for (int k = 1; k <= g.n[2]; k++)
    for (int j = 1; j <= g.n[1]; j++)
      for (int i = 1; i <= g.n[0]; i++) {
        const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
        double uc = interp_o4_at_half(U[IX(&g, wrap1(i - 2, nx), j, k)], U[IX(&g, wrap1(i - 1, nx), j, k)],
                                      U[IX(&g, i, j, k)], U[IX(&g, wrap1(i + 1, nx), j, k)]);
        double vc = interp_o4_at_half(V[IX(&g, i, wrap1(j - 2, ny), k)], V[IX(&g, i, wrap1(j - 1, ny), k)],
                                      V[IX(&g, i, j, k)], V[IX(&g, i, wrap1(j + 1, ny), k)]);
        double wc = interp_o4_at_half(W[IX(&g, i, j, wrap1(k - 2, nz))], W[IX(&g, i, j, wrap1(k - 1, nz))],
                                      W[IX(&g, i, j, k)], W[IX(&g, i, j, wrap1(k + 1, nz))]);
        mx[0] = jl_max(mx[0], fabs(uc));
        mx[1] = jl_max(mx[1], fabs(vc));
        mx[2] = jl_max(mx[2], fabs(wc));
      }
  double dx = DOMAIN_LENGTH / g.n[0], dy = DOMAIN_LENGTH / g.n[1], dz = DOMAIN_LENGTH / g.n[2];
  double d = dtmax;
  d = jl_min(d, cfl * dx / (mx[0] + 1e-10));
  d = jl_min(d, cfl * dy / (mx[1] + 1e-10));
  d = jl_min(d, cfl * dz / (mx[2] + 1e-10));
  d = jl_min(d, 0.5 * ((dx / 2.0) * (dx / 2.0)) / (1.0 / Re));
  *dt_out = d;
  return LCS_OK;
}
