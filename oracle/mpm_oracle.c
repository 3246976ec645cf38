/*
 * mpm_oracle.c — CPU restatement of Matter's explicit MPM time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it.
 * The product (libmatter_gpu.so) never links or calls it.
 *
 * It restates, in plain C with run-time dim (2|3) and spline degree (2|3),
 * the per-step algorithm of the reference's src/simulation/*.cpp and
 * src/plasticity_helpers/*.hpp (paths relative to the reference project);
 * each function cites the file:line it follows.  Arithmetic is FP64 and the
 * operation order follows the reference expression by expression, so that the
 * restatement agrees with the reference compiled from source (oracle/_ref/,
 * built by oracle/Makefile) bit for bit.  Matrices are stored per particle
 * column-major like Eigen's TM.
 *
 * Pinned against: the reference compiled from its own sources, 3D and 2D,
 * quadratic and cubic (the 2D builds compile a copy of src/ in which the
 * `#define THREEDIM` of tools.hpp:20 is commented out), by
 * tests/test_oracle_pin.py.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/matter_gpu.h"

#define MAXP 16
#define MAXO 16

typedef struct orc {
  mtr_params P;
  int dim, deg;
  uint32_t Np;
  /* particle state, AoS like data_structures.hpp:8-47 */
  double *x, *v, *pic, *flip, *F, *B, *dPsidF, *Fe;
  double *eps_pl_dev, *eps_pl_vol, *eps_pl_vol_pradhana, *delta_gamma, *viscosity, *muI;
  uint32_t* keys; /* blocked cell key of each particle at the last step (GPU sort key) */
  /* periodic ghosts of this step (PBCAddParticles, pbc.cpp:37-85): source particle and position */
  uint32_t ng;
  uint32_t* gsrc;
  double* gpos;
  /* grid, data_structures.hpp:49-66 */
  double *gx, *gy, *gz;
  uint32_t Nx, Ny, Nz, G;
  size_t cap_axis[3], cap_nodes;
  double xc, yc, zc;
  double *gmass, *gv, *gflip, *gfric;
  /* remesh bookkeeping, simulation.hpp:206-224 */
  double min_init[3], max_init[3], low_init[3], high_init[3];
  /* objects */
  int nplates, nobjects;
  mtr_plate plates[MAXP];
  mtr_object objects[MAXO];
  /* dense level sets of MTR_OBJ_LEVELSET objects (orc_set_levelset) */
  struct {
    float *phi, *grad;
    uint32_t n[3];
    double org[3], h, inv_h, background;
  } ls[MTR_MAX_LEVELSETS];
  /* constants derived in simulate(), simulation.cpp:94-136 */
  double lambda, mu, K, wave_speed, dt_max, frame_dt, final_time;
  double one_over_dx, one_over_dx_square, apicDinverse;
  double q_prefac, d_prefac, e_mu_prefac, f_mu_prefac, rma_prefac, fac_Q;
  double gravity[3], gravity_final[3];
  /* clock */
  double time, dt;
  uint32_t step, frame;
  int done, exit_flag;
  uint32_t status;
  uint64_t plastic_count;
} orc;

/* ------------------------------------------------------------------------ */
/* small helpers                                                             */
/* ------------------------------------------------------------------------ */

static int sgn(double v) { return (0.0 < v) - (v < 0.0); } /* tools.hpp:90-92 */

static double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */
static double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */

typedef double M3[3][3];

static void m_load(int d, const double* src, M3 A) {
  for (int c = 0; c < d; ++c)
    for (int r = 0; r < d; ++r) A[r][c] = src[c * d + r];
}
static void m_store(int d, M3 A, double* dst) {
  for (int c = 0; c < d; ++c)
    for (int r = 0; r < d; ++r) dst[c * d + r] = A[r][c];
}
static void m_mul(int d, M3 A, M3 B, M3 C) { /* C = A*B */
  M3 T;
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) {
      double s = A[i][0] * B[0][j];
      for (int k = 1; k < d; ++k) s += A[i][k] * B[k][j];
      T[i][j] = s;
    }
  memcpy(C, T, sizeof(M3));
}
static void m_mul_bt(int d, M3 A, M3 B, M3 C) { /* C = A*B^T */
  M3 T;
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) {
      double s = A[i][0] * B[j][0];
      for (int k = 1; k < d; ++k) s += A[i][k] * B[j][k];
      T[i][j] = s;
    }
  memcpy(C, T, sizeof(M3));
}
static void m_eye(M3 A) {
  memset(A, 0, sizeof(M3));
  A[0][0] = A[1][1] = A[2][2] = 1.0;
}
static double m_det(int d, M3 A) {
  if (d == 2) return A[0][0] * A[1][1] - A[0][1] * A[1][0];
  return A[0][0] * (A[1][1] * A[2][2] - A[2][1] * A[1][2]) -
         A[1][0] * (A[0][1] * A[2][2] - A[2][1] * A[0][2]) +
         A[2][0] * (A[0][1] * A[1][2] - A[1][1] * A[0][2]);
}
static void m_inv(int d, M3 A, M3 R) { /* cofactor inverse */
  double det = m_det(d, A);
  M3 T;
  if (d == 2) {
    T[0][0] = A[1][1] / det; T[0][1] = -A[0][1] / det;
    T[1][0] = -A[1][0] / det; T[1][1] = A[0][0] / det;
  } else {
    T[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) / det;
    T[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) / det;
    T[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) / det;
    T[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) / det;
    T[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) / det;
    T[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) / det;
    T[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) / det;
    T[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) / det;
    T[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) / det;
  }
  memcpy(R, T, sizeof(M3));
}

/* ------------------------------------------------------------------------ */
/* SVD: two-sided cyclic Jacobi (Golub & Van Loan, 4th ed., §8.6.3 with the  */
/* 2x2 symmetrising rotation of §8.6.2 and symSchur2 of Alg. 8.5.1).         */
/* Output convention of Eigen::JacobiSVD as called at plasticity.cpp:19 and  */
/* simulation.hpp:232: singular values >= 0 in decreasing order, U and V     */
/* orthogonal (either may have determinant -1), A = U diag(S) V^T.           */
/* ------------------------------------------------------------------------ */
void orc_svd(int d, const double* Acm, double* Ucm, double* S, double* Vcm) {
  M3 A, U, V;
  m_load(d, Acm, A);
  m_eye(U);
  m_eye(V);
  double scale = 0.0;
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) scale = dmax(scale, fabs(A[i][j]));
  if (scale == 0.0 || !isfinite(scale)) scale = 1.0;
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) A[i][j] /= scale;
  double maxdiag = 0.0;
  for (int i = 0; i < d; ++i) maxdiag = dmax(maxdiag, fabs(A[i][i]));
  for (int sweep = 0; sweep < 64; ++sweep) {
    int rotated = 0;
    for (int p = 1; p < d; ++p) {
      for (int q = 0; q < p; ++q) {
        double thr = dmax(DBL_MIN, 2.0 * DBL_EPSILON * maxdiag);
        if (!(fabs(A[p][q]) > thr || fabs(A[q][p]) > thr)) continue;
        rotated = 1;
        double a = A[q][q], b = A[q][p], c = A[p][q], e = A[p][p];
        /* symmetrising rotation G1 = [c1 s1; -s1 c1]: (G1^T M) symmetric */
        double c1 = 1.0, s1 = 0.0;
        double tr = a + e, df = b - c;
        if (fabs(df) >= DBL_MIN) {
          double u = tr / df;
          double r = sqrt(1.0 + u * u);
          s1 = 1.0 / r;
          c1 = u / r;
        }
        double m00 = c1 * a - s1 * c;
        double m01 = c1 * b - s1 * e;
        double m11 = s1 * b + c1 * e;
        /* symmetric Schur rotation J = [cj sj; -sj cj] */
        double cj = 1.0, sj = 0.0;
        if (m01 != 0.0) {
          double tau = (m11 - m00) / (2.0 * m01);
          double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
          cj = 1.0 / sqrt(1.0 + t * t);
          sj = t * cj;
        }
        /* L = G1 * J */
        double l00 = c1 * cj - s1 * sj, l01 = c1 * sj + s1 * cj;
        double l10 = -s1 * cj - c1 * sj, l11 = -s1 * sj + c1 * cj;
        /* rows q,p of A <- L^T * rows */
        for (int k = 0; k < d; ++k) {
          double aq = A[q][k], ap = A[p][k];
          A[q][k] = l00 * aq + l10 * ap;
          A[p][k] = l01 * aq + l11 * ap;
        }
        /* cols q,p of A <- cols * J */
        for (int k = 0; k < d; ++k) {
          double aq = A[k][q], ap = A[k][p];
          A[k][q] = cj * aq - sj * ap;
          A[k][p] = sj * aq + cj * ap;
        }
        for (int k = 0; k < d; ++k) {
          double uq = U[k][q], up = U[k][p];
          U[k][q] = l00 * uq + l10 * up;
          U[k][p] = l01 * uq + l11 * up;
          double vq = V[k][q], vp = V[k][p];
          V[k][q] = cj * vq - sj * vp;
          V[k][p] = sj * vq + cj * vp;
        }
        maxdiag = dmax(maxdiag, dmax(fabs(A[p][p]), fabs(A[q][q])));
      }
    }
    if (!rotated) break;
  }
  double s[3];
  for (int i = 0; i < d; ++i) {
    double a = A[i][i];
    s[i] = fabs(a) * scale;
    if (a < 0.0)
      for (int k = 0; k < d; ++k) U[k][i] = -U[k][i];
  }
  /* decreasing order */
  for (int i = 0; i < d - 1; ++i) {
    int m = i;
    for (int j = i + 1; j < d; ++j)
      if (s[j] > s[m]) m = j;
    if (m != i) {
      double t = s[i]; s[i] = s[m]; s[m] = t;
      for (int k = 0; k < d; ++k) {
        t = U[k][i]; U[k][i] = U[k][m]; U[k][m] = t;
        t = V[k][i]; V[k][i] = V[k][m]; V[k][m] = t;
      }
    }
  }
  for (int i = 0; i < d; ++i) S[i] = s[i];
  m_store(d, U, Ucm);
  m_store(d, V, Vcm);
}

static void svd_m(int d, M3 A, M3 U, double* S, M3 V) {
  double a[9], u[9], v[9];
  m_store(d, A, a);
  orc_svd(d, a, u, S, v);
  m_load(d, u, U);
  m_load(d, v, V);
}

/* U * diag(e) * V^T, as written at plasticity.cpp:44 and friends */
static void usv(int d, M3 U, const double* e, M3 V, M3 out) {
  M3 UD;
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) UD[i][j] = U[i][j] * e[j];
  m_mul_bt(d, UD, V, out);
}

/* ------------------------------------------------------------------------ */
/* B-spline basis, tools.hpp:108-188                                         */
/* ------------------------------------------------------------------------ */
static double Nq(double u) { /* quadratic, tools.hpp:151-162 */
  double a = fabs(u);
  if (a < 0.5) return 0.75 - a * a;
  if (a < 1.5) return 0.5 * (1.5 - a) * (1.5 - a);
  return 0.0;
}
static double dNq(double u) { /* tools.hpp:164-175 */
  double a = fabs(u);
  if (a < 0.5) return -2 * u;
  if (a < 1.5) return u - 1.5 * sgn(u);
  return 0.0;
}
static double Nc(double u) { /* cubic, tools.hpp:110-121 */
  double a = fabs(u);
  if (a < 1.0) return 0.5 * a * a * a - a * a + 2.0 / 3.0;
  if (a < 2.0) return (1.0 / 6.0) * (2.0 - a) * (2.0 - a) * (2.0 - a);
  return 0.0;
}
static double dNc(double u) { /* tools.hpp:123-134 */
  double a = fabs(u);
  if (a < 1.0) return u * (1.5 * a - 2.0);
  if (a < 2.0) return -0.5 * sgn(u) * (2.0 - a) * (2.0 - a);
  return 0.0;
}
static inline double Nb(const orc* s, double u) { return s->deg == 3 ? Nc(u) : Nq(u); }
static inline double dNb(const orc* s, double u) { return s->deg == 3 ? dNc(u) : dNq(u); }

/* wip, tools.hpp:222-224 (3D) and :243-245 (2D) */
static double wip(const orc* s, const double* xp, const double* xi) {
  double ioh = s->one_over_dx;
  double w = Nb(s, (xp[0] - xi[0]) * ioh) * Nb(s, (xp[1] - xi[1]) * ioh);
  if (s->dim == 3) w = w * Nb(s, (xp[2] - xi[2]) * ioh);
  return w;
}
/* grad_wip, tools.hpp:226-232 (3D) and :247-252 (2D) */
static void grad_wip(const orc* s, const double* xp, const double* xi, double* g) {
  double ioh = s->one_over_dx;
  double ux = (xp[0] - xi[0]) * ioh, uy = (xp[1] - xi[1]) * ioh;
  if (s->dim == 3) {
    double uz = (xp[2] - xi[2]) * ioh;
    g[0] = dNb(s, ux) * Nb(s, uy) * Nb(s, uz) * ioh;
    g[1] = dNb(s, uy) * Nb(s, ux) * Nb(s, uz) * ioh;
    g[2] = dNb(s, uz) * Nb(s, ux) * Nb(s, uy) * ioh;
  } else {
    g[0] = dNb(s, ux) * Nb(s, uy) * ioh;
    g[1] = dNb(s, uy) * Nb(s, ux) * ioh;
  }
}

static inline uint32_t gind(const orc* s, int i, int j, int k) { /* simulation.hpp:196-204 */
  return s->dim == 3 ? ((uint32_t)i * s->Ny + (uint32_t)j) * s->Nz + (uint32_t)k
                     : (uint32_t)i * s->Ny + (uint32_t)j;
}

/* ------------------------------------------------------------------------ */
/* grid construction: arange (tools.hpp:291-296), remesh.cpp                 */
/* ------------------------------------------------------------------------ */
static double* arange(double start, double stop, double step, uint32_t* n, double* buf,
                      size_t* cap) {
  uint32_t cnt = 0;
  for (double value = start; value < stop; value += step) {
    if (cnt >= *cap) {
      *cap = (*cap ? *cap * 2 : 256);
      buf = (double*)realloc(buf, *cap * sizeof(double));
    }
    buf[cnt++] = value;
  }
  *n = cnt;
  return buf;
}

static void set_grid_axes(orc* s, const double* low, const double* high) {
  double dx = s->P.dx;
  s->gx = arange(low[0], high[0] + dx, dx, &s->Nx, s->gx, &s->cap_axis[0]);
  s->gy = arange(low[1], high[1] + dx, dx, &s->Ny, s->gy, &s->cap_axis[1]);
  if (s->dim == 3)
    s->gz = arange(low[2], high[2] + dx, dx, &s->Nz, s->gz, &s->cap_axis[2]);
  else
    s->Nz = 1;
  s->xc = s->gx[0];
  s->yc = s->gy[0];
  s->zc = s->dim == 3 ? s->gz[0] : 0.0;
  s->G = s->Nx * s->Ny * s->Nz;
}

/* per-axis max/min of particle positions (remesh.cpp:42-83 std::max_element) */
static void particle_bbox(const orc* s, double* mn, double* mx) {
  int d = s->dim;
  for (int a = 0; a < d; ++a) {
    mn[a] = s->x[a];
    mx[a] = s->x[a];
  }
  for (uint32_t p = 1; p < s->Np; ++p)
    for (int a = 0; a < d; ++a) {
      double v = s->x[(size_t)p * d + a];
      if (mx[a] < v) mx[a] = v;
      if (v < mn[a]) mn[a] = v;
    }
}

/* remeshFixed(extra_nodes), remesh.cpp:14-36: the fixed grid of periodic runs */
static void remesh_fixed(orc* s, unsigned int extra) {
  double dx = s->P.dx;
  double e1 = (double)(1 + extra), e2 = (double)(2 + extra);
  s->gx = arange(-dx * e1, s->P.L[0] + e2 * dx, dx, &s->Nx, s->gx, &s->cap_axis[0]);
  s->gy = arange(-dx, s->P.L[1] + e2 * dx, dx, &s->Ny, s->gy, &s->cap_axis[1]);
  if (s->dim == 3)
    s->gz = arange(-dx * e1, s->P.L[2] + e2 * dx, dx, &s->Nz, s->gz, &s->cap_axis[2]);
  else
    s->Nz = 1;
  s->xc = s->gx[0];
  s->yc = s->gy[0];
  s->zc = s->dim == 3 ? s->gz[0] : 0.0;
  s->G = s->Nx * s->Ny * s->Nz;
}

/* PBCAddParticles(safety_factor), pbc.cpp:37-85: a particle within
 * safety_factor * dx of x = Lx (else of x = 0) gets a copy shifted by -Lx
 * (else +Lx); copies follow the particles in index order */
static void pbc_add(orc* s, unsigned int safety_factor) {
  int d = s->dim;
  double Lx = s->P.L[0], lim = safety_factor * s->P.dx;
  s->ng = 0;
  s->gsrc = (uint32_t*)realloc(s->gsrc, (s->Np ? s->Np : 1) * sizeof(uint32_t));
  s->gpos = (double*)realloc(s->gpos, (size_t)(s->Np ? s->Np : 1) * d * sizeof(double));
  for (uint32_t p = 0; p < s->Np; ++p) {
    const double* x = s->x + (size_t)p * d;
    double xg0;
    double diff = Lx - x[0];
    if (diff < lim && diff > 0) {
      xg0 = -diff;
    } else {
      diff = x[0];
      if (!(diff < lim && diff >= 0)) continue;
      xg0 = Lx + diff;
    }
    double* g = s->gpos + (size_t)s->ng * d;
    for (int a = 0; a < d; ++a) g[a] = x[a];
    g[0] = xg0;
    s->gsrc[s->ng++] = p;
  }
}

/* remeshFixedInit(2,2,2), remesh.cpp:38-182 */
static void remesh_init(orc* s) {
  int d = s->dim;
  double mn[3], mx[3];
  particle_bbox(s, mn, mx);
  const double* grp = s->P.grid_reference_point;
  if (grp[0] < 1e10) { /* remesh.cpp:88-109 */
    for (int a = 0; a < d; ++a) {
      if (grp[a] < mn[a])
        mn[a] = grp[a];
      else if (grp[a] > mx[a])
        mx[a] = grp[a];
    }
  }
  double low[3], high[3];
  for (int a = 0; a < d; ++a) {
    s->max_init[a] = mx[a];
    s->min_init[a] = mn[a];
    s->low_init[a] = mn[a] - s->P.dx * 2.0;
    s->high_init[a] = mx[a] + s->P.dx * 2.0;
    low[a] = s->low_init[a];
    high[a] = s->high_init[a];
  }
  set_grid_axes(s, low, high);
}

/* remeshFixedCont, remesh.cpp:184-311 */
static void remesh_cont(orc* s) {
  int d = s->dim;
  double dx = s->P.dx;
  double mn[3], mx[3], low[3], high[3];
  particle_bbox(s, mn, mx);
  for (int a = 0; a < d; ++a) {
    if (mx[a] < s->max_init[a]) {
      unsigned int f = (unsigned int)floor(dmax(0.0, (s->max_init[a] - mx[a]) / dx - 1e-8 * dx));
      high[a] = s->high_init[a] - f * dx;
    } else {
      unsigned int f = (unsigned int)floor(dmax(0.0, (mx[a] - s->max_init[a]) / dx - 1e-8 * dx));
      high[a] = s->high_init[a] + f * dx;
    }
    if (mn[a] > s->min_init[a]) {
      unsigned int f = (unsigned int)floor(dmax(0.0, (mn[a] - s->min_init[a]) / dx - 1e-8 * dx));
      low[a] = s->low_init[a] + f * dx;
    } else {
      unsigned int f = (unsigned int)floor(dmax(0.0, (s->min_init[a] - mn[a]) / dx - 1e-8 * dx));
      low[a] = s->low_init[a] - f * dx;
    }
  }
  set_grid_axes(s, low, high);
}

/* resizeGrid, remesh.cpp:5-11 */
static void resize_grid(orc* s) {
  if (s->G > s->cap_nodes) {
    s->cap_nodes = s->G + s->G / 2;
    s->gmass = (double*)realloc(s->gmass, s->cap_nodes * sizeof(double));
    s->gfric = (double*)realloc(s->gfric, s->cap_nodes * sizeof(double));
    s->gv = (double*)realloc(s->gv, s->cap_nodes * 3 * sizeof(double));
    s->gflip = (double*)realloc(s->gflip, s->cap_nodes * 3 * sizeof(double));
  }
  memset(s->gmass, 0, s->G * sizeof(double));
  memset(s->gfric, 0, s->G * sizeof(double));
  memset(s->gv, 0, (size_t)s->G * s->dim * sizeof(double));
  memset(s->gflip, 0, (size_t)s->G * s->dim * sizeof(double));
}

/* Blocked cell key used by the GPU's particle sort: cell c = floor((x-xc)/dx)
 * per axis (the stencil anchor of p2g.cpp:21-24 before its -1), tiles of 4^3
 * cells in 3D and 8^2 in 2D, key = tile_linear * 64 + cell_in_tile. */
static void compute_keys(orc* s) {
  int d = s->dim;
  int tb = d == 3 ? 4 : 8, sh = d == 3 ? 2 : 3;
  uint32_t TY = (s->Ny + tb - 1) / tb, TZ = d == 3 ? (s->Nz + tb - 1) / tb : 1;
  double org[3] = {s->xc, s->yc, s->zc};
  for (uint32_t p = 0; p < s->Np; ++p) {
    int c[3] = {0, 0, 0};
    for (int a = 0; a < d; ++a) c[a] = (int)floor((s->x[(size_t)p * d + a] - org[a]) * s->one_over_dx);
    uint32_t t, in;
    if (d == 3) {
      t = ((uint32_t)(c[0] >> sh) * TY + (uint32_t)(c[1] >> sh)) * TZ + (uint32_t)(c[2] >> sh);
      in = ((uint32_t)(c[0] & 3) * 4 + (uint32_t)(c[1] & 3)) * 4 + (uint32_t)(c[2] & 3);
    } else {
      t = (uint32_t)(c[0] >> sh) * TY + (uint32_t)(c[1] >> sh);
      in = (uint32_t)(c[0] & 7) * 8 + (uint32_t)(c[1] & 7);
    }
    s->keys[p] = t * 64u + in;
  }
}

/* ------------------------------------------------------------------------ */
/* updateDt, update_dt.cpp:5-66                                              */
/* ------------------------------------------------------------------------ */
static void update_dt(orc* s) {
  int d = s->dim;
  double best = -1.0;
  uint32_t bi = 0;
  for (uint32_t p = 0; p < s->Np; ++p) {
    const double* v = s->v + (size_t)p * d;
    double sq = v[0] * v[0] + v[1] * v[1];
    if (d == 3) sq += v[2] * v[2];
    if (p == 0 || best < sq) {
      best = sq;
      bi = p;
    }
  }
  const double* vb = s->v + (size_t)bi * d;
  double sq = vb[0] * vb[0] + vb[1] * vb[1];
  if (d == 3) sq += vb[2] * vb[2];
  double max_speed = sqrt(sq);
  double dt;
  if (fabs(max_speed) > 1e-10) {
    double dt_cfl = s->P.cfl * s->P.dx / max_speed;
    dt = dmin(dt_cfl, s->dt_max);
  } else {
    dt = s->dt_max;
  }
  dt = dmin(dt, s->frame_dt * (s->frame + 1) - s->time);
  dt = dmin(dt, s->final_time - s->time);
  s->dt = dt;
  if (s->P.gravity_special) { /* update_dt.cpp:44-61 */
    if (s->time < s->P.gravity_time) {
      for (int a = 0; a < d; ++a) s->gravity[a] = s->gravity_final[a] * s->time / s->P.gravity_time;
    } else {
      for (int a = 0; a < d; ++a) s->gravity[a] = s->gravity_final[a];
    }
  }
}

/* ------------------------------------------------------------------------ */
/* P2G, p2g.cpp:6-100                                                        */
/* ------------------------------------------------------------------------ */
static void p2g(orc* s) {
  int d = s->dim;
  double org[3] = {s->xc, s->yc, s->zc};
  for (uint32_t it = 0; it < s->Np + s->ng; ++it) {  /* particles, then periodic copies */
    const uint32_t p = it < s->Np ? it : s->gsrc[it - s->Np];
    const double* xp = it < s->Np ? s->x + (size_t)p * d : s->gpos + (size_t)(it - s->Np) * d;
    const double* vp = s->v + (size_t)p * d;
    M3 Bp;
    m_load(d, s->B + (size_t)p * d * d, Bp);
    int base[3] = {0, 0, 0};
    for (int a = 0; a < d; ++a) {
      int b = (int)floor((xp[a] - org[a]) * s->one_over_dx) - 1;
      base[a] = b < 0 ? 0 : b;
    }
    int kn = d == 3 ? 4 : 1;
    for (int i = base[0]; i < base[0] + 4; ++i)
      for (int j = base[1]; j < base[1] + 4; ++j)
        for (int kk = 0; kk < kn; ++kk) {
          int k = base[2] + kk;
          double xi[3] = {s->gx[i], s->gy[j], d == 3 ? s->gz[k] : 0.0};
          double weight = wip(s, xp, xi);
          if (weight > 1e-25) {
            uint32_t id = gind(s, i, j, k);
            s->gmass[id] += weight;
            for (int a = 0; a < d; ++a) s->gv[(size_t)id * d + a] += vp[a] * weight;
            if (s->P.flip_ratio < 0) {
              double pd[3];
              for (int a = 0; a < d; ++a) pd[a] = xi[a] - xp[a];
              for (int a = 0; a < d; ++a) {
                double bv = Bp[a][0] * pd[0];
                for (int c = 1; c < d; ++c) bv += Bp[a][c] * pd[c];
                s->gv[(size_t)id * d + a] += bv * s->apicDinverse * weight;
              }
            }
            if (s->P.use_mibf) s->gfric[id] += s->muI[p] * weight;
          }
        }
  }
  for (uint32_t l = 0; l < s->G; ++l) {
    double mi = s->gmass[l];
    for (int a = 0; a < d; ++a) {
      if (mi > 0)
        s->gv[(size_t)l * d + a] /= mi;
      else
        s->gv[(size_t)l * d + a] = 0.0;
    }
    if (s->P.use_mibf) s->gfric[l] /= mi;
  }
  for (uint32_t l = 0; l < s->G; ++l) s->gmass[l] *= s->P.particle_mass;
}

/* ------------------------------------------------------------------------ */
/* stresses, simulation.hpp:227-238                                          */
/* ------------------------------------------------------------------------ */
static void hencky_piola(orc* s, M3 Fe, M3 P) {
  int d = s->dim;
  M3 U, V;
  double S[3], D[3];
  svd_m(d, Fe, U, S, V);
  double tr = 0.0;
  double lg[3];
  for (int i = 0; i < d; ++i) lg[i] = log(fabs(S[i]));
  tr = lg[0];
  for (int i = 1; i < d; ++i) tr += lg[i];
  for (int i = 0; i < d; ++i) {
    double inv = 1.0 / S[i];
    D[i] = 2 * s->mu * inv * lg[i] + s->lambda * tr * inv;
  }
  usv(d, U, D, V, P);
}
static void neohookean_piola(orc* s, M3 Fe, M3 P) {
  int d = s->dim;
  M3 FT, FinvT; /* inverse of the transpose, in that order (simulation.hpp:228) */
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) FT[i][j] = Fe[j][i];
  m_inv(d, FT, FinvT);
  double lj = log(m_det(d, Fe));
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j)
      P[i][j] = s->mu * (Fe[i][j] - FinvT[i][j]) + s->lambda * lj * FinvT[i][j];
}

/* ------------------------------------------------------------------------ */
/* boundary collision, boundary_collision.cpp:5-394 and object_*.hpp         */
/* ------------------------------------------------------------------------ */
/* Dense level set: the signed distance an ObjectVdb samples (object_vdb.hpp:
 * 17-94) on a uniform lattice.  Trilinear (2D: bilinear) sample in index
 * coordinates u = (X - org) / h with weights u - floor(u) and
 * lerp(a, b, w) = a + w (b - a) along x, then y, then z (OpenVDB's
 * BoxSampler); lattice points outside read `outside`. */
static double ls_sample(const orc* s, int slot, const float* f, int stride, int comp, const double* X,
                        double outside) {
  int d = s->dim;
  int i0[3] = {0, 0, 0};
  double w[3] = {0.0, 0.0, 0.0};
  for (int a = 0; a < d; ++a) {
    double u = (X[a] - s->ls[slot].org[a]) * s->ls[slot].inv_h;
    double fl = floor(u);
    i0[a] = fl < -2.0 ? -2 : (fl > 2.0e9 ? 2000000000 : (int)fl);
    w[a] = u - fl;
  }
  double c[8];
  for (int q = 0; q < 8; ++q) {
    int i = i0[0] + (q & 1), j = i0[1] + ((q >> 1) & 1), k = i0[2] + ((q >> 2) & 1);
    if (d == 2 && (q >> 2)) {
      c[q] = 0.0;
      continue;
    }
    const uint32_t* n = s->ls[slot].n;
    if (i < 0 || j < 0 || k < 0 || i >= (int)n[0] || j >= (int)n[1] || k >= (int)n[2])
      c[q] = outside;
    else
      c[q] = (double)f[(((size_t)i * n[1] + j) * n[2] + k) * stride + comp];
  }
#define LERP(a, b, t) ((a) + (t) * ((b) - (a)))
  double c0 = LERP(c[0], c[1], w[0]), c1 = LERP(c[2], c[3], w[0]);
  if (d == 2) return LERP(c0, c1, w[1]);
  double c2 = LERP(c[4], c[5], w[0]), c3 = LERP(c[6], c[7], w[0]);
  return LERP(LERP(c0, c1, w[1]), LERP(c2, c3, w[1]), w[2]);
#undef LERP
}

static int obj_inside(const orc* s, const mtr_object* o, const double* X) {
  double x = X[0], y = X[1];
  switch (o->kind) {
    case MTR_OBJ_LEVELSET: { /* object_vdb.hpp:45-57: phi <= 0 */
      int sl = (int)o->prm[0];
      return ls_sample(s, sl, s->ls[sl].phi, 1, 0, X, s->ls[sl].background) <= 0.0;
    }
    case MTR_OBJ_BUMP: return y < 0.0475 / cosh(25 * (x - 0.43)); /* object_bump.hpp:15-27 */
    case MTR_OBJ_GROUND: return !(y > o->prm[0]);                 /* object_ground.hpp:16-25 */
    case MTR_OBJ_RAMP: return y < 0.1 * tanh(-100 * x);           /* object_ramp.hpp:15-26 */
    case MTR_OBJ_CURVE: return !(y > x * x);                       /* object_curve.hpp:15-25 */
    case MTR_OBJ_GATE: return y > o->prm[0] + 100 * x * x;         /* object_gate.hpp:16-28 */
    case MTR_OBJ_SILO: {                                           /* object_silo.hpp:16-35 */
      double z = X[2];
      if (y < o->prm[0]) return 0;
      double r = tanh(y) + 1;
      return !(x * x + z * z < r * r);
    }
    case MTR_OBJ_BOX_ROTATED: { /* object_box.hpp:18-24 */
      int d = s->dim;
      double loc[3];
      for (int i = 0; i < d; ++i) {
        double acc = 0.0;
        for (int k = 0; k < d; ++k) {
          double Rki = o->prm[6 + i * d + k]; /* R(k,i), column-major */
          acc += Rki * (X[k] - o->prm[k]);
        }
        loc[i] = acc;
      }
      for (int i = 0; i < d; ++i)
        if (fabs(loc[i]) > o->prm[3 + i]) return 0;
      return 1;
    }
    case MTR_OBJ_TERRAIN_GAUSS: {
      double ys = o->prm[0];
      int nb = (int)o->prm[1];
      for (int b = 0; b < nb && b < 4; ++b) {
        const double* q = o->prm + 2 + 4 * b;
        double dxx = x - q[0];
        double r2 = dxx * dxx;
        if (s->dim == 3) {
          double dz = X[2] - q[1];
          r2 += dz * dz;
        }
        ys += q[2] * exp(-r2 / (2.0 * q[3] * q[3]));
      }
      return y < ys;
    }
  }
  return 0;
}

static void normalize(int d, double* n) {
  double sq = n[0] * n[0] + n[1] * n[1];
  if (d == 3) sq += n[2] * n[2];
  double nr = sqrt(sq);
  if (nr > 0)
    for (int a = 0; a < d; ++a) n[a] /= nr;
}

static void obj_normal(const orc* s, const mtr_object* o, const double* X, double* n) {
  int d = s->dim;
  double x = X[0], y = X[1];
  n[0] = n[1] = n[2] = 0.0;
  switch (o->kind) {
    case MTR_OBJ_LEVELSET: { /* object_vdb.hpp:59-78: sampled gradient, normalised */
      int sl = (int)o->prm[0];
      for (int a = 0; a < d; ++a) n[a] = ls_sample(s, sl, s->ls[sl].grad, 3, a, X, 0.0);
      normalize(d, n);
      break;
    }
    case MTR_OBJ_BUMP: { /* object_bump.hpp:29-41 */
      double arg = 25 * (x - 0.43);
      double b_der = -25 * 0.0475 * tanh(arg) / cosh(arg);
      n[0] = -b_der;
      n[1] = 1;
      normalize(d, n);
      break;
    }
    case MTR_OBJ_GROUND: /* object_ground.hpp:27-36 (n(2) left unset there; 0 here) */
      n[0] = 0;
      n[1] = 1;
      break;
    case MTR_OBJ_RAMP: { /* object_ramp.hpp:28-40 */
      double tmp = cosh(-100 * x);
      double b_der = 0.1 * (-100) / (tmp * tmp);
      n[0] = -b_der;
      n[1] = 1;
      normalize(d, n);
      break;
    }
    case MTR_OBJ_CURVE: /* object_curve.hpp:27-37 */
      n[0] = -2 * x;
      n[1] = 1;
      normalize(d, n);
      break;
    case MTR_OBJ_GATE: { /* object_gate.hpp:30-41 */
      double b_der = 2.0 * 100 * x;
      n[0] = -b_der;
      n[1] = 1;
      n[0] *= -1;
      n[1] *= -1;
      normalize(d, n);
      break;
    }
    case MTR_OBJ_SILO: { /* object_silo.hpp:37-54 */
      double z = X[2];
      double theta = atan2(z, x);
      double sech_y = 1.0 / cosh(y);
      n[0] = -cos(theta);
      n[1] = sech_y * sech_y;
      n[2] = -sin(theta);
      normalize(d, n);
      break;
    }
    case MTR_OBJ_BOX_ROTATED: { /* object_box.hpp:26-43 */
      double loc[3];
      for (int i = 0; i < d; ++i) {
        double acc = 0.0;
        for (int k = 0; k < d; ++k) acc += o->prm[6 + i * d + k] * (X[k] - o->prm[k]);
        loc[i] = acc;
      }
      int ca = 0;
      double md = 0.0;
      for (int i = 0; i < d; ++i) {
        double dist = fabs(o->prm[3 + i] - fabs(loc[i]));
        if (dist > md) {
          md = dist;
          ca = i;
        }
      }
      double ln[3] = {0, 0, 0};
      ln[ca] = (loc[ca] > 0) ? 1 : -1;
      for (int r = 0; r < d; ++r) {
        double acc = 0.0;
        for (int k = 0; k < d; ++k) acc += o->prm[6 + k * d + r] * ln[k]; /* R(r,k) */
        n[r] = acc;
      }
      break;
    }
    case MTR_OBJ_TERRAIN_GAUSS: {
      double gxs = 0.0, gzs = 0.0;
      int nb = (int)o->prm[1];
      for (int b = 0; b < nb && b < 4; ++b) {
        const double* q = o->prm + 2 + 4 * b;
        double dxx = x - q[0], dz = d == 3 ? X[2] - q[1] : 0.0;
        double r2 = dxx * dxx;
        if (d == 3) r2 += dz * dz;
        double sg2 = q[3] * q[3];
        double h = q[2] * exp(-r2 / (2.0 * sg2));
        gxs += -h * dxx / sg2;
        gzs += -h * dz / sg2;
      }
      n[0] = -gxs;
      n[1] = 1;
      if (d == 3) n[2] = -gzs;
      normalize(d, n);
      break;
    }
  }
}

static int plate_inside(const orc* s, const mtr_plate* o, const double* X) { /* object_plate.hpp:30-103 */
  switch (o->plate_type) {
    case MTR_PLATE_LEFT: return X[1] < o->pos_upper && X[1] > o->pos_lower && (X[0] - o->pos_object) <= 0;
    case MTR_PLATE_RIGHT: return X[1] < o->pos_upper && X[1] > o->pos_lower && (o->pos_object - X[0]) <= 0;
    case MTR_PLATE_BOTTOM: return X[0] < o->pos_upper && X[0] > o->pos_lower && (X[1] - o->pos_object) <= 0;
    case MTR_PLATE_TOP: return X[0] < o->pos_upper && X[0] > o->pos_lower && (o->pos_object - X[1]) <= 0;
    case MTR_PLATE_BACK: return s->dim == 3 && X[2] - o->pos_object <= 0;
    case MTR_PLATE_FRONT: return s->dim == 3 && o->pos_object - X[2] <= 0;
  }
  return 0;
}

/* Coulomb reduction of two tangential components a,b against normal speed vn
 * (boundary_collision.cpp:103-123 and its five siblings). */
static void coulomb3(double friction, double vn, double* a, double* b) {
  double vel_t = sqrt(*a * *a + *b * *b);
  double fric_vel_n = friction * fabs(vn);
  if (friction == 0) {
  } else if (vel_t <= fric_vel_n) {
    *a = 0;
    *b = 0;
  } else {
    *a = sgn(*a) * (vel_t - fric_vel_n) / sqrt(1 + *b * *b / (*a * *a));
    *b = sgn(*b) * (vel_t - fric_vel_n) / sqrt(1 + *a * *a / (*b * *b));
  }
}
/* 2D variant, boundary_collision.cpp:286-297 */
static void coulomb2(double friction, double vn, double* a) {
  if (friction == 0) {
  } else if (fabs(*a) < friction * fabs(vn)) {
    *a = 0;
  } else {
    if (*a > 0)
      *a -= friction * fabs(vn);
    else
      *a += friction * fabs(vn);
  }
}

static void boundary_collision(orc* s, uint32_t index, const double* Xin, double* vi) {
  int d = s->dim;
  double vi_orig[3] = {vi[0], vi[1], d == 3 ? vi[2] : 0.0};
  double X[3];
  for (int a = 0; a < d; ++a) X[a] = Xin[a] + s->dt * vi[a];
  X[2] = d == 3 ? X[2] : 0.0;
  for (int oi = 0; oi < s->nobjects; ++oi) { /* boundary_collision.cpp:13-79 */
    const mtr_object* o = &s->objects[oi];
    if (!obj_inside(s, o, X)) continue;
    double vr[3] = {vi_orig[0], vi_orig[1], vi_orig[2]};
    if (o->bc == MTR_BC_NOSLIP) {
      vr[0] = vr[1] = vr[2] = 0.0;
    } else if (o->bc == MTR_BC_SLIPFREE) {
      double n[3];
      obj_normal(s, o, X, n);
      double dot = vr[0] * n[0] + vr[1] * n[1];
      if (d == 3) dot += vr[2] * n[2];
      if (dot < 0) {
        double friction = o->friction;
        if (s->P.use_mibf) friction = s->gfric[index];
        double vt[3];
        for (int a = 0; a < d; ++a) vt[a] = vr[a] - dot * n[a];
        if (friction > 0) {
          double sq = vt[0] * vt[0] + vt[1] * vt[1];
          if (d == 3) sq += vt[2] * vt[2];
          double nt = sqrt(sq);
          if (-dot * friction < nt) {
            for (int a = 0; a < d; ++a) vr[a] = vt[a] + (vt[a] / nt) * dot * friction;
          } else {
            vr[0] = vr[1] = vr[2] = 0.0;
          }
        } else {
          for (int a = 0; a < d; ++a) vr[a] = vt[a];
        }
      }
    } else if (o->bc == MTR_BC_SLIPSTICK) {
      double n[3];
      obj_normal(s, o, X, n);
      double dot = vr[0] * n[0] + vr[1] * n[1];
      if (d == 3) dot += vr[2] * n[2];
      for (int a = 0; a < d; ++a) vr[a] = vr[a] - dot * n[a];
      if (dot < 0) {
        double friction = o->friction;
        if (s->P.use_mibf) friction = s->gfric[index];
        if (friction > 0) {
          double sq = vr[0] * vr[0] + vr[1] * vr[1];
          if (d == 3) sq += vr[2] * vr[2];
          double nt = sqrt(sq);
          if (-dot * friction < nt) {
            for (int a = 0; a < d; ++a) vr[a] = vr[a] + (vr[a] / nt) * dot * friction;
          } else {
            vr[0] = vr[1] = vr[2] = 0.0;
          }
        }
      }
    } else {
      s->exit_flag = 1;
      s->status |= MTR_STATUS_BAD_BC;
      return;
    }
    for (int a = 0; a < d; ++a) vi[a] = vr[a];
    for (int a = 0; a < d; ++a) vi_orig[a] = vi[a];
  }
  for (int pi = 0; pi < s->nplates; ++pi) { /* boundary_collision.cpp:84-261 / 267-390 */
    const mtr_plate* o = &s->plates[pi];
    if (!plate_inside(s, o, X)) continue;
    double vx = vi_orig[0] - o->v_object[0];
    double vy = vi_orig[1] - o->v_object[1];
    double vz = d == 3 ? vi_orig[2] - o->v_object[2] : 0.0;
    int pt = o->plate_type;
    if (o->bc == MTR_BC_NOSLIP) {
      vx = vy = vz = 0;
    } else if (o->bc == MTR_BC_SLIPSTICK || o->bc == MTR_BC_SLIPFREE) {
      double friction = o->friction;
      if (s->P.use_mibf) friction = s->gfric[index];
      int stick = o->bc == MTR_BC_SLIPSTICK;
      if (d == 3) {
        if ((stick && (pt == MTR_PLATE_TOP || pt == MTR_PLATE_BOTTOM)) ||
            (!stick && ((pt == MTR_PLATE_TOP && vy > 0) || (pt == MTR_PLATE_BOTTOM && vy < 0)))) {
          coulomb3(friction, vy, &vx, &vz);
          vy = 0;
        } else if ((stick && (pt == MTR_PLATE_LEFT || pt == MTR_PLATE_RIGHT)) ||
                   (!stick && ((pt == MTR_PLATE_LEFT && vx < 0) || (pt == MTR_PLATE_RIGHT && vx > 0)))) {
          coulomb3(friction, vx, &vy, &vz);
          vx = 0;
        } else if ((stick && (pt == MTR_PLATE_FRONT || pt == MTR_PLATE_BACK)) ||
                   (!stick && ((pt == MTR_PLATE_FRONT && vz > 0) || (pt == MTR_PLATE_BACK && vz < 0)))) {
          coulomb3(friction, vz, &vx, &vy);
          vz = 0;
        }
      } else {
        if ((stick && (pt == MTR_PLATE_TOP || pt == MTR_PLATE_BOTTOM)) ||
            (!stick && ((pt == MTR_PLATE_TOP && vy > 0) || (pt == MTR_PLATE_BOTTOM && vy < 0)))) {
          coulomb2(friction, vy, &vx);
          vy = 0;
        } else if ((stick && (pt == MTR_PLATE_LEFT || pt == MTR_PLATE_RIGHT)) ||
                   (!stick && ((pt == MTR_PLATE_LEFT && vx < 0) || (pt == MTR_PLATE_RIGHT && vx > 0)))) {
          coulomb2(friction, vx, &vy);
          vx = 0;
        }
      }
    } else {
      s->exit_flag = 1;
      s->status |= MTR_STATUS_BAD_BC;
      return;
    }
    vi[0] = vx + o->v_object[0];
    vi[1] = vy + o->v_object[1];
    if (d == 3) vi[2] = vz + o->v_object[2];
    for (int a = 0; a < d; ++a) vi_orig[a] = vi[a];
  }
}

/* ------------------------------------------------------------------------ */
/* explicitEulerUpdate, explicit_euler_update.cpp:7-134                     */
/* ------------------------------------------------------------------------ */
static void explicit_euler(orc* s, double* force) {
  int d = s->dim;
  double org[3] = {s->xc, s->yc, s->zc};
  memset(force, 0, (size_t)s->G * d * sizeof(double));
  for (uint32_t it = 0; it < s->Np + s->ng; ++it) {  /* particles, then periodic copies */
    const uint32_t p = it < s->Np ? it : s->gsrc[it - s->Np];
    M3 Fe, dPsidF, tau;
    m_load(d, s->F + (size_t)p * d * d, Fe);
    if (s->P.plastic_model == MTR_PM_SNOW) {
      M3 Fep;
      m_load(d, s->dPsidF + (size_t)p * d * d, dPsidF);
      m_load(d, s->Fe + (size_t)p * d * d, Fep);
      m_mul_bt(d, dPsidF, Fep, tau);
    } else {
      if (s->P.elastic_model == MTR_EL_NEOHOOKEAN)
        neohookean_piola(s, Fe, dPsidF);
      else
        hencky_piola(s, Fe, dPsidF);
      m_mul_bt(d, dPsidF, Fe, tau);
    }
    const double* xp = it < s->Np ? s->x + (size_t)p * d : s->gpos + (size_t)(it - s->Np) * d;
    int base[3] = {0, 0, 0};
    for (int a = 0; a < d; ++a) {
      int b = (int)floor((xp[a] - org[a]) * s->one_over_dx) - 1;
      base[a] = b < 0 ? 0 : b;
    }
    int kn = d == 3 ? 4 : 1;
    for (int i = base[0]; i < base[0] + 4; ++i)
      for (int j = base[1]; j < base[1] + 4; ++j)
        for (int kk = 0; kk < kn; ++kk) {
          int k = base[2] + kk;
          uint32_t id = gind(s, i, j, k);
          if (s->gmass[id] > 0) {
            double xi[3] = {s->gx[i], s->gy[j], d == 3 ? s->gz[k] : 0.0};
            double g[3];
            grad_wip(s, xp, xi, g);
            for (int a = 0; a < d; ++a) {
              double f = tau[a][0] * g[0];
              for (int c = 1; c < d; ++c) f += tau[a][c] * g[c];
              force[(size_t)id * d + a] += f;
            }
          }
        }
  }
  double dtpv = s->dt * s->P.particle_volume;
  double dtg[3];
  for (int a = 0; a < d; ++a) dtg[a] = s->dt * s->gravity[a];
  for (uint32_t i = 0; i < s->Nx; ++i)
    for (uint32_t j = 0; j < s->Ny; ++j)
      for (uint32_t k = 0; k < s->Nz; ++k) {
        uint32_t index = gind(s, i, j, k);
        double mi = s->gmass[index];
        if (mi > 0) {
          double oldv[3], newv[3];
          for (int a = 0; a < d; ++a) {
            double inc = -dtpv * force[(size_t)index * d + a] / mi + dtg[a];
            oldv[a] = s->gv[(size_t)index * d + a];
            newv[a] = oldv[a] + inc;
          }
          double Xi[3] = {s->gx[i], s->gy[j], d == 3 ? s->gz[k] : 0.0};
          boundary_collision(s, index, Xi, newv);
          for (int a = 0; a < d; ++a) {
            s->gv[(size_t)index * d + a] = newv[a];
            s->gflip[(size_t)index * d + a] = newv[a] - oldv[a];
          }
        }
      }
}

/* ------------------------------------------------------------------------ */
/* G2P, g2p.cpp:7-94 (stencil base NOT clamped, g2p.cpp:29)                  */
/* ------------------------------------------------------------------------ */
static void g2p(orc* s) {
  int d = s->dim, dd = d * d;
  double org[3] = {s->xc, s->yc, s->zc};
  double fr = s->P.flip_ratio;
  memset(s->pic, 0, (size_t)s->Np * d * sizeof(double));
  memset(s->flip, 0, (size_t)s->Np * d * sizeof(double));
  memset(s->B, 0, (size_t)s->Np * dd * sizeof(double));
  for (uint32_t p = 0; p < s->Np; ++p) {
    const double* xp = s->x + (size_t)p * d;
    double vp[3] = {0, 0, 0}, fp[3] = {0, 0, 0};
    M3 Bp;
    memset(Bp, 0, sizeof(M3));
    int base[3] = {0, 0, 0};
    for (int a = 0; a < d; ++a) base[a] = (int)(floor((xp[a] - org[a]) * s->one_over_dx) - 1);
    int kn = d == 3 ? 4 : 1;
    for (int i = base[0]; i < base[0] + 4; ++i)
      for (int j = base[1]; j < base[1] + 4; ++j)
        for (int kk = 0; kk < kn; ++kk) {
          int k = base[2] + kk;
          double xi[3] = {s->gx[i], s->gy[j], d == 3 ? s->gz[k] : 0.0};
          double weight = wip(s, xp, xi);
          uint32_t id = gind(s, i, j, k);
          const double* gvv = s->gv + (size_t)id * d;
          for (int a = 0; a < d; ++a) vp[a] += gvv[a] * weight;
          if (fr < 0) {
            double pd[3];
            for (int a = 0; a < d; ++a) pd[a] = xi[a] - xp[a];
            for (int r = 0; r < d; ++r)
              for (int c = 0; c < d; ++c) Bp[r][c] += gvv[r] * pd[c] * weight;
          }
          if (fr >= -1) {
            const double* gf = s->gflip + (size_t)id * d;
            for (int a = 0; a < d; ++a) fp[a] += gf[a] * weight;
          }
        }
    for (int a = 0; a < d; ++a) s->pic[(size_t)p * d + a] = vp[a];
    if (fr < 0) m_store(d, Bp, s->B + (size_t)p * dd);
    if (fr >= -1)
      for (int a = 0; a < d; ++a) s->flip[(size_t)p * d + a] = fp[a];
  }
}

/* velocity blend of position_update.cpp:16-24 and musl.cpp:15-22 */
static void blend_v(orc* s, uint32_t p) {
  int d = s->dim;
  double fr = s->P.flip_ratio;
  double* v = s->v + (size_t)p * d;
  const double* pic = s->pic + (size_t)p * d;
  const double* fl = s->flip + (size_t)p * d;
  for (int a = 0; a < d; ++a) {
    if (fr < -1)
      v[a] = pic[a];
    else if (fr < 0)
      v[a] = (-fr) * (v[a] + fl[a]) + (1 - (-fr)) * pic[a];
    else
      v[a] = fr * (v[a] + fl[a]) + (1 - fr) * pic[a];
  }
}

/* MUSL, musl.cpp:6-96 */
static void musl(orc* s) {
  int d = s->dim;
  double org[3] = {s->xc, s->yc, s->zc};
  for (uint32_t p = 0; p < s->Np; ++p) blend_v(s, p);
  memset(s->gv, 0, (size_t)s->G * d * sizeof(double));
  for (uint32_t p = 0; p < s->Np; ++p) {
    const double* xp = s->x + (size_t)p * d;
    const double* vp = s->v + (size_t)p * d;
    M3 Bp;
    m_load(d, s->B + (size_t)p * d * d, Bp);
    int base[3] = {0, 0, 0};
    for (int a = 0; a < d; ++a) {
      int b = (int)floor((xp[a] - org[a]) * s->one_over_dx) - 1;
      base[a] = b < 0 ? 0 : b;
    }
    int kn = d == 3 ? 4 : 1;
    for (int i = base[0]; i < base[0] + 4; ++i)
      for (int j = base[1]; j < base[1] + 4; ++j)
        for (int kk = 0; kk < kn; ++kk) {
          int k = base[2] + kk;
          double xi[3] = {s->gx[i], s->gy[j], d == 3 ? s->gz[k] : 0.0};
          double weight = wip(s, xp, xi);
          if (weight > 1e-25) {
            uint32_t id = gind(s, i, j, k);
            for (int a = 0; a < d; ++a) s->gv[(size_t)id * d + a] += vp[a] * weight;
            if (s->P.flip_ratio < 0) {
              double pd[3];
              for (int a = 0; a < d; ++a) pd[a] = xi[a] - xp[a];
              for (int a = 0; a < d; ++a) {
                double bv = Bp[a][0] * pd[0];
                for (int c = 1; c < d; ++c) bv += Bp[a][c] * pd[c];
                s->gv[(size_t)id * d + a] += bv * s->apicDinverse * weight;
              }
            }
          }
        }
  }
  for (uint32_t l = 0; l < s->G; ++l) {
    double mi = s->gmass[l];
    for (int a = 0; a < d; ++a) {
      if (mi > 0)
        s->gv[(size_t)l * d + a] /= (mi / s->P.particle_mass);
      else
        s->gv[(size_t)l * d + a] = 0.0;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* return mapping helpers, plasticity_helpers/*.hpp                          */
/* ------------------------------------------------------------------------ */

/* MCCRMAExplicit, mcc_rma_explicit.hpp:8-96 */
static int mcc_rma_explicit(orc* s, double* p_io, double* q_io, double M, double p0, double beta,
                            double mu, double K, double rma_prefac) {
  double p = *p_io, q = *q_io;
  double y = M * M * (p - p0) * (p + beta * p0) + (q * q);
  if (!(y > 0)) return 0;
  double delta_gamma = 0;
  double pt = p, qt = q;
  double dkdp = 2 * M * M;
  double dldq = 2;
  double max_iter = 40;
  for (int iter = 0; iter < max_iter; iter++) {
    y = M * M * (p - p0) * (p + beta * p0) + (q * q);
    double k = M * M * (beta * p0 + 2 * p - p0);
    double l = 2 * q;
    double r1 = pt - p - K * delta_gamma * k;
    double r2 = qt - q - rma_prefac * mu * delta_gamma * l;
    if (iter > 4 && fabs(y) < 1e-3 && fabs(r1) < 1e-3 && fabs(r2) < 1e-3) break;
    if (iter == max_iter - 1) {
      if (p0 > 0.1) {
        break;
      } else {
        p = 1e-15;
        q = 1e-15;
        break;
      }
    }
    double J11 = -1 - K * delta_gamma * dkdp;
    double J13 = -K * k;
    double J22 = -1 - rma_prefac * mu * delta_gamma * dldq;
    double J23 = -rma_prefac * mu * l;
    double J31 = k;
    double J32 = l;
    double det = J11 * (-J32 * J23) + J13 * (-J31 * J22);
    if (fabs(det) < 1e-6) {
      p -= 0.001 * r1;
      q -= 0.001 * r2;
      delta_gamma -= 0.001 * y / (p0 * p0);
    } else {
      p -= (-J32 * J23 * r1 + J32 * J13 * r2 - J22 * J13 * y) / det;
      q -= (J31 * J23 * r1 - J31 * J13 * r2 - J11 * J23 * y) / det;
      delta_gamma -= (-J31 * J22 * r1 - J11 * J32 * r2 + J11 * J22 * y) / det;
    }
    if (q < 1e-15) q = 1e-15;
  }
  p = dmax(p, -beta * p0);
  p = dmin(p, p0);
  q = M * sqrt((p0 - p) * (beta * p0 + p));
  *p_io = p;
  *q_io = q;
  return 1;
}

/* limited_search_exponential, limited_search_exponential.hpp:8-71 */
static double limited_search_exp(double epv, double epv_t, double epv_delta, double xi, double K,
                                 double p_t, double p00, double beta, int* right) {
  double scale = 1.;
  int tries = 0, max_tries = 32, f = 0;
  double test_epv = epv;
  while (tries < max_tries) {
    test_epv = epv - scale * epv_delta;
    double pp0 = p00 * exp(-xi * test_epv);
    double pp = K * (test_epv - epv_t) + p_t;
    double val = 2. * pp + (beta - 1.) * pp0;
    double midpoint = (pp0 - beta * pp0) * 0.5;
    if (fabs(pp - midpoint) <= 1.e-5) break;
    if (((*right == 1 && (pp < midpoint || p_t < midpoint)) ||
         (*right == 0 && (pp > midpoint || p_t > midpoint))) &&
        tries > -1) {
      test_epv = epv;
      *right = -1;
      break;
    }
    if (sgn(epv_t - test_epv) == sgn(val) || sgn(epv_t - test_epv) == 0) break;
    scale *= 0.5;
    tries++;
    if (tries != max_tries) continue;
    tries = 0;
    scale = 1.;
    epv_delta *= -1.;
    f++;
    if (f > 1) return INFINITY;
  }
  return test_epv;
}

/* MCCRMAImplicitExponentialOnevar, mcc_rma_implicit_exponential_onevar.hpp:9-166
 * (the unqualified abs() there resolves to the double overload when Eigen's
 * SSE headers are included, so fabs here). */
static int mcc_rma_impl_exp(orc* s, double* p_io, double* q_io, double M, double p00, double beta,
                            double mu, double K, double xi, double epv) {
  double p = *p_io, q = *q_io;
  double p0_t = p00 * exp(-xi * epv);
  double Msq = M * M;
  double damping_factor = 1;
  double y = Msq * (p * p + (beta - 1.) * p0_t * p - beta * p0_t * p0_t) + damping_factor * q * q;
  if (y <= 0) return 0;
  double scale_factor = 1. / p0_t;
  double p0 = 1.;
  p00 *= scale_factor;
  p *= scale_factor;
  q *= scale_factor;
  mu *= scale_factor;
  K *= scale_factor;
  double p_t = p, q_t = q, epv_t = epv;
  int right = 0;
  if (p_t > 0.5 * (p0 - beta * p0)) right = 1;
  int max_iter = 30;
  for (int iter = 0; iter < max_iter; iter++) {
    double midpoint = (p0 - beta * p0) * 0.5;
    if (fabs(p - midpoint) < 1e-4) {
      q = M * sqrt((p0 - p) * (beta * p0 + p) / damping_factor);
      q *= p0_t;
      p *= p0_t;
      *p_io = p;
      *q_io = q;
      return 1;
    }
    p = (epv - epv_t) * K + p_t;
    p0 = p00 * exp(-xi * epv);
    double denom = 2. * K * Msq * p + Msq * (beta - 1.) * K * p0;
    double dg_step = (p_t - p) / denom;
    double q_denom = 1 + 2. * mu * damping_factor * dg_step;
    q = q_t / q_denom;
    y = Msq * (p - p0) * (p + beta * p0) + damping_factor * q * q;
    if (iter > 5 && fabs(y) < 1.e-4) break;
    double dp_depv = K;
    double dp0_depv = -xi * p0;
    double ddelta_gamma_depv = (-dp_depv / denom) -
                               (p_t - p) * (2. * K * Msq * dp_depv + Msq * (beta - 1.) * K * dp0_depv) /
                                   (denom * denom);
    double dq_depv = -q_t * 2. * mu * damping_factor * ddelta_gamma_depv / (q_denom * q_denom);
    double dy_depv = Msq * (dp_depv - dp0_depv) * (p + beta * p0) +
                     Msq * (p - p0) * (beta * dp0_depv + dp_depv) + 2. * damping_factor * q * dq_depv;
    epv = limited_search_exp(epv, epv_t, y / dy_depv, xi, K, p_t, p00, beta, &right);
    if (epv == INFINITY) {
      s->exit_flag = 1;
      s->status |= MTR_STATUS_RMA_NOSTEP;
      break;
    }
  }
  p = dmax(p, -beta * p0);
  p = dmin(p, p0);
  q = M * sqrt((p0 - p) * (beta * p0 + p) / damping_factor);
  p *= p0_t;
  q *= p0_t;
  *p_io = p;
  *q_io = q;
  return 1;
}

/* limited_search_sinh, limited_search_sinh.hpp:8-72 */
static double limited_search_sinh(double epv, double epv_t, double epv_delta, double xi, double K,
                                  double p_t, double p00, double p0_min, double beta, int* right) {
  double scale = 1.;
  int tries = 0, max_tries = 32, f = 0;
  double test_epv = epv;
  while (tries < max_tries) {
    test_epv = epv - scale * epv_delta;
    double pp0 = dmax(p0_min, K * sinh(-xi * test_epv + asinh(p00 / K)));
    double pp = K * (test_epv - epv_t) + p_t;
    double val = 2. * pp + (beta - 1.) * pp0;
    double midpoint = (pp0 - beta * pp0) * 0.5;
    if (fabs(pp - midpoint) <= 1.e-5) break;
    if (((*right == 1 && (pp < midpoint || p_t < midpoint)) ||
         (*right == 0 && (pp > midpoint || p_t > midpoint))) &&
        tries > -1) {
      test_epv = epv;
      *right = -1;
      break;
    }
    if (sgn(epv_t - test_epv) == sgn(val) || sgn(epv_t - test_epv) == 0) break;
    scale *= 0.5;
    tries++;
    if (tries != max_tries) continue;
    tries = 0;
    scale = 1.;
    epv_delta *= -1.;
    f++;
    if (f > 1) return INFINITY;
  }
  return test_epv;
}

/* MCCRMAImplicitSinhOnevar, mcc_rma_implicit_sinh_onevar.hpp:9-171 */
static int mcc_rma_impl_sinh(orc* s, double* p_io, double* q_io, double M, double p00, double beta,
                             double mu, double K, double xi, double epv) {
  double p = *p_io, q = *q_io;
  double p0 = dmax(0.01, K * sinh(-xi * epv + asinh(p00 / K)));
  double Msq = M * M;
  double damping_factor = 1;
  double y = Msq * (p * p + (beta - 1.) * p0 * p - beta * p0 * p0) + damping_factor * q * q;
  if (y <= 0) return 0;
  double p0_t = p0;
  double scale_factor = 1. / p0_t;
  double p0_min = 0.01 * scale_factor;
  p00 *= scale_factor;
  p0 = 1.;
  p *= scale_factor;
  q *= scale_factor;
  mu *= scale_factor;
  K *= scale_factor;
  double p_t = p, q_t = q, epv_t = epv;
  int right = 0;
  if (p_t > 0.5 * (p0 - beta * p0)) right = 1;
  int max_iter = 40;
  for (int iter = 0; iter < max_iter; iter++) {
    double midpoint = (p0 - beta * p0) * 0.5;
    if (fabs(p - midpoint) < 1.e-4) {
      q = M * sqrt((p0 - p) * (beta * p0 + p) / damping_factor);
      p *= p0_t;
      q *= p0_t;
      *p_io = p;
      *q_io = q;
      return 1;
    }
    p = (epv - epv_t) * K + p_t;
    double p0_helper = K * sinh(-xi * epv + asinh(p00 / K));
    p0 = dmax(p0_min, p0_helper);
    double denom = 2. * K * Msq * p + Msq * (beta - 1.) * K * p0;
    double dg_step = (p_t - p) / denom;
    double q_denom = 1. + 2. * mu * damping_factor * dg_step;
    q = q_t / q_denom;
    y = Msq * (p - p0) * (p + beta * p0) + damping_factor * q * q;
    if (iter > 5 && fabs(y) < 1e-4) break;
    if (iter == max_iter - 1) {
      if (p0 > p0_min) {
        s->exit_flag = 1;
        s->status |= MTR_STATUS_RMA_NOCONV;
      }
    }
    double dp_depv = K;
    double dp0_depv;
    double dp0_depv_helper = -xi * K * cosh(-xi * epv + asinh(p00 / K));
    if (p0_helper > p0_min)
      dp0_depv = 0.5 * (dp0_depv_helper + dp0_depv_helper - p0_min);
    else
      dp0_depv = 0.5 * (dp0_depv_helper + p0_min - dp0_depv_helper);
    double ddelta_gamma_depv = (-dp_depv / denom) -
                               (p_t - p) * (2. * K * Msq * dp_depv + Msq * (beta - 1.) * K * dp0_depv) /
                                   (denom * denom);
    double dq_depv = -q_t * 2. * mu * damping_factor * ddelta_gamma_depv / (q_denom * q_denom);
    double dy_depv = Msq * (dp_depv - dp0_depv) * (p + beta * p0) +
                     Msq * (p - p0) * (beta * dp0_depv + dp_depv) + 2. * damping_factor * q * dq_depv;
    epv = limited_search_sinh(epv, epv_t, y / dy_depv, xi, K, p_t, p00, p0_min, beta, &right);
    if (epv == INFINITY) {
      s->exit_flag = 1;
      s->status |= MTR_STATUS_RMA_NOSTEP;
      break;
    }
  }
  p = dmax(p, -beta * p0);
  p = dmin(p, p0);
  q = M * sqrt((p0 - p) * (beta * p0 + p) / damping_factor);
  p *= p0_t;
  q *= p0_t;
  *p_io = p;
  *q_io = q;
  return 1;
}

/* Perzyna Newton loop shared by VMVisc/DPVisc/MCCVisc (plasticity.cpp:197-229,
 * 293-323, 558-588); VMVisc's yield depends on delta_gamma (is_vm). */
static double perzyna_newton(orc* s, double q_trial, double q_yield, int is_vm, double eps_pl_dev) {
  double dt = s->dt, pe = s->P.perzyna_exp, pv = s->P.perzyna_visc, fm = s->f_mu_prefac;
  double delta_gamma = 0.01 * (q_trial - q_yield) / fm;
  int max_iter = 60;
  for (int iter = 0; iter < max_iter; iter++) {
    if (iter == max_iter - 1) {
      s->exit_flag = 1;
      s->status |= MTR_STATUS_RMA_NOCONV;
    }
    double tm = pv * delta_gamma + dt;
    double tmp = dt / tm;
    double tmp1 = pow(tmp, pe);
    double qdiff = 0.0;
    if (is_vm) {
      double ex = exp(-s->P.xi * (eps_pl_dev + (1.0 / s->d_prefac) * delta_gamma));
      q_yield = s->P.q_min + (s->P.q_max - s->P.q_min) * ex;
      qdiff = -s->P.xi / s->d_prefac * (s->P.q_max - s->P.q_min) *
              exp(-s->P.xi * (eps_pl_dev + (1.0 / s->d_prefac) * delta_gamma));
    }
    double residual = (q_trial - fm * delta_gamma) * tmp1 - q_yield;
    if (fabs(residual) < 1e-2) break;
    double residual_diff = -fm * tmp1 + (q_trial - fm * delta_gamma) * pe * pow(tmp, pe - 1) * (-pv * dt) / (tm * tm);
    if (is_vm) residual_diff -= qdiff;
    if (fabs(residual_diff) < 1e-14) {
      s->exit_flag = 1;
      s->status |= MTR_STATUS_RESID_DIFF;
    }
    delta_gamma -= residual / residual_diff;
    if (delta_gamma < 0) delta_gamma = 1e-10;
  }
  return delta_gamma;
}

/* ------------------------------------------------------------------------ */
/* plasticity, plasticity.cpp:11-665                                         */
/* ------------------------------------------------------------------------ */
static void plasticity(orc* s, uint32_t p, M3 Fe_trial) {
  int d = s->dim, dd = d * d;
  int pm = s->P.plastic_model;
  if (pm == MTR_PM_NOPLASTICITY) return;
  if (pm < 0 || pm > MTR_PM_SNOW) {
    s->status |= MTR_STATUS_BAD_MODEL;
    return;
  }
  const double dim = (double)d;
  double dt = s->dt, K = s->K, M = s->P.M, qc = s->P.q_cohesion;
  double e_mu = s->e_mu_prefac, d_pre = s->d_prefac, f_mu = s->f_mu_prefac;
  M3 U, V;
  double S[3];
  svd_m(d, Fe_trial, U, S, V);
  double hencky[3], hdev[3];
  for (int i = 0; i < d; ++i) hencky[i] = log(dmax(fabs(S[i]), 1e-4)); /* plasticity.cpp:21 */
  double hencky_trace = hencky[0];
  for (int i = 1; i < d; ++i) hencky_trace += hencky[i];
  for (int i = 0; i < d; ++i) hdev[i] = hencky[i] - (hencky_trace / dim) * 1.0;
  double sq = hdev[0] * hdev[0];
  for (int i = 1; i < d; ++i) sq += hdev[i] * hdev[i];
  double hdn = sqrt(sq);
  if (hdn > 0)
    for (int i = 0; i < d; ++i) hdev[i] /= hdn;

  double* F = s->F + (size_t)p * dd;
  double* ep_dev = &s->eps_pl_dev[p];
  double* ep_vol = &s->eps_pl_vol[p];
  double* ep_pr = &s->eps_pl_vol_pradhana[p];
  double* dg_out = &s->delta_gamma[p];
  double* muI = &s->muI[p];
  double* visc = &s->viscosity[p];

#define WRITE_F(h)                        \
  do {                                    \
    double e_[3];                         \
    M3 Fn_;                               \
    for (int i_ = 0; i_ < d; ++i_) e_[i_] = exp((h)[i_]); \
    usv(d, U, e_, V, Fn_);                \
    m_store(d, Fn_, F);                   \
  } while (0)
#define SET_ISO(pp)                                          \
  do {                                                       \
    for (int i_ = 0; i_ < d; ++i_) hencky[i_] = -(pp) / (K * dim) * 1.0; \
  } while (0)

  if (pm == MTR_PM_VM) { /* plasticity.cpp:30-49 */
    double q_yield = s->P.q_max;
    double delta_gamma = hdn - q_yield / e_mu;
    if (delta_gamma > 0) {
      s->plastic_count++;
      *dg_out = d_pre * delta_gamma / dt;
      for (int i = 0; i < d; ++i) hencky[i] -= delta_gamma * hdev[i];
      WRITE_F(hencky);
      *ep_dev += delta_gamma;
    }
  } else if (pm == MTR_PM_DP) { /* plasticity.cpp:51-85 */
    double p_trial = -K * hencky_trace;
    double q_yield = M * p_trial + qc;
    if (q_yield < 1e-10) {
      s->plastic_count++;
      double p_proj = -qc / M;
      SET_ISO(p_proj);
      WRITE_F(hencky);
      double delta_gamma = d_pre * hdn;
      *dg_out = delta_gamma / dt;
      *ep_dev += (1.0 / d_pre) * delta_gamma;
      *ep_vol += (p_proj - p_trial) / K;
    } else {
      double delta_gamma = d_pre * (hdn - q_yield / e_mu);
      if (delta_gamma > 0) {
        s->plastic_count++;
        *dg_out = delta_gamma / dt;
        for (int i = 0; i < d; ++i) hencky[i] -= (1.0 / d_pre) * delta_gamma * hdev[i];
        WRITE_F(hencky);
        *ep_dev += (1.0 / d_pre) * delta_gamma;
      }
    }
  } else if (pm == MTR_PM_DPSOFT) { /* plasticity.cpp:87-162 */
    double p_trial = -K * hencky_trace;
    double q_trial = e_mu * hdn;
    double p_tip_orig = -qc / M;
    double p_tip = p_tip_orig * exp(-s->P.xi * *ep_dev);
    double p_shift = 0;
    if (s->P.use_pradhana) p_shift = -K * *ep_pr;
    double q_yield = M * (p_trial + p_shift) + (-p_tip * M);
    if ((p_trial + p_shift) <= p_tip) {
      s->plastic_count++;
      double p_proj = p_tip_orig * exp(-s->P.xi * *ep_dev);
      SET_ISO(p_proj);
      WRITE_F(hencky);
      double delta_gamma = d_pre * hdn;
      *dg_out = delta_gamma / dt;
      *ep_dev += (1.0 / d_pre) * delta_gamma;
      double inst = (p_proj - p_trial) / K;
      *ep_vol += inst;
      if (s->P.use_pradhana) *ep_pr += inst;
    }
    if ((p_trial + p_shift) > p_tip && q_trial <= q_yield) {
      if (s->P.use_pradhana) *ep_pr = 0;
      *dg_out = 0;
    }
    if ((p_trial + p_shift) > p_tip && q_trial > q_yield) {
      s->plastic_count++;
      double temp_eps_pl_dev = *ep_dev + (hdn - q_yield / e_mu);
      double p_proj = p_tip_orig * exp(-s->P.xi * temp_eps_pl_dev);
      if ((p_trial + p_shift) < p_proj) {
        double delta_gamma = d_pre * hdn;
        *dg_out = delta_gamma / dt;
        *ep_dev += (1.0 / d_pre) * delta_gamma;
        double inst = (p_proj - p_trial) / K;
        *ep_vol += inst;
        if (s->P.use_pradhana) *ep_pr += inst;
        SET_ISO(p_proj);
        WRITE_F(hencky);
      } else {
        double q_yield_new = M * (p_trial + p_shift) + (-p_proj * M);
        double delta_gamma = d_pre * (hdn - q_yield_new / e_mu);
        for (int i = 0; i < d; ++i) hencky[i] -= (1.0 / d_pre) * delta_gamma * hdev[i];
        WRITE_F(hencky);
        *ep_dev += (1.0 / d_pre) * delta_gamma;
        *dg_out = delta_gamma / dt;
        if (s->P.use_pradhana) *ep_pr = 0;
      }
    }
  } else if (pm == MTR_PM_VMVISC) { /* plasticity.cpp:164-238 */
    double q_trial = e_mu * hdn;
    double q_yield = s->P.q_min + (s->P.q_max - s->P.q_min) * exp(-s->P.xi * *ep_dev);
    double p_trial = -K * hencky_trace;
    if (p_trial < s->P.p_min * exp(-s->P.xi * *ep_vol)) {
      double delta_gamma = q_trial / f_mu;
      double inst = -p_trial / K;
      M3 Fn;
      m_mul_bt(d, U, V, Fn);
      m_store(d, Fn, F);
      *ep_vol += inst;
      *ep_dev += (1.0 / d_pre) * delta_gamma;
      *dg_out = delta_gamma / dt;
    } else if (q_trial > q_yield) {
      s->plastic_count++;
      double delta_gamma;
      if (s->P.perzyna_exp == 1 && s->P.xi == 0) {
        delta_gamma = (q_trial - q_yield) / (f_mu + q_yield * s->P.perzyna_visc / dt);
        if (delta_gamma < 0) {
          s->exit_flag = 1;
          s->status |= MTR_STATUS_NEG_DGAMMA;
        }
      } else {
        delta_gamma = perzyna_newton(s, q_trial, q_yield, 1, *ep_dev);
      }
      for (int i = 0; i < d; ++i) hencky[i] -= (1.0 / d_pre) * delta_gamma * hdev[i];
      WRITE_F(hencky);
      *ep_dev += (1.0 / d_pre) * delta_gamma;
      *dg_out = delta_gamma / dt;
    }
  } else if (pm == MTR_PM_DPVISC) { /* plasticity.cpp:240-339 */
    double p_trial = -K * hencky_trace;
    double q_trial = e_mu * hdn;
    double p_tip = -qc / M;
    double p_shift = 0;
    if (s->P.use_pradhana) p_shift = -K * *ep_pr;
    double q_yield = M * (p_trial + p_shift) + qc;
    if (s->P.use_mibf) *muI = M;
    if ((p_trial + p_shift) < p_tip) {
      double delta_gamma = d_pre * hdn;
      double p_proj = p_tip;
      double inst = (p_proj - p_trial) / K;
      s->plastic_count++;
      SET_ISO(p_proj);
      WRITE_F(hencky);
      *dg_out = delta_gamma / dt;
      *ep_dev += (1.0 / d_pre) * delta_gamma;
      *ep_vol += inst;
      if (s->P.use_pradhana) *ep_pr += inst;
    } else {
      if (s->P.use_pradhana) *ep_pr = 0;
      *dg_out = 0;
    }
    if ((p_trial + p_shift) > p_tip && q_trial > q_yield) {
      s->plastic_count++;
      double delta_gamma;
      if (s->P.perzyna_exp == 1) {
        delta_gamma = (q_trial - q_yield) / (f_mu + q_yield * s->P.perzyna_visc / dt);
        if (delta_gamma < 0) {
          s->exit_flag = 1;
          s->status |= MTR_STATUS_NEG_DGAMMA;
        }
      } else {
        delta_gamma = perzyna_newton(s, q_trial, q_yield, 0, 0.0);
      }
      if (s->P.use_mibf) {
        if (fabs(p_trial + p_shift) < 1e-10)
          *muI = 1e10;
        else
          *muI = ((q_trial - f_mu * delta_gamma) - qc) / (p_trial + p_shift);
      }
      for (int i = 0; i < d; ++i) hencky[i] -= (1.0 / d_pre) * delta_gamma * hdev[i];
      WRITE_F(hencky);
      *ep_dev += (1.0 / d_pre) * delta_gamma;
      *dg_out = delta_gamma / dt;
    }
  } else if (pm == MTR_PM_DPMUI) { /* plasticity.cpp:342-403 */
    double p_trial = -K * hencky_trace;
    double q_trial = e_mu * hdn;
    double mu_1 = s->P.mu_1, mu_2 = s->P.mu_2, fac_Q = s->fac_Q;
    double p_tip = -qc / mu_1;
    double p_shift = 0;
    if (s->P.use_pradhana) p_shift = -K * *ep_pr;
    *muI = mu_1;
    *visc = 0;
    if ((p_trial + p_shift) < p_tip) {
      double delta_gamma = d_pre * hdn;
      double inst = (p_tip - p_trial) / K;
      s->plastic_count++;
      SET_ISO(p_tip);
      WRITE_F(hencky);
      *dg_out = delta_gamma; /* plasticity.cpp:364: no /dt in this branch */
      *ep_dev += (1.0 / d_pre) * delta_gamma;
      *ep_vol += inst;
      *ep_pr += inst;
    } else {
      *ep_pr = 0;
    }
    double q_yield = mu_1 * (p_trial + p_shift) + qc;
    if ((p_trial + p_shift) > p_tip && q_trial > (q_yield + s->P.stress_tolerance)) {
      s->plastic_count++;
      double p_special = p_trial + p_shift - p_tip + s->P.stress_tolerance;
      double fac_a = f_mu * dt;
      double fac_b = p_trial * (mu_2 - mu_1) + f_mu * dt * fac_Q * sqrt(p_special) - (q_trial - q_yield);
      double fac_c = -(q_trial - q_yield) * fac_Q * sqrt(p_special);
      double delta_gamma = (-fac_b + sqrt(fac_b * fac_b - 4 * fac_a * fac_c)) / (2 * fac_a);
      double mu_i = mu_1 + (mu_2 - mu_1) / (fac_Q * sqrt(p_special) / delta_gamma + 1.0);
      *muI = mu_i;
      *visc = (mu_i - mu_1) * p_special / delta_gamma;
      delta_gamma *= dt;
      for (int i = 0; i < d; ++i) hencky[i] -= (1.0 / d_pre) * delta_gamma * hdev[i];
      WRITE_F(hencky);
      *ep_dev += (1.0 / d_pre) * delta_gamma;
      *dg_out = delta_gamma / dt;
    }
  } else if (pm == MTR_PM_MCCMUI) { /* plasticity.cpp:405-484 */
    double p_stress = -K * hencky_trace;
    double q_stress = e_mu * hdn;
    double q_trial = q_stress;
    double mu_1 = s->P.mu_1, mu_2 = s->P.mu_2, fac_Q = s->fac_Q;
    double p0 = s->P.p0, beta = s->P.beta, xi = s->P.xi, st = s->P.stress_tolerance;
    int perform_rma = 0;
    double p_c = 0.0;
    int hl = s->P.hardening_law;
    if (hl == MTR_HL_EXPOEXPL) {
      p_c = dmax(st, p0 * exp(-xi * *ep_vol));
      perform_rma = mcc_rma_explicit(s, &p_stress, &q_stress, mu_1, p_c, beta, s->mu, K, s->rma_prefac);
    } else if (hl == MTR_HL_SINHEXPL) {
      p_c = dmax(st, K * sinh(-xi * *ep_vol + asinh(p0 / K)));
      perform_rma = mcc_rma_explicit(s, &p_stress, &q_stress, mu_1, p_c, beta, s->mu, K, s->rma_prefac);
    } else if (hl == MTR_HL_EXPOIMPL) {
      perform_rma = mcc_rma_impl_exp(s, &p_stress, &q_stress, mu_1, p0, beta, s->mu, K, xi, *ep_vol);
    } else if (hl == MTR_HL_SINHIMPL) {
      perform_rma = mcc_rma_impl_sinh(s, &p_stress, &q_stress, mu_1, p0, beta, s->mu, K, xi, *ep_vol);
    } else {
      s->exit_flag = 1;
      s->status |= MTR_STATUS_BAD_MODEL;
    }
    *muI = mu_1;
    *visc = 0;
    if (perform_rma) {
      s->plastic_count++;
      double ep = p_stress / (K * dim);
      double inst = hencky_trace + dim * ep;
      *ep_vol += inst;
      if (q_trial > (q_stress + st)) {
        if (hl == MTR_HL_EXPOIMPL)
          p_c = dmax(p0 * exp(-xi * *ep_vol), p_stress + st);
        else if (hl == MTR_HL_SINHIMPL)
          p_c = dmax(K * sinh(-xi * *ep_vol + asinh(p0 / K)), p_stress + st);
        double p_special = p_stress + beta * p_c + st;
        double fac_a = f_mu * dt;
        double fac_b = sqrt((p_c - p_stress) * p_special) * (mu_2 - mu_1) + f_mu * dt * fac_Q * sqrt(p_special) -
                       (q_trial - q_stress);
        double fac_c = -(q_trial - q_stress) * fac_Q * sqrt(p_special);
        double gamma_dot_S = (-fac_b + sqrt(fac_b * fac_b - 4 * fac_a * fac_c)) / (2 * fac_a);
        q_stress = dmax(q_stress, q_trial - f_mu * dt * gamma_dot_S);
        double mu_i = mu_1 + (mu_2 - mu_1) / (fac_Q * sqrt(p_special) / gamma_dot_S + 1.0);
        *muI = mu_i;
        *visc = (mu_i - mu_1) * sqrt((p_c - p_stress) * p_special) / gamma_dot_S;
        double delta_gamma = (q_trial - q_stress) / f_mu;
        *ep_dev += (1.0 / d_pre) * delta_gamma;
        *dg_out = delta_gamma / dt;
      }
      for (int i = 0; i < d; ++i) hencky[i] = q_stress / e_mu * hdev[i] - ep * 1.0;
      WRITE_F(hencky);
    }
  } else if (pm == MTR_PM_MCC || pm == MTR_PM_MCCVISC) { /* plasticity.cpp:487-621 */
    double p_stress = -K * hencky_trace;
    double q_stress = e_mu * hdn;
    double q_trial = q_stress;
    double p0 = s->P.p0, beta = s->P.beta, xi = s->P.xi, st = s->P.stress_tolerance;
    if (pm == MTR_PM_MCCVISC && s->P.use_mibf) *muI = M;
    int perform_rma = 0;
    double p_c = 0.0;
    int hl = s->P.hardening_law;
    if (hl == MTR_HL_NOHARD) {
      perform_rma = mcc_rma_explicit(s, &p_stress, &q_stress, M, p0, beta, s->mu, K, s->rma_prefac);
    } else if (hl == MTR_HL_EXPOEXPL) {
      p_c = dmax(st, p0 * exp(-xi * *ep_vol));
      perform_rma = mcc_rma_explicit(s, &p_stress, &q_stress, M, p_c, beta, s->mu, K, s->rma_prefac);
    } else if (hl == MTR_HL_SINHEXPL) {
      p_c = dmax(st, K * sinh(-xi * *ep_vol + asinh(p0 / K)));
      perform_rma = mcc_rma_explicit(s, &p_stress, &q_stress, M, p_c, beta, s->mu, K, s->rma_prefac);
    } else if (hl == MTR_HL_EXPOIMPL) {
      perform_rma = mcc_rma_impl_exp(s, &p_stress, &q_stress, M, p0, beta, s->mu, K, xi, *ep_vol);
    } else if (hl == MTR_HL_SINHIMPL) {
      perform_rma = mcc_rma_impl_sinh(s, &p_stress, &q_stress, M, p0, beta, s->mu, K, xi, *ep_vol);
    } else {
      s->exit_flag = 1;
      s->status |= MTR_STATUS_BAD_MODEL;
    }
    if (perform_rma) {
      s->plastic_count++;
      double ep = p_stress / (K * dim);
      double inst = hencky_trace + dim * ep;
      *ep_vol += inst;
      double delta_gamma;
      if (pm == MTR_PM_MCCVISC) {
        double q_yield = q_stress;
        if (s->P.perzyna_exp == 1) {
          delta_gamma = (q_trial - q_yield) / (f_mu + q_yield * s->P.perzyna_visc / dt);
          if (delta_gamma < 0) {
            if (delta_gamma > -1e-14) {
              delta_gamma = 0;
            } else {
              s->exit_flag = 1;
              s->status |= MTR_STATUS_NEG_DGAMMA;
            }
          }
        } else {
          delta_gamma = perzyna_newton(s, q_trial, q_yield, 0, 0.0);
        }
        q_stress = dmax(q_yield, q_trial - f_mu * delta_gamma);
        if (s->P.use_mibf) {
          if (hl == MTR_HL_EXPOIMPL)
            p_c = dmax(0.0, p0 * exp(-xi * *ep_vol));
          else if (hl == MTR_HL_SINHIMPL)
            p_c = dmax(0.0, K * sinh(-xi * *ep_vol + asinh(p0 / K)));
          if ((p_stress < -beta * p_c + st) || (p_stress > p_c - st))
            *muI = M;
          else
            *muI = q_stress / sqrt((p_stress + beta * p_c) * (p_c - p_stress));
        }
      }
      delta_gamma = (q_trial - q_stress) / f_mu;
      *ep_dev += (1.0 / d_pre) * delta_gamma;
      *dg_out = delta_gamma / dt;
      for (int i = 0; i < d; ++i) hencky[i] = q_stress / e_mu * hdev[i] - ep * 1.0;
      WRITE_F(hencky);
    }
  } else if (pm == MTR_PM_SNOW) { /* plasticity.cpp:623-658 */
    double Sx[3];
    for (int i = 0; i < d; ++i) {
      Sx[i] = S[i];
      if (Sx[i] > 7.5e-3) Sx[i] = 7.5e-3;
    }
    for (int i = 0; i < d; ++i)
      if (Sx[i] < 2.5e-2) Sx[i] = 2.5e-2;
    M3 Fe, Fe_new_inv, Fp;
    usv(d, U, Sx, V, Fe);
    double Sinv[3];
    for (int i = 0; i < d; ++i) Sinv[i] = (fabs(Sx[i]) > 1e-9) ? 1.0 / Sx[i] : 0.0;
    usv(d, V, Sinv, U, Fe_new_inv);
    m_mul(d, Fe_new_inv, Fe_trial, Fp);
    double one_minus_Jp = 1.0 - m_det(d, Fp);
    double power = dmin(10.0 * one_minus_Jp, 5.0);
    double E = s->P.E, nu = s->P.nu;
    double lambda0 = (E * nu) / ((1 + nu) * (1 - 2 * nu));
    double mu0 = E / (2 * (1 + nu));
    double lam = exp(power) * lambda0;
    double mu = exp(power) * mu0;
    double lse[3], tr = 0.0;
    for (int i = 0; i < d; ++i) lse[i] = log(Sx[i]);
    tr = lse[0];
    for (int i = 1; i < d; ++i) tr += lse[i];
    double ph[3];
    for (int i = 0; i < d; ++i) ph[i] = ((2.0 * mu * lse[i]) + (lam * tr) * 1.0) * Sinv[i];
    M3 dP;
    usv(d, U, ph, V, dP);
    m_store(d, dP, s->dPsidF + (size_t)p * dd);
    m_store(d, Fe, s->Fe + (size_t)p * dd);
    s->lambda = lam; /* the reference writes the members (plasticity.cpp:646-647) */
    s->mu = mu;
  }
#undef WRITE_F
#undef SET_ISO
}

/* deformationUpdate, deformation_update.cpp:7-53 */
static void deformation_update(orc* s) {
  int d = s->dim, dd = d * d;
  double org[3] = {s->xc, s->yc, s->zc};
  memset(s->delta_gamma, 0, s->Np * sizeof(double));
  for (uint32_t p = 0; p < s->Np; ++p) {
    M3 sum;
    memset(sum, 0, sizeof(M3));
    const double* xp = s->x + (size_t)p * d;
    int base[3] = {0, 0, 0};
    for (int a = 0; a < d; ++a) base[a] = (int)(floor((xp[a] - org[a]) * s->one_over_dx) - 1);
    int kn = d == 3 ? 4 : 1;
    for (int i = base[0]; i < base[0] + 4; ++i)
      for (int j = base[1]; j < base[1] + 4; ++j)
        for (int kk = 0; kk < kn; ++kk) {
          int k = base[2] + kk;
          double xi[3] = {s->gx[i], s->gy[j], d == 3 ? s->gz[k] : 0.0};
          double g[3];
          grad_wip(s, xp, xi, g);
          const double* gvv = s->gv + (size_t)gind(s, i, j, k) * d;
          for (int r = 0; r < d; ++r)
            for (int c = 0; c < d; ++c) sum[r][c] += gvv[r] * g[c];
        }
    M3 Fe, T1, T2;
    m_load(d, s->F + (size_t)p * dd, Fe);
    for (int r = 0; r < d; ++r)
      for (int c = 0; c < d; ++c) T1[r][c] = s->dt * sum[r][c];
    m_mul(d, T1, Fe, T2);
    for (int r = 0; r < d; ++r)
      for (int c = 0; c < d; ++c) Fe[r][c] = Fe[r][c] + T2[r][c];
    m_store(d, Fe, s->F + (size_t)p * dd);
    plasticity(s, p, Fe);
  }
}

/* positionUpdate, position_update.cpp:6-46 */
static void position_update(orc* s) {
  int d = s->dim;
  for (uint32_t p = 0; p < s->Np; ++p) {
    double* x = s->x + (size_t)p * d;
    for (int a = 0; a < d; ++a) x[a] = x[a] + s->dt * s->pic[(size_t)p * d + a];
    if (!s->P.use_musl) blend_v(s, p);
    if (s->P.pbc) { /* position_update.cpp:26-33 */
      if (x[0] > s->P.L[0])
        x[0] = x[0] - s->P.L[0];
      else if (x[0] < 0)
        x[0] = s->P.L[0] + x[0];
    }
    if (s->P.change_particle_positions) { /* position_update.cpp:35-41 */
      if (x[0] > 0.8) {
        x[0] = -0.1;
        x[1] += 0.27;
      }
    }
  }
}

/* ObjectPlate::move, object_plate.hpp:136-162 */
static void move_objects(orc* s) {
  for (int i = 0; i < s->nplates; ++i) {
    mtr_plate* o = &s->plates[i];
    double factor = (s->time < o->load_factor * s->frame_dt) ? (1.0 / o->vmin_factor) : 1.0;
    for (int a = 0; a < 3; ++a) o->v_object[a] = o->v_object_original[a] * factor;
    if (s->dim == 2) o->v_object[2] = 0.0;
    if (o->plate_type == MTR_PLATE_LEFT || o->plate_type == MTR_PLATE_RIGHT) {
      o->pos_object += s->dt * o->v_object[0];
      o->pos_upper += s->dt * o->v_object[1];
      o->pos_lower += s->dt * o->v_object[1];
    } else if (o->plate_type == MTR_PLATE_BOTTOM || o->plate_type == MTR_PLATE_TOP) {
      o->pos_object += s->dt * o->v_object[1];
      o->pos_upper += s->dt * o->v_object[0];
      o->pos_lower += s->dt * o->v_object[0];
    } else if (s->dim == 3 && (o->plate_type == MTR_PLATE_BACK || o->plate_type == MTR_PLATE_FRONT)) {
      o->pos_object += s->dt * o->v_object[2];
    }
  }
}

/* ------------------------------------------------------------------------ */
/* public API (ctypes)                                                       */
/* ------------------------------------------------------------------------ */
static double* xalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

orc* orc_create(const mtr_params* P) {
  if (!P || (P->dim != 2 && P->dim != 3) || (P->spline_deg != 2 && P->spline_deg != 3)) return NULL;
  orc* s = (orc*)calloc(1, sizeof(orc));
  s->P = *P;
  s->dim = P->dim;
  s->deg = P->spline_deg;
  int d = s->dim;
  /* simulation.cpp:94-136 */
  s->apicDinverse = s->deg == 3 ? 3.0 / (P->dx * P->dx) : 4.0 / (P->dx * P->dx);
  s->lambda = P->nu * P->E / ((1.0 + P->nu) * (1.0 - 2.0 * P->nu));
  s->mu = P->E / (2.0 * (1.0 + P->nu));
  s->K = s->lambda + 2.0 * s->mu / d; /* simulation.cpp:288-290 */
  s->wave_speed = sqrt(P->E / P->rho);
  s->dt_max = P->cfl_elastic * P->dx / s->wave_speed;
  s->frame_dt = 1.0 / P->fps;
  for (int a = 0; a < 3; ++a) {
    s->gravity[a] = a < d ? P->gravity[a] : 0.0;
    s->gravity_final[a] = s->gravity[a];
  }
  s->one_over_dx = 1.0 / P->dx;
  s->one_over_dx_square = s->one_over_dx * s->one_over_dx;
  if (P->use_mises_q) {
    s->q_prefac = sqrt(3.0) / sqrt(2.0);
    s->d_prefac = sqrt(2.0) / sqrt(3.0);
  } else {
    s->q_prefac = 1.0 / sqrt(2.0);
    s->d_prefac = sqrt(2.0);
  }
  s->e_mu_prefac = 2 * s->q_prefac * s->mu;
  s->f_mu_prefac = 2 * s->q_prefac / s->d_prefac * s->mu;
  s->rma_prefac = 2 * s->q_prefac * s->q_prefac;
  s->fac_Q = P->I_ref / (P->grain_diameter * sqrt(P->rho_s));
  s->time = 0;
  s->frame = 0;
  s->final_time = P->end_frame * s->frame_dt;
  return s;
}

int orc_set_particles(orc* s, uint32_t Np, const double* x, const double* v, const double* F,
                      const double* B, const double* scalars) {
  int d = s->dim, dd = d * d;
  s->Np = Np;
  s->x = xalloc((size_t)Np * d);
  s->v = xalloc((size_t)Np * d);
  s->pic = xalloc((size_t)Np * d);
  s->flip = xalloc((size_t)Np * d);
  s->F = xalloc((size_t)Np * dd);
  s->B = xalloc((size_t)Np * dd);
  s->dPsidF = xalloc((size_t)Np * dd);
  s->Fe = xalloc((size_t)Np * dd);
  s->eps_pl_dev = xalloc(Np);
  s->eps_pl_vol = xalloc(Np);
  s->eps_pl_vol_pradhana = xalloc(Np);
  s->delta_gamma = xalloc(Np);
  s->viscosity = xalloc(Np);
  s->muI = xalloc(Np);
  s->keys = (uint32_t*)calloc(Np ? Np : 1, sizeof(uint32_t));
  memcpy(s->x, x, sizeof(double) * Np * d);
  if (v) memcpy(s->v, v, sizeof(double) * Np * d);
  for (uint32_t p = 0; p < Np; ++p)
    for (int i = 0; i < d; ++i) {
      s->F[(size_t)p * dd + i * d + i] = 1.0;
      s->Fe[(size_t)p * dd + i * d + i] = 1.0;
    }
  if (F) memcpy(s->F, F, sizeof(double) * Np * dd);
  if (B) memcpy(s->B, B, sizeof(double) * Np * dd);
  if (scalars)
    for (uint32_t p = 0; p < Np; ++p) {
      s->eps_pl_dev[p] = scalars[p * 6 + 0];
      s->eps_pl_vol[p] = scalars[p * 6 + 1];
      s->eps_pl_vol_pradhana[p] = scalars[p * 6 + 2];
      s->delta_gamma[p] = scalars[p * 6 + 3];
      s->viscosity[p] = scalars[p * 6 + 4];
      s->muI[p] = scalars[p * 6 + 5];
    }
  if (s->P.use_mibf) { /* simulation.cpp:138-145 */
    double m0 = (s->P.plastic_model == MTR_PM_DPMUI || s->P.plastic_model == MTR_PM_MCCMUI) ? s->P.mu_1 : s->P.M;
    for (uint32_t p = 0; p < Np; ++p) s->muI[p] = m0;
  }
  return 0;
}

int orc_set_objects(orc* s, const mtr_plate* plates, int np, const mtr_object* objs, int no) {
  if (np > MAXP || no > MAXO) return -1;
  s->nplates = np;
  s->nobjects = no;
  for (int i = 0; i < np; ++i) s->plates[i] = plates[i];
  for (int i = 0; i < no; ++i) s->objects[i] = objs[i];
  return 0;
}

/* A dense level set for MTR_OBJ_LEVELSET objects; normals NULL = the
 * second-order central-difference gradient 0.5 (phi[i+1] - phi[i-1]) / h
 * (OpenVDB's Gradient with CD_2ND), neighbours outside the lattice reading
 * the background 3 h. */
int orc_set_levelset(orc* s, int slot, const float* phi, const float* normals, const uint32_t* dims,
                     const double* origin, double spacing) {
  if (slot < 0 || slot >= MTR_MAX_LEVELSETS || !(spacing > 0)) return -1;
  size_t n = (size_t)dims[0] * dims[1] * dims[2];
  free(s->ls[slot].phi);
  free(s->ls[slot].grad);
  s->ls[slot].phi = (float*)malloc(sizeof(float) * n);
  s->ls[slot].grad = (float*)malloc(sizeof(float) * 3 * n);
  memcpy(s->ls[slot].phi, phi, sizeof(float) * n);
  float bg = (float)(3.0 * spacing);
  if (normals) {
    memcpy(s->ls[slot].grad, normals, sizeof(float) * 3 * n);
  } else {
    double half_inv_h = 0.5 / spacing;
    for (size_t l = 0; l < n; ++l) {
      uint32_t k = (uint32_t)(l % dims[2]), j = (uint32_t)((l / dims[2]) % dims[1]);
      uint32_t i = (uint32_t)(l / ((size_t)dims[1] * dims[2]));
      uint32_t c[3] = {i, j, k};
      size_t step[3] = {(size_t)dims[1] * dims[2], dims[2], 1};
      for (int a = 0; a < 3; ++a) {
        float g = 0.0f;
        if (a < s->dim) {
          float plus = c[a] + 1 < dims[a] ? phi[l + step[a]] : bg;
          float minus = c[a] >= 1 ? phi[l - step[a]] : bg;
          float diff = plus - minus;
          g = (float)((double)diff * half_inv_h);
        }
        s->ls[slot].grad[l * 3 + a] = g;
      }
    }
  }
  for (int a = 0; a < 3; ++a) {
    s->ls[slot].n[a] = dims[a];
    s->ls[slot].org[a] = a < s->dim ? origin[a] : 0.0;
  }
  s->ls[slot].h = spacing;
  s->ls[slot].inv_h = 1.0 / spacing;
  s->ls[slot].background = (double)bg;
  return 0;
}

/* advanceStep, simulation.cpp:219-273, plus the loop body of simulate(),
 * simulation.cpp:175-200.  Returns the number of steps executed. */
int orc_step(orc* s, int nsteps) {
  int d = s->dim;
  int done = 0;
  double* force = NULL;
  for (int it = 0; it < nsteps; ++it) {
    if (s->done || s->exit_flag || s->frame >= s->P.end_frame) break;
    update_dt(s);
    if (s->P.pbc) { /* simulation.cpp:222-233 */
      if (s->step == 0) remesh_fixed(s, 4);
    } else if (s->step == 0) {
      remesh_init(s);
    } else {
      remesh_cont(s);
    }
    resize_grid(s);
    compute_keys(s);
    if (s->P.pbc) pbc_add(s, 4);
    p2g(s);
    force = (double*)realloc(force, (size_t)s->G * d * sizeof(double) + 8);
    explicit_euler(s, force);
    s->ng = 0; /* PBCDelParticles, pbc.cpp:87-101 */
    g2p(s);
    if (s->P.use_musl) musl(s);
    deformation_update(s);
    position_update(s);
    move_objects(s);
    if (s->exit_flag) break;
    s->time += s->dt;
    s->step++;
    if (s->frame_dt * (s->frame + 1) - s->time < 1e-15) s->frame++;
    if (fabs(s->final_time - s->time) < 1e-15 || s->final_time < s->time) s->done = 1;
    done++;
  }
  free(force);
  return done;
}

void orc_get_particles(orc* s, double* x, double* v, double* F, double* B, double* scalars, double* pic,
                       double* flip) {
  int d = s->dim, dd = d * d;
  uint32_t Np = s->Np;
  if (x) memcpy(x, s->x, sizeof(double) * Np * d);
  if (v) memcpy(v, s->v, sizeof(double) * Np * d);
  if (F) memcpy(F, s->F, sizeof(double) * Np * dd);
  if (B) memcpy(B, s->B, sizeof(double) * Np * dd);
  if (pic) memcpy(pic, s->pic, sizeof(double) * Np * d);
  if (flip) memcpy(flip, s->flip, sizeof(double) * Np * d);
  if (scalars)
    for (uint32_t p = 0; p < Np; ++p) {
      scalars[p * 6 + 0] = s->eps_pl_dev[p];
      scalars[p * 6 + 1] = s->eps_pl_vol[p];
      scalars[p * 6 + 2] = s->eps_pl_vol_pradhana[p];
      scalars[p * 6 + 3] = s->delta_gamma[p];
      scalars[p * 6 + 4] = s->viscosity[p];
      scalars[p * 6 + 5] = s->muI[p];
    }
}

void orc_get_grid(orc* s, uint32_t* dims, double* gx, double* gy, double* gz, double* mass, double* v,
                  double* flip) {
  int d = s->dim;
  dims[0] = s->Nx;
  dims[1] = s->Ny;
  dims[2] = s->Nz;
  if (gx) memcpy(gx, s->gx, sizeof(double) * s->Nx);
  if (gy) memcpy(gy, s->gy, sizeof(double) * s->Ny);
  if (gz && d == 3) memcpy(gz, s->gz, sizeof(double) * s->Nz);
  if (mass) memcpy(mass, s->gmass, sizeof(double) * s->G);
  if (v) memcpy(v, s->gv, sizeof(double) * s->G * d);
  if (flip) memcpy(flip, s->gflip, sizeof(double) * s->G * d);
}

void orc_get_keys(orc* s, uint32_t* keys) { memcpy(keys, s->keys, sizeof(uint32_t) * s->Np); }

void orc_get_clock(orc* s, double* out) { /* time, dt, step, frame, done, exit, status, plastic_count */
  out[0] = s->time;
  out[1] = s->dt;
  out[2] = s->step;
  out[3] = s->frame;
  out[4] = s->done;
  out[5] = s->exit_flag;
  out[6] = s->status;
  out[7] = (double)s->plastic_count;
}

void orc_get_plates(orc* s, mtr_plate* out, int n) {
  for (int i = 0; i < n && i < s->nplates; ++i) out[i] = s->plates[i];
}

void orc_get_constants(orc* s, double* out) {
  out[0] = s->lambda; out[1] = s->mu; out[2] = s->K; out[3] = s->wave_speed; out[4] = s->dt_max;
  out[5] = s->apicDinverse; out[6] = s->e_mu_prefac; out[7] = s->f_mu_prefac; out[8] = s->d_prefac;
  out[9] = s->fac_Q;
}

void orc_destroy(orc* s) {
  if (!s) return;
  free(s->x); free(s->v); free(s->pic); free(s->flip); free(s->F); free(s->B); free(s->dPsidF);
  free(s->Fe); free(s->eps_pl_dev); free(s->eps_pl_vol); free(s->eps_pl_vol_pradhana);
  free(s->delta_gamma); free(s->viscosity); free(s->muI); free(s->keys); free(s->gsrc); free(s->gpos);
  free(s->gx); free(s->gy); free(s->gz); free(s->gmass); free(s->gv); free(s->gflip); free(s->gfric);
  for (int i = 0; i < MTR_MAX_LEVELSETS; ++i) {
    free(s->ls[i].phi);
    free(s->ls[i].grad);
  }
  free(s);
}

size_t orc_sizeof_params(void) { return sizeof(mtr_params); }
size_t orc_sizeof_plate(void) { return sizeof(mtr_plate); }
size_t orc_sizeof_object(void) { return sizeof(mtr_object); }

/* ------------------------------------------------------------------------ */
/* P2G alone onto a caller's grid: the checker of mtr_p2g_noalloc            */
/* ------------------------------------------------------------------------ */
/* The P2G of p2g.cpp:6-100 (via p2g() above) over a grid the caller gives
 * (uniform axes gx, gy, gz at params->dx; dims nodes per axis), with
 * mtr_p2g_noalloc's rule for particles the grid cannot hold: a particle whose
 * cell floor((x - x0)/dx) lies outside [0, N) on any axis, or whose clamped
 * stencil base + 3 reaches N, is left out.  x, v are AoS [Np][dim], B AoS
 * column-major [Np][dim*dim] (read when flip_ratio < 0).  Writes grid_mass[G]
 * and grid_v[G][dim]; returns the number of particles left out. */
uint32_t orc_p2g_grid(const mtr_params* P, uint32_t Np, const double* x, const double* v, const double* B,
                      const double* gx, const double* gy, const double* gz, const uint32_t* dims,
                      double* grid_mass, double* grid_v) {
  orc* s = orc_create(P);
  if (!s) return 0xffffffffu;
  int d = s->dim, dd = d * d;
  uint32_t kept = 0;
  double org[3] = {gx[0], gy[0], d == 3 ? gz[0] : 0.0};
  /* the kept particles, in input order */
  double* kx = xalloc((size_t)Np * d);
  double* kv = xalloc((size_t)Np * d);
  double* kB = xalloc((size_t)Np * dd);
  for (uint32_t p = 0; p < Np; ++p) {
    int ok = 1;
    for (int a = 0; a < d; ++a) {
      double u = (x[(size_t)p * d + a] - org[a]) * s->one_over_dx;
      if (!(u >= 0.0 && u < (double)dims[a])) { ok = 0; break; }
      int b = (int)floor(u) - 1;
      if (b < 0) b = 0;
      if (b + 3 >= (int)dims[a]) ok = 0;
    }
    if (!ok) continue;
    memcpy(kx + (size_t)kept * d, x + (size_t)p * d, sizeof(double) * d);
    memcpy(kv + (size_t)kept * d, v + (size_t)p * d, sizeof(double) * d);
    if (B) memcpy(kB + (size_t)kept * dd, B + (size_t)p * dd, sizeof(double) * dd);
    kept++;
  }
  orc_set_particles(s, kept, kx, kv, NULL, B ? kB : NULL, NULL);
  free(kx); free(kv); free(kB);
  s->Nx = dims[0];
  s->Ny = dims[1];
  s->Nz = d == 3 ? dims[2] : 1;
  s->G = s->Nx * s->Ny * s->Nz;
  s->gx = (double*)malloc(sizeof(double) * s->Nx);
  s->gy = (double*)malloc(sizeof(double) * s->Ny);
  s->gz = (double*)malloc(sizeof(double) * s->Nz);
  memcpy(s->gx, gx, sizeof(double) * s->Nx);
  memcpy(s->gy, gy, sizeof(double) * s->Ny);
  if (d == 3) memcpy(s->gz, gz, sizeof(double) * s->Nz); else s->gz[0] = 0.0;
  s->xc = org[0];
  s->yc = org[1];
  s->zc = org[2];
  s->ng = 0;
  resize_grid(s);
  p2g(s);
  memcpy(grid_mass, s->gmass, sizeof(double) * s->G);
  memcpy(grid_v, s->gv, sizeof(double) * s->G * d);
  orc_destroy(s);
  return Np - kept;
}
