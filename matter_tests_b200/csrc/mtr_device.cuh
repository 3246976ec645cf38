// mtr_device.cuh — device-side types and math shared by the MPM step kernels.
//
// Everything here is written for sm_100a.  The return mapping, the SVD and
// every projection are FP64 on both paths; the spline weights are templated on
// the arithmetic type so the mixed-precision path can evaluate them in FP32.
// Small matrices are register arrays indexed with compile-time indices only
// (all loops over DIM are unrolled), so nothing spills to local memory.
#pragma once
#include <cstdint>

#include "../../include/matter_gpu.h"

#define MTR_MAXP 16
#define MTR_MAXO 16

namespace mtr {

// FP64 transcendental functions as out-of-line calls for the return mapping:
// its kernels stall most on instruction fetch, and one shared copy of each
// function is smaller than an inlined copy per singular value, branch and
// model.  The results are those of the functions themselves.
static __device__ __noinline__ double ool_log(double x) { return log(x); }
static __device__ __noinline__ double ool_exp(double x) { return exp(x); }
static __device__ __noinline__ double ool_pow(double x, double y) { return pow(x, y); }
static __device__ __noinline__ double ool_sinh(double x) { return sinh(x); }
static __device__ __noinline__ double ool_asinh(double x) { return asinh(x); }

// Constants of Simulation::simulate (simulation.cpp:94-136) plus the public
// fields the step reads (simulation.hpp:36-106), packed for the device.
struct DevParams {
  int dim, deg;
  int plastic_model, elastic_model, hardening_law;
  int use_pradhana, use_mises_q, use_mibf, use_musl, gravity_special, change_particle_positions;
  int store_pic_flip;  // keep per-particle pic/flip of the last step for inspection
  int nobjects, nplates;
  uint32_t end_frame;
  uint32_t Np;
  double flip_ratio, cfl, dx, one_over_dx, apicDinverse, particle_mass, particle_volume;
  double lambda, mu, K, wave_speed, dt_max, frame_dt, final_time;
  double q_prefac, d_prefac, e_mu_prefac, f_mu_prefac, rma_prefac, fac_Q;
  double gravity_final[3], gravity_time, grid_ref[3];
  double E, nu, stress_tolerance, xi, q_max, q_min, p_min, M, q_cohesion, perzyna_exp, perzyna_visc, beta, p0,
      mu_1, mu_2;
  double mui0;  // muI every particle starts from when use_mibf (simulation.cpp:138-145)
  // Jacobi SVD stopping size relative to the largest diagonal entry: FP64
  // epsilon on the FP64 path; 1e-12 on the mixed path, whose FP32 F - I
  // holds the strain to about 1e-10 (smaller off-diagonals carry no data)
  double svd_rel;
  int pbc;       // periodic in x over [0, L[0]] (pbc.cpp)
  double L[3];   // Lx, Ly, Lz (simulation.hpp:60-66)
  // a Perzyna plastic multiplier in (-dgamma_tol, 0) is rounding and is taken
  // as zero rather than reported: 0 on the FP64 path (the reference's checks,
  // plasticity.cpp:190,286; 1e-14 for Cam-Clay, plasticity.cpp:546-547) and
  // 1e-9 on the mixed path, whose FP32 strains carry about that much
  double dgamma_tol;
  mtr_object objects[MTR_MAXO];
  // dense level sets of MTR_OBJ_LEVELSET objects (mtr_set_levelset)
  struct LevelSet {
    const float* phi;   // n[0] * n[1] * n[2] samples
    const float* grad;  // 3 per sample
    uint32_t n[3];
    double org[3], h, inv_h, background;
  } ls[MTR_MAX_LEVELSETS];
};

// Per-step state that lives on the device so a whole step (and many steps in
// a CUDA graph) runs without a host round trip: the clock of simulate()
// (simulation.cpp:168-200), the grid of remesh.cpp and the moving plates.
struct StepHeader {
  double time, dt;
  uint32_t step, frame;
  int32_t done, abort;
  int32_t cur;  // particle buffer (0/1) holding the state after the last completed step
  uint32_t status, first_bad;
  uint32_t stop_frame;  // steps are skipped once frame >= stop_frame (frame-by-frame runs)
  uint32_t stop_step;   // steps are skipped once step >= stop_step (batched runs)
  double gravity[3];
  double org[3];        // grid.xc, grid.yc, grid.zc
  uint32_t N[3];        // Nx, Ny, Nz (Nz = 1 in 2D)
  uint32_t G;           // grid_nodes
  uint32_t T[3];        // tiles per axis
  uint32_t ntiles;
  double min_init[3], max_init[3], low_init[3], high_init[3];
  unsigned long long plastic_count;
  // FP64 balances of the last step (simulation.cpp:292-333): grid mass and
  // momentum right after P2G, particle mass and momentum before it
  double grid_mass, grid_mom[3], part_mom[3];
  mtr_plate plates[MTR_MAXP];
};

// Per-block partial of the step's opening reductions (update_dt.cpp:7-12,
// remesh.cpp:42-83): min and max of x per axis and max |v|^2.
struct BBoxPartial {
  double mn[3], mx[3], v2;
  double vsum[3];  // sum of particle velocities (for the momentum balance)
};

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ int sgn(double v) { return (0.0 < v) - (v < 0.0); }  // tools.hpp:90-92
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }  // std::max

template <int D>
struct Mat {
  double m[D][D];
};

template <int D>
__device__ __forceinline__ void mat_eye(double (&A)[D][D]) {
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) A[i][j] = (i == j) ? 1.0 : 0.0;
}

template <int D>
__device__ __forceinline__ double mat_det(const double (&A)[D][D]) {
  if constexpr (D == 2) {
    return A[0][0] * A[1][1] - A[0][1] * A[1][0];
  } else {
    return A[0][0] * (A[1][1] * A[2][2] - A[2][1] * A[1][2]) - A[1][0] * (A[0][1] * A[2][2] - A[2][1] * A[0][2]) +
           A[2][0] * (A[0][1] * A[1][2] - A[1][1] * A[0][2]);
  }
}

// C = A * B
template <int D>
__device__ __forceinline__ void mat_mul(const double (&A)[D][D], const double (&B)[D][D], double (&C)[D][D]) {
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      double s = A[i][0] * B[0][j];
#pragma unroll
      for (int k = 1; k < D; ++k) s += A[i][k] * B[k][j];
      C[i][j] = s;
    }
}

// out = U diag(e) V^T
template <int D>
__device__ __forceinline__ void usv(const double (&U)[D][D], const double (&e)[D], const double (&V)[D][D],
                                    double (&out)[D][D]) {
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      double s = U[i][0] * e[0] * V[j][0];
#pragma unroll
      for (int k = 1; k < D; ++k) s += U[i][k] * e[k] * V[j][k];
      out[i][j] = s;
    }
}

// symmetric U diag(e) U^T packed as 3 (2D: xx, yy, xy) or 6 (3D: xx, yy, zz, xy, xz, yz) values
template <int D>
struct Sym {
  static constexpr int n = D == 3 ? 6 : 3;
};

template <int D>
__device__ __forceinline__ void usu_packed(const double (&U)[D][D], const double (&e)[D], double* t) {
  auto ent = [&](int i, int j) {
    double s = U[i][0] * e[0] * U[j][0];
#pragma unroll
    for (int k = 1; k < D; ++k) s += U[i][k] * e[k] * U[j][k];
    return s;
  };
  if constexpr (D == 3) {
    t[0] = ent(0, 0);
    t[1] = ent(1, 1);
    t[2] = ent(2, 2);
    t[3] = ent(0, 1);
    t[4] = ent(0, 2);
    t[5] = ent(1, 2);
  } else {
    t[0] = ent(0, 0);
    t[1] = ent(1, 1);
    t[2] = ent(0, 1);
  }
}

template <int D, typename T>
__device__ __forceinline__ T sym_at(const T* t, int i, int j) {
  if constexpr (D == 3) {
    if (i == j) return t[i];
    int s = i + j;  // (0,1)->1, (0,2)->2, (1,2)->3
    return t[2 + s];
  } else {
    return i == j ? t[i] : t[2];
  }
}

// ---------------------------------------------------------------------------
// B-spline basis (tools.hpp:108-188): quadratic (DEG 2) and cubic (DEG 3)
// ---------------------------------------------------------------------------
// R is the arithmetic type: double on the FP64 path, float for the FP32
// weights of the mixed-precision path (same expressions, same order).
template <int DEG, typename R>
__device__ __forceinline__ R bspline_N(R u) {
  R a = fabs(u);
  if constexpr (DEG == 3) {
    if (a < R(1.0)) return R(0.5) * a * a * a - a * a + R(2.0 / 3.0);
    if (a < R(2.0)) return R(1.0 / 6.0) * (R(2.0) - a) * (R(2.0) - a) * (R(2.0) - a);
    return R(0.0);
  } else {
    if (a < R(0.5)) return R(0.75) - a * a;
    if (a < R(1.5)) return R(0.5) * (R(1.5) - a) * (R(1.5) - a);
    return R(0.0);
  }
}

template <int DEG, typename R>
__device__ __forceinline__ R bspline_dN(R u) {
  R a = fabs(u);
  const R sg = R((R(0.0) < u) - (u < R(0.0)));  // tools.hpp:90-92
  if constexpr (DEG == 3) {
    if (a < R(1.0)) return u * (R(1.5) * a - R(2.0));
    if (a < R(2.0)) return R(-0.5) * sg * (R(2.0) - a) * (R(2.0) - a);
    return R(0.0);
  } else {
    if (a < R(0.5)) return R(-2) * u;
    if (a < R(1.5)) return u - R(1.5) * sg;
    return R(0.0);
  }
}

// ---------------------------------------------------------------------------
// SVD: two-sided cyclic Jacobi (Golub & Van Loan, 4th ed., §8.6.3; 2x2
// symmetrising rotation §8.6.2; symSchur2 Alg. 8.5.1).  Output convention of
// the Eigen::JacobiSVD the reference calls (plasticity.cpp:19,
// simulation.hpp:232): singular values >= 0 in decreasing order, U and V
// orthogonal (either may be improper), A = U diag(S) V^T.  The cosines come
// from one reciprocal square root each instead of a square root and a
// division (same rotation, rounded differently at the last bit).  `rel` is
// the off-diagonal size (relative to the largest diagonal entry) below which
// a pair counts as diagonal: FP64 epsilon by default.
// ---------------------------------------------------------------------------
struct JacobiAngles {
  double l00, l01, l10, l11, cj, sj;
};

// The rotations of one 2x2 block [a b; c e].  Out of line (OOL), the three
// pivot pairs of a 3x3 sweep share one copy of this code, which keeps the
// return-mapping kernels that hold several models smaller (they stall most on
// instruction fetch: Cam-Clay G2P 7-10% faster); the kernel compiled for
// mu(I) alone measured 1-3% faster with it inline.
static __device__ __forceinline__ JacobiAngles jacobi_angles(double a, double b, double c, double e) {
  double c1 = 1.0, s1 = 0.0;
  const double tr = a + e, df = b - c;
  if (fabs(df) >= 2.2250738585072014e-308) {
    const double u = tr / df;
    const double ri = rsqrt(1.0 + u * u);  // 1 / sqrt(1 + u^2) in one operation
    s1 = ri;
    c1 = u * ri;
  }
  const double m00 = c1 * a - s1 * c;
  const double m01 = c1 * b - s1 * e;
  const double m11 = s1 * b + c1 * e;
  double cj = 1.0, sj = 0.0;
  if (m01 != 0.0) {
    double tau = (m11 - m00) / (2.0 * m01);
    double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
    cj = rsqrt(1.0 + t * t);
    sj = t * cj;
  }
  JacobiAngles r;
  r.l00 = c1 * cj - s1 * sj;
  r.l01 = c1 * sj + s1 * cj;
  r.l10 = -s1 * cj - c1 * sj;
  r.l11 = -s1 * sj + c1 * cj;
  r.cj = cj;
  r.sj = sj;
  return r;
}
static __device__ __noinline__ JacobiAngles jacobi_angles_ool(double a, double b, double c, double e) {
  return jacobi_angles(a, b, c, e);
}

template <int D, bool OOL = false>
__device__ __forceinline__ void jacobi_rotate(double (&A)[D][D], double (&U)[D][D], double (&V)[D][D], int q, int p,
                                              double& maxdiag) {
  const JacobiAngles r = OOL ? jacobi_angles_ool(A[q][q], A[q][p], A[p][q], A[p][p])
                             : jacobi_angles(A[q][q], A[q][p], A[p][q], A[p][p]);
  const double l00 = r.l00, l01 = r.l01, l10 = r.l10, l11 = r.l11, cj = r.cj, sj = r.sj;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    double aq = A[q][k], ap = A[p][k];
    A[q][k] = l00 * aq + l10 * ap;
    A[p][k] = l01 * aq + l11 * ap;
  }
#pragma unroll
  for (int k = 0; k < D; ++k) {
    double aq = A[k][q], ap = A[k][p];
    A[k][q] = cj * aq - sj * ap;
    A[k][p] = sj * aq + cj * ap;
  }
#pragma unroll
  for (int k = 0; k < D; ++k) {
    double uq = U[k][q], up = U[k][p];
    U[k][q] = l00 * uq + l10 * up;
    U[k][p] = l01 * uq + l11 * up;
    double vq = V[k][q], vp = V[k][p];
    V[k][q] = cj * vq - sj * vp;
    V[k][p] = sj * vq + cj * vp;
  }
  maxdiag = dmax(maxdiag, dmax(fabs(A[p][p]), fabs(A[q][q])));
}

template <int D>
__device__ __forceinline__ bool jacobi_needs(const double (&A)[D][D], int q, int p, double maxdiag, double rel) {
  double thr = dmax(2.2250738585072014e-308, 2.0 * rel * maxdiag);
  return fabs(A[p][q]) > thr || fabs(A[q][p]) > thr;
}

template <int D>
__device__ __forceinline__ void col_swap(double (&U)[D][D], double (&V)[D][D], double (&s)[D], int i, int j) {
  double t = s[i];
  s[i] = s[j];
  s[j] = t;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    t = U[k][i];
    U[k][i] = U[k][j];
    U[k][j] = t;
    t = V[k][i];
    V[k][i] = V[k][j];
    V[k][j] = t;
  }
}

template <int D, bool OOL = false>
__device__ void svd(const double (&Ain)[D][D], double (&U)[D][D], double (&S)[D], double (&V)[D][D],
                    double rel = 2.220446049250313e-16) {
  double A[D][D];
  double scale = 0.0;
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) scale = dmax(scale, fabs(Ain[i][j]));
  if (scale == 0.0 || !isfinite(scale)) scale = 1.0;
  const double inv = 1.0 / scale;
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) A[i][j] = Ain[i][j] * inv;
  mat_eye<D>(U);
  mat_eye<D>(V);
  double maxdiag = 0.0;
#pragma unroll
  for (int i = 0; i < D; ++i) maxdiag = dmax(maxdiag, fabs(A[i][i]));
  for (int sweep = 0; sweep < 32; ++sweep) {
    bool rotated = false;
    if (jacobi_needs<D>(A, 0, 1, maxdiag, rel)) {
      jacobi_rotate<D, OOL>(A, U, V, 0, 1, maxdiag);
      rotated = true;
    }
    if constexpr (D == 3) {
      if (jacobi_needs<D>(A, 0, 2, maxdiag, rel)) {
        jacobi_rotate<D, OOL>(A, U, V, 0, 2, maxdiag);
        rotated = true;
      }
      if (jacobi_needs<D>(A, 1, 2, maxdiag, rel)) {
        jacobi_rotate<D, OOL>(A, U, V, 1, 2, maxdiag);
        rotated = true;
      }
    }
    if (!rotated) break;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) {
    double a = A[i][i];
    S[i] = fabs(a) * scale;
    if (a < 0.0) {
#pragma unroll
      for (int k = 0; k < D; ++k) U[k][i] = -U[k][i];
    }
  }
  // decreasing order (selection order of the oracle: i = 0, then 1)
  if constexpr (D == 3) {
    int m = 0;
    double sm = S[0];
    if (S[1] > sm) {
      m = 1;
      sm = S[1];
    }
    if (S[2] > sm) m = 2;
    if (m == 1) col_swap<D>(U, V, S, 0, 1);
    if (m == 2) col_swap<D>(U, V, S, 0, 2);
    if (S[2] > S[1]) col_swap<D>(U, V, S, 1, 2);
  } else {
    if (S[1] > S[0]) col_swap<D>(U, V, S, 0, 1);
  }
}

// ---------------------------------------------------------------------------
// SVD through the symmetric eigenproblem of B = F F^T = U S^2 U^T: cyclic
// Jacobi on B (Golub & Van Loan, 4th ed., Alg. 8.5.2 with the symmetric
// 2x2 Schur rotation of Alg. 8.5.1), S = sqrt of the eigenvalues, V =
// F^T U S^-1, so that F = U S V^T.  Per rotation it updates the symmetric B
// and U only (15 live values instead of the 27 of A, U and V), about a third
// of the arithmetic of the two-sided iteration.  S has the relative accuracy
// of FP64 (the eigenvalues of B carry an absolute error of ~eps |B|, and the
// singular values stay far from zero), and within a cluster of nearly equal
// singular values U is some orthonormal basis of the cluster, which the
// isotropic return mapping and Hencky stress do not see; the results differ
// from the two-sided iteration's by rounding only.  The singular values are
// not sorted.  A singular value below 1e-6 of the largest (where F^T U S^-1
// loses accuracy) falls back to the two-sided iteration.
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void sym_rotate(double (&Bm)[D][D], double (&U)[D][D], int p, int q, double& maxdiag) {
  const double bpq = Bm[p][q];
  const double tau = (Bm[q][q] - Bm[p][p]) / (2.0 * bpq);
  const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
  const double c = rsqrt(1.0 + t * t), sn = t * c;
  Bm[p][p] -= t * bpq;
  Bm[q][q] += t * bpq;
  Bm[p][q] = Bm[q][p] = 0.0;
#pragma unroll
  for (int r = 0; r < D; ++r) {
    if (r == p || r == q) continue;
    const double brp = Bm[r][p], brq = Bm[r][q];
    Bm[r][p] = Bm[p][r] = c * brp - sn * brq;
    Bm[r][q] = Bm[q][r] = sn * brp + c * brq;
  }
#pragma unroll
  for (int k = 0; k < D; ++k) {
    const double ukp = U[k][p], ukq = U[k][q];
    U[k][p] = c * ukp - sn * ukq;
    U[k][q] = sn * ukp + c * ukq;
  }
  maxdiag = dmax(maxdiag, dmax(fabs(Bm[p][p]), fabs(Bm[q][q])));
}

template <int D>
__device__ void svd_sym(const double (&F)[D][D], double (&U)[D][D], double (&S)[D], double (&V)[D][D],
                        double rel) {
  double Bm[D][D];
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = i; j < D; ++j) {
      double b = F[i][0] * F[j][0];
#pragma unroll
      for (int k = 1; k < D; ++k) b += F[i][k] * F[j][k];
      Bm[i][j] = Bm[j][i] = b;
    }
  mat_eye<D>(U);
  double maxdiag = 0.0;
#pragma unroll
  for (int i = 0; i < D; ++i) maxdiag = dmax(maxdiag, fabs(Bm[i][i]));
  for (int sweep = 0; sweep < 16; ++sweep) {
    bool rotated = false;
    if (fabs(Bm[0][1]) > rel * maxdiag) {
      sym_rotate<D>(Bm, U, 0, 1, maxdiag);
      rotated = true;
    }
    if constexpr (D == 3) {
      if (fabs(Bm[0][2]) > rel * maxdiag) {
        sym_rotate<D>(Bm, U, 0, 2, maxdiag);
        rotated = true;
      }
      if (fabs(Bm[1][2]) > rel * maxdiag) {
        sym_rotate<D>(Bm, U, 1, 2, maxdiag);
        rotated = true;
      }
    }
    if (!rotated) break;
  }
  double smax = 0.0;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    S[i] = sqrt(dmax(Bm[i][i], 0.0));
    smax = dmax(smax, S[i]);
  }
  bool small = !(smax > 0.0);
#pragma unroll
  for (int i = 0; i < D; ++i) small = small || !(S[i] >= 1e-6 * smax);
  if (small) {
    svd<D, true>(F, U, S, V, rel);
    return;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) {
    const double inv = 1.0 / S[i];
#pragma unroll
    for (int k = 0; k < D; ++k) {
      double v = F[0][k] * U[0][i];
#pragma unroll
      for (int j = 1; j < D; ++j) v += F[j][k] * U[j][i];
      V[k][i] = v * inv;
    }
  }
}

// ---------------------------------------------------------------------------
// status reporting (the reference's int exit, simulation.hpp:28)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void raise_status(StepHeader* H, uint32_t flag, uint32_t id) {
  atomicOr(&H->status, flag);
  atomicMin(&H->first_bad, id);
}

}  // namespace mtr
