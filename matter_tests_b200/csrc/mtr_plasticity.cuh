// mtr_plasticity.cuh — per-particle elasto-viscoplastic return mapping in
// Hencky-strain space (Simulation::plasticity, plasticity.cpp:11-665, and the
// MCC helpers of plasticity_helpers/*.hpp), fused with the Kirchhoff stress
// the next step's force scatter needs.
//
// The reference recomputes tau = P(F) F^T with a second SVD of the stored F at
// the start of the next step (explicit_euler_update.cpp:22-40 via
// HenckyPiola, simulation.hpp:231-238).  Because F leaves this function either
// unchanged (its SVD is at hand) or rebuilt as U exp(h) V^T, tau is
//   tau = U diag(2 mu log s_i + lambda sum_j log s_j) U^T
// with log s = log of the trial singular values or h; it is stored packed
// (symmetric, 3 or 6 values) so the force scatter needs no SVD at all.
#pragma once
#include "mtr_device.cuh"

namespace mtr {

// flags that make simulate() return (the reference's exit = 1)
constexpr uint32_t kExitMask = MTR_STATUS_BAD_BC | MTR_STATUS_RMA_NOCONV | MTR_STATUS_RMA_NOSTEP |
                               MTR_STATUS_NEG_DGAMMA | MTR_STATUS_BAD_MODEL | MTR_STATUS_RESID_DIFF |
                               MTR_STATUS_STENCIL_OOB;

struct PScalars {
  double eps_pl_dev, eps_pl_vol, eps_pl_vol_pradhana, delta_gamma, viscosity, muI;
};

// MCCRMAExplicit (mcc_rma_explicit.hpp:8-96)
__device__ inline bool mcc_rma_explicit(double& p_io, double& q_io, double M, double p0, double beta, double mu, double K,
                                 double rma_prefac) {
  double p = p_io, q = q_io;
  double y = M * M * (p - p0) * (p + beta * p0) + (q * q);
  if (!(y > 0)) return false;
  double delta_gamma = 0;
  const double pt = p, qt = q;
  const double dkdp = 2 * M * M;
  const double dldq = 2;
  const int max_iter = 40;
  for (int iter = 0; iter < max_iter; iter++) {
    y = M * M * (p - p0) * (p + beta * p0) + (q * q);
    double k = M * M * (beta * p0 + 2 * p - p0);
    double l = 2 * q;
    double r1 = pt - p - K * delta_gamma * k;
    double r2 = qt - q - rma_prefac * mu * delta_gamma * l;
    if (iter > 4 && fabs(y) < 1e-3 && fabs(r1) < 1e-3 && fabs(r2) < 1e-3) break;
    if (iter == max_iter - 1) {
      if (!(p0 > 0.1)) {
        p = 1e-15;
        q = 1e-15;
      }
      break;
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
  p_io = p;
  q_io = q;
  return true;
}

// limited_search_exponential / limited_search_sinh (limited_search_*.hpp)
template <bool SINH>
__device__ double limited_search(double epv, double epv_t, double epv_delta, double xi, double K, double p_t,
                                 double p00, double p0_min, double beta, int& right) {
  double scale = 1.;
  int tries = 0, f = 0;
  const int max_tries = 32;
  double test_epv = epv;
  while (tries < max_tries) {
    test_epv = epv - scale * epv_delta;
    double pp0 = SINH ? dmax(p0_min, K * ool_sinh(-xi * test_epv + ool_asinh(p00 / K))) : p00 * ool_exp(-xi * test_epv);
    double pp = K * (test_epv - epv_t) + p_t;
    double val = 2. * pp + (beta - 1.) * pp0;
    double midpoint = (pp0 - beta * pp0) * 0.5;
    if (fabs(pp - midpoint) <= 1.e-5) break;
    if (((right == 1 && (pp < midpoint || p_t < midpoint)) || (right == 0 && (pp > midpoint || p_t > midpoint))) &&
        tries > -1) {
      test_epv = epv;
      right = -1;
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
    if (f > 1) return __longlong_as_double(0x7ff0000000000000LL);  // +inf
  }
  return test_epv;
}

// MCCRMAImplicitExponentialOnevar (mcc_rma_implicit_exponential_onevar.hpp:9-166)
// and MCCRMAImplicitSinhOnevar (mcc_rma_implicit_sinh_onevar.hpp:9-171).
template <bool SINH>
__device__ bool mcc_rma_implicit(double& p_io, double& q_io, double M, double p00, double beta, double mu, double K,
                                 double xi, double epv, uint32_t& flags) {
  double p = p_io, q = q_io;
  const double Msq = M * M;
  const double damping_factor = 1;
  double p0 = SINH ? dmax(0.01, K * ool_sinh(-xi * epv + ool_asinh(p00 / K))) : p00 * ool_exp(-xi * epv);
  const double p0_t = p0;
  double y = Msq * (p * p + (beta - 1.) * p0 * p - beta * p0 * p0) + damping_factor * q * q;
  if (y <= 0) return false;
  const double scale_factor = 1. / p0_t;
  const double p0_min = 0.01 * scale_factor;
  p0 = 1.;
  p00 *= scale_factor;
  p *= scale_factor;
  q *= scale_factor;
  mu *= scale_factor;
  K *= scale_factor;
  const double p_t = p, q_t = q, epv_t = epv;
  int right = (p_t > 0.5 * (p0 - beta * p0)) ? 1 : 0;
  const int max_iter = SINH ? 40 : 30;
  for (int iter = 0; iter < max_iter; iter++) {
    double midpoint = (p0 - beta * p0) * 0.5;
    if (fabs(p - midpoint) < 1e-4) {
      q = M * sqrt((p0 - p) * (beta * p0 + p) / damping_factor);
      p *= p0_t;
      q *= p0_t;
      p_io = p;
      q_io = q;
      return true;
    }
    p = (epv - epv_t) * K + p_t;
    double p0_helper = 0.0;
    if (SINH) {
      p0_helper = K * ool_sinh(-xi * epv + ool_asinh(p00 / K));
      p0 = dmax(p0_min, p0_helper);
    } else {
      p0 = p00 * ool_exp(-xi * epv);
    }
    double denom = 2. * K * Msq * p + Msq * (beta - 1.) * K * p0;
    double dg_step = (p_t - p) / denom;
    double q_denom = 1. + 2. * mu * damping_factor * dg_step;
    q = q_t / q_denom;
    y = Msq * (p - p0) * (p + beta * p0) + damping_factor * q * q;
    if (iter > 5 && fabs(y) < 1e-4) break;
    if (SINH && iter == max_iter - 1 && p0 > p0_min) flags |= MTR_STATUS_RMA_NOCONV;
    double dp_depv = K;
    double dp0_depv;
    if (SINH) {
      double h = -xi * K * cosh(-xi * epv + ool_asinh(p00 / K));
      dp0_depv = (p0_helper > p0_min) ? 0.5 * (h + h - p0_min) : 0.5 * (h + p0_min - h);
    } else {
      dp0_depv = -xi * p0;
    }
    double ddelta_gamma_depv =
        (-dp_depv / denom) - (p_t - p) * (2. * K * Msq * dp_depv + Msq * (beta - 1.) * K * dp0_depv) / (denom * denom);
    double dq_depv = -q_t * 2. * mu * damping_factor * ddelta_gamma_depv / (q_denom * q_denom);
    double dy_depv = Msq * (dp_depv - dp0_depv) * (p + beta * p0) + Msq * (p - p0) * (beta * dp0_depv + dp_depv) +
                     2. * damping_factor * q * dq_depv;
    epv = limited_search<SINH>(epv, epv_t, y / dy_depv, xi, K, p_t, p00, p0_min, beta, right);
    if (isinf(epv) && epv > 0) {
      flags |= MTR_STATUS_RMA_NOSTEP;
      break;
    }
  }
  p = dmax(p, -beta * p0);
  p = dmin(p, p0);
  q = M * sqrt((p0 - p) * (beta * p0 + p) / damping_factor);
  p *= p0_t;
  q *= p0_t;
  p_io = p;
  q_io = q;
  return true;
}

// Perzyna Newton loop of VMVisc / DPVisc / MCCVisc (plasticity.cpp:197-229,
// 293-323, 558-588); VMVisc's yield stress depends on delta_gamma (is_vm).
__device__ inline double perzyna_newton(const DevParams& P, double dt, double q_trial, double q_yield, bool is_vm,
                                 double eps_pl_dev, uint32_t& flags) {
  const double pe = P.perzyna_exp, pv = P.perzyna_visc, fm = P.f_mu_prefac;
  double delta_gamma = 0.01 * (q_trial - q_yield) / fm;
  const int max_iter = 60;
  for (int iter = 0; iter < max_iter; iter++) {
    if (iter == max_iter - 1) flags |= MTR_STATUS_RMA_NOCONV;
    double tm = pv * delta_gamma + dt;
    double tmp = dt / tm;
    double tmp1 = ool_pow(tmp, pe);
    double qdiff = 0.0;
    if (is_vm) {
      double ex = ool_exp(-P.xi * (eps_pl_dev + (1.0 / P.d_prefac) * delta_gamma));
      q_yield = P.q_min + (P.q_max - P.q_min) * ex;
      qdiff = -P.xi / P.d_prefac * (P.q_max - P.q_min) * ex;
    }
    double residual = (q_trial - fm * delta_gamma) * tmp1 - q_yield;
    if (fabs(residual) < 1e-2) break;
    double residual_diff = -fm * tmp1 + (q_trial - fm * delta_gamma) * pe * ool_pow(tmp, pe - 1) * (-pv * dt) / (tm * tm);
    if (is_vm) residual_diff -= qdiff;
    if (fabs(residual_diff) < 1e-14) flags |= MTR_STATUS_RESID_DIFF;
    delta_gamma -= residual / residual_diff;
    if (delta_gamma < 0) delta_gamma = 1e-10;
  }
  return delta_gamma;
}

// Kirchhoff stress of a Hencky material from log-stretches h and left
// singular vectors U: tau = U diag(2 mu h_i + lambda tr h) U^T.
template <int D>
__device__ __forceinline__ void hencky_tau(const DevParams& P, const double (&U)[D][D], const double (&h)[D],
                                           double* tau) {
  double tr = h[0];
#pragma unroll
  for (int i = 1; i < D; ++i) tr += h[i];
  double e[D];
#pragma unroll
  for (int i = 0; i < D; ++i) e[i] = 2.0 * P.mu * h[i] + P.lambda * tr;
  usu_packed<D>(U, e, tau);
}

// NeoHookeanPiola (simulation.hpp:227-229) times F^T:
// tau = mu (F F^T - I) + lambda log(det F) I.
template <int D>
__device__ __forceinline__ void neohookean_tau(const DevParams& P, const double (&F)[D][D], double* tau) {
  const double lj = ool_log(mat_det<D>(F));
  auto ffT = [&](int i, int j) {
    double s = F[i][0] * F[j][0];
#pragma unroll
    for (int k = 1; k < D; ++k) s += F[i][k] * F[j][k];
    return s;
  };
  if constexpr (D == 3) {
    tau[0] = P.mu * (ffT(0, 0) - 1.0) + P.lambda * lj;
    tau[1] = P.mu * (ffT(1, 1) - 1.0) + P.lambda * lj;
    tau[2] = P.mu * (ffT(2, 2) - 1.0) + P.lambda * lj;
    tau[3] = P.mu * ffT(0, 1);
    tau[4] = P.mu * ffT(0, 2);
    tau[5] = P.mu * ffT(1, 2);
  } else {
    tau[0] = P.mu * (ffT(0, 0) - 1.0) + P.lambda * lj;
    tau[1] = P.mu * (ffT(1, 1) - 1.0) + P.lambda * lj;
    tau[2] = P.mu * ffT(0, 1);
  }
}

// The elastic stress of the initial state (what HenckyPiola / NeoHookeanPiola
// give for the uploaded F at the first step).
template <int D>
__device__ void initial_tau(const DevParams& P, const double (&F)[D][D], double* tau) {
  if (P.plastic_model == MTR_PM_SNOW) {  // dPsidF starts at zero (data_structures.hpp:21)
#pragma unroll
    for (int i = 0; i < Sym<D>::n; ++i) tau[i] = 0.0;
    return;
  }
  if (P.elastic_model == MTR_EL_NEOHOOKEAN) {
    neohookean_tau<D>(P, F, tau);
    return;
  }
  double U[D][D], V[D][D], S[D], h[D];
  svd<D>(F, U, S, V, P.svd_rel);
#pragma unroll
  for (int i = 0; i < D; ++i) h[i] = ool_log(fabs(S[i]));
  hencky_tau<D>(P, U, h, tau);
}

// Simulation::plasticity for one particle (plasticity.cpp:11-665).
// F: in = Fe_trial, out = the particle's new F.  Returns true when the
// particle was projected (the reference's plastic_count).
// PM >= 0 compiles the function for that plastic model only (the step's
// model is then known at compile time and the other models' code is not
// emitted: a smaller kernel that fits the instruction cache); PM = -1 reads
// the model from P at run time.
// SYM selects the SVD through the symmetric eigenproblem of F F^T
// (svd_sym); otherwise the two-sided Jacobi iteration with the reference's
// conventions.
template <int D, int PM = -1, bool SYM = false>
__device__ bool return_map(const DevParams& P, double dt, double (&F)[D][D], PScalars& s, double* tau,
                           uint32_t& flags) {
  const int pm = PM >= 0 ? PM : P.plastic_model;
  if (pm == MTR_PM_NOPLASTICITY) {
    if (P.elastic_model == MTR_EL_NEOHOOKEAN) {
      neohookean_tau<D>(P, F, tau);
    } else {
      double U[D][D], V[D][D], S[D], h[D];
      if constexpr (SYM)
        svd_sym<D>(F, U, S, V, P.svd_rel);
      else
        svd<D>(F, U, S, V, P.svd_rel);
#pragma unroll
      for (int i = 0; i < D; ++i) h[i] = ool_log(fabs(S[i]));
      hencky_tau<D>(P, U, h, tau);
    }
    return false;
  }
  if (pm < 0 || pm > MTR_PM_SNOW) {
    flags |= MTR_STATUS_BAD_MODEL;
    return false;
  }
  const double dim = (double)D;
  const double K = P.K, M = P.M, qc = P.q_cohesion;
  const double e_mu = P.e_mu_prefac, d_pre = P.d_prefac, f_mu = P.f_mu_prefac;
  double U[D][D], V[D][D], S[D];
  if constexpr (SYM)
    svd_sym<D>(F, U, S, V, P.svd_rel);
  else
    svd<D, PM != MTR_PM_DPMUI>(F, U, S, V, P.svd_rel);
  double hencky[D], hdev[D];
#pragma unroll
  for (int i = 0; i < D; ++i) hencky[i] = ool_log(dmax(fabs(S[i]), 1e-4));  // plasticity.cpp:21
  double hencky_trace = hencky[0];
#pragma unroll
  for (int i = 1; i < D; ++i) hencky_trace += hencky[i];
#pragma unroll
  for (int i = 0; i < D; ++i) hdev[i] = hencky[i] - (hencky_trace / dim) * 1.0;
  double sq = hdev[0] * hdev[0];
#pragma unroll
  for (int i = 1; i < D; ++i) sq += hdev[i] * hdev[i];
  const double hdn = sqrt(sq);
  if (hdn > 0) {
#pragma unroll
    for (int i = 0; i < D; ++i) hdev[i] /= hdn;
  }

  bool rewrite = false;  // F <- U exp(hencky) V^T
  bool plastic = false;
  auto set_iso = [&](double pp) {
#pragma unroll
    for (int i = 0; i < D; ++i) hencky[i] = -pp / (K * dim) * 1.0;
  };
  auto shrink_dev = [&](double dg) {
#pragma unroll
    for (int i = 0; i < D; ++i) hencky[i] -= (1.0 / d_pre) * dg * hdev[i];
  };

  if (pm == MTR_PM_VM) {  // plasticity.cpp:30-49
    double delta_gamma = hdn - P.q_max / e_mu;
    if (delta_gamma > 0) {
      plastic = true;
      s.delta_gamma = d_pre * delta_gamma / dt;
#pragma unroll
      for (int i = 0; i < D; ++i) hencky[i] -= delta_gamma * hdev[i];
      rewrite = true;
      s.eps_pl_dev += delta_gamma;
    }
  } else if (pm == MTR_PM_DP) {  // plasticity.cpp:51-85
    double p_trial = -K * hencky_trace;
    double q_yield = M * p_trial + qc;
    if (q_yield < 1e-10) {
      plastic = true;
      double p_proj = -qc / M;
      set_iso(p_proj);
      rewrite = true;
      double delta_gamma = d_pre * hdn;
      s.delta_gamma = delta_gamma / dt;
      s.eps_pl_dev += (1.0 / d_pre) * delta_gamma;
      s.eps_pl_vol += (p_proj - p_trial) / K;
    } else {
      double delta_gamma = d_pre * (hdn - q_yield / e_mu);
      if (delta_gamma > 0) {
        plastic = true;
        s.delta_gamma = delta_gamma / dt;
        shrink_dev(delta_gamma);
        rewrite = true;
        s.eps_pl_dev += (1.0 / d_pre) * delta_gamma;
      }
    }
  } else if (pm == MTR_PM_DPSOFT) {  // plasticity.cpp:87-162
    double p_trial = -K * hencky_trace;
    double q_trial = e_mu * hdn;
    double p_tip_orig = -qc / M;
    double p_tip = p_tip_orig * ool_exp(-P.xi * s.eps_pl_dev);
    double p_shift = P.use_pradhana ? -K * s.eps_pl_vol_pradhana : 0.0;
    double q_yield = M * (p_trial + p_shift) + (-p_tip * M);
    if ((p_trial + p_shift) <= p_tip) {
      plastic = true;
      double p_proj = p_tip_orig * ool_exp(-P.xi * s.eps_pl_dev);
      set_iso(p_proj);
      rewrite = true;
      double delta_gamma = d_pre * hdn;
      s.delta_gamma = delta_gamma / dt;
      s.eps_pl_dev += (1.0 / d_pre) * delta_gamma;
      double inst = (p_proj - p_trial) / K;
      s.eps_pl_vol += inst;
      if (P.use_pradhana) s.eps_pl_vol_pradhana += inst;
    }
    if ((p_trial + p_shift) > p_tip && q_trial <= q_yield) {
      if (P.use_pradhana) s.eps_pl_vol_pradhana = 0;
      s.delta_gamma = 0;
    }
    if ((p_trial + p_shift) > p_tip && q_trial > q_yield) {
      plastic = true;
      double temp_eps_pl_dev = s.eps_pl_dev + (hdn - q_yield / e_mu);
      double p_proj = p_tip_orig * ool_exp(-P.xi * temp_eps_pl_dev);
      if ((p_trial + p_shift) < p_proj) {
        double delta_gamma = d_pre * hdn;
        s.delta_gamma = delta_gamma / dt;
        s.eps_pl_dev += (1.0 / d_pre) * delta_gamma;
        double inst = (p_proj - p_trial) / K;
        s.eps_pl_vol += inst;
        if (P.use_pradhana) s.eps_pl_vol_pradhana += inst;
        set_iso(p_proj);
        rewrite = true;
      } else {
        double q_yield_new = M * (p_trial + p_shift) + (-p_proj * M);
        double delta_gamma = d_pre * (hdn - q_yield_new / e_mu);
        shrink_dev(delta_gamma);
        rewrite = true;
        s.eps_pl_dev += (1.0 / d_pre) * delta_gamma;
        s.delta_gamma = delta_gamma / dt;
        if (P.use_pradhana) s.eps_pl_vol_pradhana = 0;
      }
    }
  } else if (pm == MTR_PM_VMVISC) {  // plasticity.cpp:164-238
    double q_trial = e_mu * hdn;
    double q_yield = P.q_min + (P.q_max - P.q_min) * ool_exp(-P.xi * s.eps_pl_dev);
    double p_trial = -K * hencky_trace;
    if (p_trial < P.p_min * ool_exp(-P.xi * s.eps_pl_vol)) {
      double delta_gamma = q_trial / f_mu;
      double inst = -p_trial / K;
#pragma unroll
      for (int i = 0; i < D; ++i) hencky[i] = 0.0;  // F = U V^T
      rewrite = true;
      s.eps_pl_vol += inst;
      s.eps_pl_dev += (1.0 / d_pre) * delta_gamma;
      s.delta_gamma = delta_gamma / dt;
    } else if (q_trial > q_yield) {
      plastic = true;
      double delta_gamma;
      if (P.perzyna_exp == 1 && P.xi == 0) {
        delta_gamma = (q_trial - q_yield) / (f_mu + q_yield * P.perzyna_visc / dt);
        if (delta_gamma < 0) {
          if (delta_gamma > -P.dgamma_tol)
            delta_gamma = 0;
          else
            flags |= MTR_STATUS_NEG_DGAMMA;
        }
      } else {
        delta_gamma = perzyna_newton(P, dt, q_trial, q_yield, true, s.eps_pl_dev, flags);
      }
      shrink_dev(delta_gamma);
      rewrite = true;
      s.eps_pl_dev += (1.0 / d_pre) * delta_gamma;
      s.delta_gamma = delta_gamma / dt;
    }
  } else if (pm == MTR_PM_DPVISC) {  // plasticity.cpp:240-339
    double p_trial = -K * hencky_trace;
    double q_trial = e_mu * hdn;
    double p_tip = -qc / M;
    double p_shift = P.use_pradhana ? -K * s.eps_pl_vol_pradhana : 0.0;
    double q_yield = M * (p_trial + p_shift) + qc;
    if (P.use_mibf) s.muI = M;
    if ((p_trial + p_shift) < p_tip) {
      double delta_gamma = d_pre * hdn;
      double p_proj = p_tip;
      double inst = (p_proj - p_trial) / K;
      plastic = true;
      set_iso(p_proj);
      rewrite = true;
      s.delta_gamma = delta_gamma / dt;
      s.eps_pl_dev += (1.0 / d_pre) * delta_gamma;
      s.eps_pl_vol += inst;
      if (P.use_pradhana) s.eps_pl_vol_pradhana += inst;
    } else {
      if (P.use_pradhana) s.eps_pl_vol_pradhana = 0;
      s.delta_gamma = 0;
    }
    if ((p_trial + p_shift) > p_tip && q_trial > q_yield) {
      plastic = true;
      double delta_gamma;
      if (P.perzyna_exp == 1) {
        delta_gamma = (q_trial - q_yield) / (f_mu + q_yield * P.perzyna_visc / dt);
        if (delta_gamma < 0) {
          if (delta_gamma > -P.dgamma_tol)
            delta_gamma = 0;
          else
            flags |= MTR_STATUS_NEG_DGAMMA;
        }
      } else {
        delta_gamma = perzyna_newton(P, dt, q_trial, q_yield, false, 0.0, flags);
      }
      if (P.use_mibf) {
        if (fabs(p_trial + p_shift) < 1e-10)
          s.muI = 1e10;
        else
          s.muI = ((q_trial - f_mu * delta_gamma) - qc) / (p_trial + p_shift);
      }
      shrink_dev(delta_gamma);
      rewrite = true;
      s.eps_pl_dev += (1.0 / d_pre) * delta_gamma;
      s.delta_gamma = delta_gamma / dt;
    }
  } else if (pm == MTR_PM_DPMUI) {  // plasticity.cpp:342-403
    double p_trial = -K * hencky_trace;
    double q_trial = e_mu * hdn;
    const double mu_1 = P.mu_1, mu_2 = P.mu_2, fac_Q = P.fac_Q;
    double p_tip = -qc / mu_1;
    double p_shift = P.use_pradhana ? -K * s.eps_pl_vol_pradhana : 0.0;
    s.muI = mu_1;
    s.viscosity = 0;
    if ((p_trial + p_shift) < p_tip) {
      double delta_gamma = d_pre * hdn;
      double inst = (p_tip - p_trial) / K;
      plastic = true;
      set_iso(p_tip);
      rewrite = true;
      s.delta_gamma = delta_gamma;  // plasticity.cpp:364: no /dt in this branch
      s.eps_pl_dev += (1.0 / d_pre) * delta_gamma;
      s.eps_pl_vol += inst;
      s.eps_pl_vol_pradhana += inst;
    } else {
      s.eps_pl_vol_pradhana = 0;
    }
    double q_yield = mu_1 * (p_trial + p_shift) + qc;
    if ((p_trial + p_shift) > p_tip && q_trial > (q_yield + P.stress_tolerance)) {
      plastic = true;
      double p_special = p_trial + p_shift - p_tip + P.stress_tolerance;
      double fac_a = f_mu * dt;
      double fac_b = p_trial * (mu_2 - mu_1) + f_mu * dt * fac_Q * sqrt(p_special) - (q_trial - q_yield);
      double fac_c = -(q_trial - q_yield) * fac_Q * sqrt(p_special);
      double delta_gamma = (-fac_b + sqrt(fac_b * fac_b - 4 * fac_a * fac_c)) / (2 * fac_a);
      double mu_i = mu_1 + (mu_2 - mu_1) / (fac_Q * sqrt(p_special) / delta_gamma + 1.0);
      s.muI = mu_i;
      s.viscosity = (mu_i - mu_1) * p_special / delta_gamma;
      delta_gamma *= dt;
      shrink_dev(delta_gamma);
      rewrite = true;
      s.eps_pl_dev += (1.0 / d_pre) * delta_gamma;
      s.delta_gamma = delta_gamma / dt;
    }
  } else if (pm == MTR_PM_MCCMUI || pm == MTR_PM_MCC || pm == MTR_PM_MCCVISC) {  // plasticity.cpp:405-621
    const bool mui = pm == MTR_PM_MCCMUI;
    const double Mm = mui ? P.mu_1 : M;
    double p_stress = -K * hencky_trace;
    double q_stress = e_mu * hdn;
    const double q_trial = q_stress;
    const double p0 = P.p0, beta = P.beta, xi = P.xi, st = P.stress_tolerance;
    if (pm == MTR_PM_MCCVISC && P.use_mibf) s.muI = M;
    bool perform_rma = false;
    double p_c = 0.0;
    const int hl = P.hardening_law;
    if (hl == MTR_HL_NOHARD && !mui) {
      perform_rma = mcc_rma_explicit(p_stress, q_stress, Mm, p0, beta, P.mu, K, P.rma_prefac);
    } else if (hl == MTR_HL_EXPOEXPL) {
      p_c = dmax(st, p0 * ool_exp(-xi * s.eps_pl_vol));
      perform_rma = mcc_rma_explicit(p_stress, q_stress, Mm, p_c, beta, P.mu, K, P.rma_prefac);
    } else if (hl == MTR_HL_SINHEXPL) {
      p_c = dmax(st, K * ool_sinh(-xi * s.eps_pl_vol + ool_asinh(p0 / K)));
      perform_rma = mcc_rma_explicit(p_stress, q_stress, Mm, p_c, beta, P.mu, K, P.rma_prefac);
    } else if (hl == MTR_HL_EXPOIMPL) {
      perform_rma = mcc_rma_implicit<false>(p_stress, q_stress, Mm, p0, beta, P.mu, K, xi, s.eps_pl_vol, flags);
    } else if (hl == MTR_HL_SINHIMPL) {
      perform_rma = mcc_rma_implicit<true>(p_stress, q_stress, Mm, p0, beta, P.mu, K, xi, s.eps_pl_vol, flags);
    } else {
      flags |= MTR_STATUS_BAD_MODEL;
    }
    if (mui) {
      s.muI = P.mu_1;
      s.viscosity = 0;
    }
    if (perform_rma) {
      plastic = true;
      double ep = p_stress / (K * dim);
      double inst = hencky_trace + dim * ep;
      s.eps_pl_vol += inst;
      if (mui) {
        if (q_trial > (q_stress + st)) {
          const double mu_1 = P.mu_1, mu_2 = P.mu_2, fac_Q = P.fac_Q;
          if (hl == MTR_HL_EXPOIMPL)
            p_c = dmax(p0 * ool_exp(-xi * s.eps_pl_vol), p_stress + st);
          else if (hl == MTR_HL_SINHIMPL)
            p_c = dmax(K * ool_sinh(-xi * s.eps_pl_vol + ool_asinh(p0 / K)), p_stress + st);
          double p_special = p_stress + beta * p_c + st;
          double fac_a = f_mu * dt;
          double fac_b =
              sqrt((p_c - p_stress) * p_special) * (mu_2 - mu_1) + f_mu * dt * fac_Q * sqrt(p_special) - (q_trial - q_stress);
          double fac_c = -(q_trial - q_stress) * fac_Q * sqrt(p_special);
          double gamma_dot_S = (-fac_b + sqrt(fac_b * fac_b - 4 * fac_a * fac_c)) / (2 * fac_a);
          q_stress = dmax(q_stress, q_trial - f_mu * dt * gamma_dot_S);
          double mu_i = mu_1 + (mu_2 - mu_1) / (fac_Q * sqrt(p_special) / gamma_dot_S + 1.0);
          s.muI = mu_i;
          s.viscosity = (mu_i - mu_1) * sqrt((p_c - p_stress) * p_special) / gamma_dot_S;
          double delta_gamma = (q_trial - q_stress) / f_mu;
          s.eps_pl_dev += (1.0 / d_pre) * delta_gamma;
          s.delta_gamma = delta_gamma / dt;
        }
      } else {
        if (pm == MTR_PM_MCCVISC) {
          double q_yield = q_stress;
          double delta_gamma;
          if (P.perzyna_exp == 1) {
            delta_gamma = (q_trial - q_yield) / (f_mu + q_yield * P.perzyna_visc / dt);
            if (delta_gamma < 0) {
              if (delta_gamma > -dmax(1e-14, P.dgamma_tol))
                delta_gamma = 0;
              else
                flags |= MTR_STATUS_NEG_DGAMMA;
            }
          } else {
            delta_gamma = perzyna_newton(P, dt, q_trial, q_yield, false, 0.0, flags);
          }
          q_stress = dmax(q_yield, q_trial - f_mu * delta_gamma);
          if (P.use_mibf) {
            if (hl == MTR_HL_EXPOIMPL)
              p_c = dmax(0.0, p0 * ool_exp(-xi * s.eps_pl_vol));
            else if (hl == MTR_HL_SINHIMPL)
              p_c = dmax(0.0, K * ool_sinh(-xi * s.eps_pl_vol + ool_asinh(p0 / K)));
            if ((p_stress < -beta * p_c + st) || (p_stress > p_c - st))
              s.muI = M;
            else
              s.muI = q_stress / sqrt((p_stress + beta * p_c) * (p_c - p_stress));
          }
        }
        double delta_gamma = (q_trial - q_stress) / f_mu;
        s.eps_pl_dev += (1.0 / d_pre) * delta_gamma;
        s.delta_gamma = delta_gamma / dt;
      }
#pragma unroll
      for (int i = 0; i < D; ++i) hencky[i] = q_stress / e_mu * hdev[i] - ep * 1.0;
      rewrite = true;
    }
  } else if (pm == MTR_PM_SNOW) {  // plasticity.cpp:623-658
    double Sx[D], Sinv[D], ph[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      Sx[i] = S[i];
      if (Sx[i] > 7.5e-3) Sx[i] = 7.5e-3;
    }
#pragma unroll
    for (int i = 0; i < D; ++i)
      if (Sx[i] < 2.5e-2) Sx[i] = 2.5e-2;
#pragma unroll
    for (int i = 0; i < D; ++i) Sinv[i] = (fabs(Sx[i]) > 1e-9) ? 1.0 / Sx[i] : 0.0;
    double Fe_new_inv[D][D], Fp[D][D];
    usv<D>(V, Sinv, U, Fe_new_inv);
    mat_mul<D>(Fe_new_inv, F, Fp);
    double one_minus_Jp = 1.0 - mat_det<D>(Fp);
    double power = dmin(10.0 * one_minus_Jp, 5.0);
    double lambda0 = (P.E * P.nu) / ((1 + P.nu) * (1 - 2 * P.nu));
    double mu0 = P.E / (2 * (1 + P.nu));
    double lam = ool_exp(power) * lambda0;
    double mu = ool_exp(power) * mu0;
    double tr = 0.0;
    double lse[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      lse[i] = ool_log(Sx[i]);
      tr += lse[i];
    }
#pragma unroll
    for (int i = 0; i < D; ++i) ph[i] = ((2.0 * mu * lse[i]) + (lam * tr)) * Sinv[i] * Sx[i];
    // tau = dPsidF Fe^T = U diag(P_hat * S) U^T; F itself is not updated
    usu_packed<D>(U, ph, tau);
    return false;
  }

  if (rewrite) {
    double e[D];
#pragma unroll
    for (int i = 0; i < D; ++i) e[i] = ool_exp(hencky[i]);
    usv<D>(U, e, V, F);
    hencky_tau<D>(P, U, hencky, tau);
  } else {
    double h[D];
#pragma unroll
    for (int i = 0; i < D; ++i) h[i] = ool_log(fabs(S[i]));
    hencky_tau<D>(P, U, h, tau);
  }
  return plastic;
}

}  // namespace mtr
