// mtr_boundary.cuh — grid-node boundary conditions: Simulation::boundaryCollision
// (boundary_collision.cpp:5-394) against analytic level-set objects
// (objects/object_*.hpp) and axis-aligned plates (object_plate.hpp:30-103).
//
// The reference dispatches through virtual inside()/normal() per node and
// object; here an object is a small POD descriptor (kind + parameters) and the
// dispatch is a switch, so the whole loop stays in registers.
#pragma once
#include "mtr_device.cuh"

namespace mtr {

template <int D>
__device__ __forceinline__ void normalize(double (&n)[3]) {
  double sq = n[0] * n[0] + n[1] * n[1];
  if constexpr (D == 3) sq += n[2] * n[2];
  double nr = sqrt(sq);
  if (nr > 0) {
#pragma unroll
    for (int a = 0; a < D; ++a) n[a] /= nr;
  }
}

// Trilinear (2D: bilinear) sample of component `comp` of a dense level-set
// lattice field with `stride` floats per sample; lattice points outside read
// `outside`.  The sample is the OpenVDB BoxSampler's: index coordinates
// u = (X - org) / h, weights from u - floor(u), and lerp(a, b, w) = a + w (b - a)
// applied along x, then y, then z, each operation rounded on its own.
template <int D>
__device__ double ls_sample(const DevParams::LevelSet& L, const float* f, int stride, int comp,
                            const double (&X)[3], double outside) {
  int i0[3] = {0, 0, 0};
  double w[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const double u = __dmul_rn(__dsub_rn(X[a], L.org[a]), L.inv_h);
    const double fl = floor(u);
    i0[a] = fl < -2.0 ? -2 : (fl > 2.0e9 ? 2000000000 : (int)fl);
    w[a] = __dsub_rn(u, fl);
  }
  auto at = [&](int i, int j, int k) -> double {
    if (i < 0 || j < 0 || k < 0 || i >= (int)L.n[0] || j >= (int)L.n[1] || k >= (int)L.n[2]) return outside;
    return (double)f[((size_t)((size_t)i * L.n[1] + j) * L.n[2] + k) * stride + comp];
  };
  auto lerp = [](double a, double b, double t) { return __dadd_rn(a, __dmul_rn(t, __dsub_rn(b, a))); };
  const int i = i0[0], j = i0[1], k = i0[2];
  if constexpr (D == 3) {
    const double c00 = lerp(at(i, j, k), at(i + 1, j, k), w[0]);
    const double c10 = lerp(at(i, j + 1, k), at(i + 1, j + 1, k), w[0]);
    const double c01 = lerp(at(i, j, k + 1), at(i + 1, j, k + 1), w[0]);
    const double c11 = lerp(at(i, j + 1, k + 1), at(i + 1, j + 1, k + 1), w[0]);
    return lerp(lerp(c00, c10, w[1]), lerp(c01, c11, w[1]), w[2]);
  } else {
    const double c0 = lerp(at(i, j, 0), at(i + 1, j, 0), w[0]);
    const double c1 = lerp(at(i, j + 1, 0), at(i + 1, j + 1, 0), w[0]);
    return lerp(c0, c1, w[1]);
  }
}

template <int D>
__device__ bool obj_inside(const DevParams& P, const mtr_object& o, const double (&X)[3]) {
  const double x = X[0], y = X[1];
  switch (o.kind) {
    case MTR_OBJ_LEVELSET: {  // object_vdb.hpp:45-57: phi <= 0
      const DevParams::LevelSet& L = P.ls[(int)o.prm[0]];
      return ls_sample<D>(L, L.phi, 1, 0, X, L.background) <= 0.0;
    }
    case MTR_OBJ_BUMP: return y < 0.0475 / cosh(25 * (x - 0.43));  // object_bump.hpp:15-27
    case MTR_OBJ_GROUND: return !(y > o.prm[0]);                  // object_ground.hpp:16-25
    case MTR_OBJ_RAMP: return y < 0.1 * tanh(-100 * x);           // object_ramp.hpp:15-26
    case MTR_OBJ_CURVE: return !(y > x * x);                       // object_curve.hpp:15-25
    case MTR_OBJ_GATE: return y > o.prm[0] + 100 * x * x;          // object_gate.hpp:16-28
    case MTR_OBJ_SILO: {                                           // object_silo.hpp:16-35
      if constexpr (D == 3) {
        const double z = X[2];
        if (y < o.prm[0]) return false;
        const double r = tanh(y) + 1;
        return !(x * x + z * z < r * r);
      }
      return false;
    }
    case MTR_OBJ_BOX_ROTATED: {  // object_box.hpp:18-24 (R^T (X - c), |local| <= half)
      double loc[3];
#pragma unroll
      for (int i = 0; i < D; ++i) {
        double acc = o.prm[6 + i * D] * (X[0] - o.prm[0]);
#pragma unroll
        for (int k = 1; k < D; ++k) acc += o.prm[6 + i * D + k] * (X[k] - o.prm[k]);
        loc[i] = acc;
      }
#pragma unroll
      for (int i = 0; i < D; ++i)
        if (fabs(loc[i]) > o.prm[3 + i]) return false;
      return true;
    }
    case MTR_OBJ_TERRAIN_GAUSS: {
      double ys = o.prm[0];
      const int nb = (int)o.prm[1];
      for (int b = 0; b < nb && b < 4; ++b) {
        const double* q = o.prm + 2 + 4 * b;
        double dxx = x - q[0];
        double r2 = dxx * dxx;
        if constexpr (D == 3) {
          double dz = X[2] - q[1];
          r2 += dz * dz;
        }
        ys += q[2] * exp(-r2 / (2.0 * q[3] * q[3]));
      }
      return y < ys;
    }
  }
  return false;
}

template <int D>
__device__ void obj_normal(const DevParams& P, const mtr_object& o, const double (&X)[3], double (&n)[3]) {
  const double x = X[0], y = X[1];
  n[0] = n[1] = n[2] = 0.0;
  switch (o.kind) {
    case MTR_OBJ_BUMP: {  // object_bump.hpp:29-41
      double arg = 25 * (x - 0.43);
      double b_der = -25 * 0.0475 * tanh(arg) / cosh(arg);
      n[0] = -b_der;
      n[1] = 1;
      normalize<D>(n);
      break;
    }
    case MTR_OBJ_GROUND:  // object_ground.hpp:27-36 (its n(2) is never set; 0 here)
      n[0] = 0;
      n[1] = 1;
      break;
    case MTR_OBJ_RAMP: {  // object_ramp.hpp:28-40
      double tmp = cosh(-100 * x);
      double b_der = 0.1 * (-100) / (tmp * tmp);
      n[0] = -b_der;
      n[1] = 1;
      normalize<D>(n);
      break;
    }
    case MTR_OBJ_CURVE:  // object_curve.hpp:27-37
      n[0] = -2 * x;
      n[1] = 1;
      normalize<D>(n);
      break;
    case MTR_OBJ_GATE: {  // object_gate.hpp:30-41
      double b_der = 2.0 * 100 * x;
      n[0] = b_der;
      n[1] = -1;
      normalize<D>(n);
      break;
    }
    case MTR_OBJ_SILO: {  // object_silo.hpp:37-54
      if constexpr (D == 3) {
        double theta = atan2(X[2], x);
        double sech_y = 1.0 / cosh(y);
        n[0] = -cos(theta);
        n[1] = sech_y * sech_y;
        n[2] = -sin(theta);
        normalize<D>(n);
      }
      break;
    }
    case MTR_OBJ_BOX_ROTATED: {  // object_box.hpp:26-43
      double loc[3];
#pragma unroll
      for (int i = 0; i < D; ++i) {
        double acc = o.prm[6 + i * D] * (X[0] - o.prm[0]);
#pragma unroll
        for (int k = 1; k < D; ++k) acc += o.prm[6 + i * D + k] * (X[k] - o.prm[k]);
        loc[i] = acc;
      }
      int ca = 0;
      double md = 0.0, sgnl = 0.0;
#pragma unroll
      for (int i = 0; i < D; ++i) {
        double dist = fabs(o.prm[3 + i] - fabs(loc[i]));
        if (dist > md) {
          md = dist;
          ca = i;
        }
      }
#pragma unroll
      for (int i = 0; i < D; ++i)
        if (ca == i) sgnl = (loc[i] > 0) ? 1.0 : -1.0;
      // world normal = R * e_ca * sgnl = sgnl * column ca of R
#pragma unroll
      for (int r = 0; r < D; ++r) {
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) acc += o.prm[6 + k * D + r] * ((k == ca) ? sgnl : 0.0);
        n[r] = acc;
      }
      break;
    }
    case MTR_OBJ_TERRAIN_GAUSS: {
      double gxs = 0.0, gzs = 0.0;
      const int nb = (int)o.prm[1];
      for (int b = 0; b < nb && b < 4; ++b) {
        const double* q = o.prm + 2 + 4 * b;
        double dxx = x - q[0], dz = (D == 3) ? X[2] - q[1] : 0.0;
        double r2 = dxx * dxx;
        if constexpr (D == 3) r2 += dz * dz;
        double sg2 = q[3] * q[3];
        double h = q[2] * exp(-r2 / (2.0 * sg2));
        gxs += -h * dxx / sg2;
        gzs += -h * dz / sg2;
      }
      n[0] = -gxs;
      n[1] = 1;
      if constexpr (D == 3) n[2] = -gzs;
      normalize<D>(n);
      break;
    }
    case MTR_OBJ_LEVELSET: {  // object_vdb.hpp:59-78: sampled gradient, normalised (zero stays zero)
      const DevParams::LevelSet& L = P.ls[(int)o.prm[0]];
#pragma unroll
      for (int a = 0; a < D; ++a) n[a] = ls_sample<D>(L, L.grad, 3, a, X, 0.0);
      normalize<D>(n);
      break;
    }
  }
}

template <int D>
__device__ __forceinline__ bool plate_inside(const mtr_plate& o, const double (&X)[3]) {  // object_plate.hpp:30-103
  switch (o.plate_type) {
    case MTR_PLATE_LEFT: return X[1] < o.pos_upper && X[1] > o.pos_lower && (X[0] - o.pos_object) <= 0;
    case MTR_PLATE_RIGHT: return X[1] < o.pos_upper && X[1] > o.pos_lower && (o.pos_object - X[0]) <= 0;
    case MTR_PLATE_BOTTOM: return X[0] < o.pos_upper && X[0] > o.pos_lower && (X[1] - o.pos_object) <= 0;
    case MTR_PLATE_TOP: return X[0] < o.pos_upper && X[0] > o.pos_lower && (o.pos_object - X[1]) <= 0;
    case MTR_PLATE_BACK: return D == 3 && X[2] - o.pos_object <= 0;
    case MTR_PLATE_FRONT: return D == 3 && o.pos_object - X[2] <= 0;
  }
  return false;
}

// Coulomb reduction of the two tangential components against the normal
// speed (boundary_collision.cpp:103-123 and its five 3D siblings).
__device__ __forceinline__ void coulomb3(double friction, double vn, double& a, double& b) {
  double vel_t = sqrt(a * a + b * b);
  double fric_vel_n = friction * fabs(vn);
  if (friction == 0) {
  } else if (vel_t <= fric_vel_n) {
    a = 0;
    b = 0;
  } else {
    a = sgn(a) * (vel_t - fric_vel_n) / sqrt(1 + b * b / (a * a));
    b = sgn(b) * (vel_t - fric_vel_n) / sqrt(1 + a * a / (b * b));
  }
}
// 2D variant (boundary_collision.cpp:286-297)
__device__ __forceinline__ void coulomb2(double friction, double vn, double& a) {
  if (friction == 0) {
  } else if (fabs(a) < friction * fabs(vn)) {
    a = 0;
  } else {
    if (a > 0)
      a -= friction * fabs(vn);
    else
      a += friction * fabs(vn);
  }
}

// Simulation::boundaryCollision for one grid node (boundary_collision.cpp:5-394).
// Returns false on an invalid BC enum (the reference sets exit = 1).
template <int D>
__device__ bool boundary_collision(const DevParams& P, const mtr_plate* plates, double node_friction,
                                   const double (&Xi)[3], double dt, double (&vi)[3]) {
  double vo[3] = {vi[0], vi[1], D == 3 ? vi[2] : 0.0};
  double X[3] = {Xi[0] + dt * vi[0], Xi[1] + dt * vi[1], D == 3 ? Xi[2] + dt * vi[2] : 0.0};
  for (int oi = 0; oi < P.nobjects; ++oi) {  // boundary_collision.cpp:13-79
    const mtr_object& o = P.objects[oi];
    if (!obj_inside<D>(P, o, X)) continue;
    double vr[3] = {vo[0], vo[1], vo[2]};
    if (o.bc == MTR_BC_NOSLIP) {
      vr[0] = vr[1] = vr[2] = 0.0;
    } else if (o.bc == MTR_BC_SLIPFREE) {
      double n[3];
      obj_normal<D>(P, o, X, n);
      double dot = vr[0] * n[0] + vr[1] * n[1];
      if constexpr (D == 3) dot += vr[2] * n[2];
      if (dot < 0) {
        double friction = P.use_mibf ? node_friction : o.friction;
        double vt[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int a = 0; a < D; ++a) vt[a] = vr[a] - dot * n[a];
        if (friction > 0) {
          double sq = vt[0] * vt[0] + vt[1] * vt[1];
          if constexpr (D == 3) sq += vt[2] * vt[2];
          double nt = sqrt(sq);
          if (-dot * friction < nt) {
#pragma unroll
            for (int a = 0; a < D; ++a) vr[a] = vt[a] + (vt[a] / nt) * dot * friction;
          } else {
            vr[0] = vr[1] = vr[2] = 0.0;
          }
        } else {
#pragma unroll
          for (int a = 0; a < D; ++a) vr[a] = vt[a];
        }
      }
    } else if (o.bc == MTR_BC_SLIPSTICK) {
      double n[3];
      obj_normal<D>(P, o, X, n);
      double dot = vr[0] * n[0] + vr[1] * n[1];
      if constexpr (D == 3) dot += vr[2] * n[2];
#pragma unroll
      for (int a = 0; a < D; ++a) vr[a] = vr[a] - dot * n[a];
      if (dot < 0) {
        double friction = P.use_mibf ? node_friction : o.friction;
        if (friction > 0) {
          double sq = vr[0] * vr[0] + vr[1] * vr[1];
          if constexpr (D == 3) sq += vr[2] * vr[2];
          double nt = sqrt(sq);
          if (-dot * friction < nt) {
#pragma unroll
            for (int a = 0; a < D; ++a) vr[a] = vr[a] + (vr[a] / nt) * dot * friction;
          } else {
            vr[0] = vr[1] = vr[2] = 0.0;
          }
        }
      }
    } else {
      return false;
    }
#pragma unroll
    for (int a = 0; a < D; ++a) vi[a] = vo[a] = vr[a];
  }
  for (int pi = 0; pi < P.nplates; ++pi) {  // boundary_collision.cpp:84-261 (3D) / 267-390 (2D)
    const mtr_plate& o = plates[pi];
    if (!plate_inside<D>(o, X)) continue;
    double vx = vo[0] - o.v_object[0];
    double vy = vo[1] - o.v_object[1];
    double vz = D == 3 ? vo[2] - o.v_object[2] : 0.0;
    const int pt = o.plate_type;
    if (o.bc == MTR_BC_NOSLIP) {
      vx = vy = vz = 0;
    } else if (o.bc == MTR_BC_SLIPSTICK || o.bc == MTR_BC_SLIPFREE) {
      const double friction = P.use_mibf ? node_friction : o.friction;
      const bool stick = o.bc == MTR_BC_SLIPSTICK;
      const bool tb = stick ? (pt == MTR_PLATE_TOP || pt == MTR_PLATE_BOTTOM)
                            : ((pt == MTR_PLATE_TOP && vy > 0) || (pt == MTR_PLATE_BOTTOM && vy < 0));
      const bool lr = stick ? (pt == MTR_PLATE_LEFT || pt == MTR_PLATE_RIGHT)
                            : ((pt == MTR_PLATE_LEFT && vx < 0) || (pt == MTR_PLATE_RIGHT && vx > 0));
      const bool fb = stick ? (pt == MTR_PLATE_FRONT || pt == MTR_PLATE_BACK)
                            : ((pt == MTR_PLATE_FRONT && vz > 0) || (pt == MTR_PLATE_BACK && vz < 0));
      if constexpr (D == 3) {
        if (tb) {
          coulomb3(friction, vy, vx, vz);
          vy = 0;
        } else if (lr) {
          coulomb3(friction, vx, vy, vz);
          vx = 0;
        } else if (fb) {
          coulomb3(friction, vz, vx, vy);
          vz = 0;
        }
      } else {
        if (tb) {
          coulomb2(friction, vy, vx);
          vy = 0;
        } else if (lr) {
          coulomb2(friction, vx, vy);
          vx = 0;
        }
      }
    } else {
      return false;
    }
    vi[0] = vx + o.v_object[0];
    vi[1] = vy + o.v_object[1];
    if constexpr (D == 3) vi[2] = vz + o.v_object[2];
#pragma unroll
    for (int a = 0; a < D; ++a) vo[a] = vi[a];
  }
  return true;
}

}  // namespace mtr
