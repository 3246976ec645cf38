// object_terrain.hpp — ObjectTerrainGauss (no counterpart in the reference):
// the ground below y = y0 + sum_k h_k exp(-r_k^2 / (2 sigma_k^2)), a plane
// with up to four Gaussian bumps at (x_k, z_k); r_k is the horizontal
// distance (x only in 2D).  Used by the incline workload.
#ifndef OBJECTTERRAINGAUSS_HPP
#define OBJECTTERRAINGAUSS_HPP
#include "object_general.hpp"

class ObjectTerrainGauss : public ObjectGeneral {
 public:
  struct Bump {
    T x, z, h, sigma;
  };
  T y0;
  std::vector<Bump> bumps;
  ObjectTerrainGauss(BC bc_in, T friction_in, T y0_in, std::vector<Bump> bumps_in, std::string name_in = "")
      : ObjectGeneral(bc_in, friction_in, name_in), y0(y0_in), bumps(std::move(bumps_in)) {
    if (bumps.size() > 4) bumps.resize(4);
  }
  T surface(const TV& X, T* gx, T* gz) const {
    T ys = y0, ax = 0, az = 0;
    for (const Bump& b : bumps) {
      const T dx = X(0) - b.x;
#ifdef THREEDIM
      const T dz = X(2) - b.z;
#else
      const T dz = 0;
#endif
      const T s2 = b.sigma * b.sigma;
      const T hk = b.h * std::exp(-(dx * dx + dz * dz) / (2.0 * s2));
      ys += hk;
      ax += -hk * dx / s2;
      az += -hk * dz / s2;
    }
    if (gx) *gx = ax;
    if (gz) *gz = az;
    return ys;
  }
  bool inside(const TV& X) const override { return X(1) < surface(X, nullptr, nullptr); }
  TV normal(const TV& X) const override {
    T gx, gz;
    surface(X, &gx, &gz);
    TV n = TV::Zero();
    n(0) = -gx;
    n(1) = 1;
#ifdef THREEDIM
    n(2) = -gz;
#endif
    return n.normalized();
  }
  bool describe(mtr_object& o) const override {
    o = base_descriptor(MTR_OBJ_TERRAIN_GAUSS);
    o.prm[0] = y0;
    o.prm[1] = (T)bumps.size();
    for (size_t k = 0; k < bumps.size(); ++k) {
      o.prm[2 + 4 * k] = bumps[k].x;
      o.prm[3 + 4 * k] = bumps[k].z;
      o.prm[4 + 4 * k] = bumps[k].h;
      o.prm[5 + 4 * k] = bumps[k].sigma;
    }
    return true;
  }
};
#endif
