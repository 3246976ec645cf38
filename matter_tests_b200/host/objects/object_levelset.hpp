// object_levelset.hpp — a level-set object on a dense lattice: what the
// reference's ObjectVdb (src/objects/object_vdb.hpp:17-94) samples from an
// OpenVDB grid, held as a dense array so the GPU step can sample it
// (MTR_OBJ_LEVELSET, mtr_set_levelset).  OpenVDB is not used: a .vdb file is
// converted to a dense phi elsewhere, or phi comes from any signed-distance
// source.
//
// inside(X): trilinear (2D: bilinear) sample of phi <= 0; normal(X): the
// sample of the central-difference gradient of phi (or of given normals),
// normalised — the same arithmetic as the device (mtr_boundary.cuh) so host
// diagnostics and the GPU agree.  Lattice points outside read phi = 3 * spacing
// and a zero gradient.
//
// ObjectLevelSet::bake turns any ObjectGeneral (a user subclass whose inside()
// and normal() are host code the GPU cannot call) into a dense level set over a
// box from inside() and normal() alone: a sample next to a lattice edge whose
// ends disagree takes the signed distance, along that edge, to the crossing
// found by bisection (the nearest such crossing over its edges), so the
// interpolated surface passes through the object's surface on every lattice
// edge it cuts; other samples take +-spacing; normals = normal() at the
// samples.
#ifndef OBJECTLEVELSET_HPP
#define OBJECTLEVELSET_HPP

#include <algorithm>
#include <array>
#include <cmath>
#include <memory>
#include <vector>

#include "object_general.hpp"

class ObjectLevelSet : public ObjectGeneral {
 public:
  std::vector<float> phi;      // dims[0] * dims[1] * dims[2], index (i * dims[1] + j) * dims[2] + k
  std::vector<float> normals;  // empty (use the gradient of phi) or 3 per sample
  std::array<unsigned int, 3> dims;
  TV origin;
  T spacing;

  ObjectLevelSet(std::vector<float> phi_in, std::array<unsigned int, 3> dims_in, TV origin_in, T spacing_in,
                 BC bc_in = BC::NoSlip, T friction_in = 0.0, std::string name_in = "")
      : ObjectGeneral(bc_in, friction_in, name_in),
        phi(std::move(phi_in)),
        dims(dims_in),
        origin(origin_in),
        spacing(spacing_in) {
#ifndef THREEDIM
    dims[2] = 1;
#endif
    build_gradient();
  }

  bool inside(const TV& X_in) const override { return sample(phi.data(), 1, 0, X_in, background()) <= 0; }

  TV normal(const TV& X_in) const override {
    TV n;
    const float* g = normals.empty() ? grad.data() : normals.data();
    for (int a = 0; a < DIMENSION; ++a) n(a) = sample(g, 3, a, X_in, 0.0);
    const T nr = n.norm();
    if (nr > 0) return n / nr;
    return TV::Zero();
  }

  const ObjectLevelSet* levelset() const override { return this; }

  mtr_object descriptor(int slot) const {
    mtr_object o = base_descriptor(MTR_OBJ_LEVELSET);
    o.prm[0] = slot;
    return o;
  }

  // A dense level set of `obj` over [lo, hi] at `h` (see the file comment).
  static std::unique_ptr<ObjectLevelSet> bake(const ObjectGeneral& obj, const TV& lo, const TV& hi, T h) {
    std::array<unsigned int, 3> n = {1, 1, 1};
    for (int a = 0; a < DIMENSION; ++a) n[a] = (unsigned int)std::ceil((hi(a) - lo(a)) / h) + 1;
    const size_t total = (size_t)n[0] * n[1] * n[2];
    const size_t step[3] = {(size_t)n[1] * n[2], n[2], 1};
    auto point = [&](size_t l) {
      const unsigned int c[3] = {(unsigned int)(l / step[0]), (unsigned int)((l / n[2]) % n[1]),
                                 (unsigned int)(l % n[2])};
      TV X;
      for (int a = 0; a < DIMENSION; ++a) X(a) = lo(a) + c[a] * h;
      return X;
    };
    std::vector<char> in(total);
    std::vector<float> ph(total), nm(3 * total, 0.0f);
    for (size_t l = 0; l < total; ++l) {
      const TV X = point(l);
      in[l] = obj.inside(X) ? 1 : 0;
      const TV nv = obj.normal(X);
      for (int a = 0; a < DIMENSION; ++a) nm[3 * l + a] = std::isfinite(nv(a)) ? (float)nv(a) : 0.0f;
    }
    for (size_t l = 0; l < total; ++l) {
      const TV X = point(l);
      const unsigned int c[3] = {(unsigned int)(l / step[0]), (unsigned int)((l / n[2]) % n[1]),
                                 (unsigned int)(l % n[2])};
      double dist = h;
      for (int a = 0; a < DIMENSION; ++a)
        for (int dir = -1; dir <= 1; dir += 2) {
          if ((dir < 0 && c[a] == 0) || (dir > 0 && c[a] + 1 >= n[a])) continue;
          const size_t m = dir < 0 ? l - step[a] : l + step[a];
          if (in[m] == in[l]) continue;
          double t0 = 0.0, t1 = 1.0;  // inside(X + t h e_a) equals in[l] at t0, differs at t1
          for (int it = 0; it < 30; ++it) {
            const double tm = 0.5 * (t0 + t1);
            TV Y = X;
            Y(a) += dir * tm * h;
            if ((obj.inside(Y) ? 1 : 0) == in[l])
              t0 = tm;
            else
              t1 = tm;
          }
          dist = std::min(dist, 0.5 * (t0 + t1) * h);
        }
      ph[l] = (float)(in[l] ? -dist : dist);
    }
    auto out = std::make_unique<ObjectLevelSet>(std::move(ph), n, lo, h, obj.bc, obj.friction, obj.name);
    out->normals = std::move(nm);
    return out;
  }

 private:
  std::vector<float> grad;  // central-difference gradient of phi, 3 per sample

  double background() const { return (double)(float)(3.0 * spacing); }

  void build_gradient() {
    const size_t total = (size_t)dims[0] * dims[1] * dims[2];
    grad.assign(3 * total, 0.0f);
    const float bg = (float)(3.0 * spacing);
    const double half_inv_h = 0.5 / spacing;
    const size_t step[3] = {(size_t)dims[1] * dims[2], dims[2], 1};
    for (size_t l = 0; l < total && l < phi.size(); ++l) {
      const unsigned int c[3] = {(unsigned int)(l / step[0]), (unsigned int)((l / dims[2]) % dims[1]),
                                 (unsigned int)(l % dims[2])};
      for (int a = 0; a < DIMENSION; ++a) {
        const float plus = c[a] + 1 < dims[a] ? phi[l + step[a]] : bg;
        const float minus = c[a] >= 1 ? phi[l - step[a]] : bg;
        const float diff = plus - minus;
        grad[3 * l + a] = (float)((double)diff * half_inv_h);
      }
    }
  }

  double at(const float* f, int stride, int comp, int i, int j, int k, double outside) const {
    if (i < 0 || j < 0 || k < 0 || i >= (int)dims[0] || j >= (int)dims[1] || k >= (int)dims[2]) return outside;
    return (double)f[(((size_t)i * dims[1] + j) * dims[2] + k) * stride + comp];
  }

  static double lerp(double a, double b, double t) { return a + t * (b - a); }

  double sample(const float* f, int stride, int comp, const TV& X, double outside) const {
    int i0[3] = {0, 0, 0};
    double w[3] = {0.0, 0.0, 0.0};
    const double inv_h = 1.0 / spacing;
    for (int a = 0; a < DIMENSION; ++a) {
      const double u = (X(a) - origin(a)) * inv_h;
      const double fl = std::floor(u);
      i0[a] = fl < -2.0 ? -2 : (fl > 2.0e9 ? 2000000000 : (int)fl);
      w[a] = u - fl;
    }
    const int i = i0[0], j = i0[1], k = i0[2];
#ifdef THREEDIM
    const double c00 = lerp(at(f, stride, comp, i, j, k, outside), at(f, stride, comp, i + 1, j, k, outside), w[0]);
    const double c10 =
        lerp(at(f, stride, comp, i, j + 1, k, outside), at(f, stride, comp, i + 1, j + 1, k, outside), w[0]);
    const double c01 =
        lerp(at(f, stride, comp, i, j, k + 1, outside), at(f, stride, comp, i + 1, j, k + 1, outside), w[0]);
    const double c11 =
        lerp(at(f, stride, comp, i, j + 1, k + 1, outside), at(f, stride, comp, i + 1, j + 1, k + 1, outside), w[0]);
    return lerp(lerp(c00, c10, w[1]), lerp(c01, c11, w[1]), w[2]);
#else
    (void)k;
    const double c0 = lerp(at(f, stride, comp, i, j, 0, outside), at(f, stride, comp, i + 1, j, 0, outside), w[0]);
    const double c1 =
        lerp(at(f, stride, comp, i, j + 1, 0, outside), at(f, stride, comp, i + 1, j + 1, 0, outside), w[0]);
    return lerp(c0, c1, w[1]);
#endif
  }
};

#endif  // OBJECTLEVELSET_HPP
