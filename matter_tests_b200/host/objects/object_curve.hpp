// object_curve.hpp — ObjectCurve (reference src/objects/object_curve.hpp:8-37):
// the parabola y <= x^2.
#ifndef OBJECTCURVE_HPP
#define OBJECTCURVE_HPP
#include "object_general.hpp"

class ObjectCurve : public ObjectGeneral {
 public:
  ObjectCurve(BC bc_in = BC::NoSlip, T friction_in = 0.0, std::string name_in = "")
      : ObjectGeneral(bc_in, friction_in, name_in) {}
  bool inside(const TV& X) const override { return !(X(1) > X(0) * X(0)); }
  TV normal(const TV& X) const override {
    TV n = TV::Zero();
    n(0) = -2 * X(0);
    n(1) = 1;
    return n.normalized();
  }
  bool describe(mtr_object& o) const override {
    o = base_descriptor(MTR_OBJ_CURVE);
    return true;
  }
};
#endif
