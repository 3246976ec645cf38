// object_ramp.hpp — ObjectRamp (reference src/objects/object_ramp.hpp:8-40):
// the ground y < 0.1 tanh(-100 x).
#ifndef OBJECTRAMP_HPP
#define OBJECTRAMP_HPP
#include "object_general.hpp"

class ObjectRamp : public ObjectGeneral {
 public:
  ObjectRamp(BC bc_in, T friction_in, std::string name_in = "") : ObjectGeneral(bc_in, friction_in, name_in) {}
  bool inside(const TV& X) const override { return X(1) < 0.1 * std::tanh(-100 * X(0)); }
  TV normal(const TV& X) const override {
    TV n = TV::Zero();
    const T c = std::cosh(-100 * X(0));
    n(0) = 10.0 / (c * c);
    n(1) = 1;
    return n.normalized();
  }
  bool describe(mtr_object& o) const override {
    o = base_descriptor(MTR_OBJ_RAMP);
    return true;
  }
};
#endif
