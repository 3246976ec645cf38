// object_bump.hpp — ObjectBump (reference src/objects/object_bump.hpp:8-41):
// the ground y < 0.0475 / cosh(25 (x - 0.43)).
#ifndef OBJECTBUMP_HPP
#define OBJECTBUMP_HPP
#include "object_general.hpp"

class ObjectBump : public ObjectGeneral {
 public:
  ObjectBump(BC bc_in, T friction_in, std::string name_in = "") : ObjectGeneral(bc_in, friction_in, name_in) {}
  bool inside(const TV& X) const override { return X(1) < 0.0475 / std::cosh(25 * (X(0) - 0.43)); }
  TV normal(const TV& X) const override {
    TV n = TV::Zero();
    const T arg = 25 * (X(0) - 0.43);
    n(0) = 25 * 0.0475 * std::tanh(arg) / std::cosh(arg);
    n(1) = 1;
    return n.normalized();
  }
  bool describe(mtr_object& o) const override {
    o = base_descriptor(MTR_OBJ_BUMP);
    return true;
  }
};
#endif
