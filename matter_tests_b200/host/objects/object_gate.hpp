// object_gate.hpp — ObjectGate (reference src/objects/object_gate.hpp:8-41):
// the region above y = height + 100 x^2, normal pointing down.
#ifndef OBJECTGATE_HPP
#define OBJECTGATE_HPP
#include "object_general.hpp"

class ObjectGate : public ObjectGeneral {
 public:
  T height;
  ObjectGate(BC bc_in, T friction_in, std::string name_in = "", T height_in = 0.016)
      : ObjectGeneral(bc_in, friction_in, name_in), height(height_in) {}
  bool inside(const TV& X) const override { return X(1) > height + 100 * X(0) * X(0); }
  TV normal(const TV& X) const override {
    TV n = TV::Zero();
    n(0) = 200.0 * X(0);
    n(1) = -1;
    return n.normalized();
  }
  bool describe(mtr_object& o) const override {
    o = base_descriptor(MTR_OBJ_GATE);
    o.prm[0] = height;
    return true;
  }
};
#endif
