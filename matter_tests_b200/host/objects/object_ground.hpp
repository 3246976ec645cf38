// object_ground.hpp — ObjectGround (reference src/objects/object_ground.hpp:8-36):
// the half space y <= y_ground with normal +y.
#ifndef OBJECTGROUND_HPP
#define OBJECTGROUND_HPP
#include "object_general.hpp"

class ObjectGround : public ObjectGeneral {
 public:
  T y_ground;
  ObjectGround(BC bc_in = BC::NoSlip, T friction_in = 0.0, std::string name_in = "", T y_ground_in = 0)
      : ObjectGeneral(bc_in, friction_in, name_in), y_ground(y_ground_in) {}
  bool inside(const TV& X) const override { return !(X(1) > y_ground); }
  TV normal(const TV&) const override {
    TV n = TV::Zero();
    n(1) = 1;
    return n;
  }
  bool describe(mtr_object& o) const override {
    o = base_descriptor(MTR_OBJ_GROUND);
    o.prm[0] = y_ground;
    return true;
  }
};
#endif
