// object_silo.hpp — ObjectSilo (reference src/objects/object_silo.hpp:8-54):
// outside the surface of revolution r = tanh(y) + 1 above y = cut (3D only).
#ifndef OBJECTSILO_HPP
#define OBJECTSILO_HPP
#include "object_general.hpp"

#ifdef THREEDIM
class ObjectSilo : public ObjectGeneral {
 public:
  T cut;
  ObjectSilo(BC bc_in, T friction_in, std::string name_in = "", T cut_in = -1)
      : ObjectGeneral(bc_in, friction_in, name_in), cut(cut_in) {}
  bool inside(const TV& X) const override {
    if (X(1) < cut) return false;
    const T r = std::tanh(X(1)) + 1;
    return !(X(0) * X(0) + X(2) * X(2) < r * r);
  }
  TV normal(const TV& X) const override {
    TV n;
    const T theta = std::atan2(X(2), X(0));
    const T sech = 1.0 / std::cosh(X(1));
    n(0) = -std::cos(theta);
    n(1) = sech * sech;
    n(2) = -std::sin(theta);
    return n.normalized();
  }
  bool describe(mtr_object& o) const override {
    o = base_descriptor(MTR_OBJ_SILO);
    o.prm[0] = cut;
    return true;
  }
};
#endif
#endif
