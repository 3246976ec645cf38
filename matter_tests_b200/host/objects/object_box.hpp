// object_box.hpp — ObjectBoxRotated (reference src/objects/object_box.hpp:6-43):
// a box with half extents, rotated by R about its center.
#ifndef OBJECTBOXROTATED_HPP
#define OBJECTBOXROTATED_HPP
#include "object_general.hpp"

class ObjectBoxRotated : public ObjectGeneral {
 public:
  TV center;
  TV half_extents;
  TM rotation;
  ObjectBoxRotated(BC bc_in, T friction_in, const TV& center_in, const TV& half_extents_in, const TM& rotation_in,
                   std::string name_in = "")
      : ObjectGeneral(bc_in, friction_in, name_in), center(center_in), half_extents(half_extents_in),
        rotation(rotation_in) {}
  bool inside(const TV& X) const override {
    const TV local = rotation.transpose() * (X - center);
    for (int i = 0; i < local.size(); ++i)
      if (std::abs(local(i)) > half_extents(i)) return false;
    return true;
  }
  TV normal(const TV& X) const override {
    const TV local = rotation.transpose() * (X - center);
    int axis = 0;
    T best = 0.0;
    for (int i = 0; i < local.size(); ++i) {
      const T dist = std::abs(half_extents(i) - std::abs(local(i)));
      if (dist > best) {
        best = dist;
        axis = i;
      }
    }
    TV ln = TV::Zero();
    ln(axis) = local(axis) > 0 ? 1 : -1;
    return rotation * ln;
  }
  bool describe(mtr_object& o) const override {
    o = base_descriptor(MTR_OBJ_BOX_ROTATED);
    for (int a = 0; a < DIMENSION; ++a) {
      o.prm[a] = center(a);
      o.prm[3 + a] = half_extents(a);
    }
    for (int i = 0; i < DIMENSION * DIMENSION; ++i) o.prm[6 + i] = rotation.d[i];
    return true;
  }
};
#endif
