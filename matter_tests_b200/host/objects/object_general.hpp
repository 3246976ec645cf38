// object_general.hpp — the level-set object interface of the reference's
// src/objects/object_general.hpp:8-23 (bc, friction, name; virtual inside and
// normal), plus describe(): the B200 step evaluates objects on the GPU, so an
// object must be able to describe itself as an mtr_object (kind + parameters).
// The built-in objects do; a user subclass that does not override describe()
// is baked by Simulation::simulate into a dense level set (object_levelset.hpp)
// over the box the flow can reach.
#ifndef OBJECTGENERAL_HPP
#define OBJECTGENERAL_HPP

#include <cstring>

#include "../tools.hpp"
#include "matter_gpu.h"

class ObjectLevelSet;

class ObjectGeneral {
 public:
  BC bc;
  T friction;
  std::string name;

  ObjectGeneral(BC bc, T friction, std::string name) : bc(bc), friction(friction), name(name) {}
  virtual ~ObjectGeneral() {}
  virtual bool inside(const TV& X_in) const = 0;
  virtual TV normal(const TV& X_in) const = 0;

  // Fills `out` with this object's GPU descriptor; false if there is none
  // (Simulation then bakes the object into a dense level set).
  virtual bool describe(mtr_object& out) const { return false; }
  // The dense level set of an ObjectLevelSet (objects/object_levelset.hpp).
  virtual const ObjectLevelSet* levelset() const { return nullptr; }

 protected:
  mtr_object base_descriptor(int kind) const {
    mtr_object o;
    std::memset(&o, 0, sizeof(o));
    o.kind = kind;
    o.bc = static_cast<int>(bc);
    o.friction = friction;
    return o;
  }
};

#endif  // OBJECTGENERAL_HPP
