// object_plate.hpp — ObjectPlate (reference src/objects/object_plate.hpp:8-190):
// an axis-aligned, optionally moving plate bounded by [pos_lower, pos_upper]
// along its tangential axis, with the same constructor arguments.  The GPU
// step moves the plate (move(), object_plate.hpp:136-162) on the device;
// Simulation::simulate copies the final position back.
#ifndef OBJECTPLATE_HPP
#define OBJECTPLATE_HPP

#include "../tools.hpp"

class ObjectPlate {
 public:
#ifdef THREEDIM
  ObjectPlate(T pos_object, PlateType plate_type, BC bc = BC::NoSlip, T friction = 0, T pos_lower = -1e15,
              T pos_upper = 1e15, T vx_object = 0.0, T vy_object = 0.0, T vz_object = 0.0, T vmin_factor = 1.0,
              T load_factor = 0.0, std::string name = "")
      : pos_object(pos_object), plate_type(plate_type), bc(bc), friction(friction), pos_upper(pos_upper),
        pos_lower(pos_lower), vx_object(vx_object), vy_object(vy_object), vz_object(vz_object),
        vx_object_original(vx_object), vy_object_original(vy_object), vz_object_original(vz_object),
        vmin_factor(vmin_factor), load_factor(load_factor), name(name) {}
#else
  ObjectPlate(T pos_object, PlateType plate_type, BC bc = BC::NoSlip, T friction = 0, T pos_lower = -1e15,
              T pos_upper = 1e15, T vx_object = 0.0, T vy_object = 0.0, T vmin_factor = 1.0, T load_factor = 0.0,
              std::string name = "")
      : pos_object(pos_object), plate_type(plate_type), bc(bc), friction(friction), pos_upper(pos_upper),
        pos_lower(pos_lower), vx_object(vx_object), vy_object(vy_object), vx_object_original(vx_object),
        vy_object_original(vy_object), vmin_factor(vmin_factor), load_factor(load_factor), name(name) {}
#endif

  bool inside(const TV& X) const {
    switch (plate_type) {
      case PlateType::left: return X(1) < pos_upper && X(1) > pos_lower && (X(0) - pos_object) <= 0;
      case PlateType::right: return X(1) < pos_upper && X(1) > pos_lower && (pos_object - X(0)) <= 0;
      case PlateType::bottom: return X(0) < pos_upper && X(0) > pos_lower && (X(1) - pos_object) <= 0;
      case PlateType::top: return X(0) < pos_upper && X(0) > pos_lower && (pos_object - X(1)) <= 0;
#ifdef THREEDIM
      case PlateType::back: return X(2) - pos_object <= 0;
      case PlateType::front: return pos_object - X(2) <= 0;
#endif
      default: return false;
    }
  }

  void move(T dt, T frame_dt, T time) {
    const T factor = (time < load_factor * frame_dt) ? (1.0 / vmin_factor) : 1.0;
    vx_object = vx_object_original * factor;
    vy_object = vy_object_original * factor;
#ifdef THREEDIM
    vz_object = vz_object_original * factor;
#endif
    if (plate_type == PlateType::left || plate_type == PlateType::right) {
      pos_object += dt * vx_object;
      pos_upper += dt * vy_object;
      pos_lower += dt * vy_object;
    } else if (plate_type == PlateType::bottom || plate_type == PlateType::top) {
      pos_object += dt * vy_object;
      pos_upper += dt * vx_object;
      pos_lower += dt * vx_object;
    }
#ifdef THREEDIM
    else if (plate_type == PlateType::back || plate_type == PlateType::front) {
      pos_object += dt * vz_object;
    }
#endif
  }

  T pos_object;
  PlateType plate_type;
  BC bc;
  T friction;
  T pos_upper;
  T pos_lower;
  T vx_object;
  T vy_object;
#ifdef THREEDIM
  T vz_object;
#endif
  T vx_object_original;
  T vy_object_original;
#ifdef THREEDIM
  T vz_object_original;
#endif
  T vmin_factor;
  T load_factor;
  std::string name;
};

#endif  // OBJECTPLATE_HPP
