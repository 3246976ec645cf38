// data_structures.hpp — Particles and Grid with the fields and layout of the
// reference's src/data_structures.hpp:8-66.  The vectors are the host mirror
// of the particle state; Simulation::simulate uploads them to the GPU at the
// start, downloads them at every saved frame and at the end.
#ifndef DATA_STRUCTURES_HPP
#define DATA_STRUCTURES_HPP

#include "tools.hpp"

class Particles {
 public:
  Particles(unsigned int Np = 1) {
    x.assign(Np, TV::Zero());
    v.assign(Np, TV::Zero());
    pic.assign(Np, TV::Zero());
    flip.assign(Np, TV::Zero());
    eps_pl_dev.assign(Np, 0.0);
    eps_pl_vol.assign(Np, 0.0);
    eps_pl_vol_pradhana.assign(Np, 0.0);
    delta_gamma.assign(Np, 0.0);
    viscosity.assign(Np, 0.0);
    muI.assign(Np, 0.0);
    dPsidF.assign(Np, TM::Zero());
    Fe.assign(Np, TM::Identity());
    F.assign(Np, TM::Identity());
    Bmat.assign(Np, TM::Zero());
  }

  std::vector<TV> x;
  std::vector<TV> v;
  std::vector<TV> pic;
  std::vector<TV> flip;

  std::vector<T> eps_pl_dev;
  std::vector<T> eps_pl_vol;
  std::vector<T> eps_pl_vol_pradhana;
  std::vector<T> delta_gamma;
  std::vector<T> viscosity;
  std::vector<T> muI;
  std::vector<TM> dPsidF;
  std::vector<TM> Fe;

  std::vector<TM> F;
  std::vector<TM> Bmat;
};

class Grid {
 public:
  Grid() {}
  std::vector<T> x;
  std::vector<T> y;
#ifdef THREEDIM
  std::vector<T> z;
#endif
  std::vector<TV> v;
  std::vector<TV> flip;
  std::vector<T> mass;
  std::vector<T> friction;
  T xc = 0;
  T yc = 0;
#ifdef THREEDIM
  T zc = 0;
#endif
};

#endif  // DATA_STRUCTURES_HPP
