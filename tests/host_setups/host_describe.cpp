// Prints, one line per object, the device description (mtr_object) that each
// host object class produces, and one line per plate constructor form, for the
// descriptor tests.  Also samples a Poisson-disk block (argv[1] = radius) and
// writes its points to argv[2].
#include <cstdio>
#include <cstdlib>

#include "objects/object_box.hpp"
#include "objects/object_bump.hpp"
#include "objects/object_curve.hpp"
#include "objects/object_gate.hpp"
#include "objects/object_ground.hpp"
#include "objects/object_ramp.hpp"
#include "objects/object_terrain.hpp"
#include "sampling/sampling_particles.hpp"
#include "simulation/simulation.hpp"
#include "tools.hpp"
#ifdef THREEDIM
#include "objects/object_silo.hpp"
#endif

static void show(const ObjectGeneral& o) {
  mtr_object m;
  if (!o.describe(m)) {
    std::printf("none\n");
    return;
  }
  std::printf("%d %d %.17g", m.kind, m.bc, m.friction);
  for (int i = 0; i < 24; ++i) std::printf(" %.17g", m.prm[i]);
  std::printf("\n");
}

int main(int argc, char** argv) {
  show(ObjectBump(BC::SlipFree, 0.1));
  show(ObjectGround(BC::SlipStick, 0.2, "g", -0.25));
  show(ObjectRamp(BC::NoSlip, 0.3));
  show(ObjectCurve(BC::SlipFree, 0.4));
  show(ObjectGate(BC::SlipStick, 0.5, "gate", 0.03));
#ifdef THREEDIM
  show(ObjectSilo(BC::SlipFree, 0.6, "silo", 0.07));
  TM R = TM::Identity();
  R(0, 1) = -0.6;
  R(1, 0) = 0.6;
  R(0, 0) = R(1, 1) = 0.8;
  show(ObjectBoxRotated(BC::NoSlip, 0.7, TV(1, 2, 3), TV(0.1, 0.2, 0.3), R));
#endif
  show(ObjectTerrainGauss(BC::SlipFree, 0.45, -0.5, {{0.1, 0.2, 0.3, 0.4}, {1.1, 1.2, 1.3, 1.4}}));
  if (argc == 3) {
    Simulation sim;
    sim.Lx = 0.3;
    sim.Ly = 0.2;
#ifdef THREEDIM
    sim.Lz = 0.1;
#endif
    sampleParticles(sim, std::atof(argv[1]));
    FILE* f = std::fopen(argv[2], "wb");
    const double meta[3] = {double(sim.Np), sim.dx, sim.particle_volume};
    std::fwrite(meta, sizeof(double), 3, f);
    for (unsigned int p = 0; p < sim.Np; ++p) std::fwrite(sim.particles.x[p].data(), sizeof(double), DIMENSION, f);
    std::fclose(f);
  }
  return 0;
}
