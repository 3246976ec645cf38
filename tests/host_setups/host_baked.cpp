// A Matter setup file with a user-defined object: a subclass of ObjectGeneral
// that only implements inside() and normal() (here by delegating to the bump
// of object_bump.hpp), which the GPU step cannot call and so bakes into a
// dense level set.  The same run with the built-in ObjectBump (evaluated
// analytically on the GPU) is the comparison.
//
//   host_baked builtin|user OUTFILE   -> final positions (Np, then x AoS) as doubles
#include <cstdio>
#include <memory>
#include <string>

#include "objects/object_bump.hpp"
#include "simulation/simulation.hpp"
#include "tools.hpp"

class UserBump : public ObjectGeneral {
 public:
  ObjectBump inner;
  UserBump(BC bc, T friction) : ObjectGeneral(bc, friction, "user_bump"), inner(bc, friction) {}
  bool inside(const TV& X) const override { return inner.inside(X); }
  TV normal(const TV& X) const override { return inner.normal(X); }
};

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  const std::string mode = argv[1];
  Simulation sim;
  sim.initialize(false);
  sim.reduce_verbose = true;
  sim.end_frame = 2;
  sim.fps = 100;
  sim.cfl = 0.5;
  sim.flip_ratio = -0.95;
  sim.gravity = TV::Zero();
  sim.gravity[1] = -9.81;
  sim.plastic_model = PlasticModel::DP;
  sim.M = 0.6;
  sim.E = 1e6;
  sim.nu = 0.3;
  sim.rho = 1500;
  sim.dx = 0.01;
  sim.bake_spacing = 0.0025;
  const int per = 2, nx = 30, ny = 10, nz = DIMENSION == 3 ? 6 : 1;
  sim.particle_volume = std::pow(sim.dx, DIMENSION) / std::pow(per, DIMENSION);
  sim.particle_mass = sim.rho * sim.particle_volume;
  sim.Np = nx * ny * nz;
  sim.particles = Particles(sim.Np);
  const T h = sim.dx / per;
  unsigned int p = 0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k, ++p) {
        sim.particles.x[p](0) = 0.36 + (i + 0.5) * h;
        sim.particles.x[p](1) = 0.05 + (j + 0.5) * h;
        sim.particles.v[p](1) = -1.0;
#ifdef THREEDIM
        sim.particles.x[p](2) = (k + 0.5) * h;
#endif
      }
  if (mode == "user")
    sim.objects.push_back(std::make_unique<UserBump>(BC::SlipFree, 0.3));
  else
    sim.objects.push_back(std::make_unique<ObjectBump>(BC::SlipFree, 0.3));
  sim.simulate();
  if (sim.exit) return 1;
  FILE* f = std::fopen(argv[2], "wb");
  if (!f) return 3;
  const double n = sim.Np;
  std::fwrite(&n, sizeof(double), 1, f);
  for (unsigned int q = 0; q < sim.Np; ++q) std::fwrite(sim.particles.x[q].data(), sizeof(double), DIMENSION, f);
  std::fclose(f);
  return 0;
}
