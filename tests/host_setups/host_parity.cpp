// A Matter setup file for the host Simulation parity tests: it builds a small
// granular block with plates and objects through the reference-style API,
// writes the initial particles, runs, and writes the final state, so that the
// test can run the same scene through the oracle and compare.
//
//   host_parity steps  N  OUTDIR   -> N calls of advanceStep()
//   host_parity frames N  OUTDIR   -> simulate() with end_frame = N
//   host_parity saved  N  OUTDIR   -> the same with save_sim and save_grid:
//                                     frame files under OUTDIR/run/
//
// OUTDIR/init.bin and OUTDIR/final.bin hold Np, then x, v, F, B (AoS, column-
// major matrices) and the six plastic scalars per particle, as doubles;
// final.bin ends with time and step.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "objects/object_bump.hpp"
#include "objects/object_plate.hpp"
#include "simulation/simulation.hpp"
#include "tools.hpp"
#ifdef THREEDIM
#include "objects/object_box.hpp"
#endif

static void dump(const Simulation& sim, const std::string& path, bool with_clock, double time, double step) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) std::exit(3);
  const double n = sim.Np;
  std::fwrite(&n, sizeof(double), 1, f);
  for (unsigned int p = 0; p < sim.Np; ++p) std::fwrite(sim.particles.x[p].data(), sizeof(double), DIMENSION, f);
  for (unsigned int p = 0; p < sim.Np; ++p) std::fwrite(sim.particles.v[p].data(), sizeof(double), DIMENSION, f);
  for (unsigned int p = 0; p < sim.Np; ++p)
    std::fwrite(sim.particles.F[p].data(), sizeof(double), DIMENSION * DIMENSION, f);
  for (unsigned int p = 0; p < sim.Np; ++p)
    std::fwrite(sim.particles.Bmat[p].data(), sizeof(double), DIMENSION * DIMENSION, f);
  for (unsigned int p = 0; p < sim.Np; ++p) {
    const double s[6] = {sim.particles.eps_pl_dev[p], sim.particles.eps_pl_vol[p],
                         sim.particles.eps_pl_vol_pradhana[p], sim.particles.delta_gamma[p],
                         sim.particles.viscosity[p], sim.particles.muI[p]};
    std::fwrite(s, sizeof(double), 6, f);
  }
  if (with_clock) {
    std::fwrite(&time, sizeof(double), 1, f);
    std::fwrite(&step, sizeof(double), 1, f);
  }
  std::fclose(f);
}

int main(int argc, char** argv) {
  if (argc != 4) return 2;
  const std::string mode = argv[1], out = argv[3];
  const int n = std::atoi(argv[2]);

  Simulation sim;
  if (mode == "saved") {
    sim.initialize(true, out + "/", "run");
    sim.save_grid = true;
  } else {
    sim.initialize(false);
  }
  sim.reduce_verbose = true;
  sim.end_frame = mode == "steps" ? 1000 : n;
  sim.fps = 400;
  sim.cfl = 0.5;
  sim.flip_ratio = -0.95;
  sim.use_musl = true;
  sim.gravity = TV::Zero();
  sim.gravity[0] = 2.0;
  sim.gravity[1] = -9.81;
  sim.elastic_model = ElasticModel::Hencky;
  sim.plastic_model = PlasticModel::DPVisc;
  sim.use_pradhana = true;
  sim.M = std::tan(30.0 * M_PI / 180.0);
  sim.q_cohesion = 50;
  sim.perzyna_exp = 1;
  sim.perzyna_visc = 0.01;
  sim.E = 1e6;
  sim.nu = 0.3;
  sim.rho = 1500;

  // 2 x 2 (x 2) particles per cell on a sheared lattice, 10 x 5 (x 4) cells
  sim.dx = 0.02;
  const int per = 2, nx = 20, ny = 10, nz = DIMENSION == 3 ? 8 : 1;
  sim.particle_volume = std::pow(sim.dx, DIMENSION) / std::pow(per, DIMENSION);
  sim.particle_mass = sim.rho * sim.particle_volume;
  sim.Np = nx * ny * nz;
  sim.particles = Particles(sim.Np);
  const T h = sim.dx / per;
  unsigned int p = 0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k, ++p) {
        const T xi = 0.011 + (i + 0.5) * h, yj = 0.004 + (j + 0.5) * h;
        sim.particles.x[p](0) = xi + 0.1 * yj;
        sim.particles.x[p](1) = yj;
        sim.particles.v[p](0) = 0.4 - 3.0 * yj;
        sim.particles.v[p](1) = -0.2 + 1.5 * xi;
#ifdef THREEDIM
        const T zk = 0.02 + (k + 0.5) * h;
        sim.particles.x[p](2) = zk;
        sim.particles.v[p](2) = 0.5 * xi * yj;
#endif
      }
  sim.grid_reference_point = TV::Zero();

  sim.plates.push_back(std::make_unique<ObjectPlate>(0.0, PlateType::bottom, BC::SlipStick, 0.35));
  sim.plates.push_back(std::make_unique<ObjectPlate>(0.01, PlateType::left, BC::SlipFree, 0.2));
  sim.plates.push_back(std::make_unique<ObjectPlate>(0.3, PlateType::right, BC::NoSlip));
  sim.objects.push_back(std::make_unique<ObjectBump>(BC::SlipFree, 0.3));
#ifdef THREEDIM
  TM R = TM::Identity();
  const T th = 0.3;
  R(0, 0) = std::cos(th);
  R(0, 1) = -std::sin(th);
  R(1, 0) = std::sin(th);
  R(1, 1) = std::cos(th);
  sim.objects.push_back(std::make_unique<ObjectBoxRotated>(BC::SlipStick, 0.25, TV(0.2, 0.16, 0.06),
                                                           TV(0.03, 0.02, 0.2), R));
#endif

  dump(sim, out + "/init.bin", false, 0, 0);
  double time = 0, step = 0;
  if (mode == "steps") {
    for (int s = 0; s < n && !sim.exit; ++s) sim.advanceStep();
  } else {
    sim.simulate();
  }
  if (sim.exit) return 1;
  time = sim.elapsed_time();
  step = sim.elapsed_steps();
  dump(sim, out + "/final.bin", true, time, step);
  return 0;
}
