// simulation.hpp — class Simulation with the public surface of the
// reference's src/simulation/simulation.hpp:23-147 (same fields, defaults and
// methods), so setup files written for the reference build unchanged.  The
// step itself runs on a B200 through the C ABI of include/matter_gpu.h:
// simulate() uploads the particles, advances frame by frame on the device,
// downloads at saved frames and at the end.  There is no CPU fallback.
#ifndef SIMULATION_HPP
#define SIMULATION_HPP

#include <sys/stat.h>
#include <sys/types.h>

#include <chrono>
#include <cmath>
#include <memory>
#include <thread>
#include <utility>

#include "../data_structures.hpp"
#include "../objects/object_general.hpp"
#include "../objects/object_levelset.hpp"
#include "../objects/object_plate.hpp"
#include "../timer.hpp"
#include "../tools.hpp"
#include "matter_gpu.h"

class Simulation {
 public:
  Simulation();
  ~Simulation();
  Simulation(const Simulation&) = delete;
  Simulation& operator=(const Simulation&) = delete;

  int exit = 0;

#ifdef THREEDIM
  const unsigned int dim = 3;
#else
  const unsigned int dim = 2;
#endif

  unsigned int n_threads = 1;  // kept for setup files; the step runs on the GPU
  unsigned int end_frame = 1;

  bool is_initialized = false;
  bool save_sim = true;
  bool reduce_verbose = false;
  bool pbc = false;
  bool change_particle_positions = false;
  bool gravity_special = false;
  bool save_grid = false;
  bool use_mibf = false;
  bool use_musl = false;

  TV grid_reference_point = 2e10 * TV::Ones();
  TV gravity = TV::Zero();

  T fps = 1;
  T cfl = 0.5;
  T cfl_elastic = 0.5;
  T flip_ratio = -0.95;
  T rho = 1000;
  T gravity_time = 0;
  T Lx = 1;
  T Ly = 1;
#ifdef THREEDIM
  T Lz = 1;
#endif

  Particles particles;
  unsigned int Np = 0;
  unsigned int num_add_pbc_particles = 0;
  T particle_mass = 0;
  T particle_volume = 0;
  T dx = 0;

  ElasticModel elastic_model = ElasticModel::Hencky;
  PlasticModel plastic_model = PlasticModel::NoPlasticity;
  HardeningLaw hardening_law = HardeningLaw::ExpoImpl;
  bool use_pradhana = true;
  bool use_mises_q = false;
  T E = 1e6;
  T nu = 0.3;
  T stress_tolerance = 1e-5;
  T xi = 0;

  T q_max = 100;
  T q_min = 100;
  T p_min = -1e20;

  T M = 1;
  T q_cohesion = 0;

  T perzyna_exp = 1;
  T perzyna_visc = 0;

  T beta = 0;
  T p0 = 1000;

  T rho_s = 2500;
  T grain_diameter = 1e-3;
  T I_ref = 0.279;
  T mu_1 = std::tan(20.9 * M_PI / 180.0);
  T mu_2 = std::tan(32.8 * M_PI / 180.0);

  std::vector<std::unique_ptr<ObjectPlate>> plates;
  std::vector<std::unique_ptr<ObjectGeneral>> objects;

  // B200 additions: which GPU runs the step, and the arithmetic
  // (MTR_PREC_FP64 is the reference's double precision)
  int device = 0;
  int precision = MTR_PREC_FP64;
  // Objects without a GPU description (user subclasses of ObjectGeneral) are
  // baked into dense level sets (objects/object_levelset.hpp) at this lattice
  // spacing (0: dx / 2) over [bake_min, bake_max] (equal corners: the initial
  // particle box grown on every side by half its largest extent plus 8 dx).
  T bake_spacing = 0;
  TV bake_min = TV::Zero(), bake_max = TV::Zero();
  // simulated time and step count reached (the reference keeps them private)
  T elapsed_time() const { return time; }
  unsigned int elapsed_steps() const { return current_time_step; }

  void initialize(bool save = true, std::string dir = "output/", std::string name = "dummy");
  void simulate();
  void saveInfo();
  void saveTiming();
  void saveAvgData();
  void computeAvgData(TM& volavg_cauchy, TM& volavg_kirchh, T& Javg);
  void saveParticleData(std::string extra = "");
  void saveGridData(std::string extra = "");
  void createDirectory();
  void advanceStep();
  // The phases below are fused into the GPU step; calling one alone reports
  // that and sets exit = 1.  advanceStep() runs them all.
  void updateDt();
  void resizeGrid();
  void remeshFixed(unsigned int extra_nodes);
  void remeshFixedInit(unsigned int sfx, unsigned int sfy, unsigned int sfz);
  void remeshFixedCont();
  void P2G();
  void explicitEulerUpdate();
  void G2P();
  void deformationUpdate();
  void MUSL();
  void positionUpdate();
  void PBCAddParticles1D();
  void PBCAddParticles(unsigned int safety_factor);
  void PBCDelParticles();
  void plasticity(unsigned int p, unsigned int& plastic_count, TM& Fe_trial);
  void moveObjects();
  void boundaryCollision(int index, TV Xi, TV& vi);
  void overwriteGridVelocity(TV Xi, TV& vi);
  void checkMomentumConservation();
  void checkMassConservation();
  void addExternalParticleGravity();
  T calculateBulkModulus();
  TM NeoHookeanPiola(TM& Fe);
  TM HenckyPiola(TM& Fe);

 private:
  unsigned int current_time_step = 0;
  unsigned int frame = 0;
  T time = 0;
  T runtime_p2g = 0;
  T runtime_g2p = 0;
  T runtime_euler = 0;
  T runtime_defgrad = 0;
  T runtime_total = 0;

  std::string sim_name;
  std::string directory;

  TV gravity_final;

  T final_time = 0;
  T frame_dt = 1;
  T dt = 0;
  T dt_max = 5e-3;
  T dt_min = 1e-6;
  T wave_speed = 0;
  T mu = 0;
  T lambda = 0;
  T K = 0;
  T fac_Q = 0;

  T q_prefac = 0, d_prefac = 0, e_mu_prefac = 0, f_mu_prefac = 0, rma_prefac = 0;
  T one_over_dx = 0, one_over_dx_square = 0, apicDinverse = 0;

  Grid grid;
  unsigned int Nx = 0, Ny = 0;
#ifdef THREEDIM
  unsigned int Nz = 0;
#endif
  unsigned int grid_nodes = 0;

  // GPU context of the running simulation
  mtr_ctx* ctx_ = nullptr;
  // writes the particle file of the last snapshot (mtr_frame_begin) while the
  // next frame steps on the GPU
  std::thread frame_writer_;
  void save_frame_async();
  void finish_frame_output();
  bool prepare_device();
  void derive_constants();
  void download_state();
  void read_clock();
  void report_device_error(int rc, const char* where);
  void phase_unavailable(const char* name);
};

// tau-free Piola stresses for host-side diagnostics (simulation.hpp:227-238)
inline TM Simulation::NeoHookeanPiola(TM& Fe) {
  const TM FinvT = Fe.transpose().inverse();
  return mu * (Fe - FinvT) + lambda * std::log(Fe.determinant()) * FinvT;
}

#endif  // SIMULATION_HPP
