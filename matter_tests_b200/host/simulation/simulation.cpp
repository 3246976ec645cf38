// simulation.cpp — Simulation on top of the B200 step (include/matter_gpu.h).
//
// simulate() follows the control flow of the reference's Simulation::simulate
// (src/simulation/simulation.cpp:73-213): validation, the derived constants,
// the frame loop with its "End of frame" and end-of-simulation handling,
// frame output when save_sim is set, and the runtime report.  Each frame's
// steps run on the GPU without host round trips (mtr_run_frame); the particle
// vectors are refreshed from the device at every saved frame and at the end.
#include "simulation.hpp"

#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <cstdlib>
#include <cstring>

namespace {

// Symmetric eigen-decomposition by cyclic Jacobi rotations (for host-side
// diagnostics only): A = Q diag(w) Q^T.
void sym_eig(const TM& A_in, TM& Q, TV& w) {
  TM A = A_in;
  Q = TM::Identity();
  const int n = DIMENSION;
  for (int sweep = 0; sweep < 50; ++sweep) {
    T off = 0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += A(p, q) * A(p, q);
    if (off < 1e-300) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        if (A(p, q) == 0) continue;
        const T tau = (A(q, q) - A(p, p)) / (2 * A(p, q));
        const T t = (tau >= 0 ? 1 : -1) / (std::abs(tau) + std::sqrt(1 + tau * tau));
        const T c = 1 / std::sqrt(1 + t * t), s = t * c;
        for (int k = 0; k < n; ++k) {
          const T akp = A(k, p), akq = A(k, q);
          A(k, p) = c * akp - s * akq;
          A(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const T apk = A(p, k), aqk = A(q, k);
          A(p, k) = c * apk - s * aqk;
          A(q, k) = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const T qkp = Q(k, p), qkq = Q(k, q);
          Q(k, p) = c * qkp - s * qkq;
          Q(k, q) = s * qkp + c * qkq;
        }
      }
  }
  for (int i = 0; i < n; ++i) w(i) = A(i, i);
}

// Kirchhoff stress of the Hencky model, tau = 2 mu ln V + lambda tr(ln V) I
// with V^2 = F F^T (the value HenckyPiola(F) F^T has, simulation.hpp:231-238).
TM hencky_tau(const TM& F, T mu, T lambda) {
  TM Q;
  TV w;
  sym_eig(F * F.transpose(), Q, w);
  TV h;
  T tr = 0;
  for (int i = 0; i < DIMENSION; ++i) {
    h(i) = 0.5 * std::log(w(i));
    tr += h(i);
  }
  TM D = TM::Zero();
  for (int i = 0; i < DIMENSION; ++i) D(i, i) = 2 * mu * h(i) + lambda * tr;
  return Q * D * Q.transpose();
}

const char* status_text(uint32_t f) {
  if (f & MTR_STATUS_BAD_BC) return "INVALID BOUNDARY CONDITION!!!";
  if (f & MTR_STATUS_RMA_NOSTEP) return "RMA: FATAL no valid epv value found";
  if (f & MTR_STATUS_RMA_NOCONV) return "FATAL did not exit the Newton loop";
  if (f & MTR_STATUS_NEG_DGAMMA) return "FATAL negative delta_gamma";
  if (f & MTR_STATUS_RESID_DIFF) return "FATAL residual_diff too small in abs value";
  if (f & MTR_STATUS_BAD_MODEL) return "You specified an invalid HARDENING LAW!";
  if (f & MTR_STATUS_STENCIL_OOB) return "a particle left the grid";
  return "device status error";
}

}  // namespace

Simulation::Simulation() {}

Simulation::~Simulation() {
  finish_frame_output();
  if (ctx_) mtr_ctx_destroy(ctx_);
}

void Simulation::initialize(bool save, std::string dir, std::string name) {
  std::cout << "-----------------------------------------------------------------------------------" << std::endl;
  std::cout << "    Matter (explicit MPM) -- B200 step" << std::endl;
  std::cout << "-----------------------------------------------------------------------------------" << std::endl;
  save_sim = save;
  directory = dir;
  sim_name = name;
  if (save_sim) createDirectory();
  is_initialized = true;
}

void Simulation::createDirectory() {
  if (mkdir(directory.c_str(), 0777) == -1)
    std::cerr << "Directory " << directory << " has already been created:  " << strerror(errno) << std::endl;
  else
    std::cout << "Directory " << directory << " was created now" << std::endl;
  if (mkdir((directory + sim_name).c_str(), 0777) == -1)
    std::cerr << "Simulation " << sim_name << " has already been created: " << strerror(errno) << std::endl;
  else
    std::cout << "Simulation " << sim_name << " was created now" << std::endl;
}

void Simulation::derive_constants() {  // simulation.cpp:94-136
  apicDinverse = SPLINEDEG == 3 ? 3.0 / (dx * dx) : 4.0 / (dx * dx);
  lambda = nu * E / ((1.0 + nu) * (1.0 - 2.0 * nu));
  mu = E / (2.0 * (1.0 + nu));
  K = calculateBulkModulus();
  wave_speed = std::sqrt(E / rho);
  dt_max = cfl_elastic * dx / wave_speed;
  frame_dt = 1.0 / fps;
  gravity_final = gravity;
  one_over_dx = 1.0 / dx;
  one_over_dx_square = one_over_dx * one_over_dx;
  if (use_mises_q) {
    q_prefac = std::sqrt(3.0) / std::sqrt(2.0);
    d_prefac = std::sqrt(2.0) / std::sqrt(3.0);
  } else {
    q_prefac = 1.0 / std::sqrt(2.0);
    d_prefac = std::sqrt(2.0);
  }
  e_mu_prefac = 2 * q_prefac * mu;
  f_mu_prefac = 2 * q_prefac / d_prefac * mu;
  rma_prefac = 2 * q_prefac * q_prefac;
  fac_Q = I_ref / (grain_diameter * std::sqrt(rho_s));
}

T Simulation::calculateBulkModulus() { return lambda + 2.0 * mu / dim; }

void Simulation::report_device_error(int rc, const char* where) {
  uint32_t flags = 0, first = 0;
  if (ctx_) mtr_status(ctx_, &flags, &first);
  if (rc == MTR_ERR_DEVICE_STATUS)
    debug(where, ": ", status_text(flags), " (status 0x", std::hex, flags, std::dec, ", particle ", first, ")");
  else
    debug(where, " failed (", rc, "): ", mtr_last_error());
  exit = 1;
}

bool Simulation::prepare_device() {
  if (ctx_) {
    mtr_ctx_destroy(ctx_);
    ctx_ = nullptr;
  }
  if (particles.x.size() < Np || Np == 0) {
    debug("No particles: set Np and sim.particles (or call sampleParticles) before simulate().");
    exit = 1;
    return false;
  }
  mtr_params p;
  std::memset(&p, 0, sizeof(p));
  p.dim = DIMENSION;
  p.spline_deg = SPLINEDEG;
  p.precision = precision;
  p.elastic_model = static_cast<int>(elastic_model);
  p.plastic_model = static_cast<int>(plastic_model);
  p.hardening_law = static_cast<int>(hardening_law);
  p.use_pradhana = use_pradhana;
  p.use_mises_q = use_mises_q;
  p.use_mibf = use_mibf;
  p.use_musl = use_musl;
  p.gravity_special = gravity_special;
  p.pbc = pbc;
  p.L[0] = Lx;
  p.L[1] = Ly;
#ifdef THREEDIM
  p.L[2] = Lz;
#else
  p.L[2] = 1.0;
#endif
  p.end_frame = end_frame;
  p.change_particle_positions = change_particle_positions;
  p.fps = fps;
  p.cfl = cfl;
  p.cfl_elastic = cfl_elastic;
  p.flip_ratio = flip_ratio;
  p.rho = rho;
  p.gravity_time = gravity_time;
  for (int a = 0; a < 3; ++a) {
    p.gravity[a] = a < DIMENSION ? gravity(a) : 0.0;
    p.grid_reference_point[a] = a < DIMENSION ? grid_reference_point(a) : 2e10;
  }
  p.dx = dx;
  p.particle_mass = particle_mass;
  p.particle_volume = particle_volume;
  p.E = E;
  p.nu = nu;
  p.stress_tolerance = stress_tolerance;
  p.xi = xi;
  p.q_max = q_max;
  p.q_min = q_min;
  p.p_min = p_min;
  p.M = M;
  p.q_cohesion = q_cohesion;
  p.perzyna_exp = perzyna_exp;
  p.perzyna_visc = perzyna_visc;
  p.beta = beta;
  p.p0 = p0;
  p.rho_s = rho_s;
  p.grain_diameter = grain_diameter;
  p.I_ref = I_ref;
  p.mu_1 = mu_1;
  p.mu_2 = mu_2;
  int rc = mtr_ctx_create(&p, device, &ctx_);
  if (rc != MTR_OK) {
    report_device_error(rc, "mtr_ctx_create");
    ctx_ = nullptr;
    return false;
  }
  std::vector<double> sc((size_t)Np * MTR_NUM_SCALARS);
  for (unsigned int i = 0; i < Np; ++i) {
    double* s = &sc[(size_t)i * MTR_NUM_SCALARS];
    s[MTR_SCALAR_EPS_PL_DEV] = particles.eps_pl_dev[i];
    s[MTR_SCALAR_EPS_PL_VOL] = particles.eps_pl_vol[i];
    s[MTR_SCALAR_EPS_PL_VOL_PRADHANA] = particles.eps_pl_vol_pradhana[i];
    s[MTR_SCALAR_DELTA_GAMMA] = particles.delta_gamma[i];
    s[MTR_SCALAR_VISCOSITY] = particles.viscosity[i];
    s[MTR_SCALAR_MUI] = particles.muI[i];
  }
  static_assert(sizeof(TV) == sizeof(double) * DIMENSION, "TV must be packed");
  static_assert(sizeof(TM) == sizeof(double) * DIMENSION * DIMENSION, "TM must be packed");
  rc = mtr_upload(ctx_, particles.x[0].data(), particles.v[0].data(), particles.F[0].data(), particles.Bmat[0].data(),
                  sc.data(), Np);
  if (rc != MTR_OK) {
    report_device_error(rc, "mtr_upload");
    return false;
  }
  std::vector<mtr_plate> pl;
  for (const auto& q : plates) {
    mtr_plate m;
    std::memset(&m, 0, sizeof(m));
    m.plate_type = static_cast<int>(q->plate_type);
    m.bc = static_cast<int>(q->bc);
    m.friction = q->friction;
    m.pos_object = q->pos_object;
    m.pos_lower = q->pos_lower;
    m.pos_upper = q->pos_upper;
    m.v_object[0] = q->vx_object;
    m.v_object[1] = q->vy_object;
    m.v_object_original[0] = q->vx_object_original;
    m.v_object_original[1] = q->vy_object_original;
#ifdef THREEDIM
    m.v_object[2] = q->vz_object;
    m.v_object_original[2] = q->vz_object_original;
#endif
    m.vmin_factor = q->vmin_factor;
    m.load_factor = q->load_factor;
    pl.push_back(m);
  }
  std::vector<mtr_object> ob;
  std::vector<std::unique_ptr<ObjectLevelSet>> baked;
  int slot = 0;
  for (const auto& o : objects) {
    mtr_object m;
    const ObjectLevelSet* ls = o->levelset();
    if (!ls && !o->describe(m)) {
      TV lo = bake_min, hi = bake_max;
      if (!(hi - lo).norm()) {  // the initial particle box, grown
        lo = particles.x[0];
        hi = particles.x[0];
        for (unsigned int q = 1; q < Np; ++q)
          for (int a = 0; a < DIMENSION; ++a) {
            lo(a) = std::min(lo(a), particles.x[q](a));
            hi(a) = std::max(hi(a), particles.x[q](a));
          }
        T ext = 0;
        for (int a = 0; a < DIMENSION; ++a) ext = std::max(ext, hi(a) - lo(a));
        for (int a = 0; a < DIMENSION; ++a) {
          lo(a) -= 0.5 * ext + 8 * dx;
          hi(a) += 0.5 * ext + 8 * dx;
        }
      }
      const T h = bake_spacing > 0 ? bake_spacing : 0.5 * dx;
      double samples = 1;
      for (int a = 0; a < DIMENSION; ++a) samples *= std::ceil((hi(a) - lo(a)) / h) + 1;
      if (samples > 4.0e8) {
        debug("Object '", o->name, "': baking it at spacing ", h, " needs ", samples,
              " samples; set bake_spacing or bake_min/bake_max.");
        exit = 1;
        return false;
      }
      if (!reduce_verbose)
        debug("Object '", o->name, "' has no GPU description: baking it into a level set (", samples,
              " samples, spacing ", h, ").");
      baked.push_back(ObjectLevelSet::bake(*o, lo, hi, h));
      ls = baked.back().get();
    }
    if (ls) {
      if (slot >= MTR_MAX_LEVELSETS) {
        debug("At most ", MTR_MAX_LEVELSETS, " level-set objects (baked or given) per simulation.");
        exit = 1;
        return false;
      }
      const uint32_t dims[3] = {ls->dims[0], ls->dims[1], ls->dims[2]};
      double org[3] = {0.0, 0.0, 0.0};
      for (int a = 0; a < DIMENSION; ++a) org[a] = ls->origin(a);
      rc = mtr_set_levelset(ctx_, slot, ls->phi.data(), ls->normals.empty() ? nullptr : ls->normals.data(), dims,
                            org, ls->spacing);
      if (rc != MTR_OK) {
        report_device_error(rc, "mtr_set_levelset");
        return false;
      }
      m = ls->descriptor(slot++);
    }
    ob.push_back(m);
  }
  rc = mtr_set_objects(ctx_, pl.data(), (int)pl.size(), ob.data(), (int)ob.size());
  if (rc != MTR_OK) {
    report_device_error(rc, "mtr_set_objects");
    return false;
  }
  return true;
}

void Simulation::read_clock() {
  mtr_clock ck;
  if (ctx_ && mtr_get_clock(ctx_, &ck) == MTR_OK) {
    time = ck.time;
    dt = ck.dt;
    current_time_step = ck.step;
    frame = ck.frame;
  }
}

void Simulation::download_state() {
  if (!ctx_) return;
  std::vector<double> sc((size_t)Np * MTR_NUM_SCALARS);
  int rc = mtr_download(ctx_, particles.x[0].data(), particles.v[0].data(), particles.F[0].data(),
                        particles.Bmat[0].data(), sc.data());
  if (rc != MTR_OK) {
    report_device_error(rc, "mtr_download");
    return;
  }
  for (unsigned int i = 0; i < Np; ++i) {
    const double* s = &sc[(size_t)i * MTR_NUM_SCALARS];
    particles.eps_pl_dev[i] = s[MTR_SCALAR_EPS_PL_DEV];
    particles.eps_pl_vol[i] = s[MTR_SCALAR_EPS_PL_VOL];
    particles.eps_pl_vol_pradhana[i] = s[MTR_SCALAR_EPS_PL_VOL_PRADHANA];
    particles.delta_gamma[i] = s[MTR_SCALAR_DELTA_GAMMA];
    particles.viscosity[i] = s[MTR_SCALAR_VISCOSITY];
    particles.muI[i] = s[MTR_SCALAR_MUI];
  }
  std::vector<mtr_plate> pl(plates.size());
  if (!pl.empty() && mtr_get_plates(ctx_, pl.data(), (int)pl.size()) == MTR_OK) {
    for (size_t i = 0; i < plates.size(); ++i) {
      plates[i]->pos_object = pl[i].pos_object;
      plates[i]->pos_lower = pl[i].pos_lower;
      plates[i]->pos_upper = pl[i].pos_upper;
      plates[i]->vx_object = pl[i].v_object[0];
      plates[i]->vy_object = pl[i].v_object[1];
#ifdef THREEDIM
      plates[i]->vz_object = pl[i].v_object[2];
#endif
    }
  }
  read_clock();
}

void Simulation::simulate() {
  if (!is_initialized) {
    debug("Simulation not initialized. Call the initialize(...) function in your input file.");
    return;
  }
  if (elastic_model != ElasticModel::Hencky && plastic_model != PlasticModel::NoPlasticity) {
    debug("This plastic model is only compatible with Hencky's elasticity model");
    debug("Please use: elastic_model = Hencky");
    return;
  }
#ifdef THREEDIM
  debug("This is a 3D simulation.");
#else
  debug("This is a 2D simulation.");
#endif
  debug(SPLINEDEG == 3 ? "Using cubic splines." : "Using quadratic splines.");
  if (exit) return;
  derive_constants();
  if (use_mibf) {  // simulation.cpp:138-145
    const T m0 = (plastic_model == PlasticModel::DPMui || plastic_model == PlasticModel::MCCMui) ? mu_1 : M;
    std::fill(particles.muI.begin(), particles.muI.end(), m0);
  }
  debug("Number of particles: ", Np);
  debug("Grid spacing dx:     ", dx);
  debug("Elastic wave speed:  ", wave_speed);
  debug("Maximum dt:          ", dt_max);
  debug("Particle volume:     ", particle_volume);
  debug("Particle mass:       ", particle_mass);
  time = 0;
  frame = 0;
  current_time_step = 0;
  final_time = end_frame * frame_dt;
  if (!prepare_device()) return;
  if (save_sim) {
    saveInfo();
    saveParticleData();
  }
  const auto begin = std::chrono::steady_clock::now();
  while (frame < end_frame) {
    if (!reduce_verbose) {
      std::cout << "Frame: " << frame << " / " << end_frame << std::endl;
      std::cout << "               Name: " << sim_name << std::endl;
      std::cout << "               Step: " << current_time_step << std::endl;
      std::cout << "               Time: " << time << " -> " << (frame + 1) * frame_dt << std::endl;
    }
    int frame_done = 0;
    const int rc = mtr_run_frame(ctx_, &frame_done);
    if (rc != MTR_OK) {
      finish_frame_output();
      report_device_error(rc, "step");
      download_state();
      return;
    }
    mtr_clock ck;
    mtr_get_clock(ctx_, &ck);
    time = ck.time;
    dt = ck.dt;
    current_time_step = ck.step;
    frame = ck.frame;
    if (frame_done) {
      std::cout << "End of frame " << frame << std::endl;
      if (save_sim) {
        if (save_grid) saveGridData();
        save_frame_async();
      }
    }
    if (ck.done) {
      std::cout << "The simulation ended at time = " << time << std::endl;
      if (save_sim) {
        if (save_grid) saveGridData();
        save_frame_async();
      }
      break;
    }
  }
  finish_frame_output();
  const auto end = std::chrono::steady_clock::now();
  runtime_total = std::chrono::duration_cast<std::chrono::milliseconds>(end - begin).count();
  download_state();
  std::cout << "Simulation took " << runtime_total << " milliseconds" << std::endl;
  if (save_sim) saveTiming();
}

void Simulation::advanceStep() {
  if (!ctx_) {
    derive_constants();
    final_time = end_frame * frame_dt;
    if (!prepare_device()) return;
  }
  const int rc = mtr_step(ctx_, 1);
  if (rc != MTR_OK) report_device_error(rc, "advanceStep");
  download_state();
}

void Simulation::phase_unavailable(const char* name) {
  debug("Simulation::", name, " runs fused inside the B200 step; call advanceStep() or simulate().");
  exit = 1;
}

void Simulation::updateDt() { phase_unavailable("updateDt"); }
void Simulation::resizeGrid() { phase_unavailable("resizeGrid"); }
void Simulation::remeshFixed(unsigned int) { phase_unavailable("remeshFixed"); }
void Simulation::remeshFixedInit(unsigned int, unsigned int, unsigned int) { phase_unavailable("remeshFixedInit"); }
void Simulation::remeshFixedCont() { phase_unavailable("remeshFixedCont"); }
void Simulation::P2G() { phase_unavailable("P2G"); }
void Simulation::explicitEulerUpdate() { phase_unavailable("explicitEulerUpdate"); }
void Simulation::G2P() { phase_unavailable("G2P"); }
void Simulation::deformationUpdate() { phase_unavailable("deformationUpdate"); }
void Simulation::MUSL() { phase_unavailable("MUSL"); }
void Simulation::positionUpdate() { phase_unavailable("positionUpdate"); }
void Simulation::PBCAddParticles1D() { phase_unavailable("PBCAddParticles1D"); }
void Simulation::PBCAddParticles(unsigned int) { phase_unavailable("PBCAddParticles"); }
void Simulation::PBCDelParticles() { phase_unavailable("PBCDelParticles"); }
void Simulation::plasticity(unsigned int, unsigned int&, TM&) { phase_unavailable("plasticity"); }
void Simulation::moveObjects() { phase_unavailable("moveObjects"); }
void Simulation::boundaryCollision(int, TV, TV&) { phase_unavailable("boundaryCollision"); }
void Simulation::overwriteGridVelocity(TV, TV&) { phase_unavailable("overwriteGridVelocity"); }
void Simulation::addExternalParticleGravity() {}

// simulation.cpp:292-333, from the FP64 balance the device keeps for the last step
void Simulation::checkMassConservation() {
  if (!ctx_) return;
  double gm = 0, pm = 0;
  if (mtr_balance(ctx_, &gm, nullptr, &pm, nullptr) != MTR_OK) return;
  debug("               Total grid mass = ", gm);
  debug("               Total part mass = ", pm);
  if (std::abs(gm - pm) > 1e-10 * pm) {
    debug("MASS NOT CONSERVED!!!");
    exit = 1;
  }
}

void Simulation::checkMomentumConservation() {
  if (!ctx_) return;
  double gp[3] = {0, 0, 0}, pp[3] = {0, 0, 0};
  if (mtr_balance(ctx_, nullptr, gp, nullptr, pp) != MTR_OK) return;
  T gn = 0, pn = 0, dn = 0;
  for (int a = 0; a < DIMENSION; ++a) {
    gn += gp[a] * gp[a];
    pn += pp[a] * pp[a];
    dn += (gp[a] - pp[a]) * (gp[a] - pp[a]);
  }
  debug("               Total part momentum = ", std::sqrt(pn));
  debug("               Total grid momentum = ", std::sqrt(gn));
  if (std::sqrt(dn) > 1e-10 * std::sqrt(pn)) {
    debug("MOMENTUM NOT CONSERVED!!!");
    exit = 1;
  }
}

TM Simulation::HenckyPiola(TM& Fe) { return hencky_tau(Fe, mu, lambda) * Fe.transpose().inverse(); }

void Simulation::computeAvgData(TM& volavg_cauchy, TM& volavg_kirchh, T& Javg) {  // save_data.cpp:264-292
  volavg_cauchy = TM::Zero();
  volavg_kirchh = TM::Zero();
  T Jsum = 0;
  for (unsigned int p = 0; p < Np; ++p) {
    TM Fe = particles.F[p];
    TM tau = elastic_model == ElasticModel::NeoHookean ? NeoHookeanPiola(Fe) * Fe.transpose()
                                                        : hencky_tau(Fe, mu, lambda);
    const T J = Fe.determinant() * std::exp(particles.eps_pl_vol[p]);
    Jsum += J;
    volavg_cauchy += tau;
    volavg_kirchh += tau * J;
  }
  volavg_cauchy /= Jsum;
  volavg_kirchh /= Jsum;
  Javg = Jsum / Np;
}

void Simulation::saveAvgData() {
  TM c, k;
  T J;
  computeAvgData(c, k, J);
  std::ofstream f1(directory + sim_name + "/avg_cauchy_frame_" + std::to_string(frame) + ".csv");
  std::ofstream f2(directory + sim_name + "/avg_kirchh_frame_" + std::to_string(frame) + ".csv");
  for (int i = 0; i < DIMENSION * DIMENSION; ++i) {
    f1 << c.d[(i % DIMENSION) * DIMENSION + i / DIMENSION] << (i + 1 < DIMENSION * DIMENSION ? "," : "\n");
    f2 << k.d[(i % DIMENSION) * DIMENSION + i / DIMENSION] << (i + 1 < DIMENSION * DIMENSION ? "," : "\n");
  }
  std::ofstream f3(directory + sim_name + "/avg_J_frame_" + std::to_string(frame) + ".csv");
  f3 << J << "\n";
}

// Binary little-endian PLY files with one `vertex` element of FP64
// properties, one row per vertex: the layout the reference writes through
// tinyply (save_data.cpp:7-171), with its property names and order.
namespace {
void write_ply_header(std::ofstream& out, size_t n, const std::vector<std::string>& names) {
  out << "ply\nformat binary_little_endian 1.0\nelement vertex " << n << "\n";
  for (const auto& c : names) out << "property double " << c << "\n";
  out << "end_header\n";
}

void write_ply(const std::string& path, size_t n, const std::vector<std::pair<std::string, const double*>>& cols) {
  std::ofstream out(path, std::ios::binary);
  std::vector<std::string> names;
  for (const auto& c : cols) names.push_back(c.first);
  write_ply_header(out, n, names);
  std::vector<double> row(cols.size());
  for (size_t i = 0; i < n; ++i) {
    for (size_t k = 0; k < cols.size(); ++k) row[k] = cols[k].second[i];
    out.write(reinterpret_cast<const char*>(row.data()), sizeof(double) * row.size());
  }
}

// rows: n rows of names.size() doubles, already in file order
void write_ply_rows(const std::string& path, size_t n, const std::vector<std::string>& names, const double* rows) {
  std::ofstream out(path, std::ios::binary);
  write_ply_header(out, n, names);
  out.write(reinterpret_cast<const char*>(rows), (std::streamsize)(sizeof(double) * n * names.size()));
}
}  // namespace

// Snapshot of the particle file's rows, taken on the GPU behind the frame's
// steps (mtr_frame_begin); a writer thread waits for the copy and writes the
// file while the next frame steps.  At most one file is in flight.
void Simulation::save_frame_async() {
  finish_frame_output();
  const int rc = mtr_frame_begin(ctx_);
  if (rc != MTR_OK) {
    report_device_error(rc, "mtr_frame_begin");
    return;
  }
  const std::string path = directory + sim_name + "/particles_f" + std::to_string(frame) + ".ply";
  const std::string marker = directory + sim_name + "/last_written.txt";
  const unsigned int f = frame;
  mtr_ctx* ctx = ctx_;
  frame_writer_ = std::thread([ctx, path, marker, f]() {
    const double* rows = nullptr;
    uint32_t n = 0;
    int ncols = 0;
    mtr_clock ck;
    if (mtr_frame_wait(ctx, 3600.0, &rows, &n, &ncols, &ck) != MTR_OK) {
      std::cerr << "frame " << f << " not written: " << mtr_last_error() << std::endl;
      return;
    }
    std::vector<const char*> cn(ncols);
    mtr_frame_columns(ctx, cn.data(), ncols);
    write_ply_rows(path, n, std::vector<std::string>(cn.begin(), cn.end()), rows);
    std::ofstream(marker) << f << "\n";
  });
}

void Simulation::finish_frame_output() {
  if (frame_writer_.joinable()) frame_writer_.join();
}

void Simulation::saveParticleData(std::string extra) {
  const size_t n = Np;
  std::vector<double> X[3], V[3], pres(n), dev(n), Je(n);
  for (int a = 0; a < DIMENSION; ++a) {
    X[a].resize(n);
    V[a].resize(n);
  }
  for (size_t p = 0; p < n; ++p) {
    for (int a = 0; a < DIMENSION; ++a) {
      X[a][p] = particles.x[p](a);
      V[a][p] = particles.v[p](a);
    }
    TM Fe = particles.F[p];
    TM tau = elastic_model == ElasticModel::NeoHookean ? NeoHookeanPiola(Fe) * Fe.transpose()
                                                        : hencky_tau(Fe, mu, lambda);
    const T pressure = -tau.trace() / dim;
    const TM tau_dev = tau + pressure * TM::Identity();
    pres[p] = pressure;
    dev[p] = std::sqrt((use_mises_q ? 1.5 : 0.5) * selfDoubleDot(tau_dev));
    Je[p] = Fe.determinant();
  }
  // save_data.cpp:44-164: x, v, p, q, Je, then the plastic fields the model has
  std::vector<std::pair<std::string, const double*>> cols;
  const char* xs[3] = {"x", "y", "z"};
  const char* vs[3] = {"vx", "vy", "vz"};
  for (int a = 0; a < DIMENSION; ++a) cols.push_back({xs[a], X[a].data()});
  for (int a = 0; a < DIMENSION; ++a) cols.push_back({vs[a], V[a].data()});
  cols.push_back({"p", pres.data()});
  cols.push_back({"q", dev.data()});
  cols.push_back({"Je", Je.data()});
  if (plastic_model != PlasticModel::NoPlasticity) {
    cols.push_back({"eps_pl_vol", particles.eps_pl_vol.data()});
    cols.push_back({"eps_pl_dev", particles.eps_pl_dev.data()});
    cols.push_back({"delta_gamma", particles.delta_gamma.data()});
    const bool mui_model = plastic_model == PlasticModel::DPMui || plastic_model == PlasticModel::MCCMui;
    if (((plastic_model == PlasticModel::DPVisc || plastic_model == PlasticModel::MCCVisc) && use_mibf) || mui_model)
      cols.push_back({"muI", particles.muI.data()});
    if (mui_model) cols.push_back({"viscosity", particles.viscosity.data()});
  }
  write_ply(directory + sim_name + "/particles_f" + extra + std::to_string(frame) + ".ply", n, cols);
  std::ofstream(directory + sim_name + "/last_written.txt") << frame << "\n";
}

void Simulation::saveGridData(std::string extra) {
  if (!ctx_) return;
  uint32_t dims[3];
  if (mtr_get_grid(ctx_, dims, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr) != MTR_OK) return;
  const size_t G = (size_t)dims[0] * dims[1] * dims[2];
  grid.x.resize(dims[0]);
  grid.y.resize(dims[1]);
#ifdef THREEDIM
  grid.z.resize(dims[2]);
#endif
  std::vector<double> m(G), v(G * DIMENSION);
  mtr_get_grid(ctx_, dims, grid.x.data(), grid.y.data(),
#ifdef THREEDIM
               grid.z.data(),
#else
               nullptr,
#endif
               m.data(), v.data(), nullptr);
  Nx = dims[0];
  Ny = dims[1];
#ifdef THREEDIM
  Nz = dims[2];
#endif
  grid_nodes = (unsigned int)G;
  std::vector<double> X[3], V[3];
  for (int a = 0; a < DIMENSION; ++a) {
    X[a].resize(G);
    V[a].resize(G);
  }
  for (size_t l = 0; l < G; ++l) {
    const size_t k = l % dims[2], j = (l / dims[2]) % dims[1], i = l / ((size_t)dims[1] * dims[2]);
    X[0][l] = grid.x[i];
    X[1][l] = grid.y[j];
#ifdef THREEDIM
    X[2][l] = grid.z[k];
#else
    (void)k;
#endif
    for (int a = 0; a < DIMENSION; ++a) V[a][l] = v[l * DIMENSION + a];
  }
  std::vector<std::pair<std::string, const double*>> cols;
  const char* xs[3] = {"x", "y", "z"};
  const char* vs[3] = {"vx", "vy", "vz"};
  for (int a = 0; a < DIMENSION; ++a) cols.push_back({xs[a], X[a].data()});
  for (int a = 0; a < DIMENSION; ++a) cols.push_back({vs[a], V[a].data()});
  cols.push_back({"mass", m.data()});
  std::vector<double> fric;
  if (use_mibf) {  // save_data.cpp:247-255
    fric.resize(G);
    if (mtr_get_grid_friction(ctx_, fric.data()) == MTR_OK) cols.push_back({"friction", fric.data()});
  }
  write_ply(directory + sim_name + "/grid_f" + extra + std::to_string(frame) + ".ply", G, cols);
}

void Simulation::saveInfo() {
  std::ofstream f(directory + sim_name + "/info.txt");
  f << "end_frame " << end_frame << "\nfps " << fps << "\ncfl " << cfl << "\ncfl_elastic " << cfl_elastic
    << "\nflip_ratio " << flip_ratio << "\nrho " << rho << "\ndx " << dx << "\nNp " << Np << "\nE " << E << "\nnu "
    << nu << "\nplastic_model " << static_cast<int>(plastic_model) << "\nM " << M << "\nq_cohesion " << q_cohesion
    << "\nuse_musl " << use_musl << "\nuse_mibf " << use_mibf << "\ndim " << dim << "\nsplinedeg " << SPLINEDEG
    << "\n";
}

void Simulation::saveTiming() {
  std::ofstream f(directory + sim_name + "/info_timing.txt");
  f << "total_ms " << runtime_total << "\nsteps " << current_time_step << "\n";
}
