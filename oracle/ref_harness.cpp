// ref_harness.cpp — drives the reference's own Simulation class, compiled from
// its unmodified sources (oracle/Makefile), behind the same C API as the C
// restatement (mpm_oracle.c), so tests can run both on one scene.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product links this.
//
// Setup follows what a reference setup file does (examples/collapse.cpp:20-85):
// public fields are assigned, particles are written into sim.particles, plates
// and objects are pushed as unique_ptr.  Simulation::simulate() is called once
// with end_frame = 0 so that its own constant block (simulation.cpp:94-136)
// runs; the step loop of simulate() (simulation.cpp:168-200) is then repeated
// here one advanceStep() at a time so tests can stop after any step.  The build
// force-includes ref_access_prelude.hpp to read the grid and clock.
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>

#include "simulation/simulation.hpp"
#include "objects/object_box.hpp"
#include "objects/object_bump.hpp"
#include "objects/object_curve.hpp"
#include "objects/object_gate.hpp"
#include "objects/object_ground.hpp"
#include "objects/object_ramp.hpp"
#include "objects/object_plate.hpp"
#ifdef THREEDIM
#include "objects/object_silo.hpp"
#endif

#include "../include/matter_gpu.h"

#ifndef MATTER_REF_SPLINEDEG
#define MATTER_REF_SPLINEDEG SPLINEDEG
#endif

// The 6 output functions of save_data.cpp need tinyply, which is absent; the
// harness never saves (save_sim = false), so they are defined empty here.
void Simulation::saveInfo() {}
void Simulation::saveTiming() {}
void Simulation::saveAvgData() {}
void Simulation::saveParticleData(std::string) {}
void Simulation::saveGridData(std::string) {}
void Simulation::computeAvgData(TM&, TM&, T&) {}

// The incline terrain of the 3D Perzyna-MCC workload: a user-defined
// ObjectGeneral subclass, as a setup file would write it (no counterpart in
// the reference).  Surface y = y0 + sum_k h_k exp(-r_k^2 / (2 sigma_k^2)).
class ObjectTerrainGauss : public ObjectGeneral {
 public:
  double prm[24];
  ObjectTerrainGauss(BC bc, T friction, const double* p) : ObjectGeneral(bc, friction, "terrain") {
    std::memcpy(prm, p, sizeof(prm));
  }
  bool inside(const TV& X) const override {
    double ys = prm[0];
    int nb = (int)prm[1];
    for (int b = 0; b < nb && b < 4; ++b) {
      const double* q = prm + 2 + 4 * b;
      double dxx = X(0) - q[0];
      double r2 = dxx * dxx;
#ifdef THREEDIM
      double dz = X(2) - q[1];
      r2 += dz * dz;
#endif
      ys += q[2] * std::exp(-r2 / (2.0 * q[3] * q[3]));
    }
    return X(1) < ys;
  }
  TV normal(const TV& X) const override {
    double gxs = 0.0, gzs = 0.0;
    int nb = (int)prm[1];
    for (int b = 0; b < nb && b < 4; ++b) {
      const double* q = prm + 2 + 4 * b;
      double dxx = X(0) - q[0];
#ifdef THREEDIM
      double dz = X(2) - q[1];
#else
      double dz = 0.0;
#endif
      double r2 = dxx * dxx;
#ifdef THREEDIM
      r2 += dz * dz;
#endif
      double sg2 = q[3] * q[3];
      double h = q[2] * std::exp(-r2 / (2.0 * sg2));
      gxs += -h * dxx / sg2;
      gzs += -h * dz / sg2;
    }
    TV n = TV::Zero();
    n(0) = -gxs;
    n(1) = 1;
#ifdef THREEDIM
    n(2) = -gzs;
#endif
    return n.normalized();
  }
};

struct RefSim {
  Simulation sim;
  mtr_params P;
  bool started = false;
  bool done = false;
};

static const int kDim = DIMENSION;

extern "C" {

int ref_dim(void) { return kDim; }
int ref_deg(void) { return MATTER_REF_SPLINEDEG; }

void* ref_create(const mtr_params* P, int n_threads) {
  if (!P || P->dim != kDim || P->spline_deg != MATTER_REF_SPLINEDEG) return nullptr;
  RefSim* r = new RefSim();
  r->P = *P;
  Simulation& s = r->sim;
  s.initialize(false);
  s.reduce_verbose = true;
  s.n_threads = n_threads > 0 ? n_threads : 1;
  s.end_frame = P->end_frame;
  s.fps = P->fps;
  s.cfl = P->cfl;
  s.cfl_elastic = P->cfl_elastic;
  s.flip_ratio = P->flip_ratio;
  s.rho = P->rho;
  s.gravity_time = P->gravity_time;
  s.gravity_special = P->gravity_special;
  s.change_particle_positions = P->change_particle_positions;
  s.use_mibf = P->use_mibf;
  s.use_musl = P->use_musl;
  s.pbc = P->pbc != 0;
  s.Lx = P->L[0];
  s.Ly = P->L[1];
#ifdef THREEDIM
  s.Lz = P->L[2];
#endif
  for (int a = 0; a < kDim; ++a) {
    s.gravity(a) = P->gravity[a];
    s.grid_reference_point(a) = P->grid_reference_point[a];
  }
  s.dx = P->dx;
  s.particle_mass = P->particle_mass;
  s.particle_volume = P->particle_volume;
  s.elastic_model = static_cast<ElasticModel>(P->elastic_model);
  s.plastic_model = static_cast<PlasticModel>(P->plastic_model);
  s.hardening_law = static_cast<HardeningLaw>(P->hardening_law);
  s.use_pradhana = P->use_pradhana;
  s.use_mises_q = P->use_mises_q;
  s.E = P->E;
  s.nu = P->nu;
  s.stress_tolerance = P->stress_tolerance;
  s.xi = P->xi;
  s.q_max = P->q_max;
  s.q_min = P->q_min;
  s.p_min = P->p_min;
  s.M = P->M;
  s.q_cohesion = P->q_cohesion;
  s.perzyna_exp = P->perzyna_exp;
  s.perzyna_visc = P->perzyna_visc;
  s.beta = P->beta;
  s.p0 = P->p0;
  s.rho_s = P->rho_s;
  s.grain_diameter = P->grain_diameter;
  s.I_ref = P->I_ref;
  s.mu_1 = P->mu_1;
  s.mu_2 = P->mu_2;
  return r;
}

int ref_set_particles(void* h, uint32_t Np, const double* x, const double* v, const double* F, const double* B,
                      const double* sc) {
  RefSim* r = static_cast<RefSim*>(h);
  Simulation& s = r->sim;
  const int d = kDim, dd = d * d;
  s.Np = Np;
  s.particles = Particles(Np);
  for (uint32_t p = 0; p < Np; ++p) {
    for (int a = 0; a < d; ++a) {
      s.particles.x[p](a) = x[(size_t)p * d + a];
      if (v) s.particles.v[p](a) = v[(size_t)p * d + a];
    }
    if (F)
      for (int i = 0; i < dd; ++i) s.particles.F[p].d[i] = F[(size_t)p * dd + i];
    if (B)
      for (int i = 0; i < dd; ++i) s.particles.Bmat[p].d[i] = B[(size_t)p * dd + i];
    if (sc) {
      s.particles.eps_pl_dev[p] = sc[p * 6 + 0];
      s.particles.eps_pl_vol[p] = sc[p * 6 + 1];
      s.particles.eps_pl_vol_pradhana[p] = sc[p * 6 + 2];
      s.particles.delta_gamma[p] = sc[p * 6 + 3];
      s.particles.viscosity[p] = sc[p * 6 + 4];
      s.particles.muI[p] = sc[p * 6 + 5];
    }
  }
  return 0;
}

int ref_set_objects(void* h, const mtr_plate* plates, int np, const mtr_object* objs, int no) {
  RefSim* r = static_cast<RefSim*>(h);
  Simulation& s = r->sim;
  s.plates.clear();
  s.objects.clear();
  for (int i = 0; i < np; ++i) {
    const mtr_plate& q = plates[i];
#ifdef THREEDIM
    auto pl = std::make_unique<ObjectPlate>(q.pos_object, static_cast<PlateType>(q.plate_type), static_cast<BC>(q.bc),
                                            q.friction, q.pos_lower, q.pos_upper, q.v_object_original[0],
                                            q.v_object_original[1], q.v_object_original[2], q.vmin_factor,
                                            q.load_factor);
    pl->vz_object = q.v_object[2];
#else
    auto pl = std::make_unique<ObjectPlate>(q.pos_object, static_cast<PlateType>(q.plate_type), static_cast<BC>(q.bc),
                                            q.friction, q.pos_lower, q.pos_upper, q.v_object_original[0],
                                            q.v_object_original[1], q.vmin_factor, q.load_factor);
#endif
    pl->vx_object = q.v_object[0];
    pl->vy_object = q.v_object[1];
    s.plates.push_back(std::move(pl));
  }
  for (int i = 0; i < no; ++i) {
    const mtr_object& o = objs[i];
    BC bc = static_cast<BC>(o.bc);
    switch (o.kind) {
      case MTR_OBJ_BUMP: s.objects.push_back(std::make_unique<ObjectBump>(bc, o.friction)); break;
      case MTR_OBJ_GROUND: s.objects.push_back(std::make_unique<ObjectGround>(bc, o.friction, "", o.prm[0])); break;
      case MTR_OBJ_RAMP: s.objects.push_back(std::make_unique<ObjectRamp>(bc, o.friction)); break;
      case MTR_OBJ_CURVE: s.objects.push_back(std::make_unique<ObjectCurve>(bc, o.friction)); break;
      case MTR_OBJ_GATE: s.objects.push_back(std::make_unique<ObjectGate>(bc, o.friction, "", o.prm[0])); break;
#ifdef THREEDIM
      case MTR_OBJ_SILO: s.objects.push_back(std::make_unique<ObjectSilo>(bc, o.friction, "", o.prm[0])); break;
#endif
      case MTR_OBJ_BOX_ROTATED: {
        TV c, hx;
        TM R;
        for (int a = 0; a < kDim; ++a) {
          c(a) = o.prm[a];
          hx(a) = o.prm[3 + a];
        }
        for (int i2 = 0; i2 < kDim * kDim; ++i2) R.d[i2] = o.prm[6 + i2];
        s.objects.push_back(std::make_unique<ObjectBoxRotated>(bc, o.friction, c, hx, R));
        break;
      }
      case MTR_OBJ_TERRAIN_GAUSS:
        s.objects.push_back(std::make_unique<ObjectTerrainGauss>(bc, o.friction, o.prm));
        break;
      default: return -1;
    }
  }
  return 0;
}

static void ref_start(RefSim* r) {
  Simulation& s = r->sim;
  unsigned int ef = s.end_frame;
  s.end_frame = 0;  // run only simulate()'s constant block
  s.simulate();
  s.end_frame = ef;
  s.final_time = ef * s.frame_dt;
#if MATTER_REF_SPLINEDEG == 3
  s.apicDinverse = 3.0 / (s.dx * s.dx);  // simulation.cpp:95 for the cubic build
#endif
  r->started = true;
}

// The loop body of Simulation::simulate (simulation.cpp:168-200).
int ref_step(void* h, int nsteps) {
  RefSim* r = static_cast<RefSim*>(h);
  Simulation& s = r->sim;
  if (!r->started) ref_start(r);
  int done = 0;
  for (int it = 0; it < nsteps; ++it) {
    if (r->done || s.exit == 1 || !(s.frame < s.end_frame)) break;
    s.advanceStep();
    if (s.exit == 1) break;
    s.time += s.dt;
    s.current_time_step++;
    if (s.frame_dt * (s.frame + 1) - s.time < 1e-15) s.frame++;
    if (std::abs(s.final_time - s.time) < 1e-15 || s.final_time < s.time) r->done = true;
    done++;
  }
  return done;
}

void ref_get_particles(void* h, double* x, double* v, double* F, double* B, double* sc, double* pic, double* flip) {
  RefSim* r = static_cast<RefSim*>(h);
  Simulation& s = r->sim;
  const int d = kDim, dd = d * d;
  for (uint32_t p = 0; p < s.Np; ++p) {
    for (int a = 0; a < d; ++a) {
      if (x) x[(size_t)p * d + a] = s.particles.x[p](a);
      if (v) v[(size_t)p * d + a] = s.particles.v[p](a);
      if (pic) pic[(size_t)p * d + a] = s.particles.pic[p](a);
      if (flip) flip[(size_t)p * d + a] = s.particles.flip[p](a);
    }
    for (int i = 0; i < dd; ++i) {
      if (F) F[(size_t)p * dd + i] = s.particles.F[p].d[i];
      if (B) B[(size_t)p * dd + i] = s.particles.Bmat[p].d[i];
    }
    if (sc) {
      sc[p * 6 + 0] = s.particles.eps_pl_dev[p];
      sc[p * 6 + 1] = s.particles.eps_pl_vol[p];
      sc[p * 6 + 2] = s.particles.eps_pl_vol_pradhana[p];
      sc[p * 6 + 3] = s.particles.delta_gamma[p];
      sc[p * 6 + 4] = s.particles.viscosity[p];
      sc[p * 6 + 5] = s.particles.muI[p];
    }
  }
}

void ref_get_grid(void* h, uint32_t* dims, double* gx, double* gy, double* gz, double* mass, double* v,
                  double* flip) {
  RefSim* r = static_cast<RefSim*>(h);
  Simulation& s = r->sim;
  const int d = kDim;
  dims[0] = s.Nx;
  dims[1] = s.Ny;
#ifdef THREEDIM
  dims[2] = s.Nz;
#else
  dims[2] = 1;
#endif
  if (gx) std::memcpy(gx, s.grid.x.data(), sizeof(double) * s.Nx);
  if (gy) std::memcpy(gy, s.grid.y.data(), sizeof(double) * s.Ny);
#ifdef THREEDIM
  if (gz) std::memcpy(gz, s.grid.z.data(), sizeof(double) * s.Nz);
#endif
  for (unsigned int l = 0; l < s.grid_nodes; ++l) {
    if (mass) mass[l] = s.grid.mass[l];
    for (int a = 0; a < d; ++a) {
      if (v) v[(size_t)l * d + a] = s.grid.v[l](a);
      if (flip) flip[(size_t)l * d + a] = s.grid.flip[l](a);
    }
  }
}

void ref_get_clock(void* h, double* out) {
  RefSim* r = static_cast<RefSim*>(h);
  Simulation& s = r->sim;
  out[0] = s.time;
  out[1] = s.dt;
  out[2] = s.current_time_step;
  out[3] = s.frame;
  out[4] = r->done;
  out[5] = s.exit;
  out[6] = 0;
  out[7] = 0;
}

void ref_get_plates(void* h, mtr_plate* out, int n) {
  RefSim* r = static_cast<RefSim*>(h);
  Simulation& s = r->sim;
  for (int i = 0; i < n && i < (int)s.plates.size(); ++i) {
    const ObjectPlate& q = *s.plates[i];
    out[i].plate_type = static_cast<int>(q.plate_type);
    out[i].bc = static_cast<int>(q.bc);
    out[i].friction = q.friction;
    out[i].pos_object = q.pos_object;
    out[i].pos_lower = q.pos_lower;
    out[i].pos_upper = q.pos_upper;
    out[i].v_object[0] = q.vx_object;
    out[i].v_object[1] = q.vy_object;
    out[i].v_object_original[0] = q.vx_object_original;
    out[i].v_object_original[1] = q.vy_object_original;
#ifdef THREEDIM
    out[i].v_object[2] = q.vz_object;
    out[i].v_object_original[2] = q.vz_object_original;
#else
    out[i].v_object[2] = 0;
    out[i].v_object_original[2] = 0;
#endif
    out[i].vmin_factor = q.vmin_factor;
    out[i].load_factor = q.load_factor;
  }
}

void ref_destroy(void* h) { delete static_cast<RefSim*>(h); }

}  // extern "C"
