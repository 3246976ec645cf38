// sampling_particles.hpp — sampleParticles with the signature and side effects
// of the reference's src/sampling/sampling_particles.hpp:12-123: Poisson-disk
// samples of radius kRadius in [0,Lx]x[0,Ly](x[0,Lz]), optional cropping
// (3D: 1 cylinder, 2 silo; 2D: 1 quadratic gate), then dx from ppc and the
// sample count, particle_volume, particle_mass, Np and particles.x.
//
// The reference samples with the tph_poisson library, which is not available;
// this is this project's own implementation of Bridson's algorithm ("Fast
// Poisson disk sampling in arbitrary dimensions", SIGGRAPH 2007 sketch):
// background grid of cell r/sqrt(d), active list, `attempts` candidates per
// active point drawn uniformly from the annulus r <= |d| < 2r around it.  Samples differ from the reference's
// point for point, with the same density and minimum spacing.
#ifndef SAMPLING_PARTICLES_HPP
#define SAMPLING_PARTICLES_HPP

#include <random>

#include "../data_structures.hpp"
#include "../tools.hpp"

namespace matter {

template <int D>
std::vector<std::array<T, D>> poisson_disk(T r, const std::array<T, D>& lo, const std::array<T, D>& hi,
                                          uint32_t attempts, uint32_t seed) {
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<T> uni(0.0, 1.0);
  const T cell = r / std::sqrt((T)D);
  std::array<int64_t, D> n;
  int64_t total = 1;
  for (int a = 0; a < D; ++a) {
    n[a] = std::max<int64_t>(1, (int64_t)std::ceil((hi[a] - lo[a]) / cell));
    total *= n[a];
  }
  std::vector<int32_t> grid((size_t)total, -1);
  std::vector<std::array<T, D>> pts;
  std::vector<int32_t> active;
  auto cell_of = [&](const std::array<T, D>& p, std::array<int64_t, D>& c) {
    for (int a = 0; a < D; ++a) c[a] = std::min<int64_t>(n[a] - 1, std::max<int64_t>(0, (int64_t)((p[a] - lo[a]) / cell)));
  };
  auto lin = [&](const std::array<int64_t, D>& c) {
    int64_t l = 0;
    for (int a = 0; a < D; ++a) l = l * n[a] + c[a];
    return l;
  };
  auto far_enough = [&](const std::array<T, D>& p) {
    std::array<int64_t, D> c;
    cell_of(p, c);
    std::array<int64_t, D> k;
    const int span = 2;
    int64_t combos = 1;
    for (int a = 0; a < D; ++a) combos *= 2 * span + 1;
    for (int64_t m = 0; m < combos; ++m) {
      int64_t t = m;
      bool ok = true;
      for (int a = D - 1; a >= 0; --a) {
        k[a] = c[a] + (t % (2 * span + 1)) - span;
        t /= 2 * span + 1;
        if (k[a] < 0 || k[a] >= n[a]) ok = false;
      }
      if (!ok) continue;
      const int32_t q = grid[(size_t)lin(k)];
      if (q < 0) continue;
      T d2 = 0;
      for (int a = 0; a < D; ++a) d2 += (pts[q][a] - p[a]) * (pts[q][a] - p[a]);
      if (d2 < r * r) return false;
    }
    return true;
  };
  auto add = [&](const std::array<T, D>& p) {
    std::array<int64_t, D> c;
    cell_of(p, c);
    grid[(size_t)lin(c)] = (int32_t)pts.size();
    active.push_back((int32_t)pts.size());
    pts.push_back(p);
  };
  std::array<T, D> p0;
  for (int a = 0; a < D; ++a) p0[a] = lo[a] + uni(rng) * (hi[a] - lo[a]);
  add(p0);
  while (!active.empty()) {
    const size_t ai = (size_t)(uni(rng) * active.size()) % active.size();
    const std::array<T, D> base = pts[active[ai]];
    bool found = false;
    for (uint32_t t = 0; t < attempts && !found; ++t) {
      // uniform in the annulus r <= |d| < 2r: rejection from the cube [-2r, 2r]^D
      std::array<T, D> dir;
      T nn = 0;
      do {
        nn = 0;
        for (int a = 0; a < D; ++a) {
          dir[a] = (4 * uni(rng) - 2) * r;
          nn += dir[a] * dir[a];
        }
      } while (nn < r * r || nn >= 4 * r * r);
      std::array<T, D> cand;
      bool in = true;
      for (int a = 0; a < D; ++a) {
        cand[a] = base[a] + dir[a];
        if (cand[a] < lo[a] || cand[a] > hi[a]) in = false;
      }
      if (in && far_enough(cand)) {
        add(cand);
        found = true;
      }
    }
    if (!found) {
      active[ai] = active.back();
      active.pop_back();
    }
  }
  return pts;
}

}  // namespace matter

#ifdef THREEDIM

template <typename S>
void sampleParticles(S& sim, T kRadius, T ppc = 8, unsigned int crop_to_shape = 0, std::uint32_t attempts = 30,
                     std::uint32_t seed = 42) {
  const T Lx = sim.Lx, Ly = sim.Ly, Lz = sim.Lz;
  debug("Sampling particles...");
  auto square = matter::poisson_disk<3>(kRadius, {0, 0, 0}, {Lx, Ly, Lz}, attempts, seed);
  debug("    Number of square samples: ", square.size());
  sim.dx = std::cbrt(ppc / T(square.size()) * Lx * Ly * Lz);
  sim.particle_volume = sim.dx * sim.dx * sim.dx / ppc;
  sim.particle_mass = sim.rho * sim.particle_volume;
  debug("    dx set to ", sim.dx);
  std::vector<std::array<T, 3>> samples;
  if (crop_to_shape == 1) {  // cylinder
    for (const auto& s : square)
      if ((s[0] - Lx / 2.0) * (s[0] - Lx / 2.0) + (s[2] - Lz / 2.0) * (s[2] - Lz / 2.0) < (Lx / 2.0) * (Lx / 2.0))
        samples.push_back(s);
  } else if (crop_to_shape == 2) {  // silo
    for (const auto& s : square) {
      const T x = s[0] - Lx / 2.0, y = s[1], z = s[2] - Lz / 2.0;
      const T rs = std::tanh(y) + 1;
      if (x * x + z * z < rs * rs) samples.push_back(s);
    }
  } else {
    samples = square;
  }
  sim.Np = samples.size();
  debug("    Number of particles samples: ", sim.Np);
  sim.particles = Particles(sim.Np);
  for (unsigned int p = 0; p < sim.Np; ++p)
    for (int d = 0; d < 3; ++d) sim.particles.x[p](d) = samples[p][d];
}

#else

template <typename S>
void sampleParticles(S& sim, T kRadius, T ppc = 6, unsigned int crop_to_shape = 0, std::uint32_t attempts = 200,
                     std::uint32_t seed = 42) {
  (void)attempts;
  (void)seed;  // the 2D variant of the reference fixes 200 attempts and seed 42
  const T Lx = sim.Lx, Ly = sim.Ly;
  debug("Sampling particles...");
  auto square = matter::poisson_disk<2>(kRadius, {0, 0}, {Lx, Ly}, 200, 42);
  debug("    Number of square samples: ", square.size());
  sim.dx = std::sqrt(ppc / T(square.size()) * Lx * Ly);
  sim.particle_volume = sim.dx * sim.dx / ppc;
  sim.particle_mass = sim.rho * sim.particle_volume;
  debug("    dx set to ", sim.dx);
  std::vector<std::array<T, 2>> samples;
  if (crop_to_shape == 1) {  // quadratic gate
    const T height = 0.05;
    for (const auto& s : square) {
      const T y_gate = height + 100 * (s[0] - Lx) * (s[0] - Lx) - 0.5 * sim.dx;
      if (s[1] < y_gate) samples.push_back(s);
    }
  } else {
    samples = square;
  }
  sim.Np = samples.size();
  debug("    Number of particles samples: ", sim.Np);
  sim.particles = Particles(sim.Np);
  for (unsigned int p = 0; p < sim.Np; ++p)
    for (int d = 0; d < 2; ++d) sim.particles.x[p](d) = samples[p][d];
}

#endif

#endif  // SAMPLING_PARTICLES_HPP
