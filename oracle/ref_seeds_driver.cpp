// ref_seeds_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The RandomSeeds initial condition evaluated with the reference project's own
// Seed class (include/openpfc/kernel/simulation/initial_conditions/seed.hpp,
// header-only, compiled in place from the reference sources by oracle/Makefile;
// nothing is copied): rotation, inside test and seed value come from it.  The
// draws and the fill restate RandomSeeds::apply (random_seeds.hpp:54-101), whose
// own header needs the MPI-based Model and cannot be built here: 150 seeds of
// radius 20, x ~ U(-108, -68), y, z ~ U(-128, 128), angles U(0, 2 pi), from
// std::mt19937_64(42); the first seed containing a cell sets it, else 0.
//
// usage: ref_seeds n0 n1 n2 dx dy dz ox oy oz density amplitude out.bin
// out.bin = n0*n1*n2 doubles, x fastest, coordinate origin + i*spacing.
#include <array>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include <openpfc/kernel/simulation/initial_conditions/seed.hpp>

int main(int argc, char **argv) {
  if (argc != 13) {
    std::fprintf(stderr, "usage: ref_seeds n0 n1 n2 dx dy dz ox oy oz density amplitude out.bin\n");
    return 2;
  }
  const int n[3] = {std::atoi(argv[1]), std::atoi(argv[2]), std::atoi(argv[3])};
  const double dx[3] = {std::atof(argv[4]), std::atof(argv[5]), std::atof(argv[6])};
  const double org[3] = {std::atof(argv[7]), std::atof(argv[8]), std::atof(argv[9])};
  const double density = std::atof(argv[10]), amplitude = std::atof(argv[11]);
  using vec3 = std::array<double, 3>;
  const double radius = 20.0;
  std::mt19937_64 re(42);
  std::uniform_real_distribution<double> rx(-128.0 + radius, -128.0 + 3 * radius);
  std::uniform_real_distribution<double> ry(-128.0, 128.0), rz(-128.0, 128.0);
  std::uniform_real_distribution<double> ro(0.0, 8.0 * std::atan(1.0));
  std::vector<pfc::Seed> seeds;
  for (int s = 0; s < 150; ++s) {
    const vec3 loc = {rx(re), ry(re), rz(re)};
    const vec3 ori = {ro(re), ro(re), ro(re)};
    seeds.emplace_back(loc, ori, radius, density, amplitude);
  }
  std::vector<double> psi((size_t)n[0] * n[1] * n[2], 0.0);
  size_t idx = 0;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i, ++idx) {
        const vec3 X = {org[0] + i * dx[0], org[1] + j * dx[1], org[2] + k * dx[2]};
        for (const auto &sd : seeds)
          if (sd.is_inside(X)) {
            psi[idx] = sd.get_value(X);
            break;
          }
      }
  FILE *f = std::fopen(argv[12], "wb");
  if (!f) return 1;
  const bool ok = std::fwrite(psi.data(), sizeof(double), psi.size(), f) == psi.size();
  return (std::fclose(f) == 0 && ok) ? 0 : 1;
}
