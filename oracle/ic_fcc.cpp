/* ic_fcc.cpp -- TEST INFRASTRUCTURE ONLY (part of the CPU oracle).
 *
 * Restatement of the seeded initial conditions whose seeds come from the
 * standard library's random distributions: the Aluminum app's
 * SeedGridFCC::apply (apps/aluminumNew/SeedGridFCC.hpp) with SeedFCC
 * (apps/aluminumNew/SeedFCC.hpp), and RandomSeeds::apply
 * (include/openpfc/kernel/simulation/initial_conditions/random_seeds.hpp:54-101)
 * with Seed (seed.hpp).  C++ because the seed positions and
 * orientations come from std::uniform_real_distribution<double> over
 * std::mt19937_64, whose mapping is the standard library's (implementation
 * defined); this file uses the same library as the reference build would
 * (libstdc++), so the draws are the same.
 */
#include <array>
#include <cmath>
#include <random>
#include <vector>

namespace {

using vec3 = std::array<double, 3>;
using mat3 = std::array<vec3, 3>;

mat3 mul(const mat3 &A, const mat3 &B) {
  mat3 C{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) C[i][j] += A[i][k] * B[k][j];
  return C;
}

vec3 mul(const mat3 &A, const vec3 &b) {
  vec3 c{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) c[i] += A[i][j] * b[j];
  return c;
}

struct Seed {
  vec3 c;
  std::vector<vec3> q;
  double r, rho, amp;
  bool inside(double x, double y, double z) const {
    const double ex = x - c[0], ey = y - c[1], ez = z - c[2];
    return ex * ex + ey * ey + ez * ez < r * r;
  }
  // rho + sum_q 2 amp cos(q . X) at the absolute position X
  double value(double x, double y, double z) const {
    double u = rho;
    for (const vec3 &v : q) u += 2.0 * amp * std::cos(v[0] * x + v[1] * y + v[2] * z);
    return u;
  }
};

mat3 rotation(const vec3 &ori) {
  const double ca = std::cos(ori[0]), sa = std::sin(ori[0]);
  const double cb = std::cos(ori[1]), sb = std::sin(ori[1]);
  const double cc = std::cos(ori[2]), sc = std::sin(ori[2]);
  const mat3 Ra = {vec3{ca, -sa, 0.0}, vec3{sa, ca, 0.0}, vec3{0.0, 0.0, 1.0}};
  const mat3 Rb = {vec3{cb, 0.0, sb}, vec3{0.0, 1.0, 0.0}, vec3{-sb, 0.0, cb}};
  const mat3 Rc = {vec3{1.0, 0.0, 0.0}, vec3{0.0, cc, -sc}, vec3{0.0, sc, cc}};
  return mul(Ra, mul(Rb, Rc));
}

// Seed (seed.hpp): the six <110>/sqrt(2) wave vectors rotated by yaw pitch roll
Seed make_bcc_seed(const vec3 &loc, const vec3 &ori, double r, double rho, double amp) {
  const mat3 R = rotation(ori);
  const double s = 1.0 / std::sqrt(2.0);
  Seed sd;
  sd.c = loc;
  sd.q = {mul(R, vec3{s, s, 0}), mul(R, vec3{s, 0, s}),  mul(R, vec3{0, s, s}),
          mul(R, vec3{s, 0, -s}), mul(R, vec3{s, -s, 0}), mul(R, vec3{0, s, -s})};
  sd.r = r;
  sd.rho = rho;
  sd.amp = amp;
  return sd;
}

// SeedFCC: the four <111>/sqrt(3) wave vectors rotated by yaw(a) pitch(b) roll(c)
Seed make_seed(const vec3 &loc, const vec3 &ori, double r, double rho, double amp) {
  const double ca = std::cos(ori[0]), sa = std::sin(ori[0]);
  const double cb = std::cos(ori[1]), sb = std::sin(ori[1]);
  const double cc = std::cos(ori[2]), sc = std::sin(ori[2]);
  const mat3 Ra = {vec3{ca, -sa, 0.0}, vec3{sa, ca, 0.0}, vec3{0.0, 0.0, 1.0}};
  const mat3 Rb = {vec3{cb, 0.0, sb}, vec3{0.0, 1.0, 0.0}, vec3{-sb, 0.0, cb}};
  const mat3 Rc = {vec3{1.0, 0.0, 0.0}, vec3{0.0, cc, -sc}, vec3{0.0, sc, cc}};
  const mat3 R = mul(Ra, mul(Rb, Rc));
  const double s = 1.0 / std::sqrt(3.0);
  Seed sd;
  sd.c = loc;
  sd.q = {mul(R, vec3{-s, s, s}), mul(R, vec3{s, -s, s}), mul(R, vec3{s, s, -s}), mul(R, vec3{s, s, s})};
  sd.r = r;
  sd.rho = rho;
  sd.amp = amp;
  return sd;
}

}  // namespace

extern "C" int orc_ic_seed_grid_fcc(double *psi, const int n[3], const double dx[3], const double origin[3], int Nx,
                                    int Ny, int Nz, double X0, double radius, double amplitude, double rho,
                                    double rseed) {
  (void)Nx;  // the reference places one seed column: x = X0 for every (j, k)
  const double Dy = dx[1] * n[1] / Ny, Dz = dx[2] * n[2] / Nz;
  const double Y0 = Dy / 2.0, Z0 = Dz / 2.0;
  std::mt19937_64 re((std::mt19937_64::result_type)rseed);
  std::uniform_real_distribution<double> rt(-0.2 * radius, 0.2 * radius);
  std::uniform_real_distribution<double> rr(0.0, 8.0 * std::atan(1.0));
  std::vector<Seed> seeds;
  for (int j = 0; j < Ny; ++j)
    for (int k = 0; k < Nz; ++k) {
      const double lx = X0 + rt(re);
      const double ly = Y0 + Dy * j + rt(re);
      const double lz = Z0 + Dz * k + rt(re);
      const double o0 = rr(re);
      const double o1 = rr(re);
      const double o2 = rr(re);
      seeds.push_back(make_seed({lx, ly, lz}, {o0, o1, o2}, radius, rho, amplitude));
    }
  size_t idx = 0;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i, ++idx) {
        const double x = origin[0] + i * dx[0], y = origin[1] + j * dx[1], z = origin[2] + k * dx[2];
        for (const Seed &sd : seeds) {
          const double ex = x - sd.c[0], ey = y - sd.c[1], ez = z - sd.c[2];
          if (ex * ex + ey * ey + ez * ez < sd.r * sd.r) {
            double u = sd.rho;
            for (int q = 0; q < 4; ++q) u += 2.0 * sd.amp * std::cos(sd.q[q][0] * x + sd.q[q][1] * y + sd.q[q][2] * z);
            psi[idx] = u;
            break;
          }
        }
      }
  return 0;
}

// RandomSeeds: 150 seeds of radius 20, centres U(-108, -68) x U(-128, 128)^2 and
// angles U(0, 2 pi), drawn in that order seed by seed from mt19937_64(42); the
// first seed containing a cell sets it, every other cell is 0.
extern "C" int orc_ic_random_seeds(double *psi, const int n[3], const double dx[3], const double origin[3],
                                   double density, double amplitude) {
  const double radius = 20.0;
  std::mt19937_64 re(42);
  std::uniform_real_distribution<double> rx(-128.0 + radius, -128.0 + 3 * radius);
  std::uniform_real_distribution<double> ryz(-128.0, 128.0);
  std::uniform_real_distribution<double> ro(0.0, 8.0 * std::atan(1.0));
  std::vector<Seed> seeds;
  for (int i = 0; i < 150; ++i) {
    const double lx = rx(re);
    const double ly = ryz(re);
    const double lz = ryz(re);
    const double o0 = ro(re);
    const double o1 = ro(re);
    const double o2 = ro(re);
    seeds.push_back(make_bcc_seed({lx, ly, lz}, {o0, o1, o2}, radius, density, amplitude));
  }
  size_t idx = 0;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i, ++idx) {
        const double x = origin[0] + i * dx[0], y = origin[1] + j * dx[1], z = origin[2] + k * dx[2];
        double u = 0.0;
        for (const Seed &sd : seeds)
          if (sd.inside(x, y, z)) {
            u = sd.value(x, y, z);
            break;
          }
        psi[idx] = u;
      }
  return 0;
}
