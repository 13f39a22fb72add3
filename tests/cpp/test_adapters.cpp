// C++ drop-in adapters (include/openpfc_b200/pfc_b200.hpp) used the way the
// reference's tests use pfc::fft::IFFT and the Tungsten model:
//   - FFT known answers (tests/unit/kernel/fft/test_fft.cpp:28-70)
//   - Tungsten golden L2^2 norms at 32^3 (apps/tungsten/tests/test_tungsten.cpp:177-356),
//   - Aluminum golden norms at 32^3 (apps/aluminumNew/aluminumTest.cpp:48-110),
//     initial condition applied to the host field exactly as that test does
//   - plain PFC: mean density conserved, free energy finite
// usage: test_adapters <tests/golden/tungsten_norms_32.json>; exit code 0 on success.
#include <openpfc_b200/pfc_b200.hpp>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

static int failures = 0;
#define EXPECT(cond, ...)                 \
  do {                                    \
    if (!(cond)) {                        \
      std::printf("FAIL: " __VA_ARGS__);  \
      std::printf("\n");                  \
      std::fflush(stdout);                \
      ++failures;                         \
    }                                     \
  } while (0)

static std::vector<double> golden_norms(const char *path) {
  std::ifstream f(path);
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string s = ss.str();
  std::vector<double> v;
  size_t p = s.find("\"norms\"");
  if (p == std::string::npos) return v;
  p = s.find('[', p);
  const size_t e = s.find(']', p);
  std::stringstream list(s.substr(p + 1, e - p - 1));
  std::string tok;
  while (std::getline(list, tok, ',')) v.push_back(std::stod(tok));
  return v;
}

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  {  // FFT known answers
    pfc::b200::B200FFT fft({8, 1, 1});
    std::vector<double> in = {0.000, 0.785, 1.571, 2.356, 3.142, 3.927, 4.712, 5.498};
    std::vector<std::complex<double>> out(fft.size_outbox());
    fft.forward(in, out);
    EXPECT(std::abs(out[0].real() - 21.991) <= 0.01, "8-point DC %f", out[0].real());
    pfc::b200::B200FFT fft2({2, 1, 1});
    std::vector<std::complex<double>> k = {{1.0, 0.0}, {2.0, 0.0}};
    std::vector<double> r(fft2.size_inbox());
    fft2.backward(k, r);
    EXPECT(std::abs(r[0] - 1.5) <= 0.01, "2-point backward %f", r[0]);
    bool threw = false;
    try {
      std::vector<double> bad(7);
      fft.forward(bad, out);
    } catch (const std::invalid_argument &) {
      threw = true;
    }
    EXPECT(threw, "size mismatch must throw std::invalid_argument");
  }
  {  // Tungsten regression norms
    const std::vector<double> expected = golden_norms(argv[1]);
    EXPECT(expected.size() == 11, "golden file");
    const double dx = 1.1107207345395915;
    const int L = 32;
    const double x0 = -0.5 * dx * L;
    pfc::b200::TungstenB200<double> tungsten({L, L, L}, {dx, dx, dx}, {x0, x0, x0});
    tungsten.params.set_n0(-0.10);
    tungsten.params.set_T(3300.0);
    tungsten.params.set_T0(156000.0);
    tungsten.initialize(1.0);
    std::vector<double> &psi = tungsten.get_real_field("psi");
    std::fill(psi.begin(), psi.end(), -0.4);
    const double s = 1.0 / std::sqrt(2.0);
    const double q[6][3] = {{s, s, 0}, {s, 0, s}, {0, s, s}, {s, 0, -s}, {s, -s, 0}, {0, s, -s}};
    size_t idx = 0;
    for (int kk = 0; kk < L; ++kk)
      for (int j = 0; j < L; ++j)
        for (int i = 0; i < L; ++i, ++idx) {
          const double x = x0 + i * dx, y = x0 + j * dx, z = x0 + kk * dx;
          if (x * x + y * y + z * z < 18.0 * 18.0) {
            double u = -0.047;
            for (int qi = 0; qi < 6; ++qi) u += 2.0 * 0.215936 * std::cos(q[qi][0] * x + q[qi][1] * y + q[qi][2] * z);
            psi[idx] = u;
          }
        }
    double n0 = 0;
    for (double v : psi) n0 += v * v;
    EXPECT(std::abs(n0 - expected[0]) <= 0.1, "initial norm %.6f", n0);
    for (int stp = 0; stp < 10; ++stp) {
      tungsten.step(1.0);
      const std::vector<double> &p = tungsten.get_real_field("psi");
      double nrm = 0;
      for (double v : p) nrm += v * v;
      EXPECT(std::abs(nrm - expected[stp + 1]) <= 0.1, "step %d norm %.6f expected %.6f", stp + 1, nrm,
             expected[stp + 1]);
    }
    EXPECT(tungsten.has_real_field("psiMF") && tungsten.has_real_field("default"), "fields");
    bool threw = false;
    try {
      tungsten.get_real_field("nope");
    } catch (const std::out_of_range &) {
      threw = true;
    }
    EXPECT(threw, "unknown field must throw std::out_of_range");
  }
  {  // plain PFC in FP32
    const double d = M_PI / 4;
    pfc::b200::PfcB200<float> pfcm({32, 32, 32}, {d, d, d}, -0.25);
    pfcm.initialize(0.5);
    std::vector<double> &psi = pfcm.get_real_field("psi");
    opfc_ic_noise(psi.data(), psi.size(), -0.285, 0.01, 42);
    double m0 = 0;
    for (double v : psi) m0 += v;
    m0 /= psi.size();
    for (int stp = 0; stp < 5; ++stp) pfcm.step(0.5 * stp);
    EXPECT(std::abs(pfcm.mean_density() - m0) <= 1e-15, "mean density %.17g vs %.17g", pfcm.mean_density(), m0);
    EXPECT(std::isfinite(pfcm.free_energy()), "free energy");
  }
  {  // Aluminum golden norms, written as apps/aluminumNew/aluminumTest.cpp:48-110 is
    pfc::b200::AluminumB200<double> aluminum({32, 32, 32}, {1.0, 1.0, 1.0});
    aluminum.set_n0(-0.0060);
    aluminum.set_alpha(0.20);
    aluminum.set_n_sol(-0.036);
    aluminum.set_n_vap(-1.297);
    aluminum.set_T_const(980);
    aluminum.set_T_min(780);
    aluminum.set_T_max(1280);
    aluminum.set_T0(89285.0);
    aluminum.set_Bx(0.817900686921996);
    aluminum.set_G_grid(0);
    aluminum.set_V_grid(0);
    aluminum.set_x_initial(130);
    aluminum.set_alpha_farTol(0.001);
    aluminum.set_alpha_highOrd(0);
    aluminum.set_lambda(0.22);
    aluminum.set_stabP(0.0);
    aluminum.set_shift_u(1.0);
    aluminum.set_shift_s(0.0);
    aluminum.set_p2_bar(0.8286531831);
    aluminum.set_p3_bar(-0.04204863);
    aluminum.set_p4_bar(0.007533);
    aluminum.set_q20_bar(0.016531729105214);
    aluminum.set_q21_bar(5.467);
    aluminum.set_q30_bar(1.7152418049986);
    aluminum.set_q31_bar(0.45);
    aluminum.set_q40_bar(0.787482);
    aluminum.initialize(1.0e-2);
    std::vector<double> &psi = aluminum.get_real_field("psi");
    std::fill(psi.begin(), psi.end(), -0.0060);
    const int n[3] = {32, 32, 32};
    const double dx1[3] = {1, 1, 1}, o[3] = {0, 0, 0};
    opfc_ic_seed_grid_fcc(psi.data(), n, dx1, o, 1, 2, 2, 8.0, 4.0, 0.4, -0.036, 42);
    const double expected[5] = {1297.08, 1250.21, 1209.28, 1173.19, 1141.09};
    for (int i = 0; i < 5; ++i) {
      std::vector<double> &p = aluminum.get_real_field("psi");
      double norm2 = 0.0;
      for (double x : p) norm2 += x * x;
      EXPECT(std::abs(norm2 - expected[i]) <= 0.1, "aluminum norm %d: %.6f vs %.2f", i, norm2, expected[i]);
      aluminum.step(1.0);
    }
  }
  std::printf(failures ? "FAILED (%d)\n" : "OK\n", failures);
  return failures ? 1 : 0;
}
