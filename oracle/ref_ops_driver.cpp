// ref_ops_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Builds the Tungsten operator tables with the reference project's own
// header-only code (compiled in place from the reference sources by
// oracle/Makefile; nothing is copied):
//   apps/tungsten/include/tungsten/common/tungsten_params.hpp   (derived params)
//   apps/tungsten/include/tungsten/common/tungsten_spectral.hpp (physics_for_mode)
//   apps/tungsten/include/tungsten/common/tungsten_etd_workspace.hpp (n_weight)
//   include/openpfc/kernel/integrator/spectral_exp_coefficients.hpp
//   include/openpfc/kernel/fft/kspace.hpp (k_component, k_laplacian_value)
// The k-loop order restates prepare_operators,
// apps/tungsten/include/tungsten/cpu/tungsten_model.hpp:223-279.
//
// usage: ref_ops n0 n1 n2 dx dt out.bin
// out.bin = 12 derived doubles (tau p2b p3b p4b q20b q21b q30b q31b q40b q2b q3b q4b)
//           then Nc doubles each of filterMF, exp_Ldt, n_weight (x fastest,
//           (n0/2+1) x n1 x n2).  Parameters are the TungstenParams defaults,
//           which equal the regression test's set (test_tungsten.cpp:199-219).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <openpfc/kernel/fft/kspace.hpp>
#include <openpfc/kernel/integrator/spectral_exp_coefficients.hpp>
#include <tungsten/common/tungsten_etd_workspace.hpp>
#include <tungsten/common/tungsten_spectral.hpp>

int main(int argc, char **argv) {
  if (argc != 7) {
    std::fprintf(stderr, "usage: ref_ops n0 n1 n2 dx dt out.bin\n");
    return 2;
  }
  const int n[3] = {std::atoi(argv[1]), std::atoi(argv[2]), std::atoi(argv[3])};
  const double dx = std::atof(argv[4]);
  const double dt = std::atof(argv[5]);
  TungstenParams params;
  const double derived[12] = {params.get_tau(),     params.get_p2_bar(),
                              params.get_p3_bar(),  params.get_p4_bar(),
                              params.get_q20_bar(), params.get_q21_bar(),
                              params.get_q30_bar(), params.get_q31_bar(),
                              params.get_q40_bar(), params.get_q2_bar(),
                              params.get_q3_bar(),  params.get_q4_bar()};
  const double two_pi = 2.0 * 3.14159265358979323846;
  const double f[3] = {two_pi / (dx * n[0]), two_pi / (dx * n[1]),
                       two_pi / (dx * n[2])};
  const auto op = tungsten::spectral::make_operator_params(params);
  const int h = n[0] / 2 + 1;
  const std::size_t nc = static_cast<std::size_t>(h) * n[1] * n[2];
  std::vector<double> klap(nc), opck(nc), fmf(nc);
  std::size_t idx = 0;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < h; ++i) {
        const double ki = pfc::fft::kspace::k_component(i, n[0], f[0]);
        const double kj = pfc::fft::kspace::k_component(j, n[1], f[1]);
        const double kk = pfc::fft::kspace::k_component(k, n[2], f[2]);
        const double kl = pfc::fft::kspace::k_laplacian_value(ki, kj, kk);
        const auto phys = tungsten::spectral::physics_for_mode(kl, op);
        fmf[idx] = phys.filterMF;
        klap[idx] = kl;
        opck[idx] = phys.opCk;
        ++idx;
      }
  tungsten::etd::TungstenEtdWorkspace<> etd;
  etd.ensure(klap, opck, dt, pfc::integrator::SpectralExpOperatorId{.value = 1},
             tungsten::etd::k_tungsten_etd_config_id);
  std::FILE *fp = std::fopen(argv[6], "wb");
  if (!fp) return 3;
  std::fwrite(derived, sizeof(double), 12, fp);
  std::fwrite(fmf.data(), sizeof(double), nc, fp);
  std::fwrite(etd.exp_Ldt().data(), sizeof(double), nc, fp);
  std::fwrite(etd.n_weight().data(), sizeof(double), nc, fp);
  std::fclose(fp);
  return 0;
}
