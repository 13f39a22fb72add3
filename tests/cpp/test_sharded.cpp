// The C++ sharded field (include/openpfc_b200/sharded.hpp) against one
// unsharded handle of the same grid, through the C ABI: P ranks emulated in
// one process (LocalShardComm) on one GPU.  Plain model 10 steps and filtered
// model 6 steps, FP64 (rel-L2 <= 1e-11) and FP32 (rel-L2 <= 1e-5 against the
// FP64 handle); the sharded transform (ShardedFft) against one handle's
// opfc_fft_forward and its round trip (FP64, 1e-12); P = 1, 2, 4.  The grid must divide: P = 3 on N2 = 32 is refused
// with std::invalid_argument.  Exit status 0 when every check passes.
#include <openpfc_b200/sharded.hpp>

#include <cmath>
#include <complex>
#include <cstdio>
#include <utility>
#include <vector>

using pfc::b200::LocalShardComm;
using pfc::b200::ShardedParams;
using pfc::b200::ShardedPfc;

namespace {

const int kN[3] = {32, 16, 32};
const double kPi = 3.14159265358979323846;
int failures = 0;

// psi0 = n0 + a deterministic perturbation of amplitude ~0.01 (x fastest)
std::vector<double> initial_field() {
  std::vector<double> f(size_t(kN[0]) * kN[1] * kN[2]);
  for (int z = 0; z < kN[2]; ++z)
    for (int y = 0; y < kN[1]; ++y)
      for (int x = 0; x < kN[0]; ++x) {
        const double h = std::sin(12.9898 * x + 78.233 * y + 37.719 * z) * 43758.5453;
        f[x + size_t(kN[0]) * (y + size_t(kN[1]) * z)] = -0.285 + 0.02 * (h - std::floor(h) - 0.5);
      }
  return f;
}

std::vector<double> unsharded(const std::vector<double> &psi0, const ShardedParams &p, int steps) {
  opfc_desc d;
  opfc_desc_default(&d);
  for (int a = 0; a < 3; ++a) {
    d.n[a] = kN[a];
    d.dx[a] = kPi / 4;
  }
  d.precision = OPFC_FP64;
  d.model = p.model;
  d.r = p.r;
  d.filter_alpha = p.alpha;
  d.p2 = p.p2;
  d.p3 = p.p3;
  d.p4 = p.p4;
  opfc_handle *h = nullptr;
  pfc::b200::check(opfc_create(&d, &h), "opfc_create");
  pfc::b200::check(opfc_initialize(h, 0.5), "opfc_initialize");
  pfc::b200::check(opfc_set_psi(h, psi0.data(), psi0.size(), OPFC_F64, OPFC_HOST), "opfc_set_psi");
  pfc::b200::check(opfc_step(h, steps), "opfc_step");
  std::vector<double> out(psi0.size());
  pfc::b200::check(opfc_get_psi(h, out.data(), out.size(), OPFC_F64, OPFC_HOST), "opfc_get_psi");
  opfc_destroy(h);
  return out;
}

template <typename T>
std::vector<double> sharded(const std::vector<double> &psi0, const ShardedParams &p, int steps, int P) {
  LocalShardComm comm(P);
  ShardedPfc<T> m({kN[0], kN[1], kN[2]}, {kPi / 4, kPi / 4, kPi / 4}, comm, p);
  m.initialize(0.5);
  const size_t slab = psi0.size() / P;
  std::vector<const double *> in;
  for (int q = 0; q < P; ++q) in.push_back(psi0.data() + q * slab);
  m.set_psi(in);
  m.step(steps);
  m.sync();
  std::vector<double> out(psi0.size());
  std::vector<double *> outs;
  for (int q = 0; q < P; ++q) outs.push_back(out.data() + q * slab);
  m.get_psi(outs);
  return out;
}

double rel_l2_fwd(const std::vector<double> &a, const std::vector<double> &b) {
  double num = 0, den = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    num += (a[i] - b[i]) * (a[i] - b[i]);
    den += b[i] * b[i];
  }
  return std::sqrt(num / den);
}

// Sharded forward transform against one handle's (reference layout, kx
// fastest over M + 1 columns); returns the larger relative L2 error of the
// forward transform and of backward(forward(psi0)) against psi0.
std::pair<double, double> fft_errors(const std::vector<double> &psi0, int P) {
  const int M = kN[0] / 2;
  const size_t lines = size_t(kN[1]) * kN[2];
  opfc_desc d;
  opfc_desc_default(&d);
  for (int a = 0; a < 3; ++a) d.n[a] = kN[a];
  d.precision = OPFC_FP64;
  opfc_handle *h = nullptr;
  pfc::b200::check(opfc_create(&d, &h), "opfc_create");
  std::vector<std::complex<double>> ref(size_t(M + 1) * lines);
  pfc::b200::check(opfc_fft_forward(h, psi0.data(), ref.data(), OPFC_F64, OPFC_HOST), "opfc_fft_forward");
  opfc_destroy(h);

  LocalShardComm comm(P);
  pfc::b200::ShardedFft<double> f({kN[0], kN[1], kN[2]}, comm);
  const size_t slab = psi0.size() / P;
  std::vector<const double *> in;
  std::vector<std::vector<std::complex<double>>> spec(P);
  std::vector<std::complex<double> *> outs;
  std::vector<const std::complex<double> *> cins;
  for (int q = 0; q < P; ++q) {
    in.push_back(psi0.data() + q * slab);
    spec[q].resize(lines * f.columns(q));
    outs.push_back(spec[q].data());
    cins.push_back(spec[q].data());
  }
  f.forward(in, outs);
  double num = 0, den = 0;
  const int mloc = M / P;
  for (int q = 0; q < P; ++q)
    for (size_t l = 0; l < lines; ++l)
      for (int k = 0; k < f.columns(q); ++k) {
        const std::complex<double> a = spec[q][l * f.columns(q) + k], b = ref[l * (M + 1) + q * mloc + k];
        num += std::norm(a - b);
        den += std::norm(b);
      }
  std::vector<double> back(psi0.size());
  std::vector<double *> bouts;
  for (int q = 0; q < P; ++q) bouts.push_back(back.data() + q * slab);
  f.backward(cins, bouts);
  return {std::sqrt(num / den), rel_l2_fwd(back, psi0)};
}

double rel_l2(const std::vector<double> &a, const std::vector<double> &b) {
  double num = 0, den = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    num += (a[i] - b[i]) * (a[i] - b[i]);
    den += b[i] * b[i];
  }
  return std::sqrt(num / den);
}

void expect(bool ok, const char *what, double v) {
  std::printf("%-52s %.3e %s\n", what, v, ok ? "ok" : "FAILED");
  if (!ok) ++failures;
}

}  // namespace

int main() {
  const std::vector<double> psi0 = initial_field();
  ShardedParams plain;
  ShardedParams filtered;
  filtered.model = OPFC_MODEL_FILTERED;
  filtered.r = -0.3;
  try {
    for (const auto &cfg : {std::make_pair(plain, 10), std::make_pair(filtered, 6)}) {
      const ShardedParams &p = cfg.first;
      const int steps = cfg.second;
      const bool is_plain = p.model == OPFC_MODEL_PLAIN;
      const std::vector<double> ref = unsharded(psi0, p, steps);
      for (int P : {1, 2, 4}) {
        char what[96];
        std::snprintf(what, sizeof what, "%s, %d steps, P = %d, FP64", is_plain ? "plain" : "filtered", steps, P);
        const double e64 = rel_l2(sharded<double>(psi0, p, steps, P), ref);
        expect(e64 <= 1e-11, what, e64);
        std::snprintf(what, sizeof what, "%s, %d steps, P = %d, FP32", is_plain ? "plain" : "filtered", steps, P);
        const double e32 = rel_l2(sharded<float>(psi0, p, steps, P), ref);
        expect(e32 <= 1e-5, what, e32);
      }
    }
    for (int P : {1, 2, 4}) {
      const auto e = fft_errors(psi0, P);
      char what[96];
      std::snprintf(what, sizeof what, "sharded forward transform, P = %d, FP64", P);
      expect(e.first <= 1e-12, what, e.first);
      std::snprintf(what, sizeof what, "sharded backward(forward), P = %d, FP64", P);
      expect(e.second <= 1e-12, what, e.second);
    }
    bool refused = false;
    try {
      LocalShardComm comm(3);
      ShardedPfc<float> m({kN[0], kN[1], kN[2]}, {1.0, 1.0, 1.0}, comm);
    } catch (const std::invalid_argument &) {
      refused = true;
    }
    expect(refused, "P = 3 on N2 = 32 refused (std::invalid_argument)", 0.0);
  } catch (const std::exception &e) {
    std::printf("exception: %s\n", e.what());
    return 2;
  }
  return failures == 0 ? 0 : 1;
}
