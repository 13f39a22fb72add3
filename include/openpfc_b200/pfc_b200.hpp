// pfc_b200.hpp -- C++ drop-in adapters over the C ABI (openpfc_b200.h).
//
// Header-only mirrors of the reference's host interface for the spectral PFC
// step, with the same names, argument meaning and error behaviour:
//   pfc::b200::B200FFT      -- pfc::fft::IFFT (include/openpfc/kernel/fft/fft_interface.hpp:40-83)
//   pfc::b200::TungstenParams -- TungstenParams (apps/tungsten/include/tungsten/common/tungsten_params.hpp)
//   pfc::b200::TungstenB200<T> -- the Tungsten model (cpu/tungsten_model.hpp:123-380,
//                              cuda/tungsten_model.hpp:80-500)
//   pfc::b200::PfcB200<T>   -- the plain conserved PFC model (docs/api/examples/10_complete_pfc_model.cpp:62-214)
//   pfc::b200::BinaryWriter / BinaryReader / VTKWriter / FileReader / format_with_number
//                           -- the on-disk formats (frontend/io/binary_writer.hpp,
//                              kernel/simulation/binary_reader.hpp, frontend/io/vtk_writer.hpp,
//                              initial_conditions/file_reader.hpp, frontend/utils/utils.hpp)
// A field decomposed over ranks (fft.cpp:72-81) is in openpfc_b200/sharded.hpp
// (ShardedPfc, ShardedFft).
// Size contracts throw std::invalid_argument, unknown fields std::out_of_range,
// everything else std::runtime_error (as in the reference).  T selects the
// device precision (float or double); host fields are std::vector<double>.
//
// Build: #include <openpfc_b200/pfc_b200.hpp>, link libopenpfc_b200.so.
#pragma once

#include <array>
#include <complex>
#include <cstddef>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../openpfc_b200.h"

namespace pfc {
namespace b200 {

inline void check(int rc, const char *what, const char *detail = "") {
  if (rc == OPFC_OK) return;
  std::string msg = std::string(what) + ": " + opfc_status_string(rc) + (detail && *detail ? std::string(" (") + detail + ")" : "");
  if (rc == OPFC_ERR_SIZE) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

/// Inclusive index box, as pfc::types::Box3i (fft_interface.hpp:77-82).
struct Box3i {
  std::array<int, 3> low{}, high{}, size{};
};

/// pfc::fft::IFFT on one B200.  forward: R2C unnormalised; backward: C2R with
/// 1/(N0 N1 N2) (fft_heffte_backend.hpp:216,243).
class B200FFT {
 public:
  explicit B200FFT(std::array<int, 3> n, int precision = OPFC_FP64, int device = 0) : n_(n) {
    opfc_desc d;
    opfc_desc_default(&d);
    for (int a = 0; a < 3; ++a) d.n[a] = n[a];
    d.precision = precision;
    d.device = device;
    check(opfc_create(&d, &h_), "B200FFT");
  }
  ~B200FFT() {
    if (h_) opfc_destroy(h_);
  }
  B200FFT(const B200FFT &) = delete;
  B200FFT &operator=(const B200FFT &) = delete;

  void forward(const std::vector<double> &in, std::vector<std::complex<double>> &out) {
    size_check(in.size(), out.size());
    check(opfc_fft_forward(h_, in.data(), out.data(), OPFC_F64, OPFC_HOST), "B200FFT::forward",
          opfc_last_error(h_));
  }
  void backward(const std::vector<std::complex<double>> &in, std::vector<double> &out) {
    size_check(out.size(), in.size());
    check(opfc_fft_backward(h_, in.data(), out.data(), OPFC_F64, OPFC_HOST), "B200FFT::backward",
          opfc_last_error(h_));
  }
  /// Device-resident buffers (the reference's DataBuffer<CudaTag, T> overloads,
  /// fft_heffte_backend.hpp:146-170,200-227): T = float or double, sizes as above.
  template <typename T> void forward_device(const T *in, std::complex<T> *out) {
    check(opfc_fft_forward(h_, in, out, dtype<T>(), OPFC_DEVICE), "B200FFT::forward_device", opfc_last_error(h_));
  }
  template <typename T> void backward_device(const std::complex<T> *in, T *out) {
    check(opfc_fft_backward(h_, in, out, dtype<T>(), OPFC_DEVICE), "B200FFT::backward_device", opfc_last_error(h_));
  }

  void reset_fft_time() { time_ = 0; }
  double get_fft_time() const { return time_; }
  size_t size_inbox() const { return opfc_size_inbox(h_); }
  size_t size_outbox() const { return opfc_size_outbox(h_); }
  size_t size_workspace() const { return size_outbox(); }
  size_t get_allocated_memory_bytes() const { return opfc_allocated_bytes(h_); }
  Box3i get_inbox_bounds() const { return box(n_[0]); }
  Box3i get_outbox_bounds() const { return box(n_[0] / 2 + 1); }

 private:
  template <typename T> static int dtype() {
    static_assert(std::is_same<T, float>::value || std::is_same<T, double>::value, "float or double");
    return std::is_same<T, double>::value ? OPFC_F64 : OPFC_F32;
  }
  void size_check(size_t real, size_t cplx) const {
    if (real != size_inbox() || cplx != size_outbox())
      throw std::invalid_argument("B200FFT: expected " + std::to_string(size_inbox()) + " reals and " +
                                  std::to_string(size_outbox()) + " complex values, got " +
                                  std::to_string(real) + " and " + std::to_string(cplx));
  }
  Box3i box(int nx) const {
    Box3i b;
    b.size = {nx, n_[1], n_[2]};
    b.high = {nx - 1, n_[1] - 1, n_[2] - 1};
    return b;
  }
  opfc_handle *h_ = nullptr;
  std::array<int, 3> n_;
  double time_ = 0;
};

/// TungstenParams: base parameters with setters/getters and derived getters,
/// defaults of tungsten_params.hpp:33-57, formulas of tungsten_params.hpp:339-411.
class TungstenParams {
 public:
  TungstenParams() {
    opfc_desc d;
    opfc_desc_default(&d);
    p_ = d.tungsten;
  }
#define OPFC_PARAM(name, type)                  \
  void set_##name(type v) { p_.name = v; }      \
  type get_##name() const { return p_.name; }
  OPFC_PARAM(n0, double)
  OPFC_PARAM(n_sol, double)
  OPFC_PARAM(n_vap, double)
  OPFC_PARAM(T, double)
  OPFC_PARAM(T0, double)
  OPFC_PARAM(Bx, double)
  OPFC_PARAM(alpha, double)
  OPFC_PARAM(alpha_farTol, double)
  OPFC_PARAM(alpha_highOrd, int)
  OPFC_PARAM(lambda, double)
  OPFC_PARAM(stabP, double)
  OPFC_PARAM(shift_u, double)
  OPFC_PARAM(shift_s, double)
  OPFC_PARAM(p2, double)
  OPFC_PARAM(p3, double)
  OPFC_PARAM(p4, double)
  OPFC_PARAM(q20, double)
  OPFC_PARAM(q21, double)
  OPFC_PARAM(q30, double)
  OPFC_PARAM(q31, double)
  OPFC_PARAM(q40, double)
#undef OPFC_PARAM
  double get_tau() const { return p_.T / p_.T0; }
  double get_p2_bar() const { return p_.p2 + 2 * p_.shift_s * p_.p3 + 3 * sq(p_.shift_s) * p_.p4; }
  double get_p3_bar() const { return p_.shift_u * (p_.p3 + 3 * p_.shift_s * p_.p4); }
  double get_p4_bar() const { return sq(p_.shift_u) * p_.p4; }
  double get_q20_bar() const { return p_.q20 + 2.0 * p_.shift_s * p_.q30 + 3.0 * sq(p_.shift_s) * p_.q40; }
  double get_q21_bar() const { return p_.q21 + 2.0 * p_.shift_s * p_.q31; }
  double get_q30_bar() const { return p_.shift_u * (p_.q30 + 3.0 * p_.shift_s * p_.q40); }
  double get_q31_bar() const { return p_.shift_u * p_.q31; }
  double get_q40_bar() const { return sq(p_.shift_u) * p_.q40; }
  double get_q2_bar() const { return get_q21_bar() * get_tau() + get_q20_bar(); }
  double get_q3_bar() const { return get_q31_bar() * get_tau() + get_q30_bar(); }
  double get_q4_bar() const { return get_q40_bar(); }
  const opfc_tungsten_params &raw() const { return p_; }

 private:
  static double sq(double x) { return x * x; }
  opfc_tungsten_params p_;
};

namespace detail {

/// Shared model body: host field mirrors synchronised on demand, like the GPU
/// model's prepare_for_field_modifiers / finalize_after_field_modifiers
/// (cuda/tungsten_model.hpp:265-291).
template <typename T> class ModelBase {
 public:
  ModelBase(std::array<int, 3> n, std::array<double, 3> dx, std::array<double, 3> origin, int device)
      : n_(n), dx_(dx), origin_(origin), device_(device) {}
  virtual ~ModelBase() {
    if (h_) opfc_destroy(h_);
  }
  ModelBase(const ModelBase &) = delete;
  ModelBase &operator=(const ModelBase &) = delete;

  virtual void initialize(double dt) {
    if (!h_) {
      opfc_desc d = describe();
      check(opfc_create(&d, &h_), "initialize");
    }
    check(opfc_initialize(h_, dt), "initialize", opfc_last_error(h_));
    for (auto &kv : fields_) kv.second.assign(cells(), 0.0);
  }

  /// One time step (Model::step, model.hpp:319).  Host edits of "psi" since the
  /// last step are uploaded first.
  virtual void step(double /*t*/) {
    finalize_after_field_modifiers();
    check(opfc_step(h_, 1), "step", opfc_last_error(h_));
    check(opfc_sync(h_), "step", opfc_last_error(h_));
    device_newer_ = true;
  }

  bool has_real_field(const std::string &name) const { return fields_.count(name) != 0; }

  /// Registered real field by name (model.hpp:536); downloads the device state
  /// if it is newer.  Throws std::out_of_range for unknown names.
  std::vector<double> &get_real_field(const std::string &name) {
    auto it = fields_.find(name);
    if (it == fields_.end()) throw std::out_of_range("unknown field: " + name);
    prepare_for_field_modifiers();
    host_dirty_ = true;  // the caller may write through the reference
    return it->second;
  }

  void prepare_for_field_modifiers() {
    if (!device_newer_ || !h_) return;
    std::vector<double> &psi = fields_.at("psi");
    check(opfc_get_psi(h_, psi.data(), psi.size(), OPFC_F64, OPFC_HOST), "prepare_for_field_modifiers",
          opfc_last_error(h_));
    download_extra();
    device_newer_ = false;
  }

  void finalize_after_field_modifiers() {
    if (!host_dirty_ || !h_) return;
    const std::vector<double> &psi = fields_.at("psi");
    check(opfc_set_psi(h_, psi.data(), psi.size(), OPFC_F64, OPFC_HOST), "finalize_after_field_modifiers",
          opfc_last_error(h_));
    host_dirty_ = false;
  }

  size_t get_allocated_memory_bytes() const { return h_ ? opfc_allocated_bytes(h_) : 0; }
  opfc_handle *handle() { return h_; }
  size_t cells() const { return (size_t)n_[0] * n_[1] * n_[2]; }
  std::array<int, 3> dims() const { return n_; }

 protected:
  virtual opfc_desc describe() const = 0;
  virtual void download_extra() {}
  opfc_desc base_desc() const {
    opfc_desc d;
    opfc_desc_default(&d);
    for (int a = 0; a < 3; ++a) {
      d.n[a] = n_[a];
      d.dx[a] = dx_[a];
      d.origin[a] = origin_[a];
    }
    d.precision = std::is_same<T, double>::value ? OPFC_FP64 : OPFC_FP32;
    d.device = device_;
    return d;
  }
  std::array<int, 3> n_;
  std::array<double, 3> dx_, origin_;
  int device_;
  opfc_handle *h_ = nullptr;
  std::map<std::string, std::vector<double>> fields_;
  bool device_newer_ = false, host_dirty_ = true;
};

}  // namespace detail

/// Tungsten model on one B200: fields "psi", "default" (an alias filled with
/// psi) and "psiMF" (cpu/tungsten_model.hpp:198-200); `params` as the reference.
template <typename T = double> class TungstenB200 : public detail::ModelBase<T> {
 public:
  TungstenB200(std::array<int, 3> n, std::array<double, 3> dx, std::array<double, 3> origin = {}, int device = 0)
      : detail::ModelBase<T>(n, dx, origin, device) {
    this->fields_["psi"];
    this->fields_["default"];
    this->fields_["psiMF"];
  }
  TungstenParams params;

 protected:
  opfc_desc describe() const override {
    opfc_desc d = this->base_desc();
    d.model = OPFC_MODEL_TUNGSTEN;
    d.tungsten = params.raw();
    return d;
  }
  void download_extra() override {
    this->fields_.at("default") = this->fields_.at("psi");
    std::vector<double> &mf = this->fields_.at("psiMF");
    check(opfc_get_psi_mf(this->h_, mf.data(), mf.size(), OPFC_F64, OPFC_HOST), "psiMF");
  }
};

/// Aluminum PFC variant (apps/aluminumNew/Aluminum.hpp): fields "psi",
/// "default" and "psiMF"; the same setters as Aluminum (set_n0 ... set_q2_bar_L)
/// on a parameter block that starts at 0 (T0 = 1) like Aluminum::params.
/// step(t) uses t for the moving temperature T_var(x, t) (G_grid != 0), as
/// Aluminum::step(t) does.
template <typename T = double> class AluminumB200 : public detail::ModelBase<T> {
 public:
  AluminumB200(std::array<int, 3> n, std::array<double, 3> dx, std::array<double, 3> origin = {}, int device = 0)
      : detail::ModelBase<T>(n, dx, origin, device) {
    opfc_desc d;
    opfc_desc_default(&d);
    params = d.aluminum;
    this->fields_["psi"];
    this->fields_["default"];
    this->fields_["psiMF"];
  }
  opfc_aluminum_params params;
  void step(double t) override {
    check(opfc_set_time(this->h_, t, 0.0), "step", opfc_last_error(this->h_));
    detail::ModelBase<T>::step(t);
  }
#define OPFC_ALU(name, type) \
  void set_##name(type v) { params.name = v; }
  OPFC_ALU(n0, double)
  OPFC_ALU(n_sol, double)
  OPFC_ALU(n_vap, double)
  OPFC_ALU(T, double)
  OPFC_ALU(T0, double)
  OPFC_ALU(Bx, double)
  OPFC_ALU(T_const, double)
  OPFC_ALU(T_max, double)
  OPFC_ALU(T_min, double)
  OPFC_ALU(G_grid, double)
  OPFC_ALU(V_grid, double)
  OPFC_ALU(x_initial, double)
  OPFC_ALU(m_xpos, double)
  OPFC_ALU(alpha, double)
  OPFC_ALU(alpha_farTol, double)
  OPFC_ALU(alpha_highOrd, int)
  OPFC_ALU(tau_const, double)
  OPFC_ALU(lambda, double)
  OPFC_ALU(stabP, double)
  OPFC_ALU(shift_u, double)
  OPFC_ALU(shift_s, double)
  OPFC_ALU(p2, double)
  OPFC_ALU(p3, double)
  OPFC_ALU(p4, double)
  OPFC_ALU(p2_bar, double)
  OPFC_ALU(p3_bar, double)
  OPFC_ALU(p4_bar, double)
  OPFC_ALU(q20, double)
  OPFC_ALU(q21, double)
  OPFC_ALU(q30, double)
  OPFC_ALU(q31, double)
  OPFC_ALU(q40, double)
  OPFC_ALU(q20_bar, double)
  OPFC_ALU(q21_bar, double)
  OPFC_ALU(q30_bar, double)
  OPFC_ALU(q31_bar, double)
  OPFC_ALU(q40_bar, double)
  OPFC_ALU(q2_bar, double)
  OPFC_ALU(q3_bar, double)
  OPFC_ALU(q4_bar, double)
  OPFC_ALU(q2_bar_L, double)
#undef OPFC_ALU

 protected:
  opfc_desc describe() const override {
    opfc_desc d = this->base_desc();
    d.model = OPFC_MODEL_ALUMINUM;
    d.aluminum = params;
    return d;
  }
  void download_extra() override {
    this->fields_.at("default") = this->fields_.at("psi");
    std::vector<double> &mf = this->fields_.at("psiMF");
    check(opfc_get_psi_mf(this->h_, mf.data(), mf.size(), OPFC_F64, OPFC_HOST), "psiMF");
  }
};

/// Plain conserved PFC (10_complete_pfc_model.cpp:62-214): field "density"
/// (registered name in the example) and "psi".
template <typename T = double> class PfcB200 : public detail::ModelBase<T> {
 public:
  PfcB200(std::array<int, 3> n, std::array<double, 3> dx, double epsilon, std::array<double, 3> origin = {},
          int device = 0)
      : detail::ModelBase<T>(n, dx, origin, device), epsilon_(epsilon) {
    this->fields_["psi"];
  }
  double get_epsilon() const { return epsilon_; }
  void set_epsilon(double e) {
    epsilon_ = e;
    if (this->h_) check(opfc_set_r(this->h_, e), "set_epsilon");
  }
  double free_energy() {
    this->finalize_after_field_modifiers();
    double f = 0;
    check(opfc_free_energy(this->h_, &f), "free_energy");
    return f;
  }
  double mean_density() {
    this->finalize_after_field_modifiers();
    double m = 0;
    check(opfc_mass(this->h_, &m), "mean_density");
    return m;
  }

 protected:
  opfc_desc describe() const override {
    opfc_desc d = this->base_desc();
    d.model = OPFC_MODEL_PLAIN;
    d.r = epsilon_;
    return d;
  }

 private:
  double epsilon_;
};

// ---------------------------------------------------------------------------
// On-disk formats: host-side mirrors of the reference's writers and readers
// for one process (set_domain(global, local, offset) as the MPI versions; the
// box is written at its place in the global file).  Same file layouts:
// BinaryWriter / BinaryReader (frontend/io/binary_writer.hpp,
// kernel/simulation/binary_reader.hpp), VTKWriter (frontend/io/vtk_writer.hpp),
// FileReader (kernel/simulation/initial_conditions/file_reader.hpp).
// ---------------------------------------------------------------------------

/// pfc::utils::format_with_number; throws std::invalid_argument on a bad pattern.
inline std::string format_with_number(const std::string &pattern, int increment) {
  std::vector<char> out(pattern.size() + 64);
  const int rc = opfc_format_filename(pattern.c_str(), increment, out.data(), out.size());
  if (rc == OPFC_ERR_ARG) throw std::invalid_argument("format_with_number: invalid filename pattern '" + pattern + "'");
  check(rc, "format_with_number");
  return std::string(out.data());
}

class DomainIO {
 public:
  explicit DomainIO(std::string filename) : filename_(std::move(filename)) {}
  void set_domain(const std::array<int, 3> &global, const std::array<int, 3> &local,
                  const std::array<int, 3> &offset) {
    for (int a = 0; a < 3; ++a)
      if (global[a] < 1 || local[a] < 1 || offset[a] < 0 || offset[a] + local[a] > global[a])
        throw std::invalid_argument("set_domain: local box outside the global box");
    global_ = global;
    local_ = local;
    offset_ = offset;
    valid_ = true;
  }

 protected:
  size_t expect(const char *who, size_t got) const {
    if (!valid_) throw std::runtime_error(std::string(who) + ": set_domain() was not called");
    const size_t n = (size_t)local_[0] * local_[1] * local_[2];
    if (got != n)
      throw std::runtime_error(std::string(who) + ": buffer size mismatch (expected " + std::to_string(n) +
                               " elements from set_domain, got " + std::to_string(got) + ")");
    return n;
  }
  std::string filename_;
  std::array<int, 3> global_{}, local_{}, offset_{};
  bool valid_ = false;
};

/// Raw native doubles of the global array, x fastest, no header.
class BinaryWriter : public DomainIO {
 public:
  using DomainIO::DomainIO;
  /// Truncate the file of `increment` and size it to the global array: the
  /// one-time step before several writers each write their own box (the
  /// reference does it collectively with MPI_File_set_size(fh, 0)).  A writer
  /// whose box is the whole array truncates by itself.
  void prepare(int increment, int ncomp = 1) {
    const std::string fn = format_with_number(filename_, increment);
    check(opfc_prepare_raw(fn.c_str(), global_.data(), ncomp), "BinaryWriter::prepare", fn.c_str());
  }
  void write(int increment, const std::vector<double> &data) {
    expect("BinaryWriter::write", data.size());
    const std::string fn = format_with_number(filename_, increment);
    check(opfc_write_raw(fn.c_str(), global_.data(), local_.data(), offset_.data(), data.data(), 1),
          "BinaryWriter::write", fn.c_str());
  }
  void write(int increment, const std::vector<std::complex<double>> &data) {
    expect("BinaryWriter::write", data.size());
    const std::string fn = format_with_number(filename_, increment);
    check(opfc_write_raw(fn.c_str(), global_.data(), local_.data(), offset_.data(),
                         reinterpret_cast<const double *>(data.data()), 2),
          "BinaryWriter::write", fn.c_str());
  }
};

class BinaryReader : public DomainIO {
 public:
  BinaryReader() : DomainIO("") {}
  void read(const std::string &filename, std::vector<double> &data) {
    expect("BinaryReader::read", data.size());
    check(opfc_read_raw(filename.c_str(), global_.data(), local_.data(), offset_.data(), data.data(), 1),
          "BinaryReader::read", filename.c_str());
  }
  void read(const std::string &filename, std::vector<std::complex<double>> &data) {
    expect("BinaryReader::read", data.size());
    check(opfc_read_raw(filename.c_str(), global_.data(), local_.data(), offset_.data(),
                        reinterpret_cast<double *>(data.data()), 2),
          "BinaryReader::read", filename.c_str());
  }
};

/// VTK XML ImageData piece (.vti), Float64 point data appended raw; a complex
/// field is written as its magnitude.
class VTKWriter : public DomainIO {
 public:
  using DomainIO::DomainIO;
  void set_origin(const std::array<double, 3> &o) { origin_ = o; }
  void set_spacing(const std::array<double, 3> &s) {
    for (double v : s)
      if (!(v > 0)) throw std::invalid_argument("VTKWriter::set_spacing: spacing must be positive");
    spacing_ = s;
  }
  void set_field_name(const std::string &name) { name_ = name; }
  void write(int increment, const std::vector<double> &data) {
    expect("VTKWriter::write", data.size());
    const std::string fn = format_with_number(filename_, increment);
    check(opfc_write_vti_raw(fn.c_str(), global_.data(), local_.data(), offset_.data(), origin_.data(),
                             spacing_.data(), name_.c_str(), data.data()),
          "VTKWriter::write", fn.c_str());
  }
  void write(int increment, const std::vector<std::complex<double>> &data) {
    std::vector<double> mag(data.size());
    for (size_t i = 0; i < data.size(); ++i) mag[i] = std::abs(data[i]);
    write(increment, mag);
  }

 private:
  std::array<double, 3> origin_{0, 0, 0}, spacing_{1, 1, 1};
  std::string name_ = "Field";
};

/// Initial condition from a raw FP64 file (FieldModifier::apply).
class FileReader {
 public:
  FileReader() = default;
  explicit FileReader(std::string filename) : filename_(std::move(filename)) {}
  void set_filename(std::string filename) { filename_ = std::move(filename); }
  const std::string &get_filename() const { return filename_; }
  template <typename Model> void apply(Model &m, double /*time*/) {
    std::vector<double> &psi = m.get_real_field("psi");
    BinaryReader r;
    r.set_domain(m.dims(), m.dims(), {0, 0, 0});
    try {
      r.read(filename_, psi);
    } catch (const std::exception &ex) {
      throw std::runtime_error("FileReader failed to read \"" + filename_ + "\" into field \"psi\": " + ex.what());
    }
  }

 private:
  std::string filename_;
};

}  // namespace b200
}  // namespace pfc
