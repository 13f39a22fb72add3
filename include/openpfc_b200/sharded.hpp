// sharded.hpp -- one field sharded over ranks, host side in C++ over the C ABI.
//
// The reference splits a field over MPI ranks and lets HeFFTe reshape it
// between the decompositions each FFT direction needs
// (src/openpfc/runtime/cpu/fft.cpp:72-81, its plan_options).  Here a grid
// N0 x N1 x N2 on P ranks is held
//   * in z slabs for the x and y passes: rank q owns the planes
//     z in [q N2/P, (q+1) N2/P) of the real field and of the half spectrum
//     transformed along x and y;
//   * in kx slabs for the z transform and the z update: rank r owns the
//     half-spectrum columns kx in [r M/P, (r+1) M/P), M = N0/2, for every ky
//     and kz; the last rank also the kx = M (Nyquist) plane,
// with an all-to-all transpose between the two (two per PFC step, as the
// reference's reshapes).  Each rank's compute runs on two library handles (a
// z-slab handle and a kx-slab handle whose operators use the global wave
// numbers) through opfc_pass; a transpose packs each peer's block with strided
// device copies, exchanges the blocks through a ShardComm and unpacks them.
// Every block holds M/P + 1 columns, the last one being the next rank's first
// column (or the Nyquist plane on the last rank), so every pair exchanges the
// same number of bytes; a kx-slab handle's own Nyquist plane thus holds a copy
// of the next rank's first column, which it evolves like that rank and never
// sends back.
//
// ShardComm is the exchange: LocalShardComm emulates P ranks in one process
// (device copies; the 1-GPU form of the whole decomposition), NcclShardComm
// (compiled when nccl.h is included first) runs one rank per process over NCCL,
// and an MPI build supplies its own ShardComm over a CUDA-aware MPI_Alltoall.
//
// Build: #include <openpfc_b200/sharded.hpp>; link libopenpfc_b200.so and the
// CUDA runtime (-lcudart).
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cmath>
#include <complex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../openpfc_b200.h"
#include "pfc_b200.hpp"

namespace pfc {
namespace b200 {

inline void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

/// Compensated (Neumaier) sum of doubles.
inline double neumaier_sum(const double *v, size_t n) {
  double s = 0.0, c = 0.0;
  for (size_t i = 0; i < n; ++i) {
    const double t = s + v[i];
    c += std::fabs(s) >= std::fabs(v[i]) ? (s - t) + v[i] : (v[i] - t) + s;
    s = t;
  }
  return s + c;
}

/// The exchange of a sharded field.  A process holds the ranks local_ranks();
/// in alltoall, local rank i sends send[i] + p * bytes to rank p and receives
/// rank p's block at recv[i] + p * bytes, all enqueued on `stream` (device
/// buffers).  allreduce_sum returns the sum over every rank of the values the
/// local ranks contribute (one per local rank).
struct ShardComm {
  virtual ~ShardComm() = default;
  virtual int size() const = 0;
  virtual std::vector<int> local_ranks() const = 0;
  virtual void alltoall(const std::vector<const void *> &send, const std::vector<void *> &recv, size_t bytes,
                        cudaStream_t stream) = 0;
  virtual double allreduce_sum(const std::vector<double> &local) = 0;
};

/// P ranks emulated in one process: every rank is local and an all-to-all is a
/// set of device copies between their buffers.
class LocalShardComm : public ShardComm {
 public:
  explicit LocalShardComm(int p) : p_(p) {
    if (p < 1) throw std::invalid_argument("LocalShardComm: at least one rank");
  }
  int size() const override { return p_; }
  std::vector<int> local_ranks() const override {
    std::vector<int> r(p_);
    std::iota(r.begin(), r.end(), 0);
    return r;
  }
  void alltoall(const std::vector<const void *> &send, const std::vector<void *> &recv, size_t bytes,
                cudaStream_t stream) override {
    for (int d = 0; d < p_; ++d)
      for (int s = 0; s < p_; ++s)
        cuda_check(cudaMemcpyAsync(static_cast<char *>(recv[d]) + size_t(s) * bytes,
                                   static_cast<const char *>(send[s]) + size_t(d) * bytes, bytes,
                                   cudaMemcpyDeviceToDevice, stream),
                   "LocalShardComm::alltoall");
  }
  double allreduce_sum(const std::vector<double> &local) override {
    return neumaier_sum(local.data(), local.size());
  }

 private:
  int p_;
};

#if defined(NCCL_MAJOR)
/// One rank per process over NCCL: the all-to-all is a group of point-to-point
/// send / receive pairs (every peer at the NVSwitch's full bandwidth), the
/// reduction an ncclAllReduce of one double.  The communicator, its device and
/// rank are the caller's (ncclCommInitRank); `scratch` needs one double of
/// device memory.
class NcclShardComm : public ShardComm {
 public:
  NcclShardComm(ncclComm_t comm, int rank, int size, double *scratch)
      : comm_(comm), rank_(rank), size_(size), scratch_(scratch) {}
  int size() const override { return size_; }
  std::vector<int> local_ranks() const override { return {rank_}; }
  void alltoall(const std::vector<const void *> &send, const std::vector<void *> &recv, size_t bytes,
                cudaStream_t stream) override {
    nccl_check(ncclGroupStart());
    for (int p = 0; p < size_; ++p) {
      nccl_check(ncclSend(static_cast<const char *>(send[0]) + size_t(p) * bytes, bytes, ncclChar, p, comm_, stream));
      nccl_check(ncclRecv(static_cast<char *>(recv[0]) + size_t(p) * bytes, bytes, ncclChar, p, comm_, stream));
    }
    nccl_check(ncclGroupEnd());
  }
  double allreduce_sum(const std::vector<double> &local) override {
    double v = local.at(0), out = 0.0;
    cuda_check(cudaMemcpy(scratch_, &v, sizeof(double), cudaMemcpyHostToDevice), "NcclShardComm");
    nccl_check(ncclAllReduce(scratch_, scratch_, 1, ncclDouble, ncclSum, comm_, nullptr));
    cuda_check(cudaMemcpy(&out, scratch_, sizeof(double), cudaMemcpyDeviceToHost), "NcclShardComm");
    return out;
  }

 private:
  static void nccl_check(ncclResult_t r) {
    if (r != ncclSuccess) throw std::runtime_error(std::string("NcclShardComm: ") + ncclGetErrorString(r));
  }
  ncclComm_t comm_;
  int rank_, size_;
  double *scratch_;
};
#endif

/// A plain or filtered PFC field on the ranks of a ShardComm (the reference's
/// Model over a decomposed World, model.hpp:151; the decomposition of
/// fft.cpp:72-81), held as real z slabs per rank.  N2 and N0/2 must be
/// multiples of the number of ranks P, and N2/P, N0/(2P) supported transform
/// lengths (else std::invalid_argument).  T selects the device precision; all
/// handles and copies of the process run on one CUDA stream.
/// Model and parameters of a sharded field (the descriptor's PLAIN / FILTERED
/// fields).
struct ShardedParams {
  int model = OPFC_MODEL_PLAIN;  // OPFC_MODEL_PLAIN or OPFC_MODEL_FILTERED
  double r = -0.25, alpha = 0.5, p2 = -0.1, p3 = -0.5, p4 = 0.3;
};

template <typename T = float> class ShardedPfc {
  static_assert(std::is_same<T, float>::value || std::is_same<T, double>::value, "float or double");

 public:
  using Params = ShardedParams;

  ShardedPfc(std::array<int, 3> n, std::array<double, 3> dx, ShardComm &comm, Params p = Params(),
             int device = 0)
      : n_(n), dx_(dx), comm_(comm), p_(p), device_(device), P_(comm.size()) {
    const int M = n[0] / 2;
    if (n[2] % P_ || M % P_)
      throw std::invalid_argument("ShardedPfc: N2 and N0/2 must be multiples of the number of ranks");
    n2loc_ = n[2] / P_;
    mloc_ = M / P_;
    rows_ = size_t(n2loc_) * n[1];
    block_ = rows_ * size_t(mloc_ + 1) * kCs;
    cuda_check(cudaSetDevice(device), "ShardedPfc");
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "ShardedPfc");
    try {
      for (int rk : comm.local_ranks()) {
        ranks_.push_back(Rank{});
        Rank &R = ranks_.back();
        R.rank = rk;
        R.zs = create({n[0], n[1], n2loc_}, 0);
        R.kx = create({2 * mloc_, n[1], n[2]}, rk * mloc_);
        cuda_check(cudaMalloc(&R.send, block_ * P_), "ShardedPfc");
        cuda_check(cudaMalloc(&R.recv, block_ * P_), "ShardedPfc");
      }
    } catch (...) {
      release();
      throw;
    }
  }
  ~ShardedPfc() { release(); }
  ShardedPfc(const ShardedPfc &) = delete;
  ShardedPfc &operator=(const ShardedPfc &) = delete;

  /// Operator tables of every kx-slab handle (Model::initialize(dt)).
  void initialize(double dt) {
    for (Rank &R : ranks_) check(opfc_initialize(R.kx, dt), "ShardedPfc::initialize", opfc_last_error(R.kx));
  }

  /// slabs[i]: local rank i's real z slab, N2/P x N1 x N0 values, x fastest.
  void set_psi(const std::vector<const double *> &slabs) {
    need(slabs.size(), "set_psi");
    const size_t cells = rows_ * size_t(n_[0]);
    std::vector<double> sums;
    for (const double *s : slabs) sums.push_back(neumaier_sum(s, cells));
    mean_ = comm_.allreduce_sum(sums) / (double(n_[0]) * n_[1] * n_[2]);
    host_.assign(ranks_.size(), std::vector<T>());
    for (size_t i = 0; i < ranks_.size(); ++i) {
      host_[i].assign(slabs[i], slabs[i] + cells);
      cuda_check(cudaMemcpyAsync(opfc_array(ranks_[i].zs, OPFC_ARRAY_REAL), host_[i].data(), cells * sizeof(T),
                                 cudaMemcpyHostToDevice, stream_),
                 "ShardedPfc::set_psi");
    }
    for (Rank &R : ranks_) pass(R.zs, OPFC_PASS_XY_FORWARD);
    z_to_kx();
    // the k = 0 slot (global rank 0's first column) stays zero; the mean is carried apart
    for (Rank &R : ranks_) pass(R.kx, OPFC_PASS_Z_FORWARD, 0.0, R.rank == 0 ? 4 : 0);
    a_ready_ = false;
    sync();
  }

  /// n_steps PFC steps (Model::step, model.hpp:319), two transposes each.
  void step(int n_steps = 1) {
    if (!a_ready_) {
      for (Rank &R : ranks_) pass(R.kx, OPFC_PASS_Z_INVERSE);
      kx_to_z();
      for (Rank &R : ranks_) pass(R.zs, OPFC_PASS_Y_INVERSE);
      a_ready_ = true;
    }
    for (int s = 0; s < n_steps; ++s) {
      for (Rank &R : ranks_) {
        pass(R.zs, OPFC_PASS_X_FUSED, mean_);
        pass(R.zs, OPFC_PASS_Y_FORWARD);
      }
      z_to_kx();
      for (Rank &R : ranks_)
        pass(R.kx, OPFC_PASS_Z_UPDATE, 0.0, (R.rank == 0 ? 1 : 0) | (R.rank == P_ - 1 ? 2 : 0));
      kx_to_z();
      for (Rank &R : ranks_) pass(R.zs, OPFC_PASS_Y_INVERSE);
    }
  }

  /// Waits for the stream; throws on a handle's error (non-finite field, timeout).
  void sync() {
    cuda_check(cudaStreamSynchronize(stream_), "ShardedPfc::sync");
    for (Rank &R : ranks_)
      for (opfc_handle *h : {R.zs, R.kx}) check(opfc_sync(h), "ShardedPfc::sync", opfc_last_error(h));
  }

  /// slabs[i] receives local rank i's real z slab (N2/P x N1 x N0 doubles).
  void get_psi(const std::vector<double *> &slabs) {
    need(slabs.size(), "get_psi");
    for (Rank &R : ranks_) pass(R.kx, OPFC_PASS_Z_INVERSE_STATE);
    kx_to_z();
    for (Rank &R : ranks_) pass(R.zs, OPFC_PASS_XY_BACKWARD, mean_);
    const size_t cells = rows_ * size_t(n_[0]);
    host_.assign(ranks_.size(), std::vector<T>(cells));
    for (size_t i = 0; i < ranks_.size(); ++i)
      cuda_check(cudaMemcpyAsync(host_[i].data(), opfc_array(ranks_[i].zs, OPFC_ARRAY_REAL), cells * sizeof(T),
                                 cudaMemcpyDeviceToHost, stream_),
                 "ShardedPfc::get_psi");
    sync();
    for (size_t i = 0; i < ranks_.size(); ++i)
      for (size_t c = 0; c < cells; ++c) slabs[i][c] = double(host_[i][c]);
    a_ready_ = false;  // the work arrays were used for the output
  }

  double mass() const { return mean_; }
  int ranks() const { return P_; }
  std::vector<int> local_ranks() const { return comm_.local_ranks(); }
  cudaStream_t stream() const { return stream_; }

 private:
  template <typename> friend class ShardedFft;
  static constexpr size_t kCs = 2 * sizeof(T);  // one complex value
  struct Rank {
    int rank = 0;
    opfc_handle *zs = nullptr, *kx = nullptr;
    void *send = nullptr, *recv = nullptr;
  };

  opfc_handle *create(std::array<int, 3> n, int kx0) {
    opfc_desc d;
    opfc_desc_default(&d);
    for (int a = 0; a < 3; ++a) {
      d.n[a] = n[a];
      d.dx[a] = dx_[a];
      d.n_global[a] = n_[a];
    }
    d.kx0 = kx0;
    d.precision = std::is_same<T, double>::value ? OPFC_FP64 : OPFC_FP32;
    d.model = p_.model;
    d.r = p_.r;
    d.filter_alpha = p_.alpha;
    d.p2 = p_.p2;
    d.p3 = p_.p3;
    d.p4 = p_.p4;
    d.device = device_;
    d.stream = stream_;
    opfc_handle *h = nullptr;
    check(opfc_create(&d, &h), "ShardedPfc");
    return h;
  }
  void release() {
    for (Rank &R : ranks_) {
      if (R.zs) opfc_destroy(R.zs);
      if (R.kx) opfc_destroy(R.kx);
      if (R.send) cudaFree(R.send);
      if (R.recv) cudaFree(R.recv);
      R = Rank{};
    }
    ranks_.clear();
    if (stream_) cudaStreamDestroy(stream_);
    stream_ = nullptr;
  }
  void need(size_t k, const char *what) const {
    if (k != ranks_.size())
      throw std::invalid_argument(std::string("ShardedPfc::") + what + ": one slab per local rank");
  }
  void pass(opfc_handle *h, int p, double mean = 0.0, int flags = 0) {
    check(opfc_pass(h, p, mean, flags), "ShardedPfc: opfc_pass", opfc_last_error(h));
  }
  void copy2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width) {
    cuda_check(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows_, cudaMemcpyDeviceToDevice, stream_),
               "ShardedPfc: transpose copy");
  }
  // A handle's work array: main part [z][y][nx] complex values, then the
  // Nyquist plane [z][y].
  char *work(opfc_handle *h) { return static_cast<char *>(opfc_array(h, OPFC_ARRAY_WORK)); }

  // z slabs -> kx slabs: the block for rank r holds columns r Mloc .. r Mloc + Mloc
  // of every (z, y) row of the slab (the last one from the Nyquist plane on the
  // last rank); blocks from z slab q fill rows q N2/P .. of the kx slab.
  void z_to_kx() {
    const size_t M = size_t(n_[0]) / 2, ml = size_t(mloc_), bp = (ml + 1) * kCs;
    std::vector<const void *> send;
    std::vector<void *> recv;
    for (Rank &R : ranks_) {
      char *zm = work(R.zs), *zn = zm + M * rows_ * kCs;
      char *dst = static_cast<char *>(R.send);
      for (int r = 0; r < P_; ++r, dst += block_) {
        copy2d(dst, bp, zm + size_t(r) * ml * kCs, M * kCs, ml * kCs);
        if (r < P_ - 1)
          copy2d(dst + ml * kCs, bp, zm + size_t(r + 1) * ml * kCs, M * kCs, kCs);
        else
          copy2d(dst + ml * kCs, bp, zn, kCs, kCs);
      }
      send.push_back(R.send);
      recv.push_back(R.recv);
    }
    comm_.alltoall(send, recv, block_, stream_);
    for (Rank &R : ranks_) {
      char *km = work(R.kx), *kn = km + ml * size_t(n_[1]) * n_[2] * kCs;
      const char *src = static_cast<const char *>(R.recv);
      for (int q = 0; q < P_; ++q, src += block_) {
        copy2d(km + size_t(q) * rows_ * ml * kCs, ml * kCs, src, bp, ml * kCs);
        copy2d(kn + size_t(q) * rows_ * kCs, kCs, src + ml * kCs, bp, kCs);
      }
    }
  }

  // kx slabs -> z slabs: the inverse; only the last rank's extra column (the
  // Nyquist plane) is kept, the others duplicate the next rank's first column.
  void kx_to_z() {
    const size_t M = size_t(n_[0]) / 2, ml = size_t(mloc_), bp = (ml + 1) * kCs;
    std::vector<const void *> send;
    std::vector<void *> recv;
    for (Rank &R : ranks_) {
      char *km = work(R.kx), *kn = km + ml * size_t(n_[1]) * n_[2] * kCs;
      char *dst = static_cast<char *>(R.send);
      for (int q = 0; q < P_; ++q, dst += block_) {
        copy2d(dst, bp, km + size_t(q) * rows_ * ml * kCs, ml * kCs, ml * kCs);
        copy2d(dst + ml * kCs, bp, kn + size_t(q) * rows_ * kCs, kCs, kCs);
      }
      send.push_back(R.send);
      recv.push_back(R.recv);
    }
    comm_.alltoall(send, recv, block_, stream_);
    for (Rank &R : ranks_) {
      char *zm = work(R.zs), *zn = zm + M * rows_ * kCs;
      const char *src = static_cast<const char *>(R.recv);
      for (int r = 0; r < P_; ++r, src += block_) {
        copy2d(zm + size_t(r) * ml * kCs, M * kCs, src, bp, ml * kCs);
        if (r == P_ - 1) copy2d(zn, kCs, src + ml * kCs, bp, kCs);
      }
    }
  }

  std::array<int, 3> n_;
  std::array<double, 3> dx_;
  ShardComm &comm_;
  Params p_;
  int device_, P_;
  int n2loc_ = 0, mloc_ = 0;
  size_t rows_ = 0, block_ = 0;  // (z, y) rows of a z slab; bytes of one exchanged block
  cudaStream_t stream_ = nullptr;
  std::vector<Rank> ranks_;
  std::vector<std::vector<T>> host_;  // host staging of set_psi / get_psi
  double mean_ = 0.0;
  bool a_ready_ = false;
};

/// The sharded 3D transform alone, the IFFT contract over a decomposed field
/// (fft_interface.hpp:51,61 on the decomposition of fft.cpp:72-81): forward
/// takes each local rank's real z slab (N2/P x N1 x N0, x fastest) and returns
/// its kx slab of the half spectrum, N2 x N1 x cols complex values in the
/// reference order, cols = N0/(2P) plus the kx = N0/2 plane on the last rank;
/// backward is the inverse with the 1/(N0 N1 N2) scaling.
template <typename T = double> class ShardedFft {
 public:
  ShardedFft(std::array<int, 3> n, ShardComm &comm, int device = 0)
      : m_(n, {1.0, 1.0, 1.0}, comm, ShardedParams(), device) {}

  /// Columns of local rank i's kx slab (reference order, last rank + 1).
  int columns(size_t i) const { return m_.mloc_ + (m_.ranks_[i].rank == m_.P_ - 1 ? 1 : 0); }

  void forward(const std::vector<const double *> &slabs, const std::vector<std::complex<double> *> &out) {
    m_.need(slabs.size(), "forward");
    m_.need(out.size(), "forward");
    upload_real(slabs);
    for (auto &R : m_.ranks_) m_.pass(R.zs, OPFC_PASS_XY_FORWARD);
    m_.z_to_kx();
    for (auto &R : m_.ranks_) m_.pass(R.kx, OPFC_PASS_Z_FORWARD);
    const size_t lines = size_t(m_.n_[1]) * m_.n_[2], ml = size_t(m_.mloc_);
    std::vector<std::vector<T>> h(m_.ranks_.size(), std::vector<T>(2 * (ml + 1) * lines));
    for (size_t i = 0; i < m_.ranks_.size(); ++i)
      cuda_check(cudaMemcpyAsync(h[i].data(), opfc_array(m_.ranks_[i].kx, OPFC_ARRAY_STATE),
                                 h[i].size() * sizeof(T), cudaMemcpyDeviceToHost, m_.stream_),
                 "ShardedFft::forward");
    m_.sync();
    for (size_t i = 0; i < m_.ranks_.size(); ++i) {
      const size_t cols = size_t(columns(i));
      const T *main = h[i].data(), *nyq = main + 2 * ml * lines;
      for (size_t l = 0; l < lines; ++l) {
        for (size_t k = 0; k < ml; ++k)
          out[i][l * cols + k] = std::complex<double>(main[2 * (l * ml + k)], main[2 * (l * ml + k) + 1]);
        if (cols > ml) out[i][l * cols + ml] = std::complex<double>(nyq[2 * l], nyq[2 * l + 1]);
      }
    }
  }

  void backward(const std::vector<const std::complex<double> *> &in, const std::vector<double *> &slabs) {
    m_.need(in.size(), "backward");
    m_.need(slabs.size(), "backward");
    const size_t lines = size_t(m_.n_[1]) * m_.n_[2], ml = size_t(m_.mloc_);
    std::vector<std::vector<T>> h(m_.ranks_.size(), std::vector<T>(2 * (ml + 1) * lines, T(0)));
    for (size_t i = 0; i < m_.ranks_.size(); ++i) {
      const size_t cols = size_t(columns(i));
      T *main = h[i].data(), *nyq = main + 2 * ml * lines;
      for (size_t l = 0; l < lines; ++l) {
        for (size_t k = 0; k < ml; ++k) {
          main[2 * (l * ml + k)] = T(in[i][l * cols + k].real());
          main[2 * (l * ml + k) + 1] = T(in[i][l * cols + k].imag());
        }
        if (cols > ml) {  // the kx = N0/2 plane lives on the last rank only
          nyq[2 * l] = T(in[i][l * cols + ml].real());
          nyq[2 * l + 1] = T(in[i][l * cols + ml].imag());
        }
      }
      cuda_check(cudaMemcpyAsync(opfc_array(m_.ranks_[i].kx, OPFC_ARRAY_STATE), h[i].data(),
                                 h[i].size() * sizeof(T), cudaMemcpyHostToDevice, m_.stream_),
                 "ShardedFft::backward");
    }
    for (auto &R : m_.ranks_) m_.pass(R.kx, OPFC_PASS_Z_INVERSE_STATE);
    m_.kx_to_z();
    for (auto &R : m_.ranks_) m_.pass(R.zs, OPFC_PASS_XY_BACKWARD, 0.0);
    download_real(slabs);
  }

 private:
  void upload_real(const std::vector<const double *> &slabs) {
    const size_t cells = m_.rows_ * size_t(m_.n_[0]);
    m_.host_.assign(m_.ranks_.size(), std::vector<T>());
    for (size_t i = 0; i < m_.ranks_.size(); ++i) {
      m_.host_[i].assign(slabs[i], slabs[i] + cells);
      cuda_check(cudaMemcpyAsync(opfc_array(m_.ranks_[i].zs, OPFC_ARRAY_REAL), m_.host_[i].data(),
                                 cells * sizeof(T), cudaMemcpyHostToDevice, m_.stream_),
                 "ShardedFft");
    }
  }
  void download_real(const std::vector<double *> &slabs) {
    const size_t cells = m_.rows_ * size_t(m_.n_[0]);
    m_.host_.assign(m_.ranks_.size(), std::vector<T>(cells));
    for (size_t i = 0; i < m_.ranks_.size(); ++i)
      cuda_check(cudaMemcpyAsync(m_.host_[i].data(), opfc_array(m_.ranks_[i].zs, OPFC_ARRAY_REAL),
                                 cells * sizeof(T), cudaMemcpyDeviceToHost, m_.stream_),
                 "ShardedFft");
    m_.sync();
    for (size_t i = 0; i < m_.ranks_.size(); ++i)
      for (size_t c = 0; c < cells; ++c) slabs[i][c] = double(m_.host_[i][c]);
  }
  ShardedPfc<T> m_;
};

}  // namespace b200
}  // namespace pfc
