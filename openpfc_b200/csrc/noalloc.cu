// noalloc.cu -- forward 3D R2C transform that allocates no device memory.
//
// Some callers cannot call cudaMalloc: latency-bound loops cannot absorb its
// implicit device-wide synchronisation and unbounded run time, and some host
// applications own every device allocation through their own memory manager
// and do not let a library allocate.  For them opfc_fft_forward_noalloc runs the
// same passes as opfc_fft_forward (x R2C -> y -> z -> reference layout) but
// keeps its intermediate half spectrum in the file-scope device array below
// instead of a handle's work array.
//
// The array is a fixed 16 MiB per GPU that loads the library and lives until the
// process exits.  Every call shares it and it keeps the last call's contents;
// nothing in it needs to start at zero (each call overwrites what it reads).
// Calls that overlap on the GPU (different streams, or threads racing on one
// device) race on the array and on the twiddle tables.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "../../include/openpfc_b200.h"
#include "launch.h"
#include "twiddle.h"

using namespace opfc;

namespace {
constexpr size_t kScratchBytes = size_t(16) << 20;  // intermediate half spectrum
constexpr int kMaxLen = 1024;                       // longest axis with a twiddle table
constexpr int kMaxDevices = 64;
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];
// twiddles of the three axes: x at [0, kMaxLen), y at [kMaxLen, 2 kMaxLen), z after
static __device__ __align__(256) double g_noalloc_twiddles[3 * kMaxLen * 2];

namespace {

struct DeviceSymbols {
  bool ready = false;
  void *scratch = nullptr;
  void *twiddles = nullptr;
};
DeviceSymbols g_dev[kMaxDevices];
std::mutex g_mu;

bool len_ok(int n) {
  static const int ok[] = {1, 2, 4, 8, 16, 24, 32, 40, 48, 64, 80, 96, 128, 256, 512, 1024};
  for (int v : ok)
    if (v == n) return true;
  return false;
}

// Host-side addresses of the file-scope arrays, once per device with that device
// current (in host code the array names are only stand-ins, not device addresses).
int device_symbols(int dev, DeviceSymbols *out) {
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceSymbols &d = g_dev[dev];
  if (!d.ready) {
    if (cudaGetSymbolAddress(&d.scratch, g_noalloc_scratch) != cudaSuccess) {
      cudaGetLastError();
      return OPFC_ERR_CUDA;
    }
    if (cudaGetSymbolAddress(&d.twiddles, g_noalloc_twiddles) != cudaSuccess) {
      cudaGetLastError();
      return OPFC_ERR_CUDA;
    }
    d.ready = true;
  }
  *out = d;
  return OPFC_OK;
}

}  // namespace

extern "C" int opfc_fft_forward_noalloc(const void *in_real, void *out_complex, const int n[3],
                                        int precision, void *stream) {
  if (!in_real || !out_complex || !n) return OPFC_ERR_ARG;
  if (precision != OPFC_FP32 && precision != OPFC_FP64) return OPFC_ERR_ARG;
  const int n0 = n[0], n1 = n[1], n2 = n[2];
  if (n0 < 2 || n0 % 2 != 0 || n1 < 1 || n2 < 1) return OPFC_ERR_SIZE;
  const int M = n0 / 2;
  if (!len_ok(M) || !len_ok(n1) || !len_ok(n2) || n0 > kMaxLen || n1 > kMaxLen || n2 > kMaxLen)
    return OPFC_ERR_SIZE;
  const size_t es = precision == OPFC_FP64 ? 8 : 4;
  const size_t nc = (size_t)(M + 1) * n1 * n2;
  if (nc * 2 * es > kScratchBytes) return OPFC_ERR_SIZE;  // beyond the fixed 16 MiB scratch

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return OPFC_ERR_CUDA;
  }
  DeviceSymbols sym;
  int rc = device_symbols(dev, &sym);
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

  // twiddle tables of the three axes, rounded to the compute precision
  unsigned char *twb = static_cast<unsigned char *>(sym.twiddles);
  const void *tw[3];
  const int lens[3] = {n0, n1, n2};
  for (int a = 0; a < 3; ++a) {
    std::vector<double> d = twiddle_table(lens[a]);
    void *dst = twb + (size_t)a * kMaxLen * 2 * sizeof(double);
    cudaError_t e;
    if (precision == OPFC_FP64) {
      e = cudaMemcpyAsync(dst, d.data(), d.size() * sizeof(double), cudaMemcpyHostToDevice, s);
    } else {
      std::vector<float> f(d.begin(), d.end());
      e = cudaMemcpyAsync(dst, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice, s);
    }
    if (e != cudaSuccess) return OPFC_ERR_CUDA;
    tw[a] = dst;
  }

  void *scratch = sym.scratch;
  const long long nyq_off = (long long)M * n1 * n2;
  const bool f64 = precision == OPFC_FP64;
  const int W = f64 ? 8 : 16;

  // x pass: real rows -> split-layout half spectrum in the scratch array
  XLaunch X{};
  X.M = M;
  X.rows = n1 * n2;
  X.mode = X_R2C;
  X.nyq_off = nyq_off;
  X.rin = in_real;
  X.out = scratch;
  X.tw = tw[0];
  X.scale = 1.0;
  rc = f64 ? launch_x<double>(X, s) : launch_x<float>(X, s);
  if (rc) return OPFC_ERR_CUDA;

  // y and z passes in place on the scratch array (direct-load kernels)
  for (int axis = 1; axis <= 2; ++axis) {
    const int N = axis == 1 ? n1 : n2;
    if (N == 1) continue;
    ColLaunch L{};
    ColSeg &m = L.seg[0];
    ColSeg &q = L.seg[1];
    m.col_stride = 1;
    m.ncols = M;
    m.tiles_inner = (M + W - 1) / W;
    q.off = nyq_off;
    if (axis == 1) {
      m.s_outer = (long long)M * n1;
      m.fft_stride = M;
      m.ntiles = m.tiles_inner * n2;
      q.fft_stride = 1;
      q.col_stride = n1;
      q.ncols = n2;
    } else {
      m.s_outer = M;
      m.fft_stride = (long long)M * n1;
      m.ntiles = m.tiles_inner * n1;
      q.fft_stride = n1;
      q.col_stride = 1;
      q.ncols = n1;
    }
    q.tiles_inner = (q.ncols + W - 1) / W;
    q.ntiles = q.tiles_inner;
    L.nseg = 2;
    L.N = N;
    L.dir = -1;
    L.mode = COL_PLAIN;
    L.nsets = 1;
    L.in[0] = L.in[1] = scratch;
    L.out[0] = L.out[1] = scratch;
    L.tw = tw[axis];
    L.axis = axis;
    rc = f64 ? launch_col<double>(L, s) : launch_col<float>(L, s);
    if (rc) return OPFC_ERR_CUDA;
  }

  // split layout -> reference layout ((N0/2+1) x N1 x N2, interleaved)
  rc = f64 ? launch_to_ref<double>(scratch, out_complex, 1, M, n1, n2, nyq_off, 0, 0.0, s)
           : launch_to_ref<float>(scratch, out_complex, 0, M, n1, n2, nyq_off, 0, 0.0, s);
  return rc ? OPFC_ERR_CUDA : OPFC_OK;
}
