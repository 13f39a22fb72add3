// launch.h -- host-side launch descriptors shared by the C-ABI and the kernels.
//
// Internal k-space layout ("split half spectrum"): for a grid N0 x N1 x N2 with
// M = N0/2, the Nc = (M+1) N1 N2 modes are stored as
//   main[kx + M (ky + N1 kz)]     for kx in [0, M)      (M*N1*N2 elements)
//   nyq [ky + N1 kz]              for kx = M (Nyquist)  (N1*N2 elements)
// in one allocation (nyq right after main).  Every main row is M complex values,
// so tiles of W consecutive kx are aligned, full-width HBM segments; the
// reference layout ((M+1) values per row, fft.cpp:58-70) is produced only at
// the ABI boundary.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace opfc {

// One family of column tiles.  Tile t covers columns [ti*W, ti*W + W) of the
// outer index `to`, with ti = t % tiles_inner and to = t / tiles_inner.
struct ColSeg {
  long long off;         // element offset of outer index 0, column 0
  long long s_outer;     // element stride between outer indices
  long long fft_stride;  // element stride along the transformed axis
  long long col_stride;  // element stride between neighbouring columns
  int tiles_inner;       // tiles per outer index
  int ncols;             // columns per outer index (bounds check)
  int ntiles;            // tiles in this family
  int pad_;
};

enum ColMode { COL_PLAIN = 0, COL_UPDATE = 1 };
// MK_ALUMINUM_G: the Aluminum model with a moving temperature gradient (three
// real fields per step: psi, psi_MF and P*psi; direct-load kernels only)
enum ModelKind { MK_PLAIN = 0, MK_TUNGSTEN = 1, MK_FILTERED = 2, MK_ALUMINUM_G = 3 };

struct ColLaunch {
  int N;        // transform length
  int dir;      // -1 forward, +1 inverse (COL_PLAIN)
  int mode;     // ColMode
  int model;    // ModelKind (COL_UPDATE)
  int nsets;    // 1 or 2 independent arrays (blockIdx.y)
  int inverse_after;  // COL_UPDATE: also write the inverse transform(s)
  ColSeg seg[2];
  int nseg;
  const void *in[2];
  void *out[2];
  const void *tw;     // exp(-2 pi i k / N), N entries, compute precision
  // COL_UPDATE operands (all in the split layout, compute precision)
  void *psi_hat;      // state, updated in place
  const void *tab_a;  // opL / exp_Ldt
  const void *tab_b;  // opN / n_weight
  const void *tab_chi;  // mean-field filter (TUNGSTEN, FILTERED)
  const void *tab_p;    // MK_ALUMINUM_G: the correlation peak P_F
  void *out_p;          // MK_ALUMINUM_G: inverse z transform of P_F psi_hat
  // TMA path (main segment): host CUtensorMap objects, see tma_col_width().
  // PLAIN: tmap[0], tmap[1] = input of array set 0 / 1; UPDATE: A, psi_hat,
  // tab_a, tab_b, tab_chi.  tmap[0] == nullptr selects the direct-load kernel.
  const void *tmap[5];
  // COL_UPDATE on isotropic grids: operators indexed by m = kx^2 + ky^2 + kz^2
  // (folded integer indices) instead of per-mode tables; rad_ops holds (opL, opN)
  // pairs in the compute precision, rad_chi the filter (or nullptr)
  const void *rad_ops;
  const void *rad_chi;
  int rad_M, rad_n1, rad_n2;
  // COL_UPDATE, PLAIN and FILTERED models: operators computed per mode from k^2
  // in the compute precision (no table is read); kf = 2 pi / (dx n) per axis,
  // op_chi = 1 / (2 alpha^2) of the filter (FILTERED).  Uses rad_M/n1/n2.
  int computed;
  double kf[3], op_r, op_dt, op_chi;
  // COL_UPDATE: operators from the folded FP64-built tables (opL, opN pairs and
  // the filter over kx in [0, M], |ky| <= N1/2, |kz| <= N2/2; split layout with
  // the kx = M plane at fold_nyq), the z tiles walked in (ky, N1 - ky) pairs so
  // a table row is read from HBM once per step.  Uses rad_M/n1/n2.
  const void *fold_ops;
  const void *fold_chi;
  long long fold_nyq;
  // COL_PLAIN: half-width tiles (64-byte rows) with two CTAs per SM
  int narrow;
  // ping-pong FFT exchange buffers (one CTA barrier per exchange; one ring
  // stage fewer): COL_PLAIN and the computed-operator update
  int pingpong;
  // COL_PLAIN direct-load kernel with 32 values per thread (N = 512, 1024:
  // one exchange per transform)
  int e32;
  // COL_UPDATE with the folded tables at N = 1024: the box-ring kernel with
  // 128-byte tile rows (tensor maps built for Width<Real>::W columns)
  int wide;
  int axis;            // 1 = y, 2 = z
  unsigned int *flag;  // bit 1: a bounded wait expired
  int num_sms;
};

// Tile width (columns) of the TMA column kernels: 128-byte rows for the plain
// transforms (64-byte rows and half the tile for the narrow variant) and 64-byte
// rows for the fused update (which stages psi_hat and the tables too), capped so
// one tile stays near 64 KB / 32 KB.  Host and device use this one definition.
// The folded-table update stages its table rows as 3 TMA boxes of N/4 rows.
constexpr int tma_col_width(int N, int csize, int mode, bool narrow = false) {
  int w = (mode == COL_PLAIN && !narrow ? 128 : 64) / csize;
  const int cap = (mode == COL_PLAIN && !narrow ? 65536 : 32768) / (N * csize);
  if (cap < w) w = cap;
  return w < 4 ? 4 : w;
}

enum XMode { X_R2C = 0, X_C2R = 1, X_FUSED = 2 };

struct XLaunch {
  int M;           // N0 / 2 (half length of the real transform)
  int rows;        // N1 * N2
  int mode;        // XMode
  int model;       // ModelKind (X_FUSED)
  long long nyq_off;
  const void *in0;   // complex input (split layout)
  const void *in1;   // second complex input (TUNGSTEN psi_MF)
  const void *in2;   // third complex input (MK_ALUMINUM_G: P*psi)
  void *out;         // complex output (split layout)
  const void *rin;   // real rows (X_R2C)
  void *rout;        // real rows (X_C2R)
  const void *tw;    // exp(-2 pi i k / N0), N0 = 2M entries
  double scale;      // C2R normalisation 1/(N0 N1 N2)
  double mean;       // mean density added after the C2R (k = 0 mode in FP64)
  double c[8];       // nonlinearity coefficients
  // MK_ALUMINUM_G: temperature T_var(x, t) = G (dist - x_init - V t) with
  // dist = x + fullruns - (x > steppoint) l, x = x0 + i dx, t read from *time;
  // N = p3b u^2 + p4b u^3 + q21b T/T0 v + (q31b (T_const + T)/T0 + q30b) v^2
  //     + q4b v^3 + (1 - exp(-T/T0)) P*psi - stabP u
  // (the mean of P*psi is P_F(0) times the mean density: PF0)
  double al[18];       // x0 dx l fullruns steppoint G x_init V T0 T_const q21b q30b q31b p3b p4b q4b stabP PF0
  const double *time;
  unsigned int *flag;  // bit 0: a non-finite value was produced; bit 1: a wait expired
  int use_tma;         // X_FUSED: persistent bulk-copy-fed kernel when the size allows
  int no_sq;           // X_FUSED: skip the warp-square kernel (x_sq.cuh) for x_tma.cuh
  int sq_direct;       // X_FUSED: warp-square kernel with rows loaded straight into registers
                       // (1; 2 = the same, loading the next row during the current one)
  int num_sms;
};

// Per-device kernel set-up: the dynamic shared-memory attribute is a property
// of the kernel on one device, so it is applied, and the resident CTAs per SM
// are computed, once per device ordinal (cache[dev]); ordinals beyond the cache
// are set up on every call.  Returns the resident CTAs per SM (>= 1).
constexpr int kDevCache = 64;
template <typename K> inline int kernel_setup(K k, int threads, size_t smem, int (&cache)[kDevCache]) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    dev = -1;
  }
  int *slot = (dev >= 0 && dev < kDevCache) ? &cache[dev] : nullptr;
  if (slot && *slot) return *slot;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, threads, smem) != cudaSuccess || occ < 1) {
    cudaGetLastError();
    occ = 1;
  }
  if (slot) *slot = occ;
  return occ;
}

// The pass kernels' bounded mbarrier wait on a barrier that never completes,
// with a limit of limit_ms (0.1 .. 1000): sets bit 2 of *flag when it expires
// (wait_check.cu).  Returns cudaError_t as int.
int launch_wait_check(unsigned *flag, double limit_ms, cudaStream_t s);

// Kernel launchers (kernels_f32.cu / kernels_f64.cu).  Return cudaError_t as int.
template <typename Real> int launch_col(const ColLaunch &a, cudaStream_t s);
template <typename Real> int launch_x(const XLaunch &a, cudaStream_t s);
// planes: bit 0 the kx = 0 plane, bit 1 the Nyquist plane
template <typename Real>
int launch_herm_fix(void *psi, long long nyq_off, int M, int n1, int n2, cudaStream_t s,
                    double *time = nullptr, double dt_time = 0.0, int planes = 3);
template <typename Real>
int launch_to_ref(const void *in, void *out, int out_is_f64, int M, int n1, int n2,
                  long long nyq_off, int dc_override, double dc_re, cudaStream_t s);
template <typename Real>
int launch_from_ref(const void *in, int in_is_f64, void *out, int M, int n1, int n2,
                    long long nyq_off, cudaStream_t s);
template <typename Real>
int launch_cast_real(const void *in, int in_is_f64, void *out, int out_is_f64, size_t n,
                     cudaStream_t s);
// FP64 partial sums of x (p = 1) or x^4 (p = 4); `partials` holds `nblocks`
// doubles; the host finishes with a compensated sum.
template <typename Real>
int launch_sum_pow(const void *x, size_t n, int p, double *partials, int nblocks, cudaStream_t s);
// FP64 partial sums of w_kx G(k) |psi_hat|^2 with G = r + (1 - k^2)^2.
template <typename Real>
int launch_energy_k(const void *psi_hat, int M, int n1, int n2, long long nyq_off,
                    const double *dx, double r, double *partials, int nblocks, cudaStream_t s);

}  // namespace opfc
