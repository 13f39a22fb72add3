// opfc.cu -- the C ABI (include/openpfc_b200.h): handle life cycle, FP64
// operator tables, field I/O, the step sequence and its CUDA graph.
//
// Step sequence with the state psi_hat resident in k-space (split layout, see
// launch.h) and one work array A that holds F_z^-1[psi_hat] between steps:
//   YI(A) ; X(A: C2R -> N(psi) -> R2C) ; YF(A) ; ZU(A -> psi_hat, A) ; HERM(psi_hat)
// The reference performs the same mathematics as
// F[psi] -> multiply -> F^-1 -> nonlinearity -> F -> ETD combine -> F^-1
// (apps/tungsten/include/tungsten/cpu/tungsten_model.hpp:306-366,
//  docs/api/examples/10_complete_pfc_model.cpp:121-144).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/openpfc_b200.h"
#include "fft_core.cuh"
#include "launch.h"
#include "twiddle.h"
#include "autotune.h"
#include "io.h"

using namespace opfc;

int opfc_scale_by_table(opfc_handle *h, const void *in, const void *tab, void *out);

namespace {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr int kVarY = 5, kVarX = 5, kVarZ = 10;
// z-update variants by how they obtain opL / opN
inline bool z_computed(int v) { return v >= 3 && v <= 5; }  // from k^2 in the compute precision
inline bool z_folded(int v) { return v >= 6 && v <= 9; }    // folded FP64-built tables
inline bool z_direct(int v) { return v == 2 || v == 4 || v == 7; }
// OPFC_FP32_COMPUTED_OPERATORS=1 lets FP32 handles use (and tune) the update
// variants that compute opL / opN per mode in FP32 (expm1f, fast divide)
// instead of reading FP64-built tables rounded to FP32.
inline bool computed_ops_allowed() {
  const char *e = std::getenv("OPFC_FP32_COMPUTED_OPERATORS");
  return e && e[0] == '1';
}
// models with two real fields per step (psi and psi_MF): Tungsten, Aluminum
inline bool two_field(int model) { return model == OPFC_MODEL_TUNGSTEN || model == OPFC_MODEL_ALUMINUM; }
// operator tables supplied by the caller (opfc_set_operators), filtered-model passes
inline bool user_ops_model(int model) { return model == OPFC_MODEL_USER_ETD; }  // kernel variants per pass (opfc_autotune)

bool supported_len(int n) {
  static const int ok[] = {1, 2, 4, 8, 16, 24, 32, 40, 48, 64, 80, 96, 128, 256, 512, 1024};
  for (int v : ok)
    if (v == n) return true;
  return false;
}

void unit_root(long k, long n, double *c, double *s) { unit_root_host(k, n, c, s); }

double neumaier(const double *a, size_t n) {
  double s = 0, c = 0;
  for (size_t i = 0; i < n; ++i) {
    const double t = s + a[i];
    if (std::fabs(s) >= std::fabs(a[i]))
      c += (s - t) + a[i];
    else
      c += (a[i] - t) + s;
    s = t;
  }
  return s + c;
}

template <typename F> void parallel_for(long n, F &&f) {
  unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  if ((long)nt > n) nt = (unsigned)std::max(1L, n);
  std::vector<std::thread> th;
  const long chunk = (n + nt - 1) / nt;
  for (unsigned t = 0; t < nt; ++t) {
    const long lo = t * chunk, hi = std::min(n, lo + chunk);
    if (lo >= hi) break;
    th.emplace_back([lo, hi, &f] {
      for (long i = lo; i < hi; ++i) f(i);
    });
  }
  for (auto &x : th) x.join();
}

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

}  // namespace

struct opfc_handle {
  opfc_desc desc{};
  int n0 = 0, n1 = 0, n2 = 0, M = 0;
  // the whole grid this handle is a slab of (its own n otherwise) and the
  // global index of its first half-spectrum column
  int g0 = 0, g1 = 0, g2 = 0, kx0 = 0;
  bool slab = false;
  // opfc_pass: the mean density the x pass adds (the whole grid's, for a slab)
  bool use_pass_mean = false;
  double pass_mean = 0.0;
  size_t nr = 0, nc = 0;
  long long nyq_off = 0;
  int prec = OPFC_FP32;
  size_t rsz = 4;  // bytes per real in compute precision
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = 0;

  void *psi_hat = nullptr;   // state (split layout, DC slot kept at zero)
  void *work_a = nullptr;    // F_z^-1 of the state, then the step's working array
  void *work_b = nullptr;    // TUNGSTEN: F_z^-1 of chi * state
  void *tab_a = nullptr, *tab_b = nullptr, *tab_chi = nullptr;
  // Aluminum with a moving temperature gradient (G_grid != 0): the peak table
  // P_F, F_z^-1[P_F psi_hat] between steps, and the device time of the next
  // step (advanced by time_dt at the end of every step)
  bool al_grad = false;
  bool user_ops = false;  // OPFC_MODEL_USER_ETD: tables set by opfc_set_operators
  void *tab_p = nullptr, *work_c = nullptr;
  double *time_dev = nullptr;
  double time_dt = 0.0, pf0 = 0.0;
  void *tw_x = nullptr, *tw_y = nullptr, *tw_z = nullptr;
  void *real_buf = nullptr;  // real-space staging (N0 N1 N2 reals)
  unsigned int *flag = nullptr;
  double *partials = nullptr;
  int npartials = 1184;
  size_t allocated = 0;

  double mass_sum = 0.0;  // sum over cells of psi (the k = 0 mode), FP64
  bool initialized = false;
  bool have_state = false;
  bool a_valid = false;
  double dt = 0.0;

  // adjoint of the plain model: state snapshots every K steps of the last
  // checkpointed forward run, the r-derivatives of the tables, and work arrays
  std::vector<void *> ckpt;  // psi_hat at steps 0, K, 2K, ... and the final state
  int ckpt_K = 0, ckpt_steps = 0;
  std::vector<void *> seg;   // psi_hat of each step of one recomputed segment
  void *tab_ar = nullptr, *tab_br = nullptr;
  // isotropic grids: (opL, opN) and the filter as functions of m = |k_index|^2
  void *rad_ops = nullptr, *rad_chi = nullptr;
  // every grid: (opL, opN) pairs and the filter over (kx, |ky|, |kz|), the
  // FP64-built per-mode tables folded by the evenness of k^2 in ky and kz
  void *fold_ops = nullptr, *fold_chi = nullptr;
  long long fold_nyq = 0;
  void *adj_c[2] = {nullptr, nullptr};
  void *adj_r[4] = {nullptr, nullptr, nullptr, nullptr};

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;

  bool use_tma = true;  // TMA-fed column passes (OPFC_NO_TMA=1 disables)
  // OPFC_NVTX=1: steps run eagerly (no CUDA graph) with one NVTX range per
  // kernel named after the reference's profiling regions
  bool nvtx = false;
  // kernel variants per pass, chosen by the autotuner (see opfc_autotune):
  // var_y: 0 pipelined, 1 direct, 2 pipelined narrow tiles (two CTAs per SM),
  //        3 pipelined with ping-pong exchange buffers, 4 direct with 32
  //        values per thread (one exchange per transform at N = 512, 1024);
  // var_x: 0 pipelined (warp-square kernel where it applies), 1 direct,
  //        2 pipelined without the warp-square kernel, 3 warp-square kernel
  //        with rows loaded straight into registers (PLAIN, FILTERED), 4 as 3
  //        loading the next row while the current one is transformed;
  // var_z: 0 pipelined with streamed tables, 1 pipelined with radial tables,
  //        2 direct with streamed tables, 3 pipelined with computed operators,
  //        4 direct with computed operators, 5 as 3 with ping-pong exchange
  //        buffers (3-5: PLAIN and FILTERED), 6 pipelined with the folded
  //        tables and ping-pong exchange buffers, 7 direct with the folded
  //        tables, 8 pipelined with the folded tables, 9 box-ring kernel with
  //        the folded tables and 128-byte rows (z length 1024, PLAIN and
  //        FILTERED; else as 7)
  int var_y = 0, var_x = 0, var_z = 0;
  int num_sms = 148;
  struct Tmap {
    const void *ptr;
    int axis, W, real;
    CUtensorMap map;
  };
  std::vector<Tmap> tmaps;
  std::string err;
};

namespace {

int fail(opfc_handle *h, int code, const char *fmt, ...) {
  if (h) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    h->err = buf;
  }
  return code;
}

#define CUDA_TRY(h, expr)                                                                 \
  do {                                                                                    \
    cudaError_t e_ = (expr);                                                              \
    if (e_ != cudaSuccess) return fail(h, OPFC_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
  } while (0)

#define LAUNCH_TRY(h, expr)                                                                \
  do {                                                                                     \
    int e_ = (expr);                                                                       \
    if (e_ != 0)                                                                           \
      return fail(h, OPFC_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString((cudaError_t)e_)); \
  } while (0)

int dev_alloc(opfc_handle *h, void **p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(h, OPFC_ERR_OOM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
  }
  h->allocated += bytes;
  return OPFC_OK;
}

int upload_twiddles(opfc_handle *h, int n, void **dst) {
  std::vector<double> d(2 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    double c, s;
    unit_root(k, n, &c, &s);
    d[2 * k] = c;
    d[2 * k + 1] = -s;
  }
  int rc = dev_alloc(h, dst, (size_t)n * 2 * h->rsz);
  if (rc) return rc;
  if (h->prec == OPFC_FP64) {
    CUDA_TRY(h, cudaMemcpy(*dst, d.data(), d.size() * sizeof(double), cudaMemcpyHostToDevice));
  } else {
    std::vector<float> f(d.begin(), d.end());
    CUDA_TRY(h, cudaMemcpy(*dst, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  return OPFC_OK;
}

// split-layout index of reference mode (kx, ky, kz)
inline size_t split_index(const opfc_handle *h, int kx, int ky, int kz) {
  const size_t row = (size_t)ky + (size_t)h->n1 * (size_t)kz;
  return kx < h->M ? (size_t)kx + (size_t)h->M * row : (size_t)h->nyq_off + row;
}

// Column-pass segments along y (axis 1) or z (axis 2), see launch.h.
void col_segments(const opfc_handle *h, int axis, ColLaunch &L) {
  const int W = (h->prec == OPFC_FP64) ? 8 : 16;
  const int M = h->M, n1 = h->n1, n2 = h->n2;
  ColSeg &a = L.seg[0];
  ColSeg &b = L.seg[1];
  a = ColSeg{};
  b = ColSeg{};
  a.col_stride = 1;
  a.ncols = M;
  a.tiles_inner = (M + W - 1) / W;
  if (axis == 1) {
    a.off = 0;
    a.s_outer = (long long)M * n1;
    a.fft_stride = M;
    a.ntiles = a.tiles_inner * n2;
    // Nyquist plane: y lines are contiguous, columns are the z index
    b.off = h->nyq_off;
    b.s_outer = 0;
    b.fft_stride = 1;
    b.col_stride = n1;
    b.ncols = n2;
    b.tiles_inner = (n2 + W - 1) / W;
    b.ntiles = b.tiles_inner;
  } else {
    a.off = 0;
    a.s_outer = M;
    a.fft_stride = (long long)M * n1;
    a.ntiles = a.tiles_inner * n1;
    b.off = h->nyq_off;
    b.s_outer = 0;
    b.fft_stride = n1;
    b.col_stride = 1;
    b.ncols = n1;
    b.tiles_inner = (n1 + W - 1) / W;
    b.ntiles = b.tiles_inner;
  }
  L.nseg = 2;
  L.N = (axis == 1) ? n1 : n2;
}

int col(opfc_handle *h, ColLaunch L) {
  L.flag = h->flag;
  L.num_sms = h->num_sms;
  return h->prec == OPFC_FP64 ? launch_col<double>(L, h->stream) : launch_col<float>(L, h->stream);
}
int xpass(opfc_handle *h, const XLaunch &L) {
  return h->prec == OPFC_FP64 ? launch_x<double>(L, h->stream) : launch_x<float>(L, h->stream);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                   const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                   const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    else
      cudaGetLastError();
  }
  return fn;
}

// Tensor map of a split-layout array's main part viewed as scalars
// [N2][N1][S*M] (S = 2 for complex, 1 for real tables), box = W columns x
// min(N, 256) rows of `axis`.  Cached per (pointer, axis, W, real).
const CUtensorMap *tmap_for(opfc_handle *h, const void *ptr, int axis, int W, bool real);

// plain batched transform along y/z, in place (in == out) or out of place
int col_plain(opfc_handle *h, int axis, int dir, const void *in0, void *out0,
              const void *in1 = nullptr, void *out1 = nullptr) {
  ColLaunch L{};
  col_segments(h, axis, L);
  L.dir = dir;
  L.mode = COL_PLAIN;
  L.nsets = in1 ? 2 : 1;
  L.in[0] = in0;
  L.out[0] = out0;
  L.in[1] = in1 ? in1 : in0;
  L.out[1] = out1 ? out1 : out0;
  L.tw = axis == 1 ? h->tw_y : h->tw_z;
  L.axis = axis;
  L.narrow = h->var_y == 2;
  L.pingpong = h->var_y == 3;
  L.e32 = h->var_y == 4;
  const int W = tma_col_width(L.N, 2 * (int)h->rsz, COL_PLAIN, L.narrow);
  if (h->use_tma && h->var_y != 1 && h->var_y != 4 && L.N > 1 && h->M % W == 0) {
    L.tmap[0] = tmap_for(h, in0, axis, W, false);
    L.tmap[1] = in1 ? tmap_for(h, in1, axis, W, false) : nullptr;
    if (in1 && !L.tmap[1]) L.tmap[0] = nullptr;
  }
  return col(h, L);
}

const CUtensorMap *tmap_for(opfc_handle *h, const void *ptr, int axis, int W, bool real) {
  if (!ptr) return nullptr;
  for (const auto &t : h->tmaps)
    if (t.ptr == ptr && t.axis == axis && t.W == W && t.real == (int)real) return &t.map;
  EncodeTiledFn enc = encode_fn();
  // returned pointers must stay valid while a launch is assembled: never grow
  if (!enc || h->tmaps.size() == h->tmaps.capacity()) return nullptr;
  const cuuint64_t es = h->rsz, S = real ? 1 : 2;
  const int N = axis == 1 ? h->n1 : h->n2;
  const cuuint32_t RB = (cuuint32_t)std::min(N, 256);
  cuuint64_t dims[3] = {S * (cuuint64_t)h->M, (cuuint64_t)h->n1, (cuuint64_t)h->n2};
  cuuint64_t strides[2] = {S * h->M * es, S * h->M * (cuuint64_t)h->n1 * es};
  cuuint32_t box[3] = {(cuuint32_t)(S * W), axis == 1 ? RB : 1u, axis == 1 ? 1u : RB};
  cuuint32_t estr[3] = {1, 1, 1};
  opfc_handle::Tmap t{};
  t.ptr = ptr;
  t.axis = axis;
  t.W = W;
  t.real = (int)real;
  const CUresult r = enc(&t.map, es == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                         3, const_cast<void *>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE,
                         // full 128-byte rows may pull in the neighbouring tile's
                         // row; narrower rows (the update's 64/32-byte rows) fetch
                         // only what they use
                         S * W * es >= 128 ? CU_TENSOR_MAP_L2_PROMOTION_L2_256B
                                           : CU_TENSOR_MAP_L2_PROMOTION_NONE,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return nullptr;
  h->tmaps.push_back(t);
  return &h->tmaps.back().map;
}

// Tensor map of a folded table ((M+1) x (N1/2+1) x (N2/2+1) modes in the split
// layout, main part [N2/2+1][N1/2+1][S*M], S = 2 for (opL, opN) pairs, 1 for the
// filter), box = W columns x 1 x N2/4 rows of |kz| (3 boxes cover |kz| <= N2/2).
const CUtensorMap *tmap_fold(opfc_handle *h, const void *ptr, int W, bool pairs) {
  if (!ptr || h->n2 % 16 != 0) return nullptr;
  const int axis = pairs ? 3 : 4;  // cache keys apart from the full arrays' maps
  for (const auto &t : h->tmaps)
    if (t.ptr == ptr && t.axis == axis && t.W == W) return &t.map;
  EncodeTiledFn enc = encode_fn();
  if (!enc || h->tmaps.size() == h->tmaps.capacity()) return nullptr;
  const cuuint64_t es = h->rsz, S = pairs ? 2 : 1;
  const cuuint64_t F1 = h->n1 / 2 + 1, F2 = h->n2 / 2 + 1;
  cuuint64_t dims[3] = {S * (cuuint64_t)h->M, F1, F2};
  cuuint64_t strides[2] = {S * h->M * es, S * h->M * F1 * es};
  cuuint32_t box[3] = {(cuuint32_t)(S * W), 1u, (cuuint32_t)(h->n2 / 4)};
  cuuint32_t estr[3] = {1, 1, 1};
  opfc_handle::Tmap t{};
  t.ptr = ptr;
  t.axis = axis;
  t.W = W;
  t.real = pairs ? 0 : 1;
  const CUresult r = enc(&t.map, es == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                         3, const_cast<void *>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return nullptr;
  h->tmaps.push_back(t);
  return &h->tmaps.back().map;
}

XLaunch x_base(opfc_handle *h) {
  XLaunch L{};
  L.M = h->M;
  L.rows = h->n1 * h->n2;
  L.nyq_off = h->nyq_off;
  L.tw = h->tw_x;
  L.scale = 1.0 / ((double)h->g0 * h->g1 * h->g2);
  L.mean = 0.0;
  L.flag = h->flag;
  L.use_tma = h->use_tma && h->var_x != 1;
  L.no_sq = h->var_x == 2;
  L.sq_direct = h->var_x == 3 ? 1 : (h->var_x == 4 ? 2 : 0);
  L.num_sms = h->num_sms;
  return L;
}

double mean_density(const opfc_handle *h) { return h->mass_sum / (double)h->nr; }

// autotuner cache key of one pass of this handle's step
std::string tune_key(const opfc_handle *h, const char *pass) {
  static const char *models[] = {"plain", "tungsten", "filtered", "aluminum", "user_etd"};
  static_assert(sizeof(models) / sizeof(models[0]) == OPFC_MODEL_USER_ETD + 1, "a name per model");
  char b[160];
  std::snprintf(b, sizeof b, "step/%s/%s/%dx%dx%d/%s/f%s", h->prec == OPFC_FP64 ? "fp64" : "fp32",
                models[h->desc.model], h->n0, h->n1, h->n2, pass,
                (h->desc.dx[0] == h->desc.dx[1] && h->desc.dx[1] == h->desc.dx[2]) ? "iso" : "aniso");
  return b;
}

// A <- F_z^-1[psi_hat] (and, for TUNGSTEN, B <- F_z^-1[chi psi_hat]); FILTERED
// keeps only the filtered density in A.
int prepare_a(opfc_handle *h) {
  const int model = h->desc.model;
  if (model == OPFC_MODEL_PLAIN) {
    LAUNCH_TRY(h, col_plain(h, 2, +1, h->psi_hat, h->work_a));
  } else {
    ColLaunch L{};
    col_segments(h, 2, L);
    L.mode = COL_PLAIN;
    L.dir = +1;
    L.nsets = 1;
    // psi part (two-field models) in A
    if (two_field(model)) {
      L.in[0] = h->psi_hat;
      L.out[0] = h->work_a;
      L.in[1] = h->psi_hat;
      L.out[1] = h->work_a;
      L.tw = h->tw_z;
      LAUNCH_TRY(h, col(h, L));
    }
    // chi * psi_hat -> scratch, then inverse z
    void *dst = two_field(model) ? h->work_b : h->work_a;
    int rc = opfc_scale_by_table(h, h->psi_hat, h->tab_chi, dst);
    if (rc) return rc;
    LAUNCH_TRY(h, col_plain(h, 2, +1, dst, dst));
    if (h->al_grad) {  // P_F psi_hat -> C
      if ((rc = opfc_scale_by_table(h, h->psi_hat, h->tab_p, h->work_c))) return rc;
      LAUNCH_TRY(h, col_plain(h, 2, +1, h->work_c, h->work_c));
    }
  }
  h->a_valid = true;
  return OPFC_OK;
}

// Number of kernels one step launches (YI, X, YF, ZU, HERM).
constexpr int kStepKernels = 5;
const char *const kStepKernelNames[kStepKernels] = {"y_inverse", "x_fused", "y_forward",
                                                     "z_update", "hermitian_fix"};
// NVTX range of each step kernel, named after the profiling regions of the
// reference's step (OPENPFC_PROFILE, apps/tungsten/include/tungsten/cpu/
// tungsten_model.hpp:313-362) whose work the kernel does, with the pass in brackets.
const char *const kStepRegions[kStepKernels] = {
    "gradient/mean_field/backward [y inverse]",
    "gradient/mean_field/backward + nonlinear + gradient/evolve/forward [x: C2R, N, R2C]",
    "gradient/evolve/forward [y forward]",
    "gradient/evolve/forward + multiply + backward [z forward, ETD combine, z inverse]",
    "gradient/evolve/multiply [Hermitian projection]"};

// nvtxRangePushA / nvtxRangePop around a scope (a no-op without an NVTX tool)
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

int enqueue_step_kernels(opfc_handle *h, int only);

// Enqueue the step's kernels on h->stream; `only` >= 0 enqueues that one
// kernel.  With NVTX ranges on (eager steps, opfc_profile_step) each kernel is
// enqueued inside the range of its reference region.
int enqueue_step(opfc_handle *h, int only = -1) {
  if (!h->nvtx) return enqueue_step_kernels(h, only);
  for (int k = 0; k < kStepKernels; ++k) {
    if (only >= 0 && k != only) continue;
    NvtxRange range(kStepRegions[k]);
    const int rc = enqueue_step_kernels(h, k);
    if (rc) return rc;
  }
  return OPFC_OK;
}

int enqueue_step_kernels(opfc_handle *h, int only) {
  const int model = h->desc.model;
  if (only < 0 || only == 0) {  // YI
    if (two_field(model)) {
      LAUNCH_TRY(h, col_plain(h, 1, +1, h->work_a, h->work_a, h->work_b, h->work_b));
      if (h->al_grad) LAUNCH_TRY(h, col_plain(h, 1, +1, h->work_c, h->work_c));
    } else {
      LAUNCH_TRY(h, col_plain(h, 1, +1, h->work_a, h->work_a));
    }
  }
  if (only < 0 || only == 1) {  // X
    XLaunch X = x_base(h);
    X.mode = X_FUSED;
    X.in0 = h->work_a;
    X.out = h->work_a;
    X.mean = h->use_pass_mean ? h->pass_mean : mean_density(h);
    if (model == OPFC_MODEL_PLAIN) {
      X.model = MK_PLAIN;
    } else if (model == OPFC_MODEL_FILTERED || user_ops_model(model)) {
      X.model = MK_FILTERED;
      X.c[0] = h->desc.p2 / 2.0;
      X.c[1] = h->desc.p3 / 3.0;
      X.c[2] = h->desc.p4 / 4.0;
    } else if (model == OPFC_MODEL_ALUMINUM) {
      // Aluminum.hpp:285-307 with the temperature offset T_var = 0 (G_grid = 0):
      // N = p3_bar u^2 + p4_bar u^3 + q3 v^2 + q4_bar v^3 - stabP u,
      // q3 = q31_bar T_const / T0 + q30_bar
      X.model = MK_TUNGSTEN;
      X.in1 = h->work_b;
      const opfc_aluminum_params &p = h->desc.aluminum;
      X.c[0] = p.p3_bar;
      X.c[1] = p.p4_bar;
      X.c[2] = p.q31_bar * p.T_const / p.T0 + p.q30_bar;
      X.c[3] = p.q4_bar;
      X.c[4] = p.stabP;
      if (h->al_grad) {
        // moving temperature: position- and time-dependent terms, third field
        // P*psi (Aluminum.hpp:270-307); direct-load x kernel
        X.model = MK_ALUMINUM_G;
        X.in2 = h->work_c;
        X.time = h->time_dev;
        const double l = h->n0 * h->desc.dx[0];
        const double al[18] = {h->desc.origin[0], h->desc.dx[0], l, std::floor(p.m_xpos / l) * l,
                               std::fmod(p.m_xpos, l), p.G_grid, p.x_initial, p.V_grid, p.T0, p.T_const,
                               p.q21_bar, p.q30_bar, p.q31_bar, p.p3_bar, p.p4_bar, p.q4_bar, p.stabP, h->pf0};
        for (int i = 0; i < 18; ++i) X.al[i] = al[i];
      }
    } else {
      X.model = MK_TUNGSTEN;
      X.in1 = h->work_b;
      const opfc_tungsten_params &p = h->desc.tungsten;
      const double tau = p.T / p.T0;
      const double p3b = p.shift_u * (p.p3 + 3 * p.shift_s * p.p4);
      const double p4b = std::pow(p.shift_u, 2) * p.p4;
      const double q30b = p.shift_u * (p.q30 + 3.0 * p.shift_s * p.q40);
      const double q31b = p.shift_u * p.q31;
      const double q40b = std::pow(p.shift_u, 2) * p.q40;
      X.c[0] = p3b;
      X.c[1] = p4b;
      X.c[2] = q31b * tau + q30b;
      X.c[3] = q40b;
      X.c[4] = p.stabP;
    }
    LAUNCH_TRY(h, xpass(h, X));
  }
  if (only < 0 || only == 2)  // YF
    LAUNCH_TRY(h, col_plain(h, 1, -1, h->work_a, h->work_a));
  if (only < 0 || only == 3) {  // ZU
    ColLaunch Z{};
    col_segments(h, 2, Z);
    Z.mode = COL_UPDATE;
    Z.model = model == OPFC_MODEL_PLAIN ? MK_PLAIN : (two_field(model) ? MK_TUNGSTEN : MK_FILTERED);
    if (h->al_grad) {  // three inverse transforms; direct-load kernel with per-mode tables
      Z.model = MK_ALUMINUM_G;
      Z.tab_p = h->tab_p;
      Z.out_p = h->work_c;
    }
    Z.inverse_after = 1;
    Z.nsets = 1;
    Z.in[0] = h->work_a;
    Z.out[0] = h->work_a;
    Z.in[1] = h->work_b;
    Z.out[1] = h->work_b;
    Z.tw = h->tw_z;
    Z.psi_hat = h->psi_hat;
    Z.tab_a = h->tab_a;
    Z.tab_b = h->tab_b;
    Z.tab_chi = h->tab_chi;
    Z.axis = 2;
    // computed operators (variants 3-5): PLAIN and FILTERED models
    Z.computed = z_computed(h->var_z) && !two_field(model) && !user_ops_model(model);
    Z.pingpong = h->var_z == 5 || h->var_z == 6;
    if (z_folded(h->var_z) && h->fold_ops) {
      Z.fold_ops = h->fold_ops;
      Z.fold_chi = h->fold_chi;
      Z.fold_nyq = h->fold_nyq;
    }
    Z.rad_M = h->M;
    Z.rad_n1 = h->n1;
    Z.rad_n2 = h->n2;
    const int nn[3] = {h->n0, h->n1, h->n2};
    for (int a = 0; a < 3; ++a) Z.kf[a] = 2.0 * kPi / (h->desc.dx[a] * nn[a]);
    Z.op_r = h->desc.r;
    Z.op_dt = h->dt;
    Z.op_chi = model == OPFC_MODEL_FILTERED ? 1.0 / (2.0 * h->desc.filter_alpha * h->desc.filter_alpha) : 0.0;
    // variant 9: 128-byte rows (the box-ring kernel's tensor maps)
    Z.wide = h->var_z == 9 && Z.fold_ops && !h->al_grad;
    const int W = Z.wide ? 128 / (2 * (int)h->rsz) : tma_col_width(Z.N, 2 * (int)h->rsz, COL_UPDATE);
    if (h->use_tma && !h->al_grad && !z_direct(h->var_z) && Z.N > 1 && h->M % W == 0) {
      Z.tmap[0] = tmap_for(h, h->work_a, 2, W, false);
      Z.tmap[1] = tmap_for(h, h->psi_hat, 2, W, false);
      if (Z.computed) {
        if (!Z.tmap[1]) Z.tmap[0] = nullptr;
      } else if (Z.fold_ops) {
        Z.tmap[2] = tmap_fold(h, h->fold_ops, W, true);
        Z.tmap[3] = h->fold_chi ? tmap_fold(h, h->fold_chi, W, false) : nullptr;
        if (!Z.tmap[1] || !Z.tmap[2] || (h->fold_chi && !Z.tmap[3])) Z.tmap[0] = nullptr;
      } else if (h->rad_ops && h->var_z == 1) {
        // isotropic grid: operators from the L2-resident radial tables
        Z.rad_ops = h->rad_ops;
        Z.rad_chi = h->rad_chi;
        Z.rad_M = h->M;
        Z.rad_n1 = h->n1;
        Z.rad_n2 = h->n2;
        if (!Z.tmap[1]) Z.tmap[0] = nullptr;
      } else {
        Z.tmap[2] = tmap_for(h, h->tab_a, 2, W, true);
        Z.tmap[3] = tmap_for(h, h->tab_b, 2, W, true);
        Z.tmap[4] = h->tab_chi ? tmap_for(h, h->tab_chi, 2, W, true) : nullptr;
        if (!Z.tmap[1] || !Z.tmap[2] || !Z.tmap[3] || (h->tab_chi && !Z.tmap[4])) Z.tmap[0] = nullptr;
      }
    }
    LAUNCH_TRY(h, col(h, Z));
  }
  if (only < 0 || only == 4) {  // Hermitian projection of the kx = 0 / Nyquist planes
    if (h->prec == OPFC_FP64)
      LAUNCH_TRY(h, launch_herm_fix<double>(h->psi_hat, h->nyq_off, h->M, h->n1, h->n2, h->stream,
                                            h->time_dev, h->time_dt));
    else
      LAUNCH_TRY(h, launch_herm_fix<float>(h->psi_hat, h->nyq_off, h->M, h->n1, h->n2, h->stream,
                                           h->time_dev, h->time_dt));
  }
  return OPFC_OK;
}

void release_graph(opfc_handle *h) {
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->graph_exec = nullptr;
  h->graph = nullptr;
}

int build_graph(opfc_handle *h) {
  release_graph(h);
  CUDA_TRY(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_step(h);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail(h, OPFC_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  h->graph = g;
  e = cudaGraphInstantiate(&h->graph_exec, g, 0);
  if (e != cudaSuccess) {
    release_graph(h);
    return fail(h, OPFC_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  }
  return OPFC_OK;
}

int ensure_real_buf(opfc_handle *h) {
  if (h->real_buf) return OPFC_OK;
  return dev_alloc(h, &h->real_buf, h->nr * h->rsz);
}

int check_count(opfc_handle *h, size_t count, size_t expect, const char *what) {
  if (count != expect)
    return fail(h, OPFC_ERR_SIZE, "%s: expected %zu elements, got %zu", what, expect, count);
  return OPFC_OK;
}

int check_dtype_where(opfc_handle *h, int dtype, int where) {
  if (dtype != OPFC_F32 && dtype != OPFC_F64) return fail(h, OPFC_ERR_ARG, "bad dtype %d", dtype);
  if (where != OPFC_HOST && where != OPFC_DEVICE) return fail(h, OPFC_ERR_ARG, "bad location %d", where);
  return OPFC_OK;
}

// copy a user real field (any dtype, host or device) into real_buf
int real_in(opfc_handle *h, const void *src, int dtype, int where) {
  int rc = ensure_real_buf(h);
  if (rc) return rc;
  const bool same = (dtype == OPFC_F64) == (h->prec == OPFC_FP64);
  if (where == OPFC_HOST) {
    if (same) {
      CUDA_TRY(h, cudaMemcpyAsync(h->real_buf, src, h->nr * h->rsz, cudaMemcpyHostToDevice, h->stream));
    } else if (h->prec == OPFC_FP64) {
      std::vector<double> tmp(h->nr);
      const float *f = (const float *)src;
      for (size_t i = 0; i < h->nr; ++i) tmp[i] = f[i];
      CUDA_TRY(h, cudaMemcpyAsync(h->real_buf, tmp.data(), h->nr * 8, cudaMemcpyHostToDevice, h->stream));
      CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    } else {
      std::vector<float> tmp(h->nr);
      const double *d = (const double *)src;
      for (size_t i = 0; i < h->nr; ++i) tmp[i] = (float)d[i];
      CUDA_TRY(h, cudaMemcpyAsync(h->real_buf, tmp.data(), h->nr * 4, cudaMemcpyHostToDevice, h->stream));
      CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    }
  } else {
    if (same) {
      CUDA_TRY(h, cudaMemcpyAsync(h->real_buf, src, h->nr * h->rsz, cudaMemcpyDeviceToDevice, h->stream));
    } else if (h->prec == OPFC_FP64) {
      LAUNCH_TRY(h, launch_cast_real<double>(src, 0, h->real_buf, 1, h->nr, h->stream));
    } else {
      LAUNCH_TRY(h, launch_cast_real<float>(src, 1, h->real_buf, 0, h->nr, h->stream));
    }
  }
  return OPFC_OK;
}

// copy real_buf out to a user buffer
int real_out(opfc_handle *h, void *dst, int dtype, int where) {
  const bool same = (dtype == OPFC_F64) == (h->prec == OPFC_FP64);
  if (where == OPFC_HOST) {
    if (same) {
      CUDA_TRY(h, cudaMemcpyAsync(dst, h->real_buf, h->nr * h->rsz, cudaMemcpyDeviceToHost, h->stream));
      CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    } else if (h->prec == OPFC_FP64) {
      std::vector<double> tmp(h->nr);
      CUDA_TRY(h, cudaMemcpyAsync(tmp.data(), h->real_buf, h->nr * 8, cudaMemcpyDeviceToHost, h->stream));
      CUDA_TRY(h, cudaStreamSynchronize(h->stream));
      float *f = (float *)dst;
      for (size_t i = 0; i < h->nr; ++i) f[i] = (float)tmp[i];
    } else {
      std::vector<float> tmp(h->nr);
      CUDA_TRY(h, cudaMemcpyAsync(tmp.data(), h->real_buf, h->nr * 4, cudaMemcpyDeviceToHost, h->stream));
      CUDA_TRY(h, cudaStreamSynchronize(h->stream));
      double *d = (double *)dst;
      for (size_t i = 0; i < h->nr; ++i) d[i] = tmp[i];
    }
  } else {
    if (same) {
      CUDA_TRY(h, cudaMemcpyAsync(dst, h->real_buf, h->nr * h->rsz, cudaMemcpyDeviceToDevice, h->stream));
    } else if (h->prec == OPFC_FP64) {
      LAUNCH_TRY(h, launch_cast_real<double>(h->real_buf, 1, dst, 0, h->nr, h->stream));
    } else {
      LAUNCH_TRY(h, launch_cast_real<float>(h->real_buf, 0, dst, 1, h->nr, h->stream));
    }
  }
  return OPFC_OK;
}

// compensated FP64 sum of real_buf (p = 1) or of real_buf^4 (p = 4)
int device_sum(opfc_handle *h, int p, double *out) {
  if (h->prec == OPFC_FP64)
    LAUNCH_TRY(h, launch_sum_pow<double>(h->real_buf, h->nr, p, h->partials, h->npartials, h->stream));
  else
    LAUNCH_TRY(h, launch_sum_pow<float>(h->real_buf, h->nr, p, h->partials, h->npartials, h->stream));
  std::vector<double> part(h->npartials);
  CUDA_TRY(h, cudaMemcpyAsync(part.data(), h->partials, sizeof(double) * h->npartials,
                              cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  *out = neumaier(part.data(), part.size());
  return OPFC_OK;
}

// Compensated FP64 sum of a user field (host: threaded Neumaier chunks
// combined with Neumaier; device: the FP64 reduction kernel in the field's dtype).
int user_sum(opfc_handle *h, const void *src, int dtype, int where, double *out) {
  if (where == OPFC_DEVICE) {
    if (dtype == OPFC_F64)
      LAUNCH_TRY(h, launch_sum_pow<double>(src, h->nr, 1, h->partials, h->npartials, h->stream));
    else
      LAUNCH_TRY(h, launch_sum_pow<float>(src, h->nr, 1, h->partials, h->npartials, h->stream));
    std::vector<double> part(h->npartials);
    CUDA_TRY(h, cudaMemcpyAsync(part.data(), h->partials, sizeof(double) * h->npartials,
                                cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    *out = neumaier(part.data(), part.size());
    return OPFC_OK;
  }
  const long nchunk = 64;
  const size_t len = (h->nr + nchunk - 1) / nchunk;
  std::vector<double> part(nchunk, 0.0);
  parallel_for(nchunk, [&](long c) {
    const size_t lo = (size_t)c * len, hi = std::min(h->nr, lo + len);
    double s = 0, comp = 0;
    for (size_t i = lo; i < hi; ++i) {
      const double v = dtype == OPFC_F64 ? ((const double *)src)[i] : (double)((const float *)src)[i];
      const double t = s + v;
      comp += (std::fabs(s) >= std::fabs(v)) ? (s - t) + v : (v - t) + s;
      s = t;
    }
    part[c] = s + comp;
  });
  *out = neumaier(part.data(), part.size());
  return OPFC_OK;
}

// real_buf -> work_a (forward R2C, full spectrum in the split layout)
int forward_real_buf(opfc_handle *h, void *dst) {
  XLaunch X = x_base(h);
  X.mode = X_R2C;
  X.rin = h->real_buf;
  X.out = dst;
  LAUNCH_TRY(h, xpass(h, X));
  LAUNCH_TRY(h, col_plain(h, 1, -1, dst, dst));
  LAUNCH_TRY(h, col_plain(h, 2, -1, dst, dst));
  return OPFC_OK;
}

// src (split layout spectrum, z and y not yet inverted) -> real_buf, scaled, + mean
int backward_to_real_buf(opfc_handle *h, void *src, double mean, bool z_done) {
  if (!z_done) LAUNCH_TRY(h, col_plain(h, 2, +1, src, src));
  LAUNCH_TRY(h, col_plain(h, 1, +1, src, src));
  int rc = ensure_real_buf(h);
  if (rc) return rc;
  XLaunch X = x_base(h);
  X.mode = X_C2R;
  X.in0 = src;
  X.rout = h->real_buf;
  X.mean = mean;
  LAUNCH_TRY(h, xpass(h, X));
  return OPFC_OK;
}

}  // namespace

// elementwise out = psi_hat * table (split layout); used for psi_MF
__global__ void scale_by_table_f32(const float2 *in, const float *t, float2 *out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float2 v = in[i];
    const float s = t[i];
    out[i] = make_float2(v.x * s, v.y * s);
  }
}
__global__ void scale_by_table_f64(const double2 *in, const double *t, double2 *out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = in[i];
    const double s = t[i];
    out[i] = make_double2(v.x * s, v.y * s);
  }
}

int opfc_scale_by_table(opfc_handle *h, const void *in, const void *tab, void *out) {
  const int blocks = 148 * 8;
  if (h->prec == OPFC_FP64)
    scale_by_table_f64<<<blocks, 256, 0, h->stream>>>((const double2 *)in, (const double *)tab, (double2 *)out, h->nc);
  else
    scale_by_table_f32<<<blocks, 256, 0, h->stream>>>((const float2 *)in, (const float *)tab, (float2 *)out, h->nc);
  CUDA_TRY(h, cudaGetLastError());
  return OPFC_OK;
}

extern "C" {

void opfc_desc_default(opfc_desc *d) {
  if (!d) return;
  std::memset(d, 0, sizeof *d);
  d->n[0] = d->n[1] = d->n[2] = 32;
  d->dx[0] = d->dx[1] = d->dx[2] = 1.0;
  d->precision = OPFC_FP32;
  d->model = OPFC_MODEL_PLAIN;
  d->r = -0.25;
  d->filter_alpha = 0.5;
  d->p2 = -0.1;
  d->p3 = -0.5;
  d->p4 = 0.3;
  opfc_tungsten_params &p = d->tungsten;
  p.n0 = -0.10; p.n_sol = -0.047; p.n_vap = -0.464; p.T = 3300.0; p.T0 = 156000.0;
  p.Bx = 0.8582; p.alpha = 0.50; p.alpha_farTol = 0.001; p.alpha_highOrd = 4;
  p.lambda = 0.22; p.stabP = 0.2; p.shift_u = 0.3341; p.shift_s = 0.1898;
  p.p2 = 1.0; p.p3 = -0.5; p.p4 = 0.333333333; p.q20 = -0.0037; p.q21 = 1.0;
  p.q30 = -12.4567; p.q31 = 20.0; p.q40 = 45.0;
  d->aluminum.T0 = 1.0;  // Aluminum::params: everything 0 except T0 = 1
}

const char *opfc_status_string(int s) {
  switch (s) {
    case OPFC_OK: return "ok";
    case OPFC_ERR_ARG: return "invalid argument";
    case OPFC_ERR_SIZE: return "size contract violated";
    case OPFC_ERR_CUDA: return "CUDA error";
    case OPFC_ERR_NONFINITE: return "non-finite value in field";
    case OPFC_ERR_TIMEOUT: return "device wait timed out";
    case OPFC_ERR_OOM: return "device out of memory";
    case OPFC_ERR_STATE: return "call out of order";
    case OPFC_ERR_IO: return "file I/O failed";
  }
  return "unknown status";
}

const char *opfc_last_error(const opfc_handle *h) { return h ? h->err.c_str() : "null handle"; }

int opfc_set_operators(opfc_handle *h, const double *exp_Ldt, const double *n_weight, const double *chi,
                       size_t count) {
  if (!h || !exp_Ldt || !n_weight) return h ? fail(h, OPFC_ERR_ARG, "null operator table") : OPFC_ERR_ARG;
  if (!user_ops_model(h->desc.model)) return fail(h, OPFC_ERR_ARG, "opfc_set_operators: not a user ETD model");
  int rc;
  if ((rc = check_count(h, count, h->nc, "opfc_set_operators"))) return rc;
  // the mean is carried exactly on the host: the operators must conserve it
  if (std::fabs(exp_Ldt[0] - 1.0) > 1e-12 || n_weight[0] != 0.0 || (chi && std::fabs(chi[0] - 1.0) > 1e-12))
    return fail(h, OPFC_ERR_ARG,
                "opfc_set_operators: k = 0 must have exp_Ldt = 1, n_weight = 0, chi = 1 (conserved dynamics)");
  CUDA_TRY(h, cudaSetDevice(h->device));
  const int H = h->M + 1;
  std::vector<double> t[3] = {std::vector<double>(h->nc), std::vector<double>(h->nc), std::vector<double>(h->nc)};
  const double *src[3] = {exp_Ldt, n_weight, chi};
  parallel_for((long)h->n2 * h->n1, [&](long row) {
    const int ky = (int)(row % h->n1), kz = (int)(row / h->n1);
    for (int kx = 0; kx < H; ++kx) {
      const size_t r = (size_t)kx + (size_t)H * (size_t)row;  // reference layout
      const size_t o = split_index(h, kx, ky, kz);
      for (int q = 0; q < 3; ++q) t[q][o] = src[q] ? src[q][r] : 1.0;
    }
  });
  void **dst[3] = {&h->tab_a, &h->tab_b, &h->tab_chi};
  for (int q = 0; q < 3; ++q) {
    if (!*dst[q] && (rc = dev_alloc(h, dst[q], h->nc * h->rsz))) return rc;
    if (h->prec == OPFC_FP64) {
      CUDA_TRY(h, cudaMemcpy(*dst[q], t[q].data(), h->nc * 8, cudaMemcpyHostToDevice));
    } else {
      std::vector<float> f(t[q].begin(), t[q].end());
      CUDA_TRY(h, cudaMemcpy(*dst[q], f.data(), h->nc * 4, cudaMemcpyHostToDevice));
    }
  }
  h->user_ops = true;
  h->a_valid = false;
  release_graph(h);
  return OPFC_OK;
}

int opfc_set_time(opfc_handle *h, double t, double dt_per_step) {
  if (!h) return OPFC_ERR_ARG;
  if (!h->time_dev) return OPFC_OK;  // the model's step does not depend on the time
  CUDA_TRY(h, cudaSetDevice(h->device));
  CUDA_TRY(h, cudaMemcpyAsync(h->time_dev, &t, sizeof t, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (h->time_dt != dt_per_step) {
    h->time_dt = dt_per_step;
    release_graph(h);  // the captured step bakes in the increment
  }
  return OPFC_OK;
}

// ---------------------------------------------------------------------------
// on-disk formats (io.h): the field goes through the host in FP64
// ---------------------------------------------------------------------------
static int io_fail(opfc_handle *h, int rc, const std::string &msg) { return fail(h, rc, "%s", msg.c_str()); }

int opfc_write_binary(opfc_handle *h, const char *pattern, int increment) {
  if (!h) return OPFC_ERR_ARG;
  std::string fn, err;
  int rc;
  if ((rc = io::format_with_number(pattern, increment, fn, err))) return io_fail(h, rc, err);
  std::vector<double> psi(h->nr);
  if ((rc = opfc_get_psi(h, psi.data(), h->nr, OPFC_F64, OPFC_HOST))) return rc;
  const int n[3] = {h->n0, h->n1, h->n2}, zero[3] = {0, 0, 0};
  if ((rc = io::write_box(fn, n, n, zero, psi.data(), 1, err))) return io_fail(h, rc, err);
  return OPFC_OK;
}

int opfc_write_binary_hat(opfc_handle *h, const char *pattern, int increment) {
  if (!h) return OPFC_ERR_ARG;
  std::string fn, err;
  int rc;
  if ((rc = io::format_with_number(pattern, increment, fn, err))) return io_fail(h, rc, err);
  std::vector<double> hat(2 * h->nc);
  if ((rc = opfc_get_psi_hat(h, hat.data(), h->nc, OPFC_F64, OPFC_HOST))) return rc;
  const int n[3] = {h->n0 / 2 + 1, h->n1, h->n2}, zero[3] = {0, 0, 0};
  if ((rc = io::write_box(fn, n, n, zero, hat.data(), 2, err))) return io_fail(h, rc, err);
  return OPFC_OK;
}

int opfc_read_binary(opfc_handle *h, const char *filename) {
  if (!h) return OPFC_ERR_ARG;
  if (!filename) return fail(h, OPFC_ERR_ARG, "null file name");
  std::string err;
  std::vector<double> psi(h->nr);
  const int n[3] = {h->n0, h->n1, h->n2}, zero[3] = {0, 0, 0};
  int rc;
  if ((rc = io::read_box(filename, n, n, zero, psi.data(), 1, err))) return io_fail(h, rc, err);
  return opfc_set_psi(h, psi.data(), h->nr, OPFC_F64, OPFC_HOST);
}

int opfc_write_vti(opfc_handle *h, const char *pattern, int increment, const char *field_name) {
  if (!h) return OPFC_ERR_ARG;
  std::string fn, err;
  int rc;
  if ((rc = io::format_with_number(pattern, increment, fn, err))) return io_fail(h, rc, err);
  std::vector<double> psi(h->nr);
  if ((rc = opfc_get_psi(h, psi.data(), h->nr, OPFC_F64, OPFC_HOST))) return rc;
  const int n[3] = {h->n0, h->n1, h->n2}, zero[3] = {0, 0, 0};
  if ((rc = io::write_vti(fn, n, n, zero, h->desc.origin, h->desc.dx, field_name, psi.data(), err)))
    return io_fail(h, rc, err);
  return OPFC_OK;
}

int opfc_destroy(opfc_handle *h) {
  if (!h) return OPFC_ERR_ARG;
  int dev_prev = 0;
  cudaGetDevice(&dev_prev);
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  release_graph(h);
  void *bufs[] = {h->psi_hat, h->work_a, h->work_b, h->tab_a, h->tab_b, h->tab_chi,
                  h->tw_x, h->tw_y, h->tw_z, h->real_buf, h->flag, h->partials};
  for (void *p : bufs)
    if (p) cudaFree(p);
  for (void *p : h->ckpt)
    if (p) cudaFree(p);
  for (void *p : h->seg)
    if (p) cudaFree(p);
  void *adj[] = {h->tab_ar,   h->tab_br,   h->adj_c[0], h->adj_c[1], h->adj_r[0], h->adj_r[1],
                 h->adj_r[2], h->adj_r[3], h->rad_ops,  h->rad_chi,  h->tab_p,    h->work_c,
                 h->time_dev, h->fold_ops, h->fold_chi};
  for (void *p : adj)
    if (p) cudaFree(p);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  cudaSetDevice(dev_prev);
  delete h;
  return OPFC_OK;
}

int opfc_create(const opfc_desc *d, opfc_handle **out) {
  if (!d || !out) return OPFC_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<opfc_handle> h(new opfc_handle);
  h->desc = *d;
  if (d->precision != OPFC_FP32 && d->precision != OPFC_FP64) return OPFC_ERR_ARG;
  if (d->model < OPFC_MODEL_PLAIN || d->model > OPFC_MODEL_USER_ETD) return OPFC_ERR_ARG;
  for (int a = 0; a < 3; ++a)
    if (d->n[a] < 1 || !(d->dx[a] > 0)) return OPFC_ERR_SIZE;
  if (d->n[0] < 2 || d->n[0] % 2 != 0) return OPFC_ERR_SIZE;
  if (!supported_len(d->n[0] / 2) || !supported_len(d->n[1]) || !supported_len(d->n[2]))
    return OPFC_ERR_SIZE;
  h->n0 = d->n[0];
  h->n1 = d->n[1];
  h->n2 = d->n[2];
  h->M = h->n0 / 2;
  h->g0 = d->n_global[0] > 0 ? d->n_global[0] : h->n0;
  h->g1 = d->n_global[1] > 0 ? d->n_global[1] : h->n1;
  h->g2 = d->n_global[2] > 0 ? d->n_global[2] : h->n2;
  h->kx0 = d->kx0;
  h->slab = h->g0 != h->n0 || h->g1 != h->n1 || h->g2 != h->n2 || h->kx0 != 0;
  if (h->slab) {
    if (d->model != OPFC_MODEL_PLAIN && d->model != OPFC_MODEL_FILTERED) return OPFC_ERR_ARG;
    if (h->g0 % 2 != 0 || h->kx0 < 0 || h->kx0 + h->M > h->g0 / 2 || h->n1 > h->g1 || h->n2 > h->g2)
      return OPFC_ERR_SIZE;
  }
  h->nr = (size_t)h->n0 * h->n1 * h->n2;
  h->nc = (size_t)(h->M + 1) * h->n1 * h->n2;
  h->nyq_off = (long long)h->M * h->n1 * h->n2;
  h->prec = d->precision;
  h->rsz = h->prec == OPFC_FP64 ? 8 : 4;
  h->device = d->device;
  {
    const char *no = std::getenv("OPFC_NO_TMA");
    h->use_tma = !(no && no[0] == '1');
    const char *nv = std::getenv("OPFC_NVTX");
    h->nvtx = nv && nv[0] == '1';
  }
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return OPFC_ERR_CUDA;
  if (d->stream) {
    h->stream = (cudaStream_t)d->stream;
  } else {
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return OPFC_ERR_CUDA;
    h->own_stream = true;
  }
  const size_t cb = h->nc * 2 * h->rsz;
  int rc = 0;
  opfc_handle *hp = h.get();
  auto cleanup = [&](int code) {
    opfc_destroy(h.release());
    return code;
  };
  if ((rc = dev_alloc(hp, &hp->psi_hat, cb))) return cleanup(rc);
  if ((rc = dev_alloc(hp, &hp->work_a, cb))) return cleanup(rc);
  if (two_field(d->model) && (rc = dev_alloc(hp, &hp->work_b, cb))) return cleanup(rc);
  hp->al_grad = d->model == OPFC_MODEL_ALUMINUM && d->aluminum.G_grid != 0.0;
  if (hp->al_grad) {
    if ((rc = dev_alloc(hp, &hp->work_c, cb))) return cleanup(rc);
    if ((rc = dev_alloc(hp, (void **)&hp->time_dev, sizeof(double)))) return cleanup(rc);
    if (cudaMemset(hp->time_dev, 0, sizeof(double)) != cudaSuccess) return cleanup(OPFC_ERR_CUDA);
  }
  if ((rc = upload_twiddles(hp, hp->n0, &hp->tw_x))) return cleanup(rc);
  if ((rc = upload_twiddles(hp, hp->n1, &hp->tw_y))) return cleanup(rc);
  if ((rc = upload_twiddles(hp, hp->n2, &hp->tw_z))) return cleanup(rc);
  if ((rc = dev_alloc(hp, (void **)&hp->flag, sizeof(unsigned int)))) return cleanup(rc);
  if ((rc = dev_alloc(hp, (void **)&hp->partials, sizeof(double) * hp->npartials))) return cleanup(rc);
  if (cudaMemset(hp->flag, 0, sizeof(unsigned int)) != cudaSuccess) return cleanup(OPFC_ERR_CUDA);
  if (cudaMemset(hp->psi_hat, 0, cb) != cudaSuccess) return cleanup(OPFC_ERR_CUDA);
  if (cudaDeviceGetAttribute(&hp->num_sms, cudaDevAttrMultiProcessorCount, hp->device) != cudaSuccess)
    hp->num_sms = 148;
  hp->tmaps.reserve(64);
  *out = h.release();
  return OPFC_OK;
}

static int finish_initialize(opfc_handle *h);

int opfc_initialize(opfc_handle *h, double dt) {
  if (!h) return OPFC_ERR_ARG;
  if (!(dt > 0) || !std::isfinite(dt)) return fail(h, OPFC_ERR_ARG, "dt must be positive and finite");
  CUDA_TRY(h, cudaSetDevice(h->device));
  if (user_ops_model(h->desc.model)) {  // the caller's tables already include dt
    if (!h->user_ops) return fail(h, OPFC_ERR_STATE, "user ETD model: call opfc_set_operators first");
    h->dt = dt;
    return finish_initialize(h);
  }
  // a slab handle (opfc_pass) takes its wave numbers from the whole grid: the
  // half-spectrum column kx is the global column kx0 + kx; its y and z axes
  // span the whole grid whenever it runs a z update
  const int n0 = h->g0, n1 = h->n1, n2 = h->n2, H = h->M + 1, kxo = h->kx0;
  const double f0 = 2.0 * kPi / (h->desc.dx[0] * n0);
  const double f1 = 2.0 * kPi / (h->desc.dx[1] * n1);
  const double f2 = 2.0 * kPi / (h->desc.dx[2] * n2);
  const int model = h->desc.model;
  const bool need_chi = model != OPFC_MODEL_PLAIN;
  std::vector<double> ta(h->nc), tb(h->nc), tc(need_chi ? h->nc : 0);
  auto kc = [](int i, int n, double f) { return (i <= n / 2) ? i * f : (i - n) * f; };
  const opfc_tungsten_params P = h->desc.tungsten;
  // Tungsten scalars (tungsten_params.hpp:339-411, tungsten_spectral.hpp:67-75)
  const double tau = P.T / P.T0;
  const double p2b = P.p2 + 2 * P.shift_s * P.p3 + 3 * std::pow(P.shift_s, 2) * P.p4;
  const double q20b = P.q20 + 2.0 * P.shift_s * P.q30 + 3.0 * std::pow(P.shift_s, 2) * P.q40;
  const double q21b = P.q21 + 2.0 * P.shift_s * P.q31;
  const double q2b = q21b * tau + q20b;
  const double alpha2 = 2.0 * P.alpha * P.alpha;
  const double lambda2 = 2.0 * P.lambda * P.lambda;
  const double rTol = -alpha2 * std::log(P.alpha_farTol) - 1.0;
  const double peak = P.Bx * std::exp(-P.T / P.T0);
  const double r = h->desc.r;
  const double fa = h->desc.filter_alpha;
  const opfc_aluminum_params A = h->desc.aluminum;
  if (model == OPFC_MODEL_ALUMINUM && A.T0 == 0.0) return fail(h, OPFC_ERR_ARG, "Aluminum: T0 must be nonzero");
  // Aluminum.hpp:186-242 (prepare_operators): chi = exp(kLap/(2 lambda^2)); the
  // peak is the larger of the Gaussians around |k| = 1 and 2/sqrt(3);
  // P_F = Bx exp(-tau_const) peak; opCk = stabP + p2_bar - P_F + q2_bar_L chi;
  // opL = exp(kLap opCk dt); opN = kLap dt if opCk == 0 else (opL - 1)/opCk
  auto aluminum_peak = [&](double kLap) {
    const double a2 = 2.0 * A.alpha * A.alpha;
    const double kw = std::sqrt(-kLap) - 1.0, kp = std::sqrt(-kLap) - 2.0 / std::sqrt(3.0);
    const double g1 = std::exp(-(kw * kw) / a2), gp1 = std::exp(-(kp * kp) / a2);
    return A.Bx * std::exp(-A.tau_const) * (g1 > gp1 ? g1 : gp1);
  };
  auto aluminum_mode = [&](double kLap, double &oa, double &ob, double &oc) {
    const double l2 = 2.0 * A.lambda * A.lambda;
    const double fMF = std::exp(kLap / l2);
    const double PF = aluminum_peak(kLap);
    const double opCk = A.stabP + A.p2_bar - PF + A.q2_bar_L * fMF;
    oa = std::exp(kLap * opCk * dt);
    ob = (opCk == 0.0) ? kLap * dt : (oa - 1.0) / opCk;
    oc = fMF;
  };
  // operators of one mode from its wave-vector components (FP64, the
  // reference's formulas): oa = opL / exp_Ldt, ob = opN / n_weight, oc = filter
  auto mode_ops = [&](double kx_, double ky_, double kz_, double &oa, double &ob, double &oc) {
    if (model == OPFC_MODEL_ALUMINUM) {
      const double kLap = -((kx_ * kx_) + (ky_ * ky_) + (kz_ * kz_));
      aluminum_mode(kLap, oa, ob, oc);
    } else if (model == OPFC_MODEL_TUNGSTEN) {
      // physics_for_mode (tungsten_spectral.hpp:83-104) + spectral_exp_coeffs
      // (spectral_exp_coefficients.hpp:68-82) + n_weight (tungsten_etd_workspace.hpp:111-130)
      const double kLap = -((kx_ * kx_) + (ky_ * ky_) + (kz_ * kz_));
      const double fMF = std::exp(kLap / lambda2);
      const double kv = std::sqrt(-kLap) - 1.0;
      const double k2 = kv * kv;
      const double g1 = (P.alpha_highOrd == 0)
                            ? std::exp(-k2 / alpha2)
                            : std::exp(-(k2 + rTol * std::pow(kv, P.alpha_highOrd)) / alpha2);
      const double g2 = 1.0 - 1.0 / alpha2 * k2;
      const double gf = (kv < 0.0) ? g1 : g2;
      const double opCk = P.stabP + p2b - peak * gf + q2b * fMF;
      const double L = kLap * opCk;
      const double arg = L * dt;
      const double phi1 = (std::fabs(L) < 1e-12) ? dt + 0.5 * L * dt * dt : std::expm1(arg) / L;
      oa = std::exp(arg);
      ob = kLap * phi1;
      oc = fMF;
    } else {
      // 10_complete_pfc_model.cpp:189-207
      const double k2 = kx_ * kx_ + ky_ * ky_ + kz_ * kz_;
      const double k2_lap = -k2;
      const double L = k2_lap * (r + (1.0 - k2) * (1.0 - k2));
      const double eL = std::exp(L * dt);
      oa = eL;
      ob = (std::fabs(L) > 1e-14) ? (eL - 1.0) / L * k2_lap : dt * k2_lap;
      oc = need_chi ? std::exp(-k2 / (2.0 * fa * fa)) : 1.0;
    }
  };
  std::vector<double> tp(h->al_grad ? h->nc : 0);
  parallel_for((long)n2 * n1, [&](long row) {
    const int ky = (int)(row % n1), kz = (int)(row / n1);
    for (int kx = 0; kx < H; ++kx) {
      const double kx_ = kc(kx + kxo, n0, f0), ky_ = kc(ky, n1, f1), kz_ = kc(kz, n2, f2);
      const size_t o = split_index(h, kx, ky, kz);
      double oc = 1.0;
      mode_ops(kx_, ky_, kz_, ta[o], tb[o], oc);
      if (need_chi) tc[o] = oc;
      if (h->al_grad) tp[o] = aluminum_peak(-((kx_ * kx_) + (ky_ * ky_) + (kz_ * kz_)));
    }
  });
  // Folded tables: every operator is a function of k^2, and ky, n1 - ky (kz,
  // n2 - kz) give the same k^2 bit for bit ((i - n) f = -((n - i) f) exactly),
  // so the (M+1) x (n1/2+1) x (n2/2+1) modes with folded indices hold every
  // per-mode value; the z update reads them (pairs (opL, opN) and the filter)
  // instead of the full tables.  Not for the moving-gradient Aluminum model
  // (its P_F term stays per mode).
  std::vector<double> fo, fc;
  const int F1 = n1 / 2 + 1, F2 = n2 / 2 + 1;
  const size_t nf = (size_t)H * F1 * F2;
  if (!h->al_grad) {
    fo.resize(2 * nf);
    if (need_chi) fc.resize(nf);
    h->fold_nyq = (long long)h->M * F1 * F2;
    parallel_for((long)F2 * F1, [&](long row) {
      const int fy = (int)(row % F1), fz = (int)(row / F1);
      for (int kx = 0; kx < H; ++kx) {
        const size_t o = kx < h->M ? (size_t)kx + (size_t)h->M * row : (size_t)h->fold_nyq + row;
        double oc = 1.0;
        mode_ops(kc(kx + kxo, n0, f0), fy * f1, fz * f2, fo[2 * o], fo[2 * o + 1], oc);
        if (need_chi) fc[o] = oc;
      }
    });
  }
  auto upload = [&](std::vector<double> &src, void **dst) -> int {
    if (!*dst) {
      int rc = dev_alloc(h, dst, h->nc * h->rsz);
      if (rc) return rc;
    }
    if (h->prec == OPFC_FP64) {
      CUDA_TRY(h, cudaMemcpy(*dst, src.data(), h->nc * 8, cudaMemcpyHostToDevice));
    } else {
      std::vector<float> f(src.begin(), src.end());
      CUDA_TRY(h, cudaMemcpy(*dst, f.data(), h->nc * 4, cudaMemcpyHostToDevice));
    }
    return OPFC_OK;
  };
  auto upload_n = [&](const std::vector<double> &src, void **dst) -> int {
    if (*dst) cudaFree(*dst);
    *dst = nullptr;
    int rc2 = dev_alloc(h, dst, src.size() * h->rsz);
    if (rc2) return rc2;
    if (h->prec == OPFC_FP64) {
      CUDA_TRY(h, cudaMemcpy(*dst, src.data(), src.size() * 8, cudaMemcpyHostToDevice));
    } else {
      std::vector<float> f(src.begin(), src.end());
      CUDA_TRY(h, cudaMemcpy(*dst, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
    }
    return OPFC_OK;
  };
  int rc;
  if ((rc = upload(ta, &h->tab_a))) return rc;
  if ((rc = upload(tb, &h->tab_b))) return rc;
  if (need_chi && (rc = upload(tc, &h->tab_chi))) return rc;
  if (!fo.empty() && (rc = upload_n(fo, &h->fold_ops))) return rc;
  if (!fc.empty() && (rc = upload_n(fc, &h->fold_chi))) return rc;
  if (h->al_grad) {
    if ((rc = upload(tp, &h->tab_p))) return rc;
    h->pf0 = aluminum_peak(0.0);
    h->time_dt = dt;
    CUDA_TRY(h, cudaMemset(h->time_dev, 0, sizeof(double)));
  }

  // Isotropic grids (one frequency step f on all axes): every operator depends
  // only on m = i^2 + j^2 + k^2 of the folded integer indices (k^2 = f^2 m), so
  // the fused z update reads small L2-resident tables instead of streaming the
  // per-mode tables from HBM.  Same formulas, FP64, rounded once.
  const char *no_rad = std::getenv("OPFC_NO_RADIAL");
  if (f0 == f1 && f1 == f2 && !(no_rad && no_rad[0] == '1') && !h->al_grad && !h->slab) {
    const long mmax = (long)(n0 / 2) * (n0 / 2) + (long)(n1 / 2) * (n1 / 2) + (long)(n2 / 2) * (n2 / 2);
    const size_t cnt = (size_t)mmax + 1;
    std::vector<double> ops(2 * cnt), chi(need_chi ? cnt : 0);
    parallel_for((long)cnt, [&](long m) {
      const double k2 = f0 * f0 * (double)m;
      if (model == OPFC_MODEL_ALUMINUM) {
        aluminum_mode(-k2, ops[2 * m], ops[2 * m + 1], chi[m]);
      } else if (model == OPFC_MODEL_TUNGSTEN) {
        const double kLap = -k2;
        const double fMF = std::exp(kLap / lambda2);
        const double kv = std::sqrt(-kLap) - 1.0;
        const double kk = kv * kv;
        const double g1 = (P.alpha_highOrd == 0)
                              ? std::exp(-kk / alpha2)
                              : std::exp(-(kk + rTol * std::pow(kv, P.alpha_highOrd)) / alpha2);
        const double g2 = 1.0 - 1.0 / alpha2 * kk;
        const double opCk = P.stabP + p2b - peak * ((kv < 0.0) ? g1 : g2) + q2b * fMF;
        const double L = kLap * opCk;
        const double arg = L * dt;
        const double phi1 = (std::fabs(L) < 1e-12) ? dt + 0.5 * L * dt * dt : std::expm1(arg) / L;
        ops[2 * m] = std::exp(arg);
        ops[2 * m + 1] = kLap * phi1;
        chi[m] = fMF;
      } else {
        const double L = -k2 * (r + (1.0 - k2) * (1.0 - k2));
        const double eL = std::exp(L * dt);
        ops[2 * m] = eL;
        ops[2 * m + 1] = (std::fabs(L) > 1e-14) ? (eL - 1.0) / L * (-k2) : dt * (-k2);
        if (need_chi) chi[m] = std::exp(-k2 / (2.0 * fa * fa));
      }
    });
    auto up = [&](const std::vector<double> &src, void **dst) -> int {
      if (*dst) cudaFree(*dst);
      *dst = nullptr;
      int rc2 = dev_alloc(h, dst, src.size() * h->rsz);
      if (rc2) return rc2;
      if (h->prec == OPFC_FP64) {
        CUDA_TRY(h, cudaMemcpy(*dst, src.data(), src.size() * 8, cudaMemcpyHostToDevice));
      } else {
        std::vector<float> f(src.begin(), src.end());
        CUDA_TRY(h, cudaMemcpy(*dst, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
      }
      return OPFC_OK;
    };
    if ((rc = up(ops, &h->rad_ops))) return rc;
    if (need_chi && (rc = up(chi, &h->rad_chi))) return rc;
  }
  h->dt = dt;
  return finish_initialize(h);
}

// kernel variants and handle state after the operator tables exist
static int finish_initialize(opfc_handle *h) {
  const int model = h->desc.model;
  // kernel variants: the autotuner's cached choice, else the defaults;
  // OPFC_Y_VARIANT / OPFC_X_VARIANT / OPFC_Z_VARIANT force a pass's variant
  h->var_y = AutoTuner::instance().get_config(tune_key(h, "y"), 0);
  h->var_x = AutoTuner::instance().get_config(tune_key(h, "x"), 0);
  h->var_z = AutoTuner::instance().get_config(tune_key(h, "z"), 0);
  // a cached FP32 choice with per-mode FP32 operators needs the opt-in
  if (z_computed(h->var_z) && h->prec == OPFC_FP32 && !computed_ops_allowed()) h->var_z = h->fold_ops ? 6 : 0;
  if (const char *zv = std::getenv("OPFC_Z_VARIANT")) h->var_z = std::atoi(zv);
  if (const char *yv = std::getenv("OPFC_Y_VARIANT")) h->var_y = std::atoi(yv);
  if (const char *xv = std::getenv("OPFC_X_VARIANT")) h->var_x = std::atoi(xv);
  if (h->var_x < 0 || h->var_x >= kVarX) h->var_x = 0;
  if (h->var_z < 0 || h->var_z >= kVarZ) h->var_z = 0;
  if (h->var_z == 1 && !h->rad_ops) h->var_z = 0;
  if (z_computed(h->var_z) && (two_field(model) || user_ops_model(model) || h->slab))
    h->var_z = h->var_z == 4 ? 2 : 0;
  if (z_folded(h->var_z) && !h->fold_ops) h->var_z = h->var_z == 7 ? 2 : 0;
  if (h->var_y < 0 || h->var_y >= kVarY) h->var_y = 0;
  h->initialized = true;
  h->a_valid = false;
  release_graph(h);
  return OPFC_OK;
}

int opfc_set_psi(opfc_handle *h, const void *psi, size_t count, int dtype, int where) {
  if (!h || !psi) return h ? fail(h, OPFC_ERR_ARG, "null field pointer") : OPFC_ERR_ARG;
  int rc;
  if ((rc = check_dtype_where(h, dtype, where))) return rc;
  if ((rc = check_count(h, count, h->nr, "opfc_set_psi"))) return rc;
  CUDA_TRY(h, cudaSetDevice(h->device));
  if ((rc = real_in(h, psi, dtype, where))) return rc;
  // k = 0 mode in FP64 with compensated summation of the caller's values in
  // their own precision (before any rounding to the compute precision).  A
  // host field already in the compute precision arrives bit for bit in the
  // device buffer, so its sum runs there (one pass of the GPU) instead of on
  // the host threads after the copy.
  const bool same_prec = (dtype == OPFC_F64) == (h->prec == OPFC_FP64);
  if (where == OPFC_HOST && same_prec)
    rc = user_sum(h, h->real_buf, dtype, OPFC_DEVICE, &h->mass_sum);
  else
    rc = user_sum(h, psi, dtype, where, &h->mass_sum);
  if (rc) return rc;
  if ((rc = forward_real_buf(h, h->psi_hat))) return rc;
  // the DC slot of the FP32/FP64 array stays zero; mass_sum carries it
  CUDA_TRY(h, cudaMemsetAsync(h->psi_hat, 0, 2 * h->rsz, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  h->have_state = true;
  h->a_valid = false;
  release_graph(h);  // the captured step bakes in the mean density
  return OPFC_OK;
}

int opfc_get_psi(opfc_handle *h, void *psi, size_t count, int dtype, int where) {
  if (!h || !psi) return h ? fail(h, OPFC_ERR_ARG, "null field pointer") : OPFC_ERR_ARG;
  int rc;
  if ((rc = check_dtype_where(h, dtype, where))) return rc;
  if ((rc = check_count(h, count, h->nr, "opfc_get_psi"))) return rc;
  if (!h->have_state) return fail(h, OPFC_ERR_STATE, "opfc_get_psi before opfc_set_psi");
  CUDA_TRY(h, cudaSetDevice(h->device));
  LAUNCH_TRY(h, col_plain(h, 2, +1, h->psi_hat, h->work_a));
  if ((rc = backward_to_real_buf(h, h->work_a, mean_density(h), true))) return rc;
  h->a_valid = false;
  return real_out(h, psi, dtype, where);
}

int opfc_get_psi_mf(opfc_handle *h, void *psi, size_t count, int dtype, int where) {
  if (!h || !psi) return h ? fail(h, OPFC_ERR_ARG, "null field pointer") : OPFC_ERR_ARG;
  int rc;
  if ((rc = check_dtype_where(h, dtype, where))) return rc;
  if ((rc = check_count(h, count, h->nr, "opfc_get_psi_mf"))) return rc;
  if (!h->have_state || !h->initialized) return fail(h, OPFC_ERR_STATE, "need state and tables");
  if (!h->tab_chi) return fail(h, OPFC_ERR_STATE, "model has no mean-field filter");
  CUDA_TRY(h, cudaSetDevice(h->device));
  if ((rc = opfc_scale_by_table(h, h->psi_hat, h->tab_chi, h->work_a))) return rc;
  // chi(0) = 1 in every model, so the mean carries over unchanged
  if ((rc = backward_to_real_buf(h, h->work_a, mean_density(h), false))) return rc;
  h->a_valid = false;
  return real_out(h, psi, dtype, where);
}

int opfc_get_psi_hat(opfc_handle *h, void *out, size_t count, int dtype, int where) {
  if (!h || !out) return h ? fail(h, OPFC_ERR_ARG, "null pointer") : OPFC_ERR_ARG;
  int rc;
  if ((rc = check_dtype_where(h, dtype, where))) return rc;
  if ((rc = check_count(h, count, h->nc, "opfc_get_psi_hat"))) return rc;
  if (!h->have_state) return fail(h, OPFC_ERR_STATE, "opfc_get_psi_hat before opfc_set_psi");
  CUDA_TRY(h, cudaSetDevice(h->device));
  const size_t esz = dtype == OPFC_F64 ? 8 : 4;
  void *dst = out;
  void *tmp = nullptr;
  if (where == OPFC_HOST) {
    CUDA_TRY(h, cudaMallocAsync(&tmp, h->nc * 2 * esz, h->stream));
    dst = tmp;
  }
  const int f64 = dtype == OPFC_F64;
  if (h->prec == OPFC_FP64)
    rc = launch_to_ref<double>(h->psi_hat, dst, f64, h->M, h->n1, h->n2, h->nyq_off, 1, h->mass_sum, h->stream);
  else
    rc = launch_to_ref<float>(h->psi_hat, dst, f64, h->M, h->n1, h->n2, h->nyq_off, 1, h->mass_sum, h->stream);
  if (rc) return fail(h, OPFC_ERR_CUDA, "to_ref: %s", cudaGetErrorString((cudaError_t)rc));
  if (tmp) {
    CUDA_TRY(h, cudaMemcpyAsync(out, tmp, h->nc * 2 * esz, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaFreeAsync(tmp, h->stream));
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return OPFC_OK;
}

int opfc_step(opfc_handle *h, int n_steps) {
  if (!h) return OPFC_ERR_ARG;
  if (n_steps < 0) return fail(h, OPFC_ERR_ARG, "negative step count");
  if (!h->initialized) return fail(h, OPFC_ERR_STATE, "opfc_step before opfc_initialize");
  if (!h->have_state) return fail(h, OPFC_ERR_STATE, "opfc_step before opfc_set_psi");
  if (n_steps == 0) return OPFC_OK;
  CUDA_TRY(h, cudaSetDevice(h->device));
  int rc;
  if (!h->a_valid && (rc = prepare_a(h))) return rc;
  if (h->nvtx) {  // eager, one NVTX range per kernel
    for (int s = 0; s < n_steps; ++s) {
      NvtxRange range("step");
      if ((rc = enqueue_step(h))) return rc;
    }
    return OPFC_OK;
  }
  if (!h->graph_exec) {
    if ((rc = build_graph(h))) return rc;
  }
  for (int s = 0; s < n_steps; ++s) CUDA_TRY(h, cudaGraphLaunch(h->graph_exec, h->stream));
  return OPFC_OK;
}

int opfc_sync(opfc_handle *h) {
  if (!h) return OPFC_ERR_ARG;
  CUDA_TRY(h, cudaSetDevice(h->device));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  unsigned int f = 0;
  CUDA_TRY(h, cudaMemcpy(&f, h->flag, sizeof f, cudaMemcpyDeviceToHost));
  if (f) {
    cudaMemset(h->flag, 0, sizeof f);
    if (f & 2u) return fail(h, OPFC_ERR_TIMEOUT, "a bounded device wait expired (TMA load never landed)");
    return fail(h, OPFC_ERR_NONFINITE, "non-finite value produced by the nonlinearity");
  }
  return OPFC_OK;
}

int opfc_pass(opfc_handle *h, int pass, double mean, int flags) {
  if (!h) return OPFC_ERR_ARG;
  if (pass < OPFC_PASS_Y_INVERSE || pass > OPFC_PASS_Z_INVERSE_STATE) return fail(h, OPFC_ERR_ARG, "unknown pass");
  if (pass == OPFC_PASS_Z_UPDATE && !h->initialized) return fail(h, OPFC_ERR_STATE, "the z update needs opfc_initialize");
  if (two_field(h->desc.model) || h->al_grad) return fail(h, OPFC_ERR_ARG, "opfc_pass: PLAIN, FILTERED or USER_ETD");
  CUDA_TRY(h, cudaSetDevice(h->device));
  int rc = OPFC_OK;
  release_graph(h);  // the step graph, if any, bakes in the handle's own mean
  switch (pass) {
    case OPFC_PASS_Y_INVERSE:
      return enqueue_step_kernels(h, 0);
    case OPFC_PASS_X_FUSED:
      h->use_pass_mean = true;
      h->pass_mean = mean;
      rc = enqueue_step_kernels(h, 1);
      h->use_pass_mean = false;
      return rc;
    case OPFC_PASS_Y_FORWARD:
      return enqueue_step_kernels(h, 2);
    case OPFC_PASS_Z_UPDATE: {
      if ((rc = enqueue_step_kernels(h, 3))) return rc;
      const int planes = flags & 3;
      if (h->prec == OPFC_FP64)
        LAUNCH_TRY(h, launch_herm_fix<double>(h->psi_hat, h->nyq_off, h->M, h->n1, h->n2, h->stream, nullptr, 0.0,
                                              planes));
      else
        LAUNCH_TRY(h, launch_herm_fix<float>(h->psi_hat, h->nyq_off, h->M, h->n1, h->n2, h->stream, nullptr, 0.0,
                                             planes));
      return OPFC_OK;
    }
    case OPFC_PASS_XY_FORWARD: {  // real_buf -> A: x R2C, y forward
      if ((rc = ensure_real_buf(h))) return rc;
      XLaunch X = x_base(h);
      X.mode = X_R2C;
      X.rin = h->real_buf;
      X.out = h->work_a;
      LAUNCH_TRY(h, xpass(h, X));
      LAUNCH_TRY(h, col_plain(h, 1, -1, h->work_a, h->work_a));
      return OPFC_OK;
    }
    case OPFC_PASS_XY_BACKWARD:  // A -> real_buf: y inverse, x C2R (scaled by the whole grid), + mean
      return backward_to_real_buf(h, h->work_a, mean, true);
    case OPFC_PASS_Z_FORWARD:  // A -> psi_hat
      LAUNCH_TRY(h, col_plain(h, 2, -1, h->work_a, h->psi_hat));
      if (flags & 4) CUDA_TRY(h, cudaMemsetAsync(h->psi_hat, 0, 2 * h->rsz, h->stream));
      h->have_state = true;
      h->a_valid = false;
      return OPFC_OK;
    case OPFC_PASS_Z_INVERSE:  // psi_hat -> A as the step starts (chi-filtered for FILTERED)
      return prepare_a(h);
    case OPFC_PASS_Z_INVERSE_STATE:  // psi_hat -> A, unfiltered
      LAUNCH_TRY(h, col_plain(h, 2, +1, h->psi_hat, h->work_a));
      return OPFC_OK;
  }
  return OPFC_ERR_ARG;
}

void *opfc_array(opfc_handle *h, int which) {
  if (!h) return nullptr;
  if (which == OPFC_ARRAY_WORK) return h->work_a;
  if (which == OPFC_ARRAY_STATE) return h->psi_hat;
  if (which == OPFC_ARRAY_REAL) {
    if (cudaSetDevice(h->device) != cudaSuccess || ensure_real_buf(h)) return nullptr;
    return h->real_buf;
  }
  return nullptr;
}

int opfc_check_bounded_wait(opfc_handle *h, double limit_ms) {
  if (!h) return OPFC_ERR_ARG;
  if (!(limit_ms >= 0.1 && limit_ms <= 1000.0)) return fail(h, OPFC_ERR_ARG, "limit_ms must be in [0.1, 1000]");
  CUDA_TRY(h, cudaSetDevice(h->device));
  LAUNCH_TRY(h, launch_wait_check(h->flag, limit_ms, h->stream));
  return OPFC_OK;
}

int opfc_fft_forward(opfc_handle *h, const void *in_real, void *out_complex, int dtype, int where) {
  if (!h || !in_real || !out_complex) return h ? fail(h, OPFC_ERR_ARG, "null pointer") : OPFC_ERR_ARG;
  int rc;
  if ((rc = check_dtype_where(h, dtype, where))) return rc;
  CUDA_TRY(h, cudaSetDevice(h->device));
  if ((rc = real_in(h, in_real, dtype, where))) return rc;
  if ((rc = forward_real_buf(h, h->work_a))) return rc;
  h->a_valid = false;
  const size_t esz = dtype == OPFC_F64 ? 8 : 4;
  void *dst = out_complex, *tmp = nullptr;
  if (where == OPFC_HOST) {
    CUDA_TRY(h, cudaMallocAsync(&tmp, h->nc * 2 * esz, h->stream));
    dst = tmp;
  }
  const int f64 = dtype == OPFC_F64;
  if (h->prec == OPFC_FP64)
    rc = launch_to_ref<double>(h->work_a, dst, f64, h->M, h->n1, h->n2, h->nyq_off, 0, 0.0, h->stream);
  else
    rc = launch_to_ref<float>(h->work_a, dst, f64, h->M, h->n1, h->n2, h->nyq_off, 0, 0.0, h->stream);
  if (rc) return fail(h, OPFC_ERR_CUDA, "to_ref: %s", cudaGetErrorString((cudaError_t)rc));
  if (tmp) {
    CUDA_TRY(h, cudaMemcpyAsync(out_complex, tmp, h->nc * 2 * esz, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaFreeAsync(tmp, h->stream));
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return OPFC_OK;
}

int opfc_fft_backward(opfc_handle *h, const void *in_complex, void *out_real, int dtype, int where) {
  if (!h || !in_complex || !out_real) return h ? fail(h, OPFC_ERR_ARG, "null pointer") : OPFC_ERR_ARG;
  int rc;
  if ((rc = check_dtype_where(h, dtype, where))) return rc;
  CUDA_TRY(h, cudaSetDevice(h->device));
  const size_t esz = dtype == OPFC_F64 ? 8 : 4;
  const void *src = in_complex;
  void *tmp = nullptr;
  if (where == OPFC_HOST) {
    CUDA_TRY(h, cudaMallocAsync(&tmp, h->nc * 2 * esz, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(tmp, in_complex, h->nc * 2 * esz, cudaMemcpyHostToDevice, h->stream));
    src = tmp;
  }
  const int f64 = dtype == OPFC_F64;
  if (h->prec == OPFC_FP64)
    rc = launch_from_ref<double>(src, f64, h->work_a, h->M, h->n1, h->n2, h->nyq_off, h->stream);
  else
    rc = launch_from_ref<float>(src, f64, h->work_a, h->M, h->n1, h->n2, h->nyq_off, h->stream);
  if (rc) return fail(h, OPFC_ERR_CUDA, "from_ref: %s", cudaGetErrorString((cudaError_t)rc));
  if (tmp) CUDA_TRY(h, cudaFreeAsync(tmp, h->stream));
  h->a_valid = false;
  if ((rc = backward_to_real_buf(h, h->work_a, 0.0, false))) return rc;
  return real_out(h, out_real, dtype, where);
}

int opfc_mass(opfc_handle *h, double *mean) {
  if (!h || !mean) return OPFC_ERR_ARG;
  if (!h->have_state) return fail(h, OPFC_ERR_STATE, "no state");
  *mean = mean_density(h);
  return OPFC_OK;
}

int opfc_free_energy(opfc_handle *h, double *energy) {
  if (!h || !energy) return OPFC_ERR_ARG;
  if (!h->have_state) return fail(h, OPFC_ERR_STATE, "no state");
  if (two_field(h->desc.model) || user_ops_model(h->desc.model))
    return fail(h, OPFC_ERR_ARG, "free energy is defined for the plain and filtered models");
  CUDA_TRY(h, cudaSetDevice(h->device));
  // quadratic part by Parseval in k-space (FP64 accumulation of the resident state)
  if (h->prec == OPFC_FP64)
    LAUNCH_TRY(h, launch_energy_k<double>(h->psi_hat, h->M, h->n1, h->n2, h->nyq_off, h->desc.dx,
                                          h->desc.r, h->partials, h->npartials, h->stream));
  else
    LAUNCH_TRY(h, launch_energy_k<float>(h->psi_hat, h->M, h->n1, h->n2, h->nyq_off, h->desc.dx,
                                         h->desc.r, h->partials, h->npartials, h->stream));
  std::vector<double> part(h->npartials);
  CUDA_TRY(h, cudaMemcpyAsync(part.data(), h->partials, sizeof(double) * h->npartials,
                              cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  double sk = neumaier(part.data(), part.size());
  sk += (h->desc.r + 1.0) * h->mass_sum * h->mass_sum;  // k = 0 mode, G(0) = r + 1
  // quartic part in real space
  int rc;
  LAUNCH_TRY(h, col_plain(h, 2, +1, h->psi_hat, h->work_a));
  if ((rc = backward_to_real_buf(h, h->work_a, mean_density(h), true))) return rc;
  h->a_valid = false;
  double s4 = 0;
  if ((rc = device_sum(h, 4, &s4))) return rc;
  const double dV = h->desc.dx[0] * h->desc.dx[1] * h->desc.dx[2];
  *energy = dV * (0.5 * sk / (double)h->nr + 0.25 * s4);
  return OPFC_OK;
}

size_t opfc_size_inbox(const opfc_handle *h) { return h ? h->nr : 0; }
size_t opfc_size_outbox(const opfc_handle *h) { return h ? h->nc : 0; }
size_t opfc_allocated_bytes(const opfc_handle *h) { return h ? h->allocated : 0; }
void *opfc_get_stream(const opfc_handle *h) { return h ? (void *)h->stream : nullptr; }
// (the Aluminum gradient model's y pass launches once more, for P*psi)
// (the box-ring z update of z variant 9 launches once more, for the Nyquist
// plane, where it applies: z length 1024, PLAIN or FILTERED, TMA-fed passes)
int opfc_kernels_per_step(const opfc_handle *h) {
  if (!h) return 0;
  const int model = h->desc.model;
  const bool ring = h->var_z == 9 && h->n2 == 1024 && h->fold_ops && h->use_tma && !h->al_grad &&
                    (model == OPFC_MODEL_PLAIN || model == OPFC_MODEL_FILTERED) &&
                    h->M % (128 / (2 * (int)h->rsz)) == 0;
  return kStepKernels + (h->al_grad ? 1 : 0) + (ring ? 1 : 0);
}

int opfc_autotune(opfc_handle *h, double *ms) {
  if (!h) return OPFC_ERR_ARG;
  if (!h->initialized) return fail(h, OPFC_ERR_STATE, "opfc_autotune needs the operator tables");
  CUDA_TRY(h, cudaSetDevice(h->device));
  release_graph(h);
  AutoTuner &T = AutoTuner::instance();
  std::vector<double> my, mx, mz;
  // each candidate runs its pass alone, in place on whatever the arrays hold
  h->var_y = T.tune(tune_key(h, "y"), kVarY, [&](int v) { h->var_y = v; return enqueue_step(h, 0); }, h->stream, &my);
  h->var_x = T.tune(tune_key(h, "x"), kVarX, [&](int v) { h->var_x = v; return enqueue_step(h, 1); }, h->stream, &mx);
  h->var_z = T.tune(
      tune_key(h, "z"), kVarZ,
      [&](int v) {
        if (v == 1 && !h->rad_ops) return (int)OPFC_ERR_ARG;
        if (z_computed(v) && (two_field(h->desc.model) || user_ops_model(h->desc.model) || h->slab))
          return (int)OPFC_ERR_ARG;
        // FP32: operators computed in FP32 only when the caller opts in; the
        // default keeps FP64-built tables rounded once to the compute precision
        if (z_computed(v) && h->prec == OPFC_FP32 && !computed_ops_allowed()) return (int)OPFC_ERR_ARG;
        if (z_folded(v) && !h->fold_ops) return (int)OPFC_ERR_ARG;
        h->var_z = v;
        return enqueue_step(h, 3);
      },
      h->stream, &mz);
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  cudaMemset(h->flag, 0, sizeof(unsigned int));
  h->have_state = false;  // the passes overwrote the state
  h->a_valid = false;
  if (ms) {
    const std::vector<double> *all[3] = {&my, &mx, &mz};
    const int cnt[3] = {kVarY, kVarX, kVarZ};
    int o = 0;
    for (int p = 0; p < 3; ++p)
      for (int v = 0; v < cnt[p]; ++v) ms[o++] = (int)all[p]->size() > v ? (*all[p])[v] : -1.0;
  }
  return OPFC_OK;
}

int opfc_variants(const opfc_handle *h, int *var) {
  if (!h || !var) return OPFC_ERR_ARG;
  var[0] = h->var_y;
  var[1] = h->var_x;
  var[2] = h->var_z;
  return OPFC_OK;
}

int opfc_profile_step(opfc_handle *h, int reps, double *ms, int max_kernels) {
  if (!h || !ms || reps < 1) return OPFC_ERR_ARG;
  if (!h->initialized || !h->have_state) return fail(h, OPFC_ERR_STATE, "profile needs tables and a state");
  CUDA_TRY(h, cudaSetDevice(h->device));
  int rc;
  if (!h->a_valid && (rc = prepare_a(h))) return rc;
  cudaEvent_t e0, e1;
  CUDA_TRY(h, cudaEventCreate(&e0));
  CUDA_TRY(h, cudaEventCreate(&e1));
  const int nk = std::min(max_kernels, kStepKernels);
  for (int k = 0; k < nk; ++k) {
    // one untimed launch, then `reps` timed launches of kernel k alone, inside
    // the NVTX range of its reference region
    NvtxRange range(kStepRegions[k]);
    if ((rc = enqueue_step_kernels(h, k))) break;
    cudaEventRecord(e0, h->stream);
    for (int r = 0; r < reps && !rc; ++r) rc = enqueue_step_kernels(h, k);
    cudaEventRecord(e1, h->stream);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    ms[k] = (double)t / reps;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // the repeated in-place passes leave the field undefined
  h->have_state = false;
  h->a_valid = false;
  cudaMemset(h->flag, 0, sizeof(unsigned int));
  if (rc) return rc;
  return nk;
}

// ---------------------------------------------------------------------------
// initial conditions (host; set-up only).  Cells in x-fastest order
// (include/openpfc/kernel/field/operations.hpp:96-103), one 64-bit draw of
// std::mt19937_64 per random number, u = (draw >> 11) * 2^-53.
// ---------------------------------------------------------------------------
static inline double mt_unit(std::mt19937_64 &g) { return (double)(g() >> 11) * (1.0 / 9007199254740992.0); }

int opfc_ic_noise(double *psi, size_t count, double n0, double amp, uint64_t seed) {
  if (!psi) return OPFC_ERR_ARG;
  std::mt19937_64 g(seed);
  for (size_t i = 0; i < count; ++i) psi[i] = n0 + (-amp + 2.0 * amp * mt_unit(g));
  return OPFC_OK;
}

// One-mode BCC seed of the reference (single_seed.hpp, seed.hpp): six
// <110>/sqrt(2) vectors, u = rho + sum_q 2 amp cos(q.x) for |x - c| < radius.
static const double kQ[6][3] = {{1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 0, -1}, {1, -1, 0}, {0, 1, -1}};

int opfc_ic_seed(double *psi, const int n[3], const double dx[3], const double origin[3],
                 const double center[3], double radius, double rho, double amp, int outside_zero) {
  if (!psi || !n || !dx || !origin || !center) return OPFC_ERR_ARG;
  const double s = 1.0 / std::sqrt(2.0);
  const double r2 = std::pow(radius, 2);
  size_t idx = 0;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i, ++idx) {
        const double x = origin[0] + i * dx[0] - center[0];
        const double y = origin[1] + j * dx[1] - center[1];
        const double z = origin[2] + k * dx[2] - center[2];
        if (x * x + y * y + z * z < r2) {
          double u = rho;
          for (int q = 0; q < 6; ++q)
            u += 2.0 * amp * std::cos(s * kQ[q][0] * x + s * kQ[q][1] * y + s * kQ[q][2] * z);
          psi[idx] = u;
        } else if (outside_zero) {
          psi[idx] = 0.0;
        }
      }
  return OPFC_OK;
}

int opfc_ic_seeds(double *psi, const int n[3], const double dx[3], double n0, double noise,
                  int nseeds, double radius_cells, double amp, uint64_t seed) {
  if (!psi || !n || !dx || nseeds < 0) return OPFC_ERR_ARG;
  const size_t ncell = (size_t)n[0] * n[1] * n[2];
  std::mt19937_64 g(seed);
  for (size_t i = 0; i < ncell; ++i) psi[i] = n0 + (-noise + 2.0 * noise * mt_unit(g));
  const double s = 1.0 / std::sqrt(2.0);
  for (int sd = 0; sd < nseeds; ++sd) {
    double c[3];
    for (int a = 0; a < 3; ++a) c[a] = mt_unit(g) * n[a];
    const double R2 = radius_cells * radius_cells;
    // visit only the (periodically wrapped) bounding box of the sphere
    int lo[3], cnt[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = (int)std::floor(c[a] - radius_cells) - 1;
      cnt[a] = std::min(n[a], (int)std::ceil(c[a] + radius_cells) + 2 - lo[a]);
      if (cnt[a] == n[a]) lo[a] = 0;
    }
    for (int kk = 0; kk < cnt[2]; ++kk)
      for (int jj = 0; jj < cnt[1]; ++jj)
        for (int ii = 0; ii < cnt[0]; ++ii) {
          const int i = ((lo[0] + ii) % n[0] + n[0]) % n[0];
          const int j = ((lo[1] + jj) % n[1] + n[1]) % n[1];
          const int k = ((lo[2] + kk) % n[2] + n[2]) % n[2];
          const size_t idx = (size_t)i + (size_t)n[0] * ((size_t)j + (size_t)n[1] * k);
          double d[3] = {i - c[0], j - c[1], k - c[2]};
          for (int a = 0; a < 3; ++a) {  // periodic minimum image
            if (d[a] > 0.5 * n[a]) d[a] -= n[a];
            if (d[a] < -0.5 * n[a]) d[a] += n[a];
          }
          if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] >= R2) continue;
          const double X = d[0] * dx[0], Y = d[1] * dx[1], Z = d[2] * dx[2];
          double u = n0;
          for (int q = 0; q < 6; ++q) u += amp * std::cos(s * kQ[q][0] * X + s * kQ[q][1] * Y + s * kQ[q][2] * Z);
          psi[idx] = u;
        }
  }
  return OPFC_OK;
}

// Rotation of a seed's wave vectors (seed.hpp rotate(), SeedFCC.hpp):
// R = yaw(a0) (pitch(a1) roll(a2)), each matrix product and R q summed in index
// order from zero, as the reference does, so the values agree bit for bit.
static void rotate_q(const double ang[3], const double (*q0)[3], int nq, double (*out)[3]) {
  const double ca = std::cos(ang[0]), sa = std::sin(ang[0]), cb = std::cos(ang[1]), sb = std::sin(ang[1]);
  const double cc = std::cos(ang[2]), sc = std::sin(ang[2]);
  const double Ra[3][3] = {{ca, -sa, 0}, {sa, ca, 0}, {0, 0, 1}};
  const double Rb[3][3] = {{cb, 0, sb}, {0, 1, 0}, {-sb, 0, cb}};
  const double Rc[3][3] = {{1, 0, 0}, {0, cc, -sc}, {0, sc, cc}};
  double BC[3][3] = {}, R[3][3] = {};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      for (int c = 0; c < 3; ++c) BC[a][b] += Rb[a][c] * Rc[c][b];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      for (int c = 0; c < 3; ++c) R[a][b] += Ra[a][c] * BC[c][b];
  for (int v = 0; v < nq; ++v)
    for (int a = 0; a < 3; ++a) {
      double acc = 0;
      for (int b = 0; b < 3; ++b) acc += R[a][b] * q0[v][b];
      out[v][a] = acc;
    }
}

// SeedGridFCC::apply (apps/aluminumNew/SeedGridFCC.hpp) with SeedFCC
// (apps/aluminumNew/SeedFCC.hpp): one column of Ny x Nz seeds at x = X0 (Nx is
// not used for placement), centres jittered by U(-0.2 r, 0.2 r) and Euler angles
// U(0, 2 pi) from std::mt19937_64(rseed) through std::uniform_real_distribution
// (drawn in the reference's order); inside |X - c| < r the value is
// rho + sum_{4 <111>/sqrt(3) vectors q, rotated by yaw pitch roll} 2 amp cos(q . X)
// with X the absolute coordinate; the first seed that contains a point wins.
int opfc_ic_seed_grid_fcc(double *psi, const int n[3], const double dx[3], const double origin[3], int Nx, int Ny,
                          int Nz, double X0, double radius, double amplitude, double rho, double rseed) {
  if (!psi || !n || !dx || !origin || Nx < 1 || Ny < 1 || Nz < 1 || !(radius > 0)) return OPFC_ERR_ARG;
  struct Seed {
    double c[3], q[4][3];
  };
  const double Dy = dx[1] * n[1] / Ny, Dz = dx[2] * n[2] / Nz;
  std::mt19937_64 re((std::mt19937_64::result_type)rseed);
  std::uniform_real_distribution<double> rt(-0.2 * radius, 0.2 * radius);
  std::uniform_real_distribution<double> rr(0.0, 8.0 * std::atan(1.0));
  std::vector<Seed> seeds;
  const double s = 1.0 / std::sqrt(3.0);
  const double q0[4][3] = {{-s, s, s}, {s, -s, s}, {s, s, -s}, {s, s, s}};
  for (int j = 0; j < Ny; ++j)
    for (int k = 0; k < Nz; ++k) {
      Seed sd;
      sd.c[0] = X0 + rt(re);
      sd.c[1] = Dy / 2.0 + Dy * j + rt(re);
      sd.c[2] = Dz / 2.0 + Dz * k + rt(re);
      double ang[3];
      for (double &a : ang) a = rr(re);
      rotate_q(ang, q0, 4, sd.q);
      seeds.push_back(sd);
    }
  const double r2 = radius * radius;
  parallel_for((long)n[2] * n[1], [&](long row) {
    const int j = (int)(row % n[1]), k = (int)(row / n[1]);
    const double y = origin[1] + j * dx[1], z = origin[2] + k * dx[2];
    for (int i = 0; i < n[0]; ++i) {
      const double x = origin[0] + i * dx[0];
      for (const Seed &sd : seeds) {
        const double ex = x - sd.c[0], ey = y - sd.c[1], ez = z - sd.c[2];
        if (ex * ex + ey * ey + ez * ez < r2) {
          double u = rho;
          for (int v = 0; v < 4; ++v) u += 2.0 * amplitude * std::cos(sd.q[v][0] * x + sd.q[v][1] * y + sd.q[v][2] * z);
          psi[(size_t)row * n[0] + i] = u;
          break;
        }
      }
    }
  });
  return OPFC_OK;
}

// RandomSeeds::apply (include/openpfc/kernel/simulation/initial_conditions/
// random_seeds.hpp:54-101) with Seed (seed.hpp): 150 seeds of radius 20 with
// centres x ~ U(-108, -68), y, z ~ U(-128, 128) and Euler angles U(0, 2 pi),
// drawn from std::mt19937_64(42) through std::uniform_real_distribution in the
// reference's order (x, y, z, then the three angles, seed by seed).  Every cell
// X = origin + i dx takes the value of the first seed that contains it,
// rho + sum_q 2 amp cos(q . X) over the six rotated <110>/sqrt(2) vectors, and 0
// outside every seed.
int opfc_ic_random_seeds(double *psi, const int n[3], const double dx[3], const double origin[3], double density,
                         double amplitude) {
  if (!psi || !n || !dx || !origin || n[0] < 1 || n[1] < 1 || n[2] < 1) return OPFC_ERR_ARG;
  constexpr int kSeeds = 150;
  constexpr double kRadius = 20.0;
  struct Seed {
    double c[3], q[6][3];
  };
  std::mt19937_64 re(42);
  std::uniform_real_distribution<double> rx(-128.0 + kRadius, -128.0 + 3 * kRadius);
  std::uniform_real_distribution<double> ry(-128.0, 128.0);
  std::uniform_real_distribution<double> rz(-128.0, 128.0);
  std::uniform_real_distribution<double> ro(0.0, 8.0 * std::atan(1.0));
  const double s = 1.0 / std::sqrt(2.0);
  const double q0[6][3] = {{s, s, 0}, {s, 0, s}, {0, s, s}, {s, 0, -s}, {s, -s, 0}, {0, s, -s}};
  std::vector<Seed> seeds(kSeeds);
  for (Seed &sd : seeds) {
    sd.c[0] = rx(re);
    sd.c[1] = ry(re);
    sd.c[2] = rz(re);
    double ang[3];
    for (double &a : ang) a = ro(re);
    rotate_q(ang, q0, 6, sd.q);
  }
  const double r2 = kRadius * kRadius;
  parallel_for((long)n[2] * n[1], [&](long row) {
    const int j = (int)(row % n[1]), k = (int)(row / n[1]);
    const double y = origin[1] + j * dx[1], z = origin[2] + k * dx[2];
    for (int i = 0; i < n[0]; ++i) {
      const double x = origin[0] + i * dx[0];
      double u = 0.0;
      for (const Seed &sd : seeds) {
        const double ex = x - sd.c[0], ey = y - sd.c[1], ez = z - sd.c[2];
        if (ex * ex + ey * ey + ez * ez < r2) {
          u = density;
          for (int v = 0; v < 6; ++v) u += 2.0 * amplitude * std::cos(sd.q[v][0] * x + sd.q[v][1] * y + sd.q[v][2] * z);
          break;
        }
      }
      psi[(size_t)row * n[0] + i] = u;
    }
  });
  return OPFC_OK;
}

const char *opfc_step_kernel_name(int k) {
  return (k >= 0 && k < kStepKernels) ? kStepKernelNames[k] : "";
}

const char *opfc_step_kernel_region(int k) { return (k >= 0 && k < kStepKernels) ? kStepRegions[k] : ""; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Adjoint of the PFC step (checkpoint-and-recompute) for the plain, filtered,
// Tungsten and Aluminum (G_grid = 0) models and caller-supplied operators.
//
// In real space one step is psi' = A psi + B N(psi, C psi) with A = F^-1 opL F,
// B = F^-1 opN F and the mean-field filter C = F^-1 chi F (C = 1 for the plain
// model): N = psi^3 (10_complete_pfc_model.cpp:121-144); N = c0 v^2 + c1 v^3 +
// c2 v^4 of v = C psi (filtered, caller-supplied operators); N = c0 u^2 +
// c1 u^3 + c2 v^2 + c3 v^3 - c4 u of u = psi, v = C psi (Tungsten,
// cpu/tungsten_model.hpp:334-350, tungsten_ops_kernels.cu:25-58; Aluminum
// with G_grid = 0, Aluminum.hpp:285-307).  opL, opN and chi are real and even
// in k, so A, B and C are symmetric and the adjoint step is
//   lambda_n = A lambda_{n+1} + dN/du (B lambda_{n+1}) + C[dN/dv (B lambda_{n+1})]
// (the conjugate spectral multiplies are the multiplies themselves, the
// adjoint filter is the filter).  For the models with L = -k^2 (r + (1-k^2)^2)
// (plain, filtered), opL = exp(L dt) and opN = dt (-k^2) phi(L dt) with
// phi(x) = (e^x - 1)/x, so
//   dLoss/dr = sum_n <lambda_{n+1}, F^-1[dopL/dr psi_hat_n + dopN/dr N_hat_n]>
//            = sum_n (1/N) sum_k w_kx Re(conj(lambda_hat) (...)),
// dopL/dr = -k^2 dt opL,  dopN/dr = dt^2 k^4 phi'(L dt),
// accumulated in FP64 per reduction block on the device across all steps.
// psi_n comes from re-running the forward step (the same CUDA graph) from the
// nearest snapshot.
// ---------------------------------------------------------------------------

// Nonlinearity of the step's model from u = psi and v = C psi (in real space,
// the mean included); `kind` 0 plain, 1 filtered, 2 Tungsten form.
template <typename Real>
__global__ void adj_nonlin_kernel(const Real *u, const Real *v, Real *out, size_t n, int kind, double c0,
                                  double c1, double c2, double c3, double c4) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const Real a = u[i];
    Real r;
    if (kind == 0) {
      r = a * a * a;
    } else if (kind == 1) {
      const Real b = v[i];
      r = b * b * (Real(c0) + Real(c1) * b + Real(c2) * b * b);
    } else {
      const Real b = v[i];
      r = a * a * (Real(c0) + Real(c1) * a) + b * b * (Real(c2) + Real(c3) * b) - Real(c4) * a;
    }
    out[i] = r;
  }
}

// lam += dN/du (u, v) w  and  g = dN/dv (u, v) w  (g unused for the plain model)
template <typename Real>
__global__ void adj_jacobian_kernel(const Real *u, const Real *v, const Real *w, Real *lam, Real *g, size_t n,
                                    int kind, double c0, double c1, double c2, double c3, double c4) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const Real a = u[i], x = w[i];
    if (kind == 0) {
      lam[i] += Real(3) * a * a * x;  // d(psi^3)/dpsi
    } else if (kind == 1) {
      const Real b = v[i];  // d(c0 v^2 + c1 v^3 + c2 v^4)/dv
      g[i] = b * (Real(2 * c0) + Real(3 * c1) * b + Real(4 * c2) * b * b) * x;
    } else {
      const Real b = v[i];
      lam[i] += (a * (Real(2 * c0) + Real(3 * c1) * a) - Real(c4)) * x;  // dN/du
      g[i] = b * (Real(2 * c2) + Real(3 * c3) * b) * x;                  // dN/dv
    }
  }
}

template <typename Real>
__global__ void adj_add_kernel(Real *lam, const Real *x, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    lam[i] += x[i];
}

// U = opL lam_hat (in place over lam_hat), V = opN lam_hat (over n_hat, after
// it is read), and (tar != nullptr) FP64 sums of w_kx Re(conj(lam_hat)(dA psi_hat
// + dB n_hat)) added to this block's running partial.
template <typename Real>
__global__ void adj_modes_kernel(typename opfc::Cx<Real>::T *lam_hat, const typename opfc::Cx<Real>::T *psi_hat,
                                 typename opfc::Cx<Real>::T *n_hat, const Real *ta, const Real *tb,
                                 const Real *tar, const Real *tbr, int M, long long nyq_off,
                                 double *partials) {
  __shared__ double red[256];
  const long long nc = nyq_off + nyq_off / M;
  double s = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nc;
       i += (long long)gridDim.x * blockDim.x) {
    const auto l = lam_hat[i];
    if (tar) {
      const auto p = psi_hat[i];
      const auto q = n_hat[i];
      const double ar = tar[i], br = tbr[i];
      const double gx = ar * p.x + br * q.x, gy = ar * p.y + br * q.y;
      const int kx = i < nyq_off ? (int)(i % M) : M;
      const double wgt = (kx == 0 || kx == M) ? 1.0 : 2.0;
      s += wgt * ((double)l.x * gx + (double)l.y * gy);
    }
    const Real a = ta[i], b = tb[i];
    lam_hat[i].x = a * l.x;
    lam_hat[i].y = a * l.y;
    n_hat[i].x = b * l.x;
    n_hat[i].y = b * l.y;
  }
  if (!tar) return;
  red[threadIdx.x] = s;
  __syncthreads();
  for (int hh = blockDim.x / 2; hh > 0; hh >>= 1) {
    if (threadIdx.x < hh) red[threadIdx.x] += red[threadIdx.x + hh];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] += red[0];
}

namespace {

const int kEltBlocks = 148 * 8;

// real `in` (device, compute precision) -> split-layout spectrum `out`
int fwd_real(opfc_handle *h, const void *in, void *out) {
  XLaunch X = x_base(h);
  X.mode = X_R2C;
  X.rin = in;
  X.out = out;
  LAUNCH_TRY(h, xpass(h, X));
  LAUNCH_TRY(h, col_plain(h, 1, -1, out, out));
  LAUNCH_TRY(h, col_plain(h, 2, -1, out, out));
  return OPFC_OK;
}

// split-layout spectrum `spec` (destroyed) -> real `out`, scaled by 1/N, + mean
int bwd_real(opfc_handle *h, void *spec, void *out, double mean) {
  LAUNCH_TRY(h, col_plain(h, 2, +1, spec, spec));
  LAUNCH_TRY(h, col_plain(h, 1, +1, spec, spec));
  XLaunch X = x_base(h);
  X.mode = X_C2R;
  X.in0 = spec;
  X.rout = out;
  X.mean = mean;
  LAUNCH_TRY(h, xpass(h, X));
  return OPFC_OK;
}

// phi'(x) for phi(x) = (e^x - 1)/x, stable near 0
double dphi(double x) {
  if (std::fabs(x) < 1e-4) return 0.5 + x / 3.0 + x * x / 8.0 + x * x * x / 30.0;
  return (x * std::exp(x) - std::expm1(x)) / (x * x);
}

// models whose operators depend on r (L = -k^2 (r + (1 - k^2)^2))
bool has_r(const opfc_handle *h) {
  return h->desc.model == OPFC_MODEL_PLAIN || h->desc.model == OPFC_MODEL_FILTERED;
}

// nonlinearity kind and coefficients of the adjoint kernels
int adj_kind(const opfc_handle *h, double c[5]) {
  const int model = h->desc.model;
  for (int i = 0; i < 5; ++i) c[i] = 0.0;
  if (model == OPFC_MODEL_PLAIN) return 0;
  if (model == OPFC_MODEL_FILTERED || user_ops_model(model)) {
    c[0] = h->desc.p2 / 2.0;
    c[1] = h->desc.p3 / 3.0;
    c[2] = h->desc.p4 / 4.0;
    return 1;
  }
  if (model == OPFC_MODEL_ALUMINUM) {  // as the forward x pass (G_grid = 0)
    const opfc_aluminum_params &p = h->desc.aluminum;
    c[0] = p.p3_bar;
    c[1] = p.p4_bar;
    c[2] = p.q31_bar * p.T_const / p.T0 + p.q30_bar;
    c[3] = p.q4_bar;
    c[4] = p.stabP;
    return 2;
  }
  const opfc_tungsten_params &p = h->desc.tungsten;  // tungsten_params.hpp:339-411
  const double tau = p.T / p.T0;
  c[0] = p.shift_u * (p.p3 + 3 * p.shift_s * p.p4);
  c[1] = std::pow(p.shift_u, 2) * p.p4;
  c[2] = p.shift_u * p.q31 * tau + p.shift_u * (p.q30 + 3.0 * p.shift_s * p.q40);
  c[3] = std::pow(p.shift_u, 2) * p.q40;
  c[4] = p.stabP;
  return 2;
}

int adjoint_tables(opfc_handle *h) {
  if (!has_r(h)) return OPFC_OK;  // no r-derivative tables
  const int n0 = h->n0, n1 = h->n1, n2 = h->n2, H = h->M + 1;
  const double f0 = 2.0 * kPi / (h->desc.dx[0] * n0);
  const double f1 = 2.0 * kPi / (h->desc.dx[1] * n1);
  const double f2 = 2.0 * kPi / (h->desc.dx[2] * n2);
  const double r = h->desc.r, dt = h->dt;
  std::vector<double> ar(h->nc), br(h->nc);
  auto kc = [](int i, int n, double f) { return (i <= n / 2) ? i * f : (i - n) * f; };
  parallel_for((long)n2 * n1, [&](long row) {
    const int ky = (int)(row % n1), kz = (int)(row / n1);
    for (int kx = 0; kx < H; ++kx) {
      const double a = kc(kx, n0, f0), b = kc(ky, n1, f1), c = kc(kz, n2, f2);
      const double k2 = a * a + b * b + c * c;
      const double L = -k2 * (r + (1.0 - k2) * (1.0 - k2));
      const size_t o = split_index(h, kx, ky, kz);
      ar[o] = -k2 * dt * std::exp(L * dt);
      br[o] = dt * dt * k2 * k2 * dphi(L * dt);
    }
  });
  for (int t = 0; t < 2; ++t) {
    void **dst = t == 0 ? &h->tab_ar : &h->tab_br;
    std::vector<double> &src = t == 0 ? ar : br;
    if (!*dst) {
      int rc = dev_alloc(h, dst, h->nc * h->rsz);
      if (rc) return rc;
    }
    if (h->prec == OPFC_FP64) {
      CUDA_TRY(h, cudaMemcpy(*dst, src.data(), h->nc * 8, cudaMemcpyHostToDevice));
    } else {
      std::vector<float> f(src.begin(), src.end());
      CUDA_TRY(h, cudaMemcpy(*dst, f.data(), h->nc * 4, cudaMemcpyHostToDevice));
    }
  }
  return OPFC_OK;
}

int copy_state(opfc_handle *h, void *dst, const void *src) {
  CUDA_TRY(h, cudaMemcpyAsync(dst, src, h->nc * 2 * h->rsz, cudaMemcpyDeviceToDevice, h->stream));
  return OPFC_OK;
}

int adjoint_buffers(opfc_handle *h) {
  int rc;
  for (auto &p : h->adj_c)
    if (!p && (rc = dev_alloc(h, &p, h->nc * 2 * h->rsz))) return rc;
  for (auto &p : h->adj_r)
    if (!p && (rc = dev_alloc(h, &p, h->nr * h->rsz))) return rc;
  while ((int)h->seg.size() < h->ckpt_K) {
    void *p = nullptr;
    if ((rc = dev_alloc(h, &p, h->nc * 2 * h->rsz))) return rc;
    h->seg.push_back(p);
  }
  return OPFC_OK;
}

template <typename Real, typename K, typename... A> int elt(opfc_handle *h, K k, A... args) {
  k<<<kEltBlocks, 256, 0, h->stream>>>(args...);
  CUDA_TRY(h, cudaGetLastError());
  return OPFC_OK;
}

// lambda (adj_r[0]) <- adjoint of the step taken from psi_hat_n; for the models
// with r the step's dLoss/dr terms are added to the running per-block FP64
// partials (h->partials, summed once at the end).
int adjoint_step(opfc_handle *h, const void *psi_hat_n) {
  void *lam = h->adj_r[0], *u = h->adj_r[1], *tmp = h->adj_r[2], *v = h->adj_r[3];
  void *c0 = h->adj_c[0], *c1 = h->adj_c[1];
  const bool f64 = h->prec == OPFC_FP64;
  double cf[5];
  const int kind = adj_kind(h, cf);
  const double mean = mean_density(h);
  int rc;
  // u = psi_n, v = C psi_n in real space; N_hat_n = F[N(u, v)]
  if ((rc = copy_state(h, c0, psi_hat_n))) return rc;
  if ((rc = bwd_real(h, c0, u, mean))) return rc;
  if (kind != 0) {
    if ((rc = opfc_scale_by_table(h, psi_hat_n, h->tab_chi, c0))) return rc;
    if ((rc = bwd_real(h, c0, v, mean))) return rc;  // chi(0) = 1: the mean passes the filter
  }
  if (f64)
    rc = elt<double>(h, adj_nonlin_kernel<double>, (const double *)u, (const double *)v, (double *)tmp, h->nr,
                     kind, cf[0], cf[1], cf[2], cf[3], cf[4]);
  else
    rc = elt<float>(h, adj_nonlin_kernel<float>, (const float *)u, (const float *)v, (float *)tmp, h->nr, kind,
                    cf[0], cf[1], cf[2], cf[3], cf[4]);
  if (rc) return rc;
  if ((rc = fwd_real(h, tmp, c1))) return rc;
  // lambda_hat = F[lambda_{n+1}]; c0 <- opL lambda_hat, c1 <- opN lambda_hat
  if ((rc = fwd_real(h, lam, c0))) return rc;
  const bool dr = has_r(h);
  if (f64)
    adj_modes_kernel<double><<<h->npartials, 256, 0, h->stream>>>(
        (double2 *)c0, (const double2 *)psi_hat_n, (double2 *)c1, (const double *)h->tab_a,
        (const double *)h->tab_b, dr ? (const double *)h->tab_ar : nullptr, (const double *)h->tab_br, h->M,
        h->nyq_off, h->partials);
  else
    adj_modes_kernel<float><<<h->npartials, 256, 0, h->stream>>>(
        (float2 *)c0, (const float2 *)psi_hat_n, (float2 *)c1, (const float *)h->tab_a, (const float *)h->tab_b,
        dr ? (const float *)h->tab_ar : nullptr, (const float *)h->tab_br, h->M, h->nyq_off, h->partials);
  CUDA_TRY(h, cudaGetLastError());
  // lam = A lambda ; tmp = w = B lambda ; lam += dN/du w ; v <- g = dN/dv w
  if ((rc = bwd_real(h, c0, lam, 0.0))) return rc;
  if ((rc = bwd_real(h, c1, tmp, 0.0))) return rc;
  if (f64)
    rc = elt<double>(h, adj_jacobian_kernel<double>, (const double *)u, (const double *)v, (const double *)tmp,
                     (double *)lam, (double *)v, h->nr, kind, cf[0], cf[1], cf[2], cf[3], cf[4]);
  else
    rc = elt<float>(h, adj_jacobian_kernel<float>, (const float *)u, (const float *)v, (const float *)tmp,
                    (float *)lam, (float *)v, h->nr, kind, cf[0], cf[1], cf[2], cf[3], cf[4]);
  if (rc) return rc;
  if (kind != 0) {  // lam += C g: the adjoint of the mean-field filter is the filter
    if ((rc = fwd_real(h, v, c0))) return rc;
    if ((rc = opfc_scale_by_table(h, c0, h->tab_chi, c0))) return rc;
    if ((rc = bwd_real(h, c0, tmp, 0.0))) return rc;
    if (f64)
      rc = elt<double>(h, adj_add_kernel<double>, (double *)lam, (const double *)tmp, h->nr);
    else
      rc = elt<float>(h, adj_add_kernel<float>, (float *)lam, (const float *)tmp, h->nr);
    if (rc) return rc;
  }
  return OPFC_OK;
}

}  // namespace

extern "C" {

int opfc_set_r(opfc_handle *h, double r) {
  if (!h) return OPFC_ERR_ARG;
  if (two_field(h->desc.model) || user_ops_model(h->desc.model))
    return fail(h, OPFC_ERR_ARG, "r is not a parameter of this model");
  h->desc.r = r;
  release_graph(h);
  h->ckpt_steps = 0;
  if (h->initialized) return opfc_initialize(h, h->dt);
  return OPFC_OK;
}

int opfc_forward_checkpointed(opfc_handle *h, int n_steps, int K) {
  if (!h) return OPFC_ERR_ARG;
  if (h->al_grad)
    return fail(h, OPFC_ERR_ARG, "no adjoint for the Aluminum model with a moving temperature gradient");
  if (n_steps < 1 || K < 1) return fail(h, OPFC_ERR_ARG, "need n_steps >= 1 and K >= 1");
  if (!h->initialized || !h->have_state) return fail(h, OPFC_ERR_STATE, "need tables and a state");
  CUDA_TRY(h, cudaSetDevice(h->device));
  const int nck = (n_steps + K - 1) / K + 1;  // segment starts + final state
  int rc;
  while ((int)h->ckpt.size() < nck) {
    void *p = nullptr;
    if ((rc = dev_alloc(h, &p, h->nc * 2 * h->rsz))) return rc;
    h->ckpt.push_back(p);
  }
  for (int s = 0; s < n_steps; ++s) {
    if (s % K == 0 && (rc = copy_state(h, h->ckpt[s / K], h->psi_hat))) return rc;
    if ((rc = opfc_step(h, 1))) return rc;
  }
  if ((rc = copy_state(h, h->ckpt[nck - 1], h->psi_hat))) return rc;
  h->ckpt_K = K;
  h->ckpt_steps = n_steps;
  return opfc_sync(h);
}

int opfc_adjoint(opfc_handle *h, const void *grad_psi_T, int dtype, int where, void *grad_psi0,
                 double *grad_r, double *grad_n0) {
  if (!h || !grad_psi_T || !grad_psi0 || !grad_r || !grad_n0)
    return h ? fail(h, OPFC_ERR_ARG, "null pointer") : OPFC_ERR_ARG;
  int rc;
  if ((rc = check_dtype_where(h, dtype, where))) return rc;
  if (h->ckpt_steps < 1) return fail(h, OPFC_ERR_STATE, "run opfc_forward_checkpointed first");
  CUDA_TRY(h, cudaSetDevice(h->device));
  if ((rc = adjoint_tables(h))) return rc;  // r or dt may have changed since the last call
  if ((rc = adjoint_buffers(h))) return rc;
  // lambda_T = dLoss/dpsi_T
  if ((rc = real_in(h, grad_psi_T, dtype, where))) return rc;
  CUDA_TRY(h, cudaMemcpyAsync(h->adj_r[0], h->real_buf, h->nr * h->rsz, cudaMemcpyDeviceToDevice, h->stream));
  const int K = h->ckpt_K, n = h->ckpt_steps;
  const int nseg = (n + K - 1) / K;
  CUDA_TRY(h, cudaMemsetAsync(h->partials, 0, sizeof(double) * h->npartials, h->stream));
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int len = std::min(K, n - sg * K);
    // recompute the segment's states with the forward step itself
    if ((rc = copy_state(h, h->psi_hat, h->ckpt[sg]))) return rc;
    h->a_valid = false;
    for (int i = 0; i < len; ++i) {
      if ((rc = copy_state(h, h->seg[i], h->psi_hat))) return rc;
      if ((rc = opfc_step(h, 1))) return rc;
    }
    for (int i = len - 1; i >= 0; --i)
      if ((rc = adjoint_step(h, h->seg[i]))) return rc;
  }
  double dr = std::nan("");  // not a parameter of the model
  if (has_r(h)) {
    std::vector<double> part(h->npartials);
    CUDA_TRY(h, cudaMemcpyAsync(part.data(), h->partials, sizeof(double) * h->npartials, cudaMemcpyDeviceToHost,
                                h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    dr = neumaier(part.data(), part.size()) / (double)h->nr;
  }
  // leave the handle at the end state of the forward run
  if ((rc = copy_state(h, h->psi_hat, h->ckpt[nseg]))) return rc;
  h->a_valid = false;
  CUDA_TRY(h, cudaMemcpyAsync(h->real_buf, h->adj_r[0], h->nr * h->rsz, cudaMemcpyDeviceToDevice, h->stream));
  if ((rc = device_sum(h, 1, grad_n0))) return rc;  // psi0 = n0 + noise: dLoss/dn0 = sum lambda_0
  *grad_r = dr;
  if ((rc = real_out(h, grad_psi0, dtype, where))) return rc;
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return opfc_sync(h);
}

}  // extern "C"
