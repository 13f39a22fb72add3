// ensemble.cu -- C ABI of the uneven-size ensemble (include/openpfc_b200.h,
// opfc_ensemble_*): independent plain-PFC fields of different sizes and
// parameters advanced together, one persistent kernel per stage, the step loop
// captured in one CUDA graph, tile shapes picked by the autotuner.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/openpfc_b200.h"
#include "autotune.h"
#include "ensemble.cuh"
#include "twiddle.h"

using namespace opfc;

namespace {

bool ens_len_ok(int n) { return n == 16 || n == 32 || n == 48 || n == 64 || n == 80 || n == 96 || n == 128; }
bool ens_half_ok(int m) { return m == 16 || m == 24 || m == 32 || m == 40 || m == 48 || m == 64; }

constexpr int kVariants = 6;  // tile width W in {16, 8} x CTAs per SM in {4, 8, 16}
int var_w(int v) { return v < 3 ? 16 : 8; }
int var_g(int v) { return 4 << (v % 3); }

}  // namespace

struct opfc_ensemble {
  int count = 0;
  int prec = OPFC_FP32;
  size_t rsz = 4;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 148;
  std::vector<opfc_desc> desc;
  std::vector<EnsInst> inst;
  size_t nc_total = 0, nr_max = 0;
  double dt = 0;
  bool initialized = false, a_valid = false;
  std::vector<bool> have_state;
  void *psi_hat = nullptr, *work = nullptr, *tw = nullptr;
  void *real_buf = nullptr;
  EnsInst *d_inst = nullptr;
  int *d_prefix[3] = {nullptr, nullptr, nullptr};  // y col, z col, x tiles (per W variant)
  int total[2][3] = {};                           // [W = 16, 8][stage]
  int *d_prefix8[3] = {nullptr, nullptr, nullptr};
  // members per stage kind (y columns, z columns, x rows) sorted by that
  // stage's line length, longest first: CTAs that run at the same time then
  // run the same length's code (one kernel holds every length's unrolled
  // transforms; mixing them thrashed the instruction cache) and the longest
  // tiles start first
  int *d_order[3] = {nullptr, nullptr, nullptr};
  unsigned *flag = nullptr;
  int var_col = 0, var_x = 0, var_upd = 0;  // y passes, x pass, z update
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  std::string err;
  std::string key;
};

namespace {

int efail(opfc_ensemble *e, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  e->err = buf;
  return code;
}

#define ECUDA(e, expr)                                                                        \
  do {                                                                                        \
    cudaError_t x_ = (expr);                                                                  \
    if (x_ != cudaSuccess) return efail(e, OPFC_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(x_)); \
  } while (0)

int ealloc(opfc_ensemble *e, void **p, size_t bytes) {
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return efail(e, OPFC_ERR_OOM, "cudaMalloc(%zu) failed", bytes);
  }
  return OPFC_OK;
}

int col_tiles(const EnsInst &in, int axis, int W) {
  const int n_outer = axis == 1 ? in.n2 : in.n1;
  const int ncols = axis == 1 ? in.n2 : in.n1;
  return ((in.M + W - 1) / W) * n_outer + (ncols + W - 1) / W;
}
int x_tiles(const EnsInst &in, int W) { return (in.n1 * in.n2 + W - 1) / W; }

EnsArgs args(opfc_ensemble *e, const int *prefix, const int *order) {
  EnsArgs a;
  a.inst = e->d_inst;
  a.count = e->count;
  a.prefix = prefix;
  a.order = order;
  a.work = e->work;
  a.psi_hat = e->psi_hat;
  a.dt = e->dt;
  a.tw = e->tw;
  a.flag = e->flag;
  return a;
}

// stage kernels: ensemble_f32.cu / ensemble_f64.cu
int launch_stage(opfc_ensemble *e, int stage, int variant) {
  const int W = var_w(variant), G = var_g(variant);
  const int wi = W == 16 ? 0 : 1;
  const int *const *pre = wi == 0 ? e->d_prefix : e->d_prefix8;
  // prefix sums per stage: y columns (YI, YF), z columns (ZU), x rows (X)
  const int which = stage == 1 ? 2 : (stage == 3 ? 1 : 0);
  const int *p = stage == 4 ? nullptr : pre[which];
  // the Hermitian fix takes the largest instance's n1 * n2 in place of a tile count
  int tiles = stage == 4 ? 0 : e->total[wi][which];
  if (stage == 4)
    for (const auto &in : e->inst) tiles = std::max(tiles, in.n1 * in.n2);
  const EnsArgs a = args(e, p, stage == 4 ? nullptr : e->d_order[which]);
  return e->prec == OPFC_FP64 ? ens_launch_stage<double>(stage, W, G, e->num_sms, tiles, e->count, a, e->stream)
                              : ens_launch_stage<float>(stage, W, G, e->num_sms, tiles, e->count, a, e->stream);
}

int enqueue_step(opfc_ensemble *e) {
  const int v[5] = {e->var_col, e->var_x, e->var_col, e->var_upd, 0};
  for (int s = 0; s < 5; ++s) {
    const int rc = launch_stage(e, s, v[s]);
    if (rc) return efail(e, OPFC_ERR_CUDA, "ensemble stage %d: %s", s, cudaGetErrorString((cudaError_t)rc));
  }
  return OPFC_OK;
}

// ColLaunch for one instance's y or z pass (direct kernels), in place on `arr`
ColLaunch inst_col(opfc_ensemble *e, const EnsInst &in, int axis, int dir, void *arr, const void *src) {
  const int W = e->prec == OPFC_FP64 ? 8 : 16;
  ColLaunch L{};
  ColSeg &a = L.seg[0];
  ColSeg &b = L.seg[1];
  const int M = in.M, n1 = in.n1, n2 = in.n2;
  a.col_stride = 1;
  a.ncols = M;
  a.tiles_inner = (M + W - 1) / W;
  b.off = (long long)M * n1 * n2;
  if (axis == 1) {
    a.s_outer = (long long)M * n1;
    a.fft_stride = M;
    a.ntiles = a.tiles_inner * n2;
    b.fft_stride = 1;
    b.col_stride = n1;
    b.ncols = n2;
  } else {
    a.s_outer = M;
    a.fft_stride = (long long)M * n1;
    a.ntiles = a.tiles_inner * n1;
    b.fft_stride = n1;
    b.col_stride = 1;
    b.ncols = n1;
  }
  b.tiles_inner = (b.ncols + W - 1) / W;
  b.ntiles = b.tiles_inner;
  L.nseg = 2;
  L.N = axis == 1 ? n1 : n2;
  L.dir = dir;
  L.mode = COL_PLAIN;
  L.nsets = 1;
  L.in[0] = L.in[1] = src;
  L.out[0] = L.out[1] = arr;
  const size_t cs = 2 * e->rsz;
  L.tw = static_cast<char *>(e->tw) + (size_t)(axis == 1 ? in.tw1 : in.tw2) * cs;
  L.axis = axis;
  return L;
}

int col_run(opfc_ensemble *e, const ColLaunch &L) {
  const int rc = e->prec == OPFC_FP64 ? launch_col<double>(L, e->stream) : launch_col<float>(L, e->stream);
  return rc ? efail(e, OPFC_ERR_CUDA, "instance column pass: %s", cudaGetErrorString((cudaError_t)rc)) : OPFC_OK;
}

XLaunch inst_x(opfc_ensemble *e, const EnsInst &in) {
  XLaunch X{};
  X.M = in.M;
  X.rows = in.n1 * in.n2;
  X.nyq_off = (long long)in.M * in.n1 * in.n2;
  X.tw = static_cast<char *>(e->tw) + (size_t)in.tw0 * 2 * e->rsz;
  X.scale = 1.0 / ((double)in.n0 * in.n1 * in.n2);
  X.flag = e->flag;
  return X;
}

int x_run(opfc_ensemble *e, const XLaunch &X) {
  const int rc = e->prec == OPFC_FP64 ? launch_x<double>(X, e->stream) : launch_x<float>(X, e->stream);
  return rc ? efail(e, OPFC_ERR_CUDA, "instance x pass: %s", cudaGetErrorString((cudaError_t)rc)) : OPFC_OK;
}

void *at(opfc_ensemble *e, void *base, const EnsInst &in) {
  return static_cast<char *>(base) + (size_t)in.off_c * 2 * e->rsz;
}

int prepare_a(opfc_ensemble *e) {
  for (const auto &in : e->inst) {
    int rc = col_run(e, inst_col(e, in, 2, +1, at(e, e->work, in), at(e, e->psi_hat, in)));
    if (rc) return rc;
  }
  e->a_valid = true;
  return OPFC_OK;
}

void drop_graph(opfc_ensemble *e) {
  if (e->graph) cudaGraphExecDestroy(e->graph);
  e->graph = nullptr;
  e->graph_steps = 0;
}

double neumaier_sum(const double *a, size_t n) {
  double s = 0, c = 0;
  for (size_t i = 0; i < n; ++i) {
    const double t = s + a[i];
    c += (std::fabs(s) >= std::fabs(a[i])) ? (s - t) + a[i] : (a[i] - t) + s;
    s = t;
  }
  return s + c;
}

}  // namespace

extern "C" {

const char *opfc_ensemble_last_error(const opfc_ensemble *e) { return e ? e->err.c_str() : "null ensemble"; }

int opfc_ensemble_destroy(opfc_ensemble *e) {
  if (!e) return OPFC_ERR_ARG;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  drop_graph(e);
  void *bufs[] = {e->psi_hat, e->work, e->tw, e->real_buf, e->d_inst, e->flag,
                  e->d_prefix[0], e->d_prefix[1], e->d_prefix[2], e->d_prefix8[0], e->d_prefix8[1],
                  e->d_prefix8[2], e->d_order[0], e->d_order[1], e->d_order[2]};
  for (void *p : bufs)
    if (p) cudaFree(p);
  if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return OPFC_OK;
}

int opfc_ensemble_create(int count, const opfc_desc *descs, opfc_ensemble **out) {
  if (!out || !descs || count < 1) return OPFC_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<opfc_ensemble> e(new opfc_ensemble);
  e->count = count;
  e->prec = descs[0].precision;
  e->rsz = e->prec == OPFC_FP64 ? 8 : 4;
  e->device = descs[0].device;
  e->desc.assign(descs, descs + count);
  for (int i = 0; i < count; ++i) {
    const opfc_desc &d = descs[i];
    if (d.model != OPFC_MODEL_PLAIN || d.precision != e->prec || d.device != e->device) return OPFC_ERR_ARG;
    if (d.n[0] % 2 || !ens_half_ok(d.n[0] / 2) || !ens_len_ok(d.n[1]) || !ens_len_ok(d.n[2]))
      return OPFC_ERR_SIZE;
  }
  if (cudaSetDevice(e->device) != cudaSuccess) return OPFC_ERR_CUDA;
  if (descs[0].stream) {
    e->stream = (cudaStream_t)descs[0].stream;
  } else {
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) return OPFC_ERR_CUDA;
    e->own_stream = true;
  }
  cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, e->device);
  // instance layout and the distinct twiddle tables
  std::vector<int> lens;
  auto tw_off = [&](int n) {
    int off = 0;
    for (int l : lens) {
      if (l == n) return off;
      off += l;
    }
    lens.push_back(n);
    return off;
  };
  size_t off = 0;
  e->inst.resize(count);
  char sig[64];
  std::string key = e->prec == OPFC_FP64 ? "ens/fp64/" : "ens/fp32/";
  for (int i = 0; i < count; ++i) {
    EnsInst &in = e->inst[i];
    in.n0 = descs[i].n[0];
    in.n1 = descs[i].n[1];
    in.n2 = descs[i].n[2];
    in.M = in.n0 / 2;
    in.off_c = (long long)off;
    in.tw0 = tw_off(in.n0);
    in.tw1 = tw_off(in.n1);
    in.tw2 = tw_off(in.n2);
    in.mean = 0;
    for (int a = 0; a < 3; ++a) in.kf[a] = 2.0 * 3.14159265358979323846 / (descs[i].dx[a] * descs[i].n[a]);
    in.r = descs[i].r;
    off += (size_t)(in.M + 1) * in.n1 * in.n2;
    e->nr_max = std::max(e->nr_max, (size_t)in.n0 * in.n1 * in.n2);
  }
  std::snprintf(sig, sizeof sig, "count%d_modes%zu", count, off);
  e->key = key + sig;
  e->nc_total = off;
  e->have_state.assign(count, false);
  opfc_ensemble *ep = e.get();
  auto bail = [&](int rc) {
    opfc_ensemble_destroy(e.release());
    return rc;
  };
  int rc;
  const size_t cb = off * 2 * e->rsz;
  if ((rc = ealloc(ep, &ep->psi_hat, cb)) || (rc = ealloc(ep, &ep->work, cb)) ||
      (rc = ealloc(ep, &ep->real_buf, e->nr_max * e->rsz)) ||
      (rc = ealloc(ep, (void **)&ep->d_inst, sizeof(EnsInst) * count)) ||
      (rc = ealloc(ep, (void **)&ep->flag, sizeof(unsigned))))
    return bail(rc);
  size_t twn = 0;
  for (int l : lens) twn += l;
  if ((rc = ealloc(ep, &ep->tw, twn * 2 * e->rsz))) return bail(rc);
  std::vector<double> twh;
  for (int l : lens) {
    std::vector<double> t = twiddle_table(l);
    twh.insert(twh.end(), t.begin(), t.end());
  }
  if (e->prec == OPFC_FP64) {
    if (cudaMemcpy(ep->tw, twh.data(), twh.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess) return bail(OPFC_ERR_CUDA);
  } else {
    std::vector<float> f(twh.begin(), twh.end());
    if (cudaMemcpy(ep->tw, f.data(), f.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) return bail(OPFC_ERR_CUDA);
  }
  std::vector<int> order[3];
  for (int st = 0; st < 3; ++st) {
    auto len = [&](int i) { const EnsInst &in = e->inst[i]; return st == 0 ? in.n1 : (st == 1 ? in.n2 : in.M); };
    order[st].resize(count);
    for (int i = 0; i < count; ++i) order[st][i] = i;
    std::stable_sort(order[st].begin(), order[st].end(), [&](int x, int y) { return len(x) > len(y); });
    if ((rc = ealloc(ep, (void **)&ep->d_order[st], sizeof(int) * count))) return bail(rc);
    if (cudaMemcpy(ep->d_order[st], order[st].data(), sizeof(int) * count, cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(OPFC_ERR_CUDA);
  }
  for (int wi = 0; wi < 2; ++wi) {
    const int W = wi == 0 ? 16 : 8;
    for (int st = 0; st < 3; ++st) {
      std::vector<int> pre(count + 1, 0);
      for (int k = 0; k < count; ++k) {
        const EnsInst &in = e->inst[order[st][k]];
        pre[k + 1] = pre[k] + (st < 2 ? col_tiles(in, st + 1, W) : x_tiles(in, W));
      }
      ep->total[wi][st] = pre[count];
      int **dst = wi == 0 ? &ep->d_prefix[st] : &ep->d_prefix8[st];
      if ((rc = ealloc(ep, (void **)dst, sizeof(int) * (count + 1)))) return bail(rc);
      if (cudaMemcpy(*dst, pre.data(), sizeof(int) * (count + 1), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(OPFC_ERR_CUDA);
    }
  }
  if (cudaMemset(ep->flag, 0, sizeof(unsigned)) != cudaSuccess || cudaMemset(ep->psi_hat, 0, cb) != cudaSuccess ||
      cudaMemset(ep->work, 0, cb) != cudaSuccess)
    return bail(OPFC_ERR_CUDA);
  // every instance's descriptor is on the device from the start (set_psi
  // refreshes its mean), so the stage kernels -- and the autotuner timing
  // them before any state is set -- walk every member's tiles
  if (cudaMemcpy(ep->d_inst, ep->inst.data(), sizeof(EnsInst) * count, cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(OPFC_ERR_CUDA);
  // dynamic shared memory above 48 KB is never needed (N <= 128)
  // cached choices come from a file: out-of-range entries fall back to variant 0
  auto cached = [&](const char *stage) {
    const int v = AutoTuner::instance().get_config(ep->key + stage, 0);
    return (v >= 0 && v < kVariants) ? v : 0;
  };
  ep->var_col = cached("/col");
  ep->var_x = cached("/x");
  ep->var_upd = cached("/upd");
  *out = e.release();
  return OPFC_OK;
}

int opfc_ensemble_initialize(opfc_ensemble *e, double dt) {
  if (!e) return OPFC_ERR_ARG;
  if (!(dt > 0)) return efail(e, OPFC_ERR_ARG, "dt must be positive");
  // the operators of every instance are computed per mode inside the z
  // update (10_complete_pfc_model.cpp:189-207 with opL = 1 + expm1(L dt),
  // opN = expm1(L dt) / (r + (1 - k^2)^2)) from its r, k steps and dt
  e->dt = dt;
  e->initialized = true;
  drop_graph(e);
  return OPFC_OK;
}

int opfc_ensemble_set_psi(opfc_ensemble *e, int i, const double *psi, size_t count) {
  if (!e || !psi || i < 0 || i >= e->count) return e ? efail(e, OPFC_ERR_ARG, "bad instance or pointer") : OPFC_ERR_ARG;
  EnsInst &in = e->inst[i];
  const size_t nr = (size_t)in.n0 * in.n1 * in.n2;
  if (count != nr) return efail(e, OPFC_ERR_SIZE, "instance %d: expected %zu values", i, nr);
  ECUDA(e, cudaSetDevice(e->device));
  in.mean = neumaier_sum(psi, nr) / (double)nr;
  if (e->prec == OPFC_FP64) {
    ECUDA(e, cudaMemcpyAsync(e->real_buf, psi, nr * 8, cudaMemcpyHostToDevice, e->stream));
  } else {
    std::vector<float> f(psi, psi + nr);
    ECUDA(e, cudaMemcpyAsync(e->real_buf, f.data(), nr * 4, cudaMemcpyHostToDevice, e->stream));
    ECUDA(e, cudaStreamSynchronize(e->stream));
  }
  XLaunch X = inst_x(e, in);
  X.mode = X_R2C;
  X.rin = e->real_buf;
  void *dst = at(e, e->psi_hat, in);
  X.out = dst;
  int rc;
  if ((rc = x_run(e, X))) return rc;
  if ((rc = col_run(e, inst_col(e, in, 1, -1, dst, dst)))) return rc;
  if ((rc = col_run(e, inst_col(e, in, 2, -1, dst, dst)))) return rc;
  ECUDA(e, cudaMemsetAsync(dst, 0, 2 * e->rsz, e->stream));  // mean carried in FP64
  ECUDA(e, cudaMemcpyAsync(e->d_inst + i, &in, sizeof(EnsInst), cudaMemcpyHostToDevice, e->stream));
  ECUDA(e, cudaStreamSynchronize(e->stream));
  e->have_state[i] = true;
  e->a_valid = false;
  return OPFC_OK;
}

int opfc_ensemble_get_psi(opfc_ensemble *e, int i, double *psi, size_t count) {
  if (!e || !psi || i < 0 || i >= e->count) return e ? efail(e, OPFC_ERR_ARG, "bad instance or pointer") : OPFC_ERR_ARG;
  const EnsInst &in = e->inst[i];
  const size_t nr = (size_t)in.n0 * in.n1 * in.n2;
  if (count != nr) return efail(e, OPFC_ERR_SIZE, "instance %d: expected %zu values", i, nr);
  ECUDA(e, cudaSetDevice(e->device));
  void *w = at(e, e->work, in);
  int rc;
  if ((rc = col_run(e, inst_col(e, in, 2, +1, w, at(e, e->psi_hat, in))))) return rc;
  if ((rc = col_run(e, inst_col(e, in, 1, +1, w, w)))) return rc;
  XLaunch X = inst_x(e, in);
  X.mode = X_C2R;
  X.in0 = w;
  X.rout = e->real_buf;
  X.mean = in.mean;
  if ((rc = x_run(e, X))) return rc;
  e->a_valid = false;
  if (e->prec == OPFC_FP64) {
    ECUDA(e, cudaMemcpyAsync(psi, e->real_buf, nr * 8, cudaMemcpyDeviceToHost, e->stream));
    ECUDA(e, cudaStreamSynchronize(e->stream));
  } else {
    std::vector<float> f(nr);
    ECUDA(e, cudaMemcpyAsync(f.data(), e->real_buf, nr * 4, cudaMemcpyDeviceToHost, e->stream));
    ECUDA(e, cudaStreamSynchronize(e->stream));
    for (size_t k = 0; k < nr; ++k) psi[k] = f[k];
  }
  return OPFC_OK;
}

int opfc_ensemble_step(opfc_ensemble *e, int n_steps) {
  if (!e || n_steps < 0) return OPFC_ERR_ARG;
  if (!e->initialized) return efail(e, OPFC_ERR_STATE, "opfc_ensemble_step before initialize");
  for (int i = 0; i < e->count; ++i)
    if (!e->have_state[i]) return efail(e, OPFC_ERR_STATE, "instance %d has no state", i);
  ECUDA(e, cudaSetDevice(e->device));
  int rc;
  if (!e->a_valid && (rc = prepare_a(e))) return rc;
  if (n_steps == 0) return OPFC_OK;  // step(0) only prepares the work arrays
  if (!e->graph || e->graph_steps != n_steps) {
    drop_graph(e);
    // the whole n-step loop is one graph: 5 kernels per step
    ECUDA(e, cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    for (int s = 0; s < n_steps && !rc; ++s) rc = enqueue_step(e);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ce != cudaSuccess) return efail(e, OPFC_ERR_CUDA, "capture: %s", cudaGetErrorString(ce));
    const cudaError_t ie = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return efail(e, OPFC_ERR_CUDA, "instantiate: %s", cudaGetErrorString(ie));
    e->graph_steps = n_steps;
  }
  ECUDA(e, cudaGraphLaunch(e->graph, e->stream));
  return OPFC_OK;
}

int opfc_ensemble_sync(opfc_ensemble *e) {
  if (!e) return OPFC_ERR_ARG;
  ECUDA(e, cudaSetDevice(e->device));
  ECUDA(e, cudaStreamSynchronize(e->stream));
  unsigned f = 0;
  ECUDA(e, cudaMemcpy(&f, e->flag, sizeof f, cudaMemcpyDeviceToHost));
  if (f) {
    cudaMemset(e->flag, 0, sizeof f);
    return efail(e, OPFC_ERR_NONFINITE, "non-finite value in an ensemble member");
  }
  return OPFC_OK;
}

int opfc_ensemble_autotune(opfc_ensemble *e, double *ms_col, double *ms_x, double *ms_upd) {
  if (!e) return OPFC_ERR_ARG;
  if (!e->initialized) return efail(e, OPFC_ERR_STATE, "initialize before tuning");
  ECUDA(e, cudaSetDevice(e->device));
  std::vector<double> mc, mx, mu;
  // the passes run in place on whatever the arrays hold; states are re-set after
  e->var_col = AutoTuner::instance().tune(e->key + "/col", kVariants,
                                          [&](int v) { return launch_stage(e, 2, v); }, e->stream, &mc);
  e->var_x = AutoTuner::instance().tune(e->key + "/x", kVariants, [&](int v) { return launch_stage(e, 1, v); },
                                        e->stream, &mx);
  e->var_upd = AutoTuner::instance().tune(e->key + "/upd", kVariants,
                                          [&](int v) { return launch_stage(e, 3, v); }, e->stream, &mu);
  ECUDA(e, cudaStreamSynchronize(e->stream));
  cudaMemset(e->flag, 0, sizeof(unsigned));
  for (int i = 0; i < e->count; ++i) e->have_state[i] = false;
  e->a_valid = false;
  drop_graph(e);
  if (ms_col)
    for (int v = 0; v < kVariants; ++v) ms_col[v] = mc.empty() ? -1 : mc[v];
  if (ms_x)
    for (int v = 0; v < kVariants; ++v) ms_x[v] = mx.empty() ? -1 : mx[v];
  if (ms_upd)
    for (int v = 0; v < kVariants; ++v) ms_upd[v] = mu.empty() ? -1 : mu[v];
  return OPFC_OK;
}

int opfc_ensemble_variants(const opfc_ensemble *e, int *var_col, int *var_x, int *var_upd) {
  if (!e || !var_col || !var_x || !var_upd) return OPFC_ERR_ARG;
  *var_col = e->var_col;
  *var_x = e->var_x;
  *var_upd = e->var_upd;
  return OPFC_OK;
}

size_t opfc_ensemble_cells(const opfc_ensemble *e) {
  if (!e) return 0;
  size_t s = 0;
  for (const auto &in : e->inst) s += (size_t)in.n0 * in.n1 * in.n2;
  return s;
}

void *opfc_ensemble_stream(const opfc_ensemble *e) { return e ? (void *)e->stream : nullptr; }

}  // extern "C"
