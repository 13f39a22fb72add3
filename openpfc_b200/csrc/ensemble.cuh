// ensemble.cuh -- one persistent kernel per stage for a batch of independent
// PFC fields of uneven sizes (parameter sweeps).
//
// Every stage (y inverse, fused x, y forward, fused z update, Hermitian fix)
// is a single launch over a flat list of (instance, tile) work items; a CTA
// finds its instance by binary search in the stage's tile prefix sums and
// branches on the instance's transform length to an inlined, fully unrolled
// FFT.  All sizes use the same CTA shape: W lines x 4 threads per line (each
// thread owns E = N/4 values), so the CTA-wide barriers of every branch match.
#pragma once
#include "kernels.cuh"

namespace opfc {

OPFC_EXTERN(float)
OPFC_EXTERN(double)

struct EnsInst {
  int n0, n1, n2, M;
  long long off_c;     // element offset of the instance's split-layout arrays
  int tw0, tw1, tw2;   // element offsets of its x (N0), y (N1), z (N2) twiddles
  int pad_;
  double mean;         // mean density (k = 0 mode, FP64)
  double kf[3];        // wavenumber steps 2 pi / (dx_a N_a)
  double r;            // the instance's r (operators computed per mode)
};

struct EnsArgs {
  const EnsInst *inst;
  int count;
  const int *prefix;   // tile prefix sums of this stage, count + 1 entries, in `order`
  const int *order;    // members in tile order (by line length), or nullptr
  void *work;          // F_z^-1 of the states / the step's working arrays
  void *psi_hat;       // states (DC slot zero)
  const void *tw;      // concatenated twiddle tables
  unsigned *flag;
  double dt;
};

constexpr int kEnsT = 4;  // threads per line

__device__ __forceinline__ int ens_find(const int *prefix, int count, int g) {
  int lo = 0, hi = count;  // prefix[lo] <= g < prefix[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= g)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Per-thread asynchronous copy of one complex value from global to shared
// memory (cp.async, 8 or 16 bytes); cp_async_wait_all() waits for this
// thread's copies only.
template <typename C> __device__ __forceinline__ void cp_async_value(C *dst, const C *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const size_t g = __cvta_generic_to_global(src);
  if constexpr (sizeof(C) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(g) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Column tile (y or z pass) of one instance; mirrors col_kernel's body.
// pbuf (z update only): N x W complex staging space for the tile's psi_hat.
template <typename Real, int N, int W, int MODE, int DIR>
__device__ __forceinline__ void ens_col_tile(const EnsArgs &a, const EnsInst &in, int axis, int t,
                                             typename Cx<Real>::T *tw, typename Cx<Real>::T *sm,
                                             typename Cx<Real>::T *pbuf, int &tw_cur) {
  using C = typename Cx<Real>::T;
  constexpr int E = N / kEnsT;
  constexpr int ld = W + 1;
  const int tid = threadIdx.x, c = tid % W, j = tid / W;
  const int M = in.M, n1 = in.n1, n2 = in.n2;
  const long long nyq = (long long)M * n1 * n2;
  // the CTA's previous tile usually had the same length (tiles are walked in
  // members sorted by length): reload the twiddles only when they change (the
  // previous tile's closing barrier orders the reuse of the shared arrays)
  const int two = axis == 1 ? in.tw1 : in.tw2;
  if (two != tw_cur) {
    const C *gtw = reinterpret_cast<const C *>(a.tw) + two;
    for (int i = tid; i < N; i += W * kEnsT) tw[i] = gtw[i];
    __syncthreads();
    tw_cur = two;
  }
  // main segment: columns kx, outer z (y pass) or y (z pass); then the Nyquist plane
  const int ti_main = (M + W - 1) / W;
  const int n_outer = axis == 1 ? n2 : n1;
  long long base;
  long long fs;
  bool ok;
  int kx, ky;  // z pass: the column's (kx, ky)
  if (t < ti_main * n_outer) {
    const int ti = t % ti_main, to = t / ti_main;
    const int cg = ti * W + c;
    ok = cg < M;
    base = (axis == 1 ? (long long)to * M * n1 : (long long)to * M) + cg;
    fs = axis == 1 ? M : (long long)M * n1;
    kx = cg;
    ky = to;
  } else {
    const int tn = t - ti_main * n_outer;
    const int cg = tn * W + c;
    const int ncols = axis == 1 ? n2 : n1;
    ok = cg < ncols;
    base = nyq + (axis == 1 ? (long long)cg * n1 : (long long)cg);
    fs = axis == 1 ? 1 : n1;
    kx = M;
    ky = cg;
  }
  C *work = reinterpret_cast<C *>(a.work) + in.off_c;
  C v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) v[m] = ok ? work[base + (long long)(j + kEnsT * m) * fs] : mk<C>(0, 0);
  if constexpr (MODE == COL_PLAIN) {
    fft_line_e<C, N, DIR, N>(v, sm, ld, c, j, tw);
  } else {
    // z update: psi_hat <- opL psi_hat + opN N_hat with opL, opN computed from
    // k^2 and the instance's r.  The tile's psi_hat values are loaded as one
    // batch -- before the transform when they fit in registers beside it -- so
    // the tile waits on memory once, not once per value.
    C *ph = reinterpret_cast<C *>(a.psi_hat) + in.off_c;
    // the tile's psi_hat is copied to shared memory while the forward
    // transform runs; each thread reads back only the values it copied
    if (ok) {
#pragma unroll
      for (int m = 0; m < E; ++m)
        cp_async_value(pbuf + (j + kEnsT * m) * W + c, ph + base + (long long)(j + kEnsT * m) * fs);
    }
    fft_line_e<C, N, -1, N>(v, sm, ld, c, j, tw);
    cp_async_wait_all();
    const int fy = ky <= n1 / 2 ? ky : n1 - ky;
    const Real qx = Real(in.kf[0]) * Real(kx), qy = Real(in.kf[1]) * Real(fy);
    const Real qxy = qx * qx + qy * qy;
    const Real kf2 = Real(in.kf[2]), r = Real(in.r), dt = Real(a.dt);
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int kz = j + kEnsT * m;
      const int fz = kz <= n2 / 2 ? kz : n2 - kz;
      const Real qz = kf2 * Real(fz);
      Real la, lb;
      ops_from_k2(qxy + qz * qz, r, dt, la, lb);
      const C pm = ok ? pbuf[kz * W + c] : mk<C>(0, 0);
      v[m] = mk<C>(la * pm.x + lb * v[m].x, la * pm.y + lb * v[m].y);
      if (ok) ph[base + (long long)kz * fs] = v[m];
    }
    fft_line_e<C, N, +1, N>(v, sm, ld, c, j, tw);
  }
  if (ok) {
#pragma unroll
    for (int m = 0; m < E; ++m) work[base + (long long)(j + kEnsT * m) * fs] = v[m];
  }
  __syncthreads();  // tw / sm are reused by the next tile
}

// G = CTAs per SM the kernel is compiled for (__launch_bounds__ minimum): one
// kernel serves every length, so its register budget would otherwise be set
// by the longest line (32 values per thread at N = 128); a larger G caps the
// registers (65536 / (G * threads)) and trades spills in the long branches for
// occupancy in the short ones.  The autotuner times every (W, G).
template <typename Real, int W, int MODE, int DIR, int G>
__global__ void __launch_bounds__(W *kEnsT, G) ens_col_kernel(const EnsArgs a, int axis) {
  using C = typename Cx<Real>::T;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *tw = reinterpret_cast<C *>(smraw);
  C *sm = tw + 128;
  C *pb = sm + 128 * (W + 1);  // z update: psi_hat staging (ens_col_smem)
  const int total = a.prefix[a.count];
  int tw_cur = -1;  // twiddle table offset held in tw
  int k = -1;  // position (in a.order) of the previous tile's member
  for (int g = blockIdx.x; g < total; g += gridDim.x) {
    // a CTA's tiles increase, so after the first search the position only advances
    if (k < 0)
      k = ens_find(a.prefix, a.count, g);
    else
      while (a.prefix[k + 1] <= g) ++k;
    const EnsInst in = a.inst[a.order ? a.order[k] : k];
    const int t = g - a.prefix[k];
    const int N = axis == 1 ? in.n1 : in.n2;
    switch (N) {
      case 16: ens_col_tile<Real, 16, W, MODE, DIR>(a, in, axis, t, tw, sm, pb, tw_cur); break;
      case 32: ens_col_tile<Real, 32, W, MODE, DIR>(a, in, axis, t, tw, sm, pb, tw_cur); break;
      case 48: ens_col_tile<Real, 48, W, MODE, DIR>(a, in, axis, t, tw, sm, pb, tw_cur); break;
      case 64: ens_col_tile<Real, 64, W, MODE, DIR>(a, in, axis, t, tw, sm, pb, tw_cur); break;
      case 80: ens_col_tile<Real, 80, W, MODE, DIR>(a, in, axis, t, tw, sm, pb, tw_cur); break;
      case 96: ens_col_tile<Real, 96, W, MODE, DIR>(a, in, axis, t, tw, sm, pb, tw_cur); break;
      case 128: ens_col_tile<Real, 128, W, MODE, DIR>(a, in, axis, t, tw, sm, pb, tw_cur); break;
      default: break;  // sizes are validated on the host
    }
  }
}

// Fused x tile (C2R -> psi^3 -> R2C) of W rows of one instance; mirrors x_kernel.
template <typename Real, int M, int W>
__device__ __forceinline__ void ens_x_tile(const EnsArgs &a, const EnsInst &in, int t,
                                           typename Cx<Real>::T *tw, typename Cx<Real>::T *buf,
                                           bool &bad, int &tw_cur) {
  using C = typename Cx<Real>::T;
  constexpr int E = M / kEnsT;
  constexpr int NT = W * kEnsT;
  constexpr int ld = W + 1;
  constexpr int N0 = 2 * M;
  const int tid = threadIdx.x, c = tid % W, j = tid / W;
  const int rows = in.n1 * in.n2;
  const long long nyq = (long long)M * rows;
  if (in.tw0 != tw_cur) {  // made visible by the barrier after the row loads
    const C *gtw = reinterpret_cast<const C *>(a.tw) + in.tw0;
    for (int i = tid; i < N0; i += NT) tw[i] = gtw[i];
    tw_cur = in.tw0;
  }
  C *work = reinterpret_cast<C *>(a.work) + in.off_c;
  const int row0 = t * W;
  x_load_rows<C, M, W, NT>(work, nyq, row0, rows, buf, tid);
  __syncthreads();
  C v[E];
  x_pre<C, M, W, E>(buf, tw, c, j, v);
  __syncthreads();
  fft_line_e<C, M, +1, N0>(v, buf, ld, c, j, tw);
  // normalisation and mean in the compute precision (as the single-grid x pass)
  const Real sc = Real(1.0 / ((double)in.n0 * rows)), mn = Real(in.mean);
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const Real x = v[m].x * sc + mn;
    const Real y = v[m].y * sc + mn;
    const Real nx = x * x * x, ny = y * y * y;
    bad |= !(isfinite(nx) && isfinite(ny));
    v[m] = mk<C>(nx, ny);
  }
  fft_line_e<C, M, -1, N0>(v, buf, ld, c, j, tw);
#pragma unroll
  for (int m = 0; m < E; ++m) buf[(j + kEnsT * m) * ld + c] = v[m];
  __syncthreads();
  x_post_store<C, M, W, NT>(buf, tw, work, nyq, row0, rows, tid);
  __syncthreads();
}

template <typename Real, int W, int G>
__global__ void __launch_bounds__(W *kEnsT, G) ens_x_kernel(const EnsArgs a) {
  using C = typename Cx<Real>::T;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *tw = reinterpret_cast<C *>(smraw);
  C *buf = tw + 128;
  const int total = a.prefix[a.count];
  bool bad = false;
  int tw_cur = -1;  // twiddle table offset held in tw
  int k = -1;  // position (in a.order) of the previous tile's member
  for (int g = blockIdx.x; g < total; g += gridDim.x) {
    // a CTA's tiles increase, so after the first search the position only advances
    if (k < 0)
      k = ens_find(a.prefix, a.count, g);
    else
      while (a.prefix[k + 1] <= g) ++k;
    const EnsInst in = a.inst[a.order ? a.order[k] : k];
    const int t = g - a.prefix[k];
    switch (in.M) {
      case 16: ens_x_tile<Real, 16, W>(a, in, t, tw, buf, bad, tw_cur); break;
      case 24: ens_x_tile<Real, 24, W>(a, in, t, tw, buf, bad, tw_cur); break;
      case 32: ens_x_tile<Real, 32, W>(a, in, t, tw, buf, bad, tw_cur); break;
      case 40: ens_x_tile<Real, 40, W>(a, in, t, tw, buf, bad, tw_cur); break;
      case 48: ens_x_tile<Real, 48, W>(a, in, t, tw, buf, bad, tw_cur); break;
      case 64: ens_x_tile<Real, 64, W>(a, in, t, tw, buf, bad, tw_cur); break;
      default: break;
    }
  }
  if (bad && a.flag) atomicOr(a.flag, 1u);
}

// Hermitian projection of every instance's kx = 0 and Nyquist planes.  One
// thread per mode of the two planes (blockIdx.y = instance; the grid's x extent
// covers the largest instance, so each thread makes one pass: the loop below
// runs more than once only for a grid sized smaller than that).
template <typename Real>
__global__ void ens_herm_kernel(const EnsArgs a) {
  using C = typename Cx<Real>::T;
  const int i = blockIdx.y;
  const EnsInst in = a.inst[i];
  const long long plane = (long long)in.n1 * in.n2;
  if ((long long)blockIdx.x * blockDim.x >= 2 * plane) return;
  C *psi = reinterpret_cast<C *>(a.psi_hat) + in.off_c;
  const long long nyq = (long long)in.M * plane;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < 2 * plane;
       e += (long long)gridDim.x * blockDim.x) {
    const bool second = e >= plane;
    const long long q = second ? e - plane : e;
    const int y = (int)(q % in.n1), z = (int)(q / in.n1);
    const long long p = (long long)((in.n1 - y) % in.n1) + (long long)in.n1 * ((in.n2 - z) % in.n2);
    C *P = second ? psi + nyq : psi;
    const long long st = second ? 1 : in.M;
    if (q < p) {
      const C u = P[q * st], w = P[p * st];
      const C h = mk<C>(Real(0.5) * (u.x + w.x), Real(0.5) * (u.y - w.y));
      P[q * st] = h;
      P[p * st] = mk<C>(h.x, -h.y);
    } else if (q == p) {
      P[q * st].y = 0;
    }
  }
}

// largest dynamic shared memory any ensemble kernel needs (N, M <= 128 / 64)
template <typename Real, int W, int MODE = COL_PLAIN> constexpr size_t ens_col_smem() {
  return sizeof(typename Cx<Real>::T) * (128 + 128 * (W + 1) + (MODE == COL_UPDATE ? 128 * W : 0));
}
template <typename Real, int W> constexpr size_t ens_x_smem() {
  return sizeof(typename Cx<Real>::T) * (128 + 65 * (W + 1));
}

// Persistent launch of kernel k: G CTAs per SM, or as many as fit (a CTA that
// is not resident would hold its whole tile list back until a slot frees).
template <typename K, typename... Args>
int ens_persistent(K k, int G, int num_sms, int tiles, size_t smem, int threads, cudaStream_t s,
                   int (&setup)[kDevCache], const Args &...args) {
  int occ = kernel_setup(k, threads, smem, setup);
  if (occ > G) occ = G;
  const int grid = tiles < num_sms * occ ? tiles : num_sms * occ;
  if (grid < 1) return 0;
  k<<<grid, threads, smem, s>>>(args...);
  return (int)cudaGetLastError();
}

template <typename Real, int W, int G>
int ens_launch_stage_w(int stage, int num_sms, int tiles, int count, const EnsArgs &a, cudaStream_t s) {
  constexpr int NT = W * kEnsT;
  if (stage == 0) {
    static int setup[kDevCache];
    return ens_persistent(ens_col_kernel<Real, W, COL_PLAIN, +1, G>, G, num_sms, tiles, ens_col_smem<Real, W>(),
                          NT, s, setup, a, 1);
  } else if (stage == 2) {
    static int setup[kDevCache];
    return ens_persistent(ens_col_kernel<Real, W, COL_PLAIN, -1, G>, G, num_sms, tiles, ens_col_smem<Real, W>(),
                          NT, s, setup, a, 1);
  } else if (stage == 3) {
    static int setup[kDevCache];
    return ens_persistent(ens_col_kernel<Real, W, COL_UPDATE, -1, G>, G, num_sms, tiles,
                          ens_col_smem<Real, W, COL_UPDATE>(), NT, s, setup, a, 2);
  } else if (stage == 1) {
    static int setup[kDevCache];
    return ens_persistent(ens_x_kernel<Real, W, G>, G, num_sms, tiles, ens_x_smem<Real, W>(), NT, s, setup, a);
  } else {
    // `tiles` = the largest instance's n1 * n2 (one thread per mode of its two planes)
    const int bx = tiles > 0 ? (2 * tiles + 255) / 256 : 8;
    ens_herm_kernel<Real><<<dim3(bx, count), 256, 0, s>>>(a);
  }
  return (int)cudaGetLastError();
}

// One stage of the ensemble step (0 y inverse, 1 fused x, 2 y forward, 3 z
// update, 4 Hermitian fix) with tiles of W = 16 or 8 lines and at most G CTAs
// per SM; `tiles` is the stage's tile count (a.prefix[count]).  Instantiated
// per precision in ensemble_f32.cu / ensemble_f64.cu.
template <typename Real>
int ens_launch_stage(int stage, int W, int G, int num_sms, int tiles, int count, const EnsArgs &a,
                     cudaStream_t s) {
#define OPFC_ENS_WG(w, g) \
  if (W == w && G == g) return ens_launch_stage_w<Real, w, g>(stage, num_sms, tiles, count, a, s);
  OPFC_ENS_WG(16, 4) OPFC_ENS_WG(16, 8) OPFC_ENS_WG(16, 16)
  OPFC_ENS_WG(8, 4) OPFC_ENS_WG(8, 8) OPFC_ENS_WG(8, 16)
#undef OPFC_ENS_WG
  return (int)cudaErrorInvalidValue;
}

extern template int ens_launch_stage<float>(int, int, int, int, int, int, const EnsArgs &, cudaStream_t);
extern template int ens_launch_stage<double>(int, int, int, int, int, int, const EnsArgs &, cudaStream_t);

}  // namespace opfc
