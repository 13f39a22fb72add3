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

struct EnsInst {
  int n0, n1, n2, M;
  long long off_c;     // element offset of the instance's split-layout arrays
  int tw0, tw1, tw2;   // element offsets of its x (N0), y (N1), z (N2) twiddles
  int pad_;
  double mean;         // mean density (k = 0 mode, FP64)
};

struct EnsArgs {
  const EnsInst *inst;
  int count;
  const int *prefix;   // tile prefix sums of this stage, count + 1 entries
  void *work;          // F_z^-1 of the states / the step's working arrays
  void *psi_hat;       // states (DC slot zero)
  const void *tab_a, *tab_b;
  const void *tw;      // concatenated twiddle tables
  unsigned *flag;
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

// Column tile (y or z pass) of one instance; mirrors col_kernel's body.
template <typename Real, int N, int W, int MODE, int DIR>
__device__ __forceinline__ void ens_col_tile(const EnsArgs &a, const EnsInst &in, int axis, int t,
                                             typename Cx<Real>::T *tw, typename Cx<Real>::T *sm) {
  using C = typename Cx<Real>::T;
  constexpr int E = N / kEnsT;
  constexpr int ld = W + 1;
  const int tid = threadIdx.x, c = tid % W, j = tid / W;
  const int M = in.M, n1 = in.n1, n2 = in.n2;
  const long long nyq = (long long)M * n1 * n2;
  const C *gtw = reinterpret_cast<const C *>(a.tw) + (axis == 1 ? in.tw1 : in.tw2);
  for (int i = tid; i < N; i += W * kEnsT) tw[i] = gtw[i];
  __syncthreads();
  // main segment: columns kx, outer z (y pass) or y (z pass); then the Nyquist plane
  const int ti_main = (M + W - 1) / W;
  const int n_outer = axis == 1 ? n2 : n1;
  long long base;
  long long fs;
  bool ok;
  if (t < ti_main * n_outer) {
    const int ti = t % ti_main, to = t / ti_main;
    const int cg = ti * W + c;
    ok = cg < M;
    base = (axis == 1 ? (long long)to * M * n1 : (long long)to * M) + cg;
    fs = axis == 1 ? M : (long long)M * n1;
  } else {
    const int tn = t - ti_main * n_outer;
    const int cg = tn * W + c;
    const int ncols = axis == 1 ? n2 : n1;
    ok = cg < ncols;
    base = nyq + (axis == 1 ? (long long)cg * n1 : (long long)cg);
    fs = axis == 1 ? 1 : n1;
  }
  C *work = reinterpret_cast<C *>(a.work) + in.off_c;
  C v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) v[m] = ok ? work[base + (long long)(j + kEnsT * m) * fs] : mk<C>(0, 0);
  if constexpr (MODE == COL_PLAIN) {
    fft_line_e<C, N, DIR, N>(v, sm, ld, c, j, tw);
  } else {
    fft_line_e<C, N, -1, N>(v, sm, ld, c, j, tw);
    C *ph = reinterpret_cast<C *>(a.psi_hat) + in.off_c;
    const Real *ta = reinterpret_cast<const Real *>(a.tab_a) + in.off_c;
    const Real *tb = reinterpret_cast<const Real *>(a.tab_b) + in.off_c;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const long long idx = base + (long long)(j + kEnsT * m) * fs;
      C np = mk<C>(0, 0);
      if (ok) {
        const C p = ph[idx];
        np = mk<C>(ta[idx] * p.x + tb[idx] * v[m].x, ta[idx] * p.y + tb[idx] * v[m].y);
        ph[idx] = np;
      }
      v[m] = np;
    }
    fft_line_e<C, N, +1, N>(v, sm, ld, c, j, tw);
  }
  if (ok) {
#pragma unroll
    for (int m = 0; m < E; ++m) work[base + (long long)(j + kEnsT * m) * fs] = v[m];
  }
  __syncthreads();  // tw / sm are reused by the next tile
}

template <typename Real, int W, int MODE, int DIR>
__global__ void __launch_bounds__(W *kEnsT) ens_col_kernel(const EnsArgs a, int axis) {
  using C = typename Cx<Real>::T;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *tw = reinterpret_cast<C *>(smraw);
  C *sm = tw + 128;
  const int total = a.prefix[a.count];
  for (int g = blockIdx.x; g < total; g += gridDim.x) {
    const int i = ens_find(a.prefix, a.count, g);
    const EnsInst in = a.inst[i];
    const int t = g - a.prefix[i];
    const int N = axis == 1 ? in.n1 : in.n2;
    switch (N) {
      case 16: ens_col_tile<Real, 16, W, MODE, DIR>(a, in, axis, t, tw, sm); break;
      case 32: ens_col_tile<Real, 32, W, MODE, DIR>(a, in, axis, t, tw, sm); break;
      case 48: ens_col_tile<Real, 48, W, MODE, DIR>(a, in, axis, t, tw, sm); break;
      case 64: ens_col_tile<Real, 64, W, MODE, DIR>(a, in, axis, t, tw, sm); break;
      case 80: ens_col_tile<Real, 80, W, MODE, DIR>(a, in, axis, t, tw, sm); break;
      case 96: ens_col_tile<Real, 96, W, MODE, DIR>(a, in, axis, t, tw, sm); break;
      case 128: ens_col_tile<Real, 128, W, MODE, DIR>(a, in, axis, t, tw, sm); break;
      default: break;  // sizes are validated on the host
    }
  }
}

// Fused x tile (C2R -> psi^3 -> R2C) of W rows of one instance; mirrors x_kernel.
template <typename Real, int M, int W>
__device__ __forceinline__ void ens_x_tile(const EnsArgs &a, const EnsInst &in, int t,
                                           typename Cx<Real>::T *tw, typename Cx<Real>::T *buf,
                                           bool &bad) {
  using C = typename Cx<Real>::T;
  constexpr int E = M / kEnsT;
  constexpr int NT = W * kEnsT;
  constexpr int ld = W + 1;
  constexpr int N0 = 2 * M;
  const int tid = threadIdx.x, c = tid % W, j = tid / W;
  const int rows = in.n1 * in.n2;
  const long long nyq = (long long)M * rows;
  const C *gtw = reinterpret_cast<const C *>(a.tw) + in.tw0;
  for (int i = tid; i < N0; i += NT) tw[i] = gtw[i];
  C *work = reinterpret_cast<C *>(a.work) + in.off_c;
  const int row0 = t * W;
  x_load_rows<C, M, W, NT>(work, nyq, row0, rows, buf, tid);
  __syncthreads();
  C v[E];
  x_pre<C, M, W, E>(buf, tw, c, j, v);
  __syncthreads();
  fft_line_e<C, M, +1, N0>(v, buf, ld, c, j, tw);
  const double scale = 1.0 / ((double)in.n0 * rows);
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const Real x = to_real_plus_mean(v[m].x, scale, in.mean);
    const Real y = to_real_plus_mean(v[m].y, scale, in.mean);
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

template <typename Real, int W>
__global__ void __launch_bounds__(W *kEnsT) ens_x_kernel(const EnsArgs a) {
  using C = typename Cx<Real>::T;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *tw = reinterpret_cast<C *>(smraw);
  C *buf = tw + 128;
  const int total = a.prefix[a.count];
  bool bad = false;
  for (int g = blockIdx.x; g < total; g += gridDim.x) {
    const int i = ens_find(a.prefix, a.count, g);
    const EnsInst in = a.inst[i];
    const int t = g - a.prefix[i];
    switch (in.M) {
      case 16: ens_x_tile<Real, 16, W>(a, in, t, tw, buf, bad); break;
      case 24: ens_x_tile<Real, 24, W>(a, in, t, tw, buf, bad); break;
      case 32: ens_x_tile<Real, 32, W>(a, in, t, tw, buf, bad); break;
      case 40: ens_x_tile<Real, 40, W>(a, in, t, tw, buf, bad); break;
      case 48: ens_x_tile<Real, 48, W>(a, in, t, tw, buf, bad); break;
      case 64: ens_x_tile<Real, 64, W>(a, in, t, tw, buf, bad); break;
      default: break;
    }
  }
  if (bad && a.flag) atomicOr(a.flag, 1u);
}

// Hermitian projection of every instance's kx = 0 and Nyquist planes.
template <typename Real>
__global__ void ens_herm_kernel(const EnsArgs a) {
  using C = typename Cx<Real>::T;
  const int i = blockIdx.y;
  const EnsInst in = a.inst[i];
  const long long plane = (long long)in.n1 * in.n2;
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
template <typename Real, int W> constexpr size_t ens_col_smem() {
  return sizeof(typename Cx<Real>::T) * (128 + 128 * (W + 1));
}
template <typename Real, int W> constexpr size_t ens_x_smem() {
  return sizeof(typename Cx<Real>::T) * (128 + 65 * (W + 1));
}

}  // namespace opfc
