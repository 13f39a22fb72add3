// kernels.cuh -- the pass kernels of the spectral PFC step (sm_100a).
//
// One PFC step with the state psi_hat resident in k-space is four passes over
// the spectrum (the reference runs 3-4 full 3D FFTs plus 3-4 elementwise sweeps,
// apps/tungsten/include/tungsten/cuda/tungsten_model.hpp:392-455):
//
//   YI  inverse y transform of A = F_z^-1[psi_hat]                (col pass)
//   X   per x-row: C2R -> nonlinearity -> R2C, in place on A       (x pass)
//   YF  forward y transform                                        (col pass)
//   ZU  forward z transform of N_hat, ETD update psi_hat = opL psi_hat + opN
//       N_hat (in place), inverse z transform of the new state into A   (col pass)
//
// plus a tiny Hermitian projection of the kx = 0 and Nyquist planes.  Every
// pass reads and writes each mode once; the nonlinearity, the mean-field filter
// and the k-space update never make a sweep of their own.
#pragma once
#include "fft_core.cuh"
#include "launch.h"

namespace opfc {

template <typename Real> struct Width;       // columns / rows per CTA
template <> struct Width<float> { static constexpr int W = 16; };
template <> struct Width<double> { static constexpr int W = 8; };

template <typename Real> struct ColArgs {
  ColSeg seg0, seg1;
  const void *in[2];
  void *out[2];
  const void *tw;
  void *psi_hat;
  const Real *tab_a, *tab_b, *tab_chi;
  const Real *tab_p;  // MK_ALUMINUM_G: P_F
  void *out_p;        // MK_ALUMINUM_G: F_z^-1[P_F psi_hat]
  // radial operators (isotropic grids): rad_ops[m] = (opL, opN), rad_chi[m],
  // m = kx^2 + ky^2 + kz^2 in folded integer indices
  const void *rad_ops;
  const Real *rad_chi;
  int rad_M, rad_n1, rad_n2;
  // computed operators: wavenumber steps, r, dt, 1/(2 alpha^2)
  Real kf0, kf1, kf2, op_r, op_dt, op_chi;
  // folded tables: (opL, opN) pairs and the filter of the modes (kx, |ky|, |kz|),
  // kx in [0, M], folded |ky| <= N1/2 and |kz| <= N2/2, in the split layout of an
  // (M+1) x (N1/2+1) x (N2/2+1) grid (kx < M first, the kx = M plane at fold_nyq)
  const void *fold_ops;
  const Real *fold_chi;
  long long fold_nyq;
};

// Operator selection of the fused z update.
enum OpsKind { OPS_TABLES = 0, OPS_RADIAL = 1, OPS_COMPUTED = 2, OPS_FOLDED = 3 };

// |k| index of a frequency index i of an axis of length n (i and n - i give
// the same k^2, so every operator of k^2 is even in it)
__device__ __forceinline__ int fold_index(int i, int n) { return i <= n / 2 ? i : n - i; }

// Index of mode (kx, ky, kz) in the folded tables.
template <typename Real>
__device__ __forceinline__ long long fold_at(const ColArgs<Real> &a, int kx, int ky, int kz) {
  const long long r =
      (long long)fold_index(ky, a.rad_n1) + (long long)(a.rad_n1 / 2 + 1) * fold_index(kz, a.rad_n2);
  return kx < a.rad_M ? kx + (long long)a.rad_M * r : a.fold_nyq + r;
}

// Operators of mode (kx, ky, kz) read from the folded tables (direct loads).
template <typename Real, int MODEL>
__device__ __forceinline__ void folded_ops(const ColArgs<Real> &a, int kx, int ky, int kz, Real &la, Real &lb,
                                           Real &ch) {
  using C = typename Cx<Real>::T;
  const long long i = fold_at(a, kx, ky, kz);
  const C o = __ldg(reinterpret_cast<const C *>(a.fold_ops) + i);
  la = o.x;
  lb = o.y;
  ch = MODEL != MK_PLAIN ? __ldg(a.fold_chi + i) : Real(1);
}

// Plain-PFC operators of mode (kx, ky, kz) (kx unfolded, ky / kz folded), in
// the compute precision (10_complete_pfc_model.cpp:189-207, kspace.hpp:97-103):
//   k^2 = sum (f_a i_a)^2, g = r + (1 - k^2)^2, L = -k^2 g,
//   opL = exp(L dt),  opN = (opL - 1)/L (-k^2) = expm1(L dt)/g  (|L| > 1e-14),
//   opN = dt (-k^2) otherwise;  FILTERED: chi = exp(-k^2 / (2 alpha^2)).
// One expm1 gives both: opL = 1 + expm1(L dt) (within half an ulp of 1 of
// exp), and expm1 keeps the long-wavelength modes (|L dt| << 1) accurate in
// FP32.  FP32 divides with the fast reciprocal (2 ulp); FP64 divides exactly.
__device__ __forceinline__ float ops_div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double ops_div(double a, double b) { return a / b; }

template <typename Real>
__device__ __forceinline__ void ops_from_k2(Real k2, Real r, Real dt, Real &la, Real &lb) {
  const Real u = Real(1) - k2;
  const Real g = r + u * u;
  const Real L = -k2 * g;
  const Real em1 = expm1(L * dt);
  la = Real(1) + em1;
  lb = fabs(L) > Real(1e-14) ? ops_div(em1, g) : -dt * k2;
}

template <typename Real, int MODEL>
__device__ __forceinline__ void computed_ops(const ColArgs<Real> &a, int kx, int ky, int kz, Real &la,
                                             Real &lb, Real &ch) {
  const int fy = ky <= a.rad_n1 / 2 ? ky : a.rad_n1 - ky;
  const int fz = kz <= a.rad_n2 / 2 ? kz : a.rad_n2 - kz;
  const Real qx = a.kf0 * Real(kx), qy = a.kf1 * Real(fy), qz = a.kf2 * Real(fz);
  const Real k2 = qx * qx + qy * qy + qz * qz;
  ops_from_k2(k2, a.op_r, a.op_dt, la, lb);
  ch = MODEL == MK_FILTERED ? exp(-k2 * a.op_chi) : Real(1);
}

template <typename C> __device__ __forceinline__ C czero() { return mk<C>(0, 0); }
}  // namespace opfc

#include "col_tma.cuh"

namespace opfc {

// ---------------------------------------------------------------------------
// column pass: batched FFT along a strided axis (y or z), optional ETD update
// ---------------------------------------------------------------------------
// EE values per thread (plan PlanE<N, EE>; EE = 32 gives one exchange per
// transform at N = 512, 1024).
template <typename Real, int N, int MODE, int DIR, int MODEL, bool INV, int OPS, int EE = Plan<N>::E>
__global__ void __launch_bounds__(Width<Real>::W *(N / EE)) col_kernel(const ColArgs<Real> a) {
  using C = typename Cx<Real>::T;
  constexpr int W = Width<Real>::W;
  constexpr int E = EE;
  constexpr int T = N / E;
  constexpr int NT = W * T;
  constexpr int ld = W + 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *tw = reinterpret_cast<C *>(smraw);
  C *sm = tw + N;

  const int tid = threadIdx.x;
  const int c = tid % W;
  const int j = tid / W;
  const C *gtw = reinterpret_cast<const C *>(a.tw);
  for (int i = tid; i < N; i += NT) tw[i] = gtw[i];

  int t = blockIdx.x;
  const bool second = t >= a.seg0.ntiles;
  const ColSeg sg = second ? a.seg1 : a.seg0;
  if (second) t -= a.seg0.ntiles;
  const int ti = t % sg.tiles_inner;
  const int to = t / sg.tiles_inner;
  const int cg = ti * W + c;
  const bool ok = cg < sg.ncols;
  const long long base = sg.off + (long long)to * sg.s_outer + (long long)cg * sg.col_stride;
  const long long fs = sg.fft_stride;
  const int set = blockIdx.y;
  const C *in = reinterpret_cast<const C *>(a.in[set]);
  C *out = reinterpret_cast<C *>(a.out[set]);

  C v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) v[m] = ok ? in[base + (long long)(j + T * m) * fs] : czero<C>();

  if constexpr (MODE == COL_PLAIN) {
    fft_line_e<C, N, DIR, N, E>(v, sm, ld, c, j, tw);
    if (ok) {
#pragma unroll
      for (int m = 0; m < E; ++m) out[base + (long long)(j + T * m) * fs] = v[m];
    }
  } else {
    // forward z transform completes N_hat; ETD update of the resident state
    fft_line_e<C, N, -1, N, E>(v, sm, ld, c, j, tw);
    C *ph = reinterpret_cast<C *>(a.psi_hat);
    C w[(MODEL == MK_PLAIN) ? 1 : E];
    C pw[(MODEL == MK_ALUMINUM_G) ? E : 1];
    // psi_hat in groups of GB values: each group's loads are issued together,
    // then combined and stored (a store to psi_hat keeps every later load --
    // psi_hat, tables -- behind it, so a value-by-value loop would make one
    // memory round trip per value; larger groups cost registers)
    constexpr int GB = E % 4 == 0 ? 4 : 1;
#pragma unroll
    for (int m0 = 0; m0 < E; m0 += GB) {
      C pv[GB];
#pragma unroll
      for (int q = 0; q < GB; ++q) pv[q] = ok ? ph[base + (long long)(j + T * (m0 + q)) * fs] : czero<C>();
#pragma unroll
      for (int q = 0; q < GB; ++q) {
        const int m = m0 + q;
        const long long idx = base + (long long)(j + T * m) * fs;
        C np = czero<C>();
        if constexpr (MODEL == MK_ALUMINUM_G) pw[m] = czero<C>();
        if (ok) {
          const C p = pv[q];
          Real la, lb, ch = Real(1);
          if constexpr (OPS == OPS_COMPUTED) {
            // z pass: main plane kx = column, ky = outer; Nyquist plane kx = M, ky = column
            computed_ops<Real, MODEL>(a, second ? a.rad_M : cg, second ? cg : to, j + T * m, la, lb, ch);
          } else if constexpr (OPS == OPS_FOLDED) {
            folded_ops<Real, MODEL>(a, second ? a.rad_M : cg, second ? cg : to, j + T * m, la, lb, ch);
          } else {
            la = a.tab_a[idx];
            lb = a.tab_b[idx];
            if constexpr (MODEL != MK_PLAIN) ch = a.tab_chi[idx];
          }
          np = mk<C>(la * p.x + lb * v[m].x, la * p.y + lb * v[m].y);
          if constexpr (MODEL != MK_PLAIN) w[m] = cscale(np, ch);
          if constexpr (MODEL == MK_ALUMINUM_G) pw[m] = cscale(np, a.tab_p[idx]);
        } else if constexpr (MODEL != MK_PLAIN) {
          w[m] = czero<C>();
        }
        v[m] = np;
      }
      if (ok) {
#pragma unroll
        for (int q = 0; q < GB; ++q) ph[base + (long long)(j + T * (m0 + q)) * fs] = v[m0 + q];
      }
    }
    if constexpr (INV) {
      if constexpr (MODEL == MK_FILTERED) {
        fft_line_e<C, N, +1, N, E>(w, sm, ld, c, j, tw);
        if (ok) {
#pragma unroll
          for (int m = 0; m < E; ++m) out[base + (long long)(j + T * m) * fs] = w[m];
        }
      } else {
        fft_line_e<C, N, +1, N, E>(v, sm, ld, c, j, tw);
        if (ok) {
#pragma unroll
          for (int m = 0; m < E; ++m) out[base + (long long)(j + T * m) * fs] = v[m];
        }
        if constexpr (MODEL == MK_TUNGSTEN || MODEL == MK_ALUMINUM_G) {
          C *out2 = reinterpret_cast<C *>(a.out[1]);
          fft_line_e<C, N, +1, N, E>(w, sm, ld, c, j, tw);
          if (ok) {
#pragma unroll
            for (int m = 0; m < E; ++m) out2[base + (long long)(j + T * m) * fs] = w[m];
          }
        }
        if constexpr (MODEL == MK_ALUMINUM_G) {
          C *out3 = reinterpret_cast<C *>(a.out_p);
          fft_line_e<C, N, +1, N, E>(pw, sm, ld, c, j, tw);
          if (ok) {
#pragma unroll
            for (int m = 0; m < E; ++m) out3[base + (long long)(j + T * m) * fs] = pw[m];
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// x pass: each row of N0 = 2M reals <-> M+1 complex modes, via one complex FFT
// of length M of z[p] = x[2p] + i x[2p+1] and the split/merge post-processing.
// ---------------------------------------------------------------------------
template <typename Real> struct XArgs {
  const void *in0, *in1, *in2;
  void *out;
  const Real *rin;
  Real *rout;
  const void *tw;
  long long nyq_off;
  int rows;
  double scale, mean;
  Real c0, c1, c2, c3, c4, c5;
  unsigned int *flag;
  double al[18];  // MK_ALUMINUM_G coefficients (XLaunch::al)
  const double *time;
};

// rows [row0, row0+W) of a split-layout complex array -> smem buf[k][c], k<=M
template <typename C, int M, int W, int NT>
__device__ __forceinline__ void x_load_rows(const C *in, long long nyq_off, int row0, int rows,
                                            C *buf, int tid) {
  constexpr int ld = W + 1;
  for (int f = tid; f < W * M; f += NT) {
    const int cc = f / M, k = f - cc * M;
    const int row = row0 + cc;
    buf[k * ld + cc] = (row < rows) ? in[(long long)row * M + k] : mk<C>(0, 0);
  }
  if (tid < W) {
    const int row = row0 + tid;
    buf[M * ld + tid] = (row < rows) ? in[nyq_off + row] : mk<C>(0, 0);
  }
}

// C2R pre-processing: Z'[k] = (X[k] + conj X[M-k]) + i e^{+2 pi i k/N0} (X[k] - conj X[M-k]),
// with the imaginary parts of the DC and Nyquist bins ignored (C2R semantics).
template <typename C, int M, int W, int E>
__device__ __forceinline__ void x_pre(const C *buf, const C *tw, int c, int j, C (&v)[E]) {
  constexpr int ld = W + 1;
  constexpr int T = M / E;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int k = j + T * m;
    C X = buf[k * ld + c];
    C Y = buf[(M - k) * ld + c];
    if (k == 0) {
      X.y = 0;
      Y.y = 0;
    }
    const C s = mk<C>(X.x + Y.x, X.y - Y.y);
    const C d = mk<C>(X.x - Y.x, X.y + Y.y);
    const C e = twmul<+1>(d, tw[k]);  // d * e^{+2 pi i k / N0}
    v[m] = mk<C>(s.x - e.y, s.y + e.x);
  }
}

// R2C post-processing and store:
// X[k] = 1/2 (Z[k] + conj Z[M-k]) - i/2 e^{-2 pi i k/N0} (Z[k] - conj Z[M-k]),
// X[M] = Re Z[0] - Im Z[0].
template <typename C, int M, int W, int NT>
__device__ __forceinline__ void x_post_store(const C *buf, const C *tw, C *out, long long nyq_off,
                                             int row0, int rows, int tid) {
  using S = decltype(C::x);
  constexpr int ld = W + 1;
  for (int f = tid; f < W * M; f += NT) {
    const int cc = f / M, k = f - cc * M;
    const int row = row0 + cc;
    const int km = (k == 0) ? 0 : M - k;
    const C Z = buf[k * ld + cc];
    const C Y = buf[km * ld + cc];
    const C s = mk<C>(Z.x + Y.x, Z.y - Y.y);
    const C d = mk<C>(Z.x - Y.x, Z.y + Y.y);
    const C e = twmul<-1>(d, tw[k]);  // d * e^{-2 pi i k / N0}
    const C X = mk<C>(S(0.5) * (s.x + e.y), S(0.5) * (s.y - e.x));
    if (row < rows) out[(long long)row * M + k] = X;
  }
  if (tid < W) {
    const int row = row0 + tid;
    const C Z = buf[tid];
    if (row < rows) out[nyq_off + row] = mk<C>(Z.x - Z.y, S(0));
  }
}

template <typename Real>
__device__ __forceinline__ Real to_real_plus_mean(Real z, double scale, double mean) {
  return (Real)((double)z * scale + mean);
}

template <typename Real, int M, int MODE, int MODEL>
__global__ void __launch_bounds__(Width<Real>::W *(M / Plan<M>::E)) x_kernel(const XArgs<Real> a) {
  using C = typename Cx<Real>::T;
  constexpr int W = Width<Real>::W;
  constexpr int E = Plan<M>::E;
  constexpr int T = M / E;
  constexpr int NT = W * T;
  constexpr int ld = W + 1;
  constexpr int N0 = 2 * M;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *tw = reinterpret_cast<C *>(smraw);
  C *buf = tw + N0;

  const int tid = threadIdx.x;
  const int c = tid % W;
  const int j = tid / W;
  const C *gtw = reinterpret_cast<const C *>(a.tw);
  for (int i = tid; i < N0; i += NT) tw[i] = gtw[i];
  const int row0 = blockIdx.x * W;
  C v[E];

  if constexpr (MODE == X_R2C) {
    // real rows -> buf[p][c] as (x[2p], x[2p+1])
    for (int f = tid; f < W * M; f += NT) {
      const int cc = f / M, p = f - cc * M;
      const int row = row0 + cc;
      C z = mk<C>(0, 0);
      if (row < a.rows) z = reinterpret_cast<const C *>(a.rin + (long long)row * N0)[p];
      buf[p * ld + cc] = z;
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = buf[(j + T * m) * ld + c];
    __syncthreads();
    fft_line<C, M, -1, N0>(v, buf, ld, c, j, tw);
  } else {
    const C *in0 = reinterpret_cast<const C *>(a.in0);
    x_load_rows<C, M, W, NT>(in0, a.nyq_off, row0, a.rows, buf, tid);
    __syncthreads();
    x_pre<C, M, W, E>(buf, tw, c, j, v);
    __syncthreads();
    fft_line<C, M, +1, N0>(v, buf, ld, c, j, tw);
#pragma unroll
    for (int m = 0; m < E; ++m)
      v[m] = mk<C>(to_real_plus_mean(v[m].x, a.scale, a.mean),
                   to_real_plus_mean(v[m].y, a.scale, a.mean));
    if constexpr (MODE == X_C2R) {
#pragma unroll
      for (int m = 0; m < E; ++m) buf[(j + T * m) * ld + c] = v[m];
      __syncthreads();
      for (int f = tid; f < W * M; f += NT) {
        const int cc = f / M, p = f - cc * M;
        const int row = row0 + cc;
        if (row < a.rows) reinterpret_cast<C *>(a.rout + (long long)row * N0)[p] = buf[p * ld + cc];
      }
      return;
    } else {
      bool bad = false;
      if constexpr (MODEL == MK_TUNGSTEN) {
        C u[E];
#pragma unroll
        for (int m = 0; m < E; ++m) u[m] = v[m];
        const C *in1 = reinterpret_cast<const C *>(a.in1);
        // buf is free: the inverse FFT's last stage only touched registers
        x_load_rows<C, M, W, NT>(in1, a.nyq_off, row0, a.rows, buf, tid);
        __syncthreads();
        x_pre<C, M, W, E>(buf, tw, c, j, v);
        __syncthreads();
        fft_line<C, M, +1, N0>(v, buf, ld, c, j, tw);
        // N = p3b u^2 + p4b u^3 + q3b v^2 + q4b v^3 - stabP u
        // (apps/tungsten/include/tungsten/cpu/tungsten_model.hpp:334-350)
#pragma unroll
        for (int m = 0; m < E; ++m) {
          const Real vx = to_real_plus_mean(v[m].x, a.scale, a.mean);
          const Real vy = to_real_plus_mean(v[m].y, a.scale, a.mean);
          const Real ux = u[m].x, uy = u[m].y;
          const Real nx = a.c0 * ux * ux + a.c1 * ux * ux * ux + a.c2 * vx * vx +
                          a.c3 * vx * vx * vx - a.c4 * ux;
          const Real ny = a.c0 * uy * uy + a.c1 * uy * uy * uy + a.c2 * vy * vy +
                          a.c3 * vy * vy * vy - a.c4 * uy;
          bad |= !(isfinite(nx) && isfinite(ny));
          v[m] = mk<C>(nx, ny);
        }
      } else if constexpr (MODEL == MK_ALUMINUM_G) {
        // Aluminum.hpp:270-307: psi (u), psi_MF (v) and P*psi (q) in real space;
        // moving temperature T_var(x, t); real cells 2p (re) and 2p + 1 (im)
        C u[E];
#pragma unroll
        for (int m = 0; m < E; ++m) u[m] = v[m];
        x_load_rows<C, M, W, NT>(reinterpret_cast<const C *>(a.in1), a.nyq_off, row0, a.rows, buf, tid);
        __syncthreads();
        x_pre<C, M, W, E>(buf, tw, c, j, v);
        __syncthreads();
        fft_line<C, M, +1, N0>(v, buf, ld, c, j, tw);
        C q[E];
        x_load_rows<C, M, W, NT>(reinterpret_cast<const C *>(a.in2), a.nyq_off, row0, a.rows, buf, tid);
        __syncthreads();
        x_pre<C, M, W, E>(buf, tw, c, j, q);
        __syncthreads();
        fft_line<C, M, +1, N0>(q, buf, ld, c, j, tw);
        const double *al = a.al;
        const double t = *a.time;
        auto nl = [&](double x, Real uu, Real vv, Real qq) -> Real {
          const double dist = x + al[3] - (x > al[4] ? al[2] : 0.0);
          const double Tv = al[5] * (dist - al[6] - al[7] * t);
          const Real q2N = (Real)(al[10] * Tv / al[8]);
          const Real q3 = (Real)(al[12] * (al[9] + Tv) / al[8] + al[11]);
          const Real kern = (Real)(-(1.0 - exp(-Tv / al[8]))) * qq;
          return (Real)al[13] * uu * uu + (Real)al[14] * uu * uu * uu + q2N * vv + q3 * vv * vv +
                 (Real)al[15] * vv * vv * vv - kern - (Real)al[16] * uu;
        };
#pragma unroll
        for (int m = 0; m < E; ++m) {
          const Real vx = to_real_plus_mean(v[m].x, a.scale, a.mean);
          const Real vy = to_real_plus_mean(v[m].y, a.scale, a.mean);
          const Real qx = to_real_plus_mean(q[m].x, a.scale, al[17] * a.mean);
          const Real qy = to_real_plus_mean(q[m].y, a.scale, al[17] * a.mean);
          const int i0 = 2 * (j + T * m);
          const Real nx = nl(al[0] + i0 * al[1], u[m].x, vx, qx);
          const Real ny = nl(al[0] + (i0 + 1) * al[1], u[m].y, vy, qy);
          bad |= !(isfinite(nx) && isfinite(ny));
          v[m] = mk<C>(nx, ny);
        }
      } else if constexpr (MODEL == MK_FILTERED) {
        // N = p2 v^2/2 + p3 v^3/3 + p4 v^4/4 of the filtered density
#pragma unroll
        for (int m = 0; m < E; ++m) {
          const Real x = v[m].x, y = v[m].y;
          const Real x2 = x * x, y2 = y * y;
          const Real nx = x2 * (a.c0 + a.c1 * x + a.c2 * x2);
          const Real ny = y2 * (a.c0 + a.c1 * y + a.c2 * y2);
          bad |= !(isfinite(nx) && isfinite(ny));
          v[m] = mk<C>(nx, ny);
        }
      } else {
        // N = psi^3 (docs/api/examples/10_complete_pfc_model.cpp:128-130)
#pragma unroll
        for (int m = 0; m < E; ++m) {
          const Real x = v[m].x, y = v[m].y;
          const Real nx = x * x * x, ny = y * y * y;
          bad |= !(isfinite(nx) && isfinite(ny));
          v[m] = mk<C>(nx, ny);
        }
      }
      if (bad && a.flag) atomicOr(a.flag, 1u);
      fft_line<C, M, -1, N0>(v, buf, ld, c, j, tw);
    }
  }
  // Z in registers -> buf -> post-process -> store
#pragma unroll
  for (int m = 0; m < E; ++m) buf[(j + T * m) * ld + c] = v[m];
  __syncthreads();
  x_post_store<C, M, W, NT>(buf, tw, reinterpret_cast<C *>(a.out), a.nyq_off, row0, a.rows, tid);
}

}  // namespace opfc

#include "x_tma.cuh"
#include "x_sq.cuh"

namespace opfc {

// ---------------------------------------------------------------------------
// small helper kernels (not on the per-step hot path except herm_fix)
// ---------------------------------------------------------------------------

// Hermitian projection of the kx = 0 and kx = N0/2 planes: a real field's
// spectrum satisfies X(0,-ky,-kz) = conj X(0,ky,kz) there; the C2R ignores the
// anti-Hermitian part, so it is removed from the resident state instead of
// being left to grow under exp(L dt) > 1.
template <typename Real>
__global__ void herm_fix_kernel(typename Cx<Real>::T *psi, long long nyq_off, int M, int n1, int n2, double *time,
                                double dt_time) {
  using C = typename Cx<Real>::T;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  // the step's last kernel also advances the device time of the next step
  if (time && e == 0 && blockIdx.y == 0) *time += dt_time;
  const long long plane = (long long)n1 * n2;
  if (e >= plane) return;
  const int y = (int)(e % n1), z = (int)(e / n1);
  const int yp = (n1 - y) % n1, zp = (n2 - z) % n2;
  const long long p = (long long)yp + (long long)n1 * zp;
  C *P;
  long long stride;
  if (blockIdx.y == 0) {
    P = psi;
    stride = M;
  } else {
    P = psi + nyq_off;
    stride = 1;
  }
  if (e < p) {
    const C u = P[e * stride], w = P[p * stride];
    const C h = mk<C>(Real(0.5) * (u.x + w.x), Real(0.5) * (u.y - w.y));
    P[e * stride] = h;
    P[p * stride] = mk<C>(h.x, -h.y);
  } else if (e == p) {
    P[e * stride].y = 0;
  }
}

template <typename Real, typename Out>
__global__ void to_ref_kernel(const typename Cx<Real>::T *in, Out *out, int M, int n1, int n2,
                              long long nyq_off, int dc_override, double dc_re) {
  const long long nc = (long long)(M + 1) * n1 * n2;
  for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < nc;
       o += (long long)gridDim.x * blockDim.x) {
    const long long row = o / (M + 1);
    const int kx = (int)(o - row * (M + 1));
    typename Cx<Real>::T v = (kx < M) ? in[row * M + kx] : in[nyq_off + row];
    double re = v.x, im = v.y;
    if (dc_override && o == 0) {
      re = dc_re;
      im = 0;
    }
    out[2 * o] = (Out)re;
    out[2 * o + 1] = (Out)im;
  }
}

template <typename Real, typename In>
__global__ void from_ref_kernel(const In *in, typename Cx<Real>::T *out, int M, int n1, int n2,
                                long long nyq_off) {
  const long long nc = (long long)(M + 1) * n1 * n2;
  for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < nc;
       o += (long long)gridDim.x * blockDim.x) {
    const long long row = o / (M + 1);
    const int kx = (int)(o - row * (M + 1));
    typename Cx<Real>::T v;
    v.x = (Real)in[2 * o];
    v.y = (Real)in[2 * o + 1];
    if (kx < M)
      out[row * M + kx] = v;
    else
      out[nyq_off + row] = v;
  }
}

template <typename In, typename Out>
__global__ void cast_kernel(const In *in, Out *out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = (Out)in[i];
}

// FP64 partial sums with Neumaier compensation per thread and per block.
template <typename Real>
__global__ void sum_pow_kernel(const Real *x, size_t n, int p, double *partials) {
  __shared__ double rs[256], rc[256];
  double s = 0, c = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double v0 = x[i];
    const double v = (p == 4) ? (v0 * v0) * (v0 * v0) : v0;
    const double t = s + v;
    c += (fabs(s) >= fabs(v)) ? (s - t) + v : (v - t) + s;
    s = t;
  }
  rs[threadIdx.x] = s;
  rc[threadIdx.x] = c;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      const double a = rs[threadIdx.x], b = rs[threadIdx.x + h];
      const double t = a + b;
      rc[threadIdx.x] += rc[threadIdx.x + h] + ((fabs(a) >= fabs(b)) ? (a - t) + b : (b - t) + a);
      rs[threadIdx.x] = t;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = rs[0] + rc[0];
}

struct EnergyK {
  double f0, f1, f2, r;
};

__device__ __forceinline__ double kcomp(int i, int n, double f) {
  return (i <= n / 2) ? i * f : (i - n) * f;
}

template <typename Real>
__global__ void energy_k_kernel(const typename Cx<Real>::T *ph, int M, int n1, int n2,
                                long long nyq_off, EnergyK ek, double *partials) {
  __shared__ double red[256];
  const long long nc = (long long)(M + 1) * n1 * n2;
  const int n0 = 2 * M;
  double s = 0;
  for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < nc;
       o += (long long)gridDim.x * blockDim.x) {
    int kx, ky, kz;
    typename Cx<Real>::T v;
    if (o < (long long)M * n1 * n2) {
      kx = (int)(o % M);
      const long long row = o / M;
      ky = (int)(row % n1);
      kz = (int)(row / n1);
      v = ph[o];
    } else {
      const long long row = o - (long long)M * n1 * n2;
      kx = M;
      ky = (int)(row % n1);
      kz = (int)(row / n1);
      v = ph[nyq_off + row];
    }
    const double kxx = kcomp(kx, n0, ek.f0), kyy = kcomp(ky, n1, ek.f1), kzz = kcomp(kz, n2, ek.f2);
    const double k2 = kxx * kxx + kyy * kyy + kzz * kzz;
    const double G = ek.r + (1.0 - k2) * (1.0 - k2);
    const double wgt = (kx == 0 || kx == M) ? 1.0 : 2.0;
    s += wgt * G * ((double)v.x * v.x + (double)v.y * v.y);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
// Rebuild a segment's tiling for tile width W (strides do not depend on W).
static inline ColSeg retile(ColSeg g, int W, int Wold) {
  if (g.ntiles == 0) return g;
  const int n_outer = g.ntiles / g.tiles_inner;
  (void)Wold;
  g.tiles_inner = (g.ncols + W - 1) / W;
  g.ntiles = g.tiles_inner * n_outer;
  return g;
}

template <typename Real> static ColArgs<Real> col_args(const ColLaunch &L) {
  ColArgs<Real> a;
  a.seg0 = L.seg[0];
  a.seg1 = L.seg[1];
  if (L.nseg < 2) a.seg1.ntiles = 0;
  a.in[0] = L.in[0];
  a.in[1] = L.in[1];
  a.out[0] = L.out[0];
  a.out[1] = L.out[1];
  a.tw = L.tw;
  a.psi_hat = L.psi_hat;
  a.tab_a = reinterpret_cast<const Real *>(L.tab_a);
  a.tab_b = reinterpret_cast<const Real *>(L.tab_b);
  a.tab_chi = reinterpret_cast<const Real *>(L.tab_chi);
  a.tab_p = reinterpret_cast<const Real *>(L.tab_p);
  a.out_p = L.out_p;
  a.rad_ops = L.rad_ops;
  a.rad_chi = reinterpret_cast<const Real *>(L.rad_chi);
  a.rad_M = L.rad_M;
  a.rad_n1 = L.rad_n1;
  a.rad_n2 = L.rad_n2;
  a.kf0 = (Real)L.kf[0];
  a.kf1 = (Real)L.kf[1];
  a.kf2 = (Real)L.kf[2];
  a.op_r = (Real)L.op_r;
  a.op_dt = (Real)L.op_dt;
  a.op_chi = (Real)L.op_chi;
  a.fold_ops = L.fold_ops;
  a.fold_chi = reinterpret_cast<const Real *>(L.fold_chi);
  a.fold_nyq = L.fold_nyq;
  return a;
}

template <typename Real, int N, int MODE, int DIR, int MODEL, bool INV, int OPS, int EE = Plan<N>::E>
static int launch_col_direct(const ColLaunch &L, cudaStream_t s) {
  using C = typename Cx<Real>::T;
  constexpr int W = Width<Real>::W;
  constexpr int NT = W * (N / EE);
  const size_t smem = sizeof(C) * ((size_t)N + (size_t)N * (W + 1));
  auto k = col_kernel<Real, N, MODE, DIR, MODEL, INV, OPS, EE>;
  static int setup[kDevCache];
  kernel_setup(k, NT, smem, setup);
  ColArgs<Real> a = col_args<Real>(L);
  const int tiles = a.seg0.ntiles + a.seg1.ntiles;
  if (tiles == 0) return 0;
  dim3 grid(tiles, MODE == COL_PLAIN ? L.nsets : 1);
  k<<<grid, NT, smem, s>>>(a);
  return (int)cudaGetLastError();
}

template <typename Real, int N, int MODE, int DIR, int MODEL, bool INV, int OPS, bool NARROW, bool PP = false>
static int launch_col_tma(const ColLaunch &L, cudaStream_t s) {
  using C = typename Cx<Real>::T;
  constexpr int W = tma_col_width(N, (int)sizeof(C), MODE, NARROW);
  constexpr int NT = W * (N / Plan<N>::E);
  // NARROW (plain transforms): half-width tiles, two CTAs per SM when their
  // shared memory fits and each has at most 512 threads (64 registers per thread)
  using Cfg = TmaCfg<Real, N, W, MODE, MODEL, OPS, 3, PP>;
  constexpr int MINB = (NARROW && MODE == COL_PLAIN && 2 * (Cfg::SMEM + 1024) <= 233472 && NT <= 512) ? 2 : 1;
  if constexpr (Cfg::STAGES < 1 || (NARROW && MINB < 2) ||
                (OPS == OPS_COMPUTED && MODEL == MK_TUNGSTEN) || (OPS == OPS_FOLDED && N % 16 != 0)) {
    return -1;
  } else {
    if (L.seg[0].ncols % W != 0 || L.seg[0].col_stride != 1) return -1;
    auto k = col_tma_kernel<Real, N, W, MODE, DIR, MODEL, INV, OPS, MINB, PP>;
    static int setup[kDevCache];
    int occ = kernel_setup(k, NT, Cfg::SMEM, setup);
    if (occ > MINB) occ = MINB;
    ColArgs<Real> a = col_args<Real>(L);
    a.seg0 = retile(L.seg[0], W, Width<Real>::W);
    a.seg1 = L.nseg < 2 ? ColSeg{} : retile(L.seg[1], W, Width<Real>::W);
    const CUtensorMap *t0 = reinterpret_cast<const CUtensorMap *>(L.tmap[0]);
    auto pick = [&](int i) { return L.tmap[i] ? *reinterpret_cast<const CUtensorMap *>(L.tmap[i]) : *t0; };
    int G = (L.num_sms > 0 ? L.num_sms : 148) * occ;
    const int most = a.seg0.ntiles > a.seg1.ntiles ? a.seg0.ntiles : a.seg1.ntiles;
    if (G > most) G = most;
    if (G < 1) return 0;
    dim3 grid(G, MODE == COL_PLAIN ? L.nsets : 1);
    k<<<grid, NT, Cfg::SMEM, s>>>(*t0, pick(1), pick(2), pick(3), pick(4), a, L.axis, L.flag);
    return (int)cudaGetLastError();
  }
}

// Box-ring update with 128-byte rows (N = 1024, folded tables, PLAIN and
// FILTERED; tensor maps built for Width<Real>::W columns) on the main segment,
// then the Nyquist plane with the direct-load kernel.  -1 when it does not apply.
template <typename Real, int N, int MODEL>
static int launch_col_ring(const ColLaunch &L, cudaStream_t s) {
  if constexpr (N != 1024 || (MODEL != MK_PLAIN && MODEL != MK_FILTERED)) {
    return -1;
  } else {
    using Cfg = RingCfg<Real, N>;
    static_assert(Cfg::FITS, "box ring: shared memory and box shape");
    static_assert(Cfg::W == Width<Real>::W, "128-byte rows are the direct kernels' tile width");
    if (!L.fold_ops || !L.tmap[0] || !L.tmap[1]) return -1;
    if (L.seg[0].ncols % Cfg::W != 0 || L.seg[0].col_stride != 1) return -1;
    if ((long long)N * L.seg[0].fft_stride >= (1ll << 31)) return -1;  // in-column offsets are 32-bit
    auto k = col_ring_kernel<Real, N, MODEL>;
    static int setup[kDevCache];
    kernel_setup(k, Cfg::NT, Cfg::SMEM, setup);
    ColArgs<Real> a = col_args<Real>(L);
    a.seg1 = ColSeg{};
    int G = L.num_sms > 0 ? L.num_sms : 148;
    if (G > a.seg0.ntiles) G = a.seg0.ntiles;
    if (G >= 1) {
      k<<<G, Cfg::NT, Cfg::SMEM, s>>>(*reinterpret_cast<const CUtensorMap *>(L.tmap[0]),
                                     *reinterpret_cast<const CUtensorMap *>(L.tmap[1]), a, L.flag);
      const int rc = (int)cudaGetLastError();
      if (rc) return rc;
    }
    if (L.nseg < 2 || L.seg[1].ntiles == 0) return 0;
    // the Nyquist plane: every tile of the direct kernel's launch is a segment-1 tile
    ColLaunch Ln = L;
    Ln.seg[0].ntiles = 0;
    return launch_col_direct<Real, N, COL_UPDATE, -1, MODEL, true, OPS_FOLDED>(Ln, s);
  }
}

template <typename Real, int N, int MODE, int DIR, int MODEL, bool INV>
static int launch_col_t(const ColLaunch &L, cudaStream_t s) {
  if constexpr (MODE == COL_UPDATE && INV && MODEL != MK_ALUMINUM_G) {
    if (L.wide && L.fold_ops) {
      if (L.tmap[0]) {
        const int rc = launch_col_ring<Real, N, MODEL>(L, s);
        if (rc >= 0) return rc;
      }
      // the tensor maps were built for the ring kernel's width: direct loads
      return launch_col_direct<Real, N, MODE, DIR, MODEL, INV, OPS_FOLDED>(L, s);
    }
  }
  if (L.tmap[0]) {
    int rc;
    if constexpr (MODE == COL_UPDATE)
      rc = L.rad_ops    ? launch_col_tma<Real, N, MODE, DIR, MODEL, INV, OPS_RADIAL, false>(L, s)
           : L.computed ? (L.pingpong ? launch_col_tma<Real, N, MODE, DIR, MODEL, INV, OPS_COMPUTED, false, true>(L, s)
                                      : launch_col_tma<Real, N, MODE, DIR, MODEL, INV, OPS_COMPUTED, false>(L, s))
           : L.fold_ops ? (L.pingpong ? launch_col_tma<Real, N, MODE, DIR, MODEL, INV, OPS_FOLDED, false, true>(L, s)
                                      : launch_col_tma<Real, N, MODE, DIR, MODEL, INV, OPS_FOLDED, false>(L, s))
                        : launch_col_tma<Real, N, MODE, DIR, MODEL, INV, OPS_TABLES, false>(L, s);
    else
      rc = L.narrow     ? launch_col_tma<Real, N, MODE, DIR, MODEL, INV, OPS_TABLES, true>(L, s)
           : L.pingpong ? launch_col_tma<Real, N, MODE, DIR, MODEL, INV, OPS_TABLES, false, true>(L, s)
                        : launch_col_tma<Real, N, MODE, DIR, MODEL, INV, OPS_TABLES, false>(L, s);
    if (rc >= 0) return rc;
  }
  // plain transforms with 32 values per thread: one shared-memory exchange per
  // transform (N = 512, 1024)
  constexpr bool E32 = (N == 512 || N == 1024);
  if constexpr (MODE == COL_UPDATE && MODEL != MK_TUNGSTEN) {
    if (L.computed) return launch_col_direct<Real, N, MODE, DIR, MODEL, INV, OPS_COMPUTED>(L, s);
  }
  if constexpr (MODE == COL_UPDATE && MODEL != MK_ALUMINUM_G) {
    if (L.fold_ops) return launch_col_direct<Real, N, MODE, DIR, MODEL, INV, OPS_FOLDED>(L, s);
  }
  if constexpr (MODE == COL_PLAIN && E32)
    if (L.e32) return launch_col_direct<Real, N, MODE, DIR, MODEL, INV, OPS_TABLES, 32>(L, s);
  return launch_col_direct<Real, N, MODE, DIR, MODEL, INV, OPS_TABLES>(L, s);
}

template <typename Real, int N>
static int launch_col_n(const ColLaunch &L, cudaStream_t s) {
  if (L.mode == COL_PLAIN) {
    if (L.dir < 0) return launch_col_t<Real, N, COL_PLAIN, -1, 0, false>(L, s);
    return launch_col_t<Real, N, COL_PLAIN, +1, 0, false>(L, s);
  }
  switch (L.model) {
    case MK_PLAIN:
      return L.inverse_after ? launch_col_t<Real, N, COL_UPDATE, -1, MK_PLAIN, true>(L, s)
                             : launch_col_t<Real, N, COL_UPDATE, -1, MK_PLAIN, false>(L, s);
    case MK_TUNGSTEN:
      return L.inverse_after ? launch_col_t<Real, N, COL_UPDATE, -1, MK_TUNGSTEN, true>(L, s)
                             : launch_col_t<Real, N, COL_UPDATE, -1, MK_TUNGSTEN, false>(L, s);
    case MK_FILTERED:
      return L.inverse_after ? launch_col_t<Real, N, COL_UPDATE, -1, MK_FILTERED, true>(L, s)
                             : launch_col_t<Real, N, COL_UPDATE, -1, MK_FILTERED, false>(L, s);
    case MK_ALUMINUM_G:  // direct-load kernel, per-mode tables (opL, opN, chi, P_F)
      if (!L.inverse_after) return (int)cudaErrorInvalidValue;
      return launch_col_direct<Real, N, COL_UPDATE, -1, MK_ALUMINUM_G, true, OPS_TABLES>(L, s);
  }
  return (int)cudaErrorInvalidValue;
}

template <typename Real> static XArgs<Real> x_args(const XLaunch &L) {
  XArgs<Real> a;
  a.in0 = L.in0;
  a.in1 = L.in1;
  a.in2 = L.in2;
  a.time = L.time;
  for (int i = 0; i < 18; ++i) a.al[i] = L.al[i];
  a.out = L.out;
  a.rin = reinterpret_cast<const Real *>(L.rin);
  a.rout = reinterpret_cast<Real *>(L.rout);
  a.tw = L.tw;
  a.nyq_off = L.nyq_off;
  a.rows = L.rows;
  a.scale = L.scale;
  a.mean = L.mean;
  a.c0 = (Real)L.c[0];
  a.c1 = (Real)L.c[1];
  a.c2 = (Real)L.c[2];
  a.c3 = (Real)L.c[3];
  a.c4 = (Real)L.c[4];
  a.c5 = (Real)L.c[5];
  a.flag = L.flag;
  return a;
}

template <typename Real, int R, int MODEL, int H = 1>
static int launch_x_sq(const XLaunch &L, cudaStream_t s) {
  using Cfg = XSqCfg<Real, R, MODEL, H>;
  if (L.rows % Cfg::W != 0 || Cfg::SMEM > (size_t)kMaxDynSmem) return -1;
  constexpr int NT = Cfg::W * R;
  auto k = x_sq_kernel<Real, R, MODEL, H>;
  static int setup[kDevCache];
  const int occ = kernel_setup(k, NT, Cfg::SMEM, setup);
  const int ntiles = L.rows / Cfg::W;
  int G = (L.num_sms > 0 ? L.num_sms : 148) * occ;
  if (G > ntiles) G = ntiles;
  k<<<G, NT, Cfg::SMEM, s>>>(x_args<Real>(L));
  return (int)cudaGetLastError();
}

template <typename Real, int R, int MODEL, int H, int MINB = (H == 1 ? 4 : 2), bool PF = false>
static int launch_x_sqd(const XLaunch &L, cudaStream_t s) {
  using Cfg = XSqdCfg<Real, R, MODEL, H>;
  if (L.rows % Cfg::ROWS != 0 || Cfg::SMEM > (size_t)kMaxDynSmem) return -1;
  auto k = x_sqd_kernel<Real, R, MODEL, H, MINB, PF>;
  static int setup[kDevCache];
  const int occ = kernel_setup(k, Cfg::NT, Cfg::SMEM, setup);
  const int ngroups = L.rows / Cfg::ROWS;
  int G = (L.num_sms > 0 ? L.num_sms : 148) * occ;
  if (G > ngroups) G = ngroups;
  k<<<G, Cfg::NT, Cfg::SMEM, s>>>(x_args<Real>(L));
  return (int)cudaGetLastError();
}

template <typename Real, int M, int MODEL>
static int launch_x_tma(const XLaunch &L, cudaStream_t s) {
  if constexpr (M < 16) {
    return -1;
  } else {
    using Cfg = XCfg<Real, M, MODEL>;
    if (L.rows % Cfg::W != 0 || Cfg::SMEM > (size_t)kMaxDynSmem) return -1;
    constexpr int NT = Cfg::W * (M / Plan<M>::E);
    auto k = x_tma_kernel<Real, M, MODEL>;
    static int setup[kDevCache];
    const int occ = kernel_setup(k, NT, Cfg::SMEM, setup);
    XArgs<Real> a;
    a.in0 = L.in0;
    a.in1 = L.in1;
    a.in2 = L.in2;
    a.time = L.time;
    for (int i = 0; i < 18; ++i) a.al[i] = L.al[i];
    a.out = L.out;
    a.rin = nullptr;
    a.rout = nullptr;
    a.tw = L.tw;
    a.nyq_off = L.nyq_off;
    a.rows = L.rows;
    a.scale = L.scale;
    a.mean = L.mean;
    a.c0 = (Real)L.c[0];
    a.c1 = (Real)L.c[1];
    a.c2 = (Real)L.c[2];
    a.c3 = (Real)L.c[3];
    a.c4 = (Real)L.c[4];
    a.c5 = (Real)L.c[5];
    a.flag = L.flag;
    const int ntiles = L.rows / Cfg::W;
    int G = (L.num_sms > 0 ? L.num_sms : 148) * occ;
    if (G > ntiles) G = ntiles;
    k<<<G, NT, Cfg::SMEM, s>>>(a);
    return (int)cudaGetLastError();
  }
}

template <typename Real, int M, int MODE, int MODEL>
static int launch_x_t(const XLaunch &L, cudaStream_t s) {
  using C = typename Cx<Real>::T;
  constexpr int W = Width<Real>::W;
  constexpr int NT = W * (M / Plan<M>::E);
  const size_t smem = sizeof(C) * ((size_t)2 * M + (size_t)(M + 1) * (W + 1));
  auto k = x_kernel<Real, M, MODE, MODEL>;
  static int setup[kDevCache];
  kernel_setup(k, NT, smem, setup);
  XArgs<Real> a;
  a.in0 = L.in0;
  a.in1 = L.in1;
  a.in2 = L.in2;
  a.time = L.time;
  for (int i = 0; i < 18; ++i) a.al[i] = L.al[i];
  a.out = L.out;
  a.rin = reinterpret_cast<const Real *>(L.rin);
  a.rout = reinterpret_cast<Real *>(L.rout);
  a.tw = L.tw;
  a.nyq_off = L.nyq_off;
  a.rows = L.rows;
  a.scale = L.scale;
  a.mean = L.mean;
  a.c0 = (Real)L.c[0];
  a.c1 = (Real)L.c[1];
  a.c2 = (Real)L.c[2];
  a.c3 = (Real)L.c[3];
  a.c4 = (Real)L.c[4];
  a.c5 = (Real)L.c[5];
  a.flag = L.flag;
  const int blocks = (L.rows + W - 1) / W;
  k<<<blocks, NT, smem, s>>>(a);
  return (int)cudaGetLastError();
}

template <typename Real, int M>
static int launch_x_m(const XLaunch &L, cudaStream_t s) {
  if (L.mode == X_R2C) return launch_x_t<Real, M, X_R2C, 0>(L, s);
  if (L.mode == X_C2R) return launch_x_t<Real, M, X_C2R, 0>(L, s);
  if (L.sq_direct) {  // warp-square transforms, rows loaded straight into registers
    int rc = -1;
    if constexpr (M == 64 || M == 256 || ((M == 128 || M == 512) && sizeof(Real) == 4)) {
      constexpr int H = (M == 64 || M == 256) ? 1 : 2;
      constexpr int R = (M == 64 || M == 128) ? 8 : 16;
      // sq_direct 2: the next row loaded into registers during the current
      // row's transforms, at half the resident CTAs (twice the registers)
      constexpr int MINB_PF = H == 1 ? 2 : 1;
      if (L.sq_direct == 2) {
        if (L.model == MK_PLAIN) rc = launch_x_sqd<Real, R, MK_PLAIN, H, MINB_PF, true>(L, s);
        if (L.model == MK_FILTERED) rc = launch_x_sqd<Real, R, MK_FILTERED, H, MINB_PF, true>(L, s);
      } else {
        if (L.model == MK_PLAIN) rc = launch_x_sqd<Real, R, MK_PLAIN, H>(L, s);
        if (L.model == MK_FILTERED) rc = launch_x_sqd<Real, R, MK_FILTERED, H>(L, s);
      }
    }
    if (rc >= 0) return rc;
  }
  if (L.use_tma) {
    int rc = -1;
    if constexpr (M == 64 || M == 256) {
      constexpr int R = M == 64 ? 8 : 16;
      if (!L.no_sq) switch (L.model) {
          case MK_PLAIN: rc = launch_x_sq<Real, R, MK_PLAIN>(L, s); break;
          case MK_TUNGSTEN: rc = launch_x_sq<Real, R, MK_TUNGSTEN>(L, s); break;
          case MK_FILTERED: rc = launch_x_sq<Real, R, MK_FILTERED>(L, s); break;
        }
      if (rc >= 0) return rc;
    }
    // M = 2 R^2 (FP32, one field per row): radix-2 around two R^2 transforms
    if constexpr ((M == 128 || M == 512) && sizeof(Real) == 4) {
      constexpr int R = M == 128 ? 8 : 16;
      if (!L.no_sq) switch (L.model) {
          case MK_PLAIN: rc = launch_x_sq<Real, R, MK_PLAIN, 2>(L, s); break;
          case MK_FILTERED: rc = launch_x_sq<Real, R, MK_FILTERED, 2>(L, s); break;
          default: break;
        }
      if (rc >= 0) return rc;
    }
    switch (L.model) {
      case MK_PLAIN: rc = launch_x_tma<Real, M, MK_PLAIN>(L, s); break;
      case MK_TUNGSTEN: rc = launch_x_tma<Real, M, MK_TUNGSTEN>(L, s); break;
      case MK_FILTERED: rc = launch_x_tma<Real, M, MK_FILTERED>(L, s); break;
    }
    if (rc >= 0) return rc;
  }
  switch (L.model) {
    case MK_PLAIN: return launch_x_t<Real, M, X_FUSED, MK_PLAIN>(L, s);
    case MK_TUNGSTEN: return launch_x_t<Real, M, X_FUSED, MK_TUNGSTEN>(L, s);
    case MK_FILTERED: return launch_x_t<Real, M, X_FUSED, MK_FILTERED>(L, s);
    case MK_ALUMINUM_G: return launch_x_t<Real, M, X_FUSED, MK_ALUMINUM_G>(L, s);
  }
  return (int)cudaErrorInvalidValue;
}

#define OPFC_SIZES(X) X(2) X(4) X(8) X(16) X(24) X(32) X(40) X(48) X(64) X(80) X(96) X(128) X(256) X(512) X(1024)

template <typename Real> int launch_col(const ColLaunch &L, cudaStream_t s) {
  switch (L.N) {
#define OPFC_CASE(n) \
  case n: return launch_col_n<Real, n>(L, s);
    OPFC_SIZES(OPFC_CASE)
#undef OPFC_CASE
    case 1:
      if (L.mode == COL_PLAIN && L.in[0] == L.out[0] && (L.nsets < 2 || L.in[1] == L.out[1])) return 0;
      return launch_col_n<Real, 1>(L, s);
  }
  return (int)cudaErrorInvalidValue;
}

template <typename Real> int launch_x(const XLaunch &L, cudaStream_t s) {
  switch (L.M) {
#define OPFC_CASE(n) \
  case n: return launch_x_m<Real, n>(L, s);
    OPFC_SIZES(OPFC_CASE)
#undef OPFC_CASE
    case 1: return launch_x_m<Real, 1>(L, s);
  }
  return (int)cudaErrorInvalidValue;
}

template <typename Real>
int launch_herm_fix(void *psi, long long nyq_off, int M, int n1, int n2, cudaStream_t s, double *time,
                    double dt_time, int planes) {
  const long long plane = (long long)n1 * n2;
  using C = typename Cx<Real>::T;
  C *p = reinterpret_cast<C *>(psi);
  if ((planes & 3) == 3) {
    dim3 grid((unsigned)((plane + 255) / 256), 2);
    herm_fix_kernel<Real><<<grid, 256, 0, s>>>(p, nyq_off, M, n1, n2, time, dt_time);
  } else if (planes & 1) {  // the kx = 0 plane only (stride M)
    herm_fix_kernel<Real><<<(unsigned)((plane + 255) / 256), 256, 0, s>>>(p, nyq_off, M, n1, n2, time, dt_time);
  } else if (planes & 2) {  // the Nyquist plane only: its rows are contiguous (stride 1)
    herm_fix_kernel<Real><<<(unsigned)((plane + 255) / 256), 256, 0, s>>>(p + nyq_off, 0, 1, n1, n2, time, dt_time);
  } else if (time) {  // no plane: only the device time advances
    herm_fix_kernel<Real><<<1, 1, 0, s>>>(p, nyq_off, M, 0, 0, time, dt_time);
  }
  return (int)cudaGetLastError();
}

static inline int grid_for(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

template <typename Real>
int launch_to_ref(const void *in, void *out, int out_is_f64, int M, int n1, int n2, long long nyq_off,
                  int dc_override, double dc_re, cudaStream_t s) {
  const long long nc = (long long)(M + 1) * n1 * n2;
  const auto *pin = reinterpret_cast<const typename Cx<Real>::T *>(in);
  if (out_is_f64)
    to_ref_kernel<Real, double><<<grid_for(nc), 256, 0, s>>>(pin, (double *)out, M, n1, n2, nyq_off,
                                                             dc_override, dc_re);
  else
    to_ref_kernel<Real, float><<<grid_for(nc), 256, 0, s>>>(pin, (float *)out, M, n1, n2, nyq_off,
                                                            dc_override, dc_re);
  return (int)cudaGetLastError();
}

template <typename Real>
int launch_from_ref(const void *in, int in_is_f64, void *out, int M, int n1, int n2, long long nyq_off,
                    cudaStream_t s) {
  const long long nc = (long long)(M + 1) * n1 * n2;
  auto *pout = reinterpret_cast<typename Cx<Real>::T *>(out);
  if (in_is_f64)
    from_ref_kernel<Real, double><<<grid_for(nc), 256, 0, s>>>((const double *)in, pout, M, n1, n2,
                                                               nyq_off);
  else
    from_ref_kernel<Real, float><<<grid_for(nc), 256, 0, s>>>((const float *)in, pout, M, n1, n2,
                                                              nyq_off);
  return (int)cudaGetLastError();
}

template <typename Real>
int launch_cast_real(const void *in, int in_is_f64, void *out, int out_is_f64, size_t n,
                     cudaStream_t s) {
  const int g = grid_for((long long)n);
  if (in_is_f64 && out_is_f64)
    cast_kernel<double, double><<<g, 256, 0, s>>>((const double *)in, (double *)out, n);
  else if (in_is_f64)
    cast_kernel<double, float><<<g, 256, 0, s>>>((const double *)in, (float *)out, n);
  else if (out_is_f64)
    cast_kernel<float, double><<<g, 256, 0, s>>>((const float *)in, (double *)out, n);
  else
    cast_kernel<float, float><<<g, 256, 0, s>>>((const float *)in, (float *)out, n);
  return (int)cudaGetLastError();
}

template <typename Real>
int launch_sum_pow(const void *x, size_t n, int p, double *partials, int nblocks, cudaStream_t s) {
  sum_pow_kernel<Real><<<nblocks, 256, 0, s>>>(reinterpret_cast<const Real *>(x), n, p, partials);
  return (int)cudaGetLastError();
}

template <typename Real>
int launch_energy_k(const void *psi_hat, int M, int n1, int n2, long long nyq_off, const double *dx,
                    double r, double *partials, int nblocks, cudaStream_t s) {
  const double two_pi = 6.283185307179586476925286766559;
  EnergyK ek;
  ek.f0 = two_pi / (dx[0] * (2 * M));
  ek.f1 = two_pi / (dx[1] * n1);
  ek.f2 = two_pi / (dx[2] * n2);
  ek.r = r;
  energy_k_kernel<Real><<<nblocks, 256, 0, s>>>(
      reinterpret_cast<const typename Cx<Real>::T *>(psi_hat), M, n1, n2, nyq_off, ek, partials);
  return (int)cudaGetLastError();
}

#define OPFC_INSTANTIATE(R)                                                                          \
  template int launch_col<R>(const ColLaunch &, cudaStream_t);                                       \
  template int launch_x<R>(const XLaunch &, cudaStream_t);                                           \
  template int launch_herm_fix<R>(void *, long long, int, int, int, cudaStream_t, double *, double, int);  \
  template int launch_to_ref<R>(const void *, void *, int, int, int, int, long long, int, double,    \
                                cudaStream_t);                                                       \
  template int launch_from_ref<R>(const void *, int, void *, int, int, int, long long, cudaStream_t); \
  template int launch_cast_real<R>(const void *, int, void *, int, size_t, cudaStream_t);            \
  template int launch_sum_pow<R>(const void *, size_t, int, double *, int, cudaStream_t);            \
  template int launch_energy_k<R>(const void *, int, int, int, long long, const double *, double,    \
                                  double *, int, cudaStream_t);

// Other translation units that include this header (ensemble*.cu) call the
// launchers without instantiating the pass kernels a second time; the
// instantiations live in kernels_f32.cu and kernels_f64.cu.
#define OPFC_EXTERN(R)                                                                                      \
  extern template int launch_col<R>(const ColLaunch &, cudaStream_t);                                       \
  extern template int launch_x<R>(const XLaunch &, cudaStream_t);                                           \
  extern template int launch_herm_fix<R>(void *, long long, int, int, int, cudaStream_t, double *, double, int);  \
  extern template int launch_to_ref<R>(const void *, void *, int, int, int, int, long long, int, double,    \
                                       cudaStream_t);                                                       \
  extern template int launch_from_ref<R>(const void *, int, void *, int, int, int, long long, cudaStream_t); \
  extern template int launch_cast_real<R>(const void *, int, void *, int, size_t, cudaStream_t);            \
  extern template int launch_sum_pow<R>(const void *, size_t, int, double *, int, cudaStream_t);            \
  extern template int launch_energy_k<R>(const void *, int, int, int, long long, const double *, double,    \
                                         double *, int, cudaStream_t);

}  // namespace opfc
