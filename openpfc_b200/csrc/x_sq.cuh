// x_sq.cuh -- fused x pass for half lengths M = H*R*R (R = 8, 16; H = 1, 2): one
// x-row is owned by R lanes of one warp, each holding E = H*R values.
//
// The complex FFT of length M is a two-stage Stockham (radix R, then radix R
// with twiddles W_M^{j r}); its single exchange is a padded R x (R+1) transpose
// private to the warp (__syncwarp only).  Stage-2 twiddles come from a per-stage
// table indexed [r-1][j], so the R lanes of a line read consecutive entries.
// The C2R pre-processing reads the bulk-copied rows directly; the R2C
// post-processing pairs Z[k] with Z[M-k] through warp shuffles (lane j holds
// k = j + R m, its partner is lane R-j), and stores the modes straight to HBM.
// Tiles of W rows arrive by cp.async.bulk exactly as in x_tma.cuh.
//
// H = 2 (M = 2 R^2): the inverse transform is one radix-2 decimation-in-
// frequency step (pairs p, p + M/2 sit in the same lane) followed by two
// length-R^2 transforms, which leaves the even and odd output positions in the
// two register halves; the nonlinearity is pointwise, and the forward transform
// is the matching decimation-in-time form (two length-R^2 transforms of the
// even / odd halves, then the radix-2 combine), which returns natural order.
#pragma once
#include "x_tma.cuh"

namespace opfc {

template <typename Real, int R, int MODEL, int H = 1> struct XSqCfg {
  using C = typename CxP<Real>::T;
  static constexpr int M = H * R * R;
  static constexpr int E = H * R;                // values per lane
  static constexpr int W = Width<Real>::W / H;  // rows (lines) per tile
  static constexpr int P = M + 2;           // padded row pitch of the landed tile
  static constexpr int EXL = R * (R + 1);   // exchange space per line
  static constexpr size_t TILE = (size_t(W) * P + W) * sizeof(C);
  static constexpr size_t EXCH = size_t(W) * EXL * sizeof(C);
  static constexpr size_t BUF = align128(TILE > EXCH ? TILE : EXCH);
  static constexpr int NARR = MODEL == MK_TUNGSTEN ? 2 : 1;
  static constexpr size_t STAGE = BUF * NARR;
  // only W_N0^k for k < M is read per tile (pre/post-processing); the stage-2
  // table is built from the global table, so 3 CTAs fit per SM
  static constexpr size_t TW = align128(size_t(M) * sizeof(C));
  static constexpr size_t TWS = align128(size_t(R) * R * sizeof(C));
  static constexpr int STAGES = 2;
  static constexpr size_t SMEM = TW + TWS + STAGES * STAGE + 64;
  static constexpr unsigned TX = unsigned((size_t(W) * M + W) * sizeof(C)) * NARR;
};

template <typename C> __device__ __forceinline__ C shfl_c(C v, int lane) {
  C r;
  r.x = __shfl_sync(0xffffffffu, v.x, lane);
  r.y = __shfl_sync(0xffffffffu, v.y, lane);
  return r;
}

// Pointwise nonlinearity of the pair of real values packed in one complex
// (z = x[2p] + i x[2p+1]), with the C2R scale and the mean added first:
// u = v sc + mn, N = u^3 (PLAIN) or u^2 (c0 + c1 u + c2 u^2) (FILTERED).  `guard`
// accumulates N * 0, which becomes NaN once any N is infinite or NaN: the pass's
// non-finite check at one fused multiply-add per value.  The FP32 form (pf2)
// issues every operation as a packed FP32x2 instruction; the cube rounds as
// (u u) u either way.
template <int MODEL, typename C, typename Real>
__device__ __forceinline__ C x_nonlin(C v, Real sc, Real mn, Real c0, Real c1, Real c2, C &guard) {
  const Real x = v.x * sc + mn, y = v.y * sc + mn;
  Real nx, ny;
  if constexpr (MODEL == MK_FILTERED) {
    nx = x * x * (c0 + c1 * x + c2 * x * x);
    ny = y * y * (c0 + c1 * y + c2 * y * y);
  } else {
    nx = x * x * x;
    ny = y * y * y;
  }
  guard.x = __fma_rn(nx, Real(0), guard.x);
  guard.y = __fma_rn(ny, Real(0), guard.y);
  return mk<C>(nx, ny);
}
template <int MODEL>
__device__ __forceinline__ pf2 x_nonlin(pf2 v, float sc, float mn, float c0, float c1, float c2, pf2 &guard) {
  const float2 u = __ffma2_rn(f2(v), make_float2(sc, sc), make_float2(mn, mn));
  const float2 u2 = __fmul2_rn(u, u);
  float2 n;
  if constexpr (MODEL == MK_FILTERED) {  // c0 + c1 u + c2 u^2 as (c2 u + c1) u + c0
    const float2 q = __ffma2_rn(u, make_float2(c2, c2), make_float2(c1, c1));
    n = __fmul2_rn(u2, __ffma2_rn(q, u, make_float2(c0, c0)));
  } else {
    n = __fmul2_rn(u2, u);
  }
  guard = p2(__ffma2_rn(n, make_float2(0.f, 0.f), f2(guard)));
  return p2(n);
}
// Length R*R transform of one line held as v[m] = x[j + R m]; same layout on exit.
template <typename C, int R, int DIR>
__device__ __forceinline__ void fft_sq(C (&v)[R], C *ex, int j, const C *tws) {
  Dft<R, DIR, C>::run(v);  // stage 1 (Ns = 1): outputs y[j R + r]
#pragma unroll
  for (int r = 0; r < R; ++r) ex[j * (R + 1) + r] = v[r];
  __syncwarp();
#pragma unroll
  for (int m = 0; m < R; ++m) v[m] = ex[m * (R + 1) + j];  // x[j + R m]
  __syncwarp();
#pragma unroll
  for (int r = 1; r < R; ++r) v[r] = twmul<DIR>(v[r], tws[(r - 1) * R + j]);
  Dft<R, DIR, C>::run(v);  // stage 2 (Ns = R): outputs x[j + R r]
}

// Length H*R*R inverse-style transform: natural order in (v[m] = x[j + R m],
// m < H R); H = 2 leaves the even outputs in v[0, R) and the odd ones in v[R, 2R)
// (v[m] = X[2 (j + R m)], v[R + m] = X[2 (j + R m) + 1]).  tw = W_{2M}^k, k < M.
template <typename C, int R, int H, int DIR>
__device__ __forceinline__ void fft_sq_dif(C (&v)[H * R], C *ex, int j, const C *tws, const C *tw) {
  if constexpr (H == 1) {
    fft_sq<C, R, DIR>(v, ex, j, tws);
  } else {
#pragma unroll
    for (int m = 0; m < R; ++m) {  // p = j + R m and p + M/2 share the lane
      const C a = v[m], b = v[m + R];
      v[m] = cadd(a, b);
      v[m + R] = twmul<DIR>(csub(a, b), tw[2 * (j + R * m)]);  // W_M^p
    }
    C h[R];
#pragma unroll
    for (int m = 0; m < R; ++m) h[m] = v[m];
    fft_sq<C, R, DIR>(h, ex, j, tws);
#pragma unroll
    for (int m = 0; m < R; ++m) {
      v[m] = h[m];
      h[m] = v[m + R];
    }
    fft_sq<C, R, DIR>(h, ex, j, tws);
#pragma unroll
    for (int m = 0; m < R; ++m) v[m + R] = h[m];
  }
}

// The matching forward-style transform: even / odd halves in (as fft_sq_dif
// leaves them), natural order out.
template <typename C, int R, int H, int DIR>
__device__ __forceinline__ void fft_sq_dit(C (&v)[H * R], C *ex, int j, const C *tws, const C *tw) {
  if constexpr (H == 1) {
    fft_sq<C, R, DIR>(v, ex, j, tws);
  } else {
    C h[R];
#pragma unroll
    for (int m = 0; m < R; ++m) h[m] = v[m];
    fft_sq<C, R, DIR>(h, ex, j, tws);
#pragma unroll
    for (int m = 0; m < R; ++m) {
      v[m] = h[m];
      h[m] = v[m + R];
    }
    fft_sq<C, R, DIR>(h, ex, j, tws);
#pragma unroll
    for (int m = 0; m < R; ++m) {  // X[k] = A[k] + W_M^k B[k], X[k + M/2] = A[k] - W_M^k B[k]
      const C t = twmul<DIR>(h[m], tw[2 * (j + R * m)]);
      const C a0 = v[m];
      v[m] = cadd(a0, t);
      v[m + R] = csub(a0, t);
    }
  }
}

template <typename Real, int R, int MODEL, int H>
__global__ void __launch_bounds__(XSqCfg<Real, R, MODEL, H>::W *R) x_sq_kernel(const XArgs<Real> a) {
  using Cfg = XSqCfg<Real, R, MODEL, H>;
  using C = typename CxP<Real>::T;
  constexpr int M = Cfg::M;
  constexpr int E = Cfg::E;
  constexpr int W = Cfg::W;
  constexpr int NT = W * R;
  constexpr int N0 = 2 * M;
  constexpr int STAGES = Cfg::STAGES;
  extern __shared__ __align__(128) unsigned char smraw[];
  C *tw = reinterpret_cast<C *>(smraw);
  C *tws = reinterpret_cast<C *>(smraw + Cfg::TW);
  unsigned char *stage0 = smraw + Cfg::TW + Cfg::TWS;
  uint64_t *bars = reinterpret_cast<uint64_t *>(stage0 + STAGES * Cfg::STAGE);

  const int tid = threadIdx.x;
  const int j = tid % R;
  const int c = tid / R;
  const int lane = tid & 31;
  const int partner = (lane & ~(R - 1)) | ((R - j) & (R - 1));
  const C *gtw = reinterpret_cast<const C *>(a.tw);
  for (int i = tid; i < M; i += NT) tw[i] = gtw[i];
  for (int i = tid; i < (R - 1) * R; i += NT) {
    const int r = i / R + 1, k = i % R;
    tws[i] = gtw[((N0 / (R * R)) * k * r) % N0];  // W_{R^2}^{k r} = exp(-2 pi i k r / R^2)
  }
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();

  const int ntiles = a.rows / W;
  const int G = gridDim.x;
  const C *src[2] = {reinterpret_cast<const C *>(a.in0), reinterpret_cast<const C *>(a.in1)};
  auto issue = [&](int s, int t) {
    unsigned char *st = stage0 + s * Cfg::STAGE;
    mbar_expect_tx(&bars[s], Cfg::TX);
    const long long row0 = (long long)t * W;
#pragma unroll
    for (int q = 0; q < Cfg::NARR; ++q) {
      C *tile = reinterpret_cast<C *>(st + q * Cfg::BUF);
      for (int cc = 0; cc < W; ++cc)
        bulk_load(tile + cc * Cfg::P, src[q] + (row0 + cc) * M, unsigned(M * sizeof(C)), &bars[s]);
      bulk_load(tile + W * Cfg::P, src[q] + a.nyq_off + row0, unsigned(W * sizeof(C)), &bars[s]);
    }
  };
  if (tid == 0)
    for (int s = 0; s < STAGES; ++s) {
      const int t = blockIdx.x + s * G;
      if (t < ntiles) issue(s, t);
    }

  const Real sc = (Real)a.scale, mn = (Real)a.mean;
  C *out = reinterpret_cast<C *>(a.out);
  int it = 0;
  bool alive = true, bad = false;
  for (int t = blockIdx.x; t < ntiles; t += G, ++it) {
    const int s = it % STAGES;
    const bool ok = mbar_wait(&bars[s], (unsigned)(it / STAGES) & 1u);
    if (!__syncthreads_and(ok)) {
      alive = false;
      break;
    }
    unsigned char *st = stage0 + s * Cfg::STAGE;
    C *buf0 = reinterpret_cast<C *>(st);
    C *ex0 = buf0 + c * Cfg::EXL;
    C v[E];
    x_pre_rows<C, M, Cfg::P, E>(buf0, buf0 + W * Cfg::P, tw, c, j, v);
    if constexpr (MODEL == MK_TUNGSTEN) {
      static_assert(H == 1, "two-field rows use H = 1");
      C *buf1 = reinterpret_cast<C *>(st + Cfg::BUF);
      C u[E];
      x_pre_rows<C, M, Cfg::P, E>(buf1, buf1 + W * Cfg::P, tw, c, j, u);
      __syncthreads();  // landed rows consumed: the buffers become exchange space
      fft_sq<C, R, +1>(v, ex0, j, tws);
      fft_sq<C, R, +1>(u, buf1 + c * Cfg::EXL, j, tws);
      // N = p3b u^2 + p4b u^3 + q3b v^2 + q4b v^3 - stabP u with u = psi, v = psi_MF
      // (apps/tungsten/include/tungsten/cpu/tungsten_model.hpp:334-350)
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const Real ux = v[m].x * sc + mn, uy = v[m].y * sc + mn;
        const Real vx = u[m].x * sc + mn, vy = u[m].y * sc + mn;
        const Real nx = ux * ux * (a.c0 + a.c1 * ux) + vx * vx * (a.c2 + a.c3 * vx) - a.c4 * ux;
        const Real ny = uy * uy * (a.c0 + a.c1 * uy) + vy * vy * (a.c2 + a.c3 * vy) - a.c4 * uy;
        bad |= !(isfinite(nx) && isfinite(ny));
        v[m] = mk<C>(nx, ny);
      }
    } else {
      __syncthreads();
      fft_sq_dif<C, R, H, +1>(v, ex0, j, tws, tw);
      C guard = mk<C>(0, 0);
#pragma unroll
      for (int m = 0; m < E; ++m) v[m] = x_nonlin<MODEL>(v[m], sc, mn, a.c0, a.c1, a.c2, guard);
      bad |= isnan(guard.x) || isnan(guard.y);
    }
    fft_sq_dit<C, R, H, -1>(v, ex0, j, tws, tw);
    // R2C post-processing: X[k] = 1/2 (Z[k] + conj Z[M-k]) - i/2 W_N0^k (Z[k] - conj Z[M-k]);
    // lane j holds k = j + R m, Z[M - k] is element E-1-m of lane R-j (lane 0: element E-m)
    const long long row = (long long)t * W + c;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int k = j + R * m;
      C Y = shfl_c(v[E - 1 - m], partner);
      if (j == 0) Y = v[(E - m) % E];
      const C Z = v[m];
      const C sm = mk<C>(Z.x + Y.x, Z.y - Y.y);
      const C d = mk<C>(Z.x - Y.x, Z.y + Y.y);
      const C e = twmul<-1>(d, tw[k]);
      out[row * M + k] = mk<C>(Real(0.5) * (sm.x + e.y), Real(0.5) * (sm.y - e.x));
    }
    if (j == 0) out[a.nyq_off + row] = mk<C>(v[0].x - v[0].y, Real(0));
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      const int tn = t + STAGES * G;
      if (tn < ntiles) issue(s, tn);
    }
  }
  if (bad && a.flag) atomicOr(a.flag, 1u);
  if (!alive) {
    if (tid == 0 && a.flag) atomicOr(a.flag, 2u);
    const int mine = (ntiles - (int)blockIdx.x + G - 1) / G;
    const int issued = mine < it + STAGES ? mine : it + STAGES;
    for (int k = it; k < issued; ++k) mbar_wait(&bars[k % STAGES], (unsigned)(k / STAGES) & 1u);
  }
}

// ---------------------------------------------------------------------------
// Direct-load form (no staging ring): each lane loads its E values of the row
// straight from HBM (k = j + R m: 128-byte coalesced segments), parks them in
// the row's warp-private buffer in natural order, and the C2R pre-processing
// reads X[k] and X[M-k] from there; the rest is the kernel above.  Without the
// staged tiles a CTA needs only the exchange buffers, so more warps fit per SM
// (registers, not shared memory, bound the occupancy) and no CTA barrier runs
// inside the loop.  One field per row (PLAIN, FILTERED).
// ---------------------------------------------------------------------------
template <typename Real, int R, int MODEL, int H> struct XSqdCfg {
  using C = typename CxP<Real>::T;
  static constexpr int M = H * R * R;
  static constexpr int E = H * R;
  static constexpr int NT = 256;
  static constexpr int ROWS = NT / R;  // rows per CTA pass
  static constexpr int EXL0 = R * (R + 1);
  static constexpr int EXL = EXL0 > M + 1 ? EXL0 : M + 1;
  static constexpr size_t TW = align128(size_t(M) * sizeof(C));
  static constexpr size_t TWS = align128(size_t(R) * R * sizeof(C));
  static constexpr size_t SMEM = TW + TWS + size_t(ROWS) * EXL * sizeof(C);
};

// MINB resident CTAs per SM set the register budget (65536 / (256 MINB)).
// PF: the next row's values are loaded into registers while the current row is
// transformed (each row is read and written by the warp that owns it, so the
// early read of a later row never races its write).
template <typename Real, int R, int MODEL, int H, int MINB = (H == 1 ? 4 : 2), bool PF = false>
__global__ void __launch_bounds__(256, MINB) x_sqd_kernel(const XArgs<Real> a) {
  using Cfg = XSqdCfg<Real, R, MODEL, H>;
  using C = typename CxP<Real>::T;
  constexpr int M = Cfg::M;
  constexpr int E = Cfg::E;
  constexpr int NT = Cfg::NT;
  constexpr int ROWS = Cfg::ROWS;
  constexpr int N0 = 2 * M;
  extern __shared__ __align__(128) unsigned char smraw[];
  C *tw = reinterpret_cast<C *>(smraw);
  C *tws = reinterpret_cast<C *>(smraw + Cfg::TW);
  C *exall = reinterpret_cast<C *>(smraw + Cfg::TW + Cfg::TWS);

  const int tid = threadIdx.x;
  const int j = tid % R;
  const int c = tid / R;
  const int lane = tid & 31;
  const int partner = (lane & ~(R - 1)) | ((R - j) & (R - 1));
  const C *gtw = reinterpret_cast<const C *>(a.tw);
  for (int i = tid; i < M; i += NT) tw[i] = gtw[i];
  for (int i = tid; i < (R - 1) * R; i += NT) {
    const int r = i / R + 1, k = i % R;
    tws[i] = gtw[((N0 / (R * R)) * k * r) % N0];
  }
  __syncthreads();

  C *ex = exall + c * Cfg::EXL;
  const C *in = reinterpret_cast<const C *>(a.in0);
  C *out = reinterpret_cast<C *>(a.out);
  const Real sc = (Real)a.scale, mn = (Real)a.mean;
  C guard = mk<C>(0, 0);  // N * 0 summed over the rows: NaN once any N is not finite
  const long long rstep = (long long)gridDim.x * ROWS;
  C vn[PF ? E : 1];
  C nyqn = mk<C>(0, 0);
  if constexpr (PF) {
    const long long row = (long long)blockIdx.x * ROWS + c;
    if (row < a.rows) {
#pragma unroll
      for (int m = 0; m < E; ++m) vn[m] = in[row * M + j + R * m];
      nyqn = in[a.nyq_off + row];
    }
  }
  for (long long row0 = (long long)blockIdx.x * ROWS; row0 < a.rows; row0 += rstep) {
    const long long row = row0 + c;  // rows is a multiple of ROWS (launcher)
    C v[E];
    C nyq;
    if constexpr (PF) {
#pragma unroll
      for (int m = 0; m < E; ++m) v[m] = vn[m];
      nyq = nyqn;
      const long long rn = row + rstep;
      if (rn < a.rows) {
#pragma unroll
        for (int m = 0; m < E; ++m) vn[m] = in[rn * M + j + R * m];
        nyqn = in[a.nyq_off + rn];
      }
    } else {
#pragma unroll
      for (int m = 0; m < E; ++m) v[m] = in[row * M + j + R * m];
      nyq = in[a.nyq_off + row];
    }
    // natural order into the row buffer: ex[k] = X[k], ex[M] = X[M]
#pragma unroll
    for (int m = 0; m < E; ++m) ex[j + R * m] = v[m];
    if (j == 0) ex[M] = nyq;
    __syncwarp();
    // C2R pre-processing (x_pre_rows): Z'[k] from X[k] and X[M-k]
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int k = j + R * m;
      C X = v[m];
      C Y = ex[M - k];
      if (k == 0) {
        X.y = 0;
        Y.y = 0;
      }
      const C s2 = mk<C>(X.x + Y.x, X.y - Y.y);
      const C d = mk<C>(X.x - Y.x, X.y + Y.y);
      const C e = twmul<+1>(d, tw[k]);
      v[m] = mk<C>(s2.x - e.y, s2.y + e.x);
    }
    __syncwarp();  // row buffer free: it becomes the FFT exchange space
    fft_sq_dif<C, R, H, +1>(v, ex, j, tws, tw);
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = x_nonlin<MODEL>(v[m], sc, mn, a.c0, a.c1, a.c2, guard);
    fft_sq_dit<C, R, H, -1>(v, ex, j, tws, tw);
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int k = j + R * m;
      C Y = shfl_c(v[E - 1 - m], partner);
      if (j == 0) Y = v[(E - m) % E];
      const C Z = v[m];
      const C sm = mk<C>(Z.x + Y.x, Z.y - Y.y);
      const C d = mk<C>(Z.x - Y.x, Z.y + Y.y);
      const C e = twmul<-1>(d, tw[k]);
      out[row * M + k] = mk<C>(Real(0.5) * (sm.x + e.y), Real(0.5) * (sm.y - e.x));
    }
    if (j == 0) out[a.nyq_off + row] = mk<C>(v[0].x - v[0].y, Real(0));
    __syncwarp();  // exchange space reused by the next row
  }
  if ((isnan(guard.x) || isnan(guard.y)) && a.flag) atomicOr(a.flag, 1u);
}

}  // namespace opfc
