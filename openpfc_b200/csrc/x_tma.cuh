// x_tma.cuh -- persistent fused x pass (C2R -> nonlinearity -> R2C per row),
// fed by bulk copies.
//
// A tile is W consecutive rows of the split layout (W x M contiguous complex
// values plus W contiguous Nyquist values).  One thread per CTA issues one
// cp.async.bulk per row into a padded shared row (pitch M+2 complex, so the
// c-fastest reads of the C2R pre-processing are conflict-free) and one for the
// Nyquist values, all completing on the stage's mbarrier.  STAGES tiles are in
// flight per CTA; after the pre-processing has pulled a tile into registers the
// same buffer becomes the FFT exchange space ([p][c], pitch W+1).
#pragma once
#include "col_tma.cuh"

namespace opfc {

__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(src)), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

template <typename Real, int M, int MODEL> struct XCfg {
  using C = typename CxP<Real>::T;
  static constexpr int W = Width<Real>::W;
  static constexpr int P = M + 2;  // padded row pitch in complex values (16-byte multiple)
  static constexpr size_t TILE = size_t(W) * P * sizeof(C) + size_t(W) * sizeof(C);
  static constexpr size_t EXCH = size_t(M + 1) * (W + 1) * sizeof(C);
  static constexpr size_t BUF = align128(TILE > EXCH ? TILE : EXCH);
  static constexpr int NARR = MODEL == MK_TUNGSTEN ? 2 : 1;
  static constexpr size_t STAGE = BUF * NARR;
  static constexpr size_t TW = align128(size_t(2 * M) * sizeof(C));
  static constexpr int STAGES = 2;
  static constexpr size_t SMEM = TW + STAGES * STAGE + 64;
  static constexpr unsigned TX = unsigned((size_t(W) * M + W) * sizeof(C)) * NARR;
};

// C2R pre-processing from row-major padded rows: Z'[k] of row c.
template <typename C, int M, int P, int E>
__device__ __forceinline__ void x_pre_rows(const C *tile, const C *nyq, const C *tw, int c, int j,
                                           C (&v)[E]) {
  constexpr int T = M / E;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int k = j + T * m;
    C X = k == 0 ? tile[c * P] : tile[c * P + k];
    C Y = k == 0 ? nyq[c] : tile[c * P + (M - k)];
    if (k == 0) {
      X.y = 0;
      Y.y = 0;
    }
    const C s = mk<C>(X.x + Y.x, X.y - Y.y);
    const C d = mk<C>(X.x - Y.x, X.y + Y.y);
    const C e = twmul<+1>(d, tw[k]);
    v[m] = mk<C>(s.x - e.y, s.y + e.x);
  }
}

template <typename Real, int M, int MODEL>
__global__ void __launch_bounds__(Width<Real>::W *(M / Plan<M>::E))
    x_tma_kernel(const XArgs<Real> a) {
  using Cfg = XCfg<Real, M, MODEL>;
  using C = typename CxP<Real>::T;
  constexpr int W = Cfg::W;
  constexpr int E = Plan<M>::E;
  constexpr int T = M / E;
  constexpr int NT = W * T;
  constexpr int N0 = 2 * M;
  constexpr int ld = W + 1;
  constexpr int STAGES = Cfg::STAGES;
  extern __shared__ __align__(128) unsigned char smraw[];
  C *tw = reinterpret_cast<C *>(smraw);
  unsigned char *stage0 = smraw + Cfg::TW;
  uint64_t *bars = reinterpret_cast<uint64_t *>(stage0 + STAGES * Cfg::STAGE);

  const int tid = threadIdx.x;
  const int c = tid % W;
  const int j = tid / W;
  const C *gtw = reinterpret_cast<const C *>(a.tw);
  for (int i = tid; i < N0; i += NT) tw[i] = gtw[i];
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

  C *out = reinterpret_cast<C *>(a.out);
  int it = 0;
  bool alive = true;
  bool bad = false;
  for (int t = blockIdx.x; t < ntiles; t += G, ++it) {
    const int s = it % STAGES;
    const bool ok = mbar_wait(&bars[s], (unsigned)(it / STAGES) & 1u);
    if (!__syncthreads_and(ok)) {
      alive = false;
      break;
    }
    unsigned char *st = stage0 + s * Cfg::STAGE;
    C *buf0 = reinterpret_cast<C *>(st);
    C v[E];
    x_pre_rows<C, M, Cfg::P, E>(buf0, buf0 + W * Cfg::P, tw, c, j, v);
    if constexpr (MODEL == MK_TUNGSTEN) {
      C *buf1 = reinterpret_cast<C *>(st + Cfg::BUF);
      C u[E];
      x_pre_rows<C, M, Cfg::P, E>(buf1, buf1 + W * Cfg::P, tw, c, j, u);
      __syncthreads();
      fft_line<C, M, +1, N0>(v, buf0, ld, c, j, tw);
      fft_line<C, M, +1, N0>(u, buf1, ld, c, j, tw);
      // N = p3b u^2 + p4b u^3 + q3b v^2 + q4b v^3 - stabP u with u = psi, v = psi_MF
      // (apps/tungsten/include/tungsten/cpu/tungsten_model.hpp:334-350)
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const Real ux = to_real_plus_mean(v[m].x, a.scale, a.mean);
        const Real uy = to_real_plus_mean(v[m].y, a.scale, a.mean);
        const Real vx = to_real_plus_mean(u[m].x, a.scale, a.mean);
        const Real vy = to_real_plus_mean(u[m].y, a.scale, a.mean);
        const Real nx = a.c0 * ux * ux + a.c1 * ux * ux * ux + a.c2 * vx * vx + a.c3 * vx * vx * vx - a.c4 * ux;
        const Real ny = a.c0 * uy * uy + a.c1 * uy * uy * uy + a.c2 * vy * vy + a.c3 * vy * vy * vy - a.c4 * uy;
        bad |= !(isfinite(nx) && isfinite(ny));
        v[m] = mk<C>(nx, ny);
      }
    } else {
      __syncthreads();
      fft_line<C, M, +1, N0>(v, buf0, ld, c, j, tw);
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const Real x = to_real_plus_mean(v[m].x, a.scale, a.mean);
        const Real y = to_real_plus_mean(v[m].y, a.scale, a.mean);
        Real nx, ny;
        if constexpr (MODEL == MK_FILTERED) {
          // N = p2 v^2/2 + p3 v^3/3 + p4 v^4/4 of the filtered density
          nx = x * x * (a.c0 + a.c1 * x + a.c2 * x * x);
          ny = y * y * (a.c0 + a.c1 * y + a.c2 * y * y);
        } else {
          // N = psi^3 (docs/api/examples/10_complete_pfc_model.cpp:128-130)
          nx = x * x * x;
          ny = y * y * y;
        }
        bad |= !(isfinite(nx) && isfinite(ny));
        v[m] = mk<C>(nx, ny);
      }
    }
    fft_line<C, M, -1, N0>(v, buf0, ld, c, j, tw);
#pragma unroll
    for (int m = 0; m < E; ++m) buf0[(j + T * m) * ld + c] = v[m];
    __syncthreads();
    x_post_store<C, M, W, NT>(buf0, tw, out, a.nyq_off, t * W, a.rows, tid);
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

}  // namespace opfc
