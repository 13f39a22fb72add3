// col_tma.cuh -- persistent, TMA-fed column passes (y and z transforms, and
// the fused z transform + ETD update).
//
// Each CTA owns one SM and walks the tiles t = blockIdx.x + i * gridDim.x.  A
// tile is W adjacent columns x N rows of one strided axis; it arrives in shared
// memory through cp.async.bulk.tensor (no multicast) and is consumed from an
// mbarrier-guarded ring of STAGES buffers, so the loads of the next tiles are in
// flight while the current tile is transformed.  The shared tile [p][c] (pitch
// W, c fastest) is also the FFT's exchange buffer.  For the ETD update the state
// psi_hat and the operator tables of the same tile ride in the same stage.
// Every wait is bounded (4 s of globaltimer); on expiry the CTA records
// OPFC timeout bit 2 in `flag`, drains its own loads (bounded) and leaves.
#pragma once
#include <cuda.h>

#include "fft_core.cuh"

namespace opfc {

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for phase `parity` of `bar`; false after limit_ns of %globaltimer (4 s
// in the pass kernels).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity,
                                          unsigned long long limit_ns = 4000000000ull) {
  const unsigned a = smem_u32(bar);
  unsigned long long t0 = 0;
  for (unsigned i = 0;; ++i) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if (i == 0)
      t0 = global_ns();
    else if ((i & 31u) == 0 && global_ns() - t0 > limit_ns)
      return false;
  }
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x,
                                            int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

constexpr size_t align128(size_t b) { return (b + 127) & ~size_t(127); }
constexpr int kMaxDynSmem = 232448;  // 227 KB opt-in per CTA on sm_100

template <typename Real, int N, int W, int MODE, int MODEL, int OPS = 0, int SCAP = 3, bool PP = false>
struct TmaCfg {
  using C = typename Cx<Real>::T;
  static constexpr bool UPD = MODE == COL_UPDATE;
  static constexpr bool CHI = UPD && MODEL != MK_PLAIN;
  static constexpr size_t TILE_C = size_t(N) * W * sizeof(C);
  static constexpr size_t TILE_R = size_t(N) * W * sizeof(Real);
  // folded tables (OPS 3): rows |kz| = 0 .. N/2 of the tile's columns, as 3
  // boxes of RBF = N/4 rows of (opL, opN) pairs (and of the filter)
  static constexpr int RBF = N / 4;
  static constexpr size_t FOLD_C = 3 * size_t(RBF) * W * sizeof(C);
  static constexpr size_t FOLD = FOLD_C + (CHI ? 3 * size_t(RBF) * W * sizeof(Real) : 0);
  // radial operators come from an L2-resident table and computed operators
  // from k^2: only the per-mode and the folded tables are staged
  static constexpr size_t STAGE =
      TILE_C + (UPD ? TILE_C + (OPS == 0 ? 2 * TILE_R + (CHI ? TILE_R : 0) : OPS == 3 ? FOLD : 0) : 0);
  static constexpr size_t TW = align128(size_t(N) * sizeof(C));
  // PP: a second FFT exchange buffer (ping-pong with the landed tile)
  static constexpr size_t XB = PP ? align128(TILE_C) : 0;
  static constexpr int S0 = int((kMaxDynSmem - TW - XB - 128) / STAGE);
  static constexpr int STAGES = S0 > SCAP ? SCAP : S0;
  static constexpr size_t SMEM = TW + XB + size_t(STAGES > 0 ? STAGES : 1) * STAGE + 64;
  static constexpr int RB = N < 256 ? N : 256;  // rows per TMA box (box dims <= 256)
  static constexpr int NB = N / RB;
};

// Radial operator lookup: kx <= M unfolded, ky / kz folded to |k|.
template <typename Real>
__device__ __forceinline__ void radial_ops(const ColArgs<Real> &a, int kx, int ky, int kz, Real &la, Real &lb,
                                           Real &ch) {
  using C = typename Cx<Real>::T;
  const int fy = ky <= a.rad_n1 / 2 ? ky : a.rad_n1 - ky;
  const int fz = kz <= a.rad_n2 / 2 ? kz : a.rad_n2 - kz;
  const int m = kx * kx + fy * fy + fz * fz;
  const C o = __ldg(reinterpret_cast<const C *>(a.rad_ops) + m);
  la = o.x;
  lb = o.y;
  ch = a.rad_chi ? __ldg(a.rad_chi + m) : Real(1);
}

// Update-mode transform: stage twiddles from the register cache (TWR) or the
// shared table; PP exchanges through (buf, xb) in turn.
// K = index of this transform within the tile (continues the exchange parity).
template <typename C, int N, int D, bool TWR, bool PP = false, int K = 0>
__device__ __forceinline__ void upd_fft(C (&x)[Plan<N>::E], C *buf, int ld, int c, int j, const C *tw,
                                        const TwReg<C, N> &twr, C *xb = nullptr) {
  if constexpr (PP)
    fft_line_pp<C, N, D, TWR, K * fft_exchanges<N>()>(x, buf, xb, ld, c, j, tw, twr);
  else if constexpr (TWR)
    fft_line_rt<C, N, D>(x, buf, ld, c, j, twr);
  else
    fft_line<C, N, D, N>(x, buf, ld, c, j, tw);
}

// Outer index (ky of a z tile) of the o-th tile row in the order
// 0, 1, n-1, 2, n-2, ...: the rows ky and n - ky, which read the same folded
// table rows, follow each other, so the second read hits L2.  A bijection of
// [0, n).
__device__ __forceinline__ int paired_outer(int o, int n) {
  return o == 0 ? 0 : ((o & 1) ? (o + 1) / 2 : n - o / 2);
}

// Tensor maps: PLAIN uses m0 (array set 0) and m1 (array set 1); UPDATE uses
// m0 = N_hat partial (A), m1 = psi_hat, m2 = tab_a, m3 = tab_b, m4 = tab_chi
// (m2..m4 unused unless OPS == 0, per-mode tables); with OPS == 3, m2 = the
// folded (opL, opN) pairs and m3 = the folded filter.  MINB CTAs share an SM.
template <typename Real, int N, int W, int MODE, int DIR, int MODEL, bool INV, int OPS, int MINB, bool PP>
__global__ void __launch_bounds__(W *(N / Plan<N>::E), MINB)
    col_tma_kernel(const __grid_constant__ CUtensorMap m0, const __grid_constant__ CUtensorMap m1,
                   const __grid_constant__ CUtensorMap m2, const __grid_constant__ CUtensorMap m3,
                   const __grid_constant__ CUtensorMap m4, const ColArgs<Real> a, const int axis,
                   unsigned *flag) {
  using Cfg = TmaCfg<Real, N, W, MODE, MODEL, OPS, 3, PP>;
  using C = typename Cx<Real>::T;
  constexpr bool RADIAL = OPS == 1;
  constexpr bool COMPUTED = OPS == 2;
  constexpr bool FOLDED = OPS == 3;
  constexpr int E = Plan<N>::E;
  constexpr int T = N / E;
  constexpr int NT = W * T;
  constexpr int STAGES = Cfg::STAGES;
  constexpr bool UPD = Cfg::UPD;
  extern __shared__ __align__(128) unsigned char smraw[];
  C *tw = reinterpret_cast<C *>(smraw);
  C *xb = reinterpret_cast<C *>(smraw + Cfg::TW);  // PP exchange buffer (XB bytes)
  unsigned char *stage0 = smraw + Cfg::TW + Cfg::XB;
  uint64_t *bars = reinterpret_cast<uint64_t *>(stage0 + STAGES * Cfg::STAGE);

  const int tid = threadIdx.x;
  const int c = tid % W;
  const int j = tid / W;
  const C *gtw = reinterpret_cast<const C *>(a.tw);
  for (int i = tid; i < N; i += NT) tw[i] = gtw[i];
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // the update's two transforms per tile take their stage twiddles from
  // registers when few enough (loaded once: they depend only on j)
  constexpr bool TWR = UPD && TwReg<C, N>::CNT > 0 && TwReg<C, N>::CNT <= 16;
  TwReg<C, N> twr;
  if constexpr (TWR) twr.load(j, tw);

  const int set = blockIdx.y;
  const CUtensorMap *min = (MODE == COL_PLAIN && set == 1) ? &m1 : &m0;
  const ColSeg sg = a.seg0;
  const int ntm = sg.ntiles;
  const int G = gridDim.x;
  // FOLDED walks the z tiles' ky in (ky, N1 - ky) pairs
  const int nout = sg.tiles_inner > 0 ? ntm / sg.tiles_inner : 0;
  auto outer = [&](int o) { return FOLDED ? paired_outer(o, nout) : o; };

  auto issue = [&](int s, int t) {
    const int ti = t % sg.tiles_inner, to = outer(t / sg.tiles_inner);
    unsigned char *st = stage0 + s * Cfg::STAGE;
    mbar_expect_tx(&bars[s], (unsigned)Cfg::STAGE);
#pragma unroll
    for (int b = 0; b < Cfg::NB; ++b) {
      const int r0 = b * Cfg::RB;
      const int y = axis == 1 ? r0 : to, z = axis == 1 ? to : r0;
      const size_t offc = size_t(b) * Cfg::RB * W * sizeof(C);
      tma_load_3d(st + offc, min, &bars[s], ti * W * 2, y, z);
      if constexpr (UPD) {
        const size_t offr = size_t(b) * Cfg::RB * W * sizeof(Real);
        tma_load_3d(st + Cfg::TILE_C + offc, &m1, &bars[s], ti * W * 2, y, z);
        if constexpr (OPS != 0) continue;
        tma_load_3d(st + 2 * Cfg::TILE_C + offr, &m2, &bars[s], ti * W, y, z);
        tma_load_3d(st + 2 * Cfg::TILE_C + Cfg::TILE_R + offr, &m3, &bars[s], ti * W, y, z);
        if constexpr (Cfg::CHI)
          tma_load_3d(st + 2 * Cfg::TILE_C + 2 * Cfg::TILE_R + offr, &m4, &bars[s], ti * W, y, z);
      }
    }
    if constexpr (FOLDED) {
      // the tile's folded table rows |kz| = 0 .. N/2 at |ky| (rows past N/2 of
      // the last box lie outside the table and arrive zero-filled, unread)
      const int fy = fold_index(to, a.rad_n1);
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        tma_load_3d(st + 2 * Cfg::TILE_C + size_t(b) * Cfg::RBF * W * sizeof(C), &m2, &bars[s], ti * W * 2, fy,
                    b * Cfg::RBF);
        if constexpr (Cfg::CHI)
          tma_load_3d(st + 2 * Cfg::TILE_C + Cfg::FOLD_C + size_t(b) * Cfg::RBF * W * sizeof(Real), &m3, &bars[s],
                      ti * W, fy, b * Cfg::RBF);
      }
    }
  };

  if (tid == 0)
    for (int s = 0; s < STAGES; ++s) {
      const int t = blockIdx.x + s * G;
      if (t < ntm) issue(s, t);
    }

  const C *gin = reinterpret_cast<const C *>(a.in[set]);
  C *gout = reinterpret_cast<C *>(a.out[set]);
  (void)gin;
  int it = 0;
  bool alive = true;
  for (int t = blockIdx.x; t < ntm; t += G, ++it) {
    const int s = it % STAGES;
    const unsigned par = (unsigned)(it / STAGES) & 1u;
    const bool ok = mbar_wait(&bars[s], par);
    if (!__syncthreads_and(ok)) {
      alive = false;
      break;
    }
    unsigned char *st = stage0 + s * Cfg::STAGE;
    C *tin = reinterpret_cast<C *>(st);
    const int ti = t % sg.tiles_inner, to = outer(t / sg.tiles_inner);
    const long long base =
        sg.off + (long long)to * sg.s_outer + (long long)(ti * W + c) * sg.col_stride;
    const long long fs = sg.fft_stride;
    C v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = tin[(j + T * m) * W + c];
    // PP: the first exchange writes xb, so the tile needs no barrier here
    if constexpr (!PP) __syncthreads();
    if constexpr (MODE == COL_PLAIN) {
      if constexpr (PP)
        fft_line_pp<C, N, DIR, false>(v, tin, xb, W, c, j, tw, twr);
      else
        fft_line<C, N, DIR, N>(v, tin, W, c, j, tw);
#pragma unroll
      for (int m = 0; m < E; ++m) gout[base + (long long)(j + T * m) * fs] = v[m];
    } else {
      // radial operators: gather from L2 before the transform so the loads
      // overlap it (z pass: kx = column, ky = outer index, kz = p)
      Real rla[RADIAL ? E : 1], rlb[RADIAL ? E : 1], rch[RADIAL && Cfg::CHI ? E : 1];
      if constexpr (RADIAL) {
#pragma unroll
        for (int m = 0; m < E; ++m) {
          Real ch;
          radial_ops(a, ti * W + c, to, j + T * m, rla[m], rlb[m], ch);
          if constexpr (Cfg::CHI) rch[m] = ch;
        }
      }
      upd_fft<C, N, -1, TWR, PP, 0>(v, tin, W, c, j, tw, twr, xb);
      const C *tpsi = reinterpret_cast<const C *>(st + Cfg::TILE_C);
      const Real *ta = reinterpret_cast<const Real *>(st + 2 * Cfg::TILE_C);
      const Real *tb = ta + N * W;
      const Real *tc = tb + N * W;
      C *ph = reinterpret_cast<C *>(a.psi_hat);
      C w[Cfg::CHI ? E : 1];
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int e = (j + T * m) * W + c;
        const C p = tpsi[e];
        Real la, lb, ch = Real(1);
        if constexpr (RADIAL) {
          la = rla[m];
          lb = rlb[m];
          if constexpr (Cfg::CHI) ch = rch[m];
        } else if constexpr (COMPUTED) {
          computed_ops<Real, MODEL>(a, ti * W + c, to, j + T * m, la, lb, ch);
        } else if constexpr (FOLDED) {
          const int fz = fold_index(j + T * m, N);
          const C o = reinterpret_cast<const C *>(st + 2 * Cfg::TILE_C)[fz * W + c];
          la = o.x;
          lb = o.y;
          if constexpr (Cfg::CHI) ch = reinterpret_cast<const Real *>(st + 2 * Cfg::TILE_C + Cfg::FOLD_C)[fz * W + c];
        } else {
          la = ta[e];
          lb = tb[e];
          if constexpr (Cfg::CHI) ch = tc[e];
        }
        const C np = mk<C>(la * p.x + lb * v[m].x, la * p.y + lb * v[m].y);
        ph[base + (long long)(j + T * m) * fs] = np;
        if constexpr (Cfg::CHI) w[m] = cscale(np, ch);
        v[m] = np;
      }
      if constexpr (INV) {
        if constexpr (MODEL == MK_FILTERED) {
          upd_fft<C, N, +1, TWR, PP, 1>(w, tin, W, c, j, tw, twr, xb);
#pragma unroll
          for (int m = 0; m < E; ++m) gout[base + (long long)(j + T * m) * fs] = w[m];
        } else {
          upd_fft<C, N, +1, TWR, PP, 1>(v, tin, W, c, j, tw, twr, xb);
#pragma unroll
          for (int m = 0; m < E; ++m) gout[base + (long long)(j + T * m) * fs] = v[m];
          if constexpr (MODEL == MK_TUNGSTEN) {
            C *gout2 = reinterpret_cast<C *>(a.out[1]);
            upd_fft<C, N, +1, TWR, PP, 2>(w, tin, W, c, j, tw, twr, xb);
#pragma unroll
            for (int m = 0; m < E; ++m) gout2[base + (long long)(j + T * m) * fs] = w[m];
          }
        }
      }
    }
    // the stage's buffers were read and (as exchange space) written by the
    // generic proxy; order that before the next asynchronous fill
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      const int tn = t + STAGES * G;
      if (tn < ntm) issue(s, tn);
    }
  }

  if (!alive) {
    if (tid == 0) atomicOr(flag, 2u);
    // drain the loads this CTA still has in flight (bounded), then leave
    const int mine = (ntm - (int)blockIdx.x + G - 1) / G;
    const int issued = mine < it + STAGES ? mine : it + STAGES;
    for (int k = it; k < issued; ++k) mbar_wait(&bars[k % STAGES], (unsigned)(k / STAGES) & 1u);
    return;
  }

  // Nyquist-plane tiles: direct loads, stage 0 as the exchange buffer
  const ColSeg sn = a.seg1;
  C *sm = reinterpret_cast<C *>(stage0);
  for (int t = blockIdx.x; t < sn.ntiles; t += G) {
    const int ti = t % sn.tiles_inner, to = t / sn.tiles_inner;
    const int cg = ti * W + c;
    const bool ok = cg < sn.ncols;
    const long long base = sn.off + (long long)to * sn.s_outer + (long long)cg * sn.col_stride;
    const long long fs = sn.fft_stride;
    const C *in = reinterpret_cast<const C *>(a.in[set]);
    C v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = ok ? in[base + (long long)(j + T * m) * fs] : mk<C>(0, 0);
    if constexpr (MODE == COL_PLAIN) {
      fft_line<C, N, DIR, N>(v, sm, W, c, j, tw);
      if (ok) {
#pragma unroll
        for (int m = 0; m < E; ++m) gout[base + (long long)(j + T * m) * fs] = v[m];
      }
    } else {
      upd_fft<C, N, -1, TWR>(v, sm, W, c, j, tw, twr);
      C *ph = reinterpret_cast<C *>(a.psi_hat);
      C w[Cfg::CHI ? E : 1];
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const long long idx = base + (long long)(j + T * m) * fs;
        C np = mk<C>(0, 0);
        Real ch = Real(1);
        if (ok) {
          const C p = ph[idx];
          Real la, lb;
          if constexpr (RADIAL) {
            radial_ops(a, a.rad_M, cg, j + T * m, la, lb, ch);  // Nyquist plane: kx = M, ky = column
          } else if constexpr (COMPUTED) {
            computed_ops<Real, MODEL>(a, a.rad_M, cg, j + T * m, la, lb, ch);
          } else if constexpr (FOLDED) {
            folded_ops<Real, MODEL>(a, a.rad_M, cg, j + T * m, la, lb, ch);
          } else {
            la = a.tab_a[idx];
            lb = a.tab_b[idx];
            if constexpr (Cfg::CHI) ch = a.tab_chi[idx];
          }
          np = mk<C>(la * p.x + lb * v[m].x, la * p.y + lb * v[m].y);
          ph[idx] = np;
        }
        if constexpr (Cfg::CHI) w[m] = ok ? cscale(np, ch) : mk<C>(0, 0);
        v[m] = np;
      }
      if constexpr (INV) {
        if constexpr (MODEL == MK_FILTERED) {
          upd_fft<C, N, +1, TWR>(w, sm, W, c, j, tw, twr);
          if (ok) {
#pragma unroll
            for (int m = 0; m < E; ++m) gout[base + (long long)(j + T * m) * fs] = w[m];
          }
        } else {
          upd_fft<C, N, +1, TWR>(v, sm, W, c, j, tw, twr);
          if (ok) {
#pragma unroll
            for (int m = 0; m < E; ++m) gout[base + (long long)(j + T * m) * fs] = v[m];
          }
          if constexpr (MODEL == MK_TUNGSTEN) {
            C *gout2 = reinterpret_cast<C *>(a.out[1]);
            upd_fft<C, N, +1, TWR>(w, sm, W, c, j, tw, twr);
            if (ok) {
#pragma unroll
              for (int m = 0; m < E; ++m) gout2[base + (long long)(j + T * m) * fs] = w[m];
            }
          }
        }
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Box-ring fused z update with 128-byte tile rows (folded tables, N = 1024).
//
// Along z the rows of a column are one kz plane apart (4 MB at 1024^3 FP32), so
// each row of a tile is its own address translation and the bytes a row brings
// set the bandwidth: 64-byte rows (the ring kernel above, whose A + psi_hat +
// table stages do not fit twice at 128-byte rows) hold a plain z transform to
// ~2.5 TB/s at 1024^3, 128-byte rows reach 4-4.8 TB/s.  This kernel keeps
// tiles of W = Width<Real>::W columns (128-byte rows) and streams them through
// shared memory in boxes of 256 rows: per tile A boxes 0..3, then psi_hat boxes
// 0..3, through a ring of two 32 KB slots, the next box issued as soon as a
// slot is read; the transforms exchange through their own buffer.  32 values
// per thread (one exchange per transform): box b holds values 8b .. 8b+7 of
// every thread.  Operators from the folded tables through L2: a box's (opL,
// opN) pairs are issued before the box is waited for, the filter values after
// (fewer live registers).  Main segment only; the Nyquist
// plane runs as a separate direct-load launch.  Bounded waits as in
// col_tma_kernel (timeout bit 2 of `flag`).
// ---------------------------------------------------------------------------
template <typename Real, int N> struct RingCfg {
  using C = typename Cx<Real>::T;
  static constexpr int W = 128 / int(sizeof(C));
  static constexpr int E = 32;
  static constexpr int T = N / E;
  static constexpr int NT = W * T;
  static constexpr int RB = 256;                  // rows per box
  static constexpr int NB = N / RB;               // boxes per operand
  static constexpr int VB = RB / T;               // values per thread per box
  static constexpr size_t BOX = size_t(RB) * W * sizeof(C);
  static constexpr int LD = W + 1;                // exchange pitch
  static constexpr size_t TW = align128(size_t(N) * sizeof(C));
  static constexpr size_t XB = align128(size_t(N) * LD * sizeof(C));
  static constexpr size_t SLOTS = TW + XB;
  static constexpr size_t BARS = SLOTS + 2 * BOX;
  static constexpr size_t SMEM = BARS + 64;
  static constexpr bool FITS = SMEM <= size_t(kMaxDynSmem) && N % RB == 0 && RB % T == 0 && VB * NB == E;
};

template <typename Real, int N, int MODEL>
__global__ void __launch_bounds__(RingCfg<Real, N>::NT, 1)
    col_ring_kernel(const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mP,
                    const ColArgs<Real> a, unsigned *flag) {
  using Cfg = RingCfg<Real, N>;
  using C = typename Cx<Real>::T;
  constexpr int W = Cfg::W, E = Cfg::E, T = Cfg::T, NT = Cfg::NT, VB = Cfg::VB, NB = Cfg::NB;
  constexpr bool CHI = MODEL != MK_PLAIN;
  extern __shared__ __align__(128) unsigned char smraw[];
  C *tw = reinterpret_cast<C *>(smraw);
  C *xb = reinterpret_cast<C *>(smraw + Cfg::TW);
  unsigned char *slot_b = smraw + Cfg::SLOTS;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smraw + Cfg::BARS);

  const int tid = threadIdx.x;
  const int c = tid % W;
  const int j = tid / W;
  const C *gtw = reinterpret_cast<const C *>(a.tw);
  for (int i = tid; i < N; i += NT) tw[i] = gtw[i];
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  __syncthreads();

  const ColSeg sg = a.seg0;
  const int ntm = sg.ntiles;
  const int G = gridDim.x;
  const int nout = sg.tiles_inner > 0 ? ntm / sg.tiles_inner : 0;
  const int mine = (int)blockIdx.x < ntm ? (ntm - (int)blockIdx.x + G - 1) / G : 0;
  const int nq = mine * 2 * NB;  // boxes this CTA consumes
  // box q: tile blockIdx.x + (q / 2NB) G, A box (q % 2NB) or psi_hat box (q % 2NB - NB)
  auto issue = [&](int q) {
    const int t = (int)blockIdx.x + (q / (2 * NB)) * G;
    const int k = q % (2 * NB);
    const int ti = t % sg.tiles_inner, to = paired_outer(t / sg.tiles_inner, nout);
    uint64_t *bar = &bars[q & 1];
    mbar_expect_tx(bar, (unsigned)Cfg::BOX);
    tma_load_3d(slot_b + size_t(q & 1) * Cfg::BOX, k < NB ? &mA : &mP, bar, ti * W * 2, to, (k % NB) * Cfg::RB);
  };
  int qn = 0, qc = 0;  // next box to issue / to consume (the same on every thread)
  if (tid == 0)
    for (int q = 0; q < 2 && q < nq; ++q) issue(q);
  qn = nq < 2 ? nq : 2;
  bool alive = true;
  // wait for box qc; false (and the CTA leaves the loop) when the wait expires
  auto take = [&]() -> const C * {
    if (!__syncthreads_and(mbar_wait(&bars[qc & 1], (unsigned)(qc >> 1) & 1u))) return nullptr;
    return reinterpret_cast<const C *>(slot_b + size_t(qc & 1) * Cfg::BOX);
  };
  // box qc was read by every thread: refill its slot with box qc + 2
  auto release = [&]() {
    fence_proxy_async();
    __syncthreads();
    if (qn < nq) {
      if (tid == 0) issue(qn);
      ++qn;
    }
    ++qc;
  };

  C *ph = reinterpret_cast<C *>(a.psi_hat);
  C *gout = reinterpret_cast<C *>(a.out[0]);
  for (int t = blockIdx.x; t < ntm && alive; t += G) {
    const int ti = t % sg.tiles_inner, to = paired_outer(t / sg.tiles_inner, nout);
    const int kx = ti * W + c;
    const long long base = sg.off + (long long)to * sg.s_outer + (long long)kx * sg.col_stride;
    const long long fs = sg.fft_stride;
    // this thread's rows j + T m of the column: pcol[m * rs] (the launcher
    // checks that N * fs fits a 32-bit offset)
    const int rs = T * (int)fs;
    C *pcol = ph + base + (long long)j * fs;
    C *ocol = gout + base + (long long)j * fs;
    C v[E];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const C *bx = take();
      if (!bx) {
        alive = false;
        break;
      }
#pragma unroll
      for (int u = 0; u < VB; ++u) v[b * VB + u] = bx[(j + T * u) * W + c];
      release();
    }
    if (!alive) break;
    fft_line_e<C, N, -1, N, E>(v, xb, Cfg::LD, c, j, tw);
    C w[CHI ? E : 1];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      // this box's operators first: their L2 round trip overlaps the wait
      // (the filter values, needed last, are loaded after it)
      C ops[VB];
#pragma unroll
      for (int u = 0; u < VB; ++u) ops[u] = __ldg(reinterpret_cast<const C *>(a.fold_ops) + fold_at(a, kx, to, j + T * (b * VB + u)));
      const C *bx = take();
      if (!bx) {
        alive = false;
        break;
      }
#pragma unroll
      for (int u = 0; u < VB; ++u) {
        const int m = b * VB + u;
        const C p = bx[(j + T * u) * W + c];
        const C np = mk<C>(ops[u].x * p.x + ops[u].y * v[m].x, ops[u].x * p.y + ops[u].y * v[m].y);
        pcol[m * rs] = np;
        if constexpr (CHI) w[m] = cscale(np, __ldg(a.fold_chi + fold_at(a, kx, to, j + T * m)));
        v[m] = np;
      }
      release();
    }
    if (!alive) break;
    if constexpr (MODEL == MK_FILTERED) {
      fft_line_e<C, N, +1, N, E>(w, xb, Cfg::LD, c, j, tw);
#pragma unroll
      for (int m = 0; m < E; ++m) ocol[m * rs] = w[m];
    } else {
      fft_line_e<C, N, +1, N, E>(v, xb, Cfg::LD, c, j, tw);
#pragma unroll
      for (int m = 0; m < E; ++m) ocol[m * rs] = v[m];
      if constexpr (MODEL == MK_TUNGSTEN) {
        C *gout2 = reinterpret_cast<C *>(a.out[1]);
        fft_line_e<C, N, +1, N, E>(w, xb, Cfg::LD, c, j, tw);
#pragma unroll
        for (int m = 0; m < E; ++m) gout2[base + (long long)j * fs + m * rs] = w[m];
      }
    }
  }
  if (!alive) {
    if (tid == 0) atomicOr(flag, 2u);
    // drain this CTA's boxes still in flight (at most two; bounded)
    for (int k = qc; k < qn; ++k) mbar_wait(&bars[k & 1], (unsigned)(k >> 1) & 1u);
  }
}

}  // namespace opfc
