// zy_fused.cuh -- the z update and the next step's inverse y transform in one
// persistent kernel, chained through L2 per kx slab.
//
// The step's last two HBM sweeps of A are the z update's write of
// F_z^-1[psi_hat'] and the next step's inverse y pass reading it back.  Both
// work on the same kx slab at a time -- the z update's tiles are W columns x
// N2 rows at fixed ky, the y pass's tiles W columns x N1 rows at fixed kz, for
// the same W kx columns -- so a slab (W x N1 x N2 complex, 16.8 MB at 512^3
// FP32) written by the z-update tiles can be transformed along y while it is
// still in the 126 MB L2, and only the y pass's output goes back to HBM.
//
// Work items, handed out in order through an atomic counter, are
//   B(s, t): z-update tile t of slab s (t walks ky in (ky, N1 - ky) pairs),
//   C(s, t): inverse-y tile t (= kz) of slab s,
// queued as B(0) | B(1) C(0) | B(2) C(1) | ... with the kx = M (Nyquist) plane as
// slab S, so a C item's slab was handed out a whole slab earlier.  C(s, *)
// needs every B(s, *) done: a per-slab counter, incremented (release) after a B
// item's stores, is acquired before a C item's tiles are loaded.  The producer
// thread issues a C item only when the counter is full; while its own ring
// still holds items it defers the C item instead of waiting, so a wait never
// depends on this CTA's own unfinished work, and the grid is sized to the
// resident CTAs, so every item it waits for is held by a running CTA.  Every
// wait is bounded (4 s); on expiry the CTA records the timeout bit, drains its
// own loads and leaves.
//
// PLAIN and FILTERED models, N1 == N2 == N (one twiddle table serves both
// transforms), operators from the folded FP64-built tables.
#pragma once

namespace opfc {

struct ZyArgs {
  int *ctr;           // [0] next work item, [1 + s] z-update tiles done of slab s (s = S: Nyquist)
  ColSeg ymain, ynyq;  // inverse-y segments (main columns, kx = M plane)
  int S;              // main slabs (M / W)
  int BQ, CQ;         // Nyquist-plane tiles of the z update and of the y inverse
};

__device__ __forceinline__ int ld_acquire_gpu(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// generic-proxy global writes <-> async-proxy (TMA) global reads
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <int N> struct ZyItem {
  int phase;  // 0 = z update (B), 1 = inverse y (C)
  int slab;   // kx slab; S = the Nyquist plane
  int tile;
};

// Item i of the queue B(0) | B(1) C(0) | ... | B(S) C(S-1) | C(S) with N tiles per
// main slab and phase, BQ / CQ tiles for the Nyquist plane.
template <int N> __device__ __forceinline__ ZyItem<N> zy_decode(long long i, int S, int BQ, int CQ) {
  const long long G1 = 2LL * N;
  const long long offS = N + (long long)(S - 1) * G1;
  const long long offS1 = offS + BQ + N;
  ZyItem<N> it;
  if (i < N) {
    it = {0, 0, (int)i};
  } else if (i < offS) {
    const long long j = i - N;
    const int g = 1 + (int)(j / G1);
    const int r = (int)(j % G1);
    it = r < N ? ZyItem<N>{0, g, r} : ZyItem<N>{1, g - 1, r - N};
  } else if (i < offS1) {
    const int r = (int)(i - offS);
    it = r < BQ ? ZyItem<N>{0, S, r} : ZyItem<N>{1, S - 1, r - BQ};
  } else {
    it = {1, S, (int)(i - offS1)};
  }
  return it;
}
template <int N> __device__ __forceinline__ long long zy_total(int S, int BQ, int CQ) {
  return N + (long long)(S - 1) * 2 * N + BQ + N + CQ;
}

// Tensor maps: mz = A with z boxes, mpsi = psi_hat with z boxes, mfold = folded
// (opL, opN) pairs, mchi = folded filter (FILTERED), my = A with y boxes.
template <typename Real, int N, int W, int MODEL>
__global__ void __launch_bounds__(W *(N / Plan<N>::E), 1)
    zy_kernel(const __grid_constant__ CUtensorMap mz, const __grid_constant__ CUtensorMap mpsi,
              const __grid_constant__ CUtensorMap mfold, const __grid_constant__ CUtensorMap mchi,
              const __grid_constant__ CUtensorMap my, const ColArgs<Real> a, const ZyArgs z, unsigned *flag) {
  using Cfg = TmaCfg<Real, N, W, COL_UPDATE, MODEL, 3, 2, false>;
  using C = typename Cx<Real>::T;
  constexpr int E = Plan<N>::E;
  constexpr int T = N / E;
  constexpr int NT = W * T;
  constexpr int STAGES = Cfg::STAGES;
  constexpr bool CHI = Cfg::CHI;
  extern __shared__ __align__(128) unsigned char smraw[];
  C *tw = reinterpret_cast<C *>(smraw);
  unsigned char *stage0 = smraw + Cfg::TW;
  uint64_t *bars = reinterpret_cast<uint64_t *>(stage0 + STAGES * Cfg::STAGE);
  // control block, written by thread 0 only, read by all after a barrier
  int *item_of = reinterpret_cast<int *>(bars + STAGES);  // work item held by each stage
  int *ctl = item_of + STAGES;  // [0] next stage to fill [1] stages in flight [2] pending item [3] abort
  long long *pend = reinterpret_cast<long long *>(ctl + 4);

  const int tid = threadIdx.x;
  const int c = tid % W;
  const int j = tid / W;
  const C *gtw = reinterpret_cast<const C *>(a.tw);
  for (int i = tid; i < N; i += NT) tw[i] = gtw[i];
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
    ctl[0] = 0;
    ctl[1] = 0;
    ctl[3] = 0;
    *pend = -1;
  }
  __syncthreads();
  constexpr bool TWR = TwReg<C, N>::CNT > 0 && TwReg<C, N>::CNT <= 16;
  TwReg<C, N> twr;
  if constexpr (TWR) twr.load(j, tw);

  const int S = z.S, BQ = z.BQ, CQ = z.CQ;
  const long long total = zy_total<N>(S, BQ, CQ);
  const int n1 = a.rad_n1;

  auto issue = [&](int s, const ZyItem<N> &it) {
    unsigned char *st = stage0 + s * Cfg::STAGE;
    if (it.slab == S) {  // Nyquist plane: direct loads, nothing to wait for
      mbar_arrive(&bars[s]);
      return;
    }
    const int ti = it.slab;
    if (it.phase == 0) {
      const int ky = paired_outer(it.tile, n1);
      mbar_expect_tx(&bars[s], (unsigned)Cfg::STAGE);
#pragma unroll
      for (int b = 0; b < Cfg::NB; ++b) {
        const size_t offc = size_t(b) * Cfg::RB * W * sizeof(C);
        tma_load_3d(st + offc, &mz, &bars[s], ti * W * 2, ky, b * Cfg::RB);
        tma_load_3d(st + Cfg::TILE_C + offc, &mpsi, &bars[s], ti * W * 2, ky, b * Cfg::RB);
      }
      const int fy = fold_index(ky, n1);
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        tma_load_3d(st + 2 * Cfg::TILE_C + size_t(b) * Cfg::RBF * W * sizeof(C), &mfold, &bars[s], ti * W * 2, fy,
                    b * Cfg::RBF);
        if constexpr (CHI)
          tma_load_3d(st + 2 * Cfg::TILE_C + Cfg::FOLD_C + size_t(b) * Cfg::RBF * W * sizeof(Real), &mchi, &bars[s],
                      ti * W, fy, b * Cfg::RBF);
      }
    } else {
      mbar_expect_tx(&bars[s], (unsigned)Cfg::TILE_C);
#pragma unroll
      for (int b = 0; b < Cfg::NB; ++b)
        tma_load_3d(st + size_t(b) * Cfg::RB * W * sizeof(C), &my, &bars[s], ti * W * 2, b * Cfg::RB, it.tile);
    }
  };

  // thread 0: fill the free stages in queue order; a C item waits for its
  // slab's z-update tiles only when no item of this CTA is in flight
  auto fill = [&]() {
    while (ctl[1] < STAGES && !ctl[3]) {
      if (*pend < 0) {
        const long long i = atomicAdd(z.ctr, 1);
        *pend = i < total ? i : total;
      }
      if (*pend >= total) break;
      const ZyItem<N> it = zy_decode<N>(*pend, S, BQ, CQ);
      if (it.phase == 1) {
        const int need = it.slab < S ? N : BQ;
        const int *done = z.ctr + 1 + it.slab;
        if (ld_acquire_gpu(done) < need) {
          if (ctl[1] > 0) break;
          const unsigned long long t0 = global_ns();
          unsigned k = 0;
          while (ld_acquire_gpu(done) < need) {
            if ((++k & 63u) == 0 && global_ns() - t0 > 4000000000ull) {
              ctl[3] = 1;
              break;
            }
          }
          if (ctl[3]) break;
        }
        fence_proxy_async_global();  // the slab's generic stores before this thread's TMA reads
      }
      const int s = ctl[0];
      item_of[s] = (int)*pend;
      issue(s, it);
      ctl[0] = (s + 1) % STAGES;
      ctl[1] += 1;
      *pend = -1;
    }
  };

  C *ph = reinterpret_cast<C *>(a.psi_hat);
  C *gA = reinterpret_cast<C *>(a.out[0]);
  const C *gAin = reinterpret_cast<const C *>(a.in[0]);
  int head = 0;
  unsigned uses[STAGES];
#pragma unroll
  for (int s = 0; s < STAGES; ++s) uses[s] = 0;
  bool alive = true;
  while (true) {
    if (tid == 0) fill();
    __syncthreads();
    if (ctl[3]) {
      alive = false;
      break;
    }
    if (ctl[1] == 0) break;  // queue exhausted and nothing in flight
    const int s = head;
    const bool ok = mbar_wait(&bars[s], uses[s] & 1u);
    if (!__syncthreads_and(ok)) {
      alive = false;
      break;
    }
    const ZyItem<N> it = zy_decode<N>(item_of[s], S, BQ, CQ);
    unsigned char *st = stage0 + s * Cfg::STAGE;
    C *tin = reinterpret_cast<C *>(st);
    if (it.phase == 0 && it.slab < S) {
      // ---- z update of tile (slab, ky): the fused update of col_tma_kernel ----
      const ColSeg &sg = a.seg0;
      const int ky = paired_outer(it.tile, n1);
      const long long base = sg.off + (long long)ky * sg.s_outer + (long long)(it.slab * W + c) * sg.col_stride;
      const long long fs = sg.fft_stride;
      C v[E];
#pragma unroll
      for (int m = 0; m < E; ++m) v[m] = tin[(j + T * m) * W + c];
      __syncthreads();
      upd_fft<C, N, -1, TWR>(v, tin, W, c, j, tw, twr);
      const C *tpsi = reinterpret_cast<const C *>(st + Cfg::TILE_C);
      const C *tfold = reinterpret_cast<const C *>(st + 2 * Cfg::TILE_C);
      const Real *tchi = reinterpret_cast<const Real *>(st + 2 * Cfg::TILE_C + Cfg::FOLD_C);
      C w[CHI ? E : 1];
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int p = j + T * m;
        const C q = tpsi[p * W + c];
        const int fz = fold_index(p, N);
        const C o = tfold[fz * W + c];
        const C np = mk<C>(o.x * q.x + o.y * v[m].x, o.x * q.y + o.y * v[m].y);
        ph[base + (long long)p * fs] = np;
        if constexpr (CHI) w[m] = cscale(np, tchi[fz * W + c]);
        v[m] = np;
      }
      if constexpr (CHI) {
        upd_fft<C, N, +1, TWR>(w, tin, W, c, j, tw, twr);
#pragma unroll
        for (int m = 0; m < E; ++m) gA[base + (long long)(j + T * m) * fs] = w[m];
      } else {
        upd_fft<C, N, +1, TWR>(v, tin, W, c, j, tw, twr);
#pragma unroll
        for (int m = 0; m < E; ++m) gA[base + (long long)(j + T * m) * fs] = v[m];
      }
      fence_proxy_async_global();
    } else if (it.phase == 0) {
      // ---- z update of Nyquist-plane lines (kx = M, columns = ky) ----
      const ColSeg &sn = a.seg1;
      C *sm = tin;
      const int cg = it.tile * W + c;
      const bool okc = cg < sn.ncols;
      const long long base = sn.off + (long long)cg * sn.col_stride;
      const long long fs = sn.fft_stride;
      C v[E];
#pragma unroll
      for (int m = 0; m < E; ++m) v[m] = okc ? gAin[base + (long long)(j + T * m) * fs] : mk<C>(0, 0);
      upd_fft<C, N, -1, TWR>(v, sm, W, c, j, tw, twr);
      C w[CHI ? E : 1];
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const long long idx = base + (long long)(j + T * m) * fs;
        C np = mk<C>(0, 0);
        Real ch = Real(1);
        if (okc) {
          const C q = ph[idx];
          Real la, lb;
          folded_ops<Real, MODEL>(a, a.rad_M, cg, j + T * m, la, lb, ch);
          np = mk<C>(la * q.x + lb * v[m].x, la * q.y + lb * v[m].y);
          ph[idx] = np;
        }
        if constexpr (CHI) w[m] = okc ? cscale(np, ch) : mk<C>(0, 0);
        v[m] = np;
      }
      if constexpr (CHI) {
        upd_fft<C, N, +1, TWR>(w, sm, W, c, j, tw, twr);
        if (okc) {
#pragma unroll
          for (int m = 0; m < E; ++m) gA[base + (long long)(j + T * m) * fs] = w[m];
        }
      } else {
        upd_fft<C, N, +1, TWR>(v, sm, W, c, j, tw, twr);
        if (okc) {
#pragma unroll
          for (int m = 0; m < E; ++m) gA[base + (long long)(j + T * m) * fs] = v[m];
        }
      }
      fence_proxy_async_global();
    } else if (it.slab < S) {
      // ---- inverse y transform of tile (slab, kz) ----
      const ColSeg &sg = z.ymain;
      const long long base =
          sg.off + (long long)it.tile * sg.s_outer + (long long)(it.slab * W + c) * sg.col_stride;
      const long long fs = sg.fft_stride;
      C v[E];
#pragma unroll
      for (int m = 0; m < E; ++m) v[m] = tin[(j + T * m) * W + c];
      __syncthreads();
      upd_fft<C, N, +1, TWR>(v, tin, W, c, j, tw, twr);
#pragma unroll
      for (int m = 0; m < E; ++m) gA[base + (long long)(j + T * m) * fs] = v[m];
    } else {
      // ---- inverse y transform of Nyquist-plane lines (columns = kz) ----
      const ColSeg &sn = z.ynyq;
      C *sm = tin;
      const int cg = it.tile * W + c;
      const bool okc = cg < sn.ncols;
      const long long base = sn.off + (long long)cg * sn.col_stride;
      const long long fs = sn.fft_stride;
      C v[E];
#pragma unroll
      for (int m = 0; m < E; ++m) v[m] = okc ? gAin[base + (long long)(j + T * m) * fs] : mk<C>(0, 0);
      upd_fft<C, N, +1, TWR>(v, sm, W, c, j, tw, twr);
      if (okc) {
#pragma unroll
        for (int m = 0; m < E; ++m) gA[base + (long long)(j + T * m) * fs] = v[m];
      }
    }
    // the stage was read and used as exchange space by the generic proxy:
    // order that before its next asynchronous fill; then publish a finished
    // z-update tile to the CTAs that wait for its slab
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      if (it.phase == 0) {
        __threadfence();
        atomicAdd(z.ctr + 1 + it.slab, 1);
      }
      ctl[1] -= 1;
    }
    uses[s] += 1;
    head = (head + 1) % STAGES;
  }
  if (!alive) {
    if (tid == 0) atomicOr(flag, 2u);
    // drain this CTA's own loads still in flight (bounded), then leave
    const int inflight = ctl[1];
    for (int k = 0; k < inflight; ++k) {
      const int s = (head + k) % STAGES;
      mbar_wait(&bars[s], uses[s] & 1u);
    }
  }
}

}  // namespace opfc
