// fft_core.cuh -- register-resident Stockham FFT building blocks for sm_100a.
//
// A line of length N is owned by T = N/E threads of one CTA; each thread keeps
// E complex values in registers.  On entry to a transform thread j holds the
// line positions p = j + T*m (m = 0..E-1) and on exit it holds the transformed
// values at the same positions (Stockham autosort: the first stage reads and the
// last stage writes the "stride N/R" pattern, so nothing is permuted).  Between
// stages the line is exchanged through shared memory laid out [p][c] with a
// row pitch `ld` (W lines interleaved, c fastest) -- conflict-free for the
// c-fastest thread mapping used by every kernel.
//
// Twiddles come from a per-CTA shared-memory table tw[i] = exp(-2 pi i i / TWS)
// built on the host in FP64 and rounded to the compute precision; the inverse
// direction uses the conjugate.  TWS is a multiple of N (TWS = 2N for the
// half-length complex FFT inside a real transform of length 2N).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace opfc {

template <typename R> struct Cx;
template <> struct Cx<float> { using T = float2; };
template <> struct Cx<double> { using T = double2; };

template <typename C> __device__ __forceinline__ C mk(decltype(C::x) a, decltype(C::x) b) {
  C r;
  r.x = a;
  r.y = b;
  return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return mk<C>(a.x * s, a.y * s); }

// pf2: FP32 complex whose add / subtract / real scale issue as one packed
// FP32x2 instruction (sm_100) instead of two scalar ones.  Each lane is rounded
// exactly as the scalar operation (a - b is fma(b, -1, a): one rounding of the
// exact difference), so results are bit-identical to float2 arithmetic.  Kernels
// opt in through CxP (the x passes, where it measured faster; the column passes
// stay on float2, where it did not).
struct __align__(8) pf2 {
  float x, y;
};
template <typename R> struct CxP { using T = typename Cx<R>::T; };
template <> struct CxP<float> { using T = pf2; };

__device__ __forceinline__ float2 f2(pf2 a) { return make_float2(a.x, a.y); }
__device__ __forceinline__ pf2 p2(float2 a) { return pf2{a.x, a.y}; }
template <> __device__ __forceinline__ pf2 cadd<pf2>(pf2 a, pf2 b) { return p2(__fadd2_rn(f2(a), f2(b))); }
template <> __device__ __forceinline__ pf2 csub<pf2>(pf2 a, pf2 b) {
  return p2(__ffma2_rn(f2(b), make_float2(-1.f, -1.f), f2(a)));
}
template <> __device__ __forceinline__ pf2 cscale<pf2>(pf2 a, float s) {
  return p2(__fmul2_rn(f2(a), make_float2(s, s)));
}

// a * w (DIR < 0) or a * conj(w) (DIR > 0)
template <int DIR, typename C> __device__ __forceinline__ C twmul(C a, C w) {
  if (DIR < 0) return mk<C>(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
  return mk<C>(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y);
}
// a * exp(DIR * i pi / 2): -i for the forward direction, +i for the inverse
template <int DIR, typename C> __device__ __forceinline__ C rot90(C a) {
  return DIR < 0 ? mk<C>(a.y, -a.x) : mk<C>(-a.y, a.x);
}

// ---------------------------------------------------------------------------
// radix-R DFT kernels on registers, sign DIR (-1 forward, +1 inverse)
// ---------------------------------------------------------------------------
template <int R, int DIR, typename C> struct Dft;

template <int DIR, typename C> struct Dft<1, DIR, C> {
  static __device__ __forceinline__ void run(C (&)[1]) {}
};

template <int DIR, typename C> struct Dft<2, DIR, C> {
  static __device__ __forceinline__ void run(C (&v)[2]) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <int DIR, typename C> struct Dft<4, DIR, C> {
  static __device__ __forceinline__ void run4(C &v0, C &v1, C &v2, C &v3) {
    C a = cadd(v0, v2), b = csub(v0, v2);
    C c = cadd(v1, v3), d = rot90<DIR>(csub(v1, v3));
    v0 = cadd(a, c);
    v2 = csub(a, c);
    v1 = cadd(b, d);
    v3 = csub(b, d);
  }
  static __device__ __forceinline__ void run(C (&v)[4]) { run4(v[0], v[1], v[2], v[3]); }
};

template <int DIR, typename C> struct Dft<8, DIR, C> {
  static __device__ __forceinline__ void run(C (&v)[8]) {
    using S = decltype(C::x);
    const S h = S(0.70710678118654752440084436210484904);
    Dft<4, DIR, C>::run4(v[0], v[2], v[4], v[6]);
    Dft<4, DIR, C>::run4(v[1], v[3], v[5], v[7]);
    // twiddle the odd half by w8^k, w8 = exp(DIR * 2 pi i / 8)
    C o1 = v[3], o2 = v[5], o3 = v[7];
    if (DIR < 0) {
      o1 = mk<C>(h * (o1.x + o1.y), h * (o1.y - o1.x));
      o3 = mk<C>(h * (o3.y - o3.x), -h * (o3.x + o3.y));
    } else {
      o1 = mk<C>(h * (o1.x - o1.y), h * (o1.x + o1.y));
      o3 = mk<C>(-h * (o3.x + o3.y), h * (o3.x - o3.y));
    }
    o2 = rot90<DIR>(o2);
    C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1];
    v[0] = cadd(e0, o0);
    v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1);
    v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2);
    v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3);
    v[7] = csub(e3, o3);
  }
};

// 16 = 4 x 4: n = 4 n1 + n2, k = k1 + 4 k2 (DFT4 over n1, twiddle W16^{n2 k1},
// DFT4 over n2, then a 4 x 4 transpose of the register order).
template <int DIR, typename C> struct Dft<16, DIR, C> {
  static __device__ __forceinline__ C w(C a, decltype(C::x) c, decltype(C::x) s) {
    // a * (c + DIR i s)
    return DIR < 0 ? mk<C>(a.x * c + a.y * s, a.y * c - a.x * s) : mk<C>(a.x * c - a.y * s, a.y * c + a.x * s);
  }
  static __device__ __forceinline__ void run(C (&v)[16]) {
    using S = decltype(C::x);
    const S c1 = S(0.92387953251128675612818318939678829);  // cos(pi/8)
    const S s1 = S(0.38268343236508977172845998403039887);  // sin(pi/8)
    const S h = S(0.70710678118654752440084436210484904);
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) Dft<4, DIR, C>::run4(v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]);
    v[5] = w(v[5], c1, s1);    // W16^1
    v[9] = w(v[9], h, h);      // W16^2
    v[13] = w(v[13], s1, c1);  // W16^3
    v[6] = w(v[6], h, h);      // W16^2
    v[10] = rot90<DIR>(v[10]);  // W16^4
    v[14] = w(v[14], -h, h);   // W16^6
    v[7] = w(v[7], s1, c1);    // W16^3
    v[11] = w(v[11], -h, h);   // W16^6
    v[15] = w(v[15], -c1, -s1);  // W16^9
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) Dft<4, DIR, C>::run4(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    C t[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) t[i] = v[i];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[4 * k1 + k2];
  }
};

// 32 = 2 x 16 (decimation in time): E, O = DFT16 of the even / odd samples,
// X[k] = E[k] + W32^k O[k], X[k + 16] = E[k] - W32^k O[k], W32 = exp(DIR 2 pi i / 32).
template <int DIR, typename C> struct Dft<32, DIR, C> {
  static __device__ __forceinline__ void run(C (&v)[32]) {
    using S = decltype(C::x);
    // cos(pi k / 16) and sin(pi k / 16), k = 0..15
    constexpr double cs[16] = {1.0,
                               0.980785280403230449126182236134239037,
                               0.923879532511286756128183189396788287,
                               0.831469612302545237078788377617905757,
                               0.707106781186547524400844362104849039,
                               0.555570233019602224742830813948532874,
                               0.382683432365089771728459984030398867,
                               0.195090322016128267848284868477022241,
                               0.0,
                               -0.195090322016128267848284868477022241,
                               -0.382683432365089771728459984030398867,
                               -0.555570233019602224742830813948532874,
                               -0.707106781186547524400844362104849039,
                               -0.831469612302545237078788377617905757,
                               -0.923879532511286756128183189396788287,
                               -0.980785280403230449126182236134239037};
    constexpr double sn[16] = {0.0,
                               0.195090322016128267848284868477022241,
                               0.382683432365089771728459984030398867,
                               0.555570233019602224742830813948532874,
                               0.707106781186547524400844362104849039,
                               0.831469612302545237078788377617905757,
                               0.923879532511286756128183189396788287,
                               0.980785280403230449126182236134239037,
                               1.0,
                               0.980785280403230449126182236134239037,
                               0.923879532511286756128183189396788287,
                               0.831469612302545237078788377617905757,
                               0.707106781186547524400844362104849039,
                               0.555570233019602224742830813948532874,
                               0.382683432365089771728459984030398867,
                               0.195090322016128267848284868477022241};
    C e[16], o[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      e[i] = v[2 * i];
      o[i] = v[2 * i + 1];
    }
    Dft<16, DIR, C>::run(e);
    Dft<16, DIR, C>::run(o);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const C t = k == 0 ? o[0] : Dft<16, DIR, C>::w(o[k], S(cs[k]), S(sn[k]));
      v[k] = cadd(e[k], t);
      v[k + 16] = csub(e[k], t);
    }
  }
};

template <int DIR, typename C> struct Dft<3, DIR, C> {
  static __device__ __forceinline__ void run(C (&v)[3]) {
    using S = decltype(C::x);
    const S s3 = S(0.86602540378443864676372317075293618);
    C a = v[0], b = v[1], c = v[2];
    C t = cadd(b, c);
    C m = mk<C>(a.x - S(0.5) * t.x, a.y - S(0.5) * t.y);
    C d = csub(b, c);
    // forward: X1 = m - i s3 d, X2 = m + i s3 d ; inverse flips the sign
    C id = mk<C>(-s3 * d.y, s3 * d.x);  // i * s3 * d
    v[0] = cadd(a, t);
    if (DIR < 0) {
      v[1] = csub(m, id);
      v[2] = cadd(m, id);
    } else {
      v[1] = cadd(m, id);
      v[2] = csub(m, id);
    }
  }
};

template <int DIR, typename C> struct Dft<5, DIR, C> {
  static __device__ __forceinline__ void run(C (&v)[5]) {
    using S = decltype(C::x);
    const S c1 = S(0.30901699437494742410229341718281906);
    const S c2 = S(-0.80901699437494742410229341718281906);
    const S s1 = S(0.95105651629515357211643933337938214);
    const S s2 = S(0.58778525229247312916870595463907277);
    C a = v[0];
    C be = cadd(v[1], v[4]), bm = csub(v[1], v[4]);
    C cd = cadd(v[2], v[3]), cm = csub(v[2], v[3]);
    C r1 = mk<C>(a.x + c1 * be.x + c2 * cd.x, a.y + c1 * be.y + c2 * cd.y);
    C r2 = mk<C>(a.x + c2 * be.x + c1 * cd.x, a.y + c2 * be.y + c1 * cd.y);
    // q1 = s1 bm + s2 cm ; q2 = s2 bm - s1 cm ; X1 = r1 - i q1 (forward)
    C q1 = mk<C>(s1 * bm.x + s2 * cm.x, s1 * bm.y + s2 * cm.y);
    C q2 = mk<C>(s2 * bm.x - s1 * cm.x, s2 * bm.y - s1 * cm.y);
    C iq1 = mk<C>(-q1.y, q1.x), iq2 = mk<C>(-q2.y, q2.x);
    v[0] = mk<C>(a.x + be.x + cd.x, a.y + be.y + cd.y);
    if (DIR < 0) {
      v[1] = csub(r1, iq1);
      v[2] = csub(r2, iq2);
      v[3] = cadd(r2, iq2);
      v[4] = cadd(r1, iq1);
    } else {
      v[1] = cadd(r1, iq1);
      v[2] = cadd(r2, iq2);
      v[3] = csub(r2, iq2);
      v[4] = csub(r1, iq1);
    }
  }
};

// ---------------------------------------------------------------------------
// plans: elements per thread E and the radix sequence for each line length
// ---------------------------------------------------------------------------
template <int... Rs> struct Radices {};

template <int N> struct Plan;
template <> struct Plan<1> { static constexpr int E = 1; using R = Radices<>; };
template <> struct Plan<2> { static constexpr int E = 2; using R = Radices<2>; };
template <> struct Plan<4> { static constexpr int E = 4; using R = Radices<4>; };
template <> struct Plan<8> { static constexpr int E = 8; using R = Radices<8>; };
template <> struct Plan<16> { static constexpr int E = 8; using R = Radices<2, 8>; };
template <> struct Plan<32> { static constexpr int E = 8; using R = Radices<4, 8>; };
template <> struct Plan<64> { static constexpr int E = 8; using R = Radices<8, 8>; };
template <> struct Plan<128> { static constexpr int E = 8; using R = Radices<2, 8, 8>; };
template <> struct Plan<256> { static constexpr int E = 8; using R = Radices<4, 8, 8>; };
template <> struct Plan<512> { static constexpr int E = 8; using R = Radices<8, 8, 8>; };
template <> struct Plan<1024> { static constexpr int E = 16; using R = Radices<16, 8, 8>; };
// non power-of-two lengths used by uneven ensembles (x half lengths 24, 40, 48)
template <> struct Plan<24> { static constexpr int E = 24; using R = Radices<3, 8>; };
template <> struct Plan<40> { static constexpr int E = 20; using R = Radices<5, 2, 4>; };
template <> struct Plan<48> { static constexpr int E = 12; using R = Radices<3, 4, 4>; };
template <> struct Plan<80> { static constexpr int E = 20; using R = Radices<5, 4, 4>; };
template <> struct Plan<96> { static constexpr int E = 24; using R = Radices<3, 4, 8>; };

// One Stockham stage (radix R, input sub-length Ns) and the stages after it.
template <typename C, int N, int E, int DIR, int TWS, int Ns, int R, int... Rest>
__device__ __forceinline__ void stages(C (&v)[E], C *sm, int ld, int c, int j, const C *tw) {
  constexpr int T = N / E;
  constexpr int B = E / R;
  constexpr bool last = sizeof...(Rest) == 0;
  static_assert(E % R == 0, "plan: radix must divide E");
#pragma unroll
  for (int t = 0; t < B; ++t) {
    C x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = v[t + r * B];
    const int b = j + t * T;
    const int k = (Ns > 1) ? (b % Ns) : 0;
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) x[r] = twmul<DIR>(x[r], tw[k * r * (TWS / (Ns * R))]);
    }
    Dft<R, DIR, C>::run(x);
    if (last) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[t + r * B] = x[r];
    } else {
      const int base = (b / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) sm[(base + r * Ns) * ld + c] = x[r];
    }
  }
  if constexpr (!last) {
    __syncthreads();
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = sm[(j + T * m) * ld + c];
    __syncthreads();
    stages<C, N, E, DIR, TWS, Ns * R, Rest...>(v, sm, ld, c, j, tw);
  }
}

// Plans with a prescribed number of elements per thread E (T = N/E threads per
// line); the uneven-ensemble kernels use T = 4 for every size so that one CTA
// shape serves all of them.  Each radix divides E.
template <int N, int E> struct PlanE { using R = typename Plan<N>::R; };
template <> struct PlanE<16, 4> { using R = Radices<4, 4>; };
template <> struct PlanE<24, 6> { using R = Radices<2, 2, 2, 3>; };
template <> struct PlanE<40, 10> { using R = Radices<2, 2, 2, 5>; };
template <> struct PlanE<64, 16> { using R = Radices<8, 8>; };
// one shared-memory exchange per transform (32 values per thread)
template <> struct PlanE<512, 32> { using R = Radices<16, 32>; };
template <> struct PlanE<1024, 32> { using R = Radices<32, 32>; };

template <typename C, int N, int E, int DIR, int TWS, int... Rs>
__device__ __forceinline__ void fft_run(Radices<Rs...>, C (&v)[E], C *sm, int ld, int c, int j,
                                        const C *tw) {
  if constexpr (sizeof...(Rs) > 0) stages<C, N, E, DIR, TWS, 1, Rs...>(v, sm, ld, c, j, tw);
}

// Transform one line of length N held as v[m] at positions j + (N/E)*m.
template <typename C, int N, int DIR, int TWS>
__device__ __forceinline__ void fft_line(C (&v)[Plan<N>::E], C *sm, int ld, int c, int j,
                                         const C *tw) {
  fft_run<C, N, Plan<N>::E, DIR, TWS>(typename Plan<N>::R{}, v, sm, ld, c, j, tw);
}

// Same with E taken from the register array (plan PlanE<N, E>).
template <typename C, int N, int DIR, int TWS, int E>
__device__ __forceinline__ void fft_line_e(C (&v)[E], C *sm, int ld, int c, int j, const C *tw) {
  fft_run<C, N, E, DIR, TWS>(typename PlanE<N, E>::R{}, v, sm, ld, c, j, tw);
}

// ---------------------------------------------------------------------------
// Register-resident twiddles.  A thread's stage twiddles depend only on its
// line position j, so a persistent kernel can load them once (TwReg::load) and
// run every later transform of the same length from registers (fft_line_rt),
// both directions (the inverse uses the conjugates).  Count per thread:
// sum over stages with Ns > 1 of (E/R)(R-1).
// ---------------------------------------------------------------------------
template <int E, int... Rs> constexpr int tw_count(Radices<Rs...>) {
  constexpr int rs[] = {1, Rs...};
  int ns = 1, cnt = 0;
  for (int i = 1; i <= (int)sizeof...(Rs); ++i) {
    if (ns > 1) cnt += (E / rs[i]) * (rs[i] - 1);
    ns *= rs[i];
  }
  return cnt;
}

template <typename C, int N, int E, int TWS, int Ns, int OFF, int CNT, int R, int... Rest>
__device__ __forceinline__ void tw_load(C (&w)[CNT], int j, const C *tw) {
  constexpr int T = N / E;
  constexpr int B = E / R;
  if constexpr (Ns > 1) {
#pragma unroll
    for (int t = 0; t < B; ++t) {
      const int k = (j + t * T) % Ns;
#pragma unroll
      for (int r = 1; r < R; ++r) w[OFF + t * (R - 1) + r - 1] = tw[k * r * (TWS / (Ns * R))];
    }
  }
  if constexpr (sizeof...(Rest) > 0)
    tw_load<C, N, E, TWS, Ns * R, OFF + (Ns > 1 ? B * (R - 1) : 0), CNT, Rest...>(w, j, tw);
}

// stages() with the twiddles taken from the register cache w
template <typename C, int N, int E, int DIR, int Ns, int OFF, int CNT, int R, int... Rest>
__device__ __forceinline__ void stages_rt(C (&v)[E], C *sm, int ld, int c, int j, const C (&w)[CNT]) {
  constexpr int T = N / E;
  constexpr int B = E / R;
  constexpr bool last = sizeof...(Rest) == 0;
#pragma unroll
  for (int t = 0; t < B; ++t) {
    C x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = v[t + r * B];
    const int b = j + t * T;
    const int k = (Ns > 1) ? (b % Ns) : 0;
    if constexpr (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) x[r] = twmul<DIR>(x[r], w[OFF + t * (R - 1) + r - 1]);
    }
    Dft<R, DIR, C>::run(x);
    if constexpr (last) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[t + r * B] = x[r];
    } else {
      const int base = (b / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) sm[(base + r * Ns) * ld + c] = x[r];
    }
  }
  if constexpr (!last) {
    __syncthreads();
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = sm[(j + T * m) * ld + c];
    __syncthreads();
    stages_rt<C, N, E, DIR, Ns * R, OFF + (Ns > 1 ? B * (R - 1) : 0), CNT, Rest...>(v, sm, ld, c, j, w);
  }
}

// ---------------------------------------------------------------------------
// Ping-pong exchange: exchange e writes buffer (e even ? b1 : b0) and reads it
// back, so one CTA barrier per exchange suffices (a buffer is rewritten only
// two exchanges later, after a barrier every thread has passed since its last
// read of it).  b0 may be the landed input tile: exchange 0 never writes it.
// Twiddles from the shared table (TWR = false) or a TwReg cache (TWR = true).
// ---------------------------------------------------------------------------
template <typename C, int N, int E, int DIR, int TWS, bool TWR, int EX, int Ns, int OFF, int CNT, int R,
          int... Rest>
__device__ __forceinline__ void stages_pp(C (&v)[E], C *b0, C *b1, int ld, int c, int j, const C *tw,
                                          const C (&w)[CNT]) {
  constexpr int T = N / E;
  constexpr int B = E / R;
  constexpr bool last = sizeof...(Rest) == 0;
  C *sm = (EX % 2 == 0) ? b1 : b0;
#pragma unroll
  for (int t = 0; t < B; ++t) {
    C x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = v[t + r * B];
    const int b = j + t * T;
    const int k = (Ns > 1) ? (b % Ns) : 0;
    if constexpr (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        if constexpr (TWR)
          x[r] = twmul<DIR>(x[r], w[OFF + t * (R - 1) + r - 1]);
        else
          x[r] = twmul<DIR>(x[r], tw[k * r * (TWS / (Ns * R))]);
      }
    }
    Dft<R, DIR, C>::run(x);
    if constexpr (last) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[t + r * B] = x[r];
    } else {
      const int base = (b / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) sm[(base + r * Ns) * ld + c] = x[r];
    }
  }
  if constexpr (!last) {
    __syncthreads();
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = sm[(j + T * m) * ld + c];
    stages_pp<C, N, E, DIR, TWS, TWR, EX + 1, Ns * R, OFF + (Ns > 1 ? B * (R - 1) : 0), CNT, Rest...>(
        v, b0, b1, ld, c, j, tw, w);
  }
}

template <typename C, int N, int DIR, bool TWR, int EX0, int CNT, int... Rs>
__device__ __forceinline__ void fft_pp_run(Radices<Rs...>, C (&v)[Plan<N>::E], C *b0, C *b1, int ld, int c, int j,
                                           const C *tw, const C (&w)[CNT]) {
  if constexpr (sizeof...(Rs) > 0)
    stages_pp<C, N, Plan<N>::E, DIR, N, TWR, EX0, 1, 0, CNT, Rs...>(v, b0, b1, ld, c, j, tw, w);
}

// shared-memory exchanges of one length-N transform
template <int... Rs> constexpr int n_exchanges(Radices<Rs...>) { return sizeof...(Rs) > 0 ? int(sizeof...(Rs)) - 1 : 0; }
template <int N> constexpr int fft_exchanges() { return n_exchanges(typename Plan<N>::R{}); }

template <typename C, int N> struct TwReg {
  static constexpr int E = Plan<N>::E;
  static constexpr int CNT = tw_count<E>(typename Plan<N>::R{});
  C w[CNT > 0 ? CNT : 1];
  template <int... Rs> __device__ __forceinline__ void load_(Radices<Rs...>, int j, const C *tw) {
    if constexpr (CNT > 0 && sizeof...(Rs) > 0) tw_load<C, N, E, N, 1, 0, CNT, Rs...>(w, j, tw);
  }
  __device__ __forceinline__ void load(int j, const C *tw) { load_(typename Plan<N>::R{}, j, tw); }
};

template <typename C, int N, int DIR, int... Rs>
__device__ __forceinline__ void fft_rt_run(Radices<Rs...>, C (&v)[Plan<N>::E], C *sm, int ld, int c, int j,
                                           const TwReg<C, N> &w) {
  if constexpr (sizeof...(Rs) > 0)
    stages_rt<C, N, Plan<N>::E, DIR, 1, 0, (TwReg<C, N>::CNT > 0 ? TwReg<C, N>::CNT : 1), Rs...>(v, sm, ld, c, j,
                                                                                                 w.w);
}

// fft_line<C, N, DIR, N> with the twiddles from a TwReg cache
template <typename C, int N, int DIR>
__device__ __forceinline__ void fft_line_rt(C (&v)[Plan<N>::E], C *sm, int ld, int c, int j, const TwReg<C, N> &w) {
  fft_rt_run<C, N, DIR>(typename Plan<N>::R{}, v, sm, ld, c, j, w);
}

// fft_line<C, N, DIR, N> with ping-pong exchange buffers (b0, b1); TWR selects
// the twiddles of the TwReg cache w over the shared table tw.  Transforms run
// back to back without a barrier between them continue the exchange count:
// EX0 = exchanges made since the last CTA-wide barrier that ended a tile.
template <typename C, int N, int DIR, bool TWR, int EX0 = 0>
__device__ __forceinline__ void fft_line_pp(C (&v)[Plan<N>::E], C *b0, C *b1, int ld, int c, int j, const C *tw,
                                            const TwReg<C, N> &w) {
  constexpr int CNT = TwReg<C, N>::CNT > 0 ? TwReg<C, N>::CNT : 1;
  fft_pp_run<C, N, DIR, TWR, EX0, CNT>(typename Plan<N>::R{}, v, b0, b1, ld, c, j, tw, w.w);
}

}  // namespace opfc
