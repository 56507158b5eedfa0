// Line-FFT engine for sm_100a (FP64 and FP32 lines).
//
// One line of N complex points is owned by T = N/P threads of ONE warp (or of
// the whole CTA when T > 32); thread t keeps the P points at positions
// t + T*s (s = 0..P-1) in registers.  The transform is Stockham autosort
// (Govindaraju et al., "High performance discrete Fourier transforms on
// graphics processors", SC 2008): a sequence of radix-R stages, each thread
// doing P/R register butterflies per stage, with the data re-distributed
// between stages through a padded shared-memory line buffer.  Input and
// output both use the "position t + T*s" distribution, so the first stage
// reads straight from global memory and the last stage writes straight to it.
//
// Small DFTs (R = 2, 3, 4 and the composites 6, 8, 12, 16 built by a
// two-factor Cooley-Tukey split) run fully in registers with compile-time
// twiddles.  Stage twiddles come from a per-CTA shared-memory table
// tw[e] = (cos 2*pi*e/N, sin 2*pi*e/N), e in [0, N).
//
// DIR = +1 is the inverse (e^{+i}) transform, DIR = -1 the forward one; both
// unnormalised.  Lines are double2 (FP64) or float2 (FP32, the precision
// mode); the twiddle tables are FP64 in global memory and rounded on load.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>
#include <utility>

namespace ns3d {

// ---------------------------------------------------------------------------
// complex helpers, for double2 (FP64) and float2 (FP32) lines
// ---------------------------------------------------------------------------
template <typename C>
struct CTraits;
template <>
struct CTraits<double2> {
  using R = double;
  __host__ __device__ __forceinline__ static double2 make(double x, double y) {
    return make_double2(x, y);
  }
};
template <>
struct CTraits<float2> {
  using R = float;
  __host__ __device__ __forceinline__ static float2 make(float x, float y) {
    return make_float2(x, y);
  }
};
template <typename C>
using RealOf = typename CTraits<C>::R;
template <typename C>
__device__ __forceinline__ C mkc(RealOf<C> x, RealOf<C> y) {
  return CTraits<C>::make(x, y);
}
// a complex value of another precision (FP64 state <-> FP32 scratch)
template <typename C, typename D>
__device__ __forceinline__ C cvt(D a) {
  return mkc<C>((RealOf<C>)a.x, (RealOf<C>)a.y);
}

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { return mkc<C>(a.x + b.x, a.y + b.y); }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { return mkc<C>(a.x - b.x, a.y - b.y); }
template <typename C>
__device__ __forceinline__ C cscale(C a, RealOf<C> s) { return mkc<C>(a.x * s, a.y * s); }
template <typename C>
__device__ __forceinline__ C cconj(C a) { return mkc<C>(a.x, -a.y); }
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  return mkc<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * (DIR * i)
template <int DIR, typename C>
__device__ __forceinline__ C cmul_i(C a) {
  return DIR > 0 ? mkc<C>(-a.y, a.x) : mkc<C>(a.y, -a.x);
}

// ---------------------------------------------------------------------------
// compile-time twiddles: cos/sin of 2*pi*a/48 for the angles small DFTs use
// (multiples of 22.5 and 30 degrees)
// ---------------------------------------------------------------------------
constexpr double kC225 = 0.92387953251128675613;  // cos(pi/8)
constexpr double kS225 = 0.38268343236508977173;  // sin(pi/8)
constexpr double kR3H = 0.86602540378443864676;   // sqrt(3)/2
constexpr double kR12 = 0.70710678118654752440;   // sqrt(1/2)

__host__ __device__ constexpr double cos_quarter(int a) {  // a in [0, 12], unit 7.5 deg
  return a == 0 ? 1.0 : a == 3 ? kC225 : a == 4 ? kR3H : a == 6 ? kR12 : a == 8 ? 0.5
       : a == 9 ? kS225 : a == 12 ? 0.0 : -2.0;  // -2: angle not representable
}
__host__ __device__ constexpr double cos48(int a) {
  return (a = ((a % 48) + 48) % 48, a <= 12 ? cos_quarter(a)
          : a <= 24 ? -cos_quarter(24 - a) : a <= 36 ? -cos_quarter(a - 24) : cos_quarter(48 - a));
}
__host__ __device__ constexpr double sin48(int a) { return cos48(a - 12); }

// v * exp(DIR * 2*pi*i * E / R)
template <int R, int E, int DIR, typename C>
__device__ __forceinline__ C rot(C v) {
  using Rt = RealOf<C>;
  constexpr int a = ((E % R) * (48 / R)) % 48;
  static_assert(48 % R == 0, "radix must divide 48");
  static_assert(cos48(a) > -1.5 || a % 12 == 0, "angle not in table");
  if constexpr (a == 0) {
    return v;
  } else if constexpr (a == 24) {
    return mkc<C>(-v.x, -v.y);
  } else if constexpr (a == 12) {
    return cmul_i<DIR>(v);
  } else if constexpr (a == 36) {
    return cmul_i<-DIR>(v);
  } else {
    constexpr Rt c = (Rt)cos48(a);
    constexpr Rt s = (Rt)(DIR * sin48(a));
    return mkc<C>(v.x * c - v.y * s, v.x * s + v.y * c);
  }
}

// ---------------------------------------------------------------------------
// small DFTs in registers: V[k] = sum_r v[r] exp(DIR*2*pi*i*r*k/R)
// ---------------------------------------------------------------------------
template <int R, int DIR>
struct DFT;

template <int DIR>
struct DFT<1, DIR> {
  template <typename C>
  __device__ __forceinline__ static void run(C*) {}
};

template <int DIR>
struct DFT<2, DIR> {
  template <typename C>
  __device__ __forceinline__ static void run(C* v) {
    C a = cadd(v[0], v[1]);
    v[1] = csub(v[0], v[1]);
    v[0] = a;
  }
};

template <int DIR>
struct DFT<3, DIR> {
  template <typename C>
  __device__ __forceinline__ static void run(C* v) {
    using Rt = RealOf<C>;
    C t = cadd(v[1], v[2]);
    C d = cmul_i<DIR>(cscale(csub(v[1], v[2]), (Rt)kR3H));
    C m = mkc<C>(v[0].x - (Rt)0.5 * t.x, v[0].y - (Rt)0.5 * t.y);
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, d);
    v[2] = csub(m, d);
  }
};

template <int DIR>
struct DFT<4, DIR> {
  template <typename C>
  __device__ __forceinline__ static void run(C* v) {
    C a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    C b0 = cadd(v[1], v[3]), b1 = cmul_i<DIR>(csub(v[1], v[3]));
    v[0] = cadd(a0, b0);
    v[2] = csub(a0, b0);
    v[1] = cadd(a1, b1);
    v[3] = csub(a1, b1);
  }
};

// Two-factor Cooley-Tukey: R = A*B, n = B*n1 + n2, k = k1 + A*k2.
template <int A, int B, int DIR>
struct DFT_CT {
  static constexpr int R = A * B;
  template <typename C>
  __device__ __forceinline__ static void run(C* v) {
    C y[R];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
      C t[A];
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) t[n1] = v[B * n1 + n2];
      DFT<A, DIR>::run(t);
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) y[n2 * A + k1] = t[k1];
    }
    twiddle_all(y, std::make_integer_sequence<int, A * B>{});
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
      C t[B];
#pragma unroll
      for (int n2 = 0; n2 < B; ++n2) t[n2] = y[n2 * A + k1];
      DFT<B, DIR>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = t[k2];
    }
  }
  template <typename C, int... I>
  __device__ __forceinline__ static void twiddle_all(C* y, std::integer_sequence<int, I...>) {
    ((y[I] = rot<R, (I / A) * (I % A), DIR>(y[I])), ...);
  }
};

template <int DIR>
struct DFT<6, DIR> : DFT_CT<2, 3, DIR> {};
template <int DIR>
struct DFT<8, DIR> : DFT_CT<2, 4, DIR> {};
template <int DIR>
struct DFT<12, DIR> : DFT_CT<4, 3, DIR> {};
template <int DIR>
struct DFT<16, DIR> : DFT_CT<4, 4, DIR> {};

// ---------------------------------------------------------------------------
// synchronisation of the threads that own a line: SW is the width of the
// group that shares the line buffers (the T threads of the line when they
// sit in one warp, the whole CTA when lines are spread over warps)
// ---------------------------------------------------------------------------
template <int SW>
__device__ __forceinline__ void line_sync() {
  if constexpr (SW <= 32) {
    __syncwarp();
  } else {
    __syncthreads();
  }
}

// shared-memory line buffer index with one pad slot every PADW entries;
// PADW = 0: no padding, the position inside each row of 16 elements XORed
// with bits 3..6 of the index (the 8-byte lines of the FP32 z pass, whose
// Stockham exchanges the padding leaves 2-way bank conflicted)
template <int PADW>
__device__ __forceinline__ int spad(int p) {
  if constexpr (PADW == 0) {
    return (p & ~15) | ((p & 15) ^ ((p >> 3) & 15));
  } else {
    return p + p / PADW;
  }
}
template <int N, int PADW>
constexpr int line_buf_len() {
  return N + N / PADW + 1;
}

// ---------------------------------------------------------------------------
// Stockham stages
// ---------------------------------------------------------------------------
// Radix > 4 stages: read w, w^2, w^4, w^8 and compose the other twiddle
// powers (1), or read every power from the table (0).
#ifndef NS3D_TW_COMPOSE
#define NS3D_TW_COMPOSE 1
#endif
constexpr bool kComposeTwiddles = NS3D_TW_COMPOSE != 0;
template <int N, int T, int DIR, int PADW, int SW, int NS, int R, int... Rest>
struct Stages {
  static constexpr int P = N / T;
  static constexpr int U = P / R;
  static_assert(P % R == 0, "radix must divide the points per thread");

  template <typename C>
  __device__ __forceinline__ static void run(C (&x)[P], int t, C* sbuf,
                                             const C* __restrict__ tw) {
    constexpr bool last = sizeof...(Rest) == 0;
    static_assert(!last || NS * R == N, "radices must multiply to N");
    if constexpr (!last) line_sync<SW>();  // previous readers of sbuf are done
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int b = t + T * u;
      C v[R];
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = x[u + r * U];
      if constexpr (NS > 1) {
        // stage table [r-1][jm] = w^r, w = exp(2 pi i jm / (NS R)); consecutive
        // lanes read consecutive entries.  For R > 4 only w, w^2, w^4, w^8 are
        // read and the other powers composed (at most 3 products deep).
        const int jm = b % NS;
        C W[R];
#pragma unroll
        for (int r = 1; r < R; ++r) {
          if (!kComposeTwiddles || R <= 4 || r == 1 || r == 2 || r == 4 || r == 8) {
            W[r] = tw[(r - 1) * NS + jm];
          } else {
            // r = hi + lo with hi the largest of 8, 4, 2 below r (lo >= 1)
            const int hi = r > 8 ? 8 : (r > 4 ? 4 : 2);
            W[r] = cmul(W[hi], W[r - hi]);
          }
        }
#pragma unroll
        for (int r = 1; r < R; ++r) v[r] = cmul(v[r], mkc<C>(W[r].x, DIR * W[r].y));
      }
      DFT<R, DIR>::run(v);
      if constexpr (last) {
#pragma unroll
        for (int k = 0; k < R; ++k) x[u + k * U] = v[k];
      } else {
        const int base = (b / NS) * NS * R + (b % NS);
#pragma unroll
        for (int k = 0; k < R; ++k) sbuf[spad<PADW>(base + k * NS)] = v[k];
      }
    }
    if constexpr (!last) {
      line_sync<SW>();
#pragma unroll
      for (int s = 0; s < P; ++s) x[s] = sbuf[spad<PADW>(t + T * s)];
      Stages<N, T, DIR, PADW, SW, NS * R, Rest...>::run(x, t, sbuf,
                                                    NS > 1 ? tw + (R - 1) * NS : tw);
    }
  }
};

// Radix plans: Plan<N, P>::Rs... multiply to N and each divides P.
template <int... Rs>
struct RadixList {};

template <int N, int P>
struct Plan;
template <> struct Plan<8, 8> { using L = RadixList<8>; };
template <> struct Plan<8, 4> { using L = RadixList<4, 2>; };
template <> struct Plan<24, 6> { using L = RadixList<6, 2, 2>; };
template <> struct Plan<32, 4> { using L = RadixList<4, 4, 2>; };
template <> struct Plan<48, 6> { using L = RadixList<6, 2, 2, 2>; };
template <> struct Plan<64, 4> { using L = RadixList<4, 4, 4>; };
template <> struct Plan<96, 6> { using L = RadixList<6, 2, 2, 2, 2>; };
template <> struct Plan<128, 4> { using L = RadixList<4, 4, 4, 2>; };
template <> struct Plan<192, 6> { using L = RadixList<6, 2, 2, 2, 2, 2>; };
template <> struct Plan<256, 4> { using L = RadixList<4, 4, 4, 4>; };
template <> struct Plan<384, 6> { using L = RadixList<6, 2, 2, 2, 2, 2, 2>; };
template <> struct Plan<512, 4> { using L = RadixList<4, 4, 4, 4, 2>; };
template <> struct Plan<16, 4> { using L = RadixList<4, 4>; };
template <> struct Plan<16, 8> { using L = RadixList<8, 2>; };
template <> struct Plan<16, 16> { using L = RadixList<16>; };
template <> struct Plan<24, 12> { using L = RadixList<12, 2>; };
template <> struct Plan<32, 8> { using L = RadixList<8, 4>; };
template <> struct Plan<32, 16> { using L = RadixList<16, 2>; };
template <> struct Plan<48, 12> { using L = RadixList<12, 4>; };
template <> struct Plan<64, 8> { using L = RadixList<8, 8>; };
template <> struct Plan<64, 16> { using L = RadixList<16, 4>; };
template <> struct Plan<96, 12> { using L = RadixList<6, 4, 4>; };
template <> struct Plan<128, 8> { using L = RadixList<8, 4, 4>; };
template <> struct Plan<128, 16> { using L = RadixList<16, 8>; };
template <> struct Plan<192, 12> { using L = RadixList<12, 4, 4>; };
template <> struct Plan<256, 8> { using L = RadixList<8, 8, 4>; };
template <> struct Plan<256, 16> { using L = RadixList<16, 16>; };
template <> struct Plan<384, 12> { using L = RadixList<6, 4, 4, 4>; };
template <> struct Plan<512, 8> { using L = RadixList<8, 8, 8>; };
template <> struct Plan<512, 16> { using L = RadixList<16, 16, 2>; };

template <int N, int T, int DIR, int PADW, int SW, typename L>
struct RunPlan;
template <int N, int T, int DIR, int PADW, int SW, int... Rs>
struct RunPlan<N, T, DIR, PADW, SW, RadixList<Rs...>> {
  template <typename C>
  __device__ __forceinline__ static void run(C (&x)[N / T], int t, C* sbuf,
                                             const C* __restrict__ tw) {
    Stages<N, T, DIR, PADW, SW, 1, Rs...>::run(x, t, sbuf, tw);
  }
};

// First radix of a plan (the stride of the first exchange; used for padding).
template <typename L>
struct FirstRadix;
template <int R0, int... Rs>
struct FirstRadix<RadixList<R0, Rs...>> {
  static constexpr int value = R0;
};

// Per-stage twiddle tables of a plan, stage after stage (stages with NS > 1):
// entry (r-1)*NS + jm of a stage = exp(2 pi i jm r step / N), step = N/(NS R).
template <int N, int NS, typename L>
struct StageTw;
template <int N, int NS>
struct StageTw<N, NS, RadixList<>> {
  static constexpr int len = 0;
  template <typename C>
  __device__ __forceinline__ static void fill(C*, const double2* __restrict__) {}
};
template <int N, int NS, int R, int... Rest>
struct StageTw<N, NS, RadixList<R, Rest...>> {
  static constexpr int own = NS > 1 ? (R - 1) * NS : 0;
  using Next = StageTw<N, NS * R, RadixList<Rest...>>;
  static constexpr int len = own + Next::len;
  template <typename C>
  __device__ __forceinline__ static void fill(C* tws, const double2* __restrict__ tw_g) {
    if constexpr (NS > 1) {
      constexpr int step = N / (NS * R);
      for (int e = threadIdx.x; e < own; e += blockDim.x) {
        const int r = e / NS + 1, jm = e - (r - 1) * NS;
        tws[e] = cvt<C>(tw_g[jm * r * step]);  // FP64 table, rounded for FP32 lines
      }
    }
    Next::fill(tws + own, tw_g);
  }
};

// Radix schedules of one (N, P): V = 0 the plan above, V = 1 the same
// radices in reverse order (a different first-exchange stride and padding,
// other twiddle tables per stage); the tile autotuner times both where they
// differ.
template <typename L, typename Acc = RadixList<>>
struct ReverseList;
template <int... A>
struct ReverseList<RadixList<>, RadixList<A...>> {
  using type = RadixList<A...>;
};
template <int R, int... Rs, int... A>
struct ReverseList<RadixList<R, Rs...>, RadixList<A...>> {
  using type = typename ReverseList<RadixList<Rs...>, RadixList<R, A...>>::type;
};
template <int N, int P, int V>
struct PlanV {
  using L = typename Plan<N, P>::L;
};
template <int N, int P>
struct PlanV<N, P, 1> {
  using L = typename ReverseList<typename Plan<N, P>::L>::type;
};
// whether the reversed schedule differs from the plan (not a palindrome)
template <int N, int P>
__host__ __device__ constexpr bool plan_reversible() {
  return !std::is_same<typename PlanV<N, P, 0>::L, typename PlanV<N, P, 1>::L>::value;
}

template <int N, int P, int V = 0>
struct LineFFT {
  static constexpr int T = N / P;
  using L = typename PlanV<N, P, V>::L;
  static constexpr int PADW = FirstRadix<L>::value < 4 ? 4 : FirstRadix<L>::value;
  static constexpr int BUF = line_buf_len<N, PADW>();
  // shared-memory twiddle words the plan needs (N - first radix), at least 1
  static constexpr int TWLEN = StageTw<N, 1, L>::len > 0 ? StageTw<N, 1, L>::len : 1;
  // fills the per-stage table from the global table tw_g[e] = exp(2 pi i e / N);
  // ends with a CTA barrier
  template <typename C>
  __device__ __forceinline__ static void load_tw(C* tws, const double2* __restrict__ tw_g) {
    StageTw<N, 1, L>::fill(tws, tw_g);
    __syncthreads();
  }
  // PW: the line-buffer index scheme (PADW, or 0 for the XOR swizzle);
  // SW: the synchronisation width (T: the line's threads share a warp)
  template <int DIR, int PW = PADW, int SW = T, typename C>
  __device__ __forceinline__ static void run(C (&x)[P], int t, C* sbuf,
                                             const C* __restrict__ tw) {
    RunPlan<N, T, DIR, PW, SW, L>::run(x, t, sbuf, tw);
  }
};

}  // namespace ns3d
