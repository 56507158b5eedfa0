// Per-extent dispatch of the pass kernels (host side).
#pragma once

#include <cuda_runtime.h>

#include <atomic>

#include "passes.cuh"

namespace ns3d {

// Extents with compiled plans.
#ifndef NS3D_FOR_EACH_EXTENT
#define NS3D_FOR_EACH_EXTENT(X) \
  X(8) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512)
#endif

// Points per thread of power-of-two extents, per pass family.
#ifndef NS3D_PXY
#define NS3D_PXY 16
#endif
#ifndef NS3D_PZ
#define NS3D_PZ 8
#endif
#ifndef NS3D_PFX
#define NS3D_PFX 16
#endif

// Points per thread: x/y passes that hold one or two lines per thread, and
// the z / fwd_x passes that hold several fields per thread at once.
constexpr int p_pow2(int n, int p) { return p > n ? n : p; }
constexpr int p_xy(int n) { return n % 3 == 0 ? 12 : p_pow2(n, NS3D_PXY); }
constexpr int p_z(int n) { return n % 3 == 0 ? 12 : p_pow2(n, NS3D_PZ); }
constexpr int p_fx(int n) { return n % 3 == 0 ? 12 : p_pow2(n, NS3D_PFX); }
// the tangent z pass keeps u, v and the three products live: fewer points
constexpr int p_zuv(int n) { return n % 3 == 0 ? 6 : 4; }
// The nonlinear term's z pass with the velocities stashed in shared memory
// (z_kernel_st): 16 points per thread for powers of two (one Stockham
// exchange per 256-point transform instead of two), 12 for multiples of 3.
// NS3D_Z_STASH 0 keeps z_kernel with p_z points per thread.
#ifndef NS3D_Z_STASH
#define NS3D_Z_STASH 1
#endif
#ifndef NS3D_PZST
#define NS3D_PZST 16
#endif
constexpr int p_zst(int n) { return n % 3 == 0 ? 12 : p_pow2(n, NS3D_PZST); }
// FP32 lines of the nonlinear term's z pass: half the registers per point,
// so 16 points per thread fit without the stash (one exchange per transform)
#ifndef NS3D_PZ32
#define NS3D_PZ32 16
#endif
constexpr int p_z32(int n) { return n % 3 == 0 ? 12 : p_pow2(n, NS3D_PZ32); }
// points per thread of the plain line passes (8 measured slower than 16 at 256^3 and 512^3)
#ifndef NS3D_PLINE
#define NS3D_PLINE 16
#endif
constexpr int p_line(int n) { return n % 3 == 0 ? 12 : p_pow2(n, NS3D_PLINE); }
// points per thread of the plain transforms' z passes (pairs of real lines)
#ifndef NS3D_PZPLAIN
#define NS3D_PZPLAIN 8
#endif
constexpr int p_zplain(int n) { return n % 3 == 0 ? 12 : p_pow2(n, NS3D_PZPLAIN); }
// The autotuner's alternative tile of the pipelined x / y passes: 8 points
// per thread for powers of two from 32, 6 for multiples of 3 from 48 (twice
// the lines per CTA, half the registers and prefetch buffers); 0: none.
constexpr int p_alt(int n) {
  return n % 3 == 0 ? (n >= 48 ? 6 : 0) : (n >= 32 ? 8 : 0);
}
inline bool has_alt_tile(int n) {
  switch (n) {
#define NS3D_CASE(N) \
  case N:            \
    return p_alt(N) > 0;
    NS3D_FOR_EACH_EXTENT(NS3D_CASE)
#undef NS3D_CASE
    default:
      return false;
  }
}

// The bulk-copy (TMA) form of inv_y (inv_y_tma_kernel): FP64 lines spread
// over the CTA (y extents from 48).  It is tile 2 of the inv_y family, at p_tma(n) points per
// thread (the default or the alternative points per thread, whichever
// spreads its lines over the CTA; 0: no such form for this extent), and runs
// where the handle built tensor maps for its scratch; the tangent form and
// the FP32 mode run the cp.async form at p_tma(n) points per thread instead.
// NS3D_Y_TMA 0 compiles no bulk-copy form.
#ifndef NS3D_Y_TMA
#define NS3D_Y_TMA 1
#endif
// 1: the TMA form runs persistent CTAs (resident CTAs, groups dealt round
// robin), so each CTA's copy ring runs across many groups; 0: NS3D_SCHED.
#ifndef NS3D_Y_TMA_PERSIST
#define NS3D_Y_TMA_PERSIST 0
#endif
constexpr int p_tma(int n) {
  return NS3D_Y_TMA == 0                              ? 0
         : n / p_xy(n) >= NS3D_SPREAD_T                          ? p_xy(n)
         : (p_alt(n) > 0 && n / p_alt(n) >= NS3D_SPREAD_T) ? p_alt(n)
                                                      : 0;
}

// Lines per CTA of the TMA form of inv_y for extent n, 0 when it has none.
inline int inv_y_tma_lpc_inline(int n) {
  switch (n) {
#define NS3D_CASE(N) \
  case N:            \
    return p_tma(N) > 0 ? LaneMap<N / (p_tma(N) > 0 ? p_tma(N) : 1)>::LPC : 0;
    NS3D_FOR_EACH_EXTENT(NS3D_CASE)
#undef NS3D_CASE
    default:
      return 0;
  }
}

inline bool extent_supported_inline(int n) {
  switch (n) {
#define NS3D_CASE(N) case N:
    NS3D_FOR_EACH_EXTENT(NS3D_CASE)
#undef NS3D_CASE
    return true;
    default:
      return false;
  }
}

template <int N, int P>
constexpr int lines_per_cta_xy() {
  return LaneMap<N / P>::LPC;
}
template <int N, int P>
constexpr int lines_per_cta_z() {
  return ZLaneMap<N / P>::LPC;
}

inline unsigned blocks_for(long long lines, int lpc) { return (unsigned)((lines + lpc - 1) / lpc); }

// Persistent grid for a pipelined pass: set the dynamic shared-memory
// attribute and query the resident CTAs per SM once per kernel instantiation
// (Tag) and device; grid = min(groups, SMs x resident CTAs).
template <int KIND, int N, int P, int X>
struct KTag {};

// The caches are atomics: host threads that launch on the same device may
// race to fill them, and each writes the same values.
// kCap: cap the grid at the resident CTAs whatever NS3D_SCHED says (kernels
// whose CTAs keep a copy pipeline running across their groups).
template <typename Tag, bool kCap = (NS3D_SCHED != 0), typename Kern>
inline unsigned persistent_grid(Kern kern, size_t smem, long long groups) {
  static std::atomic<int> per_sm[64] = {};
  static std::atomic<int> sms[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  dev &= 63;
  if (per_sm[dev].load(std::memory_order_acquire) == 0) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, smem);
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    sms[dev].store(n > 0 ? n : 1, std::memory_order_relaxed);
    per_sm[dev].store(occ > 0 ? occ : 1, std::memory_order_release);
  }
  const long long cap = !kCap ? groups : (long long)sms[dev].load() * per_sm[dev].load();
  return (unsigned)(groups < cap ? (groups > 0 ? groups : 1) : cap);
}

// KTag's last argument separates the FP64 and FP32 instantiations.
template <typename C>
constexpr int prec_tag() { return sizeof(C) == 16 ? 0 : 100; }

template <int N, int P, int NF, typename C, int V = 0>
cudaError_t launch_inv_x_p(const InvXArgs<NF, C>& a, const PassGeom& g, cudaStream_t st,
                           bool prepare_only) {
  const long long lines = (long long)g.Ny * g.Mz * nbatch(g);
  using S = PassSmem<N, P, C, double2, V>;
  const unsigned grid = persistent_grid<KTag<0, N, P, NF + prec_tag<C>() + 1000 * V>>(
      inv_x_kernel<N, P, NF, C, V>, S::BYTES, (lines + S::LPC - 1) / S::LPC);
  if (prepare_only) return cudaGetLastError();
  inv_x_kernel<N, P, NF, C, V><<<grid, kThreads, S::BYTES, st>>>(a, g);
  return cudaGetLastError();
}

// The x / y families' tiles 3 and 4: the default and the alternative points
// per thread with the reversed radix schedule, where it differs.
template <int N>
constexpr bool rev_tile_default() {
  return plan_reversible<N, p_xy(N)>();
}
template <int N>
constexpr bool rev_tile_alt() {
  if constexpr (p_alt(N) > 0) {
    return plan_reversible<N, p_alt(N)>();
  } else {
    return false;
  }
}
inline bool rev_tile_exists_inline(int n, int tile) {
  switch (n) {
#define NS3D_CASE(N) \
  case N:            \
    return tile == 3 ? rev_tile_default<N>() : (tile == 4 ? rev_tile_alt<N>() : false);
    NS3D_FOR_EACH_EXTENT(NS3D_CASE)
#undef NS3D_CASE
    default:
      return false;
  }
}

// V = 0: tiles 0 and 1; V = 1: tiles 3 and 4 (the reversed schedules)
template <int NF, typename C, int V = 0>
cudaError_t launch_inv_x(const InvXArgs<NF, C>& a, const PassGeom& g, cudaStream_t st,
                         bool prepare_only = false) {
  const int tile = g.tile[kTileInvX];
  switch (g.Nx) {
#define NS3D_CASE(N)                                                                \
  case N:                                                                           \
    if constexpr (V == 0) {                                                         \
      if constexpr (p_alt(N) > 0) {                                                 \
        if (tile == 1) return launch_inv_x_p<N, p_alt(N), NF, C>(a, g, st, prepare_only); \
      }                                                                             \
      return launch_inv_x_p<N, p_xy(N), NF, C>(a, g, st, prepare_only);             \
    } else {                                                                        \
      if constexpr (rev_tile_alt<N>()) {                                            \
        if (tile == 4)                                                              \
          return launch_inv_x_p<N, p_alt(N), NF, C, 1>(a, g, st, prepare_only);     \
      }                                                                             \
      if constexpr (rev_tile_default<N>()) {                                        \
        if (tile == 3)                                                              \
          return launch_inv_x_p<N, p_xy(N), NF, C, 1>(a, g, st, prepare_only);      \
      }                                                                             \
      return cudaErrorInvalidValue;                                                 \
    }
    NS3D_FOR_EACH_EXTENT(NS3D_CASE)
#undef NS3D_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <int N, int P>
cudaError_t launch_inv_y_tma(const InvYArgs<3, double2>& a, const PassGeom& g, cudaStream_t st,
                             bool prepare_only) {
  using S = InvYTmaSmem<N, P>;
  const long long groups = (long long)g.Nx * ((g.Mz + S::LPC - 1) / S::LPC);
  const unsigned grid = persistent_grid<KTag<90, N, P, 3>, NS3D_Y_TMA_PERSIST != 0>(
      inv_y_tma_kernel<N, P, 3>, S::BYTES, groups);
  if (prepare_only) return cudaGetLastError();
  InvYTmaArgs<3> t;
  t.m = *a.maps;
  for (int f = 0; f < 3; ++f) {
    t.C[f] = a.C[f];
    t.D[f] = a.D[f];
    t.E[f] = a.E[f];
  }
  t.tw = a.tw;
  t.err = a.err;
  inv_y_tma_kernel<N, P, 3><<<grid, kThreads, S::BYTES, st>>>(t, g);
  return cudaGetLastError();
}

template <int N, int P, int NF, typename C, int V = 0>
cudaError_t launch_inv_y_p(const InvYArgs<NF, C>& a, const PassGeom& g, cudaStream_t st,
                           bool prepare_only, bool bulk = false) {
  if constexpr (V == 0 && NF == 3 && sizeof(C) == 16 && P == p_tma(N)) {
    if (bulk && (a.maps || prepare_only)) {
      const cudaError_t e = launch_inv_y_tma<N, P>(a, g, st, prepare_only);
      if (!prepare_only || e != cudaSuccess) return e;
    }
  }
  const long long lines = (long long)g.Nx * g.Mz;
  using S = PassSmem<N, P, C, C, V>;
  const unsigned grid = persistent_grid<KTag<1, N, P, NF + prec_tag<C>() + 1000 * V>>(
      inv_y_kernel<N, P, NF, C, V>, S::BYTES, (lines + S::LPC - 1) / S::LPC);
  if (prepare_only) return cudaGetLastError();
  inv_y_kernel<N, P, NF, C, V><<<grid, kThreads, S::BYTES, st>>>(a, g);
  return cudaGetLastError();
}

template <int NF, typename C, int V = 0>
cudaError_t launch_inv_y(const InvYArgs<NF, C>& a, const PassGeom& gi, cudaStream_t st,
                         bool prepare_only = false) {
  const PassGeom g = planes_geom(gi);
  const int tile = g.tile[kTileInvY];
  switch (g.Ny) {
#define NS3D_CASE(N)                                                                \
  case N:                                                                           \
    if constexpr (V == 0) {                                                         \
      if constexpr (p_tma(N) > 0) {                                                 \
        if (tile == 2)                                                              \
          return launch_inv_y_p<N, p_tma(N), NF, C>(a, g, st, prepare_only, true);  \
      }                                                                             \
      if constexpr (p_alt(N) > 0) {                                                 \
        if (tile == 1) return launch_inv_y_p<N, p_alt(N), NF, C>(a, g, st, prepare_only); \
      }                                                                             \
      return launch_inv_y_p<N, p_xy(N), NF, C>(a, g, st, prepare_only);             \
    } else {                                                                        \
      if constexpr (rev_tile_alt<N>()) {                                            \
        if (tile == 4)                                                              \
          return launch_inv_y_p<N, p_alt(N), NF, C, 1>(a, g, st, prepare_only);     \
      }                                                                             \
      if constexpr (rev_tile_default<N>()) {                                        \
        if (tile == 3)                                                              \
          return launch_inv_y_p<N, p_xy(N), NF, C, 1>(a, g, st, prepare_only);      \
      }                                                                             \
      return cudaErrorInvalidValue;                                                 \
    }
    NS3D_FOR_EACH_EXTENT(NS3D_CASE)
#undef NS3D_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <int N, typename C>
cudaError_t launch_z_stash(const ZArgs<3, C>& a, const PassGeom& g, cudaStream_t st) {
  constexpr int P = p_zst(N);
  using S = ZStashSmem<N, P, C>;
  constexpr bool TM = z_tmem(N);
  constexpr size_t bytes = TM ? S::TM_BYTES : S::BYTES;
  const long long lines = (long long)g.Nx * g.Ny;
  const unsigned grid = persistent_grid<KTag<40, N, P, prec_tag<C>()>>(
      z_kernel_st<N, P, C, TM>, bytes, blocks_for(lines, lines_per_cta_z<N, P>()));
  z_kernel_st<N, P, C, TM><<<grid, kThreads, bytes, st>>>(a, g);
  return cudaGetLastError();
}

template <bool UV, typename C>
cudaError_t launch_z(const ZArgs<UV ? 6 : 3, C>& a, const PassGeom& gi, cudaStream_t st) {
  const PassGeom g = planes_geom(gi);
  const long long lines = (long long)g.Nx * g.Ny;
  switch (g.Nz) {
#define NS3D_CASE(N)                                                               \
  case N: {                                                                        \
    if constexpr (!UV && NS3D_Z_STASH && sizeof(C) == 16) {                        \
      return launch_z_stash<N, C>(a, g, st);                                       \
    }                                                                              \
    constexpr int P = UV ? p_zuv(N) : (sizeof(C) == 8 ? p_z32(N) : p_z(N));        \
    z_kernel<N, P, UV, C><<<blocks_for(lines, lines_per_cta_z<N, P>()),           \
                         kWarpsPerCta * 32, 0, st>>>(a, g);                        \
    return cudaGetLastError();                                                     \
  }
    NS3D_FOR_EACH_EXTENT(NS3D_CASE)
#undef NS3D_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <int N, int P, int MODE, bool COMBINE, typename C>
cudaError_t launch_fwd_x_p(const FwdXArgs<C>& a, const PassGeom& g, cudaStream_t st,
                           bool prepare_only) {
  const long long lines = (long long)g.Ny * g.Mz * nbatch(g);
  using S = PassSmem<N, P, C, C>;
  const unsigned grid =
      persistent_grid<KTag<2 + 2 * MODE + (COMBINE ? 1 : 0), N, P, prec_tag<C>()>>(
          fwd_x_kernel<N, P, MODE, COMBINE, C>, S::BYTES, (lines + S::LPC - 1) / S::LPC);
  if (prepare_only) return cudaGetLastError();
  fwd_x_kernel<N, P, MODE, COMBINE, C><<<grid, kThreads, S::BYTES, st>>>(a, g);
  return cudaGetLastError();
}

// fwd_x with the update operands in the prefetch ring (fwd_x_ring_kernel):
// 8 points per thread for powers of two, 12 for multiples of 3, and as many
// slots as two CTAs per SM leave room for; used where a line fits in a warp
// (to 256 and 384 points).  At 512 points the ring's lines would spread over
// the CTA two at a time (32-byte rows): measured 4.69 ms per launch
// there against 3.42 ms for fwd_x_kernel with 16 points per thread.
#ifndef NS3D_FX_RING
#define NS3D_FX_RING 1
#endif
#ifndef NS3D_FX_RING32
#define NS3D_FX_RING32 1
#endif
#ifndef NS3D_PFXR
#define NS3D_PFXR 8
#endif
constexpr int p_fxr(int n) { return n % 3 == 0 ? 12 : p_pow2(n, NS3D_PFXR); }
constexpr int nslot_fxr(int p) { return p > 8 ? 3 : NS3D_FX_SLOTS; }
// The ring where its lines are a warp wide (64-byte rows over the CTA), or
// where fwd_x_kernel's own lines would stay inside their warps; elsewhere
// fwd_x_kernel's lines, interleaved over the CTA, read wider rows than the
// ring's.  Per plain launch on a B200: 256^3 ring 295 us, fwd_x_kernel (16
// points) 383 us; 128^3 ring 65.5 us, fwd_x_kernel 61.7 us.
template <int N, typename C>
constexpr bool fx_use_ring() {
  return NS3D_FX_RING && N / p_fxr(N) <= 32 && (NS3D_FX_RING32 || sizeof(C) == 16) &&
         (N / p_fxr(N) == 32 || N / p_fx(N) < NS3D_SPREAD_T);
}

template <int N, int P, int MODE, bool COMBINE, typename C>
cudaError_t launch_fwd_x_ring(const FwdXArgs<C>& a, const PassGeom& g, cudaStream_t st,
                              bool prepare_only) {
  constexpr int NSLOT = nslot_fxr(P);
  const long long lines = (long long)g.Ny * g.Mz * nbatch(g);
  using S = FxRingSmem<N, P, NSLOT, C>;
  const unsigned grid =
      persistent_grid<KTag<50 + 2 * MODE + (COMBINE ? 1 : 0), N, P, prec_tag<C>()>>(
          fwd_x_ring_kernel<N, P, MODE, COMBINE, NSLOT, C>, S::BYTES,
          (lines + S::LPC - 1) / S::LPC);
  if (prepare_only) return cudaGetLastError();
  fwd_x_ring_kernel<N, P, MODE, COMBINE, NSLOT, C><<<grid, kThreads, S::BYTES, st>>>(a, g);
  return cudaGetLastError();
}

template <int MODE, bool COMBINE, typename C>
cudaError_t launch_fwd_x(const FwdXArgs<C>& a, const PassGeom& g, cudaStream_t st,
                         bool prepare_only = false) {
  switch (g.Nx) {
#define NS3D_CASE(N)                                                                  \
  case N:                                                                             \
    if constexpr (p_alt(N) > 0) {                                                     \
      if (g.tile[kTileFwdX])                                                          \
        return launch_fwd_x_p<N, p_alt(N), MODE, COMBINE, C>(a, g, st, prepare_only); \
    }                                                                                 \
    if constexpr (fx_use_ring<N, C>())                                                \
      return launch_fwd_x_ring<N, p_fxr(N), MODE, COMBINE, C>(a, g, st, prepare_only); \
    return launch_fwd_x_p<N, p_fx(N), MODE, COMBINE, C>(a, g, st, prepare_only);
    NS3D_FOR_EACH_EXTENT(NS3D_CASE)
#undef NS3D_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <int N, int P, typename C, int V = 0>
cudaError_t launch_fwd_y_p(const FwdYArgs<C>& a, const PassGeom& g, cudaStream_t st,
                           bool prepare_only) {
  const long long lines = (long long)g.Nx * g.Mz;
  using S = PassSmem<N, P, C, C, V>;
  const unsigned grid = persistent_grid<KTag<20, N, P, prec_tag<C>() + 1000 * V>>(
      fwd_y_kernel<N, P, C, V>, S::BYTES, (lines + S::LPC - 1) / S::LPC);
  if (prepare_only) return cudaGetLastError();
  fwd_y_kernel<N, P, C, V><<<grid, kThreads, S::BYTES, st>>>(a, g);
  return cudaGetLastError();
}

template <typename C, int V = 0>
cudaError_t launch_fwd_y(const FwdYArgs<C>& a, const PassGeom& gi, cudaStream_t st,
                         bool prepare_only = false) {
  const PassGeom g = planes_geom(gi);
  const int tile = g.tile[kTileFwdY];
  switch (g.Ny) {
#define NS3D_CASE(N)                                                                \
  case N:                                                                           \
    if constexpr (V == 0) {                                                         \
      if constexpr (p_alt(N) > 0) {                                                 \
        if (tile == 1) return launch_fwd_y_p<N, p_alt(N), C>(a, g, st, prepare_only); \
      }                                                                             \
      return launch_fwd_y_p<N, p_xy(N), C>(a, g, st, prepare_only);                 \
    } else {                                                                        \
      if constexpr (rev_tile_alt<N>()) {                                            \
        if (tile == 4) return launch_fwd_y_p<N, p_alt(N), C, 1>(a, g, st, prepare_only); \
      }                                                                             \
      if constexpr (rev_tile_default<N>()) {                                        \
        if (tile == 3) return launch_fwd_y_p<N, p_xy(N), C, 1>(a, g, st, prepare_only); \
      }                                                                             \
      return cudaErrorInvalidValue;                                                 \
    }
    NS3D_FOR_EACH_EXTENT(NS3D_CASE)
#undef NS3D_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <int AXIS, int DIR>
cudaError_t launch_line(const LineArgs& a, const PassGeom& g, cudaStream_t st,
                        bool prepare_only = false) {
  const long long lines = AXIS == 0 ? (long long)g.Ny * g.Mz : (long long)g.Nx * g.Mz;
  switch (AXIS == 0 ? g.Nx : g.Ny) {
#define NS3D_CASE(N)                                                                    \
  case N: {                                                                             \
    constexpr int P = p_line(N);                                                           \
    using S = PassSmem<N, P>;                                                           \
    const unsigned grid = persistent_grid<KTag<30 + 2 * AXIS + (DIR > 0 ? 1 : 0), N, P, 0>>( \
        line_kernel<N, P, AXIS, DIR>, S::BYTES, (lines + S::LPC - 1) / S::LPC);         \
    if (prepare_only) return cudaGetLastError();                                        \
    line_kernel<N, P, AXIS, DIR><<<grid, kThreads, S::BYTES, st>>>(a, g);                \
    return cudaGetLastError();                                                          \
  }
    NS3D_FOR_EACH_EXTENT(NS3D_CASE)
#undef NS3D_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <bool C2R>
cudaError_t launch_z_plain(const ZPlainArgs& a, const PassGeom& g, cudaStream_t st) {
  const long long pairs = ((long long)g.Nx * g.Ny) / 2;
  switch (g.Nz) {
#define NS3D_CASE(N)                                                                  \
  case N: {                                                                           \
    constexpr int P = p_zplain(N);                                                    \
    const unsigned grid = blocks_for(pairs, lines_per_cta_z<N, P>());                 \
    if (C2R)                                                                          \
      z_c2r_kernel<N, P><<<grid, kWarpsPerCta * 32, 0, st>>>(a, g);                   \
    else                                                                              \
      z_r2c_kernel<N, P><<<grid, kWarpsPerCta * 32, 0, st>>>(a, g);                   \
    return cudaGetLastError();                                                        \
  }
    NS3D_FOR_EACH_EXTENT(NS3D_CASE)
#undef NS3D_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace ns3d
