// Pass kernels of the pseudo-spectral right-hand side.
//
// Spectral fields use the reference layout [Nx][Ny][Mz] of double2
// (Source/Macros.h:11 IN(i,j,k) with Nz = Mz), Mz = Nz/2 + 1.  One RHS
// evaluation is five launches over that layout ("P3L": three passes per 3-D
// transform, derivatives formed lazily, products and the forward z transform
// fused in one pass, projection/diffusion/RK combination fused into the last):
//
//   inv_x : u (3)            -> A = IFFT_x(M u), B = IFFT_x(i kx M u)     (M = 2/3 mask)
//   inv_y : A, B (6)         -> C = IFFT_y A, D = IFFT_y(i ky A), E = IFFT_y B
//   z     : C, D, E (9)      -> C2R along z (12 real lines = 6 complex IFFTs),
//                               Q_i = sum_j u_j d_j u_i, R2C along z  -> Qh (3)
//   fwd_y : Qh (3) in place  -> FFT_y
//   fwd_x : Qh (3), u, ...   -> FFT_x, Re(Qh)=0, Qh(0)=0, Leray, diffusion,
//                               forcing, RK combination -> new state
//
// The tangent (B(u,v)) variant carries 6 fields through inv_x / inv_y and
// forms (v.grad)u + (u.grad)v in the z pass (Source/advection_2_3.cu:401-475).
#pragma once

#include <cstdint>

#include "fft_engine.cuh"
#include "tma.cuh"
#include "tmem.cuh"

namespace ns3d {

constexpr int kWarpsPerCta = 4;
// Minimum resident CTAs per SM requested from ptxas (caps registers/thread).
#ifndef NS3D_MINCTA_XY
#define NS3D_MINCTA_XY 2
#endif
#ifndef NS3D_MINCTA_Z
#define NS3D_MINCTA_Z 2
#endif
#ifndef NS3D_MINCTA_FX
#define NS3D_MINCTA_FX 2
#endif
constexpr int kMinCtasXY = NS3D_MINCTA_XY;
// The x / y passes' tiles of 8 points or fewer per thread (the autotuner's
// alternative for long lines) ask for NS3D_MINCTA_XY8 CTAs per SM (at most
// 168 registers; 152-168 used, no spills).  B200, 256^3 with 3: the tuner
// keeps the 8-point tiles of inv_x, inv_y and fwd_y (264 / 463 / 172 us
// against 293 / 479 / 181 us), RK3 step 5.23 -> 5.08 ms; FP32 mode 4.05 ->
// 3.94 ms; 128^3 unchanged (the 16-point defaults stay faster there).
#ifndef NS3D_MINCTA_XY8
#define NS3D_MINCTA_XY8 3
#endif
__host__ __device__ constexpr int min_ctas_xy(int p) { return p <= 8 ? NS3D_MINCTA_XY8 : kMinCtasXY; }
constexpr int kMinCtasZ = NS3D_MINCTA_Z;
constexpr int kMinCtasFwdX = NS3D_MINCTA_FX;

struct PassGeom {
  int Nx, Ny, Nz, Mz;
  double kfx, kfy, kfz;  // 2*pi/L per direction (Source/math_support.cu:350-370)
  double inv_vol;        // 1/(Nx*Ny*Nz), the scale_double factor
  // Independent instances of one grid stored back to back ([batch][Nx][Ny][Mz]
  // per field).  The y and z passes see them as one grid of batch*Nx planes;
  // the x passes split their line index into (instance, y*Mz + z).  0 or 1:
  // a single instance.
  int batch;
  // Tile choice per pipelined pass family (TileFamily), set by the autotuner:
  // 0 the default points per thread, 1 the alternative (p_alt), 2 inv_y's
  // bulk-copy form, 3 / 4 the default / alternative points per thread with
  // the reversed radix schedule (x / y families inv_x, inv_y, fwd_y).
  int tile[4];
};
enum TileFamily { kTileInvX = 0, kTileInvY = 1, kTileFwdY = 2, kTileFwdX = 3 };
__host__ __device__ __forceinline__ int nbatch(const PassGeom& g) {
  return g.batch > 1 ? g.batch : 1;
}
// The geometry the y and z passes use: the instances as extra x planes.
__host__ __device__ __forceinline__ PassGeom planes_geom(const PassGeom& g) {
  PassGeom p = g;
  p.Nx = g.Nx * nbatch(g);
  p.batch = 1;
  return p;
}

// signed wavenumber index: j < N/2 -> j, else j - N (x and y; the Nyquist
// index N/2 is stored as -N/2, Source/math_support.cu:354-357)
__device__ __forceinline__ int signed_idx(int j, int n) { return j < (n >> 1) ? j : j - n; }

// Thread -> (line slot, t) for passes whose batch index is contiguous in
// memory: lanes with the same t and consecutive lines are adjacent, so a warp
// reads runs of consecutive elements of each row.  Lines of NS3D_SPREAD_T
// threads or more are interleaved over the whole CTA (line threadIdx % LPC,
// t = threadIdx / LPC, synchronised per CTA), so the LPC = 128 / T lines of
// a CTA put LPC x 16 contiguous bytes of each row into one load: 64 bytes
// for 32-thread lines, 128 for 16, 256 for 8.  Narrower lines stay inside
// their warp (LPW lines per warp, synchronised per warp).  Measured on a B200
// (us per launch, 16 points per thread, lines of 16 threads: 32-byte rows
// inside a warp -> 128-byte rows over the CTA): 256^3 inv_x 294 -> 217,
// inv_y 535 -> 440, fwd_y 182 -> 151; 128^3 (8 threads, 32 -> 256 bytes)
// inv_y 64.5 -> 58.8; the extra CTA barriers cost less than the narrow rows.
#ifndef NS3D_SPREAD_T
#define NS3D_SPREAD_T 8
#endif
template <int T>
struct LaneMap {
  static constexpr bool kSpread = T >= NS3D_SPREAD_T;
  static constexpr int LPW = T < 32 ? 32 / T : 1;
  static constexpr int LPC = (kWarpsPerCta * 32) / T;
  static constexpr int SW = kSpread ? kWarpsPerCta * 32 : T;  // line_sync width
  // lines side by side in the lanes of one load
  static constexpr int ADJ = kSpread ? LPC : LPW;
  __device__ __forceinline__ static void get(int& li, int& t) {
    if constexpr (!kSpread) {
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
      t = lane / LPW;
      li = warp * LPW + lane % LPW;
    } else {
      li = threadIdx.x % LPC;
      t = threadIdx.x / LPC;
    }
  }
};


// ---------------------------------------------------------------------------
// Software-pipelined x / y passes.  A CTA handles groups of LPC lines (one
// group per CTA by default, see NS3D_SCHED); every thread owns a private
// double buffer in shared memory and, while the current line of field f is
// transformed, prefetches with cp.async the P samples it will need for the
// next unit (the next field of the same lines, or the first field of the
// next group).
// ---------------------------------------------------------------------------
constexpr int kThreads = kWarpsPerCta * 32;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred = true) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = pred ? 16 : 0;  // 0: nothing is read, the slot is zero-filled
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool pred = true) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n)
               : "memory");
}
// one complex element: 16 bytes (FP64) or 8 bytes (FP32)
template <typename E>
__device__ __forceinline__ void cp_async_elem(E* smem, const E* gmem, bool pred) {
  static_assert(sizeof(E) == 16 || sizeof(E) == 8, "complex element");
  if constexpr (sizeof(E) == 16) {
    cp_async16(smem, gmem, pred);
  } else {
    cp_async8(smem, gmem, pred);
  }
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Copies the P samples t + T*s (s < P) of one line into a private slot:
// slot[s*SS] <- src[base + (t + T*s) * stride], skipping (zero-filling)
// the samples whose bit in `keep` is clear.  SS is the slot's sample stride
// in elements (kThreads: each thread's samples interleaved with the others').
template <int P, int T, int SS = kThreads, typename E>
__device__ __forceinline__ void issue_line(E* slot, const E* __restrict__ src,
                                           size_t base, size_t stride, int t,
                                           uint32_t keep = 0xffffffffu) {
#pragma unroll
  for (int s = 0; s < P; ++s)
    cp_async_elem(slot + s * SS, src + base + (size_t)(t + T * s) * stride,
                  (keep >> s) & 1u);
}

// Smallest line-buffer stride >= len whose residue mod 8 (16-byte slots; one
// shared-memory wavefront is 8 slots) is `target`, 0 meaning any.
constexpr int line_stride(int len, int target) {
  return target == 0 ? len : (len % 8 == target % 8 ? len : line_stride(len + 1, target));
}
// LaneMap puts ADJ lines side by side in a quarter warp: give each its own
// 16-byte slots.
template <int T>
constexpr int xy_stride_target() {
  constexpr int adj = LaneMap<T>::ADJ;
  constexpr int per_phase = adj < 8 ? adj : 8;
  return per_phase <= 1 ? 0 : 8 / per_phase;
}


// Work distribution of the pipelined passes over groups of lines:
//   NS3D_SCHED 0: one group per CTA (grid = groups; the hardware scheduler
//                 keeps the resident CTAs on a window of neighbouring groups),
//   NS3D_SCHED 1: persistent CTAs, groups dealt round robin,
//   NS3D_SCHED 2: persistent CTAs, one contiguous range of groups each.
#ifndef NS3D_SCHED
#define NS3D_SCHED 0
#endif
struct GroupRange {
  int grp, end, step;
};
__device__ __forceinline__ GroupRange group_range(int groups) {
  if (NS3D_SCHED == 2) {
    return {(int)(((long long)blockIdx.x * groups) / gridDim.x),
            (int)(((long long)(blockIdx.x + 1) * groups) / gridDim.x), 1};
  }
  return {(int)blockIdx.x, groups, (int)gridDim.x};
}

constexpr size_t align16(size_t b) { return (b + 15) / 16 * 16; }

// Dynamic shared memory of a pipelined pass: the stage twiddles and the line
// buffers in the line precision C, then each thread's double buffer of
// prefetched elements of type E (the pass's input, FP64 state or scratch).
// V: the radix schedule (PlanV).
template <int N, int P, typename C = double2, typename E = C, int V = 0>
struct PassSmem {
  using F = LineFFT<N, P, V>;
  using LM = LaneMap<F::T>;
  static constexpr int LPC = LM::LPC;
  static constexpr int STRIDE = line_stride(F::BUF, xy_stride_target<F::T>());
  static constexpr size_t SBUF_OFF = align16((size_t)F::TWLEN * sizeof(C));
  static constexpr size_t PF_OFF = align16(SBUF_OFF + (size_t)LPC * STRIDE * sizeof(C));
  static constexpr size_t BYTES = PF_OFF + (size_t)2 * P * kThreads * sizeof(E);
  static_assert(BYTES <= 227 * 1024, "shared memory per CTA");
  __device__ __forceinline__ static C* tw(unsigned char* base) { return (C*)base; }
  __device__ __forceinline__ static C* sbuf(unsigned char* base, int li) {
    return (C*)(base + SBUF_OFF) + li * STRIDE;
  }
  __device__ __forceinline__ static E* pf(unsigned char* base) {
    return (E*)(base + PF_OFF) + threadIdx.x;
  }
};

template <int NX>
__device__ __forceinline__ uint32_t mask_bits(const uint16_t* __restrict__ qcut, int Ny, int y,
                                              int z, int L, bool valid, int t, int T, int P) {
  uint32_t keep = 0;
  for (int s = 0; s < P; ++s) {
    const int x = t + T * s;
    const bool k = valid && z < (int)__ldg(qcut + x * Ny + y) && !(x == 0 && L == 0);
    keep |= (uint32_t)k << s;
  }
  return keep;
}

// ---------------------------------------------------------------------------
// inv_x: lines along x, batch L = y*Mz + z (contiguous), NF = 3 or 6 fields
// ---------------------------------------------------------------------------
template <int NF, typename C = double2>
struct InvXArgs {
  const double2* in[NF];  // the FP64 state
  C* A[NF];
  C* B[NF];
  const uint16_t* qcut;  // [Nx][Ny]: mask(j,k,l) = l < qcut[j*Ny+k], minus (0,0,0)
  const double2* tw;
};

template <int NX, int P, int NF, typename C, int V = 0>
__global__ void __launch_bounds__(kThreads, min_ctas_xy(P)) inv_x_kernel(InvXArgs<NF, C> a, PassGeom g) {
  using S = PassSmem<NX, P, C, double2, V>;
  using F = typename S::F;
  using LM = typename S::LM;
  using Rt = RealOf<C>;
  constexpr int T = F::T;
  extern __shared__ __align__(16) unsigned char dsm[];
  F::load_tw(S::tw(dsm), a.tw);
  const C* tw_s = S::tw(dsm);
  int li, t;
  LM::get(li, t);
  C* sbuf = S::sbuf(dsm, li);
  double2* pf = S::pf(dsm);
  const int nlines = g.Ny * g.Mz;               // lines of one instance
  const int tlines = nlines * nbatch(g);        // lines of all instances
  const int groups = (tlines + LM::LPC - 1) / LM::LPC;
  // line G of the batch: instance G / nlines, line G % nlines of it
  auto line_off = [&](int G) -> size_t {
    const int b = G / nlines;
    return (size_t)b * NX * nlines + (size_t)(G - b * nlines);
  };
  // each CTA takes a contiguous range of groups, so neighbouring lines (which
  // share partially covered 32-byte sectors) are handled back to back
  const GroupRange gr = group_range(groups);
  const int g_end = gr.end;
  int grp = gr.grp;
  if (grp >= g_end) return;  // uniform across the CTA
  uint32_t keep;             // bit s: mode (t + T s, y, z) survives the 2/3 mask
  {
    const int G = grp * LM::LPC + li;
    const bool valid = G < tlines;
    const int Gc = valid ? G : 0;
    const int Lc = Gc % nlines;
    const int y = Lc / g.Mz, z = Lc - y * g.Mz;
    keep = mask_bits<NX>(a.qcut, g.Ny, y, z, Lc, valid, t, T, P);
    issue_line<P, T>(pf, a.in[0], line_off(Gc), (size_t)nlines, t, keep);
    cp_async_commit();
  }
  int ub = 0;
  for (; grp < g_end; grp += gr.step) {
    const int G = grp * LM::LPC + li;
    const bool valid = G < tlines;
    const int Gc = valid ? G : 0;
    const size_t off = line_off(Gc);
    const int gn = grp + gr.step;
    const int Gn = gn * LM::LPC + li;
    const bool validn = Gn < tlines;
    const int Gnc = validn ? Gn : 0;
    const int Lnc = Gnc % nlines;
    uint32_t keep_next = 0;
    if (gn < g_end) {
      const int yn = Lnc / g.Mz, zn = Lnc - yn * g.Mz;
      keep_next = mask_bits<NX>(a.qcut, g.Ny, yn, zn, Lnc, validn, t, T, P);
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      const double2* cur = pf + ub * (P * kThreads);
      double2* nxt = pf + (ub ^ 1) * (P * kThreads);
      if (f + 1 < NF) {
        issue_line<P, T>(nxt, a.in[f + 1], off, (size_t)nlines, t, keep);
      } else if (gn < g_end) {
        issue_line<P, T>(nxt, a.in[0], line_off(Gnc), (size_t)nlines, t, keep_next);
      }
      cp_async_commit();
      cp_async_wait<1>();
      // X (masked) then i kx X, both from the prefetched samples
      C v[P];
#pragma unroll
      for (int s = 0; s < P; ++s) v[s] = cvt<C>(cur[s * kThreads]);
      F::template run<+1, F::PADW, LM::SW>(v, t, sbuf, tw_s);
      if (valid) {
#pragma unroll
        for (int s = 0; s < P; ++s) a.A[f][off + (size_t)(t + T * s) * nlines] = v[s];
      }
#pragma unroll
      for (int s = 0; s < P; ++s) {
        const C u = cvt<C>(cur[s * kThreads]);
        const Rt kx = (Rt)(g.kfx * (double)signed_idx(t + T * s, NX));
        v[s] = mkc<C>(-u.y * kx, u.x * kx);  // i kx u (build_ders_device)
      }
      F::template run<+1, F::PADW, LM::SW>(v, t, sbuf, tw_s);
      if (valid) {
#pragma unroll
        for (int s = 0; s < P; ++s) a.B[f][off + (size_t)(t + T * s) * nlines] = v[s];
      }
      ub ^= 1;
    }
    keep = keep_next;
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// inv_y: lines along y, batch b = x*Mz + z, base = x*Ny*Mz + z, stride Mz
// ---------------------------------------------------------------------------
struct InvYMaps;
template <int NF, typename Cx = double2>
struct InvYArgs {
  const Cx* A[NF];
  const Cx* B[NF];
  Cx* C[NF];
  Cx* D[NF];
  Cx* E[NF];
  const double2* tw;
  // tensor maps over A and B for the bulk-copy form of the nonlinear term's
  // pass (InvYMaps, built for the handle's scratch), or null
  const InvYMaps* maps = nullptr;
  int* err = nullptr;  // error flag of the bulk-copy form's bounded waits
};

template <int NY, int P, int NF, typename C, int V = 0>
__global__ void __launch_bounds__(kThreads, min_ctas_xy(P)) inv_y_kernel(InvYArgs<NF, C> a, PassGeom g) {
  using S = PassSmem<NY, P, C, C, V>;
  using F = typename S::F;
  using LM = typename S::LM;
  using Rt = RealOf<C>;
  constexpr int T = F::T;
  extern __shared__ __align__(16) unsigned char dsm[];
  F::load_tw(S::tw(dsm), a.tw);
  const C* tw_s = S::tw(dsm);
  int li, t;
  LM::get(li, t);
  C* sbuf = S::sbuf(dsm, li);
  C* pf = S::pf(dsm);
  const int nb = g.Nx * g.Mz;
  const int groups = (nb + LM::LPC - 1) / LM::LPC;
  const size_t stride = (size_t)g.Mz;
  const GroupRange gr = group_range(groups);
  const int g_end = gr.end;
  int grp = gr.grp;
  if (grp >= g_end) return;
  auto line_base = [&](int gidx) -> size_t {
    const int b = gidx * LM::LPC + li;
    const int bc = b < nb ? b : 0;
    const int x = bc / g.Mz, z = bc - x * g.Mz;
    return (size_t)x * g.Ny * g.Mz + z;
  };
  issue_line<P, T>(pf, a.A[0], line_base(grp), stride, t);
  cp_async_commit();
  int ub = 0;
  for (; grp < g_end; grp += gr.step) {
    const bool valid = grp * LM::LPC + li < nb;
    const size_t base = line_base(grp);
    const int gn = grp + gr.step;
    const size_t basen = line_base(gn < g_end ? gn : grp);
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      // unit A[f] -> C[f] = IFFT_y A, D[f] = IFFT_y(i ky A)
      {
        const C* cur = pf + ub * (P * kThreads);
        C* nxt = pf + (ub ^ 1) * (P * kThreads);
        issue_line<P, T>(nxt, a.B[f], base, stride, t);
        cp_async_commit();
        cp_async_wait<1>();
        C v[P];
#pragma unroll
        for (int s = 0; s < P; ++s) v[s] = cur[s * kThreads];
        F::template run<+1, F::PADW, LM::SW>(v, t, sbuf, tw_s);
        if (valid) {
#pragma unroll
          for (int s = 0; s < P; ++s) a.C[f][base + (size_t)(t + T * s) * stride] = v[s];
        }
#pragma unroll
        for (int s = 0; s < P; ++s) {
          const C u = cur[s * kThreads];
          const Rt ky = (Rt)(g.kfy * (double)signed_idx(t + T * s, NY));
          v[s] = mkc<C>(-u.y * ky, u.x * ky);
        }
        F::template run<+1, F::PADW, LM::SW>(v, t, sbuf, tw_s);
        if (valid) {
#pragma unroll
          for (int s = 0; s < P; ++s) a.D[f][base + (size_t)(t + T * s) * stride] = v[s];
        }
        ub ^= 1;
      }
      // unit B[f] -> E[f] = IFFT_y B
      {
        const C* cur = pf + ub * (P * kThreads);
        C* nxt = pf + (ub ^ 1) * (P * kThreads);
        if (f + 1 < NF) {
          issue_line<P, T>(nxt, a.A[f + 1], base, stride, t);
        } else if (gn < g_end) {
          issue_line<P, T>(nxt, a.A[0], basen, stride, t);
        }
        cp_async_commit();
        cp_async_wait<1>();
        C v[P];
#pragma unroll
        for (int s = 0; s < P; ++s) v[s] = cur[s * kThreads];
        F::template run<+1, F::PADW, LM::SW>(v, t, sbuf, tw_s);
        if (valid) {
#pragma unroll
          for (int s = 0; s < P; ++s) a.E[f][base + (size_t)(t + T * s) * stride] = v[s];
        }
        ub ^= 1;
      }
    }
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// inv_y fed by bulk tensor copies (TMA), FP64 lines spread over the CTA.
//
// The cp.async form makes every thread issue P 16-byte copies per unit (a
// field of the group's lines): at 12 warps per SM the memory-instruction
// queue saturates (MIO-throttle and long-scoreboard stalls).  Here one thread
// asks the TMA unit for a unit's whole box - the LPC consecutive z lines of
// one x plane, all Ny samples - with one instruction per 256 samples, into a
// ring of NST shared-memory slots whose completions are counted on
// mbarriers; the other threads only wait and read.  A group never straddles
// two x planes: a plane has ceil(Mz / LPC) groups, and the lines past Mz of
// its last group are filled with zeros by the copy and not stored.  In a
// slot, sample y of line li sits at y * LPC + li (the box's own order), so
// the lanes of a load (consecutive li, then t) read consecutive 16-byte
// words.  A slot is refilled only after every thread has passed the CTA
// barrier at the start of the transforms of the unit that used it, and only
// after the issuing thread's own wait for that unit succeeded: a slot's
// barrier never holds two armed phases.  When a wait gives up, the issuer
// stops issuing and, before it returns, drains (with bounded waits) the
// copies it issued and did not see complete.
// ---------------------------------------------------------------------------
// Rows of one box along y: the largest divisor of ny that is at most 256
// (the longest box side a tensor map allows); a unit takes ny / that boxes.
constexpr int tma_box_y(int ny, int b = 256) {
  return b <= 1 ? 1 : (ny % b == 0 ? b : tma_box_y(ny, b - 1));
}

// Tensor maps of one pass: A_f at 2f, B_f at 2f + 1.  Dimensions (2 Mz
// doubles, Ny, planes), box (2 LPC, tma_box_y(Ny), 1).
struct alignas(64) InvYMaps {
  CUtensorMap map[6];
};

template <int NF>
struct alignas(64) InvYTmaArgs {
  InvYMaps m;
  double2* C[NF];
  double2* D[NF];
  double2* E[NF];
  const double2* tw;
  int* err;
};

template <int NY, int P>
struct InvYTmaSmem {
  using F = LineFFT<NY, P>;
  using LM = LaneMap<F::T>;
  static constexpr int LPC = LM::LPC;
  static constexpr int STRIDE = line_stride(F::BUF, xy_stride_target<F::T>());
  static constexpr int BOXY = tma_box_y(NY);
  static constexpr uint32_t SLOT = (uint32_t)NY * LPC * sizeof(double2);
  static constexpr size_t REST = align16((size_t)F::TWLEN * sizeof(double2)) +
                                 align16((size_t)LPC * STRIDE * sizeof(double2)) + 64;
  // ring depth: 3 slots where the CTAs the registers allow still fit, else 2
  static constexpr int NST =
      (3 * (size_t)SLOT + REST) * (size_t)min_ctas_xy(P) <= 227 * 1024 ? 3 : 2;
  static constexpr size_t TW_OFF = (size_t)NST * SLOT;  // slots are 128-byte multiples
  static constexpr size_t SBUF_OFF = TW_OFF + align16((size_t)F::TWLEN * sizeof(double2));
  static constexpr size_t BAR_OFF = SBUF_OFF + align16((size_t)LPC * STRIDE * sizeof(double2));
  static constexpr size_t BAD_OFF = BAR_OFF + 8 * NST;  // the CTA's broken-ring flag
  static constexpr size_t BYTES = BAD_OFF + 8;
  static_assert(SLOT % 128 == 0, "slot alignment");
  static_assert(NY % BOXY == 0 && (BOXY * LPC * sizeof(double2)) % 128 == 0, "box alignment");
  static_assert(BYTES * min_ctas_xy(P) <= 227 * 1024 || min_ctas_xy(P) <= 1, "CTAs per SM");
};

template <int NY, int P, int NF>
__global__ void __launch_bounds__(kThreads, min_ctas_xy(P))
    inv_y_tma_kernel(const __grid_constant__ InvYTmaArgs<NF> a, PassGeom g) {
  using S = InvYTmaSmem<NY, P>;
  using F = typename S::F;
  using LM = typename S::LM;
  static_assert(LM::kSpread, "lines spread over the CTA");
  constexpr int T = F::T, LPC = LM::LPC, NST = S::NST;
  constexpr int UPG = 2 * NF;  // units per group: A_f, B_f
  extern __shared__ __align__(128) unsigned char dsm[];
  double2* tw_s = (double2*)(dsm + S::TW_OFF);
  uint64_t* full = (uint64_t*)(dsm + S::BAR_OFF);
  int li, t;
  LM::get(li, t);
  double2* sbuf = (double2*)(dsm + S::SBUF_OFF) + li * S::STRIDE;
  const int gpp = (g.Mz + LPC - 1) / LPC;  // groups per x plane
  const int groups = g.Nx * gpp;
  const GroupRange gr = group_range(groups);
  if (gr.grp >= gr.end) return;  // uniform across the CTA
  const int ngrp = (gr.end - gr.grp + gr.step - 1) / gr.step;
  const int nunits = ngrp * UPG;
  volatile int* bad = (volatile int*)(dsm + S::BAD_OFF);  // a wait of this CTA gave up
  auto issue = [&](int k) {  // thread 0
    const int gi = k / UPG, j = k - gi * UPG;
    const int grp = gr.grp + gi * gr.step;
    const int x = grp / gpp, z0 = (grp - x * gpp) * LPC;
    unsigned char* dst = dsm + (size_t)(k % NST) * S::SLOT;
    uint64_t* bar = &full[k % NST];
    mbar_expect_tx(bar, S::SLOT);
#pragma unroll
    for (int by = 0; by < NY / S::BOXY; ++by)
      tma_load_3d(dst + (size_t)by * S::BOXY * LPC * sizeof(double2), &a.m.map[j], 2 * z0,
                  by * S::BOXY, x, bar);
  };
  // thread 0: units issued so far, and the first whose completion it did not see
  int issued = 0, unseen = nunits;
  if (threadIdx.x == 0) {
    // a slot ring off its 128-byte alignment: no copies, the host sees the
    // flag at its next synchronisation
    *bad = (smem_u32(dsm) & 127u) != 0u;
    if (*bad && a.err) atomicExch(a.err, kErrTimeout);
    for (int s = 0; s < NST; ++s) mbar_init(&full[s], 1);
    mbar_init_fence();
    // the first copies start before the twiddle table is read
    if (!*bad)
      for (; issued < NST - 1 && issued < nunits; ++issued) issue(issued);
  }
  F::load_tw(tw_s, a.tw);  // ends with a CTA barrier: the barriers are initialised
  if (*bad) return;        // uniform: read after the barrier
  for (int k = 0; k < nunits; ++k) {
    if (threadIdx.x == 0 && unseen == nunits && k + NST - 1 < nunits) {
      fence_proxy_async_smem();  // the slot's earlier reads (generic proxy) come first
      issue(k + NST - 1);
      issued = k + NST;
    }
    const bool seen = mbar_wait(&full[k % NST], (uint32_t)((k / NST) & 1), a.err, bad);
    if (threadIdx.x == 0 && !seen && unseen == nunits) unseen = k;
    const double2* cur = (const double2*)(dsm + (size_t)(k % NST) * S::SLOT) + li;
    const int gi = k / UPG, j = k - gi * UPG, f = j >> 1;
    const int grp = gr.grp + gi * gr.step;
    const int x = grp / gpp, z = (grp - x * gpp) * LPC + li;
    const bool valid = z < g.Mz;
    const size_t base = (size_t)x * g.Ny * g.Mz + (valid ? z : 0);
    const size_t stride = (size_t)g.Mz;
    double2 v[P];
#pragma unroll
    for (int s = 0; s < P; ++s) v[s] = cur[(t + T * s) * LPC];
    F::template run<+1, F::PADW, LM::SW>(v, t, sbuf, tw_s);
    if ((j & 1) == 0) {
      // unit A_f -> C_f = IFFT_y A, D_f = IFFT_y(i ky A)
      if (valid) {
#pragma unroll
        for (int s = 0; s < P; ++s) a.C[f][base + (size_t)(t + T * s) * stride] = v[s];
      }
#pragma unroll
      for (int s = 0; s < P; ++s) {
        const double2 u = cur[(t + T * s) * LPC];
        const double ky = g.kfy * (double)signed_idx(t + T * s, NY);
        v[s] = make_double2(-u.y * ky, u.x * ky);
      }
      F::template run<+1, F::PADW, LM::SW>(v, t, sbuf, tw_s);
      if (valid) {
#pragma unroll
        for (int s = 0; s < P; ++s) a.D[f][base + (size_t)(t + T * s) * stride] = v[s];
      }
    } else {
      // unit B_f -> E_f = IFFT_y B
      if (valid) {
#pragma unroll
        for (int s = 0; s < P; ++s) a.E[f][base + (size_t)(t + T * s) * stride] = v[s];
      }
    }
  }
  if (threadIdx.x == 0)  // a broken ring: the copies that may still be in flight
    for (int k = unseen; k < issued; ++k) mbar_drain(&full[k % NST], (uint32_t)((k / NST) & 1));
}

// ---------------------------------------------------------------------------
// z pass: lines along z (contiguous), batch b = x*Ny + y, base = b*Mz
// ---------------------------------------------------------------------------
template <int NF, typename Cx = double2>
struct ZArgs {
  // per velocity field (u, then v for the tangent form) and component:
  const Cx* C[NF];  // IFFT_xy(M u_i)
  const Cx* D[NF];  // IFFT_xy(i ky M u_i)
  const Cx* E[NF];  // IFFT_xy(i kx M u_i)
  Cx* Qh[3];        // R2C_z of the products (x, y still physical)
  const double2* tw;
};

// L2 prefetch of one contiguous run (16-byte aligned, a multiple of 16 bytes)
// by the bulk-copy unit: no registers, no shared memory, nothing to wait for.
__device__ __forceinline__ void prefetch_l2_bulk(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}

// L2 prefetch of the z pass's input (NS3D_Z_L2PF): 0 none; 1 the CTA's nine
// input runs (one contiguous run of LPC lines per field) at kernel start, in
// the order the transforms read them; 2 each transform's two runs one
// transform ahead (the bulk-copy unit fetches them while the current
// transform runs, and the loads then hit L2).  Measured on a B200 (z pass per
// launch, 256^3 / 128^3 FP64): none 503 / 80.4 us, 1: 462 / 81 us, 2: 439 /
// 67.5 us (two repeats each, within 0.5%).
#ifndef NS3D_Z_L2PF
#define NS3D_Z_L2PF 2
#endif

// L2 prefetch of a CTA's `nv` consecutive z lines (from element run0) of one
// field: one contiguous run, trimmed to 16-byte boundaries inside it (FP32
// rows of an odd Mz start at 8-byte offsets).
template <typename C>
__device__ __forceinline__ void prefetch_z_run(const C* f, size_t run0, int nv, int Mz) {
  const uintptr_t a = (uintptr_t)(f + run0) & ~(uintptr_t)15;
  const uintptr_t e = (uintptr_t)(f + run0 + (size_t)nv * Mz) & ~(uintptr_t)15;
  if (e > a) prefetch_l2_bulk((const void*)a, (unsigned)(e - a));
}

// The CTA's runs of one z pass: lines b0 .. b0 + nv - 1 of every field.
struct ZRun {
  size_t run0;
  int nv, Mz;
};
__device__ __forceinline__ ZRun z_run(int lpc, int nb, int Mz) {
  const int b0 = blockIdx.x * lpc;
  return {(size_t)b0 * Mz, nb - b0 < lpc ? nb - b0 : lpc, Mz};
}
// the next transform's two input runs (threads 0 and 1 ask the bulk-copy unit)
template <typename C>
__device__ __forceinline__ void prefetch_z_pair(const C* f1, const C* f2, const ZRun& r) {
  if (NS3D_Z_L2PF == 0) return;
  if (threadIdx.x == 0) prefetch_z_run(f1, r.run0, r.nv, r.Mz);
  if (threadIdx.x == 1 && f2 != f1) prefetch_z_run(f2, r.run0, r.nv, r.Mz);
}

// Load W[k] = H(X1)[k] + i H(X2)[k] for positions k = t + T s, where H is the
// Hermitian extension of a z half-line (H[0], H[N/2] keep only real parts),
// X = line (optionally times i kz).
template <int NZ, int P, bool IK1, bool IK2, typename C>
__device__ __forceinline__ void load_pair(C (&w)[P], const C* __restrict__ f1,
                                          const C* __restrict__ f2, size_t base, int t,
                                          RealOf<C> kfz) {
  using Rt = RealOf<C>;
  constexpr int T = NZ / P;
#pragma unroll
  for (int s = 0; s < P; ++s) {
    const int k = t + T * s;
    const bool upper = k > NZ / 2;
    const int q = upper ? NZ - k : k;
    C c1 = __ldg(f1 + base + q);
    C c2 = __ldg(f2 + base + q);
    const Rt kz = kfz * (Rt)q;
    if constexpr (IK1) c1 = mkc<C>(-c1.y * kz, c1.x * kz);
    if constexpr (IK2) c2 = mkc<C>(-c2.y * kz, c2.x * kz);
    if (k == 0 || k == NZ / 2) {
      c1.y = (Rt)0;
      c2.y = (Rt)0;
    }
    if (upper) {
      c1.y = -c1.y;
      c2.y = -c2.y;
    }
    w[s] = mkc<C>(c1.x - c2.y, c1.y + c2.x);
  }
}

// w holds FFT_z(Q1 + i Q2) at k = t + T s.  Split it with the mirror bin
// W[N-k] (exchanged through shared memory) and store the half spectra
// Q1h[k], Q2h[k] for k = 0..N/2.
// Line-buffer index scheme of the z pass: the XOR swizzle for FP32 lines of
// 128 points and more (fewer shared-memory wavefronts), the padding else.
template <int NZ, int P, typename C>
__host__ __device__ constexpr int z_pw() {
  return (sizeof(C) == 8 && P == 8 && (NZ & (NZ - 1)) == 0 && NZ >= 128)
             ? 0 : LineFFT<NZ, P>::PADW;
}

template <int NZ, int P, typename C>
__device__ __forceinline__ void store_pair_spectrum(const C (&w)[P], C* sbuf, int t,
                                                    C* __restrict__ o1,
                                                    C* __restrict__ o2, size_t base,
                                                    bool valid) {
  using Rt = RealOf<C>;
  using F = LineFFT<NZ, P>;
  constexpr int T = F::T;
  line_sync<T>();
#pragma unroll
  for (int s = 0; s < P; ++s) sbuf[spad<z_pw<NZ, P, C>()>(t + T * s)] = w[s];
  line_sync<T>();
#pragma unroll
  for (int s = 0; s < P; ++s) {
    const int k = t + T * s;
    if (k <= NZ / 2 && valid) {
      const C a = w[s];
      const C m = sbuf[spad<z_pw<NZ, P, C>()>(k == 0 ? 0 : NZ - k)];
      o1[base + k] = mkc<C>((Rt)0.5 * (a.x + m.x), (Rt)0.5 * (a.y - m.y));
      o2[base + k] = mkc<C>((Rt)0.5 * (a.y + m.y), (Rt)-0.5 * (a.x - m.x));
    }
  }
}

template <int T>
struct ZLaneMap {  // lanes of one line are adjacent: the line is contiguous in memory
  static constexpr int LPW = T <= 32 ? 32 / T : 1;
  static constexpr int LPC = T <= 32 ? kWarpsPerCta * LPW : (kWarpsPerCta * 32) / T;
  __device__ __forceinline__ static void get(int& li, int& t) {
    if constexpr (T <= 32) {
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
      t = lane % T;
      li = warp * LPW + lane / T;
    } else {
      t = threadIdx.x % T;
      li = threadIdx.x / T;
    }
  }
};

// One component of B(u,v)_i = (v.grad) u_i + (u.grad) v_i in the z pass
// (convolute_2p3_UV, Source/advection_2_3.cu:414-466); 3 paired C2R lines.
template <int NZ, int P, typename C, typename Rt = RealOf<C>>
__device__ __forceinline__ void uv_component(Rt (&q)[P], int i, const ZArgs<6, C>& a, size_t base,
                                             int t, Rt kfz, Rt sc, C* sbuf,
                                             const C* tw_s, const Rt (&ux)[P],
                                             const Rt (&uy)[P], const Rt (&uz)[P],
                                             const Rt (&vx)[P], const Rt (&vy)[P],
                                             const Rt (&vz)[P], const ZRun& run) {
  using F = LineFFT<NZ, P>;
  C w[P];
  // (d_x u_i, d_y u_i)
  prefetch_z_pair(a.C[i], a.E[3 + i], run);
  load_pair<NZ, P, false, false>(w, a.E[i], a.D[i], base, t, kfz);
  F::template run<+1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
#pragma unroll
  for (int s = 0; s < P; ++s) q[s] = vx[s] * (w[s].x * sc) + vy[s] * (w[s].y * sc);
  // (d_z u_i, d_x v_i)
  prefetch_z_pair(a.D[3 + i], a.C[3 + i], run);
  load_pair<NZ, P, true, false>(w, a.C[i], a.E[3 + i], base, t, kfz);
  F::template run<+1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
#pragma unroll
  for (int s = 0; s < P; ++s) {
    q[s] = q[s] + vz[s] * (w[s].x * sc);
    q[s] = q[s] + ux[s] * (w[s].y * sc);
  }
  // (d_y v_i, d_z v_i)
  if (i < 2) prefetch_z_pair(a.E[i + 1], a.D[i + 1], run);
  load_pair<NZ, P, false, true>(w, a.D[3 + i], a.C[3 + i], base, t, kfz);
  F::template run<+1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
#pragma unroll
  for (int s = 0; s < P; ++s) q[s] = q[s] + (uy[s] * (w[s].x * sc) + uz[s] * (w[s].y * sc));
}

template <int NZ, int P, bool UV, typename C>
__global__ void __launch_bounds__(kWarpsPerCta * 32, kMinCtasZ) z_kernel(ZArgs<UV ? 6 : 3, C> a, PassGeom g) {
  using F = LineFFT<NZ, P>;
  using Rt = RealOf<C>;
  constexpr int T = F::T;
  using LM = ZLaneMap<T>;
  __shared__ C tw_s[F::TWLEN];
  __shared__ C sbuf_all[LM::LPC][F::BUF];
  F::load_tw(tw_s, a.tw);
  int li, t;
  LM::get(li, t);
  const int nb = g.Nx * g.Ny;
  const int b = blockIdx.x * LM::LPC + li;
  const bool valid = b < nb;
  const size_t base = (size_t)(valid ? b : 0) * g.Mz;
  C* sbuf = sbuf_all[li];
  const Rt sc = (Rt)g.inv_vol;
  const Rt kfz = (Rt)g.kfz;
  const ZRun run = z_run(LM::LPC, nb, g.Mz);  // one transform ahead into L2
  C w[P];
  Rt ux[P], uy[P], uz[P], q0[P], q1[P], q2[P];
  if constexpr (!UV) {
    // Q_z first, so at most five real lines (u_x, u_y, u_z and two products)
    // are live at any time.
    // (u_x, u_y)
    prefetch_z_pair(a.C[2], a.C[2], run);
    load_pair<NZ, P, false, false>(w, a.C[0], a.C[1], base, t, kfz);
    F::template run<+1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s) { ux[s] = w[s].x * sc; uy[s] = w[s].y * sc; }
    // (u_z, d_z u_z) from one field
    prefetch_z_pair(a.E[2], a.D[2], run);
    load_pair<NZ, P, false, true>(w, a.C[2], a.C[2], base, t, kfz);
    F::template run<+1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s) { uz[s] = w[s].x * sc; q2[s] = w[s].y * sc; }
    // Q_z = u_x d_x u_z + u_y d_y u_z + u_z d_z u_z  (calc_vels_nabla_vels)
    prefetch_z_pair(a.E[0], a.D[0], run);
    load_pair<NZ, P, false, false>(w, a.E[2], a.D[2], base, t, kfz);
    F::template run<+1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s)
      q2[s] = ux[s] * (w[s].x * sc) + uy[s] * (w[s].y * sc) + uz[s] * q2[s];
    // R2C of Q_z alone
#pragma unroll
    for (int s = 0; s < P; ++s) w[s] = mkc<C>(q2[s], (Rt)0);
    F::template run<-1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
    if (valid) {
#pragma unroll
      for (int s = 0; s < P; ++s) {
        const int k = t + T * s;
        if (k <= NZ / 2) a.Qh[2][base + k] = w[s];
      }
    }
    // (d_z u_x, d_z u_y)
    load_pair<NZ, P, true, true>(w, a.C[0], a.C[1], base, t, kfz);
    F::template run<+1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s) { q0[s] = w[s].x * sc; q1[s] = w[s].y * sc; }
    prefetch_z_pair(a.E[1], a.D[1], run);
    load_pair<NZ, P, false, false>(w, a.E[0], a.D[0], base, t, kfz);
    F::template run<+1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s)
      q0[s] = ux[s] * (w[s].x * sc) + uy[s] * (w[s].y * sc) + uz[s] * q0[s];
    load_pair<NZ, P, false, false>(w, a.E[1], a.D[1], base, t, kfz);
    F::template run<+1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s)
      q1[s] = ux[s] * (w[s].x * sc) + uy[s] * (w[s].y * sc) + uz[s] * q1[s];
    // R2C of (Q_x, Q_y) packed
#pragma unroll
    for (int s = 0; s < P; ++s) w[s] = mkc<C>(q0[s], q1[s]);
    F::template run<-1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
    store_pair_spectrum<NZ, P>(w, sbuf, t, a.Qh[0], a.Qh[1], base, valid);
    return;
  } else {
    // B(u,v)_i = (v.grad) u_i + (u.grad) v_i; fields 0..2 are u, 3..5 are v
    Rt vx[P], vy[P], vz[P];
    prefetch_z_pair(a.C[2], a.C[3], run);
    load_pair<NZ, P, false, false>(w, a.C[0], a.C[1], base, t, kfz);
    F::template run<+1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s) { ux[s] = w[s].x * sc; uy[s] = w[s].y * sc; }
    prefetch_z_pair(a.C[4], a.C[5], run);
    load_pair<NZ, P, false, false>(w, a.C[2], a.C[3], base, t, kfz);
    F::template run<+1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s) { uz[s] = w[s].x * sc; vx[s] = w[s].y * sc; }
    prefetch_z_pair(a.E[0], a.D[0], run);
    load_pair<NZ, P, false, false>(w, a.C[4], a.C[5], base, t, kfz);
    F::template run<+1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s) { vy[s] = w[s].x * sc; vz[s] = w[s].y * sc; }
    uv_component<NZ, P>(q0, 0, a, base, t, kfz, sc, sbuf, tw_s, ux, uy, uz, vx, vy, vz, run);
    uv_component<NZ, P>(q1, 1, a, base, t, kfz, sc, sbuf, tw_s, ux, uy, uz, vx, vy, vz, run);
    uv_component<NZ, P>(q2, 2, a, base, t, kfz, sc, sbuf, tw_s, ux, uy, uz, vx, vy, vz, run);
  }
  // forward R2C along z: (Q0, Q1) packed, then Q2 alone
#pragma unroll
  for (int s = 0; s < P; ++s) w[s] = mkc<C>(q0[s], q1[s]);
  F::template run<-1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
  store_pair_spectrum<NZ, P>(w, sbuf, t, a.Qh[0], a.Qh[1], base, valid);
#pragma unroll
  for (int s = 0; s < P; ++s) w[s] = mkc<C>(q2[s], (Rt)0);
  F::template run<-1, z_pw<NZ, P, C>()>(w, t, sbuf, tw_s);
  if (valid) {
#pragma unroll
    for (int s = 0; s < P; ++s) {
      const int k = t + T * s;
      if (k <= NZ / 2) a.Qh[2][base + k] = w[s];
    }
  }
}

// ---------------------------------------------------------------------------
// z pass with the physical velocities stashed in shared memory (the nonlinear
// term; the tangent form keeps z_kernel).
//
// The line transforms are what bound the z pass: each Stockham exchange moves
// the whole line through shared memory, so at 8 points per thread a 256-point
// line takes two exchanges per transform (16 per line and pass) and the
// shared-memory pipe, not HBM, sets the pace.  With 16 points per thread the
// same transform needs one exchange, but u_x, u_y, u_z, two products and the
// line no longer fit in registers.  Here each thread parks its own P samples
// of u_x, u_y, u_z in a private shared-memory slot ([component][s][thread]:
// the lanes of a warp touch consecutive words, conflict-free) right after
// their transforms and reads them back for each product; no other thread
// reads them, so no barrier is needed.  The arithmetic of every product is
// the one z_kernel does.
// ---------------------------------------------------------------------------
template <int NZ, int P, typename C>
struct ZStashSmem {
  using F = LineFFT<NZ, P>;
  using LM = ZLaneMap<F::T>;
  using Rt = RealOf<C>;
  static constexpr size_t SBUF_OFF = align16((size_t)F::TWLEN * sizeof(C));
  static constexpr size_t ST_OFF = align16(SBUF_OFF + (size_t)LM::LPC * F::BUF * sizeof(C));
  static constexpr size_t BYTES = ST_OFF + (size_t)3 * P * kThreads * sizeof(Rt);
  static_assert(BYTES <= 113 * 1024, "two CTAs per SM");
  // The TMEM form (NS3D_Z_TMEM) keeps the stash in tensor memory instead:
  // TM_COLS columns per CTA (3 P doubles per thread = 6 P words, rounded up
  // to a power of two).  Its launch asks for at least TM_BYTES of shared
  // memory, which caps the CTAs per SM that hold columns at
  // kTmemColsPerSm / TM_COLS, so an allocation never waits for good.
  static constexpr uint32_t TM_COLS = 6 * P <= 32 ? 32 : (6 * P <= 64 ? 64 : (6 * P <= 128 ? 128 : 256));
  static constexpr int TM_MAXCTAS = (int)(kTmemColsPerSm / TM_COLS);
  static constexpr size_t TM_BYTES =
      BYTES > (228 * 1024) / (TM_MAXCTAS + 1) + 1 ? BYTES : (228 * 1024) / (TM_MAXCTAS + 1) + 1;
  static_assert(sizeof(Rt) == 8, "the TMEM form holds FP64 stash words in pairs");
  static_assert(P % 4 == 0 && 6 * P <= 256, "TMEM stash columns");
  static_assert((TM_BYTES + 1024) * (TM_MAXCTAS + 1) > 228 * 1024, "CTAs per SM bound");
};

// Where the nonlinear term's z pass keeps its velocity stash: 0 in shared
// memory, 1 in tensor memory, 2 in tensor memory for z extents from 512.
// Measured on a B200 (z pass per launch, shared / tensor memory): 128^3
// 69.4 / 71.5 us, 256^3 453.5 / 457 us, 512^3 4553 / 4453 us.
#ifndef NS3D_Z_TMEM
#define NS3D_Z_TMEM 2
#endif
__host__ __device__ constexpr bool z_tmem(int nz) {
  return NS3D_Z_TMEM == 1 || (NS3D_Z_TMEM == 2 && nz >= 512);
}

template <int NZ, int P, typename C, bool TM = false>
__global__ void __launch_bounds__(kThreads, kMinCtasZ) z_kernel_st(ZArgs<3, C> a, PassGeom g) {
  using F = LineFFT<NZ, P>;
  using Rt = RealOf<C>;
  using S = ZStashSmem<NZ, P, C>;
  constexpr int T = F::T;
  using LM = ZLaneMap<T>;
  constexpr int PW = z_pw<NZ, P, C>();
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ uint32_t tm_base_s;  // TMEM address of the CTA's columns (TM)
  const int warp = threadIdx.x >> 5;
  if constexpr (TM) {
    if (warp == 0) tmem_alloc_warp(&tm_base_s, S::TM_COLS);
    tmem_fence_before_sync();
  }
  C* tw_s = (C*)dsm;
  F::load_tw(tw_s, a.tw);  // ends with a CTA barrier: the TMEM address is published
  uint32_t tm = 0;         // this warp's lane quarter, column 0
  if constexpr (TM) {
    tmem_fence_after_sync();
    tm = tmem_addr(tm_base_s, 32 * (warp & 3), 0);
  }
  int li, t;
  LM::get(li, t);
  const int nb = g.Nx * g.Ny;
  const int b = blockIdx.x * LM::LPC + li;
  const bool valid = b < nb;
  const size_t base = (size_t)(valid ? b : 0) * g.Mz;
  C* sbuf = (C*)(dsm + S::SBUF_OFF) + li * F::BUF;
  Rt* stash = (Rt*)(dsm + S::ST_OFF) + threadIdx.x;
  // the CTA's lines are consecutive: each field's input is one run
  const ZRun run = z_run(LM::LPC, nb, g.Mz);
  const C* order[9] = {a.C[0], a.C[1], a.C[2], a.E[2], a.D[2], a.E[0], a.D[0], a.E[1], a.D[1]};
  auto pf = [&](int i) {
    if (NS3D_Z_L2PF != 0 && i < 9) prefetch_z_run(order[i], run.run0, run.nv, run.Mz);
  };
  if (NS3D_Z_L2PF == 1 && threadIdx.x < 9) pf(threadIdx.x);
  if (NS3D_Z_L2PF == 2 && threadIdx.x < 2) pf(threadIdx.x);  // C0, C1
  auto ux = [&](int s) -> Rt& { return stash[(0 * P + s) * kThreads]; };
  auto uy = [&](int s) -> Rt& { return stash[(1 * P + s) * kThreads]; };
  auto uz = [&](int s) -> Rt& { return stash[(2 * P + s) * kThreads]; };
  // stash component c (0 u_x, 1 u_y, 2 u_z): the P values v(s)
  auto park = [&](int c, auto v) {
    if constexpr (TM) {
#pragma unroll
      for (int s0 = 0; s0 < P; s0 += 4) {
        uint32_t r[8];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const double d = v(s0 + k);
          r[2 * k] = (uint32_t)__double2loint(d);
          r[2 * k + 1] = (uint32_t)__double2hiint(d);
        }
        tmem_st8(tm + (uint32_t)(c * 2 * P + 2 * s0), r);
      }
      tmem_wait_st();
    } else {
#pragma unroll
      for (int s = 0; s < P; ++s) stash[(c * P + s) * kThreads] = v(s);
    }
  };
  const Rt sc = (Rt)g.inv_vol;
  const Rt kfz = (Rt)g.kfz;
  C w[P];
  Rt q0[P], q1[P];
  // q[s] = u_x(s) (w[s].x sc) + u_y(s) (w[s].y sc) + u_z(s) q[s]  (calc_vels_nabla_vels)
  auto product = [&](Rt (&q)[P]) {
    if constexpr (TM) {
#pragma unroll
      for (int s0 = 0; s0 < P; s0 += 4) {
        uint32_t rx[8], ry[8], rz[8];
        tmem_ld8(tm + (uint32_t)(0 * 2 * P + 2 * s0), rx);
        tmem_ld8(tm + (uint32_t)(1 * 2 * P + 2 * s0), ry);
        tmem_ld8(tm + (uint32_t)(2 * 2 * P + 2 * s0), rz);
        tmem_wait_ld();
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int s = s0 + k;
          const Rt vx = __hiloint2double((int)rx[2 * k + 1], (int)rx[2 * k]);
          const Rt vy = __hiloint2double((int)ry[2 * k + 1], (int)ry[2 * k]);
          const Rt vz = __hiloint2double((int)rz[2 * k + 1], (int)rz[2 * k]);
          q[s] = vx * (w[s].x * sc) + vy * (w[s].y * sc) + vz * q[s];
        }
      }
    } else {
#pragma unroll
      for (int s = 0; s < P; ++s)
        q[s] = ux(s) * (w[s].x * sc) + uy(s) * (w[s].y * sc) + uz(s) * q[s];
    }
  };
  // (u_x, u_y)
  if (NS3D_Z_L2PF == 2 && threadIdx.x == 0) pf(2);  // C2
  load_pair<NZ, P, false, false>(w, a.C[0], a.C[1], base, t, kfz);
  F::template run<+1, PW>(w, t, sbuf, tw_s);
  park(0, [&](int s) { return w[s].x * sc; });
  park(1, [&](int s) { return w[s].y * sc; });
  // (u_z, d_z u_z); q0 accumulates Q_z first
  if (NS3D_Z_L2PF == 2 && threadIdx.x < 2) pf(3 + threadIdx.x);  // E2, D2
  load_pair<NZ, P, false, true>(w, a.C[2], a.C[2], base, t, kfz);
  F::template run<+1, PW>(w, t, sbuf, tw_s);
  park(2, [&](int s) { return w[s].x * sc; });
#pragma unroll
  for (int s = 0; s < P; ++s) q0[s] = w[s].y * sc;
  // Q_z = u_x d_x u_z + u_y d_y u_z + u_z d_z u_z
  if (NS3D_Z_L2PF == 2 && threadIdx.x < 2) pf(5 + threadIdx.x);  // E0, D0
  load_pair<NZ, P, false, false>(w, a.E[2], a.D[2], base, t, kfz);
  F::template run<+1, PW>(w, t, sbuf, tw_s);
  product(q0);
  // R2C of Q_z alone
#pragma unroll
  for (int s = 0; s < P; ++s) w[s] = mkc<C>(q0[s], (Rt)0);
  F::template run<-1, PW>(w, t, sbuf, tw_s);
  if (valid) {
#pragma unroll
    for (int s = 0; s < P; ++s) {
      const int k = t + T * s;
      if (k <= NZ / 2) a.Qh[2][base + k] = w[s];
    }
  }
  // (d_z u_x, d_z u_y)
  load_pair<NZ, P, true, true>(w, a.C[0], a.C[1], base, t, kfz);
  F::template run<+1, PW>(w, t, sbuf, tw_s);
#pragma unroll
  for (int s = 0; s < P; ++s) { q0[s] = w[s].x * sc; q1[s] = w[s].y * sc; }
  if (NS3D_Z_L2PF == 2 && threadIdx.x < 2) pf(7 + threadIdx.x);  // E1, D1
  load_pair<NZ, P, false, false>(w, a.E[0], a.D[0], base, t, kfz);
  F::template run<+1, PW>(w, t, sbuf, tw_s);
  product(q0);
  load_pair<NZ, P, false, false>(w, a.E[1], a.D[1], base, t, kfz);
  F::template run<+1, PW>(w, t, sbuf, tw_s);
  product(q1);
  // R2C of (Q_x, Q_y) packed
#pragma unroll
  for (int s = 0; s < P; ++s) w[s] = mkc<C>(q0[s], q1[s]);
  F::template run<-1, PW>(w, t, sbuf, tw_s);
  store_pair_spectrum<NZ, P>(w, sbuf, t, a.Qh[0], a.Qh[1], base, valid);
  if constexpr (TM) {
    // every thread's TMEM reads have completed (waited); free the columns
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    if (warp == 0) tmem_dealloc_warp(tm_base_s, S::TM_COLS);
  }
}

// ---------------------------------------------------------------------------
// fwd_y: in-place forward transform along y of the 3 product spectra
// ---------------------------------------------------------------------------
template <typename Cx = double2>
struct FwdYArgs {
  Cx* Q[3];
  const double2* tw;
};

template <int NY, int P, typename C, int V = 0>
__global__ void __launch_bounds__(kThreads, min_ctas_xy(P)) fwd_y_kernel(FwdYArgs<C> a, PassGeom g) {
  using S = PassSmem<NY, P, C, C, V>;
  using F = typename S::F;
  using LM = typename S::LM;
  constexpr int T = F::T;
  extern __shared__ __align__(16) unsigned char dsm[];
  F::load_tw(S::tw(dsm), a.tw);
  const C* tw_s = S::tw(dsm);
  int li, t;
  LM::get(li, t);
  C* sbuf = S::sbuf(dsm, li);
  C* pf = S::pf(dsm);
  const int nb = g.Nx * g.Mz;
  const int groups = (nb + LM::LPC - 1) / LM::LPC;
  const size_t stride = (size_t)g.Mz;
  const GroupRange gr = group_range(groups);
  const int g_end = gr.end;
  int grp = gr.grp;
  if (grp >= g_end) return;
  auto line_base = [&](int gidx) -> size_t {
    const int b = gidx * LM::LPC + li;
    const int bc = b < nb ? b : 0;
    const int x = bc / g.Mz, z = bc - x * g.Mz;
    return (size_t)x * g.Ny * g.Mz + z;
  };
  issue_line<P, T>(pf, a.Q[0], line_base(grp), stride, t);
  cp_async_commit();
  int ub = 0;
  for (; grp < g_end; grp += gr.step) {
    const bool valid = grp * LM::LPC + li < nb;
    const size_t base = line_base(grp);
    const int gn = grp + gr.step;
    const size_t basen = line_base(gn < g_end ? gn : grp);
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const C* cur = pf + ub * (P * kThreads);
      C* nxt = pf + (ub ^ 1) * (P * kThreads);
      if (f + 1 < 3) {
        issue_line<P, T>(nxt, a.Q[f + 1], base, stride, t);
      } else if (gn < g_end) {
        issue_line<P, T>(nxt, a.Q[0], basen, stride, t);
      }
      cp_async_commit();
      cp_async_wait<1>();
      C v[P];
#pragma unroll
      for (int s = 0; s < P; ++s) v[s] = cur[s * kThreads];
      F::template run<-1, F::PADW, LaneMap<T>::SW>(v, t, sbuf, tw_s);
      if (valid) {
#pragma unroll
        for (int s = 0; s < P; ++s) a.Q[f][base + (size_t)(t + T * s) * stride] = v[s];
      }
      ub ^= 1;
    }
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// Plain 3-D transforms of one field (FFTN_Device / iFFTN_Device,
// Source/math_support.cu:301-334): no mask, no derivatives.
//
// line_kernel: one complex line pass, lines along x (AXIS 0: batch
// L = y*Mz + z, stride Ny*Mz) or y (AXIS 1: batch b = x*Mz + z, base
// x*Ny*Mz + z, stride Mz); `out` may alias `in` (every line is read before it
// is written, and the prefetch only touches lines of later groups).
// ---------------------------------------------------------------------------
struct LineArgs {
  const double2* in;
  double2* out;
  const double2* tw;
};

template <int N, int P, int AXIS, int DIR>
__global__ void __launch_bounds__(kThreads, kMinCtasXY) line_kernel(LineArgs a, PassGeom g) {
  using S = PassSmem<N, P>;
  using F = typename S::F;
  using LM = typename S::LM;
  constexpr int T = F::T;
  extern __shared__ __align__(16) unsigned char dsm[];
  F::load_tw(S::tw(dsm), a.tw);
  const double2* tw_s = S::tw(dsm);
  int li, t;
  LM::get(li, t);
  double2* sbuf = S::sbuf(dsm, li);
  double2* pf = S::pf(dsm);
  const int nb = AXIS == 0 ? g.Ny * g.Mz : g.Nx * g.Mz;
  const size_t stride = AXIS == 0 ? (size_t)g.Ny * g.Mz : (size_t)g.Mz;
  const int groups = (nb + LM::LPC - 1) / LM::LPC;
  const GroupRange gr = group_range(groups);
  int grp = gr.grp;
  if (grp >= gr.end) return;
  auto line_base = [&](int gidx) -> size_t {
    const int b = gidx * LM::LPC + li;
    const int bc = b < nb ? b : 0;
    if (AXIS == 0) return (size_t)bc;
    const int x = bc / g.Mz, z = bc - x * g.Mz;
    return (size_t)x * g.Ny * g.Mz + z;
  };
  issue_line<P, T>(pf, a.in, line_base(grp), stride, t);
  cp_async_commit();
  int ub = 0;
  for (; grp < gr.end; grp += gr.step) {
    const bool valid = grp * LM::LPC + li < nb;
    const size_t base = line_base(grp);
    const int gn = grp + gr.step;
    const double2* cur = pf + ub * (P * kThreads);
    double2* nxt = pf + (ub ^ 1) * (P * kThreads);
    if (gn < gr.end) issue_line<P, T>(nxt, a.in, line_base(gn), stride, t);
    cp_async_commit();
    cp_async_wait<1>();
    double2 v[P];
#pragma unroll
    for (int s = 0; s < P; ++s) v[s] = cur[s * kThreads];
    F::template run<DIR, F::PADW, LM::SW>(v, t, sbuf, tw_s);
    if (valid) {
#pragma unroll
      for (int s = 0; s < P; ++s) a.out[base + (size_t)(t + T * s) * stride] = v[s];
    }
    ub ^= 1;
  }
  cp_async_wait<0>();
}

// z passes of the plain transforms: two z lines b and b + nb/2 of one field
// share one complex FFT (nb = Nx*Ny, even for every compiled extent).
struct ZPlainArgs {
  const double2* cin;  // complex [nb][Mz] (C2R input)
  const double* rin;   // real [nb][Nz]   (R2C input)
  double2* cout;       // complex [nb][Mz] (R2C output)
  double* rout;        // real [nb][Nz]   (C2R output)
  double scale;        // C2R output factor: 1/(Nx Ny Nz) or 1
  const double2* tw;
};

// C2R along z times `scale`: the Hermitian extension of each
// half line keeps only the real part of its kz = 0 and kz = Nz/2 bins (what
// cufftExecZ2D does with the non-Hermitian planes the reference produces).
template <int NZ, int P>
__global__ void __launch_bounds__(kWarpsPerCta * 32, kMinCtasZ) z_c2r_kernel(ZPlainArgs a,
                                                                              PassGeom g) {
  using F = LineFFT<NZ, P>;
  constexpr int T = F::T;
  using LM = ZLaneMap<T>;
  __shared__ double2 tw_s[F::TWLEN];
  __shared__ double2 sbuf_all[LM::LPC][F::BUF];
  F::load_tw(tw_s, a.tw);
  int li, t;
  LM::get(li, t);
  const int half = (g.Nx * g.Ny) >> 1;
  const int p = blockIdx.x * LM::LPC + li;
  const bool valid = p < half;
  const int pc = valid ? p : 0;
  double2* sbuf = sbuf_all[li];
  double2 w[P];
#pragma unroll
  for (int s = 0; s < P; ++s) {
    const int k = t + T * s;
    const bool upper = k > NZ / 2;
    const int q = upper ? NZ - k : k;
    double2 c1 = __ldg(a.cin + (size_t)pc * g.Mz + q);
    double2 c2 = __ldg(a.cin + (size_t)(pc + half) * g.Mz + q);
    if (k == 0 || k == NZ / 2) {
      c1.y = 0.0;
      c2.y = 0.0;
    }
    if (upper) {
      c1.y = -c1.y;
      c2.y = -c2.y;
    }
    w[s] = make_double2(c1.x - c2.y, c1.y + c2.x);
  }
  F::template run<+1>(w, t, sbuf, tw_s);
  if (valid) {
    const double sc = a.scale;
#pragma unroll
    for (int s = 0; s < P; ++s) {
      const int k = t + T * s;
      a.rout[(size_t)pc * NZ + k] = w[s].x * sc;
      a.rout[(size_t)(pc + half) * NZ + k] = w[s].y * sc;
    }
  }
}

// R2C along z (unnormalised), the half spectra k = 0..Nz/2.
template <int NZ, int P>
__global__ void __launch_bounds__(kWarpsPerCta * 32, kMinCtasZ) z_r2c_kernel(ZPlainArgs a,
                                                                              PassGeom g) {
  using F = LineFFT<NZ, P>;
  constexpr int T = F::T;
  using LM = ZLaneMap<T>;
  __shared__ double2 tw_s[F::TWLEN];
  __shared__ double2 sbuf_all[LM::LPC][F::BUF];
  F::load_tw(tw_s, a.tw);
  int li, t;
  LM::get(li, t);
  const int half = (g.Nx * g.Ny) >> 1;
  const int p = blockIdx.x * LM::LPC + li;
  const bool valid = p < half;
  const int pc = valid ? p : 0;
  double2* sbuf = sbuf_all[li];
  double2 w[P];
#pragma unroll
  for (int s = 0; s < P; ++s) {
    const int k = t + T * s;
    w[s] = make_double2(__ldg(a.rin + (size_t)pc * NZ + k),
                        __ldg(a.rin + (size_t)(pc + half) * NZ + k));
  }
  F::template run<-1>(w, t, sbuf, tw_s);
  store_pair_spectrum<NZ, P>(w, sbuf, t, a.cout + (size_t)pc * g.Mz,
                             a.cout + (size_t)(pc + half) * g.Mz, 0, valid);
}

// ---------------------------------------------------------------------------
// fwd_x + pointwise update (Source/diffusion.cu:96-365, RK_time_step.cu:82-115)
// ---------------------------------------------------------------------------
enum UpdateMode : int {
  kExplicit = 0,  // base = (1 - dt|k|^2/Re) us + dt (AM.Q - Q) + dt f
  kRhs = 1,       // base = (AM.Q - Q) - |k|^2/Re us + f
  kImplicit = 2,  // base = (us + dt (AM.Q - Q)) / (1 + dt |k|^2/Re)
  kConvOut = 3,   // out = Qhat with Re(Qhat) = 0, Qhat(0) = 0 (calculate_convolution_2p3)
};

// points of the fwd_x update whose state samples are loaded together in the
// plain explicit form (the combining form, which also loads the RK partner,
// the RHS / implicit forms and lines spread over the CTA keep one point's
// loads where they are used: chunks spill there).  B200, per launch of the
// plain form: 2 points 128^3 64.5 -> 59.4 us, 256^3 455 -> 415 us (FP32
// lines 419 -> 367 us); 4 points 60.0 / 444-449 us.
#ifndef NS3D_FX_CHUNK
#define NS3D_FX_CHUNK 2
#endif
// a divisor of P near NS3D_FX_CHUNK (P is 2^k or 3 * 2^k)
__host__ __device__ constexpr int fx_chunk(int P) {
  return NS3D_FX_CHUNK >= P ? P
         : P % NS3D_FX_CHUNK == 0 ? NS3D_FX_CHUNK
         : (NS3D_FX_CHUNK >= 6 && P % 6 == 0) ? 6 : 3;
}

// Load of an update operand (the state u^s or the RK partner u^n) that the
// same thread may overwrite afterwards: in the in-place update `out` aliases
// `us` or `un`.  The read-only (.nc) path is used on purpose.  Every element
// is read exactly once, by the thread that later writes it, and that store
// depends on the loaded value; no other thread reads or writes the element.
// So no load in the kernel can follow a store to its address, and the
// non-coherent cache can never hand out a stale copy.  Measured on a B200
// (256^3 FP64, per fwd_x launch): 413 us with this load against 463 us with a
// coherent ld.global.cg (__ldcg or inline asm); the RK3 step 5.93 against
// 6.59 ms.  The in-place forms (single_time_step: out == us; RK stage 3:
// out == un) are covered by parity tests in both precisions.
__device__ __forceinline__ double2 ld_update(const double2* p) { return __ldg(p); }

template <typename Cx = double2>
struct FwdXArgs {
  const Cx* Qh[3];
  const double2* us[3];
  const double2* un[3];     // combination partner (COMBINE only)
  double2* out[3];
  const double2* fd[3];     // dense forcing or null
  const int* fidx;          // sparse forcing: flat spectral indices
  const double2* fval;      // sparse forcing values, 3 per entry
  int fnnz;
  double dt, Re, ca, cb;    // out = ca * un + cb * base  (COMBINE), else out = base
  const double* dtRe;       // per instance (dt, Re) of a batch, replacing dt and Re; or null
  const double2* tw;
};

// One line of the forward x pass: FFT_x of the 3 product spectra (from the
// prefetch slots), then the pointwise update of Source/diffusion.cu.
template <int NX, int P, int MODE, bool COMBINE, typename C>
__device__ __forceinline__ void fwd_x_line(const FwdXArgs<C>& a, const PassGeom& g, int t, int L,
                                           size_t off, int inst, bool valid, C* sbuf,
                                           const C* tw_s, C* pf, int& ub,
                                           bool more, size_t offn) {
  constexpr int T = NX / P;
  using F = LineFFT<NX, P>;
  const int nlines = g.Ny * g.Mz;
  const int y = L / g.Mz, z = L - y * g.Mz;
  // Re(Qh) is set to zero (set_to_zero_real), so only the imaginary part of
  // each transformed component is kept
  double qi[3][P];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const C* cur = pf + ub * (P * kThreads);
    C* nxt = pf + (ub ^ 1) * (P * kThreads);
    if (c + 1 < 3) {
      issue_line<P, T>(nxt, a.Qh[c + 1], off, (size_t)nlines, t);
    } else if (more) {
      issue_line<P, T>(nxt, a.Qh[0], offn, (size_t)nlines, t);
    }
    cp_async_commit();
    cp_async_wait<1>();
    C v[P];
#pragma unroll
    for (int s = 0; s < P; ++s) v[s] = cur[s * kThreads];
    F::template run<-1, F::PADW, LaneMap<T>::SW>(v, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s) qi[c][s] = (double)v[s].y;
    ub ^= 1;
  }
  if (!valid) return;
  if constexpr (MODE == kConvOut) {
#pragma unroll
    for (int s = 0; s < P; ++s) {
      const int x = t + T * s;
      const size_t idx = off + (size_t)x * nlines;
      const bool origin = (x == 0) && (L == 0);
#pragma unroll
      for (int c = 0; c < 3; ++c) a.out[c][idx] = make_double2(0.0, origin ? 0.0 : qi[c][s]);
    }
    return;
  }
  const double ky = g.kfy * (double)signed_idx(y, g.Ny);
  const double kz = g.kfz * (double)z;
  const bool dense_f = a.fd[0] != nullptr;
  const double dt = a.dtRe ? __ldg(a.dtRe + 2 * inst) : a.dt;
  const double Re = a.dtRe ? __ldg(a.dtRe + 2 * inst + 1) : a.Re;
  // The state samples of CH points are loaded before any of them is
  // updated: the stores may alias the loads (an in-place update), so the
  // compiler keeps every load behind the previous point's store, and point by
  // point each load would wait a full memory round trip.  Each element is
  // still read before it is written, by the same thread.
  constexpr int CH =
      (COMBINE || MODE != kExplicit || LaneMap<T>::kSpread) ? 1 : fx_chunk(P);
  static_assert(P % CH == 0, "update chunk");
#pragma unroll
  for (int s0 = 0; s0 < P; s0 += CH) {
    // CH == 1: each sample is loaded where it is used (fewest live registers)
    double2 us[3][CH];
    double2 un[3][COMBINE ? CH : 1];
    if constexpr (CH > 1) {
#pragma unroll
      for (int j = 0; j < CH; ++j) {
        const size_t idx = off + (size_t)(t + T * (s0 + j)) * nlines;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          us[c][j] = ld_update(a.us[c] + idx);
          if constexpr (COMBINE) un[c][j] = ld_update(a.un[c] + idx);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < CH; ++j) {
      const int s = s0 + j;
      const int x = t + T * s;
      const size_t fi = (size_t)x * nlines + L;  // index inside the instance (forcing)
      const size_t idx = off + (size_t)x * nlines;
      const double kx = g.kfx * (double)signed_idx(x, NX);
      const double kk = kx * kx + ky * ky + kz * kz;
      // set_to_zero_real: Re(Qh) = 0 everywhere, Qh(0,0,0) = 0
      const bool origin = (x == 0) && (L == 0);
      const double Q0 = origin ? 0.0 : qi[0][s];
      const double Q1 = origin ? 0.0 : qi[1][s];
      const double Q2 = origin ? 0.0 : qi[2][s];
      // AM.Q - Q with AM_ij = k_i k_j / |k|^2 (0 at k = 0); imaginary part only
      const double kq = kk > 0.0 ? (kx * Q0 + ky * Q1 + kz * Q2) / kk : 0.0;
      const double p[3] = {kx * kq - Q0, ky * kq - Q1, kz * kq - Q2};
      double2 f[3] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
      if constexpr (MODE != kImplicit) {
        if (dense_f) {
#pragma unroll
          for (int c = 0; c < 3; ++c) f[c] = __ldg(a.fd[c] + fi);
        } else {
          for (int e = 0; e < a.fnnz; ++e) {
            if (__ldg(a.fidx + e) == (int)fi) {
#pragma unroll
              for (int c = 0; c < 3; ++c) f[c] = cadd(f[c], __ldg(a.fval + 3 * e + c));
            }
          }
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double2 u = CH > 1 ? us[c][j] : ld_update(a.us[c] + idx);
        double2 r;
        if constexpr (MODE == kExplicit) {
          const double G = 1.0 - kk * dt / Re;
          r = make_double2(G * u.x + dt * f[c].x, dt * p[c] + G * u.y + dt * f[c].y);
        } else if constexpr (MODE == kRhs) {
          const double G = -kk / Re;
          r = make_double2(G * u.x + f[c].x, p[c] + G * u.y + f[c].y);
        } else {
          const double G = 1.0 + kk * dt / Re;
          r = make_double2(u.x / G, (dt * p[c] + u.y) / G);
        }
        if constexpr (COMBINE) {
          const double2 n = CH > 1 ? un[c][j] : ld_update(a.un[c] + idx);
          r = make_double2(a.ca * n.x + a.cb * r.x, a.ca * n.y + a.cb * r.y);
        }
        a.out[c][idx] = r;
      }
    }
  }
}


// The update at the end of a fwd_x group reads, for every x, the state (and
// combination partner) elements of the group's LPC consecutive lines: one
// contiguous row of LPC x 16 bytes per (x, field).  Requesting those rows into
// L2 when the group starts lets the group's three transforms cover their DRAM
// latency, and the update's loads then hit L2.  A group whose lines straddle
// two instances of a batch is not prefetched, nor are the groups of lines
// spread over the CTA (LPC <= 4: rows of 64 bytes or less).
template <int NX, int LPC, bool COMBINE, typename C, typename Off>
__device__ __forceinline__ void prefetch_update_rows(const FwdXArgs<C>& a, int G0, int tlines,
                                                     int nlines, Off line_off) {
  int nv = tlines - G0;
  if (nv > LPC) nv = LPC;
  if (nv <= 0 || G0 / nlines != (G0 + nv - 1) / nlines) return;
  const size_t off0 = line_off(G0);
  const unsigned bytes = (unsigned)nv * (unsigned)sizeof(double2);
  constexpr int NFLD = COMBINE ? 6 : 3;
  for (int r = threadIdx.x; r < NX * NFLD; r += kThreads) {
    const int f = r / NX, x = r - f * NX;
    const double2* fld = f < 3 ? a.us[f] : a.un[f - 3];
    if (fld) prefetch_l2_bulk(fld + off0 + (size_t)x * nlines, bytes);
  }
}

template <int NX, int P, int MODE, bool COMBINE, typename C>
__global__ void __launch_bounds__(kThreads, kMinCtasFwdX) fwd_x_kernel(FwdXArgs<C> a, PassGeom g) {
  using S = PassSmem<NX, P, C, C>;
  using F = typename S::F;
  using LM = typename S::LM;
  constexpr int T = F::T;
  extern __shared__ __align__(16) unsigned char dsm[];
  F::load_tw(S::tw(dsm), a.tw);
  const C* tw_s = S::tw(dsm);
  int li, t;
  LM::get(li, t);
  C* sbuf = S::sbuf(dsm, li);
  C* pf = S::pf(dsm);
  const int nlines = g.Ny * g.Mz;
  const int tlines = nlines * nbatch(g);
  const int groups = (tlines + LM::LPC - 1) / LM::LPC;
  auto line_off = [&](int G) -> size_t {
    const int b = G / nlines;
    return (size_t)b * NX * nlines + (size_t)(G - b * nlines);
  };
  const GroupRange gr = group_range(groups);
  const int g_end = gr.end;
  int grp = gr.grp;
  if (grp >= g_end) return;
  {
    const int G0 = grp * LM::LPC + li;
    issue_line<P, T>(pf, a.Qh[0], line_off(G0 < tlines ? G0 : 0), (size_t)nlines, t);
    cp_async_commit();
  }
  int ub = 0;
  for (; grp < g_end; grp += gr.step) {
    const int G = grp * LM::LPC + li;
    const bool valid = G < tlines;
    const int Gc = valid ? G : 0;
    const int inst = Gc / nlines;
    const int gn = grp + gr.step;
    const int Gn = gn * LM::LPC + li;
    if constexpr (MODE != kConvOut && !LM::kSpread)
      prefetch_update_rows<NX, LM::LPC, COMBINE>(a, grp * LM::LPC, tlines, nlines, line_off);
    fwd_x_line<NX, P, MODE, COMBINE, C>(a, g, t, Gc - inst * nlines, line_off(Gc), inst, valid,
                                     sbuf, tw_s, pf, ub, gn < g_end,
                                     line_off(Gn < tlines ? Gn : 0));
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// fwd_x with the update's operands in the prefetch ring.
//
// fwd_x_kernel reads the state (and RK partner) samples of its update with
// plain loads after the three transforms, two points at a time: every group
// waits several memory round trips with little in flight.  Here the unit
// sequence of a group is Qh_x, Qh_y, Qh_z (transformed), then u^s_c (and
// u^n_c when combining) for c = x, y, z, and every unit goes through one ring
// of NSLOT per-thread cp.async slots, issued NSLOT - 1 units ahead.  The
// update runs component by component as its operands arrive: component c of
// the update needs only u^s_c (u^n_c) and the three transformed products,
// whose Leray term k (k.Q)/|k|^2 is formed once per point.  Slots hold one
// 16-byte cell per sample and thread (the state is FP64 in both precisions):
// an FP32 product sample sits in the first half of its thread's cell, so a
// slot stays private to each thread whichever kind of unit it holds (with
// 8-byte product cells a thread's cell would overlap another warp's, and a
// warp that runs ahead would overwrite samples not yet read).  Arithmetic
// per point as in fwd_x_line.
// ---------------------------------------------------------------------------
// Ring depth of the 8-point lines and the CTAs per SM requested from ptxas:
// 3 slots at 3 CTAs per SM (168 registers) measured 292 us per plain launch
// at 256^3 against 399 us with 4 slots at 2 CTAs per SM.  Lines of 12 points
// keep 3 slots; shapes whose shared memory does not fit 3 CTAs per SM (12
// points, or the many short lines of 8-point extents) ask for 2.
#ifndef NS3D_FX_SLOTS
#define NS3D_FX_SLOTS 3
#endif
#ifndef NS3D_MINCTA_FXR
#define NS3D_MINCTA_FXR 3
#endif

template <int N, int P, int NSLOT, typename C>
struct FxRingSmem {
  using F = LineFFT<N, P>;
  using LM = LaneMap<F::T>;
  static constexpr int LPC = LM::LPC;
  static constexpr int STRIDE = line_stride(F::BUF, xy_stride_target<F::T>());
  static constexpr size_t SBUF_OFF = align16((size_t)F::TWLEN * sizeof(C));
  static constexpr size_t RING_OFF = align16(SBUF_OFF + (size_t)LPC * STRIDE * sizeof(C));
  static constexpr size_t SLOT = (size_t)P * kThreads * sizeof(double2);
  static constexpr size_t BYTES = RING_OFF + (size_t)NSLOT * SLOT;
  // CTAs per SM asked of ptxas (registers): as many as the shared memory allows
  static constexpr int MINC =
      (P <= 8 && BYTES * NS3D_MINCTA_FXR <= 227 * 1024) ? NS3D_MINCTA_FXR : 2;
  static_assert(BYTES * MINC <= 227 * 1024, "CTAs per SM");
};

template <int NX, int P, int MODE, bool COMBINE, int NSLOT, typename C>
__global__ void __launch_bounds__(kThreads, (FxRingSmem<NX, P, NSLOT, C>::MINC))
    fwd_x_ring_kernel(FwdXArgs<C> a, PassGeom g) {
  using S = FxRingSmem<NX, P, NSLOT, C>;
  using F = typename S::F;
  using LM = typename S::LM;
  constexpr int T = F::T;
  constexpr int NUPD = MODE == kConvOut ? 0 : (COMBINE ? 6 : 3);
  constexpr int UPG = 3 + NUPD;  // units per group
  static_assert(NSLOT >= 2 && (!COMBINE || NSLOT >= 3), "ring depth");
  extern __shared__ __align__(16) unsigned char dsm[];
  F::load_tw((C*)dsm, a.tw);
  const C* tw_s = (const C*)dsm;
  int li, t;
  LM::get(li, t);
  C* sbuf = (C*)(dsm + S::SBUF_OFF) + li * S::STRIDE;
  unsigned char* ring = dsm + S::RING_OFF;
  const int nlines = g.Ny * g.Mz;
  const int tlines = nlines * nbatch(g);
  const int groups = (tlines + LM::LPC - 1) / LM::LPC;
  auto line_off = [&](int G) -> size_t {
    const int b = G / nlines;
    return (size_t)b * NX * nlines + (size_t)(G - b * nlines);
  };
  const GroupRange gr = group_range(groups);
  if (gr.grp >= gr.end) return;  // uniform across the CTA
  const int ngrp = (gr.end - gr.grp + gr.step - 1) / gr.step;
  const int nunits = ngrp * UPG;
  // issue unit k of this CTA's sequence (an empty commit group past the end)
  auto issue = [&](int k) {
    if (k < nunits) {
      const int gi = k / UPG, j = k - gi * UPG;
      const int G = (gr.grp + gi * gr.step) * LM::LPC + li;
      const size_t off = line_off(G < tlines ? G : 0);
      unsigned char* sl = ring + (size_t)(k % NSLOT) * S::SLOT;
      if (j < 3) {
        constexpr int CELL = (int)(sizeof(double2) / sizeof(C));  // C elements per cell
        issue_line<P, T, CELL * kThreads>((C*)sl + CELL * threadIdx.x, a.Qh[j], off,
                                          (size_t)nlines, t);
      } else {
        const int u = j - 3;
        const double2* src = COMBINE ? ((u & 1) ? a.un[u >> 1] : a.us[u >> 1]) : a.us[u];
        issue_line<P, T>((double2*)sl + threadIdx.x, src, off, (size_t)nlines, t);
      }
    }
    cp_async_commit();
  };
  auto slot = [&](int k) -> unsigned char* { return ring + (size_t)(k % NSLOT) * S::SLOT; };
#pragma unroll
  for (int k = 0; k < NSLOT - 1; ++k) issue(k);
  int k = 0;
  for (int gi = 0; gi < ngrp; ++gi) {
    const int G = (gr.grp + gi * gr.step) * LM::LPC + li;
    const bool valid = G < tlines;
    const int Gc = valid ? G : 0;
    const int inst = Gc / nlines;
    const int L = Gc - inst * nlines;
    const size_t off = line_off(Gc);
    // transformed products: Re(Qh) is set to zero (set_to_zero_real), so only
    // the imaginary parts are kept; Qh(0,0,0) = 0
    double qi[3][P];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      issue(k + NSLOT - 1);
      cp_async_wait<NSLOT - 1>();
      constexpr int CELL = (int)(sizeof(double2) / sizeof(C));
      const C* cur = (const C*)slot(k) + CELL * threadIdx.x;
      C v[P];
#pragma unroll
      for (int s = 0; s < P; ++s) v[s] = cur[s * CELL * kThreads];
      F::template run<-1, F::PADW, LM::SW>(v, t, sbuf, tw_s);
#pragma unroll
      for (int s = 0; s < P; ++s) {
        const bool origin = (t + T * s == 0) && (L == 0);
        qi[c][s] = origin ? 0.0 : (double)v[s].y;
      }
      ++k;
    }
    if constexpr (MODE == kConvOut) {
      if (valid) {
#pragma unroll
        for (int s = 0; s < P; ++s) {
          const size_t idx = off + (size_t)(t + T * s) * nlines;
#pragma unroll
          for (int c = 0; c < 3; ++c) a.out[c][idx] = make_double2(0.0, qi[c][s]);
        }
      }
      continue;
    } else {
      const int y = L / g.Mz, z = L - y * g.Mz;
      const double ky = g.kfy * (double)signed_idx(y, g.Ny);
      const double kz = g.kfz * (double)z;
      const bool dense_f = a.fd[0] != nullptr;
      const double dt = a.dtRe ? __ldg(a.dtRe + 2 * inst) : a.dt;
      const double Re = a.dtRe ? __ldg(a.dtRe + 2 * inst + 1) : a.Re;
      // sparse forcing: does any listed mode lie on this line?  (the scan
      // per point below is skipped for the lines without one)
      bool line_f = false;
      if constexpr (MODE != kImplicit) {
        if (!dense_f)
          for (int e = 0; e < a.fnnz; ++e) line_f |= (__ldg(a.fidx + e) % nlines) == L;
      }
      // AM.Q with AM_ij = k_i k_j / |k|^2 (0 at k = 0): kq = k.Q / |k|^2
      double kq[P];
#pragma unroll
      for (int s = 0; s < P; ++s) {
        const double kx = g.kfx * (double)signed_idx(t + T * s, NX);
        const double kk = kx * kx + ky * ky + kz * kz;
        kq[s] = kk > 0.0 ? (kx * qi[0][s] + ky * qi[1][s] + kz * qi[2][s]) / kk : 0.0;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        // issued so far: units 0 .. k + NSLOT - 2; the next issue refills the
        // slot of unit k - 1, consumed already
        issue(k + NSLOT - 1);
        // the combining form reads two units (u^s_c, u^n_c) at once: wait for
        // both, and refill the first one's slot only after the update below
        if constexpr (COMBINE) {
          cp_async_wait<NSLOT - 2>();
        } else {
          cp_async_wait<NSLOT - 1>();
        }
        const double2* us = (const double2*)slot(k) + threadIdx.x;
        const double2* un = COMBINE ? (const double2*)slot(k + 1) + threadIdx.x : us;
        const double kc = c == 0 ? 0.0 : (c == 1 ? ky : kz);
        if (valid) {
#pragma unroll
        for (int s = 0; s < P; ++s) {
          const int x = t + T * s;
          const size_t fi = (size_t)x * nlines + L;  // index inside the instance (forcing)
          const size_t idx = off + (size_t)x * nlines;
          const double kx = g.kfx * (double)signed_idx(x, NX);
          const double kk = kx * kx + ky * ky + kz * kz;
          // AM.Q - Q, imaginary part only
          const double pc = (c == 0 ? kx : kc) * kq[s] - qi[c][s];
          double2 f = make_double2(0.0, 0.0);
          if constexpr (MODE != kImplicit) {
            if (dense_f) {
              f = __ldg(a.fd[c] + fi);
            } else if (line_f) {
              for (int e = 0; e < a.fnnz; ++e)
                if (__ldg(a.fidx + e) == (int)fi) f = cadd(f, __ldg(a.fval + 3 * e + c));
            }
          }
          const double2 u = us[s * kThreads];
          double2 r;
          if constexpr (MODE == kExplicit) {
            const double Gf = 1.0 - kk * dt / Re;
            r = make_double2(Gf * u.x + dt * f.x, dt * pc + Gf * u.y + dt * f.y);
          } else if constexpr (MODE == kRhs) {
            const double Gf = -kk / Re;
            r = make_double2(Gf * u.x + f.x, pc + Gf * u.y + f.y);
          } else {
            const double Gf = 1.0 + kk * dt / Re;
            r = make_double2(u.x / Gf, (dt * pc + u.y) / Gf);
          }
          if constexpr (COMBINE) {
            const double2 n = un[s * kThreads];
            r = make_double2(a.ca * n.x + a.cb * r.x, a.ca * n.y + a.cb * r.y);
          }
          a.out[c][idx] = r;
        }
        }
        ++k;
        if constexpr (COMBINE) {
          issue(k + NSLOT - 1);  // into the slot of u^s_c, read above
          ++k;
        }
      }
    }
  }
  cp_async_wait<0>();
}

}  // namespace ns3d
