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
constexpr int kMinCtasZ = NS3D_MINCTA_Z;
constexpr int kMinCtasFwdX = NS3D_MINCTA_FX;

struct PassGeom {
  int Nx, Ny, Nz, Mz;
  double kfx, kfy, kfz;  // 2*pi/L per direction (Source/math_support.cu:350-370)
  double inv_vol;        // 1/(Nx*Ny*Nz), the scale_double factor
};

// signed wavenumber index: j < N/2 -> j, else j - N (x and y; the Nyquist
// index N/2 is stored as -N/2, Source/math_support.cu:354-357)
__device__ __forceinline__ int signed_idx(int j, int n) { return j < (n >> 1) ? j : j - n; }

// Thread -> (line slot, t) for passes whose batch index is contiguous in
// memory: lanes with the same t and consecutive lines are adjacent, so a warp
// reads LPW consecutive elements of each row.
template <int T>
struct LaneMap {
  static constexpr int LPW = T <= 32 ? 32 / T : 1;
  static constexpr int LPC = T <= 32 ? kWarpsPerCta * LPW : (kWarpsPerCta * 32) / T;
  __device__ __forceinline__ static void get(int& li, int& t) {
    if constexpr (T <= 32) {
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
      t = lane / LPW;
      li = warp * LPW + lane % LPW;
    } else {
      t = threadIdx.x % T;
      li = threadIdx.x / T;
    }
  }
};

// ---------------------------------------------------------------------------
// inv_x: lines along x, batch L = y*Mz + z (contiguous), NF = 3 or 6 fields
// ---------------------------------------------------------------------------
template <int NF>
struct InvXArgs {
  const double2* in[NF];
  double2* A[NF];
  double2* B[NF];
  const uint16_t* qcut;  // [Nx][Ny]: mask(j,k,l) = l < qcut[j*Ny+k], minus (0,0,0)
  const double2* tw;
};

template <int NX, int P, int NF>
__global__ void __launch_bounds__(kWarpsPerCta * 32, kMinCtasXY) inv_x_kernel(InvXArgs<NF> a, PassGeom g) {
  using F = LineFFT<NX, P>;
  constexpr int T = F::T;
  using LM = LaneMap<T>;
  __shared__ double2 tw_s[F::TWLEN];
  __shared__ double2 sbuf_all[LM::LPC][F::BUF];
  F::load_tw(tw_s, a.tw);
  int li, t;
  LM::get(li, t);
  const int nlines = g.Ny * g.Mz;
  const int L = blockIdx.x * LM::LPC + li;
  const bool valid = L < nlines;
  const int Lc = valid ? L : 0;
  const int y = Lc / g.Mz, z = Lc - y * g.Mz;
  double2* sbuf = sbuf_all[li];
  uint32_t keep = 0;  // bit s: mode (t + T s, y, z) survives the 2/3 mask
#pragma unroll
  for (int s = 0; s < P; ++s) {
    const int x = t + T * s;
    const bool k = valid && z < (int)__ldg(a.qcut + x * g.Ny + y) && !(x == 0 && Lc == 0);
    keep |= (uint32_t)k << s;
  }
#pragma unroll 1
  for (int f = 0; f < NF; ++f) {
    // X then i kx X, one transform at a time: the second read of the line hits
    // L1/L2, and only one line of P points is live in registers
    double2 v[P];
#pragma unroll
    for (int s = 0; s < P; ++s) {
      const int x = t + T * s;
      v[s] = ((keep >> s) & 1u) ? __ldg(a.in[f] + (size_t)x * nlines + Lc) : make_double2(0.0, 0.0);
    }
    F::template run<+1>(v, t, sbuf, tw_s);
    if (valid) {
#pragma unroll
      for (int s = 0; s < P; ++s) a.A[f][(size_t)(t + T * s) * nlines + L] = v[s];
    }
#pragma unroll
    for (int s = 0; s < P; ++s) {
      const int x = t + T * s;
      const double2 u =
          ((keep >> s) & 1u) ? __ldg(a.in[f] + (size_t)x * nlines + Lc) : make_double2(0.0, 0.0);
      const double kx = g.kfx * (double)signed_idx(x, NX);
      v[s] = make_double2(-u.y * kx, u.x * kx);  // i kx u (build_ders_device)
    }
    F::template run<+1>(v, t, sbuf, tw_s);
    if (valid) {
#pragma unroll
      for (int s = 0; s < P; ++s) a.B[f][(size_t)(t + T * s) * nlines + L] = v[s];
    }
  }
}

// ---------------------------------------------------------------------------
// inv_y: lines along y, batch b = x*Mz + z, base = x*Ny*Mz + z, stride Mz
// ---------------------------------------------------------------------------
template <int NF>
struct InvYArgs {
  const double2* A[NF];
  const double2* B[NF];
  double2* C[NF];
  double2* D[NF];
  double2* E[NF];
  const double2* tw;
};

template <int NY, int P, int NF>
__global__ void __launch_bounds__(kWarpsPerCta * 32, kMinCtasXY) inv_y_kernel(InvYArgs<NF> a, PassGeom g) {
  using F = LineFFT<NY, P>;
  constexpr int T = F::T;
  using LM = LaneMap<T>;
  __shared__ double2 tw_s[F::TWLEN];
  __shared__ double2 sbuf_all[LM::LPC][F::BUF];
  F::load_tw(tw_s, a.tw);
  int li, t;
  LM::get(li, t);
  const int nb = g.Nx * g.Mz;
  const int b = blockIdx.x * LM::LPC + li;
  const bool valid = b < nb;
  const int bc = valid ? b : 0;
  const int x = bc / g.Mz, z = bc - x * g.Mz;
  const size_t base = (size_t)x * g.Ny * g.Mz + z;
  const int stride = g.Mz;
  double2* sbuf = sbuf_all[li];
#pragma unroll 1
  for (int f = 0; f < NF; ++f) {
    double2 v[P];
#pragma unroll
    for (int s = 0; s < P; ++s) v[s] = __ldg(a.A[f] + base + (size_t)(t + T * s) * stride);
    F::template run<+1>(v, t, sbuf, tw_s);
    if (valid) {
#pragma unroll
      for (int s = 0; s < P; ++s) a.C[f][base + (size_t)(t + T * s) * stride] = v[s];
    }
#pragma unroll
    for (int s = 0; s < P; ++s) {
      const int y = t + T * s;
      const double2 u = __ldg(a.A[f] + base + (size_t)y * stride);
      const double ky = g.kfy * (double)signed_idx(y, NY);
      v[s] = make_double2(-u.y * ky, u.x * ky);
    }
    F::template run<+1>(v, t, sbuf, tw_s);
    if (valid) {
#pragma unroll
      for (int s = 0; s < P; ++s) a.D[f][base + (size_t)(t + T * s) * stride] = v[s];
    }
#pragma unroll
    for (int s = 0; s < P; ++s) v[s] = __ldg(a.B[f] + base + (size_t)(t + T * s) * stride);
    F::template run<+1>(v, t, sbuf, tw_s);
    if (valid) {
#pragma unroll
      for (int s = 0; s < P; ++s) a.E[f][base + (size_t)(t + T * s) * stride] = v[s];
    }
  }
}

// ---------------------------------------------------------------------------
// z pass: lines along z (contiguous), batch b = x*Ny + y, base = b*Mz
// ---------------------------------------------------------------------------
template <int NF>
struct ZArgs {
  // per velocity field (u, then v for the tangent form) and component:
  const double2* C[NF];  // IFFT_xy(M u_i)
  const double2* D[NF];  // IFFT_xy(i ky M u_i)
  const double2* E[NF];  // IFFT_xy(i kx M u_i)
  double2* Qh[3];        // R2C_z of the products (x, y still physical)
  const double2* tw;
};

// Load W[k] = H(X1)[k] + i H(X2)[k] for positions k = t + T s, where H is the
// Hermitian extension of a z half-line (H[0], H[N/2] keep only real parts),
// X = line (optionally times i kz).
template <int NZ, int P, bool IK1, bool IK2>
__device__ __forceinline__ void load_pair(double2 (&w)[P], const double2* __restrict__ f1,
                                          const double2* __restrict__ f2, size_t base, int t,
                                          double kfz) {
  constexpr int T = NZ / P;
#pragma unroll
  for (int s = 0; s < P; ++s) {
    const int k = t + T * s;
    const bool upper = k > NZ / 2;
    const int q = upper ? NZ - k : k;
    double2 c1 = __ldg(f1 + base + q);
    double2 c2 = __ldg(f2 + base + q);
    const double kz = kfz * (double)q;
    if constexpr (IK1) c1 = make_double2(-c1.y * kz, c1.x * kz);
    if constexpr (IK2) c2 = make_double2(-c2.y * kz, c2.x * kz);
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
}

// w holds FFT_z(Q1 + i Q2) at k = t + T s.  Split it with the mirror bin
// W[N-k] (exchanged through shared memory) and store the half spectra
// Q1h[k], Q2h[k] for k = 0..N/2.
template <int NZ, int P>
__device__ __forceinline__ void store_pair_spectrum(const double2 (&w)[P], double2* sbuf, int t,
                                                    double2* __restrict__ o1,
                                                    double2* __restrict__ o2, size_t base,
                                                    bool valid) {
  using F = LineFFT<NZ, P>;
  constexpr int T = F::T;
  line_sync<T>();
#pragma unroll
  for (int s = 0; s < P; ++s) sbuf[spad<F::PADW>(t + T * s)] = w[s];
  line_sync<T>();
#pragma unroll
  for (int s = 0; s < P; ++s) {
    const int k = t + T * s;
    if (k <= NZ / 2 && valid) {
      const double2 a = w[s];
      const double2 m = sbuf[spad<F::PADW>(k == 0 ? 0 : NZ - k)];
      o1[base + k] = make_double2(0.5 * (a.x + m.x), 0.5 * (a.y - m.y));
      o2[base + k] = make_double2(0.5 * (a.y + m.y), -0.5 * (a.x - m.x));
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
template <int NZ, int P>
__device__ __forceinline__ void uv_component(double (&q)[P], int i, const ZArgs<6>& a, size_t base,
                                             int t, double kfz, double sc, double2* sbuf,
                                             const double2* tw_s, const double (&ux)[P],
                                             const double (&uy)[P], const double (&uz)[P],
                                             const double (&vx)[P], const double (&vy)[P],
                                             const double (&vz)[P]) {
  using F = LineFFT<NZ, P>;
  double2 w[P];
  // (d_x u_i, d_y u_i)
  load_pair<NZ, P, false, false>(w, a.E[i], a.D[i], base, t, kfz);
  F::template run<+1>(w, t, sbuf, tw_s);
#pragma unroll
  for (int s = 0; s < P; ++s) q[s] = vx[s] * (w[s].x * sc) + vy[s] * (w[s].y * sc);
  // (d_z u_i, d_x v_i)
  load_pair<NZ, P, true, false>(w, a.C[i], a.E[3 + i], base, t, kfz);
  F::template run<+1>(w, t, sbuf, tw_s);
#pragma unroll
  for (int s = 0; s < P; ++s) {
    q[s] = q[s] + vz[s] * (w[s].x * sc);
    q[s] = q[s] + ux[s] * (w[s].y * sc);
  }
  // (d_y v_i, d_z v_i)
  load_pair<NZ, P, false, true>(w, a.D[3 + i], a.C[3 + i], base, t, kfz);
  F::template run<+1>(w, t, sbuf, tw_s);
#pragma unroll
  for (int s = 0; s < P; ++s) q[s] = q[s] + (uy[s] * (w[s].x * sc) + uz[s] * (w[s].y * sc));
}

template <int NZ, int P, bool UV>
__global__ void __launch_bounds__(kWarpsPerCta * 32, kMinCtasZ) z_kernel(ZArgs<UV ? 6 : 3> a, PassGeom g) {
  using F = LineFFT<NZ, P>;
  constexpr int T = F::T;
  using LM = ZLaneMap<T>;
  __shared__ double2 tw_s[F::TWLEN];
  __shared__ double2 sbuf_all[LM::LPC][F::BUF];
  F::load_tw(tw_s, a.tw);
  int li, t;
  LM::get(li, t);
  const int nb = g.Nx * g.Ny;
  const int b = blockIdx.x * LM::LPC + li;
  const bool valid = b < nb;
  const size_t base = (size_t)(valid ? b : 0) * g.Mz;
  double2* sbuf = sbuf_all[li];
  const double sc = g.inv_vol;
  const double kfz = g.kfz;
  double2 w[P];
  double ux[P], uy[P], uz[P], q0[P], q1[P], q2[P];
  if constexpr (!UV) {
    // Q_z first, so at most five real lines (u_x, u_y, u_z and two products)
    // are live at any time.
    // (u_x, u_y)
    load_pair<NZ, P, false, false>(w, a.C[0], a.C[1], base, t, kfz);
    F::template run<+1>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s) { ux[s] = w[s].x * sc; uy[s] = w[s].y * sc; }
    // (u_z, d_z u_z) from one field
    load_pair<NZ, P, false, true>(w, a.C[2], a.C[2], base, t, kfz);
    F::template run<+1>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s) { uz[s] = w[s].x * sc; q2[s] = w[s].y * sc; }
    // Q_z = u_x d_x u_z + u_y d_y u_z + u_z d_z u_z  (calc_vels_nabla_vels)
    load_pair<NZ, P, false, false>(w, a.E[2], a.D[2], base, t, kfz);
    F::template run<+1>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s)
      q2[s] = ux[s] * (w[s].x * sc) + uy[s] * (w[s].y * sc) + uz[s] * q2[s];
    // R2C of Q_z alone
#pragma unroll
    for (int s = 0; s < P; ++s) w[s] = make_double2(q2[s], 0.0);
    F::template run<-1>(w, t, sbuf, tw_s);
    if (valid) {
#pragma unroll
      for (int s = 0; s < P; ++s) {
        const int k = t + T * s;
        if (k <= NZ / 2) a.Qh[2][base + k] = w[s];
      }
    }
    // (d_z u_x, d_z u_y)
    load_pair<NZ, P, true, true>(w, a.C[0], a.C[1], base, t, kfz);
    F::template run<+1>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s) { q0[s] = w[s].x * sc; q1[s] = w[s].y * sc; }
    load_pair<NZ, P, false, false>(w, a.E[0], a.D[0], base, t, kfz);
    F::template run<+1>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s)
      q0[s] = ux[s] * (w[s].x * sc) + uy[s] * (w[s].y * sc) + uz[s] * q0[s];
    load_pair<NZ, P, false, false>(w, a.E[1], a.D[1], base, t, kfz);
    F::template run<+1>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s)
      q1[s] = ux[s] * (w[s].x * sc) + uy[s] * (w[s].y * sc) + uz[s] * q1[s];
    // R2C of (Q_x, Q_y) packed
#pragma unroll
    for (int s = 0; s < P; ++s) w[s] = make_double2(q0[s], q1[s]);
    F::template run<-1>(w, t, sbuf, tw_s);
    store_pair_spectrum<NZ, P>(w, sbuf, t, a.Qh[0], a.Qh[1], base, valid);
    return;
  } else {
    // B(u,v)_i = (v.grad) u_i + (u.grad) v_i; fields 0..2 are u, 3..5 are v
    double vx[P], vy[P], vz[P];
    load_pair<NZ, P, false, false>(w, a.C[0], a.C[1], base, t, kfz);
    F::template run<+1>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s) { ux[s] = w[s].x * sc; uy[s] = w[s].y * sc; }
    load_pair<NZ, P, false, false>(w, a.C[2], a.C[3], base, t, kfz);
    F::template run<+1>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s) { uz[s] = w[s].x * sc; vx[s] = w[s].y * sc; }
    load_pair<NZ, P, false, false>(w, a.C[4], a.C[5], base, t, kfz);
    F::template run<+1>(w, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s) { vy[s] = w[s].x * sc; vz[s] = w[s].y * sc; }
    uv_component<NZ, P>(q0, 0, a, base, t, kfz, sc, sbuf, tw_s, ux, uy, uz, vx, vy, vz);
    uv_component<NZ, P>(q1, 1, a, base, t, kfz, sc, sbuf, tw_s, ux, uy, uz, vx, vy, vz);
    uv_component<NZ, P>(q2, 2, a, base, t, kfz, sc, sbuf, tw_s, ux, uy, uz, vx, vy, vz);
  }
  // forward R2C along z: (Q0, Q1) packed, then Q2 alone
#pragma unroll
  for (int s = 0; s < P; ++s) w[s] = make_double2(q0[s], q1[s]);
  F::template run<-1>(w, t, sbuf, tw_s);
  store_pair_spectrum<NZ, P>(w, sbuf, t, a.Qh[0], a.Qh[1], base, valid);
#pragma unroll
  for (int s = 0; s < P; ++s) w[s] = make_double2(q2[s], 0.0);
  F::template run<-1>(w, t, sbuf, tw_s);
  if (valid) {
#pragma unroll
    for (int s = 0; s < P; ++s) {
      const int k = t + T * s;
      if (k <= NZ / 2) a.Qh[2][base + k] = w[s];
    }
  }
}

// ---------------------------------------------------------------------------
// fwd_y: in-place forward transform along y of the 3 product spectra
// ---------------------------------------------------------------------------
struct FwdYArgs {
  double2* Q[3];
  const double2* tw;
};

template <int NY, int P>
__global__ void __launch_bounds__(kWarpsPerCta * 32, kMinCtasXY) fwd_y_kernel(FwdYArgs a, PassGeom g) {
  using F = LineFFT<NY, P>;
  constexpr int T = F::T;
  using LM = LaneMap<T>;
  __shared__ double2 tw_s[F::TWLEN];
  __shared__ double2 sbuf_all[LM::LPC][F::BUF];
  F::load_tw(tw_s, a.tw);
  int li, t;
  LM::get(li, t);
  const int nb = g.Nx * g.Mz;
  const int b = blockIdx.x * LM::LPC + li;
  const bool valid = b < nb;
  const int bc = valid ? b : 0;
  const int x = bc / g.Mz, z = bc - x * g.Mz;
  const size_t base = (size_t)x * g.Ny * g.Mz + z;
  const int stride = g.Mz;
  double2* sbuf = sbuf_all[li];
#pragma unroll 1
  for (int f = 0; f < 3; ++f) {
    double2 v[P];
#pragma unroll
    for (int s = 0; s < P; ++s) v[s] = a.Q[f][base + (size_t)(t + T * s) * stride];
    F::template run<-1>(v, t, sbuf, tw_s);
    if (valid) {
#pragma unroll
      for (int s = 0; s < P; ++s) a.Q[f][base + (size_t)(t + T * s) * stride] = v[s];
    }
  }
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

struct FwdXArgs {
  const double2* Qh[3];
  const double2* us[3];
  const double2* un[3];     // combination partner (COMBINE only)
  double2* out[3];
  const double2* fd[3];     // dense forcing or null
  const int* fidx;          // sparse forcing: flat spectral indices
  const double2* fval;      // sparse forcing values, 3 per entry
  int fnnz;
  double dt, Re, ca, cb;    // out = ca * un + cb * base  (COMBINE), else out = base
  const double2* tw;
};

template <int NX, int P, int MODE, bool COMBINE>
__global__ void __launch_bounds__(kWarpsPerCta * 32, kMinCtasFwdX) fwd_x_kernel(FwdXArgs a, PassGeom g) {
  using F = LineFFT<NX, P>;
  constexpr int T = F::T;
  using LM = LaneMap<T>;
  __shared__ double2 tw_s[F::TWLEN];
  __shared__ double2 sbuf_all[LM::LPC][F::BUF];
  F::load_tw(tw_s, a.tw);
  int li, t;
  LM::get(li, t);
  const int nlines = g.Ny * g.Mz;
  const int L = blockIdx.x * LM::LPC + li;
  const bool valid = L < nlines;
  const int Lc = valid ? L : 0;
  const int y = Lc / g.Mz, z = Lc - y * g.Mz;
  double2* sbuf = sbuf_all[li];
  // Re(Qh) is set to zero (set_to_zero_real), so only the imaginary part of
  // each transformed component is kept
  double qi[3][P];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double2 v[P];
#pragma unroll
    for (int s = 0; s < P; ++s) v[s] = __ldg(a.Qh[c] + (size_t)(t + T * s) * nlines + Lc);
    F::template run<-1>(v, t, sbuf, tw_s);
#pragma unroll
    for (int s = 0; s < P; ++s) qi[c][s] = v[s].y;
  }
  if (!valid) return;
  if constexpr (MODE == kConvOut) {
#pragma unroll
    for (int s = 0; s < P; ++s) {
      const int x = t + T * s;
      const size_t idx = (size_t)x * nlines + L;
      const bool origin = (x == 0) && (L == 0);
#pragma unroll
      for (int c = 0; c < 3; ++c) a.out[c][idx] = make_double2(0.0, origin ? 0.0 : qi[c][s]);
    }
    return;
  }
  const double ky = g.kfy * (double)signed_idx(y, g.Ny);
  const double kz = g.kfz * (double)z;
  const bool dense_f = a.fd[0] != nullptr;
#pragma unroll
  for (int s = 0; s < P; ++s) {
    const int x = t + T * s;
    const size_t idx = (size_t)x * nlines + L;
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
        for (int c = 0; c < 3; ++c) f[c] = __ldg(a.fd[c] + idx);
      } else {
        for (int e = 0; e < a.fnnz; ++e) {
          if (__ldg(a.fidx + e) == (int)idx) {
#pragma unroll
            for (int c = 0; c < 3; ++c) f[c] = cadd(f[c], __ldg(a.fval + 3 * e + c));
          }
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double2 u = __ldg(a.us[c] + idx);
      double2 r;
      if constexpr (MODE == kExplicit) {
        const double G = 1.0 - kk * a.dt / a.Re;
        r = make_double2(G * u.x + a.dt * f[c].x, a.dt * p[c] + G * u.y + a.dt * f[c].y);
      } else if constexpr (MODE == kRhs) {
        const double G = -kk / a.Re;
        r = make_double2(G * u.x + f[c].x, p[c] + G * u.y + f[c].y);
      } else {
        const double G = 1.0 + kk * a.dt / a.Re;
        r = make_double2(u.x / G, (a.dt * p[c] + u.y) / G);
      }
      if constexpr (COMBINE) {
        const double2 n = __ldg(a.un[c] + idx);
        r = make_double2(a.ca * n.x + a.cb * r.x, a.ca * n.y + a.cb * r.y);
      }
      a.out[c][idx] = r;
    }
  }
}

}  // namespace ns3d
