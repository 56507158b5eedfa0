// Krylov eigen-analysis on the device: the Arnoldi factorisation with
// classical Gram-Schmidt and iterative reorthogonalisation, and the
// implicit-restart update of the basis.
//
// Reference behaviour followed:
//   Arnoldi_driver       Source/Arnoldi/Arnoldi_Driver.cu:29-120
//   restart update       Source/Arnoldi/Implicit_restart_Arnoldi.cu:544-563
//   built-in maps        Source/NS3D_periodic.cu:340-385,444-470 and the
//                        Krylov self-test operator
//                        Source/Arnoldi/Matrix_Vector_emulator.cu:10-36
//
// The reference issues one cuBLAS call per BLAS-1/2 operation and keeps H on
// the host.  Here each Gram-Schmidt pass is two bandwidth-bound kernels over
// the tall-skinny basis V (n x j+1, column-major, ld n):
//   gemv_t_partial  per-block partial dot products of up to 8 columns per
//                   sweep, the right-hand vector re-read from L2 per sweep;
//   reduce_cols     one block folds the partials in a fixed order
//                   (deterministic), updates h += c and ||c|| on the device;
//   gemv_n_sub      y = y_in - V c with c staged in shared memory.
// Only the scalars the host must branch on (||f||, ||c||) and the Hessenberg
// column travel to the host, through one pinned buffer per pass.
// The restart forms V Q (first k0 columns) and the new residual
// f = hl V q + ql f in ONE pass over V: each row of V is staged in shared
// memory once and every output column is produced from it, in place.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "ns3d.h"

struct ns3d_krylov {
  int64_t n = 0;
  int m_max = 0;
  int device = 0;
  cudaStream_t stream = nullptr;  // nullptr = legacy default stream
  double* v = nullptr;            // n: the normalised Krylov vector handed to the map
  double* w = nullptr;            // n: the map's output
  double* part = nullptr;         // m_max * kMaxBlocks partial sums
  double* small = nullptr;        // [0] norm, [1] ||c||, [2..2+m) h, [2+m..2+2m) c
  double* qcoef = nullptr;        // m_max * (m_max + 1): the Q columns used by a restart
  double* host = nullptr;         // pinned: mirror of `small` + staging of qcoef
  double* lin = nullptr;          // BiCGStab(L) vectors: r[0..L], u[0..L], r~
  int lin_L = 0;
  double* newton = nullptr;       // Newton vectors: delta, -F(x)
  int max_passes = 0;
  int limit_hits = 0;
  long long launches = 0;  // kernels the driver launched in its last call
  std::string err;
};

namespace {

constexpr int kThreads = 256;
constexpr int kColTile = 8;
constexpr int kMaxBlocks = 148 * 4;
constexpr int kRestartThreads = 128;
constexpr int kMaxColumns = 200;        // restart row staging: m * 1 KB of shared memory
constexpr double kReorthTol = 5.0e-12;  // Arnoldi_Driver.cu:31
constexpr int kPassLimitIndex = 12;     // "if(it>12) break" after the pass

int blocks_for(int64_t n, int threads, int cap) {
  const int64_t b = (n + threads - 1) / threads;
  return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// part[c * gridDim.x + b] = sum over the rows of block b of V[c*ldv + r] x[r]
__global__ void __launch_bounds__(kThreads) gemv_t_partial(const double* __restrict__ V,
                                                           int64_t ldv, int ncols,
                                                           const double* __restrict__ x,
                                                           int64_t n, double* __restrict__ part) {
  __shared__ double red[kColTile][kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  for (int c0 = 0; c0 < ncols; c0 += kColTile) {
    const int nc = min(kColTile, ncols - c0);
    const double* Vc = V + (int64_t)c0 * ldv;
    double acc[kColTile];
#pragma unroll
    for (int t = 0; t < kColTile; ++t) acc[t] = 0.0;
    for (int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x; r < n; r += stride) {
      const double xr = __ldg(x + r);
#pragma unroll
      for (int t = 0; t < kColTile; ++t)
        if (t < nc) acc[t] = fma(__ldg(Vc + (int64_t)t * ldv + r), xr, acc[t]);
    }
#pragma unroll
    for (int t = 0; t < kColTile; ++t) {
      double s = acc[t];
#pragma unroll
      for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) red[t][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x < nc) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < kThreads / 32; ++w) s += red[threadIdx.x][w];
      part[(int64_t)(c0 + threadIdx.x) * gridDim.x + blockIdx.x] = s;
    }
    __syncthreads();
  }
}

enum ReduceMode : int {
  kNorm = 0,        // out[0] = sqrt(sum)             (ncols == 1)
  kStore = 1,       // out[c] = sum
  kAccumulate = 2,  // out[c] = sum, acc[c] += sum, nrm[0] = ||out||
};

// One block: column c folded by warp (c mod 8) over the nb partials, lanes
// strided, then a fixed shuffle tree.
__global__ void __launch_bounds__(kThreads) reduce_cols(const double* __restrict__ part, int nb,
                                                        int ncols, int mode, double* out,
                                                        double* acc, double* nrm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = warp; c < ncols; c += kThreads / 32) {
    double s = 0.0;
    for (int b = lane; b < nb; b += 32) s += part[(int64_t)c * nb + b];
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      if (mode == kNorm) {
        out[0] = sqrt(s);
      } else {
        out[c] = s;
        if (mode == kAccumulate) acc[c] += s;
      }
    }
  }
  if (mode == kAccumulate) {
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int c = 0; c < ncols; ++c) s = fma(out[c], out[c], s);
      nrm[0] = sqrt(s);
    }
  }
}

// v = f / ||f|| and V(:, col) = v, with ||f|| read from the device.
__global__ void __launch_bounds__(kThreads) scale_copy(const double* __restrict__ f,
                                                       const double* __restrict__ norm,
                                                       double* __restrict__ v,
                                                       double* __restrict__ vcol, int64_t n) {
  const double inv = 1.0 / norm[0];
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  for (int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x; r < n; r += stride) {
    const double x = f[r] * inv;
    v[r] = x;
    vcol[r] = x;
  }
}

// y_out = y_in - V(:, 0..ncols) c
__global__ void __launch_bounds__(kThreads) gemv_n_sub(const double* __restrict__ V, int64_t ldv,
                                                       int ncols, const double* __restrict__ c,
                                                       const double* y_in, double* y_out,
                                                       int64_t n) {
  extern __shared__ double sc[];
  for (int i = threadIdx.x; i < ncols; i += kThreads) sc[i] = c[i];
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  for (int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x; r < n; r += stride) {
    double s = 0.0;
    int i = 0;
    for (; i + 4 <= ncols; i += 4) {
      const double a0 = __ldg(V + (int64_t)i * ldv + r);
      const double a1 = __ldg(V + (int64_t)(i + 1) * ldv + r);
      const double a2 = __ldg(V + (int64_t)(i + 2) * ldv + r);
      const double a3 = __ldg(V + (int64_t)(i + 3) * ldv + r);
      s = fma(a0, sc[i], s);
      s = fma(a1, sc[i + 1], s);
      s = fma(a2, sc[i + 2], s);
      s = fma(a3, sc[i + 3], s);
    }
    for (; i < ncols; ++i) s = fma(__ldg(V + (int64_t)i * ldv + r), sc[i], s);
    y_out[r] = y_in[r] - s;
  }
}

// In place, per row r of V (n x m, ld n):
//   V(r, j) = sum_c V(r, c) Q(c, j)          for j < k0
//   f(r)    = hl * sum_c V(r, c) Q(c, k0) + ql * f(r)
// qc holds Q(:, 0..k0) column-major (ld m); every lane of a warp reads the
// same coefficient, so those loads are L1 broadcasts.  Each thread stages
// its own row in shared memory (column-strided, conflict-free) before any
// output column is written, so no block barrier is needed.
__global__ void __launch_bounds__(kRestartThreads) restart_rows(double* V, int64_t n, int m,
                                                                int k0,
                                                                const double* __restrict__ qc,
                                                                double hl, double ql, double* f,
                                                                double* W) {
  extern __shared__ double row[];  // m * kRestartThreads
  const int t = threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * kRestartThreads;
  for (int64_t r = (int64_t)blockIdx.x * kRestartThreads + t; r < n; r += stride) {
    for (int c = 0; c < m; ++c) row[c * kRestartThreads + t] = V[(int64_t)c * n + r];
    for (int j = 0; j <= k0; ++j) {
      const double* q = qc + (size_t)j * m;
      double s = 0.0;
      if (j == k0 && !f) break;
      for (int c = 0; c < m; ++c) s = fma(row[c * kRestartThreads + t], __ldg(q + c), s);
      if (j < k0)
        W[(int64_t)j * n + r] = s;
      else
        f[r] = hl * s + ql * f[r];
    }
  }
}

// Register-tiled form of restart_rows for k0 <= KMAX basis outputs: each
// thread keeps the outputs of RR rows (2, or 1 for KMAX = 64) in registers,
// streams its rows of V in chunks of 8 columns (coalesced across the warp)
// and reads each coefficient, staged in shared memory, once per RR rows (a
// broadcast).  The residual column Q(:, k0) has its own accumulator, so no
// output is selected by a runtime index.  Outputs go to W (W = V: in place;
// each thread reads its whole row before writing it); f = null skips the
// residual.
template <int KMAX, int RR>
__global__ void __launch_bounds__(kRestartThreads) restart_rows_reg(double* V, int64_t n, int m,
                                                                    int k0,
                                                                    const double* __restrict__ qc,
                                                                    double hl, double ql,
                                                                    double* f, double* W) {
  // sq: Q(:, 0..k0-1) column-major, zero-padded to KMAX columns, then
  // Q(:, k0); 8 words of zero padding after each part
  extern __shared__ double sq[];
  const int nb = m * KMAX + 8;
  for (int i = threadIdx.x; i < nb + m + 8; i += kRestartThreads) {
    double x = 0.0;
    if (i < m * k0)
      x = qc[i];
    else if (f && i >= nb && i < nb + m)
      x = qc[(size_t)k0 * m + (i - nb)];
    sq[i] = x;
  }
  __syncthreads();
  const double* sqf = sq + nb;
  const int64_t stride = (int64_t)gridDim.x * kRestartThreads * RR;
  for (int64_t r0 = (int64_t)blockIdx.x * kRestartThreads * RR + threadIdx.x; r0 < n;
       r0 += stride) {
    double acc[RR][KMAX];
    double accf[RR];
#pragma unroll
    for (int rr = 0; rr < RR; ++rr) {
      accf[rr] = 0.0;
#pragma unroll
      for (int j = 0; j < KMAX; ++j) acc[rr][j] = 0.0;
    }
#pragma unroll 1
    for (int c0 = 0; c0 < m; c0 += 8) {
      double v[RR][8];
#pragma unroll
      for (int rr = 0; rr < RR; ++rr) {
        const int64_t r = r0 + (int64_t)rr * kRestartThreads;
#pragma unroll
        for (int t = 0; t < 8; ++t)
          v[rr][t] = (r < n && c0 + t < m) ? V[(int64_t)(c0 + t) * n + r] : 0.0;
      }
#pragma unroll
      for (int j = 0; j < KMAX; ++j) {
        const double* q = sq + j * m + c0;  // entries past column j meet v = 0
#pragma unroll
        for (int t = 0; t < 8; ++t) {
          const double qv = q[t];
#pragma unroll
          for (int rr = 0; rr < RR; ++rr) acc[rr][j] = fma(v[rr][t], qv, acc[rr][j]);
        }
      }
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const double qv = sqf[c0 + t];
#pragma unroll
        for (int rr = 0; rr < RR; ++rr) accf[rr] = fma(v[rr][t], qv, accf[rr]);
      }
    }
#pragma unroll
    for (int rr = 0; rr < RR; ++rr) {
      const int64_t r = r0 + (int64_t)rr * kRestartThreads;
      if (r < n) {
#pragma unroll
        for (int j = 0; j < KMAX; ++j)
          if (j < k0) W[(int64_t)j * n + r] = acc[rr][j];
        if (f) f[r] = hl * accf[rr] + ql * f[r];
      }
    }
  }
}

// Launches the restart pass for the basis columns 0..k0-1 and the residual.
cudaError_t launch_restart(double* V, int64_t n, int m, int k0, const double* qc, double hl,
                           double ql, double* f, cudaStream_t st, double* W = nullptr) {
  if (!W) W = V;
  const int kmax = k0 <= 8 ? 8 : k0 <= 16 ? 16 : k0 <= 32 ? 32 : 64;
  const size_t sq = sizeof(double) * ((size_t)m * kmax + 8 + m + 8);
  const int b2 = blocks_for(n, kRestartThreads * 2, 148 * 8);
  const int b1 = blocks_for(n, kRestartThreads, 148 * 8);
  if (k0 <= 8)
    restart_rows_reg<8, 2><<<b2, kRestartThreads, sq, st>>>(V, n, m, k0, qc, hl, ql, f, W);
  else if (k0 <= 16)
    restart_rows_reg<16, 2><<<b2, kRestartThreads, sq, st>>>(V, n, m, k0, qc, hl, ql, f, W);
  else if (k0 <= 32)
    restart_rows_reg<32, 2><<<b2, kRestartThreads, sq, st>>>(V, n, m, k0, qc, hl, ql, f, W);
  else if (k0 <= 64)
    restart_rows_reg<64, 1><<<b1, kRestartThreads, sq, st>>>(V, n, m, k0, qc, hl, ql, f, W);
  else
    restart_rows<<<b1, kRestartThreads, sizeof(double) * (size_t)m * kRestartThreads, st>>>(
        V, n, m, k0, qc, hl, ql, f, W);
  return cudaGetLastError();
}

// out = a x + b y (out may be y); b = 0 ignores y
__global__ void __launch_bounds__(kThreads) axpby(int64_t n, double a, const double* x, double b,
                                                  const double* y, double* out) {
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride)
    out[i] = b == 0.0 ? a * x[i] : a * x[i] + b * y[i];
}

// zeros with 1.0, 1.5, 0.5, 1.0, 1.0 at 1, n/4, n/2, n-1, n-4
// (set_initial_Krylov_vector_value_kernel, Source/Arnoldi/cuda_supp.cu:451-465)
__global__ void __launch_bounds__(kThreads) newton_start(int64_t n, double* d) {
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
    double v = 0.0;
    if (i == 1 || i == n - 1 || i == n - 4) v = 1.0;
    if (i == n / 4) v = 1.5;
    if (i == n / 2) v = 0.5;
    d[i] = v;
  }
}

// out_i = in_{i+1} - 2 in_i + in_{i-1} (periodic), out_0 = 0
__global__ void __launch_bounds__(kThreads) laplace1d_kernel(const double* __restrict__ in,
                                                             double* __restrict__ out, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
    if (i == 0) {
      out[0] = 0.0;
      continue;
    }
    const int64_t ip = (i + 1 == n) ? 0 : i + 1;
    out[i] = in[ip] - 2.0 * in[i] + in[i - 1];
  }
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------

ns3d_status kfail(ns3d_krylov* kr, ns3d_status s, const std::string& msg) {
  if (kr) kr->err = msg;
  return s;
}

ns3d_status kcuda(ns3d_krylov* kr, cudaError_t e, const char* where) {
  if (e == cudaSuccess) return NS3D_OK;
  return kfail(kr, e == cudaErrorMemoryAllocation ? NS3D_ERR_OOM : NS3D_ERR_CUDA,
               std::string(where) + ": " + cudaGetErrorString(e));
}

#define KR_TRY(expr)                 \
  do {                               \
    ns3d_status s_ = (expr);         \
    if (s_ != NS3D_OK) return s_;    \
  } while (0)
#define KR_CHECK(kr, expr, where) KR_TRY(kcuda(kr, (expr), where))


ns3d_status enter(ns3d_krylov* kr) {
  if (!kr) return NS3D_ERR_BAD_ARG;
  KR_CHECK(kr, cudaSetDevice(kr->device), "cudaSetDevice");
  kr->err.clear();
  return NS3D_OK;
}

// dst[0..ncols) = V(:, 0..ncols)^T x, written by reduce_cols in `mode`.
ns3d_status dots(ns3d_krylov* kr, const double* V, int ncols, const double* x, int mode,
                 double* out, double* acc, double* nrm) {
  const int nb = blocks_for(kr->n, kThreads, kMaxBlocks);
  gemv_t_partial<<<nb, kThreads, 0, kr->stream>>>(V, kr->n, ncols, x, kr->n, kr->part);
  KR_CHECK(kr, cudaGetLastError(), "gemv_t_partial");
  reduce_cols<<<1, kThreads, 0, kr->stream>>>(kr->part, nb, ncols, mode, out, acc, nrm);
  KR_CHECK(kr, cudaGetLastError(), "reduce_cols");
  kr->launches += 2;
  return NS3D_OK;
}

ns3d_status subtract(ns3d_krylov* kr, const double* V, int ncols, const double* c,
                     const double* y_in, double* y_out) {
  const int nb = blocks_for(kr->n, kThreads, kMaxBlocks * 2);
  gemv_n_sub<<<nb, kThreads, sizeof(double) * ncols, kr->stream>>>(V, kr->n, ncols, c, y_in,
                                                                   y_out, kr->n);
  KR_CHECK(kr, cudaGetLastError(), "gemv_n_sub");
  kr->launches += 1;
  return NS3D_OK;
}

// ||f|| -> small[0]; v = V(:, col) = f / ||f||.
ns3d_status normalise_into(ns3d_krylov* kr, double* f, double* vcol) {
  KR_TRY(dots(kr, f, 1, f, kNorm, kr->small, nullptr, nullptr));
  scale_copy<<<blocks_for(kr->n, kThreads, kMaxBlocks * 2), kThreads, 0, kr->stream>>>(
      f, kr->small, kr->v, vcol, kr->n);
  KR_CHECK(kr, cudaGetLastError(), "scale_copy");
  kr->launches += 1;
  return NS3D_OK;
}

ns3d_status fetch(ns3d_krylov* kr, int count) {
  KR_CHECK(kr, cudaMemcpyAsync(kr->host, kr->small, sizeof(double) * count,
                               cudaMemcpyDeviceToHost, kr->stream),
           "scalar copy");
  KR_CHECK(kr, cudaStreamSynchronize(kr->stream), "scalar sync");
  return NS3D_OK;
}

ns3d_status call_map(ns3d_krylov* kr, ns3d_user_map_vector Axb, void* user) {
  // the map may run on any stream: v must be complete before it starts
  KR_CHECK(kr, cudaStreamSynchronize(kr->stream), "sync before map");
  Axb(user, kr->v, kr->w);
  KR_CHECK(kr, cudaGetLastError(), "matrix-vector map");
  return NS3D_OK;
}

ns3d_status apply_map(ns3d_krylov* kr, ns3d_user_map_vector Axb, void* user, const double* in,
                      double* out) {
  KR_CHECK(kr, cudaStreamSynchronize(kr->stream), "sync before map");
  Axb(user, const_cast<double*>(in), out);
  KR_CHECK(kr, cudaGetLastError(), "matrix-vector map");
  return NS3D_OK;
}

// out = a x + b y
ns3d_status combine(ns3d_krylov* kr, double a, const double* x, double b, const double* y,
                double* out) {
  axpby<<<blocks_for(kr->n, kThreads, kMaxBlocks * 2), kThreads, 0, kr->stream>>>(kr->n, a, x, b,
                                                                                y, out);
  KR_CHECK(kr, cudaGetLastError(), "axpby");
  kr->launches += 1;
  return NS3D_OK;
}

// x . y, returned to the host (synchronous, like cublasDdot)
ns3d_status dot(ns3d_krylov* kr, const double* x, const double* y, double* out) {
  double* cd = kr->small + 2 + kr->m_max;
  KR_TRY(dots(kr, x, 1, y, kStore, cd, nullptr, nullptr));
  KR_CHECK(kr, cudaMemcpyAsync(kr->host, cd, sizeof(double), cudaMemcpyDeviceToHost, kr->stream),
           "dot copy");
  KR_CHECK(kr, cudaStreamSynchronize(kr->stream), "dot sync");
  *out = kr->host[0];
  return NS3D_OK;
}

ns3d_status norm2(ns3d_krylov* kr, const double* x, double* out) {
  KR_TRY(dots(kr, x, 1, x, kNorm, kr->small, nullptr, nullptr));
  KR_TRY(fetch(kr, 1));
  *out = kr->host[0];
  return NS3D_OK;
}

// BiCGStabL (Source/Arnoldi/BiCGStabL.cu:18-185) on the workspace's vectors.
ns3d_status bicgstabl(ns3d_krylov* kr, int L, ns3d_user_map_vector Axb, void* user, double* x,
                      const double* rhs, double* tol, int* iter, int* flag_out) {
  const int64_t n = kr->n;
  if (!kr->lin || kr->lin_L < L) {
    cudaFree(kr->lin);
    kr->lin = nullptr;
    kr->lin_L = 0;
    KR_CHECK(kr, cudaMalloc(&kr->lin, sizeof(double) * (size_t)(2 * L + 3) * n),
             "BiCGStab(L) vectors");
    kr->lin_L = L;
  }
  double* r0 = kr->lin;
  double* u0 = kr->lin + (size_t)(L + 1) * n;
  double* rt = kr->lin + (size_t)(2 * L + 2) * n;
  auto r = [&](int i) { return r0 + (size_t)i * n; };
  auto u = [&](int i) { return u0 + (size_t)i * n; };
  KR_CHECK(kr, cudaMemsetAsync(kr->lin, 0, sizeof(double) * (size_t)(2 * L + 2) * n, kr->stream),
           "BiCGStab(L) clear");
  std::vector<double> tau((size_t)L * L, 0.0), sigma(L + 1, 0.0), gamma(L + 1, 0.0),
      gamma_p(L + 1, 0.0), gamma_pp(L + 1, 0.0);
  const double tl = *tol;
  const int maxit = *iter;
  int flag = 1, it = 0;
  double error = 1.0, bnrm = 0.0, t = 0.0;
  KR_TRY(norm2(kr, rhs, &bnrm));
  if (bnrm < 1.0e-15) bnrm = 1.0;
  // r0 = -(A x - b)
  KR_TRY(apply_map(kr, Axb, user, x, r(0)));
  KR_TRY(combine(kr, 1.0, r(0), -1.0, rhs, r(0)));
  KR_TRY(combine(kr, -1.0, r(0), 0.0, nullptr, r(0)));
  KR_TRY(norm2(kr, r(0), &t));
  error = t / bnrm;
  if (error < tl) flag = 0;
  if (std::isnan(error)) flag = -3;
  if (flag == 1) KR_TRY(combine(kr, 1.0 / t, r(0), 0.0, nullptr, rt));
  double rho = 1.0, alpha = 0.0, omega = 1.0;
  if (flag == 1) {
    for (it = 0; it < maxit; ++it) {
      rho = -omega * rho;
      for (int j = 0; j < L; ++j) {
        if (rho == 0.0) {
          flag = -1;
          rho = 1.0;
        }
        double rho1 = 0.0;
        KR_TRY(dot(kr, r(j), rt, &rho1));
        const double beta = alpha * rho1 / rho;
        rho = rho1;
        for (int i = 0; i <= j; ++i) KR_TRY(combine(kr, 1.0, r(i), -beta, u(i), u(i)));
        KR_TRY(apply_map(kr, Axb, user, u(j), u(j + 1)));
        double d = 0.0;
        KR_TRY(dot(kr, u(j + 1), rt, &d));
        alpha = rho / d;
        for (int i = 0; i <= j; ++i) KR_TRY(combine(kr, -alpha, u(i + 1), 1.0, r(i), r(i)));
        KR_TRY(apply_map(kr, Axb, user, r(j), r(j + 1)));
        KR_TRY(combine(kr, alpha, u(0), 1.0, x, x));
      }
      for (int j = 1; j <= L; ++j) {
        for (int i = 1; i < j; ++i) {
          const int ij = (j - 1) * L + (i - 1);
          double d = 0.0;
          KR_TRY(dot(kr, r(j), r(i), &d));
          tau[ij] = d / sigma[i];
          KR_TRY(combine(kr, -tau[ij], r(i), 1.0, r(j), r(j)));
        }
        KR_TRY(dot(kr, r(j), r(j), &sigma[j]));
        double d = 0.0;
        KR_TRY(dot(kr, r(0), r(j), &d));
        gamma_p[j] = d / sigma[j];
      }
      gamma[L] = gamma_p[L];
      omega = gamma[L];
      for (int j = L - 1; j >= 1; --j) {
        gamma[j] = gamma_p[j];
        for (int i = j + 1; i <= L; ++i) gamma[j] -= tau[(i - 1) * L + (j - 1)] * gamma[i];
      }
      for (int j = 1; j < L; ++j) {
        gamma_pp[j] = gamma[j + 1];
        for (int i = j + 1; i < L; ++i) gamma_pp[j] += tau[(i - 1) * L + (j - 1)] * gamma[i + 1];
      }
      KR_TRY(combine(kr, gamma[1], r(0), 1.0, x, x));
      KR_TRY(combine(kr, -gamma_p[L], r(L), 1.0, r(0), r(0)));
      KR_TRY(combine(kr, -gamma[L], u(L), 1.0, u(0), u(0)));
      for (int j = 1; j < L; ++j) {
        KR_TRY(combine(kr, gamma_pp[j], r(j), 1.0, x, x));
        KR_TRY(combine(kr, -gamma_p[j], r(j), 1.0, r(0), r(0)));
        KR_TRY(combine(kr, -gamma[j], u(j), 1.0, u(0), u(0)));
      }
      KR_TRY(norm2(kr, r(0), &t));
      error = t / bnrm;
      if (error < tl) {
        flag = 0;
        break;
      }
      if (error != error) {
        flag = -3;
        break;
      }
      if (flag < 0) break;
    }
  }
  *iter = it;
  *tol = error;
  *flag_out = flag;
  return NS3D_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

ns3d_status ns3d_krylov_create(int64_t n, int m_max, ns3d_krylov** out) {
  if (!out) return NS3D_ERR_BAD_ARG;
  *out = nullptr;
  if (n < 2 || m_max < 2 || m_max > kMaxColumns) return NS3D_ERR_BAD_ARG;
  ns3d_krylov* kr = new ns3d_krylov();
  kr->n = n;
  kr->m_max = m_max;
  cudaGetDevice(&kr->device);
  const size_t small = 2 + 2 * (size_t)m_max;
  const size_t qc = (size_t)m_max * (m_max + 1);
  cudaError_t e = cudaMalloc(&kr->v, sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMalloc(&kr->w, sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMalloc(&kr->part, sizeof(double) * (size_t)m_max * kMaxBlocks);
  if (e == cudaSuccess) e = cudaMalloc(&kr->small, sizeof(double) * small);
  if (e == cudaSuccess) e = cudaMalloc(&kr->qcoef, sizeof(double) * qc);
  if (e == cudaSuccess) e = cudaMallocHost(&kr->host, sizeof(double) * (small + qc));
  if (e == cudaSuccess) e = cudaMemset(kr->v, 0, sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMemset(kr->w, 0, sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMemset(kr->small, 0, sizeof(double) * small);
  // The dynamic shared-memory caps are attributes of the kernels, shared by
  // every workspace on the device: set them for the largest basis any
  // workspace may have (kMaxColumns), so a workspace created later with a
  // smaller m_max cannot lower the cap below what an earlier one launches.
  if (e == cudaSuccess) {
    const size_t smem = sizeof(double) * (size_t)kMaxColumns * kRestartThreads;
    e = cudaFuncSetAttribute(restart_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
  }
  if (e == cudaSuccess) {
    const int sq = (int)(sizeof(double) * ((size_t)kMaxColumns * 64 + 8 + kMaxColumns + 8));
    e = cudaFuncSetAttribute(restart_rows_reg<8, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             sq);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(restart_rows_reg<16, 2>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, sq);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(restart_rows_reg<32, 2>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, sq);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(restart_rows_reg<64, 1>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, sq);
  }
  if (e != cudaSuccess) {
    ns3d_krylov_destroy(kr);
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? NS3D_ERR_OOM : NS3D_ERR_CUDA;
  }
  *out = kr;
  return NS3D_OK;
}

ns3d_status ns3d_krylov_destroy(ns3d_krylov* kr) {
  if (!kr) return NS3D_ERR_BAD_ARG;
  cudaSetDevice(kr->device);
  cudaStreamSynchronize(kr->stream);
  cudaFree(kr->v);
  cudaFree(kr->w);
  cudaFree(kr->part);
  cudaFree(kr->small);
  cudaFree(kr->qcoef);
  cudaFree(kr->lin);
  cudaFree(kr->newton);
  cudaFreeHost(kr->host);
  delete kr;
  return NS3D_OK;
}

ns3d_status ns3d_krylov_set_stream(ns3d_krylov* kr, void* stream) {
  KR_TRY(enter(kr));
  kr->stream = (cudaStream_t)stream;
  return NS3D_OK;
}

const char* ns3d_krylov_last_error(const ns3d_krylov* kr) {
  return kr ? kr->err.c_str() : "null workspace";
}

ns3d_status ns3d_krylov_stats(const ns3d_krylov* kr, int* max_passes, int* limit_hits,
                              int64_t* launches) {
  if (!kr) return NS3D_ERR_BAD_ARG;
  if (max_passes) *max_passes = kr->max_passes;
  if (limit_hits) *limit_hits = kr->limit_hits;
  if (launches) *launches = kr->launches;
  return NS3D_OK;
}

ns3d_status ns3d_arnoldi(ns3d_krylov* kr, ns3d_user_map_vector Axb, void* user, double* V,
                         double* H, double* f, int k, int m) {
  KR_TRY(enter(kr));
  if (!Axb || !V || !H || !f) return kfail(kr, NS3D_ERR_BAD_ARG, "null pointer");
  if (m < 2 || m > kr->m_max || k < 0 || k >= m)
    return kfail(kr, NS3D_ERR_BAD_ARG, "need 0 <= k < m <= m_max and m >= 2");
  kr->max_passes = 0;
  kr->limit_hits = 0;
  kr->launches = 0;
  const int64_t n = kr->n;
  double* hd = kr->small + 2;      // h on the device
  double* cd = kr->small + 2 + m;  // c on the device (k == 0 uses cd[0] as the scalar)
  const double* hh = kr->host + 2;

  if (k == 0) {
    KR_TRY(normalise_into(kr, f, V));
    KR_TRY(fetch(kr, 1));
    const double beta = kr->host[0];
    if (!std::isfinite(beta)) return kfail(kr, NS3D_ERR_NONFINITE, "||f|| is not finite");
    if (beta < 1.0e-15)
      return kfail(kr, NS3D_ERR_BAD_ARG, "norm of the input vector ||f|| < 1e-15");
    KR_TRY(call_map(kr, Axb, user));
    KR_TRY(dots(kr, kr->v, 1, kr->w, kStore, cd, nullptr, nullptr));
    KR_TRY(subtract(kr, kr->v, 1, cd, kr->w, f));
    KR_CHECK(kr, cudaMemcpyAsync(kr->host, cd, sizeof(double), cudaMemcpyDeviceToHost,
                                 kr->stream), "alpha copy");
    KR_CHECK(kr, cudaStreamSynchronize(kr->stream), "alpha sync");
    double alpha = kr->host[0];
    double c = 1.0;
    int it = 0;
    while (c > kReorthTol) {  // signed, as the reference tests it
      ++it;
      KR_TRY(dots(kr, kr->v, 1, f, kStore, cd, nullptr, nullptr));
      KR_TRY(subtract(kr, kr->v, 1, cd, f, f));
      KR_CHECK(kr, cudaMemcpyAsync(kr->host, cd, sizeof(double), cudaMemcpyDeviceToHost,
                                   kr->stream), "c copy");
      KR_CHECK(kr, cudaStreamSynchronize(kr->stream), "c sync");
      c = kr->host[0];
      alpha += c;
      if (!std::isfinite(c)) return kfail(kr, NS3D_ERR_NONFINITE, "reorthogonalisation");
      if (it > kPassLimitIndex) {
        ++kr->limit_hits;
        break;
      }
    }
    if (it > kr->max_passes) kr->max_passes = it;
    if (!std::isfinite(alpha)) return kfail(kr, NS3D_ERR_NONFINITE, "H(0,0) is not finite");
    H[0] = alpha;
  }

  for (int j = k + 1; j < m; ++j) {
    KR_TRY(normalise_into(kr, f, V + (int64_t)j * n));
    KR_TRY(fetch(kr, 1));
    const double beta = kr->host[0];
    if (!std::isfinite(beta)) return kfail(kr, NS3D_ERR_NONFINITE, "||f|| is not finite");
    H[j + (int64_t)(j - 1) * m] = beta;
    KR_TRY(call_map(kr, Axb, user));
    KR_CHECK(kr, cudaMemsetAsync(hd, 0, sizeof(double) * 2 * m, kr->stream), "h reset");
    KR_TRY(dots(kr, V, j + 1, kr->w, kStore, hd, nullptr, nullptr));
    KR_TRY(subtract(kr, V, j + 1, hd, kr->w, f));
    double cn = 1.0;
    int it = 0;
    while (cn > kReorthTol) {
      ++it;
      KR_TRY(dots(kr, V, j + 1, f, kAccumulate, cd, hd, kr->small + 1));
      KR_TRY(subtract(kr, V, j + 1, cd, f, f));
      KR_TRY(fetch(kr, 2 + m));
      cn = kr->host[1];
      if (!std::isfinite(cn)) return kfail(kr, NS3D_ERR_NONFINITE, "reorthogonalisation");
      if (it > kPassLimitIndex) {
        ++kr->limit_hits;
        break;
      }
    }
    if (it > kr->max_passes) kr->max_passes = it;
    for (int i = 0; i < m; ++i) {
      const double x = i <= j ? hh[i] : 0.0;
      if (!std::isfinite(x)) return kfail(kr, NS3D_ERR_NONFINITE, "H column is not finite");
      H[i + (int64_t)j * m] = x;
    }
  }
  return NS3D_OK;
}

ns3d_status ns3d_ira_restart(ns3d_krylov* kr, double* V, double* f, double* Q, const double* H,
                             int k0, int m, double* f_norm) {
  KR_TRY(enter(kr));
  if (!V || !f || !Q || !H) return kfail(kr, NS3D_ERR_BAD_ARG, "null pointer");
  if (m < 2 || m > kr->m_max || k0 < 1 || k0 >= m)
    return kfail(kr, NS3D_ERR_BAD_ARG, "need 1 <= k0 < m <= m_max");
  const double hl = H[k0 + (int64_t)(k0 - 1) * m];
  const double ql = Q[(m - 1) + (int64_t)(k0 - 1) * m];
  const size_t small = 2 + 2 * (size_t)kr->m_max;
  double* staged = kr->host + small;
  const size_t nq = (size_t)m * (k0 + 1);
  std::memcpy(staged, Q, sizeof(double) * nq);  // Q(:, 0..k0), column-major
  KR_CHECK(kr, cudaMemcpyAsync(kr->qcoef, staged, sizeof(double) * nq, cudaMemcpyHostToDevice,
                               kr->stream), "Q upload");
  KR_TRY(dots(kr, f, 1, f, kNorm, kr->small, nullptr, nullptr));
  KR_CHECK(kr, launch_restart(V, kr->n, m, k0, kr->qcoef, hl, ql, f, kr->stream),
           "restart_rows");
  KR_TRY(fetch(kr, 1));
  if (f_norm) *f_norm = kr->host[0];
  for (int j = k0; j < m; ++j)
    for (int i = 0; i < m; ++i) Q[i + (int64_t)j * m] = (i == j) ? 1.0 : 0.0;
  if (!std::isfinite(kr->host[0])) return kfail(kr, NS3D_ERR_NONFINITE, "||f|| is not finite");
  return NS3D_OK;
}

ns3d_status ns3d_krylov_profile(ns3d_krylov* kr, const double* V, int ncols, const double* x,
                                int reps, double* ms) {
  KR_TRY(enter(kr));
  if (!V || !x || !ms || reps < 1 || ncols < 1 || ncols > kr->m_max)
    return kfail(kr, NS3D_ERR_BAD_ARG, "need V, x, ms, reps >= 1, 1 <= ncols <= m_max");
  cudaEvent_t e0, e1;
  KR_CHECK(kr, cudaEventCreate(&e0), "event");
  KR_CHECK(kr, cudaEventCreate(&e1), "event");
  double* cd = kr->small + 2 + kr->m_max;
  // identity coefficients for the restart: V Q = V, f = 0 * (V q) + 1 * f
  std::vector<double> eye((size_t)ncols * ncols, 0.0);
  for (int i = 0; i < ncols; ++i) eye[(size_t)i * ncols + i] = 1.0;
  const int k0 = ncols - 1;
  KR_CHECK(kr, cudaMemcpy(kr->qcoef, eye.data(), sizeof(double) * (size_t)ncols * (k0 + 1),
                          cudaMemcpyHostToDevice), "Q upload");
  KR_CHECK(kr, cudaMemcpyAsync(kr->w, x, sizeof(double) * kr->n, cudaMemcpyDeviceToDevice,
                               kr->stream), "x copy");
  for (int which = 0; which < 3; ++which) {
    for (int r = -1; r < reps; ++r) {  // r = -1: warm-up
      if (r == 0) cudaEventRecord(e0, kr->stream);
      if (which == 0) {
        KR_TRY(dots(kr, V, ncols, x, kStore, cd, nullptr, nullptr));
      } else if (which == 1) {
        KR_TRY(subtract(kr, V, ncols, cd, x, kr->w));
      } else {
        KR_CHECK(kr, launch_restart(const_cast<double*>(V), kr->n, ncols, k0, kr->qcoef, 0.0,
                                    1.0, kr->w, kr->stream),
                 "restart_rows");
      }
    }
    cudaEventRecord(e1, kr->stream);
    KR_CHECK(kr, cudaEventSynchronize(e1), "profile sync");
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    ms[which] = (double)t / reps;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return NS3D_OK;
}

ns3d_status ns3d_krylov_combine(ns3d_krylov* kr, const double* V, int m, const double* C, int p,
                                double* W) {
  KR_TRY(enter(kr));
  if (!V || !C || !W || m < 1 || m > kr->m_max || p < 1 || p > kr->m_max)
    return kfail(kr, NS3D_ERR_BAD_ARG, "need 1 <= m, p <= m_max and non-null pointers");
  const size_t nq = (size_t)m * p;
  double* staged = kr->host + 2 + 2 * (size_t)kr->m_max;
  std::memcpy(staged, C, sizeof(double) * nq);
  KR_CHECK(kr, cudaMemcpyAsync(kr->qcoef, staged, sizeof(double) * nq, cudaMemcpyHostToDevice,
                               kr->stream), "C upload");
  KR_CHECK(kr, launch_restart(const_cast<double*>(V), kr->n, m, p, kr->qcoef, 0.0, 0.0, nullptr,
                              kr->stream, W),
           "combine");
  KR_CHECK(kr, cudaStreamSynchronize(kr->stream), "combine sync");
  return NS3D_OK;
}

ns3d_status ns3d_bicgstabl(ns3d_krylov* kr, int L, ns3d_user_map_vector Axb, void* user,
                           double* x, const double* rhs, double* tol, int* iter, int* flag) {
  KR_TRY(enter(kr));
  if (!Axb || !x || !rhs || !tol || !iter || !flag || L < 1 || L > 16 || *iter < 0)
    return kfail(kr, NS3D_ERR_BAD_ARG, "need 1 <= L <= 16, non-null pointers, *iter >= 0");
  kr->launches = 0;
  return bicgstabl(kr, L, Axb, user, x, rhs, tol, iter, flag);
}

ns3d_status ns3d_newton(ns3d_krylov* kr, ns3d_user_map_vector jacobian, void* jacobian_user,
                        ns3d_user_map_vector residual, void* residual_user, double* x,
                        double* tol, int* iter, double tol_linsolve, int iter_linsolve,
                        int* flag, int* linsolve_flag) {
  KR_TRY(enter(kr));
  if (!jacobian || !residual || !x || !tol || !iter || !flag || !linsolve_flag || *iter < 0 ||
      kr->n < 5)
    return kfail(kr, NS3D_ERR_BAD_ARG, "need non-null maps and pointers, *iter >= 0, n >= 5");
  const int64_t n = kr->n;
  kr->launches = 0;
  if (!kr->newton)
    KR_CHECK(kr, cudaMalloc(&kr->newton, sizeof(double) * 2 * (size_t)n), "Newton vectors");
  double* delta = kr->newton;
  double* bn = kr->newton + n;
  newton_start<<<blocks_for(n, kThreads, kMaxBlocks * 2), kThreads, 0, kr->stream>>>(n, delta);
  KR_CHECK(kr, cudaGetLastError(), "newton_start");
  constexpr double kDamping = 0.8;  // Newton.cu:66
  constexpr int kL = 6;             // Newton.cu:21
  *linsolve_flag = 0;
  int fl = 1, ll = 0;
  double norm_rhs = 0.0;
  KR_TRY(apply_map(kr, residual, residual_user, x, bn));
  KR_TRY(norm2(kr, bn, &norm_rhs));
  if (norm_rhs < *tol) {
    fl = 0;
  } else {
    for (ll = 0; ll < *iter; ++ll) {
      double tol_b = tol_linsolve;
      int it_b = iter_linsolve, lf = 0;
      KR_TRY(apply_map(kr, residual, residual_user, x, bn));
      KR_TRY(combine(kr, -1.0, bn, 0.0, nullptr, bn));
      KR_TRY(bicgstabl(kr, kL, jacobian, jacobian_user, delta, bn, &tol_b, &it_b, &lf));
      if (lf != 0) {  // the reference prints and exits here
        *linsolve_flag = lf;
        *iter = ll;
        *flag = 2;
        return NS3D_OK;
      }
      KR_TRY(combine(kr, kDamping, delta, 1.0, x, x));
      double tol_newton = 0.0;
      KR_TRY(norm2(kr, delta, &tol_newton));
      KR_TRY(norm2(kr, bn, &norm_rhs));
      if (!std::isfinite(tol_newton) || !std::isfinite(norm_rhs))
        return kfail(kr, NS3D_ERR_NONFINITE, "Newton update is not finite");
      if (norm_rhs < *tol && ll > 2) {
        *tol = tol_newton;
        fl = 0;
        break;
      }
    }
  }
  *iter = ll;
  *flag = fl;
  return NS3D_OK;
}

// ---------------------------------------------------------------------------
// built-in matrix-vector maps
// ---------------------------------------------------------------------------

static void map_poison(ns3d_map_context* c, double* out) {
  const int64_t n = ns3d_krylov_length(c->solver);
  if (n > 0 && out) cudaMemset(out, 0xff, sizeof(double) * n);  // NaN: the driver stops
}

void ns3d_map_linearised(void* user, void* in, void* out) {
  ns3d_map_context* c = static_cast<ns3d_map_context*>(user);
  if (!c) return;
  ns3d_status s = ns3d_matvec_reduced(c->solver, c->ux, c->uy, c->uz,
                                      static_cast<const double*>(in), static_cast<double*>(out),
                                      c->Re, c->tau);
  if (s == NS3D_OK) s = ns3d_synchronize(c->solver);
  if (s != NS3D_OK) {
    if (c->status == NS3D_OK) c->status = s;
    map_poison(c, static_cast<double*>(out));
  }
}

void ns3d_map_rhs(void* user, void* in, void* out) {
  ns3d_map_context* c = static_cast<ns3d_map_context*>(user);
  if (!c) return;
  ns3d_status s = ns3d_unpack_reduced(c->solver, static_cast<const double*>(in), c->ux, c->uy,
                                      c->uz);
  if (s == NS3D_OK) s = ns3d_rhs(c->solver, c->ux, c->uy, c->uz, c->vx, c->vy, c->vz, c->Re);
  if (s == NS3D_OK)
    s = ns3d_pack_reduced(c->solver, c->vx, c->vy, c->vz, static_cast<double*>(out));
  if (s == NS3D_OK) s = ns3d_synchronize(c->solver);
  if (s != NS3D_OK) {
    if (c->status == NS3D_OK) c->status = s;
    map_poison(c, static_cast<double*>(out));
  }
}

void ns3d_map_exponential(void* user, void* in, void* out) {
  ns3d_map_context* c = static_cast<ns3d_map_context*>(user);
  if (!c) return;
  ns3d_status s = ns3d_unpack_reduced(c->solver, static_cast<const double*>(in), c->vx, c->vy,
                                      c->vz);
  if (s == NS3D_OK)
    s = ns3d_jvp_steps(c->solver, c->ux, c->uy, c->uz, c->vx, c->vy, c->vz, c->dt, c->Re,
                       c->steps);
  if (s == NS3D_OK)
    s = ns3d_pack_reduced(c->solver, c->vx, c->vy, c->vz, static_cast<double*>(out));
  if (s == NS3D_OK) s = ns3d_synchronize(c->solver);
  if (s != NS3D_OK) {
    if (c->status == NS3D_OK) c->status = s;
    map_poison(c, static_cast<double*>(out));
  }
}

// Shift-invert maps.  E = `steps` implicit tangent steps of v = unpack(in)
// about the fixed base flow; the result stays in the context's v fields.
static ns3d_status implicit_tangent_steps(ns3d_map_context* c, const double* in) {
  ns3d_status s = ns3d_unpack_reduced(c->solver, in, c->vx, c->vy, c->vz);
  for (int t = 0; t < c->steps && s == NS3D_OK; ++t)
    s = ns3d_implicit_tangent_step(c->solver, c->ux, c->uy, c->uz, c->vx, c->vy, c->vz, c->dt,
                                   c->Re);
  return s;
}

static void shift_map_fail(ns3d_shift_invert_context* c, ns3d_status s, double* out,
                           int64_t count) {
  if (c->map.status == NS3D_OK) c->map.status = s;
  if (count > 0 && out) cudaMemset(out, 0xff, sizeof(double) * count);
}

void ns3d_map_exponential_shifted(void* user, void* in, void* out) {
  ns3d_shift_invert_context* c = static_cast<ns3d_shift_invert_context*>(user);
  if (!c) return;
  ns3d_map_context* m = &c->map;
  const double* x = static_cast<const double*>(in);
  ns3d_status s = implicit_tangent_steps(m, x);
  if (s == NS3D_OK)
    s = ns3d_pack_reduced_shifted(m->solver, m->vx, m->vy, m->vz, x, c->shift_real, nullptr,
                                  0.0, static_cast<double*>(out));
  if (s == NS3D_OK) s = ns3d_synchronize(m->solver);
  if (s != NS3D_OK)
    shift_map_fail(c, s, static_cast<double*>(out), ns3d_krylov_length(m->solver));
}

void ns3d_map_exponential_rotated(void* user, void* in, void* out) {
  ns3d_shift_invert_context* c = static_cast<ns3d_shift_invert_context*>(user);
  if (!c) return;
  ns3d_map_context* m = &c->map;
  const int64_t n = ns3d_krylov_length(m->solver);
  const double sr = c->shift_real * std::cos(c->rotate_angle);
  const double si = c->shift_real * std::sin(c->rotate_angle);
  const double* xr = static_cast<const double*>(in);
  const double* xi = xr + n;
  double* yr = static_cast<double*>(out);
  double* yi = yr + n;
  ns3d_status s = implicit_tangent_steps(m, xr);
  if (s == NS3D_OK)
    s = ns3d_pack_reduced_shifted(m->solver, m->vx, m->vy, m->vz, xr, sr, xi, si, yr);
  if (s == NS3D_OK) s = implicit_tangent_steps(m, xi);
  if (s == NS3D_OK)
    s = ns3d_pack_reduced_shifted(m->solver, m->vx, m->vy, m->vz, xi, sr, xr, -si, yi);
  if (s == NS3D_OK) s = ns3d_synchronize(m->solver);
  if (s != NS3D_OK) shift_map_fail(c, s, yr, 2 * n);
}

static void exponent_invert(ns3d_shift_invert_context* c, ns3d_user_map_vector A, int64_t n,
                            const double* rhs, double* x) {
  ns3d_krylov* kr = c->inner;
  if (!kr || kr->n != n || !rhs || !x || c->L < 1 || c->L > 16 || c->max_iter < 0) {
    shift_map_fail(c, NS3D_ERR_BAD_ARG, x, n);
    return;
  }
  if (!c->warm_start) {
    cudaError_t e = cudaMemsetAsync(x, 0, sizeof(double) * n, kr->stream);
    if (e != cudaSuccess) {
      shift_map_fail(c, NS3D_ERR_CUDA, x, n);
      return;
    }
  }
  double tol = c->tol;
  int iter = c->max_iter, flag = 1;
  ns3d_status s = ns3d_bicgstabl(kr, c->L, A, c, x, rhs, &tol, &iter, &flag);
  c->last_flag = flag;
  c->last_iter = iter;
  c->last_tol = tol;
  c->solves += 1;
  c->inner_iter += iter;
  if (s == NS3D_OK && c->map.status != NS3D_OK) s = (ns3d_status)c->map.status;
  if (s == NS3D_OK && flag != 0)
    s = flag == -3 ? NS3D_ERR_NONFINITE : NS3D_ERR_NOT_CONVERGED;
  if (s != NS3D_OK) shift_map_fail(c, s, x, n);
}

void ns3d_map_exponent_invert(void* user, void* in, void* out) {
  ns3d_shift_invert_context* c = static_cast<ns3d_shift_invert_context*>(user);
  if (!c) return;
  exponent_invert(c, ns3d_map_exponential_shifted, ns3d_krylov_length(c->map.solver),
                  static_cast<const double*>(in), static_cast<double*>(out));
}

void ns3d_map_rotated_exponent_invert(void* user, void* in, void* out) {
  ns3d_shift_invert_context* c = static_cast<ns3d_shift_invert_context*>(user);
  if (!c) return;
  exponent_invert(c, ns3d_map_exponential_rotated, 2 * ns3d_krylov_length(c->map.solver),
                  static_cast<const double*>(in), static_cast<double*>(out));
}

void ns3d_map_laplace1d(void* user, void* in, void* out) {
  ns3d_laplace_context* c = static_cast<ns3d_laplace_context*>(user);
  if (!c) return;
  if (c->n < 2 || !in || !out) {
    if (c->status == NS3D_OK) c->status = NS3D_ERR_BAD_ARG;
    return;
  }
  cudaStream_t st = (cudaStream_t)c->stream;
  laplace1d_kernel<<<blocks_for(c->n, kThreads, kMaxBlocks * 2), kThreads, 0, st>>>(
      static_cast<const double*>(in), static_cast<double*>(out), c->n);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess && c->status == NS3D_OK) c->status = NS3D_ERR_CUDA;
}

}  // extern "C"
