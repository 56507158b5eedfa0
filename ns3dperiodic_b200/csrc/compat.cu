// The reference's C++ entry points (include/ns3d_compat.h) over the C ABI of
// include/ns3d.h.  Built into its own library, libns3d_compat.so, which uses
// only the public C ABI of libns3d_b200.so plus a few pointwise kernels of
// its own for the reference functions that work on caller-built tables.
//
// Grid handles: one ns3d_solver per (device, Nx, Ny, Nz, Lx, Ly, Lz),
// created on first use and kept until clean_dealiasing().  The steppers get
// the box from dx*N; the convolutions from the first entry of the nabla
// tables (build_Nabla_Wavenumbers stores 2 pi / L * m).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "ns3d.h"
#include "ns3d_compat.h"

namespace {

using cplx = cufftDoubleComplex;

struct Grid {
  int dev, Nx, Ny, Nz;
  double Lx, Ly, Lz;
  bool operator<(const Grid& o) const {
    return std::tie(dev, Nx, Ny, Nz, Lx, Ly, Lz) <
           std::tie(o.dev, o.Nx, o.Ny, o.Nz, o.Lx, o.Ly, o.Lz);
  }
};

struct Entry {
  ns3d_solver* h = nullptr;
  const void* f[3] = {nullptr, nullptr, nullptr};
  bool f_set = false;
};

std::mutex g_mu;
std::map<Grid, Entry> g_solvers;
Entry* g_current = nullptr;
bool g_forcing_dirty = false;
std::map<std::tuple<const double*, const double*, const double*>, std::tuple<double, double, double>>
    g_box_from_tables;

void report(ns3d_status s, ns3d_solver* h, const char* where, bool fatal) {
  if (s == NS3D_OK) return;
  std::fprintf(stderr, "%s failed: %s%s%s\n", where, ns3d_status_string(s),
               h ? ": " : "", h ? ns3d_last_error(h) : "");
  if (fatal) std::exit(1);
}

Entry* entry_for(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz) {
  std::lock_guard<std::mutex> lock(g_mu);
  int dev = 0;
  cudaGetDevice(&dev);
  Grid key{dev, Nx, Ny, Nz, Lx, Ly, Lz};
  auto it = g_solvers.find(key);
  if (it == g_solvers.end()) {
    Entry e;
    const ns3d_status s = ns3d_create(Nx, Ny, Nz, Lx, Ly, Lz, &e.h);
    // the reference exits when it cannot allocate its arrays
    report(s, nullptr, "ns3d_create", true);
    it = g_solvers.emplace(key, e).first;
  }
  g_current = &it->second;
  return &it->second;
}

// Any handle with this grid (the plain transforms do not depend on the box).
Entry* entry_any_box(int Nx, int Ny, int Nz) {
  {
    std::lock_guard<std::mutex> lock(g_mu);
    int dev = 0;
    cudaGetDevice(&dev);
    for (auto& kv : g_solvers)
      if (kv.first.dev == dev && kv.first.Nx == Nx && kv.first.Ny == Ny && kv.first.Nz == Nz) {
        g_current = &kv.second;
        return &kv.second;
      }
  }
  const double two_pi = 2.0 * M_PI;
  return entry_for(Nx, Ny, Nz, two_pi, two_pi, two_pi);
}

Entry* entry_from_steps(int Nx, int Ny, int Nz, double dx, double dy, double dz) {
  return entry_for(Nx, Ny, Nz, dx * Nx, dy * Ny, dz * Nz);
}

// Box lengths from the nabla tables: k[1] = 2 pi / L.
Entry* entry_from_tables(int Nx, int Ny, int Nz, const double* kx, const double* ky,
                         const double* kz) {
  auto key = std::make_tuple(kx, ky, kz);
  double L[3];
  {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_box_from_tables.find(key);
    if (it != g_box_from_tables.end()) {
      L[0] = std::get<0>(it->second);
      L[1] = std::get<1>(it->second);
      L[2] = std::get<2>(it->second);
    } else {
      double k1[3] = {0, 0, 0};
      const double* t[3] = {kx, ky, kz};
      for (int d = 0; d < 3; ++d)
        if (cudaMemcpy(&k1[d], t[d] + 1, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
            !(k1[d] > 0.0)) {
          std::fprintf(stderr, "calculate_convolution_2p3: unreadable nabla table\n");
          std::exit(1);
        }
      for (int d = 0; d < 3; ++d) L[d] = 2.0 * M_PI / k1[d];
      g_box_from_tables[key] = std::make_tuple(L[0], L[1], L[2]);
    }
  }
  return entry_for(Nx, Ny, Nz, L[0], L[1], L[2]);
}

void use_forcing(Entry* e, const cplx* fx, const cplx* fy, const cplx* fz) {
  if (e->f_set && !g_forcing_dirty && e->f[0] == fx && e->f[1] == fy && e->f[2] == fz) return;
  const ns3d_status s = ns3d_set_forcing(e->h, (const ns3d_complex*)fx, (const ns3d_complex*)fy,
                                         (const ns3d_complex*)fz);
  report(s, e->h, "forcing", false);
  e->f[0] = fx;
  e->f[1] = fy;
  e->f[2] = fz;
  e->f_set = true;
  g_forcing_dirty = false;
}

inline ns3d_complex* C(cplx* p) { return reinterpret_cast<ns3d_complex*>(p); }

// ---------------------------------------------------------------------------
// pointwise kernels on caller tables (flat index over Nx*Ny*Nz points; the
// callers pass Mz as Nz for spectral arrays)
// ---------------------------------------------------------------------------
enum TableMode : int {
  kExplicitF = 0,  // u <- dt(AM.Q - Q) + (1 - dt din/Re) u + dt f
  kExplicit = 1,   // v <- dt(AM.Q - Q) + (1 - dt din/Re) v
  kImplicit = 2,   // v <- (dt(AM.Q - Q) + v) / (1 + dt din/Re)
  kRhsInPlace = 3, // v <- (AM.Q - Q) - din/Re v
  kRhsF = 4,       // rhs <- (AM.Q - Q) - din/Re u + f
};

struct TableArgs {
  const double* din;
  const double* am[6];  // 11, 22, 33, 12, 13, 23
  cplx* u[3];
  const cplx* f[3];
  const cplx* q[3];
  cplx* out[3];
  double Re, dt;
  long long n;
};

template <int MODE>
__global__ void table_update(TableArgs a) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    const double a11 = a.am[0][i], a22 = a.am[1][i], a33 = a.am[2][i];
    const double a12 = a.am[3][i], a13 = a.am[4][i], a23 = a.am[5][i];
    const cplx q0 = a.q[0][i], q1 = a.q[1][i], q2 = a.q[2][i];
    // P Q - Q with the symmetric Leray matrix, real and imaginary parts
    double p[3][2];
    p[0][0] = a11 * q0.x + a12 * q1.x + a13 * q2.x - q0.x;
    p[0][1] = a11 * q0.y + a12 * q1.y + a13 * q2.y - q0.y;
    p[1][0] = a12 * q0.x + a22 * q1.x + a23 * q2.x - q1.x;
    p[1][1] = a12 * q0.y + a22 * q1.y + a23 * q2.y - q1.y;
    p[2][0] = a13 * q0.x + a23 * q1.x + a33 * q2.x - q2.x;
    p[2][1] = a13 * q0.y + a23 * q1.y + a33 * q2.y - q2.y;
    const double din = a.din[i];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const cplx u = a.u[c][i];
      cplx r;
      if (MODE == kExplicitF || MODE == kExplicit) {
        const double G = 1.0 - din * a.dt / a.Re;
        r.x = a.dt * p[c][0] + G * u.x;
        r.y = a.dt * p[c][1] + G * u.y;
        if (MODE == kExplicitF) {
          r.x += a.dt * a.f[c][i].x;
          r.y += a.dt * a.f[c][i].y;
        }
      } else if (MODE == kImplicit) {
        const double G = 1.0 + din * a.dt / a.Re;
        r.x = (a.dt * p[c][0] + u.x) / G;
        r.y = (a.dt * p[c][1] + u.y) / G;
      } else {
        const double G = -din / a.Re;
        r.x = p[c][0] + G * u.x;
        r.y = p[c][1] + G * u.y;
        if (MODE == kRhsF) {
          r.x += a.f[c][i].x;
          r.y += a.f[c][i].y;
        }
      }
      if (MODE == kRhsF)
        a.out[c][i] = r;
      else
        a.u[c][i] = r;
    }
  }
}

unsigned grid_for(long long n) {
  long long b = (n + 255) / 256;
  return (unsigned)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

template <int MODE>
void run_table(TableArgs a) {
  table_update<MODE><<<grid_for(a.n), 256>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) std::fprintf(stderr, "table update: %s\n", cudaGetErrorString(e));
}

TableArgs table_args(int Nx, int Ny, int Nz, const double* din, cplx* u0, cplx* u1, cplx* u2,
                     const double* a11, const double* a22, const double* a33, const double* a12,
                     const double* a13, const double* a23, const cplx* q0, const cplx* q1,
                     const cplx* q2, double Re, double dt) {
  TableArgs a{};
  a.din = din;
  a.am[0] = a11; a.am[1] = a22; a.am[2] = a33; a.am[3] = a12; a.am[4] = a13; a.am[5] = a23;
  a.u[0] = u0; a.u[1] = u1; a.u[2] = u2;
  a.q[0] = q0; a.q[1] = q1; a.q[2] = q2;
  a.Re = Re;
  a.dt = dt;
  a.n = (long long)Nx * Ny * Nz;
  return a;
}

// Re := 0 everywhere, the (0,0,0) mode := 0 (set_to_zero_real)
__global__ void zero_real(cplx* a0, cplx* a1, cplx* a2, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    a0[i].x = 0.0; a1[i].x = 0.0; a2[i].x = 0.0;
    if (i == 0) { a0[0].y = 0.0; a1[0].y = 0.0; a2[0].y = 0.0; }
  }
}

__global__ void split_complex(const cplx* u, double* re, double* im, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const cplx v = u[i];
    re[i] = v.x;
    im[i] = v.y;
  }
}

__global__ void merge_complex(const double* re, const double* im, cplx* u, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    u[i] = make_cuDoubleComplex(re[i], im[i]);
}

// div = i k.u / dt with the caller's nabla tables
__global__ void divergence_kernel(cplx* div, const cplx* ux, const cplx* uy, const cplx* uz,
                                  const double* kx, const double* ky, const double* kz, int Ny,
                                  int Nz, long long n, double dt) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const long long t = i / Nz;
    const int l = (int)(i - t * Nz);
    const int j = (int)(t / Ny);
    const int k = (int)(t - (long long)j * Ny);
    const cplx a = ux[i], b = uy[i], c = uz[i];
    div[i].x = (-a.y * kx[j] - b.y * ky[k] - c.y * kz[l]) / dt;
    div[i].y = (a.x * kx[j] + b.x * ky[k] + c.x * kz[l]) / dt;
  }
}

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// per-block partial sums of the reference's energy (0.5 (uy^2 + uz^2) dx dy)
// or central-difference dissipation density
template <bool DISS>
__global__ void physical_sum(const double* ux, const double* uy, const double* uz, int Nx, int Ny,
                             int Nz, double dx, double dy, double dz, double* part) {
  __shared__ double red[256 / 32];
  const long long n = (long long)Nx * Ny * Nz;
  const long long stride = (long long)gridDim.x * blockDim.x;
  double s = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    if (!DISS) {
      s += 0.5 * (uy[i] * uy[i] + uz[i] * uz[i]) * dx * dy;
    } else {
      const long long t = i / Nz;
      const int l = (int)(i - t * Nz);
      const int j = (int)(t / Ny);
      const int k = (int)(t - (long long)j * Ny);
      auto at = [&](const double* f, int jj, int kk, int ll) {
        return f[((long long)wrap(jj, Nx) * Ny + wrap(kk, Ny)) * Nz + wrap(ll, Nz)];
      };
      const double ux_x = (at(ux, j + 1, k, l) - at(ux, j - 1, k, l)) / dx;
      const double ux_y = (at(ux, j, k + 1, l) - at(ux, j, k - 1, l)) / dy;
      const double ux_z = (at(ux, j, k, l + 1) - at(ux, j, k, l - 1)) / dz;
      const double uy_x = (at(uy, j + 1, k, l) - at(uy, j - 1, k, l)) / dx;
      const double uy_y = (at(uy, j, k + 1, l) - at(uy, j, k - 1, l)) / dy;
      const double uy_z = (at(uy, j, k, l + 1) - at(uy, j, k, l - 1)) / dz;
      const double uz_x = (at(uz, j + 1, k, l) - at(uz, j - 1, k, l)) / dx;
      const double uz_y = (at(uz, j, k + 1, l) - at(uz, j, k - 1, l)) / dy;
      const double uz_z = (at(uz, j, k, l + 1) - at(uz, j, k, l - 1)) / dz;
      s += dx * dy * dz *
           (2.0 * (ux_x * ux_x + uy_y * uy_y + uz_z * uz_z) + (uy_z + uz_y) * (uy_z + uz_y) +
            (ux_z + uz_x) * (ux_z + uz_x) + (ux_y + uy_x) * (ux_y + uy_x));
    }
  }
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int w = 0; w < 256 / 32; ++w) b += red[w];
    part[blockIdx.x] = b;
  }
}

double physical_reduce(bool diss, int Nx, int Ny, int Nz, double dx, double dy, double dz,
                       const double* ux, const double* uy, const double* uz) {
  constexpr int kBlocks = 592;
  double* part = nullptr;
  if (cudaMalloc(&part, sizeof(double) * kBlocks) != cudaSuccess) {
    std::fprintf(stderr, "reduction: out of device memory\n");
    std::exit(1);
  }
  if (diss)
    physical_sum<true><<<kBlocks, 256>>>(ux, uy, uz, Nx, Ny, Nz, dx, dy, dz, part);
  else
    physical_sum<false><<<kBlocks, 256>>>(ux, uy, uz, Nx, Ny, Nz, dx, dy, dz, part);
  std::vector<double> h(kBlocks);
  cudaMemcpy(h.data(), part, sizeof(double) * kBlocks, cudaMemcpyDeviceToHost);
  cudaFree(part);
  double s = 0.0;
  for (double v : h) s += v;
  return s;
}

void c2r_scaled(int Nx, int Ny, int Nz, cplx* src, double* dst) {
  Entry* e = entry_any_box(Nx, Ny, Nz);
  report(ns3d_fft_c2r(e->h, C(src), dst), e->h, "iFFTN_Device", false);
}

}  // namespace

// ---------------------------------------------------------------------------
// RK_time_step.h
// ---------------------------------------------------------------------------
void copy_arrays(dim3, dim3, int Nx, int Ny, int Nz, cplx* s1, cplx* s2, cplx* s3, cplx* d1,
                 cplx* d2, cplx* d3) {
  const size_t b = sizeof(cplx) * (size_t)Nx * Ny * Nz;
  cudaMemcpyAsync(d1, s1, b, cudaMemcpyDeviceToDevice, 0);
  cudaMemcpyAsync(d2, s2, b, cudaMemcpyDeviceToDevice, 0);
  cudaMemcpyAsync(d3, s3, b, cudaMemcpyDeviceToDevice, 0);
}

void single_time_step(dim3, dim3, dim3, dim3, double dx, double dy, double dz, double dt,
                      double Re, int Nx, int Ny, int Nz, int, cplx* ux, cplx* uy, cplx* uz,
                      cplx* fx, cplx* fy, cplx* fz, cplx*, cplx*, cplx*, cplx*, double*, double*,
                      double*, double*, double*, cplx*, cplx*, cplx*, double*, double*, double*,
                      double*, double*, double*) {
  Entry* e = entry_from_steps(Nx, Ny, Nz, dx, dy, dz);
  use_forcing(e, fx, fy, fz);
  report(ns3d_euler_step(e->h, C(ux), C(uy), C(uz), dt, Re), e->h, "single_time_step", false);
}

void single_time_step_UV(dim3, dim3, dim3, dim3, double dx, double dy, double dz, double dt,
                         double Re, int Nx, int Ny, int Nz, int, cplx* ux, cplx* uy, cplx* uz,
                         cplx* vx, cplx* vy, cplx* vz, cplx*, cplx*, cplx*, cplx*, double*,
                         double*, double*, double*, double*, double*, double*, double*, double*,
                         double*, double*) {
  Entry* e = entry_from_steps(Nx, Ny, Nz, dx, dy, dz);
  report(ns3d_tangent_euler_step(e->h, C(ux), C(uy), C(uz), C(vx), C(vy), C(vz), dt, Re), e->h,
         "single_time_step_UV", false);
}

void single_time_step_iUV_RHS(dim3, dim3, dim3, dim3, double dx, double dy, double dz, double dt,
                              double Re, int Nx, int Ny, int Nz, int, cplx* ux, cplx* uy,
                              cplx* uz, cplx* vx, cplx* vy, cplx* vz, cplx*, cplx*, cplx*, cplx*,
                              double*, double*, double*, double*, double*, double*, double*,
                              double*, double*, double*, double*) {
  Entry* e = entry_from_steps(Nx, Ny, Nz, dx, dy, dz);
  report(ns3d_implicit_tangent_step(e->h, C(ux), C(uy), C(uz), C(vx), C(vy), C(vz), dt, Re),
         e->h, "single_time_step_iUV_RHS", false);
}

void RK3_SSP(dim3, dim3, dim3, dim3, double dx, double dy, double dz, double dt, double Re,
             int Nx, int Ny, int Nz, int, cplx* ux, cplx* uy, cplx* uz, cplx*, cplx*, cplx*,
             cplx*, cplx*, cplx*, cplx*, cplx*, cplx*, cplx* fx, cplx* fy, cplx* fz, cplx*, cplx*,
             cplx*, cplx*, double*, double*, double*, double*, double*, double*, double*,
             double*, double*, double*, double*) {
  Entry* e = entry_from_steps(Nx, Ny, Nz, dx, dy, dz);
  use_forcing(e, fx, fy, fz);
  report(ns3d_rk3_step(e->h, C(ux), C(uy), C(uz), dt, Re), e->h, "RK3_SSP", false);
}

void RK3_SSP_UV_RHS(dim3, dim3, dim3, dim3, double dx, double dy, double dz, double, double Re,
                    int Nx, int Ny, int Nz, int, cplx* ux, cplx* uy, cplx* uz, cplx* vx,
                    cplx* vy, cplx* vz, cplx*, cplx*, cplx*, cplx*, cplx*, cplx*, cplx*, cplx*,
                    cplx*, cplx*, cplx*, cplx*, cplx*, cplx*, cplx*, cplx*, double*, double*,
                    double*, double*, double*, double*, double*, double*, double*, double*,
                    double*) {
  Entry* e = entry_from_steps(Nx, Ny, Nz, dx, dy, dz);
  report(ns3d_linearised_rhs(e->h, C(ux), C(uy), C(uz), C(vx), C(vy), C(vz), Re), e->h,
         "RK3_SSP_UV_RHS", false);
}

void RK3_SSP_UV(dim3, dim3, dim3, dim3, double dx, double dy, double dz, double dt, double Re,
                int Nx, int Ny, int Nz, int, cplx* ux, cplx* uy, cplx* uz, cplx* vx, cplx* vy,
                cplx* vz, cplx*, cplx*, cplx*, cplx*, cplx*, cplx*, cplx*, cplx*, cplx*, cplx*,
                cplx*, cplx*, cplx* fx, cplx* fy, cplx* fz, cplx*, cplx*, cplx*, cplx*, double*,
                double*, double*, double*, double*, double*, double*, double*, double*, double*,
                double*) {
  Entry* e = entry_from_steps(Nx, Ny, Nz, dx, dy, dz);
  use_forcing(e, fx, fy, fz);
  report(ns3d_jvp_step(e->h, C(ux), C(uy), C(uz), C(vx), C(vy), C(vz), dt, Re), e->h,
         "RK3_SSP_UV", false);
}

void return_RHS(dim3, dim3, dim3, dim3, double dx, double dy, double dz, double Re, int Nx,
                int Ny, int Nz, int, cplx* ux, cplx* uy, cplx* uz, cplx* fx, cplx* fy, cplx* fz,
                cplx*, cplx*, cplx*, cplx*, double*, double*, double*, double*, double*, double*,
                double*, double*, double*, double*, double*, cplx* rx, cplx* ry, cplx* rz) {
  Entry* e = entry_from_steps(Nx, Ny, Nz, dx, dy, dz);
  use_forcing(e, fx, fy, fz);
  report(ns3d_rhs(e->h, C(ux), C(uy), C(uz), C(rx), C(ry), C(rz), Re), e->h, "return_RHS",
         false);
}

// ---------------------------------------------------------------------------
// advection_2_3.h
// ---------------------------------------------------------------------------
void set_to_zero(dim3, dim3, int Nx, int Ny, int Nz, cplx* a1, cplx* a2, cplx* a3) {
  const long long n = (long long)Nx * Ny * Nz;
  zero_real<<<grid_for(n), 256>>>(a1, a2, a3, n);
}

void init_dealiasing(dim3, dim3, dim3, dim3, int, int, int, int, double*) {
  // the handle owns its scratch and evaluates the 2/3 mask from indices;
  // handles are created on first use
}

void clean_dealiasing() {
  std::lock_guard<std::mutex> lock(g_mu);
  for (auto& kv : g_solvers) ns3d_destroy(kv.second.h);
  g_solvers.clear();
  g_box_from_tables.clear();
  g_current = nullptr;
}

void calculate_convolution_2p3(dim3, dim3, dim3, dim3, int Nx, int Ny, int Nz, int, cplx* ux,
                               cplx* uy, cplx* uz, double* kx, double* ky, double* kz, cplx* Qx,
                               cplx* Qy, cplx* Qz) {
  Entry* e = entry_from_tables(Nx, Ny, Nz, kx, ky, kz);
  report(ns3d_convolution(e->h, C(ux), C(uy), C(uz), C(Qx), C(Qy), C(Qz)), e->h,
         "calculate_convolution_2p3", false);
}

void calculate_convolution_2p3_UV(dim3, dim3, dim3, dim3, int Nx, int Ny, int Nz, int, cplx* ux,
                                  cplx* uy, cplx* uz, cplx* vx, cplx* vy, cplx* vz, double* kx,
                                  double* ky, double* kz, cplx* Qx, cplx* Qy, cplx* Qz) {
  Entry* e = entry_from_tables(Nx, Ny, Nz, kx, ky, kz);
  report(ns3d_convolution_uv(e->h, C(ux), C(uy), C(uz), C(vx), C(vy), C(vz), C(Qx), C(Qy),
                             C(Qz)),
         e->h, "calculate_convolution_2p3_UV", false);
}

// ---------------------------------------------------------------------------
// diffusion.h
// ---------------------------------------------------------------------------
void diffusion_device(int, int, int, double*, cplx*, cplx*, cplx*, cplx*, cplx*, cplx*, double,
                      double, cplx*, cplx*, cplx*) {
  // the reference's body is empty (Source/diffusion.cu)
}

void velocity_to_double(dim3, dim3, int Nx, int Ny, int Nz, cplx* ux_hat, double* ux,
                        cplx* uy_hat, double* uy, cplx* uz_hat, double* uz) {
  c2r_scaled(Nx, Ny, Nz, ux_hat, ux);
  c2r_scaled(Nx, Ny, Nz, uz_hat, uz);
  c2r_scaled(Nx, Ny, Nz, uy_hat, uy);
}

void solve_advection_diffusion_projection(dim3, dim3, int Nx, int Ny, int Nz, double* din,
                                          cplx* ux, cplx* uy, cplx* uz, cplx* fx, cplx* fy,
                                          cplx* fz, double Re, double dt, cplx* Qx, cplx* Qy,
                                          cplx* Qz, double* a11, double* a22, double* a33,
                                          double* a12, double* a13, double* a23) {
  TableArgs a = table_args(Nx, Ny, Nz, din, ux, uy, uz, a11, a22, a33, a12, a13, a23, Qx, Qy, Qz,
                           Re, dt);
  a.f[0] = fx; a.f[1] = fy; a.f[2] = fz;
  run_table<kExplicitF>(a);
}

void solve_advection_diffusion_projection_UV(dim3, dim3, int Nx, int Ny, int Nz, double* din,
                                             cplx* vx, cplx* vy, cplx* vz, double Re, double dt,
                                             cplx* Qx, cplx* Qy, cplx* Qz, double* a11,
                                             double* a22, double* a33, double* a12, double* a13,
                                             double* a23) {
  run_table<kExplicit>(table_args(Nx, Ny, Nz, din, vx, vy, vz, a11, a22, a33, a12, a13, a23, Qx,
                                  Qy, Qz, Re, dt));
}

void solve_advection_implicit_diffusion_projection_UV(dim3, dim3, int Nx, int Ny, int Nz,
                                                      double* din, cplx* vx, cplx* vy, cplx* vz,
                                                      double Re, double dt, cplx* Qx, cplx* Qy,
                                                      cplx* Qz, double* a11, double* a22,
                                                      double* a33, double* a12, double* a13,
                                                      double* a23) {
  run_table<kImplicit>(table_args(Nx, Ny, Nz, din, vx, vy, vz, a11, a22, a33, a12, a13, a23, Qx,
                                  Qy, Qz, Re, dt));
}

void solve_advection_diffusion_projection_UV_RHS(dim3, dim3, int Nx, int Ny, int Nz, double* din,
                                                 cplx* vx, cplx* vy, cplx* vz, double Re,
                                                 double dt, cplx* Qx, cplx* Qy, cplx* Qz,
                                                 double* a11, double* a22, double* a33,
                                                 double* a12, double* a13, double* a23) {
  run_table<kRhsInPlace>(table_args(Nx, Ny, Nz, din, vx, vy, vz, a11, a22, a33, a12, a13, a23,
                                    Qx, Qy, Qz, Re, dt));
}

void RHS_advection_diffusion_projection(dim3, dim3, int Nx, int Ny, int Nz, double* din,
                                        cplx* ux, cplx* uy, cplx* uz, cplx* fx, cplx* fy,
                                        cplx* fz, double Re, cplx* Qx, cplx* Qy, cplx* Qz,
                                        double* a11, double* a22, double* a33, double* a12,
                                        double* a13, double* a23, cplx* rx, cplx* ry,
                                        cplx* rz) {
  TableArgs a = table_args(Nx, Ny, Nz, din, ux, uy, uz, a11, a22, a33, a12, a13, a23, Qx, Qy, Qz,
                           Re, 0.0);
  a.f[0] = fx; a.f[1] = fy; a.f[2] = fz;
  a.out[0] = rx; a.out[1] = ry; a.out[2] = rz;
  run_table<kRhsF>(a);
}

// ---------------------------------------------------------------------------
// math_support.h
// ---------------------------------------------------------------------------
void init_fft_plans(cufftHandle, cufftHandle) {
  // transforms run on the handle of the grid in use; nothing to record
}

void FFTN_Device(double* source, cplx* destination) {
  Entry* e = g_current;
  if (!e) {
    std::fprintf(stderr, "*CUFFT R->C* failed: no grid in use\n");
    std::exit(1);
  }
  report(ns3d_fft_r2c(e->h, source, C(destination)), e->h, "*CUFFT R->C*", true);
}

void iFFTN_Device(cplx* source, double* destination) {
  Entry* e = g_current;
  if (!e) {
    std::fprintf(stderr, "*CUFFT C->R* failed: no grid in use\n");
    std::exit(1);
  }
  report(ns3d_fft_c2r_unscaled(e->h, C(source), destination), e->h, "*CUFFT C->R*", true);
}

void iFFTN_Device(dim3, dim3, cplx* source, double* destination, int Nx, int Ny, int Nz) {
  c2r_scaled(Nx, Ny, Nz, source, destination);
}

void Image_to_Domain(dim3, dim3, int Nx, int Ny, int Nz, double* ux, cplx* ux_hat, double* uy,
                     cplx* uy_hat, double* uz, cplx* uz_hat) {
  c2r_scaled(Nx, Ny, Nz, ux_hat, ux);
  c2r_scaled(Nx, Ny, Nz, uy_hat, uy);
  c2r_scaled(Nx, Ny, Nz, uz_hat, uz);
}

void Domain_to_Image(dim3, dim3, int Nx, int Ny, int Nz, cplx* ux_hat, double* ux, cplx* uy_hat,
                     double* uy, cplx* uz_hat, double* uz) {
  Entry* e = entry_any_box(Nx, Ny, Nz);
  report(ns3d_fft_r2c(e->h, ux, C(ux_hat)), e->h, "*CUFFT R->C*", true);
  report(ns3d_fft_r2c(e->h, uy, C(uy_hat)), e->h, "*CUFFT R->C*", true);
  report(ns3d_fft_r2c(e->h, uz, C(uz_hat)), e->h, "*CUFFT R->C*", true);
}

void all_Fourier2double(dim3, dim3, cplx* ux_hat, double* ux_re, double* ux_im, cplx* uy_hat,
                        double* uy_re, double* uy_im, cplx* uz_hat, double* uz_re, double* uz_im,
                        int Nx, int Ny, int Nz) {
  const long long n = (long long)Nx * Ny * Nz;
  split_complex<<<grid_for(n), 256>>>(ux_hat, ux_re, ux_im, n);
  split_complex<<<grid_for(n), 256>>>(uy_hat, uy_re, uy_im, n);
  split_complex<<<grid_for(n), 256>>>(uz_hat, uz_re, uz_im, n);
}

void all_double2Fourier(dim3, dim3, double* ux_re, double* ux_im, cplx* ux_hat, double* uy_re,
                        double* uy_im, cplx* uy_hat, double* uz_re, double* uz_im, cplx* uz_hat,
                        int Nx, int Ny, int Nz) {
  const long long n = (long long)Nx * Ny * Nz;
  merge_complex<<<grid_for(n), 256>>>(ux_re, ux_im, ux_hat, n);
  merge_complex<<<grid_for(n), 256>>>(uy_re, uy_im, uy_hat, n);
  merge_complex<<<grid_for(n), 256>>>(uz_re, uz_im, uz_hat, n);
}

void get_curl(dim3, dim3, int Nx, int Ny, int Nz, double dx, double dy, double dz, double* ux,
              double* uy, double* uz, double* rx, double* ry, double* rz) {
  Entry* e = entry_from_steps(Nx, Ny, Nz, dx, dy, dz);
  report(ns3d_curl(e->h, ux, uy, uz, rx, ry, rz), e->h, "get_curl", false);
}

namespace {
void filter_then_c2r(bool helmholtz, int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                     cplx* ux_hat, cplx* uy_hat, cplx* uz_hat, cplx* fx_hat, cplx* fy_hat,
                     cplx* fz_hat, double p, double* fx, double* fy, double* fz) {
  Entry* e = entry_for(Nx, Ny, Nz, Lx, Ly, Lz);
  const ns3d_status s =
      helmholtz ? ns3d_helmholtz_filter(e->h, C(ux_hat), C(uy_hat), C(uz_hat), p, C(fx_hat),
                                        C(fy_hat), C(fz_hat))
                : ns3d_cutoff_filter(e->h, C(ux_hat), C(uy_hat), C(uz_hat), p, C(fx_hat),
                                     C(fy_hat), C(fz_hat));
  report(s, e->h, helmholtz ? "Helmholz_Fourier_Filter" : "CutOff_Fourier_Filter", false);
  report(ns3d_fft_c2r(e->h, C(fx_hat), fx), e->h, "*CUFFT C->R*", false);
  report(ns3d_fft_c2r(e->h, C(fy_hat), fy), e->h, "*CUFFT C->R*", false);
  report(ns3d_fft_c2r(e->h, C(fz_hat), fz), e->h, "*CUFFT C->R*", false);
}
}  // namespace

void Helmholz_Fourier_Filter(dim3, dim3, dim3, dim3, int Nx, int Ny, int Nz, int, double Lx,
                             double Ly, double Lz, cplx* ux_hat, cplx* uy_hat, cplx* uz_hat,
                             cplx* fx_hat, cplx* fy_hat, cplx* fz_hat, double eps, double* fx,
                             double* fy, double* fz) {
  filter_then_c2r(true, Nx, Ny, Nz, Lx, Ly, Lz, ux_hat, uy_hat, uz_hat, fx_hat, fy_hat, fz_hat,
                  eps, fx, fy, fz);
}

void CutOff_Fourier_Filter(dim3, dim3, dim3, dim3, int Nx, int Ny, int Nz, int, double Lx,
                           double Ly, double Lz, cplx* ux_hat, cplx* uy_hat, cplx* uz_hat,
                           cplx* fx_hat, cplx* fy_hat, cplx* fz_hat, double radius, double* fx,
                           double* fy, double* fz) {
  filter_then_c2r(false, Nx, Ny, Nz, Lx, Ly, Lz, ux_hat, uy_hat, uz_hat, fx_hat, fy_hat, fz_hat,
                  radius, fx, fy, fz);
}

void calculate_energy_spectrum(char* file_name, int Nx, int Ny, int Mz, double* ux_re,
                               double* ux_im, double* uy_re, double* uy_im, double* uz_re,
                               double* uz_im) {
  // host arrays, summed in the reference's loop order so the text is identical
  const int size = Nx / 2 + Ny / 2 + Mz;
  const int norm = Nx * Ny * Mz;
  std::vector<double> E(size, 0.0);
  for (int j = 0; j < Nx / 2; ++j)
    for (int k = 0; k < Ny / 2; ++k)
      for (int l = 0; l < Mz; ++l) {
        const size_t i = ((size_t)j * Ny + k) * Mz + l;
        const int n = j + k + l;
        E[n] += ux_re[i] * ux_re[i] / norm / norm + ux_im[i] * ux_im[i] / norm / norm;
        E[n] += uy_re[i] * uy_re[i] / norm / norm + uy_im[i] * uy_im[i] / norm / norm;
        E[n] += uz_re[i] * uz_re[i] / norm / norm + uz_im[i] * uz_im[i] / norm / norm;
      }
  report(ns3d_write_energy_spectrum_host(file_name, Nx, Ny, 2 * (Mz - 1), E.data()), nullptr,
         "calculate_energy_spectrum", false);
}

double Shapiro_test_case(dim3, dim3, double dx, double dy, double dz, double t, double Re,
                         double* ux, double* uy, double* uz, int Nx, int Ny, int Nz, double*,
                         double*, double* ret) {
  Entry* e = entry_from_steps(Nx, Ny, Nz, dx, dy, dz);
  double mm[2] = {0.0, 0.0};
  report(ns3d_shapiro_error_physical(e->h, ux, uy, uz, t, Re, mm), e->h, "Shapiro_test_case",
         false);
  ret[0] = mm[0];
  ret[1] = mm[1];
  return mm[1];
}

namespace {
// signed wavenumber index of the x / y tables (j >= N/2 -> j - N)
inline int sidx(int j, int n) { return j >= n / 2 ? j - n : j; }
inline size_t flat(int j, int k, int l, int Ny, int Nz) {
  return ((size_t)j * Ny + k) * Nz + l;
}
}  // namespace

void build_Laplace_Wavenumbers(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                               double* kx, double* ky, double* kz) {
  for (int j = 0; j < Nx; ++j) kx[j] = 2.0 * M_PI / Lx * sidx(j, Nx);
  for (int k = 0; k < Ny; ++k) ky[k] = 2.0 * M_PI / Ly * sidx(k, Ny);
  for (int l = 0; l < Nz; ++l) kz[l] = 2.0 * M_PI / Lz * l;
}

void build_Laplace_and_Diffusion(int Nx, int Ny, int Nz, double* din_poisson,
                                 double* din_diffusion, double* kx, double* ky, double* kz) {
  for (int j = 0; j < Nx; ++j)
    for (int k = 0; k < Ny; ++k)
      for (int l = 0; l < Nz; ++l) {
        const size_t i = flat(j, k, l, Ny, Nz);
        din_poisson[i] = -(kx[j] * kx[j] + ky[k] * ky[k] + kz[l] * kz[l]);
        din_diffusion[i] = -din_poisson[i];
      }
  din_poisson[0] = 1.0;
}

void build_Nabla_Wavenumbers(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz, double* kx,
                             double* ky, double* kz) {
  build_Laplace_Wavenumbers(Nx, Ny, Nz, Lx, Ly, Lz, kx, ky, kz);
}

double TotalEnergy(int Nx, int Ny, int Nz, double* ux, double* uy, double* uz, double dx,
                   double dy, double dz, double alpha, double beta) {
  double e = 0.0;
  for (int l = 0; l < Nz; ++l)
    for (int j = 0; j < Nx; ++j)
      for (int k = 0; k < Ny; ++k) {
        const size_t i = flat(j, k, l, Ny, Nz);
        e += (ux[i] * ux[i] + uy[i] * uy[i] + uz[i] * uz[i]) * dx * dy * dz;
      }
  return alpha * beta * e / (4.0 * 2.0 * M_PI);
}

double TotalDissipation(int Nx, int Ny, int Nz, double* ux, double* uy, double* uz, double dx,
                        double dy, double dz, double alpha, double, double) {
  auto at = [&](const double* f, int j, int k, int l) {
    j = j < 0 ? j + Nx : (j >= Nx ? j - Nx : j);
    k = k < 0 ? k + Ny : (k >= Ny ? k - Ny : k);
    l = l < 0 ? l + Nz : (l >= Nz ? l - Nz : l);
    return f[flat(j, k, l, Ny, Nz)];
  };
  double d = 0.0;
  for (int l = 0; l < Nz; ++l)
    for (int j = 0; j < Nx; ++j)
      for (int k = 0; k < Ny; ++k) {
        const double ux_x = (at(ux, j + 1, k, l) - at(ux, j - 1, k, l)) / dx;
        const double ux_y = (at(ux, j, k + 1, l) - at(ux, j, k - 1, l)) / dy;
        const double ux_z = (at(ux, j, k, l + 1) - at(ux, j, k, l - 1)) / dz;
        const double uy_x = (at(uy, j + 1, k, l) - at(uy, j - 1, k, l)) / dx;
        const double uy_y = (at(uy, j, k + 1, l) - at(uy, j, k - 1, l)) / dy;
        const double uy_z = (at(uy, j, k, l + 1) - at(uy, j, k, l - 1)) / dz;
        const double uz_x = (at(uz, j + 1, k, l) - at(uz, j - 1, k, l)) / dx;
        const double uz_y = (at(uz, j, k + 1, l) - at(uz, j, k - 1, l)) / dy;
        const double uz_z = (at(uz, j, k, l + 1) - at(uz, j, k, l - 1)) / dz;
        d += dx * dy * dz *
             (2.0 * (ux_x * ux_x + uy_y * uy_y + uz_z * uz_z) + (uy_z + uz_y) * (uy_z + uz_y) +
              (ux_z + uz_x) * (ux_z + uz_x) + (ux_y + uy_x) * (ux_y + uy_x));
      }
  return alpha * d / (8.0 * M_PI * M_PI * M_PI);
}

void build_projection_matrix_elements(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                                      double* a11, double* a22, double* a33, double* a12,
                                      double* a13, double* a23) {
  const double k1 = 2.0 * M_PI / Lx, k2 = 2.0 * M_PI / Ly, k3 = 2.0 * M_PI / Lz;
  for (int l = 0; l < Nz; ++l)
    for (int j = 0; j < Nx; ++j)
      for (int k = 0; k < Ny; ++k) {
        const int m = sidx(j, Nx), n = sidx(k, Ny), q = l;
        double din = k1 * k1 * m * m + k2 * k2 * n * n + k3 * k3 * q * q;
        if (m * m + n * n + q * q == 0) din = 1.0;
        const size_t i = flat(j, k, l, Ny, Nz);
        a11[i] = k1 * k1 * m * m / din;
        a22[i] = k2 * k2 * n * n / din;
        a33[i] = k3 * k3 * q * q / din;
        a12[i] = k1 * k2 * m * n / din;
        a13[i] = k1 * k3 * m * q / din;
        a23[i] = k2 * k3 * n * q / din;
      }
  a11[0] = a22[0] = a33[0] = a12[0] = a13[0] = a23[0] = 0.0;
}

void build_mask_matrix(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz, double* mask) {
  for (int l = 0; l < Nz; ++l)
    for (int j = 0; j < Nx; ++j)
      for (int k = 0; k < Ny; ++k) {
        const int m = sidx(j, Nx), n = sidx(k, Ny), q = l;
        const double kx = m * 2 * M_PI / Lx, ky = n * 2 * M_PI / Ly, kz = q * 2 * M_PI / Lz;
        const double kxm = 2 * Nx * M_PI / Lx, kym = 2 * Ny * M_PI / Ly,
                     kzm = 2 * Nz * M_PI / Lz;
        const double r =
            std::sqrt(kx * kx / (kxm * kxm) + ky * ky / (kym * kym) + kz * kz / (kzm * kzm));
        mask[flat(j, k, l, Ny, Nz)] = r < 2.0 / 3.0 ? 1.0 : 0.0;
      }
  mask[0] = 0.0;
}

double get_kinetic_energy(dim3, dim3, int Nx, int Ny, int Nz, double dx, double dy, double dz,
                          double* ux, double* uy, double* uz, double*, double*, double*) {
  return physical_reduce(false, Nx, Ny, Nz, dx, dy, dz, ux, uy, uz);
}

double get_dissipation(dim3, dim3, int Nx, int Ny, int Nz, double dx, double dy, double dz,
                       double* ux, double* uy, double* uz, double*, double*, double*) {
  return physical_reduce(true, Nx, Ny, Nz, dx, dy, dz, ux, uy, uz);
}

// ---------------------------------------------------------------------------
// divergence.h
// ---------------------------------------------------------------------------
void divergence_device(dim3, dim3, int Nx, int Ny, int Nz, cplx* div, cplx* ux, cplx* uy,
                       cplx* uz, double* kx, double* ky, double* kz, double dt, double) {
  const long long n = (long long)Nx * Ny * Nz;
  divergence_kernel<<<grid_for(n), 256>>>(div, ux, uy, uz, kx, ky, kz, Ny, Nz, n, dt);
}

void devergence_to_double(dim3, dim3, int Nx, int Ny, int Nz, cplx* div_hat, double* div) {
  c2r_scaled(Nx, Ny, Nz, div_hat, div);
}

// ---------------------------------------------------------------------------
// advection_WENO.h
// ---------------------------------------------------------------------------
void init_WENO(int, int, int, int) {}
void clean_WENO() {}

void ns3d_compat_forcing_changed() {
  std::lock_guard<std::mutex> lock(g_mu);
  g_forcing_dirty = true;
}
