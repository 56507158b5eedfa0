// Harness around the reference's own CUDA build (TEST INFRASTRUCTURE).
//
// This file is project-written.  It links against the UNMODIFIED reference
// sources (RK_time_step.cu, advection_2_3.cu, diffusion.cu, math_support.cu,
// cuda_supp.cu, min_max_reduction.cu, memory_operations.cu, divergence.cu,
// Shapiro_test.cu), compiled for sm_100a by oracle/Makefile into
// oracle/_ref/libns3d_ref.so, and exposes a flat C ABI so tests and the
// reference arm of bench.py can drive the reference path through its public
// functions.  It is the checker and the reference baseline, never the product.
//
// Initialisation mirrors Source/NS3D_periodic.cu:1141-1272: host builders
// called with Mz in the Nz slot, cufftPlan3d D2Z/Z2D + init_fft_plans,
// init_dealiasing with the device mask, the 16x8 launch geometry of
// Source/NS3D_periodic.cu:1215-1241.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>
#include <cufft.h>

#include "Macros.h"
#include "RK_time_step.h"
#include "advection_2_3.h"
#include "diffusion.h"
#include "math_support.h"
#include "cuda_supp.h"
#include "Shapiro_test.h"

namespace {

struct RefState {
  bool live = false;
  int Nx = 0, Ny = 0, Nz = 0, Mz = 0;
  double Lx = 0, Ly = 0, Lz = 0, dx = 0, dy = 0, dz = 0;
  dim3 dimBlock, dimGrid, dimBlock_C, dimGrid_C;
  cufftHandle planR2C = 0, planC2R = 0;
  // spectral fields [Nx][Ny][Mz]
  cudaComplex *u[3] = {}, *u1[3] = {}, *u2[3] = {}, *u3[3] = {};
  cudaComplex *v[3] = {}, *v1[3] = {}, *f[3] = {}, *Q[3] = {}, *R[3] = {};
  cudaComplex *div_hat = nullptr, *tmp_c = nullptr;
  // tables
  real *kx = nullptr, *ky = nullptr, *kz = nullptr;
  real *din_poisson = nullptr, *din_diffusion = nullptr;
  real *AM[6] = {};
  real *mask = nullptr;
  // physical scratch for diagnostics and transform tests
  real *phys[3] = {};
  real *red[3] = {};
};

RefState S;

size_t nc() { return (size_t)S.Nx * S.Ny * S.Mz; }
size_t nr() { return (size_t)S.Nx * S.Ny * S.Nz; }

int check(const char* what) {
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "ref_harness: %s: %s\n", what, cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

dim3 grid_for(size_t points) {
  // Source/NS3D_periodic.cu:1218-1238
  unsigned int nthreads = block_size_x * block_size_y;
  unsigned int nblocks = (unsigned int)((points + nthreads - 1) / nthreads);
  float db = (float)nblocks;
  unsigned int k1 = (unsigned int)floor(sqrt(db));
  unsigned int k2 = (unsigned int)ceil(db / ((float)k1));
  return dim3(k2, k1, 1);
}

cudaComplex* alloc_c() {
  cudaComplex* p = nullptr;
  if (cudaMalloc((void**)&p, sizeof(cudaComplex) * nc()) != cudaSuccess) return nullptr;
  cudaMemset(p, 0, sizeof(cudaComplex) * nc());
  return p;
}

real* alloc_r(size_t n) {
  real* p = nullptr;
  if (cudaMalloc((void**)&p, sizeof(real) * n) != cudaSuccess) return nullptr;
  cudaMemset(p, 0, sizeof(real) * n);
  return p;
}

void h2d3(cudaComplex* const* dst, const double* src) {
  for (int i = 0; i < 3; ++i)
    cudaMemcpy(dst[i], src + 2 * nc() * i, sizeof(cudaComplex) * nc(), cudaMemcpyHostToDevice);
}

void d2h3(double* dst, cudaComplex* const* src) {
  for (int i = 0; i < 3; ++i)
    cudaMemcpy(dst + 2 * nc() * i, src[i], sizeof(cudaComplex) * nc(), cudaMemcpyDeviceToHost);
}

void rk3(double dt, double Re) {
  RK3_SSP(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, S.dx, S.dy, S.dz, dt, Re, S.Nx, S.Ny,
          S.Nz, S.Mz, S.u[0], S.u[1], S.u[2], S.u1[0], S.u1[1], S.u1[2], S.u2[0], S.u2[1], S.u2[2],
          S.u3[0], S.u3[1], S.u3[2], S.f[0], S.f[1], S.f[2], S.Q[0], S.Q[1], S.Q[2], S.div_hat, S.kx,
          S.ky, S.kz, S.din_diffusion, S.din_poisson, S.AM[0], S.AM[1], S.AM[2], S.AM[3], S.AM[4],
          S.AM[5]);
}

// The reference's reduced Krylov packing (velocities_from_A_vector_reduced_kernel
// and A_vector_from_velocities_reduced_kernel, Source/NS3D_periodic.cu:173-200,
// 239-250; those kernels live in the reference's main file, which this
// harness does not compile): v(0) = 0, v(i) = i vec(i-1); vec(i-1) = Im v(i).
__global__ void harness_unpack_reduced(long long n, const double* vec, cudaComplex* vx,
                                       cudaComplex* vy, cudaComplex* vz) {
  const long long m = n - 1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (i == 0) {
      vx[0].x = vx[0].y = vy[0].x = vy[0].y = vz[0].x = vz[0].y = 0.0;
    } else {
      vx[i].x = 0.0;
      vx[i].y = vec[i - 1];
      vy[i].x = 0.0;
      vy[i].y = vec[i - 1 + m];
      vz[i].x = 0.0;
      vz[i].y = vec[i - 1 + 2 * m];
    }
  }
}

__global__ void harness_pack_reduced(long long n, const cudaComplex* vx, const cudaComplex* vy,
                                     const cudaComplex* vz, double* vec) {
  const long long m = n - 1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
       i += (long long)gridDim.x * blockDim.x) {
    vec[i] = vx[i + 1].y;
    vec[i + m] = vy[i + 1].y;
    vec[i + 2 * m] = vz[i + 1].y;
  }
}

}  // namespace

extern "C" {

// NSCallMatrixVector_reduced (Source/NS3D_periodic.cu:340-361) on the
// harness state, as a user_map_vector for the reference's Krylov code:
// ctx = double[2] {Re, dt}; vec_in -> S.v (reduced unpacking),
// RK3_SSP_UV_RHS about S.u (set with ref_set_u), S.v -> vec_out.  No
// synchronisation, as in the reference (its cuBLAS calls follow on the
// legacy stream).
void ref_map_linearised_reduced(void* ctx, void* in, void* out) {
  const double* c = static_cast<const double*>(ctx);
  const long long n = (long long)nc();
  harness_unpack_reduced<<<592, 256>>>(n, static_cast<const double*>(in), S.v[0], S.v[1],
                                       S.v[2]);
  RK3_SSP_UV_RHS(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, S.dx, S.dy, S.dz, c[1], c[0],
                 S.Nx, S.Ny, S.Nz, S.Mz, S.u[0], S.u[1], S.u[2], S.v[0], S.v[1], S.v[2],
                 S.u1[0], S.u1[1], S.u1[2], S.u2[0], S.u2[1], S.u2[2], S.u3[0], S.u3[1],
                 S.u3[2], S.f[0], S.f[1], S.f[2], S.Q[0], S.Q[1], S.Q[2], S.div_hat, S.kx, S.ky,
                 S.kz, S.din_diffusion, S.din_poisson, S.AM[0], S.AM[1], S.AM[2], S.AM[3],
                 S.AM[4], S.AM[5]);
  harness_pack_reduced<<<592, 256>>>(n, S.v[0], S.v[1], S.v[2], static_cast<double*>(out));
}

// NSCallMatrixVector_exponential (Source/NS3D_periodic.cu:444-470) over the
// harness state: ctx = double[3] {Re, dt, steps}; vec_in -> S.v (reduced
// unpacking), `steps` RK3_SSP_UV steps of (S.u, S.v) (the base flow
// advances with every call, as in the reference), S.v -> vec_out.  The
// reduced packing is used on both sides, as the library's
// ns3d_map_exponential does.
void ref_map_exponential_reduced(void* ctx, void* in, void* out) {
  const double* c = static_cast<const double*>(ctx);
  const long long n = (long long)nc();
  harness_unpack_reduced<<<592, 256>>>(n, static_cast<const double*>(in), S.v[0], S.v[1],
                                       S.v[2]);
  const int steps = (int)c[2];
  for (int s = 0; s < steps; ++s)
    RK3_SSP_UV(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, S.dx, S.dy, S.dz, c[1], c[0],
               S.Nx, S.Ny, S.Nz, S.Mz, S.u[0], S.u[1], S.u[2], S.v[0], S.v[1], S.v[2], S.u1[0],
               S.u1[1], S.u1[2], S.v1[0], S.v1[1], S.v1[2], S.u2[0], S.u2[1], S.u2[2], S.u3[0],
               S.u3[1], S.u3[2], S.f[0], S.f[1], S.f[2], S.Q[0], S.Q[1], S.Q[2], S.div_hat,
               S.kx, S.ky, S.kz, S.din_diffusion, S.din_poisson, S.AM[0], S.AM[1], S.AM[2],
               S.AM[3], S.AM[4], S.AM[5]);
  harness_pack_reduced<<<592, 256>>>(n, S.v[0], S.v[1], S.v[2], static_cast<double*>(out));
}


int ref_create(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz) {
  if (S.live) return -2;
  S.Nx = Nx; S.Ny = Ny; S.Nz = Nz; S.Mz = Nz / 2 + 1;
  S.Lx = Lx; S.Ly = Ly; S.Lz = Lz;
  S.dx = Lx / (real)Nx; S.dy = Ly / (real)Ny; S.dz = Lz / (real)Nz;
  const int Mz = S.Mz;
  S.dimBlock = dim3(block_size_x, block_size_y, 1);
  S.dimBlock_C = S.dimBlock;
  S.dimGrid = grid_for(nr());
  S.dimGrid_C = grid_for(nc());

  for (int i = 0; i < 3; ++i) {
    S.u[i] = alloc_c(); S.u1[i] = alloc_c(); S.u2[i] = alloc_c(); S.u3[i] = alloc_c();
    S.v[i] = alloc_c(); S.v1[i] = alloc_c(); S.f[i] = alloc_c(); S.Q[i] = alloc_c();
    S.R[i] = alloc_c();
    S.phys[i] = alloc_r(nr());
    S.red[i] = alloc_r(nr());
  }
  S.div_hat = alloc_c();
  S.tmp_c = alloc_c();
  S.kx = alloc_r(Nx); S.ky = alloc_r(Ny); S.kz = alloc_r(Mz);
  S.din_poisson = alloc_r(nc()); S.din_diffusion = alloc_r(nc());
  for (int i = 0; i < 6; ++i) S.AM[i] = alloc_r(nc());
  S.mask = alloc_r(nc());
  if (check("alloc")) return -1;

  // host builders, Mz in the Nz slot (Source/NS3D_periodic.cu:1153-1161)
  std::vector<real> kxl(Nx), kyl(Ny), kzl(Mz), kxn(Nx), kyn(Ny), kzn(Mz);
  std::vector<real> dp(nc()), dd(nc()), msk(nc());
  std::vector<std::vector<real>> am(6, std::vector<real>(nc()));
  build_Laplace_Wavenumbers(Nx, Ny, Mz, Lx, Ly, Lz, kxl.data(), kyl.data(), kzl.data());
  build_Laplace_and_Diffusion(Nx, Ny, Mz, dp.data(), dd.data(), kxl.data(), kyl.data(), kzl.data());
  build_Nabla_Wavenumbers(Nx, Ny, Mz, Lx, Ly, Lz, kxn.data(), kyn.data(), kzn.data());
  build_projection_matrix_elements(Nx, Ny, Mz, Lx, Ly, Lz, am[0].data(), am[1].data(), am[2].data(),
                                   am[3].data(), am[4].data(), am[5].data());
  build_mask_matrix(Nx, Ny, Mz, Lx, Ly, Lz, msk.data());
  cudaMemcpy(S.kx, kxn.data(), sizeof(real) * Nx, cudaMemcpyHostToDevice);
  cudaMemcpy(S.ky, kyn.data(), sizeof(real) * Ny, cudaMemcpyHostToDevice);
  cudaMemcpy(S.kz, kzn.data(), sizeof(real) * Mz, cudaMemcpyHostToDevice);
  cudaMemcpy(S.din_poisson, dp.data(), sizeof(real) * nc(), cudaMemcpyHostToDevice);
  cudaMemcpy(S.din_diffusion, dd.data(), sizeof(real) * nc(), cudaMemcpyHostToDevice);
  for (int i = 0; i < 6; ++i)
    cudaMemcpy(S.AM[i], am[i].data(), sizeof(real) * nc(), cudaMemcpyHostToDevice);
  cudaMemcpy(S.mask, msk.data(), sizeof(real) * nc(), cudaMemcpyHostToDevice);

  if (cufftPlan3d(&S.planR2C, Nx, Ny, Nz, RealToComplex) != CUFFT_SUCCESS) return -3;
  if (cufftPlan3d(&S.planC2R, Nx, Ny, Nz, ComplexToReal) != CUFFT_SUCCESS) return -3;
  init_fft_plans(S.planR2C, S.planC2R);
  init_dealiasing(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, Nx, Ny, Nz, Mz, S.mask);
  if (check("init")) return -1;
  S.live = true;
  return 0;
}

void ref_destroy() {
  if (!S.live) return;
  cudaDeviceSynchronize();
  clean_dealiasing();
  cufftDestroy(S.planR2C);
  cufftDestroy(S.planC2R);
  for (int i = 0; i < 3; ++i) {
    cudaFree(S.u[i]); cudaFree(S.u1[i]); cudaFree(S.u2[i]); cudaFree(S.u3[i]);
    cudaFree(S.v[i]); cudaFree(S.v1[i]); cudaFree(S.f[i]); cudaFree(S.Q[i]); cudaFree(S.R[i]);
    cudaFree(S.phys[i]); cudaFree(S.red[i]);
  }
  cudaFree(S.div_hat); cudaFree(S.tmp_c);
  cudaFree(S.kx); cudaFree(S.ky); cudaFree(S.kz);
  cudaFree(S.din_poisson); cudaFree(S.din_diffusion);
  for (int i = 0; i < 6; ++i) cudaFree(S.AM[i]);
  cudaFree(S.mask);
  S = RefState();
}

// Fields are host arrays of 3 components, each [Nx][Ny][Mz] complex (interleaved re, im).
int ref_set_u(const double* u) { h2d3(S.u, u); return check("set_u"); }
int ref_set_v(const double* v) { h2d3(S.v, v); return check("set_v"); }
int ref_set_f(const double* f) { h2d3(S.f, f); return check("set_f"); }
int ref_get_u(double* u) { d2h3(u, S.u); return check("get_u"); }
int ref_get_v(double* v) { d2h3(v, S.v); return check("get_v"); }

int ref_rk3(int nsteps, double dt, double Re) {
  for (int s = 0; s < nsteps; ++s) rk3(dt, Re);
  return check("rk3");
}

int ref_euler(double dt, double Re) {
  single_time_step(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, S.dx, S.dy, S.dz, dt, Re, S.Nx,
                   S.Ny, S.Nz, S.Mz, S.u[0], S.u[1], S.u[2], S.f[0], S.f[1], S.f[2], S.Q[0], S.Q[1],
                   S.Q[2], S.div_hat, S.kx, S.ky, S.kz, S.din_diffusion, S.din_poisson, S.u3[0],
                   S.u3[1], S.u3[2], S.AM[0], S.AM[1], S.AM[2], S.AM[3], S.AM[4], S.AM[5]);
  return check("euler");
}

int ref_rhs(double Re, double* out) {
  return_RHS(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, S.dx, S.dy, S.dz, Re, S.Nx, S.Ny,
             S.Nz, S.Mz, S.u[0], S.u[1], S.u[2], S.f[0], S.f[1], S.f[2], S.Q[0], S.Q[1], S.Q[2],
             S.div_hat, S.kx, S.ky, S.kz, S.din_diffusion, S.din_poisson, S.AM[0], S.AM[1],
             S.AM[2], S.AM[3], S.AM[4], S.AM[5], S.R[0], S.R[1], S.R[2]);
  if (check("rhs")) return -1;
  d2h3(out, S.R);
  return check("rhs copy");
}

int ref_conv(double* out) {
  calculate_convolution_2p3(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, S.Nx, S.Ny, S.Nz, S.Mz,
                            S.u[0], S.u[1], S.u[2], S.kx, S.ky, S.kz, S.Q[0], S.Q[1], S.Q[2]);
  if (check("conv")) return -1;
  d2h3(out, S.Q);
  return check("conv copy");
}

int ref_conv_uv(double* out) {
  calculate_convolution_2p3_UV(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, S.Nx, S.Ny, S.Nz,
                               S.Mz, S.u[0], S.u[1], S.u[2], S.v[0], S.v[1], S.v[2], S.kx, S.ky,
                               S.kz, S.Q[0], S.Q[1], S.Q[2]);
  if (check("conv_uv")) return -1;
  d2h3(out, S.Q);
  return check("conv_uv copy");
}

int ref_jvp(int nsteps, double dt, double Re) {
  for (int s = 0; s < nsteps; ++s)
    RK3_SSP_UV(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, S.dx, S.dy, S.dz, dt, Re, S.Nx,
               S.Ny, S.Nz, S.Mz, S.u[0], S.u[1], S.u[2], S.v[0], S.v[1], S.v[2], S.u1[0], S.u1[1],
               S.u1[2], S.v1[0], S.v1[1], S.v1[2], S.u2[0], S.u2[1], S.u2[2], S.u3[0], S.u3[1],
               S.u3[2], S.f[0], S.f[1], S.f[2], S.Q[0], S.Q[1], S.Q[2], S.div_hat, S.kx, S.ky, S.kz,
               S.din_diffusion, S.din_poisson, S.AM[0], S.AM[1], S.AM[2], S.AM[3], S.AM[4],
               S.AM[5]);
  return check("jvp");
}

int ref_linrhs(double dt, double Re) {
  RK3_SSP_UV_RHS(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, S.dx, S.dy, S.dz, dt, Re, S.Nx,
                 S.Ny, S.Nz, S.Mz, S.u[0], S.u[1], S.u[2], S.v[0], S.v[1], S.v[2], S.u1[0],
                 S.u1[1], S.u1[2], S.u2[0], S.u2[1], S.u2[2], S.u3[0], S.u3[1], S.u3[2], S.f[0],
                 S.f[1], S.f[2], S.Q[0], S.Q[1], S.Q[2], S.div_hat, S.kx, S.ky, S.kz,
                 S.din_diffusion, S.din_poisson, S.AM[0], S.AM[1], S.AM[2], S.AM[3], S.AM[4],
                 S.AM[5]);
  return check("linrhs");
}

int ref_iuv(double dt, double Re) {
  single_time_step_iUV_RHS(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, S.dx, S.dy, S.dz, dt,
                           Re, S.Nx, S.Ny, S.Nz, S.Mz, S.u[0], S.u[1], S.u[2], S.v[0], S.v[1],
                           S.v[2], S.Q[0], S.Q[1], S.Q[2], S.div_hat, S.kx, S.ky, S.kz,
                           S.din_diffusion, S.din_poisson, S.AM[0], S.AM[1], S.AM[2], S.AM[3],
                           S.AM[4], S.AM[5]);
  return check("iuv");
}

// cuFFT Z2D + 1/(NxNyNz) on one half spectrum (host in, host out).  The input
// is copied first: an out-of-place multi-dimensional C2R may overwrite it.
int ref_c2r(const double* X, double* x) {
  cudaMemcpy(S.tmp_c, X, sizeof(cudaComplex) * nc(), cudaMemcpyHostToDevice);
  iFFTN_Device(S.dimGrid, S.dimBlock, S.tmp_c, S.phys[0], S.Nx, S.Ny, S.Nz);
  if (check("c2r")) return -1;
  cudaMemcpy(x, S.phys[0], sizeof(real) * nr(), cudaMemcpyDeviceToHost);
  return check("c2r copy");
}

int ref_r2c(const double* x, double* X) {
  cudaMemcpy(S.phys[0], x, sizeof(real) * nr(), cudaMemcpyHostToDevice);
  FFTN_Device(S.phys[0], S.tmp_c);
  if (check("r2c")) return -1;
  cudaMemcpy(X, S.tmp_c, sizeof(cudaComplex) * nc(), cudaMemcpyDeviceToHost);
  return check("r2c copy");
}

// Per-step diagnostics of the reference main loop (Source/NS3D_periodic.cu:1325-1452,
// energy/dissipation part): C2R of a copy of the state, then the two reductions.
int ref_diag(double* energy, double* diss) {
  for (int i = 0; i < 3; ++i) {
    cudaMemcpy(S.u3[i], S.u[i], sizeof(cudaComplex) * nc(), cudaMemcpyDeviceToDevice);
  }
  Image_to_Domain(S.dimGrid, S.dimBlock, S.Nx, S.Ny, S.Nz, S.phys[0], S.u3[0], S.phys[1], S.u3[1],
                  S.phys[2], S.u3[2]);
  *energy = get_kinetic_energy(S.dimGrid, S.dimBlock, S.Nx, S.Ny, S.Nz, S.dx, S.dy, S.dz, S.phys[0],
                               S.phys[1], S.phys[2], S.red[0], S.red[1], S.red[2]);
  *diss = get_dissipation(S.dimGrid, S.dimBlock, S.Nx, S.Ny, S.Nz, S.dx, S.dy, S.dz, S.phys[0],
                          S.phys[1], S.phys[2], S.red[0], S.red[1], S.red[2]);
  return check("diag");
}

// One step of the main loop's diagnostic block (Source/NS3D_periodic.cu:1325-1452)
// on the state itself, in main's order and with main's index arithmetic:
// Image_to_Domain of the state, the Helmholtz and then the cut-off filter, the
// curls, get_kinetic_energy / get_dissipation, the point reads, and
// all_Fourier2double.  rec[0] = total_time, rec[1..49] = columns 2..50 of
// time_dependant.dat.  preserve = 0: as main, Image_to_Domain transforms the
// state arrays themselves (cuFFT's out-of-place multi-dimensional
// complex-to-real transform may overwrite its input, and on B200 with cuFFT
// 12.9 it does, so the filters and the spectral reads that follow see what
// the transform left there; ref_get_u shows it).  preserve = 1: Image_to_Domain
// reads a copy, so everything after it sees the state.
int ref_diag_record(double total_time, double Re, double* rec, int preserve) {
  int Nx = S.Nx, Ny = S.Ny, Nz = S.Nz;
  const int Mz = S.Mz;
  const double dx = S.dx, dy = S.dy, dz = S.dz;
  real *ux_d = S.phys[0], *uy_d = S.phys[1], *uz_d = S.phys[2];
  real *filt[3], *rot[3], *reim[6], *div_pos_d;
  cudaComplex* fh[3];
  for (int i = 0; i < 3; ++i) {
    filt[i] = alloc_r(nr());
    rot[i] = alloc_r(nr());
    fh[i] = alloc_c();
  }
  for (int i = 0; i < 6; ++i) reim[i] = alloc_r(nc());
  div_pos_d = alloc_r(nr());
  if (check("record alloc")) return -1;
  auto rd = [](const real* p, long long i) {
    real v = 0.0;
    cudaMemcpy(&v, p + i, sizeof(real), cudaMemcpyDeviceToHost);
    return v;
  };
  cudaComplex* src[3] = {S.u[0], S.u[1], S.u[2]};
  if (preserve) {
    for (int i = 0; i < 3; ++i) {
      cudaMemcpy(S.u3[i], S.u[i], sizeof(cudaComplex) * nc(), cudaMemcpyDeviceToDevice);
      src[i] = S.u3[i];
    }
  }
  Image_to_Domain(S.dimGrid, S.dimBlock, Nx, Ny, Nz, ux_d, src[0], uy_d, src[1], uz_d, src[2]);
  Helmholz_Fourier_Filter(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, Nx, Ny, Nz, Mz, S.Lx,
                          S.Ly, S.Lz, S.u[0], S.u[1], S.u[2], fh[0], fh[1], fh[2], 1.0, filt[0],
                          filt[1], filt[2]);
  CutOff_Fourier_Filter(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, Nx, Ny, Nz, Mz, S.Lx,
                        S.Ly, S.Lz, S.u[0], S.u[1], S.u[2], fh[0], fh[1], fh[2], 0.1, filt[0],
                        filt[1], filt[2]);
  get_curl(S.dimGrid, S.dimBlock, Nx, Ny, Nz, dx, dy, dz, ux_d, uy_d, uz_d, rot[0], rot[1], rot[2]);
  const real energy = get_kinetic_energy(S.dimGrid, S.dimBlock, Nx, Ny, Nz, dx, dy, dz, ux_d, uy_d,
                                         uz_d, S.red[0], S.red[1], S.red[2]);
  const real dissipation = get_dissipation(S.dimGrid, S.dimBlock, Nx, Ny, Nz, dx, dy, dz, ux_d,
                                           uy_d, uz_d, S.red[0], S.red[1], S.red[2]);
  int c = 0;
  rec[c++] = total_time;
  const long long P[3] = {IN(Nx / 2 - 4, Ny / 2 - 3, Nz / 2 - 2), IN(Nx / 3, Ny / 3, Nz / 3),
                          IN(Nx / 8, Ny / 8, Nz / 8)};
  const real tail[3] = {energy, dissipation, energy - dissipation / Re};
  for (int p = 0; p < 3; ++p) {
    rec[c++] = rd(ux_d, P[p]); rec[c++] = rd(uy_d, P[p]); rec[c++] = rd(uz_d, P[p]);
    rec[c++] = rd(rot[0], P[p]); rec[c++] = rd(rot[1], P[p]); rec[c++] = rd(rot[2], P[p]);
    rec[c++] = tail[p];
  }
  get_curl(S.dimGrid, S.dimBlock, Nx, Ny, Nz, dx, dy, dz, filt[0], filt[1], filt[2], rot[0], rot[1],
           rot[2]);
  rec[c++] = rd(filt[0], P[1]); rec[c++] = rd(filt[1], P[1]); rec[c++] = rd(filt[2], P[1]);
  rec[c++] = rd(rot[0], P[1]); rec[c++] = rd(rot[1], P[1]); rec[c++] = rd(rot[2], P[1]);
  rec[c++] = energy;
  Nz = Mz;  // main switches IN to the spectral layout here
  all_Fourier2double(S.dimGrid_C, S.dimBlock_C, S.u[0], reim[0], reim[1], S.u[1], reim[2], reim[3],
                     S.u[2], reim[4], reim[5], Nx, Ny, Mz);
  const long long F1 = IN(Nx - 6, Ny - 6, Nz - 6);
  for (int i = 0; i < 6; ++i) rec[c++] = rd(reim[i], F1);
  rec[c++] = dissipation;
  const long long F2 = IN(Nx / 5, Ny / 4 - 3, Nz / 4 - 1), F3 = IN(Nx / 5, Ny / 5, Nz / 5);
  for (int i = 1; i < 6; i += 2) {
    rec[c++] = rd(reim[i], F2);
    rec[c++] = rd(reim[i], F3);
  }
  rec[c++] = rd(reim[1], IN(2, 2, 2));
  const long long F[7] = {IN(1, 0, 0),      IN(0, 0, 0),           IN(1, 1, 0),
                          IN(1, 1, 1),      IN(Nx - 1, 0, 0),      IN(Nx - 1, Ny - 1, 0),
                          IN(Nx - 1, Ny - 1, Nz - 1)};
  for (int i = 0; i < 7; ++i) rec[c++] = rd(reim[1], F[i]);
  for (int i = 0; i < 3; ++i) {
    cudaFree(filt[i]);
    cudaFree(rot[i]);
    cudaFree(fh[i]);
  }
  for (int i = 0; i < 6; ++i) cudaFree(reim[i]);
  cudaFree(div_pos_d);
  return check("record");
}

// The two spectral filters on a copy of the state, as main calls them:
// Helmholz_Fourier_Filter(eps) and CutOff_Fourier_Filter(radius), each
// followed by its scaled complex-to-real transform; phys_h / phys_c receive
// the filtered physical velocities (3 host fields each).
int ref_filters(double eps, double radius, double* phys_h, double* phys_c) {
  cudaComplex* fh[3];
  real* filt[3];
  for (int i = 0; i < 3; ++i) {
    fh[i] = alloc_c();
    filt[i] = alloc_r(nr());
    cudaMemcpy(S.u3[i], S.u[i], sizeof(cudaComplex) * nc(), cudaMemcpyDeviceToDevice);
  }
  if (check("filters alloc")) return -1;
  Helmholz_Fourier_Filter(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, S.Nx, S.Ny, S.Nz, S.Mz,
                          S.Lx, S.Ly, S.Lz, S.u3[0], S.u3[1], S.u3[2], fh[0], fh[1], fh[2], eps,
                          filt[0], filt[1], filt[2]);
  for (int i = 0; i < 3; ++i)
    cudaMemcpy(phys_h + nr() * i, filt[i], sizeof(real) * nr(), cudaMemcpyDeviceToHost);
  CutOff_Fourier_Filter(S.dimGrid, S.dimBlock, S.dimGrid_C, S.dimBlock_C, S.Nx, S.Ny, S.Nz, S.Mz,
                        S.Lx, S.Ly, S.Lz, S.u3[0], S.u3[1], S.u3[2], fh[0], fh[1], fh[2], radius,
                        filt[0], filt[1], filt[2]);
  for (int i = 0; i < 3; ++i)
    cudaMemcpy(phys_c + nr() * i, filt[i], sizeof(real) * nr(), cudaMemcpyDeviceToHost);
  for (int i = 0; i < 3; ++i) {
    cudaFree(fh[i]);
    cudaFree(filt[i]);
  }
  return check("filters");
}

// get_curl on 3 physical host fields (rot: 3 physical host fields).
int ref_curl(const double* u, double* rot) {
  real* r[3];
  for (int i = 0; i < 3; ++i) {
    r[i] = alloc_r(nr());
    cudaMemcpy(S.phys[i], u + nr() * i, sizeof(real) * nr(), cudaMemcpyHostToDevice);
  }
  get_curl(S.dimGrid, S.dimBlock, S.Nx, S.Ny, S.Nz, S.dx, S.dy, S.dz, S.phys[0], S.phys[1],
           S.phys[2], r[0], r[1], r[2]);
  if (check("curl")) return -1;
  for (int i = 0; i < 3; ++i) {
    cudaMemcpy(rot + nr() * i, r[i], sizeof(real) * nr(), cudaMemcpyDeviceToHost);
    cudaFree(r[i]);
  }
  return check("curl copy");
}

// Shapiro_test_case (Source/Shapiro_test.cu:38-50) on the physical velocity of
// a copy of the state.
int ref_shapiro_error(double t, double Re, double* err) {
  for (int i = 0; i < 3; ++i)
    cudaMemcpy(S.u3[i], S.u[i], sizeof(cudaComplex) * nc(), cudaMemcpyDeviceToDevice);
  Image_to_Domain(S.dimGrid, S.dimBlock, S.Nx, S.Ny, S.Nz, S.phys[0], S.u3[0], S.phys[1], S.u3[1],
                  S.phys[2], S.u3[2]);
  real ret[2] = {0.0, 0.0};
  *err = Shapiro_test_case(S.dimGrid, S.dimBlock, S.dx, S.dy, S.dz, t, Re, S.phys[0], S.phys[1],
                           S.phys[2], S.Nx, S.Ny, S.Nz, S.red[0], S.red[1], ret);
  return check("shapiro");
}

// Device-resident timing of nsteps RK3_SSP calls with CUDA events (ms total).
double ref_time_rk3(int nsteps, double dt, double Re) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaDeviceSynchronize();
  cudaEventRecord(a, 0);
  for (int s = 0; s < nsteps; ++s) rk3(dt, Re);
  cudaEventRecord(b, 0);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (check("time_rk3")) return -1.0;
  return (double)ms;
}

// Device pointers of the state, for timing with host<->device copies outside.
void* ref_u_ptr(int i) { return (void*)S.u[i]; }
void* ref_f_ptr(int i) { return (void*)S.f[i]; }

}  // extern "C"
