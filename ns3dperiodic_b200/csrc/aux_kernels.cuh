// Small kernels around the RHS pipeline: forcing capture, Krylov vector
// packing (Source/NS3D_periodic.cu:173-317) and the spectral diagnostics
// reduction (Source/math_support.cu:720-806, Source/divergence.cu:8-31).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace ns3d {

// Compacts the non-zero modes of a 3-component spectral field.  Entries past
// `cap` are counted but not stored (the host then keeps the dense field).
__global__ void forcing_scan_kernel(const double2* __restrict__ fx, const double2* __restrict__ fy,
                                    const double2* __restrict__ fz, long long n, int cap,
                                    int* __restrict__ count, int* __restrict__ idx,
                                    double2* __restrict__ val);

// vec[i + c*(n-1)] = Im v_c[i+1]  (A_vector_from_velocities_reduced_kernel),
// then vec -= coef * vec_shift when vec_shift != null and vec += coef2 *
// vec_shift2 when vec_shift2 != null, in that order (the shifted and
// rotated packings, Source/NS3D_periodic.cu:253-300).
__global__ void pack_reduced_kernel(const double2* __restrict__ vx, const double2* __restrict__ vy,
                                    const double2* __restrict__ vz, long long n,
                                    double* __restrict__ vec, const double* __restrict__ vec_shift,
                                    double coef, const double* __restrict__ vec_shift2,
                                    double coef2);

// v_c[i+1] = (0, vec[i + c*(n-1)]), v_c[0] = 0 (velocities_from_A_vector_reduced_kernel).
__global__ void unpack_reduced_kernel(const double* __restrict__ vec, long long n,
                                      double2* __restrict__ vx, double2* __restrict__ vy,
                                      double2* __restrict__ vz);

struct DiagGeom {
  int Nx, Ny, Nz, Mz;
  double kfx, kfy, kfz;  // 2 pi / L
  double dx, dy, dz;
  double inv_vol;        // 1/(Nx Ny Nz)
};

// Largest extent per direction (the compiled extents go to 512).
constexpr int kDiagMaxExtent = 512;

// Per-block partial sums: [0] energy, [1] dissipation, [2] max |div|.
__global__ void diag_partial_kernel(const double2* __restrict__ ux, const double2* __restrict__ uy,
                                    const double2* __restrict__ uz, DiagGeom g,
                                    double* __restrict__ partial);
__global__ void diag_final_kernel(const double* __restrict__ partial, int nblocks,
                                  double* __restrict__ out);

}  // namespace ns3d
