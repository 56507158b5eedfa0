// Kernels of the main loop's per-step diagnostics and their helpers:
// spectral filters and the finite-difference curl (Source/math_support.cu:
// 680-717, 866-987), the time_dependant.dat record
// (Source/NS3D_periodic.cu:1324-1452), the energy spectrum
// (Source/math_support.cu:819-860) and Shapiro's exact solution and error
// (Source/Shapiro_test.cu:8-50, Source/NS3D_periodic.cu:807-829).
#pragma once

#include <cuda_runtime.h>

namespace ns3d {

struct FilterGeom {
  int Nx, Ny, Mz;
  double Lx, Ly, Lz;
};

// mode 0: Helmholz_Fourier_Filter_Device, f = u / (1 + p^2 |k|^2);
// mode 1: CutOff_Fourier_Filter_Device launched with Mz as Nz, f = u where
// m^2/Nx^2 + n^2/Ny^2 + q^2/Mz^2 <= p^2, else 0.  f may alias u.
__global__ void spectral_filter_kernel(const double2* __restrict__ ux, const double2* __restrict__ uy,
                                       const double2* __restrict__ uz, double2* fx, double2* fy,
                                       double2* fz, FilterGeom g, int mode, double p);

struct GridGeom {
  int Nx, Ny, Nz;
  double dx, dy, dz;
};

// get_curl_device on physical fields, periodic wrap, including the
// reference's rot_y term 0.5 (uz(j+1) - ux(j-1)) / dx.
__global__ void curl_kernel(const double* __restrict__ ux, const double* __restrict__ uy,
                            const double* __restrict__ uz, double* __restrict__ rx,
                            double* __restrict__ ry, double* __restrict__ rz, GridGeom g);

// The record's point values as linear functionals of the spectrum.  For a
// point p = (px, py, pz) the scaled complex-to-real transform gives
//   u(p) = 1/N sum_{j,k,l < Mz} w_l Re(u_hat(j,k,l) e^{2 pi i (j px/Nx + k py/Ny + l pz/Nz)}),
// w_l = 1 on the kz = 0 and kz = Nz/2 planes and 2 elsewhere (the real part
// of the full-plane sum is exactly the Hermitian part the transform uses),
// and a shift by one grid step multiplies the mode by e^{2 pi i j/Nx}, so a
// central difference at p is the same sum with i sin(2 pi j/Nx)/dx applied.
// Slots 0..2 are the three probe points on the state, slot 3 the second
// point on the cut-off filtered state; per slot ux, uy, uz, rot_x, rot_y,
// rot_z.  The table holds, per point s, e^{2 pi i j p_s / N} along each axis,
// then e^{2 pi i j / Nx} and sin(2 pi j / N)/h per axis.
constexpr int kRecordSums = 24;
struct RecordGeom {
  int Nx, Ny, Nz, Mz;
  double dx, dy, dz;
  double cut2;  // squared cut-off radius of slot 3
};
// Table layout (double2 entries): ex[3][Nx], ey[3][Ny], ez[3][Mz], shx[Nx],
// then sx[Nx], sy[Ny], sz[Mz] in .x.
__host__ __device__ inline long long record_table_size(int Nx, int Ny, int Mz) {
  return 3LL * (Nx + Ny + Mz) + Nx + (Nx + Ny + Mz);
}
__global__ void record_partial_kernel(const double2* __restrict__ ux,
                                      const double2* __restrict__ uy,
                                      const double2* __restrict__ uz, RecordGeom g,
                                      const double2* __restrict__ tab, double* __restrict__ partial);

// Spectral flat indices the record reads directly (IN with Nz = Mz).
struct RecordReads {
  long long f[11];
};
// Sums the partials of record_partial_kernel in a fixed order and writes the
// 50 columns: rec[0] = total_time; energy and dissipation come from
// diag_out[0..1] (diag_final_kernel).  One block of 32 * kRecordSums threads.
__global__ void record_final_kernel(const double* __restrict__ partial, int nblocks,
                                    const double* __restrict__ diag_out,
                                    const double2* __restrict__ ux,
                                    const double2* __restrict__ uy,
                                    const double2* __restrict__ uz, RecordReads reads,
                                    double total_time, double Re, double inv_n,
                                    double* __restrict__ rec);

// calculate_energy_spectrum's sums: one block per bin n = j + k + l over
// j < Nx/2, k < Ny/2, l < Mz; E[n] = sum |u_hat|^2 / norm^2 (norm = Nx Ny Mz),
// accumulated per thread in index order and folded in a fixed tree.
__global__ void spectrum_kernel(const double2* __restrict__ ux, const double2* __restrict__ uy,
                                const double2* __restrict__ uz, int Nx, int Ny, int Mz,
                                double norm, double* __restrict__ E);

// Shapiro's Beltrami field (Initial_Shapiro at time t; decay = exp(-3 t/Re))
// into physical fields, and the per-point error norm's per-block min / max.
__global__ void shapiro_field_kernel(double* __restrict__ ux, double* __restrict__ uy,
                                     double* __restrict__ uz, GridGeom g, double decay);
__global__ void shapiro_error_kernel(const double* __restrict__ ux, const double* __restrict__ uy,
                                     const double* __restrict__ uz, GridGeom g, double decay,
                                     double* __restrict__ partial);
// out[0] = min, out[1] = max over nblocks (min, max) pairs.
__global__ void minmax_final_kernel(const double* __restrict__ partial, int nblocks,
                                    double* __restrict__ out);

}  // namespace ns3d
