// Flat C entry points for the reference's checkpoint reader and writer
// (Source/file_operations.cu:4-228) and its energy-spectrum writer
// (Source/math_support.cu:819-860), for ctypes (TEST INFRASTRUCTURE).  The
// reference functions use fixed file names in the working directory
// (control_file.dat, control_file_Fourier.dat).  Host code only: no GPU.
// Linked into oracle/_ref/libns3d_ref.so together with the unmodified
// reference sources.
#include <cstring>
#include <vector>

#include "Macros.h"
#include "file_operations.h"
#include "math_support.h"

extern "C" {

// u: 3 host fields [Nx][Ny][Mz] of interleaved complex; writes
// control_file_Fourier.dat in the working directory.
void ref_write_control_fourier(int Nx, int Ny, int Mz, const double* u) {
  const size_t n = (size_t)Nx * Ny * Mz;
  std::vector<double> re[3], im[3];
  for (int c = 0; c < 3; ++c) {
    re[c].resize(n);
    im[c].resize(n);
    for (size_t i = 0; i < n; ++i) {
      re[c][i] = u[2 * (c * n + i)];
      im[c][i] = u[2 * (c * n + i) + 1];
    }
  }
  write_control_file_fourier(Nx, Ny, Mz, re[0].data(), im[0].data(), re[1].data(), im[1].data(),
                             re[2].data(), im[2].data());
}

// Reads control_file_Fourier.dat (same size, or a coarser grid the
// reference recognises) into zeroed host fields.
void ref_read_control_fourier(int Nx, int Ny, int Mz, double* u) {
  const size_t n = (size_t)Nx * Ny * Mz;
  std::vector<double> re[3], im[3];
  for (int c = 0; c < 3; ++c) {
    re[c].assign(n, 0.0);
    im[c].assign(n, 0.0);
  }
  read_control_fourier(Nx, Ny, Mz, re[0].data(), im[0].data(), re[1].data(), im[1].data(),
                       re[2].data(), im[2].data());
  for (int c = 0; c < 3; ++c)
    for (size_t i = 0; i < n; ++i) {
      u[2 * (c * n + i)] = re[c][i];
      u[2 * (c * n + i) + 1] = im[c][i];
    }
}

void ref_write_control_file(int Nx, int Ny, int Nz, double* ux, double* uy, double* uz) {
  write_control_file(Nx, Ny, Nz, ux, uy, uz);
}

void ref_read_control_file(int Nx, int Ny, int Nz, double* ux, double* uy, double* uz) {
  read_control_file(Nx, Ny, Nz, ux, uy, uz);
}

// u: 3 host fields [Nx][Ny][Mz] of interleaved complex; writes `path` with
// calculate_energy_spectrum (called as main calls it, with Mz).
void ref_energy_spectrum(const char* path, int Nx, int Ny, int Mz, const double* u) {
  const size_t n = (size_t)Nx * Ny * Mz;
  std::vector<double> re[3], im[3];
  for (int c = 0; c < 3; ++c) {
    re[c].resize(n);
    im[c].resize(n);
    for (size_t i = 0; i < n; ++i) {
      re[c][i] = u[2 * (c * n + i)];
      im[c][i] = u[2 * (c * n + i) + 1];
    }
  }
  std::vector<char> name(path, path + strlen(path) + 1);
  calculate_energy_spectrum(name.data(), Nx, Ny, Mz, re[0].data(), im[0].data(), re[1].data(),
                            im[1].data(), re[2].data(), im[2].data());
}

}  // extern "C"
