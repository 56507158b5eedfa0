// Checkpoint wire format of the reference (Source/file_operations.cu:4-225):
//
//   control_file.dat          one line per physical point (j, k, l) in
//                             [Nx][Ny][Nz] order: "%.16le %.16le %.16le\n"
//                             (ux, uy, uz);
//   control_file_Fourier.dat  one line per mode (j, k, l) in [Nx][Ny][Mz]
//                             order: "%.16le" x 6 (Re, Im of ux, uy, uz).
//
// 17 significant digits make the text round trip exact, so states move
// between the reference and this library without loss.  A Fourier file of a
// coarser grid is read into a finer one the reference's way
// (read_control_fourier, get_control_fourier_size): the file's extents are
// found from its line count with the target's aspect ratios, x and y modes
// keep their signed wavenumber (the upper half shifts by N - N_file), z modes
// keep their index, and the values are scaled by the reference's integer
// ratio Nx Ny (2 Mz - 1) / (Nx_f Ny_f (2 Mz_f - 1)).
//
// These functions work on host arrays; the solver-side wrappers
// (ns3d_save_* / ns3d_load_* in solver.cu) copy device fields through host
// buffers.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ns3d.h"

namespace {

struct File {
  FILE* f = nullptr;
  explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

// Reads whitespace-separated doubles, `per_line` at a time, until EOF;
// returns false on a malformed number or a short last record.
bool read_records(const char* path, int per_line, std::vector<double>& out) {
  File in(path, "r");
  if (!in.f) return false;
  out.clear();
  std::vector<char> buf(1 << 16);
  std::string carry;
  size_t got;
  while ((got = std::fread(buf.data(), 1, buf.size(), in.f)) > 0) {
    carry.append(buf.data(), got);
    size_t pos = 0;
    const char* s = carry.c_str();
    for (;;) {
      while (pos < carry.size() && (s[pos] == ' ' || s[pos] == '\n' || s[pos] == '\t' ||
                                    s[pos] == '\r'))
        ++pos;
      if (pos >= carry.size()) break;
      // a token may be cut at the buffer end: keep it for the next read
      size_t end = pos;
      while (end < carry.size() && !(s[end] == ' ' || s[end] == '\n' || s[end] == '\t' ||
                                     s[end] == '\r'))
        ++end;
      if (end == carry.size() && !std::feof(in.f)) break;
      char* stop = nullptr;
      const double v = std::strtod(s + pos, &stop);
      if (stop != s + end) return false;
      out.push_back(v);
      pos = end;
    }
    carry.erase(0, pos);
  }
  if (!carry.empty()) {
    char* stop = nullptr;
    const double v = std::strtod(carry.c_str(), &stop);
    if (stop == carry.c_str()) return false;
    out.push_back(v);
  }
  return out.size() % per_line == 0;
}

bool valid_grid(int Nx, int Ny, int Nz) { return Nx > 0 && Ny > 0 && Nz > 0; }

}  // namespace

extern "C" {

ns3d_status ns3d_write_control_fourier_host(const char* path, int Nx, int Ny, int Nz,
                                            const ns3d_complex* ux, const ns3d_complex* uy,
                                            const ns3d_complex* uz) {
  if (!path || !ux || !uy || !uz || !valid_grid(Nx, Ny, Nz)) return NS3D_ERR_BAD_ARG;
  const size_t nc = (size_t)Nx * Ny * (Nz / 2 + 1);
  File out(path, "w");
  if (!out.f) return NS3D_ERR_BAD_ARG;
  char line[256];
  for (size_t i = 0; i < nc; ++i) {
    const int len = std::snprintf(line, sizeof(line), "%.16le %.16le %.16le %.16le %.16le %.16le\n",
                                  ux[i].x, ux[i].y, uy[i].x, uy[i].y, uz[i].x, uz[i].y);
    if (std::fwrite(line, 1, (size_t)len, out.f) != (size_t)len) return NS3D_ERR_BAD_ARG;
  }
  return NS3D_OK;
}

ns3d_status ns3d_read_control_fourier_host(const char* path, int Nx, int Ny, int Nz,
                                           ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                                           int* Nx_file, int* Ny_file, int* Mz_file) {
  if (!path || !ux || !uy || !uz || !valid_grid(Nx, Ny, Nz)) return NS3D_ERR_BAD_ARG;
  const int Mz = Nz / 2 + 1;
  const size_t nc = (size_t)Nx * Ny * Mz;
  std::vector<double> v;
  if (!read_records(path, 6, v)) return NS3D_ERR_BAD_ARG;
  const long long lines = (long long)(v.size() / 6);
  int nxr = Nx, nyr = Ny, mzr = Mz;
  if (lines != (long long)nc) {
    // get_control_fourier_size: the target's aspect ratios, Ny = 4, 6, 8 ...
    // (the reference searches without a bound; here up to the target's Ny)
    const int ratio_xy = Nx / Ny, ratio_zy = (2 * Mz - 1) / Ny;
    bool found = false;
    for (int ny = 4; ny <= Ny; ny += 2) {
      const int nx = ratio_xy * ny, nz = ratio_zy * ny, mz = nz / 2 + 1;
      if ((long long)nx * ny * mz == lines) {
        nxr = nx;
        nyr = ny;
        mzr = mz;
        found = true;
        break;
      }
    }
    if (!found || nxr > Nx || mzr > Mz) return NS3D_ERR_BAD_ARG;
  }
  if (Nx_file) *Nx_file = nxr;
  if (Ny_file) *Ny_file = nyr;
  if (Mz_file) *Mz_file = mzr;
  ns3d_complex* u[3] = {ux, uy, uz};
  if (nxr == Nx && nyr == Ny && mzr == Mz) {
    for (size_t i = 0; i < nc; ++i)
      for (int c = 0; c < 3; ++c) u[c][i] = {v[6 * i + 2 * c], v[6 * i + 2 * c + 1]};
    return NS3D_OK;
  }
  for (int c = 0; c < 3; ++c) std::memset(u[c], 0, sizeof(ns3d_complex) * nc);
  // the reference's scale, evaluated in integer arithmetic as it is there
  const double scale = (double)((Nx * Ny * (2 * Mz - 1)) / (nxr * nyr * (2 * mzr - 1)));
  size_t i = 0;
  for (int j = 0; j < nxr; ++j)
    for (int k = 0; k < nyr; ++k)
      for (int l = 0; l < mzr; ++l, ++i) {
        const int jj = j >= nxr / 2 ? j + (Nx - nxr) : j;
        const int kk = k >= nyr / 2 ? k + (Ny - nyr) : k;
        const size_t d = ((size_t)jj * Ny + kk) * Mz + l;
        for (int c = 0; c < 3; ++c)
          u[c][d] = {scale * v[6 * i + 2 * c], scale * v[6 * i + 2 * c + 1]};
      }
  return NS3D_OK;
}

ns3d_status ns3d_write_control_file_host(const char* path, int Nx, int Ny, int Nz, const double* ux,
                                         const double* uy, const double* uz) {
  if (!path || !ux || !uy || !uz || !valid_grid(Nx, Ny, Nz)) return NS3D_ERR_BAD_ARG;
  const size_t nr = (size_t)Nx * Ny * Nz;
  File out(path, "w");
  if (!out.f) return NS3D_ERR_BAD_ARG;
  char line[128];
  for (size_t i = 0; i < nr; ++i) {
    const int len = std::snprintf(line, sizeof(line), "%.16le %.16le %.16le\n", ux[i], uy[i],
                                  uz[i]);
    if (std::fwrite(line, 1, (size_t)len, out.f) != (size_t)len) return NS3D_ERR_BAD_ARG;
  }
  return NS3D_OK;
}

ns3d_status ns3d_read_control_file_host(const char* path, int Nx, int Ny, int Nz, double* ux,
                                        double* uy, double* uz) {
  if (!path || !ux || !uy || !uz || !valid_grid(Nx, Ny, Nz)) return NS3D_ERR_BAD_ARG;
  const size_t nr = (size_t)Nx * Ny * Nz;
  std::vector<double> v;
  if (!read_records(path, 3, v) || v.size() != 3 * nr) return NS3D_ERR_BAD_ARG;
  for (size_t i = 0; i < nr; ++i) {
    ux[i] = v[3 * i];
    uy[i] = v[3 * i + 1];
    uz[i] = v[3 * i + 2];
  }
  return NS3D_OK;
}

}  // extern "C"
