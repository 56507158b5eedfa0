// Text writers of the main loop's diagnostic files (host only):
//
//   time_dependant.dat  one line per step, fprintf'd in pieces by
//                       Source/NS3D_periodic.cu:1375-1452: 50 "%le" fields
//                       separated by single spaces, newline after the last;
//   Ek.dat              calculate_energy_spectrum (Source/math_support.cu:
//                       819-860): per bin "%i %.16le %.16le\n".
#include <cmath>
#include <cstdio>

#include "ns3d.h"

struct ns3d_series {
  FILE* f = nullptr;
};

extern "C" {

ns3d_status ns3d_series_open(const char* path, ns3d_series** out) {
  if (!path || !out) return NS3D_ERR_BAD_ARG;
  *out = nullptr;
  FILE* f = std::fopen(path, "w");
  if (!f) return NS3D_ERR_BAD_ARG;
  *out = new ns3d_series{f};
  return NS3D_OK;
}

ns3d_status ns3d_series_write(ns3d_series* s, const double* rec, int ncols) {
  if (!s || !s->f || !rec || ncols <= 0) return NS3D_ERR_BAD_ARG;
  for (int i = 0; i < ncols; ++i)
    if (std::fprintf(s->f, i + 1 < ncols ? "%le " : "%le\n", rec[i]) < 0) return NS3D_ERR_BAD_ARG;
  return NS3D_OK;
}

ns3d_status ns3d_series_close(ns3d_series* s) {
  if (!s) return NS3D_ERR_BAD_ARG;
  const int rc = s->f ? std::fclose(s->f) : 0;
  delete s;
  return rc == 0 ? NS3D_OK : NS3D_ERR_BAD_ARG;
}

ns3d_status ns3d_write_energy_spectrum_host(const char* path, int Nx, int Ny, int Nz,
                                            const double* E) {
  if (!path || !E || Nx <= 0 || Ny <= 0 || Nz <= 0) return NS3D_ERR_BAD_ARG;
  const int Mz = Nz / 2 + 1;
  const int size = Nx / 2 + Ny / 2 + Mz;
  // the highest bin a mode of the positive quadrant reaches; the reference's
  // table keeps zeros (and a zero bin label) above it
  const int nmax = (Nx / 2 - 1) + (Ny / 2 - 1) + (Mz - 1);
  FILE* f = std::fopen(path, "w");
  if (!f) return NS3D_ERR_BAD_ARG;
  int bad = 0;
  for (int n = 0; n < size && !bad; ++n) {
    if (n <= nmax)
      bad = std::fprintf(f, "%i %.16le %.16le\n", n, 0.5 * E[n],
                         0.5 * (0.5 * std::pow(1.0 * n, -5.0 / 3.0))) < 0;
    else
      bad = std::fprintf(f, "%i %.16le %.16le\n", 0, 0.0, 0.0) < 0;
  }
  if (std::fclose(f) != 0) bad = 1;
  return bad ? NS3D_ERR_BAD_ARG : NS3D_OK;
}

}  // extern "C"
