// Allocation-free variant of the nonlinear-term entry point.
//
// ns3d_convolution() needs about 15 complex fields of scratch, which the
// handle allocates with cudaMalloc when it is created.  Some callers cannot
// do that: programs that reserve all of their device memory up front and
// hand it out from their own pool (a cudaMalloc would fail or fragment it),
// callers that have nowhere to keep a handle alive between calls, and code
// that must not pay for the device-wide synchronisation cudaMalloc and
// cudaFree can imply.  ns3d_convolution_noalloc() serves them: it takes the
// grid and the input/output fields directly and works in a fixed scratch
// array compiled into the library, so it never allocates device memory.
//
// The scratch is one file-scope device array (NS3D_NOALLOC_SCRATCH_BYTES,
// about 33 MB).  A GPU holds it for as long as the process keeps this module
// loaded on that device; with CUDA's default lazy module loading that starts
// at the first call on the device.  All calls on a device share the one
// array: two calls whose work overlaps on the GPU (other streams, other host
// threads) corrupt each other's results, so callers must serialise them.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/ns3d.h"
#include "dispatch.h"
#include "launch.cuh"

namespace {

constexpr long long kMaxPoints = NS3D_NOALLOC_MAX_POINTS;   // complex points per field
constexpr int kMaxExtent = 512;                              // largest compiled extent
constexpr long long kFieldWords = 15 * kMaxPoints;           // A, B, C, D, E x 3
constexpr long long kTwWords = 3 * kMaxExtent;               // twiddles of x, y, z
constexpr long long kQcutWords = kMaxPoints / 4;             // uint16 cut-offs, 8 per word
constexpr long long kWords = kFieldWords + kTwWords + kQcutWords;
static_assert(kWords * 16 == NS3D_NOALLOC_SCRATCH_BYTES, "scratch size and header disagree");
// the twiddle slots hold kMaxExtent entries per direction: every compiled
// extent must fit (a build that adds a larger extent must raise kMaxExtent)
#define NS3D_NOALLOC_EXTENT_FITS(N) static_assert(N <= kMaxExtent, "extent above kMaxExtent");
NS3D_FOR_EACH_EXTENT(NS3D_NOALLOC_EXTENT_FITS)
#undef NS3D_NOALLOC_EXTENT_FITS

// The scratch itself.  Host code must not use this name as an address: on the
// host it is only a stand-in, so it is resolved with cudaGetSymbolAddress.
static __device__ __align__(256) double2 g_scratch[kWords];

constexpr int kMaxDevices = 64;

struct DeviceSlot {
  double2* base = nullptr;  // device address of g_scratch on this device
  // grid whose tables are currently in the scratch
  int Nx = 0, Ny = 0, Nz = 0;
  double Lx = 0, Ly = 0, Lz = 0;
};

std::mutex g_mutex;
DeviceSlot g_slots[kMaxDevices];
uint16_t g_host_qcut[kQcutWords * 8];
double g_host_tw[3][2 * kMaxExtent];

}  // namespace

extern "C" ns3d_status ns3d_convolution_noalloc(int Nx, int Ny, int Nz, double Lx, double Ly,
                                                double Lz, const ns3d_complex* ux,
                                                const ns3d_complex* uy, const ns3d_complex* uz,
                                                ns3d_complex* Qx, ns3d_complex* Qy,
                                                ns3d_complex* Qz, void* stream) {
  if (!ux || !uy || !uz || !Qx || !Qy || !Qz) return NS3D_ERR_BAD_ARG;
  if (Nx <= 0 || Ny <= 0 || Nz <= 0 || !(Lx > 0) || !(Ly > 0) || !(Lz > 0))
    return NS3D_ERR_BAD_ARG;
  if (!ns3d::extent_supported(Nx) || !ns3d::extent_supported(Ny) || !ns3d::extent_supported(Nz))
    return NS3D_ERR_UNSUPPORTED;
  if (Nx > kMaxExtent || Ny > kMaxExtent || Nz > kMaxExtent) return NS3D_ERR_UNSUPPORTED;
  const int Mz = Nz / 2 + 1;
  const long long nc = (long long)Nx * Ny * Mz;
  if (nc > kMaxPoints) return NS3D_ERR_BAD_ARG;  // larger than the fixed scratch
  cudaStream_t st = (cudaStream_t)stream;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return NS3D_ERR_CUDA;

  std::lock_guard<std::mutex> lock(g_mutex);
  DeviceSlot& slot = g_slots[dev];
  if (!slot.base) {
    // once per device, with that device current: the array's device address
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return NS3D_ERR_CUDA;
    }
    slot.base = (double2*)p;
  }
  double2* fields = slot.base;
  double2* tw = slot.base + kFieldWords;
  uint16_t* qcut = (uint16_t*)(slot.base + kFieldWords + kTwWords);

  // wave-number tables: refreshed only when the grid differs from the last call
  if (slot.Nx != Nx || slot.Ny != Ny || slot.Nz != Nz || slot.Lx != Lx || slot.Ly != Ly ||
      slot.Lz != Lz) {
    // the refresh copies from pageable host memory and synchronises the
    // stream, which a stream capture does not allow: refuse it there
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
      cudaGetLastError();
      return NS3D_ERR_CUDA;
    }
    if (cap != cudaStreamCaptureStatusNone) return NS3D_ERR_BAD_ARG;
    if (ns3d_mask_cutoff(Nx, Ny, Nz, Lx, Ly, Lz, g_host_qcut) != NS3D_OK) return NS3D_ERR_BAD_ARG;
    const int ext[3] = {Nx, Ny, Nz};
    for (int d = 0; d < 3; ++d) {
      if (ns3d_twiddles(ext[d], g_host_tw[d]) != NS3D_OK) return NS3D_ERR_BAD_ARG;
      if (cudaMemcpyAsync(tw + d * kMaxExtent, g_host_tw[d], sizeof(double2) * ext[d],
                          cudaMemcpyHostToDevice, st) != cudaSuccess)
        return NS3D_ERR_CUDA;
    }
    if (cudaMemcpyAsync(qcut, g_host_qcut, sizeof(uint16_t) * Nx * Ny, cudaMemcpyHostToDevice,
                        st) != cudaSuccess)
      return NS3D_ERR_CUDA;
    // the host staging arrays are reused by the next refresh
    if (cudaStreamSynchronize(st) != cudaSuccess) return NS3D_ERR_CUDA;
    slot.Nx = Nx; slot.Ny = Ny; slot.Nz = Nz;
    slot.Lx = Lx; slot.Ly = Ly; slot.Lz = Lz;
  }

  ns3d::PassGeom g{};
  g.Nx = Nx; g.Ny = Ny; g.Nz = Nz; g.Mz = Mz;
  g.kfx = 2.0 * M_PI / Lx;
  g.kfy = 2.0 * M_PI / Ly;
  g.kfz = 2.0 * M_PI / Lz;
  g.inv_vol = 1.0 / (1.0 * Nx * Ny * Nz);

  // carve A, B, C, D, E (3 components each) out of the fixed array; every
  // entry is written before it is read, so nothing needs clearing
  double2* A[3];
  double2* B[3];
  double2* C[3];
  double2* D[3];
  double2* E[3];
  for (int i = 0; i < 3; ++i) {
    A[i] = fields + (0 + i) * nc;
    B[i] = fields + (3 + i) * nc;
    C[i] = fields + (6 + i) * nc;
    D[i] = fields + (9 + i) * nc;
    E[i] = fields + (12 + i) * nc;
  }
  const double2* u[3] = {(const double2*)ux, (const double2*)uy, (const double2*)uz};
  double2* Q[3] = {(double2*)Qx, (double2*)Qy, (double2*)Qz};

  ns3d::InvXArgs<3> ax{};
  ns3d::InvYArgs<3> ay{};
  ns3d::ZArgs<3> az{};
  ns3d::FwdYArgs<> fy{};
  ns3d::FwdXArgs<> fx{};
  for (int i = 0; i < 3; ++i) {
    ax.in[i] = u[i]; ax.A[i] = A[i]; ax.B[i] = B[i];
    ay.A[i] = A[i]; ay.B[i] = B[i]; ay.C[i] = C[i]; ay.D[i] = D[i]; ay.E[i] = E[i];
    az.C[i] = C[i]; az.D[i] = D[i]; az.E[i] = E[i]; az.Qh[i] = A[i];
    fy.Q[i] = A[i];
    fx.Qh[i] = A[i]; fx.out[i] = Q[i];
  }
  ax.qcut = qcut;
  ax.tw = tw;
  ay.tw = tw + kMaxExtent;
  az.tw = tw + 2 * kMaxExtent;
  fy.tw = tw + kMaxExtent;
  fx.tw = tw;
  fx.cb = 1.0;
  fx.Re = 1.0;
  if (ns3d::run_inv_x(ax, g, st) != cudaSuccess) return NS3D_ERR_CUDA;
  if (ns3d::run_inv_y(ay, g, st) != cudaSuccess) return NS3D_ERR_CUDA;
  if (ns3d::run_z(az, g, st) != cudaSuccess) return NS3D_ERR_CUDA;
  if (ns3d::run_fwd_y(fy, g, st) != cudaSuccess) return NS3D_ERR_CUDA;
  if (ns3d::run_fwd_x(ns3d::kConvOut, false, fx, g, st) != cudaSuccess) return NS3D_ERR_CUDA;
  return NS3D_OK;
}
