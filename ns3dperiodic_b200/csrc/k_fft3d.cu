// Plain 3-D transform instantiations: complex line passes along x and y in
// both directions, and the paired C2R / R2C z passes.
#include "dispatch.h"
#include "launch.cuh"

namespace ns3d {

cudaError_t run_line(int axis, int dir, const LineArgs& a, const PassGeom& g, cudaStream_t st) {
  if (axis == 0) return dir > 0 ? launch_line<0, +1>(a, g, st) : launch_line<0, -1>(a, g, st);
  return dir > 0 ? launch_line<1, +1>(a, g, st) : launch_line<1, -1>(a, g, st);
}

cudaError_t run_z_c2r(const ZPlainArgs& a, const PassGeom& g, cudaStream_t st) {
  return launch_z_plain<true>(a, g, st);
}

cudaError_t run_z_r2c(const ZPlainArgs& a, const PassGeom& g, cudaStream_t st) {
  return launch_z_plain<false>(a, g, st);
}

cudaError_t prepare_fft3d(const PassGeom& g) {
  cudaError_t e;
  if ((e = launch_line<0, +1>(LineArgs{}, g, nullptr, true)) != cudaSuccess) return e;
  if ((e = launch_line<0, -1>(LineArgs{}, g, nullptr, true)) != cudaSuccess) return e;
  if ((e = launch_line<1, +1>(LineArgs{}, g, nullptr, true)) != cudaSuccess) return e;
  return launch_line<1, -1>(LineArgs{}, g, nullptr, true);
}

}  // namespace ns3d
