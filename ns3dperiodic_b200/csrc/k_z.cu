// z pass instantiations (C2R along z, products, R2C along z).
#include "dispatch.h"
#include "launch.cuh"

namespace ns3d {

cudaError_t run_z(const ZArgs<3>& a, const PassGeom& g, cudaStream_t st) {
  return launch_z<false>(a, g, st);
}
cudaError_t run_z(const ZArgs<6>& a, const PassGeom& g, cudaStream_t st) {
  return launch_z<true>(a, g, st);
}
cudaError_t run_z(const ZArgs<3, float2>& a, const PassGeom& g, cudaStream_t st) {
  return launch_z<false>(a, g, st);
}
cudaError_t run_z(const ZArgs<6, float2>& a, const PassGeom& g, cudaStream_t st) {
  return launch_z<true>(a, g, st);
}

}  // namespace ns3d
