// Forward x pass + pointwise update instantiations.
#include "dispatch.h"
#include "launch.cuh"

namespace ns3d {

cudaError_t run_fwd_x(int mode, bool combine, const FwdXArgs& a, const PassGeom& g,
                      cudaStream_t st) {
  switch (mode) {
    case kExplicit:
      return combine ? launch_fwd_x<kExplicit, true>(a, g, st)
                     : launch_fwd_x<kExplicit, false>(a, g, st);
    case kRhs:
      return launch_fwd_x<kRhs, false>(a, g, st);
    case kImplicit:
      return launch_fwd_x<kImplicit, false>(a, g, st);
    case kConvOut:
      return launch_fwd_x<kConvOut, false>(a, g, st);
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t prepare_fwdx(const PassGeom& g) {
  const FwdXArgs a{};
  cudaError_t e;
  if ((e = launch_fwd_x<kExplicit, false>(a, g, nullptr, true)) != cudaSuccess) return e;
  if ((e = launch_fwd_x<kExplicit, true>(a, g, nullptr, true)) != cudaSuccess) return e;
  if ((e = launch_fwd_x<kRhs, false>(a, g, nullptr, true)) != cudaSuccess) return e;
  if ((e = launch_fwd_x<kImplicit, false>(a, g, nullptr, true)) != cudaSuccess) return e;
  return launch_fwd_x<kConvOut, false>(a, g, nullptr, true);
}

}  // namespace ns3d
