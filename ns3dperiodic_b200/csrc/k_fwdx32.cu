// Forward x pass + pointwise update instantiations, FP32 lines (the
// precision mode; the state and the update stay FP64).
#include "dispatch.h"
#include "k_fwdx.cuh"

namespace ns3d {

cudaError_t run_fwd_x(int mode, bool combine, const FwdXArgs<float2>& a, const PassGeom& g,
                      cudaStream_t st) {
  return fwd_x_mode(mode, combine, a, g, st);
}

cudaError_t prepare_fwdx_f32(const PassGeom& g) { return prepare_fwdx_tiles<float2>(g); }

}  // namespace ns3d
