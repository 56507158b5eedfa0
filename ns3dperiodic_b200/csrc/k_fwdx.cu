// Forward x pass + pointwise update instantiations, FP64 lines (the FP32
// lines of the precision mode are in k_fwdx32.cu: the two halves compile in
// parallel).
#include "dispatch.h"
#include "k_fwdx.cuh"

namespace ns3d {

cudaError_t run_fwd_x(int mode, bool combine, const FwdXArgs<>& a, const PassGeom& g,
                      cudaStream_t st) {
  return fwd_x_mode(mode, combine, a, g, st);
}

cudaError_t prepare_fwdx(const PassGeom& g) {
  cudaError_t e = prepare_fwdx_tiles<double2>(g);
  if (e == cudaSuccess) e = prepare_fwdx_f32(g);
  return e;
}

}  // namespace ns3d
