// Mode dispatch of the forward x pass, shared by the FP64 and FP32
// translation units (k_fwdx.cu, k_fwdx32.cu).
#pragma once

#include "launch.cuh"

namespace ns3d {
namespace {

template <typename C>
cudaError_t fwd_x_mode(int mode, bool combine, const FwdXArgs<C>& a, const PassGeom& g,
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

template <typename C>
cudaError_t prepare_fwdx_prec(const PassGeom& g) {
  const FwdXArgs<C> a{};
  cudaError_t e;
  if ((e = launch_fwd_x<kExplicit, false>(a, g, nullptr, true)) != cudaSuccess) return e;
  if ((e = launch_fwd_x<kExplicit, true>(a, g, nullptr, true)) != cudaSuccess) return e;
  if ((e = launch_fwd_x<kRhs, false>(a, g, nullptr, true)) != cudaSuccess) return e;
  if ((e = launch_fwd_x<kImplicit, false>(a, g, nullptr, true)) != cudaSuccess) return e;
  return launch_fwd_x<kConvOut, false>(a, g, nullptr, true);
}

// launch attributes of both tiles of one precision
template <typename C>
cudaError_t prepare_fwdx_tiles(const PassGeom& g) {
  for (int tile = 0; tile < 2; ++tile) {
    PassGeom gt = g;
    for (int& f : gt.tile) f = tile;
    const cudaError_t e = prepare_fwdx_prec<C>(gt);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace
}  // namespace ns3d
