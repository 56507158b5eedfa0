// x and y pass instantiations with the reversed radix schedules (tiles 3 and
// 4 of the inv_x, inv_y and fwd_y families), compiled apart from k_xy.cu so
// the two halves build in parallel.
#include "dispatch.h"
#include "launch.cuh"

namespace ns3d {

bool rev_tile_exists(int n, int tile) { return rev_tile_exists_inline(n, tile); }

cudaError_t run_inv_x_rev(const InvXArgs<3>& a, const PassGeom& g, cudaStream_t st) {
  return launch_inv_x<3, double2, 1>(a, g, st);
}
cudaError_t run_inv_x_rev(const InvXArgs<6>& a, const PassGeom& g, cudaStream_t st) {
  return launch_inv_x<6, double2, 1>(a, g, st);
}
cudaError_t run_inv_x_rev(const InvXArgs<3, float2>& a, const PassGeom& g, cudaStream_t st) {
  return launch_inv_x<3, float2, 1>(a, g, st);
}
cudaError_t run_inv_x_rev(const InvXArgs<6, float2>& a, const PassGeom& g, cudaStream_t st) {
  return launch_inv_x<6, float2, 1>(a, g, st);
}
cudaError_t run_inv_y_rev(const InvYArgs<3>& a, const PassGeom& g, cudaStream_t st) {
  return launch_inv_y<3, double2, 1>(a, g, st);
}
cudaError_t run_inv_y_rev(const InvYArgs<6>& a, const PassGeom& g, cudaStream_t st) {
  return launch_inv_y<6, double2, 1>(a, g, st);
}
cudaError_t run_inv_y_rev(const InvYArgs<3, float2>& a, const PassGeom& g, cudaStream_t st) {
  return launch_inv_y<3, float2, 1>(a, g, st);
}
cudaError_t run_inv_y_rev(const InvYArgs<6, float2>& a, const PassGeom& g, cudaStream_t st) {
  return launch_inv_y<6, float2, 1>(a, g, st);
}
cudaError_t run_fwd_y_rev(const FwdYArgs<>& a, const PassGeom& g, cudaStream_t st) {
  return launch_fwd_y<double2, 1>(a, g, st);
}
cudaError_t run_fwd_y_rev(const FwdYArgs<float2>& a, const PassGeom& g, cudaStream_t st) {
  return launch_fwd_y<float2, 1>(a, g, st);
}

namespace {
template <typename C>
cudaError_t prepare_rev_prec(const PassGeom& g, int tile) {
  PassGeom gt = g;
  cudaError_t e;
  gt.tile[kTileInvX] = tile;
  if (rev_tile_exists_inline(g.Nx, tile)) {
    if ((e = launch_inv_x<3, C, 1>(InvXArgs<3, C>{}, gt, nullptr, true)) != cudaSuccess) return e;
    if ((e = launch_inv_x<6, C, 1>(InvXArgs<6, C>{}, gt, nullptr, true)) != cudaSuccess) return e;
  }
  gt.tile[kTileInvY] = gt.tile[kTileFwdY] = tile;
  if (rev_tile_exists_inline(g.Ny, tile)) {
    if ((e = launch_inv_y<3, C, 1>(InvYArgs<3, C>{}, gt, nullptr, true)) != cudaSuccess) return e;
    if ((e = launch_inv_y<6, C, 1>(InvYArgs<6, C>{}, gt, nullptr, true)) != cudaSuccess) return e;
    if ((e = launch_fwd_y<C, 1>(FwdYArgs<C>{}, gt, nullptr, true)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}
}  // namespace

cudaError_t prepare_xy_rev(const PassGeom& g) {
  for (int tile = 3; tile <= 4; ++tile) {
    cudaError_t e = prepare_rev_prec<double2>(g, tile);
    if (e == cudaSuccess) e = prepare_rev_prec<float2>(g, tile);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace ns3d
