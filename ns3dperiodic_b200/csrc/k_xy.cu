// x and y pass instantiations (inverse x/y with lazy derivatives, forward y).
#include "dispatch.h"
#include "launch.cuh"

namespace ns3d {

bool extent_supported(int n) { return extent_supported_inline(n); }
bool extent_has_alt_tile(int n) { return has_alt_tile(n); }
int inv_y_tma_lpc(int n) { return inv_y_tma_lpc_inline(n); }

cudaError_t run_inv_x(const InvXArgs<3>& a, const PassGeom& g, cudaStream_t st) {
  if (g.tile[kTileInvX] >= 3) return run_inv_x_rev(a, g, st);
  return launch_inv_x<3>(a, g, st);
}
cudaError_t run_inv_x(const InvXArgs<6>& a, const PassGeom& g, cudaStream_t st) {
  if (g.tile[kTileInvX] >= 3) return run_inv_x_rev(a, g, st);
  return launch_inv_x<6>(a, g, st);
}
cudaError_t run_inv_y(const InvYArgs<3>& a, const PassGeom& g, cudaStream_t st) {
  if (g.tile[kTileInvY] >= 3) return run_inv_y_rev(a, g, st);
  return launch_inv_y<3>(a, g, st);
}
cudaError_t run_inv_y(const InvYArgs<6>& a, const PassGeom& g, cudaStream_t st) {
  if (g.tile[kTileInvY] >= 3) return run_inv_y_rev(a, g, st);
  return launch_inv_y<6>(a, g, st);
}
cudaError_t run_fwd_y(const FwdYArgs<>& a, const PassGeom& g, cudaStream_t st) {
  if (g.tile[kTileFwdY] >= 3) return run_fwd_y_rev(a, g, st);
  return launch_fwd_y(a, g, st);
}
cudaError_t run_inv_x(const InvXArgs<3, float2>& a, const PassGeom& g, cudaStream_t st) {
  if (g.tile[kTileInvX] >= 3) return run_inv_x_rev(a, g, st);
  return launch_inv_x<3>(a, g, st);
}
cudaError_t run_inv_x(const InvXArgs<6, float2>& a, const PassGeom& g, cudaStream_t st) {
  if (g.tile[kTileInvX] >= 3) return run_inv_x_rev(a, g, st);
  return launch_inv_x<6>(a, g, st);
}
cudaError_t run_inv_y(const InvYArgs<3, float2>& a, const PassGeom& g, cudaStream_t st) {
  if (g.tile[kTileInvY] >= 3) return run_inv_y_rev(a, g, st);
  return launch_inv_y<3>(a, g, st);
}
cudaError_t run_inv_y(const InvYArgs<6, float2>& a, const PassGeom& g, cudaStream_t st) {
  if (g.tile[kTileInvY] >= 3) return run_inv_y_rev(a, g, st);
  return launch_inv_y<6>(a, g, st);
}
cudaError_t run_fwd_y(const FwdYArgs<float2>& a, const PassGeom& g, cudaStream_t st) {
  if (g.tile[kTileFwdY] >= 3) return run_fwd_y_rev(a, g, st);
  return launch_fwd_y(a, g, st);
}

namespace {
template <typename C>
cudaError_t prepare_xy_prec(const PassGeom& g) {
  cudaError_t e;
  if ((e = launch_inv_x<3>(InvXArgs<3, C>{}, g, nullptr, true)) != cudaSuccess) return e;
  if ((e = launch_inv_x<6>(InvXArgs<6, C>{}, g, nullptr, true)) != cudaSuccess) return e;
  if ((e = launch_inv_y<3>(InvYArgs<3, C>{}, g, nullptr, true)) != cudaSuccess) return e;
  if ((e = launch_inv_y<6>(InvYArgs<6, C>{}, g, nullptr, true)) != cudaSuccess) return e;
  return launch_fwd_y(FwdYArgs<C>{}, g, nullptr, true);
}
}  // namespace

cudaError_t prepare_xy(const PassGeom& g) {
  // both tiles of every pass family, then the inv_y family's bulk-copy tile
  for (int tile = 0; tile < 3; ++tile) {
    PassGeom gt = g;
    for (int& f : gt.tile) f = tile < 2 ? tile : 0;
    if (tile == 2) gt.tile[kTileInvY] = 2;
    cudaError_t e = prepare_xy_prec<double2>(gt);
    if (e == cudaSuccess) e = prepare_xy_prec<float2>(gt);
    if (e != cudaSuccess) return e;
  }
  return prepare_xy_rev(g);  // tiles 3 and 4
}

}  // namespace ns3d
