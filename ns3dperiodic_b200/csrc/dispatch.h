// Concrete launch entry points of the pass kernels.  Each group lives in its
// own translation unit (k_xy.cu, k_z.cu, k_fwdx.cu) so the per-extent
// template instantiations compile in parallel.
#pragma once

#include <cuda_runtime.h>

#include "passes.cuh"

namespace ns3d {

bool extent_supported(int n);
// whether extent n has an alternative tile for the autotuner (p_alt)
bool extent_has_alt_tile(int n);
// lines per CTA of inv_y's bulk-copy (TMA) form (tile 2 of the inv_y family)
// for extent n, 0 when the extent has no such form
int inv_y_tma_lpc(int n);
// whether the x / y families' tile 3 (default points per thread) or 4 (the
// alternative) - the reversed radix schedule - exists for extent n
bool rev_tile_exists(int n, int tile);
// Tiles 3 and 4 of inv_x, inv_y and fwd_y (k_xy_rev.cu); run_inv_x etc.
// forward to these for those tiles.
cudaError_t run_inv_x_rev(const InvXArgs<3>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_inv_x_rev(const InvXArgs<6>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_inv_x_rev(const InvXArgs<3, float2>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_inv_x_rev(const InvXArgs<6, float2>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_inv_y_rev(const InvYArgs<3>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_inv_y_rev(const InvYArgs<6>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_inv_y_rev(const InvYArgs<3, float2>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_inv_y_rev(const InvYArgs<6, float2>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_fwd_y_rev(const FwdYArgs<>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_fwd_y_rev(const FwdYArgs<float2>& a, const PassGeom& g, cudaStream_t st);
cudaError_t prepare_xy_rev(const PassGeom& g);

// FP64 scratch (double2) and the FP32 precision mode (float2 scratch).
cudaError_t run_inv_x(const InvXArgs<3>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_inv_x(const InvXArgs<6>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_inv_y(const InvYArgs<3>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_inv_y(const InvYArgs<6>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_fwd_y(const FwdYArgs<>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_z(const ZArgs<3>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_z(const ZArgs<6>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_inv_x(const InvXArgs<3, float2>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_inv_x(const InvXArgs<6, float2>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_inv_y(const InvYArgs<3, float2>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_inv_y(const InvYArgs<6, float2>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_fwd_y(const FwdYArgs<float2>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_z(const ZArgs<3, float2>& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_z(const ZArgs<6, float2>& a, const PassGeom& g, cudaStream_t st);
// Launch attributes of the pipelined passes for this geometry on the current
// device; called when a handle is created (outside any stream capture).
cudaError_t prepare_xy(const PassGeom& g);
cudaError_t prepare_fwdx(const PassGeom& g);
cudaError_t prepare_fwdx_f32(const PassGeom& g);  // the FP32 half (k_fwdx32.cu)
// Plain 3-D transforms (k_fft3d.cu): one complex line pass along x (axis 0)
// or y (axis 1), dir +1 inverse / -1 forward; the paired z passes.
cudaError_t run_line(int axis, int dir, const LineArgs& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_z_c2r(const ZPlainArgs& a, const PassGeom& g, cudaStream_t st);
cudaError_t run_z_r2c(const ZPlainArgs& a, const PassGeom& g, cudaStream_t st);
cudaError_t prepare_fft3d(const PassGeom& g);
// mode: UpdateMode; combine: out = ca*un + cb*base
cudaError_t run_fwd_x(int mode, bool combine, const FwdXArgs<>& a, const PassGeom& g,
                      cudaStream_t st);
cudaError_t run_fwd_x(int mode, bool combine, const FwdXArgs<float2>& a, const PassGeom& g,
                      cudaStream_t st);

}  // namespace ns3d
