// Internals of the solver handle shared by the translation units that build
// on it (solver.cu: the C ABI of the single grid and the ensembles;
// server.cu: the request server).  Not part of the public ABI.
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/ns3d.h"
#include "aux_kernels.cuh"
#include "diag_kernels.cuh"
#include "passes.cuh"

struct ns3d_solver {
  int Nx = 0, Ny = 0, Nz = 0, Mz = 0;
  double Lx = 0, Ly = 0, Lz = 0;
  size_t nc = 0;  // complex points per field (one instance)
  int batch = 1;  // instances stepped together (ns3d_ensemble); scratch is batch x nc
  int precision = 0;  // NS3D_PRECISION_FP64, or _FP32: transforms and products in FP32
  int tiles[2][4] = {};  // per precision: tile of each pass family (geom.tile is the current)
  double* dtRe = nullptr;  // per instance (dt, Re) of a batch, device
  double ens_dt = 0.0, ens_Re = 0.0;  // the same for an ensemble of one
  bool ens_params = false;            // ns3d_ensemble_set_params was called
  int device = 0;
  ns3d::PassGeom geom{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // tables
  uint16_t* qcut = nullptr;
  double2* tw[3] = {};
  // scratch: base pool (21 fields) and tangent pool (18 fields, lazily)
  double2* pool_base = nullptr;
  double2* pool_uv = nullptr;
  double2* A[6] = {};
  double2* B[6] = {};
  double2* C[6] = {};
  double2* D[6] = {};
  double2* E[6] = {};
  double2* u1[3] = {};
  double2* u2[3] = {};
  double2* v1[3] = {};
  // forcing
  int* f_count = nullptr;
  int* f_idx = nullptr;
  double2* f_val = nullptr;
  int f_nnz = 0;
  const double2* f_dense[3] = {};
  // diagnostics
  double* diag_partial = nullptr;
  double* diag_out = nullptr;
  // record / spectrum / Shapiro buffers (allocated on first use)
  double2* rec_tab = nullptr;
  double* rec_partial = nullptr;  // kDiagBlocks x kRecordSums, then 2 x kDiagBlocks min/max
  double* rec_out = nullptr;      // 50 record columns, then 2 min/max
  ns3d::RecordReads rec_reads{};
  long long rec_points[3] = {};
  // cached RK3 step graph
  cudaGraphExec_t rk3_exec = nullptr;
  const void* rk3_key[3] = {};
  double rk3_dt = 0.0, rk3_Re = 0.0;
  cudaStream_t rk3_stream = nullptr;
  int f_version = 0, rk3_fversion = -1;
  bool graphs_off = false;
  // the captured tangent step (RK3_SSP_UV) of ns3d_jvp_steps and its key
  cudaGraphExec_t jvp_exec = nullptr;
  const void* jvp_key[6] = {};
  double jvp_dt = 0.0, jvp_Re = 0.0;
  cudaStream_t jvp_stream = nullptr;
  int jvp_fversion = -1;
  // tensor maps of inv_y's bulk-copy form (tile 2 of the inv_y family) over
  // A and B; null when the extent has no such form
  ns3d::InvYMaps* ymaps = nullptr;
  int* dev_err = nullptr;  // device flag of the bounded mbarrier waits (0: none gave up)
  size_t bytes = 0;
  std::string err;
};

namespace ns3d_detail {

constexpr int kForcingCap = 4096;
constexpr int kDiagBlocks = 592;  // 4 x 148 SMs
constexpr int kDiagThreads = 256;

ns3d_status fail(ns3d_solver* h, ns3d_status s, const std::string& msg);
ns3d_status cuda_fail(ns3d_solver* h, cudaError_t e, const char* where);
ns3d_status check_handle(ns3d_solver* h);
// a handle for `batch` instances of one grid (batch = 1: ns3d_create)
ns3d_status create_solver(int batch, int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                          ns3d_solver** out);
// the tangent scratch (B(u,v) fields and v1), for the whole batch
ns3d_status ensure_uv_pool(ns3d_solver* h);
// inv_x -> inv_y -> z -> fwd_y (v null: the nonlinear term; else B(u, v))
ns3d_status conv_front(ns3d_solver* h, const double2* const u[3], const double2* const v[3]);
// fwd_x with the pointwise update of `mode` (ns3d::UpdateMode)
ns3d_status finish(ns3d_solver* h, int mode, bool forcing, const double2* const us[3],
                   double2* const out[3], const double2* const un[3], double ca, double cb,
                   double dt, double Re);
// one RK3_SSP step of the state u (all instances of a batch)
ns3d_status rk3_launches(ns3d_solver* h, double2* const u[3], double dt, double Re);

}  // namespace ns3d_detail

#define NS3D_CHECK(h, call, where)                                      \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess) return ns3d_detail::cuda_fail(h, e_, where); \
  } while (0)

#define NS3D_TRY(expr)            \
  do {                            \
    ns3d_status s_ = (expr);      \
    if (s_ != NS3D_OK) return s_; \
  } while (0)
