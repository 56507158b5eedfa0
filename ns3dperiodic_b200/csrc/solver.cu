// Host side of the C ABI (include/ns3d.h): handle, scratch, RHS pipelines and
// the steppers of Source/RK_time_step.cu rebuilt on the fused pass kernels.
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled

#include "../../include/ns3d.h"
#include "aux_kernels.cuh"
#include "diag_kernels.cuh"
#include "dispatch.h"
#include "solver_internal.h"

using ns3d::FwdXArgs;
using ns3d::FwdYArgs;
using ns3d::InvXArgs;
using ns3d::InvYArgs;
using ns3d::PassGeom;
using ns3d::ZArgs;
using namespace ns3d_detail;



namespace ns3d_detail {

ns3d_status fail(ns3d_solver* h, ns3d_status s, const std::string& msg) {
  if (h) h->err = msg;
  return s;
}

ns3d_status cuda_fail(ns3d_solver* h, cudaError_t e, const char* where) {
  return fail(h, e == cudaErrorMemoryAllocation ? NS3D_ERR_OOM : NS3D_ERR_CUDA,
              std::string(where) + ": " + cudaGetErrorString(e));
}


void build_twiddles(int N, std::vector<double2>& out) {
  out.resize(N);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int e = 0; e < N; ++e) {
    // exact symmetric values where they exist, long double elsewhere
    long double a = two_pi * (long double)e / (long double)N;
    double c = (double)cosl(a), s = (double)sinl(a);
    if ((4 * e) % N == 0) {
      const int q = (4 * e) / N;  // multiples of 90 degrees
      c = q == 0 ? 1.0 : q == 2 ? -1.0 : 0.0;
      s = q == 1 ? 1.0 : q == 3 ? -1.0 : 0.0;
    }
    out[e] = make_double2(c, s);
  }
}

// build_mask_matrix (Source/math_support.cu:471-519) evaluated as main()
// calls it: Nz slot = Mz, so kzMax = 2*Mz*PI/Lz.  Returns false if the kept
// modes of some (j,k) column are not a prefix in l.
bool build_mask_cutoff(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                       uint16_t* qcut) {
  const double PI = 3.141592653589793238462643383279502884197169399375105820974944592307816406;
  const int Mz = Nz / 2 + 1;
  volatile double kxMax = 2 * Nx * PI / Lx;
  volatile double kyMax = 2 * Ny * PI / Ly;
  volatile double kzMax = 2 * Mz * PI / Lz;
  for (int j = 0; j < Nx; ++j) {
    const int m = j >= Nx / 2 ? j - Nx : j;
    for (int k = 0; k < Ny; ++k) {
      const int n = k >= Ny / 2 ? k - Ny : k;
      int cut = 0;
      bool ended = false;
      for (int l = 0; l < Mz; ++l) {
        const int q = l;
        volatile double kx = m * 2 * PI / Lx;
        volatile double ky = n * 2 * PI / Ly;
        volatile double kz = q * 2 * PI / Lz;
        volatile double tx = kx * kx / (kxMax * kxMax);
        volatile double ty = ky * ky / (kyMax * kyMax);
        volatile double tz = kz * kz / (kzMax * kzMax);
        volatile double s2 = tx + ty;
        s2 = s2 + tz;
        const double sphere2 = std::sqrt((double)s2);
        const bool keep = sphere2 < 2.0 / 3.0;
        if (keep) {
          if (ended) return false;
          ++cut;
        } else {
          ended = true;
        }
      }
      qcut[j * Ny + k] = (uint16_t)cut;
    }
  }
  return true;
}

bool valid_extents(int Nx, int Ny, int Nz) {
  return ns3d::extent_supported(Nx) && ns3d::extent_supported(Ny) && ns3d::extent_supported(Nz);
}

ns3d_status ensure_uv_pool(ns3d_solver* h) {
  if (h->pool_uv) return NS3D_OK;
  const size_t field = h->nc * (size_t)h->batch;
  const size_t bytes = sizeof(double2) * field * 18;
  NS3D_CHECK(h, cudaMalloc(&h->pool_uv, bytes), "cudaMalloc(tangent scratch)");
  h->bytes += bytes;
  double2* p = h->pool_uv;
  for (int i = 3; i < 6; ++i) {
    h->A[i] = p; p += field;
    h->B[i] = p; p += field;
    h->C[i] = p; p += field;
    h->D[i] = p; p += field;
    h->E[i] = p; p += field;
  }
  for (int i = 0; i < 3; ++i) { h->v1[i] = p; p += field; }
  return NS3D_OK;
}

// inv_x -> inv_y -> z -> fwd_y: leaves the y,z-transformed products in A[0..2]
// (FP64 scratch, or FP32 scratch in the precision mode).
template <typename C>
ns3d_status conv_front_t(ns3d_solver* h, const double2* const u[3],
                         const double2* const v[3]) {
  auto sc = [](double2* p) { return reinterpret_cast<C*>(p); };
  const PassGeom& g = h->geom;
  cudaStream_t st = h->stream;
  if (!v) {
    InvXArgs<3, C> ax{};
    InvYArgs<3, C> ay{};
    ZArgs<3, C> az{};
    for (int i = 0; i < 3; ++i) {
      ax.in[i] = u[i]; ax.A[i] = sc(h->A[i]); ax.B[i] = sc(h->B[i]);
      ay.A[i] = sc(h->A[i]); ay.B[i] = sc(h->B[i]);
      ay.C[i] = sc(h->C[i]); ay.D[i] = sc(h->D[i]); ay.E[i] = sc(h->E[i]);
      az.C[i] = sc(h->C[i]); az.D[i] = sc(h->D[i]); az.E[i] = sc(h->E[i]);
      az.Qh[i] = sc(h->A[i]);
    }
    ax.qcut = h->qcut; ax.tw = h->tw[0];
    ay.tw = h->tw[1];
    az.tw = h->tw[2];
    if (sizeof(C) == 16 && g.tile[ns3d::kTileInvY] == 2) {  // FP64: the bulk-copy form
      ay.maps = h->ymaps;
      ay.err = h->dev_err;
    }
    NS3D_CHECK(h, ns3d::run_inv_x(ax, g, st), "inv_x");
    NS3D_CHECK(h, ns3d::run_inv_y(ay, g, st), "inv_y");
    NS3D_CHECK(h, ns3d::run_z(az, g, st), "z");
  } else {
    ns3d_status s = ensure_uv_pool(h);
    if (s != NS3D_OK) return s;
    InvXArgs<6, C> ax{};
    InvYArgs<6, C> ay{};
    ZArgs<6, C> az{};
    for (int i = 0; i < 6; ++i) {
      ax.in[i] = i < 3 ? u[i] : v[i - 3];
      ax.A[i] = sc(h->A[i]); ax.B[i] = sc(h->B[i]);
      ay.A[i] = sc(h->A[i]); ay.B[i] = sc(h->B[i]);
      ay.C[i] = sc(h->C[i]); ay.D[i] = sc(h->D[i]); ay.E[i] = sc(h->E[i]);
      az.C[i] = sc(h->C[i]); az.D[i] = sc(h->D[i]); az.E[i] = sc(h->E[i]);
    }
    for (int i = 0; i < 3; ++i) az.Qh[i] = sc(h->A[i]);
    ax.qcut = h->qcut; ax.tw = h->tw[0];
    ay.tw = h->tw[1];
    az.tw = h->tw[2];
    NS3D_CHECK(h, ns3d::run_inv_x(ax, g, st), "inv_x(uv)");
    NS3D_CHECK(h, ns3d::run_inv_y(ay, g, st), "inv_y(uv)");
    NS3D_CHECK(h, ns3d::run_z(az, g, st), "z(uv)");
  }
  FwdYArgs<C> fy{};
  for (int i = 0; i < 3; ++i) fy.Q[i] = sc(h->A[i]);
  fy.tw = h->tw[1];
  NS3D_CHECK(h, ns3d::run_fwd_y(fy, g, st), "fwd_y");
  return NS3D_OK;
}

ns3d_status conv_front(ns3d_solver* h, const double2* const u[3], const double2* const v[3]) {
  return h->precision == NS3D_PRECISION_FP32 ? conv_front_t<float2>(h, u, v)
                                             : conv_front_t<double2>(h, u, v);
}

// fwd_x + pointwise update on the products left by conv_front.
template <typename C>
ns3d_status finish_t(ns3d_solver* h, int mode, bool forcing, const double2* const us[3],
                     double2* const out[3], const double2* const un[3], double ca, double cb,
                     double dt, double Re) {
  FwdXArgs<C> a{};
  for (int i = 0; i < 3; ++i) {
    a.Qh[i] = reinterpret_cast<const C*>(h->A[i]);
    a.us[i] = us ? us[i] : nullptr;
    a.un[i] = un ? un[i] : nullptr;
    a.out[i] = out[i];
    a.fd[i] = (forcing && h->f_dense[0]) ? h->f_dense[i] : nullptr;
  }
  a.fidx = h->f_idx;
  a.fval = h->f_val;
  a.fnnz = (forcing && !h->f_dense[0]) ? h->f_nnz : 0;
  a.dt = dt;
  a.Re = Re;
  a.dtRe = h->dtRe;  // allocated for batches (and server grids) only
  a.ca = ca;
  a.cb = cb;
  a.tw = h->tw[0];
  NS3D_CHECK(h, ns3d::run_fwd_x(mode, un != nullptr, a, h->geom, h->stream), "fwd_x");
  return NS3D_OK;
}

ns3d_status finish(ns3d_solver* h, int mode, bool forcing, const double2* const us[3],
                   double2* const out[3], const double2* const un[3], double ca, double cb,
                   double dt, double Re) {
  return h->precision == NS3D_PRECISION_FP32
             ? finish_t<float2>(h, mode, forcing, us, out, un, ca, cb, dt, Re)
             : finish_t<double2>(h, mode, forcing, us, out, un, ca, cb, dt, Re);
}


// RK3_SSP (Source/RK_time_step.cu:310-327) with every stage fused:
//   u1 = u + dt L(u); u2 = 3/4 u + 1/4 (u1 + dt L(u1)); u = 1/3 u + 2/3 (u2 + dt L(u2))
ns3d_status rk3_launches(ns3d_solver* h, double2* const u[3], double dt, double Re) {
  const double2* uc[3] = {u[0], u[1], u[2]};
  const double2* u1c[3] = {h->u1[0], h->u1[1], h->u1[2]};
  const double2* u2c[3] = {h->u2[0], h->u2[1], h->u2[2]};
  NS3D_TRY(conv_front(h, uc, nullptr));
  NS3D_TRY(finish(h, ns3d::kExplicit, true, uc, h->u1, nullptr, 0.0, 1.0, dt, Re));
  NS3D_TRY(conv_front(h, u1c, nullptr));
  NS3D_TRY(finish(h, ns3d::kExplicit, true, u1c, h->u2, uc, 3.0 / 4.0, 1.0 / 4.0, dt, Re));
  NS3D_TRY(conv_front(h, u2c, nullptr));
  NS3D_TRY(finish(h, ns3d::kExplicit, true, u2c, u, uc, 1.0 / 3.0, 2.0 / 3.0, dt, Re));
  return NS3D_OK;
}

bool args_ok3(const void* a, const void* b, const void* c) { return a && b && c; }

ns3d_status check_handle(ns3d_solver* h) {
  if (!h) return NS3D_ERR_BAD_ARG;
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
  h->err.clear();
  return NS3D_OK;
}

ns3d_status check_step(ns3d_solver* h, double dt, double Re) {
  if (!(Re > 0.0) || !std::isfinite(Re) || !std::isfinite(dt))
    return fail(h, NS3D_ERR_BAD_ARG, "dt must be finite and Re > 0");
  return NS3D_OK;
}

void drop_graph(ns3d_solver* h) {
  if (h->rk3_exec) cudaGraphExecDestroy(h->rk3_exec);
  h->rk3_exec = nullptr;
  if (h->jvp_exec) cudaGraphExecDestroy(h->jvp_exec);
  h->jvp_exec = nullptr;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int ns3d_supported_extent(int n) { return ns3d::extent_supported(n) ? 1 : 0; }

const char* ns3d_status_string(ns3d_status s) {
  switch (s) {
    case NS3D_OK: return "ok";
    case NS3D_ERR_BAD_ARG: return "bad argument";
    case NS3D_ERR_UNSUPPORTED: return "unsupported grid extent";
    case NS3D_ERR_OOM: return "out of device memory";
    case NS3D_ERR_CUDA: return "CUDA error";
    case NS3D_ERR_NONFINITE: return "non-finite value";
    case NS3D_ERR_TIMEOUT: return "device wait timed out";
    case NS3D_ERR_NOT_CONVERGED: return "inner linear solve did not converge";
    case NS3D_ERR_CANCELLED: return "request cancelled";
  }
  return "unknown status";
}

const char* ns3d_last_error(const ns3d_solver* h) { return h ? h->err.c_str() : ""; }

size_t ns3d_device_bytes(const ns3d_solver* h) { return h ? h->bytes : 0; }

ns3d_status ns3d_mask_cutoff(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                             uint16_t* qcut) {
  if (Nx <= 0 || Ny <= 0 || Nz <= 0 || !qcut || !(Lx > 0) || !(Ly > 0) || !(Lz > 0))
    return NS3D_ERR_BAD_ARG;
  return build_mask_cutoff(Nx, Ny, Nz, Lx, Ly, Lz, qcut) ? NS3D_OK : NS3D_ERR_BAD_ARG;
}

extern "C++" {
namespace {
// One CTA waits on a phase of an mbarrier that nothing arrives on.
__global__ void bounded_wait_probe(int* err) {
  __shared__ uint64_t bar;
  __shared__ int bad;
  if (threadIdx.x == 0) {
    ns3d::mbar_init(&bar, 1);
    bad = 0;
  }
  __syncthreads();
  ns3d::mbar_wait(&bar, 0, err, &bad);
}
}  // namespace
}  // extern "C++"

ns3d_status ns3d_selftest_bounded_wait(double* seconds) {
  int* flag = nullptr;
  if (cudaMalloc(&flag, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return NS3D_ERR_OOM;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int got = 0;
  cudaError_t e = cudaMemset(flag, 0, sizeof(int));
  if (e == cudaSuccess) {
    cudaEventRecord(e0);
    bounded_wait_probe<<<1, 64>>>(flag);
    cudaEventRecord(e1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  if (e == cudaSuccess) e = cudaMemcpy(&got, flag, sizeof(int), cudaMemcpyDeviceToHost);
  float ms = 0.f;
  if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(flag);
  if (seconds) *seconds = 1e-3 * ms;
  return (e == cudaSuccess && got == ns3d::kErrTimeout) ? NS3D_OK : NS3D_ERR_CUDA;
}

ns3d_status ns3d_twiddles(int N, double* tw) {
  if (N <= 0 || !tw) return NS3D_ERR_BAD_ARG;
  std::vector<double2> t;
  build_twiddles(N, t);
  std::memcpy(tw, t.data(), sizeof(double2) * N);
  return NS3D_OK;
}

extern "C++" {
namespace ns3d_detail {
// L2 promotion of inv_y's bulk copies (CUtensorMapL2promotion: 0 none,
// 1 64 B, 2 128 B, 3 256 B)
#ifndef NS3D_TMA_L2PROMO
#define NS3D_TMA_L2PROMO 3
#endif

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library does not link the driver; null when it is not available)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    cudaGetLastError();
  });
  return fn;
}

// Tensor maps of inv_y's bulk-copy form over the FP64 scratch A_f, B_f (all
// instances of a batch as x planes).  A field is dims (2 Mz doubles, Ny,
// planes) with row strides Mz * 16 and Ny * Mz * 16 bytes; a box is
// (2 LPC, tma_box_y(Ny), 1).  Any failure leaves the handle without the form
// (ns3d_set_tiles then refuses tile 2 of the inv_y family).
void build_inv_y_maps(ns3d_solver* h) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return;
  {
    const int lpc = ns3d::inv_y_tma_lpc(h->Ny);
    if (lpc <= 0) return;
    auto* m = new ns3d::InvYMaps();
    bool ok = true;
    for (int f = 0; f < 6 && ok; ++f) {
      const double2* base = (f & 1) ? h->B[f >> 1] : h->A[f >> 1];
      const cuuint64_t dims[3] = {2ull * (cuuint64_t)h->Mz, (cuuint64_t)h->Ny,
                                  (cuuint64_t)h->Nx * (cuuint64_t)h->batch};
      const cuuint64_t strides[2] = {16ull * (cuuint64_t)h->Mz,
                                     16ull * (cuuint64_t)h->Mz * (cuuint64_t)h->Ny};
      const cuuint32_t box[3] = {2u * (cuuint32_t)lpc, (cuuint32_t)ns3d::tma_box_y(h->Ny), 1u};
      const cuuint32_t estr[3] = {1u, 1u, 1u};
      ok = enc(&m->map[f], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void*)base, dims, strides, box,
               estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               (CUtensorMapL2promotion)NS3D_TMA_L2PROMO, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
    }
    if (ok) {
      h->ymaps = m;
    } else {
      delete m;
    }
  }
}

ns3d_status create_solver(int batch, int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                          ns3d_solver** out) {
  if (!out) return NS3D_ERR_BAD_ARG;
  *out = nullptr;
  if (Nx <= 0 || Ny <= 0 || Nz <= 0 || !(Lx > 0) || !(Ly > 0) || !(Lz > 0) || batch < 1)
    return NS3D_ERR_BAD_ARG;
  if (!valid_extents(Nx, Ny, Nz)) return NS3D_ERR_UNSUPPORTED;
  // the x passes index lines of the whole batch with 32-bit integers
  if ((long long)batch * Ny * (Nz / 2 + 1) >= (1LL << 31) ||
      (long long)batch * Nx * Ny >= (1LL << 31))
    return NS3D_ERR_BAD_ARG;
  ns3d_solver* h = new ns3d_solver();
  h->Nx = Nx; h->Ny = Ny; h->Nz = Nz; h->Mz = Nz / 2 + 1;
  h->Lx = Lx; h->Ly = Ly; h->Lz = Lz;
  h->nc = (size_t)Nx * Ny * h->Mz;
  h->batch = batch;
  cudaGetDevice(&h->device);
  h->geom.Nx = Nx; h->geom.Ny = Ny; h->geom.Nz = Nz; h->geom.Mz = h->Mz;
  h->geom.batch = batch;
  // 2.0*M_PI/L as in build_Nabla_Wavenumbers (Source/math_support.cu:398-413)
  h->geom.kfx = 2.0 * M_PI / Lx;
  h->geom.kfy = 2.0 * M_PI / Ly;
  h->geom.kfz = 2.0 * M_PI / Lz;
  h->geom.inv_vol = 1.0 / (1.0 * Nx * Ny * Nz);

  auto bail = [&](ns3d_status s) {
    ns3d_destroy(h);
    cudaGetLastError();  // a failed allocation must not surface at the next launch check
    return s;
  };
  std::vector<uint16_t> qc((size_t)Nx * Ny);
  if (!build_mask_cutoff(Nx, Ny, Nz, Lx, Ly, Lz, qc.data())) return bail(NS3D_ERR_BAD_ARG);
  cudaError_t e;
  if ((e = cudaStreamCreate(&h->stream)) != cudaSuccess) return bail(NS3D_ERR_CUDA);
  h->own_stream = true;
  if ((e = cudaMalloc(&h->qcut, sizeof(uint16_t) * qc.size())) != cudaSuccess)
    return bail(NS3D_ERR_OOM);
  cudaMemcpy(h->qcut, qc.data(), sizeof(uint16_t) * qc.size(), cudaMemcpyHostToDevice);
  const int ext[3] = {Nx, Ny, Nz};
  for (int d = 0; d < 3; ++d) {
    std::vector<double2> t;
    build_twiddles(ext[d], t);
    if (cudaMalloc(&h->tw[d], sizeof(double2) * t.size()) != cudaSuccess) return bail(NS3D_ERR_OOM);
    cudaMemcpy(h->tw[d], t.data(), sizeof(double2) * t.size(), cudaMemcpyHostToDevice);
  }
  const size_t field = h->nc * (size_t)batch;  // one scratch field of the whole batch
  const size_t base_bytes = sizeof(double2) * field * 21;
  if (cudaMalloc(&h->pool_base, base_bytes) != cudaSuccess) return bail(NS3D_ERR_OOM);
  h->bytes = base_bytes + sizeof(uint16_t) * qc.size() + sizeof(double2) * (Nx + Ny + Nz);
  double2* p = h->pool_base;
  for (int i = 0; i < 3; ++i) {
    h->A[i] = p; p += field;
    h->B[i] = p; p += field;
    h->C[i] = p; p += field;
    h->D[i] = p; p += field;
    h->E[i] = p; p += field;
    h->u1[i] = p; p += field;
    h->u2[i] = p; p += field;
  }
  if (cudaMalloc(&h->f_count, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&h->f_idx, sizeof(int) * kForcingCap) != cudaSuccess ||
      cudaMalloc(&h->f_val, sizeof(double2) * 3 * kForcingCap) != cudaSuccess ||
      cudaMalloc(&h->diag_partial, sizeof(double) * 3 * kDiagBlocks) != cudaSuccess ||
      cudaMalloc(&h->diag_out, sizeof(double) * 3 * batch) != cudaSuccess)
    return bail(NS3D_ERR_OOM);
  if (cudaMalloc(&h->dev_err, sizeof(int)) != cudaSuccess) return bail(NS3D_ERR_OOM);
  cudaMemset(h->dev_err, 0, sizeof(int));
  build_inv_y_maps(h);
  if (batch > 1) {
    if (cudaMalloc(&h->dtRe, sizeof(double) * 2 * batch) != cudaSuccess) return bail(NS3D_ERR_OOM);
    std::vector<double> ones(2 * batch, 1.0);
    cudaMemcpy(h->dtRe, ones.data(), sizeof(double) * 2 * batch, cudaMemcpyHostToDevice);
  }
  if ((e = ns3d::prepare_xy(h->geom)) != cudaSuccess) return bail(NS3D_ERR_CUDA);
  if ((e = ns3d::prepare_fwdx(h->geom)) != cudaSuccess) return bail(NS3D_ERR_CUDA);
  if ((e = ns3d::prepare_fft3d(h->geom)) != cudaSuccess) return bail(NS3D_ERR_CUDA);
  if ((e = cudaDeviceSynchronize()) != cudaSuccess) return bail(NS3D_ERR_CUDA);
  *out = h;
  return NS3D_OK;
}
}  // namespace ns3d_detail
}  // extern "C++"

ns3d_status ns3d_create(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                        ns3d_solver** out) {
  return create_solver(1, Nx, Ny, Nz, Lx, Ly, Lz, out);
}

ns3d_status ns3d_destroy(ns3d_solver* h) {
  if (!h) return NS3D_ERR_BAD_ARG;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  drop_graph(h);
  cudaFree(h->qcut);
  for (auto* t : h->tw) cudaFree(t);
  cudaFree(h->pool_base);
  cudaFree(h->pool_uv);
  cudaFree(h->f_count);
  cudaFree(h->f_idx);
  cudaFree(h->f_val);
  cudaFree(h->diag_partial);
  cudaFree(h->diag_out);
  cudaFree(h->dtRe);
  cudaFree(h->rec_tab);
  cudaFree(h->rec_partial);
  cudaFree(h->rec_out);
  cudaFree(h->dev_err);
  delete h->ymaps;
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return NS3D_OK;
}

ns3d_status ns3d_set_stream(ns3d_solver* h, void* stream) {
  NS3D_TRY(check_handle(h));
  if (h->own_stream && h->stream) {
    cudaStreamSynchronize(h->stream);
    cudaStreamDestroy(h->stream);
  }
  h->own_stream = false;
  h->stream = (cudaStream_t)stream;
  drop_graph(h);
  h->graphs_off = false;
  return NS3D_OK;
}

ns3d_status ns3d_synchronize(ns3d_solver* h) {
  NS3D_TRY(check_handle(h));
  NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
  // a bounded wait of a bulk-copy pass that gave up (its results are invalid)
  int flag = 0;
  if (h->dev_err) {
    NS3D_CHECK(h, cudaMemcpyAsync(&flag, h->dev_err, sizeof(int), cudaMemcpyDeviceToHost,
                                  h->stream), "error flag");
    NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "error flag");
  }
  if (flag) {
    cudaMemsetAsync(h->dev_err, 0, sizeof(int), h->stream);
    return fail(h, NS3D_ERR_TIMEOUT, "a bounded wait of a pass kernel gave up");
  }
  return NS3D_OK;
}

ns3d_status ns3d_set_forcing(ns3d_solver* h, const ns3d_complex* fx, const ns3d_complex* fy,
                             const ns3d_complex* fz) {
  NS3D_TRY(check_handle(h));
  h->f_version++;
  h->f_dense[0] = h->f_dense[1] = h->f_dense[2] = nullptr;
  h->f_nnz = 0;
  if (!fx && !fy && !fz) return NS3D_OK;
  if (!args_ok3(fx, fy, fz)) return fail(h, NS3D_ERR_BAD_ARG, "forcing needs 3 components");
  NS3D_CHECK(h, cudaMemsetAsync(h->f_count, 0, sizeof(int), h->stream), "memset");
  ns3d::forcing_scan_kernel<<<592, 256, 0, h->stream>>>(
      (const double2*)fx, (const double2*)fy, (const double2*)fz, (long long)h->nc, kForcingCap,
      h->f_count, h->f_idx, h->f_val);
  NS3D_CHECK(h, cudaGetLastError(), "forcing_scan");
  int count = 0;
  NS3D_CHECK(h, cudaMemcpyAsync(&count, h->f_count, sizeof(int), cudaMemcpyDeviceToHost, h->stream),
             "forcing count");
  NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "forcing sync");
  if (count > kForcingCap) {
    h->f_dense[0] = (const double2*)fx;
    h->f_dense[1] = (const double2*)fy;
    h->f_dense[2] = (const double2*)fz;
  } else {
    h->f_nnz = count;
  }
  return NS3D_OK;
}

int ns3d_forcing_modes(const ns3d_solver* h) {
  if (!h) return 0;
  return h->f_dense[0] ? -1 : h->f_nnz;
}

ns3d_status ns3d_rk3_step(ns3d_solver* h, ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                          double dt, double Re) {
  return ns3d_rk3_steps(h, ux, uy, uz, dt, Re, 1);
}

extern "C++" {
namespace ns3d_detail {
// nsteps RK3 steps, through a captured graph where the stream allows it.  A
// batch reads its per-instance dt and Re from h->dtRe (dt, Re here are 0).
ns3d_status rk3_steps_impl(ns3d_solver* h, ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                           double dt, double Re, int nsteps) {
  double2* u[3] = {(double2*)ux, (double2*)uy, (double2*)uz};
  if (nsteps == 0) return NS3D_OK;
  // The legacy default stream cannot be captured: launch directly there.
  if (h->stream == nullptr) {
    for (int s = 0; s < nsteps; ++s) NS3D_TRY(rk3_launches(h, u, dt, Re));
    return NS3D_OK;
  }
  const bool hit = h->rk3_exec && h->rk3_key[0] == ux && h->rk3_key[1] == uy &&
                   h->rk3_key[2] == uz && h->rk3_dt == dt && h->rk3_Re == Re &&
                   h->rk3_stream == h->stream && h->rk3_fversion == h->f_version;
  if (!hit && !h->graphs_off) {
    if (h->rk3_exec) cudaGraphExecDestroy(h->rk3_exec);
    h->rk3_exec = nullptr;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      ns3d_status s = rk3_launches(h, u, dt, Re);
      e = cudaStreamEndCapture(h->stream, &graph);
      if (s != NS3D_OK) {
        if (graph) cudaGraphDestroy(graph);
        return s;
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&h->rk3_exec, graph, 0);
      if (graph) cudaGraphDestroy(graph);
    }
    if (e != cudaSuccess) {
      // capture not possible on this stream: launch directly from now on
      cudaGetLastError();
      h->rk3_exec = nullptr;
      h->graphs_off = true;
    } else {
      h->rk3_key[0] = ux; h->rk3_key[1] = uy; h->rk3_key[2] = uz;
      h->rk3_dt = dt; h->rk3_Re = Re; h->rk3_stream = h->stream;
      h->rk3_fversion = h->f_version;
    }
  }
  if (h->graphs_off) {
    for (int s = 0; s < nsteps; ++s) NS3D_TRY(rk3_launches(h, u, dt, Re));
    return NS3D_OK;
  }
  for (int s = 0; s < nsteps; ++s)
    NS3D_CHECK(h, cudaGraphLaunch(h->rk3_exec, h->stream), "graph launch");
  return NS3D_OK;
}
}  // namespace ns3d_detail
}  // extern "C++"

ns3d_status ns3d_rk3_steps(ns3d_solver* h, ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                           double dt, double Re, int nsteps) {
  NS3D_TRY(check_handle(h));
  NS3D_TRY(check_step(h, dt, Re));
  if (!args_ok3(ux, uy, uz) || nsteps < 0) return fail(h, NS3D_ERR_BAD_ARG, "null field");
  return rk3_steps_impl(h, ux, uy, uz, dt, Re, nsteps);
}

ns3d_status ns3d_euler_step(ns3d_solver* h, ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                            double dt, double Re) {
  NS3D_TRY(check_handle(h));
  NS3D_TRY(check_step(h, dt, Re));
  if (!args_ok3(ux, uy, uz)) return fail(h, NS3D_ERR_BAD_ARG, "null field");
  double2* u[3] = {(double2*)ux, (double2*)uy, (double2*)uz};
  const double2* uc[3] = {u[0], u[1], u[2]};
  NS3D_TRY(conv_front(h, uc, nullptr));
  return finish(h, ns3d::kExplicit, true, uc, u, nullptr, 0.0, 1.0, dt, Re);
}

ns3d_status ns3d_rhs(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                     const ns3d_complex* uz, ns3d_complex* rx, ns3d_complex* ry, ns3d_complex* rz,
                     double Re) {
  NS3D_TRY(check_handle(h));
  NS3D_TRY(check_step(h, 0.0, Re));
  if (!args_ok3(ux, uy, uz) || !args_ok3(rx, ry, rz))
    return fail(h, NS3D_ERR_BAD_ARG, "null field");
  const double2* uc[3] = {(const double2*)ux, (const double2*)uy, (const double2*)uz};
  double2* r[3] = {(double2*)rx, (double2*)ry, (double2*)rz};
  NS3D_TRY(conv_front(h, uc, nullptr));
  return finish(h, ns3d::kRhs, true, uc, r, nullptr, 0.0, 1.0, 0.0, Re);
}

ns3d_status ns3d_fft_r2c(ns3d_solver* h, const double* in, ns3d_complex* out) {
  NS3D_TRY(check_handle(h));
  if (!in || !out) return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  const PassGeom& g = h->geom;
  ns3d::ZPlainArgs z{};
  z.rin = in;
  z.cout = (double2*)out;
  z.tw = h->tw[2];
  NS3D_CHECK(h, ns3d::run_z_r2c(z, g, h->stream), "z_r2c");
  ns3d::LineArgs l{};
  l.in = (const double2*)out;
  l.out = (double2*)out;
  l.tw = h->tw[1];
  NS3D_CHECK(h, ns3d::run_line(1, -1, l, g, h->stream), "line_y");
  l.tw = h->tw[0];
  NS3D_CHECK(h, ns3d::run_line(0, -1, l, g, h->stream), "line_x");
  return NS3D_OK;
}

extern "C++" {
namespace ns3d_detail {
ns3d_status fft_c2r(ns3d_solver* h, const ns3d_complex* in, double* out, double scale) {
  NS3D_TRY(check_handle(h));
  if (!in || !out) return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  const PassGeom& g = h->geom;
  ns3d::LineArgs l{};
  l.in = (const double2*)in;
  l.out = h->A[0];
  l.tw = h->tw[0];
  NS3D_CHECK(h, ns3d::run_line(0, +1, l, g, h->stream), "line_x");
  l.in = h->A[0];
  l.tw = h->tw[1];
  NS3D_CHECK(h, ns3d::run_line(1, +1, l, g, h->stream), "line_y");
  ns3d::ZPlainArgs z{};
  z.cin = h->A[0];
  z.rout = out;
  z.scale = scale;
  z.tw = h->tw[2];
  NS3D_CHECK(h, ns3d::run_z_c2r(z, g, h->stream), "z_c2r");
  return NS3D_OK;
}
}  // namespace ns3d_detail
}  // extern "C++"

ns3d_status ns3d_fft_c2r(ns3d_solver* h, const ns3d_complex* in, double* out) {
  return h ? fft_c2r(h, in, out, h->geom.inv_vol) : NS3D_ERR_BAD_ARG;
}

ns3d_status ns3d_fft_c2r_unscaled(ns3d_solver* h, const ns3d_complex* in, double* out) {
  return fft_c2r(h, in, out, 1.0);
}

// Checkpoints of device fields through host buffers (the wire format is
// written and parsed by the host functions of checkpoint.cpp).
ns3d_status ns3d_save_control_fourier(ns3d_solver* h, const char* path, const ns3d_complex* ux,
                                      const ns3d_complex* uy, const ns3d_complex* uz) {
  NS3D_TRY(check_handle(h));
  if (!path || !args_ok3(ux, uy, uz)) return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  std::vector<ns3d_complex> b[3];
  const ns3d_complex* d[3] = {ux, uy, uz};
  for (int c = 0; c < 3; ++c) {
    b[c].resize(h->nc);
    NS3D_CHECK(h, cudaMemcpyAsync(b[c].data(), d[c], sizeof(ns3d_complex) * h->nc,
                                  cudaMemcpyDeviceToHost, h->stream), "checkpoint copy");
  }
  NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "checkpoint sync");
  const ns3d_status s = ns3d_write_control_fourier_host(path, h->Nx, h->Ny, h->Nz, b[0].data(),
                                                        b[1].data(), b[2].data());
  return s == NS3D_OK ? s : fail(h, s, std::string("cannot write ") + path);
}

ns3d_status ns3d_load_control_fourier(ns3d_solver* h, const char* path, ns3d_complex* ux,
                                      ns3d_complex* uy, ns3d_complex* uz) {
  NS3D_TRY(check_handle(h));
  if (!path || !args_ok3(ux, uy, uz)) return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  std::vector<ns3d_complex> b[3];
  for (int c = 0; c < 3; ++c) b[c].resize(h->nc);
  const ns3d_status s = ns3d_read_control_fourier_host(path, h->Nx, h->Ny, h->Nz, b[0].data(),
                                                       b[1].data(), b[2].data(), nullptr,
                                                       nullptr, nullptr);
  if (s != NS3D_OK) return fail(h, s, std::string("cannot read a matching state from ") + path);
  ns3d_complex* d[3] = {ux, uy, uz};
  for (int c = 0; c < 3; ++c)
    NS3D_CHECK(h, cudaMemcpyAsync(d[c], b[c].data(), sizeof(ns3d_complex) * h->nc,
                                  cudaMemcpyHostToDevice, h->stream), "checkpoint copy");
  NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "checkpoint sync");
  return NS3D_OK;
}

ns3d_status ns3d_save_control_file(ns3d_solver* h, const char* path, const ns3d_complex* ux,
                                   const ns3d_complex* uy, const ns3d_complex* uz) {
  NS3D_TRY(check_handle(h));
  if (!path || !args_ok3(ux, uy, uz)) return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  const size_t nr = (size_t)h->Nx * h->Ny * h->Nz;
  std::vector<double> b[3];
  const ns3d_complex* d[3] = {ux, uy, uz};
  double* phys = reinterpret_cast<double*>(h->B[0]);  // S_c bytes >= S_r bytes
  for (int c = 0; c < 3; ++c) {
    b[c].resize(nr);
    NS3D_TRY(ns3d_fft_c2r(h, d[c], phys));
    NS3D_CHECK(h, cudaMemcpyAsync(b[c].data(), phys, sizeof(double) * nr, cudaMemcpyDeviceToHost,
                                  h->stream), "checkpoint copy");
  }
  NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "checkpoint sync");
  const ns3d_status s = ns3d_write_control_file_host(path, h->Nx, h->Ny, h->Nz, b[0].data(),
                                                     b[1].data(), b[2].data());
  return s == NS3D_OK ? s : fail(h, s, std::string("cannot write ") + path);
}

ns3d_status ns3d_load_control_file(ns3d_solver* h, const char* path, ns3d_complex* ux,
                                   ns3d_complex* uy, ns3d_complex* uz) {
  NS3D_TRY(check_handle(h));
  if (!path || !args_ok3(ux, uy, uz)) return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  const size_t nr = (size_t)h->Nx * h->Ny * h->Nz;
  std::vector<double> b[3];
  for (int c = 0; c < 3; ++c) b[c].resize(nr);
  const ns3d_status s = ns3d_read_control_file_host(path, h->Nx, h->Ny, h->Nz, b[0].data(),
                                                    b[1].data(), b[2].data());
  if (s != NS3D_OK) return fail(h, s, std::string("cannot read a matching field from ") + path);
  ns3d_complex* d[3] = {ux, uy, uz};
  double* phys = reinterpret_cast<double*>(h->B[0]);
  for (int c = 0; c < 3; ++c) {
    NS3D_CHECK(h, cudaMemcpyAsync(phys, b[c].data(), sizeof(double) * nr, cudaMemcpyHostToDevice,
                                  h->stream), "checkpoint copy");
    NS3D_TRY(ns3d_fft_r2c(h, phys, d[c]));
  }
  NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "checkpoint sync");
  return NS3D_OK;
}

ns3d_status ns3d_convolution(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                             const ns3d_complex* uz, ns3d_complex* Qx, ns3d_complex* Qy,
                             ns3d_complex* Qz) {
  NS3D_TRY(check_handle(h));
  if (!args_ok3(ux, uy, uz) || !args_ok3(Qx, Qy, Qz))
    return fail(h, NS3D_ERR_BAD_ARG, "null field");
  const double2* uc[3] = {(const double2*)ux, (const double2*)uy, (const double2*)uz};
  double2* q[3] = {(double2*)Qx, (double2*)Qy, (double2*)Qz};
  NS3D_TRY(conv_front(h, uc, nullptr));
  return finish(h, ns3d::kConvOut, false, nullptr, q, nullptr, 0.0, 1.0, 0.0, 1.0);
}

ns3d_status ns3d_convolution_uv(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                                const ns3d_complex* uz, const ns3d_complex* vx,
                                const ns3d_complex* vy, const ns3d_complex* vz, ns3d_complex* Qx,
                                ns3d_complex* Qy, ns3d_complex* Qz) {
  NS3D_TRY(check_handle(h));
  if (!args_ok3(ux, uy, uz) || !args_ok3(vx, vy, vz) || !args_ok3(Qx, Qy, Qz))
    return fail(h, NS3D_ERR_BAD_ARG, "null field");
  const double2* uc[3] = {(const double2*)ux, (const double2*)uy, (const double2*)uz};
  const double2* vc[3] = {(const double2*)vx, (const double2*)vy, (const double2*)vz};
  double2* q[3] = {(double2*)Qx, (double2*)Qy, (double2*)Qz};
  NS3D_TRY(conv_front(h, uc, vc));
  return finish(h, ns3d::kConvOut, false, nullptr, q, nullptr, 0.0, 1.0, 0.0, 1.0);
}

// single_time_step_UV (Source/RK_time_step.cu:265-278): v <- v + dt J(u) v.
ns3d_status ns3d_tangent_euler_step(ns3d_solver* h, const ns3d_complex* ux,
                                    const ns3d_complex* uy, const ns3d_complex* uz,
                                    ns3d_complex* vx, ns3d_complex* vy, ns3d_complex* vz,
                                    double dt, double Re) {
  NS3D_TRY(check_handle(h));
  NS3D_TRY(check_step(h, dt, Re));
  if (!args_ok3(ux, uy, uz) || !args_ok3(vx, vy, vz))
    return fail(h, NS3D_ERR_BAD_ARG, "null field");
  const double2* uc[3] = {(const double2*)ux, (const double2*)uy, (const double2*)uz};
  double2* v[3] = {(double2*)vx, (double2*)vy, (double2*)vz};
  const double2* vc[3] = {v[0], v[1], v[2]};
  NS3D_TRY(conv_front(h, uc, vc));
  return finish(h, ns3d::kExplicit, false, vc, v, nullptr, 0.0, 1.0, dt, Re);
}

ns3d_status ns3d_jvp_step(ns3d_solver* h, ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                          ns3d_complex* vx, ns3d_complex* vy, ns3d_complex* vz, double dt,
                          double Re) {
  return ns3d_jvp_steps(h, ux, uy, uz, vx, vy, vz, dt, Re, 1);
}

// RK3_SSP_UV (Source/RK_time_step.cu:342-355):
//   v1 = v + dt J(u) v; u <- RK3(u); v = 1/2 v + 1/2 (v1 + dt J(u_new) v1)
ns3d_status ns3d_jvp_steps(ns3d_solver* h, ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                           ns3d_complex* vx, ns3d_complex* vy, ns3d_complex* vz, double dt,
                           double Re, int nsteps) {
  NS3D_TRY(check_handle(h));
  NS3D_TRY(check_step(h, dt, Re));
  if (!args_ok3(ux, uy, uz) || !args_ok3(vx, vy, vz) || nsteps < 0)
    return fail(h, NS3D_ERR_BAD_ARG, "null field");
  NS3D_TRY(ensure_uv_pool(h));
  double2* u[3] = {(double2*)ux, (double2*)uy, (double2*)uz};
  double2* v[3] = {(double2*)vx, (double2*)vy, (double2*)vz};
  const double2* uc[3] = {u[0], u[1], u[2]};
  const double2* vc[3] = {v[0], v[1], v[2]};
  const double2* v1c[3] = {h->v1[0], h->v1[1], h->v1[2]};
  // the 25 launches of one step
  auto one = [&]() -> ns3d_status {
    NS3D_TRY(conv_front(h, uc, vc));
    NS3D_TRY(finish(h, ns3d::kExplicit, false, vc, h->v1, nullptr, 0.0, 1.0, dt, Re));
    NS3D_TRY(rk3_launches(h, u, dt, Re));
    NS3D_TRY(conv_front(h, uc, v1c));
    return finish(h, ns3d::kExplicit, false, v1c, v, vc, 0.5, 0.5, dt, Re);
  };
  if (nsteps == 0) return NS3D_OK;
  // As for the RK3 steps: replay a captured step where the stream allows it
  // (the legacy default stream cannot be captured).
  if (h->stream != nullptr && !h->graphs_off) {
    const void* key[6] = {ux, uy, uz, vx, vy, vz};
    bool hit = h->jvp_exec && h->jvp_dt == dt && h->jvp_Re == Re &&
               h->jvp_stream == h->stream && h->jvp_fversion == h->f_version;
    for (int i = 0; i < 6 && hit; ++i) hit = h->jvp_key[i] == key[i];
    if (!hit) {
      if (h->jvp_exec) cudaGraphExecDestroy(h->jvp_exec);
      h->jvp_exec = nullptr;
      cudaGraph_t graph = nullptr;
      cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        ns3d_status s = one();
        e = cudaStreamEndCapture(h->stream, &graph);
        if (s != NS3D_OK) {
          if (graph) cudaGraphDestroy(graph);
          return s;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&h->jvp_exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
      }
      if (e != cudaSuccess) {
        cudaGetLastError();
        h->jvp_exec = nullptr;
        h->graphs_off = true;
      } else {
        for (int i = 0; i < 6; ++i) h->jvp_key[i] = key[i];
        h->jvp_dt = dt; h->jvp_Re = Re; h->jvp_stream = h->stream;
        h->jvp_fversion = h->f_version;
      }
    }
    if (!h->graphs_off) {
      for (int s = 0; s < nsteps; ++s)
        NS3D_CHECK(h, cudaGraphLaunch(h->jvp_exec, h->stream), "graph launch");
      return NS3D_OK;
    }
  }
  for (int s = 0; s < nsteps; ++s) NS3D_TRY(one());
  return NS3D_OK;
}

ns3d_status ns3d_linearised_rhs(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                                const ns3d_complex* uz, ns3d_complex* vx, ns3d_complex* vy,
                                ns3d_complex* vz, double Re) {
  NS3D_TRY(check_handle(h));
  NS3D_TRY(check_step(h, 0.0, Re));
  if (!args_ok3(ux, uy, uz) || !args_ok3(vx, vy, vz))
    return fail(h, NS3D_ERR_BAD_ARG, "null field");
  const double2* uc[3] = {(const double2*)ux, (const double2*)uy, (const double2*)uz};
  double2* v[3] = {(double2*)vx, (double2*)vy, (double2*)vz};
  const double2* vc[3] = {v[0], v[1], v[2]};
  NS3D_TRY(conv_front(h, uc, vc));
  return finish(h, ns3d::kRhs, false, vc, v, nullptr, 0.0, 1.0, 0.0, Re);
}

ns3d_status ns3d_implicit_tangent_step(ns3d_solver* h, const ns3d_complex* ux,
                                       const ns3d_complex* uy, const ns3d_complex* uz,
                                       ns3d_complex* vx, ns3d_complex* vy, ns3d_complex* vz,
                                       double dt, double Re) {
  NS3D_TRY(check_handle(h));
  NS3D_TRY(check_step(h, dt, Re));
  if (!args_ok3(ux, uy, uz) || !args_ok3(vx, vy, vz))
    return fail(h, NS3D_ERR_BAD_ARG, "null field");
  const double2* uc[3] = {(const double2*)ux, (const double2*)uy, (const double2*)uz};
  double2* v[3] = {(double2*)vx, (double2*)vy, (double2*)vz};
  const double2* vc[3] = {v[0], v[1], v[2]};
  NS3D_TRY(conv_front(h, uc, vc));
  return finish(h, ns3d::kImplicit, false, vc, v, nullptr, 0.0, 1.0, dt, Re);
}

int64_t ns3d_krylov_length(const ns3d_solver* h) { return h ? 3 * ((int64_t)h->nc - 1) : 0; }

ns3d_status ns3d_pack_reduced(ns3d_solver* h, const ns3d_complex* vx, const ns3d_complex* vy,
                              const ns3d_complex* vz, double* vec) {
  NS3D_TRY(check_handle(h));
  if (!args_ok3(vx, vy, vz) || !vec) return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  ns3d::pack_reduced_kernel<<<592, 256, 0, h->stream>>>(
      (const double2*)vx, (const double2*)vy, (const double2*)vz, (long long)h->nc, vec, nullptr,
      0.0, nullptr, 0.0);
  NS3D_CHECK(h, cudaGetLastError(), "pack_reduced");
  return NS3D_OK;
}

ns3d_status ns3d_pack_reduced_shifted(ns3d_solver* h, const ns3d_complex* vx,
                                      const ns3d_complex* vy, const ns3d_complex* vz,
                                      const double* vec_a, double a, const double* vec_b,
                                      double b, double* vec) {
  NS3D_TRY(check_handle(h));
  if (!args_ok3(vx, vy, vz) || !vec || !vec_a) return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  ns3d::pack_reduced_kernel<<<592, 256, 0, h->stream>>>(
      (const double2*)vx, (const double2*)vy, (const double2*)vz, (long long)h->nc, vec, vec_a, a,
      vec_b, b);
  NS3D_CHECK(h, cudaGetLastError(), "pack_reduced_shifted");
  return NS3D_OK;
}

ns3d_status ns3d_unpack_reduced(ns3d_solver* h, const double* vec, ns3d_complex* vx,
                                ns3d_complex* vy, ns3d_complex* vz) {
  NS3D_TRY(check_handle(h));
  if (!args_ok3(vx, vy, vz) || !vec) return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  ns3d::unpack_reduced_kernel<<<592, 256, 0, h->stream>>>(vec, (long long)h->nc, (double2*)vx,
                                                          (double2*)vy, (double2*)vz);
  NS3D_CHECK(h, cudaGetLastError(), "unpack_reduced");
  return NS3D_OK;
}

ns3d_status ns3d_matvec_reduced(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                                const ns3d_complex* uz, const double* vec_in, double* vec_out,
                                double Re, double tau) {
  NS3D_TRY(check_handle(h));
  NS3D_TRY(check_step(h, 0.0, Re));
  if (!args_ok3(ux, uy, uz) || !vec_in || !vec_out)
    return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  NS3D_TRY(ensure_uv_pool(h));
  double2* v[3] = {h->v1[0], h->v1[1], h->v1[2]};
  const double2* vc[3] = {v[0], v[1], v[2]};
  const double2* uc[3] = {(const double2*)ux, (const double2*)uy, (const double2*)uz};
  ns3d::unpack_reduced_kernel<<<592, 256, 0, h->stream>>>(vec_in, (long long)h->nc, v[0], v[1],
                                                          v[2]);
  NS3D_CHECK(h, cudaGetLastError(), "unpack_reduced");
  NS3D_TRY(conv_front(h, uc, vc));
  NS3D_TRY(finish(h, ns3d::kRhs, false, vc, v, nullptr, 0.0, 1.0, 0.0, Re));
  ns3d::pack_reduced_kernel<<<592, 256, 0, h->stream>>>(v[0], v[1], v[2], (long long)h->nc,
                                                        vec_out, tau > 0.0 ? vec_in : nullptr,
                                                        tau > 0.0 ? 1.0 / tau : 0.0, nullptr,
                                                        0.0);
  NS3D_CHECK(h, cudaGetLastError(), "pack_reduced");
  return NS3D_OK;
}

ns3d_status ns3d_diagnostics(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                             const ns3d_complex* uz, double* energy, double* dissipation,
                             double* div_max) {
  NS3D_TRY(check_handle(h));
  if (!args_ok3(ux, uy, uz)) return fail(h, NS3D_ERR_BAD_ARG, "null field");
  ns3d::DiagGeom g{};
  g.Nx = h->Nx; g.Ny = h->Ny; g.Nz = h->Nz; g.Mz = h->Mz;
  g.kfx = h->geom.kfx; g.kfy = h->geom.kfy; g.kfz = h->geom.kfz;
  g.dx = h->Lx / (double)h->Nx;
  g.dy = h->Ly / (double)h->Ny;
  g.dz = h->Lz / (double)h->Nz;
  g.inv_vol = h->geom.inv_vol;
  ns3d::diag_partial_kernel<<<kDiagBlocks, kDiagThreads, 0, h->stream>>>(
      (const double2*)ux, (const double2*)uy, (const double2*)uz, g, h->diag_partial);
  NS3D_CHECK(h, cudaGetLastError(), "diag_partial");
  ns3d::diag_final_kernel<<<1, 1024, 0, h->stream>>>(h->diag_partial, kDiagBlocks, h->diag_out);
  NS3D_CHECK(h, cudaGetLastError(), "diag_final");
  double r[3];
  NS3D_CHECK(h, cudaMemcpyAsync(r, h->diag_out, sizeof(r), cudaMemcpyDeviceToHost, h->stream),
             "diag copy");
  NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "diag sync");
  if (energy) *energy = r[0];
  if (dissipation) *dissipation = r[1];
  if (div_max) *div_max = r[2];
  if (!std::isfinite(r[0]) || !std::isfinite(r[1]) || !std::isfinite(r[2]))
    return fail(h, NS3D_ERR_NONFINITE, "diagnostics are not finite");
  return NS3D_OK;
}

// ---------------------------------------------------------------------------
// Filters, curl, the per-step record, the energy spectrum, Shapiro's solution
// ---------------------------------------------------------------------------

extern "C++" {
namespace ns3d_detail {

ns3d::GridGeom grid_geom(const ns3d_solver* h) {
  ns3d::GridGeom g{};
  g.Nx = h->Nx; g.Ny = h->Ny; g.Nz = h->Nz;
  g.dx = h->Lx / (double)h->Nx;
  g.dy = h->Ly / (double)h->Ny;
  g.dz = h->Lz / (double)h->Nz;
  return g;
}

int elementwise_blocks(long long n) {
  const long long b = (n + kDiagThreads - 1) / kDiagThreads;
  return (int)(b < 8 * kDiagBlocks ? (b > 0 ? b : 1) : 8 * kDiagBlocks);
}

// The probe points and spectral reads of the main loop's record
// (Source/NS3D_periodic.cu:1357-1450, IN of Source/Macros.h:11 with the
// physical Nz, then with Nz = Mz), and the phase tables of
// record_partial_kernel.  Allocated on first use.
ns3d_status ensure_record(ns3d_solver* h) {
  if (h->rec_tab) return NS3D_OK;
  const long long Nx = h->Nx, Ny = h->Ny, Nz = h->Nz, Mz = h->Mz;
  auto in_r = [&](long long i, long long j, long long k) { return i * (Ny * Nz) + j * Nz + k; };
  auto in_c = [&](long long i, long long j, long long k) { return i * (Ny * Mz) + j * Mz + k; };
  const long long P[3] = {in_r(Nx / 2 - 4, Ny / 2 - 3, Nz / 2 - 2), in_r(Nx / 3, Ny / 3, Nz / 3),
                          in_r(Nx / 8, Ny / 8, Nz / 8)};
  const long long F[11] = {in_c(Nx - 6, Ny - 6, Mz - 6), in_c(Nx / 5, Ny / 4 - 3, Mz / 4 - 1),
                           in_c(Nx / 5, Ny / 5, Mz / 5),  in_c(2, 2, 2),
                           in_c(1, 0, 0),                 in_c(0, 0, 0),
                           in_c(1, 1, 0),                 in_c(1, 1, 1),
                           in_c(Nx - 1, 0, 0),            in_c(Nx - 1, Ny - 1, 0),
                           in_c(Nx - 1, Ny - 1, Mz - 1)};
  for (long long p : P)
    if (p < 0 || p >= Nx * Ny * Nz)
      return fail(h, NS3D_ERR_BAD_ARG, "grid too small for the record's probe points");
  for (long long f : F)
    if (f < 0 || f >= (long long)h->nc)
      return fail(h, NS3D_ERR_BAD_ARG, "grid too small for the record's spectral reads");
  const int nx = h->Nx, ny = h->Ny, mz = h->Mz;
  std::vector<double2> tab((size_t)ns3d::record_table_size(nx, ny, mz));
  auto phase = [](long long r, long long n) {
    const double a = 2.0 * M_PI * (double)r / (double)n;
    return make_double2(std::cos(a), std::sin(a));
  };
  size_t o = 0;
  const long long ext[3] = {Nx, Ny, Mz};
  for (int axis = 0; axis < 3; ++axis)
    for (int s = 0; s < 3; ++s) {
      const long long p = P[s];
      const long long c[3] = {p / (Ny * Nz), (p / Nz) % Ny, p % Nz};
      const long long n = axis == 0 ? Nx : axis == 1 ? Ny : Nz;
      for (long long j = 0; j < ext[axis]; ++j) tab[o++] = phase((j * c[axis]) % n, n);
    }
  for (long long j = 0; j < Nx; ++j) tab[o++] = phase(j, Nx);
  const double h3[3] = {h->Lx / Nx, h->Ly / Ny, h->Lz / Nz};
  for (int axis = 0; axis < 3; ++axis) {
    const long long n = axis == 0 ? Nx : axis == 1 ? Ny : Nz;
    for (long long j = 0; j < ext[axis]; ++j)
      tab[o++] = make_double2(std::sin(2.0 * M_PI * (double)j / (double)n) / h3[axis], 0.0);
  }
  for (int i = 0; i < 11; ++i) h->rec_reads.f[i] = F[i];
  for (int i = 0; i < 3; ++i) h->rec_points[i] = P[i];
  double2* t = nullptr;
  double* part = nullptr;
  double* out = nullptr;
  cudaError_t e = cudaMalloc(&t, sizeof(double2) * tab.size());
  if (e == cudaSuccess) e = cudaMalloc(&part, sizeof(double) * ns3d::kRecordSums * kDiagBlocks);
  if (e == cudaSuccess) e = cudaMalloc(&out, sizeof(double) * 64);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(t, tab.data(), sizeof(double2) * tab.size(), cudaMemcpyHostToDevice,
                        h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    cudaFree(t);
    cudaFree(part);
    cudaFree(out);
    return cuda_fail(h, e, "record buffers");
  }
  h->rec_tab = t;
  h->rec_partial = part;
  h->rec_out = out;
  return NS3D_OK;
}

ns3d_status spectral_filter(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                            const ns3d_complex* uz, int mode, double p, ns3d_complex* fx,
                            ns3d_complex* fy, ns3d_complex* fz) {
  NS3D_TRY(check_handle(h));
  if (!args_ok3(ux, uy, uz) || !args_ok3(fx, fy, fz)) return fail(h, NS3D_ERR_BAD_ARG, "null field");
  if (!std::isfinite(p)) return fail(h, NS3D_ERR_BAD_ARG, "filter parameter not finite");
  ns3d::FilterGeom g{h->Nx, h->Ny, h->Mz, h->Lx, h->Ly, h->Lz};
  ns3d::spectral_filter_kernel<<<elementwise_blocks((long long)h->nc), kDiagThreads, 0,
                                 h->stream>>>((const double2*)ux, (const double2*)uy,
                                              (const double2*)uz, (double2*)fx, (double2*)fy,
                                              (double2*)fz, g, mode, p);
  NS3D_CHECK(h, cudaGetLastError(), "spectral_filter");
  return NS3D_OK;
}

ns3d_status diag_sums(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                      const ns3d_complex* uz) {
  ns3d::DiagGeom g{};
  g.Nx = h->Nx; g.Ny = h->Ny; g.Nz = h->Nz; g.Mz = h->Mz;
  g.kfx = h->geom.kfx; g.kfy = h->geom.kfy; g.kfz = h->geom.kfz;
  g.dx = h->Lx / (double)h->Nx;
  g.dy = h->Ly / (double)h->Ny;
  g.dz = h->Lz / (double)h->Nz;
  g.inv_vol = h->geom.inv_vol;
  ns3d::diag_partial_kernel<<<kDiagBlocks, kDiagThreads, 0, h->stream>>>(
      (const double2*)ux, (const double2*)uy, (const double2*)uz, g, h->diag_partial);
  NS3D_CHECK(h, cudaGetLastError(), "diag_partial");
  ns3d::diag_final_kernel<<<1, 1024, 0, h->stream>>>(h->diag_partial, kDiagBlocks, h->diag_out);
  NS3D_CHECK(h, cudaGetLastError(), "diag_final");
  return NS3D_OK;
}

ns3d_status shapiro_minmax(ns3d_solver* h, const double* ux, const double* uy, const double* uz,
                           double t, double Re, double* mm) {
  NS3D_TRY(ensure_record(h));
  const double f = std::sqrt(3.0);
  const double decay = std::exp(-(f * f) * t / Re);
  ns3d::shapiro_error_kernel<<<kDiagBlocks, kDiagThreads, 0, h->stream>>>(
      ux, uy, uz, grid_geom(h), decay, h->rec_partial);
  NS3D_CHECK(h, cudaGetLastError(), "shapiro_error");
  ns3d::minmax_final_kernel<<<1, 1024, 0, h->stream>>>(h->rec_partial, kDiagBlocks,
                                                       h->rec_out + 50);
  NS3D_CHECK(h, cudaGetLastError(), "minmax_final");
  NS3D_CHECK(h, cudaMemcpyAsync(mm, h->rec_out + 50, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                h->stream), "shapiro copy");
  NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "shapiro sync");
  return NS3D_OK;
}

}  // namespace ns3d_detail
}  // extern "C++"

ns3d_status ns3d_helmholtz_filter(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                                  const ns3d_complex* uz, double eps, ns3d_complex* fx,
                                  ns3d_complex* fy, ns3d_complex* fz) {
  return spectral_filter(h, ux, uy, uz, 0, eps, fx, fy, fz);
}

ns3d_status ns3d_cutoff_filter(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                               const ns3d_complex* uz, double radius, ns3d_complex* fx,
                               ns3d_complex* fy, ns3d_complex* fz) {
  return spectral_filter(h, ux, uy, uz, 1, radius, fx, fy, fz);
}

ns3d_status ns3d_curl(ns3d_solver* h, const double* ux, const double* uy, const double* uz,
                      double* rx, double* ry, double* rz) {
  NS3D_TRY(check_handle(h));
  if (!ux || !uy || !uz || !rx || !ry || !rz) return fail(h, NS3D_ERR_BAD_ARG, "null field");
  const long long n = (long long)h->Nx * h->Ny * h->Nz;
  ns3d::curl_kernel<<<elementwise_blocks(n), kDiagThreads, 0, h->stream>>>(ux, uy, uz, rx, ry, rz,
                                                                           grid_geom(h));
  NS3D_CHECK(h, cudaGetLastError(), "curl");
  return NS3D_OK;
}

ns3d_status ns3d_record(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                        const ns3d_complex* uz, double total_time, double Re, double* rec) {
  NS3D_TRY(check_handle(h));
  if (!args_ok3(ux, uy, uz) || !rec) return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  if (!(Re > 0.0) || !std::isfinite(Re)) return fail(h, NS3D_ERR_BAD_ARG, "Re must be > 0");
  NS3D_TRY(ensure_record(h));
  NS3D_TRY(diag_sums(h, ux, uy, uz));
  ns3d::RecordGeom g{};
  g.Nx = h->Nx; g.Ny = h->Ny; g.Nz = h->Nz; g.Mz = h->Mz;
  g.dx = h->Lx / (double)h->Nx;
  g.dy = h->Ly / (double)h->Ny;
  g.dz = h->Lz / (double)h->Nz;
  g.cut2 = 0.1 * 0.1;  // CutOff_Fourier_Filter(..., 0.1, ...) of the main loop
  ns3d::record_partial_kernel<<<kDiagBlocks, kDiagThreads, 0, h->stream>>>(
      (const double2*)ux, (const double2*)uy, (const double2*)uz, g, h->rec_tab, h->rec_partial);
  NS3D_CHECK(h, cudaGetLastError(), "record_partial");
  ns3d::record_final_kernel<<<1, 32 * ns3d::kRecordSums, 0, h->stream>>>(
      h->rec_partial, kDiagBlocks, h->diag_out, (const double2*)ux, (const double2*)uy,
      (const double2*)uz, h->rec_reads, total_time, Re, h->geom.inv_vol, h->rec_out);
  NS3D_CHECK(h, cudaGetLastError(), "record_final");
  NS3D_CHECK(h, cudaMemcpyAsync(rec, h->rec_out, sizeof(double) * NS3D_RECORD_COLUMNS,
                                cudaMemcpyDeviceToHost, h->stream), "record copy");
  NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "record sync");
  for (int i = 0; i < NS3D_RECORD_COLUMNS; ++i)
    if (!std::isfinite(rec[i])) return fail(h, NS3D_ERR_NONFINITE, "record is not finite");
  return NS3D_OK;
}

ns3d_status ns3d_energy_spectrum(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                                 const ns3d_complex* uz, double* E, int nbins) {
  NS3D_TRY(check_handle(h));
  if (!args_ok3(ux, uy, uz) || !E) return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  const int size = h->Nx / 2 + h->Ny / 2 + h->Mz;
  if (nbins != size) return fail(h, NS3D_ERR_BAD_ARG, "nbins must be Nx/2 + Ny/2 + Nz/2 + 1");
  double* d = reinterpret_cast<double*>(h->B[0]);  // nc complex >= size doubles
  const double norm = (double)h->Nx * (double)h->Ny * (double)h->Mz;
  ns3d::spectrum_kernel<<<size, kDiagThreads, 0, h->stream>>>(
      (const double2*)ux, (const double2*)uy, (const double2*)uz, h->Nx, h->Ny, h->Mz, norm, d);
  NS3D_CHECK(h, cudaGetLastError(), "spectrum");
  NS3D_CHECK(h, cudaMemcpyAsync(E, d, sizeof(double) * size, cudaMemcpyDeviceToHost, h->stream),
             "spectrum copy");
  NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "spectrum sync");
  return NS3D_OK;
}

ns3d_status ns3d_shapiro_state(ns3d_solver* h, double t, double Re, ns3d_complex* ux,
                               ns3d_complex* uy, ns3d_complex* uz) {
  NS3D_TRY(check_handle(h));
  if (!args_ok3(ux, uy, uz)) return fail(h, NS3D_ERR_BAD_ARG, "null field");
  if (!(Re > 0.0) || !std::isfinite(t)) return fail(h, NS3D_ERR_BAD_ARG, "bad t or Re");
  const double f = std::sqrt(3.0);
  const double decay = std::exp(-(f * f) * t / Re);
  double* p[3];
  for (int c = 0; c < 3; ++c) p[c] = reinterpret_cast<double*>(h->B[c]);
  const long long n = (long long)h->Nx * h->Ny * h->Nz;
  ns3d::shapiro_field_kernel<<<elementwise_blocks(n), kDiagThreads, 0, h->stream>>>(
      p[0], p[1], p[2], grid_geom(h), decay);
  NS3D_CHECK(h, cudaGetLastError(), "shapiro_field");
  ns3d_complex* out[3] = {ux, uy, uz};
  for (int c = 0; c < 3; ++c) NS3D_TRY(ns3d_fft_r2c(h, p[c], out[c]));
  return NS3D_OK;
}

ns3d_status ns3d_shapiro_error_physical(ns3d_solver* h, const double* ux, const double* uy,
                                        const double* uz, double t, double Re, double* min_max) {
  NS3D_TRY(check_handle(h));
  if (!ux || !uy || !uz || !min_max) return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  if (!(Re > 0.0) || !std::isfinite(t)) return fail(h, NS3D_ERR_BAD_ARG, "bad t or Re");
  return shapiro_minmax(h, ux, uy, uz, t, Re, min_max);
}

ns3d_status ns3d_shapiro_error(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                               const ns3d_complex* uz, double t, double Re, double* err) {
  NS3D_TRY(check_handle(h));
  if (!args_ok3(ux, uy, uz) || !err) return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  if (!(Re > 0.0) || !std::isfinite(t)) return fail(h, NS3D_ERR_BAD_ARG, "bad t or Re");
  double* p[3];
  for (int c = 0; c < 3; ++c) p[c] = reinterpret_cast<double*>(h->B[c]);
  const ns3d_complex* u[3] = {ux, uy, uz};
  for (int c = 0; c < 3; ++c) NS3D_TRY(ns3d_fft_c2r(h, u[c], p[c]));
  double mm[2];
  NS3D_TRY(shapiro_minmax(h, p[0], p[1], p[2], t, Re, mm));
  *err = mm[1];
  return NS3D_OK;
}

extern "C++" {
namespace ns3d_detail {
template <typename C>
ns3d_status profile_passes_t(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                             const ns3d_complex* uz, double dt, double Re, int reps,
                             double* ms) {
  auto sc = [](double2* p) { return reinterpret_cast<C*>(p); };
  const PassGeom& g = h->geom;
  cudaStream_t st = h->stream;
  const double2* u[3] = {(const double2*)ux, (const double2*)uy, (const double2*)uz};
  InvXArgs<3, C> ax{};
  InvYArgs<3, C> ay{};
  ZArgs<3, C> az{};
  FwdYArgs<C> fy{};
  FwdXArgs<C> fx{};
  for (int i = 0; i < 3; ++i) {
    ax.in[i] = u[i]; ax.A[i] = sc(h->A[i]); ax.B[i] = sc(h->B[i]);
    ay.A[i] = sc(h->A[i]); ay.B[i] = sc(h->B[i]);
    ay.C[i] = sc(h->C[i]); ay.D[i] = sc(h->D[i]); ay.E[i] = sc(h->E[i]);
    az.C[i] = sc(h->C[i]); az.D[i] = sc(h->D[i]); az.E[i] = sc(h->E[i]);
    az.Qh[i] = sc(h->A[i]);
    fy.Q[i] = sc(h->A[i]);
    fx.Qh[i] = sc(h->A[i]); fx.us[i] = u[i]; fx.out[i] = h->u1[i];
    fx.fd[i] = h->f_dense[0] ? h->f_dense[i] : nullptr;
  }
  ax.qcut = h->qcut; ax.tw = h->tw[0];
  ay.tw = h->tw[1]; az.tw = h->tw[2]; fy.tw = h->tw[1]; fx.tw = h->tw[0];
  if (sizeof(C) == 16 && g.tile[ns3d::kTileInvY] == 2) {  // as conv_front
    ay.maps = h->ymaps;
    ay.err = h->dev_err;
  }
  fx.fidx = h->f_idx; fx.fval = h->f_val; fx.fnnz = h->f_dense[0] ? 0 : h->f_nnz;
  fx.dt = dt; fx.Re = Re; fx.ca = 0.0; fx.cb = 1.0;
  cudaEvent_t ev[6];
  for (auto& e : ev) cudaEventCreate(&e);
  double acc[5] = {0, 0, 0, 0, 0};
  cudaError_t err = cudaSuccess;
  for (int r = 0; r <= reps && err == cudaSuccess; ++r) {
    cudaEventRecord(ev[0], st);
    if ((err = ns3d::run_inv_x(ax, g, st)) != cudaSuccess) break;
    cudaEventRecord(ev[1], st);
    if ((err = ns3d::run_inv_y(ay, g, st)) != cudaSuccess) break;
    cudaEventRecord(ev[2], st);
    if ((err = ns3d::run_z(az, g, st)) != cudaSuccess) break;
    cudaEventRecord(ev[3], st);
    if ((err = ns3d::run_fwd_y(fy, g, st)) != cudaSuccess) break;
    cudaEventRecord(ev[4], st);
    if ((err = ns3d::run_fwd_x(ns3d::kExplicit, false, fx, g, st)) != cudaSuccess) break;
    cudaEventRecord(ev[5], st);
    if ((err = cudaEventSynchronize(ev[5])) != cudaSuccess) break;
    if (r == 0) continue;  // warm-up
    for (int k = 0; k < 5; ++k) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
      acc[k] += t;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (err != cudaSuccess) return cuda_fail(h, err, "profile_passes");
  for (int k = 0; k < 5; ++k) ms[k] = acc[k] / reps;
  return NS3D_OK;
}
}  // namespace ns3d_detail
}  // extern "C++"

// ---------------------------------------------------------------------------
// Autotuner of the pipelined pass tiles
// ---------------------------------------------------------------------------
namespace {
std::mutex g_tune_mu;
std::map<std::array<int, 6>, std::array<int, 4>> g_tune_cache;

// the extent each pass family transforms along (x: inv_x, fwd_x; y: inv_y, fwd_y)
int family_extent(const ns3d_solver* h, int f) {
  return (f == ns3d::kTileInvX || f == ns3d::kTileFwdX) ? h->Nx : h->Ny;
}

// whether family f (TileFamily) has tile `tile` on this handle: 0 always; 1
// the alternative points per thread; 2 inv_y's bulk-copy form (tensor maps
// built); 3 / 4 the reversed radix schedule of the default / alternative
// points per thread (inv_x, inv_y, fwd_y)
bool tile_exists(const ns3d_solver* h, int f, int tile) {
  const int n = family_extent(h, f);
  switch (tile) {
    case 0:
      return true;
    case 1:
      return ns3d::extent_has_alt_tile(n);
    case 2:
      return f == ns3d::kTileInvY && h->ymaps != nullptr;
    case 3:
    case 4:
      return f != ns3d::kTileFwdX && ns3d::rev_tile_exists(n, tile);
    default:
      return false;
  }
}

void apply_tiles(ns3d_solver* h, const int* tiles) {
  drop_graph(h);  // a captured step holds the previous kernels
  for (int f = 0; f < 4; ++f) {
    h->tiles[h->precision][f] = tiles[f];
    h->geom.tile[f] = tiles[f];
  }
}
}  // namespace

extern "C" {

ns3d_status ns3d_get_tiles(const ns3d_solver* h, int* tiles) {
  if (!h || !tiles) return NS3D_ERR_BAD_ARG;
  for (int f = 0; f < 4; ++f) tiles[f] = h->geom.tile[f];
  return NS3D_OK;
}

ns3d_status ns3d_set_tiles(ns3d_solver* h, const int* tiles) {
  NS3D_TRY(check_handle(h));
  if (!tiles) return fail(h, NS3D_ERR_BAD_ARG, "null tiles");
  for (int f = 0; f < 4; ++f) {
    if (tiles[f] < 0 || tiles[f] >= NS3D_TILES_PER_FAMILY)
      return fail(h, NS3D_ERR_BAD_ARG, "a tile is 0 .. 4");
    if (!tile_exists(h, f, tiles[f]))
      return fail(h, NS3D_ERR_BAD_ARG, "no such tile for this family and extent");
  }
  NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "tiles sync");
  apply_tiles(h, tiles);
  return NS3D_OK;
}

ns3d_status ns3d_autotune(ns3d_solver* h, int reps, int force, double* ms) {
  NS3D_TRY(check_handle(h));
  if (reps < 1) return fail(h, NS3D_ERR_BAD_ARG, "reps must be >= 1");
  const std::array<int, 6> key = {h->device, h->Nx, h->Ny, h->Nz, h->batch, h->precision};
  constexpr int kT = NS3D_TILES_PER_FAMILY;
  // the tiles each family has here (the bulk-copy tile is timed for FP64 lines)
  bool has[4][kT];
  for (int f = 0; f < 4; ++f)
    for (int tile = 0; tile < kT; ++tile)
      has[f][tile] = tile_exists(h, f, tile) &&
                     (tile != 2 || h->precision == NS3D_PRECISION_FP64);
  if (ms)
    for (int i = 0; i < NS3D_TUNE_TIMES; ++i) ms[i] = -1.0;
  NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "autotune sync");
  if (!force) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      apply_tiles(h, it->second.data());
      return NS3D_OK;
    }
  }
  // time every pass with each tile on the handle's own scratch: zeros in
  // u2 stand for the state, fwd_x writes u1 (profile_passes_t).  Round r
  // runs tile r in every family that has it, the default elsewhere.
  const size_t fb = sizeof(double2) * h->nc * (size_t)h->batch;
  for (int c = 0; c < 3; ++c)
    NS3D_CHECK(h, cudaMemsetAsync(h->u2[c], 0, fb, h->stream), "autotune input");
  const ns3d_complex* u[3] = {(const ns3d_complex*)h->u2[0], (const ns3d_complex*)h->u2[1],
                              (const ns3d_complex*)h->u2[2]};
  const int saved[4] = {h->geom.tile[0], h->geom.tile[1], h->geom.tile[2], h->geom.tile[3]};
  double t[kT][5] = {};
  for (int tile = 0; tile < kT; ++tile) {
    bool any = tile == 0;
    for (int f = 0; f < 4; ++f) {
      h->geom.tile[f] = has[f][tile] ? tile : 0;
      any |= has[f][tile];
    }
    if (!any) continue;
    const ns3d_status s =
        h->precision == NS3D_PRECISION_FP32
            ? profile_passes_t<float2>(h, u[0], u[1], u[2], 1.0e-3, 100.0, reps, t[tile])
            : profile_passes_t<double2>(h, u[0], u[1], u[2], 1.0e-3, 100.0, reps, t[tile]);
    if (s != NS3D_OK) {
      for (int f = 0; f < 4; ++f) h->geom.tile[f] = saved[f];
      return s;
    }
  }
  // pass index of each family in profile_passes_t: inv_x 0, inv_y 1, fwd_y 3, fwd_x 4;
  // the fastest tile, kept if at least 2% faster than the default
  const int pass_of[4] = {0, 1, 3, 4};
  std::array<int, 4> best{};
  for (int f = 0; f < 4; ++f) {
    const double t0 = t[0][pass_of[f]];
    int b = 0;
    for (int tile = 1; tile < kT; ++tile)
      if (has[f][tile] && t[tile][pass_of[f]] < t[b][pass_of[f]]) b = tile;
    best[f] = t[b][pass_of[f]] < 0.98 * t0 ? b : 0;
    if (ms)
      for (int tile = 0; tile < kT; ++tile)
        ms[kT * f + tile] = (tile == 0 || has[f][tile]) ? t[tile][pass_of[f]] : -1.0;
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = best;
  }
  apply_tiles(h, best.data());
  return NS3D_OK;
}

}  // extern "C"

ns3d_status ns3d_profile_passes(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                                const ns3d_complex* uz, double dt, double Re, int reps,
                                double* ms) {
  NS3D_TRY(check_handle(h));
  NS3D_TRY(check_step(h, dt, Re));
  if (!args_ok3(ux, uy, uz) || !ms || reps <= 0) return fail(h, NS3D_ERR_BAD_ARG, "bad args");
  return h->precision == NS3D_PRECISION_FP32
             ? profile_passes_t<float2>(h, ux, uy, uz, dt, Re, reps, ms)
             : profile_passes_t<double2>(h, ux, uy, uz, dt, Re, reps, ms);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Ensembles: `batch` independent instances of one grid stepped together
// ---------------------------------------------------------------------------
struct ns3d_ensemble {
  ns3d_solver* h = nullptr;
};

ns3d_status ns3d_set_precision(ns3d_solver* h, int precision) {
  NS3D_TRY(check_handle(h));
  if (precision != NS3D_PRECISION_FP64 && precision != NS3D_PRECISION_FP32)
    return fail(h, NS3D_ERR_BAD_ARG, "precision must be NS3D_PRECISION_FP64 or _FP32");
  if (precision != h->precision) {
    NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "precision sync");
    drop_graph(h);  // the captured step launches the other kernels
    h->precision = precision;
    for (int f = 0; f < 4; ++f) h->geom.tile[f] = h->tiles[precision][f];
  }
  return NS3D_OK;
}

int ns3d_get_precision(const ns3d_solver* h) { return h ? h->precision : -1; }

ns3d_status ns3d_ensemble_set_precision(ns3d_ensemble* e, int precision) {
  return e ? ns3d_set_precision(e->h, precision) : NS3D_ERR_BAD_ARG;
}

ns3d_status ns3d_ensemble_autotune(ns3d_ensemble* e, int reps, int force, double* ms) {
  return e ? ns3d_autotune(e->h, reps, force, ms) : NS3D_ERR_BAD_ARG;
}

ns3d_status ns3d_ensemble_get_tiles(const ns3d_ensemble* e, int* tiles) {
  return e ? ns3d_get_tiles(e->h, tiles) : NS3D_ERR_BAD_ARG;
}

ns3d_status ns3d_ensemble_set_tiles(ns3d_ensemble* e, const int* tiles) {
  return e ? ns3d_set_tiles(e->h, tiles) : NS3D_ERR_BAD_ARG;
}

ns3d_status ns3d_ensemble_create(int batch, int Nx, int Ny, int Nz, double Lx, double Ly,
                                 double Lz, ns3d_ensemble** out) {
  if (!out) return NS3D_ERR_BAD_ARG;
  *out = nullptr;
  ns3d_solver* h = nullptr;
  const ns3d_status s = create_solver(batch, Nx, Ny, Nz, Lx, Ly, Lz, &h);
  if (s != NS3D_OK) return s;
  *out = new ns3d_ensemble{h};
  return NS3D_OK;
}

ns3d_status ns3d_ensemble_destroy(ns3d_ensemble* e) {
  if (!e) return NS3D_ERR_BAD_ARG;
  const ns3d_status s = ns3d_destroy(e->h);
  delete e;
  return s;
}

ns3d_status ns3d_ensemble_set_stream(ns3d_ensemble* e, void* stream) {
  return e ? ns3d_set_stream(e->h, stream) : NS3D_ERR_BAD_ARG;
}

const char* ns3d_ensemble_last_error(const ns3d_ensemble* e) {
  return e ? ns3d_last_error(e->h) : "null ensemble";
}

size_t ns3d_ensemble_device_bytes(const ns3d_ensemble* e) {
  return e ? ns3d_device_bytes(e->h) : 0;
}

ns3d_status ns3d_ensemble_set_forcing(ns3d_ensemble* e, const ns3d_complex* fx,
                                      const ns3d_complex* fy, const ns3d_complex* fz) {
  return e ? ns3d_set_forcing(e->h, fx, fy, fz) : NS3D_ERR_BAD_ARG;
}

ns3d_status ns3d_ensemble_set_params(ns3d_ensemble* e, const double* dt, const double* Re) {
  if (!e) return NS3D_ERR_BAD_ARG;
  ns3d_solver* h = e->h;
  if (!dt || !Re) return fail(h, NS3D_ERR_BAD_ARG, "null parameter array");
  std::vector<double> p(2 * (size_t)h->batch);
  for (int b = 0; b < h->batch; ++b) {
    if (!(dt[b] > 0.0) || !std::isfinite(dt[b]) || !(Re[b] > 0.0) || !std::isfinite(Re[b]))
      return fail(h, NS3D_ERR_BAD_ARG, "dt and Re must be finite and > 0");
    p[2 * b] = dt[b];
    p[2 * b + 1] = Re[b];
  }
  if (h->batch == 1) {  // a single instance keeps them on the host
    h->ens_dt = dt[0];
    h->ens_Re = Re[0];
    h->ens_params = true;
    return NS3D_OK;
  }
  NS3D_CHECK(h, cudaMemcpyAsync(h->dtRe, p.data(), sizeof(double) * p.size(),
                                cudaMemcpyHostToDevice, h->stream), "parameter copy");
  NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "parameter sync");
  h->ens_params = true;
  return NS3D_OK;
}

ns3d_status ns3d_ensemble_rk3_steps(ns3d_ensemble* e, ns3d_complex* ux, ns3d_complex* uy,
                                    ns3d_complex* uz, int nsteps) {
  if (!e) return NS3D_ERR_BAD_ARG;
  ns3d_solver* h = e->h;
  NS3D_TRY(check_handle(h));
  if (!args_ok3(ux, uy, uz) || nsteps < 0) return fail(h, NS3D_ERR_BAD_ARG, "null field");
  if (!h->ens_params) return fail(h, NS3D_ERR_BAD_ARG, "ns3d_ensemble_set_params first");
  if (h->batch == 1) return rk3_steps_impl(h, ux, uy, uz, h->ens_dt, h->ens_Re, nsteps);
  return rk3_steps_impl(h, ux, uy, uz, 0.0, 0.0, nsteps);
}

ns3d_status ns3d_ensemble_diagnostics(ns3d_ensemble* e, const ns3d_complex* ux,
                                      const ns3d_complex* uy, const ns3d_complex* uz,
                                      double* energy, double* dissipation) {
  if (!e) return NS3D_ERR_BAD_ARG;
  ns3d_solver* h = e->h;
  NS3D_TRY(check_handle(h));
  if (!args_ok3(ux, uy, uz) || !energy || !dissipation)
    return fail(h, NS3D_ERR_BAD_ARG, "null pointer");
  ns3d::DiagGeom g{};
  g.Nx = h->Nx; g.Ny = h->Ny; g.Nz = h->Nz; g.Mz = h->Mz;
  g.kfx = h->geom.kfx; g.kfy = h->geom.kfy; g.kfz = h->geom.kfz;
  g.dx = h->Lx / (double)h->Nx;
  g.dy = h->Ly / (double)h->Ny;
  g.dz = h->Lz / (double)h->Nz;
  g.inv_vol = h->geom.inv_vol;
  for (int b = 0; b < h->batch; ++b) {
    const size_t o = (size_t)b * h->nc;
    ns3d::diag_partial_kernel<<<kDiagBlocks, kDiagThreads, 0, h->stream>>>(
        (const double2*)ux + o, (const double2*)uy + o, (const double2*)uz + o, g,
        h->diag_partial);
    NS3D_CHECK(h, cudaGetLastError(), "diag_partial");
    ns3d::diag_final_kernel<<<1, 1024, 0, h->stream>>>(h->diag_partial, kDiagBlocks,
                                                       h->diag_out + 3 * b);
    NS3D_CHECK(h, cudaGetLastError(), "diag_final");
  }
  std::vector<double> r(3 * (size_t)h->batch);
  NS3D_CHECK(h, cudaMemcpyAsync(r.data(), h->diag_out, sizeof(double) * r.size(),
                                cudaMemcpyDeviceToHost, h->stream), "diag copy");
  NS3D_CHECK(h, cudaStreamSynchronize(h->stream), "diag sync");
  bool finite = true;
  for (int b = 0; b < h->batch; ++b) {
    energy[b] = r[3 * b];
    dissipation[b] = r[3 * b + 1];
    finite = finite && std::isfinite(r[3 * b]) && std::isfinite(r[3 * b + 1]);
  }
  return finite ? NS3D_OK : fail(h, NS3D_ERR_NONFINITE, "diagnostics are not finite");
}
