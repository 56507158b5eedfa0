// Harness around the reference's own Krylov code (TEST INFRASTRUCTURE).
//
// oracle/Makefile compiles the reference's Source/Arnoldi/{Arnoldi_Driver.cu,
// BiCGStabL.cu, Newton.cu, cuda_supp.cu, memory_operations.cu, Matrix_Vector_emulator.cu,
// Implicit_restart_Arnoldi.cu, Products.cpp, QR_Shifts.cpp, Select_Shifts.cpp,
// LAPACK_routines.cpp, timer.cpp, file_operations.cpp}
// unmodified (with oracle/c99_complex_prelude.h force-included) together with
// this file into oracle/_ref/libarnoldi_ref.so.  This file adds only:
//   * flat C entry points for ctypes (host arrays in, host arrays out);
//   * the matrix-vector callbacks handed to Arnoldi_driver: the reference's
//     own 1-D periodic Laplacian (user_Ax_function,
//     Source/Arnoldi/Matrix_Vector_emulator.cu:27-36) and a dense matrix
//     applied with cublasDgemv;
//   * forwarding of the Fortran LAPACK names the reference calls (dgeqrf_,
//     dormqr_, zgeev_, dhseqr_) and of openblas_set_num_threads to the LP64
//     OpenBLAS that scipy ships (exported there with a "scipy_" prefix); the
//     image has no other LAPACK.
// Arnoldi_driver needs a GPU; the QR-shift and shift-selection entry points
// are host code and run anywhere the library loads.
#include "Arnoldi_Driver.h"
#include "Implicit_restart_Arnoldi.h"
#include "BiCGStabL.h"
#include "Newton.h"
#include "QR_Shifts.h"
#include "Select_Shifts.h"
#include "Matrix_Vector_emulator.h"

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <vector>

extern "C" {
void scipy_dgeqrf_(int*, int*, double*, int*, double*, double*, int*, int*);
void scipy_dormqr_(char*, char*, int*, int*, int*, double*, int*, double*, double*, int*,
                   double*, int*, int*);
void scipy_zgeev_(char*, char*, int*, double _Complex*, int*, double _Complex*,
                  double _Complex*, int*, double _Complex*, int*, double _Complex*, int*,
                  double _Complex*, int*);
void scipy_dhseqr_(char*, char*, int*, int*, int*, double*, int*, double*, double*, double*,
                   int*, double*, int*, int*);

void dgeqrf_(int* M, int* N, double* A, int* LDA, double* TAU, double* WORK, int* LWORK,
             int* INFO)
{
    scipy_dgeqrf_(M, N, A, LDA, TAU, WORK, LWORK, INFO);
}
void dormqr_(char* SIDE, char* TRANS, int* M, int* N, int* K, double* A, int* LDA, double* TAU,
             double* C, int* LDC, double* WORK, int* LWORK, int* INFO)
{
    scipy_dormqr_(SIDE, TRANS, M, N, K, A, LDA, TAU, C, LDC, WORK, LWORK, INFO);
}
void zgeev_(char* jobvl, char* jobvr, int* n, double _Complex* a, int* lda, double _Complex* w,
            double _Complex* vl, int* ldvl, double _Complex* vr, int* ldvr,
            double _Complex* work, int* lwork, double _Complex* rwork, int* info)
{
    scipy_zgeev_(jobvl, jobvr, n, a, lda, w, vl, ldvl, vr, ldvr, work, lwork, rwork, info);
}
void scipy_openblas_set_num_threads(int);
void openblas_set_num_threads(int n) { scipy_openblas_set_num_threads(n); }

void dhseqr_(char* JOB, char* COMPZ, int* N, int* ILO, int* IHI, double* H, int* LDH, double* WR,
             double* WI, double* Z, int* LDZ, double* WORK, int* LWORK, int* INFO)
{
    scipy_dhseqr_(JOB, COMPZ, N, ILO, IHI, H, LDH, WR, WI, Z, LDZ, WORK, LWORK, INFO);
}
}

namespace {

struct DenseMap {
    cublasHandle_t handle;
    int n;
    double* A;  // column-major n x n on the device
};

void dense_map(void* ctx, void* in, void* out)
{
    DenseMap* d = static_cast<DenseMap*>(ctx);
    const double one = 1.0, zero = 0.0;
    cublasDgemv(d->handle, CUBLAS_OP_N, d->n, d->n, &one, d->A, d->n,
                static_cast<double*>(in), 1, &zero, static_cast<double*>(out), 1);
}

void laplace_map(void* ctx, void* in, void* out)
{
    user_Ax_function(static_cast<Ax_struct*>(ctx), static_cast<real*>(in),
                     static_cast<real*>(out));
}

// Runs Arnoldi_driver on host copies of V (n x m), H (m x m) and f (n).
int run_arnoldi(int n, int m, int k, user_map_vector Axb, void* ctx, cublasHandle_t handle,
                double* V, double* H, double* f)
{
    double *V_d = nullptr, *f_d = nullptr, *v_d = nullptr, *w_d = nullptr, *c_d = nullptr,
           *h_d = nullptr;
    const size_t nb = sizeof(double) * static_cast<size_t>(n);
    if (cudaMalloc(&V_d, nb * m) != cudaSuccess) return 1;
    cudaMalloc(&f_d, nb);
    cudaMalloc(&v_d, nb);
    cudaMalloc(&w_d, nb);
    cudaMalloc(&c_d, sizeof(double) * m);
    cudaMalloc(&h_d, sizeof(double) * m);
    cudaMemcpy(V_d, V, nb * m, cudaMemcpyHostToDevice);
    cudaMemcpy(f_d, f, nb, cudaMemcpyHostToDevice);
    cudaMemset(v_d, 0, nb);
    cudaMemset(w_d, 0, nb);
    std::vector<double> vec_h(m, 0.0);
    Arnoldi_driver(handle, n, Axb, ctx, V_d, H, f_d, k, m, v_d, w_d, c_d, h_d, vec_h.data());
    cudaMemcpy(V, V_d, nb * m, cudaMemcpyDeviceToHost);
    cudaMemcpy(f, f_d, nb, cudaMemcpyDeviceToHost);
    const cudaError_t err = cudaDeviceSynchronize();
    cudaFree(V_d);
    cudaFree(f_d);
    cudaFree(v_d);
    cudaFree(w_d);
    cudaFree(c_d);
    cudaFree(h_d);
    return err == cudaSuccess ? 0 : 2;
}

}  // namespace

extern "C" {

// Arnoldi_driver (Source/Arnoldi/Arnoldi_Driver.cu:29) with the reference's
// 1-D periodic Laplacian test operator.
int ref_arnoldi_laplace(int n, int m, int k, double* V, double* H, double* f)
{
    cublasHandle_t handle;
    if (cublasCreate(&handle) != CUBLAS_STATUS_SUCCESS) return 3;
    Ax_struct ctx;
    ctx.N = n;
    const int rc = run_arnoldi(n, m, k, laplace_map, &ctx, handle, V, H, f);
    cublasDestroy(handle);
    return rc;
}

// Arnoldi_driver with a dense column-major n x n matrix A.
int ref_arnoldi_dense(int n, int m, int k, const double* A, double* V, double* H, double* f)
{
    cublasHandle_t handle;
    if (cublasCreate(&handle) != CUBLAS_STATUS_SUCCESS) return 3;
    DenseMap ctx;
    ctx.handle = handle;
    ctx.n = n;
    if (cudaMalloc(&ctx.A, sizeof(double) * n * static_cast<size_t>(n)) != cudaSuccess) {
        cublasDestroy(handle);
        return 1;
    }
    cudaMemcpy(ctx.A, A, sizeof(double) * n * static_cast<size_t>(n), cudaMemcpyHostToDevice);
    const int rc = run_arnoldi(n, m, k, dense_map, &ctx, handle, V, H, f);
    cudaFree(ctx.A);
    cublasDestroy(handle);
    return rc;
}

// Device-resident timing of `reps` factorisations (k = 0 to m) with the
// reference's Laplacian, each restarted from the same f0 (a device copy
// inside the timed region): CUDA events on the legacy stream, ms total.
// *h00 receives H(0,0) of the last factorisation (a consistency check).
double ref_time_arnoldi_laplace(int n, int m, int reps, const double* f0, double* h00)
{
    cublasHandle_t handle;
    if (cublasCreate(&handle) != CUBLAS_STATUS_SUCCESS) return -1.0;
    Ax_struct ctx;
    ctx.N = n;
    const size_t nb = sizeof(double) * static_cast<size_t>(n);
    double *V_d = nullptr, *f_d = nullptr, *f0_d = nullptr, *v_d = nullptr, *w_d = nullptr,
           *c_d = nullptr, *h_d = nullptr;
    if (cudaMalloc(&V_d, nb * m) != cudaSuccess) return -1.0;
    cudaMalloc(&f_d, nb);
    cudaMalloc(&f0_d, nb);
    cudaMalloc(&v_d, nb);
    cudaMalloc(&w_d, nb);
    cudaMalloc(&c_d, sizeof(double) * m);
    cudaMalloc(&h_d, sizeof(double) * m);
    cudaMemset(V_d, 0, nb * m);
    cudaMemcpy(f0_d, f0, nb, cudaMemcpyHostToDevice);
    std::vector<double> H(static_cast<size_t>(m) * m, 0.0), vec_h(m, 0.0);
    // one untimed factorisation (cuBLAS initialisation, first touches)
    cudaMemcpy(f_d, f0_d, nb, cudaMemcpyDeviceToDevice);
    Arnoldi_driver(handle, n, laplace_map, &ctx, V_d, H.data(), f_d, 0, m, v_d, w_d, c_d, h_d,
                   vec_h.data());
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a, 0);
    for (int r = 0; r < reps; ++r) {
        cudaMemcpyAsync(f_d, f0_d, nb, cudaMemcpyDeviceToDevice, 0);
        Arnoldi_driver(handle, n, laplace_map, &ctx, V_d, H.data(), f_d, 0, m, v_d, w_d, c_d,
                       h_d, vec_h.data());
    }
    cudaEventRecord(b, 0);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (h00) *h00 = H[0];
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(V_d);
    cudaFree(f_d);
    cudaFree(f0_d);
    cudaFree(v_d);
    cudaFree(w_d);
    cudaFree(c_d);
    cudaFree(h_d);
    cublasDestroy(handle);
    return cudaDeviceSynchronize() == cudaSuccess ? static_cast<double>(ms) : -1.0;
}

// BiCGStabL (Source/Arnoldi/BiCGStabL.cu:18-185) on A x = rhs with a dense
// column-major A; x is the initial guess on entry and the result on exit,
// *tol / *iter are the reference's in/out arguments.  Returns its flag.
int ref_bicgstabl_dense(int n, int L, const double* A, double* x, const double* rhs,
                        double* tol, int* iter)
{
    cublasHandle_t handle;
    if (cublasCreate(&handle) != CUBLAS_STATUS_SUCCESS) return 99;
    DenseMap ctx;
    ctx.handle = handle;
    ctx.n = n;
    const size_t nb = sizeof(double) * static_cast<size_t>(n);
    double *x_d = nullptr, *b_d = nullptr;
    cudaMalloc(&ctx.A, nb * n);
    cudaMalloc(&x_d, nb);
    cudaMalloc(&b_d, nb);
    cudaMemcpy(ctx.A, A, nb * n, cudaMemcpyHostToDevice);
    cudaMemcpy(x_d, x, nb, cudaMemcpyHostToDevice);
    cudaMemcpy(b_d, rhs, nb, cudaMemcpyHostToDevice);
    const int flag = BiCGStabL(handle, L, n, dense_map, &ctx, x_d, b_d, tol, iter, false, 1000);
    cudaMemcpy(x, x_d, nb, cudaMemcpyDeviceToHost);
    cudaFree(ctx.A);
    cudaFree(x_d);
    cudaFree(b_d);
    cublasDestroy(handle);
    return cudaDeviceSynchronize() == cudaSuccess ? flag : 98;
}

// The nonlinear test problem of the Newton golden vectors:
//   F(x) = A x + c x^3 - b (elementwise cube),  J(x) v = A v + 3 c x^2 v.
// As with the reference's own NSCallRHS_reduced / Jacobian pair, the
// residual map stores its argument as the point the Jacobian map linearises
// about.
struct CubicMap {
    cublasHandle_t handle;
    int n;
    double* A;     // column-major n x n
    double* b;
    double* base;  // the point of the last residual evaluation
    double c;
};

__global__ void cubic_rhs_tail(int n, double c, const double* x, const double* b, double* out,
                               double* base)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double xi = x[i];
        base[i] = xi;
        out[i] = out[i] + c * xi * xi * xi - b[i];
    }
}

__global__ void cubic_jac_tail(int n, double c, const double* v, const double* base, double* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = out[i] + 3.0 * c * base[i] * base[i] * v[i];
}

void cubic_rhs(void* ctx, void* in, void* out)
{
    CubicMap* m = static_cast<CubicMap*>(ctx);
    const double one = 1.0, zero = 0.0;
    cublasDgemv(m->handle, CUBLAS_OP_N, m->n, m->n, &one, m->A, m->n,
                static_cast<double*>(in), 1, &zero, static_cast<double*>(out), 1);
    cubic_rhs_tail<<<(m->n + 255) / 256, 256>>>(m->n, m->c, static_cast<double*>(in), m->b,
                                                static_cast<double*>(out), m->base);
}

void cubic_jac(void* ctx, void* in, void* out)
{
    CubicMap* m = static_cast<CubicMap*>(ctx);
    const double one = 1.0, zero = 0.0;
    cublasDgemv(m->handle, CUBLAS_OP_N, m->n, m->n, &one, m->A, m->n,
                static_cast<double*>(in), 1, &zero, static_cast<double*>(out), 1);
    cubic_jac_tail<<<(m->n + 255) / 256, 256>>>(m->n, m->c, static_cast<double*>(in), m->base,
                                                static_cast<double*>(out));
}

// Newton (Source/Arnoldi/Newton.cu:9-98) on the cubic problem above; x is
// the initial guess on entry, the result on exit.  Returns its flag.
int ref_newton_cubic(int n, const double* A, const double* b, double c, double* x, double* tol,
                     int* iter, double tol_lin, int iter_lin)
{
    cublasHandle_t handle;
    if (cublasCreate(&handle) != CUBLAS_STATUS_SUCCESS) return 99;
    CubicMap m;
    m.handle = handle;
    m.n = n;
    m.c = c;
    const size_t nb = sizeof(double) * static_cast<size_t>(n);
    double* x_d = nullptr;
    cudaMalloc(&m.A, nb * n);
    cudaMalloc(&m.b, nb);
    cudaMalloc(&m.base, nb);
    cudaMalloc(&x_d, nb);
    cudaMemcpy(m.A, A, nb * n, cudaMemcpyHostToDevice);
    cudaMemcpy(m.b, b, nb, cudaMemcpyHostToDevice);
    cudaMemcpy(x_d, x, nb, cudaMemcpyHostToDevice);
    cudaMemset(m.base, 0, nb);
    const int flag = Newton(handle, cubic_jac, &m, cubic_rhs, &m, n, x_d, tol, iter, tol_lin,
                            iter_lin, false, 100);
    cudaMemcpy(x, x_d, nb, cudaMemcpyDeviceToHost);
    cudaFree(m.A);
    cudaFree(m.b);
    cudaFree(m.base);
    cudaFree(x_d);
    cublasDestroy(handle);
    return cudaDeviceSynchronize() == cudaSuccess ? flag : 98;
}

// The reference's 1-D periodic Laplacian applied once (for checking the
// project's copy of the test operator).
int ref_laplace_apply(int n, const double* in, double* out)
{
    double *a = nullptr, *b = nullptr;
    if (cudaMalloc(&a, sizeof(double) * n) != cudaSuccess) return 1;
    cudaMalloc(&b, sizeof(double) * n);
    cudaMemcpy(a, in, sizeof(double) * n, cudaMemcpyHostToDevice);
    cudaMemset(b, 0, sizeof(double) * n);
    Ax_struct ctx;
    ctx.N = n;
    laplace_map(&ctx, a, b);
    cudaMemcpy(out, b, sizeof(double) * n, cudaMemcpyDeviceToHost);
    const cudaError_t err = cudaDeviceSynchronize();
    cudaFree(a);
    cudaFree(b);
    return err == cudaSuccess ? 0 : 2;
}

// QR_shifts (Source/Arnoldi/QR_Shifts.cpp:46-72); host only.  Q (m x m) is
// output, H (m x m) is updated in place, eigenvalues are given as separate
// real and imaginary arrays of length m.
void ref_qr_shifts(int k, int m, double* Q, double* H, const double* eig_re,
                   const double* eig_im, int* ko)
{
    std::vector<double _Complex> eig(m);
    for (int i = 0; i < m; ++i) {
        __real__ eig[i] = eig_re[i];
        __imag__ eig[i] = eig_im[i];
    }
    QR_shifts(k, m, Q, H, eig.data(), ko);
}

// Implicit_restart_Arnoldi_GPU_data_Matrix_Exponent
// (Source/Arnoldi/Implicit_restart_Arnoldi.cu:456-742) with dense operators:
// the shift-invert map is the column-major n_rot x n_rot matrix Minv
// (n_rot = 2n when rotated, else n) and the original map the column-major
// n x n matrix A, both applied with cublasDgemv; which = "LR",
// which_exponent = "LM" as main passes them (Source/NS3D_periodic.cu:1710).
// The reference prints its progress and eigenvalues, writes H_pre.dat,
// H_Schur.dat and Q_Schur.dat into the working directory and seeds its start
// vector from the clock; it never fills its eigenvalue argument, so this
// entry returns the k eigenvectors (rows of the k x n arrays vec_re, vec_im,
// in the reference's column order) and the final Ritz norm in *ritz.
int ref_ira_matrix_exponent_dense(int n, int rotated, const double* Minv, const double* A, int k,
                                  int m, double tol, int max_iter, double* vec_re,
                                  double* vec_im, double* ritz)
{
    const int n_rot = rotated ? 2 * n : n;
    cublasHandle_t handle;
    if (cublasCreate(&handle) != CUBLAS_STATUS_SUCCESS) return 1;
    double *Minv_d = nullptr, *A_d = nullptr, *er_d = nullptr, *ei_d = nullptr;
    cudaMalloc(&Minv_d, sizeof(double) * static_cast<size_t>(n_rot) * n_rot);
    cudaMalloc(&A_d, sizeof(double) * static_cast<size_t>(n) * n);
    cudaMalloc(&er_d, sizeof(double) * static_cast<size_t>(n) * k);
    cudaMalloc(&ei_d, sizeof(double) * static_cast<size_t>(n) * k);
    cudaMemcpy(Minv_d, Minv, sizeof(double) * static_cast<size_t>(n_rot) * n_rot,
               cudaMemcpyHostToDevice);
    cudaMemcpy(A_d, A, sizeof(double) * static_cast<size_t>(n) * n, cudaMemcpyHostToDevice);
    DenseMap inv{handle, n_rot, Minv_d};
    DenseMap orig{handle, n, A_d};
    std::vector<double _Complex> eigenvalues(static_cast<size_t>(m));
    char which[2] = {'L', 'R'};
    char which_exponent[2] = {'L', 'M'};
    *ritz = Implicit_restart_Arnoldi_GPU_data_Matrix_Exponent(
        handle, false, n, dense_map, &inv, dense_map, &orig, which, which_exponent, k, m,
        eigenvalues.data(), tol, max_iter, rotated != 0, er_d, ei_d, 1);
    cudaMemcpy(vec_re, er_d, sizeof(double) * static_cast<size_t>(n) * k, cudaMemcpyDeviceToHost);
    cudaMemcpy(vec_im, ei_d, sizeof(double) * static_cast<size_t>(n) * k, cudaMemcpyDeviceToHost);
    const cudaError_t err = cudaDeviceSynchronize();
    cudaFree(Minv_d);
    cudaFree(A_d);
    cudaFree(er_d);
    cudaFree(ei_d);
    cublasDestroy(handle);
    return err == cudaSuccess ? 0 : 2;
}

// Implicit_restart_Arnoldi_GPU_data (Source/Arnoldi/Implicit_restart_Arnoldi.cu:
// 444-453) with a caller's map (a user_map_vector, e.g. the NS harness's
// ref_map_linearised_reduced) on vectors of length n, verbose off, the
// eigenvector arrays allocated here beforehand as main does; which = "LR"
// (which_lm = 0) or "LM".  The reference prints its timer and eigenvalues to
// stdout and writes H_pre.dat, H_Schur.dat and Q_Schur.dat into the working
// directory.  Returns the Ritz norm; *ms the device time of the call (CUDA
// events on the legacy stream, synchronised).  With tol = 0 the loop runs
// exactly max_iter restart cycles before the final stage.
double ref_ira_map(int n, void* Axb, void* ctx, int k, int m, double tol, int max_iter,
                   int which_lm, double* ms)
{
    cublasHandle_t handle;
    if (cublasCreate(&handle) != CUBLAS_STATUS_SUCCESS) return -1.0;
    double *er_d = nullptr, *ei_d = nullptr;
    cudaMalloc(&er_d, sizeof(double) * static_cast<size_t>(n) * k);
    cudaMalloc(&ei_d, sizeof(double) * static_cast<size_t>(n) * k);
    std::vector<double _Complex> eigenvalues(static_cast<size_t>(m));
    char which[2] = {'L', which_lm ? 'M' : 'R'};
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a, 0);
    const double ritz = Implicit_restart_Arnoldi_GPU_data(
        handle, false, n, reinterpret_cast<user_map_vector>(Axb), ctx, which, k, m,
        eigenvalues.data(), tol, max_iter, er_d, ei_d, 1);
    cudaEventRecord(b, 0);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    *ms = t;
    const cudaError_t err = cudaDeviceSynchronize();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(er_d);
    cudaFree(ei_d);
    cublasDestroy(handle);
    return err == cudaSuccess ? ritz : -1.0;
}

// select_shifts (Source/Arnoldi/Select_Shifts.cpp:86-133); host only.
void ref_select_shifts(int m, double* H, const char* which, double* eig_re, double* eig_im,
                       double* ritz)
{
    std::vector<double _Complex> vecs(static_cast<size_t>(m) * m), eig(m);
    char w[2] = {which[0], which[1]};
    select_shifts(m, H, w, vecs.data(), eig.data(), ritz);
    for (int i = 0; i < m; ++i) {
        eig_re[i] = __real__ eig[i];
        eig_im[i] = __imag__ eig[i];
    }
}

}  // extern "C"
