/*
 * ns3d.h - C ABI of the B200 (sm_100a) pseudo-spectral Navier-Stokes path.
 *
 * Drop-in for the RK3 / tangent / Krylov-matvec entry points of
 * evstigneevnm/NS3DPeriodic.  Every velocity field is a DEVICE array in the
 * reference's own layout: [Nx][Ny][Mz] complex doubles (interleaved re, im;
 * cufftDoubleComplex), Mz = Nz/2 + 1, element (j,k,l) at j*Ny*Mz + k*Mz + l
 * (Source/Macros.h:11 IN(i,j,k) with Nz = Mz).  Spectra are unnormalised
 * (forward D2Z without scaling, inverse followed by 1/(Nx Ny Nz)), exactly as
 * Source/math_support.cu:301-334.  Viscosity is 1/Re.
 *
 * The reference keeps cuFFT plans, the 2/3 scratch and the wave-number /
 * Leray / mask tables in file-static state set up by main()
 * (Source/NS3D_periodic.cu:1141-1272).  Here a handle owns the equivalent:
 * its own scratch, tables computed on the fly inside the kernels, and one
 * CUDA stream.  Handles are independent and re-entrant; one handle must not
 * be used from two host threads at once.
 *
 * All functions return an ns3d_status; nothing prints or exits.  Functions
 * that launch work are asynchronous on the handle's stream unless stated.
 * The default stream of a handle is a blocking stream, so it is ordered with
 * work on the legacy default stream (the reference's stream).
 */
#ifndef NS3D_H_
#define NS3D_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ns3d_solver ns3d_solver;

typedef struct ns3d_complex {
  double x, y;
} ns3d_complex;

typedef enum ns3d_status {
  NS3D_OK = 0,
  NS3D_ERR_BAD_ARG = 1,     /* null handle/pointer, non-positive size, bad dt/Re */
  NS3D_ERR_UNSUPPORTED = 2, /* a grid extent without a compiled FFT plan */
  NS3D_ERR_OOM = 3,         /* device allocation failed */
  NS3D_ERR_CUDA = 4,        /* a CUDA launch or API call failed (see ns3d_last_error) */
  NS3D_ERR_NONFINITE = 5,   /* a diagnostic reduction met NaN/Inf */
  NS3D_ERR_TIMEOUT = 6,     /* a bounded device wait gave up */
  NS3D_ERR_NOT_CONVERGED = 7, /* an inner linear solve stopped without converging */
  NS3D_ERR_CANCELLED = 8      /* a server request was cancelled (ns3d_server_cancel) */
} ns3d_status;

/* ----------------------------------------------------------------------- */
/* lifetime                                                                 */
/* ----------------------------------------------------------------------- */

/* Creates a solver for an Nx x Ny x Nz grid on a box Lx x Ly x Lz, on the
 * current CUDA device.  Replaces cufftPlan3d + init_fft_plans
 * (Source/math_support.h:15), the host table builders build_*
 * (Source/math_support.h:49-58, called with Mz as Nz at
 * Source/NS3D_periodic.cu:1153-1161) and init_dealiasing
 * (Source/advection_2_3.h:40).  Supported extents: ns3d_supported_extent(). */
ns3d_status ns3d_create(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                        ns3d_solver** out);

/* Releases the handle.  Replaces clean_dealiasing (Source/advection_2_3.h:42). */
ns3d_status ns3d_destroy(ns3d_solver* h);

/* 1 if n has a compiled FFT plan (8, 16, 24, 32, 48, 64, 96, 128, 192, 256,
 * 384, 512), else 0.  Host only. */
int ns3d_supported_extent(int n);

/* Uses `stream` (a cudaStream_t, may be 0 for the legacy default stream) for
 * every later launch of this handle. */
ns3d_status ns3d_set_stream(ns3d_solver* h, void* stream);

/* Blocks until the handle's stream is idle. */
ns3d_status ns3d_synchronize(ns3d_solver* h);

/* Human-readable text of the last error on this handle ("" if none). */
const char* ns3d_last_error(const ns3d_solver* h);
const char* ns3d_status_string(ns3d_status s);

/* Self-test of the bounded device waits (no reference counterpart): one CTA
 * waits, with the waits the tensor-copy (TMA) passes use, on an mbarrier
 * phase that nothing completes.  The wait gives up after about 0.1 s, writes
 * the timeout code to a device flag and the kernel returns, leaving the
 * context usable.  *seconds (may be NULL) receives the time the launch
 * took.  NS3D_OK when the wait gave up and flagged it, NS3D_ERR_CUDA
 * otherwise.  Synchronous on the current device; allocates a 4-byte flag. */
ns3d_status ns3d_selftest_bounded_wait(double* seconds);

/* Device bytes the handle holds (scratch + tables). */
size_t ns3d_device_bytes(const ns3d_solver* h);

/* ----------------------------------------------------------------------- */
/* forcing                                                                  */
/* ----------------------------------------------------------------------- */

/* Captures the body force f_hat (3 device fields, reference layout) used by
 * every later explicit step and RHS evaluation.  The reference passes
 * fx_hat_d.. to each call (Source/RK_time_step.h:26); the handle instead
 * scans the field once (synchronously) and keeps it as a sparse list of its
 * non-zero modes when there are at most 4096 of them, else references the
 * caller's arrays, which must then stay alive and unchanged.  Null pointers
 * clear the forcing. */
ns3d_status ns3d_set_forcing(ns3d_solver* h, const ns3d_complex* fx, const ns3d_complex* fy,
                             const ns3d_complex* fz);

/* Number of non-zero forcing modes kept (-1: dense forcing referenced). */
int ns3d_forcing_modes(const ns3d_solver* h);

/* ----------------------------------------------------------------------- */
/* time stepping: Source/RK_time_step.h                                     */
/* ----------------------------------------------------------------------- */

/* One Shu-Osher SSP-RK3 step in place: RK3_SSP (Source/RK_time_step.h:26,
 * Source/RK_time_step.cu:310-327).  The reference's scratch arguments
 * (u_1..u_3, Q, div, tables) are owned by the handle. */
ns3d_status ns3d_rk3_step(ns3d_solver* h, ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                          double dt, double Re);

/* nsteps RK3 steps in place, replayed from one captured CUDA graph (the time
 * loop of Source/NS3D_periodic.cu:1303-1315 without diagnostics). */
ns3d_status ns3d_rk3_steps(ns3d_solver* h, ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                           double dt, double Re, int nsteps);

/* One explicit Euler stage u <- u + dt L(u): single_time_step
 * (Source/RK_time_step.h:19, Source/RK_time_step.cu:248-263). */
ns3d_status ns3d_euler_step(ns3d_solver* h, ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                            double dt, double Re);

/* rhs = -P.Q(u) - |k|^2/Re u + f: return_RHS (Source/RK_time_step.h:34,
 * Source/RK_time_step.cu:231-245).  rhs may be u itself (in place), as in
 * NSCallRHS_reduced (Source/NS3D_periodic.cu:415-441). */
ns3d_status ns3d_rhs(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                     const ns3d_complex* uz, ns3d_complex* rx, ns3d_complex* ry, ns3d_complex* rz,
                     double Re);

/* Qhat = FFT[(Mu.grad)(Mu)] with Re(Qhat)=0, Qhat(0)=0:
 * calculate_convolution_2p3 (Source/advection_2_3.h:44). */
ns3d_status ns3d_convolution(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                             const ns3d_complex* uz, ns3d_complex* Qx, ns3d_complex* Qy,
                             ns3d_complex* Qz);

/* Qhat = FFT[(Mv.grad)(Mu) + (Mu.grad)(Mv)], Re(Qhat)=0, Qhat(0)=0:
 * calculate_convolution_2p3_UV (Source/advection_2_3.h:46). */
ns3d_status ns3d_convolution_uv(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                                const ns3d_complex* uz, const ns3d_complex* vx,
                                const ns3d_complex* vy, const ns3d_complex* vz, ns3d_complex* Qx,
                                ns3d_complex* Qy, ns3d_complex* Qz);

/* ----------------------------------------------------------------------- */
/* tangent (Jacobian-vector) steppers                                       */
/* ----------------------------------------------------------------------- */

/* One tangent step: Heun on v about an RK3 base step of u, both in place:
 * RK3_SSP_UV (Source/RK_time_step.h:31, Source/RK_time_step.cu:342-355). */
ns3d_status ns3d_jvp_step(ns3d_solver* h, ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                          ns3d_complex* vx, ns3d_complex* vy, ns3d_complex* vz, double dt,
                          double Re);

/* v <- v + dt (-P.B(u,v) - |k|^2/Re v): single_time_step_UV
 * (Source/RK_time_step.h:21, Source/RK_time_step.cu:265-278); u is not
 * changed. */
ns3d_status ns3d_tangent_euler_step(ns3d_solver* h, const ns3d_complex* ux,
                                    const ns3d_complex* uy, const ns3d_complex* uz,
                                    ns3d_complex* vx, ns3d_complex* vy, ns3d_complex* vz,
                                    double dt, double Re);

/* nsteps tangent steps (the Timesteps_period loop of
 * NSCallMatrixVector_exponential, Source/NS3D_periodic.cu:444-470). */
ns3d_status ns3d_jvp_steps(ns3d_solver* h, ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                           ns3d_complex* vx, ns3d_complex* vy, ns3d_complex* vz, double dt,
                           double Re, int nsteps);

/* v <- J(u) v = -P.B(u,v) - |k|^2/Re v in place: RK3_SSP_UV_RHS
 * (Source/RK_time_step.h:28, Source/RK_time_step.cu:330-338). */
ns3d_status ns3d_linearised_rhs(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                                const ns3d_complex* uz, ns3d_complex* vx, ns3d_complex* vy,
                                ns3d_complex* vz, double Re);

/* v <- (v - dt P.B(u,v)) / (1 + dt |k|^2/Re) in place: single_time_step_iUV_RHS
 * (Source/RK_time_step.h:23, Source/RK_time_step.cu:296-306). */
ns3d_status ns3d_implicit_tangent_step(ns3d_solver* h, const ns3d_complex* ux,
                                       const ns3d_complex* uy, const ns3d_complex* uz,
                                       ns3d_complex* vx, ns3d_complex* vy, ns3d_complex* vz,
                                       double dt, double Re);

/* ----------------------------------------------------------------------- */
/* Krylov adapters: Source/NS3D_periodic.cu:173-385                          */
/* ----------------------------------------------------------------------- */

/* Length of a reduced Krylov vector: 3*(Nx*Ny*Mz - 1). */
int64_t ns3d_krylov_length(const ns3d_solver* h);

/* vec = [Im vx(1..), Im vy(1..), Im vz(1..)]: A_vector_from_velocities_reduced_kernel
 * (Source/NS3D_periodic.cu:271-284).  vec is a device array of doubles. */
ns3d_status ns3d_pack_reduced(ns3d_solver* h, const ns3d_complex* vx, const ns3d_complex* vy,
                              const ns3d_complex* vz, double* vec);

/* vec = Im v(1..) - a*vec_a (+ b*vec_b when vec_b is not NULL), in that
 * order, on reduced vectors: A_vector_from_velocities_reduced_shifted_kernel
 * (a = shift_real, vec_b = NULL) and the
 * A_vector_from_velocities_reduced_shifted_rotated_kernel_Real / _Imag pair
 * (Source/NS3D_periodic.cu:253-300; with the halves of a rotated vector as
 * vec_a and vec_b).  vec_a is required. */
ns3d_status ns3d_pack_reduced_shifted(ns3d_solver* h, const ns3d_complex* vx,
                                      const ns3d_complex* vy, const ns3d_complex* vz,
                                      const double* vec_a, double a, const double* vec_b,
                                      double b, double* vec);

/* v = i*vec, Re := 0, mode 0 := 0: velocities_from_A_vector_reduced_kernel
 * (Source/NS3D_periodic.cu:173-200). */
ns3d_status ns3d_unpack_reduced(ns3d_solver* h, const double* vec, ns3d_complex* vx,
                                ns3d_complex* vy, ns3d_complex* vz);

/* vec_out = J(u) vec_in - vec_in/tau on reduced vectors (device arrays):
 * NSCallMatrixVector_reduced (tau <= 0) and
 * NSCallMatrixVector_reduced_Newton_Globalization (tau > 0),
 * Source/NS3D_periodic.cu:340-385. */
ns3d_status ns3d_matvec_reduced(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                                const ns3d_complex* uz, const double* vec_in, double* vec_out,
                                double Re, double tau);

/* ----------------------------------------------------------------------- */
/* plain 3-D transforms (Source/math_support.cu:301-334)                      */
/* ----------------------------------------------------------------------- */

/* FFTN_Device: the unnormalised forward real-to-complex 3-D transform
 * (cufftExecD2Z) of a real [Nx][Ny][Nz] device array (z fastest) into the
 * [Nx][Ny][Mz] complex layout.  in and out must not overlap. */
ns3d_status ns3d_fft_r2c(ns3d_solver* h, const double* in, ns3d_complex* out);

/* iFFTN_Device: complex-to-real 3-D transform (cufftExecZ2D) followed by the
 * 1/(Nx Ny Nz) scale (scale_double).  As cuFFT does, only the Hermitian part
 * of the kz = 0 and kz = Nz/2 planes contributes.  `in` is not modified
 * (cuFFT's Z2D may overwrite its input); the handle's scratch is used. */
ns3d_status ns3d_fft_c2r(ns3d_solver* h, const ns3d_complex* in, double* out);

/* The same transform without the scale: iFFTN_Device(source, destination)
 * (Source/math_support.cu:314-322), which runs cufftExecZ2D alone. */
ns3d_status ns3d_fft_c2r_unscaled(ns3d_solver* h, const ns3d_complex* in, double* out);

/* ----------------------------------------------------------------------- */
/* diagnostics (Source/math_support.cu:720-806, Source/divergence.cu:8-31)    */
/* ----------------------------------------------------------------------- */

/* Synchronous.  energy = sum 0.5 (uy^2 + uz^2) dx dy over the physical grid
 * (get_kinetic_energy), dissipation = the reference's central-difference
 * sum (get_dissipation), div_max = max |i k . u_hat| (solve_divergence with
 * dt = 1).  Returns NS3D_ERR_NONFINITE if any of them is not finite.  Any
 * output pointer may be null. */
ns3d_status ns3d_diagnostics(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                             const ns3d_complex* uz, double* energy, double* dissipation,
                             double* div_max);

/* ----------------------------------------------------------------------- */
/* filters, curl and the main loop's diagnostics (Source/math_support.cu:    */
/* 680-717, 819-987; Source/NS3D_periodic.cu:1291-1452, 1853;               */
/* Source/Shapiro_test.cu:8-50)                                             */
/* ----------------------------------------------------------------------- */

/* Helmholz_Fourier_Filter's spectral step: f = u / (1 + eps^2 |k|^2), with
 * signed x/y wave numbers (Nyquist -N/2) and the stored z index.  Follow it
 * with ns3d_fft_c2r for the filtered physical field, as the reference does.
 * f may alias u.  Asynchronous on the handle's stream. */
ns3d_status ns3d_helmholtz_filter(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                                  const ns3d_complex* uz, double eps, ns3d_complex* fx,
                                  ns3d_complex* fy, ns3d_complex* fz);

/* CutOff_Fourier_Filter's spectral step as main launches it (Mz in its Nz
 * slot): keep the modes with m^2/Nx^2 + n^2/Ny^2 + q^2/Mz^2 <= radius^2,
 * zero the rest.  f may alias u.  Asynchronous. */
ns3d_status ns3d_cutoff_filter(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                               const ns3d_complex* uz, double radius, ns3d_complex* fx,
                               ns3d_complex* fy, ns3d_complex* fz);

/* get_curl on physical fields [Nx][Ny][Nz]: second-order central differences
 * with periodic wrap, including the reference's rot_y term
 * 0.5 (uz(j+1) - ux(j-1)) / dx (it mixes uz and ux; kept so that the numbers
 * match the reference's output).  r must not alias u.  Asynchronous. */
ns3d_status ns3d_curl(ns3d_solver* h, const double* ux, const double* uy, const double* uz,
                      double* rx, double* ry, double* rz);

/* One line of time_dependant.dat (Source/NS3D_periodic.cu:1324-1452) from
 * the spectral state, into host rec[NS3D_RECORD_COLUMNS]:
 *   rec[0]      total_time (the caller's TotalTime; main adds dt twice per
 *               step before writing it)
 *   rec[1..21]  at the three probe points IN(Nx/2-4,Ny/2-3,Nz/2-2),
 *               IN(Nx/3,Ny/3,Nz/3), IN(Nx/8,Ny/8,Nz/8): ux uy uz, the curl
 *               of ns3d_curl, then energy / dissipation / energy-dissipation/Re
 *   rec[22..28] the same at the second point for the velocity cut-off
 *               filtered at radius 0.1, then energy
 *   rec[29..49] Re/Im reads of the spectral state at the reference's flat
 *               indices, with dissipation at rec[35].
 * energy and dissipation are those of ns3d_diagnostics.  The point values are
 * evaluated from the spectrum directly (no transforms): the same numbers as
 * the reference's transform-then-read, to rounding.  Synchronous; returns
 * NS3D_ERR_NONFINITE, with rec filled, when a column is not finite (main
 * prints "nans!" and carries on).  NS3D_ERR_BAD_ARG when the grid is too
 * small for the reference's indices. */
#define NS3D_RECORD_COLUMNS 50
ns3d_status ns3d_record(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                        const ns3d_complex* uz, double total_time, double Re, double* rec);

/* The sums of calculate_energy_spectrum as main calls it (Source/
 * NS3D_periodic.cu:1853, Mz in its Nz slot): E[n] = sum over j < Nx/2,
 * k < Ny/2, l < Mz with j + k + l = n of |u_hat|^2 / (Nx Ny Mz)^2, summed over
 * the three components; nbins must be Nx/2 + Ny/2 + Nz/2 + 1.  Host E.
 * Synchronous.  ns3d_write_energy_spectrum_host writes Ek.dat from it. */
ns3d_status ns3d_energy_spectrum(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                                 const ns3d_complex* uz, double* E, int nbins);

/* Shapiro's exact Beltrami solution (Initial_Shapiro, Source/
 * NS3D_periodic.cu:807-829) at time t, transformed to spectral fields.  The
 * formula is the reference's for a 2 pi box.  Asynchronous. */
ns3d_status ns3d_shapiro_state(ns3d_solver* h, double t, double Re, ns3d_complex* ux,
                               ns3d_complex* uy, ns3d_complex* uz);

/* Shapiro_test_case on physical fields: min_max[0..1] = min and max over
 * the grid of |u - u_exact(t)|; the reference returns the max.  Synchronous. */
ns3d_status ns3d_shapiro_error_physical(ns3d_solver* h, const double* ux, const double* uy,
                                        const double* uz, double t, double Re, double* min_max);

/* The same from the spectral state (inverse transform first): err = max. */
ns3d_status ns3d_shapiro_error(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                               const ns3d_complex* uz, double t, double Re, double* err);

/* Host-only writers of the two diagnostic files.  A series is the main
 * loop's time_dependant.dat: ns3d_series_open truncates the file (fopen
 * "w"), each ns3d_series_write appends one line of ncols "%le" fields
 * separated by single spaces, ns3d_series_close flushes and closes. */
typedef struct ns3d_series ns3d_series;
ns3d_status ns3d_series_open(const char* path, ns3d_series** out);
ns3d_status ns3d_series_write(ns3d_series* s, const double* rec, int ncols);
ns3d_status ns3d_series_close(ns3d_series* s);

/* Ek.dat as calculate_energy_spectrum writes it from E of
 * ns3d_energy_spectrum: per bin "%i %.16le %.16le" of n, E[n]/2 and
 * 0.25 n^(-5/3) (inf at n = 0); bins no mode reaches print "0 0 0". */
ns3d_status ns3d_write_energy_spectrum_host(const char* path, int Nx, int Ny, int Nz,
                                            const double* E);

/* Times the five pass kernels of one RHS evaluation (the first RK3 stage:
 * inv_x, inv_y, z, fwd_y, fwd_x; u is read, handle scratch is written) with
 * CUDA events on the handle's stream, `reps` times after one warm-up, and
 * stores the mean milliseconds per launch in ms[0..4].  Synchronous.  No
 * reference counterpart: it serves the roofline report. */
ns3d_status ns3d_profile_passes(ns3d_solver* h, const ns3d_complex* ux, const ns3d_complex* uy,
                                const ns3d_complex* uz, double dt, double Re, int reps,
                                double* ms);

/* Autotuner of the pass tiles (no reference counterpart).  Each of the four
 * pipelined pass families -- 0 inv_x, 1 inv_y, 2 fwd_y, 3 fwd_x -- has up to
 * five tiles:
 *   0  the default: 16 points per thread for powers of two, 12 for multiples
 *      of 3, with its radix schedule (16.16 at 256, 16.16.2 at 512, ...);
 *   1  the alternative, for extents >= 32 (powers of two) or >= 48 (multiples
 *      of 3): 8 or 6 points per thread (twice the lines per CTA, half the
 *      registers and prefetch buffers) and their schedule (8.8.4 at 256);
 *   2  inv_y only, y extents from 48: the bulk-copy form, where
 *      one thread per CTA loads each field's box of lines into shared memory
 *      with a tensor copy (TMA) instead of every thread copying its own
 *      samples (the tangent form and the FP32 mode run the per-thread copies
 *      at the same points per thread);
 *   3, 4  inv_x, inv_y and fwd_y: tile 0's or tile 1's points per thread with
 *      the radices in reverse order (4.8.8 instead of 8.8.4 at 256, 2.16.16
 *      instead of 16.16.2 at 512), where that order differs.
 * Different tiles change the order of the floating-point operations of the
 * transforms, so results agree to round-off, not bit for bit.  The tiles are
 * per precision; a new handle starts with the defaults. */
#define NS3D_TILE_FAMILIES 4
#define NS3D_TILES_PER_FAMILY 5
#define NS3D_TUNE_TIMES 20
ns3d_status ns3d_get_tiles(const ns3d_solver* h, int* tiles);
/* NS3D_ERR_BAD_ARG for a tile the family or the extent lacks.  Synchronises
 * the handle's stream. */
ns3d_status ns3d_set_tiles(ns3d_solver* h, const int* tiles);
/* Times every family with each of its tiles on the handle's own scratch
 * (`reps` launches after one warm-up, CUDA events, as ns3d_profile_passes;
 * the state is not touched), keeps the fastest where it is at least 2%
 * faster than the default, and applies the choice.  Choices are cached per
 * process and device for (Nx, Ny, Nz, batch, precision): unless `force`, a
 * cached choice is applied without timing.  ms (NS3D_TUNE_TIMES = 20
 * doubles, may be NULL) receives the mean ms of tile t of family f at
 * ms[5 f + t] (-1: the family has no such tile here, or it was not timed).
 * Synchronous. */
ns3d_status ns3d_autotune(ns3d_solver* h, int reps, int force, double* ms);

/* ----------------------------------------------------------------------- */
/* precision mode                                                           */
/* ----------------------------------------------------------------------- */

/* No reference counterpart (the reference is FP64 throughout).  In the FP32
 * mode the nonlinear term is formed in single precision: the inverse and
 * forward transforms of the RHS pipeline and the physical-space products
 * run on float2 scratch, while the state, the forcing, the projection,
 * diffusion and RK combination of the update, and every diagnostic stay in
 * FP64 (the state is read in FP64 and rounded once per stage; the FP32
 * products are widened before the update).  It applies to every stepper of
 * the handle (RK3, Euler, RHS, the tangent steppers) until changed; the
 * plain transforms (ns3d_fft_*) and diagnostics stay FP64.  The default is
 * FP64, the reference's arithmetic.  Synchronises the handle's stream. */
#define NS3D_PRECISION_FP64 0
#define NS3D_PRECISION_FP32 1
ns3d_status ns3d_set_precision(ns3d_solver* h, int precision);
int ns3d_get_precision(const ns3d_solver* h);

/* ----------------------------------------------------------------------- */
/* ensembles: many independent instances of one grid stepped together       */
/* ----------------------------------------------------------------------- */

/* No reference counterpart (the reference steps one field per process).  An
 * ensemble holds `batch` instances of one Nx x Ny x Nz grid and box, each
 * with its own dt and Re, and advances all of them with the launches of one
 * RK3 step (15 kernels for the whole batch, replayed from a captured CUDA
 * graph), so small grids are not bound by launch latency.  Fields are
 * [batch][Nx][Ny][Nz/2+1] per component: instance b of component c starts at
 * u_c + b * Nx*Ny*(Nz/2+1).  Each instance's step is RK3_SSP exactly (the same
 * arithmetic as ns3d_rk3_step, bit for bit).  Several ensembles of different
 * grids overlap on the GPU when they run on different streams. */
typedef struct ns3d_ensemble ns3d_ensemble;

ns3d_status ns3d_ensemble_create(int batch, int Nx, int Ny, int Nz, double Lx, double Ly,
                                 double Lz, ns3d_ensemble** out);
ns3d_status ns3d_ensemble_destroy(ns3d_ensemble* e);
ns3d_status ns3d_ensemble_set_stream(ns3d_ensemble* e, void* stream);
const char* ns3d_ensemble_last_error(const ns3d_ensemble* e);
size_t ns3d_ensemble_device_bytes(const ns3d_ensemble* e);
/* One instance-sized forcing, shared by every instance (as ns3d_set_forcing). */
ns3d_status ns3d_ensemble_set_forcing(ns3d_ensemble* e, const ns3d_complex* fx,
                                      const ns3d_complex* fy, const ns3d_complex* fz);
/* ns3d_set_precision for the whole ensemble. */
ns3d_status ns3d_ensemble_set_precision(ns3d_ensemble* e, int precision);
/* ns3d_autotune / ns3d_get_tiles / ns3d_set_tiles for the ensemble's batch. */
ns3d_status ns3d_ensemble_autotune(ns3d_ensemble* e, int reps, int force, double* ms);
ns3d_status ns3d_ensemble_get_tiles(const ns3d_ensemble* e, int* tiles);
ns3d_status ns3d_ensemble_set_tiles(ns3d_ensemble* e, const int* tiles);
/* Host arrays of `batch` entries; synchronous.  Required before stepping. */
ns3d_status ns3d_ensemble_set_params(ns3d_ensemble* e, const double* dt, const double* Re);
/* nsteps RK3 steps of every instance, in place.  Asynchronous. */
ns3d_status ns3d_ensemble_rk3_steps(ns3d_ensemble* e, ns3d_complex* ux, ns3d_complex* uy,
                                    ns3d_complex* uz, int nsteps);
/* ns3d_diagnostics' energy and dissipation per instance (host arrays of
 * `batch` entries).  Synchronous. */
ns3d_status ns3d_ensemble_diagnostics(ns3d_ensemble* e, const ns3d_complex* ux,
                                      const ns3d_complex* uy, const ns3d_complex* uz,
                                      double* energy, double* dissipation);

/* ----------------------------------------------------------------------- */
/* request server: tangent integrations with continuous batching            */
/* ----------------------------------------------------------------------- */

/* No reference counterpart.  A request asks for the tangent (Jacobian-vector
 * product) integration that NSCallMatrixVector_exponential performs
 * (Source/NS3D_periodic.cu:444-470: RK3_SSP_UV steps, Source/RK_time_step.cu:
 * 342-355) on an N^3 2 pi box: base state u = Kolmogorov laminar profile
 * (Re/16) sin(4y) x plus a seeded 1e-3 perturbation, forcing sin(4y) x,
 * tangent v = a seeded unit perturbation (both pure-imaginary,
 * divergence-free, |k|^-2 on 1 <= |k| <= 8, made on the device from `seed`;
 * ns3d_request_fields gives the same fields on a single-grid handle),
 * steps = ceil(T / dt) with dt = 0.3 (2 pi / N) / (Re / 16).  The result is
 * |v(T)| (L2 over the stored half spectrum) and, with keep = 1, v(T).
 *
 * The server reserves, per grid N, as many instance slots as hbm_fraction of
 * the free device memory (split evenly over the grids) holds, at most
 * capacity[i] when `capacity` is given (hbm_fraction outside (0, 1) with a
 * capacity: exactly capacity[i]), and serves requests with continuous
 * batching: whenever a grid's step finishes, finished requests leave,
 * requests that have arrived take the free slots (first come, first served
 * per grid), and the next step runs all active slots in one batch.  Grids
 * run on their own streams and overlap.  A result does not depend on the mix
 * it ran in (bit for bit).  Times are seconds on the server clock, which
 * starts at the first ns3d_server_run. */
typedef struct ns3d_server ns3d_server;
typedef struct ns3d_request {
  int N;
  double Re, T;
  unsigned long long seed;
  double arrival; /* server-clock seconds; requests are submitted in arrival order */
  int keep;       /* keep v(T) for ns3d_server_result_field */
} ns3d_request;
typedef struct ns3d_result {
  long long id;
  int N;
  double Re, T;
  int steps;
  double arrival, admitted, done; /* -1: not yet */
  double v_norm;
  int status; /* -1 pending, NS3D_OK, NS3D_ERR_NONFINITE, NS3D_ERR_CANCELLED */
} ns3d_result;

/* A request that brings its own fields: the work a Newton-Krylov,
 * BiCGStab(L) or Arnoldi caller hands out with every matrix-vector product
 * (NSCallMatrixVector_exponential, Source/NS3D_periodic.cu:444-470, and the
 * Jacobian maps Source/Arnoldi/Newton.cu:40-47 calls): `steps` RK3_SSP_UV
 * steps of the base state u and tangent v with time step dt and Reynolds
 * number Re, under the grid's forcing (ns3d_server_set_forcing; sin(4y) x
 * unless set).  u_in and v_in are read when the request is admitted; v_out
 * (and u_out, unless null) are written when it completes, before its status
 * leaves -1.  The buffers hold [N][N][N/2+1] complex values each, in device
 * memory or in host memory cudaMemcpyAsync can read and write (pinned), and
 * must stay valid until the request is done; v_out may be v_in and u_out
 * u_in.  arrival < 0 stands for the server clock at submission (at least the
 * previous request's arrival).  The result's T is steps * dt. */
typedef struct ns3d_field_request {
  int N;
  double Re, dt;
  int steps;
  const ns3d_complex* u_in[3];
  const ns3d_complex* v_in[3];
  ns3d_complex* u_out[3];
  ns3d_complex* v_out[3];
  double arrival;
} ns3d_field_request;

ns3d_status ns3d_server_create(const int* Ns, int nN, const int* capacity, double hbm_fraction,
                               ns3d_server** out);
ns3d_status ns3d_server_destroy(ns3d_server* s);
const char* ns3d_server_last_error(const ns3d_server* s);
ns3d_status ns3d_server_capacity(const ns3d_server* s, int N, int* slots);
/* ns3d_set_precision for every grid of the server (between runs). */
ns3d_status ns3d_server_set_precision(ns3d_server* s, int precision);
/* ns3d_autotune for every grid at its full slot count, between runs.  Tuned
 * grids give results that agree with the single-grid API to round-off; with
 * the default tiles (no call) they agree bit for bit. */
ns3d_status ns3d_server_autotune(ns3d_server* s, int reps);
/* JVP steps the grid N has launched so far, summed over its active slots
 * (the work done, finished requests or not). */
ns3d_status ns3d_server_stats(const ns3d_server* s, int N, long long* instance_steps);
/* Queues n requests (ids first_id .. first_id + n - 1). */
ns3d_status ns3d_server_submit(ns3d_server* s, const ns3d_request* r, int n, long long* first_id);
/* Queues n requests that carry their own fields (ns3d_field_request); they
 * share the ids, the arrival order and the slots of ns3d_server_submit's. */
ns3d_status ns3d_server_submit_fields(ns3d_server* s, const ns3d_field_request* r, int n,
                                      long long* first_id);
/* Forcing of grid N's base flow (device memory, [N][N][N/2+1] each), for the
 * requests admitted from now on; between runs. */
ns3d_status ns3d_server_set_forcing(ns3d_server* s, int N, const ns3d_complex* fx,
                                    const ns3d_complex* fy, const ns3d_complex* fz);
/* Cancels a request that has not finished: a queued request never starts, an
 * admitted one leaves its slot at its grid's next step boundary, and the slot
 * goes to the next arrival.  Its status becomes NS3D_ERR_CANCELLED (its
 * output fields are not written).  The one call that may come from another
 * host thread while ns3d_server_run runs.  NS3D_ERR_BAD_ARG for an unknown
 * or finished request. */
ns3d_status ns3d_server_cancel(ns3d_server* s, long long id);
/* Runs the engine like ns3d_server_run but returns as soon as request `id`
 * is done (other requests progress meanwhile and keep their slots). */
ns3d_status ns3d_server_run_until(ns3d_server* s, long long id, double max_seconds,
                                  int* completed);
/* Runs the engine on the calling thread until every submitted request is
 * done or max_seconds have passed (then nothing more is admitted or launched
 * and the steps in flight are finished; unfinished requests keep their slots
 * for the next call); *completed = requests finished in this call. */
ns3d_status ns3d_server_run(ns3d_server* s, double max_seconds, int* completed);
/* All requests so far, in id order (*n = their count; up to cap copied). */
ns3d_status ns3d_server_results(const ns3d_server* s, ns3d_result* out, int cap, int* n);
ns3d_status ns3d_server_result_field(const ns3d_server* s, long long id, ns3d_complex* vx,
                                     ns3d_complex* vy, ns3d_complex* vz);
/* The request's initial (u, v) on a cubic single-grid handle, and its step count. */
ns3d_status ns3d_request_fields(ns3d_solver* h, double Re, unsigned long long seed,
                                ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                                ns3d_complex* vx, ns3d_complex* vy, ns3d_complex* vz);
int ns3d_request_steps(int N, double Re, double T);

/* ----------------------------------------------------------------------- */
/* allocation-free nonlinear term                                           */
/* ----------------------------------------------------------------------- */

/* Largest grid the allocation-free entry point accepts, as complex points
 * per field (Nx * Ny * (Nz/2+1)); 64^3 fits.  The fixed scratch behind it is
 * NS3D_NOALLOC_SCRATCH_BYTES of device memory. */
#define NS3D_NOALLOC_MAX_POINTS 135168
#define NS3D_NOALLOC_SCRATCH_BYTES 33005568

/* No counterpart in the reference (which allocates its scratch in
 * init_dealiasing).  Same result as ns3d_convolution, but without a handle and
 * without allocating device memory: for callers that reserve all device
 * memory up front in their own pool, that keep no handle between calls, or
 * that cannot afford the synchronisation of cudaMalloc/cudaFree.  The
 * scratch is a fixed array compiled into the library (about 33 MB per GPU,
 * held from the first call on a device until the process exits).  The first
 * call on each device looks up that array's device address and uploads the
 * grid's twiddle and mask tables; make that first call before capturing the
 * stream.  Later calls with the same grid and box reuse the tables; a call
 * whose grid or box differs from the previous call's on that device uploads
 * new tables and synchronises `stream`, which is refused (NS3D_ERR_BAD_ARG,
 * nothing launched) while `stream` is being captured.  All calls on a device
 * share the array, so calls that overlap on the GPU race: serialise them
 * (one stream, one host thread).  Runs on `stream` (cudaStream_t, 0 for the
 * legacy default stream) on the current device.  Returns NS3D_ERR_BAD_ARG
 * when Nx*Ny*(Nz/2+1) > NS3D_NOALLOC_MAX_POINTS (nothing is launched),
 * NS3D_ERR_UNSUPPORTED for an extent without a compiled plan. */
ns3d_status ns3d_convolution_noalloc(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                                     const ns3d_complex* ux, const ns3d_complex* uy,
                                     const ns3d_complex* uz, ns3d_complex* Qx, ns3d_complex* Qy,
                                     ns3d_complex* Qz, void* stream);

/* ----------------------------------------------------------------------- */
/* Krylov eigen-analysis: Arnoldi factorisation and implicit restart        */
/* (Source/Arnoldi/Arnoldi_Driver.cu, Source/Arnoldi/QR_Shifts.cpp,          */
/*  Source/Arnoldi/Implicit_restart_Arnoldi.cu:531-563)                      */
/* ----------------------------------------------------------------------- */

typedef struct ns3d_krylov ns3d_krylov;

/* Matrix-vector map out = A in on device vectors of the workspace length n;
 * the same type as the reference's user_map_vector
 * (Source/Arnoldi/Matrix_Vector_emulator.h:11), so its NSCall* adapters can
 * be passed unchanged.  The map must not write `in`, and its work must be
 * complete when it returns (or be ordered before later work on the
 * workspace stream: same stream, or a blocking stream while the workspace
 * runs on the legacy default stream). */
typedef void (*ns3d_user_map_vector)(void* user, void* in, void* out);

/* Workspace for Krylov vectors of length n >= 2 and bases of up to
 * 2 <= m_max <= 200 columns on the current device: the vectors v, w and the
 * reduction buffers of Arnoldi_driver (its vec_v_d, vec_w_d, vec_c_d,
 * vec_h_d arguments) plus pinned host staging.  Work runs on the legacy
 * default stream until ns3d_krylov_set_stream. */
ns3d_status ns3d_krylov_create(int64_t n, int m_max, ns3d_krylov** out);
ns3d_status ns3d_krylov_destroy(ns3d_krylov* kr);
ns3d_status ns3d_krylov_set_stream(ns3d_krylov* kr, void* stream);
const char* ns3d_krylov_last_error(const ns3d_krylov* kr);

/* Arnoldi_driver (Source/Arnoldi/Arnoldi_Driver.cu:29-120): extends
 * A V = V H + f e_k^T to m columns (k = 0 starts from f).  V: DEVICE,
 * n x m column-major (leading dimension n); H: HOST, m x m column-major
 * (leading dimension m; columns k+1..m-1 are overwritten whole, H(k+1,k) and
 * for k = 0 also H(0,0) are set); f: DEVICE, length n, the residual on entry
 * and exit.  Classical Gram-Schmidt with iterative reorthogonalisation,
 * tolerance 5e-12, at most 13 passes per column; a column that reaches the
 * limit is counted (ns3d_krylov_stats) and the factorisation goes on, as in
 * the reference.  Synchronous.  NS3D_ERR_BAD_ARG when k = 0 and
 * ||f|| < 1e-15 (the reference exits), NS3D_ERR_NONFINITE when a norm, dot
 * product or H entry is not finite (the reference checks element 0 of v, w
 * and f for NaN and exits). */
ns3d_status ns3d_arnoldi(ns3d_krylov* kr, ns3d_user_map_vector Axb, void* user, double* V,
                         double* H, double* f, int k, int m);

/* Largest number of reorthogonalisation passes a column of the last
 * ns3d_arnoldi call took, how many columns reached the pass limit, and how
 * many kernels the driver itself launched (the map's launches not
 * included).  Any output pointer may be null. */
ns3d_status ns3d_krylov_stats(const ns3d_krylov* kr, int* max_passes, int* limit_hits,
                              int64_t* launches);

/* HOST ONLY (no GPU needed).  QR_shifts (Source/Arnoldi/QR_Shifts.cpp:46-72):
 * for j = m, m-1, ... while j > k, one shifted QR step of H with the shift
 * eig[j-1] (a double step with (H - Re)^2 + Im^2 when |Im| > 1e-15, which
 * also consumes eig[j-2]); Q (m x m, column-major, output) accumulates the
 * orthogonal factors, H (m x m, column-major) becomes Q^T H Q with the
 * entries below the subdiagonal zeroed, *ko = the final j.  The Q factors
 * are Householder QR factors with LAPACK's conventions (dgeqrf + dormqr,
 * Source/Arnoldi/LAPACK_routines.cpp:289-345).  eig_re/eig_im: the m Ritz
 * values in the order the shifts are taken from (select_shifts). */
ns3d_status ns3d_qr_shifts(int k, int m, double* Q, double* H, const double* eig_re,
                           const double* eig_im, int* ko);

/* Restart update (Source/Arnoldi/Implicit_restart_Arnoldi.cu:544-563) with
 * q = Q(:,k0), hl = H(k0,k0-1), ql = Q(m-1,k0-1):  f = hl V q + ql f;
 * Q(:, k0..m-1) := the identity columns (in the host array, as the
 * reference does); V = V Q in place (columns k0.. keep their values).
 * V, f: DEVICE; Q, H: HOST m x m column-major; 1 <= k0 < m.  *f_norm (may be
 * null) receives ||f|| before the update (the Ritz-estimate scale, :547).
 * One pass over V.  Synchronous. */
ns3d_status ns3d_ira_restart(ns3d_krylov* kr, double* V, double* f, double* Q, const double* H,
                             int k0, int m, double* f_norm);

/* Device time per launch (CUDA events on the workspace stream, averaged over
 * `reps` after one warm-up) of the three basis kernels on the first `ncols`
 * columns of V (device, n x ncols, leading dimension n) and the vector x:
 * ms[0] the dot products V^T x (with their fixed-order reduction), ms[1]
 * y = x - V c, ms[2] the restart pass over V with identity coefficients (V
 * and x are not changed).  For roofline reports. */
ns3d_status ns3d_krylov_profile(ns3d_krylov* kr, const double* V, int ncols, const double* x,
                                int reps, double* ms);

/* W = V C: W(:, j) = sum_c V(:, c) C(c, j) for j < p, c < m; V and W DEVICE
 * n x m and n x p column-major (leading dimension n, W not overlapping V),
 * C HOST m x p column-major.  The basis products of the final eigenvector
 * stage of the implicit restart (V1 = V Q_Schur and the eigenvector
 * combinations, Source/Arnoldi/Implicit_restart_Arnoldi.cu:255-330,640-643):
 * one pass over V, the outputs kept in registers.  Synchronous. */
ns3d_status ns3d_krylov_combine(ns3d_krylov* kr, const double* V, int m, const double* C, int p,
                                double* W);

/* BiCGStabL (Source/Arnoldi/BiCGStabL.cu:18-185): solves A x = rhs with
 * BiCGStab(L), 1 <= L <= 16, x (device, length n) the initial guess on entry
 * and the solution on exit, rhs (device) unchanged.  *tol and *iter are the
 * reference's in/out arguments: the relative residual ||b - A x|| / ||b||
 * to reach and the iteration cap on entry; the residual reached and the
 * index of the last iteration on exit.  *flag receives the reference's
 * outcome: 0 converged, 1 not converged, -1 rho = 0, -3 NaN.  Synchronous
 * (one host read per inner product, as the reference). */
ns3d_status ns3d_bicgstabl(ns3d_krylov* kr, int L, ns3d_user_map_vector Axb, void* user,
                           double* x, const double* rhs, double* tol, int* iter, int* flag);

/* Newton (Source/Arnoldi/Newton.cu:9-98): damped (0.8) Newton iteration for
 * F(x) = 0 with BiCGStab(6) linear solves J delta = -F(x), delta starting
 * from the reference's initial vector and carried between iterations.
 * `residual` maps x to F(x) and, as the reference's NSCallRHS_reduced does,
 * may record x as the point `jacobian` linearises about.  *tol: the residual
 * norm to reach (on success it receives ||delta|| of the last step); *iter:
 * the iteration cap on entry, the iterations run on exit.  *flag: 0
 * converged, 1 not converged, 2 a linear solve failed with
 * *linsolve_flag (the reference prints and exits there).  n >= 5. */
ns3d_status ns3d_newton(ns3d_krylov* kr, ns3d_user_map_vector jacobian, void* jacobian_user,
                        ns3d_user_map_vector residual, void* residual_user, double* x,
                        double* tol, int* iter, double tol_linsolve, int iter_linsolve,
                        int* flag, int* linsolve_flag);

/* Built-in maps for ns3d_arnoldi.  Each finishes its work before returning
 * and, on failure, records the first non-OK status in `status` and fills
 * `out` with NaN so the driver stops with NS3D_ERR_NONFINITE. */
typedef struct ns3d_map_context {
  ns3d_solver* solver;
  ns3d_complex* ux; /* base flow (advanced in place by the exponential map) */
  ns3d_complex* uy;
  ns3d_complex* uz;
  ns3d_complex* vx; /* tangent fields, scratch of the exponential map */
  ns3d_complex* vy;
  ns3d_complex* vz;
  double dt, Re, tau;
  int steps;
  int status; /* NS3D_OK until a call fails */
} ns3d_map_context;

/* user = ns3d_map_context*: out = J(u) in - in/tau (tau <= 0: no shift) on
 * reduced vectors: NSCallMatrixVector_reduced[_Newton_Globalization]
 * (Source/NS3D_periodic.cu:340-385) through ns3d_matvec_reduced. */
void ns3d_map_linearised(void* user, void* in, void* out);

/* user = ns3d_map_context*: NSCallRHS_reduced (Source/NS3D_periodic.cu:
 * 415-441): in -> u (the context's base flow, reduced unpacking), out =
 * RHS(u) = -P.Q(u) - |k|^2/Re u + f packed, with the context's v fields as
 * scratch.  Setting u is what lets a linearised map sharing the same u
 * serve as the Newton Jacobian. */
void ns3d_map_rhs(void* user, void* in, void* out);

/* user = ns3d_map_context*: in -> v (reduced unpacking), `steps` Heun tangent
 * steps of (u, v) with ns3d_jvp_steps, v -> out: NSCallMatrixVector_exponential
 * (Source/NS3D_periodic.cu:444-470).  As in the reference, the base flow u
 * advances with every call.  The reference packs with the full-length
 * kernels of a 3*Nc vector while its IRA call passes the reduced length
 * 3*Nc-3 (Source/NS3D_periodic.cu:1717); this map uses the reduced packing
 * consistently. */
void ns3d_map_exponential(void* user, void* in, void* out);

/* The exponential map served by a request server: what ns3d_map_exponential
 * computes (in -> v, `steps` RK3_SSP_UV steps of (u, v), v -> out; the base
 * flow u advances with every call), with the steps run by `server` as a
 * field request (ns3d_server_submit_fields + ns3d_server_run_until), so the
 * matrix-vector products of a Krylov driver share the device with the
 * server's other requests.  `solver` (a handle of the server's grid N)
 * packs and unpacks the reduced vectors; with the server's default tiles and
 * the same forcing the result equals ns3d_map_exponential's bit for bit. */
typedef struct ns3d_served_map_context {
  ns3d_map_context map; /* solver, base flow u, tangent v, dt, Re, steps; status */
  ns3d_server* server;
  long long requests;   /* out: requests served so far */
} ns3d_served_map_context;
void ns3d_map_exponential_served(void* user, void* in, void* out);

/* Shift-invert maps of the matrix-exponent IRA
 * (Implicit_restart_Arnoldi_GPU_data_Matrix_Exponent,
 * Source/Arnoldi/Implicit_restart_Arnoldi.cu:456-742, driven by
 * Source/NS3D_periodic.cu:1650-1711).  E below is `map.steps` implicit
 * tangent steps (ns3d_implicit_tangent_step with map.dt and map.Re) of a
 * reduced vector about the base flow map.u*, which stays fixed; map.v* are
 * their scratch.  A reduced vector has n = ns3d_krylov_length(map.solver)
 * entries; a rotated vector has 2n, its real half first. */
typedef struct ns3d_shift_invert_context {
  ns3d_map_context map; /* solver, base flow, tangent scratch, dt, Re, steps; status */
  double shift_real;    /* sigma (shift_real) */
  double rotate_angle;  /* theta: the rotated maps shift by sigma e^{i theta} */
  int L;                /* BiCGStab(L) order of the inverse maps (BiCG_L) */
  double tol;           /* their relative residual to reach (BiCG_tol) */
  int max_iter;         /* their iteration cap (BiCG_Iter) */
  int warm_start;       /* 0: every solve starts from x = 0; 1: from the contents
                           of `out`, as the reference's solve does */
  ns3d_krylov* inner;   /* workspace of the solves, length n (2n rotated); not the
                           workspace of the driver that calls the map */
  int last_flag;        /* out: BiCGStabL flag of the last solve */
  int last_iter;        /* out: its iteration index */
  double last_tol;      /* out: its relative residual */
  long long solves;     /* out: solves so far */
  long long inner_iter; /* out: their iterations, summed */
} ns3d_shift_invert_context;

/* user = ns3d_shift_invert_context*: out = E in - sigma*in on reduced
 * vectors: NSCallMatrixVector_exponential_reduced
 * (Source/NS3D_periodic.cu:473-500). */
void ns3d_map_exponential_shifted(void* user, void* in, void* out);

/* user = ns3d_shift_invert_context*, vectors of length 2n: with
 * (sr, si) = sigma (cos theta, sin theta),
 *   out_r = E in_r - sr*in_r + si*in_i,  out_i = E in_i - sr*in_i - si*in_r,
 * the real form of (E - sigma e^{i theta}) (in_r + i in_i):
 * NSCallMatrixVector_exponential_rotated_reduced
 * (Source/NS3D_periodic.cu:552-586). */
void ns3d_map_exponential_rotated(void* user, void* in, void* out);

/* user = ns3d_shift_invert_context*: out = (E - sigma)^{-1} in, solved with
 * ns3d_bicgstabl(inner, L, ns3d_map_exponential_shifted, ...) to `tol`:
 * Axb_exponent_invert (Source/NS3D_periodic.cu:506-548).  The reference
 * exits when the solve does not converge; here the map records
 * NS3D_ERR_NOT_CONVERGED in map.status (NS3D_ERR_NONFINITE for flag -3) and
 * fills out with NaN, so the calling driver stops. */
void ns3d_map_exponent_invert(void* user, void* in, void* out);

/* The same on rotated vectors with ns3d_map_exponential_rotated:
 * Axb_rotated_exponent_invert (Source/NS3D_periodic.cu:590-630). */
void ns3d_map_rotated_exponent_invert(void* user, void* in, void* out);

/* The reference's Krylov self-test operator (user_Ax_function,
 * Source/Arnoldi/Matrix_Vector_emulator.cu:10-36): out_i = in_{i+1} - 2 in_i
 * + in_{i-1} with periodic indices, then out_0 = 0. */
typedef struct ns3d_laplace_context {
  int64_t n;
  void* stream; /* cudaStream_t, 0 = legacy default stream */
  int status;
} ns3d_laplace_context;
void ns3d_map_laplace1d(void* user, void* in, void* out);

/* ----------------------------------------------------------------------- */
/* checkpoints in the reference's wire format (Source/file_operations.cu)   */
/* ----------------------------------------------------------------------- */

/* write_control_file_fourier / read_control_fourier
 * (Source/file_operations.cu:196-228, 104-191) for the handle's DEVICE
 * fields: one line per mode of [Nx][Ny][Mz], "%.16le" x 6 (Re, Im of ux, uy,
 * uz).  Loading accepts the handle's own size or a coarser grid with the
 * same aspect ratios, up-sampled the reference's way (see
 * ns3d_read_control_fourier_host).  Synchronous. */
ns3d_status ns3d_save_control_fourier(ns3d_solver* h, const char* path, const ns3d_complex* ux,
                                      const ns3d_complex* uy, const ns3d_complex* uz);
ns3d_status ns3d_load_control_fourier(ns3d_solver* h, const char* path, ns3d_complex* ux,
                                      ns3d_complex* uy, ns3d_complex* uz);

/* write_control_file / read_control_file (Source/file_operations.cu:4-45):
 * the physical velocity, one line per point of [Nx][Ny][Nz],
 * "%.16le %.16le %.16le".  Save transforms the spectral DEVICE fields to
 * physical space (iFFTN_Device with the 1/N scale, as main does before
 * writing); load reads the physical field and transforms it back (FFTN).
 * Synchronous. */
ns3d_status ns3d_save_control_file(ns3d_solver* h, const char* path, const ns3d_complex* ux,
                                   const ns3d_complex* uy, const ns3d_complex* uz);
ns3d_status ns3d_load_control_file(ns3d_solver* h, const char* path, ns3d_complex* ux,
                                   ns3d_complex* uy, ns3d_complex* uz);

/* ----------------------------------------------------------------------- */
/* host-only helpers (no GPU needed)                                        */
/* ----------------------------------------------------------------------- */

/* The Fourier checkpoint of HOST fields [Nx][Ny][Nz/2+1] (Nz is the
 * physical extent).  Reading a file of a coarser grid: its extents are
 * found from its line count with the target's ratios Nx/Ny and (2Mz-1)/Ny,
 * Ny_file = 4, 6, ... (get_control_fourier_size, Source/file_operations.cu:
 * 48-101; the reference searches without a bound and writes out of range
 * for a finer file, here the search stops at Ny and a finer or unmatched
 * file is NS3D_ERR_BAD_ARG); modes are placed at the same signed x / y
 * wavenumber and z index, the rest set to zero, and scaled by the integer
 * ratio Nx Ny (2Mz-1) / (Nx_f Ny_f (2Mz_f-1)) the reference computes.
 * Nx_file, Ny_file, Mz_file (may be null) receive the extents read. */
ns3d_status ns3d_write_control_fourier_host(const char* path, int Nx, int Ny, int Nz,
                                            const ns3d_complex* ux, const ns3d_complex* uy,
                                            const ns3d_complex* uz);
ns3d_status ns3d_read_control_fourier_host(const char* path, int Nx, int Ny, int Nz,
                                           ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                                           int* Nx_file, int* Ny_file, int* Mz_file);
/* The physical checkpoint of HOST fields [Nx][Ny][Nz]. */
ns3d_status ns3d_write_control_file_host(const char* path, int Nx, int Ny, int Nz, const double* ux,
                                         const double* uy, const double* uz);
ns3d_status ns3d_read_control_file_host(const char* path, int Nx, int Ny, int Nz, double* ux,
                                        double* uy, double* uz);

/* The 2/3 mask as a kz cut-off per (x, y) column: mode (j,k,l) is kept iff
 * l < qcut[j*Ny + k] (and (j,k,l) != 0), evaluated with the arithmetic of
 * build_mask_matrix (Source/math_support.cu:471-519) called with Mz as Nz.
 * Returns NS3D_ERR_BAD_ARG if the mask is not a kz-prefix in some column. */
ns3d_status ns3d_mask_cutoff(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                             uint16_t* qcut);

/* Twiddle table tw[2e] = cos(2 pi e/N), tw[2e+1] = sin(2 pi e/N), e < N. */
ns3d_status ns3d_twiddles(int N, double* tw);

#ifdef __cplusplus
}
#endif

#endif /* NS3D_H_ */
