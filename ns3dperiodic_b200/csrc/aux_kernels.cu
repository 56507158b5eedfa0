#include "aux_kernels.cuh"

namespace ns3d {

__global__ void forcing_scan_kernel(const double2* __restrict__ fx, const double2* __restrict__ fy,
                                    const double2* __restrict__ fz, long long n, int cap,
                                    int* __restrict__ count, int* __restrict__ idx,
                                    double2* __restrict__ val) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 a = fx[i], b = fy[i], c = fz[i];
    if (a.x != 0.0 || a.y != 0.0 || b.x != 0.0 || b.y != 0.0 || c.x != 0.0 || c.y != 0.0) {
      const int p = atomicAdd(count, 1);
      if (p < cap) {
        idx[p] = (int)i;
        val[3 * p + 0] = a;
        val[3 * p + 1] = b;
        val[3 * p + 2] = c;
      }
    }
  }
}

__global__ void pack_reduced_kernel(const double2* __restrict__ vx, const double2* __restrict__ vy,
                                    const double2* __restrict__ vz, long long n,
                                    double* __restrict__ vec, const double* __restrict__ vec_shift,
                                    double coef, const double* __restrict__ vec_shift2,
                                    double coef2) {
  const long long m = n - 1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
       i += (long long)gridDim.x * blockDim.x) {
    double a = vx[i + 1].y, b = vy[i + 1].y, c = vz[i + 1].y;
    if (vec_shift) {
      a -= coef * vec_shift[i];
      b -= coef * vec_shift[i + m];
      c -= coef * vec_shift[i + 2 * m];
    }
    if (vec_shift2) {
      a += coef2 * vec_shift2[i];
      b += coef2 * vec_shift2[i + m];
      c += coef2 * vec_shift2[i + 2 * m];
    }
    vec[i] = a;
    vec[i + m] = b;
    vec[i + 2 * m] = c;
  }
}

__global__ void unpack_reduced_kernel(const double* __restrict__ vec, long long n,
                                      double2* __restrict__ vx, double2* __restrict__ vy,
                                      double2* __restrict__ vz) {
  const long long m = n - 1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (i == 0) {
      vx[0] = vy[0] = vz[0] = make_double2(0.0, 0.0);
    } else {
      vx[i] = make_double2(0.0, vec[i - 1]);
      vy[i] = make_double2(0.0, vec[i - 1 + m]);
      vz[i] = make_double2(0.0, vec[i - 1 + 2 * m]);
    }
  }
}

namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Hermitian part of the kz = 0 / kz = Nz/2 planes: what the complex-to-real
// transform actually sees (the imaginary parts of each z line's DC/Nyquist
// bins are dropped after the x and y passes).
__device__ __forceinline__ double2 herm(const double2* __restrict__ f, double2 v, long long mirror) {
  const double2 m = f[mirror];
  return make_double2(0.5 * (v.x + m.x), 0.5 * (v.y - m.y));
}

__device__ __forceinline__ double sq(double2 a) { return a.x * a.x + a.y * a.y; }

}  // namespace

// Parseval form of get_kinetic_energy / get_dissipation.  The central
// difference (u(x+h) - u(x-h))/h is i*2 sin(k h)/h in Fourier space, so both
// physical sums become weighted sums over the half spectrum (weight 1 on the
// kz = 0 and kz = Nz/2 planes, 2 elsewhere).  The per-direction factors
// 2 sin(2 pi q / N) / h come from tables built once per block in shared
// memory; each thread walks its modes with a stride of the whole grid and
// carries (j, k, l) along instead of dividing the flat index; the divergence
// maximum is taken over |div|^2 and rooted once per block.
__global__ void diag_partial_kernel(const double2* __restrict__ ux, const double2* __restrict__ uy,
                                    const double2* __restrict__ uz, DiagGeom g,
                                    double* __restrict__ partial) {
  __shared__ double tab_x[kDiagMaxExtent], tab_y[kDiagMaxExtent], tab_z[kDiagMaxExtent / 2 + 1];
  for (int q = threadIdx.x; q < g.Nx; q += blockDim.x)
    tab_x[q] = 2.0 * sinpi(2.0 * (double)q / g.Nx) / g.dx;
  for (int q = threadIdx.x; q < g.Ny; q += blockDim.x)
    tab_y[q] = 2.0 * sinpi(2.0 * (double)q / g.Ny) / g.dy;
  for (int q = threadIdx.x; q < g.Mz; q += blockDim.x)
    tab_z[q] = 2.0 * sinpi(2.0 * (double)q / g.Nz) / g.dz;
  __syncthreads();
  const int n = g.Nx * g.Ny * g.Mz;  // below 2^31 for every compiled grid
  const int S = gridDim.x * blockDim.x;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int l = i % g.Mz, k = (i / g.Mz) % g.Ny, j = (i / g.Mz) / g.Ny;
  const int Sl = S % g.Mz, Sk = (S / g.Mz) % g.Ny, Sj = (S / g.Mz) / g.Ny;
  double e = 0.0, d = 0.0, dv2 = 0.0;
  for (; i < n; i += S) {
    const int m = j < g.Nx / 2 ? j : j - g.Nx;  // reference signed index (Nyquist -> -N/2)
    const int nn = k < g.Ny / 2 ? k : k - g.Ny;
    double2 a = ux[i], b = uy[i], c = uz[i];
    // divergence (solve_divergence with dt = 1, reference wave numbers)
    {
      const double kx = g.kfx * (double)m, ky = g.kfy * (double)nn, kz = g.kfz * (double)l;
      const double re = -a.y * kx - b.y * ky - c.y * kz;
      const double im = a.x * kx + b.x * ky + c.x * kz;
      dv2 = fmax(dv2, re * re + im * im);
    }
    const bool edge = (l == 0) || (2 * l == g.Nz);
    double w = 2.0;
    if (edge) {
      w = 1.0;
      const int jm = j == 0 ? 0 : g.Nx - j;
      const int km = k == 0 ? 0 : g.Ny - k;
      const long long mi = ((long long)jm * g.Ny + km) * g.Mz + l;
      a = herm(ux, a, mi);
      b = herm(uy, b, mi);
      c = herm(uz, c, mi);
    }
    e += w * (sq(b) + sq(c));
    const double Dx = tab_x[j], Dy = tab_y[k], Dz = tab_z[l];
    // |d_b u_a| up to the common factor i: D_b * u_a
    const double2 xx = make_double2(Dx * a.x, Dx * a.y), yy = make_double2(Dy * b.x, Dy * b.y);
    const double2 zz = make_double2(Dz * c.x, Dz * c.y);
    const double2 yz = make_double2(Dz * b.x + Dy * c.x, Dz * b.y + Dy * c.y);
    const double2 xz = make_double2(Dz * a.x + Dx * c.x, Dz * a.y + Dx * c.y);
    const double2 xy = make_double2(Dy * a.x + Dx * b.x, Dy * a.y + Dx * b.y);
    d += w * (2.0 * (sq(xx) + sq(yy) + sq(zz)) + sq(yz) + sq(xz) + sq(xy));
    // (j, k, l) of i + S
    l += Sl;
    int carry = l >= g.Mz;
    l -= carry ? g.Mz : 0;
    k += Sk + carry;
    carry = k >= g.Ny;
    k -= carry ? g.Ny : 0;
    j += Sj + carry;
  }
  __shared__ double red[3][32];
  e = warp_sum(e);
  d = warp_sum(d);
  dv2 = warp_max(dv2);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = e;
    red[1][warp] = d;
    red[2][warp] = dv2;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    e = lane < nw ? red[0][lane] : 0.0;
    d = lane < nw ? red[1][lane] : 0.0;
    dv2 = lane < nw ? red[2][lane] : 0.0;
    e = warp_sum(e);
    d = warp_sum(d);
    dv2 = warp_max(dv2);
    if (lane == 0) {
      partial[3 * blockIdx.x + 0] = 0.5 * g.dx * g.dy * g.inv_vol * e;
      partial[3 * blockIdx.x + 1] = g.dx * g.dy * g.dz * g.inv_vol * d;
      partial[3 * blockIdx.x + 2] = sqrt(dv2);  // max |div| (sqrt is monotonic)
    }
  }
}

__global__ void diag_final_kernel(const double* __restrict__ partial, int nblocks,
                                  double* __restrict__ out) {
  double e = 0.0, d = 0.0, dv = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    e += partial[3 * b];
    d += partial[3 * b + 1];
    dv = fmax(dv, partial[3 * b + 2]);
  }
  __shared__ double red[3][32];
  e = warp_sum(e);
  d = warp_sum(d);
  dv = warp_max(dv);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = e;
    red[1][warp] = d;
    red[2][warp] = dv;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    e = lane < nw ? red[0][lane] : 0.0;
    d = lane < nw ? red[1][lane] : 0.0;
    dv = lane < nw ? red[2][lane] : 0.0;
    e = warp_sum(e);
    d = warp_sum(d);
    dv = warp_max(dv);
    if (lane == 0) {
      out[0] = e;
      out[1] = d;
      out[2] = dv;
    }
  }
}

}  // namespace ns3d
