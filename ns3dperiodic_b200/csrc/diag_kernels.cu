#include "diag_kernels.cuh"

namespace ns3d {

namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Re(c e)
__device__ __forceinline__ double re_mul(double2 c, double2 e) { return c.x * e.x - c.y * e.y; }

__device__ __forceinline__ int wrap_next(int i, int n) { return i + 1 == n ? 0 : i + 1; }
__device__ __forceinline__ int wrap_prev(int i, int n) { return i == 0 ? n - 1 : i - 1; }

}  // namespace

__global__ void spectral_filter_kernel(const double2* __restrict__ ux, const double2* __restrict__ uy,
                                       const double2* __restrict__ uz, double2* fx, double2* fy,
                                       double2* fz, FilterGeom g, int mode, double p) {
  const long long n = (long long)g.Nx * g.Ny * g.Mz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(i % g.Mz);
    const long long jk = i / g.Mz;
    const int k = (int)(jk % g.Ny);
    const int j = (int)(jk / g.Ny);
    const int m = j >= g.Nx / 2 ? j - g.Nx : j;
    const int nn = k >= g.Ny / 2 ? k - g.Ny : k;
    const int q = l;
    double f;
    if (mode == 0) {
      // the reference's product order: 2 pi / L * m * 2 pi / L * m
      const double tx = 2.0 * M_PI / g.Lx * m * 2.0 * M_PI / g.Lx * m;
      const double ty = 2.0 * M_PI / g.Ly * nn * 2.0 * M_PI / g.Ly * nn;
      const double tz = 2.0 * M_PI / g.Lz * q * 2.0 * M_PI / g.Lz * q;
      f = 1.0 / (1.0 + p * p * (tx + ty + tz));
    } else {
      const double r2 = 1.0 * m * m / (1.0 * g.Nx * g.Nx) + 1.0 * nn * nn / (1.0 * g.Ny * g.Ny) +
                        1.0 * q * q / (1.0 * g.Mz * g.Mz);
      f = r2 <= p * p ? 1.0 : 0.0;
    }
    const double2 a = ux[i], b = uy[i], c = uz[i];
    fx[i] = make_double2(f * a.x, f * a.y);
    fy[i] = make_double2(f * b.x, f * b.y);
    fz[i] = make_double2(f * c.x, f * c.y);
  }
}

__global__ void curl_kernel(const double* __restrict__ ux, const double* __restrict__ uy,
                            const double* __restrict__ uz, double* __restrict__ rx,
                            double* __restrict__ ry, double* __restrict__ rz, GridGeom g) {
  const long long n = (long long)g.Nx * g.Ny * g.Nz;
  const long long sy = g.Nz, sx = (long long)g.Ny * g.Nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(i % g.Nz);
    const long long jk = i / g.Nz;
    const int k = (int)(jk % g.Ny);
    const int j = (int)(jk / g.Ny);
    const long long xp = wrap_next(j, g.Nx) * sx + k * sy + l;
    const long long xm = wrap_prev(j, g.Nx) * sx + k * sy + l;
    const long long yp = j * sx + wrap_next(k, g.Ny) * sy + l;
    const long long ym = j * sx + wrap_prev(k, g.Ny) * sy + l;
    const long long zp = j * sx + k * sy + wrap_next(l, g.Nz);
    const long long zm = j * sx + k * sy + wrap_prev(l, g.Nz);
    rx[i] = 0.5 * (uz[yp] - uz[ym]) / g.dy - 0.5 * (uy[zp] - uy[zm]) / g.dz;
    ry[i] = 0.5 * (ux[zp] - ux[zm]) / g.dz - 0.5 * (uz[xp] - ux[xm]) / g.dx;
    rz[i] = 0.5 * (uy[xp] - uy[xm]) / g.dx - 0.5 * (ux[yp] - ux[ym]) / g.dy;
  }
}

__global__ void record_partial_kernel(const double2* __restrict__ ux,
                                      const double2* __restrict__ uy,
                                      const double2* __restrict__ uz, RecordGeom g,
                                      const double2* __restrict__ tab,
                                      double* __restrict__ partial) {
  const int Nx = g.Nx, Ny = g.Ny, Mz = g.Mz;
  const double2* ex = tab;
  const double2* ey = ex + 3 * Nx;
  const double2* ez = ey + 3 * Ny;
  const double2* shx = ez + 3 * Mz;
  const double2* sxt = shx + Nx;
  const double2* syt = sxt + Nx;
  const double2* szt = syt + Ny;
  double acc[kRecordSums];
#pragma unroll
  for (int v = 0; v < kRecordSums; ++v) acc[v] = 0.0;
  const double half_idx = 0.5 / g.dx;
  const long long n = (long long)Nx * Ny * Mz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(i % Mz);
    const long long jk = i / Mz;
    const int k = (int)(jk % Ny);
    const int j = (int)(jk / Ny);
    const double w = (l == 0 || 2 * l == g.Nz) ? 1.0 : 2.0;
    const double2 a = ux[i], b = uy[i], c = uz[i];
    const double sx = sxt[j].x, sy = syt[k].x, sz = szt[l].x;
    const double2 sh = shx[j];
    // coefficients C of the six functionals Re(C e^{i theta(p)})
    double2 C[6];
    C[0] = a;
    C[1] = b;
    C[2] = c;
    // rot_x = i (sy c - sz b)
    C[3] = make_double2(-(sy * c.y - sz * b.y), sy * c.x - sz * b.x);
    // rot_y = i sz a - (sh c - conj(sh) a) / (2 dx)
    {
      const double2 shc = cmul(sh, c);
      const double2 sha = cmul(make_double2(sh.x, -sh.y), a);
      C[4] = make_double2(-sz * a.y - half_idx * (shc.x - sha.x),
                          sz * a.x - half_idx * (shc.y - sha.y));
    }
    // rot_z = i (sx b - sy a)
    C[5] = make_double2(-(sx * b.y - sy * a.y), sx * b.x - sy * a.x);
    const int m = j >= Nx / 2 ? j - Nx : j;
    const int nn = k >= Ny / 2 ? k - Ny : k;
    const double r2 = 1.0 * m * m / (1.0 * Nx * Nx) + 1.0 * nn * nn / (1.0 * Ny * Ny) +
                      1.0 * l * l / (1.0 * Mz * Mz);
    const bool in_cut = r2 <= g.cut2;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const double2 e = cmul(cmul(ex[s * Nx + j], ey[s * Ny + k]), ez[s * Mz + l]);
#pragma unroll
      for (int f = 0; f < 6; ++f) acc[6 * s + f] += w * re_mul(C[f], e);
      if (s == 1 && in_cut) {
#pragma unroll
        for (int f = 0; f < 6; ++f) acc[18 + f] += w * re_mul(C[f], e);
      }
    }
  }
  __shared__ double red[kRecordSums][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int v = 0; v < kRecordSums; ++v) {
    const double s = warp_sum(acc[v]);
    if (lane == 0) red[v][warp] = s;
  }
  __syncthreads();
  if (threadIdx.x < kRecordSums) {
    double s = 0.0;
    for (int q = 0; q < nw; ++q) s += red[threadIdx.x][q];
    partial[(long long)blockIdx.x * kRecordSums + threadIdx.x] = s;
  }
}

__global__ void record_final_kernel(const double* __restrict__ partial, int nblocks,
                                    const double* __restrict__ diag_out,
                                    const double2* __restrict__ ux,
                                    const double2* __restrict__ uy,
                                    const double2* __restrict__ uz, RecordReads reads,
                                    double total_time, double Re, double inv_n,
                                    double* __restrict__ rec) {
  __shared__ double sums[kRecordSums];
  const int lane = threadIdx.x & 31, v = threadIdx.x >> 5;
  if (v < kRecordSums) {
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += partial[(long long)b * kRecordSums + v];
    s = warp_sum(s);
    if (lane == 0) sums[v] = s * inv_n;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const double energy = diag_out[0], diss = diag_out[1];
  const double tail[4] = {energy, diss, energy - diss / Re, energy};
  int c = 0;
  rec[c++] = total_time;
  for (int s = 0; s < 4; ++s) {
    for (int f = 0; f < 6; ++f) rec[c++] = sums[6 * s + f];
    rec[c++] = tail[s];
  }
  const long long* F = reads.f;
  const double2 a = ux[F[0]], b = uy[F[0]], cc = uz[F[0]];
  rec[c++] = a.x;
  rec[c++] = a.y;
  rec[c++] = b.x;
  rec[c++] = b.y;
  rec[c++] = cc.x;
  rec[c++] = cc.y;
  rec[c++] = diss;
  rec[c++] = ux[F[1]].y;
  rec[c++] = ux[F[2]].y;
  rec[c++] = uy[F[1]].y;
  rec[c++] = uy[F[2]].y;
  rec[c++] = uz[F[1]].y;
  rec[c++] = uz[F[2]].y;
  for (int q = 3; q < 11; ++q) rec[c++] = ux[F[q]].y;
}

__global__ void spectrum_kernel(const double2* __restrict__ ux, const double2* __restrict__ uy,
                                const double2* __restrict__ uz, int Nx, int Ny, int Mz,
                                double norm, double* __restrict__ E) {
  const int n = blockIdx.x;
  const int hx = Nx / 2, hy = Ny / 2;
  const long long pairs = (long long)hx * hy;
  double s = 0.0;
  for (long long p = threadIdx.x; p < pairs; p += blockDim.x) {
    const int j = (int)(p / hy), k = (int)(p % hy);
    const int l = n - j - k;
    if (l < 0 || l >= Mz) continue;
    const long long i = ((long long)j * Ny + k) * Mz + l;
    const double2 a = ux[i], b = uy[i], c = uz[i];
    s += a.x * a.x / norm / norm + a.y * a.y / norm / norm;
    s += b.x * b.x / norm / norm + b.y * b.y / norm / norm;
    s += c.x * c.x / norm / norm + c.y * c.y / norm / norm;
  }
  __shared__ double red[32];
  s = warp_sum(s);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = s;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    s = lane < nw ? red[lane] : 0.0;
    s = warp_sum(s);
    if (lane == 0) E[n] = s;
  }
}

namespace {

struct Beltrami {
  double x, y, z;
};

__device__ __forceinline__ Beltrami shapiro_at(const GridGeom& g, long long i, double decay) {
  const int l = (int)(i % g.Nz);
  const long long jk = i / g.Nz;
  const int k = (int)(jk % g.Ny);
  const int j = (int)(jk / g.Ny);
  double sx, cx, sy, cy, sz, cz;
  sincos(j * g.dx, &sx, &cx);
  sincos(k * g.dy, &sy, &cy);
  sincos(l * g.dz, &sz, &cz);
  const double f = sqrt(3.0);
  Beltrami v;
  v.x = -0.5 * (f * cx * sy * sz + sx * cy * cz) * decay;
  v.y = 0.5 * (f * sx * cy * sz - cx * sy * cz) * decay;
  v.z = cx * cy * sz * decay;
  return v;
}

}  // namespace

__global__ void shapiro_field_kernel(double* __restrict__ ux, double* __restrict__ uy,
                                     double* __restrict__ uz, GridGeom g, double decay) {
  const long long n = (long long)g.Nx * g.Ny * g.Nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const Beltrami v = shapiro_at(g, i, decay);
    ux[i] = v.x;
    uy[i] = v.y;
    uz[i] = v.z;
  }
}

__global__ void shapiro_error_kernel(const double* __restrict__ ux, const double* __restrict__ uy,
                                     const double* __restrict__ uz, GridGeom g, double decay,
                                     double* __restrict__ partial) {
  const long long n = (long long)g.Nx * g.Ny * g.Nz;
  double lo = INFINITY, hi = -INFINITY;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const Beltrami v = shapiro_at(g, i, decay);
    const double ex = ux[i] - v.x, ey = uy[i] - v.y, ez = uz[i] - v.z;
    const double e = sqrt(ex * ex + ey * ey + ez * ez);
    lo = fmin(lo, e);
    hi = fmax(hi, e);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  __shared__ double red[2][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = lo;
    red[1][warp] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
      lo = fmin(lo, red[0][q]);
      hi = fmax(hi, red[1][q]);
    }
    partial[2 * blockIdx.x] = lo;
    partial[2 * blockIdx.x + 1] = hi;
  }
}

__global__ void minmax_final_kernel(const double* __restrict__ partial, int nblocks,
                                    double* __restrict__ out) {
  double lo = INFINITY, hi = -INFINITY;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    lo = fmin(lo, partial[2 * b]);
    hi = fmax(hi, partial[2 * b + 1]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  __shared__ double red[2][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = lo;
    red[1][warp] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
      lo = fmin(lo, red[0][q]);
      hi = fmax(hi, red[1][q]);
    }
    out[0] = lo;
    out[1] = hi;
  }
}

}  // namespace ns3d
