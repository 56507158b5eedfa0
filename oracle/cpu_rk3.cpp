// CPU restatement of the reference's RK3 step in C++17 + OpenMP, FP64
// (TEST INFRASTRUCTURE and the CPU baseline of bench.py).
//
// This is the checker's second form (after oracle/ns3d_oracle.py) and the
// host-core baseline the GPU path is reported next to.  Only tests/,
// __graft_entry__ and bench.py's cpu_baseline leg load it; the product never
// does.  FFTW is not installed in this image, so the transforms are this
// file's own: a mixed-radix (2, 3, 4) Stockham FFT per line, batched over the
// other two axes with OpenMP.
//
// Algorithm, with the reference's quirks (as in oracle/ns3d_oracle.py):
//  * spectral layout [Nx][Ny][Mz] complex, Mz = Nz/2 + 1 (Source/Macros.h:11);
//  * x / y wavenumber index j < N/2 -> j, else j - N (the Nyquist stored as
//    -N/2), z index l (Source/math_support.cu:350-414);
//  * the anisotropic 2/3 mask evaluated with Mz in the Nz slot, minus the
//    (0,0,0) mode (Source/math_support.cu:471-519, NS3D_periodic.cu:1153-1161);
//  * Q_i = sum_j u_j d_j u_i from 3 masked velocities and 9 masked gradients
//    (12 C2R, 3 R2C; Source/advection_2_3.cu:146-397,480-497);
//  * Re(Qhat) := 0, Qhat(0) := 0 (Source/advection_2_3.cu:35-70);
//  * u <- (1 - dt|k|^2/Re) u + dt (AM.Q - Q) + dt f (Source/diffusion.cu:96-142);
//  * Shu-Osher SSP-RK3 (Source/RK_time_step.cu:310-327);
//  * C2R keeps only the Hermitian part of the kz = 0 and kz = Nz/2 planes and
//    scales by 1/(Nx Ny Nz); R2C is unnormalised (Source/math_support.cu:301-334).
#include <omp.h>

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

namespace {

using cd = std::complex<double>;
constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// 1-D mixed-radix Stockham FFT (radix 4, 2, 3), out of place with ping-pong
// ---------------------------------------------------------------------------
struct Line {
  int n = 0;
  std::vector<int> radix;
  // per stage: twiddles w^(q k) for q = 1..r-1, k = 0..Ns-1, both signs
  std::vector<std::vector<cd>> tw_fwd, tw_inv;

  explicit Line(int n_) : n(n_) {
    int m = n;
    while (m % 4 == 0) { radix.push_back(4); m /= 4; }
    while (m % 2 == 0) { radix.push_back(2); m /= 2; }
    while (m % 3 == 0) { radix.push_back(3); m /= 3; }
    if (m != 1) radix.clear();  // unsupported length
    int Ns = 1;
    for (int r : radix) {
      std::vector<cd> f((size_t)(r - 1) * Ns), b((size_t)(r - 1) * Ns);
      for (int q = 1; q < r; ++q)
        for (int k = 0; k < Ns; ++k) {
          const double a = 2.0 * kPi * (double)(q * k) / (double)(Ns * r);
          f[(size_t)(q - 1) * Ns + k] = cd(std::cos(a), -std::sin(a));
          b[(size_t)(q - 1) * Ns + k] = cd(std::cos(a), std::sin(a));
        }
      tw_fwd.push_back(std::move(f));
      tw_inv.push_back(std::move(b));
      Ns *= r;
    }
  }

  // x (length n) -> result, using `work` (length n); returns a pointer to
  // whichever of x / work holds the result.  sign: -1 forward, +1 inverse.
  cd* run(cd* x, cd* work, int sign) const {
    cd* in = x;
    cd* out = work;
    int Ns = 1;
    const double s3 = sign * std::sqrt(3.0) / 2.0;
    for (size_t st = 0; st < radix.size(); ++st) {
      const int r = radix[st];
      const std::vector<cd>& tw = sign < 0 ? tw_fwd[st] : tw_inv[st];
      const int m = n / r;
      for (int j = 0; j < m; ++j) {
        const int k = j % Ns;
        const int o = (j / Ns) * Ns * r + k;
        if (r == 2) {
          cd a = in[j], b = in[j + m] * tw[k];
          out[o] = a + b;
          out[o + Ns] = a - b;
        } else if (r == 4) {
          cd a = in[j], b = in[j + m] * tw[k], c = in[j + 2 * m] * tw[Ns + k],
             d = in[j + 3 * m] * tw[2 * Ns + k];
          cd t0 = a + c, t1 = a - c, t2 = b + d, t3 = b - d;
          // t3 times sign * i
          cd t3i = sign < 0 ? cd(t3.imag(), -t3.real()) : cd(-t3.imag(), t3.real());
          out[o] = t0 + t2;
          out[o + Ns] = t1 + t3i;
          out[o + 2 * Ns] = t0 - t2;
          out[o + 3 * Ns] = t1 - t3i;
        } else {  // 3
          cd a = in[j], b = in[j + m] * tw[k], c = in[j + 2 * m] * tw[Ns + k];
          cd sbc = b + c, dbc = b - c;
          cd t = a - 0.5 * sbc;
          cd u = cd(-dbc.imag() * s3, dbc.real() * s3);  // i * s3 * (b - c)
          out[o] = a + sbc;
          out[o + Ns] = t + u;
          out[o + 2 * Ns] = t - u;
        }
      }
      std::swap(in, out);
      Ns *= r;
    }
    return in;
  }
};

struct Cpu {
  int Nx, Ny, Nz, Mz;
  double Lx, Ly, Lz, kfx, kfy, kfz;
  size_t nc, nr;
  std::unique_ptr<Line> lx, ly, lz;
  std::vector<uint8_t> mask;     // [Nx][Ny][Mz]
  std::vector<cd> f[3];          // forcing
  std::vector<cd> spec[12];      // masked fields and gradients
  std::vector<double> phys[12];  // their physical values, then the products
  std::vector<cd> Q[3], u1[3], u2[3];

  size_t ci(int j, int k, int l) const { return ((size_t)j * Ny + k) * Mz + l; }
  int sx(int j) const { return j < Nx / 2 ? j : j - Nx; }
  int sy(int k) const { return k < Ny / 2 ? k : k - Ny; }

  Cpu(int nx, int ny, int nz, double lx_, double ly_, double lz_)
      : Nx(nx), Ny(ny), Nz(nz), Mz(nz / 2 + 1), Lx(lx_), Ly(ly_), Lz(lz_) {
    kfx = 2.0 * kPi / Lx;
    kfy = 2.0 * kPi / Ly;
    kfz = 2.0 * kPi / Lz;
    nc = (size_t)Nx * Ny * Mz;
    nr = (size_t)Nx * Ny * Nz;
    lx.reset(new Line(Nx));
    ly.reset(new Line(Ny));
    lz.reset(new Line(Nz));
    mask.assign(nc, 0);
    // build_mask_matrix's arithmetic with Mz in the Nz slot
    for (int j = 0; j < Nx; ++j)
      for (int k = 0; k < Ny; ++k)
        for (int l = 0; l < Mz; ++l) {
          const int m = j >= Nx / 2 ? j - Nx : j, n = k >= Ny / 2 ? k - Ny : k, q = l;
          const double kx = m * 2 * kPi / Lx, ky = n * 2 * kPi / Ly, kz = q * 2 * kPi / Lz;
          const double kxm = 2 * Nx * kPi / Lx, kym = 2 * Ny * kPi / Ly, kzm = 2 * Mz * kPi / Lz;
          const double r =
              std::sqrt(kx * kx / (kxm * kxm) + ky * ky / (kym * kym) + kz * kz / (kzm * kzm));
          mask[ci(j, k, l)] = r < 2.0 / 3.0 ? 1 : 0;
        }
    mask[0] = 0;
    for (int c = 0; c < 3; ++c) {
      f[c].assign(nc, cd(0, 0));
      Q[c].assign(nc, cd(0, 0));
      u1[c].assign(nc, cd(0, 0));
      u2[c].assign(nc, cd(0, 0));
    }
    for (int i = 0; i < 12; ++i) {
      spec[i].assign(nc, cd(0, 0));
      phys[i].assign(nr, 0.0);
    }
  }

  bool ok() const { return !lx->radix.empty() && !ly->radix.empty() && !lz->radix.empty(); }

  // complex transforms along x and y of one [Nx][Ny][Mz] array, in place
  void pass_x(cd* a, int sign) const {
#pragma omp parallel
    {
      std::vector<cd> buf(Nx), work(Nx);
#pragma omp for collapse(2) schedule(static)
      for (int k = 0; k < Ny; ++k)
        for (int l = 0; l < Mz; ++l) {
          for (int j = 0; j < Nx; ++j) buf[j] = a[ci(j, k, l)];
          const cd* r = lx->run(buf.data(), work.data(), sign);
          for (int j = 0; j < Nx; ++j) a[ci(j, k, l)] = r[j];
        }
    }
  }
  void pass_y(cd* a, int sign) const {
#pragma omp parallel
    {
      std::vector<cd> buf(Ny), work(Ny);
#pragma omp for collapse(2) schedule(static)
      for (int j = 0; j < Nx; ++j)
        for (int l = 0; l < Mz; ++l) {
          for (int k = 0; k < Ny; ++k) buf[k] = a[ci(j, k, l)];
          const cd* r = ly->run(buf.data(), work.data(), sign);
          for (int k = 0; k < Ny; ++k) a[ci(j, k, l)] = r[k];
        }
    }
  }
  // C2R along z of two half spectra at once (x and y already inverse
  // transformed), times `sc`: the Hermitian part of bins 0 and Nz/2 only
  void c2r_z_pair(const cd* a, const cd* b, double* ra, double* rb, double sc) const {
#pragma omp parallel
    {
      std::vector<cd> buf(Nz), work(Nz);
#pragma omp for schedule(static)
      for (long long line = 0; line < (long long)Nx * Ny; ++line) {
        const cd* pa = a + line * Mz;
        const cd* pb = b + line * Mz;
        for (int q = 0; q < Nz; ++q) {
          const bool up = q > Nz / 2;
          const int s = up ? Nz - q : q;
          cd x = pa[s], y = pb[s];
          if (s == 0 || s == Nz / 2) {
            x = cd(x.real(), 0.0);
            y = cd(y.real(), 0.0);
          }
          if (up) {
            x = std::conj(x);
            y = std::conj(y);
          }
          buf[q] = cd(x.real() - y.imag(), x.imag() + y.real());
        }
        const cd* r = lz->run(buf.data(), work.data(), +1);
        for (int q = 0; q < Nz; ++q) {
          ra[line * Nz + q] = r[q].real() * sc;
          rb[line * Nz + q] = r[q].imag() * sc;
        }
      }
    }
  }
  // R2C along z of two real fields at once into half spectra
  void r2c_z_pair(const double* ra, const double* rb, cd* a, cd* b) const {
#pragma omp parallel
    {
      std::vector<cd> buf(Nz), work(Nz);
#pragma omp for schedule(static)
      for (long long line = 0; line < (long long)Nx * Ny; ++line) {
        for (int q = 0; q < Nz; ++q)
          buf[q] = cd(ra[line * Nz + q], rb ? rb[line * Nz + q] : 0.0);
        const cd* r = lz->run(buf.data(), work.data(), -1);
        for (int q = 0; q < Mz; ++q) {
          const cd w = r[q], mi = std::conj(r[q == 0 ? 0 : Nz - q]);
          a[line * Mz + q] = 0.5 * (w + mi);
          if (b) b[line * Mz + q] = cd(0.0, -0.5) * (w - mi);
        }
      }
    }
  }

  // Qhat of the advective term for the state U
  void convolution(const cd* const U[3]) {
    // masked velocities (0..2) and gradients d_x u_i (3..5), d_y (6..8), d_z (9..11)
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 0; j < Nx; ++j)
      for (int k = 0; k < Ny; ++k)
        for (int l = 0; l < Mz; ++l) {
          const size_t i = ci(j, k, l);
          const double kx = kfx * sx(j), ky = kfy * sy(k), kz = kfz * l;
          for (int c = 0; c < 3; ++c) {
            const cd v = mask[i] ? U[c][i] : cd(0.0, 0.0);
            spec[c][i] = v;
            spec[3 + c][i] = cd(-v.imag() * kx, v.real() * kx);
            spec[6 + c][i] = cd(-v.imag() * ky, v.real() * ky);
            spec[9 + c][i] = cd(-v.imag() * kz, v.real() * kz);
          }
        }
    const double sc = 1.0 / (double)nr;
    for (int f2 = 0; f2 < 12; ++f2) {
      pass_x(spec[f2].data(), +1);
      pass_y(spec[f2].data(), +1);
    }
    for (int p = 0; p < 12; p += 2)
      c2r_z_pair(spec[p].data(), spec[p + 1].data(), phys[p].data(), phys[p + 1].data(), sc);
    // Q_i = u_x d_x u_i + u_y d_y u_i + u_z d_z u_i  (into phys[3..5])
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)nr; ++i) {
      const double ux = phys[0][i], uy = phys[1][i], uz = phys[2][i];
      for (int c = 0; c < 3; ++c)
        phys[3 + c][i] = ux * phys[3 + c][i] + uy * phys[6 + c][i] + uz * phys[9 + c][i];
    }
    r2c_z_pair(phys[3].data(), phys[4].data(), Q[0].data(), Q[1].data());
    r2c_z_pair(phys[5].data(), nullptr, Q[2].data(), nullptr);
    for (int c = 0; c < 3; ++c) {
      pass_y(Q[c].data(), -1);
      pass_x(Q[c].data(), -1);
    }
  }

  // out = ca * un + cb * [ (1 - dt|k|^2/Re) us + dt (AM.Q - Q) + dt f ]
  void update(const cd* const us[3], cd* const out[3], const cd* const un[3], double ca,
              double cb, double dt, double Re) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 0; j < Nx; ++j)
      for (int k = 0; k < Ny; ++k)
        for (int l = 0; l < Mz; ++l) {
          const size_t i = ci(j, k, l);
          const double kx = kfx * sx(j), ky = kfy * sy(k), kz = kfz * l;
          const double kk = kx * kx + ky * ky + kz * kz;
          const bool origin = i == 0;
          cd q[3];
          for (int c = 0; c < 3; ++c) q[c] = origin ? cd(0, 0) : cd(0.0, Q[c][i].imag());
          const cd kq = kk > 0.0 ? (kx * q[0] + ky * q[1] + kz * q[2]) / kk : cd(0, 0);
          const cd p[3] = {kx * kq - q[0], ky * kq - q[1], kz * kq - q[2]};
          const double G = 1.0 - kk * dt / Re;
          for (int c = 0; c < 3; ++c) {
            const cd r = G * us[c][i] + dt * p[c] + dt * f[c][i];
            out[c][i] = un ? ca * un[c][i] + cb * r : r;
          }
        }
  }

  void rk3(cd* const u[3], double dt, double Re) {
    const cd* uc[3] = {u[0], u[1], u[2]};
    cd* p1[3] = {u1[0].data(), u1[1].data(), u1[2].data()};
    cd* p2[3] = {u2[0].data(), u2[1].data(), u2[2].data()};
    const cd* c1[3] = {p1[0], p1[1], p1[2]};
    const cd* c2[3] = {p2[0], p2[1], p2[2]};
    convolution(uc);
    update(uc, p1, nullptr, 0.0, 1.0, dt, Re);
    convolution(c1);
    update(c1, p2, uc, 0.75, 0.25, dt, Re);
    convolution(c2);
    update(c2, u, uc, 1.0 / 3.0, 2.0 / 3.0, dt, Re);
  }
};

}  // namespace

extern "C" {

void* cpu_rk3_create(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz) {
  Cpu* c = new Cpu(Nx, Ny, Nz, Lx, Ly, Lz);
  if (!c->ok()) {
    delete c;
    return nullptr;
  }
  return c;
}

void cpu_rk3_destroy(void* h) { delete static_cast<Cpu*>(h); }

int cpu_rk3_threads() { return omp_get_max_threads(); }

// fields: 3 components, each [Nx][Ny][Mz] complex (interleaved re, im)
void cpu_rk3_set_forcing(void* h, const double* f) {
  Cpu* c = static_cast<Cpu*>(h);
  for (int i = 0; i < 3; ++i)
    std::memcpy(c->f[i].data(), f + 2 * c->nc * i, sizeof(cd) * c->nc);
}

void cpu_rk3_steps(void* h, double* u, double dt, double Re, int nsteps) {
  Cpu* c = static_cast<Cpu*>(h);
  cd* p[3] = {reinterpret_cast<cd*>(u), reinterpret_cast<cd*>(u) + c->nc,
              reinterpret_cast<cd*>(u) + 2 * c->nc};
  for (int s = 0; s < nsteps; ++s) c->rk3(p, dt, Re);
}

void cpu_convolution(void* h, const double* u, double* q) {
  Cpu* c = static_cast<Cpu*>(h);
  const cd* p[3] = {reinterpret_cast<const cd*>(u), reinterpret_cast<const cd*>(u) + c->nc,
                    reinterpret_cast<const cd*>(u) + 2 * c->nc};
  c->convolution(p);
  cd* out = reinterpret_cast<cd*>(q);
  for (int i = 0; i < 3; ++i)
    for (size_t e = 0; e < c->nc; ++e)
      out[i * c->nc + e] = e == 0 ? cd(0, 0) : cd(0.0, c->Q[i][e].imag());
}

}  // extern "C"
