// Request server: time integrations of the tangent (Jacobian-vector product)
// equations for Newton-Krylov / Arnoldi clients, served with continuous
// batching.  No reference counterpart: the reference integrates one field per
// process (RK3_SSP_UV, Source/RK_time_step.cu:342-355, called through
// NSCallMatrixVector_exponential, Source/NS3D_periodic.cu:444-470).
//
// A request is either (N, Re, T, seed): a Kolmogorov base state u (laminar
// (Re/16) sin 4y x plus a seeded 1e-3 perturbation) and a seeded unit
// perturbation v, both generated on the device from the seed, advanced by
// ceil(T/dt) JVP steps (RK3 base, Heun tangent; dt the CFL-0.3 step of the
// laminar peak); or a field request: the caller's own u and v (copied in at
// admission), dt, Re and step count, with v (and u) copied back to the
// caller's buffers when it completes.  Either reports |v(T)|.
//
// Per grid N the server owns one batched handle of `capacity` instance slots
// (its memory is reserved when the server is created, from the free HBM),
// a stream and an event.  The engine loop, on the calling host thread,
// polls each grid's event; when a grid's step has finished it retires the
// requests that reached their step count (slot compaction: the last active
// slot moves into the freed one), admits requests that have arrived while
// slots are free, and launches the next step for all active slots at once.
// Grids progress independently and overlap on the device.  An instance's
// arithmetic does not depend on its slot or on the other instances, so a
// result is bit for bit the same alone and in any mix.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "solver_internal.h"

using namespace ns3d_detail;

namespace {

// ---------------------------------------------------------------------------
// seeded fields on the device
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// standard normal of (seed, stream, index): Box-Muller on two 53-bit uniforms
__device__ __forceinline__ double gauss(uint64_t seed, uint64_t stream, uint64_t idx) {
  const uint64_t a = mix64(seed * 0x9e3779b97f4a7c15ULL + stream * 0xd1b54a32d192ed03ULL +
                           2 * idx + 1);
  const uint64_t b = mix64(a ^ 0x632be59bd9b4e019ULL);
  const double u1 = ((a >> 11) + 1) * (1.0 / 9007199254740993.0);  // (0, 1]
  const double u2 = (b >> 11) * (1.0 / 9007199254740992.0);        // [0, 1)
  return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

struct GenGeom {
  int N, Mz;
  double kf;  // 2 pi / L
};

// Pure-imaginary divergence-free perturbation, amplitude |k|^-2 on
// 1 <= |k| <= 8 (index units), zero on the x / y Nyquist rows, antisymmetric
// imaginary parts (Hermitian, to rounding) on the kz = 0 and kz = N/2 planes, Leray-
// projected, mode 0 removed; not normalised.  Same recipe as the host
// generator of ns3dperiodic_b200/workload.py, with a counter-based RNG.
__global__ void gen_perturbation_kernel(double2* wx, double2* wy, double2* wz, GenGeom g,
                                        uint64_t seed) {
  const long long n = (long long)g.N * g.N * g.Mz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(i % g.Mz);
    const long long jk = i / g.Mz;
    const int k = (int)(jk % g.N), j = (int)(jk / g.N);
    const int m = j >= g.N / 2 ? j - g.N : j, nn = k >= g.N / 2 ? k - g.N : k;
    const double kk = sqrt((double)(m * m + nn * nn + l * l));
    double amp = (kk >= 1.0 && kk <= 8.0) ? 1.0 / (kk * kk) : 0.0;
    if (j == g.N / 2 || k == g.N / 2) amp = 0.0;
    double w[3];
    const bool plane = (l == 0) || (2 * l == g.N);
    const long long mirror = ((long long)((g.N - j) % g.N) * g.N + (g.N - k) % g.N) * g.Mz + l;
    for (int c = 0; c < 3; ++c) {
      const double a = gauss(seed, c, (uint64_t)i);
      w[c] = plane ? 0.5 * (a - gauss(seed, c, (uint64_t)mirror)) : a;
      w[c] *= amp;
    }
    const double kx = g.kf * m, ky = g.kf * nn, kz = g.kf * l;
    const double k2 = kx * kx + ky * ky + kz * kz;
    if (k2 > 0.0) {
      const double kw = (kx * w[0] + ky * w[1] + kz * w[2]) / k2;
      w[0] -= kx * kw;
      w[1] -= ky * kw;
      w[2] -= kz * kw;
    } else {
      w[0] = w[1] = w[2] = 0.0;
    }
    wx[i] = make_double2(0.0, w[0]);
    wy[i] = make_double2(0.0, w[1]);
    wz[i] = make_double2(0.0, w[2]);
  }
}

constexpr int kSumBlocks = 296;
constexpr int kSumThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  v = 0.0;
  if (threadIdx.x == 0)
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) v += red[q];
  return v;
}

// sum |w|^2 over the stored half spectrum of 3 components: per-block partials
__global__ void sumsq_partial_kernel(const double2* wx, const double2* wy, const double2* wz,
                                     long long n, double* partial) {
  __shared__ double red[32];
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 a = wx[i], b = wy[i], c = wz[i];
    s += a.x * a.x + a.y * a.y + b.x * b.x + b.y * b.y + c.x * c.x + c.y * c.y;
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void sum_final_kernel(const double* partial, int nb, double* out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[b];
  s = block_sum(s, red);
  if (threadIdx.x == 0) *out = s;
}

// w *= factor / sqrt(*sumsq)
__global__ void normalise_kernel(double2* wx, double2* wy, double2* wz, long long n,
                                 const double* sumsq, double factor) {
  const double s = factor / sqrt(*sumsq);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    wx[i] = make_double2(wx[i].x * s, wx[i].y * s);
    wy[i] = make_double2(wy[i].x * s, wy[i].y * s);
    wz[i] = make_double2(wz[i].x * s, wz[i].y * s);
  }
}

// the laminar profile (Re/16) sin(4y) x: ux(0, +-4, 0) += -+ i (Re/16) N^3/2
__global__ void add_laminar_kernel(double2* ux, int N, int Mz, double Re) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double a = 0.5 * (double)N * N * N * (Re / 16.0);
  const long long p = (long long)(4 % N) * Mz, q = (long long)((N - 4) % N) * Mz;
  ux[p].y -= a;
  ux[q].y += a;
}

// Sets one instance's (u, v) as a request of (N, Re, seed) defines them.
// scratch: kSumBlocks + 1 doubles.
cudaError_t request_fields(double2* const u[3], double2* const v[3], int N, double Re,
                           uint64_t seed, double* scratch, cudaStream_t st) {
  const int Mz = N / 2 + 1;
  const long long n = (long long)N * N * Mz;
  const GenGeom g{N, Mz, 1.0};
  const int blocks = (int)std::min<long long>((n + 255) / 256, 1184);
  // u: laminar + 1e-3 |U0| P(seed'), |U0| = sqrt(2) (Re/16) N^3 / 2
  gen_perturbation_kernel<<<blocks, 256, 0, st>>>(u[0], u[1], u[2], g, seed ^ 0x5bd1e995u);
  sumsq_partial_kernel<<<kSumBlocks, kSumThreads, 0, st>>>(u[0], u[1], u[2], n, scratch);
  sum_final_kernel<<<1, 1024, 0, st>>>(scratch, kSumBlocks, scratch + kSumBlocks);
  const double u0 = std::sqrt(2.0) * (Re / 16.0) * 0.5 * (double)N * N * N;
  normalise_kernel<<<blocks, 256, 0, st>>>(u[0], u[1], u[2], n, scratch + kSumBlocks,
                                           1e-3 * u0);
  add_laminar_kernel<<<1, 32, 0, st>>>(u[0], N, Mz, Re);
  // v: unit perturbation
  gen_perturbation_kernel<<<blocks, 256, 0, st>>>(v[0], v[1], v[2], g, seed);
  sumsq_partial_kernel<<<kSumBlocks, kSumThreads, 0, st>>>(v[0], v[1], v[2], n, scratch);
  sum_final_kernel<<<1, 1024, 0, st>>>(scratch, kSumBlocks, scratch + kSumBlocks);
  normalise_kernel<<<blocks, 256, 0, st>>>(v[0], v[1], v[2], n, scratch + kSumBlocks, 1.0);
  return cudaGetLastError();
}

double cfl_dt(int N, double Re) { return 0.3 * (2.0 * M_PI / N) / (Re / 16.0); }

int request_steps(int N, double Re, double T) {
  return (int)std::ceil(T / cfl_dt(N, Re) - 1e-9);
}

// One JVP step (RK3_SSP_UV) of the first `active` instances of a batched handle.
ns3d_status jvp_step_active(ns3d_solver* h, double2* const u[3], double2* const v[3],
                            int active) {
  h->geom.batch = active;
  const double2* uc[3] = {u[0], u[1], u[2]};
  const double2* vc[3] = {v[0], v[1], v[2]};
  const double2* v1c[3] = {h->v1[0], h->v1[1], h->v1[2]};
  NS3D_TRY(conv_front(h, uc, vc));
  NS3D_TRY(finish(h, ns3d::kExplicit, false, vc, h->v1, nullptr, 0.0, 1.0, 0.0, 0.0));
  NS3D_TRY(rk3_launches(h, u, 0.0, 0.0));
  NS3D_TRY(conv_front(h, uc, v1c));
  NS3D_TRY(finish(h, ns3d::kExplicit, false, v1c, v, vc, 0.5, 0.5, 0.0, 0.0));
  return NS3D_OK;
}

// slot-sized device copy of 3 components (from slot a to slot b)
cudaError_t copy_slot(double2* const f[3], size_t nc, int from, int to, cudaStream_t st) {
  for (int c = 0; c < 3; ++c) {
    const cudaError_t e = cudaMemcpyAsync(f[c] + (size_t)to * nc, f[c] + (size_t)from * nc,
                                          sizeof(double2) * nc, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

using Clock = std::chrono::steady_clock;

struct Slot {
  long long req;
  int steps_total, steps_launched;
};

struct Group {
  int N = 0, capacity = 0;
  size_t nc = 0;
  ns3d_solver* h = nullptr;
  double2* u[3] = {};
  double2* v[3] = {};
  cudaEvent_t ev = nullptr;
  bool busy = false;
  std::vector<Slot> slots;        // active, in slot order
  double* params_host = nullptr;  // pinned (dt, Re) x capacity
  double* scratch = nullptr;      // kSumBlocks + 1 doubles
  double* norm_host = nullptr;    // pinned
  std::deque<long long> queue;    // requests of this grid not yet admitted, arrival order
  long long instance_steps = 0;   // JVP steps launched, summed over the active slots
  // captured JVP step per active-slot count (index active - 1): the 25
  // launches replay as one graph; dropped when tiles, precision or forcing change
  std::vector<cudaGraphExec_t> step_exec;
  bool graphs_off = false;
};

void drop_step_graphs(Group& g) {
  for (auto& e : g.step_exec)
    if (e) cudaGraphExecDestroy(e);
  g.step_exec.clear();
}

}  // namespace

// the caller's buffers of a field request
struct FieldIO {
  bool fields = false;
  double dt = 0.0;
  const double2* u_in[3] = {};
  const double2* v_in[3] = {};
  double2* u_out[3] = {};
  double2* v_out[3] = {};
};

struct ns3d_server {
  bool started = false;
  Clock::time_point t0;  // server clock: zero at the first ns3d_server_run
  std::vector<Group> groups;
  std::vector<ns3d_request> req;
  std::vector<FieldIO> io;  // per request
  std::vector<ns3d_result> res;
  std::map<long long, std::vector<double2>> kept;  // keep = 1 results (3 components)
  std::string err;
  // ns3d_server_cancel may run on another host thread: the flags it sets and
  // the finished marks it reads are guarded by `mu`
  std::mutex mu;
  std::vector<char> cancel_flag, finished;
};

namespace {

ns3d_status sfail(ns3d_server* s, ns3d_status st, const std::string& m) {
  if (s) s->err = m;
  return st;
}

#define SRV_CHECK(s, call, where)                                                     \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return sfail(s, e_ == cudaErrorMemoryAllocation ? NS3D_ERR_OOM : NS3D_ERR_CUDA, \
                   std::string(where) + ": " + cudaGetErrorString(e_));               \
  } while (0)

Group* group_of(ns3d_server* s, int N) {
  for (auto& g : s->groups)
    if (g.N == N) return &g;
  return nullptr;
}

size_t slot_bytes(int N) {
  const size_t Sc = sizeof(double2) * (size_t)N * N * (N / 2 + 1);
  return 45 * Sc;  // u, v (6) + base scratch (21) + tangent scratch (18)
}

// Frees slot b of a grid whose stream is idle: the last active slot moves
// into it (compaction), so the active slots stay 0 .. active-1.
ns3d_status free_slot(ns3d_server* s, Group& g, size_t b) {
  const size_t last = g.slots.size() - 1;
  if (b != last) {
    cudaStream_t st = g.h->stream;
    SRV_CHECK(s, copy_slot(g.u, g.nc, (int)last, (int)b, st), "compaction");
    SRV_CHECK(s, copy_slot(g.v, g.nc, (int)last, (int)b, st), "compaction");
    g.params_host[2 * b] = g.params_host[2 * last];
    g.params_host[2 * b + 1] = g.params_host[2 * last + 1];
    g.slots[b] = g.slots[last];
  }
  g.slots.pop_back();
  return NS3D_OK;
}

// retire finished requests of a grid whose stream is idle
ns3d_status retire(ns3d_server* s, Group& g, double now) {
  for (size_t b = 0; b < g.slots.size();) {
    Slot& sl = g.slots[b];
    if (sl.steps_launched < sl.steps_total) {
      ++b;
      continue;
    }
    ns3d_result& r = s->res[(size_t)sl.req];
    double2* vv[3] = {g.v[0] + b * g.nc, g.v[1] + b * g.nc, g.v[2] + b * g.nc};
    cudaStream_t st = g.h->stream;
    sumsq_partial_kernel<<<kSumBlocks, kSumThreads, 0, st>>>(vv[0], vv[1], vv[2],
                                                            (long long)g.nc, g.scratch);
    sum_final_kernel<<<1, 1024, 0, st>>>(g.scratch, kSumBlocks, g.scratch + kSumBlocks);
    SRV_CHECK(s, cudaGetLastError(), "norm");
    SRV_CHECK(s, cudaMemcpyAsync(g.norm_host, g.scratch + kSumBlocks, sizeof(double),
                                 cudaMemcpyDeviceToHost, st), "norm copy");
    if (s->req[(size_t)sl.req].keep) {
      std::vector<double2>& out = s->kept[sl.req];
      out.resize(3 * g.nc);
      for (int c = 0; c < 3; ++c)
        SRV_CHECK(s, cudaMemcpyAsync(out.data() + c * g.nc, vv[c], sizeof(double2) * g.nc,
                                     cudaMemcpyDeviceToHost, st), "result copy");
    }
    const FieldIO& io = s->io[(size_t)sl.req];
    if (io.fields) {  // the caller's output buffers (device or pinned host)
      for (int c = 0; c < 3; ++c) {
        SRV_CHECK(s, cudaMemcpyAsync(io.v_out[c], vv[c], sizeof(double2) * g.nc,
                                     cudaMemcpyDefault, st), "v_out copy");
        if (io.u_out[c])
          SRV_CHECK(s, cudaMemcpyAsync(io.u_out[c], g.u[c] + b * g.nc, sizeof(double2) * g.nc,
                                       cudaMemcpyDefault, st), "u_out copy");
      }
    }
    SRV_CHECK(s, cudaStreamSynchronize(st), "retire sync");
    r.v_norm = std::sqrt(*g.norm_host);
    r.done = now;
    r.status = std::isfinite(r.v_norm) ? NS3D_OK : NS3D_ERR_NONFINITE;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->finished[(size_t)sl.req] = 1;
    }
    NS3D_TRY(free_slot(s, g, b));
  }
  return NS3D_OK;
}

// Cancellations flagged by ns3d_server_cancel: queued requests leave the
// queue; admitted ones leave their slot (the grid's stream is idle here).
ns3d_status apply_cancels(ns3d_server* s, Group& g, double now) {
  std::vector<long long> gone;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (auto it = g.queue.begin(); it != g.queue.end();) {
      if (s->cancel_flag[(size_t)*it]) {
        s->finished[(size_t)*it] = 1;
        gone.push_back(*it);
        it = g.queue.erase(it);
      } else {
        ++it;
      }
    }
  }
  for (size_t b = 0; b < g.slots.size();) {
    const long long id = g.slots[b].req;
    bool cancel;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      cancel = s->cancel_flag[(size_t)id] != 0;
      if (cancel) s->finished[(size_t)id] = 1;
    }
    if (!cancel) {
      ++b;
      continue;
    }
    gone.push_back(id);
    NS3D_TRY(free_slot(s, g, b));
  }
  for (long long id : gone) {
    ns3d_result& r = s->res[(size_t)id];
    r.status = NS3D_ERR_CANCELLED;
    r.done = now;
  }
  return NS3D_OK;
}

ns3d_status admit(ns3d_server* s, Group& g, double now) {
  while ((int)g.slots.size() < g.capacity && !g.queue.empty()) {
    const long long id = g.queue.front();
    const ns3d_request& q = s->req[(size_t)id];
    if (q.arrival > now) break;  // FIFO per grid: later requests arrive later
    g.queue.pop_front();
    const size_t b = g.slots.size();
    double2* uu[3] = {g.u[0] + b * g.nc, g.u[1] + b * g.nc, g.u[2] + b * g.nc};
    double2* vv[3] = {g.v[0] + b * g.nc, g.v[1] + b * g.nc, g.v[2] + b * g.nc};
    const FieldIO& io = s->io[(size_t)id];
    if (io.fields) {  // the caller's fields, read now
      for (int c = 0; c < 3; ++c) {
        SRV_CHECK(s, cudaMemcpyAsync(uu[c], io.u_in[c], sizeof(double2) * g.nc,
                                     cudaMemcpyDefault, g.h->stream), "u_in copy");
        SRV_CHECK(s, cudaMemcpyAsync(vv[c], io.v_in[c], sizeof(double2) * g.nc,
                                     cudaMemcpyDefault, g.h->stream), "v_in copy");
      }
    } else {
      SRV_CHECK(s, request_fields(uu, vv, g.N, q.Re, q.seed, g.scratch, g.h->stream),
                "request fields");
    }
    g.params_host[2 * b] = io.fields ? io.dt : cfl_dt(g.N, q.Re);
    g.params_host[2 * b + 1] = q.Re;
    ns3d_result& r = s->res[(size_t)id];
    r.admitted = now;
    g.slots.push_back(Slot{id, r.steps, 0});
  }
  return NS3D_OK;
}

ns3d_status launch_step(ns3d_server* s, Group& g) {
  const int active = (int)g.slots.size();
  if (active == 0) return NS3D_OK;
  cudaStream_t st = g.h->stream;
  SRV_CHECK(s, cudaMemcpyAsync(g.h->dtRe, g.params_host, sizeof(double) * 2 * active,
                               cudaMemcpyHostToDevice, st), "params");
  if ((int)g.step_exec.size() < g.capacity) g.step_exec.resize((size_t)g.capacity, nullptr);
  cudaGraphExec_t& exec = g.step_exec[(size_t)active - 1];
  if (!exec && !g.graphs_off) {
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      const ns3d_status r = jvp_step_active(g.h, g.u, g.v, active);
      e = cudaStreamEndCapture(st, &graph);
      if (r != NS3D_OK) {
        if (graph) cudaGraphDestroy(graph);
        return sfail(s, r, std::string("jvp step: ") + ns3d_last_error(g.h));
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
      if (graph) cudaGraphDestroy(graph);
    }
    if (e != cudaSuccess) {  // launch directly from now on
      cudaGetLastError();
      exec = nullptr;
      g.graphs_off = true;
    }
  }
  if (exec) {
    SRV_CHECK(s, cudaGraphLaunch(exec, st), "step graph");
  } else {
    const ns3d_status r = jvp_step_active(g.h, g.u, g.v, active);
    if (r != NS3D_OK) return sfail(s, r, std::string("jvp step: ") + ns3d_last_error(g.h));
  }
  for (auto& sl : g.slots) ++sl.steps_launched;
  g.instance_steps += active;
  SRV_CHECK(s, cudaEventRecord(g.ev, st), "event");
  g.busy = true;
  return NS3D_OK;
}

// Appends a request (its id is its index) and queues it on its grid.
void enqueue(ns3d_server* s, const ns3d_request& q, int steps, const FieldIO& io) {
  const long long id = (long long)s->req.size();
  s->req.push_back(q);
  s->io.push_back(io);
  ns3d_result res{};
  res.id = id;
  res.N = q.N;
  res.Re = q.Re;
  res.T = q.T;
  res.steps = steps;
  res.arrival = q.arrival;
  res.admitted = -1.0;
  res.done = -1.0;
  res.v_norm = 0.0;
  res.status = -1;
  s->res.push_back(res);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->cancel_flag.push_back(0);
    s->finished.push_back(0);
  }
  group_of(s, q.N)->queue.push_back(id);
}

// The engine loop of ns3d_server_run (until < 0) and ns3d_server_run_until.
ns3d_status engine(ns3d_server* s, double max_seconds, long long until, int* completed) {
  int done = 0;
  if (!s->started) {
    s->t0 = Clock::now();
    s->started = true;
  }
  auto now = [&]() { return std::chrono::duration<double>(Clock::now() - s->t0).count(); };
  auto target_done = [&]() { return until >= 0 && s->res[(size_t)until].status != -1; };
  const double deadline = now() + max_seconds;
  while (!target_done()) {
    const double t = now();
    bool work_left = false, progressed = false;
    for (auto& g : s->groups) {
      if (g.busy) {
        const cudaError_t q = cudaEventQuery(g.ev);
        if (q == cudaErrorNotReady) {
          work_left = true;
          continue;
        }
        if (q != cudaSuccess) return sfail(s, NS3D_ERR_CUDA, cudaGetErrorString(q));
        g.busy = false;
        const size_t before = g.slots.size();
        NS3D_TRY(retire(s, g, now()));
        done += (int)(before - g.slots.size());
        progressed = true;
      }
      NS3D_TRY(apply_cancels(s, g, now()));
      // admission time after this grid's retirements (a slot frees, then fills)
      if (t <= deadline) NS3D_TRY(admit(s, g, now()));
      if (!g.slots.empty() && t <= deadline) {
        NS3D_TRY(launch_step(s, g));
        progressed = true;
        work_left = true;
      }
      if (!g.queue.empty()) work_left = true;
    }
    if (!work_left || t > deadline) break;
    if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  // leave no step in flight
  for (auto& g : s->groups)
    if (g.busy) {
      SRV_CHECK(s, cudaEventSynchronize(g.ev), "drain");
      g.busy = false;
      const size_t before = g.slots.size();
      NS3D_TRY(retire(s, g, now()));
      done += (int)(before - g.slots.size());
    }
  if (completed) *completed = done;
  return NS3D_OK;
}

}  // namespace

extern "C" {

ns3d_status ns3d_server_create(const int* Ns, int nN, const int* capacity, double hbm_fraction,
                               ns3d_server** out) {
  if (!out || !Ns || nN <= 0) return NS3D_ERR_BAD_ARG;
  *out = nullptr;
  const bool by_hbm = hbm_fraction > 0.0 && hbm_fraction < 1.0;
  if (!capacity && !by_hbm) return NS3D_ERR_BAD_ARG;
  ns3d_server* s = new ns3d_server();
  auto bail = [&](ns3d_status st) {
    ns3d_server_destroy(s);
    cudaGetLastError();  // a failed allocation must not surface at the next launch check
    return st;
  };
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return bail(NS3D_ERR_CUDA);
  s->groups.reserve((size_t)nN);
  for (int i = 0; i < nN; ++i) {
    const int N = Ns[i];
    if (N <= 0 || !ns3d_supported_extent(N)) return bail(NS3D_ERR_UNSUPPORTED);
    for (int k = 0; k < i; ++k)
      if (Ns[k] == N) return bail(NS3D_ERR_BAD_ARG);
    // slots that hbm_fraction of the free memory (split evenly) holds, capped
    // by the caller's limit when there is one
    const long long fit =
        by_hbm ? (long long)((hbm_fraction * (double)free_b / nN) / (double)slot_bytes(N))
               : (long long)1 << 30;
    if (capacity && capacity[i] < 1) return bail(NS3D_ERR_BAD_ARG);
    const int cap = (int)std::min<long long>(capacity ? capacity[i] : fit, fit);
    if (cap < 1) return bail(NS3D_ERR_OOM);
    s->groups.emplace_back();
    Group& g = s->groups.back();
    g.N = N;
    g.capacity = cap;
    g.nc = (size_t)N * N * (N / 2 + 1);
    ns3d_status st = create_solver(cap, N, N, N, 2.0 * M_PI, 2.0 * M_PI, 2.0 * M_PI, &g.h);
    if (st != NS3D_OK) return bail(st);
    if ((st = ensure_uv_pool(g.h)) != NS3D_OK) return bail(st);
    if (!g.h->dtRe && cudaMalloc(&g.h->dtRe, sizeof(double) * 2 * cap) != cudaSuccess)
      return bail(NS3D_ERR_OOM);
    for (int c = 0; c < 3; ++c)
      if (cudaMalloc(&g.u[c], sizeof(double2) * g.nc * cap) != cudaSuccess ||
          cudaMalloc(&g.v[c], sizeof(double2) * g.nc * cap) != cudaSuccess)
        return bail(NS3D_ERR_OOM);
    if (cudaMalloc(&g.scratch, sizeof(double) * (kSumBlocks + 1)) != cudaSuccess ||
        cudaMallocHost(&g.params_host, sizeof(double) * 2 * cap) != cudaSuccess ||
        cudaMallocHost(&g.norm_host, sizeof(double)) != cudaSuccess ||
        cudaEventCreateWithFlags(&g.ev, cudaEventDisableTiming) != cudaSuccess)
      return bail(NS3D_ERR_OOM);
    // the Kolmogorov forcing sin(4y) x of the base flow
    std::vector<double2> f(g.nc, make_double2(0.0, 0.0));
    const double a = 0.5 * (double)N * N * N;
    f[(size_t)(4 % N) * (N / 2 + 1)].y = -a;
    f[(size_t)((N - 4) % N) * (N / 2 + 1)].y = a;
    double2* fd[3] = {};
    for (int c = 0; c < 3; ++c)
      if (cudaMalloc(&fd[c], sizeof(double2) * g.nc) != cudaSuccess) {
        for (int k = 0; k < c; ++k) cudaFree(fd[k]);
        return bail(NS3D_ERR_OOM);
      }
    cudaMemcpy(fd[0], f.data(), sizeof(double2) * g.nc, cudaMemcpyHostToDevice);
    cudaMemset(fd[1], 0, sizeof(double2) * g.nc);
    cudaMemset(fd[2], 0, sizeof(double2) * g.nc);
    st = ns3d_set_forcing(g.h, (ns3d_complex*)fd[0], (ns3d_complex*)fd[1],
                          (ns3d_complex*)fd[2]);
    const bool dense = ns3d_forcing_modes(g.h) < 0;
    for (int c = 0; c < 3; ++c) cudaFree(fd[c]);  // sparse: the handle keeps its own copy
    if (st != NS3D_OK || dense) return bail(NS3D_ERR_CUDA);
  }
  *out = s;
  return NS3D_OK;
}

ns3d_status ns3d_server_destroy(ns3d_server* s) {
  if (!s) return NS3D_ERR_BAD_ARG;
  for (auto& g : s->groups) {
    if (g.h) cudaStreamSynchronize(g.h->stream);
    drop_step_graphs(g);
    for (int c = 0; c < 3; ++c) {
      cudaFree(g.u[c]);
      cudaFree(g.v[c]);
    }
    cudaFree(g.scratch);
    if (g.params_host) cudaFreeHost(g.params_host);
    if (g.norm_host) cudaFreeHost(g.norm_host);
    if (g.ev) cudaEventDestroy(g.ev);
    if (g.h) ns3d_destroy(g.h);
  }
  delete s;
  return NS3D_OK;
}

const char* ns3d_server_last_error(const ns3d_server* s) { return s ? s->err.c_str() : "null"; }

ns3d_status ns3d_server_capacity(const ns3d_server* s, int N, int* slots) {
  if (!s || !slots) return NS3D_ERR_BAD_ARG;
  for (const auto& g : s->groups)
    if (g.N == N) {
      *slots = g.capacity;
      return NS3D_OK;
    }
  return NS3D_ERR_BAD_ARG;
}

ns3d_status ns3d_server_set_precision(ns3d_server* s, int precision) {
  if (!s) return NS3D_ERR_BAD_ARG;
  for (auto& g : s->groups) {
    if (g.busy) return sfail(s, NS3D_ERR_BAD_ARG, "set the precision between runs");
    const ns3d_status st = ns3d_set_precision(g.h, precision);
    if (st != NS3D_OK) return sfail(s, st, ns3d_last_error(g.h));
    drop_step_graphs(g);
  }
  return NS3D_OK;
}

ns3d_status ns3d_server_autotune(ns3d_server* s, int reps) {
  if (!s || reps < 1) return NS3D_ERR_BAD_ARG;
  for (auto& g : s->groups) {
    if (g.busy) return sfail(s, NS3D_ERR_BAD_ARG, "tune between runs");
    g.h->geom.batch = g.h->batch;  // tune for the full slot count
    const ns3d_status st = ns3d_autotune(g.h, reps, 0, nullptr);
    if (st != NS3D_OK) return sfail(s, st, ns3d_last_error(g.h));
    drop_step_graphs(g);
  }
  return NS3D_OK;
}

ns3d_status ns3d_server_stats(const ns3d_server* s, int N, long long* instance_steps) {
  if (!s || !instance_steps) return NS3D_ERR_BAD_ARG;
  for (const auto& g : s->groups)
    if (g.N == N) {
      *instance_steps = g.instance_steps;
      return NS3D_OK;
    }
  return NS3D_ERR_BAD_ARG;
}

ns3d_status ns3d_server_submit(ns3d_server* s, const ns3d_request* r, int n, long long* first_id) {
  if (!s || (!r && n > 0) || n < 0) return NS3D_ERR_BAD_ARG;
  double last = s->req.empty() ? -1e300 : s->req.back().arrival;
  for (int i = 0; i < n; ++i) {
    if (!group_of(s, r[i].N)) return sfail(s, NS3D_ERR_BAD_ARG, "no grid of that N");
    if (!(r[i].Re > 0.0) || !(r[i].T > 0.0) || !std::isfinite(r[i].arrival))
      return sfail(s, NS3D_ERR_BAD_ARG, "Re and T must be > 0");
    if (r[i].arrival < last)
      return sfail(s, NS3D_ERR_BAD_ARG, "requests must come in arrival order");
    last = r[i].arrival;
  }
  if (first_id) *first_id = (long long)s->req.size();
  for (int i = 0; i < n; ++i) enqueue(s, r[i], request_steps(r[i].N, r[i].Re, r[i].T), FieldIO{});
  return NS3D_OK;
}

ns3d_status ns3d_server_submit_fields(ns3d_server* s, const ns3d_field_request* r, int n,
                                      long long* first_id) {
  if (!s || (!r && n > 0) || n < 0) return NS3D_ERR_BAD_ARG;
  double last = s->req.empty() ? 0.0 : s->req.back().arrival;
  std::vector<double> arrival((size_t)n);
  const double now = s->started
                         ? std::chrono::duration<double>(Clock::now() - s->t0).count()
                         : 0.0;
  for (int i = 0; i < n; ++i) {
    const ns3d_field_request& q = r[i];
    if (!group_of(s, q.N)) return sfail(s, NS3D_ERR_BAD_ARG, "no grid of that N");
    if (!(q.Re > 0.0) || !(q.dt > 0.0) || q.steps < 1)
      return sfail(s, NS3D_ERR_BAD_ARG, "Re and dt must be > 0 and steps >= 1");
    for (int c = 0; c < 3; ++c)
      if (!q.u_in[c] || !q.v_in[c] || !q.v_out[c])
        return sfail(s, NS3D_ERR_BAD_ARG, "u_in, v_in and v_out are required");
    if ((q.u_out[0] != nullptr) != (q.u_out[1] != nullptr) ||
        (q.u_out[0] != nullptr) != (q.u_out[2] != nullptr))
      return sfail(s, NS3D_ERR_BAD_ARG, "u_out: all three components or none");
    double a = q.arrival;
    if (a < 0.0) a = std::max(now, last);
    if (!std::isfinite(a) || a < last)
      return sfail(s, NS3D_ERR_BAD_ARG, "requests must come in arrival order");
    arrival[(size_t)i] = last = a;
  }
  if (first_id) *first_id = (long long)s->req.size();
  for (int i = 0; i < n; ++i) {
    const ns3d_field_request& q = r[i];
    ns3d_request base{};
    base.N = q.N;
    base.Re = q.Re;
    base.T = q.steps * q.dt;
    base.arrival = arrival[(size_t)i];
    FieldIO io;
    io.fields = true;
    io.dt = q.dt;
    for (int c = 0; c < 3; ++c) {
      io.u_in[c] = (const double2*)q.u_in[c];
      io.v_in[c] = (const double2*)q.v_in[c];
      io.u_out[c] = (double2*)q.u_out[c];
      io.v_out[c] = (double2*)q.v_out[c];
    }
    enqueue(s, base, q.steps, io);
  }
  return NS3D_OK;
}

ns3d_status ns3d_server_set_forcing(ns3d_server* s, int N, const ns3d_complex* fx,
                                    const ns3d_complex* fy, const ns3d_complex* fz) {
  if (!s) return NS3D_ERR_BAD_ARG;
  Group* g = group_of(s, N);
  if (!g) return sfail(s, NS3D_ERR_BAD_ARG, "no grid of that N");
  if (g->busy) return sfail(s, NS3D_ERR_BAD_ARG, "set the forcing between runs");
  const ns3d_status st = ns3d_set_forcing(g->h, fx, fy, fz);
  if (st != NS3D_OK) return sfail(s, st, ns3d_last_error(g->h));
  drop_step_graphs(*g);
  return NS3D_OK;
}

ns3d_status ns3d_server_cancel(ns3d_server* s, long long id) {
  if (!s) return NS3D_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  if (id < 0 || id >= (long long)s->cancel_flag.size() || s->finished[(size_t)id])
    return NS3D_ERR_BAD_ARG;
  s->cancel_flag[(size_t)id] = 1;
  return NS3D_OK;
}

ns3d_status ns3d_server_run(ns3d_server* s, double max_seconds, int* completed) {
  if (!s || !(max_seconds >= 0.0)) return NS3D_ERR_BAD_ARG;
  return engine(s, max_seconds, -1, completed);
}

ns3d_status ns3d_server_run_until(ns3d_server* s, long long id, double max_seconds,
                                  int* completed) {
  if (!s || !(max_seconds >= 0.0) || id < 0 || id >= (long long)s->res.size())
    return NS3D_ERR_BAD_ARG;
  return engine(s, max_seconds, id, completed);
}

ns3d_status ns3d_server_results(const ns3d_server* s, ns3d_result* out, int cap, int* n) {
  if (!s || !n || (cap > 0 && !out)) return NS3D_ERR_BAD_ARG;
  const int m = (int)s->res.size();
  for (int i = 0; i < m && i < cap; ++i) out[i] = s->res[(size_t)i];
  *n = m;
  return NS3D_OK;
}

ns3d_status ns3d_server_result_field(const ns3d_server* s, long long id, ns3d_complex* vx,
                                     ns3d_complex* vy, ns3d_complex* vz) {
  if (!s || !vx || !vy || !vz) return NS3D_ERR_BAD_ARG;
  auto it = s->kept.find(id);
  if (it == s->kept.end()) return NS3D_ERR_BAD_ARG;
  const size_t nc = it->second.size() / 3;
  std::memcpy(vx, it->second.data(), sizeof(double2) * nc);
  std::memcpy(vy, it->second.data() + nc, sizeof(double2) * nc);
  std::memcpy(vz, it->second.data() + 2 * nc, sizeof(double2) * nc);
  return NS3D_OK;
}

ns3d_status ns3d_request_fields(ns3d_solver* h, double Re, unsigned long long seed,
                                ns3d_complex* ux, ns3d_complex* uy, ns3d_complex* uz,
                                ns3d_complex* vx, ns3d_complex* vy, ns3d_complex* vz) {
  NS3D_TRY(check_handle(h));
  if (h->Nx != h->Ny || h->Nx != h->Nz || !(Re > 0.0) || !ux || !uy || !uz || !vx || !vy || !vz)
    return fail(h, NS3D_ERR_BAD_ARG, "cubic grid, Re > 0 and 6 fields");
  double* scratch = nullptr;
  NS3D_CHECK(h, cudaMalloc(&scratch, sizeof(double) * (kSumBlocks + 1)), "scratch");
  double2* u[3] = {(double2*)ux, (double2*)uy, (double2*)uz};
  double2* v[3] = {(double2*)vx, (double2*)vy, (double2*)vz};
  cudaError_t e = request_fields(u, v, h->Nx, Re, (uint64_t)seed, scratch, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(scratch);
  NS3D_CHECK(h, e, "request fields");
  return NS3D_OK;
}

int ns3d_request_steps(int N, double Re, double T) { return request_steps(N, Re, T); }

void ns3d_map_exponential_served(void* user, void* in, void* out) {
  ns3d_served_map_context* c = static_cast<ns3d_served_map_context*>(user);
  if (!c) return;
  ns3d_map_context* m = &c->map;
  ns3d_status st = (m->solver && c->server) ? NS3D_OK : NS3D_ERR_BAD_ARG;
  if (st == NS3D_OK && (m->solver->Nx != m->solver->Ny || m->solver->Nx != m->solver->Nz))
    st = NS3D_ERR_BAD_ARG;
  if (st == NS3D_OK)
    st = ns3d_unpack_reduced(m->solver, static_cast<const double*>(in), m->vx, m->vy, m->vz);
  // the server copies v in on its own stream
  if (st == NS3D_OK) st = ns3d_synchronize(m->solver);
  long long id = -1;
  if (st == NS3D_OK) {
    ns3d_field_request r{};
    r.N = m->solver->Nx;
    r.Re = m->Re;
    r.dt = m->dt;
    r.steps = m->steps;
    ns3d_complex* u[3] = {m->ux, m->uy, m->uz};
    ns3d_complex* v[3] = {m->vx, m->vy, m->vz};
    for (int k = 0; k < 3; ++k) {
      r.u_in[k] = u[k];
      r.v_in[k] = v[k];
      r.u_out[k] = u[k];  // the base flow advances with every call
      r.v_out[k] = v[k];
    }
    r.arrival = -1.0;
    st = ns3d_server_submit_fields(c->server, &r, 1, &id);
  }
  if (st == NS3D_OK) st = ns3d_server_run_until(c->server, id, 1e30, nullptr);
  if (st == NS3D_OK) {
    const int rs = c->server->res[(size_t)id].status;
    st = rs == NS3D_OK ? NS3D_OK : (rs == -1 ? NS3D_ERR_CUDA : (ns3d_status)rs);
  }
  if (st == NS3D_OK)
    st = ns3d_pack_reduced(m->solver, m->vx, m->vy, m->vz, static_cast<double*>(out));
  if (st == NS3D_OK) st = ns3d_synchronize(m->solver);
  if (st != NS3D_OK) {
    if (m->status == NS3D_OK) m->status = st;
    // NaN in the output makes the Krylov driver stop
    if (out && m->solver)
      cudaMemset(out, 0xff, sizeof(double) * (size_t)ns3d_krylov_length(m->solver));
    return;
  }
  ++c->requests;
}

}  // extern "C"
