#!/usr/bin/env python
"""Benchmark of the FP64 pseudo-spectral SSP-RK3 step (forced Kolmogorov flow).

Workload (default): N^3 = 256^3 on the 2pi-periodic box, f = (sin 4y, 0, 0),
Re = 400 (200 below 256^3), laminar profile plus a seeded 1e-3 divergence-free perturbation,
dt from CFL 0.3 on the laminar peak velocity, FP64 throughout.  A "step" is
one RK3_SSP step (3 right-hand sides).  The metric is RK3 steps/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--N 256]
  python bench.py --workload arnoldi [--n-arnoldi 2300000] [--m-arnoldi 30] [...]

--impl ours       : the CUDA library (libns3d_b200.so) through its C ABI.
--impl reference  : the reference's own CUDA path (unmodified sources built
                    for sm_100a with cuFFT, oracle/_ref) on the same GPU and
                    workload.
Multi-GPU runs (torchrun) are independent replicas, one per GPU (the path
does not shard); value = steps of all ranks / max elapsed over ranks.

--workload arnoldi: one "step" is one Arnoldi factorisation (k = 0 to m,
classical Gram-Schmidt with reorthogonalisation) with the reference's
Krylov self-test operator, the 1-D periodic Laplacian of
Source/Arnoldi/Matrix_Vector_emulator.cu at its test size n = 2,300,000,
m = 30 (Source/Arnoldi/cuda_test.cu:63-70); the reference arm runs the
reference's own Arnoldi_driver (cuBLAS) on the same operator and start
vector.

--workload ira: one "step" is one implicitly restarted Arnoldi run about the
laminar Kolmogorov flow u0 = Re/16 sin(4y) x (forced by sin(4y) x) at 64^3,
Re = 200, k = 20, m = 40, from a fresh N(0, 2) start vector, with the final
Schur / Galerkin eigenvector stage.  Default (--ira-map exponential): the
exponential map NSCallMatrixVector_exponential (--ira-steps RK3_SSP_UV steps
per product at the CFL-0.3 dt), "LM", run until the Ritz norm is below
--ira-tol (5e-8, main's IRA_tol) - the reference main's IRA branch for
Timesteps_period > 1 (Source/NS3D_periodic.cu:1714-1718).  --ira-map
linearised: the Jacobian J(u0) itself (NSCallMatrixVector_reduced), "LR",
--ira-cycles forced cycles.  The reference arm runs the reference's own
Implicit_restart_Arnoldi_GPU_data (cuBLAS + host LAPACK) with its own map
(RK3_SSP_UV, or RK3_SSP_UV_RHS) on the same base flow and forcing.

  python bench.py --workload ira --steps 3 --warmup 1
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--Re", type=float, default=None,
                    help="default: 400 for the rk3 workload from 256^3 (the precision-mode "
                         "configuration), else 200")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default pass tiles (ours; the tuner runs before the "
                         "warm-up, outside the timed region)")
    ap.add_argument("--e2e-steps", type=int, default=0, help="0: same as --steps")
    ap.add_argument("--workload", choices=["rk3", "arnoldi", "ira", "ensemble", "serving"],
                    default="rk3",
                    help="rk3: the RK3 step (default); arnoldi: the Krylov factorisation; "
                         "ensemble: mixed-N Kolmogorov instances stepped as batches")
    ap.add_argument("--instances", type=int, default=64, help="ensemble size")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64",
                    help="fp32: transforms and products in FP32, state and update in FP64")
    ap.add_argument("--rate", type=float, default=200.0, help="serving: mean arrivals per s")
    ap.add_argument("--window", type=float, default=45.0, help="serving: seconds of arrivals")
    ap.add_argument("--slots", default="16,8,4", help="serving: slots for N = 64,96,128")
    ap.add_argument("--ira-N", type=int, default=64, help="ira: grid size")
    ap.add_argument("--ira-k", type=int, default=20, help="ira: wanted eigenvalues")
    ap.add_argument("--ira-m", type=int, default=40, help="ira: Krylov basis size")
    ap.add_argument("--ira-map", choices=["exponential", "linearised"], default="exponential",
                    help="ira: the exponential map (NSCallMatrixVector_exponential, 'LM', run "
                         "to --ira-tol) or the linearised map (NSCallMatrixVector_reduced, "
                         "'LR', --ira-cycles forced cycles)")
    ap.add_argument("--ira-steps", type=int, default=20,
                    help="ira: tangent steps per product of the exponential map")
    ap.add_argument("--ira-tol", type=float, default=5e-8,
                    help="ira: Ritz-norm tolerance of the exponential-map run "
                         "(IRA_tol of the reference's main)")
    ap.add_argument("--ira-cycles", type=int, default=None,
                    help="ira: restart cycles per run (linearised map: exactly this many, "
                         "default 20; exponential map: the cap, default 3000)")
    ap.add_argument("--n-arnoldi", type=int, default=2300000)
    ap.add_argument("--m-arnoldi", type=int, default=30)
    a = ap.parse_args()
    if a.ira_cycles is None:
        a.ira_cycles = 3000 if a.ira_map == "exponential" else 20
    if a.Re is None:
        a.Re = 400.0 if (a.workload == "rk3" and a.N >= 256) else 200.0
    return a


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def traffic_from_profiles(kernel: str, N: int):
    """DRAM bytes per launch from the committed ncu summary, if there is one."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        # | kernel | N | dram_bytes_per_launch | ...
        c = [x.strip() for x in line.strip().strip("|").split("|")]
        if len(c) >= 3 and c[0] == kernel and c[1] == str(N):
            try:
                return float(c[2])
            except ValueError:
                return None
    return None


def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(x: float, pg):
    if pg is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    import torch

    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()


def workload(N, Re, seed):
    from ns3dperiodic_b200 import workload as W

    U, F = W.kolmogorov_state(N, Re, seed)
    return U, F, W.kolmogorov_dt(N, Re)


def sizes(N):
    nc = N * N * (N // 2 + 1)
    Sc, Sr = 16 * nc, 8 * N ** 3
    return nc, Sc, Sr


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (numpy/scipy pocketfft) on the host cores
# ---------------------------------------------------------------------------
def cpu_baseline(N, Re, seed):
    """The C++ / OpenMP restatement (oracle/cpu_rk3.cpp, all host threads) on
    a bounded sample; the numpy/scipy oracle as a secondary figure."""
    from oracle import cpu_lib

    secondary = cpu_baseline_scipy(N, Re, seed)
    if not cpu_lib.available():
        return secondary
    U, F, dt = workload(N, Re, seed)
    with cpu_lib.CpuRK3(N, N, N) as C:
        C.set_forcing(F)
        t0 = time.perf_counter()
        U = C.rk3_ssp(U, dt, Re, 1)  # warm-up (page faults, thread pool)
        t1 = time.perf_counter()
        k = max(5, min(200, int(15.0 / max(t1 - t0, 1e-3))))
        t0 = time.perf_counter()
        U = C.rk3_ssp(U, dt, Re, k)
        el = time.perf_counter() - t0
        threads = C.threads
    return {"value": k / el, "unit": "steps/s", "cores": threads, "kind": "port",
            "sample": f"{k} RK3 steps of the {N}^3 Kolmogorov workload after 1 warm-up step, "
                      f"{el:.1f} s (oracle/cpu_rk3.cpp: C++17 + OpenMP, project-written "
                      f"mixed-radix FFT; FFTW is not installed)",
            "secondary": secondary}


def cpu_baseline_scipy(N, Re, seed):
    from oracle import ns3d_oracle as O

    cores = os.cpu_count() or 1
    os.environ["NS3D_ORACLE_THREADS"] = str(cores)
    U, F, dt = workload(N, Re, seed)
    g = O.Grid(N, N, N)
    t0 = time.perf_counter()
    U = O.rk3_ssp(g, U, F, dt, Re)  # warm-up (plans, page faults)
    t1 = time.perf_counter()
    k = max(1, min(50, int(15.0 / max(t1 - t0, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(k):
        U = O.rk3_ssp(g, U, F, dt, Re)
    el = time.perf_counter() - t0
    return {"value": k / el, "unit": "steps/s", "cores": cores, "kind": "port",
            "sample": f"{k} RK3 steps of the {N}^3 Kolmogorov workload (oracle: numpy + "
                      f"scipy.fft pocketfft, workers={cores}) after 1 warm-up step, {el:.1f} s"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, world, rank, local, pg):
    import torch

    from ns3dperiodic_b200 import Solver

    N, Re = args.N, args.Re
    U0, F0, dt = workload(N, Re, args.seed + rank)
    nc, Sc, Sr = sizes(N)
    S = Solver(N, N, N)
    stream = torch.cuda.Stream()
    S.set_stream(stream)
    S.precision = args.precision
    tiles = S.tiles if args.no_autotune else S.autotune()["tiles"]
    fp32 = args.precision == "fp32"
    U = S.to_device(U0)
    F = S.to_device(F0)
    torch.cuda.synchronize()
    S.set_forcing(F)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            S.rk3_ssp(U, dt, Re)
    barrier(pg)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
        for _ in range(args.steps):
            S.rk3_ssp(U, dt, Re)
        ev1.record(stream)
    ev1.synchronize()
    ms_local = ev0.elapsed_time(ev1)
    clocks = sampler.stop()
    barrier(pg)
    ms = max_over_ranks(ms_local, pg)
    ms_step = ms / args.steps
    value = world * args.steps / (ms / 1e3)

    # per-pass timing (CUDA events on the launching stream), dominant kernel
    names = ["inv_x", "inv_y", "z", "fwd_y", "fwd_x"]
    # algorithmic bytes per launch; FP32 scratch halves every field but the state
    alg = ([6 * Sc, 7.5 * Sc, 6 * Sc, 3 * Sc, 7.5 * Sc] if fp32 else
           [9 * Sc, 15 * Sc, 12 * Sc, 6 * Sc, 9 * Sc])
    with torch.cuda.stream(stream):
        pm = S.profile_passes(U, dt, Re, reps=20)
    dom = max(range(5), key=lambda i: pm[i])
    peak, peak_src = peaks()
    achieved = alg[dom] / (pm[dom] * 1e-3) / 1e9
    # the kernels the step launches: the nonlinear term's z pass with the
    # velocities in shared memory for FP64 lines; the ring-pipelined fwd_x
    # where a line fits in a warp (8 points per thread, 12 for multiples of 3)
    t_ring = N // (12 if N % 3 == 0 else min(N, 8))
    t_plain = N // (12 if N % 3 == 0 else min(N, 16))
    ring = t_ring <= 32 and (t_ring == 32 or t_plain < 8)
    # inv_y's tile 2 is the bulk-copy (TMA) form for FP64 lines
    ytma = S.tiles[1] == 2 and not fp32
    kname = {0: "inv_x_kernel", 1: "inv_y_tma_kernel" if ytma else "inv_y_kernel",
             2: "z_kernel" if fp32 else "z_kernel_st",
             3: "fwd_y_kernel", 4: "fwd_x_ring_kernel" if ring else "fwd_x_kernel"}[dom]
    traffic = traffic_from_profiles(kname, N)
    roofline = {"bound": "hbm", "kernel": kname, "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": traffic, "peak_source": peak_src,
                "alg_bytes_per_launch": alg[dom], "ms_per_launch": round(pm[dom], 5),
                "pass_ms": {n: round(t, 5) for n, t in zip(names, pm)},
                "pass_frac": {n: round(a / (t * 1e-3) / 1e9 / peak, 4)
                              for n, a, t in zip(names, alg, pm)},
                "pass_timing": ("CUDA events recorded between the five launches of one "
                                "right-hand side on the launching stream, one host "
                                "synchronisation per repetition, 20 repetitions; the event "
                                "gaps count in the pass times, whose per-step sum runs about "
                                "2% above the graph-replayed step")}

    # e2e through the public API with host buffers
    K = args.e2e_steps or args.steps
    hU = [torch.from_numpy(u).pin_memory() for u in U0]
    hF = [torch.from_numpy(f).pin_memory() for f in F0]
    outU = [torch.empty_like(h).pin_memory() for h in hU]
    Ue = S.zeros()
    Fe = S.zeros()
    barrier(pg)
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        for d, h in zip(Ue + Fe, hU + hF):
            d.copy_(h, non_blocking=True)
        stream.synchronize()
        S.set_forcing(Fe)
        diag = None
        for _ in range(K):
            S.rk3_ssp(Ue, dt, Re)
            diag = S.diagnostics(Ue)  # energy, dissipation, max|div| read back each step
        for h, d in zip(outU, Ue):
            h.copy_(d, non_blocking=True)
        stream.synchronize()
    el = time.perf_counter() - t0
    el = max_over_ranks(el, pg)
    e2e = {"value": round(world * K / el, 3), "unit": "steps/s",
           "h2d_bytes_per_step": round(6 * Sc / K, 1),
           "d2h_bytes_per_step": round(24 + 3 * Sc / K, 1),
           "steps": K,
           "protocol": "pinned host state+forcing -> device, K x (ns3d_rk3_step + "
                       "ns3d_diagnostics read-back), final state -> host; wall clock"}
    accuracy = None
    if fp32:
        # the FP32 mode against FP64 from the same state over the timed steps
        with torch.cuda.stream(stream):
            U32 = S.rk3_ssp(S.to_device(U0), dt, Re, nsteps=args.steps)
            e32 = S.diagnostics(U32)[0]
            S.precision = "fp64"
            U64 = S.rk3_ssp(S.to_device(U0), dt, Re, nsteps=args.steps)
            e64 = S.diagnostics(U64)[0]
            num = sum(float(torch.linalg.vector_norm(a - b)) ** 2 for a, b in zip(U32, U64))
            den = sum(float(torch.linalg.vector_norm(b)) ** 2 for b in U64)
        stream.synchronize()
        accuracy = {"steps": args.steps, "rel_l2_u_vs_fp64": math.sqrt(num / den),
                    "energy_rel_diff_vs_fp64": abs(e32 - e64) / abs(e64),
                    "tolerance": 1e-5}
    S.close()
    # P3L bytes; FP32 mode: 3 RHS of 30 S_c (6 + 7.5 + 6 + 3 + 7.5) plus the
    # FP64 partners u^n of stages 2 and 3 (6 S_c)
    p3l = (90 + 6) * Sc + 9 * Sr if fp32 else 159 * Sc + 18 * Sr
    line = {
        "metric": f"RK3 steps/s (Kolmogorov {N}^3 {'FP32 mode' if fp32 else 'FP64'})",
        "value": round(value, 3),
        "unit": "steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (transforms, products); f64 (state, update)" if fp32 else "f64",
        "data": "synthetic",
        "config": {"workload": f"kolmogorov_{N}^3_{args.precision}", "N": N, "Re": Re, "dt": dt,
                   "forcing": "sin(4y) x", "perturbation": "seeded 1e-3, |k|^-2 on 1<=|k|<=8",
                   "parallelism": f"replicas x{world}",
                   "tiles": dict(zip(("inv_x", "inv_y", "fwd_y", "fwd_x"), tiles)),
                   "l2": f"working set {(24 * Sc) / 1e6:.0f} MB (state + scratch) > 126 MB L2",
                   "mpts_steps_per_s": round(value * N ** 3 / 1e6, 1),
                   "p3l_bytes_per_step": p3l,
                   "p3l_gbs": round(p3l / (ms_step * 1e-3) / 1e9, 1),
                   "p3l_frac": round(p3l / (ms_step * 1e-3) / 1e9 / peak, 4),
                   "diag_last": diag,
                   "fp32_accuracy": accuracy},
        "roofline": roofline,
        "e2e": e2e,
        "gpu_launches": 15 * args.steps,
        "clocks": clocks,
    }
    return line


# ---------------------------------------------------------------------------
# reference arm: the reference's own CUDA build
# ---------------------------------------------------------------------------
def run_reference(args, world, rank, local, pg):
    from oracle import ref_lib

    if rank != 0:
        return None
    if not ref_lib.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libns3d_ref.so not built "
                                                    "(needs the reference tree to compile)"}
    N, Re = args.N, args.Re
    U0, F0, dt = workload(N, Re, args.seed)
    nc, Sc, Sr = sizes(N)
    sampler = ClockSampler(local)
    with ref_lib.RefSolver(N, N, N) as R:
        R.set_u(U0)
        R.set_f(F0)
        R.rk3(args.warmup, dt, Re)
        sampler.start()
        time.sleep(0.3)
        ms = R.time_rk3(args.steps, dt, Re)
        clocks = sampler.stop()
        value = args.steps / (ms / 1e3)
        K = args.e2e_steps or args.steps
        t0 = time.perf_counter()
        R.set_u(U0)
        R.set_f(F0)
        for _ in range(K):
            R.rk3(1, dt, Re)
            R.diag()
        R.get_u()
        el = time.perf_counter() - t0
    p3l = 159 * Sc + 18 * Sr
    return {
        "impl": "reference",
        "metric": f"RK3 steps/s (Kolmogorov {N}^3 FP64)",
        "value": round(value, 3),
        "unit": "steps/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"kolmogorov_{N}^3_fp64", "N": N, "Re": Re, "dt": dt,
                   "reference": "unmodified reference CUDA sources (RK3_SSP, cuFFT D2Z/Z2D) "
                                "built for sm_100a, legacy default stream",
                   "p3l_gbs": round(p3l / (ms / args.steps * 1e-3) / 1e9, 1)},
        "e2e": {"value": round(K / el, 3), "unit": "steps/s",
                "h2d_bytes_per_step": round(6 * Sc / K, 1),
                "d2h_bytes_per_step": round(16 + 3 * Sc / K, 1), "steps": K,
                "protocol": "host state+forcing -> device, K x (RK3_SSP + the main loop's "
                            "energy/dissipation diagnostics), final state -> host; wall clock"},
        "clocks": clocks,
    }


# ---------------------------------------------------------------------------
# Krylov workload: Arnoldi factorisations with the reference's self-test
# operator (Source/Arnoldi/cuda_test.cu:63-70: N = 2,300,000, m = k*5 = 30)
# ---------------------------------------------------------------------------
def arnoldi_bytes(n, m):
    """Gram-Schmidt bytes of one factorisation: the sum over columns of
    4 (j+1) n 8 B (one classical pass plus one reorthogonalisation pass,
    each reading V(:, 0..j) twice)."""
    return sum(4 * (j + 1) * n * 8 for j in range(1, m))


def arnoldi_start(n, seed):
    import numpy as np

    return np.random.default_rng(seed).standard_normal(n)


def run_ours_arnoldi(args, world, rank, local, pg):
    import numpy as np
    import torch

    from ns3dperiodic_b200 import Krylov

    n, m = args.n_arnoldi, args.m_arnoldi
    f0 = arnoldi_start(n, args.seed + rank)
    kr = Krylov(n, m)
    A = kr.laplace_map()
    V = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    H = np.zeros((m, m))
    f0d = torch.as_tensor(f0, device="cuda")
    f = f0d.clone()
    for _ in range(args.warmup):
        f.copy_(f0d)
        kr.arnoldi(A, V, H, f, 0, m)
    barrier(pg)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    s0 = torch.cuda.default_stream()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(s0)
    st = None
    for _ in range(args.steps):
        f.copy_(f0d)
        st = kr.arnoldi(A, V, H, f, 0, m)
    ev1.record(s0)
    ev1.synchronize()
    ms_local = ev0.elapsed_time(ev1)
    clocks = sampler.stop()
    barrier(pg)
    ms = max_over_ranks(ms_local, pg)
    ms_step = ms / args.steps
    value = world * args.steps / (ms / 1e3)
    peak, peak_src = peaks()
    # dominant kernel: the dot products over all m columns (the widest launch)
    pm = kr.profile(V, m, f0d, reps=20)
    alg_t = (m + 1) * n * 8
    achieved = alg_t / (pm[0] * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "gemv_t_partial+reduce_cols",
                "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": None, "peak_source": peak_src,
                "alg_bytes_per_launch": alg_t, "ms_per_launch": round(pm[0], 5),
                "kernel_ms": {"dots": round(pm[0], 5), "update": round(pm[1], 5),
                              "restart": round(pm[2], 5)},
                "kernel_frac": {"dots": round(alg_t / (pm[0] * 1e-3) / 1e9 / peak, 4),
                                "update": round((m + 2) * n * 8 / (pm[1] * 1e-3) / 1e9 / peak, 4),
                                "restart": round((2 * m + 1) * n * 8 / (pm[2] * 1e-3) / 1e9
                                                 / peak, 4)}}
    # e2e: the start vector from pinned host memory each factorisation; H is
    # assembled on the host column by column, as in the reference
    K = args.e2e_steps or args.steps
    hf = torch.from_numpy(f0).pin_memory()
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(K):
        f.copy_(hf, non_blocking=True)
        kr.arnoldi(A, V, H, f, 0, m)
    torch.cuda.synchronize()
    el = max_over_ranks(time.perf_counter() - t0, pg)
    kr.close()
    B = arnoldi_bytes(n, m)
    return {
        "metric": f"Arnoldi factorisations/s (1-D periodic Laplacian, n={n}, m={m}, FP64)",
        "value": round(value, 3),
        "unit": "factorisations/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"arnoldi_laplace1d_n{n}_m{m}", "n": n, "m": m,
                   "operator": "Source/Arnoldi/Matrix_Vector_emulator.cu:10-36",
                   "parallelism": f"replicas x{world}",
                   "l2": f"basis {m * n * 8 / 1e6:.0f} MB > 126 MB L2",
                   "gs_bytes_per_factorisation": B,
                   "gs_gbs": round(B / (ms_step * 1e-3) / 1e9, 1),
                   "gs_frac": round(B / (ms_step * 1e-3) / 1e9 / peak, 4),
                   "max_reorth_passes": st["max_passes"], "H00": float(H[0, 0])},
        "roofline": roofline,
        "e2e": {"value": round(world * K / el, 3), "unit": "factorisations/s",
                "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * m * (m + 2), "steps": K,
                "protocol": "pinned host start vector -> device, ns3d_arnoldi (H to the host "
                            "per column, as the reference); wall clock"},
        # the driver's own launches plus one Laplacian launch per column
        "gpu_launches": args.steps * (st["launches"] + m),
        "clocks": clocks,
    }


def cpu_baseline_arnoldi(n, m, seed):
    import numpy as np

    from oracle import krylov_oracle as K

    f = arnoldi_start(n, seed)
    V, H = np.zeros((m, n)), np.zeros((m, m))
    t0 = time.perf_counter()
    K.arnoldi_driver(K.laplace1d, V, H, f.copy(), 0, m)
    el = time.perf_counter() - t0
    k = max(1, min(10, int(15.0 / max(el, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(k):
        K.arnoldi_driver(K.laplace1d, V, H, f.copy(), 0, m)
    el = time.perf_counter() - t0
    return {"value": k / el, "unit": "factorisations/s", "cores": os.cpu_count() or 1,
            "kind": "port",
            "sample": f"{k} factorisations (oracle: numpy, BLAS threads as numpy configures "
                      f"them) after 1 warm-up, {el:.1f} s"}


def run_reference_arnoldi(args, world, rank, local, pg):
    import ctypes

    import numpy as np

    if rank != 0:
        return None
    path = os.path.join(ROOT, "oracle", "_ref", "libarnoldi_ref.so")
    if not os.path.exists(path):
        return {"impl": "reference", "unavailable": "oracle/_ref/libarnoldi_ref.so not built "
                                                    "(needs the reference tree to compile)"}
    lib = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.ref_time_arnoldi_laplace.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp]
    lib.ref_time_arnoldi_laplace.restype = ctypes.c_double
    n, m = args.n_arnoldi, args.m_arnoldi
    f0 = np.ascontiguousarray(arnoldi_start(n, args.seed))
    h00 = np.zeros(1)
    sampler = ClockSampler(local)
    lib.ref_time_arnoldi_laplace(n, m, args.warmup, f0.ctypes.data_as(dp), h00.ctypes.data_as(dp))
    sampler.start()
    time.sleep(0.3)
    ms = lib.ref_time_arnoldi_laplace(n, m, args.steps, f0.ctypes.data_as(dp),
                                      h00.ctypes.data_as(dp))
    clocks = sampler.stop()
    if ms < 0:
        return {"impl": "reference", "unavailable": "reference Arnoldi_driver run failed"}
    value = args.steps / (ms / 1e3)
    B = arnoldi_bytes(n, m)
    return {"impl": "reference",
            "metric": f"Arnoldi factorisations/s (1-D periodic Laplacian, n={n}, m={m}, FP64)",
            "value": round(value, 3), "unit": "factorisations/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"arnoldi_laplace1d_n{n}_m{m}", "n": n, "m": m,
                       "reference": "unmodified Source/Arnoldi/Arnoldi_Driver.cu with cuBLAS and "
                                    "its user_Ax_function, sm_100a",
                       "gs_gbs": round(B / (ms / args.steps * 1e-3) / 1e9, 1),
                       "H00": float(h00[0])},
            "e2e": {"value": round(value, 3), "unit": "factorisations/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "clocks": clocks}


# ---------------------------------------------------------------------------
# implicit restart of the linearised operator about the laminar Kolmogorov
# flow (64^3, Re = 200, k = 20, m = 40)
# ---------------------------------------------------------------------------
def ira_state(N, Re):
    from ns3dperiodic_b200 import workload as W

    U, _ = W.kolmogorov_state(N, Re, 0, rel_amp=0.0)
    return U


def ira_start(n, seed):
    import numpy as np

    return np.random.default_rng(seed).normal(0.0, 2.0, n)


def ira_setup(args):
    """(N, Re, k, m, which, tol, max_iter, dt, steps) of the ira workload."""
    from ns3dperiodic_b200 import workload as W

    N, Re, k, m = args.ira_N, args.Re, args.ira_k, args.ira_m
    if args.ira_map == "exponential":
        return N, Re, k, m, "LM", args.ira_tol, args.ira_cycles, W.kolmogorov_dt(N, Re), \
            args.ira_steps
    return N, Re, k, m, "LR", 0.0, args.ira_cycles, 0.0, 0


def ira_metric(args, N, Re, k, m):
    if args.ira_map == "exponential":
        return (f"IRA runs/s to Ritz norm <= {args.ira_tol:g} (exponential map, "
                f"{args.ira_steps} RK3_SSP_UV steps per product, of the linearised NS about "
                f"laminar Kolmogorov, {N}^3, Re={Re:g}, k={k}, m={m}, LM, FP64)")
    return (f"IRA runs/s (linearised NS about laminar Kolmogorov, {N}^3, Re={Re:g}, "
            f"k={k}, m={m}, {args.ira_cycles} restart cycles + eigenvector stage, FP64)")


def run_ours_ira(args, world, rank, local, pg):
    import numpy as np
    import torch

    from ns3dperiodic_b200 import Krylov, Solver
    from ns3dperiodic_b200 import workload as W

    N, Re, k, m, which, tol, max_iter, dt, steps = ira_setup(args)
    expo = args.ira_map == "exponential"
    U = ira_state(N, Re)
    S = Solver(N, N, N)
    tiles = S.tiles if args.no_autotune else S.autotune()["tiles"]
    S.set_forcing(S.to_device(W.kolmogorov_forcing(N, N, N)))
    Ud = S.to_device(U)
    Vs = S.zeros()
    n = S.krylov_length
    kr = Krylov(n, m)
    A = kr.exponential_map(S, Ud, Vs, dt, Re, steps) if expo else kr.linearised_map(S, Ud, Re)
    # launches per map call: unpack, the steps' passes (JVP step: 2 tangent
    # right-hand sides of 5 launches and a base RK3 step of 15), pack
    per_call = 2 + 25 * steps if expo else 7

    launches = [0]

    def one_run(f0d):
        _, rn, it, V, H = kr.implicit_restart_arnoldi(A, which, k, m, tol, max_iter, f0=f0d)
        w, X, res = kr.eigenpairs(A, V, H, k, which)
        cols = list(kr.last_restart_columns)
        launches[0] += kr.last_restart_launches + per_call * (sum(cols) + k) + 3
        return w, X, res, rn, cols, it

    f0d = torch.as_tensor(ira_start(n, args.seed + rank), device="cuda")
    for _ in range(args.warmup):
        Ud_reset(Ud, S, U)
        one_run(f0d)
    barrier(pg)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    s0 = torch.cuda.default_stream()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    Ud_reset(Ud, S, U)
    torch.cuda.synchronize()
    ev0.record(s0)
    out = None
    launches[0] = 0
    for _ in range(args.steps):
        out = one_run(f0d)
    ev1.record(s0)
    timed_launches = launches[0]
    ev1.synchronize()
    ms_local = ev0.elapsed_time(ev1)
    clocks = sampler.stop()
    barrier(pg)
    ms = max_over_ranks(ms_local, pg)
    ms_step = ms / args.steps
    value = world * args.steps / (ms / 1e3)
    w, X, res, rn, cols, it = out
    peak, peak_src = peaks()
    # bytes of one run: map calls (P3L) + Gram-Schmidt (one reorthogonalisation)
    _, Sc, Sr = sizes(N)
    mv_bytes = steps * (330 * Sc + 30 * Sr) if expo else 84 * Sc + 6 * Sr
    calls = sum(cols) + k
    gs = 0
    for c in cols:
        for j in range(m - c, m):
            gs += 4 * (j + 1) * 8 * n
    B = mv_bytes * calls + gs
    # the map alone, timed on the device
    x = torch.as_tensor(ira_start(n, 99), device="cuda")
    y = torch.empty_like(x)
    Ud_reset(Ud, S, U)
    for _ in range(3):
        kr.apply(A, x, y)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = 5 if expo else 50
    e0.record(s0)
    for _ in range(reps):
        kr.apply(A, x, y)
    e1.record(s0)
    e1.synchronize()
    mv_ms = e0.elapsed_time(e1) / reps
    achieved = mv_bytes / (mv_ms * 1e-3) / 1e9
    kname = (f"exponential map ({steps} RK3_SSP_UV steps, pack/unpack)" if expo else
             "linearised map (unpack, 5-pass B(u,v) + update, pack)")
    roofline = {"bound": "hbm", "kernel": kname,
                "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": None, "peak_source": peak_src,
                "alg_bytes_per_launch": mv_bytes, "ms_per_launch": round(mv_ms, 5),
                "note": "per map call (host-synchronised, as the Krylov drivers call it); "
                        "pack/unpack bytes not counted"}
    # e2e: base flow from pinned host memory, eigenvalues and eigenvectors back
    K = args.e2e_steps or args.steps
    hU = [torch.from_numpy(np.ascontiguousarray(u)).pin_memory() for u in U]
    hX = torch.empty((k, n), dtype=torch.complex128).pin_memory()
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(K):
        for d, h in zip(Ud, hU):
            d.copy_(h, non_blocking=True)
        w2, X2, _, _, _, _ = one_run(f0d)
        hX.copy_(X2)
    torch.cuda.synchronize()
    el = max_over_ranks(time.perf_counter() - t0, pg)
    kr.close()
    S.close()
    nc = N * N * (N // 2 + 1)
    cfg_map = (f"ns3d_map_exponential (NSCallMatrixVector_exponential), {steps} steps of "
               f"dt={dt:.6g}" if expo else "ns3d_map_linearised (NSCallMatrixVector_reduced)")
    return {
        "metric": ira_metric(args, N, Re, k, m),
        "value": round(value, 4),
        "unit": "runs/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": (f"ira_expo{steps}_kolmogorov_laminar_{N}_Re{Re:g}_k{k}_m{m}_"
                                f"tol{tol:g}" if expo else
                                f"ira_kolmogorov_laminar_{N}_Re{Re:g}_k{k}_m{m}_c{max_iter}"),
                   "N": N, "Re": Re, "k": k, "m": m, "n": n, "which": which, "tol": tol,
                   "max_cycles": max_iter, "cycles": it, "map": cfg_map,
                   "tiles": dict(zip(("inv_x", "inv_y", "fwd_y", "fwd_x"), tiles)),
                   "parallelism": f"replicas x{world}",
                   "l2": f"basis {m * n * 8 / 1e6:.0f} MB + fields > 126 MB L2",
                   "map_calls_per_run": calls, "alg_bytes_per_run": B,
                   "achieved_gbs_per_run": round(B / (ms_step * 1e-3) / 1e9, 1),
                   "ritz_norm": float(rn),
                   "leading_eigenvalues": [[round(float(z.real), 8), round(float(z.imag), 8)]
                                           for z in w[:4]],
                   "max_schur_residual": float(np.max(res))},
        "roofline": roofline,
        "e2e": {"value": round(world * K / el, 4), "unit": "runs/s",
                "h2d_bytes_per_step": 3 * 16 * nc, "d2h_bytes_per_step": 16 * k * n,
                "steps": K,
                "protocol": "base flow from pinned host memory -> device, the run, the k "
                            "complex eigenvectors back to pinned host memory; wall clock"},
        "gpu_launches": timed_launches,
        "clocks": clocks,
    }


def Ud_reset(Ud, S, U):
    """The base flow back to u0 (the exponential map advances it with every call)."""
    import torch

    for d, h in zip(Ud, S.to_device(U)):
        d.copy_(h)
    torch.cuda.synchronize()


def cpu_baseline_ira(N, Re, m, calls, seed, steps=0, dt=0.0):
    """The oracle on the host cores, on a bounded sample.  Exponential map
    (steps > 0): one oracle RK3_SSP_UV step (numpy + scipy.fft) timed and
    scaled to a run's products x steps (the Gram-Schmidt, a few percent of a
    run, is left out).  Linearised map: one factorisation from k = 0 with
    min(m, 8) columns over the oracle's linearised map, scaled to a run's
    map calls."""
    import numpy as np

    from oracle import krylov_oracle as K
    from oracle import ns3d_oracle as O

    g = O.Grid(N, N, N)
    U = ira_state(N, Re)
    if steps > 0:
        os.environ["NS3D_ORACLE_THREADS"] = str(os.cpu_count() or 1)
        F = O.kolmogorov_forcing(g)
        V = O.random_perturbation(g, seed)
        O.rk3_ssp_uv(g, U, V, F, dt, Re)  # warm-up (plans, page faults)
        reps = 3
        t0 = time.perf_counter()
        for _ in range(reps):
            U2, V = O.rk3_ssp_uv(g, U, V, F, dt, Re)
        el = (time.perf_counter() - t0) / reps
        return {"value": 1.0 / (el * steps * calls), "unit": "runs/s",
                "cores": os.cpu_count() or 1, "kind": "port",
                "sample": f"{reps} oracle RK3_SSP_UV steps at {N}^3 (numpy + scipy.fft), "
                          f"{el:.2f} s each, scaled to the {calls} products x {steps} steps "
                          f"of one run (Gram-Schmidt not counted)"}
    n = 3 * (N * N * (N // 2 + 1) - 1)
    mm = min(m, 8)
    f = ira_start(n, seed)
    V, H = np.zeros((mm, n)), np.zeros((mm, mm))
    t0 = time.perf_counter()
    K.arnoldi_driver(lambda v: O.linearised_matvec_reduced(g, U, v, 0.0, Re), V, H, f.copy(), 0,
                     mm)
    el = time.perf_counter() - t0
    per_col = el / mm
    return {"value": 1.0 / (per_col * calls), "unit": "runs/s", "cores": os.cpu_count() or 1,
            "kind": "port",
            "sample": f"one {mm}-column Arnoldi factorisation of the oracle's linearised map "
                      f"(numpy + scipy.fft) in {el:.1f} s, scaled to the {calls} map calls "
                      f"(and their Gram-Schmidt) of one run"}


def run_reference_ira(args, world, rank, local, pg):
    import ctypes
    import tempfile

    if rank != 0:
        return None
    path = os.path.join(ROOT, "oracle", "_ref", "libarnoldi_ref.so")
    if not os.path.exists(path):
        return {"impl": "reference", "unavailable": "oracle/_ref/libarnoldi_ref.so not built "
                                                    "(needs the reference tree to compile)"}
    from oracle.ref_lib import RefSolver

    from ns3dperiodic_b200 import workload as W

    N, Re, k, m, which, tol, R, dt, steps = ira_setup(args)
    expo = args.ira_map == "exponential"
    ns = RefSolver(N, N, N)
    U0 = ira_state(N, Re)
    ns.set_u(U0)
    ns.set_f(W.kolmogorov_forcing(N, N, N))
    arn = ctypes.CDLL(path)
    arn.ref_ira_map.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_double)]
    arn.ref_ira_map.restype = ctypes.c_double
    if expo:
        fn = ctypes.cast(ns.lib.ref_map_exponential_reduced, ctypes.c_void_p).value
        ctx = (ctypes.c_double * 3)(Re, dt, float(steps))
    else:
        fn = ctypes.cast(ns.lib.ref_map_linearised_reduced, ctypes.c_void_p).value
        ctx = (ctypes.c_double * 2)(Re, 0.0)
    lm = 1 if which == "LM" else 0
    n = 3 * (N * N * (N // 2 + 1) - 1)
    libc = ctypes.CDLL(None)
    sampler = ClockSampler(local)
    total, rn = 0.0, 0.0
    # the reference prints to stdout and writes H_pre.dat, H_Schur.dat and
    # Q_Schur.dat into the working directory: send both elsewhere
    sys.stdout.flush()
    saved = os.dup(1)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.dup2(2, 1)
        os.chdir(tmp)
        try:
            t = ctypes.c_double(0.0)
            for _ in range(args.warmup):
                ns.set_u(U0)  # the exponential map advances the base flow
                arn.ref_ira_map(n, fn, ctypes.cast(ctx, ctypes.c_void_p), k, m, tol, R, lm,
                                ctypes.byref(t))
            sampler.start()
            time.sleep(0.3)
            for _ in range(args.steps):
                ns.set_u(U0)  # outside the call's CUDA-event timing
                rn = arn.ref_ira_map(n, fn, ctypes.cast(ctx, ctypes.c_void_p), k, m, tol, R, lm,
                                     ctypes.byref(t))
                total += t.value
            clocks = sampler.stop()
        finally:
            libc.fflush(None)
            os.chdir(cwd)
            os.dup2(saved, 1)
            os.close(saved)
    ns.close()
    if rn < 0:
        return {"impl": "reference", "unavailable": "reference Implicit_restart_Arnoldi_GPU_data "
                                                    "run failed"}
    value = args.steps / (total / 1e3)
    mapname = (f"RK3_SSP_UV x {steps} as NSCallMatrixVector_exponential (reduced packing)"
               if expo else "RK3_SSP_UV_RHS as NSCallMatrixVector_reduced")
    return {"impl": "reference",
            "metric": ira_metric(args, N, Re, k, m),
            "value": round(value, 4), "unit": "runs/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": (f"ira_expo{steps}_kolmogorov_laminar_{N}_Re{Re:g}_k{k}_"
                                    f"m{m}_tol{tol:g}" if expo else
                                    f"ira_kolmogorov_laminar_{N}_Re{Re:g}_k{k}_m{m}_c{R}"),
                       "N": N, "Re": Re, "k": k, "m": m, "which": which, "tol": tol,
                       "max_cycles": R, "n": n,
                       "reference": "unmodified Implicit_restart_Arnoldi_GPU_data (cuBLAS, "
                                    f"LAPACK from scipy's OpenBLAS) with {mapname}, verbose "
                                    "off, sm_100a",
                       "ritz_norm": rn},
            "cpu_baseline": None,
            "e2e": {"value": round(value, 4), "unit": "runs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "clocks": clocks}


# ---------------------------------------------------------------------------
# mixed-N ensemble: 64 Kolmogorov instances, N in {32,48,64,96,128},
# Re ~ U[50, 500], seeds 0..63, 200 RK3 steps each
# ---------------------------------------------------------------------------
ENS_NS = (32, 48, 64, 96, 128)


def ensemble_instances(count, seed0=0):
    """(seed, N, Re) per instance: N and Re drawn from a generator seeded with
    the instance's seed, which also seeds its perturbation."""
    import numpy as np

    out = []
    for i in range(count):
        rng = np.random.default_rng(seed0 + i)
        out.append((seed0 + i, int(rng.choice(ENS_NS)), float(rng.uniform(50.0, 500.0))))
    return out


def ensemble_bytes(instances, steps, fp32=False):
    """P3L bytes of every instance (FP32 mode: scratch fields halved, state FP64)."""
    tot = 0
    for _, N, _ in instances:
        _, Sc, Sr = sizes(N)
        tot += steps * ((96 * Sc + 9 * Sr) if fp32 else (159 * Sc + 18 * Sr))
    return tot


def run_ours_ensemble(args, world, rank, local, pg):
    import numpy as np
    import torch

    from ns3dperiodic_b200 import Ensemble, Solver
    from ns3dperiodic_b200 import workload as W

    steps = args.steps
    inst = ensemble_instances(args.instances, rank * args.instances)
    groups = {}
    for seed, N, Re in inst:
        groups.setdefault(N, []).append((seed, Re))
    ens, fields, pristine, hosts, streams, ens_tiles = {}, {}, {}, {}, {}, {}
    for N, members in sorted(groups.items()):
        states = [W.kolmogorov_state(N, Re, seed) for seed, Re in members]
        E = Ensemble(len(members), N, N, N)
        E.set_precision(args.precision)
        if not args.no_autotune:
            E.autotune()
        ens_tiles[N] = E.tiles
        st = torch.cuda.Stream()
        E.set_stream(st)
        E.set_forcing(states[0][1])
        E.set_params([W.kolmogorov_dt(N, Re) for _, Re in members], [Re for _, Re in members])
        hosts[N] = [torch.from_numpy(np.stack([s[0][c] for s in states])).pin_memory()
                    for c in range(3)]
        pristine[N] = [h.to("cuda") for h in hosts[N]]
        fields[N] = [p.clone() for p in pristine[N]]
        ens[N], streams[N] = E, st
    torch.cuda.synchronize()
    # warm-up (graph capture, first launches), then back to the initial states
    for N, E in ens.items():
        with torch.cuda.stream(streams[N]):
            E.rk3_steps(fields[N], max(1, args.warmup))
    torch.cuda.synchronize()
    for N in ens:
        for f, p in zip(fields[N], pristine[N]):
            f.copy_(p)
    torch.cuda.synchronize()
    barrier(pg)
    main_st = torch.cuda.current_stream()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(main_st)
    ends = []
    for N, E in ens.items():
        streams[N].wait_event(ev0)
        with torch.cuda.stream(streams[N]):
            E.rk3_steps(fields[N], steps)
        e = torch.cuda.Event()
        e.record(streams[N])
        ends.append(e)
    for e in ends:
        main_st.wait_event(e)
    ev1.record(main_st)
    ev1.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1), pg)
    clocks = sampler.stop()
    energies = {N: E.diagnostics(fields[N])[0] for N, E in ens.items()}
    diverged = sorted(seed for N, members in groups.items()
                      for (seed, _), e in zip(members, energies[N]) if not math.isfinite(e))

    # the same instances one by one through the single-instance API (plain FP64)
    solo_st = torch.cuda.Stream()
    solo = {N: Solver(N, N, N) for N in groups}
    for N, S in solo.items():
        S.set_stream(solo_st)
        if not args.no_autotune:
            S.autotune()
        S.set_forcing(S.to_device(W.kolmogorov_forcing(N, N, N)))
    one = {N: [S.zeros() for _ in range(1)] for N, S in solo.items()}
    torch.cuda.synchronize()
    t_serial = 0.0
    rel_err = []
    cm = torch.cuda.stream(solo_st)
    cm.__enter__()
    for N, members in sorted(groups.items()):
        S = solo[N]
        for b, (seed, Re) in enumerate(members):
            U = one[N][0]
            for c in range(3):
                U[c].copy_(pristine[N][c][b])
            dt = W.kolmogorov_dt(N, Re)
            S.rk3_ssp(U, dt, Re, nsteps=max(1, args.warmup))  # warm the per-instance graph
            for c in range(3):
                U[c].copy_(pristine[N][c][b])
            a = torch.cuda.Event(enable_timing=True)
            z = torch.cuda.Event(enable_timing=True)
            a.record()
            S.rk3_ssp(U, dt, Re, nsteps=steps)
            z.record()
            z.synchronize()
            t_serial += a.elapsed_time(z)
            # identical to the batched result, instance by instance (with the
            # ensemble's tiles: the solo timing above used the tiles tuned for
            # one instance, which may differ)
            if args.precision != "fp32" and S.tiles != ens_tiles[N]:
                solo_tiles = S.tiles
                S.tiles = ens_tiles[N]
                for c in range(3):
                    U[c].copy_(pristine[N][c][b])
                S.rk3_ssp(U, dt, Re, nsteps=steps)
                S.tiles = solo_tiles
            if args.precision == "fp32":  # error of the FP32 ensemble against FP64 alone
                num = sum(float(torch.linalg.vector_norm(fields[N][c][b] - U[c])) ** 2
                          for c in range(3))
                den = sum(float(torch.linalg.vector_norm(U[c])) ** 2 for c in range(3))
                if math.isfinite(num) and math.isfinite(den) and den > 0:
                    rel_err.append(math.sqrt(num / den))
                continue
            for c in range(3):  # (diverged instances hold NaN in the same places)
                if not torch.equal(torch.nan_to_num(U[c]), torch.nan_to_num(fields[N][c][b])):
                    raise AssertionError(f"ensemble instance {seed} (N={N}) differs from its solo run")
    cm.__exit__(None, None, None)
    for S in solo.values():
        S.close()

    # e2e: pinned host states -> device, all solves, energies back to the host
    barrier(pg)
    t0 = time.perf_counter()
    for N, E in ens.items():
        with torch.cuda.stream(streams[N]):
            for f, h in zip(fields[N], hosts[N]):
                f.copy_(h, non_blocking=True)
            E.rk3_steps(fields[N], steps)
    e2e_energy = {N: E.diagnostics(fields[N])[0] for N, E in ens.items()}
    el = max_over_ranks(time.perf_counter() - t0, pg)
    h2d = sum(3 * h[0].numel() * 16 for h in hosts.values())
    for E in ens.values():
        E.close()

    peak, peak_src = peaks()
    B = ensemble_bytes(inst, steps, args.precision == "fp32")
    value = world * len(inst) / (ms / 1e3)
    serial = len(inst) / (t_serial / 1e3)
    return {
        "metric": f"mixed-N ensemble solves/s ({len(inst)} Kolmogorov instances, N in "
                  f"{{32,48,64,96,128}}, Re in [50,500], {steps} RK3 steps each, "
                  f"{args.precision.upper()})",
        "value": round(value, 3),
        "unit": "solves/s",
        "n_gpus": world,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms / steps, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": ("f32 (transforms, products); f64 (state, update)"
                  if args.precision == "fp32" else "f64"),
        "data": "synthetic",
        "config": {"workload": f"ensemble_{len(inst)}x_mixedN_{args.precision}",
                   "fp32_rel_l2_vs_fp64": ({"max": max(rel_err), "median":
                                            statistics.median(rel_err),
                                            "instances": len(rel_err), "tolerance": 1e-5}
                                           if rel_err else None),
                   "instances_per_N": {str(N): len(m) for N, m in sorted(groups.items())},
                   "tiles_per_N (inv_x, inv_y, fwd_y, fwd_x)": {str(N): t for N, t in
                                                                sorted(ens_tiles.items())},
                   "dt": "CFL 0.3 of the laminar peak Re/16 per instance",
                   "parallelism": f"replicas x{world}; one batched ensemble per N, each on its "
                                  "own stream",
                   "l2": f"state + scratch {sum(24 * sizes(N)[1] * len(m) for N, m in groups.items()) / 1e9:.1f} GB > 126 MB L2",
                   "serial_solves_per_s": round(serial, 3),
                   "serial_protocol": "the same instances one by one, ns3d_rk3_steps of a "
                                      "single-instance handle (plain FP64), CUDA events; "
                                      "FP64 batched results identical to them",
                   "speedup_vs_serial": round(value / world / serial, 3),
                   "diverged_instances": diverged,
                   "diverged_note": "under-resolved high-Re instances overflow within the "
                                    "200 steps; the reference's RK3_SSP does the same "
                                    "arithmetic (the timing covers them all)",
                   "energy_first": {str(N): (float(e[0]) if math.isfinite(e[0]) else None)
                                    for N, e in energies.items()}},
        "roofline": {"bound": "hbm", "kernel": "all passes (P3L bytes of every instance)",
                     "achieved": round(B / (ms / 1e3) / 1e9, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(B / (ms / 1e3) / 1e9 / peak, 4), "traffic": None,
                     "peak_source": peak_src, "alg_bytes_per_step": B // steps},
        "e2e": {"value": round(world * len(inst) / el, 3), "unit": "solves/s",
                "h2d_bytes_per_step": round(h2d / steps, 1),
                "d2h_bytes_per_step": round(16 * len(inst) / steps, 1),
                "protocol": "pinned host initial states -> device, all solves, energy and "
                            "dissipation per instance -> host; wall clock"},
        "gpu_launches": 15 * steps * len(groups),
        "clocks": clocks,
    }


def run_reference_ensemble(args, world, rank, local, pg):
    from oracle import ref_lib

    from ns3dperiodic_b200 import workload as W

    if rank != 0:
        return None
    if not ref_lib.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libns3d_ref.so not built "
                                                    "(needs the reference tree at build time)"}
    steps = args.steps
    inst = ensemble_instances(args.instances, 0)
    sampler = ClockSampler(local)
    sampler.start()
    total_ms = 0.0
    diverged = []
    for seed, N, Re in inst:
        U, F = W.kolmogorov_state(N, Re, seed)
        with ref_lib.RefSolver(N, N, N) as R:
            R.set_f(F)
            R.set_u(U)
            R.time_rk3(max(1, args.warmup), W.kolmogorov_dt(N, Re), Re)
            R.set_u(U)
            total_ms += R.time_rk3(steps, W.kolmogorov_dt(N, Re), Re)
            if not math.isfinite(R.diag()[0]):
                diverged.append(seed)
    clocks = sampler.stop()
    value = len(inst) / (total_ms / 1e3)
    return {"impl": "reference",
            "metric": f"mixed-N ensemble solves/s ({len(inst)} Kolmogorov instances, N in "
                      f"{{32,48,64,96,128}}, Re in [50,500], {steps} RK3 steps each, FP64)",
            "value": round(value, 3), "unit": "solves/s", "n_gpus": 1, "steps": steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / steps, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"ensemble_{len(inst)}x_mixedN_fp64",
                       "reference": "unmodified RK3_SSP with cuFFT, one instance at a time "
                                    "(its state is file-static), CUDA events around each run",
                       "diverged_instances": diverged},
            "e2e": {"value": round(value, 3), "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "clocks": clocks}


# ---------------------------------------------------------------------------
# serving: Poisson arrivals of tangent-integration (JVP) requests
# ---------------------------------------------------------------------------
SERVE_NS = (64, 96, 128)


def serving_requests(rate, window, seed=0):
    """(N, Re, T, seed, arrival): N in {64,96,128}, Re in {100,200,400},
    T ~ U[1, 5], Poisson arrivals of mean `rate` per second over `window` s."""
    import numpy as np

    rng = np.random.default_rng(seed)
    out, t, i = [], 0.0, 0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > window:
            return out
        out.append((int(rng.choice(SERVE_NS)), float(rng.choice((100.0, 200.0, 400.0))),
                    float(rng.uniform(1.0, 5.0)), i, t))
        i += 1


def latency_stats(res):
    import numpy as np

    done = [r for r in res if r["done"] >= 0.0]
    if not done:
        return {"completed": 0}
    lat = np.array([r["done"] - r["arrival"] for r in done])
    wait = np.array([r["admitted"] - r["arrival"] for r in done])
    return {"completed": len(done),
            "p50_s": round(float(np.percentile(lat, 50)), 4),
            "p99_s": round(float(np.percentile(lat, 99)), 4),
            "mean_wait_s": round(float(wait.mean()), 4),
            "per_N": {str(N): sum(1 for r in done if r["N"] == N) for N in SERVE_NS}}


def jvp_bytes(N):
    _, Sc, Sr = sizes(N)
    return 330 * Sc + 30 * Sr


def run_ours_serving(args, world, rank, local, pg):
    import torch

    from ns3dperiodic_b200 import Server, Solver, request_steps
    from ns3dperiodic_b200 import workload as W

    slots = [int(x) for x in args.slots.split(",")]
    reqs = serving_requests(args.rate, args.window, seed=rank)
    peak, peak_src = peaks()

    # 1. the offered load (far beyond one GPU at 200/s): completions in the window
    sampler = ClockSampler(local)
    sampler.start()
    with Server(SERVE_NS, capacity=slots, hbm_fraction=0.8) as srv:
        if not args.no_autotune:
            srv.autotune()
        caps = {N: srv.capacity(N) for N in SERVE_NS}
        srv.submit([(N, Re, T, sd, a, 0) for N, Re, T, sd, a in reqs])
        t0 = time.perf_counter()
        srv.run(args.window)
        wall = time.perf_counter() - t0
        res = srv.results()
        work = {N: srv.instance_steps(N) for N in SERVE_NS}
    clocks = sampler.stop()
    done = [r for r in res if r["done"] >= 0.0]
    wall = max_over_ranks(wall, pg)
    thr = world * len(done) / wall
    step_bytes = sum(jvp_bytes(N) * k for N, k in work.items())
    sat = latency_stats(res)

    # 2. below saturation: 60% of the measured completion rate, drained
    sub_rate = max(0.6 * len(done) / wall, 0.05)
    reqs2 = serving_requests(sub_rate, args.window, seed=1000 + rank)
    with Server(SERVE_NS, capacity=slots, hbm_fraction=0.8) as srv:
        if not args.no_autotune:
            srv.autotune()
        if reqs2:
            srv.submit([(N, Re, T, sd, a, 0) for N, Re, T, sd, a in reqs2])
            srv.run()
        sub = latency_stats(srv.results())
    sub["offered_rate_per_s"] = round(sub_rate, 3)
    sub["offered"] = len(reqs2)

    # 3. plain FP64 serial: the first requests of the stream, one at a time
    sample = reqs[:6]
    serial_s = 0.0
    st = torch.cuda.Stream()
    for N, Re, T, sd, _ in sample:
        with Solver(N, N, N) as S:
            S.set_stream(st)
            S.set_forcing(S.to_device(W.kolmogorov_forcing(N, N, N)))
            with torch.cuda.stream(st):
                U, V = S.request_fields(Re, sd)
                a = torch.cuda.Event(enable_timing=True)
                z = torch.cuda.Event(enable_timing=True)
                a.record()
                S.rk3_ssp_uv(U, V, W.kolmogorov_dt(N, Re), Re,
                             nsteps=request_steps(N, Re, T))
                z.record()
            z.synchronize()
            serial_s += a.elapsed_time(z) / 1e3
    serial = len(sample) / serial_s
    return {
        "metric": "JVP-request serving: completions/s with p50/p99 latency (Poisson "
                  f"{args.rate:g}/s, N in {{64,96,128}}, Re in {{100,200,400}}, T ~ U[1,5], FP64)",
        "value": round(thr, 4),
        "unit": "completions/s",
        "n_gpus": world,
        "steps": len(done),
        "warmup": 0,
        "ms_per_step": round(1e3 / thr, 3) if thr > 0 else None,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "serving_jvp_poisson",
                   "offered": len(reqs), "window_s": args.window,
                   "slots": {str(N): caps[N] for N in SERVE_NS},
                   "admission": "slots reserved from 80% of the free HBM, capped per grid; "
                                "first come first served per grid; continuous batching "
                                "per step",
                   "saturated": sat, "sub_saturation": sub,
                   "instance_steps": {str(N): k for N, k in work.items()},
                   "serial_completions_per_s": round(serial, 4),
                   "serial_protocol": "the first 6 requests one at a time through "
                                      "ns3d_jvp_steps of a single-grid handle (plain FP64), "
                                      "CUDA events",
                   "speedup_vs_serial": round(thr / world / serial, 3)},
        "roofline": {"bound": "hbm", "kernel": "all passes of every JVP step the server ran "
                                               "in the window (330 S_c + 30 S_r per step)",
                     "achieved": round(step_bytes / wall / 1e9, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(step_bytes / wall / 1e9 / peak, 4),
                     "traffic": None, "peak_source": peak_src},
        "e2e": {"value": round(thr, 4), "unit": "completions/s", "h2d_bytes_per_step": 48,
                "d2h_bytes_per_step": 8,
                "protocol": "requests (N, Re, T, seed) from the host, fields made on the "
                            "device, |v(T)| back per request; wall clock"},
        "gpu_launches": None,
        "clocks": clocks,
    }


def main():
    args = parse()
    world, rank, local, pg = dist_setup(args)
    try:
        if args.workload == "serving":
            if args.impl == "reference":
                line = {"impl": "reference", "unavailable": "the reference has no request "
                                                            "server; its one-at-a-time JVP is "
                                                            "the serial figure of our line"}
            else:
                line = run_ours_serving(args, world, rank, local, pg)
        elif args.workload == "ensemble":
            if args.impl == "reference":
                line = run_reference_ensemble(args, world, rank, local, pg)
            else:
                line = run_ours_ensemble(args, world, rank, local, pg)
        elif args.workload == "ira":
            if args.impl == "reference":
                line = run_reference_ira(args, world, rank, local, pg)
            else:
                line = run_ours_ira(args, world, rank, local, pg)
                if rank == 0 and world == 1 and not args.no_cpu_baseline:
                    _, _, _, _, _, _, _, dt, steps = ira_setup(args)
                    line["cpu_baseline"] = cpu_baseline_ira(
                        args.ira_N, args.Re, args.ira_m, line["config"]["map_calls_per_run"],
                        args.seed, steps, dt)
        elif args.workload == "arnoldi":
            if args.impl == "reference":
                line = run_reference_arnoldi(args, world, rank, local, pg)
            else:
                line = run_ours_arnoldi(args, world, rank, local, pg)
                if rank == 0 and world == 1 and not args.no_cpu_baseline:
                    line["cpu_baseline"] = cpu_baseline_arnoldi(args.n_arnoldi, args.m_arnoldi,
                                                                args.seed)
        elif args.impl == "reference":
            line = run_reference(args, world, rank, local, pg)
        else:
            line = run_ours(args, world, rank, local, pg)
            if rank == 0 and world == 1 and not args.no_cpu_baseline:
                line["cpu_baseline"] = cpu_baseline(args.N, args.Re, args.seed)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
