#!/usr/bin/env python
"""Benchmark: seconds per parquet iteration of the TUPS loop on one B200.

Workload (default): the plain PA Hubbard loop on an 8x8 k grid with 5 form
factors and 32 fermionic / 16 bosonic Matsubara frequencies, t=1, t'=0,
U=2, beta=5, n=1, linear mixing 0.5, complex128 storage.  A step is one
parquet iteration (Green's function + mu bisection, BSE, Phi(R), parquet
equation, Schwinger-Dyson, convergence check, vertex update).  The state
(~0.9 GB) is resident in HBM and larger than L2, so no L2 flush is needed.
The timed iterations replay a CUDA graph of the iteration captured in the
warm-up (``--no-graph``: kernel by kernel); per-phase times come from K
further iterations launched kernel by kernel with phase events.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl {tups,reference}]

Prints one JSON line (rank 0).  ``--impl reference`` times the CPU
restatement of the reference (the reference's Fortran cannot be built in
this image) on the host cores.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    # name: prms fields
    "pa_8x8_nl5_nf32": dict(beta=5.0, U=2.0, nParticle=1.0, Nx=8, Nf=32, neighbours=2, f_damping=0.5,
                            use_U2=True, ite_max=100000),
    "pa_4x4_nl1_nf16": dict(beta=2.0, U=2.0, nParticle=1.0, Nx=4, Nf=16, neighbours=1, f_damping=0.5,
                            use_U2=True, ite_max=100000),
    # 9 form factors on the 8x8 lattice: the crossing and BSE tile configurations
    # of the 16x16 loop on a case small enough for kernel profiling
    "pa_8x8_nl9_nf32": dict(beta=5.0, U=2.0, nParticle=1.0, Nx=8, Nf=32, neighbours=3, f_damping=0.5,
                            use_U2=True, ite_max=100000),
    "pa_16x16_nl9_nf64": dict(beta=10.0, U=3.0, nParticle=0.85, Nx=16, Nf=64, neighbours=3, f_damping=0.5,
                              use_U2=True, ite_max=100000, tprime=-0.2),
}
DEFAULT_WORKLOAD = "pa_8x8_nl5_nf32"
METRIC = "s/parquet-iter"
METRIC_FULL = "s/parquet-iter & BSE TFLOP/s: split-precision vs FP64 GPU path, Σ rel.err≤1e-10"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def fp64_peak_tflops(device: int) -> float:
    """cuBLAS ZGEMM throughput (torch complex128 matmul, 4096^3, best of 5)."""
    import torch
    n = 4096
    a = torch.randn(n, n, dtype=torch.complex128, device=f"cuda:{device}")
    b = torch.randn(n, n, dtype=torch.complex128, device=f"cuda:{device}")
    for _ in range(2):
        a @ b
    torch.cuda.synchronize(device)
    best = math.inf
    for _ in range(5):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        a @ b
        e.record()
        torch.cuda.synchronize(device)
        best = min(best, s.elapsed_time(e))
    del a, b
    torch.cuda.empty_cache()
    return 8.0 * n ** 3 / (best * 1e-3) / 1e12


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except ValueError:
            pass
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


def pae_valid_count(d: dict, ibz: np.ndarray) -> int:
    """Number of (slot, nu1, nu2, target pair, contribution type) that the
    crossing kernel contracts (each over Nl^4 NR terms per target)."""
    Nf = d["Nf"]
    nh = Nf // 2
    W = ibz[:, 2][:, None, None]
    n1 = np.arange(1, Nf + 1)[None, :, None]
    n2 = np.arange(1, Nf + 1)[None, None, :]
    tot = 0
    for ww, lo in ((n2 - n1 + 1, 1), (n1 - n2 + 1, 2), (n1 + n2 + W - Nf - 1, 1), (Nf + 3 - n1 - n2 - W, 2),
                   (W - n1 - n2 + Nf + 1, 1), (n1 + n2 - W - Nf + 1, 2), (n2 - n1 + 1, 1), (n1 - n2 + 1, 2)):
        ww = np.broadcast_to(ww, (len(ibz), Nf, Nf))
        tot += int(np.count_nonzero((ww >= lo) & (ww <= nh)))
    return tot


def read_traffic(kernel: str, workload: str):
    """Per-launch DRAM bytes of a kernel from the committed ncu summary
    ``profiles/traffic.txt`` (lines: kernel workload bytes_per_launch)."""
    p = ROOT / "profiles" / "traffic.txt"
    if not p.exists():
        return None
    for ln in p.read_text().splitlines():
        f = ln.split()
        if len(f) >= 3 and not ln.startswith("#") and f[0] == kernel and f[1] == workload:
            try:
                return float(f[2])
            except ValueError:
                return None
    return None


def oracle_params(wl: dict):
    from oracle import tups_oracle as O
    kw = {k: v for k, v in wl.items() if k in O.Params.__dataclass_fields__}
    return O.Params(**kw)


CPU_PORT_SAMPLE = ("oracle port on the host cores: the numpy restatement of the reference with its crossing "
                   "and Phi(R) compiled (C++/OpenMP loop nests, oracle/port) and the BSE's ZGEMMs on OpenBLAS")


def cpu_oracle_seconds_per_iteration(wl: dict, timed_iterations: int = 1, warm_iterations: int = 1):
    """Time the oracle port (oracle.port.iteration): warm (untimed)
    iterations, then timed ones."""
    from oracle import tups_oracle as O
    from oracle import port as OP
    OP.threads(os.cpu_count() or 1)
    st = O.initialize(oracle_params(wl))
    for ite in range(warm_iterations):
        OP.iteration(st, ite)
    t0 = time.perf_counter()
    for ite in range(warm_iterations, warm_iterations + timed_iterations):
        OP.iteration(st, ite)
    return (time.perf_counter() - t0) / timed_iterations


def blas_threads() -> int:
    try:
        from threadpoolctl import threadpool_info
        n = [i.get("num_threads", 1) for i in threadpool_info() if i.get("user_api") == "blas"]
        if n:
            return int(max(n))
    except Exception:
        pass
    return os.cpu_count() or 1


def workload_config(wl_name: str, wl: dict, ws: int) -> dict:
    """The `config` record, identical in both arms: the prms fields, the
    derived sizes (from the host-side tables, no device needed) and the L2
    statement."""
    from tups_b200 import Params
    from tups_b200.parquet import host_tables
    d = host_tables(Params(**{k: v for k, v in wl.items() if k in Params.__dataclass_fields__}))["dims"]
    Nz, Nb = d["Nz"], d["Nb"]
    return {"workload": wl_name, **{k: wl[k] for k in ("Nx", "Nf", "neighbours", "beta", "U", "nParticle")},
            "tprime": wl.get("tprime", 0.0), "Nl": d["Nl"], "Nz": Nz, "Nred": d["Nred"], "NR": d["NR"],
            "l2": "resident state ~%.2f GB > 126 MB L2; no flush" % ((8 * Nz * Nz * Nb * 16) / 1e9),
            "parallelism": "replicas" if ws > 1 else "single process"}


def fortran_toolchain() -> dict:
    """Which Fortran/MPI compilers this host has (the reference needs mpif90,
    MKL and HDF5-Fortran)."""
    import shutil
    return {t: shutil.which(t) for t in ("gfortran", "mpif90", "mpifort", "ifort", "ifx", "h5fc")}


def run_reference(args, wl_name: str, wl: dict):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    steps, warm = args.steps, args.warmup
    spi = cpu_oracle_seconds_per_iteration(wl, timed_iterations=steps, warm_iterations=warm)
    cores = max(blas_threads(), os.cpu_count() or 1)
    tools = fortran_toolchain()
    line = {
        "impl": "reference", "metric": METRIC, "metric_full": METRIC_FULL, "value": spi, "unit": "s/iter",
        "n_gpus": ws, "steps": steps, "warmup": warm, "ms_per_step": spi * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(wl_name, wl, ws),
        "cpu_baseline": {"value": spi, "unit": "s/iter", "cores": cores, "kind": "port",
                         "sample": f"{steps} iteration(s) after {warm} untimed; " + CPU_PORT_SAMPLE},
        "reference_toolchain": tools,
        "reference_note": ("the Fortran reference needs mpif90 + MKL + HDF5-Fortran; none of the compilers "
                           "probed here is present" if not any(tools.values()) else
                           "a Fortran compiler is present; the port is still the timed arm"),
        "e2e": {"value": spi, "unit": "s/iter", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_tups(args, wl_name: str, wl: dict):
    import torch
    from tups_b200 import replicas
    ws, rank, local = dist_env()
    device = local
    torch.cuda.set_device(device)
    ranks = replicas.init("nccl")
    from tups_b200 import Params, Solver, load
    from tups_b200.parquet import tuning_table
    load()
    peak64 = fp64_peak_tflops(device)
    params = Params(**{k: v for k, v in wl.items() if k in Params.__dataclass_fields__})
    sol = Solver(params, device=device)
    if args.crossing_products:
        sol.set_crossing_products(args.crossing_products)
    if args.bse_slices:
        sol.set_bse_precision(args.bse_slices)
    K, W = args.steps, args.warmup
    # iterations replay a captured CUDA graph (captured in the warm-up)
    sol.set_graph(not args.no_graph)
    for ite in range(W):
        sol.iteration(ite)
    sol.synchronize()
    # ---- timed region: K iterations, device-resident state ----
    l0 = sol.kernel_launches
    replicas.barrier(ranks)
    torch.cuda.synchronize(device)
    sol.synchronize()
    clocks = ClockSampler(device)
    clocks.start()
    sol.record_event(0)
    infos = []
    for k in range(K):
        infos.append(sol.iteration(W + k))
    sol.record_event(1)
    ms = sol.event_elapsed_ms(0, 1)
    sol.synchronize()
    torch.cuda.synchronize(device)
    clk = clocks.stop()
    launches = sol.kernel_launches - l0
    # ---- e2e: Sigma from pinned host, one iteration, Sigma back to pinned host ----
    nt = sol.Nt
    h_in = torch.empty(2 * nt, dtype=torch.float64, pin_memory=True).numpy().view(np.complex128)
    h_out = torch.empty(2 * nt, dtype=torch.float64, pin_memory=True).numpy().view(np.complex128)
    h_in[:] = sol.Sigma
    replicas.barrier(ranks)
    sol.synchronize()
    sol.record_event(2)
    for k in range(K):
        sol.set_sigma_from(h_in)
        sol.iteration(W + K + k)
        sol.get_sigma_into(h_out)
        h_in[:] = h_out
    sol.record_event(3)
    ms_e2e = sol.event_elapsed_ms(2, 3)
    # ---- per-phase device times (events around each phase; no graph) ----
    sol.set_timing(True)
    for k in range(K):
        sol.iteration(W + 2 * K + k)
    phases = sol.phase_times()
    sol.set_timing(False)
    readout_ms = None
    if args.with_readout:
        # one output iteration with the chi readout (off the timed path)
        ite = W + 2 * K
        ite += (5 - ite % 5) % 5
        sol.record_event(6)
        sol.iteration(ite, readout=True)
        sol.record_event(7)
        readout_ms = sol.event_elapsed_ms(6, 7)
    # ---- max over ranks ----
    ms, ms_e2e = replicas.max_over_ranks(ranks, [ms, ms_e2e])
    value = replicas.seconds_per_iteration(ms, K, ws)
    e2e_value = replicas.seconds_per_iteration(ms_e2e, K, ws)
    d = sol.dims
    # ---- roofline of the kernels ----
    tab = sol.tables()
    n_valid = pae_valid_count(d, tab["ibz"])
    Nz, Nl, NR, Nb, nh = d["Nz"], d["Nl"], d["NR"], d["Nb"], d["Nf"] // 2
    kern = {}
    ms_g, c_g = phases["bse_gemm"]
    if c_g:
        # per launch: 16 Nz^3 for each (q, r) instance; launches split the Nb slots in chunks
        fl = 16.0 * Nz ** 3 * 4 * Nb / (c_g / K)
        kern["k_bse_gemm"] = {"ms": ms_g, "timed_intervals": c_g, "bound": "tensor", "unit": "TFLOP/s",
                              "achieved": fl / (ms_g / c_g * 1e-3) / 1e12, "peak": peak64,
                              "peak_source": "FP64 cuBLAS ZGEMM 4096^3 measured in this run"}
    ms_p, c_p = phases["pae"]
    if c_p:
        fl = 8.0 * 2 * Nl ** 4 * NR * n_valid / (c_p / K)
        kern["k_pae_mma"] = {"ms": ms_p, "timed_intervals": c_p, "bound": "tensor", "unit": "TFLOP/s",
                             "achieved": fl / (ms_p / c_p * 1e-3) / 1e12, "peak": peak64,
                             "peak_source": "FP64 cuBLAS ZGEMM 4096^3 measured in this run (FP64 pipe)",
                             "note": "one interval per iteration: k_pae_base and the two family launches"}
    ms_r, c_r = phases["phir"]
    if c_r:
        by = 16.0 * (4 * Nb * Nz * Nz + 4 * Nz * Nz * nh * NR)
        pk = measured_peaks()
        kern["k_phir"] = {"ms": ms_r, "timed_intervals": c_r, "bound": "hbm", "unit": "GB/s",
                          "achieved": by / (ms_r / c_r * 1e-3) / 1e9, "peak": pk.get("hbm_gbs"),
                          "peak_source": "MEASURED_PEAKS.json hbm_gbs" + (" (fallback)" if pk.get("fallback") else "")}
    dom = max(kern, key=lambda k: kern[k]["ms"]) if kern else None
    roof = None
    if dom:
        kd = kern[dom]
        roof = {"kernel": dom, "bound": kd["bound"], "achieved": kd["achieved"], "peak": kd["peak"],
                "unit": kd["unit"], "frac": kd["achieved"] / kd["peak"] if kd["peak"] else None,
                "traffic": read_traffic(dom, wl_name), "peak_source": kd["peak_source"]}
    bse_tflops = kern.get("k_bse_gemm", {}).get("achieved")
    split = None
    conv = None
    graph = None
    if not args.no_split and ws == 1:
        split = split_iterations(params, device, K, W, Nz, Nb, peak64)
        graph = graph_iterations(params, device, K, W)
    if ws == 1 and (Nz <= 256 or args.convergence) and not args.no_convergence:
        conv = to_convergence(params, device)
    target = None
    if ws == 1 and not args.no_target and wl_name != TARGET_WORKLOAD:
        sol.close()
        target = target_record(device)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        sec = cpu_oracle_seconds_per_iteration(wl, timed_iterations=2)
        cpu = {"value": sec, "unit": "s/iter", "cores": max(blas_threads(), os.cpu_count() or 1), "kind": "port",
               "sample": "2 iterations (ite 1-2, after an untimed ite 0) of the same workload; " + CPU_PORT_SAMPLE}
    if rank == 0:
        line = {
            "metric": METRIC, "metric_full": METRIC_FULL, "value": value, "unit": "s/iter", "n_gpus": ws,
            "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if not args.bse_slices else f"f64 + int8x{args.bse_slices} BSE GEMM",
            "data": "synthetic",
            "config": workload_config(wl_name, wl, ws),
            "bse_tflops": bse_tflops,
            "split_precision": split,
            "cuda_graph": graph,
            "to_convergence": conv,
            "target": target,
            "roofline": roof,
            "kernels": kern,
            "phase_ms_per_iter": {p: v[0] / K for p, v in phases.items()},
            "phase_note": "per-phase CUDA-event times from K further iterations launched kernel by kernel",
            "launch_mode": "kernel by kernel" if args.no_graph else "CUDA graph per iteration (captured in warm-up)",
            "e2e": {"value": e2e_value, "unit": "s/iter", "h2d_bytes_per_step": 16 * nt,
                    "d2h_bytes_per_step": 16 * nt + 2 * 16 * 8,
                    "api": "Solver.set_sigma_from(pinned) + Solver.iteration + Solver.get_sigma_into(pinned)"},
            "gpu_launches": launches,
            "clocks": clk,
            "tuning": tuning_table(),
            "readout_iteration_ms": readout_ms,
            "cpu_baseline": cpu,
            "last_conv": {k: infos[-1][k] for k in ("rel_sig_max", "dsigma_inf", "mu")} if infos else None,
        }
        print(json.dumps(line), flush=True)
    sol.close()
    replicas.finish(ranks)


SPLIT_SLICES = (3, 5, 7, 8)


def split_iterations(params, device: int, K: int, W: int, Nz: int, Nb: int, peak64: float) -> dict:
    """The same K iterations with the BSE GEMM on int8 slices (tcgen05 kind::i8):
    device ms per iteration and per BSE GEMM phase for each slice count."""
    from tups_b200 import Solver
    out = {}
    for s in SPLIT_SLICES:
        sol = Solver(params, device=device)
        sol.set_bse_precision(s)
        for ite in range(W):
            sol.iteration(ite)
        sol.synchronize()
        sol.set_timing(True)
        sol.record_event(0)
        for k in range(K):
            sol.iteration(W + k)
        sol.record_event(1)
        ms = sol.event_elapsed_ms(0, 1) / K
        ph = sol.phase_times()
        sol.close()
        gemm_ms = ph["bse_gemm"][0] / K
        flops = 16.0 * Nz ** 3 * 4 * Nb
        out[str(s)] = {"ms_per_iter": ms, "bse_gemm_ms": gemm_ms,
                       "bse_effective_tflops": flops / (gemm_ms * 1e-3) / 1e12,
                       "int8_tops": 2.0 * s * (s + 1) / 2 * Nz * (2 * Nz) * (4 * Nz) * 4 * Nb / (gemm_ms * 1e-3) / 1e12,
                       "gemm_rel_err_model": 10.0 ** (1.1 - 2.0 * s)}
    out["fp64_peak_tflops"] = peak64
    out["note"] = ("effective TFLOP/s = FP64-equivalent 16 Nz^3 per (q, r) / split GEMM time; int8_tops = "
                   "s(s+1)/2 slice products x 2 M (2N) (2K) / time")
    return out


def graph_iterations(params, device: int, K: int, W: int) -> dict:
    """The same K iterations replayed from a captured CUDA graph (one host
    synchronisation per iteration)."""
    from tups_b200 import Solver
    sol = Solver(params, device=device)
    sol.set_graph(True)
    for ite in range(W):
        sol.iteration(ite)
    sol.synchronize()
    l0 = sol.kernel_launches
    sol.record_event(0)
    for k in range(K):
        sol.iteration(W + k)
    sol.record_event(1)
    ms = sol.event_elapsed_ms(0, 1) / K
    launches = (sol.kernel_launches - l0) / K
    sol.close()
    return {"ms_per_iter": ms, "kernels_per_iter": launches}


def _final_state(sol, n: int, full_vertices: bool, sample_slots) -> dict:
    """One more iteration of a converged loop with the readout (outside any
    timed region): Sigma, F_r, Gamma_r (after the vertex update), chi0 and
    sus_r.  Large grids keep only the sampled slots of the vertices."""
    sol.iteration(n, readout=True)
    out = {"Sigma": sol.Sigma}
    for r in "dmst":
        if full_vertices:
            out["F_" + r] = sol.F(r)
            out["Gamma_" + r] = sol.G(r)
        else:
            out["F_" + r] = np.stack([sol.vertex_slots(r, 0, q)[:, :, 0] for q in sample_slots])
            out["Gamma_" + r] = np.stack([sol.vertex_slots(r, 1, q)[:, :, 0] for q in sample_slots])
        out["sus_" + r] = sol.sus(r)
    out.update(sol.chi0())
    return out


def _rel(a, b) -> float:
    den = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b))) / den if den > 0 else float(np.max(np.abs(a - b)))


def to_convergence(params, device: int, conv_abs: float = 1e-10, ref_abs: float = 1e-13, max_iter: int = 3000,
                   graph: bool = True, ref_extra: int = 80) -> dict:
    """Wall time (device events around the host-driven loop) and iterations to
    max|dSigma| < conv_abs from the reference's initial state: FP64 BSE vs the
    precision ladder, both replaying CUDA graphs.  Then the converged states,
    max-norm relative error per quantity (Sigma, F_r and Gamma_r of each
    channel, the chi0 bubble and the susceptibilities sus_r of the readout):
    the ladder's against the FP64 loop's, and both against the fixed point
    itself, the FP64 loop continued (untimed) to max|dSigma| < ref_abs.  The
    FP64 path equals the oracle to 1e-12 per phase."""
    from dataclasses import replace
    from tups_b200 import Solver
    p = replace(params, conv_abs=conv_abs, ite_max=10 ** 6)
    res = {"conv_abs": conv_abs}
    fin = {}
    for name in ("fp64", "ladder"):
        sol = Solver(p, device=device)
        sol.set_graph(graph)
        if name == "ladder":
            sol.set_bse_precision(0, ladder=True)
        used, dsig = [], []
        sol.synchronize()
        sol.record_event(4)
        n, ok = 0, False
        while n < max_iter:
            used.append(sol.bse_slices)
            ci = sol.iteration(n)
            dsig.append(ci["dsigma_inf"])
            n += 1
            if ci["converged"]:
                ok = True
                break
        sol.record_event(5)
        sec = sol.event_elapsed_ms(4, 5) * 1e-3
        full = sol.Nz * sol.Nz * sol.Nb * 16 * 8 < 4e9
        slots = [0, sol.Nb // 2, sol.Nb - 1]
        fin[name] = _final_state(sol, n, full, slots)
        res[name] = {"iterations": n, "seconds": sec, "s_per_iter": sec / n, "converged": ok}
        if name == "ladder":
            res[name]["slices_per_iteration"] = used
        else:
            # contraction rate of the loop near its fixed point
            tail = [d for d in dsig[-20:] if d > 0]
            if len(tail) >= 2:
                res[name]["contraction_rate"] = float((tail[-1] / tail[0]) ** (1.0 / (len(tail) - 1)))
            # continue towards the fixed point until max|dSigma| < ref_abs, or
            # until it stops falling (the FP64 rounding floor: no new minimum
            # in 10 iterations), or for at most ref_extra more iterations
            m, best, since, why = n, float("inf"), 0, "iteration cap"
            while m < n + ref_extra:
                ci = sol.iteration(m)
                m += 1
                d = ci["dsigma_inf"]
                if d < ref_abs:
                    best, why = d, "reached"
                    break
                if d < best:
                    best, since = d, 0
                else:
                    since += 1
                    if since >= 10:
                        why = "rounding floor"
                        break
            fin["fixed"] = _final_state(sol, m, full, slots)
            res["fixed_point"] = {"target_max_dsigma": ref_abs, "max_dsigma_reached": best, "iterations": m,
                                  "stopped": why, "note": "the FP64 loop continued past its stop, untimed"}
        sol.close()
    errs = {k: _rel(fin["ladder"][k], fin["fp64"][k]) for k in fin["fp64"]}
    res["rel_err_ladder_vs_fp64"] = errs
    res["rel_err_vs_fixed_point"] = {name: {k: _rel(fin[name][k], fin["fixed"][k]) for k in fin["fixed"]}
                                     for name in ("fp64", "ladder")}
    res["rel_err_note"] = ("max-norm relative differences of converged states, both loops stopped at max|dSigma| < "
                           f"{conv_abs:g}; vertices " + ("whole" if full else "at slots [0, Nb/2, Nb-1]") +
                           "; Gamma_r after the vertex update; chi0/sus from the readout of one more iteration")
    res["sigma_rel_err_ladder_vs_fp64"] = errs["Sigma"]
    res["speedup_ladder_vs_fp64"] = res["fp64"]["seconds"] / res["ladder"]["seconds"]
    res["launch_mode"] = "CUDA graph per iteration" if graph else "kernel by kernel"
    return res


TARGET_WORKLOAD = "pa_16x16_nl9_nf64"


def target_record(device: int) -> dict:
    """The 16x16 k / 9 form factor / 64 frequency loop (t' = -0.2, n = 0.85,
    U = 3, beta = 10): FP64 vs precision-ladder time to max|dSigma| < 1e-11
    and the converged states' errors, with its own clock samples.  The
    learned warm start is trained on the 8x8 / 5 form-factor grid and has no
    network for this grid, so the ladder runs from the cold start."""
    from tups_b200 import Params
    wl = WORKLOADS[TARGET_WORKLOAD]
    params = Params(**{k: v for k, v in wl.items() if k in Params.__dataclass_fields__})
    clocks = ClockSampler(device)
    clocks.start()
    t0 = time.perf_counter()
    # max|dSigma| < 1e-11: with the loop's contraction rate near 0.87 both
    # runs then stop within about 1e-10 of the fixed point in Sigma
    conv = to_convergence(params, device, conv_abs=1e-11, max_iter=400)
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    return {"workload": TARGET_WORKLOAD,
            "config": {k: wl[k] for k in ("Nx", "Nf", "neighbours", "beta", "U", "nParticle", "tprime")},
            "fp64_s_per_iter": conv["fp64"]["s_per_iter"], "to_convergence": conv, "host_wall_s": wall,
            "warm_start": "not run: the network is trained on the 8x8 / 5 form-factor grid only",
            "clocks": clk}


LU_WORKLOAD = "bse_lu_1024"
SPLIT_LU_SLICES = (3, 4, 5, 6)
SPLIT_LU_TOL = 1e-12


def run_bse_batched(args):
    """Standalone batched BSE in its LU form: 1024 (q, Omega) instances on an
    8x8 lattice, N_ff in {1,5,9,13} by seed, 64 frequencies (n = 64..832),
    Hermitian Gaussian Gamma scaled to rho(Gamma chi) = 0.9, chi the beta = 10
    bare bubble.  One step = the whole batch, F = (1 - Gamma chi)^{-1} Gamma."""
    ws, rank, local = dist_env()
    if args.impl == "reference" and rank != 0:
        return
    from tups_b200.bse_batched import algorithmic_flops, make_instances
    from oracle import lu as LU
    workers = min(16, os.cpu_count() or 1)
    inst = make_instances(n_q=args.lu_q, n_w=16, nf=64, seed=0, workers=workers)
    flops = algorithmic_flops(inst.n)
    # CPU sample: two instances of each size, LAPACK zgetrf/zgetrs on all host threads
    sample = []
    for n in sorted(set(inst.n.tolist())):
        sample += [int(i) for i in np.nonzero(inst.n == n)[0][:2]]
    t0 = time.perf_counter()
    ref = {i: LU.bse_lu(inst.gamma[i], inst.chi[i], 1.0) for i in sample}
    cpu_s = time.perf_counter() - t0
    cpu_tf = algorithmic_flops(inst.n[sample]) / cpu_s / 1e12
    cpu = {"value": cpu_tf, "unit": "TFLOP/s", "cores": blas_threads(), "kind": "port",
           "sample": f"{len(sample)} instances (2 per size {sorted(set(inst.n.tolist()))}), scipy/OpenBLAS "
                     "zgetrf+zgetrs, FP64"}
    cfg = {"workload": LU_WORKLOAD, "instances": int(len(inst.n)), "n_sizes": sorted(set(inst.n.tolist())),
           "Nnu": 64, "lattice": "8x8", "beta": 10.0, "rho": 0.9, "l2": "inputs 4.7 GB > L2; no flush"}
    if args.impl == "reference":
        line = {"impl": "reference", "metric": "BSE TFLOP/s", "value": cpu_tf, "unit": "TFLOP/s", "n_gpus": ws,
                "steps": 1, "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic", "config": cfg, "cpu_baseline": cpu,
                "e2e": {"value": cpu_tf, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    import torch
    from tups_b200.bse_batched import LuBatch
    device = local
    torch.cuda.set_device(device)
    peak64 = fp64_peak_tflops(device)
    batch = LuBatch(inst, device)
    K, W = args.steps, args.warmup
    batch.run(check=True)
    for _ in range(W - 1):
        batch.run(check=False)
    stream = torch.cuda.current_stream(device)
    torch.cuda.synchronize(device)
    clocks = ClockSampler(device)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(K):
        batch.run(check=False)
    e1.record(stream)
    torch.cuda.synchronize(device)
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / K
    tf = flops / (ms * 1e-3) / 1e12
    res = batch.results()
    err = max(float(np.abs(res[i] - ref[i]).max() / np.abs(ref[i]).max()) for i in sample)
    # e2e: Gamma, chi from pinned host, solve, F back to pinned host
    hg = torch.from_numpy(batch.g_host).pin_memory()
    hc = torch.from_numpy(batch.c_host).pin_memory()
    ho = torch.empty_like(hg).pin_memory()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(K):
        batch.dg.copy_(hg, non_blocking=True)
        batch.dc.copy_(hc, non_blocking=True)
        batch.run(check=False)
        ho.copy_(batch.out, non_blocking=True)
    e3.record(stream)
    torch.cuda.synchronize(device)
    ms_e2e = e2.elapsed_time(e3) / K
    split = {}
    for sl in SPLIT_LU_SLICES:
        info = batch.run_split(slices=sl, tol=SPLIT_LU_TOL, max_refine=8)
        torch.cuda.synchronize(device)
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(K):
            batch.run_split(slices=sl, tol=SPLIT_LU_TOL, max_refine=8, check=False)
        s1.record(stream)
        torch.cuda.synchronize(device)
        ms_s = s0.elapsed_time(s1) / K
        res_s = batch.results()
        err_s = max(float(np.abs(res_s[i] - ref[i]).max() / np.abs(ref[i]).max()) for i in sample)
        split[str(sl)] = {"ms": ms_s, "effective_tflops": flops / (ms_s * 1e-3) / 1e12, "speedup_vs_fp64_lu": ms / ms_s,
                          "max_rel_err_vs_lapack": err_s, "refinements": int(info["refinements"].max()),
                          "max_rel_residual": float(info["residual"].max())}
    line = {"metric": "BSE TFLOP/s", "value": tf, "unit": "TFLOP/s", "n_gpus": ws, "steps": K, "warmup": W,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg,
            "roofline": {"kernel": "k_lu_batched", "bound": "tensor", "achieved": tf, "peak": peak64,
                         "unit": "TFLOP/s", "frac": tf / peak64, "traffic": None,
                         "peak_source": "FP64 cuBLAS ZGEMM 4096^3 measured in this run"},
            "max_rel_err_vs_lapack": err,
            "split_precision_refined": split,
            "split_note": ("tups_bse_lu_split_batched: LU and solve updates on s int8 slices (tcgen05), FP64 residual "
                           "Gamma - A F, corrections until max|residual| <= 1e-12 max|Gamma|; effective TFLOP/s = "
                           "the FP64 LU's algorithmic (8/3 + 8) n^3 / time"),
            "e2e": {"value": flops / (ms_e2e * 1e-3) / 1e12, "unit": "TFLOP/s",
                    "h2d_bytes_per_step": int(hg.numel() * 16 + hc.numel() * 16),
                    "d2h_bytes_per_step": int(ho.numel() * 16)},
            "gpu_launches": K, "clocks": clk, "cpu_baseline": cpu}
    if rank == 0:
        print(json.dumps(line), flush=True)


ZGEMM_WORKLOAD = "zgemm_split"


def run_zgemm_split(args):
    """Throughput of the split-precision batched ZGEMM (tups_zgemm_split)
    against cuBLAS ZGEMM at the BSE GEMM's shape: batched C_b = A_b B_b with
    M = N = Nz and K = 2 Nz ([Gamma chi | F] [F ; chi Gamma] for
    Nz = Nl * Nf).  Seeded random complex128 inputs, device-resident; CUDA
    events on the launching stream after one untimed call.  One JSON line with
    a record per slice count: effective FP64-equivalent TFLOP/s (8 M N K per
    entry), int8 tensor rate and the error against the FP64 product."""
    import ctypes as C
    import torch
    from tups_b200 import load
    ws_, rank, local = dist_env()
    if rank != 0:
        return
    lib = load()
    torch.cuda.set_device(local)
    Nz, batch, reps = args.nz, args.batch, max(1, args.steps)
    M = N = Nz
    K = 2 * Nz
    g = torch.Generator(device="cuda")
    g.manual_seed(1234)
    A = torch.randn((batch, K, M), dtype=torch.complex128, device="cuda", generator=g)
    B = torch.randn((batch, N, K), dtype=torch.complex128, device="cuda", generator=g)
    Cm = torch.zeros((batch, N, M), dtype=torch.complex128, device="cuda")
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    At, Bt = A.transpose(1, 2), B.transpose(1, 2)
    ref = torch.matmul(At[:1], Bt[:1])[0]

    def time_cublas() -> float:
        for _ in range(3):
            torch.matmul(At, Bt)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            torch.matmul(At, Bt)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    zgemm_ms = time_cublas()
    flops = 8.0 * M * N * K * batch
    out = {}
    lib.tups_set_split_cta_pairs(1 if args.cta_pairs else 0)
    for nt in args.n_tile:
        if lib.tups_set_split_tile(nt):
            raise RuntimeError(f"tups_set_split_tile({nt}) refused")
        for s in args.slices:
            wsz = lib.tups_zgemm_split_workspace(batch, M, N, K, s)
            work = torch.empty(wsz, dtype=torch.uint8, device="cuda")
            cargs = (batch, M, N, K, C.c_void_p(A.data_ptr()), C.c_void_p(B.data_ptr()), C.c_void_p(Cm.data_ptr()),
                     s, C.c_void_p(work.data_ptr()), wsz, C.c_void_p(stream.cuda_stream))
            rc = lib.tups_zgemm_split(*cargs)
            if rc:
                raise RuntimeError(f"tups_zgemm_split failed with {rc}")
            err = float((Cm[0].transpose(0, 1) - ref).abs().max() / ref.abs().max())
            torch.cuda.synchronize()
            e0.record()
            for _ in range(reps):
                lib.tups_zgemm_split(*cargs)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            pairs = s * (s + 1) // 2
            key = str(s) if len(args.n_tile) == 1 else f"{s}/n_tile={nt or 'auto'}"
            out[key] = {"ms": ms, "effective_tflops": flops / ms / 1e9,
                        "int8_tops": 2.0 * pairs * M * (2 * N) * (2 * K) * batch / ms / 1e9,
                        "rel_err_vs_fp64": err}
            del work
    lib.tups_set_split_tile(0)
    zgemm_ms = min(zgemm_ms, time_cublas())
    line = {"metric": "split ZGEMM effective TFLOP/s", "unit": "TFLOP/s", "workload": ZGEMM_WORKLOAD,
            "config": {"Nz": Nz, "batch": batch, "M": M, "N": N, "K": K, "cta_pairs": bool(args.cta_pairs)},
            "steps": reps,
            "cublas_zgemm_ms": zgemm_ms, "cublas_zgemm_tflops": flops / zgemm_ms / 1e9, "slices": out}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["tups", "reference"], default="tups")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + [LU_WORKLOAD, ZGEMM_WORKLOAD], default=DEFAULT_WORKLOAD)
    ap.add_argument("--nz", type=int, default=576, help="zgemm_split: M = N = Nz, K = 2 Nz")
    ap.add_argument("--batch", type=int, default=64, help="zgemm_split: batch entries")
    ap.add_argument("--slices", type=int, nargs="+", default=[2, 3, 4, 5, 6, 7, 8], help="zgemm_split: slice counts")
    ap.add_argument("--n-tile", type=int, nargs="+", default=[0],
                    help="zgemm_split: column tiles of the split GEMM to compare (0 = automatic)")
    ap.add_argument("--cta-pairs", action="store_true",
                    help="zgemm_split: run the split GEMM on CTA pairs (M = 256 tiles over two SMs)")
    ap.add_argument("--lu-q", type=int, default=64,
                    help="bse_lu_1024: momenta (x 16 frequencies = instances); fewer for a small profiling case")
    ap.add_argument("--crossing-products", type=int, default=0, choices=[0, 3, 4],
                    help="real tensor-core products per complex one in the crossing GEMM (0 = library default)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-split", action="store_true", help="skip the split-precision iterations")
    ap.add_argument("--no-graph", action="store_true", help="launch the timed iterations kernel by kernel")
    ap.add_argument("--bse-slices", type=int, default=0,
                    help="BSE GEMM of the main timed region on this many int8 slices (0 = FP64)")
    ap.add_argument("--no-convergence", action="store_true", help="skip the runs to convergence")
    ap.add_argument("--convergence", action="store_true",
                    help="also run the loops to convergence when Nz > 256 (minutes at 16x16)")
    ap.add_argument("--with-readout", action="store_true",
                    help="after the timed region, one output iteration with the chi readout")
    ap.add_argument("--no-target", action="store_true",
                    help="skip the 16x16 / 9 form factor FP64-vs-ladder record (about 6 minutes)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "tups":
        args.warmup = 3
    if args.workload == LU_WORKLOAD:
        run_bse_batched(args)
        return
    if args.workload == ZGEMM_WORKLOAD:
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the split ZGEMM has no CPU counterpart"}))
            return
        run_zgemm_split(args)
        return
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, args.workload, wl)
    else:
        run_tups(args, args.workload, wl)


if __name__ == "__main__":
    main()
